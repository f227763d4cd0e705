// C ABI of the FDTD core (include/afd.h): status codes and last-error
// strings around the C++ model and engine; no exception crosses it.
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/afd.h"
#include "engine.hpp"
#include "filters.hpp"
#include "geometry.hpp"
#include "model.hpp"

struct afd_model {
    afd::Model m;
    std::string err;
    // the last afd_model_boundary result (a model never changes after it is
    // made), so that the size query and the copy classify once
    std::vector<afd::BoundaryPoint> boundary;
    int32_t boundary_dev = -2;  // -1 host, >= 0 device ordinal, -2 none
};

struct afd_sim {
    std::unique_ptr<afd::Engine> eng;
    std::string err;
};

namespace {

template <typename F>
int guard(std::string& err, F&& f) {
    try {
        f();
        err.clear();
        return AFD_OK;
    } catch (const afd::Error& e) {
        err = e.what();
        return e.status;
    } catch (const std::bad_alloc&) {
        err = "out of host memory";
        return AFD_ERR_ARG;
    } catch (const std::exception& e) {
        err = e.what();
        return AFD_ERR_ARG;
    }
}

thread_local std::string g_create_error;

}  // namespace

extern "C" {

void afd_default_params(afd_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    // simulation.hpp:162-166 and main.cpp:118
    p->dx = 0.02f;
    p->c = 340.0f;
    p->dt = 3.125e-05f;
    p->fs = 32000.0f;
    p->mode = AFD_MODE_REF;
    p->storage = AFD_STORE_FP32;
    p->batch = 1;
    p->device = 0;
    p->watchdog = 1;
    p->graphs = 1;
    p->fused = 1;
    p->profile = 0;
}

const char* afd_version(void) { return "afd 0.1 (sm_100a)"; }

int afd_device_name(int32_t index, char* out, int64_t cap) {
    if (!out || cap < 1) return AFD_ERR_ARG;
    std::string name;
    const int st = afd::device_name(index, &name);
    if (st != AFD_OK) return st;
    std::strncpy(out, name.c_str(), (size_t)cap - 1);
    out[cap - 1] = '\0';
    return AFD_OK;
}

// ---- model ----------------------------------------------------------------
int afd_model_load_kerkythea(afd_model** out, const char* xml_path, float res) {
    if (!out || !xml_path) return AFD_ERR_ARG;
    *out = nullptr;
    std::unique_ptr<afd_model> m(new afd_model);
    int st = guard(g_create_error, [&] { m->m = afd::load_kerkythea(xml_path, res); });
    if (st != AFD_OK) return st;
    *out = m.release();
    return AFD_OK;
}

int afd_model_load_kerkythea_on(afd_model** out, const char* xml_path, float res, int32_t device) {
    if (!out || !xml_path) return AFD_ERR_ARG;
    *out = nullptr;
    std::unique_ptr<afd_model> m(new afd_model);
    int st = guard(g_create_error, [&] { m->m = afd::load_kerkythea_on(xml_path, res, device); });
    if (st != AFD_OK) return st;
    *out = m.release();
    return AFD_OK;
}

int afd_model_from_voxels(afd_model** out, int32_t nx, int32_t ny, int32_t nz, const int32_t* vox,
                          int32_t nmat, int32_t ncoef, const float* a, const float* b) {
    if (!out) return AFD_ERR_ARG;
    *out = nullptr;
    std::unique_ptr<afd_model> m(new afd_model);
    int st = guard(g_create_error, [&] {
        if (nx < 1 || ny < 1 || nz < 1 || !vox) throw afd::Error(AFD_ERR_ARG, "bad grid");
        if (nmat < 0 || ncoef < 0 || (nmat > 0 && (ncoef < 1 || !a || !b)))
            throw afd::Error(AFD_ERR_ARG, "bad material table");
        afd::Model& M = m->m;
        M.nx = nx;
        M.ny = ny;
        M.nz = nz;
        M.vox.assign(vox, vox + (size_t)nx * ny * nz);
        M.nmat = nmat;
        M.ncoef = nmat > 0 ? ncoef : 1;
        if (nmat > 0) {
            M.a.assign(a, a + (size_t)nmat * ncoef);
            M.b.assign(b, b + (size_t)nmat * ncoef);
        }
        for (int32_t k = 0; k < nmat; ++k) M.material_names.push_back("m" + std::to_string(k));
        for (int32_t v : M.vox)
            if (v < -1 || v >= nmat) throw afd::Error(AFD_ERR_ARG, "voxel material index out of range");
    });
    if (st != AFD_OK) return st;
    *out = m.release();
    return AFD_OK;
}

int afd_model_dims(const afd_model* m, int32_t dims[3], int32_t* nmat, int32_t* ncoef) {
    if (!m || !dims) return AFD_ERR_ARG;
    dims[0] = m->m.nx;
    dims[1] = m->m.ny;
    dims[2] = m->m.nz;
    if (nmat) *nmat = m->m.nmat;
    if (ncoef) *ncoef = m->m.ncoef;
    return AFD_OK;
}

int afd_model_voxels(const afd_model* m, int32_t* out, int64_t cap) {
    if (!m || !out) return AFD_ERR_ARG;
    if (cap < m->m.cells()) return AFD_ERR_ARG;
    std::memcpy(out, m->m.vox.data(), (size_t)m->m.cells() * sizeof(int32_t));
    return AFD_OK;
}

int afd_model_coefs(const afd_model* m, float* a, float* b, int64_t cap) {
    if (!m || !a || !b) return AFD_ERR_ARG;
    const size_t n = m->m.a.size();
    if ((size_t)cap < n) return AFD_ERR_ARG;
    std::memcpy(a, m->m.a.data(), n * sizeof(float));
    std::memcpy(b, m->m.b.data(), n * sizeof(float));
    return AFD_OK;
}

int afd_model_material_names(const afd_model* m, char* out, int64_t cap) {
    if (!m || !out || cap < 1) return AFD_ERR_ARG;
    std::string s;
    for (size_t k = 0; k < m->m.material_names.size(); ++k) {
        if (k) s += '\n';
        s += m->m.material_names[k];
    }
    if ((int64_t)s.size() + 1 > cap) return AFD_ERR_ARG;
    std::memcpy(out, s.c_str(), s.size() + 1);
    return AFD_OK;
}

int afd_model_classify(const afd_model* m, int64_t counts[AFD_NUM_GROUPS]) {
    if (!m || !counts) return AFD_ERR_ARG;
    afd_model* mm = const_cast<afd_model*>(m);
    return guard(mm->err, [&] {
        std::vector<afd::BoundaryPoint> pts = afd::classify(m->m);
        for (int g = 0; g < AFD_NUM_GROUPS; ++g) counts[g] = 0;
        for (auto& p : pts) counts[p.group]++;
    });
}

int afd_model_group_points(const afd_model* m, int32_t group, int32_t* out, int64_t cap,
                           int64_t* n_out) {
    if (!m || group < 0 || group >= AFD_NUM_GROUPS) return AFD_ERR_ARG;
    afd_model* mm = const_cast<afd_model*>(m);
    return guard(mm->err, [&] {
        std::vector<afd::BoundaryPoint> pts = afd::classify(m->m);
        int64_t n = 0;
        for (auto& p : pts) {
            if (p.group != group) continue;
            if (out) {
                if ((n + 1) * 6 > cap) throw afd::Error(AFD_ERR_ARG, "output buffer too small");
                int32_t* o = out + n * 6;
                o[0] = p.x;
                o[1] = p.y;
                o[2] = p.z;
                o[3] = p.mat[0];
                o[4] = p.mat[1];
                o[5] = p.mat[2];
            }
            ++n;
        }
        if (n_out) *n_out = n;
    });
}

int afd_model_boundary(const afd_model* m, int32_t device, int32_t* out, int64_t cap, int64_t* n_out) {
    if (!m) return AFD_ERR_ARG;
    afd_model* mm = const_cast<afd_model*>(m);
    return guard(mm->err, [&] {
        const int32_t key = device < 0 ? -1 : device;
        if (mm->boundary_dev != key) {
            mm->boundary_dev = -2;
            mm->boundary = key < 0 ? afd::classify(m->m) : afd::classify_on(m->m, key);
            mm->boundary_dev = key;
        }
        const std::vector<afd::BoundaryPoint>& pts = mm->boundary;
        const int64_t n = (int64_t)pts.size();
        if (out) {
            if (n * 7 > cap) throw afd::Error(AFD_ERR_ARG, "output buffer too small");
            std::memcpy(out, pts.data(), (size_t)n * sizeof(afd::BoundaryPoint));
        }
        if (n_out) *n_out = n;
    });
}

const char* afd_model_last_error(const afd_model* m) {
    return m ? m->err.c_str() : g_create_error.c_str();
}

void afd_model_destroy(afd_model* m) { delete m; }

int afd_check_filters(int32_t nmat, int32_t ncoef, const double* a, const double* b, int32_t n_freq,
                      int32_t* status, double* min_real, double* max_root) {
    if (nmat < 1 || ncoef < 1 || !a || !b || n_freq < 2 || !status) return AFD_ERR_ARG;
    return guard(g_create_error, [&] {
        afd::check_filters(nmat, ncoef, a, b, n_freq, status, min_real, max_root);
    });
}

int afd_check_filters_static(int32_t nmat, int32_t ncoef, const double* a, const double* b, int32_t n_freq,
                             int32_t* status, double* min_real, double* max_root) {
    if (nmat < 1 || ncoef < 1 || !a || !b || n_freq < 2 || !status) return AFD_ERR_ARG;
    return guard(g_create_error, [&] {
        afd::check_filters_static(nmat, ncoef, a, b, n_freq, status, min_real, max_root);
    });
}

// ---- simulation -------------------------------------------------------------
int afd_create(afd_sim** out, const afd_params* p) {
    if (!out) return AFD_ERR_ARG;
    *out = nullptr;
    afd_params prm;
    if (p) prm = *p;
    else afd_default_params(&prm);
    std::unique_ptr<afd_sim> s(new afd_sim);
    int st = guard(g_create_error, [&] { s->eng.reset(new afd::Engine(prm)); });
    if (st != AFD_OK) return st;
    *out = s.release();
    return AFD_OK;
}

#define SIM_CALL(s, body)                                   \
    do {                                                    \
        if (!(s)) return AFD_ERR_ARG;                       \
        return guard((s)->err, [&] { body; });              \
    } while (0)

int afd_set_min_size(afd_sim* s, float x, float y, float z) { SIM_CALL(s, s->eng->set_min_size(x, y, z)); }

int afd_load(afd_sim* s, const char* xml_path) {
    SIM_CALL(s, {
        if (!xml_path) throw afd::Error(AFD_ERR_ARG, "null path");
        // Simulation::Load uses res_ = 0.02 from the constructor; here the
        // cell size is params.dx.
        s->eng->load_kerkythea(xml_path);
    });
}

int afd_set_model(afd_sim* s, const afd_model* m) {
    SIM_CALL(s, {
        if (!m) throw afd::Error(AFD_ERR_ARG, "null model");
        s->eng->set_model(m->m);
    });
}

int afd_set_pml(afd_sim* s, int32_t width, uint32_t face_mask, const float* kx, const float* ky,
                const float* kz) {
    SIM_CALL(s, s->eng->set_pml(width, face_mask, kx, ky, kz));
}

int afd_set_pml_profile(afd_sim* s, int32_t width, const float* prof, int32_t len) {
    SIM_CALL(s, s->eng->set_pml_profile(width, prof, len));
}

int afd_add_source(afd_sim* s, int32_t batch, const float pos[3], const float* sig, int64_t len) {
    SIM_CALL(s, {
        if (!pos) throw afd::Error(AFD_ERR_ARG, "null position");
        s->eng->add_source_pos(batch, pos, sig, len);
    });
}

int afd_add_source_cell(afd_sim* s, int32_t batch, const int32_t ijk[3], const float* sig, int64_t len) {
    SIM_CALL(s, {
        if (!ijk) throw afd::Error(AFD_ERR_ARG, "null cell");
        s->eng->add_source_cell(batch, ijk, sig, len);
    });
}

int afd_add_receiver(afd_sim* s, const float pos[3]) {
    SIM_CALL(s, {
        if (!pos) throw afd::Error(AFD_ERR_ARG, "null position");
        s->eng->add_receiver_pos(pos);
    });
}

int afd_add_receiver_cell(afd_sim* s, const int32_t ijk[3]) {
    SIM_CALL(s, {
        if (!ijk) throw afd::Error(AFD_ERR_ARG, "null cell");
        s->eng->add_receiver_cell(ijk);
    });
}

int afd_run(afd_sim* s, int64_t steps, afd_progress_fn cb, void* user) {
    if (!s) return AFD_ERR_ARG;
    int status = AFD_OK;
    int st = guard(s->err, [&] { status = s->eng->run(steps, cb, user); });
    if (st != AFD_OK) return st;
    if (status != AFD_OK) s->err = "run stopped by the progress callback";
    return status;
}

int afd_set_capture(afd_sim* s, int32_t batch, int32_t axis, int32_t index, int32_t every, int32_t max_frames) {
    SIM_CALL(s, { s->eng->set_capture(batch, axis, index, every, max_frames); });
}

int afd_set_timeline(afd_sim* s, int64_t first, int32_t steps) {
    SIM_CALL(s, { s->eng->set_timeline(first, steps); });
}

int afd_get_timeline(afd_sim* s, double* out, int64_t cap, int32_t* n_steps) {
    SIM_CALL(s, {
        const int32_t n = s->eng->get_timeline(out, cap);
        if (n_steps) *n_steps = n;
    });
}

int afd_get_frames(afd_sim* s, float* out, int64_t cap, int64_t* steps, int64_t steps_cap, int32_t* n_frames) {
    SIM_CALL(s, {
        const int32_t n = s->eng->get_frames(out, cap, steps, steps_cap);
        if (n_frames) *n_frames = n;
    });
}

int afd_prepare(afd_sim* s, int64_t steps) {
    SIM_CALL(s, { s->eng->prepare(steps); });
}

int afd_get_receivers(afd_sim* s, int32_t batch, float* out, int64_t cap) {
    SIM_CALL(s, {
        if (!out && cap > 0) throw afd::Error(AFD_ERR_ARG, "null output");
        s->eng->get_receivers(batch, out, cap);
    });
}

int afd_update_source(afd_sim* s, int64_t index, int64_t t0, const float* sig, int64_t len) {
    SIM_CALL(s, {
        if (len < 0 || (len > 0 && !sig)) throw afd::Error(AFD_ERR_ARG, "bad signal");
        s->eng->update_source(index, t0, sig, len);
    });
}

int afd_get_receivers_range(afd_sim* s, int32_t batch, int64_t t0, int64_t t1, float* out, int64_t cap) {
    SIM_CALL(s, {
        if (!out && cap > 0) throw afd::Error(AFD_ERR_ARG, "null output");
        s->eng->get_receivers_range(batch, t0, t1, out, cap);
    });
}

int afd_get_field(afd_sim* s, int32_t batch, float* out, int64_t cap) {
    SIM_CALL(s, {
        if (!out) throw afd::Error(AFD_ERR_ARG, "null output");
        s->eng->get_field(batch, out, cap);
    });
}

int afd_get_plane(afd_sim* s, int32_t batch, int32_t axis, int32_t index, float* out, int64_t cap) {
    SIM_CALL(s, {
        if (!out) throw afd::Error(AFD_ERR_ARG, "null output");
        s->eng->get_plane(batch, axis, index, out, cap);
    });
}

int afd_get_info(afd_sim* s, afd_info* info) {
    SIM_CALL(s, {
        if (!info) throw afd::Error(AFD_ERR_ARG, "null info");
        s->eng->get_info(info);
    });
}

int afd_energy(afd_sim* s, int32_t batch, double* energy) {
    SIM_CALL(s, {
        if (!energy) throw afd::Error(AFD_ERR_ARG, "null output");
        *energy = s->eng->energy(batch);
    });
}

int afd_set_stream(afd_sim* s, void* stream) { SIM_CALL(s, s->eng->set_stream(stream)); }

int afd_set_plan(afd_sim* s, const afd_plan* plan) { SIM_CALL(s, s->eng->set_plan(plan)); }

int afd_set_slab(afd_sim* s, int32_t z_offset, int32_t nz_global) {
    SIM_CALL(s, s->eng->set_slab(z_offset, nz_global));
}

int afd_step_phase(afd_sim* s, int32_t phase) { SIM_CALL(s, s->eng->step(phase)); }

int afd_halo(afd_sim* s, int32_t side, int32_t dir, int32_t field, void* dev, int64_t cap) {
    SIM_CALL(s, s->eng->halo(side, dir, field, dev, cap));
}

int afd_kernel_stats(afd_sim* s, int32_t idx, char* name, int64_t cap, int64_t* launches, double* ms) {
    if (!s) return AFD_ERR_ARG;
    return s->eng->kernel_stats(idx, name, cap, launches, ms);
}

const char* afd_last_error(const afd_sim* s) { return s ? s->err.c_str() : g_create_error.c_str(); }

void afd_destroy(afd_sim* s) { delete s; }

}  // extern "C"
