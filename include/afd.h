/*
 * afd.h - C ABI of the B200 acoustic FDTD core (anc-field drop-in).
 *
 * Two handle types:
 *   afd_model  host-only geometry: Kerkythea XML -> int32 voxel grid plus
 *              per-material admittance filter coefficients, and the
 *              boundary (LRS) classification. Needs no GPU.
 *   afd_sim    one simulation on one CUDA device: pressure fields, boundary
 *              filter state, PML fields, sources, receivers, the step loop.
 *
 * Conventions
 *   - Every call returns an int status: AFD_OK (0) or a negative AFD_ERR_*.
 *     The message of the last failure is afd_last_error() /
 *     afd_model_last_error(). No C++ exception crosses this boundary.
 *   - The library copies every input; outputs go into caller buffers whose
 *     capacity (in elements) is passed as `cap`.
 *   - Grids are x-fastest: index(x,y,z) = (z*ny + y)*nx + x, as the
 *     reference's clh macros define it (anc-field/clh/clh-kernel.hpp:238-248).
 *   - One handle per host thread. Calls are synchronous.
 *
 * Reference interfaces replaced (paths inside szarvas/anc-field):
 *   Simulation class   anc-field/src/simulation.hpp:83-156
 *   Kerkythea loader   anc-field/src/kerkythea.hpp:133-196
 *   LrsData            anc-field/src/lrs-data.hpp:116-215
 *   clh::Kernel launch anc-field/clh/clh-kernel.hpp:163-183
 */
#ifndef AFD_H
#define AFD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AFD_OK              0
#define AFD_ERR_ARG        -1  /* bad argument, size or index */
#define AFD_ERR_STATE      -2  /* call not valid in the current state */
#define AFD_ERR_IO         -3  /* file missing or unparsable */
#define AFD_ERR_GEOMETRY   -4  /* unphysical surfaces (lrs-data.hpp:327) */
#define AFD_ERR_CUDA       -5  /* CUDA runtime failure or no device */
#define AFD_ERR_NUMERIC    -6  /* watchdog: a pressure value left the finite bound */
#define AFD_ERR_FILTER     -7  /* filter stability / passivity check failed */
#define AFD_ERR_ABORTED    -8  /* the progress callback asked to stop */

/* Boundary update semantics. */
#define AFD_MODE_REF    0  /* the reference kernels' arithmetic, quirks included */
#define AFD_MODE_FIXED  1  /* the intended scheme: quirks of the reference removed */

/* Field storage precision. */
#define AFD_STORE_FP32  0
#define AFD_STORE_FP16  1

/* PML face bits (FIXED mode; REF mode always uses all six ends). */
#define AFD_FACE_XM 1u
#define AFD_FACE_XP 2u
#define AFD_FACE_YM 4u
#define AFD_FACE_YP 8u
#define AFD_FACE_ZM 16u
#define AFD_FACE_ZP 32u

/* The 26 boundary groups, numbered as lrs-data.hpp:53-78 numbers them. */
#define AFD_NUM_GROUPS 26

typedef struct afd_params {
    float dx;          /* cell size in metres; also the position->cell divisor (ref 0.02) */
    float c;           /* speed of sound, m/s (ref 340) */
    float dt;          /* time step, s (ref 3.125e-5) */
    float fs;          /* samples per second used by run-in-seconds callers (ref 32000) */
    int32_t mode;      /* AFD_MODE_REF or AFD_MODE_FIXED */
    int32_t storage;   /* AFD_STORE_FP32 or AFD_STORE_FP16 */
    int32_t batch;     /* independent source sets sharing one geometry (>= 1) */
    int32_t device;    /* CUDA device ordinal */
    int32_t watchdog;  /* nonzero: stop a run whose field leaves |p| < 1e30 */
    int32_t graphs;    /* nonzero: replay captured CUDA graphs of step chunks */
    int32_t fused;     /* nonzero: one fused kernel per step; zero: one launch per sub-step */
    int32_t profile;   /* nonzero: time every kernel launch with CUDA events (no graphs) */
    int32_t reserved[4];
} afd_params;

/* Fills the reference constants: dx=0.02, c=340, dt=3.125e-5, fs=32000,
 * REF mode, FP32, batch 1, device 0, watchdog on, graphs on, fused on. */
void afd_default_params(afd_params* p);

/* Version string of the library build. */
const char* afd_version(void);

/* Name of CUDA device `index` (the `lsd` listing, main.cpp:38-50).
 * Returns AFD_ERR_ARG past the last device, AFD_ERR_CUDA without one. */
int afd_device_name(int32_t index, char* out, int64_t cap);

/* ------------------------------------------------------------------ */
/* Host-only geometry                                                  */
/* ------------------------------------------------------------------ */
typedef struct afd_model afd_model;

/* Kerkythea XML -> voxels + filters (replaces kerkythea.hpp:133-196 and
 * LoadBoxes kerkythea.hpp:63-130). Material files <dir>/<name>_a.dat and
 * _b.dat are read next to the XML, one coefficient per line. */
int afd_model_load_kerkythea(afd_model** out, const char* xml_path, float res);

/* The same loader with the rasterisation (kerkythea.hpp:180-195) on CUDA
 * device `device`: the same model, voxel for voxel. afd_load uses this form
 * on the simulation's device. */
int afd_model_load_kerkythea_on(afd_model** out, const char* xml_path, float res, int32_t device);

/* Builds a model from a caller voxel grid (-1 air, else material index)
 * and per-material coefficients a[nmat][ncoef], b[nmat][ncoef]. */
int afd_model_from_voxels(afd_model** out, int32_t nx, int32_t ny, int32_t nz,
                          const int32_t* vox, int32_t nmat, int32_t ncoef,
                          const float* a, const float* b);

/* dims[3] = {nx, ny, nz}; nmat, ncoef may be NULL. */
int afd_model_dims(const afd_model* m, int32_t dims[3], int32_t* nmat, int32_t* ncoef);
int afd_model_voxels(const afd_model* m, int32_t* out, int64_t cap);
/* a and b each receive nmat*ncoef floats, material order = sorted names. */
int afd_model_coefs(const afd_model* m, float* a, float* b, int64_t cap);
/* Material names joined by '\n' (sorted as std::set sorts them). */
int afd_model_material_names(const afd_model* m, char* out, int64_t cap);

/* Boundary classification of lrs-data.hpp:116-215: counts[g] = number of
 * air cells in group g. Fails with AFD_ERR_GEOMETRY on an unphysical
 * pattern (opposite solid neighbours or more than three). */
int afd_model_classify(const afd_model* m, int64_t counts[AFD_NUM_GROUPS]);
/* Per-group point list {x,y,z,mat0,mat1,mat2} (unused mats = -1), in the
 * reference's z-y-x scan order. n_out receives the point count. */
int afd_model_group_points(const afd_model* m, int32_t group, int32_t* out,
                           int64_t cap, int64_t* n_out);
/* The whole boundary list of lrs-data.hpp:154-210 as rows {x, y, z, group,
 * mat0, mat1, mat2} in z-y-x scan order; cap counts int32 values, out may be
 * NULL to query n_out. device < 0 classifies on the host, device >= 0 on that
 * CUDA device (the classifier afd_set_model and afd_load run), with the same
 * list, or the same AFD_ERR_GEOMETRY message naming the same cell. */
int afd_model_boundary(const afd_model* m, int32_t device, int32_t* out, int64_t cap,
                       int64_t* n_out);

const char* afd_model_last_error(const afd_model* m);
void afd_model_destroy(afd_model* m);

/* FP64 admittance-filter check, a coefficient check made once before a
 * run (not part of the step): on the GPU when one is present; without a CUDA
 * device the same FP64 arithmetic runs on the host, so that models can be
 * checked on machines without a GPU. Stability = every root of b(z) (the recursion's
 * denominator, coefficient order b0 + b1 z^-1 + ...) inside |z| < 1 - margin;
 * passivity = Re{A(e^jw)/B(e^jw)} >= 0 on n_freq uniformly spaced
 * frequencies in [0, pi]. status[i] bit0 = unstable, bit1 = not passive.
 * min_real[i] receives the minimum real part found. */
int afd_check_filters(int32_t nmat, int32_t ncoef, const double* a, const double* b,
                      int32_t n_freq, int32_t* status, double* min_real, double* max_root);

/* No counterpart in the reference. The same check as afd_check_filters for
 * callers that must not allocate device memory (a process held to a fixed
 * GPU memory budget by its host application, or a setup path that re-checks
 * coefficients after simulations have taken the rest of the device, where a
 * cudaMalloc could fail): its scratch is one file-scope device array of 64
 * materials x 16 coefficients (about 21 KB, held by every device that loads
 * the library until exit). Sizes beyond that return AFD_ERR_ARG. Needs a
 * CUDA device. Each call looks up the array's address with the device
 * current (valid after a cudaDeviceReset too); the first call on a device
 * loads the module there, so make it before any stream capture. The copies
 * are synchronous and the kernels run on the legacy default stream: a call
 * waits for work on the device's blocking streams. All calls share the
 * array: calls that overlap on the GPU race, so the caller serialises them.
 * The error text is afd_model_last_error(NULL). */
int afd_check_filters_static(int32_t nmat, int32_t ncoef, const double* a, const double* b,
                             int32_t n_freq, int32_t* status, double* min_real, double* max_root);

/* ------------------------------------------------------------------ */
/* Simulation                                                          */
/* ------------------------------------------------------------------ */
typedef struct afd_sim afd_sim;

/* Progress callback, called on the calling thread after step i (0-based,
 * run-local) when i == 0 and every 200 steps, and once more with
 * i == steps at the end (simulation.hpp:403-409, 433). A nonzero return
 * stops the run with AFD_ERR_ABORTED after the current chunk. */
typedef int (*afd_progress_fn)(int64_t i, int64_t steps, void* user);

/* Replaces Simulation::Simulation (simulation.hpp:158-171). */
int afd_create(afd_sim** out, const afd_params* p);

/* Replaces Simulation::SetMinSize (simulation.hpp:279-284): each edge
 * becomes RoundTo((int)(len/dx)+1, 32); the grid is the per-axis maximum
 * of this and the model grid. */
int afd_set_min_size(afd_sim* s, float x_m, float y_m, float z_m);

/* Replaces Simulation::Load (simulation.hpp:173-199). */
int afd_load(afd_sim* s, const char* xml_path);
/* Same, from a model built by afd_model_* (the model is copied). */
int afd_set_model(afd_sim* s, const afd_model* m);

/* Replaces Simulation::SetPml (simulation.hpp:233-277). ksi_x/y/z hold nx,
 * ny, nz damping values (1/s). REF mode: the whole interior 2..N-3 is
 * updated by the PML kernel and the auxiliary fields in the end slabs of
 * `width` cells (pml.cl:182, 231-262); face_mask is ignored. FIXED mode:
 * only non-boundary air cells inside the slabs of the faces in face_mask.
 * width 0 disables the PML. */
int afd_set_pml(afd_sim* s, int32_t width, uint32_t face_mask,
                const float* ksi_x, const float* ksi_y, const float* ksi_z);
/* Builds the reference ksi arrays from a profile file's values as
 * SetPml does (ksi[i] = ksi[n-1-i] = prof[L-1-i], i < L) and sets them. */
int afd_set_pml_profile(afd_sim* s, int32_t width, const float* prof, int32_t len);

/* Replaces Simulation::AddSource (simulation.hpp:309-324): the cell is
 * (int)(pos/dx) per axis. Samples past len are zero. batch selects the
 * source set (0 .. params.batch-1). */
int afd_add_source(afd_sim* s, int32_t batch, const float pos_m[3],
                   const float* signal, int64_t len);
int afd_add_source_cell(afd_sim* s, int32_t batch, const int32_t ijk[3],
                        const float* signal, int64_t len);

/* Replaces Simulation::AddMic (simulation.hpp:326-340). Receivers are
 * shared by every batch member. */
int afd_add_receiver(afd_sim* s, const float pos_m[3]);
int afd_add_receiver_cell(afd_sim* s, const int32_t ijk[3]);

/* Replaces Simulation::Run (simulation.hpp:342-434): advances `steps`
 * time steps; the time index continues across runs. */
int afd_run(afd_sim* s, int64_t steps, afd_progress_fn cb, void* user);

/* No counterpart in the reference: does the setup work of
 * afd_run(s, steps, ...) without running a step (device buffers, uploads,
 * the CUDA graphs of the run's chunks), so that a caller timing the run on
 * the device measures only the steps. */
int afd_prepare(afd_sim* s, int64_t steps);

/* Receiver signals of one batch member, [n_receivers][t_end] row-major,
 * t_end = total steps run so far (the `save` layout, datafile.hpp:87-94). */
int afd_get_receivers(afd_sim* s, int32_t batch, float* out, int64_t cap);

/* Streaming variants for callers that feed and drain a long run in parts:
 * replaces the samples of source `index` (insertion order over all batch
 * members) from time index t0 on (the signal grows when needed), and copies
 * receiver samples t0 .. t1-1 of one batch member into out[n_receivers][t1-t0].
 * Replace the clh host/device sync of simulation.hpp:95 and source.cl's
 * argument upload for long runs split into parts. */
int afd_update_source(afd_sim* s, int64_t index, int64_t t0, const float* signal, int64_t len);
int afd_get_receivers_range(afd_sim* s, int32_t batch, int64_t t0, int64_t t1, float* out, int64_t cap);

/* The latest pressure field p^n of one batch member, dense [nz][ny][nx]. */
int afd_get_field(afd_sim* s, int32_t batch, float* out, int64_t cap);
/* Headless 'vis': one plane of p^n (copy_plane.cl:29-34 takes axis 1).
 * axis 0: out[nz][ny] at x=index; axis 1: out[nz][nx] at y=index;
 * axis 2: out[ny][nx] at z=index. */
int afd_get_plane(afd_sim* s, int32_t batch, int32_t axis, int32_t index,
                  float* out, int64_t cap);

/* Headless visualisation, replacing the copy of the newest level's y plane
 * after every third step of a run for the MJPEG stream
 * (simulation.hpp:393-400, copy_plane.cl:29-34): from the next run on, the
 * plane of afd_get_plane(batch, axis, index) is copied on the device after
 * every step whose index within the run is a multiple of `every`, into a
 * ring of max_frames frames. every <= 0 turns it off. */
int afd_set_capture(afd_sim* s, int32_t batch, int32_t axis, int32_t index, int32_t every,
                    int32_t max_frames);
/* The captured frames, oldest first: out[n][rows][cols] (the afd_get_plane
 * layout), steps[n] the global step after which each was taken (either
 * pointer may be NULL); *n_frames receives n <= max_frames. */
int afd_get_frames(afd_sim* s, float* out, int64_t cap, int64_t* steps, int64_t steps_cap,
                   int32_t* n_frames);

/* Step timeline (measurement, no reference counterpart): from the next run
 * on, the kernels of global steps first .. first+steps-1 record on the
 * device (%globaltimer) the start of their first block and the end of their
 * last block, for AFD_TIMELINE_SLOTS kernel kinds: 0 streaming or interior
 * kernel, 1 boundary (LRS) kernel, 2 PML pressure, 3/4/5 PML auxiliary
 * update of fi_x/fi_y/fi_z, 6 source/receiver kernel. Kernels with one block
 * column per batch member record member 0's blocks. steps <= 0 turns it
 * off; at most 4096 steps. */
#define AFD_TIMELINE_SLOTS 7
int afd_set_timeline(afd_sim* s, int64_t first, int32_t steps);
/* The recorded timeline: out[steps][AFD_TIMELINE_SLOTS][2] (start, end) in
 * nanoseconds from the earliest recorded start, -1 where a kind did not run
 * at a step; cap >= 2 * steps * AFD_TIMELINE_SLOTS; *n_steps receives the
 * number of steps (0 when no timeline is armed). */
int afd_get_timeline(afd_sim* s, double* out, int64_t cap, int32_t* n_steps);

typedef struct afd_info {
    int32_t nx, ny, nz;          /* simulation grid */
    int32_t ncoef, nmat;
    int32_t batch;
    int64_t steps_done;          /* global time index */
    int64_t n_sources, n_receivers;
    int64_t n_boundary;          /* LRS points, all groups */
    int64_t group_counts[AFD_NUM_GROUPS];
    int64_t n_pml_cells;         /* FIXED: cells with the PML update */
    float lambda2;               /* (dt*c/dx)^2 in FP32 */
    int32_t mode, storage;
    double last_run_ms;          /* device time of the last afd_run (CUDA events) */
    int64_t kernel_launches;     /* kernels launched by the last afd_run */
    int32_t tile_x, tile_y, tile_z;  /* tile (cells) and z-chunk depth of the streaming kernel's plan */
    int32_t stream_blocks;       /* resident blocks of the streaming kernel's plan */
    int32_t tuned;               /* 1 once the online autotuner has chosen the plan */
    int32_t stream_beside;       /* 1: the plan runs the boundary and PML kernels beside the streaming kernel */
    int32_t stream_per_sm;       /* resident streaming blocks per SM of the plan */
    int32_t stream_tail;         /* 1: the plan does the boundary and PML pressure work in the streaming kernel */
    int32_t reserved[4];
} afd_info;
int afd_get_info(afd_sim* s, afd_info* info);

/* Discrete energy of the SLF scheme, accumulated in FP64 on the GPU:
 * kinetic + potential terms between the two latest time levels, over the air
 * cells 1..n-2 and the edges between air cells. A cell with walls (solid
 * neighbours) counts 1/2 per walled axis, an edge 1/2 per other axis on which
 * both ends have the same wall; without a model every weight is 1. Constant
 * for rigid walls and non-increasing for passive walls (constant admittance
 * >= 0) around a box-shaped room without PML. */
int afd_energy(afd_sim* s, int32_t batch, double* energy);

/* Runs the simulation's work on the caller's CUDA stream (a cudaStream_t
 * passed as void*), e.g. so that the caller can bracket afd_run with its own
 * CUDA events. NULL restores the library's own stream. */
int afd_set_stream(afd_sim* s, void* stream);

/* A streaming-kernel plan (the autotuner's search space). Zero fields take
 * the default: the 64x16 tile, as many resident blocks per SM as fit, the
 * z-chunk depth rule. beside = 1 runs the boundary and PML pressure kernels
 * beside the streaming kernel, which then skips their cells (FIXED scheme
 * with CUDA graphs; ignored elsewhere). The autotuner tries neither the
 * beside nor the tail order (both measured slower). */
typedef struct afd_plan {
    int32_t tile_x, tile_y;  /* streaming tile in cells: 64x16, 128x8 or 32x32 (FP16 storage doubles x) */
    int32_t per_sm;          /* resident streaming blocks per SM */
    int32_t dz;              /* planes per z-chunk work item (1..1024) */
    int32_t beside;
    int32_t tail;            /* 1: the boundary and PML pressure work in the streaming kernel's tail warps
                                (FIXED scheme, FP32 storage; ignored elsewhere) */
    int32_t reserved[2];
} afd_plan;

/* Fixes the streaming plan of later runs and turns the online autotuner off
 * for this simulation (no counterpart in the reference, whose kernels have
 * one launch shape: clh-kernel.hpp:163-183). NULL gives the plan back to the
 * autotuner, which tries its candidates again. Every plan gives the same
 * receivers bit for bit, and the same pressure at every cell an air cell
 * reads; the 32x32 tile leaves out work items whose region holds no air, so
 * solid cells more than one cell from air keep older values there. */
int afd_set_plan(afd_sim* s, const afd_plan* plan);

/* z-slab domain decomposition (no counterpart in the reference, which runs
 * one device: simulation.hpp:176-178, 356-402). The simulation's grid is
 * global planes z_offset .. z_offset+nz-1 of a grid of nz_global planes:
 * its planes 0 and nz-1 are halos (or the global end faces) that the caller
 * fills from the neighbouring slabs, its planes 1..nz-2 are its own; the
 * PML cell rule and the z slabs of the PML use global planes. FIXED scheme
 * and FP32 storage only. nz_global = 0 turns it off. */
int afd_set_slab(afd_sim* s, int32_t z_offset, int32_t nz_global);

/* One half of the next time step, launched in the serial order (no graphs):
 * phase 1 the interior, boundary and PML pressure updates; phase 2 the PML
 * auxiliary updates, sources, receivers and capture, which completes the
 * step. A slab run refreshes the high-z halo of the new pressure (and psi)
 * between the phases, where the auxiliary update of its last plane reads
 * it, and both halos of the new pressure and the new auxiliary fields after
 * phase 2. Call afd_prepare(total steps) first to size the receiver record.
 * Synchronous. */
int afd_step_phase(afd_sim* s, int32_t phase);

/* Copies one plane of every batch member between the simulation and the
 * caller's device buffer dev ([batch][ny][pitch] floats, pitch = nx rounded
 * up to 32; cap in floats). side 0: the low-z end, 1: the high-z end. dir 0
 * reads the outermost own plane of that end (local 1 or nz-2) into dev,
 * dir 1 writes dev into the halo plane (local 0 or nz-1). field 0: the
 * pressure level of the open (after phase 1) or last completed step;
 * 1, 2, 3: that step's new PML auxiliary field of axis x, y, z; 4: its new
 * psi. Synchronous. */
int afd_halo(afd_sim* s, int32_t side, int32_t dir, int32_t field, void* dev, int64_t cap);

/* Per-kernel statistics of the last afd_run made with params.profile set:
 * kernel idx (0-based) -> name, launches and summed device milliseconds.
 * Returns AFD_ERR_ARG when idx is past the last kernel. */
int afd_kernel_stats(afd_sim* s, int32_t idx, char* name, int64_t cap,
                     int64_t* launches, double* ms);

/* Self-test of the bounded device waits (no reference counterpart): one
 * block on `device` waits on a shared-memory mbarrier with the streaming
 * kernel's wait (which = 0) or the tensor-core GEMM kernels' wait
 * (which = 1). complete = 0 leaves the barrier incomplete, so the wait gives
 * up at its 2 s limit instead of hanging; *timed_out receives 1 when it gave
 * up, *waited_ns the device time it waited. The kernel returns normally
 * either way and the context stays usable. */
int afd_wait_selftest(int32_t device, int32_t which, int32_t complete, int32_t* timed_out,
                      int64_t* waited_ns);

const char* afd_last_error(const afd_sim* s);
void afd_destroy(afd_sim* s);

#ifdef __cplusplus
}
#endif

#endif /* AFD_H */
