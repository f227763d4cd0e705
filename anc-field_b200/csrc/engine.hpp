// The simulation engine behind the C ABI: owns device memory, builds the
// compact boundary/PML/source/receiver lists and runs the step loop.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/afd.h"
#include "model.hpp"

namespace afd {

struct KernelStat {
    std::string name;
    int64_t launches = 0;
    double ms = 0.0;
};

class Engine {
public:
    explicit Engine(const afd_params& p);
    ~Engine();

    void set_min_size(float x, float y, float z);
    void set_model(const Model& m);
    void load_kerkythea(const std::string& xml_path);
    void set_pml(int32_t width, uint32_t faces, const float* kx, const float* ky, const float* kz);
    void set_pml_profile(int32_t width, const float* prof, int32_t len);
    void add_source_cell(int32_t batch, const int32_t ijk[3], const float* sig, int64_t len);
    void add_source_pos(int32_t batch, const float pos[3], const float* sig, int64_t len);
    void add_receiver_cell(const int32_t ijk[3]);
    void add_receiver_pos(const float pos[3]);
    int run(int64_t steps, afd_progress_fn cb, void* user);
    void prepare(int64_t steps);
    void get_receivers(int32_t batch, float* out, int64_t cap);
    void get_receivers_range(int32_t batch, int64_t t0, int64_t t1, float* out, int64_t cap);
    void update_source(int64_t index, int64_t t0, const float* sig, int64_t len);
    void get_field(int32_t batch, float* out, int64_t cap);
    void get_plane(int32_t batch, int32_t axis, int32_t index, float* out, int64_t cap);
    void set_capture(int32_t batch, int32_t axis, int32_t index, int32_t every, int32_t max_frames);
    int32_t get_frames(float* out, int64_t cap, int64_t* steps, int64_t steps_cap);
    void set_timeline(int64_t first, int32_t steps);
    int32_t get_timeline(double* out, int64_t cap);
    void get_info(afd_info* info);
    double energy(int32_t batch);
    void set_stream(void* stream);
    void set_plan(const afd_plan* plan);
    void set_slab(int32_t z_offset, int32_t nz_global);
    void step(int32_t phase);
    void halo(int32_t side, int32_t dir, int32_t field, void* dev, int64_t cap);
    float cell_size() const;
    int kernel_stats(int32_t idx, char* name, int64_t cap, int64_t* launches, double* ms);

    std::string last_error;
    struct Impl;

private:
    std::unique_ptr<Impl> d_;
};

}  // namespace afd
