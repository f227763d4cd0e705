// Geometry set-up on the GPU: the rasterisation loop of the Kerkythea
// constructor (anc-field/src/kerkythea.hpp:180-195) and the boundary
// classification of LrsData::Init (anc-field/src/lrs-data.hpp:154-210),
// which the reference runs as host loops over every cell. On a 512x384x320
// grid the host classification alone takes longer than a thousand steps of
// the simulation; here both are a few passes over the int32 voxel grid.
//
// Rasterisation: later boxes overwrite earlier ones, so a cell takes the
// material of the LAST box in file order that covers it. Every box's cells
// take atomicMax of the box index (grid pre-set to -1), then one pass maps
// box indices to materials: the same grid as the ordered loop, in one
// launch whatever the number of boxes.
//
// Classification, one warp per (y, z) row, x in chunks of 32 lanes:
//   k_count  boundary cells per row (ballot + popc) and the first
//            unphysical cell (atomicMin of the z-y-x linear index, which is
//            the host loop's scan order, so the error names the same cell)
//   k_scan   exclusive scan of the row counts (one CTA)
//   k_emit   the points at row offset + ballot prefix, so the list comes out
//            in the host's z-y-x order with materials in direction order.
#include <algorithm>
#include <cstdio>
#include <string>

#include <cuda_runtime.h>

#include "../../include/afd.h"
#include "geometry.hpp"

namespace afd {
namespace {

#define GK(call)                                                                                      \
    do {                                                                                              \
        cudaError_t e__ = (call);                                                                     \
        if (e__ != cudaSuccess) throw Error(AFD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e__)); \
    } while (0)

template <typename T>
struct Scratch {
    T* p = nullptr;
    explicit Scratch(size_t n) {
        if (n) GK(cudaMalloc(&p, n * sizeof(T)));
    }
    ~Scratch() {
        if (p) cudaFree(p);
    }
    Scratch(const Scratch&) = delete;
    Scratch& operator=(const Scratch&) = delete;
};

// group index of every 6-bit solid-neighbour mask, -1 where unphysical
struct GroupTable {
    int8_t g[64];
};

static_assert(sizeof(BoundaryPoint) == 7 * sizeof(int32_t), "BoundaryPoint is 7 packed int32");

__global__ void k_raster(const BoxCells* __restrict__ boxes, int nbox, int nx, int ny, int32_t* owner) {
    for (int b = blockIdx.y; b < nbox; b += gridDim.y) {
        const BoxCells c = boxes[b];
        const int64_t wx = c.hi[0] - c.lo[0] + 1, wy = c.hi[1] - c.lo[1] + 1, wz = c.hi[2] - c.lo[2] + 1;
        const int64_t n = wx * wy * wz;
        for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
            const int64_t x = c.lo[0] + t % wx, r = t / wx;
            const int64_t y = c.lo[1] + r % wy, z = c.lo[2] + r / wy;
            atomicMax(owner + ((z * ny + y) * nx + x), b);
        }
    }
}

__global__ void k_owner_to_material(int64_t cells, const BoxCells* __restrict__ boxes, int32_t* vox) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cells; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t b = vox[i];
        if (b >= 0) vox[i] = boxes[b].mat;
    }
}

__global__ void k_range(const int32_t* __restrict__ v, int64_t cells, int32_t nmat, unsigned long long* first) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cells; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t m = v[i];
        if (m < -1 || m >= nmat) atomicMin(first, (unsigned long long)i);
    }
}

// Solid-neighbour mask of air cell (x, y, z): bit d set when the neighbour in
// direction d (X_P, X_M, Y_P, Y_M, Z_P, Z_M) is solid.
__device__ __forceinline__ unsigned solid_mask(const int32_t* __restrict__ v, int64_t c, int64_t sy, int64_t sz,
                                               int32_t nb[6]) {
    nb[0] = v[c + 1];
    nb[1] = v[c - 1];
    nb[2] = v[c + sy];
    nb[3] = v[c - sy];
    nb[4] = v[c + sz];
    nb[5] = v[c - sz];
    unsigned m = 0;
#pragma unroll
    for (int d = 0; d < 6; ++d) m |= (nb[d] != -1 ? 1u : 0u) << d;
    return m;
}

// The table into shared memory; constant indices keep it in parameter space.
__device__ __forceinline__ void stage_table(const GroupTable& tab, int8_t* g_of) {
    if (threadIdx.x < 64) {
        int8_t v = -1;
#pragma unroll
        for (int i = 0; i < 64; ++i)
            if (i == (int)threadIdx.x) v = tab.g[i];
        g_of[threadIdx.x] = v;
    }
}

// One warp per interior row (y, z), 1 <= y <= ny-2, 1 <= z <= nz-2.
__global__ void k_count(const int32_t* __restrict__ v, int nx, int ny, int64_t rows, GroupTable tab,
                        int32_t* __restrict__ row_n, unsigned long long* first_bad) {
    __shared__ int8_t g_of[64];
    stage_table(tab, g_of);
    __syncthreads();
    const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= rows) return;  // whole warps
    const int64_t y = 1 + row % (ny - 2), z = 1 + row / (ny - 2);
    const int64_t sy = nx, sz = (int64_t)nx * ny;
    int n = 0;
    for (int x0 = 1; x0 < nx - 1; x0 += 32) {
        const int x = x0 + lane;
        const int64_t c = z * sz + y * sy + x;
        bool isb = false, bad = false;
        if (x < nx - 1 && v[c] == -1) {
            int32_t nb[6];
            const unsigned m = solid_mask(v, c, sy, sz, nb);
            isb = m != 0;
            bad = isb && g_of[m] < 0;
        }
        const unsigned bb = __ballot_sync(0xffffffffu, bad);
        if (bb && lane == __ffs(bb) - 1) atomicMin(first_bad, (unsigned long long)c);
        n += __popc(__ballot_sync(0xffffffffu, isb));
    }
    if (lane == 0) row_n[row] = n;
}

// off[i] = sum of cnt[0 .. i-1], off[n] = the total. One CTA of 1024.
__global__ void __launch_bounds__(1024) k_scan(const int32_t* __restrict__ cnt, int64_t n, int64_t* __restrict__ off) {
    __shared__ long long part[1024];
    const int t = threadIdx.x;
    const int64_t per = (n + 1023) / 1024, b = t * per, e = min(n, b + per);
    long long s = 0;
    for (int64_t i = b; i < e; ++i) s += cnt[i];
    part[t] = s;
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1) {
        const long long add = t >= d ? part[t - d] : 0;
        __syncthreads();
        part[t] += add;
        __syncthreads();
    }
    long long base = part[t] - s;
    for (int64_t i = b; i < e; ++i) {
        off[i] = base;
        base += cnt[i];
    }
    if (t == 1023) off[n] = part[1023];
}

__global__ void k_emit(const int32_t* __restrict__ v, int nx, int ny, int64_t rows, GroupTable tab,
                       const int64_t* __restrict__ off, int32_t* __restrict__ out) {
    __shared__ int8_t g_of[64];
    stage_table(tab, g_of);
    __syncthreads();
    const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= rows) return;
    const int64_t y = 1 + row % (ny - 2), z = 1 + row / (ny - 2);
    const int64_t sy = nx, sz = (int64_t)nx * ny;
    int64_t pos = off[row];
    for (int x0 = 1; x0 < nx - 1; x0 += 32) {
        const int x = x0 + lane;
        const int64_t c = z * sz + y * sy + x;
        unsigned m = 0;
        int32_t nb[6];
        if (x < nx - 1 && v[c] == -1) m = solid_mask(v, c, sy, sz, nb);
        const unsigned bal = __ballot_sync(0xffffffffu, m != 0);
        if (m) {
            int32_t* o = out + (pos + __popc(bal & ((1u << lane) - 1))) * 7;
            o[0] = x;
            o[1] = (int32_t)y;
            o[2] = (int32_t)z;
            o[3] = g_of[m];
            // materials of the set bits in direction order (at most three)
            int32_t m0 = -1, m1 = -1, m2 = -1;
#pragma unroll
            for (int d = 5; d >= 0; --d)
                if ((m >> d) & 1u) {
                    m2 = m1;
                    m1 = m0;
                    m0 = nb[d];
                }
            o[4] = m0;
            o[5] = m1;
            o[6] = m2;
        }
        pos += __popc(bal);
    }
}

// ---- engine masks ----------------------------------------------------------

// bits of word w (cells 32w .. 32w+31) for the cells lo .. hi (inclusive)
__device__ __forceinline__ uint32_t range_bits(int64_t w, int64_t lo, int64_t hi) {
    const int64_t a = max(lo - w * 32, (int64_t)0), b = min(hi - w * 32, (int64_t)31);
    if (a > b) return 0u;
    return (uint32_t)(((2ull << b) - 1ull) ^ ((1ull << a) - 1ull));
}

// word w of row (y, z) of the model's solid bits, zero outside the model
__device__ __forceinline__ uint32_t solid_word(const SolidBits& s, int64_t w, int64_t y, int64_t z) {
    if (!s.bits || y >= s.ny || z >= s.nz || w >= s.w) return 0u;
    return __ldg(s.bits + (z * s.ny + y) * s.w + w);
}

// one warp per word: lane = bit
__global__ void k_solid_bits(const int32_t* __restrict__ v, int nx, int64_t rows, int64_t mw, uint32_t* bits) {
    const int lane = threadIdx.x & 31;
    for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < rows * mw;
         w += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int64_t row = w / mw, x = (w % mw) * 32 + lane;
        const bool solid = x < nx && v[row * nx + x] != -1;
        const uint32_t b = __ballot_sync(0xffffffffu, solid);
        if (lane == 0) bits[w] = b;
    }
}

__global__ void k_cell_bits(const int32_t* __restrict__ cells, int64_t n, uint32_t* bits) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t c = cells[i];
        atomicOr(bits + (c >> 5), 1u << (c & 31));
    }
}

// one thread per word of the engine grid
// zoff, gzg: the grid's planes are global planes zoff.. of a grid of gzg
// planes (a z-slab of it); the slab rules use global planes.
__global__ void k_pml_masks(SolidBits s, const uint32_t* __restrict__ lrs, int gx, int gy, int gz, int wpr, int W,
                            uint32_t F, uint32_t* owned, unsigned long long* count, int zoff, int gzg) {
    const int64_t total = (int64_t)gz * gy * wpr;
    unsigned long long n = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t w = i % wpr, y = i / wpr % gy, z = i / wpr / gy;
        const int64_t zg = z + zoff;
        const uint32_t a = ~solid_word(s, w, y, z) & ~lrs[i] & range_bits(w, 0, gx - 1);
        uint32_t o = 0u;
        if (a && y >= 2 && y <= gy - 3 && zg >= 2 && zg <= gzg - 3 && z >= 1 && z <= gz - 2) {
            const bool yz = ((F & AFD_FACE_YM) && y < W) || ((F & AFD_FACE_YP) && y > gy - W - 1) ||
                            ((F & AFD_FACE_ZM) && zg < W) || ((F & AFD_FACE_ZP) && zg > gzg - W - 1);
            uint32_t slab = yz ? 0xffffffffu : 0u;
            if (F & AFD_FACE_XM) slab |= range_bits(w, 0, W - 1);
            if (F & AFD_FACE_XP) slab |= range_bits(w, gx - W, gx - 1);
            o = a & slab & range_bits(w, 2, gx - 3);
        }
        owned[i] = o;
        n += __popc(o);
    }
    for (int d = 16; d > 0; d >>= 1) n += __shfl_down_sync(0xffffffffu, n, d);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(count, n);
}

__global__ void k_or(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b, uint32_t* out, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (a ? a[i] : 0u) | b[i];
}

// one thread per (z, tile)
__global__ void k_air_flags(SolidBits s, int gx, int gy, int gz, int tw, int th, int tiles_x, int tiles_y,
                            uint8_t* flags) {
    const int64_t ntile = (int64_t)tiles_x * tiles_y, total = ntile * gz;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t z = i / ntile, t = i % ntile, ty = t / tiles_x, tx = t % tiles_x;
        const int64_t x0 = max(tx * tw - 1, (int64_t)0), x1 = min(tx * tw + tw, (int64_t)gx - 1);
        const int64_t y0 = max(ty * th - 1, (int64_t)0), y1 = min(ty * th + th, (int64_t)gy - 1);
        bool air = false;
        for (int64_t y = y0; y <= y1 && !air; ++y)
            for (int64_t w = x0 / 32; w <= x1 / 32 && !air; ++w)
                air = (~solid_word(s, w, y, z) & range_bits(w, x0, x1)) != 0u;
        flags[i] = air ? 1 : 0;
    }
}

int grid_for(int64_t n, int threads) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, 148 * 16));
}

}  // namespace

void rasterize_device(const Scene& sc, int32_t* d_vox, void* stream) {
    cudaStream_t st = (cudaStream_t)stream;
    const Model& m = sc.model;
    const int64_t cells = m.cells();
    GK(cudaMemsetAsync(d_vox, 0xff, (size_t)cells * sizeof(int32_t), st));  // -1 everywhere
    const int nbox = (int)sc.boxes.size();
    if (!nbox) return;
    int64_t vmax = 1;
    for (const BoxCells& c : sc.boxes) {
        for (int k = 0; k < 3; ++k) {
            const int32_t n = k == 0 ? m.nx : (k == 1 ? m.ny : m.nz);
            if (c.lo[k] < 0 || c.hi[k] < c.lo[k] || c.hi[k] >= n)
                throw Error(AFD_ERR_ARG, "box cell range outside the grid");
        }
        vmax = std::max<int64_t>(vmax, (int64_t)(c.hi[0] - c.lo[0] + 1) * (c.hi[1] - c.lo[1] + 1) *
                                           (c.hi[2] - c.lo[2] + 1));
    }
    Scratch<BoxCells> boxes((size_t)nbox);
    GK(cudaMemcpyAsync(boxes.p, sc.boxes.data(), (size_t)nbox * sizeof(BoxCells), cudaMemcpyHostToDevice, st));
    const dim3 grid((unsigned)std::min<int64_t>((vmax + 255) / 256, 1024), (unsigned)std::min(nbox, 65535));
    k_raster<<<grid, 256, 0, st>>>(boxes.p, nbox, m.nx, m.ny, d_vox);
    k_owner_to_material<<<grid_for(cells, 256), 256, 0, st>>>(cells, boxes.p, d_vox);
    GK(cudaGetLastError());
    GK(cudaStreamSynchronize(st));  // the box table is freed on return
}

std::vector<BoundaryPoint> classify_device(const int32_t* d_vox, int32_t nx, int32_t ny, int32_t nz, int32_t nmat,
                                           void* stream) {
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t cells = (int64_t)nx * ny * nz;
    // flags: [0] first voxel out of range, [1] first unphysical cell
    Scratch<unsigned long long> flags(2);
    GK(cudaMemsetAsync(flags.p, 0xff, 2 * sizeof(unsigned long long), st));
    if (nmat > 0 && cells > 0) {
        k_range<<<grid_for(cells, 256), 256, 0, st>>>(d_vox, cells, nmat, flags.p);
        GK(cudaGetLastError());
    }
    const int64_t rows = (nx >= 3 && ny >= 3 && nz >= 3) ? (int64_t)(ny - 2) * (nz - 2) : 0;
    GroupTable tab;
    for (unsigned mk = 0; mk < 64; ++mk) tab.g[mk] = (int8_t)(mk ? group_of_mask(mk) : -1);
    Scratch<int32_t> row_n((size_t)rows);
    Scratch<int64_t> off((size_t)rows + 1);
    const int threads = 256;
    const int64_t blocks = (rows * 32 + threads - 1) / threads;
    if (rows) {
        k_count<<<(unsigned)blocks, threads, 0, st>>>(d_vox, nx, ny, rows, tab, row_n.p, flags.p + 1);
        k_scan<<<1, 1024, 0, st>>>(row_n.p, rows, off.p);
        GK(cudaGetLastError());
    }
    unsigned long long hf[2];
    int64_t total = 0;
    GK(cudaMemcpyAsync(hf, flags.p, sizeof hf, cudaMemcpyDeviceToHost, st));
    if (rows) GK(cudaMemcpyAsync(&total, off.p + rows, sizeof total, cudaMemcpyDeviceToHost, st));
    GK(cudaStreamSynchronize(st));
    if (hf[0] != ~0ull) throw Error(AFD_ERR_ARG, "voxel material index out of range");
    if (hf[1] != ~0ull) {
        const int64_t c = (int64_t)hf[1];
        char buf[160];
        std::snprintf(buf, sizeof buf, "Unphysical surfaces encountered at cell (%lld,%lld,%lld)",
                      (long long)(c % nx), (long long)(c / nx % ny), (long long)(c / ((int64_t)nx * ny)));
        throw Error(AFD_ERR_GEOMETRY, buf);
    }
    std::vector<BoundaryPoint> pts((size_t)total);
    if (total) {
        Scratch<int32_t> out((size_t)total * 7);
        k_emit<<<(unsigned)blocks, threads, 0, st>>>(d_vox, nx, ny, rows, tab, off.p, out.p);
        GK(cudaGetLastError());
        GK(cudaMemcpyAsync(pts.data(), out.p, (size_t)total * sizeof(BoundaryPoint), cudaMemcpyDeviceToHost, st));
        GK(cudaStreamSynchronize(st));
    }
    return pts;
}

void solid_bits_device(const int32_t* d_vox, int32_t nx, int32_t ny, int32_t nz, uint32_t* d_bits, void* stream) {
    const int64_t rows = (int64_t)ny * nz, mw = row_words(nx);
    if (rows * mw == 0) return;
    k_solid_bits<<<grid_for(rows * mw * 32, 256), 256, 0, (cudaStream_t)stream>>>(d_vox, nx, rows, mw, d_bits);
    GK(cudaGetLastError());
}

void boundary_bits_device(const int32_t* d_cells, int64_t n, int64_t words, uint32_t* d_bits, void* stream) {
    cudaStream_t st = (cudaStream_t)stream;
    GK(cudaMemsetAsync(d_bits, 0, (size_t)words * sizeof(uint32_t), st));
    if (n) k_cell_bits<<<grid_for(n, 256), 256, 0, st>>>(d_cells, n, d_bits);
    GK(cudaGetLastError());
}

int64_t pml_masks_device(const SolidBits& s, const uint32_t* d_boundary, int32_t gx, int32_t gy, int32_t gz,
                         int32_t wpr, int32_t width, uint32_t faces, uint32_t* d_owned, void* stream, int32_t zoff,
                         int32_t gz_global) {
    cudaStream_t st = (cudaStream_t)stream;
    if ((int64_t)wpr * 32 < gx) throw Error(AFD_ERR_ARG, "mask rows narrower than the grid");
    Scratch<unsigned long long> cnt(1);
    GK(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long), st));
    const int64_t words = (int64_t)gz * gy * wpr;
    k_pml_masks<<<grid_for(words, 256), 256, 0, st>>>(s, d_boundary, gx, gy, gz, wpr, width, faces, d_owned, cnt.p,
                                                       zoff, gz_global > 0 ? gz_global : gz);
    GK(cudaGetLastError());
    unsigned long long h = 0;
    GK(cudaMemcpyAsync(&h, cnt.p, sizeof h, cudaMemcpyDeviceToHost, st));
    GK(cudaStreamSynchronize(st));
    return (int64_t)h;
}

void or_masks_device(const uint32_t* a, const uint32_t* b, uint32_t* out, int64_t n, void* stream) {
    if (!n) return;
    k_or<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(a, b, out, n);
    GK(cudaGetLastError());
}

void air_flags_device(const SolidBits& s, int32_t gx, int32_t gy, int32_t gz, int32_t tile_w, int32_t tile_h,
                      int32_t tiles_x, int32_t tiles_y, uint8_t* d_flags, void* stream) {
    const int64_t total = (int64_t)tiles_x * tiles_y * gz;
    if (!total) return;
    k_air_flags<<<grid_for(total, 128), 128, 0, (cudaStream_t)stream>>>(s, gx, gy, gz, tile_w, tile_h, tiles_x,
                                                                         tiles_y, d_flags);
    GK(cudaGetLastError());
}

namespace {

// a device selected and a stream of its own for one synchronous call
struct DeviceScope {
    int prev = -1;
    cudaStream_t st = nullptr;
    explicit DeviceScope(int32_t device) {
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw Error(AFD_ERR_CUDA, "no CUDA device available");
        if (device < 0 || device >= ndev) throw Error(AFD_ERR_ARG, "device ordinal out of range");
        GK(cudaGetDevice(&prev));
        GK(cudaSetDevice(device));
        GK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    }
    ~DeviceScope() {
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

std::vector<BoundaryPoint> classify_on(const Model& m, int32_t device) {
    if ((int64_t)m.vox.size() != m.cells()) throw Error(AFD_ERR_ARG, "voxel count mismatch");
    DeviceScope ds(device);
    Scratch<int32_t> dv((size_t)m.cells());
    if (m.cells())
        GK(cudaMemcpyAsync(dv.p, m.vox.data(), (size_t)m.cells() * sizeof(int32_t), cudaMemcpyHostToDevice, ds.st));
    return classify_device(dv.p, m.nx, m.ny, m.nz, 0, ds.st);  // no range check, as classify()
}

Model load_kerkythea_on(const std::string& xml_path, float res, int32_t device) {
    Scene sc = parse_kerkythea(xml_path, res);
    DeviceScope ds(device);
    Model& m = sc.model;
    Scratch<int32_t> dv((size_t)m.cells());
    rasterize_device(sc, dv.p, ds.st);
    m.vox.resize((size_t)m.cells());
    GK(cudaMemcpyAsync(m.vox.data(), dv.p, (size_t)m.cells() * sizeof(int32_t), cudaMemcpyDeviceToHost, ds.st));
    GK(cudaStreamSynchronize(ds.st));
    return std::move(m);
}

}  // namespace afd
