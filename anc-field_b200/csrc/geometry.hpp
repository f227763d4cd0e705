// Device-side geometry set-up: rasterisation of a parsed Kerkythea scene into
// the voxel grid and the LRS boundary classification, as CUDA kernels on the
// calling thread's current device. Same results as rasterize_host and
// classify (model.hpp), bit for bit, including the order of the boundary
// list and the cell named by an unphysical-pattern error.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "model.hpp"

namespace afd {

// Writes the scene's voxels into d_vox (model.nx * ny * nz int32 on the
// device, z-y-x order) on `stream` (a cudaStream_t).
void rasterize_device(const Scene& sc, int32_t* d_vox, void* stream);

// The boundary list of the voxels at d_vox, in the z-y-x scan order of
// classify(). With nmat > 0 a voxel outside -1 .. nmat-1 raises
// Error(AFD_ERR_ARG) first; an unphysical pattern raises Error(AFD_ERR_GEOMETRY)
// naming the first such cell in scan order. Synchronises `stream`.
std::vector<BoundaryPoint> classify_device(const int32_t* d_vox, int32_t nx, int32_t ny, int32_t nz, int32_t nmat,
                                           void* stream);

// Whole-model forms on device `device`, each on a stream of its own and
// synchronous: the boundary list of m's voxels (what classify(m) returns or
// throws), and the Kerkythea loader with the rasterisation on the device.
std::vector<BoundaryPoint> classify_on(const Model& m, int32_t device);
Model load_kerkythea_on(const std::string& xml_path, float res, int32_t device);

// ---- engine masks, all 32-bit words with bit (x % 32) of word x / 32 ----

// Solid cells of a voxel grid as bits: row (z, y) holds w = row_words(nx)
// words.
inline int32_t row_words(int32_t nx) { return (nx + 31) / 32; }
struct SolidBits {
    const uint32_t* bits = nullptr;  // null: no model, every cell air
    int32_t nx = 0, ny = 0, nz = 0, w = 0;
};

// The solid bits of the voxels at d_vox ([nz][ny][nx] int32, -1 air) into
// d_bits (nz * ny * row_words(nx) words).
void solid_bits_device(const int32_t* d_vox, int32_t nx, int32_t ny, int32_t nz, uint32_t* d_bits, void* stream);

// For an engine grid (gx, gy, gz) whose rows hold wpr words (wpr * 32 >= gx),
// the model's solid bits placed at the origin (cells outside the model are
// air):
//   boundary_bits_device  d_bits (zeroed here) gets the cells of the n linear
//                         indices z * ny * wpr * 32 + y * wpr * 32 + x
//   pml_masks_device      the FIXED-scheme PML cells: air cells that are
//                         neither solid nor boundary, with 2 <= x,y,z <= n-3,
//                         inside an enabled face slab of `width` cells, into
//                         d_owned; returns their number (synchronises
//                         `stream`). zoff, gz_global: the grid is a z-slab
//                         (planes zoff.. of gz_global); the rules then use
//                         global planes and skip the slab's two end planes
//   or_masks_device       out = a | b over n words (a may be null)
//   air_flags_device      flags[z][ty * tiles_x + tx] = 1 where an air cell
//                         lies in tile (tx, ty) of plane z widened by one
//                         cell in x and y (tiles tile_w x tile_h)
void boundary_bits_device(const int32_t* d_cells, int64_t n, int64_t words, uint32_t* d_bits, void* stream);
int64_t pml_masks_device(const SolidBits& s, const uint32_t* d_boundary, int32_t gx, int32_t gy, int32_t gz,
                         int32_t wpr, int32_t width, uint32_t faces, uint32_t* d_owned, void* stream,
                         int32_t zoff = 0, int32_t gz_global = 0);
void or_masks_device(const uint32_t* a, const uint32_t* b, uint32_t* out, int64_t n, void* stream);
void air_flags_device(const SolidBits& s, int32_t gx, int32_t gy, int32_t gz, int32_t tile_w, int32_t tile_h,
                      int32_t tiles_x, int32_t tiles_y, uint8_t* d_flags, void* stream);

}  // namespace afd
