// Host-side geometry of the FDTD core: Kerkythea XML reading, voxelisation,
// material filter tables and the locally-reacting-surface (LRS) boundary
// classification. Pure C++17, no CUDA.
#pragma once

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace afd {

// Error with an AFD_ERR_* status attached; converted to a status code at the
// C ABI boundary.
struct Error : std::runtime_error {
    int status;
    Error(int st, const std::string& msg) : std::runtime_error(msg), status(st) {}
};

// One axis-aligned box read from the model: {min_x, max_x, min_y, max_y,
// min_z, max_z} in metres after the (x,y,z) <- (a,c,-b) axis remap, and the
// material name (text after the last '_' of the model name).
struct Box {
    std::array<float, 6> ext;
    std::string material;
};

// Parses the Kerkythea scene: Root/Object[Type=Scene]/Object[Type=Model],
// first child Object, its Parameter[Name="Vertex List"] P@xyz points.
// Follows LoadBoxes, anc-field/src/kerkythea.hpp:63-130.
std::vector<Box> load_boxes(const std::string& xml_path);

// One coefficient per line, each parsed as double and rounded to float
// (Util::FileToVariable, anc-field/src/util.hpp:100-115).
std::vector<float> read_coefficients(const std::string& path);

// Reference grid rounding (Util::RoundTo, anc-field/src/util.hpp:43-47).
inline uint32_t round_to(uint32_t n, uint32_t unit) {
    return (n % unit == 0) ? n : n + (unit - n % unit);
}

// Cell index of a coordinate: (size_t)(pos / res) in FP32, as
// kerkythea.hpp:185-189 and simulation.hpp:281-283 compute it.
inline int64_t cell_of(float pos, float res) {
    float q = pos / res;
    return (int64_t)q;
}

// Voxel model: int32 grid, -1 = air, else material index; coefficient
// tables a[nmat][ncoef], b[nmat][ncoef] in sorted-name material order.
struct Model {
    int32_t nx = 0, ny = 0, nz = 0;
    std::vector<int32_t> vox;
    int32_t nmat = 0, ncoef = 0;
    std::vector<float> a, b;
    std::vector<std::string> material_names;

    int64_t cells() const { return (int64_t)nx * ny * nz; }
    int32_t at(int64_t x, int64_t y, int64_t z) const { return vox[(z * ny + y) * nx + x]; }
};

// Inclusive cell ranges [lo, hi] of one box and its material index.
struct BoxCells {
    int32_t lo[3], hi[3];
    int32_t mat;
};

// A parsed scene: the model with grid, materials and filter tables but no
// voxels yet, and the cell ranges of its boxes in file order.
struct Scene {
    Model model;
    std::vector<BoxCells> boxes;
};

// Kerkythea constructor up to the rasterisation, kerkythea.hpp:133-179.
Scene parse_kerkythea(const std::string& xml_path, float res);

// The rasterisation loop of kerkythea.hpp:180-195: every cell air (-1), then
// each box's cells set to its material, later boxes overwriting earlier ones.
void rasterize_host(const Scene& sc, Model& m);

// Kerkythea constructor, kerkythea.hpp:133-196: parse_kerkythea followed by
// rasterize_host.
Model load_kerkythea(const std::string& xml_path, float res);

// Group numbering of anc-field/src/lrs-data.hpp:53-78 (X_P=0 ... X_M_Y_M_Z_M=25).
// Direction order inside a pattern: X_P, X_M, Y_P, Y_M, Z_P, Z_M.
enum Dir { DXP = 0, DXM = 1, DYP = 2, DYM = 3, DZP = 4, DZM = 5 };
constexpr int kNumGroups = 26;

// Bit mask (bit d = direction d solid) of every group, in group order.
extern const uint8_t kGroupMask[kNumGroups];
// Number of solid neighbours of every group (1, 2 or 3).
int group_faces(int g);
// Group index of a 6-bit solid-neighbour mask, or -1 if the pattern is
// unphysical (lrs-data.hpp:217-330).
int group_of_mask(unsigned mask);

// One boundary air cell.
struct BoundaryPoint {
    int32_t x, y, z;
    int32_t group;
    int32_t mat[3];   // materials of the solid neighbours in direction order; -1 unused
};

// LrsData::Init, anc-field/src/lrs-data.hpp:116-215: every air cell with
// 1 <= x,y,z <= n-2 and at least one solid face neighbour, in z-y-x scan
// order. Throws Error(AFD_ERR_GEOMETRY) on an unphysical pattern.
std::vector<BoundaryPoint> classify(const Model& m);

// Whitespace-separated text matrix, one row per line, values parsed with
// atof into float (df::Load, anc-field/src/datafile.hpp:28-67). Returns the
// values in file order; rows gives the row count and cols the first row's
// column count.
std::vector<float> load_text_matrix(const std::string& path, int64_t* rows, int64_t* cols);

// Row-per-receiver text output with ostream default formatting (6
// significant digits), a trailing space after every value and a final blank
// line (df::Save, anc-field/src/datafile.hpp:70-102).
void save_rows(const std::string& path, const float* data, int64_t rows, int64_t cols);

}  // namespace afd
