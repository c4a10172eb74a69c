// Octree mesh construction on the device (mesh/builder.py,
// build_octree_mesh_device; the reference takes its mesh from the external
// fluxel package, core/grid/factory.py:32-65, whose contract for hanging
// faces is core/grid/axis_projected.py:715-767).
//
// The octree is given as the id of the leaf covering each finest-level cell
// ([FX][FY][FZ], C order) and the leaves' finest-level lower corners.  An
// internal face joins two leaves that touch across a finest-level face; two
// leaves of a coarse-fine interface, or two coarse leaves, touch across a
// whole rectangle of finest faces.  Only the rectangle's corner with the
// smallest tangential coordinates emits the pair, so every owner/neighbour
// pair appears exactly once and no deduplication pass is needed.
#include "gf_common.cuh"

namespace gf {

constexpr int kMeshThreads = 256;
constexpr int64_t kKeyNone = -1;
constexpr int64_t kKeyBadId = -2;

// One thread per finest-level face position along `axis` (positions in the
// C order of the [ex][ey][ez] array of lower cells, ex = FX - 1 for x and so
// on).  keys[q] = A * n_cells + B for the emitting position of the face
// between leaf A (lower coordinate, the owner) and leaf B; kKeyNone
// elsewhere; kKeyBadId when an id is outside [0, n_cells).
__global__ void k_octree_face_keys(const int64_t* __restrict__ ids, int64_t FX, int64_t FY, int64_t FZ,
                                   const int64_t* __restrict__ corner, int64_t n_cells, int axis,
                                   int64_t* __restrict__ keys) {
    const int64_t ex = FX - (axis == 0), ey = FY - (axis == 1), ez = FZ - (axis == 2);
    const int64_t total = ex * ey * ez;
    const int64_t stride = axis == 0 ? FY * FZ : (axis == 1 ? FZ : 1);
    const int t0 = axis == 0 ? 1 : 0;  // tangential axes
    const int t1 = axis == 2 ? 1 : 2;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = q % ez;
        const int64_t r = q / ez;
        const int64_t j = r % ey;
        const int64_t i = r / ey;
        const int64_t pa = (i * FY + j) * FZ + k;
        const int64_t a = ids[pa], b = ids[pa + stride];
        int64_t key = kKeyNone;
        if (a < 0 || a >= n_cells || b < 0 || b >= n_cells) {
            key = kKeyBadId;
        } else if (a != b) {
            const int64_t pos[3] = {i, j, k};
            const int64_t ca0 = corner[t0 * n_cells + a], cb0 = corner[t0 * n_cells + b];
            const int64_t ca1 = corner[t1 * n_cells + a], cb1 = corner[t1 * n_cells + b];
            if (pos[t0] == (ca0 > cb0 ? ca0 : cb0) && pos[t1] == (ca1 > cb1 ? ca1 : cb1)) key = a * n_cells + b;
        }
        keys[q] = key;
    }
}

}  // namespace gf

using namespace gf;

extern "C" {

int gf_octree_face_keys(const int64_t* ids, int64_t fx, int64_t fy, int64_t fz, const int64_t* corner,
                        int64_t n_cells, int32_t axis, int64_t* keys, void* stream) {
    if (ids == nullptr || corner == nullptr || keys == nullptr || axis < 0 || axis > 2 || fx < 1 || fy < 1 ||
        fz < 1 || n_cells < 1 || n_cells > ((int64_t)1 << 31)) {
        set_error("gf_octree_face_keys: invalid arguments");
        return GF_ERR_INVALID;
    }
    const int64_t total = (fx - (axis == 0)) * (fy - (axis == 1)) * (fz - (axis == 2));
    if (total == 0) return GF_OK;
    int64_t blocks = (total + kMeshThreads - 1) / kMeshThreads;
    if (blocks > 148 * 32) blocks = 148 * 32;
    k_octree_face_keys<<<(unsigned)blocks, kMeshThreads, 0, GF_STREAM(stream)>>>(ids, fx, fy, fz, corner, n_cells,
                                                                                  axis, keys);
    return check_launch("gf_octree_face_keys");
}

}  // extern "C"
