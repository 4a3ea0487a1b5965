// 3D Laguerre-cell kernels (sm_100a), FP64: cell volumes, centroids, Hessian
// rows (face area / |x_i - x_j|) and neighbour lists.
#pragma once
#include "cell2d.cuh"
#include "common.cuh"
#include "tree.cuh"

namespace sdot {

// Hessian rows and neighbour lists of 3D cells (ELL widths; longer rows go to
// the side buffer of Rows).
constexpr int ROWCAP_3D = 32;
constexpr int NBCAP_3D = 48;

struct Cell3DArgs {
    long long n = 0;
    const double *pos = nullptr;  // 3n, sorted order
    const double *w = nullptr;    // n, sorted order
    const TreeNode<3> *nodes = nullptr;
    int max_nodes = 1 << 30;
    double box_lo[3] = {0, 0, 0}, box_hi[3] = {1, 1, 1};  // the starting box (a domain shape's box)
    double coeff = 1.0;                                    // the shape's density
    // a convex shape: the box cut by nplanes half-spaces a . x <= b
    // (absolute coordinates; 4 doubles per plane: a, b); faces of the shape
    // get the ids domain_id(6 + k)
    int nplanes = 0;
    const double *planes = nullptr;
    // piecewise-constant voxel image (ScaledImage, nb_coeffs = 1): nx x ny x nz
    // values, x fastest, over [img_lo, img_hi]; each cell is integrated voxel
    // by voxel (the density of a piece is the voxel's value times coeff).
    // img_backup: per warp a copy of the faces (img_backup_bytes per warp).
    const double *img = nullptr;
    int img_n[3] = {0, 0, 0};
    double img_lo[3] = {0, 0, 0}, img_hi[3] = {1, 1, 1};
    char *img_backup = nullptr;
    // optional multilinear density factor (has_poly): coeff * (p0 + p1 x +
    // p2 y + p3 z + p4 xy + p5 xz + p6 yz + p7 xyz), absolute coordinates
    int has_poly = 0;
    double poly[8] = {1, 0, 0, 0, 0, 0, 0, 0};
    double *mass = nullptr;  // n
    double *ctd = nullptr;   // 3n
    Rows rows;               // Hessian rows (rows.cnt null: skipped)
    Rows nb;                 // neighbour ids (nb.cnt null: skipped)
    int *ovf_list = nullptr;  // cells handed to the second pass
    int *ovf_cnt = nullptr;
    int *ovf_list2 = nullptr;  // cells handed to the third pass
    int *ovf_cnt2 = nullptr;
    int *ovf_list3 = nullptr;  // cells handed to the fourth pass
    int *ovf_cnt3 = nullptr;
    // per cell (sorted order): the pass (0..3) its last build needed; with
    // use_hint the first pass sends each cell straight to that pass (the
    // positions, hence the tree order, must not have changed)
    unsigned char *hint = nullptr;
    int use_hint = 0;
    unsigned *err = nullptr;
    int *guard = nullptr;
};

// First pass over every cell (up to 32 faces of 16 vertices, shared memory),
// then the cells that overflowed it (64 faces of 32 vertices, shared memory),
// then those that overflowed again (128 faces of 64 vertices, then 256 faces
// of 128 vertices, both in `scratch` of cells3d_scratch_bytes() bytes).
size_t cells3d_scratch_bytes();
// Bytes of the per-warp face copies of the voxel-image mode (all passes).
size_t cells3d_image_backup_bytes();
void cells3d_launch(const Cell3DArgs &a, void *scratch, cudaStream_t st);

}  // namespace sdot
