// 2D Laguerre-cell kernels: traversal + clipping + integrals + Hessian rows.
#pragma once
#include "common.cuh"
#include "tree.cuh"

namespace sdot {

// DM_IMAGE: piecewise-constant image (nb_coeffs = 1); DM_IMAGE6: piecewise
// quadratic (nb_coeffs = 6, planes of img_nx * img_ny coefficients)
// DM_RASTER: no cell outputs; each cell (with the starting shape's density)
// is integrated over the pixels of a raster (get_image_integrals,
// get_image_of_cell_nums)
// DM_PERIODIC: DM_SINGLE with translated copies of the Diracs (ntrans > 0)
enum DomainMode : int { DM_SINGLE = 0, DM_MULTI = 1, DM_IMAGE = 2, DM_IMAGE6 = 3, DM_RASTER = 4, DM_PERIODIC = 5 };

// Cell polygon capacities of the two tiers.  Every cell is first built by
// the fast kernel (one thread per cell, polygon in shared memory); cells that
// overflow it are rebuilt by the warp tier (one warp per cell, polygon in
// global scratch).  Beyond the warp tier's capacity the call reports
// ST_CAPACITY.
// 13 fast vertices (260 B of shared memory per cell): with the fast
// kernel's shared-memory carveout an SM holds more warps than with 14 or 16,
// and the few cells of 14 or more vertices on the 1M clustered mix cost less
// in the warp tier than the smaller occupancy would (measured: 13 vertices
// 4.13 ms, 12: 4.16, 14: 4.23, 16: 4.54).
constexpr int CAP_FAST_2D = 13;
static_assert(CAP_FAST_2D <= 32, "the fast tier keeps one bit per vertex in a 32-bit mask");
constexpr int CAP_HUGE_2D = 1024;
// Hessian rows and neighbour lists are stored slot-major (ELL) with these
// widths; longer rows (only cells of the warp tier) go to a side buffer,
// their offset in Rows::side[s].
constexpr int ROWCAP_2D = 24;
constexpr int NBCAP_2D = 40;

// Row storage shared by the cell kernels, the CSR assembly and the solver.
struct Rows {
    int *cnt = nullptr;        // entries per row (sorted order)
    int *col = nullptr;        // ELL columns (sorted order)
    double *val = nullptr;     // ELL values (may be null for id lists)
    long long stride = 0;      // ELL slot stride (>= n)
    int cap = 0;               // ELL width
    long long *side = nullptr; // per row: offset in the side buffer when cnt > cap
    int *side_col = nullptr;
    double *side_val = nullptr;
    long long side_cap = 0;
    unsigned long long *side_used = nullptr;
    __host__ __device__ int *colp(long long s, int k) const {
        return cnt[s] > cap ? side_col + side[s] + k : col + k * stride + s;
    }
    __host__ __device__ double *valp(long long s, int k) const {
        return cnt[s] > cap ? side_val + side[s] + k : val + k * stride + s;
    }
};

struct Cell2DArgs {
    long long n = 0;
    const double *pos = nullptr;   // 2n, sorted order
    const double *w = nullptr;     // n, sorted order
    const TreeNode<2> *nodes = nullptr;
    int max_nodes = 1 << 30;       // node array size (debug checks)
    // starting polygon (single item polygon, inflated bbox, or image box)
    int start_n = 0;
    const double *start_xy = nullptr;  // 2 * start_n
    double coeff = 1.0;                // single-item density
    int mode = DM_SINGLE;
    int mixed = 0;                     // FP32 build + FP64 re-clip (SDOT_MIXED)
    int ball = 0;
    // image (nb_coeffs == 1)
    double img_lo[2] = {0, 0}, img_hi[2] = {1, 1};
    int img_nx = 0, img_ny = 0;
    const double *img = nullptr;
    // multi items: item k has vertices [item_off[k], item_off[k+1]) in item_xy
    // (2 per vertex) with outward unit normals item_nrm, density item_coeff[k]
    int nitems = 0;
    const int *item_off = nullptr;
    const double *item_xy = nullptr;
    const double *item_nrm = nullptr;
    const double *item_coeff = nullptr;
    // outputs (sorted order); null pointers skip that output
    double *mass = nullptr;       // get_integrals
    double *mass_c = nullptr;     // mass as get_centroids computes it
    double *ctd = nullptr;        // 2n centroids
    Rows rows;                    // Hessian rows (rows.cnt null: skipped)
    Rows nb;                      // boundary ids of each cell (nb.cnt null: skipped)
    // cells that overflow the fast tier (sorted indices handed to the warp tier)
    int *ovf_list = nullptr;
    int *ovf_cnt = nullptr;
    // raster outputs (DM_RASTER): per pixel (x-fastest) the sums of m x_i,
    // m y_i and m over the cells i, m the integral of cell i over the pixel
    // (ras, 3 doubles per pixel), and the largest caller index of a cell of
    // non-zero integral over the pixel (ras_nums, -1 if none)
    double *ras = nullptr;
    long long *ras_nums = nullptr;
    double ras_lo[2] = {0, 0}, ras_hi[2] = {1, 1};
    int ras_nx = 0, ras_ny = 0;
    const int *perm = nullptr;     // sorted -> caller index
    // periodic domains (DM_PERIODIC): ntrans translations (x, y pairs); the
    // image of sorted Dirac j under translation k cuts with id j + (k + 1) n
    int ntrans = 0;
    const double *trans = nullptr;
    unsigned *err = nullptr;
    int *guard = nullptr;          // first failed guard: (code, sorted index, value)
    long long item_nv = 0;         // number of item vertices (multi items)
};

size_t cells2d_scratch_bytes();
// First failed debug check of the cell kernels (code, line, value); zeros in
// release builds.
void cells2d_read_checks(unsigned long long out[3]);
// Work counts of the fast tier's walks (counting builds, -DSDOT_COUNT; zeros
// otherwise), optionally reset.
void cells2d_read_work(unsigned long long out[8], bool reset);
// Fast kernel over all cells, then the big and huge tiers over the overflow
// lists.  `scratch` must hold cells2d_scratch_bytes() bytes.
void cells2d_launch(const Cell2DArgs &a, void *scratch, cudaStream_t st);

}  // namespace sdot
