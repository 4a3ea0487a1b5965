// Derivatives of the cell centroids and masses with respect to the weights
// and the positions (2D): get_der_centroids_and_integrals_wrt_weight_and_positions
// (src/sdot/PowerDiagram/get_der_centroids_and_integrals_wrt_weight_and_positions.h:17-216).
//
// The cells come from the neighbour pass (one row per cell in sorted order:
// the cut id of the edge leaving each vertex, domain edges included); each
// vertex is rebuilt in FP64 as the intersection of the lines of its two edges
// (a weighted bisector, or a domain edge), in coordinates relative to the
// cell's Dirac.  Per edge with a Dirac on the other side the reference's
// boundary item gives the measure (coeff * length), the position integral
// 1/2 l (p0 + p1) and the second moments l/6 (2 (p0 p0' + p1 p1') + p0 p1'
// + p1 p0') (ConvexPolyhedron2.tcc:437-478); the row items are the reference's
// 3 x 3 blocks (rows: centroid x, centroid y, mass; columns: position x,
// position y, weight), corrected by the centroid and divided by
// mass + (mass == 1) as the reference divides (.h:178-182), sorted by column
// and merged.  One thread per cell; cells of more than DP_CAP vertices report
// a capacity error.
#include "derpos.cuh"

namespace sdot {

namespace {

constexpr int TB = 128;
constexpr int DP_CAP = 64;   // vertices of a cell
constexpr int DP_ROW = 65;   // blocks of a row (one per edge and the diagonal)

struct DpArgs {
    Rows nb;
    long long n;
    const double *pos, *w;
    const int *idx;
    int start_n;
    const double *start_xy;
    double coeff;
    int ntrans;
    const double *trans;
};

// position of the Dirac (or periodic image) on the other side of an edge with this id
__device__ void other_site(const DpArgs &A, int id, double &x, double &y, double &w, int &j) {
    j = int(id % A.n);
    const int k = int(id / A.n) - 1;
    x = A.pos[2 * j];
    y = A.pos[2 * j + 1];
    if (k >= 0) {
        x += A.trans[2 * k];
        y += A.trans[2 * k + 1];
    }
    w = A.w[j];
}

// line a . u = b of the edge with this id, u relative to c0
__device__ void edge_line(const DpArgs &A, int id, double c0x, double c0y, double w0, double &ax, double &ay,
                          double &b) {
    if (id >= 0) {
        double x, y, w1;
        int j;
        other_site(A, id, x, y, w1, j);
        const double dx = x - c0x, dy = y - c0y;
        ax = dx;
        ay = dy;
        b = 0.5 * (dx * dx + dy * dy) + 0.5 * (w0 - w1);
    } else {
        const int e = domain_edge(id), e1 = e + 1 < A.start_n ? e + 1 : 0;
        const double p0x = A.start_xy[2 * e] - c0x, p0y = A.start_xy[2 * e + 1] - c0y;
        const double p1x = A.start_xy[2 * e1] - c0x, p1y = A.start_xy[2 * e1 + 1] - c0y;
        ax = p0y - p1y;
        ay = p1x - p0x;
        b = ax * p0x + ay * p0y;
    }
}

// a cell rebuilt from its row of cut ids
struct CellGeo {
    int m;
    double c0x, c0y, w0;
    double vx[DP_CAP], vy[DP_CAP];
    int id[DP_CAP];
    double cx, cy, mass;
};

// vertices, mass and centroid of cell s (sorted order); false past the
// capacity (or for an edge id this pass does not handle)
__device__ bool cell_geo(const DpArgs &A, long long s, CellGeo &g) {
    const int m = A.nb.cnt[s];
    if (m > DP_CAP) return false;
    g.m = m;
    g.c0x = A.pos[2 * s];
    g.c0y = A.pos[2 * s + 1];
    g.w0 = A.w[s];
    const long long nid = (A.ntrans + 1LL) * A.n;
    for (int k = 0; k < m; ++k) {
        const int id = *A.nb.colp(s, k);
        // a Dirac (or an image) or a domain edge; anything else (an arc) is not handled
        if (id >= 0 ? id >= nid : id > ID_DOMAIN0 || domain_edge(id) >= A.start_n) return false;
        g.id[k] = id;
    }
    // vertex k: the intersection of edges k - 1 and k
    for (int k = 0; k < m; ++k) {
        double a1x, a1y, b1, a2x, a2y, b2;
        edge_line(A, g.id[k == 0 ? m - 1 : k - 1], g.c0x, g.c0y, g.w0, a1x, a1y, b1);
        edge_line(A, g.id[k], g.c0x, g.c0y, g.w0, a2x, a2y, b2);
        const double det = a1x * a2y - a1y * a2x;
        g.vx[k] = g.c0x + (b1 * a2y - b2 * a1y) / det;
        g.vy[k] = g.c0y + (a1x * b2 - a2x * b1) / det;
    }
    // mass and centroid: fan from vertex 0 (add_centroid_contrib, ConvexPolyhedron2.tcc:1047-1074)
    double mass = 0, mx = 0, my = 0;
    for (int k = 2; k < m; ++k) {
        const double ax = g.vx[0], ay = g.vy[0], bx = g.vx[k - 1], by = g.vy[k - 1], cx = g.vx[k], cy = g.vy[k];
        const double lea = 0.5 * (ax * (by - cy) + bx * (cy - ay) + cx * (ay - by)) * A.coeff;
        mx += lea * (1.0 / 3.0) * (ax + bx + cx);
        my += lea * (1.0 / 3.0) * (ay + by + cy);
        mass += lea;
    }
    g.mass = mass;
    g.cx = mass != 0 ? mx / mass : 0.0;
    g.cy = mass != 0 ? my / mass : 0.0;
    return true;
}

// The block of the edge leaving vertex i0 (a Dirac on the other side): t
// receives the off-diagonal block (row-major, rows centroid x, centroid y,
// mass; columns x, y, weight), d0 accumulates the diagonal's share.  Returns
// the caller column.
__device__ long long edge_block(const DpArgs &A, const CellGeo &g, int i0, double *t, double *d0) {
    const int i1 = i0 + 1 < g.m ? i0 + 1 : 0;
    double x1, y1, w1;
    int j;
    other_site(A, g.id[i0], x1, y1, w1, j);
    const double p0[2] = {g.vx[i0], g.vy[i0]}, p1[2] = {g.vx[i1], g.vy[i1]};
    const double l = sqrt((p1[0] - p0[0]) * (p1[0] - p0[0]) + (p1[1] - p0[1]) * (p1[1] - p0[1]));
    const double meas = A.coeff * l;
    const double P[2] = {0.5 * l * (p0[0] + p1[0]), 0.5 * l * (p0[1] + p1[1])};
    double M[2][2];
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            M[a][b] = l / 6 * (2 * (p0[a] * p0[b] + p1[a] * p1[b]) + p0[a] * p1[b] + p1[a] * p0[b]);
    const double c0[2] = {g.c0x, g.c0y}, c1[2] = {x1, y1};
    const double dist = sqrt((x1 - g.c0x) * (x1 - g.c0x) + (y1 - g.c0y) * (y1 - g.c0y));
    const double bd = 0.5 * meas / dist;
    for (int k = 0; k < 9; ++k) t[k] = 0;
    d0[8] += bd;
    t[8] = -bd;
    for (int q = 0; q < 2; ++q) {
        const double value = 0.5 * P[q] / dist;
        d0[3 * q + 2] += value;
        t[3 * q + 2] = -value;
    }
    for (int d = 0; d < 2; ++d) {
        d0[6 + d] += (P[d] - meas * c0[d]) / dist;
        t[6 + d] = (meas * c1[d] - P[d]) / dist;
    }
    for (int d = 0; d < 2; ++d)
        for (int q = 0; q < 2; ++q) {
            d0[3 * q + d] += (M[d][q] - P[q] * c0[d]) / dist;
            t[3 * q + d] = (P[q] * c1[d] - M[d][q]) / dist;
        }
    return A.idx[j];
}

// centroid correction, as the reference divides (.h:178-182)
__device__ void correct(const CellGeo &g, double *t) {
    const double div = g.mass + (g.mass == 1);
    const double c[2] = {g.cx, g.cy};
    for (int r = 0; r < 2; ++r)
        for (int e = 0; e < 3; ++e) t[3 * r + e] = (t[3 * r + e] - t[6 + e] * c[r]) / div;
}

// The row's items in column order: ord[0..cnt) the item indices (edge index,
// or m for the diagonal) sorted by (column, index); col[] their columns.
// Returns the number of items (equal columns not merged yet).
__device__ int sorted_items(const DpArgs &A, long long s, const CellGeo &g, long long *col, unsigned char *ord) {
    int cnt = 0;
    for (int k = 0; k < g.m; ++k) {
        if (g.id[k] < 0) continue;  // a domain edge
        double x, y, w;
        int j;
        other_site(A, g.id[k], x, y, w, j);
        col[k] = A.idx[j];
        ord[cnt++] = (unsigned char)k;
    }
    col[g.m] = A.idx[s];
    ord[cnt++] = (unsigned char)g.m;
    for (int i = 1; i < cnt; ++i) {
        const unsigned char x = ord[i];
        int q = i - 1;
        while (q >= 0 && (col[ord[q]] > col[x] || (col[ord[q]] == col[x] && ord[q] > x))) {
            ord[q + 1] = ord[q];
            --q;
        }
        ord[q + 1] = x;
    }
    return cnt;
}

__device__ int distinct(const long long *col, const unsigned char *ord, int cnt) {
    int d = 0;
    for (int i = 0; i < cnt; ++i) d += i == 0 || col[ord[i]] != col[ord[i - 1]];
    return d;
}

__global__ void k_dp_count(DpArgs A, long long *nblocks, unsigned *err) {
    const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s >= A.n) return;
    CellGeo g;
    long long col[DP_ROW];
    unsigned char ord[DP_ROW];
    long long cnt = 0;
    if (!cell_geo(A, s, g)) {
        atomicOr(err, unsigned(DE_CAPACITY));
    } else {
        cnt = distinct(col, ord, sorted_items(A, s, g, col, ord));
    }
    nblocks[A.idx[s]] = cnt;
}

// block offsets boff (caller order, exclusive scan of the counts) -> CSR of
// 3 n rows: row 3 i + d holds, for every block of Dirac i, its row d; the
// items of one column are corrected, then added in (column, index) order
__global__ void k_dp_write(DpArgs A, const long long *boff, long long *off, long long *cols, double *vals, double *v) {
    const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s >= A.n) return;
    const long long i = A.idx[s];
    const long long base = 9 * boff[i];
    if (s == 0) off[3 * A.n] = 9 * boff[A.n];
    CellGeo g;
    if (!cell_geo(A, s, g)) {
        for (int d = 0; d < 3; ++d) {
            off[3 * i + d] = base;
            v[3 * i + d] = 0;
        }
        return;
    }
    v[3 * i] = g.cx;
    v[3 * i + 1] = g.cy;
    v[3 * i + 2] = g.mass;
    long long col[DP_ROW];
    unsigned char ord[DP_ROW];
    const int items = sorted_items(A, s, g, col, ord);
    const int cnt = distinct(col, ord, items);
    for (int d = 0; d < 3; ++d) off[3 * i + d] = base + 3LL * cnt * d;
    // the diagonal: every edge's share
    double d0[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, t[9], dummy[9];
    for (int k = 0; k < g.m; ++k)
        if (g.id[k] >= 0) edge_block(A, g, k, t, d0);
    correct(g, d0);
    int b = -1;
    double acc[9];
    for (int it = 0; it < items; ++it) {
        const int k = ord[it];
        if (k == g.m) {
            for (int q = 0; q < 9; ++q) t[q] = d0[q];
        } else {
            for (int q = 0; q < 9; ++q) dummy[q] = 0;
            edge_block(A, g, k, t, dummy);
            correct(g, t);
        }
        const bool first = it == 0 || col[ord[it - 1]] != col[k];
        if (first) {
            ++b;
            for (int q = 0; q < 9; ++q) acc[q] = t[q];
        } else {
            for (int q = 0; q < 9; ++q) acc[q] += t[q];
        }
        const bool last = it + 1 == items || col[ord[it + 1]] != col[k];
        if (!last) continue;
        for (int d = 0; d < 3; ++d)
            for (int e = 0; e < 3; ++e) {
                const long long o = base + 3LL * cnt * d + 3 * b + e;
                cols[o] = 3 * col[k] + e;
                vals[o] = acc[3 * d + e];
            }
    }
}

}  // namespace

void derpos_count(const Rows &nb, long long n, const double *pos, const double *w, const int *idx, int start_n,
                  const double *start_xy, double coeff, int ntrans, const double *trans, long long *nblocks,
                  unsigned *err, cudaStream_t st) {
    if (n <= 0) return;
    const DpArgs A{nb, n, pos, w, idx, start_n, start_xy, coeff, ntrans, trans};
    k_dp_count<<<ceil_div(n, TB), TB, 0, st>>>(A, nblocks, err);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}

void derpos_write(const Rows &nb, long long n, const double *pos, const double *w, const int *idx, int start_n,
                  const double *start_xy, double coeff, int ntrans, const double *trans, const long long *boff,
                  long long *off, long long *cols, double *vals, double *v, cudaStream_t st) {
    if (n <= 0) return;
    const DpArgs A{nb, n, pos, w, idx, start_n, start_xy, coeff, ntrans, trans};
    k_dp_write<<<ceil_div(n, TB), TB, 0, st>>>(A, boff, off, cols, vals, v);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}

}  // namespace sdot
