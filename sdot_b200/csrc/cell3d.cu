// 3D Laguerre-cell kernels (see cell3d.cuh).
//
// One warp builds one cell.  The cell is a convex polyhedron held as its
// faces, one face per lane (2, 4 or 8 in the larger passes): each face is a polygon
// (vertices counter-clockwise seen from outside, in coordinates relative to
// the cell's Dirac) whose edge k carries the id of the face across it, plus
// the face's plane a . u <= b and its cut id (a Dirac index, or a domain
// face).  A plane cut is then a 2D polygon cut done by every lane on its own
// face at once, followed by the new face, whose vertices are the points where
// the cut faces enter the cut: starting from one cut face, the next is the
// face across its exit edge.  The point where an edge is cut is computed from
// the edge's inside vertex in both faces that share the edge, so the copies
// agree bitwise and the new face closes exactly.
//
// Reference behaviour restated (ConvexPolyhedron3 and the 3D traversal):
//  * traversal and eviction test: SpZGrid::for_each_laguerre_cell, as in 2D
//    (SpZGrid.tcc:494-719, eviction :475-480), weighted bisector :506-522;
//  * volume: sum over faces of (O . N) area / 3 (ConvexPolyhedron3.tcc:1022-1057),
//    here with the cell's Dirac as the apex (O . N is the signed distance of the
//    face plane from it);
//  * centroid: pyramid centroids weighted by their volumes
//    (ConvexPolyhedron3::add_centroid_contrib, ConvexPolyhedron3.tcc:884-924);
//  * face area by a fan of triangles (ConvexPolyhedron3::area, :1367-1419);
//  * Hessian row: -1/2 coeff area / |x_i - x_j| per neighbour face, the
//    diagonal their sum; domain faces skipped (get_der_integrals_wrt_weights.h:43-88).
//
// Multilinear density (an extension: the reference's 3D densities are
// piecewise constant).  Relative to the cell's Dirac the density is
// sum_k g_k(u), g_k homogeneous of degree k <= 3, and by Euler's identity
// div(u g_k) = (k + 3) g_k, so the pyramid of a face at signed distance h
// holds h/(k+3) times the face integral of g_k (and u g_k, of degree k + 1,
// h/(k+4) times its face integral).  The face integrals use Dunavant's
// degree-4 rule on each fan triangle (6 points; D. A. Dunavant, "High degree
// efficient symmetrical Gaussian quadrature rules for the triangle", IJNME
// 21, 1985), exact for every term here.
#include "cell3d.cuh"

namespace sdot {

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int STACK3 = 96;  // depth <= 10 levels (10 key bits per axis), <= 7 pending siblings each

// Faces of one warp: vertex v of face slot f at [v * MAXF + f].
template <int FPL, int MAXV>
struct Faces {
    static constexpr int MAXF = 32 * FPL;
    double *X, *Y, *Z;
    int *E;
    __device__ int at(int v, int f) const { return v * MAXF + f; }
};

template <int FPL, int MAXV>
constexpr size_t warp_smem_bytes() {
    return size_t(MAXV) * (32 * FPL) * (3 * sizeof(double) + sizeof(int)) + STACK3 * sizeof(int);
}

// One cell's state in a warp: the faces (shared memory) and, per lane and
// face slot r (face lane + 32 r), the face's plane, id and vertex count.
template <int FPL, int MAXV>
struct Cell3 {
    Faces<FPL, MAXV> F;
    int *stack;
    int fid[FPL], nv[FPL];
    double ax[FPL], ay[FPL], az[FPL], b[FPL];
};

__device__ inline double shfl(double v, int src) { return __shfl_sync(FULL, v, src); }

// Outcome of a cut: 0 done, 1 a capacity was exceeded, 2 degenerate geometry.
template <int FPL, int MAXV>
__device__ __forceinline__ int cut3(Cell3<FPL, MAXV> &C, double qx, double qy, double qz, double qb, int qid) {
    const int lane = threadIdx.x & 31;
    auto &F = C.F;
    auto outside = [&](int v, int f) {
        const int i = F.at(v, f);
        return qb - (qx * F.X[i] + qy * F.Y[i] + qz * F.Z[i]) < 0.0;
    };
    // faces of at most 32 vertices keep the classification as a bit mask
    constexpr bool MASKED = MAXV <= 32;
    int nouts[FPL];
    unsigned om[FPL];
    bool has = false;
#pragma unroll
    for (int r = 0; r < FPL; ++r) {
        const int f = lane + 32 * r;
        int c = 0;
        unsigned mk = 0;
        for (int v = 0; v < C.nv[r]; ++v) {
            const bool o = outside(v, f);
            c += o;
            if (MASKED) mk |= unsigned(o) << v;
        }
        nouts[r] = c;
        om[r] = mk;
        has |= c != 0;
    }
    if (!__any_sync(FULL, has)) return 0;
    // ---- cut every face
    bool cut[FPL];
    int exit_nb[FPL];
    double ex[FPL], ey[FPL], ez[FPL];  // entry point of each cut face
    bool bad = false, over = false;
#pragma unroll
    for (int r = 0; r < FPL; ++r) {
        const int f = lane + 32 * r;
        cut[r] = false;
        exit_nb[r] = 0;
        ex[r] = ey[r] = ez[r] = 0;
        const int n = C.nv[r];
        const int nout = nouts[r];
        if (n == 0 || nout == 0) continue;
        if (nout == n) {  // the whole face is removed
            C.nv[r] = 0;
            continue;
        }
        // the outside run: o1 its first vertex (predecessor inside), o2 its
        // last (successor inside); one run only, else the face is cut twice
        int o1 = -1, o2 = -1, runs = 0;
        if (MASKED) {
            // run starts: outside with the previous vertex inside; ends:
            // outside with the next vertex inside (cyclic over n bits)
            const unsigned mk = om[r], valid = n >= 32 ? ~0u : (1u << n) - 1u;
            const unsigned prevm = ((mk << 1) | (mk >> (n - 1))) & valid;
            const unsigned nextm = ((mk >> 1) | ((mk & 1u) << (n - 1))) & valid;
            const unsigned starts = mk & ~prevm, ends = mk & ~nextm;
            runs = __popc(starts);
            o1 = __ffs(int(starts)) - 1;
            o2 = __ffs(int(ends)) - 1;
        } else {
            bool prev = outside(n - 1, f);
            for (int v = 0; v < n; ++v) {
                const bool o = outside(v, f);
                if (o && !prev) {
                    o1 = v;
                    ++runs;
                }
                if (!o && prev) o2 = v == 0 ? n - 1 : v - 1;
                prev = o;
            }
        }
        if (runs != 1 || o1 < 0 || o2 < 0) {
            bad = true;
            continue;
        }
        const int il = o1 == 0 ? n - 1 : o1 - 1;  // last inside vertex before the run
        const int fi = o2 == n - 1 ? 0 : o2 + 1;  // first inside vertex after it
        const int nn = n - nout + 2;
        if (nn > MAXV) {
            over = true;
            continue;
        }
        // the two new points, each from its edge's inside vertex
        auto interp = [&](int vin, int vout, double &px, double &py, double &pz) {
            const int a = F.at(vin, f), c = F.at(vout, f);
            const double din = qb - (qx * F.X[a] + qy * F.Y[a] + qz * F.Z[a]);
            const double dout = qb - (qx * F.X[c] + qy * F.Y[c] + qz * F.Z[c]);
            const double t = din / (din - dout);
            px = F.X[a] + t * (F.X[c] - F.X[a]);
            py = F.Y[a] + t * (F.Y[c] - F.Y[a]);
            pz = F.Z[a] + t * (F.Z[c] - F.Z[a]);
        };
        double xx, xy, xz, nx, ny, nz;
        interp(il, o1, xx, xy, xz);  // exit point, on edge il -> o1
        interp(fi, o2, nx, ny, nz);  // entry point, on edge o2 -> fi
        const int xnb = F.E[F.at(il, f)], nnb = F.E[F.at(o2, f)];
        auto move = [&](int dst, int src) {
            const int a = F.at(dst, f), c = F.at(src, f);
            F.X[a] = F.X[c];
            F.Y[a] = F.Y[c];
            F.Z[a] = F.Z[c];
            F.E[a] = F.E[c];
        };
        int px_at;  // index of the exit point in the new polygon
        if (o1 <= o2) {
            // outside run inside the list: [0, o1) X N [o2 + 1, n)
            const int delta = (o1 + 2) - (o2 + 1);
            if (delta > 0)
                for (int k = n - 1; k > o2; --k) move(k + delta, k);
            else if (delta < 0)
                for (int k = o2 + 1; k < n; ++k) move(k + delta, k);
            px_at = o1;
        } else {
            // the outside run wraps: inside run [o2 + 1, o1) moves to the front
            const int m = o1 - o2 - 1;
            for (int k = 0; k < m; ++k) move(k, o2 + 1 + k);
            px_at = m;
        }
        const int a0 = F.at(px_at, f), a1 = F.at(px_at + 1, f);
        F.X[a0] = xx;
        F.Y[a0] = xy;
        F.Z[a0] = xz;
        F.E[a0] = qid;
        F.X[a1] = nx;
        F.Y[a1] = ny;
        F.Z[a1] = nz;
        F.E[a1] = nnb;
        C.nv[r] = nn;
        cut[r] = true;
        exit_nb[r] = xnb;
        ex[r] = nx;
        ey[r] = ny;
        ez[r] = nz;
    }
    if (__any_sync(FULL, bad)) return 2;
    if (__any_sync(FULL, over)) return 1;
    // ---- the new face: a free slot, vertices chained over the cut faces
    unsigned cutm[FPL], freem[FPL];
#pragma unroll
    for (int r = 0; r < FPL; ++r) {
        cutm[r] = __ballot_sync(FULL, cut[r]);
        freem[r] = __ballot_sync(FULL, C.nv[r] == 0);
    }
    int m = 0, slot = -1, start = -1;
#pragma unroll
    for (int r = 0; r < FPL; ++r) {
        m += __popc(cutm[r]);
        if (slot < 0 && freem[r]) slot = 32 * r + __ffs(freem[r]) - 1;
        if (start < 0 && cutm[r]) start = 32 * r + __ffs(cutm[r]) - 1;
    }
    if (m == 0) return 0;  // only whole faces were removed
    if (m < 3) return 2;
    if (slot < 0 || m > MAXV) return 1;
    int cur = start;
    for (int i = 0; i < m; ++i) {
        // broadcast the current cut face's entry point, exit neighbour and id
        const int cl = cur & 31, cr = cur >> 5;
        double px = 0, py = 0, pz = 0;
        int nb = 0, id = 0;
#pragma unroll
        for (int r = 0; r < FPL; ++r)
            if (r == cr) {
                px = shfl(ex[r], cl);
                py = shfl(ey[r], cl);
                pz = shfl(ez[r], cl);
                nb = __shfl_sync(FULL, exit_nb[r], cl);
                id = __shfl_sync(FULL, C.fid[r], cl);
            }
        if (lane == (slot & 31)) {
            const int a = F.at(i, slot);
            F.X[a] = px;
            F.Y[a] = py;
            F.Z[a] = pz;
            F.E[a] = id;
        }
        // next: the cut face whose id is the exit neighbour
        int next = -1;
#pragma unroll
        for (int r = 0; r < FPL; ++r) {
            const unsigned hit = __ballot_sync(FULL, cut[r] && C.fid[r] == nb);
            if (next < 0 && hit) next = 32 * r + __ffs(hit) - 1;
        }
        if (next < 0) return 2;
        cur = next;
    }
    if (cur != start) return 2;
#pragma unroll
    for (int r = 0; r < FPL; ++r)
        if (lane + 32 * r == slot) {
            C.fid[r] = qid;
            C.nv[r] = m;
            C.ax[r] = qx;
            C.ay[r] = qy;
            C.az[r] = qz;
            C.b[r] = qb;
        }
    __syncwarp();
    return 0;
}

// A multilinear density rewritten about the cell's Dirac c: coefficients of
// 1, u_x, u_y, u_z, u_x u_y, u_x u_z, u_y u_z, u_x u_y u_z for u = x - c.
struct PolyRel {
    double b1, bx, by, bz, bxy, bxz, byz, bxyz;
    __device__ PolyRel(const double *a, double cx, double cy, double cz) {
        bxyz = a[7];
        bxy = a[4] + a[7] * cz;
        bxz = a[5] + a[7] * cy;
        byz = a[6] + a[7] * cx;
        bx = a[1] + a[4] * cy + a[5] * cz + a[7] * cy * cz;
        by = a[2] + a[4] * cx + a[6] * cz + a[7] * cx * cz;
        bz = a[3] + a[5] * cx + a[6] * cy + a[7] * cx * cy;
        b1 = a[0] + a[1] * cx + a[2] * cy + a[3] * cz + a[4] * cx * cy + a[5] * cx * cz + a[6] * cy * cz +
             a[7] * cx * cy * cz;
    }
    // One point q (relative coordinates) of a face rule with weight wt:
    // pm += wt * sum_k g_k(q)/(k+3), pd += wt * q * sum_k g_k(q)/(k+4),
    // pf += wt * sum_k g_k(q).
    __device__ void add(double qx, double qy, double qz, double wt, double &pm, double &pdx, double &pdy, double &pdz,
                        double &pf) const {
        const double g0 = b1;
        const double g1 = bx * qx + by * qy + bz * qz;
        const double g2 = bxy * qx * qy + bxz * qx * qz + byz * qy * qz;
        const double g3 = bxyz * qx * qy * qz;
        pm += wt * (g0 * (1.0 / 3) + g1 * 0.25 + g2 * 0.2 + g3 * (1.0 / 6));
        const double gd = wt * (g0 * 0.25 + g1 * 0.2 + g2 * (1.0 / 6) + g3 * (1.0 / 7));
        pdx += gd * qx;
        pdy += gd * qy;
        pdz += gd * qz;
        pf += wt * (g0 + g1 + g2 + g3);
    }
    // Dunavant's degree-4 rule on the triangle p0, p0 + e1, p0 + e2 of area ta.
    __device__ void triangle(double x0, double y0, double z0, double e1x, double e1y, double e1z, double e2x,
                             double e2y, double e2z, double ta, double &pm, double &pdx, double &pdy, double &pdz,
                             double &pf) const {
        constexpr double A[2] = {0.4459484909159648863, 0.0915762135097707435};
        constexpr double W[2] = {0.2233815896780114657, 0.1099517436553218676};
#pragma unroll
        for (int g = 0; g < 2; ++g) {
            const double a = A[g], b = 1.0 - 2.0 * A[g], wt = W[g] * ta;
            add(x0 + a * (e1x + e2x), y0 + a * (e1y + e2y), z0 + a * (e1z + e2z), wt, pm, pdx, pdy, pdz, pf);
            add(x0 + b * e1x + a * e2x, y0 + b * e1y + a * e2y, z0 + b * e1z + a * e2z, wt, pm, pdx, pdy, pdz, pf);
            add(x0 + a * e1x + b * e2x, y0 + a * e1y + b * e2y, z0 + a * e1z + b * e2z, wt, pm, pdx, pdy, pdz, pf);
        }
    }
};

// The domain box as six faces (slots 0..5), relative to c0.
template <int FPL, int MAXV>
__device__ __forceinline__ void init_box(Cell3<FPL, MAXV> &C, const Cell3DArgs &A, double c0x, double c0y, double c0z) {
    const int lane = threadIdx.x & 31;
    const double lo[3] = {A.box_lo[0] - c0x, A.box_lo[1] - c0y, A.box_lo[2] - c0z};
    const double hi[3] = {A.box_hi[0] - c0x, A.box_hi[1] - c0y, A.box_hi[2] - c0z};
    // corners: bit 0 -> x, bit 1 -> y, bit 2 -> z (0: lo, 1: hi)
    // per face: 4 corners counter-clockwise seen from outside, and the face
    // across each edge (faces: 0 x-lo, 1 x-hi, 2 y-lo, 3 y-hi, 4 z-lo, 5 z-hi)
    constexpr int corner[6][4] = {{0, 4, 6, 2}, {1, 3, 7, 5}, {0, 1, 5, 4}, {2, 6, 7, 3}, {0, 2, 3, 1}, {4, 5, 7, 6}};
    constexpr int across[6][4] = {{2, 5, 3, 4}, {4, 3, 5, 2}, {4, 1, 5, 0}, {0, 5, 1, 4}, {0, 3, 1, 2}, {2, 1, 3, 0}};
#pragma unroll
    for (int r = 0; r < FPL; ++r) {
        const int f = lane + 32 * r;
        C.nv[r] = 0;
        C.fid[r] = 0;
        C.ax[r] = C.ay[r] = C.az[r] = C.b[r] = 0;
        if (f < 6) {
            const int ax = f >> 1, side = f & 1;
            C.nv[r] = 4;
            C.fid[r] = domain_id(f);
            double nrm[3] = {0, 0, 0};
            nrm[ax] = side ? 1.0 : -1.0;
            C.ax[r] = nrm[0];
            C.ay[r] = nrm[1];
            C.az[r] = nrm[2];
            C.b[r] = side ? hi[ax] : -lo[ax];
            for (int v = 0; v < 4; ++v) {
                const int c = corner[f][v];
                const int a = C.F.at(v, f);
                C.F.X[a] = (c & 1) ? hi[0] : lo[0];
                C.F.Y[a] = (c & 2) ? hi[1] : lo[1];
                C.F.Z[a] = (c & 4) ? hi[2] : lo[2];
                C.F.E[a] = domain_id(across[f][v]);
            }
        }
    }
    __syncwarp();
}

// Writes a row of `cnt` entries: the lanes' neighbour faces (slot r of a
// lane writes entry pos[r] when mine[r]), then the diagonal from lane 0 when
// with_diag, into the ELL slots or, for a long row, the side buffer.
template <int FPL>
__device__ __forceinline__ bool write_row(const Rows &R, long long s, int cnt, const int *pos, const bool *mine, const int *col,
                          const double *val, bool with_diag, int diag_col, double diag_val) {
    const int lane = threadIdx.x & 31;
    long long off = 0;
    const bool side = cnt > R.cap;
    if (side) {
        unsigned long long o = 0;
        if (lane == 0) o = atomicAdd(R.side_used, (unsigned long long)cnt);
        o = __shfl_sync(FULL, o, 0);
        if ((long long)(o + cnt) > R.side_cap) return false;
        off = (long long)o;
        if (lane == 0) R.side[s] = off;
    }
    auto put = [&](int k, int c, double v) {
        if (side) {
            R.side_col[off + k] = c;
            if (R.side_val) R.side_val[off + k] = v;
        } else {
            R.col[k * R.stride + s] = c;
            if (R.val) R.val[k * R.stride + s] = v;
        }
    };
#pragma unroll
    for (int r = 0; r < FPL; ++r)
        if (mine[r]) put(pos[r], col[r], val[r]);
    if (with_diag && lane == 0) put(cnt - 1, diag_col, diag_val);
    if (lane == 0) R.cnt[s] = cnt;
    return true;
}

// First failed guard of a 3D cell (the 2D kernels' guard_fail).
__device__ void guard_fail3(const Cell3DArgs &A, int code, long long s, long long value) {
    if (A.guard && atomicCAS(&A.guard[0], 0, code) == 0) {
        A.guard[1] = int(s);
        A.guard[2] = int(value);
    }
    flag_error(A.err, DE_GUARD);
}

// Volume, first moments (relative to c0) and per face slot the area of the
// faces of C, the pyramids of apex c0 over the faces (this lane's slots only;
// the caller sums over the warp).  Constant density.
template <int FPL, int MAXV>
__device__ __forceinline__ void face_volumes(const Cell3<FPL, MAXV> &C, double &vol, double &mx, double &my, double &mz,
                             double *area_r) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int r = 0; r < FPL; ++r) {
        const int f = lane + 32 * r;
        const int n = C.nv[r];
        area_r[r] = 0;
        if (n < 3) continue;
        const double na = sqrt(C.ax[r] * C.ax[r] + C.ay[r] * C.ay[r] + C.az[r] * C.az[r]);
        const double ux = C.ax[r] / na, uy = C.ay[r] / na, uz = C.az[r] / na;
        const int i0 = C.F.at(0, f);
        const double x0 = C.F.X[i0], y0 = C.F.Y[i0], z0 = C.F.Z[i0];
        double area = 0, fx = 0, fy = 0, fz = 0;
        for (int k = 1; k + 1 < n; ++k) {
            const int i1 = C.F.at(k, f), i2 = C.F.at(k + 1, f);
            const double e1x = C.F.X[i1] - x0, e1y = C.F.Y[i1] - y0, e1z = C.F.Z[i1] - z0;
            const double e2x = C.F.X[i2] - x0, e2y = C.F.Y[i2] - y0, e2z = C.F.Z[i2] - z0;
            const double ta =
                0.5 * ((e1y * e2z - e1z * e2y) * ux + (e1z * e2x - e1x * e2z) * uy + (e1x * e2y - e1y * e2x) * uz);
            area += ta;
            fx += ta * (3 * x0 + e1x + e2x);
            fy += ta * (3 * y0 + e1y + e2y);
            fz += ta * (3 * z0 + e1z + e2z);
        }
        const double h = C.b[r] / na;
        const double v = h * area / 3;
        vol += v;
        if (area != 0) {
            const double k = v * 0.75 / (3 * area);
            mx += k * fx;
            my += k * fy;
            mz += k * fz;
        }
        area_r[r] = area;
    }
}

// The cell integrated voxel by voxel (ScaledImage::for_each_intersection,
// ScaledImage.tcc:98-149: each voxel box intersected with the cell and
// integrated with the voxel's value): the faces are saved to the warp's
// backup, and for every voxel that the cell's bounding box meets the faces
// are restored and cut by the voxel's six planes, then integrated.  Sums
// (this lane's slots) into vol, m*, and per slot the value-weighted area of
// the Dirac faces.  Returns 0, or 1 / 2 as cut3 (capacity, degenerate).
template <int FPL, int MAXV>
__device__ __forceinline__ int voxel_integrals(const Cell3DArgs &A, Cell3<FPL, MAXV> &C, char *backup, double c0x, double c0y,
                               double c0z, double &vol, double &mx, double &my, double &mz, double *wa_r) {
    const int lane = threadIdx.x & 31;
    Faces<FPL, MAXV> B;
    constexpr int MAXF = 32 * FPL;
    B.X = reinterpret_cast<double *>(backup);
    B.Y = B.X + MAXV * MAXF;
    B.Z = B.Y + MAXV * MAXF;
    B.E = reinterpret_cast<int *>(B.Z + MAXV * MAXF);
    int fid0[FPL], nv0[FPL];
    double ax0[FPL], ay0[FPL], az0[FPL], b0[FPL];
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
#pragma unroll
    for (int r = 0; r < FPL; ++r) {
        const int f = lane + 32 * r;
        fid0[r] = C.fid[r];
        nv0[r] = C.nv[r];
        ax0[r] = C.ax[r];
        ay0[r] = C.ay[r];
        az0[r] = C.az[r];
        b0[r] = C.b[r];
        wa_r[r] = 0;
        for (int v = 0; v < C.nv[r]; ++v) {
            const int i = C.F.at(v, f);
            B.X[i] = C.F.X[i];
            B.Y[i] = C.F.Y[i];
            B.Z[i] = C.F.Z[i];
            B.E[i] = C.F.E[i];
            lo[0] = fmin(lo[0], C.F.X[i]); hi[0] = fmax(hi[0], C.F.X[i]);
            lo[1] = fmin(lo[1], C.F.Y[i]); hi[1] = fmax(hi[1], C.F.Y[i]);
            lo[2] = fmin(lo[2], C.F.Z[i]); hi[2] = fmax(hi[2], C.F.Z[i]);
        }
    }
    for (int d = 0; d < 3; ++d)
        for (int o = 16; o > 0; o >>= 1) {
            lo[d] = fmin(lo[d], __shfl_xor_sync(FULL, lo[d], o));
            hi[d] = fmax(hi[d], __shfl_xor_sync(FULL, hi[d], o));
        }
    __syncwarp();
    if (!(lo[0] <= hi[0])) return 0;  // an empty cell
    const double c0[3] = {c0x, c0y, c0z};
    int i0[3], i1[3];
    double ps[3];
    for (int d = 0; d < 3; ++d) {
        ps[d] = (A.img_hi[d] - A.img_lo[d]) / A.img_n[d];
        i0[d] = max(0, int(floor((lo[d] + c0[d] - A.img_lo[d]) / ps[d])));
        i1[d] = min(A.img_n[d] - 1, int(floor((hi[d] + c0[d] - A.img_lo[d]) / ps[d])));
    }
    for (int iz = i0[2]; iz <= i1[2]; ++iz)
        for (int iy = i0[1]; iy <= i1[1]; ++iy)
            for (int ix = i0[0]; ix <= i1[0]; ++ix) {
                const double val = A.img[((long long)iz * A.img_n[1] + iy) * A.img_n[0] + ix];
                // restore the cell
#pragma unroll
                for (int r = 0; r < FPL; ++r) {
                    const int f = lane + 32 * r;
                    C.fid[r] = fid0[r];
                    C.nv[r] = nv0[r];
                    C.ax[r] = ax0[r];
                    C.ay[r] = ay0[r];
                    C.az[r] = az0[r];
                    C.b[r] = b0[r];
                    for (int v = 0; v < nv0[r]; ++v) {
                        const int i = C.F.at(v, f);
                        C.F.X[i] = B.X[i];
                        C.F.Y[i] = B.Y[i];
                        C.F.Z[i] = B.Z[i];
                        C.F.E[i] = B.E[i];
                    }
                }
                __syncwarp();
                // the voxel's six planes, relative to c0
                const int ii[3] = {ix, iy, iz};
                for (int d = 0; d < 3; ++d) {
                    const double vlo = A.img_lo[d] + ps[d] * ii[d] - c0[d];
                    const double vhi = A.img_lo[d] + ps[d] * (ii[d] + 1) - c0[d];
                    double a[3] = {0, 0, 0};
                    a[d] = -1.0;
                    int st = cut3(C, a[0], a[1], a[2], -vlo, domain_id(200 + 2 * d));
                    if (st) return st;
                    a[d] = 1.0;
                    st = cut3(C, a[0], a[1], a[2], vhi, domain_id(201 + 2 * d));
                    if (st) return st;
                }
                double v = 0, px = 0, py = 0, pz = 0, ar[FPL];
                face_volumes(C, v, px, py, pz, ar);
                vol += val * v;
                mx += val * px;
                my += val * py;
                mz += val * pz;
#pragma unroll
                for (int r = 0; r < FPL; ++r)
                    if (C.fid[r] >= 0 && C.nv[r] >= 3) wa_r[r] += val * ar[r];
            }
    // restore the cell for the outputs that follow (its faces' ids and planes)
#pragma unroll
    for (int r = 0; r < FPL; ++r) {
        const int f = lane + 32 * r;
        C.fid[r] = fid0[r];
        C.nv[r] = nv0[r];
        C.ax[r] = ax0[r];
        C.ay[r] = ay0[r];
        C.az[r] = az0[r];
        C.b[r] = b0[r];
        for (int v = 0; v < nv0[r]; ++v) {
            const int i = C.F.at(v, f);
            C.F.X[i] = B.X[i];
            C.F.Y[i] = B.Y[i];
            C.F.Z[i] = B.Z[i];
            C.F.E[i] = B.E[i];
        }
    }
    __syncwarp();
    return 0;
}

// Builds and integrates the cell of sorted Dirac s.  Returns 0 (outputs
// written), 1 (a capacity was exceeded: retry in the large pass), 2 (failed:
// outputs written as NaN / empty row, error flagged).
template <int FPL, int MAXV>
__device__ __forceinline__ int cell3d(const Cell3DArgs &A, long long s, Cell3<FPL, MAXV> &C, char *backup) {
    const int lane = threadIdx.x & 31;
    const double c0x = A.pos[3 * s], c0y = A.pos[3 * s + 1], c0z = A.pos[3 * s + 2], w0 = A.w[s];
    init_box(C, A, c0x, c0y, c0z);
    int status = 0;
    // a convex shape: its half-spaces cut the box first (relative to c0:
    // a . u <= b - a . c0), as ConvexPolyhedronAssembly::add_convex_polyhedron
    // cuts its box (ConvexPolyhedronAssembly.tcc:7-33)
    for (int k = 0; k < A.nplanes && status == 0; ++k) {
        const double ax = A.planes[4 * k], ay = A.planes[4 * k + 1], az = A.planes[4 * k + 2];
        const double b = A.planes[4 * k + 3] - (ax * c0x + ay * c0y + az * c0z);
        const int r = cut3(C, ax, ay, az, b, domain_id(6 + k));
        if (r) status = r;
    }
    if (lane == 0) C.stack[0] = 0;
    __syncwarp();
    int sp = 1;
    for (int visits = 0; sp > 0 && status == 0; ++visits) {
        if (visits > A.max_nodes) {
            if (lane == 0) flag_error(A.err, DE_ITER);
            status = 2;
            break;
        }
        const int node = C.stack[--sp];
        __syncwarp();
        const TreeNode<3> nd = A.nodes[node];
        // eviction test (SpZGrid.tcc:475-480) on every vertex of every face
        const double lo0 = nd.lo[0] - c0x, lo1 = nd.lo[1] - c0y, lo2 = nd.lo[2] - c0z;
        const double hi0 = nd.hi[0] - c0x, hi1 = nd.hi[1] - c0y, hi2 = nd.hi[2] - c0z;
        bool fail = false;
#pragma unroll
        for (int r = 0; r < FPL; ++r) {
            const int f = lane + 32 * r;
            for (int v = 0; v < C.nv[r] && !fail; ++v) {
                const int i = C.F.at(v, f);
                const double px = C.F.X[i], py = C.F.Y[i], pz = C.F.Z[i];
                const double qx = fmin(hi0, fmax(lo0, px)) - px, qy = fmin(hi1, fmax(lo1, py)) - py,
                             qz = fmin(hi2, fmax(lo2, pz)) - pz;
                const double lhs = px * px + py * py + pz * pz - w0;
                const double rhs = qx * qx + qy * qy + qz * qz - nd.maxw;
                fail = !(lhs <= rhs);
            }
        }
        if (!__any_sync(FULL, fail)) continue;
        if (nd.b < 0) {
            const int first = nd.a, nch = -nd.b;
            if (nch < 2 || nch > 8 || first < 1 || first + nch > A.max_nodes) {
                if (lane == 0) guard_fail3(A, 1, s, node);
                status = 2;
                break;
            }
            if (sp + nch > STACK3) {
                if (lane == 0) flag_error(A.err, DE_STACK);
                status = 2;
                break;
            }
            // children farthest first (nearest popped first): lane c keys child
            // c and writes it at its rank among the keys (larger keys first,
            // equal keys in child order, as a stable sort would place them)
            float key = 0;
            if (lane < nch) {
                const TreeNode<3> &cn = A.nodes[first + lane];
                const double mx = 0.5 * (cn.lo[0] + cn.hi[0]) - c0x, my = 0.5 * (cn.lo[1] + cn.hi[1]) - c0y,
                             mz = 0.5 * (cn.lo[2] + cn.hi[2]) - c0z;
                key = float(mx * mx + my * my + mz * mz);
            }
            int rank = 0;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const float kc = __shfl_sync(FULL, key, c);
                rank += c < nch && (kc > key || (kc == key && c < lane));
            }
            if (lane < nch) C.stack[sp + rank] = first + lane;
            __syncwarp();
            sp += nch;
        } else {
            if (nd.a < 0 || nd.b > A.n) {
                if (lane == 0) guard_fail3(A, 2, s, node);
                status = 2;
                break;
            }
            for (int j = nd.a; j < nd.b && status == 0; ++j) {
                if (j == s) continue;
                // weighted bisector, relative to c0: V . u <= 1/2 |V|^2 + 1/2 (w0 - w1)
                const double vx = A.pos[3 * j] - c0x, vy = A.pos[3 * j + 1] - c0y, vz = A.pos[3 * j + 2] - c0z;
                const double qb = 0.5 * (vx * vx + vy * vy + vz * vz) + 0.5 * (w0 - A.w[j]);
                const int r = cut3(C, vx, vy, vz, qb, j);
                if (r) status = r;
            }
        }
    }
    if (status == 1) return 1;
    // ---- integrals over the faces (pyramids with apex c0)
    double vol = 0, mx = 0, my = 0, mz = 0, der0 = 0;
    int nrow = 0, nnb = 0;
    int rpos[FPL], npos[FPL];
    double rval[FPL];
    bool rmine[FPL], nmine[FPL];
    double img_area[FPL];  // voxel image: the value-weighted area of each Dirac face
    if (status == 0 && A.img) {
        status = voxel_integrals(A, C, backup, c0x, c0y, c0z, vol, mx, my, mz, img_area);
        if (status == 1) return 1;
    }
    if (status == 0) {
        const bool poly = A.has_poly;
        const PolyRel pr(A.poly, c0x, c0y, c0z);
#pragma unroll
        for (int r = 0; r < FPL; ++r) {
            const int f = lane + 32 * r;
            const int n = C.nv[r];
            rmine[r] = false;
            nmine[r] = n > 0;
            rval[r] = 0;
            if (n < 3) continue;
            const double na = sqrt(C.ax[r] * C.ax[r] + C.ay[r] * C.ay[r] + C.az[r] * C.az[r]);
            if (A.img) {
                // integrated voxel by voxel above
                if (C.fid[r] >= 0) {
                    const double bd = 0.5 * A.coeff * img_area[r] / na;
                    rmine[r] = true;
                    rval[r] = -bd;
                    der0 += bd;
                }
                continue;
            }
            const double ux = C.ax[r] / na, uy = C.ay[r] / na, uz = C.az[r] / na;
            const int i0 = C.F.at(0, f);
            const double x0 = C.F.X[i0], y0 = C.F.Y[i0], z0 = C.F.Z[i0];
            double area = 0, fx = 0, fy = 0, fz = 0;
            double pm = 0, pdx = 0, pdy = 0, pdz = 0, pf = 0;  // density-weighted (poly)
            for (int k = 1; k + 1 < n; ++k) {
                const int i1 = C.F.at(k, f), i2 = C.F.at(k + 1, f);
                const double e1x = C.F.X[i1] - x0, e1y = C.F.Y[i1] - y0, e1z = C.F.Z[i1] - z0;
                const double e2x = C.F.X[i2] - x0, e2y = C.F.Y[i2] - y0, e2z = C.F.Z[i2] - z0;
                const double ta = 0.5 * ((e1y * e2z - e1z * e2y) * ux + (e1z * e2x - e1x * e2z) * uy +
                                         (e1x * e2y - e1y * e2x) * uz);
                if (poly) {
                    pr.triangle(x0, y0, z0, e1x, e1y, e1z, e2x, e2y, e2z, ta, pm, pdx, pdy, pdz, pf);
                } else {
                    area += ta;
                    fx += ta * (3 * x0 + e1x + e2x);
                    fy += ta * (3 * y0 + e1y + e2y);
                    fz += ta * (3 * z0 + e1z + e2z);
                }
            }
            const double h = C.b[r] / na;  // signed distance of the face plane from c0
            if (poly) {
                vol += h * pm;
                mx += h * pdx;
                my += h * pdy;
                mz += h * pdz;
                area = pf;  // the face's density integral
            } else {
                const double v = h * area / 3;
                vol += v;
                // pyramid centroid: 3/4 of the way from the apex to the face centroid
                if (area != 0) {
                    const double k = v * 0.75 / (3 * area);
                    mx += k * fx;
                    my += k * fy;
                    mz += k * fz;
                }
            }
            if (C.fid[r] >= 0) {
                const double bd = 0.5 * A.coeff * area / na;  // |x_i - x_j| = |a|
                rmine[r] = true;
                rval[r] = -bd;
                der0 += bd;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            vol += __shfl_xor_sync(FULL, vol, o);
            mx += __shfl_xor_sync(FULL, mx, o);
            my += __shfl_xor_sync(FULL, my, o);
            mz += __shfl_xor_sync(FULL, mz, o);
            der0 += __shfl_xor_sync(FULL, der0, o);
        }
        // positions of the row and neighbour entries: slot order
        const unsigned below = (1u << lane) - 1u;
#pragma unroll
        for (int r = 0; r < FPL; ++r) {
            const unsigned rm = __ballot_sync(FULL, rmine[r]), nm = __ballot_sync(FULL, nmine[r]);
            rpos[r] = nrow + __popc(rm & below);
            npos[r] = nnb + __popc(nm & below);
            nrow += __popc(rm);
            nnb += __popc(nm);
        }
    }
    bool ok = true;  // the rows fit the side buffer
    if (status == 0 && A.hint) {
        // the smallest pass that holds this polyhedron (faces, vertices per face)
        int faces = 0, maxv = 0;
#pragma unroll
        for (int r = 0; r < FPL; ++r) {
            faces += __popc(__ballot_sync(FULL, C.nv[r] > 0));
            maxv = max(maxv, C.nv[r]);
        }
        for (int o = 16; o > 0; o >>= 1) maxv = max(maxv, __shfl_xor_sync(FULL, maxv, o));
        const int level = (faces <= 32 && maxv <= 16) ? 0 : (faces <= 64 && maxv <= 32) ? 1
                          : (faces <= 128 && maxv <= 64) ? 2 : 3;
        // polyhedra grow larger during the build than at its end, so the
        // hint is the pass that held this build, lowered by one level at most
        // when the final polyhedron is smaller (a cell that then overflows
        // simply moves on to the next pass again)
        constexpr int pass = FPL == 1 ? 0 : FPL == 2 ? 1 : FPL == 4 ? 2 : 3;
        const int hint = level >= pass ? pass : pass - 1;
        if (lane == 0) A.hint[s] = (unsigned char)hint;
    }
    if (status == 0) {
        const double mass = A.coeff * vol;
        if (lane == 0) {
            if (A.mass) A.mass[s] = mass;
            if (A.ctd) {
                const bool empty = vol == 0;
                A.ctd[3 * s] = empty ? 0.0 : c0x + mx / vol;
                A.ctd[3 * s + 1] = empty ? 0.0 : c0y + my / vol;
                A.ctd[3 * s + 2] = empty ? 0.0 : c0z + mz / vol;
            }
        }
        if (A.rows.cnt) ok &= write_row<FPL>(A.rows, s, nrow + 1, rpos, rmine, C.fid, rval, true, int(s), der0);
        if (A.nb.cnt) ok &= write_row<FPL>(A.nb, s, nnb, npos, nmine, C.fid, rval, false, 0, 0.0);
        ok = __all_sync(FULL, ok);
    }
    if (status == 2 || !ok) {
        if (lane == 0) {
            flag_error(A.err, status == 2 ? DE_DEGEN : DE_SIDE);
            if (A.mass) A.mass[s] = nan("");
            if (A.ctd) A.ctd[3 * s] = A.ctd[3 * s + 1] = A.ctd[3 * s + 2] = nan("");
            if (A.rows.cnt) {
                A.rows.cnt[s] = 1;
                A.rows.col[s] = int(s);
                A.rows.val[s] = 0.0;
            }
            if (A.nb.cnt) A.nb.cnt[s] = 0;
        }
        return 2;
    }
    return 0;
}

// The faces of a warp live in shared memory, or, for the largest capacity,
// in global scratch (gscratch != null: WB bytes per warp).
// Launch shapes of the passes: the first runs two warps per block (seven
// blocks per SM, bounded by shared memory), the others one warp per block
// (three per SM for the second pass, eight for the global-scratch passes);
// the bounds let the compiler use every register those counts leave (128 in
// the first pass, up to 255 in the others, which then spill little or not at
// all: 8.7% faster on the 200k 3D mix, 3% on the largest serving request,
// than the compiler's own choice under a bound of 64 threads alone).
constexpr int k3_threads(int fpl) { return fpl == 1 ? 64 : 32; }
constexpr int k3_min_blocks(int fpl) { return fpl == 1 ? 7 : fpl == 2 ? 3 : 8; }

template <int FPL, int MAXV>
__global__ void __launch_bounds__(k3_threads(FPL), k3_min_blocks(FPL)) k_cells3d(const Cell3DArgs A, const int *list, const int *list_cnt,
                                                int *next_list, int *next_cnt, int nwarps, char *gscratch) {
    extern __shared__ double smem3[];
    constexpr int MAXF = 32 * FPL;
    constexpr size_t WB = warp_smem_bytes<FPL, MAXV>();
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gw = blockIdx.x * (blockDim.x >> 5) + wib;
    char *base = gscratch ? gscratch + WB * size_t(gw) : reinterpret_cast<char *>(smem3) + WB * wib;
    Cell3<FPL, MAXV> C;
    C.F.X = reinterpret_cast<double *>(base);
    C.F.Y = C.F.X + MAXV * MAXF;
    C.F.Z = C.F.Y + MAXV * MAXF;
    C.F.E = reinterpret_cast<int *>(C.F.Z + MAXV * MAXF);
    C.stack = C.F.E + MAXV * MAXF;
    const long long cnt = list ? *list_cnt : A.n;
    for (long long i = gw; i < cnt; i += nwarps) {
        const long long s = list ? list[i] : i;
        if (!list && A.use_hint && A.hint) {
            // a cell that needed a larger pass last time goes straight there
            const int h = A.hint[s];
            int *to = h == 1 ? next_list : h == 2 ? A.ovf_list2 : h == 3 ? A.ovf_list3 : nullptr;
            int *tc = h == 1 ? next_cnt : h == 2 ? A.ovf_cnt2 : h == 3 ? A.ovf_cnt3 : nullptr;
            if (to && tc) {
                if (lane == 0) to[atomicAdd(tc, 1)] = int(s);
                __syncwarp();
                continue;
            }
        }
        const int r = cell3d<FPL, MAXV>(A, s, C, A.img_backup ? A.img_backup + WB * size_t(gw) : nullptr);
        if (r == 1) {
            if (next_list) {
                if (lane == 0) next_list[atomicAdd(next_cnt, 1)] = int(s);
            } else if (lane == 0) {
                flag_error(A.err, DE_CAPACITY);
                if (A.mass) A.mass[s] = nan("");
                if (A.ctd) A.ctd[3 * s] = A.ctd[3 * s + 1] = A.ctd[3 * s + 2] = nan("");
                if (A.rows.cnt) {
                    A.rows.cnt[s] = 1;
                    A.rows.col[s] = int(s);
                    A.rows.val[s] = 0.0;
                }
                if (A.nb.cnt) A.nb.cnt[s] = 0;
            }
        }
        __syncwarp();
    }
}

template <int FPL, int MAXV, int WPB>
void launch3(const Cell3DArgs &a, const int *list, const int *list_cnt, int *next_list, int *next_cnt, long long ncells,
             char *gscratch, long long max_blocks, cudaStream_t st) {
    const size_t smem = gscratch ? 0 : warp_smem_bytes<FPL, MAXV>() * WPB;
    static PerDevice<int> attr;
    if (!gscratch)
        attr.once([&] {
            SDOT_CUDA(cudaFuncSetAttribute(k_cells3d<FPL, MAXV>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        });
    long long blocks = (ncells + WPB - 1) / WPB;
    if (blocks > max_blocks) blocks = max_blocks;
    if (blocks < 1) blocks = 1;
    k_cells3d<FPL, MAXV><<<int(blocks), 32 * WPB, smem, st>>>(a, list, list_cnt, next_list, next_cnt,
                                                               int(blocks) * WPB, gscratch);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}

// warps of the third and fourth passes (faces in global memory, 230 KB and
// 918 KB per warp; the two passes share the scratch, 1.09 GB): 8 per SM,
// the most that the fourth pass's registers let an SM hold
constexpr long long G3_WARPS = 148 * 8;

}  // namespace

constexpr long long G4_WARPS = 148 * 8;
size_t cells3d_scratch_bytes() {
    const size_t a = warp_smem_bytes<4, 64>() * G3_WARPS, b = warp_smem_bytes<8, 128>() * G4_WARPS;
    return (a > b ? a : b) + 256;
}

size_t cells3d_image_backup_bytes() {
    // the most warps of any pass times its face storage
    const size_t p1 = warp_smem_bytes<1, 16>() * 148 * 7 * 2, p2 = warp_smem_bytes<2, 32>() * 148 * 3;
    const size_t p3 = warp_smem_bytes<4, 64>() * G3_WARPS, p4 = warp_smem_bytes<8, 128>() * G4_WARPS;
    return std::max(std::max(p1, p2), std::max(p3, p4)) + 256;
}

void cells3d_launch(const Cell3DArgs &a, void *scratch, cudaStream_t st) {
    if (a.n == 0) return;
    SDOT_CUDA(cudaMemsetAsync(a.ovf_cnt, 0, sizeof(int), st));
    SDOT_CUDA(cudaMemsetAsync(a.ovf_cnt2, 0, sizeof(int), st));
    SDOT_CUDA(cudaMemsetAsync(a.ovf_cnt3, 0, sizeof(int), st));
    if (a.rows.side_used) SDOT_CUDA(cudaMemsetAsync(a.rows.side_used, 0, sizeof(unsigned long long), st));
    if (a.nb.side_used) SDOT_CUDA(cudaMemsetAsync(a.nb.side_used, 0, sizeof(unsigned long long), st));
    launch3<1, 16, 2>(a, nullptr, nullptr, a.ovf_list, a.ovf_cnt, a.n, nullptr, 148LL * 7, st);
    // the larger passes take the overflow lists (their lengths are on the
    // device: every warp of the launch reads them)
    launch3<2, 32, 1>(a, a.ovf_list, a.ovf_cnt, a.ovf_list2, a.ovf_cnt2, 148LL * 3, nullptr, 148LL * 3, st);
    // passes 3 and 4 share the scratch, one after the other
    launch3<4, 64, 1>(a, a.ovf_list2, a.ovf_cnt2, a.ovf_list3, a.ovf_cnt3, G3_WARPS, static_cast<char *>(scratch),
                      G3_WARPS, st);
    launch3<8, 128, 1>(a, a.ovf_list3, a.ovf_cnt3, nullptr, nullptr, G4_WARPS, static_cast<char *>(scratch), G4_WARPS,
                       st);
}

}  // namespace sdot
