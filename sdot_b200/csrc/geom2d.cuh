// 2D convex-polygon geometry shared by the cell kernels (device) and the
// host-side domain builder.  Polygons are counter-clockwise vertex lists; the
// edge leaving vertex k carries id[k] (see common.cuh for id meanings).
//
// plane_cut restates ConvexPolyhedron2::plane_cut (reference
// src/sdot/Geometry/ConvexPolyhedron2.tcc:687-924) including its index
// bookkeeping (where the two new vertices land, and the rotation when the
// removed run wraps over vertex 0), so that a cell built from the same cut
// sequence has the same vertex order, hence the same fan triangulation.
#pragma once
#include "common.cuh"
#include <cmath>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace sdot {

#define SDOT_HD __host__ __device__ __forceinline__
// members of the streaming stages: left to the compiler's inlining choice
// (forcing them inline multiplies the code of the nested pixel pipelines)
#define SDOT_HDI __host__ __device__

constexpr double kPi = 3.141592653589793238462643383279502884;

// Vertex storage with an element stride (SoA in shared or global memory).
template <class T>
struct PolyView {
    T *x;
    T *y;
    int *id;
    int st;
    int cap = 1 << 30;  // vertex slots (bound of the debug checks)
    SDOT_HDI T &X(int k) const { return x[SDOT_CHECK_IDX(k, cap, 1) * st]; }
    SDOT_HDI T &Y(int k) const { return y[SDOT_CHECK_IDX(k, cap, 1) * st]; }
    SDOT_HDI int &I(int k) const { return id[SDOT_CHECK_IDX(k, cap, 1) * st]; }
    SDOT_HDI void copy(int dst, int src) const {
        X(dst) = X(src);
        Y(dst) = Y(src);
        I(dst) = I(src);
    }
};

// Cut the polygon (n vertices, capacity cap) by the half-plane
// {p : (o - p) . nrm >= 0}; the new edge gets `cut_id`.  The reference
// divides its distances by |nrm| for un-normalised normals (N<0>); the
// interpolation ratios are the same without it.
// Returns the new vertex count, or -1 if the result would exceed `cap`.
// The facts the reference reads from its `outside` bitset: count, first set
// bit, first clear bit, bits 1 and n - 1 (one pass over the vertices).
struct CutFacts {
    int nb_out = 0, first_out = -1, first_in = -1;
    bool out1 = false, out_last = false;
    SDOT_HD void add(int k, int n, bool o) {
        nb_out += o;
        if (o && first_out < 0) first_out = k;
        if (!o && first_in < 0) first_in = k;
        if (k == 1) out1 = o;
        if (k == n - 1) out_last = o;
    }
};

// The same facts from a bit mask of the outside vertices (bit k: vertex k;
// polygons of at most 32 vertices).
SDOT_HD CutFacts cut_facts(unsigned mask, int n) {
    CutFacts f;
    const unsigned valid = n >= 32 ? 0xffffffffu : ((1u << n) - 1u);
    const unsigned in = ~mask & valid;
#ifdef __CUDA_ARCH__
    f.nb_out = __popc(mask);
    f.first_out = __ffs(int(mask)) - 1;
    f.first_in = __ffs(int(in)) - 1;
#else
    f.nb_out = __builtin_popcount(mask);
    f.first_out = __builtin_ffs(int(mask)) - 1;
    f.first_in = __builtin_ffs(int(in)) - 1;
#endif
    f.out1 = n > 1 && ((mask >> 1) & 1u);
    f.out_last = (mask >> (n - 1)) & 1u;
    return f;
}

template <class T>
SDOT_HD int plane_cut_apply(const PolyView<T> &p, int n, int cap, T ox, T oy, T nx, T ny, int cut_id,
                            const CutFacts &f);

template <class T>
SDOT_HD int plane_cut(const PolyView<T> &p, int n, int cap, T ox, T oy, T nx, T ny, int cut_id) {
    CutFacts f;
    for (int k = 0; k < n; ++k) {
        const T d = (ox - p.X(k)) * nx + (oy - p.Y(k)) * ny;
        f.add(k, n, d < T(0));
    }
    return plane_cut_apply(p, n, cap, ox, oy, nx, ny, cut_id, f);
}

// The cut itself, given the classification of the vertices.  The new
// vertices sit at the ratios s_a / (s_b - s_a) of the signed distances along
// their edges; the ratios do not depend on the scale of the normal, so the
// distances are left unnormalised, and in FP64 both ratios come from one
// division (1 / (u v), u and v the two distance differences: products of
// coordinates, far from underflow).
template <class T>
SDOT_HD int plane_cut_apply(const PolyView<T> &p, int n, int cap, T ox, T oy, T nx, T ny, int cut_id,
                            const CutFacts &f) {
    const int nb_out = f.nb_out, first_out = f.first_out, first_in = f.first_in;
    const bool out_last = f.out_last;
    if (nb_out == 0) return n;
    if (nb_out == n) return 0;
    auto dist = [&](int k) -> T { return (ox - p.X(k)) * nx + (oy - p.Y(k)) * ny; };
    // the two edge ratios a / (b - a), c / (d - c)
    auto ratios = [](T a, T b, T c, T d, T &m1, T &m2) {
        const T u = b - a, v = d - c;
        if constexpr (sizeof(T) == 8) {
            const T r = T(1) / (u * v);
            m1 = a * v * r;
            m2 = c * u * r;
        } else {  // FP32: u v of small cells can underflow
            m1 = a / u;
            m2 = c / v;
        }
    };

    // One layout for every case.  The removed run is [i1, i2] (cyclic), the
    // kept run [i3, i0]; A (on edge i0 -> i1) takes the cut's id, B (on edge
    // i2 -> i3) the id of that edge.  Without wrap (the run does not hold
    // both vertex n - 1 and vertex 0): A at i1, B at i1 + 1, the kept tail
    // [i3, n) shifted by 2 - nb_out.  With wrap: B at 0, the kept run moved
    // to [1, nb_in], A after it.  These are the positions of the reference's
    // four cases (one vertex out, two, a wrapping run, a longer run).
    const int nb_in = n - nb_out;
    if (nb_out == 1 && n + 1 > cap) return -1;
    const bool wrap = out_last && first_out == 0;  // nb_out >= 2 here, as nb_out == 1 cannot be both
    const int i3 = wrap ? first_in : first_out + nb_out;  // may be n: vertex 0
    const int i1 = wrap ? first_in + nb_in : first_out;
    const int i0 = i1 == 0 ? n - 1 : i1 - 1;
    const int i2 = i3 == 0 ? n - 1 : i3 - 1;
    const int i3c = i3 == n ? 0 : i3;
    T p0x = p.X(i0), p0y = p.Y(i0), p1x = p.X(i1), p1y = p.Y(i1);
    T p2x = p.X(i2), p2y = p.Y(i2), p3x = p.X(i3c), p3y = p.Y(i3c);
    T s0 = dist(i0), s1 = dist(i1), s2 = dist(i2), s3 = dist(i3c);
    T m1, m2;
    ratios(s0, s1, s3, s2, m1, m2);
    const T ax = p0x - m1 * (p1x - p0x), ay = p0y - m1 * (p1y - p0y);
    const T bx = p3x - m2 * (p2x - p3x), by = p3y - m2 * (p2y - p3y);
    const int id2 = p.I(i2);
    if (wrap) {
        for (int k = 0; k < nb_in; ++k) p.copy(1 + k, i3 + k);
        p.X(0) = bx;
        p.Y(0) = by;
        p.I(0) = id2;
        p.X(nb_in + 1) = ax;
        p.Y(nb_in + 1) = ay;
        p.I(nb_in + 1) = cut_id;
    } else {
        if (nb_out == 1) {
            for (int i = n - 1; i >= i3; --i) p.copy(i + 1, i);
        } else {
            for (int i = i3; i < n; ++i) p.copy(i + 2 - nb_out, i);
        }
        p.X(i1) = ax;
        p.Y(i1) = ay;
        p.I(i1) = cut_id;
        p.X(i1 + 1) = bx;
        p.Y(i1 + 1) = by;
        p.I(i1 + 1) = id2;
    }
    return nb_in + 2;
}

#ifdef __CUDACC__
// plane_cut done by a whole warp on one polygon (all 32 lanes call it with the
// same arguments): the lanes classify 32 vertices at a time, the facts the
// scalar version gathers in its pass come from warp votes, and vertex moves
// are done 32 at a time, each chunk read before it is written, in the order
// that keeps the scalar loop's result.  Same cases, same new vertices, same
// vertex order as plane_cut.
template <class T>
__device__ int plane_cut_warp(const PolyView<T> &p, int n, int cap, T ox, T oy, T nx, T ny, int cut_id,
                              bool normalize) {
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    int nb_out = 0, first_out = -1, first_in = -1;
    bool out1 = false, out_last = false;
    for (int base = 0; base < n; base += 32) {
        const int k = base + lane;
        const bool valid = k < n;
        bool o = false;
        if (valid) {
            const T d = (ox - p.X(k)) * nx + (oy - p.Y(k)) * ny;
            o = d < T(0);
        }
        const unsigned mo = __ballot_sync(FULL, o), mi = __ballot_sync(FULL, valid && !o);
        nb_out += __popc(mo);
        if (first_out < 0 && mo) first_out = base + __ffs(mo) - 1;
        if (first_in < 0 && mi) first_in = base + __ffs(mi) - 1;
        if (base == 0 && n > 1) out1 = (mo >> 1) & 1u;
        if (n - 1 < base + 32) out_last = (mo >> (n - 1 - base)) & 1u;
    }
    if (nb_out == 0) return n;
    if (nb_out == n) return 0;
    T inv = T(1);
    if (normalize) inv = T(1) / sqrt(nx * nx + ny * ny);
    auto dist = [&](int k) -> T { return ((ox - p.X(k)) * nx + (oy - p.Y(k)) * ny) * inv; };
    int i1 = first_out;
    if (nb_out == 1) {
        if (n + 1 > cap) return -1;
        const int i0 = (i1 + n - 1) % n, i2 = (i1 + 1) % n;
        const T p0x = p.X(i0), p0y = p.Y(i0), p1x = p.X(i1), p1y = p.Y(i1), p2x = p.X(i2), p2y = p.Y(i2);
        const T s0 = dist(i0), s1 = dist(i1), s2 = dist(i2);
        const T m0 = s0 / (s1 - s0), m1 = s2 / (s1 - s2);
        const int id1 = p.I(i1);
        __syncwarp();
        for (int hi = n; hi > i1 + 1; hi -= 32) {  // [i1 + 1, n) moves up by one, top chunk first
            const int lo = hi - 32 > i1 + 1 ? hi - 32 : i1 + 1;
            const int k = lo + lane;
            T vx = T(0), vy = T(0);
            int vi = 0;
            if (k < hi) {
                vx = p.X(k);
                vy = p.Y(k);
                vi = p.I(k);
            }
            __syncwarp();
            if (k < hi) {
                p.X(k + 1) = vx;
                p.Y(k + 1) = vy;
                p.I(k + 1) = vi;
            }
            __syncwarp();
        }
        if (lane == 0) {
            p.X(i1 + 1) = p2x - m1 * (p1x - p2x);
            p.Y(i1 + 1) = p2y - m1 * (p1y - p2y);
            p.I(i1 + 1) = id1;
            p.X(i1) = p0x - m0 * (p1x - p0x);
            p.Y(i1) = p0y - m0 * (p1y - p0y);
            p.I(i1) = cut_id;
        }
        __syncwarp();
        return n + 1;
    }
    if (nb_out == 2) {
        if (i1 == 0 && !out1) i1 = n - 1;
        const int i0 = (i1 + n - 1) % n, i2 = (i1 + 1) % n, i3 = (i1 + 2) % n;
        const T p0x = p.X(i0), p0y = p.Y(i0), p1x = p.X(i1), p1y = p.Y(i1);
        const T p2x = p.X(i2), p2y = p.Y(i2), p3x = p.X(i3), p3y = p.Y(i3);
        const T s0 = dist(i0), s1 = dist(i1), s2 = dist(i2), s3 = dist(i3);
        const T m1 = s0 / (s1 - s0), m2 = s3 / (s2 - s3);
        __syncwarp();
        if (lane == 0) {
            p.X(i1) = p0x - m1 * (p1x - p0x);
            p.Y(i1) = p0y - m1 * (p1y - p0y);
            p.I(i1) = cut_id;
            p.X(i2) = p3x - m2 * (p2x - p3x);
            p.Y(i2) = p3y - m2 * (p2y - p3y);
        }
        __syncwarp();
        return n;
    }
    // left move of [src0, src0 + cnt) to [src0 - by, ...), low chunk first
    auto move_down = [&](int src0, int cnt, int by) {
        for (int c = 0; c < cnt; c += 32) {
            const int k = src0 + c + lane;
            const bool v = c + lane < cnt;
            T vx = T(0), vy = T(0);
            int vi = 0;
            if (v) {
                vx = p.X(k);
                vy = p.Y(k);
                vi = p.I(k);
            }
            __syncwarp();
            if (v) {
                p.X(k - by) = vx;
                p.Y(k - by) = vy;
                p.I(k - by) = vi;
            }
            __syncwarp();
        }
    };
    if (i1 == 0 && out_last) {
        const int nb_in = n - nb_out;
        const int i3 = first_in;
        i1 = nb_in + i3;
        const int i0 = i1 - 1, i2 = i3 - 1;
        const T p0x = p.X(i0), p0y = p.Y(i0), p1x = p.X(i1), p1y = p.Y(i1);
        const T p2x = p.X(i2), p2y = p.Y(i2), p3x = p.X(i3), p3y = p.Y(i3);
        const T s0 = dist(i0), s1 = dist(i1), s2 = dist(i2), s3 = dist(i3);
        const T m1 = s0 / (s1 - s0), m2 = s3 / (s2 - s3);
        const int id2 = p.I(i2);
        __syncwarp();
        if (lane == 0) {
            p.X(0) = p3x - m2 * (p2x - p3x);
            p.Y(0) = p3y - m2 * (p2y - p3y);
            p.I(0) = id2;
        }
        __syncwarp();
        if (i2 > 0) move_down(i2 + 1, nb_in, i2);
        if (lane == 0) {
            p.X(nb_in + 1) = p0x - m1 * (p1x - p0x);
            p.Y(nb_in + 1) = p0y - m1 * (p1y - p0y);
            p.I(nb_in + 1) = cut_id;
        }
        __syncwarp();
        return nb_in + 2;
    }
    const int i0 = (i1 + n - 1) % n, i2 = (i1 + nb_out - 1) % n, i3 = (i1 + nb_out) % n;
    const T p0x = p.X(i0), p0y = p.Y(i0), p1x = p.X(i1), p1y = p.Y(i1);
    const T p2x = p.X(i2), p2y = p.Y(i2), p3x = p.X(i3), p3y = p.Y(i3);
    const T s0 = dist(i0), s1 = dist(i1), s2 = dist(i2), s3 = dist(i3);
    const T m1 = s0 / (s1 - s0), m2 = s3 / (s2 - s3);
    const int id2 = p.I(i2);
    __syncwarp();
    if (lane == 0) {
        p.X(i1) = p0x - m1 * (p1x - p0x);
        p.Y(i1) = p0y - m1 * (p1y - p0y);
        p.I(i1) = cut_id;
        p.X(i1 + 1) = p3x - m2 * (p2x - p3x);
        p.Y(i1 + 1) = p3y - m2 * (p2y - p3y);
        p.I(i1 + 1) = id2;
    }
    __syncwarp();
    const int nb_rem = nb_out - 2;
    if (i2 + 1 < n) move_down(i2 + 1, n - i2 - 1, nb_rem);
    return n - nb_rem;
}
#endif

// Weighted bisector of (c0, w0) and (c1, w1) as the reference's traversal
// builds it (src/sdot/PowerDiagram/Visitors/SpZGrid.tcc:506-522): origin
// c0 + x V, normal V = c1 - c0, x = 1/2 + 1/2 (w0 - w1) / |V|^2.
template <class T>
SDOT_HD void bisector(T c0x, T c0y, T w0, T c1x, T c1y, T w1, T &ox, T &oy, T &nx, T &ny) {
    nx = c1x - c0x;
    ny = c1y - c0y;
    T nn = nx * nx + ny * ny;
    T x = T(0.5) + T(0.5) * (w0 - w1) / nn;
    ox = c0x + x * nx;
    oy = c0y + x * ny;
}

// ------------------------------------------------------------------------
// Streaming stages.  A polygon is pushed vertex by vertex (push(x, y, tag),
// tag = id of the edge leaving that vertex) then closed with finish().
// Each stage forwards a transformed polygon to the next stage, so clipped
// pieces never need their own vertex buffer.

// Keep the half-plane  s * (coord - c) >= 0  (coord = x if axis == 0 else y).
// New edges along the clip line get tag `own`.
template <class Next>
struct AxisClip {
    Next &next;
    int axis;
    double c, s;
    int own;
    bool has_first = false;
    double fx = 0, fy = 0;
    int ft = 0;
    double px = 0, py = 0;
    int pt = 0;
    SDOT_HDI AxisClip(Next &nx, int ax, double cc, double ss, int ow) : next(nx), axis(ax), c(cc), s(ss), own(ow) {}
    SDOT_HDI double val(double x, double y) const { return s * ((axis == 0 ? x : y) - c); }
    SDOT_HDI void edge(double ax, double ay, int at, double bx, double by) {
        double va = val(ax, ay), vb = val(bx, by);
        bool ina = va >= 0, inb = vb >= 0;
        if (ina) {
            next.push(ax, ay, at);
            if (!inb) {
                double t = va / (va - vb);
                double ix = ax + t * (bx - ax), iy = ay + t * (by - ay);
                if (axis == 0) ix = c; else iy = c;
                next.push(ix, iy, own);
            }
        } else if (inb) {
            double t = va / (va - vb);
            double ix = ax + t * (bx - ax), iy = ay + t * (by - ay);
            if (axis == 0) ix = c; else iy = c;
            next.push(ix, iy, at);
        }
    }
    SDOT_HDI void push(double x, double y, int tag) {
        if (!has_first) {
            has_first = true;
            fx = x; fy = y; ft = tag;
        } else {
            edge(px, py, pt, x, y);
        }
        px = x; py = y; pt = tag;
    }
    SDOT_HDI void finish() {
        if (has_first) edge(px, py, pt, fx, fy);
        next.finish();
    }
};

// Disc clipping restated from ConvexPolyhedron2::ball_cut
// (ConvexPolyhedron2.tcc:534-666): each edge (P -> C) emits 0, 1 or 2
// vertices (LINE keeps the edge's tag, ARC gets ID_ARC).  When nothing is
// emitted, the result is the full disc unless the centre lies outside one
// of the edges' half-planes (then it is empty).
template <class Next>
struct DiscClip {
    Next &next;
    double cx, cy, r;
    int nin = 0, nout = 0;
    bool center_out = false;
    bool has_first = false;
    double fx = 0, fy = 0;
    int ft = 0;
    double px = 0, py = 0;
    int pt = 0;
    SDOT_HDI DiscClip(Next &nx, double x, double y, double rr) : next(nx), cx(x), cy(y), r(rr) {}
    SDOT_HDI double dist(double x, double y) const { return (x - cx) * (x - cx) + (y - cy) * (y - cy) - r * r; }
    SDOT_HDI void unique_inter(double p0x, double p0y, double p1x, double p1y, double &ox, double &oy) const {
        double dx = p1x - p0x, dy = p1y - p0y;
        double a = dx * dx + dy * dy;
        double b = (p0x - cx) * dx + (p0y - cy) * dy;
        double c = (p0x - cx) * (p0x - cx) + (p0y - cy) * (p0y - cy) - r * r;
        double d = sqrt(fmax(0.0, b * b - a * c));
        double u = (-b + d) / a;
        double v = (-b - d) / a;
        double t = fabs(u - 0.5) <= fabs(v - 0.5) ? u : v;
        t = fmin(1.0, fmax(0.0, t));
        ox = p0x + t * dx;
        oy = p0y + t * dy;
    }
    SDOT_HDI bool two_cuts(double p0x, double p0y, double p1x, double p1y, double &ax, double &ay, double &bx,
                             double &by) const {
        double dx = p1x - p0x, dy = p1y - p0y;
        double a = dx * dx + dy * dy;
        if (a == 0) return false;
        double b = (p0x - cx) * dx + (p0y - cy) * dy;
        double c = (p0x - cx) * (p0x - cx) + (p0y - cy) * (p0y - cy) - r * r;
        double s = b * b - a * c;
        if (s <= 0) return false;
        double d = sqrt(s);
        double u = (-b - d) / a;
        double v = (-b + d) / a;
        if (u > 0 && u < 1)
            v = fmax(0.0, fmin(1.0, v));
        else if (v > 0 && v < 1)
            u = fmax(0.0, fmin(1.0, u));
        else
            return false;
        ax = p0x + u * dx;
        ay = p0y + u * dy;
        bx = p0x + v * dx;
        by = p0y + v * dy;
        double a0 = atan2(ay - cy, ax - cx);
        double a1 = atan2(by - cy, bx - cx);
        return a0 != a1;
    }
    SDOT_HDI void emit(double x, double y, int tag) {
        ++nout;
        next.push(x, y, tag);
    }
    SDOT_HDI void edge(double ax, double ay, int at, double bx, double by) {
        // outward normal of a counter-clockwise edge is (dy, -dx)
        if ((cx - ax) * (by - ay) - (cy - ay) * (bx - ax) > 0) center_out = true;
        double da = dist(ax, ay), db = dist(bx, by);
        if (da <= 0) {
            emit(ax, ay, at);
            if (db > 0) {
                double ix, iy;
                unique_inter(ax, ay, bx, by, ix, iy);
                emit(ix, iy, ID_ARC);
            }
        } else if (db <= 0) {
            double ix, iy;
            unique_inter(bx, by, ax, ay, ix, iy);
            emit(ix, iy, at);
        } else {
            double qx, qy, sx, sy;
            if (two_cuts(ax, ay, bx, by, qx, qy, sx, sy)) {
                emit(qx, qy, at);
                emit(sx, sy, ID_ARC);
            }
        }
    }
    SDOT_HDI void push(double x, double y, int tag) {
        ++nin;
        if (!has_first) {
            has_first = true;
            fx = x; fy = y; ft = tag;
        } else {
            edge(px, py, pt, x, y);
        }
        px = x; py = y; pt = tag;
    }
    SDOT_HDI void finish() {
        if (has_first) edge(px, py, pt, fx, fy);
        next.finish();
    }
    // radius of the result as the reference stores it: 0 if void, r otherwise
    SDOT_HDI double result_radius() const {
        if (nin == 0) return 0.0;
        if (nout == 0 && center_out) return 0.0;
        return r;
    }
};

// Arc helpers restated from ConvexPolyhedron2::_arc_area / _centroid_arc /
// _arc_length (ConvexPolyhedron2.tcc:2296-2381).
SDOT_HD double arc_angles(double p0x, double p0y, double p1x, double p1y, double cx, double cy, double &a0) {
    a0 = atan2(p0y - cy, p0x - cx);
    double a1 = atan2(p1y - cy, p1x - cx);
    if (a1 < a0) a1 += 2 * kPi;
    return a1;
}

SDOT_HD double arc_area(double p0x, double p0y, double p1x, double p1y, double cx, double cy, double r) {
    double a0;
    double a1 = arc_angles(p0x, p0y, p1x, p1y, cx, cy, a0);
    double ex = p0x - p1x, ey = p0y - p1y;
    double d0 = sqrt(ex * ex + ey * ey) / 2;
    double d1 = sqrt(fmax(0.0, r * r - d0 * d0));
    double rs = r * r * (a1 - a0) / 2;
    if (a1 - a0 > kPi)
        rs += d1 * d0;
    else
        rs -= d1 * d0;
    return rs;
}

SDOT_HD void centroid_arc(double &ctx, double &cty, double &mea, double p0x, double p0y, double p1x, double p1y,
                          double cx, double cy, double r, double coeff) {
    p0x -= cx; p0y -= cy;
    p1x -= cx; p1y -= cy;
    double a0 = atan2(p0y, p0x);
    double a1 = atan2(p1y, p1x);
    if (a1 < a0) a1 += 2 * kPi;
    double ex = p0x - p1x, ey = p0y - p1y;
    double d0 = sqrt(ex * ex + ey * ey) / 2;
    double d1 = sqrt(fmax(0.0, r * r - d0 * d0));
    double tri_area = d1 * d0;
    double tbx = (1.0 / 3.0) * (p0x + p1x), tby = (1.0 / 3.0) * (p0y + p1y);
    double pie_area = r * r * (a1 - a0) / 2;
    double f = 2.0 / 3.0 * (r * r * r) * sin((a1 - a0) / 2);
    double pmx = f * cos((a1 + a0) / 2), pmy = f * sin((a1 + a0) / 2);
    double lea;
    if (a1 - a0 > kPi) {
        ctx += coeff * (pmx + tri_area * tbx);
        cty += coeff * (pmy + tri_area * tby);
        lea = (pie_area + tri_area) * coeff;
    } else {
        ctx += coeff * (pmx - tri_area * tbx);
        cty += coeff * (pmy - tri_area * tby);
        lea = (pie_area - tri_area) * coeff;
    }
    ctx += lea * cx;
    cty += lea * cy;
    mea += lea;
}

}  // namespace sdot
