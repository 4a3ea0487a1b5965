// Preconditioned conjugate gradients on the device (see solve.cuh).
//
// Every reduction is two-stage with a fixed order (per-block partials, then
// one block sums them), so a solve is bitwise reproducible run to run.  The
// scalars of the iteration (alpha, beta, |r|^2) stay on the device; the host
// only reads |r|^2 every `check` iterations to decide to stop.
#include "solve.cuh"

#include <algorithm>
#include <cmath>

namespace sdot {

namespace {

constexpr int TB = 256;
enum { S_RZ = 0, S_RR = 1, S_RR0 = 2, S_PQ = 3, S_ALPHA = 4, S_BETA = 5, S_GDIAG = 6, S_BAD = 7, S_NSCAL = 8 };

__device__ double block_sum(double v, double *sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double r = 0;
    if (warp == 0) {
        r = lane < (blockDim.x >> 5) ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    return r;  // valid in thread 0
}

// Matrix views for the PCG kernels: row s times x, and the diagonal entry
// (sums in double whatever the precision of the values and vectors).
// RowsMatT: the Hessian rows (ELL + side buffer) with values of type V
// (rows.val itself, or an FP32 copy in the same layout).
template <class V>
struct RowsMatT {
    Rows R;
    const V *val;
    const V *side_val;
    template <class X>
    __device__ double row_dot(long long s, const X *x) const {
        const int m = R.cnt[s];
        double acc = 0;
        if (m <= R.cap) {
            for (int k = 0; k < m; ++k) acc += double(val[k * R.stride + s]) * double(x[R.col[k * R.stride + s]]);
        } else {
            const long long o = R.side[s];
            for (int k = 0; k < m; ++k) acc += double(side_val[o + k]) * double(x[R.side_col[o + k]]);
        }
        return acc;
    }
    __device__ int len(long long s) const { return R.cnt[s]; }
    __device__ long long colk(long long s, int k) const { return *R.colp(s, k); }
    __device__ double valk(long long s, int k) const {
        return R.cnt[s] > R.cap ? double(side_val[R.side[s] + k]) : double(val[k * R.stride + s]);
    }
    __device__ double diag(long long s) const {
        double d = 0;
        for (int k = 0, m = R.cnt[s]; k < m; ++k)
            if (colk(s, k) == s) d += valk(s, k);
        return d;
    }
    // sum_k a_sk f(col_sk)
    template <class F>
    __device__ double row_sum(long long s, const F &f) const {
        const int m = R.cnt[s];
        double acc = 0;
        if (m <= R.cap) {
            for (int k = 0; k < m; ++k) acc += double(val[k * R.stride + s]) * f(R.col[k * R.stride + s]);
        } else {
            const long long o = R.side[s];
            for (int k = 0; k < m; ++k) acc += double(side_val[o + k]) * f(R.side_col[o + k]);
        }
        return acc;
    }
};
using RowsMat = RowsMatT<double>;
inline RowsMat rows_mat(const Rows &R) { return RowsMat{R, R.val, R.side_val}; }

// The FP32 copy of the Hessian rows in Laplacian form: an off-diagonal entry
// holds the edge weight w_sj = -a_sj, the diagonal entry the row sum r_s (the
// part of the diagonal that is not the sum of the edge weights: disc arcs),
// so that (A x)_s = r_s x_s + sum_j w_sj (x_s - x_j).  Rounding the weights to
// FP32 then perturbs each edge by a relative 6e-8, which bounds the FP32
// operator between (1 -+ 6e-8) times the exact one; rounding the entries
// themselves would break the zero row sums by 6e-8 of the diagonal, far
// above the smallest eigenvalues of these systems.  Sums in double.
struct RowsLap32 {
    Rows R;
    const float *val;
    const float *side_val;
    __device__ int len(long long s) const { return R.cnt[s]; }
    __device__ long long colk(long long s, int k) const { return *R.colp(s, k); }
    __device__ double raw(long long s, int k) const {
        return R.cnt[s] > R.cap ? double(side_val[R.side[s] + k]) : double(val[k * R.stride + s]);
    }
    template <class F>
    __device__ double row_sum(long long s, const F &f) const {
        const int m = R.cnt[s];
        const double fs = f(s);
        double acc = 0;
        for (int k = 0; k < m; ++k) {
            const long long c = colk(s, k);
            acc += c == s ? raw(s, k) * fs : raw(s, k) * (fs - f(c));
        }
        return acc;
    }
    template <class X>
    __device__ double row_dot(long long s, const X *x) const {
        return row_sum(s, [&](long long j) { return double(x[j]); });
    }
    __device__ double diag(long long s) const {
        double d = 0;
        for (int k = 0, m = R.cnt[s]; k < m; ++k) d += raw(s, k);  // r_s + sum of the weights
        return d;
    }
    __device__ double valk(long long s, int k) const { return colk(s, k) == s ? diag(s) : -raw(s, k); }
};

struct CsrView {
    CsrMat M;
    template <class X>
    __device__ double row_dot(long long s, const X *x) const {
        double acc = 0;
        for (long long k = M.off[s], e = M.off[s + 1]; k < e; ++k) acc += M.val[k] * double(x[M.col[k]]);
        return acc;
    }
    __device__ double diag(long long s) const {
        double d = 0;
        for (long long k = M.off[s], e = M.off[s + 1]; k < e; ++k)
            if (M.col[k] == s) d += M.val[k];
        return d;
    }
    __device__ int len(long long s) const { return int(M.off[s + 1] - M.off[s]); }
    __device__ long long colk(long long s, int k) const { return M.col[M.off[s] + k]; }
    __device__ double valk(long long s, int k) const { return M.val[M.off[s] + k]; }
    template <class F>
    __device__ double row_sum(long long s, const F &f) const {
        double acc = 0;
        for (long long k = M.off[s], e = M.off[s + 1]; k < e; ++k) acc += M.val[k] * f(M.col[k]);
        return acc;
    }
};

// ---- multilevel preconditioner (one V-cycle per application) ------------
// Aggregates: MG_B consecutive rows (the rows are in Morton order, so an
// aggregate is a compact patch of cells).  Coarse matrices P^T A P with P
// piecewise constant on the aggregates, stored as ELL (width MG_CAP);
// damped-Jacobi smoothing (MG_OMEGA) before and after the coarse
// correction; the coarsest level (<= MG_COARSE rows) is applied as its dense
// inverse.  Same smoother on both sides and an exact coarsest solve: the
// cycle is a symmetric positive operator, a valid CG preconditioner.
constexpr int MG_B = 8;
constexpr int MG_CAP_MAX = 128;  // coarse ELL width: w.mg_cap (64 in 2D, 128 in 3D)
constexpr int MG_COARSE = 48;  // dense coarsest level: two 48 x 49 doubles in shared memory
constexpr double MG_OMEGA = 0.67;

template <class V>
struct EllViewT {
    const int *cnt;
    const int *col;
    const V *val;
    long long stride;
    __device__ int len(long long s) const { return cnt[s]; }
    __device__ long long colk(long long s, int k) const { return col[k * stride + s]; }
    __device__ double valk(long long s, int k) const { return double(val[k * stride + s]); }
    template <class F>
    __device__ double row_sum(long long s, const F &f) const {
        double acc = 0;
        for (int k = 0, m = cnt[s]; k < m; ++k) acc += double(val[k * stride + s]) * f(col[k * stride + s]);
        return acc;
    }
};

template <class M, class T>
__global__ void k_diag_inv(M A, long long n, long long g, T *dinv, double *scal) {
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        double d = A.diag(s);
        if (s == g) {
            scal[S_GDIAG] = d;
            d *= 2;
        }
        dinv[s] = T(d != 0 ? 1.0 / d : 0.0);
    }
}

template <class T>
__global__ void k_init(const T *b, T *x, T *r, T *z, T *p, const T *dinv, double *partial, long long n) {
    __shared__ double sh[32];
    double rz = 0, rr = 0;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        const T rv = b[s];
        const T zv = dinv[s] * rv;
        x[s] = 0;
        r[s] = rv;
        z[s] = zv;
        p[s] = zv;
        rz += double(rv) * double(zv);
        rr += double(rv) * double(rv);
    }
    rz = block_sum(rz, sh);
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = rz;
        partial[gridDim.x + blockIdx.x] = rr;
    }
}

// mode 0: after init (rz, rr, rr0); 1: after spmv (pq -> alpha); 2: after update (rz_new, rr -> beta)
__global__ void k_final(const double *partial, int nb, double *scal, int mode) {
    __shared__ double sh[32];
    double a = 0, b = 0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        a += partial[i];
        b += partial[nb + i];
    }
    a = block_sum(a, sh);
    b = block_sum(b, sh);
    if (threadIdx.x == 0) {
        if (mode == 0) {
            scal[S_RZ] = a;
            scal[S_RR] = b;
            scal[S_RR0] = b;
            scal[S_BAD] = 0;
        } else if (mode == 1) {
            scal[S_PQ] = a;
            const double alpha = scal[S_RZ] / a;
            if (!(a > 0) || !isfinite(alpha)) scal[S_BAD] = 1;
            scal[S_ALPHA] = scal[S_BAD] != 0 ? 0.0 : alpha;
        } else {
            const double beta = a / scal[S_RZ];
            scal[S_BETA] = isfinite(beta) ? beta : 0.0;
            scal[S_RZ] = a;
            scal[S_RR] = b;
        }
    }
}

template <class M, class T>
__global__ void k_spmv(M A, long long n, long long g, const T *p, T *q, const double *scal, double *partial) {
    __shared__ double sh[32];
    double pq = 0;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        double v = A.row_dot(s, p);
        if (s == g) v += scal[S_GDIAG] * double(p[s]);
        const T qv = T(v);
        q[s] = qv;
        pq += double(p[s]) * double(qv);
    }
    pq = block_sum(pq, sh);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = pq;
        partial[gridDim.x + blockIdx.x] = 0;
    }
}

template <class T>
__global__ void k_update(T *x, T *r, T *z, const T *p, const T *q, const T *dinv, const double *scal, double *partial,
                         long long n) {
    __shared__ double sh[32];
    const T alpha = T(scal[S_ALPHA]);
    double rz = 0, rr = 0;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        x[s] += alpha * p[s];
        const T rv = r[s] - alpha * q[s];
        r[s] = rv;
        const T zv = dinv[s] * rv;
        z[s] = zv;
        rz += double(rv) * double(zv);
        rr += double(rv) * double(rv);
    }
    rz = block_sum(rz, sh);
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = rz;
        partial[gridDim.x + blockIdx.x] = rr;
    }
}

template <class T>
__global__ void k_pupdate(const T *z, T *p, const double *scal, long long n) {
    const T beta = T(scal[S_BETA]);
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x)
        p[s] = z[s] + beta * p[s];
}

__global__ void k_mass_partial(const double *m, const double *t, long long n, double *partial) {
    __shared__ double sh[32];
    __shared__ double shmax[32], shmin[32];
    double mx = 0, mn = 1.0 / 0.0, ss = 0;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        const double d = m[s] - t[s];
        mx = fmax(mx, fabs(d) / t[s]);
        mn = fmin(mn, m[s]);
        ss += d * d;
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
        mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        shmax[warp] = mx;
        shmin[warp] = mn;
    }
    ss = block_sum(ss, sh);
    if (threadIdx.x == 0) {
        for (int w = 1; w < (blockDim.x >> 5); ++w) {
            mx = fmax(mx, shmax[w]);
            mn = fmin(mn, shmin[w]);
        }
        partial[3 * blockIdx.x] = mx;
        partial[3 * blockIdx.x + 1] = mn;
        partial[3 * blockIdx.x + 2] = ss;
    }
}

__global__ void k_mass_final(const double *partial, int nb, double *out) {
    if (threadIdx.x != 0) return;
    double mx = 0, mn = 1.0 / 0.0, ss = 0;
    for (int b = 0; b < nb; ++b) {
        mx = fmax(mx, partial[3 * b]);
        mn = fmin(mn, partial[3 * b + 1]);
        ss += partial[3 * b + 2];
    }
    out[0] = mx;
    out[1] = mn;
    out[2] = ss;
}

__global__ void k_axpby(const double *a, const double *b, double *out, double alpha, double beta, long long n) {
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x)
        out[s] = alpha * a[s] + beta * b[s];
}

__global__ void k_apply_step(const double *w_base, const double *d, const int *idx, double tau, double *w_out,
                             long long n) {
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        const int i = idx[s];
        w_out[i] = w_base[i] - tau * d[s];
    }
}

__global__ void k_gather_sorted(const double *t, const int *idx, double *out, long long n) {
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x)
        out[s] = t[idx[s]];
}

// One warp per coarse row c: the entries of fine rows c*MG_B .. c*MG_B+7, in
// row order then stored order, are merged by coarse column into a table of
// 32 SLOTS entries (SLOTS per lane), so the sums have a fixed order.  The
// gauge term of the fine level joins the coarse diagonal.  A row with more
// than 32 SLOTS coarse columns sets *flag (the solve falls back to Jacobi).
template <class M, int SLOTS, class T>
__global__ void k_mg_coarsen(M A, long long nf, long long gauge, const double *scal, MgLevelT<T> out, int *flag) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long c = warp; c < out.n; c += nwarps) {
        int key[SLOTS], count = 0;
        double v[SLOTS];
#pragma unroll
        for (int q = 0; q < SLOTS; ++q) {
            key[q] = -1;
            v[q] = 0;
        }
        bool over = false;
        auto insert = [&](int cc, double x) {
            bool found = false;
#pragma unroll
            for (int q = 0; q < SLOTS; ++q) {
                const unsigned m = __ballot_sync(FULL, key[q] == cc);
                if (!found && m) {
                    if (lane == __ffs(int(m)) - 1) v[q] += x;
                    found = true;
                }
            }
            if (found) return;
            if (count < 32 * SLOTS) {
                if (lane == (count & 31)) {
#pragma unroll
                    for (int q = 0; q < SLOTS; ++q)
                        if (q == (count >> 5)) {
                            key[q] = cc;
                            v[q] = x;
                        }
                }
                ++count;
            } else {
                over = true;
            }
        };
        for (int r = 0; r < MG_B; ++r) {
            const long long s = c * MG_B + r;
            if (s >= nf) break;
            const int len = A.len(s);
            for (int k = 0; k < len; ++k) insert(int(A.colk(s, k) / MG_B), A.valk(s, k));
            if (s == gauge) insert(int(c), scal[S_GDIAG]);
        }
        double diag = 0;
#pragma unroll
        for (int q = 0; q < SLOTS; ++q)
            if (lane + 32 * q < count) {
                out.col[(lane + 32 * q) * out.n + c] = key[q];
                out.val[(lane + 32 * q) * out.n + c] = T(v[q]);
                if (key[q] == c) diag = v[q];
            }
        for (int o = 16; o > 0; o >>= 1) diag += __shfl_xor_sync(FULL, diag, o);
        if (lane == 0) {
            out.cnt[c] = count;
            out.dinv[c] = T(diag > 0 ? 1.0 / diag : 0.0);
            if (over) atomicExch(flag, 1);
        }
    }
}

// Pre-smoothing and restriction of one level: z = w D^-1 r, and
// rc[aggregate] = sum over its rows of (r - A z).  Rows are taken a block at a
// time so that the MG_B rows of an aggregate sit in consecutive lanes.
template <class M, class T, class TC>
__global__ void k_mg_pre(M A, long long n, long long gauge, const double *scal, const T *dinv, const T *r, T *z,
                         TC *rc) {
    const unsigned FULL = 0xffffffffu;
    for (long long i0 = blockIdx.x * (long long)blockDim.x; i0 < n; i0 += (long long)gridDim.x * blockDim.x) {
        const long long i = i0 + threadIdx.x;
        double t = 0;
        if (i < n) {
            const double ri = double(r[i]);
            const double zi = MG_OMEGA * double(dinv[i]) * ri;
            z[i] = T(zi);
            double acc = A.row_sum(i, [&](long long j) { return MG_OMEGA * double(dinv[j]) * double(r[j]); });
            if (i == gauge) acc += scal[S_GDIAG] * zi;
            t = ri - acc;
        }
        for (int o = MG_B / 2; o > 0; o >>= 1) t += __shfl_down_sync(FULL, t, o, MG_B);
        if ((threadIdx.x & (MG_B - 1)) == 0 && i < n) rc[i / MG_B] = TC(t);
    }
}

// Coarse correction and post-smoothing: z' = z + P zc, zo = z' + w D^-1 (r - A z').
// On the finest level (FINE) it also sums r . zo per block into partial[]
// and, when p is given, writes p = zo (the first CG direction).
template <class M, bool FINE, class T, class TC>
__global__ void k_mg_post(M A, long long n, long long gauge, const double *scal, const T *dinv, const T *r, const T *z,
                          const TC *zc, T *zo, double *partial, T *p) {
    __shared__ double sh[32];
    double rz = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        auto zp = [&](long long j) { return double(z[j]) + double(zc[j / MG_B]); };
        const double zi = zp(i);
        double acc = A.row_sum(i, zp);
        if (i == gauge) acc += scal[S_GDIAG] * zi;
        const T v = T(zi + MG_OMEGA * double(dinv[i]) * (double(r[i]) - acc));
        zo[i] = v;
        if (FINE) {
            rz += double(r[i]) * double(v);
            if (p) p[i] = v;
        }
    }
    if (FINE) {
        rz = block_sum(rz, sh);
        if (threadIdx.x == 0) partial[blockIdx.x] = rz;
    }
}

// The same two steps on a coarse level, four lanes per row (a warp holds the
// eight rows of one aggregate): the coarse rows are up to MG_CAP_MAX entries
// wide and the levels small, so one thread per row left each kernel bound by
// the latency of a long chain of dependent loads.  Each lane sums every
// fourth entry of its row; the partial sums are combined in a fixed order.
constexpr int CL = 4;  // lanes per coarse row
__global__ void k_mg_pre_coarse(EllViewT<double> A, long long n, const double *dinv, const double *r, double *z,
                                double *rc) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, sub = lane & (CL - 1);
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long nagg = (n + MG_B - 1) / MG_B;
    for (long long g = warp; g < nagg; g += nw) {
        const long long i = g * MG_B + (lane >> 2);
        // z = w D^-1 r; t = r - A z (A z from the smoothed values w D^-1 r)
        double acc = 0, ri = 0;
        if (i < n) {
            ri = r[i];
            if (sub == 0) z[i] = MG_OMEGA * dinv[i] * ri;
            const int m = A.cnt[i];
            for (int k = sub; k < m; k += CL) {
                const long long c = A.col[k * A.stride + i];
                acc += A.val[k * A.stride + i] * (MG_OMEGA * dinv[c] * r[c]);
            }
        }
        acc += __shfl_xor_sync(FULL, acc, 1);
        acc += __shfl_xor_sync(FULL, acc, 2);
        double t = i < n && sub == 0 ? ri - acc : 0.0;
        // the aggregate's residual: the rows in order (lanes 0, 4, ..., 28)
        for (int o = 4; o < 32; o <<= 1) t += __shfl_xor_sync(FULL, t, o);
        if (lane == 0) rc[g] = t;
    }
}

__global__ void k_mg_post_coarse(EllViewT<double> A, long long n, const double *dinv, const double *r, const double *z,
                                 const double *zc, double *zo) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, sub = lane & (CL - 1);
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long nrow = (n + 7) / 8 * 8;
    for (long long i0 = warp * 8; i0 < nrow; i0 += nw * 8) {
        const long long i = i0 + (lane >> 2);
        double acc = 0;
        if (i < n) {
            const int m = A.cnt[i];
            for (int k = sub; k < m; k += CL) {
                const long long c = A.col[k * A.stride + i];
                acc += A.val[k * A.stride + i] * (z[c] + zc[c / MG_B]);
            }
        }
        acc += __shfl_xor_sync(FULL, acc, 1);
        acc += __shfl_xor_sync(FULL, acc, 2);
        if (i < n && sub == 0) {
            const double zi = z[i] + zc[i / MG_B];
            zo[i] = zi + MG_OMEGA * dinv[i] * (r[i] - acc);
        }
    }
}

// Dense inverse of the coarsest level (nc <= MG_COARSE rows, one block of
// MG_COARSE threads, thread t owns row t).  Gauss-Jordan without pivoting
// (the matrix is symmetric positive semi-definite); a pivot below 1e-13 of
// the largest diagonal entry marks a null direction, left out of the inverse.
template <class V>
__global__ void k_mg_coarsest_setup(EllViewT<V> A, int nc, double *cinv) {
    __shared__ double M[MG_COARSE][MG_COARSE + 1], I[MG_COARSE][MG_COARSE + 1];
    __shared__ double dmax;
    const int t = threadIdx.x;
    if (t < nc) {
        for (int c = 0; c < nc; ++c) {
            M[t][c] = 0;
            I[t][c] = c == t ? 1.0 : 0.0;
        }
        for (int k = 0, m = A.cnt[t]; k < m; ++k) M[t][A.col[k * A.stride + t]] += double(A.val[k * A.stride + t]);
    }
    __syncthreads();
    if (t == 0) {
        double d = 0;
        for (int c = 0; c < nc; ++c) d = fmax(d, M[c][c]);
        dmax = d;
    }
    __syncthreads();
    for (int k = 0; k < nc; ++k) {
        const double piv = M[k][k];
        const bool ok = piv > 1e-13 * dmax;
        __syncthreads();
        if (t == k) {
            const double inv = ok ? 1.0 / piv : 0.0;
            for (int c = 0; c < nc; ++c) {
                M[k][c] *= inv;
                I[k][c] *= inv;
            }
        }
        __syncthreads();
        if (t < nc && t != k && ok) {
            const double f = M[t][k];
            for (int c = 0; c < nc; ++c) {
                M[t][c] -= f * M[k][c];
                I[t][c] -= f * I[k][c];
            }
        }
        __syncthreads();
    }
    if (t < nc)
        for (int c = 0; c < nc; ++c) cinv[t * nc + c] = I[t][c];
}

template <class T>
__global__ void k_mg_coarsest_apply(const double *cinv, int nc, const T *r, T *zo) {
    const int t = threadIdx.x;
    if (t < nc) {
        double acc = 0;
        for (int c = 0; c < nc; ++c) acc += cinv[t * nc + c] * double(r[c]);
        zo[t] = T(acc);
    }
}

// CG start and update for the multilevel preconditioner: z, p and r . z come
// from the V-cycle (k_mg_post on the finest level).
template <class T>
__global__ void k_init_mg(const T *b, T *x, T *r, double *partial, long long n) {
    __shared__ double sh[32];
    double rr = 0;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        const T rv = b[s];
        x[s] = 0;
        r[s] = rv;
        rr += double(rv) * double(rv);
    }
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) partial[gridDim.x + blockIdx.x] = rr;
}

template <class T>
__global__ void k_update_mg(T *x, T *r, const T *p, const T *q, const double *scal, double *partial, long long n) {
    __shared__ double sh[32];
    const T alpha = T(scal[S_ALPHA]);
    double rr = 0;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        x[s] += alpha * p[s];
        const T rv = r[s] - alpha * q[s];
        r[s] = rv;
        rr += double(rv) * double(rv);
    }
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) partial[gridDim.x + blockIdx.x] = rr;
}

int grid_of(long long n) {
    long long g = (n + TB - 1) / TB;
    return int(g < PCG_BLOCKS ? (g < 1 ? 1 : g) : PCG_BLOCKS);
}

}  // namespace

size_t pcg_work_doubles(long long n) { return size_t(5) * (n + 32) + 6 * PCG_BLOCKS + S_NSCAL + 64; }

namespace {

constexpr int MG_MAX_LEV = 16;

template <class T>
struct MgPlan {
    int L = 0;                        // coarse levels 1..L (level L is the coarsest)
    MgLevelT<double> lev[MG_MAX_LEV + 1];  // lev[0]: the fine level (n only); coarse levels in FP64
    double *cinv = nullptr;           // coarsest dense inverse
    int *flag = nullptr;              // coarse-row overflow
};

// Carves the levels of an n-row solve out of `base` (null: sizes only);
// returns the doubles used.
template <class T>
size_t mg_plan(long long n, int cap, double *base, MgPlan<T> &pl) {
    auto pad = [](size_t k) { return (k + 31) & ~size_t(31); };
    size_t used = 0;
    // room for `count` elements of type E, in doubles
    auto take = [&](size_t count, auto *type) {
        using E = std::remove_pointer_t<decltype(type)>;
        E *p = base ? reinterpret_cast<E *>(base + used) : nullptr;
        used += pad((count * sizeof(E) + sizeof(double) - 1) / sizeof(double));
        return p;
    };
    pl = MgPlan<T>{};
    pl.lev[0].n = n;
    long long m = n;
    while (m > MG_COARSE && pl.L < MG_MAX_LEV) {
        m = (m + MG_B - 1) / MG_B;
        MgLevelT<double> &v = pl.lev[++pl.L];
        v.n = m;
        v.val = take(size_t(cap) * m, (double *)nullptr);
        v.dinv = take(m, (double *)nullptr);
        v.r = take(m, (double *)nullptr);
        v.z = take(m, (double *)nullptr);
        v.zo = take(m, (double *)nullptr);
        v.cnt = take(m, (int *)nullptr);
        v.col = take(size_t(cap) * m, (int *)nullptr);
    }
    if (pl.L > 0) {
        pl.cinv = take(size_t(MG_COARSE) * MG_COARSE, (double *)nullptr);
        pl.flag = take(1, (int *)nullptr);
    }
    return used;
}

int coarse_grid(long long n) {
    long long g = (n + TB - 1) / TB;
    return int(g < 148 * 8 ? (g < 1 ? 1 : g) : 148 * 8);
}

inline EllViewT<double> ell(const MgLevelT<double> &v) { return EllViewT<double>{v.cnt, v.col, v.val, v.n}; }

// Builds the coarse levels of A; false when a coarse row outgrew MG_CAP.
template <class M, int SLOTS, class T>
void mg_coarsen_all(const M &A, long long gauge, const double *scal, const MgPlan<T> &pl, cudaStream_t st) {
    for (int l = 1; l <= pl.L; ++l) {
        const int g = coarse_grid(32 * pl.lev[l].n);  // one warp per coarse row
        if (l == 1)
            k_mg_coarsen<M, SLOTS, double><<<g, TB, 0, st>>>(A, pl.lev[0].n, gauge, scal, pl.lev[1], pl.flag);
        else
            k_mg_coarsen<EllViewT<double>, SLOTS, double><<<g, TB, 0, st>>>(ell(pl.lev[l - 1]), pl.lev[l - 1].n, -1, scal,
                                                                  pl.lev[l], pl.flag);
        note_launch();
    }
}

template <class M, class T>
bool mg_setup(const M &A, long long gauge, const double *scal, const MgPlan<T> &pl, int cap, cudaStream_t st) {
    SDOT_CUDA(cudaMemsetAsync(pl.flag, 0, sizeof(int), st));
    if (cap > 64)
        mg_coarsen_all<M, 4>(A, gauge, scal, pl, st);
    else
        mg_coarsen_all<M, 2>(A, gauge, scal, pl, st);
    k_mg_coarsest_setup<double><<<1, MG_COARSE, 0, st>>>(ell(pl.lev[pl.L]), int(pl.lev[pl.L].n), pl.cinv);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
    int flag = 0;
    SDOT_CUDA(cudaMemcpyAsync(&flag, pl.flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    SDOT_CUDA(cudaStreamSynchronize(st));
    return flag == 0;
}

// z0 = V-cycle(r0) on the finest level (pre-smoothed values in zpre0), with
// r0 . z0 per block into partial[0 .. g) and, when p0 is given, p0 = z0.
template <class M, class T>
void mg_vcycle(const M &A, long long gauge, const double *scal, const T *dinv0, const MgPlan<T> &pl, const T *r0,
               T *zpre0, T *z0, double *partial, T *p0, int g, cudaStream_t st) {
    const long long n = pl.lev[0].n;
    k_mg_pre<M, T, double><<<g, TB, 0, st>>>(A, n, gauge, scal, dinv0, r0, zpre0, pl.lev[1].r);
    for (int l = 1; l < pl.L; ++l) {
        const MgLevelT<double> &v = pl.lev[l];
        k_mg_pre_coarse<<<coarse_grid(4 * v.n), TB, 0, st>>>(ell(v), v.n, v.dinv, v.r, v.z, pl.lev[l + 1].r);
    }
    const MgLevelT<double> &c = pl.lev[pl.L];
    k_mg_coarsest_apply<double><<<1, MG_COARSE, 0, st>>>(pl.cinv, int(c.n), c.r, c.zo);
    for (int l = pl.L - 1; l >= 1; --l) {
        const MgLevelT<double> &v = pl.lev[l];
        k_mg_post_coarse<<<coarse_grid(4 * v.n), TB, 0, st>>>(ell(v), v.n, v.dinv, v.r, v.z, pl.lev[l + 1].zo, v.zo);
    }
    k_mg_post<M, true, T, double><<<g, TB, 0, st>>>(A, n, gauge, scal, dinv0, r0, zpre0, pl.lev[1].zo, z0, partial, p0);
}

template <class T>
int mg_launches(const MgPlan<T> &pl) { return 2 * pl.L + 1; }

}  // namespace

size_t mg_work_doubles(long long n, int cap) {
    MgPlan<double> pl;
    return mg_plan(n, cap, nullptr, pl);
}

template <class T>
void pcg_bind(PcgWorkT<T> &w, double *base, long long n) {
    const long long m = n + 32;
    T *v = reinterpret_cast<T *>(base);
    w.r = v;
    w.z = v + m;
    w.p = v + 2 * m;
    w.q = v + 3 * m;
    w.dinv = v + 4 * m;
    w.partial = base + (5 * m * (long long)sizeof(T) + 7) / 8;
    w.scal = w.partial + 6 * PCG_BLOCKS;
}
template void pcg_bind<double>(PcgWorkT<double> &, double *, long long);
template void pcg_bind<float>(PcgWorkT<float> &, double *, long long);

namespace {

// stall_checks > 0: also stop once |r|^2 has not halved over the last
// stall_checks checks (the inner FP32 solves, whose attainable accuracy ends
// above the tolerance on ill-conditioned systems).
template <class M, class T>
PcgResult pcg_run(const M &A, long long n, long long gauge_row, const T *b, T *x, double rel_tol, int max_iter,
                  const PcgWorkT<T> &w, cudaStream_t st, int check, bool graph, bool multilevel,
                  int stall_checks = 0) {
    PcgResult res;
    if (n <= 0) {
        res.converged = true;
        return res;
    }
    const int g = grid_of(n);
    k_diag_inv<M, T><<<g, TB, 0, st>>>(A, n, gauge_row, w.dinv, w.scal);
    note_launch();
    MgPlan<T> pl;
    const int cap = w.mg_cap > 64 ? MG_CAP_MAX : 64;
    bool mg = multilevel && n > MG_COARSE && w.mg && mg_plan(n, cap, nullptr, pl) <= w.mg_doubles;
    if (mg) {
        mg_plan(n, cap, w.mg, pl);
        mg = mg_setup(A, gauge_row, w.scal, pl, cap, st);
    }
    if (mg) {
        k_init_mg<T><<<g, TB, 0, st>>>(b, x, w.r, w.partial, n);
        mg_vcycle(A, gauge_row, w.scal, w.dinv, pl, w.r, w.q, w.z, w.partial, w.p, g, st);
        for (int c = 0; c < 1 + mg_launches(pl); ++c) note_launch();
        res.levels = pl.L;
    } else {
        k_init<T><<<g, TB, 0, st>>>(b, x, w.r, w.z, w.p, w.dinv, w.partial, n);
        note_launch();
    }
    k_final<<<1, TB, 0, st>>>(w.partial, g, w.scal, 0);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
    double hs[S_NSCAL];
    SDOT_CUDA(cudaMemcpyAsync(hs, w.scal, sizeof(hs), cudaMemcpyDeviceToHost, st));
    SDOT_CUDA(cudaStreamSynchronize(st));
    const double rr0 = hs[S_RR0];
    if (rr0 == 0) {
        res.converged = true;
        return res;
    }
    const double target = rel_tol * rel_tol * rr0;
    auto launch_chunk = [&](int chunk) {
        for (int c = 0; c < chunk; ++c) {
            k_spmv<M, T><<<g, TB, 0, st>>>(A, n, gauge_row, w.p, w.q, w.scal, w.partial);
            k_final<<<1, TB, 0, st>>>(w.partial, g, w.scal, 1);
            if (mg) {
                // q is free once r is updated: it holds the pre-smoothed values
                k_update_mg<T><<<g, TB, 0, st>>>(x, w.r, w.p, w.q, w.scal, w.partial, n);
                mg_vcycle(A, gauge_row, w.scal, w.dinv, pl, w.r, w.q, w.z, w.partial, (T *)nullptr, g, st);
            } else {
                k_update<T><<<g, TB, 0, st>>>(x, w.r, w.z, w.p, w.q, w.dinv, w.scal, w.partial, n);
            }
            k_final<<<1, TB, 0, st>>>(w.partial, g, w.scal, 2);
            k_pupdate<T><<<g, TB, 0, st>>>(w.z, w.p, w.scal, n);
        }
    };
    const int per_iter = 5 + (mg ? mg_launches(pl) : 0);
    // With `graph`, a full chunk of iterations is captured once as a CUDA
    // graph and replayed: one launch instead of 5 * check.
    cudaGraphExec_t exec = nullptr;
    struct ExecGuard {
        cudaGraphExec_t &e;
        ~ExecGuard() {
            if (e) cudaGraphExecDestroy(e);
        }
    } exec_guard{exec};
    if (graph && max_iter >= check) {
        cudaGraph_t gr = nullptr;
        SDOT_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        launch_chunk(check);
        const cudaError_t le = cudaGetLastError();
        const cudaError_t ce = cudaStreamEndCapture(st, &gr);
        SDOT_CUDA(le);
        SDOT_CUDA(ce);
        const cudaError_t ie = cudaGraphInstantiate(&exec, gr, 0);
        cudaGraphDestroy(gr);
        SDOT_CUDA(ie);
    }
    int it = 0;
    double hist[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int nchecks = 0;
    while (it < max_iter) {
        const int chunk = check < max_iter - it ? check : max_iter - it;
        if (exec && chunk == check)
            SDOT_CUDA(cudaGraphLaunch(exec, st));
        else
            launch_chunk(chunk);
        for (int c = 0; c < per_iter * chunk; ++c) note_launch();
        SDOT_CUDA(cudaGetLastError());
        it += chunk;
        SDOT_CUDA(cudaMemcpyAsync(hs, w.scal, sizeof(hs), cudaMemcpyDeviceToHost, st));
        SDOT_CUDA(cudaStreamSynchronize(st));
        if (hs[S_BAD] != 0 || !(hs[S_RR] == hs[S_RR])) break;
        if (hs[S_RR] <= target) {
            res.converged = true;
            break;
        }
        if (stall_checks > 0) {
            const int k = stall_checks < 8 ? stall_checks : 8;
            if (nchecks >= k && !(hs[S_RR] <= 0.5 * hist[(nchecks - k) % 8])) break;
            hist[nchecks % 8] = hs[S_RR];
            ++nchecks;
        }
    }
    res.iterations = it;
    res.rel_residual = std::sqrt(hs[S_RR] / rr0);
    if (res.rel_residual <= rel_tol) res.converged = true;
    return res;
}

}  // namespace

PcgResult pcg_solve(const Rows &rows, long long n, long long gauge_row, const double *b, double *x, double rel_tol,
                    int max_iter, const PcgWork &w, cudaStream_t st, int check, bool graph, bool multilevel) {
    return pcg_run(rows_mat(rows), n, gauge_row, b, x, rel_tol, max_iter, w, st, check, graph, multilevel);
}

PcgResult pcg_solve_csr(const CsrMat &A, long long n, long long gauge_row, const double *b, double *x, double rel_tol,
                        int max_iter, const PcgWork &w, cudaStream_t st, int check) {
    return pcg_run(CsrView{A}, n, gauge_row, b, x, rel_tol, max_iter, w, st, check, false, false);
}

void mass_errors(const double *m, const double *t, long long n, double *partial, double *out, cudaStream_t st) {
    const int g = grid_of(n);
    k_mass_partial<<<g, TB, 0, st>>>(m, t, n, partial);
    note_launch();
    k_mass_final<<<1, 32, 0, st>>>(partial, g, out);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}

void axpby(const double *a, const double *b, double *out, double alpha, double beta, long long n, cudaStream_t st) {
    k_axpby<<<grid_of(n), TB, 0, st>>>(a, b, out, alpha, beta, n);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}

void apply_step(const double *w_base, const double *d_sorted, const int *idx, double tau, double *w_out, long long n,
                cudaStream_t st) {
    k_apply_step<<<grid_of(n), TB, 0, st>>>(w_base, d_sorted, idx, tau, w_out, n);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}

void gather_sorted(const double *t_orig, const int *idx, double *t_sorted, long long n, cudaStream_t st) {
    k_gather_sorted<<<grid_of(n), TB, 0, st>>>(t_orig, idx, t_sorted, n);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}

// ---- FP32 solves with FP64 iterative refinement ---------------------------
namespace {

// the Laplacian form of RowsLap32, one thread per row
__global__ void k_rows_to_float(Rows R, long long n, float *val32, float *side32) {
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        const int m = R.cnt[s];
        double rs = 0;
        for (int k = 0; k < m; ++k) rs += *R.valp(s, k);
        const bool side = m > R.cap;
        for (int k = 0; k < m; ++k) {
            const float v = float(*R.colp(s, k) == s ? rs : -*R.valp(s, k));
            if (side)
                side32[R.side[s] + k] = v;
            else
                val32[k * R.stride + s] = v;
        }
    }
}

// partial[block] = sum of v^2 over the block's entries
__global__ void k_sumsq(const double *v, long long n, double *partial) {
    __shared__ double sh[32];
    double a = 0;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x)
        a += v[s] * v[s];
    a = block_sum(a, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = a;
}
__global__ void k_sum_partials(const double *partial, int nb, double *out) {
    __shared__ double sh[32];
    double a = 0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) a += partial[i];
    a = block_sum(a, sh);
    if (threadIdx.x == 0) *out = a;
}
// out32 = scale * r (rounded to float)
__global__ void k_to_float(const double *r, double scale, float *out32, long long n) {
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x)
        out32[s] = float(scale * r[s]);
}
// x += scale * d (d in float or double)
template <class T>
__global__ void k_add_scaled(double *x, const T *d, double scale, long long n) {
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x)
        x[s] += scale * double(d[s]);
}
// r = b - (H + gauge term) x, in FP64
template <class M>
__global__ void k_residual(M A, long long n, long long g, const double *scal, const double *b, const double *x,
                           double *r) {
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        double v = A.row_dot(s, x);
        if (s == g) v += scal[S_GDIAG] * x[s];
        r[s] = b[s] - v;
    }
}

double sumsq(const double *v, long long n, double *partial, double *dev_out, cudaStream_t st) {
    const int g = grid_of(n);
    k_sumsq<<<g, TB, 0, st>>>(v, n, partial);
    k_sum_partials<<<1, TB, 0, st>>>(partial, g, dev_out);
    note_launch();
    note_launch();
    double h = 0;
    SDOT_CUDA(cudaMemcpyAsync(&h, dev_out, sizeof(double), cudaMemcpyDeviceToHost, st));
    SDOT_CUDA(cudaStreamSynchronize(st));
    return h;
}

}  // namespace

void rows_to_float(const Rows &rows, long long n, float *val32, float *side_val32, cudaStream_t st) {
    if (n <= 0) return;
    k_rows_to_float<<<PCG_BLOCKS, TB, 0, st>>>(rows, n, val32, side_val32);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}

PcgResult pcg_solve_refined(const Rows &rows, const float *val32, const float *side_val32, long long n,
                            long long gauge_row, const double *b, double *x, double rel_tol, int max_iter,
                            const PcgWork &w64, const PcgWorkT<float> &w32, double *res64, cudaStream_t st,
                            double inner_tol, int check, bool multilevel) {
    PcgResult res;
    if (n <= 0) {
        res.converged = true;
        return res;
    }
    const RowsMat A64 = rows_mat(rows);
    const RowsLap32 A32{rows, val32, side_val32};
    const int g = grid_of(n);
    double *r64 = res64;                                        // n doubles: the FP64 residual
    float *b32 = reinterpret_cast<float *>(res64 + n);          // n floats: the scaled residual
    float *d32 = b32 + n;                                       // n floats: the FP32 correction
    double *e64 = res64 + n;                                    // n doubles (FP64 fallback, reuses b32 / d32)
    double *dev_sum = w64.scal + S_NSCAL;                       // a spare device scalar
    // the FP64 gauge term (scal[S_GDIAG]) for the residuals
    k_diag_inv<RowsMat, double><<<g, TB, 0, st>>>(A64, n, gauge_row, w64.dinv, w64.scal);
    note_launch();
    SDOT_CUDA(cudaMemsetAsync(x, 0, size_t(n) * sizeof(double), st));
    SDOT_CUDA(cudaMemcpyAsync(r64, b, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, st));
    const double bb = sumsq(b, n, w64.partial, dev_sum, st);
    if (!(bb > 0)) {
        res.converged = bb == 0;
        return res;
    }
    const double target = rel_tol * rel_tol * bb;
    double rr = bb;
    int it = 0;
    bool fp32_ok = true;
    for (int outer = 0; outer < 60 && it < max_iter; ++outer) {
        if (rr <= target) break;
        const double nr = std::sqrt(rr);
        if (fp32_ok) {
            // the correction for the current residual, solved in FP32
            k_to_float<<<g, TB, 0, st>>>(r64, 1.0 / nr, b32, n);
            note_launch();
            const PcgResult in = pcg_run(A32, n, gauge_row, b32, d32, inner_tol, std::min(max_iter - it, 4000), w32,
                                         st, check, st != nullptr, multilevel, 4);
            it += in.iterations;
            res.levels = in.levels;
            k_add_scaled<float><<<g, TB, 0, st>>>(x, d32, nr, n);
        } else {
            // the rest in FP64: solve H e = r, x += e
            const PcgResult in = pcg_run(A64, n, gauge_row, r64, e64, std::sqrt(target / rr), max_iter - it, w64,
                                         st, check, st != nullptr, multilevel);
            it += in.iterations;
            res.levels = in.levels;
            k_add_scaled<double><<<g, TB, 0, st>>>(x, e64, 1.0, n);
        }
        note_launch();
        k_residual<RowsMat><<<g, TB, 0, st>>>(A64, n, gauge_row, w64.scal, b, x, r64);
        note_launch();
        SDOT_CUDA(cudaGetLastError());
        const double rr_new = sumsq(r64, n, w64.partial, dev_sum, st);
        if (!(rr_new == rr_new)) break;
        // an outer step that does not halve |r|: the FP32 matrix is too far
        // from H for this system
        if (fp32_ok && !(rr_new <= 0.25 * rr)) fp32_ok = false;
        rr = rr_new;
    }
    res.iterations = it;
    res.rel_residual = std::sqrt(rr / bb);
    res.converged = rr <= target;
    return res;
}

}  // namespace sdot
