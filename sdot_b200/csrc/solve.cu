// Preconditioned conjugate gradients on the device (see solve.cuh).
//
// Every reduction is two-stage with a fixed order (per-block partials, then
// one block sums them), so a solve is bitwise reproducible run to run.  The
// scalars of the iteration (alpha, beta, |r|^2) stay on the device; the host
// only reads |r|^2 every `check` iterations to decide to stop.
#include "solve.cuh"

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

// Matrix views for the PCG kernels: row s times x, and the diagonal entry.
struct RowsMat {
    Rows R;
    __device__ double row_dot(long long s, const double *x) const {
        const int m = R.cnt[s];
        double acc = 0;
        if (m <= R.cap) {
            for (int k = 0; k < m; ++k) acc += R.val[k * R.stride + s] * x[R.col[k * R.stride + s]];
        } else {
            const long long o = R.side[s];
            for (int k = 0; k < m; ++k) acc += R.side_val[o + k] * x[R.side_col[o + k]];
        }
        return acc;
    }
    __device__ double diag(long long s) const {
        double d = 0;
        for (int k = 0, m = R.cnt[s]; k < m; ++k)
            if (*R.colp(s, k) == s) d += *R.valp(s, k);
        return d;
    }
    __device__ int len(long long s) const { return R.cnt[s]; }
    __device__ long long colk(long long s, int k) const { return *R.colp(s, k); }
    __device__ double valk(long long s, int k) const { return *R.valp(s, k); }
    // sum_k a_sk f(col_sk)
    template <class F>
    __device__ double row_sum(long long s, const F &f) const {
        const int m = R.cnt[s];
        double acc = 0;
        if (m <= R.cap) {
            for (int k = 0; k < m; ++k) acc += R.val[k * R.stride + s] * f(R.col[k * R.stride + s]);
        } else {
            const long long o = R.side[s];
            for (int k = 0; k < m; ++k) acc += R.side_val[o + k] * f(R.side_col[o + k]);
        }
        return acc;
    }
};
struct CsrView {
    CsrMat M;
    __device__ double row_dot(long long s, const double *x) const {
        double acc = 0;
        for (long long k = M.off[s], e = M.off[s + 1]; k < e; ++k) acc += M.val[k] * x[M.col[k]];
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

struct EllView {
    const int *cnt;
    const int *col;
    const double *val;
    long long stride;
    __device__ int len(long long s) const { return cnt[s]; }
    __device__ long long colk(long long s, int k) const { return col[k * stride + s]; }
    __device__ double valk(long long s, int k) const { return val[k * stride + s]; }
    template <class F>
    __device__ double row_sum(long long s, const F &f) const {
        double acc = 0;
        for (int k = 0, m = cnt[s]; k < m; ++k) acc += val[k * stride + s] * f(col[k * stride + s]);
        return acc;
    }
};

template <class M>
__global__ void k_diag_inv(M A, long long n, long long g, double *dinv, double *scal) {
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        double d = A.diag(s);
        if (s == g) {
            scal[S_GDIAG] = d;
            d *= 2;
        }
        dinv[s] = d != 0 ? 1.0 / d : 0.0;
    }
}

__global__ void k_init(const double *b, double *x, double *r, double *z, double *p, const double *dinv, double *partial,
                       long long n) {
    __shared__ double sh[32];
    double rz = 0, rr = 0;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        const double rv = b[s];
        const double zv = dinv[s] * rv;
        x[s] = 0;
        r[s] = rv;
        z[s] = zv;
        p[s] = zv;
        rz += rv * zv;
        rr += rv * rv;
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

template <class M>
__global__ void k_spmv(M A, long long n, long long g, const double *p, double *q, const double *scal,
                       double *partial) {
    __shared__ double sh[32];
    double pq = 0;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        double v = A.row_dot(s, p);
        if (s == g) v += scal[S_GDIAG] * p[s];
        q[s] = v;
        pq += p[s] * v;
    }
    pq = block_sum(pq, sh);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = pq;
        partial[gridDim.x + blockIdx.x] = 0;
    }
}

__global__ void k_update(double *x, double *r, double *z, const double *p, const double *q, const double *dinv,
                         const double *scal, double *partial, long long n) {
    __shared__ double sh[32];
    const double alpha = scal[S_ALPHA];
    double rz = 0, rr = 0;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        x[s] += alpha * p[s];
        const double rv = r[s] - alpha * q[s];
        r[s] = rv;
        const double zv = dinv[s] * rv;
        z[s] = zv;
        rz += rv * zv;
        rr += rv * rv;
    }
    rz = block_sum(rz, sh);
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = rz;
        partial[gridDim.x + blockIdx.x] = rr;
    }
}

__global__ void k_pupdate(const double *z, double *p, const double *scal, long long n) {
    const double beta = scal[S_BETA];
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
template <class M, int SLOTS>
__global__ void k_mg_coarsen(M A, long long nf, long long gauge, const double *scal, MgLevel out, int *flag) {
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
                out.val[(lane + 32 * q) * out.n + c] = v[q];
                if (key[q] == c) diag = v[q];
            }
        for (int o = 16; o > 0; o >>= 1) diag += __shfl_xor_sync(FULL, diag, o);
        if (lane == 0) {
            out.cnt[c] = count;
            out.dinv[c] = diag > 0 ? 1.0 / diag : 0.0;
            if (over) atomicExch(flag, 1);
        }
    }
}

// Pre-smoothing and restriction of one level: z = w D^-1 r, and
// rc[aggregate] = sum over its rows of (r - A z).  Rows are taken a block at a
// time so that the MG_B rows of an aggregate sit in consecutive lanes.
template <class M>
__global__ void k_mg_pre(M A, long long n, long long gauge, const double *scal, const double *dinv, const double *r,
                         double *z, double *rc) {
    const unsigned FULL = 0xffffffffu;
    for (long long i0 = blockIdx.x * (long long)blockDim.x; i0 < n; i0 += (long long)gridDim.x * blockDim.x) {
        const long long i = i0 + threadIdx.x;
        double t = 0;
        if (i < n) {
            const double ri = r[i];
            const double zi = MG_OMEGA * dinv[i] * ri;
            z[i] = zi;
            double acc = A.row_sum(i, [&](long long j) { return MG_OMEGA * dinv[j] * r[j]; });
            if (i == gauge) acc += scal[S_GDIAG] * zi;
            t = ri - acc;
        }
        for (int o = MG_B / 2; o > 0; o >>= 1) t += __shfl_down_sync(FULL, t, o, MG_B);
        if ((threadIdx.x & (MG_B - 1)) == 0 && i < n) rc[i / MG_B] = t;
    }
}

// Coarse correction and post-smoothing: z' = z + P zc, zo = z' + w D^-1 (r - A z').
// On the finest level (FINE) it also sums r . zo per block into partial[]
// and, when p is given, writes p = zo (the first CG direction).
template <class M, bool FINE>
__global__ void k_mg_post(M A, long long n, long long gauge, const double *scal, const double *dinv, const double *r,
                          const double *z, const double *zc, double *zo, double *partial, double *p) {
    __shared__ double sh[32];
    double rz = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        auto zp = [&](long long j) { return z[j] + zc[j / MG_B]; };
        const double zi = zp(i);
        double acc = A.row_sum(i, zp);
        if (i == gauge) acc += scal[S_GDIAG] * zi;
        const double v = zi + MG_OMEGA * dinv[i] * (r[i] - acc);
        zo[i] = v;
        if (FINE) {
            rz += r[i] * v;
            if (p) p[i] = v;
        }
    }
    if (FINE) {
        rz = block_sum(rz, sh);
        if (threadIdx.x == 0) partial[blockIdx.x] = rz;
    }
}

// Dense inverse of the coarsest level (nc <= MG_COARSE rows, one block of
// MG_COARSE threads, thread t owns row t).  Gauss-Jordan without pivoting
// (the matrix is symmetric positive semi-definite); a pivot below 1e-13 of
// the largest diagonal entry marks a null direction, left out of the inverse.
__global__ void k_mg_coarsest_setup(EllView A, int nc, double *cinv) {
    __shared__ double M[MG_COARSE][MG_COARSE + 1], I[MG_COARSE][MG_COARSE + 1];
    __shared__ double dmax;
    const int t = threadIdx.x;
    if (t < nc) {
        for (int c = 0; c < nc; ++c) {
            M[t][c] = 0;
            I[t][c] = c == t ? 1.0 : 0.0;
        }
        for (int k = 0, m = A.cnt[t]; k < m; ++k) M[t][A.col[k * A.stride + t]] += A.val[k * A.stride + t];
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

__global__ void k_mg_coarsest_apply(const double *cinv, int nc, const double *r, double *zo) {
    const int t = threadIdx.x;
    if (t < nc) {
        double acc = 0;
        for (int c = 0; c < nc; ++c) acc += cinv[t * nc + c] * r[c];
        zo[t] = acc;
    }
}

// CG start and update for the multilevel preconditioner: z, p and r . z come
// from the V-cycle (k_mg_post on the finest level).
__global__ void k_init_mg(const double *b, double *x, double *r, double *partial, long long n) {
    __shared__ double sh[32];
    double rr = 0;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        const double rv = b[s];
        x[s] = 0;
        r[s] = rv;
        rr += rv * rv;
    }
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) partial[gridDim.x + blockIdx.x] = rr;
}

__global__ void k_update_mg(double *x, double *r, const double *p, const double *q, const double *scal,
                            double *partial, long long n) {
    __shared__ double sh[32];
    const double alpha = scal[S_ALPHA];
    double rr = 0;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        x[s] += alpha * p[s];
        const double rv = r[s] - alpha * q[s];
        r[s] = rv;
        rr += rv * rv;
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

struct MgPlan {
    int L = 0;                     // coarse levels 1..L (level L is the coarsest)
    MgLevel lev[MG_MAX_LEV + 1];   // lev[0]: the fine level (n only)
    double *cinv = nullptr;        // coarsest dense inverse
    int *flag = nullptr;           // coarse-row overflow
};

// Carves the levels of an n-row solve out of `base` (null: sizes only);
// returns the doubles used.
size_t mg_plan(long long n, int cap, double *base, MgPlan &pl) {
    auto pad = [](size_t k) { return (k + 31) & ~size_t(31); };
    size_t used = 0;
    auto take = [&](size_t doubles) {
        double *p = base ? base + used : nullptr;
        used += pad(doubles);
        return p;
    };
    pl = MgPlan{};
    pl.lev[0].n = n;
    long long m = n;
    while (m > MG_COARSE && pl.L < MG_MAX_LEV) {
        m = (m + MG_B - 1) / MG_B;
        MgLevel &v = pl.lev[++pl.L];
        v.n = m;
        v.val = take(size_t(cap) * m);
        v.dinv = take(m);
        v.r = take(m);
        v.z = take(m);
        v.zo = take(m);
        v.cnt = reinterpret_cast<int *>(take((m + 1) / 2));
        v.col = reinterpret_cast<int *>(take((size_t(cap) * m + 1) / 2));
    }
    if (pl.L > 0) {
        pl.cinv = take(size_t(MG_COARSE) * MG_COARSE);
        pl.flag = reinterpret_cast<int *>(take(1));
    }
    return used;
}

int coarse_grid(long long n) {
    long long g = (n + TB - 1) / TB;
    return int(g < 148 * 8 ? (g < 1 ? 1 : g) : 148 * 8);
}

EllView ell(const MgLevel &v) { return EllView{v.cnt, v.col, v.val, v.n}; }

// Builds the coarse levels of A; false when a coarse row outgrew MG_CAP.
template <class M, int SLOTS>
void mg_coarsen_all(const M &A, long long gauge, const double *scal, const MgPlan &pl, cudaStream_t st) {
    for (int l = 1; l <= pl.L; ++l) {
        const int g = coarse_grid(32 * pl.lev[l].n);  // one warp per coarse row
        if (l == 1)
            k_mg_coarsen<M, SLOTS><<<g, TB, 0, st>>>(A, pl.lev[0].n, gauge, scal, pl.lev[1], pl.flag);
        else
            k_mg_coarsen<EllView, SLOTS><<<g, TB, 0, st>>>(ell(pl.lev[l - 1]), pl.lev[l - 1].n, -1, scal, pl.lev[l],
                                                          pl.flag);
        note_launch();
    }
}

template <class M>
bool mg_setup(const M &A, long long gauge, const double *scal, const MgPlan &pl, int cap, cudaStream_t st) {
    SDOT_CUDA(cudaMemsetAsync(pl.flag, 0, sizeof(int), st));
    if (cap > 64)
        mg_coarsen_all<M, 4>(A, gauge, scal, pl, st);
    else
        mg_coarsen_all<M, 2>(A, gauge, scal, pl, st);
    k_mg_coarsest_setup<<<1, MG_COARSE, 0, st>>>(ell(pl.lev[pl.L]), int(pl.lev[pl.L].n), pl.cinv);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
    int flag = 0;
    SDOT_CUDA(cudaMemcpyAsync(&flag, pl.flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    SDOT_CUDA(cudaStreamSynchronize(st));
    return flag == 0;
}

// z0 = V-cycle(r0) on the finest level (pre-smoothed values in zpre0), with
// r0 . z0 per block into partial[0 .. g) and, when p0 is given, p0 = z0.
template <class M>
void mg_vcycle(const M &A, long long gauge, const double *scal, const double *dinv0, const MgPlan &pl,
               const double *r0, double *zpre0, double *z0, double *partial, double *p0, int g, cudaStream_t st) {
    const long long n = pl.lev[0].n;
    k_mg_pre<M><<<g, TB, 0, st>>>(A, n, gauge, scal, dinv0, r0, zpre0, pl.lev[1].r);
    for (int l = 1; l < pl.L; ++l) {
        const MgLevel &v = pl.lev[l];
        k_mg_pre<EllView><<<coarse_grid(v.n), TB, 0, st>>>(ell(v), v.n, -1, scal, v.dinv, v.r, v.z, pl.lev[l + 1].r);
    }
    const MgLevel &c = pl.lev[pl.L];
    k_mg_coarsest_apply<<<1, MG_COARSE, 0, st>>>(pl.cinv, int(c.n), c.r, c.zo);
    for (int l = pl.L - 1; l >= 1; --l) {
        const MgLevel &v = pl.lev[l];
        k_mg_post<EllView, false><<<coarse_grid(v.n), TB, 0, st>>>(ell(v), v.n, -1, scal, v.dinv, v.r, v.z,
                                                                   pl.lev[l + 1].zo, v.zo, nullptr, nullptr);
    }
    k_mg_post<M, true><<<g, TB, 0, st>>>(A, n, gauge, scal, dinv0, r0, zpre0, pl.lev[1].zo, z0, partial, p0);
}

int mg_launches(const MgPlan &pl) { return 2 * pl.L + 1; }

}  // namespace

size_t mg_work_doubles(long long n, int cap) {
    MgPlan pl;
    return mg_plan(n, cap, nullptr, pl);
}

void pcg_bind(PcgWork &w, double *base, long long n) {
    const long long m = n + 32;
    w.r = base;
    w.z = base + m;
    w.p = base + 2 * m;
    w.q = base + 3 * m;
    w.dinv = base + 4 * m;
    w.partial = base + 5 * m;
    w.scal = w.partial + 6 * PCG_BLOCKS;
}

namespace {

template <class M>
PcgResult pcg_run(const M &A, long long n, long long gauge_row, const double *b, double *x, double rel_tol,
                  int max_iter, const PcgWork &w, cudaStream_t st, int check, bool graph, bool multilevel) {
    PcgResult res;
    if (n <= 0) {
        res.converged = true;
        return res;
    }
    const int g = grid_of(n);
    k_diag_inv<M><<<g, TB, 0, st>>>(A, n, gauge_row, w.dinv, w.scal);
    note_launch();
    MgPlan pl;
    const int cap = w.mg_cap > 64 ? MG_CAP_MAX : 64;
    bool mg = multilevel && n > MG_COARSE && w.mg && mg_plan(n, cap, nullptr, pl) <= w.mg_doubles;
    if (mg) {
        mg_plan(n, cap, w.mg, pl);
        mg = mg_setup(A, gauge_row, w.scal, pl, cap, st);
    }
    if (mg) {
        k_init_mg<<<g, TB, 0, st>>>(b, x, w.r, w.partial, n);
        mg_vcycle(A, gauge_row, w.scal, w.dinv, pl, w.r, w.q, w.z, w.partial, w.p, g, st);
        for (int c = 0; c < 1 + mg_launches(pl); ++c) note_launch();
        res.levels = pl.L;
    } else {
        k_init<<<g, TB, 0, st>>>(b, x, w.r, w.z, w.p, w.dinv, w.partial, n);
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
            k_spmv<M><<<g, TB, 0, st>>>(A, n, gauge_row, w.p, w.q, w.scal, w.partial);
            k_final<<<1, TB, 0, st>>>(w.partial, g, w.scal, 1);
            if (mg) {
                // q is free once r is updated: it holds the pre-smoothed values
                k_update_mg<<<g, TB, 0, st>>>(x, w.r, w.p, w.q, w.scal, w.partial, n);
                mg_vcycle(A, gauge_row, w.scal, w.dinv, pl, w.r, w.q, w.z, w.partial, nullptr, g, st);
            } else {
                k_update<<<g, TB, 0, st>>>(x, w.r, w.z, w.p, w.q, w.dinv, w.scal, w.partial, n);
            }
            k_final<<<1, TB, 0, st>>>(w.partial, g, w.scal, 2);
            k_pupdate<<<g, TB, 0, st>>>(w.z, w.p, w.scal, n);
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
    }
    res.iterations = it;
    res.rel_residual = std::sqrt(hs[S_RR] / rr0);
    if (res.rel_residual <= rel_tol) res.converged = true;
    return res;
}

}  // namespace

PcgResult pcg_solve(const Rows &rows, long long n, long long gauge_row, const double *b, double *x, double rel_tol,
                    int max_iter, const PcgWork &w, cudaStream_t st, int check, bool graph, bool multilevel) {
    return pcg_run(RowsMat{rows}, n, gauge_row, b, x, rel_tol, max_iter, w, st, check, graph, multilevel);
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

}  // namespace sdot
