// Jacobi-PCG on the device (see solve.cuh).
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

int grid_of(long long n) {
    long long g = (n + TB - 1) / TB;
    return int(g < PCG_BLOCKS ? (g < 1 ? 1 : g) : PCG_BLOCKS);
}

}  // namespace

size_t pcg_work_doubles(long long n) { return size_t(5) * (n + 32) + 6 * PCG_BLOCKS + S_NSCAL + 64; }

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
                  int max_iter, const PcgWork &w, cudaStream_t st, int check, bool graph) {
    PcgResult res;
    if (n <= 0) {
        res.converged = true;
        return res;
    }
    const int g = grid_of(n);
    k_diag_inv<M><<<g, TB, 0, st>>>(A, n, gauge_row, w.dinv, w.scal);
    note_launch();
    k_init<<<g, TB, 0, st>>>(b, x, w.r, w.z, w.p, w.dinv, w.partial, n);
    note_launch();
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
            k_update<<<g, TB, 0, st>>>(x, w.r, w.z, w.p, w.q, w.dinv, w.scal, w.partial, n);
            k_final<<<1, TB, 0, st>>>(w.partial, g, w.scal, 2);
            k_pupdate<<<g, TB, 0, st>>>(w.z, w.p, w.scal, n);
        }
    };
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
        for (int c = 0; c < 5 * chunk; ++c) note_launch();
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
                    int max_iter, const PcgWork &w, cudaStream_t st, int check, bool graph) {
    return pcg_run(RowsMat{rows}, n, gauge_row, b, x, rel_tol, max_iter, w, st, check, graph);
}

PcgResult pcg_solve_csr(const CsrMat &A, long long n, long long gauge_row, const double *b, double *x, double rel_tol,
                        int max_iter, const PcgWork &w, cudaStream_t st, int check) {
    return pcg_run(CsrView{A}, n, gauge_row, b, x, rel_tol, max_iter, w, st, check, false);
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
