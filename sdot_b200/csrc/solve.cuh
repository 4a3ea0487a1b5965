// Device linear algebra for Newton on the weights: preconditioned conjugate
// gradient on the Hessian rows (ELL + side buffer, sorted order), with a
// Jacobi or a multilevel (aggregation V-cycle) preconditioner.
//
// Replaces the reference's sparse direct solve EigenSolver::solve
// (src/sdot/Solvers/EigenSolver.cpp:9-41, Eigen::SimplicialCholesky) used by
// OptimalTransportSolver::solve (src/sdot/Solvers/OptimalTransportSolver.tcc:97-101).
#pragma once
#include "cell2d.cuh"
#include "common.cuh"

namespace sdot {

// Scratch of one PCG solve over n rows (device buffers owned by the caller).
// T: the precision of the vectors and of the matrix values (double, or float
// for the inner solves of the iterative refinement); the scalars of the
// iteration and every reduction stay in double.
template <class T>
struct PcgWorkT {
    T *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr, *dinv = nullptr;
    double *partial = nullptr;  // PCG_BLOCKS partial sums (x 2)
    double *scal = nullptr;     // device scalars (see solve.cu)
    double *mg = nullptr;       // multilevel storage (mg_work_doubles(n, mg_cap) doubles), or null
    size_t mg_doubles = 0;
    int mg_cap = 64;            // coarse row width: 64 or 128 (3D)
};
using PcgWork = PcgWorkT<double>;

// One coarse level of the multilevel preconditioner (device arrays).
template <class T>
struct MgLevelT {
    long long n = 0;
    int *cnt = nullptr, *col = nullptr;  // ELL rows (width PcgWork::mg_cap)
    T *val = nullptr, *dinv = nullptr;
    T *r = nullptr, *z = nullptr, *zo = nullptr;  // right-hand side, smoothed, output
};

// Doubles of multilevel storage a solve over n rows needs (coarse rows of
// width cap, 64 or 128).
size_t mg_work_doubles(long long n, int cap);
constexpr int PCG_BLOCKS = 148 * 4;

size_t pcg_work_doubles(long long n);
template <class T>
void pcg_bind(PcgWorkT<T> &w, double *base, long long n);

struct PcgResult {
    int iterations = 0;
    double rel_residual = 0;
    bool converged = false;
    int levels = 0;  // multilevel preconditioner levels (0: Jacobi)
};

// Solves (H + g e_g e_g^T) x = b where H is given by `rows` (sorted order,
// n rows) and the optional gauge term doubles the diagonal of row `gauge_row`
// (the reference's m_values[0] *= 2, OptimalTransportSolver.tcc:62-63);
// gauge_row < 0 disables it.  x starts at 0.  Stops when
// |r| <= rel_tol |b| or after max_iter iterations (checked every `check`
// iterations, the only host synchronisations).
// graph: replay full chunks of `check` iterations from one captured CUDA
// graph (st must be a created stream).
// multilevel: precondition with one V-cycle over Morton aggregates (needs
// w.mg); Jacobi when n is small, when w.mg is too small, or when a coarse row
// outgrows its ELL width.
PcgResult pcg_solve(const Rows &rows, long long n, long long gauge_row, const double *b, double *x, double rel_tol,
                    int max_iter, const PcgWork &w, cudaStream_t st, int check = 32, bool graph = false,
                    bool multilevel = false);

// The same system solved by iterative refinement: each outer step solves
// H d = r for the current FP64 residual r (scaled to unit norm) by PCG in FP32
// on an FP32 copy of the rows' values (val32 / side_val32: same layout as
// rows.val / rows.side_val; see rows_to_float), to the relative tolerance
// inner_tol, adds d to x in FP64 and recomputes r = b - H x with the FP64
// rows.  Stops at |r| <= rel_tol |b|.  An outer step that does not halve |r|
// (the FP32 matrix too far from H for this system) hands the rest of the
// solve to the FP64 PCG.  Iterations of both kinds are counted.
PcgResult pcg_solve_refined(const Rows &rows, const float *val32, const float *side_val32, long long n,
                            long long gauge_row, const double *b, double *x, double rel_tol, int max_iter,
                            const PcgWork &w64, const PcgWorkT<float> &w32, double *res64, cudaStream_t st,
                            double inner_tol = 1e-5, int check = 32, bool multilevel = true);
// FP32 copy of the rows' values in Laplacian form (off-diagonal entries:
// the edge weights -a_sj; diagonal entry: the row sum), same layout.
void rows_to_float(const Rows &rows, long long n, float *val32, float *side_val32, cudaStream_t st);

// The same solve on a CSR matrix (device arrays: off[n + 1], col[nnz], val[nnz]).
struct CsrMat {
    const long long *off = nullptr;
    const long long *col = nullptr;
    const double *val = nullptr;
};
PcgResult pcg_solve_csr(const CsrMat &A, long long n, long long gauge_row, const double *b, double *x, double rel_tol,
                        int max_iter, const PcgWork &w, cudaStream_t st, int check = 32);

// Device reductions used by the Newton loop (deterministic order).
// out[0] = max_i |m_i - t_i| / t_i, out[1] = min_i m_i, out[2] = sum_i (m_i - t_i)^2
void mass_errors(const double *m, const double *t, long long n, double *partial, double *out, cudaStream_t st);
// r = m - t
void axpby(const double *a, const double *b, double *out, double alpha, double beta, long long n, cudaStream_t st);
// w_orig[idx[s]] = w_base_orig[idx[s]] - tau * d_sorted[s]
void apply_step(const double *w_base, const double *d_sorted, const int *idx, double tau, double *w_out, long long n,
                cudaStream_t st);
// t_sorted[s] = t_orig[idx[s]]
void gather_sorted(const double *t_orig, const int *idx, double *t_sorted, long long n, cudaStream_t st);

}  // namespace sdot
