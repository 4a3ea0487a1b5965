// Hessian row assembly: rows in sorted (Morton) order -> reference CSR.
#pragma once
#include "cell2d.cuh"
#include "common.cuh"

namespace sdot {

// Sort each row by (original column, value) and merge equal columns the way
// get_der_integrals_wrt_weights does (get_der_integrals_wrt_weights.h:76-88):
// values of equal columns are summed in ascending value order.  Rewrites the
// rows in place and stores the merged count both in R.cnt[s] (rows keep
// their storage) and in cnt_orig[idx[s]] (original order, for the scan).
// short_rows: stage rows of at most 16 entries in shared memory (2D rows)
void csr_sort_merge(const Rows &R, long long n, const int *idx, long long *cnt_orig, bool short_rows, cudaStream_t st);
// Write rows to CSR in original order: columns as original indices (int64).
void csr_write(const Rows &R, long long n, const int *idx, const long long *offsets, long long *cols, double *vals,
               cudaStream_t st);
// Neighbour lists: ids mapped (sorted -> original; domain edges -> -1; arcs -> -2).
void nb_counts(const Rows &NB, long long n, const int *idx, long long *cnt_orig, cudaStream_t st);
void nb_write(const Rows &NB, long long n, const int *idx, const long long *offsets, long long *ids, cudaStream_t st);
// First failed debug check of the assembly kernels (zeros in release builds).
void csr_read_checks(unsigned long long out[3]);
// Domains of several shapes (one cell pass per shape): empty all rows;
// append the rows of one pass; sum one pass's masses and centroid moments;
// divide the moments (get_centroids' mass + (mass == 0)).
void rows_clear(const Rows &R, long long n, cudaStream_t st);
void rows_append(const Rows &dst, const Rows &src, long long n, unsigned *err, cudaStream_t st);
void accum_pass(double *mass, double *mass_c, double *mom, const double *t_mass, const double *t_mass_c,
                const double *t_ctd, long long n, int dim, cudaStream_t st);
void centroids_final(double *ctd, const double *mom, const double *mass_c, long long n, int dim, cudaStream_t st);
// *count += number of i < n with m[i] == 0 (the empty cells)
void count_zeros(const double *m, long long n, unsigned long long *count, cudaStream_t st);
// out[idx[s] * d + k] = in[s * d + k]
void unpermute(const double *in, double *out, long long n, int d, const int *idx, cudaStream_t st);

}  // namespace sdot
