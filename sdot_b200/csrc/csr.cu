// Hessian row assembly (see csr.cuh).
#include "csr.cuh"

namespace sdot {

namespace {

constexpr int TB = 256;

// Merging never lengthens a row.  A side-buffer row whose merged count fits
// the ELL width is moved to its ELL slots, so that Rows::colp (which picks
// the storage from the count) stays consistent.
// STAGE (2D rows, short): rows of at most SM_ROW entries (every row of the
// fast tier) are sorted in shared memory: one gather of idx per entry, then
// the insertion sort and the merge on the staged copy (24% faster on the 1M
// 2D mix); longer rows, and every row without STAGE (3D rows are longer, and
// the staging area would cost them occupancy), are sorted in place.
constexpr int SM_ROW = 16;
constexpr int SM_TB = 128;

template <bool STAGE>
__global__ void __launch_bounds__(STAGE ? SM_TB : TB) k_sort_merge(Rows R, long long n, const int *idx,
                                                                   long long *cnt_orig) {
    __shared__ int s_key[STAGE ? SM_ROW * SM_TB : 1], s_col[STAGE ? SM_ROW * SM_TB : 1];
    __shared__ double s_val[STAGE ? SM_ROW * SM_TB : 1];
    const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int m = R.cnt[s];
#ifdef SDOT_CHECKS
    if (m < 0 || m > 4096 || (m > R.cap && (R.side[s] < 0 || R.side[s] + m > R.side_cap))) {
        check_fail(20, __LINE__, m);
        R.cnt[s] = 0;
        cnt_orig[idx[s]] = 0;
        return;
    }
    for (int i = 0; i < m; ++i) {
        const int c = *R.colp(s, i);
        if (c < 0 || c >= n) {
            check_fail(21, __LINE__, c);
            *R.colp(s, i) = int(s);
        }
    }
#endif
    int o = 0;
    if (STAGE && m <= SM_ROW) {
        // entry i of this thread at [i * SM_TB + t]: no bank conflicts
        const int t = threadIdx.x;
        for (int i = 0; i < m; ++i) {
            const int c = *R.colp(s, i);
            s_col[i * SM_TB + t] = c;
            s_val[i * SM_TB + t] = *R.valp(s, i);
            s_key[i * SM_TB + t] = idx[c];
        }
        // insertion sort by (original column, value), as below
        for (int i = 1; i < m; ++i) {
            const int oc = s_key[i * SM_TB + t], c = s_col[i * SM_TB + t];
            const double v = s_val[i * SM_TB + t];
            int j = i - 1;
            while (j >= 0) {
                const int ocj = s_key[j * SM_TB + t];
                const double vj = s_val[j * SM_TB + t];
                if (ocj < oc || (ocj == oc && !(vj > v))) break;
                s_key[(j + 1) * SM_TB + t] = ocj;
                s_col[(j + 1) * SM_TB + t] = s_col[j * SM_TB + t];
                s_val[(j + 1) * SM_TB + t] = vj;
                --j;
            }
            s_key[(j + 1) * SM_TB + t] = oc;
            s_col[(j + 1) * SM_TB + t] = c;
            s_val[(j + 1) * SM_TB + t] = v;
        }
        // merge equal columns (each into the next) and write back
        for (int i = 0; i < m; ++i) {
            const int c = s_col[i * SM_TB + t];
            const double v = s_val[i * SM_TB + t];
            if (i + 1 < m && s_col[(i + 1) * SM_TB + t] == c) {
                s_val[(i + 1) * SM_TB + t] += v;
                continue;
            }
            *R.colp(s, o) = c;
            *R.valp(s, o) = v;
            ++o;
        }
    } else {
        // insertion sort in place
        for (int i = 1; i < m; ++i) {
            const int c = *R.colp(s, i);
            const double v = *R.valp(s, i);
            const int oc = idx[c];
            int j = i - 1;
            while (j >= 0) {
                const int cj = *R.colp(s, j);
                const int ocj = idx[cj];
                const double vj = *R.valp(s, j);
                if (ocj < oc || (ocj == oc && !(vj > v))) break;
                *R.colp(s, j + 1) = cj;
                *R.valp(s, j + 1) = vj;
                --j;
            }
            *R.colp(s, j + 1) = c;
            *R.valp(s, j + 1) = v;
        }
        // merge equal columns
        for (int i = 0; i < m; ++i) {
            const int c = *R.colp(s, i);
            const double v = *R.valp(s, i);
            if (i + 1 < m && *R.colp(s, i + 1) == c) {
                *R.valp(s, i + 1) += v;
                continue;
            }
            *R.colp(s, o) = c;
            *R.valp(s, o) = v;
            ++o;
        }
    }
    if (m > R.cap && o <= R.cap) {
        for (int k = 0; k < o; ++k) {
            const int c = *R.colp(s, k);
            const double v = *R.valp(s, k);
            R.col[k * R.stride + s] = c;
            R.val[k * R.stride + s] = v;
        }
    }
    R.cnt[s] = o;
    cnt_orig[idx[s]] = o;
}

__global__ void k_write(Rows R, long long n, const int *idx, const long long *offsets, long long *cols, double *vals) {
    const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int m = R.cnt[s];
    const long long o = offsets[idx[s]];
    for (int i = 0; i < m; ++i) {
        cols[o + i] = idx[*R.colp(s, i)];
        vals[o + i] = *R.valp(s, i);
    }
}

__global__ void k_nb_counts(Rows NB, long long n, const int *idx, long long *cnt_orig) {
    const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s >= n) return;
    cnt_orig[idx[s]] = NB.cnt[s];
}

__global__ void k_nb_write(Rows NB, long long n, const int *idx, const long long *offsets, long long *ids) {
    const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int m = NB.cnt[s];
    const long long o = offsets[idx[s]];
    for (int i = 0; i < m; ++i) {
        const int id = *NB.colp(s, i);
        // periodic images: id j + (k + 1) n keeps its translation k
        ids[o + i] = id >= 0 ? (long long)idx[id % n] + (long long)(id / n) * n : (id == ID_ARC ? -2 : -1);
    }
}

__global__ void k_unpermute(const double *in, double *out, long long n, int d, const int *idx) {
    const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s >= n) return;
    const long long i = idx[s];
    for (int k = 0; k < d; ++k) out[i * d + k] = in[s * d + k];
}

// number of zero entries (empty cells), added to *count
__global__ void k_count_zeros(const double *m, long long n, unsigned long long *count) {
    const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int z = __syncthreads_count(s < n && m[s] == 0.0);  // one atomic per block
    if (threadIdx.x == 0 && z) atomicAdd(count, (unsigned long long)z);
}

// ---- domains of several shapes: one cell pass per shape, summed here
__global__ void k_rows_clear(Rows R, long long n) {
    const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s < n) R.cnt[s] = 0;
}

// dst row s += src row s (entries appended; a row that outgrows the ELL
// width moves, with the new entries, to a fresh place in the side buffer)
__global__ void k_rows_append(Rows dst, Rows src, long long n, unsigned *err) {
    const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int m0 = dst.cnt[s], m1 = src.cnt[s], m = m0 + m1;
    if (m1 == 0) return;
    if (m <= dst.cap) {
        for (int k = 0; k < m1; ++k) {
            dst.col[(m0 + k) * dst.stride + s] = *src.colp(s, k);
            if (dst.val) dst.val[(m0 + k) * dst.stride + s] = *src.valp(s, k);
        }
        dst.cnt[s] = m;
        return;
    }
    const unsigned long long off = atomicAdd(dst.side_used, (unsigned long long)m);
    if ((long long)(off + m) > dst.side_cap) {
        atomicOr(err, unsigned(DE_SIDE));
        return;
    }
    for (int k = 0; k < m0; ++k) {
        dst.side_col[off + k] = *dst.colp(s, k);
        if (dst.side_val) dst.side_val[off + k] = *dst.valp(s, k);
    }
    for (int k = 0; k < m1; ++k) {
        dst.side_col[off + m0 + k] = *src.colp(s, k);
        if (dst.side_val) dst.side_val[off + m0 + k] = *src.valp(s, k);
    }
    dst.side[s] = (long long)off;
    dst.cnt[s] = m;
}

// mass += t_mass, mass_c += t_mass_c, mom += t_ctd * t_mass_c (dim 2 or 3)
__global__ void k_accum(double *mass, double *mass_c, double *mom, const double *t_mass, const double *t_mass_c,
                        const double *t_ctd, long long n, int dim) {
    const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s >= n) return;
    mass[s] += t_mass[s];
    mass_c[s] += t_mass_c[s];
    for (int d = 0; d < dim; ++d) mom[dim * s + d] += t_ctd[dim * s + d] * t_mass_c[s];
}

// centroid = moment / (mass + (mass == 0)), as get_centroids divides
__global__ void k_ctd_final(double *ctd, const double *mom, const double *mass_c, long long n, int dim) {
    const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s >= n) return;
    const double d = mass_c[s] + (mass_c[s] == 0);
    for (int k = 0; k < dim; ++k) ctd[dim * s + k] = mom[dim * s + k] / d;
}

}  // namespace

void csr_read_checks(unsigned long long out[3]) {
#ifdef SDOT_CHECKS
    SDOT_CUDA(cudaMemcpyFromSymbol(out, sdot_dbg_word, 3 * sizeof(unsigned long long)));
#else
    out[0] = out[1] = out[2] = 0;
#endif
}

void csr_sort_merge(const Rows &R, long long n, const int *idx, long long *cnt_orig, bool short_rows, cudaStream_t st) {
    if (n <= 0) return;
    if (short_rows)
        k_sort_merge<true><<<ceil_div(n, SM_TB), SM_TB, 0, st>>>(R, n, idx, cnt_orig);
    else
        k_sort_merge<false><<<ceil_div(n, TB), TB, 0, st>>>(R, n, idx, cnt_orig);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}
void csr_write(const Rows &R, long long n, const int *idx, const long long *offsets, long long *cols, double *vals,
               cudaStream_t st) {
    if (n <= 0) return;
    k_write<<<ceil_div(n, TB), TB, 0, st>>>(R, n, idx, offsets, cols, vals);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}
void nb_counts(const Rows &NB, long long n, const int *idx, long long *cnt_orig, cudaStream_t st) {
    if (n <= 0) return;
    k_nb_counts<<<ceil_div(n, TB), TB, 0, st>>>(NB, n, idx, cnt_orig);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}
void nb_write(const Rows &NB, long long n, const int *idx, const long long *offsets, long long *ids, cudaStream_t st) {
    if (n <= 0) return;
    k_nb_write<<<ceil_div(n, TB), TB, 0, st>>>(NB, n, idx, offsets, ids);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}
void unpermute(const double *in, double *out, long long n, int d, const int *idx, cudaStream_t st) {
    if (n <= 0) return;
    k_unpermute<<<ceil_div(n, TB), TB, 0, st>>>(in, out, n, d, idx);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}

void rows_clear(const Rows &R, long long n, cudaStream_t st) {
    if (n <= 0) return;
    k_rows_clear<<<ceil_div(n, TB), TB, 0, st>>>(R, n);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}
void rows_append(const Rows &dst, const Rows &src, long long n, unsigned *err, cudaStream_t st) {
    if (n <= 0) return;
    k_rows_append<<<ceil_div(n, TB), TB, 0, st>>>(dst, src, n, err);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}
void accum_pass(double *mass, double *mass_c, double *mom, const double *t_mass, const double *t_mass_c,
                const double *t_ctd, long long n, int dim, cudaStream_t st) {
    if (n <= 0) return;
    k_accum<<<ceil_div(n, TB), TB, 0, st>>>(mass, mass_c, mom, t_mass, t_mass_c, t_ctd, n, dim);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}
void centroids_final(double *ctd, const double *mom, const double *mass_c, long long n, int dim, cudaStream_t st) {
    if (n <= 0) return;
    k_ctd_final<<<ceil_div(n, TB), TB, 0, st>>>(ctd, mom, mass_c, n, dim);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}

void count_zeros(const double *m, long long n, unsigned long long *count, cudaStream_t st) {
    if (n <= 0) return;
    k_count_zeros<<<ceil_div(n, TB), TB, 0, st>>>(m, n, count);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}

}  // namespace sdot
