// Exclusive scan and stable LSD radix sort (see prims.cuh).
#include "prims.cuh"

namespace sdot {

namespace {

constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

template <class T>
__device__ T block_exclusive_scan(T v, T *warp_tot, T *total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        T t = lane < nw ? warp_tot[lane] : T(0);
        T ti = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T u = __shfl_up_sync(0xffffffffu, ti, o);
            if (lane >= o) ti += u;
        }
        if (lane < nw) warp_tot[lane] = ti - t;
        if (lane == nw - 1) *total = ti;
    }
    __syncthreads();
    T r = warp_tot[warp] + incl - v;
    __syncthreads();
    return r;
}

template <class T>
__global__ void k_block_sums(const T *in, T *sums, long long n) {
    __shared__ T wt[32];
    __shared__ T tot;
    long long base = (long long)blockIdx.x * SCAN_TILE;
    T s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        long long i = base + (long long)k * SCAN_THREADS + threadIdx.x;
        if (i < n) s += in[i];
    }
    block_exclusive_scan<T>(s, wt, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

template <class T>
__global__ void k_block_scan(const T *in, T *out, long long n, const T *offsets, T *grand_total) {
    __shared__ T tile[SCAN_TILE];
    __shared__ T wt[32];
    __shared__ T tot;
    long long base = (long long)blockIdx.x * SCAN_TILE;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        long long i = base + (long long)k * SCAN_THREADS + threadIdx.x;
        tile[k * SCAN_THREADS + threadIdx.x] = i < n ? in[i] : T(0);
    }
    __syncthreads();
    T loc[SCAN_ITEMS];
    T s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        loc[k] = tile[threadIdx.x * SCAN_ITEMS + k];
        s += loc[k];
    }
    T ex = block_exclusive_scan<T>(s, wt, &tot);
    T off = offsets ? offsets[blockIdx.x] : T(0);
    T run = off + ex;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        tile[threadIdx.x * SCAN_ITEMS + k] = run;
        run += loc[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        long long i = base + (long long)k * SCAN_THREADS + threadIdx.x;
        if (i < n) out[i] = tile[k * SCAN_THREADS + threadIdx.x];
    }
    if (grand_total && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *grand_total = off + tot;
}

template <class T>
void scan_rec(const T *in, T *out, long long n, char *tmp, T *grand_total, cudaStream_t st) {
    if (n <= 0) {
        if (grand_total) SDOT_CUDA(cudaMemsetAsync(grand_total, 0, sizeof(T), st));
        return;
    }
    long long nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (nb == 1) {
        k_block_scan<T><<<1, SCAN_THREADS, 0, st>>>(in, out, n, nullptr, grand_total);
        note_launch();
        SDOT_CUDA(cudaGetLastError());
        return;
    }
    T *sums = reinterpret_cast<T *>(tmp);
    T *sums_scanned = sums + nb;
    char *next = reinterpret_cast<char *>(sums_scanned + nb);
    next = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(next) + 255) & ~uintptr_t(255));
    k_block_sums<T><<<unsigned(nb), SCAN_THREADS, 0, st>>>(in, sums, n);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
    scan_rec<T>(sums, sums_scanned, nb, next, nullptr, st);
    k_block_scan<T><<<unsigned(nb), SCAN_THREADS, 0, st>>>(in, out, n, sums_scanned, grand_total);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------- radix ----
constexpr int RADIX_THREADS = 256;
constexpr int RADIX_ROUNDS = 16;
constexpr int RADIX_TILE = RADIX_THREADS * RADIX_ROUNDS;

__global__ void k_radix_hist(const unsigned *keys, long long n, int shift, unsigned *ghist, int nb) {
    __shared__ unsigned h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    long long base = (long long)blockIdx.x * RADIX_TILE;
    for (int r = 0; r < RADIX_ROUNDS; ++r) {
        long long i = base + (long long)r * RADIX_THREADS + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    ghist[(long long)threadIdx.x * nb + blockIdx.x] = h[threadIdx.x];
}

__global__ void k_radix_scatter(const unsigned *keys_in, const unsigned *vals_in, unsigned *keys_out,
                                unsigned *vals_out, long long n, int shift, const unsigned *goff, int nb) {
    __shared__ unsigned run[256];
    __shared__ unsigned wcnt[RADIX_THREADS / 32][256];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    run[tid] = goff[(long long)tid * nb + blockIdx.x];
    const unsigned lt_mask = (1u << lane) - 1u;
    long long base = (long long)blockIdx.x * RADIX_TILE;
    for (int r = 0; r < RADIX_ROUNDS; ++r) {
        long long i = base + (long long)r * RADIX_THREADS + tid;
        bool valid = i < n;
        unsigned key = valid ? keys_in[i] : 0u;
        unsigned d = valid ? ((key >> shift) & 255u) : 256u;
#pragma unroll
        for (int w = 0; w < RADIX_THREADS / 32; ++w) wcnt[w][tid] = 0;
        __syncthreads();
        unsigned peers = __match_any_sync(0xffffffffu, d);
        unsigned rank = __popc(peers & lt_mask);
        if (valid && lane == __ffs(peers) - 1) wcnt[warp][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            unsigned off = run[d] + rank;
            for (int w = 0; w < warp; ++w) off += wcnt[w][d];
            keys_out[off] = key;
            vals_out[off] = vals_in[i];
        }
        __syncthreads();
        unsigned tot = 0;
#pragma unroll
        for (int w = 0; w < RADIX_THREADS / 32; ++w) tot += wcnt[w][tid];
        run[tid] += tot;
        __syncthreads();
    }
}

}  // namespace

size_t scan_tmp_size(long long n, size_t elem) {
    size_t s = 0;
    while (true) {
        long long nb = (n + SCAN_TILE - 1) / SCAN_TILE;
        if (nb <= 1) break;
        s += 2 * size_t(nb) * elem + 256;
        n = nb;
    }
    return s + 256;
}

template <class T>
void scan_exclusive(const T *in, T *out, long long n, void *tmp, cudaStream_t st) {
    scan_rec<T>(in, out, n, static_cast<char *>(tmp), nullptr, st);
}
template <class T>
void scan_exclusive_total(const T *in, T *out, long long n, void *tmp, cudaStream_t st) {
    scan_rec<T>(in, out, n, static_cast<char *>(tmp), out + n, st);
}

template void scan_exclusive<int>(const int *, int *, long long, void *, cudaStream_t);
template void scan_exclusive<unsigned>(const unsigned *, unsigned *, long long, void *, cudaStream_t);
template void scan_exclusive<long long>(const long long *, long long *, long long, void *, cudaStream_t);
template void scan_exclusive_total<int>(const int *, int *, long long, void *, cudaStream_t);
template void scan_exclusive_total<long long>(const long long *, long long *, long long, void *, cudaStream_t);

size_t radix_tmp_size(long long n) {
    long long nb = (n + RADIX_TILE - 1) / RADIX_TILE;
    if (nb < 1) nb = 1;
    size_t hist = size_t(256) * nb * sizeof(unsigned);
    return 2 * hist + scan_tmp_size(256 * nb, sizeof(unsigned)) + 512;
}

void radix_sort_pairs(const unsigned *keys_in, const unsigned *vals_in, unsigned *keys_out, unsigned *vals_out,
                      unsigned *keys_alt, unsigned *vals_alt, long long n, int bits, void *tmp, cudaStream_t st) {
    if (n <= 0) return;
    int nb = int((n + RADIX_TILE - 1) / RADIX_TILE);
    char *t = static_cast<char *>(tmp);
    unsigned *ghist = reinterpret_cast<unsigned *>(t);
    unsigned *goff = ghist + size_t(256) * nb;
    char *scan_tmp = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(goff + size_t(256) * nb) + 255) & ~uintptr_t(255));
    int passes = (bits + 7) / 8;
    if (passes < 1) passes = 1;
    // ping-pong so that the final pass lands in (keys_out, vals_out)
    const unsigned *src_k = keys_in, *src_v = vals_in;
    for (int p = 0; p < passes; ++p) {
        const bool to_out = ((passes - 1 - p) % 2) == 0;
        unsigned *dk = to_out ? keys_out : keys_alt;
        unsigned *dv = to_out ? vals_out : vals_alt;
        k_radix_hist<<<nb, RADIX_THREADS, 0, st>>>(src_k, n, 8 * p, ghist, nb);
        note_launch();
        SDOT_CUDA(cudaGetLastError());
        scan_exclusive<unsigned>(ghist, goff, 256LL * nb, scan_tmp, st);
        k_radix_scatter<<<nb, RADIX_THREADS, 0, st>>>(src_k, src_v, dk, dv, n, 8 * p, goff, nb);
        note_launch();
        SDOT_CUDA(cudaGetLastError());
        src_k = dk;
        src_v = dv;
    }
}

}  // namespace sdot
