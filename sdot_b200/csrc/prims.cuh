// Device-wide primitives written for this library: exclusive scan and a
// stable LSD radix sort of (uint32 key, uint32 value) pairs.
#pragma once
#include "common.cuh"

namespace sdot {

// ---------------------------------------------------------------- scan ----
// Exclusive prefix sum over `n` items of type T (int, long long, unsigned).
// Three passes: per-block totals, scan of totals (recursive), block scans.
// `tmp` must hold scan_tmp_size<T>(n) bytes.
size_t scan_tmp_size(long long n, size_t elem);
template <class T>
void scan_exclusive(const T *in, T *out, long long n, void *tmp, cudaStream_t st);
// Same, with `out[n]` receiving the grand total (out must hold n + 1 items).
template <class T>
void scan_exclusive_total(const T *in, T *out, long long n, void *tmp, cudaStream_t st);

// ---------------------------------------------------------- radix sort ----
// Sorts keys ascending, carrying values, stable.  `bits` is the number of
// significant key bits (passes = ceil(bits / 8)).  Result ends in
// (keys_out, vals_out); the *_alt buffers are scratch of n items each.
size_t radix_tmp_size(long long n);
void radix_sort_pairs(const unsigned *keys_in, const unsigned *vals_in, unsigned *keys_out, unsigned *vals_out,
                      unsigned *keys_alt, unsigned *vals_alt, long long n, int bits, void *tmp, cudaStream_t st);

}  // namespace sdot
