// sdot_csr_solve_noalloc: the CSR conjugate-gradient solve of sdot_csr_solve
// without any device allocation (see include/sdot_gpu.h).
//
// Some callers cannot allocate device memory when they solve: a process whose
// free HBM is held by another allocator (a framework's caching allocator that
// reserves most of the device) would see cudaMalloc fail or fragment that
// pool, and a latency-bound loop (one small solve per request inside a serving
// step) cannot afford the device-wide synchronisation that cudaMalloc and
// cudaFree bring on every call.  This entry point works in a fixed scratch
// area compiled into the library instead, so it is limited to
// SDOT_NOALLOC_MAX_ROWS rows, and calls that overlap on one device share that
// scratch.
#include "../../include/sdot_gpu.h"
#include "solve.cuh"

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

namespace {

constexpr long long kMaxRows = SDOT_NOALLOC_MAX_ROWS;
constexpr int kMaxDevices = 64;

// Work vectors of one solve of up to kMaxRows rows (r, z, p, q, 1/diag, block
// partials, device scalars): 331,464 doubles, 2.65 MB per device.
constexpr size_t kScratchDoubles = 5 * (kMaxRows + 32) + 6 * sdot::PCG_BLOCKS + 8 + 64;
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_setup_mutex;
double *g_scratch_ptr[kMaxDevices] = {};

// Address of this device's copy of the scratch array, looked up once per
// device with that device current (the first call on each device).
int scratch_for_current_device(double **out, std::string &msg) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        msg = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
        return SDOT_CUDA_ERROR;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        msg = "device ordinal beyond the supported range";
        return SDOT_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            msg = std::string("cudaGetSymbolAddress of the scratch array: ") + cudaGetErrorString(e);
            return SDOT_CUDA_ERROR;
        }
        g_scratch_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_ptr[dev];
    return SDOT_OK;
}

}  // namespace

extern "C" int sdot_csr_solve_noalloc(const int64_t *offsets, const int64_t *columns, const double *values, int64_t n,
                                      const double *b, double *x, int gauge_fix, double rel_tol, int max_iter,
                                      void *stream, int64_t *iterations, double *rel_residual, char *errbuf,
                                      int64_t errbuf_len) {
    auto fail = [&](int code, const std::string &m) {
        if (errbuf && errbuf_len > 0) {
            const size_t k = std::min<size_t>(m.size(), size_t(errbuf_len - 1));
            std::memcpy(errbuf, m.data(), k);
            errbuf[k] = 0;
        }
        return code;
    };
    if (errbuf && errbuf_len > 0) errbuf[0] = 0;
    if (n > kMaxRows)
        return fail(SDOT_BAD_ARG, "sdot_csr_solve_noalloc: " + std::to_string(n) + " rows exceed the limit of " +
                                      std::to_string(kMaxRows) + " rows of the allocation-free solve");
    if (n < 0 || (n > 0 && (!offsets || !columns || !values || !b || !x)) || max_iter <= 0 || !(rel_tol > 0))
        return fail(SDOT_BAD_ARG, "sdot_csr_solve_noalloc: bad arguments");
    if (n == 0) return SDOT_OK;
    double *scratch = nullptr;
    std::string msg;
    const int st0 = scratch_for_current_device(&scratch, msg);
    if (st0 != SDOT_OK) return fail(st0, "sdot_csr_solve_noalloc: " + msg);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    try {
        sdot::PcgWork w;
        sdot::pcg_bind(w, scratch, n);
        // the device scalars must start at zero; every other work vector is
        // written before it is read
        SDOT_CUDA(cudaMemsetAsync(w.scal, 0, 8 * sizeof(double), st));
        const sdot::PcgResult r =
            sdot::pcg_solve_csr(sdot::CsrMat{reinterpret_cast<const long long *>(offsets),
                                             reinterpret_cast<const long long *>(columns), values},
                                n, gauge_fix ? 0 : -1, b, x, rel_tol, max_iter, w, st);
        SDOT_CUDA(cudaStreamSynchronize(st));
        if (iterations) *iterations = r.iterations;
        if (rel_residual) *rel_residual = r.rel_residual;
        return r.converged ? int(SDOT_OK)
                           : fail(SDOT_NOT_CONVERGED, "sdot_csr_solve_noalloc: conjugate gradients did not reach the "
                                                      "tolerance");
    } catch (const sdot::CudaError &e) {
        return fail(SDOT_CUDA_ERROR, std::string(cudaGetErrorString(e.err)) + " in " + e.where);
    }
}
