// Shared definitions for the sdot_b200 CUDA library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>

namespace sdot {

// Status codes of the C ABI (mirrored in include/sdot_gpu.h).
enum Status : int {
    ST_OK = 0,
    ST_VOID_CELL = 1,          // reference: for_each_laguerre_cell(stop_if_void) -> 1
    ST_CAPACITY = 2,           // a cell needed more vertices than the fallback capacity
    ST_NOT_CONVERGED = 3,
    ST_ITER_CAP = 4,
    ST_OOM = 5,
    ST_BAD_ARG = 6,
    ST_CUDA = 7,
    ST_UNSUPPORTED = 8,
};

// Cut identifiers stored with each polygon edge (edge k joins vertex k and k+1).
//  id >= 0            : the bisector with the Dirac at that SORTED position
//  id == ID_ARC       : an arc of the clipping disc
//  id <= ID_DOMAIN0   : edge (ID_DOMAIN0 - id) of the starting polygon (domain)
constexpr int ID_ARC = -2;
constexpr int ID_DOMAIN0 = -3;
__host__ __device__ inline int domain_id(int e) { return ID_DOMAIN0 - e; }
__host__ __device__ inline int domain_edge(int id) { return ID_DOMAIN0 - id; }
// Edges of the local square that starts an FP32 build (mixed path); a cell
// that keeps one is rebuilt in FP64, so these ids never reach an output.
constexpr int ID_LOCAL = -(1 << 30);

// Inside a piece (cell intersected with a domain item or a pixel):
//  id >= 0       : came from edge `id` of the cell polygon
//  id == PID_OWN : an edge of the item/pixel itself
//  id == ID_ARC  : an arc
constexpr int PID_OWN = -1;

struct CudaError {
    cudaError_t err;
    const char *where;
};

#define SDOT_STR2(x) #x
#define SDOT_STR(x) SDOT_STR2(x)
#define SDOT_CUDA(call)                                                                             \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) throw ::sdot::CudaError{e_, #call " (" __FILE__ ":" SDOT_STR(__LINE__) ")"}; \
    } while (0)

// Debug builds (-DSDOT_CHECKS) bounds-check buffer accesses in the kernels:
// a failing check records (code, line, value) of the first failure in a
// per-translation-unit device word and the access is redirected to index 0.
// Release builds compile the checks away.
#ifdef SDOT_CHECKS
static __device__ unsigned long long sdot_dbg_word[3];
__host__ __device__ inline void check_fail(int code, int line, long long value) {
#ifdef __CUDA_ARCH__
    if (atomicCAS(&sdot_dbg_word[0], 0ull, (unsigned long long)code) == 0ull) {
        sdot_dbg_word[1] = (unsigned long long)line;
        sdot_dbg_word[2] = (unsigned long long)value;
    }
#else
    printf("sdot check %d failed at line %d value %lld\n", code, line, value);
#endif
}
#define SDOT_CHECK_IDX(k, n, code) \
    (((k) < 0 || (k) >= (n)) ? (::sdot::check_fail(code, __LINE__, (long long)(k)), 0) : (k))
#else
#define SDOT_CHECK_IDX(k, n, code) (k)
#endif

inline int ceil_div(long long a, long long b) { return int((a + b - 1) / b); }

// Per-device state of a kernel launcher (shared-memory attributes, tuned block
// sizes): one slot per device ordinal, read and written under one mutex, so
// that contexts on several devices, or several threads, can launch at once.
constexpr int kDeviceSlots = 64;
template <class T>
struct PerDevice {
    std::mutex m;
    T slot[kDeviceSlots] = {};
    // the current device's slot index (throws on an ordinal beyond the table)
    static int device() {
        int d = 0;
        SDOT_CUDA(cudaGetDevice(&d));
        if (d < 0 || d >= kDeviceSlots) throw CudaError{cudaErrorInvalidDevice, "device ordinal beyond 64"};
        return d;
    }
    T get() {
        const int d = device();
        std::lock_guard<std::mutex> g(m);
        return slot[d];
    }
    void set(const T &v) {
        const int d = device();
        std::lock_guard<std::mutex> g(m);
        slot[d] = v;
    }
    // runs f() unless this device's slot is already set, then sets it (f runs
    // under the lock: concurrent first calls on one device wait for it)
    template <class F>
    void once(const F &f) {
        const int d = device();
        std::lock_guard<std::mutex> g(m);
        if (slot[d]) return;
        f();
        slot[d] = T(1);
    }
};

// Process-wide count of this library's kernel launches (sdot_kernel_launches).
void note_launch();
void note_launches(unsigned long long k);
// While one of these lives, the launches this thread notes are counted into
// it instead (a stream capture: they run, and are counted, when the graph
// is launched).
struct CaptureCount {
    unsigned long long n = 0;
    unsigned long long *prev;
    CaptureCount();
    ~CaptureCount();
    CaptureCount(const CaptureCount &) = delete;
    CaptureCount &operator=(const CaptureCount &) = delete;
};

// Per-cell kernel bodies are device functions; a host build of them (for
// CPU-side debugging of the kernels) is compiled with SDOT_HOST_KERNELS.
#ifdef SDOT_HOST_KERNELS
#define SDOT_KFN __host__ __device__
#else
#define SDOT_KFN __device__
#endif

// Sets bits of the sticky error word (atomically on the device).
__host__ __device__ inline void flag_error(unsigned *word, unsigned bits) {
#ifdef __CUDA_ARCH__
    atomicOr(word, bits);
#else
    *word |= bits;
#endif
}

// Sticky per-context error word written by kernels (never __trap).
enum DevErr : unsigned {
    DE_CAPACITY = 1u,      // cell polygon overflowed its capacity (re-run in the large path)
    DE_STACK = 2u,         // traversal stack overflow (should not happen: depth bounded)
    DE_ITER = 4u,          // an iteration cap was reached
    DE_PIECE = 8u,         // a piece overflowed its capacity
    DE_GUARD = 16u,        // an input failed a consistency guard (see the debug triple)
    DE_DEGEN = 32u,        // a 3D cut met degenerate geometry (a face cut twice, an open new face)
    DE_SIDE = 64u,         // a long row did not fit the side buffer (the host grows it and runs again)
};

}  // namespace sdot
