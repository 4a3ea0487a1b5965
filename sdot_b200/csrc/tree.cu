// Device Z-order tree (see tree.cuh).
#include "prims.cuh"
#include "tree.cuh"

namespace sdot {

namespace {

constexpr int TB = 256;

__device__ __forceinline__ unsigned long long ord_bits(double v) {
    unsigned long long b = __double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double from_ord_bits(unsigned long long b) {
    return __longlong_as_double((b >> 63) ? (b & 0x7fffffffffffffffull) : ~b);
}

template <int D>
__global__ void k_bbox_init(unsigned long long *bits) {
    int t = threadIdx.x;
    if (t < D) {
        bits[t] = ~0ull;
        bits[D + t] = 0ull;
    }
}

template <int D>
__global__ void k_bbox(const double *pos, long long n, unsigned long long *bits) {
    __shared__ unsigned long long smin[D], smax[D];
    if (threadIdx.x < D) {
        smin[threadIdx.x] = ~0ull;
        smax[threadIdx.x] = 0ull;
    }
    __syncthreads();
    unsigned long long lmin[D], lmax[D];
    for (int d = 0; d < D; ++d) { lmin[d] = ~0ull; lmax[d] = 0ull; }
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        for (int d = 0; d < D; ++d) {
            unsigned long long o = ord_bits(pos[D * i + d]);
            lmin[d] = o < lmin[d] ? o : lmin[d];
            lmax[d] = o > lmax[d] ? o : lmax[d];
        }
    }
    for (int d = 0; d < D; ++d) {
        atomicMin(&smin[d], lmin[d]);
        atomicMax(&smax[d], lmax[d]);
    }
    __syncthreads();
    if (threadIdx.x < D) {
        atomicMin(&bits[threadIdx.x], smin[threadIdx.x]);
        atomicMax(&bits[D + threadIdx.x], smax[threadIdx.x]);
    }
}

template <int D>
__global__ void k_bbox_final(const unsigned long long *bits, double *bbox) {
    int t = threadIdx.x;
    if (t < 2 * D) bbox[t] = from_ord_bits(bits[t]);
}

__device__ __forceinline__ unsigned spread2(unsigned v) {  // 16 bits -> even bits
    v &= 0xffffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}
__device__ __forceinline__ unsigned spread3(unsigned v) {  // 10 bits -> every third bit
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

template <int D>
__global__ void k_morton(const double *pos, long long n, const double *bbox, int bits, unsigned *keys, unsigned *vals) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double top = double((1u << bits) - 1u);
    unsigned q[D];
    for (int d = 0; d < D; ++d) {
        double lo = bbox[d], hi = bbox[D + d];
        double ext = hi - lo;
        double t = ext > 0 ? (pos[D * i + d] - lo) / ext * double(1u << bits) : 0.0;
        t = fmin(fmax(t, 0.0), top);
        q[d] = unsigned(t);
    }
    unsigned k;
    if (D == 2)
        k = spread2(q[0]) | (spread2(q[1]) << 1);
    else
        k = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2 % D]) << 2);
    keys[i] = k;
    vals[i] = unsigned(i);
}

template <int D>
__global__ void k_gather(const double *pos, const double *w, const unsigned *order, long long n, double *pos_s,
                         double *w_s, int *idx, int *inv) {
    long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s >= n) return;
    unsigned i = order[s];
    for (int d = 0; d < D; ++d) pos_s[D * s + d] = pos[D * (long long)i + d];
    w_s[s] = w[i];
    idx[s] = int(i);
    inv[i] = int(s);
}

template <int D>
__global__ void k_gather_w(const double *w, const int *idx, long long n, double *w_s) {
    long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s >= n) return;
    w_s[s] = w[idx[s]];
}

template <int D>
__global__ void k_tree_init(TreeNode<D> *nodes, int *level, int *counters, int npass, long long n) {
    nodes[0].a = 0;
    nodes[0].b = int(n);
    level[0] = 0;
    counters[0] = 1;
    counters[1] = 0;
    counters[2] = 1;
    for (int p = 3; p < npass + 3; ++p) counters[p] = 1;
}

// First index of [lo, hi) whose key is >= v, found by the 32 lanes of a warp
// together (every lane gets it): each round probes 32 evenly spaced keys and
// keeps the stretch between the last one below v and the next, so a range of
// r keys takes about log32(r) dependent reads instead of log2(r).
__device__ __forceinline__ int warp_lower_bound(const unsigned *keys, int lo, int hi, unsigned long long v) {
    const int lane = threadIdx.x & 31;
    while (hi - lo > 32) {
        const int step = (hi - lo + 31) / 32;
        const int i = lo + lane * step;
        const bool below = i < hi && (unsigned long long)keys[i] < v;
        const int cnt = __popc(__ballot_sync(0xffffffffu, below));  // probes 0 .. cnt - 1 are below v
        if (cnt == 0) return lo;
        const int nlo = lo + (cnt - 1) * step + 1;
        const int nhi = lo + cnt * step;
        lo = nlo;
        if (nhi < hi) hi = nhi;
    }
    const int i = lo + lane;
    const bool below = i < hi && (unsigned long long)keys[i] < v;
    return lo + __popc(__ballot_sync(0xffffffffu, below));
}

// One level of the top-down split, one warp per node of the level: the node's
// key range is cut at the 2^D child prefixes of its next Morton level (single-
// child levels skipped); children are appended at the node counter.
template <int D>
__global__ void k_split(TreeNode<D> *nodes, int *level, int *counters, int pass, const unsigned *keys, int bits,
                        int max_per_leaf, int max_nodes) {
    const int beg = counters[1 + pass], end = counters[2 + pass];
    constexpr int C = 1 << D;
    const int lane = threadIdx.x & 31;
    const int warp = int((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    const int nwarps = int((gridDim.x * (long long)blockDim.x) >> 5);
    for (int node = beg + warp; node < end; node += nwarps) {
        int a = nodes[node].a, b = nodes[node].b, L = level[node];
        while (true) {
            if (b - a <= max_per_leaf || L >= bits) break;  // leaf
            int shift = D * (bits - L - 1);
            unsigned long long prefix = (unsigned long long)keys[a] >> (shift + D);
            int st[C + 1];
            st[0] = a;
            st[C] = b;
            for (int c = 1; c < C; ++c)
                st[c] = warp_lower_bound(keys, st[c - 1], b, ((prefix << D) | (unsigned long long)c) << shift);
            int ne = 0;
            for (int c = 0; c < C; ++c) ne += st[c + 1] > st[c];
            if (ne == 1) {
                ++L;
                continue;
            }
            int first = 0;
            if (lane == 0) first = atomicAdd(&counters[0], ne);
            first = __shfl_sync(0xffffffffu, first, 0);
            if (first + ne > max_nodes) break;  // cannot happen: nodes <= 2n
            if (lane == 0) {
                int k = 0;
                for (int c = 0; c < C; ++c) {
                    if (st[c + 1] > st[c]) {
                        nodes[first + k].a = st[c];
                        nodes[first + k].b = st[c + 1];
                        level[first + k] = L + 1;
                        ++k;
                    }
                }
                nodes[node].a = first;
                nodes[node].b = -ne;
            }
            break;
        }
        if (lane == 0) level[node] = L;
    }
}

__global__ void k_mark_pass(int *counters, int pass) { counters[3 + pass] = counters[0]; }

template <int D>
__global__ void k_reduce(TreeNode<D> *nodes, const int *counters, int pass, const double *pos, const double *w,
                         bool bbox_too) {
    const int beg = counters[1 + pass], end = counters[2 + pass];
    for (int node = beg + blockIdx.x * blockDim.x + threadIdx.x; node < end; node += gridDim.x * blockDim.x) {
        TreeNode<D> nd = nodes[node];
        double lo[D], hi[D], mw = -1.0 / 0.0;
        for (int d = 0; d < D; ++d) { lo[d] = 1.0 / 0.0; hi[d] = -1.0 / 0.0; }
        if (nd.b > 0) {
            for (int s = nd.a; s < nd.b; ++s) {
                mw = fmax(mw, w[s]);
                if (bbox_too)
                    for (int d = 0; d < D; ++d) {
                        double v = pos[D * (long long)s + d];
                        lo[d] = fmin(lo[d], v);
                        hi[d] = fmax(hi[d], v);
                    }
            }
        } else {
            for (int c = nd.a; c < nd.a - nd.b; ++c) {
                const TreeNode<D> &ch = nodes[c];
                mw = fmax(mw, ch.maxw);
                if (bbox_too)
                    for (int d = 0; d < D; ++d) {
                        lo[d] = fmin(lo[d], ch.lo[d]);
                        hi[d] = fmax(hi[d], ch.hi[d]);
                    }
            }
        }
        nodes[node].maxw = mw;
        if (bbox_too)
            for (int d = 0; d < D; ++d) {
                nodes[node].lo[d] = lo[d];
                nodes[node].hi[d] = hi[d];
            }
    }
}

template <class T>
void dev_alloc(T *&p, size_t count) {
    SDOT_CUDA(cudaMalloc(reinterpret_cast<void **>(&p), count * sizeof(T) + 16));
}
template <class T>
void dev_free(T *&p) {
    if (p) cudaFree(p);
    p = nullptr;
}

int grid_for(long long n, int tb) {
    long long g = (n + tb - 1) / tb;
    if (g < 1) g = 1;
    if (g > 148 * 16) g = 148 * 16;
    return int(g);
}

// Captures the launches `f` makes on `st` into an executable graph; false
// (nothing launched, nothing captured) where the stream cannot be captured:
// the legacy default stream, or a stream already being captured.
template <class F>
bool capture(cudaStream_t st, cudaGraphExec_t &exec, unsigned long long &launches, F &&f) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return false;
    }
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    cudaGraph_t g = nullptr;
    unsigned long long counted = 0;
    {
        CaptureCount cc;
        try {
            f();
        } catch (...) {
            cudaStreamEndCapture(st, &g);
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            throw;
        }
        counted = cc.n;
    }
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (e == cudaSuccess && g) e = cudaGraphInstantiate(&exec, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        cudaGetLastError();
        exec = nullptr;
        return false;
    }
    launches = counted;
    return true;
}

}  // namespace

template <int D>
void DeviceTree<D>::reserve(long long nn) {
    if (nn <= cap_n && pos) return;
    release();
    cap_n = nn < 1 ? 1 : nn;
    key_bits = D == 2 ? 16 : 10;
    npass = key_bits + 1;
    max_nodes = int(2 * cap_n + 2);
    dev_alloc(pos, size_t(D) * cap_n);
    dev_alloc(w, cap_n);
    dev_alloc(idx, cap_n);
    dev_alloc(inv, cap_n);
    dev_alloc(nodes, max_nodes);
    dev_alloc(node_level, max_nodes);
    dev_alloc(counters, npass + 4);
    dev_alloc(keys, cap_n);
    dev_alloc(keys2, cap_n);
    dev_alloc(keys3, cap_n);
    dev_alloc(vals, cap_n);
    dev_alloc(vals2, cap_n);
    dev_alloc(vals3, cap_n);
    tmp_bytes = radix_tmp_size(cap_n);
    SDOT_CUDA(cudaMalloc(&tmp, tmp_bytes));
    dev_alloc(bbox, 2 * D);
    dev_alloc(bbox_bits, 2 * D);
}

template <int D>
void DeviceTree<D>::drop_graphs() {
    if (build_graph) cudaGraphExecDestroy(build_graph);
    if (weights_graph) cudaGraphExecDestroy(weights_graph);
    build_graph = weights_graph = nullptr;
    bg_n = wg_n = -1;
}

template <int D>
void DeviceTree<D>::release() {
    drop_graphs();
    dev_free(pos); dev_free(w); dev_free(idx); dev_free(inv);
    dev_free(nodes); dev_free(node_level); dev_free(counters);
    dev_free(keys); dev_free(keys2); dev_free(keys3);
    dev_free(vals); dev_free(vals2); dev_free(vals3);
    if (tmp) cudaFree(tmp);
    tmp = nullptr;
    dev_free(bbox); dev_free(bbox_bits);
    cap_n = 0;
}

template <int D>
void DeviceTree<D>::build(const double *pos_orig, const double *w_orig, long long nn, cudaStream_t st) {
    reserve(nn);
    n = nn;
    if (n == 0) return;
    if (!(build_graph && bg_n == n && bg_pos == pos_orig && bg_w == w_orig && bg_leaf == max_per_leaf)) {
        if (build_graph) cudaGraphExecDestroy(build_graph);
        build_graph = nullptr;
        bg_n = -1;
        if (!capture(st, build_graph, bg_launches, [&] { build_launches(pos_orig, w_orig, st); })) {
            build_launches(pos_orig, w_orig, st);
            return;
        }
        bg_n = n;
        bg_pos = pos_orig;
        bg_w = w_orig;
        bg_leaf = max_per_leaf;
    }
    SDOT_CUDA(cudaGraphLaunch(build_graph, st));
    note_launches(bg_launches);
}

template <int D>
void DeviceTree<D>::build_launches(const double *pos_orig, const double *w_orig, cudaStream_t st) {
    k_bbox_init<D><<<1, 32, 0, st>>>(bbox_bits);
    note_launch();
    k_bbox<D><<<grid_for(n, TB), TB, 0, st>>>(pos_orig, n, bbox_bits);
    note_launch();
    k_bbox_final<D><<<1, 32, 0, st>>>(bbox_bits, bbox);
    note_launch();
    k_morton<D><<<ceil_div(n, TB), TB, 0, st>>>(pos_orig, n, bbox, key_bits, keys, vals);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
    radix_sort_pairs(keys, vals, keys2, vals2, keys3, vals3, n, D * key_bits, tmp, st);
    k_gather<D><<<ceil_div(n, TB), TB, 0, st>>>(pos_orig, w_orig, vals2, n, pos, w, idx, inv);
    note_launch();
    k_tree_init<D><<<1, 1, 0, st>>>(nodes, node_level, counters, npass, n);
    note_launch();
    const int g = grid_for(n / 2 + 1, TB);
    for (int p = 0; p < npass; ++p) {
        k_split<D><<<g, TB, 0, st>>>(nodes, node_level, counters, p, keys2, key_bits, max_per_leaf, max_nodes);
        note_launch();
        k_mark_pass<<<1, 1, 0, st>>>(counters, p);
        note_launch();
    }
    for (int p = npass - 1; p >= 0; --p) {
        k_reduce<D><<<g, TB, 0, st>>>(nodes, counters, p, pos, w, true);
        note_launch();
    }
    SDOT_CUDA(cudaGetLastError());
}

template <int D>
void DeviceTree<D>::update_weights(const double *w_orig, cudaStream_t st) {
    if (n == 0) return;
    if (!(weights_graph && wg_n == n && wg_w == w_orig)) {
        if (weights_graph) cudaGraphExecDestroy(weights_graph);
        weights_graph = nullptr;
        wg_n = -1;
        if (!capture(st, weights_graph, wg_launches, [&] { weights_launches(w_orig, st); })) {
            weights_launches(w_orig, st);
            return;
        }
        wg_n = n;
        wg_w = w_orig;
    }
    SDOT_CUDA(cudaGraphLaunch(weights_graph, st));
    note_launches(wg_launches);
}

template <int D>
void DeviceTree<D>::weights_launches(const double *w_orig, cudaStream_t st) {
    k_gather_w<D><<<ceil_div(n, TB), TB, 0, st>>>(w_orig, idx, n, w);
    note_launch();
    refresh_maxw(st);
}

template <int D>
void DeviceTree<D>::refresh_maxw(cudaStream_t st) {
    if (n == 0) return;
    const int g = grid_for(n / 2 + 1, TB);
    for (int p = npass - 1; p >= 0; --p) {
        k_reduce<D><<<g, TB, 0, st>>>(nodes, counters, p, pos, w, false);
        note_launch();
    }
    SDOT_CUDA(cudaGetLastError());
}

template struct DeviceTree<2>;
template struct DeviceTree<3>;

}  // namespace sdot
