// Device Z-order tree over the Diracs: the B200 counterpart of the
// reference's SpZGrid (src/sdot/PowerDiagram/Visitors/SpZGrid.{h,tcc}).
//
// SpZGrid is a 2^d-tree built serially by recursive partition of an index
// array (SpZGrid.tcc:41-187); each box keeps the bounding box of its Diracs
// and their maximum weight (degree-0 weight approximation, :123-143), and
// boxes are split while they hold more than max_diracs_per_cell Diracs.
// Here the same tree is built in parallel: Morton keys of quantised
// positions are radix-sorted, so every tree node is a contiguous range of
// the sorted order; nodes are split top-down level by level (binary search
// for child ranges, single-child chains collapsed), then the tight bounding
// box and max weight of every node are reduced bottom-up.
#pragma once
#include "common.cuh"

namespace sdot {

template <int D>
struct alignas(16) TreeNode {
    double lo[D];
    double hi[D];
    double maxw;
    int a;  // leaf: first sorted index; internal: first child node
    int b;  // leaf: one past the last sorted index (> a); internal: -(number of children)
};

// Device state of the tree and of the Diracs in sorted (Morton) order.
template <int D>
struct DeviceTree {
    long long n = 0;
    long long cap_n = 0;      // allocated Dirac capacity
    int max_nodes = 0;
    int key_bits = 0;         // bits per axis
    int max_per_leaf = 11;    // SpZGrid default max_diracs_per_cell
    // sorted arrays
    double *pos = nullptr;    // D * n
    double *w = nullptr;      // n
    int *idx = nullptr;       // sorted -> original
    int *inv = nullptr;       // original -> sorted
    TreeNode<D> *nodes = nullptr;
    int *node_level = nullptr;
    int *counters = nullptr;  // [0] node count, [1 + p] start of pass p
    int npass = 0;
    // scratch
    unsigned *keys = nullptr, *keys2 = nullptr, *keys3 = nullptr;
    unsigned *vals = nullptr, *vals2 = nullptr, *vals3 = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    double *bbox = nullptr;   // 2 * D doubles (min, max) of the positions
    unsigned long long *bbox_bits = nullptr;

    // build() and update_weights() replay their launches from CUDA graphs,
    // captured on the first call for the same input buffers, size and leaf
    // size (about 80 and 20 small launches; direct launches where the stream
    // cannot be captured)
    cudaGraphExec_t build_graph = nullptr, weights_graph = nullptr;
    const void *bg_pos = nullptr, *bg_w = nullptr, *wg_w = nullptr;
    long long bg_n = -1, wg_n = -1;
    int bg_leaf = -1;
    unsigned long long bg_launches = 0, wg_launches = 0;

    void reserve(long long n);
    void release();
    void drop_graphs();
    void build_launches(const double *pos_orig, const double *w_orig, cudaStream_t st);
    void weights_launches(const double *w_orig, cudaStream_t st);
    // positions (D * n, AoS) and weights in original order, device pointers
    void build(const double *pos_orig, const double *w_orig, long long n, cudaStream_t st);
    // new weights (original order, device pointer): re-gather and refresh maxw
    void update_weights(const double *w_orig, cudaStream_t st);
    // refresh the node max weights from the sorted weights already in `w`
    void refresh_maxw(cudaStream_t st);
};

extern template struct DeviceTree<2>;
extern template struct DeviceTree<3>;

}  // namespace sdot
