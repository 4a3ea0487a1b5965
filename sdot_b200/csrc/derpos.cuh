// Derivatives of the cell centroids and masses with respect to the weights
// and positions (2D), from the cells of the neighbour pass (see derpos.cu).
#pragma once
#include "cell2d.cuh"
#include "common.cuh"

namespace sdot {

// Per Dirac (caller order) the number of 3 x 3 blocks of its rows; flags
// DE_CAPACITY in *err for a cell of more than 64 vertices.
void derpos_count(const Rows &nb, long long n, const double *pos, const double *w, const int *idx, int start_n,
                  const double *start_xy, double coeff, int ntrans, const double *trans, long long *nblocks,
                  unsigned *err, cudaStream_t st);
// The CSR of 3 n rows (offsets[3 n + 1], columns and values of 9 * total
// blocks entries) and v[3 n] = (centroid x, centroid y, mass) per Dirac;
// boff: exclusive scan of the block counts (n + 1 entries, caller order).
void derpos_write(const Rows &nb, long long n, const double *pos, const double *w, const int *idx, int start_n,
                  const double *start_xy, double coeff, int ntrans, const double *trans, const long long *boff,
                  long long *off, long long *cols, double *vals, double *v, cudaStream_t st);

}  // namespace sdot
