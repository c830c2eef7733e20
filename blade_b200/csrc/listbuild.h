// List-builder entry points used by the C ABI layer.
#pragma once
#include <cuda_runtime.h>

#include "bnb_internal.h"

namespace bnb {
// Exclusive scan of n ints into out[0..n); the total goes to *total.
// Returns the number of kernels launched (1 up to 16,384 items, else 3).
int scan_exclusive(const int *in, int *out, int n, int *total, int *partial, cudaStream_t s);
// Full list rebuild (bin, sort, blocks, AABBs, cull at sqrt(rcull2), masks, work items).
// Returns the number of kernels launched.
int rebuild_list(const Dev &d, const int *colRep, const float *pos, float rcull2, cudaStream_t s);
// Per-step packing of coordinates into block slots plus AABBs.
void pack_positions(const Dev &d, const float *pos, cudaStream_t s);
}  // namespace bnb
