// Pair-kernel entry points used by the C ABI layer.
#pragma once
#include <cuda_runtime.h>

#include "bnb_internal.h"

namespace bnb {
// alch: 0 none, 1 MSLD scaling, 2 MSLD + soft core.
int launch_pair(const Dev &d, const PairConst &pc, const float *lambda, int elec, int vdw,
                int alch, bool energy, bool count, int grid, cudaStream_t s);
void launch_finalize(const Dev &d, const bnb_outputs &o, cudaStream_t s);
}  // namespace bnb
