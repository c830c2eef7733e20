// Pair-kernel entry points used by the C ABI layer.
#pragma once
#include <cuda_runtime.h>

#include "bnb_internal.h"

namespace bnb {
// alch: 0 none, 1 MSLD scaling, 2 MSLD + soft core.
int launch_pair(const Dev &d, const PairConst &pc, const float *lambda, int elec, int vdw,
                int alch, bool energy, bool count, int grid, cudaStream_t s);
void launch_finalize(const Dev &d, const bnb_outputs &o, int mode, cudaStream_t s);
// Sorts the work items by the cycles the last pair launch measured for them,
// longest first, into Dev::order, which the following launches follow until
// the next rebuild; one launch.
void launch_order(const Dev &d, cudaStream_t s);

// All-pairs evaluation of one small system (bnb_nbdirect_noalloc).  accF is
// [3 * stride] (component planes), accE one entry; both must be zero on
// entry and are zero again once the launched kernels complete.
struct AllPairsArgs {
  PairConst pc;
  int N, nTypes, stride;
  float sqrtK;
  float3 box, boxInv;
  const float *x;            // [3N]
  const bnb_nbond *nb;       // [N]
  const bnb_vdw *vdw;        // [nTypes * nTypes]
  const int *exclStart;      // [N+1]
  const int *exclAtom;       // sorted within each row
  long long *accF, *accE;
};
int launch_allpairs(const AllPairsArgs &a, const bnb_outputs &o, int elec, int vdw, bool energy,
                    cudaStream_t s);
}  // namespace bnb
