// nb14 / nbex pair-list kernels used by the C ABI layer.
#pragma once
#include <cuda_runtime.h>

#include "bnb.h"
#include "bnb_internal.h"

namespace bnb {
struct PairsArgs {
  int N, R, lamTotal, n14, nex;
  float rCut, rSwitch, beta, kElectric, softR;
  const float *x;            // [3N] caller positions (State::position_fd)
  const float *lambda;       // [lamTotal] (State::lambda_fd)
  const int *atomRep;        // [N]
  const RepInfo *rep;        // [R] boxes
  const bnb_nb14 *nb14;      // [n14]
  const bnb_nbex *nbex;      // [nex]
  long long *accF;           // [3N] fixed-point dU/dx, atom order
  long long *accL;           // [lamTotal]
  long long *accE;           // [R]
  int mode;                  // BNB_OUT_SET / BNB_OUT_ADD64 bits of the call
};
int launch_nb14(const PairsArgs &a, const bnb_outputs &o, int elec, int vdw, bool soft, bool energy,
                cudaStream_t s);
int launch_nbex(const PairsArgs &a, const bnb_outputs &o, bool energy, cudaStream_t s);
}  // namespace bnb
