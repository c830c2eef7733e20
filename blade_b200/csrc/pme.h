// PME reciprocal space and Ewald self term used by the C ABI layer.
#pragma once
#include <cuda_runtime.h>

#include "bnb.h"
#include "bnb_internal.h"

namespace bnb {

struct PmeRep {            // per replica: grid sizes and offsets into the concatenated grids
  int K[3];
  int gridOff;             // real grid [K0][K1][K2]
  int cplxOff;             // half spectrum [K0][K1][K2/2+1]
  int modOff;              // moduli: K0 + K1 + (K2/2+1) values
  int pad[2];
};

struct PmeArgs {
  int N, R, lamTotal, order;
  int totalGrid, totalCplx, maxCplx;  // maxCplx: largest half spectrum of one replica
  float beta;
  const float *x;          // [3N] caller positions (State::position_fd)
  const float *lambda;     // [lamTotal] or null (every scale 1)
  const float *q;          // [N] charge * sqrt(kElectric)
  const int *siteBlock;    // [N] (site<<16)|block
  const int *atomRep;      // [N]
  const RepInfo *rep;      // [R] boxes
  const PmeRep *prep;      // [R]
  const float *mod;        // moduli 1/|b(m)|^2, per replica and dimension
  long long *qfix;         // [totalGrid] fixed-point charge grid (zero between calls)
  float *grid;             // [totalGrid] charge grid, then (after C2R) the potential grid
  float2 *cplx;            // [totalCplx] spectrum
  long long *accL;         // [lamTotal]
  long long *accE;         // [R]
  unsigned int *done;      // CTAs finished in the current gather / self launch (zero between launches)
  int mode;                // BNB_OUT_SET / BNB_OUT_ADD64 bits of the call
  int tric;                // boxes are triclinic cells (RepInfo::box and ::tric)
};

// Spread lambda-scaled charges into qfix and convert to the FP32 grid
// (clearing qfix); two launches.
int pme_spread(const PmeArgs &a, cudaStream_t s);
// Multiply the spectrum by the influence function; one launch.
int pme_convolve(const PmeArgs &a, cudaStream_t s);
// Gather forces, dU/dlambda and energy from the potential grid; the last
// CTA writes the lambda and energy outputs; one launch.
int pme_gather(const PmeArgs &a, const bnb_outputs &o, bool energy, cudaStream_t s);
// Ewald self energy and its dU/dlambda; one launch.
int pme_self(const PmeArgs &a, const bnb_outputs &o, bool energy, cudaStream_t s);

}  // namespace bnb
