// Comparison harness around the reference's own CUDA direct-space path.
//
// TEST AND MEASUREMENT INFRASTRUCTURE ONLY.  This file is compiled together
// with the reference's unmodified sources src/nbdirect/nbdirect.cu and
// src/domdec/*.cu (see Makefile in this directory) into
// oracle/_ref/libbladeref.so.  It builds the handful of System fields that
// path reads -- State buffers in the [lambda | x | theta] layout
// (src/system/state.cxx), the Potential nonbonded tables and the vdW texture
// (src/system/potential.cxx:1336-1420), the Run cutoffs/methods/streams and
// the Msld block count -- and provides the few out-of-path functions the
// path calls (printlog/fatal from src/io, calc_virtual_position from
// src/holonomic, State::broadcast_position/broadcast_box from src/system).
// Each step it calls Domdec::update_domdec and getforce_nbdirect exactly as
// Run::dynamics and Potential::calc_force do (src/run/run.cu:554-564,
// src/system/potential.cxx:1839-1929), on one stream; ref_evaluate_pairs
// calls getforce_nb14 / getforce_nbex (src/bonded/pair.cu) the same way, and
// ref_evaluate_pme getforce_ewald / getforce_ewaldself (src/nbrecip/nbrecip.cu)
// on PME grids set up as Potential::initialize does (potential.cxx:1202-1300),
// and ref_holonomic holonomic_position / holonomic_velocity
// (src/holonomic/holonomic.cu) on given constraint clusters.  The MSLD entry
// points call Msld::calc_lambda_from_theta, calc_thetaForce_from_lambdaForce
// and getforce_fixedBias / getforce_variableBias (src/msld/msld.cu:863-1153),
// and ref_update_step one State::update (src/update/update.cu:233-305).
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <string>

#include "bonded/pair.h"
#include "domdec/domdec.h"
#include "main/defines.h"
#include "msld/msld.h"
#include "nbdirect/nbdirect.h"
#include "nbrecip/nbrecip.h"
#include "holonomic/holonomic.h"
#include "run/run.h"
#include "system/potential.h"
#include "system/selections.h"
#include "system/state.h"
#include "system/system.h"

// ---- out-of-path functions the path calls ---------------------------------
void printlog(const char *format, ...) { (void)format; }

void fatal(const char *fnm, int i, const char *format, ...) {
  va_list args;
  va_start(args, format);
  fprintf(stderr, "reference fatal at %s:%d: ", fnm, i);
  vfprintf(stderr, format, args);
  va_end(args);
  abort();
}

void calc_virtual_position(System *, bool) {}  // no virtual sites in these systems

__global__ void harness_set_fd(int n, float *pf, const double *pd) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) pf[i] = (float)pd[i];
}

// Single GPU: broadcast_position reduces to State::set_fd
// (src/system/state.cxx:411-442, src/update/update.cu:308-330).
void State::broadcast_position(System *system) {
  int n = 3 * atomCount + 2 * lambdaCount;
  harness_set_fd<<<(n + 255) / 256, 256, 0, system->run->updateStream>>>(n, positionBuffer_fd,
                                                                         positionBuffer_d);
}

void State::broadcast_box(System *) {}  // the harness sets orthBox and orthBox_f itself

// ---- harness ---------------------------------------------------------------
struct ref_handle {
  System *sys;
  State *st;
  Run *run;
  Potential *pot;
  Msld *msld;
  void *message[1];
  cudaStream_t stream;
  cudaEvent_t e0, e1;
  int N, nL;
  bool initialized;
};

template <typename T>
static T *raw_object() {
  void *p = calloc(1, sizeof(T));  // fields the path does not read stay zero
  return static_cast<T *>(p);
}

extern "C" int ref_create(int N, const int *siteBlock, const float *q, const int *typeIdx,
                          int nTypes, const float *vdw, int exclCount, const int *excl,
                          int nLambda, int useSoftCore, float rCut, float rSwitch, float beta,
                          int elecMethod, int vdwMethod, float cullPad, const double *box,
                          ref_handle **out) {
  ref_handle *h = new ref_handle();
  h->N = N;
  h->nL = nLambda < 1 ? 1 : nLambda;
  if (cudaStreamCreate(&h->stream) != cudaSuccess) return 2;
  cudaEventCreate(&h->e0);
  cudaEventCreate(&h->e1);

  System *sys = raw_object<System>();
  State *st = raw_object<State>();
  Run *run = raw_object<Run>();
  Potential *pot = raw_object<Potential>();
  Msld *msld = raw_object<Msld>();
  h->sys = sys; h->st = st; h->run = run; h->pot = pot; h->msld = msld;
  sys->id = 0;
  sys->idCount = 1;
  sys->verbose = 0;
  sys->message = h->message;
  sys->state = st;
  sys->run = run;
  sys->potential = pot;
  sys->msld = msld;

  // Run: cutoffs, methods, one stream for every role (serial execution)
  new (&run->calcTermFlag) std::map<int, bool>();
  run->calcTermFlag[eenbdirect] = true;
  run->cutoffs.betaEwald = beta;
  run->cutoffs.rCut = rCut;
  run->cutoffs.rSwitch = rSwitch;
  run->betaEwald = beta;
  run->rCut = rCut;
  run->rSwitch = rSwitch;
  run->elecMethod = (EElec)elecMethod;
  run->vdwMethod = (EVdw)vdwMethod;
  run->updateStream = run->bondedStream = run->biaspotStream = run->nbdirectStream =
      run->nbrecipStream = run->mlpotStream = h->stream;
  // Domdec::initialize sets cullPad = 2*sqrt(30 kB T)*freqDomdec*dt
  // (src/domdec/domdec.cu:138); pick dt so that the pad equals cullPad.
  run->T = 300;
  run->dt = cullPad / (2 * std::sqrt(30 * kB * run->T) * 10);

  // Msld
  msld->blockCount = h->nL;
  msld->useSoftCore = useSoftCore != 0;

  // State buffers in the [lambda | x | theta] layout
  st->atomCount = N;
  st->lambdaCount = h->nL;
  int nbuf = 3 * N + 2 * h->nL;
  cudaMalloc(&st->positionBuffer_d, sizeof(double) * nbuf);
  cudaMalloc(&st->positionBuffer_fd, sizeof(float) * nbuf);
  cudaMalloc(&st->forceBuffer_d, sizeof(float) * nbuf);
  cudaMalloc(&st->energy_d, sizeof(double) * eeend);
  cudaMemset(st->positionBuffer_d, 0, sizeof(double) * nbuf);
  st->lambda_d = st->positionBuffer_d;
  st->position_d = (double(*)[3])(st->positionBuffer_d + h->nL);
  st->theta_d = st->positionBuffer_d + h->nL + 3 * N;
  st->lambda_fd = st->positionBuffer_fd;
  st->position_fd = (float(*)[3])(st->positionBuffer_fd + h->nL);
  st->theta_fd = st->positionBuffer_fd + h->nL + 3 * N;
  st->lambdaForce_d = st->forceBuffer_d;
  st->force_d = (float(*)[3])(st->forceBuffer_d + h->nL);
  st->thetaForce_d = st->forceBuffer_d + h->nL + 3 * N;
  st->typeBox = false;
  st->orthBox.x = box[0]; st->orthBox.y = box[1]; st->orthBox.z = box[2];
  st->orthBox_f.x = (float)box[0]; st->orthBox_f.y = (float)box[1]; st->orthBox_f.z = (float)box[2];
  {
    double one = 1.0;
    cudaMemcpy(st->lambda_d, &one, sizeof(double), cudaMemcpyHostToDevice);
  }

  // Potential: nonbonded tables (potential.cxx:1336-1420) and exclusions
  pot->atomCount = N;
  NbondPotential *nb = (NbondPotential *)malloc(sizeof(NbondPotential) * (N > 0 ? N : 1));
  for (int i = 0; i < N; i++) {
    nb[i].siteBlock = siteBlock[i];
    nb[i].q = q[i];
    nb[i].typeIdx = typeIdx[i];
  }
  cudaMalloc(&pot->nbonds_d, sizeof(NbondPotential) * (N > 0 ? N : 1));
  cudaMemcpy(pot->nbonds_d, nb, sizeof(NbondPotential) * N, cudaMemcpyHostToDevice);
  free(nb);
  pot->vdwParameterCount = nTypes;
  size_t vb = sizeof(VdwPotential) * nTypes * nTypes;
  cudaMalloc(&pot->vdwParameters_d, vb);
  cudaMemcpy(pot->vdwParameters_d, vdw, vb, cudaMemcpyHostToDevice);
  {
    cudaResourceDesc rd;
    memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeLinear;
    rd.res.linear.devPtr = pot->vdwParameters_d;
    rd.res.linear.desc = cudaCreateChannelDesc<float2>();
    rd.res.linear.sizeInBytes = vb;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.readMode = cudaReadModeElementType;
    if (cudaCreateTextureObject(&pot->vdwParameters_tex, &rd, &td, NULL) != cudaSuccess) return 2;
  }
  pot->exclCount = exclCount;
  cudaMalloc(&pot->excls_d, sizeof(ExclPotential) * (exclCount > 0 ? exclCount : 1));
  cudaMemcpy(pot->excls_d, excl, sizeof(int) * 2 * exclCount, cudaMemcpyHostToDevice);

  sys->domdec = new Domdec();
  *out = h;
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// Coordinates (host FP64, [N][3]) and lambda (host FP64 [nL]) into position_d / lambda_d.
extern "C" int ref_set_state(ref_handle *h, const double *xyz, const double *lambda) {
  State *st = h->st;
  if (xyz) cudaMemcpyAsync(st->position_d, xyz, sizeof(double) * 3 * h->N, cudaMemcpyHostToDevice, h->stream);
  if (lambda) cudaMemcpyAsync(st->lambda_d, lambda, sizeof(double) * h->nL, cudaMemcpyHostToDevice, h->stream);
  cudaStreamSynchronize(h->stream);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// Same from a device buffer of 3N doubles (timed trajectories).
extern "C" int ref_set_positions_device(ref_handle *h, const double *xyz_d) {
  cudaMemcpyAsync(h->st->position_d, xyz_d, sizeof(double) * 3 * h->N, cudaMemcpyDeviceToDevice,
                  h->stream);
  return 0;
}

// One step of the path: list maintenance then the force call, as the step
// loop does it.  reset: rebuild the list (every freqDomdec steps).
static void ref_step(ref_handle *h, int reset, int calcEnergy) {
  System *sys = h->sys;
  if (!h->initialized) {
    sys->domdec->initialize(sys);  // includes the first reset_domdec
    h->initialized = true;
  } else {
    sys->domdec->update_domdec(sys, reset != 0);
  }
  // Potential::reset_force (potential.cxx:1839-1849), nbdirect part
  cudaMemsetAsync(sys->state->forceBuffer_d, 0, sizeof(float) * (3 * h->N + 2 * h->nL), h->stream);
  cudaMemsetAsync(sys->domdec->localForce_d, 0, 32 * sys->domdec->maxBlocks * sizeof(float) * 3, h->stream);
  cudaMemsetAsync(sys->state->energy_d, 0, sizeof(double) * eeend, h->stream);
  getforce_nbdirect(sys, calcEnergy != 0);
}

extern "C" int ref_evaluate(ref_handle *h, int reset, int calcEnergy, double *grad, double *energy,
                            double *lambdaForce) {
  ref_step(h, reset, calcEnergy);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return 2;
  State *st = h->st;
  int n = 3 * h->N;
  float *tmp = (float *)malloc(sizeof(float) * (n + h->nL));
  cudaMemcpy(tmp, st->force_d, sizeof(float) * n, cudaMemcpyDeviceToHost);
  for (int i = 0; i < n; i++) grad[i] = tmp[i];
  if (lambdaForce) {
    cudaMemcpy(tmp, st->lambdaForce_d, sizeof(float) * h->nL, cudaMemcpyDeviceToHost);
    for (int i = 0; i < h->nL; i++) lambdaForce[i] = tmp[i];
  }
  free(tmp);
  if (energy) cudaMemcpy(energy, st->energy_d + eenbdirect, sizeof(double), cudaMemcpyDeviceToHost);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// Times `steps` steps over a device trajectory frames_d [steps][3N] (FP64),
// rebuilding every `rebuildEvery` steps and computing the energy every
// `energyEvery` steps (0: never); returns the summed device time of
// each step (events on the path's stream) in *ms.  flush_d (flushBytes) is
// overwritten between steps, outside the timed events, to evict L2.
extern "C" int ref_time(ref_handle *h, const double *frames_d, int steps, int rebuildEvery,
                        int energyEvery, void *flush_d, size_t flushBytes, double *ms) {
  double total = 0;
  for (int k = 0; k < steps; k++) {
    ref_set_positions_device(h, frames_d + (size_t)k * 3 * h->N);
    if (flush_d) cudaMemsetAsync(flush_d, k & 0xFF, flushBytes, h->stream);
    cudaEventRecord(h->e0, h->stream);
    ref_step(h, k % rebuildEvery == 0, energyEvery > 0 && k % energyEvery == 0);
    cudaEventRecord(h->e1, h->stream);
    cudaEventSynchronize(h->e1);
    float t = 0;
    cudaEventElapsedTime(&t, h->e0, h->e1);
    total += t;
  }
  *ms = total;
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

extern "C" int ref_list_info(ref_handle *h, int *blocks, int *maxPartners) {
  Domdec *d = h->sys->domdec;
  if (blocks) *blocks = d->blockCount ? d->blockCount[1] : 0;
  if (maxPartners) *maxPartners = d->maxPartnersPerBlock;
  return 0;
}

// nb14 / nbex lists (host arrays in the layouts of Nb14Potential /
// NbExPotential) into Potential, and Msld::useSoftCore14.
extern "C" int ref_set_pairs(ref_handle *h, int n14, const void *nb14, int nex, const void *nbex, int soft14) {
  Potential *pot = h->pot;
  pot->nb14Count = n14;
  pot->nbexCount = nex;
  cudaMalloc(&pot->nb14s_d, sizeof(Nb14Potential) * (n14 > 0 ? n14 : 1));
  cudaMalloc(&pot->nbexs_d, sizeof(NbExPotential) * (nex > 0 ? nex : 1));
  if (n14) cudaMemcpy(pot->nb14s_d, nb14, sizeof(Nb14Potential) * n14, cudaMemcpyHostToDevice);
  if (nex) cudaMemcpy(pot->nbexs_d, nbex, sizeof(NbExPotential) * nex, cudaMemcpyHostToDevice);
  h->msld->useSoftCore14 = soft14 != 0;
  h->run->calcTermFlag[eenb14] = true;
  h->run->calcTermFlag[eenbrecipexcl] = true;
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// One nb14 (which 0) or nbex (which 1) evaluation on the current state.
extern "C" int ref_evaluate_pairs(ref_handle *h, int which, int calcEnergy, double *grad, double *energy,
                                  double *lambdaForce) {
  System *sys = h->sys;
  State *st = h->st;
  st->broadcast_position(sys);
  cudaMemsetAsync(st->forceBuffer_d, 0, sizeof(float) * (3 * h->N + 2 * h->nL), h->stream);
  cudaMemsetAsync(st->energy_d, 0, sizeof(double) * eeend, h->stream);
  if (which == 0) getforce_nb14(sys, calcEnergy != 0);
  else getforce_nbex(sys, calcEnergy != 0);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return 2;
  int n = 3 * h->N;
  float *tmp = (float *)malloc(sizeof(float) * (n + h->nL));
  cudaMemcpy(tmp, st->force_d, sizeof(float) * n, cudaMemcpyDeviceToHost);
  for (int i = 0; i < n; i++) grad[i] = tmp[i];
  if (lambdaForce) {
    cudaMemcpy(tmp, st->lambdaForce_d, sizeof(float) * h->nL, cudaMemcpyDeviceToHost);
    for (int i = 0; i < h->nL; i++) lambdaForce[i] = tmp[i];
  }
  free(tmp);
  if (energy) cudaMemcpy(energy, st->energy_d + (which == 0 ? eenb14 : eenbrecipexcl), sizeof(double),
                         cudaMemcpyDeviceToHost);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}


// PME grids, B-spline moduli, cuFFT plans and per-atom charges/blocks as
// Potential::initialize / Msld set them up (potential.cxx:1202-1300), for the
// grid K[3] and interpolation order given.  q: raw charges [N]; block: the
// atom's lambda block (0 = environment) [N].
extern "C" int ref_set_pme(ref_handle *h, int order, const int *K, const float *q, const int *block) {
  System *sys = h->sys;
  Potential *pot = h->pot;
  Run *run = h->run;
  State *st = h->st;
  const int N = h->N;
  run->orderEwald = order;
  run->calcTermFlag[eenbrecip] = true;
  run->calcTermFlag[eenbrecipself] = true;
  st->kOrthBox_f.x = 1 / st->orthBox_f.x;
  st->kOrthBox_f.y = 1 / st->orthBox_f.y;
  st->kOrthBox_f.z = 1 / st->orthBox_f.z;
  for (int k = 0; k < 3; k++) pot->gridDimPME[k] = K[k];
  const size_t nr = (size_t)K[0] * K[1] * K[2], nc = (size_t)K[0] * K[1] * (K[2] / 2 + 1);
  cudaMalloc(&pot->charge_d, sizeof(float) * (N > 0 ? N : 1));
  cudaMemcpy(pot->charge_d, q, sizeof(float) * N, cudaMemcpyHostToDevice);
  cudaMalloc(&sys->msld->atomBlock_d, sizeof(int) * (N > 0 ? N : 1));
  cudaMemcpy(sys->msld->atomBlock_d, block, sizeof(int) * N, cudaMemcpyHostToDevice);
  cudaMalloc(&pot->chargeGridPME_d, sizeof(cufftReal) * nr);
  cudaMalloc(&pot->fourierGridPME_d, sizeof(cufftComplex) * nc);
  cudaMalloc(&pot->potentialGridPME_d, sizeof(cufftReal) * nr);
  {
    cudaResourceDesc rd;
    memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeLinear;
    rd.res.linear.devPtr = pot->potentialGridPME_d;
    rd.res.linear.desc = cudaCreateChannelDesc<float>();
    rd.res.linear.sizeInBytes = sizeof(float) * nr;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.readMode = cudaReadModeElementType;
    if (cudaCreateTextureObject(&pot->potentialGridPME_tex, &rd, &td, NULL) != cudaSuccess) return 2;
  }
  // 1/|b(m)|^2 per dimension from M_n at the integers, product over the half grid
  double M[12] = {0};
  M[1] = 1.0;
  for (int k = 3; k <= order; k++) {
    double nw[12] = {0};
    for (int l = 0; l <= k; l++) nw[l] = (l * M[l] + (k - l) * (l >= 1 ? M[l - 1] : 0.0)) / (k - 1);
    for (int l = 0; l < 12; l++) M[l] = nw[l];
  }
  float *inv[3];
  for (int d = 0; d < 3; d++) {
    inv[d] = (float *)malloc(sizeof(float) * K[d]);
    for (int m = 0; m < K[d]; m++) {
      double re = 0, im = 0;
      for (int l = 1; l < order; l++) {
        re += M[l] * cos(2 * M_PI * m * l / K[d]);
        im += M[l] * sin(2 * M_PI * m * l / K[d]);
      }
      inv[d][m] = (float)(1.0 / (re * re + im * im));
    }
  }
  float *bg = (float *)malloc(sizeof(float) * nc);
  for (int i = 0; i < K[0]; i++)
    for (int j = 0; j < K[1]; j++)
      for (int k = 0; k < K[2] / 2 + 1; k++)
        bg[((size_t)i * K[1] + j) * (K[2] / 2 + 1) + k] = inv[0][i] * inv[1][j] * inv[2][k];
  cudaMalloc(&pot->bGridPME_d, sizeof(float) * nc);
  cudaMemcpy(pot->bGridPME_d, bg, sizeof(float) * nc, cudaMemcpyHostToDevice);
  free(bg);
  for (int d = 0; d < 3; d++) free(inv[d]);
  if (cufftPlan3d(&pot->planFFTPME, K[0], K[1], K[2], CUFFT_R2C) != CUFFT_SUCCESS) return 2;
  if (cufftPlan3d(&pot->planIFFTPME, K[0], K[1], K[2], CUFFT_C2R) != CUFFT_SUCCESS) return 2;
  cufftSetStream(pot->planFFTPME, h->stream);
  cufftSetStream(pot->planIFFTPME, h->stream);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// One reciprocal (which 0) or self (which 1) evaluation on the current state.
extern "C" int ref_evaluate_pme(ref_handle *h, int which, int calcEnergy, double *grad, double *energy,
                                double *lambdaForce) {
  System *sys = h->sys;
  State *st = h->st;
  st->broadcast_position(sys);
  cudaMemsetAsync(st->forceBuffer_d, 0, sizeof(float) * (3 * h->N + 2 * h->nL), h->stream);
  cudaMemsetAsync(st->energy_d, 0, sizeof(double) * eeend, h->stream);
  if (which == 0) getforce_ewald(sys, calcEnergy != 0);
  else getforce_ewaldself(sys, calcEnergy != 0);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return 2;
  int n = 3 * h->N;
  float *tmp = (float *)malloc(sizeof(float) * (n + h->nL));
  cudaMemcpy(tmp, st->force_d, sizeof(float) * n, cudaMemcpyDeviceToHost);
  for (int i = 0; i < n; i++) grad[i] = tmp[i];
  if (lambdaForce) {
    cudaMemcpy(tmp, st->lambdaForce_d, sizeof(float) * h->nL, cudaMemcpyDeviceToHost);
    for (int i = 0; i < h->nL; i++) lambdaForce[i] = tmp[i];
  }
  free(tmp);
  if (energy)
    cudaMemcpy(energy, st->energy_d + (which == 0 ? eenbrecip : eenbrecipself), sizeof(double),
               cudaMemcpyDeviceToHost);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// Device time of `reps` reciprocal evaluations (getforce_ewald alone, energy
// every `energyEvery`-th call), summed over CUDA events on the path's stream.
extern "C" int ref_time_pme(ref_handle *h, int reps, int energyEvery, double *ms) {
  System *sys = h->sys;
  State *st = h->st;
  st->broadcast_position(sys);
  double total = 0;
  for (int k = 0; k < reps; k++) {
    cudaEventRecord(h->e0, h->stream);
    getforce_ewald(sys, energyEvery > 0 && k % energyEvery == 0);
    cudaEventRecord(h->e1, h->stream);
    cudaEventSynchronize(h->e1);
    float t = 0;
    cudaEventElapsedTime(&t, h->e0, h->e1);
    total += t;
  }
  *ms = total;
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// Constraint clusters in the layouts of TriangleCons / Branch1Cons /
// Branch2Cons / Branch3Cons (host arrays); xPrev, x: host double [3N];
// ism: host float [3N] (LeapState::ism); v: host float [3N] in/out.
// which 0: holonomic_position (x corrected, v from the displacement);
// which 1: holonomic_velocity (v projected, x unchanged).
extern "C" int ref_holonomic(ref_handle *h, int which, int nTri, const void *tri, int n1, const void *b1, int n2,
                             const void *b2, int n3, const void *b3, const double *xPrev, double *x, float *v,
                             const float *ism, float halfdt, float tolerance) {
  System *sys = h->sys;
  Potential *pot = h->pot;
  State *st = h->st;
  const int N = h->N;
  pot->triangleConsCount = nTri;
  pot->branch1ConsCount = n1;
  pot->branch2ConsCount = n2;
  pot->branch3ConsCount = n3;
  cudaMalloc(&pot->triangleCons_d, sizeof(TriangleCons) * (nTri > 0 ? nTri : 1));
  cudaMalloc(&pot->branch1Cons_d, sizeof(Branch1Cons) * (n1 > 0 ? n1 : 1));
  cudaMalloc(&pot->branch2Cons_d, sizeof(Branch2Cons) * (n2 > 0 ? n2 : 1));
  cudaMalloc(&pot->branch3Cons_d, sizeof(Branch3Cons) * (n3 > 0 ? n3 : 1));
  if (nTri) cudaMemcpy(pot->triangleCons_d, tri, sizeof(TriangleCons) * nTri, cudaMemcpyHostToDevice);
  if (n1) cudaMemcpy(pot->branch1Cons_d, b1, sizeof(Branch1Cons) * n1, cudaMemcpyHostToDevice);
  if (n2) cudaMemcpy(pot->branch2Cons_d, b2, sizeof(Branch2Cons) * n2, cudaMemcpyHostToDevice);
  if (n3) cudaMemcpy(pot->branch3Cons_d, b3, sizeof(Branch3Cons) * n3, cudaMemcpyHostToDevice);
  h->run->shakeTolerance = tolerance;
  double *x_d, *xp_d;
  float *v_d, *ism_d;
  cudaMalloc(&x_d, sizeof(double) * 3 * N);
  cudaMalloc(&xp_d, sizeof(double) * 3 * N);
  cudaMalloc(&v_d, sizeof(float) * 3 * N);
  cudaMalloc(&ism_d, sizeof(float) * 3 * N);
  cudaMemcpy(x_d, x, sizeof(double) * 3 * N, cudaMemcpyHostToDevice);
  cudaMemcpy(xp_d, xPrev, sizeof(double) * 3 * N, cudaMemcpyHostToDevice);
  cudaMemcpy(v_d, v, sizeof(float) * 3 * N, cudaMemcpyHostToDevice);
  cudaMemcpy(ism_d, ism, sizeof(float) * 3 * N, cudaMemcpyHostToDevice);
  LeapState ls;
  memset(&ls, 0, sizeof(ls));
  ls.N1 = 3 * N;
  ls.N = 3 * N;
  ls.x = x_d;
  ls.v = v_d;
  ls.ism = ism_d;
  LeapParms2 lp;
  memset(&lp, 0, sizeof(lp));
  lp.halfdt = halfdt;
  st->leapState = &ls;
  st->leapParms2 = &lp;
  st->positionCons_d = xp_d;
  if (which == 0) holonomic_position(sys);
  else holonomic_velocity(sys);
  int rc = cudaStreamSynchronize(h->stream) == cudaSuccess ? 0 : 2;
  cudaMemcpy(x, x_d, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost);
  cudaMemcpy(v, v_d, sizeof(float) * 3 * N, cudaMemcpyDeviceToHost);
  st->leapState = NULL;
  st->leapParms2 = NULL;
  st->positionCons_d = NULL;
  cudaFree(x_d);
  cudaFree(xp_d);
  cudaFree(v_d);
  cudaFree(ism_d);
  cudaFree(pot->triangleCons_d);
  cudaFree(pot->branch1Cons_d);
  cudaFree(pot->branch2Cons_d);
  cudaFree(pot->branch3Cons_d);
  return rc ? rc : (cudaGetLastError() == cudaSuccess ? 0 : 2);
}

// ---- MSLD lambda maps, biases and the integrator step -----------------------
// Out-of-path symbols that src/msld/msld.cu (its script parser) and
// src/update/update.cu (the barostat) reference; never called here.
void io_nexta(char *, char *) { fatal(__FILE__, __LINE__, "parser not available\n"); }
std::string io_nexts(char *) { fatal(__FILE__, __LINE__, "parser not available\n"); return std::string(); }
bool io_nextb(char *) { fatal(__FILE__, __LINE__, "parser not available\n"); return false; }
int io_nexti(char *) { fatal(__FILE__, __LINE__, "parser not available\n"); return 0; }
real io_nextf(char *) { fatal(__FILE__, __LINE__, "parser not available\n"); return 0; }
void Selections::dump() {}
void pressure_coupling(System *) { fatal(__FILE__, __LINE__, "barostat not available\n"); }

// MSLD layout and biases into Msld, as Msld::initialize leaves them
// (src/msld/msld.cu): siteBound[siteCount+1], lambdaSite[nL], blockFixed[nL]
// (bytes), lambdaBias[nL] (the fixed bias b_i), the VariableBias list, fnex.
extern "C" int ref_set_msld(ref_handle *h, int siteCount, const int *siteBound, const int *lambdaSite,
                            const unsigned char *blockFixed, const float *lambdaBias, int varCount,
                            const void *varBias, float fnex) {
  Msld *m = h->msld;
  const int nL = h->nL;
  m->siteCount = siteCount;
  m->blockCount = nL;
  m->fnex = fnex;
  m->fix = false;
  m->new_implicit = false;
  cudaMalloc(&m->siteBound_d, sizeof(int) * (siteCount + 1));
  cudaMemcpy(m->siteBound_d, siteBound, sizeof(int) * (siteCount + 1), cudaMemcpyHostToDevice);
  cudaMalloc(&m->lambdaSite_d, sizeof(int) * nL);
  cudaMemcpy(m->lambdaSite_d, lambdaSite, sizeof(int) * nL, cudaMemcpyHostToDevice);
  cudaMalloc(&m->blockFixed_d, sizeof(bool) * nL);
  cudaMemcpy(m->blockFixed_d, blockFixed, sizeof(bool) * nL, cudaMemcpyHostToDevice);
  cudaMalloc(&m->lambdaBias_d, sizeof(real) * nL);
  cudaMemcpy(m->lambdaBias_d, lambdaBias, sizeof(real) * nL, cudaMemcpyHostToDevice);
  m->variableBiasCount = varCount;
  cudaMalloc(&m->variableBias_d, sizeof(VariableBias) * (varCount > 0 ? varCount : 1));
  if (varCount) cudaMemcpy(m->variableBias_d, varBias, sizeof(VariableBias) * varCount, cudaMemcpyHostToDevice);
  m->theta0_d = NULL;
  m->dcdt_d = NULL;
  h->run->calcTermFlag[eelambda] = true;
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// Msld::calc_lambda_from_theta on theta (host double [nL]); lambda out
// (host double [nL]).
extern "C" int ref_msld_lambda(ref_handle *h, const double *theta, double *lambda) {
  State *st = h->st;
  cudaMemcpy(st->theta_d, theta, sizeof(double) * h->nL, cudaMemcpyHostToDevice);
  h->msld->calc_lambda_from_theta(h->stream, h->sys);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return 2;
  cudaMemcpy(lambda, st->lambda_d, sizeof(double) * h->nL, cudaMemcpyDeviceToHost);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// Msld::calc_thetaForce_from_lambdaForce on the FP32 mirrors lambda_fd,
// theta_fd and lambdaForce_d (host float [nL] each); thetaForce_d starts at
// zero and is returned (host float [nL]).
extern "C" int ref_msld_theta_force(ref_handle *h, const float *lambda_f, const float *theta_f,
                                    const float *lambdaForce, float *thetaForce) {
  State *st = h->st;
  const int nL = h->nL;
  cudaMemcpy(st->lambda_fd, lambda_f, sizeof(float) * nL, cudaMemcpyHostToDevice);
  cudaMemcpy(st->theta_fd, theta_f, sizeof(float) * nL, cudaMemcpyHostToDevice);
  cudaMemcpy(st->lambdaForce_d, lambdaForce, sizeof(float) * nL, cudaMemcpyHostToDevice);
  cudaMemset(st->thetaForce_d, 0, sizeof(float) * nL);
  h->msld->calc_thetaForce_from_lambdaForce(h->stream, h->sys);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return 2;
  cudaMemcpy(thetaForce, st->thetaForce_d, sizeof(float) * nL, cudaMemcpyDeviceToHost);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// Msld::getforce_fixedBias + getforce_variableBias on lambda_fd (host float
// [nL]); lambdaForce_d and energy_d[eelambda] start at zero and are returned.
extern "C" int ref_msld_bias(ref_handle *h, const float *lambda_f, int calcEnergy, float *lambdaForce,
                             double *energy) {
  State *st = h->st;
  const int nL = h->nL;
  cudaMemcpy(st->lambda_fd, lambda_f, sizeof(float) * nL, cudaMemcpyHostToDevice);
  cudaMemset(st->lambdaForce_d, 0, sizeof(float) * nL);
  cudaMemset(st->energy_d, 0, sizeof(double) * eeend);
  h->msld->getforce_fixedBias(h->sys, calcEnergy != 0);
  h->msld->getforce_variableBias(h->sys, calcEnergy != 0);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return 2;
  cudaMemcpy(lambdaForce, st->lambdaForce_d, sizeof(float) * nL, cudaMemcpyDeviceToHost);
  if (energy) cudaMemcpy(energy, st->energy_d + eelambda, sizeof(double), cudaMemcpyDeviceToHost);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// One State::update (src/update/update.cu:233-305) on a step that is not an
// energy step: dU/dtheta from dU/dlambda, update_VVhbpR, holonomic_position,
// update_OOhbpR, holonomic_position, lambda from theta.  The Msld layout must
// be set (ref_set_msld).  Host arrays in the reference's precisions:
//   pos    double [nL + 3N + nL]  [lambda | x | theta] in/out
//   vel    float [3N + nL]        velocityBuffer_d (x then theta) in/out
//   frc    float [nL + 3N + nL]   [dU/dlambda | dU/dx | dU/dtheta]; the theta
//                                 part is added to by the step (returned)
//   ism    float [3N + nL]        1/sqrt(m)
//   random float [3N + nL]        the Gaussian numbers update_OOhbpR reads
//   lp     float [6]              friction, noise, halfdt for x then theta
// Constraint clusters as in ref_holonomic (counts may be zero).
extern "C" int ref_update_step(ref_handle *h, double *pos, float *vel, float *frc, const float *ism,
                               const float *random, const float *lp, int nTri, const void *tri, int n1,
                               const void *b1, int n2, const void *b2, int n3, const void *b3, float tolerance) {
  System *sys = h->sys;
  State *st = h->st;
  Potential *pot = h->pot;
  Run *run = h->run;
  const int N = h->N, nL = h->nL;
  const int nbuf = 3 * N + 2 * nL, ndof = 3 * N + nL;
  pot->triangleConsCount = nTri;
  pot->branch1ConsCount = n1;
  pot->branch2ConsCount = n2;
  pot->branch3ConsCount = n3;
  cudaMalloc(&pot->triangleCons_d, sizeof(TriangleCons) * (nTri > 0 ? nTri : 1));
  cudaMalloc(&pot->branch1Cons_d, sizeof(Branch1Cons) * (n1 > 0 ? n1 : 1));
  cudaMalloc(&pot->branch2Cons_d, sizeof(Branch2Cons) * (n2 > 0 ? n2 : 1));
  cudaMalloc(&pot->branch3Cons_d, sizeof(Branch3Cons) * (n3 > 0 ? n3 : 1));
  if (nTri) cudaMemcpy(pot->triangleCons_d, tri, sizeof(TriangleCons) * nTri, cudaMemcpyHostToDevice);
  if (n1) cudaMemcpy(pot->branch1Cons_d, b1, sizeof(Branch1Cons) * n1, cudaMemcpyHostToDevice);
  if (n2) cudaMemcpy(pot->branch2Cons_d, b2, sizeof(Branch2Cons) * n2, cudaMemcpyHostToDevice);
  if (n3) cudaMemcpy(pot->branch3Cons_d, b3, sizeof(Branch3Cons) * n3, cudaMemcpyHostToDevice);
  run->shakeTolerance = tolerance;
  run->step = 1;
  run->freqNRG = 1000;  // step % freqNRG != 0: the VVhbpR branch
  run->freqNPT = 0;
  cudaMemcpy(st->positionBuffer_d, pos, sizeof(double) * nbuf, cudaMemcpyHostToDevice);
  cudaMemcpy(st->forceBuffer_d, frc, sizeof(float) * nbuf, cudaMemcpyHostToDevice);
  float *v_d, *ism_d, *rnd_d;
  cudaMalloc(&v_d, sizeof(float) * ndof);
  cudaMalloc(&ism_d, sizeof(float) * ndof);
  cudaMalloc(&rnd_d, sizeof(float) * ndof);
  cudaMalloc(&st->positionCons_d, sizeof(double) * ndof);
  cudaMalloc(&st->nanFlag_d, sizeof(int));
  cudaMemset(st->nanFlag_d, 0xFF, sizeof(int));
  cudaMemcpy(v_d, vel, sizeof(float) * ndof, cudaMemcpyHostToDevice);
  cudaMemcpy(ism_d, ism, sizeof(float) * ndof, cudaMemcpyHostToDevice);
  cudaMemcpy(rnd_d, random, sizeof(float) * ndof, cudaMemcpyHostToDevice);
  LeapState ls;
  memset(&ls, 0, sizeof(ls));
  ls.N1 = 3 * N;
  ls.N = ndof;
  ls.x = (real_x *)st->position_d;
  ls.v = v_d;
  ls.f = (real_f *)st->force_d;
  ls.ism = ism_d;
  ls.random = rnd_d;
  LeapParms2 lpx = {lp[0], lp[1], lp[2]}, lpt = {lp[3], lp[4], lp[5]};
  st->leapState = &ls;
  st->leapParms2 = &lpx;
  st->lambdaLeapParms2 = &lpt;
  sys->id = 0;
  st->broadcast_position(sys);  // FP32 mirrors the theta force reads
  st->update(1, sys);
  int rc = cudaStreamSynchronize(h->stream) == cudaSuccess ? 0 : 2;
  cudaMemcpy(pos, st->positionBuffer_d, sizeof(double) * nbuf, cudaMemcpyDeviceToHost);
  cudaMemcpy(frc, st->forceBuffer_d, sizeof(float) * nbuf, cudaMemcpyDeviceToHost);
  cudaMemcpy(vel, v_d, sizeof(float) * ndof, cudaMemcpyDeviceToHost);
  st->leapState = NULL;
  st->leapParms2 = NULL;
  st->lambdaLeapParms2 = NULL;
  cudaFree(v_d);
  cudaFree(ism_d);
  cudaFree(rnd_d);
  cudaFree(st->positionCons_d);
  cudaFree(st->nanFlag_d);
  st->positionCons_d = NULL;
  st->nanFlag_d = NULL;
  cudaFree(pot->triangleCons_d);
  cudaFree(pot->branch1Cons_d);
  cudaFree(pot->branch2Cons_d);
  cudaFree(pot->branch3Cons_d);
  return rc ? rc : (cudaGetLastError() == cudaSuccess ? 0 : 2);
}

// Triclinic cell for the handle (State::typeBox = true): tric host double [6]
// in the layout of State::tricBox (A_x, B_x, B_y, C_x, C_y, C_z), also the
// FP32 copy tricBox_f the direct-space path reads.
extern "C" int ref_set_tric(ref_handle *h, const double *tric) {
  State *st = h->st;
  st->typeBox = true;
  st->tricBox.a.x = tric[0];
  st->tricBox.b.x = tric[1]; st->tricBox.b.y = tric[2];
  st->tricBox.c.x = tric[3]; st->tricBox.c.y = tric[4]; st->tricBox.c.z = tric[5];
  st->tricBox_f.a.x = (float)tric[0];
  st->tricBox_f.b.x = (float)tric[1]; st->tricBox_f.b.y = (float)tric[2];
  st->tricBox_f.c.x = (float)tric[3]; st->tricBox_f.c.y = (float)tric[4]; st->tricBox_f.c.z = (float)tric[5];
  st->orthBox.x = tric[0]; st->orthBox.y = tric[2]; st->orthBox.z = tric[5];
  st->orthBox_f.x = (float)tric[0]; st->orthBox_f.y = (float)tric[2]; st->orthBox_f.z = (float)tric[5];
  // reciprocal cell the PME kernels read (State::kTricBox_f, as set by
  // src/system/state.cxx:485-491 from tricBox_f, in the reference's real)
  const real Vinv = 1 / (st->tricBox_f.a.x * st->tricBox_f.b.y * st->tricBox_f.c.z);
  st->kTricBox_f.a.x = st->tricBox_f.b.y * st->tricBox_f.c.z * Vinv;
  st->kTricBox_f.a.y = -st->tricBox_f.b.x * st->tricBox_f.c.z * Vinv;
  st->kTricBox_f.a.z = (st->tricBox_f.b.x * st->tricBox_f.c.y - st->tricBox_f.b.y * st->tricBox_f.c.x) * Vinv;
  st->kTricBox_f.b.x = st->tricBox_f.c.z * st->tricBox_f.a.x * Vinv;
  st->kTricBox_f.b.y = -st->tricBox_f.c.y * st->tricBox_f.a.x * Vinv;
  st->kTricBox_f.c.x = st->tricBox_f.a.x * st->tricBox_f.b.y * Vinv;
  return 0;
}
