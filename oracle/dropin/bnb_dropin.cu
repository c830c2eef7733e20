// The drop-in binding of libbnb into BLaDE, compiled.
//
// COMPARISON INFRASTRUCTURE.  oracle/dropin/Makefile builds the reference's
// own sources twice: unmodified (blade_ref) and with this file in place of
// src/domdec/*.cu and src/nbdirect/nbdirect.cu (blade_bnb).  The reference's
// headers stay as they are, so the Domdec class keeps its members; the libbnb
// handle of each Domdec lives in a table keyed by the object.  Everything
// else -- parser, structure and parameter readers, Potential::initialize, the
// step loop, bonded terms, PME, MSLD, the integrator -- is the reference's.
//
// What this file provides is what the rest of the reference calls of the
// replaced files (src/domdec/domdec.h:93-110, src/nbdirect/nbdirect.h:7-8):
//   Domdec::Domdec / ~Domdec / initialize / reset_domdec / update_domdec
//   getforce_nbdirect / getforce_nbdirect_reduce
// Domdec::localForce_d and maxBlocks stay valid because
// Potential::reset_force clears them (src/system/potential.cxx:1845).
#include <cuda_runtime.h>

#include <cmath>
#include <map>
#include <mutex>

#include "bnb.h"
#include "domdec/domdec.h"
#include "io/io.h"
#include "main/defines.h"
#include "main/gpu_check.h"
#include "msld/msld.h"
#include "nbdirect/nbdirect.h"
#include "run/run.h"
#include "system/potential.h"
#include "system/state.h"
#include "system/system.h"

void calc_virtual_position(System *system, bool rectify);  // src/holonomic/virtual.cu

namespace {
struct Binding {
  bnb_handle *h = nullptr;
  float box[6];
};
std::map<const Domdec *, Binding> g_bind;
std::mutex g_lock;

Binding &binding(const Domdec *d) {
  std::lock_guard<std::mutex> lock(g_lock);
  return g_bind[d];
}

void check(int rc, const char *what) {
  if (rc != BNB_OK) fatal(__FILE__, __LINE__, "libbnb %s failed with code %d\n", what, rc);
}

// The boxes argument of libbnb from the State: orthBox_f, or tricBox_f in its
// memory order (A_x, B_x, B_y, C_x, C_y, C_z).
void state_box(const State *s, float *box) {
  if (s->typeBox) {
    box[0] = s->tricBox_f.a.x;
    box[1] = s->tricBox_f.b.x; box[2] = s->tricBox_f.b.y;
    box[3] = s->tricBox_f.c.x; box[4] = s->tricBox_f.c.y; box[5] = s->tricBox_f.c.z;
  } else {
    box[0] = s->orthBox_f.x; box[1] = s->orthBox_f.y; box[2] = s->orthBox_f.z;
  }
}

// In-place wrap of the FP64 positions into the cell, as Domdec::assign_domain
// does (src/domdec/assign_domain.cu:14-45), so that the reference's other
// terms (PME, output) see the coordinates they see in the unmodified build.
template <bool TRIC>
__global__ void k_wrap(int n, double *x, double ax, double bx, double by, double cx, double cy, double cz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double p0 = x[3 * i], p1 = x[3 * i + 1], p2 = x[3 * i + 2];
  if (TRIC) {
    double k = floor(p2 / cz);
    p0 -= cx * k; p1 -= cy * k; p2 -= cz * k;
    k = floor(p1 / by);
    p0 -= bx * k; p1 -= by * k;
    p0 -= ax * floor(p0 / ax);
  } else {
    p0 = fmod(p0, ax); p0 += p0 < 0 ? ax : 0;
    p1 = fmod(p1, by); p1 += p1 < 0 ? by : 0;
    p2 = fmod(p2, cz); p2 += p2 < 0 ? cz : 0;
  }
  x[3 * i] = p0; x[3 * i + 1] = p1; x[3 * i + 2] = p2;
}
}  // namespace

Domdec::Domdec() {
  domain = NULL; domain_d = NULL; localToGlobal_d = NULL; globalToLane_d = NULL; globalToBlock_d = NULL;
  localPosition_d = NULL; localForce_d = NULL; localNbonds_d = NULL; blockSort_d = NULL; blockToken_d = NULL;
  blockBounds_d = NULL; blockCount = NULL; blockCount_d = NULL; blockVolume_d = NULL;
  blockCandidateCount_d = NULL; blockCandidates_d = NULL; blockPartnerCount_d = NULL; blockPartners_d = NULL;
  localExcls_d = NULL; firstExcl_d = NULL; mapExcl_d = NULL; exclSort_d = NULL; sortedExcls_d = NULL;
  blockExcls_d = NULL; overflowFlag_d = NULL;
  maxBlocks = 0;
}

Domdec::~Domdec() {
  Binding b;
  {
    std::lock_guard<std::mutex> lock(g_lock);
    auto it = g_bind.find(this);
    if (it != g_bind.end()) { b = it->second; g_bind.erase(it); }
  }
  if (b.h) bnb_destroy(b.h);
  if (localForce_d) cudaFree(localForce_d);
  if (blockCount) free(blockCount);
}

void Domdec::initialize(System *system) {
  calc_virtual_position(system, true);
  system->state->broadcast_position(system);
  system->state->broadcast_box(system);
  id = system->id;
  idCount = system->idCount;
  if (idCount > 1) fatal(__FILE__, __LINE__, "the libbnb drop-in runs one system per GPU\n");
  gridDomdec = make_int3(1, 1, 1);
  idDomdec = make_int3(0, 0, 0);
  globalCount = system->state->atomCount;
  blockCount = (int *)calloc(2, sizeof(int));
  // Potential::reset_force clears 32*maxBlocks forces here; libbnb keeps its own accumulators
  maxBlocks = 1;
  gpuCheck(cudaMalloc(&localForce_d, 32 * maxBlocks * sizeof(real3_f)));
  // the reference's rebuild period and list pad (src/domdec/domdec.cu:137-138)
  freqDomdec = 10;
  cullPad = 2 * sqrt(30 * kB * system->run->T / 1) * freqDomdec * system->run->dt;

  Run *r = system->run;
  Potential *p = system->potential;
  bnb_params prm;
  bnb_default_params(&prm);
  prm.rCut = r->cutoffs.rCut;
  prm.rSwitch = r->cutoffs.rSwitch;
  prm.betaEwald = r->cutoffs.betaEwald;
  prm.elecMethod = r->elecMethod;
  prm.vdwMethod = r->vdwMethod;
  prm.useSoftCore = system->msld->useSoftCore;
  prm.cullPad = cullPad;
  prm.kElectric = kELECTRIC;
  prm.softCoreRadius = SOFTCORERADIUS;
  Binding &b = binding(this);
  int n = globalCount;
  check(bnb_create(&prm, 1, &n, &b.h), "bnb_create");
  int lambdas = system->msld->blockCount;
  check(bnb_set_topology(b.h, (const bnb_nbond *)p->nbonds, &p->vdwParameterCount,
                         (const bnb_vdw *)p->vdwParameters, &lambdas, p->exclCount, (const int *)p->excls, NULL),
        "bnb_set_topology");
  if (system->state->typeBox) check(bnb_set_box_type(b.h, 1), "bnb_set_box_type");
  reset_domdec(system);
}

void Domdec::reset_domdec(System *system) {
  State *s = system->state;
  Run *r = system->run;
  Binding &b = binding(this);
  const int n = s->atomCount;
  if (n > 0) {
    const int grid = (n + 255) / 256;
    if (s->typeBox)
      k_wrap<true><<<grid, 256, 0, r->updateStream>>>(n, (double *)s->position_d, s->tricBox.a.x, s->tricBox.b.x,
                                                      s->tricBox.b.y, s->tricBox.c.x, s->tricBox.c.y,
                                                      s->tricBox.c.z);
    else
      k_wrap<false><<<grid, 256, 0, r->updateStream>>>(n, (double *)s->position_d, s->orthBox.x, 0, s->orthBox.y,
                                                       0, 0, s->orthBox.z);
    gpuCheck(cudaGetLastError());
  }
  s->broadcast_position(system);  // the FP32 mirror (State::set_fd)
  state_box(s, b.box);
  check(bnb_rebuild(b.h, (const float *)s->position_fd, b.box, r->updateStream, 0), "bnb_rebuild");
}

void Domdec::update_domdec(System *system, bool resetFlag) {
  calc_virtual_position(system, resetFlag);
  if (resetFlag) {
    reset_domdec(system);
  } else {
    system->state->broadcast_position(system);
  }
}

void getforce_nbdirect(System *system, bool calcEnergy) {
  if (system->run->calcTermFlag[eenbdirect] == false) return;
  State *s = system->state;
  Binding &b = binding(system->domdec);
  state_box(s, b.box);
  bnb_outputs out = {0};
  out.force = (float *)s->force_d;      // dU/dx, added like unpack_forces
  out.lambdaForce = s->lambdaForce_d;   // dU/dlambda, added
  out.energy = calcEnergy ? s->energy_d + eenbdirect : NULL;
  check(bnb_compute(b.h, (const float *)s->position_fd, s->lambda_fd, b.box, calcEnergy ? 1 : 0, &out,
                    system->run->nbdirectStream),
        "bnb_compute");
}

void getforce_nbdirect_reduce(System *system, bool calcEnergy) {}  // one GPU: nothing to reduce
