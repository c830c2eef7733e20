// C ABI of libbnb: handle life cycle, topology upload, list rebuild with
// capacity growth, and the per-step direct-space evaluation.
//
// Host-side counterpart of Domdec::initialize/reset_domdec/update_domdec
// (src/domdec/domdec.cu:83-222) and getforce_nbdirect
// (src/nbdirect/nbdirect.cu:492-581).  All device memory of a handle lives in
// two arenas (topology, list); capacities grow only inside a synchronous
// rebuild, never during an asynchronous (graph-capturable) call.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <new>
#include <tuple>
#include <vector>

#include "bnb.h"
#include "bnb_internal.h"
#include "erfc_fit.h"
#include "listbuild.h"
#include "nbdirect.h"
#include "pairs.h"
#include "pme.h"

using bnb::Dev;
using bnb::PairConst;
using bnb::RepInfo;

struct bnb_handle {
  bnb_params p;
  int R = 0, N = 0;
  int triclinic = 0;  // boxes arrays: 3 floats per replica, or 6 (State::tricBox_f layout)
  std::vector<int> atomCount, atomStart;
  // topology
  bool topo = false;
  int nTypes = 0, combine = 0, lamTotal = 0, alch = 0;
  std::vector<int> lamStart, lamCount;
  size_t exclTotal = 0;
  // columns / replicas
  std::vector<RepInfo> rep;
  std::vector<RepInfo> repDev;  // copy of what the device holds
  std::vector<int> colRep;
  int totalCols = 0;
  // capacities
  int maxBlocks = 0, capCand = 0, capMask = 0, capWork = 0;
  bool listBuilt = false;
  int lastWork = 0;
  int resTiles = 0, resMasks = 0, resWork = 0;
  bool reserveDirty = false;
  int tilesPerWork = bnb::kTilesPerWork, ctasPerSM = 0;  // tuning (bnb_set_tuning / bnb_autotune)
  int tailItems = bnb::kTailItems;
  int smCount = 0;
  bool counting = false;
  bool orderPending = false;  // sort the work items by cost after the next pair launch
  // profiling (bnb_profile)
  bool prof = false;
  std::vector<cudaEvent_t> pairEv, rebEv;
  int pairN = 0, rebN = 0;
  unsigned long long launches = 0;
  // device
  Dev d{};
  void *topoArena = nullptr, *listArena = nullptr;
  size_t listBytes = 0;
  int *colRep_d = nullptr;
  PairConst pc{};
  // nb14 / nbex lists (bnb_set_pairs)
  void *pairArena = nullptr;
  int n14 = 0, nex = 0;
  bool soft14 = false;
  bnb_nb14 *nb14_d = nullptr;
  bnb_nbex *nbex_d = nullptr;
  long long *accP = nullptr, *accPL = nullptr, *accPE = nullptr;
  // PME reciprocal space (bnb_set_pme)
  void *pmeArena = nullptr;
  int pmeOrder = 0, pmeTotalGrid = 0, pmeTotalCplx = 0, pmeMaxCplx = 0;
  std::vector<bnb::PmeRep> pmeRep;
  struct PmePlan { cufftHandle r2c, c2r; int first, count; };
  std::vector<PmePlan> pmePlans;
  bnb::PmeRep *pmeRep_d = nullptr;
  float *pmeMod_d = nullptr, *pmeGrid_d = nullptr;
  float2 *pmeCplx_d = nullptr;
  long long *pmeFix_d = nullptr, *pmeAccL = nullptr, *pmeAccE = nullptr;
  unsigned int *pmeDone = nullptr;
};

namespace {

// Largest list capacity: the three-pass scan handles up to 4096 x 4096 items.
constexpr long long kCapLimit = 4096LL * 4096LL;
constexpr int kProfSlots = 4096;

void destroy_events(bnb_handle *h) {
  for (auto e : h->pairEv) cudaEventDestroy(e);
  for (auto e : h->rebEv) cudaEventDestroy(e);
  h->pairEv.clear();
  h->rebEv.clear();
  h->pairN = h->rebN = 0;
}

struct Arena {
  size_t off = 0;
  template <typename T>
  size_t take(size_t n) {
    size_t o = off;
    off += ((sizeof(T) * (n > 0 ? n : 1)) + 255) & ~size_t(255);
    return o;
  }
};

inline bool ok(cudaError_t e) { return e == cudaSuccess; }

// calcEnergy of the compute calls: bit 0 the energy path, BNB_OUT_SET and
// BNB_OUT_ADD64 the output modes; nothing else.
inline bool flags_ok(int calcEnergy) { return (calcEnergy & ~(1 | BNB_OUT_SET | BNB_OUT_ADD64)) == 0; }
inline int out_mode(int calcEnergy) { return calcEnergy & (BNB_OUT_SET | BNB_OUT_ADD64); }

PairConst make_const(const bnb_params &p) {
  PairConst c{};
  double rc = p.rCut, rs = p.rSwitch, b = p.betaEwald;
  c.rcut = (float)rc;
  c.rswitch = (float)rs;
  c.rc2 = (float)rc * (float)rc;
  c.beta = (float)b;
  c.softR = p.softCoreRadius;
  c.mBeta2Log2e = (float)(-b * b / std::log(2.0));
  c.pBeta = bnb::kErfcP * (float)b;
  c.twoBetaSqrtPi = (float)(2.0 * b / std::sqrt(M_PI));
  double rc3 = rc * rc * rc, rs3 = rs * rs * rs;
  c.k6 = (float)(rc3 / (rc3 - rs3));
  c.k12 = (float)(rc3 * rc3 / (rc3 * rc3 - rs3 * rs3));
  c.rci3 = (float)(1.0 / rc3);
  c.rci6 = (float)(1.0 / (rc3 * rc3));
  c.k6rci3 = (float)(rc3 / (rc3 - rs3) / rc3);
  c.k12rci6 = (float)(rc3 * rc3 / (rc3 * rc3 - rs3 * rs3) / (rc3 * rc3));
  double dv6 = 1.0 / (rc3 * rs3);
  c.dv6 = (float)dv6;
  c.dv12 = (float)(dv6 * dv6);
  double roff2 = rc * rc, ron2 = rs * rs;
  c.roff2 = (float)roff2;
  c.ron2 = (float)ron2;
  double rul3 = (roff2 - ron2) * (roff2 - ron2) * (roff2 - ron2);
  c.rul3inv = (float)(1.0 / rul3);
  c.rul12 = (float)(12.0 / rul3);
  double ginv = 1.0 / rul3;
  c.fA = (float)(roff2 * roff2 * (roff2 - 3 * ron2) * ginv);
  c.fB = (float)(6 * roff2 * ron2 * ginv);
  c.fC = (float)(-(ron2 + roff2) * ginv);
  c.fD = (float)(2 * ginv / 5);
  c.fdvc = (float)(8 * (ron2 * roff2 * (rc - rs) - (roff2 * roff2 * rc - ron2 * ron2 * rs) / 5) * ginv);
  c.rcinv = (float)(1.0 / rc);
  c.fsG = (float)ginv;
  c.fsG5 = (float)(ginv / 5);
  c.fsC1 = (float)(roff2 - 3 * ron2);
  c.fsP1 = (float)(6 * rc);
  c.fsP2 = (float)(7 * rc * rc - 5 * rs * rs);
  c.fsP3 = (float)(5 * rc * rc * rc - 15 * rc * rs * rs);
  double rc6 = roff2 * roff2 * roff2;
  c.vshRc6inv = (float)(1.0 / rc6);
  c.vshRc12inv = (float)(1.0 / (rc6 * rc6));
  c.vshRc18inv = (float)(1.0 / (rc6 * rc6 * rc6));
  return c;
}

void free_pme(bnb_handle *h) {
  for (auto &p : h->pmePlans) {
    cufftDestroy(p.r2c);
    cufftDestroy(p.c2r);
  }
  h->pmePlans.clear();
  if (h->pmeArena) cudaFree(h->pmeArena);
  h->pmeArena = nullptr;
  h->pmeOrder = 0;
  h->pmeRep.clear();
}

void free_list(bnb_handle *h) {
  if (h->listArena) cudaFree(h->listArena);
  h->listArena = nullptr;
  h->listBytes = 0;
  h->listBuilt = false;
}

// (Re)allocates the list arena for the current capacities.
int alloc_list(bnb_handle *h) {
  free_list(h);
  Dev &d = h->d;
  const int N = h->N, C = h->totalCols, MB = h->maxBlocks;
  Arena a;
  size_t o_wrap = a.take<int>(N), o_col = a.take<int>(N), o_z = a.take<uint32_t>(N);
  size_t o_cc = a.take<int>(C), o_csa = a.take<int>(C + 1), o_csb = a.take<int>(C + 1),
         o_cf = a.take<int>(C), o_colrep = a.take<int>(C);
  size_t o_bucket = a.take<int>(N), o_sorted = a.take<int>(N);
  size_t o_bb = a.take<int>(MB + 1), o_brep = a.take<int>(MB), o_rbs = a.take<int>(h->R + 1);
  size_t o_slotA = a.take<int>(32 * MB), o_atomSlot = a.take<int>(N), o_slotQ = a.take<float>(32 * MB),
         o_slotT = a.take<int>(32 * MB), o_slotSB = a.take<int>(32 * MB);
  size_t o_ckey = a.take<uint32_t>(6 * (size_t)C), o_eb = a.take<int>(bnb::kExclBlk * MB),
         o_ebc = a.take<int>(MB);
  size_t o_cullC = a.take<int>(MB * bnb::kNumShifts), o_cullO = a.take<int>(MB * bnb::kNumShifts + 1);
  size_t o_cand = a.take<int4>(h->capCand), o_cflag = a.take<int>(h->capCand),
         o_cmo = a.take<int>(h->capCand + 1);
  size_t o_masks = a.take<uint32_t>(32 * (size_t)h->capMask);
  size_t o_cs = a.take<int>(MB + 1), o_work = a.take<int2>(h->capWork), o_cost = a.take<unsigned int>(h->capWork),
         o_order = a.take<int>(h->capWork);
  size_t o_part = a.take<int>(4096);
  size_t o_xyzq = a.take<float4>(32 * MB), o_bmin = a.take<float4>(MB), o_bmax = a.take<float4>(MB);
  size_t o_acc = a.take<long long>(3 * 32 * (size_t)MB);
  void *base = nullptr;
  if (!ok(cudaMalloc(&base, a.off))) return BNB_ERR_CUDA;
  h->listArena = base;
  h->listBytes = a.off;
  char *b = static_cast<char *>(base);
  d.wrap = (int *)(b + o_wrap);
  d.atomCol = (int *)(b + o_col);
  d.atomZKey = (uint32_t *)(b + o_z);
  d.colCount = (int *)(b + o_cc);
  d.colStartAtom = (int *)(b + o_csa);
  d.colStartBlock = (int *)(b + o_csb);
  d.colFill = (int *)(b + o_cf);
  h->colRep_d = (int *)(b + o_colrep);
  d.bucket = (int *)(b + o_bucket);
  d.sortedAtom = (int *)(b + o_sorted);
  d.blockBounds = (int *)(b + o_bb);
  d.blockRep = (int *)(b + o_brep);
  d.repBlockStart = (int *)(b + o_rbs);
  d.slotAtom = (int *)(b + o_slotA);
  d.atomSlot = (int *)(b + o_atomSlot);
  d.slotQ = (float *)(b + o_slotQ);
  d.slotType = (int *)(b + o_slotT);
  d.slotSiteBlock = (int *)(b + o_slotSB);
  d.colKey = (uint32_t *)(b + o_ckey);
  d.exclBlk = (int *)(b + o_eb);
  d.exclBlkCount = (int *)(b + o_ebc);
  d.cullCount = (int *)(b + o_cullC);
  d.cullOffset = (int *)(b + o_cullO);
  d.cand = (int4 *)(b + o_cand);
  d.candFlag = (int *)(b + o_cflag);
  d.candMaskOff = (int *)(b + o_cmo);
  d.masks = (uint32_t *)(b + o_masks);
  d.candStart = (int *)(b + o_cs);
  d.work = (int2 *)(b + o_work);
  d.itemCost = (unsigned int *)(b + o_cost);
  d.order = (int *)(b + o_order);
  d.scanPartial = (int *)(b + o_part);
  d.xyzq = (float4 *)(b + o_xyzq);
  d.bmin = (float4 *)(b + o_bmin);
  d.bmax = (float4 *)(b + o_bmax);
  d.accF = (long long *)(b + o_acc);
  d.totalCols = C;
  d.maxBlocks = MB;
  d.capCand = h->capCand;
  d.capMask = h->capMask;
  d.capWork = h->capWork;
  if (!ok(cudaMemset(base, 0, a.off))) return BNB_ERR_CUDA;
  if (!ok(cudaMemcpy(h->colRep_d, h->colRep.data(), sizeof(int) * std::max(C, 1),
                     cudaMemcpyHostToDevice)))
    return BNB_ERR_CUDA;
  return BNB_OK;
}

// Box of replica r from a caller's boxes array: three edge lengths, or after
// bnb_set_box_type(h, 1) six floats in the layout of State::tricBox_f
// (A_x, B_x, B_y, C_x, C_y, C_z; src/system/state.h).
void box_of(const bnb_handle *h, const float *boxes, int r, float b[3], float t[3]) {
  if (h->triclinic) {
    const float *q = boxes + 6 * r;
    b[0] = q[0]; b[1] = q[2]; b[2] = q[5];
    t[0] = q[1]; t[1] = q[3]; t[2] = q[4];
  } else {
    for (int k = 0; k < 3; k++) { b[k] = boxes[3 * r + k]; t[k] = 0.f; }
  }
}

// Image shift vectors of the 14 half-shell codes for a replica's box.  The
// integer shifts follow the reference's cull over neighbouring domains for a
// single domain (src/domdec/cull.cu:141-190): z in {0,1}; y in y0 + {-z..1}
// with y0 = -floor(z C_y / B_y + 1/2); x in x0 + {-(y'!=0||z!=0)..1} with
// x0 = -floor((z C_x + y B_x) / A_x + 1/2), y' the uncentred y.  For an
// orthorhombic box y0 = x0 = 0 and the codes are the plain half shell.
void set_shifts(RepInfo &ri) {
  for (int code = 0; code < bnb::kNumShifts; code++) {
    int x, y, z;
    if (code < 2) { x = code; y = 0; z = 0; }
    else if (code < 5) { x = code - 3; y = 1; z = 0; }
    else { int c = code - 5; x = c % 3 - 1; y = c / 3 - 1; z = 1; }
    // one rounding per operation (no contraction), as the CPU restatement
    volatile float ty = (float)z * ri.tric[2];
    volatile float qy = ty / ri.box[1];
    const int y0 = -(int)std::floor(qy + 0.5f);
    const int sy = y + y0;
    volatile float tx0 = (float)z * ri.tric[1], tx1 = (float)sy * ri.tric[0];
    volatile float sxy = tx0 + tx1;
    volatile float qx = sxy / ri.box[0];
    const int x0 = -(int)std::floor(qx + 0.5f);
    const int sx = x + x0;
    const float3 v = bnb::lattice_shift(ri.box, ri.tric, sx, sy, z);
    ri.shift[code] = make_float4(v.x, v.y, v.z, 0.f);
  }
}

// Stores the boxes of all replicas; returns true if any changed.
bool store_boxes(bnb_handle *h, const float *boxes) {
  bool changed = false;
  for (int r = 0; r < h->R; r++) {
    float b[3], t[3];
    box_of(h, boxes, r, b, t);
    RepInfo &ri = h->rep[r];
    bool c = false;
    for (int k = 0; k < 3; k++)
      if (ri.box[k] != b[k] || ri.tric[k] != t[k]) c = true;
    if (c) {
      for (int k = 0; k < 3; k++) { ri.box[k] = b[k]; ri.tric[k] = t[k]; }
      set_shifts(ri);
      changed = true;
    }
  }
  return changed;
}

// Column grid per replica from its box; returns true if the layout changed.
bool layout_columns(bnb_handle *h, const float *boxes) {
  bool changed = false;
  int col = 0;
  std::vector<int> colRep;
  for (int r = 0; r < h->R; r++) {
    RepInfo &ri = h->rep[r];
    int dx, dy;
    float b[3], t[3];
    box_of(h, boxes, r, b, t);
    bnb_domain_div(h->atomCount[r], b, &dx, &dy);
    if (dx != ri.divX || dy != ri.divY || col != ri.colStart) changed = true;
    ri.divX = dx;
    ri.divY = dy;
    ri.colStart = col;
    ri.nCols = dx * dy;
    for (int c = 0; c < ri.nCols; c++) colRep.push_back(r);
    col += ri.nCols;
  }
  h->totalCols = col;
  h->colRep.swap(colRep);
  store_boxes(h, boxes);
  return changed;
}

void estimate_capacities(bnb_handle *h, int &mb, long long &cand, long long &work, long long &mask) {
  mb = 0;
  cand = 0;
  for (int r = 0; r < h->R; r++) {
    const RepInfo &ri = h->rep[r];
    int n = h->atomCount[r];
    int blocks = n / 32 + ri.nCols + 1;
    mb += blocks;
    if (n == 0) continue;
    double vol = (double)ri.box[0] * ri.box[1] * ri.box[2];
    double invDens = vol / n;
    double approx = std::cbrt(32 * invDens);
    double edge = approx + 2.0 * (h->p.rCut + h->p.cullPad);
    double perBlock = 0.75 * edge * edge * edge / (32 * invDens) + 16;
    cand += (long long)(perBlock * (n / 32 + 1)) + 14;
  }
  work = cand / bnb::kMinTilesPerWork + mb + 16;
  mask = (long long)(4 * h->exclTotal + 1024) / 32 + 64;
}

// Uploads the per-replica table only when it changed, so steady-state calls
// issue no host-to-device copy (a requirement inside CUDA graph capture).
int upload_rep(bnb_handle *h, cudaStream_t s) {
  for (int r = 0; r < h->R; r++) {
    h->rep[r].atomStart = h->atomStart[r];
    h->rep[r].atomCount = h->atomCount[r];
    h->rep[r].lamStart = h->lamStart.empty() ? 0 : h->lamStart[r];
    h->rep[r].lamCount = h->lamCount.empty() ? 1 : h->lamCount[r];
  }
  if (h->repDev.size() == h->rep.size() &&
      memcmp(h->repDev.data(), h->rep.data(), sizeof(RepInfo) * h->R) == 0)
    return BNB_OK;
  h->repDev = h->rep;
  return ok(cudaMemcpyAsync(h->d.rep, h->repDev.data(), sizeof(RepInfo) * h->R,
                            cudaMemcpyHostToDevice, s))
             ? BNB_OK
             : BNB_ERR_CUDA;
}

}  // namespace

extern "C" {

void bnb_default_params(bnb_params *p) {
  if (!p) return;
  p->rCut = 12.0f;
  p->rSwitch = 10.0f;
  p->betaEwald = 0.32f;
  p->elecMethod = 1;
  p->vdwMethod = 0;
  p->useSoftCore = 1;
  p->cullPad = 2.0f;
  p->kElectric = 332.0716f;
  p->softCoreRadius = 4.0f;
}

const char *bnb_version(void) { return "bnb 0.1 (sm_100a)"; }

int bnb_set_box_type(bnb_handle *h, int triclinic) {
  if (!h || (triclinic != 0 && triclinic != 1)) return BNB_ERR_ARG;
  if (h->triclinic != triclinic) {
    h->triclinic = triclinic;
    h->listBuilt = false;  // the next rebuild reads the boxes in the new layout
  }
  return BNB_OK;
}

int bnb_domain_div(int atomCount, const float *box, int *divX, int *divY) {
  if (!box || !divX || !divY || atomCount < 0) return BNB_ERR_ARG;
  if (atomCount == 0) {
    *divX = *divY = 1;
    return BNB_OK;
  }
  // Same FP32 steps as Domdec::initialize, src/domdec/domdec.cu:114-117.
  float invDensity = box[0] * box[1] * box[2] / (float)atomCount;
  float approx = expf(logf(32.0f * invDensity) / 3.0f);
  int x = (int)ceilf(box[0] / approx), y = (int)ceilf(box[1] / approx);
  *divX = x < 1 ? 1 : x;
  *divY = y < 1 ? 1 : y;
  return BNB_OK;
}

int bnb_create(const bnb_params *p, int replicas, const int *atomCounts, bnb_handle **out) {
  if (!p || !out || replicas < 1 || !atomCounts) return BNB_ERR_ARG;
  if (p->elecMethod < 0 || p->elecMethod > 2 || p->vdwMethod < 0 || p->vdwMethod > 2) return BNB_ERR_ARG;
  if (!(p->rCut > 0) || !(p->rSwitch > 0) || p->rSwitch > p->rCut || p->cullPad < 0) return BNB_ERR_ARG;
  bnb_handle *h = new (std::nothrow) bnb_handle();
  if (!h) return BNB_ERR_ARG;
  h->p = *p;
  h->R = replicas;
  h->atomCount.assign(atomCounts, atomCounts + replicas);
  h->atomStart.resize(replicas + 1);
  h->atomStart[0] = 0;
  for (int r = 0; r < replicas; r++) {
    if (atomCounts[r] < 0) { delete h; return BNB_ERR_ARG; }
    h->atomStart[r + 1] = h->atomStart[r] + atomCounts[r];
  }
  h->N = h->atomStart[replicas];
  h->rep.assign(replicas, RepInfo{});
  for (auto &r : h->rep) { r.divX = -1; r.divY = -1; r.colStart = -1; }
  h->pc = make_const(*p);
  *out = h;
  return BNB_OK;
}

int bnb_destroy(bnb_handle *h) {
  if (!h) return BNB_ERR_ARG;
  free_list(h);
  if (h->topoArena) cudaFree(h->topoArena);
  if (h->pairArena) cudaFree(h->pairArena);
  free_pme(h);
  destroy_events(h);
  delete h;
  return BNB_OK;
}

int bnb_set_topology(bnb_handle *h, const bnb_nbond *nbonds, const int *typeCounts,
                     const bnb_vdw *vdw, const int *lambdaCounts, int exclCount, const int *excl,
                     const int *exclReplica) {
  if (!h || (h->N > 0 && !nbonds) || !typeCounts || !vdw || exclCount < 0 ||
      (exclCount > 0 && !excl) || (exclCount > 0 && h->R > 1 && !exclReplica))
    return BNB_ERR_ARG;
  const int R = h->R, N = h->N;
  std::vector<int> typeStart(R + 1, 0);
  for (int r = 0; r < R; r++) {
    if (typeCounts[r] < 1) return BNB_ERR_ARG;
    typeStart[r + 1] = typeStart[r] + typeCounts[r];
  }
  const int T = typeStart[R];
  h->lamStart.assign(R, 0);
  h->lamCount.assign(R, 1);
  int lam = 0;
  h->alch = 0;
  for (int r = 0; r < R; r++) {
    int c = lambdaCounts ? lambdaCounts[r] : 1;
    if (c < 1) return BNB_ERR_ARG;
    h->lamStart[r] = lam;
    h->lamCount[r] = c;
    if (c > 1) h->alch = 1;
    lam += c;
  }
  if (lam > bnb::kMaxLambdaShared || lam >= 65536) return BNB_ERR_UNSUPPORTED;
  h->lamTotal = lam;

  // Per-atom arrays.
  std::vector<int> atomRep(N), atomType(N), atomSB(N);
  std::vector<float> atomQ(N);
  const float sk = std::sqrt(h->p.kElectric);
  for (int r = 0; r < R; r++)
    for (int a = h->atomStart[r]; a < h->atomStart[r + 1]; a++) {
      const bnb_nbond nb = nbonds[a];
      if (nb.typeIdx < 0 || nb.typeIdx >= typeCounts[r]) return BNB_ERR_ARG;
      atomRep[a] = r;
      atomType[a] = typeStart[r] + nb.typeIdx;
      atomQ[a] = nb.q * sk;
      int blk = nb.siteBlock & 0xFFFF, site = (nb.siteBlock >> 16) & 0xFFFF;
      if (nb.siteBlock == 0) {
        atomSB[a] = 0;
      } else {
        if (blk >= h->lamCount[r] || blk == 0) return BNB_ERR_ARG;
        atomSB[a] = (site << 16) | (h->lamStart[r] + blk);
      }
    }

  // LJ: shared-memory table when small, otherwise per-type combination
  // parameters (requires the table to follow the combination rule of
  // potential.cxx:1393-1403, i.e. no NBFIX overrides).
  h->nTypes = T;
  h->combine = T > bnb::kMaxTableTypes ? 1 : 0;
  std::vector<float2> table, ljType;
  if (!h->combine) {
    table.assign((size_t)T * T, make_float2(0.f, 0.f));
    size_t off = 0;
    for (int r = 0; r < R; r++) {
      int t = typeCounts[r];
      for (int i = 0; i < t; i++)
        for (int j = 0; j < t; j++) {
          bnb_vdw v = vdw[off + (size_t)i * t + j];
          table[(size_t)(typeStart[r] + i) * T + typeStart[r] + j] = make_float2(v.c12, v.c6);
        }
      off += (size_t)t * t;
    }
  } else {
    ljType.resize(T);
    size_t off = 0;
    for (int r = 0; r < R; r++) {
      int t = typeCounts[r];
      std::vector<double> e(t), rh(t);
      for (int i = 0; i < t; i++) {
        bnb_vdw v = vdw[off + (size_t)i * t + i];
        if (v.c6 > 0 && v.c12 > 0) {
          double R6 = 2.0 * v.c12 / v.c6;      // (2 Rmin/2)^6
          e[i] = (double)v.c6 * v.c6 / (4.0 * v.c12);
          rh[i] = 0.5 * std::pow(R6, 1.0 / 6.0);
        } else {
          e[i] = 0;
          rh[i] = 0;
        }
      }
      for (int i = 0; i < t; i++)
        for (int j = 0; j < t; j++) {
          bnb_vdw v = vdw[off + (size_t)i * t + j];
          double eps = std::sqrt(e[i] * e[j]), Rm = rh[i] + rh[j];
          double c6 = 2 * eps * std::pow(Rm, 6), c12 = eps * std::pow(Rm, 12);
          if (std::fabs(c6 - v.c6) > 1e-4 * std::fabs(c6) + 1e-12 ||
              std::fabs(c12 - v.c12) > 1e-4 * std::fabs(c12) + 1e-12)
            return BNB_ERR_UNSUPPORTED;
        }
      for (int i = 0; i < t; i++)
        ljType[typeStart[r] + i] = make_float2((float)std::sqrt(12.0 * e[i]), (float)rh[i]);
      off += (size_t)t * t;
    }
  }

  // Exclusions -> per-atom CSR over global indices (sorted, no duplicates).
  std::vector<std::pair<int, int>> ex;
  ex.reserve(exclCount);
  for (int e = 0; e < exclCount; e++) {
    int r = h->R > 1 ? exclReplica[e] : 0;
    if (r < 0 || r >= R) return BNB_ERR_ARG;
    int a = excl[2 * e], b = excl[2 * e + 1];
    if (a < 0 || b < 0 || a >= h->atomCount[r] || b >= h->atomCount[r]) return BNB_ERR_ARG;
    a += h->atomStart[r];
    b += h->atomStart[r];
    if (a == b) continue;
    ex.emplace_back(a, b);
    ex.emplace_back(b, a);
  }
  std::sort(ex.begin(), ex.end());
  ex.erase(std::unique(ex.begin(), ex.end()), ex.end());
  std::vector<int> exStart(N + 1, 0), exAtom(ex.size());
  for (auto &pr : ex) exStart[pr.first + 1]++;
  for (int a = 0; a < N; a++) exStart[a + 1] += exStart[a];
  for (size_t k = 0; k < ex.size(); k++) exAtom[k] = ex[k].second;
  h->exclTotal = ex.size();

  // Upload into the topology arena.
  if (h->topoArena) cudaFree(h->topoArena);
  h->topoArena = nullptr;
  Arena a;
  size_t o_rep = a.take<RepInfo>(R), o_arep = a.take<int>(N), o_q = a.take<float>(N),
         o_t = a.take<int>(N), o_sb = a.take<int>(N),
         o_tab = a.take<float2>(h->combine ? 1 : (size_t)T * T),
         o_lt = a.take<float2>(h->combine ? T : 1), o_es = a.take<int>(N + 1),
         o_ea = a.take<int>(ex.size()), o_accL = a.take<long long>(lam), o_accE = a.take<long long>(R),
         o_ctr = a.take<bnb::Counters>(1);
  void *base = nullptr;
  if (!ok(cudaMalloc(&base, a.off))) return BNB_ERR_CUDA;
  h->topoArena = base;
  char *b = static_cast<char *>(base);
  Dev &d = h->d;
  d.N = N;
  d.R = R;
  d.nTypes = T;
  d.ljCombine = h->combine;
  d.lamTotal = lam;
  d.rep = (RepInfo *)(b + o_rep);
  d.atomRep = (int *)(b + o_arep);
  d.atomQ = (float *)(b + o_q);
  d.atomType = (int *)(b + o_t);
  d.atomSiteBlock = (int *)(b + o_sb);
  d.ljTable = (float2 *)(b + o_tab);
  d.ljType = (float2 *)(b + o_lt);
  d.exclStart = (int *)(b + o_es);
  d.exclAtom = (int *)(b + o_ea);
  d.accL = (long long *)(b + o_accL);
  d.accE = (long long *)(b + o_accE);
  d.ctr = (bnb::Counters *)(b + o_ctr);
  bool good = ok(cudaMemset(base, 0, a.off));
  auto up = [&](void *dst, const void *src, size_t n) {
    if (n) good = good && ok(cudaMemcpy(dst, src, n, cudaMemcpyHostToDevice));
  };
  up(d.atomRep, atomRep.data(), sizeof(int) * N);
  up(d.atomQ, atomQ.data(), sizeof(float) * N);
  up(d.atomType, atomType.data(), sizeof(int) * N);
  up(d.atomSiteBlock, atomSB.data(), sizeof(int) * N);
  if (!h->combine) up(d.ljTable, table.data(), sizeof(float2) * table.size());
  else up(d.ljType, ljType.data(), sizeof(float2) * ljType.size());
  up(d.exclStart, exStart.data(), sizeof(int) * (N + 1));
  up(d.exclAtom, exAtom.data(), sizeof(int) * exAtom.size());
  if (!good) return BNB_ERR_CUDA;
  h->repDev.clear();  // new device table: upload on the next rebuild
  h->topo = true;
  free_list(h);  // any previous list refers to the old topology
  for (auto &r : h->rep) { r.divX = -1; r.divY = -1; r.colStart = -1; }
  return BNB_OK;
}

// Tail of the work list: the pair kernel's warps take work items in list
// order, and the last item each warp takes decides when it finishes.  Each
// i block's last tailItems * tilesPerWork candidate tiles therefore form
// items of halving size (bnb::work_split) placed after all the full-size
// items, smallest last, so that warps that run out of large items early keep
// taking small ones while the rest finish.  The split depends on the block's
// own candidates only: an i atom's force is summed in FP32 over the tiles of
// one item, so a replica gives the same bits alone and in a batch.
static void set_tail(bnb_handle *h) {
  h->d.tailTiles = h->tailItems * h->tilesPerWork;
}

int bnb_rebuild(bnb_handle *h, const float *position, const float *boxes, void *stream, int flags) {
  if (!h || !boxes || (h->N > 0 && !position)) return BNB_ERR_ARG;
  if (!h->topo) return BNB_ERR_STATE;
  for (int r = 0; r < h->R; r++) {
    float b[3], t[3];
    box_of(h, boxes, r, b, t);
    for (int k = 0; k < 3; k++)  // single-image scheme needs rCut <= half of every brick edge
      if (!(b[k] >= 2 * h->p.rCut) || !std::isfinite(t[k])) return BNB_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const bool async = (flags & BNB_ASYNC) != 0;
  bool changed = layout_columns(h, boxes);
  int mb;
  long long cand, work, mask;
  estimate_capacities(h, mb, cand, work, mask);
  bool need = !h->listArena || mb > h->maxBlocks || h->totalCols != h->d.totalCols || changed ||
              h->reserveDirty;
  if (need) {
    if (async && !h->reserveDirty) return BNB_ERR_STATE;  // sizes change only in a synchronous rebuild
    cudaStreamSynchronize(s);
    h->maxBlocks = std::max(mb, h->maxBlocks);
    h->capCand = h->resTiles > 0 ? h->resTiles
                                 : (int)std::max<long long>(h->capCand, std::min<long long>(cand, kCapLimit));
    h->capWork = h->resWork > 0 ? h->resWork
                                : (int)std::max<long long>(h->capWork, std::min<long long>(work, kCapLimit));
    h->capMask = h->resMasks > 0 ? h->resMasks : (int)std::max<long long>(h->capMask, mask);
    h->reserveDirty = false;
    int rc = alloc_list(h);
    if (rc) return rc;
  }
  int rc = upload_rep(h, s);
  if (rc) return rc;
  const float rcull = h->p.rCut + h->p.cullPad;
  const float rcull2 = rcull * rcull;
  h->d.tilesPerWork = h->tilesPerWork;
  set_tail(h);
  for (int attempt = 0; attempt < 12; attempt++) {
    const bool rec = h->prof && h->rebN < kProfSlots;
    if (rec) cudaEventRecord(h->rebEv[2 * h->rebN], s);
    h->launches += bnb::rebuild_list(h->d, h->colRep_d, position, rcull2, s);
    h->orderPending = true;
    if (rec) cudaEventRecord(h->rebEv[2 * h->rebN++ + 1], s);
    if (!ok(cudaGetLastError())) return BNB_ERR_CUDA;
    if (async) {
      h->listBuilt = true;
      return BNB_OK;
    }
    bnb::Counters c;
    if (!ok(cudaMemcpyAsync(&c, h->d.ctr, sizeof(c), cudaMemcpyDeviceToHost, s))) return BNB_ERR_CUDA;
    if (!ok(cudaStreamSynchronize(s))) return BNB_ERR_CUDA;
    int bad = c.status & bnb::kStatusListInvalid;
    if (!bad) {
      // Keep at least 50 % headroom after a synchronous build, so that the
      // asynchronous rebuilds that follow (graph-captured steps) absorb the
      // drift of the coordinates without overflowing.
      bool grow = false;
      if (3LL * c.candCount > 2LL * h->capCand && h->capCand < kCapLimit) {
        h->capCand = (int)std::min<long long>(2LL * c.candCount + 64, kCapLimit);
        grow = true;
      }
      if (3LL * c.maskCount > 2LL * h->capMask) { h->capMask = 2 * c.maskCount + 64; grow = true; }
      if (3LL * c.workCount > 2LL * h->capWork) { h->capWork = 2 * c.workCount + 64; grow = true; }
      if (!grow) {
        h->listBuilt = true;
        h->lastWork = c.workCount;
        return BNB_OK;
      }
      rc = alloc_list(h);
      if (rc) return rc;
      h->repDev.clear();
      rc = upload_rep(h, s);
      if (rc) return rc;
      continue;
    }
    if (bad & bnb::kStatusBlockOverflow) return BNB_ERR_CAPACITY;  // cannot happen by construction
    // Grow what overflowed by 1.5x (src/domdec/cull.cu:337-375) and retry.
    int needCand = 0;
    if (bad & bnb::kStatusCandOverflow) {
      cudaMemcpy(&needCand, h->d.cullOffset + h->maxBlocks * bnb::kNumShifts, sizeof(int),
                 cudaMemcpyDeviceToHost);
      h->capCand = (int)std::min<long long>((long long)std::max(needCand, h->capCand) * 3 / 2, kCapLimit);
      h->capWork = std::max(h->capWork, h->capCand / bnb::kMinTilesPerWork + h->maxBlocks + 16);
    }
    if (bad & bnb::kStatusMaskOverflow) {
      int needMask = 0;
      cudaMemcpy(&needMask, h->d.candMaskOff + h->d.capCand, sizeof(int), cudaMemcpyDeviceToHost);
      h->capMask = std::max(needMask, h->capMask) * 3 / 2 + 64;
    }
    if (bad & bnb::kStatusWorkOverflow) h->capWork = h->capWork * 3 / 2 + 64;
    rc = alloc_list(h);
    if (rc) return rc;
    rc = upload_rep(h, s);
    if (rc) return rc;
  }
  return BNB_ERR_CAPACITY;
}

int bnb_compute(bnb_handle *h, const float *position, const float *lambda, const float *boxes,
                int calcEnergy, const bnb_outputs *out, void *stream) {
  if (!h || !out || !boxes || (h->N > 0 && !position) || !flags_ok(calcEnergy)) return BNB_ERR_ARG;
  if (!h->listBuilt) return BNB_ERR_STATE;
  if (h->alch && !lambda) return BNB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const bool boxChanged = store_boxes(h, boxes);
  if (boxChanged) {
    int rc = upload_rep(h, s);
    if (rc) return rc;
  }
  if (h->counting) cudaMemsetAsync(&h->d.ctr->pairCount, 0, sizeof(unsigned long long), s);
  bnb::pack_positions(h->d, position, s);
  int alch = h->alch ? (h->p.useSoftCore ? 2 : 1) : 0;
  int work = h->lastWork > 0 ? h->lastWork : h->capWork;
  if (h->smCount == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&h->smCount, cudaDevAttrMultiProcessorCount, dev);
  }
  int grid = (work + 7) / 8;  // at most one work item per warp in the first round
  const int cap = h->ctasPerSM > 0 ? h->ctasPerSM * h->smCount : 8 * h->smCount;
  grid = std::max(1, std::min(grid, cap));
  const bool rec = h->prof && h->pairN < kProfSlots;
  if (rec) cudaEventRecord(h->pairEv[2 * h->pairN], s);
  int rc = bnb::launch_pair(h->d, h->pc, lambda, h->p.elecMethod, h->p.vdwMethod, alch,
                            (calcEnergy & 1) != 0, h->counting, grid, s);
  if (rec) cudaEventRecord(h->pairEv[2 * h->pairN++ + 1], s);
  if (rc) return rc;
  bnb::launch_finalize(h->d, *out, out_mode(calcEnergy), s);
  if (h->orderPending) {  // the costs of this launch order the items of the next ones
    bnb::launch_order(h->d, s);
    h->orderPending = false;
    h->launches += 1;
  }
  h->launches += 3;
  return ok(cudaGetLastError()) ? BNB_OK : BNB_ERR_CUDA;
}

int bnb_profile(bnb_handle *h, int enable) {
  if (!h) return BNB_ERR_ARG;
  if (enable && h->pairEv.empty()) {
    h->pairEv.resize(2 * kProfSlots);
    h->rebEv.resize(2 * kProfSlots);
    for (auto &e : h->pairEv)
      if (!ok(cudaEventCreate(&e))) return BNB_ERR_CUDA;
    for (auto &e : h->rebEv)
      if (!ok(cudaEventCreate(&e))) return BNB_ERR_CUDA;
  }
  h->prof = enable != 0;
  h->pairN = h->rebN = 0;
  return BNB_OK;
}

int bnb_profile_read(bnb_handle *h, double *pairMs, int *pairLaunches, double *rebuildMs,
                     int *rebuilds, unsigned long long *kernelLaunches, int reset) {
  if (!h) return BNB_ERR_ARG;
  double pm = 0, rm = 0;
  for (int i = 0; i < h->pairN; i++) {
    float ms = 0;
    if (!ok(cudaEventSynchronize(h->pairEv[2 * i + 1])) ||
        !ok(cudaEventElapsedTime(&ms, h->pairEv[2 * i], h->pairEv[2 * i + 1])))
      return BNB_ERR_CUDA;
    pm += ms;
  }
  for (int i = 0; i < h->rebN; i++) {
    float ms = 0;
    if (!ok(cudaEventSynchronize(h->rebEv[2 * i + 1])) ||
        !ok(cudaEventElapsedTime(&ms, h->rebEv[2 * i], h->rebEv[2 * i + 1])))
      return BNB_ERR_CUDA;
    rm += ms;
  }
  if (pairMs) *pairMs = pm;
  if (pairLaunches) *pairLaunches = h->pairN;
  if (rebuildMs) *rebuildMs = rm;
  if (rebuilds) *rebuilds = h->rebN;
  if (kernelLaunches) *kernelLaunches = h->launches;
  if (reset) {
    h->pairN = h->rebN = 0;
    h->launches = 0;
  }
  return BNB_OK;
}

int bnb_set_tuning(bnb_handle *h, int tilesPerWork, int ctasPerSM, int tailItems) {
  if (!h || tilesPerWork < bnb::kMinTilesPerWork || tilesPerWork > 32 || ctasPerSM < 0 || ctasPerSM > 8 ||
      tailItems < 0 || tailItems > 8)
    return BNB_ERR_ARG;
  // work items must be rebuilt
  if (tilesPerWork != h->tilesPerWork || tailItems != h->tailItems) h->listBuilt = false;
  h->tilesPerWork = tilesPerWork;
  h->ctasPerSM = ctasPerSM;
  h->tailItems = tailItems;
  return BNB_OK;
}

int bnb_get_tuning(bnb_handle *h, int *tilesPerWork, int *ctasPerSM, int *tailItems) {
  if (!h) return BNB_ERR_ARG;
  if (tilesPerWork) *tilesPerWork = h->tilesPerWork;
  if (ctasPerSM) *ctasPerSM = h->ctasPerSM;
  if (tailItems) *tailItems = h->tailItems;
  return BNB_OK;
}

// Tries tiles-per-work-item x CTAs-per-SM x tail settings on the caller's
// system and keeps the fastest pair-kernel time (CUDA events, median of
// `reps`).
int bnb_autotune(bnb_handle *h, const float *position, const float *lambda, const float *boxes,
                 int reps, void *stream, float *bestMs) {
  if (!h || !boxes || (h->N > 0 && !position) || reps < 1) return BNB_ERR_ARG;
  if (!h->topo) return BNB_ERR_STATE;
  cudaStream_t s = (cudaStream_t)stream;
  static const int kTiles[] = {1, 2, 4, 8, 16, 32};
  static const int kCtas[] = {0, 2, 3};
  static const int kTails[] = {bnb::kTailItems, 0};
  bnb_outputs none;
  memset(&none, 0, sizeof(none));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int bt = h->tilesPerWork, bc = h->ctasPerSM, bl = h->tailItems;
  for (int l : kTails)
  for (int t : kTiles) {
    for (int c : kCtas) {
      int rc = bnb_set_tuning(h, t, c, l);
      if (!rc) rc = bnb_rebuild(h, position, boxes, stream, 0);
      if (rc) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
      std::vector<float> ms;
      for (int k = 0; k < reps + 2; k++) {
        cudaEventRecord(e0, s);
        rc = bnb_compute(h, position, lambda, boxes, 0, &none, stream);
        cudaEventRecord(e1, s);
        if (rc) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
        cudaEventSynchronize(e1);
        float t_ms = 0;
        cudaEventElapsedTime(&t_ms, e0, e1);
        if (k >= 2) ms.push_back(t_ms);
      }
      std::sort(ms.begin(), ms.end());
      float med = ms[ms.size() / 2];
      if (med < best) { best = med; bt = t; bc = c; bl = l; }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int rc = bnb_set_tuning(h, bt, bc, bl);
  if (!rc) rc = bnb_rebuild(h, position, boxes, stream, 0);
  if (bestMs) *bestMs = best;
  return rc;
}

int bnb_reserve(bnb_handle *h, int tiles, int masks, int work) {
  if (!h) return BNB_ERR_ARG;
  h->resTiles = tiles > 0 ? tiles : 0;
  h->resMasks = masks > 0 ? masks : 0;
  h->resWork = work > 0 ? work : 0;
  h->reserveDirty = true;
  return BNB_OK;
}

int bnb_status(bnb_handle *h, void *stream, int clear, int *status) {
  if (!h || !status) return BNB_ERR_ARG;
  if (!h->topo) { *status = 0; return BNB_OK; }
  cudaStream_t s = (cudaStream_t)stream;
  int v = 0;
  if (!ok(cudaMemcpyAsync(&v, &h->d.ctr->status, sizeof(int), cudaMemcpyDeviceToHost, s)) ||
      !ok(cudaStreamSynchronize(s)))
    return BNB_ERR_CUDA;
  if (clear) cudaMemsetAsync(&h->d.ctr->status, 0, sizeof(int), s);
  *status = v;
  return BNB_OK;
}

int bnb_list_sizes(bnb_handle *h, void *stream, int *blocks, int *tiles, int *masks, int *work) {
  if (!h) return BNB_ERR_ARG;
  if (!h->listBuilt) return BNB_ERR_STATE;
  bnb::Counters c;
  cudaStream_t s = (cudaStream_t)stream;
  if (!ok(cudaMemcpyAsync(&c, h->d.ctr, sizeof(c), cudaMemcpyDeviceToHost, s)) ||
      !ok(cudaStreamSynchronize(s)))
    return BNB_ERR_CUDA;
  if (blocks) *blocks = c.blockCount;
  if (tiles) *tiles = c.candCount;
  if (masks) *masks = c.maskCount;
  if (work) *work = c.workCount;
  return BNB_OK;
}

int bnb_get_list(bnb_handle *h, void *stream, int *wrap, int *blockBounds, int *sortedAtom,
                 int *slotAtom, float *bmin, float *bmax, int *candStart, int *cand, int *candMask,
                 uint32_t *masks) {
  int B, T, M, W;
  int rc = bnb_list_sizes(h, stream, &B, &T, &M, &W);
  if (rc) return rc;
  const Dev &d = h->d;
  bool good = true;
  auto dn = [&](void *dst, const void *src, size_t n) {
    if (dst && n) good = good && ok(cudaMemcpy(dst, src, n, cudaMemcpyDeviceToHost));
  };
  dn(wrap, d.wrap, sizeof(int) * h->N);
  dn(blockBounds, d.blockBounds, sizeof(int) * (B + 1));
  dn(sortedAtom, d.sortedAtom, sizeof(int) * h->N);
  dn(slotAtom, d.slotAtom, sizeof(int) * 32 * B);
  if (bmin || bmax) {
    std::vector<float4> t(B > 0 ? B : 1);
    if (bmin) {
      dn(t.data(), d.bmin, sizeof(float4) * B);
      for (int b = 0; b < B; b++) { bmin[3 * b] = t[b].x; bmin[3 * b + 1] = t[b].y; bmin[3 * b + 2] = t[b].z; }
    }
    if (bmax) {
      dn(t.data(), d.bmax, sizeof(float4) * B);
      for (int b = 0; b < B; b++) { bmax[3 * b] = t[b].x; bmax[3 * b + 1] = t[b].y; bmax[3 * b + 2] = t[b].z; }
    }
  }
  dn(candStart, d.candStart, sizeof(int) * (B + 1));
  if (cand || candMask) {
    std::vector<int4> t(T > 0 ? T : 1);
    dn(t.data(), d.cand, sizeof(int4) * T);
    for (int c = 0; c < T; c++) {
      if (cand) { cand[2 * c] = t[c].x; cand[2 * c + 1] = t[c].y; }
      if (candMask) candMask[c] = t[c].z;
    }
  }
  dn(masks, d.masks, sizeof(uint32_t) * 32 * (size_t)M);
  return good ? BNB_OK : BNB_ERR_CUDA;
}

int bnb_set_counting(bnb_handle *h, int enable) {
  if (!h) return BNB_ERR_ARG;
  h->counting = enable != 0;
  return BNB_OK;
}

int bnb_pair_count(bnb_handle *h, void *stream, unsigned long long *pairs) {
  if (!h || !pairs) return BNB_ERR_ARG;
  if (!h->topo) return BNB_ERR_STATE;
  cudaStream_t s = (cudaStream_t)stream;
  if (!ok(cudaMemcpyAsync(pairs, &h->d.ctr->pairCount, sizeof(*pairs), cudaMemcpyDeviceToHost, s)) ||
      !ok(cudaStreamSynchronize(s)))
    return BNB_ERR_CUDA;
  return BNB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// bnb_nbdirect_noalloc: the all-pairs variant of the pair kernel for one small
// system, for callers that may not allocate device memory at all -- not even
// once, to create a handle.  Examples: an engine that has handed all of the
// device's memory to its own pool before it loads this library, or a caller
// that steps while other streams run and cannot accept the device-wide
// synchronisation that cudaMalloc and cudaFree may bring.  The kernel's only
// scratch, its fixed-point accumulators, is the fixed array below; every
// other buffer is the caller's.
// ---------------------------------------------------------------------------
namespace {
// [3 * BNB_NOALLOC_MAX_ATOMS] dU/dx component planes, then the energy (and
// padding): about 98 KB, held by every device that loads this library until
// the process exits.
constexpr int kNoallocScratch = 3 * BNB_NOALLOC_MAX_ATOMS + 32;
constexpr int kNoallocDevices = 64;
long long *g_noallocPtr[kNoallocDevices];  // device address of the array, per device
std::mutex g_noallocLock;
}  // namespace

static __device__ __align__(256) long long g_noallocScratch[kNoallocScratch];

namespace {
// Set-up, once per device, with that device current.  In host code the name
// g_noallocScratch is only a host-side stand-in for the device array, never
// an address a kernel may use; the device address comes from
// cudaGetSymbolAddress and is cached per device.
int noalloc_scratch(long long **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return BNB_ERR_CUDA;
  if (dev < 0 || dev >= kNoallocDevices) return BNB_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_noallocLock);
  if (!g_noallocPtr[dev]) {
    long long *p = nullptr;
    if (cudaGetSymbolAddress((void **)&p, g_noallocScratch) != cudaSuccess || !p) return BNB_ERR_CUDA;
    g_noallocPtr[dev] = p;
  }
  *out = g_noallocPtr[dev];
  return BNB_OK;
}
}  // namespace

extern "C" int bnb_nbdirect_noalloc(const bnb_params *p, int atomCount, const float *position,
                                    const float *box, const bnb_nbond *nbonds, int typeCount,
                                    const bnb_vdw *vdw, const int *exclStart, const int *exclAtom,
                                    int calcEnergy, const bnb_outputs *out, void *stream) {
  if (!p || !box || !out || atomCount < 0 || typeCount < 0) return BNB_ERR_ARG;
  if (atomCount > BNB_NOALLOC_MAX_ATOMS) return BNB_ERR_TOO_LARGE;
  if (atomCount > 0 && (!position || !nbonds || !vdw || typeCount < 1 || !exclStart || !exclAtom))
    return BNB_ERR_ARG;
  if (p->elecMethod < 0 || p->elecMethod > 2 || p->vdwMethod < 0 || p->vdwMethod > 2) return BNB_ERR_ARG;
  if (!(p->rCut > 0) || !(p->rSwitch > 0) || p->rSwitch > p->rCut) return BNB_ERR_ARG;
  for (int k = 0; k < 3; k++)  // minimum image: one image of each pair inside the cutoff
    if (!(box[k] > 0) || 2.0f * p->rCut > box[k]) return BNB_ERR_ARG;
  long long *scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  // The array keeps whatever the last call left; clear the part this call
  // accumulates into (three planes of atomCount entries and the energy).
  for (int k = 0; k < 3; k++)
    if (atomCount > 0 &&
        cudaMemsetAsync(scratch + (size_t)k * BNB_NOALLOC_MAX_ATOMS, 0, sizeof(long long) * atomCount, s) !=
            cudaSuccess)
      return BNB_ERR_CUDA;
  if (cudaMemsetAsync(scratch + 3 * BNB_NOALLOC_MAX_ATOMS, 0, sizeof(long long), s) != cudaSuccess)
    return BNB_ERR_CUDA;
  bnb::AllPairsArgs a{};
  a.pc = make_const(*p);
  a.N = atomCount;
  a.nTypes = typeCount;
  a.stride = BNB_NOALLOC_MAX_ATOMS;
  a.sqrtK = std::sqrt(p->kElectric);
  a.box = make_float3(box[0], box[1], box[2]);
  a.boxInv = make_float3(1.0f / box[0], 1.0f / box[1], 1.0f / box[2]);
  a.x = position;
  a.nb = nbonds;
  a.vdw = vdw;
  a.exclStart = exclStart;
  a.exclAtom = exclAtom;
  a.accF = scratch;
  a.accE = scratch + 3 * BNB_NOALLOC_MAX_ATOMS;
  return bnb::launch_allpairs(a, *out, p->elecMethod, p->vdwMethod, calcEnergy != 0, s);
}

// ---------------------------------------------------------------------------
// nb14 / nbex pair lists (getforce_nb14 / getforce_nbex, src/bonded/pair.cu)
// ---------------------------------------------------------------------------
namespace {
int pairs_boxes(bnb_handle *h, const float *boxes, cudaStream_t s) {
  return store_boxes(h, boxes) ? upload_rep(h, s) : BNB_OK;
}

bnb::PairsArgs pairs_args(bnb_handle *h, const float *position, const float *lambda) {
  bnb::PairsArgs a{};
  a.N = h->N;
  a.R = h->R;
  a.lamTotal = h->lamTotal;
  a.n14 = h->n14;
  a.nex = h->nex;
  a.rCut = h->p.rCut;
  a.rSwitch = h->p.rSwitch;
  a.beta = h->p.betaEwald;
  a.kElectric = h->p.kElectric;
  a.softR = h->p.softCoreRadius;
  a.x = position;
  a.lambda = lambda;
  a.atomRep = h->d.atomRep;
  a.rep = h->d.rep;
  a.nb14 = h->nb14_d;
  a.nbex = h->nbex_d;
  a.accF = h->accP;
  a.accL = h->accPL;
  a.accE = h->accPE;
  return a;
}
}  // namespace

extern "C" int bnb_set_pairs(bnb_handle *h, int nb14Count, const bnb_nb14 *nb14, int nbexCount,
                             const bnb_nbex *nbex, int useSoftCore14) {
  if (!h || nb14Count < 0 || nbexCount < 0 || (nb14Count && !nb14) || (nbexCount && !nbex)) return BNB_ERR_ARG;
  if (!h->topo) return BNB_ERR_STATE;
  std::vector<int> atomRep(h->N);
  for (int r = 0; r < h->R; r++)
    for (int i = h->atomStart[r]; i < h->atomStart[r + 1]; i++) atomRep[i] = r;
  auto okPair = [&](const int idx[2], const int sb[2]) {
    if (idx[0] < 0 || idx[0] >= h->N || idx[1] < 0 || idx[1] >= h->N) return false;
    if (atomRep[idx[0]] != atomRep[idx[1]]) return false;
    for (int k = 0; k < 2; k++)
      if ((sb[k] & 0xFFFF) >= h->lamTotal) return false;
    return true;
  };
  for (int t = 0; t < nb14Count; t++)
    if (!okPair(nb14[t].idx, nb14[t].siteBlock)) return BNB_ERR_ARG;
  for (int t = 0; t < nbexCount; t++)
    if (!okPair(nbex[t].idx, nbex[t].siteBlock)) return BNB_ERR_ARG;
  if (h->pairArena) cudaFree(h->pairArena);
  h->pairArena = nullptr;
  Arena a;
  size_t o14 = a.take<bnb_nb14>(std::max(nb14Count, 1)), oex = a.take<bnb_nbex>(std::max(nbexCount, 1)),
         of = a.take<long long>(3 * (size_t)std::max(h->N, 1)), ol = a.take<long long>(std::max(h->lamTotal, 1)),
         oe = a.take<long long>(std::max(h->R, 1));
  void *base = nullptr;
  if (!ok(cudaMalloc(&base, a.off))) return BNB_ERR_CUDA;
  h->pairArena = base;
  char *b = static_cast<char *>(base);
  h->nb14_d = (bnb_nb14 *)(b + o14);
  h->nbex_d = (bnb_nbex *)(b + oex);
  h->accP = (long long *)(b + of);
  h->accPL = (long long *)(b + ol);
  h->accPE = (long long *)(b + oe);
  if (!ok(cudaMemset(base, 0, a.off))) return BNB_ERR_CUDA;
  if (nb14Count && !ok(cudaMemcpy(h->nb14_d, nb14, sizeof(bnb_nb14) * nb14Count, cudaMemcpyHostToDevice)))
    return BNB_ERR_CUDA;
  if (nbexCount && !ok(cudaMemcpy(h->nbex_d, nbex, sizeof(bnb_nbex) * nbexCount, cudaMemcpyHostToDevice)))
    return BNB_ERR_CUDA;
  h->n14 = nb14Count;
  h->nex = nbexCount;
  h->soft14 = useSoftCore14 != 0;
  return BNB_OK;
}

extern "C" int bnb_compute_nb14(bnb_handle *h, const float *position, const float *lambda, const float *boxes,
                                int calcEnergy, const bnb_outputs *out, void *stream) {
  if (!h || !out || !boxes || (h->N > 0 && !position) || !flags_ok(calcEnergy)) return BNB_ERR_ARG;
  if (!h->pairArena) return BNB_ERR_STATE;
  if (h->alch && !lambda) return BNB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  int rc = pairs_boxes(h, boxes, s);
  if (rc) return rc;
  bnb::PairsArgs a = pairs_args(h, position, lambda);
  a.mode = out_mode(calcEnergy);
  return bnb::launch_nb14(a, *out, h->p.elecMethod, h->p.vdwMethod, h->soft14 && h->alch, (calcEnergy & 1) != 0, s);
}

extern "C" int bnb_compute_nbex(bnb_handle *h, const float *position, const float *lambda, const float *boxes,
                                int calcEnergy, const bnb_outputs *out, void *stream) {
  if (!h || !out || !boxes || (h->N > 0 && !position) || !flags_ok(calcEnergy)) return BNB_ERR_ARG;
  if (!h->pairArena) return BNB_ERR_STATE;
  if (h->alch && !lambda) return BNB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  int rc = pairs_boxes(h, boxes, s);
  if (rc) return rc;
  bnb::PairsArgs a = pairs_args(h, position, lambda);
  if (h->p.elecMethod != 1) a.nex = 0;  // the correction exists for PME only (pair.cu:379)
  a.mode = out_mode(calcEnergy);
  return bnb::launch_nbex(a, *out, (calcEnergy & 1) != 0, s);
}


// ---------------------------------------------------------------------------
// PME reciprocal space and Ewald self term (getforce_ewald /
// getforce_ewaldself, src/nbrecip/nbrecip.cu:19-555); grid sizes and B-spline
// moduli as Potential::initialize (src/system/potential.cxx:1202-1300).
// ---------------------------------------------------------------------------
namespace {
constexpr int kPmePad = 64;  // grid offsets in multiples of 64 elements

// The reference's grid rule: the smallest of j*{32,27,24,20,18} above
// L/spacing, with j the power of two that puts L/spacing in [16j, 32j).
int pme_grid_size(float L, float spacing) {
  static const int good[] = {32, 27, 24, 20, 18, 16};
  const float md = L / spacing;
  int j = 1;
  while (md >= 32.0f * j) j *= 2;
  int k = 0;
  while (k < 5 && md < (float)(j * good[k])) k++;
  return j * good[k - 1];
}

// 1/|b(m)|^2, b(m) = sum_{l=1}^{n-1} M_n(l) exp(2 pi i m l / K), m = 0..count-1.
void pme_moduli(int K, int order, int count, float *out) {
  double M[12] = {0};
  M[1] = 1.0;  // M_2 at the integers 0, 1, 2
  for (int k = 3; k <= order; k++) {
    double nw[12] = {0};
    for (int l = 0; l <= k; l++) nw[l] = (l * M[l] + (k - l) * (l >= 1 ? M[l - 1] : 0.0)) / (k - 1);
    for (int l = 0; l < 12; l++) M[l] = nw[l];
  }
  const double tau = 6.283185307179586476925;
  for (int m = 0; m < count; m++) {
    double re = 0.0, im = 0.0;
    for (int l = 1; l < order; l++) {
      re += M[l] * std::cos(tau * m * l / K);
      im += M[l] * std::sin(tau * m * l / K);
    }
    out[m] = (float)(1.0 / (re * re + im * im));
  }
}

inline long long pad_to(long long n) { return (n + kPmePad - 1) / kPmePad * kPmePad; }

bnb::PmeArgs pme_args(bnb_handle *h, const float *position, const float *lambda) {
  bnb::PmeArgs a{};
  a.N = h->N;
  a.R = h->R;
  a.lamTotal = h->lamTotal;
  a.order = h->pmeOrder;
  a.totalGrid = h->pmeTotalGrid;
  a.totalCplx = h->pmeTotalCplx;
  a.beta = h->p.betaEwald;
  a.x = position;
  a.lambda = lambda;
  a.q = h->d.atomQ;
  a.siteBlock = h->d.atomSiteBlock;
  a.atomRep = h->d.atomRep;
  a.rep = h->d.rep;
  a.prep = h->pmeRep_d;
  a.maxCplx = h->pmeMaxCplx;
  a.mod = h->pmeMod_d;
  a.qfix = h->pmeFix_d;
  a.grid = h->pmeGrid_d;
  a.cplx = h->pmeCplx_d;
  a.accL = h->pmeAccL;
  a.accE = h->pmeAccE;
  a.done = h->pmeDone;
  a.tric = h->triclinic;
  return a;
}
}  // namespace

extern "C" int bnb_set_pme(bnb_handle *h, int order, float gridSpace, const int *grid, const float *boxes) {
  if (!h || !boxes || (order != 4 && order != 6 && order != 8) || (!grid && !(gridSpace > 0.f)))
    return BNB_ERR_ARG;
  if (!h->topo) return BNB_ERR_STATE;
  const int R = h->R;
  std::vector<bnb::PmeRep> pr(R);
  for (int r = 0; r < R; r++) {
    // grid sizes from the edge lengths |A|, |B|, |C| (potential.cxx:1206, box.a)
    float b[3], t[3];
    box_of(h, boxes, r, b, t);
    const double len[3] = {(double)b[0], std::sqrt((double)t[0] * t[0] + (double)b[1] * b[1]),
                           std::sqrt((double)t[1] * t[1] + (double)t[2] * t[2] + (double)b[2] * b[2])};
    for (int k = 0; k < 3; k++) {
      if (!(b[k] > 0.f) || !std::isfinite(len[k])) return BNB_ERR_ARG;
      const int K = grid ? grid[3 * r + k] : pme_grid_size((float)len[k], gridSpace);
      if (K < order || K > 4096) return BNB_ERR_ARG;
      pr[r].K[k] = K;
    }
  }
  // Grids are laid out grouped by size (stable in replica order), so every
  // set of equal grids is one batched FFT plan.
  std::vector<int> layout(R);
  for (int r = 0; r < R; r++) layout[r] = r;
  auto key = [&](int r) { return std::make_tuple(pr[r].K[0], pr[r].K[1], pr[r].K[2]); };
  std::stable_sort(layout.begin(), layout.end(), [&](int x, int y) { return key(x) < key(y); });
  long long gOff = 0, cOff = 0, mOff = 0;
  for (int r : layout) {
    pr[r].gridOff = (int)gOff;
    pr[r].cplxOff = (int)cOff;
    pr[r].modOff = (int)mOff;
    gOff += pad_to((long long)pr[r].K[0] * pr[r].K[1] * pr[r].K[2]);
    cOff += pad_to((long long)pr[r].K[0] * pr[r].K[1] * (pr[r].K[2] / 2 + 1));
    mOff += pr[r].K[0] + pr[r].K[1] + pr[r].K[2] / 2 + 1;
    if (gOff > (1LL << 30) || cOff > (1LL << 30)) return BNB_ERR_TOO_LARGE;
  }
  free_pme(h);
  Arena a;
  size_t oRep = a.take<bnb::PmeRep>(std::max(R, 1)), oMod = a.take<float>(mOff), oFix = a.take<long long>(gOff),
         oGrid = a.take<float>(gOff), oCplx = a.take<float2>(cOff), oL = a.take<long long>(std::max(h->lamTotal, 1)),
         oE = a.take<long long>(std::max(R, 1)), oDone = a.take<unsigned int>(1);
  void *base = nullptr;
  if (!ok(cudaMalloc(&base, a.off))) return BNB_ERR_CUDA;
  h->pmeArena = base;
  char *b = static_cast<char *>(base);
  h->pmeRep_d = (bnb::PmeRep *)(b + oRep);
  h->pmeMod_d = (float *)(b + oMod);
  h->pmeFix_d = (long long *)(b + oFix);
  h->pmeGrid_d = (float *)(b + oGrid);
  h->pmeCplx_d = (float2 *)(b + oCplx);
  h->pmeAccL = (long long *)(b + oL);
  h->pmeAccE = (long long *)(b + oE);
  h->pmeDone = (unsigned int *)(b + oDone);
  std::vector<float> mod(mOff);
  for (int r = 0; r < R; r++) {
    float *m = mod.data() + pr[r].modOff;
    pme_moduli(pr[r].K[0], order, pr[r].K[0], m);
    pme_moduli(pr[r].K[1], order, pr[r].K[1], m + pr[r].K[0]);
    pme_moduli(pr[r].K[2], order, pr[r].K[2] / 2 + 1, m + pr[r].K[0] + pr[r].K[1]);
  }
  if (!ok(cudaMemset(base, 0, a.off)) ||
      !ok(cudaMemcpy(h->pmeRep_d, pr.data(), sizeof(bnb::PmeRep) * R, cudaMemcpyHostToDevice)) ||
      !ok(cudaMemcpy(h->pmeMod_d, mod.data(), sizeof(float) * mOff, cudaMemcpyHostToDevice))) {
    free_pme(h);
    return BNB_ERR_CUDA;
  }
  // one batched plan pair per set of equal grids (contiguous in the layout)
  for (int i = 0; i < R;) {
    const int r = layout[i];
    int e = i + 1;
    while (e < R && key(layout[e]) == key(r)) e++;
    int n[3] = {pr[r].K[0], pr[r].K[1], pr[r].K[2]};
    int nc[3] = {pr[r].K[0], pr[r].K[1], pr[r].K[2] / 2 + 1};
    const int dr = (int)pad_to((long long)n[0] * n[1] * n[2]);
    const int dc = (int)pad_to((long long)nc[0] * nc[1] * nc[2]);
    bnb_handle::PmePlan p{};
    p.first = r;
    p.count = e - i;
    if (cufftPlanMany(&p.r2c, 3, n, n, 1, dr, nc, 1, dc, CUFFT_R2C, p.count) != CUFFT_SUCCESS) {
      free_pme(h);
      return BNB_ERR_CUDA;
    }
    if (cufftPlanMany(&p.c2r, 3, n, nc, 1, dc, n, 1, dr, CUFFT_C2R, p.count) != CUFFT_SUCCESS) {
      cufftDestroy(p.r2c);
      free_pme(h);
      return BNB_ERR_CUDA;
    }
    h->pmePlans.push_back(p);
    i = e;
  }
  h->pmeRep = pr;
  h->pmeOrder = order;
  h->pmeTotalGrid = (int)gOff;
  h->pmeTotalCplx = (int)cOff;
  h->pmeMaxCplx = 0;
  for (int r = 0; r < R; r++)
    h->pmeMaxCplx = std::max(h->pmeMaxCplx, pr[r].K[0] * pr[r].K[1] * (pr[r].K[2] / 2 + 1));
  return BNB_OK;
}

extern "C" int bnb_pme_grid(bnb_handle *h, int replica, int *K) {
  if (!h || !K || replica < 0 || replica >= h->R) return BNB_ERR_ARG;
  if (!h->pmeOrder) return BNB_ERR_STATE;
  for (int k = 0; k < 3; k++) K[k] = h->pmeRep[replica].K[k];
  return BNB_OK;
}

extern "C" int bnb_compute_pme(bnb_handle *h, const float *position, const float *lambda, const float *boxes,
                               int calcEnergy, const bnb_outputs *out, void *stream) {
  if (!h || !out || !boxes || (h->N > 0 && !position) || !flags_ok(calcEnergy)) return BNB_ERR_ARG;
  if (!h->pmeOrder) return BNB_ERR_STATE;
  if (h->alch && !lambda) return BNB_ERR_ARG;
  if (h->p.elecMethod != 1) return BNB_OK;  // reciprocal space exists for PME only (nbrecip.cu:486)
  cudaStream_t s = (cudaStream_t)stream;
  int rc = pairs_boxes(h, boxes, s);
  if (rc) return rc;
  bnb::PmeArgs a = pme_args(h, position, lambda);
  a.mode = out_mode(calcEnergy);
  if ((rc = bnb::pme_spread(a, s))) return rc;
  for (auto &p : h->pmePlans) {
    const bnb::PmeRep &f = h->pmeRep[p.first];
    if (cufftSetStream(p.r2c, s) != CUFFT_SUCCESS ||
        cufftExecR2C(p.r2c, h->pmeGrid_d + f.gridOff, reinterpret_cast<cufftComplex *>(h->pmeCplx_d + f.cplxOff)) !=
            CUFFT_SUCCESS)
      return BNB_ERR_CUDA;
  }
  if ((rc = bnb::pme_convolve(a, s))) return rc;
  for (auto &p : h->pmePlans) {
    const bnb::PmeRep &f = h->pmeRep[p.first];
    if (cufftSetStream(p.c2r, s) != CUFFT_SUCCESS ||
        cufftExecC2R(p.c2r, reinterpret_cast<cufftComplex *>(h->pmeCplx_d + f.cplxOff), h->pmeGrid_d + f.gridOff) !=
            CUFFT_SUCCESS)
      return BNB_ERR_CUDA;
  }
  h->launches += 4;
  return bnb::pme_gather(a, *out, (calcEnergy & 1) != 0, s);
}

extern "C" int bnb_compute_ewald_self(bnb_handle *h, const float *lambda, int calcEnergy, const bnb_outputs *out,
                                      void *stream) {
  if (!h || !out || !flags_ok(calcEnergy)) return BNB_ERR_ARG;
  if (!h->pmeOrder) return BNB_ERR_STATE;
  if (h->alch && !lambda) return BNB_ERR_ARG;
  if (h->p.elecMethod != 1) return BNB_OK;  // nbrecip.cu:64
  bnb::PmeArgs a = pme_args(h, nullptr, lambda);
  a.mode = out_mode(calcEnergy);
  h->launches += 1;
  return bnb::pme_self(a, *out, (calcEnergy & 1) != 0, (cudaStream_t)stream);
}
