// Internal device-side layout of libbnb (not part of the public C ABI).
//
// One handle holds R >= 1 independent systems ("replicas").  Atoms, columns,
// blocks, candidate tiles and lambda blocks of all replicas are concatenated;
// no block or tile ever spans two replicas.  A single system is the R == 1
// case, so the plain and batched paths run the same kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "bnb.h"
#include "work_split.h"

#include <utility>

namespace bnb {

constexpr int kNumShifts = 14;        // own image + 13 half-shell images
constexpr int kExclBlk = 16;          // exclusion-partner blocks listed per block
constexpr int kTilesPerWork = 8;      // default candidate tiles per pair-kernel work item
constexpr int kMinTilesPerWork = 1;   // smallest setting (sizes the work-item capacity)
constexpr int kTailItems = 2;         // full-size items' worth of tiles per i block in the tail levels
constexpr int kMaxTableTypes = 64;    // LJ table kept in shared memory up to 64 types
constexpr int kMaxLambdaShared = 2048;
constexpr int kSortCap = 4096;        // column sort in shared memory up to 4096 atoms
constexpr double kFixScale = 4294967296.0;      // 2^32 fixed-point units per kcal/mol(/A)
constexpr float kFixScaleF = 4294967296.0f;

// Status bits written by the device (bnb_status).
enum : int {
  kStatusBlockOverflow = BNB_STATUS_BLOCK_OVERFLOW,
  kStatusCandOverflow = BNB_STATUS_TILE_OVERFLOW,
  kStatusMaskOverflow = BNB_STATUS_MASK_OVERFLOW,
  kStatusWorkOverflow = BNB_STATUS_WORK_OVERFLOW,
  kStatusNonFinite = BNB_STATUS_NONFINITE,
  kStatusListInvalid = BNB_STATUS_BLOCK_OVERFLOW | BNB_STATUS_TILE_OVERFLOW |
                       BNB_STATUS_MASK_OVERFLOW | BNB_STATUS_WORK_OVERFLOW,
};

// Output modes (BNB_OUT_SET / BNB_OUT_ADD64 of the public header).
__device__ __forceinline__ void out64(double *p, double v, int mode) {
  if (mode & BNB_OUT_ADD64) *p += v;
  else *p = v;
}
__device__ __forceinline__ void out32(float *p, float v, int mode) {  // atomic unless overwriting
  if (mode & BNB_OUT_SET) *p = v;
  else if (v != 0.f) atomicAdd(p, v);
}
__device__ __forceinline__ void outE(double *p, double v, int mode) {
  if (mode & BNB_OUT_SET) *p = v;
  else *p += v;
}

// Box of a replica.  A = (box[0], 0, 0), B = (tric[0], box[1], 0),
// C = (tric[1], tric[2], box[2]): the lower-triangular cell of the
// reference's State::tricBox (src/system/state.h); tric is zero for an
// orthorhombic box.  Atoms are wrapped into the brick [0,A)x[0,B_y)x[0,C_z),
// a fundamental domain of that lattice (src/main/real3.h:340-360).
// shift[code] = sx A + sy B + sz C for the 14 half-shell images.
struct RepInfo {          // per replica, device copy in Dev::rep
  float box[3];
  int atomStart, atomCount;
  int colStart, nCols;
  int divX, divY;
  int lamStart, lamCount;
  float tric[3];          // B_x, C_x, C_y
  float4 shift[14];       // image shift vectors by shift code (kNumShifts)
};

// Lattice translation sx A + sy B + sz C in FP32, one rounding per operation
// in a fixed order (the reference's xj.x += shift.z*C_x + shift.y*B_x +
// shift.x*A_x, src/nbdirect/nbdirect.cu:196-199).
__host__ __device__ __forceinline__ float3 lattice_shift(const float *box, const float *tric, int sx, int sy,
                                                         int sz) {
  const float fx = (float)sx, fy = (float)sy, fz = (float)sz;
  float3 v;
#ifdef __CUDA_ARCH__
  v.x = __fadd_rn(__fadd_rn(__fmul_rn(fz, tric[1]), __fmul_rn(fy, tric[0])), __fmul_rn(fx, box[0]));
  v.y = __fadd_rn(__fmul_rn(fz, tric[2]), __fmul_rn(fy, box[1]));
  v.z = __fmul_rn(fz, box[2]);
#else
  volatile float t0 = fz * tric[1], t1 = fy * tric[0], t2 = fx * box[0];
  volatile float s0 = t0 + t1;
  v.x = s0 + t2;
  volatile float u0 = fz * tric[2], u1 = fy * box[1];
  v.y = u0 + u1;
  v.z = fz * box[2];
#endif
  return v;
}

// Device-side scalar counters written by the list builder.
struct Counters {
  int blockCount;
  int candCount;
  int maskCount;
  int workCount;
  int status;
  int workNext;            // dynamic work-item counter of the pair kernel
  int orderValid;          // Dev::order holds the measured longest-first order of the work items
  int pad;
  unsigned long long pairCount;
  int levelCount[kWorkLevels];  // work items per level of the work list (rebuild)
  int levelFill[kWorkLevels];   // items written per level (rebuild)
};

struct Dev {
  // --- static topology (set_topology) -------------------------------------
  int N, R, nTypes, ljCombine, lamTotal;
  int tilesPerWork;        // candidate tiles per work item (tuning knob, 1..32)
  int tailTiles;           // last candidate tiles of each i block that go to the tail levels
  RepInfo *rep;            // [R]
  int *atomRep;            // [N]
  float *atomQ;            // [N] charge * sqrt(kElectric)
  int *atomType;           // [N]
  int *atomSiteBlock;      // [N] (site<<16)|global lambda index, 0 = environment
  float2 *ljTable;         // [nTypes*nTypes] (c12,c6)   table mode
  float2 *ljType;          // [nTypes] (sqrt(12 eps), Rmin/2) combine mode
  int *exclStart;          // [N+1]
  int *exclAtom;           // [E]
  // --- capacities ----------------------------------------------------------
  int totalCols, maxBlocks, capCand, capMask, capWork;
  // --- rebuild products ----------------------------------------------------
  int *wrap;               // [N] packed integer image shift
  int *atomCol;            // [N]
  uint32_t *atomZKey;      // [N]
  int *colCount;           // [totalCols]
  int *colStartAtom;       // [totalCols+1]
  int *colStartBlock;      // [totalCols+1]
  int *colFill;            // [totalCols]
  int *bucket;             // [N]
  int *sortedAtom;         // [N]
  int *blockBounds;        // [maxBlocks+1]
  int *blockRep;           // [maxBlocks]
  int *repBlockStart;      // [R+1]
  int *slotAtom;           // [32*maxBlocks]
  int *atomSlot;           // [N]
  float *slotQ;            // [32*maxBlocks]
  int *slotType;           // [32*maxBlocks]
  int *slotSiteBlock;      // [32*maxBlocks]
  uint32_t *colKey;        // [6*totalCols] column AABB (union of its blocks) as order-preserving keys
  int *exclBlk;            // [maxBlocks*kExclBlk] distinct blocks holding excluded partners
  int *exclBlkCount;       // [maxBlocks] entries in exclBlk, -1 = more than kExclBlk
  int *cullCount;          // [maxBlocks*kNumShifts]
  int *cullOffset;         // [maxBlocks*kNumShifts+1]
  int4 *cand;              // [capCand] (jBlock, shiftCode, maskIdx, iBlock)
  int *candFlag;           // [capCand]
  int *candMaskOff;        // [capCand+1]
  uint32_t *masks;         // [capMask*32]
  int *candStart;          // [maxBlocks+1]
  int2 *work;              // [capWork] (iBlock | tiles << 22, candidate start)
  unsigned int *itemCost;  // [capWork] clock cycles of each work item in the last pair launch
  int *order;              // [capWork] work items by decreasing measured cost
  int *scanPartial;        // scratch for multi-CTA scans
  // --- per-step buffers -----------------------------------------------------
  float4 *xyzq;            // [32*maxBlocks]
  float4 *bmin, *bmax;     // [maxBlocks]
  long long *accF;         // [3*32*maxBlocks] SoA fixed-point dU/dx per slot
  long long *accL;         // [lamTotal]
  long long *accE;         // [1]
  Counters *ctr;
};

struct PairConst {        // uniform parameters of the pair kernel
  float rc2, rcut, rswitch, beta;
  float softR;            // soft-core radius (4 A in AKMA)
  // PME
  float mBeta2Log2e;      // -beta^2 * log2(e)
  float pBeta;            // erfc fit parameter p times beta
  float twoBetaSqrtPi;    // 2*beta/sqrt(pi)
  // VFSWITCH
  float k6, k12, rci3, rci6, dv6, dv12;
  float k6rci3, k12rci6;  // k6 rc^-3, k12 rc^-6 (the folded switch outside rSwitch)
  // VSWITCH / VSHIFT / FSWITCH / FSHIFT helpers
  float roff2, ron2, rul3inv, rul12;
  float fA, fB, fC, fD, fdvc, rcinv;
  float fsG, fsG5, fsC1, fsP1, fsP2, fsP3;   // factored FSWITCH (see pair_terms)
  float vshRc6inv, vshRc12inv, vshRc18inv;
};

// Programmatic dependent launch for the kernels of the list rebuild and the
// per-step path: each is launched with programmatic stream serialization, so
// its launch (and the scheduling of its CTAs) overlaps the end of the kernel
// before it in the stream instead of following it; every such kernel calls
// pdl_wait() before it touches device memory, which returns once the kernel
// before it has completed and its writes are visible.  Since each kernel
// waits for its predecessor, the stream keeps its order transitively.  A
// kernel launched without the attribute returns from pdl_wait() at once.
__device__ __forceinline__ void pdl_wait() {
#if defined(__CUDA_ARCH__)
  cudaGridDependencySynchronize();
#endif
}

template <typename... P, typename... A>
inline cudaError_t launch_pdl(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              A &&...args) {
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

}  // namespace bnb
