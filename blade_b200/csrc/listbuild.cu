// Block neighbour-list builder for the direct-space path (sm_100a).
//
// Counterpart of the reference's Domdec::reset_domdec
// (src/domdec/domdec.cu:201-211): bin atoms into x/y columns
// (assign_blocks.cu:24-60), order each column by z (assign_blocks.cu:62-178),
// cut columns into blocks of <=32 atoms (assign_blocks.cu:189-308), build
// AABBs (assign_blocks.cu:340-382), cull block pairs over the 14-image half
// shell at rCut+pad (cull.cu:44-299) and attach 32x32 exclusion masks
// (assign_excl.cu:17-313).  Differences by design:
//   * deterministic: z ties broken by atom index; all compactions are
//     order-preserving scans, so the list is identical run to run;
//   * no host synchronisation: counts stay on the device and capacity
//     overflow raises a status bit instead of a host readback;
//   * batched: R replicas in one pass, tiles never cross replicas.
// Every FP32 step is one IEEE operation (__f*_rn, built with -fmad=false),
// the sequence restated on the CPU in oracle/listbuild_oracle.c.
#include <cuda_runtime.h>
#include <stdint.h>

#include "bnb_internal.h"
#include "listbuild.h"

namespace bnb {

namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t z_key(float z) {
  uint32_t u = __float_as_uint(z);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}



// AABB gap^2 <= c2 with the operation order of orc_aabb_hit.
__device__ __forceinline__ bool aabb_hit(float4 imin, float4 imax, float4 jmin,
                                         float4 jmax, float3 sh, float c2) {
  float lo, hi, g1, g2, g, acc;
  lo = __fadd_rn(jmin.x, sh.x); hi = __fadd_rn(jmax.x, sh.x);
  g1 = __fsub_rn(lo, imax.x); g2 = __fsub_rn(imin.x, hi);
  g = g1 > g2 ? g1 : g2; g = g > 0.0f ? g : 0.0f;
  acc = __fmul_rn(g, g);
  lo = __fadd_rn(jmin.y, sh.y); hi = __fadd_rn(jmax.y, sh.y);
  g1 = __fsub_rn(lo, imax.y); g2 = __fsub_rn(imin.y, hi);
  g = g1 > g2 ? g1 : g2; g = g > 0.0f ? g : 0.0f;
  acc = __fadd_rn(acc, __fmul_rn(g, g));
  lo = __fadd_rn(jmin.z, sh.z); hi = __fadd_rn(jmax.z, sh.z);
  g1 = __fsub_rn(lo, imax.z); g2 = __fsub_rn(imin.z, hi);
  g = g1 > g2 ? g1 : g2; g = g > 0.0f ? g : 0.0f;
  acc = __fadd_rn(acc, __fmul_rn(g, g));
  return acc <= c2;
}

// ---------------------------------------------------------------------------
// Exclusive scan over int arrays (three passes, 4096 items per CTA).
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ int block_excl_scan(int v, int *total) {
  __shared__ int warpSums[kScanThreads / 32];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warpSums[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = lane < kScanThreads / 32 ? warpSums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(kFull, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kScanThreads / 32) warpSums[lane] = s;
  }
  __syncthreads();
  int before = w > 0 ? warpSums[w - 1] : 0;
  *total = warpSums[kScanThreads / 32 - 1];
  __syncthreads();
  return before + x - v;
}

__global__ void k_scan_reduce(const int *in, int n, int *partial) {
  pdl_wait();
  int base = blockIdx.x * kScanTile;
  int s = 0;
  for (int i = threadIdx.x; i < kScanTile; i += kScanThreads) {
    int k = base + i;
    if (k < n) s += in[k];
  }
  int tot;
  block_excl_scan(s, &tot);
  if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

__global__ void k_scan_top(int *partial, int nParts, int *total) {
  pdl_wait();
  // nParts <= kScanTile
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    int i = threadIdx.x * kScanItems + k;
    v[k] = i < nParts ? partial[i] : 0;
    s += v[k];
  }
  int tot;
  int off = block_excl_scan(s, &tot);
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    int i = threadIdx.x * kScanItems + k;
    if (i < nParts) partial[i] = off;
    off += v[k];
  }
  if (threadIdx.x == 0 && total) *total = tot;
}

__global__ void k_scan_down(const int *in, int *out, int n, const int *partial) {
  pdl_wait();
  int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    int i = base + k;
    v[k] = i < n ? in[i] : 0;
    s += v[k];
  }
  int tot;
  int off = block_excl_scan(s, &tot) + partial[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    int i = base + k;
    if (i < n) out[i] = off;
    off += v[k];
  }
}

// Small arrays: one CTA walks the array tile by tile with a running carry.
__global__ void k_scan_single(const int *in, int *out, int n, int *total) {
  pdl_wait();
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += kScanTile) {
    const int first = base + threadIdx.x * kScanItems;
    int v[kScanItems];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
      v[k] = first + k < n ? in[first + k] : 0;
      sum += v[k];
    }
    int tot;
    int off = block_excl_scan(sum, &tot) + carry;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
      if (first + k < n) out[first + k] = off;
      off += v[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

}  // namespace

int scan_exclusive(const int *in, int *out, int n, int *total, int *partial,
                   cudaStream_t s) {
  if (n <= 4 * kScanTile) {  // up to 16,384 items: one launch instead of three
    launch_pdl(k_scan_single, 1, kScanThreads, 0, s, in, out, n, total);
    return 1;
  }
  int parts = (n + kScanTile - 1) / kScanTile;
  if (parts < 1) parts = 1;
  launch_pdl(k_scan_reduce, parts, kScanThreads, 0, s, in, n, partial);
  launch_pdl(k_scan_top, 1, kScanThreads, 0, s, partial, parts, total);
  launch_pdl(k_scan_down, parts, kScanThreads, 0, s, in, out, n, partial);
  return 3;
}

namespace {

// ---------------------------------------------------------------------------
// 1. Binning: wrap shift, column and z key per atom.
// ---------------------------------------------------------------------------
__global__ void k_bin(Dev d, const float *__restrict__ pos) {
  pdl_wait();
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a == 0) atomicAnd(&d.ctr->status, ~kStatusListInvalid);  // this rebuild starts a fresh list
  if (a >= d.N) return;
  const RepInfo &ri = d.rep[d.atomRep[a]];
  const float x = pos[3 * a], y = pos[3 * a + 1], z = pos[3 * a + 2];
  if (!(isfinite(x) && isfinite(y) && isfinite(z))) atomicOr(&d.ctr->status, kStatusNonFinite);
  // Image shift as the reference's triclinic modulus (src/main/real3.h:340-360):
  // z by C, then y by B, then x by A; for an orthorhombic box the three are
  // independent.
  float fz = floorf(__fdiv_rn(z, ri.box[2]));
  fz = fminf(fmaxf(fz, -127.0f), 127.0f);
  const float yz = __fsub_rn(y, __fmul_rn(fz, ri.tric[2]));
  const float xz = __fsub_rn(x, __fmul_rn(fz, ri.tric[1]));
  float fy = floorf(__fdiv_rn(yz, ri.box[1]));
  fy = fminf(fmaxf(fy, -127.0f), 127.0f);
  const float xy = __fsub_rn(xz, __fmul_rn(fy, ri.tric[0]));
  float fx = floorf(__fdiv_rn(xy, ri.box[0]));
  fx = fminf(fmaxf(fx, -127.0f), 127.0f);
  int s[3] = {(int)fx, (int)fy, (int)fz};
  // the packed (wrapped) coordinates, as k_pack computes them
  const float3 L = lattice_shift(ri.box, ri.tric, s[0], s[1], s[2]);
  float w[3] = {__fsub_rn(x, L.x), __fsub_rn(y, L.y), __fsub_rn(z, L.z)};
  d.wrap[a] = (s[0] + 128) | ((s[1] + 128) << 8) | ((s[2] + 128) << 16);
  int ix = (int)floorf(__fmul_rn(__fdiv_rn(w[0], ri.box[0]), (float)ri.divX));
  ix = ix >= ri.divX ? ri.divX - 1 : ix;
  ix = ix < 0 ? 0 : ix;
  int iy = (int)floorf(__fmul_rn(__fdiv_rn(w[1], ri.box[1]), (float)ri.divY));
  iy = iy >= ri.divY ? ri.divY - 1 : iy;
  iy = iy < 0 ? 0 : iy;
  int col = ri.colStart + ix * ri.divY + iy;
  d.atomCol[a] = col;
  d.atomZKey[a] = z_key(w[2]);
  atomicAdd(&d.colCount[col], 1);
}

// ---------------------------------------------------------------------------
// 2. Column scan (single CTA): atom offsets, block offsets, block bounds.
// ---------------------------------------------------------------------------
__global__ void k_colscan(Dev d, const int *__restrict__ colRep) {
  pdl_wait();
  __shared__ int carryA, carryB;
  if (threadIdx.x == 0) { carryA = 0; carryB = 0; }
  __syncthreads();
  const int nc = d.totalCols;
  for (int c0 = 0; c0 < nc; c0 += blockDim.x) {
    int c = c0 + threadIdx.x;
    int n = c < nc ? d.colCount[c] : 0;
    int nb = (n + 31) >> 5;
    // two block-wide scans via warp shuffles and shared memory
    __shared__ int wa[32], wb[32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int xa = n, xb = nb;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int ya = __shfl_up_sync(kFull, xa, o), yb = __shfl_up_sync(kFull, xb, o);
      if (lane >= o) { xa += ya; xb += yb; }
    }
    if (lane == 31) { wa[w] = xa; wb[w] = xb; }
    __syncthreads();
    if (w == 0) {
      int sa = lane < nw ? wa[lane] : 0, sb = lane < nw ? wb[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int ya = __shfl_up_sync(kFull, sa, o), yb = __shfl_up_sync(kFull, sb, o);
        if (lane >= o) { sa += ya; sb += yb; }
      }
      if (lane < nw) { wa[lane] = sa; wb[lane] = sb; }
    }
    __syncthreads();
    int offA = carryA + (w ? wa[w - 1] : 0) + xa - n;
    int offB = carryB + (w ? wb[w - 1] : 0) + xb - nb;
    if (c < nc) {
      d.colStartAtom[c] = offA;
      d.colStartBlock[c] = offB;
      d.colFill[c] = 0;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        d.colKey[6 * c + k] = 0xFFFFFFFFu;  // min keys: larger than any value
        d.colKey[6 * c + 3 + k] = 0u;       // max keys: smaller than any value
      }
      int r = colRep[c];
      for (int k = 0; k < nb; k++) {
        int b = offB + k;
        if (b < d.maxBlocks) {
          d.blockBounds[b] = offA + 32 * k;
          d.blockRep[b] = r;
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) { carryA += wa[nw - 1]; carryB += wb[nw - 1]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    int B = carryB;
    d.colStartAtom[nc] = carryA;
    d.colStartBlock[nc] = B;
    if (B > d.maxBlocks) {
      atomicOr(&d.ctr->status, kStatusBlockOverflow);
      B = d.maxBlocks;
    }
    d.blockBounds[B] = carryA;
    d.ctr->blockCount = B;
  }
  if (threadIdx.x < kWorkLevels) {  // the work list of this rebuild is counted afresh
    d.ctr->levelCount[threadIdx.x] = 0;
    d.ctr->levelFill[threadIdx.x] = 0;
  }
  if (threadIdx.x == 0) d.ctr->orderValid = 0;  // until the new items are measured
  __syncthreads();
  for (int r = threadIdx.x; r <= d.R; r += blockDim.x) {
    int b = r < d.R ? d.colStartBlock[d.rep[r].colStart] : d.colStartBlock[nc];
    d.repBlockStart[r] = b < d.maxBlocks ? b : d.maxBlocks;
  }
}

// 3. Scatter atoms into column buckets (arbitrary order within a column).
__global__ void k_scatter(Dev d) {
  pdl_wait();
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= d.N) return;
  int col = d.atomCol[a];
  int p = d.colStartAtom[col] + atomicAdd(&d.colFill[col], 1);
  d.bucket[p] = a;
}

// 4. Sort each column by (z key, atom index): bitonic sort in shared memory,
//    rank counting for columns larger than kSortCap.
__global__ void k_colsort(Dev d) {
  pdl_wait();
  __shared__ unsigned long long key[kSortCap];
  const int c = blockIdx.x;
  const int n = d.colCount[c];
  const int base = d.colStartAtom[c];
  if (n == 0) return;
  __syncthreads();  // every thread has read the count
  if (threadIdx.x == 0) d.colCount[c] = 0;  // zero for the next rebuild's binning
  if (n <= kSortCap) {
    int n2 = 1;
    while (n2 < n) n2 <<= 1;
    for (int i = threadIdx.x; i < n2; i += blockDim.x) {
      if (i < n) {
        int a = d.bucket[base + i];
        key[i] = ((unsigned long long)d.atomZKey[a] << 32) | (unsigned)a;
      } else {
        key[i] = ~0ull;
      }
    }
    __syncthreads();
    for (int k = 2; k <= n2; k <<= 1) {
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int i = threadIdx.x; i < n2; i += blockDim.x) {
          int ixj = i ^ j;
          if (ixj > i) {
            unsigned long long x = key[i], y = key[ixj];
            bool up = (i & k) == 0;
            if ((x > y) == up) { key[i] = y; key[ixj] = x; }
          }
        }
        __syncthreads();
      }
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      d.sortedAtom[base + i] = (int)(key[i] & 0xFFFFFFFFull);
  } else {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      int a = d.bucket[base + i];
      unsigned long long ki = ((unsigned long long)d.atomZKey[a] << 32) | (unsigned)a;
      int rank = 0;
      for (int j = 0; j < n; j++) {
        int b = d.bucket[base + j];
        unsigned long long kj = ((unsigned long long)d.atomZKey[b] << 32) | (unsigned)b;
        rank += kj < ki;
      }
      d.sortedAtom[base + rank] = a;
    }
  }
}

// 5. Slots: atom of each of the 32 lanes of each block, per-slot parameters.
__global__ void k_slots(Dev d) {
  pdl_wait();
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int b = t >> 5, lane = t & 31;
  if (b >= d.maxBlocks) return;
  int B = d.ctr->blockCount;
  if (b >= B) return;
  int i0 = d.blockBounds[b], i1 = d.blockBounds[b + 1];
  int idx = i0 + lane;
  // a block never extends past its column: bounds of the next block start a
  // new column or lie 32 further in the same column
  int end = i0 + 32 < i1 ? i0 + 32 : i1;
  if (idx < end) {
    int a = d.sortedAtom[idx];
    d.slotAtom[t] = a;
    d.atomSlot[a] = t;
    d.slotQ[t] = d.atomQ[a];
    d.slotType[t] = d.atomType[a];
    d.slotSiteBlock[t] = d.atomSiteBlock[a];
  } else {
    d.slotAtom[t] = -1;
    d.slotQ[t] = 0.0f;
    d.slotType[t] = 0;
    d.slotSiteBlock[t] = 0;
  }
}

}  // namespace

// 6. Pack coordinates with the stored image shift; per-block AABBs.  At a
//    rebuild (columns) also the column AABBs, the union of the column's block
//    boxes, by atomic min/max of order-preserving keys (order-independent, so
//    reproducible).  A block that hits implies its column hits under the
//    rounding of aabb_hit, so the cull may skip columns that miss.
__global__ void k_pack(Dev d, const float *__restrict__ pos, bool columns) {
  pdl_wait();
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int b = t >> 5;
  if (b >= d.maxBlocks) return;
  if (b >= d.ctr->blockCount) return;
  int a = d.slotAtom[t];
  const RepInfo &ri = d.rep[d.blockRep[b]];
  float3 p = make_float3(0.f, 0.f, 0.f);
  float3 mn = make_float3(INFINITY, INFINITY, INFINITY);
  float3 mx = make_float3(-INFINITY, -INFINITY, -INFINITY);
  if (a >= 0) {
    int w = d.wrap[a];
    const float3 L = lattice_shift(ri.box, ri.tric, (w & 0xFF) - 128, ((w >> 8) & 0xFF) - 128,
                                   ((w >> 16) & 0xFF) - 128);
    p.x = __fsub_rn(pos[3 * a], L.x);
    p.y = __fsub_rn(pos[3 * a + 1], L.y);
    p.z = __fsub_rn(pos[3 * a + 2], L.z);
    mn = p;
    mx = p;
  }
  d.xyzq[t] = make_float4(p.x, p.y, p.z, d.slotQ[t]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn.x = fminf(mn.x, __shfl_xor_sync(kFull, mn.x, o));
    mn.y = fminf(mn.y, __shfl_xor_sync(kFull, mn.y, o));
    mn.z = fminf(mn.z, __shfl_xor_sync(kFull, mn.z, o));
    mx.x = fmaxf(mx.x, __shfl_xor_sync(kFull, mx.x, o));
    mx.y = fmaxf(mx.y, __shfl_xor_sync(kFull, mx.y, o));
    mx.z = fmaxf(mx.z, __shfl_xor_sync(kFull, mx.z, o));
  }
  if ((t & 31) == 0) {
    d.bmin[b] = make_float4(mn.x, mn.y, mn.z, 0.f);
    d.bmax[b] = make_float4(mx.x, mx.y, mx.z, 0.f);
    if (columns) {
      unsigned *key = d.colKey + 6 * d.atomCol[a];  // lane 0 of a block always holds an atom
      atomicMin(key + 0, z_key(mn.x));
      atomicMin(key + 1, z_key(mn.y));
      atomicMin(key + 2, z_key(mn.z));
      atomicMax(key + 3, z_key(mx.x));
      atomicMax(key + 4, z_key(mx.y));
      atomicMax(key + 5, z_key(mx.z));
    }
  }
}

namespace {

__device__ __forceinline__ float key_float(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k ^ 0x80000000u) : ~k);
}

// 7/9. Cull: one warp per (iBlock, shift code); count pass then write pass.
//      The j blocks of the replica are visited column by column: lanes test
//      32 columns' AABBs at once, the blocks of the columns that hit are
//      concatenated (warp scan of their counts) and tested 32 at a time.
//      Columns and the blocks inside them are in increasing block order, so
//      the candidates come out in the order of a scan over all j blocks.
template <bool kWrite>
__global__ void k_cull(Dev d, float rcull2) {
  pdl_wait();
  const int lane = threadIdx.x & 31;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  const int B = d.ctr->blockCount;
  const int total = d.maxBlocks * kNumShifts;
  for (int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; gw < total; gw += nWarps) {
    int iBlock = gw / kNumShifts, code = gw - iBlock * kNumShifts;
    if (iBlock >= B) {
      if (!kWrite && lane == 0) d.cullCount[gw] = 0;
      continue;
    }
    int r = d.blockRep[iBlock];
    const RepInfo &ri = d.rep[r];
    const float4 sv = ri.shift[code];
    const float3 sh = make_float3(sv.x, sv.y, sv.z);
    float4 imin = d.bmin[iBlock], imax = d.bmax[iBlock];
    const int j0 = code == 0 ? iBlock : d.repBlockStart[r];
    const int j1 = d.repBlockStart[r + 1];
    int cnt = 0;
    int base = kWrite ? d.cullOffset[gw] : 0;
    for (int cb = 0; cb < ri.nCols; cb += 32) {
      const int c = ri.colStart + cb + lane;
      int bs = 0, n = 0;
      if (cb + lane < ri.nCols) {
        bs = d.colStartBlock[c];
        int be = d.colStartBlock[c + 1];
        bs = bs > j0 ? bs : j0;
        be = be < j1 ? be : j1;
        if (bs < be) {
          const uint32_t *key = d.colKey + 6 * c;
          const float4 cmin = make_float4(key_float(key[0]), key_float(key[1]), key_float(key[2]), 0.f);
          const float4 cmax = make_float4(key_float(key[3]), key_float(key[4]), key_float(key[5]), 0.f);
          if (aabb_hit(imin, imax, cmin, cmax, sh, rcull2)) n = be - bs;
        }
      }
      int inc = n;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, inc, o);
        if (lane >= o) inc += y;
      }
      const int tot = __shfl_sync(kFull, inc, 31);
      const int exc = inc - n;
      for (int t0 = 0; t0 < tot; t0 += 32) {
        const int t = t0 + lane;
        // column lane k holding item t: the first lane whose inclusive count exceeds t
        int k = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1)
          if (__shfl_sync(kFull, inc, k + step - 1) <= t) k += step;
        const int jStart = __shfl_sync(kFull, bs, k);
        const int jOff = __shfl_sync(kFull, exc, k);
        bool hit = false;
        if (t < tot) {
          const int j = jStart + (t - jOff);
          hit = aabb_hit(imin, imax, d.bmin[j], d.bmax[j], sh, rcull2);
        }
        const unsigned m = __ballot_sync(kFull, hit);
        if (kWrite && hit) {
          const int j = jStart + (t - jOff);
          int p = base + cnt + __popc(m & ((1u << lane) - 1u));
          if (p < d.capCand) d.cand[p] = make_int4(j, code, -1, iBlock);
        }
        cnt += __popc(m);
      }
    }
    if (!kWrite && lane == 0) d.cullCount[gw] = cnt;
    if (kWrite && lane == 0 && code == 0) {  // candidate range and work items of this i block
      int c0 = d.cullOffset[gw], c1 = d.cullOffset[gw + kNumShifts];
      c0 = c0 < d.capCand ? c0 : d.capCand;
      c1 = c1 < d.capCand ? c1 : d.capCand;
      d.candStart[iBlock] = c0;
      int tiles[kWorkLevels], items[kWorkLevels];
      const int L = work_split(c1 - c0, d.tilesPerWork, d.tailTiles, tiles, items);
      for (int l = 0; l < L; l++)
        if (items[l]) atomicAdd(&d.ctr->levelCount[l], items[l]);
    }
  }
  if (kWrite && blockIdx.x == 0 && threadIdx.x == 0) {
    const int tot = d.cullOffset[d.maxBlocks * kNumShifts];
    d.ctr->candCount = tot < d.capCand ? tot : d.capCand;
    if (tot > d.capCand) atomicOr(&d.ctr->status, kStatusCandOverflow);
    d.candStart[B] = d.ctr->candCount;
  }
}

// 10/12. Exclusion rows of a candidate tile: one warp, lane = i atom.
__device__ __forceinline__ uint32_t excl_row(const Dev &d, int iBlock, int jBlock, int lane) {
  uint32_t row = 0xFFFFFFFFu;
  int a = d.slotAtom[32 * iBlock + lane];
  if (a >= 0) {
    int e1 = d.exclStart[a + 1];
    for (int e = d.exclStart[a]; e < e1; e++) {
      int b = d.exclAtom[e];
      if (b == a) continue;
      int sl = d.atomSlot[b];
      if ((sl >> 5) == jBlock) row &= ~(1u << (sl & 31));
    }
  }
  return row;
}

// 10a. Exclusion-partner blocks: per block, the distinct blocks that hold an
//      excluded partner of one of its atoms (one warp per block, lane = atom).
//      Candidate tiles whose j block is not listed carry no exclusion, so
//      k_excl skips their per-atom scan.  More than kExclBlk blocks: count -1,
//      and every tile of the block takes the full scan.
__global__ void k_excl_blocks(Dev d) {
  pdl_wait();
  __shared__ int sList[8][kExclBlk];
  const int lane = threadIdx.x & 31;
  const int warp = (threadIdx.x >> 5) & 7;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  const int B = d.ctr->blockCount;
  for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < B; b += nWarps) {
    const int a = d.slotAtom[32 * b + lane];
    int e = 0, e1 = 0;
    if (a >= 0) {
      e = d.exclStart[a];
      e1 = d.exclStart[a + 1];
    }
    int n = 0;       // blocks listed so far (warp-uniform)
    int mine = -1;   // lane k < n holds the k-th listed block
    while (__any_sync(kFull, e < e1) && n <= kExclBlk) {
      int jb = -1;
      if (e < e1) {
        const int p = d.exclAtom[e++];
        if (p != a) jb = d.atomSlot[p] >> 5;
      }
      const int listed = n < kExclBlk ? n : kExclBlk;
      for (int k = 0; k < listed; k++)
        if (jb == __shfl_sync(kFull, mine, k)) jb = -1;
      const unsigned grp = __match_any_sync(kFull, jb);
      const bool lead = jb >= 0 && (__ffs(grp) - 1) == lane;
      const unsigned leaders = __ballot_sync(kFull, lead);
      const int pos = n + __popc(leaders & ((1u << lane) - 1u));
      if (lead && pos < kExclBlk) sList[warp][pos] = jb;
      n += __popc(leaders);
      __syncwarp();
      mine = lane < (n < kExclBlk ? n : kExclBlk) ? sList[warp][lane] : -1;
      __syncwarp();
    }
    if (lane < kExclBlk) d.exclBlk[kExclBlk * b + lane] = mine;
    if (lane == 0) d.exclBlkCount[b] = n <= kExclBlk ? n : -1;
  }
}

template <bool kWrite>
__global__ void k_excl(Dev d) {
  pdl_wait();
  const int lane = threadIdx.x & 31;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  const int n = d.ctr->candCount;
  for (int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < d.capCand; c += nWarps) {
    if (c >= n) {
      if (!kWrite && lane == 0) d.candFlag[c] = 0;
      continue;
    }
    if (kWrite && d.candMaskOff[c + 1] == d.candMaskOff[c]) {  // the flag pass found no exclusion here
      if (lane == 0) d.cand[c].z = -1;
      continue;
    }
    int4 t = d.cand[c];
    const int nb = d.exclBlkCount[t.w];
    bool scan = true;
    if (nb >= 0) {
      const int v = lane < nb ? d.exclBlk[kExclBlk * t.w + lane] : -1;
      scan = __any_sync(kFull, v == t.x);
    }
    uint32_t row = scan ? excl_row(d, t.w, t.x, lane) : 0xFFFFFFFFu;
    bool any = __any_sync(kFull, row != 0xFFFFFFFFu);
    if (!kWrite) {
      if (lane == 0) d.candFlag[c] = any ? 1 : 0;
    } else {
      int idx = -1;
      if (any) {
        idx = d.candMaskOff[c];
        if (idx < d.capMask) d.masks[32 * (size_t)idx + lane] = row;
        else idx = -1;
      }
      if (lane == 0) d.cand[c].z = idx;
    }
  }
  if (kWrite && blockIdx.x == 0 && threadIdx.x == 0) {
    const int tot = d.candMaskOff[d.capCand];
    d.ctr->maskCount = tot < d.capMask ? tot : d.capMask;
    if (tot > d.capMask) atomicOr(&d.ctr->status, kStatusMaskOverflow);
  }
}

// 13. Work items (iBlock | tiles << 22, first candidate), by level: all
//     level-0 items (tilesPerWork tiles) first, then the level-1 items, and
//     so on down to 1-tile items (work_split).  The pair kernel's warps take
//     items in list order, so the last items they take are small and the
//     warps finish close together.  Within a level the order follows the
//     atomics; the items themselves depend on their block only.
__global__ void k_work(Dev d) {
  pdl_wait();
  const int B = d.ctr->blockCount;
  int off[kWorkLevels + 1];
  off[0] = 0;
  for (int l = 0; l < kWorkLevels; l++) off[l + 1] = off[l] + d.ctr->levelCount[l];
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) {
    const int total = off[kWorkLevels];
    d.ctr->workCount = total < d.capWork ? total : d.capWork;
    if (total > d.capWork) atomicOr(&d.ctr->status, kStatusWorkOverflow);
  }
  // one warp per block: lane 0 reserves each level's items, the lanes write them
  const int lane = threadIdx.x & 31, nWarps = (gridDim.x * blockDim.x) >> 5;
  for (int b = t >> 5; b < B; b += nWarps) {
    const int c0 = d.candStart[b], nc = d.candStart[b + 1] - c0;
    int tiles[kWorkLevels], items[kWorkLevels];
    const int L = work_split(nc, d.tilesPerWork, d.tailTiles, tiles, items);
    int s = c0;  // first candidate of the level (the order of work_walk)
    for (int l = 0; l < L; l++) {
      const int size = work_item_size(d.tilesPerWork, l), end = s + tiles[l];
      if (items[l]) {
        int base = 0;
        if (lane == 0) base = off[l] + atomicAdd(&d.ctr->levelFill[l], items[l]);
        base = __shfl_sync(kFull, base, 0);
        for (int k = lane; k < items[l]; k += 32) {
          const int first = s + k * size, n = end - first < size ? end - first : size;
          if (base + k < d.capWork) d.work[base + k] = make_int2(b | (n << 22), first);
        }
      }
      s = end;
    }
  }
}

inline int grid_for(long long n, int threads) {
  long long g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > 65535LL * 16) g = 65535LL * 16;
  return (int)g;
}

}  // namespace

void pack_positions(const Dev &d, const float *pos, cudaStream_t s) {
  int n = 32 * d.maxBlocks;
  launch_pdl(k_pack, grid_for(n, 256), 256, 0, s, d, pos, false);
}

namespace {
__global__ void k_clear_status(Counters *c) {
  pdl_wait();
  atomicAnd(&c->status, ~kStatusListInvalid);
}
}  // namespace

int rebuild_list(const Dev &d, const int *colRep, const float *pos, float rcull2,
                 cudaStream_t s) {
  int launches = 8;  // bin or clear, colscan, colsort, slots, pack, excl_blocks, work, + scatter or not below
  // colCount is zero here: set so at allocation and by k_colsort after use
  if (d.N > 0) launch_pdl(k_bin, grid_for(d.N, 256), 256, 0, s, d, pos);  // also clears the list-invalid bits
  else launch_pdl(k_clear_status, 1, 1, 0, s, d.ctr);
  launch_pdl(k_colscan, 1, 1024, 0, s, d, colRep);
  if (d.N > 0) {
    launch_pdl(k_scatter, grid_for(d.N, 256), 256, 0, s, d);
    launches++;
  }
  launch_pdl(k_colsort, d.totalCols, 512, 0, s, d);
  launch_pdl(k_slots, grid_for(32LL * d.maxBlocks, 256), 256, 0, s, d);
  launch_pdl(k_pack, grid_for(32LL * d.maxBlocks, 256), 256, 0, s, d, pos, true);
  launch_pdl(k_excl_blocks, grid_for(32LL * d.maxBlocks, 256), 256, 0, s, d);
  // cull: count, scan, write
  const int cullWarps = d.maxBlocks * kNumShifts;
  const int cullGrid = grid_for(32LL * cullWarps, 256) < 148 * 32 ? grid_for(32LL * cullWarps, 256) : 148 * 32;
  launch_pdl(k_cull<false>, cullGrid, 256, 0, s, d, rcull2);
  launches += 4;  // two cull and two exclusion passes
  launches += scan_exclusive(d.cullCount, d.cullOffset, cullWarps, d.cullOffset + cullWarps, d.scanPartial, s);
  launch_pdl(k_cull<true>, cullGrid, 256, 0, s, d, rcull2);  // also candStart, work counts, candCount
  // exclusion masks: flag, scan, write
  const int exGrid = grid_for(32LL * d.capCand, 256) < 148 * 16 ? grid_for(32LL * d.capCand, 256) : 148 * 16;
  launch_pdl(k_excl<false>, exGrid, 256, 0, s, d);
  launches += scan_exclusive(d.candFlag, d.candMaskOff, d.capCand, d.candMaskOff + d.capCand, d.scanPartial, s);
  launch_pdl(k_excl<true>, exGrid, 256, 0, s, d);  // also maskCount
  // work items
  launch_pdl(k_work, grid_for(32LL * d.maxBlocks, 256), 256, 0, s, d);
  return launches;
}

}  // namespace bnb
