/*
 * FP32/integer CPU restatement of the block neighbour list.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Follows the reference's list algorithm:
 *   - column grid from the density heuristic   src/domdec/domdec.cu:114-117
 *   - column token (ix,iy) per atom             src/domdec/assign_blocks.cu:24-60
 *   - sort by (column, z), cut each column into blocks of <=32 atoms
 *                                               assign_blocks.cu:154-308
 *   - per-block AABBs                           assign_blocks.cu:340-382
 *   - half-shell culling with 14 image shifts, own image keeps jBlock>=iBlock
 *                                               src/domdec/cull.cu:44-299
 *   - 32x32 exclusion masks per (iBlock,jBlock) src/domdec/assign_excl.cu:167-313
 *   - per-step recull at rCut                   src/domdec/recull.cu:41-122
 * with two deliberate differences: ties in z are broken by atom index (the
 * reference's concurrent tree sort orders equal keys arbitrarily), and the
 * wrap into the box is an integer image shift kept per atom instead of an
 * in-place rewrite of the caller's coordinates.
 *
 * Every floating-point step is a single IEEE FP32 operation in a fixed order
 * (compile with -ffp-contract=off); the CUDA list builder performs the same
 * operations with __f*_rn intrinsics, so the two agree bit for bit.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

void orc_domain_div(int N, const float box[3], int *divX, int *divY) {
  float invDensity = box[0] * box[1] * box[2] / (float)N;
  float approx = expf(logf(32.0f * invDensity) / 3.0f);
  *divX = (int)ceilf(box[0] / approx);
  *divY = (int)ceilf(box[1] / approx);
  if (*divX < 1) *divX = 1;
  if (*divY < 1) *divY = 1;
}

void orc_shift_vector(int code, int *sx, int *sy, int *sz) {
  /* Enumerate z in {0,1}; y in {-z..1}; x in {-(y!=0||z!=0)..1}. */
  int c = 0;
  for (int z = 0; z < 2; z++)
    for (int y = -z; y < 2; y++)
      for (int x = -((y != 0) || (z != 0)); x < 2; x++) {
        if (c == code) { *sx = x; *sy = y; *sz = z; return; }
        c++;
      }
  *sx = *sy = *sz = 0;
}

int orc_aabb_hit(const float *imin, const float *imax, const float *jmin,
                 const float *jmax, const float shift[3], float c2) {
  float acc = 0.0f;
  for (int d = 0; d < 3; d++) {
    float lo = jmin[d] + shift[d];
    float hi = jmax[d] + shift[d];
    float g1 = lo - imax[d];
    float g2 = imin[d] - hi;
    float g = g1 > g2 ? g1 : g2;
    g = g > 0.0f ? g : 0.0f;
    float gg = g * g;
    acc = acc + gg;
  }
  return acc <= c2;
}

static inline uint32_t zkey(float z) {
  uint32_t u;
  memcpy(&u, &z, 4);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

/* Box of 6 floats: A_x, B_y, C_z (the brick) then B_x, C_x, C_y (zero for an
 * orthorhombic box): A = (A_x,0,0), B = (B_x,B_y,0), C = (C_x,C_y,C_z). */
static inline float clamp_shift(float f) { return f < -127.0f ? -127.0f : (f > 127.0f ? 127.0f : f); }

/* Lattice translation sx A + sy B + sz C, one rounding per operation in the
 * order of the reference's shift (src/nbdirect/nbdirect.cu:196-199). */
void orc_lattice_shift(const float box[6], int sx, int sy, int sz, float out[3]) {
  float fx = (float)sx, fy = (float)sy, fz = (float)sz;
  float t0 = fz * box[4], t1 = fy * box[3], t2 = fx * box[0];
  float s0 = t0 + t1;
  out[0] = s0 + t2;
  float u0 = fz * box[5], u1 = fy * box[1];
  out[1] = u0 + u1;
  out[2] = fz * box[2];
}

/* Integer image shift of a position: z by C, then y by B, then x by A (the
 * reference's triclinic modulus, src/main/real3.h:340-360). */
static inline void wrap_shift(const float *x, const float box[6], int s[3]) {
  float fz = clamp_shift(floorf(x[2] / box[2]));
  float t = fz * box[5];
  float yz = x[1] - t;
  t = fz * box[4];
  float xz = x[0] - t;
  float fy = clamp_shift(floorf(yz / box[1]));
  t = fy * box[3];
  float xy = xz - t;
  float fx = clamp_shift(floorf(xy / box[0]));
  s[0] = (int)fx; s[1] = (int)fy; s[2] = (int)fz;
}

/* Shift vectors of the 14 half-shell codes, centred under the shear as the
 * reference's cull (src/domdec/cull.cu:141-190). */
void orc_shift_table(const float box[6], float table[14][3]) {
  for (int code = 0; code < 14; code++) {
    int x, y, z;
    orc_shift_vector(code, &x, &y, &z);
    float ty = (float)z * box[5];
    float qy = ty / box[1];
    int y0 = -(int)floorf(qy + 0.5f);
    int sy = y + y0;
    float tx0 = (float)z * box[4], tx1 = (float)sy * box[3];
    float sxy = tx0 + tx1;
    float qx = sxy / box[0];
    int x0 = -(int)floorf(qx + 0.5f);
    orc_lattice_shift(box, x + x0, sy, z, table[code]);
  }
}

typedef struct { uint64_t key; int col; int atom; } sort_rec;
static int cmp_rec(const void *a, const void *b) {
  const sort_rec *x = (const sort_rec *)a, *y = (const sort_rec *)b;
  if (x->col != y->col) return x->col < y->col ? -1 : 1;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return 0;
}

void orc_pack(const orc_list *l, const float *xyz, const float box[6],
              float *packed, float *bmin, float *bmax) {
  int B = l->blockCount;
  for (int b = 0; b < B; b++) {
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int lane = 0; lane < 32; lane++) {
      int slot = 32 * b + lane;
      int a = l->slotAtom[slot];
      if (a < 0) {
        packed[3 * slot] = packed[3 * slot + 1] = packed[3 * slot + 2] = 0.0f;
        continue;
      }
      int w = l->wrap[a];
      float L[3];
      orc_lattice_shift(box, (w & 0xFF) - 128, ((w >> 8) & 0xFF) - 128, ((w >> 16) & 0xFF) - 128, L);
      for (int d = 0; d < 3; d++) {
        float v = xyz[3 * a + d] - L[d];
        packed[3 * slot + d] = v;
        if (v < mn[d]) mn[d] = v;
        if (v > mx[d]) mx[d] = v;
      }
    }
    for (int d = 0; d < 3; d++) { bmin[3 * b + d] = mn[d]; bmax[3 * b + d] = mx[d]; }
  }
}

int orc_build_list(int N, const float *xyz, const float box[6], float rCull,
                   const int *exclStart, const int *exclAtom, orc_list *out) {
  memset(out, 0, sizeof(*out));
  out->N = N;
  orc_domain_div(N, box, &out->divX, &out->divY);
  int divX = out->divX, divY = out->divY, nCols = divX * divY;
  out->nCols = nCols;
  out->wrap = (int *)malloc(sizeof(int) * N);
  sort_rec *rec = (sort_rec *)malloc(sizeof(sort_rec) * (N > 0 ? N : 1));
  out->colCount = (int *)calloc(nCols, sizeof(int));
  for (int a = 0; a < N; a++) {
    int s[3];
    float w[3], L[3];
    wrap_shift(&xyz[3 * a], box, s);
    orc_lattice_shift(box, s[0], s[1], s[2], L);
    for (int d = 0; d < 3; d++) w[d] = xyz[3 * a + d] - L[d];
    out->wrap[a] = (s[0] + 128) | ((s[1] + 128) << 8) | ((s[2] + 128) << 16);
    float px = w[0] / box[0];
    int ix = (int)floorf(px * (float)divX);
    ix = ix >= divX ? divX - 1 : ix;
    ix = ix < 0 ? 0 : ix;
    float py = w[1] / box[1];
    int iy = (int)floorf(py * (float)divY);
    iy = iy >= divY ? divY - 1 : iy;
    iy = iy < 0 ? 0 : iy;
    rec[a].col = ix * divY + iy;
    rec[a].key = ((uint64_t)zkey(w[2]) << 32) | (uint32_t)a;
    rec[a].atom = a;
    out->colCount[rec[a].col]++;
  }
  qsort(rec, N, sizeof(sort_rec), cmp_rec);
  out->sortedAtom = (int *)malloc(sizeof(int) * (N > 0 ? N : 1));
  for (int i = 0; i < N; i++) out->sortedAtom[i] = rec[i].atom;
  free(rec);

  int B = 0;
  for (int c = 0; c < nCols; c++) B += (out->colCount[c] + 31) / 32;
  out->blockCount = B;
  out->blockBounds = (int *)malloc(sizeof(int) * (B + 1));
  out->slotAtom = (int *)malloc(sizeof(int) * 32 * (B > 0 ? B : 1));
  int b = 0, start = 0;
  for (int c = 0; c < nCols; c++) {
    int n = out->colCount[c];
    for (int k = 0; k < n; k += 32) {
      out->blockBounds[b] = start + k;
      for (int lane = 0; lane < 32; lane++)
        out->slotAtom[32 * b + lane] = (k + lane < n) ? out->sortedAtom[start + k + lane] : -1;
      b++;
    }
    start += n;
  }
  out->blockBounds[B] = N;

  /* AABBs from the packed coordinates. */
  float *packed = (float *)malloc(sizeof(float) * 96 * (B > 0 ? B : 1));
  out->bmin = (float *)malloc(sizeof(float) * 3 * (B > 0 ? B : 1));
  out->bmax = (float *)malloc(sizeof(float) * 3 * (B > 0 ? B : 1));
  orc_pack(out, xyz, box, packed, out->bmin, out->bmax);
  free(packed);

  /* Atom -> (block, lane). */
  int *blockOf = (int *)malloc(sizeof(int) * (N > 0 ? N : 1));
  int *laneOf = (int *)malloc(sizeof(int) * (N > 0 ? N : 1));
  for (int s = 0; s < 32 * B; s++)
    if (out->slotAtom[s] >= 0) { blockOf[out->slotAtom[s]] = s / 32; laneOf[out->slotAtom[s]] = s % 32; }

  /* Candidates in (iBlock, shiftCode, jBlock) order. */
  float c2 = rCull * rCull;
  int cap = 1024, cnt = 0, mcap = 64, mcnt = 0;
  int *cand = (int *)malloc(sizeof(int) * 2 * cap);
  int *candExcl = (int *)malloc(sizeof(int) * cap);
  uint32_t *masks = (uint32_t *)malloc(sizeof(uint32_t) * 32 * mcap);
  out->candStart = (int *)malloc(sizeof(int) * (B + 1));
  float table[14][3];
  orc_shift_table(box, table);
  for (int i = 0; i < B; i++) {
    out->candStart[i] = cnt;
    for (int code = 0; code < 14; code++) {
      const float *sh = table[code];
      for (int j = (code == 0 ? i : 0); j < B; j++) {
        if (!orc_aabb_hit(&out->bmin[3 * i], &out->bmax[3 * i], &out->bmin[3 * j],
                          &out->bmax[3 * j], sh, c2))
          continue;
        if (cnt == cap) {
          cap *= 2;
          cand = (int *)realloc(cand, sizeof(int) * 2 * cap);
          candExcl = (int *)realloc(candExcl, sizeof(int) * cap);
        }
        cand[2 * cnt] = j;
        cand[2 * cnt + 1] = code;
        /* Exclusion rows. */
        uint32_t rows[32];
        int any = 0;
        for (int lane = 0; lane < 32; lane++) {
          rows[lane] = 0xFFFFFFFFu;
          int a = out->slotAtom[32 * i + lane];
          if (a < 0 || !exclStart) continue;
          for (int e = exclStart[a]; e < exclStart[a + 1]; e++) {
            int bb = exclAtom[e];
            if (bb == a) continue;
            if (blockOf[bb] == j) { rows[lane] &= ~(1u << laneOf[bb]); any = 1; }
          }
        }
        if (any) {
          if (mcnt == mcap) {
            mcap *= 2;
            masks = (uint32_t *)realloc(masks, sizeof(uint32_t) * 32 * mcap);
          }
          memcpy(&masks[32 * mcnt], rows, sizeof(rows));
          candExcl[cnt] = mcnt++;
        } else {
          candExcl[cnt] = -1;
        }
        cnt++;
      }
    }
  }
  out->candStart[B] = cnt;
  out->candCount = cnt;
  out->cand = cand;
  out->candExcl = candExcl;
  out->maskCount = mcnt;
  out->masks = masks;
  free(blockOf);
  free(laneOf);
  return 0;
}

void orc_free_list(orc_list *l) {
  free(l->wrap); free(l->colCount); free(l->blockBounds); free(l->sortedAtom);
  free(l->slotAtom); free(l->bmin); free(l->bmax); free(l->candStart);
  free(l->cand); free(l->candExcl); free(l->masks);
  memset(l, 0, sizeof(*l));
}
