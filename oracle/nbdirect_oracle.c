/*
 * FP64 CPU oracle: direct-space pair physics and MSLD lambda maps.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * The pair function restates src/nbdirect/nbdirect.cu:242-433 branch by
 * branch in double precision with exact libm erfc/exp.  Pairs are found with
 * a minimum-image cell list (one image per pair, valid while rCut < box/2),
 * which is the set of pairs the reference's half-shell block list visits.
 */
#include "oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Pair physics                                                              */
/* ------------------------------------------------------------------------ */

/* Energy eij and dE/drEff (fij) at distance rEff, before MSLD scaling.
 * Electrostatics: nbdirect.cu:281-323; van der Waals: nbdirect.cu:326-396. */
static void pair_terms(double rEff, double kqq, double c12, double c6,
                       const orc_params *p, double *eij, double *fij) {
  const double rc = p->rCut, rs = p->rSwitch;
  const double rinv = 1.0 / rEff;
  double e = 0, f = 0;
  if (p->elecMethod == 0) { /* FSWITCH: nbdirect.cu:281-300 */
    double roff2 = rc * rc, ron2 = rs * rs;
    double ginv = 1.0 / ((roff2 - ron2) * (roff2 - ron2) * (roff2 - ron2));
    double A = roff2 * roff2 * (roff2 - 3 * ron2) * ginv;
    double B = 6 * roff2 * ron2 * ginv;
    double C = -(ron2 + roff2) * ginv;
    double D = 2 * ginv / 5;
    double dvc = 8 * (ron2 * roff2 * (rc - rs) -
                      (roff2 * roff2 * rc - ron2 * ron2 * rs) / 5) * ginv;
    double r2 = rEff * rEff, r3 = r2 * rEff, r5 = r3 * r2;
    if (rEff <= rs) {
      f = -kqq * rinv * rinv;
      e = kqq * (rinv + dvc);
    } else {
      f = -kqq * rinv * (A * rinv + B * rEff + 3 * C * r3 + 5 * D * r5);
      e = kqq * (A * (rinv - 1 / rc) + B * (rc - rEff) + C * (roff2 * rc - r3) +
                 D * (roff2 * roff2 * rc - r5));
    }
  } else if (p->elecMethod == 1) { /* PME real space: nbdirect.cu:301-311 */
    double br = p->betaEwald * rEff;
    double erfcrinv = erfc(br) * rinv;
    f = -kqq * (erfcrinv + (2.0 / sqrt(M_PI)) * p->betaEwald * exp(-br * br)) * rinv;
    e = kqq * erfcrinv;
  } else { /* FSHIFT: nbdirect.cu:312-323 */
    double roffinv = 1 / rc, roffinv2 = roffinv * roffinv;
    f = -kqq * (rinv * rinv - roffinv2);
    e = kqq * (rinv - 2 * roffinv + rEff * roffinv2);
  }

  double rinv3 = rinv * rinv * rinv, rinv6 = rinv3 * rinv3;
  if (p->vdwMethod == 0) { /* VFSWITCH: nbdirect.cu:331-350 */
    double rc3 = rc * rc * rc, rs3 = rs * rs * rs;
    if (rEff < rs) {
      f += (6 * c6 - 12 * c12 * rinv6) * rinv6 * rinv;
      double dv6 = 1 / (rc3 * rs3);
      e += c12 * (rinv6 * rinv6 - dv6 * dv6) - c6 * (rinv6 - dv6);
    } else {
      double k6 = rc3 / (rc3 - rs3);
      double k12 = rc3 * rc3 / (rc3 * rc3 - rs3 * rs3);
      double rci3 = 1 / rc3;
      f += (6 * c6 * k6 * (rinv3 - rci3) * rinv3 -
            12 * c12 * k12 * (rinv6 - rci3 * rci3) * rinv6) * rinv;
      e += c12 * k12 * (rinv6 - rci3 * rci3) * (rinv6 - rci3 * rci3) -
           c6 * k6 * (rinv3 - rci3) * (rinv3 - rci3);
    }
  } else if (p->vdwMethod == 1) { /* VSWITCH: nbdirect.cu:351-372 */
    if (rEff < rs) {
      f += (6 * c6 - 12 * c12 * rinv6) * rinv6 * rinv;
      e += c12 * rinv6 * rinv6 - c6 * rinv6;
    } else {
      double c2of = rc * rc, c2on = rs * rs;
      double rul3 = (c2of - c2on) * (c2of - c2on) * (c2of - c2on);
      double rul12 = 12 / rul3;
      double rijl = c2on - rEff * rEff, riju = c2of - rEff * rEff;
      double fsw = riju * riju * (riju - 3 * rijl) / rul3;
      double dfsw = rijl * riju * rul12;
      f += fsw * (6 * c6 - 12 * c12 * rinv6) * rinv6 * rinv +
           dfsw * (c12 * rinv6 - c6) * rinv6;
      e += fsw * (c12 * rinv6 - c6) * rinv6;
    }
  } else { /* VSHIFT: nbdirect.cu:373-396 */
    double r2 = rEff * rEff, r5 = r2 * r2 * rEff, r6 = r2 * r2 * r2;
    double rinv7 = rinv6 * rinv, rinv12 = rinv6 * rinv6, rinv13 = rinv12 * rinv;
    double rc2 = rc * rc, rc6 = rc2 * rc2 * rc2, rc12 = rc6 * rc6, rc18 = rc12 * rc6;
    f += 6 * c6 * (rinv7 - r5 / rc12) - 12 * c12 * (rinv13 + r5 / rc18);
    e += c12 * (rinv12 + 2 * r6 / rc18 - 3 / rc12) - c6 * (rinv6 + r6 / rc12 - 2 / rc6);
  }
  *eij = e;
  *fij = f;
}

void orc_pair(double r, double qi, double qj, double c12, double c6,
              int bi, int bj, double li, double lj, const orc_params *p,
              double *E_scaled, double *fij_over_r, double *fli, double *flj) {
  double s = 1.0;
  *fli = 0;
  *flj = 0;
  if (p->calcAlch) { /* nbdirect.cu:244-254 */
    if ((bi & 0xFFFF0000) == (bj & 0xFFFF0000))
      s = (bi == bj) ? li : 0.0;
    else
      s = li * lj;
  }
  double rEff = r, dredr = 1, dredll = 0;
  if (p->calcAlch && p->useSoftCore && (bi || bj)) { /* nbdirect.cu:257-275 */
    double rSoft = p->softCoreRadius * (1 - s);
    if (r < rSoft) {
      double q = r / rSoft;
      double f = 0.5 + q * q * q * (1 - 0.5 * q);
      dredr = (3 - 2 * q) * q * q;
      dredll = -p->softCoreRadius * (f - dredr * q);
      rEff = f * rSoft;
    }
  }
  double eij, fij;
  pair_terms(rEff, p->kElectric * qi * qj, c12, c6, p, &eij, &fij);
  if (p->calcAlch) fij *= s;
  if (p->calcAlch && (bi || bj)) { /* nbdirect.cu:400-415 */
    double fl = eij + fij * dredll;
    if ((bi & 0xFFFF0000) == (bj & 0xFFFF0000)) {
      if (bi == bj) *fli = fl;
    } else {
      *fli = lj * fl;
      *flj = li * fl;
    }
  }
  fij *= dredr; /* nbdirect.cu:418-421 (dredr==1 without soft core) */
  *fij_over_r = fij / r;
  *E_scaled = p->calcAlch ? s * eij : eij;
}

/* ------------------------------------------------------------------------ */
/* Exclusion lookup: sorted array of undirected 64-bit keys                  */
/* ------------------------------------------------------------------------ */
static int cmp_u64(const void *a, const void *b) {
  uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
  return x < y ? -1 : (x > y ? 1 : 0);
}

typedef struct { uint64_t *k; int n; } excl_set;

static excl_set make_excl(int exclCount, const int *excl) {
  excl_set s;
  s.k = (uint64_t *)malloc(sizeof(uint64_t) * (exclCount > 0 ? exclCount : 1));
  int n = 0;
  for (int e = 0; e < exclCount; e++) {
    uint32_t a = (uint32_t)excl[2 * e], b = (uint32_t)excl[2 * e + 1];
    if (a == b) continue;
    uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    s.k[n++] = ((uint64_t)lo << 32) | hi;
  }
  qsort(s.k, n, sizeof(uint64_t), cmp_u64);
  int m = 0;
  for (int i = 0; i < n; i++)
    if (m == 0 || s.k[i] != s.k[m - 1]) s.k[m++] = s.k[i];
  s.n = m;
  return s;
}

static int is_excluded(const excl_set *s, int a, int b) {
  uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
  uint64_t key = ((uint64_t)lo << 32) | hi;
  int l = 0, h = s->n - 1;
  while (l <= h) {
    int m = (l + h) >> 1;
    if (s->k[m] == key) return 1;
    if (s->k[m] < key) l = m + 1; else h = m - 1;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Pair loops                                                                */
/* ------------------------------------------------------------------------ */
static inline double min_image(double d, double L) { return d - L * nearbyint(d / L); }

typedef struct {
  const double *xyz; const orc_nbond *nb; int nTypes; const orc_vdw *vdw;
  const orc_params *p; const double *lambda; int nLambda; double box[3];
  excl_set ex;
} pair_ctx;

static inline void do_pair(const pair_ctx *c, int i, int j, double *grad,
                           double *lf, double *energy, long long *count) {
  double dx = min_image(c->xyz[3 * i] - c->xyz[3 * j], c->box[0]);
  double dy = min_image(c->xyz[3 * i + 1] - c->xyz[3 * j + 1], c->box[1]);
  double dz = min_image(c->xyz[3 * i + 2] - c->xyz[3 * j + 2], c->box[2]);
  double r2 = dx * dx + dy * dy + dz * dz;
  if (!(r2 < c->p->rCut * c->p->rCut)) return;
  if (is_excluded(&c->ex, i, j)) return;
  double r = sqrt(r2);
  const orc_nbond a = c->nb[i], b = c->nb[j];
  orc_vdw v = c->vdw[a.typeIdx * c->nTypes + b.typeIdx];
  double li = 1, lj = 1;
  if (c->p->calcAlch) {
    if (a.siteBlock) li = c->lambda[a.siteBlock & 0xFFFF];
    if (b.siteBlock) lj = c->lambda[b.siteBlock & 0xFFFF];
  }
  double E, fr, fli, flj;
  orc_pair(r, a.q, b.q, v.c12, v.c6, a.siteBlock, b.siteBlock, li, lj, c->p, &E, &fr, &fli, &flj);
  grad[3 * i] += fr * dx; grad[3 * i + 1] += fr * dy; grad[3 * i + 2] += fr * dz;
  grad[3 * j] -= fr * dx; grad[3 * j + 1] -= fr * dy; grad[3 * j + 2] -= fr * dz;
  if (c->p->calcAlch) {
    if (a.siteBlock) lf[a.siteBlock & 0xFFFF] += fli;
    if (b.siteBlock) lf[b.siteBlock & 0xFFFF] += flj;
  }
  *energy += E;
  *count += 1;
}

int orc_nbdirect_brute64(int N, const double *xyz, const double box[3],
                         const orc_nbond *nb, int nTypes, const orc_vdw *vdw,
                         int exclCount, const int *excl, const orc_params *p,
                         const double *lambda, int nLambda,
                         double *grad, double *lambdaForce, double *energy,
                         long long *pairCount) {
  if (box[0] < 2 * p->rCut || box[1] < 2 * p->rCut || box[2] < 2 * p->rCut) return -1;
  pair_ctx c = {xyz, nb, nTypes, vdw, p, lambda, nLambda, {box[0], box[1], box[2]},
                make_excl(exclCount, excl)};
  memset(grad, 0, sizeof(double) * 3 * N);
  if (lambdaForce && nLambda > 0) memset(lambdaForce, 0, sizeof(double) * nLambda);
  double e = 0;
  long long n = 0;
  for (int i = 0; i < N; i++)
    for (int j = i + 1; j < N; j++) do_pair(&c, i, j, grad, lambdaForce, &e, &n);
  *energy = e;
  if (pairCount) *pairCount = n;
  free(c.ex.k);
  return 0;
}

int orc_nbdirect_window64(int N, const double *xyz, const double box[3],
                          const orc_nbond *nb, int nTypes, const orc_vdw *vdw,
                          int exclCount, const int *excl, const orc_params *p,
                          const double *lambda, int nLambda,
                          double *grad, double *lambdaForce, double *energy,
                          long long *pairCount, int nthreads, int i0, int i1) {
  if (box[0] < 2 * p->rCut || box[1] < 2 * p->rCut || box[2] < 2 * p->rCut) return -1;
  if (i0 < 0) i0 = 0;
  if (i1 > N) i1 = N;
  pair_ctx c = {xyz, nb, nTypes, vdw, p, lambda, nLambda, {box[0], box[1], box[2]},
                make_excl(exclCount, excl)};
  /* Cells at least rCut wide; at least 3 per side so the 27 neighbours are
   * distinct cells. */
  int nc[3];
  for (int d = 0; d < 3; d++) {
    nc[d] = (int)floor(box[d] / p->rCut);
    if (nc[d] < 3) nc[d] = 3;
  }
  int ncell = nc[0] * nc[1] * nc[2];
  int *head = (int *)malloc(sizeof(int) * ncell), *next = (int *)malloc(sizeof(int) * N);
  int *cellOf = (int *)malloc(sizeof(int) * N);
  for (int k = 0; k < ncell; k++) head[k] = -1;
  for (int i = N - 1; i >= 0; i--) {
    int ci[3];
    for (int d = 0; d < 3; d++) {
      double x = xyz[3 * i + d];
      x -= box[d] * floor(x / box[d]);
      int q = (int)(x / box[d] * nc[d]);
      if (q >= nc[d]) q = nc[d] - 1;
      if (q < 0) q = 0;
      ci[d] = q;
    }
    int cc = (ci[0] * nc[1] + ci[1]) * nc[2] + ci[2];
    cellOf[i] = cc;
    next[i] = head[cc];
    head[cc] = i;
  }
  int nt = 1;
#ifdef _OPENMP
  nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#endif
  double *g = (double *)calloc((size_t)nt * 3 * N, sizeof(double));
  int nl = nLambda > 0 ? nLambda : 1;
  double *lf = (double *)calloc((size_t)nt * nl, sizeof(double));
  double *et = (double *)calloc(nt, sizeof(double));
  long long *ct = (long long *)calloc(nt, sizeof(long long));
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64) num_threads(nt)
#endif
  for (int i = i0; i < i1; i++) {
    int t = 0;
#ifdef _OPENMP
    t = omp_get_thread_num();
#endif
    int cc = cellOf[i];
    int cz = cc % nc[2], cy = (cc / nc[2]) % nc[1], cx = cc / (nc[1] * nc[2]);
    for (int ox = -1; ox <= 1; ox++)
      for (int oy = -1; oy <= 1; oy++)
        for (int oz = -1; oz <= 1; oz++) {
          int x = (cx + ox + nc[0]) % nc[0], y = (cy + oy + nc[1]) % nc[1],
              z = (cz + oz + nc[2]) % nc[2];
          for (int j = head[(x * nc[1] + y) * nc[2] + z]; j >= 0; j = next[j])
            if (j > i) do_pair(&c, i, j, g + (size_t)t * 3 * N, lf + (size_t)t * nl, &et[t], &ct[t]);
        }
  }
  memset(grad, 0, sizeof(double) * 3 * N);
  if (lambdaForce && nLambda > 0) memset(lambdaForce, 0, sizeof(double) * nLambda);
  double e = 0;
  long long n = 0;
  for (int t = 0; t < nt; t++) {
    for (int k = 0; k < 3 * N; k++) grad[k] += g[(size_t)t * 3 * N + k];
    if (lambdaForce)
      for (int k = 0; k < nLambda; k++) lambdaForce[k] += lf[(size_t)t * nl + k];
    e += et[t];
    n += ct[t];
  }
  *energy = e;
  if (pairCount) *pairCount = n;
  free(g); free(lf); free(et); free(ct); free(head); free(next); free(cellOf);
  free(c.ex.k);
  return 0;
}

int orc_nbdirect64(int N, const double *xyz, const double box[3],
                   const orc_nbond *nb, int nTypes, const orc_vdw *vdw,
                   int exclCount, const int *excl, const orc_params *p,
                   const double *lambda, int nLambda,
                   double *grad, double *lambdaForce, double *energy,
                   long long *pairCount, int nthreads) {
  return orc_nbdirect_window64(N, xyz, box, nb, nTypes, vdw, exclCount, excl, p, lambda,
                               nLambda, grad, lambdaForce, energy, pairCount, nthreads, 0, N);
}

static double *promote(int N, const float *xyz) {
  double *x = (double *)malloc(sizeof(double) * 3 * (N > 0 ? N : 1));
  for (int k = 0; k < 3 * N; k++) x[k] = xyz[k];
  return x;
}

int orc_nbdirect(int N, const float *xyz, const double box[3],
                 const orc_nbond *nb, int nTypes, const orc_vdw *vdw,
                 int exclCount, const int *excl, const orc_params *p,
                 const double *lambda, int nLambda,
                 double *grad, double *lambdaForce, double *energy,
                 long long *pairCount, int nthreads) {
  double *x = promote(N, xyz);
  int rc = orc_nbdirect64(N, x, box, nb, nTypes, vdw, exclCount, excl, p, lambda, nLambda,
                          grad, lambdaForce, energy, pairCount, nthreads);
  free(x);
  return rc;
}

/* Triclinic cell (box6: A_x, B_y, C_z, B_x, C_x, C_y): every pair i<j over
 * all lattice images within rCut.  The difference is first reduced as the
 * reference's real3_subpbc<true> (src/main/real3.h:215-240: by C, then B,
 * then A), then the 27 images around it are tested; with A_x, B_y, C_z >=
 * 2 rCut at most one of them lies inside rCut. */
int orc_nbdirect_tric64(int N, const double *xyz, const double box6[6],
                        const orc_nbond *nb, int nTypes, const orc_vdw *vdw,
                        int exclCount, const int *excl, const orc_params *p,
                        const double *lambda, int nLambda,
                        double *grad, double *lambdaForce, double *energy,
                        long long *pairCount) {
  const double ax = box6[0], by = box6[1], cz = box6[2], bx = box6[3], cx = box6[4], cy = box6[5];
  if (ax < 2 * p->rCut || by < 2 * p->rCut || cz < 2 * p->rCut) return -1;
  excl_set ex = make_excl(exclCount, excl);
  memset(grad, 0, sizeof(double) * 3 * N);
  if (lambdaForce && nLambda > 0) memset(lambdaForce, 0, sizeof(double) * nLambda);
  const double rc2 = p->rCut * p->rCut;
  double e = 0;
  long long n = 0;
  for (int i = 0; i < N; i++)
    for (int j = i + 1; j < N; j++) {
      double d0[3] = {xyz[3 * i] - xyz[3 * j], xyz[3 * i + 1] - xyz[3 * j + 1], xyz[3 * i + 2] - xyz[3 * j + 2]};
      double k = floor(d0[2] / cz + 0.5);
      d0[0] -= cx * k; d0[1] -= cy * k; d0[2] -= cz * k;
      k = floor(d0[1] / by + 0.5);
      d0[0] -= bx * k; d0[1] -= by * k;
      d0[0] -= ax * floor(d0[0] / ax + 0.5);
      for (int c = -1; c <= 1; c++)
        for (int b = -1; b <= 1; b++)
          for (int a = -1; a <= 1; a++) {
            const double dx = d0[0] + a * ax + b * bx + c * cx;
            const double dy = d0[1] + b * by + c * cy;
            const double dz = d0[2] + c * cz;
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (!(r2 < rc2) || is_excluded(&ex, i, j)) continue;
            const double r = sqrt(r2);
            const orc_nbond A = nb[i], Bn = nb[j];
            const orc_vdw v = vdw[A.typeIdx * nTypes + Bn.typeIdx];
            double li = 1, lj = 1;
            if (p->calcAlch) {
              if (A.siteBlock) li = lambda[A.siteBlock & 0xFFFF];
              if (Bn.siteBlock) lj = lambda[Bn.siteBlock & 0xFFFF];
            }
            double E, fr, fli, flj;
            orc_pair(r, A.q, Bn.q, v.c12, v.c6, A.siteBlock, Bn.siteBlock, li, lj, p, &E, &fr, &fli, &flj);
            grad[3 * i] += fr * dx; grad[3 * i + 1] += fr * dy; grad[3 * i + 2] += fr * dz;
            grad[3 * j] -= fr * dx; grad[3 * j + 1] -= fr * dy; grad[3 * j + 2] -= fr * dz;
            if (p->calcAlch) {
              if (A.siteBlock) lambdaForce[A.siteBlock & 0xFFFF] += fli;
              if (Bn.siteBlock) lambdaForce[Bn.siteBlock & 0xFFFF] += flj;
            }
            e += E;
            n++;
          }
    }
  *energy = e;
  if (pairCount) *pairCount = n;
  free(ex.k);
  return 0;
}

int orc_nbdirect_brute(int N, const float *xyz, const double box[3],
                       const orc_nbond *nb, int nTypes, const orc_vdw *vdw,
                       int exclCount, const int *excl, const orc_params *p,
                       const double *lambda, int nLambda,
                       double *grad, double *lambdaForce, double *energy,
                       long long *pairCount) {
  double *x = promote(N, xyz);
  int rc = orc_nbdirect_brute64(N, x, box, nb, nTypes, vdw, exclCount, excl, p, lambda,
                                nLambda, grad, lambdaForce, energy, pairCount);
  free(x);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* MSLD lambda maps and biases                                               */
/* ------------------------------------------------------------------------ */
void orc_lambda_from_theta(int siteCount, const int *siteBound, double fnex,
                           const double *theta, const int *blockFixed,
                           double *lambda) {
  for (int i = 0; i < siteCount; i++) { /* msld.cu:874-898 */
    int ji = siteBound[i], jf = siteBound[i + 1];
    double fixsum = 0, norm = 0;
    for (int j = ji; j < jf; j++) {
      if (blockFixed && blockFixed[j]) {
        fixsum += theta[j];
      } else {
        lambda[j] = exp(fnex * sin(theta[j]));
        norm += lambda[j];
      }
    }
    double rfrac = 1.0 - fixsum;
    if (norm > 0) norm = rfrac / norm;
    for (int j = ji; j < jf; j++)
      lambda[j] = (blockFixed && blockFixed[j]) ? theta[j] : lambda[j] * norm;
  }
}

void orc_thetaForce_from_lambdaForce(int blockCount, const int *lambdaSite,
                                     const int *siteBound, double fnex,
                                     const double *lambda, const double *theta,
                                     const double *lambdaForce,
                                     const int *blockFixed, double *thetaForce) {
  for (int i = 0; i < blockCount; i++) { /* msld.cu:949-972 */
    thetaForce[i] = 0;
    if (blockFixed && blockFixed[i]) continue;
    int ji = siteBound[lambdaSite[i]], jf = siteBound[lambdaSite[i] + 1];
    double fixsum = 0, dyn = 0;
    for (int j = ji; j < jf; j++) {
      if (blockFixed && blockFixed[j]) fixsum += lambda[j];
      else dyn += lambda[j] * lambdaForce[j];
    }
    double fi = lambdaForce[i];
    double rfrac = 1.0 - fixsum;
    if (rfrac > 0) fi = fi - dyn / rfrac;
    thetaForce[i] = fi * lambda[i] * fnex * cos(theta[i]);
  }
}

void orc_bias(int blockCount, const double *lambda, const double *fixedBias,
              int nVar, const orc_varbias *vb, double *lambdaForce,
              double *energy) {
  double e = 0;
  if (fixedBias) /* msld.cu:1000-1018 */
    for (int i = 0; i < blockCount; i++) {
      lambdaForce[i] += fixedBias[i];
      e += fixedBias[i] * lambda[i];
    }
  for (int b = 0; b < nVar; b++) { /* msld.cu:1042-1139 */
    const orc_varbias v = vb[b];
    double li = lambda[v.i], lj = lambda[v.j], k = v.k, l0 = v.l0, n = v.n;
    double E = 0, fi = 0, fj = 0;
    switch (v.type) {
      case 6: E = k * li * lj; fi = k * lj; fj = k * li; break;
      case 8: E = k * li * lj / (li + l0); fi = k * l0 * lj / ((li + l0) * (li + l0));
              fj = k * li / (li + l0); break;
      case 10: E = k * lj * (1 - exp(l0 * li)); fi = k * lj * (-l0 * exp(l0 * li));
               fj = k * (1 - exp(l0 * li)); break;
      case 1: E = li < l0 ? k * pow(li - l0, n) : 0; fi = li < l0 ? n * k * pow(li - l0, n - 1) : 0; break;
      case 2: E = li > l0 ? k * pow(li - l0, n) : 0; fi = li > l0 ? n * k * pow(li - l0, n - 1) : 0; break;
      case 3: E = k * pow(li - lj, n); fi = n * k * pow(li - lj, n - 1); fj = -fi; break;
      case 4: E = li > l0 ? -k : -k * (1 - (li - l0) * (li - l0) / (l0 * l0));
              fi = li > l0 ? 0 : 2 * k * (li - l0) / (l0 * l0); break;
      case 5: E = -k * li; fi = -k; break;
      case 7: E = k * li * (1 - li) / (li + l0); fi = k * (l0 * (1 + l0) / ((li + l0) * (li + l0)) - 1); break;
      case 9: E = k * lj * (1 - pow((li + l0) / l0, n)); fi = -k * lj * pow((li + l0) / l0, n - 1) / l0;
              fj = k * (1 - pow((li + l0) / l0, n)); break;
      case 11: E = k * pow(li, l0) * pow(lj, n); fi = k * l0 * pow(li, l0 - 1) * pow(lj, n);
               fj = k * n * pow(li, l0) * pow(lj, n - 1); break;
      case 12: E = k * li * pow(lj, n) / (li + l0); fi = k * l0 * pow(lj, n) / ((li + l0) * (li + l0));
               fj = k * n * li * pow(lj, n - 1) / (li + l0); break;
      default: break;
    }
    lambdaForce[v.i] += fi;
    lambdaForce[v.j] += fj;
    e += E;
  }
  if (energy) *energy += e;
}

/* ===========================================================================
 * nb14 / nbex pair lists: FP64 restatement of src/bonded/pair.cu.
 * ======================================================================== */

/* function_pair(Nb14Potential...), pair.cu:63-187: dE/dr and E. */
static void nb14_terms(const orc_nb14 *pp, const orc_params *p, double r, double *fpair, double *E) {
  *fpair = 0;
  *E = 0;
  if (!(r < p->rCut)) return;
  const double rinv = 1 / r, rinv3 = rinv * rinv * rinv, rinv6 = rinv3 * rinv3;
  const double c12 = pp->c12, c6 = pp->c6, rc = p->rCut, rs = p->rSwitch;
  if (p->vdwMethod == 0) { /* VFSWITCH, pair.cu:70-93 */
    const double rc3 = rc * rc * rc, rc6 = rc3 * rc3, rs3 = rs * rs * rs, rs6 = rs3 * rs3;
    const double k6 = rc3 / (rc3 - rs3), k12 = rc6 / (rc6 - rs6);
    const int in = r < rs;
    const double A6 = in ? 1 : k6, A12 = in ? 1 : k12, B6 = in ? 0 : 1 / rc3, B12 = in ? 0 : 1 / rc6;
    *fpair = 6 * c6 * A6 * (rinv3 - B6) * rinv3 * rinv - 12 * c12 * A12 * (rinv6 - B12) * rinv6 * rinv;
    const double CC6 = in ? -1 / rc6 : 0, CC12 = in ? -1 / (rc6 * rc6) : 0;
    *E = c12 * (A12 * (rinv6 - B12) * (rinv6 - B12) + CC12) - c6 * (A6 * (rinv3 - B6) * (rinv3 - B6) + CC6);
  } else if (p->vdwMethod == 1) { /* VSWITCH, pair.cu:94-106 (force expression as written) */
    const double c2of = rc * rc, c2on = rs * rs;
    const double rul3 = (c2of - c2on) * (c2of - c2on) * (c2of - c2on), rul12 = 12 / rul3;
    const double rijl = c2on - r * r, riju = c2of - r * r;
    const double fsw = r < rs ? 1 : riju * riju * (riju - 3 * rijl) / rul3;
    const double dfsw = r < rs ? 0 : rijl * riju * rul12;
    *fpair = fsw * (6 * c6 - 12 * c12 * rinv6) * rinv6 * rinv + dfsw * (c12 * rinv6 - c6) * rinv6;
    *E = fsw * (c12 * rinv6 - c6) * rinv6;
  } else { /* VSHIFT, pair.cu:107-133 (as written) */
    const double r2 = r * r, r5 = r2 * r2 * r, r6 = r2 * r2 * r2;
    const double rinv7 = rinv6 * rinv, rinv12 = rinv6 * rinv6, rinv13 = rinv12 * rinv;
    const double rc2 = rc * rc, rc6 = rc2 * rc2 * rc2, rc12 = rc6 * rc6, rc18 = rc12 * rc6;
    *fpair = 6 * c6 * (rinv7 - r5 / rc12) - 12 * c12 * (rinv13 + r5 / rc18);
    *E = c12 * (rinv12 + 2 * r6 / rc18 - 3 / rc12) - c6 * (rinv6 + r6 / rc12 - 2 / rc6);
  }
  const double kqq = p->kElectric * pp->qxq;
  if (p->elecMethod == 0) { /* FSWITCH, pair.cu:136-156 */
    const double kqqe14 = kqq * pp->e14fac;
    const double roff2 = rc * rc, ron2 = rs * rs;
    const double ginv = 1 / ((roff2 - ron2) * (roff2 - ron2) * (roff2 - ron2));
    const double A = roff2 * roff2 * (roff2 - 3 * ron2) * ginv, B = 6 * roff2 * ron2 * ginv;
    const double Cc = -(ron2 + roff2) * ginv, D = 2 * ginv / 5;
    const double dvc = 8 * (ron2 * roff2 * (rc - rs) - (roff2 * roff2 * rc - ron2 * ron2 * rs) / 5) * ginv;
    const double r2 = r * r, r3 = r2 * r, r5 = r3 * r2;
    *fpair += r <= rs ? -kqqe14 * rinv * rinv : -kqqe14 * rinv * (A * rinv + B * r + 3 * Cc * r3 + 5 * D * r5);
    *E += r <= rs ? kqqe14 * (rinv + dvc)
                  : kqqe14 * (A * (rinv - 1 / rc) + B * (rc - r) + Cc * (roff2 * rc - r3) + D * (roff2 * roff2 * rc - r5));
  } else if (p->elecMethod == 1) { /* PME, pair.cu:157-165: erfc(br) + e14fac - 1 */
    const double br = p->betaEwald * r;
    const double erfcrinv = (erfc(br) + pp->e14fac - 1) * rinv;
    *fpair += kqq * (-erfcrinv - 2 / sqrt(M_PI) * p->betaEwald * exp(-br * br)) * rinv;
    *E += kqq * erfcrinv;
  } else { /* FSHIFT, pair.cu:166-174 */
    const double kqqe14 = kqq * pp->e14fac, roffinv = 1 / rc;
    *fpair += -kqqe14 * (rinv * rinv - roffinv * roffinv);
    *E += kqqe14 * (rinv - 2 * roffinv + r * roffinv * roffinv);
  }
}

/* box: A_x, B_y, C_z, B_x, C_x, C_y; the reference's real3_subpbc (by C, then
 * B, then A; per axis for an orthorhombic box, src/main/real3.h:215-240). */
static void pl_min_image(const double *xi, const double *xj, const double box[6], double d[3]) {
  for (int k = 0; k < 3; k++) d[k] = xi[k] - xj[k];
  double k = nearbyint(d[2] / box[2]);
  d[0] -= box[4] * k; d[1] -= box[5] * k; d[2] -= box[2] * k;
  k = nearbyint(d[1] / box[1]);
  d[0] -= box[3] * k; d[1] -= box[1] * k;
  d[0] -= box[0] * nearbyint(d[0] / box[0]);
}

/* getforce_pair_kernel's scaling, soft core and routing (pair.cu:205-283). */
static void pair_apply(int ii, int jj, const int sb[2], const double d[3], double r, double rEff, double dredr,
                       double dredll, int soft, double fpair, double E, const double *lambda, double *grad,
                       double *lambdaForce, double *energy) {
  int b0 = 0xFFFF & sb[0], b1 = 0xFFFF & sb[1];
  double l0 = 1, l1 = 1;
  if (b0) {
    l0 = lambda[b0];
    if (b1) l1 = lambda[b1];
  }
  (void)rEff;
  fpair *= l0 * l1;
  if (b0) {
    const double fl = soft ? E + fpair * dredll : E;
    lambdaForce[b0] += l1 * fl;
    if (b1) lambdaForce[b1] += l0 * fl;
  }
  if (soft) fpair *= dredr;
  for (int k = 0; k < 3; k++) {
    grad[3 * ii + k] += fpair / r * d[k];
    grad[3 * jj + k] -= fpair / r * d[k];
  }
  energy[0] += E * l0 * l1;
}

void orc_nb14_pairs(int n, const orc_nb14 *pp, const double *xyz, const double box[6], const double *lambda,
                    const orc_params *p, int useSoftCore14, double *grad, double *lambdaForce, double *energy) {
  for (int t = 0; t < n; t++) {
    const int ii = pp[t].idx[0], jj = pp[t].idx[1];
    double d[3];
    pl_min_image(xyz + 3 * ii, xyz + 3 * jj, box, d);
    const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    int b0 = 0xFFFF & pp[t].siteBlock[0], b1 = 0xFFFF & pp[t].siteBlock[1];
    double l0 = 1, l1 = 1;
    if (b0) {
      l0 = lambda[b0];
      if (b1) l1 = lambda[b1];
    }
    double rEff = r, dredr = 1, dredll = 0;
    if (useSoftCore14 && b0) { /* pair.cu:240-254 */
      const double rSoft = p->softCoreRadius * (1 - l0 * l1);
      if (r < rSoft) {
        const double q = r / rSoft;
        rEff = (1 - 0.5 * q) * q * q * q + 0.5;
        dredr = (3 - 2 * q) * q * q;
        dredll = -p->softCoreRadius * (rEff - dredr * q);
        rEff *= rSoft;
      }
    }
    double fpair, E;
    nb14_terms(&pp[t], p, rEff, &fpair, &E);
    pair_apply(ii, jj, pp[t].siteBlock, d, r, rEff, dredr, dredll, useSoftCore14, fpair, E, lambda, grad,
               lambdaForce, energy);
  }
}

void orc_nbex_pairs(int n, const orc_nbex *pp, const double *xyz, const double box[6], const double *lambda,
                    const orc_params *p, double *grad, double *lambdaForce, double *energy) {
  for (int t = 0; t < n; t++) {
    const int ii = pp[t].idx[0], jj = pp[t].idx[1];
    double d[3];
    pl_min_image(xyz + 3 * ii, xyz + 3 * jj, box, d);
    const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    /* function_pair(NbExPotential...), pair.cu:190-202: -kqq erf(br)/r */
    const double br = p->betaEwald * r, kqq = p->kElectric * pp[t].qxq;
    const double fpair = kqq * (erf(br) / r - 2 / sqrt(M_PI) * p->betaEwald * exp(-br * br)) / r;
    const double E = -kqq * erf(br) / r;
    pair_apply(ii, jj, pp[t].siteBlock, d, r, r, 1, 0, 0, fpair, E, lambda, grad, lambdaForce, energy);
  }
}
