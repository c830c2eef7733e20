/*
 * CPU oracle for BLaDE's nonbonded direct-space path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (libbnb.so, the host
 * wrappers) links, loads or calls this code.  It is used by the tests as the
 * checker, by bench.py as the timed CPU baseline, and by __graft_entry__.smoke()
 * as the reference for one small case.
 *
 * Two halves:
 *   1. FP64 restatement of the pair physics of src/nbdirect/nbdirect.cu:232-433
 *      (all elecMethod/vdwMethod branches, MSLD lambda scaling and soft core),
 *      the MSLD theta<->lambda maps (src/msld/msld.cu:863-998) and the lambda
 *      biases (src/msld/msld.cu:1000-1153).  Exact erfc/exp from libm.
 *   2. FP32/integer restatement of the block neighbour list (binning, column
 *      sort, 32-atom blocks, AABBs, half-shell culling, 32x32 exclusion masks)
 *      following src/domdec/assign_blocks.cu, cull.cu, recull.cu and
 *      assign_excl.cu, with a deterministic tie rule.  The CUDA builder must
 *      reproduce it bit for bit.
 */
#ifndef BNB_ORACLE_H
#define BNB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as struct NbondPotential, src/system/potential.h:106-110. */
typedef struct { int siteBlock; float q; int typeIdx; } orc_nbond;
/* Same layout as struct VdwPotential, src/system/potential.h:112-114. */
typedef struct { float c12, c6; } orc_vdw;

typedef struct {
  double rCut, rSwitch, betaEwald;
  int elecMethod;      /* 0 FSWITCH, 1 PME, 2 FSHIFT   (src/run/run.h:28-32) */
  int vdwMethod;       /* 0 VFSWITCH, 1 VSWITCH, 2 VSHIFT (src/run/run.h:34-38) */
  int calcAlch;        /* blockCount>1 in src/nbdirect/nbdirect.cu:565 */
  int useSoftCore;
  double kElectric;    /* 332.0716 in AKMA (src/main/defines.h:55) */
  double softCoreRadius; /* 4.0 A in AKMA (src/main/defines.h:48) */
} orc_params;

/*
 * Direct-space energy, gradient (dU/dx, the quantity BLaDE stores in force_d)
 * and dU/dlambda over all non-excluded minimum-image pairs with r<rCut.
 * xyz: 3N floats (FP32 coordinates, promoted to double).  box: orthorhombic
 * edge lengths.  lambda: per MSLD block (index = siteBlock&0xFFFF), ignored when
 * calcAlch==0.  excl: exclCount directed pairs (both orders may be present).
 * Outputs are OVERWRITTEN: grad[3N], lambdaForce[nLambda], energy[1],
 * pairCount[1] (pairs with r<rCut that were evaluated).  nthreads<=0: all.
 * Returns 0, or -1 if the box is smaller than 2*rCut.
 */
int orc_nbdirect(int N, const float *xyz, const double box[3],
                 const orc_nbond *nb, int nTypes, const orc_vdw *vdw,
                 int exclCount, const int *excl, const orc_params *p,
                 const double *lambda, int nLambda,
                 double *grad, double *lambdaForce, double *energy,
                 long long *pairCount, int nthreads);

/* Only pairs (i,j>i) with i in [i0,i1): a bounded sample for CPU timing. */
int orc_nbdirect_window64(int N, const double *xyz, const double box[3],
                          const orc_nbond *nb, int nTypes, const orc_vdw *vdw,
                          int exclCount, const int *excl, const orc_params *p,
                          const double *lambda, int nLambda,
                          double *grad, double *lambdaForce, double *energy,
                          long long *pairCount, int nthreads, int i0, int i1);

/* Same with FP64 coordinates (finite-difference tests). */
int orc_nbdirect64(int N, const double *xyz, const double box[3],
                   const orc_nbond *nb, int nTypes, const orc_vdw *vdw,
                   int exclCount, const int *excl, const orc_params *p,
                   const double *lambda, int nLambda,
                   double *grad, double *lambdaForce, double *energy,
                   long long *pairCount, int nthreads);
int orc_nbdirect_tric64(int N, const double *xyz, const double box6[6],
                        const orc_nbond *nb, int nTypes, const orc_vdw *vdw,
                        int exclCount, const int *excl, const orc_params *p,
                        const double *lambda, int nLambda,
                        double *grad, double *lambdaForce, double *energy,
                        long long *pairCount);
int orc_nbdirect_brute64(int N, const double *xyz, const double box[3],
                         const orc_nbond *nb, int nTypes, const orc_vdw *vdw,
                         int exclCount, const int *excl, const orc_params *p,
                         const double *lambda, int nLambda,
                         double *grad, double *lambdaForce, double *energy,
                         long long *pairCount);

/* Same, by O(N^2) minimum-image loop (independent check of the cell list). */
int orc_nbdirect_brute(int N, const float *xyz, const double box[3],
                       const orc_nbond *nb, int nTypes, const orc_vdw *vdw,
                       int exclCount, const int *excl, const orc_params *p,
                       const double *lambda, int nLambda,
                       double *grad, double *lambdaForce, double *energy,
                       long long *pairCount);

/* One pair, for unit tests: energy (unscaled eij), dE/dr (scaled by s) and
 * the lambda derivative routing.  Mirrors nbdirect.cu:242-433. */
void orc_pair(double r, double qi, double qj, double c12, double c6,
              int bi, int bj, double li, double lj, const orc_params *p,
              double *E_scaled, double *fij_over_r, double *fli, double *flj);

/* ---- MSLD lambda kernels (FP64) ----------------------------------------- */
/* src/msld/msld.cu:863-908 (non-fixed, non-implicit branch). */
void orc_lambda_from_theta(int siteCount, const int *siteBound, double fnex,
                           const double *theta, const int *blockFixed,
                           double *lambda);
/* src/msld/msld.cu:937-985. thetaForce is OVERWRITTEN. */
void orc_thetaForce_from_lambdaForce(int blockCount, const int *lambdaSite,
                                     const int *siteBound, double fnex,
                                     const double *lambda, const double *theta,
                                     const double *lambdaForce,
                                     const int *blockFixed, double *thetaForce);
/* src/msld/msld.cu:1000-1018 and 1042-1153: ADDS to lambdaForce and energy. */
typedef struct { int i, j, type; float l0, k; int n; } orc_varbias; /* msld.h:13-19 */
void orc_bias(int blockCount, const double *lambda, const double *fixedBias,
              int nVar, const orc_varbias *vb, double *lambdaForce,
              double *energy);

/* ---- Block neighbour list (FP32 / integer, bit-exact target) ------------ */
typedef struct {
  int N, divX, divY, nCols;
  int blockCount;        /* B */
  int *wrap;             /* [N] packed image shift (sx+128)|(sy+128)<<8|(sz+128)<<16 */
  int *colCount;         /* [nCols] */
  int *blockBounds;      /* [B+1] in sorted order */
  int *sortedAtom;       /* [N] localToGlobal */
  int *slotAtom;         /* [32B] atom or -1 */
  float *bmin, *bmax;    /* [3B] AABBs */
  int candCount;
  int *candStart;        /* [B+1] CSR over candidates */
  int *cand;             /* [candCount*2] (jBlock, shiftCode) */
  int *candExcl;         /* [candCount] mask index or -1 */
  int maskCount;
  uint32_t *masks;       /* [maskCount*32] */
} orc_list;

/* Heuristic column counts, src/domdec/domdec.cu:114-117. */
void orc_domain_div(int N, const float box[3], int *divX, int *divY);
/* Build the list with culling distance rCull (=rCut+pad).  The exclusion
 * list is CSR over atoms (exclStart[N+1], exclAtom[]) sorted per atom. */
/* box: A_x, B_y, C_z, B_x, C_x, C_y (the last three zero for an orthorhombic
 * box): the lower-triangular cell of the reference's State::tricBox. */
int orc_build_list(int N, const float *xyz, const float box[6], float rCull,
                   const int *exclStart, const int *exclAtom, orc_list *out);
void orc_free_list(orc_list *l);
/* Pack positions with the stored wrap shift and recompute AABBs
 * (assign_blocks.cu:340-382). */
void orc_shift_table(const float box[6], float table[14][3]);
void orc_lattice_shift(const float box[6], int sx, int sy, int sz, float out[3]);
void orc_pack(const orc_list *l, const float *xyz, const float box[6],
              float *packed /* [32B*3] */, float *bmin, float *bmax);
/* Shift code (0..13) -> integer shift, half shell of cull.cu:127-173. */
void orc_shift_vector(int code, int *sx, int *sy, int *sz);
/* AABB gap^2 test, fixed FP32 operation order shared with the CUDA code. */
int orc_aabb_hit(const float *imin, const float *imax, const float *jmin,
                 const float *jmax, const float shift[3], float c2);

/* ---- nb14 / nbex pair lists (src/bonded/pair.cu:63-286) ---------------- */
/* Same layouts as struct Nb14Potential / NbExPotential, src/system/potential.h:91-104. */
typedef struct { int idx[2]; int siteBlock[2]; float qxq, c12, c6, e14fac; } orc_nb14;
typedef struct { int idx[2]; int siteBlock[2]; float qxq; } orc_nbex;

/*
 * FP64 restatement of getforce_pair_kernel with function_pair for
 * Nb14Potential (pair.cu:63-187: switched LJ and e14fac-scaled elec) and for
 * NbExPotential (pair.cu:190-202: the PME erf correction of excluded pairs),
 * MSLD scaling l0*l1 and, for nb14 with useSoftCore14, the soft core
 * (pair.cu:205-283).  Minimum image in the cell box (A_x, B_y, C_z, B_x, C_x,
 * C_y; the last three zero for an orthorhombic box).  Outputs are
 * ADDED: grad[3N] (dU/dx), lambdaForce, energy[1].
 */
void orc_nb14_pairs(int n, const orc_nb14 *pp, const double *xyz, const double box[6],
                    const double *lambda, const orc_params *p, int useSoftCore14,
                    double *grad, double *lambdaForce, double *energy);
void orc_nbex_pairs(int n, const orc_nbex *pp, const double *xyz, const double box[6],
                    const double *lambda, const orc_params *p,
                    double *grad, double *lambdaForce, double *energy);

#ifdef __cplusplus
}
#endif
#endif
