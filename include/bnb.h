/*
 * libbnb -- B200-native nonbonded direct space for BLaDE (C ABI).
 *
 * Replaces BLaDE's nonbonded direct-space path: the pair-force routine
 * getforce_nbdirect (src/nbdirect/nbdirect.h:7) fed by the Domdec neighbour
 * list (src/domdec/domdec.h:93-110) and scaled by the Msld lambda blocks
 * (src/msld/msld.h:134-139).  Plain C types only: every array argument is a
 * device pointer unless its comment says "host", streams are cudaStream_t
 * passed as void*, and every function returns 0 or a BNB_ERR_* code.  No
 * function exits, traps or prints.
 *
 * Units follow the caller (AKMA by default: A, kcal/mol).  "force" arrays hold
 * dU/dx, the quantity BLaDE keeps in State::force_d.
 */
#ifndef BNB_H
#define BNB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes ------------------------------------------------------ */
#define BNB_OK 0
#define BNB_ERR_ARG 1          /* bad argument (null, size, method)          */
#define BNB_ERR_CUDA 2         /* a CUDA call failed                         */
#define BNB_ERR_CAPACITY 3     /* list capacity exceeded and could not grow  */
#define BNB_ERR_UNSUPPORTED 4  /* feature this library does not implement     */
#define BNB_ERR_STATE 5        /* call order (e.g. compute before rebuild)   */
#define BNB_ERR_DEVICE 6       /* device status word reports a failure       */
#define BNB_ERR_TOO_LARGE 7    /* size above a fixed limit of this library   */

/* ---- device status bits (bnb_status) ------------------------------------ */
#define BNB_STATUS_BLOCK_OVERFLOW 1
#define BNB_STATUS_TILE_OVERFLOW 2
#define BNB_STATUS_MASK_OVERFLOW 4
#define BNB_STATUS_WORK_OVERFLOW 8
#define BNB_STATUS_NONFINITE 16

/* Same layout as struct NbondPotential, src/system/potential.h:106-110. */
typedef struct { int siteBlock; float q; int typeIdx; } bnb_nbond;
/* Same layout as struct VdwPotential, src/system/potential.h:112-114. */
typedef struct { float c12, c6; } bnb_vdw;
/* Same layouts as struct Nb14Potential / NbExPotential, src/system/potential.h:91-104. */
typedef struct { int idx[2]; int siteBlock[2]; float qxq, c12, c6, e14fac; } bnb_nb14;
typedef struct { int idx[2]; int siteBlock[2]; float qxq; } bnb_nbex;
/* Same layout as struct VariableBias, src/msld/msld.h:13-19. */
typedef struct { int i, j, type; float l0, k; int n; } bnb_varbias;

/*
 * Run parameters of the path: Cutoffs{betaEwald,rCut,rSwitch}
 * (src/run/run.h:16-20), elecMethod/vdwMethod (run.h:28-38), the MSLD
 * soft-core flag (src/msld/msld.h:89) and the list pad
 * (Domdec::cullPad, src/domdec/domdec.cu:138).
 */
typedef struct {
  float rCut, rSwitch, betaEwald;
  int elecMethod;        /* 0 FSWITCH, 1 PME, 2 FSHIFT */
  int vdwMethod;         /* 0 VFSWITCH, 1 VSWITCH, 2 VSHIFT */
  int useSoftCore;
  float cullPad;         /* list buffer in length units (reference: computed) */
  float kElectric;       /* 332.0716 AKMA, 138.935455103336 NMPS (defines.h) */
  float softCoreRadius;  /* 4.0 AKMA, 0.4 NMPS (defines.h:48,74) */
} bnb_params;

/* Fills defaults: AKMA units, PME + VFSWITCH, rCut 12, rSwitch 10, beta 0.32,
 * soft core on, pad 2. */
void bnb_default_params(bnb_params *p);

typedef struct bnb_handle bnb_handle;

/*
 * Creates a handle for `replicas` independent systems that share `p`.
 * atomCounts: host [replicas].  Allocates device memory on the current device
 * (the counterpart of Domdec::initialize, src/domdec/domdec.cu:83-199).
 */
int bnb_create(const bnb_params *p, int replicas, const int *atomCounts,
               bnb_handle **out);
int bnb_destroy(bnb_handle *h);

/*
 * Topology of all replicas, concatenated (host arrays):
 *   nbonds[N]   per-atom {siteBlock,q,typeIdx}; siteBlock=(site<<16)|block
 *               with blocks numbered within each replica (Msld::nbond_scaling,
 *               src/msld/msld.cu:670-673); typeIdx indexes that replica's table.
 *   typeCounts  host [replicas]; vdw: concatenated per-replica tables of
 *               typeCounts[r]^2 entries (Potential::vdwParameters,
 *               src/system/potential.cxx:1369-1403).
 *   lambdaCounts host [replicas]: MSLD blocks per replica (1 = no alchemy).
 *   excl[2*exclCount] directed atom pairs, atom indices local to their replica,
 *               replica given by exclReplica[exclCount] (Potential::excls,
 *               src/system/potential.cxx:1156-1163).  exclReplica may be NULL
 *               when replicas==1.
 */
int bnb_set_topology(bnb_handle *h, const bnb_nbond *nbonds,
                     const int *typeCounts, const bnb_vdw *vdw,
                     const int *lambdaCounts, int exclCount, const int *excl,
                     const int *exclReplica);

/*
 * Box shape of every boxes argument of this handle (State::typeBox,
 * src/system/state.h): 0 (default) orthorhombic, boxes are host float
 * [3*replicas] edge lengths (State::orthBox_f); 1 triclinic, boxes are host
 * float [6*replicas] in the layout of State::tricBox_f: A_x, B_x, B_y, C_x,
 * C_y, C_z of the lower-triangular cell A = (A_x,0,0), B = (B_x,B_y,0),
 * C = (C_x,C_y,C_z).  Atoms are wrapped into the brick A_x x B_y x C_z as the
 * reference's triclinic modulus does (src/main/real3.h:340-360), and the
 * half-shell images are centred under the shear as its cull does
 * (src/domdec/cull.cu:141-190); A_x, B_y and C_z must each be at least
 * 2 rCut.  Direct space, nb14/nbex, the list and PME reciprocal space (the
 * reference's flagBox branch of getforce_ewald) all take the cell.  Changing
 * the type requires a synchronous rebuild.
 */
int bnb_set_box_type(bnb_handle *h, int triclinic);

/*
 * Rebuilds the block list from coordinates (the counterpart of
 * Domdec::reset_domdec, src/domdec/domdec.cu:201-211: bin, sort, 32-atom
 * blocks, AABBs, half-shell cull at rCut+cullPad, exclusion masks).
 * position: device float [3N] (State::position_fd layout, all replicas).
 * boxes: host float [3*replicas] orthorhombic edges, or [6*replicas]
 * triclinic cells after bnb_set_box_type(h, 1).
 * flags: 0 = synchronise and grow capacities on overflow (as the reference's
 * cull loop, src/domdec/cull.cu:337-375); BNB_ASYNC = enqueue only (graph
 * capturable), overflow is reported through bnb_status and the pair kernel
 * then does no work.
 */
#define BNB_ASYNC 1
int bnb_rebuild(bnb_handle *h, const float *position, const float *boxes,
                void *stream, int flags);

/*
 * One direct-space evaluation (getforce_nbdirect, src/nbdirect/nbdirect.cu:574;
 * pack_positions + recull_blocks + kernel + unpack_forces, :492-526).
 * position: device float [3N]; lambda: device float [sum lambdaCounts]
 * (State::lambda_fd, ignored for replicas without alchemy); boxes host
 * [3*replicas].  Outputs (device, any may be NULL):
 *   force        float [3N]   dU/dx ADDED (State::force_d)
 *   lambdaForce  float [sum lambdaCounts] dU/dlambda ADDED (State::lambdaForce_d)
 *   energy       double [replicas] ADDED (State::energy_d[eenbdirect])
 *   force64      double [3N]  OVERWRITTEN with the exact fixed-point totals
 *   lambdaForce64 double [sum lambdaCounts] OVERWRITTEN
 *   energy64     double [replicas] OVERWRITTEN
 * calcEnergy selects the energy path as in the reference.
 */
typedef struct {
  float *force;
  float *lambdaForce;
  double *energy;
  double *force64;
  double *lambdaForce64;
  double *energy64;
} bnb_outputs;
/*
 * Output modes, ORed into calcEnergy (whose bit 0 alone selects the energy
 * path) of bnb_compute, bnb_compute_nb14/nbex, bnb_compute_pme and
 * bnb_compute_ewald_self.  No reference counterpart; they save the caller a
 * clearing launch (BNB_OUT_SET: force, lambdaForce and energy are written
 * rather than added to -- on a force-only call energy receives 0) or an
 * addition per term (BNB_OUT_ADD64: force64, lambdaForce64 and energy64 are
 * added to rather than written; calls that add into one array must be ordered
 * on one stream).
 */
#define BNB_OUT_SET 2
#define BNB_OUT_ADD64 4
int bnb_compute(bnb_handle *h, const float *position, const float *lambda,
                const float *boxes, int calcEnergy, const bnb_outputs *out,
                void *stream);

/*
 * All-pairs direct space of ONE small periodic system, allocating nothing.
 * No counterpart in the reference, whose direct space always runs on the
 * Domdec block list (getforce_nbdirect, src/nbdirect/nbdirect.cu:574).
 *
 * For callers that may not allocate device memory at all -- not even once,
 * to create a handle -- such as an engine that has given the device's whole
 * memory to its own pool, or one that steps while other streams run and
 * cannot accept the device-wide synchronisation that cudaMalloc/cudaFree may
 * bring.  No handle: every input and output is the caller's, and the only
 * scratch (the fixed-point force and energy accumulators) is a fixed array
 * of about 98 KB inside this library, which every device that loads the
 * library holds until the process exits.
 *
 * Physics: bnb_compute's for atoms outside any MSLD site (siteBlock is not
 * read: every pair is scaled by 1), exclusions skipped, pairs with
 * r^2 < rCut^2 under the minimum image.  The block list is replaced by
 * every pair of atoms, so the cost grows as atomCount^2.
 *   p        host: methods, rCut, rSwitch, betaEwald, kElectric (cullPad and
 *            the soft-core fields are not used)
 *   position device float [3*atomCount]; box host float [3] orthorhombic
 *            edges, each at least 2*rCut (else BNB_ERR_ARG)
 *   nbonds   device [atomCount], typeIdx in [0, typeCount);
 *   vdw      device [typeCount*typeCount] table
 *   exclStart device int [atomCount+1], exclAtom device int: the excluded
 *            partners of atom a are exclAtom[exclStart[a]..exclStart[a+1]-1],
 *            sorted ascending, every pair listed from both ends
 *   out      as bnb_compute (force, energy ADDED; force64, energy64
 *            OVERWRITTEN; the energy arrays have one entry; the lambda
 *            outputs are not written).  With calcEnergy == 0, energy is
 *            left as it was and energy64 is set to 0.
 *
 * Non-finite input: there is no status word.  A NaN or infinite coordinate
 * or parameter makes the forces of the atoms it meets meaningless (the
 * fixed-point conversion of a non-finite value is not flagged) while the
 * call still returns 0; check the inputs beforehand when they can be
 * non-finite, or use a handle, whose bnb_status reports them.
 *
 * Limit: atomCount <= BNB_NOALLOC_MAX_ATOMS; a larger system returns
 * BNB_ERR_TOO_LARGE and launches nothing (use a handle for it).
 * Set-up: the first call on each device looks up the device address of the
 * scratch array with that device current (cudaGetSymbolAddress; this may
 * also load the library's device code on that device); make that first call
 * before any stream capture begins.  Later calls on the device reuse it, so
 * every call must run in the device's primary context (the one the CUDA
 * runtime uses): resetting the device (cudaDeviceReset) after the first call,
 * or calling from another driver-API context on the device, is not supported.
 * Scratch state: the array keeps what the last call left in it; each call
 * first clears, on its stream, the entries it accumulates into.
 * Concurrency: all calls on one device share the one array.  Calls that may
 * overlap on the GPU (different streams without an ordering event, several
 * host threads) race on it and give wrong results; order them on one stream
 * or with events.
 */
#define BNB_NOALLOC_MAX_ATOMS 4096
int bnb_nbdirect_noalloc(const bnb_params *p, int atomCount, const float *position,
                         const float *box, const bnb_nbond *nbonds, int typeCount,
                         const bnb_vdw *vdw, const int *exclStart, const int *exclAtom,
                         int calcEnergy, const bnb_outputs *out, void *stream);

/*
 * 1-4 pairs and the PME correction of excluded pairs (getforce_nb14 and
 * getforce_nbex, src/bonded/pair.cu:288-398; the lists Potential::nb14s and
 * Potential::nbexs, src/system/potential.cxx:1093-1160).  bnb_set_pairs
 * copies the host lists (atom indices of the concatenated replicas, both
 * atoms in one replica; siteBlock as the reference's nb14_scaling /
 * nbex_scaling leave them, with the block part (low 16 bits) indexing the
 * concatenated lambda blocks of all replicas) and allocates their
 * accumulators (BNB_ERR_ARG for an index out of range); useSoftCore14 is
 * Msld::useSoftCore14.  bnb_compute_nb14 / bnb_compute_nbex evaluate one list
 * on position (device float [3N]) and lambda (device float, State::lambda_fd)
 * into `out` with bnb_compute's output semantics; energies are the eenb14 and
 * eenbrecipexcl terms.  The nbex call does no pair work unless elecMethod is
 * PME (as the reference).  The list of a handle need not be built.
 */
int bnb_set_pairs(bnb_handle *h, int nb14Count, const bnb_nb14 *nb14, int nbexCount,
                  const bnb_nbex *nbex, int useSoftCore14);
int bnb_compute_nb14(bnb_handle *h, const float *position, const float *lambda,
                     const float *boxes, int calcEnergy, const bnb_outputs *out, void *stream);
int bnb_compute_nbex(bnb_handle *h, const float *position, const float *lambda,
                     const float *boxes, int calcEnergy, const bnb_outputs *out, void *stream);

/*
 * PME reciprocal space and the Ewald self term (getforce_ewald and
 * getforce_ewaldself, src/nbrecip/nbrecip.cu:19-555; grids and B-spline
 * moduli as Potential::initialize, src/system/potential.cxx:1202-1300).
 * bnb_set_pme sizes one grid per replica and makes the cuFFT plans:
 *   order    B-spline order 4, 6 or 8 (Run::orderEwald, default 6)
 *   gridSpace, grid  host int [3*replicas] grid sizes, or NULL for the
 *            reference's rule from the spacing (Run::gridSpace, default 1 A):
 *            per edge the smallest of j*{32,27,24,20,18} above L/gridSpace
 *   boxes    host float [3*replicas] edges the grids are sized for, or
 *            [6*replicas] triclinic cells (bnb_set_box_type): the grids are
 *            sized for the edge lengths |A|, |B|, |C| (the reference's box.a)
 * Charges, MSLD blocks and replicas come from bnb_set_topology; an atom of
 * block b > 0 carries lambda_b q (Msld atomBlock, nbrecip.cu:101-106).
 * bnb_compute_pme evaluates the reciprocal term (spread, R2C, influence
 * function, C2R, gather) on position (device float [3N], State::position_fd)
 * and lambda (device float, State::lambda_fd) with the boxes `boxes` (host
 * float [3*replicas] edges or [6*replicas] cells; the grids stay as set; in
 * a triclinic cell the grid axes follow the fractional coordinates H^-1 x of
 * the cell matrix H, nbrecip.cu:116-178, 236-242, 456-462), into `out` with
 * bnb_compute's output semantics; energies are the eenbrecip term.
 * bnb_compute_ewald_self adds the self term (energy eenbrecipself and
 * dU/dlambda; no spatial force).  Both do nothing unless elecMethod is PME
 * (as the reference).  They share the handle's dU/dlambda and energy
 * accumulators, so calls on one handle must be ordered (one stream, as the
 * reference's nbrecipStream), not concurrent.  bnb_pme_grid returns the grid
 * of one replica.
 */
int bnb_set_pme(bnb_handle *h, int order, float gridSpace, const int *grid, const float *boxes);
int bnb_pme_grid(bnb_handle *h, int replica, int *K);
int bnb_compute_pme(bnb_handle *h, const float *position, const float *lambda,
                    const float *boxes, int calcEnergy, const bnb_outputs *out, void *stream);
int bnb_compute_ewald_self(bnb_handle *h, const float *lambda, int calcEnergy,
                           const bnb_outputs *out, void *stream);

/*
 * Sets list capacities (candidate tiles, 32-row exclusion masks, work items)
 * before the next rebuild; values <= 0 keep the current/estimated size.  The
 * counterpart of the reference's maxPartnersPerBlock / maxBlockExclCount
 * heuristics (src/domdec/domdec.cu:124-139).  A synchronous rebuild still
 * grows any capacity that overflows; an asynchronous one reports the overflow.
 */
int bnb_reserve(bnb_handle *h, int tiles, int masks, int work);

/* Device status word (ORed BNB_STATUS_* bits since the last clear);
 * synchronises the stream.  clear!=0 resets it. */
int bnb_status(bnb_handle *h, void *stream, int clear, int *status);

/* Sizes of the current list (synchronises): blocks, candidate tiles, mask
 * rows (in 32-row units), work items. */
int bnb_list_sizes(bnb_handle *h, void *stream, int *blocks, int *tiles,
                   int *masks, int *work);

/*
 * Copies the list structures to host arrays (test and inspection hook;
 * synchronises).  Sizes from bnb_list_sizes.  Any pointer may be NULL.
 *   wrap[N] blockBounds[B+1] sortedAtom[N] slotAtom[32B] bmin/bmax[3B]
 *   candStart[B+1] cand[2*T] (jBlock, shiftCode) candMask[T] masks[32*M]
 */
int bnb_get_list(bnb_handle *h, void *stream, int *wrap, int *blockBounds,
                 int *sortedAtom, int *slotAtom, float *bmin, float *bmax,
                 int *candStart, int *cand, int *candMask, uint32_t *masks);

/* Pairs with r<rCut evaluated by the last bnb_compute with counting enabled
 * (bnb_set_counting).  Synchronises. */
int bnb_set_counting(bnb_handle *h, int enable);
int bnb_pair_count(bnb_handle *h, void *stream, unsigned long long *pairs);

/*
 * Per-phase timing with CUDA events recorded on the launching stream
 * (profiling aid, no reference counterpart).  When enabled, every
 * bnb_compute records events around the pair kernel and every bnb_rebuild
 * around the list build.  bnb_profile_read synchronises, returns the summed
 * milliseconds and counts since the last reset, and the number of kernels
 * libbnb launched.
 */
int bnb_profile(bnb_handle *h, int enable);
int bnb_profile_read(bnb_handle *h, double *pairMs, int *pairLaunches,
                     double *rebuildMs, int *rebuilds,
                     unsigned long long *kernelLaunches, int reset);

/* Measured FP32 FMA throughput of the current device (flop/s), the roofline
 * denominator of the FP32-bound pair kernel.  No reference counterpart. */
int bnb_fp32_peak(void *stream, double *flopsPerSecond);

/* Heuristic column grid of one replica (Domdec::initialize,
 * src/domdec/domdec.cu:114-117), host computation. */
int bnb_domain_div(int atomCount, const float *box, int *divX, int *divY);

/* ---- MSLD lambda maps and biases (stateless, device arrays) -------------- */
/* All of them compute in FP64.  blockFixed is a byte per block (the layout
 * of Msld::blockFixed_d, a bool array) and may be NULL. */
/*
 * lambda_j = exp(fnex*sin(theta_j)) / sum over the site
 * (Msld::calc_lambda_from_theta, src/msld/msld.cu:863-921).  Also writes the
 * FP32 mirror lambda_f (State::lambda_fd) when non-NULL.  siteBound[sites+1];
 * fixed blocks keep lambda = theta.
 */
int bnb_lambda_from_theta(int siteCount, const int *siteBound, double fnex,
                          const double *theta, const uint8_t *blockFixed,
                          double *lambda, float *lambda_f, void *stream);
/*
 * dU/dtheta from dU/dlambda (Msld::calc_thetaForce_from_lambdaForce,
 * src/msld/msld.cu:937-998).  thetaForce is ADDED to.  The _f32 form takes
 * the FP32 buffers the reference passes (lambda_fd, theta_fd, lambdaForce_d,
 * thetaForce_d, msld.cu:987-991).
 */
int bnb_theta_force(int blockCount, const int *lambdaSite,
                    const int *siteBound, double fnex, const double *lambda,
                    const double *theta, const double *lambdaForce,
                    const uint8_t *blockFixed, double *thetaForce, void *stream);
int bnb_theta_force_f32(int blockCount, const int *lambdaSite,
                        const int *siteBound, double fnex, const float *lambda,
                        const float *theta, const float *lambdaForce,
                        const uint8_t *blockFixed, float *thetaForce, void *stream);
/*
 * Fixed bias b_i*lambda_i and variable biases (types 1-12) on lambda
 * (Msld::getforce_fixedBias/getforce_variableBias, src/msld/msld.cu:1000-1153).
 * lambdaForce and energy (may be NULL) are ADDED to.  The _f32 form takes the
 * reference's FP32 lambda_fd / lambdaBias_d / lambdaForce_d buffers.
 */
int bnb_bias(int blockCount, const double *lambda, const double *fixedBias,
             int varCount, const bnb_varbias *varBias, double *lambdaForce,
             double *energy, void *stream);
int bnb_bias_f32(int blockCount, const float *lambda, const float *fixedBias,
                 int varCount, const bnb_varbias *varBias, float *lambdaForce,
                 double *energy, void *stream);

/* ---- batched stepping: tuning and integrator ----------------------------- */
/*
 * Tuning knobs of the pair kernel: candidate tiles per work item (1..32),
 * CTAs per SM of the persistent grid (0 = as many as fit) and the tail of the
 * work list (0..8): the last tailItems * tilesPerWork candidate tiles of every
 * i block become items of a quarter of the size, taken after all others, so
 * that the persistent warps finish close together (0 = no tail; default 2).
 * A changed tile count or tail takes effect at the next bnb_rebuild.  The
 * split of each block's tiles depends on that block alone, so a replica gives
 * the same bits alone and in a batch at equal settings.  No reference
 * counterpart.
 */
int bnb_set_tuning(bnb_handle *h, int tilesPerWork, int ctasPerSM, int tailItems);
int bnb_get_tuning(bnb_handle *h, int *tilesPerWork, int *ctasPerSM, int *tailItems);
/*
 * Adds one sampling step of lambda (FP64, [blockCount]) to histograms, the
 * statistics adaptive landscape flattening takes from the .lmd lambda
 * trajectory (written by src/io/io.cxx:347-371): hist1[32*b + k] counts
 * lambda_b in bin k of 32 on [0,1]; endCount[b] counts lambda_b > 0.99;
 * hist2[64*p + 8*a + c] counts (lambda_i, lambda_j) of pair p =
 * (pairs[2p], pairs[2p+1]) in the 8x8 bin (a, c).  Blocks with blockFixed
 * set are skipped.  Any output may be NULL.  Counts are uint32.
 */
int bnb_lambda_histogram(int blockCount, const double *lambda, const uint8_t *blockFixed,
                         int pairCount, const int *pairs, unsigned int *hist1,
                         unsigned int *hist2, unsigned int *endCount, void *stream);

/*
 * Autotuner: times every (tiles per work item in {1,2,4,8,16,32}) x (CTAs per
 * SM in {auto,2,3}) x (tail in {2,0}) setting on the caller's coordinates
 * (median of `reps` evaluations, CUDA events), keeps the fastest and rebuilds
 * the list with it.  Synchronises.  bestMs: the kept setting's
 * pair-evaluation time.
 */
int bnb_autotune(bnb_handle *h, const float *position, const float *lambda,
                 const float *boxes, int reps, void *stream, float *bestMs);
/*
 * Harmonic bond gradient, U = sum_bonds kb/2 (r - b0)^2, the bond form of
 * the reference's bonded kernel (src/bonded/bonded.cu:83-112, without its
 * soft-bond branch): adds dU/dx to grad (FP64, [3n]).  Bonds are given per
 * atom as a CSR: for atom a, entries start[a]..start[a+1]-1 of partner and
 * kbB0 (float pairs kb, b0), every bond listed from both ends.  Bonded atoms
 * must be stored as one periodic image (no minimum image is taken).  The
 * batched MSLD step uses it in place of the reference's bonded terms and
 * constraints, which are not part of the direct-space path.
 */
int bnb_bond_gradient(int n, const int *start, const int *partner, const float *kbB0, const double *x,
                      double *grad, void *stream);
/*
 * Langevin VRORV step of nx coordinates and nt theta values (FP64 state),
 * the scheme of State::update (src/update/update.cu:233-305):
 *   v -= dt ism^2 dU/dx;  x += dt/2 v;  v = a v + b ism xi;  x += dt/2 v
 * with (a, b) = (friction, noise) = (exp(-gamma dt), sqrt((1-a^2) kT))
 * separately for coordinates and theta (State::alloc_leapparms2), ism =
 * 1/sqrt(mass) (non-finite: frozen).  xi are counter-based Gaussian numbers
 * from (seed, step + *stepCounter, index); stepCounter (device, 2 x u64, may
 * be NULL) is advanced by one per call, so a CUDA graph replaying the call
 * draws new numbers each time.  x_f (may be NULL) receives the FP32 mirror of
 * x (State::set_fd); nanFlag (may be NULL) is raised on a non-finite velocity.
 */
int bnb_langevin_vrorv(int nx, int nt, double *x, double *v, const double *fx,
                       const double *ismx, double *theta, double *vtheta,
                       const double *ftheta, const double *ismtheta, double dt,
                       double frictionX, double noiseX, double frictionTheta,
                       double noiseTheta, unsigned long long seed,
                       unsigned long long step, unsigned long long *stepCounter,
                       float *x_f, int *nanFlag, void *stream);

/*
 * The Langevin step split at its middle for holonomic constraints
 * (update_VVhbpR / update_OOhbpR, src/update/update.cu:276-303): phase 0
 * kicks and drifts half a step, phase 1 applies friction and noise and drifts
 * the other half; each phase first copies x to xPrev (device double [nx],
 * may be NULL without constraints), and bnb_holonomic_position follows each
 * phase.  Arguments as bnb_langevin_vrorv; without constraints phase 0 then
 * phase 1 equals one bnb_langevin_vrorv bit for bit.  x_f is written by
 * phase 1 (and by bnb_holonomic_position for constrained atoms).
 */
int bnb_langevin_half(int phase, int nx, int nt, double *x, double *v, double *xPrev, const double *fx,
                      const double *ismx, double *theta, double *vtheta, const double *ftheta,
                      const double *ismtheta, double dt, double frictionX, double noiseX,
                      double frictionTheta, double noiseTheta, unsigned long long seed,
                      unsigned long long step, unsigned long long *stepCounter, float *x_f,
                      int *nanFlag, void *stream);

/*
 * Holonomic bond constraints (holonomic_position / holonomic_velocity,
 * src/holonomic/holonomic.cu:238-758).  The cluster layouts are the
 * reference's TriangleCons / Branch1Cons / Branch2Cons / Branch3Cons
 * (src/system/potential.h:120-138): a rigid triangle with b0 = |01|, |02|,
 * |12|, or a heavy atom (idx[0]) with 1-3 hydrogens, b0[k] = |0 (k+1)|;
 * every atom in at most one cluster; device arrays.
 * bnb_holonomic_position corrects the drifted positions x (device double
 * [3N]) along the bond vectors of xPrev until |b0^2 - r^2| < 2 b0^2 tolerance
 * (Run::shakeTolerance) or maxIter iterations (then status bit 1 is set, if
 * status is given), and sets v = (x - xPrev) / halfdt for the cluster atoms
 * (v may be NULL).  ism: device double [3N], 1/sqrt(m) per degree of freedom
 * (LeapState::ism).  x_f (optional): FP32 copy of the constrained positions.
 * bnb_holonomic_velocity removes the bond-direction relative velocities.
 * Coordinates must be unwrapped: a cluster is not split across images.
 */
typedef struct { int idx[3]; float b0[3]; } bnb_triangle_cons;
typedef struct { int idx[2]; float b0[1]; } bnb_branch1_cons;
typedef struct { int idx[3]; float b0[2]; } bnb_branch2_cons;
typedef struct { int idx[4]; float b0[3]; } bnb_branch3_cons;
typedef struct {
  int nTriangle, nBranch1, nBranch2, nBranch3;
  const bnb_triangle_cons *triangle;
  const bnb_branch1_cons *branch1;
  const bnb_branch2_cons *branch2;
  const bnb_branch3_cons *branch3;
} bnb_constraints;
int bnb_holonomic_position(const bnb_constraints *cs, const double *xPrev, double *x, double *v,
                           const double *ism, double halfdt, double tolerance, int maxIter,
                           float *x_f, int *status, void *stream);
int bnb_holonomic_velocity(const bnb_constraints *cs, const double *x, double *v, const double *ism,
                           void *stream);

/* ---- BF16 MLP of learned landscape flattening (no reference counterpart;
 * BLaDE's src/mlp is TorchANI inference, unrelated).  Row-major arrays,
 * BF16 as uint16_t bit patterns, products with BF16 operands and FP32
 * accumulation in a fixed order.  act: 0 identity, 1 SiLU. ---------------- */
/* Z[M,N] = X[M,K] W[N,K]^T + bias[N] (FP32, bias may be NULL); Y = act(Z)
 * as BF16 [M,N] and/or FP32 Yf [M,N] (either may be NULL). */
int bnb_mlp_linear_forward(int M, int N, int K, const uint16_t *X, const uint16_t *W,
                           const float *bias, int act, float *Z, uint16_t *Y, float *Yf,
                           void *stream);
/* Given dY = dLoss/dY [M,N] (FP32) and the forward's Z: dZ = dY act'(Z)
 * (FP32 [M,N] and its BF16 copy dZb), dW[N,K] = dZb^T X, db[N] = sum_m dZ,
 * and, when dX is not NULL, dX[M,K] = dZb W.  dW and db are overwritten. */
int bnb_mlp_linear_backward(int M, int N, int K, const float *dY, const float *Z, int act,
                            const uint16_t *X, const uint16_t *W, float *dZ, uint16_t *dZb,
                            float *dX, float *dW, float *db, void *stream);
/* loss = (1/M) sum_{m,n} w[n] we[m,n] (Y-T)^2, dY = dloss/dY; the column
 * weights w [N] and element weights we [M,N] may each be NULL (all 1). */
int bnb_mlp_mse(int M, int N, const float *Y, const float *T, const float *weight,
                const float *elemWeight, float *dY, double *loss, void *stream);
/* Adam step (bias-corrected, decoupled weight decay) on FP32 master weights;
 * writes the BF16 working copy when weightBf16 is not NULL.  step >= 1. */
int bnb_mlp_adam(int n, float *master, uint16_t *weightBf16, const float *grad, float *m,
                 float *v, float lr, float beta1, float beta2, float eps, float weightDecay,
                 int step, void *stream);
/* y = bf16(x), round to nearest even. */
int bnb_to_bf16(int n, const float *x, uint16_t *y, void *stream);

/* Library version string. */
const char *bnb_version(void);

#ifdef __cplusplus
}
#endif
#endif
