/*
 * pmo_b200.h — C ABI of the B200 voxel Monte Carlo photon-transport engine.
 *
 * Everything here is plain C: device pointers, sizes and a cudaStream_t passed
 * as an opaque pointer.  Every entry point is stream-ordered and asynchronous:
 * it validates its arguments on the host, enqueues work on `stream` and
 * returns a status code without synchronising.  Device-side faults that can
 * only be seen while photons run (a photon that exceeds its event cap, a step
 * out of the volume, a label without optical properties) are counted in the
 * caller's `counters` buffer; `pmo_check_counters` turns those counts into a
 * status code after the caller has synchronised the stream.
 *
 * Photon p of a run draws all its random numbers from Philox4x32-10
 * (Salmon et al., SC'11) with key = (seed_lo, seed_hi) and counter
 * (n, stream, p_lo, p_hi): stream 0 gives the four uniforms of interaction n
 * (step length, a spare uniform, Henyey-Greenstein cos(theta), azimuth).  The
 * spare uniform serves the first decision of the step that needs one more:
 * a Fresnel decision with 0 < R < 1 during the step's face crossings, or the
 * roulette at its end.  A later Fresnel decision of the same step takes word
 * 0 of stream 1 at counter n = the photon's Fresnel-decision index, a later
 * roulette word 0 of stream 3 at the interaction's index.  Stream 2 gives the
 * source uniforms.  A photon's history therefore depends only on (seed, p, optics),
 * never on the launch shape, so runs over photon ranges can be split, resumed
 * and replayed.
 *
 * Label volume layout follows the reference: C-order (nx, ny, nz) uint8
 * array, linear index (ix*ny + iy)*nz + iz, padded by a one-voxel shell of
 * `end_label` on all six faces (pymopt/voxel_gpu/_classes.py:439-459).
 */
#ifndef PMO_B200_H
#define PMO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PMO_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
#define PMO_OK                 0
#define PMO_ERR_ARG            1   /* bad argument (null pointer, size, range) */
#define PMO_ERR_GEOMETRY       2   /* a photon stepped outside the volume       */
#define PMO_ERR_LABEL          3   /* a photon entered a label without optics   */
#define PMO_ERR_STEP_CAP       4   /* a photon exceeded max_events              */
#define PMO_ERR_CUDA           5   /* a CUDA runtime call failed                */
#define PMO_ERR_WORKSPACE      6   /* workspace missing or too small            */
#define PMO_ERR_TIMEOUT        7   /* a bounded device wait gave up             */
#define PMO_ERR_NUMERIC        8   /* a non-finite weight or direction appeared */

/* ---- precision of the transport arithmetic ----------------------------- */
#define PMO_FP32 0               /* the product path                           */
#define PMO_FP64 1               /* the per-photon FP64 build (validation)     */

/* ---- photon sources ----------------------------------------------------- */
#define PMO_SRC_PENCIL   0       /* every photon starts at (ix,iy,iz, p, v, w0) */
#define PMO_SRC_GAUSSIAN 1       /* pencil + lateral N(0, sigma^2) in x and y    */
#define PMO_SRC_STATE    2       /* per-photon initial state arrays (cuVMC form) */

/* ---- optical-property modes --------------------------------------------- */
#define PMO_PROPS_LABEL  0       /* ma/ms/g/n indexed by voxel label            */
#define PMO_PROPS_VOXEL  1       /* ma/ms per voxel, g/n per label              */

/* ---- fluence tally modes ------------------------------------------------ */
#define PMO_FLU_NONE     0
#define PMO_FLU_GLOBAL   1       /* fp32 atomics straight to the padded grid    */
#define PMO_ABSORBED_SHIFT 32   /* fixed-point scale of the absorbed grid */
#define PMO_FLU_SHARED   2       /* + per-block shared-memory window            */

/* ---- ledger slots (double), accumulated by the kernels ------------------ */
#define PMO_L_WINIT      0       /* sum of launched photon weights              */
#define PMO_L_RD         1       /* exit weight with v_z < 0 (reference Rd)     */
#define PMO_L_TT         2       /* exit weight with v_z > 0 (reference Tt)     */
#define PMO_L_EXIT0      3       /* exit weight with v_z == 0                    */
#define PMO_L_ABS        4       /* absorbed weight                              */
#define PMO_L_RGAIN      5       /* weight created by roulette survival          */
#define PMO_L_RLOSS      6       /* weight removed by roulette death             */
#define PMO_L_ERRW       7       /* weight of photons killed by an error         */
#define PMO_L_RD_TOP     8       /* exit weight through a -z face                */
#define PMO_L_TT_BOTTOM  9       /* exit weight through a +z face                */
#define PMO_L_SPEC       10      /* specular weight of source-reflected photons  */
#define PMO_LEDGER_N     16

/* ---- event counters (unsigned long long) -------------------------------- */
#define PMO_C_PHOTONS    0       /* photons finished                             */
#define PMO_C_INTERACT   1       /* interactions (hop-drop-spin cycles)          */
#define PMO_C_CROSS      2       /* voxel-face crossings                         */
#define PMO_C_FRESNEL    3       /* Fresnel evaluations (index mismatch)         */
#define PMO_C_REFLECT    4       /* Fresnel/TIR reflections                      */
#define PMO_C_ROULETTE   5       /* roulette draws                               */
#define PMO_C_EXITS      6       /* photons that left through the end label      */
#define PMO_C_ERR_GEOM   7
#define PMO_C_ERR_LABEL  8
#define PMO_C_ERR_CAP    9
#define PMO_C_ERR_NUM    10
#define PMO_C_SAMECROSS  11      /* same-label crossings (counted by the oracle)  */
#define PMO_C_XDRAWS     12      /* Philox draws beyond one per interaction: a
                                    Fresnel decision or roulette after the step's
                                    spare uniform was taken                      */
#define PMO_COUNTERS_N   16

/* ---- R(r) / T(r) histogram categories, layout [PMO_RR_CATS][nr] --------- */
#define PMO_RR_TOP       0       /* exits through a -z face                      */
#define PMO_RR_BOTTOM    1       /* exits through a +z face                      */
#define PMO_RR_LAT_NEG   2       /* exits through an x/y face with v_z < 0       */
#define PMO_RR_LAT_POS   3       /* exits through an x/y face with v_z > 0       */
#define PMO_RR_CATS      4

/* ---- run flags ---------------------------------------------------------- */
#define PMO_FLAG_EXPORT_EXITS  1u  /* write per-photon final state arrays        */
#define PMO_FLAG_PHOTON_STATS  2u  /* write per-photon event counts (validation) */
#define PMO_FLAG_SCORE_RECORD  4u  /* write per-photon exit bin and weight, the
                                      input of the gradient replay             */

typedef struct pmo_problem {
    /* geometry: padded label volume, C-order (nx, ny, nz) */
    const uint8_t *labels;
    int32_t nx, ny, nz;
    float voxel_space;           /* l [mm] */
    /* optional uniform-box map from pmo_build_voxel_words (label in the low
       byte, the box's z half-extent and lateral code in the high byte).  With
       it, photons in per-label optics step from the face of one label-uniform
       box to the next instead of from voxel face to voxel face: the same
       path, fewer crossings.
       NULL: voxel-by-voxel stepping exactly as the reference. */
    const uint16_t *voxel_words;
    int32_t end_label;           /* shell label; photons leave when they enter it */

    /* optics: per-label tables of n_labels entries (n_labels <= 256);
       n[end_label] is the ambient refractive index. */
    int32_t props_mode;          /* PMO_PROPS_LABEL or PMO_PROPS_VOXEL */
    int32_t n_labels;
    const float *ma, *ms, *g, *n;
    const float *vox_ma, *vox_ms; /* PMO_PROPS_VOXEL: nx*ny*nz each */

    /* source */
    int32_t source;              /* PMO_SRC_* */
    int32_t src_ix, src_iy, src_iz;
    float src_p[3], src_v[3];
    float src_w0;                /* initial weight of transported photons */
    float beam_sigma;            /* PMO_SRC_GAUSSIAN: sigma of x and y [mm] */
    float spec_prob;             /* probability that the source photon is reflected
                                    specularly before entering (w = 1, v = spec_v) */
    float spec_v[3];
    int32_t center_ix, center_iy; /* exit-position origin (reference _encooder) */
    /* PMO_SRC_STATE: SoA arrays of 3*count (add, p, v) and count (w),
       indexed by photon - photon_begin; final states are written back. */
    int32_t *state_add;
    float *state_p, *state_v, *state_w;

    /* photons */
    uint64_t seed;
    uint64_t photon_begin, photon_count;
    uint32_t max_events;         /* per-photon event cap, 0 = default (2^26) */
    int32_t precision;           /* PMO_FP32 or PMO_FP64 */
    uint32_t flags;              /* PMO_FLAG_* */
} pmo_problem;

typedef struct pmo_tallies {
    double *ledger;                   /* PMO_LEDGER_N doubles, accumulated */
    unsigned long long *counters;     /* PMO_COUNTERS_N, accumulated */
    float *rr;                        /* PMO_RR_CATS * nr, accumulated, or NULL */
    int32_t nr;
    float dr;                         /* bin width [mm]; bins (i*dr, (i+1)*dr] */
    int32_t fluence_mode;             /* PMO_FLU_* */
    /* nx*ny*nz absorbed weight, accumulated, in unsigned 64-bit fixed point:
       weight * 2^PMO_ABSORBED_SHIFT per deposit, rounded to nearest.
       Integer atomics make each voxel's sum exact and independent of the
       order of the deposits. */
    unsigned long long *absorbed;
    int32_t win_lo[3];                /* PMO_FLU_SHARED: window origin (voxel) */
    int32_t win_dim[3];               /* PMO_FLU_SHARED: window extent (voxels) */
    /* PMO_FLAG_EXPORT_EXITS: final state per photon (index photon - begin).
       add/p/v are SoA 3*photon_count; killed photons are all zero as in the
       reference (pymopt/voxel_gpu/_cukernel.py:182-190). */
    int32_t *exit_add;
    float *exit_p, *exit_v, *exit_w;
    /* PMO_FLAG_PHOTON_STATS: per-photon interaction / crossing / Fresnel counts */
    uint32_t *ph_interact, *ph_cross, *ph_fresnel;
    /* PMO_FLAG_SCORE_RECORD: per photon, the R(r)/T(r) bin its exit weight went
       to (category * nr + bin, -1 for none) and that weight */
    int32_t *score_bin;
    float *score_w;
    /* Angle-resolved exits (pymopt/metrics/_scoring.py:27-38): weight per bin
       (i*da, (i+1)*da] of arccos|v_z|, da = pi / (2 * n_ang); row 0 holds
       exits with v_z < 0, row 1 those with v_z > 0.  2 * n_ang floats,
       accumulated; n_ang = 0 or ang = NULL: off. */
    float *ang;
    int32_t n_ang;
    /* Line profile of exits moving towards -x (the side-face profile of
       pymopt/virtualOBD.py:171-172 through pymopt/metrics/_scoring.py:40-51):
       weight per bin (i*line_dr, (i+1)*line_dr] of the exit depth
       z = l*(add_z - 1) + p_z + l/2 (rounded to 1e-6 mm) for |y| < line_y_range.
       n_line floats, accumulated; n_line = 0 or line = NULL: off. */
    float *line;
    int32_t n_line;
    float line_dr;
    float line_y_range;
} pmo_tallies;

/*
 * Gradient replay (pmo_run_grad).  The forward run wrote score records; the
 * loss gradient with respect to the binned exit weight is `coef`
 * ([PMO_RR_CATS][nr]: dLoss / d(sum of exit weights in bin)).  Each photon
 * with q = coef[bin] * w != 0 is replayed from its Philox counters and
 * contributes the perturbation Monte Carlo terms of implicit-capture
 * weighting: for every voxel v it crossed, dLoss/dmu_a(v) += -q * L_v and
 * dLoss/dmu_s(v) += q * (n_v / mu_s(v) - L_v), with L_v its path length and n_v
 * its interactions in v.  Outputs are accumulated, never cleared.
 */
typedef struct pmo_grad {
    const float *coef;               /* PMO_RR_CATS * nr */
    int32_t nr;
    float dr;
    const int32_t *score_bin;        /* forward records, index photon - begin */
    const float *score_w;
    float *d_ma_voxel, *d_ms_voxel;  /* nx*ny*nz or NULL (needs voxel stepping) */
    double *d_ma_label, *d_ms_label; /* n_labels or NULL */
    unsigned long long *counters;    /* PMO_G_* */
    /* optional central finite difference by reweighting the same photons
       (perturbation Monte Carlo), for up to PMO_FD_MAX targets: fd_target maps
       every voxel to a target index or -1; target t scales mu_a (fd_param 0)
       or mu_s (fd_param 1) of its voxels by (1 +- fd_h).  fd_out[2 * t + 0/1]
       accumulates sum over replayed photons of coef[bin] * w * (f -+ 1), with
       f = (1 +- h)^n_t * exp(-(+-h) mu_t_param L_t) (mu_s) or exp(-(+-h) mu_a L_t)
       (mu_a); (fd_out[2t] - fd_out[2t+1]) / (2 h mu) is the central difference. */
    const int16_t *fd_target;        /* nx*ny*nz or NULL */
    int32_t fd_n;
    int32_t fd_param;
    float fd_h;
    double *fd_out;                  /* 2 * fd_n */
} pmo_grad;

#define PMO_FD_MAX 32

#define PMO_G_REPLAYED   0           /* photons replayed (q != 0)               */
#define PMO_G_SKIPPED    1           /* photons with q == 0                     */
#define PMO_G_MISMATCH   2           /* replay ended in another bin or weight   */
#define PMO_G_COUNTERS_N 4

typedef struct pmo_launch {
    int32_t block_threads;       /* 0 = default: 256 for pmo_run_plain, 128 for the others */
    int32_t blocks_per_sm;       /* 0 = occupancy maximum */
} pmo_launch;

/* Library identity. */
int pmo_abi_version(void);
const char *pmo_status_string(int status);
int pmo_device_info(int *sm_count, int *cc_major, int *cc_minor);

/* Bytes of device scratch the caller passes as `workspace` to the run
   entry points (work counters; contents need not be initialised; the entry
   points clear what they use, stream-ordered).  pmo_cuvmc, whose reference
   signature has no tally arguments, leaves its ledger (PMO_LEDGER_N doubles)
   and counters (PMO_COUNTERS_N unsigned long long) in the workspace at the
   byte offsets below. */
#define PMO_WS_LEDGER_OFFSET   64
#define PMO_WS_COUNTERS_OFFSET 256
size_t pmo_workspace_bytes(void);

/*
 * Forward transport with on-device tallies.
 * Replaces the launch of cuVMC in BaseVoxelMonteCarlo.start
 * (pymopt/voxel_gpu/_classes.py:105-111) together with the host reductions
 * that follow it: getRdTtRate (pymopt/voxel_gpu/_classes.py:326-334) and
 * metrics.radialDistance (pymopt/metrics/_scoring.py:16-25).
 * Tallies are accumulated, never cleared, so consecutive runs over photon
 * ranges [a, b), [b, c) with one seed equal one run over [a, c).
 */
int pmo_run_plain(const pmo_problem *prob, const pmo_tallies *tal,
                  const pmo_launch *launch, void *workspace,
                  size_t workspace_bytes, void *stream);

/*
 * Backward kernel: replay the photons of a forward run (same problem, seed
 * and photon range; the forward ran with PMO_FLAG_SCORE_RECORD) and
 * accumulate dLoss/dmu_a and dLoss/dmu_s per voxel and per label.  With
 * per-voxel outputs the problem must step voxel by voxel (voxel_words NULL),
 * in the forward run as well.  No counterpart in the reference, which has no
 * derivatives.
 */
int pmo_run_grad(const pmo_problem *prob, const pmo_grad *grad, const pmo_launch *launch,
                 void *workspace, size_t workspace_bytes, void *stream);

/* ---- batched slab problems ------------------------------------------- */

/* One laterally infinite single-layer slab: the geometry of a PlateModel with
   one layer (pymopt/voxel_gpu/_classes.py:396-459) when x_size, y_size grow
   without bound.  Photons enter at the origin of the top face along +z with
   weight w0 = 1 - Rsp (pymopt/voxel_gpu/_classes.py:204-221). */
typedef struct pmo_slab {
    float ma, ms, g;              /* mu_a, mu_s [1/mm], anisotropy */
    float n_tissue, n_ambient;    /* refractive indices inside / outside */
    float thickness;              /* [mm] */
    float dr;                     /* R(r) bin width [mm] */
    uint32_t photons;             /* photon budget */
} pmo_slab;

/* A work item: photons [begin, begin + count) of one problem. */
typedef struct pmo_batch_item {
    uint32_t problem, begin, count;
} pmo_batch_item;

/* Per-problem raw sums (double), accumulated by pmo_run_batched. */
#define PMO_BS_RD      0          /* sum w of exits through the top face       */
#define PMO_BS_RD_L    1          /* sum w * L (path length)                   */
#define PMO_BS_RD_N    2          /* sum w * n (interactions)                  */
#define PMO_BS_TT      3          /* bottom face                               */
#define PMO_BS_TT_L    4
#define PMO_BS_TT_N    5
#define PMO_BS_ABS     6          /* absorbed weight                           */
#define PMO_BS_WINIT   7          /* launched weight                           */
#define PMO_BS_RGAIN   8
#define PMO_BS_RLOSS   9
#define PMO_BS_ERRW    10
#define PMO_BS_INTER   11         /* interactions (count)                      */
#define PMO_BS_N       16

/* Per-problem results of pmo_batch_finalize (double): */
#define PMO_BR_RD        0        /* Rd                                        */
#define PMO_BR_TT        1        /* Tt                                        */
#define PMO_BR_A         2        /* absorbed fraction                         */
#define PMO_BR_DRD_DMA   3        /* dRd/dmu_a = -E[w L 1_top]                 */
#define PMO_BR_DRD_DMS   4        /* dRd/dmu_s = E[w (n/mu_s - L) 1_top]       */
#define PMO_BR_DTT_DMA   5
#define PMO_BR_DTT_DMS   6
#define PMO_BR_BALANCE   7        /* energy ledger residual / launched weight  */
#define PMO_BR_N         8

/* pmo_batch.tally_mode.  PMO_BT_THREAD: each thread keeps the sums of the
   problem it works on in shared memory and adds them to global memory when
   it moves to another problem (few global atomics; shared memory of
   threads * 13 doubles).  PMO_BT_GLOBAL: every sum goes straight to global
   memory with an atomic (no shared memory; atomics on the same few addresses
   for photons of one problem). */
#define PMO_BT_THREAD 0
#define PMO_BT_GLOBAL 1

typedef struct pmo_batch {
    const pmo_slab *slabs;        /* device array of n_problems */
    int32_t n_problems;
    const pmo_batch_item *items;  /* device work queue of n_items, in order */
    int32_t n_items;
    uint64_t seed;
    int32_t nr;                   /* R(r) bins per problem */
    double *sums;                 /* n_problems * PMO_BS_N, accumulated */
    float *bins;                  /* n_problems * nr * 3: sum w, w L, w n of
                                     top exits in (i dr, (i+1) dr] */
    uint32_t *remaining;          /* per problem photons still in flight (set
                                     to the budget by the caller) or NULL */
    unsigned long long *t_done;   /* per problem completion time (ns, device
                                     global timer) or NULL */
    int32_t precision;            /* PMO_FP32 or PMO_FP64 */
    uint32_t max_events;          /* 0 = 2^26 */
    int32_t tally_mode;           /* where per-problem sums gather:
                                     PMO_BT_THREAD or PMO_BT_GLOBAL */
} pmo_batch;

/*
 * Run every work item in one persistent launch: forward transport and the
 * perturbation Monte Carlo derivatives of Rd, Tt and R(r) with respect to
 * mu_a and mu_s, in the same pass (single layer, so the per-photon path
 * length and interaction count suffice).  Photon j of problem p draws from
 * Philox with counter (n, stream + 4 p, j, 0): problem 0 has the streams of
 * pmo_run_plain.  No counterpart in the reference, which runs one problem
 * per launch.
 */
int pmo_run_batched(const pmo_batch *batch, const pmo_launch *launch, void *workspace,
                    size_t workspace_bytes, void *stream);

/* Per-problem results (n_problems * PMO_BR_N doubles) and normalised R(r)
   with its derivatives (n_problems * nr * 3 doubles: R, dR/dmu_a, dR/dmu_s,
   [1/mm^2]) from the sums of pmo_run_batched. */
int pmo_batch_finalize(const pmo_batch *batch, double *results, double *rr, void *stream);

/* ---- batched layered slabs ------------------------------------------- */

/* One layer of a laterally infinite layered slab: a PlateModel stack
   (pymopt/voxel_gpu/_classes.py:396-459) with x_size, y_size unbounded. */
typedef struct pmo_layer {
    float ma, ms, g, n;           /* mu_a, mu_s [1/mm], anisotropy, index */
    float thickness;              /* [mm] */
} pmo_layer;

#define PMO_MAX_LAYERS 8

/* One problem: layers [first_layer, first_layer + n_layers) of the layer
   table, top to bottom.  Photons enter at the origin of the top face along +z
   with weight 1 - Rsp, Rsp = ((n_ambient - n_top) / (n_ambient + n_top))^2
   (pymopt/voxel_gpu/_classes.py:204-221). */
typedef struct pmo_stack {
    uint32_t first_layer;
    uint32_t n_layers;            /* 1 .. PMO_MAX_LAYERS */
    float n_ambient;
    float dr;                     /* R(r) bin width [mm] */
    uint32_t photons;             /* photon budget */
} pmo_stack;

/* Per-problem raw sums (double) of pmo_run_stack_batch: the scalars below,
   then for layer i at PMO_SS_LAYER0 + 4 i: sum w L_i and sum w n_i of top
   exits (+0, +1) and of bottom exits (+2, +3), with L_i the photon's path
   length and n_i its interactions in layer i. */
#define PMO_SS_RD      0
#define PMO_SS_TT      1
#define PMO_SS_ABS     2
#define PMO_SS_WINIT   3
#define PMO_SS_RGAIN   4
#define PMO_SS_RLOSS   5
#define PMO_SS_ERRW    6
#define PMO_SS_INTER   7
#define PMO_SS_LAYER0  8
#define PMO_SS_N       40         /* PMO_SS_LAYER0 + 4 * PMO_MAX_LAYERS */

/* Per-problem results of pmo_stack_batch_finalize (double): Rd, Tt, A, the
   energy residual, then for layer i at PMO_SR_LAYER0 + 4 i: dRd/dmu_a_i,
   dRd/dmu_s_i, dTt/dmu_a_i, dTt/dmu_s_i (perturbation Monte Carlo:
   d/dmu_a_i = -E[w L_i], d/dmu_s_i = E[w (n_i / mu_s_i - L_i)]). */
#define PMO_SR_RD      0
#define PMO_SR_TT      1
#define PMO_SR_A       2
#define PMO_SR_BALANCE 3
#define PMO_SR_LAYER0  4
#define PMO_SR_N       36         /* PMO_SR_LAYER0 + 4 * PMO_MAX_LAYERS */

/* R(r) bin record of a stack problem: PMO_SB_N floats per bin: sum w of the
   top exits in (i dr, (i+1) dr], then per layer sum w L_i and sum w n_i.
   Finalised R(r) has the same layout in doubles: R, then per layer
   dR/dmu_a_i and dR/dmu_s_i [1/mm^2]. */
#define PMO_SB_N       17         /* 1 + 2 * PMO_MAX_LAYERS */

typedef struct pmo_stack_batch {
    const pmo_stack *stacks;      /* device array of n_problems */
    int32_t n_problems;
    const pmo_layer *layers;      /* device layer table */
    int32_t n_layer_rows;
    const pmo_batch_item *items;  /* device work queue of n_items, in order */
    int32_t n_items;
    uint64_t seed;
    int32_t nr;                   /* R(r) bins per problem */
    double *sums;                 /* n_problems * PMO_SS_N, accumulated */
    float *bins;                  /* n_problems * nr * PMO_SB_N, accumulated */
    uint32_t *remaining;          /* per problem photons in flight, or NULL */
    unsigned long long *t_done;   /* per problem completion time, or NULL */
    int32_t precision;            /* PMO_FP32 or PMO_FP64 */
    uint32_t max_events;          /* 0 = 2^26 */
} pmo_stack_batch;

/*
 * Many layered slab problems in one persistent launch, forward and gradient
 * together: the batched form of pmo_run_batched for PlateModel stacks.  Same
 * work queue, Philox layout (problem p uses stream word 4p + s) and transport
 * rules; a stack of one layer follows the photons of pmo_run_batched.  At an
 * inner interface with equal refractive indices the photon keeps its optical
 * depth and takes the next layer's mu (:154-167); otherwise Fresnel /
 * refraction as at an outer face.  Sums go to global memory with atomics.
 * No counterpart in the reference, which runs one problem per launch.
 */
int pmo_run_stack_batch(const pmo_stack_batch *batch, const pmo_launch *launch,
                        void *workspace, size_t workspace_bytes, void *stream);

/* Per-problem results (n_problems * PMO_SR_N doubles) and R(r) with its
   per-layer derivatives (n_problems * nr * PMO_SB_N doubles) from the sums. */
int pmo_stack_batch_finalize(const pmo_stack_batch *batch, double *results, double *rr,
                             void *stream);

/*
 * pmo_run_plain without a caller-allocated workspace.  No counterpart in the
 * reference.  For callers that cannot allocate device memory themselves (a
 * plugin in a host application that owns all device memory through its own
 * pool, or a path where cudaMalloc, which may synchronise the device, is not
 * allowed): the scratch lives in a file-scope device array of
 * PMO_STATIC_WORKSPACE_BYTES bytes that every GPU loading the library holds
 * until exit.  Returns PMO_ERR_WORKSPACE if the run needs more scratch than
 * that.  The first call in a CUDA context (the device's primary context, or a
 * context the caller made current) looks up the array's device address with
 * that context current and caches it for that context only, so a context
 * created after cudaDeviceReset gets a fresh lookup; make that first call
 * before any stream capture.  All
 * calls share the array: calls on one stream in sequence are fine, calls that
 * overlap on the GPU (other streams or host threads) race on it.  Allocates
 * nothing; the caller still passes the problem and the tally buffers.
 */
#define PMO_STATIC_WORKSPACE_BYTES 512
int pmo_run_plain_static(const pmo_problem *prob, const pmo_tallies *tal,
                         const pmo_launch *launch, void *stream);

/*
 * Drop-in for the reference kernel cuVMC (pymopt/voxel_gpu/_cukernel.py:27-35):
 * same argument list and meaning (SoA state add[3*nPh], p[3*nPh], v[3*nPh],
 * w[nPh] updated in place; ma/ms/g indexed by label < end_point; n indexed
 * by label <= end_point; voxel index (x*M + y)*L + z), plus `nx`
 * (voxel_model.shape[0], for bounds checking), a workspace and a stream.
 * The random stream is the Philox scheme above with seed = rand_seed.
 */
int pmo_cuvmc(int32_t *add, float *p, float *v, float *w,
              const float *ma, const float *ms, const float *n, const float *g,
              const int8_t *voxel_model, float l, int32_t M, int32_t L,
              int32_t nPh, int8_t end_point, int32_t rand_seed, int32_t nx,
              void *workspace, size_t workspace_bytes, void *stream);

/*
 * Fluence normalisation in FP64: phi = absorbed * 2^-PMO_ABSORBED_SHIFT
 * / (n_photons * l^3 * mu_a)
 * over the interior (nx-2, ny-2, nz-2) of the padded grid; voxels with
 * mu_a == 0 get 0.  mu_a comes from the label table or the voxel grid of
 * `prob`.  No counterpart in the reference GPU path (the reference tallies
 * fluence only in pymopt/fluence/intarnal_fluence.py:12-152, on the host).
 */
int pmo_normalize_fluence(const pmo_problem *prob, const unsigned long long *absorbed,
                          double n_photons, double *phi_out, void *stream);

/* ---- optical bench after the transport (pymopt.optics OBD) ---------------- */

/* Element parameters of the reference's OBD and SideOBD
   (pymopt/optics/_classes.py:381-402, keys of OBD.params; lengths in mm). */
typedef struct pmo_obd_params {
    double outer_d1, ct1, r1, n1, bfl1;     /* lens 1 (N-BK7 by default) */
    double outer_d2, ct2, r2, n2, bfl2;     /* lens 2 (N-SF11 by default) */
    double slit_d, slit_width, slit_thickness, distance_2slits;
    double d_pd, pd_correction;             /* photodiode diameter, z offset */
    int32_t ld_fix_part;                    /* laser-diode mount between the slits */
    int32_t side;                           /* SideOBD: x shifted by -(Z + side_dz) * side_tan */
    double side_dz, side_tan;
    const double *z;                        /* device array: the scan's Z offsets */
    int32_t n_z;                            /* 1 .. 4096 */
    uint64_t seed;                          /* Philox key of the Fresnel decisions */
    double fixed_u;                         /* in [0, 1): use it instead of every
                                               draw (deterministic); < 0: draw */
} pmo_obd_params;

/* Intensity at the photodiode for every Z of a scan: intensity[i] +=
   sum of w over the exit photons (p, v, w: SoA device arrays, 3n/3n/n floats,
   already selected and prepared as OBD.opticalAnalysisMeth does,
   pymopt/optics/_classes.py:495-526) that pass lens 1, the slits, the
   optional mount and lens 2 at detector offset z[i] and land on the
   photodiode.  Restates the reference's NumPy ray tracing
   (pymopt/optics/_classes.py:50-380, :454-493, :528-566) per photon;
   intensity is an FP64 device array of n_z, accumulated. */
int pmo_run_obd(const pmo_obd_params *prm, const float *p, const float *v, const float *w, int64_t n,
            double *intensity, void *stream);

/* ---- test and benchmark hooks ------------------------------------------
   The three entry points below serve the test-suite and bench.py only (the
   random-stream known-answer checks and the measured denominator of the
   roofline); no transport path calls them. */

/* Test hook.  Philox4x32-10 words of the engine's generator for n counters ctr[4*n]
   (device arrays) under key (key0, key1): known-answer checks of the random
   stream layout.  No counterpart in the reference (it uses cuRAND XORWOW,
   pymopt/voxel_gpu/_cukernel.py:42-43). */
int pmo_philox_words(const uint32_t *ctr, uint32_t key0, uint32_t key1,
                     uint32_t *out, int n, void *stream);

/* Test hook.  cuRAND's Philox4_32_10 for comparison: words of curand4() after
   curand_init(seed, subsequence[i], 4 * block[i]). */
int pmo_philox_words_curand(unsigned long long seed,
                            const unsigned long long *subsequence,
                            const unsigned long long *block, uint32_t *out,
                            int n, void *stream);

/* Benchmark hook.  FP32 issue-rate probe: blocks x threads threads each issue iters * 128
   independent FFMA instructions.  Timed by the caller; gives the measured
   denominator of the FP32-issue roofline.  No counterpart in the reference. */
int pmo_fp32_probe(float *out, int blocks, int threads, int iters, void *stream);

/* Uniform-box map of a label volume.  words[i] = labels[i] | d << 8 | c << 12
   describes a box {|dx|, |dy| <= e, |dz| <= d} of voxels around voxel i that
   all carry labels[i] and lie inside the array:
   - d (0 .. cap, cap <= 15) is the Chebyshev distance from voxel i to the
     nearest voxel with a 26-neighbour of another label (array border
     counted as such);
   - e = max(d, lat(c)) with lat(0) = 0 and
     lat(c) = ((2 | (c & 1)) << (c >> 1)) >> 1 (1, 2, 3, 4, 6, ... 192);
   - c is the largest code whose lat(c) does not exceed the smallest
     in-plane uniform radius over the box's z-planes.
   scratch: PMO_VOXEL_WORDS_SCRATCH * nx*ny*nz bytes of device memory,
   4-byte aligned; nx*ny*nz < 2^32.  No counterpart in the reference, which
   steps voxel by voxel (pymopt/voxel_gpu/_cukernel.py:77-176). */
#define PMO_VOXEL_WORDS_SCRATCH 5   /* scratch bytes per voxel */
int pmo_build_voxel_words(const uint8_t *labels, int nx, int ny, int nz, int cap,
                          uint16_t *words, void *scratch, size_t scratch_bytes,
                          void *stream);

/* Turn device-side counters (after the caller synchronised) into a status. */
int pmo_check_counters(const unsigned long long *host_counters);

#ifdef __cplusplus
}
#endif
#endif /* PMO_B200_H */
