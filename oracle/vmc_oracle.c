/*
 * vmc_oracle.c — CPU oracle for the voxel Monte Carlo transport path.
 *
 * TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py load this library, and only as the checker or as
 * the timed CPU restatement of the reference; the product path never does.
 *
 * What it restates: the reference transport kernel cuVMC
 * (pymopt/voxel_gpu/_cukernel.py:27-227) and its Numba twin vmc_kernel
 * (pymopt/voxel/_kernel.py:23-172), plus the host reductions around them:
 * photon source (pymopt/voxel_gpu/_classes.py:148-254), Rd/Tt split by the
 * sign of v_z (:326-334), exit-position encoding (:302-310) and R(r) binning
 * (pymopt/metrics/_scoring.py:16-25).  The random numbers follow the Philox
 * layout of include/pmo_b200.h, so photon p of (seed, optics) has the same
 * history here and in the device kernels: in FP64 the two agree per photon to
 * rounding; the FP32 build is the timed CPU baseline.
 *
 * Build: oracle/build.py (gcc -O2 -fopenmp -shared).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/pmo_b200.h"
#include "philox_ref.h"

#define PMO_CAT_(a, b) a##b
#define PMO_CAT(a, b) PMO_CAT_(a, b)

typedef struct oracle_tallies {
    double ledger[PMO_LEDGER_N];
    unsigned long long counters[PMO_COUNTERS_N];
    double *rr;           /* PMO_RR_CATS * nr or NULL */
    int32_t nr;
    double dr;
    double *absorbed;     /* nx*ny*nz or NULL */
    double *ph_state;     /* 10 per photon: p[3], v[3], w, add[3]; or NULL */
    uint32_t *ph_counts;  /* 4 per photon: interactions, crossings, fresnel, status */
    /* perturbation Monte Carlo gradient (all NULL or all set): for a photon
       whose exit weight w lands in bin b, q = grad_coef[b] * w is spread over
       the voxels it crossed: g_ma += -q*L, g_ms += q*(n/mu_s - L) */
    const double *grad_coef;          /* PMO_RR_CATS * nr */
    double *g_ma_voxel, *g_ms_voxel;  /* nx*ny*nz */
    double *g_ma_label, *g_ms_label;  /* n_labels */
} oracle_tallies;

/* per-thread scratch: ledger, counters and a photon's cell log */
typedef struct {
    double ledger[PMO_LEDGER_N];
    unsigned long long counters[PMO_COUNTERS_N];
    int nseg, capseg;
    int64_t *seg_lin;
    int *seg_lab;
    double *seg_L, *seg_N;
} oracle_acc;

static void seg_push(oracle_acc *acc, int64_t lin, int lab, double L, double N) {
    if (L == 0.0 && N == 0.0) return;
    if (acc->nseg == acc->capseg) {
        int cap = acc->capseg ? 2 * acc->capseg : 256;
        acc->seg_lin = (int64_t *)realloc(acc->seg_lin, cap * sizeof(int64_t));
        acc->seg_lab = (int *)realloc(acc->seg_lab, cap * sizeof(int));
        acc->seg_L = (double *)realloc(acc->seg_L, cap * sizeof(double));
        acc->seg_N = (double *)realloc(acc->seg_N, cap * sizeof(double));
        acc->capseg = cap;
    }
    acc->seg_lin[acc->nseg] = lin;
    acc->seg_lab[acc->nseg] = lab;
    acc->seg_L[acc->nseg] = L;
    acc->seg_N[acc->nseg] = N;
    acc->nseg++;
}

static void seg_apply(oracle_acc *acc, const oracle_tallies *tal, double q) {
    for (int i = 0; i < acc->nseg; ++i) {
        const double dma = -q * acc->seg_L[i];
        const double dms = q * acc->seg_N[i] - q * acc->seg_L[i];
        if (tal->g_ma_voxel) {
#pragma omp atomic
            tal->g_ma_voxel[acc->seg_lin[i]] += dma;
#pragma omp atomic
            tal->g_ms_voxel[acc->seg_lin[i]] += dms;
        }
        if (tal->g_ma_label) {
#pragma omp atomic
            tal->g_ma_label[acc->seg_lab[i]] += dma;
#pragma omp atomic
            tal->g_ms_label[acc->seg_lab[i]] += dms;
        }
    }
}

/* ---- FP32 build ---- */
#define REAL float
#define SUFFIX _f32
#define LOG logf
#define SQRT sqrtf
#define SIN sinf
#define COS cosf
#define FABS fabsf
#define FLOOR floorf
#define CEIL ceilf
#define TWO_PI 6.28318530717958647692f
#include "vmc_oracle_body.h"
#undef REAL
#undef SUFFIX
#undef LOG
#undef SQRT
#undef SIN
#undef COS
#undef FABS
#undef FLOOR
#undef CEIL
#undef TWO_PI

/* ---- FP64 build ---- */
#define REAL double
#define SUFFIX _f64
#define LOG log
#define SQRT sqrt
#define SIN sin
#define COS cos
#define FABS fabs
#define FLOOR floor
#define CEIL ceil
#define TWO_PI 6.28318530717958647692
#include "vmc_oracle_body.h"

/* Exported entry point: precision chosen by P->precision. */
int oracle_run(const pmo_problem *P, oracle_tallies *tal, int threads) {
    if (!P || !tal || !P->labels || P->nx < 3 || P->ny < 3 || P->nz < 3) return PMO_ERR_ARG;
    if (P->n_labels < 1 || P->n_labels > 256 || P->end_label < 0 || P->end_label >= P->n_labels)
        return PMO_ERR_ARG;
    if (P->precision == PMO_FP64) return oracle_run_f64(P, tal, threads);
    return oracle_run_f32(P, tal, threads);
}

/* Raw Philox words, for the known-answer comparison with the device code. */
void oracle_philox(const uint32_t *ctr, const uint32_t *key, uint32_t *out, int n) {
    for (int i = 0; i < n; ++i) pmo_philox4x32_10(ctr + 4 * i, key, out + 4 * i);
}

size_t oracle_tallies_size(void) { return sizeof(oracle_tallies); }
