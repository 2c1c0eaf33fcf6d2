// pmo_internal.h — shared between the kernel translation units and the C ABI.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/pmo_b200.h"
#include "philox.cuh"

namespace pmo {

// Device scratch the run entry points need (pmo_workspace_bytes): the photon
// chunk counter, and pmo_cuvmc's ledger and counters at PMO_WS_LEDGER_OFFSET
// and PMO_WS_COUNTERS_OFFSET.
constexpr size_t kWorkspaceBytes = 512;
static_assert(PMO_WS_COUNTERS_OFFSET + PMO_COUNTERS_N * sizeof(unsigned long long) <=
                  kWorkspaceBytes,
              "pmo_cuvmc's counters must fit in the workspace");
static_assert(kWorkspaceBytes <= PMO_STATIC_WORKSPACE_BYTES,
              "pmo_run_plain_static must be able to provide the workspace");

// Everything a transport kernel reads, passed by value (kernel parameter
// space).  Built by the C ABI from pmo_problem / pmo_tallies.
struct KParams {
    // geometry
    const uint8_t *labels;
    const uint16_t *words;         // label | uniform-box radius << 8, or null
    int32_t nx, ny, nz;
    uint32_t sx, sy;               // strides of x and y in the label volume
    float l, hl, inv_l;            // voxel size, l/2, 1/l
    int32_t end_label;
    int32_t n_labels;
    // optics
    const float *ma, *ms, *g, *n;
    const float *vox_ma, *vox_ms;
    // source
    int32_t source;
    int32_t src_ix, src_iy, src_iz;
    float src_p[3], src_v[3];
    float src_w0, beam_sigma, spec_prob;
    float spec_v[3];
    int32_t cx, cy;
    int32_t *state_add;
    float *state_p, *state_v, *state_w;
    // photons
    uint32_t key0, key1;
    PhiloxKeys rk;                 // round keys of (key0, key1)
    uint64_t begin, count;
    uint32_t max_events;
    uint32_t flags;
    // tallies
    double *ledger;
    unsigned long long *counters;
    float *rr;
    int32_t nr;
    float dr;
    // exit histograms: angle-resolved (2 x n_ang) and line profile (n_line)
    float *ang;
    int32_t n_ang;
    float inv_da;                  // 2 * n_ang / pi
    float *line;
    int32_t n_line;
    float line_dr, line_y;
    // R(r), angle and line histograms privatised in shared memory (hist_n
    // entries: PMO_RR_CATS * nr + 2 * n_ang + n_line) when they are small
    int32_t rr_shared;
    int32_t hist_n;
    unsigned long long *absorbed;  // fixed point, 2^PMO_ABSORBED_SHIFT per unit
    int32_t win_lo[3], win_dim[3]; // shared fluence window (PMO_FLU_SHARED)
    int32_t *exit_add;
    float *exit_p, *exit_v, *exit_w;
    uint32_t *ph_interact, *ph_cross, *ph_fresnel;
    int32_t *score_bin;            // forward: written; gradient replay: read
    float *score_w;
    // gradient replay
    const float *coef;             // dLoss/d(bin weight), [PMO_RR_CATS][nr]
    float *d_ma_voxel, *d_ms_voxel;
    double *d_ma_label, *d_ms_label;
    unsigned long long *gcounters;
    const int16_t *fd_target;      // pMC-reweighted central difference
    int32_t fd_n, fd_param;
    float fd_h;
    double *fd_out;
    // scratch: [0] next photon chunk
    unsigned long long *work;
};

// Launch configuration chosen by the caller or by the occupancy query.
struct LaunchShape {
    int block_threads;
    int blocks;
    size_t smem;
};

// vmc_plain.cu
cudaError_t launch_grad(const KParams &kp, int precision, int props_mode, int block_threads,
                        int blocks_per_sm, cudaStream_t stream);
cudaError_t launch_plain(const KParams &kp, int precision, int props_mode, int fluence_mode,
                         int block_threads, int blocks_per_sm, cudaStream_t stream,
                         LaunchShape *shape_out);
cudaError_t launch_normalize_fluence(const KParams &kp, int props_mode,
                                     const unsigned long long *absorbed,
                                     double n_photons, double *phi, cudaStream_t stream);

}  // namespace pmo
