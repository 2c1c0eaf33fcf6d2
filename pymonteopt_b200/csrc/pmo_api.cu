// pmo_api.cu — the C ABI of include/pmo_b200.h: argument validation, kernel
// parameter assembly, dispatch to the FP32/FP64 transport instantiations, and
// the FP64 fluence normalisation kernel.
#include <cmath>
#include <cstring>

#include "pmo_internal.h"

namespace pmo {
cudaError_t launch_plain_f32(const KParams &kp, int props, int flu, int threads, int bps,
                             cudaStream_t s, LaunchShape *out);
cudaError_t launch_plain_f64(const KParams &kp, int props, int flu, int threads, int bps,
                             cudaStream_t s, LaunchShape *out);
cudaError_t launch_grad_f32(const KParams &kp, int props, int threads, int bps, cudaStream_t s);
cudaError_t launch_grad_f64(const KParams &kp, int props, int threads, int bps, cudaStream_t s);

// phi = absorbed * 2^-PMO_ABSORBED_SHIFT / (n_photons * l^3 * mu_a) over the
// interior voxels, FP64.
__global__ void normalize_fluence_kernel(const unsigned long long *__restrict__ absorbed,
                                         const uint8_t *__restrict__ labels,
                                         const float *__restrict__ ma_tab,
                                         const float *__restrict__ vox_ma, int props_mode,
                                         int end_label, int nx, int ny, int nz, double scale,
                                         double *__restrict__ phi) {
    const uint64_t ix_n = (uint64_t)(nx - 2), iy_n = (uint64_t)(ny - 2), iz_n = (uint64_t)(nz - 2);
    const uint64_t total = ix_n * iy_n * iz_n;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t z = i % iz_n, y = (i / iz_n) % iy_n, x = i / (iz_n * iy_n);
        const uint64_t lin = ((x + 1) * (uint64_t)ny + (y + 1)) * (uint64_t)nz + (z + 1);
        const int lab = labels[lin];
        double ma = 0.0;
        if (lab != end_label) ma = props_mode == PMO_PROPS_VOXEL ? (double)vox_ma[lin] : (double)ma_tab[lab];
        phi[i] = ma > 0.0 ? (double)absorbed[lin] * scale / ma : 0.0;
    }
}

cudaError_t launch_normalize_fluence(const KParams &kp, int props_mode,
                                     const unsigned long long *absorbed,
                                     double n_photons, double *phi, cudaStream_t stream) {
    const double l = (double)kp.l;
    const double scale = 1.0 / (n_photons * l * l * l) / (double)(1ull << PMO_ABSORBED_SHIFT);
    const uint64_t total = (uint64_t)(kp.nx - 2) * (kp.ny - 2) * (kp.nz - 2);
    uint64_t blocks = (total + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    if (blocks < 1) blocks = 1;
    normalize_fluence_kernel<<<(unsigned)blocks, 256, 0, stream>>>(
        absorbed, kp.labels, kp.ma, kp.vox_ma, props_mode, kp.end_label, kp.nx, kp.ny, kp.nz,
        scale, phi);
    return cudaGetLastError();
}

}  // namespace pmo

using pmo::KParams;
using pmo::kWorkspaceBytes;

namespace {

constexpr size_t kWsLedgerOff = PMO_WS_LEDGER_OFFSET;
constexpr size_t kWsCountersOff = PMO_WS_COUNTERS_OFFSET;

bool finite_pos(float x) { return std::isfinite(x) && x > 0.f; }

// Fill the geometry/optics/source part of KParams from a problem.
int problem_to_params(const pmo_problem *p, KParams *kp) {
    if (!p || !p->labels) return PMO_ERR_ARG;
    if (p->nx < 3 || p->ny < 3 || p->nz < 3) return PMO_ERR_ARG;
    const uint64_t vox = (uint64_t)p->nx * (uint64_t)p->ny * (uint64_t)p->nz;
    if (vox >= (1ull << 32)) return PMO_ERR_ARG;
    if (!finite_pos(p->voxel_space)) return PMO_ERR_ARG;
    if (p->n_labels < 1 || p->n_labels > 256) return PMO_ERR_ARG;
    if (p->end_label < 0 || p->end_label >= p->n_labels) return PMO_ERR_ARG;
    if (!p->n || !p->g) return PMO_ERR_ARG;
    if (p->props_mode == PMO_PROPS_LABEL) {
        if (!p->ma || !p->ms) return PMO_ERR_ARG;
    } else if (p->props_mode == PMO_PROPS_VOXEL) {
        if (!p->vox_ma || !p->vox_ms) return PMO_ERR_ARG;
    } else {
        return PMO_ERR_ARG;
    }
    if (p->source != PMO_SRC_PENCIL && p->source != PMO_SRC_GAUSSIAN && p->source != PMO_SRC_STATE)
        return PMO_ERR_ARG;
    if (p->source == PMO_SRC_STATE &&
        (!p->state_add || !p->state_p || !p->state_v || !p->state_w))
        return PMO_ERR_ARG;
    if (p->source == PMO_SRC_GAUSSIAN && !(std::isfinite(p->beam_sigma) && p->beam_sigma >= 0.f))
        return PMO_ERR_ARG;
    if (!(p->spec_prob >= 0.f && p->spec_prob <= 1.f)) return PMO_ERR_ARG;
    if (p->precision != PMO_FP32 && p->precision != PMO_FP64) return PMO_ERR_ARG;

    std::memset(kp, 0, sizeof(*kp));
    kp->labels = p->labels;
    kp->words = p->voxel_words;
    kp->nx = p->nx;
    kp->ny = p->ny;
    kp->nz = p->nz;
    kp->sx = (uint32_t)p->ny * (uint32_t)p->nz;
    kp->sy = (uint32_t)p->nz;
    kp->l = p->voxel_space;
    kp->hl = p->voxel_space * 0.5f;
    kp->inv_l = 1.0f / p->voxel_space;
    kp->end_label = p->end_label;
    kp->n_labels = p->n_labels;
    kp->ma = p->ma;
    kp->ms = p->ms;
    kp->g = p->g;
    kp->n = p->n;
    kp->vox_ma = p->vox_ma;
    kp->vox_ms = p->vox_ms;
    kp->source = p->source;
    kp->src_ix = p->src_ix;
    kp->src_iy = p->src_iy;
    kp->src_iz = p->src_iz;
    for (int a = 0; a < 3; ++a) {
        kp->src_p[a] = p->src_p[a];
        kp->src_v[a] = p->src_v[a];
        kp->spec_v[a] = p->spec_v[a];
    }
    kp->src_w0 = p->src_w0;
    kp->beam_sigma = p->beam_sigma;
    kp->spec_prob = p->spec_prob;
    kp->cx = p->center_ix;
    kp->cy = p->center_iy;
    kp->state_add = p->state_add;
    kp->state_p = p->state_p;
    kp->state_v = p->state_v;
    kp->state_w = p->state_w;
    kp->key0 = (uint32_t)p->seed;
    kp->key1 = (uint32_t)(p->seed >> 32);
    kp->rk = pmo::philox_round_keys(kp->key0, kp->key1);
    kp->begin = p->photon_begin;
    kp->count = p->photon_count;
    kp->max_events = p->max_events;
    kp->flags = p->flags;
    return PMO_OK;
}

int tallies_to_params(const pmo_problem *p, const pmo_tallies *t, KParams *kp) {
    if (!t || !t->ledger || !t->counters) return PMO_ERR_ARG;
    if (t->nr < 0) return PMO_ERR_ARG;
    if (t->nr > 0 && (!t->rr || !finite_pos(t->dr))) return PMO_ERR_ARG;
    if (t->ang && (t->n_ang < 0 || t->n_ang > 1 << 20)) return PMO_ERR_ARG;
    if (t->line && (t->n_line < 0 || t->n_line > 1 << 20 ||
                    (t->n_line > 0 && (!finite_pos(t->line_dr) || !finite_pos(t->line_y_range)))))
        return PMO_ERR_ARG;
    if (t->fluence_mode != PMO_FLU_NONE && t->fluence_mode != PMO_FLU_GLOBAL &&
        t->fluence_mode != PMO_FLU_SHARED)
        return PMO_ERR_ARG;
    if (t->fluence_mode != PMO_FLU_NONE && !t->absorbed) return PMO_ERR_ARG;
    if (t->fluence_mode == PMO_FLU_SHARED) {
        const int dims[3] = {p->nx, p->ny, p->nz};
        uint64_t cells = 1;
        for (int a = 0; a < 3; ++a) {
            if (t->win_dim[a] < 1 || t->win_lo[a] < 0 || t->win_lo[a] + t->win_dim[a] > dims[a])
                return PMO_ERR_ARG;
            cells *= (uint64_t)t->win_dim[a];
        }
        if (cells * sizeof(unsigned long long) > 160 * 1024) return PMO_ERR_ARG;
    }
    if ((p->flags & PMO_FLAG_EXPORT_EXITS) &&
        (!t->exit_add || !t->exit_p || !t->exit_v || !t->exit_w))
        return PMO_ERR_ARG;
    if ((p->flags & PMO_FLAG_PHOTON_STATS) && (!t->ph_interact || !t->ph_cross || !t->ph_fresnel))
        return PMO_ERR_ARG;
    kp->ledger = t->ledger;
    kp->counters = t->counters;
    kp->rr = t->rr;
    kp->nr = t->nr;
    kp->dr = t->dr;
    kp->n_ang = t->ang ? t->n_ang : 0;
    kp->ang = t->ang;
    kp->inv_da = kp->n_ang > 0 ? (float)(2.0 * kp->n_ang / 3.14159265358979323846) : 0.f;
    kp->n_line = t->line ? t->n_line : 0;
    kp->line = t->line;
    kp->line_dr = t->line_dr;
    kp->line_y = t->line_y_range;
    // privatise the exit histograms in shared memory when they are small
    const int hist = PMO_RR_CATS * (t->nr > 0 ? t->nr : 0) + 2 * kp->n_ang + kp->n_line;
    kp->rr_shared = (hist > 0 && hist <= 4096) ? 1 : 0;
    kp->hist_n = kp->rr_shared ? hist : 0;
    kp->absorbed = t->absorbed;
    for (int a = 0; a < 3; ++a) {
        kp->win_lo[a] = t->win_lo[a];
        kp->win_dim[a] = t->fluence_mode == PMO_FLU_SHARED ? t->win_dim[a] : 0;
    }
    kp->exit_add = t->exit_add;
    kp->exit_p = t->exit_p;
    kp->exit_v = t->exit_v;
    kp->exit_w = t->exit_w;
    kp->ph_interact = t->ph_interact;
    kp->ph_cross = t->ph_cross;
    kp->ph_fresnel = t->ph_fresnel;
    if ((p->flags & PMO_FLAG_SCORE_RECORD) && (!t->score_bin || !t->score_w || t->nr <= 0))
        return PMO_ERR_ARG;
    kp->score_bin = t->score_bin;
    kp->score_w = t->score_w;
    return PMO_OK;
}

// Default block of the plain transport: 256 threads.  At 64 registers a
// thread, 4 such blocks fill an SM as 8 blocks of 128 do; measured on one
// B200, 256 was 0.2-0.8 % faster on the skin slab, the CT-like volume (with
// and without the fluence grid) and the homogeneous slab.
constexpr int kPlainThreads = 256;

int launch_kp(const KParams &kp, int precision, int props, int flu, const pmo_launch *launch,
              cudaStream_t s) {
    int threads = launch && launch->block_threads > 0 ? launch->block_threads : kPlainThreads;
    if (threads % 32 != 0 || threads > 512) return PMO_ERR_ARG;
    const int bps = launch ? launch->blocks_per_sm : 0;
    cudaError_t e = cudaMemsetAsync(kp.work, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return PMO_ERR_CUDA;
    e = precision == PMO_FP64 ? pmo::launch_plain_f64(kp, props, flu, threads, bps, s, nullptr)
                              : pmo::launch_plain_f32(kp, props, flu, threads, bps, s, nullptr);
    return e == cudaSuccess ? PMO_OK : PMO_ERR_CUDA;
}

}  // namespace

extern "C" {

int pmo_abi_version(void) { return PMO_ABI_VERSION; }

const char *pmo_status_string(int status) {
    switch (status) {
        case PMO_OK: return "ok";
        case PMO_ERR_ARG: return "bad argument";
        case PMO_ERR_GEOMETRY: return "photon stepped outside the volume";
        case PMO_ERR_LABEL: return "photon entered a label without optical properties";
        case PMO_ERR_STEP_CAP: return "photon exceeded its event cap";
        case PMO_ERR_CUDA: return "CUDA runtime error";
        case PMO_ERR_WORKSPACE: return "workspace missing or too small";
        case PMO_ERR_TIMEOUT: return "bounded device wait timed out";
        case PMO_ERR_NUMERIC: return "non-finite weight or direction";
        default: return "unknown status";
    }
}

int pmo_device_info(int *sm_count, int *cc_major, int *cc_minor) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PMO_ERR_CUDA;
    if (sm_count && cudaDeviceGetAttribute(sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return PMO_ERR_CUDA;
    if (cc_major && cudaDeviceGetAttribute(cc_major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess)
        return PMO_ERR_CUDA;
    if (cc_minor && cudaDeviceGetAttribute(cc_minor, cudaDevAttrComputeCapabilityMinor, dev) != cudaSuccess)
        return PMO_ERR_CUDA;
    return PMO_OK;
}

size_t pmo_workspace_bytes(void) { return kWorkspaceBytes; }

int pmo_run_plain(const pmo_problem *prob, const pmo_tallies *tal, const pmo_launch *launch,
                  void *workspace, size_t workspace_bytes, void *stream) {
    KParams kp;
    int st = problem_to_params(prob, &kp);
    if (st != PMO_OK) return st;
    st = tallies_to_params(prob, tal, &kp);
    if (st != PMO_OK) return st;
    if (!workspace || workspace_bytes < kWorkspaceBytes) return PMO_ERR_WORKSPACE;
    kp.work = static_cast<unsigned long long *>(workspace);
    if (prob->photon_count == 0) return PMO_OK;
    return launch_kp(kp, prob->precision, prob->props_mode, tal->fluence_mode, launch,
                     static_cast<cudaStream_t>(stream));
}

int pmo_run_grad(const pmo_problem *prob, const pmo_grad *g, const pmo_launch *launch,
                 void *workspace, size_t workspace_bytes, void *stream) {
    KParams kp;
    int st = problem_to_params(prob, &kp);
    if (st != PMO_OK) return st;
    if (!g || !g->coef || g->nr <= 0 || !finite_pos(g->dr) || !g->score_bin || !g->score_w ||
        !g->counters)
        return PMO_ERR_ARG;
    if ((g->d_ma_voxel == nullptr) != (g->d_ms_voxel == nullptr)) return PMO_ERR_ARG;
    if ((g->d_ma_label == nullptr) != (g->d_ms_label == nullptr)) return PMO_ERR_ARG;
    if (!g->d_ma_voxel && !g->d_ma_label) return PMO_ERR_ARG;
    // per-voxel derivatives need the voxel-by-voxel path
    if (g->d_ma_voxel && prob->voxel_words) return PMO_ERR_ARG;
    if (!workspace || workspace_bytes < kWorkspaceBytes) return PMO_ERR_WORKSPACE;
    if (prob->photon_count == 0) return PMO_OK;
    int threads = launch && launch->block_threads > 0 ? launch->block_threads : 128;
    if (threads % 32 != 0 || threads > 512) return PMO_ERR_ARG;
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(ws, 0, kWorkspaceBytes, s) != cudaSuccess) return PMO_ERR_CUDA;
    kp.work = reinterpret_cast<unsigned long long *>(ws);
    kp.ledger = reinterpret_cast<double *>(ws + kWsLedgerOff);
    kp.counters = reinterpret_cast<unsigned long long *>(ws + kWsCountersOff);
    kp.nr = g->nr;
    kp.dr = g->dr;
    kp.coef = g->coef;
    kp.score_bin = const_cast<int32_t *>(g->score_bin);
    kp.score_w = const_cast<float *>(g->score_w);
    kp.d_ma_voxel = g->d_ma_voxel;
    kp.d_ms_voxel = g->d_ms_voxel;
    kp.d_ma_label = g->d_ma_label;
    kp.d_ms_label = g->d_ms_label;
    kp.gcounters = g->counters;
    if (g->fd_n > 0) {
        if (g->fd_n > PMO_FD_MAX || !g->fd_target || !g->fd_out || !(g->fd_h > 0.f) ||
            (g->fd_param != 0 && g->fd_param != 1))
            return PMO_ERR_ARG;
        kp.fd_target = g->fd_target;
        kp.fd_n = g->fd_n;
        kp.fd_param = g->fd_param;
        kp.fd_h = g->fd_h;
        kp.fd_out = g->fd_out;
    }
    kp.flags = 0;
    const int bps = launch ? launch->blocks_per_sm : 0;
    cudaError_t e = prob->precision == PMO_FP64
                        ? pmo::launch_grad_f64(kp, prob->props_mode, threads, bps, s)
                        : pmo::launch_grad_f32(kp, prob->props_mode, threads, bps, s);
    return e == cudaSuccess ? PMO_OK : PMO_ERR_CUDA;
}

int pmo_cuvmc(int32_t *add, float *p, float *v, float *w, const float *ma, const float *ms,
              const float *n, const float *g, const int8_t *voxel_model, float l, int32_t M,
              int32_t L, int32_t nPh, int8_t end_point, int32_t rand_seed, int32_t nx,
              void *workspace, size_t workspace_bytes, void *stream) {
    if (!add || !p || !v || !w || !ma || !ms || !n || !g || !voxel_model) return PMO_ERR_ARG;
    if (nPh < 0 || end_point < 0) return PMO_ERR_ARG;
    if (!workspace || workspace_bytes < kWorkspaceBytes) return PMO_ERR_WORKSPACE;
    pmo_problem pr;
    std::memset(&pr, 0, sizeof(pr));
    pr.labels = reinterpret_cast<const uint8_t *>(voxel_model);
    pr.nx = nx;
    pr.ny = M;
    pr.nz = L;
    pr.voxel_space = l;
    pr.end_label = end_point;
    pr.props_mode = PMO_PROPS_LABEL;
    pr.n_labels = (int)end_point + 1;  // ma/ms/g: end_point entries; n: end_point + 1
    pr.ma = ma;
    pr.ms = ms;
    pr.g = g;
    pr.n = n;
    pr.source = PMO_SRC_STATE;
    pr.state_add = add;
    pr.state_p = p;
    pr.state_v = v;
    pr.state_w = w;
    pr.seed = (uint64_t)(uint32_t)rand_seed;
    pr.photon_begin = 0;
    pr.photon_count = (uint64_t)nPh;
    pr.precision = PMO_FP32;
    pr.flags = PMO_FLAG_EXPORT_EXITS;
    KParams kp;
    int st = problem_to_params(&pr, &kp);
    if (st != PMO_OK) return st;
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(ws, 0, kWorkspaceBytes, s) != cudaSuccess) return PMO_ERR_CUDA;
    kp.ledger = reinterpret_cast<double *>(ws + kWsLedgerOff);
    kp.counters = reinterpret_cast<unsigned long long *>(ws + kWsCountersOff);
    kp.exit_add = add;
    kp.exit_p = p;
    kp.exit_v = v;
    kp.exit_w = w;
    kp.work = reinterpret_cast<unsigned long long *>(ws);
    if (nPh == 0) return PMO_OK;
    return launch_kp(kp, PMO_FP32, PMO_PROPS_LABEL, PMO_FLU_NONE, nullptr, s);
}

int pmo_normalize_fluence(const pmo_problem *prob, const unsigned long long *absorbed,
                          double n_photons,
                          double *phi_out, void *stream) {
    KParams kp;
    int st = problem_to_params(prob, &kp);
    if (st != PMO_OK) return st;
    if (!absorbed || !phi_out || !(n_photons > 0.0)) return PMO_ERR_ARG;
    cudaError_t e = pmo::launch_normalize_fluence(kp, prob->props_mode, absorbed, n_photons,
                                                  phi_out, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? PMO_OK : PMO_ERR_CUDA;
}

int pmo_check_counters(const unsigned long long *c) {
    if (!c) return PMO_ERR_ARG;
    if (c[PMO_C_ERR_GEOM]) return PMO_ERR_GEOMETRY;
    if (c[PMO_C_ERR_LABEL]) return PMO_ERR_LABEL;
    if (c[PMO_C_ERR_CAP]) return PMO_ERR_STEP_CAP;
    if (c[PMO_C_ERR_NUM]) return PMO_ERR_NUMERIC;
    return PMO_OK;
}

}  // extern "C"
