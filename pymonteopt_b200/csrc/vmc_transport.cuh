// vmc_transport.cuh — the photon-transport kernel, templated on the arithmetic
// type R (float: the product; double: the per-photon FP64 build), the
// optical-property mode and the fluence tally mode.
//
// One thread owns one photon at a time, keeps its whole state in registers and
// runs it hop -> drop -> spin until it enters the end label or dies in Russian
// roulette, following the reference kernel cuVMC
// (pymopt/voxel_gpu/_cukernel.py:27-227).  A warp pulls photon ids in chunks
// from one global counter, so a lane whose photon finished starts the next one
// at once and warps stay full until the pool runs dry (the reference launches
// one thread per photon and keeps p/v/add/w in volatile global arrays).
//
// Per block: the per-label property table (mt, 1/mt, ma/mt, n and the
// Henyey-Greenstein constants) lives in shared memory; R(r)/T(r) histograms and
// the FP64 ledger are privatised in shared memory and flushed once at the end;
// the absorbed-weight grid gets 64-bit fixed-point integer atomics (exact and
// order-independent), merged in registers while a photon stays in one voxel
// and optionally privatised in a shared window.
#pragma once
#include <cstdint>

#include "philox.cuh"
#include "pmo_internal.h"

namespace pmo {

template <typename R>
struct __align__(16) LabelProps {
    R mt, imt, ma_mt, n;       // mu_t, 1/mu_t, mu_a/mu_t, refractive index
    R hgA, hgB, hgC, hgE;      // 1+g^2, 1-g^2, 1-g, 1/(2g) (0 when g == 0)
    R hgD, ims, pad1, pad2;    // 2g, 1/mu_s (0 when mu_s == 0)
};

// ---- arithmetic.  Every single-precision add, multiply, fused multiply-add
// and divide on the photon path is an explicitly rounded intrinsic, so the
// compiler cannot fuse or split them differently in different kernel
// instantiations: the gradient replay then follows the forward run's photon
// paths bit for bit.  The FP64 build uses plain operators in a translation
// unit compiled with -fmad=false, which round every operation separately in
// the order the CPU oracle does.
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float xsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float xfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float xdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return a * b; }
__device__ __forceinline__ double xadd(double a, double b) { return a + b; }
__device__ __forceinline__ double xsub(double a, double b) { return a - b; }
__device__ __forceinline__ double xfma(double a, double b, double c) { return a * b + c; }
__device__ __forceinline__ double xdiv(double a, double b) { return a / b; }
// -ln(u) for u in (0, 1]
__device__ __forceinline__ float pneglog(float u) { return __fmul_rn(__log2f(u), -0.69314718055994531f); }
__device__ __forceinline__ double pneglog(double u) { return -log(u); }
__device__ __forceinline__ float psqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double psqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float pinvnorm(float s) { return rsqrtf(s); }
__device__ __forceinline__ double pinvnorm(double s) { return 1.0 / sqrt(s); }
// sin and cos of 2*pi*u for u in (0, 1]
__device__ __forceinline__ void psincos2pi(float u, float *s, float *c) {
    // 2*pi*(u - 1/2) lies in (-pi, pi], where the hardware sine is accurate;
    // sin(x + pi) = -sin(x), cos(x + pi) = -cos(x).
    const float a = __fmul_rn(6.28318530717958647692f, __fsub_rn(u, 0.5f));
    float ss, cc;
    __sincosf(a, &ss, &cc);
    *s = -ss;
    *c = -cc;
}
__device__ __forceinline__ void psincos2pi(double u, double *s, double *c) {
    sincospi(2.0 * u, s, c);
}
template <typename R>
__device__ __forceinline__ R sgn(R x) { return signbit(x) ? R(-1) : R(1); }
// sum of squares in the oracle's order ((x*x + y*y) + z*z)
template <typename R>
__device__ __forceinline__ R sumsq(R x, R y, R z) {
    return xfma(z, z, xfma(y, y, xmul(x, x)));
}

template <typename R>
__device__ __forceinline__ void make_props(LabelProps<R> &t, float ma, float ms, float g,
                                           float n) {
    t.mt = xadd((R)ma, (R)ms);
    t.imt = t.mt > R(0) ? xdiv(R(1), t.mt) : R(0);
    t.ma_mt = t.mt > R(0) ? xdiv((R)ma, t.mt) : R(0);
    t.n = (R)n;
    const R gg = (R)g;
    t.hgA = xfma(gg, gg, R(1));
    t.hgB = xfma(-gg, gg, R(1));
    t.hgC = xsub(R(1), gg);
    t.hgD = xmul(R(2), gg);
    t.hgE = gg != R(0) ? xdiv(R(1), xmul(R(2), gg)) : R(0);
    t.ims = ms > 0.f ? xdiv(R(1), (R)ms) : R(0);
    t.pad1 = t.pad2 = R(0);
}

// Weight -> fixed point of the absorbed grid, rounded to nearest.  dw <= 1,
// so one deposit is at most 2^PMO_ABSORBED_SHIFT.
__device__ __forceinline__ unsigned long long to_fixed(float dw) {
    return __float2ull_rn(__fmul_rn(dw, (float)(1ull << PMO_ABSORBED_SHIFT)));
}
__device__ __forceinline__ unsigned long long to_fixed(double dw) {
    return __double2ull_rn(dw * (double)(1ull << PMO_ABSORBED_SHIFT));
}

// Box half-extents (voxels) of a uniform-box map word: z half-extent d in
// bits 8-11, lateral code c in bits 12-15 with lateral half-extent
// max(d, lat(c)), lat(0) = 0, lat(c) = ((2 | (c & 1)) << (c >> 1)) >> 1.
__device__ __forceinline__ void box_extents(uint32_t word, int &bz, int &bl) {
    bz = (int)((word >> 8) & 0xfu);
    const int c = (int)(word >> 12);
    const int lat = c ? ((2 | (c & 1)) << (c >> 1)) >> 1 : 0;
    bl = lat > bz ? lat : bz;
}

// theta(g, rand) of the reference (pymopt/voxel_gpu/_cukernel.py:14-25)
template <typename R>
__device__ __forceinline__ R hg_cos(const LabelProps<R> &t, R u) {
    if (t.hgE != R(0)) {
        const R q = xdiv(t.hgB, xfma(t.hgD, u, t.hgC));
        const R c = xmul(xfma(-q, q, t.hgA), t.hgE);
        return c < R(-1) ? R(-1) : c;
    }
    return xsub(xmul(R(2), u), R(1));
}

// Dynamic shared memory layout of a transport block.
template <typename R>
struct SmemLayout {
    static constexpr size_t tab_bytes = 256 * sizeof(LabelProps<R>);
    static constexpr size_t led_off = tab_bytes;
    static constexpr size_t cnt_off = led_off + PMO_LEDGER_N * sizeof(double);
    static constexpr size_t valid_off = cnt_off + PMO_COUNTERS_N * sizeof(unsigned long long);
    static constexpr size_t gl_off = valid_off + 256;  // per-label gradient sums
    static constexpr size_t rr_off = gl_off + 2 * 256 * sizeof(double);
    // privatised exit histograms (hist_n entries), then the fluence window
    __host__ __device__ static size_t win_off(int hist_n) {
        size_t o = rr_off + (size_t)hist_n * sizeof(R);
        return (o + 15) & ~size_t(15);
    }
    __host__ __device__ static size_t total(int hist_n, int flu, const int32_t win_dim[3]) {
        size_t o = win_off(hist_n);
        if (flu == PMO_FLU_SHARED)
            o += (size_t)win_dim[0] * win_dim[1] * win_dim[2] * sizeof(unsigned long long);
        return (o + 15) & ~size_t(15);
    }
    // gradient replay with the reweighted finite difference: per-target sums
    // (2 * PMO_FD_MAX doubles) and per-thread target accumulators
    __host__ __device__ static size_t fd_bytes(int threads) {
        return 2 * PMO_FD_MAX * sizeof(double) + (size_t)threads * 2 * PMO_FD_MAX * sizeof(float);
    }
};

enum : int { kChunk = 64 };

// Face crossings a lane may process per pass of the warp loop before it
// yields.  A warp executes the crossing loop until its slowest lane is done;
// capping it keeps lanes that are ready to interact from idling behind one
// lane that crosses many faces.  The photon's sequence of operations, and so
// its result, does not depend on this value.  Measured on C2 (one B200):
// 1 -> 1.30e8 photons/s, 2 -> 0.90e8, 4 -> 0.82e8, unlimited -> 0.80e8.
// With uniform boxes a lane that crossed yields at once, so the interaction
// code runs once per pass; with voxel-by-voxel stepping, where crossings are
// as frequent as interactions, it goes on to hop in the same pass.
#ifndef PMO_CROSS_PER_ITER
#define PMO_CROSS_PER_ITER 1
#endif
constexpr int kCrossPerIter = PMO_CROSS_PER_ITER;

// With uniform boxes, face crossings are rare next to interactions, so a warp
// that runs the crossing code for one or two lanes spends a full warp
// instruction per lane used.  A lane that needs a crossing therefore waits, its state untouched,
// until at least this many lanes of its warp (or a quarter of the active
// lanes, or all of them) need one; the crossing code then runs for all of
// them at once.  Photon histories do not depend on it.
#ifndef PMO_CROSS_BATCH
#define PMO_CROSS_BATCH 8
#endif
constexpr int kCrossBatch = PMO_CROSS_BATCH;

// GRAD: the gradient replay (pmo_run_grad).  It replays the photons whose
// forward score record gives q = coef[bin] * w != 0 along the same path (same
// arithmetic, same Philox draws) and accumulates -q*L and q*(n/mu_s - L) per
// cell it crosses (a voxel, or a label-uniform box when only per-label
// derivatives are asked for).
template <typename R, int PROPS, int FLU, bool SKIP, bool GRAD = false>
__global__ void __launch_bounds__(512) vmc_plain_kernel(const KParams kp) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using L = SmemLayout<R>;
    LabelProps<R> *s_tab = reinterpret_cast<LabelProps<R> *>(smem_raw);
    double *s_led = reinterpret_cast<double *>(smem_raw + L::led_off);
    unsigned long long *s_cnt = reinterpret_cast<unsigned long long *>(smem_raw + L::cnt_off);
    uint8_t *s_valid = smem_raw + L::valid_off;
    R *s_rr = reinterpret_cast<R *>(smem_raw + L::rr_off);
    double *s_gma = reinterpret_cast<double *>(smem_raw + L::gl_off);
    double *s_gms = s_gma + 256;
    unsigned long long *s_win =
        reinterpret_cast<unsigned long long *>(smem_raw + L::win_off(kp.hist_n));
    R *s_ang = s_rr + PMO_RR_CATS * kp.nr;    // with rr_shared: 2 x n_ang
    R *s_line = s_ang + 2 * kp.n_ang;         // and n_line
    const int n_win = FLU == PMO_FLU_SHARED ? kp.win_dim[0] * kp.win_dim[1] * kp.win_dim[2] : 0;
    const bool fd = GRAD && kp.fd_n > 0;
    double *s_fdsum = reinterpret_cast<double *>(
        smem_raw + L::total(kp.hist_n, FLU, kp.win_dim));
    float *s_fdL = reinterpret_cast<float *>(s_fdsum + 2 * PMO_FD_MAX) +
                   threadIdx.x * 2 * PMO_FD_MAX;   // this thread's sum of mu * L per target
    float *s_fdN = s_fdL + PMO_FD_MAX;             // and interaction count per target

    // ---- block set-up: property table, zeroed privatised tallies ----
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        const bool has = i < kp.n_labels;
        const bool ok = has && i != kp.end_label;
        LabelProps<R> t;
        make_props<R>(t, (ok && PROPS == PMO_PROPS_LABEL) ? kp.ma[i] : 0.f,
                      (ok && PROPS == PMO_PROPS_LABEL) ? kp.ms[i] : 0.f, ok ? kp.g[i] : 0.f,
                      has ? kp.n[i] : 1.f);
        s_tab[i] = t;
        s_valid[i] = ok ? 1 : 0;
    }
    for (int i = threadIdx.x; i < PMO_LEDGER_N; i += blockDim.x) s_led[i] = 0.0;
    if (GRAD)
        for (int i = threadIdx.x; i < 512; i += blockDim.x) s_gma[i] = 0.0;
    if (fd)
        for (int i = threadIdx.x; i < 2 * PMO_FD_MAX; i += blockDim.x) s_fdsum[i] = 0.0;
    for (int i = threadIdx.x; i < PMO_COUNTERS_N; i += blockDim.x) s_cnt[i] = 0ull;
    for (int i = threadIdx.x; i < kp.hist_n; i += blockDim.x) s_rr[i] = R(0);
    for (int i = threadIdx.x; i < n_win; i += blockDim.x) s_win[i] = 0ull;
    __syncthreads();

    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const R l = (R)kp.l;
    const R hl = (R)kp.hl;
    const R inv_l = (R)kp.inv_l;
    const uint32_t cap = kp.max_events ? kp.max_events : (1u << 26);
    const uint64_t N = kp.count;
    const bool export_exits = (kp.flags & PMO_FLAG_EXPORT_EXITS) != 0;
    const bool photon_stats = (kp.flags & PMO_FLAG_PHOTON_STATS) != 0;
    const bool score_record = !GRAD && (kp.flags & PMO_FLAG_SCORE_RECORD) != 0;


    // photon state (registers).  The photon sits in a label-uniform box
    // {|dx|, |dy| <= bl, |dz| <= bz} (voxels) around voxel (ix, iy, iz) with
    // linear index lin; (px, py, pz) is its offset from that voxel's centre,
    // hwl and hwz the box's lateral and z half-widths.  bl == bz == 0 is the
    // reference's voxel-by-voxel stepping.
    uint64_t pid = 0;
    int ix = 0, iy = 0, iz = 0, lab = 0, bz = 0, bl = 0;
    uint32_t lin = 0;
    R px = 0, py = 0, pz = 0, vx = 0, vy = 0, vz = 0, ivx = 0, ivy = 0, ivz = 0, w = 0;
    R hwl = 0, hwz = 0;
    // weight at the start of the current absorption segment (photon start or
    // the last roulette gain): the segment's absorbed weight is wseg - w, the
    // exact sum of its implicit-capture decrements (each a difference of two
    // floats, exact in double, telescoping)
    R wseg = 0;
    R mt = 0, imt = 0, ma_mt = 0;   // of label lab; its index n is s_tab[lab].n
    uint32_t k = 0, f = 0, ncr = 0;
    // the current interaction's draws, kept while its step crosses faces;
    // ry is the step's spare uniform (see cycle) and ry_free says it is unused
    uint32_t ry = 0, rz = 0, rw = 0;
    R st = 0;
    bool pending = false, ry_free = false;
    // gradient replay: q of the photon, path length and sum of 1/mu_s over
    // interactions in the current cell, 1/mu_s of the cell
    float gq = 0.f, gL = 0.f, gN = 0.f, gC = 0.f;
    R ims = 0;
    uint32_t pend_lin = 0xffffffffu;
    unsigned long long pend_q = 0;   // fixed-point deposit not yet written

    auto deposit_flush = [&]() {
        if (pend_q != 0ull) atomicAdd(kp.absorbed + pend_lin, pend_q);
        pend_q = 0ull;
        pend_lin = 0xffffffffu;
    };
    // offset of the voxel holding the photon from the box centre along an
    // axis of half-extent m, in voxels
    auto box_k = [&](R q, int m) -> int {
        int k = (int)rint(xmul(q, inv_l));
        return k < -m ? -m : (k > m ? m : k);
    };
    auto set_box = [&](uint32_t word) {
        box_extents(word, bz, bl);
        hwz = xfma((R)bz, l, hl);
        hwl = xfma((R)bl, l, hl);
    };
    auto deposit = [&](R dw) {
        const unsigned long long q = to_fixed(dw);
        int cx = ix, cy = iy, cz = iz;
        uint32_t clin = lin;
        if (SKIP && bl > 0) {
            const int kx = box_k(px, bl), ky = box_k(py, bl), kz = box_k(pz, bz);
            // a map from pmo_build_voxel_words keeps every box inside the
            // array; a caller-supplied map that does not loses the deposit
            // to the box centre instead of writing outside the grid
            if ((unsigned)(cx + kx) < (unsigned)kp.nx && (unsigned)(cy + ky) < (unsigned)kp.ny &&
                (unsigned)(cz + kz) < (unsigned)kp.nz) {
                cx += kx;
                cy += ky;
                cz += kz;
                clin += (uint32_t)kx * kp.sx + (uint32_t)ky * kp.sy + (uint32_t)kz;
            }
        }
        if (FLU == PMO_FLU_SHARED) {
            const unsigned wx = (unsigned)(cx - kp.win_lo[0]);
            const unsigned wy = (unsigned)(cy - kp.win_lo[1]);
            const unsigned wz = (unsigned)(cz - kp.win_lo[2]);
            if (wx < (unsigned)kp.win_dim[0] && wy < (unsigned)kp.win_dim[1] &&
                wz < (unsigned)kp.win_dim[2]) {
                atomicAdd(s_win + ((wx * kp.win_dim[1] + wy) * kp.win_dim[2] + wz), q);
                return;
            }
        }
        if (clin == pend_lin) {
            pend_q += q;
        } else {
            deposit_flush();
            pend_lin = clin;
            pend_q = q;
        }
    };
    // The FP64 build keeps 1/v per direction, as the CPU oracle does; the FP32
    // product divides in place (a * rcp(v), the same value as a * (1/v) with
    // the approximate divide) and keeps three registers free.
    constexpr bool kInv = sizeof(R) != sizeof(float);
    auto set_dir_inverse = [&]() {
        if (!kInv) return;
        ivx = xdiv(R(1), vx);
        ivy = xdiv(R(1), vy);
        ivz = xdiv(R(1), vz);
    };
    auto load_props = [&]() {
        if (PROPS == PMO_PROPS_VOXEL) {
            const float a = __ldg(kp.vox_ma + lin), s = __ldg(kp.vox_ms + lin);
            mt = xadd((R)a, (R)s);
            imt = mt > R(0) ? xdiv(R(1), mt) : R(0);
            ma_mt = mt > R(0) ? xdiv((R)a, mt) : R(0);
            if (GRAD) ims = s > 0.f ? xdiv(R(1), (R)s) : R(0);
        } else {
            mt = s_tab[lab].mt;
            imt = s_tab[lab].imt;
            ma_mt = s_tab[lab].ma_mt;
            if (GRAD) ims = s_tab[lab].ims;
        }
    };
    // gradient replay: hand the current cell's path length and 1/mu_s sum to
    // the per-voxel grids and the per-label sums
    auto grad_flush = [&]() {
        if (GRAD && fd && (gL != 0.f || gC != 0.f)) {
            const int t = __ldg(kp.fd_target + lin);
            if (t >= 0 && t < kp.fd_n) {
                const float mu_a = (float)xmul(ma_mt, mt);
                const float mu = kp.fd_param == 0 ? mu_a : (float)mt - mu_a;
                s_fdL[t] += mu * gL;
                s_fdN[t] += gC;
            }
            gC = 0.f;
        }
        if (GRAD && (gL != 0.f || gN != 0.f)) {
            const float dma = -gq * gL;
            const float dms = gq * gN - gq * gL;
            if (kp.d_ma_voxel) {
                atomicAdd(kp.d_ma_voxel + lin, dma);
                atomicAdd(kp.d_ms_voxel + lin, dms);
            }
            if (kp.d_ma_label) {
                atomicAdd(s_gma + lab, (double)dma);
                atomicAdd(s_gms + lab, (double)dms);
            }
            gL = 0.f;
            gN = 0.f;
        }
    };
    // photon end: per-photon outputs and counters
    // code: the exit's R(r) bin code (category * nr + bin), -1 for none
    auto finish = [&](int code = -1) {
        atomicAdd(s_led + PMO_L_ABS, (double)wseg - (double)w);
        wseg = w;
        if (FLU != PMO_FLU_NONE) deposit_flush();
        // a replayed photon that ends without a binned exit left the forward path
        if (GRAD && code < 0) atomicAdd(kp.gcounters + PMO_G_MISMATCH, 1ull);
        const uint64_t j = pid - kp.begin;
        if (export_exits) {
            kp.exit_add[j] = ix;
            kp.exit_add[N + j] = iy;
            kp.exit_add[2 * N + j] = iz;
            kp.exit_p[j] = (float)px;
            kp.exit_p[N + j] = (float)py;
            kp.exit_p[2 * N + j] = (float)pz;
            kp.exit_v[j] = (float)vx;
            kp.exit_v[N + j] = (float)vy;
            kp.exit_v[2 * N + j] = (float)vz;
            kp.exit_w[j] = (float)w;
        }
        if (score_record) {
            kp.score_bin[j] = code;
            kp.score_w[j] = (float)w;
        }
        if (photon_stats) {
            kp.ph_interact[j] = k;
            kp.ph_cross[j] = ncr;
            kp.ph_fresnel[j] = f;
        }
        atomicAdd(s_cnt + PMO_C_INTERACT, (unsigned long long)k);
        atomicAdd(s_cnt + PMO_C_CROSS, (unsigned long long)ncr);
        if (f) atomicAdd(s_cnt + PMO_C_FRESNEL, (unsigned long long)f);
        atomicAdd(s_cnt + PMO_C_PHOTONS, 1ull);
    };
    auto fail = [&](int counter) {
        atomicAdd(s_led + PMO_L_ERRW, (double)w);
        atomicAdd(s_cnt + counter, 1ull);
        finish();
    };
    // exit into the end label: reference Rd/Tt split by the sign of v_z
    // (pymopt/voxel_gpu/_classes.py:326-334) and radialDistance binning of the
    // encoded exit position (:302-310, pymopt/metrics/_scoring.py:16-25)
    auto exit_tally = [&](int ax) -> int {
        int ecode = -1;
        const double wd = (double)w;
        if (!GRAD)
            atomicAdd(s_led + (vz < R(0) ? PMO_L_RD : (vz > R(0) ? PMO_L_TT : PMO_L_EXIT0)), wd);
        int cat = -1;
        if (ax == 2) {
            cat = vz < R(0) ? PMO_RR_TOP : PMO_RR_BOTTOM;
            if (!GRAD) atomicAdd(s_led + (vz < R(0) ? PMO_L_RD_TOP : PMO_L_TT_BOTTOM), wd);
        } else if (vz < R(0)) {
            cat = PMO_RR_LAT_NEG;
        } else if (vz > R(0)) {
            cat = PMO_RR_LAT_POS;
        }
        if (cat >= 0 && kp.nr > 0) {
            const R x = xfma(l, (R)(ix - kp.cx), px);
            const R y = xfma(l, (R)(iy - kp.cy), py);
            const R r = psqrt(xfma(y, y, xmul(x, x)));
            if (r > R(0)) {
                const R q = ceil(xdiv(r, (R)kp.dr));
                if (q >= R(1) && q <= (R)kp.nr) {
                    const int b = (int)q - 1;
                    ecode = cat * kp.nr + b;
                    if (GRAD) {
                    } else if (kp.rr_shared) {
                        atomicAdd(s_rr + cat * kp.nr + b, (R)w);
                    } else {
                        atomicAdd(kp.rr + cat * kp.nr + b, (float)w);
                    }
                }
            }
        }
        if (!GRAD && kp.n_ang > 0 && vz != R(0)) {
            // arccos|v_z| in bins (i da, (i+1) da] (pymopt/metrics/_scoring.py:27-38);
            // a normal exit (angle 0) falls in no bin, as there
            const float at = acosf(fminf(fabsf((float)vz), 1.f));
            if (at > 0.f) {
                const int b = (int)ceilf(at * kp.inv_da) - 1;
                if (b >= 0 && b < kp.n_ang) {
                    const int i = (vz < R(0) ? 0 : kp.n_ang) + b;
                    if (kp.rr_shared) atomicAdd(s_ang + i, (R)w);
                    else atomicAdd(kp.ang + i, (float)w);
                }
            }
        }
        if (!GRAD && kp.n_line > 0 && vx < R(0)) {
            // exit depth profile of photons moving towards -x within
            // |y| < y_range (pymopt/metrics/_scoring.py:40-51), with the
            // model's z encoding rounded to 1e-6 mm
            // (pymopt/voxel_gpu/_classes.py:302-310)
            const double ld = (double)kp.l;
            const double y = ld * (double)(iy - kp.cy) + (double)py;
            if (fabs(y) < (double)kp.line_y) {
                const double z = rint((ld * (double)(iz - 1) + (double)pz + ld / 2) * 1e6) / 1e6;
                if (z > 0.0) {
                    const int b = (int)ceil(z / (double)kp.line_dr) - 1;
                    if (b >= 0 && b < kp.n_line) {
                        if (kp.rr_shared) atomicAdd(s_line + b, (R)w);
                        else atomicAdd(kp.line + b, (float)w);
                    }
                }
            }
        }
        if (GRAD) {
            // the replay must end where the forward run did
            const uint64_t jr = pid - kp.begin;
            if (ecode != kp.score_bin[jr] || (float)w != kp.score_w[jr])
                atomicAdd(kp.gcounters + PMO_G_MISMATCH, 1ull);
            if (fd) {
                // reweight this photon for mu * (1 +- h) in each target it crossed
                const float h = kp.fd_h;
                for (int t = 0; t < kp.fd_n; ++t) {
                    const float A = s_fdL[t], n = s_fdN[t];
                    if (A == 0.f && n == 0.f) continue;
                    float ep, em;
                    if (kp.fd_param == 0) {
                        ep = expm1f(-h * A);
                        em = expm1f(h * A);
                    } else {
                        ep = expm1f(n * log1pf(h) - h * A);
                        em = expm1f(n * log1pf(-h) + h * A);
                    }
                    atomicAdd(s_fdsum + 2 * t, (double)gq * (double)ep);
                    atomicAdd(s_fdsum + 2 * t + 1, (double)gq * (double)em);
                }
            }
        }
        atomicAdd(s_cnt + PMO_C_EXITS, 1ull);
        return ecode;
    };

    // Start photon j: source (pymopt/voxel_gpu/_classes.py:148-254).
    // Returns true when the photon is in flight.
    auto start = [&](uint64_t jj) -> bool {
        pid = kp.begin + jj;
        k = f = ncr = 0;
        pending = false;
        if (GRAD) {
            const int code = kp.score_bin[jj];
            gq = code >= 0 ? __ldg(kp.coef + code) * kp.score_w[jj] : 0.f;
            gL = gN = gC = 0.f;
            if (fd)
                for (int t = 0; t < kp.fd_n; ++t) s_fdL[t] = s_fdN[t] = 0.f;
            if (gq == 0.f) {
                atomicAdd(kp.gcounters + PMO_G_SKIPPED, 1ull);
                return false;
            }
            atomicAdd(kp.gcounters + PMO_G_REPLAYED, 1ull);
        }
        if (kp.source == PMO_SRC_STATE) {
            ix = kp.state_add[jj];
            iy = kp.state_add[N + jj];
            iz = kp.state_add[2 * N + jj];
            px = (R)kp.state_p[jj];
            py = (R)kp.state_p[N + jj];
            pz = (R)kp.state_p[2 * N + jj];
            vx = (R)kp.state_v[jj];
            vy = (R)kp.state_v[N + jj];
            vz = (R)kp.state_v[2 * N + jj];
            w = (R)kp.state_w[jj];
        } else {
            ix = kp.src_ix;
            iy = kp.src_iy;
            iz = kp.src_iz;
            px = (R)kp.src_p[0];
            py = (R)kp.src_p[1];
            pz = (R)kp.src_p[2];
            vx = (R)kp.src_v[0];
            vy = (R)kp.src_v[1];
            vz = (R)kp.src_v[2];
            w = (R)kp.src_w0;
            if (kp.source == PMO_SRC_GAUSSIAN || kp.spec_prob > 0.f) {
                const uint4 rs = philox4x32_10(make_uint4(0u, 2u, (uint32_t)pid, (uint32_t)(pid >> 32)), kp.rk);
                if (kp.source == PMO_SRC_GAUSSIAN) {
                    // x, y ~ N(0, sigma) (gaussianBeam, :267-287) by Box-Muller,
                    // split into the voxel whose centre is nearest and the
                    // offset from that centre, in [-l/2, l/2]: the position
                    // l * (index - centre) + offset is x exactly, as the
                    // reference's split (:242-252) gives it
                    const R u0 = u01<R>(rs.x), u1 = u01<R>(rs.y);
                    const R rad = xmul((R)kp.beam_sigma, psqrt(xmul(R(2), pneglog(u0))));
                    R sn, cs;
                    psincos2pi(u1, &sn, &cs);
                    const R xy[2] = {xmul(rad, cs), xmul(rad, sn)};
#pragma unroll
                    for (int a = 0; a < 2; ++a) {
                        const R fl = floor(xadd(xdiv(xy[a], l), R(0.5)));
                        R off = xfma(-fl, l, xy[a]);
                        if (fabs(off) >= hl) off = copysign(hl, off);
                        if (a == 0) { ix += (int)fl; px = off; }
                        else { iy += (int)fl; py = off; }
                    }
                }
                if (kp.spec_prob > 0.f && u01<R>(rs.z) <= (R)kp.spec_prob) {
                    // specular reflection at the entry (:184-200): recorded
                    // with w = 1 and the mirrored direction
                    vx = (R)kp.spec_v[0];
                    vy = (R)kp.spec_v[1];
                    vz = (R)kp.spec_v[2];
                    w = R(1);
                    wseg = w;
                    atomicAdd(s_led + PMO_L_SPEC, 1.0);
                    if (vz < R(0)) atomicAdd(s_led + PMO_L_RD, 1.0);
                    else if (vz > R(0)) atomicAdd(s_led + PMO_L_TT, 1.0);
                    finish();
                    return false;
                }
            }
        }
        wseg = w;
        atomicAdd(s_led + PMO_L_WINIT, (double)w);
        if ((unsigned)ix >= (unsigned)kp.nx || (unsigned)iy >= (unsigned)kp.ny ||
            (unsigned)iz >= (unsigned)kp.nz) {
            fail(PMO_C_ERR_GEOM);
            return false;
        }
        lin = ((uint32_t)ix * (uint32_t)kp.ny + (uint32_t)iy) * (uint32_t)kp.nz + (uint32_t)iz;
        if (SKIP) {
            const uint32_t word = __ldg(kp.words + lin);
            lab = (int)(word & 0xffu);
            set_box(word);
        } else {
            lab = __ldg(kp.labels + lin);
            bz = bl = 0;
            hwz = hwl = hl;
        }
        if (!s_valid[lab]) {
            fail(PMO_C_ERR_LABEL);
            return false;
        }
        load_props();
        set_dir_inverse();
        return true;
    };

    // One interaction cycle of the photon in flight: draw a step, cross voxel
    // faces until the step is spent, then absorb, roulette and scatter.
    // Returns true while the photon stays in flight.
    // act: the warp's lanes with a photon in flight (all of them call cycle).
    // Box stepping batches crossings and yields after one; voxel stepping,
    // whose crossings are frequent, does neither (measured: each costs it
    // 3-16 %).
    constexpr int kBatch = SKIP ? kCrossBatch : 1;
    constexpr bool kYield = SKIP;
    auto cycle = [&](unsigned act) -> bool {
        if (!pending) {
            const uint4 rn =
                philox4x32_10(make_uint4(k, 0u, (uint32_t)pid, (uint32_t)(pid >> 32)), kp.rk);
            ++k;
            st = pneglog(u01<R>(rn.x));  // step in optical depths (:75)
            ry = rn.y;
            rz = rn.z;
            rw = rn.w;
            ry_free = true;
            pending = true;
        }
        int budget = kCrossPerIter;
        bool first = true;
        for (;;) {
            // distance to the nearest face; db starts at 1000 (:80-90)
            const R ax_ = xsub(copysign(hwl, vx), px);
            const R ay_ = xsub(copysign(hwl, vy), py);
            const R az_ = xsub(copysign(hwz, vz), pz);
            const R dx = kInv ? xmul(ax_, ivx) : xdiv(ax_, vx);
            const R dy = kInv ? xmul(ay_, ivy) : xdiv(ay_, vy);
            const R dz = kInv ? xmul(az_, ivz) : xdiv(az_, vz);
            // min without the axis (a NaN distance, 0/0 on a face the photon
            // runs along, is skipped as by the reference's comparisons); the
            // axis is only needed for a crossing and is found there
            const R db = fmin(fmin(fmin(R(1000), dx), dy), dz);
            const R dbmt = xmul(db, mt);
            const bool hop = !(st >= dbmt);
            if (kBatch > 1 && first) {
                first = false;
                const unsigned xm = __ballot_sync(act, !hop);
                const int nx = __popc(xm), na = __popc(act);
                const bool go = nx >= kCrossBatch || 4 * nx >= na || nx == na;
                if (!hop && !go) return true;   // wait; the draws and st are kept
            }
            if (hop) {
                // hop inside the voxel or box (:170-175)
                const R s = xmul(st, imt);
                px = xfma(vx, s, px);
                py = xfma(vy, s, py);
                pz = xfma(vz, s, pz);
                if (GRAD) gL += (float)s;
                break;
            }
            if (budget == 0) return true;  // yield; this crossing comes next pass
            --budget;
            // the first axis at the minimum, the reference's strict-less scan
            // from x to z (a tie goes to the lower axis)
            const int ax = dx == db ? 0 : (dy == db ? 1 : (dz == db ? 2 : 0));
            // move to the face and snap (:92-96)
            px = xfma(vx, db, px);
            py = xfma(vy, db, py);
            pz = xfma(vz, db, pz);
            if (GRAD) gL += (float)db;
            const R va = ax == 0 ? vx : (ax == 1 ? vy : vz);
            const R face = copysign(ax == 2 ? hwz : hwl, va);
            if (ax == 0) px = face;
            else if (ax == 1) py = face;
            else pz = face;
            st = xsub(st, dbmt);
            ++ncr;
            if (ncr + k - 1 > cap) { fail(PMO_C_ERR_CAP); return false; }
            const bool neg = signbit(va);
            // the voxel of the box that touches this face, and the photon's
            // offset inside it (for a one-voxel box: the box itself)
            int cx = ix, cy = iy, cz = iz;
            uint32_t clin = lin;
            R fx = px, fy = py, fz = pz;
            if (SKIP && bl > 0) {
                const int ma = ax == 2 ? bz : bl;
                const int m = neg ? -ma : ma;
                const int kx = ax == 0 ? m : box_k(px, bl);
                const int ky = ax == 1 ? m : box_k(py, bl);
                const int kz = ax == 2 ? m : box_k(pz, bz);
                fx = ax == 0 ? copysign(hl, va) : xfma(-(R)kx, l, px);
                fy = ax == 1 ? copysign(hl, va) : xfma(-(R)ky, l, py);
                fz = ax == 2 ? copysign(hl, va) : xfma(-(R)kz, l, pz);
                cx += kx;
                cy += ky;
                cz += kz;
                clin += (uint32_t)kx * kp.sx + (uint32_t)ky * kp.sy + (uint32_t)kz;
                if ((unsigned)cx >= (unsigned)kp.nx || (unsigned)cy >= (unsigned)kp.ny ||
                    (unsigned)cz >= (unsigned)kp.nz) {
                    fail(PMO_C_ERR_GEOM);  // only a malformed caller-supplied map
                    return false;
                }
            }
            const int cc = ax == 0 ? cx : (ax == 1 ? cy : cz);
            const int dim = ax == 0 ? kp.nx : (ax == 1 ? kp.ny : kp.nz);
            const int nc = neg ? cc - 1 : cc + 1;
            if ((unsigned)nc >= (unsigned)dim) { fail(PMO_C_ERR_GEOM); return false; }
            const uint32_t stride = ax == 0 ? kp.sx : (ax == 1 ? kp.sy : 1u);
            const uint32_t nlin = neg ? clin - stride : clin + stride;
            int nlab;
            uint32_t nword = 0;
            if (SKIP) {
                nword = __ldg(kp.words + nlin);
                nlab = (int)(nword & 0xffu);
            } else {
                nlab = __ldg(kp.labels + nlin);
            }
            // step into the neighbour voxel and take its box (:137-148)
            auto enter = [&]() {
                grad_flush();
                ix = ax == 0 ? nc : cx;
                iy = ax == 1 ? nc : cy;
                iz = ax == 2 ? nc : cz;
                px = ax == 0 ? -fx : fx;
                py = ax == 1 ? -fy : fy;
                pz = ax == 2 ? -fz : fz;
                lin = nlin;
                if (SKIP) set_box(nword);
            };
            if (PROPS == PMO_PROPS_LABEL && nlab == lab) {
                // same label on the other side: same n and mu (:154-167)
                enter();
                if (kYield) return true;   // the step goes on next pass
                continue;
            }
            if (nlab != kp.end_label && !s_valid[nlab]) { fail(PMO_C_ERR_LABEL); return false; }
            const R nt = s_tab[nlab].n;
            const R ni = s_tab[lab].n;
            if (ni != nt) {
                // Fresnel / total internal reflection (:105-153) with the
                // cosines and sines of the incidence/transmission angles
                R ca = fabs(va);
                if (ca > R(1)) ca = R(1);
                const R nr = xdiv(ni, nt);
                const R sa = psqrt(xfma(-ca, ca, R(1)));
                const R sb = xmul(nr, sa);
                R ra, cb = R(1);
                if (ni > nt && sb >= R(1)) {
                    ra = R(1);  // TIR
                } else {
                    cb = psqrt(xfma(-sb, sb, R(1)));
                    if (ca == R(1)) {
                        ra = R(0);  // ai == 0 (:113-120)
                    } else {
                        const R cacb = xmul(ca, cb), sasb = xmul(sa, sb);
                        const R sacb = xmul(sa, cb), casb = xmul(ca, sb);
                        const R cap_ = xsub(cacb, sasb);   // cos(ai + at)
                        const R cam = xadd(cacb, sasb);    // cos(ai - at)
                        const R sap = xadd(sacb, casb);    // sin(ai + at)
                        const R sam = xsub(sacb, casb);    // sin(ai - at)
                        const R num = xmul(xmul(xmul(R(0.5), sam), sam),
                                           xfma(cap_, cap_, xmul(cam, cam)));
                        const R den = xmul(xmul(xmul(sap, sap), cam), cam);
                        ra = xdiv(num, den);
                    }
                }
                // transmit when ra < u for a uniform u in (0, 1] (:150).  Only
                // 0 < ra < 1 needs u: ra == 0 always transmits; ra >= 1 (total
                // internal reflection) or a NaN always reflects.  u is the
                // step's spare word ry when no earlier decision of this step
                // took it, else the draw (f, 1, photon) of this decision.
                bool reflect;
                if (ra > R(0) && ra < R(1)) {
                    uint32_t word = ry;
                    if (!ry_free) {
                        word = philox4x32_10(make_uint4(f, 1u, (uint32_t)pid, (uint32_t)(pid >> 32)),
                                             kp.rk).x;
                        atomicAdd(s_cnt + PMO_C_XDRAWS, 1ull);
                    }
                    ry_free = false;
                    reflect = !(ra < u01<R>(word));
                } else {
                    reflect = !(ra <= R(0));
                }
                ++f;
                if (reflect) {
                    // reflect: stay at the face with v_axis mirrored (:150-152)
                    if (ax == 0) { vx = -vx; ivx = -ivx; }
                    else if (ax == 1) { vy = -vy; ivy = -ivy; }
                    else { vz = -vz; ivz = -ivz; }
                    atomicAdd(s_cnt + PMO_C_REFLECT, 1ull);
                    if (kYield) return true;
                    continue;
                }
                // refract: tangential * ni/nt, normal = sign * cos(at) (:124-134)
                vx = ax == 0 ? xmul(sgn(vx), cb) : xmul(vx, nr);
                vy = ax == 1 ? xmul(sgn(vy), cb) : xmul(vy, nr);
                vz = ax == 2 ? xmul(sgn(vz), cb) : xmul(vz, nr);
                const R inv = pinvnorm(sumsq(vx, vy, vz));
                vx = xmul(vx, inv);
                vy = xmul(vy, inv);
                vz = xmul(vz, inv);
                set_dir_inverse();
            }
            // cross (:137-148)
            enter();
            lab = nlab;
            if (lab == kp.end_label) {
                finish(exit_tally(ax));
                return false;
            }
            load_props();
            if (kYield) return true;
        }

        pending = false;
        if (GRAD) {
            gN += (float)ims;
            gC += 1.f;
        }
        // absorption by implicit capture (:179)
        {
            const R wn = xfma(-w, ma_mt, w);
            if (FLU != PMO_FLU_NONE) deposit(xsub(w, wn));
            w = wn;
        }
        // Russian roulette (:182-195): its uniform is the step's spare word,
        // or the draw (k - 1, 3, photon) when a Fresnel decision took it
        if (w <= R(0.0001)) {
            atomicAdd(s_cnt + PMO_C_ROULETTE, 1ull);
            atomicAdd(s_led + PMO_L_ABS, (double)wseg - (double)w);
            uint32_t word = ry;
            if (!ry_free) {
                word = philox4x32_10(make_uint4(k - 1u, 3u, (uint32_t)pid, (uint32_t)(pid >> 32)),
                                     kp.rk).x;
                atomicAdd(s_cnt + PMO_C_XDRAWS, 1ull);
            }
            if (R(0.1) < u01<R>(word)) {
                atomicAdd(s_led + PMO_L_RLOSS, (double)w);
                w = wseg = R(0);
                px = py = pz = R(0);
                vx = vy = vz = R(0);
                ix = iy = iz = 0;
                finish();
                return false;
            }
            const R wn = xmul(w, R(10));
            atomicAdd(s_led + PMO_L_RGAIN, (double)wn - (double)w);
            w = wseg = wn;
        }
        // scattering: HG polar angle, uniform azimuth, rotation (:197-219)
        {
            const R ct = hg_cos<R>(s_tab[lab], u01<R>(rz));
            const R s2 = xfma(-ct, ct, R(1));
            const R sth = psqrt(s2 > R(0) ? s2 : R(0));
            R sf, cf;
            psincos2pi(u01<R>(rw), &sf, &cf);
            if (R(0.99999) < fabs(vz)) {
                const R sz = sgn(vz);
                vx = xmul(sth, cf);
                vy = xmul(sth, sf);
                vz = xmul(sz, ct);
            } else {
                const R tmp = psqrt(xfma(-vz, vz, R(1)));
                const R fct = xdiv(sth, tmp);
                const R ox = vx, oy = vy, oz = vz;
                const R tx = xsub(xmul(xmul(ox, oz), cf), xmul(oy, sf));
                const R ty = xadd(xmul(xmul(oy, oz), cf), xmul(ox, sf));
                vx = xfma(fct, tx, xmul(ox, ct));
                vy = xfma(fct, ty, xmul(oy, ct));
                vz = xfma(xmul(-sth, cf), tmp, xmul(oz, ct));
            }
            const R inv = pinvnorm(sumsq(vx, vy, vz));
            vx = xmul(vx, inv);
            vy = xmul(vy, inv);
            vz = xmul(vz, inv);
            set_dir_inverse();
        }
        if (ncr + k > cap) { fail(PMO_C_ERR_CAP); return false; }
        return true;
    };

    // ---- persistent photon loop: warp-uniform chunked feed ----
    unsigned long long f_next = 0, f_end = 0;
    bool active = false, more = true;
    for (;;) {
        unsigned need = __ballot_sync(FULL, (!active) && more);
        while (need) {
            if (f_next >= f_end) {
                unsigned long long b = 0;
                if (lane == 0) b = atomicAdd(kp.work, (unsigned long long)kChunk);
                b = __shfl_sync(FULL, b, 0);
                if (b >= N) {
                    if ((need >> lane) & 1u) more = false;
                    f_next = f_end = N;
                    need = 0;
                    break;
                }
                f_next = b;
                f_end = b + kChunk < N ? b + kChunk : N;
            }
            const unsigned long long avail = f_end - f_next;
            const unsigned rank = __popc(need & ((1u << lane) - 1u));
            const bool mine = ((need >> lane) & 1u) && (unsigned long long)rank < avail;
            const unsigned taken = __ballot_sync(FULL, mine);
            if (mine) active = start(f_next + rank);
            f_next += __popc(taken);
            need &= ~taken;
        }
        if (!__any_sync(FULL, active || more)) break;
        const unsigned act = __ballot_sync(FULL, active);
        if (active) active = cycle(act);
    }

    // ---- block epilogue: flush the privatised tallies ----
    __syncthreads();
    for (int i = threadIdx.x; i < PMO_LEDGER_N; i += blockDim.x)
        if (s_led[i] != 0.0) atomicAdd(kp.ledger + i, s_led[i]);
    for (int i = threadIdx.x; i < PMO_COUNTERS_N; i += blockDim.x)
        if (s_cnt[i] != 0ull) atomicAdd(kp.counters + i, s_cnt[i]);
    if (kp.rr_shared) {
        const int n_rr = PMO_RR_CATS * kp.nr, n_ang2 = 2 * kp.n_ang;
        for (int i = threadIdx.x; i < kp.hist_n; i += blockDim.x) {
            if (s_rr[i] == R(0)) continue;
            float *dst = i < n_rr ? kp.rr + i
                                  : (i < n_rr + n_ang2 ? kp.ang + (i - n_rr)
                                                       : kp.line + (i - n_rr - n_ang2));
            atomicAdd(dst, (float)s_rr[i]);
        }
    }
    if (fd)
        for (int i = threadIdx.x; i < 2 * kp.fd_n; i += blockDim.x)
            if (s_fdsum[i] != 0.0) atomicAdd(kp.fd_out + i, s_fdsum[i]);
    if (GRAD) {
        for (int i = threadIdx.x; i < kp.n_labels; i += blockDim.x) {
            if (kp.d_ma_label && s_gma[i] != 0.0) atomicAdd(kp.d_ma_label + i, s_gma[i]);
            if (kp.d_ms_label && s_gms[i] != 0.0) atomicAdd(kp.d_ms_label + i, s_gms[i]);
        }
    }
    if (FLU == PMO_FLU_SHARED) {
        const int wy = kp.win_dim[1], wz = kp.win_dim[2];
        for (int i = threadIdx.x; i < n_win; i += blockDim.x) {
            if (s_win[i] != 0ull) {
                const int a = i / (wy * wz), b = (i / wz) % wy, c = i % wz;
                const uint32_t g = ((uint32_t)(kp.win_lo[0] + a) * (uint32_t)kp.ny +
                                    (uint32_t)(kp.win_lo[1] + b)) * (uint32_t)kp.nz +
                                   (uint32_t)(kp.win_lo[2] + c);
                atomicAdd(kp.absorbed + g, s_win[i]);
            }
        }
    }
}

}  // namespace pmo
