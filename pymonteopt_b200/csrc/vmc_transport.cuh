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
// the absorbed-weight grid gets fp32 atomics, merged in registers while a
// photon stays in one voxel and optionally privatised in a shared window.
#pragma once
#include <cstdint>

#include "philox.cuh"
#include "pmo_internal.h"

namespace pmo {

template <typename R>
struct __align__(16) LabelProps {
    R mt, imt, ma_mt, n;       // mu_t, 1/mu_t, mu_a/mu_t, refractive index
    R hgA, hgB, hgC, hgE;      // 1+g^2, 1-g^2, 1-g, 1/(2g) (0 when g == 0)
    R hgD, pad0, pad1, pad2;   // 2g
};

// ---- arithmetic helpers: fast single-precision forms for the product,
// IEEE double forms for the FP64 build (its translation unit also disables
// FMA contraction so that it rounds like the CPU oracle).
__device__ __forceinline__ float plog(float x) { return __logf(x); }
__device__ __forceinline__ double plog(double x) { return log(x); }
__device__ __forceinline__ float psqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double psqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float pinvnorm(float s) { return rsqrtf(s); }
__device__ __forceinline__ double pinvnorm(double s) { return 1.0 / sqrt(s); }
// sin and cos of 2*pi*u for u in (0, 1]
__device__ __forceinline__ void psincos2pi(float u, float *s, float *c) {
    // 2*pi*(u - 1/2) lies in (-pi, pi], where the hardware sine is accurate;
    // sin(x + pi) = -sin(x), cos(x + pi) = -cos(x).
    float a = 6.28318530717958647692f * (u - 0.5f);
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

template <typename R>
__device__ __forceinline__ void make_props(LabelProps<R> &t, float ma, float ms, float g,
                                           float n) {
    t.mt = (R)ma + (R)ms;
    t.imt = t.mt > R(0) ? R(1) / t.mt : R(0);
    t.ma_mt = t.mt > R(0) ? (R)ma / t.mt : R(0);
    t.n = (R)n;
    R gg = (R)g;
    t.hgA = 1 + gg * gg;
    t.hgB = 1 - gg * gg;
    t.hgC = 1 - gg;
    t.hgD = 2 * gg;
    t.hgE = gg != R(0) ? R(1) / (2 * gg) : R(0);
    t.pad0 = t.pad1 = t.pad2 = R(0);
}

// theta(g, rand) of the reference (pymopt/voxel_gpu/_cukernel.py:14-25)
template <typename R>
__device__ __forceinline__ R hg_cos(const LabelProps<R> &t, R u) {
    if (t.hgE != R(0)) {
        R q = t.hgB / (t.hgC + t.hgD * u);
        R c = (t.hgA - q * q) * t.hgE;
        return c < R(-1) ? R(-1) : c;
    }
    return 2 * u - 1;
}

// Dynamic shared memory layout of a transport block.
template <typename R>
struct SmemLayout {
    static constexpr size_t tab_bytes = 256 * sizeof(LabelProps<R>);
    static constexpr size_t led_off = tab_bytes;
    static constexpr size_t cnt_off = led_off + PMO_LEDGER_N * sizeof(double);
    static constexpr size_t valid_off = cnt_off + PMO_COUNTERS_N * sizeof(unsigned long long);
    static constexpr size_t rr_off = valid_off + 256;
    __host__ __device__ static size_t win_off(int nr, int rr_shared) {
        size_t o = rr_off + (rr_shared ? (size_t)PMO_RR_CATS * nr * sizeof(R) : 0);
        return (o + 15) & ~size_t(15);
    }
    __host__ __device__ static size_t total(int nr, int rr_shared, int flu, const int32_t win_dim[3]) {
        size_t o = win_off(nr, rr_shared);
        if (flu == PMO_FLU_SHARED) o += (size_t)win_dim[0] * win_dim[1] * win_dim[2] * sizeof(float);
        return o;
    }
};

enum : int { kChunk = 64 };

template <typename R, int PROPS, int FLU, bool SKIP>
__global__ void __launch_bounds__(512) vmc_plain_kernel(const KParams kp) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using L = SmemLayout<R>;
    LabelProps<R> *s_tab = reinterpret_cast<LabelProps<R> *>(smem_raw);
    double *s_led = reinterpret_cast<double *>(smem_raw + L::led_off);
    unsigned long long *s_cnt = reinterpret_cast<unsigned long long *>(smem_raw + L::cnt_off);
    uint8_t *s_valid = smem_raw + L::valid_off;
    R *s_rr = reinterpret_cast<R *>(smem_raw + L::rr_off);
    float *s_win = reinterpret_cast<float *>(smem_raw + L::win_off(kp.nr, kp.rr_shared));
    const int n_win = FLU == PMO_FLU_SHARED ? kp.win_dim[0] * kp.win_dim[1] * kp.win_dim[2] : 0;

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
    for (int i = threadIdx.x; i < PMO_COUNTERS_N; i += blockDim.x) s_cnt[i] = 0ull;
    if (kp.rr_shared)
        for (int i = threadIdx.x; i < PMO_RR_CATS * kp.nr; i += blockDim.x) s_rr[i] = R(0);
    for (int i = threadIdx.x; i < n_win; i += blockDim.x) s_win[i] = 0.f;
    __syncthreads();

    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const uint2 key = make_uint2(kp.key0, kp.key1);
    const R l = (R)kp.l;
    const R hl = (R)kp.hl;
    const R inv_l = (R)kp.inv_l;
    const uint32_t cap = kp.max_events ? kp.max_events : (1u << 26);
    const uint64_t N = kp.count;
    const bool export_exits = (kp.flags & PMO_FLAG_EXPORT_EXITS) != 0;
    const bool photon_stats = (kp.flags & PMO_FLAG_PHOTON_STATS) != 0;

    // thread totals, reduced once at the end
    double t_abs = 0.0;

    // photon state (registers).  The photon sits in a label-uniform box of
    // (2 rad - 1)^3 voxels centred on voxel (ix, iy, iz) with linear index
    // lin; (px, py, pz) is its offset from that voxel's centre and hw the
    // box half-width.  rad == 1 is the reference's voxel-by-voxel stepping.
    uint64_t pid = 0;
    int ix = 0, iy = 0, iz = 0, lab = 0, rad = 1;
    uint32_t lin = 0;
    R px = 0, py = 0, pz = 0, vx = 0, vy = 0, vz = 0, ivx = 0, ivy = 0, ivz = 0, w = 0;
    R hw = 0;
    R mt = 0, imt = 0, ma_mt = 0, ni = 1;
    uint32_t k = 0, f = 0, ncr = 0;
    uint32_t pend_lin = 0xffffffffu;
    float pend_w = 0.f;

    auto deposit_flush = [&]() {
        if (pend_w != 0.f) atomicAdd(kp.absorbed + pend_lin, pend_w);
        pend_w = 0.f;
        pend_lin = 0xffffffffu;
    };
    // offset of the voxel holding the photon from the box centre, in voxels
    auto box_k = [&](R q) -> int {
        const int m = rad - 1;
        int k = (int)rint(q * inv_l);
        return k < -m ? -m : (k > m ? m : k);
    };
    auto deposit = [&](float dw) {
        int cx = ix, cy = iy, cz = iz;
        uint32_t clin = lin;
        if (SKIP && rad > 1) {
            const int kx = box_k(px), ky = box_k(py), kz = box_k(pz);
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
                atomicAdd(s_win + ((wx * kp.win_dim[1] + wy) * kp.win_dim[2] + wz), dw);
                return;
            }
        }
        if (clin == pend_lin) {
            pend_w += dw;
        } else {
            deposit_flush();
            pend_lin = clin;
            pend_w = dw;
        }
    };
    auto set_dir_inverse = [&]() {
        ivx = R(1) / vx;
        ivy = R(1) / vy;
        ivz = R(1) / vz;
    };
    auto load_props = [&]() {
        if (PROPS == PMO_PROPS_VOXEL) {
            const float a = __ldg(kp.vox_ma + lin), s = __ldg(kp.vox_ms + lin);
            mt = (R)a + (R)s;
            imt = mt > R(0) ? R(1) / mt : R(0);
            ma_mt = mt > R(0) ? (R)a / mt : R(0);
        } else {
            mt = s_tab[lab].mt;
            imt = s_tab[lab].imt;
            ma_mt = s_tab[lab].ma_mt;
        }
    };
    // photon end: per-photon outputs and counters
    auto finish = [&]() {
        if (FLU != PMO_FLU_NONE) deposit_flush();
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
    auto exit_tally = [&](int ax) {
        const double wd = (double)w;
        atomicAdd(s_led + (vz < R(0) ? PMO_L_RD : (vz > R(0) ? PMO_L_TT : PMO_L_EXIT0)), wd);
        int cat = -1;
        if (ax == 2) {
            cat = vz < R(0) ? PMO_RR_TOP : PMO_RR_BOTTOM;
            atomicAdd(s_led + (vz < R(0) ? PMO_L_RD_TOP : PMO_L_TT_BOTTOM), wd);
        } else if (vz < R(0)) {
            cat = PMO_RR_LAT_NEG;
        } else if (vz > R(0)) {
            cat = PMO_RR_LAT_POS;
        }
        if (cat >= 0 && kp.nr > 0) {
            const R x = l * (R)(ix - kp.cx) + px;
            const R y = l * (R)(iy - kp.cy) + py;
            const R r = psqrt(x * x + y * y);
            if (r > R(0)) {
                const R q = ceil(r / (R)kp.dr);
                if (q >= R(1) && q <= (R)kp.nr) {
                    const int b = (int)q - 1;
                    if (kp.rr_shared)
                        atomicAdd(s_rr + cat * kp.nr + b, (R)w);
                    else
                        atomicAdd(kp.rr + cat * kp.nr + b, (float)w);
                }
            }
        }
        atomicAdd(s_cnt + PMO_C_EXITS, 1ull);
    };

    // Start photon j: source (pymopt/voxel_gpu/_classes.py:148-254).
    // Returns true when the photon is in flight.
    auto start = [&](uint64_t jj) -> bool {
        pid = kp.begin + jj;
        k = f = ncr = 0;
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
                const uint4 rs = philox4x32_10(make_uint4(0u, 2u, (uint32_t)pid, (uint32_t)(pid >> 32)), key);
                if (kp.source == PMO_SRC_GAUSSIAN) {
                    // x, y ~ N(0, sigma) (gaussianBeam, :267-287) by Box-Muller,
                    // split into voxel index + offset in [-l/2, l/2] (:242-252)
                    const R u0 = u01<R>(rs.x), u1 = u01<R>(rs.y);
                    const R rad = (R)kp.beam_sigma * psqrt(-2 * plog(u0));
                    R sn, cs;
                    psincos2pi(u1, &sn, &cs);
                    const R xy[2] = {rad * cs, rad * sn};
#pragma unroll
                    for (int a = 0; a < 2; ++a) {
                        const R fl = floor(xy[a] / l);
                        R off = xy[a] - (fl + R(0.5)) * l;
                        if (fabs(off) >= hl) off = sgn(off) * hl;
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
                    atomicAdd(s_led + PMO_L_SPEC, 1.0);
                    if (vz < R(0)) atomicAdd(s_led + PMO_L_RD, 1.0);
                    else if (vz > R(0)) atomicAdd(s_led + PMO_L_TT, 1.0);
                    finish();
                    return false;
                }
            }
        }
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
            rad = (int)(word >> 8);
        } else {
            lab = __ldg(kp.labels + lin);
            rad = 1;
        }
        hw = (R)rad * l - hl;
        if (!s_valid[lab]) {
            fail(PMO_C_ERR_LABEL);
            return false;
        }
        load_props();
        ni = s_tab[lab].n;
        set_dir_inverse();
        return true;
    };

    // One interaction cycle of the photon in flight: draw a step, cross voxel
    // faces until the step is spent, then absorb, roulette and scatter.
    // Returns true while the photon stays in flight.
    auto cycle = [&]() -> bool {
        const uint4 rn = philox4x32_10(make_uint4(k, 0u, (uint32_t)pid, (uint32_t)(pid >> 32)), key);
        ++k;
        R st = -plog(u01<R>(rn.x));  // step in optical depths (:75)

        for (;;) {
            // distance to the nearest face; db starts at 1000 (:80-90)
            const R dx = (copysign(hw, vx) - px) * ivx;
            const R dy = (copysign(hw, vy) - py) * ivy;
            const R dz = (copysign(hw, vz) - pz) * ivz;
            R db = R(1000);
            int ax = 0;
            if (dx < db) { db = dx; ax = 0; }
            if (dy < db) { db = dy; ax = 1; }
            if (dz < db) { db = dz; ax = 2; }
            const R dbmt = db * mt;
            if (!(st >= dbmt)) {
                // hop inside the voxel (:170-175)
                const R s = st * imt;
                px += vx * s;
                py += vy * s;
                pz += vz * s;
                break;
            }
            // move to the face and snap (:92-96)
            px += vx * db;
            py += vy * db;
            pz += vz * db;
            const R va = ax == 0 ? vx : (ax == 1 ? vy : vz);
            const R face = copysign(hw, va);
            if (ax == 0) px = face;
            else if (ax == 1) py = face;
            else pz = face;
            st -= dbmt;
            ++ncr;
            if (ncr + k - 1 > cap) { fail(PMO_C_ERR_CAP); return false; }
            const bool neg = signbit(va);
            // the voxel of the box that touches this face, and the photon's
            // offset inside it (for rad == 1: the box itself)
            int cx = ix, cy = iy, cz = iz;
            uint32_t clin = lin;
            R fx = px, fy = py, fz = pz;
            if (SKIP && rad > 1) {
                const int m = neg ? -(rad - 1) : rad - 1;
                const int kx = ax == 0 ? m : box_k(px);
                const int ky = ax == 1 ? m : box_k(py);
                const int kz = ax == 2 ? m : box_k(pz);
                fx = ax == 0 ? copysign(hl, va) : px - (R)kx * l;
                fy = ax == 1 ? copysign(hl, va) : py - (R)ky * l;
                fz = ax == 2 ? copysign(hl, va) : pz - (R)kz * l;
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
            int nlab, nrad = 1;
            if (SKIP) {
                const uint32_t word = __ldg(kp.words + nlin);
                nlab = (int)(word & 0xffu);
                nrad = (int)(word >> 8);
            } else {
                nlab = __ldg(kp.labels + nlin);
            }
            // step into the neighbour voxel and take its box (:137-148)
            auto enter = [&]() {
                ix = ax == 0 ? nc : cx;
                iy = ax == 1 ? nc : cy;
                iz = ax == 2 ? nc : cz;
                px = ax == 0 ? -fx : fx;
                py = ax == 1 ? -fy : fy;
                pz = ax == 2 ? -fz : fz;
                lin = nlin;
                rad = nrad;
                hw = (R)rad * l - hl;
            };
            if (PROPS == PMO_PROPS_LABEL && nlab == lab) {
                // same label on the other side: same n and mu (:154-167)
                enter();
                continue;
            }
            if (nlab != kp.end_label && !s_valid[nlab]) { fail(PMO_C_ERR_LABEL); return false; }
            const R nt = s_tab[nlab].n;
            if (ni != nt) {
                // Fresnel / total internal reflection (:105-153) with the
                // cosines and sines of the incidence/transmission angles
                const uint4 fr = philox4x32_10(make_uint4(f, 1u, (uint32_t)pid, (uint32_t)(pid >> 32)), key);
                ++f;
                const R u = u01<R>(fr.x);
                R ca = fabs(va);
                if (ca > R(1)) ca = R(1);
                const R nr = ni / nt;
                const R sa = psqrt(1 - ca * ca);
                const R sb = nr * sa;
                R ra, cb = R(1);
                if (ni > nt && sb >= R(1)) {
                    ra = R(1);  // TIR
                } else {
                    cb = psqrt(1 - sb * sb);
                    if (ca == R(1)) {
                        ra = R(0);  // ai == 0 (:113-120)
                    } else {
                        const R cap_ = ca * cb - sa * sb;
                        const R cam = ca * cb + sa * sb;
                        const R sap = sa * cb + ca * sb;
                        const R sam = sa * cb - ca * sb;
                        ra = R(0.5) * sam * sam * (cam * cam + cap_ * cap_) / (sap * sap * cam * cam);
                    }
                }
                if (!(ra < u)) {
                    // reflect: stay at the face with v_axis mirrored (:150-152)
                    if (ax == 0) { vx = -vx; ivx = -ivx; }
                    else if (ax == 1) { vy = -vy; ivy = -ivy; }
                    else { vz = -vz; ivz = -ivz; }
                    atomicAdd(s_cnt + PMO_C_REFLECT, 1ull);
                    continue;
                }
                // refract: tangential * ni/nt, normal = sign * cos(at) (:124-134)
                vx = ax == 0 ? sgn(vx) * cb : vx * nr;
                vy = ax == 1 ? sgn(vy) * cb : vy * nr;
                vz = ax == 2 ? sgn(vz) * cb : vz * nr;
                const R inv = pinvnorm(vx * vx + vy * vy + vz * vz);
                vx *= inv;
                vy *= inv;
                vz *= inv;
                set_dir_inverse();
            }
            // cross (:137-148)
            enter();
            lab = nlab;
            ni = nt;
            if (lab == kp.end_label) {
                exit_tally(ax);
                finish();
                return false;
            }
            load_props();
        }

        // absorption by implicit capture (:179)
        {
            const R wn = w - w * ma_mt;
            const double dw = (double)w - (double)wn;
            w = wn;
            t_abs += dw;
            if (FLU != PMO_FLU_NONE) deposit((float)dw);
        }
        // Russian roulette (:182-195)
        if (w <= R(0.0001)) {
            atomicAdd(s_cnt + PMO_C_ROULETTE, 1ull);
            if (R(0.1) < u01<R>(rn.y)) {
                atomicAdd(s_led + PMO_L_RLOSS, (double)w);
                w = R(0);
                px = py = pz = R(0);
                vx = vy = vz = R(0);
                ix = iy = iz = 0;
                finish();
                return false;
            }
            const R wn = w * 10;
            atomicAdd(s_led + PMO_L_RGAIN, (double)wn - (double)w);
            w = wn;
        }
        // scattering: HG polar angle, uniform azimuth, rotation (:197-219)
        {
            const R ct = hg_cos<R>(s_tab[lab], u01<R>(rn.z));
            const R s2 = 1 - ct * ct;
            const R sth = psqrt(s2 > R(0) ? s2 : R(0));
            R sf, cf;
            psincos2pi(u01<R>(rn.w), &sf, &cf);
            if (R(0.99999) < fabs(vz)) {
                const R sz = sgn(vz);
                vx = sth * cf;
                vy = sth * sf;
                vz = sz * ct;
            } else {
                const R tmp = psqrt(1 - vz * vz);
                const R fct = sth / tmp;
                const R ox = vx, oy = vy, oz = vz;
                vx = fct * (ox * oz * cf - oy * sf) + ox * ct;
                vy = fct * (oy * oz * cf + ox * sf) + oy * ct;
                vz = -sth * cf * tmp + oz * ct;
            }
            const R inv = pinvnorm(vx * vx + vy * vy + vz * vz);
            vx *= inv;
            vy *= inv;
            vz *= inv;
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
        if (active) active = cycle();
    }

    // ---- block epilogue: reduce thread totals, flush privatised tallies ----
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        t_abs += __shfl_xor_sync(FULL, t_abs, o);
    }
    if (lane == 0) {
        atomicAdd(s_led + PMO_L_ABS, t_abs);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < PMO_LEDGER_N; i += blockDim.x)
        if (s_led[i] != 0.0) atomicAdd(kp.ledger + i, s_led[i]);
    for (int i = threadIdx.x; i < PMO_COUNTERS_N; i += blockDim.x)
        if (s_cnt[i] != 0ull) atomicAdd(kp.counters + i, s_cnt[i]);
    if (kp.rr_shared)
        for (int i = threadIdx.x; i < PMO_RR_CATS * kp.nr; i += blockDim.x)
            if (s_rr[i] != R(0)) atomicAdd(kp.rr + i, (float)s_rr[i]);
    if (FLU == PMO_FLU_SHARED) {
        const int wy = kp.win_dim[1], wz = kp.win_dim[2];
        for (int i = threadIdx.x; i < n_win; i += blockDim.x) {
            if (s_win[i] != 0.f) {
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
