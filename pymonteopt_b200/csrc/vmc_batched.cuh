// vmc_batched.cuh — many independent slab problems in one persistent launch.
//
// Each problem is a laterally infinite single-layer slab (the PlateModel
// geometry of the reference, pymopt/voxel_gpu/_classes.py:396-459, with the
// lateral size taken to infinity): photons enter at the origin of the top
// face, are transported with the reference's hop/drop/spin and Fresnel rules
// (pymopt/voxel_gpu/_cukernel.py:27-227; only the two z faces are boundaries)
// and leave through the top (Rd, R(r)) or bottom (Tt) face.
//
// Work arrives as a queue of (problem, photon range) items.  A warp takes one
// item at a time and its lanes pull photons from it; a lane that finishes a
// photon starts the next at once, whatever problem it belongs to, so the
// launch stays full across thousands of problems with uneven budgets.  Each
// lane keeps the problem parameters of its own photon.  Per-problem sums are
// either privatised per thread in shared memory and flushed when the thread
// moves on to another problem (PMO_BT_THREAD), or added to global memory as
// they occur (PMO_BT_GLOBAL); the batch autotuner times both.  A photon's
// absorbed weight is summed per segment (start or last roulette gain to the
// next roulette or the end) as the weight it lost, so no sum is touched per
// interaction.
//
// Forward and gradient in one pass: with one layer the perturbation Monte
// Carlo derivative of an exit weight needs only the photon's total path
// length L and interaction count n: d/dmu_a = -w L, d/dmu_s = w (n/mu_s - L).
#pragma once
#include "vmc_transport.cuh"

namespace pmo {

struct BParams {
    const pmo_slab *slabs;
    int32_t n_problems;
    const pmo_batch_item *items;
    int32_t n_items;
    uint32_t key0, key1;
    PhiloxKeys rk;                 // round keys of (key0, key1)
    int32_t nr;
    double *sums;
    float *bins;
    uint32_t *remaining;
    unsigned long long *t_done;
    uint32_t max_events;
    int32_t tally_mode;           // PMO_BT_THREAD or PMO_BT_GLOBAL
    unsigned long long *work;     // [0] next item, [1] launch start time
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// per-thread accumulator slots of the problem a thread is working on
enum : int {
    kSlotRd = 0, kSlotRdL, kSlotRdN, kSlotTt, kSlotTtL, kSlotTtN, kSlotAbs, kSlotWinit,
    kSlotGain, kSlotLoss, kSlotErr, kSlotInter, kSlotDone, kSlots
};

template <typename R>
__global__ void __launch_bounds__(512) vmc_batched_kernel(const BParams bp) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const bool priv = bp.tally_mode == PMO_BT_THREAD;
    double *acc = reinterpret_cast<double *>(smem_raw) + threadIdx.x * kSlots;
    if (priv)
        for (int i = 0; i < kSlots; ++i) acc[i] = 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicMin(bp.work + 1, global_ns());

    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t cap = bp.max_events ? bp.max_events : (1u << 26);
    const int map[12] = {PMO_BS_RD, PMO_BS_RD_L, PMO_BS_RD_N, PMO_BS_TT, PMO_BS_TT_L,
                         PMO_BS_TT_N, PMO_BS_ABS, PMO_BS_WINIT, PMO_BS_RGAIN, PMO_BS_RLOSS,
                         PMO_BS_ERRW, PMO_BS_INTER};

    // photons of problem pp ended: count them down, stamp the completion time
    auto complete = [&](int pp, uint32_t done) {
        if (bp.remaining && done) {
            const uint32_t before = atomicSub(bp.remaining + pp, done);
            if (before == done && bp.t_done) bp.t_done[pp] = global_ns();
        }
    };
    int acc_p = -1;  // problem held in acc[]
    auto flush = [&]() {
        if (acc_p < 0) return;
        double *dst = bp.sums + (size_t)acc_p * PMO_BS_N;
#pragma unroll
        for (int i = 0; i < 12; ++i)
            if (acc[i] != 0.0) atomicAdd(dst + map[i], acc[i]);
        complete(acc_p, (uint32_t)acc[kSlotDone]);
        for (int i = 0; i < kSlots; ++i) acc[i] = 0.0;
        acc_p = -1;
    };

    // photon state; wseg: weight at the start of the absorption segment
    int p = -1;
    uint32_t j = 0, k = 0, f = 0, ncr = 0;
    R x = 0, y = 0, z = 0, vx = 0, vy = 0, vz = 1, w = 0, wseg = 0, L = 0;
    PhiloxFixed pfix{0u, 0u, 0u};   // the photon's fixed part of its interaction draws
    // add v to sum `slot` of the photon's problem
    auto add = [&](int slot, double v) {
        if (priv) acc[slot] += v;
        else if (v != 0.0) atomicAdd(bp.sums + (size_t)p * PMO_BS_N + map[slot], v);
    };
    // problem constants of the photon in flight
    R mt = 0, imt = 0, ma_mt = 0, ims = 0, nin = 1, nout = 1, th = 1, dr = 1;
    LabelProps<R> hg;

    auto start = [&](int pp, uint32_t jj) -> bool {
        if (priv && pp != acc_p) {
            flush();
            acc_p = pp;
        }
        p = pp;
        j = jj;
        k = f = ncr = 0;
        pfix = philox_fixed(4u * (uint32_t)pp, jj, bp.rk);
        const pmo_slab sl = bp.slabs[pp];
        make_props<R>(hg, sl.ma, sl.ms, sl.g, sl.n_tissue);
        mt = hg.mt;
        imt = hg.imt;
        ma_mt = hg.ma_mt;
        ims = hg.ims;
        nin = (R)sl.n_tissue;
        nout = (R)sl.n_ambient;
        th = (R)sl.thickness;
        dr = (R)sl.dr;
        // specular loss at the entry, in single precision as the reference
        // computes it (pymopt/voxel_gpu/_classes.py:204-221)
        float rsp = 0.f;
        if (sl.n_ambient != sl.n_tissue) {
            const float q = __fdiv_rn(__fsub_rn(sl.n_ambient, sl.n_tissue),
                                      __fadd_rn(sl.n_ambient, sl.n_tissue));
            rsp = __fmul_rn(q, q);
        }
        w = (R)__fsub_rn(1.0f, rsp);
        x = y = z = R(0);
        vx = vy = R(0);
        vz = R(1);
        wseg = w;
        L = R(0);
        add(kSlotWinit, (double)w);
        return true;
    };
    auto finish = [&]() {
        add(kSlotAbs, (double)wseg - (double)w);
        add(kSlotInter, (double)k);
        if (priv) acc[kSlotDone] += 1.0;
        else complete(p, 1u);
    };

    // one interaction cycle; returns true while the photon is in flight
    auto cycle = [&]() -> bool {
        const uint4 rn = philox4x32_10_fixed(k, 0u, pfix, bp.rk);
        ++k;
        R st = pneglog(u01<R>(rn.x));
        // rn.y is the step's spare uniform: the first Fresnel decision with
        // 0 < ra < 1 or the roulette takes it, as in the plain kernel
        bool ry_free = true;
        for (;;) {
            // distance to the slab face ahead (only z faces bound the slab)
            const R dzf = vz > R(0) ? xsub(th, z) : (vz < R(0) ? -z : R(0));
            const R db = vz != R(0) ? xdiv(dzf, vz) : R(1e30);
            const R dbmt = xmul(db, mt);
            if (!(st >= dbmt)) {
                const R s = xmul(st, imt);
                x = xfma(vx, s, x);
                y = xfma(vy, s, y);
                z = xfma(vz, s, z);
                L = xadd(L, s);
                break;
            }
            x = xfma(vx, db, x);
            y = xfma(vy, db, y);
            z = vz > R(0) ? th : R(0);
            L = xadd(L, db);
            st = xsub(st, dbmt);
            ++ncr;
            if (ncr + k - 1 > cap) {
                add(kSlotErr, (double)w);
                finish();
                return false;
            }
            // Fresnel / total internal reflection at the face (:105-153)
            bool transmit = true;
            R cb = R(1), nr = R(1);
            if (nin != nout) {
                const uint32_t fk = f++;   // this decision's Philox counter
                R ca = fabs(vz);
                if (ca > R(1)) ca = R(1);
                nr = xdiv(nin, nout);
                const R sa = psqrt(xfma(-ca, ca, R(1)));
                const R sb = xmul(nr, sa);
                R ra;
                if (nin > nout && sb >= R(1)) {
                    ra = R(1);
                } else {
                    cb = psqrt(xfma(-sb, sb, R(1)));
                    if (ca == R(1)) {
                        ra = R(0);
                    } else {
                        const R cacb = xmul(ca, cb), sasb = xmul(sa, sb);
                        const R sacb = xmul(sa, cb), casb = xmul(ca, sb);
                        const R cap_ = xsub(cacb, sasb), cam = xadd(cacb, sasb);
                        const R sap = xadd(sacb, casb), sam = xsub(sacb, casb);
                        const R num = xmul(xmul(xmul(R(0.5), sam), sam),
                                           xfma(cap_, cap_, xmul(cam, cam)));
                        const R den = xmul(xmul(xmul(sap, sap), cam), cam);
                        ra = xdiv(num, den);
                    }
                }
                // transmit when ra < u for the uniform u in (0, 1] (:150).
                // Only 0 < ra < 1 needs u: ra == 0 always transmits, and
                // ra >= 1 (total internal reflection, frequent at a slab's
                // faces) or a NaN always reflects, so those take no uniform.
                // u is the step's spare word when it is still free, else the
                // draw (fk, 1, photon) of this decision; the decision counter
                // advances either way.
                if (ra > R(0) && ra < R(1)) {
                    uint32_t word = rn.y;
                    if (!ry_free)
                        word = philox4x32_10(make_uint4(fk, 1u + 4u * (uint32_t)p, j, 0u),
                                             bp.rk).x;
                    ry_free = false;
                    transmit = ra < u01<R>(word);
                } else {
                    transmit = ra <= R(0);
                }
            }
            if (!transmit) {
                vz = -vz;
                continue;
            }
            // leave the slab: refracted direction, exit tallies
            if (nin != nout) {
                vx = xmul(vx, nr);
                vy = xmul(vy, nr);
                vz = xmul(sgn(vz), cb);
                const R inv = pinvnorm(sumsq(vx, vy, vz));
                vx = xmul(vx, inv);
                vy = xmul(vy, inv);
                vz = xmul(vz, inv);
            }
            // interactions so far: every earlier cycle ended in one
            const double wd = (double)w;
            const double wl = wd * (double)L, wn = wd * (double)(k - 1u);
            if (vz < R(0)) {
                add(kSlotRd, wd);
                add(kSlotRdL, wl);
                add(kSlotRdN, wn);
                // R(r) of the exit point around the entry point
                const R r = psqrt(xfma(y, y, xmul(x, x)));
                if (r > R(0) && bp.nr > 0) {
                    const R q = ceil(xdiv(r, dr));
                    if (q >= R(1) && q <= (R)bp.nr) {
                        float *b = bp.bins + ((size_t)p * bp.nr + ((int)q - 1)) * 3;
                        atomicAdd(b, (float)wd);
                        atomicAdd(b + 1, (float)wl);
                        atomicAdd(b + 2, (float)wn);
                    }
                }
            } else {
                add(kSlotTt, wd);
                add(kSlotTtL, wl);
                add(kSlotTtN, wn);
            }
            finish();
            return false;
        }
        // absorption (:179)
        w = xfma(-w, ma_mt, w);
        // roulette (:182-195)
        if (w <= R(0.0001)) {
            uint32_t word = rn.y;
            if (!ry_free)
                word = philox4x32_10(make_uint4(k - 1u, 3u + 4u * (uint32_t)p, j, 0u), bp.rk).x;
            if (R(0.1) < u01<R>(word)) {
                add(kSlotLoss, (double)w);
                finish();
                return false;
            }
            add(kSlotAbs, (double)wseg - (double)w);
            const R wn = xmul(w, R(10));
            add(kSlotGain, (double)wn - (double)w);
            w = wseg = wn;
        }
        // spin (:197-219)
        {
            const R ct = hg_cos<R>(hg, u01<R>(rn.z));
            const R s2 = xfma(-ct, ct, R(1));
            const R sth = psqrt(s2 > R(0) ? s2 : R(0));
            R sf, cf;
            psincos2pi(u01<R>(rn.w), &sf, &cf);
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
        }
        if (ncr + k > cap) {
            add(kSlotErr, (double)w);
            finish();
            return false;
        }
        return true;
    };

    // warp-uniform feed over the work items
    int item_p = -1;
    uint32_t i_next = 0, i_end = 0;
    bool active = false, more = true;
    for (;;) {
        unsigned need = __ballot_sync(FULL, (!active) && more);
        while (need) {
            if (i_next >= i_end) {
                unsigned long long it = 0;
                if (lane == 0) it = atomicAdd(bp.work, 1ull);
                it = __shfl_sync(FULL, it, 0);
                if (it >= (unsigned long long)bp.n_items) {
                    if ((need >> lane) & 1u) more = false;
                    i_next = i_end = 0;
                    need = 0;
                    break;
                }
                const pmo_batch_item itm = bp.items[it];
                item_p = (int)itm.problem;
                i_next = itm.begin;
                i_end = itm.begin + itm.count;
            }
            const uint32_t avail = i_end - i_next;
            const unsigned rank = __popc(need & ((1u << lane) - 1u));
            const bool mine = ((need >> lane) & 1u) && rank < avail;
            const unsigned taken = __ballot_sync(FULL, mine);
            if (mine) active = start(item_p, i_next + rank);
            i_next += __popc(taken);
            need &= ~taken;
        }
        if (!__any_sync(FULL, active || more)) break;
        if (active) active = cycle();
    }
    flush();
}

}  // namespace pmo
