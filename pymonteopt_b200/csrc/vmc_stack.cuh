// vmc_stack.cuh — many layered slab problems in one persistent launch.
//
// Each problem is a laterally infinite stack of up to PMO_MAX_LAYERS layers:
// the PlateModel geometry of the reference (pymopt/voxel_gpu/_classes.py:
// 396-459) with the lateral size taken to infinity.  Photons enter at the
// origin of the top face and are transported with the reference's
// hop/drop/spin and Fresnel rules (pymopt/voxel_gpu/_cukernel.py:27-227), where
// the only boundaries are the planes between layers and the two outer faces:
// - at an inner plane with equal refractive indices the photon enters the
//   next layer and keeps its remaining optical depth, which the next layer's
//   mu_t then spends (:154-167);
// - at a plane with an index step it is reflected or refracted as at any
//   Fresnel boundary (:105-153), the outer faces against the ambient index;
// - it leaves through the top (Rd, R(r)) or the bottom (Tt).
//
// The work queue, the warp feed and the Philox layout are those of the slab
// kernel (vmc_batched.cuh): problem p draws from stream word 4p + s, so a
// one-layer stack follows the photons of pmo_run_batched exactly.
//
// Forward and gradient in one pass: the perturbation Monte Carlo derivative
// of an exit weight with respect to layer i's optics needs the photon's path
// length L_i and interaction count n_i in that layer: d/dmu_a_i = -w L_i,
// d/dmu_s_i = w (n_i / mu_s_i - L_i).  The current layer's L and n stay in
// registers and go to per-thread shared memory when the photon changes layer.
#pragma once
#include "vmc_batched.cuh"

namespace pmo {

// lanes at a plane that cross together (or fewer, when no lane can interact)
#ifndef PMO_STACK_CROSS_BATCH
#define PMO_STACK_CROSS_BATCH 8
#endif
constexpr int kStackCrossBatch = PMO_STACK_CROSS_BATCH;

struct SParams {
    const pmo_stack *stacks;
    int32_t n_problems;
    const pmo_layer *layers;
    int32_t n_layer_rows;
    const pmo_batch_item *items;
    int32_t n_items;
    uint32_t key0, key1;
    PhiloxKeys rk;
    int32_t nr;
    double *sums;
    float *bins;
    uint32_t *remaining;
    unsigned long long *t_done;
    uint32_t max_events;
    unsigned long long *work;     // [0] next item, [1] launch start time
};

template <typename R>
__global__ void __launch_bounds__(512) vmc_stack_kernel(const SParams sp) {
    extern __shared__ __align__(16) unsigned char smem_stack[];
    // this thread's per-layer path length and interaction count of its photon
    R *accL = reinterpret_cast<R *>(smem_stack) + threadIdx.x * (2 * PMO_MAX_LAYERS);
    R *accN = accL + PMO_MAX_LAYERS;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicMin(sp.work + 1, global_ns());

    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t cap = sp.max_events ? sp.max_events : (1u << 26);

    auto gadd = [&](int pp, int slot, double v) {
        if (v != 0.0) atomicAdd(sp.sums + (size_t)pp * PMO_SS_N + slot, v);
    };
    auto complete = [&](int pp) {
        if (sp.remaining) {
            const uint32_t before = atomicSub(sp.remaining + pp, 1u);
            if (before == 1u && sp.t_done) sp.t_done[pp] = global_ns();
        }
    };

    // photon state; wseg: weight at the start of the absorption segment
    int p = -1;
    uint32_t j = 0, k = 0, f = 0, ncr = 0;
    R x = 0, y = 0, z = 0, vx = 0, vy = 0, vz = 1, w = 0, wseg = 0;
    PhiloxFixed pfix{0u, 0u, 0u};   // the photon's fixed part of its interaction draws
    // the flight in progress: drawn from Philox block k - 1, st optical depth
    // left, ry the block's spare word (free until a Fresnel decision or the
    // roulette takes it).  A flight may span several passes of the feed
    // loop, one plane crossing per pass.
    R st = 0;
    uint32_t ry = 0;
    bool flying = false, ry_free = false;
    // layer state: current layer li of nl (rows l0 + i of the table), its
    // planes z_top < z_bot, its index and optics; Lc, Nc: path length and
    // interactions in the current layer since the photon entered it
    int li = 0, nl = 1;
    uint32_t l0 = 0;
    R z_top = 0, z_bot = 0, ncur = 1, n_amb = 1, dr = 1, Lc = 0, Nc = 0;
    LabelProps<R> hg;

    auto set_layer = [&](int i) {
        const pmo_layer L = sp.layers[l0 + i];
        make_props<R>(hg, L.ma, L.ms, L.g, L.n);
        ncur = (R)L.n;
    };
    auto flush_layer = [&]() {
        accL[li] = xadd(accL[li], Lc);
        accN[li] = xadd(accN[li], Nc);
        Lc = Nc = R(0);
    };
    auto finish = [&]() {
        gadd(p, PMO_SS_ABS, (double)wseg - (double)w);
        gadd(p, PMO_SS_INTER, (double)k);
        complete(p);
    };

    auto start = [&](int pp, uint32_t jj) -> bool {
        p = pp;
        j = jj;
        k = f = ncr = 0;
        pfix = philox_fixed(4u * (uint32_t)pp, jj, sp.rk);
        flying = false;
        const pmo_stack st = sp.stacks[pp];
        l0 = st.first_layer;
        nl = (int)st.n_layers;
        n_amb = (R)st.n_ambient;
        dr = (R)st.dr;
        if (nl < 1 || nl > PMO_MAX_LAYERS || (uint64_t)l0 + (uint64_t)nl > (uint64_t)sp.n_layer_rows) {
            // a malformed stack: its photons count as error weight
            gadd(pp, PMO_SS_WINIT, 1.0);
            gadd(pp, PMO_SS_ERRW, 1.0);
            complete(pp);
            return false;
        }
        li = 0;
        set_layer(0);
        // specular loss at the entry, in single precision as the reference
        // computes it (pymopt/voxel_gpu/_classes.py:204-221)
        const float nt0 = sp.layers[l0].n;
        float rsp = 0.f;
        if (st.n_ambient != nt0) {
            const float q = __fdiv_rn(__fsub_rn(st.n_ambient, nt0), __fadd_rn(st.n_ambient, nt0));
            rsp = __fmul_rn(q, q);
        }
        w = (R)__fsub_rn(1.0f, rsp);
        x = y = z = R(0);
        vx = vy = R(0);
        vz = R(1);
        wseg = w;
        z_top = R(0);
        z_bot = (R)sp.layers[l0].thickness;
        Lc = Nc = R(0);
        for (int i = 0; i < nl; ++i) accL[i] = accN[i] = R(0);
        gadd(p, PMO_SS_WINIT, (double)w);
        return true;
    };

    // the plane ahead in the photon's layer: distance db, optical depth dbmt
    auto plane_ahead = [&](R &db, R &dbmt) {
        const R dzf = vz > R(0) ? xsub(z_bot, z) : (vz < R(0) ? xsub(z_top, z) : R(0));
        db = vz != R(0) ? xdiv(dzf, vz) : R(1e30);
        dbmt = xmul(db, hg.mt);
    };

    // one plane crossing of the flight (st >= dbmt): the photon moves to the
    // plane, then reflects, enters the next layer or leaves; the flight goes
    // on with the optical depth left.  Returns true while the photon is in
    // flight.
    auto cross = [&](R db, R dbmt) -> bool {
        x = xfma(vx, db, x);
        y = xfma(vy, db, y);
        z = vz > R(0) ? z_bot : z_top;
        Lc = xadd(Lc, db);
        st = xsub(st, dbmt);
        ++ncr;
        if (ncr + k - 1 > cap) {
            gadd(p, PMO_SS_ERRW, (double)w);
            finish();
            return false;
        }
        // the layer (or the ambient medium) across the plane
        const int nxt = vz > R(0) ? li + 1 : li - 1;
        const bool out = nxt < 0 || nxt >= nl;
        const R nn = out ? n_amb : (R)sp.layers[l0 + nxt].n;
        bool transmit = true;
        R cb = R(1), nr = R(1);
        if (ncur != nn) {
            // Fresnel / total internal reflection (:105-153)
            const uint32_t fk = f++;   // this decision's Philox counter
            R ca = fabs(vz);
            if (ca > R(1)) ca = R(1);
            nr = xdiv(ncur, nn);
            const R sa = psqrt(xfma(-ca, ca, R(1)));
            const R sb = xmul(nr, sa);
            R ra;
            if (ncur > nn && sb >= R(1)) {
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
            // transmit when ra < u (:150); only 0 < ra < 1 needs u, which
            // is the step's spare word while free, else draw (fk, 1)
            if (ra > R(0) && ra < R(1)) {
                uint32_t word = ry;
                if (!ry_free)
                    word = philox4x32_10(make_uint4(fk, 1u + 4u * (uint32_t)p, j, 0u),
                                         sp.rk).x;
                ry_free = false;
                transmit = ra < u01<R>(word);
            } else {
                transmit = ra <= R(0);
            }
        }
        if (!transmit) {
            vz = -vz;   // reflect and stay in the layer (:150-152)
            return true;
        }
        if (ncur != nn) {
            // refracted direction (:124-134)
            vx = xmul(vx, nr);
            vy = xmul(vy, nr);
            vz = xmul(sgn(vz), cb);
            const R inv = pinvnorm(sumsq(vx, vy, vz));
            vx = xmul(vx, inv);
            vy = xmul(vy, inv);
            vz = xmul(vz, inv);
        }
        flush_layer();
        if (out) {
            // exit: Rd or Tt with the per-layer derivative sums, R(r)
            const double wd = (double)w;
            const bool top = vz < R(0);
            gadd(p, top ? PMO_SS_RD : PMO_SS_TT, wd);
            const int off = top ? 0 : 2;
            for (int i = 0; i < nl; ++i) {
                gadd(p, PMO_SS_LAYER0 + 4 * i + off, wd * (double)accL[i]);
                gadd(p, PMO_SS_LAYER0 + 4 * i + off + 1, wd * (double)accN[i]);
            }
            if (top && sp.nr > 0) {
                const R r = psqrt(xfma(y, y, xmul(x, x)));
                if (r > R(0)) {
                    const R q = ceil(xdiv(r, dr));
                    if (q >= R(1) && q <= (R)sp.nr) {
                        float *b = sp.bins + ((size_t)p * sp.nr + ((int)q - 1)) * PMO_SB_N;
                        atomicAdd(b, (float)wd);
                        for (int i = 0; i < nl; ++i) {
                            const double a = wd * (double)accL[i];
                            const double c = wd * (double)accN[i];
                            if (a != 0.0) atomicAdd(b + 1 + 2 * i, (float)a);
                            if (c != 0.0) atomicAdd(b + 2 + 2 * i, (float)c);
                        }
                    }
                }
            }
            finish();
            return false;
        }
        // enter the next layer; the remaining optical depth carries over
        li = nxt;
        set_layer(li);
        const R t = (R)sp.layers[l0 + li].thickness;
        if (vz > R(0)) {
            z_top = z_bot;
            z_bot = xadd(z_top, t);
        } else {
            z_bot = z_top;
            z_top = xsub(z_bot, t);
        }
        return true;
    };

    // the end of the flight inside the layer: hop, absorption, roulette and
    // spin, the last two from the words rz, rw of the flight's block.
    // Returns true while the photon is in flight.
    auto interact = [&](uint32_t rz, uint32_t rw) -> bool {
        const R s = xmul(st, hg.imt);
        x = xfma(vx, s, x);
        y = xfma(vy, s, y);
        z = xfma(vz, s, z);
        Lc = xadd(Lc, s);
        flying = false;
        Nc = xadd(Nc, R(1));
        // absorption (:179)
        w = xfma(-w, hg.ma_mt, w);
        // roulette (:182-195): the spare word, or draw (k - 1, 3)
        if (w <= R(0.0001)) {
            uint32_t word = ry;
            if (!ry_free)
                word = philox4x32_10(make_uint4(k - 1u, 3u + 4u * (uint32_t)p, j, 0u), sp.rk).x;
            if (R(0.1) < u01<R>(word)) {
                gadd(p, PMO_SS_RLOSS, (double)w);
                finish();
                return false;
            }
            gadd(p, PMO_SS_ABS, (double)wseg - (double)w);
            const R wn = xmul(w, R(10));
            gadd(p, PMO_SS_RGAIN, (double)wn - (double)w);
            w = wseg = wn;
        }
        // spin (:197-219)
        {
            const R ct = hg_cos<R>(hg, u01<R>(rz));
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
        }
        if (ncr + k > cap) {
            gadd(p, PMO_SS_ERRW, (double)w);
            finish();
            return false;
        }
        return true;
    };

    // warp-uniform feed over the work items (as in the slab kernel)
    int item_p = -1;
    uint32_t i_next = 0, i_end = 0;
    bool active = false, more = true;
    for (;;) {
        unsigned need = __ballot_sync(FULL, (!active) && more);
        while (need) {
            if (i_next >= i_end) {
                unsigned long long it = 0;
                if (lane == 0) it = atomicAdd(sp.work, 1ull);
                it = __shfl_sync(FULL, it, 0);
                if (it >= (unsigned long long)sp.n_items) {
                    if ((need >> lane) & 1u) more = false;
                    i_next = i_end = 0;
                    need = 0;
                    break;
                }
                const pmo_batch_item itm = sp.items[it];
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
        // One pass: a lane without a flight draws one (block k, as the slab
        // kernel); then it either ends the flight inside its layer or, at a
        // plane, crosses it.  Lanes at a plane cross together once
        // kStackCrossBatch of them wait, or when no lane can interact; else
        // they wait a pass.  Every lane meets the next pass's ballots, so the
        // warp runs the interaction code whole after any crossing.
        R db = R(0), dbmt = R(0);
        uint4 rn = make_uint4(0u, 0u, 0u, 0u);
        bool fresh = false, at_plane = false;
        if (active) {
            if (!flying) {
                rn = philox4x32_10_fixed(k, 0u, pfix, sp.rk);
                ++k;
                st = pneglog(u01<R>(rn.x));
                ry = rn.y;
                ry_free = true;
                flying = fresh = true;
            }
            plane_ahead(db, dbmt);
            at_plane = st >= dbmt;
        }
        const unsigned waiting = __ballot_sync(FULL, at_plane);
        const bool go = __popc(waiting) >= kStackCrossBatch ||
                        __ballot_sync(FULL, active && !at_plane) == 0u;
        if (active) {
            if (!at_plane) {
                // the block's last two words: in registers when it was drawn
                // this pass, else drawn again (after a crossing or a wait)
                if (!fresh)
                    rn = philox4x32_10_fixed(k - 1u, 0u, pfix, sp.rk);
                active = interact(rn.z, rn.w);
            } else if (go) {
                active = cross(db, dbmt);
            }
        }
    }
}

}  // namespace pmo
