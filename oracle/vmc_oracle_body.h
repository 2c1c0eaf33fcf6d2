/*
 * vmc_oracle_body.h — one photon history, written once and included twice by
 * vmc_oracle.c with REAL = float and REAL = double.
 *
 * TEST INFRASTRUCTURE (oracle).  A CPU restatement of the reference transport
 * kernel cuVMC (pymopt/voxel_gpu/_cukernel.py:27-227) and its Numba twin
 * vmc_kernel (pymopt/voxel/_kernel.py:23-172), with the random numbers taken
 * from the Philox layout of include/pmo_b200.h instead of cuRAND/NumPy.
 * Line references below are to pymopt/voxel_gpu/_cukernel.py unless stated.
 */

#define PFX(name) PMO_CAT(name, SUFFIX)

typedef struct {
    REAL mt, imt, ma_mt, ma, ms, n, g, ims;
    REAL hgA, hgB, hgC, hgD, hgE;
    int valid;
} PFX(props_t);

/* Per-label constants.  mt = ma + ms (:62), HG constants of theta() (:14-25). */
static void PFX(make_props)(PFX(props_t) *t, float ma, float ms, float g, float n,
                            int valid) {
    t->ma = (REAL)ma; t->ms = (REAL)ms; t->g = (REAL)g; t->n = (REAL)n;
    t->mt = (REAL)ma + (REAL)ms;
    t->imt = t->mt > 0 ? (REAL)1 / t->mt : (REAL)0;
    t->ma_mt = t->mt > 0 ? (REAL)ma / t->mt : (REAL)0;
    REAL gg = (REAL)g;
    t->hgA = 1 + gg * gg;
    t->hgB = 1 - gg * gg;
    t->hgC = 1 - gg;
    t->hgD = 2 * gg;
    t->hgE = gg != 0 ? (REAL)1 / (2 * gg) : (REAL)0;
    t->ims = ms > 0 ? (REAL)1 / (REAL)ms : (REAL)0;
    t->valid = valid;
}

/* theta(g, rand) (:14-25): Henyey-Greenstein cos(theta), clamped at -1;
   isotropic 2u-1 when g == 0. */
static inline REAL PFX(hg_cos)(const PFX(props_t) *t, REAL u) {
    if (t->g != 0) {
        REAL q = t->hgB / (t->hgC + t->hgD * u);
        REAL c = (t->hgA - q * q) * t->hgE;
        return c < -1 ? (REAL)-1 : c;
    }
    return 2 * u - 1;
}

static inline REAL PFX(sgn)(REAL x) { return signbit(x) ? (REAL)-1 : (REAL)1; }

/*
 * Trace photon `pid` of problem P.  Tallies go to `acc` (thread-private
 * ledger/counters) and to the shared grids in `tal` (atomically).
 * Returns the photon's status (PMO_OK or an error code).
 */
static int PFX(trace)(const pmo_problem *P, const PFX(props_t) *tab,
                      const oracle_tallies *tal, oracle_acc *acc, uint64_t pid) {
    const REAL l = (REAL)P->voxel_space;
    const REAL hl = l / 2;
    const int64_t sx = (int64_t)P->ny * P->nz, sy = P->nz;
    const uint32_t key[2] = {(uint32_t)P->seed, (uint32_t)(P->seed >> 32)};
    const uint32_t idlo = (uint32_t)pid, idhi = (uint32_t)(pid >> 32);
    const uint64_t j = pid - P->photon_begin;
    const int end = P->end_label;
    const uint32_t cap = P->max_events ? P->max_events : (1u << 26);
    uint32_t rnd[4], ctr[4];

    int c[3];
    REAL p[3], v[3], w;
    int status = PMO_OK;
    uint32_t n_int = 0, n_cross = 0, n_fres = 0, events = 0;
    /* gradient: path length and sum of 1/mu_s in the current voxel */
    const int grad = tal->grad_coef != NULL;
    double gL = 0.0, gN = 0.0;
    acc->nseg = 0;

    /* ---- source (pymopt/voxel_gpu/_classes.py:148-254) ---- */
    ctr[0] = 0; ctr[1] = 2; ctr[2] = idlo; ctr[3] = idhi;
    pmo_philox4x32_10(ctr, key, rnd);
    if (P->source == PMO_SRC_STATE) {
        uint64_t N = P->photon_count;
        for (int a = 0; a < 3; ++a) {
            c[a] = P->state_add[a * N + j];
            p[a] = (REAL)P->state_p[a * N + j];
            v[a] = (REAL)P->state_v[a * N + j];
        }
        w = (REAL)P->state_w[j];
    } else {
        c[0] = P->src_ix; c[1] = P->src_iy; c[2] = P->src_iz;
        for (int a = 0; a < 3; ++a) { p[a] = (REAL)P->src_p[a]; v[a] = (REAL)P->src_v[a]; }
        w = (REAL)P->src_w0;
        if (P->source == PMO_SRC_GAUSSIAN) {
            /* x, y ~ N(0, sigma) (gaussianBeam :267-287) by Box-Muller, split into
               voxel index and an in-voxel offset in [-l/2, l/2] (:242-252). */
            REAL u0 = (REAL)pmo_u01(rnd[0]), u1 = (REAL)pmo_u01(rnd[1]);
            REAL rad = (REAL)P->beam_sigma * SQRT(-2 * LOG(u0));
            REAL xy[2] = {rad * COS(TWO_PI * u1), rad * SIN(TWO_PI * u1)};
            for (int a = 0; a < 2; ++a) {
                REAL f = FLOOR(xy[a] / l + (REAL)0.5);   /* nearest voxel centre */
                REAL off = xy[a] - f * l;
                if (FABS(off) >= hl) off = PFX(sgn)(off) * hl;
                c[a] += (int)f;
                p[a] = off;
            }
        }
        if (P->spec_prob > 0 && (REAL)pmo_u01(rnd[2]) <= (REAL)P->spec_prob) {
            /* Specular reflection at the entry (_set_inital_vector :184-200):
               the photon is recorded with w = 1 and the mirrored direction. */
            for (int a = 0; a < 3; ++a) v[a] = (REAL)P->spec_v[a];
            w = 1;
            acc->ledger[PMO_L_SPEC] += (double)w;
            acc->ledger[PMO_L_RD] += v[2] < 0 ? (double)w : 0.0;
            acc->ledger[PMO_L_TT] += v[2] > 0 ? (double)w : 0.0;
            acc->counters[PMO_C_PHOTONS]++;
            goto record;
        }
    }
    acc->ledger[PMO_L_WINIT] += (double)w;

    if (c[0] < 0 || c[0] >= P->nx || c[1] < 0 || c[1] >= P->ny || c[2] < 0 || c[2] >= P->nz) {
        status = PMO_ERR_GEOMETRY;
        goto fail;
    }
    int64_t lin = ((int64_t)c[0] * P->ny + c[1]) * P->nz + c[2];
    int lab = P->labels[lin];
    if (lab == end || lab >= P->n_labels || !tab[lab].valid) { status = PMO_ERR_LABEL; goto fail; }
    PFX(props_t) cur = tab[lab];
    if (P->props_mode == PMO_PROPS_VOXEL)
        PFX(make_props)(&cur, P->vox_ma[lin], P->vox_ms[lin], P->g[lab], P->n[lab], 1);
    REAL ni = cur.n;
    REAL ia[3];
    for (int a = 0; a < 3; ++a) ia[a] = (REAL)1 / FABS(v[a]);

    for (;;) {
        /* step size in optical-depth units (:75) */
        ctr[0] = n_int; ctr[1] = 0; ctr[2] = idlo; ctr[3] = idhi;
        pmo_philox4x32_10(ctr, key, rnd);
        n_int++;
        REAL st = -LOG((REAL)pmo_u01(rnd[0]));
        /* rnd[1] is the step's spare uniform: the first Fresnel decision with
           0 < R < 1 in this step, or else the roulette, takes it */
        int ry_free = 1;

        for (;;) {
            /* distance to the nearest voxel face, db capped at 1000 (:80-90) */
            REAL db = 1000;
            int ax = 0;
            for (int a = 0; a < 3; ++a) {
                if (v[a] != 0) {
                    REAL d = (hl - PFX(sgn)(v[a]) * p[a]) * ia[a];
                    if (d < db) { db = d; ax = a; }
                }
            }
            REAL dbmt = db * cur.mt;
            if (!(st >= dbmt)) {
                /* hop inside the voxel (:170-175) */
                REAL s = st * cur.imt;
                for (int a = 0; a < 3; ++a) p[a] += v[a] * s;
                gL += (double)s;
                break;
            }
            /* move to the face and snap (:92-96) */
            for (int a = 0; a < 3; ++a) p[a] += v[a] * db;
            gL += (double)db;
            p[ax] = PFX(sgn)(v[ax]) * hl;
            st -= dbmt;
            n_cross++;
            if (++events > cap) { status = PMO_ERR_STEP_CAP; goto fail; }
            int step = signbit(v[ax]) ? -1 : 1;
            int dim = ax == 0 ? P->nx : (ax == 1 ? P->ny : P->nz);
            int nc = c[ax] + step;
            if (nc < 0 || nc >= dim) { status = PMO_ERR_GEOMETRY; goto fail; }
            int64_t stride = ax == 0 ? sx : (ax == 1 ? sy : 1);
            int64_t nlin = lin + step * stride;
            int nlab = P->labels[nlin];
            if (nlab >= P->n_labels || (nlab != end && !tab[nlab].valid)) {
                status = PMO_ERR_LABEL; goto fail;
            }
            REAL nt = nlab == end ? (REAL)P->n[end] : tab[nlab].n;
            int transmit = 1;
            if (ni != nt) {
                /* Fresnel / total internal reflection (:105-153), written with
                   cos/sin of the incidence and transmission angles. */
                REAL ca = FABS(v[ax]);
                if (ca > 1) ca = 1;
                REAL ra, cb = 1;
                REAL nr = ni / nt;
                REAL sa = SQRT(1 - ca * ca);
                REAL sb = nr * sa;
                if (ni > nt && sb >= 1) {
                    ra = 1;                     /* TIR: ai >= asin(nt/ni) */
                } else {
                    cb = SQRT(1 - sb * sb);
                    if (ca == 1) {
                        ra = 0;                 /* ai == 0 (:113-120) */
                    } else {
                        REAL cap_ = ca * cb - sa * sb;   /* cos(ai+at) */
                        REAL cam = ca * cb + sa * sb;    /* cos(ai-at) */
                        REAL sap = sa * cb + ca * sb;    /* sin(ai+at) */
                        REAL sam = sa * cb - ca * sb;    /* sin(ai-at) */
                        ra = (REAL)0.5 * sam * sam * (cam * cam + cap_ * cap_) / (sap * sap * cam * cam);
                    }
                }
                acc->counters[PMO_C_FRESNEL]++;
                /* transmit when R < u, u uniform in (0, 1] (:150).  Only
                   0 < R < 1 needs u: R == 0 always transmits, R >= 1 (TIR) or
                   a NaN always reflects.  u is the spare word of the step while
                   it is free, else word 0 of the draw (decision index, 1). */
                int refract;
                if (ra > 0 && ra < 1) {
                    uint32_t word = rnd[1];
                    if (!ry_free) {
                        uint32_t frn[4];
                        ctr[0] = n_fres; ctr[1] = 1; ctr[2] = idlo; ctr[3] = idhi;
                        pmo_philox4x32_10(ctr, key, frn);
                        word = frn[0];
                        acc->counters[PMO_C_XDRAWS]++;
                    }
                    ry_free = 0;
                    refract = ra < (REAL)pmo_u01(word);
                } else {
                    refract = ra <= 0;
                }
                n_fres++;
                if (refract) {
                    /* refract: tangential * ni/nt, normal = sign * cos(at),
                       renormalise (:124-134) */
                    for (int a = 0; a < 3; ++a) v[a] = a == ax ? PFX(sgn)(v[a]) * cb : v[a] * nr;
                    REAL inv = (REAL)1 / SQRT(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
                    for (int a = 0; a < 3; ++a) { v[a] *= inv; ia[a] = (REAL)1 / FABS(v[a]); }
                } else {
                    transmit = 0;
                    v[ax] = -v[ax];             /* Fresnel reflection (:150-152) */
                    acc->counters[PMO_C_REFLECT]++;
                }
            }
            if (!transmit) continue;
            /* cross into the neighbour (:137-148, :156-167) */
            if (nlab == lab && P->props_mode == PMO_PROPS_LABEL) acc->counters[PMO_C_SAMECROSS]++;
            if (grad) { seg_push(acc, lin, lab, gL, gN); gL = gN = 0.0; }
            c[ax] = nc;
            lin = nlin;
            p[ax] = -p[ax];
            lab = nlab;
            ni = nt;
            if (lab == end) {
                /* the photon left the medium: reference Rd/Tt split by the sign
                   of v_z (pymopt/voxel_gpu/_classes.py:326-334) */
                double wd = (double)w;
                if (v[2] < 0) acc->ledger[PMO_L_RD] += wd;
                else if (v[2] > 0) acc->ledger[PMO_L_TT] += wd;
                else acc->ledger[PMO_L_EXIT0] += wd;
                int cat = -1;
                if (ax == 2) {
                    cat = v[2] < 0 ? PMO_RR_TOP : PMO_RR_BOTTOM;
                    acc->ledger[v[2] < 0 ? PMO_L_RD_TOP : PMO_L_TT_BOTTOM] += wd;
                } else if (v[2] < 0) cat = PMO_RR_LAT_NEG;
                else if (v[2] > 0) cat = PMO_RR_LAT_POS;
                if (cat >= 0 && tal->rr) {
                    /* radialDistance bins (i*dr, (i+1)*dr] on the encoded exit
                       position x = l*(add_x - cx) + p_x (:302-310) */
                    REAL x = l * (REAL)(c[0] - P->center_ix) + p[0];
                    REAL y = l * (REAL)(c[1] - P->center_iy) + p[1];
                    REAL r = SQRT(x * x + y * y);
                    if (r > 0) {
                        REAL q = CEIL(r / (REAL)tal->dr);
                        if (q >= 1 && q <= (REAL)tal->nr) {
                            int b = (int)q - 1;
#pragma omp atomic
                            tal->rr[cat * tal->nr + b] += wd;
                            if (grad) seg_apply(acc, tal, tal->grad_coef[cat * tal->nr + b] * wd);
                        }
                    }
                }
                acc->counters[PMO_C_EXITS]++;
                acc->counters[PMO_C_PHOTONS]++;
                goto record;
            }
            if (P->props_mode == PMO_PROPS_VOXEL)
                PFX(make_props)(&cur, P->vox_ma[lin], P->vox_ms[lin], P->g[lab], P->n[lab], 1);
            else
                cur = tab[lab];
        }

        gN += (double)cur.ims;
        /* absorption, implicit capture (:179) */
        {
            REAL wn = w - w * cur.ma_mt;
            double dw = (double)w - (double)wn;
            w = wn;
            acc->ledger[PMO_L_ABS] += dw;
            if (tal->absorbed) {
#pragma omp atomic
                tal->absorbed[lin] += dw;
            }
        }
        /* Russian roulette (:182-195) */
        if (w <= (REAL)0.0001) {
            acc->counters[PMO_C_ROULETTE]++;
            /* the spare word of the step, or word 0 of the draw (interaction
               index, 3) when a Fresnel decision of the step took it */
            uint32_t word = rnd[1];
            if (!ry_free) {
                uint32_t rrn[4];
                ctr[0] = n_int - 1; ctr[1] = 3; ctr[2] = idlo; ctr[3] = idhi;
                pmo_philox4x32_10(ctr, key, rrn);
                word = rrn[0];
                acc->counters[PMO_C_XDRAWS]++;
            }
            if ((REAL)0.1 < (REAL)pmo_u01(word)) {
                acc->ledger[PMO_L_RLOSS] += (double)w;
                w = 0;
                for (int a = 0; a < 3; ++a) { p[a] = 0; v[a] = 0; c[a] = 0; }
                acc->counters[PMO_C_PHOTONS]++;
                goto record;
            }
            REAL wn = w * 10;
            acc->ledger[PMO_L_RGAIN] += (double)wn - (double)w;
            w = wn;
        }
        /* scattering: HG polar angle, uniform azimuth, MCML rotation (:197-219) */
        {
            REAL ct = PFX(hg_cos)(&cur, (REAL)pmo_u01(rnd[2]));
            REAL s2 = 1 - ct * ct;
            REAL sth = SQRT(s2 > 0 ? s2 : 0);
            REAL phi = TWO_PI * (REAL)pmo_u01(rnd[3]);
            REAL cf = COS(phi), sf = SIN(phi);
            if ((REAL)0.99999 < FABS(v[2])) {
                REAL sz = PFX(sgn)(v[2]);
                v[0] = sth * cf;
                v[1] = sth * sf;
                v[2] = sz * ct;
            } else {
                REAL tmp = SQRT(1 - v[2] * v[2]);
                REAL f = sth / tmp;
                REAL vx = v[0], vy = v[1], vz = v[2];
                v[0] = f * (vx * vz * cf - vy * sf) + vx * ct;
                v[1] = f * (vy * vz * cf + vx * sf) + vy * ct;
                v[2] = -sth * cf * tmp + vz * ct;
            }
            REAL inv = (REAL)1 / SQRT(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            for (int a = 0; a < 3; ++a) { v[a] *= inv; ia[a] = (REAL)1 / FABS(v[a]); }
        }
        if (++events > cap) { status = PMO_ERR_STEP_CAP; goto fail; }
    }

fail:
    acc->ledger[PMO_L_ERRW] += (double)w;
    acc->counters[status == PMO_ERR_GEOMETRY ? PMO_C_ERR_GEOM
                  : status == PMO_ERR_LABEL ? PMO_C_ERR_LABEL : PMO_C_ERR_CAP]++;
    acc->counters[PMO_C_PHOTONS]++;
record:
    acc->counters[PMO_C_INTERACT] += n_int;
    acc->counters[PMO_C_CROSS] += n_cross;
    if (tal->ph_state) {
        double *o = tal->ph_state + 10 * j;
        for (int a = 0; a < 3; ++a) { o[a] = (double)p[a]; o[3 + a] = (double)v[a]; }
        o[6] = (double)w;
        o[7] = (double)c[0]; o[8] = (double)c[1]; o[9] = (double)c[2];
    }
    if (tal->ph_counts) {
        uint32_t *o = tal->ph_counts + 4 * j;
        o[0] = n_int; o[1] = n_cross; o[2] = n_fres; o[3] = (uint32_t)status;
    }
    return status;
}

/* Run photons [photon_begin, photon_begin + photon_count) of P. */
int PFX(oracle_run)(const pmo_problem *P, oracle_tallies *tal, int threads) {
    PFX(props_t) tab[256];
    for (int i = 0; i < 256; ++i) {
        int ok = i < P->n_labels && i != P->end_label;
        if (ok && P->props_mode == PMO_PROPS_LABEL)
            PFX(make_props)(&tab[i], P->ma[i], P->ms[i], P->g[i], P->n[i], 1);
        else if (ok)
            PFX(make_props)(&tab[i], 0.f, 0.f, P->g[i], P->n[i], 1);
        else
            PFX(make_props)(&tab[i], 0.f, 0.f, 0.f, i < P->n_labels ? P->n[i] : 1.f, 0);
    }
    int nthreads = threads > 0 ? threads : 1;
    int worst = PMO_OK;
#pragma omp parallel num_threads(nthreads)
    {
        oracle_acc acc;
        memset(&acc, 0, sizeof(acc));
        (void)seg_push;
        int st_local = PMO_OK;
#pragma omp for schedule(dynamic, 64)
        for (int64_t k = 0; k < (int64_t)P->photon_count; ++k) {
            int s = PFX(trace)(P, tab, tal, &acc, P->photon_begin + (uint64_t)k);
            if (s != PMO_OK) st_local = s;
        }
#pragma omp critical
        {
            for (int i = 0; i < PMO_LEDGER_N; ++i) tal->ledger[i] += acc.ledger[i];
            for (int i = 0; i < PMO_COUNTERS_N; ++i) tal->counters[i] += acc.counters[i];
            if (st_local != PMO_OK) worst = st_local;
        }
        free(acc.seg_lin);
        free(acc.seg_lab);
        free(acc.seg_L);
        free(acc.seg_N);
    }
    return worst;
}

#undef PFX
