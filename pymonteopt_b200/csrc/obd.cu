// obd.cu — the optical bench that follows the transport: exit photons through
// a lens, two annular slits, an optional laser-diode mount, a second lens and
// a photodiode, for every detector offset Z of a scan.
//
// This restates the reference's vectorised NumPy ray tracing
// (pymopt/optics/_classes.py:50-380 for the elements, :454-526 for the
// scan, :528-566 for the side geometry) per photon:
// - a warp per exit photon, its lanes spread over the scan's Z values;
//   photons that miss lens 1 at every Z are dropped first by a test that
//   cannot drop a photon the exact per-Z test would keep;
// - the intensity of each Z summed in shared memory, then one FP64 atomic
//   per block and Z.
//
// Arithmetic follows the reference's NumPy types:
// - exit photons arrive as float32 and the first normalisation of v runs in
//   single precision;
// - every element position depends on Z, a float64 scalar of np.arange, so
//   from the first plane hit on the positions, normals, directions and
//   Fresnel terms are float64 (:133-136, :152-222);
// - the side geometry's shifted x is rounded back to float32, as it is
//   stored into the float32 array (:561-562);
// - this file is built without FMA contraction, so products and sums round
//   one by one as in NumPy.
//
// The reference's Fresnel decision at each lens surface is
// np.random.rand() - R > 0 (:212-215).  Here the four uniforms of a
// (photon, Z) pair come from one Philox4x32-10 draw, key (seed_lo, seed_hi)
// and counter (Z index, 5, photon_lo, photon_hi), as x * 2^-32 in [0, 1).
// A fixed uniform (fixed_u in [0, 1)) replaces the draws for deterministic
// comparisons.
//
// Work is ordered for speed without changing any decision:
// - lens 1's flat face has a fixed normal, so its refraction and reflectance
//   are computed once per photon rather than once per Z;
// - the decisions do not change the ray, so the geometry is traced first;
// - the reflectances (two acos, two sin, two tan each) and the draw are
//   evaluated only for photons that reach the photodiode.
#include "pmo_internal.h"

namespace {

struct Ray {
    double px, py, pz, vx, vy, vz;
};

__device__ __forceinline__ void normalize(Ray &r) {
    const double s = sqrt(r.vx * r.vx + r.vy * r.vy + r.vz * r.vz);
    r.vx = r.vx / s;
    r.vy = r.vy / s;
    r.vz = r.vz / s;
}

// move to the plane z = zp along v (:64-66, :133-136, :325-327)
__device__ __forceinline__ void hit_plane(Ray &r, double zp) {
    const double a = (zp - r.pz) / r.vz;
    r.px = r.px + a * r.vx;
    r.py = r.py + a * r.vy;
    r.pz = r.pz + a * r.vz;
}

__device__ __forceinline__ double radius(const Ray &r) {
    return sqrt(r.px * r.px + r.py * r.py);
}

// Cosines of the incidence and transmission angles at one surface.
struct Cosines {
    double ai, at;
};

// Refraction through a surface with unit normal nn, from air into glass of
// index n or out of it (:152-188): leaves the refracted direction, not yet
// normalised, in r and returns the two cosines.  tir: the threshold
// asin(1/n) when leaving the glass, where angles at or above it reflect
// totally and the photon is gone (returns false).
__device__ __forceinline__ bool refract(Ray &r, double nx, double ny, double nz, double n,
                                        bool lens_to_air, double tir, Cosines &c) {
    const double cos_ai = nx * r.vx + ny * r.vy + nz * r.vz;
    const double a = lens_to_air ? n / 1.0 : 1.0 / n;
    if (lens_to_air && acos(cos_ai) >= tir) return false;   // total internal reflection
    const double sgn = cos_ai > 0.0 ? 1.0 : (cos_ai < 0.0 ? -1.0 : 0.0);
    const double cos_at = sgn * sqrt(1.0 - (a * a) * (1.0 - cos_ai * cos_ai));
    const double g = cos_at - a * cos_ai;
    r.vx = a * r.vx + g * nx;
    r.vy = a * r.vy + g * ny;
    r.vz = a * r.vz + g * nz;
    c.ai = cos_ai;
    c.at = cos_at;
    return true;
}

// Fresnel reflectance of the reference, 0.5 [(sin(ai-at)/sin(ai+at))^2 +
// (tan(ai-at)/tan(ai+at))^2] (:212-215); NaN at normal incidence.  It does
// not change the ray, so the kernel evaluates it only for photons that reach
// the photodiode.
__device__ __forceinline__ double reflectance(const Cosines &c) {
    const double ai = acos(c.ai), at = acos(c.at);
    const double s1 = sin(ai - at) / sin(ai + at);
    const double t1 = tan(ai - at) / tan(ai + at);
    return 0.5 * (s1 * s1 + t1 * t1);
}

// the reference's decision rand - R > 0 (false for NaN R)
__device__ __forceinline__ bool passes(double u, double R) { return u - R > 0.0; }

// the lens's spherical surface: intersection (:138-150), normal (:200-210)
// and refraction; the cosines go to c for the deferred Fresnel decision
__device__ __forceinline__ bool convex(Ray &r, double center, double rad, bool inward,
                                       double half_outer, double n, double tir, Cosines &c) {
    normalize(r);
    const double pp = r.pz - center;
    const double A = r.vx * r.vx + r.vy * r.vy + r.vz * r.vz;
    const double B = 2.0 * (r.px * r.vx + r.py * r.vy + pp * r.vz);
    const double C = r.px * r.px + r.py * r.py + pp * pp - rad * rad;
    const double disc = sqrt(B * B - 4.0 * A * C);
    const double t = inward ? (-B - disc) / (2.0 * A) : (-B + disc) / (2.0 * A);
    r.px = r.px + r.vx * t;
    r.py = r.py + r.vy * t;
    r.pz = r.pz + r.vz * t;
    if (!(radius(r) <= half_outer)) return false;
    const double d = sqrt(rad * rad - (r.px * r.px + r.py * r.py));
    const double dx = -r.px / d, dy = -r.py / d;
    double nx = inward ? dx : -dx, ny = inward ? dy : -dy, nz = -1.0;
    const double s = sqrt(nx * nx + ny * ny + nz * nz);
    nx = nx / s;
    ny = ny / s;
    nz = nz / s;
    // lens 1 (outward) leaves the glass here, lens 2 (inward) enters it
    if (!refract(r, nx, ny, nz, n, !inward, tir, c)) return false;
    normalize(r);
    return true;
}

// lens 2's flat face at z = pos, normal (0, 0, -1), leaving the glass
// (:103-113)
__device__ __forceinline__ bool plano_out(Ray &r, double pos, double half_outer, double n,
                                          double tir, Cosines &c) {
    normalize(r);
    hit_plane(r, pos);
    if (!(radius(r) <= half_outer)) return false;
    if (!refract(r, 0.0, 0.0, -1.0, n, true, tir, c)) return false;
    normalize(r);
    return true;
}

// annular slit: front and back faces (:79-84)
__device__ __forceinline__ bool slit(Ray &r, double front, double back, double d_in,
                                     double d_out) {
    hit_plane(r, front);
    double pp = radius(r);
    if (!(pp < d_out && pp > d_in)) return false;
    hit_plane(r, back);
    pp = radius(r);
    return pp < d_out && pp > d_in;
}

// laser-diode mount: photons pass where the mount is not (:336-376)
__device__ __forceinline__ bool ld_mount(Ray &r, double front, double back, double a1,
                                         double b1, double a2, double b2, double b3) {
    hit_plane(r, front);
    if (!(r.py > a1 * r.px + b1 || r.py < a2 * r.px + b2 || r.py < b3)) return false;
    hit_plane(r, back);
    return r.py > a1 * r.px + b1 || r.py < a2 * r.px + b2 || r.py < b3;
}

constexpr int kMaxZ = 4096;
constexpr int kObdThreads = 256;

// Constants of one scan, shared by every photon.
struct ScanConsts {
    double d_in, d_out;                 // annular slit radii
    double a1, b1, a2, b2, b3;          // laser-diode mount edges
    double tir1, tir2;                  // total-internal-reflection thresholds
    double zlo, zhi;                    // smallest and largest Z of the scan
    pmo::PhiloxKeys rk;
};

// The exit photon's direction, normalised in float32 like its input.
__device__ __forceinline__ void exit_direction(const float *v, int64_t n, int64_t i, double &ux,
                                               double &uy, double &uz) {
    const float vx0 = v[i], vy0 = v[n + i], vz0 = v[2 * n + i];
    const float vs = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(vx0, vx0), __fmul_rn(vy0, vy0)),
                                          __fmul_rn(vz0, vz0)));
    ux = (double)__fdiv_rn(vx0, vs);
    uy = (double)__fdiv_rn(vy0, vs);
    uz = (double)__fdiv_rn(vz0, vs);
}

// Whether photon i can pass lens 1's aperture for some Z of the scan.  Its
// hit point on lens 1's plane is affine in Z, A + B Z (the plane sits at
// Z - bfl1; the side geometry's x shift is affine in Z too), so the distance
// from the axis is convex in Z and smallest at the clamped vertex Z*.  The
// test uses an aperture 1 um wider than the lens, far more than the rounding
// of the exact per-Z test (and of the side geometry's float32 x), so it only
// drops photons that the exact test rejects at every Z.  A direction with
// v_z = 0 or a zero vector gives NaN, which no Z passes either.
__device__ __forceinline__ bool reaches_lens1(const pmo_obd_params &prm, const ScanConsts &k,
                                              const float *p, const float *v, const float *w,
                                              int64_t n, int64_t i) {
    if (!(w[i] != 0.0f)) return false;   // adds nothing to any Z
    double ux, uy, uz;
    exit_direction(v, n, i, ux, uy, uz);
    const double iz = 1.0 / uz;
    const double st = prm.side ? prm.side_tan : 0.0;
    const double bx = ux * iz - st, by = uy * iz;
    const double ax = (double)p[i] - (prm.side ? prm.side_dz * st : 0.0) - prm.bfl1 * ux * iz;
    const double ay = (double)p[n + i] - prm.bfl1 * uy * iz;
    const double bb = bx * bx + by * by;
    double zs = bb > 0.0 ? -(ax * bx + ay * by) / bb : k.zlo;
    zs = fmin(fmax(zs, k.zlo), k.zhi);
    const double qx = ax + bx * zs, qy = ay + by * zs;
    const double rm = prm.outer_d1 / 2 + 1e-3;
    return qx * qx + qy * qy <= rm * rm;
}

// Photon i through the bench, the lanes of a warp taking every 32nd Z of
// the scan (lane, lane + 32, ...).  Neighbouring Z send the photon along
// nearly the same path, so the lanes pass and fail the same elements far
// more often than 32 different photons would.  Each Z that reaches the
// photodiode and passes the four Fresnel decisions adds w_i to s_int[Z].
__device__ void scan_photon(const pmo_obd_params &prm, const ScanConsts &k, const float *p,
                            const float *v, const float *w, int64_t n, int64_t i, int lane,
                            double *s_int) {
    const float x0 = p[i], y0 = p[n + i];
    double ux, uy, uz;
    exit_direction(v, n, i, ux, uy, uz);
    const double wi = (double)w[i];
    // Lens 1's flat face has the fixed normal (0, 0, -1): the incidence
    // angle, the reflectance and the refracted direction do not depend on
    // Z, only the hit point and the draw do.  The direction is computed once
    // per photon, the reflectance the first time a Z reaches the photodiode,
    // with the same operations as inside the scan.
    Ray r1;
    r1.px = r1.py = r1.pz = 0.0;
    r1.vx = ux;
    r1.vy = uy;
    r1.vz = uz;
    Cosines c1;
    refract(r1, 0.0, 0.0, -1.0, prm.n1, false, 0.0, c1);
    double R1 = -1.0;   // not computed yet (a computed R1 is >= 0 or NaN)
    normalize(r1);
    for (int zi = lane; zi < prm.n_z; zi += 32) {
        const double Z = prm.z[zi];
        // element positions of this Z (:454-470)
        const double zl1 = -prm.bfl1 + Z;
        const double zl2 = zl1 - prm.ct1 - prm.slit_thickness * 2 - prm.ct2 - prm.distance_2slits;
        const double zs1 = zl1 - prm.ct1;
        const double zs2 = zl2 + prm.ct2 + prm.slit_thickness;
        const double zpd = zl2 - prm.bfl2 - prm.pd_correction;
        Ray r;
        r.px = prm.side ? (double)(float)((double)x0 - (Z + prm.side_dz) * prm.side_tan)
                        : (double)x0;
        r.py = (double)y0;
        r.pz = 0.0;
        r.vx = ux;
        r.vy = uy;
        r.vz = uz;
        // lens 1: flat face (the float32-normalised v goes in as it is)
        // then curved face (:295-302)
        hit_plane(r, zl1);
        if (!(radius(r) <= prm.outer_d1 / 2)) continue;
        r.vx = r1.vx;
        r.vy = r1.vy;
        r.vz = r1.vz;
        Cosines c2, c3, c4;
        if (!convex(r, zl1 - (prm.ct1 - prm.r1), prm.r1, false, prm.outer_d1 / 2, prm.n1,
                    k.tir1, c2))
            continue;
        if (!slit(r, zs1, zs1 - prm.slit_thickness, k.d_in, k.d_out)) continue;
        if (prm.ld_fix_part) {
            const double zf = zs1 - prm.slit_thickness - 10;
            if (!ld_mount(r, zf, zf - 5, k.a1, k.b1, k.a2, k.b2, k.b3)) continue;
        }
        if (!slit(r, zs2, zs2 - prm.slit_thickness, k.d_in, k.d_out)) continue;
        // lens 2: curved face then flat face (:305-313)
        if (!convex(r, zl2 + (prm.ct2 - prm.r2), prm.r2, true, prm.outer_d2 / 2, prm.n2,
                    0.0, c3))
            continue;
        if (!plano_out(r, zl2, prm.outer_d2 / 2, prm.n2, k.tir2, c4)) continue;
        // photodiode (:325-334)
        hit_plane(r, zpd);
        if (!(radius(r) < prm.d_pd / 2)) continue;
        // the four Fresnel decisions, which do not change the ray: drawn
        // and taken only for photons that reach the photodiode
        double u[4];
        if (prm.fixed_u >= 0.0) {
            u[0] = u[1] = u[2] = u[3] = prm.fixed_u;
        } else {
            const uint4 q = pmo::philox4x32_10(
                make_uint4((uint32_t)zi, 5u, (uint32_t)i, (uint32_t)((uint64_t)i >> 32)), k.rk);
            u[0] = (double)q.x * 0x1p-32;
            u[1] = (double)q.y * 0x1p-32;
            u[2] = (double)q.z * 0x1p-32;
            u[3] = (double)q.w * 0x1p-32;
        }
        if (R1 < 0.0) R1 = reflectance(c1);
        if (!passes(u[0], R1) || !passes(u[1], reflectance(c2)) ||
            !passes(u[2], reflectance(c3)) || !passes(u[3], reflectance(c4)))
            continue;
        atomicAdd(s_int + zi, wi);
    }
}

// Each warp walks tiles of 32 photons.  Its lanes test one photon each for
// lens 1 (about 60 % of Lambertian exits miss it at every Z of the default
// scan), then the warp scans the photons that may pass one after another,
// its lanes spread over Z.
__global__ void __launch_bounds__(kObdThreads, 3) obd_kernel(pmo_obd_params prm,
                                                             const float *__restrict__ p,
                                                             const float *__restrict__ v,
                                                             const float *__restrict__ w,
                                                             int64_t n,
                                                             double *__restrict__ intensity) {
    extern __shared__ double s_int[];
    __shared__ double s_zlo[kObdThreads / 32], s_zhi[kObdThreads / 32];
    __shared__ ScanConsts s_k;
    const int tid = threadIdx.x;
    for (int i = tid; i < prm.n_z; i += blockDim.x) s_int[i] = 0.0;
    // the scan's Z range
    double lo = prm.z[0], hi = prm.z[0];
    for (int i = tid; i < prm.n_z; i += blockDim.x) {
        lo = fmin(lo, prm.z[i]);
        hi = fmax(hi, prm.z[i]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((tid & 31) == 0) {
        s_zlo[tid >> 5] = lo;
        s_zhi[tid >> 5] = hi;
    }
    if (tid == 0) {
        // scan constants, read from shared memory by every thread (in
        // registers they would spill)
        ScanConsts &k = s_k;
        k.rk = pmo::philox_round_keys((uint32_t)prm.seed, (uint32_t)(prm.seed >> 32));
        k.d_out = prm.slit_d / 2 + prm.slit_width / 2;
        k.d_in = prm.slit_d / 2 - prm.slit_width / 2;
        // mount edges: angle 68/180 rad, thickness 5, width 6 (:338-350)
        const double ang = 68.0 / 180.0;
        k.a1 = 1.0 / tan(ang) - 1.0 / (sin(ang) * cos(ang));
        k.b1 = 6.0 / cos(ang);
        k.a2 = (cos(ang) + 1.0) / sin(ang);
        k.b2 = -6.0;
        k.b3 = -6.0;
        // total-internal-reflection thresholds asin(nt / ni) of the
        // glass-to-air surfaces (:176)
        k.tir1 = asin(1.0 / prm.n1);
        k.tir2 = asin(1.0 / prm.n2);
    }
    __syncthreads();
    if (tid == 0) {
        double zlo = s_zlo[0], zhi = s_zhi[0];
        for (int j = 1; j < kObdThreads / 32; ++j) {
            zlo = fmin(zlo, s_zlo[j]);
            zhi = fmax(zhi, s_zhi[j]);
        }
        s_k.zlo = zlo;
        s_k.zhi = zhi;
    }
    __syncthreads();
    const ScanConsts &k = s_k;

    const int lane = tid & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + tid) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * 32; base < n; base += n_warps * 32) {   // warp-uniform
        const int64_t i = base + lane;
        const bool live = i < n && reaches_lens1(prm, k, p, v, w, n, i);
        unsigned m = __ballot_sync(0xffffffffu, live);
        while (m) {
            const int b = __ffs(m) - 1;
            m &= m - 1;
            scan_photon(prm, k, p, v, w, n, base + b, lane, s_int);
        }
    }
    __syncthreads();
    for (int i = tid; i < prm.n_z; i += blockDim.x)
        if (s_int[i] != 0.0) atomicAdd(intensity + i, s_int[i]);
}

}  // namespace

extern "C" {

int pmo_run_obd(const pmo_obd_params *prm, const float *p, const float *v, const float *w, int64_t n,
            double *intensity, void *stream) {
    if (!prm || !intensity || n < 0 || (n > 0 && (!p || !v || !w))) return PMO_ERR_ARG;
    if (!prm->z || prm->n_z < 1 || prm->n_z > kMaxZ) return PMO_ERR_ARG;
    if (!(prm->fixed_u < 1.0)) return PMO_ERR_ARG;
    if (n == 0) return PMO_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int sms = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t smem = (size_t)prm->n_z * sizeof(double);
    if (smem > 40 * 1024 &&
        cudaFuncSetAttribute(obd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
        return PMO_ERR_CUDA;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, obd_kernel, kObdThreads, smem) !=
            cudaSuccess ||
        occ < 1)
        return PMO_ERR_CUDA;
    // one resident wave of blocks; each walks tiles of photons
    int64_t blocks = (n + kObdThreads - 1) / kObdThreads;
    if (blocks > (int64_t)sms * occ) blocks = (int64_t)sms * occ;
    obd_kernel<<<(unsigned)blocks, kObdThreads, smem, s>>>(*prm, p, v, w, n, intensity);
    return cudaGetLastError() == cudaSuccess ? PMO_OK : PMO_ERR_CUDA;
}

}  // extern "C"
