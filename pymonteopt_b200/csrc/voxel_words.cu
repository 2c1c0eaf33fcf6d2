// voxel_words.cu — the uniform-box map the transport kernel steps on.
//
// Each voxel v gets a box {|dx| <= e, |dy| <= e, |dz| <= d} (in voxels,
// around v) whose voxels all carry label(v).  The word holds
//   bits 0-7   label(v)
//   bits 8-11  d, the half-extent along z (0 .. 15)
//   bits 12-15 c, a code of the lateral half-extent: e = max(d, lat(c)) with
//              lat(0) = 0 and lat(c) = ((2 | (c & 1)) << (c >> 1)) >> 1 for
//              c >= 1 (1, 2, 3, 4, 6, 8, 12, ... 192).
// A photon in v may treat the box as one cell: it meets no label change,
// hence no index step and no change of mu, before the box's faces.  Crossing
// a face between two voxels of one label changes nothing in the reference's
// transport (pymopt/voxel_gpu/_cukernel.py:154-167), so stepping box to box
// follows the same path as stepping voxel to voxel.
//
// d: the cube of half-extent d = min(cap, D_E(v)) is uniform, where D_E is the
// L-infinity distance to the edge set E (voxels with a 26-neighbour of another
// label, and the array border).  If a voxel w of another label were within
// distance D_E(v) of v, the voxel next to w on the way from v would be in E and
// closer than D_E(v).
//
// e: P(u), the same construction inside u's z-plane with the 8 in-plane
// neighbours and the lateral border (capped at 192), is the half-extent of a
// uniform in-plane square around u.  The box's slices are the squares around
// v + dz*z_hat for |dz| <= d, which lie in v's cube and so carry label(v).
// Hence e_true = min over |dz| <= d of P(v + dz*z_hat), and e_true >= d.  The
// word stores the largest code with lat(c) <= e_true.  This widens the boxes
// of thin layers, such as a 2-voxel skin layer whose voxels all have d = 0.
//
// Both are found by counting edge voxels in boxes.  D_E(v) >= r exactly when
// the cube of half-extent r - 1 around v holds no voxel of E (clipped to the
// array: a cube that reaches past it holds border voxels, which are in E), so
// d is the largest r <= cap whose cube count is zero.  Likewise lat(c) <=
// e_true exactly when the box of half-extents (lat(c) - 1, lat(c) - 1, d)
// holds no voxel of E2 (the in-plane edge set), so c is the largest code
// whose box count is zero.  Both counts fall as the box shrinks, so a binary
// search over r (0 .. 15) and over c (0 .. 15) takes four box counts each.  A
// box count is eight reads of a summed-area table (inclusive 3-D prefix sums
// of the edge indicator), kept as uint32: the counts are exact modulo 2^32
// and no box holds 2^32 voxels.
//
// Passes (each streams the volume once, coalesced along z):
//   1. edges + z prefix: one warp per (x, y) row; the E and E2 bits of each
//      voxel into the mask byte, the warp-scanned z prefix of E into the table;
//   2. y prefix, 3. x prefix: one thread per row, a running sum;
//   4. d per voxel (binary search on the table of E), into the mask byte;
//   5-7. the table again, for E2;
//   8. c per voxel (binary search on the table of E2) and the word.
// Passes 4 and 8 also run one warp per row, so that x and y are found once
// per row rather than by divisions per voxel, and index in 32 bits.
#include "pmo_internal.h"

namespace {

constexpr unsigned kFull = 0xffffffffu;

__host__ __device__ inline int lat_of(int c) {
    return c ? ((2 | (c & 1)) << (c >> 1)) >> 1 : 0;
}

// Pass 1.  mask = E | E2 << 1; sat = prefix of E along z.  One warp per
// (x, y) row; the row index is warp-uniform, so are the loop bounds.
__global__ void edge_scan_z_kernel(const uint8_t *__restrict__ lab, int nx, int ny, int nz,
                                   uint8_t *__restrict__ mask, uint32_t *__restrict__ sat) {
    const int lane = threadIdx.x & 31;
    const uint32_t rows = (uint32_t)nx * (uint32_t)ny;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < rows; row += warps) {
        const int x = (int)(row / (uint32_t)ny), y = (int)(row % (uint32_t)ny);
        const bool lateral = x == 0 || y == 0 || x == nx - 1 || y == ny - 1;
        const size_t base = (size_t)row * nz;
        uint32_t carry = 0;
        for (int z0 = 0; z0 < nz; z0 += 32) {
            const int z = z0 + lane;
            uint32_t e = 0, e2 = 0;
            if (z < nz) {
                if (lateral) {
                    e = e2 = 1;
                } else {
                    // interior row: the 8 neighbouring rows exist
                    const uint8_t me = lab[base + z];
                    uint32_t plane = 0, off = 0;
                    for (int dx = -1; dx <= 1; ++dx) {
                        for (int dy = -1; dy <= 1; ++dy) {
                            const uint8_t *r = lab + (size_t)((ptrdiff_t)base +
                                                              ((ptrdiff_t)dx * ny + dy) * nz);
                            plane |= r[z] != me;
                            if (z > 0) off |= r[z - 1] != me;
                            if (z < nz - 1) off |= r[z + 1] != me;
                        }
                    }
                    e2 = plane;
                    e = plane | off | (z == 0) | (z == nz - 1);
                }
                mask[base + z] = (uint8_t)(e | (e2 << 1));
            }
            uint32_t s = e;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(kFull, s, o);
                if (lane >= o) s += t;
            }
            if (z < nz) sat[base + z] = carry + s;
            carry += __shfl_sync(kFull, s, 31);
        }
    }
}

// Pass 5.  sat = prefix along z of bit `bit` of the mask.
__global__ void scan_z_bit_kernel(const uint8_t *__restrict__ mask, int nx, int ny, int nz,
                                  int bit, uint32_t *__restrict__ sat) {
    const int lane = threadIdx.x & 31;
    const uint32_t rows = (uint32_t)nx * (uint32_t)ny;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < rows; row += warps) {
        const size_t base = (size_t)row * nz;
        uint32_t carry = 0;
        for (int z0 = 0; z0 < nz; z0 += 32) {
            const int z = z0 + lane;
            uint32_t s = z < nz ? (mask[base + z] >> bit) & 1u : 0u;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(kFull, s, o);
                if (lane >= o) s += t;
            }
            if (z < nz) sat[base + z] = carry + s;
            carry += __shfl_sync(kFull, s, 31);
        }
    }
}

// Passes 2 and 3.  In-place running sum along y (stride nz) or x (stride
// ny*nz); one thread per row, consecutive threads on consecutive z.  Eight
// loads are issued before their sums are stored.
__global__ void scan_strided_kernel(uint32_t *__restrict__ sat, uint32_t rows, int nz,
                                    size_t outer_stride, size_t stride, int len) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < rows;
         t += gridDim.x * blockDim.x) {
        uint32_t *p = sat + (size_t)(t / (uint32_t)nz) * outer_stride + (t % (uint32_t)nz);
        uint32_t run = 0;
        int k = 0;
        for (; k + 8 <= len; k += 8) {
            uint32_t v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = p[(size_t)(k + j) * stride];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                run += v[j];
                p[(size_t)(k + j) * stride] = run;
            }
        }
        for (; k < len; ++k) {
            run += p[(size_t)k * stride];
            p[(size_t)k * stride] = run;
        }
    }
}

struct Grid3 {
    int nx, ny, nz;
};

// Edge voxels in [x-h, x+h] x [y-h, y+h] x [z-hz, z+hz], clipped to the
// array (h, hz >= 0).  The lower corners sit one below the box; a corner
// below 0 reads as 0 and is skipped.  Every offset is below the voxel count,
// hence below 2^32.
__device__ inline uint32_t box_count(const uint32_t *__restrict__ s, const Grid3 &g, int x, int y,
                                     int z, int h, int hz) {
    const int xa = x - h - 1, xb = min(x + h, g.nx - 1);
    const int ya = y - h - 1, yb = min(y + h, g.ny - 1);
    const int za = z - hz - 1, zb = min(z + hz, g.nz - 1);
    const uint32_t ny = (uint32_t)g.ny, nz = (uint32_t)g.nz;
    const uint32_t rbb = ((uint32_t)xb * ny + (uint32_t)yb) * nz;
    uint32_t sum = __ldg(s + rbb + zb);
    if (za >= 0) sum -= __ldg(s + rbb + za);
    if (ya >= 0) {
        const uint32_t rba = ((uint32_t)xb * ny + (uint32_t)ya) * nz;
        sum -= __ldg(s + rba + zb);
        if (za >= 0) sum += __ldg(s + rba + za);
    }
    if (xa >= 0) {
        const uint32_t rab = ((uint32_t)xa * ny + (uint32_t)yb) * nz;
        sum -= __ldg(s + rab + zb);
        if (za >= 0) sum += __ldg(s + rab + za);
        if (ya >= 0) {
            const uint32_t raa = ((uint32_t)xa * ny + (uint32_t)ya) * nz;
            sum += __ldg(s + raa + zb);
            if (za >= 0) sum -= __ldg(s + raa + za);
        }
    }
    return sum;
}

// Pass 4.  d into bits 2-5 of the mask.  One warp per (x, y) row, as in the
// scans: x and y come once per row, a lane takes z = lane, lane + 32, ...
__global__ void depth_kernel(const uint32_t *__restrict__ sat, Grid3 g, int cap,
                             uint8_t *__restrict__ mask) {
    const int lane = threadIdx.x & 31;
    const uint32_t rows = (uint32_t)g.nx * (uint32_t)g.ny;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < rows; row += warps) {
        const int x = (int)(row / (uint32_t)g.ny), y = (int)(row % (uint32_t)g.ny);
        uint8_t *mrow = mask + (size_t)row * g.nz;
        for (int z = lane; z < g.nz; z += 32) {
            const uint8_t m = mrow[z];
            int d = 0;
            if (!(m & 1) && cap > 0) {
                int lo = 1, hi = cap + 1;   // r = lo is uniform (v is not in E); r = hi is not
                // most voxels of thick regions reach the cap: one count settles them
                if (box_count(sat, g, x, y, z, cap - 1, cap - 1) == 0u) lo = cap;
                else hi = cap;
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (box_count(sat, g, x, y, z, mid - 1, mid - 1) == 0u) lo = mid;
                    else hi = mid;
                }
                d = lo;
            }
            mrow[z] = (uint8_t)((m & 3) | (d << 2));
        }
    }
}

// Pass 8.  The lateral code and the word; one warp per (x, y) row.
__global__ void pack_kernel(const uint8_t *__restrict__ lab, const uint8_t *__restrict__ mask,
                            const uint32_t *__restrict__ sat, Grid3 g,
                            uint16_t *__restrict__ words) {
    const int lane = threadIdx.x & 31;
    const uint32_t rows = (uint32_t)g.nx * (uint32_t)g.ny;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < rows; row += warps) {
        const int x = (int)(row / (uint32_t)g.ny), y = (int)(row % (uint32_t)g.ny);
        const size_t base = (size_t)row * g.nz;
        for (int z = lane; z < g.nz; z += 32) {
            const uint8_t m = mask[base + z];
            const int d = (m >> 2) & 15;
            int lo = 0, hi = 16;   // code 0 needs no uniform square
            if (!(m & 2)) {
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (box_count(sat, g, x, y, z, lat_of(mid) - 1, d) == 0u) lo = mid;
                    else hi = mid;
                }
            }
            words[base + z] = (uint16_t)(lab[base + z] | (d << 8) | (lo << 12));
        }
    }
}

}  // namespace

extern "C" {

// words[nvox] (uint16) from labels[nvox]; scratch: PMO_VOXEL_WORDS_SCRATCH
// bytes per voxel (the uint32 table, then the mask byte), 4-byte aligned.
int pmo_build_voxel_words(const uint8_t *labels, int nx, int ny, int nz, int cap,
                          uint16_t *words, void *scratch, size_t scratch_bytes, void *stream) {
    if (!labels || !words || !scratch || nx < 1 || ny < 1 || nz < 1) return PMO_ERR_ARG;
    if (cap < 0 || cap > 15) return PMO_ERR_ARG;
    const uint64_t total = (uint64_t)nx * ny * nz;
    if (total >= (1ull << 32)) return PMO_ERR_ARG;
    if (reinterpret_cast<uintptr_t>(scratch) % 4 != 0) return PMO_ERR_ARG;
    if (scratch_bytes < PMO_VOXEL_WORDS_SCRATCH * total) return PMO_ERR_WORKSPACE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t *sat = static_cast<uint32_t *>(scratch);
    uint8_t *mask = reinterpret_cast<uint8_t *>(sat + total);
    const Grid3 g{nx, ny, nz};
    // one warp per (x, y) row or one thread per strided row, no grid-stride
    // reuse: blocks start in row order, so the probes of resident blocks
    // sweep the table as one front along x and the planes they read stay in
    // L2 between uses
    auto blocks_for = [](uint64_t threads) { return (unsigned)((threads + 255) / 256); };
    const unsigned g_rows = blocks_for((uint64_t)nx * ny * 32);   // a warp per (x, y) row
    const uint32_t rows_y = (uint32_t)nx * nz, rows_x = (uint32_t)ny * nz;
    const size_t plane = (size_t)ny * nz;
    // d: table of E, then the binary search
    edge_scan_z_kernel<<<g_rows, 256, 0, s>>>(labels, nx, ny, nz, mask, sat);
    scan_strided_kernel<<<blocks_for(rows_y), 256, 0, s>>>(sat, rows_y, nz, plane, nz, ny);
    scan_strided_kernel<<<blocks_for(rows_x), 256, 0, s>>>(sat, rows_x, nz, nz, plane, nx);
    depth_kernel<<<g_rows, 256, 0, s>>>(sat, g, cap, mask);
    // c: table of E2, then the binary search and the words
    scan_z_bit_kernel<<<g_rows, 256, 0, s>>>(mask, nx, ny, nz, 1, sat);
    scan_strided_kernel<<<blocks_for(rows_y), 256, 0, s>>>(sat, rows_y, nz, plane, nz, ny);
    scan_strided_kernel<<<blocks_for(rows_x), 256, 0, s>>>(sat, rows_x, nz, nz, plane, nx);
    pack_kernel<<<g_rows, 256, 0, s>>>(labels, mask, sat, g, words);
    return cudaGetLastError() == cudaSuccess ? PMO_OK : PMO_ERR_CUDA;
}

}  // extern "C"
