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
// closer than D_E(v).  The transform is separable:
// D(v) = min over |k| <= cap of max(|k|, D_prev(v + k e_axis)), one pass per
// axis, the first pass starting from 0 on E and "infinity" elsewhere.
//
// e: P(u), the same construction inside u's z-plane with the 8 in-plane
// neighbours and the lateral border (two passes, x and y, capped at 192), is
// the half-extent of a uniform in-plane square around u.  The box's slices
// are the squares around v + dz*z_hat for |dz| <= d, which lie in v's cube and
// so carry label(v).  Hence e_true = min over |dz| <= d of P(v + dz*z_hat), and
// e_true >= d.  The word stores the largest code with lat(c) <= e_true.  This
// widens the boxes of thin layers, such as a 2-voxel skin layer whose voxels
// all have d = 0.
#include "pmo_internal.h"

namespace {

constexpr uint8_t kInf = 255;
constexpr int kLatCap = 192;   // lat(15)

__host__ __device__ inline int lat_of(int c) {
    return c ? ((2 | (c & 1)) << (c >> 1)) >> 1 : 0;
}

// E: 0 where a 26-neighbour (inside the array) has another label, else kInf.
__global__ void edge_kernel(const uint8_t *__restrict__ lab, int nx, int ny, int nz,
                            uint8_t *__restrict__ out) {
    const uint64_t total = (uint64_t)nx * ny * nz;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const int z = (int)(i % nz);
        const int y = (int)((i / nz) % ny);
        const int x = (int)(i / ((uint64_t)nz * ny));
        const uint8_t me = lab[i];
        bool edge = false;
        for (int dx = -1; dx <= 1 && !edge; ++dx) {
            const int xx = x + dx;
            if (xx < 0 || xx >= nx) continue;
            for (int dy = -1; dy <= 1 && !edge; ++dy) {
                const int yy = y + dy;
                if (yy < 0 || yy >= ny) continue;
                const uint64_t row = ((uint64_t)xx * ny + yy) * nz;
                for (int dz = -1; dz <= 1; ++dz) {
                    const int zz = z + dz;
                    if (zz < 0 || zz >= nz) continue;
                    if (lab[row + zz] != me) { edge = true; break; }
                }
            }
        }
        // the array border counts as an edge: boxes never reach past it
        if (x == 0 || y == 0 || z == 0 || x == nx - 1 || y == ny - 1 || z == nz - 1) edge = true;
        out[i] = edge ? 0 : kInf;
    }
}

// E2: 0 where an in-plane 8-neighbour has another label, or on the lateral
// array border; else kInf.
__global__ void edge2_kernel(const uint8_t *__restrict__ lab, int nx, int ny, int nz,
                             uint8_t *__restrict__ out) {
    const uint64_t total = (uint64_t)nx * ny * nz;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const int z = (int)(i % nz);
        const int y = (int)((i / nz) % ny);
        const int x = (int)(i / ((uint64_t)nz * ny));
        const uint8_t me = lab[i];
        bool edge = x == 0 || y == 0 || x == nx - 1 || y == ny - 1;
        for (int dx = -1; dx <= 1 && !edge; ++dx) {
            for (int dy = -1; dy <= 1; ++dy) {
                if (lab[((uint64_t)(x + dx) * ny + (y + dy)) * nz + z] != me) {
                    edge = true;
                    break;
                }
            }
        }
        out[i] = edge ? 0 : kInf;
    }
}

// One separable pass of the L-infinity distance transform along `axis`.
__global__ void dt_pass_kernel(const uint8_t *__restrict__ in, int nx, int ny, int nz, int axis,
                               int cap, uint8_t *__restrict__ out) {
    const uint64_t total = (uint64_t)nx * ny * nz;
    const int dim = axis == 0 ? nx : (axis == 1 ? ny : nz);
    const uint64_t stride = axis == 0 ? (uint64_t)ny * nz : (axis == 1 ? (uint64_t)nz : 1);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const int c = axis == 0 ? (int)(i / ((uint64_t)nz * ny))
                                : (axis == 1 ? (int)((i / nz) % ny) : (int)(i % nz));
        int best = in[i];
        for (int k = 1; k <= cap && k < best; ++k) {
            if (c - k >= 0) {
                const int v = in[i - k * stride];
                const int m = v > k ? v : k;
                if (m < best) best = m;
            }
            if (c + k < dim) {
                const int v = in[i + k * stride];
                const int m = v > k ? v : k;
                if (m < best) best = m;
            }
        }
        out[i] = (uint8_t)best;
    }
}

// words from the labels, the cube half-extent map dmap and the in-plane
// radius map pmap
__global__ void pack_kernel(const uint8_t *__restrict__ lab, const uint8_t *__restrict__ dmap,
                            const uint8_t *__restrict__ pmap, int nz, uint64_t total, int cap,
                            uint16_t *__restrict__ words) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const int z = (int)(i % nz);
        const int d = dmap[i] < cap ? dmap[i] : cap;
        int e = kLatCap;
        for (int dz = -d; dz <= d; ++dz) {
            const int zz = z + dz;
            if (zz < 0 || zz >= nz) { e = 0; break; }   // never with a valid d
            const int p = pmap[(int64_t)i + dz];
            if (p < e) e = p;
        }
        int c = 0;
        while (c < 15 && lat_of(c + 1) <= e) ++c;
        words[i] = (uint16_t)(lab[i] | (d << 8) | (c << 12));
    }
}

}  // namespace

extern "C" {

// words[nvox] (uint16) from labels[nvox]; scratch: 3 * nvox bytes.
int pmo_build_voxel_words(const uint8_t *labels, int nx, int ny, int nz, int cap,
                          uint16_t *words, void *scratch, size_t scratch_bytes, void *stream) {
    if (!labels || !words || !scratch || nx < 1 || ny < 1 || nz < 1) return PMO_ERR_ARG;
    if (cap < 0 || cap > 15) return PMO_ERR_ARG;
    const uint64_t total = (uint64_t)nx * ny * nz;
    if (scratch_bytes < 3 * total) return PMO_ERR_WORKSPACE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint8_t *a = static_cast<uint8_t *>(scratch);
    uint8_t *b = a + total;
    uint8_t *c = b + total;
    uint64_t blocks = (total + 255) / 256;
    if (blocks > 148ull * 64) blocks = 148ull * 64;
    const unsigned g = (unsigned)blocks;
    // d: 3-D distance to the edge set, capped
    edge_kernel<<<g, 256, 0, s>>>(labels, nx, ny, nz, a);
    dt_pass_kernel<<<g, 256, 0, s>>>(a, nx, ny, nz, 0, cap, b);
    dt_pass_kernel<<<g, 256, 0, s>>>(b, nx, ny, nz, 1, cap, a);
    dt_pass_kernel<<<g, 256, 0, s>>>(a, nx, ny, nz, 2, cap, b);
    // P: in-plane distance to the in-plane edge set, capped at lat(15)
    edge2_kernel<<<g, 256, 0, s>>>(labels, nx, ny, nz, a);
    dt_pass_kernel<<<g, 256, 0, s>>>(a, nx, ny, nz, 0, kLatCap, c);
    dt_pass_kernel<<<g, 256, 0, s>>>(c, nx, ny, nz, 1, kLatCap, a);
    pack_kernel<<<g, 256, 0, s>>>(labels, b, a, nz, total, cap, words);
    return cudaGetLastError() == cudaSuccess ? PMO_OK : PMO_ERR_CUDA;
}

}  // extern "C"
