// voxel_words.cu — the uniform-box map the transport kernel steps on.
//
// For every voxel v the word holds label(v) in the low byte and, in the high
// byte, R(v) = the Chebyshev distance (in voxels) from v to the nearest voxel
// with a different label, capped at cap + 1.  Every voxel u with
// |u - v|_inf <= R(v) - 1 then carries label(v), so a photon in v may treat the
// cube of half-width (R(v) - 1/2) voxels around v's centre as one cell: it
// meets no label change, hence no index step and no change of mu, before that
// cube's faces.  Crossing a face between two voxels of one label changes
// nothing in the reference's transport (pymopt/voxel_gpu/_cukernel.py:154-167),
// so stepping cube to cube follows the same path as stepping voxel to voxel.
//
// R is computed as 1 + the L-infinity distance transform of the edge set E
// (voxels with a 26-neighbour of another label): if the nearest different
// label is at distance R, the voxel next to it on the way is in E at distance
// R - 1, and no voxel of E is closer.  The transform is separable:
// d(v) = min over |k| <= cap of max(|k|, d_prev(v + k e_axis)), one pass per
// axis, the first pass starting from 0 on E and "infinity" elsewhere.
#include "pmo_internal.h"

namespace {

constexpr uint8_t kInf = 255;

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

__global__ void pack_kernel(const uint8_t *__restrict__ lab, const uint8_t *__restrict__ d,
                            uint64_t total, int cap, uint16_t *__restrict__ words) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const int dist = d[i] < cap ? d[i] : cap;
        words[i] = (uint16_t)(lab[i] | ((dist + 1) << 8));
    }
}

}  // namespace

extern "C" {

// words[nvox] (uint16) from labels[nvox]; scratch: 2 * nvox bytes.
int pmo_build_voxel_words(const uint8_t *labels, int nx, int ny, int nz, int cap,
                          uint16_t *words, void *scratch, size_t scratch_bytes, void *stream) {
    if (!labels || !words || !scratch || nx < 1 || ny < 1 || nz < 1) return PMO_ERR_ARG;
    if (cap < 0 || cap > 200) return PMO_ERR_ARG;
    const uint64_t total = (uint64_t)nx * ny * nz;
    if (scratch_bytes < 2 * total) return PMO_ERR_WORKSPACE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint8_t *a = static_cast<uint8_t *>(scratch);
    uint8_t *b = a + total;
    uint64_t blocks = (total + 255) / 256;
    if (blocks > 148ull * 64) blocks = 148ull * 64;
    edge_kernel<<<(unsigned)blocks, 256, 0, s>>>(labels, nx, ny, nz, a);
    dt_pass_kernel<<<(unsigned)blocks, 256, 0, s>>>(a, nx, ny, nz, 0, cap, b);
    dt_pass_kernel<<<(unsigned)blocks, 256, 0, s>>>(b, nx, ny, nz, 1, cap, a);
    dt_pass_kernel<<<(unsigned)blocks, 256, 0, s>>>(a, nx, ny, nz, 2, cap, b);
    pack_kernel<<<(unsigned)blocks, 256, 0, s>>>(labels, b, total, cap, words);
    return cudaGetLastError() == cudaSuccess ? PMO_OK : PMO_ERR_CUDA;
}

}  // extern "C"
