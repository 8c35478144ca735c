// Volume preprocessing on the device: whole-volume normalisation (pyALDVC io/volume_ops.py:52-121) and the
// Gaussian-bead renderer of the synthetic volume pairs.
#include <algorithm>

#include "common.cuh"
#include "internal.cuh"

namespace aldvc {

constexpr int VOL_THREADS = 256;

// FP64 sum and sum of squares of (v - pilot), one partial per block (deterministic for a fixed grid).
template <typename T>
__global__ void moments_kernel(const T* __restrict__ v, int64_t n, double pilot, double* part) {
    double s = 0.0, q = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double d = (double)v[i] - pilot;
        s += d;
        q += d * d;
    }
    __shared__ double rs[VOL_THREADS / 32], rq[VOL_THREADS / 32];
    s = warp_sum_d(s);
    q = warp_sum_d(q);
    if ((threadIdx.x & 31) == 0) {
        rs[threadIdx.x >> 5] = s;
        rq[threadIdx.x >> 5] = q;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ts = 0.0, tq = 0.0;
        for (int w = 0; w < VOL_THREADS / 32; ++w) {
            ts += rs[w];
            tq += rq[w];
        }
        part[2 * blockIdx.x] = ts;
        part[2 * blockIdx.x + 1] = tq;
    }
}

// mean/std from the partials (single thread, fixed order), then (v - mean) * (1/std) -> float32
template <typename T>
__global__ void normalize_kernel(const T* __restrict__ v, int64_t n, double pilot, const double* part, int nparts, float* out,
                                 double* stats) {
    __shared__ double s_mean, s_inv;
    if (threadIdx.x == 0) {
        double ts = 0.0, tq = 0.0;
        for (int b = 0; b < nparts; ++b) {
            ts += part[2 * b];
            tq += part[2 * b + 1];
        }
        const double ms = ts / (double)n;
        double var = tq / (double)n - ms * ms;
        var = var > 0.0 ? var : 0.0;
        double sd = sqrt(var);
        if (sd < 1e-12) sd = 1.0;
        s_mean = pilot + ms;
        s_inv = 1.0 / sd;
        if (blockIdx.x == 0 && stats) {
            stats[0] = s_mean;
            stats[1] = sd;
        }
    }
    __syncthreads();
    const double m = s_mean, inv = s_inv;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)(((double)v[i] - m) * inv);
}

// One block per bead: peak * exp(-|x - c|^2 / (2 sigma^2)) over the (2R+1)^3 voxels around the bead,
// accumulated in FP64 (the rounding to float32 afterwards hides the order of the atomic sums).
__global__ void render_beads_kernel(double* acc, int nz, int ny, int nx, const double* centres, const double* peaks, int64_t nbeads,
                                    double inv2s2, int R) {
    const int64_t b = blockIdx.x;
    if (b >= nbeads) return;
    const double cz = centres[3 * b], cy = centres[3 * b + 1], cx = centres[3 * b + 2];
    const double pk = peaks[b];
    const int bz = (int)floor(cz), by = (int)floor(cy), bx = (int)floor(cx);
    const int K = 2 * R + 1;
    const int total = K * K * K;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        const int kz = t / (K * K), r = t - kz * K * K, ky = r / K, kx = r - ky * K;
        const int z = bz - R + kz, y = by - R + ky, x = bx - R + kx;
        if (z < 0 || y < 0 || x < 0 || z >= nz || y >= ny || x >= nx) continue;
        const double dz = z - cz, dy = y - cy, dx = x - cx;
        const double w = pk * exp(-dz * dz * inv2s2) * exp(-dy * dy * inv2s2) * exp(-dx * dx * inv2s2);
        atomicAdd(acc + ((int64_t)z * ny + y) * nx + x, w);
    }
}

}  // namespace aldvc

using namespace aldvc;

static int normalize_any(const void* v, int is_u16, int64_t n, double pilot, float* out, double* stats, void* workspace,
                         size_t workspace_bytes, cudaStream_t s) {
    const int parts = 1024;
    if (workspace_bytes < (size_t)parts * 2 * sizeof(double)) return arg_fail("aldvc_normalize: workspace");
    double* part = (double*)workspace;
    if (is_u16) {
        moments_kernel<uint16_t><<<parts, VOL_THREADS, 0, s>>>((const uint16_t*)v, n, pilot, part);
        normalize_kernel<uint16_t><<<parts, VOL_THREADS, 0, s>>>((const uint16_t*)v, n, pilot, part, parts, out, stats);
    } else {
        moments_kernel<float><<<parts, VOL_THREADS, 0, s>>>((const float*)v, n, pilot, part);
        normalize_kernel<float><<<parts, VOL_THREADS, 0, s>>>((const float*)v, n, pilot, part, parts, out, stats);
    }
    return check_launch("aldvc_normalize");
}

extern "C" size_t aldvc_normalize_workspace_size(void) { return 1024 * 2 * sizeof(double); }

extern "C" int aldvc_normalize(const void* vol, int32_t is_uint16, int64_t n_voxels, double pilot, float* out, double* stats,
                               void* workspace, size_t workspace_bytes, void* stream) {
    ALDVC_REQUIRE(vol && out && workspace, "aldvc_normalize: null pointer");
    ALDVC_REQUIRE(n_voxels > 0, "aldvc_normalize: empty volume");
    return normalize_any(vol, is_uint16, n_voxels, pilot, out, stats, workspace, workspace_bytes, (cudaStream_t)stream);
}

extern "C" int aldvc_render_beads(double* accum, int64_t nz, int64_t ny, int64_t nx, const double* centres_zyx, const double* peaks,
                                  int64_t n_beads, double sigma, int32_t radius, void* stream) {
    ALDVC_REQUIRE(accum && centres_zyx && peaks, "aldvc_render_beads: null pointer");
    ALDVC_REQUIRE(sigma > 0.0 && radius >= 0 && radius <= 64, "aldvc_render_beads: bad sigma/radius");
    ALDVC_REQUIRE(nz > 0 && ny > 0 && nx > 0 && nz < (1 << 30) && ny < (1 << 30) && nx < (1 << 30), "aldvc_render_beads: shape");
    if (n_beads <= 0) return ALDVC_OK;
    ALDVC_REQUIRE(n_beads < (1LL << 31), "aldvc_render_beads: too many beads");
    render_beads_kernel<<<(unsigned)n_beads, 256, 0, (cudaStream_t)stream>>>(accum, (int)nz, (int)ny, (int)nx, centres_zyx, peaks,
                                                                               n_beads, 1.0 / (2.0 * sigma * sigma), radius);
    return check_launch("aldvc_render_beads");
}
