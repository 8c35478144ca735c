// Volume preprocessing on the device: whole-volume normalisation (pyALDVC io/volume_ops.py:52-121), the separable
// filters run before the local step (B-spline prefilter io/volume_ops.py:215-222, Gaussian presmoothing :200-212),
// the deformed-frame mask fill (:225-244) and the Gaussian-bead renderer of the synthetic volume pairs.
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

// mean and std of n voxels from their sums of (v - pilot) and (v - pilot)^2 (io/volume_ops.py:92-96; std < 1e-12 -> 1)
__device__ __forceinline__ void stats_from_sums(double ts, double tq, int64_t n, double pilot, double& mean, double& sd) {
    const double ms = ts / (double)n;
    double var = tq / (double)n - ms * ms;
    var = var > 0.0 ? var : 0.0;
    sd = sqrt(var);
    if (sd < 1e-12) sd = 1.0;
    mean = pilot + ms;
}

// mean/std from the partials (single thread, fixed order) or, with part == NULL, from accumulated sums[2], then
// (v - mean) * (1/std) -> float32
template <typename T>
__global__ void normalize_kernel(const T* __restrict__ v, int64_t n, double pilot, const double* part, int nparts, float* out,
                                 double* stats, const double* sums = nullptr, int64_t n_total = 0) {
    __shared__ double s_mean, s_inv;
    if (threadIdx.x == 0) {
        double ts = 0.0, tq = 0.0, mean, sd;
        if (sums) {
            ts = sums[0];
            tq = sums[1];
        } else {
            for (int b = 0; b < nparts; ++b) {
                ts += part[2 * b];
                tq += part[2 * b + 1];
            }
        }
        stats_from_sums(ts, tq, sums ? n_total : n, pilot, mean, sd);
        s_mean = mean;
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

// sums[0..1] += the partials, in block order (one thread): a volume streamed slab by slab accumulates its moments
__global__ void moments_add_kernel(const double* part, int nparts, double* sums) {
    double ts = 0.0, tq = 0.0;
    for (int b = 0; b < nparts; ++b) {
        ts += part[2 * b];
        tq += part[2 * b + 1];
    }
    sums[0] += ts;
    sums[1] += tq;
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

// ----------------------------------------------------------------------------- separable symmetric filter
// out[k] = w[0] s[k] + sum_{j=1..J} w[j] (s[k-j] + s[k+j]) along one axis, FP64 products and sums in that order
// (no contraction into fused multiply-adds), float32 out.  Boundary 0 "mirror" (period 2n - 2, edge sample not
// repeated), 1 "nearest" (edge sample repeated).  The B-spline prefilter is this filter with w[j] = sqrt(3) z^j,
// z = sqrt(3) - 2, J = 32, mirror; the Gaussian presmoothing is the normalised Gaussian with nearest.
//
// A CTA filters a tile of SEP_COLS lines x SEP_LEN outputs; the tile's samples, halo included, are staged once in
// shared memory, so every input is read from HBM about (SEP_LEN + 2J) / SEP_LEN times and every output written
// once.  For the x axis lanes run along the line (rows of the tile contiguous); for y and z lanes run across 32
// neighbouring x columns, so every global access is a 128-byte row.
constexpr int SEP_MAX_HALF = 63;
constexpr int SEP_COLS = 32;
constexpr int SEP_LEN = 192;
constexpr int SEP_THREADS = 256;
constexpr int SEP_SMEM_FLOATS = (SEP_LEN + 2 * SEP_MAX_HALF) * SEP_COLS;  // 40,704 bytes

struct SepTaps {
    double w[SEP_MAX_HALF + 1];
};

__device__ __forceinline__ int64_t sep_reflect(int64_t k, int64_t n, int boundary) {
    if (boundary == 1) return k < 0 ? 0 : (k >= n ? n - 1 : k);
    if (n == 1) return 0;
    const int64_t p = 2 * n - 2;
    k %= p;
    if (k < 0) k += p;
    return k < n ? k : p - k;
}

__device__ __forceinline__ float sep_apply(const float* t, int step, const SepTaps& w, int J) {
    double acc = __dmul_rn(w.w[0], (double)t[0]);
    for (int j = 1; j <= J; ++j) acc = __dadd_rn(acc, __dmul_rn(w.w[j], __dadd_rn((double)t[-j * step], (double)t[j * step])));
    return (float)acc;
}

// filter axis x: tile rows are 32 consecutive y of one z plane
__global__ void __launch_bounds__(SEP_THREADS) sep_filter_x_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                                   int nz, int ny, int nx, SepTaps w, int J, int boundary) {
    __shared__ float tile[SEP_SMEM_FLOATS];
    const int A = SEP_LEN + 2 * J;
    const int x0 = blockIdx.x * SEP_LEN, y0 = blockIdx.y * SEP_COLS, z = blockIdx.z;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r = warp; r < SEP_COLS; r += SEP_THREADS / 32) {
        const int y = y0 + r;
        if (y >= ny) break;
        const float* row = in + ((int64_t)z * ny + y) * nx;
        for (int a = lane; a < A; a += 32) tile[r * A + a] = __ldg(row + sep_reflect((int64_t)x0 - J + a, nx, boundary));
    }
    __syncthreads();
    for (int r = warp; r < SEP_COLS; r += SEP_THREADS / 32) {
        const int y = y0 + r;
        if (y >= ny) break;
        float* orow = out + ((int64_t)z * ny + y) * nx;
        for (int o = lane; o < SEP_LEN && x0 + o < nx; o += 32) orow[x0 + o] = sep_apply(tile + r * A + o + J, 1, w, J);
    }
}

// filter axis y (AXIS 1) or z (AXIS 2): tile columns are 32 consecutive x
template <int AXIS>
__global__ void __launch_bounds__(SEP_THREADS) sep_filter_yz_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                                    int nz, int ny, int nx, SepTaps w, int J, int boundary) {
    __shared__ float tile[SEP_SMEM_FLOATS];
    const int A = SEP_LEN + 2 * J;
    const int n = AXIS == 1 ? ny : nz;
    const int64_t stride = AXIS == 1 ? (int64_t)nx : (int64_t)nx * ny;
    const int x0 = blockIdx.x * SEP_COLS, k0 = blockIdx.y * SEP_LEN;
    const int64_t base = AXIS == 1 ? (int64_t)blockIdx.z * ny * nx : (int64_t)blockIdx.z * nx;  // plane z, or row y
    const int c = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const bool col_ok = x0 + c < nx;
    for (int a = ty; a < A; a += SEP_THREADS / 32)
        tile[a * SEP_COLS + c] = col_ok ? __ldg(in + base + sep_reflect((int64_t)k0 - J + a, n, boundary) * stride + x0 + c) : 0.0f;
    __syncthreads();
    if (!col_ok) return;
    for (int o = ty; o < SEP_LEN && k0 + o < n; o += SEP_THREADS / 32)
        out[base + (int64_t)(k0 + o) * stride + x0 + c] = sep_apply(tile + (o + J) * SEP_COLS + c, SEP_COLS, w, J);
}

// deformed-frame mask (io/volume_ops.py:238-243 and the NCC input of core/pipeline.py:260-262): value where mask == 0
__global__ void mask_fill_kernel(float* __restrict__ v, const uint8_t* __restrict__ mask, int64_t n, float value) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (mask[i] == 0) v[i] = value;
}

// q[i] = (v[i], v[i+1], v[i+2], v[i+3]), indices clamped to the last voxel
__global__ void make_quads_kernel(const float* __restrict__ v, int64_t n, float4* __restrict__ q) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t l = n - 1;
        q[i] = make_float4(__ldg(v + i), __ldg(v + (i + 1 < l ? i + 1 : l)), __ldg(v + (i + 2 < l ? i + 2 : l)),
                           __ldg(v + (i + 3 < l ? i + 3 : l)));
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

extern "C" int aldvc_volume_moments(const void* vol, int32_t is_uint16, int64_t n_voxels, double pilot, double* sums, void* workspace,
                                    size_t workspace_bytes, void* stream) {
    ALDVC_REQUIRE(vol && sums && workspace, "aldvc_volume_moments: null pointer");
    ALDVC_REQUIRE(n_voxels > 0, "aldvc_volume_moments: empty array");
    const int parts = 1024;
    if (workspace_bytes < (size_t)parts * 2 * sizeof(double)) return arg_fail("aldvc_volume_moments: workspace");
    cudaStream_t s = (cudaStream_t)stream;
    double* part = (double*)workspace;
    if (is_uint16)
        moments_kernel<uint16_t><<<parts, VOL_THREADS, 0, s>>>((const uint16_t*)vol, n_voxels, pilot, part);
    else
        moments_kernel<float><<<parts, VOL_THREADS, 0, s>>>((const float*)vol, n_voxels, pilot, part);
    moments_add_kernel<<<1, 1, 0, s>>>(part, parts, sums);
    return check_launch("aldvc_volume_moments");
}

extern "C" int aldvc_normalize_sums(const void* vol, int32_t is_uint16, int64_t n_voxels, const double* sums, int64_t n_total,
                                    double pilot, float* out, double* stats, void* stream) {
    ALDVC_REQUIRE(vol && sums && out, "aldvc_normalize_sums: null pointer");
    ALDVC_REQUIRE(n_voxels > 0 && n_total > 0, "aldvc_normalize_sums: empty array");
    cudaStream_t s = (cudaStream_t)stream;
    const int blocks = (int)std::min<int64_t>(1024, (n_voxels + VOL_THREADS - 1) / VOL_THREADS);
    if (is_uint16)
        normalize_kernel<uint16_t><<<blocks, VOL_THREADS, 0, s>>>((const uint16_t*)vol, n_voxels, pilot, nullptr, 0, out, stats, sums,
                                                                  n_total);
    else
        normalize_kernel<float><<<blocks, VOL_THREADS, 0, s>>>((const float*)vol, n_voxels, pilot, nullptr, 0, out, stats, sums, n_total);
    return check_launch("aldvc_normalize_sums");
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

extern "C" int aldvc_sep_filter(const float* in, float* out, int64_t nz, int64_t ny, int64_t nx, int32_t axis, const double* weights,
                                int32_t half_taps, int32_t boundary, void* stream) {
    ALDVC_REQUIRE(in && out && weights, "aldvc_sep_filter: null pointer");
    ALDVC_REQUIRE(in != out, "aldvc_sep_filter: in and out must be different buffers");
    ALDVC_REQUIRE(axis >= 0 && axis <= 2, "aldvc_sep_filter: axis must be 0 (x), 1 (y) or 2 (z)");
    ALDVC_REQUIRE(half_taps >= 0 && half_taps <= SEP_MAX_HALF, "aldvc_sep_filter: half_taps must be in [0, 63]");
    ALDVC_REQUIRE(boundary == 0 || boundary == 1, "aldvc_sep_filter: boundary must be 0 (mirror) or 1 (nearest)");
    ALDVC_REQUIRE(nz > 0 && ny > 0 && nx > 0 && nz <= 65535 && ny <= 65535 && nx < (1 << 30), "aldvc_sep_filter: shape");
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t n = axis == 0 ? nx : (axis == 1 ? ny : nz);
    if (boundary == 0 && n == 1) {  // a mirrored line of one sample is its own coefficient
        cudaError_t e = cudaMemcpyAsync(out, in, (size_t)(nz * ny * nx) * sizeof(float), cudaMemcpyDeviceToDevice, s);
        return e == cudaSuccess ? ALDVC_OK : cuda_fail(e, "aldvc_sep_filter: copy");
    }
    SepTaps w{};
    for (int j = 0; j <= half_taps; ++j) w.w[j] = weights[j];
    const int Z = (int)nz, Y = (int)ny, X = (int)nx;
    KTimer kt_("sep_filter", s);
    if (axis == 0) {
        dim3 grid((unsigned)((nx + SEP_LEN - 1) / SEP_LEN), (unsigned)((ny + SEP_COLS - 1) / SEP_COLS), (unsigned)nz);
        sep_filter_x_kernel<<<grid, SEP_THREADS, 0, s>>>(in, out, Z, Y, X, w, half_taps, boundary);
    } else if (axis == 1) {
        dim3 grid((unsigned)((nx + SEP_COLS - 1) / SEP_COLS), (unsigned)((ny + SEP_LEN - 1) / SEP_LEN), (unsigned)nz);
        sep_filter_yz_kernel<1><<<grid, SEP_THREADS, 0, s>>>(in, out, Z, Y, X, w, half_taps, boundary);
    } else {
        dim3 grid((unsigned)((nx + SEP_COLS - 1) / SEP_COLS), (unsigned)((nz + SEP_LEN - 1) / SEP_LEN), (unsigned)ny);
        sep_filter_yz_kernel<2><<<grid, SEP_THREADS, 0, s>>>(in, out, Z, Y, X, w, half_taps, boundary);
    }
    return check_launch("aldvc_sep_filter");
}

extern "C" int aldvc_mask_fill(float* vol, const uint8_t* mask, int64_t n_voxels, float value, void* stream) {
    ALDVC_REQUIRE(vol && mask, "aldvc_mask_fill: null pointer");
    if (n_voxels <= 0) return ALDVC_OK;
    const int64_t blocks = std::min<int64_t>((n_voxels + 255) / 256, 148 * 16);
    mask_fill_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(vol, mask, n_voxels, value);
    return check_launch("aldvc_mask_fill");
}

extern "C" int aldvc_make_quads(const float* vol, int64_t n_voxels, float* quads, void* stream) {
    ALDVC_REQUIRE(vol && quads, "aldvc_make_quads: null pointer");
    ALDVC_REQUIRE((reinterpret_cast<uintptr_t>(quads) & 15) == 0, "aldvc_make_quads: quads must be 16-byte aligned");
    if (n_voxels <= 0) return ALDVC_OK;
    const int64_t blocks = std::min<int64_t>((n_voxels + 255) / 256, 148 * 16);
    make_quads_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(vol, n_voxels, reinterpret_cast<float4*>(quads));
    return check_launch("aldvc_make_quads");
}
