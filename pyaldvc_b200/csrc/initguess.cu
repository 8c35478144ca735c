// The initial-guess pipeline around the NCC search, on the device:
//   block-mean downsampling        (pyALDVC solver/integer_search.py:235-244 block_downsample)
//   VOI statistics, normalisation  (io/volume_ops.py:52-121 voi_mean_std / normalize_volume with a VOI box)
//   global phase-correlation shift (solver/integer_search.py:247-291 phase_correlation_shift)
// The coarse-to-fine driver (pyramid_search) stays on the host side of the library: it chains these kernels with
// the NCC search, the median test and the inpainting, all of which run here.
#include <algorithm>

#include "common.cuh"
#include "internal.cuh"

namespace aldvc {

constexpr int IG_THREADS = 256;
constexpr int IG_PARTS = 1024;  // partial sums of the moment reductions (fixed, so the result is deterministic)
constexpr int DFT_MAX_N = 1024;

// ----------------------------------------------------------------------------- block mean
// One thread per output voxel: the FP64 sum of its factor^3 block (C order), / factor^3, rounded to float32.
__global__ void block_downsample_kernel(const float* __restrict__ in, int ny, int nx, int f, float* __restrict__ out, int oz, int oy,
                                        int ox) {
    const int64_t n = (int64_t)oz * oy * ox;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % ox);
        const int64_t r = i / ox;
        const int y = (int)(r % oy), z = (int)(r / oy);
        double s = 0.0;
        for (int a = 0; a < f; ++a)
            for (int b = 0; b < f; ++b) {
                const float* row = in + ((int64_t)(z * f + a) * ny + (y * f + b)) * nx + (int64_t)x * f;
                for (int c = 0; c < f; ++c) s += (double)__ldg(row + c);
            }
        out[i] = (float)(s / (double)(f * f * f));
    }
}

// ----------------------------------------------------------------------------- statistics over a box
struct Box {
    int64_t z0, z1, y0, y1, x0, x1;
};

// FP64 sum and sum of squares of (v - pilot) over the box, one partial per block
template <typename T>
__global__ void box_moments_kernel(const T* __restrict__ v, int64_t ny, int64_t nx, Box b, double pilot, double* part) {
    const int64_t bx = b.x1 - b.x0, by = b.y1 - b.y0, n = (b.z1 - b.z0) * by * bx;
    double s = 0.0, q = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t x = i % bx, r = i / bx, y = r % by, z = r / by;
        const double d = (double)v[((b.z0 + z) * ny + (b.y0 + y)) * nx + (b.x0 + x)] - pilot;
        s += d;
        q += d * d;
    }
    __shared__ double rs[IG_THREADS / 32], rq[IG_THREADS / 32];
    s = warp_sum_d(s);
    q = warp_sum_d(q);
    if ((threadIdx.x & 31) == 0) {
        rs[threadIdx.x >> 5] = s;
        rq[threadIdx.x >> 5] = q;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ts = 0.0, tq = 0.0;
        for (int w = 0; w < IG_THREADS / 32; ++w) {
            ts += rs[w];
            tq += rq[w];
        }
        part[2 * blockIdx.x] = ts;
        part[2 * blockIdx.x + 1] = tq;
    }
}

// stats = (mean, population std) from the partials, in a fixed order (io/volume_ops.py:88-96)
__global__ void stats_finalize_kernel(const double* part, int nparts, int64_t n, double pilot, double* stats) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double ts = 0.0, tq = 0.0;
    for (int b = 0; b < nparts; ++b) {
        ts += part[2 * b];
        tq += part[2 * b + 1];
    }
    const double ms = ts / (double)n;
    double var = tq / (double)n - ms * ms;
    var = var > 0.0 ? var : 0.0;
    stats[0] = pilot + ms;
    stats[1] = sqrt(var);
}

// (v - mean) * (1 / std) -> float32 over the whole volume, std < 1e-12 taken as 1 (io/volume_ops.py:113-120)
template <typename T>
__global__ void normalize_apply_kernel(const T* __restrict__ v, int64_t n, const double* stats, float* __restrict__ out) {
    const double m = stats[0];
    const double sd = stats[1] < 1e-12 ? 1.0 : stats[1];
    const double inv = 1.0 / sd;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)(((double)v[i] - m) * inv);
}

// ----------------------------------------------------------------------------- phase correlation
// Z = (fs - mean fs) w + i (gs - mean gs) w in FP64, the centring and the separable Hann window in float32 as the
// reference computes them: w = (w_z w_y) w_x, each factor 0.5 + 0.5 cos(pi m / (n - 1)), m = 2k - n + 1 (the
// symmetric Hann window, 1 for n = 1), rounded to float32.
__device__ __forceinline__ float hann(int k, int n) {
    return n <= 1 ? 1.0f : (float)(0.5 + 0.5 * cospi((double)(2 * k - n + 1) / (double)(n - 1)));
}

__global__ void pc_pack_kernel(const float* __restrict__ fs, const float* __restrict__ gs, int nz, int ny, int nx,
                               const double* stats_f, const double* stats_g, double2* __restrict__ z) {
    const int64_t n = (int64_t)nz * ny * nx;
    const float mf = (float)stats_f[0], mg = (float)stats_g[0];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx);
        const int64_t r = i / nx;
        const int y = (int)(r % ny), zz = (int)(r / ny);
        const float w = __fmul_rn(__fmul_rn(hann(zz, nz), hann(y, ny)), hann(x, nx));
        const float a = __fmul_rn(__fsub_rn(fs[i], mf), w), b = __fmul_rn(__fsub_rn(gs[i], mg), w);
        z[i] = make_double2((double)a, (double)b);
    }
}

// Direct DFT of every line along one axis: out[k] = sum_j in[j] exp(SIGN 2 pi i j k / n), FP64.  One CTA per line,
// the line and the n twiddles staged in shared memory, one output per thread.
template <int SIGN>
__global__ void dft_lines_kernel(const double2* __restrict__ in, double2* __restrict__ out, int n, int64_t stride, int64_t n_inner,
                                 int64_t inner_stride, int64_t outer_stride) {
    __shared__ double2 line[DFT_MAX_N], tw[DFT_MAX_N];
    const int64_t L = blockIdx.x;
    const int64_t base = (L % n_inner) * inner_stride + (L / n_inner) * outer_stride;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        line[j] = in[base + j * stride];
        double s, c;
        sincospi(2.0 * (double)j / (double)n, &s, &c);
        tw[j] = make_double2(c, SIGN * s);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double re = 0.0, im = 0.0;
        int m = 0;
        for (int j = 0; j < n; ++j) {
            const double2 a = line[j], w = tw[m];
            re += a.x * w.x - a.y * w.y;
            im += a.x * w.y + a.y * w.x;
            m += k;
            if (m >= n) m -= n;
        }
        out[base + k * stride] = make_double2(re, im);
    }
}

// Cross-power spectrum R = G conj(F) / |G conj(F)| (|.| <= 1e-12 leaves it unscaled) from the spectrum Z of
// F + iG: F[k] = (Z[k] + conj Z[-k]) / 2, G[k] = (Z[k] - conj Z[-k]) / 2i.
__global__ void pc_cross_kernel(const double2* __restrict__ Z, double2* __restrict__ R, int nz, int ny, int nx) {
    const int64_t n = (int64_t)nz * ny * nx;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx);
        const int64_t r = i / nx;
        const int y = (int)(r % ny), z = (int)(r / ny);
        const int xm = (nx - x) % nx, ym = (ny - y) % ny, zm = (nz - z) % nz;
        const double2 a = Z[i], b = Z[((int64_t)zm * ny + ym) * nx + xm];
        const double fr = 0.5 * (a.x + b.x), fi = 0.5 * (a.y - b.y);  // F
        const double gr = 0.5 * (a.y + b.y), gi = 0.5 * (b.x - a.x);  // G
        double cr = gr * fr + gi * fi, ci = gi * fr - gr * fi;        // G conj(F)
        const double mag = sqrt(cr * cr + ci * ci);
        if (mag > 1e-12) {
            cr /= mag;
            ci /= mag;
        }
        R[i] = make_double2(cr, ci);
    }
}

// first maximum (C order) of the real part: per-block partials, then one block over the partials
__device__ __forceinline__ void argmax_merge(double& bv, int64_t& bi, double v, int64_t i) {
    if (v > bv || (v == bv && i < bi)) {
        bv = v;
        bi = i;
    }
}

__device__ void argmax_block(double& bv, int64_t& bi) {
    __shared__ double sv[IG_THREADS / 32];
    __shared__ int64_t si[IG_THREADS / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
        const int64_t oi = __shfl_xor_sync(0xffffffffu, bi, o);
        argmax_merge(bv, bi, ov, oi);
    }
    if ((threadIdx.x & 31) == 0) {
        sv[threadIdx.x >> 5] = bv;
        si[threadIdx.x >> 5] = bi;
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) argmax_merge(bv, bi, sv[w], si[w]);
}

__global__ void argmax_re_kernel(const double2* __restrict__ v, int64_t n, double* pv, int64_t* pi) {
    double bv = -INFINITY;
    int64_t bi = INT64_MAX;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        argmax_merge(bv, bi, v[i].x, i);
    argmax_block(bv, bi);
    if (threadIdx.x == 0) {
        pv[blockIdx.x] = bv;
        pi[blockIdx.x] = bi;
    }
}

__global__ void argmax_final_kernel(const double* pv, const int64_t* pi, int nparts, int64_t* out) {
    double bv = -INFINITY;
    int64_t bi = INT64_MAX;
    for (int p = threadIdx.x; p < nparts; p += blockDim.x) argmax_merge(bv, bi, pv[p], pi[p]);
    argmax_block(bv, bi);
    if (threadIdx.x == 0) out[0] = bi;
}

}  // namespace aldvc

using namespace aldvc;

static int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + IG_THREADS - 1) / IG_THREADS, 148 * 8)); }

extern "C" int aldvc_block_downsample(const float* in, int64_t nz, int64_t ny, int64_t nx, int32_t factor, float* out, void* stream) {
    ALDVC_REQUIRE(in && out, "aldvc_block_downsample: null pointer");
    ALDVC_REQUIRE(factor >= 1 && factor <= 64, "aldvc_block_downsample: factor must be in [1, 64]");
    ALDVC_REQUIRE(nz >= factor && ny >= factor && nx >= factor && nz < (1 << 30) && ny < (1 << 30) && nx < (1 << 30),
                  "aldvc_block_downsample: every axis must hold at least one block");
    const int64_t oz = nz / factor, oy = ny / factor, ox = nx / factor;
    block_downsample_kernel<<<grid_for(oz * oy * ox), IG_THREADS, 0, (cudaStream_t)stream>>>(in, (int)ny, (int)nx, factor, out, (int)oz,
                                                                                             (int)oy, (int)ox);
    return check_launch("aldvc_block_downsample");
}

extern "C" size_t aldvc_stats_workspace_size(void) { return (size_t)IG_PARTS * 2 * sizeof(double); }

static int box_of(const int64_t* box, int64_t nz, int64_t ny, int64_t nx, Box& b) {
    if (box) {
        b = Box{box[0], box[1], box[2], box[3], box[4], box[5]};
    } else {
        b = Box{0, nz, 0, ny, 0, nx};
    }
    if (b.z0 < 0 || b.y0 < 0 || b.x0 < 0 || b.z1 > nz || b.y1 > ny || b.x1 > nx || b.z1 <= b.z0 || b.y1 <= b.y0 || b.x1 <= b.x0)
        return arg_fail("aldvc_volume_stats: the VOI box is empty or outside the volume");
    return ALDVC_OK;
}

static int stats_any(const void* vol, int32_t is_u16, int64_t ny, int64_t nx, const Box& b, double pilot, double* stats, void* ws,
                     size_t ws_bytes, cudaStream_t s) {
    if (ws_bytes < aldvc_stats_workspace_size()) return arg_fail("aldvc_volume_stats: workspace");
    double* part = (double*)ws;
    if (is_u16)
        box_moments_kernel<uint16_t><<<IG_PARTS, IG_THREADS, 0, s>>>((const uint16_t*)vol, ny, nx, b, pilot, part);
    else
        box_moments_kernel<float><<<IG_PARTS, IG_THREADS, 0, s>>>((const float*)vol, ny, nx, b, pilot, part);
    const int64_t n = (b.z1 - b.z0) * (b.y1 - b.y0) * (b.x1 - b.x0);
    stats_finalize_kernel<<<1, 32, 0, s>>>(part, IG_PARTS, n, pilot, stats);
    return check_launch("aldvc_volume_stats");
}

extern "C" int aldvc_volume_stats(const void* vol, int32_t is_uint16, int64_t nz, int64_t ny, int64_t nx, const int64_t* box, double pilot,
                                  double* stats, void* workspace, size_t workspace_bytes, void* stream) {
    ALDVC_REQUIRE(vol && stats && workspace, "aldvc_volume_stats: null pointer");
    ALDVC_REQUIRE(nz > 0 && ny > 0 && nx > 0, "aldvc_volume_stats: empty volume");
    Box b;
    const int rc = box_of(box, nz, ny, nx, b);
    if (rc) return rc;
    return stats_any(vol, is_uint16, ny, nx, b, pilot, stats, workspace, workspace_bytes, (cudaStream_t)stream);
}

extern "C" int aldvc_normalize_voi(const void* vol, int32_t is_uint16, int64_t nz, int64_t ny, int64_t nx, const int64_t* box, double pilot,
                                   float* out, double* stats, void* workspace, size_t workspace_bytes, void* stream) {
    ALDVC_REQUIRE(vol && out && stats && workspace, "aldvc_normalize_voi: null pointer");
    ALDVC_REQUIRE(nz > 0 && ny > 0 && nx > 0, "aldvc_normalize_voi: empty volume");
    Box b;
    int rc = box_of(box, nz, ny, nx, b);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    rc = stats_any(vol, is_uint16, ny, nx, b, pilot, stats, workspace, workspace_bytes, s);
    if (rc) return rc;
    const int64_t n = nz * ny * nx;
    if (is_uint16)
        normalize_apply_kernel<uint16_t><<<grid_for(n), IG_THREADS, 0, s>>>((const uint16_t*)vol, n, stats, out);
    else
        normalize_apply_kernel<float><<<grid_for(n), IG_THREADS, 0, s>>>((const float*)vol, n, stats, out);
    return check_launch("aldvc_normalize_voi");
}

extern "C" size_t aldvc_phase_correlation_workspace_size(int64_t nz, int64_t ny, int64_t nx) {
    return (size_t)2 * nz * ny * nx * sizeof(double2) + (size_t)IG_PARTS * (2 * sizeof(double) + sizeof(int64_t)) + 64;
}

extern "C" int aldvc_phase_correlation(const float* fs, const float* gs, int64_t nz, int64_t ny, int64_t nx, int64_t* peak, void* workspace,
                                       size_t workspace_bytes, void* stream) {
    ALDVC_REQUIRE(fs && gs && peak && workspace, "aldvc_phase_correlation: null pointer");
    ALDVC_REQUIRE(nz > 0 && ny > 0 && nx > 0 && nz <= DFT_MAX_N && ny <= DFT_MAX_N && nx <= DFT_MAX_N,
                  "aldvc_phase_correlation: every axis must be in [1, 1024] (downsample first)");
    ALDVC_REQUIRE(workspace_bytes >= aldvc_phase_correlation_workspace_size(nz, ny, nx), "aldvc_phase_correlation: workspace");
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t n = nz * ny * nx;
    double2* A = (double2*)workspace;
    double2* B = A + n;
    double* part = (double*)(B + n);
    double* pv = part;  // the moment partials are done with before the argmax reuses them
    int64_t* pi = (int64_t*)(part + 2 * IG_PARTS);
    double* stats = (double*)(pi + IG_PARTS);  // 4 doubles: mean, std of fs and of gs
    const Box b{0, nz, 0, ny, 0, nx};
    box_moments_kernel<float><<<IG_PARTS, IG_THREADS, 0, s>>>(fs, ny, nx, b, 0.0, part);
    stats_finalize_kernel<<<1, 32, 0, s>>>(part, IG_PARTS, n, 0.0, stats);
    box_moments_kernel<float><<<IG_PARTS, IG_THREADS, 0, s>>>(gs, ny, nx, b, 0.0, part);
    stats_finalize_kernel<<<1, 32, 0, s>>>(part, IG_PARTS, n, 0.0, stats + 2);
    pc_pack_kernel<<<grid_for(n), IG_THREADS, 0, s>>>(fs, gs, (int)nz, (int)ny, (int)nx, stats, stats + 2, A);
    auto dft3 = [&](const double2* src, double2* tmp, double2* dst, bool inverse) {
        // x lines (contiguous), then y, then z; each CTA one line
        auto launch = [&](const double2* i, double2* o, int len, int64_t stride, int64_t n_inner, int64_t inner_stride, int64_t outer_stride) {
            const int64_t lines = n / len;
            const int th = std::min(IG_THREADS, ((len + 31) / 32) * 32);
            if (inverse)
                dft_lines_kernel<1><<<(unsigned)lines, th, 0, s>>>(i, o, len, stride, n_inner, inner_stride, outer_stride);
            else
                dft_lines_kernel<-1><<<(unsigned)lines, th, 0, s>>>(i, o, len, stride, n_inner, inner_stride, outer_stride);
        };
        launch(src, tmp, (int)nx, 1, 1, 0, nx);             // line L = (z, y): base L * nx
        launch(tmp, dst, (int)ny, nx, nx, 1, nx * ny);      // line L = (z, x): base x + z * nx * ny
        launch(dst, tmp, (int)nz, nx * ny, nx * ny, 1, 0);  // line L = (y, x): base y * nx + x
        return tmp;
    };
    double2* spec = dft3(A, B, A, false);  // spectrum of F + iG in B
    pc_cross_kernel<<<grid_for(n), IG_THREADS, 0, s>>>(spec, A, (int)nz, (int)ny, (int)nx);
    double2* r = dft3(A, B, A, true);  // inverse (unnormalised: a positive scale leaves the argmax)
    argmax_re_kernel<<<IG_PARTS, IG_THREADS, 0, s>>>(r, n, pv, pi);
    argmax_final_kernel<<<1, IG_THREADS, 0, s>>>(pv, pi, IG_PARTS, peak);
    return check_launch("aldvc_phase_correlation");
}
