// Shared device code of the AL-DVC hot-path kernels (sm_100a).
//
// Conventions follow pyALDVC (src/al_dvc/solver/numba_kernels.py:9-17):
//   volumes are (nz, ny, nx) float32 C order; node coordinates int64 [x, y, z];
//   P[0:9] = F row-major (F_ij = du_i/dx_j), P[9:12] = (u, v, w);
//   x_def = x0 + u + (I + F)(x - x0).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/aldvc_b200.h"

namespace aldvc {

constexpr int ST_CONVERGED = 0;
constexpr int ST_MAX_ITER = 1;
constexpr int ST_OOB = 2;
constexpr int ST_INVALID = 3;
constexpr int ST_SINGULAR = 4;
constexpr int ST_NAN = 5;
constexpr int ST_SKIPPED = 6;
constexpr int ST_STALLED = 7;

// numba_kernels.py:38-44, 81-85
constexpr double ABS_TOL = 1e-5;
constexpr double STALL_ZNCC_EPS = 1e-4;
constexpr double STALL_STEP_DECAY = 0.999;
constexpr int MIN_SUBSET_VOXELS = 27;
constexpr double MIN_VALID_FRACTION = 0.5;
constexpr double LM_DAMPING_3DOF = 1e-3;
constexpr double MIN_CORRECTED_FRACTION = 0.5;
constexpr double NOISE_CORR_STEP = 0.5;
constexpr double PREDICT_CONTRACTION = 0.5;

__host__ __device__ inline int64_t subset_count(int hx, int hy, int hz, int stride) {
    return (int64_t)((2 * hx) / stride + 1) * ((2 * hy) / stride + 1) * ((2 * hz) / stride + 1);
}

__device__ __forceinline__ bool kept_bit(const uint8_t* keep, int64_t idx) {
    return ((keep[idx >> 3] >> (idx & 7)) & 1) != 0;
}

// interp_kernels.interp_margin_ok (:127-136), evaluated in FP64 like the reference
__device__ __forceinline__ bool margin_ok(double z, double y, double x, int nz, int ny, int nx) {
    if (x < 1.0 || x > (double)nx - 3.0) return false;
    if (y < 1.0 || y > (double)ny - 3.0) return false;
    if (z < 1.0 || z > (double)nz - 3.0) return false;
    return true;
}

// Catmull-Rom (Keys a = -0.5) and cubic B-spline weights for taps -1..2 (interp_kernels.py:34-53), FP32
__device__ __forceinline__ void keys_w(float t, float& w0, float& w1, float& w2, float& w3) {
    w0 = ((-0.5f * t + 1.0f) * t - 0.5f) * t;
    w1 = (1.5f * t - 2.5f) * t * t + 1.0f;
    w2 = ((-1.5f * t + 2.0f) * t + 0.5f) * t;
    w3 = (0.5f * t - 0.5f) * t * t;
}

__device__ __forceinline__ void bspl_w(float t, float& w0, float& w1, float& w2, float& w3) {
    const float t2 = t * t, t3 = t2 * t;
    const float s = 1.0f / 6.0f;
    w0 = (1.0f - 3.0f * t + 3.0f * t2 - t3) * s;
    w1 = (4.0f - 6.0f * t2 + 3.0f * t3) * s;
    w2 = (1.0f + 3.0f * t + 3.0f * t2 - 3.0f * t3) * s;
    w3 = t3 * s;
}

// Sample a dense float brick (pitch bx, plane bx*by) at a position relative to its origin.
// (ix, iy, iz) = floor of the position, already clamped so every tap is inside the brick.
template <int MODE>
__device__ __forceinline__ float sample_brick(const float* __restrict__ b, int bx, int bxy, int ix, int iy, int iz, float fx,
                                              float fy, float fz) {
    if (MODE == 0) {
        const float* p = b + ((int64_t)iz * bxy + (int64_t)iy * bx + ix);
        const float c00 = p[0] * (1.0f - fx) + p[1] * fx;
        const float c10 = p[bx] * (1.0f - fx) + p[bx + 1] * fx;
        const float c01 = p[bxy] * (1.0f - fx) + p[bxy + 1] * fx;
        const float c11 = p[bxy + bx] * (1.0f - fx) + p[bxy + bx + 1] * fx;
        const float c0 = c00 * (1.0f - fy) + c10 * fy;
        const float c1 = c01 * (1.0f - fy) + c11 * fy;
        return c0 * (1.0f - fz) + c1 * fz;
    }
    float wx0, wx1, wx2, wx3, wy0, wy1, wy2, wy3, wz0, wz1, wz2, wz3;
    if (MODE == 1) {
        keys_w(fx, wx0, wx1, wx2, wx3);
        keys_w(fy, wy0, wy1, wy2, wy3);
        keys_w(fz, wz0, wz1, wz2, wz3);
    } else {
        bspl_w(fx, wx0, wx1, wx2, wx3);
        bspl_w(fy, wy0, wy1, wy2, wy3);
        bspl_w(fz, wz0, wz1, wz2, wz3);
    }
    const float* p = b + ((int64_t)(iz - 1) * bxy + (int64_t)(iy - 1) * bx + (ix - 1));
    float acc = 0.0f;
    const float wz[4] = {wz0, wz1, wz2, wz3};
    const float wy[4] = {wy0, wy1, wy2, wy3};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        float pl = 0.0f;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float* r = p + (int64_t)k * bxy + j * bx;
            const float row = r[0] * wx0 + r[1] * wx1 + r[2] * wx2 + r[3] * wx3;
            pl += row * wy[j];
        }
        acc += pl * wz[k];
    }
    return acc;
}

// sample_brick over the overlapping-quad copy of the volume (q[i] = b[i..i+3]): each of the 16 tap rows of a cubic
// sample is one 16-byte load; the same products and sums in the same order as sample_brick<MODE>.
// I32: every tap index below 2^31 (the caller checks the volume), so each load takes a 32-bit index.
template <int MODE, bool I32 = false>
__device__ __forceinline__ float sample_quad(const float4* __restrict__ q, int bx, int bxy, int ix, int iy, int iz, float fx,
                                             float fy, float fz) {
    float wx0, wx1, wx2, wx3, wy0, wy1, wy2, wy3, wz0, wz1, wz2, wz3;
    if (MODE == 1) {
        keys_w(fx, wx0, wx1, wx2, wx3);
        keys_w(fy, wy0, wy1, wy2, wy3);
        keys_w(fz, wz0, wz1, wz2, wz3);
    } else {
        bspl_w(fx, wx0, wx1, wx2, wx3);
        bspl_w(fy, wy0, wy1, wy2, wy3);
        bspl_w(fz, wz0, wz1, wz2, wz3);
    }
    const float4* p = q + ((int64_t)(iz - 1) * bxy + (int64_t)(iy - 1) * bx + (ix - 1));
    const int i0 = (iz - 1) * bxy + (iy - 1) * bx + (ix - 1);  // used when I32
    float acc = 0.0f;
    const float wz[4] = {wz0, wz1, wz2, wz3};
    const float wy[4] = {wy0, wy1, wy2, wy3};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        float pl = 0.0f;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float4 r = I32 ? __ldg(q + (i0 + k * bxy + j * bx)) : __ldg(p + (int64_t)k * bxy + j * bx);
            const float row = r.x * wx0 + r.y * wx1 + r.z * wx2 + r.w * wx3;
            pl += row * wy[j];
        }
        acc += pl * wz[k];
    }
    return acc;
}

// Stencil-7 reference gradient on the fly (numba_kernels._grad_at :188-212). The differences of two
// float32 voxels round to float32 as in the reference; indices are clamped so the read stays inside f.
__device__ __forceinline__ void grad_otf(const float* __restrict__ f, int nz, int ny, int nx, int zz, int yy, int xx, float& gx,
                                         float& gy, float& gz) {
    const int64_t sxy = (int64_t)nx * ny;
    auto at = [&](int z, int y, int x) -> float {
        z = min(max(z, 0), nz - 1);
        y = min(max(y, 0), ny - 1);
        x = min(max(x, 0), nx - 1);
        return __ldg(f + (int64_t)z * sxy + (int64_t)y * nx + x);
    };
    const float c1 = 0.75f, c2 = -0.15f, c3 = 1.0f / 60.0f;
    gx = c1 * (at(zz, yy, xx + 1) - at(zz, yy, xx - 1)) + c2 * (at(zz, yy, xx + 2) - at(zz, yy, xx - 2)) +
         c3 * (at(zz, yy, xx + 3) - at(zz, yy, xx - 3));
    gy = c1 * (at(zz, yy + 1, xx) - at(zz, yy - 1, xx)) + c2 * (at(zz, yy + 2, xx) - at(zz, yy - 2, xx)) +
         c3 * (at(zz, yy + 3, xx) - at(zz, yy - 3, xx));
    gz = c1 * (at(zz + 1, yy, xx) - at(zz - 1, yy, xx)) + c2 * (at(zz + 2, yy, xx) - at(zz - 2, yy, xx)) +
         c3 * (at(zz + 3, yy, xx) - at(zz - 3, yy, xx));
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ int warp_sum_i(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ----------------------------------------------------------------------------- small dense FP64 algebra
// numba_kernels.py:58-180, restated for one thread.
__device__ inline bool chol12(const double* H, double* L) {
    for (int i = 0; i < 144; ++i) L[i] = 0.0;
    for (int j = 0; j < 12; ++j) {
        double s = H[j * 12 + j];
        for (int k = 0; k < j; ++k) s -= L[j * 12 + k] * L[j * 12 + k];
        if (s <= 0.0 || !isfinite(s)) return false;
        const double ljj = sqrt(s);
        L[j * 12 + j] = ljj;
        for (int i = j + 1; i < 12; ++i) {
            double t = H[i * 12 + j];
            for (int k = 0; k < j; ++k) t -= L[i * 12 + k] * L[j * 12 + k];
            L[i * 12 + j] = t / ljj;
        }
    }
    return true;
}

__device__ inline void chol_solve12(const double* L, const double* b, double* x) {
    double y[12];
    for (int i = 0; i < 12; ++i) {
        double s = b[i];
        for (int k = 0; k < i; ++k) s -= L[i * 12 + k] * y[k];
        y[i] = s / L[i * 12 + i];
    }
    for (int i = 11; i >= 0; --i) {
        double s = y[i];
        for (int k = i + 1; k < 12; ++k) s -= L[k * 12 + i] * x[k];
        x[i] = s / L[i * 12 + i];
    }
}

__device__ inline double inv3(const double a[3][3], double out[3][3]) {
    const double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                       a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
    if (fabs(det) < 1e-300) return 0.0;
    const double inv = 1.0 / det;
    out[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) * inv;
    out[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) * inv;
    out[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) * inv;
    out[1][0] = (a[1][2] * a[2][0] - a[1][0] * a[2][2]) * inv;
    out[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) * inv;
    out[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) * inv;
    out[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) * inv;
    out[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) * inv;
    out[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) * inv;
    return det;
}

// W(P) <- W(P) o W(dP)^-1 (compose_warp_inplace :145-180)
__device__ inline bool compose_warp(double* P, const double* dP) {
    double A[3][3], dA[3][3], dAi[3][3], An[3][3];
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) {
            A[i][j] = P[3 * i + j];
            dA[i][j] = dP[3 * i + j];
        }
        A[i][i] += 1.0;
        dA[i][i] += 1.0;
    }
    if (inv3(dA, dAi) == 0.0) return false;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += A[i][k] * dAi[k][j];
            An[i][j] = s;
        }
    for (int i = 0; i < 3; ++i) {
        double s = 0.0;
        for (int k = 0; k < 3; ++k) s += An[i][k] * dP[9 + k];
        P[9 + i] = P[9 + i] - s;
    }
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) P[3 * i + j] = An[i][j];
        P[3 * i + i] -= 1.0;
    }
    return true;
}

}  // namespace aldvc
