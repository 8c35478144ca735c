// In-register FFT of a compile-time length N (2,3,5-smooth): one thread transforms one line of N complex
// values held in registers.  Recursive decimation in time, fully unrolled: every index, radix and twiddle
// exponent is a compile-time constant, the twiddles exp(-2 pi i e / N) come from a constant-memory table,
// so a stage costs only its arithmetic.
#pragma once

#include <cuda_runtime.h>

namespace aldvc {

// line lengths with a compiled in-register transform (cubic FFT boxes of the NCC engine): 36, 40, 48, 50, 54,
// 60, 64; fftr_offset is the position of a length's twiddles in the shared table, -1 for any other length
__host__ __device__ constexpr int fftr_offset(int n) {
    return n == 36 ? 0 : n == 40 ? 36 : n == 48 ? 76 : n == 50 ? 124 : n == 54 ? 174 : n == 60 ? 228 : n == 64 ? 288 : -1;
}
constexpr int FFTR_TOTAL = 352;
constexpr int FFTR_NSIZES = 7;
constexpr int FFTR_SIZES[FFTR_NSIZES] = {36, 40, 48, 50, 54, 60, 64};  // host code only

__host__ __device__ constexpr bool fftr_supported(int n) { return fftr_offset(n) >= 0; }

__host__ __device__ constexpr int fftr_radix(int n) { return (n % 4 == 0 && n > 4) ? 4 : (n % 2 == 0 ? 2 : (n % 3 == 0 ? 3 : (n % 5 == 0 ? 5 : n))); }

// exp(-2 pi i k / n) for every supported n, at fftr_offset(n) + k (filled once per device); host code (tests of
// the transform on the CPU) reads the same values from h_fftr_tw.  One translation unit includes this header.
static __constant__ float2 c_fftr_tw[FFTR_TOTAL];
static float2 h_fftr_tw[FFTR_TOTAL];

__host__ __device__ __forceinline__ float2 fr_tw(int idx) {
#ifdef __CUDA_ARCH__
    return c_fftr_tw[idx];
#else
    return h_fftr_tw[idx];
#endif
}

__host__ __device__ __forceinline__ float2 fr_mul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__host__ __device__ __forceinline__ float2 fr_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 fr_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// (SIGN i) a
template <int SIGN>
__host__ __device__ __forceinline__ float2 fr_muli(float2 a) {
    return SIGN < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}

// In-place DFT of R (2, 3, 4, 5) values, exponent sign SIGN.
template <int R, int SIGN>
__host__ __device__ __forceinline__ void fr_small(float2* v) {
    if constexpr (R == 2) {
        const float2 a = v[0], b = v[1];
        v[0] = fr_add(a, b);
        v[1] = fr_sub(a, b);
    } else if constexpr (R == 4) {
        const float2 s02 = fr_add(v[0], v[2]), d02 = fr_sub(v[0], v[2]), s13 = fr_add(v[1], v[3]);
        const float2 d13 = fr_muli<SIGN>(fr_sub(v[1], v[3]));
        v[0] = fr_add(s02, s13);
        v[2] = fr_sub(s02, s13);
        v[1] = fr_add(d02, d13);
        v[3] = fr_sub(d02, d13);
    } else if constexpr (R == 3) {
        const float c1 = -0.5f, s1 = 0.86602540378443864676f;  // cos and sin of 2 pi / 3
        const float2 a = v[0], t = fr_add(v[1], v[2]), d = fr_sub(v[1], v[2]);
        const float2 u = fr_muli<SIGN>(make_float2(s1 * d.x, s1 * d.y));
        const float2 m = make_float2(a.x + c1 * t.x, a.y + c1 * t.y);
        v[0] = fr_add(a, t);
        v[1] = fr_add(m, u);
        v[2] = fr_sub(m, u);
    } else {  // R == 5
        const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;  // cos 2pi/5, cos 4pi/5
        const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;   // sin 2pi/5, sin 4pi/5
        const float2 a = v[0];
        const float2 t1 = fr_add(v[1], v[4]), t2 = fr_add(v[2], v[3]);
        const float2 d1 = fr_sub(v[1], v[4]), d2 = fr_sub(v[2], v[3]);
        const float2 m1 = make_float2(a.x + c1 * t1.x + c2 * t2.x, a.y + c1 * t1.y + c2 * t2.y);
        const float2 m2 = make_float2(a.x + c2 * t1.x + c1 * t2.x, a.y + c2 * t1.y + c1 * t2.y);
        const float2 n1 = fr_muli<SIGN>(make_float2(s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y));
        const float2 n2 = fr_muli<SIGN>(make_float2(s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y));
        v[0] = fr_add(a, fr_add(t1, t2));
        v[1] = fr_add(m1, n1);
        v[4] = fr_sub(m1, n1);
        v[2] = fr_add(m2, n2);
        v[3] = fr_sub(m2, n2);
    }
}

// y[k] = sum_j x[j STRIDE] w_N^(j k), w_N = exp(SIGN 2 pi i / N); TOP is the length whose twiddle table is read.
template <int N, int TOP, int SIGN, int STRIDE>
__host__ __device__ __forceinline__ void fr_rec(const float2* x, float2* y) {
    constexpr int R = fftr_radix(N);
    if constexpr (R == N) {
        float2 v[N];
#pragma unroll
        for (int j = 0; j < N; ++j) v[j] = x[j * STRIDE];
        fr_small<N, SIGN>(v);
#pragma unroll
        for (int k = 0; k < N; ++k) y[k] = v[k];
    } else {
        constexpr int M = N / R;
        float2 s[N];
#pragma unroll
        for (int r = 0; r < R; ++r) fr_rec<M, TOP, SIGN, STRIDE * R>(x + r * STRIDE, s + r * M);
#pragma unroll
        for (int k = 0; k < M; ++k) {
            float2 t[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (r == 0 || k == 0) {
                    t[r] = s[r * M + k];
                } else {
                    float2 w = fr_tw(fftr_offset(TOP) + ((r * k * (TOP / N)) % TOP));
                    if (SIGN > 0) w.y = -w.y;
                    t[r] = fr_mul(s[r * M + k], w);
                }
            }
            fr_small<R, SIGN>(t);
#pragma unroll
            for (int q = 0; q < R; ++q) y[k + q * M] = t[q];
        }
    }
}

// In-place transform of the N values of v (natural order in and out).
template <int N, int SIGN>
__host__ __device__ __forceinline__ void fft_line(float2 (&v)[N]) {
    float2 out[N];
    fr_rec<N, N, SIGN, 1>(v, out);
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = out[k];
}

}  // namespace aldvc
