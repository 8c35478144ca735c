// ZNSSD residual of warped subsets, forward and hand-written backward.
//
// The residual is the one IC-GN minimises (pyALDVC solver/numba_kernels.py:705-708 with the dynamic valid-set
// statistics of :586-598):  r_v = (f_v - mf) / bf - (g(W(x_v; P)) - mg) / bg,  C = sum_v r_v^2,
// for a subset of (2h+1)^3 voxels around an integer node, with the 12-parameter affine warp
// W(x; P) = x0 + (u, v, w) + (I + F)(x - x0), P = [F row-major, u, v, w].
//
// Forward: per subset, sample g at the warped voxels (FP64 positions, FP32 interpolation), reduce the
// statistics in FP64 and the cost in a second sweep (residuals in FP64); save (n, mf, bf, mg, bg,
// R1 = sum r, R2 = sum r b) with b_v = (g_v - mg) / bg.
// Backward (weights recomputed, nothing per voxel stored):
//   dC/dg_u = -(2 / bg) (r_u - R1 / n - b_u R2)          (mg and bg depend on every g_u)
//   dC/dP[3i+j] = sum_u dC/dg_u d_i g(x_u) X_j,   dC/dP[9+i] = sum_u dC/dg_u d_i g(x_u)
//   dC/dG[q] += dC/dg_u w_q(x_u) for the interpolation taps q of every sample (atomic scatter).
// The gradient of the interpolant is the derivative of its weights (Keys a = -0.5, trilinear, B-spline).
#include <algorithm>

#include "common.cuh"
#include "internal.cuh"

namespace aldvc {

constexpr int ZN_THREADS = 128;
constexpr int ZN_STATS = 7;

struct ZnArgs {
    const float* f;
    const float* g;
    int nz, ny, nx;
    const int64_t* coords;
    int64_t n;
    int hx, hy, hz, mode;
    const double* P;
    double* cost;
    double* stats;
    const double* gcost;
    double* gP;
    float* gG;
};

__device__ __forceinline__ void keys_dw(float t, float& d0, float& d1, float& d2, float& d3) {
    d0 = (-1.5f * t + 2.0f) * t - 0.5f;
    d1 = (4.5f * t - 5.0f) * t;
    d2 = (-4.5f * t + 4.0f) * t + 0.5f;
    d3 = (1.5f * t - 1.0f) * t;
}

__device__ __forceinline__ void bspl_dw(float t, float& d0, float& d1, float& d2, float& d3) {
    const float u = 1.0f - t;
    d0 = -0.5f * u * u;
    d1 = (1.5f * t - 2.0f) * t;
    d2 = (-1.5f * t + 1.0f) * t + 0.5f;
    d3 = 0.5f * t * t;
}

// Interpolation taps of one sample: 2 (linear) or 4 (cubic) per axis, their weights and weight derivatives,
// and the volume index of the first tap.  (ix, iy, iz) = floor of the position, clamped like the sampler.
template <int MODE>
struct Taps {
    static constexpr int K = MODE == 0 ? 2 : 4;
    float wx[K], wy[K], wz[K], dx[K], dy[K], dz[K];
    int64_t base;
    // position = (xc + xr, yc + yr, zc + zr): integer node plus an FP64 offset; the fractions are exact to FP32
    __device__ __forceinline__ void make(int xc, double xr, int yc, double yr, int zc, double zr, int nx, int ny, int nz) {
        const double flx = floor(xr), fly = floor(yr), flz = floor(zr);
        const float fx = (float)(xr - flx), fy = (float)(yr - fly), fz = (float)(zr - flz);
        int ix = xc + (int)flx, iy = yc + (int)fly, iz = zc + (int)flz;
        if (MODE == 0) {
            ix = min(max(ix, 0), nx - 2);
            iy = min(max(iy, 0), ny - 2);
            iz = min(max(iz, 0), nz - 2);
        } else {
            ix = min(max(ix, 1), nx - 3);
            iy = min(max(iy, 1), ny - 3);
            iz = min(max(iz, 1), nz - 3);
        }
        const int o = MODE == 0 ? 0 : 1;
        base = ((int64_t)(iz - o) * ny + (iy - o)) * nx + (ix - o);
        if (MODE == 0) {
            wx[0] = 1.0f - fx, wx[1] = fx, dx[0] = -1.0f, dx[1] = 1.0f;
            wy[0] = 1.0f - fy, wy[1] = fy, dy[0] = -1.0f, dy[1] = 1.0f;
            wz[0] = 1.0f - fz, wz[1] = fz, dz[0] = -1.0f, dz[1] = 1.0f;
        } else if (MODE == 1) {
            keys_w(fx, wx[0], wx[1], wx[2], wx[3]);
            keys_w(fy, wy[0], wy[1], wy[2], wy[3]);
            keys_w(fz, wz[0], wz[1], wz[2], wz[3]);
            keys_dw(fx, dx[0], dx[1], dx[2], dx[3]);
            keys_dw(fy, dy[0], dy[1], dy[2], dy[3]);
            keys_dw(fz, dz[0], dz[1], dz[2], dz[3]);
        } else {
            bspl_w(fx, wx[0], wx[1], wx[2], wx[3]);
            bspl_w(fy, wy[0], wy[1], wy[2], wy[3]);
            bspl_w(fz, wz[0], wz[1], wz[2], wz[3]);
            bspl_dw(fx, dx[0], dx[1], dx[2], dx[3]);
            bspl_dw(fy, dy[0], dy[1], dy[2], dy[3]);
            bspl_dw(fz, dz[0], dz[1], dz[2], dz[3]);
        }
    }
    // value and, with GRAD, the three partial derivatives
    template <bool GRAD>
    __device__ __forceinline__ float eval(const float* __restrict__ g, int nx, int64_t sxy, float& gx, float& gy, float& gz) const {
        float v = 0.0f;
        gx = gy = gz = 0.0f;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            float p = 0.0f, pdx = 0.0f, pdy = 0.0f;
#pragma unroll
            for (int j = 0; j < K; ++j) {
                const float* r = g + base + k * sxy + (int64_t)j * nx;
                float rx = 0.0f, rdx = 0.0f;
#pragma unroll
                for (int i = 0; i < K; ++i) {
                    const float s = __ldg(r + i);
                    rx = fmaf(wx[i], s, rx);
                    if (GRAD) rdx = fmaf(dx[i], s, rdx);
                }
                p = fmaf(wy[j], rx, p);
                if (GRAD) {
                    pdx = fmaf(wy[j], rdx, pdx);
                    pdy = fmaf(dy[j], rx, pdy);
                }
            }
            v = fmaf(wz[k], p, v);
            if (GRAD) {
                gx = fmaf(wz[k], pdx, gx);
                gy = fmaf(wz[k], pdy, gy);
                gz = fmaf(dz[k], p, gz);
            }
        }
        return v;
    }
    __device__ __forceinline__ void scatter(float* gG, int nx, int64_t sxy, float c) const {
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
            for (int j = 0; j < K; ++j) {
                const float cjk = c * wz[k] * wy[j];
                float* r = gG + base + k * sxy + (int64_t)j * nx;
#pragma unroll
                for (int i = 0; i < K; ++i) atomicAdd(r + i, cjk * wx[i]);
            }
    }
};

// FP64 block sum of NV values per thread (thread 0 gets the totals in out).
template <int NV>
__device__ void zn_block_sum(const double* v, double (*red)[ZN_THREADS / 32], double* out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        const double s = warp_sum_d(v[i]);
        if (lane == 0) red[i][warp] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int i = 0; i < NV; ++i) {
            double t = 0.0;
            for (int w = 0; w < ZN_THREADS / 32; ++w) t += red[i][w];
            out[i] = t;
        }
    __syncthreads();
}

// The warp in FP64: sample positions are formed in FP64 (9 FMAs per voxel) so that the backward sees the same
// function the FP64 finite differences of the oracle see.
struct ZnWarp {
    double A[9], t[3];
    __device__ void load(const double* P) {
        for (int k = 0; k < 9; ++k) A[k] = P[k];
        A[0] += 1.0;
        A[4] += 1.0;
        A[8] += 1.0;
        t[0] = P[9];
        t[1] = P[10];
        t[2] = P[11];
    }
    template <int MODE>
    __device__ __forceinline__ void taps(Taps<MODE>& tp, int64_t xc, int64_t yc, int64_t zc, double X, double Y, double Z, int nx, int ny,
                                         int nz) const {
        tp.make((int)xc, A[0] * X + A[1] * Y + A[2] * Z + t[0], (int)yc, A[3] * X + A[4] * Y + A[5] * Z + t[1], (int)zc,
                A[6] * X + A[7] * Y + A[8] * Z + t[2], nx, ny, nz);
    }
};

// the reference subset inside f, and every warped voxel inside the sampler's admissible domain (the warp is
// affine: the 8 corners decide)
__device__ bool zn_inside(const ZnArgs& a, const double* P, int64_t xc, int64_t yc, int64_t zc) {
    bool in = xc - a.hx >= 0 && xc + a.hx < a.nx && yc - a.hy >= 0 && yc + a.hy < a.ny && zc - a.hz >= 0 && zc + a.hz < a.nz;
    for (int c = 0; c < 8; ++c) {
        const double X = (c & 1) ? a.hx : -a.hx, Y = (c & 2) ? a.hy : -a.hy, Z = (c & 4) ? a.hz : -a.hz;
        const double xw = (1.0 + P[0]) * X + P[1] * Y + P[2] * Z + ((double)xc + P[9]);
        const double yw = P[3] * X + (1.0 + P[4]) * Y + P[5] * Z + ((double)yc + P[10]);
        const double zw = P[6] * X + P[7] * Y + (1.0 + P[8]) * Z + ((double)zc + P[11]);
        in = in && margin_ok(zw, yw, xw, a.nz, a.ny, a.nx);
    }
    return in;
}

template <int MODE>
__global__ void __launch_bounds__(ZN_THREADS) znssd_forward_kernel(ZnArgs a) {
    __shared__ double red[6][ZN_THREADS / 32];
    __shared__ double tot[6];
    __shared__ int s_in;
    const int64_t s = blockIdx.x;
    const int64_t xc = a.coords[3 * s], yc = a.coords[3 * s + 1], zc = a.coords[3 * s + 2];
    const double* P = a.P + 12 * s;
    if (threadIdx.x == 0) s_in = zn_inside(a, P, xc, yc, zc) ? 1 : 0;
    __syncthreads();
    double* st = a.stats + ZN_STATS * s;
    if (!s_in) {  // a voxel leaves the admissible domain: no cost (the solver's OOB status)
        if (threadIdx.x == 0) {
            a.cost[s] = nan("");
            for (int i = 0; i < ZN_STATS; ++i) st[i] = 0.0;
        }
        return;
    }
    ZnWarp w;
    w.load(P);
    const int64_t sxy = (int64_t)a.nx * a.ny;
    const int nX = 2 * a.hx + 1, nY = 2 * a.hy + 1, S = nX * nY * (2 * a.hz + 1);
    double cnt = 0.0, sg = 0.0, sgg = 0.0, sf = 0.0, sff = 0.0;
    for (int v = threadIdx.x; v < S; v += ZN_THREADS) {
        const int ix = v % nX, r = v / nX, iy = r % nY, iz = r / nY;
        const int X = ix - a.hx, Y = iy - a.hy, Z = iz - a.hz;
        Taps<MODE> tp;
        w.taps(tp, xc, yc, zc, (double)X, (double)Y, (double)Z, a.nx, a.ny, a.nz);
        float d0, d1, d2;
        const float gv = tp.template eval<false>(a.g, a.nx, sxy, d0, d1, d2);
        if (gv != gv) continue;  // NaN voxel of g: outside the valid set
        const float fv = __ldg(a.f + (zc + Z) * sxy + (yc + Y) * a.nx + (xc + X));
        cnt += 1.0;
        sg += (double)gv;
        sgg += (double)gv * (double)gv;
        sf += (double)fv;
        sff += (double)(fv * fv);  // float32 square, as the reference's statistics
    }
    double v5[5] = {cnt, sg, sgg, sf, sff};
    zn_block_sum<5>(v5, red, tot);
    if (threadIdx.x == 0) {
        const double n = tot[0];
        const double mg = tot[1] / n, mf = tot[3] / n;
        double ssg = tot[2] - n * mg * mg, ssf = tot[4] - n * mf * mf;
        ssg = ssg < 0.0 ? 0.0 : ssg;
        ssf = ssf < 0.0 ? 0.0 : ssf;
        tot[0] = n;
        tot[1] = mf;
        tot[2] = sqrt(ssf > 1e-30 ? ssf : 1e-30);
        tot[3] = mg;
        tot[4] = sqrt(ssg > 1e-30 ? ssg : 1e-30);
    }
    __syncthreads();
    const double n = tot[0], mfd = tot[1], bf = tot[2], mgd = tot[3], bg = tot[4];
    const double ibf = 1.0 / bf, ibg = 1.0 / bg;
    __syncthreads();
    double c2 = 0.0, r1 = 0.0, r2 = 0.0;
    for (int v = threadIdx.x; v < S; v += ZN_THREADS) {
        const int ix = v % nX, r = v / nX, iy = r % nY, iz = r / nY;
        const int X = ix - a.hx, Y = iy - a.hy, Z = iz - a.hz;
        Taps<MODE> tp;
        w.taps(tp, xc, yc, zc, (double)X, (double)Y, (double)Z, a.nx, a.ny, a.nz);
        float d0, d1, d2;
        const float gv = tp.template eval<false>(a.g, a.nx, sxy, d0, d1, d2);
        if (gv != gv) continue;
        const float fv = __ldg(a.f + (zc + Z) * sxy + (yc + Y) * a.nx + (xc + X));
        const double b = ((double)gv - mgd) * ibg;
        const double res = ((double)fv - mfd) * ibf - b;
        c2 = fma(res, res, c2);
        r1 += res;
        r2 = fma(res, b, r2);
    }
    double v3[3] = {c2, r1, r2};
    zn_block_sum<3>(v3, red, tot);
    if (threadIdx.x == 0) {
        const bool ok = n >= MIN_SUBSET_VOXELS && n >= MIN_VALID_FRACTION * (double)S;
        a.cost[s] = ok ? tot[0] : nan("");
        st[0] = ok ? n : 0.0;
        st[1] = mfd;
        st[2] = bf;
        st[3] = mgd;
        st[4] = bg;
        st[5] = tot[1];
        st[6] = tot[2];
    }
}

template <int MODE>
__global__ void __launch_bounds__(ZN_THREADS) znssd_backward_kernel(ZnArgs a) {
    __shared__ double red[12][ZN_THREADS / 32];
    __shared__ double tot[12];
    const int64_t s = blockIdx.x;
    const double* st = a.stats + ZN_STATS * s;
    const double n = st[0];
    const double gc = a.gcost[s];
    double* gP = a.gP ? a.gP + 12 * s : nullptr;
    if (!(n > 0.0) || gc == 0.0 || !isfinite(gc)) {  // invalid subset or no incoming gradient
        if (gP && threadIdx.x < 12) gP[threadIdx.x] = 0.0;
        return;
    }
    const int64_t xc = a.coords[3 * s], yc = a.coords[3 * s + 1], zc = a.coords[3 * s + 2];
    ZnWarp w;
    w.load(a.P + 12 * s);
    const int64_t sxy = (int64_t)a.nx * a.ny;
    const int nX = 2 * a.hx + 1, nY = 2 * a.hy + 1, S = nX * nY * (2 * a.hz + 1);
    const double mf = st[1], ibf = 1.0 / st[2], mg = st[3], ibg = 1.0 / st[4];
    const double R1n = st[5] / n, R2 = st[6];
    const double scale = -2.0 * gc / st[4];
    double acc[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[k] = 0.0;
    for (int v = threadIdx.x; v < S; v += ZN_THREADS) {
        const int ix = v % nX, r = v / nX, iy = r % nY, iz = r / nY;
        const int X = ix - a.hx, Y = iy - a.hy, Z = iz - a.hz;
        Taps<MODE> tp;
        w.taps(tp, xc, yc, zc, (double)X, (double)Y, (double)Z, a.nx, a.ny, a.nz);
        float dgx, dgy, dgz;
        const float gv = tp.template eval<true>(a.g, a.nx, sxy, dgx, dgy, dgz);
        if (gv != gv) continue;
        const float fv = __ldg(a.f + (zc + Z) * sxy + (yc + Y) * a.nx + (xc + X));
        const double b = ((double)gv - mg) * ibg;
        const double res = ((double)fv - mf) * ibf - b;
        const double dc = scale * (res - R1n - b * R2);  // dC/dg at this voxel times the incoming gradient
        if (gP) {
            const double q[3] = {dc * (double)dgx, dc * (double)dgy, dc * (double)dgz};
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                acc[3 * i] = fma(q[i], (double)X, acc[3 * i]);
                acc[3 * i + 1] = fma(q[i], (double)Y, acc[3 * i + 1]);
                acc[3 * i + 2] = fma(q[i], (double)Z, acc[3 * i + 2]);
                acc[9 + i] += q[i];
            }
        }
        if (a.gG) tp.scatter(a.gG, a.nx, sxy, (float)dc);
    }
    if (gP) {
        zn_block_sum<12>(acc, red, tot);
        if (threadIdx.x < 12) gP[threadIdx.x] = tot[threadIdx.x];
    }
}

static int zn_fill(ZnArgs& a, const aldvc_volumes* vol, const int64_t* coords, int64_t n, int32_t hx, int32_t hy, int32_t hz,
                   int32_t mode, const double* P) {
    ALDVC_REQUIRE(vol && vol->f && vol->g && coords && P, "znssd: null pointer");
    ALDVC_REQUIRE(mode >= 0 && mode <= 2, "znssd: mode must be 0, 1 or 2");
    ALDVC_REQUIRE(hx >= 1 && hy >= 1 && hz >= 1, "znssd: half-widths must be >= 1");
    ALDVC_REQUIRE(vol->nz >= 4 && vol->ny >= 4 && vol->nx >= 4 && vol->nx * vol->ny < (1LL << 31), "znssd: bad volume shape");
    ALDVC_REQUIRE(n < (1LL << 31), "znssd: too many subsets");
    a = ZnArgs{};
    a.f = vol->f;
    a.g = vol->g;
    a.nz = (int)vol->nz;
    a.ny = (int)vol->ny;
    a.nx = (int)vol->nx;
    a.coords = coords;
    a.n = n;
    a.hx = hx;
    a.hy = hy;
    a.hz = hz;
    a.mode = mode;
    a.P = P;
    return ALDVC_OK;
}

}  // namespace aldvc

using namespace aldvc;

extern "C" int aldvc_znssd_forward(const aldvc_volumes* vol, const int64_t* coords, int64_t n, int32_t hx, int32_t hy, int32_t hz,
                                   int32_t mode, const double* P, double* cost, double* stats, void* stream) {
    ZnArgs a;
    int rc = zn_fill(a, vol, coords, n, hx, hy, hz, mode, P);
    if (rc) return rc;
    ALDVC_REQUIRE(cost && stats, "aldvc_znssd_forward: null output");
    if (n <= 0) return ALDVC_OK;
    a.cost = cost;
    a.stats = stats;
    cudaStream_t s = (cudaStream_t)stream;
    if (mode == 0)
        {
            KTimer kt_("znssd_forward", s);
            znssd_forward_kernel<0><<<(unsigned)n, ZN_THREADS, 0, s>>>(a);
        }
    else if (mode == 1)
        {
            KTimer kt_("znssd_forward", s);
            znssd_forward_kernel<1><<<(unsigned)n, ZN_THREADS, 0, s>>>(a);
        }
    else
        {
            KTimer kt_("znssd_forward", s);
            znssd_forward_kernel<2><<<(unsigned)n, ZN_THREADS, 0, s>>>(a);
        }
    return check_launch("znssd forward");
}

extern "C" int aldvc_znssd_backward(const aldvc_volumes* vol, const int64_t* coords, int64_t n, int32_t hx, int32_t hy, int32_t hz,
                                    int32_t mode, const double* P, const double* stats, const double* grad_cost, double* grad_P,
                                    float* grad_g, void* stream) {
    ZnArgs a;
    int rc = zn_fill(a, vol, coords, n, hx, hy, hz, mode, P);
    if (rc) return rc;
    ALDVC_REQUIRE(stats && grad_cost, "aldvc_znssd_backward: null input");
    if (n <= 0 || (!grad_P && !grad_g)) return ALDVC_OK;
    a.stats = const_cast<double*>(stats);
    a.gcost = grad_cost;
    a.gP = grad_P;
    a.gG = grad_g;
    cudaStream_t s = (cudaStream_t)stream;
    if (mode == 0)
        {
            KTimer kt_("znssd_backward", s);
            znssd_backward_kernel<0><<<(unsigned)n, ZN_THREADS, 0, s>>>(a);
        }
    else if (mode == 1)
        {
            KTimer kt_("znssd_backward", s);
            znssd_backward_kernel<1><<<(unsigned)n, ZN_THREADS, 0, s>>>(a);
        }
    else
        {
            KTimer kt_("znssd_backward", s);
            znssd_backward_kernel<2><<<(unsigned)n, ZN_THREADS, 0, s>>>(a);
        }
    return check_launch("znssd backward");
}
