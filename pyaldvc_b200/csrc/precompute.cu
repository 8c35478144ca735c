// Per-node precomputation of the local solver: Gauss-Newton Hessian, its FP64 Cholesky factor and the
// ZNSSD normalisation of the reference subset (pyALDVC numba_kernels._precompute_one :326-418).
//
// One CTA per node.  H[(i,j),(k,l)] = sum g_i g_k X_j X_l with X = (X, Y, Z, 1) has only 6 x 10 = 60
// distinct sums (Kronecker structure of the steepest-descent images), accumulated per thread in FP32 blocks of
// 16 voxels folded into Kahan-compensated totals, then reduced across the warp and across warps in FP64.  Sum f and sum f^2
// are taken relative to the centre voxel so the variance does not cancel for offset intensities.
#include "common.cuh"
#include "internal.cuh"

namespace aldvc {

constexpr int PRE_THREADS = 256;
constexpr int PRE_NSUM = 60 + 2;  // 60 Hessian moments, sum(f - c), sum((f - c)^2)
constexpr int PRE_BLOCK = 16;     // voxels per plain FP32 block sum before its compensated fold

struct PreArgs {
    const float* f;
    const float* gx;
    const float* gy;
    const float* gz;
    const uint8_t* mask;
    int nz, ny, nx;
    int hx, hy, hz, stride;
    const int64_t* split_index;
    const uint8_t* split_keep;
    int64_t keep_bytes;
    const int64_t* coords;
    int64_t n_nodes;
    double min_valid_ratio, cond_max;
    double* H;
    double* L;
    double* meanf;
    double* bottomf;
    int64_t* n_valid;
    uint8_t* valid;
    const int32_t* node_half;  // (N,3) per-node half-widths, NULL: (hx, hy, hz) for every node
};

// (i,k) pair index of the gradient products gg: 00 01 02 11 12 22
__device__ __forceinline__ int gg_index(int i, int k) {
    if (i > k) {
        int t = i;
        i = k;
        k = t;
    }
    return i == 0 ? k : (i == 1 ? 2 + k : 5);
}

// (j,l) pair index of the coordinate products xx over (X, Y, Z, 1): 00 01 02 03 11 12 13 22 23 33
__device__ __forceinline__ int xx_index(int j, int l) {
    if (j > l) {
        int t = j;
        j = l;
        l = t;
    }
    const int base[4] = {0, 4, 7, 9};
    return base[j] + (l - j);
}

// Kahan step: s + x with the rounding error carried in c (the compensated total is s - c)
__device__ __forceinline__ void kahan_add(float& s, float& c, float x) {
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

template <bool STORED>
__global__ void __launch_bounds__(PRE_THREADS, 2) precompute_kernel(PreArgs a) {
    const int64_t node = blockIdx.x;
    if (node >= a.n_nodes) return;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    __shared__ double red[PRE_THREADS / 32][PRE_NSUM];
    __shared__ int red_n[PRE_THREADS / 32];
    __shared__ double tot[PRE_NSUM];
    extern __shared__ float kah[];  // Kahan (sum, compensation) pairs of every thread: [2][31][PRE_THREADS]

    const int64_t x0 = a.coords[3 * node], y0 = a.coords[3 * node + 1], z0 = a.coords[3 * node + 2];
    // this node's subset shape; a per-node shape beyond the call's maximum is rejected like an outside subset
    int hx = a.hx, hy = a.hy, hz = a.hz;
    bool shape_ok = true;
    if (a.node_half) {
        hx = a.node_half[3 * node];
        hy = a.node_half[3 * node + 1];
        hz = a.node_half[3 * node + 2];
        shape_ok = hx >= 0 && hy >= 0 && hz >= 0 && hx <= a.hx && hy <= a.hy && hz <= a.hz;
    }
    const int64_t r = a.split_index ? a.split_index[node] : -1;
    const bool use_keep = r >= 0;
    const uint8_t* keep = use_keep ? a.split_keep + r * a.keep_bytes : nullptr;
    double* H = a.H + node * 144;
    double* L = a.L + node * 144;

    const bool inside = x0 - hx >= 0 && x0 + hx < a.nx && y0 - hy >= 0 && y0 + hy < a.ny && z0 - hz >= 0 && z0 + hz < a.nz;
    if ((!use_keep && !inside) || !shape_ok) {
        for (int i = tid; i < 144; i += PRE_THREADS) {
            H[i] = 0.0;
            L[i] = 0.0;
        }
        if (tid == 0) {
            a.meanf[node] = 0.0;
            a.bottomf[node] = 1.0;
            a.n_valid[node] = 0;
            a.valid[node] = 0;
        }
        return;
    }
    const int64_t sxy = (int64_t)a.nx * a.ny;
    // pilot value for the f moments: the centre voxel (clamped into the volume)
    auto clampi = [](int64_t v, int64_t hi) -> int64_t { return v < 0 ? 0 : (v > hi ? hi : v); };
    const int64_t cz = clampi(z0, a.nz - 1), cy = clampi(y0, a.ny - 1), cx = clampi(x0, a.nx - 1);
    const float pilot = __ldg(a.f + cz * sxy + cy * a.nx + cx);

    int n = 0;
    const int nX = (2 * hx) / a.stride + 1, nY = (2 * hy) / a.stride + 1, nZ = (2 * hz) / a.stride + 1;
    const int S = nX * nY * nZ;
    // mixed-radix step of PRE_THREADS voxels through (iz, iy, ix)
    const int st_z = PRE_THREADS / (nX * nY), rem = PRE_THREADS % (nX * nY);
    const int st_y = rem / nX, st_x = rem % nX;
    // Compensated FP32 sums: plain FP32 block sums over PRE_BLOCK voxels in registers, folded into Kahan
    // (sum, compensation) pairs kept in shared memory.  The 62 moments are swept in two halves of 31 (gradient
    // products 00 01 02 with sum f, then 11 12 22 with sum f^2); each thread's corrected totals are reduced in FP64.
    // (Measured on the 1024 x 1024 x 306 workload: 98 ms per pass, against 112 ms for one sweep of all 62 with the
    // pairs of every moment in shared memory, and 106 ms for per-voxel Kahan steps in registers.)
#pragma unroll 1
    for (int part = 0; part < 2; ++part) {
        float blk[31];
        float* ksum = kah + tid;  // this thread's Kahan pairs in shared memory, [31][PRE_THREADS] each
        float* kcmp = kah + 31 * PRE_THREADS + tid;
#pragma unroll
        for (int i = 0; i < 31; ++i) {
            blk[i] = 0.0f;
            ksum[i * PRE_THREADS] = 0.0f;
            kcmp[i * PRE_THREADS] = 0.0f;
        }
        int in_blk = 0;
        int ix = tid % nX, iy = (tid / nX) % nY, iz = tid / (nX * nY);
        for (int v = tid; v < S; v += PRE_THREADS) {
            const int dx = -hx + ix * a.stride, dy = -hy + iy * a.stride, dz = -hz + iz * a.stride;
            const int64_t xx = x0 + dx, yy = y0 + dy, zz = z0 + dz;
            bool k;
            if (use_keep) {
                k = kept_bit(keep, v) && xx >= 0 && xx < a.nx && yy >= 0 && yy < a.ny && zz >= 0 && zz < a.nz;
            } else {
                k = (a.mask == nullptr) || __ldg(a.mask + zz * sxy + yy * a.nx + xx) != 0;
            }
            if (k) {
                const int64_t o = zz * sxy + yy * a.nx + xx;
                const float fv = __ldg(a.f + o) - pilot;
                float g0, g1, g2;
                if (STORED) {
                    g0 = __ldg(a.gx + o);
                    g1 = __ldg(a.gy + o);
                    g2 = __ldg(a.gz + o);
                } else {
                    grad_otf(a.f, a.nz, a.ny, a.nx, (int)zz, (int)yy, (int)xx, g0, g1, g2);
                }
                const float X = (float)dx, Y = (float)dy, Z = (float)dz;
                // this part's gradient products: (00, 01, 02) or (11, 12, 22)
                const float ga = part == 0 ? g0 : g1, gb = part == 0 ? g1 : g2;
                const float gg[3] = {ga * ga, ga * gb, part == 0 ? g0 * g2 : g2 * g2};
                const float xq[10] = {X * X, X * Y, X * Z, X, Y * Y, Y * Z, Y, Z * Z, Z, 1.0f};
#pragma unroll
                for (int p = 0; p < 3; ++p)
#pragma unroll
                    for (int q = 0; q < 10; ++q) blk[p * 10 + q] = fmaf(gg[p], xq[q], blk[p * 10 + q]);
                blk[30] += part == 0 ? fv : fv * fv;
                if (part == 0) ++n;
            }
            if (++in_blk == PRE_BLOCK) {  // fold the block sums into the compensated totals
                in_blk = 0;
#pragma unroll
                for (int i = 0; i < 31; ++i) {
                    float su = ksum[i * PRE_THREADS], cm = kcmp[i * PRE_THREADS];
                    kahan_add(su, cm, blk[i]);
                    ksum[i * PRE_THREADS] = su;
                    kcmp[i * PRE_THREADS] = cm;
                    blk[i] = 0.0f;
                }
            }
            ix += st_x;
            if (ix >= nX) {
                ix -= nX;
                ++iy;
            }
            iy += st_y;
            if (iy >= nY) {
                iy -= nY;
                ++iz;
            }
            iz += st_z;
        }
#pragma unroll
        for (int i = 0; i < 31; ++i) {
            float su = ksum[i * PRE_THREADS], cm = kcmp[i * PRE_THREADS];
            kahan_add(su, cm, blk[i]);
            const double t = warp_sum_d((double)su - (double)cm);
            if (lane == 0) red[warp][i < 30 ? 30 * part + i : 60 + part] = t;
        }
    }
    n = warp_sum_i(n);
    if (lane == 0) red_n[warp] = n;
    __syncthreads();
    if (tid < PRE_NSUM) {
        double s = 0.0;
        for (int w = 0; w < PRE_THREADS / 32; ++w) s += red[w][tid];
        tot[tid] = s;
    }
    __syncthreads();
    if (tid != 0) return;
    int64_t nv = 0;
    for (int w = 0; w < PRE_THREADS / 32; ++w) nv += red_n[w];
    // assemble H over SD = [g0 X, g0 Y, g0 Z, g1 X, g1 Y, g1 Z, g2 X, g2 Y, g2 Z, g0, g1, g2]
    auto comp = [](int a_) { return a_ < 9 ? a_ / 3 : a_ - 9; };
    auto coord = [](int a_) { return a_ < 9 ? a_ % 3 : 3; };
    double Hl[144];
    for (int p = 0; p < 12; ++p)
        for (int q = 0; q < 12; ++q) Hl[p * 12 + q] = tot[gg_index(comp(p), comp(q)) * 10 + xx_index(coord(p), coord(q))];
    for (int i = 0; i < 144; ++i) H[i] = Hl[i];
    a.n_valid[node] = nv;
    const int64_t total = subset_count(hx, hy, hz, a.stride);
    double Ll[144];
    for (int i = 0; i < 144; ++i) Ll[i] = 0.0;
    bool ok = !(nv < 27 || (double)nv < a.min_valid_ratio * (double)total);
    double meanf = 0.0, bottomf = 1.0;
    if (ok) {
        const double m_rel = tot[60] / (double)nv;
        meanf = (double)pilot + m_rel;
        double ssf = tot[61] - (double)nv * m_rel * m_rel;
        if (ssf < 0.0) ssf = 0.0;
        bottomf = sqrt(ssf > 1e-30 ? ssf : 1e-30);
        if (bottomf < 1e-10) ok = false;
        if (ok) ok = chol12(Hl, Ll);
        if (ok) {
            double dmin = Ll[0], dmax = Ll[0];
            for (int i = 1; i < 12; ++i) {
                const double d = Ll[i * 12 + i];
                dmin = d < dmin ? d : dmin;
                dmax = d > dmax ? d : dmax;
            }
            if (dmin <= 0.0 || (dmax / dmin) * (dmax / dmin) > a.cond_max) ok = false;
        }
    }
    for (int i = 0; i < 144; ++i) L[i] = Ll[i];
    a.meanf[node] = meanf;
    a.bottomf[node] = bottomf;
    a.valid[node] = ok ? 1 : 0;
}

// ----------------------------------------------------------------------------- node grids, separable form
// On a tensor grid of nodes (x centres xs, y centres ys, z centres zs) with no split rows, one subset shape,
// stride 1 and stored gradients (a mask allowed: its voxels drop out of every sum and the count), every node's 60 Hessian moments sum g_a g_b X^i Y^j Z^k (i + j + k <= 2)
// factor along the axes: pass x sums each product against 1, X, X^2 along the node's x window for every voxel row
// (z, y) (FP32 with Kahan compensation, 33 terms for a 32-voxel subset), pass y sums those rows against 1, Y, Y^2
// for every plane z (FP64), pass z against 1, Z, Z^2 (FP64), so the subset is swept once per row instead of once
// per node.  Sum f and sum f^2 follow the same path relative to the row, plane and node centre voxels, shifted
// exactly in FP64 between the passes, so they are taken relative to the node's centre voxel as in precompute_kernel.
constexpr int PG_X = 21;  // per row and node column: 6 products x (1, X, X^2), sum (f - c), sum (f - c)^2, voxel count
constexpr int PG_Y = 39;  // per plane and node: 6 products x (1, X, X^2, Y, XY, Y^2), f sums, voxel count

struct PreGridArgs {
    const float* f;
    const float* gx;
    const float* gy;
    const float* gz;
    const uint8_t* mask;  // NULL: every voxel
    int nz, ny, nx;
    int hx, hy, hz;
    const int64_t* xs;
    const int64_t* ys;
    const int64_t* zs;
    int ngx, ngy, ngz;
    float* Mx;   // [PG_X][nz][ny][ngx]
    double* My;  // [PG_Y][nz][ngy][ngx]
    double min_valid_ratio, cond_max;
    double* H;
    double* L;
    double* meanf;
    double* bottomf;
    int64_t* n_valid;
    uint8_t* valid;
};

// pass x: one CTA per voxel row (z, y), the row of f, gx, gy, gz (and the mask) staged in shared memory, one thread
// per node column; voxels outside the mask add nothing and are not counted
__global__ void __launch_bounds__(128) pregrid_x_kernel(PreGridArgs a) {
    extern __shared__ float prow[];  // [5][nx]: f, gx, gy, gz, mask (0 / 1)
    const int y = blockIdx.x, z = blockIdx.y;
    const int64_t ro = ((int64_t)z * a.ny + y) * a.nx;
    for (int x = threadIdx.x; x < a.nx; x += blockDim.x) {
        prow[x] = __ldg(a.f + ro + x);
        prow[a.nx + x] = __ldg(a.gx + ro + x);
        prow[2 * a.nx + x] = __ldg(a.gy + ro + x);
        prow[3 * a.nx + x] = __ldg(a.gz + ro + x);
        prow[4 * a.nx + x] = (a.mask == nullptr || __ldg(a.mask + ro + x) != 0) ? 1.0f : 0.0f;
    }
    __syncthreads();
    const int64_t plane = (int64_t)a.nz * a.ny * a.ngx, oi = ((int64_t)z * a.ny + y) * a.ngx;
    for (int c = threadIdx.x; c < a.ngx; c += blockDim.x) {
        const int64_t xc = a.xs[c];
        float sum[PG_X - 1], cmp[PG_X - 1];
#pragma unroll
        for (int k = 0; k < PG_X - 1; ++k) sum[k] = cmp[k] = 0.0f;
        int count = 0;
        if (xc - a.hx >= 0 && xc + a.hx < a.nx) {  // a column past the volume edge belongs to invalid nodes only
            const float cf = prow[xc];
            for (int d = -a.hx; d <= a.hx; ++d) {
                const int x = (int)xc + d;
                if (prow[4 * a.nx + x] == 0.0f) continue;
                ++count;
                const float g0 = prow[a.nx + x], g1 = prow[2 * a.nx + x], g2 = prow[3 * a.nx + x];
                const float X = (float)d, X2 = X * X, fv = prow[x] - cf;
                const float gg[6] = {g0 * g0, g0 * g1, g0 * g2, g1 * g1, g1 * g2, g2 * g2};
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    kahan_add(sum[3 * q], cmp[3 * q], gg[q]);
                    kahan_add(sum[3 * q + 1], cmp[3 * q + 1], gg[q] * X);
                    kahan_add(sum[3 * q + 2], cmp[3 * q + 2], gg[q] * X2);
                }
                kahan_add(sum[18], cmp[18], fv);
                kahan_add(sum[19], cmp[19], fv * fv);
            }
        }
#pragma unroll
        for (int k = 0; k < PG_X - 1; ++k) a.Mx[k * plane + oi + c] = sum[k] - cmp[k];
        a.Mx[20 * plane + oi + c] = (float)count;
    }
}

// pass y: one thread per (z, node row, node column), FP64
__global__ void __launch_bounds__(128) pregrid_y_kernel(PreGridArgs a) {
    const int64_t n = (int64_t)a.nz * a.ngy * a.ngx;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = (int)(i % a.ngx), r = (int)((i / a.ngx) % a.ngy), z = (int)(i / ((int64_t)a.ngx * a.ngy));
    const int64_t yc = a.ys[r], xc = a.xs[c];
    double acc[PG_Y];
#pragma unroll
    for (int k = 0; k < PG_Y; ++k) acc[k] = 0.0;
    const int64_t xplane = (int64_t)a.nz * a.ny * a.ngx, yplane = (int64_t)a.nz * a.ngy * a.ngx;
    if (yc - a.hy >= 0 && yc + a.hy < a.ny && xc - a.hx >= 0 && xc + a.hx < a.nx) {
        const int64_t sxy = (int64_t)a.nx * a.ny;
        const double c2 = (double)__ldg(a.f + z * sxy + yc * a.nx + xc);  // this plane's centre voxel
        for (int d = -a.hy; d <= a.hy; ++d) {
            const int64_t y = yc + d;
            const int64_t o = ((int64_t)z * a.ny + y) * a.ngx + c;
            const double Y = (double)d, Y2 = Y * Y;
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                const double m0 = a.Mx[(3 * q) * xplane + o], m1 = a.Mx[(3 * q + 1) * xplane + o], m2 = a.Mx[(3 * q + 2) * xplane + o];
                acc[6 * q + 0] += m0;      // 1
                acc[6 * q + 1] += m1;      // X
                acc[6 * q + 2] += m2;      // X^2
                acc[6 * q + 3] += m0 * Y;  // Y
                acc[6 * q + 4] += m1 * Y;  // XY
                acc[6 * q + 5] += m0 * Y2; // Y^2
            }
            // the row's sums are relative to its centre voxel cr: shift them to c2
            const double cr = (double)__ldg(a.f + z * sxy + y * a.nx + xc), s = cr - c2;
            const double a0 = a.Mx[18 * xplane + o], a1 = a.Mx[19 * xplane + o], cnt = a.Mx[20 * xplane + o];
            acc[36] += a0 + cnt * s;
            acc[37] += a1 + 2.0 * s * a0 + cnt * s * s;
            acc[38] += cnt;
        }
    }
    const int64_t oo = ((int64_t)z * a.ngy + r) * a.ngx + c;
#pragma unroll
    for (int k = 0; k < PG_Y; ++k) a.My[k * yplane + oo] = acc[k];
}

// pass z and the per-node finish of precompute_kernel: one thread per node
__global__ void __launch_bounds__(64) pregrid_z_kernel(PreGridArgs a) {
    const int64_t n_nodes = (int64_t)a.ngz * a.ngy * a.ngx;
    const int64_t node = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (node >= n_nodes) return;
    const int c = (int)(node % a.ngx), r = (int)((node / a.ngx) % a.ngy), t = (int)(node / ((int64_t)a.ngx * a.ngy));
    const int64_t xc = a.xs[c], yc = a.ys[r], zc = a.zs[t];
    double* H = a.H + node * 144;
    double* L = a.L + node * 144;
    const bool inside = xc - a.hx >= 0 && xc + a.hx < a.nx && yc - a.hy >= 0 && yc + a.hy < a.ny && zc - a.hz >= 0 && zc + a.hz < a.nz;
    if (!inside) {
        for (int i = 0; i < 144; ++i) H[i] = L[i] = 0.0;
        a.meanf[node] = 0.0;
        a.bottomf[node] = 1.0;
        a.n_valid[node] = 0;
        a.valid[node] = 0;
        return;
    }
    const int64_t sxy = (int64_t)a.nx * a.ny, yplane = (int64_t)a.nz * a.ngy * a.ngx;
    const double p = (double)__ldg(a.f + zc * sxy + yc * a.nx + xc);  // the node's centre voxel
    double tot[PRE_NSUM], nvd = 0.0;
    for (int k = 0; k < PRE_NSUM; ++k) tot[k] = 0.0;
    for (int d = -a.hz; d <= a.hz; ++d) {
        const int64_t z = zc + d;
        const int64_t o = (z * a.ngy + r) * a.ngx + c;
        const double Z = (double)d, Z2 = Z * Z;
        for (int q = 0; q < 6; ++q) {
            const double* m = a.My + (6 * q) * yplane + o;
            const double m1 = m[0], mX = m[yplane], mXX = m[2 * yplane], mY = m[3 * yplane], mXY = m[4 * yplane], mYY = m[5 * yplane];
            double* tq = tot + 10 * q;  // XX XY XZ X YY YZ Y ZZ Z 1
            tq[0] += mXX;
            tq[1] += mXY;
            tq[2] += mX * Z;
            tq[3] += mX;
            tq[4] += mYY;
            tq[5] += mY * Z;
            tq[6] += mY;
            tq[7] += m1 * Z2;
            tq[8] += m1 * Z;
            tq[9] += m1;
        }
        const double cz = (double)__ldg(a.f + z * sxy + yc * a.nx + xc), s = cz - p;
        const double b0 = a.My[36 * yplane + o], b1 = a.My[37 * yplane + o], cnt = a.My[38 * yplane + o];
        tot[60] += b0 + cnt * s;
        tot[61] += b1 + 2.0 * s * b0 + cnt * s * s;
        nvd += cnt;
    }
    const int64_t nv = (int64_t)nvd, total = subset_count(a.hx, a.hy, a.hz, 1);
    auto comp = [](int a_) { return a_ < 9 ? a_ / 3 : a_ - 9; };
    auto coord = [](int a_) { return a_ < 9 ? a_ % 3 : 3; };
    double Hl[144], Ll[144];
    for (int pp = 0; pp < 12; ++pp)
        for (int qq = 0; qq < 12; ++qq) Hl[pp * 12 + qq] = tot[gg_index(comp(pp), comp(qq)) * 10 + xx_index(coord(pp), coord(qq))];
    for (int i = 0; i < 144; ++i) {
        H[i] = Hl[i];
        Ll[i] = 0.0;
    }
    a.n_valid[node] = nv;
    bool ok = !(nv < 27 || (double)nv < a.min_valid_ratio * (double)total);
    double meanf = 0.0, bottomf = 1.0;
    if (ok) {
        const double m_rel = tot[60] / (double)nv;
        meanf = p + m_rel;
        double ssf = tot[61] - (double)nv * m_rel * m_rel;
        if (ssf < 0.0) ssf = 0.0;
        bottomf = sqrt(ssf > 1e-30 ? ssf : 1e-30);
        if (bottomf < 1e-10) ok = false;
        if (ok) ok = chol12(Hl, Ll);
        if (ok) {
            double dmin = Ll[0], dmax = Ll[0];
            for (int i = 1; i < 12; ++i) {
                const double dd = Ll[i * 12 + i];
                dmin = dd < dmin ? dd : dmin;
                dmax = dd > dmax ? dd : dmax;
            }
            if (dmin <= 0.0 || (dmax / dmin) * (dmax / dmin) > a.cond_max) ok = false;
        }
    }
    for (int i = 0; i < 144; ++i) L[i] = Ll[i];
    a.meanf[node] = meanf;
    a.bottomf[node] = bottomf;
    a.valid[node] = ok ? 1 : 0;
}

}  // namespace aldvc

using namespace aldvc;

extern "C" int aldvc_precompute(const aldvc_volumes* vol, const aldvc_subset* sub, const int64_t* coords, int64_t n_nodes,
                                double min_valid_ratio, double cond_max, double* H_all, double* L_all, double* meanf,
                                double* bottomf, int64_t* n_valid, uint8_t* valid, void* stream) {
    ALDVC_REQUIRE(vol && sub, "aldvc_precompute: null descriptor");
    ALDVC_REQUIRE(vol->f && coords && H_all && L_all && meanf && bottomf && n_valid && valid, "aldvc_precompute: null pointer");
    ALDVC_REQUIRE(sub->hx >= 0 && sub->hy >= 0 && sub->hz >= 0 && sub->stride >= 1, "aldvc_precompute: bad subset");
    ALDVC_REQUIRE(vol->nz > 0 && vol->ny > 0 && vol->nx > 0 && vol->nz < (1 << 30) && vol->ny < (1 << 30) && vol->nx < (1 << 30),
                  "aldvc_precompute: bad volume shape");
    const bool stored = vol->gx && vol->gy && vol->gz;
    ALDVC_REQUIRE(stored || (!vol->gx && !vol->gy && !vol->gz), "aldvc_precompute: give all three gradients or none");
    ALDVC_REQUIRE(!sub->split_index || (sub->split_keep && sub->keep_bytes > 0), "aldvc_precompute: split rows missing");
    ALDVC_REQUIRE(!(sub->node_half && sub->split_index), "aldvc_precompute: per-node shapes do not combine with split rows");
    if (n_nodes <= 0) return ALDVC_OK;
    ALDVC_REQUIRE(n_nodes < (1LL << 31), "aldvc_precompute: too many nodes");
    PreArgs a{vol->f, vol->gx, vol->gy, vol->gz, vol->mask, (int)vol->nz, (int)vol->ny, (int)vol->nx, sub->hx, sub->hy, sub->hz,
              sub->stride, sub->split_index, sub->split_keep, sub->keep_bytes, coords, n_nodes, min_valid_ratio, cond_max,
              H_all, L_all, meanf, bottomf, n_valid, valid, sub->node_half};
    cudaStream_t s = (cudaStream_t)stream;
    constexpr size_t KAH = (size_t)2 * 31 * PRE_THREADS * sizeof(float);
    static bool attr[2] = {false, false};  // set once per instantiation, outside any capture (the first call)
    if (!attr[stored ? 1 : 0]) {
        cudaError_t e = stored ? cudaFuncSetAttribute(precompute_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)KAH)
                               : cudaFuncSetAttribute(precompute_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)KAH);
        if (e != cudaSuccess) return cuda_fail(e, "aldvc_precompute: shared memory attribute");
        attr[stored ? 1 : 0] = true;
    }
    if (stored)
        {
            KTimer kt_("precompute", s);
            precompute_kernel<true><<<(unsigned)n_nodes, PRE_THREADS, KAH, s>>>(a);
        }
    else
        {
            KTimer kt_("precompute", s);
            precompute_kernel<false><<<(unsigned)n_nodes, PRE_THREADS, KAH, s>>>(a);
        }
    return check_launch("aldvc_precompute");
}

extern "C" size_t aldvc_precompute_grid_workspace_size(int64_t nz, int64_t ny, int64_t nx, int64_t ngx, int64_t ngy) {
    return (size_t)PG_X * nz * ny * ngx * sizeof(float) + 256 + (size_t)PG_Y * nz * ngy * ngx * sizeof(double);
}

extern "C" int aldvc_precompute_grid(const aldvc_volumes* vol, const aldvc_subset* sub, const int64_t* xs, int64_t ngx, const int64_t* ys,
                                     int64_t ngy, const int64_t* zs, int64_t ngz, double min_valid_ratio, double cond_max, double* H_all,
                                     double* L_all, double* meanf, double* bottomf, int64_t* n_valid, uint8_t* valid, void* workspace,
                                     size_t workspace_bytes, void* stream) {
    ALDVC_REQUIRE(vol && sub, "aldvc_precompute_grid: null descriptor");
    ALDVC_REQUIRE(vol->f && vol->gx && vol->gy && vol->gz && xs && ys && zs && H_all && L_all && meanf && bottomf && n_valid && valid &&
                      workspace,
                  "aldvc_precompute_grid: null pointer (the gradients must be stored)");
    ALDVC_REQUIRE(!sub->split_index && !sub->node_half && sub->stride == 1,
                  "aldvc_precompute_grid: split rows, per-node shapes and strides take aldvc_precompute");
    ALDVC_REQUIRE(sub->hx >= 0 && sub->hy >= 0 && sub->hz >= 0, "aldvc_precompute_grid: bad subset");
    ALDVC_REQUIRE(vol->nz > 0 && vol->ny > 0 && vol->nx > 0 && vol->nz <= 65535 && vol->ny <= 65535 && vol->nx <= 8192,
                  "aldvc_precompute_grid: volume shape (nz, ny <= 65535, nx <= 8192)");
    ALDVC_REQUIRE(ngx > 0 && ngy > 0 && ngz > 0 && ngx * ngy * ngz < (1LL << 31), "aldvc_precompute_grid: node grid");
    ALDVC_REQUIRE(workspace_bytes >= aldvc_precompute_grid_workspace_size(vol->nz, vol->ny, vol->nx, ngx, ngy),
                  "aldvc_precompute_grid: workspace");
    const size_t xbytes = (size_t)PG_X * vol->nz * vol->ny * ngx * sizeof(float);
    PreGridArgs a{vol->f, vol->gx, vol->gy, vol->gz, vol->mask, (int)vol->nz, (int)vol->ny, (int)vol->nx, sub->hx, sub->hy, sub->hz, xs, ys, zs,
                  (int)ngx, (int)ngy, (int)ngz, (float*)workspace, (double*)((char*)workspace + align_up(xbytes, 256)), min_valid_ratio,
                  cond_max, H_all, L_all, meanf, bottomf, n_valid, valid};
    cudaStream_t s = (cudaStream_t)stream;
    const size_t row_smem = (size_t)5 * vol->nx * sizeof(float);
    static int attr = 0;  // largest dynamic shared size set so far (the first call sets it, outside any capture)
    if (row_smem > 48 * 1024 && (int)row_smem > attr) {
        cudaError_t e = cudaFuncSetAttribute(pregrid_x_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)row_smem);
        if (e != cudaSuccess) return cuda_fail(e, "aldvc_precompute_grid: shared memory attribute");
        attr = (int)row_smem;
    }
    const int64_t ny_planes = (int64_t)vol->nz * ngy * ngx, nodes = ngz * ngy * ngx;
    {
        KTimer kt_("precompute", s);
        pregrid_x_kernel<<<dim3((unsigned)vol->ny, (unsigned)vol->nz), 128, row_smem, s>>>(a);
        pregrid_y_kernel<<<(unsigned)((ny_planes + 127) / 128), 128, 0, s>>>(a);
        pregrid_z_kernel<<<(unsigned)((nodes + 63) / 64), 64, 0, s>>>(a);
    }
    return check_launch("aldvc_precompute_grid");
}
