// Node-grid post-processing of the local solvers, on the device so a whole AL-DVC pass needs no host step.
//
// aldvc_inpaint       <- utils/inpaint.fill_nan_grid (:35-125), "spring" model: for every unknown node
//                        sum over its 6 grid neighbours (x_u - x_n) = 0 with the known nodes as Dirichlet
//                        data plus a 1e-10 Tikhonov term; solved by CG on the unknowns (one cooperative
//                        kernel, bounded grid barriers), all columns at once.
// aldvc_median_test   <- utils/outlier_detection.universal_median_test (:135-160) without a cut mesh:
//                        invalid nodes inpainted, 26-neighbour median with nearest-edge padding (the
//                        upper median, scipy.ndimage.median_filter's rank size//2), normalised fluctuation
//                        |u - med| / (median of the neighbours' |u - med| + eps), flagged above threshold.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "common.cuh"
#include "internal.cuh"

namespace aldvc {

constexpr int PP_THREADS = 256;
constexpr int MAX_COLS = 12;

struct Grid3 {
    int nx, ny, nz;
    int64_t n;
};

__device__ __forceinline__ void grid_xyz(const Grid3& g, int64_t n, int& ix, int& iy, int& iz) {
    ix = (int)(n % g.nx);
    const int64_t r = n / g.nx;
    iy = (int)(r % g.ny);
    iz = (int)(r / g.ny);
}

struct InpArgs {
    Grid3 g;
    int C;
    double* vals;        // (N, C) in/out
    const uint8_t* unk;  // (N,) 1 = unknown
    double tol;
    int max_iter;
    double* R;
    double* P;
    double* AP;
    double* X;
    double* part;
    unsigned int* bar;
    unsigned int bar_extra;  // arrivals beyond the grid before a barrier opens (0; > 0 only in the give-up tests)
    long long spin_limit;    // polls before a waiting block gives up
    int32_t* iters;
    int32_t* err;
};

// Grid-wide barrier of the cooperative inpainting kernel; bounded wait: on give-up the error word is set
// and the caller returns.
__device__ bool pp_grid_sync(const InpArgs& a) {
    unsigned int* bar = a.bar;
    int32_t* err = a.err;
    __syncthreads();
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        volatile unsigned int* gen = bar + 1;
        const unsigned int g0 = *gen;
        __threadfence();
        const unsigned int arrived = atomicAdd(bar, 1u) + 1u;
        int ok = 1;
        if (arrived == gridDim.x + a.bar_extra) {
            bar[0] = 0u;
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long spins = 0;
            while (*gen == g0) {
                if (++spins > a.spin_limit) {
                    atomicExch(err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        if (*(volatile int32_t*)err != 0) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// block partials of k <= 2*MAX_COLS values, then a fixed-order total over blocks (every block)
__device__ void pp_partials(double* part, int slot, const double* v, int k) {
    __shared__ double red[PP_THREADS / 32][2 * MAX_COLS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = 0; i < k; ++i) {
        const double s = warp_sum_d(v[i]);
        if (lane == 0) red[warp][i] = s;
    }
    __syncthreads();
    if (threadIdx.x < k) {
        double s = 0.0;
        for (int w = 0; w < PP_THREADS / 32; ++w) s += red[w][threadIdx.x];
        part[((int64_t)slot * gridDim.x + blockIdx.x) * (2 * MAX_COLS) + threadIdx.x] = s;
    }
    __syncthreads();
}

__device__ void pp_total(const double* part, int slot, int k, double* out) {
    __shared__ double red[PP_THREADS / 32][2 * MAX_COLS];
    __shared__ double tot[2 * MAX_COLS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double v[2 * MAX_COLS];
    for (int i = 0; i < k; ++i) v[i] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
        for (int i = 0; i < k; ++i) v[i] += part[((int64_t)slot * gridDim.x + b) * (2 * MAX_COLS) + i];
    for (int i = 0; i < k; ++i) {
        const double s = warp_sum_d(v[i]);
        if (lane == 0) red[warp][i] = s;
    }
    __syncthreads();
    if (threadIdx.x < k) {
        double s = 0.0;
        for (int w = 0; w < PP_THREADS / 32; ++w) s += red[w][threadIdx.x];
        tot[threadIdx.x] = s;
    }
    __syncthreads();
    for (int i = 0; i < k; ++i) out[i] = tot[i];
    __syncthreads();
}

// (A x)_u for unknown u: (deg(u) + 1e-10) x_u - sum_{unknown nbrs} x_n; known nodes carry x = 0
__device__ __forceinline__ double lap_apply(const InpArgs& a, int64_t n, int ix, int iy, int iz, const double* x, int c) {
    double deg = 0.0, s = 0.0;
    const int nb[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    for (int k = 0; k < 6; ++k) {
        const int jx = ix + nb[k][0], jy = iy + nb[k][1], jz = iz + nb[k][2];
        if (jx < 0 || jy < 0 || jz < 0 || jx >= a.g.nx || jy >= a.g.ny || jz >= a.g.nz) continue;
        deg += 1.0;
        const int64_t j = ((int64_t)jz * a.g.ny + jy) * a.g.nx + jx;
        if (a.unk[j]) s += x[j * a.C + c];
    }
    return (deg + 1e-10) * x[n * a.C + c] - s;
}

__global__ void __launch_bounds__(PP_THREADS) inpaint_cg_kernel(InpArgs a) {
    const int64_t N = a.g.n;
    const int C = a.C;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int nb[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    double loc[2 * MAX_COLS];
    for (int i = 0; i < 2 * MAX_COLS; ++i) loc[i] = 0.0;
    // x0 = 0 on the unknowns; r = b = sum of known neighbour values; p = r
    for (int64_t n = t0; n < N; n += stride) {
        for (int c = 0; c < C; ++c) a.X[n * C + c] = 0.0;
        if (!a.unk[n]) {
            for (int c = 0; c < C; ++c) a.R[n * C + c] = a.P[n * C + c] = 0.0;
            continue;
        }
        int ix, iy, iz;
        grid_xyz(a.g, n, ix, iy, iz);
        double b[MAX_COLS];
        for (int c = 0; c < C; ++c) b[c] = 0.0;
        for (int k = 0; k < 6; ++k) {
            const int jx = ix + nb[k][0], jy = iy + nb[k][1], jz = iz + nb[k][2];
            if (jx < 0 || jy < 0 || jz < 0 || jx >= a.g.nx || jy >= a.g.ny || jz >= a.g.nz) continue;
            const int64_t j = ((int64_t)jz * a.g.ny + jy) * a.g.nx + jx;
            if (!a.unk[j])
                for (int c = 0; c < C; ++c) b[c] += a.vals[j * C + c];
        }
        for (int c = 0; c < C; ++c) {
            a.R[n * C + c] = b[c];
            a.P[n * C + c] = b[c];
            loc[c] += b[c] * b[c];
        }
    }
    pp_partials(a.part, 0, loc, C);
    if (!pp_grid_sync(a)) return;
    double tot[2 * MAX_COLS], rr[MAX_COLS], bn[MAX_COLS];
    pp_total(a.part, 0, C, tot);
    for (int c = 0; c < C; ++c) {
        rr[c] = tot[c];
        bn[c] = sqrt(tot[c]);
        if (bn[c] == 0.0) bn[c] = 1.0;
    }
    bool conv0 = true;
    for (int c = 0; c < C; ++c) conv0 = conv0 && (sqrt(rr[c]) / bn[c] < a.tol);
    int it = 0;
    if (!conv0) {
        for (it = 1; it <= a.max_iter; ++it) {
            for (int i = 0; i < C; ++i) loc[i] = 0.0;
            for (int64_t n = t0; n < N; n += stride) {
                if (!a.unk[n]) continue;
                int ix, iy, iz;
                grid_xyz(a.g, n, ix, iy, iz);
                for (int c = 0; c < C; ++c) {
                    const double ap = lap_apply(a, n, ix, iy, iz, a.P, c);
                    a.AP[n * C + c] = ap;
                    loc[c] += a.P[n * C + c] * ap;
                }
            }
            pp_partials(a.part, 1, loc, C);
            if (!pp_grid_sync(a)) return;
            pp_total(a.part, 1, C, tot);
            double al[MAX_COLS];
            for (int c = 0; c < C; ++c) al[c] = tot[c] > 0.0 ? rr[c] / tot[c] : 0.0;
            for (int i = 0; i < C; ++i) loc[i] = 0.0;
            for (int64_t n = t0; n < N; n += stride) {
                if (!a.unk[n]) continue;
                for (int c = 0; c < C; ++c) {
                    a.X[n * C + c] += al[c] * a.P[n * C + c];
                    const double r = a.R[n * C + c] - al[c] * a.AP[n * C + c];
                    a.R[n * C + c] = r;
                    loc[c] += r * r;
                }
            }
            pp_partials(a.part, 2, loc, C);
            if (!pp_grid_sync(a)) return;
            pp_total(a.part, 2, C, tot);
            bool conv = true;
            double be[MAX_COLS];
            for (int c = 0; c < C; ++c) {
                conv = conv && (sqrt(tot[c]) / bn[c] < a.tol);
                be[c] = rr[c] > 0.0 ? tot[c] / rr[c] : 0.0;
                rr[c] = tot[c];
            }
            if (conv) break;
            for (int64_t n = t0; n < N; n += stride) {
                if (!a.unk[n]) continue;
                for (int c = 0; c < C; ++c) a.P[n * C + c] = a.R[n * C + c] + be[c] * a.P[n * C + c];
            }
            if (!pp_grid_sync(a)) return;
        }
    }
    for (int64_t n = t0; n < N; n += stride)
        if (a.unk[n])
            for (int c = 0; c < C; ++c) a.vals[n * C + c] = a.X[n * C + c];
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.iters = it > a.max_iter ? a.max_iter : it;
}

// 26-neighbour median (rank 13 of 26, nearest-edge padding) of column c of a (N, C) field
__device__ double median26(const Grid3& g, const double* v, int C, int c, int ix, int iy, int iz) {
    double w[26];
    int k = 0;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                if (dx == 0 && dy == 0 && dz == 0) continue;
                const int jx = min(max(ix + dx, 0), g.nx - 1), jy = min(max(iy + dy, 0), g.ny - 1),
                          jz = min(max(iz + dz, 0), g.nz - 1);
                w[k++] = v[(((int64_t)jz * g.ny + jy) * g.nx + jx) * C + c];
            }
    // partial selection sort up to rank 13
    for (int i = 0; i <= 13; ++i) {
        int m = i;
        for (int j = i + 1; j < 26; ++j)
            if (w[j] < w[m]) m = j;
        const double t = w[i];
        w[i] = w[m];
        w[m] = t;
    }
    return w[13];
}

struct MedArgs {
    Grid3 g;
    int C;
    const double* field;  // (N, C) after inpainting
    double* absfl;        // (N, C) |field - med|
    double* mag2;         // (N,)
    const uint8_t* nanmask;
    const uint8_t* valid;
    double threshold, eps;
    uint8_t* flag;
};

__global__ void med_fluct_kernel(MedArgs a) {
    const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (n >= a.g.n) return;
    int ix, iy, iz;
    grid_xyz(a.g, n, ix, iy, iz);
    for (int c = 0; c < a.C; ++c) a.absfl[n * a.C + c] = fabs(a.field[n * a.C + c] - median26(a.g, a.field, a.C, c, ix, iy, iz));
}

__global__ void med_flag_kernel(MedArgs a) {
    const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (n >= a.g.n) return;
    int ix, iy, iz;
    grid_xyz(a.g, n, ix, iy, iz);
    double m2 = 0.0;
    for (int c = 0; c < a.C; ++c) {
        const double r = a.absfl[n * a.C + c];
        double nf = r / (median26(a.g, a.absfl, a.C, c, ix, iy, iz) + a.eps);
        if (a.nanmask[n] || !isfinite(nf)) nf = 0.0;
        m2 += nf * nf;
    }
    const bool v = a.valid == nullptr || a.valid[n] != 0;
    a.flag[n] = (sqrt(m2) > a.threshold && v) ? 1 : 0;
}

// unknown mask of the median test: invalid or NaN in any column
__global__ void nanmask_kernel(const double* field, int C, int64_t n, const uint8_t* valid, uint8_t* out, double* copy) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool bad = valid != nullptr && valid[i] == 0;
    for (int c = 0; c < C; ++c) {
        const double v = field[i * C + c];
        bad = bad || !(v == v);
        copy[i * C + c] = v;
    }
    out[i] = bad ? 1 : 0;
}

static std::mutex g_inp_grid_mu;
static int g_inp_grid[128] = {0};  // co-resident grid of the cooperative inpainting kernel, per device ordinal

// queried once per device: no configuration call inside a stream capture after the first use
static int inpaint_grid(int* grid) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "inpaint: current device");
    if (dev < 0 || dev >= 128) return arg_fail("inpaint: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_inp_grid_mu);
    if (g_inp_grid[dev] == 0) {
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, inpaint_cg_kernel, PP_THREADS, 0);
        if (e != cudaSuccess) return cuda_fail(e, "inpaint: occupancy");
        if (per_sm < 1) return arg_fail("inpaint: kernel does not fit");
        cudaDeviceProp p;
        e = cudaGetDeviceProperties(&p, dev);
        if (e != cudaSuccess) return cuda_fail(e, "inpaint: device properties");
        g_inp_grid[dev] = per_sm * p.multiProcessorCount;
    }
    *grid = g_inp_grid[dev];
    return ALDVC_OK;
}

static size_t inpaint_ws(int64_t n, int C, int grid) {
    return 4 * align_up((size_t)n * C * sizeof(double), 256) + align_up((size_t)3 * grid * 2 * MAX_COLS * sizeof(double), 256) +
           256;
}

static int run_inpaint(const Grid3& g, int C, double* vals, const uint8_t* unk, double tol, int max_iter, char* ws, size_t ws_bytes,
                       int32_t* iters, int32_t* err, cudaStream_t s) {
    int grid = 0;
    int rc = inpaint_grid(&grid);
    if (rc) return rc;
    if (ws_bytes < inpaint_ws(g.n, C, grid)) return arg_fail("inpaint: workspace too small");
    InpArgs a;
    a.g = g;
    a.C = C;
    a.vals = vals;
    a.unk = unk;
    a.tol = tol;
    a.max_iter = max_iter;
    const size_t v = align_up((size_t)g.n * C * sizeof(double), 256);
    a.R = (double*)ws;
    a.P = (double*)(ws + v);
    a.AP = (double*)(ws + 2 * v);
    a.X = (double*)(ws + 3 * v);
    a.part = (double*)(ws + 4 * v);
    a.bar = (unsigned int*)(ws + 4 * v + align_up((size_t)3 * grid * 2 * MAX_COLS * sizeof(double), 256));
    const BarrierParams bp = barrier_params();
    a.bar_extra = bp.extra;
    a.spin_limit = bp.spin_limit;
    a.iters = iters;
    a.err = err;
    cudaError_t e = cudaMemsetAsync(a.bar, 0, 2 * sizeof(unsigned int), s);
    if (e != cudaSuccess) return cuda_fail(e, "inpaint: barrier reset");
    void* args[] = {&a};
    {
        KTimer kt_("inpaint_cg", s);
        e = cudaLaunchCooperativeKernel((const void*)inpaint_cg_kernel, dim3(grid), dim3(PP_THREADS), args, 0, s);
    }
    if (e != cudaSuccess) return cuda_fail(e, "inpaint: cooperative launch");
    count_launch();
    return ALDVC_OK;
}

static int make_grid(int64_t nz, int64_t ny, int64_t nx, Grid3& g) {
    if (nz < 1 || ny < 1 || nx < 1 || nz >= (1 << 30) || ny >= (1 << 30) || nx >= (1 << 30)) return arg_fail("grid: bad shape");
    g.nx = (int)nx;
    g.ny = (int)ny;
    g.nz = (int)nz;
    g.n = nx * ny * nz;
    return ALDVC_OK;
}

}  // namespace aldvc

using namespace aldvc;

extern "C" size_t aldvc_inpaint_workspace_size(int64_t nz, int64_t ny, int64_t nx, int32_t ncols) {
    int grid = 0;
    if (inpaint_grid(&grid) != ALDVC_OK) grid = 148 * 8;
    return inpaint_ws(nx * ny * nz, std::max(1, (int)ncols), grid);
}

extern "C" int aldvc_inpaint(double* values, int64_t nz, int64_t ny, int64_t nx, int32_t ncols, const uint8_t* unknown, double tol,
                             int32_t max_iter, void* workspace, size_t workspace_bytes, int32_t* iters, int32_t* err, void* stream) {
    ALDVC_REQUIRE(values && unknown && iters && err && workspace, "aldvc_inpaint: null pointer");
    ALDVC_REQUIRE(ncols >= 1 && ncols <= MAX_COLS, "aldvc_inpaint: 1..12 columns");
    Grid3 g;
    int rc = make_grid(nz, ny, nx, g);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int32_t), s);
    if (e != cudaSuccess) return cuda_fail(e, "aldvc_inpaint: error word reset");
    return run_inpaint(g, ncols, values, unknown, tol, max_iter, (char*)workspace, workspace_bytes, iters, err, s);
}

extern "C" size_t aldvc_median_test_workspace_size(int64_t nz, int64_t ny, int64_t nx, int32_t ncols) {
    const int64_t n = nx * ny * nz;
    return 2 * align_up((size_t)n * ncols * sizeof(double), 256) + align_up((size_t)n, 256) + 256 +
           aldvc_inpaint_workspace_size(nz, ny, nx, ncols);
}

extern "C" int aldvc_median_test(const double* field, int64_t nz, int64_t ny, int64_t nx, int32_t ncols, const uint8_t* valid,
                                 double threshold, double eps, uint8_t* flag, void* workspace, size_t workspace_bytes, int32_t* err,
                                 void* stream) {
    ALDVC_REQUIRE(field && flag && workspace && err, "aldvc_median_test: null pointer");
    ALDVC_REQUIRE(ncols >= 1 && ncols <= MAX_COLS, "aldvc_median_test: 1..12 columns");
    Grid3 g;
    int rc = make_grid(nz, ny, nx, g);
    if (rc) return rc;
    if (workspace_bytes < aldvc_median_test_workspace_size(nz, ny, nx, ncols)) return arg_fail("aldvc_median_test: workspace");
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t n = g.n;
    char* w = (char*)workspace;
    const size_t v = align_up((size_t)n * ncols * sizeof(double), 256);
    double* copy = (double*)w;
    double* absfl = (double*)(w + v);
    uint8_t* nanmask = (uint8_t*)(w + 2 * v);
    int32_t* iters = (int32_t*)(w + 2 * v + align_up((size_t)n, 256));
    char* iws = w + 2 * v + align_up((size_t)n, 256) + 256;
    const size_t iws_bytes = workspace_bytes - (size_t)(iws - w);
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int32_t), s);
    if (e != cudaSuccess) return cuda_fail(e, "aldvc_median_test: error word reset");
    const unsigned blocks = (unsigned)((n + 255) / 256);
    nanmask_kernel<<<blocks, 256, 0, s>>>(field, ncols, n, valid, nanmask, copy);
    rc = check_launch("median test: mask");
    if (rc) return rc;
    // invalid nodes are inpainted first so they do not poison the medians (outlier_detection.py:112-121)
    rc = run_inpaint(g, ncols, copy, nanmask, 1e-12, 4000, iws, iws_bytes, iters, err, s);
    if (rc) return rc;
    MedArgs a{g, ncols, copy, absfl, nullptr, nanmask, valid, threshold, eps, flag};
    med_fluct_kernel<<<blocks, 256, 0, s>>>(a);
    rc = check_launch("median test: fluctuation");
    if (rc) return rc;
    med_flag_kernel<<<blocks, 256, 0, s>>>(a);
    return check_launch("median test: flag");
}
