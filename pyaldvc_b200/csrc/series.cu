// Node-grid fields sampled at arbitrary points (pyALDVC utils/grid_interp.py:18-51 interp_grid_field), the step of
// the cumulative displacements of a frame series (core/pipeline.py:455-491 _compose_cumulative): each frame's
// displacement grid is interpolated at the positions its parent frame's material points have reached.
//
// Order 1: trilinear interpolation of the grid, taps clamped to the grid (map_coordinates order 1, mode nearest).
// Order 3: cubic B-spline interpolation.  The reference pads the grid by odd reflection, SciPy pads it again by
// edge values and runs the B-spline prefilter; all of that is linear along each axis, so the caller passes one
// operator per axis, op_a ((n_a + pad) x n_a, FP64), and the coefficient grid is op_z (op_y (op_x field)): three
// passes of small dense products.  The points are then evaluated with the cubic B-spline weights, taps clamped
// to the coefficient grid.  Everything is FP64.
#include <algorithm>

#include "common.cuh"
#include "internal.cuh"

namespace aldvc {

constexpr int GI_THREADS = 256;

// out[o][j][i] = sum_k op[j][k] in[o][k][i]: one axis of an array seen as [outer][n_in][inner]
__global__ void grid_axis_op_kernel(const double* __restrict__ in, double* __restrict__ out, const double* __restrict__ op, int n_in,
                                    int n_out, int64_t outer, int64_t inner) {
    const int64_t total = outer * n_out * inner;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % inner, r = e / inner;
        const int j = (int)(r % n_out);
        const int64_t o = r / n_out;
        const double* src = in + o * n_in * inner + i;
        const double* w = op + (int64_t)j * n_in;
        double s = 0.0;
        for (int k = 0; k < n_in; ++k) s += w[k] * src[(int64_t)k * inner];
        out[e] = s;
    }
}

__device__ __forceinline__ void bspline3_w(double t, double w[4]) {
    const double u = 1.0 - t, t2 = t * t, t3 = t2 * t;
    w[0] = u * u * u / 6.0;
    w[1] = (3.0 * t3 - 6.0 * t2 + 4.0) / 6.0;
    w[2] = (-3.0 * t3 + 3.0 * t2 + 3.0 * t + 1.0) / 6.0;
    w[3] = t3 / 6.0;
}

struct GridInterpArgs {
    const double* grid;  // [nz][ny][nx][C]: the field (order 1) or its coefficients (order 3)
    int nz, ny, nx, C;
    double ox, oy, oz, hx, hy, hz;  // first node and spacing per axis
    double sx, sy, sz;              // index offset of node 0 in `grid` per axis (the padding of the order-3 coefficients)
    const double* points;           // (M, 3) [x, y, z]
    int64_t M;
    int order;
    double* out;  // (M, C)
};

__device__ __forceinline__ int gi_clamp(int i, int n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }

__global__ void grid_eval_kernel(GridInterpArgs a) {
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < a.M; m += (int64_t)gridDim.x * blockDim.x) {
        const double fx = (a.points[3 * m] - a.ox) / a.hx + a.sx;
        const double fy = (a.points[3 * m + 1] - a.oy) / a.hy + a.sy;
        const double fz = (a.points[3 * m + 2] - a.oz) / a.hz + a.sz;
        const double flx = floor(fx), fly = floor(fy), flz = floor(fz);
        const double tx = fx - flx, ty = fy - fly, tz = fz - flz;
        const int ix = (int)flx, iy = (int)fly, iz = (int)flz;
        if (a.order == 1) {
            const double wx[2] = {1.0 - tx, tx}, wy[2] = {1.0 - ty, ty}, wz[2] = {1.0 - tz, tz};
            for (int c = 0; c < a.C; ++c) {
                double s = 0.0;
                for (int k = 0; k < 2; ++k)
                    for (int j = 0; j < 2; ++j)
                        for (int i = 0; i < 2; ++i) {
                            const int64_t o = (((int64_t)gi_clamp(iz + k, a.nz) * a.ny + gi_clamp(iy + j, a.ny)) * a.nx +
                                               gi_clamp(ix + i, a.nx)) * a.C + c;
                            s += wz[k] * wy[j] * wx[i] * a.grid[o];
                        }
                a.out[m * a.C + c] = s;
            }
        } else {
            double wx[4], wy[4], wz[4];
            bspline3_w(tx, wx);
            bspline3_w(ty, wy);
            bspline3_w(tz, wz);
            for (int c = 0; c < a.C; ++c) {
                double s = 0.0;
                for (int k = 0; k < 4; ++k) {
                    double sy = 0.0;
                    for (int j = 0; j < 4; ++j) {
                        double sx = 0.0;
                        for (int i = 0; i < 4; ++i) {
                            const int64_t o = (((int64_t)gi_clamp(iz - 1 + k, a.nz) * a.ny + gi_clamp(iy - 1 + j, a.ny)) * a.nx +
                                               gi_clamp(ix - 1 + i, a.nx)) * a.C + c;
                            sx += wx[i] * a.grid[o];
                        }
                        sy += wy[j] * sx;
                    }
                    s += wz[k] * sy;
                }
                a.out[m * a.C + c] = s;
            }
        }
    }
}

// ----------------------------------------------------------------------------- displacement uncertainty
// solver/uncertainty.py:83-137: at a converged node with n_valid > 14 voxels, s^2 = (1 - ZNCC) bf^2 / n, the
// parameter factor 2 (1 - ZNCC) bf^2 / (n - 12), the stored Hessian less the reference-gradient noise it carries
// (gain s^2 (n / pattern[9][9]) pattern, at most (1 - min_frac) of each translation diagonal), its inverse, and
// var = factor diag(inv)[9..11] + gain s^4 diag(inv pattern' inv)[9..11] (pattern' = pattern n / pattern[9][9]).
// One thread per node, the 12 x 12 system in FP64, Gauss-Jordan elimination with partial pivoting; a zero pivot
// leaves the node NaN.
struct UncArgs {
    const double* H;        // (N, 12, 12)
    const double* zncc;     // (N,)
    const int8_t* status;   // (N,) or NULL
    const uint8_t* valid;   // (N,)
    const int64_t* n_valid; // (N,)
    const double* bottomf;  // (N,)
    int64_t N;
    double pattern[144];
    double gain, min_frac;
    int noise_correction;
    double* out;  // (N, 3)
};

__global__ void uncertainty_kernel(UncArgs a) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < a.N; n += (int64_t)gridDim.x * blockDim.x) {
        const double nanv = __longlong_as_double(0x7ff8000000000000LL);
        a.out[3 * n] = a.out[3 * n + 1] = a.out[3 * n + 2] = nanv;
        const double z = a.zncc[n];
        const int64_t nv = a.n_valid[n];
        if (!a.valid[n] || !isfinite(z) || nv <= 14 || (a.status && a.status[n] != 0)) continue;
        const double bf = a.bottomf[n], omz = fmax(1.0 - z, 0.0);
        const double factor = 2.0 * omz / (double)(nv - 12) * (bf * bf);
        const double s2 = omz * (bf * bf) / (double)nv;
        const double scale = (double)nv / a.pattern[9 * 12 + 9];
        double A[144], inv[144];
        for (int i = 0; i < 144; ++i) A[i] = a.H[n * 144 + i];
        if (a.noise_correction) {
            const double g = a.gain * s2 * scale;
            double limit = 1e300;
            for (int i = 9; i < 12; ++i) {
                const double cd = g * a.pattern[i * 12 + i], td = A[i * 12 + i];
                limit = fmin(limit, cd > 0.0 ? (1.0 - a.min_frac) * td / fmax(cd, 1e-300) : 1.0);
            }
            limit = fmin(fmax(limit, 0.0), 1.0);
            for (int i = 0; i < 144; ++i) A[i] -= g * a.pattern[i] * limit;
        }
        for (int i = 0; i < 144; ++i) inv[i] = (i / 12 == i % 12) ? 1.0 : 0.0;
        bool singular = false;
        for (int c = 0; c < 12 && !singular; ++c) {
            int piv = c;
            for (int r = c + 1; r < 12; ++r)
                if (fabs(A[r * 12 + c]) > fabs(A[piv * 12 + c])) piv = r;
            if (A[piv * 12 + c] == 0.0) {
                singular = true;
                break;
            }
            if (piv != c)
                for (int k = 0; k < 12; ++k) {
                    double t = A[c * 12 + k];
                    A[c * 12 + k] = A[piv * 12 + k];
                    A[piv * 12 + k] = t;
                    t = inv[c * 12 + k];
                    inv[c * 12 + k] = inv[piv * 12 + k];
                    inv[piv * 12 + k] = t;
                }
            const double d = 1.0 / A[c * 12 + c];
            for (int k = 0; k < 12; ++k) {
                A[c * 12 + k] *= d;
                inv[c * 12 + k] *= d;
            }
            for (int r = 0; r < 12; ++r) {
                if (r == c) continue;
                const double m = A[r * 12 + c];
                if (m == 0.0) continue;
                for (int k = 0; k < 12; ++k) {
                    A[r * 12 + k] -= m * A[c * 12 + k];
                    inv[r * 12 + k] -= m * inv[c * 12 + k];
                }
            }
        }
        if (singular) continue;
        for (int i = 0; i < 3; ++i) {
            const int d = 9 + i;
            double var = factor * inv[d * 12 + d];
            if (a.noise_correction) {
                double cross = 0.0;
                for (int p = 0; p < 12; ++p) {
                    double t = 0.0;
                    for (int q = 0; q < 12; ++q) t += a.pattern[p * 12 + q] * scale * inv[q * 12 + d];
                    cross += inv[d * 12 + p] * t;
                }
                var += a.gain * s2 * s2 * cross;
            }
            a.out[3 * n + i] = sqrt(fmax(var, 0.0));
        }
    }
}

static unsigned gi_blocks(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + GI_THREADS - 1) / GI_THREADS, 148 * 16)); }

}  // namespace aldvc

using namespace aldvc;

extern "C" size_t aldvc_grid_interp_workspace_size(int64_t nz, int64_t ny, int64_t nx, int32_t C, int32_t pad_x, int32_t pad_y,
                                                   int32_t pad_z) {
    const int64_t Nz = nz + pad_z, Ny = ny + pad_y, Nx = nx + pad_x;
    return (size_t)2 * (size_t)(Nz * Ny * Nx * C) * sizeof(double) + 256;
}

extern "C" int aldvc_grid_interp(const double* field, int64_t nz, int64_t ny, int64_t nx, int32_t C, const double* op_x, const double* op_y,
                                 const double* op_z, int32_t pad_x, int32_t pad_y, int32_t pad_z, double ox, double oy, double oz,
                                 double hx, double hy, double hz,
                                 const double* points, int64_t M, int32_t order, double* out, void* workspace, size_t workspace_bytes,
                                 void* stream) {
    ALDVC_REQUIRE(field && points && out, "aldvc_grid_interp: null pointer");
    ALDVC_REQUIRE(order == 1 || order == 3, "aldvc_grid_interp: order must be 1 or 3");
    ALDVC_REQUIRE(nz > 0 && ny > 0 && nx > 0 && C > 0 && nz * ny * nx < (1LL << 31), "aldvc_grid_interp: grid shape");
    ALDVC_REQUIRE(hx != 0.0 && hy != 0.0 && hz != 0.0, "aldvc_grid_interp: zero spacing");
    if (M <= 0) return ALDVC_OK;
    cudaStream_t s = (cudaStream_t)stream;
    GridInterpArgs a{};
    a.C = C;
    a.ox = ox;
    a.oy = oy;
    a.oz = oz;
    a.hx = hx;
    a.hy = hy;
    a.hz = hz;
    a.points = points;
    a.M = M;
    a.order = order;
    a.out = out;
    KTimer kt_("grid_interp", s);
    if (order == 1) {
        a.grid = field;
        a.nz = (int)nz;
        a.ny = (int)ny;
        a.nx = (int)nx;
        a.sx = a.sy = a.sz = 0.0;
    } else {
        ALDVC_REQUIRE(op_x && op_y && op_z, "aldvc_grid_interp: order 3 needs the three axis operators");
        ALDVC_REQUIRE(pad_x >= 0 && pad_y >= 0 && pad_z >= 0 && pad_x % 2 == 0 && pad_y % 2 == 0 && pad_z % 2 == 0,
                      "aldvc_grid_interp: paddings must be even and non-negative");
        ALDVC_REQUIRE(workspace && workspace_bytes >= aldvc_grid_interp_workspace_size(nz, ny, nx, C, pad_x, pad_y, pad_z),
                      "aldvc_grid_interp: workspace");
        const int64_t Nz = nz + pad_z, Ny = ny + pad_y, Nx = nx + pad_x;
        double* t1 = (double*)workspace;             // [nz][ny][Nx][C], then [Nz][Ny][Nx][C]
        double* t2 = t1 + Nz * Ny * Nx * C;         // [nz][Ny][Nx][C]
        grid_axis_op_kernel<<<gi_blocks(nz * ny * Nx * C), GI_THREADS, 0, s>>>(field, t1, op_x, (int)nx, (int)Nx, nz * ny, (int64_t)C);
        grid_axis_op_kernel<<<gi_blocks(nz * Ny * Nx * C), GI_THREADS, 0, s>>>(t1, t2, op_y, (int)ny, (int)Ny, nz, Nx * C);
        grid_axis_op_kernel<<<gi_blocks(Nz * Ny * Nx * C), GI_THREADS, 0, s>>>(t2, t1, op_z, (int)nz, (int)Nz, 1, Ny * Nx * C);
        a.grid = t1;
        a.nz = (int)Nz;
        a.ny = (int)Ny;
        a.nx = (int)Nx;
        a.sx = (double)(pad_x / 2);
        a.sy = (double)(pad_y / 2);
        a.sz = (double)(pad_z / 2);
    }
    grid_eval_kernel<<<gi_blocks(M), GI_THREADS, 0, s>>>(a);
    return check_launch("aldvc_grid_interp");
}

extern "C" int aldvc_displacement_uncertainty(const double* H, const double* zncc, const int8_t* status, const uint8_t* valid,
                                             const int64_t* n_valid, const double* bottomf, int64_t n_nodes, const double* pattern,
                                             double gain, double min_frac, int32_t noise_correction, double* out, void* stream) {
    ALDVC_REQUIRE(H && zncc && valid && n_valid && bottomf && pattern && out, "aldvc_displacement_uncertainty: null pointer");
    ALDVC_REQUIRE(pattern[9 * 12 + 9] > 0.0, "aldvc_displacement_uncertainty: pattern[9][9] must be the subset's voxel count");
    if (n_nodes <= 0) return ALDVC_OK;
    UncArgs a{};
    a.H = H;
    a.zncc = zncc;
    a.status = status;
    a.valid = valid;
    a.n_valid = n_valid;
    a.bottomf = bottomf;
    a.N = n_nodes;
    for (int i = 0; i < 144; ++i) a.pattern[i] = pattern[i];
    a.gain = gain;
    a.min_frac = min_frac;
    a.noise_correction = noise_correction ? 1 : 0;
    a.out = out;
    cudaStream_t s = (cudaStream_t)stream;
    KTimer kt_("uncertainty", s);
    uncertainty_kernel<<<gi_blocks(n_nodes), 128, 0, s>>>(a);
    return check_launch("aldvc_displacement_uncertainty");
}
