// Strain after the path (pyALDVC strain/), on the node grid, FP64 throughout:
//   aldvc_gradient_plane_fit <- strain/gradient_methods.py:151-228 gradient_plane_fit (no cut mesh)
//   aldvc_gradient_fd        <- strain/gradient_methods.py:231-283 gradient_fd (no cut mesh)
//   aldvc_grid_smooth        <- utils/grid_interp.py:54-79 smooth_grid_field (normalised Gaussian, edge repeat)
//   aldvc_strain_measures    <- strain/strain_types.py:19-114 (strain tensors, principal strains, von Mises,
//                               maximum shear, volumetric strain, det F, polar rotation angle)
// One thread per node; a node's window and its 3 x 3 algebra stay in registers.
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "internal.cuh"

namespace aldvc {

constexpr int ST_THREADS = 128;
constexpr int GS_MAX_HALF = 63;

struct NodeGrid {
    int nx, ny, nz;
    int64_t n;
    double hx, hy, hz;
};

__device__ __forceinline__ bool node_ok(const double* U, const uint8_t* valid, int64_t n) {
    return (valid == nullptr || valid[n] != 0) && isfinite(U[3 * n]) && isfinite(U[3 * n + 1]) && isfinite(U[3 * n + 2]);
}

// Gaussian elimination with partial pivoting on the 4 x 4 normal equations, three right-hand sides.
__device__ void solve4(double A[4][4], double B[4][3]) {
    for (int c = 0; c < 4; ++c) {
        int p = c;
        for (int r = c + 1; r < 4; ++r)
            if (fabs(A[r][c]) > fabs(A[p][c])) p = r;
        if (p != c) {
            for (int k = 0; k < 4; ++k) {
                const double t = A[c][k];
                A[c][k] = A[p][k];
                A[p][k] = t;
            }
            for (int k = 0; k < 3; ++k) {
                const double t = B[c][k];
                B[c][k] = B[p][k];
                B[p][k] = t;
            }
        }
        for (int r = c + 1; r < 4; ++r) {
            const double m = A[r][c] / A[c][c];
            for (int k = c; k < 4; ++k) A[r][k] -= m * A[c][k];
            for (int k = 0; k < 3; ++k) B[r][k] -= m * B[c][k];
        }
    }
    for (int c = 3; c >= 0; --c)
        for (int k = 0; k < 3; ++k) {
            double s = B[c][k];
            for (int j = c + 1; j < 4; ++j) s -= A[c][j] * B[j][k];
            B[c][k] = s / A[c][c];
        }
}

// Least-squares plane u_c = a + b X + c Y + d Z over the valid nodes of the (2r+1)^3 window (offsets in spacing
// units), F[c][j] = the slope along j; NaN for an invalid node or a window of fewer than 5 valid nodes; complete =
// every window node valid (windows past the grid edge count those nodes as missing).
__global__ void __launch_bounds__(ST_THREADS) plane_fit_kernel(const double* __restrict__ U, const uint8_t* __restrict__ valid, NodeGrid g,
                                                               int rx, int ry, int rz, double* __restrict__ F, uint8_t* __restrict__ complete) {
    const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (n >= g.n) return;
    const int ix = (int)(n % g.nx), iy = (int)((n / g.nx) % g.ny), iz = (int)(n / ((int64_t)g.nx * g.ny));
    double* Fo = F + 9 * n;
    complete[n] = 0;
    if (!node_ok(U, valid, n)) {
        for (int k = 0; k < 9; ++k) Fo[k] = nan("");
        return;
    }
    double A[4][4] = {}, B[4][3] = {};
    for (int dz = -rz; dz <= rz; ++dz) {
        const int jz = iz + dz;
        if (jz < 0 || jz >= g.nz) continue;
        for (int dy = -ry; dy <= ry; ++dy) {
            const int jy = iy + dy;
            if (jy < 0 || jy >= g.ny) continue;
            for (int dx = -rx; dx <= rx; ++dx) {
                const int jx = ix + dx;
                if (jx < 0 || jx >= g.nx) continue;
                const int64_t m = ((int64_t)jz * g.ny + jy) * g.nx + jx;
                if (!node_ok(U, valid, m)) continue;
                const double X = dx * g.hx, Y = dy * g.hy, Z = dz * g.hz;
                A[0][0] += 1.0;
                A[0][1] += X;
                A[0][2] += Y;
                A[0][3] += Z;
                A[1][1] += X * X;
                A[2][2] += Y * Y;
                A[3][3] += Z * Z;
                A[1][2] += X * Y;
                A[1][3] += X * Z;
                A[2][3] += Y * Z;
                for (int c = 0; c < 3; ++c) {
                    const double u = U[3 * m + c];
                    B[0][c] += u;
                    B[1][c] += u * X;
                    B[2][c] += u * Y;
                    B[3][c] += u * Z;
                }
            }
        }
    }
    const double count = A[0][0];
    const double n_win = (double)(2 * rx + 1) * (2 * ry + 1) * (2 * rz + 1);
    complete[n] = fabs(count - n_win) < 0.5 ? 1 : 0;
    if (count < 4.5) {  // at least 5 points pin a plane
        for (int k = 0; k < 9; ++k) Fo[k] = nan("");
        return;
    }
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < i; ++j) A[i][j] = A[j][i];
    const double reg = 1e-12 * fmax(fabs(A[0][0]), 1.0);  // degenerate (coplanar) windows
    for (int i = 0; i < 4; ++i) A[i][i] += reg;
    solve4(A, B);
    for (int c = 0; c < 3; ++c)
        for (int j = 0; j < 3; ++j) Fo[3 * c + j] = B[1 + j][c];
}

// Central differences, one-sided next to an invalid or missing neighbour, NaN with neither; complete = central
// along every axis.
__global__ void __launch_bounds__(ST_THREADS) fd_kernel(const double* __restrict__ U, const uint8_t* __restrict__ valid, NodeGrid g,
                                                        double* __restrict__ F, uint8_t* __restrict__ complete) {
    const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (n >= g.n) return;
    const int ix = (int)(n % g.nx), iy = (int)((n / g.nx) % g.ny), iz = (int)(n / ((int64_t)g.nx * g.ny));
    double* Fo = F + 9 * n;
    const bool ok = node_ok(U, valid, n);
    bool comp = ok;
    const int pos[3] = {ix, iy, iz}, ext[3] = {g.nx, g.ny, g.nz};
    const int64_t stride[3] = {1, g.nx, (int64_t)g.nx * g.ny};
    const double h[3] = {g.hx, g.hy, g.hz};
    for (int j = 0; j < 3; ++j) {
        const bool vp = ok && pos[j] > 0 && node_ok(U, valid, n - stride[j]);
        const bool vn = ok && pos[j] + 1 < ext[j] && node_ok(U, valid, n + stride[j]);
        comp = comp && vp && vn;
        for (int c = 0; c < 3; ++c) {
            double d = nan("");
            if (vp && vn)
                d = (U[3 * (n + stride[j]) + c] - U[3 * (n - stride[j]) + c]) / (2.0 * h[j]);
            else if (vn)
                d = (U[3 * (n + stride[j]) + c] - U[3 * n + c]) / h[j];
            else if (vp)
                d = (U[3 * n + c] - U[3 * (n - stride[j]) + c]) / h[j];
            Fo[3 * c + j] = d;
        }
    }
    complete[n] = comp ? 1 : 0;
}

// ----------------------------------------------------------------------------- grid smoothing (FP64)
struct GsTaps {
    double w[GS_MAX_HALF + 1];
};

// a = field where weight else 0, w = weight (finite and valid) as 0/1
__global__ void gs_prepare_kernel(const double* __restrict__ field, const uint8_t* __restrict__ valid, int64_t n, double* a, double* w) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const bool k = isfinite(field[i]) && (valid == nullptr || valid[i] != 0);
        a[i] = k ? field[i] : 0.0;
        w[i] = k ? 1.0 : 0.0;
    }
}

// one axis of the symmetric Gaussian with edge repeat, out = w0 s + sum_j wj (s[-j] + s[+j]) in that order
__global__ void gs_axis_kernel(const double* __restrict__ in, double* __restrict__ out, NodeGrid g, int axis, GsTaps t, int J) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < g.n; i += (int64_t)gridDim.x * blockDim.x) {
        const int ix = (int)(i % g.nx), iy = (int)((i / g.nx) % g.ny), iz = (int)(i / ((int64_t)g.nx * g.ny));
        const int p = axis == 0 ? ix : (axis == 1 ? iy : iz), e = axis == 0 ? g.nx : (axis == 1 ? g.ny : g.nz);
        const int64_t s = axis == 0 ? 1 : (axis == 1 ? (int64_t)g.nx : (int64_t)g.nx * g.ny);
        const double* line = in + (i - (int64_t)p * s);
        double acc = __dmul_rn(t.w[0], line[(int64_t)p * s]);
        for (int j = 1; j <= J; ++j) {
            const int a = max(p - j, 0), b = min(p + j, e - 1);
            acc = __dadd_rn(acc, __dmul_rn(t.w[j], __dadd_rn(line[(int64_t)a * s], line[(int64_t)b * s])));
        }
        out[i] = acc;
    }
}

__global__ void gs_finish_kernel(const double* __restrict__ field, const uint8_t* __restrict__ valid, const double* num,
                                 const double* den, int64_t n, double* out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const bool k = isfinite(field[i]) && (valid == nullptr || valid[i] != 0);
        out[i] = (k && den[i] > 1e-12) ? num[i] / den[i] : nan("");
    }
}

// ----------------------------------------------------------------------------- strain measures
// Cyclic Jacobi eigen-decomposition of a symmetric 3 x 3 matrix: eigenvalues d (descending) and eigenvectors as
// the columns of V.
__device__ void eig_sym3(const double A_in[3][3], double d[3], double V[3][3]) {
    double A[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            A[i][j] = A_in[i][j];
            V[i][j] = i == j ? 1.0 : 0.0;
        }
    for (int sweep = 0; sweep < 64; ++sweep) {
        const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
        const double diag = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
        if (off <= 1e-36 * diag || off == 0.0) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                if (A[p][q] == 0.0) continue;
                const double theta = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
                const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) {  // A <- J^T A J, V <- V J
                    const double akp = A[k][p], akq = A[k][q];
                    A[k][p] = c * akp - s * akq;
                    A[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {
                    const double apk = A[p][k], aqk = A[q][k];
                    A[p][k] = c * apk - s * aqk;
                    A[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; ++k) {
                    const double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - s * vkq;
                    V[k][q] = s * vkp + c * vkq;
                }
            }
    }
    for (int i = 0; i < 3; ++i) d[i] = A[i][i];
    for (int i = 0; i < 2; ++i)  // sort descending, columns with them
        for (int j = i + 1; j < 3; ++j)
            if (d[j] > d[i]) {
                const double t = d[i];
                d[i] = d[j];
                d[j] = t;
                for (int k = 0; k < 3; ++k) {
                    const double v = V[k][i];
                    V[k][i] = V[k][j];
                    V[k][j] = v;
                }
            }
}

__device__ __forceinline__ double det3(const double M[3][3]) {
    return M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
           M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
}

struct StrainOut {
    double* E;          // (N, 9)
    double* principal;  // (N, 3) descending
    double* max_shear;
    double* von_mises;
    double* volumetric;
    double* det_F;
    double* rotation_deg;
};

// type 0 infinitesimal 0.5 (H + H^T); 1 Green-Lagrange 0.5 (F^T F - I); 2 Euler-Almansi 0.5 (I - (F F^T)^-1);
// 3 Hencky 0.5 log(F F^T), F = I + H
__global__ void __launch_bounds__(ST_THREADS) strain_measures_kernel(const double* __restrict__ Hg, int64_t N, int type, StrainOut o) {
    const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (n >= N) return;
    double H[3][3], Fm[3][3], E[3][3];
    bool finite = true;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            H[i][j] = Hg[9 * n + 3 * i + j];
            Fm[i][j] = H[i][j] + (i == j ? 1.0 : 0.0);
            finite = finite && isfinite(H[i][j]);
        }
    const double qnan = nan("");
    if (type == 0) {  // elementwise: a NaN reaches only the entries it touches
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) E[i][j] = 0.5 * (H[i][j] + H[j][i]);
    } else if (!finite) {
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) E[i][j] = qnan;
    } else if (type == 1) {
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double c = 0.0;
                for (int k = 0; k < 3; ++k) c += Fm[k][i] * Fm[k][j];
                E[i][j] = 0.5 * (c - (i == j ? 1.0 : 0.0));
            }
    } else {
        double B[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double c = 0.0;
                for (int k = 0; k < 3; ++k) c += Fm[i][k] * Fm[j][k];
                B[i][j] = c;
            }
        if (type == 2) {
            double Bi[3][3];
            const double dt = inv3(B, Bi);
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) E[i][j] = dt != 0.0 ? 0.5 * ((i == j ? 1.0 : 0.0) - Bi[i][j]) : qnan;
        } else {
            double d[3], V[3][3];
            eig_sym3(B, d, V);
            double lg[3];
            for (int k = 0; k < 3; ++k) lg[k] = 0.5 * log(fmax(d[k], 1e-30));
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    double s = 0.0;
                    for (int k = 0; k < 3; ++k) s += V[i][k] * lg[k] * V[j][k];
                    E[i][j] = s;
                }
        }
    }
    bool efin = true;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            o.E[9 * n + 3 * i + j] = E[i][j];
            efin = efin && isfinite(E[i][j]);
        }
    // principal strains of the symmetric part, descending
    double p[3] = {qnan, qnan, qnan};
    if (efin) {
        double S[3][3], V[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) S[i][j] = 0.5 * (E[i][j] + E[j][i]);
        eig_sym3(S, p, V);
    }
    for (int k = 0; k < 3; ++k) o.principal[3 * n + k] = p[k];
    o.max_shear[n] = 0.5 * (p[0] - p[2]);
    const double tr = E[0][0] + E[1][1] + E[2][2];
    double dd = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const double v = E[i][j] - (i == j ? tr / 3.0 : 0.0);
            dd += v * v;
        }
    o.von_mises[n] = sqrt(2.0 / 3.0 * dd);
    o.volumetric[n] = tr;
    o.det_F[n] = finite ? det3(Fm) : qnan;
    // polar rotation R of F = R U: F^T F = V S^2 V^T (V proper), u1 = F v1 / s1, u2 = F v2 / s2 made orthogonal to u1,
    // u3 = u1 x u2, R = [u1 u2 u3] V^T (the rotation also for det F < 0, as the reference's sign flip gives)
    double ang = qnan;
    if (finite) {
        double C[3][3], d[3], V[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double c = 0.0;
                for (int k = 0; k < 3; ++k) c += Fm[k][i] * Fm[k][j];
                C[i][j] = c;
            }
        eig_sym3(C, d, V);
        if (det3(V) < 0.0)
            for (int k = 0; k < 3; ++k) V[k][2] = -V[k][2];
        double u[3][3];  // u[i] = the i-th left singular vector
        for (int i = 0; i < 2; ++i) {
            const double s = sqrt(fmax(d[i], 0.0));
            for (int r = 0; r < 3; ++r) {
                double a = 0.0;
                for (int k = 0; k < 3; ++k) a += Fm[r][k] * V[k][i];
                u[i][r] = s > 0.0 ? a / s : 0.0;
            }
        }
        double dp = u[0][0] * u[1][0] + u[0][1] * u[1][1] + u[0][2] * u[1][2];
        for (int r = 0; r < 3; ++r) u[1][r] -= dp * u[0][r];
        double nn = sqrt(u[1][0] * u[1][0] + u[1][1] * u[1][1] + u[1][2] * u[1][2]);
        for (int r = 0; r < 3; ++r) u[1][r] = nn > 0.0 ? u[1][r] / nn : 0.0;
        u[2][0] = u[0][1] * u[1][2] - u[0][2] * u[1][1];
        u[2][1] = u[0][2] * u[1][0] - u[0][0] * u[1][2];
        u[2][2] = u[0][0] * u[1][1] - u[0][1] * u[1][0];
        double R[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double s = 0.0;
                for (int k = 0; k < 3; ++k) s += u[k][i] * V[j][k];
                R[i][j] = s;
            }
        const double cos_t = (R[0][0] + R[1][1] + R[2][2] - 1.0) / 2.0;
        const double ax = 0.5 * (R[2][1] - R[1][2]), ay = 0.5 * (R[0][2] - R[2][0]), az = 0.5 * (R[1][0] - R[0][1]);
        ang = atan2(sqrt(ax * ax + ay * ay + az * az), cos_t) * (180.0 / 3.14159265358979323846);
    }
    o.rotation_deg[n] = ang;
}

}  // namespace aldvc

using namespace aldvc;

static int grid_ok(int64_t nz, int64_t ny, int64_t nx) { return nz > 0 && ny > 0 && nx > 0 && nz < (1 << 30) && ny < (1 << 30) && nx < (1 << 30); }

extern "C" int aldvc_gradient_plane_fit(const double* U, const uint8_t* valid, int64_t nz, int64_t ny, int64_t nx, double hx, double hy,
                                        double hz, int32_t rx, int32_t ry, int32_t rz, double* F, uint8_t* complete, void* stream) {
    ALDVC_REQUIRE(U && F && complete, "aldvc_gradient_plane_fit: null pointer");
    ALDVC_REQUIRE(grid_ok(nz, ny, nx), "aldvc_gradient_plane_fit: grid shape");
    ALDVC_REQUIRE(rx >= 0 && ry >= 0 && rz >= 0 && rx <= 16 && ry <= 16 && rz <= 16, "aldvc_gradient_plane_fit: half-widths in [0, 16]");
    const NodeGrid g{(int)nx, (int)ny, (int)nz, nz * ny * nx, hx, hy, hz};
    plane_fit_kernel<<<(unsigned)((g.n + ST_THREADS - 1) / ST_THREADS), ST_THREADS, 0, (cudaStream_t)stream>>>(U, valid, g, rx, ry, rz, F,
                                                                                                             complete);
    return check_launch("aldvc_gradient_plane_fit");
}

extern "C" int aldvc_gradient_fd(const double* U, const uint8_t* valid, int64_t nz, int64_t ny, int64_t nx, double hx, double hy, double hz,
                                 double* F, uint8_t* complete, void* stream) {
    ALDVC_REQUIRE(U && F && complete, "aldvc_gradient_fd: null pointer");
    ALDVC_REQUIRE(grid_ok(nz, ny, nx), "aldvc_gradient_fd: grid shape");
    const NodeGrid g{(int)nx, (int)ny, (int)nz, nz * ny * nx, hx, hy, hz};
    fd_kernel<<<(unsigned)((g.n + ST_THREADS - 1) / ST_THREADS), ST_THREADS, 0, (cudaStream_t)stream>>>(U, valid, g, F, complete);
    return check_launch("aldvc_gradient_fd");
}

extern "C" size_t aldvc_grid_smooth_workspace_size(int64_t nz, int64_t ny, int64_t nx) { return (size_t)4 * nz * ny * nx * sizeof(double); }

extern "C" int aldvc_grid_smooth(const double* field, const uint8_t* valid, int64_t nz, int64_t ny, int64_t nx, const double* weights,
                                 int32_t half_taps, double* out, void* workspace, size_t workspace_bytes, void* stream) {
    ALDVC_REQUIRE(field && out && weights && workspace, "aldvc_grid_smooth: null pointer");
    ALDVC_REQUIRE(grid_ok(nz, ny, nx), "aldvc_grid_smooth: grid shape");
    ALDVC_REQUIRE(half_taps >= 0 && half_taps <= GS_MAX_HALF, "aldvc_grid_smooth: half_taps must be in [0, 63]");
    ALDVC_REQUIRE(workspace_bytes >= aldvc_grid_smooth_workspace_size(nz, ny, nx), "aldvc_grid_smooth: workspace");
    const NodeGrid g{(int)nx, (int)ny, (int)nz, nz * ny * nx, 1.0, 1.0, 1.0};
    GsTaps t{};
    for (int j = 0; j <= half_taps; ++j) t.w[j] = weights[j];
    double* a = (double*)workspace;
    double* w = a + g.n;
    double* ta = w + g.n;
    double* tw = ta + g.n;
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned blocks = (unsigned)std::min<int64_t>((g.n + 255) / 256, 148 * 8);
    gs_prepare_kernel<<<blocks, 256, 0, s>>>(field, valid, g.n, a, w);
    // axes z, y, x in turn (the order of scipy.ndimage.gaussian_filter over array axes 0, 1, 2)
    gs_axis_kernel<<<blocks, 256, 0, s>>>(a, ta, g, 2, t, half_taps);
    gs_axis_kernel<<<blocks, 256, 0, s>>>(w, tw, g, 2, t, half_taps);
    gs_axis_kernel<<<blocks, 256, 0, s>>>(ta, a, g, 1, t, half_taps);
    gs_axis_kernel<<<blocks, 256, 0, s>>>(tw, w, g, 1, t, half_taps);
    gs_axis_kernel<<<blocks, 256, 0, s>>>(a, ta, g, 0, t, half_taps);
    gs_axis_kernel<<<blocks, 256, 0, s>>>(w, tw, g, 0, t, half_taps);
    gs_finish_kernel<<<blocks, 256, 0, s>>>(field, valid, ta, tw, g.n, out);
    return check_launch("aldvc_grid_smooth");
}

extern "C" int aldvc_strain_measures(const double* H, int64_t n_nodes, int32_t strain_type, double* E, double* principal, double* max_shear,
                                     double* von_mises, double* volumetric, double* det_F, double* rotation_deg, void* stream) {
    ALDVC_REQUIRE(H && E && principal && max_shear && von_mises && volumetric && det_F && rotation_deg, "aldvc_strain_measures: null pointer");
    ALDVC_REQUIRE(strain_type >= 0 && strain_type <= 3, "aldvc_strain_measures: strain_type must be 0..3");
    if (n_nodes <= 0) return ALDVC_OK;
    const StrainOut o{E, principal, max_shear, von_mises, volumetric, det_F, rotation_deg};
    strain_measures_kernel<<<(unsigned)((n_nodes + ST_THREADS - 1) / ST_THREADS), ST_THREADS, 0, (cudaStream_t)stream>>>(H, n_nodes,
                                                                                                                       strain_type, o);
    return check_launch("aldvc_strain_measures");
}
