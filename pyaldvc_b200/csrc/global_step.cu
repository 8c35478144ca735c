// ADMM subproblem 2 on the hex8 node grid (pyALDVC solver/subpb2_solver.py, solver/global_operators.py).
//
// Matrix-free: every element of a uniform grid is the same box, so the element matrices K, M, G_j
// (mesh/hex8.py:74-105, Gauss order 1-3) are computed once per block in shared memory (FP64) and applied
// per node by summing over its <= 8 kept elements.  No host round trip: every entry point is
// stream-ordered and can be captured in a CUDA graph.  A node is active when one of its elements is kept.
//
// The PCG (subpb2_solver.pcg_multi :77-108) runs as ONE cooperative persistent kernel: three grid
// barriers per iteration, FP64 everywhere, dot products reduced per block and then over the block
// partials in a fixed order (deterministic).  Every barrier wait is bounded: on give-up the kernel sets
// the error word and returns.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "common.cuh"
#include "internal.cuh"

namespace aldvc {

constexpr int PCG_THREADS = 256;

struct ElemMats {
    double K[64], M[64], G[3][64];
};

struct Spacing {
    double sx, sy, sz;
    int order;
};

// mesh/hex8.hex8_box_matrices (:74-105) computed by the first 64 threads of a block into shared memory:
// thread t owns entry (a, b) = (t / 8, t % 8) of K, M and G_j, summed over the Gauss points in order.
__device__ void block_elem_mats(const Spacing& sp, ElemMats& E) {
    const int t = threadIdx.x;
    if (t < 64) {
        const int a = t / 8, b = t % 8;
        const double S[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}, {-1, -1, 1}, {1, -1, 1}, {1, 1, 1}, {-1, 1, 1}};
        double p[3], w[3];
        int n;
        if (sp.order == 1) {
            n = 1;
            p[0] = 0.0;
            w[0] = 2.0;
        } else if (sp.order == 3) {
            n = 3;
            const double g = sqrt(3.0 / 5.0);
            p[0] = -g;
            p[1] = 0.0;
            p[2] = g;
            w[0] = 5.0 / 9.0;
            w[1] = 8.0 / 9.0;
            w[2] = 5.0 / 9.0;
        } else {
            n = 2;
            const double g = 1.0 / sqrt(3.0);
            p[0] = -g;
            p[1] = g;
            w[0] = 1.0;
            w[1] = 1.0;
        }
        const double inv[3] = {2.0 / sp.sx, 2.0 / sp.sy, 2.0 / sp.sz};
        const double det_j = (sp.sx / 2.0) * (sp.sy / 2.0) * (sp.sz / 2.0);
        double k = 0.0, m = 0.0, g3[3] = {0.0, 0.0, 0.0};
        for (int kk = 0; kk < n; ++kk)
            for (int jj = 0; jj < n; ++jj)
                for (int ii = 0; ii < n; ++ii) {
                    const double ksi = p[ii], eta = p[jj], zeta = p[kk];
                    const double wj = w[ii] * w[jj] * w[kk] * det_j;
                    double N[2], dN[2][3];
                    const int ab[2] = {a, b};
                    for (int q = 0; q < 2; ++q) {
                        const int c = ab[q];
                        N[q] = 0.125 * (1 + S[c][0] * ksi) * (1 + S[c][1] * eta) * (1 + S[c][2] * zeta);
                        dN[q][0] = 0.125 * S[c][0] * (1 + S[c][1] * eta) * (1 + S[c][2] * zeta) * inv[0];
                        dN[q][1] = 0.125 * (1 + S[c][0] * ksi) * S[c][1] * (1 + S[c][2] * zeta) * inv[1];
                        dN[q][2] = 0.125 * (1 + S[c][0] * ksi) * (1 + S[c][1] * eta) * S[c][2] * inv[2];
                    }
                    k += wj * (dN[0][0] * dN[1][0] + dN[0][1] * dN[1][1] + dN[0][2] * dN[1][2]);
                    m += wj * (N[0] * N[1]);
                    for (int d = 0; d < 3; ++d) g3[d] += wj * (dN[0][d] * N[1]);
                }
        E.K[t] = k;
        E.M[t] = m;
        for (int d = 0; d < 3; ++d) E.G[d][t] = g3[d];
    }
    __syncthreads();
}

// local corner index of offset (dx, dy, dz) in {0,1}^3 (mesh/hex8.py:1-13 node order)
__device__ __forceinline__ int corner(int dx, int dy, int dz) {
    const int t[2][2] = {{0, 3}, {1, 2}};  // [dx][dy] within a z layer
    return t[dx][dy] + 4 * dz;
}

struct Mesh {
    int nx, ny, nz;
    int64_t n;
    const uint8_t* elem_active;
};

__device__ __forceinline__ bool elem_on(const Mesh& m, int ex, int ey, int ez) {
    if (ex < 0 || ey < 0 || ez < 0 || ex >= m.nx - 1 || ey >= m.ny - 1 || ez >= m.nz - 1) return false;
    if (!m.elem_active) return true;
    return m.elem_active[((int64_t)ez * (m.ny - 1) + ey) * (m.nx - 1) + ex] != 0;
}

__device__ __forceinline__ int64_t nid(const Mesh& m, int ix, int iy, int iz) {
    return ((int64_t)iz * m.ny + iy) * m.nx + ix;
}

// y[n] = sum_e sum_b Ae[a(n), b] x[node(e, b)] for 3 interleaved components (stride 3) or, with
// TRANSPOSE, sum_e sum_b Ae[b, a(n)] x[...].  Ae is given as the (s_k K + s_m M) combination or G_j.
template <bool TRANSPOSE>
__device__ __forceinline__ void apply_node(const Mesh& m, int ix, int iy, int iz, const double* __restrict__ Ae,
                                           const double* __restrict__ x, int xs, int ncomp, double* y, bool& active) {
    for (int c = 0; c < ncomp; ++c) y[c] = 0.0;
    active = false;
    for (int ez = iz - 1; ez <= iz; ++ez)
        for (int ey = iy - 1; ey <= iy; ++ey)
            for (int ex = ix - 1; ex <= ix; ++ex) {
                if (!elem_on(m, ex, ey, ez)) continue;
                active = true;
                const int a = corner(ix - ex, iy - ey, iz - ez);
                for (int b = 0; b < 8; ++b) {
                    const int bx = (b == 1 || b == 2 || b == 5 || b == 6) ? 1 : 0;
                    const int by = (b == 2 || b == 3 || b == 6 || b == 7) ? 1 : 0;
                    const int bz = b >= 4 ? 1 : 0;
                    const double w = TRANSPOSE ? Ae[b * 8 + a] : Ae[a * 8 + b];
                    const int64_t j = nid(m, ex + bx, ey + by, ez + bz);
                    for (int c = 0; c < ncomp; ++c) y[c] += w * x[j * xs + c];
                }
            }
}

__device__ __forceinline__ void node_xyz(const Mesh& m, int64_t n, int& ix, int& iy, int& iz) {
    ix = (int)(n % m.nx);
    const int64_t r = n / m.nx;
    iy = (int)(r % m.ny);
    iz = (int)(r / m.ny);
}

// ----------------------------------------------------------------------------- rhs / gradient
struct RhsArgs {
    Mesh m;
    Spacing sp;
    double beta, mu, alpha;
    const double* U1;
    const double* F1;
    const double* W;
    const double* v;
    double* b;
};

// b = mu M (U1 - v) + beta sum_j G_j (F1 - W)[:,:,j] + alpha Kg U1 (subpb2_solver.global_rhs :111-130)
__global__ void rhs_kernel(RhsArgs a) {
    __shared__ ElemMats c_em;
    block_elem_mats(a.sp, c_em);
    const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (n >= a.m.n) return;
    int ix, iy, iz;
    node_xyz(a.m, n, ix, iy, iz);
    double out[3] = {0.0, 0.0, 0.0};
    for (int ez = iz - 1; ez <= iz; ++ez)
        for (int ey = iy - 1; ey <= iy; ++ey)
            for (int ex = ix - 1; ex <= ix; ++ex) {
                if (!elem_on(a.m, ex, ey, ez)) continue;
                const int ai = corner(ix - ex, iy - ey, iz - ez);
                for (int bb = 0; bb < 8; ++bb) {
                    const int bx = (bb == 1 || bb == 2 || bb == 5 || bb == 6) ? 1 : 0;
                    const int by = (bb == 2 || bb == 3 || bb == 6 || bb == 7) ? 1 : 0;
                    const int bz = bb >= 4 ? 1 : 0;
                    const int64_t j = nid(a.m, ex + bx, ey + by, ez + bz);
                    const double mw = c_em.M[ai * 8 + bb];
                    for (int c = 0; c < 3; ++c) {
                        double t = a.mu * mw * (a.U1[3 * j + c] - a.v[3 * j + c]);
                        for (int d = 0; d < 3; ++d)
                            t += a.beta * c_em.G[d][ai * 8 + bb] * (a.F1[9 * j + 3 * c + d] - a.W[9 * j + 3 * c + d]);
                        if (a.alpha != 0.0) t += a.alpha * c_em.K[ai * 8 + bb] * a.U1[3 * j + c];
                        out[c] += t;
                    }
                }
            }
    for (int c = 0; c < 3; ++c) a.b[3 * n + c] = out[c];
}

struct GradArgs {
    Mesh m;
    Spacing sp;
    const double* U;
    double* F;
};

// F_ij = (G_j^T u_i) / m_L, NaN off the active set (global_operators.nodal_gradient :151-170)
__global__ void grad_kernel(GradArgs a) {
    __shared__ ElemMats c_em;
    block_elem_mats(a.sp, c_em);
    const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (n >= a.m.n) return;
    int ix, iy, iz;
    node_xyz(a.m, n, ix, iy, iz);
    double mL = 0.0;
    double acc[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    bool active = false;
    for (int ez = iz - 1; ez <= iz; ++ez)
        for (int ey = iy - 1; ey <= iy; ++ey)
            for (int ex = ix - 1; ex <= ix; ++ex) {
                if (!elem_on(a.m, ex, ey, ez)) continue;
                active = true;
                const int bi = corner(ix - ex, iy - ey, iz - ez);
                for (int aa = 0; aa < 8; ++aa) {
                    const int ax = (aa == 1 || aa == 2 || aa == 5 || aa == 6) ? 1 : 0;
                    const int ay = (aa == 2 || aa == 3 || aa == 6 || aa == 7) ? 1 : 0;
                    const int az = aa >= 4 ? 1 : 0;
                    const int64_t j = nid(a.m, ex + ax, ey + ay, ez + az);
                    mL += c_em.M[bi * 8 + aa];
                    for (int d = 0; d < 3; ++d) {
                        const double w = c_em.G[d][aa * 8 + bi];  // (G_d^T)[n, j] = G_d[j, n]
                        for (int i = 0; i < 3; ++i) acc[i][d] += w * a.U[3 * j + i];
                    }
                }
            }
    const double safe = mL > 1e-15 ? mL : 1.0;
    for (int i = 0; i < 3; ++i)
        for (int d = 0; d < 3; ++d) a.F[9 * n + 3 * i + d] = active ? acc[i][d] / safe : nan("");
}

// ----------------------------------------------------------------------------- persistent PCG
struct PcgArgs {
    Mesh m;
    Spacing sp;
    double sk, sm;  // A = sk * Kg + sm * M
    const double* B;
    const double* X0;
    double* X;
    double* R;
    double* Z;
    double* P;
    double* AP;
    double* inv_diag;
    uint8_t* active;
    double* part;  // (3 slots, nblocks, 8)
    unsigned int* bar_count;
    unsigned int* bar_gen;
    unsigned int bar_extra;  // arrivals beyond the grid before a barrier opens (0; > 0 only in the give-up tests)
    long long spin_limit;    // polls before a waiting block gives up
    double tol;
    int max_iter;
    int32_t* iters;
    int32_t* err;
};

// Grid-wide barrier for a cooperative launch (all blocks co-resident).  The wait is bounded: on give-up
// the error word is set and the caller leaves its loop.
__device__ bool grid_sync(const PcgArgs& a) {
    __syncthreads();
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        volatile unsigned int* gen = a.bar_gen;
        const unsigned int g0 = *gen;
        __threadfence();
        const unsigned int arrived = atomicAdd(a.bar_count, 1u) + 1u;
        int ok = 1;
        if (arrived == gridDim.x + a.bar_extra) {
            *a.bar_count = 0u;
            __threadfence();
            atomicAdd(a.bar_gen, 1u);
        } else {
            long long spins = 0;
            while (*gen == g0) {
                if (++spins > a.spin_limit) {
                    atomicExch(a.err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        if (*(volatile int32_t*)a.err != 0) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// block sums of k values -> part[slot][block][0..k)
__device__ void block_partials(const PcgArgs& a, int slot, const double* v, int k) {
    __shared__ double red[PCG_THREADS / 32][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = 0; i < k; ++i) {
        const double s = warp_sum_d(v[i]);
        if (lane == 0) red[warp][i] = s;
    }
    __syncthreads();
    if (threadIdx.x < k) {
        double s = 0.0;
        for (int w = 0; w < PCG_THREADS / 32; ++w) s += red[w][threadIdx.x];
        a.part[((int64_t)slot * gridDim.x + blockIdx.x) * 8 + threadIdx.x] = s;
    }
    __syncthreads();
}

// sum over blocks (fixed order) of part[slot][*][0..k) -> out (every block gets the same values)
__device__ void total_partials(const PcgArgs& a, int slot, int k, double* out) {
    __shared__ double red[PCG_THREADS / 32][8];
    __shared__ double tot[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double v[8];
    for (int i = 0; i < k; ++i) v[i] = 0.0;
    // contiguous ranges per thread keep the order fixed for a given grid size
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
        for (int i = 0; i < k; ++i) v[i] += a.part[((int64_t)slot * gridDim.x + b) * 8 + i];
    for (int i = 0; i < k; ++i) {
        const double s = warp_sum_d(v[i]);
        if (lane == 0) red[warp][i] = s;
    }
    __syncthreads();
    if (threadIdx.x < k) {
        double s = 0.0;
        for (int w = 0; w < PCG_THREADS / 32; ++w) s += red[w][threadIdx.x];
        tot[threadIdx.x] = s;
    }
    __syncthreads();
    for (int i = 0; i < k; ++i) out[i] = tot[i];
    __syncthreads();
}

__global__ void __launch_bounds__(PCG_THREADS) pcg_kernel(PcgArgs a) {
    const int64_t N = a.m.n;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    __shared__ ElemMats c_em;
    __shared__ double Ae[64];
    block_elem_mats(a.sp, c_em);
    for (int i = threadIdx.x; i < 64; i += blockDim.x) Ae[i] = a.sk * c_em.K[i] + a.sm * c_em.M[i];
    __syncthreads();
    // set-up: active set, Jacobi diagonal, X = X0, R = B - A X, Z = D^-1 R, P = Z; dots rz and |B|^2
    double loc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int64_t n = t0; n < N; n += stride) {
        int ix, iy, iz;
        node_xyz(a.m, n, ix, iy, iz);
        double dg = 0.0;
        bool act = false;
        for (int ez = iz - 1; ez <= iz; ++ez)
            for (int ey = iy - 1; ey <= iy; ++ey)
                for (int ex = ix - 1; ex <= ix; ++ex) {
                    if (!elem_on(a.m, ex, ey, ez)) continue;
                    act = true;
                    const int c = corner(ix - ex, iy - ey, iz - ez);
                    dg += Ae[c * 8 + c];
                }
        a.active[n] = act ? 1 : 0;
        a.inv_diag[n] = (act && fabs(dg) > 1e-300) ? 1.0 / dg : 1.0;
        for (int c = 0; c < 3; ++c) {
            const double x0 = act ? a.X0[3 * n + c] : 0.0;
            a.X[3 * n + c] = x0;
            a.P[3 * n + c] = x0;  // P carries X for the first product
        }
    }
    if (!grid_sync(a)) return;
    for (int64_t n = t0; n < N; n += stride) {
        if (!a.active[n]) {
            for (int c = 0; c < 3; ++c) a.R[3 * n + c] = a.Z[3 * n + c] = a.AP[3 * n + c] = 0.0;
            continue;
        }
        int ix, iy, iz;
        node_xyz(a.m, n, ix, iy, iz);
        double ax[3];
        bool act;
        apply_node<false>(a.m, ix, iy, iz, Ae, a.P, 3, 3, ax, act);
        for (int c = 0; c < 3; ++c) {
            const double b = a.B[3 * n + c];
            const double r = b - ax[c];
            const double z = a.inv_diag[n] * r;
            a.R[3 * n + c] = r;
            a.Z[3 * n + c] = z;
            loc[c] += r * z;
            loc[3 + c] += b * b;
        }
    }
    if (!grid_sync(a)) return;
    for (int64_t n = t0; n < N; n += stride)
        for (int c = 0; c < 3; ++c) a.P[3 * n + c] = a.Z[3 * n + c];
    block_partials(a, 0, loc, 6);
    if (!grid_sync(a)) return;
    double tot[8];
    total_partials(a, 0, 6, tot);
    double rz[3], bnorm[3];
    for (int c = 0; c < 3; ++c) {
        rz[c] = tot[c];
        bnorm[c] = sqrt(tot[3 + c]);
        if (bnorm[c] == 0.0) bnorm[c] = 1.0;
    }
    int it = 0;
    for (it = 1; it <= a.max_iter; ++it) {
        // AP = A P, denom = P . AP
        for (int c = 0; c < 8; ++c) loc[c] = 0.0;
        for (int64_t n = t0; n < N; n += stride) {
            if (!a.active[n]) continue;
            int ix, iy, iz;
            node_xyz(a.m, n, ix, iy, iz);
            double ap[3];
            bool act;
            apply_node<false>(a.m, ix, iy, iz, Ae, a.P, 3, 3, ap, act);
            for (int c = 0; c < 3; ++c) {
                a.AP[3 * n + c] = ap[c];
                loc[c] += a.P[3 * n + c] * ap[c];
            }
        }
        block_partials(a, 1, loc, 3);
        if (!grid_sync(a)) return;
        total_partials(a, 1, 3, tot);
        double alpha[3];
        for (int c = 0; c < 3; ++c) {
            const double den = tot[c] == 0.0 ? INFINITY : tot[c];
            alpha[c] = rz[c] / den;
        }
        // X += alpha P, R -= alpha AP, |R|^2, Z = D^-1 R, R . Z
        for (int c = 0; c < 8; ++c) loc[c] = 0.0;
        for (int64_t n = t0; n < N; n += stride) {
            if (!a.active[n]) continue;
            for (int c = 0; c < 3; ++c) {
                a.X[3 * n + c] += a.P[3 * n + c] * alpha[c];
                const double r = a.R[3 * n + c] - a.AP[3 * n + c] * alpha[c];
                a.R[3 * n + c] = r;
                const double z = a.inv_diag[n] * r;
                a.Z[3 * n + c] = z;
                loc[c] += r * r;
                loc[3 + c] += r * z;
            }
        }
        block_partials(a, 2, loc, 6);
        if (!grid_sync(a)) return;
        total_partials(a, 2, 6, tot);
        bool conv = true;
        for (int c = 0; c < 3; ++c) conv = conv && (sqrt(tot[c]) / bnorm[c] < a.tol);
        if (conv) break;
        double beta[3];
        for (int c = 0; c < 3; ++c) {
            beta[c] = tot[3 + c] / (rz[c] == 0.0 ? INFINITY : rz[c]);
            rz[c] = tot[3 + c];
        }
        for (int64_t n = t0; n < N; n += stride) {
            if (!a.active[n]) continue;
            for (int c = 0; c < 3; ++c) a.P[3 * n + c] = a.Z[3 * n + c] + a.P[3 * n + c] * beta[c];
        }
        if (!grid_sync(a)) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.iters = it > a.max_iter ? a.max_iter : it;
    // off the active set X keeps X0 (solve_subpb2 :152-153)
    for (int64_t n = t0; n < N; n += stride)
        if (!a.active[n])
            for (int c = 0; c < 3; ++c) a.X[3 * n + c] = a.X0[3 * n + c];
}

static int set_mesh(const aldvc_hex8_mesh* mesh, Mesh& m, Spacing& sp) {
    ALDVC_REQUIRE(mesh, "hex8: null mesh");
    ALDVC_REQUIRE(mesh->nx >= 2 && mesh->ny >= 2 && mesh->nz >= 2, "hex8: need >= 2 nodes per axis");
    ALDVC_REQUIRE(mesh->sx > 0 && mesh->sy > 0 && mesh->sz > 0, "hex8: spacing must be positive");
    ALDVC_REQUIRE(mesh->gauss_order >= 1 && mesh->gauss_order <= 3, "hex8: gauss_order must be 1, 2 or 3");
    ALDVC_REQUIRE(mesh->nx < (1 << 30) && mesh->ny < (1 << 30) && mesh->nz < (1 << 30), "hex8: grid too large");
    m.nx = (int)mesh->nx;
    m.ny = (int)mesh->ny;
    m.nz = (int)mesh->nz;
    m.n = mesh->nx * mesh->ny * mesh->nz;
    m.elem_active = mesh->elem_active;
    sp.sx = mesh->sx;
    sp.sy = mesh->sy;
    sp.sz = mesh->sz;
    sp.order = mesh->gauss_order;
    return ALDVC_OK;
}

}  // namespace aldvc

using namespace aldvc;

extern "C" int aldvc_global_rhs(const aldvc_hex8_mesh* mesh, double beta, double mu, double alpha, const double* U1,
                                const double* F1, const double* W, const double* v, double* b, void* stream) {
    ALDVC_REQUIRE(U1 && F1 && W && v && b, "aldvc_global_rhs: null pointer");
    cudaStream_t s = (cudaStream_t)stream;
    Mesh m;
    Spacing sp;
    int rc = set_mesh(mesh, m, sp);
    if (rc) return rc;
    RhsArgs a{m, sp, beta, mu, alpha, U1, F1, W, v, b};
    {
        KTimer kt_("global_rhs", s);
        rhs_kernel<<<(unsigned)((m.n + 255) / 256), 256, 0, s>>>(a);
    }
    return check_launch("aldvc_global_rhs");
}

extern "C" int aldvc_nodal_gradient(const aldvc_hex8_mesh* mesh, const double* U, double* F, void* stream) {
    ALDVC_REQUIRE(U && F, "aldvc_nodal_gradient: null pointer");
    cudaStream_t s = (cudaStream_t)stream;
    Mesh m;
    Spacing sp;
    int rc = set_mesh(mesh, m, sp);
    if (rc) return rc;
    GradArgs a{m, sp, U, F};
    {
        KTimer kt_("nodal_gradient", s);
        grad_kernel<<<(unsigned)((m.n + 255) / 256), 256, 0, s>>>(a);
    }
    return check_launch("aldvc_nodal_gradient");
}

static std::mutex g_pcg_grid_mu;
static int g_pcg_grid[128] = {0};  // co-resident grid of the cooperative PCG, per device ordinal

// The cooperative grid of the current device: every block resident at once.  Queried once per device
// (no configuration call inside a stream capture after the first use).
static int pcg_grid(int* grid_out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "pcg: current device");
    if (dev < 0 || dev >= 128) return arg_fail("pcg: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_pcg_grid_mu);
    if (g_pcg_grid[dev] == 0) {
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_kernel, PCG_THREADS, 0);
        if (e != cudaSuccess) return cuda_fail(e, "pcg: occupancy");
        if (per_sm < 1) return arg_fail("pcg: kernel does not fit on an SM");
        cudaDeviceProp p;
        e = cudaGetDeviceProperties(&p, dev);
        if (e != cudaSuccess) return cuda_fail(e, "pcg: device properties");
        g_pcg_grid[dev] = per_sm * p.multiProcessorCount;
    }
    *grid_out = g_pcg_grid[dev];
    return ALDVC_OK;
}

extern "C" size_t aldvc_pcg_workspace_size(const aldvc_hex8_mesh* mesh) {
    if (!mesh) return 0;
    const int64_t n = mesh->nx * mesh->ny * mesh->nz;
    int grid = 0;
    if (pcg_grid(&grid) != ALDVC_OK) grid = 148 * 8;
    return align_up((size_t)n * 3 * sizeof(double), 256) * 5 + align_up((size_t)n * sizeof(double), 256) +
           align_up((size_t)n, 256) + align_up((size_t)3 * grid * 8 * sizeof(double), 256) + 256;
}

extern "C" int aldvc_pcg_hex8(const aldvc_hex8_mesh* mesh, double beta, double mu, double alpha, const double* B,
                              const double* X0, double tol, int32_t max_iter, void* workspace, size_t workspace_bytes, double* X,
                              int32_t* iters, int32_t* err, void* stream) {
    ALDVC_REQUIRE(B && X0 && X && iters && err, "aldvc_pcg_hex8: null pointer");
    ALDVC_REQUIRE(max_iter >= 0, "aldvc_pcg_hex8: max_iter must be >= 0");
    cudaStream_t s = (cudaStream_t)stream;
    Mesh m;
    Spacing sp;
    int rc = set_mesh(mesh, m, sp);
    if (rc) return rc;
    const size_t need = aldvc_pcg_workspace_size(mesh);
    if (!workspace || workspace_bytes < need) {
        set_error("aldvc_pcg_hex8: workspace of %zu bytes needed, %zu given", need, workspace_bytes);
        return ALDVC_ERR_WORKSPACE;
    }
    int grid = 0;
    rc = pcg_grid(&grid);
    if (rc) return rc;
    const int64_t n = m.n;
    char* w = (char*)workspace;
    const size_t v3 = align_up((size_t)n * 3 * sizeof(double), 256);
    PcgArgs a;
    a.m = m;
    a.sp = sp;
    a.sk = beta + alpha;
    a.sm = mu;
    a.B = B;
    a.X0 = X0;
    a.X = X;
    a.R = (double*)w;
    a.Z = (double*)(w + v3);
    a.P = (double*)(w + 2 * v3);
    a.AP = (double*)(w + 3 * v3);
    a.part = (double*)(w + 4 * v3);
    const size_t pb = align_up((size_t)3 * grid * 8 * sizeof(double), 256);
    a.inv_diag = (double*)(w + 4 * v3 + pb);
    a.active = (uint8_t*)(w + 4 * v3 + pb + align_up((size_t)n * sizeof(double), 256));
    a.bar_count = (unsigned int*)(w + 4 * v3 + pb + align_up((size_t)n * sizeof(double), 256) + align_up((size_t)n, 256));
    a.bar_gen = a.bar_count + 1;
    const BarrierParams bp = barrier_params();
    a.bar_extra = bp.extra;
    a.spin_limit = bp.spin_limit;
    a.tol = tol;
    a.max_iter = max_iter;
    a.iters = iters;
    a.err = err;
    cudaError_t e = cudaMemsetAsync(a.bar_count, 0, 2 * sizeof(unsigned int), s);
    if (e != cudaSuccess) return cuda_fail(e, "pcg: barrier reset");
    e = cudaMemsetAsync(err, 0, sizeof(int32_t), s);
    if (e != cudaSuccess) return cuda_fail(e, "pcg: error word reset");
    void* args[] = {&a};
    {
        KTimer kt_("pcg_hex8", s);
        e = cudaLaunchCooperativeKernel((const void*)pcg_kernel, dim3(grid), dim3(PCG_THREADS), args, 0, s);
    }
    if (e != cudaSuccess) return cuda_fail(e, "pcg: cooperative launch");
    count_launch();
    return ALDVC_OK;
}

// ----------------------------------------------------------------------------- PCG without allocation
// Some callers cannot allocate device memory at all: a plugin running inside a larger imaging
// application whose own allocator owns the device budget, or a real-time acquisition loop that must not
// call cudaMalloc (it synchronises the device and can stall for milliseconds).  For them this variant
// of the PCG keeps its scratch (residual, preconditioned residual, direction, A*direction, Jacobi
// diagonal, active set, block partials, barrier words) in one file-scope device array instead of a
// caller-provided workspace.  The caller still passes B, X0, X, iters and err.
//
// The array is NOALLOC_PCG_BYTES of device memory held by every GPU that loads the library, until the
// process exits.  It bounds the mesh to NOALLOC_PCG_MAX_NODES nodes; larger meshes are rejected.
// All calls share the array and it keeps the last call's contents: the barrier words are cleared on
// every call and every other region is written by the kernel before it is read.  Calls whose kernels
// overlap on the GPU (different streams without ordering, or different host threads) race on the
// array.  The first call on a device looks up the array's device address (cudaGetSymbolAddress,
// with that device current); make that first call before any stream capture.
constexpr int64_t NOALLOC_PCG_MAX_NODES = 262144;
constexpr int NOALLOC_PCG_MAX_GRID = 4096;
constexpr size_t NOALLOC_V3 = (size_t)NOALLOC_PCG_MAX_NODES * 3 * sizeof(double);
constexpr size_t NOALLOC_PART = (size_t)3 * NOALLOC_PCG_MAX_GRID * 8 * sizeof(double);
constexpr size_t NOALLOC_PCG_BYTES =
    4 * NOALLOC_V3 + NOALLOC_PART + (size_t)NOALLOC_PCG_MAX_NODES * sizeof(double) + (size_t)NOALLOC_PCG_MAX_NODES + 256;

static __device__ __align__(256) unsigned char g_pcg_scratch[NOALLOC_PCG_BYTES];

static std::mutex g_pcg_scratch_mu;
static char* g_pcg_scratch_ptr[128] = {nullptr};  // device address of the array, per device ordinal

// set-up once per device, with that device current
static int pcg_scratch_address(char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "aldvc_pcg_hex8_noalloc: current device");
    if (dev < 0 || dev >= 128) return arg_fail("aldvc_pcg_hex8_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_pcg_scratch_mu);
    if (!g_pcg_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_pcg_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "aldvc_pcg_hex8_noalloc: scratch address");
        g_pcg_scratch_ptr[dev] = (char*)p;
    }
    *out = g_pcg_scratch_ptr[dev];
    return ALDVC_OK;
}

extern "C" int64_t aldvc_pcg_hex8_noalloc_max_nodes(void) { return NOALLOC_PCG_MAX_NODES; }

extern "C" int aldvc_pcg_hex8_noalloc(const aldvc_hex8_mesh* mesh, double beta, double mu, double alpha, const double* B,
                                      const double* X0, double tol, int32_t max_iter, double* X, int32_t* iters, int32_t* err,
                                      void* stream) {
    ALDVC_REQUIRE(B && X0 && X && iters && err, "aldvc_pcg_hex8_noalloc: null pointer");
    ALDVC_REQUIRE(max_iter >= 0, "aldvc_pcg_hex8_noalloc: max_iter must be >= 0");
    Mesh m;
    Spacing sp;
    int rc = set_mesh(mesh, m, sp);
    if (rc) return rc;
    if (m.n > NOALLOC_PCG_MAX_NODES) {
        set_error("aldvc_pcg_hex8_noalloc: mesh of %lld nodes exceeds the %lld-node limit of the built-in scratch; "
                  "use aldvc_pcg_hex8 with a workspace",
                  (long long)m.n, (long long)NOALLOC_PCG_MAX_NODES);
        return ALDVC_ERR_ARG;
    }
    int grid = 0;
    rc = pcg_grid(&grid);
    if (rc) return rc;
    if (grid > NOALLOC_PCG_MAX_GRID) grid = NOALLOC_PCG_MAX_GRID;
    char* w = nullptr;
    rc = pcg_scratch_address(&w);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    PcgArgs a;
    a.m = m;
    a.sp = sp;
    a.sk = beta + alpha;
    a.sm = mu;
    a.B = B;
    a.X0 = X0;
    a.X = X;
    a.R = (double*)w;
    a.Z = (double*)(w + NOALLOC_V3);
    a.P = (double*)(w + 2 * NOALLOC_V3);
    a.AP = (double*)(w + 3 * NOALLOC_V3);
    a.part = (double*)(w + 4 * NOALLOC_V3);
    a.inv_diag = (double*)(w + 4 * NOALLOC_V3 + NOALLOC_PART);
    a.active = (uint8_t*)(w + 4 * NOALLOC_V3 + NOALLOC_PART + (size_t)NOALLOC_PCG_MAX_NODES * sizeof(double));
    a.bar_count = (unsigned int*)(w + 4 * NOALLOC_V3 + NOALLOC_PART + (size_t)NOALLOC_PCG_MAX_NODES * sizeof(double) +
                                  (size_t)NOALLOC_PCG_MAX_NODES);
    a.bar_gen = a.bar_count + 1;
    const BarrierParams bp = barrier_params();
    a.bar_extra = bp.extra;
    a.spin_limit = bp.spin_limit;
    a.tol = tol;
    a.max_iter = max_iter;
    a.iters = iters;
    a.err = err;
    // the barrier words must start at zero on every call; everything else is written before it is read
    cudaError_t e = cudaMemsetAsync(a.bar_count, 0, 2 * sizeof(unsigned int), s);
    if (e != cudaSuccess) return cuda_fail(e, "aldvc_pcg_hex8_noalloc: barrier reset");
    e = cudaMemsetAsync(err, 0, sizeof(int32_t), s);
    if (e != cudaSuccess) return cuda_fail(e, "aldvc_pcg_hex8_noalloc: error word reset");
    void* args[] = {&a};
    {
        KTimer kt_("pcg_hex8_noalloc", s);
        e = cudaLaunchCooperativeKernel((const void*)pcg_kernel, dim3(grid), dim3(PCG_THREADS), args, 0, s);
    }
    if (e != cudaSuccess) return cuda_fail(e, "aldvc_pcg_hex8_noalloc: cooperative launch");
    count_launch();
    return ALDVC_OK;
}
