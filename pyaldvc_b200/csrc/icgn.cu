// 12-DOF and 3-DOF inverse-compositional Gauss-Newton subset solvers (pyALDVC numba_kernels.py:517-1208).
//
// Two forms of the same method:
//
//  * BATCHED -- a persistent kernel: one CTA per SM slot pulls node indices from a device work counter and
//    iterates each node to its own exit.  Per iteration the warped subset is covered by one or more
//    z-chunks; each chunk's deformed-volume box is staged in shared memory with coalesced row loads and
//    every subset voxel samples it there.  The residual of the ZNSSD criterion is linear in the sampled
//    value, so one pass accumulates all moments (sum SD_k, SD_k f, SD_k g, f, f^2, g, g^2, f g) and the
//    gradient b and the ZNCC follow from them in FP64 -- no per-voxel sample buffer, no second pass.
//    Intensities are centred (f - meanf_precomputed, g - meang_previous) so the moments do not cancel.
//
//  * PLAIN -- one block per node, the layout of the reference's numba-cuda kernels: pass 1 samples g from
//    global memory into a per-node global buffer and reduces the statistics, pass 2 re-reads the buffer
//    and reduces the gradient.  It is the comparison baseline for the batched form.
//
// Both accumulate in FP32 per thread (<= S / threads voxels each), reduce in FP32 within a warp and in
// FP64 across warps; thread 0 runs the per-iteration control in FP64 (Cholesky solve, stopping rules,
// warp composition) exactly as the reference does.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include <cudaTypedefs.h>

#include "common.cuh"
#include "internal.cuh"

namespace aldvc {

struct IcgnArgs {
    // volumes
    const float* f;
    const float* gx;
    const float* gy;
    const float* gz;
    const uint8_t* mask;
    const float* g;
    const float4* g4;  // optional overlapping-quad copy of g (cubic modes of the persistent kernel)
    int nz, ny, nx;
    // subset
    int hx, hy, hz, stride, nX, nY, nZ;
    const int64_t* split_index;
    const uint8_t* split_keep;
    int64_t keep_bytes;
    // nodes
    const int64_t* coords;
    int64_t n_nodes;
    int64_t node_base;  // plain: first node of this launch
    const uint8_t* valid;
    const double* meanf;
    // 12-DOF
    const double* P0;
    const double* L;
    const double* H;
    const double* pattern;
    // 3-DOF
    const double* U_old;
    const double* F_fixed;
    const double* vdual;
    const double* bottomf;
    double mu, n_full;
    // controls
    double tol, dp_tol, noise_gain;
    int max_iter, patience, predictive;
    // outputs
    double* P_out;  // 12-DOF (N,12) / 3-DOF (N,3)
    int32_t* n_iter;
    int8_t* status;
    double* zncc;
    // scratch
    int* counter;       // batched work queue
    float* gbuf;        // plain: (blocks, S)
    int brick_cap;      // batched: floats of the shared brick
    const int32_t* node_half;  // (N,3) per-node half-widths (<= hx, hy, hz), NULL: one shape
    int sweep_rows;     // lean: subset rows per sweep tile (0 automatic, < 0 the whole subset)
    const int32_t* node_order;  // persistent forms: the work queue's permutation of the nodes, NULL: index order
    int32_t* err;       // persistent forms: nonzero when a bounded wait on a staged copy gave up
    int idx32;          // every voxel index of the volumes below 2^31: the lean sweep forms 32-bit indices
};

// ----------------------------------------------------------------------------- TMA staging of the lean sweep
// The staged form of the lean kernel copies, for each chunk of its sweep (a tile of `by` subset rows times
// TMA_KZ sample planes), the box of g that the chunk's cubic taps read into shared memory with one tensor copy
// (cp.async.bulk.tensor, completion on an mbarrier), double-buffered: the copy of chunk c + 2 runs while chunk c + 1
// is sampled.  The box is fixed (TMA_BX x TMA_BY x TMA_BZ floats, x fastest); a chunk whose warped footprint does not
// fit is sampled from global memory.  The tensor map covers this device's g only; no multicast.
constexpr int TMA_BX = 48, TMA_BY = 12, TMA_BZ = 10, TMA_KZ = 3;
constexpr int TMA_BOX = TMA_BX * TMA_BY * TMA_BZ;                // floats per buffer
constexpr unsigned TMA_BOX_BYTES = TMA_BOX * sizeof(float);       // 23,040 bytes
constexpr size_t TMA_SMEM = 2 * (size_t)TMA_BOX_BYTES + 128;      // two buffers, 128-byte aligned
constexpr long long TMA_WAIT_LIMIT = 1LL << 20;                    // polls of an mbarrier before a wait gives up

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint32_t mb, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mb), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t mb, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t mb, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(mb), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait for the phase `parity` of an mbarrier to complete; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint32_t mb, uint32_t parity) {
    for (long long i = 0; i < TMA_WAIT_LIMIT; ++i)
        if (mbar_try_wait(mb, parity)) return true;
    return false;
}
// 3-D tiled tensor copy of the box at (x, y, z) of the map into shared memory; x must be a multiple of 4 (16 bytes)
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t mb) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(mb)
        : "memory");
}

// The node the q-th work item solves: node_order[q] (entries outside 0..n-1 are skipped: -2), or q; -1 past the end.
__device__ __forceinline__ int64_t queue_node(const IcgnArgs& a, int q) {
    if (q >= a.n_nodes) return -1;
    if (!a.node_order) return q;
    const int64_t nd = a.node_order[q];
    return (nd >= 0 && nd < a.n_nodes) ? nd : -2;
}

// Rows per sweep tile of the lean kernel.  The subset is swept tile by tile, each tile plane by plane (z) and
// row by row, so the tap rows a plane of samples shares with the next planes are still in L1 when they are
// read again: the working set is (rows + 3) tap rows of four planes instead of the whole subset's rows.
// req > 0: that height (at most nY); req < 0: the whole subset (C order); 0: a height of 3 to 6 rows that pads
// the fewest rows of the last tile (ties: the shorter), the whole subset when it has at most 6 rows.  On the
// 1024 x 1024 x 306 workload (33^3 subsets) the 12-DOF sweep takes 225 ms per pass in C order, 201 ms with
// 11-row tiles, 191 with 6 and 182 with 3 (the 3-DOF sweep 89, 86 and 82 ms).
__device__ __forceinline__ int sweep_rows(int nY, int req) {
    if (req < 0 || nY <= 6) return nY;
    if (req > 0) return req < nY ? req : nY;
    int best = nY, waste = 1 << 30;
    for (int b = 3; b <= 6; ++b) {
        const int w = (nY + b - 1) / b * b - nY;
        if (w < waste) {
            waste = w;
            best = b;
        }
    }
    return best;
}

// Subset shape of one node: the call's, or the node's own (node_half); ok is false when a node's own shape
// exceeds the call's maximum (the node is then invalid: buffers and bricks are sized by the maximum).
struct Shape {
    int hx, hy, hz, nX, nY, nZ;
};

__device__ __forceinline__ Shape node_shape(const IcgnArgs& a, int64_t node, bool& ok) {
    ok = true;
    if (!a.node_half) return Shape{a.hx, a.hy, a.hz, a.nX, a.nY, a.nZ};
    const int hx = a.node_half[3 * node], hy = a.node_half[3 * node + 1], hz = a.node_half[3 * node + 2];
    ok = hx >= 0 && hy >= 0 && hz >= 0 && hx <= a.hx && hy <= a.hy && hz <= a.hz;
    if (!ok) return Shape{a.hx, a.hy, a.hz, a.nX, a.nY, a.nZ};
    return Shape{hx, hy, hz, (2 * hx) / a.stride + 1, (2 * hy) / a.stride + 1, (2 * hz) / a.stride + 1};
}

// ----------------------------------------------------------------------------- per-node control state
struct Ctl12 {
    double P[12], P_best[12];
    double norm_init, last_dp, dp_prev, best_zncc, best_dp, zncc;
    int stall;
    double half_scale;
};

struct Ctl3 {
    double P[12];
    double Hinv[3][3];
    double u_old[3], vd[3];
    double bf2, norm_init, last_dn, dn_prev, best_dn, zncc;
    int stall;
    const double* H;
};

// Sums of one iteration after the block reduction (FP64, shifted moments).
struct Moments {
    int64_t n, nref;
    int oob;
    double Sg, Sgg, Sf, Sff, Sfg;
    double SD[12], SDf[12], SDg[12];
};

// Statistics of the dynamic valid set (numba_kernels._warp_and_sample :586-598) and the gradient
// b_k = bottomf * sum SD_k * res with res = (f - mf)/bf - (g - mg)/bg, from the shifted moments.
// Returns 0 = ok, ST_OOB or ST_INVALID.
__device__ __noinline__ int finish_moments(const Moments& m, double cf, double cg, int nb, double* b, double& bf, double& bg, double& s_cc,
                              int64_t& n_valid) {
    n_valid = m.n;
    if (m.oob) return ST_OOB;
    if (m.n < MIN_SUBSET_VOXELS || (double)m.n < MIN_VALID_FRACTION * (double)m.nref) return ST_INVALID;
    const double n = (double)m.n;
    const double mg = m.Sg / n, mf = m.Sf / n;
    double ssg = m.Sgg - n * mg * mg;
    if (ssg < 0.0) ssg = 0.0;
    double ssf = m.Sff - n * mf * mf;
    if (ssf < 0.0) ssf = 0.0;
    bg = sqrt(ssg > 1e-30 ? ssg : 1e-30);
    bf = sqrt(ssf > 1e-30 ? ssf : 1e-30);
    const double r = bf / bg;
    for (int k = 0; k < nb; ++k) b[k] = (m.SDf[k] - mf * m.SD[k]) - r * (m.SDg[k] - mg * m.SD[k]);
    s_cc = m.Sfg - n * mf * mg;
    (void)cf;
    (void)cg;
    return 0;
}

__device__ __noinline__ bool corrected_chol12(const double* H, const double* pattern, double corr, double* H0, double* L0) {
    double limit = 1.0;
    for (int i = 9; i < 12; ++i) {
        const double c = corr * pattern[i * 12 + i];
        if (c > 0.0) {
            const double lim = (1.0 - MIN_CORRECTED_FRACTION) * H[i * 12 + i] / c;
            if (lim < limit) limit = lim;
        }
    }
    if (limit <= 0.0) return false;
    for (int i = 0; i < 144; ++i) H0[i] = H[i] - corr * limit * pattern[i];
    return chol12(H0, L0);
}

// One 12-DOF control step after the sampling pass (numba_kernels._icgn_12dof_single :686-790).
// Returns -1 to continue, else the final status; writes zncc_out on finish.
__device__ __noinline__ int control12(Ctl12& s, const double* b_in, double bottomf_d, double bottomg, double s_cc, int64_t n_valid,
                         const double* L, const double* H, const double* pattern, double noise_gain, double tol, double dp_tol,
                         int patience, int predictive, double& zncc_out) {
    double b[12], negb[12], dP[12];
    double norm_abs = 0.0;
    for (int k = 0; k < 12; ++k) {
        b[k] = b_in[k];
        norm_abs += b[k] * b[k];
    }
    norm_abs = sqrt(norm_abs);
    if (!isfinite(norm_abs)) {
        zncc_out = nan("");
        return ST_NAN;
    }
    if (s.norm_init < 0.0) s.norm_init = norm_abs;
    const double norm_rel = s.norm_init > 1e-300 ? norm_abs / s.norm_init : 0.0;
    const double inv_bf = 1.0 / bottomf_d, inv_bg = 1.0 / bottomg;
    const double zncc = s_cc * inv_bf * inv_bg;
    s.zncc = zncc;
    if (norm_rel < tol || norm_abs < ABS_TOL) {
        zncc_out = zncc;
        return ST_CONVERGED;
    }
    for (int k = 0; k < 12; ++k) negb[k] = -b[k];
    bool use_corr = false;
    double H0[144], L0[144];
    const double n_full = pattern ? pattern[9 * 12 + 9] : 0.0;
    if (noise_gain > 0.0 && n_full > 0.0 && s.last_dp < NOISE_CORR_STEP && H) {
        const double s2 = (1.0 - zncc > 0.0 ? 1.0 - zncc : 0.0) * bottomf_d * bottomf_d / (double)n_valid;
        const double corr = noise_gain * s2 * ((double)n_valid / n_full);
        use_corr = corrected_chol12(H, pattern, corr, H0, L0);
    }
    chol_solve12(use_corr ? L0 : L, negb, dP);
    double dp_norm = 0.0;
    for (int k = 0; k < 9; ++k) {
        const double v = dP[k] * s.half_scale;
        dp_norm += v * v;
    }
    for (int k = 9; k < 12; ++k) dp_norm += dP[k] * dP[k];
    dp_norm = sqrt(dp_norm);
    if (!isfinite(dp_norm)) {
        zncc_out = nan("");
        return ST_NAN;
    }
    s.last_dp = dp_norm;
    if (dp_norm < dp_tol) {
        zncc_out = zncc;
        return ST_CONVERGED;
    }
    if (predictive && s.dp_prev > 0.0 && dp_norm < PREDICT_CONTRACTION * s.dp_prev && dp_norm * dp_norm < dp_tol * s.dp_prev) {
        zncc_out = zncc;
        if (!compose_warp(s.P, dP)) return ST_SINGULAR;
        return ST_CONVERGED;
    }
    s.dp_prev = dp_norm;
    bool improved = zncc > s.best_zncc + STALL_ZNCC_EPS;
    if (improved) {
        s.best_zncc = zncc;
        for (int k = 0; k < 12; ++k) s.P_best[k] = s.P[k];
    }
    if (dp_norm < s.best_dp * STALL_STEP_DECAY) {
        s.best_dp = dp_norm;
        improved = true;
    }
    if (improved) {
        s.stall = 0;
    } else {
        s.stall += 1;
        if (patience > 0 && s.stall >= patience) {
            for (int k = 0; k < 12; ++k) s.P[k] = s.P_best[k];
            zncc_out = s.best_zncc;
            return ST_STALLED;
        }
    }
    if (!compose_warp(s.P, dP)) {
        zncc_out = zncc;
        return ST_SINGULAR;
    }
    return -1;
}

// numba_kernels._build_h3 (:910-928)
__device__ __noinline__ bool build_h3(const double* H, double bf2, double mu, double corr, double Hinv[3][3]) {
    double H3[3][3], Hd[3][3];
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) H3[i][j] = H[(9 + i) * 12 + 9 + j] * 2.0 / bf2;
        const double limit_i = (1.0 - MIN_CORRECTED_FRACTION) * H[(9 + i) * 12 + 9 + i];
        const double cc = corr < limit_i ? corr : limit_i;
        H3[i][i] -= cc * 2.0 / bf2;
        H3[i][i] += mu;
    }
    const double md = H3[1][1] > H3[2][2] ? H3[1][1] : H3[2][2];
    const double max_diag = H3[0][0] > md ? H3[0][0] : md;
    if (!(max_diag > 0.0)) return false;
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) Hd[i][j] = H3[i][j];
        Hd[i][i] += LM_DAMPING_3DOF * max_diag;
    }
    return inv3(Hd, Hinv) != 0.0;
}

// One 3-DOF control step (numba_kernels._icgn_3dof_single :1033-1080).
__device__ __noinline__ int control3(Ctl3& s, const double* b_in, double bottomf_d, double bottomg, double s_cc, int64_t n_valid, double mu,
                        double noise_gain, double tol, double dp_tol, int patience, int predictive, double& zncc_out) {
    double tb[3], dt[3];
    double norm_abs = 0.0;
    for (int k = 0; k < 3; ++k) {
        tb[k] = b_in[k] * 2.0 / s.bf2 + mu * (s.P[9 + k] - s.u_old[k] - s.vd[k]);
        norm_abs += tb[k] * tb[k];
    }
    norm_abs = sqrt(norm_abs);
    if (!isfinite(norm_abs)) {
        zncc_out = nan("");
        return ST_NAN;
    }
    if (s.norm_init < 0.0) s.norm_init = norm_abs;
    const double norm_rel = s.norm_init > 1e-300 ? norm_abs / s.norm_init : 0.0;
    const double zncc = s_cc * (1.0 / bottomf_d) * (1.0 / bottomg);
    s.zncc = zncc;
    if (norm_rel < tol || norm_abs < mu * 1e-4) {
        zncc_out = zncc;
        return ST_CONVERGED;
    }
    if (noise_gain > 0.0 && s.last_dn < NOISE_CORR_STEP) {
        const double s2 = (1.0 - zncc > 0.0 ? 1.0 - zncc : 0.0) * bottomf_d * bottomf_d / (double)n_valid;
        if (!build_h3(s.H, s.bf2, mu, noise_gain * s2 * (double)n_valid, s.Hinv)) build_h3(s.H, s.bf2, mu, 0.0, s.Hinv);
    }
    for (int i = 0; i < 3; ++i) {
        double t = 0.0;
        for (int j = 0; j < 3; ++j) t += s.Hinv[i][j] * tb[j];
        dt[i] = -t;
    }
    const double dn = sqrt(dt[0] * dt[0] + dt[1] * dt[1] + dt[2] * dt[2]);
    if (!isfinite(dn)) {
        zncc_out = nan("");
        return ST_NAN;
    }
    s.last_dn = dn;
    if (dn < dp_tol) {
        zncc_out = zncc;
        return ST_CONVERGED;
    }
    const double a00 = 1.0 + s.P[0], a01 = s.P[1], a02 = s.P[2];
    const double a10 = s.P[3], a11 = 1.0 + s.P[4], a12 = s.P[5];
    const double a20 = s.P[6], a21 = s.P[7], a22 = 1.0 + s.P[8];
    if (predictive && s.dn_prev > 0.0 && dn < PREDICT_CONTRACTION * s.dn_prev && dn * dn < dp_tol * s.dn_prev) {
        s.P[9] -= a00 * dt[0] + a01 * dt[1] + a02 * dt[2];
        s.P[10] -= a10 * dt[0] + a11 * dt[1] + a12 * dt[2];
        s.P[11] -= a20 * dt[0] + a21 * dt[1] + a22 * dt[2];
        zncc_out = zncc;
        return ST_CONVERGED;
    }
    s.dn_prev = dn;
    if (dn < s.best_dn * STALL_STEP_DECAY) {
        s.best_dn = dn;
        s.stall = 0;
    } else {
        s.stall += 1;
        if (patience > 0 && s.stall >= patience) {
            zncc_out = zncc;
            return ST_STALLED;
        }
    }
    s.P[9] -= a00 * dt[0] + a01 * dt[1] + a02 * dt[2];
    s.P[10] -= a10 * dt[0] + a11 * dt[1] + a12 * dt[2];
    s.P[11] -= a20 * dt[0] + a21 * dt[1] + a22 * dt[2];
    return -1;
}

// ----------------------------------------------------------------------------- node set-up / write-back (thread 0)
// Returns true when the node is to be iterated; otherwise its outputs are already written.
template <int NDOF>
__device__ __noinline__ bool node_begin(const IcgnArgs& a, int64_t node, Ctl12& c12, Ctl3& c3, const Shape& sh, bool shape_ok) {
    if (NDOF == 12) {
        const double* P0 = a.P0 + node * 12;
        double* Po = a.P_out + node * 12;
        bool finite = true;
        for (int k = 0; k < 12; ++k) {
            const double v = P0[k];
            Po[k] = v;
            c12.P[k] = v;
            c12.P_best[k] = v;
            finite = finite && isfinite(v);
        }
        a.n_iter[node] = 0;
        a.zncc[node] = nan("");
        if (!a.valid[node] || !shape_ok) {
            a.status[node] = ST_INVALID;
            return false;
        }
        if (!finite) {
            a.status[node] = ST_NAN;
            return false;
        }
        c12.norm_init = -1.0;
        c12.last_dp = 1e300;
        c12.dp_prev = -1.0;
        c12.best_zncc = -2.0;
        c12.best_dp = 1e300;
        c12.zncc = nan("");
        c12.stall = 0;
        c12.half_scale = (double)max(sh.hx, max(sh.hy, sh.hz));
        return true;
    } else {
        double* Uo = a.P_out + node * 3;
        bool finite = true;
        for (int k = 0; k < 9; ++k) {
            c3.P[k] = a.F_fixed[node * 9 + k];
            finite = finite && isfinite(c3.P[k]);
        }
        for (int k = 0; k < 3; ++k) {
            const double u = a.U_old[node * 3 + k];
            Uo[k] = u;
            c3.P[9 + k] = u;
            c3.u_old[k] = u;
            c3.vd[k] = a.vdual[node * 3 + k];
            finite = finite && isfinite(u);
        }
        a.n_iter[node] = 0;
        a.zncc[node] = nan("");
        if (!a.valid[node] || !shape_ok) {
            a.status[node] = ST_INVALID;
            return false;
        }
        if (!finite) {
            a.status[node] = ST_NAN;
            return false;
        }
        double bf = a.bottomf[node];
        double bf2 = bf * bf;
        if (bf2 < 1e-30) bf2 = 1e-30;
        c3.bf2 = bf2;
        c3.H = a.H + node * 144;
        if (!build_h3(c3.H, bf2, a.mu, 0.0, c3.Hinv)) {
            a.status[node] = ST_SINGULAR;
            return false;
        }
        c3.norm_init = -1.0;
        c3.last_dn = 1e300;
        c3.dn_prev = -1.0;
        c3.best_dn = 1e300;
        c3.zncc = nan("");
        c3.stall = 0;
        return true;
    }
}

template <int NDOF>
__device__ __noinline__ void node_end(const IcgnArgs& a, int64_t node, const Ctl12& c12, const Ctl3& c3, int it, int st, double zc) {
    if (NDOF == 12) {
        for (int k = 0; k < 12; ++k) a.P_out[node * 12 + k] = c12.P[k];
    } else {
        for (int k = 0; k < 3; ++k) a.P_out[node * 3 + k] = c3.P[9 + k];
    }
    a.n_iter[node] = it;
    a.status[node] = (int8_t)st;
    a.zncc[node] = zc;
}

// ----------------------------------------------------------------------------- sampling helpers
// Sampling box of subset planes [zc0, zc1) under warp P: voxel bounds of every tap plus one voxel of
// margin for FP32 rounding, clamped to the volume.  Also reports whether all 8 corners lie in the
// admissible domain (then no voxel can leave it: the warp is affine).
struct Box {
    int x0, y0, z0, bx, by, bz;
    bool corners_in;
};

__device__ __noinline__ Box warp_box(const IcgnArgs& a, const Shape& sh, const double* P, int64_t xc, int64_t yc, int64_t zc, int zc0,
                                     int zc1, int mode) {
    const double a00 = 1.0 + P[0], a01 = P[1], a02 = P[2], a10 = P[3], a11 = 1.0 + P[4], a12 = P[5], a20 = P[6], a21 = P[7],
                 a22 = 1.0 + P[8];
    const double tx = (double)xc + P[9], ty = (double)yc + P[10], tz = (double)zc + P[11];
    const double Xs[2] = {(double)-sh.hx, (double)(-sh.hx + (sh.nX - 1) * a.stride)};
    const double Ys[2] = {(double)-sh.hy, (double)(-sh.hy + (sh.nY - 1) * a.stride)};
    const double Zs[2] = {(double)(-sh.hz + zc0 * a.stride), (double)(-sh.hz + (zc1 - 1) * a.stride)};
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    bool in = true;
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j)
            for (int k = 0; k < 2; ++k) {
                const double X = Xs[i], Y = Ys[j], Z = Zs[k];
                const double p[3] = {a00 * X + a01 * Y + a02 * Z + tx, a10 * X + a11 * Y + a12 * Z + ty,
                                     a20 * X + a21 * Y + a22 * Z + tz};
                for (int d = 0; d < 3; ++d) {
                    lo[d] = fmin(lo[d], p[d]);
                    hi[d] = fmax(hi[d], p[d]);
                }
                in = in && margin_ok(p[2], p[1], p[0], a.nz, a.ny, a.nx);
            }
    const int tl = mode == 0 ? 0 : 1, th = mode == 0 ? 1 : 2;  // taps below / above floor(x)
    const int n[3] = {a.nx, a.ny, a.nz};
    int b0[3], b1[3];
    for (int d = 0; d < 3; ++d) {
        // finite guard: a NaN warp never reaches here (checked at node start / after compose)
        double l = fmax(fmin(lo[d], 1e9), -1e9), h = fmax(fmin(hi[d], 1e9), -1e9);
        long long f0 = (long long)floor(l) - tl - 1, f1 = (long long)floor(h) + th + 1;
        // both ends inside the volume, so the staged rows are always readable
        f0 = f0 < 0 ? 0 : (f0 > n[d] - 1 ? n[d] - 1 : f0);
        f1 = f1 > n[d] - 1 ? n[d] - 1 : (f1 < 0 ? 0 : f1);
        if (f1 < f0) f1 = f0;
        b0[d] = (int)f0;
        b1[d] = (int)f1;
    }
    Box bx;
    bx.x0 = b0[0];
    bx.y0 = b0[1];
    bx.z0 = b0[2];
    bx.bx = b1[0] - b0[0] + 1;
    bx.by = b1[1] - b0[1] + 1;
    bx.bz = b1[2] - b0[2] + 1;
    bx.corners_in = in;
    return bx;
}

// Interpolate at a position relative to a brick origin (pitch bx, plane bxy, extent ex/ey/ez).
// Indices are clamped into the brick so no read can leave it.
template <int MODE>
__device__ __forceinline__ float sample_rel(const float* __restrict__ base, int bx, int bxy, int ex, int ey, int ez, float xr,
                                            float yr, float zr) {
    int ix = __float2int_rd(xr), iy = __float2int_rd(yr), iz = __float2int_rd(zr);
    const float fx = xr - (float)ix, fy = yr - (float)iy, fz = zr - (float)iz;
    if (MODE == 0) {
        ix = min(max(ix, 0), ex - 2);
        iy = min(max(iy, 0), ey - 2);
        iz = min(max(iz, 0), ez - 2);
        return sample_brick<0>(base, bx, bxy, ix, iy, iz, fx, fy, fz);
    }
    ix = min(max(ix, 1), ex - 3);
    iy = min(max(iy, 1), ey - 3);
    iz = min(max(iz, 1), ez - 3);
    return sample_brick<MODE>(base, bx, bxy, ix, iy, iz, fx, fy, fz);
}

// Per-thread FP32 moments of the single-pass accumulation.
template <int NDOF>
struct Acc {
    static constexpr int NB = NDOF == 12 ? 12 : 3;
    float Sg, Sgg, Sf, Sff, Sfg;
    float SD[NB], SDf[NB], SDg[NB];
    int n, nref, oob;
    __device__ void zero() {
        Sg = Sgg = Sf = Sff = Sfg = 0.0f;
#pragma unroll
        for (int k = 0; k < NB; ++k) SD[k] = SDf[k] = SDg[k] = 0.0f;
        n = nref = oob = 0;
    }
    __device__ __forceinline__ void add(float fs, float gs, float q0, float q1, float q2, float X, float Y, float Z) {
        Sg += gs;
        Sgg += gs * gs;
        Sf += fs;
        Sff += fs * fs;
        Sfg += fs * gs;
        const float q[3] = {q0, q1, q2};
        if (NDOF == 12) {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const float qf = q[i] * fs, qg = q[i] * gs;
                SD[3 * i] += q[i] * X;
                SD[3 * i + 1] += q[i] * Y;
                SD[3 * i + 2] += q[i] * Z;
                SD[9 + i] += q[i];
                SDf[3 * i] += qf * X;
                SDf[3 * i + 1] += qf * Y;
                SDf[3 * i + 2] += qf * Z;
                SDf[9 + i] += qf;
                SDg[3 * i] += qg * X;
                SDg[3 * i + 1] += qg * Y;
                SDg[3 * i + 2] += qg * Z;
                SDg[9 + i] += qg;
            }
        } else {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                SD[i] += q[i];
                SDf[i] += q[i] * fs;
                SDg[i] += q[i] * gs;
            }
        }
        ++n;
    }
    // The same sums split by what they depend on: REF the reference-frame sums (Σ f, Σ f², Σ SD, Σ SD·f, fixed
    // for a node), WARP the sums over the sampled g and the valid count.  Each field is updated by the same
    // expression as in add(), so a sweep of either part gives the FP32 partials add() would give.
    template <bool REF, bool WARP>
    __device__ __forceinline__ void add_part(float fs, float gs, float q0, float q1, float q2, float X, float Y, float Z) {
        if (WARP) {
            Sg += gs;
            Sgg += gs * gs;
        }
        if (REF) {
            Sf += fs;
            Sff += fs * fs;
        }
        if (WARP) Sfg += fs * gs;
        const float q[3] = {q0, q1, q2};
        if (NDOF == 12) {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                if (REF) {
                    const float qf = q[i] * fs;
                    SD[3 * i] += q[i] * X;
                    SD[3 * i + 1] += q[i] * Y;
                    SD[3 * i + 2] += q[i] * Z;
                    SD[9 + i] += q[i];
                    SDf[3 * i] += qf * X;
                    SDf[3 * i + 1] += qf * Y;
                    SDf[3 * i + 2] += qf * Z;
                    SDf[9 + i] += qf;
                }
                if (WARP) {
                    const float qg = q[i] * gs;
                    SDg[3 * i] += qg * X;
                    SDg[3 * i + 1] += qg * Y;
                    SDg[3 * i + 2] += qg * Z;
                    SDg[9 + i] += qg;
                }
            }
        } else {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                if (REF) {
                    SD[i] += q[i];
                    SDf[i] += q[i] * fs;
                }
                if (WARP) SDg[i] += q[i] * gs;
            }
        }
        if (WARP) ++n;
    }
};

template <int K>
struct SweepKind {
    static constexpr int value = K;
};

// Cross-warp FP64 totals in a fixed order (deterministic), thread 0 only.
__device__ __noinline__ void total_moments(double (*red)[48], int (*redi)[3], int nw, int nb, Moments& out) {
    double t[5 + 3 * 12];
    for (int i = 0; i < 5 + 3 * nb; ++i) {
        double s = 0.0;
        for (int w = 0; w < nw; ++w) s += red[w][i];
        t[i] = s;
    }
    int64_t nn = 0, nrr = 0;
    int oo = 0;
    for (int w = 0; w < nw; ++w) {
        nn += redi[w][0];
        nrr += redi[w][1];
        oo |= redi[w][2];
    }
    out.n = nn;
    out.nref = nrr;
    out.oob = oo;
    out.Sg = t[0];
    out.Sgg = t[1];
    out.Sf = t[2];
    out.Sff = t[3];
    out.Sfg = t[4];
    for (int k = 0; k < nb; ++k) {
        out.SD[k] = t[5 + k];
        out.SDf[k] = t[5 + nb + k];
        out.SDg[k] = t[5 + 2 * nb + k];
    }
}

// Reduce the per-thread moments into FP64 totals in shared memory (all threads call; totals valid
// after the final __syncthreads in thread 0's view and everyone else's).
template <int NDOF, int THREADS>
__device__ void reduce_moments(Acc<NDOF>& acc, double (*red)[48], int (*redi)[3], Moments& out) {
    constexpr int NB = Acc<NDOF>::NB;
    constexpr int NW = THREADS / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float v[5 + 3 * NB];
    v[0] = acc.Sg;
    v[1] = acc.Sgg;
    v[2] = acc.Sf;
    v[3] = acc.Sff;
    v[4] = acc.Sfg;
#pragma unroll
    for (int k = 0; k < NB; ++k) {
        v[5 + k] = acc.SD[k];
        v[5 + NB + k] = acc.SDf[k];
        v[5 + 2 * NB + k] = acc.SDg[k];
    }
#pragma unroll
    for (int i = 0; i < 5 + 3 * NB; ++i) {
        const float s = warp_sum(v[i]);
        if (lane == 0) red[warp][i] = (double)s;
    }
    const int n = warp_sum_i(acc.n), nr = warp_sum_i(acc.nref);
    const int oob = __any_sync(0xffffffffu, acc.oob != 0) ? 1 : 0;
    if (lane == 0) {
        redi[warp][0] = n;
        redi[warp][1] = nr;
        redi[warp][2] = oob;
    }
    __syncthreads();
    if (threadIdx.x == 0) total_moments(red, redi, NW, NB, out);
}

// ----------------------------------------------------------------------------- batched persistent kernel
struct SharedCtl {
    double P[12];
    float A[9];
    float t[3];  // translation relative to the brick origin
    int box[6];  // x0 y0 z0 bx by bz
    int zc1;
    int use_brick;
    int slow;
    int state;  // 0: iterate, 1: node finished
    int64_t node;
    float cf, cg;
};

template <int MODE, bool STORED, int NDOF, int THREADS>
__global__ void __launch_bounds__(THREADS, 512 / THREADS) icgn_batched_kernel(IcgnArgs a) {
    extern __shared__ __align__(16) float brick[];
    __shared__ SharedCtl sc;
    __shared__ double red[THREADS / 32][48];
    __shared__ int redi[THREADS / 32][3];
    __shared__ Moments mom;
    __shared__ double Ls[144];

    const int tid = threadIdx.x;
    const int64_t sxy = (int64_t)a.nx * a.ny;
    const int nXY = a.nX * a.nY;
    Ctl12 c12;  // live in thread 0 only
    Ctl3 c3;

    for (;;) {
        __syncthreads();  // every thread has finished reading the previous node's control block
        if (tid == 0) {
            const int q = atomicAdd(a.counter, 1);
            sc.node = queue_node(a, q);
            sc.state = 1;
            if (sc.node >= 0) {
                const int64_t node = sc.node;
                if (node_begin<NDOF>(a, node, c12, c3, Shape{a.hx, a.hy, a.hz, a.nX, a.nY, a.nZ}, true)) {
                    sc.state = 0;
                    const double* P = NDOF == 12 ? c12.P : c3.P;
                    for (int k = 0; k < 12; ++k) sc.P[k] = P[k];
                    sc.cf = (float)a.meanf[node];
                    sc.cg = sc.cf;
                }
            }
        }
        __syncthreads();
        const int64_t node = sc.node;
        if (node == -1) break;  // the queue is empty (-2: a skipped order entry)
        if (sc.state != 0) continue;
        if (NDOF == 12) {
            for (int i = tid; i < 144; i += THREADS) Ls[i] = a.L[node * 144 + i];
        }
        const int64_t xc = a.coords[3 * node], yc = a.coords[3 * node + 1], zcn = a.coords[3 * node + 2];
        const int64_t srow = a.split_index ? a.split_index[node] : -1;
        const uint8_t* keep = srow >= 0 ? a.split_keep + srow * a.keep_bytes : nullptr;
        // a subset that crosses a volume face (only possible for nodes the caller marks valid against the
        // precompute's verdict) reads no voxel outside the volume: those voxels are skipped
        const bool inside = xc - a.hx >= 0 && xc + a.hx < a.nx && yc - a.hy >= 0 && yc + a.hy < a.ny && zcn - a.hz >= 0 &&
                            zcn + a.hz < a.nz;
        __syncthreads();

        int it = 1;
        for (; it <= a.max_iter; ++it) {
            Acc<NDOF> acc;
            acc.zero();
            int zc0 = 0;
            while (zc0 < a.nZ) {
                if (tid == 0) {
                    // largest chunk of subset planes whose box fits in the brick
                    int lo = zc0 + 1, hi = a.nZ, best = zc0 + 1;
                    const Shape sh0{a.hx, a.hy, a.hz, a.nX, a.nY, a.nZ};
                    Box bb = warp_box(a, sh0, sc.P, xc, yc, zcn, zc0, hi, MODE);
                    bool fits = (long long)bb.bx * bb.by * bb.bz <= a.brick_cap;
                    if (fits) {
                        best = hi;
                    } else {
                        while (lo <= hi) {
                            const int mid = (lo + hi) / 2;
                            Box t = warp_box(a, sh0, sc.P, xc, yc, zcn, zc0, mid, MODE);
                            if ((long long)t.bx * t.by * t.bz <= a.brick_cap) {
                                best = mid;
                                bb = t;
                                lo = mid + 1;
                            } else {
                                hi = mid - 1;
                            }
                        }
                        bb = warp_box(a, sh0, sc.P, xc, yc, zcn, zc0, best, MODE);
                    }
                    const bool use = (long long)bb.bx * bb.by * bb.bz <= a.brick_cap;
                    sc.use_brick = use ? 1 : 0;
                    sc.zc1 = best;
                    sc.slow = bb.corners_in ? 0 : 1;
                    if (!use) {  // a single plane does not fit: sample the global volume directly
                        bb.x0 = 0;
                        bb.y0 = 0;
                        bb.z0 = 0;
                        bb.bx = a.nx;
                        bb.by = a.ny;
                        bb.bz = a.nz;
                    }
                    sc.box[0] = bb.x0;
                    sc.box[1] = bb.y0;
                    sc.box[2] = bb.z0;
                    sc.box[3] = bb.bx;
                    sc.box[4] = bb.by;
                    sc.box[5] = bb.bz;
                    const double* P = sc.P;
                    sc.A[0] = (float)(1.0 + P[0]);
                    sc.A[1] = (float)P[1];
                    sc.A[2] = (float)P[2];
                    sc.A[3] = (float)P[3];
                    sc.A[4] = (float)(1.0 + P[4]);
                    sc.A[5] = (float)P[5];
                    sc.A[6] = (float)P[6];
                    sc.A[7] = (float)P[7];
                    sc.A[8] = (float)(1.0 + P[8]);
                    sc.t[0] = (float)(((double)xc - bb.x0) + P[9]);
                    sc.t[1] = (float)(((double)yc - bb.y0) + P[10]);
                    sc.t[2] = (float)(((double)zcn - bb.z0) + P[11]);
                }
                __syncthreads();
                const int zc1 = sc.zc1;
                const int bx0 = sc.box[0], by0 = sc.box[1], bz0 = sc.box[2];
                const int BX = sc.box[3], BY = sc.box[4], BZ = sc.box[5];
                const bool use_brick = sc.use_brick != 0;
                const bool slow = sc.slow != 0;
                if (use_brick) {
                    // coalesced row loads of the box into shared memory
                    const int rows = BY * BZ;
                    const int warp = tid >> 5, lane = tid & 31;
                    for (int r = warp; r < rows; r += THREADS / 32) {
                        const int ry = r % BY, rz = r / BY;
                        const float* src = a.g + (int64_t)(bz0 + rz) * sxy + (int64_t)(by0 + ry) * a.nx + bx0;
                        float* dst = brick + r * BX;
                        for (int x = lane; x < BX; x += 32) dst[x] = __ldg(src + x);
                    }
                    __syncthreads();
                }
                const float* base = use_brick ? brick : a.g;
                const int pitch = use_brick ? BX : a.nx;
                const int plane = use_brick ? BX * BY : (int)sxy;
                const float A0 = sc.A[0], A1 = sc.A[1], A2 = sc.A[2], A3 = sc.A[3], A4 = sc.A[4], A5 = sc.A[5], A6 = sc.A[6],
                            A7 = sc.A[7], A8 = sc.A[8];
                const float T0 = sc.t[0], T1 = sc.t[1], T2 = sc.t[2];
                const float cf = sc.cf, cg = sc.cg;
                // voxels of planes [zc0, zc1) in sampling order
                const int v0 = zc0 * nXY, v1 = zc1 * nXY;
                for (int v = v0 + tid; v < v1; v += THREADS) {
                    const int iz = v / nXY, rem = v - iz * nXY;
                    const int iy = rem / a.nX, ix = rem - iy * a.nX;
                    const int dx = -a.hx + ix * a.stride, dy = -a.hy + iy * a.stride, dz = -a.hz + iz * a.stride;
                    const int64_t xx = xc + dx, yy = yc + dy, zz = zcn + dz;
                    bool k;
                    if (keep || !inside) {
                        k = xx >= 0 && xx < a.nx && yy >= 0 && yy < a.ny && zz >= 0 && zz < a.nz;
                        if (k) k = keep ? kept_bit(keep, v) : ((a.mask == nullptr) || __ldg(a.mask + zz * sxy + yy * a.nx + xx) != 0);
                    } else {
                        k = (a.mask == nullptr) || __ldg(a.mask + zz * sxy + yy * a.nx + xx) != 0;
                    }
                    if (!k) continue;
                    acc.nref += 1;
                    const float X = (float)dx, Y = (float)dy, Z = (float)dz;
                    if (slow) {
                        const double* P = sc.P;
                        const double xw = (1.0 + P[0]) * dx + P[1] * dy + P[2] * dz + ((double)xc + P[9]);
                        const double yw = P[3] * dx + (1.0 + P[4]) * dy + P[5] * dz + ((double)yc + P[10]);
                        const double zw = P[6] * dx + P[7] * dy + (1.0 + P[8]) * dz + ((double)zcn + P[11]);
                        if (!margin_ok(zw, yw, xw, a.nz, a.ny, a.nx)) {
                            acc.oob = 1;
                            continue;
                        }
                    }
                    const float xr = A0 * X + A1 * Y + A2 * Z + T0;
                    const float yr = A3 * X + A4 * Y + A5 * Z + T1;
                    const float zr = A6 * X + A7 * Y + A8 * Z + T2;
                    const float gv = sample_rel<MODE>(base, pitch, plane, BX, BY, BZ, xr, yr, zr);
                    if (gv != gv) continue;  // NaN: masked out in the deformed frame
                    const int64_t o = zz * sxy + yy * a.nx + xx;
                    const float fv = __ldg(a.f + o);
                    float q0, q1, q2;
                    if (STORED) {
                        q0 = __ldg(a.gx + o);
                        q1 = __ldg(a.gy + o);
                        q2 = __ldg(a.gz + o);
                    } else {
                        grad_otf(a.f, a.nz, a.ny, a.nx, (int)zz, (int)yy, (int)xx, q0, q1, q2);
                    }
                    acc.add(fv - cf, gv - cg, q0, q1, q2, X, Y, Z);
                }
                zc0 = zc1;
                __syncthreads();  // the next chunk overwrites the brick
            }
            reduce_moments<NDOF, THREADS>(acc, red, redi, mom);
            if (tid == 0) {
                double b[12], bf, bg, s_cc;
                int64_t nv;
                const int st0 = finish_moments(mom, sc.cf, sc.cg, NDOF == 12 ? 12 : 3, b, bf, bg, s_cc, nv);
                int st;
                double zc = nan("");
                if (st0 != 0) {
                    st = st0;  // OOB / invalid subset: zncc stays NaN
                } else if (NDOF == 12) {
                    st = control12(c12, b, bf, bg, s_cc, nv, Ls, a.H ? a.H + node * 144 : nullptr, a.pattern, a.noise_gain, a.tol,
                                   a.dp_tol, a.patience, a.predictive, zc);
                } else {
                    st = control3(c3, b, bf, bg, s_cc, nv, a.mu, a.noise_gain, a.tol, a.dp_tol, a.patience, a.predictive, zc);
                }
                if (st >= 0) {
                    node_end<NDOF>(a, node, c12, c3, it, st, zc);
                    sc.state = 1;
                } else {
                    const double* P = NDOF == 12 ? c12.P : c3.P;
                    for (int k = 0; k < 12; ++k) sc.P[k] = P[k];
                    sc.cg = (float)((double)sc.cg + mom.Sg / (double)mom.n);  // centre g on this iteration's mean
                    if (it == a.max_iter) {
                        const double zc_last = NDOF == 12 ? c12.zncc : c3.zncc;
                        node_end<NDOF>(a, node, c12, c3, a.max_iter, ST_MAX_ITER, zc_last);
                        sc.state = 1;
                    }
                }
            }
            __syncthreads();
            if (sc.state != 0) break;
        }
    }
}

// ----------------------------------------------------------------------------- lean persistent kernel
// NW warps per node and no shared brick: the deformed volume is sampled through L1 at positions taken
// relative to the node centre, so a CTA holds only its control block and 16 (12-DOF, 128 registers a
// thread) or 24 (3-DOF, 80) warps run per SM.  While thread 0 of one CTA runs the FP64 control step, the
// other CTAs of the SM keep the pipes busy.  Voxel indices advance incrementally (no divisions in the loop);
// the per-thread FP32 moments are reduced across the warp in FP64.  The reference-frame sums are swept
// only while a node has none stored (its first iteration, or after a NaN sample).
struct LeanCtl {
    double P[12];
    float A[9];
    float t[3];
    int slow;
    int state;
    int use_ref;  // the node's reference-frame sums are taken from ref_tot (set by its first complete sweep)
    int redo;     // this iteration met a NaN sample under use_ref: sweep it again with every sum
    int64_t node;
    float cf, cg;
};

template <int MODE, bool STORED, int NDOF, int NW, bool UNEVEN, bool TMA>
__device__ __forceinline__ void lean_body(const IcgnArgs& a, const CUtensorMap* tmap) {
    constexpr int T = NW * 32;
    constexpr int NB = Acc<NDOF>::NB;
    constexpr int NV = 5 + 3 * NB;
    constexpr int NR = 2 + 2 * NB;
    __shared__ LeanCtl sc;
    __shared__ double red[NW][NV];
    __shared__ int redi[NW][3];
    __shared__ double ref_tot[NR];  // Σ f, Σ f², Σ SD, Σ SD·f of the node's kept voxels (FP64 totals, thread 0)
    __shared__ double Ls[NDOF == 12 ? 144 : 1];  // the node's Cholesky factor: thread 0 solves with it every iteration
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t sxy = (int64_t)a.nx * a.ny;
    const int lo = MODE == 0 ? 0 : 1, hx_ = MODE == 0 ? a.nx - 2 : a.nx - 3, hy_ = MODE == 0 ? a.ny - 2 : a.ny - 3,
              hz_ = MODE == 0 ? a.nz - 2 : a.nz - 3;
    Ctl12 c12;  // live in thread 0 only
    Ctl3 c3;
    // staged form: two shared buffers, their mbarriers and the origin of the box each holds
    extern __shared__ __align__(128) unsigned char tsm_raw[];
    float* tbuf = reinterpret_cast<float*>(tsm_raw + ((128u - (smem_u32(tsm_raw) & 127u)) & 127u));  // 128-byte aligned
    __shared__ __align__(8) uint64_t t_mb[2];
    __shared__ int t_org[2][3];
    __shared__ int t_fit[2];
    __shared__ int t_dead;  // a wait gave up: no more staged copies in this CTA
    uint32_t t_phase = 0;   // bit b: parity of buffer b's next completion (identical in every thread)
    if (TMA) {
        if (tid == 0) {
            mbar_init(smem_u32(&t_mb[0]), 1);
            mbar_init(smem_u32(&t_mb[1]), 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            t_dead = 0;
        }
        __syncthreads();
    }

    for (;;) {
        __syncthreads();  // every thread has finished reading the previous node's control block
        if (tid == 0) {
            const int q = atomicAdd(a.counter, 1);
            sc.node = queue_node(a, q);
            sc.state = 1;
            bool shape_ok = true;
            const Shape sh0 = (UNEVEN && sc.node >= 0) ? node_shape(a, sc.node, shape_ok) : Shape{a.hx, a.hy, a.hz, a.nX, a.nY, a.nZ};
            if (sc.node >= 0 && node_begin<NDOF>(a, sc.node, c12, c3, sh0, shape_ok)) {
                sc.state = 0;
                const double* P = NDOF == 12 ? c12.P : c3.P;
                for (int k = 0; k < 12; ++k) sc.P[k] = P[k];
                sc.cf = (float)a.meanf[sc.node];
                sc.cg = sc.cf;
            }
        }
        __syncthreads();
        const int64_t node = sc.node;
        if (node == -1) break;  // the queue is empty (-2: a skipped order entry)
        if (sc.state != 0) continue;
        // one shape per call: the kernel parameters themselves; uneven: the node's (node_begin rejected a bad one)
        bool shape_ok = true;
        const Shape sh = UNEVEN ? node_shape(a, node, shape_ok) : Shape{a.hx, a.hy, a.hz, a.nX, a.nY, a.nZ};
        // sweep order: tiles of `by` subset rows, each swept plane by plane and row by row (by = nY: C order); the
        // last tile's rows past the subset are padding slots, skipped
        const int by = sweep_rows(sh.nY, a.sweep_rows);
        const int nXB = sh.nX * by;
        const int tileV = nXB * sh.nZ;
        const int Sp = tileV * ((sh.nY + by - 1) / by);
        const int sx_ = T % sh.nX, sb_ = (T / sh.nX) % by, sz_ = (T / nXB) % sh.nZ, st_ = T / tileV;  // index step of T slots
        const int tix = tid % sh.nX, tib = (tid / sh.nX) % by, tiz = (tid / nXB) % sh.nZ, tit = tid / tileV;
        const int64_t xc = a.coords[3 * node], yc = a.coords[3 * node + 1], zcn = a.coords[3 * node + 2];
        const int64_t srow = a.split_index ? a.split_index[node] : -1;
        const uint8_t* keep = srow >= 0 ? a.split_keep + srow * a.keep_bytes : nullptr;
        const bool inside = xc - sh.hx >= 0 && xc + sh.hx < a.nx && yc - sh.hy >= 0 && yc + sh.hy < a.ny && zcn - sh.hz >= 0 &&
                            zcn + sh.hz < a.nz;
        const int xci = (int)xc, yci = (int)yc, zci = (int)zcn;
        const float cf = sc.cf;

        // One voxel of a sweep (subset indices vx, vy, vz).  KIND 1: the sums over the sampled g and the counts; KIND 2:
        // every sum.  `smp(gx, gy, gz, fx, fy, fz)` samples g at the clamped tap origin (gx, gy, gz).
        auto visit = [&](auto kind, Acc<NDOF>& acc, bool slow, int vx, int vy, int vz, float A0, float A1, float A2, float A3,
                         float A4, float A5, float A6, float A7, float A8, float T0, float T1, float T2, float cg, auto&& smp) {
            constexpr int KIND = decltype(kind)::value;
            const int dx = -sh.hx + vx * a.stride, dy = -sh.hy + vy * a.stride, dz = -sh.hz + vz * a.stride;
            const int xx = xci + dx, yy = yci + dy, zz = zci + dz;
            bool k;
            auto in_mask = [&]() {
                return a.idx32 ? __ldg(a.mask + (zz * (int)sxy + yy * a.nx + xx)) != 0
                               : __ldg(a.mask + zz * sxy + (int64_t)yy * a.nx + xx) != 0;
            };
            if (keep || !inside) {
                k = xx >= 0 && xx < a.nx && yy >= 0 && yy < a.ny && zz >= 0 && zz < a.nz;
                if (k) k = keep ? kept_bit(keep, (vz * sh.nY + vy) * sh.nX + vx) : ((a.mask == nullptr) || in_mask());
            } else {
                k = (a.mask == nullptr) || in_mask();
            }
            if (!k) return;
            acc.nref += 1;
            const float X = (float)dx, Y = (float)dy, Z = (float)dz;
            if (slow) {
                const double* P = sc.P;
                const double xw = (1.0 + P[0]) * dx + P[1] * dy + P[2] * dz + ((double)xc + P[9]);
                const double yw = P[3] * dx + (1.0 + P[4]) * dy + P[5] * dz + ((double)yc + P[10]);
                const double zw = P[6] * dx + P[7] * dy + (1.0 + P[8]) * dz + ((double)zcn + P[11]);
                if (!margin_ok(zw, yw, xw, a.nz, a.ny, a.nx)) {
                    acc.oob = 1;
                    return;
                }
            }
            // reference-frame reads first: their latency overlaps the interpolation
            float fv, q0, q1, q2;
            auto ref_reads = [&](auto o) {
                fv = __ldg(a.f + o);
                if (STORED) {
                    q0 = __ldg(a.gx + o);
                    q1 = __ldg(a.gy + o);
                    q2 = __ldg(a.gz + o);
                } else {
                    grad_otf(a.f, a.nz, a.ny, a.nx, zz, yy, xx, q0, q1, q2);
                }
            };
            if (a.idx32)
                ref_reads(zz * (int)sxy + yy * a.nx + xx);
            else
                ref_reads(zz * sxy + (int64_t)yy * a.nx + xx);
            const float xr = A0 * X + A1 * Y + A2 * Z + T0;
            const float yr = A3 * X + A4 * Y + A5 * Z + T1;
            const float zr = A6 * X + A7 * Y + A8 * Z + T2;
            const float fxf = floorf(xr), fyf = floorf(yr), fzf = floorf(zr);
            const int gx_ = min(max(xci + (int)fxf, lo), hx_), gy_ = min(max(yci + (int)fyf, lo), hy_),
                      gz_ = min(max(zci + (int)fzf, lo), hz_);
            const float gv = smp(gx_, gy_, gz_, xr - fxf, yr - fyf, zr - fzf);
            if (gv != gv) return;  // NaN: masked out in the deformed frame
            if (KIND == 1)
                acc.template add_part<false, true>(fv - cf, gv - cg, q0, q1, q2, X, Y, Z);
            else
                acc.add(fv - cf, gv - cg, q0, q1, q2, X, Y, Z);
        };
        // sampling g in global memory: the overlapping-quad copy when there is one, else g itself
        auto smp_global = [&](int gx_, int gy_, int gz_, float fx, float fy, float fz) {
            if (MODE != 0 && a.g4)
                return a.idx32 ? sample_quad<MODE == 0 ? 1 : MODE, true>(a.g4, a.nx, (int)sxy, gx_, gy_, gz_, fx, fy, fz)
                               : sample_quad<MODE == 0 ? 1 : MODE, false>(a.g4, a.nx, (int)sxy, gx_, gy_, gz_, fx, fy, fz);
            return sample_brick<MODE>(a.g, a.nx, (int)sxy, gx_, gy_, gz_, fx, fy, fz);
        };
        // One sweep over the node's subset.  Both kinds visit the same voxels in the same per-thread order, so the
        // partials of a field do not depend on the kind that formed them.
        auto sweep = [&](auto kind, Acc<NDOF>& acc, bool slow, float A0, float A1, float A2, float A3, float A4, float A5,
                         float A6, float A7, float A8, float T0, float T1, float T2, float cg) {
            acc.zero();
            if constexpr (!TMA) {
                int ix = tix, ib = tib, iz = tiz, itl = tit;
                for (int v = tid; v < Sp; v += T) {
                    const int vx = ix, vy = itl * by + ib, vz = iz;
                    ix += sx_;
                    ib += sb_;
                    iz += sz_;
                    itl += st_;
                    if (ix >= sh.nX) {
                        ix -= sh.nX;
                        ++ib;
                    }
                    if (ib >= by) {
                        ib -= by;
                        ++iz;
                    }
                    if (iz >= sh.nZ) {
                        iz -= sh.nZ;
                        ++itl;
                    }
                    if (vy >= sh.nY) continue;  // a padding row of the last tile
                    visit(kind, acc, slow, vx, vy, vz, A0, A1, A2, A3, A4, A5, A6, A7, A8, T0, T1, T2, cg, smp_global);
                }
            } else {
                // chunks: tile t of `by` rows x sample planes [zc TMA_KZ, +TMA_KZ), in tile-major order
                const int ntile = (sh.nY + by - 1) / by, nzc = (sh.nZ + TMA_KZ - 1) / TMA_KZ, nch = ntile * nzc;
                // thread 0: the box of chunk ci's taps (corner positions, floors, taps -1..+2 and one voxel of margin
                // for FP32 rounding), its copy into buffer b when it fits
                auto issue = [&](int ci, int b) {
                    const int t = ci / nzc, zc = ci - t * nzc;
                    const int y0 = t * by, y1 = min(y0 + by, sh.nY) - 1, z0 = zc * TMA_KZ, z1 = min(z0 + TMA_KZ, sh.nZ) - 1;
                    const float cx[2] = {(float)(-sh.hx), (float)(-sh.hx + (sh.nX - 1) * a.stride)};
                    const float cy[2] = {(float)(-sh.hy + y0 * a.stride), (float)(-sh.hy + y1 * a.stride)};
                    const float cz[2] = {(float)(-sh.hz + z0 * a.stride), (float)(-sh.hz + z1 * a.stride)};
                    float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
#pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        const float X = cx[c & 1], Y = cy[(c >> 1) & 1], Z = cz[c >> 2];
                        const float p3[3] = {A0 * X + A1 * Y + A2 * Z + T0, A3 * X + A4 * Y + A5 * Z + T1, A6 * X + A7 * Y + A8 * Z + T2};
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            mn[d] = fminf(mn[d], p3[d]);
                            mx[d] = fmaxf(mx[d], p3[d]);
                        }
                    }
                    const int cc[3] = {xci, yci, zci};
                    const int ext[3] = {a.nx, a.ny, a.nz};
                    int o[3], e[3];
                    bool fit = t_dead == 0;
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const float lo_f = fmaxf(floorf(mn[d]), -(float)ext[d]), hi_f = fminf(floorf(mx[d]), (float)ext[d]);
                        o[d] = cc[d] + (int)lo_f - 2;
                        e[d] = cc[d] + (int)hi_f + 3 - o[d] + 1;
                    }
                    const int ox = o[0] >= 0 ? (o[0] & ~3) : -((-o[0] + 3) & ~3);  // 16-byte aligned x origin (rounded down)
                    fit = fit && (o[0] + e[0] - ox <= TMA_BX) && e[1] <= TMA_BY && e[2] <= TMA_BZ;
                    t_org[b][0] = ox;
                    t_org[b][1] = o[1];
                    t_org[b][2] = o[2];
                    t_fit[b] = fit ? 1 : 0;
                    if (fit) {
                        const uint32_t mb = smem_u32(&t_mb[b]);
                        mbar_expect_tx(mb, TMA_BOX_BYTES);
                        tma_load_3d(smem_u32(tbuf + b * TMA_BOX), tmap, ox, o[1], o[2], mb);
                    }
                };
                if (tid == 0) {
                    issue(0, 0);
                    if (nch > 1) issue(1, 1);
                }
                __syncthreads();
                for (int ci = 0; ci < nch; ++ci) {
                    const int b = ci & 1;
                    bool fit = t_fit[b] != 0;
                    if (fit) {
                        const bool ok = mbar_wait(smem_u32(&t_mb[b]), (t_phase >> b) & 1u);
                        t_phase ^= 1u << b;
                        if (!ok) {  // never expected: the copy did not complete in time; sample from global memory
                            if (a.err) atomicExch(a.err, 1);
                            t_dead = 1;
                            fit = false;
                        }
                    }
                    const int t = ci / nzc, zc = ci - t * nzc;
                    const int y0 = t * by, nyc = min(by, sh.nY - y0), z0 = zc * TMA_KZ, nzk = min(TMA_KZ, sh.nZ - z0);
                    const int ox = t_org[b][0], oy = t_org[b][1], oz = t_org[b][2];
                    const float* buf = tbuf + b * TMA_BOX;
                    // taps of a staged sample: inside the box, else (a sample the box does not hold) from global memory
                    auto smp_staged = [&](int gx_, int gy_, int gz_, float fx, float fy, float fz) {
                        const int lx = gx_ - ox, ly = gy_ - oy, lz = gz_ - oz;
                        if ((unsigned)(lx - 1) <= (unsigned)(TMA_BX - 4) && (unsigned)(ly - 1) <= (unsigned)(TMA_BY - 4) &&
                            (unsigned)(lz - 1) <= (unsigned)(TMA_BZ - 4))
                            return sample_brick<MODE>(buf, TMA_BX, TMA_BX * TMA_BY, lx, ly, lz, fx, fy, fz);
                        return smp_global(gx_, gy_, gz_, fx, fy, fz);
                    };
                    // the chunk's slots (x fastest, then rows, then planes), advanced incrementally by T
                    const int nxy = sh.nX * nyc, cnt = nxy * nzk;
                    const int stx = T % sh.nX, sty = (T / sh.nX) % nyc, stz = T / nxy;
                    int ix = tid % sh.nX, jy = (tid / sh.nX) % nyc, kz = tid / nxy;
                    for (int sl = tid; sl < cnt; sl += T) {
                        const int vx = ix, vy = y0 + jy, vz = z0 + kz;
                        ix += stx;
                        jy += sty;
                        kz += stz;
                        if (ix >= sh.nX) {
                            ix -= sh.nX;
                            ++jy;
                        }
                        if (jy >= nyc) {
                            jy -= nyc;
                            ++kz;
                        }
                        if (fit)
                            visit(kind, acc, slow, vx, vy, vz, A0, A1, A2, A3, A4, A5, A6, A7, A8, T0, T1, T2, cg, smp_staged);
                        else
                            visit(kind, acc, slow, vx, vy, vz, A0, A1, A2, A3, A4, A5, A6, A7, A8, T0, T1, T2, cg, smp_global);
                    }
                    __syncthreads();  // buffer b is read; its next copy may start
                    if (tid == 0 && ci + 2 < nch) {
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        issue(ci + 2, b);
                    }
                }
            }
        };
        // per-warp FP64 totals of a sweep's partials into red / redi
        auto reduce_warp = [&](const Acc<NDOF>& acc) {
            float vals[NV];
            vals[0] = acc.Sg;
            vals[1] = acc.Sgg;
            vals[2] = acc.Sf;
            vals[3] = acc.Sff;
            vals[4] = acc.Sfg;
#pragma unroll
            for (int k = 0; k < NB; ++k) {
                vals[5 + k] = acc.SD[k];
                vals[5 + NB + k] = acc.SDf[k];
                vals[5 + 2 * NB + k] = acc.SDg[k];
            }
#pragma unroll
            for (int i = 0; i < NV; ++i) {
                double s = (double)vals[i];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                if (lane == 0) red[warp][i] = s;
            }
            const int n = warp_sum_i(acc.n), nr = warp_sum_i(acc.nref);
            const int oob = __any_sync(0xffffffffu, acc.oob != 0) ? 1 : 0;
            if (lane == 0) {
                redi[warp][0] = n;
                redi[warp][1] = nr;
                redi[warp][2] = oob;
            }
        };

        if (tid == 0) sc.use_ref = 0;  // the first iteration sweeps every sum (read after the loop's first barrier)
        if (NDOF == 12)
            for (int i = tid; i < 144; i += T) Ls[i] = a.L[node * 144 + i];  // read after the loop's first barrier

        for (int it = 1; it <= a.max_iter; ++it) {
            if (tid == 0) {
                const Box bb = warp_box(a, sh, sc.P, xc, yc, zcn, 0, sh.nZ, MODE);
                sc.slow = bb.corners_in ? 0 : 1;
                const double* P = sc.P;
                sc.A[0] = (float)(1.0 + P[0]);
                sc.A[1] = (float)P[1];
                sc.A[2] = (float)P[2];
                sc.A[3] = (float)P[3];
                sc.A[4] = (float)(1.0 + P[4]);
                sc.A[5] = (float)P[5];
                sc.A[6] = (float)P[6];
                sc.A[7] = (float)P[7];
                sc.A[8] = (float)(1.0 + P[8]);
                sc.t[0] = (float)P[9];
                sc.t[1] = (float)P[10];
                sc.t[2] = (float)P[11];
            }
            __syncthreads();
            const bool slow = sc.slow != 0;
            const bool use_ref = sc.use_ref != 0;
            {
                Acc<NDOF> acc;
                if (use_ref)
                    sweep(SweepKind<1>{}, acc, slow, sc.A[0], sc.A[1], sc.A[2], sc.A[3], sc.A[4], sc.A[5], sc.A[6], sc.A[7], sc.A[8],
                          sc.t[0], sc.t[1], sc.t[2], sc.cg);
                else
                    sweep(SweepKind<2>{}, acc, slow, sc.A[0], sc.A[1], sc.A[2], sc.A[3], sc.A[4], sc.A[5], sc.A[6], sc.A[7], sc.A[8],
                          sc.t[0], sc.t[1], sc.t[2], sc.cg);
                reduce_warp(acc);
            }
            __syncthreads();
            if (tid == 0) {
                Moments mom;
                double t[NV];
                for (int i = 0; i < NV; ++i) {
                    double s = 0.0;
                    for (int w = 0; w < NW; ++w) s += red[w][i];
                    t[i] = s;
                }
                int64_t nn = 0, nrr = 0;
                int oo = 0;
                for (int w = 0; w < NW; ++w) {
                    nn += redi[w][0];
                    nrr += redi[w][1];
                    oo |= redi[w][2];
                }
                mom.n = nn;
                mom.nref = nrr;
                mom.oob = oo;
                mom.Sg = t[0];
                mom.Sgg = t[1];
                mom.Sf = t[2];
                mom.Sff = t[3];
                mom.Sfg = t[4];
                for (int k = 0; k < NB; ++k) {
                    mom.SD[k] = t[5 + k];
                    mom.SDf[k] = t[5 + NB + k];
                    mom.SDg[k] = t[5 + 2 * NB + k];
                }
                // The reference-frame sums (Σ f, Σ f², Σ SD, Σ SD·f) do not depend on the warp: a full sweep in which
                // every kept voxel entered the sums serves the later iterations whose samples are all finite.  A NaN
                // sample under use_ref left a kept voxel out: that iteration is swept again with every sum.
                const bool redo = use_ref && !oo && nn != nrr;
                sc.redo = redo ? 1 : 0;
                if (redo) {
                    sc.use_ref = 0;
                } else {
                    if (!use_ref && !oo && nn == nrr) {
                        ref_tot[0] = t[2];
                        ref_tot[1] = t[3];
                        for (int k = 0; k < NB; ++k) {
                            ref_tot[2 + k] = t[5 + k];
                            ref_tot[2 + NB + k] = t[5 + NB + k];
                        }
                        sc.use_ref = 1;
                    }
                    if (use_ref) {
                        mom.Sf = ref_tot[0];
                        mom.Sff = ref_tot[1];
                        for (int k = 0; k < NB; ++k) {
                            mom.SD[k] = ref_tot[2 + k];
                            mom.SDf[k] = ref_tot[2 + NB + k];
                        }
                    }
                    double b[12], bf, bg, s_cc;
                    int64_t nv;
                    const int st0 = finish_moments(mom, sc.cf, sc.cg, NB, b, bf, bg, s_cc, nv);
                    int st;
                    double zc = nan("");
                    if (st0 != 0) {
                        st = st0;
                    } else if (NDOF == 12) {
                        st = control12(c12, b, bf, bg, s_cc, nv, Ls, a.H ? a.H + node * 144 : nullptr, a.pattern,
                                       a.noise_gain, a.tol, a.dp_tol, a.patience, a.predictive, zc);
                    } else {
                        st = control3(c3, b, bf, bg, s_cc, nv, a.mu, a.noise_gain, a.tol, a.dp_tol, a.patience, a.predictive, zc);
                    }
                    if (st >= 0) {
                        node_end<NDOF>(a, node, c12, c3, it, st, zc);
                        sc.state = 1;
                    } else {
                        const double* P = NDOF == 12 ? c12.P : c3.P;
                        for (int k = 0; k < 12; ++k) sc.P[k] = P[k];
                        sc.cg = (float)((double)sc.cg + mom.Sg / (double)mom.n);
                        if (it == a.max_iter) {
                            node_end<NDOF>(a, node, c12, c3, a.max_iter, ST_MAX_ITER, NDOF == 12 ? c12.zncc : c3.zncc);
                            sc.state = 1;
                        }
                    }
                }
            }
            __syncthreads();
            if (sc.state != 0) break;
            if (sc.redo) --it;  // the same iteration again, every sum swept (sc.use_ref is now 0)
        }
    }
}

template <int MODE, bool STORED, int NDOF, int NW, bool UNEVEN>
__global__ void __launch_bounds__(NW * 32, (NDOF == 12 ? 16 : 24) / NW) icgn_lean_kernel(IcgnArgs a) {
    lean_body<MODE, STORED, NDOF, NW, UNEVEN, false>(a, nullptr);
}

// The staged form: 4 warps per node, stored gradients, one subset shape, cubic or B-spline sampling from the TMA
// copies of g (two 23 KB buffers per CTA, four CTAs per SM).
template <int MODE, int NDOF>
__global__ void __launch_bounds__(128, 4) icgn_tma_kernel(IcgnArgs a, const __grid_constant__ CUtensorMap tmap) {
    lean_body<MODE, true, NDOF, 4, false, true>(a, &tmap);
}

// ----------------------------------------------------------------------------- plain one-node-per-block kernel
template <int MODE, bool STORED, int NDOF>
__global__ void __launch_bounds__(256) icgn_plain_kernel(IcgnArgs a) {
    constexpr int THREADS = 256;
    constexpr int NB = NDOF == 12 ? 12 : 3;
    __shared__ SharedCtl sc;
    __shared__ double red[THREADS / 32][48];
    __shared__ int redi[THREADS / 32][3];
    __shared__ Moments mom;
    __shared__ double stat[4];  // meanf_d, meang, inv_bf, inv_bg
    __shared__ double Ls[144];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t node = a.node_base + blockIdx.x;
    if (node >= a.n_nodes) return;
    const int64_t sxy = (int64_t)a.nx * a.ny;
    bool shape_ok;
    const Shape sh = node_shape(a, node, shape_ok);
    const int nXY = sh.nX * sh.nY;
    const int S = nXY * sh.nZ;
    float* gbuf = a.gbuf + (int64_t)blockIdx.x * ((int64_t)a.nX * a.nY * a.nZ);  // rows sized by the largest shape
    Ctl12 c12;
    Ctl3 c3;
    if (tid == 0) {
        sc.state = node_begin<NDOF>(a, node, c12, c3, sh, shape_ok) ? 0 : 1;
        if (sc.state == 0) {
            const double* P = NDOF == 12 ? c12.P : c3.P;
            for (int k = 0; k < 12; ++k) sc.P[k] = P[k];
            sc.cf = (float)a.meanf[node];
        }
    }
    __syncthreads();
    if (sc.state != 0) return;
    if (NDOF == 12)
        for (int i = tid; i < 144; i += THREADS) Ls[i] = a.L[node * 144 + i];
    const int64_t xc = a.coords[3 * node], yc = a.coords[3 * node + 1], zcn = a.coords[3 * node + 2];
    const int64_t srow = a.split_index ? a.split_index[node] : -1;
    const uint8_t* keep = srow >= 0 ? a.split_keep + srow * a.keep_bytes : nullptr;
    const bool inside = xc - sh.hx >= 0 && xc + sh.hx < a.nx && yc - sh.hy >= 0 && yc + sh.hy < a.ny && zcn - sh.hz >= 0 &&
                        zcn + sh.hz < a.nz;
    __syncthreads();

    for (int it = 1; it <= a.max_iter; ++it) {
        if (tid == 0) {
            const Box bb = warp_box(a, sh, sc.P, xc, yc, zcn, 0, sh.nZ, MODE);
            sc.slow = bb.corners_in ? 0 : 1;
            const double* P = sc.P;
            sc.A[0] = (float)(1.0 + P[0]);
            sc.A[1] = (float)P[1];
            sc.A[2] = (float)P[2];
            sc.A[3] = (float)P[3];
            sc.A[4] = (float)(1.0 + P[4]);
            sc.A[5] = (float)P[5];
            sc.A[6] = (float)P[6];
            sc.A[7] = (float)P[7];
            sc.A[8] = (float)(1.0 + P[8]);
            sc.t[0] = (float)((double)xc + P[9]);
            sc.t[1] = (float)((double)yc + P[10]);
            sc.t[2] = (float)((double)zcn + P[11]);
        }
        __syncthreads();
        // pass 1: sample into the global buffer, statistics of the valid set
        Acc<NDOF> acc;
        acc.zero();
        const bool slow = sc.slow != 0;
        const float cf = sc.cf;
        for (int v = tid; v < S; v += THREADS) {
            const int iz = v / nXY, rem = v - iz * nXY;
            const int iy = rem / sh.nX, ix = rem - iy * sh.nX;
            const int dx = -sh.hx + ix * a.stride, dy = -sh.hy + iy * a.stride, dz = -sh.hz + iz * a.stride;
            const int64_t xx = xc + dx, yy = yc + dy, zz = zcn + dz;
            bool k;
            if (keep || !inside) {
                k = xx >= 0 && xx < a.nx && yy >= 0 && yy < a.ny && zz >= 0 && zz < a.nz;
                if (k) k = keep ? kept_bit(keep, v) : ((a.mask == nullptr) || __ldg(a.mask + zz * sxy + yy * a.nx + xx) != 0);
            } else {
                k = (a.mask == nullptr) || __ldg(a.mask + zz * sxy + yy * a.nx + xx) != 0;
            }
            if (!k) {
                gbuf[v] = nanf("");
                continue;
            }
            acc.nref += 1;
            const float X = (float)dx, Y = (float)dy, Z = (float)dz;
            if (slow) {
                const double* P = sc.P;
                const double xw = (1.0 + P[0]) * dx + P[1] * dy + P[2] * dz + ((double)xc + P[9]);
                const double yw = P[3] * dx + (1.0 + P[4]) * dy + P[5] * dz + ((double)yc + P[10]);
                const double zw = P[6] * dx + P[7] * dy + (1.0 + P[8]) * dz + ((double)zcn + P[11]);
                if (!margin_ok(zw, yw, xw, a.nz, a.ny, a.nx)) {
                    acc.oob = 1;
                    gbuf[v] = nanf("");
                    continue;
                }
            }
            // absolute positions (the reference's layout: no brick)
            const float xr = sc.A[0] * X + sc.A[1] * Y + sc.A[2] * Z + sc.t[0];
            const float yr = sc.A[3] * X + sc.A[4] * Y + sc.A[5] * Z + sc.t[1];
            const float zr = sc.A[6] * X + sc.A[7] * Y + sc.A[8] * Z + sc.t[2];
            const float gv = sample_rel<MODE>(a.g, a.nx, (int)sxy, a.nx, a.ny, a.nz, xr, yr, zr);
            gbuf[v] = gv;
            if (gv != gv) continue;
            const float fv = __ldg(a.f + zz * sxy + yy * a.nx + xx) - cf;
            const float gs = gv - cf;
            acc.Sg += gs;
            acc.Sgg += gs * gs;
            acc.Sf += fv;
            acc.Sff += fv * fv;
            acc.n += 1;
        }
        reduce_moments<NDOF, THREADS>(acc, red, redi, mom);
        if (tid == 0) {
            int st = 0;
            if (mom.oob)
                st = ST_OOB;
            else if (mom.n < MIN_SUBSET_VOXELS || (double)mom.n < MIN_VALID_FRACTION * (double)mom.nref)
                st = ST_INVALID;
            if (st != 0) {
                node_end<NDOF>(a, node, c12, c3, it, st, nan(""));
                sc.state = 1;
            } else {
                const double n = (double)mom.n;
                const double mg = mom.Sg / n, mf = mom.Sf / n;
                double ssg = mom.Sgg - n * mg * mg, ssf = mom.Sff - n * mf * mf;
                ssg = ssg < 0.0 ? 0.0 : ssg;
                ssf = ssf < 0.0 ? 0.0 : ssf;
                stat[0] = (double)cf + mf;
                stat[1] = (double)cf + mg;
                stat[2] = sqrt(ssf > 1e-30 ? ssf : 1e-30);
                stat[3] = sqrt(ssg > 1e-30 ? ssg : 1e-30);
            }
        }
        __syncthreads();
        if (sc.state != 0) return;
        // pass 2: residual and gradient from the buffer
        const float mfd = (float)stat[0], mgd = (float)stat[1];
        const float ibf = (float)(1.0 / stat[2]), ibg = (float)(1.0 / stat[3]);
        float b[NB];
#pragma unroll
        for (int k = 0; k < NB; ++k) b[k] = 0.0f;
        float scc = 0.0f;
        for (int v = tid; v < S; v += THREADS) {
            const float gv = gbuf[v];
            if (gv != gv) continue;
            const int iz = v / nXY, rem = v - iz * nXY;
            const int iy = rem / sh.nX, ix = rem - iy * sh.nX;
            const int dx = -sh.hx + ix * a.stride, dy = -sh.hy + iy * a.stride, dz = -sh.hz + iz * a.stride;
            const int64_t o = (zcn + dz) * sxy + (yc + dy) * a.nx + (xc + dx);
            const float fd = __ldg(a.f + o) - mfd;
            const float gd = gv - mgd;
            scc += fd * gd;
            const float res = fd * ibf - gd * ibg;
            float q0, q1, q2;
            if (STORED) {
                q0 = __ldg(a.gx + o);
                q1 = __ldg(a.gy + o);
                q2 = __ldg(a.gz + o);
            } else {
                grad_otf(a.f, a.nz, a.ny, a.nx, (int)(zcn + dz), (int)(yc + dy), (int)(xc + dx), q0, q1, q2);
            }
            const float r0 = q0 * res, r1 = q1 * res, r2 = q2 * res;
            if (NDOF == 12) {
                const float X = (float)dx, Y = (float)dy, Z = (float)dz;
                b[0] += r0 * X;
                b[1] += r0 * Y;
                b[2] += r0 * Z;
                b[3] += r1 * X;
                b[4] += r1 * Y;
                b[5] += r1 * Z;
                b[6] += r2 * X;
                b[7] += r2 * Y;
                b[8] += r2 * Z;
                b[9] += r0;
                b[10] += r1;
                b[11] += r2;
            } else {
                b[0] += r0;
                b[1] += r1;
                b[2] += r2;
            }
        }
#pragma unroll
        for (int k = 0; k < NB; ++k) {
            const float s = warp_sum(b[k]);
            if (lane == 0) red[warp][k] = (double)s;
        }
        {
            const float s = warp_sum(scc);
            if (lane == 0) red[warp][NB] = (double)s;
        }
        __syncthreads();
        if (tid == 0) {
            double bt[12], sccd = 0.0;
            for (int k = 0; k < NB; ++k) {
                double s = 0.0;
                for (int w = 0; w < THREADS / 32; ++w) s += red[w][k];
                bt[k] = s * stat[2];  // b *= bottomf (numba_kernels.py:727-729)
            }
            for (int w = 0; w < THREADS / 32; ++w) sccd += red[w][NB];
            double zc = nan("");
            int st;
            if (NDOF == 12)
                st = control12(c12, bt, stat[2], stat[3], sccd, mom.n, Ls, a.H ? a.H + node * 144 : nullptr, a.pattern,
                               a.noise_gain, a.tol, a.dp_tol, a.patience, a.predictive, zc);
            else
                st = control3(c3, bt, stat[2], stat[3], sccd, mom.n, a.mu, a.noise_gain, a.tol, a.dp_tol, a.patience,
                              a.predictive, zc);
            if (st >= 0) {
                node_end<NDOF>(a, node, c12, c3, it, st, zc);
                sc.state = 1;
            } else {
                const double* P = NDOF == 12 ? c12.P : c3.P;
                for (int k = 0; k < 12; ++k) sc.P[k] = P[k];
                if (it == a.max_iter) {
                    node_end<NDOF>(a, node, c12, c3, a.max_iter, ST_MAX_ITER, NDOF == 12 ? c12.zncc : c3.zncc);
                    sc.state = 1;
                }
            }
        }
        __syncthreads();
        if (sc.state != 0) return;
    }
}

// ----------------------------------------------------------------------------- launch plumbing
constexpr int PLAIN_CHUNK = 8192;  // nodes per plain launch (sample buffer rows)

struct LaunchCfg {
    int threads;
    int brick_cap;
    bool tma;  // 128 threads with brick_floats < 0: the lean sweep staged through TMA copies of g
};

static LaunchCfg batched_cfg(const aldvc_icgn_params* prm) {
    LaunchCfg c;
    // 32/64/128: lean kernel with 1/2/4 warps per node; 256/512: shared-brick kernel
    c.threads = prm->threads > 0 ? prm->threads : 256;
    if (c.threads != 32 && c.threads != 64 && c.threads != 128 && c.threads != 256 && c.threads != 512) c.threads = 256;
    c.tma = c.threads == 128 && prm->brick_floats < 0;
    c.brick_cap = prm->brick_floats > 0 ? prm->brick_floats : 24 * 1024;
    return c;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against the driver library)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// The tensor map of g for the staged form: a float32 (nz, ny, nx) volume, box TMA_BX x TMA_BY x TMA_BZ, no swizzle, zero
// fill outside.  False (the caller falls back to the L1 form) when the rows are not 16-byte multiples, g is not
// 16-byte aligned, or the encoder is unavailable.
static bool make_g_map(const IcgnArgs& a, CUtensorMap& map) {
    if ((a.nx & 3) != 0 || (reinterpret_cast<uintptr_t>(a.g) & 15) != 0) return false;
    const auto enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)a.nx, (cuuint64_t)a.ny, (cuuint64_t)a.nz};
    const cuuint64_t strides[2] = {(cuuint64_t)a.nx * sizeof(float), (cuuint64_t)a.nx * a.ny * sizeof(float)};
    const cuuint32_t box[3] = {TMA_BX, TMA_BY, TMA_BZ};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(a.g), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int MODE, bool STORED, int NDOF, int NW, bool UNEVEN = false>
static int launch_lean_t(const IcgnArgs& a, cudaStream_t s);

template <int MODE, int NDOF>
static int launch_tma_t(const IcgnArgs& a, cudaStream_t s) {
    auto kern = icgn_tma_kernel<MODE, NDOF>;
    static int cached_per_sm = -1;  // queried once, outside any stream capture
    static std::mutex mu;
    int per_sm;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (cached_per_sm < 0) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TMA_SMEM);
            if (e != cudaSuccess) return cuda_fail(e, "icgn staged: shared memory attribute");
            int v = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kern, 128, TMA_SMEM);
            if (e != cudaSuccess) return cuda_fail(e, "icgn staged: occupancy");
            cached_per_sm = v;
        }
        per_sm = cached_per_sm;
    }
    if (per_sm < 1) return arg_fail("icgn staged: kernel does not fit on an SM");
    CUtensorMap map;
    if (!make_g_map(a, map)) return launch_lean_t<MODE, true, NDOF, 4>(a, s);
    long long grid = (long long)per_sm * sm_count();
    if (grid > a.n_nodes) grid = a.n_nodes;
    {
        KTimer kt_(NDOF == 12 ? "icgn12_tma" : "icgn3_tma", s);
        kern<<<(unsigned)grid, 128, TMA_SMEM, s>>>(a, map);
    }
    return check_launch("icgn staged");
}

template <int MODE, bool STORED, int NDOF, int THREADS>
static int launch_batched_t(const IcgnArgs& a, int brick_cap, cudaStream_t s) {
    auto kern = icgn_batched_kernel<MODE, STORED, NDOF, THREADS>;
    const size_t smem = (size_t)brick_cap * sizeof(float);
    // attribute and occupancy are set up once per (instantiation, brick size) so that launches inside a
    // stream capture make no configuration calls
    static int cached_cap = -1, cached_per_sm = 0;
    static std::mutex mu;
    int per_sm;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (cached_cap != brick_cap) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return cuda_fail(e, "icgn batched: shared memory attribute");
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cached_per_sm, kern, THREADS, smem);
            if (e != cudaSuccess) return cuda_fail(e, "icgn batched: occupancy");
            cached_cap = brick_cap;
        }
        per_sm = cached_per_sm;
    }
    if (per_sm < 1) return arg_fail("icgn batched: brick does not fit in shared memory");
    long long grid = (long long)per_sm * sm_count();
    if (grid > a.n_nodes) grid = a.n_nodes;
    {
        KTimer kt_(NDOF == 12 ? "icgn12_batched" : "icgn3_batched", s);
        kern<<<(unsigned)grid, THREADS, smem, s>>>(a);
    }
    return check_launch("icgn batched");
}

template <int MODE, bool STORED, int NDOF, int NW, bool UNEVEN>
static int launch_lean_t(const IcgnArgs& a, cudaStream_t s) {
    auto kern = icgn_lean_kernel<MODE, STORED, NDOF, NW, UNEVEN>;
    static int cached_per_sm = -1;  // queried once, outside any stream capture
    static std::mutex mu;
    int per_sm;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (cached_per_sm < 0) {
            int v = 0;
            cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kern, NW * 32, 0);
            if (e != cudaSuccess) return cuda_fail(e, "icgn lean: occupancy");
            cached_per_sm = v;
        }
        per_sm = cached_per_sm;
    }
    if (per_sm < 1) return arg_fail("icgn lean: kernel does not fit on an SM");
    long long grid = (long long)per_sm * sm_count();
    if (grid > a.n_nodes) grid = a.n_nodes;
    {
        KTimer kt_(NDOF == 12 ? "icgn12_lean" : "icgn3_lean", s);
        kern<<<(unsigned)grid, NW * 32, 0, s>>>(a);
    }
    return check_launch("icgn lean");
}

template <int MODE, bool STORED, int NDOF>
static int launch_batched_m(const IcgnArgs& a, const LaunchCfg& c, cudaStream_t s) {
    // per-node shapes run on the lean kernel with 4 warps per node (the brick kernel stages one shape per call)
    if (a.node_half) return launch_lean_t<MODE, STORED, NDOF, 4, true>(a, s);
    if constexpr (MODE != 0 && STORED)
        if (c.tma && !a.split_index) return launch_tma_t<MODE, NDOF>(a, s);
    switch (c.threads) {
        case 32: return launch_lean_t<MODE, STORED, NDOF, 1>(a, s);
        case 64: return launch_lean_t<MODE, STORED, NDOF, 2>(a, s);
        case 128: return launch_lean_t<MODE, STORED, NDOF, 4>(a, s);
        case 512: return launch_batched_t<MODE, STORED, NDOF, 512>(a, c.brick_cap, s);
        default: return launch_batched_t<MODE, STORED, NDOF, 256>(a, c.brick_cap, s);
    }
}

// 32-bit voxel indices in the lean sweep (volumes below 2^31 voxels); ALDVC_ICGN_IDX32=0 keeps 64-bit indices (a
// comparison knob, read once)
static bool icgn_idx32() {
    static const bool on = [] {
        const char* e = std::getenv("ALDVC_ICGN_IDX32");
        return !(e && e[0] == '0');
    }();
    return on;
}

template <int MODE, bool STORED, int NDOF>
static int launch_plain_m(IcgnArgs a, cudaStream_t s) {
    for (int64_t start = 0; start < a.n_nodes; start += PLAIN_CHUNK) {
        a.node_base = start;
        const int64_t n = std::min<int64_t>(PLAIN_CHUNK, a.n_nodes - start);
        {
            KTimer kt_(NDOF == 12 ? "icgn12_plain" : "icgn3_plain", s);
            icgn_plain_kernel<MODE, STORED, NDOF><<<(unsigned)n, 256, 0, s>>>(a);
        }
        const int rc = check_launch("icgn plain");
        if (rc) return rc;
    }
    return ALDVC_OK;
}

template <int NDOF>
static int dispatch(const IcgnArgs& a, int mode, bool stored, int variant, const LaunchCfg& c, cudaStream_t s) {
    if (variant == ALDVC_PLAIN) {
        if (mode == 0) return stored ? launch_plain_m<0, true, NDOF>(a, s) : launch_plain_m<0, false, NDOF>(a, s);
        if (mode == 1) return stored ? launch_plain_m<1, true, NDOF>(a, s) : launch_plain_m<1, false, NDOF>(a, s);
        return stored ? launch_plain_m<2, true, NDOF>(a, s) : launch_plain_m<2, false, NDOF>(a, s);
    }
    if (mode == 0) return stored ? launch_batched_m<0, true, NDOF>(a, c, s) : launch_batched_m<0, false, NDOF>(a, c, s);
    if (mode == 1) return stored ? launch_batched_m<1, true, NDOF>(a, c, s) : launch_batched_m<1, false, NDOF>(a, c, s);
    return stored ? launch_batched_m<2, true, NDOF>(a, c, s) : launch_batched_m<2, false, NDOF>(a, c, s);
}

static int fill_common(IcgnArgs& a, const aldvc_volumes* vol, const aldvc_subset* sub, const int64_t* coords, int64_t n,
                       const aldvc_icgn_params* prm) {
    ALDVC_REQUIRE(vol && sub && prm, "icgn: null descriptor");
    ALDVC_REQUIRE(vol->f && vol->g && coords, "icgn: null volume/coords pointer");
    ALDVC_REQUIRE(sub->hx >= 0 && sub->hy >= 0 && sub->hz >= 0 && sub->stride >= 1, "icgn: bad subset");
    ALDVC_REQUIRE(sub->mode >= 0 && sub->mode <= 2, "icgn: mode must be 0, 1 or 2");
    ALDVC_REQUIRE(vol->nz >= 4 && vol->ny >= 4 && vol->nx >= 4 && vol->nx * vol->ny < (1LL << 31) && vol->nz < (1 << 30),
                  "icgn: bad volume shape");
    ALDVC_REQUIRE(n < (1LL << 31), "icgn: too many nodes");
    ALDVC_REQUIRE(prm->max_iter >= 1, "icgn: max_iter must be >= 1");
    const bool stored = vol->gx && vol->gy && vol->gz;
    ALDVC_REQUIRE(stored || (!vol->gx && !vol->gy && !vol->gz), "icgn: give all three gradients or none");
    ALDVC_REQUIRE(!sub->split_index || (sub->split_keep && sub->keep_bytes > 0), "icgn: split rows missing");
    std::memset(&a, 0, sizeof(a));
    a.f = vol->f;
    a.gx = vol->gx;
    a.gy = vol->gy;
    a.gz = vol->gz;
    a.mask = vol->mask;
    a.g = vol->g;
    a.g4 = reinterpret_cast<const float4*>(vol->g4);
    a.idx32 = icgn_idx32() && vol->nz * vol->ny * vol->nx < (1LL << 31) - 64 ? 1 : 0;
    a.nz = (int)vol->nz;
    a.ny = (int)vol->ny;
    a.nx = (int)vol->nx;
    a.hx = sub->hx;
    a.hy = sub->hy;
    a.hz = sub->hz;
    a.stride = sub->stride;
    a.nX = (2 * sub->hx) / sub->stride + 1;
    a.nY = (2 * sub->hy) / sub->stride + 1;
    a.nZ = (2 * sub->hz) / sub->stride + 1;
    a.split_index = sub->split_index;
    a.split_keep = sub->split_keep;
    a.keep_bytes = sub->keep_bytes;
    ALDVC_REQUIRE(!(sub->node_half && sub->split_index), "icgn: per-node shapes do not combine with split rows");
    ALDVC_REQUIRE(!(sub->node_half && prm->noise_gain > 0.0), "icgn: per-node shapes do not combine with the noise correction");
    a.node_half = sub->node_half;
    a.coords = coords;
    a.n_nodes = n;
    a.tol = prm->tol;
    a.dp_tol = prm->dp_tol;
    a.noise_gain = prm->noise_gain;
    a.max_iter = prm->max_iter;
    a.patience = prm->patience;
    a.predictive = prm->predictive;
    a.mu = prm->mu;
    a.n_full = prm->n_full;
    return ALDVC_OK;
}

static size_t workspace_bytes(const aldvc_subset* sub, int64_t n, const aldvc_icgn_params* prm) {
    size_t b = 256;  // work counter
    if (prm && prm->variant == ALDVC_PLAIN && sub) {
        const int64_t S = subset_count(sub->hx, sub->hy, sub->hz, std::max(1, sub->stride));
        b += (size_t)std::min<int64_t>(n, PLAIN_CHUNK) * (size_t)S * sizeof(float);
    }
    return b;
}

static int run(IcgnArgs& a, int ndof, int mode, bool stored, const aldvc_icgn_params* prm, void* ws, size_t ws_bytes,
               const aldvc_subset* sub, cudaStream_t s) {
    const size_t need = workspace_bytes(sub, a.n_nodes, prm);
    if (!ws || ws_bytes < need) {
        set_error("icgn: workspace of %zu bytes needed, %zu given", need, ws_bytes);
        return ALDVC_ERR_WORKSPACE;
    }
    a.counter = (int*)ws;
    a.err = (int32_t*)ws + 1;  // next to the counter; reset with it
    a.gbuf = (float*)((char*)ws + 256);
    const LaunchCfg c = batched_cfg(prm);
    a.brick_cap = c.brick_cap;
    a.sweep_rows = prm->sweep_rows;
    a.node_order = prm->node_order;
    if (prm->variant != ALDVC_PLAIN) {
        const size_t smem = (size_t)c.brick_cap * sizeof(float);
        if (smem + 8192 > (size_t)max_smem_optin()) return arg_fail("icgn: brick_floats exceeds the shared memory per block");
        cudaError_t e = cudaMemsetAsync(a.counter, 0, 2 * sizeof(int), s);
        if (e != cudaSuccess) return cuda_fail(e, "icgn: counter reset");
    }
    return ndof == 12 ? dispatch<12>(a, mode, stored, prm->variant, c, s) : dispatch<3>(a, mode, stored, prm->variant, c, s);
}

}  // namespace aldvc

using namespace aldvc;

extern "C" size_t aldvc_icgn_workspace_size(const aldvc_subset* sub, int64_t n_nodes, const aldvc_icgn_params* prm) {
    return workspace_bytes(sub, n_nodes, prm);
}

extern "C" int aldvc_icgn12(const aldvc_volumes* vol, const aldvc_subset* sub, const int64_t* coords, int64_t n_nodes,
                            const double* P0, const double* L_all, const double* H_all, const double* pattern,
                            const double* meanf_all, const uint8_t* valid, const aldvc_icgn_params* prm, void* workspace,
                            size_t workspace_bytes_, double* P_out, int32_t* n_iter, int8_t* status, double* zncc, void* stream) {
    IcgnArgs a;
    int rc = fill_common(a, vol, sub, coords, n_nodes, prm);
    if (rc) return rc;
    ALDVC_REQUIRE(P0 && L_all && meanf_all && valid && P_out && n_iter && status && zncc, "aldvc_icgn12: null pointer");
    const bool noise = prm->noise_gain > 0.0 && H_all && pattern;
    if (n_nodes <= 0) return ALDVC_OK;
    a.P0 = P0;
    a.L = L_all;
    a.H = noise ? H_all : nullptr;
    a.pattern = noise ? pattern : nullptr;
    a.noise_gain = noise ? prm->noise_gain : 0.0;
    a.meanf = meanf_all;
    a.valid = valid;
    a.P_out = P_out;
    a.n_iter = n_iter;
    a.status = status;
    a.zncc = zncc;
    return run(a, 12, sub->mode, vol->gx != nullptr, prm, workspace, workspace_bytes_, sub, (cudaStream_t)stream);
}

extern "C" int aldvc_icgn3(const aldvc_volumes* vol, const aldvc_subset* sub, const int64_t* coords, int64_t n_nodes,
                           const double* U_old, const double* F_fixed, const double* vdual, const double* H_all,
                           const double* meanf_all, const double* bottomf_all, const uint8_t* valid, const aldvc_icgn_params* prm,
                           void* workspace, size_t workspace_bytes_, double* U_out, int32_t* n_iter, int8_t* status, double* zncc,
                           void* stream) {
    IcgnArgs a;
    int rc = fill_common(a, vol, sub, coords, n_nodes, prm);
    if (rc) return rc;
    ALDVC_REQUIRE(U_old && F_fixed && vdual && H_all && meanf_all && bottomf_all && valid && U_out && n_iter && status && zncc,
                  "aldvc_icgn3: null pointer");
    if (n_nodes <= 0) return ALDVC_OK;
    a.U_old = U_old;
    a.F_fixed = F_fixed;
    a.vdual = vdual;
    a.H = H_all;
    a.meanf = meanf_all;
    a.bottomf = bottomf_all;
    a.valid = valid;
    a.P_out = U_out;
    a.n_iter = n_iter;
    a.status = status;
    a.zncc = zncc;
    a.noise_gain = prm->noise_gain > 0.0 ? prm->noise_gain : 0.0;
    return run(a, 3, sub->mode, vol->gx != nullptr, prm, workspace, workspace_bytes_, sub, (cudaStream_t)stream);
}
