/*
 * CPU oracle for the AL-DVC hot path: a plain-C, FP64 restatement of the
 * reference's Numba CPU kernels (pyALDVC v1.2.1, src/al_dvc/solver/...).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA library is
 * compared against (tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg).  Nothing in the product path (pyaldvc_b200/) links, loads
 * or calls it.
 *
 * Every arithmetic step follows the reference loop order so the results
 * agree with the reference to ~1e-12; the agreement is pinned by the golden
 * fixtures under tests/golden/ (generated by importing the reference).
 *
 * Conventions (same as the reference):
 *   volumes are (nz, ny, nx) float32, C order; node coordinates are int64
 *   [x, y, z]; warp parameters P[0:9] = F row-major (F_ij = du_i/dx_j),
 *   P[9:12] = (u, v, w); x_def = x0 + u + (I + F)(x - x0).
 *   Status codes: 0 converged, 1 max_iter, 2 out_of_bounds, 3 invalid
 *   subset, 4 singular, 5 nan, 6 skipped, 7 stalled.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ST_CONVERGED 0
#define ST_MAX_ITER 1
#define ST_OOB 2
#define ST_INVALID 3
#define ST_SINGULAR 4
#define ST_NAN 5
#define ST_SKIPPED 6
#define ST_STALLED 7

/* numba_kernels.py:38-44, 81-85 */
#define ABS_TOL 1e-5
#define STALL_ZNCC_EPS 1e-4
#define STALL_STEP_DECAY 0.999
#define MIN_SUBSET_VOXELS 27
#define MIN_VALID_FRACTION 0.5
#define LM_DAMPING_3DOF 1e-3
#define MIN_CORRECTED_FRACTION 0.5
#define NOISE_CORR_STEP 0.5
#define PREDICT_CONTRACTION 0.5

typedef struct {
    const float *p;
    int64_t nz, ny, nx;
} vol_t;

static inline double V(const vol_t *v, int64_t z, int64_t y, int64_t x) {
    return (double)v->p[(z * v->ny + y) * v->nx + x];
}

/* The reference reads volume voxels with Numba's float(), which keeps a float32
 * element in float32: a difference of two voxels and the square of a voxel are
 * rounded to float32 before they meet float64 arithmetic.  D32/SQ32 reproduce
 * exactly that (FLT_EVAL_METHOD 0 on x86-64). */
static inline float VF(const vol_t *v, int64_t z, int64_t y, int64_t x) { return v->p[(z * v->ny + y) * v->nx + x]; }
static inline double D32(float a, float b) {
    float d = a - b;
    return (double)d;
}
static inline double SQ32(float a) {
    float q = a * a;
    return (double)q;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------ interpolation
 * interp_kernels.py:34-136 */
static inline void keys_w(double t, double *w) {
    w[0] = ((-0.5 * t + 1.0) * t - 0.5) * t;
    w[1] = (1.5 * t - 2.5) * t * t + 1.0;
    w[2] = ((-1.5 * t + 2.0) * t + 0.5) * t;
    w[3] = (0.5 * t - 0.5) * t * t;
}

static inline void bspl_w(double t, double *w) {
    double t2 = t * t, t3 = t2 * t;
    w[0] = (1.0 - 3.0 * t + 3.0 * t2 - t3) / 6.0;
    w[1] = (4.0 - 6.0 * t2 + 3.0 * t3) / 6.0;
    w[2] = (1.0 + 3.0 * t + 3.0 * t2 - 3.0 * t3) / 6.0;
    w[3] = t3 / 6.0;
}

static inline int margin_ok(double z, double y, double x, int64_t nz, int64_t ny, int64_t nx) {
    if (x < 1.0 || x > (double)nx - 1.0 - 2.0) return 0;
    if (y < 1.0 || y > (double)ny - 1.0 - 2.0) return 0;
    if (z < 1.0 || z > (double)nz - 1.0 - 2.0) return 0;
    return 1;
}

static inline double row4(const vol_t *v, int64_t z, int64_t y, int64_t xb, const double *wx) {
    return V(v, z, y, xb) * wx[0] + V(v, z, y, xb + 1) * wx[1] + V(v, z, y, xb + 2) * wx[2] + V(v, z, y, xb + 3) * wx[3];
}

static inline double plane4(const vol_t *v, int64_t z, int64_t yb, int64_t xb, const double *wx, const double *wy) {
    return row4(v, z, yb, xb, wx) * wy[0] + row4(v, z, yb + 1, xb, wx) * wy[1] + row4(v, z, yb + 2, xb, wx) * wy[2] +
           row4(v, z, yb + 3, xb, wx) * wy[3];
}

/* interp_kernels.sample_volume (:71-124); the caller has checked margin_ok */
static double sample(const vol_t *v, double z, double y, double x, int mode) {
    int64_t ix = (int64_t)floor(x), iy = (int64_t)floor(y), iz = (int64_t)floor(z);
    if (ix > v->nx - 3) ix = v->nx - 3;
    if (iy > v->ny - 3) iy = v->ny - 3;
    if (iz > v->nz - 3) iz = v->nz - 3;
    double fx = x - (double)ix, fy = y - (double)iy, fz = z - (double)iz;
    if (mode == 0) {
        double c00 = V(v, iz, iy, ix) * (1.0 - fx) + V(v, iz, iy, ix + 1) * fx;
        double c10 = V(v, iz, iy + 1, ix) * (1.0 - fx) + V(v, iz, iy + 1, ix + 1) * fx;
        double c01 = V(v, iz + 1, iy, ix) * (1.0 - fx) + V(v, iz + 1, iy, ix + 1) * fx;
        double c11 = V(v, iz + 1, iy + 1, ix) * (1.0 - fx) + V(v, iz + 1, iy + 1, ix + 1) * fx;
        double c0 = c00 * (1.0 - fy) + c10 * fy;
        double c1 = c01 * (1.0 - fy) + c11 * fy;
        return c0 * (1.0 - fz) + c1 * fz;
    }
    double wx[4], wy[4], wz[4];
    if (mode == 1) {
        keys_w(fx, wx);
        keys_w(fy, wy);
        keys_w(fz, wz);
    } else {
        bspl_w(fx, wx);
        bspl_w(fy, wy);
        bspl_w(fz, wz);
    }
    int64_t xb = ix - 1, yb = iy - 1, zb = iz - 1;
    return plane4(v, zb, yb, xb, wx, wy) * wz[0] + plane4(v, zb + 1, yb, xb, wx, wy) * wz[1] +
           plane4(v, zb + 2, yb, xb, wx, wy) * wz[2] + plane4(v, zb + 3, yb, xb, wx, wy) * wz[3];
}

/* interp_kernels.sample_points (:139-152): NaN outside the admissible domain */
void orc_sample_points(const float *vol, int64_t nz, int64_t ny, int64_t nx, const double *zs, const double *ys,
                       const double *xs, int64_t n, int mode, double *out) {
    vol_t v = {vol, nz, ny, nx};
    for (int64_t i = 0; i < n; ++i)
        out[i] = margin_ok(zs[i], ys[i], xs[i], nz, ny, nx) ? sample(&v, zs[i], ys[i], xs[i], mode) : NAN;
}

/* ------------------------------------------------------------------ gradients
 * volume_ops._gradient_stencil7 (:124-155): 7-point central differences,
 * zero within `border` voxels of any face; arithmetic FP64, storage FP32. */
void orc_gradients(const float *f, int64_t nz, int64_t ny, int64_t nx, int64_t border, float *gx, float *gy, float *gz) {
    vol_t v = {f, nz, ny, nx};
    const double c1 = 3.0 / 4.0, c2 = -3.0 / 20.0, c3 = 1.0 / 60.0;
#pragma omp parallel for schedule(static)
    for (int64_t z = 0; z < nz; ++z) {
        int z_in = z >= border && z < nz - border;
        for (int64_t y = 0; y < ny; ++y) {
            int y_in = y >= border && y < ny - border;
            for (int64_t x = 0; x < nx; ++x) {
                int64_t o = (z * ny + y) * nx + x;
                if (z_in && y_in && x >= border && x < nx - border) {
                    gx[o] = (float)(c1 * D32(VF(&v, z, y, x + 1), VF(&v, z, y, x - 1)) + c2 * D32(VF(&v, z, y, x + 2), VF(&v, z, y, x - 2)) +
                                    c3 * D32(VF(&v, z, y, x + 3), VF(&v, z, y, x - 3)));
                    gy[o] = (float)(c1 * D32(VF(&v, z, y + 1, x), VF(&v, z, y - 1, x)) + c2 * D32(VF(&v, z, y + 2, x), VF(&v, z, y - 2, x)) +
                                    c3 * D32(VF(&v, z, y + 3, x), VF(&v, z, y - 3, x)));
                    gz[o] = (float)(c1 * D32(VF(&v, z + 1, y, x), VF(&v, z - 1, y, x)) + c2 * D32(VF(&v, z + 2, y, x), VF(&v, z - 2, y, x)) +
                                    c3 * D32(VF(&v, z + 3, y, x), VF(&v, z - 3, y, x)));
                } else {
                    gx[o] = gy[o] = gz[o] = 0.0f;
                }
            }
        }
    }
}

/* ------------------------------------------------------------------ shared subset context */
typedef struct {
    vol_t f, gx, gy, gz, g;
    const uint8_t *mask; /* NULL: every voxel counts (the reference's 1x1x1 placeholder) */
    int stored;          /* gradients stored (else the 7-point stencil on f, _grad_at :188-212) */
    int hx, hy, hz, stride, mode;
} ctx_t;

static inline void grad_at(const ctx_t *c, int64_t zz, int64_t yy, int64_t xx, double *gx, double *gy, double *gz) {
    if (c->stored) {
        *gx = V(&c->gx, zz, yy, xx);
        *gy = V(&c->gy, zz, yy, xx);
        *gz = V(&c->gz, zz, yy, xx);
        return;
    }
    const vol_t *f = &c->f;
    const double c1 = 0.75, c2 = -0.15, c3 = 1.0 / 60.0;
    *gx = c1 * D32(VF(f, zz, yy, xx + 1), VF(f, zz, yy, xx - 1)) + c2 * D32(VF(f, zz, yy, xx + 2), VF(f, zz, yy, xx - 2)) +
          c3 * D32(VF(f, zz, yy, xx + 3), VF(f, zz, yy, xx - 3));
    *gy = c1 * D32(VF(f, zz, yy + 1, xx), VF(f, zz, yy - 1, xx)) + c2 * D32(VF(f, zz, yy + 2, xx), VF(f, zz, yy - 2, xx)) +
          c3 * D32(VF(f, zz, yy + 3, xx), VF(f, zz, yy - 3, xx));
    *gz = c1 * D32(VF(f, zz + 1, yy, xx), VF(f, zz - 1, yy, xx)) + c2 * D32(VF(f, zz + 2, yy, xx), VF(f, zz - 2, yy, xx)) +
          c3 * D32(VF(f, zz + 3, yy, xx), VF(f, zz - 3, yy, xx));
}

static inline int kept_bit(const uint8_t *keep, int64_t idx) { return ((keep[idx >> 3] >> (idx & 7)) & 1) != 0; }

static inline int64_t subset_count(int hx, int hy, int hz, int stride) {
    return (int64_t)((2 * hx) / stride + 1) * ((2 * hy) / stride + 1) * ((2 * hz) / stride + 1);
}

/* ------------------------------------------------------------------ small dense algebra
 * numba_kernels.py:58-180 */
static int chol12(const double *H, double *L) {
    for (int i = 0; i < 144; ++i) L[i] = 0.0;
    for (int j = 0; j < 12; ++j) {
        double s = H[j * 12 + j];
        for (int k = 0; k < j; ++k) s -= L[j * 12 + k] * L[j * 12 + k];
        if (s <= 0.0 || !isfinite(s)) return 0;
        double ljj = sqrt(s);
        L[j * 12 + j] = ljj;
        for (int i = j + 1; i < 12; ++i) {
            double t = H[i * 12 + j];
            for (int k = 0; k < j; ++k) t -= L[i * 12 + k] * L[j * 12 + k];
            L[i * 12 + j] = t / ljj;
        }
    }
    return 1;
}

static int corrected_chol12(const double *H, const double *pattern, double corr, double *H0, double *L0) {
    double limit = 1.0;
    for (int i = 9; i < 12; ++i) {
        double c = corr * pattern[i * 12 + i];
        if (c > 0.0) {
            double lim = (1.0 - MIN_CORRECTED_FRACTION) * H[i * 12 + i] / c;
            if (lim < limit) limit = lim;
        }
    }
    if (limit <= 0.0) return 0;
    for (int i = 0; i < 144; ++i) H0[i] = H[i] - corr * limit * pattern[i];
    return chol12(H0, L0);
}

static void chol_solve12(const double *L, const double *b, double *x) {
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

static double inv3(const double a[3][3], double out[3][3]) {
    double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                 a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
    if (fabs(det) < 1e-300) return 0.0;
    double inv = 1.0 / det;
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

/* compose_warp_inplace (:145-180): W(P) <- W(P) o W(dP)^-1 */
int orc_compose_warp(double *P, const double *dP) {
    double A[3][3], dA[3][3], dAi[3][3], An[3][3];
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) {
            A[i][j] = P[3 * i + j];
            dA[i][j] = dP[3 * i + j];
        }
        A[i][i] += 1.0;
        dA[i][i] += 1.0;
    }
    if (inv3(dA, dAi) == 0.0) return 0;
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
    return 1;
}

/* ------------------------------------------------------------------ precompute
 * _precompute_one (:326-418) and _precompute_nodes_jit (:446-496) */
static int precompute_one(const ctx_t *c, int64_t x0, int64_t y0, int64_t z0, double min_valid_ratio, double cond_max, double *H,
                          double *L, const uint8_t *keep, int use_keep, double *meanf_o, double *bottomf_o, int64_t *nvalid_o) {
    const int hx = c->hx, hy = c->hy, hz = c->hz, stride = c->stride;
    const int64_t nz = c->f.nz, ny = c->f.ny, nx = c->f.nx;
    for (int i = 0; i < 144; ++i) H[i] = 0.0;
    if (!use_keep && (x0 - hx < 0 || x0 + hx >= nx || y0 - hy < 0 || y0 + hy >= ny || z0 - hz < 0 || z0 + hz >= nz)) {
        *meanf_o = 0.0;
        *bottomf_o = 1.0;
        *nvalid_o = 0;
        return 0;
    }
    double sd[12];
    int64_t idx = 0, n_valid = 0;
    double sum_f = 0.0, sum_f2 = 0.0;
    for (int dz = -hz; dz <= hz; dz += stride) {
        int64_t zz = z0 + dz;
        double Z = (double)dz;
        for (int dy = -hy; dy <= hy; dy += stride) {
            int64_t yy = y0 + dy;
            double Y = (double)dy;
            for (int dx = -hx; dx <= hx; dx += stride) {
                int64_t xx = x0 + dx;
                int k;
                if (use_keep)
                    k = kept_bit(keep, idx);
                else
                    k = (c->mask == NULL) || c->mask[(zz * ny + yy) * nx + xx] != 0;
                idx += 1;
                if (!k) continue;
                double X = (double)dx;
                float fv32 = VF(&c->f, zz, yy, xx);
                double fv = (double)fv32;
                double gxv, gyv, gzv;
                grad_at(c, zz, yy, xx, &gxv, &gyv, &gzv);
                n_valid += 1;
                sum_f += fv;
                sum_f2 += SQ32(fv32);
                sd[0] = gxv * X;
                sd[1] = gxv * Y;
                sd[2] = gxv * Z;
                sd[3] = gyv * X;
                sd[4] = gyv * Y;
                sd[5] = gyv * Z;
                sd[6] = gzv * X;
                sd[7] = gzv * Y;
                sd[8] = gzv * Z;
                sd[9] = gxv;
                sd[10] = gyv;
                sd[11] = gzv;
                for (int a = 0; a < 12; ++a) {
                    double sa = sd[a];
                    for (int b = a; b < 12; ++b) H[a * 12 + b] += sa * sd[b];
                }
            }
        }
    }
    for (int a = 0; a < 12; ++a)
        for (int b = 0; b < a; ++b) H[a * 12 + b] = H[b * 12 + a];
    *nvalid_o = n_valid;
    int64_t total = subset_count(hx, hy, hz, stride);
    if (n_valid < 27 || (double)n_valid < min_valid_ratio * (double)total) {
        *meanf_o = 0.0;
        *bottomf_o = 1.0;
        return 0;
    }
    double meanf = sum_f / (double)n_valid;
    double ssf = sum_f2 - (double)n_valid * meanf * meanf;
    if (ssf < 0.0) ssf = 0.0;
    double bottomf = sqrt(ssf > 1e-30 ? ssf : 1e-30);
    *meanf_o = meanf;
    *bottomf_o = bottomf;
    if (bottomf < 1e-10) return 0;
    if (!chol12(H, L)) return 0;
    double dmin = L[0], dmax = L[0];
    for (int i = 1; i < 12; ++i) {
        double d = L[i * 12 + i];
        if (d < dmin) dmin = d;
        if (d > dmax) dmax = d;
    }
    if (dmin <= 0.0 || (dmax / dmin) * (dmax / dmin) > cond_max) return 0;
    return 1;
}

static void make_ctx(ctx_t *c, const float *f, const float *gx, const float *gy, const float *gz, int stored, const uint8_t *mask,
                     const float *g, int64_t nz, int64_t ny, int64_t nx, int hx, int hy, int hz, int stride, int mode) {
    c->f = (vol_t){f, nz, ny, nx};
    c->gx = (vol_t){gx, nz, ny, nx};
    c->gy = (vol_t){gy, nz, ny, nx};
    c->gz = (vol_t){gz, nz, ny, nx};
    c->g = (vol_t){g, nz, ny, nx};
    c->mask = mask;
    c->stored = stored;
    c->hx = hx;
    c->hy = hy;
    c->hz = hz;
    c->stride = stride;
    c->mode = mode;
}

/* split_index (N,) int64 (-1: whole in-mask subset), split_keep rows of keep_bytes packed bits */
void orc_precompute(const int64_t *coords, int64_t N, int hx, int hy, int hz, int stride, const float *f, const float *gx,
                    const float *gy, const float *gz, int stored, const uint8_t *mask, int64_t nz, int64_t ny, int64_t nx,
                    const int64_t *split_index, const uint8_t *split_keep, int64_t keep_bytes, double min_valid_ratio,
                    double cond_max, double *H_all, double *L_all, double *meanf, double *bottomf, int64_t *n_valid,
                    uint8_t *valid) {
    ctx_t c;
    make_ctx(&c, f, gx, gy, gz, stored, mask, NULL, nz, ny, nx, hx, hy, hz, stride, 0);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t n = 0; n < N; ++n) {
        int64_t r = split_index ? split_index[n] : -1;
        int use_keep = r >= 0;
        const uint8_t *keep = use_keep ? split_keep + r * keep_bytes : NULL;
        double *L = L_all + n * 144;
        for (int i = 0; i < 144; ++i) L[i] = 0.0;
        valid[n] = (uint8_t)precompute_one(&c, coords[3 * n], coords[3 * n + 1], coords[3 * n + 2], min_valid_ratio, cond_max,
                                           H_all + n * 144, L, keep, use_keep, &meanf[n], &bottomf[n], &n_valid[n]);
    }
}

/* ------------------------------------------------------------------ warp + sample
 * _warp_and_sample (:517-598).  Returns ok; fills gbuf (NaN = excluded). */
static int warp_and_sample(const ctx_t *c, const double *P, int64_t x0, int64_t y0, int64_t z0, double *gbuf, const uint8_t *keep,
                           int use_keep, int64_t *nv_o, double *meanf_o, double *bottomf_o, double *meang_o, double *bottomg_o) {
    const int hx = c->hx, hy = c->hy, hz = c->hz, stride = c->stride;
    const int64_t nz = c->g.nz, ny = c->g.ny, nx = c->g.nx;
    double a00 = 1.0 + P[0], a01 = P[1], a02 = P[2];
    double a10 = P[3], a11 = 1.0 + P[4], a12 = P[5];
    double a20 = P[6], a21 = P[7], a22 = 1.0 + P[8];
    double tx = (double)x0 + P[9], ty = (double)y0 + P[10], tz = (double)z0 + P[11];
    int64_t n_valid = 0, n_ref = 0, idx = 0;
    double s1 = 0.0, s2 = 0.0, s1f = 0.0, s2f = 0.0;
    for (int dz = -hz; dz <= hz; dz += stride) {
        double Z = (double)dz;
        int64_t zz = z0 + dz;
        for (int dy = -hy; dy <= hy; dy += stride) {
            double Y = (double)dy;
            int64_t yy = y0 + dy;
            for (int dx = -hx; dx <= hx; dx += stride) {
                int skip;
                if (use_keep)
                    skip = !kept_bit(keep, idx);
                else
                    skip = (c->mask != NULL) && c->mask[(zz * ny + yy) * nx + (x0 + dx)] == 0;
                if (skip) {
                    gbuf[idx] = NAN;
                    idx += 1;
                    continue;
                }
                n_ref += 1;
                double X = (double)dx;
                double xw = a00 * X + a01 * Y + a02 * Z + tx;
                double yw = a10 * X + a11 * Y + a12 * Z + ty;
                double zw = a20 * X + a21 * Y + a22 * Z + tz;
                if (!margin_ok(zw, yw, xw, nz, ny, nx)) {
                    *nv_o = 0;
                    return 0;
                }
                double val = sample(&c->g, zw, yw, xw, c->mode);
                gbuf[idx] = val;
                idx += 1;
                if (val != val) continue;
                float fv32 = VF(&c->f, zz, yy, x0 + dx);
                n_valid += 1;
                s1 += val;
                s2 += val * val;
                s1f += (double)fv32;
                s2f += SQ32(fv32);
            }
        }
    }
    *nv_o = n_valid;
    if (n_valid < MIN_SUBSET_VOXELS || (double)n_valid < MIN_VALID_FRACTION * (double)n_ref) return 0;
    double meang = s1 / (double)n_valid;
    double ssg = s2 - (double)n_valid * meang * meang;
    if (ssg < 0.0) ssg = 0.0;
    *bottomg_o = sqrt(ssg > 1e-30 ? ssg : 1e-30);
    double meanf = s1f / (double)n_valid;
    double ssf = s2f - (double)n_valid * meanf * meanf;
    if (ssf < 0.0) ssf = 0.0;
    *bottomf_o = sqrt(ssf > 1e-30 ? ssf : 1e-30);
    *meanf_o = meanf;
    *meang_o = meang;
    return 1;
}

/* ------------------------------------------------------------------ 12-DOF IC-GN
 * _icgn_12dof_single (:624-792) */
static int icgn12_single(const ctx_t *c, double *P, int64_t x0, int64_t y0, int64_t z0, const double *L, double tol, double dp_tol,
                         int max_iter, int patience, double *gbuf, const double *H, const double *pattern, double noise_gain,
                         int predictive, const uint8_t *keep, int use_keep, int *n_iter_o, double *zncc_o) {
    const int hx = c->hx, hy = c->hy, hz = c->hz, stride = c->stride;
    double b[12], dP[12], negb[12], H0[144], L0[144], P_best[12];
    double n_full = pattern[9 * 12 + 9];
    double last_dp = 1e300, dp_prev = -1.0, norm_init = -1.0;
    int half_i = hx > hy ? hx : hy;
    if (hz > half_i) half_i = hz;
    double half_scale = (double)half_i;
    double zncc = NAN, best_zncc = -2.0, best_dp = 1e300;
    int stall = 0;
    for (int k = 0; k < 12; ++k) P_best[k] = P[k]; /* unread before the first write in the reference */
    for (int it = 1; it <= max_iter; ++it) {
        int64_t n_valid;
        double meanf_d = 0, bottomf_d = 1, meang = 0, bottomg = 1;
        int ok = warp_and_sample(c, P, x0, y0, z0, gbuf, keep, use_keep, &n_valid, &meanf_d, &bottomf_d, &meang, &bottomg);
        if (!ok) {
            *n_iter_o = it;
            *zncc_o = NAN;
            return n_valid == 0 ? ST_OOB : ST_INVALID;
        }
        for (int k = 0; k < 12; ++k) b[k] = 0.0;
        double inv_bf = 1.0 / bottomf_d, inv_bg = 1.0 / bottomg, s_cc = 0.0;
        int64_t idx = 0;
        for (int dz = -hz; dz <= hz; dz += stride) {
            double Z = (double)dz;
            int64_t zz = z0 + dz;
            for (int dy = -hy; dy <= hy; dy += stride) {
                double Y = (double)dy;
                int64_t yy = y0 + dy;
                for (int dx = -hx; dx <= hx; dx += stride) {
                    int64_t xx = x0 + dx;
                    double gv = gbuf[idx];
                    if (gv != gv) {
                        idx += 1;
                        continue;
                    }
                    double X = (double)dx;
                    double fd = V(&c->f, zz, yy, xx) - meanf_d;
                    double gd = gv - meang;
                    s_cc += fd * gd;
                    double res = fd * inv_bf - gd * inv_bg;
                    idx += 1;
                    double dfx, dfy, dfz;
                    grad_at(c, zz, yy, xx, &dfx, &dfy, &dfz);
                    double gxv = dfx * res, gyv = dfy * res, gzv = dfz * res;
                    b[0] += gxv * X;
                    b[1] += gxv * Y;
                    b[2] += gxv * Z;
                    b[3] += gyv * X;
                    b[4] += gyv * Y;
                    b[5] += gyv * Z;
                    b[6] += gzv * X;
                    b[7] += gzv * Y;
                    b[8] += gzv * Z;
                    b[9] += gxv;
                    b[10] += gyv;
                    b[11] += gzv;
                }
            }
        }
        double norm_abs = 0.0;
        for (int k = 0; k < 12; ++k) {
            b[k] *= bottomf_d;
            norm_abs += b[k] * b[k];
        }
        norm_abs = sqrt(norm_abs);
        if (!isfinite(norm_abs)) {
            *n_iter_o = it;
            *zncc_o = NAN;
            return ST_NAN;
        }
        if (norm_init < 0.0) norm_init = norm_abs;
        double norm_rel = norm_init > 1e-300 ? norm_abs / norm_init : 0.0;
        zncc = s_cc * inv_bf * inv_bg;
        if (norm_rel < tol || norm_abs < ABS_TOL) {
            *n_iter_o = it;
            *zncc_o = zncc;
            return ST_CONVERGED;
        }
        for (int k = 0; k < 12; ++k) negb[k] = -b[k];
        int use_corr = 0;
        if (noise_gain > 0.0 && n_full > 0.0 && last_dp < NOISE_CORR_STEP) {
            double s2 = (1.0 - zncc > 0.0 ? 1.0 - zncc : 0.0) * bottomf_d * bottomf_d / (double)n_valid;
            double corr = noise_gain * s2 * ((double)n_valid / n_full);
            use_corr = corrected_chol12(H, pattern, corr, H0, L0);
        }
        chol_solve12(use_corr ? L0 : L, negb, dP);
        double dp_norm = 0.0;
        for (int k = 0; k < 9; ++k) {
            double v = dP[k] * half_scale;
            dp_norm += v * v;
        }
        for (int k = 9; k < 12; ++k) dp_norm += dP[k] * dP[k];
        dp_norm = sqrt(dp_norm);
        if (!isfinite(dp_norm)) {
            *n_iter_o = it;
            *zncc_o = NAN;
            return ST_NAN;
        }
        last_dp = dp_norm;
        if (dp_norm < dp_tol) {
            *n_iter_o = it;
            *zncc_o = zncc;
            return ST_CONVERGED;
        }
        if (predictive && dp_prev > 0.0 && dp_norm < PREDICT_CONTRACTION * dp_prev && dp_norm * dp_norm < dp_tol * dp_prev) {
            *n_iter_o = it;
            *zncc_o = zncc;
            if (!orc_compose_warp(P, dP)) return ST_SINGULAR;
            return ST_CONVERGED;
        }
        dp_prev = dp_norm;
        int improved = zncc > best_zncc + STALL_ZNCC_EPS;
        if (improved) {
            best_zncc = zncc;
            for (int k = 0; k < 12; ++k) P_best[k] = P[k];
        }
        if (dp_norm < best_dp * STALL_STEP_DECAY) {
            best_dp = dp_norm;
            improved = 1;
        }
        if (improved)
            stall = 0;
        else {
            stall += 1;
            if (patience > 0 && stall >= patience) {
                for (int k = 0; k < 12; ++k) P[k] = P_best[k];
                *n_iter_o = it;
                *zncc_o = best_zncc;
                return ST_STALLED;
            }
        }
        if (!orc_compose_warp(P, dP)) {
            *n_iter_o = it;
            *zncc_o = zncc;
            return ST_SINGULAR;
        }
    }
    *n_iter_o = max_iter;
    *zncc_o = zncc;
    return ST_MAX_ITER;
}

/* _icgn_12dof_parallel_jit (:795-901).  P_out is filled from P0 first. */
void orc_icgn12(const int64_t *coords, int64_t N, const double *P0, int hx, int hy, int hz, int stride, const float *f,
                const float *gx, const float *gy, const float *gz, int stored, const uint8_t *mask, const float *g, int64_t nz,
                int64_t ny, int64_t nx, int mode, const double *L_all, const uint8_t *valid, double tol, double dp_tol, int max_iter,
                int patience, const double *H_all, const double *pattern, double noise_gain, int predictive,
                const int64_t *split_index, const uint8_t *split_keep, int64_t keep_bytes, double *P_out, int32_t *n_iter,
                int8_t *status, double *zncc) {
    ctx_t c;
    make_ctx(&c, f, gx, gy, gz, stored, mask, g, nz, ny, nx, hx, hy, hz, stride, mode);
    int64_t S = subset_count(hx, hy, hz, stride);
    double zero_pattern[144];
    for (int i = 0; i < 144; ++i) zero_pattern[i] = 0.0;
    if (pattern == NULL || H_all == NULL || noise_gain <= 0.0) {
        pattern = zero_pattern;
        noise_gain = 0.0;
    }
    for (int64_t n = 0; n < N; ++n) {
        for (int k = 0; k < 12; ++k) P_out[n * 12 + k] = P0[n * 12 + k];
        n_iter[n] = 0;
        status[n] = valid[n] ? ST_SKIPPED : ST_INVALID;
        zncc[n] = NAN;
    }
#pragma omp parallel
    {
        double *gbuf = (double *)malloc((size_t)S * sizeof(double));
#pragma omp for schedule(dynamic, 1)
        for (int64_t n = 0; n < N; ++n) {
            if (!valid[n]) continue;
            double *P = P_out + n * 12;
            int finite = 1;
            for (int k = 0; k < 12; ++k)
                if (!isfinite(P[k])) finite = 0;
            if (!finite) {
                status[n] = ST_NAN;
                continue;
            }
            int64_t r = split_index ? split_index[n] : -1;
            int use_keep = r >= 0;
            const uint8_t *keep = use_keep ? split_keep + r * keep_bytes : NULL;
            int it = 0;
            double zc = NAN;
            int st = icgn12_single(&c, P, coords[3 * n], coords[3 * n + 1], coords[3 * n + 2], L_all + n * 144, tol, dp_tol, max_iter,
                                   patience, gbuf, H_all ? H_all + n * 144 : NULL, pattern, noise_gain, predictive, keep, use_keep,
                                   &it, &zc);
            n_iter[n] = it;
            status[n] = (int8_t)st;
            zncc[n] = zc;
        }
        free(gbuf);
    }
}

/* ------------------------------------------------------------------ 3-DOF IC-GN (ADMM subproblem 1)
 * _build_h3 (:910-928), _icgn_3dof_single (:931-1082) */
static int build_h3(const double *H, double bf2, double mu, double corr, double Hinv[3][3]) {
    double H3[3][3], Hd[3][3];
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) H3[i][j] = H[(9 + i) * 12 + 9 + j] * 2.0 / bf2;
        double limit_i = (1.0 - MIN_CORRECTED_FRACTION) * H[(9 + i) * 12 + 9 + i];
        double cc = corr < limit_i ? corr : limit_i;
        H3[i][i] -= cc * 2.0 / bf2;
        H3[i][i] += mu;
    }
    double md = H3[1][1] > H3[2][2] ? H3[1][1] : H3[2][2];
    double max_diag = H3[0][0] > md ? H3[0][0] : md;
    if (!(max_diag > 0.0)) return 0;
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) Hd[i][j] = H3[i][j];
        Hd[i][i] += LM_DAMPING_3DOF * max_diag;
    }
    return inv3(Hd, Hinv) != 0.0;
}

static int icgn3_single(const ctx_t *c, double *P, int64_t x0, int64_t y0, int64_t z0, const double *H, double bottomf,
                        const double *u_old, const double *vdual, double mu, double tol, double dp_tol, int max_iter, int patience,
                        double *gbuf, double n_full, double noise_gain, int predictive, const uint8_t *keep, int use_keep,
                        int *n_iter_o, double *zncc_o) {
    (void)n_full;
    const int hx = c->hx, hy = c->hy, hz = c->hz, stride = c->stride;
    double best_dn = 1e300;
    int stall = 0;
    double bf2 = bottomf * bottomf;
    if (bf2 < 1e-30) bf2 = 1e-30;
    double Hinv[3][3];
    if (!build_h3(H, bf2, mu, 0.0, Hinv)) {
        *n_iter_o = 0;
        *zncc_o = NAN;
        return ST_SINGULAR;
    }
    double last_dn = 1e300, dn_prev = -1.0, norm_init = -1.0, zncc = NAN;
    double b[3], tb[3], dt[3];
    double a00 = 1.0 + P[0], a01 = P[1], a02 = P[2];
    double a10 = P[3], a11 = 1.0 + P[4], a12 = P[5];
    double a20 = P[6], a21 = P[7], a22 = 1.0 + P[8];
    for (int it = 1; it <= max_iter; ++it) {
        int64_t n_valid;
        double meanf_d = 0, bottomf_d = 1, meang = 0, bottomg = 1;
        int ok = warp_and_sample(c, P, x0, y0, z0, gbuf, keep, use_keep, &n_valid, &meanf_d, &bottomf_d, &meang, &bottomg);
        if (!ok) {
            *n_iter_o = it;
            *zncc_o = NAN;
            return n_valid == 0 ? ST_OOB : ST_INVALID;
        }
        b[0] = b[1] = b[2] = 0.0;
        double inv_bf = 1.0 / bottomf_d, inv_bg = 1.0 / bottomg, s_cc = 0.0;
        int64_t idx = 0;
        for (int dz = -hz; dz <= hz; dz += stride) {
            int64_t zz = z0 + dz;
            for (int dy = -hy; dy <= hy; dy += stride) {
                int64_t yy = y0 + dy;
                for (int dx = -hx; dx <= hx; dx += stride) {
                    int64_t xx = x0 + dx;
                    double gv = gbuf[idx];
                    if (gv != gv) {
                        idx += 1;
                        continue;
                    }
                    double fd = V(&c->f, zz, yy, xx) - meanf_d;
                    double gd = gv - meang;
                    s_cc += fd * gd;
                    double res = fd * inv_bf - gd * inv_bg;
                    idx += 1;
                    double dfx, dfy, dfz;
                    grad_at(c, zz, yy, xx, &dfx, &dfy, &dfz);
                    b[0] += dfx * res;
                    b[1] += dfy * res;
                    b[2] += dfz * res;
                }
            }
        }
        double norm_abs = 0.0;
        for (int k = 0; k < 3; ++k) {
            b[k] *= bottomf_d;
            tb[k] = b[k] * 2.0 / bf2 + mu * (P[9 + k] - u_old[k] - vdual[k]);
            norm_abs += tb[k] * tb[k];
        }
        norm_abs = sqrt(norm_abs);
        if (!isfinite(norm_abs)) {
            *n_iter_o = it;
            *zncc_o = NAN;
            return ST_NAN;
        }
        if (norm_init < 0.0) norm_init = norm_abs;
        double norm_rel = norm_init > 1e-300 ? norm_abs / norm_init : 0.0;
        zncc = s_cc * inv_bf * inv_bg;
        if (norm_rel < tol || norm_abs < mu * 1e-4) {
            *n_iter_o = it;
            *zncc_o = zncc;
            return ST_CONVERGED;
        }
        if (noise_gain > 0.0 && last_dn < NOISE_CORR_STEP) {
            double s2 = (1.0 - zncc > 0.0 ? 1.0 - zncc : 0.0) * bottomf_d * bottomf_d / (double)n_valid;
            if (!build_h3(H, bf2, mu, noise_gain * s2 * (double)n_valid, Hinv)) build_h3(H, bf2, mu, 0.0, Hinv);
        }
        for (int i = 0; i < 3; ++i) {
            double s = 0.0;
            for (int j = 0; j < 3; ++j) s += Hinv[i][j] * tb[j];
            dt[i] = -s;
        }
        double dn = sqrt(dt[0] * dt[0] + dt[1] * dt[1] + dt[2] * dt[2]);
        if (!isfinite(dn)) {
            *n_iter_o = it;
            *zncc_o = NAN;
            return ST_NAN;
        }
        last_dn = dn;
        if (dn < dp_tol) {
            *n_iter_o = it;
            *zncc_o = zncc;
            return ST_CONVERGED;
        }
        if (predictive && dn_prev > 0.0 && dn < PREDICT_CONTRACTION * dn_prev && dn * dn < dp_tol * dn_prev) {
            P[9] -= a00 * dt[0] + a01 * dt[1] + a02 * dt[2];
            P[10] -= a10 * dt[0] + a11 * dt[1] + a12 * dt[2];
            P[11] -= a20 * dt[0] + a21 * dt[1] + a22 * dt[2];
            *n_iter_o = it;
            *zncc_o = zncc;
            return ST_CONVERGED;
        }
        dn_prev = dn;
        if (dn < best_dn * STALL_STEP_DECAY) {
            best_dn = dn;
            stall = 0;
        } else {
            stall += 1;
            if (patience > 0 && stall >= patience) {
                *n_iter_o = it;
                *zncc_o = zncc;
                return ST_STALLED;
            }
        }
        P[9] -= a00 * dt[0] + a01 * dt[1] + a02 * dt[2];
        P[10] -= a10 * dt[0] + a11 * dt[1] + a12 * dt[2];
        P[11] -= a20 * dt[0] + a21 * dt[1] + a22 * dt[2];
    }
    *n_iter_o = max_iter;
    *zncc_o = zncc;
    return ST_MAX_ITER;
}

/* _icgn_3dof_parallel_jit (:1085-1208) */
void orc_icgn3(const int64_t *coords, int64_t N, const double *U_old, const double *F_fixed, const double *vdual, int hx, int hy,
               int hz, int stride, const float *f, const float *gx, const float *gy, const float *gz, int stored, const uint8_t *mask,
               const float *g, int64_t nz, int64_t ny, int64_t nx, int mode, const double *H_all, const double *bottomf_all,
               const uint8_t *valid, double mu, double tol, double dp_tol, int max_iter, int patience, double n_full,
               double noise_gain, int predictive, const int64_t *split_index, const uint8_t *split_keep, int64_t keep_bytes,
               double *U_out, int32_t *n_iter, int8_t *status, double *zncc) {
    ctx_t c;
    make_ctx(&c, f, gx, gy, gz, stored, mask, g, nz, ny, nx, hx, hy, hz, stride, mode);
    int64_t S = subset_count(hx, hy, hz, stride);
    for (int64_t n = 0; n < N; ++n) {
        for (int k = 0; k < 3; ++k) U_out[n * 3 + k] = U_old[n * 3 + k];
        n_iter[n] = 0;
        status[n] = valid[n] ? ST_SKIPPED : ST_INVALID;
        zncc[n] = NAN;
    }
#pragma omp parallel
    {
        double *gbuf = (double *)malloc((size_t)S * sizeof(double));
#pragma omp for schedule(dynamic, 1)
        for (int64_t n = 0; n < N; ++n) {
            if (!valid[n]) continue;
            double P[12];
            int finite = 1;
            for (int k = 0; k < 9; ++k) {
                P[k] = F_fixed[n * 9 + k];
                if (!isfinite(P[k])) finite = 0;
            }
            for (int k = 0; k < 3; ++k) {
                P[9 + k] = U_old[n * 3 + k];
                if (!isfinite(P[9 + k])) finite = 0;
            }
            if (!finite) {
                status[n] = ST_NAN;
                continue;
            }
            int64_t r = split_index ? split_index[n] : -1;
            int use_keep = r >= 0;
            const uint8_t *keep = use_keep ? split_keep + r * keep_bytes : NULL;
            int it = 0;
            double zc = NAN;
            int st = icgn3_single(&c, P, coords[3 * n], coords[3 * n + 1], coords[3 * n + 2], H_all + n * 144, bottomf_all[n],
                                  U_old + n * 3, vdual + n * 3, mu, tol, dp_tol, max_iter, patience, gbuf, n_full, noise_gain,
                                  predictive, keep, use_keep, &it, &zc);
            for (int k = 0; k < 3; ++k) U_out[n * 3 + k] = P[9 + k];
            n_iter[n] = it;
            status[n] = (int8_t)st;
            zncc[n] = zc;
        }
        free(gbuf);
    }
}

/* ------------------------------------------------------------------ direct ZNCC map
 * integer_search._zncc_direct (:44-151).  out is (N, 2rz+1, 2ry+1, 2rx+1). */
void orc_zncc_direct(const float *f, const float *g, int64_t nz, int64_t ny, int64_t nx, const int64_t *coords, int64_t N, int hx,
                     int hy, int hz, int rx, int ry, int rz, const int64_t *wx0, const int64_t *wy0, const int64_t *wz0,
                     const uint8_t *t_ok, double *out) {
    const int64_t sx = 2 * hx + 1, sy = 2 * hy + 1, sz = 2 * hz + 1;
    const int64_t vx = 2 * rx + 1, vy = 2 * ry + 1, vz = 2 * rz + 1;
    const int64_t wx = sx + 2 * rx, wy = sy + 2 * ry, wz = sz + 2 * rz;
    const double n_tpl = (double)(sx * sy * sz);
    const int64_t nmap = vz * vy * vx;
    vol_t F = {f, nz, ny, nx}, G = {g, nz, ny, nx};
#pragma omp parallel
    {
        double *T = (double *)malloc((size_t)(sx * sy * sz) * sizeof(double));
        int64_t sat_n = (wz + 1) * (wy + 1) * (wx + 1);
        double *S1 = (double *)malloc((size_t)sat_n * sizeof(double));
        double *S2 = (double *)malloc((size_t)sat_n * sizeof(double));
#define SAT(A, z, y, x) A[((z) * (wy + 1) + (y)) * (wx + 1) + (x)]
#pragma omp for schedule(dynamic, 1)
        for (int64_t n = 0; n < N; ++n) {
            double *o = out + n * nmap;
            if (!t_ok[n]) {
                for (int64_t i = 0; i < nmap; ++i) o[i] = -2.0;
                continue;
            }
            int64_t x0 = coords[3 * n], y0 = coords[3 * n + 1], z0 = coords[3 * n + 2];
            double sf = 0.0;
            for (int64_t k = 0; k < sz; ++k)
                for (int64_t j = 0; j < sy; ++j)
                    for (int64_t i = 0; i < sx; ++i) {
                        double v = V(&F, z0 - hz + k, y0 - hy + j, x0 - hx + i);
                        T[(k * sy + j) * sx + i] = v;
                        sf += v;
                    }
            double mf = sf / n_tpl, ssf = 0.0;
            for (int64_t i = 0; i < sx * sy * sz; ++i) {
                T[i] -= mf;
                ssf += T[i] * T[i];
            }
            if (ssf < 1e-20) {
                for (int64_t i = 0; i < nmap; ++i) o[i] = -2.0;
                continue;
            }
            for (int64_t i = 0; i < sat_n; ++i) S1[i] = S2[i] = 0.0;
            int64_t zb = wz0[n], yb = wy0[n], xb = wx0[n];
            for (int64_t z = 0; z < wz; ++z)
                for (int64_t y = 0; y < wy; ++y) {
                    double r1 = 0.0, r2 = 0.0;
                    for (int64_t x = 0; x < wx; ++x) {
                        float v32 = VF(&G, zb + z, yb + y, xb + x);
                        r1 += (double)v32;
                        r2 += SQ32(v32);
                        SAT(S1, z + 1, y + 1, x + 1) = SAT(S1, z, y + 1, x + 1) + SAT(S1, z + 1, y, x + 1) - SAT(S1, z, y, x + 1) + r1;
                        SAT(S2, z + 1, y + 1, x + 1) = SAT(S2, z, y + 1, x + 1) + SAT(S2, z + 1, y, x + 1) - SAT(S2, z, y, x + 1) + r2;
                    }
                }
            for (int64_t dz = 0; dz < vz; ++dz)
                for (int64_t dy = 0; dy < vy; ++dy)
                    for (int64_t dx = 0; dx < vx; ++dx) {
                        int64_t z1 = dz + sz, y1 = dy + sy, x1 = dx + sx;
                        double sg = SAT(S1, z1, y1, x1) - SAT(S1, dz, y1, x1) - SAT(S1, z1, dy, x1) - SAT(S1, z1, y1, dx) +
                                    SAT(S1, dz, dy, x1) + SAT(S1, dz, y1, dx) + SAT(S1, z1, dy, dx) - SAT(S1, dz, dy, dx);
                        double sgg = SAT(S2, z1, y1, x1) - SAT(S2, dz, y1, x1) - SAT(S2, z1, dy, x1) - SAT(S2, z1, y1, dx) +
                                     SAT(S2, dz, dy, x1) + SAT(S2, dz, y1, dx) + SAT(S2, z1, dy, dx) - SAT(S2, dz, dy, dx);
                        double var = sgg - sg * sg / n_tpl;
                        double *dst = o + (dz * vy + dy) * vx + dx;
                        if (var < 1e-20) {
                            *dst = 0.0;
                            continue;
                        }
                        double sfg = 0.0;
                        for (int64_t k = 0; k < sz; ++k)
                            for (int64_t j = 0; j < sy; ++j)
                                for (int64_t i = 0; i < sx; ++i)
                                    sfg += T[(k * sy + j) * sx + i] * V(&G, zb + dz + k, yb + dy + j, xb + dx + i);
                        double val = sfg / sqrt(var * ssf);
                        if (val > 1.0)
                            val = 1.0;
                        else if (val < -1.0)
                            val = -1.0;
                        *dst = val;
                    }
        }
#undef SAT
        free(T);
        free(S1);
        free(S2);
    }
}

/* ------------------------------------------------------------------ window box statistics of the FFT engine
 * integer_search._window_box_stats (:154-207): per node of W (N, wz, wy, wx) float32, the sums of W and of
 * its float32 squares over every (sz, sy, sx) box, from an FP64 summed-area table built row by row in the
 * reference's order; out_sum / out_sq are (N, wz-sz+1, wy-sy+1, wx-sx+1). */
void orc_window_box_stats(const float *W, int64_t N, int64_t wz, int64_t wy, int64_t wx, int64_t sz, int64_t sy, int64_t sx,
                          double *out_sum, double *out_sq) {
    const int64_t vz = wz - sz + 1, vy = wy - sy + 1, vx = wx - sx + 1;
    const int64_t sat_n = (wz + 1) * (wy + 1) * (wx + 1);
#pragma omp parallel
    {
        double *S1 = (double *)malloc((size_t)sat_n * sizeof(double));
        double *S2 = (double *)malloc((size_t)sat_n * sizeof(double));
#define SAT(A, z, y, x) A[((z) * (wy + 1) + (y)) * (wx + 1) + (x)]
#pragma omp for schedule(dynamic, 1)
        for (int64_t n = 0; n < N; ++n) {
            const float *w = W + n * wz * wy * wx;
            for (int64_t i = 0; i < sat_n; ++i) S1[i] = S2[i] = 0.0;
            for (int64_t z = 0; z < wz; ++z)
                for (int64_t y = 0; y < wy; ++y) {
                    double r1 = 0.0, r2 = 0.0;
                    for (int64_t x = 0; x < wx; ++x) {
                        float v32 = w[(z * wy + y) * wx + x];
                        r1 += (double)v32;
                        r2 += SQ32(v32);
                        SAT(S1, z + 1, y + 1, x + 1) = SAT(S1, z, y + 1, x + 1) + SAT(S1, z + 1, y, x + 1) - SAT(S1, z, y, x + 1) + r1;
                        SAT(S2, z + 1, y + 1, x + 1) = SAT(S2, z, y + 1, x + 1) + SAT(S2, z + 1, y, x + 1) - SAT(S2, z, y, x + 1) + r2;
                    }
                }
            double *os = out_sum + n * vz * vy * vx, *oq = out_sq + n * vz * vy * vx;
            for (int64_t z = 0; z < vz; ++z)
                for (int64_t y = 0; y < vy; ++y)
                    for (int64_t x = 0; x < vx; ++x) {
                        int64_t z1 = z + sz, y1 = y + sy, x1 = x + sx, o = (z * vy + y) * vx + x;
                        os[o] = SAT(S1, z1, y1, x1) - SAT(S1, z, y1, x1) - SAT(S1, z1, y, x1) - SAT(S1, z1, y1, x) + SAT(S1, z, y, x1) +
                                SAT(S1, z, y1, x) + SAT(S1, z1, y, x) - SAT(S1, z, y, x);
                        oq[o] = SAT(S2, z1, y1, x1) - SAT(S2, z, y1, x1) - SAT(S2, z1, y, x1) - SAT(S2, z1, y1, x) + SAT(S2, z, y, x1) +
                                SAT(S2, z, y1, x) + SAT(S2, z1, y, x) - SAT(S2, z, y, x);
                    }
        }
#undef SAT
        free(S1);
        free(S2);
    }
}

/* ------------------------------------------------------------------ ZNSSD cost
 * C = sum_v r_v^2 with the residual of _icgn_12dof_single (numba_kernels.py:705-708),
 * r = (float(f) - meanf) / bottomf - (g - meang) / bottomg, over the valid set and with the statistics of
 * _warp_and_sample (:586-598).  FP64; the checker of the differentiable ZNSSD kernels (their forward, and
 * central differences for their backward).  No mask, no keep bits.  NaN where the warp leaves the
 * admissible domain or the valid set is too small. */
void orc_znssd(const float *f, const float *g, int64_t nz, int64_t ny, int64_t nx, const int64_t *coords, int64_t N, int hx,
               int hy, int hz, int mode, const double *P_all, double *cost) {
    ctx_t c;
    make_ctx(&c, f, NULL, NULL, NULL, 0, NULL, g, nz, ny, nx, hx, hy, hz, 1, mode);
    int64_t S = subset_count(hx, hy, hz, 1);
#pragma omp parallel
    {
        double *gbuf = (double *)malloc((size_t)S * sizeof(double));
#pragma omp for schedule(dynamic, 1)
        for (int64_t n = 0; n < N; ++n) {
            const int64_t x0 = coords[3 * n], y0 = coords[3 * n + 1], z0 = coords[3 * n + 2];
            int64_t nv;
            double mf, bf, mg, bg;
            cost[n] = NAN;
            if (!warp_and_sample(&c, P_all + 12 * n, x0, y0, z0, gbuf, NULL, 0, &nv, &mf, &bf, &mg, &bg)) continue;
            const double ibf = 1.0 / bf, ibg = 1.0 / bg;
            double s = 0.0;
            int64_t idx = 0;
            for (int dz = -hz; dz <= hz; ++dz)
                for (int dy = -hy; dy <= hy; ++dy)
                    for (int dx = -hx; dx <= hx; ++dx, ++idx) {
                        const double gv = gbuf[idx];
                        if (gv != gv) continue;
                        const double fd = (double)VF(&c.f, z0 + dz, y0 + dy, x0 + dx) - mf;
                        const double r = fd * ibf - (gv - mg) * ibg;
                        s += r * r;
                    }
            cost[n] = s;
        }
        free(gbuf);
    }
}

/* ---------------------------------------------------------------- separable volume filters
 * The two whole-volume filters the reference runs before the local step, both scipy.ndimage calls
 * (scipy >= 1.10 per the reference's pyproject; 1.18.1 here), restated as one symmetric FIR along
 * one axis with FP64 accumulation and float32 output per axis:
 *   io/volume_ops.py:215-222 prefilter_bspline = spline_filter(order 3, mode "mirror"): the inverse of
 *     the cubic B-spline sampling filter (z + 4 + 1/z) / 6 on the mirror-symmetric extension of each line,
 *     whose impulse response is sqrt(3) z^|j|, z = sqrt(3) - 2 (Unser, Aldroubi & Eden, IEEE TSP 1993);
 *     |z|^33 < 2e-19, so 32 taps each side reach FP64 resolution;
 *   io/volume_ops.py:200-212 presmooth_volume = gaussian_filter(mode "nearest"): the normalised Gaussian
 *     of radius int(4 sigma + 0.5), edge samples repeated.
 * out[k] = w[0] s[k] + sum_{j=1..J} w[j] (s[k-j] + s[k+j]) in that order, no fused multiply-add. */
static inline int64_t reflect_index(int64_t k, int64_t n, int boundary) {
    if (boundary == 1) return k < 0 ? 0 : (k >= n ? n - 1 : k); /* nearest */
    if (n == 1) return 0;
    const int64_t p = 2 * n - 2; /* mirror: period 2n - 2, edge samples not repeated */
    k %= p;
    if (k < 0) k += p;
    return k < n ? k : p - k;
}

void orc_sep_filter(const float *in, float *out, int64_t nz, int64_t ny, int64_t nx, int axis, const double *w, int J,
                    int boundary) {
    const int64_t n = axis == 0 ? nx : (axis == 1 ? ny : nz);
    const int64_t stride = axis == 0 ? 1 : (axis == 1 ? nx : nx * ny);
    const int64_t total = nz * ny * nx;
    if (boundary == 0 && n == 1) { /* a mirrored line of one sample is its own coefficient */
        memcpy(out, in, (size_t)total * sizeof(float));
        return;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < total; ++i) {
        const int64_t k = (i / stride) % n;
        const float *line = in + (i - k * stride);
        double acc = w[0] * (double)line[k * stride];
        for (int j = 1; j <= J; ++j) {
            const double a = (double)line[reflect_index(k - j, n, boundary) * stride];
            const double b = (double)line[reflect_index(k + j, n, boundary) * stride];
            acc = acc + w[j] * (a + b);
        }
        out[i] = (float)acc;
    }
}
