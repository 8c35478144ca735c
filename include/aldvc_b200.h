/*
 * aldvc_b200 -- C ABI of the B200 (sm_100a) AL-DVC hot-path library.
 *
 * Every entry point takes device pointers, sizes and a cudaStream_t (passed
 * as void*), enqueues its work on that stream and returns an int: 0 on
 * success, a negative code on an argument or CUDA error (the message is in
 * aldvc_last_error()).  Numerical failures of single nodes are never errors:
 * they are per-node status codes, as in the reference.  Nothing here
 * allocates device memory except where a function says so; scratch memory
 * is a caller-provided workspace sized by the matching *_workspace_size().
 *
 * Reference interfaces replaced (pyALDVC v1.2.1, src/al_dvc/...):
 *   aldvc_precompute  <- solver/cuda_kernels.py:1635 precompute_nodes_cuda
 *   aldvc_precompute_grid <- the same on a tensor node grid, separable moment sums
 *                        (contract of solver/numba_kernels.py:499 precompute_nodes)
 *   aldvc_icgn12      <- solver/cuda_kernels.py:1397 icgn_12dof_cuda
 *                        (contract of solver/numba_kernels.py:1211 icgn_12dof_parallel)
 *   aldvc_icgn3       <- solver/cuda_kernels.py:1518 icgn_3dof_cuda
 *                        (contract of solver/numba_kernels.py:1281 icgn_3dof_parallel)
 *   aldvc_ncc_map     <- solver/cuda_kernels.py:1713 zncc_direct_cuda
 *                        (contract of solver/integer_search.py:44 _zncc_direct)
 *   aldvc_ncc_search  <- solver/integer_search.py:329 ncc_search (map, argmax, PCE,
 *                        clipped flag and sub-voxel refinement on the device)
 *   aldvc_global_rhs  <- solver/subpb2_solver.py:111 global_rhs
 *   aldvc_pcg_hex8    <- solver/subpb2_solver.py:77 pcg_multi over
 *                        solver/subpb2_solver.py:45 build_global_system (hex8 FEM)
 *   aldvc_nodal_gradient <- solver/global_operators.py:151 nodal_gradient (FEM)
 *   aldvc_znssd_forward / _backward: no reference counterpart (the residual of numba_kernels.py:705-708
 *                        with a hand-written gradient)
 *   aldvc_gradients   <- io/volume_ops.py:124 _gradient_stencil7
 *   aldvc_normalize   <- io/volume_ops.py:105 normalize_volume (whole volume)
 *   aldvc_sep_filter  <- io/volume_ops.py:215 prefilter_bspline (scipy spline_filter, order 3,
 *                        mirror) and :200 presmooth_volume (scipy gaussian_filter, nearest),
 *                        one axis per call
 *   aldvc_volume_stats / aldvc_normalize_voi <- io/volume_ops.py:74 voi_mean_std,
 *                        :105 normalize_volume with a VOI box
 *   aldvc_volume_moments / aldvc_normalize_sums <- io/volume_ops.py:80-121 voi_mean_std +
 *                        normalize_volume of a volume streamed from host memory slab by slab
 *                        (the tiled pass; solver/tiling.py:292 ReferenceSource serves its boxes)
 *   aldvc_block_downsample <- solver/integer_search.py:235 block_downsample
 *   aldvc_phase_correlation <- solver/integer_search.py:247 phase_correlation_shift (after the
 *                        VOI crop and the block downsampling, which the caller does)
 *   aldvc_gradient_plane_fit <- strain/gradient_methods.py:151 gradient_plane_fit (no cut mesh)
 *   aldvc_gradient_fd <- strain/gradient_methods.py:231 gradient_fd (no cut mesh)
 *   aldvc_grid_smooth <- utils/grid_interp.py:54 smooth_grid_field
 *   aldvc_grid_interp <- utils/grid_interp.py:18 interp_grid_field (the cumulative displacements of a
 *                        frame series, core/pipeline.py:455-491)
 *   aldvc_displacement_uncertainty <- solver/uncertainty.py:94 displacement_uncertainty
 *   aldvc_strain_measures <- strain/strain_types.py:19-114 (strain_tensor, principal_strains,
 *                        von_mises_strain, max_shear_strain, volumetric_strain,
 *                        det_deformation_gradient, polar_rotation_deg)
 *   aldvc_mask_fill   <- io/volume_ops.py:225 prepare_deformed (masked voxels -> NaN) and the
 *                        NCC input of core/pipeline.py:260-262 (masked voxels -> 0)
 *   aldvc_inpaint     <- utils/inpaint.py:35 fill_nan_grid ("spring" model, no cut mesh)
 *   aldvc_median_test <- utils/outlier_detection.py:135 universal_median_test (no cut mesh)
 *   aldvc_render_beads   synthetic Gaussian-bead volumes (inputs of the benchmark configurations;
 *                        pyALDVC synthetic.py:37 generate_bead_volume is the counterpart)
 */
#ifndef ALDVC_B200_H
#define ALDVC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ALDVC_ABI_VERSION 1

/* status codes of a node (pyALDVC core/data_structures.py:26-43) */
#define ALDVC_CONVERGED 0
#define ALDVC_MAX_ITER 1
#define ALDVC_OUT_OF_BOUNDS 2
#define ALDVC_INVALID_SUBSET 3
#define ALDVC_SINGULAR 4
#define ALDVC_NAN 5
#define ALDVC_SKIPPED 6
#define ALDVC_STALLED 7

/* error codes returned by the entry points */
#define ALDVC_OK 0
#define ALDVC_ERR_ARG -1
#define ALDVC_ERR_CUDA -2
#define ALDVC_ERR_WORKSPACE -3
#define ALDVC_ERR_UNSUPPORTED -4

/* IC-GN kernel variants */
#define ALDVC_BATCHED 0 /* persistent work-queue kernel, subset bricks in shared memory */
#define ALDVC_PLAIN 1   /* one node per block, two passes through a global sample buffer */

/* Reference frame and deformed frame of one correlation (all device pointers). */
typedef struct aldvc_volumes {
    const float *f;       /* reference volume (nz, ny, nx) */
    const float *gx;      /* reference gradients (nz, ny, nx); NULL: 7-point stencil on f in the kernels */
    const float *gy;
    const float *gz;
    const uint8_t *mask;  /* reference mask (nz, ny, nx), 0 = not material; NULL: every voxel counts */
    const float *g;       /* deformed volume prepared for the interpolation mode; NaN voxels are excluded */
    int64_t nz, ny, nx;
    const float *g4;      /* optional (may be NULL): g as overlapping quads, 4 floats per voxel i = g[i..i+3]
                             (aldvc_make_quads); the persistent IC-GN kernels then read each cubic tap row with
                             one 16-byte load */
} aldvc_volumes;

/* Subset geometry of a call: one shape for every node, or per-node (uneven, anisotropic) shapes. */
typedef struct aldvc_subset {
    int32_t hx, hy, hz;          /* half-widths (winsize // 2); with node_half, the largest over the nodes */
    int32_t stride;              /* sample every stride-th voxel per axis (>= 1) */
    int32_t mode;                /* 0 trilinear, 1 Keys cubic (a = -0.5), 2 cubic B-spline on prefiltered g */
    int32_t reserved;
    const int64_t *split_index;  /* (N,) row of split_keep per node, -1 = whole subset; NULL: no splitting */
    const uint8_t *split_keep;   /* (rows, keep_bytes) packed keep bits in sampling order */
    int64_t keep_bytes;
    /* (N,3) int32 [hx, hy, hz] per node, each <= (hx, hy, hz) above; NULL: every node takes (hx, hy, hz).
     * Not combined with split rows or the noise-corrected Hessian.  The reference calls its kernels once per
     * subset shape; here one persistent launch takes every shape. */
    const int32_t *node_half;
} aldvc_subset;

/* IC-GN controls (pyALDVC core/config.py:76-95 field meanings). */
typedef struct aldvc_icgn_params {
    double tol;           /* relative gradient-norm tolerance (icgn_tol) */
    double dp_tol;        /* parameter-increment tolerance in voxels (icgn_dp_tol) */
    int32_t max_iter;     /* icgn_max_iter */
    int32_t patience;     /* icgn_patience, 0 disables the stall rule */
    double noise_gain;    /* > 0 (with H_all and pattern): noise-corrected Hessian steps */
    int32_t predictive;   /* icgn_predictive_stop */
    int32_t variant;      /* ALDVC_BATCHED or ALDVC_PLAIN */
    int32_t threads;      /* threads per block: 0 = library default */
    int32_t brick_floats; /* batched: shared-memory brick capacity in floats, 0 = library default */
    double mu;            /* 3-DOF: ADMM penalty */
    double n_full;        /* 3-DOF: sampled voxels of a full subset (noise-correction scale) */
    int32_t sweep_rows;   /* persistent form with threads <= 128: subset rows per sweep tile (each tile swept plane by
                             plane), 0 = library default (a tile height of 3-6 rows that pads the fewest rows),
                             < 0 = the whole subset in C order */
    int32_t reserved;
    const int32_t *node_order; /* persistent forms: (N,) a permutation of 0..N-1, the order in which the work queue
                                  hands out the nodes (nodes solved at the same time share more of the volume in L2
                                  when they are near each other); entries outside 0..N-1 are skipped; NULL: 0..N-1 */
} aldvc_icgn_params;

/* Uniform hex8 node grid of the global step, node n = iz*ny*nx + iy*nx + ix. */
typedef struct aldvc_hex8_mesh {
    int64_t nx, ny, nz;            /* nodes per axis */
    double sx, sy, sz;             /* node spacing (element edge lengths) */
    const uint8_t *elem_active;    /* ((nz-1)(ny-1)(nx-1),) 1 = element kept; NULL: all kept */
    int32_t gauss_order;           /* 1, 2 or 3 */
    int32_t reserved;
} aldvc_hex8_mesh;

/* ---------------------------------------------------------------- library */
int aldvc_abi_version(void);
const char *aldvc_last_error(void);
/* kernels this library has launched in the process so far (a monotone counter) */
unsigned long long aldvc_launch_count(void);

/* Kernel timing for callers that measure a region (no reference counterpart): while enabled, the library
 * records CUDA events on the launch stream around each launch of its main kernels (none on a stream under
 * capture).  aldvc_kernel_timing(1) clears the records and starts, (0) clears and stops.  _read waits for
 * the recorded events and writes, per kernel name in first-launch order, the total device milliseconds and
 * the launch count (names: max_entries rows of name_len bytes); returns the number of distinct kernels. */
int aldvc_kernel_timing(int enable);
int aldvc_kernel_timing_read(int32_t max_entries, char *names, int32_t name_len, double *ms, int64_t *launches);
/* Test hook of the bounded grid-barrier waits (no reference counterpart).  The cooperative kernels (PCG,
 * inpainting) wait at their grid barriers for the launch's blocks plus `extra_arrivals` (default 0) and give
 * up after `spin_limit` polls of about 64 ns each (default 2^24; <= 0 restores it), setting their error word
 * and returning.  With extra_arrivals > 0 no barrier ever opens, so every wait runs out: the failure path of
 * a barrier whose peer never arrives, exercised without faulting or hanging the GPU.  Applies to launches
 * enqueued after the call, process-wide; for tests only. */
int aldvc_test_set_barrier(int32_t extra_arrivals, int64_t spin_limit);
/* name of device `device`, its SM count and compute capability; returns ALDVC_OK */
int aldvc_device_info(int device, char *name, int name_len, int *sm_count, int *cc_major, int *cc_minor);

/* ---------------------------------------------------------------- volume preprocessing */
/* 7-point central-difference gradients, zero within `border` voxels of a face */
int aldvc_gradients(const float *f, int64_t nz, int64_t ny, int64_t nx, int32_t border, float *gx, float *gy, float *gz,
                    void *stream);

/* (v - mean) / std of a whole float32 (is_uint16 == 0) or uint16 volume, FP64 statistics taken
 * relative to `pilot` (the reference uses the centre voxel); stats (device, 2 doubles, may be NULL)
 * receives mean and std */
size_t aldvc_normalize_workspace_size(void);
int aldvc_normalize(const void *vol, int32_t is_uint16, int64_t n_voxels, double pilot, float *out, double *stats,
                    void *workspace, size_t workspace_bytes, void *stream);

/* One axis (0 = x, 1 = y, 2 = z) of a symmetric FIR over a float32 volume:
 *   out[k] = w[0] s[k] + sum_{j=1..half_taps} w[j] (s[k-j] + s[k+j])
 * FP64 products and sums in that order (no fused multiply-add), rounded to float32.  boundary 0 = mirror
 * (period 2n - 2; a line of one sample is copied), 1 = nearest.  weights: HOST array of half_taps + 1
 * doubles, half_taps <= 63.  in != out; nz, ny <= 65535.  The cubic B-spline prefilter is the three axes
 * z, y, x in turn with w[j] = sqrt(3) (sqrt(3) - 2)^j, half_taps 32, mirror. */
int aldvc_sep_filter(const float *in, float *out, int64_t nz, int64_t ny, int64_t nx, int32_t axis, const double *weights,
                     int32_t half_taps, int32_t boundary, void *stream);

/* Mean and population standard deviation (device stats[2], FP64) of the float32 (is_uint16 == 0) or uint16
 * volume over the box[6] = {z0, z1, y0, y1, x0, x1} (host array, half-open; NULL = whole volume), moments
 * taken relative to `pilot` (the reference uses the box's centre voxel). */
size_t aldvc_stats_workspace_size(void);
int aldvc_volume_stats(const void *vol, int32_t is_uint16, int64_t nz, int64_t ny, int64_t nx, const int64_t *box, double pilot,
                       double *stats, void *workspace, size_t workspace_bytes, void *stream);
/* aldvc_volume_stats over the box, then (v - mean) / std over the WHOLE volume into out (std < 1e-12 -> 1) */
int aldvc_normalize_voi(const void *vol, int32_t is_uint16, int64_t nz, int64_t ny, int64_t nx, const int64_t *box, double pilot,
                        float *out, double *stats, void *workspace, size_t workspace_bytes, void *stream);
/* FP64 sums of (v - pilot) and (v - pilot)^2 over n_voxels of a float32 or uint16 array, ADDED to sums (device,
 * 2 doubles, zeroed by the caller before the first slab): a volume that does not fit the device is streamed
 * through in slabs and its moments accumulated (workspace: aldvc_normalize_workspace_size() bytes) */
int aldvc_volume_moments(const void *vol, int32_t is_uint16, int64_t n_voxels, double pilot, double *sums, void *workspace,
                         size_t workspace_bytes, void *stream);
/* (v - mean) / std of n_voxels into out (float32), mean and std from the accumulated sums of n_total voxels
 * about pilot (std < 1e-12 -> 1): one box of a streamed volume normalised with the whole volume's statistics;
 * stats (device, 2 doubles, may be NULL) receives mean and std */
int aldvc_normalize_sums(const void *vol, int32_t is_uint16, int64_t n_voxels, const double *sums, int64_t n_total, double pilot,
                         float *out, double *stats, void *stream);

/* Block means of factor^3 voxels (FP64 sums, float32 out); out is (nz/factor, ny/factor, nx/factor), the
 * trailing voxels of each axis dropped. */
int aldvc_block_downsample(const float *in, int64_t nz, int64_t ny, int64_t nx, int32_t factor, float *out, void *stream);

/* Phase correlation of two equal-shape float32 volumes (each axis <= 1024): both centred on their mean and
 * multiplied by a separable Hann window, cross-power spectrum G conj(F) / |G conj(F)|, inverse transform; peak
 * (device int64) receives the flat C-order index of the first maximum of its real part.  The shift along an
 * axis of length n is the peak coordinate p, or p - n when p > n / 2.  Transforms are direct FP64 DFTs. */
size_t aldvc_phase_correlation_workspace_size(int64_t nz, int64_t ny, int64_t nx);
int aldvc_phase_correlation(const float *fs, const float *gs, int64_t nz, int64_t ny, int64_t nx, int64_t *peak, void *workspace,
                            size_t workspace_bytes, void *stream);

/* quads[4 i + k] = vol[min(i + k, n - 1)], k = 0..3: the overlapping-quad copy of a volume read by the IC-GN
 * kernels through aldvc_volumes.g4 (16 bytes per voxel) */
int aldvc_make_quads(const float *vol, int64_t n_voxels, float *quads, void *stream);

/* vol[i] = value wherever mask[i] == 0 (mask: uint8, same voxel count) */
int aldvc_mask_fill(float *vol, const uint8_t *mask, int64_t n_voxels, float value, void *stream);

/* adds peak * exp(-|x - c|^2 / (2 sigma^2)) of every bead (centres (B,3) [z,y,x]) within `radius`
 * voxels into the FP64 accumulator volume (nz, ny, nx) */
int aldvc_render_beads(double *accum, int64_t nz, int64_t ny, int64_t nx, const double *centres_zyx, const double *peaks,
                       int64_t n_beads, double sigma, int32_t radius, void *stream);

/* ---------------------------------------------------------------- strain on the node grid (FP64) */
/* Displacement gradient F (N, 9) row-major, F[c][j] = du_c/dx_j in units of the node spacing (hx, hy, hz), of the
 * (N, 3) field U on the (nz, ny, nx) grid; valid (N,) uint8 or NULL (non-finite U is invalid too).  Invalid
 * nodes get NaN.  complete (N,) = the stencil was whole. */
int aldvc_gradient_plane_fit(const double *U, const uint8_t *valid, int64_t nz, int64_t ny, int64_t nx, double hx, double hy,
                             double hz, int32_t rx, int32_t ry, int32_t rz, double *F, uint8_t *complete, void *stream);
int aldvc_gradient_fd(const double *U, const uint8_t *valid, int64_t nz, int64_t ny, int64_t nx, double hx, double hy, double hz,
                      double *F, uint8_t *complete, void *stream);
/* Normalised Gaussian smoothing of an (nz, ny, nx) FP64 grid field: taps weights[0..half_taps] (HOST array),
 * edge repeat, NaN / invalid nodes neither give nor take weight and come back NaN. */
size_t aldvc_grid_smooth_workspace_size(int64_t nz, int64_t ny, int64_t nx);
int aldvc_grid_smooth(const double *field, const uint8_t *valid, int64_t nz, int64_t ny, int64_t nx, const double *weights,
                      int32_t half_taps, double *out, void *workspace, size_t workspace_bytes, void *stream);

/* An (nz, ny, nx, C) FP64 node-grid field at M points (M, 3) [x, y, z] (voxels; node (iz, iy, ix) sits at
 * (ox + ix hx, oy + iy hy, oz + iz hz)) into out (M, C), FP64.  order 1: trilinear, taps clamped to the grid.
 * order 3: cubic B-spline of the coefficient grid op_z (op_y (op_x field)), op_a an (n_a + pad_a) x n_a FP64 device
 * matrix (the caller's padding and prefilter along that axis; node 0 at coefficient index pad_a / 2), taps clamped
 * to the coefficient grid; workspace aldvc_grid_interp_workspace_size bytes (order 3 only). */
size_t aldvc_grid_interp_workspace_size(int64_t nz, int64_t ny, int64_t nx, int32_t C, int32_t pad_x, int32_t pad_y, int32_t pad_z);
int aldvc_grid_interp(const double *field, int64_t nz, int64_t ny, int64_t nx, int32_t C, const double *op_x, const double *op_y,
                      const double *op_z, int32_t pad_x, int32_t pad_y, int32_t pad_z, double ox, double oy, double oz, double hx,
                      double hy, double hz, const double *points, int64_t M, int32_t order, double *out, void *workspace,
                      size_t workspace_bytes, void *stream);
/* Standard deviation (N, 3) of u, v, w in voxels from the IC-GN normal equations (noise-corrected two-term
 * model): H (N, 12, 12) stored Hessians, zncc, status (NULL: every node), valid, n_valid, bottomf per node (device);
 * pattern: HOST 12 x 12 expectation of sum J J^T for unit gradient noise over the subset (pattern[9][9] its voxel
 * count), gain: the gradient stencil's variance gain, min_frac: the share of each translation diagonal the
 * correction keeps.  NaN at nodes that are not converged, valid, with a finite ZNCC and more than 14 voxels. */
int aldvc_displacement_uncertainty(const double *H, const double *zncc, const int8_t *status, const uint8_t *valid,
                                   const int64_t *n_valid, const double *bottomf, int64_t n_nodes, const double *pattern, double gain,
                                   double min_frac, int32_t noise_correction, double *out, void *stream);
/* Strain of every node from its gradient H (N, 9): E (N, 9) of type 0 infinitesimal, 1 Green-Lagrange,
 * 2 Euler-Almansi, 3 Hencky; principal strains (N, 3) descending; maximum shear, von Mises, volumetric
 * strain, det(I + H) and the polar rotation angle in degrees (N each).  NaN in, NaN out. */
int aldvc_strain_measures(const double *H, int64_t n_nodes, int32_t strain_type, double *E, double *principal, double *max_shear,
                          double *von_mises, double *volumetric, double *det_F, double *rotation_deg, void *stream);

/* ---------------------------------------------------------------- node-grid post-processing */
/* fills the unknown nodes of the (N, ncols) FP64 field (node n = iz*ny*nx + iy*nx + ix) with the
 * spring (discrete Laplace) solution, CG to relative residual `tol`; iters/err are device int32 */
size_t aldvc_inpaint_workspace_size(int64_t nz, int64_t ny, int64_t nx, int32_t ncols);
int aldvc_inpaint(double *values, int64_t nz, int64_t ny, int64_t nx, int32_t ncols, const uint8_t *unknown, double tol,
                  int32_t max_iter, void *workspace, size_t workspace_bytes, int32_t *iters, int32_t *err, void *stream);

/* universal median test of an (N, ncols) field: flag (N,) = 1 for valid outliers */
size_t aldvc_median_test_workspace_size(int64_t nz, int64_t ny, int64_t nx, int32_t ncols);
int aldvc_median_test(const double *field, int64_t nz, int64_t ny, int64_t nx, int32_t ncols, const uint8_t *valid,
                      double threshold, double eps, uint8_t *flag, void *workspace, size_t workspace_bytes, int32_t *err,
                      void *stream);

/* ---------------------------------------------------------------- local subset solver */
/* Per-node Hessian H (N,12,12), its Cholesky factor L (N,12,12), meanf, bottomf, n_valid, valid. */
int aldvc_precompute(const aldvc_volumes *vol, const aldvc_subset *sub, const int64_t *coords, int64_t n_nodes,
                     double min_valid_ratio, double cond_max, double *H_all, double *L_all, double *meanf, double *bottomf,
                     int64_t *n_valid, uint8_t *valid, void *stream);

/* aldvc_precompute on a tensor grid of nodes: node n = (iz * ngy + iy) * ngx + ix sits at (xs[ix], ys[iy], zs[iz])
 * (device int64 arrays).  For volumes with stored gradients, an optional mask, no split rows or per-node shapes,
 * stride 1: the moments are summed separably (each voxel row once per node column instead of once per node).  Same
 * outputs and validity rules as aldvc_precompute; workspace of aldvc_precompute_grid_workspace_size bytes.
 * nx <= 8192. */
size_t aldvc_precompute_grid_workspace_size(int64_t nz, int64_t ny, int64_t nx, int64_t ngx, int64_t ngy);
int aldvc_precompute_grid(const aldvc_volumes *vol, const aldvc_subset *sub, const int64_t *xs, int64_t ngx, const int64_t *ys,
                          int64_t ngy, const int64_t *zs, int64_t ngz, double min_valid_ratio, double cond_max, double *H_all,
                          double *L_all, double *meanf, double *bottomf, int64_t *n_valid, uint8_t *valid, void *workspace,
                          size_t workspace_bytes, void *stream);

/* bytes of workspace aldvc_icgn12/aldvc_icgn3 need for `n_nodes` nodes with these params */
size_t aldvc_icgn_workspace_size(const aldvc_subset *sub, int64_t n_nodes, const aldvc_icgn_params *prm);

/* 12-DOF IC-GN.  H_all/pattern may be NULL unless prm->noise_gain > 0; meanf_all is the precompute mean
 * (only used to centre the single-pass sums).  Outputs: P_out (N,12), n_iter (N,), status (N,), zncc (N,). */
int aldvc_icgn12(const aldvc_volumes *vol, const aldvc_subset *sub, const int64_t *coords, int64_t n_nodes, const double *P0,
                 const double *L_all, const double *H_all, const double *pattern, const double *meanf_all, const uint8_t *valid,
                 const aldvc_icgn_params *prm, void *workspace, size_t workspace_bytes, double *P_out, int32_t *n_iter,
                 int8_t *status, double *zncc, void *stream);

/* 3-DOF translation IC-GN with the ADMM proximal term (subproblem 1).  F_fixed (N,3,3), U_old/vdual (N,3). */
int aldvc_icgn3(const aldvc_volumes *vol, const aldvc_subset *sub, const int64_t *coords, int64_t n_nodes, const double *U_old,
                const double *F_fixed, const double *vdual, const double *H_all, const double *meanf_all,
                const double *bottomf_all, const uint8_t *valid, const aldvc_icgn_params *prm, void *workspace,
                size_t workspace_bytes, double *U_out, int32_t *n_iter, int8_t *status, double *zncc, void *stream);

/* ---------------------------------------------------------------- integer search */
/* ZNCC maps out (n, 2rz+1, 2ry+1, 2rx+1) float32 of centred templates against windows starting at
 * (wx0, wy0, wz0); t_ok == 0 or a flat template gives a map of -2 (the reference contract). */
int aldvc_ncc_map(const float *f, const float *g, int64_t nz, int64_t ny, int64_t nx, const int64_t *coords, int64_t n_nodes,
                  int32_t hx, int32_t hy, int32_t hz, int32_t rx, int32_t ry, int32_t rz, const int64_t *wx0, const int64_t *wy0,
                  const int64_t *wz0, const uint8_t *t_ok, float *out, void *stream);

/* NCC engines: TILED (shared-memory window ring, register-tiled cross term, box-filter volumes for the
 * window statistics; templates 5..33 voxels wide), PLAIN (one thread per offset, the reference layout) and
 * FFT (cross term by 3-D FFTs of 2,3,5-smooth lengths up to 128 per axis, replacing the reference's
 * rfftn/irfftn engine, integer_search.py:423-443; a geometry it does not take runs on TILED) */
#define ALDVC_NCC_TILED 0
#define ALDVC_NCC_PLAIN 1
#define ALDVC_NCC_FFT 2
/* the FFT engine with its shared-memory Stockham transforms for every box (the in-register transforms of cubic
 * boxes of length 36, 40, 48, 50, 54, 60 or 64 turned off): a comparison form */
#define ALDVC_NCC_FFT_STOCKHAM 3
/* the FFT engine for cubic boxes of length 36, 40, 48, 50 or 54 as one thread-block cluster kernel per node: the
 * node's spectrum stays in the distributed shared memory of 8 CTAs instead of an HBM scratch (other boxes run
 * as ALDVC_NCC_FFT) */
#define ALDVC_NCC_FFT_CLUSTER 4

size_t aldvc_ncc_search_workspace_size(int64_t nz, int64_t ny, int64_t nx, int64_t n_nodes, int32_t hx, int32_t hy, int32_t hz,
                                       int32_t rx, int32_t ry, int32_t rz, int32_t engine);

/* Whole single-level search: template size (2h+1) per axis, search radius r, optional integer prior
 * shift0 (N,3) [x,y,z] (NULL = 0).  disp (N,3) [x,y,z] (NaN where not ok), cc, pce (N,), clipped, ok (N,).
 * Every engine is stream-ordered without a host round trip. */
int aldvc_ncc_search(const float *f, const float *g, int64_t nz, int64_t ny, int64_t nx, const int64_t *coords,
                     int64_t n_nodes, int32_t hx, int32_t hy, int32_t hz, int32_t rx, int32_t ry, int32_t rz,
                     const int64_t *shift0, int32_t engine, void *workspace, size_t workspace_bytes, double *disp, double *cc,
                     double *pce, uint8_t *clipped, uint8_t *ok, void *stream);

/* ---------------------------------------------------------------- global step (ADMM subproblem 2) */
/* b = beta sum_j G_j (F1 - W)[:,:,j] + mu M (U1 - v) + alpha Kg U1, all (N,3) / (N,3,3) FP64 */
int aldvc_global_rhs(const aldvc_hex8_mesh *mesh, double beta, double mu, double alpha, const double *U1, const double *F1,
                     const double *W, const double *v, double *b, void *stream);

size_t aldvc_pcg_workspace_size(const aldvc_hex8_mesh *mesh);

/* Jacobi-PCG on A = (beta + alpha) Kg + mu M restricted to the nodes of the kept elements, three
 * right-hand sides B (N,3) at once from X0 (N,3); X (N,3) keeps X0 off the active set.  iters (device
 * int32) receives the iteration count, err (device int32) a nonzero code if a grid barrier gave up. */
int aldvc_pcg_hex8(const aldvc_hex8_mesh *mesh, double beta, double mu, double alpha, const double *B, const double *X0,
                   double tol, int32_t max_iter, void *workspace, size_t workspace_bytes, double *X, int32_t *iters,
                   int32_t *err, void *stream);

/* aldvc_pcg_hex8 without a workspace, for callers that cannot allocate device memory (a plugin inside a
 * host application that owns the device budget, a real-time loop that must not call cudaMalloc).  No
 * counterpart in the reference.  Its scratch is a file-scope device array of about 28 MB that every GPU
 * loading the library holds until exit; meshes above aldvc_pcg_hex8_noalloc_max_nodes() nodes (262144)
 * are rejected with ALDVC_ERR_ARG.  All calls share the array: calls that overlap on the GPU race.  The
 * first call on a device looks up the array's address; make it before any stream capture. */
int64_t aldvc_pcg_hex8_noalloc_max_nodes(void);
int aldvc_pcg_hex8_noalloc(const aldvc_hex8_mesh *mesh, double beta, double mu, double alpha, const double *B,
                           const double *X0, double tol, int32_t max_iter, double *X, int32_t *iters, int32_t *err,
                           void *stream);

/* F (N,3,3) = (G_j^T u_i) / m_L on the active nodes, NaN elsewhere */
int aldvc_nodal_gradient(const aldvc_hex8_mesh *mesh, const double *U, double *F, void *stream);

/* ---------------------------------------------------------------- differentiable ZNSSD residual */
/* Cost C = sum_v r_v^2 of the residual IC-GN minimises (solver/numba_kernels.py:705-708, statistics of the
 * dynamic valid set :586-598), per subset of (2h+1)^3 voxels around coords[s] [x,y,z] under the 12-parameter
 * warp P[s] (F row-major, u, v, w), mode 0 linear / 1 Keys cubic / 2 B-spline (g already prefiltered).
 * vol->mask and the gradient pointers are ignored.  stats (N,7) keeps (n_valid, mf, bf, mg, bg, sum r,
 * sum r (g - mg)/bg) for the backward.  A subset that leaves f, has a warped voxel outside the sampler's
 * domain, or has fewer than 27 or half of its voxels valid gets cost NaN and n_valid 0.  The reference has no
 * ZNSSD autograd; these two entry points back pyaldvc_b200.znssd (a torch.autograd.Function). */
int aldvc_znssd_forward(const aldvc_volumes *vol, const int64_t *coords, int64_t n, int32_t hx, int32_t hy, int32_t hz,
                        int32_t mode, const double *P, double *cost, double *stats, void *stream);

/* Backward of aldvc_znssd_forward for incoming gradients grad_cost (N,): grad_P (N,12) (NULL to skip), and
 * grad_g, the gradient with respect to the deformed volume's voxels, ADDED into (nz,ny,nx) float32 (NULL to
 * skip).  Interpolation weights are recomputed from P; nothing per voxel is kept from the forward. */
int aldvc_znssd_backward(const aldvc_volumes *vol, const int64_t *coords, int64_t n, int32_t hx, int32_t hy, int32_t hz,
                         int32_t mode, const double *P, const double *stats, const double *grad_cost, double *grad_P,
                         float *grad_g, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* ALDVC_B200_H */
