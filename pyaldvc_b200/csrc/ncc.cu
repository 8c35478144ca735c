// Integer-voxel NCC search (pyALDVC solver/integer_search.py:44-151, 297-483).
//
// aldvc_ncc_map: the zncc_direct contract.  One CTA per (node, tile of offsets); the centred template
//   (FP32, minus its FP64 mean) sits in shared memory, each thread owns one offset and accumulates the
//   cross term and the window's box sums in one sweep over the template.  Window values are centred on
//   the template mean; per template plane the FP32 partial sums are flushed into FP64 totals.
//
// aldvc_ncc_search: window placement, map, first-maximum argmax (C order), PCE, clipped flag, FP64
//   re-scoring of every offset within NEAR_TIE of the FP32 maximum and of the 27-point neighbourhood of
//   the winner, quadratic sub-voxel fit -- all on the device, in node chunks through a workspace.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "fft_reg.cuh"
#include "internal.cuh"

namespace aldvc {

constexpr int NCC_THREADS = 256;
constexpr float NEAR_TIE = 2e-4f;  // FP32 map error bound used to pick FP64 re-score candidates
constexpr int MAX_CAND = 64;

__constant__ double c_pinv[10 * 27];  // pseudo-inverse of the 27-point quadratic design (integer_search.py:210-227)

// Sweep of an (nrows x ncols) tile by linear index (every lane busy whatever ncols is); the row of index i is
// (i + 0.5) / ncols in FP32, exact for i < 2^22.  RB indices per thread are loaded before any is stored.
template <int RB, typename T, typename Ld, typename St>
__device__ __forceinline__ void sweep_lin(int nrows, int ncols, Ld ld, St st) {
    const int total = nrows * ncols;
    const float inv = 1.0f / (float)ncols;
    for (int i0 = threadIdx.x; i0 < total; i0 += RB * blockDim.x) {
        T v[RB];
        int rr[RB], cc[RB];
#pragma unroll
        for (int u = 0; u < RB; ++u) {
            const int i = i0 + u * blockDim.x;
            rr[u] = (int)(((float)i + 0.5f) * inv);
            cc[u] = i - rr[u] * ncols;
            if (i < total) v[u] = ld(rr[u], cc[u]);
        }
#pragma unroll
        for (int u = 0; u < RB; ++u)
            if (i0 + u * (int)blockDim.x < total) st(rr[u], cc[u], v[u]);
    }
}

// r / d for 0 <= r < 2^22 from the FP32 reciprocal of d (exact in that range, as in sweep_lin)
__device__ __forceinline__ int fdivi(int r, float inv_d) { return (int)(((float)r + 0.5f) * inv_d); }

// Row-by-column sweep of an (nrows x ncols <= 128) tile, one warp per row: RB rows of loads are issued before
// any of their stores, so each thread keeps up to 4 RB global loads in flight.
template <int RB, typename T, typename Ld, typename St>
__device__ __forceinline__ void copy_rows(int nrows, int ncols, Ld ld, St st) {
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int r0 = (threadIdx.x >> 5) * RB; r0 < nrows; r0 += nw * RB) {
        T v[RB][4];
#pragma unroll
        for (int u = 0; u < RB; ++u)
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                const int r = r0 + u, c = lane + 32 * h;
                if (r < nrows && c < ncols) v[u][h] = ld(r, c);
            }
#pragma unroll
        for (int u = 0; u < RB; ++u)
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                const int r = r0 + u, c = lane + 32 * h;
                if (r < nrows && c < ncols) st(r, c, v[u][h]);
            }
    }
}

__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::); }

// hint that a line is read soon: fetched into L2 without occupying a register
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

struct NccGeom {
    int nz, ny, nx;
    int hx, hy, hz, rx, ry, rz;
    int sx, sy, sz, vx, vy, vz, wx, wy, wz;
    int n_tpl, nmap;
};

__host__ inline NccGeom make_geom(int64_t nz, int64_t ny, int64_t nx, int hx, int hy, int hz, int rx, int ry, int rz) {
    NccGeom g;
    g.nz = (int)nz;
    g.ny = (int)ny;
    g.nx = (int)nx;
    g.hx = hx;
    g.hy = hy;
    g.hz = hz;
    g.rx = rx;
    g.ry = ry;
    g.rz = rz;
    g.sx = 2 * hx + 1;
    g.sy = 2 * hy + 1;
    g.sz = 2 * hz + 1;
    g.vx = 2 * rx + 1;
    g.vy = 2 * ry + 1;
    g.vz = 2 * rz + 1;
    g.wx = g.sx + 2 * rx;
    g.wy = g.sy + 2 * ry;
    g.wz = g.sz + 2 * rz;
    g.n_tpl = g.sx * g.sy * g.sz;
    g.nmap = g.vx * g.vy * g.vz;
    return g;
}

__device__ __forceinline__ double block_sum_d(double v, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum_d(v);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    return s;
}

// Centred template into shared memory (FP32) and its FP64 mean and sum of squares.
// Returns false (for every thread) when the template is flat.
__device__ bool load_template(const float* __restrict__ f, const NccGeom& G, int64_t x0, int64_t y0, int64_t z0, float* T,
                              double* red, double& mf, double& ssf) {
    const int64_t sxy = (int64_t)G.nx * G.ny;
    double s = 0.0;
    for (int i = threadIdx.x; i < G.n_tpl; i += blockDim.x) {
        const int k = i / (G.sx * G.sy), r = i - k * G.sx * G.sy, j = r / G.sx, ii = r - j * G.sx;
        const float v = __ldg(f + (z0 - G.hz + k) * sxy + (y0 - G.hy + j) * G.nx + (x0 - G.hx + ii));
        T[i] = v;
        s += (double)v;
    }
    s = block_sum_d(s, red);
    mf = s / (double)G.n_tpl;
    double q = 0.0;
    for (int i = threadIdx.x; i < G.n_tpl; i += blockDim.x) {
        const double d = (double)T[i] - mf;
        q += d * d;
        T[i] = (float)d;
    }
    ssf = block_sum_d(q, red);
    __syncthreads();
    return !(ssf < 1e-20);
}

// ZNCC of one offset from FP32 sums (cross term and window box sums), reference normalisation.
__device__ __forceinline__ float ncc_value(double sfg, double sg, double sgg, double n_tpl, double ssf) {
    const double var = sgg - sg * sg / n_tpl;
    if (var < 1e-20) return 0.0f;
    double v = sfg / sqrt(var * ssf);
    v = v > 1.0 ? 1.0 : (v < -1.0 ? -1.0 : v);
    return (float)v;
}

// One thread: the sums of one offset over the template (shared T), window read from global g.
__device__ __forceinline__ void offset_sums(const float* __restrict__ g, const NccGeom& G, const float* T, int64_t zb, int64_t yb,
                                            int64_t xb, float pilot, double& sfg, double& sg, double& sgg) {
    const int64_t sxy = (int64_t)G.nx * G.ny;
    sfg = sg = sgg = 0.0;
    for (int k = 0; k < G.sz; ++k) {
        float a = 0.0f, b = 0.0f, c = 0.0f;
        const float* Tk = T + k * G.sx * G.sy;
        for (int j = 0; j < G.sy; ++j) {
            const float* gr = g + (zb + k) * sxy + (yb + j) * G.nx + xb;
            const float* Tr = Tk + j * G.sx;
            for (int i = 0; i < G.sx; ++i) {
                const float v = __ldg(gr + i) - pilot;
                a = fmaf(Tr[i], v, a);
                b += v;
                c = fmaf(v, v, c);
            }
        }
        sfg += a;
        sg += b;
        sgg += c;
    }
}

struct MapArgs {
    const float* f;
    const float* g;
    const int64_t* coords;
    const int64_t* wx0;
    const int64_t* wy0;
    const int64_t* wz0;
    const uint8_t* t_ok;
    float* out;
    int64_t node_base, n_nodes;
    NccGeom G;
};

// grid (tiles, nodes); dynamic smem = template floats
__global__ void __launch_bounds__(NCC_THREADS) ncc_map_kernel(MapArgs a) {
    extern __shared__ float T[];
    __shared__ double red[NCC_THREADS / 32];
    __shared__ double s_stat[2];
    const NccGeom& G = a.G;
    const int64_t node = a.node_base + blockIdx.y;
    if (node >= a.n_nodes) return;
    float* out = a.out + (int64_t)blockIdx.y * G.nmap;
    const int d = blockIdx.x * NCC_THREADS + threadIdx.x;
    const int64_t x0 = a.coords[3 * node], y0 = a.coords[3 * node + 1], z0 = a.coords[3 * node + 2];
    // a template or window outside the volume is treated like t_ok == 0 (no read leaves the volume)
    const int64_t wx0 = a.wx0[node], wy0 = a.wy0[node], wz0 = a.wz0[node];
    const bool placed = x0 - G.hx >= 0 && x0 + G.hx < G.nx && y0 - G.hy >= 0 && y0 + G.hy < G.ny && z0 - G.hz >= 0 &&
                        z0 + G.hz < G.nz && wx0 >= 0 && wx0 + G.wx <= G.nx && wy0 >= 0 && wy0 + G.wy <= G.ny && wz0 >= 0 &&
                        wz0 + G.wz <= G.nz;
    if (!a.t_ok[node] || !placed) {
        if (d < G.nmap) out[d] = -2.0f;
        return;
    }
    double mf, ssf;
    const bool textured = load_template(a.f, G, x0, y0, z0, T, red, mf, ssf);
    if (threadIdx.x == 0) {
        s_stat[0] = mf;
        s_stat[1] = ssf;
    }
    __syncthreads();
    if (d >= G.nmap) return;
    if (!textured) {
        out[d] = -2.0f;
        return;
    }
    const int dz = d / (G.vy * G.vx), r = d - dz * G.vy * G.vx, dy = r / G.vx, dx = r - dy * G.vx;
    double sfg, sg, sgg;
    offset_sums(a.g, G, T, wz0 + dz, wy0 + dy, wx0 + dx, (float)s_stat[0], sfg, sg, sgg);
    out[d] = ncc_value(sfg, sg, sgg, (double)G.n_tpl, s_stat[1]);
}

// ----------------------------------------------------------------------------- fused search
// Partials of one block of a node's FP32 map (the planes one FFT pass-3 CTA writes), for the peak search: the
// maximum with its first index, the minimum, and FP64 sums of the values and their squares (values below -1, the
// unplaced-node marker, count as 0 as in the peak kernel's sweeps).
struct MapPart {
    double s1, s2;
    float mx, mn;
    int idx, pad;
};

struct SearchArgs {
    const float* f;
    const float* g;
    const int64_t* coords;
    const int64_t* shift0;
    int64_t n_nodes, node_base;
    NccGeom G;
    // per-node placement (workspace)
    int64_t* wx0;
    int64_t* wy0;
    int64_t* wz0;
    uint8_t* t_ok;
    uint8_t* freeb;  // bits: lo x,y,z (1,2,4), hi x,y,z (8,16,32)
    const float* map;  // chunk maps
    double* disp;
    double* cc;
    double* pce;
    uint8_t* clipped;
    uint8_t* ok;
    const MapPart* part;  // per-block map partials of the chunk ([node][nblk]), or null: the peak kernel sweeps the map
    int nblk, blk_planes;
};

// integer_search.py:374-386 window placement
__global__ void ncc_place_kernel(SearchArgs a) {
    const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (n >= a.n_nodes) return;
    const NccGeom& G = a.G;
    const int64_t cx = a.coords[3 * n], cy = a.coords[3 * n + 1], cz = a.coords[3 * n + 2];
    const int64_t sx0 = a.shift0 ? a.shift0[3 * n] : 0, sy0 = a.shift0 ? a.shift0[3 * n + 1] : 0,
                  sz0 = a.shift0 ? a.shift0[3 * n + 2] : 0;
    a.t_ok[n] = (cx - G.hx >= 0) && (cx + G.hx < G.nx) && (cy - G.hy >= 0) && (cy + G.hy < G.ny) && (cz - G.hz >= 0) &&
                (cz + G.hz < G.nz);
    const int64_t dx0 = cx + sx0 - G.hx - G.rx, dy0 = cy + sy0 - G.hy - G.ry, dz0 = cz + sz0 - G.hz - G.rz;
    auto clip = [](int64_t v, int64_t hi) { return v < 0 ? 0 : (v > hi ? hi : v); };
    a.wx0[n] = clip(dx0, G.nx - G.wx);
    a.wy0[n] = clip(dy0, G.ny - G.wy);
    a.wz0[n] = clip(dz0, G.nz - G.wz);
    uint8_t fb = 0;
    fb |= dx0 >= 0 ? 1 : 0;
    fb |= dy0 >= 0 ? 2 : 0;
    fb |= dz0 >= 0 ? 4 : 0;
    fb |= dx0 <= G.nx - G.wx ? 8 : 0;
    fb |= dy0 <= G.ny - G.wy ? 16 : 0;
    fb |= dz0 <= G.nz - G.wz ? 32 : 0;
    a.freeb[n] = fb;
}

// FP64 value of one offset, the reference's arithmetic (FP64 centred template, float32-rounded squares),
// computed by one warp: template voxel (k, j, i) at tp[k tsz + j tsy + i], its window voxel at
// wp[k wsz + j wsy + i].  Lanes stride the template in C order; the sums are reduced by shuffles in a fixed
// order, and every lane returns the value.
__device__ double warp_rescore(const float* tp, int64_t tsz, int64_t tsy, const float* wp, int64_t wsz, int64_t wsy,
                               const NccGeom& G, double mf, double ssf) {
    const int lane = threadIdx.x & 31;
    double sfg = 0.0, sg = 0.0, sgg = 0.0;
    int ii = lane % G.sx, j = (lane / G.sx) % G.sy, k = lane / (G.sx * G.sy);
    const int di = 32 % G.sx, dj = (32 / G.sx) % G.sy, dk = 32 / (G.sx * G.sy);
    for (int t = lane; t < G.n_tpl; t += 32) {
        const float fv = tp[k * tsz + j * tsy + ii];
        const float v = wp[k * wsz + j * wsy + ii];
        sfg += ((double)fv - mf) * (double)v;
        sg += (double)v;
        sgg += (double)(v * v);
        ii += di;
        j += dj;
        k += dk;
        if (ii >= G.sx) {
            ii -= G.sx;
            ++j;
        }
        if (j >= G.sy) {
            j -= G.sy;
            ++k;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sfg += __shfl_xor_sync(0xffffffffu, sfg, o);
        sg += __shfl_xor_sync(0xffffffffu, sg, o);
        sgg += __shfl_xor_sync(0xffffffffu, sgg, o);
    }
    const double var = sgg - sg * sg / (double)G.n_tpl;
    if (var < 1e-20) return 0.0;
    const double v = sfg / sqrt(var * ssf);
    return v > 1.0 ? 1.0 : (v < -1.0 ? -1.0 : v);
}

// warp_rescore over a template staged contiguously in shared memory, with the (k, j, i) coordinates of every
// template voxel packed in kji[t] (k << 20 | j << 10 | i): the loads of successive voxels do not wait on one
// another's index arithmetic, so a lane keeps several window loads in flight.  Same per-lane order and reduction
// as warp_rescore, hence the same value.  GLOBAL: the window is in global memory (read through the
// non-coherent path); otherwise in shared memory.
template <bool GLOBAL>
__device__ double warp_rescore_tab(const float* tp, const uint32_t* kji, const float* wp, int64_t wsz, int64_t wsy, int n_tpl,
                                   double mf, double ssf) {
    const int lane = threadIdx.x & 31;
    double sfg = 0.0, sg = 0.0, sgg = 0.0;
#pragma unroll 8
    for (int t = lane; t < n_tpl; t += 32) {
        const uint32_t c = kji[t];
        const float fv = tp[t];
        const int64_t o = (int64_t)(c >> 20) * wsz + (int64_t)((c >> 10) & 1023u) * wsy + (int64_t)(c & 1023u);
        const float v = GLOBAL ? __ldg(wp + o) : wp[o];
        sfg += ((double)fv - mf) * (double)v;
        sg += (double)v;
        sgg += (double)(v * v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sfg += __shfl_xor_sync(0xffffffffu, sfg, o);
        sg += __shfl_xor_sync(0xffffffffu, sg, o);
        sgg += __shfl_xor_sync(0xffffffffu, sgg, o);
    }
    const double var = sgg - sg * sg / (double)n_tpl;
    if (var < 1e-20) return 0.0;
    const double v = sfg / sqrt(var * ssf);
    return v > 1.0 ? 1.0 : (v < -1.0 ? -1.0 : v);
}

// One CTA per node of the chunk.  Two sweeps of the FP32 map: (1) maximum (first index on ties), minimum;
// (2) candidates within NEAR_TIE of the maximum and the PCE energy.  The template (raw FP32 f) and, for the
// sub-voxel fit, the window box around the peak are staged in shared memory when SMEM; each FP64 re-score is
// one warp's job.
template <bool SMEM>
__global__ void __launch_bounds__(NCC_THREADS, 3) ncc_peak_kernel(SearchArgs a) {
    extern __shared__ __align__(16) float psm[];
    __shared__ double red[NCC_THREADS / 32];
    __shared__ float s_best[NCC_THREADS / 32], s_mn[NCC_THREADS / 32];
    __shared__ int s_bidx[NCC_THREADS / 32];
    __shared__ int s_cand[MAX_CAND];
    __shared__ double s_cval[MAX_CAND];
    __shared__ int s_ncand;
    __shared__ double s_neigh[27];
    __shared__ double s_coef[10];
    __shared__ double s_nb[9][9];               // per (dz, dy) pair: sum (f - mf) g, sum g, sum g^2 for dx = 0, 1, 2
    __shared__ double s_p8[NCC_THREADS / 32][9];  // the warps' partials of pair 8
    __shared__ float s_max, s_min;
    __shared__ int s_pk;
    __shared__ double s_s1, s_s2;
    const NccGeom& G = a.G;
    const int64_t node = a.node_base + blockIdx.x;
    if (node >= a.n_nodes) return;
    const float* map = a.map + (int64_t)blockIdx.x * G.nmap;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = NCC_THREADS / 32;
    const int64_t sxy = (int64_t)G.nx * G.ny;
    if (!a.t_ok[node]) {
        if (tid == 0) {
            for (int c = 0; c < 3; ++c) a.disp[3 * node + c] = nan("");
            a.cc[node] = nan("");
            a.pce[node] = nan("");
            a.clipped[node] = 0;
            a.ok[node] = 0;
        }
        return;
    }
    const bool fastp = a.part != nullptr;  // map partials from the producer: only candidate blocks are swept
    if (!fastp)
        for (int i = tid * 32; i < G.nmap; i += NCC_THREADS * 32) prefetch_l2(map + i);  // the whole map towards L2
    // the template first: its loads do not depend on the map, so their latency overlaps the map sweeps'
    // template: raw FP32 f (staged when SMEM), FP64 mean and sum of squares (integer_search.py:73-88)
    const int64_t x0 = a.coords[3 * node], y0 = a.coords[3 * node + 1], z0 = a.coords[3 * node + 2];
    const float* fg = a.f + (z0 - G.hz) * sxy + (y0 - G.hy) * G.nx + (x0 - G.hx);
    const int64_t tsz = SMEM ? (int64_t)G.sy * G.sx : sxy, tsy = SMEM ? G.sx : G.nx;
    const float* tp = SMEM ? psm : fg;
    // shared layout: template (n_tpl floats), neighbour box ((sx+2)(sy+2)(sz+2) floats), packed template
    // coordinates (n_tpl words)
    uint32_t* kji = reinterpret_cast<uint32_t*>(psm + G.n_tpl + (G.sx + 2) * (G.sy + 2) * (G.sz + 2));
    double sf = 0.0;
    const int nrow = G.sz * G.sy;
    const float inv_sy = 1.0f / (float)G.sy;  // template rows: r < 2^20
    if (G.sx <= 32) {
        // one sample per lane and row: eight rows' loads in flight per warp, then the sums in the same row order
        for (int r0 = warp; r0 < nrow; r0 += 8 * NW) {
            float vv[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int r = r0 + u * NW, k = fdivi(r, inv_sy), j = r - k * G.sy;
                vv[u] = (r < nrow && lane < G.sx) ? __ldg(fg + k * sxy + (int64_t)j * G.nx + lane) : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int r = r0 + u * NW, k = fdivi(r, inv_sy), j = r - k * G.sy;
                if (r < nrow && lane < G.sx) {
                    if (SMEM) {
                        psm[r * G.sx + lane] = vv[u];
                        kji[r * G.sx + lane] = ((uint32_t)k << 20) | ((uint32_t)j << 10) | (uint32_t)lane;
                    }
                    sf += (double)vv[u];
                }
            }
        }
    } else {
        for (int r = warp; r < nrow; r += NW) {
            const int k = r / G.sy, j = r - k * G.sy;
            for (int ii = lane; ii < G.sx; ii += 32) {
                const float v = __ldg(fg + k * sxy + (int64_t)j * G.nx + ii);
                if (SMEM) {
                    psm[r * G.sx + ii] = v;
                    kji[r * G.sx + ii] = ((uint32_t)k << 20) | ((uint32_t)j << 10) | (uint32_t)ii;
                }
                sf += (double)v;
            }
        }
    }
    sf = block_sum_d(sf, red);
    const double mf = sf / (double)G.n_tpl;
    double q = 0.0;
    for (int r = warp; r < G.sz * G.sy; r += NW) {
        const int k = fdivi(r, inv_sy), j = r - k * G.sy;
        for (int ii = lane; ii < G.sx; ii += 32) {
            const double d = (double)tp[k * tsz + j * tsy + ii] - mf;
            q += d * d;
        }
    }
    const double ssf = block_sum_d(q, red);
    // flat template: the map is -2 everywhere (integer_search.py:420-421)
    const bool flat = map[0] < -1.5f;
    const MapPart* parts = fastp ? a.part + (int64_t)blockIdx.x * a.nblk : nullptr;
    if (fastp) {  // blocks in map order: the first maximum of the earliest block holding it is the first in the map
        if (tid == 0) {
            float b = -3.0f, m = 3.0f;
            int bi = 0x7fffffff;
            double t1 = 0.0, t2 = 0.0;
            for (int k0 = 0; k0 < a.nblk; k0 += 4) {  // four partials' loads in flight, then in block order
                MapPart qq[4];
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (k0 + u < a.nblk) qq[u] = parts[k0 + u];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    if (k0 + u >= a.nblk) break;
                    const MapPart& q = qq[u];
                    if (q.mx > b || (q.mx == b && q.idx < bi)) {
                        b = q.mx;
                        bi = q.idx;
                    }
                    m = fminf(m, q.mn);
                    t1 += q.s1;
                    t2 += q.s2;
                }
            }
            s_max = b;
            s_pk = bi;
            s_min = m;
            s_s1 = t1;
            s_s2 = t2;
            s_ncand = 0;
        }
        __syncthreads();
    } else {
    float best = -3.0f, mn = 3.0f;
    int bidx = 0x7fffffff;
    // eight loads in flight per thread, then the compares in ascending i (the first index wins a tie)
    for (int i0 = tid; i0 < G.nmap; i0 += 8 * NCC_THREADS) {
        float vv[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) vv[u] = i0 + u * NCC_THREADS < G.nmap ? map[i0 + u * NCC_THREADS] : -3.0f;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            if (i0 + u * NCC_THREADS >= G.nmap) break;
            const float v = vv[u] < -1.0f ? 0.0f : vv[u];
            if (v > best) {
                best = v;
                bidx = i0 + u * NCC_THREADS;
            }
            mn = fminf(mn, v);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const float ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bidx, o);
        if (ob > best || (ob == best && oi < bidx)) {
            best = ob;
            bidx = oi;
        }
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    }
    if (lane == 0) {
        s_best[warp] = best;
        s_bidx[warp] = bidx;
        s_mn[warp] = mn;
    }
    __syncthreads();
    if (tid == 0) {
        float b = s_best[0], m = s_mn[0];
        int bi = s_bidx[0];
        for (int w = 1; w < NW; ++w) {
            if (s_best[w] > b || (s_best[w] == b && s_bidx[w] < bi)) {
                b = s_best[w];
                bi = s_bidx[w];
            }
            m = fminf(m, s_mn[w]);
        }
        s_max = b;
        s_pk = bi;
        s_min = m;
        s_ncand = 0;
    }
    __syncthreads();
    }
    const float vmax = s_max, vmin = s_min;
    const float cmin = flat ? 0.0f : vmin;
    const int64_t wz0 = a.wz0[node], wy0 = a.wy0[node], wx0 = a.wx0[node];
    const int BX = G.sx + 2, BY = G.sy + 2, BZ = G.sz + 2;
    const float inv_bx = 1.0f / (float)BX, inv_by = 1.0f / (float)BY;  // neighbour box rows and columns: below 2^21
    float* box = psm + G.n_tpl;  // the neighbour box of the peak (shared layout above)
    auto interior_at = [&](int q) {
        const int qz = q / (G.vy * G.vx), qr = q - qz * G.vy * G.vx, qy = qr / G.vx, qx = qr - qy * G.vx;
        return qx > 0 && qx < 2 * G.rx && qy > 0 && qy < 2 * G.ry && qz > 0 && qz < 2 * G.rz && !flat;
    };
    auto box_origin = [&](int q) {
        const int qz = q / (G.vy * G.vx), qr = q - qz * G.vy * G.vx, qy = qr / G.vx, qx = qr - qy * G.vx;
        return a.g + (wz0 + qz - 1) * sxy + (wy0 + qy - 1) * G.nx + (wx0 + qx - 1);
    };
    // the box of the FP32 maximum, copied asynchronously while the second sweep and the candidate scores run: it
    // is the box the sub-voxel fit needs unless the FP64 re-scores move the peak
    const int spk = s_pk;
    const bool spec = SMEM && interior_at(spk);
    if (spec) {
        const float* gb0 = box_origin(spk);
        for (int i = tid; i < BZ * BY * BX; i += NCC_THREADS) {
            const int r = fdivi(i, inv_bx), ii = i - r * BX, k = fdivi(r, inv_by), j = r - k * BY;
            cp_async4(box + i, gb0 + k * sxy + (int64_t)j * G.nx + ii);
        }
        cp_async_commit();
    }
    // candidates within the FP32 error bound of the maximum, and the PCE energy on the min-shifted map
    // (integer_search.py:448-452)
    double e = 0.0;
    if (fastp) {
        // only blocks whose maximum reaches the bound can hold candidates (the same FP32 comparison); the energy
        // sum (v - c)^2 = sum v^2 - 2 c sum v + n c^2 from the blocks' FP64 sums
        const int bsz = a.blk_planes * G.vy * G.vx;
        for (int k = 0; k < a.nblk; ++k) {
            if (flat || !(parts[k].mx >= vmax - NEAR_TIE)) continue;
            const int hi = min(k * bsz + bsz, G.nmap);
            for (int i0 = k * bsz + tid; i0 < hi; i0 += 8 * NCC_THREADS) {  // eight map loads in flight per thread
                float vv[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) vv[u] = i0 + u * NCC_THREADS < hi ? map[i0 + u * NCC_THREADS] : -3.0f;
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int i = i0 + u * NCC_THREADS;
                    if (i >= hi) break;
                    const float v = vv[u] < -1.0f ? 0.0f : vv[u];
                    if (v >= vmax - NEAR_TIE) {
                        const int slot = atomicAdd(&s_ncand, 1);
                        if (slot < MAX_CAND) s_cand[slot] = i;
                    }
                }
            }
        }
        __syncthreads();
        const double c = (double)cmin, n = (double)G.nmap;
        e = (s_s2 - 2.0 * c * s_s1 + n * c * c) / n;
    } else {
    for (int i0 = tid; i0 < G.nmap; i0 += 8 * NCC_THREADS) {
        float vv[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) vv[u] = i0 + u * NCC_THREADS < G.nmap ? map[i0 + u * NCC_THREADS] : 0.0f;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int i = i0 + u * NCC_THREADS;
            if (i >= G.nmap) break;
            const float v = vv[u] < -1.0f ? 0.0f : vv[u];
            if (!flat && v >= vmax - NEAR_TIE) {
                const int slot = atomicAdd(&s_ncand, 1);
                if (slot < MAX_CAND) s_cand[slot] = i;
            }
            const double dv = (double)v - (double)cmin;
            e += dv * dv;
        }
    }
    e = block_sum_d(e, red) / (double)G.nmap;
    }
    int pk = s_pk;
    double peak = (double)vmax;
    // one candidate at an interior offset (the common case): its FP64 score is the centre of the 27-neighbourhood,
    // taken from the staged box below instead of a separate pass over the window in global memory
    bool centre_from_box = false;
    if (!flat && SMEM && min(s_ncand, MAX_CAND) == 1 && G.rx > 0 && G.ry > 0 && G.rz > 0) {
        const int qz = pk / (G.vy * G.vx), qr = pk - qz * G.vy * G.vx, qy = qr / G.vx, qx = qr - qy * G.vx;
        centre_from_box = qx > 0 && qx < 2 * G.rx && qy > 0 && qy < 2 * G.ry && qz > 0 && qz < 2 * G.rz;
    }
    if (!flat && !centre_from_box) {
        // FP64 re-score of the candidates in C order; the first maximum wins (np.argmax)
        const int nc = min(s_ncand, MAX_CAND);
        if (tid == 0) {
            for (int i = 1; i < nc; ++i) {
                const int v = s_cand[i];
                int j = i - 1;
                while (j >= 0 && s_cand[j] > v) {
                    s_cand[j + 1] = s_cand[j];
                    --j;
                }
                s_cand[j + 1] = v;
            }
        }
        __syncthreads();
        for (int c = warp; c < nc; c += NW) {
            const int i = s_cand[c];
            const int dz = i / (G.vy * G.vx), r = i - dz * G.vy * G.vx, dy = r / G.vx, dx = r - dy * G.vx;
            const float* wp = a.g + (wz0 + dz) * sxy + (wy0 + dy) * G.nx + (wx0 + dx);
            const double v = SMEM ? warp_rescore_tab<true>(tp, kji, wp, sxy, G.nx, G.n_tpl, mf, ssf)
                                  : warp_rescore(tp, tsz, tsy, wp, sxy, G.nx, G, mf, ssf);
            if (lane == 0) s_cval[c] = v;
        }
        __syncthreads();
        if (nc > 0) {
            double bv = -3.0;
            int bi = pk;
            for (int c = 0; c < nc; ++c)
                if (s_cval[c] > bv) {
                    bv = s_cval[c];
                    bi = s_cand[c];
                }
            pk = bi;
            peak = bv;
        }
    } else if (flat) {
        peak = 0.0;
        pk = 0;
    }
    const int pz = pk / (G.vy * G.vx), pr = pk - pz * G.vy * G.vx, py = pr / G.vx, px = pr - py * G.vx;
    // sub-voxel refinement on FP64 neighbours (integer_search.py:467-473, 297-321)
    const bool at_border = px == 0 || px == 2 * G.rx || py == 0 || py == 2 * G.ry || pz == 0 || pz == 2 * G.rz;
    const bool interior = !at_border && G.rx > 0 && G.ry > 0 && G.rz > 0 && !flat;
    double sub[3] = {0.0, 0.0, 0.0};
    if (spec) {  // every async copy into the box has landed before any thread reads or rewrites it
        cp_async_wait_all();
        __syncthreads();
    }
    if (interior) {
        const float* gb = a.g + (wz0 + pz - 1) * sxy + (wy0 + py - 1) * G.nx + (wx0 + px - 1);
        if (SMEM && !(spec && pk == spk)) {  // the staged box is not this peak's
            sweep_lin<8, float>(BZ * BY, BX,
                                [&](int r, int ii) {
                                    const int k = fdivi(r, inv_by), j = r - k * BY;
                                    return __ldg(gb + k * sxy + (int64_t)j * G.nx + ii);
                                },
                                [&](int r, int ii, float v) { box[r * BX + ii] = v; });
            __syncthreads();
        }
        if (SMEM) {
            // the 26 neighbours by (dz, dy) box row pairs: a lane walks whole template rows once and slides a three-
            // sample window along the box row, feeding the three dx neighbours of its pair at once.  Warp w < 8 takes
            // pair w over all template rows; pair 8 is split over the warps by row and its partials summed in order.
            static_assert(NCC_THREADS == 256, "one warp per (dz, dy) pair 0..7");
            const int rows = G.sz * G.sy;
            auto pair_rows = [&](int pr, int r0, int rstep, double acc[9]) {
                const int dzz = pr / 3, dyy = pr % 3;
                for (int r = r0; r < rows; r += rstep) {
                    const int k = fdivi(r, inv_sy), j = r - k * G.sy;
                    const float* trow = tp + (int64_t)r * G.sx;
                    const float* brow = box + ((k + dzz) * BY + (j + dyy)) * BX;
                    // the window's samples and squares carried in FP64: each box sample is converted once
                    const float b0f = brow[0], b1f = brow[1];
                    double d0 = (double)b0f, d1 = (double)b1f, q0 = (double)(b0f * b0f), q1 = (double)(b1f * b1f);
                    for (int i = 0; i < G.sx; ++i) {
                        const float b2 = brow[i + 2];
                        const double d2 = (double)b2, q2 = (double)(b2 * b2);
                        const double tf = (double)trow[i] - mf;
                        acc[0] += tf * d0;
                        acc[1] += tf * d1;
                        acc[2] += tf * d2;
                        acc[3] += d0;
                        acc[4] += d1;
                        acc[5] += d2;
                        acc[6] += q0;
                        acc[7] += q1;
                        acc[8] += q2;
                        d0 = d1;
                        d1 = d2;
                        q0 = q1;
                        q1 = q2;
                    }
                }
            };
            double acc[9];
            if (warp < 8) {
#pragma unroll
                for (int q = 0; q < 9; ++q) acc[q] = 0.0;
                pair_rows(warp, lane, 32, acc);
#pragma unroll
                for (int q = 0; q < 9; ++q) acc[q] = warp_sum_d(acc[q]);
                if (lane == 0)
                    for (int q = 0; q < 9; ++q) s_nb[warp][q] = acc[q];
            }
#pragma unroll
            for (int q = 0; q < 9; ++q) acc[q] = 0.0;
            pair_rows(8, warp * 32 + lane, 32 * NW, acc);
#pragma unroll
            for (int q = 0; q < 9; ++q) acc[q] = warp_sum_d(acc[q]);
            if (lane == 0)
                for (int q = 0; q < 9; ++q) s_p8[warp][q] = acc[q];
            __syncthreads();
            if (tid < 9) {
                double t8 = 0.0;
                for (int w = 0; w < NW; ++w) t8 += s_p8[w][tid];
                s_nb[8][tid] = t8;
            }
            __syncthreads();
            if (tid < 27) {
                const int pr = tid / 3, dxx = tid % 3;
                double v = peak;
                if (tid != 13 || centre_from_box) {
                    const double sfg = s_nb[pr][dxx], sg = s_nb[pr][3 + dxx], sgg = s_nb[pr][6 + dxx];
                    const double var = sgg - sg * sg / (double)G.n_tpl;
                    if (var < 1e-20) {
                        v = 0.0;
                    } else {
                        v = sfg / sqrt(var * ssf);
                        v = v > 1.0 ? 1.0 : (v < -1.0 ? -1.0 : v);
                    }
                }
                s_neigh[tid] = v;
            }
            if (centre_from_box) {
                __syncthreads();
                peak = s_neigh[13];
            }
        } else {
            for (int t = warp; t < 27; t += NW) {
                const int dzz = t / 9, dyy = (t / 3) % 3, dxx = t % 3;  // box coordinates of the neighbour's origin
                const double v = t == 13 ? peak
                                         : warp_rescore(tp, tsz, tsy, gb + dzz * sxy + (int64_t)dyy * G.nx + dxx, sxy, G.nx, G, mf, ssf);
                if (lane == 0) s_neigh[t] = v;
            }
        }
        __syncthreads();
        if (tid < 10) {  // one coefficient per thread, the same sum order as a serial loop
            double s = 0.0;
            for (int t = 0; t < 27; ++t) s += c_pinv[tid * 27 + t] * s_neigh[t];
            s_coef[tid] = s;
        }
        __syncthreads();
        if (tid == 0) {
            double coef[10];
            for (int r = 0; r < 10; ++r) coef[r] = s_coef[r];
            double H[3][3] = {{2 * coef[7], coef[4], coef[5]}, {coef[4], 2 * coef[8], coef[6]}, {coef[5], coef[6], 2 * coef[9]}};
            double Hi[3][3];
            const double det = inv3(H, Hi);
            if (fabs(det) > 1e-12) {
                double sol[3];
                bool good = true;
                for (int i = 0; i < 3; ++i) {
                    sol[i] = -(Hi[i][0] * coef[1] + Hi[i][1] * coef[2] + Hi[i][2] * coef[3]);
                    good = good && isfinite(sol[i]) && fabs(sol[i]) <= 1.0;
                }
                if (good)
                    for (int i = 0; i < 3; ++i) sub[i] = sol[i];
            }
        }
    }
    if (tid == 0) {
        const double pmin = peak - (double)cmin;
        const double pce = e > 1e-30 ? pmin * pmin / e : 0.0;
        const uint8_t fb = a.freeb[node];
        bool on_edge = false;
        if (G.rx > 0 || G.ry > 0 || G.rz > 0)
            on_edge = (px == 0 && (fb & 1)) || (px == 2 * G.rx && (fb & 8)) || (py == 0 && (fb & 2)) ||
                      (py == 2 * G.ry && (fb & 16)) || (pz == 0 && (fb & 4)) || (pz == 2 * G.rz && (fb & 32));
        const bool okv = isfinite(peak) && !flat;
        a.ok[node] = okv ? 1 : 0;
        a.cc[node] = peak;
        a.pce[node] = pce;
        a.clipped[node] = on_edge ? 1 : 0;
        if (okv) {
            a.disp[3 * node + 0] = (double)(wx0 + px + G.hx - x0) + sub[0];
            a.disp[3 * node + 1] = (double)(wy0 + py + G.hy - y0) + sub[1];
            a.disp[3 * node + 2] = (double)(wz0 + pz + G.hz - z0) + sub[2];
        } else {
            for (int c = 0; c < 3; ++c) a.disp[3 * node + c] = nan("");
        }
    }
}

// shared bytes of the staged peak kernel (template, neighbour box, packed template coordinates), 0 when it does
// not fit or a template side does not fit the 10-bit coordinate fields
static size_t peak_smem(const NccGeom& G) {
    if (G.sx >= 1024 || G.sy >= 1024 || G.sz >= 1024) return 0;
    const size_t b = ((size_t)2 * G.n_tpl + (size_t)(G.sx + 2) * (G.sy + 2) * (G.sz + 2)) * sizeof(float);
    return b <= 160 * 1024 ? b : 0;
}

// static shared bytes of a kernel (the opt-in attribute is needed once static plus dynamic bytes pass 48 KB)
static size_t static_smem(const void* kern) {
    cudaFuncAttributes fa{};
    return cudaFuncGetAttributes(&fa, kern) == cudaSuccess ? fa.sharedSizeBytes : (size_t)16 * 1024;
}

static int launch_peak(const SearchArgs& b, int64_t n, cudaStream_t s) {
    const size_t sm = peak_smem(b.G);
    static const size_t stat = static_smem((const void*)ncc_peak_kernel<true>);
    if (sm && sm + stat > 48 * 1024) {
        static size_t have = 0;
        static std::mutex mu;
        std::lock_guard<std::mutex> lock(mu);
        if (sm > have) {
            cudaError_t e = cudaFuncSetAttribute(ncc_peak_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            if (e != cudaSuccess) return cuda_fail(e, "ncc peak: shared memory attribute");
            have = sm;
        }
    }
    for (int64_t done = 0; done < n; done += 65535) {
        SearchArgs bb = b;
        bb.node_base = b.node_base + done;
        bb.map = b.map + done * b.G.nmap;
        const unsigned nb = (unsigned)std::min<int64_t>(65535, n - done);
        if (sm)
            {
                KTimer kt_("ncc_peak", s);
                ncc_peak_kernel<true><<<nb, NCC_THREADS, sm, s>>>(bb);
            }
        else
            {
                KTimer kt_("ncc_peak", s);
                ncc_peak_kernel<false><<<nb, NCC_THREADS, 0, s>>>(bb);
            }
        const int rc = check_launch("ncc peak");
        if (rc) return rc;
    }
    return ALDVC_OK;
}

// ----------------------------------------------------------------------------- tiled engine
// Window box sums for every template placement: separable FP32 sums of (g - c) and (g - c)^2, each
// output a direct sum of the axis length (no running subtraction), over the whole deformed volume.
__global__ void box_pass_kernel(const float* __restrict__ in1, const float* __restrict__ in2, float* __restrict__ out1,
                                float* __restrict__ out2, int nz, int ny, int nx, int axis, int len, const float* pilot_at,
                                int square_in) {
    const float pilot = square_in ? __ldg(pilot_at) : 0.0f;
    const int64_t n = (int64_t)nz * ny * nx;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int x = (int)(i % nx);
    const int64_t r = i / nx;
    const int y = (int)(r % ny), z = (int)(r / ny);
    const int64_t stride = axis == 0 ? 1 : (axis == 1 ? (int64_t)nx : (int64_t)nx * ny);
    const int pos = axis == 0 ? x : (axis == 1 ? y : z);
    const int extent = axis == 0 ? nx : (axis == 1 ? ny : nz);
    const int m = min(len, extent - pos);  // partial sums past the last placement are never read
    float s1 = 0.0f, s2 = 0.0f;
    for (int k = 0; k < m; ++k) {
        if (square_in) {
            const float v = __ldg(in1 + i + k * stride) - pilot;
            s1 += v;
            s2 += v * v;
        } else {
            s1 += __ldg(in1 + i + k * stride);
            s2 += __ldg(in2 + i + k * stride);
        }
    }
    out1[i] = s1;
    out2[i] = s2;
}

// The same box sums from shared-memory tiles: a CTA stages 32 lines x (BOX_TL + len - 1) samples once, so every
// voxel is read from HBM about (BOX_TL + len - 1) / BOX_TL times instead of len times from L2.  Each output is the
// same sequential sum as box_pass_kernel (samples past the volume end staged as zeros, which add nothing).
constexpr int BOX_TL = 128;
constexpr int BOX_MAX_LEN = 64;
constexpr int BOX_A = BOX_TL + BOX_MAX_LEN - 1;

// x axis, from g: s1 = sum (g - c), s2 = sum (g - c)^2; tile rows are 32 consecutive y of one z plane
__global__ void __launch_bounds__(256) box_tile_x_kernel(const float* __restrict__ in, float* __restrict__ out1, float* __restrict__ out2,
                                                        int ny, int nx, int len, const float* pilot_at) {
    __shared__ float tile[32 * BOX_A];
    const float pilot = __ldg(pilot_at);
    const int A = BOX_TL + len - 1;
    const int x0 = blockIdx.x * BOX_TL, y0 = blockIdx.y * 32, z = blockIdx.z;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r = warp; r < 32; r += 8) {
        const int y = y0 + r;
        if (y >= ny) break;
        const float* row = in + ((int64_t)z * ny + y) * nx;
        for (int a = lane; a < A; a += 32) tile[r * A + a] = x0 + a < nx ? __ldg(row + x0 + a) - pilot : 0.0f;
    }
    __syncthreads();
    for (int r = warp; r < 32; r += 8) {
        const int y = y0 + r;
        if (y >= ny) break;
        const int64_t ro = ((int64_t)z * ny + y) * nx;
        for (int o = lane; o < BOX_TL && x0 + o < nx; o += 32) {
            const float* t = tile + r * A + o;
            float s1 = 0.0f, s2 = 0.0f;
            for (int k = 0; k < len; ++k) {
                const float v = t[k];
                s1 += v;
                s2 = __fmaf_rn(v, v, s2);
            }
            out1[ro + x0 + o] = s1;
            out2[ro + x0 + o] = s2;
        }
    }
}

// y (AXIS 1) or z (AXIS 2) axis, summing the two partial-sum volumes of the previous pass; tile columns are 32 x
template <int AXIS>
__global__ void __launch_bounds__(256) box_tile_yz_kernel(const float* __restrict__ in1, const float* __restrict__ in2,
                                                         float* __restrict__ out1, float* __restrict__ out2, int nz, int ny, int nx,
                                                         int len) {
    __shared__ float t1[BOX_A * 32], t2[BOX_A * 32];
    const int A = BOX_TL + len - 1;
    const int n = AXIS == 1 ? ny : nz;
    const int64_t stride = AXIS == 1 ? (int64_t)nx : (int64_t)nx * ny;
    const int x0 = blockIdx.x * 32, k0 = blockIdx.y * BOX_TL;
    const int64_t base = AXIS == 1 ? (int64_t)blockIdx.z * ny * nx : (int64_t)blockIdx.z * nx;  // plane z, or row y
    const int c = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const bool col_ok = x0 + c < nx;
    for (int a = ty; a < A; a += 8) {
        const bool in = col_ok && k0 + a < n;
        const int64_t o = base + (int64_t)(k0 + a) * stride + x0 + c;
        t1[a * 32 + c] = in ? __ldg(in1 + o) : 0.0f;
        t2[a * 32 + c] = in ? __ldg(in2 + o) : 0.0f;
    }
    __syncthreads();
    if (!col_ok) return;
    for (int o = ty; o < BOX_TL && k0 + o < n; o += 8) {
        float s1 = 0.0f, s2 = 0.0f;
        for (int k = 0; k < len; ++k) {
            s1 += t1[(o + k) * 32 + c];
            s2 += t2[(o + k) * 32 + c];
        }
        const int64_t q = base + (int64_t)(k0 + o) * stride + x0 + c;
        out1[q] = s1;
        out2[q] = s2;
    }
}

struct TiledArgs {
    const float* f;
    const float* g;
    const int64_t* coords;
    const int64_t* wx0;
    const int64_t* wy0;
    const int64_t* wz0;
    const uint8_t* t_ok;
    const float* B1;
    const float* B2;
    const float* T;     // centred templates of the chunk, [node][sz][sy][sxp]
    const double* ssf;  // their sums of squares
    float* out;
    int64_t node_base, n_nodes;
    NccGeom G;
    int dz_slab;   // offset planes per CTA
    int ntile;     // thread tiles along dx
    int pitch;         // ring row pitch (floats)
    int plane_stride;  // ring plane stride (floats)
    int sxp;           // padded template row (floats, multiple of 4)
};


// Centred FP32 template of every node of a chunk (FP64 mean, FP64 sum of squares), rows padded to sxp floats.
__global__ void __launch_bounds__(256) ncc_template_kernel(TiledArgs a, float* T, double* ssf) {
    __shared__ double red[256 / 32];
    __shared__ double s_mean;
    const NccGeom& G = a.G;
    const int64_t node = a.node_base + blockIdx.x;
    const int tid = threadIdx.x;
    const int64_t x0 = a.coords[3 * node], y0 = a.coords[3 * node + 1], z0 = a.coords[3 * node + 2];
    const bool placed = x0 - G.hx >= 0 && x0 + G.hx < G.nx && y0 - G.hy >= 0 && y0 + G.hy < G.ny && z0 - G.hz >= 0 &&
                        z0 + G.hz < G.nz;
    const int n = G.sz * G.sy * a.sxp;
    float* dst = T + (int64_t)blockIdx.x * n;
    if (!a.t_ok[node] || !placed) {
        for (int i = tid; i < n; i += blockDim.x) dst[i] = 0.0f;
        if (tid == 0) ssf[blockIdx.x] = 0.0;
        return;
    }
    const int64_t sxy = (int64_t)G.nx * G.ny;
    const float inv_sxp = 1.0f / (float)a.sxp, inv_sy = 1.0f / (float)G.sy;  // indices below 2^22: fdivi is exact
    auto col = [&](int i) { return i - fdivi(i, inv_sxp) * a.sxp; };
    auto at = [&](int i) {
        const int row = fdivi(i, inv_sxp), tx = i - row * a.sxp, tz = fdivi(row, inv_sy), ty = row - tz * G.sy;
        return __ldg(a.f + (z0 - G.hz + tz) * sxy + (y0 - G.hy + ty) * G.nx + (x0 - G.hx + tx));
    };
    double sf = 0.0;
    for (int i = tid; i < n; i += blockDim.x)
        if (col(i) < G.sx) sf += (double)at(i);
    const int lane = tid & 31, warp = tid >> 5;
    sf = warp_sum_d(sf);
    if (lane == 0) red[warp] = sf;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        s_mean = t / (double)G.n_tpl;
    }
    __syncthreads();
    const double mf = s_mean;
    double q = 0.0;
    for (int i = tid; i < n; i += blockDim.x) {
        float v = 0.0f;
        if (col(i) < G.sx) {
            const double d = (double)at(i) - mf;
            q += d * d;
            v = (float)d;
        }
        dst[i] = v;
    }
    q = warp_sum_d(q);
    __syncthreads();
    if (lane == 0) red[warp] = q;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        ssf[blockIdx.x] = t;
    }
}

__device__ __forceinline__ void cp_async16(float* dst, const float* src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(src));
}

// One CTA per (node, slab of DZ offset planes).  Thread (dzl, tile, dy pair) owns R consecutive dx outputs in
// two adjacent dy rows: every window row it loads into registers serves two template rows (R * SX FMAs each),
// so one shared load feeds about 2 * R * SX / (R + SX + SX / 2) FMAs.  Window and template stream through
// shared memory one z-plane at a time (rings of DZ + 2 window planes and 3 template planes); cp.async keeps
// the next planes in flight while the current ones are used (wait_group 1), so a step waits only for data
// issued a step earlier.  Template rows are read as float4 broadcasts.  Partial sums: FP32 per template
// plane (sy * sx terms), then FP32 across planes; the peak is settled later on FP64 re-scores.
template <int SX, int R>
__global__ void __launch_bounds__(512, 1) ncc_tiled_kernel(TiledArgs a) {
    extern __shared__ __align__(16) float sm[];
    constexpr int SXP = (SX + 3) / 4 * 4;
    const NccGeom& G = a.G;
    const int64_t node = a.node_base + blockIdx.y;
    if (node >= a.n_nodes) return;
    const int DZ = a.dz_slab;
    const int NS = DZ + 2;
    const int dz0 = blockIdx.x * DZ;
    float* out = a.out + (int64_t)blockIdx.y * G.nmap;
    const int tid = threadIdx.x;
    const int npair = (G.vy + 1) / 2;
    const int dyp = tid % npair;
    const int rest = tid / npair;
    const int tile = rest % a.ntile;
    const int dzl = rest / a.ntile;
    const int dz = dz0 + dzl;
    const bool worker = dzl < DZ && dz < G.vz;
    const int dy0 = 2 * dyp;
    const bool has1 = dy0 + 1 < G.vy;
    const int dxb = tile * R;

    const int64_t x0 = a.coords[3 * node], y0 = a.coords[3 * node + 1], z0 = a.coords[3 * node + 2];
    const int64_t wx0 = a.wx0[node], wy0 = a.wy0[node], wz0 = a.wz0[node];
    const bool placed = x0 - G.hx >= 0 && x0 + G.hx < G.nx && y0 - G.hy >= 0 && y0 + G.hy < G.ny && z0 - G.hz >= 0 &&
                        z0 + G.hz < G.nz && wx0 >= 0 && wx0 + G.wx <= G.nx && wy0 >= 0 && wy0 + G.wy <= G.ny && wz0 >= 0 &&
                        wz0 + G.wz <= G.nz;
    const double ssf = a.ssf[blockIdx.y];
    auto write_all = [&](float v) {
        if (!worker) return;
        for (int q = 0; q < 2; ++q) {
            const int dy = dy0 + q;
            if (dy >= G.vy) continue;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int dx = dxb + r;
                if (dx < G.vx) out[((int64_t)dz * G.vy + dy) * G.vx + dx] = v;
            }
        }
    };
    if (!a.t_ok[node] || !placed || ssf < 1e-20) {
        write_all(-2.0f);
        return;
    }
    const int tplane = G.sy * SXP;
    float* tring = sm;               // [3][sy][SXP]
    float* ring = sm + 3 * tplane;   // [NS][plane_stride]
    const float* Tg = a.T + (int64_t)blockIdx.y * G.sz * tplane;
    const int64_t sxy = (int64_t)G.nx * G.ny;
    const int nplanes = min(DZ, G.vz - dz0) + G.sz - 1;  // window planes this slab reads
    auto load_planes = [&](int p, int t) {
        if (p < nplanes) {
            float* dst = ring + (p % NS) * a.plane_stride;
            const float* src = a.g + (wz0 + dz0 + p) * sxy + wy0 * G.nx + wx0;
            for (int e = tid; e < G.wy * G.wx; e += blockDim.x) {
                const int yy = e / G.wx, xx = e - yy * G.wx;
                cp_async4(dst + yy * a.pitch + xx, src + (int64_t)yy * G.nx + xx);
            }
        }
        if (t < G.sz) {
            float* dst = tring + (t % 3) * tplane;
            const float* src = Tg + (int64_t)t * tplane;
            for (int e = tid; e < tplane / 4; e += blockDim.x) cp_async16(dst + 4 * e, src + 4 * e);
        }
    };
    for (int p = 0; p < DZ; ++p) load_planes(p, p == 0 ? 0 : G.sz);
    cp_async_commit();
    load_planes(DZ, 1);
    cp_async_commit();

    float tot0[R], tot1[R];
#pragma unroll
    for (int r = 0; r < R; ++r) tot0[r] = tot1[r] = 0.0f;
    for (int tz = 0; tz < G.sz; ++tz) {
        asm volatile("cp.async.wait_group 1;\n" ::);
        __syncthreads();  // window planes tz .. tz+DZ-1 and template plane tz landed; slots of step tz-1 are free
        load_planes(tz + DZ + 1, tz + 2);
        cp_async_commit();
        if (worker) {
            const float* Wp = ring + ((tz + dzl) % NS) * a.plane_stride + dy0 * a.pitch + dxb;
            const float* Tp = tring + (tz % 3) * tplane;
            float acc0[R], acc1[R];
#pragma unroll
            for (int r = 0; r < R; ++r) acc0[r] = acc1[r] = 0.0f;
            const int last = has1 ? G.sy : G.sy - 1;
            for (int ty = 0; ty <= last; ++ty) {
                const float* wr = Wp + ty * a.pitch;
                float w[R + SX - 1];
#pragma unroll
                for (int k = 0; k < R + SX - 1; ++k) w[k] = wr[k];
                if (ty < G.sy) {
                    const float4* t4 = reinterpret_cast<const float4*>(Tp + ty * SXP);
#pragma unroll
                    for (int q = 0; q < SXP / 4; ++q) {
                        const float4 tv = t4[q];
                        const float tq[4] = {tv.x, tv.y, tv.z, tv.w};
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            if (4 * q + u < SX) {
#pragma unroll
                                for (int r = 0; r < R; ++r) acc0[r] = fmaf(tq[u], w[4 * q + u + r], acc0[r]);
                            }
                        }
                    }
                }
                if (ty >= 1 && has1) {
                    const float4* t4 = reinterpret_cast<const float4*>(Tp + (ty - 1) * SXP);
#pragma unroll
                    for (int q = 0; q < SXP / 4; ++q) {
                        const float4 tv = t4[q];
                        const float tq[4] = {tv.x, tv.y, tv.z, tv.w};
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            if (4 * q + u < SX) {
#pragma unroll
                                for (int r = 0; r < R; ++r) acc1[r] = fmaf(tq[u], w[4 * q + u + r], acc1[r]);
                            }
                        }
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
                tot0[r] += acc0[r];
                tot1[r] += acc1[r];
            }
        }
    }
    asm volatile("cp.async.wait_all;\n" ::);
    if (!worker) return;
    const double n_tpl = (double)G.n_tpl;
    for (int q = 0; q < 2; ++q) {
        const int dy = dy0 + q;
        if (dy >= G.vy) continue;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int dx = dxb + r;
            if (dx >= G.vx) continue;
            const int64_t c = (wz0 + dz) * sxy + (wy0 + dy) * G.nx + (wx0 + dx);
            const double s1 = (double)__ldg(a.B1 + c), s2 = (double)__ldg(a.B2 + c);
            const double var = s2 - s1 * s1 / n_tpl;
            float v = 0.0f;
            if (!(var < 1e-20)) {
                double qv = (double)(q == 0 ? tot0[r] : tot1[r]) / sqrt(var * ssf);
                qv = qv > 1.0 ? 1.0 : (qv < -1.0 ? -1.0 : qv);
                v = (float)qv;
            }
            out[((int64_t)dz * G.vy + dy) * G.vx + dx] = v;
        }
    }
}

struct TiledCfg {
    int R, ntile, dz, threads, pitch, plane_stride, sxp;
    size_t smem;
};

static bool tiled_supported(int sx) {
    switch (sx) {
        case 5: case 7: case 9: case 11: case 13: case 15: case 17: case 21: case 25: case 33: return true;
        default: return false;
    }
}

// Shared wavefronts of one window-row load, summed over the CTA's warps and over the ring rotations,
// for the lane layout of ncc_tiled_kernel (dy pair fastest, then tile, then dz plane).
static long long ring_wavefronts(const NccGeom& G, const TiledCfg& c, int pitch, int pstride) {
    const int npair = (G.vy + 1) / 2, NS = c.dz + 2;
    const int n = c.dz * c.ntile * npair;
    long long total = 0;
    for (int rot = 0; rot < NS; ++rot)
        for (int w0 = 0; w0 < n; w0 += 32) {
            int count[32] = {0};
            long long seen[32][32];
            int worst = 1;
            for (int l = w0; l < std::min(n, w0 + 32); ++l) {
                const int dyp = l % npair, rest = l / npair, tile = rest % c.ntile, dzl = rest / c.ntile;
                const long long addr = (long long)((rot + dzl) % NS) * pstride + 2LL * dyp * pitch + (long long)tile * c.R;
                const int b = (int)(addr % 32);
                bool dup = false;
                for (int k = 0; k < count[b]; ++k) dup = dup || seen[b][k] == addr;
                if (!dup) seen[b][count[b]++] = addr;
                worst = std::max(worst, count[b]);
            }
            total += worst;
        }
    return total;
}

static size_t tiled_smem(const NccGeom& G, const TiledCfg& c, int dz, int plane_stride) {
    const size_t tail = 64;  // the discarded tail outputs of the last tile read up to R + SX floats past the last row
    return ((size_t)3 * G.sy * c.sxp + (size_t)(dz + 2) * plane_stride + tail) * sizeof(float);
}

static bool tiled_config(const NccGeom& G, TiledCfg& c) {
    static std::mutex mu;
    static bool have = false;
    static NccGeom lastG;
    static TiledCfg lastC;
    std::lock_guard<std::mutex> lock(mu);
    if (have && std::memcmp(&lastG, &G, sizeof(G)) == 0) {
        c = lastC;
        return true;
    }
    if (!tiled_supported(G.sx)) return false;
    const int w9 = ((G.vx + 8) / 9) * 9 - G.vx, w11 = ((G.vx + 10) / 11) * 11 - G.vx;
    c.R = w11 <= w9 ? 11 : 9;
    c.ntile = (G.vx + c.R - 1) / c.R;
    c.sxp = (G.sx + 3) / 4 * 4;
    const int npair = (G.vy + 1) / 2;
    const int per_plane = npair * c.ntile;
    if (per_plane > 512) return false;
    const size_t smax = (size_t)max_smem_optin() - 8192;
    const int max_stride = G.wy * (G.wx + 7) + 31;
    int best = 0;
    double best_cost = 1e300;
    for (int dz = 1; dz <= G.vz && dz * per_plane <= 512; ++dz) {
        if (tiled_smem(G, c, dz, max_stride) > smax) break;
        const int slabs = (G.vz + dz - 1) / dz;
        // thread-slots per template plane (idle tail planes included) plus the per-CTA plane loads
        const double cost = (double)slabs * dz * per_plane * (G.sy + 1) * G.sx +
                            (double)slabs * (dz + G.sz) * G.wy * G.wx * 2.0;
        if (cost < best_cost) {
            best_cost = cost;
            best = dz;
        }
    }
    if (best == 0) return false;
    c.dz = best;
    c.threads = (best * per_plane + 31) / 32 * 32;
    // ring geometry with the fewest shared wavefronts for this lane layout
    long long best_w = -1;
    for (int pitch = G.wx; pitch < G.wx + 8; ++pitch)
        for (int pad = 0; pad < 32; ++pad) {
            const int ps = G.wy * pitch + pad;
            const long long wv = ring_wavefronts(G, c, pitch, ps);
            if (best_w < 0 || wv < best_w) {
                best_w = wv;
                c.pitch = pitch;
                c.plane_stride = ps;
            }
        }
    c.smem = tiled_smem(G, c, best, c.plane_stride);
    if (c.smem > smax) return false;
    lastG = G;
    lastC = c;
    have = true;
    return true;
}

// Template scratch of the tiled engine for a chunk of nodes: centred templates, then their sums of squares.
static size_t tiled_tpl_bytes(const NccGeom& G, int64_t chunk) {
    const int sxp = (G.sx + 3) / 4 * 4;
    return align_up((size_t)chunk * G.sz * G.sy * sxp * sizeof(float), 256) + align_up((size_t)chunk * sizeof(double), 256);
}

template <int SX, int R>
static int launch_tiled_t(const TiledArgs& a, const TiledCfg& c, int64_t n_chunk, cudaStream_t s) {
    auto kern = ncc_tiled_kernel<SX, R>;
    static size_t attr = 48 * 1024;
    if (c.smem > attr) {
        const size_t want = (size_t)max_smem_optin() - 4096;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)want);
        if (e != cudaSuccess) return cuda_fail(e, "ncc tiled: shared memory attribute");
        attr = want;
    }
    const unsigned slabs = (unsigned)((a.G.vz + c.dz - 1) / c.dz);
    const int64_t tsz = (int64_t)a.G.sz * a.G.sy * c.sxp;
    for (int64_t done = 0; done < n_chunk; done += 65535) {
        const unsigned nb = (unsigned)std::min<int64_t>(65535, n_chunk - done);
        TiledArgs aa = a;
        aa.node_base = a.node_base + done;
        aa.out = a.out + done * a.G.nmap;
        aa.T = a.T + done * tsz;
        aa.ssf = a.ssf + done;
        {
            KTimer kt_("ncc_template", s);
            ncc_template_kernel<<<nb, 256, 0, s>>>(aa, const_cast<float*>(aa.T), const_cast<double*>(aa.ssf));
        }
        int rc = check_launch("ncc template");
        if (rc) return rc;
        {
            KTimer kt_("ncc_tiled", s);
            kern<<<dim3(slabs, nb), c.threads, c.smem, s>>>(aa);
        }
        rc = check_launch("ncc tiled");
        if (rc) return rc;
    }
    return ALDVC_OK;
}

template <int SX>
static int launch_tiled_sx(const TiledArgs& a, const TiledCfg& c, int64_t n, cudaStream_t s) {
    return c.R == 11 ? launch_tiled_t<SX, 11>(a, c, n, s) : launch_tiled_t<SX, 9>(a, c, n, s);
}

static int launch_tiled(const TiledArgs& a, const TiledCfg& c, int64_t n, cudaStream_t s) {
    switch (a.G.sx) {
        case 5: return launch_tiled_sx<5>(a, c, n, s);
        case 7: return launch_tiled_sx<7>(a, c, n, s);
        case 9: return launch_tiled_sx<9>(a, c, n, s);
        case 11: return launch_tiled_sx<11>(a, c, n, s);
        case 13: return launch_tiled_sx<13>(a, c, n, s);
        case 15: return launch_tiled_sx<15>(a, c, n, s);
        case 17: return launch_tiled_sx<17>(a, c, n, s);
        case 21: return launch_tiled_sx<21>(a, c, n, s);
        case 25: return launch_tiled_sx<25>(a, c, n, s);
        default: return launch_tiled_sx<33>(a, c, n, s);
    }
}

// ----------------------------------------------------------------------------- FFT engine
// Cross term by FFT (integer_search.py:423-443 computes it with rfftn/irfftn): C = IFFT(FFT(W) conj(FFT(T))),
// valid offsets only, with transform lengths N >= window extent (2,3,5-smooth), so no offset wraps.
// The window W (minus the same pilot voxel as the box sums) and the centred template T are packed into one
// complex volume Z = W + iT, whose spectrum gives both: W^[k] = (Z^[k] + conj Z^[-k]) / 2 and
// T^[k] = (Z^[k] - conj Z^[-k]) / 2i.  Three passes per batch of nodes, each a CTA-wide Stockham FFT in
// shared memory (radix 2/3/4/5 stages, twiddles from a device table):
//   1. per window z-plane: FFT along x (rows < wy), then along y; plane spectrum to scratch A.
//   2. per (ky, -ky) row pair: FFT along z, the product W^ conj T^, inverse FFT along z; planes dz < vz to P.
//   3. per dz plane: inverse FFT along y, then along x (rows < vy); real part / (Nx Ny Nz) is the cross term,
//      normalised with the box-sum volumes as in the tiled engine.
constexpr int FFT_MAX_N = 128;
constexpr int FFT_THREADS = 256;

struct FftAxis {
    int n, stages;
    int radix[8];
};

struct FftArgs {
    const float* g;
    const int64_t* coords;
    const int64_t* wx0;
    const int64_t* wy0;
    const int64_t* wz0;
    const uint8_t* t_ok;
    const float* B1;
    const float* B2;
    const float* T;     // centred templates of the chunk, [node][sz][sy][sxp]
    const double* ssf;  // their sums of squares
    const float* pilot_at;
    const float2* tw;   // twiddle tables: x at 0, y at FFT_MAX_N, z at 2 FFT_MAX_N
    float2* A;          // [nb][wz][Ny][Nx]
    float2* P;          // [nb][vz][Ny][Nx]
    float* out;         // maps of the batch
    MapPart* part;      // per-block map partials of the batch ([node][nblk]) or null (in-register pass 3 only)
    int nblk;
    int64_t node_base;  // first node of the batch
    int64_t n_nodes;
    int nb;
    NccGeom G;
    int sxp;
    FftAxis ax, ay, az;
    int pitch;          // shared row pitch in float2 (odd)
};

__host__ inline bool fft_axis(int n, FftAxis& a) {
    a.n = n;
    a.stages = 0;
    int m = n;
    while (m % 4 == 0) { a.radix[a.stages++] = 4; m /= 4; }
    while (m % 2 == 0) { a.radix[a.stages++] = 2; m /= 2; }
    while (m % 3 == 0) { a.radix[a.stages++] = 3; m /= 3; }
    while (m % 5 == 0) { a.radix[a.stages++] = 5; m /= 5; }
    return m == 1 && a.stages <= 8 && n <= FFT_MAX_N;
}

__host__ inline int smooth_len(int n) {
    for (int m = n;; ++m) {
        int k = m;
        while (k % 2 == 0) k /= 2;
        while (k % 3 == 0) k /= 3;
        while (k % 5 == 0) k /= 5;
        if (k == 1) return m;
    }
}

__global__ void fft_twiddle_kernel(float2* tw, int nx, int ny, int nz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * FFT_MAX_N) return;
    const int axis = i / FFT_MAX_N, k = i % FFT_MAX_N;
    const int n = axis == 0 ? nx : (axis == 1 ? ny : nz);
    double s = 0.0, c = 1.0;
    if (k < n) sincospi(-2.0 * (double)k / (double)n, &s, &c);
    tw[i] = make_float2((float)c, (float)s);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// multiply by sgn * i
__device__ __forceinline__ float2 cmuli(float2 a, float sgn) { return make_float2(-sgn * a.y, sgn * a.x); }

// In-register R-point DFT, exponent sign sgn (-1 forward, +1 inverse).
template <int R>
__device__ __forceinline__ void small_dft(float2* v, float sgn) {
    if (R == 2) {
        const float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if (R == 4) {
        const float2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]), s13 = cadd(v[1], v[3]), d13 = cmuli(csub(v[1], v[3]), sgn);
        v[0] = cadd(s02, s13);
        v[2] = csub(s02, s13);
        v[1] = cadd(d02, d13);
        v[3] = csub(d02, d13);
    } else if (R == 3) {
        const float c1 = -0.5f, s1 = 0.86602540378443864676f;  // cos, sin of 2 pi / 3
        const float2 a = v[0], b = v[1], c = v[2];
        const float2 t = cadd(b, c), u = cmuli(csub(b, c), sgn * s1);
        v[0] = cadd(a, t);
        const float2 m = make_float2(a.x + c1 * t.x, a.y + c1 * t.y);
        v[1] = cadd(m, u);
        v[2] = csub(m, u);
    } else {  // R == 5
        const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;  // cos 2pi/5, cos 4pi/5
        const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;   // sin 2pi/5, sin 4pi/5
        const float2 a = v[0];
        const float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
        const float2 d1 = csub(v[1], v[4]), d2 = csub(v[2], v[3]);
        v[0] = cadd(a, cadd(t1, t2));
        const float2 m1 = make_float2(a.x + c1 * t1.x + c2 * t2.x, a.y + c1 * t1.y + c2 * t2.y);
        const float2 m2 = make_float2(a.x + c2 * t1.x + c1 * t2.x, a.y + c2 * t1.y + c1 * t2.y);
        // sgn i (s1 d1 + s2 d2) and sgn i (s2 d1 - s1 d2)
        const float2 n1 = cmuli(make_float2(s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y), sgn);
        const float2 n2 = cmuli(make_float2(s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y), sgn);
        v[1] = cadd(m1, n1);
        v[4] = csub(m1, n1);
        v[2] = cadd(m2, n2);
        v[3] = csub(m2, n2);
    }
}

// One radix-R Stockham stage over `rows` transforms.  Butterfly b of this thread walks (row fastest, then j)
// with incremental indices, so the loop holds no integer division; j / ns uses a multiply-high by the
// precomputed reciprocal (exact for j, ns < 2^16).  Rows q >= split sit split_stride further (rows <= 2 split).
template <int R>
__device__ __forceinline__ void stockham_stage(const float2* __restrict__ d0, float2* __restrict__ d1, const float2* tw, int n,
                                               int ns, int rows, int split, int split_stride, int row_stride, int es, float sgn) {
    const int m = n / R;
    const int total = rows * m;
    const int tstep = n / (ns * R);
    // ceil(2^32 / ns) for ns >= 2 (ns == 1 is handled apart: its reciprocal does not fit 32 bits)
    const unsigned mag = ns > 1 ? (unsigned)((0x100000000ull + (unsigned long long)ns - 1) / (unsigned long long)ns) : 0u;
    const int nt = blockDim.x, drow = nt % rows, dj = nt / rows;
    int row = threadIdx.x % rows, j = threadIdx.x / rows;
    for (int b = threadIdx.x; b < total; b += nt) {
        const int base = row < split ? row * row_stride : split_stride + (row - split) * row_stride;
        const int q = ns > 1 ? (int)__umulhi((unsigned)j, mag) : j;
        const int k = j - q * ns;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            float2 x = d0[base + (j + r * m) * es];
            if (r > 0 && k > 0) {
                float2 w = tw[r * k * tstep];  // r k tstep < n
                w.y *= -sgn;                   // the table holds exp(-2 pi i k / n); sgn = +1 conjugates it
                x = cmul(x, w);
            }
            v[r] = x;
        }
        small_dft<R>(v, sgn);
        const int od = q * ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) d1[base + (od + r * ns) * es] = v[r];
        row += drow;
        j += dj;
        if (row >= rows) {
            row -= rows;
            ++j;
        }
    }
}

// `rows` independent transforms along one axis; row q starts at q * row_stride, or at
// split_stride + (q - split) * row_stride for q >= split (rows <= 2 split), its elements es apart.
// Ping-pongs between a and b; returns the buffer holding the result.
__device__ float2* fft_rows(float2* a, float2* b, const float2* tw, const FftAxis& ax, int rows, int split, int split_stride,
                            int row_stride, int es, float sgn) {
    int ns = 1;
    for (int s = 0; s < ax.stages; ++s) {
        const int R = ax.radix[s];
        if (R == 4)
            stockham_stage<4>(a, b, tw, ax.n, ns, rows, split, split_stride, row_stride, es, sgn);
        else if (R == 2)
            stockham_stage<2>(a, b, tw, ax.n, ns, rows, split, split_stride, row_stride, es, sgn);
        else if (R == 3)
            stockham_stage<3>(a, b, tw, ax.n, ns, rows, split, split_stride, row_stride, es, sgn);
        else
            stockham_stage<5>(a, b, tw, ax.n, ns, rows, split, split_stride, row_stride, es, sgn);
        __syncthreads();
        float2* t = a;
        a = b;
        b = t;
        ns *= R;
    }
    return a;
}

__device__ __forceinline__ bool fft_node_ok(const FftArgs& a, int64_t node) {
    const NccGeom& G = a.G;
    const int64_t x0 = a.coords[3 * node], y0 = a.coords[3 * node + 1], z0 = a.coords[3 * node + 2];
    const int64_t wx0 = a.wx0[node], wy0 = a.wy0[node], wz0 = a.wz0[node];
    const bool placed = x0 - G.hx >= 0 && x0 + G.hx < G.nx && y0 - G.hy >= 0 && y0 + G.hy < G.ny && z0 - G.hz >= 0 &&
                        z0 + G.hz < G.nz && wx0 >= 0 && wx0 + G.wx <= G.nx && wy0 >= 0 && wy0 + G.wy <= G.ny && wz0 >= 0 &&
                        wz0 + G.wz <= G.nz;
    return placed && a.t_ok[node] && !(a.ssf[node - a.node_base] < 1e-20);
}

// Pass 1: grid (wz, nb).  Shared: two planes Ny x pitch float2 and the x/y twiddles.
__global__ void __launch_bounds__(FFT_THREADS, 4) fft_pass1_kernel(FftArgs a) {
    extern __shared__ __align__(16) float2 fsm[];
    const NccGeom& G = a.G;
    const int z = blockIdx.x;
    const int64_t node = a.node_base + blockIdx.y;
    if (!fft_node_ok(a, node)) return;
    const int Nx = a.ax.n, Ny = a.ay.n, pitch = a.pitch;
    float2* b0 = fsm;
    float2* b1 = fsm + Ny * pitch;
    float2* twx = b1 + Ny * pitch;
    float2* twy = twx + FFT_MAX_N;
    for (int i = threadIdx.x; i < 2 * FFT_MAX_N; i += blockDim.x) twx[i] = a.tw[i];
    const int64_t sxy = (int64_t)G.nx * G.ny;
    const float pilot = __ldg(a.pilot_at);
    const float* src = a.g + (a.wz0[node] + z) * sxy + a.wy0[node] * G.nx + a.wx0[node];
    const float* tsrc = a.T + (int64_t)blockIdx.y * G.sz * G.sy * a.sxp + (int64_t)z * G.sy * a.sxp;
    const bool tpl_plane = z < G.sz;
    copy_rows<4, float2>(
        Ny, Nx,
        [&](int y, int x) {
            float2 v = make_float2(0.0f, 0.0f);
            if (y < G.wy && x < G.wx) v.x = __ldg(src + (int64_t)y * G.nx + x) - pilot;
            if (tpl_plane && y < G.sy && x < G.sx) v.y = __ldg(tsrc + y * a.sxp + x);
            return v;
        },
        [&](int y, int x, float2 v) {
            b0[y * pitch + x] = v;
            b1[y * pitch + x] = make_float2(0.0f, 0.0f);
        });
    __syncthreads();
    float2* r = fft_rows(b0, b1, twx, a.ax, G.wy, G.wy, 0, pitch, 1, -1.0f);  // along x, rows y < wy
    float2* o = r == b0 ? b1 : b0;
    r = fft_rows(r, o, twy, a.ay, Nx, Nx, 0, 1, pitch, -1.0f);  // along y, every column
    float2* dst = a.A + ((int64_t)blockIdx.y * G.wz + z) * Ny * Nx;
    copy_rows<1, float2>(Ny, Nx, [&](int y, int x) { return r[y * pitch + x]; }, [&](int y, int x, float2 v) { dst[y * Nx + x] = v; });
}

// Pass 2: grid (2 (Ny / 2 + 1), nb).  Block (p, h) takes row ky = p and its mirror (Ny - ky) mod Ny.  A row that
// is its own mirror (ky = 0, Ny / 2) is done whole by h = 0.  Otherwise h takes the columns
// kx in [h cb, (h + 1) cb) of row ky and the mirrored columns (Nx - kx) mod Nx of the mirror row, stored at the
// same local index, so Z^[-k] of a column sits in the other row at the same index.
__global__ void __launch_bounds__(FFT_THREADS, 4) fft_pass2_kernel(FftArgs a) {
    extern __shared__ __align__(16) float2 fsm[];
    const NccGeom& G = a.G;
    const int64_t node = a.node_base + blockIdx.y;
    if (!fft_node_ok(a, node)) return;
    const int Nx = a.ax.n, Ny = a.ay.n, Nz = a.az.n;
    const int ky0 = blockIdx.x >> 1, half = blockIdx.x & 1, ky1 = (Ny - ky0) % Ny;
    const bool self = ky1 == ky0;
    if (self && half) return;
    const int cb = (Nx + 1) / 2;
    const int c0 = self ? 0 : half * cb;
    const int ncol = self ? Nx : min(cb, Nx - c0);
    const int cp = self ? a.pitch : (cb | 1);  // odd column pitch
    const int nrow = self ? 1 : 2;
    const int plane = Nz * cp;
    float2* b0 = fsm;
    float2* b1 = fsm + nrow * plane;
    float2* twz = fsm + 2 * max(a.pitch, 2 * (cb | 1)) * Nz;
    for (int i = threadIdx.x; i < FFT_MAX_N; i += blockDim.x) twz[i] = a.tw[2 * FFT_MAX_N + i];
    const float2* A = a.A + (int64_t)blockIdx.y * G.wz * Ny * Nx;
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    copy_rows<4, float2>(
        nrow * Nz, ncol,
        [&](int zr, int c) {
            const int q = zr >= Nz ? 1 : 0, z = zr - q * Nz;
            const int kx = q == 0 ? c0 + c : (Nx - c0 - c) % Nx;
            return z < G.wz ? A[((int64_t)z * Ny + (q == 0 ? ky0 : ky1)) * Nx + kx] : make_float2(0.0f, 0.0f);
        },
        [&](int zr, int c, float2 v) {
            const int q = zr >= Nz ? 1 : 0, z = zr - q * Nz;
            b0[q * plane + z * cp + c] = v;
        });
    __syncthreads();
    float2* r = fft_rows(b0, b1, twz, a.az, nrow * ncol, ncol, plane, 1, cp, -1.0f);  // along z
    float2* o = r == b0 ? b1 : b0;
    // product W^ conj(T^) from Z^[k] and Z^[-k]
    for (int zr = threadIdx.x >> 5; zr < nrow * Nz; zr += nw)
        for (int c = lane; c < ncol; c += 32) {
            const int q = zr >= Nz ? 1 : 0, kz = zr - q * Nz;
            const int kzm = (Nz - kz) % Nz;
            const int qm = self ? 0 : 1 - q, cm = self ? (Nx - c) % Nx : c;
            const float2 za = r[q * plane + kz * cp + c];
            const float2 zb = r[qm * plane + kzm * cp + cm];
            const float2 zbc = make_float2(zb.x, -zb.y);
            const float2 w = make_float2(0.5f * (za.x + zbc.x), 0.5f * (za.y + zbc.y));
            // T^ = (za - zbc) / 2i = -i (za - zbc) / 2;  conj(T^) = i conj(za - zbc) / 2
            const float2 d = csub(za, zbc);
            const float2 tc = make_float2(0.5f * d.y, 0.5f * d.x);  // i * conj(d) / 2 = (d.y + i d.x) / 2
            o[q * plane + kz * cp + c] = cmul(w, tc);
        }
    __syncthreads();
    float2* r2 = fft_rows(o, r, twz, a.az, nrow * ncol, ncol, plane, 1, cp, 1.0f);  // inverse along z
    float2* P = a.P + (int64_t)blockIdx.y * G.vz * Ny * Nx;
    for (int zr = threadIdx.x >> 5; zr < nrow * G.vz; zr += nw) {
        const int q = zr >= G.vz ? 1 : 0, z = zr - q * G.vz;
        float2* dst = P + ((int64_t)z * Ny + (q == 0 ? ky0 : ky1)) * Nx;
        for (int c = lane; c < ncol; c += 32) {
            const int kx = q == 0 ? c0 + c : (Nx - c0 - c) % Nx;
            dst[kx] = r2[q * plane + z * cp + c];
        }
    }
}

// Pass 3: grid (vz, nb).  Inverse along y and x, normalisation, the map plane dz.
__global__ void __launch_bounds__(FFT_THREADS, 4) fft_pass3_kernel(FftArgs a) {
    extern __shared__ __align__(16) float2 fsm[];
    const NccGeom& G = a.G;
    const int dz = blockIdx.x;
    const int64_t node = a.node_base + blockIdx.y;
    float* out = a.out + (int64_t)blockIdx.y * G.nmap + (int64_t)dz * G.vy * G.vx;
    if (!fft_node_ok(a, node)) {
        for (int i = threadIdx.x; i < G.vy * G.vx; i += blockDim.x) out[i] = -2.0f;
        return;
    }
    const int Nx = a.ax.n, Ny = a.ay.n, Nz = a.az.n, pitch = a.pitch;
    float2* b0 = fsm;
    float2* b1 = fsm + Ny * pitch;
    float2* twx = b1 + Ny * pitch;
    float2* twy = twx + FFT_MAX_N;
    for (int i = threadIdx.x; i < 2 * FFT_MAX_N; i += blockDim.x) twx[i] = a.tw[i];
    const float2* P = a.P + ((int64_t)blockIdx.y * G.vz + dz) * Ny * Nx;
    copy_rows<4, float2>(Ny, Nx, [&](int y, int x) { return P[y * Nx + x]; }, [&](int y, int x, float2 v) { b0[y * pitch + x] = v; });
    __syncthreads();
    float2* r = fft_rows(b0, b1, twy, a.ay, Nx, Nx, 0, 1, pitch, 1.0f);  // inverse along y
    float2* o = r == b0 ? b1 : b0;
    r = fft_rows(r, o, twx, a.ax, G.vy, G.vy, 0, pitch, 1, 1.0f);  // inverse along x, rows dy < vy
    const double scale = 1.0 / ((double)Nx * Ny * Nz);
    const double ssf = a.ssf[blockIdx.y], n_tpl = (double)G.n_tpl;
    const int64_t sxy = (int64_t)G.nx * G.ny;
    const int64_t wz0 = a.wz0[node], wy0 = a.wy0[node], wx0 = a.wx0[node];
    const float* B1 = a.B1 + (wz0 + dz) * sxy + wy0 * G.nx + wx0;
    const float* B2 = a.B2 + (wz0 + dz) * sxy + wy0 * G.nx + wx0;
    copy_rows<4, float2>(
        G.vy, G.vx, [&](int dy, int dx) { return make_float2(__ldg(B1 + (int64_t)dy * G.nx + dx), __ldg(B2 + (int64_t)dy * G.nx + dx)); },
        [&](int dy, int dx, float2 bs) {
            const double s1 = (double)bs.x, s2 = (double)bs.y;
            const double var = s2 - s1 * s1 / n_tpl;
            float v = 0.0f;
            if (!(var < 1e-20)) {
                double qv = (double)r[dy * pitch + dx].x * scale / sqrt(var * ssf);
                qv = qv > 1.0 ? 1.0 : (qv < -1.0 ? -1.0 : qv);
                v = (float)qv;
            }
            out[dy * G.vx + dx] = v;
        });
}

// ---- cubic boxes (Nx = Ny = Nz = N, a length with an in-register transform): the same three passes, each line
// transformed by one thread in registers (fft_line), shared memory only to turn lines between axes.
// Planes per CTA: as many as keep its shared tile near 70 KB (3 CTAs per SM), at most 256 / N.
template <int N>
__host__ __device__ constexpr int fftr_planes() {
    constexpr int by_smem = 70000 / (N * (N | 1) * 8);
    constexpr int by_threads = 256 / N;
    return by_smem < 1 ? 1 : (by_smem < by_threads ? by_smem : by_threads);
}

// Pass 1: thread (plane, y) reads its window row straight into registers, transforms along x, parks the row in
// shared memory; then thread (plane, x) transforms the column along y and the planes go out coalesced.
__device__ __forceinline__ float f4c(const float4& c, int i) { return i == 0 ? c.x : (i == 1 ? c.y : (i == 2 ? c.z : c.w)); }

// window row of wx samples starting O floats past the 16-byte aligned `base`: v[x].x = sample - pilot, 0 past wx;
// chunks holding none of the row's samples are not read
template <int N, int O>
__device__ __forceinline__ void fftr_row4(const float* base, int wx, float pilot, float2 (&v)[N]) {
    constexpr int NCH = (N + O + 3) / 4;
    float4 ch[NCH];
#pragma unroll
    for (int c = 0; c < NCH; ++c)
        ch[c] = 4 * c < wx + O ? __ldg(reinterpret_cast<const float4*>(base) + c) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
    for (int x = 0; x < N; ++x) v[x].x = x < wx ? f4c(ch[(x + O) / 4], (x + O) % 4) - pilot : 0.0f;
}

// template row of sx samples at the 16-byte aligned `row` (padded to a multiple of 4): v[x].y, 0 past sx
template <int N>
__device__ __forceinline__ void fftr_trow4(const float* row, int sx, float2 (&v)[N]) {
    constexpr int NCH = (N + 3) / 4;
    float4 ch[NCH];
#pragma unroll
    for (int c = 0; c < NCH; ++c)
        ch[c] = 4 * c < sx ? __ldg(reinterpret_cast<const float4*>(row) + c) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
    for (int x = 0; x < N; ++x) v[x].y = x < sx ? f4c(ch[x / 4], x % 4) : 0.0f;
}

// three CTAs per SM for the longer lines: measured faster than two at the register count the 16-byte loads reach
// (16.3 against 17.6 ms for N = 50 on a 29,791-node probe, a few spilled registers included)
template <int N>
__global__ void __launch_bounds__(fftr_planes<N>() * N, N >= 48 ? 3 : 1) fftr_pass1_kernel(FftArgs a) {
    constexpr int P = fftr_planes<N>();
    constexpr int PITCH = N | 1;
    extern __shared__ __align__(16) float2 fsm[];  // [P][N][PITCH]
    const NccGeom& G = a.G;
    const int64_t node = a.node_base + blockIdx.y;
    if (!fft_node_ok(a, node)) return;
    const int z0 = blockIdx.x * P;
    const int np = min(P, G.wz - z0);
    const int64_t sxy = (int64_t)G.nx * G.ny;
    const float pilot = __ldg(a.pilot_at);
    const int t = threadIdx.x;
    const int pl = t / N, yx = t - pl * N;  // row y in the x phase, column x in the y phase
    // 16-byte loads when every window row of this node starts at the same offset O within a 16-byte chunk (x extent a
    // multiple of 4, aligned volume): a thread then issues a quarter of the loads of its row
    const int O = (int)(a.wx0[node] & 3);
    const bool vec = (G.nx & 3) == 0 && (reinterpret_cast<uintptr_t>(a.g) & 15) == 0;
    const float* gend = a.g + (int64_t)G.nz * sxy;
    if (pl < np) {
        const int z = z0 + pl, y = yx;
        float2 v[N];
        const float* wrow = a.g + (a.wz0[node] + z) * sxy + (a.wy0[node] + y) * G.nx + a.wx0[node];
        const float* trow = a.T + (int64_t)blockIdx.y * G.sz * G.sy * a.sxp + ((int64_t)z * G.sy + y) * a.sxp;
        const bool wy_in = y < G.wy, ty_in = z < G.sz && y < G.sy;
        // the last 16-byte chunk of the row must stay inside the volume (its tail past the row is not used)
        const bool vrow = vec && wy_in && wrow - O + 4 * ((G.wx + O + 3) / 4) <= gend;
        if (vrow) {
            switch (O) {
                case 0: fftr_row4<N, 0>(wrow, G.wx, pilot, v); break;
                case 1: fftr_row4<N, 1>(wrow - 1, G.wx, pilot, v); break;
                case 2: fftr_row4<N, 2>(wrow - 2, G.wx, pilot, v); break;
                default: fftr_row4<N, 3>(wrow - 3, G.wx, pilot, v); break;
            }
        } else {
#pragma unroll
            for (int x = 0; x < N; ++x) v[x].x = (wy_in && x < G.wx) ? __ldg(wrow + x) - pilot : 0.0f;
        }
        if (ty_in && (a.sxp & 3) == 0) {  // template rows: padded to sxp (a multiple of 4) in an aligned buffer
            fftr_trow4<N>(trow, G.sx, v);
        } else {
#pragma unroll
            for (int x = 0; x < N; ++x) v[x].y = (ty_in && x < G.sx) ? __ldg(trow + x) : 0.0f;
        }
        if (wy_in) fft_line<N, -1>(v);  // rows past the window are zero and stay zero
        float2* row = fsm + (pl * N + y) * PITCH;
#pragma unroll
        for (int x = 0; x < N; ++x) row[x] = v[x];
    }
    __syncthreads();
    if (pl < np) {
        float2* col = fsm + pl * N * PITCH + yx;
        float2 v[N];
#pragma unroll
        for (int k = 0; k < N; ++k) v[k] = col[k * PITCH];
        fft_line<N, -1>(v);
#pragma unroll
        for (int k = 0; k < N; ++k) col[k * PITCH] = v[k];
    }
    __syncthreads();
    float2* dst = a.A + ((int64_t)blockIdx.y * G.wz + z0) * N * N;
    sweep_lin<2, float2>(np * N, N, [&](int r, int x) { return fsm[r * PITCH + x]; },
                         [&](int r, int x, float2 v) { dst[(int64_t)r * N + x] = v; });
}

// One CTA per (ky, -ky) row pair, one thread per column c: the thread transforms the z-line of column c of row
// -ky and parks it in shared memory, then transforms that of row ky in registers, forms the product with the
// partner lines and inverts it.  The product is Hermitian (the cross term is real), so its rows ky <= N/2 hold all
// of it: the product planes keep only those ([nb][vz][N/2 + 1][N]) and row -ky needs no inverse.
template <int N>
__global__ void __launch_bounds__(N, N > 50 ? 4 : 8) fftr_pass2_kernel(FftArgs a) {
    constexpr int PITCH = N | 1;
    constexpr int NH = N / 2 + 1;
    extern __shared__ __align__(16) float2 fsm[];  // spectrum of row -ky (of row ky when ky = -ky) [N][PITCH]
    const NccGeom& G = a.G;
    const int64_t node = a.node_base + blockIdx.y;
    if (!fft_node_ok(a, node)) return;
    const int ky0 = blockIdx.x, ky1 = (N - ky0) % N;
    const bool self = ky0 == ky1;
    const int c = threadIdx.x;
    const float2* An = a.A + (int64_t)blockIdx.y * G.wz * N * N;
    float2 v[N];
    if (!self) {
        const float2* col = An + ky1 * N + c;
#pragma unroll
        for (int z = 0; z < N; ++z) v[z] = z < G.wz ? col[(int64_t)z * N * N] : make_float2(0.0f, 0.0f);
        fft_line<N, -1>(v);
#pragma unroll
        for (int k = 0; k < N; ++k) fsm[k * PITCH + c] = v[k];
    }
    {
        const float2* col = An + ky0 * N + c;
#pragma unroll
        for (int z = 0; z < N; ++z) v[z] = z < G.wz ? col[(int64_t)z * N * N] : make_float2(0.0f, 0.0f);
        fft_line<N, -1>(v);
    }
    if (self) {
#pragma unroll
        for (int k = 0; k < N; ++k) fsm[k * PITCH + c] = v[k];
    }
    __syncthreads();
    const int cm = (N - c) % N;
#pragma unroll
    for (int kz = 0; kz < N; ++kz) {
        const float2 za = v[kz];
        const float2 zb = fsm[((N - kz) % N) * PITCH + cm];
        const float2 zbc = make_float2(zb.x, -zb.y);
        const float2 w = make_float2(0.5f * (za.x + zbc.x), 0.5f * (za.y + zbc.y));
        const float2 d = make_float2(za.x - zbc.x, za.y - zbc.y);
        const float2 tc = make_float2(0.5f * d.y, 0.5f * d.x);  // conj(T^) = i conj(za - zbc) / 2
        v[kz] = fr_mul(w, tc);
    }
    fft_line<N, 1>(v);
    float2* dst = a.P + (int64_t)blockIdx.y * G.vz * NH * N + ky0 * N + c;
#pragma unroll
    for (int dz = 0; dz < N; ++dz)
        if (dz < G.vz) dst[(int64_t)dz * NH * N] = v[dz];
}

#include "fft_tensor.cuh"

// Pass 3: planes per CTA of the half-spectrum tile [N][N/2 + 1 | 1] of each plane, at most 256 threads.
template <int N>
__host__ __device__ constexpr int fftr_planes3() {
    constexpr int NH = N / 2 + 1;
    constexpr int by_smem = 70000 / (N * (NH | 1) * 8);
    constexpr int by_threads = 256 / NH;
    return by_smem < 1 ? 1 : (by_smem < by_threads ? by_smem : by_threads);
}

// Pass 3: thread (plane, kx <= N/2) reads its y-column of the product straight into registers (rows ky > N/2 as
// the conjugates of rows N - ky at column N - kx: the product is Hermitian) and inverts along y; the columns
// kx > N/2 are the conjugates of these, so thread (plane, j) inverts the real rows 2j and 2j + 1 along x as ONE
// complex transform (row 2j in the real part, row 2j + 1 in the imaginary part).  The normalised map rows go out.
template <int N>
__host__ __device__ constexpr int fftr_pass3_threads() {  // whole warps (the partials reduce with full-warp shuffles)
    return (fftr_planes3<N>() * (N / 2 + 1) + 31) / 32 * 32;
}

template <int N>
__global__ void __launch_bounds__(fftr_pass3_threads<N>()) fftr_pass3_kernel(FftArgs a) {
    constexpr int NH = N / 2 + 1;
    constexpr int P = fftr_planes3<N>();
    constexpr int RP = NH | 1;
    extern __shared__ __align__(16) float2 fsm[];  // [P][N][RP]: y-inverted columns kx <= N/2; then map rows
    const NccGeom& G = a.G;
    const int64_t node = a.node_base + blockIdx.y;
    const int dz0 = blockIdx.x * P;
    const int np = min(P, G.vz - dz0);
    float* out = a.out + (int64_t)blockIdx.y * G.nmap + (int64_t)dz0 * G.vy * G.vx;
    if (!fft_node_ok(a, node)) {
        for (int i = threadIdx.x; i < np * G.vy * G.vx; i += blockDim.x) out[i] = -2.0f;
        if (a.part && threadIdx.x == 0) {  // every value counts as 0 in the peak search
            MapPart q;
            q.s1 = q.s2 = 0.0;
            q.mx = q.mn = 0.0f;
            q.idx = dz0 * G.vy * G.vx;
            q.pad = 0;
            a.part[(int64_t)blockIdx.y * a.nblk + blockIdx.x] = q;
        }
        return;
    }
    const int t = threadIdx.x;
    const int pl = t / NH, kx = t - pl * NH;
    {  // the box sums of these planes are read last: start them towards L2 while the transforms run
        const int64_t sxy = (int64_t)G.nx * G.ny, wz0 = a.wz0[node], wy0 = a.wy0[node], wx0 = a.wx0[node];
        const int nch = (G.vx + 31) / 32, per_row = 2 * nch;
        for (int i = t; i < np * G.vy * per_row; i += blockDim.x) {
            const int r = i / per_row, rem = i - r * per_row, p_ = r / G.vy, dy = r - p_ * G.vy;
            const float* b = (rem & 1) ? a.B2 : a.B1;
            prefetch_l2(b + (wz0 + dz0 + p_) * sxy + (wy0 + dy) * G.nx + wx0 + 32 * (rem >> 1));
        }
    }
    if (pl < np) {  // inverse along y of column kx <= N/2
        const float2* pg = a.P + ((int64_t)blockIdx.y * G.vz + dz0 + pl) * NH * N;
        const int kxm = (N - kx) % N;
        float2 v[N];
#pragma unroll
        for (int k = 0; k < NH; ++k) v[k] = pg[k * N + kx];
#pragma unroll
        for (int k = NH; k < N; ++k) {
            const float2 w = pg[(N - k) * N + kxm];
            v[k] = make_float2(w.x, -w.y);
        }
        fft_line<N, 1>(v);
        float2* col = fsm + pl * N * RP + kx;
#pragma unroll
        for (int k = 0; k < N; ++k) col[k * RP] = v[k];
    }
    __syncthreads();
    const int nj = (G.vy + 1) / 2;  // row pairs (2j, 2j + 1), 2j + 1 <= N - 1
    if (pl < np && kx < nj) {
        float2* ra = fsm + (pl * N + 2 * kx) * RP;
        float2* rb = ra + RP;
        const bool hb = 2 * kx + 1 < G.vy;
        float2 v[N];
#pragma unroll
        for (int k = 0; k < NH; ++k) {  // X_a + i X_b
            const float2 xa = ra[k], xb = hb ? rb[k] : make_float2(0.0f, 0.0f);
            v[k] = make_float2(xa.x - xb.y, xa.y + xb.x);
        }
#pragma unroll
        for (int k = NH; k < N; ++k) {  // conj X_a[N - k] + i conj X_b[N - k]
            const float2 xa = ra[N - k], xb = hb ? rb[N - k] : make_float2(0.0f, 0.0f);
            v[k] = make_float2(xa.x + xb.y, xb.x - xa.y);
        }
        fft_line<N, 1>(v);
        // the two map rows, as floats at the start of their own tile rows (both rows were read above)
        float* ma = reinterpret_cast<float*>(ra);
        float* mb = reinterpret_cast<float*>(rb);
#pragma unroll
        for (int k = 0; k < N; ++k)
            if (k < G.vx) {
                ma[k] = v[k].x;
                if (hb) mb[k] = v[k].y;
            }
    }
    __syncthreads();
    const double scale = 1.0 / ((double)N * N * N);
    const double ssf = a.ssf[blockIdx.y], n_tpl = (double)G.n_tpl;
    const int64_t sxy = (int64_t)G.nx * G.ny;
    const int64_t wz0 = a.wz0[node], wy0 = a.wy0[node], wx0 = a.wx0[node];
    // window variance in FP64 (it cancels), the normalisation itself in FP32: the map is FP32, and the peak is
    // settled on FP64 re-scores
    const float fscale = (float)scale;
    const double inv_n = 1.0 / n_tpl;
    const float* msm = reinterpret_cast<const float*>(fsm);
    // this block's partials for the peak search (values visited in ascending map index per thread)
    float lmx = -3.0f, lmn = 3.0f;
    int lidx = 0x7fffffff;
    double ls1 = 0.0, ls2 = 0.0;
    const int i0 = dz0 * G.vy * G.vx;
    const float inv_vy = 1.0f / (float)G.vy;  // map rows r < 2^22: fdivi is exact
    sweep_lin<4, float2>(
        np * G.vy, G.vx,
        [&](int r, int dx) {
            const int p_ = fdivi(r, inv_vy), dy = r - p_ * G.vy;
            const int64_t o = (wz0 + dz0 + p_) * sxy + (wy0 + dy) * G.nx + (wx0 + dx);
            return make_float2(__ldg(a.B1 + o), __ldg(a.B2 + o));
        },
        [&](int r, int dx, float2 bs) {
            const int p_ = fdivi(r, inv_vy), dy = r - p_ * G.vy;
            const double s1 = (double)bs.x;
            const double var = (double)bs.y - s1 * s1 * inv_n;
            float v = 0.0f;
            if (!(var < 1e-20)) {
                v = msm[2 * (p_ * N + dy) * RP + dx] * fscale * rsqrtf((float)(var * ssf));
                v = fminf(1.0f, fmaxf(-1.0f, v));
            }
            out[(int64_t)p_ * G.vy * G.vx + dy * G.vx + dx] = v;
            if (v > lmx) {
                lmx = v;
                lidx = i0 + r * G.vx + dx;
            }
            lmn = fminf(lmn, v);
            ls1 += (double)v;
            ls2 += (double)v * (double)v;
        });
    if (a.part) {
        __shared__ MapPart wpart[fftr_pass3_threads<N>() / 32];
        const int lane = t & 31, warp = t >> 5;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float ob = __shfl_xor_sync(0xffffffffu, lmx, o);
            const int oi = __shfl_xor_sync(0xffffffffu, lidx, o);
            if (ob > lmx || (ob == lmx && oi < lidx)) {
                lmx = ob;
                lidx = oi;
            }
            lmn = fminf(lmn, __shfl_xor_sync(0xffffffffu, lmn, o));
            ls1 += __shfl_xor_sync(0xffffffffu, ls1, o);
            ls2 += __shfl_xor_sync(0xffffffffu, ls2, o);
        }
        if (lane == 0) {
            wpart[warp].mx = lmx;
            wpart[warp].idx = lidx;
            wpart[warp].mn = lmn;
            wpart[warp].s1 = ls1;
            wpart[warp].s2 = ls2;
        }
        __syncthreads();
        if (t == 0) {
            MapPart q = wpart[0];
            for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
                const MapPart o = wpart[w];
                if (o.mx > q.mx || (o.mx == q.mx && o.idx < q.idx)) {
                    q.mx = o.mx;
                    q.idx = o.idx;
                }
                q.mn = fminf(q.mn, o.mn);
                q.s1 += o.s1;
                q.s2 += o.s2;
            }
            q.pad = 0;
            a.part[(int64_t)blockIdx.y * a.nblk + blockIdx.x] = q;
        }
    }
}

// ---- cubic boxes, one thread-block cluster per node: the three passes above without their HBM scratch.  The
// node's whole spectrum (N^3 complex, 1 MB for N = 50) lives in the distributed shared memory of a cluster of C
// CTAs, PP = ceil(N / C) z-planes each:
//   1. CTA r transforms its window planes [r PP, r PP + PP) along x and y in its own shared memory (pass 1);
//   2. after a cluster barrier, thread (row, column) of CTA r gathers the z-line of one (ky, kx) column of its
//      rows from all C CTAs (ld through DSMEM), transforms it along z and keeps it in registers; after a second
//      barrier the lines are parked in the CTA's own tile, the product W^ conj T^ is formed from row ky and its
//      partner row -ky (the rows of a pair belong to one CTA) and inverted along z (pass 2); after a third barrier
//      the output planes dz < vz are written straight into the shared memory of the CTA that owns them (p3 planes
//      each, the Hermitian half ky <= N/2 only);
//   3. after a fourth barrier each CTA inverts its output planes along y and x, normalises them and writes the map
//      and its partials (pass 3, one block of partials per CTA).
// Every line goes through the same fft_line calls in the same order as in the three-pass engine, so the maps are
// identical.  Only the map and its partials reach HBM; the window and template rows are read as in pass 1.
// The barriers are the hardware cluster barrier (no spin loop); every CTA of a cluster takes all of them, or
// leaves before the first one together with the others (the node is the same for the whole cluster).
namespace cg = cooperative_groups;

constexpr int FFTC_C = 8;         // CTAs per cluster (the portable maximum)
constexpr int FFTC_MAX_ROWS = 8;  // spectrum rows (ky) per CTA in the z phase

// rows of the z phase: CTA r owns nrows[r] rows ky[r][.], each with the local index of its partner row (N - ky) % N
struct FftcRows {
    signed char nrows[FFTC_C];
    signed char ky[FFTC_C][FFTC_MAX_ROWS];
    signed char partner[FFTC_C][FFTC_MAX_ROWS];
};

template <int N>
struct FftcShape {
    static constexpr int PP = (N + FFTC_C - 1) / FFTC_C;  // z-planes per CTA in the forward phase
    static constexpr int PITCH = N | 1;
    static constexpr int NH = N / 2 + 1;
    static constexpr int RP = NH | 1;
    static constexpr int THREADS = (PP * N + 31) / 32 * 32;
    static constexpr size_t SMEM = (size_t)PP * N * PITCH * sizeof(float2);
};

// -2 everywhere (the unplaced-node marker) in this CTA's output planes, and the matching partial
__device__ __forceinline__ void fftc_unplaced(const FftArgs& a, int blk, int dz0, int np3) {
    const NccGeom& G = a.G;
    float* out = a.out + (int64_t)blockIdx.y * G.nmap + (int64_t)dz0 * G.vy * G.vx;
    for (int i = threadIdx.x; i < np3 * G.vy * G.vx; i += blockDim.x) out[i] = -2.0f;
    if (a.part && threadIdx.x == 0) {
        MapPart q;
        q.s1 = q.s2 = 0.0;
        q.mx = q.mn = 0.0f;
        q.idx = dz0 * G.vy * G.vx;
        q.pad = 0;
        a.part[(int64_t)blockIdx.y * a.nblk + blk] = q;
    }
}

template <int N>
__global__ void __cluster_dims__(FFTC_C, 1, 1) __launch_bounds__(FftcShape<N>::THREADS, 1)
    fftc_kernel(FftArgs a, FftcRows rows, int p3) {
    using Sh = FftcShape<N>;
    constexpr int PP = Sh::PP, PITCH = Sh::PITCH, NH = Sh::NH, RP = Sh::RP;
    extern __shared__ __align__(16) float2 fsm[];  // forward: [PP][N][PITCH]; z phase: [rows][N][PITCH]; output:
                                                   // [p3][NH][N] then the pass-3 tile [p3][N][RP]
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const NccGeom& G = a.G;
    const int64_t node = a.node_base + blockIdx.y;
    const int dz0 = rank * p3;
    const int np3 = max(0, min(p3, G.vz - dz0));
    if (!fft_node_ok(a, node)) {  // the same for every CTA of the cluster: all leave before the first barrier
        if (np3 > 0) fftc_unplaced(a, rank, dz0, np3);
        return;
    }
    const int t = threadIdx.x;
    const int64_t sxy = (int64_t)G.nx * G.ny;
    const int64_t wx0 = a.wx0[node], wy0 = a.wy0[node], wz0 = a.wz0[node];
    // ---------------- phase 1: this CTA's window planes along x, then along y
    {
        const int z0 = rank * PP;
        const int np = max(0, min(PP, G.wz - z0));  // planes past the window are zero and never read
        const float pilot = __ldg(a.pilot_at);
        const int pl = t / N, yx = t - pl * N;
        const int O = (int)(wx0 & 3);
        const bool vec = (G.nx & 3) == 0 && (reinterpret_cast<uintptr_t>(a.g) & 15) == 0;
        const float* gend = a.g + (int64_t)G.nz * sxy;
        if (pl < np) {
            const int z = z0 + pl, y = yx;
            float2 v[N];
            const float* wrow = a.g + (wz0 + z) * sxy + (wy0 + y) * G.nx + wx0;
            const float* trow = a.T + (int64_t)blockIdx.y * G.sz * G.sy * a.sxp + ((int64_t)z * G.sy + y) * a.sxp;
            const bool wy_in = y < G.wy, ty_in = z < G.sz && y < G.sy;
            const bool vrow = vec && wy_in && wrow - O + 4 * ((G.wx + O + 3) / 4) <= gend;
            if (vrow) {
                switch (O) {
                    case 0: fftr_row4<N, 0>(wrow, G.wx, pilot, v); break;
                    case 1: fftr_row4<N, 1>(wrow - 1, G.wx, pilot, v); break;
                    case 2: fftr_row4<N, 2>(wrow - 2, G.wx, pilot, v); break;
                    default: fftr_row4<N, 3>(wrow - 3, G.wx, pilot, v); break;
                }
            } else {
#pragma unroll
                for (int x = 0; x < N; ++x) v[x].x = (wy_in && x < G.wx) ? __ldg(wrow + x) - pilot : 0.0f;
            }
            if (ty_in && (a.sxp & 3) == 0) {
                fftr_trow4<N>(trow, G.sx, v);
            } else {
#pragma unroll
                for (int x = 0; x < N; ++x) v[x].y = (ty_in && x < G.sx) ? __ldg(trow + x) : 0.0f;
            }
            if (wy_in) fft_line<N, -1>(v);
            float2* row = fsm + (pl * N + y) * PITCH;
#pragma unroll
            for (int x = 0; x < N; ++x) row[x] = v[x];
        }
        __syncthreads();
        if (pl < np) {
            float2* col = fsm + pl * N * PITCH + yx;
            float2 v[N];
#pragma unroll
            for (int k = 0; k < N; ++k) v[k] = col[k * PITCH];
            fft_line<N, -1>(v);
#pragma unroll
            for (int k = 0; k < N; ++k) col[k * PITCH] = v[k];
        }
        // the box sums of this CTA's output planes are read at the end: start them towards L2
        const int nch = (G.vx + 31) / 32, per_row = 2 * nch;
        for (int i = t; i < np3 * G.vy * per_row; i += blockDim.x) {
            const int r = i / per_row, rem = i - r * per_row, p_ = r / G.vy, dy = r - p_ * G.vy;
            const float* b = (rem & 1) ? a.B2 : a.B1;
            prefetch_l2(b + (wz0 + dz0 + p_) * sxy + (wy0 + dy) * G.nx + wx0 + 32 * (rem >> 1));
        }
    }
    cl.sync();  // barrier 1: every plane spectrum of the node is in the cluster
    // ---------------- phase 2: thread (r, c) transforms the z-line of column c of this CTA's row r
    const int nr = rows.nrows[rank];
    const int r = t / N, c = t - r * N;
    const bool has = r < nr;
    const int ky = has ? (int)rows.ky[rank][r] : 0;
    float2 v[N];
    if (has) {
        const float2* src[FFTC_C];
#pragma unroll
        for (int q = 0; q < FFTC_C; ++q) src[q] = cl.map_shared_rank(fsm, q) + ky * PITCH + c;
#pragma unroll
        for (int z = 0; z < N; ++z) v[z] = z < G.wz ? src[z / PP][(z % PP) * N * PITCH] : make_float2(0.0f, 0.0f);
        fft_line<N, -1>(v);
    }
    cl.sync();  // barrier 2: every CTA has read the plane spectra it needs; the tiles are free
    if (has) {
#pragma unroll
        for (int k = 0; k < N; ++k) fsm[(r * N + k) * PITCH + c] = v[k];
    }
    __syncthreads();
    const bool top = has && ky <= N / 2;  // the product is Hermitian: rows ky <= N/2 hold all of it
    if (top) {
        const float2* pb = fsm + (int)rows.partner[rank][r] * N * PITCH + (N - c) % N;
#pragma unroll
        for (int kz = 0; kz < N; ++kz) {
            const float2 za = v[kz];
            const float2 zb = pb[((N - kz) % N) * PITCH];
            const float2 zbc = make_float2(zb.x, -zb.y);
            const float2 w = make_float2(0.5f * (za.x + zbc.x), 0.5f * (za.y + zbc.y));
            const float2 d = make_float2(za.x - zbc.x, za.y - zbc.y);
            const float2 tc = make_float2(0.5f * d.y, 0.5f * d.x);  // conj(T^) = i conj(za - zbc) / 2
            v[kz] = fr_mul(w, tc);
        }
        fft_line<N, 1>(v);
    }
    cl.sync();  // barrier 3: every CTA is done with its own lines; output planes may be written anywhere
    if (top) {  // output plane dz to CTA dz / p3, plane dz % p3 of its [p3][NH][N] block
        int owner = 0, dzl = 0;
        float2* dst = cl.map_shared_rank(fsm, 0) + ky * N + c;
#pragma unroll
        for (int dz = 0; dz < N; ++dz) {
            if (dz < G.vz) {
                dst[dzl * NH * N] = v[dz];
                if (++dzl == p3) {
                    dzl = 0;
                    ++owner;
                    if (owner < FFTC_C) dst = cl.map_shared_rank(fsm, owner) + ky * N + c;
                }
            }
        }
    }
    cl.sync();  // barrier 4: every output plane is in place; no CTA touches another's memory after this
    if (np3 == 0) return;
    // ---------------- phase 3: inverse along y of columns kx <= N/2 (rows ky > N/2 as conjugates), then along x of
    // real row pairs, normalisation, map rows and the block's partials (as fftr_pass3_kernel)
    float2* tile = fsm + (size_t)p3 * NH * N;  // [p3][N][RP]
    {
        const int pl = t / NH, kx = t - pl * NH;
        if (pl < np3) {
            const float2* pg = fsm + pl * NH * N;
            const int kxm = (N - kx) % N;
#pragma unroll
            for (int k = 0; k < NH; ++k) v[k] = pg[k * N + kx];
#pragma unroll
            for (int k = NH; k < N; ++k) {
                const float2 w = pg[(N - k) * N + kxm];
                v[k] = make_float2(w.x, -w.y);
            }
            fft_line<N, 1>(v);
            float2* col = tile + pl * N * RP + kx;
#pragma unroll
            for (int k = 0; k < N; ++k) col[k * RP] = v[k];
        }
        __syncthreads();
        const int nj = (G.vy + 1) / 2;
        if (pl < np3 && kx < nj) {
            float2* ra = tile + (pl * N + 2 * kx) * RP;
            float2* rb = ra + RP;
            const bool hb = 2 * kx + 1 < G.vy;
#pragma unroll
            for (int k = 0; k < NH; ++k) {
                const float2 xa = ra[k], xb = hb ? rb[k] : make_float2(0.0f, 0.0f);
                v[k] = make_float2(xa.x - xb.y, xa.y + xb.x);
            }
#pragma unroll
            for (int k = NH; k < N; ++k) {
                const float2 xa = ra[N - k], xb = hb ? rb[N - k] : make_float2(0.0f, 0.0f);
                v[k] = make_float2(xa.x + xb.y, xb.x - xa.y);
            }
            fft_line<N, 1>(v);
            float* ma = reinterpret_cast<float*>(ra);
            float* mb = reinterpret_cast<float*>(rb);
#pragma unroll
            for (int k = 0; k < N; ++k)
                if (k < G.vx) {
                    ma[k] = v[k].x;
                    if (hb) mb[k] = v[k].y;
                }
        }
        __syncthreads();
    }
    float* out = a.out + (int64_t)blockIdx.y * G.nmap + (int64_t)dz0 * G.vy * G.vx;
    const double scale = 1.0 / ((double)N * N * N);
    const double ssf = a.ssf[blockIdx.y], n_tpl = (double)G.n_tpl;
    const float fscale = (float)scale;
    const double inv_n = 1.0 / n_tpl;
    const float* msm = reinterpret_cast<const float*>(tile);
    float lmx = -3.0f, lmn = 3.0f;
    int lidx = 0x7fffffff;
    double ls1 = 0.0, ls2 = 0.0;
    const int i0 = dz0 * G.vy * G.vx;
    const float inv_vy = 1.0f / (float)G.vy;  // map rows r < 2^22: fdivi is exact
    sweep_lin<4, float2>(
        np3 * G.vy, G.vx,
        [&](int rr, int dx) {
            const int p_ = fdivi(rr, inv_vy), dy = rr - p_ * G.vy;
            const int64_t o = (wz0 + dz0 + p_) * sxy + (wy0 + dy) * G.nx + (wx0 + dx);
            return make_float2(__ldg(a.B1 + o), __ldg(a.B2 + o));
        },
        [&](int rr, int dx, float2 bs) {
            const int p_ = fdivi(rr, inv_vy), dy = rr - p_ * G.vy;
            const double s1 = (double)bs.x;
            const double var = (double)bs.y - s1 * s1 * inv_n;
            float vv = 0.0f;
            if (!(var < 1e-20)) {
                vv = msm[2 * (p_ * N + dy) * RP + dx] * fscale * rsqrtf((float)(var * ssf));
                vv = fminf(1.0f, fmaxf(-1.0f, vv));
            }
            out[(int64_t)p_ * G.vy * G.vx + dy * G.vx + dx] = vv;
            if (vv > lmx) {
                lmx = vv;
                lidx = i0 + rr * G.vx + dx;
            }
            lmn = fminf(lmn, vv);
            ls1 += (double)vv;
            ls2 += (double)vv * (double)vv;
        });
    if (a.part) {
        __shared__ MapPart wpart[Sh::THREADS / 32];
        const int lane = t & 31, warp = t >> 5;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float ob = __shfl_xor_sync(0xffffffffu, lmx, o);
            const int oi = __shfl_xor_sync(0xffffffffu, lidx, o);
            if (ob > lmx || (ob == lmx && oi < lidx)) {
                lmx = ob;
                lidx = oi;
            }
            lmn = fminf(lmn, __shfl_xor_sync(0xffffffffu, lmn, o));
            ls1 += __shfl_xor_sync(0xffffffffu, ls1, o);
            ls2 += __shfl_xor_sync(0xffffffffu, ls2, o);
        }
        if (lane == 0) {
            wpart[warp].mx = lmx;
            wpart[warp].idx = lidx;
            wpart[warp].mn = lmn;
            wpart[warp].s1 = ls1;
            wpart[warp].s2 = ls2;
        }
        __syncthreads();
        if (t == 0) {
            MapPart q = wpart[0];
            for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
                const MapPart o = wpart[w];
                if (o.mx > q.mx || (o.mx == q.mx && o.idx < q.idx)) {
                    q.mx = o.mx;
                    q.idx = o.idx;
                }
                q.mn = fminf(q.mn, o.mn);
                q.s1 += o.s1;
                q.s2 += o.s2;
            }
            q.pad = 0;
            a.part[(int64_t)blockIdx.y * a.nblk + rank] = q;
        }
    }
}

// twiddles of the in-register transforms, once per device (before any capture: the first FFT search does it)
static int fftr_upload() {
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "ncc fft: device");
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 64 && done[dev]) return ALDVC_OK;
    float2 h[FFTR_TOTAL];
    for (int i = 0; i < FFTR_NSIZES; ++i) {
        const int n = FFTR_SIZES[i], o = fftr_offset(n);
        for (int k = 0; k < n; ++k) {
            const double ang = -2.0 * 3.14159265358979323846 * (double)k / (double)n;
            h[o + k] = make_float2((float)cos(ang), (float)sin(ang));
        }
    }
    e = cudaMemcpyToSymbol(c_fftr_tw, h, sizeof(h));
    if (e != cudaSuccess) return cuda_fail(e, "ncc fft: twiddle upload");
    if (dev < 64) done[dev] = true;
    return ALDVC_OK;
}

// pass 2 on the tensor pipe (fftt_pass2_kernel) when ALDVC_FFT_PASS2=tensor and the length has that form (a
// comparison knob, read once; each launch synchronises its stream to read the kernel's error flag)
static bool fft_pass2_tensor() {
    static const bool on = [] {
        const char* e = std::getenv("ALDVC_FFT_PASS2");
        return e && std::strcmp(e, "tensor") == 0;
    }();
    return on;
}

template <int N>
static int launch_fftt_pass2(FftArgs& a, int nb, cudaStream_t s) {
    using S = FfttShape<N>;
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(fftt_pass2_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM);
        if (e != cudaSuccess) return cuda_fail(e, "ncc fft tensor pass 2: shared memory attribute");
        attr = true;
    }
    const int64_t groups = ((int64_t)nb * (N / 2 + 1) * N + 127) / 128;
    const int grid = (int)std::min<int64_t>(groups, sm_count());
    const int zero = 0;
    cudaError_t e = cudaMemcpyToSymbolAsync(g_fftt_err, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "ncc fft tensor pass 2: error flag");
    fftt_pass2_kernel<N><<<grid, FFTT_THREADS, S::SMEM, s>>>(a, groups);
    int rc = check_launch("ncc fft tensor pass 2");
    if (rc) return rc;
    int err = 0;
    e = cudaMemcpyFromSymbolAsync(&err, g_fftt_err, sizeof(int), 0, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "ncc fft tensor pass 2");
    if (err) {
        set_error("ncc fft tensor pass 2: an MMA completion wait gave up");
        return ALDVC_ERR_CUDA;
    }
    return ALDVC_OK;
}

template <int N>
static int launch_fftr(FftArgs& a, int nb, cudaStream_t s) {
    constexpr int P = fftr_planes<N>();
    constexpr int P3 = fftr_planes3<N>();
    constexpr size_t SM = (size_t)P * N * (N | 1) * sizeof(float2);
    constexpr size_t SM2 = (size_t)N * (N | 1) * sizeof(float2);
    constexpr size_t SM3 = (size_t)P3 * N * ((N / 2 + 1) | 1) * sizeof(float2);
    static bool attr = false;  // set once, outside any capture (the first search of this length)
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(fftr_pass1_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(fftr_pass3_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM3);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(fftr_pass2_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM2);
        if (e != cudaSuccess) return cuda_fail(e, "ncc fft: shared memory attribute");
        attr = true;
    }
    const NccGeom& G = a.G;
    {
        KTimer kt_("fft_pass1", s);
        fftr_pass1_kernel<N><<<dim3((G.wz + P - 1) / P, nb), P * N, SM, s>>>(a);
    }
    int rc = check_launch("ncc fft pass 1");
    if (rc) return rc;
    if constexpr (N <= 54) {
        if (fft_pass2_tensor()) {
            {
                KTimer kt_("fft_pass2_tensor", s);
                rc = launch_fftt_pass2<N>(a, nb, s);
            }
            if (rc) return rc;
            {
                KTimer kt_("fft_pass3", s);
                fftr_pass3_kernel<N><<<dim3((G.vz + P3 - 1) / P3, nb), fftr_pass3_threads<N>(), SM3, s>>>(a);
            }
            return check_launch("ncc fft pass 3");
        }
    }
    {
        KTimer kt_("fft_pass2", s);
        fftr_pass2_kernel<N><<<dim3(N / 2 + 1, nb), N, SM2, s>>>(a);
    }
    rc = check_launch("ncc fft pass 2");
    if (rc) return rc;
    {
        KTimer kt_("fft_pass3", s);
        fftr_pass3_kernel<N><<<dim3((G.vz + P3 - 1) / P3, nb), fftr_pass3_threads<N>(), SM3, s>>>(a);
    }
    return check_launch("ncc fft pass 3");
}

template <int N>
static int launch_fftc(FftArgs& a, const FftcRows& rows, int p3, int nb, cudaStream_t s) {
    using Sh = FftcShape<N>;
    static bool attr = false;  // set once, outside any capture (the first search of this length)
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(fftc_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Sh::SMEM);
        if (e != cudaSuccess) return cuda_fail(e, "ncc fft cluster: shared memory attribute");
        attr = true;
    }
    {
        KTimer kt_("fft_cluster", s);
        fftc_kernel<N><<<dim3(FFTC_C, nb), Sh::THREADS, Sh::SMEM, s>>>(a, rows, p3);
    }
    return check_launch("ncc fft cluster");
}

static int launch_fftc_n(int n, FftArgs& a, const FftcRows& rows, int p3, int nb, cudaStream_t s) {
    switch (n) {
        case 36: return launch_fftc<36>(a, rows, p3, nb, s);
        case 40: return launch_fftc<40>(a, rows, p3, nb, s);
        case 48: return launch_fftc<48>(a, rows, p3, nb, s);
        case 50: return launch_fftc<50>(a, rows, p3, nb, s);
        default: return launch_fftc<54>(a, rows, p3, nb, s);
    }
}

// map planes per pass-3 CTA of the in-register engine (the block of one map partial)
static int fftr_planes3_n(int n) {
    switch (n) {
        case 36: return fftr_planes3<36>();
        case 40: return fftr_planes3<40>();
        case 48: return fftr_planes3<48>();
        case 50: return fftr_planes3<50>();
        case 54: return fftr_planes3<54>();
        case 60: return fftr_planes3<60>();
        default: return fftr_planes3<64>();
    }
}

static int launch_fftr_n(int n, FftArgs& a, int nb, cudaStream_t s) {
    switch (n) {
        case 36: return launch_fftr<36>(a, nb, s);
        case 40: return launch_fftr<40>(a, nb, s);
        case 48: return launch_fftr<48>(a, nb, s);
        case 50: return launch_fftr<50>(a, nb, s);
        case 54: return launch_fftr<54>(a, nb, s);
        case 60: return launch_fftr<60>(a, nb, s);
        default: return launch_fftr<64>(a, nb, s);
    }
}

struct FftCfg {
    FftAxis ax, ay, az;
    bool reg;      // cubic box of a length with an in-register transform (fftr passes)
    bool cluster;  // ... run as one cluster kernel per node (fftc_kernel): no spectra scratch
    int p3;        // cluster form: output planes per CTA (the map block of one partial)
    FftcRows rows; // cluster form: rows of the z phase per CTA
    int pitch;
    size_t smem13, smem2;  // dynamic shared bytes of passes 1/3 and 2
    int64_t per_node;      // scratch bytes per node (A and P)
};

// Cluster form of a cubic box of length n: the threads and shared bytes of fftc_kernel<n>, 0 when n has none
static void fftc_shape(int n, int& threads, size_t& smem) {
    threads = 0;
    smem = 0;
    switch (n) {
        case 36: threads = FftcShape<36>::THREADS; smem = FftcShape<36>::SMEM; break;
        case 40: threads = FftcShape<40>::THREADS; smem = FftcShape<40>::SMEM; break;
        case 48: threads = FftcShape<48>::THREADS; smem = FftcShape<48>::SMEM; break;
        case 50: threads = FftcShape<50>::THREADS; smem = FftcShape<50>::SMEM; break;
        case 54: threads = FftcShape<54>::THREADS; smem = FftcShape<54>::SMEM; break;
        default: break;
    }
}

// The z-phase rows of the cluster form: the pairs (ky, N - ky) and the single rows 0 and N/2 dealt to the CTAs so
// that no CTA holds more than PP rows (its plane tile holds PP x N lines) and a pair stays in one CTA (the
// product needs both rows).  False when they do not fit.
static bool fftc_rows(int n, int pp, FftcRows& r) {
    std::memset(&r, 0, sizeof(r));
    const int cap = std::min(pp, FFTC_MAX_ROWS);
    auto put = [&](int ky0, int ky1) {  // ky1 < 0: a single row
        const int need = ky1 < 0 ? 1 : 2;
        int best = -1;
        for (int q = 0; q < FFTC_C; ++q)  // the emptiest CTA with room
            if (r.nrows[q] + need <= cap && (best < 0 || r.nrows[q] < r.nrows[best])) best = q;
        if (best < 0) return false;
        const int i0 = r.nrows[best];
        r.ky[best][i0] = (signed char)ky0;
        r.partner[best][i0] = (signed char)(ky1 < 0 ? i0 : i0 + 1);
        if (ky1 >= 0) {
            r.ky[best][i0 + 1] = (signed char)ky1;
            r.partner[best][i0 + 1] = (signed char)i0;
        }
        r.nrows[best] = (signed char)(i0 + need);
        return true;
    };
    for (int k = 1; k < (n + 1) / 2; ++k)
        if (k != n - k && !put(k, n - k)) return false;
    if (!put(0, -1)) return false;
    if (n % 2 == 0 && !put(n / 2, -1)) return false;
    return true;
}

static bool fftc_config(const NccGeom& G, FftCfg& c) {
    const int n = c.ax.n;
    int threads;
    size_t smem;
    fftc_shape(n, threads, smem);
    if (threads == 0 || G.wz > n || G.vz > n) return false;
    const int pp = (n + FFTC_C - 1) / FFTC_C, nh = n / 2 + 1;
    c.p3 = (G.vz + FFTC_C - 1) / FFTC_C;
    const size_t out_tile = ((size_t)c.p3 * nh * n + (size_t)c.p3 * n * (nh | 1)) * sizeof(float2);
    return out_tile <= smem && c.p3 * nh <= threads && smem <= (size_t)max_smem_optin() - 2048 && fftc_rows(n, pp, c.rows);
}

static bool fft_config(const NccGeom& G, FftCfg& c, bool engine_reg = true, bool engine_cluster = false) {
    if (!fft_axis(smooth_len(G.wx), c.ax) || !fft_axis(smooth_len(G.wy), c.ay) || !fft_axis(smooth_len(G.wz), c.az)) return false;
    c.reg = engine_reg && c.ax.n == c.ay.n && c.ax.n == c.az.n && fftr_supported(c.ax.n);
    c.cluster = c.reg && engine_cluster && fftc_config(G, c);
    c.pitch = c.ax.n | 1;  // odd: rows and columns of a plane fall in distinct bank pairs
    c.smem13 = ((size_t)2 * c.ay.n * c.pitch + 2 * FFT_MAX_N) * sizeof(float2);
    // pass 2: two buffers of one whole row (Nz x pitch) or of two half rows (2 x Nz x (cb | 1))
    c.smem2 = ((size_t)2 * std::max(c.pitch, 2 * (((c.ax.n + 1) / 2) | 1)) * c.az.n + FFT_MAX_N) * sizeof(float2);
    // the in-register passes keep the product rows ky <= N/2 only
    const int64_t p_rows = c.reg ? c.ay.n / 2 + 1 : c.ay.n;
    c.per_node = c.cluster ? 0 : ((int64_t)G.wz * c.ay.n + (int64_t)G.vz * p_rows) * c.ax.n * (int64_t)sizeof(float2);
    const size_t smax = (size_t)max_smem_optin() - 4096;
    return c.smem13 <= smax && c.smem2 <= smax;
}

// scratch of one batch (spectra A and P); ALDVC_FFT_BATCH_MB overrides it (a tuning knob, read once)
constexpr int64_t FFT_BATCH_BYTES = 3LL << 30;  // larger batches fill the GPU better (0.5 -> 3 GB: 509 -> 494 ms per pass on configuration 5)
static int64_t fft_batch_bytes() {
    static const int64_t b = [] {
        const char* e = std::getenv("ALDVC_FFT_BATCH_MB");
        const long v = e ? std::atol(e) : 0;
        return v > 0 ? (int64_t)v << 20 : FFT_BATCH_BYTES;
    }();
    return b;
}

static int64_t fft_batch(const FftCfg& c, int64_t chunk) {
    const int64_t b = c.cluster ? chunk : std::min<int64_t>(chunk, fft_batch_bytes() / std::max<int64_t>(c.per_node, 1));
    return std::max<int64_t>(1, std::min<int64_t>(b, 65535));  // grid y limit
}

static int fft_set_smem(size_t s13, size_t s2) {
    static size_t have13 = 0, have2 = 0;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    if (s13 > 48 * 1024 && s13 > have13) {
        cudaError_t e = cudaFuncSetAttribute(fft_pass1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s13);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(fft_pass3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s13);
        if (e != cudaSuccess) return cuda_fail(e, "ncc fft: shared memory attribute");
        have13 = s13;
    }
    if (s2 > 48 * 1024 && s2 > have2) {
        cudaError_t e = cudaFuncSetAttribute(fft_pass2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s2);
        if (e != cudaSuccess) return cuda_fail(e, "ncc fft: shared memory attribute");
        have2 = s2;
    }
    return ALDVC_OK;
}

// Maps of nodes [a.node_base, a.node_base + n) into a.out, in batches through the scratch.
static int launch_fft(FftArgs a, const FftCfg& c, int64_t n, int64_t batch, cudaStream_t s) {
    int rc = fft_set_smem(c.smem13, c.smem2);
    if (rc) return rc;
    const NccGeom& G = a.G;
    float* out0 = a.out;
    MapPart* part0 = a.part;
    const double* ssf0 = a.ssf;
    const float* T0 = a.T;
    const int64_t tsz = (int64_t)G.sz * G.sy * a.sxp;
    const int64_t base0 = a.node_base;
    for (int64_t done = 0; done < n; done += batch) {
        const int nb = (int)std::min<int64_t>(batch, n - done);
        a.node_base = base0 + done;
        a.out = out0 + done * G.nmap;
        a.part = part0 ? part0 + done * a.nblk : nullptr;
        a.ssf = ssf0 + done;
        a.T = T0 + done * tsz;
        a.nb = nb;
        if (c.reg) {
            rc = c.cluster ? launch_fftc_n(c.ax.n, a, c.rows, c.p3, nb, s) : launch_fftr_n(c.ax.n, a, nb, s);
            if (rc) return rc;
            continue;
        }
        {
            KTimer kt_("fft_pass1", s);
            fft_pass1_kernel<<<dim3(G.wz, nb), FFT_THREADS, c.smem13, s>>>(a);
        }
        rc = check_launch("ncc fft pass 1");
        if (rc) return rc;
        {
            KTimer kt_("fft_pass2", s);
            fft_pass2_kernel<<<dim3(2 * (c.ay.n / 2 + 1), nb), FFT_THREADS, c.smem2, s>>>(a);
        }
        rc = check_launch("ncc fft pass 2");
        if (rc) return rc;
        {
            KTimer kt_("fft_pass3", s);
            fft_pass3_kernel<<<dim3(G.vz, nb), FFT_THREADS, c.smem13, s>>>(a);
        }
        rc = check_launch("ncc fft pass 3");
        if (rc) return rc;
    }
    return ALDVC_OK;
}

static int upload_pinv() {
    static bool done = false;
    if (done) return ALDVC_OK;
    // least-squares quadratic on the 3x3x3 grid: pinv(D) = (D^T D)^-1 D^T, columns
    // [1, x, y, z, xy, xz, yz, x^2, y^2, z^2], rows of D in C order over (dz, dy, dx)
    double D[27][10];
    for (int t = 0; t < 27; ++t) {
        const double z = t / 9 - 1, y = (t / 3) % 3 - 1, x = t % 3 - 1;
        const double row[10] = {1, x, y, z, x * y, x * z, y * z, x * x, y * y, z * z};
        for (int c = 0; c < 10; ++c) D[t][c] = row[c];
    }
    double N[10][20];
    for (int i = 0; i < 10; ++i) {
        for (int j = 0; j < 10; ++j) {
            double s = 0.0;
            for (int t = 0; t < 27; ++t) s += D[t][i] * D[t][j];
            N[i][j] = s;
        }
        for (int j = 0; j < 10; ++j) N[i][10 + j] = i == j ? 1.0 : 0.0;
    }
    for (int c = 0; c < 10; ++c) {  // Gauss-Jordan with partial pivoting
        int p = c;
        for (int r = c + 1; r < 10; ++r)
            if (std::fabs(N[r][c]) > std::fabs(N[p][c])) p = r;
        for (int j = 0; j < 20; ++j) std::swap(N[c][j], N[p][j]);
        const double d = N[c][c];
        for (int j = 0; j < 20; ++j) N[c][j] /= d;
        for (int r = 0; r < 10; ++r)
            if (r != c) {
                const double m = N[r][c];
                for (int j = 0; j < 20; ++j) N[r][j] -= m * N[c][j];
            }
    }
    double P[10 * 27];
    for (int i = 0; i < 10; ++i)
        for (int t = 0; t < 27; ++t) {
            double s = 0.0;
            for (int j = 0; j < 10; ++j) s += N[i][10 + j] * D[t][j];
            P[i * 27 + t] = s;
        }
    cudaError_t e = cudaMemcpyToSymbol(c_pinv, P, sizeof(P));
    if (e != cudaSuccess) return cuda_fail(e, "ncc: pinv upload");
    done = true;
    return ALDVC_OK;
}

static size_t tpl_smem(const NccGeom& G) { return (size_t)G.n_tpl * sizeof(float); }

static int launch_map(const MapArgs& m, int64_t n_chunk, cudaStream_t s) {
    const size_t smem = tpl_smem(m.G);
    static const size_t stat = static_smem((const void*)ncc_map_kernel);
    static size_t attr_set = 48 * 1024 - stat;  // largest dynamic size already allowed (no call inside a capture)
    if (smem > attr_set) {
        const size_t want = (size_t)max_smem_optin() - 4096;
        cudaError_t e = cudaFuncSetAttribute(ncc_map_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)want);
        if (e != cudaSuccess) return cuda_fail(e, "ncc map: shared memory attribute");
        attr_set = want;
    }
    const unsigned tiles = (unsigned)((m.G.nmap + NCC_THREADS - 1) / NCC_THREADS);
    for (int64_t done = 0; done < n_chunk; done += 65535) {
        MapArgs mm = m;
        mm.node_base = m.node_base + done;
        mm.out = m.out + done * m.G.nmap;
        const unsigned ny = (unsigned)std::min<int64_t>(65535, n_chunk - done);
        {
            KTimer kt_("ncc_map", s);
            ncc_map_kernel<<<dim3(tiles, ny), NCC_THREADS, smem, s>>>(mm);
        }
        const int rc = check_launch("ncc map");
        if (rc) return rc;
    }
    return ALDVC_OK;
}

static int check_geom(const NccGeom& G) {
    if (G.hx < 0 || G.hy < 0 || G.hz < 0 || G.rx < 0 || G.ry < 0 || G.rz < 0) return arg_fail("ncc: negative half-width or radius");
    if ((int64_t)G.nx * G.ny >= (1LL << 31)) return arg_fail("ncc: volume plane too large");
    if (tpl_smem(G) + 4096 > (size_t)max_smem_optin()) return arg_fail("ncc: template larger than shared memory");
    return ALDVC_OK;
}

// maps of one search chunk: 512 MB; ALDVC_NCC_CHUNK_MB overrides it (a tuning knob, read once)
static int64_t search_chunk_bytes() {
    static const int64_t b = [] {
        const char* e = std::getenv("ALDVC_NCC_CHUNK_MB");
        const long v = e ? std::atol(e) : 0;
        return v > 0 ? (int64_t)v << 20 : (512LL << 20);
    }();
    return b;
}

static int64_t search_chunk(const NccGeom& G, int64_t n) {
    const int64_t per = (int64_t)G.nmap * 4;
    int64_t c = search_chunk_bytes() / std::max<int64_t>(per, 1);
    c = std::max<int64_t>(1, std::min<int64_t>(c, n));
    return c;
}

}  // namespace aldvc

using namespace aldvc;

extern "C" int aldvc_ncc_map(const float* f, const float* g, int64_t nz, int64_t ny, int64_t nx, const int64_t* coords,
                             int64_t n_nodes, int32_t hx, int32_t hy, int32_t hz, int32_t rx, int32_t ry, int32_t rz,
                             const int64_t* wx0, const int64_t* wy0, const int64_t* wz0, const uint8_t* t_ok, float* out,
                             void* stream) {
    ALDVC_REQUIRE(f && g && coords && wx0 && wy0 && wz0 && t_ok && out, "aldvc_ncc_map: null pointer");
    const NccGeom G = make_geom(nz, ny, nx, hx, hy, hz, rx, ry, rz);
    int rc = check_geom(G);
    if (rc) return rc;
    if (n_nodes <= 0) return ALDVC_OK;
    MapArgs m{f, g, coords, wx0, wy0, wz0, t_ok, out, 0, n_nodes, G};
    return launch_map(m, n_nodes, (cudaStream_t)stream);
}

// map planes of one partial block: a pass-3 CTA's, or a cluster CTA's output planes
static int fft_blk_planes(const FftCfg& c) { return c.cluster ? c.p3 : fftr_planes3_n(c.ax.n); }

static int fft_nblk(const NccGeom& G, const FftCfg& c) {
    const int p3 = fft_blk_planes(c);
    return (G.vz + p3 - 1) / p3;
}

static bool use_fft(const NccGeom& G, int32_t engine, FftCfg& c) {
    const bool fft = engine == ALDVC_NCC_FFT || engine == ALDVC_NCC_FFT_STOCKHAM || engine == ALDVC_NCC_FFT_CLUSTER;
    return fft && fft_config(G, c, engine != ALDVC_NCC_FFT_STOCKHAM, engine == ALDVC_NCC_FFT_CLUSTER);
}

// TILED, or FFT on a geometry the FFT engine does not take
static bool use_tiled(const NccGeom& G, int32_t engine, TiledCfg& c) {
    FftCfg fc;
    const bool fft = engine == ALDVC_NCC_FFT || engine == ALDVC_NCC_FFT_STOCKHAM || engine == ALDVC_NCC_FFT_CLUSTER;
    return (engine == ALDVC_NCC_TILED || (fft && !fft_config(G, fc))) && tiled_config(G, c);
}

static int launch_templates(const TiledArgs& a, int64_t n, cudaStream_t s) {
    const int64_t tsz = (int64_t)a.G.sz * a.G.sy * a.sxp;
    for (int64_t done = 0; done < n; done += 65535) {
        const unsigned nb = (unsigned)std::min<int64_t>(65535, n - done);
        TiledArgs aa = a;
        aa.node_base = a.node_base + done;
        {
            KTimer kt_("ncc_template", s);
            ncc_template_kernel<<<nb, 256, 0, s>>>(aa, const_cast<float*>(a.T) + done * tsz, const_cast<double*>(a.ssf) + done);
        }
        const int rc = check_launch("ncc template");
        if (rc) return rc;
    }
    return ALDVC_OK;
}

extern "C" size_t aldvc_ncc_search_workspace_size(int64_t nz, int64_t ny, int64_t nx, int64_t n_nodes, int32_t hx, int32_t hy,
                                                  int32_t hz, int32_t rx, int32_t ry, int32_t rz, int32_t engine) {
    const NccGeom G = make_geom(nz, ny, nx, hx, hy, hz, rx, ry, rz);
    const int64_t n = std::max<int64_t>(n_nodes, 1);
    const int64_t chunk = search_chunk(G, n);
    size_t b = align_up((size_t)n * 32, 256) + align_up((size_t)chunk * G.nmap * sizeof(float), 256);
    TiledCfg c;
    FftCfg fc;
    const bool fft = use_fft(G, engine, fc);
    if (fft || use_tiled(G, engine, c))  // box sums + temporaries, template scratch
        b += 4 * align_up((size_t)nz * ny * nx * sizeof(float), 256) + tiled_tpl_bytes(G, chunk);
    if (fft)  // twiddles, one batch of spectra
        b += align_up(3 * FFT_MAX_N * sizeof(float2), 256) + align_up((size_t)fft_batch(fc, chunk) * fc.per_node, 256);
    if (fft && fc.reg)  // map partials of a chunk
        b += align_up((size_t)chunk * fft_nblk(G, fc) * sizeof(MapPart), 256);
    return b;
}

extern "C" int aldvc_ncc_search(const float* f, const float* g, int64_t nz, int64_t ny, int64_t nx, const int64_t* coords,
                                int64_t n_nodes, int32_t hx, int32_t hy, int32_t hz, int32_t rx, int32_t ry, int32_t rz,
                                const int64_t* shift0, int32_t engine, void* workspace, size_t workspace_bytes, double* disp,
                                double* cc, double* pce, uint8_t* clipped, uint8_t* ok, void* stream) {
    ALDVC_REQUIRE(f && g && coords && disp && cc && pce && clipped && ok, "aldvc_ncc_search: null pointer");
    ALDVC_REQUIRE(engine == ALDVC_NCC_TILED || engine == ALDVC_NCC_PLAIN || engine == ALDVC_NCC_FFT || engine == ALDVC_NCC_FFT_STOCKHAM ||
                      engine == ALDVC_NCC_FFT_CLUSTER,
                  "aldvc_ncc_search: unknown engine");
    const NccGeom G = make_geom(nz, ny, nx, hx, hy, hz, rx, ry, rz);
    int rc = check_geom(G);
    if (rc) return rc;
    ALDVC_REQUIRE(G.wx <= G.nx && G.wy <= G.ny && G.wz <= G.nz, "aldvc_ncc_search: search window larger than the volume");
    if (n_nodes <= 0) return ALDVC_OK;
    const size_t need = aldvc_ncc_search_workspace_size(nz, ny, nx, n_nodes, hx, hy, hz, rx, ry, rz, engine);
    if (!workspace || workspace_bytes < need) {
        set_error("aldvc_ncc_search: workspace of %zu bytes needed, %zu given", need, workspace_bytes);
        return ALDVC_ERR_WORKSPACE;
    }
    rc = upload_pinv();
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    char* w = (char*)workspace;
    SearchArgs a;
    a.f = f;
    a.g = g;
    a.coords = coords;
    a.shift0 = shift0;
    a.n_nodes = n_nodes;
    a.node_base = 0;
    a.G = G;
    a.wx0 = (int64_t*)w;
    a.wy0 = a.wx0 + n_nodes;
    a.wz0 = a.wy0 + n_nodes;
    a.t_ok = (uint8_t*)(a.wz0 + n_nodes);
    a.freeb = a.t_ok + n_nodes;
    const int64_t chunk = search_chunk(G, n_nodes);
    float* map = (float*)(w + align_up((size_t)n_nodes * 32, 256));
    char* box = w + align_up((size_t)n_nodes * 32, 256) + align_up((size_t)chunk * G.nmap * sizeof(float), 256);
    a.map = map;
    a.disp = disp;
    a.cc = cc;
    a.pce = pce;
    a.clipped = clipped;
    a.ok = ok;
    a.part = nullptr;
    a.nblk = 0;
    a.blk_planes = 0;
    ncc_place_kernel<<<(unsigned)((n_nodes + 255) / 256), 256, 0, s>>>(a);
    rc = check_launch("ncc place");
    if (rc) return rc;
    TiledCfg tc;
    FftCfg fc;
    const bool fft = use_fft(G, engine, fc);
    const bool tiled = !fft && use_tiled(G, engine, tc);
    if (fft) tc.sxp = (G.sx + 3) / 4 * 4;
    TiledArgs ta;
    FftArgs fa;
    if (tiled || fft) {
        // window box sums of (g - c) and (g - c)^2 for every placement, c = a voxel of g near the centre
        const size_t vb = align_up((size_t)nz * ny * nx * sizeof(float), 256);
        float* t1 = (float*)box;
        float* t2 = (float*)(box + vb);
        float* b1 = (float*)(box + 2 * vb);
        float* b2 = (float*)(box + 3 * vb);
        const float* pilot_at = g + ((nz / 2) * ny + ny / 2) * nx + nx / 2;  // read by the kernel: no host round trip
        const int64_t nv = nz * ny * nx;
        const unsigned blocks = (unsigned)((nv + 255) / 256);
        // tiled passes while the window and the grid fit their limits, else one thread per output
        const bool tiles = G.sx <= BOX_MAX_LEN && G.sy <= BOX_MAX_LEN && G.sz <= BOX_MAX_LEN && nz <= 65535 && ny <= 65535;
        const unsigned gx_t = (unsigned)((nx + BOX_TL - 1) / BOX_TL), gy_32 = (unsigned)((ny + 31) / 32), gx_32 = (unsigned)((nx + 31) / 32);
        {
            KTimer kt_("box_pass", s);
            if (tiles)
                box_tile_x_kernel<<<dim3(gx_t, gy_32, (unsigned)nz), 256, 0, s>>>(g, b1, b2, (int)ny, (int)nx, G.sx, pilot_at);
            else
                box_pass_kernel<<<blocks, 256, 0, s>>>(g, nullptr, b1, b2, (int)nz, (int)ny, (int)nx, 0, G.sx, pilot_at, 1);
        }
        rc = check_launch("ncc box x");
        if (rc) return rc;
        {
            KTimer kt_("box_pass", s);
            if (tiles)
                box_tile_yz_kernel<1><<<dim3(gx_32, (unsigned)((ny + BOX_TL - 1) / BOX_TL), (unsigned)nz), 256, 0, s>>>(
                    b1, b2, t1, t2, (int)nz, (int)ny, (int)nx, G.sy);
            else
                box_pass_kernel<<<blocks, 256, 0, s>>>(b1, b2, t1, t2, (int)nz, (int)ny, (int)nx, 1, G.sy, nullptr, 0);
        }
        rc = check_launch("ncc box y");
        if (rc) return rc;
        {
            KTimer kt_("box_pass", s);
            if (tiles)
                box_tile_yz_kernel<2><<<dim3(gx_32, (unsigned)((nz + BOX_TL - 1) / BOX_TL), (unsigned)ny), 256, 0, s>>>(
                    t1, t2, b1, b2, (int)nz, (int)ny, (int)nx, G.sz);
            else
                box_pass_kernel<<<blocks, 256, 0, s>>>(t1, t2, b1, b2, (int)nz, (int)ny, (int)nx, 2, G.sz, nullptr, 0);
        }
        rc = check_launch("ncc box z");
        if (rc) return rc;
        ta.f = f;
        ta.g = g;
        ta.coords = coords;
        ta.wx0 = a.wx0;
        ta.wy0 = a.wy0;
        ta.wz0 = a.wz0;
        ta.t_ok = a.t_ok;
        ta.B1 = b1;
        ta.B2 = b2;
        float* tpl = (float*)(box + 4 * vb);
        ta.T = tpl;
        ta.ssf = (const double*)((char*)tpl + align_up((size_t)chunk * G.sz * G.sy * tc.sxp * sizeof(float), 256));
        if (fft) {
            if (fc.reg) {
                rc = fftr_upload();
                if (rc) return rc;
            }
            ta.sxp = tc.sxp;
            char* fw = box + 4 * vb + tiled_tpl_bytes(G, chunk);
            float2* tw = (float2*)fw;
            fft_twiddle_kernel<<<(3 * FFT_MAX_N + 127) / 128, 128, 0, s>>>(tw, fc.ax.n, fc.ay.n, fc.az.n);
            rc = check_launch("ncc fft twiddles");
            if (rc) return rc;
            const int64_t batch = fft_batch(fc, chunk);
            float2* scr = (float2*)(fw + align_up(3 * FFT_MAX_N * sizeof(float2), 256));
            fa.g = g;
            fa.coords = coords;
            fa.wx0 = a.wx0;
            fa.wy0 = a.wy0;
            fa.wz0 = a.wz0;
            fa.t_ok = a.t_ok;
            fa.B1 = b1;
            fa.B2 = b2;
            fa.pilot_at = pilot_at;
            fa.tw = tw;
            fa.A = scr;
            fa.P = scr + batch * (int64_t)G.wz * fc.ay.n * fc.ax.n;
            fa.part = nullptr;
            fa.nblk = 0;
            if (fc.reg) {  // the map partials follow the spectra scratch
                fa.nblk = fft_nblk(G, fc);
                fa.part = (MapPart*)((char*)scr + align_up((size_t)batch * fc.per_node, 256));
                a.part = fa.part;
                a.nblk = fa.nblk;
                a.blk_planes = fft_blk_planes(fc);
            }
            fa.n_nodes = n_nodes;
            fa.G = G;
            fa.sxp = tc.sxp;
            fa.ax = fc.ax;
            fa.ay = fc.ay;
            fa.az = fc.az;
            fa.pitch = fc.pitch;
        }
        ta.n_nodes = n_nodes;
        ta.G = G;
        ta.dz_slab = tc.dz;
        ta.ntile = tc.ntile;
        ta.pitch = tc.pitch;
        ta.plane_stride = tc.plane_stride;
        ta.sxp = tc.sxp;
    }
    for (int64_t start = 0; start < n_nodes; start += chunk) {
        const int64_t n = std::min(chunk, n_nodes - start);
        if (fft) {
            ta.node_base = start;
            rc = launch_templates(ta, n, s);
            if (rc) return rc;
            FftArgs fb = fa;
            fb.node_base = start;
            fb.out = map;
            fb.T = ta.T;
            fb.ssf = ta.ssf;
            rc = launch_fft(fb, fc, n, fft_batch(fc, chunk), s);
        } else if (tiled) {
            ta.node_base = start;
            ta.out = map;
            rc = launch_tiled(ta, tc, n, s);
        } else {
            MapArgs m{f, g, coords, a.wx0, a.wy0, a.wz0, a.t_ok, map, start, n_nodes, G};
            rc = launch_map(m, n, s);
        }
        if (rc) return rc;
        SearchArgs b = a;
        b.node_base = start;
        b.map = map;
        rc = launch_peak(b, n, s);
        if (rc) return rc;
    }
    return ALDVC_OK;
}
