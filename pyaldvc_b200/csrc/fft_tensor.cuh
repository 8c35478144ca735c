// FFT engine, pass 2 on the tensor pipe: the z transforms of the in-register engine's pass 2 (see fftr_pass2_kernel)
// as tcgen05 matrix products, a comparison form of that pass (ALDVC_FFT_PASS2=tensor).
//
// Work is cut into line pairs: pair (node, ky <= N/2, c) owns the z line of the packed spectrum Z = W + iT at row ky,
// column c, and lends the line at row -ky, column -c (mod N), whose spectrum gives the conjugate half of the product.
// A CTA takes 128 pairs at a time as two tiles of 64; a tile is one M = 128 product with the pair's own line in even
// rows and the lent line in the odd row after it, so a pair shares one warp and trades values with one shuffle.
//   forward   D1[line][2kz + re/im] = sum_z A[line][2z + re/im] F[2kz + re/im][2z + re/im]   (DFT along z, sign -1)
//   product   Q[kz] = (Za + conj Zb) / 2 * i conj(Za - conj Zb) / 2, Za = own line at kz, Zb = lent line at -kz
//   inverse   D2[pair][2dz + re/im] = sum_kz conj Q[kz] F[...]: the forward matrix on conj Q, conjugated (sign +1)
// Operands are FP32 split into two TF32 terms (x = hi + lo); each product is hi*hi + hi*lo + lo*hi with FP32
// accumulation in tensor memory, so the transforms keep about 21 bits where a single TF32 product keeps 11.
// Shared memory holds the DFT matrix (hi, lo) and one 128-row operand (hi, lo) in the canonical no-swizzle K-major
// layout: 8-row x 16-byte core matrices, K chunks 128 bytes apart, 8-row groups K/4 * 128 bytes apart.
// Tensor memory: 256 columns, the two forward products at columns 0 and 128, the inverse at 0 once the products
// have read them (so two CTAs on one SM could both allocate).

constexpr int FFTT_THREADS = 128;
constexpr long long FFTT_WAIT_LIMIT = 1LL << 22;  // polls of an mbarrier before a wait gives up
constexpr int FFTT_TMEM_COLS = 256;

__device__ int g_fftt_err;  // set when an MMA completion wait gave up (read by the launcher)

template <int N>
struct FfttShape {
    static constexpr int K = (2 * N + 7) / 8 * 8;      // tf32 MMAs take K = 8
    static constexpr int NN = (2 * N + 15) / 16 * 16;  // M = 128 needs N a multiple of 16
    static constexpr int KC = K / 4;                   // 16-byte chunks along K
    static constexpr uint32_t SBO = KC * 128;          // bytes between 8-row groups
    static constexpr size_t A_BYTES = (size_t)128 * K * 4;
    static constexpr size_t B_BYTES = (size_t)NN * K * 4;
    static constexpr size_t SMEM = 2 * A_BYTES + 2 * B_BYTES + 64;
};

__device__ __forceinline__ uint32_t fftt_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ float fftt_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// float index of element (row r, k) in the canonical layout with KC chunks of K
template <int KC>
__device__ __forceinline__ int fftt_idx(int r, int k) {
    return (k >> 2) * 32 + (r >> 3) * (KC * 32) + (r & 7) * 4 + (k & 3);
}

// shared-memory matrix descriptor: no swizzle, K-major, leading (K chunk) offset 128 bytes, stride (8-row group) sbo
__device__ __forceinline__ uint64_t fftt_desc(uint32_t saddr, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((128u >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: D f32, A and B tf32, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t fftt_idesc(int n) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void fftt_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void fftt_commit(uint32_t mb) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mb) : "memory");
}

__device__ __forceinline__ bool fftt_try_wait(uint32_t mb, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(mb), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool fftt_wait(uint32_t mb, uint32_t parity) {
    for (long long i = 0; i < FFTT_WAIT_LIMIT; ++i)
        if (fftt_try_wait(mb, parity)) return true;
    return false;
}

__device__ __forceinline__ void fftt_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fftt_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fftt_fence_proxy() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive columns of this thread's lane
__device__ __forceinline__ void fftt_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
          "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void fftt_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// the pair's line: own (odd = 0) at (ky, c), lent (odd = 1) at (-ky, -c); false past the end or for a node without a map
template <int N>
__device__ __forceinline__ bool fftt_pair(const FftArgs& a, int64_t j, int& bn, int& ky, int& c) {
    constexpr int64_t PER = (int64_t)(N / 2 + 1) * N;
    if (j >= (int64_t)a.nb * PER) return false;
    bn = (int)(j / PER);
    const int r = (int)(j - (int64_t)bn * PER);
    ky = r / N;
    c = r - ky * N;
    return fft_node_ok(a, a.node_base + bn);
}

// one 128-row product of the operand in shared memory with the DFT matrix into tensor memory column d
template <int N>
__device__ __forceinline__ void fftt_gemm(uint32_t d, uint32_t ahi, uint32_t alo, uint32_t bhi, uint32_t blo, uint32_t mb) {
    using S = FfttShape<N>;
    constexpr uint32_t idesc = fftt_idesc(S::NN);
#pragma unroll 1
    for (int s = 0; s < S::K / 8; ++s) {
        const uint32_t ko = (uint32_t)s * 256u;
        const uint64_t ah = fftt_desc(ahi + ko, S::SBO), al = fftt_desc(alo + ko, S::SBO);
        const uint64_t bh = fftt_desc(bhi + ko, S::SBO), bl = fftt_desc(blo + ko, S::SBO);
        fftt_mma(d, ah, bh, idesc, s > 0 ? 1u : 0u);
        fftt_mma(d, ah, bl, idesc, 1u);
        fftt_mma(d, al, bh, idesc, 1u);
    }
    fftt_commit(mb);
}

template <int N>
__global__ void __launch_bounds__(FFTT_THREADS, 1) fftt_pass2_kernel(FftArgs a, int64_t n_groups) {
    using S = FfttShape<N>;
    constexpr int NH = N / 2 + 1;
    constexpr int K = S::K, KC = S::KC, NN = S::NN;
    extern __shared__ __align__(128) unsigned char tsm[];
    float* Ahi = reinterpret_cast<float*>(tsm);
    float* Alo = Ahi + 128 * K;
    float* Bhi = Alo + 128 * K;
    float* Blo = Bhi + NN * K;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(tsm + 2 * S::A_BYTES + 2 * S::B_BYTES);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
    __shared__ double2 twd[N];  // cos, sin of 2 pi j / N
    const int tid = threadIdx.x, warp = tid >> 5;
    const NccGeom& G = a.G;
    const uint32_t mb = fftt_smem(mbar);

    for (int j = tid; j < N; j += FFTT_THREADS) {
        double sn, cs;
        sincospi(2.0 * j / N, &sn, &cs);
        twd[j] = make_double2(cs, sn);
    }
    __syncthreads();
    // forward DFT matrix, row n = 2 kz + (0 re, 1 im), column k = 2 z + (0 re, 1 im):
    // Re Z[kz] = sum Re a cos t + Im a sin t, Im Z[kz] = sum Im a cos t - Re a sin t, t = 2 pi kz z / N
    for (int e = tid; e < NN * K; e += FFTT_THREADS) {
        const int n = e / K, k = e - (e / K) * K;
        double v = 0.0;
        if (n < 2 * N && k < 2 * N) {
            const double2 t = twd[((n >> 1) * (k >> 1)) % N];
            v = (n & 1) == 0 ? ((k & 1) == 0 ? t.x : t.y) : ((k & 1) == 0 ? -t.y : t.x);
        }
        const float hi = fftt_tf32((float)v);
        const int o = fftt_idx<KC>(n, k);
        Bhi[o] = hi;
        Blo[o] = fftt_tf32((float)(v - (double)hi));
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mb), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(fftt_smem(tslot)), "r"(FFTT_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fftt_fence_proxy();
    fftt_fence_before();
    __syncthreads();
    fftt_fence_after();
    const uint32_t tbase = *tslot;
    const uint32_t lane_base = tbase + ((uint32_t)(warp * 32) << 16);
    const uint32_t ahi = fftt_smem(Ahi), alo = fftt_smem(Alo), bhi = fftt_smem(Bhi), blo = fftt_smem(Blo);
    const bool odd = (tid & 1) != 0;
    uint32_t phase = 0;
    bool failed = false;

    // all threads wait for the MMAs committed last; false (everywhere) when a wait gave up
    auto wait_mma = [&]() -> bool {
        const bool ok = fftt_wait(mb, phase);
        phase ^= 1u;
        const bool bad = __syncthreads_or(!ok) != 0;
        fftt_fence_after();
        return !bad;
    };

    for (int64_t grp = blockIdx.x; grp < n_groups && !failed; grp += gridDim.x) {
        // ---- forward transforms of the group's two tiles
        for (int t = 0; t < 2 && !failed; ++t) {
            const int64_t j = grp * 128 + t * 64 + (tid >> 1);
            int bn = 0, ky = 0, c = 0;
            const bool live = fftt_pair<N>(a, j, bn, ky, c);
            float2 v[K / 2];
            if (live) {
                const int ly = odd ? (N - ky) % N : ky, lc = odd ? (N - c) % N : c;
                const float2* col = a.A + (int64_t)bn * G.wz * N * N + ly * N + lc;
#pragma unroll
                for (int z = 0; z < K / 2; ++z) v[z] = z < G.wz ? col[(int64_t)z * N * N] : make_float2(0.0f, 0.0f);
            } else {
#pragma unroll
                for (int z = 0; z < K / 2; ++z) v[z] = make_float2(0.0f, 0.0f);
            }
#pragma unroll
            for (int q = 0; q < KC; ++q) {
                const float x[4] = {v[2 * q].x, v[2 * q].y, v[2 * q + 1].x, v[2 * q + 1].y};
                float4 h, l;
                h.x = fftt_tf32(x[0]);
                h.y = fftt_tf32(x[1]);
                h.z = fftt_tf32(x[2]);
                h.w = fftt_tf32(x[3]);
                l.x = fftt_tf32(x[0] - h.x);
                l.y = fftt_tf32(x[1] - h.y);
                l.z = fftt_tf32(x[2] - h.z);
                l.w = fftt_tf32(x[3] - h.w);
                const int o = fftt_idx<KC>(tid, 4 * q);
                *reinterpret_cast<float4*>(Ahi + o) = h;
                *reinterpret_cast<float4*>(Alo + o) = l;
            }
            fftt_fence_proxy();
            fftt_fence_before();
            __syncthreads();
            if (tid == 0) {
                fftt_fence_after();
                fftt_gemm<N>(tbase + (uint32_t)(t * 128), ahi, alo, bhi, blo, mb);
            }
            failed = !wait_mma();
        }
        if (failed) break;
        // ---- products into the operand rows t * 64 + pair (conjugated for the inverse)
        for (int t = 0; t < 2; ++t) {
            float d[NN];
#pragma unroll
            for (int q = 0; q < NN / 16; ++q) fftt_ld16(lane_base + (uint32_t)(t * 128 + q * 16), d + 16 * q);
            fftt_wait_ld();
            const int row = t * 64 + (tid >> 1);
#pragma unroll
            for (int q = 0; q < KC; ++q) {
                float x[4];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int kz = 2 * q + h;
                    if (kz < N) {
                        const int km = (N - kz) % N;
                        const float zbx = __shfl_xor_sync(0xffffffffu, d[2 * km], 1);
                        const float zby = __shfl_xor_sync(0xffffffffu, d[2 * km + 1], 1);
                        const float2 za = make_float2(d[2 * kz], d[2 * kz + 1]);
                        const float2 zbc = make_float2(zbx, -zby);
                        const float2 w = make_float2(0.5f * (za.x + zbc.x), 0.5f * (za.y + zbc.y));
                        const float2 df = make_float2(za.x - zbc.x, za.y - zbc.y);
                        const float2 tc = make_float2(0.5f * df.y, 0.5f * df.x);
                        const float2 pq = make_float2(w.x * tc.x - w.y * tc.y, w.x * tc.y + w.y * tc.x);
                        x[2 * h] = pq.x;
                        x[2 * h + 1] = -pq.y;
                    } else {
                        x[2 * h] = 0.0f;
                        x[2 * h + 1] = 0.0f;
                    }
                }
                if (!odd) {
                    float4 hh, ll;
                    hh.x = fftt_tf32(x[0]);
                    hh.y = fftt_tf32(x[1]);
                    hh.z = fftt_tf32(x[2]);
                    hh.w = fftt_tf32(x[3]);
                    ll.x = fftt_tf32(x[0] - hh.x);
                    ll.y = fftt_tf32(x[1] - hh.y);
                    ll.z = fftt_tf32(x[2] - hh.z);
                    ll.w = fftt_tf32(x[3] - hh.w);
                    const int o = fftt_idx<KC>(row, 4 * q);
                    *reinterpret_cast<float4*>(Ahi + o) = hh;
                    *reinterpret_cast<float4*>(Alo + o) = ll;
                }
            }
        }
        // ---- inverse transforms of the 128 own lines
        fftt_fence_proxy();
        fftt_fence_before();
        __syncthreads();
        if (tid == 0) {
            fftt_fence_after();
            fftt_gemm<N>(tbase, ahi, alo, bhi, blo, mb);
        }
        if (!wait_mma()) {
            failed = true;
            break;
        }
        {
            float d[NN];
#pragma unroll
            for (int q = 0; q < NN / 16; ++q) fftt_ld16(lane_base + (uint32_t)(q * 16), d + 16 * q);
            fftt_wait_ld();
            const int64_t j = grp * 128 + tid;  // row tid holds pair tid of the group (tile tid / 64)
            int bn = 0, ky = 0, c = 0;
            if (fftt_pair<N>(a, j, bn, ky, c)) {
                float2* dst = a.P + (int64_t)bn * G.vz * NH * N + ky * N + c;
#pragma unroll
                for (int dz = 0; dz < N; ++dz)
                    if (dz < G.vz) dst[(int64_t)dz * NH * N] = make_float2(d[2 * dz], -d[2 * dz + 1]);
            }
        }
        fftt_fence_before();
        __syncthreads();
        fftt_fence_after();
    }
    if (failed) {
        if (tid == 0) atomicExch(&g_fftt_err, 1);
        fftt_wait(mb, phase ^ 1u);  // the last commit's MMAs, if they are still running
    }
    fftt_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(FFTT_TMEM_COLS) : "memory");
}
