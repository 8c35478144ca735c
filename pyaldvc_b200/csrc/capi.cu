// Library-level entry points: ABI version, error string, device query; the stencil-7 gradient kernel.
#include <atomic>
#include <cstring>
#include <mutex>
#include <vector>
#include <algorithm>

#include "common.cuh"
#include "internal.cuh"

namespace aldvc {

static thread_local char g_err[512] = "";
static std::atomic<unsigned long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 148;
    return n;
}

int max_smem_optin() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 227 * 1024;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 227 * 1024;
    return n;
}

// io/volume_ops._gradient_stencil7 (:124-155): one thread per voxel along x, FP64 combination of
// float32 voxel differences (the reference rounds each difference to float32), float32 result.
__global__ void gradients_kernel(const float* __restrict__ f, int nz, int ny, int nx, int border, float* __restrict__ gx,
                                 float* __restrict__ gy, float* __restrict__ gz) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= nx) return;
    const int64_t sxy = (int64_t)nx * ny;
    const int64_t o = (int64_t)z * sxy + (int64_t)y * nx + x;
    const bool in = z >= border && z < nz - border && y >= border && y < ny - border && x >= border && x < nx - border;
    if (!in) {
        gx[o] = 0.0f;
        gy[o] = 0.0f;
        gz[o] = 0.0f;
        return;
    }
    const double c1 = 3.0 / 4.0, c2 = -3.0 / 20.0, c3 = 1.0 / 60.0;
    auto d = [&](int64_t s, int k) -> double { return (double)(__ldg(f + o + k * s) - __ldg(f + o - k * s)); };
    // explicit round-to-nearest products and sums: no contraction into FMA, the reference's rounding
    auto comb = [&](int64_t s) -> float {
        return (float)__dadd_rn(__dadd_rn(__dmul_rn(c1, d(s, 1)), __dmul_rn(c2, d(s, 2))), __dmul_rn(c3, d(s, 3)));
    };
    gx[o] = comb(1);
    gy[o] = comb(nx);
    gz[o] = comb(sxy);
}

// ---- kernel timing (off by default)
static std::mutex g_tmu;
static std::atomic<bool> g_timing{false};
struct TRec {
    const char* name;
    cudaEvent_t a, b;
};
static std::vector<TRec> g_trecs;

KTimer::KTimer(const char* n, cudaStream_t st) : name(n), s(st) {
    if (!g_timing.load(std::memory_order_relaxed)) return;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
    if (cudaEventCreate(&a) != cudaSuccess) {
        a = nullptr;
        return;
    }
    cudaEventRecord(a, s);
}

KTimer::~KTimer() {
    if (!a) return;
    cudaEvent_t b;
    if (cudaEventCreate(&b) != cudaSuccess) {
        cudaEventDestroy(a);
        return;
    }
    cudaEventRecord(b, s);
    std::lock_guard<std::mutex> lock(g_tmu);
    g_trecs.push_back({name, a, b});
}

static void clear_timing() {
    for (auto& r : g_trecs) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    g_trecs.clear();
}

}  // namespace aldvc

using namespace aldvc;

extern "C" int aldvc_kernel_timing(int enable) {
    std::lock_guard<std::mutex> lock(g_tmu);
    clear_timing();
    g_timing.store(enable != 0);
    return ALDVC_OK;
}

extern "C" int aldvc_kernel_timing_read(int32_t max_entries, char* names, int32_t name_len, double* ms, int64_t* launches) {
    ALDVC_REQUIRE(max_entries >= 0 && (max_entries == 0 || (names && name_len > 1 && ms && launches)),
                  "aldvc_kernel_timing_read: bad output buffers");
    std::lock_guard<std::mutex> lock(g_tmu);
    std::vector<const char*> keys;
    std::vector<double> tot;
    std::vector<int64_t> cnt;
    for (auto& r : g_trecs) {
        cudaError_t e = cudaEventSynchronize(r.b);
        if (e != cudaSuccess) return cuda_fail(e, "aldvc_kernel_timing_read");
        float t = 0.0f;
        e = cudaEventElapsedTime(&t, r.a, r.b);
        if (e != cudaSuccess) return cuda_fail(e, "aldvc_kernel_timing_read");
        size_t k = 0;
        while (k < keys.size() && std::strcmp(keys[k], r.name) != 0) ++k;
        if (k == keys.size()) {
            keys.push_back(r.name);
            tot.push_back(0.0);
            cnt.push_back(0);
        }
        tot[k] += (double)t;
        cnt[k] += 1;
    }
    const int n = (int)std::min<size_t>(keys.size(), (size_t)max_entries);
    for (int i = 0; i < n; ++i) {
        std::strncpy(names + (size_t)i * name_len, keys[i], (size_t)name_len - 1);
        names[(size_t)i * name_len + name_len - 1] = 0;
        ms[i] = tot[i];
        launches[i] = cnt[i];
    }
    return (int)keys.size();
}

static std::atomic<unsigned int> g_bar_extra{0};
static std::atomic<long long> g_bar_spins{aldvc::DEFAULT_SPIN_LIMIT};

aldvc::BarrierParams aldvc::barrier_params() {
    return aldvc::BarrierParams{g_bar_extra.load(std::memory_order_relaxed), g_bar_spins.load(std::memory_order_relaxed)};
}

extern "C" int aldvc_test_set_barrier(int32_t extra_arrivals, int64_t spin_limit) {
    ALDVC_REQUIRE(extra_arrivals >= 0 && extra_arrivals <= 1024, "aldvc_test_set_barrier: extra_arrivals must be in [0, 1024]");
    g_bar_extra.store((unsigned int)extra_arrivals, std::memory_order_relaxed);
    g_bar_spins.store(spin_limit > 0 ? (long long)spin_limit : aldvc::DEFAULT_SPIN_LIMIT, std::memory_order_relaxed);
    return ALDVC_OK;
}

extern "C" int aldvc_abi_version(void) { return ALDVC_ABI_VERSION; }

extern "C" const char* aldvc_last_error(void) { return g_err; }

extern "C" unsigned long long aldvc_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

extern "C" int aldvc_device_info(int device, char* name, int name_len, int* sm, int* cc_major, int* cc_minor) {
    cudaDeviceProp p;
    cudaError_t e = cudaGetDeviceProperties(&p, device);
    if (e != cudaSuccess) return cuda_fail(e, "aldvc_device_info");
    if (name && name_len > 0) {
        std::strncpy(name, p.name, (size_t)name_len - 1);
        name[name_len - 1] = 0;
    }
    if (sm) *sm = p.multiProcessorCount;
    if (cc_major) *cc_major = p.major;
    if (cc_minor) *cc_minor = p.minor;
    return ALDVC_OK;
}

extern "C" int aldvc_gradients(const float* f, int64_t nz, int64_t ny, int64_t nx, int32_t border, float* gx, float* gy, float* gz,
                               void* stream) {
    ALDVC_REQUIRE(f && gx && gy && gz, "aldvc_gradients: null pointer");
    ALDVC_REQUIRE(nz > 0 && ny > 0 && nx > 0 && ny <= 65535 && nz <= 65535 && nx < (1LL << 31), "aldvc_gradients: bad shape");
    dim3 block(128);
    dim3 grid((unsigned)((nx + 127) / 128), (unsigned)ny, (unsigned)nz);
    gradients_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(f, (int)nz, (int)ny, (int)nx, border, gx, gy, gz);
    return check_launch("aldvc_gradients");
}
