// Library-level entry points: ABI version, error string, device query; the stencil-7 gradient kernel.
#include <atomic>
#include <cstring>
#include <mutex>

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

}  // namespace aldvc

using namespace aldvc;

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
