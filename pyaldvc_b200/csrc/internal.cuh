// Host-side plumbing shared by the entry points: error reporting and launch helpers.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/aldvc_b200.h"

namespace aldvc {

void set_error(const char* fmt, ...);

inline int cuda_fail(cudaError_t e, const char* where) {
    set_error("%s: %s", where, cudaGetErrorString(e));
    return ALDVC_ERR_CUDA;
}

inline int arg_fail(const char* msg) {
    set_error("%s", msg);
    return ALDVC_ERR_ARG;
}

void count_launch();

// Enqueue check after a launch: a launch error is reported, an earlier asynchronous error is left
// for the caller's next synchronisation.  Every successful check counts one kernel launch.
inline int check_launch(const char* where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, where);
    count_launch();
    return ALDVC_OK;
}

int sm_count();
int max_smem_optin();

// Device time of one launch (CUDA events on its stream, around the launch) while kernel timing is on
// (aldvc_kernel_timing); nothing is recorded otherwise, nor on a stream under capture.
struct KTimer {
    const char* name;
    cudaStream_t s;
    cudaEvent_t a = nullptr;
    KTimer(const char* n, cudaStream_t st);
    ~KTimer();
};

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Grid-barrier parameters of the cooperative kernels: a barrier opens when the launch's blocks plus
// `extra` have arrived, and a block stops waiting after `spin_limit` polls.  Production launches use
// extra = 0 and DEFAULT_SPIN_LIMIT; aldvc_test_set_barrier changes both for the tests of the give-up path.
constexpr long long DEFAULT_SPIN_LIMIT = 1LL << 24;
struct BarrierParams {
    unsigned int extra;
    long long spin_limit;
};
BarrierParams barrier_params();

}  // namespace aldvc

#define ALDVC_REQUIRE(cond, msg) \
    do {                          \
        if (!(cond)) return aldvc::arg_fail(msg); \
    } while (0)
