// graph_common.cuh -- pieces shared by the node-graph solvers (graph_pairs.cu, graph_solve.cu): constants, the
// per-job statistics record, fixed-order block reductions, the SM count and the parameter checks.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "../../include/lsb_omniscape.h"

namespace lsbg {
namespace {

// Threads per CTA: 512 (two CTAs per SM) for components of at least kWideNodes nodes, else 256 (four per SM).
constexpr int kWideNodes = 8192;
inline int threads_for(int64_t n) { return n >= kWideNodes ? 512 : 256; }
inline int ctas_per_sm(int nt) { return nt == 512 ? 2 : 4; }
constexpr int kMaxRestarts = 64;
constexpr size_t kAlign = 256;
constexpr double kScratchCap = 8.0 * 1024 * 1024 * 1024;  // bytes of per-CTA vectors at most

size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

void set_err(char *err, size_t len, const char *fmt, ...) {
    if (!err || len == 0) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, len, fmt, ap);
    va_end(ap);
}

struct JobStat {
    int32_t iters;  // CG iterations; -1: the job's node indices were out of range
    int32_t ok;     // final relative residual <= accept
    double resid;   // final relative residual ||b - A x|| / ||b||
};
static_assert(sizeof(JobStat) == 16, "JobStat layout");

// Sum of (a, b) over the block, the same value in every thread: warp butterflies, then the warps' partial sums
// added in warp order.  The leading barrier lets a previous call's readers finish with `red`.
template <int NT>
__device__ __forceinline__ double2 block_sum2(double a, double b, double2 *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = make_double2(a, b);
    __syncthreads();
    double2 s = red[0];
#pragma unroll
    for (int i = 1; i < NT / 32; ++i) {
        s.x += red[i].x;
        s.y += red[i].y;
    }
    return s;
}

template <int NT>
__device__ __forceinline__ double2 block_max2(double a, double b, double2 *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ta = __shfl_xor_sync(0xffffffffu, a, o), tb = __shfl_xor_sync(0xffffffffu, b, o);
        a = ta > a ? ta : a;
        b = tb > b ? tb : b;
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = make_double2(a, b);
    __syncthreads();
    double2 s = red[0];
#pragma unroll
    for (int i = 1; i < NT / 32; ++i) {
        s.x = red[i].x > s.x ? red[i].x : s.x;
        s.y = red[i].y > s.y ? red[i].y : s.y;
    }
    return s;
}

int device_sms() {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) {
        cudaGetLastError();  // no device here: size for a B200
        return 148;
    }
    return sms;
}

bool valid(int64_t n, int64_t n_jobs, const lsb_graph_params *p, char *err, size_t errlen) {
    if (!p) {
        set_err(err, errlen, "params is NULL");
        return false;
    }
    if (n < 1 || n > INT32_MAX) {
        set_err(err, errlen, "the component must have between 1 and 2^31 - 1 nodes (got %lld)", (long long)n);
        return false;
    }
    if (n_jobs < 0) {
        set_err(err, errlen, "n_jobs must be >= 0");
        return false;
    }
    if (!(p->tol >= 0.0) || !(p->accept > 0.0) || p->max_iter < 0 || p->max_ctas < 0) {
        set_err(err, errlen, "tol must be >= 0, accept > 0, max_iter and max_ctas >= 0");
        return false;
    }
    return true;
}

}  // namespace
}  // namespace lsbg
