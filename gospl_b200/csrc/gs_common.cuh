// Common device helpers for the goSPL hot path on sm_100a.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "../../include/gospl_b200.h"

namespace gs {

// ---------------------------------------------------------------------------
// error state (per host thread) and launch checking
// ---------------------------------------------------------------------------
void set_error(int code, const std::string& msg);
int last_code();

#define GS_CUDA(call)                                                                  \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            ::gs::set_error(GS_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
            return GS_ECUDA;                                                           \
        }                                                                              \
    } while (0)

#define GS_LAUNCH()                                                                    \
    do {                                                                               \
        cudaError_t e_ = cudaGetLastError();                                           \
        if (e_ != cudaSuccess) {                                                       \
            ::gs::set_error(GS_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
            return GS_ECUDA;                                                           \
        }                                                                              \
    } while (0)

#define GS_TRY(expr)                                                                   \
    do {                                                                               \
        int s_ = (expr);                                                               \
        if (s_ != GS_OK) return s_;                                                    \
    } while (0)

constexpr int MAXW = 12;        // neighbour slots per vertex (FVnID width)
constexpr int MAXR = 12;        // receivers per vertex

inline int grid_for(int64_t n, int block) {
    int64_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 1 << 30) g = 1 << 30;
    return (int)g;
}

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_relaxed_s32(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Total order on doubles as unsigned 64-bit keys (for atomicMin/Max on doubles).
__device__ __forceinline__ unsigned long long dkey(double x) {
    unsigned long long u = (unsigned long long)__double_as_longlong(x);
    return (u & 0x8000000000000000ULL) ? ~u : (u | 0x8000000000000000ULL);
}
__device__ __forceinline__ double dkey_inv(unsigned long long k) {
    unsigned long long u = (k & 0x8000000000000000ULL) ? (k & 0x7fffffffffffffffULL) : ~k;
    return __longlong_as_double((long long)u);
}

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace gs
