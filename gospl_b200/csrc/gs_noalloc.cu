// Allocation-free variant of the flow-accumulation solve.
//
// Some callers cannot allocate device memory: code running inside another
// application's CUDA context with a fixed memory budget, or plugins driven
// from a framework that owns every allocation and forbids cudaMalloc outside
// its own allocator.  gs_flow_solve_noalloc gives them the exact
// solve of (I - W^T) q = b for a receiver graph without any allocation: every
// scratch array lives in one file-scope __device__ array of fixed size, held
// by each GPU that loads this library until the process exits.
//
// Limits: at most GS_NOALLOC_MAX_NB vertices and GS_NOALLOC_MAX_RCV receivers
// per vertex; larger inputs are rejected with GS_EINVAL.  All calls share the
// one scratch array, so calls that overlap on the GPU (different streams, or
// different host threads on the same device) race and must be serialised by
// the caller.  The first call on a device resolves the array's device address
// with cudaGetSymbolAddress (once per device, under a lock, with the device
// of `stream` current); make that first call before any stream capture.  The
// call synchronises `stream` to read the solve's status.
#include <cub/cub.cuh>

#include <mutex>

#include "gs_plan.cuh"

namespace gs {

constexpr int NA_MAX_NB = GS_NOALLOC_MAX_NB;
constexpr int NA_MAX_R = GS_NOALLOC_MAX_RCV;
constexpr size_t NA_CUB_BYTES = 1 << 20;   // scan workspace, checked at set-up

// layout (ints unless noted): cnt[N] left[N] fill[N] queue[N] dptr[N+1]
// dlist[N*R] done(u8)[N] ctr[16] cub[NA_CUB_BYTES]
constexpr size_t NA_INTS = (size_t)NA_MAX_NB * (5 + NA_MAX_R) + 1 + 16;
constexpr size_t NA_BYTES = NA_INTS * 4 + (size_t)NA_MAX_NB + NA_CUB_BYTES + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

struct NaLayout {
    int* cnt;
    int* left;
    int* fill;
    int* queue;
    int* dptr;
    int* dlist;
    unsigned* ctr;
    uint8_t* done;
    void* cub;
};

static NaLayout na_layout(unsigned char* base) {
    NaLayout L;
    int* p = (int*)base;
    const size_t N = NA_MAX_NB;
    L.cnt = p;
    L.left = p + N;
    L.fill = p + 2 * N;
    L.queue = p + 3 * N;
    L.dptr = p + 4 * N;
    L.dlist = p + 5 * N + 1;
    L.ctr = (unsigned*)(p + 5 * N + 1 + N * NA_MAX_R);
    L.done = (uint8_t*)(L.ctr + 16);
    size_t off = (size_t)((unsigned char*)(L.done + N) - base);
    off = (off + 255) & ~(size_t)255;
    L.cub = base + off;
    return L;
}

// one address per device, resolved on first use with that device current
static std::mutex g_na_mutex;
static unsigned char* g_na_ptr[64] = {nullptr};

// The device is the one that owns `s`; it must also be the current device,
// since the symbol address and the launches are resolved there.
static int na_device(cudaStream_t s, int* out) {
    int cur = 0, dev = 0;
    GS_CUDA(cudaGetDevice(&cur));
    GS_CUDA(cudaStreamGetDevice(s, &dev));
    if (dev != cur) {
        set_error(GS_EINVAL, "gs_flow_solve_noalloc: the stream belongs to another device than the current one");
        return GS_EINVAL;
    }
    *out = dev;
    return GS_OK;
}

static int na_base(int dev, unsigned char** out) {
    if (dev < 0 || dev >= 64) {
        set_error(GS_EINVAL, "gs_flow_solve_noalloc: device index out of range");
        return GS_EINVAL;
    }
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_ptr[dev]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) {
            set_error(GS_ECUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
            return GS_ECUDA;
        }
        size_t need = 0;
        cub::DeviceScan::ExclusiveSum((void*)nullptr, need, (const int*)nullptr, (int*)nullptr, NA_MAX_NB + 1);
        if (need > NA_CUB_BYTES) {
            set_error(GS_EINVAL, "gs_flow_solve_noalloc: scan workspace too small");
            return GS_EINVAL;
        }
        g_na_ptr[dev] = (unsigned char*)ptr;
    }
    *out = g_na_ptr[dev];
    return GS_OK;
}

__global__ void k_na_count(int n, int R, const int* __restrict__ rcv, const double* __restrict__ w, int* cnt) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    for (int k = 0; k < R; k++) {
        int r = rcv[(size_t)k * n + j];
        if (r != j && r >= 0 && r < n && w[(size_t)k * n + j] != 0.0) atomicAdd(&cnt[r], 1);
    }
}

__global__ void k_na_fill(int n, int R, const int* __restrict__ rcv, const double* __restrict__ w,
                          const int* __restrict__ dptr, int* fill, int* dlist) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    for (int k = 0; k < R; k++) {
        int r = rcv[(size_t)k * n + j];
        if (r != j && r >= 0 && r < n && w[(size_t)k * n + j] != 0.0)
            dlist[dptr[r] + atomicAdd(&fill[r], 1)] = (k << 24) | j;
    }
}

// donors of each vertex in ascending id (insertion sort of the segment), so
// the pull sums have a fixed order; vertices without donors are the sources
__global__ void k_na_sort(int n, const int* __restrict__ dptr, int* dlist, const int* __restrict__ cnt,
                          int* left, uint8_t* done, unsigned* ctr) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int a = dptr[i], b = dptr[i + 1];
    for (int x = a + 1; x < b; x++) {
        int v = dlist[x];
        int y = x - 1;
        while (y >= a && (dlist[y] & 0xffffff) > (v & 0xffffff)) {
            dlist[y + 1] = dlist[y];
            y--;
        }
        dlist[y + 1] = v;
    }
    left[i] = cnt[i];
    done[i] = cnt[i] == 0 ? 2 : 0;
    if (cnt[i] == 0) atomicAdd(&ctr[4], 1u);
}

struct NaFlowOp {
    int n, R;
    const int* dptr;
    const int* dlist;
    const int* rcv;
    const double* w;
    const double* b;
    double* q;
    uint8_t* done;
    __device__ __forceinline__ void process(int i, const struct NaSched& sc) const;
};

struct NaSched {
    int* queue;
    unsigned* ctr;
    int* cnt;
    unsigned n;
    __device__ __forceinline__ void publish(int r) const {
        unsigned s = atomicAdd(&ctr[1], 1u);
        if (s < n) st_release(&queue[s], r);
    }
    __device__ __forceinline__ void dec(int r) const {
        if (atomicSub(&cnt[r], 1) == 1) publish(r);
    }
};

__device__ __forceinline__ void NaFlowOp::process(int i, const NaSched& sc) const {
    double s = b[i];
    for (int x = dptr[i]; x < dptr[i + 1]; x++) {
        int e = dlist[x];
        int j = e & 0xffffff, k = e >> 24;
        s = s + w[(size_t)k * n + j] * __ldcg(&q[j]);
    }
    __stcg(&q[i], s);
    done[i] = 1;
    __threadfence();
    for (int k = 0; k < R; k++) {
        int r = rcv[(size_t)k * n + i];
        if (r != i && r >= 0 && r < n && w[(size_t)k * n + i] != 0.0) sc.dec(r);
    }
}

__global__ void k_na_sources(NaFlowOp op, NaSched sc, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && op.done[i] == 2) op.process(i, sc);
}

// Queue-driven sweep of the remaining vertices (warp-cooperative polling,
// bounded waits: a stalled queue with nothing in flight is a cycle, and a
// wall-clock budget backs that up).
__global__ void k_na_sweep(NaFlowOp op, NaSched sc, int n_all, unsigned long long budget_ns) {
    const unsigned long long t0 = globaltimer_ns();
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    const int n = n_all - (int)sc.ctr[4];
    for (;;) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(&sc.ctr[0], 32u);
        base = __shfl_sync(full, base, 0);
        if (base >= (unsigned)n) return;
        const unsigned t = base + lane;
        unsigned pending = __ballot_sync(full, t < (unsigned)n);
        unsigned rounds = 0;
        while (pending) {
            int node = -1;
            if (pending & (1u << lane)) node = ld_relaxed_s32(&sc.queue[t]);
            unsigned ready = __ballot_sync(full, node >= 0) & pending;
            if (ready) {
                __threadfence();
                if (ready & (1u << lane)) op.process(node, sc);
                __syncwarp();
                __threadfence();
                if (lane == 0) atomicAdd(&sc.ctr[2], (unsigned)__popc(ready));
                pending &= ~ready;
                continue;
            }
            if ((++rounds & 31u) == 0) {
                int stop = 0;
                if (lane == 0) {
                    unsigned d = 0;
                    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(d) : "l"(&sc.ctr[2]) : "memory");
                    unsigned tl = ld_relaxed_u32(&sc.ctr[1]);
                    unsigned first = base + (__ffs(pending) - 1);
                    if (ld_relaxed_u32(&sc.ctr[3]) != 0) stop = 1;
                    else if (d == tl && tl <= first) {
                        atomicCAS(&sc.ctr[3], 0u, (unsigned)GS_ECYCLE);
                        stop = 1;
                    } else if (globaltimer_ns() - t0 > budget_ns) {
                        atomicCAS(&sc.ctr[3], 0u, (unsigned)GS_ETIMEOUT);
                        stop = 1;
                    }
                }
                if (__shfl_sync(full, stop, 0)) return;
            }
            __nanosleep(128);
        }
    }
}

}  // namespace gs

extern "C" int gs_flow_solve_noalloc(int64_t nb, int32_t nrcv, const int32_t* rcv, const double* wgt,
                                     const double* b, double* q, void* stream) {
    using namespace gs;
    if (nb < 0 || nb > NA_MAX_NB) {
        set_error(GS_EINVAL, "gs_flow_solve_noalloc: nb must be in 0..GS_NOALLOC_MAX_NB (1048576)");
        return GS_EINVAL;
    }
    if (nrcv < 1 || nrcv > NA_MAX_R) {
        set_error(GS_EINVAL, "gs_flow_solve_noalloc: nrcv must be in 1..GS_NOALLOC_MAX_RCV (4)");
        return GS_EINVAL;
    }
    if (nb == 0) return GS_OK;
    if (!rcv || !wgt || !b || !q) {
        set_error(GS_EINVAL, "gs_flow_solve_noalloc: null argument");
        return GS_EINVAL;
    }
    cudaStream_t s = (cudaStream_t)stream;
    int dev = 0;
    GS_TRY(na_device(s, &dev));
    unsigned char* base = nullptr;
    GS_TRY(na_base(dev, &base));
    const int n = (int)nb, R = nrcv;
    NaLayout L = na_layout(base);
    // the scratch keeps the previous call's contents: clear what must start at zero
    GS_CUDA(cudaMemsetAsync(L.cnt, 0, sizeof(int) * n, s));
    GS_CUDA(cudaMemsetAsync(L.fill, 0, sizeof(int) * n, s));
    GS_CUDA(cudaMemsetAsync(L.queue, 0xff, sizeof(int) * n, s));
    GS_CUDA(cudaMemsetAsync(L.ctr, 0, sizeof(unsigned) * 16, s));
    const int B = 256, G = grid_for(n, B);
    k_na_count<<<G, B, 0, s>>>(n, R, rcv, wgt, L.cnt);
    GS_LAUNCH();
    size_t bytes = NA_CUB_BYTES;
    GS_CUDA(cub::DeviceScan::ExclusiveSum(L.cub, bytes, L.cnt, L.dptr, n + 1, s));
    k_na_fill<<<G, B, 0, s>>>(n, R, rcv, wgt, L.dptr, L.fill, L.dlist);
    k_na_sort<<<G, B, 0, s>>>(n, L.dptr, L.dlist, L.cnt, L.left, L.done, L.ctr);
    GS_LAUNCH();
    NaSched sc{L.queue, L.ctr, L.left, (unsigned)n};
    NaFlowOp op{n, R, L.dptr, L.dlist, rcv, wgt, b, q, L.done};
    k_na_sources<<<G, B, 0, s>>>(op, sc, n);
    int sms = 148;
    GS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    k_na_sweep<<<sms * 4, 128, 0, s>>>(op, sc, n, 4000000000ULL);
    GS_LAUNCH();
    unsigned h[8];
    GS_CUDA(cudaMemcpyAsync(h, L.ctr, sizeof(h), cudaMemcpyDeviceToHost, s));
    GS_CUDA(cudaStreamSynchronize(s));
    if (h[3] != 0) {
        set_error((int)h[3], "gs_flow_solve_noalloc: receiver graph has a cycle or the sweep timed out");
        return (int)h[3];
    }
    if (h[2] + h[4] != (unsigned)n) {
        set_error(GS_ECYCLE, "gs_flow_solve_noalloc: receiver graph has a cycle");
        return GS_ECYCLE;
    }
    return GS_OK;
}
