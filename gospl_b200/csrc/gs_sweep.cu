// Exact solves of the two triangular systems of the hot path by dataflow
// sweeps over the receiver DAG.
//
// Flow accumulation (flowplex.py:429-478 assembles (I - W^T), solved by PETSc
// KSP at flowplex.py:323-427):  q_i = b_i + sum_{donors j} w_{j->i} q_j.
// Stream-power erosion (SPL.py:45-114, solved at SPL.py:297):
//     h_i = (hOld_i + sum_k c_ik h_{rcv_ik}) / (1 + sum_k c_ik).
//
// Both are solved exactly in one pass: each vertex carries a count of its
// unresolved predecessors; vertices whose count reaches zero are appended to
// a ready queue; a persistent grid pulls tickets from the queue, computes the
// vertex from its (already final) predecessors in a fixed order, then
// decrements its successors.  No level schedule, no grid-wide barrier: the
// critical path is the longest flow path.  Pull sums are in a fixed order
// (flow: ascending donor id; SPL: receiver slot order), so results do not
// depend on scheduling.  Waits are bounded: a sweep that stops making progress
// (a cycle) is detected by quiescence (all published vertices processed, queue
// not full) and reported as GS_ECYCLE, a wall-clock budget backs it up.
#include <cooperative_groups.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>

#include "gs_plan.cuh"

namespace cg = cooperative_groups;

namespace gs {

enum { C_HEAD = 0, C_TAIL = 1, C_DONE = 2, C_STATUS = 3, C_NSRC = 4 };

__device__ __forceinline__ unsigned agg_add(unsigned* ctr, unsigned v) {
    cg::coalesced_group g = cg::coalesced_threads();
    unsigned base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(ctr, v * g.size());
    base = g.shfl(base, 0);
    return base + v * g.thread_rank();
}

struct Sched {
    int* queue;
    unsigned* ctr;
    int* cnt;
    unsigned n;
    __device__ __forceinline__ void publish(int r) const {
        unsigned s = agg_add(&ctr[C_TAIL], 1u);
        if (s < n) st_release(&queue[s], r);
    }
    __device__ __forceinline__ void dec(int r) const {
        if (atomicSub(&cnt[r], 1) == 1) publish(r);
    }
};

// ---------------------------------------------------------------------------
// flow accumulation op
// ---------------------------------------------------------------------------
struct FlowOp {
    int n, R;
    const int* nbr;
    const uint32_t* mask;
    const unsigned long long* dk;
    const unsigned long long* sorder;
    const double* wgt;
    const int* rcv;
    const double* b;
    double* x;
    uint8_t* done;
    __device__ __forceinline__ void process(int i, const Sched& sc) const {
        uint32_t m = mask[i];
        unsigned long long kk = dk[i];
        unsigned long long ord = sorder[i];
        double s = b[i];
        for (int q = 0; q < MAXW && m; q++) {
            int t = (int)(ord & 15ULL);
            ord >>= 4;
            if (!(m & (1u << t))) continue;
            m &= ~(1u << t);
            int j = nbr[(size_t)t * n + i];
            int k = (int)((kk >> (4 * t)) & 15ULL);
            s = s + wgt[(size_t)k * n + j] * __ldcg(&x[j]);
        }
        __stcg(&x[i], s);
        done[i] = 1;
        __threadfence();
        for (int k = 0; k < R; k++) {
            int r = rcv[(size_t)k * n + i];
            if (r != i && wgt[(size_t)k * n + i] != 0.0) sc.dec(r);
        }
    }
    // block-sweep form: compute, then hand each ready successor to `emit`
    __device__ __forceinline__ void compute(int i) const {
        uint32_t m = mask[i];
        unsigned long long kk = dk[i];
        unsigned long long ord = sorder[i];
        double s = b[i];
        for (int q = 0; q < MAXW && m; q++) {
            int t = (int)(ord & 15ULL);
            ord >>= 4;
            if (!(m & (1u << t))) continue;
            m &= ~(1u << t);
            int j = nbr[(size_t)t * n + i];
            int k = (int)((kk >> (4 * t)) & 15ULL);
            s = s + wgt[(size_t)k * n + j] * x[j];
        }
        x[i] = s;
        done[i] = 1;
    }
    template <class Emit>
    __device__ __forceinline__ void successors(int i, int* cnt, Emit emit) const {
        for (int k = 0; k < R; k++) {
            int r = rcv[(size_t)k * n + i];
            if (r != i && wgt[(size_t)k * n + i] != 0.0)
                if (atomicSub(&cnt[r], 1) == 1) emit(r);
        }
    }
};

// ---------------------------------------------------------------------------
// SPL op
// ---------------------------------------------------------------------------
struct SplOp {
    int n, R;
    const int* nbr;
    const uint32_t* mask;   // donors with c != 0 (successors)
    const int* rcv;
    const double* c;
    const double* hold;
    double* x;
    uint8_t* done;
    __device__ __forceinline__ void process(int i, const Sched& sc) const {
        double num = hold[i], den = 1.0;
        for (int k = 0; k < R; k++) {
            double ck = c[(size_t)k * n + i];
            int r = rcv[(size_t)k * n + i];
            if (r != i && ck != 0.0) num = num + ck * __ldcg(&x[r]);
            den = den + ck;
        }
        __stcg(&x[i], num / den);
        done[i] = 1;
        __threadfence();
        uint32_t m = mask[i];
        while (m) {
            int t = __ffs(m) - 1;
            m &= m - 1;
            sc.dec(nbr[(size_t)t * n + i]);
        }
    }
    __device__ __forceinline__ void compute(int i) const {
        double num = hold[i], den = 1.0;
        for (int k = 0; k < R; k++) {
            double ck = c[(size_t)k * n + i];
            int r = rcv[(size_t)k * n + i];
            if (r != i && ck != 0.0) num = num + ck * x[r];
            den = den + ck;
        }
        x[i] = num / den;
        done[i] = 1;
    }
    template <class Emit>
    __device__ __forceinline__ void successors(int i, int* cnt, Emit emit) const {
        uint32_t m = mask[i];
        while (m) {
            int t = __ffs(m) - 1;
            m &= m - 1;
            int j = nbr[(size_t)t * n + i];
            if (atomicSub(&cnt[j], 1) == 1) emit(j);
        }
    }
};

// Warp-cooperative dataflow loop.  Each warp takes 32 consecutive tickets,
// polls all pending slots with one ballot per round and processes the lanes
// whose vertices are ready at once; lanes never sleep individually, so a ready
// vertex is never held behind a sibling lane's wait.  A warp refills only when
// all its 32 tickets are done.
template <class Op>
__global__ void k_dataflow(Op op, Sched sc, int n_all, unsigned long long budget_ns) {
    const unsigned long long t0 = globaltimer_ns();
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    const int n = n_all - (int)sc.ctr[C_NSRC];   // vertices that go through the queue
    for (;;) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(&sc.ctr[C_HEAD], 32u);
        base = __shfl_sync(full, base, 0);
        if (base >= (unsigned)n) return;
        const unsigned t = base + lane;
        unsigned pending = __ballot_sync(full, t < (unsigned)n);
        unsigned rounds = 0, nap = 0;
        while (pending) {
            int node = -1;
            if (pending & (1u << lane)) node = ld_relaxed_s32(&sc.queue[t]);
            unsigned ready = __ballot_sync(full, node >= 0) & pending;
            if (ready) {
                __threadfence();   // acquire: predecessors' values are visible
                if (ready & (1u << lane)) op.process(node, sc);
                __syncwarp();
                __threadfence();
                if (lane == 0) atomicAdd(&sc.ctr[C_DONE], (unsigned)__popc(ready));
                pending &= ~ready;
                nap = 0;
                continue;
            }
            // nothing ready: back off, watch for abort, quiescence and time budget
            if ((++rounds & 31u) == 0) {
                int stop = 0;
                if (lane == 0) {
                    if (ld_relaxed_u32(&sc.ctr[C_STATUS]) != 0) stop = 1;
                    unsigned d = 0, tl = 0;
                    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(d) : "l"(&sc.ctr[C_DONE]) : "memory");
                    tl = ld_relaxed_u32(&sc.ctr[C_TAIL]);
                    unsigned first = base + (__ffs(pending) - 1);
                    if (!stop && d == tl && tl <= first) {
                        atomicCAS(&sc.ctr[C_STATUS], 0u, (unsigned)GS_ECYCLE);
                        stop = 1;
                    }
                    if (!stop && globaltimer_ns() - t0 > budget_ns) {
                        atomicCAS(&sc.ctr[C_STATUS], 0u, (unsigned)GS_ETIMEOUT);
                        stop = 1;
                    }
                }
                if (__shfl_sync(full, stop, 0)) return;
            }
            if (nap < 256) nap += 32;
            __nanosleep(nap);
        }
    }
}

// donors of each vertex for the flow system: bit t of mask[r] <=> nbr(r,t) routes
// to r with non-zero weight; dk holds that donor's receiver index (4 bits/slot)
__global__ void k_flow_donors(int n, int R, const int* __restrict__ rcv,
                              const double* __restrict__ wgt, const int8_t* __restrict__ rslot,
                              const int8_t* __restrict__ rev, uint32_t* mask,
                              unsigned long long* dk) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    for (int k = 0; k < R; k++) {
        int r = rcv[(size_t)k * n + j];
        if (r == j || wgt[(size_t)k * n + j] == 0.0) continue;
        int s = rslot[(size_t)k * n + j];
        if (s < 0) continue;
        int t = rev[(size_t)s * n + j];
        if (t < 0) continue;
        atomicOr(&mask[r], 1u << t);
        atomicOr(&dk[r], (unsigned long long)k << (4 * t));
    }
}

__global__ void k_spl_donors(int n, int R, const int* __restrict__ rcv, const double* __restrict__ c,
                             const int8_t* __restrict__ rslot, const int8_t* __restrict__ rev,
                             uint32_t* mask, int* cnt) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    int own = 0;
    for (int k = 0; k < R; k++) {
        int r = rcv[(size_t)k * n + j];
        if (r == j || c[(size_t)k * n + j] == 0.0) continue;
        int s = rslot[(size_t)k * n + j];
        if (s < 0) continue;
        int t = rev[(size_t)s * n + j];
        if (t < 0) continue;
        own++;
        atomicOr(&mask[r], 1u << t);
    }
    cnt[j] = own;
}

// vertices without predecessors are marked (done = 2) and counted; they are
// computed by k_sources in one parallel pass, the rest by k_dataflow
__global__ void k_flow_setup(int n, const uint32_t* __restrict__ mask, int* cnt, Sched sc,
                             uint8_t* done) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = __popc(mask[i]);
    cnt[i] = c;
    done[i] = c == 0 ? 2 : 0;
    if (c == 0) agg_add(&sc.ctr[C_NSRC], 1u);
}

__global__ void k_spl_setup(int n, const int* __restrict__ cnt, Sched sc, uint8_t* done) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    done[i] = cnt[i] == 0 ? 2 : 0;
    if (cnt[i] == 0) agg_add(&sc.ctr[C_NSRC], 1u);
}

template <class Op>
__global__ void k_sources(Op op, Sched sc, int n, const uint8_t* __restrict__ mark) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (mark[i] == 2) op.process(i, sc);
}

// Jacobi iteration for the vertices a flow sweep could not order (cycle
// members and everything downstream of them); ordered vertices are final.
__global__ void k_flow_jacobi(int n, const int* __restrict__ nbr, const uint32_t* __restrict__ mask,
                              const unsigned long long* __restrict__ dk,
                              const unsigned long long* __restrict__ sorder,
                              const double* __restrict__ wgt, const double* __restrict__ b,
                              const uint8_t* __restrict__ done, const double* __restrict__ xin,
                              double* __restrict__ xout, unsigned long long* maxdiff) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (done[i]) { xout[i] = xin[i]; return; }
    uint32_t m = mask[i];
    unsigned long long kk = dk[i], ord = sorder[i];
    double s = b[i];
    for (int q = 0; q < MAXW && m; q++) {
        int t = (int)(ord & 15ULL);
        ord >>= 4;
        if (!(m & (1u << t))) continue;
        m &= ~(1u << t);
        int j = nbr[(size_t)t * n + i];
        int k = (int)((kk >> (4 * t)) & 15ULL);
        s = s + wgt[(size_t)k * n + j] * xin[j];
    }
    xout[i] = s;
    double d = fabs(s - xin[i]) / fmax(fabs(s), 1e-300);
    atomicMax(maxdiff, dkey(d));
}

static int sweep_status(gs_plan* p, int* status_out) {
    unsigned h[8];
    GS_CUDA(cudaMemcpyAsync(h, p->ctr, sizeof(h), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    *status_out = (int)h[C_STATUS];
    if (*status_out == 0 && h[C_DONE] + h[C_NSRC] != (unsigned)p->n) *status_out = GS_ECYCLE;
    return GS_OK;
}


int flow_solve_counted(gs_plan* p, const int* rcv, const double* wgt, const int8_t* rslot,
                       const double* b, double* x, int* cycle_nodes) {
    const int n = (int)p->n;
    *cycle_nodes = 0;
    if (n == 0) return GS_OK;
    GS_CUDA(cudaMemsetAsync(p->don_mask, 0, sizeof(uint32_t) * n, p->stream));
    GS_CUDA(cudaMemsetAsync(p->don_k, 0, sizeof(unsigned long long) * n, p->stream));
    GS_CUDA(cudaMemsetAsync(p->queue, 0xff, sizeof(int) * n, p->stream));
    GS_CUDA(cudaMemsetAsync(p->ctr, 0, sizeof(unsigned) * 8, p->stream));
    launch(p, k_flow_donors, grid_for(n, 256), 256, n, p->R, rcv, wgt, rslot,
           (const int8_t*)p->rev, p->don_mask, p->don_k);
    GS_LAUNCH();
    Sched sc{p->queue, p->ctr, p->cnt, (unsigned)n};
    launch(p, k_flow_setup, grid_for(n, 256), 256, n, (const uint32_t*)p->don_mask, p->cnt, sc,
           p->done_flag);
    GS_LAUNCH();
    FlowOp op{n, p->R, p->nbr, p->don_mask, p->don_k, p->sorder, wgt, rcv, b, x, p->done_flag};
    launch(p, k_sources<FlowOp>, grid_for(n, 256), 256, op, sc, n, (const uint8_t*)p->done_flag);
    launch(p, k_dataflow<FlowOp>, p->sm_count * 4, 128, op, sc, n, p->sweep_budget_ns);
    GS_LAUNCH();
    int st = 0;
    GS_TRY(sweep_status(p, &st));
    if (st == 0) return GS_OK;
    if (st == GS_ETIMEOUT) {
        set_error(GS_ETIMEOUT, "flow sweep exceeded its time budget");
        return GS_ETIMEOUT;
    }
    // Cycle: the unordered vertices are solved by bounded Jacobi iterations.
    double* xa = x;
    double* xb = p->q3;
    unsigned long long* md = p->u_scalar;
    int it = 0, converged = 0;
    const int max_it = 20000;
    for (; it < max_it && !converged; it += 16) {
        for (int r = 0; r < 16; r++) {
            GS_CUDA(cudaMemsetAsync(md, 0, sizeof(unsigned long long), p->stream));
            launch(p, k_flow_jacobi, grid_for(n, 256), 256, n, (const int*)p->nbr,
                   (const uint32_t*)p->don_mask, (const unsigned long long*)p->don_k,
                   (const unsigned long long*)p->sorder, wgt, b, (const uint8_t*)p->done_flag,
                   (const double*)xa, xb, md);
            double* t = xa; xa = xb; xb = t;
        }
        unsigned long long hmd;
        GS_CUDA(cudaMemcpyAsync(&hmd, md, sizeof(hmd), cudaMemcpyDeviceToHost, p->stream));
        GS_CUDA(cudaStreamSynchronize(p->stream));
        double d = 0.0;
        {
            unsigned long long u = (hmd & 0x8000000000000000ULL) ? (hmd & 0x7fffffffffffffffULL) : ~hmd;
            memcpy(&d, &u, sizeof(d));
        }
        if (hmd == 0 || d < 1e-15) converged = 1;
    }
    if (xa != x) GS_CUDA(cudaMemcpyAsync(x, xa, sizeof(double) * n, cudaMemcpyDeviceToDevice, p->stream));
    unsigned h[8];
    GS_CUDA(cudaMemcpyAsync(h, p->ctr, sizeof(h), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    *cycle_nodes = n - (int)h[C_DONE] - (int)h[C_NSRC];
    if (!converged) {
        set_error(GS_EMAXITER, "flow cycle fallback did not converge");
        return GS_EMAXITER;
    }
    return GS_OK;
}

int spl_sweep_counted(gs_plan* p, const int* rcv, const double* c, const int8_t* rslot,
                      const double* hold, double* s, int* cycle_nodes) {
    const int n = (int)p->n;
    *cycle_nodes = 0;
    if (n == 0) return GS_OK;
    GS_CUDA(cudaMemsetAsync(p->don_mask, 0, sizeof(uint32_t) * n, p->stream));
    GS_CUDA(cudaMemsetAsync(p->queue, 0xff, sizeof(int) * n, p->stream));
    GS_CUDA(cudaMemsetAsync(p->ctr, 0, sizeof(unsigned) * 8, p->stream));
    launch(p, k_spl_donors, grid_for(n, 256), 256, n, p->R, rcv, c, rslot, (const int8_t*)p->rev,
           p->don_mask, p->cnt);
    GS_LAUNCH();
    Sched sc{p->queue, p->ctr, p->cnt, (unsigned)n};
    launch(p, k_spl_setup, grid_for(n, 256), 256, n, (const int*)p->cnt, sc, p->done_flag);
    GS_LAUNCH();
    SplOp op{n, p->R, p->nbr, p->don_mask, rcv, c, hold, s, p->done_flag};
    launch(p, k_sources<SplOp>, grid_for(n, 256), 256, op, sc, n, (const uint8_t*)p->done_flag);
    launch(p, k_dataflow<SplOp>, p->sm_count * 4, 128, op, sc, n, p->sweep_budget_ns);
    GS_LAUNCH();
    int st = 0;
    GS_TRY(sweep_status(p, &st));
    if (st != 0) {
        unsigned h[8];
        GS_CUDA(cudaMemcpyAsync(h, p->ctr, sizeof(h), cudaMemcpyDeviceToHost, p->stream));
        GS_CUDA(cudaStreamSynchronize(p->stream));
        *cycle_nodes = n - (int)h[C_DONE] - (int)h[C_NSRC];
        set_error(st, "SPL sweep: receiver graph is not acyclic");
        return st;
    }
    return GS_OK;
}


// ===========================================================================
// Ordered sweeps.  A static topological order (elevation order) is given;
// tickets are handed out in that order and each vertex polls the values of
// its predecessors directly: unsolved values hold a sentinel NaN pattern and
// an aligned 64-bit store is single-copy atomic, so a value that is not the
// sentinel is final.  Per dependency hop the critical path is one store and
// one load through L2, with no atomics or fences.  Lanes of a warp wait
// together (one ballot per polling round) and each ready lane proceeds at
// once.  Predecessors always precede in the order (checked before the sweep),
// so the smallest unfinished ticket is always computable: no deadlock.
// ===========================================================================
constexpr unsigned long long SENT = 0x7ff4dead0badf00dULL;

__device__ __forceinline__ double ld_val(const double* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return __longlong_as_double((long long)v);
}
__device__ __forceinline__ bool is_sent(double v) {
    return (unsigned long long)__double_as_longlong(v) == SENT;
}
__device__ __forceinline__ void st_val(double* p, double v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"((unsigned long long)__double_as_longlong(v)) : "memory");
}

// 32-bit counterparts for the FP32 sweeps of the precision form
constexpr unsigned SENT32 = 0x7fa0dead;
__device__ __forceinline__ float ld_val(const float* p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return __uint_as_float(v);
}
__device__ __forceinline__ bool is_sent(float v) { return __float_as_uint(v) == SENT32; }
__device__ __forceinline__ void st_val(float* p, float v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(__float_as_uint(v)) : "memory");
}

__global__ void k_fill_sent32(int n, float* x) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = __uint_as_float(SENT32);
}

__global__ void k_gather_u64(int n, const unsigned long long* __restrict__ a, const int* __restrict__ idx,
                             unsigned long long* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = a[idx[i]];
}

__global__ void k_reverse(int n, const int* __restrict__ a, int* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = a[n - 1 - i];
}

__global__ void k_fill_sent(int n, double* x) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = __longlong_as_double((long long)SENT);
}

// order keys: descending surface (flow direction), ties by descending flat distance
__global__ void k_order_keys(int n, const double* __restrict__ z, const int* __restrict__ pdir,
                             unsigned long long* key, unsigned* key2, int* val) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    key[i] = ~dkey(z[i]);
    key2[i] = pdir ? ~(unsigned)(pdir[i] + 1) : 0u;
    val[i] = i;
}

__global__ void k_positions(int n, const int* __restrict__ order, int* pos) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) pos[order[p]] = p;
}

// every flow edge j -> r (w != 0, r != j) must have pos[j] < pos[r]
__global__ void k_check_order(int n, int R, const int* __restrict__ rcv, const double* __restrict__ w,
                              const int* __restrict__ pos, int* bad) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    for (int k = 0; k < R; k++) {
        int r = rcv[(size_t)k * n + j];
        if (r != j && w[(size_t)k * n + j] != 0.0 && pos[j] >= pos[r]) { *bad = 1; return; }
    }
}

struct FlowOrd {
    using T = double;
    int n;
    const int* nbr;
    const uint32_t* mask;
    const unsigned long long* dk;
    const unsigned long long* sorder;
    const double* wgt;
    const double* b;
    double* x;
    static constexpr int MAXP = MAXW;
    // gather the predecessors (donors, ascending id) and their weights
    __device__ __forceinline__ int prep(int i, int* pj, double* pw) const {
        uint32_t m = mask[i];
        unsigned long long kk = dk[i], ord = sorder[i];
        int np = 0;
        for (int q = 0; q < MAXW && m; q++) {
            int t = (int)(ord & 15ULL);
            ord >>= 4;
            if (!(m & (1u << t))) continue;
            m &= ~(1u << t);
            int j = nbr[(size_t)t * n + i];
            int k = (int)((kk >> (4 * t)) & 15ULL);
            pj[np] = j;
            pw[np] = wgt[(size_t)k * n + j];
            np++;
        }
        return np;
    }
    __device__ __forceinline__ double init(int i) const { return b[i]; }
    __device__ __forceinline__ double combine(double s, double w, double xj) const { return s + w * xj; }
    __device__ __forceinline__ double aux(int) const { return 0.0; }
    __device__ __forceinline__ double finish(int, double s, double) const { return s; }
};

struct SplOrd {
    using T = double;
    int n, R;
    const int* rcv;
    const double* c;
    const double* hold;
    double* x;
    static constexpr int MAXP = MAXR;
    __device__ __forceinline__ int prep(int i, int* pj, double* pw) const {
        int np = 0;
        for (int k = 0; k < R; k++) {
            double ck = c[(size_t)k * n + i];
            int r = rcv[(size_t)k * n + i];
            if (r != i && ck != 0.0) { pj[np] = r; pw[np] = ck; np++; }
        }
        return np;
    }
    __device__ __forceinline__ double init(int i) const { return hold[i]; }
    __device__ __forceinline__ double combine(double s, double w, double xj) const { return s + w * xj; }
    // the denominator, formed when the vertex is ticketed (off the hop)
    __device__ __forceinline__ double aux(int i) const {
        double den = 1.0;
        for (int k = 0; k < R; k++) den = den + c[(size_t)k * n + i];
        return den;
    }
    __device__ __forceinline__ double finish(int, double num, double den) const { return num / den; }
};

// Transposed flow system (I - W) y = g: y_i = g_i + sum_k w_ik y_{rcv_ik},
// receivers first (the flow order reversed).
struct FlowAdjOrd {
    using T = double;
    int n, R;
    const int* rcv;
    const double* wgt;
    const double* g;
    double* x;
    static constexpr int MAXP = MAXR;
    __device__ __forceinline__ int prep(int i, int* pj, double* pw) const {
        int np = 0;
        for (int k = 0; k < R; k++) {
            double w = wgt[(size_t)k * n + i];
            int r = rcv[(size_t)k * n + i];
            if (r != i && w != 0.0) { pj[np] = r; pw[np] = w; np++; }
        }
        return np;
    }
    __device__ __forceinline__ double init(int i) const { return g[i]; }
    __device__ __forceinline__ double combine(double s, double w, double xj) const { return s + w * xj; }
    __device__ __forceinline__ double aux(int) const { return 0.0; }
    __device__ __forceinline__ double finish(int, double s, double) const { return s; }
};

// Transposed SPL system M^T y = g: y_j = (g_j + sum_{donors i} c_ik y_i) / den_j,
// den_j = 1 + sum_k c_jk, donors first (the flow order).
struct SplAdjOrd {
    using T = double;
    int n, R;
    const int* nbr;
    const uint32_t* mask;
    const unsigned long long* dk;
    const unsigned long long* sorder;
    const double* c;
    const double* g;
    double* x;
    static constexpr int MAXP = MAXW;
    __device__ __forceinline__ int prep(int i, int* pj, double* pw) const {
        uint32_t m = mask[i];
        unsigned long long kk = dk[i], ord = sorder[i];
        int np = 0;
        for (int q = 0; q < MAXW && m; q++) {
            int t = (int)(ord & 15ULL);
            ord >>= 4;
            if (!(m & (1u << t))) continue;
            m &= ~(1u << t);
            int j = nbr[(size_t)t * n + i];
            int k = (int)((kk >> (4 * t)) & 15ULL);
            double cj = c[(size_t)k * n + j];
            if (cj == 0.0) continue;
            pj[np] = j;
            pw[np] = cj;
            np++;
        }
        return np;
    }
    __device__ __forceinline__ double init(int i) const { return g[i]; }
    __device__ __forceinline__ double combine(double s, double w, double xj) const { return s + w * xj; }
    __device__ __forceinline__ double aux(int i) const {
        double den = 1.0;
        for (int k = 0; k < R; k++) den = den + c[(size_t)k * n + i];
        return den;
    }
    __device__ __forceinline__ double finish(int, double s, double den) const { return s / den; }
};

// ---- FP32 operators of the precision form: values and arithmetic in FP32,
// weights, coefficients and right-hand sides read from their FP64 arrays and
// rounded on load.  They solve for corrections of an FP64 refinement loop.
struct FlowOrd32 {
    using T = float;
    int n;
    const int* nbr;
    const uint32_t* mask;
    const unsigned long long* dk;
    const unsigned long long* sorder;
    const double* wgt;
    const double* b;
    float* x;
    static constexpr int MAXP = MAXW;
    __device__ __forceinline__ int prep(int i, int* pj, float* pw) const {
        uint32_t m = mask[i];
        unsigned long long kk = dk[i], ord = sorder[i];
        int np = 0;
        for (int q = 0; q < MAXW && m; q++) {
            int t = (int)(ord & 15ULL);
            ord >>= 4;
            if (!(m & (1u << t))) continue;
            m &= ~(1u << t);
            int j = nbr[(size_t)t * n + i];
            int k = (int)((kk >> (4 * t)) & 15ULL);
            pj[np] = j;
            pw[np] = (float)wgt[(size_t)k * n + j];
            np++;
        }
        return np;
    }
    __device__ __forceinline__ float init(int i) const { return (float)b[i]; }
    __device__ __forceinline__ float combine(float s, float w, float xj) const { return s + w * xj; }
    __device__ __forceinline__ double aux(int) const { return 0.0; }
    __device__ __forceinline__ float finish(int, float s, double) const { return s; }
};

struct SplOrd32 {
    using T = float;
    int n, R;
    const int* rcv;
    const double* c;
    const double* hold;
    float* x;
    static constexpr int MAXP = MAXR;
    __device__ __forceinline__ int prep(int i, int* pj, float* pw) const {
        int np = 0;
        for (int k = 0; k < R; k++) {
            double ck = c[(size_t)k * n + i];
            int r = rcv[(size_t)k * n + i];
            if (r != i && ck != 0.0) { pj[np] = r; pw[np] = (float)ck; np++; }
        }
        return np;
    }
    __device__ __forceinline__ float init(int i) const { return (float)hold[i]; }
    __device__ __forceinline__ float combine(float s, float w, float xj) const { return s + w * xj; }
    __device__ __forceinline__ double aux(int i) const {
        float den = 1.0f;
        for (int k = 0; k < R; k++) den = den + (float)c[(size_t)k * n + i];
        return (double)den;    // exact: a float widened
    }
    __device__ __forceinline__ float finish(int, float num, double den) const { return num / (float)den; }
};

// predecessors q0..np-1 of a vertex of high degree, read together; false
// while any is unpublished (kept out of line: rare, and its registers would
// crowd the polling loop)
template <class Op>
__device__ __noinline__ bool ordered_tail(const Op& op, const int* pj, const typename Op::T* pw, int q0, int np,
                                          typename Op::T* acc) {
    using T = typename Op::T;
    T v[Op::MAXP];
    for (int q = q0; q < np; q++) v[q - q0] = ld_val(&op.x[pj[q]]);
    for (int q = q0; q < np; q++)
        if (is_sent(v[q - q0])) return false;
    T a = *acc;
    for (int q = q0; q < np; q++) a = op.combine(a, pw[q], v[q - q0]);
    *acc = a;
    return true;
}

// status of an ordered sweep whose order failed its check (skip flag set):
// no vertex computed, the caller runs the counter-based sweep instead
constexpr unsigned ORDER_REJECTED = 0x100u;

template <class Op>
__global__ void __launch_bounds__(128, 8) k_ordered(Op op, int n, const int* __restrict__ order, unsigned* ctr,
                                                 unsigned long long budget_ns, unsigned nap_max,
                                                 const int* __restrict__ skip) {
    if (skip && *skip) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(&ctr[C_STATUS], 0u, ORDER_REJECTED);
        return;
    }
    const unsigned long long t0 = globaltimer_ns();
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    using T = typename Op::T;
    int pj[Op::MAXP];
    T pw[Op::MAXP];
    for (;;) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(&ctr[C_HEAD], 32u);
        base = __shfl_sync(full, base, 0);
        if (base >= (unsigned)n) return;
        const unsigned t = base + lane;
        int node = -1, np = 0;
        T init = T(0);
        double aux = 0.0;
        if (t < (unsigned)n) {
            node = order[t];
            np = op.prep(node, pj, pw);
            init = op.init(node);
            aux = op.aux(node);
        }
        unsigned pending = __ballot_sync(full, node >= 0);
        unsigned rounds = 0, nap = 0;
        // The first PB predecessors of a lane are read until each is seen
        // published and then kept in registers: a polling round loads only
        // the predecessors still missing (mostly one), not all of them again.
        // Re-reading every predecessor each round floods the SM's load path
        // with requests that answer nothing new and stretches every round
        // well past one L2 latency.  Predecessors beyond the first PB (rare:
        // degree > 8) are read together each round.  The sum keeps the
        // predecessors' order.
        constexpr int PB = Op::MAXP < 6 ? Op::MAXP : 6;
        unsigned seen = 0u;
        T vals[PB];
        const unsigned need = np >= PB ? ((1u << PB) - 1u) : ((1u << np) - 1u);
        while (pending) {
            bool rdy = false;
            if (pending & (1u << lane)) {
#pragma unroll
                for (int u = 0; u < PB; u++)
                    if (u < np && !((seen >> u) & 1u)) vals[u] = ld_val(&op.x[pj[u]]);
#pragma unroll
                for (int u = 0; u < PB; u++)
                    if (u < np && !((seen >> u) & 1u) && !is_sent(vals[u])) seen |= 1u << u;
                rdy = (seen & need) == need;
                if (rdy) {
                    T acc = init;
#pragma unroll
                    for (int u = 0; u < PB; u++)
                        if (u < np) acc = op.combine(acc, pw[u], vals[u]);
                    if (np > PB) rdy = ordered_tail(op, pj, pw, PB, np, &acc);
                    if (rdy) st_val(&op.x[node], op.finish(node, acc, aux));
                }
            }
            unsigned done = __ballot_sync(full, rdy);
            pending &= ~done;
            if (done) { nap = 0; continue; }
            if ((++rounds & 63u) == 0) {
                int stop = 0;
                if (lane == 0) {
                    if (ld_relaxed_u32(&ctr[C_STATUS]) != 0) stop = 1;
                    else if (globaltimer_ns() - t0 > budget_ns) {
                        atomicCAS(&ctr[C_STATUS], 0u, (unsigned)GS_ETIMEOUT);
                        stop = 1;
                    }
                }
                if (__shfl_sync(full, stop, 0)) return;
            }
            if (nap < nap_max) nap += 16;
            if (nap) __nanosleep(nap);
        }
    }
}

// ---- marine flow accumulation (the coupled marine system, Gmar > 0) ----
// q_i = b_i + sum over donors j of w_j q_j, a donor being a neighbour whose
// receiver bit set (cand, over its neighbour slots) holds the slot of i; the
// weight is the donor's 1/kk.  Donors in ascending id.
struct MarineOrd {
    using T = double;
    int n;
    const int* nbr;
    const int8_t* nnb;
    const int8_t* rev;
    const unsigned long long* sorder;
    const unsigned short* cand;
    const double* w;
    const double* b;
    double* x;
    static constexpr int MAXP = MAXW;
    __device__ __forceinline__ int prep(int i, int* pj, double* pw) const {
        const unsigned long long so = sorder[i];
        int np = 0;
        for (int q = 0; q < nnb[i]; q++) {
            const int sl = (int)((so >> (4 * q)) & 15ULL);
            const int j = nbr[(size_t)sl * n + i];
            if (j < 0) continue;
            const int r = rev[(size_t)sl * n + i];
            if (r >= 0 && ((cand[j] >> r) & 1u)) {
                pj[np] = j;
                pw[np] = w[j];
                np++;
            }
        }
        return np;
    }
    __device__ __forceinline__ double init(int i) const { return b[i]; }
    __device__ __forceinline__ double combine(double s, double wj, double xj) const { return s + wj * xj; }
    __device__ __forceinline__ double aux(int) const { return 0.0; }
    __device__ __forceinline__ double finish(int, double s, double) const { return s; }
};

// every marine receiver edge j -> i must go forward in the order
__global__ void k_check_marine_order(int n, const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                                     const unsigned short* __restrict__ cand, const int* __restrict__ pos,
                                     int* bad) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const unsigned m = cand[j];
    for (int s = 0; s < nnb[j]; s++) {
        if (!((m >> s) & 1u)) continue;
        const int i = nbr[(size_t)s * n + j];
        if (i >= 0 && pos[j] >= pos[i]) { *bad = 1; return; }
    }
}

// sort vertices by (surface desc, flat distance desc); returns 1 when the
// order is topological for the given flow edges
// Tie groups of the surface-sorted order: run start of every position (max-
// scanned afterwards) and the membership flag of runs longer than one.
__global__ void k_tie_runs(int n, const unsigned long long* __restrict__ skey, int* run, int* flag) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const unsigned long long k = skey[t];
    const bool first = t == 0 || skey[t - 1] != k;
    const bool last = t == n - 1 || skey[t + 1] != k;
    run[t] = first ? t : 0;
    flag[t] = (first && last) ? 0 : 1;
}

// tie members as (run start, descending flat distance) keys, in position
// order: the low pb bits hold (2^pb - 1) - (pdir + 1), pdir + 1 < 2^pb
template <class K>
__global__ void k_tie_compact(int n, const int* __restrict__ run, const int* __restrict__ flag,
                              const int* __restrict__ scan, const int* __restrict__ order,
                              const int* __restrict__ pdir, int pb, K* ckey, int* cval, int* cpos) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n || !flag[t]) return;
    const int j = scan[t];
    const int v = order[t];
    const unsigned long long lo = ((1ULL << pb) - 1ULL) - (unsigned long long)(unsigned)(pdir[v] + 1);
    ckey[j] = (K)((((unsigned long long)(unsigned)run[t]) << pb) | lo);
    cval[j] = v;
    cpos[j] = t;
}

__global__ void k_tie_scatter(int m, const int* __restrict__ cpos, const int* __restrict__ cval, int* order) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < m) order[cpos[j]] = cval[j];
}

struct MaxOp {
    __device__ __forceinline__ int operator()(int a, int b) const { return a > b ? a : b; }
};

// Vertices by surface descending (ties by vertex id): keys and one stable
// 64-bit radix sort.  The sorted keys stay in okey2 for order_ties.
static int order_by_surface(gs_plan* p, const double* z, int* order) {
    const int n = (int)p->n;
    const int B = 256, G = grid_for(n, B);
    launch(p, k_order_keys, G, B, n, z, (const int*)nullptr, p->okey, p->ok32, p->oval);
    GS_LAUNCH();
    size_t bytes = p->cub_bytes;
    GS_CUDA(cub::DeviceRadixSort::SortPairs(p->cub_tmp, bytes, p->okey, p->okey2, p->oval, order, n, 0, 64,
                                            p->stream));
    p->launches++;
    return GS_OK;
}

static int order_ties_prepare(gs_plan* p) {
    const int n = (int)p->n;
    const int B = 256, G = grid_for(n, B);
    int* run0 = p->oval;
    int* run = (int*)p->ok32b;
    int* flag = p->oval2;
    int* scan = (int*)p->ok32;
    launch(p, k_tie_runs, G, B, n, (const unsigned long long*)p->okey2, run0, flag);
    GS_LAUNCH();
    size_t bytes = p->cub_bytes;
    GS_CUDA(cub::DeviceScan::InclusiveScan(p->cub_tmp, bytes, run0, run, MaxOp(), n, p->stream));
    p->launches++;
    bytes = p->cub_bytes;
    GS_CUDA(cub::DeviceScan::ExclusiveSum(p->cub_tmp, bytes, flag, scan, n, p->stream));
    p->launches++;
    int last[2];
    GS_CUDA(cudaMemcpyAsync(&last[0], scan + n - 1, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaMemcpyAsync(&last[1], flag + n - 1, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    p->tie_m = last[0] + last[1];
    return GS_OK;
}

static int order_ties_finish(gs_plan* p, const int* pdir, int* order) {
    const int n = (int)p->n;
    const int B = 256, G = grid_for(n, B);
    const int m = p->tie_m;
    if (m == 0) return GS_OK;
    const int* run = (const int*)p->ok32b;
    const int* flag = p->oval2;
    const int* scan = (const int*)p->ok32;
    int* cval = p->oval;
    int* cval2 = (int*)p->ok32b;   // run is consumed by the compaction before the sort writes here
    int* cpos = p->pos;            // rewritten by the positions pass that follows
    int hb = 1;
    while ((1LL << hb) <= (long long)n && hb < 31) hb++;
    // the flat distances of the plan's last fill are bounded by its BFS depth:
    // then the keys need only hb + pb bits, mostly 32 or fewer (half the key
    // bytes and about half the radix passes of the general 64-bit layout)
    int pb = 32;
    if (pdir == p->pdir && p->pdir_bound > 0) {
        pb = 1;
        while ((1LL << pb) <= (long long)p->pdir_bound + 1 && pb < 32) pb++;
    }
    size_t need32 = 0;
    if (hb + pb <= 32)
        GS_CUDA(cub::DeviceRadixSort::SortPairs((void*)nullptr, need32, (const unsigned*)nullptr, (unsigned*)nullptr,
                                                (const int*)nullptr, (int*)nullptr, m, 0, hb + pb, p->stream));
    if (hb + pb <= 32 && need32 <= p->cub_bytes) {
        unsigned* k32 = reinterpret_cast<unsigned*>(p->okey);
        unsigned* k32b = reinterpret_cast<unsigned*>(p->okey2);
        launch(p, k_tie_compact<unsigned>, G, B, n, run, flag, scan, (const int*)order, pdir, pb, k32, cval, cpos);
        GS_LAUNCH();
        size_t bytes = p->cub_bytes;
        GS_CUDA(cub::DeviceRadixSort::SortPairs(p->cub_tmp, bytes, (const unsigned*)k32, k32b, (const int*)cval,
                                                cval2, m, 0, hb + pb, p->stream));
    } else {
        pb = 32;
        launch(p, k_tie_compact<unsigned long long>, G, B, n, run, flag, scan, (const int*)order, pdir, pb, p->okey,
               cval, cpos);
        GS_LAUNCH();
        size_t bytes = p->cub_bytes;
        GS_CUDA(cub::DeviceRadixSort::SortPairs(p->cub_tmp, bytes, p->okey, p->okey2, cval, cval2, m, 0, 32 + hb,
                                                p->stream));
    }
    p->launches++;
    launch(p, k_tie_scatter, grid_for(m, B), B, m, (const int*)cpos, (const int*)cval2, order);
    GS_LAUNCH();
    return GS_OK;
}

// Breaks the surface ties of order_by_surface by flat distance descending
// (ties of both by vertex id): only the members of tie groups are re-sorted,
// by (group start, ~(pdir + 1)), and written back to their positions.  Gives
// the order of a stable sort by (surface desc, pdir desc).  The tie groups
// depend on the surface only (order_ties_prepare, which reads their count back
// to the host); the flat distances are needed only by order_ties_finish.
static int order_ties(gs_plan* p, const int* pdir, int* order) {
    GS_TRY(order_ties_prepare(p));
    return order_ties_finish(p, pdir, order);
}

// Checks that every weighted edge goes forward in `order`; the result
// (nonzero = not a topological order) is copied to the pinned host word
// bad_host without synchronising.
static int order_check_async(gs_plan* p, const int* rcv, const double* w, const int* order, int* bad_host) {
    const int n = (int)p->n;
    const int B = 256, G = grid_for(n, B);
    launch(p, k_positions, G, B, n, order, p->pos);
    GS_CUDA(cudaMemsetAsync(p->i_scalar + 14, 0, sizeof(int), p->stream));
    launch(p, k_check_order, G, B, n, p->R, rcv, w, (const int*)p->pos, p->i_scalar + 14);
    GS_LAUNCH();
    GS_CUDA(cudaMemcpyAsync(bad_host, p->i_scalar + 14, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    return GS_OK;
}

// ---- order of a surface that differs from an already ordered one in few
// places (the cascade's water surface against h): the unchanged vertices keep
// their relative order from the base order, the changed ones are sorted
// alone, and the two sorted runs are merged by (key, vertex id) ranks.
__global__ void k_changed(int n, const double* __restrict__ z, const double* __restrict__ zb, int* flag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = dkey(z[i]) != dkey(zb[i]) ? 1 : 0;
}

__global__ void k_changed_compact(int n, const int* __restrict__ flag, const int* __restrict__ scan,
                                  const double* __restrict__ z, unsigned long long* ckey, int* cid) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !flag[i]) return;
    ckey[scan[i]] = ~dkey(z[i]);
    cid[scan[i]] = i;
}

__global__ void k_kept_flag(int n, const int* __restrict__ base, const int* __restrict__ flag, int* kf) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) kf[t] = flag[base[t]] ? 0 : 1;
}

__global__ void k_kept_compact(int n, const int* __restrict__ base, const int* __restrict__ kf,
                               const int* __restrict__ scan, const double* __restrict__ z, unsigned long long* akey,
                               int* aid) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n || !kf[t]) return;
    const int v = base[t];
    akey[scan[t]] = ~dkey(z[v]);
    aid[scan[t]] = v;
}

// number of entries of the sorted run (k, id) that come before (key, vid)
__device__ __forceinline__ int rank_in(const unsigned long long* __restrict__ k, const int* __restrict__ id, int len,
                                       unsigned long long key, int vid) {
    int lo = 0, hi = len;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (k[mid] < key || (k[mid] == key && id[mid] < vid)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__global__ void k_merge_runs(int na, const unsigned long long* __restrict__ akey, const int* __restrict__ aid,
                             int nc, const unsigned long long* __restrict__ ckey, const int* __restrict__ cid,
                             int* order, unsigned long long* okey) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < na) {
        const int o = t + rank_in(ckey, cid, nc, akey[t], aid[t]);
        order[o] = aid[t];
        okey[o] = akey[t];
    } else if (t < na + nc) {
        const int c = t - na;
        const int o = c + rank_in(akey, aid, na, ckey[c], cid[c]);
        order[o] = cid[c];
        okey[o] = ckey[c];
    }
}

// The order of `surface` (descending, ties by vertex id), given the order
// `base` of `zb` built by order_by_surface; sorted keys left in okey2 as
// order_by_surface leaves them.
static int order_by_surface_from(gs_plan* p, const double* z, const double* zb, const int* base, int* order) {
    const int n = (int)p->n;
    const int B = 256, G = grid_for(n, B);
    int* flag = p->pos;
    int* cscan = (int*)p->ok32;
    launch(p, k_changed, G, B, n, z, zb, flag);
    GS_LAUNCH();
    size_t bytes = p->cub_bytes;
    GS_CUDA(cub::DeviceScan::ExclusiveSum(p->cub_tmp, bytes, (const int*)flag, cscan, n, p->stream));
    p->launches++;
    int last[2];
    GS_CUDA(cudaMemcpyAsync(&last[0], cscan + n - 1, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaMemcpyAsync(&last[1], flag + n - 1, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    // kept vertices, in the base order
    int* kf = (int*)p->ok32b;
    int* kscan = p->cnt;
    launch(p, k_kept_flag, G, B, n, base, (const int*)flag, kf);
    GS_LAUNCH();
    bytes = p->cub_bytes;
    GS_CUDA(cub::DeviceScan::ExclusiveSum(p->cub_tmp, bytes, (const int*)kf, kscan, n, p->stream));
    p->launches++;
    launch(p, k_kept_compact, G, B, n, base, (const int*)kf, (const int*)kscan, zb, p->don_k, p->queue);
    launch(p, k_changed_compact, G, B, n, (const int*)flag, (const int*)cscan, z, p->okey, p->oval);
    GS_LAUNCH();
    GS_CUDA(cudaStreamSynchronize(p->stream));
    const int nc = last[0] + last[1], na = n - nc;
    if (nc > 0) {
        int hb = 64;
        bytes = p->cub_bytes;
        GS_CUDA(cub::DeviceRadixSort::SortPairs(p->cub_tmp, bytes, p->okey, p->basinL, p->oval, p->oval2, nc, 0, hb,
                                                p->stream));
        p->launches++;
    }
    launch(p, k_merge_runs, grid_for(n, B), B, na, (const unsigned long long*)p->don_k, (const int*)p->queue, nc,
           (const unsigned long long*)p->basinL, (const int*)p->oval2, order, p->okey2);
    GS_LAUNCH();
    return GS_OK;
}

int flow_order(gs_plan* p, const double* surface, int* order) { return order_by_surface(p, surface, order); }

int flow_order_from(gs_plan* p, const double* surface, const double* base_surface, const int* base_order,
                    int* order) {
    return order_by_surface_from(p, surface, base_surface, base_order, order);
}

int flow_order_ties_prepare(gs_plan* p) { return order_ties_prepare(p); }

int flow_order_ties(gs_plan* p, const int* pdir, int* order) { return order_ties_finish(p, pdir, order); }

static int ordered_status(gs_plan* p, int* st) {
    unsigned h[8];
    GS_CUDA(cudaMemcpyAsync(h, p->ctr, sizeof(h), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    *st = (int)h[C_STATUS];
    return GS_OK;
}

// Everything of an ordered flow sweep that does not need b, for an order
// built by flow_order (+ flow_order_ties): its check (result in *bad_host once
// the stream reaches it), the donor masks and the sentinel-filled output.
int flow_prepare(gs_plan* p, const int* rcv, const double* wgt, const int8_t* rslot, double* x, const int* order,
                 int* bad_host) {
    const int n = (int)p->n;
    if (n == 0) return GS_OK;
    GS_TRY(order_check_async(p, rcv, wgt, order, bad_host));
    GS_CUDA(cudaMemsetAsync(p->don_mask, 0, sizeof(uint32_t) * n, p->stream));
    GS_CUDA(cudaMemsetAsync(p->don_k, 0, sizeof(unsigned long long) * n, p->stream));
    launch(p, k_flow_donors, grid_for(n, 256), 256, n, p->R, rcv, wgt, rslot, (const int8_t*)p->rev, p->don_mask,
           p->don_k);
    launch(p, k_fill_sent, grid_for(n, 256), 256, n, x);
    GS_LAUNCH();
    return GS_OK;
}

// The sweep proper, after flow_prepare: the ordered kernel when the order is
// valid (ok), else the counter-based dataflow solve.
int flow_run(gs_plan* p, const int* rcv, const double* wgt, const int8_t* rslot, const double* b, double* x,
             int* cycle_nodes, int* order, int ok, int* status_host) {
    const int n = (int)p->n;
    *cycle_nodes = 0;
    if (status_host) *status_host = 0;
    if (n == 0) return GS_OK;
    if (!ok) return flow_solve_counted(p, rcv, wgt, rslot, b, x, cycle_nodes);
    if (p->fp32) return flow_refine32(p, wgt, b, x, order);
    GS_CUDA(cudaMemsetAsync(p->ctr, 0, sizeof(unsigned) * 8, p->stream));
    FlowOrd op{n, p->nbr, p->don_mask, p->don_k, p->sorder, wgt, b, x};
    launch(p, k_ordered<FlowOrd>, p->sm_count * p->sweep_per_sm, 128, op, n, (const int*)order, p->ctr, p->sweep_budget_ns, p->sweep_nap, (const int*)nullptr);
    GS_LAUNCH();
    if (status_host) {
        // the caller reads the status at its next synchronisation
        GS_CUDA(cudaMemcpyAsync(status_host, p->ctr + C_STATUS, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
        return GS_OK;
    }
    int st = 0;
    GS_TRY(ordered_status(p, &st));
    if (st != 0) {
        set_error(st, "ordered flow sweep did not complete");
        return st;
    }
    return GS_OK;
}

int flow_solve(gs_plan* p, const int* rcv, const double* wgt, const int8_t* rslot, const double* b, double* x,
               int* cycle_nodes, const double* surface, const int* pdir, int* order) {
    const int n = (int)p->n;
    *cycle_nodes = 0;
    if (n == 0) return GS_OK;
    int ok = 0;
    if (surface) {
        GS_TRY(order_by_surface(p, surface, order));
        if (pdir) GS_TRY(order_ties(p, pdir, order));
        GS_TRY(flow_prepare(p, rcv, wgt, rslot, x, order, p->h_pinned));
        GS_CUDA(cudaStreamSynchronize(p->stream));
        ok = p->h_pinned[0] ? 0 : 1;
    }
    if (order == p->order_i) p->order_i_valid = ok;
    return flow_run(p, rcv, wgt, rslot, b, x, cycle_nodes, order, ok, nullptr);
}

// SPL edges i -> rcv (c != 0) run against the flow order: need pos[rcv] > pos[i]
__global__ void k_check_spl_order(int n, int R, const int* __restrict__ rcv, const double* __restrict__ c,
                                  const int* __restrict__ pos, int* bad) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = 0; k < R; k++) {
        int r = rcv[(size_t)k * n + i];
        if (r != i && c[(size_t)k * n + i] != 0.0 && pos[r] <= pos[i]) { *bad = 1; return; }
    }
}

int spl_sweep(gs_plan* p, const int* rcv, const double* c, const int8_t* rslot, const double* hold, double* s,
              int* cycle_nodes, bool reuse_order) {
    const int n = (int)p->n;
    *cycle_nodes = 0;
    if (n == 0) return GS_OK;
    const int ok = reuse_order && p->order_i_valid;
    if (!ok) return spl_sweep_counted(p, rcv, c, rslot, hold, s, cycle_nodes);
    // the check of the order against the SPL edges is read by the sweep
    // itself (no host round trip): a rejected order stops it at once and the
    // counter-based sweep runs instead
    launch(p, k_positions, grid_for(n, 256), 256, n, (const int*)p->order_i, p->pos);
    GS_CUDA(cudaMemsetAsync(p->i_scalar + 14, 0, sizeof(int), p->stream));
    launch(p, k_check_spl_order, grid_for(n, 256), 256, n, p->R, rcv, c, (const int*)p->pos, p->i_scalar + 14);
    GS_LAUNCH();
    // the SPL system is solved receivers first: the flow order reversed
    launch(p, k_reverse, grid_for(n, 256), 256, n, (const int*)p->order_i, p->order2);
    if (p->fp32) {
        // the refinement runs several sweeps: read the check first
        int bad = 0;
        GS_CUDA(cudaMemcpyAsync(&bad, p->i_scalar + 14, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
        GS_CUDA(cudaStreamSynchronize(p->stream));
        if (bad) return spl_sweep_counted(p, rcv, c, rslot, hold, s, cycle_nodes);
        return spl_refine32(p, rcv, c, hold, s, p->order2);
    }
    GS_CUDA(cudaMemsetAsync(p->ctr, 0, sizeof(unsigned) * 8, p->stream));
    launch(p, k_fill_sent, grid_for(n, 256), 256, n, s);
    SplOrd op{n, p->R, rcv, c, hold, s};
    launch(p, k_ordered<SplOrd>, p->sm_count * p->sweep_per_sm, 128, op, n, (const int*)p->order2, p->ctr,
           p->sweep_budget_ns, p->sweep_nap, (const int*)(p->i_scalar + 14));
    GS_LAUNCH();
    int st = 0;
    GS_TRY(ordered_status(p, &st));
    if ((unsigned)st == ORDER_REJECTED) return spl_sweep_counted(p, rcv, c, rslot, hold, s, cycle_nodes);
    if (st != 0) {
        set_error(st, "ordered SPL sweep did not complete");
        return st;
    }
    return GS_OK;
}

int sweep_marine(gs_plan* p, const unsigned short* cand, const double* w, const int* order, const double* b,
                 double* q) {
    const int n = (int)p->n;
    if (n == 0) return GS_OK;
    launch(p, k_positions, grid_for(n, 256), 256, n, order, p->pos);
    GS_CUDA(cudaMemsetAsync(p->i_scalar + 14, 0, sizeof(int), p->stream));
    launch(p, k_check_marine_order, grid_for(n, 256), 256, n, (const int*)p->nbr, (const int8_t*)p->nnb, cand,
           (const int*)p->pos, p->i_scalar + 14);
    GS_CUDA(cudaMemsetAsync(p->ctr, 0, sizeof(unsigned) * 8, p->stream));
    launch(p, k_fill_sent, grid_for(n, 256), 256, n, q);
    MarineOrd op{n, p->nbr, p->nnb, p->rev, p->sorder, cand, w, b, q};
    // a rejected order (a marine receiver not below its donor) stops the
    // sweep at once: the receivers are strictly lower, so it cannot happen
    launch(p, k_ordered<MarineOrd>, p->sm_count * p->sweep_per_sm, 128, op, n, order, p->ctr, p->sweep_budget_ns,
           p->sweep_nap, (const int*)(p->i_scalar + 14));
    GS_LAUNCH();
    int st = 0;
    GS_TRY(ordered_status(p, &st));
    if ((unsigned)st == ORDER_REJECTED) {
        set_error(GS_EINVAL, "marine sweep: the marine receivers are not below their donors in the surface order");
        return GS_EINVAL;
    }
    if (st != 0) {
        set_error(st, "marine sweep did not complete");
        return st;
    }
    return GS_OK;
}

// y = (I - W)^-1 g over the graph rcv/wgt whose valid flow order is `order`
int sweep_flow_adjoint(gs_plan* p, const int* rcv, const double* wgt, const int* order, const double* g, double* y) {
    const int n = (int)p->n;
    if (n == 0) return GS_OK;
    launch(p, k_reverse, grid_for(n, 256), 256, n, order, p->order2);
    GS_CUDA(cudaMemsetAsync(p->ctr, 0, sizeof(unsigned) * 8, p->stream));
    launch(p, k_fill_sent, grid_for(n, 256), 256, n, y);
    FlowAdjOrd op{n, p->R, rcv, wgt, g, y};
    launch(p, k_ordered<FlowAdjOrd>, p->sm_count * p->sweep_per_sm, 128, op, n, (const int*)p->order2, p->ctr, p->sweep_budget_ns, p->sweep_nap, (const int*)nullptr);
    GS_LAUNCH();
    int st = 0;
    GS_TRY(ordered_status(p, &st));
    if (st != 0) {
        set_error(st, "adjoint flow sweep did not complete");
        return st;
    }
    return GS_OK;
}

// y = M^-T g for the SPL matrix of coefficients c on the graph rcv/wgt/rslot
// (flow order `order`)
int sweep_spl_adjoint(gs_plan* p, const int* rcv, const double* wgt, const int8_t* rslot, const double* c,
                      const int* order, const double* g, double* y) {
    const int n = (int)p->n;
    if (n == 0) return GS_OK;
    GS_CUDA(cudaMemsetAsync(p->don_mask, 0, sizeof(uint32_t) * n, p->stream));
    GS_CUDA(cudaMemsetAsync(p->don_k, 0, sizeof(unsigned long long) * n, p->stream));
    launch(p, k_flow_donors, grid_for(n, 256), 256, n, p->R, rcv, wgt, rslot, (const int8_t*)p->rev, p->don_mask,
           p->don_k);
    GS_CUDA(cudaMemsetAsync(p->ctr, 0, sizeof(unsigned) * 8, p->stream));
    launch(p, k_fill_sent, grid_for(n, 256), 256, n, y);
    SplAdjOrd op{n, p->R, p->nbr, p->don_mask, p->don_k, p->sorder, c, g, y};
    launch(p, k_ordered<SplAdjOrd>, p->sm_count * p->sweep_per_sm, 128, op, n, order, p->ctr, p->sweep_budget_ns, p->sweep_nap, (const int*)nullptr);
    GS_LAUNCH();
    int st = 0;
    GS_TRY(ordered_status(p, &st));
    if (st != 0) {
        set_error(st, "adjoint SPL sweep did not complete");
        return st;
    }
    return GS_OK;
}

// ---------------------------------------------------------------------------
// Precision form: FP32 sweeps inside an FP64 refinement loop.  x_0 = 0, then
// repeat: d = T^-1 r in FP32 (one ordered sweep), x += d in FP64, r = b - T x
// in FP64, until max|r| <= tol max|b|.
__global__ void k_zero_d(int n, double* x) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = 0.0;
}

__global__ void k_add_f32(int n, const float* __restrict__ d, double* x) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = x[i] + (double)d[i];
}

__global__ void k_copy_dd(int n, const double* __restrict__ a, double* b) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i];
}

// r = b - (I - W^T) x, donors summed in ascending id as in the FP64 sweep
__global__ void k_flow_resid(int n, const int* __restrict__ nbr, const uint32_t* __restrict__ mask,
                             const unsigned long long* __restrict__ dk, const unsigned long long* __restrict__ sorder,
                             const double* __restrict__ wgt, const double* __restrict__ b,
                             const double* __restrict__ x, double* r) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t m = mask[i];
    unsigned long long kk = dk[i], ord = sorder[i];
    double s = b[i];
    for (int q = 0; q < MAXW && m; q++) {
        int t = (int)(ord & 15ULL);
        ord >>= 4;
        if (!(m & (1u << t))) continue;
        m &= ~(1u << t);
        int j = nbr[(size_t)t * n + i];
        int k = (int)((kk >> (4 * t)) & 15ULL);
        s = s + wgt[(size_t)k * n + j] * x[j];
    }
    r[i] = s - x[i];
}

// r = hOld - M x for the SPL matrix (den_i x_i - sum_k c_ik x_rcv)
__global__ void k_spl_resid(int n, int R, const int* __restrict__ rcv, const double* __restrict__ c,
                            const double* __restrict__ hold, const double* __restrict__ x, double* r) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double num = hold[i], den = 1.0;
    for (int k = 0; k < R; k++) {
        double ck = c[(size_t)k * n + i];
        int q = rcv[(size_t)k * n + i];
        if (q != i && ck != 0.0) num = num + ck * x[q];
        den = den + ck;
    }
    r[i] = num - den * x[i];
}

__global__ void k_absmax_key(int n, const double* __restrict__ x, unsigned long long* out) {
    unsigned long long best = 0ULL;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        unsigned long long k = dkey(fabs(x[i]));
        best = k > best ? k : best;
    }
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long v = __shfl_xor_sync(0xffffffffu, best, o);
        best = v > best ? v : best;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(out, best);
}

int precision_buffers(gs_plan* p) {
    const size_t n = (size_t)std::max<int64_t>(p->n, 1);
    if (!p->f32a) GS_CUDA(cudaMalloc((void**)&p->f32a, sizeof(float) * n));
    if (!p->r64) GS_CUDA(cudaMalloc((void**)&p->r64, sizeof(double) * n));
    return GS_OK;
}

static int absmax_ratio(gs_plan* p, const double* r, const double* b, double* ratio) {
    const int n = (int)p->n;
    GS_CUDA(cudaMemsetAsync(p->u_scalar + 2, 0, 2 * sizeof(unsigned long long), p->stream));
    launch(p, k_absmax_key, p->sm_count * 4, 256, n, r, p->u_scalar + 2);
    launch(p, k_absmax_key, p->sm_count * 4, 256, n, b, p->u_scalar + 3);
    GS_LAUNCH();
    unsigned long long k[2];
    GS_CUDA(cudaMemcpyAsync(k, p->u_scalar + 2, sizeof(k), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    auto inv = [](unsigned long long u) {
        unsigned long long v = (u & 0x8000000000000000ULL) ? (u & 0x7fffffffffffffffULL) : ~u;
        double d;
        memcpy(&d, &v, sizeof(d));
        return d;
    };
    const double rr = k[0] ? inv(k[0]) : 0.0, bb = k[1] ? inv(k[1]) : 0.0;
    *ratio = bb > 0.0 ? rr / bb : rr;
    return GS_OK;
}

// (I - W^T) x = b with the donor masks of flow_prepare and a valid flow order
int flow_refine32(gs_plan* p, const double* wgt, const double* b, double* x, const int* order) {
    const int n = (int)p->n;
    const int B = 256, G = grid_for(n, B);
    GS_TRY(precision_buffers(p));
    launch(p, k_copy_dd, G, B, n, b, p->r64);
    launch(p, k_zero_d, G, B, n, x);
    int it = 0;
    double ratio = 1.0;
    for (; it < 8; it++) {
        GS_CUDA(cudaMemsetAsync(p->ctr, 0, sizeof(unsigned) * 8, p->stream));
        launch(p, k_fill_sent32, G, B, n, p->f32a);
        FlowOrd32 op{n, p->nbr, p->don_mask, p->don_k, p->sorder, wgt, (const double*)p->r64, p->f32a};
        launch(p, k_ordered<FlowOrd32>, p->sm_count * p->sweep_per_sm, 128, op, n, order, p->ctr, p->sweep_budget_ns, p->sweep_nap, (const int*)nullptr);
        GS_LAUNCH();
        int st = 0;
        GS_TRY(ordered_status(p, &st));
        if (st != 0) {
            set_error(st, "FP32 flow sweep did not complete");
            return st;
        }
        launch(p, k_add_f32, G, B, n, (const float*)p->f32a, x);
        launch(p, k_flow_resid, G, B, n, (const int*)p->nbr, (const uint32_t*)p->don_mask,
               (const unsigned long long*)p->don_k, (const unsigned long long*)p->sorder, wgt, b, (const double*)x,
               p->r64);
        GS_LAUNCH();
        GS_TRY(absmax_ratio(p, p->r64, b, &ratio));
        if (!(ratio > p->refine_tol)) break;
    }
    p->refine_iters += it + 1;
    if (ratio > p->refine_tol) {
        set_error(GS_EMAXITER, "FP32 flow refinement did not reach its tolerance");
        return GS_EMAXITER;
    }
    return GS_OK;
}

// M s = hOld for the SPL coefficients c, receivers first (order2)
int spl_refine32(gs_plan* p, const int* rcv, const double* c, const double* hold, double* x, const int* order2) {
    const int n = (int)p->n;
    const int B = 256, G = grid_for(n, B);
    GS_TRY(precision_buffers(p));
    launch(p, k_copy_dd, G, B, n, hold, p->r64);
    launch(p, k_zero_d, G, B, n, x);
    int it = 0;
    double ratio = 1.0;
    for (; it < 8; it++) {
        GS_CUDA(cudaMemsetAsync(p->ctr, 0, sizeof(unsigned) * 8, p->stream));
        launch(p, k_fill_sent32, G, B, n, p->f32a);
        SplOrd32 op{n, p->R, rcv, c, (const double*)p->r64, p->f32a};
        launch(p, k_ordered<SplOrd32>, p->sm_count * p->sweep_per_sm, 128, op, n, order2, p->ctr, p->sweep_budget_ns, p->sweep_nap, (const int*)nullptr);
        GS_LAUNCH();
        int st = 0;
        GS_TRY(ordered_status(p, &st));
        if (st != 0) {
            set_error(st, "FP32 SPL sweep did not complete");
            return st;
        }
        launch(p, k_add_f32, G, B, n, (const float*)p->f32a, x);
        launch(p, k_spl_resid, G, B, n, p->R, rcv, c, hold, (const double*)x, p->r64);
        GS_LAUNCH();
        GS_TRY(absmax_ratio(p, p->r64, hold, &ratio));
        if (!(ratio > p->refine_tol)) break;
    }
    p->refine_iters += it + 1;
    if (ratio > p->refine_tol) {
        set_error(GS_EMAXITER, "FP32 SPL refinement did not reach its tolerance");
        return GS_EMAXITER;
    }
    return GS_OK;
}

// Plain FP64 sweeps with caller-given right-hand sides, for solvers that
// apply the flow or SPL inverse repeatedly (the coupled erosion-deposition
// system).  sweep_flow_rhs needs the donor masks of the graph (flow_prepare or
// build_donors) and a valid flow order; sweep_spl_rhs the receivers-first
// order (the flow order reversed).
int build_donors(gs_plan* p, const int* rcv, const double* wgt, const int8_t* rslot) {
    const int n = (int)p->n;
    GS_CUDA(cudaMemsetAsync(p->don_mask, 0, sizeof(uint32_t) * n, p->stream));
    GS_CUDA(cudaMemsetAsync(p->don_k, 0, sizeof(unsigned long long) * n, p->stream));
    launch(p, k_flow_donors, grid_for(n, 256), 256, n, p->R, rcv, wgt, rslot, (const int8_t*)p->rev, p->don_mask,
           p->don_k);
    GS_LAUNCH();
    return GS_OK;
}

int sweep_flow_rhs(gs_plan* p, const double* wgt, const int* order, const double* b, double* x) {
    const int n = (int)p->n;
    GS_CUDA(cudaMemsetAsync(p->ctr, 0, sizeof(unsigned) * 8, p->stream));
    launch(p, k_fill_sent, grid_for(n, 256), 256, n, x);
    FlowOrd op{n, p->nbr, p->don_mask, p->don_k, p->sorder, wgt, b, x};
    launch(p, k_ordered<FlowOrd>, p->sm_count * p->sweep_per_sm, 128, op, n, order, p->ctr, p->sweep_budget_ns, p->sweep_nap, (const int*)nullptr);
    GS_LAUNCH();
    int st = 0;
    GS_TRY(ordered_status(p, &st));
    if (st != 0) {
        set_error(st, "flow sweep did not complete");
        return st;
    }
    return GS_OK;
}

int sweep_spl_rhs(gs_plan* p, const int* rcv, const double* c, const int* order2, const double* rhs, double* x) {
    const int n = (int)p->n;
    GS_CUDA(cudaMemsetAsync(p->ctr, 0, sizeof(unsigned) * 8, p->stream));
    launch(p, k_fill_sent, grid_for(n, 256), 256, n, x);
    SplOrd op{n, p->R, rcv, c, rhs, x};
    launch(p, k_ordered<SplOrd>, p->sm_count * p->sweep_per_sm, 128, op, n, order2, p->ctr, p->sweep_budget_ns, p->sweep_nap, (const int*)nullptr);
    GS_LAUNCH();
    int st = 0;
    GS_TRY(ordered_status(p, &st));
    if (st != 0) {
        set_error(st, "SPL sweep did not complete");
        return st;
    }
    return GS_OK;
}

// order2 = the snapshot flow order reversed (receivers first)
int spl_order(gs_plan* p) {
    const int n = (int)p->n;
    launch(p, k_reverse, grid_for(n, 256), 256, n, (const int*)p->order_i, p->order2);
    GS_LAUNCH();
    return GS_OK;
}

}  // namespace gs
