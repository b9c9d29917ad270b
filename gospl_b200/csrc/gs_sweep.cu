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

#include <cstring>

#include "gs_plan.cuh"

namespace cg = cooperative_groups;

namespace gs {

enum { C_HEAD = 0, C_TAIL = 1, C_DONE = 2, C_STATUS = 3 };

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
};

template <class Op>
__global__ void k_dataflow(Op op, Sched sc, int n, unsigned long long budget_ns) {
    const unsigned long long t0 = globaltimer_ns();
    for (;;) {
        unsigned t = agg_add(&sc.ctr[C_HEAD], 1u);
        if (t >= (unsigned)n) return;
        int node;
        unsigned spins = 0, nap = 32;
        for (;;) {
            node = ld_acquire(&sc.queue[t]);
            if (node >= 0) break;
            if ((++spins & 15u) == 0) {
                if (ld_relaxed_u32(&sc.ctr[C_STATUS]) != 0) return;
                unsigned d = ld_relaxed_u32(&sc.ctr[C_DONE]);
                unsigned tl = ld_relaxed_u32(&sc.ctr[C_TAIL]);
                if (d == tl && tl <= t) {
                    atomicCAS(&sc.ctr[C_STATUS], 0u, (unsigned)GS_ECYCLE);
                    return;
                }
                if (globaltimer_ns() - t0 > budget_ns) {
                    atomicCAS(&sc.ctr[C_STATUS], 0u, (unsigned)GS_ETIMEOUT);
                    return;
                }
            }
            __nanosleep(nap);
            if (nap < 1024) nap <<= 1;
        }
        op.process(node, sc);
        __threadfence();
        agg_add(&sc.ctr[C_DONE], 1u);
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

__global__ void k_flow_setup(int n, const uint32_t* __restrict__ mask, int* cnt, Sched sc,
                             uint8_t* done) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = __popc(mask[i]);
    cnt[i] = c;
    done[i] = 0;
    if (c == 0) sc.publish(i);
}

__global__ void k_spl_setup(int n, const int* __restrict__ cnt, Sched sc, uint8_t* done) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    done[i] = 0;
    if (cnt[i] == 0) sc.publish(i);
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
    unsigned h[4];
    GS_CUDA(cudaMemcpyAsync(h, p->ctr, sizeof(h), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    *status_out = (int)h[C_STATUS];
    if (*status_out == 0 && h[C_DONE] != (unsigned)p->n) *status_out = GS_ECYCLE;
    return GS_OK;
}

static const unsigned long long SWEEP_BUDGET_NS = 4000000000ULL;   // 4 s

int flow_solve(gs_plan* p, const int* rcv, const double* wgt, const int8_t* rslot,
               const double* b, double* x, int* cycle_nodes) {
    const int n = (int)p->n;
    *cycle_nodes = 0;
    if (n == 0) return GS_OK;
    GS_CUDA(cudaMemsetAsync(p->don_mask, 0, sizeof(uint32_t) * n, p->stream));
    GS_CUDA(cudaMemsetAsync(p->don_k, 0, sizeof(unsigned long long) * n, p->stream));
    GS_CUDA(cudaMemsetAsync(p->queue, 0xff, sizeof(int) * n, p->stream));
    GS_CUDA(cudaMemsetAsync(p->ctr, 0, sizeof(unsigned) * 4, p->stream));
    launch(p, k_flow_donors, grid_for(n, 256), 256, n, p->R, rcv, wgt, rslot,
           (const int8_t*)p->rev, p->don_mask, p->don_k);
    GS_LAUNCH();
    Sched sc{p->queue, p->ctr, p->cnt, (unsigned)n};
    launch(p, k_flow_setup, grid_for(n, 256), 256, n, (const uint32_t*)p->don_mask, p->cnt, sc,
           p->done_flag);
    GS_LAUNCH();
    FlowOp op{n, p->R, p->nbr, p->don_mask, p->don_k, p->sorder, wgt, rcv, b, x, p->done_flag};
    launch(p, k_dataflow<FlowOp>, p->sm_count * 8, 256, op, sc, n, SWEEP_BUDGET_NS);
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
    unsigned h[4];
    GS_CUDA(cudaMemcpyAsync(h, p->ctr, sizeof(h), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    *cycle_nodes = n - (int)h[C_DONE];
    if (!converged) {
        set_error(GS_EMAXITER, "flow cycle fallback did not converge");
        return GS_EMAXITER;
    }
    return GS_OK;
}

int spl_sweep(gs_plan* p, const int* rcv, const double* c, const int8_t* rslot,
              const double* hold, double* s, int* cycle_nodes) {
    const int n = (int)p->n;
    *cycle_nodes = 0;
    if (n == 0) return GS_OK;
    GS_CUDA(cudaMemsetAsync(p->don_mask, 0, sizeof(uint32_t) * n, p->stream));
    GS_CUDA(cudaMemsetAsync(p->queue, 0xff, sizeof(int) * n, p->stream));
    GS_CUDA(cudaMemsetAsync(p->ctr, 0, sizeof(unsigned) * 4, p->stream));
    launch(p, k_spl_donors, grid_for(n, 256), 256, n, p->R, rcv, c, rslot, (const int8_t*)p->rev,
           p->don_mask, p->cnt);
    GS_LAUNCH();
    Sched sc{p->queue, p->ctr, p->cnt, (unsigned)n};
    launch(p, k_spl_setup, grid_for(n, 256), 256, n, (const int*)p->cnt, sc, p->done_flag);
    GS_LAUNCH();
    SplOp op{n, p->R, p->nbr, p->don_mask, rcv, c, hold, s, p->done_flag};
    launch(p, k_dataflow<SplOp>, p->sm_count * 8, 256, op, sc, n, SWEEP_BUDGET_NS);
    GS_LAUNCH();
    int st = 0;
    GS_TRY(sweep_status(p, &st));
    if (st != 0) {
        unsigned h[4];
        GS_CUDA(cudaMemcpyAsync(h, p->ctr, sizeof(h), cudaMemcpyDeviceToHost, p->stream));
        GS_CUDA(cudaStreamSynchronize(p->stream));
        *cycle_nodes = n - (int)h[C_DONE];
        set_error(st, "SPL sweep: receiver graph is not acyclic");
        return st;
    }
    return GS_OK;
}

}  // namespace gs
