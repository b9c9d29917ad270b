// Hand-written adjoint of one physics step (flow accumulation with the lake
// cascade, SPL, hillslope, uplift) for gradients of an elevation misfit with
// respect to elevation, erodibility, uplift and rainfall.
//
// The forward records what it decided in a per-step slot (gs_plan_record):
// receivers, topological orders, masks, per-pass cascade decisions and the
// solutions the transposed solves need.  gs_adjoint_step then differentiates
// the step with every discrete decision held fixed: receiver choice, pit
// labels, flat routing, the cascade's overflow/partial states and pass count,
// lake zeroing, land/sea masks.  Continuous dependencies are all
// differentiated except the levels of partially filled lakes:
//   - MFD slope weights on the surface they were built on (adaptive exponent
//     included), for the snapshot graph (on h) and every cascade rebuild (on
//     the water surface: h, or the lake level of an overflowing pit, whose
//     derivative goes to the pit's pour cell);
//   - the flow solves (transposed sweep in reverse topological order) with
//     respect to their right-hand sides and weights;
//   - the cascade's inflow sums, excess e = inV - pitVol and its placement at
//     the spill node, the pitVol recursion of partially filled pits, and the
//     initial pit volumes sum((lFill - max(h, sea)) larea) through h and the
//     lake level;
//   - SPL (Kbr, lim, weights, the implicit solve) and hillslope (CG on the
//     same symmetric operator), uplift and rainfall.
#include <vector>

#include "gs_plan.cuh"

struct PassRec {
    int solved = 0, rebuilt = 0, order_ok = 1;
    uint8_t* lsink = nullptr;
    uint8_t* state = nullptr;
    uint8_t* spillw = nullptr;
    int* rcv = nullptr;
    double* wgt = nullptr;
    int8_t* rslot = nullptr;
    int* order = nullptr;
    double* x = nullptr;
    double* wf = nullptr;
};

struct StepRec {
    int valid = 0, npass = 0, np1 = 0, order_ok = 1, lakes = 0;
    double *hold = nullptr, *wgt0 = nullptr, *dist0 = nullptr, *q0 = nullptr, *fal = nullptr, *s = nullptr,
           *hin = nullptr, *lfill = nullptr, *vol0 = nullptr;
    int *rcv0 = nullptr, *order0 = nullptr, *pit = nullptr, *seg_start = nullptr, *seg_count = nullptr,
        *seg_cells = nullptr, *pour = nullptr, *pit_info = nullptr;
    int8_t* rslot0 = nullptr;
    uint8_t *sea = nullptr, *lsink_spl = nullptr;
    std::vector<PassRec> passes;
};

struct gs_record {
    std::vector<StepRec> steps;
};

namespace gs {

template <class T>
static int ralloc(T** p, size_t count) {
    if (*p) return GS_OK;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * count);
    if (e != cudaSuccess) {
        set_error(GS_ENOMEM, std::string("record: cudaMalloc: ") + cudaGetErrorString(e));
        return GS_ENOMEM;
    }
    return GS_OK;
}

template <class T>
static int rcopy(gs_plan* p, T** dst, const T* src, size_t count) {
    GS_TRY(ralloc(dst, count));
    GS_CUDA(cudaMemcpyAsync(*dst, src, sizeof(T) * count, cudaMemcpyDeviceToDevice, p->stream));
    return GS_OK;
}

static void free_pass(PassRec& r) {
    void* ptrs[] = {r.lsink, r.state, r.spillw, r.rcv, r.wgt, r.rslot, r.order, r.x, r.wf};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    r = PassRec();
}

static void free_step(StepRec& r) {
    void* ptrs[] = {r.hold, r.wgt0, r.dist0, r.q0, r.fal, r.s, r.hin, r.lfill, r.vol0, r.rcv0, r.order0, r.pit,
                    r.seg_start, r.seg_count, r.seg_cells, r.pour, r.pit_info, r.rslot0, r.sea, r.lsink_spl};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    for (PassRec& q : r.passes) free_pass(q);
    r = StepRec();
}

void record_free(gs_plan* p) {
    if (!p->rec) return;
    for (StepRec& r : p->rec->steps) free_step(r);
    delete p->rec;
    p->rec = nullptr;
    p->rec_slot = -1;
    void* ptrs[] = {p->adj_er, p->adj_gw, p->adj_nb, p->adj_v0, p->adj_v1, p->adj_v2, p->adj_v3};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    p->adj_er = p->adj_gw = p->adj_nb = p->adj_v0 = p->adj_v1 = p->adj_v2 = p->adj_v3 = nullptr;
}

int record_setup(gs_plan* p, int nslots) {
    if (nslots < 0) {
        set_error(GS_EINVAL, "record: nslots must be >= 0");
        return GS_EINVAL;
    }
    GS_CUDA(cudaStreamSynchronize(p->stream));
    if (p->rec && nslots > 0 && (int)p->rec->steps.size() == nslots) {
        // same layout: keep the device buffers, forget the recorded steps
        for (StepRec& r : p->rec->steps) r.valid = 0;
        p->rec_slot = -1;
        return GS_OK;
    }
    record_free(p);
    if (nslots == 0) return GS_OK;
    if (p->nmem != 1) {
        set_error(GS_EINVAL, "record: the adjoint replays single-landscape plans only");
        return GS_EINVAL;
    }
    p->rec = new gs_record();
    p->rec->steps.resize(nslots);
    return GS_OK;
}

static StepRec* cur(gs_plan* p) {
    if (!p->rec || p->rec_slot < 0 || p->rec_slot >= (int)p->rec->steps.size()) return nullptr;
    return &p->rec->steps[p->rec_slot];
}

int record_select(gs_plan* p, int slot) {
    if (slot >= 0 && (!p->rec || slot >= (int)p->rec->steps.size())) {
        set_error(GS_EINVAL, "record: slot out of range (gs_plan_record first)");
        return GS_EINVAL;
    }
    p->rec_slot = slot;
    if (slot >= 0) {
        StepRec& r = p->rec->steps[slot];
        r.valid = 0;
        r.npass = 0;
    }
    return GS_OK;
}

// ---- hooks called by the forward ------------------------------------------
int rec_initial(gs_plan* p, const double* h, const int* rcv, const double* wgt, const double* dist,
                const int8_t* rslot, const int* order, int order_ok, const double* q0, const uint8_t* sea) {
    StepRec* r = cur(p);
    if (!r) return GS_OK;
    const size_t n = (size_t)p->n, Rn = (size_t)p->R * n;
    GS_TRY(rcopy(p, &r->hold, h, n));
    GS_TRY(rcopy(p, &r->rcv0, rcv, Rn));
    GS_TRY(rcopy(p, &r->wgt0, wgt, Rn));
    GS_TRY(rcopy(p, &r->dist0, dist, Rn));
    GS_TRY(rcopy(p, &r->rslot0, rslot, Rn));
    GS_TRY(rcopy(p, &r->order0, order, n));
    GS_TRY(rcopy(p, &r->q0, q0, n));
    GS_TRY(rcopy(p, &r->sea, sea, n));
    r->order_ok = order_ok;
    return GS_OK;
}

__global__ void k_spillw(int np1, const uint8_t* __restrict__ state, const int* __restrict__ info,
                         const int* __restrict__ win, uint8_t* out) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= np1) return;
    out[q] = (state[q] == 1 && info[2 * q + 1] == 0 && win[info[2 * q]] == q) ? 1 : 0;
}

static PassRec* pass_at(gs_plan* p, int t) {
    StepRec* r = cur(p);
    if (!r) return nullptr;
    if ((int)r->passes.size() <= t) r->passes.resize(t + 1);
    if (r->npass < t + 1) r->npass = t + 1;
    return &r->passes[t];
}

int rec_pass_pits(gs_plan* p, int t, const uint8_t* lsink, int np1) {
    PassRec* q = pass_at(p, t);
    if (!q) return GS_OK;
    const size_t n = (size_t)p->n;
    q->solved = q->rebuilt = 0;
    GS_TRY(rcopy(p, &q->lsink, lsink, n));
    GS_TRY(ralloc(&q->state, n + 1));
    GS_TRY(ralloc(&q->spillw, n + 1));
    GS_CUDA(cudaMemcpyAsync(q->state, p->pit_state, np1, cudaMemcpyDeviceToDevice, p->stream));
    launch(p, k_spillw, grid_for(np1, 256), 256, np1, (const uint8_t*)p->pit_state, (const int*)p->pit_info,
           (const int*)p->pit_win, q->spillw);
    GS_LAUNCH();
    return GS_OK;
}

int rec_pass_rebuild(gs_plan* p, int t, const double* surf) {
    PassRec* q = pass_at(p, t);
    if (!q) return GS_OK;
    q->rebuilt = 1;
    GS_TRY(rcopy(p, &q->wf, surf, (size_t)p->n));
    return GS_OK;
}

int rec_pass_solve(gs_plan* p, int t, const int* order, int order_ok, const double* x) {
    PassRec* q = pass_at(p, t);
    if (!q) return GS_OK;
    const size_t n = (size_t)p->n, Rn = (size_t)p->R * n;
    q->solved = 1;
    q->order_ok = order_ok;
    GS_TRY(rcopy(p, &q->rcv, (const int*)p->rcv, Rn));
    GS_TRY(rcopy(p, &q->wgt, (const double*)p->wgt, Rn));
    GS_TRY(rcopy(p, &q->rslot, (const int8_t*)p->rslot, Rn));
    GS_TRY(rcopy(p, &q->order, order, n));
    GS_TRY(rcopy(p, &q->x, x, n));
    return GS_OK;
}

// pour cell of each pit: the cell whose elevation is the lake level (the
// spill node when it sits at the level, else its lowest-id neighbour outside
// the pit at the level); -1 when none is found (no lake-level derivative)
__global__ void k_pour(int np1, int n, const int* __restrict__ info, const int* __restrict__ seg_start,
                       const int* __restrict__ seg_count, const int* __restrict__ cells, const double* __restrict__ h,
                       const double* __restrict__ lfill, const int* __restrict__ pit, const int* __restrict__ nbr,
                       const int8_t* __restrict__ nnb, int* pour) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= np1) return;
    pour[q] = -1;
    if (q == 0 || seg_count[q] == 0) return;
    const double lvl = lfill[cells[seg_start[q]]];
    const int s = info[2 * q];
    if (s < 0 || s >= n) return;
    if (h[s] == lvl) { pour[q] = s; return; }
    int best = -1;
    for (int t = 0; t < nnb[s]; t++) {
        int v = nbr[(size_t)t * n + s];
        if (v < 0 || pit[v] == q) continue;
        if (h[v] == lvl && (best < 0 || v < best)) best = v;
    }
    pour[q] = best;
}

int rec_final(gs_plan* p, int npass, const double* fal, const int* pit, const double* lfill, int lakes) {
    StepRec* r = cur(p);
    if (!r) return GS_OK;
    const size_t n = (size_t)p->n;
    const int np1 = p->npits + 1;
    r->npass = npass;
    r->np1 = np1;
    r->lakes = lakes;
    GS_TRY(rcopy(p, &r->fal, fal, n));
    GS_TRY(rcopy(p, &r->pit, pit, n));
    GS_TRY(rcopy(p, &r->lfill, lfill, n));
    GS_TRY(ralloc(&r->vol0, n + 1));
    GS_TRY(ralloc(&r->seg_start, n + 2));
    GS_TRY(ralloc(&r->seg_count, n + 2));
    GS_TRY(ralloc(&r->seg_cells, n + 1));
    GS_TRY(ralloc(&r->pour, n + 1));
    GS_TRY(ralloc(&r->pit_info, 2 * (n + 1)));
    // pit tables: pitVol (column 0 of pitParams), the per-pit cell lists
    GS_CUDA(cudaMemcpy2DAsync(r->vol0, sizeof(double), p->pit_params, 3 * sizeof(double), sizeof(double), np1,
                              cudaMemcpyDeviceToDevice, p->stream));
    GS_CUDA(cudaMemcpyAsync(r->seg_start, p->seg_start, sizeof(int) * (np1 + 1), cudaMemcpyDeviceToDevice,
                            p->stream));
    GS_CUDA(cudaMemcpyAsync(r->seg_count, p->seg_count, sizeof(int) * (np1 + 1), cudaMemcpyDeviceToDevice,
                            p->stream));
    GS_CUDA(cudaMemcpyAsync(r->seg_cells, p->seg_vals2, sizeof(int) * n, cudaMemcpyDeviceToDevice, p->stream));
    GS_CUDA(cudaMemcpyAsync(r->pit_info, p->pit_info, sizeof(int) * 2 * np1, cudaMemcpyDeviceToDevice, p->stream));
    launch(p, k_pour, grid_for(np1, 256), 256, np1, (int)n, (const int*)p->pit_info, (const int*)p->seg_start,
           (const int*)p->seg_count, (const int*)p->seg_vals2, (const double*)r->hold, lfill, pit,
           (const int*)p->nbr, (const int8_t*)p->nnb, r->pour);
    GS_LAUNCH();
    return GS_OK;
}

int rec_spl(gs_plan* p, const double* s, const uint8_t* lsink) {
    StepRec* r = cur(p);
    if (!r) return GS_OK;
    GS_TRY(rcopy(p, &r->s, s, (size_t)p->n));
    GS_TRY(rcopy(p, &r->lsink_spl, lsink, (size_t)p->n));
    return GS_OK;
}

int rec_hill(gs_plan* p, const double* h_in) {
    StepRec* r = cur(p);
    if (!r) return GS_OK;
    GS_TRY(rcopy(p, &r->hin, h_in, (size_t)p->n));
    r->valid = 1;
    return GS_OK;
}

// ---- adjoint kernels ------------------------------------------------------
__global__ void k_axpy_acc(int n, double a, const double* __restrict__ x, double* y) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += a * x[i];
}

__global__ void k_mask_pos(int n, const double* __restrict__ v, double* g) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !(v[i] > 0.0)) g[i] = 0.0;
}

// g_x = mask (h >= wf) * gfal + dt * gFA
__global__ void k_cascade_gx(int n, const double* __restrict__ h, const double* __restrict__ wf,
                             const double* __restrict__ gfal, const double* __restrict__ gfa, double dt, double* gx) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    gx[i] = ((h[i] < wf[i]) ? 0.0 : gfal[i]) + dt * gfa[i];
}

// dJ/dw_ik = x_i y_{rcv_ik} (flow solve (I - W^T) x = b), accumulated or written
__global__ void k_edge_gw(int n, int R, const int* __restrict__ rcv, const double* __restrict__ wgt,
                          const double* __restrict__ x, const double* __restrict__ y, int accumulate, double* gw) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = 0; k < R; k++) {
        int r = rcv[(size_t)k * n + i];
        double v = (r != i && wgt[(size_t)k * n + i] != 0.0) ? x[i] * y[r] : 0.0;
        if (accumulate) gw[(size_t)k * n + i] += v;
        else gw[(size_t)k * n + i] = v;
    }
}

// per pit, reverse of one cascade pass: from dJ/dnfa (gnfa = y / dt) and the
// pitVol adjoint of the next pass, dJ/dinV and the pitVol adjoint of this pass
__global__ void k_cascade_pits_adj(int np1, const uint8_t* __restrict__ state, const uint8_t* __restrict__ spillw,
                                   const int* __restrict__ info, const double* __restrict__ y, double dt, int solved,
                                   double* gvol, double* ginv) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= np1) return;
    double ge = (solved && spillw[q]) ? y[info[2 * q]] / dt : 0.0;
    const double gv_next = gvol[q];
    const uint8_t s = state[q];
    if (s == 2) ge += gv_next;           // vol_{t+1} = vol_t + e
    double gv = (s == 1) ? 0.0 : gv_next;  // overflow: vol_{t+1} = 0
    gv -= ge;                            // e = inV - vol
    ginv[q] = ge;
    gvol[q] = gv;
}

// dJ/dFA of a pass: inV_p = sum over the pit's lsink cells of FA
__global__ void k_ginv_cells(int n, const int* __restrict__ pit, const uint8_t* __restrict__ lsink,
                             const double* __restrict__ ginv, double* gfa) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int q = pit[i];
    gfa[i] = (q > 0 && lsink[i]) ? ginv[q] : 0.0;
}

// surface gradient of a cascade rebuild to elevation: water surface = h
// outside lakes; = lake level (pour cell) on overflowing lakes; the level of
// a partially filled lake is held constant
__global__ void k_surf_to_h(int n, const double* __restrict__ surf, const double* __restrict__ h,
                            const double* __restrict__ lfill, const int* __restrict__ pit,
                            const double* __restrict__ gsurf, double* lam) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool lake = pit[i] > 0 && surf[i] == lfill[i];
    if (!lake && surf[i] == h[i]) lam[i] += gsurf[i];
}

// per pit: sum of gsurf over its lake-surface cells (fixed order), added to the pour cell
__global__ void k_pit_pour_sum(int np1, const int* __restrict__ seg_start, const int* __restrict__ seg_count,
                               const int* __restrict__ cells, const double* __restrict__ surf,
                               const double* __restrict__ lfill, const int* __restrict__ pour,
                               const double* __restrict__ gsurf, double* lam) {
    __shared__ double sh[256];
    const int q = blockIdx.x;
    if (q == 0 || pour[q] < 0) return;
    const int a = seg_start[q], c = seg_count[q];
    double acc = 0.0;
    for (int t = threadIdx.x; t < c; t += blockDim.x) {
        int i = cells[a + t];
        if (surf[i] == lfill[i]) acc += gsurf[i];
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0 && sh[0] != 0.0) atomicAdd(&lam[pour[q]], sh[0]);
}

// initial pit volumes vol_p = sum_{i in p} (lFill_i - max(h_i, sea)) larea_i
__global__ void k_pitvol_adj(int np1, const int* __restrict__ seg_start, const int* __restrict__ seg_count,
                             const int* __restrict__ cells, const double* __restrict__ h,
                             const double* __restrict__ larea, double sl, const int* __restrict__ pour,
                             const double* __restrict__ gvol, double* lam) {
    __shared__ double sh[256];
    const int q = blockIdx.x;
    if (q == 0) return;
    const double g = gvol[q];
    if (g == 0.0) return;
    const int a = seg_start[q], c = seg_count[q];
    double acc = 0.0;
    for (int t = threadIdx.x; t < c; t += blockDim.x) {
        int i = cells[a + t];
        acc += larea[i];
        if (h[i] > sl) lam[i] -= g * larea[i];
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0 && pour[q] >= 0) atomicAdd(&lam[pour[q]], g * sh[0]);
}

__global__ void k_gbl(int n, const uint8_t* __restrict__ sea, const double* __restrict__ y, double* gbl) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) gbl[i] = sea[i] ? 0.0 : y[i];
}

static int adj_buffers(gs_plan* p) {
    const size_t n = (size_t)std::max<int64_t>(p->n, 1);
    GS_TRY(ralloc(&p->adj_er, (size_t)p->R * n));
    GS_TRY(ralloc(&p->adj_gw, (size_t)p->R * n));
    GS_TRY(ralloc(&p->adj_nb, (size_t)p->W * n));
    GS_TRY(ralloc(&p->adj_v0, n + 1));
    GS_TRY(ralloc(&p->adj_v1, n + 1));
    GS_TRY(ralloc(&p->adj_v2, n + 1));
    GS_TRY(ralloc(&p->adj_v3, n + 1));
    return GS_OK;
}

// dJ/dsurface of one flow graph's weights to elevation, through the pour cells
static int graph_weights_adj(gs_plan* p, const StepRec& r, const double* surf, const int8_t* rslot,
                             const double* gw, double* lam, bool snapshot, double sl) {
    const int n = (int)p->n;
    const int B = 256, G = grid_for(n, B);
    double* gsurf = p->nfa;   // free during the adjoint
    if (snapshot) return receivers_adjoint(p, surf, sl, rslot, gw, p->adj_v3, p->adj_nb, lam);
    GS_CUDA(cudaMemsetAsync(gsurf, 0, sizeof(double) * n, p->stream));
    GS_TRY(receivers_adjoint(p, surf, sl, rslot, gw, p->adj_v3, p->adj_nb, gsurf));
    launch(p, k_surf_to_h, G, B, n, surf, (const double*)r.hold, (const double*)r.lfill, (const int*)r.pit,
           (const double*)gsurf, lam);
    launch(p, k_pit_pour_sum, r.np1, 256, r.np1, (const int*)r.seg_start, (const int*)r.seg_count,
           (const int*)r.seg_cells, surf, (const double*)r.lfill, (const int*)r.pour, (const double*)gsurf, lam);
    GS_LAUNCH();
    return GS_OK;
}

int adjoint_step(gs_plan* p, int slot, double* lam, const double* rain, double k_scalar, const double* k_field,
                 double d, double m, double dt, double sealevel, double cda, double cdm, double rtol, int max_iter,
                 double* gK, double* gU, double* grain, double* gbl) {
    if (!p->rec || slot < 0 || slot >= (int)p->rec->steps.size() || !p->rec->steps[slot].valid) {
        set_error(GS_EINVAL, "adjoint: slot holds no recorded step");
        return GS_EINVAL;
    }
    StepRec& r = p->rec->steps[slot];
    if (p->fdepa > 0.0) {
        set_error(GS_EINVAL, "adjoint: transport-limited SPL (G > 0) has no adjoint here");
        return GS_EINVAL;
    }
    if (!r.order_ok) {
        set_error(GS_EINVAL, "adjoint: the recorded step used the unordered flow solve");
        return GS_EINVAL;
    }
    const int n = (int)p->n;
    if (n == 0) return GS_OK;
    const int B = 256, G = grid_for(n, B);
    GS_TRY(adj_buffers(p));
    // uplift: h_{t+1} = x + U dt
    if (gU) launch(p, k_axpy_acc, G, B, n, dt, (const double*)lam, gU);
    // hillslope
    int it = 0;
    GS_TRY(hillslope_adjoint(p, r.hin, lam, sealevel, cda, cdm, dt, rtol, max_iter, &it));
    // SPL: lam -> dJ/dhOld (SPL part), gfal, gw (snapshot weights, SPL part)
    double* gfal = p->adj_v0;
    GS_TRY(spl_adjoint(p, r.hold, r.s, r.fal, rain, k_scalar, k_field, d, m, dt, r.rcv0, r.dist0, r.wgt0, r.rslot0,
                       r.order0, r.lsink_spl, r.sea, lam, gK, grain, gfal, p->adj_gw));
    launch(p, k_mask_pos, G, B, n, (const double*)r.fal, gfal);   // lake zeroing and the clamp at 0
    // lake cascade, last pass first
    double* gfa = p->adj_v1;
    double* gx = p->adj_v2;
    double* y = p->q3;
    double* gvol = p->pit_vol;   // per-pit adjoint of pitVol
    double* ginv = p->pit_in;
    GS_CUDA(cudaMemsetAsync(gfa, 0, sizeof(double) * n, p->stream));
    if (r.np1 > 0) GS_CUDA(cudaMemsetAsync(gvol, 0, sizeof(double) * r.np1, p->stream));
    for (int t = r.npass - 1; t >= 0; t--) {
        PassRec& q = r.passes[t];
        if (q.solved) {
            if (!q.order_ok) {
                set_error(GS_EINVAL, "adjoint: a recorded cascade solve used the unordered flow solve");
                return GS_EINVAL;
            }
            launch(p, k_cascade_gx, G, B, n, (const double*)r.hold, (const double*)q.wf, (const double*)gfal,
                   (const double*)gfa, dt, gx);
            GS_LAUNCH();
            GS_TRY(sweep_flow_adjoint(p, q.rcv, q.wgt, q.order, gx, y));
            launch(p, k_edge_gw, G, B, n, p->R, (const int*)q.rcv, (const double*)q.wgt, (const double*)q.x,
                   (const double*)y, 0, p->adj_er);
            GS_LAUNCH();
            GS_TRY(graph_weights_adj(p, r, q.wf, q.rslot, p->adj_er, lam, false, sealevel));
        }
        launch(p, k_cascade_pits_adj, grid_for(r.np1, B), B, r.np1, (const uint8_t*)q.state,
               (const uint8_t*)q.spillw, (const int*)r.pit_info, (const double*)y, dt, q.solved, gvol, ginv);
        launch(p, k_ginv_cells, G, B, n, (const int*)r.pit, (const uint8_t*)q.lsink, (const double*)ginv, gfa);
        GS_LAUNCH();
    }
    // initial solve: fal = q0 (+ cascade increments), FA_0 = q0 dt
    if (r.npass > 0) launch(p, k_axpy_acc, G, B, n, dt, (const double*)gfa, gfal);
    GS_TRY(sweep_flow_adjoint(p, r.rcv0, r.wgt0, r.order0, gfal, y));
    if (gbl) launch(p, k_gbl, G, B, n, (const uint8_t*)r.sea, (const double*)y, gbl);
    launch(p, k_edge_gw, G, B, n, p->R, (const int*)r.rcv0, (const double*)r.wgt0, (const double*)r.q0,
           (const double*)y, 1, p->adj_gw);
    GS_LAUNCH();
    GS_TRY(graph_weights_adj(p, r, r.hold, r.rslot0, p->adj_gw, lam, true, sealevel));
    if (r.npass > 0 && r.np1 > 1)
        launch(p, k_pitvol_adj, r.np1, 256, r.np1, (const int*)r.seg_start, (const int*)r.seg_count,
               (const int*)r.seg_cells, (const double*)r.hold, (const double*)p->larea, sealevel,
               (const int*)r.pour, (const double*)gvol, lam);
    GS_LAUNCH();
    GS_CUDA(cudaStreamSynchronize(p->stream));
    return GS_OK;
}

}  // namespace gs
