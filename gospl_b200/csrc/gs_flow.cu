// Flow accumulation with the downstream lake cascade:
// FAMesh.flowAccumulation (flowplex.py:752-945) and _distributeDownstream
// (flowplex.py:576-686) without evaporation or ice.
//
// Control flow mirrors the reference pass by pass; the per-pit decisions
// (overflow, partial fill level, thresholds eV > 0, eV > 1e-3) run in small
// per-pit kernels, and only the handful of flags that steer the pass loop are
// read back to the host.
#include "gs_plan.cuh"

namespace gs {

enum { F_POS = 1, F_NEG = 2, F_BIG = 4 };

// deterministic sum / max (fixed two-stage tree, independent of timing)
__global__ void k_partial_sum(int64_t n, const double* __restrict__ x, double* part) {
    __shared__ double sh[256];
    double acc = 0.0;
    int64_t per = (n + gridDim.x - 1) / gridDim.x;
    int64_t lo = (int64_t)blockIdx.x * per, hi = lo + per < n ? lo + per : n;
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) acc += x[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_final_sum(int m, const double* __restrict__ part, double* out) {
    __shared__ double sh[1024];
    double acc = 0.0;
    for (int i = threadIdx.x; i < m; i += blockDim.x) acc += part[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

__global__ void k_max_key(int64_t n, const double* __restrict__ x, unsigned long long* out) {
    unsigned long long best = 0ULL;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        unsigned long long k = dkey(x[i]);
        best = k > best ? k : best;
    }
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long v = __shfl_xor_sync(0xffffffffu, best, o);
        best = v > best ? v : best;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(out, best);
}

static int sum_to_host(gs_plan* p, const double* x, int64_t n, double* out) {
    const int PARTS = 1024;
    launch(p, k_partial_sum, PARTS, 256, n, x, p->red);
    launch(p, k_final_sum, 1, 1024, PARTS, (const double*)p->red, p->red + PARTS);
    GS_LAUNCH();
    GS_CUDA(cudaMemcpyAsync(out, p->red + PARTS, sizeof(double), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    return GS_OK;
}

// ---------------------------------------------------------------------------
__global__ void k_fill_i32(int n, int* a, int v) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

__global__ void k_rain_sea(int n, const double* __restrict__ bl, const uint8_t* __restrict__ sea,
                           double* b) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = sea[i] ? 0.0 : bl[i];
}

__global__ void k_copy(int64_t n, const double* __restrict__ a, double* b) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i];
}

__global__ void k_scale(int64_t n, const double* __restrict__ a, double s, double* b) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i] * s;
}

__global__ void k_div(int64_t n, const double* __restrict__ a, double s, double* b) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i] / s;
}

// member of each pit: the member of its first cell
__global__ void k_pit_member(int np1, const int* __restrict__ seg_start, const int* __restrict__ seg_count,
                             const int* __restrict__ cells, const int* __restrict__ vmember, int* pmember) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < np1) pmember[p] = seg_count[p] > 0 ? vmember[cells[seg_start[p]]] : 0;
}

// members with a pit of positive volume
__global__ void k_any_pos(int np1, const double* __restrict__ params, const int* __restrict__ pmember,
                          uint8_t* mlakes) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < np1 && params[3 * p] > 0.0) mlakes[pmember[p]] = 1;
}

// per-member sums in a fixed order: one block per chunk, then each member's
// chunks in sequence
__global__ void k_chunk_sum(const int* __restrict__ lo, const double* __restrict__ x, double* part) {
    __shared__ double sh[256];
    const int a = lo[blockIdx.x], b = lo[blockIdx.x + 1];
    double acc = 0.0;
    for (int i = a + threadIdx.x; i < b; i += blockDim.x) acc += x[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_member_sum(int nmem, const int* __restrict__ m0, const double* __restrict__ part, double* out) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nmem) return;
    double acc = 0.0;
    for (int c = m0[m]; c < m0[m + 1]; c++) acc += part[c];
    out[m] = acc;
}

// per-member maximum of x (order-preserving keys)
__global__ void k_member_max(int n, const double* __restrict__ x, const int* __restrict__ vmember,
                             unsigned long long* mmax) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = i < n;
    const int m = in ? vmember[i] : -1;
    unsigned long long k = in ? dkey(x[i]) : 0ULL;
    const unsigned full = 0xffffffffu;
    const int m0 = __shfl_sync(full, m, 0);
    if (__all_sync(full, m == m0)) {
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long v = __shfl_xor_sync(full, k, o);
            k = v > k ? v : k;
        }
        if ((threadIdx.x & 31) == 0 && m0 >= 0) atomicMax(&mmax[m0], k);
    } else if (in) {
        atomicMax(&mmax[m], k);
    }
}

// lsink of members that did not rebuild their receivers this pass is kept
__global__ void k_lsink_keep(int n, const int* __restrict__ vmember, const uint8_t* __restrict__ mbig,
                             const uint8_t* __restrict__ prev, uint8_t* lsink) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !mbig[vmember[i]]) lsink[i] = prev[i];
}

// right-hand side only for members that solve this pass
__global__ void k_rhs_members(int n, const int* __restrict__ vmember, const uint8_t* __restrict__ msolve,
                              double* b) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !msolve[vmember[i]]) b[i] = 0.0;
}

__global__ void k_pitvol_init(int np1, const double* __restrict__ params, double* vol) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < np1) vol[p] = params[3 * p];
}

// per-pit decisions of one _distributeDownstream pass
__global__ void k_cascade_pits(int np1, const double* __restrict__ inV, double* vol,
                               const double* __restrict__ fvol, const double* __restrict__ flvl,
                               const int* __restrict__ info, const int* __restrict__ pmember,
                               const uint8_t* __restrict__ mact, double* ev, uint8_t* state,
                               double* lvl, int* win, int* mflags) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np1) return;
    const int mem = pmember[p];
    if (!mact[mem]) {   // member left the cascade loop: its pits are not touched
        state[p] = 0;
        return;
    }
    double in = inV[p];
    double e = in - vol[p];
    ev[p] = e;
    uint8_t s = 0;
    int f = 0;
    if (e > 0.0) {
        f |= F_POS;
        s = 1;
        vol[p] = 0.0;
        if (info[2 * p + 1] == 0) atomicMax(&win[info[2 * p]], p);
    }
    if (e < 0.0) {
        f |= F_NEG;
        if (in > 0.0) {
            s = 2;
            double v = vol[p] + e;
            vol[p] = v;
            int best = 0;
            double bd = fabs(fvol[5 * p] - v);
            for (int k = 1; k < 5; k++) {
                double d = fabs(fvol[5 * p + k] - v);
                if (d < bd) { bd = d; best = k; }
            }
            lvl[p] = flvl[5 * p + best];
        }
    }
    if (e > 1.0e-3) f |= F_BIG;
    state[p] = s;
    if (f) atomicOr(&mflags[mem], f);
}

__global__ void k_cascade_spill(int np1, const double* __restrict__ ev, const uint8_t* __restrict__ state,
                                const int* __restrict__ info, const int* __restrict__ win, double* nfa) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np1) return;
    if (state[p] == 1 && info[2 * p + 1] == 0 && win[info[2 * p]] == p) nfa[info[2 * p]] = ev[p];
}

__global__ void k_cascade_cells(int n, const int* __restrict__ pit, const uint8_t* __restrict__ state,
                                const double* __restrict__ lvl, const double* __restrict__ lfill,
                                double* wf) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int p = pit[i];
    if (p < 0) return;
    uint8_t s = state[p];
    if (s == 1) wf[i] = lfill[i];
    else if (s == 2) {
        double l = lvl[p];
        if (wf[i] <= l) wf[i] = l;
    }
}

__global__ void k_cascade_accum(int n, const double* __restrict__ sol, double dt,
                                const double* __restrict__ h, const double* __restrict__ wf,
                                double* nfa, double* fal) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = sol[i] * dt;
    nfa[i] = v;
    double fa = (h[i] < wf[i]) ? 0.0 : v;
    fal[i] = fal[i] + fa / dt;
}

__global__ void k_lake_zero(int n, const double* __restrict__ h, const double* __restrict__ wf,
                            const int* __restrict__ pit, const int* __restrict__ vmember,
                            const uint8_t* __restrict__ mlakes, double* fal) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (mlakes[vmember[i]] && h[i] <= wf[i] && pit[i] > -1) fal[i] = 0.0;
}

__global__ void k_flow_final(int n, const uint8_t* __restrict__ mlakes, const int* __restrict__ vmember,
                             const double* __restrict__ h, const double* __restrict__ wf,
                             const int* __restrict__ pit, const unsigned long long* __restrict__ mmax,
                             double* fal, double* fill_fal, double* water) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int m = vmember[i];
    double f = fal[i];
    double ff = f;
    if (mlakes[m] && h[i] <= wf[i] && pit[i] > -1) ff = dkey_inv(mmax[m]) * 0.1;
    fal[i] = f < 0.0 ? 0.0 : f;
    fill_fal[i] = ff < 0.0 ? 0.0 : ff;
    water[i] = wf[i] - h[i];
}

static int read_flag(gs_plan* p, int* out) {
    GS_CUDA(cudaMemcpyAsync(out, p->i_scalar + 8, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    return GS_OK;
}

int flow_accumulation(gs_plan* p, const double* h, const double* bl, double sealevel, double ofill,
                      double dt, double* fal, double* fill_fal, double* water, double* lfill,
                      int* pit_ids, int* flat_dirs, int* rcv_i, double* dist_i, double* wgt_i,
                      uint8_t* lsink, uint8_t* sea, gs_stats* st) {
    const int n = (int)p->n;
    if (n == 0) return GS_OK;
    const int B = 256, G = grid_for(n, B);
    // Receivers on the unfilled surface (down=False: they read h, not the
    // fill) and the topological order of their graph, on side_a while the
    // main stream fills depressions.
    int* bad_a = p->h_pinned + 1;
    GS_CUDA(cudaEventRecord(p->ev_fork_a, p->stream));
    GS_CUDA(cudaStreamWaitEvent(p->side_a, p->ev_fork_a, 0));
    {
        StreamSwap sw(p, p->side_a, p->cub_tmp2);
        GS_TRY(flow_direction(p, h, false, nullptr, nullptr, nullptr, sealevel, rcv_i, dist_i, wgt_i,
                              p->rslot_i, nullptr, nullptr));
        GS_TRY(flow_order(p, h, p->order_i));
        GS_TRY(flow_prepare(p, rcv_i, wgt_i, p->rslot_i, fal, p->order_i, bad_a));
    }
    GS_CUDA(cudaEventRecord(p->ev_a, p->side_a));
    GS_TRY(fill_elevation(p, h, sealevel, ofill, lfill, pit_ids, flat_dirs, st, true, sea, false, bl));
    const int P = p->npits, np1 = P + 1;

    // join: lsink of the snapshot graph, rain on land, the first flow sweep
    // (its flat directions are still being computed on side_b)
    GS_CUDA(cudaStreamWaitEvent(p->stream, p->ev_a, 0));
    GS_TRY(sink_mask(p, wgt_i, sea, lsink));
    launch(p, k_rain_sea, G, B, n, bl, (const uint8_t*)sea, p->nfa);
    GS_LAUNCH();
    GS_CUDA(cudaEventSynchronize(p->ev_a));
    const int ok_i = *bad_a ? 0 : 1;
    p->order_i_valid = ok_i;
    int cyc = 0;
    // the sweep's status is read at the next synchronisation (the lakes flag)
    int* sweep_st = p->h_pinned + 10;
    GS_TRY(flow_run(p, rcv_i, wgt_i, p->rslot_i, p->nfa, fal, &cyc, p->order_i, ok_i, sweep_st));
    GS_TRY(rec_initial(p, h, rcv_i, wgt_i, dist_i, p->rslot_i, p->order_i, ok_i, fal, sea));
    int total_cycles = cyc;
    launch(p, k_copy, G, B, (int64_t)n, h, p->wf);
    // pitVol and, per member, "any pit with volume"
    const int nm = p->nmem;
    launch(p, k_pitvol_init, grid_for(np1, B), B, np1, (const double*)p->pit_params, p->pit_vol);
    launch(p, k_pit_member, grid_for(np1, B), B, np1, (const int*)p->seg_start, (const int*)p->seg_count,
           (const int*)p->seg_vals2, (const int*)p->vmember, p->pmember);
    GS_CUDA(cudaMemsetAsync(p->mlakes, 0, nm, p->stream));
    launch(p, k_any_pos, grid_for(np1, B), B, np1, (const double*)p->pit_params, (const int*)p->pmember,
           p->mlakes);
    GS_LAUNCH();
    std::vector<uint8_t> lakes(nm, 0);
    GS_CUDA(cudaMemcpyAsync(lakes.data(), p->mlakes, nm, cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    if (*sweep_st != 0) {
        set_error(*sweep_st, "ordered flow sweep did not complete");
        return *sweep_st;
    }
    bool anyvol = false;
    for (int m = 0; m < nm; m++) anyvol = anyvol || lakes[m];
    int passes = 0, solves = 0;
    if (anyvol) {
        // Every member runs its own _distributeDownstream loop (flowplex.py:850-904):
        // a member leaves when it has no excess, after pass 100 or when its
        // residual stagnates; the pits and cells of members that left are not
        // touched by later passes of the others.
        std::vector<uint8_t> act(lakes), big(nm), solve(nm);
        std::vector<int> stall(nm, 0);
        std::vector<uint8_t> have_best(nm, 0);
        std::vector<double> best(nm, 0.0);
        double* FA = p->q;
        launch(p, k_scale, G, B, (int64_t)n, (const double*)fal, dt, FA);
        int step = 0;
        auto any = [](const std::vector<uint8_t>& v) {
            for (uint8_t x : v)
                if (x) return true;
            return false;
        };
        while (any(act) && step <= 100) {
            // ---- _distributeDownstream(pitVol, FA, hl, step) ----
            GS_CUDA(cudaMemcpyAsync(p->mact, act.data(), nm, cudaMemcpyHostToDevice, p->stream));
            GS_TRY(group_sum_by_pit(p, pit_ids, lsink, FA, p->pit_in, P));
            GS_CUDA(cudaMemsetAsync(p->mflags, 0, sizeof(int) * nm, p->stream));
            launch(p, k_fill_i32, grid_for(n, B), B, n, p->pit_win, -1);
            launch(p, k_cascade_pits, grid_for(np1, B), B, np1, (const double*)p->pit_in, p->pit_vol,
                   (const double*)p->filled_vol, (const double*)p->filled_lvl, (const int*)p->pit_info,
                   (const int*)p->pmember, (const uint8_t*)p->mact, p->pit_ev, p->pit_state, p->pit_lvl,
                   p->pit_win, p->mflags);
            GS_LAUNCH();
            GS_CUDA(cudaMemcpyAsync(p->h_mflags, p->mflags, sizeof(int) * nm, cudaMemcpyDeviceToHost, p->stream));
            GS_TRY(rec_pass_pits(p, step, lsink, np1));
            GS_CUDA(cudaStreamSynchronize(p->stream));
            int flags = 0;
            bool anybig = false, allbig = true;
            for (int m = 0; m < nm; m++) {
                const int f = act[m] ? p->h_mflags[m] : 0;
                flags |= f;
                big[m] = (f & F_BIG) ? 1 : 0;
                anybig = anybig || big[m];
                allbig = allbig && big[m];
                solve[m] = 0;
            }
            if (flags & F_POS) {
                GS_CUDA(cudaMemsetAsync(p->nfa, 0, sizeof(double) * n, p->stream));
                launch(p, k_cascade_spill, grid_for(np1, B), B, np1, (const double*)p->pit_ev,
                       (const uint8_t*)p->pit_state, (const int*)p->pit_info, (const int*)p->pit_win,
                       p->nfa);
            }
            if (flags & (F_POS | F_NEG))
                launch(p, k_cascade_cells, G, B, n, (const int*)pit_ids, (const uint8_t*)p->pit_state,
                       (const double*)p->pit_lvl, (const double*)lfill, p->wf);
            GS_LAUNCH();
            if (anybig) {
                const double* surf = (step == 100) ? lfill : p->wf;
                // lFill is final only after the flat pass (open-sea reset)
                if (step == 100) GS_TRY(fill_join(p, st));
                if (!allbig) {
                    GS_CUDA(cudaMemcpyAsync(p->lsink_prev, lsink, n, cudaMemcpyDeviceToDevice, p->stream));
                    GS_CUDA(cudaMemcpyAsync(p->mbig, big.data(), nm, cudaMemcpyHostToDevice, p->stream));
                }
                // receivers and the surface order do not need the flat BFS;
                // the flat routing and the order's ties do: join it between
                GS_TRY(receivers(p, p->R, 1.1, surf, sealevel, p->gid, p->rcv, p->dist, p->wgt, p->rslot));
                // the water surface differs from h only on lakes: reuse h's order
                GS_TRY(flow_order_from(p, surf, h, p->order_i, p->order));
                GS_TRY(flow_order_ties_prepare(p));
                launch(p, k_div, G, B, (int64_t)n, (const double*)p->nfa, dt, p->q2);
                launch(p, k_chunk_sum, p->nchunk, 256, (const int*)p->chunk_lo, (const double*)p->q2,
                       p->chunk_part);
                launch(p, k_member_sum, grid_for(nm, 128), 128, nm, (const int*)p->mchunk0,
                       (const double*)p->chunk_part, p->mresid);
                GS_LAUNCH();
                GS_CUDA(cudaMemcpyAsync(p->h_mresid, p->mresid, sizeof(double) * nm, cudaMemcpyDeviceToHost,
                                        p->stream));
                GS_TRY(fill_join(p, st));
                GS_TRY(flow_direction_post(p, surf, true, lfill, pit_ids, flat_dirs, sealevel, p->rcv, p->dist,
                                           p->wgt, p->rslot, lsink, sea));
                if (!allbig)
                    launch(p, k_lsink_keep, G, B, n, (const int*)p->vmember, (const uint8_t*)p->mbig,
                           (const uint8_t*)p->lsink_prev, lsink);
                GS_TRY(rec_pass_rebuild(p, step, surf));
                GS_TRY(flow_order_ties(p, p->pdir, p->order));
                GS_CUDA(cudaStreamSynchronize(p->stream));
                bool anysolve = false, allsolve = true;
                for (int m = 0; m < nm; m++) {
                    solve[m] = (big[m] && p->h_mresid[m] > p->mmaxarea[m]) ? 1 : 0;
                    anysolve = anysolve || solve[m];
                    allsolve = allsolve && solve[m];
                }
                if (anysolve) {
                    if (!allsolve) {
                        GS_CUDA(cudaMemcpyAsync(p->msolve, solve.data(), nm, cudaMemcpyHostToDevice, p->stream));
                        launch(p, k_rhs_members, G, B, n, (const int*)p->vmember, (const uint8_t*)p->msolve,
                               p->q2);
                    }
                    // solve into FA's buffer: FA is consumed already
                    GS_TRY(flow_prepare(p, p->rcv, p->wgt, p->rslot, p->q, p->order, p->h_pinned));
                    GS_CUDA(cudaStreamSynchronize(p->stream));
                    const int ok_c = p->h_pinned[0] ? 0 : 1;
                    GS_TRY(flow_run(p, p->rcv, p->wgt, p->rslot, p->q2, p->q, &cyc, p->order, ok_c, nullptr));
                    GS_TRY(rec_pass_solve(p, step, p->order, ok_c, p->q));
                    total_cycles += cyc;
                    launch(p, k_cascade_accum, G, B, n, (const double*)p->q, dt, h, (const double*)p->wf,
                           p->q, fal);
                    GS_LAUNCH();
                    solves++;
                }
            }
            step++;
            passes++;
            for (int m = 0; m < nm; m++) {
                if (!act[m]) continue;
                if (!solve[m]) {   // no excess: this member's loop ends
                    act[m] = 0;
                    continue;
                }
                const double r = p->h_mresid[m];
                if (!have_best[m] || r < best[m] * (1.0 - 1.0e-3)) {
                    best[m] = r;
                    have_best[m] = 1;
                    stall[m] = 0;
                } else if (++stall[m] >= 3) {
                    act[m] = 0;
                }
            }
        }
        launch(p, k_lake_zero, G, B, n, h, (const double*)p->wf, (const int*)pit_ids, (const int*)p->vmember,
               (const uint8_t*)p->mlakes, fal);
        GS_CUDA(cudaMemsetAsync(p->mmax, 0, sizeof(unsigned long long) * nm, p->stream));
        launch(p, k_member_max, G, B, n, (const double*)fal, (const int*)p->vmember, p->mmax);
        GS_LAUNCH();
    }
    GS_TRY(fill_join(p, st));
    launch(p, k_flow_final, G, B, n, (const uint8_t*)p->mlakes, (const int*)p->vmember, h, (const double*)p->wf,
           (const int*)pit_ids, (const unsigned long long*)p->mmax, fal, fill_fal, water);
    GS_LAUNCH();
    GS_TRY(rec_final(p, passes, fal, pit_ids, lfill, anyvol ? 1 : 0));
    if (st) {
        st->cascade_passes = passes;
        st->cascade_solves = solves;
        st->cycle_nodes = total_cycles;
    }
    return GS_OK;
}

}  // namespace gs
