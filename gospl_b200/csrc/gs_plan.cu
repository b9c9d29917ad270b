// Plan creation: upload of the finite-volume mesh in slot-major layout and
// allocation of every workspace the hot path needs (nothing is allocated
// per step).
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "gs_plan.cuh"

namespace gs {

template <class T>
static int dalloc(T** ptr, size_t count) {
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)ptr, sizeof(T) * count);
    if (e != cudaSuccess) {
        set_error(GS_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        return GS_ENOMEM;
    }
    return GS_OK;
}

struct ScanMax {
    __device__ __forceinline__ int operator()(int a, int b) const { return a > b ? a : b; }
};

template <class T>
static int upload(T** ptr, const std::vector<T>& h) {
    GS_TRY(dalloc(ptr, h.size()));
    if (!h.empty()) GS_CUDA(cudaMemcpy(*ptr, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
    return GS_OK;
}

static void plan_free(gs_plan* p) {
    void* ptrs[] = {p->nbr, p->elen, p->vdist, p->rev, p->sorder, p->nnb, p->farea, p->larea, p->outlet,
                    p->outlet_ids, p->open_ids, p->open_mask, p->gid, p->rcv, p->dist, p->wgt, p->rslot,
                    p->rslot_i, p->lsink, p->sea, p->don_mask, p->don_k, p->cnt, p->queue, p->ctr,
                    p->done_flag, p->q, p->q2, p->q3, p->order, p->order2, p->pos, p->order_i, p->okey, p->okey2, p->ok32, p->ok32b, p->oval, p->oval2, p->c, p->ledge, p->parent, p->basinL, p->xe_u,
                    p->xe_v, p->xe_w, p->bfs_rows, p->comp, p->minseed, p->lab, p->flagbuf, p->scanbuf, p->pdir,
                    p->front0, p->front1, p->spill_flag, p->bestlid, p->d_scalar, p->i_scalar,
                    p->u_scalar, p->pit_params, p->pit_info, p->filled_lvl, p->filled_vol, p->pit_vol,
                    p->pit_in, p->pit_ev, p->pit_win, p->pit_lvl, p->pit_state, p->seg_keys, p->seg_vals,
                    p->seg_keys2, p->seg_vals2, p->seg_start, p->seg_count, p->pit_nch, p->pit_chs, p->pit_item, p->pit_part, p->cub_tmp, p->nfa, p->wf,
                    p->hl, p->dcoef, p->dsea, p->dsea2, p->dfix, p->cg_r, p->cg_z, p->cg_p, p->cg_p2, p->cg_ap, p->cg_x, p->cg_b,
                    p->red, p->cub_tmp2, p->pflag, p->pscan, p->f32a, p->f32b, p->f32c, p->f32d, p->f32e, p->r64, p->ed_buf,
                    p->sed_buf, p->sed_mask, p->ed_basis, p->sed_pit, p->led, p->led_part, p->sea_buf, p->sea_u8, p->sea_coef, p->sea_pts, p->sea_prev, p->hill_dprev, p->xh_key, p->xh_val, p->xd_u, p->xd_v, p->xd_w, p->sed_coef, p->lake_i, p->lake_d, p->lake_u8};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    cudaEvent_t evs[] = {p->ev_fork_a, p->ev_a, p->ev_fork_b, p->ev_b};
    for (cudaEvent_t e : evs)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : p->prof_ev)
        if (e) cudaEventDestroy(e);
    p->prof_ev.clear();
    free_members(p);
    record_free(p);
    if (p->side_a) cudaStreamDestroy(p->side_a);
    if (p->side_b) cudaStreamDestroy(p->side_b);
    if (p->h_pinned) cudaFreeHost(p->h_pinned);
}

int plan_create(int64_t nb, const int32_t* nnb, const int32_t* ngb, const double* elgt, const double* vdist,
                const double* farea, const double* larea, const int32_t* outlet_ids, int64_t n_outlet,
                const int32_t* open_ids, int64_t n_open, int flat, int flow_dir, gs_plan** out) {
    if (nb < 0 || nb > (int64_t)0x7fffffff - 64 || flow_dir < 1 || flow_dir > MAXR || !out) {
        set_error(GS_EINVAL, "gs_plan_create: bad size or flow_dir");
        return GS_EINVAL;
    }
    if (nb > 0 && (!nnb || !ngb || !elgt || !vdist || !farea || !larea)) {
        set_error(GS_EINVAL, "gs_plan_create: null mesh array");
        return GS_EINVAL;
    }
    const int n = (int)nb;
    int W = 1;
    for (int i = 0; i < n; i++) {
        if (nnb[i] < 0 || nnb[i] > MAXW) {
            set_error(GS_EINVAL, "gs_plan_create: FVnNb outside 0..12");
            return GS_EINVAL;
        }
        W = std::max(W, (int)nnb[i]);
    }
    for (int64_t t = 0; t < n_outlet; t++)
        if (outlet_ids[t] < 0 || outlet_ids[t] >= n) {
            set_error(GS_EINVAL, "gs_plan_create: outlet id out of range");
            return GS_EINVAL;
        }
    for (int64_t t = 0; t < n_open; t++)
        if (open_ids[t] < 0 || open_ids[t] >= n) {
            set_error(GS_EINVAL, "gs_plan_create: open-edge id out of range");
            return GS_EINVAL;
        }
    gs_plan* p = new gs_plan();
    p->n = n;
    p->W = W;
    p->R = flow_dir;
    p->flat = flat ? 1 : 0;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&p->sm_count, cudaDevAttrMultiProcessorCount, dev);
    {
        // cooperative kernels: up to four co-resident 256-thread blocks per SM
        // (checked against occupancy), enough warps to hide the gather latency
        // of the edge-parallel rounds
        int per_sm = 0;
        if (coop_occupancy(&per_sm) == 0 && per_sm > 0) {
            p->coop_max_per_sm = per_sm;
            p->coop_blocks = p->sm_count * std::min(per_sm, 4);
        } else {
            p->coop_max_per_sm = 1;
            p->coop_blocks = p->sm_count;
        }
    }

    std::vector<int> h_nbr((size_t)W * n, -1);
    std::vector<double> h_elen((size_t)W * n, 0.0), h_vd((size_t)W * n, 0.0);
    std::vector<int8_t> h_rev((size_t)W * n, -1), h_nnb(n);
    std::vector<unsigned long long> h_sorder(n, ~0ULL);
    for (int i = 0; i < n; i++) {
        h_nnb[i] = (int8_t)nnb[i];
        for (int s = 0; s < nnb[i]; s++) {
            h_nbr[(size_t)s * n + i] = ngb[(size_t)i * 12 + s];
            h_elen[(size_t)s * n + i] = elgt[(size_t)i * 12 + s];
            h_vd[(size_t)s * n + i] = vdist[(size_t)i * 12 + s];
        }
    }
    for (int i = 0; i < n; i++) {
        int slots[12], cnt = 0;
        for (int s = 0; s < nnb[i]; s++) {
            int j = ngb[(size_t)i * 12 + s];
            if (j < 0 || j >= n) continue;
            slots[cnt++] = s;
            for (int t = 0; t < nnb[j]; t++)
                if (ngb[(size_t)j * 12 + t] == i) { h_rev[(size_t)s * n + i] = (int8_t)t; break; }
        }
        std::sort(slots, slots + cnt, [&](int a, int b) { return ngb[(size_t)i * 12 + a] < ngb[(size_t)i * 12 + b]; });
        unsigned long long o = ~0ULL;
        for (int q = cnt - 1; q >= 0; q--) o = (o << 4) | (unsigned long long)slots[q];
        h_sorder[i] = o;
    }
    std::vector<uint8_t> h_out(n, 0), h_open(n, 0);
    std::vector<int> h_oid(outlet_ids, outlet_ids + n_outlet), h_open_ids(open_ids, open_ids + n_open);
    for (int t : h_oid) h_out[t] = 1;
    for (int t : h_open_ids) h_open[t] = 1;
    std::vector<int> h_gid(n);
    for (int i = 0; i < n; i++) h_gid[i] = i;
    double maxarea = 0.0;
    for (int i = 0; i < n; i++) maxarea = (i == 0 || larea[i] > maxarea) ? larea[i] : maxarea;
    p->maxarea = maxarea;
    p->n_outlet = (int)n_outlet;
    p->n_open = (int)n_open;

    int st = GS_OK;
#define TRYP(x)                   \
    do {                          \
        st = (x);                 \
        if (st != GS_OK) goto fail; \
    } while (0)
    TRYP(upload(&p->nbr, h_nbr));
    TRYP(upload(&p->elen, h_elen));
    TRYP(upload(&p->vdist, h_vd));
    TRYP(upload(&p->rev, h_rev));
    TRYP(upload(&p->sorder, h_sorder));
    TRYP(upload(&p->nnb, h_nnb));
    TRYP(upload(&p->farea, std::vector<double>(farea, farea + n)));
    TRYP(upload(&p->larea, std::vector<double>(larea, larea + n)));
    TRYP(upload(&p->outlet, h_out));
    {
        std::vector<uint8_t> h_fix(n);
        for (int i = 0; i < n; i++) h_fix[i] = ((flat && h_out[i]) || !(farea[i] > 0)) ? 1 : 0;
        TRYP(upload(&p->dfix, h_fix));
    }
    TRYP(upload(&p->outlet_ids, h_oid));
    TRYP(upload(&p->open_ids, h_open_ids));
    TRYP(upload(&p->open_mask, h_open));
    TRYP(upload(&p->gid, h_gid));
    {
        const size_t N = (size_t)n, R = (size_t)p->R, N1 = N + 1;
        TRYP(dalloc(&p->rcv, R * N));
        TRYP(dalloc(&p->dist, R * N));
        TRYP(dalloc(&p->wgt, R * N));
        TRYP(dalloc(&p->rslot, R * N));
        TRYP(dalloc(&p->rslot_i, R * N));
        TRYP(dalloc(&p->c, R * N));
        TRYP(dalloc(&p->lsink, N));
        TRYP(dalloc(&p->sea, N));
        TRYP(dalloc(&p->don_mask, N));
        TRYP(dalloc(&p->don_k, N));
        TRYP(dalloc(&p->cnt, N));
        TRYP(dalloc(&p->queue, N));
        TRYP(dalloc(&p->ctr, 16));
        TRYP(dalloc(&p->done_flag, N));
        TRYP(dalloc(&p->q, N));
        TRYP(dalloc(&p->q2, N));
        TRYP(dalloc(&p->q3, N));
        TRYP(dalloc(&p->order, N));
        TRYP(dalloc(&p->order_i, N));
        TRYP(dalloc(&p->okey, N));
        TRYP(dalloc(&p->okey2, N));
        TRYP(dalloc(&p->ok32, N));
        TRYP(dalloc(&p->ok32b, N));
        TRYP(dalloc(&p->oval, N));
        TRYP(dalloc(&p->oval2, N));
        TRYP(dalloc(&p->order2, N));
        TRYP(dalloc(&p->pos, N));
        TRYP(dalloc(&p->ledge, N));
        TRYP(dalloc(&p->parent, N));
        TRYP(dalloc(&p->basinL, N));
        p->xe_cap = (int64_t)W * N;
        TRYP(dalloc(&p->xe_u, (size_t)p->xe_cap));
        TRYP(dalloc(&p->xe_v, (size_t)p->xe_cap));
        TRYP(dalloc(&p->xe_w, (size_t)p->xe_cap));
        TRYP(dalloc(&p->bfs_rows, (size_t)(((W + 1 + 3) / 4) * 4) * N));
        TRYP(dalloc(&p->comp, N));
        TRYP(dalloc(&p->minseed, N));
        TRYP(dalloc(&p->lab, N));
        TRYP(dalloc(&p->flagbuf, N1));
        TRYP(dalloc(&p->scanbuf, N1));
        TRYP(dalloc(&p->pdir, N));
        TRYP(dalloc(&p->front0, N));
        TRYP(dalloc(&p->front1, N));
        TRYP(dalloc(&p->spill_flag, N));
        TRYP(dalloc(&p->bestlid, N1));
        TRYP(dalloc(&p->d_scalar, 16));
        TRYP(dalloc(&p->i_scalar, 16));
        TRYP(dalloc(&p->u_scalar, 16));
        TRYP(dalloc(&p->pit_params, 3 * N1));
        TRYP(dalloc(&p->pit_info, 2 * N1));
        TRYP(dalloc(&p->filled_lvl, 5 * N1));
        TRYP(dalloc(&p->filled_vol, 5 * N1));
        TRYP(dalloc(&p->pit_vol, N1));
        TRYP(dalloc(&p->pit_in, N1));
        TRYP(dalloc(&p->pit_ev, N1));
        TRYP(dalloc(&p->pit_win, N));
        TRYP(dalloc(&p->pit_lvl, N1));
        TRYP(dalloc(&p->pit_state, N1));
        TRYP(dalloc(&p->seg_keys, N1));
        TRYP(dalloc(&p->seg_vals, N1));
        TRYP(dalloc(&p->seg_keys2, N1));
        TRYP(dalloc(&p->seg_vals2, N1));
        TRYP(dalloc(&p->seg_start, N1 + 1));
        TRYP(dalloc(&p->seg_count, N1 + 1));
        TRYP(dalloc(&p->nfa, N));
        TRYP(dalloc(&p->wf, N));
        TRYP(dalloc(&p->hl, N));
        TRYP(dalloc(&p->dcoef, (size_t)(W + 1) * N));
        TRYP(dalloc(&p->dsea, N));
        TRYP(dalloc(&p->dsea2, N));
        TRYP(dalloc(&p->cg_r, N));
        TRYP(dalloc(&p->cg_z, N));
        TRYP(dalloc(&p->cg_p, N));
        TRYP(dalloc(&p->cg_ap, N));
        TRYP(dalloc(&p->cg_x, N));
        TRYP(dalloc(&p->cg_b, N));
        TRYP(dalloc(&p->red, 8192));
        size_t b1 = 0, b2 = 0;
        cub::DeviceRadixSort::SortPairs((void*)nullptr, b1, (const int*)nullptr, (int*)nullptr,
                                        (const int*)nullptr, (int*)nullptr, (int)N1, 0, 32);
        size_t b3 = 0;
        cub::DeviceRadixSort::SortPairs((void*)nullptr, b3, (const unsigned long long*)nullptr,
                                        (unsigned long long*)nullptr, (const int*)nullptr, (int*)nullptr, (int)N1,
                                        0, 64);
        b1 = std::max(b1, b3);
        cub::DeviceScan::ExclusiveSum((void*)nullptr, b2, (const int*)nullptr, (int*)nullptr, (int)N1 + 1);
        size_t b4 = 0;
        cub::DeviceScan::InclusiveScan((void*)nullptr, b4, (const int*)nullptr, (int*)nullptr, ScanMax(), (int)N1);
        p->cub_bytes = std::max(std::max(b1, b2), b4) + 256;
        TRYP(dalloc((char**)&p->cub_tmp, p->cub_bytes));
        TRYP(dalloc((char**)&p->cub_tmp2, p->cub_bytes));
        TRYP(dalloc(&p->pflag, N1));
        TRYP(dalloc(&p->pscan, N1));
    }
    {
        cudaError_t e = cudaStreamCreateWithFlags(&p->side_a, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->side_b, cudaStreamNonBlocking);
        cudaEvent_t* evs[] = {&p->ev_fork_a, &p->ev_a, &p->ev_fork_b, &p->ev_b};
        for (cudaEvent_t* ev : evs)
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMallocHost((void**)&p->h_pinned, sizeof(int) * 16);
        if (e != cudaSuccess) {
            set_error(GS_ECUDA, std::string("plan streams: ") + cudaGetErrorString(e));
            st = GS_ECUDA;
            goto fail;
        }
    }
#undef TRYP
    {
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            set_error(GS_ECUDA, std::string("plan upload: ") + cudaGetErrorString(e));
            st = GS_ECUDA;
            goto fail;
        }
    }
    {
        const int64_t st0[2] = {0, (int64_t)n};
        const double ma0[1] = {maxarea};
        int r = set_members(p, 1, st0, ma0);
        if (r != GS_OK) {
            st = r;
            goto fail;
        }
    }
    *out = p;
    return GS_OK;
fail:
    plan_free(p);
    delete p;
    return st;
}

void free_members(gs_plan* p) {
    void* ptrs[] = {p->vmember, p->pmember, p->chunk_lo, p->mchunk0, p->chunk_part, p->mact, p->mbig,
                    p->msolve, p->mlakes, p->mflags, p->mresid, p->mmax, p->lsink_prev};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    if (p->h_mflags) cudaFreeHost(p->h_mflags);
    if (p->h_mresid) cudaFreeHost(p->h_mresid);
    p->vmember = p->pmember = p->chunk_lo = p->mchunk0 = nullptr;
    p->chunk_part = nullptr;
    p->mact = p->mbig = p->msolve = p->mlakes = nullptr;
    p->mflags = nullptr;
    p->mresid = nullptr;
    p->mmax = nullptr;
    p->lsink_prev = nullptr;
    p->h_mflags = nullptr;
    p->h_mresid = nullptr;
}

__global__ void k_fill_member(int lo, int hi, int m, int* vmember) {
    int i = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (i < hi) vmember[i] = m;
}

// Members are contiguous vertex ranges [start[m], start[m+1]); every
// reduction over a member runs over chunks of at most 8192 of its vertices
// in a fixed order.
int set_members(gs_plan* p, int nmem, const int64_t* start, const double* maxarea) {
    const int64_t n = p->n;
    if (nmem < 1 || !start || !maxarea || start[0] != 0 || start[nmem] != n) {
        set_error(GS_EINVAL, "members: need start[0] = 0, start[nmem] = nb and nmem >= 1");
        return GS_EINVAL;
    }
    for (int m = 0; m < nmem && n > 0; m++)
        if (start[m + 1] <= start[m]) {
            set_error(GS_EINVAL, "members: every member needs at least one vertex");
            return GS_EINVAL;
        }
    free_members(p);
    p->nmem = nmem;
    p->mstart.assign(start, start + nmem + 1);
    p->mmaxarea.assign(maxarea, maxarea + nmem);
    const int64_t CH = 8192;
    std::vector<int> lo, m0;
    for (int m = 0; m < nmem; m++) {
        m0.push_back((int)lo.size());
        for (int64_t a = start[m]; a < start[m + 1]; a += CH) lo.push_back((int)a);
    }
    m0.push_back((int)lo.size());
    p->nchunk = (int)lo.size();
    lo.push_back((int)n);
    const size_t N = (size_t)std::max<int64_t>(n, 1);
    GS_TRY(dalloc(&p->vmember, N));
    GS_TRY(dalloc(&p->pmember, N + 1));
    GS_TRY(upload(&p->chunk_lo, lo));
    GS_TRY(upload(&p->mchunk0, m0));
    GS_TRY(dalloc(&p->chunk_part, (size_t)p->nchunk + 1));
    GS_TRY(dalloc(&p->mact, (size_t)nmem));
    GS_TRY(dalloc(&p->mbig, (size_t)nmem));
    GS_TRY(dalloc(&p->msolve, (size_t)nmem));
    GS_TRY(dalloc(&p->mlakes, (size_t)nmem));
    GS_TRY(dalloc(&p->mflags, (size_t)nmem));
    GS_TRY(dalloc(&p->mresid, (size_t)nmem));
    GS_TRY(dalloc(&p->mmax, (size_t)nmem));
    GS_TRY(dalloc(&p->lsink_prev, N));
    GS_CUDA(cudaMallocHost((void**)&p->h_mflags, sizeof(int) * nmem));
    GS_CUDA(cudaMallocHost((void**)&p->h_mresid, sizeof(double) * nmem));
    for (int m = 0; m < nmem; m++) {
        const int a = (int)start[m], b = (int)start[m + 1];
        if (b > a) k_fill_member<<<(b - a + 255) / 256, 256, 0, p->stream>>>(a, b, m, p->vmember);
    }
    GS_CUDA(cudaGetLastError());
    GS_CUDA(cudaStreamSynchronize(p->stream));
    return GS_OK;
}

// launch-shape knobs (GS_TUNE_*): blocks per SM of the ordered sweeps
// (1..32) and of the cooperative kernels (1..their occupancy limit)
int plan_tune(gs_plan* p, int knob, int value) {
    if (knob == GS_TUNE_SWEEP_BLOCKS) {
        if (value < 1 || value > 32) {
            set_error(GS_EINVAL, "tune: sweep blocks per SM must be in 1..32");
            return GS_EINVAL;
        }
        p->sweep_per_sm = value;
        return GS_OK;
    }
    if (knob == GS_TUNE_COOP_BLOCKS) {
        if (value < 1 || value > p->coop_max_per_sm) {
            set_error(GS_EINVAL, "tune: cooperative blocks per SM must be in 1.." +
                                     std::to_string(p->coop_max_per_sm) + " (co-residency limit)");
            return GS_EINVAL;
        }
        p->coop_blocks = p->sm_count * value;
        return GS_OK;
    }
    if (knob == GS_TUNE_SWEEP_NAP) {
        if (value < 0 || value > 1024) {
            set_error(GS_EINVAL, "tune: sweep back-off must be in 0..1024 ns");
            return GS_EINVAL;
        }
        p->sweep_nap = (unsigned)value;
        return GS_OK;
    }
    if (knob == GS_TUNE_WARM_START) {
        if (value != 0 && value != 1) {
            set_error(GS_EINVAL, "tune: warm start must be 0 or 1");
            return GS_EINVAL;
        }
        p->warm_start = value;
        p->hill_dprev_ok = 0;
        p->sea_prev_ok = 0;
        return GS_OK;
    }
    if (knob == GS_TUNE_FLAT_BFS) {
        if (value < 0 || value > 4096) {
            set_error(GS_EINVAL, "tune: flat BFS must be 0 (one block) or a window of 1..4096 levels (tiles)");
            return GS_EINVAL;
        }
        p->bfs_window = value;
        return GS_OK;
    }
    if (knob == GS_TUNE_SWEEP_BUDGET) {
        if (value < 1 || value > 60000000) {
            set_error(GS_EINVAL, "tune: sweep time budget must be in 1..60000000 us");
            return GS_EINVAL;
        }
        p->sweep_budget_ns = (unsigned long long)value * 1000ULL;
        return GS_OK;
    }
    set_error(GS_EINVAL, "tune: unknown knob");
    return GS_EINVAL;
}

int plan_tuning(const gs_plan* p, int knob) {
    if (knob == GS_TUNE_SWEEP_BLOCKS) return p->sweep_per_sm;
    if (knob == GS_TUNE_COOP_BLOCKS) return p->coop_blocks / std::max(p->sm_count, 1);
    if (knob == GS_TUNE_COOP_BLOCKS + 1) return p->coop_max_per_sm;
    if (knob == GS_TUNE_SWEEP_NAP) return (int)p->sweep_nap;
    if (knob == GS_TUNE_SWEEP_BUDGET) return (int)(p->sweep_budget_ns / 1000ULL);
    if (knob == GS_TUNE_FLAT_BFS) return p->bfs_window;
    if (knob == GS_TUNE_WARM_START) return p->warm_start;
    if (knob == GS_TUNE_REFINE_PASSES) return (int)std::min<int64_t>(p->refine_iters, 0x7fffffff);
    return -1;
}

int plan_destroy(gs_plan* p) {
    if (!p) return GS_OK;
    plan_free(p);
    delete p;
    return GS_OK;
}

}  // namespace gs
