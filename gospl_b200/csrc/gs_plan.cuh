// Plan (mesh + workspaces) shared by all hot-path stages.
#pragma once
#include <vector>

#include "gs_common.cuh"

struct gs_plan {
    int64_t n = 0;      // vertices
    int W = 0;          // neighbour slots stored (max FVnNb)
    int R = 0;          // receivers per vertex (flowDir)
    int flat = 0;       // flatModel
    int n_outlet = 0;
    int n_open = 0;
    double maxarea = 0;
    cudaStream_t stream = 0;
    int64_t launches = 0;
    int sm_count = 148;
    int coop_blocks = 148;               // co-resident 256-thread blocks for cooperative launches
    int coop_max_per_sm = 1;             // occupancy limit of the cooperative kernels
    int sweep_per_sm = 8;                // 128-thread blocks per SM of the ordered sweeps
    unsigned sweep_nap = 32;             // longest back-off (ns) between polls of the ordered sweeps
    unsigned long long sweep_budget_ns = 4000000000ULL;   // wall-clock budget of one dependency sweep
    int bfs_window = 0;                  // flat-distance BFS: 0 one block, w > 0 tiles, windows of w levels
    // precision form: FP32 sweeps and CG inside FP64 refinement loops
    int fp32 = 0;
    double fdepa = 0.0;                  // SPL deposition coefficient G (0: detachment-limited)
    int ed_iters = 0;                    // operator applications of the last coupled solve
    double ed_relres = 0.0;              // its final relative residual
    double* ed_buf = nullptr;            // [6][n] coupled-solve scratch
    double* ed_basis = nullptr;          // GMRES basis [31][n] and reduction scratch
    double* sed_buf = nullptr;           // [10][n] sediment-routing scratch
    uint8_t* sed_mask = nullptr;         // [5][n] sediment-routing masks
    double* sed_pit = nullptr;           // [2][n+1] per-depression scratch
    double* led = nullptr;               // [16] sediment budget of the last sedChange (GS_LED_* slots)
    double* sea_buf = nullptr;           // [12][n] marine deposition work vectors
    uint8_t* sea_u8 = nullptr;           // [4][n] marine masks and receiver bit sets
    double* sea_coef = nullptr;          // [W+1][n] bathymetry smoothing operator
    double* sea_pts = nullptr;           // coastline points, sorted copies, keys and boxes
    int64_t sea_pts_cap = 0;             // edges the coastline buffers hold
    double* hill_dprev = nullptr;        // [n] the last hillslope change (start of the next CG)
    int hill_dprev_ok = 0;
    int warm_start = 1;                  // GS_TUNE_WARM_START
    double* sea_prev = nullptr;          // [n] the last smoothed bathymetry (start of the next smoothing)
    int sea_prev_ok = 0;                 // sea_prev holds a smoothing of this plan's mesh
    size_t sea_sort_bytes = 0;           // sort scratch at the end of sea_pts
    double* led_part = nullptr;          // [5][LED_NB] block partial sums of the budget reductions
    double* sed_coef = nullptr;          // [W+1][n] lake diffusion operator (compacted to the lake cells)
    int* lake_i = nullptr;               // [W+1][n]: lake cell list, then the compact neighbour slots
    double* lake_d = nullptr;            // [3][n]: compact cell areas, right-hand side, solution
    uint8_t* lake_u8 = nullptr;          // [2][n]: compact neighbour counts, fixed rows
    int lake_on = 0;                     // lake deposits of large deep pits by non-linear diffusion (Picard)
    double lake_K = 10.0;                // its diffusivity (nlPitK)
    double lake_bias = 0.5;              // share of the deposit piled at the inlets (pitInletBias)
    int lake_nsub = 10;                  // backward-Euler sub-steps (picardSub)
    int lake_npic = 2;                   // Picard updates per sub-step (picardIts)
    double refine_tol = 1.0e-10;         // max|r| / max|b| of every refined solve
    int64_t refine_iters = 0;            // refinement passes since the last reset
    float* f32a = nullptr;               // FP32 correction / CG vectors
    float* f32b = nullptr;
    float* f32c = nullptr;
    float* f32d = nullptr;
    float* f32e = nullptr;
    double* r64 = nullptr;               // FP64 residual

    // mesh, slot-major [W][n]
    int* nbr = nullptr;          // FVnID (-1 pad)
    double* elen = nullptr;      // FVeLgt
    double* vdist = nullptr;     // FVvDist
    int8_t* rev = nullptr;       // position of i in the list of nbr(i,s)
    unsigned long long* sorder = nullptr;  // slots in ascending neighbour id, 4 bits each
    int8_t* nnb = nullptr;       // FVnNb
    double* farea = nullptr;     // FVarea (Fortran kernels)
    double* larea = nullptr;     // larea (Python side)
    uint8_t* outlet = nullptr;   // outletIDs mask
    int* outlet_ids = nullptr;
    int* open_ids = nullptr;
    uint8_t* open_mask = nullptr;
    int* gid = nullptr;          // identity ids (input order)

    // receivers workspace ([R][n]) used for the cascade rebuilds
    int* rcv = nullptr;
    double* dist = nullptr;
    double* wgt = nullptr;
    int8_t* rslot = nullptr;     // neighbour slot of each receiver (-1 = self)
    int8_t* rslot_i = nullptr;   // same for the snapshot receivers
    uint8_t* lsink = nullptr;    // live lsink
    uint8_t* sea = nullptr;      // lFill <= sea

    // DAG sweep state
    uint32_t* don_mask = nullptr;        // bit s: nbr(i,s) is a donor of i
    unsigned long long* don_k = nullptr; // 4 bits per slot: receiver index at the donor
    int* cnt = nullptr;
    int* queue = nullptr;
    unsigned* ctr = nullptr;             // [0]=head [1]=tail [2]=done [3]=status
    uint8_t* done_flag = nullptr;
    double* q = nullptr;                 // sweep values
    double* q2 = nullptr;
    double* q3 = nullptr;
    int* order = nullptr;                // topological order of the last flow sweep
    int* order_i = nullptr;              // order of the snapshot (unfilled) flow graph
    int order_i_valid = 0;
    int tie_m = 0;                       // vertices in surface tie groups of the last flow_order
    int pdir_bound = 0;                  // pdir + 1 <= pdir_bound after the last fill (0: unknown)
    unsigned long long* okey = nullptr;
    unsigned long long* okey2 = nullptr;
    unsigned* ok32 = nullptr;
    unsigned* ok32b = nullptr;
    int* oval = nullptr;
    int* oval2 = nullptr;
    int* order2 = nullptr;
    int* pos = nullptr;
    double* c = nullptr;                 // SPL coefficients [R][n]

    // pit filling
    int8_t* ledge = nullptr;
    int* parent = nullptr;
    unsigned long long* basinL = nullptr;
    int* xe_u = nullptr;                 // cross edges (basin_u, basin_v, w)
    int* xe_v = nullptr;
    double* xe_w = nullptr;
    int64_t xe_cap = 0;
    unsigned long long* xh_key = nullptr; // [xh_cap] basin-pair table of the edge deduplication (~0: empty)
    unsigned long long* xh_val = nullptr; // [xh_cap] smallest weight key of the pair
    int64_t xh_cap = 0;                   // power of two (0: no table, edges used as emitted)
    int* xd_u = nullptr;                  // [xh_cap] deduplicated edges
    int* xd_v = nullptr;
    unsigned long long* xd_w = nullptr;
    int* bfs_rows = nullptr;             // packed BFS adjacency rows, stride ((W+4)/4)*4
    int* comp = nullptr;
    int* minseed = nullptr;
    int* lab = nullptr;
    int* flagbuf = nullptr;
    int* scanbuf = nullptr;
    int* pdir = nullptr;
    int* front0 = nullptr;
    int* front1 = nullptr;
    int* spill_flag = nullptr;
    int* bestlid = nullptr;
    int npits = 0;
    double* d_scalar = nullptr;          // small device scratch [16]
    int* i_scalar = nullptr;             // small device scratch [16]
    unsigned long long* u_scalar = nullptr;
    // per pit tables (capacity n+1 rows)
    double* pit_params = nullptr;        // [P+1][3]
    int* pit_info = nullptr;             // [P+1][2]
    double* filled_lvl = nullptr;        // [P+1][5]
    double* filled_vol = nullptr;        // [P+1][5]
    double* pit_vol = nullptr;           // cascade pitVol [P+1]
    double* pit_in = nullptr;            // inflow [P+1]
    double* pit_ev = nullptr;            // eV [P+1]
    int* pit_win = nullptr;              // winning pit per spill node
    double* pit_lvl = nullptr;           // partial fill level per pit
    uint8_t* pit_state = nullptr;        // 1 overflow, 2 partial
    // segmented reductions
    int* seg_keys = nullptr;
    int* seg_vals = nullptr;
    int* seg_keys2 = nullptr;
    int* seg_vals2 = nullptr;
    int* seg_start = nullptr;
    int* seg_count = nullptr;
    int* pit_nch = nullptr;              // [n + 2] chunks of each pit (per-pit reductions)
    int* pit_chs = nullptr;              // [n + 2] first chunk item of each pit
    int* pit_item = nullptr;             // [pit_item_cap] pit of each chunk item
    double* pit_part = nullptr;          // [4 * pit_item_cap] chunk partials
    int64_t pit_item_cap = 0;
    int pit_items_max = 0;               // chunk items of the last fill, at most (the chunk kernels' grid)
    void* cub_tmp = nullptr;
    size_t cub_bytes = 0;
    void* cub_tmp2 = nullptr;            // cub scratch of work issued on side stream A
    int* pflag = nullptr;                // pit-table compaction flags / scan (main stream)
    int* pscan = nullptr;

    // side streams: A builds the unfilled-surface receivers and their order
    // while the main stream fills depressions; B runs the flat-distance BFS
    // while the main stream builds the pit tables and the first flow sweep.
    cudaStream_t side_a = nullptr;
    cudaStream_t side_b = nullptr;
    cudaEvent_t ev_fork_a = nullptr, ev_a = nullptr, ev_fork_b = nullptr, ev_b = nullptr;
    int* h_pinned = nullptr;             // pinned host words [16]
    int bfs_pending = 0;                 // flat BFS issued on side_b, not yet joined

    // flow / cascade
    double* nfa = nullptr;
    double* wf = nullptr;                // waterFilled (absolute)
    double* hl = nullptr;                // copy of h

    // landscape members (independent meshes packed into one plan; contiguous
    // vertex ranges).  One member covering every vertex unless
    // gs_plan_set_members says otherwise.
    int nmem = 1;
    std::vector<int64_t> mstart;         // host [nmem+1]
    std::vector<double> mmaxarea;        // host [nmem]: largest cell area per member
    int* vmember = nullptr;              // [n] member of each vertex
    int* pmember = nullptr;              // [n+1] member of each pit
    int nchunk = 0;                      // reduction chunks (never straddle members)
    int* chunk_lo = nullptr;             // [nchunk+1]
    int* mchunk0 = nullptr;              // [nmem+1] first chunk of each member
    double* chunk_part = nullptr;        // [nchunk]
    uint8_t* mact = nullptr;             // [nmem] member still in the cascade loop
    uint8_t* mbig = nullptr;             // [nmem] member rebuilt its receivers this pass
    uint8_t* msolve = nullptr;           // [nmem] member solves this pass
    uint8_t* mlakes = nullptr;           // [nmem] member has pit volume
    int* mflags = nullptr;               // [nmem] per-pass flags
    double* mresid = nullptr;            // [nmem]
    unsigned long long* mmax = nullptr;  // [nmem] max FAL key
    int* h_mflags = nullptr;             // pinned host [nmem]
    double* h_mresid = nullptr;          // pinned host [nmem]
    uint8_t* lsink_prev = nullptr;       // [n]

    // adjoint scratch: [R][n] edge terms, [W][n] neighbour terms, vectors
    double* adj_er = nullptr;
    double* adj_gw = nullptr;
    double* adj_nb = nullptr;
    double* adj_v0 = nullptr;
    double* adj_v1 = nullptr;
    double* adj_v2 = nullptr;
    double* adj_v3 = nullptr;
    struct gs_record* rec = nullptr;     // per-step records of the forward (adjoint replay)
    int rec_slot = -1;                   // slot the forward writes, -1 = not recording

    // diffusion
    double* dcoef = nullptr;             // [W+1][n]: diag then off-diagonals
    uint8_t* dsea = nullptr;             // sea mask the matrix was built for
    uint8_t* dsea2 = nullptr;            // sea mask of the current solve (swapped with dsea)
    uint8_t* dfix = nullptr;             // rows held fixed (flat-model outlets, zero area)
    int dvalid = 0;
    double dvalid_dt = 0, dvalid_cda = 0, dvalid_cdm = 0;
    int hill_sea = 0;                    // dsea = land/sea mask of the last hillslope input
    double* cg_r = nullptr;
    double* cg_z = nullptr;
    double* cg_p = nullptr;
    double* cg_p2 = nullptr;             // second direction buffer of the cooperative CG
    double* cg_ap = nullptr;
    double* cg_x = nullptr;
    double* cg_b = nullptr;
    double* red = nullptr;               // reduction scratch

    // optional per-kernel timing (CUDA events around launches)
    int profiling = 0;
    std::vector<const void*> prof_fn;
    std::vector<cudaEvent_t> prof_ev;    // start/stop pairs
    std::vector<int> prof_idx;           // kernel index per pair
    std::vector<int> prof_stream;        // 0 main, 1 side_a, 2 side_b per pair
};

namespace gs {

// stage entry points (host side, issue work on plan->stream)
int receivers(gs_plan* p, int nrcv, double exp, const double* elev, double sl, const int* gid,
              int* rcv, double* dist, double* wgt, int8_t* rslot);
int flow_direction(gs_plan* p, const double* h, bool down, const double* lfill,
                   const int* pit_ids, const int* flat_dirs, double sealevel, int* rcv,
                   double* dist, double* wgt, int8_t* rslot, uint8_t* lsink, uint8_t* sea);
// the part of flow_direction after the receivers (flat routing, outlets, masks)
int flow_direction_post(gs_plan* p, const double* h, bool down, const double* lfill, const int* pit_ids,
                        const int* flat_dirs, double sealevel, int* rcv, double* dist, double* wgt,
                        int8_t* rslot, uint8_t* lsink, uint8_t* sea);
// lsink / sea masks for flow_direction(..., lsink = nullptr) graphs
int sea_mask(gs_plan* p, const double* lfill, double sl, uint8_t* sea);
int sink_mask(gs_plan* p, const double* wgt, const uint8_t* sea, uint8_t* lsink);
int flow_solve(gs_plan* p, const int* rcv, const double* wgt, const int8_t* rslot,
               const double* b, double* x, int* cycle_nodes, const double* surface, const int* pdir,
               int* order);
int receivers_adjoint(gs_plan* p, const double* z, double sl, const int8_t* rslot, const double* gw, double* gself,
                      double* gnb, double* gz);
int spl_adjoint(gs_plan* p, const double* hold, const double* s, const double* fal, const double* rain,
                double k_scalar, const double* k_field, double d, double m, double dt, const int* rcv,
                const double* dist, const double* wgt, const int8_t* rslot, const int* order, const uint8_t* lsink,
                const uint8_t* sea, double* lam, double* gK, double* grain, double* gfal, double* gw_out);
// per-step records of the forward for the adjoint replay (gs_adjoint.cu)
int record_setup(gs_plan* p, int nslots);
int record_select(gs_plan* p, int slot);
void record_free(gs_plan* p);
int rec_initial(gs_plan* p, const double* h, const int* rcv, const double* wgt, const double* dist,
                const int8_t* rslot, const int* order, int order_ok, const double* q0, const uint8_t* sea);
int rec_pass_pits(gs_plan* p, int t, const uint8_t* lsink, int np1);
int rec_pass_rebuild(gs_plan* p, int t, const double* surf);
int rec_pass_solve(gs_plan* p, int t, const int* order, int order_ok, const double* x);
int rec_final(gs_plan* p, int npass, const double* fal, const int* pit, const double* lfill, int lakes);
int rec_spl(gs_plan* p, const double* s, const uint8_t* lsink);
int rec_hill(gs_plan* p, const double* h_in);
int adjoint_step(gs_plan* p, int slot, double* lam, const double* rain, double k_scalar, const double* k_field,
                 double d, double m, double dt, double sealevel, double cda, double cdm, double rtol, int max_iter,
                 double* gK, double* gU, double* grain, double* gbl);
int hillslope_adjoint(gs_plan* p, const double* h_in, double* lam, double sealevel, double cda, double cdm,
                      double dt, double rtol, int max_iter, int* iters);
int sweep_flow_adjoint(gs_plan* p, const int* rcv, const double* wgt, const int* order, const double* g, double* y);
int sweep_spl_adjoint(gs_plan* p, const int* rcv, const double* wgt, const int8_t* rslot, const double* c,
                      const int* order, const double* g, double* y);
int spl_sweep(gs_plan* p, const int* rcv, const double* c, const int8_t* rslot, const double* hold,
              double* s, int* cycle_nodes, bool reuse_order);
// check_b: a second input checked for NaN/Inf with h (the rain volume of a
// flow accumulation); a non-finite value returns GS_ENONFINITE before the
// relaxation and any sweep
int fill_elevation(gs_plan* p, const double* h, double sealevel, double ofill, double* lfill,
                   int* pit_ids, int* flat_dirs, gs_stats* st, bool defer_flats = false,
                   uint8_t* sea_out = nullptr, bool sed = false, const double* check_b = nullptr);
// joins the flat-distance BFS of the last fill (if it ran on side_b) into the
// main stream and records its level count
int fill_join(gs_plan* p, gs_stats* st);
// topological order of a flow graph: vertices by surface descending
// (flow_order), then surface ties by flat distance descending (flow_order_ties)
int flow_order(gs_plan* p, const double* surface, int* order);
// same order as flow_order(surface), built from the order of a surface that
// differs from it at few vertices (base_order = flow_order(base_surface))
int flow_order_from(gs_plan* p, const double* surface, const double* base_surface, const int* base_order,
                    int* order);
int flow_order_ties_prepare(gs_plan* p);   // after flow_order: tie groups of the surface
int flow_order_ties(gs_plan* p, const int* pdir, int* order);   // after prepare: ties by pdir
int flow_prepare(gs_plan* p, const int* rcv, const double* wgt, const int8_t* rslot, double* x, const int* order,
                 int* bad_host);
// status_host (pinned): when given, the ordered sweep's status is copied
// there asynchronously and the caller checks it after its next
// synchronisation of the plan's stream; otherwise flow_run synchronises
// A linear operator on device vectors of the plan's length, for GMRES.
struct LinOp {
    virtual int apply(const double* x, double* y) = 0;
    virtual ~LinOp() {}
};
// Restarted GMRES(30) on op x = a from the given x to |a - op x| <= tol |a|
// (at most max_applies applications); GS_EMAXITER when it stops short.
int gmres_solve(gs_plan* p, LinOp& op, const double* a, double* x, double tol, int max_applies, int* applies,
                double* relres);
int gm_axpby(gs_plan* p, int n, double a, const double* x, double b, const double* y, double* z);
// Marine flow accumulation q = (I - W^T)^-1 b over the marine receivers
// (bit sets cand over the neighbour slots, weights w), donors summed in
// ascending id, in the order of the marine surface (descending).
int sweep_marine(gs_plan* p, const unsigned short* cand, const double* w, const int* order, const double* b,
                 double* q);
int flow_run(gs_plan* p, const int* rcv, const double* wgt, const int8_t* rslot, const double* b,
             double* x, int* cycle_nodes, int* order, int ok, int* status_host);
int group_sum_by_pit(gs_plan* p, const int* pit_ids, const uint8_t* mask, const double* vals,
                     double* out, int npits);
int flow_accumulation(gs_plan* p, const double* h, const double* bl, double sealevel, double ofill,
                      double dt, double* fal, double* fill_fal, double* water, double* lfill,
                      int* pit_ids, int* flat_dirs, int* rcv_i, double* dist_i, double* wgt_i,
                      uint8_t* lsink, uint8_t* sea, gs_stats* st);
int erodep_spl(gs_plan* p, double* h, double* cum_ed, double* eb, const double* fal,
               const double* rain, double k_scalar, const double* k_field, double d, double m,
               double dt, const int* rcv_i, const double* dist_i, const double* wgt_i,
               const uint8_t* lsink, const uint8_t* sea, gs_stats* st);
int sed_change(gs_plan* p, double* h, double* cum_ed, const double* eb, const double* xyz, double sealevel,
               double ofill, double dt, double nl_pit_volume, double nl_pit_depth, double* lfill, int* pit_ids,
               int* flat_dirs, const int* rcv_i, const double* wgt_i, uint8_t* lsink, uint8_t* sea,
               double* vsed, gs_stats* st);
int sed_budget(gs_plan* p, double* out16);
int sea_change(gs_plan* p, double* h, double* cum_ed, double* eb, const double* xyz, const double* box,
               const int* edges, int64_t nedge, double sealevel, double ofill, double dt, double clinslp,
               double offshore, double nlk, double gmar, const double* lfill, const double* vsed,
               const uint8_t* sea, gs_stats* st);
int picard_diffuse(gs_plan* p, const uint8_t* lmask, const double* zb, double* hcur, double K, double dt,
                   double* cd, double* hstart);
// guess: start of the free rows (nullptr: the right-hand side)
int diffusion_solve_on(gs_plan* p, int m, const int* nbr, const int8_t* nnb, const double* farea, const uint8_t* fix,
                       int flat, const uint8_t* outlet, const double* coef, const double* rhs, double* x, double rtol,
                       int max_iter, int* iters, const double* guess = nullptr, double* worst = nullptr);
int hillslope(gs_plan* p, double* h, double* cum_ed, double* eb, double sealevel, double cda,
              double cdm, double dt, double rtol, int max_iter, gs_stats* st);
int apply_forces(gs_plan* p, double* h, const double* rain, const double* upsub, double dt,
                 double sealevel, double* bl);
int output_fields(gs_plan* p, const double* h, const double* cum_ed, const double* eb, const double* water_filled,
                  const double* fill_fa, const double* fa, const double* vsed, const double* upsub,
                  const double* rain, const uint8_t* sea, float* out);

void prof_begin(gs_plan* p, const void* fn, cudaEvent_t* stop);
int coop_occupancy(int* per_sm);
__global__ void k_cg_coop32(int n, const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                            const double* __restrict__ coef, const double* __restrict__ farea,
                            const uint8_t* __restrict__ fix, const double* __restrict__ rhs, float* x, float* r,
                            float* z, float* pp, float* ap, double* part, double rtol, int max_iter, int* it_out,
                            double* res_out);
__global__ void k_cg_coop(int n, const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                          const double* __restrict__ coef, const double* __restrict__ farea,
                          const uint8_t* __restrict__ fix, const double* __restrict__ x0, double* x, double* b,
                          double* r, double* z, double* p0, double* p1, double* ap, double* part, double rtol,
                          int max_iter, int* it_out, double* res_out, const double* guess);
int set_members(gs_plan* p, int nmem, const int64_t* start, const double* maxarea);
int plan_tune(gs_plan* p, int knob, int value);
int precision_buffers(gs_plan* p);
int build_donors(gs_plan* p, const int* rcv, const double* wgt, const int8_t* rslot);
int spl_order(gs_plan* p);
int sweep_flow_rhs(gs_plan* p, const double* wgt, const int* order, const double* b, double* x);
int sweep_spl_rhs(gs_plan* p, const int* rcv, const double* c, const int* order2, const double* rhs, double* x);
int flow_refine32(gs_plan* p, const double* wgt, const double* b, double* x, const int* order);
int spl_refine32(gs_plan* p, const int* rcv, const double* c, const double* hold, double* x, const int* order2);
int plan_tuning(const gs_plan* p, int knob);
void free_members(gs_plan* p);

// issues the plan's work on another stream (and cub scratch) for its scope
struct StreamSwap {
    gs_plan* p;
    cudaStream_t s0;
    void* c0;
    StreamSwap(gs_plan* p_, cudaStream_t s, void* cub) : p(p_), s0(p_->stream), c0(p_->cub_tmp) {
        p->stream = s;
        if (cub) p->cub_tmp = cub;
    }
    ~StreamSwap() {
        p->stream = s0;
        p->cub_tmp = c0;
    }
};

template <class K, class... A>
inline void launch(gs_plan* p, K kernel, int grid, int block, A... args) {
    cudaEvent_t stop = nullptr;
    if (p->profiling) prof_begin(p, (const void*)kernel, &stop);
    kernel<<<grid, block, 0, p->stream>>>(args...);
    if (stop) cudaEventRecord(stop, p->stream);
    p->launches++;
}

}  // namespace gs
