// Depression filling: PITFill.fillElevation(sed=False) (pitfilling.py:849-903).
//
// Filled surface.  On one GPU the reference's three Barnes phases (per-tile
// Priority-Flood fill_tile, label-graph flood fill_edges, fill_depressions)
// reduce to the plain Priority-Flood fill: the minimax over paths to the seed
// set of the highest shifted elevation along the path.  (Each watershed label
// is created by a seed that drains to label 0, so the label-graph level of a
// watershed never exceeds the fill of its cells and fill_depressions keeps the
// flood values.)  The GPU computes that minimax without a heap:
//   1. steepest non-ascending descent (lexicographic (z, id)) links every cell
//      to a root: a seed or a local minimum (a basin);
//   2. for each pair of adjacent basins the spill height is max(z_u, z_v);
//   3. basin levels L(b) = minimax over basin-graph paths to a seed basin,
//      relaxed with atomicMin until stable;
//   4. fill = max(z, L(basin)).
// Only comparisons are involved, so the result is bit-identical to the
// reference's heap-ordered flood.  Seeds and exclusions follow edge_tile
// (functions.F90:2036-2080) on z - level; cells at or below the level keep
// their elevation (fill_depressions, 2290-2329) and open-sea cells are reset
// (pitfilling.py:689-693).
//
// Pit bookkeeping follows _pitInformation (pitfilling.py:704-847):
// label_pits (equal-fill components holding a cell with no lower neighbour,
// numbered by their smallest seed id) by union-find; pits_cons renumbering;
// spill selection by smallest id; fill_dir / nghb_dir hop distances by
// level-synchronous BFS; the (distance, id) flat receiver pick; pit volumes,
// depths and depth-volume curves (_getPitParams, getpitvol) by deterministic
// segmented reductions over pit-sorted cells.
#include <cub/cub.cuh>

#include <cfloat>
#include <climits>
#include <cstring>
#include <vector>

#include <cooperative_groups.h>

#include "gs_plan.cuh"

namespace cg = cooperative_groups;

namespace gs {

__device__ __forceinline__ int agg_append(int* cnt) {
    cg::coalesced_group g = cg::coalesced_threads();
    int base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(cnt, (int)g.size());
    return g.shfl(base, 0) + (int)g.thread_rank();
}

enum { D_MINH = 0, D_LEVEL = 1 };
enum { I_CHANGED = 0, I_NEXT = 1, I_XRAW = 2, I_XDEDUP = 3, I_NONFINITE = 13 };

// --------------------------------------------------------------------------
// reductions
// --------------------------------------------------------------------------
__global__ void k_min_key(int n, const double* __restrict__ x, unsigned long long* out) {
    unsigned long long best = ~0ULL;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        unsigned long long k = dkey(x[i]);
        best = k < best ? k : best;
    }
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long v = __shfl_xor_sync(0xffffffffu, best, o);
        best = v < best ? v : best;
    }
    if ((threadIdx.x & 31) == 0) atomicMin(out, best);
}

__global__ void k_level(const unsigned long long* minkey, int sphere, double sealevel, double ofill,
                        double* dsc) {
    double minh = dkey_inv(*minkey);
    if (sphere) minh += 1.0e-3;
    double b = sealevel + ofill;
    dsc[D_MINH] = minh;
    dsc[D_LEVEL] = (b > minh) ? b : minh;   // Python max(minh, b)
}

// --------------------------------------------------------------------------
// filled surface
// --------------------------------------------------------------------------
__global__ void k_classify(int n, const double* __restrict__ h, const double* __restrict__ dsc,
                           const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                           const uint8_t* __restrict__ outlet, int8_t* ledge) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const double level = dsc[D_LEVEL];
    const double hs = h[c] - level;
    int8_t e = -1;
    if (hs < 0.0) {
        bool ge = false;
        for (int s = 0; s < nnb[c]; s++) {
            int j = nbr[(size_t)s * n + c];
            if (j >= 0 && h[j] - level >= 0.0) { ge = true; break; }
        }
        e = ge ? (outlet[c] ? 2 : 0) : -2;
    } else if (outlet[c]) {
        e = 2;
    }
    ledge[c] = e;
}

__global__ void k_descend(int n, const double* __restrict__ h, const double* __restrict__ dsc,
                          const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                          const int8_t* __restrict__ ledge, int* parent) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    int8_t e = ledge[c];
    if (e != -1) { parent[c] = c; return; }      // seeds, excluded cells: roots
    const double level = dsc[D_LEVEL];
    double bz = h[c] - level;
    int best = c;
    for (int s = 0; s < nnb[c]; s++) {
        int j = nbr[(size_t)s * n + c];
        if (j < 0 || ledge[j] == -2) continue;
        double z = h[j] - level;
        if (z < bz || (z == bz && j < best)) { bz = z; best = j; }
    }
    parent[c] = best;
}

// Pointer jumping towards the basin roots, up to JUMP_HOPS hops per vertex
// and launch.  Other threads shorten the same chains concurrently; every
// parent value ever stored is an ancestor on the vertex's descent path, so
// reading a stale or a fresh value are both valid steps.  *changed is set
// while some vertex has not reached its root.
constexpr int JUMP_HOPS = 16;
__global__ void k_jump(int n, int* parent, int* changed) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int p0 = parent[c];
    int p = p0;
    int hop = 0;
    for (; hop < JUMP_HOPS; hop++) {
        int pp = ld_relaxed_s32(parent + p);
        if (pp == p) break;
        p = pp;
    }
    if (p != p0) parent[c] = p;
    if (hop == JUMP_HOPS) *changed = 1;
}

__global__ void k_basin_init(int n, const int* __restrict__ parent, const int8_t* __restrict__ ledge,
                             unsigned long long* L) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    if (parent[c] == c) L[c] = (ledge[c] >= 0) ? dkey(-INFINITY) : ~0ULL;
}

__global__ void k_cross_edges(int n, const double* __restrict__ h, const double* __restrict__ dsc,
                              const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                              const int8_t* __restrict__ ledge, const int* __restrict__ root,
                              int* xu, int* xv, double* xw, int* count, int64_t cap) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    if (ledge[c] == -2) return;
    const int rc = root[c];
    // a seed basin keeps level -inf: no edge can lower it
    if (ledge[rc] >= 0) return;
    const double level = dsc[D_LEVEL];
    const double zc = h[c] - level;
    // one edge per distinct neighbouring basin, with the smallest pass height
    // (parallel edges of larger weight can never lower a level further)
    int rb[MAXW];
    double wb[MAXW];
    int nb_ = 0;
    for (int s = 0; s < nnb[c]; s++) {
        int j = nbr[(size_t)s * n + c];
        if (j < 0 || ledge[j] == -2) continue;
        int rj = root[j];
        if (rj == rc) continue;
        double zj = h[j] - level;
        double w = zc > zj ? zc : zj;
        int q = 0;
        while (q < nb_ && rb[q] != rj) q++;
        if (q == nb_) {
            rb[nb_] = rj;
            wb[nb_] = w;
            nb_++;
        } else if (w < wb[q]) {
            wb[q] = w;
        }
    }
    for (int q = 0; q < nb_; q++) {
        int pos = agg_append(count);
        if (pos < cap) {
            xu[pos] = rc;
            xv[pos] = rb[q];
            xw[pos] = wb[q];
        }
    }
}

__global__ void k_fill_final(int n, const double* __restrict__ h, const double* __restrict__ dsc,
                             double sealevel, const int8_t* __restrict__ ledge,
                             const int* __restrict__ root, const unsigned long long* __restrict__ L,
                             double* lfill) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const double level = dsc[D_LEVEL];
    const double hs = h[c] - level;
    double f = hs;
    if (ledge[c] != -2) {
        unsigned long long k = L[root[c]];
        if (k != ~0ULL) {
            double lv = dkey_inv(k);
            f = lv > hs ? lv : hs;
        }
    }
    double out = (hs > 0.0) ? f : hs;          // fill_depressions: dem > lvl only
    if (out < sealevel - level) out = hs;      // open sea stays unfilled
    lfill[c] = out + level;
}

// --------------------------------------------------------------------------
// label_pits by union-find
// --------------------------------------------------------------------------
__device__ int uf_root(int* comp, int x) {
    for (int it = 0; it < 1 << 20; it++) {
        int p = ((volatile int*)comp)[x];
        if (p == x) return x;
        int gp = ((volatile int*)comp)[p];
        if (gp != p) atomicCAS(&comp[x], p, gp);
        x = p;
    }
    return x;
}

__global__ void k_fill_int(int n, int* a, int v) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

// union-find start: every cell above sea level points to its smallest-id
// equal-fill neighbour (or itself), so the linking pass starts from short
// chains instead of singletons
__global__ void k_uf_init(int n, const double* __restrict__ f, double sl, const int* __restrict__ nbr,
                          const int8_t* __restrict__ nnb, int* comp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int best = i;
    const double fi = f[i];
    if (fi > sl) {
        for (int s = 0; s < nnb[i]; s++) {
            int j = nbr[(size_t)s * n + i];
            if (j >= 0 && j < best && f[j] == fi) best = j;
        }
    }
    comp[i] = best;
}

__global__ void k_uf_link(int n, const double* __restrict__ f, double sl, const int* __restrict__ nbr,
                          const int8_t* __restrict__ nnb, int* comp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double fi = f[i];
    if (!(fi > sl)) return;
    for (int s = 0; s < nnb[i]; s++) {
        int j = nbr[(size_t)s * n + i];
        if (j < 0 || j > i || f[j] != fi) continue;
        for (int it = 0; it < 1 << 20; it++) {
            int a = uf_root(comp, i), b = uf_root(comp, j);
            if (a == b) break;
            if (a < b) { int t = a; a = b; b = t; }
            if (atomicCAS(&comp[a], a, b) == a) break;
        }
    }
}

__global__ void k_uf_flatten(int n, int* comp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) comp[i] = uf_root(comp, i);
}

__global__ void k_minseed(int n, const double* __restrict__ f, double sl, const int* __restrict__ nbr,
                          const int8_t* __restrict__ nnb, const int* __restrict__ comp, int* minseed) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double fi = f[i];
    if (!(fi > sl)) return;
    for (int s = 0; s < nnb[i]; s++) {
        int j = nbr[(size_t)s * n + i];
        if (j >= 0 && fi > f[j]) return;
    }
    atomicMin(&minseed[comp[i]], i);
}

__global__ void k_seed_flag(int n, const double* __restrict__ f, double sl, const int* __restrict__ comp,
                            const int* __restrict__ minseed, int* flag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flag[i] = (f[i] > sl && minseed[comp[i]] == i) ? 1 : 0;
}

// label (1..P0) per cell, then outlets removed; present[label] marks survivors
__global__ void k_label(int n, const double* __restrict__ f, double sl, const int* __restrict__ comp,
                        const int* __restrict__ minseed, const int* __restrict__ rank,
                        const uint8_t* __restrict__ outlet, int* lab, int* present) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int l = -1;
    if (f[i] > sl) {
        int ms = minseed[comp[i]];
        if (ms != INT_MAX) l = rank[ms] + 1;
    }
    if (outlet[i]) l = -1;
    lab[i] = l;
    if (l > 0) present[l] = 1;
}

__global__ void k_relabel(int n, const int* __restrict__ lab, const int* __restrict__ newid, int* pit) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int l = lab[i];
    pit[i] = (l > 0) ? newid[l] + 1 : -1;
}

// --------------------------------------------------------------------------
// spill points, flat distances, flat receivers
// --------------------------------------------------------------------------
__device__ __forceinline__ void rim_tests(int i, int n, const double* f, const int* pit,
                                          const int* nbr, const int8_t* nnb, const uint8_t* outlet,
                                          bool* lower, bool* eq) {
    bool lo = false, e = false;
    const double fi = f[i];
    for (int s = 0; s < nnb[i]; s++) {
        int j = nbr[(size_t)s * n + i];
        if (j < 0) continue;
        double fj = f[j];
        if (fj < fi) lo = true;
        else if (fj == fi && (outlet[j] || pit[j] == -1)) e = true;
    }
    *lower = lo;
    *eq = e;
}

__global__ void k_spill_qual(int n, const double* __restrict__ f, const int* __restrict__ pit,
                             const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                             const uint8_t* __restrict__ outlet, int* bestlid) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int p = pit[i];
    if (p < 0) return;
    bool lo, eq;
    rim_tests(i, n, f, pit, nbr, nnb, outlet, &lo, &eq);
    if (lo || eq) atomicMin(&bestlid[p], i);
}

__global__ void k_spill_pick(int np1, int n, const double* __restrict__ f, const int* __restrict__ pit,
                             const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                             const uint8_t* __restrict__ outlet, const int* __restrict__ bestlid,
                             int* pit_info, int* spill_flag) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np1) return;
    int spill = -1, rank = -1;
    int i = (p > 0) ? bestlid[p] : INT_MAX;
    if (i != INT_MAX) {
        bool lo, eq;
        rim_tests(i, n, f, pit, nbr, nnb, outlet, &lo, &eq);
        if (lo) {
            spill = i;
        } else {
            const double fi = f[i];
            int best = INT_MAX;
            for (int s = 0; s < nnb[i]; s++) {
                int j = nbr[(size_t)s * n + i];
                if (j < 0) continue;
                if (f[j] == fi && (outlet[j] || pit[j] == -1) && j < best) best = j;
            }
            spill = best;
        }
        rank = 0;
        spill_flag[spill] = 1;
    }
    pit_info[2 * p] = spill;
    pit_info[2 * p + 1] = rank;
}

__global__ void k_bfs_init(int n, const int* __restrict__ spill_flag, int* pdir, int* front, int* cnt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (spill_flag[i]) {
        pdir[i] = 1;
        front[atomicAdd(cnt, 1)] = i;
    } else {
        pdir[i] = -1;
    }
}

__global__ void k_bfs_step(int m, const int* __restrict__ front, int d, int n,
                           const double* __restrict__ f, const int* __restrict__ pit,
                           const int* __restrict__ nbr, const int8_t* __restrict__ nnb, int* pdir,
                           int* next, int* cnt) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    int i = front[t];
    const double fi = f[i];
    for (int s = 0; s < nnb[i]; s++) {
        int c = nbr[(size_t)s * n + i];
        if (c < 0 || pit[c] < 0 || !(f[c] >= fi)) continue;
        if (atomicCAS(&pdir[c], -1, d + 1) == -1) next[agg_append(cnt)] = c;
    }
}

// All remaining BFS levels in one block: frontier lists in global memory,
// __syncthreads between levels (the frontiers of lake flats are small, the
// level count is large).  Bounded by the vertex count.
__global__ void k_bfs_block(int fsize0, int* fa, int* fb, int* cnt, int d0, int n,
                            const double* __restrict__ f, const int* __restrict__ pit,
                            const int* __restrict__ nbr, const int8_t* __restrict__ nnb, int* pdir,
                            int* levels_out) {
    __shared__ int s_size;
    int fsize = fsize0, d = d0, levels = 0;
    int* cur = fa;
    int* nxt = fb;
    while (fsize > 0 && levels <= n) {
        if (threadIdx.x == 0) *cnt = 0;
        __syncthreads();
        for (int t = threadIdx.x; t < fsize; t += blockDim.x) {
            int i = cur[t];
            const double fi = f[i];
            for (int s = 0; s < nnb[i]; s++) {
                int c = nbr[(size_t)s * n + i];
                if (c < 0 || pit[c] < 0 || !(f[c] >= fi)) continue;
                if (atomicCAS(&pdir[c], -1, d + 1) == -1) nxt[agg_append(cnt)] = c;
            }
        }
        __threadfence_block();
        __syncthreads();
        if (threadIdx.x == 0) s_size = *(volatile int*)cnt;
        __syncthreads();
        fsize = s_size;
        int* tmp = cur; cur = nxt; nxt = tmp;
        d++;
        levels++;
        __syncthreads();
    }
    if (threadIdx.x == 0) *levels_out = levels;
}

// BFS successors of every vertex that can be reached (pit cells, spill
// nodes): neighbours c with pit(c) > -1 and lFill(c) >= lFill(i), row-major
__global__ void k_bfs_adj(int n, int W, const double* __restrict__ f, const int* __restrict__ pit,
                          const int* __restrict__ spill_flag, const int* __restrict__ nbr,
                          const int8_t* __restrict__ nnb, int* adj, int8_t* adjn) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int k = 0;
    if (pit[i] > -1 || spill_flag[i]) {
        const double fi = f[i];
        for (int s = 0; s < nnb[i]; s++) {
            int c = nbr[(size_t)s * n + i];
            if (c < 0 || pit[c] < 0 || !(f[c] >= fi)) continue;
            adj[(size_t)i * W + k++] = c;
        }
    }
    adjn[i] = (int8_t)k;
}

constexpr int BFS_CAP = 5120;

// remaining BFS levels in one block; frontiers in shared memory while they
// fit, mirrored to global arrays for the wider levels
__global__ void __launch_bounds__(1024) k_bfs_block2(int fsize0, int* init, int* gA, int d0,
                                                     int n, int W, const int* __restrict__ adj,
                                                     const int8_t* __restrict__ adjn, int* pdir,
                                                     int* levels_out) {
    __shared__ int sA[BFS_CAP], sB[BFS_CAP];
    __shared__ int s_next;
    const int tid = threadIdx.x, nt = blockDim.x;
    int size = fsize0, d = d0, levels = 0;
    int* curG = init;
    int* nxtG = gA;
    bool cur_sh = false;
    int* curS = sA;
    int* nxtS = sB;
    while (size > 0 && levels <= n) {
        if (tid == 0) s_next = 0;
        __syncthreads();
        for (int t = tid; t < size; t += nt) {
            int i = cur_sh ? curS[t] : curG[t];
            int k = adjn[i];
            const int* row = adj + (size_t)i * W;
            for (int q = 0; q < k; q++) {
                int c = row[q];
                if (atomicCAS(&pdir[c], -1, d + 1) == -1) {
                    int pos = atomicAdd(&s_next, 1);
                    if (pos < BFS_CAP) nxtS[pos] = c;
                    nxtG[pos] = c;
                }
            }
        }
        __syncthreads();
        size = s_next;
        __syncthreads();
        if (size <= BFS_CAP) {
            cur_sh = true;
            int* t = curS; curS = nxtS; nxtS = t;
        } else {
            cur_sh = false;
        }
        int* oldcur = curG;
        curG = nxtG;
        nxtG = oldcur;
        d++;
        levels++;
    }
    if (tid == 0) *levels_out = levels;
}

// BFS over the compacted set of reachable vertices (pit cells and spill
// nodes, local ids 0..M-1) in one block: the visited set is a shared-memory
// bitmap and the frontiers live in shared memory, so a level costs one global
// load of the adjacency rows, warp-aggregated appends and one block barrier.
__global__ void k_bfs_flag(int n, const int* __restrict__ pit, const int* __restrict__ spill_flag, int* flag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = (pit[i] > -1 || spill_flag[i]) ? 1 : 0;
}

__global__ void k_bfs_local_build(int n, int S, const double* __restrict__ f, const int* __restrict__ pit,
                                  const int* __restrict__ flag, const int* __restrict__ lid,
                                  const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                                  const int* __restrict__ spill_flag, int* rows, int* l2g, int* ld,
                                  int* seeds, int* nseed) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !flag[i]) return;
    const int li = lid[i];
    l2g[li] = i;
    ld[li] = -1;
    const double fi = f[i];
    int* row = rows + (size_t)li * S;
    int k = 0;
    for (int s = 0; s < nnb[i]; s++) {
        int c = nbr[(size_t)s * n + i];
        if (c < 0 || pit[c] < 0 || !(f[c] >= fi)) continue;
        row[1 + k++] = lid[c];
    }
    row[0] = k;
    if (spill_flag[i]) seeds[agg_append(nseed)] = li;
}

__global__ void k_bfs_local_scatter(int M, const int* __restrict__ l2g, const int* __restrict__ ld, int* pdir) {
    int li = blockIdx.x * blockDim.x + threadIdx.x;
    if (li < M && ld[li] > 0) pdir[l2g[li]] = ld[li];
}

constexpr int LBFS_CAP = 6144;

// S4: int4 words of a packed adjacency row (S = 4 * S4 ints, row[0] the
// count).  A level's cost is the instruction chain of its busiest warp, so
// the row width is a compile-time constant and the claimed cells are
// appended by walking the set bits of the claim mask.
template <int S4>
__global__ void __launch_bounds__(1024) k_bfs_local(int M, int S, const int* __restrict__ rows,
                                                    const int* __restrict__ seeds, const int* __restrict__ nseed_p,
                                                    int* gA, int* gB, int* ld, int* levels_out) {
    extern __shared__ unsigned smem_u[];
    unsigned* vis = smem_u;                           // ceil(M/32) words
    const int nw = (M + 31) >> 5;
    int* fA = (int*)(smem_u + nw);
    int* fB = fA + LBFS_CAP;
    // three rotating frontier counters: level r reads s_cnt[r%3], appends to
    // s_cnt[(r+1)%3] and clears s_cnt[(r+2)%3], so one barrier per level
    // separates every write of a counter from its reads
    __shared__ int s_cnt[3];
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31;
    for (int w = tid; w < nw; w += nt) vis[w] = 0u;
    if (tid < 3) s_cnt[tid] = 0;
    __syncthreads();
    int size = *nseed_p;
    // seeds: distance 1; frontier entries beyond LBFS_CAP live in global memory
    for (int t = tid; t < size; t += nt) {
        int li = seeds[t];
        atomicOr(&vis[li >> 5], 1u << (li & 31));
        if (t < LBFS_CAP) fA[t] = li;
        else gA[t] = li;
    }
    __syncthreads();
    int* curS = fA;
    int* nxtS = fB;
    int* curG = gA;
    int* nxtG = gB;
    int d = 1, levels = 0, r = 0;
    while (size > 0 && levels <= M) {
        int* cnt = &s_cnt[(r + 1) % 3];
        if (tid == 0) s_cnt[(r + 2) % 3] = 0;
        // every warp runs the same number of batches so that ballots see all lanes
        for (int base = 0; base < size; base += nt) {
            const int t = base + tid;
            // warps past the end of the frontier go straight to the barrier
            if (!__any_sync(0xffffffffu, t < size)) break;
            constexpr int RW = 4 * S4;
            int row[RW];
            int k = 0;
            if (t < size) {
                const int li = t < LBFS_CAP ? curS[t] : curG[t];
                const int4* r4 = reinterpret_cast<const int4*>(rows + (size_t)li * S);
#pragma unroll
                for (int q = 0; q < S4; q++) {
                    int4 v = r4[q];
                    row[4 * q] = v.x; row[4 * q + 1] = v.y; row[4 * q + 2] = v.z; row[4 * q + 3] = v.w;
                }
                k = row[0];
            }
            // claim the unvisited out-neighbours: plain checks, then the
            // atomics, all independent so their latencies overlap
            unsigned cand = 0u;
#pragma unroll
            for (int q = 1; q < RW; q++)
                if (q <= k && !(vis[row[q] >> 5] & (1u << (row[q] & 31)))) cand |= 1u << q;
            unsigned olds[RW];
#pragma unroll
            for (int q = 1; q < RW; q++)
                olds[q] = (cand & (1u << q)) ? atomicOr(&vis[row[q] >> 5], 1u << (row[q] & 31)) : 0u;
#pragma unroll
            for (int q = 1; q < RW; q++)
                if (olds[q] & (1u << (row[q] & 31))) cand &= ~(1u << q);
            // warp-aggregated append of the claimed cells
            const int mine = __popc(cand);
            int incl = mine;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            int pos0 = 0;
            if (lane == 31 && total > 0) pos0 = atomicAdd(cnt, total);
            pos0 = __shfl_sync(0xffffffffu, pos0, 31);
            int pos = pos0 + incl - mine;
#pragma unroll
            for (int q = 1; q < RW; q++) {
                if (cand & (1u << q)) {
                    const int c = row[q];
                    ld[c] = d + 1;
                    if (pos < LBFS_CAP) nxtS[pos] = c;
                    else nxtG[pos] = c;
                    pos++;
                }
            }
        }
        __syncthreads();
        size = *cnt;
        int* t1 = curS; curS = nxtS; nxtS = t1;
        int* t2 = curG; curG = nxtG; nxtG = t2;
        d++;
        levels++;
        r++;
    }
    if (tid == 0) *levels_out = levels;
}

// Flat distances by tiles, in one cooperative launch (delta-stepping).  The
// reachable cells are compacted in vertex order (local ids), and vertex ids
// follow a space-filling curve, so tile t = local ids [tT, tT + T) is a
// compact patch of the mesh; with no more tiles than blocks every block keeps
// its tile's adjacency rows in shared memory for the whole launch.
// Distances are settled by windows [lo, lo + window): in a round, every tile whose
// smallest pending distance falls in the window loads its distances, relaxes
// its cells of the window and then, one block barrier per wave, the cells they
// lower within the window; a cell lowered beyond the window only records the
// tile's pending minimum, and a hop out of the tile lowers the target's
// global distance (atomicMin) and the target tile's pending minimum.  Every
// pending minimum also lowers a global minimum for the round (three rotating
// slots), which all blocks read after the grid barrier: the same window again
// while it still holds pending cells, else the next window starts at the
// smallest pending distance, and no pending cell ends the launch.  Distances
// only decrease and a window is closed only when no cell of it is pending, so
// every distance is the breadth-first hop count (exact, no timed wait).
constexpr int BFT_THREADS = 512;

__global__ void __launch_bounds__(BFT_THREADS, 2) k_bfs_tiles(int M, int S, int T, const int* __restrict__ rows,
                                                              const int* __restrict__ seeds,
                                                              const int* __restrict__ nseed_p, int* ld, int* ctl,
                                                              int window, int* depth_out, int* rounds_out) {
    cg::grid_group grid = cg::this_grid();
    extern __shared__ int sm_bft[];
    const int INF = 0x7fffffff;
    int* rs = sm_bft;              // [T * S] adjacency rows of the tile
    int* ds = rs + T * S;          // [T] distances
    int* fl0 = ds + T;             // [T] frontier lists
    int* fl1 = fl0 + T;
    int* xc = fl1 + T;             // [T] hops out of the tile: target, distance
    int* xd = xc + T;
    __shared__ int s_cnt[3];
    __shared__ int s_over[3];
    __shared__ int s_pmin;
    __shared__ int s_nx;
    const int ntiles = (M + T - 1) / T;
    int* gmin = ctl;               // [3] smallest pending distance after rounds r % 3
    int* pend = ctl + 3;           // [ntiles] smallest pending distance of each tile
    const int tid = threadIdx.x, nt = blockDim.x;
    const unsigned gtid = grid.thread_rank(), gsz = (unsigned)grid.size();
    for (unsigned i = gtid; i < (unsigned)M; i += gsz) ld[i] = INF;
    for (unsigned t = gtid; t < (unsigned)ntiles; t += gsz) pend[t] = INF;
    if (gtid < 3) gmin[gtid] = INF;
    grid.sync();
    const int ns = *nseed_p;
    for (unsigned q = gtid; q < (unsigned)ns; q += gsz) {
        const int li = seeds[q];
        ld[li] = 1;
        pend[li / T] = 1;
    }
    grid.sync();
    int lo = 1, hi = window;
    int cached = -1;
    int rounds = 0;
    if (ns == 0) lo = INF;
    for (int r = 0; lo != INF; r++) {
        rounds++;
        int* gnext = gmin + ((r + 1) % 3);
        if (blockIdx.x == 0 && tid == 0) gmin[(r + 2) % 3] = INF;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
            __syncthreads();
            const int pt = ((volatile int*)pend)[t];
            if (pt > hi) {
                // nothing of this window here: its pending minimum stays for later
                if (tid == 0 && pt != INF) atomicMin(gnext, pt);
                continue;
            }
            const int base = t * T, len = min(T, M - base);
            if (cached != t) {
                const int4* src = reinterpret_cast<const int4*>(rows + (size_t)base * S);
                int4* dst = reinterpret_cast<int4*>(rs);
                const int nq = len * S / 4;
                for (int q = tid; q < nq; q += nt) dst[q] = src[q];
                cached = t;
            }
            if (tid == 0) {
                atomicExch(&pend[t], INF);
                __threadfence();
            }
            __syncthreads();
            for (int i = tid; i < len; i += nt) ds[i] = ((volatile int*)ld)[base + i];
            // wave 0 relaxes every cell of the tile inside the window
            if (tid < 3) {
                s_cnt[tid] = 0;
                s_over[tid] = tid == 0 ? 1 : 0;
            }
            if (tid == 0) {
                s_pmin = INF;
                s_nx = 0;
            }
            __syncthreads();
            for (int w = 0;; w++) {
                const int rd = w % 3, wr = (w + 1) % 3;
                int* lin = (w & 1) ? fl1 : fl0;
                int* lout = (w & 1) ? fl0 : fl1;
                const int full = s_over[rd];
                const int size = full ? len : s_cnt[rd];
                if (size == 0 && !full) break;
                if (tid == 0) {
                    s_cnt[(w + 2) % 3] = 0;
                    s_over[(w + 2) % 3] = 0;
                }
                for (int e = tid; e < size; e += nt) {
                    const int i = full ? e : lin[e];
                    const int d = ds[i];
                    if (d < lo || d > hi) continue;
                    const int* row = rs + i * S;
                    const int k = row[0];
                    const int nd = d + 1;
                    // lower the in-tile out-neighbours, then one append for
                    // those that dropped inside the window; hops out of the
                    // tile are buffered and applied once after the waves
                    unsigned got = 0u;
                    for (int q = 1; q <= k; q++) {
                        const int c = row[q];
                        const int lc = c - base;
                        if ((unsigned)lc < (unsigned)len) {
                            if (atomicMin(&ds[lc], nd) > nd && nd <= hi) got |= 1u << q;
                        } else {
                            const int x = atomicAdd(&s_nx, 1);
                            if (x < T) {
                                xc[x] = c;
                                xd[x] = nd;
                            } else if (atomicMin(&ld[c], nd) > nd) {
                                atomicMin(&pend[c / T], nd);
                                atomicMin(gnext, nd);
                            }
                        }
                    }
                    if (got) {
                        int pos = atomicAdd(&s_cnt[wr], __popc(got));
                        for (int q = 1; q <= k; q++) {
                            if (!(got & (1u << q))) continue;
                            if (pos < T) lout[pos] = row[q] - base;
                            else s_over[wr] = 1;
                            pos++;
                        }
                    }
                }
                __syncthreads();
            }
            // the buffered hops out of the tile, their latencies overlapped
            {
                const int nx = min(s_nx, T);
                for (int x = tid; x < nx; x += nt) {
                    const int c = xc[x], nd = xd[x];
                    if (atomicMin(&ld[c], nd) > nd) {
                        atomicMin(&pend[c / T], nd);
                        atomicMin(gnext, nd);
                    }
                }
            }
            // write back; no cell beyond the window has been relaxed yet, so
            // the smallest such distance is the tile's pending minimum
            int pmin = INF;
            for (int i = tid; i < len; i += nt) {
                const int d = ds[i];
                if (d < ((volatile int*)ld)[base + i]) atomicMin(&ld[base + i], d);
                if (d > hi && d < pmin) pmin = d;
            }
            pmin = __reduce_min_sync(0xffffffffu, pmin);
            if ((tid & 31) == 0 && pmin != INF) atomicMin(&s_pmin, pmin);
            __syncthreads();
            if (tid == 0 && s_pmin != INF) {
                atomicMin(&pend[t], s_pmin);
                atomicMin(gnext, s_pmin);
            }
        }
        grid.sync();
        // the same in every block: written before the barrier, cleared two rounds later
        const int g = ((volatile int*)gmin)[(r + 1) % 3];
        if (g == INF) break;
        if (g > hi) {
            lo = g;
            hi = g + window - 1;
        }
        if (r > 4 * M + 8) break;   // cannot happen: every round settles a pending cell or moves the window
    }
    int dmax = 0;
    for (unsigned i = gtid; i < (unsigned)M; i += gsz) {
        const int d = ld[i];
        if (d == INF) ld[i] = -1;
        else dmax = d > dmax ? d : dmax;
    }
    dmax = __reduce_max_sync(0xffffffffu, dmax);
    if ((tid & 31) == 0 && dmax > 0) atomicMax(depth_out, dmax);
    if (gtid == 0) *rounds_out = rounds;
}

// Whole BFS in one cooperative launch: wide levels use the whole grid with a
// grid-wide barrier per level; once a level is narrower than one block's
// worth, block 0 finishes the remaining levels alone with block barriers
// (the other blocks have left, so no grid barrier is used after that point).
// sizes[] holds three rotating frontier counters: round r reads sizes[r%3],
// appends to sizes[(r+1)%3], and sizes[(r+2)%3] is cleared for round r+1.
__global__ void __launch_bounds__(256) k_bfs_coop(int* fa, int* fb, int* sizes, int d0, int n, int W,
                                                  const int* __restrict__ adj, const int8_t* __restrict__ adjn,
                                                  int* pdir, int* levels_out) {
    cg::grid_group grid = cg::this_grid();
    int d = d0, levels = 0;
    int* cur = fa;
    int* nxt = fb;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gsz = gridDim.x * blockDim.x;
    int r = 0;
    int sz = sizes[0];
    while (sz > 1024 && levels <= n) {
        int* cnt = &sizes[(r + 1) % 3];
        for (int t = gtid; t < sz; t += gsz) {
            int i = cur[t];
            int k = adjn[i];
            const int* row = adj + (size_t)i * W;
            for (int q = 0; q < k; q++) {
                int c = row[q];
                if (atomicCAS(&pdir[c], -1, d + 1) == -1) nxt[agg_append(cnt)] = c;
            }
        }
        if (gtid == 0) sizes[(r + 2) % 3] = 0;
        grid.sync();
        sz = *(volatile int*)&sizes[(r + 1) % 3];
        int* tmp = cur; cur = nxt; nxt = tmp;
        d++;
        levels++;
        r++;
    }
    if (blockIdx.x != 0) return;
    // narrow tail: block 0 only
    __shared__ int s_cnt;
    while (sz > 0 && levels <= n) {
        if (threadIdx.x == 0) s_cnt = 0;
        __syncthreads();
        for (int t = threadIdx.x; t < sz; t += blockDim.x) {
            int i = cur[t];
            int k = adjn[i];
            const int* row = adj + (size_t)i * W;
            for (int q = 0; q < k; q++) {
                int c = row[q];
                if (atomicCAS(&pdir[c], -1, d + 1) == -1) nxt[atomicAdd(&s_cnt, 1)] = c;
            }
        }
        __syncthreads();
        sz = s_cnt;
        __syncthreads();
        int* tmp = cur; cur = nxt; nxt = tmp;
        d++;
        levels++;
    }
    if (threadIdx.x == 0) *levels_out = levels;
}

// Basin-graph edges deduplicated: k_cross_edges emits one edge per boundary
// cell and neighbouring basin, so a pair of basins is joined by as many
// parallel edges as it has boundary cells (about twelve per pair on the
// sphere's relief).  Only the lowest of them can lower a level, so the edges
// go through an open-addressing table keyed by (u, v) that keeps the smallest
// weight key, and the relaxation runs over one edge per pair.  The table has
// a power-of-two size of about four times the pairs of the previous fill;
// linear probing gives up after XH_PROBES slots, and then the relaxation uses
// the edges as emitted (*raw = 1) and the next fill gets a larger table.
__device__ __forceinline__ unsigned long long xh_mix(unsigned long long k) {
    // the 64-bit finaliser of MurmurHash3 (Appleby)
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ULL;
    k ^= k >> 33;
    return k;
}

constexpr int XH_PROBES = 64;

__global__ void k_xedge_insert(const int* __restrict__ m_count, int cap, const int* __restrict__ xu,
                               const int* __restrict__ xv, const double* __restrict__ xw,
                               unsigned long long* hkey, unsigned long long* hval, long long hcap, int* raw) {
    const int m = *m_count < cap ? *m_count : cap;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gsz = gridDim.x * blockDim.x;
    const unsigned long long mask = (unsigned long long)hcap - 1ULL;
    for (int e = gtid; e < m; e += gsz) {
        const unsigned long long key = ((unsigned long long)(unsigned)xu[e] << 32) | (unsigned)xv[e];
        const unsigned long long w = dkey(xw[e]);
        unsigned long long s = xh_mix(key) & mask;
        bool placed = false;
        for (int probe = 0; probe < XH_PROBES; probe++) {
            const unsigned long long k = atomicCAS(&hkey[s], ~0ULL, key);
            if (k == ~0ULL || k == key) {
                atomicMin(&hval[s], w);
                placed = true;
                break;
            }
            s = (s + 1ULL) & mask;
        }
        if (!placed) *raw = 1;
    }
}

// table -> edge list (any order: the relaxation's fixed point does not depend
// on it); every used slot is emptied again for the next fill
__global__ void k_xedge_compact(long long hcap, unsigned long long* hkey, unsigned long long* hval, int* du, int* dv,
                                unsigned long long* dw, int* count) {
    const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x, gsz = (long long)gridDim.x * blockDim.x;
    for (long long s = gtid; s < hcap; s += gsz) {
        const unsigned long long k = hkey[s];
        if (k == ~0ULL) continue;
        const int pos = agg_append(count);
        du[pos] = (int)(k >> 32);
        dv[pos] = (int)(unsigned)(k & 0xffffffffULL);
        dw[pos] = hval[s];
        hkey[s] = ~0ULL;
        hval[s] = ~0ULL;
    }
}

// Minimax relaxation over the basin graph in one cooperative launch:
// L[u] = min(L[u], max(w, L[v])) over the edges v -> u until nothing
// changes.  A thread keeps its first RELAX_REG edges (u, v, weight and the
// level of v it last used) in registers for the whole launch, and between two
// grid barriers relaxes them RELAX_SUB times, each time only when the level
// of v changed since it last relaxed that edge: a lowered level travels along
// a chain of basins within one round instead of one basin per round.  Edges
// beyond the registers are relaxed once per round.  A round ends with a grid
// barrier and continues while any level changed in it (three rotating change
// flags: round r sets flags[r % 3], reads it after the barrier and clears
// flags[(r + 1) % 3]).  Levels only decrease and a round without any change
// used only final levels, so the result is the fixed point of the all-edges
// relaxation whatever the order of the updates.
constexpr int RELAX_REG = 2;
constexpr int RELAX_SUB = 8;

__global__ void __launch_bounds__(256) k_relax_active(const int* __restrict__ m_count, int cap,
                                                      const int* __restrict__ raw_p, const int* __restrict__ xu,
                                                      const int* __restrict__ xv, const double* __restrict__ xw,
                                                      const int* __restrict__ md_count, const int* __restrict__ du,
                                                      const int* __restrict__ dv,
                                                      const unsigned long long* __restrict__ dw,
                                                      unsigned long long* L, int* flags, int max_rounds,
                                                      int* rounds_out) {
    cg::grid_group grid = cg::this_grid();
    const bool raw = *raw_p != 0;
    // raw: the edge count as k_cross_edges left it (its appends stop at the capacity)
    const int m = raw ? (*m_count < cap ? *m_count : cap) : *md_count;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gsz = gridDim.x * blockDim.x;
    int cu[RELAX_REG], cv[RELAX_REG];
    unsigned long long cw[RELAX_REG], last[RELAX_REG];
#pragma unroll
    for (int q = 0; q < RELAX_REG; q++) {
        const int e = gtid + q * gsz;
        cv[q] = -1;
        cu[q] = 0;
        cw[q] = 0ULL;
        last[q] = ~0ULL;
        if (e < m) {
            cu[q] = raw ? xu[e] : du[e];
            cv[q] = raw ? xv[e] : dv[e];
            cw[q] = raw ? dkey(xw[e]) : dw[e];
        }
    }
    volatile unsigned long long* VL = L;
    int r = 1;
    for (; r <= max_rounds; r++) {
        int changed = 0;
        for (int sub = 0; sub < RELAX_SUB; sub++) {
            unsigned long long lv[RELAX_REG];
#pragma unroll
            for (int q = 0; q < RELAX_REG; q++) lv[q] = cv[q] >= 0 ? VL[cv[q]] : ~0ULL;
#pragma unroll
            for (int q = 0; q < RELAX_REG; q++) {
                if (lv[q] == ~0ULL || lv[q] == last[q]) continue;
                last[q] = lv[q];
                const unsigned long long cand = cw[q] > lv[q] ? cw[q] : lv[q];
                if (cand < atomicMin(&L[cu[q]], cand)) changed = 1;
            }
        }
        for (int e = gtid + RELAX_REG * gsz; e < m; e += gsz) {
            const int v = raw ? xv[e] : dv[e];
            const unsigned long long lv = VL[v];
            if (lv == ~0ULL) continue;
            const unsigned long long w = raw ? dkey(xw[e]) : dw[e];
            const unsigned long long cand = w > lv ? w : lv;
            const int u = raw ? xu[e] : du[e];
            if (cand < VL[u] && cand < atomicMin(&L[u], cand)) changed = 1;
        }
        if (__any_sync(0xffffffffu, changed) && (threadIdx.x & 31) == 0) flags[r % 3] = 1;
        // clear the flag of the next round: its last readers (end of round
        // r - 2) have all passed the barrier of round r - 1.  The flag of
        // round r - 1 may still be unread by slow threads.
        if (gtid == 0) flags[(r + 1) % 3] = 0;
        grid.sync();
        if (!*(volatile int*)&flags[r % 3]) break;
    }
    if (gtid == 0) *rounds_out = r;
}

__global__ void k_flat_dirs(int n, const double* __restrict__ f, const int* __restrict__ pit,
                            const int* __restrict__ pdir, const int* __restrict__ nbr,
                            const int8_t* __restrict__ nnb, const int* __restrict__ spill_flag,
                            double sl, const double* __restrict__ h, int* flat, double* lfill) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int out = -1;
    if (pit[i] > -1) {
        const int pi = pdir[i];
        const double fi = f[i];
        int bd = INT_MAX, bj = INT_MAX;
        for (int s = 0; s < nnb[i]; s++) {
            int c = nbr[(size_t)s * n + i];
            if (c < 0) continue;
            int pc = pdir[c];
            if (pc > -1 && pc < pi && f[c] <= fi) {
                if (pc < bd || (pc == bd && c < bj)) { bd = pc; bj = c; }
            }
        }
        out = (bj != INT_MAX) ? bj : i;
    }
    if (spill_flag[i]) out = -1;
    if (f[i] <= sl) {          // open sea: unfilled, no flat routing (pitfilling.py:822-825)
        out = -1;
        lfill[i] = h[i];
    }
    flat[i] = out;
}

// --------------------------------------------------------------------------
// pit tables
// --------------------------------------------------------------------------
__global__ void k_pit_flag(int n, const int* __restrict__ pit, int* flag, int* counts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int p = pit[i];
    flag[i] = p >= 0 ? 1 : 0;
    if (p >= 0) atomicAdd(&counts[p], 1);
}

__global__ void k_pit_compact(int n, const int* __restrict__ pit, const int* __restrict__ pos,
                              int* keys, int* vals) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int p = pit[i];
    if (p < 0) return;
    keys[pos[i]] = p;
    vals[pos[i]] = i;
}

// Block-per-pit reductions in a fixed order (deterministic): strided partial
// sums per thread, then a fixed shared-memory tree.  A thread visits its
// cells t = lane, lane + 256, ... in order; the cells of PIT_UNROLL visits and
// their values are loaded before any is added, so that the gathers of a large
// pit overlap, and the additions keep the visiting order.
constexpr int PIT_UNROLL = 8;

template <int NV>
__device__ __forceinline__ void block_reduce(double (&v)[NV], bool is_max[NV]) {
    __shared__ double sh[NV][256];
    for (int q = 0; q < NV; q++) sh[q][threadIdx.x] = v[q];
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int q = 0; q < NV; q++)
                sh[q][threadIdx.x] = is_max[q] ? fmax(sh[q][threadIdx.x], sh[q][threadIdx.x + s])
                                               : sh[q][threadIdx.x] + sh[q][threadIdx.x + s];
        __syncthreads();
    }
    for (int q = 0; q < NV; q++) v[q] = sh[q][0];
}

// Per-pit reductions over chunks: a pit's cells (sorted by id, segments of
// seg_vals2) are cut into chunks of PIT_CHUNK = 256 * PIT_UNROLL cells, one
// block per chunk, so that a lake of tens of thousands of cells spreads over
// many blocks instead of holding one block while the others have finished.
// Within a chunk thread `lane` adds its cells lane, lane + 256, ... in order
// and the block tree combines the threads; a finishing pass adds a pit's chunk
// partials in chunk order.  A pit of one chunk therefore sums exactly as a
// block over the whole pit did.
constexpr int PIT_CHUNK = 256 * PIT_UNROLL;

__global__ void k_pit_nchunk(int np1, const int* __restrict__ counts, int* nch) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < np1) nch[p] = (counts[p] + PIT_CHUNK - 1) / PIT_CHUNK;
}

// item -> pit (items of pit p: chs[p] .. chs[p] + nch[p] - 1)
__global__ void k_pit_items(int np1, const int* __restrict__ nch, const int* __restrict__ chs, int* item_pit) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np1) return;
    const int c0 = chs[p], k = nch[p];
    for (int c = 0; c < k; c++) item_pit[c0 + c] = p;
}

// the item of this block: its pit, first cell and cell count; false past the last item
__device__ __forceinline__ bool pit_item(int np1, const int* __restrict__ nch, const int* __restrict__ chs,
                                         const int* __restrict__ item_pit, const int* __restrict__ start,
                                         const int* __restrict__ counts, int* p, int* s0, int* c) {
    const int i = blockIdx.x;
    if (i >= chs[np1 - 1] + nch[np1 - 1]) return false;
    const int q = item_pit[i];
    const int k = i - chs[q];
    *p = q;
    *s0 = start[q] + k * PIT_CHUNK;
    const int rest = counts[q] - k * PIT_CHUNK;
    *c = rest < PIT_CHUNK ? rest : PIT_CHUNK;
    return true;
}

// chunk partials of vol, max fill, max depth (cells sorted by id)
__global__ void __launch_bounds__(256) k_pit_params(int np1, const int* __restrict__ nch, const int* __restrict__ chs,
                                                    const int* __restrict__ item_pit,
                                                    const int* __restrict__ start, const int* __restrict__ counts,
                                                    const int* __restrict__ cells, const double* __restrict__ f,
                                                    const double* __restrict__ h, double sl,
                                                    const double* __restrict__ larea, double* part) {
    int p, s0, c;
    if (!pit_item(np1, nch, chs, item_pit, start, counts, &p, &s0, &c)) return;
    const int lane = threadIdx.x;
    double v[3] = {0.0, -INFINITY, -INFINITY};
    int ii[PIT_UNROLL];
    double fi[PIT_UNROLL], hi[PIT_UNROLL], ai[PIT_UNROLL];
#pragma unroll
    for (int u = 0; u < PIT_UNROLL; u++) ii[u] = lane + u * 256 < c ? cells[s0 + lane + u * 256] : -1;
#pragma unroll
    for (int u = 0; u < PIT_UNROLL; u++) {
        if (ii[u] < 0) continue;
        fi[u] = f[ii[u]];
        hi[u] = h[ii[u]];
        ai[u] = larea[ii[u]];
    }
#pragma unroll
    for (int u = 0; u < PIT_UNROLL; u++) {
        if (ii[u] < 0) continue;
        double hc = hi[u] < sl ? sl : hi[u];
        double d = fi[u] - hc;
        v[0] += d * ai[u];
        v[1] = fmax(v[1], fi[u]);
        v[2] = fmax(v[2], d);
    }
    bool mx[3] = {false, true, true};
    block_reduce<3>(v, mx);
    if (lane == 0)
        for (int q = 0; q < 3; q++) part[3 * (size_t)blockIdx.x + q] = v[q];
}

// pit params from the chunk partials, in chunk order
__global__ void k_pit_params_fin(int np1, const int* __restrict__ nch, const int* __restrict__ chs,
                                 const double* __restrict__ part, double* params) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np1) return;
    const int k = nch[p];
    if (k == 0) {
        params[3 * p] = 0.0;
        params[3 * p + 1] = -1.0e8;   // MISSING_DATA_SENTINEL (constants.py:34)
        params[3 * p + 2] = 0.0;
        return;
    }
    const size_t i0 = chs[p];
    double vol = part[3 * i0], hmax = part[3 * i0 + 1], dmax = part[3 * i0 + 2];
    for (int j = 1; j < k; j++) {
        vol = vol + part[3 * (i0 + j)];
        hmax = fmax(hmax, part[3 * (i0 + j) + 1]);
        dmax = fmax(dmax, part[3 * (i0 + j) + 2]);
    }
    params[3 * p] = vol;
    params[3 * p + 1] = hmax;
    params[3 * p + 2] = dmax;
}

__global__ void k_filled_lvl(int np1, const double* __restrict__ params, double* lvl) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np1) return;
    double d[6] = {0, 0, 0, 0, 0, 0};
    if (params[3 * p] > 0.0) {
        d[0] = params[3 * p + 1] - params[3 * p + 2];
        double st = params[3 * p + 2] / 5.0;
        for (int k = 1; k < 6; k++) d[k] = st;
    }
    double s = d[0];
    for (int k = 1; k < 6; k++) {
        s = s + d[k];
        lvl[5 * p + k - 1] = s;
    }
}

// chunk partials of the filled volumes at the four intermediate levels
__global__ void __launch_bounds__(256) k_filled_vol(int np1, const int* __restrict__ nch, const int* __restrict__ chs,
                                                    const int* __restrict__ item_pit,
                                                    const int* __restrict__ start, const int* __restrict__ counts,
                                                    const int* __restrict__ cells, const double* __restrict__ h,
                                                    double sl, const double* __restrict__ farea,
                                                    const double* __restrict__ lvl, double* part) {
    int p, s0, c;
    if (!pit_item(np1, nch, chs, item_pit, start, counts, &p, &s0, &c)) return;
    const int lane = threadIdx.x;
    const double l0 = lvl[5 * p], l1 = lvl[5 * p + 1], l2 = lvl[5 * p + 2], l3 = lvl[5 * p + 3];
    double v[4] = {0, 0, 0, 0};
    int ii[PIT_UNROLL];
    double hi[PIT_UNROLL], ai[PIT_UNROLL];
#pragma unroll
    for (int u = 0; u < PIT_UNROLL; u++) ii[u] = lane + u * 256 < c ? cells[s0 + lane + u * 256] : -1;
#pragma unroll
    for (int u = 0; u < PIT_UNROLL; u++) {
        if (ii[u] < 0) continue;
        hi[u] = h[ii[u]];
        ai[u] = farea[ii[u]];
    }
#pragma unroll
    for (int u = 0; u < PIT_UNROLL; u++) {
        if (ii[u] < 0) continue;
        double e = hi[u] < sl ? sl : hi[u];
        double a = ai[u];
        if (l0 > e) v[0] += (l0 - e) * a;
        if (l1 > e) v[1] += (l1 - e) * a;
        if (l2 > e) v[2] += (l2 - e) * a;
        if (l3 > e) v[3] += (l3 - e) * a;
    }
    bool mx[4] = {false, false, false, false};
    block_reduce<4>(v, mx);
    if (lane == 0)
        for (int q = 0; q < 4; q++) part[4 * (size_t)blockIdx.x + q] = v[q];
}

__global__ void k_filled_vol_fin(int np1, const int* __restrict__ nch, const int* __restrict__ chs,
                                 const double* __restrict__ part, const double* __restrict__ params, double* vol) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np1) return;
    const int k = nch[p];
    double v[4] = {0, 0, 0, 0};
    if (k > 0) {
        const size_t i0 = chs[p];
        for (int q = 0; q < 4; q++) v[q] = part[4 * i0 + q];
        for (int j = 1; j < k; j++)
            for (int q = 0; q < 4; q++) v[q] = v[q] + part[4 * (i0 + j) + q];
    }
    for (int q = 0; q < 4; q++) vol[5 * p + q] = v[q];
    vol[5 * p + 4] = params[3 * p];
}

// per-pit masked sum: chunk partials, then a pit's partials in chunk order
__global__ void __launch_bounds__(256) k_pit_masked_sum(int np1, const int* __restrict__ nch,
                                                        const int* __restrict__ chs,
                                                        const int* __restrict__ item_pit,
                                                        const int* __restrict__ start,
                                                        const int* __restrict__ counts,
                                                        const int* __restrict__ cells,
                                                        const uint8_t* __restrict__ mask,
                                                        const double* __restrict__ vals, double* part) {
    int p, s0, c;
    if (!pit_item(np1, nch, chs, item_pit, start, counts, &p, &s0, &c)) return;
    const int lane = threadIdx.x;
    double v[1] = {0.0};
    int ii[PIT_UNROLL];
    uint8_t mi[PIT_UNROLL];
    double xi[PIT_UNROLL];
#pragma unroll
    for (int u = 0; u < PIT_UNROLL; u++) ii[u] = lane + u * 256 < c ? cells[s0 + lane + u * 256] : -1;
#pragma unroll
    for (int u = 0; u < PIT_UNROLL; u++) {
        mi[u] = 0;
        if (ii[u] < 0) continue;
        mi[u] = mask[ii[u]];
        xi[u] = vals[ii[u]];
    }
#pragma unroll
    for (int u = 0; u < PIT_UNROLL; u++)
        if (mi[u]) v[0] += xi[u];
    bool mx[1] = {false};
    block_reduce<1>(v, mx);
    if (lane == 0) part[blockIdx.x] = v[0];
}

__global__ void k_pit_masked_fin(int np1, const int* __restrict__ nch, const int* __restrict__ chs,
                                 const double* __restrict__ part, double* out) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np1) return;
    const int k = nch[p];
    double v = 0.0;
    if (k > 0) {
        const int i0 = chs[p];
        v = part[i0];
        for (int j = 1; j < k; j++) v = v + part[i0 + j];
    }
    out[p] = v;
}

// --------------------------------------------------------------------------
// host driver
// --------------------------------------------------------------------------
static int launch_coop(gs_plan* p, const void* fn, void** args) {
    cudaEvent_t stop = nullptr;
    if (p->profiling) prof_begin(p, fn, &stop);
    GS_CUDA(cudaLaunchCooperativeKernel(fn, p->coop_blocks, 256, args, 0, p->stream));
    if (stop) cudaEventRecord(stop, p->stream);
    p->launches++;
    return GS_OK;
}

// Tiled flat-distance BFS (k_bfs_tiles) over the M compacted cells whose
// rows, seeds (front0, count in i_scalar[6]) and local ids k_bfs_local_build
// wrote; distances into ld (-1 unreached), depth into i_scalar[4].  Tiles of
// T cells with T * (S + 5) ints of shared memory (<= 112 KB), as many blocks
// as stay co-resident.
static int bfs_tiles(gs_plan* p, int M, int S, const int* rows, int* ld) {
    int T = 4096;
    while (T > 256 && (size_t)T * (S + 5) * sizeof(int) > 112 * 1024) T >>= 1;
    const size_t smem = (size_t)T * (S + 5) * sizeof(int);
    GS_CUDA(cudaFuncSetAttribute(k_bfs_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    GS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_bfs_tiles, BFT_THREADS, smem));
    if (occ < 1) {
        set_error(GS_ECUDA, "flat BFS: tile kernel cannot be resident");
        return GS_ECUDA;
    }
    const int ntiles = (M + T - 1) / T;
    const int grid = std::max(1, std::min(ntiles, p->sm_count * occ));
    if (3 + ntiles > (int)p->n + 1) {
        set_error(GS_EINVAL, "flat BFS: tile marks exceed their buffer");
        return GS_EINVAL;
    }
    GS_CUDA(cudaMemsetAsync(p->i_scalar + 4, 0, sizeof(int), p->stream));
    int m = M, s = S, t = T;
    const int* seeds = p->front0;
    const int* nseed = p->i_scalar + 6;
    int* ctl = p->front1;
    int* depth = p->i_scalar + 4;
    int* rounds = p->i_scalar + 15;
    int window = p->bfs_window;
    void* args[] = {(void*)&m, (void*)&s, (void*)&t, (void*)&rows, (void*)&seeds, (void*)&nseed, (void*)&ld,
                    (void*)&ctl, (void*)&window, (void*)&depth, (void*)&rounds};
    cudaEvent_t stop = nullptr;
    if (p->profiling) prof_begin(p, (const void*)k_bfs_tiles, &stop);
    GS_CUDA(cudaLaunchCooperativeKernel((const void*)k_bfs_tiles, grid, BFT_THREADS, args, smem, p->stream));
    if (stop) cudaEventRecord(stop, p->stream);
    p->launches++;
    GS_LAUNCH();
    return GS_OK;
}

static int read_ints(gs_plan* p, int* dst, const int* src, int count) {
    GS_CUDA(cudaMemcpyAsync(dst, src, sizeof(int) * count, cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    return GS_OK;
}

static int exclusive_scan(gs_plan* p, const int* in, int* out, int count) {
    size_t bytes = p->cub_bytes;
    GS_CUDA(cub::DeviceScan::ExclusiveSum(p->cub_tmp, bytes, in, out, count, p->stream));
    p->launches++;
    return GS_OK;
}

// chunk items of the pit segments (after seg_count and seg_start): at most
// np1 + ncell / PIT_CHUNK of them, the grid of the chunk kernels
static int pit_chunks(gs_plan* p, int np1, int ncell) {
    const int B = 256;
    const int64_t imax = (int64_t)np1 + ncell / PIT_CHUNK + 1;
    if (imax > INT_MAX) {
        set_error(GS_ENOMEM, "pit tables: too many chunk items");
        return GS_ENOMEM;
    }
    if (!p->pit_nch) {
        GS_CUDA(cudaMalloc((void**)&p->pit_nch, sizeof(int) * ((size_t)p->n + 2)));
        GS_CUDA(cudaMalloc((void**)&p->pit_chs, sizeof(int) * ((size_t)p->n + 2)));
    }
    if (imax > p->pit_item_cap) {
        const int64_t cap = std::max<int64_t>(imax, 2 * p->pit_item_cap);
        if (p->pit_item) cudaFree(p->pit_item);
        if (p->pit_part) cudaFree(p->pit_part);
        p->pit_item = nullptr;
        p->pit_part = nullptr;
        p->pit_item_cap = 0;
        GS_CUDA(cudaMalloc((void**)&p->pit_item, sizeof(int) * (size_t)cap));
        GS_CUDA(cudaMalloc((void**)&p->pit_part, sizeof(double) * 4 * (size_t)cap));
        p->pit_item_cap = cap;
    }
    launch(p, k_pit_nchunk, grid_for(np1, B), B, np1, (const int*)p->seg_count, p->pit_nch);
    GS_LAUNCH();
    GS_TRY(exclusive_scan(p, p->pit_nch, p->pit_chs, np1));
    launch(p, k_pit_items, grid_for(np1, B), B, np1, (const int*)p->pit_nch, (const int*)p->pit_chs, p->pit_item);
    GS_LAUNCH();
    p->pit_items_max = (int)imax;
    return GS_OK;
}

int group_sum_by_pit(gs_plan* p, const int* /*pit_ids*/, const uint8_t* mask, const double* vals,
                     double* out, int npits) {
    const int np1 = npits + 1;
    launch(p, k_pit_masked_sum, p->pit_items_max, 256, np1, (const int*)p->pit_nch, (const int*)p->pit_chs,
           (const int*)p->pit_item, (const int*)p->seg_start, (const int*)p->seg_count, (const int*)p->seg_vals2,
           mask, vals, p->pit_part);
    launch(p, k_pit_masked_fin, grid_for(np1, 256), 256, np1, (const int*)p->pit_nch, (const int*)p->pit_chs,
           (const double*)p->pit_part, out);
    GS_LAUNCH();
    return GS_OK;
}

int fill_join(gs_plan* p, gs_stats* st) {
    if (!p->bfs_pending) return GS_OK;
    p->bfs_pending = 0;
    GS_CUDA(cudaStreamWaitEvent(p->stream, p->ev_b, 0));
    GS_CUDA(cudaEventSynchronize(p->ev_b));
    if (st) st->flat_rounds = p->h_pinned[2];
    p->pdir_bound = p->h_pinned[2] + 2;   // the deepest distance is the BFS depth
    return GS_OK;
}

// 1 in *flag when a or b (may be null) holds a NaN or an infinity
__global__ void k_nonfinite(int n, const double* __restrict__ a, const double* __restrict__ b, int* flag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!isfinite(a[i]) || (b && !isfinite(b[i]))) *flag = 1;
}

int fill_elevation(gs_plan* p, const double* h, double sealevel, double ofill, double* lfill,
                   int* pit_ids, int* flat_dirs, gs_stats* st, bool defer_flats, uint8_t* sea_out, bool sed,
                   const double* check_b) {
    const int n = (int)p->n;
    GS_TRY(fill_join(p, nullptr));
    if (n == 0) { p->npits = 0; return GS_OK; }
    const int B = 256, G = grid_for(n, B);
    int hbuf[4];
    // the inputs must be finite: checked on the device now, read at the
    // first synchronisation below (the root search), before the relaxation,
    // the flat pass and any sweep
    GS_CUDA(cudaMemsetAsync(p->i_scalar + I_NONFINITE, 0, sizeof(int), p->stream));
    launch(p, k_nonfinite, G, B, n, h, check_b, p->i_scalar + I_NONFINITE);
    GS_LAUNCH();
    GS_CUDA(cudaMemcpyAsync(p->h_pinned + 9, p->i_scalar + I_NONFINITE, sizeof(int), cudaMemcpyDeviceToHost,
                            p->stream));

    // level
    GS_CUDA(cudaMemsetAsync(p->u_scalar, 0xff, sizeof(unsigned long long), p->stream));
    launch(p, k_min_key, p->sm_count * 4, 256, n, h, p->u_scalar);
    launch(p, k_level, 1, 1, (const unsigned long long*)p->u_scalar, p->flat ? 0 : 1, sealevel, ofill,
           p->d_scalar);
    GS_LAUNCH();
    // Filling with sediment (pitfilling.py:557-702, 704-847 with sed=True):
    // open-sea depressions are filled too, pits are labelled above the fill
    // level instead of sea level, and pit volumes use the unclipped surface.
    double label_sl = sealevel, clip_sl = sealevel, marine_sl = sealevel;
    if (sed) {
        GS_CUDA(cudaMemcpyAsync(&label_sl, p->d_scalar + D_LEVEL, sizeof(double), cudaMemcpyDeviceToHost,
                                p->stream));
        GS_CUDA(cudaStreamSynchronize(p->stream));
        clip_sl = -INFINITY;
        marine_sl = -INFINITY;
    }

    // seeds, descent links, roots
    launch(p, k_classify, G, B, n, h, (const double*)p->d_scalar, (const int*)p->nbr,
           (const int8_t*)p->nnb, (const uint8_t*)p->outlet, p->ledge);
    launch(p, k_descend, G, B, n, h, (const double*)p->d_scalar, (const int*)p->nbr,
           (const int8_t*)p->nnb, (const int8_t*)p->ledge, p->parent);
    GS_LAUNCH();
    for (int round = 0; round < 64; round++) {
        // two launches a round; the flag is cleared between them, so it tells
        // whether the second one still met a chain longer than JUMP_HOPS (a
        // launch in which every vertex reached its root leaves the roots)
        GS_CUDA(cudaMemsetAsync(p->i_scalar + I_CHANGED, 0, sizeof(int), p->stream));
        launch(p, k_jump, G, B, n, p->parent, p->i_scalar + I_CHANGED);
        GS_CUDA(cudaMemsetAsync(p->i_scalar + I_CHANGED, 0, sizeof(int), p->stream));
        launch(p, k_jump, G, B, n, p->parent, p->i_scalar + I_CHANGED);
        GS_LAUNCH();
        GS_TRY(read_ints(p, hbuf, p->i_scalar + I_CHANGED, 1));
        if (round == 0 && p->h_pinned[9]) {
            set_error(GS_ENONFINITE, check_b ? "non-finite elevation or rain volume (NaN or Inf)"
                                             : "non-finite elevation (NaN or Inf)");
            return GS_ENONFINITE;
        }
        if (!hbuf[0]) break;
        if (round == 63) { set_error(GS_EMAXITER, "pit fill: root search did not converge"); return GS_EMAXITER; }
    }
    // basin graph and minimax levels
    launch(p, k_basin_init, G, B, n, (const int*)p->parent, (const int8_t*)p->ledge, p->basinL);
    GS_CUDA(cudaMemsetAsync(p->i_scalar + I_NEXT, 0, sizeof(int), p->stream));
    launch(p, k_cross_edges, G, B, n, h, (const double*)p->d_scalar, (const int*)p->nbr,
           (const int8_t*)p->nnb, (const int8_t*)p->ledge, (const int*)p->parent, p->xe_u, p->xe_v,
           p->xe_w, p->i_scalar + I_NEXT, p->xe_cap);
    GS_LAUNCH();
    {
        // the edge count stays on the device: the deduplication and the
        // relaxation read it, and the host checks it against the capacity at
        // the next synchronisation
        const int* mc = p->i_scalar + I_NEXT;
        int cap = (int)std::min<int64_t>(p->xe_cap, INT_MAX), maxr = 1000000;
        int* raw = p->i_scalar + I_XRAW;
        int* mdc = p->i_scalar + I_XDEDUP;
        GS_CUDA(cudaMemsetAsync(p->i_scalar + I_XRAW, 0, sizeof(int) * 2, p->stream));
        GS_CUDA(cudaMemsetAsync(p->i_scalar + 5, 0, sizeof(int) * 3, p->stream));
        if (p->xh_cap > 0) {
            launch(p, k_xedge_insert, p->sm_count * 8, 256, mc, cap, (const int*)p->xe_u, (const int*)p->xe_v,
                   (const double*)p->xe_w, p->xh_key, p->xh_val, (long long)p->xh_cap, raw);
            launch(p, k_xedge_compact, p->sm_count * 8, 256, (long long)p->xh_cap, p->xh_key, p->xh_val, p->xd_u,
                   p->xd_v, p->xd_w, mdc);
            GS_LAUNCH();
        } else {
            // no table yet (first fill of the plan): the undeduplicated edges
            launch(p, k_fill_int, 1, 32, 1, raw, 1);
            GS_LAUNCH();
        }
        int* flags = p->i_scalar + 5;
        int* rout = p->i_scalar + I_CHANGED;
        void* args[] = {(void*)&mc,       (void*)&cap,      (void*)&raw,       (void*)&p->xe_u, (void*)&p->xe_v,
                        (void*)&p->xe_w,  (void*)&mdc,      (void*)&p->xd_u,   (void*)&p->xd_v, (void*)&p->xd_w,
                        (void*)&p->basinL, (void*)&flags,   (void*)&maxr,      (void*)&rout};
        GS_TRY(launch_coop(p, (const void*)k_relax_active, args));
        // the table's outcome, for its size at the next fill
        GS_CUDA(cudaMemcpyAsync(p->h_pinned + 11, p->i_scalar + I_XRAW, sizeof(int) * 2, cudaMemcpyDeviceToHost,
                                p->stream));
        GS_CUDA(cudaMemcpyAsync(p->h_pinned + 6, p->i_scalar + I_CHANGED, sizeof(int), cudaMemcpyDeviceToHost,
                                p->stream));
        GS_CUDA(cudaMemcpyAsync(p->h_pinned + 7, p->i_scalar + I_NEXT, sizeof(int), cudaMemcpyDeviceToHost,
                                p->stream));
    }
    launch(p, k_fill_final, G, B, n, h, (const double*)p->d_scalar, marine_sl, (const int8_t*)p->ledge,
           (const int*)p->parent, (const unsigned long long*)p->basinL, lfill);
    GS_LAUNCH();

    // label_pits: equal-fill components of cells above sea level
    launch(p, k_uf_init, G, B, n, (const double*)lfill, label_sl, (const int*)p->nbr, (const int8_t*)p->nnb,
           p->comp);
    launch(p, k_uf_link, G, B, n, (const double*)lfill, label_sl, (const int*)p->nbr,
           (const int8_t*)p->nnb, p->comp);
    launch(p, k_uf_flatten, G, B, n, p->comp);
    launch(p, k_fill_int, G, B, n, p->minseed, (int)INT_MAX);
    GS_LAUNCH();
    launch(p, k_minseed, G, B, n, (const double*)lfill, label_sl, (const int*)p->nbr,
           (const int8_t*)p->nnb, (const int*)p->comp, p->minseed);
    launch(p, k_seed_flag, G, B, n, (const double*)lfill, label_sl, (const int*)p->comp,
           (const int*)p->minseed, p->flagbuf);
    GS_LAUNCH();
    GS_TRY(exclusive_scan(p, p->flagbuf, p->scanbuf, n));
    GS_CUDA(cudaMemsetAsync(p->seg_keys, 0, sizeof(int) * (n + 1), p->stream));  // present[]
    launch(p, k_label, G, B, n, (const double*)lfill, label_sl, (const int*)p->comp,
           (const int*)p->minseed, (const int*)p->scanbuf, (const uint8_t*)p->outlet, p->lab,
           p->seg_keys);
    GS_LAUNCH();
    // consecutive ids over surviving labels (pits_cons)
    GS_TRY(exclusive_scan(p, p->seg_keys, p->seg_vals, n + 1));
    launch(p, k_relabel, G, B, n, (const int*)p->lab, (const int*)p->seg_vals, pit_ids);
    GS_LAUNCH();
    {
        int last[2];
        GS_CUDA(cudaMemcpyAsync(&last[0], p->seg_vals + n, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
        GS_CUDA(cudaMemcpyAsync(&last[1], p->seg_keys + n, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
        GS_CUDA(cudaStreamSynchronize(p->stream));
        p->npits = last[0] + last[1];
    }
    if ((int64_t)p->h_pinned[7] > p->xe_cap) {
        set_error(GS_ENOMEM, "pit fill: cross-edge capacity exceeded");
        return GS_ENOMEM;
    }
    // size the deduplication table for the next fill: four times this fill's
    // basin pairs (its edge count when the pairs are not known: no table yet,
    // or probing gave up), grown at once, shrunk only when 16 times too large
    {
        const bool known = p->xh_cap > 0 && !p->h_pinned[11];
        const int64_t pairs = known ? (int64_t)p->h_pinned[12] : (int64_t)p->h_pinned[7];
        const int64_t want = std::max<int64_t>(4 * pairs, 1 << 12);
        if (want > p->xh_cap || (known && p->xh_cap > 4 * want)) {
            int64_t cap = 1 << 12;
            while (cap < want) cap <<= 1;
            unsigned long long* ptrs[] = {p->xh_key, p->xh_val, p->xd_w};
            for (unsigned long long* q : ptrs)
                if (q) cudaFree(q);
            if (p->xd_u) cudaFree(p->xd_u);
            if (p->xd_v) cudaFree(p->xd_v);
            p->xh_key = p->xh_val = p->xd_w = nullptr;
            p->xd_u = p->xd_v = nullptr;
            p->xh_cap = 0;
            GS_CUDA(cudaMalloc((void**)&p->xh_key, sizeof(unsigned long long) * cap));
            GS_CUDA(cudaMalloc((void**)&p->xh_val, sizeof(unsigned long long) * cap));
            GS_CUDA(cudaMalloc((void**)&p->xd_u, sizeof(int) * cap));
            GS_CUDA(cudaMalloc((void**)&p->xd_v, sizeof(int) * cap));
            GS_CUDA(cudaMalloc((void**)&p->xd_w, sizeof(unsigned long long) * cap));
            GS_CUDA(cudaMemsetAsync(p->xh_key, 0xff, sizeof(unsigned long long) * cap, p->stream));
            GS_CUDA(cudaMemsetAsync(p->xh_val, 0xff, sizeof(unsigned long long) * cap, p->stream));
            p->xh_cap = cap;
        }
    }
    if (st) st->fill_rounds = p->h_pinned[6];
    const int P = p->npits, np1 = P + 1;
    if (st) st->npits = P;

    // spill points
    launch(p, k_fill_int, grid_for(np1, B), B, np1, p->bestlid, (int)INT_MAX);
    GS_CUDA(cudaMemsetAsync(p->spill_flag, 0, sizeof(int) * n, p->stream));
    launch(p, k_spill_qual, G, B, n, (const double*)lfill, (const int*)pit_ids, (const int*)p->nbr,
           (const int8_t*)p->nnb, (const uint8_t*)p->outlet, p->bestlid);
    launch(p, k_spill_pick, grid_for(np1, B), B, np1, n, (const double*)lfill, (const int*)pit_ids,
           (const int*)p->nbr, (const int8_t*)p->nnb, (const uint8_t*)p->outlet,
           (const int*)p->bestlid, p->pit_info, p->spill_flag);
    GS_LAUNCH();

    // seaID before the flat pass resets open-sea cells to h (the reset keeps
    // lFill <= sea level, so the mask is the same before and after it)
    if (sea_out) GS_TRY(sea_mask(p, lfill, sealevel, sea_out));

    // flat distances (fill_dir + nghb_dir fixed point = BFS hop distance).
    // The shared-memory BFS and the flat directions run on side_b, beside the
    // pit tables on the main stream: they share only read-only inputs, and
    // the sea reset of lFill in k_flat_dirs touches open-sea cells, which
    // hold no pit.
    GS_CUDA(cudaMemsetAsync(p->i_scalar + I_NEXT, 0, sizeof(int), p->stream));
    p->pdir_bound = 0;
    launch(p, k_bfs_init, G, B, n, (const int*)p->spill_flag, p->pdir, p->front0, p->i_scalar + I_NEXT);
    // the reachable set is compacted before the seed count is read, so one
    // synchronisation gives both (the compaction is wasted only without pits)
    launch(p, k_bfs_flag, G, B, n, (const int*)pit_ids, (const int*)p->spill_flag, p->flagbuf);
    GS_LAUNCH();
    GS_TRY(exclusive_scan(p, p->flagbuf, p->scanbuf, n));
    // pit cells, compacted in id order for the per-pit reductions below (they
    // read only the labels): their count comes back with the BFS counts
    GS_CUDA(cudaMemsetAsync(p->seg_count, 0, sizeof(int) * (np1 + 1), p->stream));
    launch(p, k_pit_flag, G, B, n, (const int*)pit_ids, p->pflag, p->seg_count);
    GS_LAUNCH();
    GS_TRY(exclusive_scan(p, p->pflag, p->pscan, n));
    launch(p, k_pit_compact, G, B, n, (const int*)pit_ids, (const int*)p->pscan, p->seg_keys, p->seg_vals);
    GS_LAUNCH();
    int last[5];
    GS_CUDA(cudaMemcpyAsync(&last[0], p->scanbuf + n - 1, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaMemcpyAsync(&last[1], p->flagbuf + n - 1, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaMemcpyAsync(&last[2], p->i_scalar + I_NEXT, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaMemcpyAsync(&last[3], p->pscan + n - 1, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaMemcpyAsync(&last[4], p->pflag + n - 1, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    const int ncell = last[3] + last[4];
    // pit cells sorted by (pit, id): segments for the per-pit reductions.
    // The ordered compaction (before the BFS) keeps id order; the stable
    // radix sort by pit then lists every pit's cells in increasing id.
    auto pit_tables = [&]() -> int {
        if (ncell > 0) {
            int bits = 1;
            while ((1 << bits) <= P && bits < 31) bits++;
            size_t bytes = p->cub_bytes;
            GS_CUDA(cub::DeviceRadixSort::SortPairs(p->cub_tmp, bytes, p->seg_keys, p->seg_keys2, p->seg_vals,
                                                    p->seg_vals2, ncell, 0, bits, p->stream));
            p->launches++;
        }
        GS_TRY(exclusive_scan(p, p->seg_count, p->seg_start, np1));
        GS_TRY(pit_chunks(p, np1, ncell));
        const int NI = p->pit_items_max;
        const int* nch = p->pit_nch;
        const int* chs = p->pit_chs;
        const int* itp = p->pit_item;
        launch(p, k_pit_params, NI, 256, np1, nch, chs, itp, (const int*)p->seg_start, (const int*)p->seg_count,
               (const int*)p->seg_vals2, (const double*)lfill, h, clip_sl, (const double*)p->larea, p->pit_part);
        launch(p, k_pit_params_fin, grid_for(np1, B), B, np1, nch, chs, (const double*)p->pit_part,
               p->pit_params);
        launch(p, k_filled_lvl, grid_for(np1, B), B, np1, (const double*)p->pit_params, p->filled_lvl);
        launch(p, k_filled_vol, NI, 256, np1, nch, chs, itp, (const int*)p->seg_start, (const int*)p->seg_count,
               (const int*)p->seg_vals2, h, clip_sl, (const double*)p->farea, (const double*)p->filled_lvl,
               p->pit_part);
        launch(p, k_filled_vol_fin, grid_for(np1, B), B, np1, nch, chs, (const double*)p->pit_part,
               (const double*)p->pit_params, p->filled_vol);
        GS_LAUNCH();
        return GS_OK;
    };
    // Without sediment the pit tables go first on the main stream, so that its
    // sort is queued before the host spends time queueing the flat pass on
    // side_b: the pit cells are above sea level and the flat pass rewrites
    // lFill only at open-sea cells, so the two read and write disjoint data.
    // The flat pass forks from here: it needs the compaction above, not the
    // pit tables.
    GS_CUDA(cudaEventRecord(p->ev_fork_b, p->stream));
    if (!sed) GS_TRY(pit_tables());
    int fsize = last[2], levels = 0;
    bool forked = false;
    if (fsize > 0) {
        const int M = last[0] + last[1];
        if (true) {
            GS_CUDA(cudaStreamWaitEvent(p->side_b, p->ev_fork_b, 0));
            {
                StreamSwap sw(p, p->side_b, nullptr);
                // packed adjacency rows: [count, ids...], stride S ints (16-byte multiple)
                const int S = ((p->W + 1 + 3) / 4) * 4;
                int* rows = p->bfs_rows;
                int* ldv = p->lab;
                GS_CUDA(cudaMemsetAsync(p->i_scalar + 6, 0, sizeof(int), p->stream));
                launch(p, k_bfs_local_build, G, B, n, S, (const double*)lfill, (const int*)pit_ids,
                       (const int*)p->flagbuf, (const int*)p->scanbuf, (const int*)p->nbr, (const int8_t*)p->nnb,
                       (const int*)p->spill_flag, rows, p->comp, ldv, p->front0, p->i_scalar + 6);
                GS_LAUNCH();
                const size_t smem1 = sizeof(unsigned) * (size_t)((M + 31) / 32) + sizeof(int) * 2 * LBFS_CAP;
                if (p->bfs_window > 0 || smem1 > 200 * 1024) {
                    GS_TRY(bfs_tiles(p, M, S, rows, ldv));
                } else {
                    // one block: visited bitmap and frontiers in shared memory
                    auto run = [&](auto kern) -> int {
                        GS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1));
                        cudaEvent_t stop = nullptr;
                        if (p->profiling) prof_begin(p, (const void*)kern, &stop);
                        kern<<<1, 1024, smem1, p->stream>>>(M, S, (const int*)rows, (const int*)p->front0,
                                                            p->i_scalar + 6, p->front1, p->minseed, ldv,
                                                            p->i_scalar + 4);
                        if (stop) cudaEventRecord(stop, p->stream);
                        return GS_OK;
                    };
                    const int S4 = S / 4;
                    if (S4 <= 1) GS_TRY(run(k_bfs_local<1>));
                    else if (S4 == 2) GS_TRY(run(k_bfs_local<2>));
                    else if (S4 == 3) GS_TRY(run(k_bfs_local<3>));
                    else GS_TRY(run(k_bfs_local<4>));
                    p->launches++;
                    GS_LAUNCH();
                }
                launch(p, k_bfs_local_scatter, grid_for(M, B), B, M, (const int*)p->comp, (const int*)ldv,
                       p->pdir);
                launch(p, k_flat_dirs, G, B, n, (const double*)lfill, (const int*)pit_ids, (const int*)p->pdir,
                       (const int*)p->nbr, (const int8_t*)p->nnb, (const int*)p->spill_flag, sealevel, h,
                       flat_dirs, lfill);
                GS_LAUNCH();
                GS_CUDA(cudaMemcpyAsync(p->h_pinned + 2, p->i_scalar + 4, sizeof(int), cudaMemcpyDeviceToHost,
                                        p->stream));
            }
            GS_CUDA(cudaEventRecord(p->ev_b, p->side_b));
            p->bfs_pending = 1;
            forked = true;
        } else {
            launch(p, k_bfs_adj, G, B, n, p->W, (const double*)lfill, (const int*)pit_ids,
                   (const int*)p->spill_flag, (const int*)p->nbr, (const int8_t*)p->nnb, p->xe_u, p->ledge);
            GS_LAUNCH();
            int* sizes = p->i_scalar + 5;
            GS_CUDA(cudaMemcpyAsync(sizes, p->i_scalar + I_NEXT, sizeof(int), cudaMemcpyDeviceToDevice, p->stream));
            GS_CUDA(cudaMemsetAsync(sizes + 1, 0, sizeof(int) * 2, p->stream));
            int d0 = 1, nn = n, W = p->W;
            int* lv = p->i_scalar + 4;
            void* args[] = {(void*)&p->front0, (void*)&p->front1, (void*)&sizes, (void*)&d0, (void*)&nn,
                            (void*)&W, (void*)&p->xe_u, (void*)&p->ledge, (void*)&p->pdir, (void*)&lv};
            GS_TRY(launch_coop(p, (const void*)k_bfs_coop, args));
            GS_TRY(read_ints(p, hbuf, p->i_scalar + 4, 1));
            levels = hbuf[0];
        }
    }
    if (!forked) {
        if (st) st->flat_rounds = levels;
        p->pdir_bound = levels + 2;
        launch(p, k_flat_dirs, G, B, n, (const double*)lfill, (const int*)pit_ids, (const int*)p->pdir,
               (const int*)p->nbr, (const int8_t*)p->nnb, (const int*)p->spill_flag, sealevel, h,
               flat_dirs, lfill);
        GS_LAUNCH();
    }

    // With sediment the open-sea reset of lFill in k_flat_dirs touches pit
    // cells (marine depressions are labelled), and the pit tables read the
    // reset lFill (pitfilling.py:820-846): join the BFS first.
    if (sed) {
        GS_TRY(fill_join(p, st));
        GS_TRY(pit_tables());
    }
    if (!defer_flats) GS_TRY(fill_join(p, st));
    return GS_OK;
}


// smallest per-SM residency of the cooperative kernels at 256 threads
int coop_occupancy(int* per_sm) {
    int a = 0, b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_bfs_coop, 256, 0) != cudaSuccess) return 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_relax_active, 256, 0) != cudaSuccess) return 1;
    int c = 0, d = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, k_cg_coop, 256, 0) != cudaSuccess) return 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d, k_cg_coop32, 256, 0) != cudaSuccess) return 1;
    *per_sm = a < b ? a : b;
    *per_sm = *per_sm < c ? *per_sm : c;
    *per_sm = *per_sm < d ? *per_sm : d;
    return 0;
}

}  // namespace gs
