// Marine deposition: goSPL's SEAMesh.seaChange (gospl/sed/seaplex.py:738-861)
// for one lithology, no stratigraphy or provenance, Gmar = 0 and the
// lagged-diffusivity (Picard) solve of the marine diffusion.
//
//   1. coastline: the sea-level contour of the elevation over the mesh edges
//      (marching triangles as vtkContourFilter, seaplex.py:105-120), and the
//      distance of every sea vertex to its nearest contour point
//      (_distanceCoasts, seaplex.py:51-135; a k-d tree in goSPL, here a
//      two-level box hierarchy over the Morton-sorted points, exact);
//   2. clinoform capacity maxDepQs from that distance and clinSlp, the
//      sediment volume reaching the sea (seaplex.py:753-783);
//   3. routing surface (_matOcean, seaplex.py:137-238): on spheres the
//      bathymetry smoothed by one implicit diffusion step with K_d = N area
//      (N = 1 land, 5 sea) and cells beyond `offshore` from the coast set to
//      the boundary sentinel, on planar meshes the elevation with the outlets
//      at the sentinel; then epsfill (functions.F90:2633-2697) and the
//      marine receivers mfdrcvrs (functions.F90:1673-1785): every strictly
//      lower neighbour with the weight 1/kk of the reference's single
//      precision literal;
//   4. the capacity-limited cascade (_distOcean, seaplex.py:404-619), one hop
//      per pass as in goSPL, pulls over the donors in ascending id;
//   5. deposit thickness (floored at 1e-3 m) smoothed by the Picard solve
//      over the sea cells (_diffuseOcean, hillslope.py:739-787).
#include <cub/cub.cuh>

#include <cfloat>

#include "gs_plan.cuh"

namespace gs {

namespace {

constexpr double SMOOTH_N_LAND = 1.0;      // gospl/tools/constants.py:126
constexpr double SMOOTH_N_SEA = 5.0;       // gospl/tools/constants.py:127
constexpr double FLOW_SENTINEL = -1.0e6;   // BOUNDARY_FLOW_SENTINEL, constants.py:90
constexpr double DEPOSIT_FLOOR = 1.0e-3;   // constants.py:58
constexpr int LEAF = 32;                   // coast points per leaf box
constexpr int SUPER = 32;                  // leaves per super box

// ---- 1. coastline ---------------------------------------------------------
// every mesh edge whose ends lie on both sides of the level (>= counts as
// inside) gives the point interpolated from its lower end
__global__ void k_coast_points(int ne, const int* __restrict__ edges, const double* __restrict__ xyz,
                               const double* __restrict__ s, double value, double* pts, int* cnt) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    const int a = edges[2 * e], b = edges[2 * e + 1];
    const double sa = s[a], sb = s[b];
    if ((sa >= value) == (sb >= value)) return;
    const bool up = (sb - sa) > 0.0;
    const int lo = up ? a : b, hi = up ? b : a;
    const double slo = up ? sa : sb, shi = up ? sb : sa;
    const double t = (value - slo) / (shi - slo);
    const int k = atomicAdd(cnt, 1);
    for (int d = 0; d < 3; d++) {
        const double xl = xyz[3 * (size_t)lo + d], xh = xyz[3 * (size_t)hi + d];
        pts[3 * (size_t)k + d] = xl + t * (xh - xl);
    }
}

__device__ __forceinline__ unsigned long long spread21(unsigned long long x) {
    x &= 0x1fffffULL;
    x = (x | (x << 32)) & 0x1f00000000ffffULL;
    x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
    x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
    x = (x | (x << 2)) & 0x1249249249249249ULL;
    return x;
}

__device__ __forceinline__ unsigned long long morton3(double x, double y, double z, const double* box) {
    unsigned long long q[3];
    const double v[3] = {x, y, z};
    for (int d = 0; d < 3; d++) {
        double u = (v[d] - box[d]) / box[3 + d] * 2097151.0;
        u = u < 0.0 ? 0.0 : (u > 2097151.0 ? 2097151.0 : u);
        q[d] = (unsigned long long)u;
    }
    return spread21(q[0]) | (spread21(q[1]) << 1) | (spread21(q[2]) << 2);
}

__global__ void k_coast_keys(int m, const double* __restrict__ pts, const double* __restrict__ box,
                             unsigned long long* key, int* idx) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    key[i] = morton3(pts[3 * (size_t)i], pts[3 * (size_t)i + 1], pts[3 * (size_t)i + 2], box);
    idx[i] = i;
}

__global__ void k_coast_gather(int m, const int* __restrict__ idx, const double* __restrict__ pts, double* sp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int j = idx[i];
    sp[i] = pts[3 * (size_t)j];
    sp[(size_t)m + i] = pts[3 * (size_t)j + 1];
    sp[2 * (size_t)m + i] = pts[3 * (size_t)j + 2];
}

// bounding box of every group of `g` consecutive items: items are points (src
// = coordinates [3][m]) or boxes (src = boxes [6][m])
__global__ void k_coast_boxes(int m, int g, int from_boxes, const double* __restrict__ src, double* box, int nb) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    const int i1 = min(m, (b + 1) * g);
    for (int i = b * g; i < i1; i++) {
        for (int d = 0; d < 3; d++) {
            const double a = from_boxes ? src[(size_t)d * m + i] : src[(size_t)d * m + i];
            const double c = from_boxes ? src[(size_t)(3 + d) * m + i] : a;
            lo[d] = a < lo[d] ? a : lo[d];
            hi[d] = c > hi[d] ? c : hi[d];
        }
    }
    for (int d = 0; d < 3; d++) {
        box[(size_t)d * nb + b] = lo[d];
        box[(size_t)(3 + d) * nb + b] = hi[d];
    }
}

// squared distance from q to a box (0 inside), a lower bound of the squared
// point distances inside it up to rounding
__device__ __forceinline__ double box_d2(const double* q, const double* box, int nb, int b) {
    double s = 0.0;
    for (int d = 0; d < 3; d++) {
        const double lo = box[(size_t)d * nb + b], hi = box[(size_t)(3 + d) * nb + b];
        const double e = q[d] < lo ? lo - q[d] : (q[d] > hi ? q[d] - hi : 0.0);
        s = s + e * e;
    }
    return s;
}

// squared Euclidean distance summed as the k-d tree sums it: (dx^2 + dy^2) + dz^2
__device__ __forceinline__ double pt_d2(const double* q, const double* sp, int m, int i) {
    const double dx = q[0] - sp[i], dy = q[1] - sp[(size_t)m + i], dz = q[2] - sp[2 * (size_t)m + i];
    return (dx * dx + dy * dy) + dz * dz;
}

// nearest coast point of every sea vertex: a first bound from the points
// next to the vertex's Morton key, then every super box and leaf box whose
// lower bound does not exceed the best distance (with a relative margin that
// covers the rounding of the bounds)
__global__ void k_coast_dist(int n, const uint8_t* __restrict__ sea, const double* __restrict__ xyz,
                             const double* __restrict__ box3, int m, const unsigned long long* __restrict__ skey,
                             const double* __restrict__ sp, int nleaf, const double* __restrict__ lbox, int nsup,
                             const double* __restrict__ sbox, double* dist) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (!sea[k] || m == 0) {
        dist[k] = 0.0;
        return;
    }
    const double q[3] = {xyz[3 * (size_t)k], xyz[3 * (size_t)k + 1], xyz[3 * (size_t)k + 2]};
    const unsigned long long key = morton3(q[0], q[1], q[2], box3);
    int lo = 0, hi = m;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (skey[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    double best = DBL_MAX;
    const int a0 = max(0, lo - LEAF), a1 = min(m, lo + LEAF);
    for (int i = a0; i < a1; i++) {
        const double d2 = pt_d2(q, sp, m, i);
        best = d2 < best ? d2 : best;
    }
    const double slack = 1.0 + 1.0e-12;
    for (int s = 0; s < nsup; s++) {
        if (box_d2(q, sbox, nsup, s) > best * slack) continue;
        const int l1 = min(nleaf, (s + 1) * SUPER);
        for (int l = s * SUPER; l < l1; l++) {
            if (box_d2(q, lbox, nleaf, l) > best * slack) continue;
            const int i1 = min(m, (l + 1) * LEAF);
            for (int i = l * LEAF; i < i1; i++) {
                const double d2 = pt_d2(q, sp, m, i);
                best = d2 < best ? d2 : best;
            }
        }
    }
    dist[k] = sqrt(best);
}

// ---- 2. clinoform capacity and the volume reaching the sea ----------------
__global__ void k_marine_capacity(int n, const double* __restrict__ hl, const double* __restrict__ lfill,
                                  const double* __restrict__ vsed, const double* __restrict__ cdist,
                                  const double* __restrict__ larea, double sealevel, double clinslp, double dt,
                                  double* maxdep, double* sedflux) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double h = hl[i];
    double c = (sealevel - 1.0e-3) - cdist[i] * clinslp;
    if (h >= sealevel) c = h;
    if (c < h) c = h;
    maxdep[i] = (c - h) * larea[i];
    double f = vsed[i] * dt;
    if (!(lfill[i] <= sealevel)) f = 0.0;
    if (f < 0.0) f = 0.0;
    sedflux[i] = f;
}

// ---- 3. routing surface ---------------------------------------------------
// rows of (I + L) with K_d = N area (N = 1 land, 5 sea): sethillslopecoeff
// (functions.F90:901-938) with a per-vertex coefficient, flat-model outlets
// held fixed as in hillslope.py:252-256
__global__ void k_smooth_rows(int n, int W, int flat, const uint8_t* __restrict__ sea,
                              const double* __restrict__ larea, const int* __restrict__ nbr,
                              const int8_t* __restrict__ nnb, const double* __restrict__ elen,
                              const double* __restrict__ vdist, const double* __restrict__ farea,
                              const uint8_t* __restrict__ outlet, double* coef) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double ck = (sea[k] ? SMOOTH_N_SEA : SMOOTH_N_LAND) * larea[k];
    double diag = 0.0;
    for (int s = 0; s < W; s++) coef[(size_t)(s + 1) * n + k] = 0.0;
    if (farea[k] > 0) {
        double s1 = 0.0;
        const double ak = farea[k];
        for (int s = 0; s < nnb[k]; s++) {
            const double vd = vdist[(size_t)s * n + k];
            if (vd > 0.0) {
                const int j = nbr[(size_t)s * n + k];
                const double cn = (sea[j] ? SMOOTH_N_SEA : SMOOTH_N_LAND) * larea[j];
                const double c = 0.5 * (ck + cn) / ak;
                const double v = c * vd / elen[(size_t)s * n + k];
                s1 = s1 + v;
                coef[(size_t)(s + 1) * n + k] = -v;
            }
        }
        diag = 1.0 + s1;
    }
    if (flat && outlet[k]) {
        diag = 1.0;
        for (int s = 0; s < W; s++) coef[(size_t)(s + 1) * n + k] = 0.0;
    }
    coef[k] = diag;
}

// smallest key of h (order-preserving encoding), for the routing level
__global__ void k_marine_min(int n, const double* __restrict__ h, unsigned long long* out) {
    unsigned long long best = ~0ULL;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned long long k = dkey(h[i]);
        best = k < best ? k : best;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long v = __shfl_xor_sync(0xffffffffu, best, o);
        best = v < best ? v : best;
    }
    if ((threadIdx.x & 31) == 0) atomicMin(out, best);
}

// surface to route over: far-offshore cells (spheres) or outlets (planar
// meshes) at the sentinel; the epsfill start: cells below the level are
// excluded, those of them next to a cell at or above it are the seeds
// (value kept), the others start unreached (+inf)
__global__ void k_marine_surface(int n, int flat, const double* __restrict__ base, const double* __restrict__ cdist,
                                 double offshore, const uint8_t* __restrict__ outlet,
                                 const unsigned long long* __restrict__ minkey, double ofill, double* z, double* lvl) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        double mh = dkey_inv(*minkey) + 0.1;
        lvl[0] = mh > ofill ? mh : ofill;
    }
    if (i >= n) return;
    double v = base[i];
    if (!flat && cdist[i] > offshore) v = FLOW_SENTINEL;
    if (flat && outlet[i]) v = FLOW_SENTINEL;
    z[i] = v;
}

__global__ void k_eps_init(int n, const double* __restrict__ z, const double* __restrict__ lvl,
                           const int* __restrict__ nbr, const int8_t* __restrict__ nnb, double* f, uint8_t* state) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double sl = lvl[0];
    const double zi = z[i];
    if (zi < sl) {
        bool seed = false;
        for (int s = 0; s < nnb[i]; s++) {
            const int c = nbr[(size_t)s * n + i];
            if (c >= 0 && z[c] >= sl) seed = true;
        }
        state[i] = seed ? 2 : 1;   // 2 seed (reached), 1 excluded
        f[i] = zi;
    } else {
        state[i] = 0;              // open: reached once its value is finite
        f[i] = INFINITY;
    }
}

// the next double above x (IEEE 754 nextUp; Fortran nearest(x, 1.0)):
// one step of the bit pattern away from or towards zero, the smallest
// subnormal above a zero
__device__ __forceinline__ double next_up(double x) {
    if (x != x || x == (double)INFINITY) return x;
    if (x == 0.0) return __longlong_as_double(1LL);
    const long long b = __double_as_longlong(x);
    return __longlong_as_double(x > 0.0 ? b + 1 : b - 1);
}

// epsfill as a fixpoint: f(c) = max(z(c), next double above the smallest f of
// its reached neighbours), iterated down from +inf; the Priority-Flood pops
// values in non-decreasing order and a cell takes its value from its first
// popped (= lowest reached) neighbour, so the fixpoint is its result
__global__ void k_eps_relax(int n, const double* __restrict__ z, const int* __restrict__ nbr,
                            const int8_t* __restrict__ nnb, const uint8_t* __restrict__ state, double* f,
                            int* changed) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n || state[c] != 0) return;
    double mn = INFINITY;
    for (int s = 0; s < nnb[c]; s++) {
        const int j = nbr[(size_t)s * n + c];
        if (j < 0 || state[j] == 1) continue;
        const double v = f[j];
        mn = v < mn ? v : mn;
    }
    if (mn == INFINITY) return;
    const double h = next_up(mn);
    const double zc = z[c];
    const double nf = zc > h ? zc : h;
    if (nf < f[c]) {
        f[c] = nf;
        *changed = 1;
    }
}

// unreached cells keep their surface; far-offshore cells (spheres) take the
// elevation back (seaplex.py:160-163)
__global__ void k_eps_final(int n, int flat, const double* __restrict__ z, const double* __restrict__ hl,
                            const double* __restrict__ cdist, double offshore, double* f) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (f[i] == INFINITY) f[i] = z[i];
    if (!flat && cdist[i] > offshore) f[i] = hl[i];
}

// mfdrcvrs with 12 receivers: every neighbour with (f_k - f_n)^e / L > 0
// (e = 1.1 above the sentinel, 0.01 at or below it) is a receiver, weight
// 1/kk computed in single precision; no candidate: a terminal sink.  Flat-
// model outlets pass nothing and are no sink.
__global__ void k_marine_rcv(int n, int flat, double expo, const double* __restrict__ f,
                             const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                             const double* __restrict__ elen, const uint8_t* __restrict__ outlet,
                             unsigned short* cand, double* w, uint8_t* sink) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double fk = f[k];
    const double e = fk > FLOW_SENTINEL ? expo : 0.01;
    unsigned m = 0u;
    int kk = 0;
    for (int s = 0; s < nnb[k]; s++) {
        const int c = nbr[(size_t)s * n + k];
        const double L = elen[(size_t)s * n + k];
        if (c < 0 || !(L > 0.0)) continue;
        const double val = pow(fk - f[c], e) / L;
        if (val > 0.0) {
            m |= 1u << s;
            kk++;
        }
    }
    const bool out = flat && outlet[k];
    cand[k] = out ? 0 : (unsigned short)m;
    w[k] = kk > 0 ? (double)__fdiv_rn(1.0f, (float)kk) : 0.0;
    sink[k] = (kk == 0 && !out) ? 1 : 0;
}

// ---- 4. capacity-limited cascade ------------------------------------------
__global__ void k_ocean_init(int n, const double* __restrict__ maxdep, const double* __restrict__ sedflux,
                             const uint8_t* __restrict__ sink, double* marvol, double* tmp, double* vdep) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    marvol[i] = maxdep[i];
    double v = sedflux[i];
    double d = 0.0;
    if (sink[i]) {
        d = v;
        v = 0.0;
    }
    vdep[i] = d;
    tmp[i] = v;
}

// one pass: the volumes move one hop down the marine receivers (pulled from
// the donors in ascending id, the order of the sorted transposed matrix), a
// cell keeps what fits in its remaining capacity, terminal sinks keep all,
// outlets lose all (seaplex.py:563-600)
__global__ void k_ocean_step(int n, int flat, const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                             const int8_t* __restrict__ rev, const unsigned long long* __restrict__ sorder,
                             const unsigned short* __restrict__ cand, const double* __restrict__ w,
                             const uint8_t* __restrict__ sink, const uint8_t* __restrict__ outlet,
                             const double* __restrict__ tmp, double* out, double* marvol, double* vdep,
                             const int* __restrict__ stop) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (*stop) {             // the loop has ended: keep the volumes in transit
        out[i] = tmp[i];
        return;
    }
    const unsigned long long so = sorder[i];
    double s = 0.0;
    for (int q = 0; q < nnb[i]; q++) {
        const int sl = (int)((so >> (4 * q)) & 15ULL);
        const int j = nbr[(size_t)sl * n + i];
        if (j < 0) continue;
        const int r = rev[(size_t)sl * n + i];
        if (r >= 0 && ((cand[j] >> r) & 1u)) s = s + w[j] * tmp[j];
    }
    const double mv = marvol[i];
    double d = vdep[i];
    if (s >= mv) {
        s = s - mv;
        d = d + mv;
        marvol[i] = 0.0;
    } else {
        marvol[i] = mv - s;
        d = d + s;
        s = 0.0;
    }
    if (flat && outlet[i]) {
        d = 0.0;
        s = 0.0;
    }
    if (sink[i]) {
        d = d + s;
        s = 0.0;
    }
    vdep[i] = d;
    out[i] = s;
}

__global__ void k_ocean_rest(int n, int flat, const uint8_t* __restrict__ outlet, const double* __restrict__ tmp,
                             double* vdep) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = vdep[i] + tmp[i];
    if (flat && outlet[i]) d = 0.0;
    vdep[i] = d;
}

// deposit thickness, floored (seaplex.py:845-849), and the Picard start
__global__ void k_marine_dh(int n, const double* __restrict__ vdep, const double* __restrict__ larea,
                            const double* __restrict__ h, double* zb, double* hcur) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double a = larea[i];
    double dh = a != 0.0 ? vdep[i] / a : 0.0;
    if (dh < DEPOSIT_FLOOR) dh = 0.0;
    zb[i] = h[i];
    hcur[i] = dh + h[i];
}

__global__ void k_marine_apply(int n, const double* __restrict__ hcur, const double* __restrict__ zb, double dt,
                               double* h, double* cum_ed, double* eb) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = hcur[i] - zb[i];
    if (d < 0.0) d = 0.0;
    cum_ed[i] = cum_ed[i] + d;
    h[i] = h[i] + d;
    eb[i] = eb[i] + d / dt;
}

// fixed-order sum over LED-like blocks: part[b] for 296 blocks, then one block
constexpr int SUM_NB = 296;

__global__ void __launch_bounds__(256) k_ocean_sum(int n, const double* __restrict__ x, double* part,
                                                   const int* __restrict__ stop) {
    __shared__ double sh[8];
    if (stop && *stop) return;
    double v = 0.0;
    for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += SUM_NB * 256) v += x[i];
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < 8; k++) t += sh[k];
        part[blockIdx.x] = t;
    }
}

// the volume in transit after a pass; with `stop`, also the loop control of
// _distOcean (seaplex.py:542-610): one more pass counted, and the loop ends
// once the volume is at most the threshold or 5000 passes have run
__global__ void __launch_bounds__(256) k_ocean_sum_final(const double* __restrict__ part, double* out, int* stop,
                                                         int* passes, const double* __restrict__ threshold) {
    __shared__ double sh[8];
    if (stop && *stop) return;
    double v = 0.0;
    for (int b = threadIdx.x; b < SUM_NB; b += 256) v += part[b];
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < 8; k++) t += sh[k];
        *out = t;
        if (stop) {
            const int ps = *passes + 1;
            *passes = ps;
            if (!(t > *threshold) || ps >= 5000) *stop = 1;
        }
    }
}

// ---- 4b. the coupled marine system ---------------------------------------
__global__ void k_marine_g(int n, const double* __restrict__ hl, double sealevel, double gmar, double* g) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = gmar > 0.99 ? 0.99 : gmar;
    if (hl[i] > sealevel) v = 0.0;
    g[i] = v;
}

// y = s x, times the area when `area` is given
__global__ void k_marine_scale(int n, double s, const double* __restrict__ x, const double* __restrict__ area,
                               double* y) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    y[i] = area ? area[i] * s * x[i] : s * x[i];
}

// y = G dt/A q, plus (1 - G) x when x is given
__global__ void k_marine_gsq(int n, const double* __restrict__ g, double dt, const double* __restrict__ area,
                             const double* __restrict__ q, const double* __restrict__ x, double* y) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double gi = g[i];
    double v = gi * dt / area[i] * q[i];
    if (x) v = (1.0 - gi) * x[i] + v;
    y[i] = v;
}

__global__ void k_marine_voldep(int n, const double* __restrict__ d, const double* __restrict__ area, double* v) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = d[i] * area[i];
    v[i] = x < 0.0 ? 0.0 : x;
}

}  // namespace

static int ocean_sum(gs_plan* p, const double* x, double* dev_out, double* host_out) {
    launch(p, k_ocean_sum, SUM_NB, 256, (int)p->n, x, p->red, (const int*)nullptr);
    launch(p, k_ocean_sum_final, 1, 256, (const double*)p->red, dev_out, (int*)nullptr, (int*)nullptr,
           (const double*)nullptr);
    GS_LAUNCH();
    GS_CUDA(cudaMemcpyAsync(host_out, dev_out, sizeof(double), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    return GS_OK;
}

// The coupled system reduced to the elevation change d = h_new - h:
// q = S [dep/dt + A/dt (h - h_new)] with S = (I - W^T)^-1 (row 2), so row 1
// reads (1 - G) d + G dt/A S[A/dt d] = G dt/A S[dep/dt]; one application is
// one ordered marine flow sweep.
struct MarineSystem : LinOp {
    gs_plan* p;
    int n;
    const double* g;
    double dt;
    const unsigned short* cand;
    const double* w;
    double* t1;
    double* t2;
    MarineSystem(gs_plan* p_, int n_, const double* g_, double dt_, const unsigned short* cand_, const double* w_,
                 double* t1_, double* t2_)
        : p(p_), n(n_), g(g_), dt(dt_), cand(cand_), w(w_), t1(t1_), t2(t2_) {}
    int apply(const double* x, double* y) override {
        const int B = 256, G = grid_for(n, B);
        launch(p, k_marine_scale, G, B, n, 1.0 / dt, x, (const double*)p->larea, t1);
        GS_LAUNCH();
        GS_TRY(sweep_marine(p, cand, w, p->order, t1, t2));
        launch(p, k_marine_gsq, G, B, n, g, dt, (const double*)p->larea, (const double*)t2, x, y);
        GS_LAUNCH();
        return GS_OK;
    }
};

int sea_change(gs_plan* p, double* h, double* cum_ed, double* eb, const double* xyz, const double* box,
               const int* edges, int64_t nedge, double sealevel, double ofill, double dt, double clinslp,
               double offshore, double nlk, double gmar, const double* lfill, const double* vsed,
               const uint8_t* sea, gs_stats* st) {
    const int n = (int)p->n;
    if (n == 0) return GS_OK;
    if (!p->lake_on) {
        set_error(GS_EINVAL, "seaChange: the marine diffusion is built for marineSolver picard only "
                             "(gs_plan_set_lake_diffusion with nsub > 0)");
        return GS_EINVAL;
    }
    const int B = 256, G = grid_for(n, B);
    const size_t N = (size_t)n;
    if (!p->sea_buf) GS_CUDA(cudaMalloc((void**)&p->sea_buf, sizeof(double) * N * 12));
    if (!p->sea_u8) GS_CUDA(cudaMalloc((void**)&p->sea_u8, N * 4));
    if (!p->sea_coef) GS_CUDA(cudaMalloc((void**)&p->sea_coef, sizeof(double) * N * (size_t)(p->W + 1)));
    // coastline buffers, in doubles: raw and sorted points [3 cap] each, keys
    // [2 cap], ids [2 cap] int32 (= cap), leaf boxes [6 (cap/LEAF + 1)],
    // super boxes [6 (cap/(LEAF SUPER) + 1)], then the sort's scratch
    auto pts_doubles = [](size_t cap) {
        return 3 * cap + 3 * cap + 2 * cap + cap + 6 * (cap / LEAF + 1) + 6 * (cap / (LEAF * SUPER) + 1) + 8;
    };
    if (p->sea_pts_cap < nedge) {
        if (p->sea_pts) cudaFree(p->sea_pts);
        p->sea_pts = nullptr;
        p->sea_pts_cap = 0;
        const size_t cap = (size_t)std::max<int64_t>(nedge, 1);
        size_t sb = 0;
        GS_CUDA(cub::DeviceRadixSort::SortPairs((void*)nullptr, sb, (const unsigned long long*)nullptr,
                                                (unsigned long long*)nullptr, (const int*)nullptr, (int*)nullptr,
                                                (int)cap, 0, 63, p->stream));
        p->sea_sort_bytes = (sb + 255) & ~(size_t)255;
        GS_CUDA(cudaMalloc((void**)&p->sea_pts, sizeof(double) * pts_doubles(cap) + p->sea_sort_bytes));
        p->sea_pts_cap = nedge;
    }
    double* cdist = p->sea_buf;
    double* maxdep = cdist + N;
    double* sedflux = maxdep + N;
    double* hsm = sedflux + N;
    double* zsurf = hsm + N;
    double* fz = zsurf + N;
    double* wgt = fz + N;
    double* marvol = wgt + N;
    double* tmpa = marvol + N;
    double* tmpb = tmpa + N;
    double* vdep = tmpb + N;
    double* hl = vdep + N;
    uint8_t* state = p->sea_u8;
    uint8_t* sink = state + N;
    unsigned short* cand = (unsigned short*)(sink + N);
    const size_t cap = (size_t)std::max<int64_t>(p->sea_pts_cap, 1);
    double* raw = p->sea_pts;
    double* spts = raw + 3 * cap;
    unsigned long long* key = (unsigned long long*)(spts + 3 * cap);
    unsigned long long* key2 = key + cap;
    int* idx = (int*)(key2 + cap);
    int* idx2 = idx + cap;
    double* lbox = (double*)(idx2 + cap);
    double* sbox = lbox + 6 * (cap / LEAF + 1);
    void* sort_tmp = (void*)(p->sea_pts + pts_doubles(cap));
    double* dbox = p->d_scalar + 8;   // [6] mesh box (lo, span)
    int* icnt = p->i_scalar + 10;
    GS_CUDA(cudaMemcpyAsync(hl, h, sizeof(double) * N, cudaMemcpyDeviceToDevice, p->stream));
    GS_CUDA(cudaMemcpyAsync(dbox, box, sizeof(double) * 6, cudaMemcpyHostToDevice, p->stream));

    // 1. coastline points, Morton-sorted, boxed; nearest distances
    GS_CUDA(cudaMemsetAsync(icnt, 0, sizeof(int), p->stream));
    if (nedge > 0)
        launch(p, k_coast_points, grid_for(nedge, B), B, (int)nedge, edges, xyz, (const double*)hl, sealevel, raw,
               icnt);
    GS_LAUNCH();
    int m = 0;
    GS_CUDA(cudaMemcpyAsync(&m, icnt, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    int nleaf = 0, nsup = 0;
    if (m > 0) {
        launch(p, k_coast_keys, grid_for(m, B), B, m, (const double*)raw, (const double*)dbox, key, idx);
        GS_LAUNCH();
        size_t bytes = 0;
        GS_CUDA(cub::DeviceRadixSort::SortPairs((void*)nullptr, bytes, key, key2, idx, idx2, m, 0, 63, p->stream));
        if (bytes > p->sea_sort_bytes || (size_t)m > cap) {
            set_error(GS_ENOMEM, "seaChange: more coastline points than the coastline buffers hold");
            return GS_ENOMEM;
        }
        bytes = p->sea_sort_bytes;
        GS_CUDA(cub::DeviceRadixSort::SortPairs(sort_tmp, bytes, key, key2, idx, idx2, m, 0, 63, p->stream));
        p->launches++;
        launch(p, k_coast_gather, grid_for(m, B), B, m, (const int*)idx2, (const double*)raw, spts);
        nleaf = (m + LEAF - 1) / LEAF;
        nsup = (nleaf + SUPER - 1) / SUPER;
        launch(p, k_coast_boxes, grid_for(nleaf, B), B, m, LEAF, 0, (const double*)spts, lbox, nleaf);
        launch(p, k_coast_boxes, grid_for(nsup, B), B, nleaf, SUPER, 1, (const double*)lbox, sbox, nsup);
        GS_LAUNCH();
    }
    launch(p, k_coast_dist, G, B, n, sea, xyz, (const double*)dbox, m, (const unsigned long long*)key2,
           (const double*)spts, nleaf, (const double*)lbox, nsup, (const double*)sbox, cdist);
    // 2. capacity and the volume reaching the sea
    launch(p, k_marine_capacity, G, B, n, (const double*)hl, lfill, vsed, (const double*)cdist,
           (const double*)p->larea, sealevel, clinslp, dt, maxdep, sedflux);
    GS_LAUNCH();

    // 3. routing surface: smoothed bathymetry (spheres), sentinel cells
    const double* base = hl;
    int smooth_iters = 0;
    if (!p->flat) {
        launch(p, k_smooth_rows, G, B, n, p->W, p->flat, sea, (const double*)p->larea, (const int*)p->nbr,
               (const int8_t*)p->nnb, (const double*)p->elen, (const double*)p->vdist, (const double*)p->farea,
               (const uint8_t*)p->outlet, p->sea_coef);
        GS_LAUNCH();
        // warm start from the last smoothing of this mesh: the residual
        // starts at the elevation change of a step, not at L h
        if (!p->sea_prev) {
            GS_CUDA(cudaMalloc((void**)&p->sea_prev, sizeof(double) * N));
            p->sea_prev_ok = 0;
        }
        GS_TRY(diffusion_solve_on(p, n, p->nbr, p->nnb, p->farea, p->dfix, p->flat, p->outlet, p->sea_coef, hl, hsm,
                                  1.0e-14, 5000, &smooth_iters, (p->sea_prev_ok && p->warm_start) ? (const double*)p->sea_prev : nullptr));
        GS_CUDA(cudaMemcpyAsync(p->sea_prev, hsm, sizeof(double) * N, cudaMemcpyDeviceToDevice, p->stream));
        p->sea_prev_ok = p->warm_start;
        base = hsm;
    }
    unsigned long long* mk = p->u_scalar + 6;
    GS_CUDA(cudaMemsetAsync(mk, 0xff, sizeof(unsigned long long), p->stream));
    launch(p, k_marine_min, p->sm_count * 4, 256, n, (const double*)hl, mk);
    double* lvl = p->d_scalar + 14;
    launch(p, k_marine_surface, G, B, n, p->flat, base, (const double*)cdist, offshore, (const uint8_t*)p->outlet,
           (const unsigned long long*)mk, ofill, zsurf, lvl);
    launch(p, k_eps_init, G, B, n, (const double*)zsurf, (const double*)lvl, (const int*)p->nbr,
           (const int8_t*)p->nnb, fz, state);
    GS_LAUNCH();
    // relaxation to the fixpoint, checked every 8 passes (extra passes change nothing)
    int* chg = p->i_scalar + 10;
    int passes = 0;
    for (;;) {
        GS_CUDA(cudaMemsetAsync(chg, 0, sizeof(int), p->stream));
        for (int r = 0; r < 8; r++)
            launch(p, k_eps_relax, G, B, n, (const double*)zsurf, (const int*)p->nbr, (const int8_t*)p->nnb,
                   (const uint8_t*)state, fz, chg);
        GS_LAUNCH();
        passes += 8;
        int c = 0;
        GS_CUDA(cudaMemcpyAsync(&c, chg, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
        GS_CUDA(cudaStreamSynchronize(p->stream));
        if (!c) break;
        if (passes > 8 * n + 64) {
            set_error(GS_EMAXITER, "seaChange: epsfill relaxation did not settle");
            return GS_EMAXITER;
        }
    }
    launch(p, k_eps_final, G, B, n, p->flat, (const double*)zsurf, (const double*)hl, (const double*)cdist,
           offshore, fz);
    launch(p, k_marine_rcv, G, B, n, p->flat, 1.1, (const double*)fz, (const int*)p->nbr, (const int8_t*)p->nnb,
           (const double*)p->elen, (const uint8_t*)p->outlet, cand, wgt, sink);
    GS_LAUNCH();

    // 4. the cascade: until the volume in transit is at most max(1, 1e-6 of
    // the input) or 5000 passes (seaplex.py:542-610); every call starts from
    // the full capacity (marvol = maxDepQs) with the given input volumes, and
    // deposits into vdep
    double* sres = p->d_scalar + 15;
    int* stop = p->i_scalar + 10;
    int* dpass = p->i_scalar + 11;
    double* dthr = p->d_scalar + 7;
    int step = 0;
    auto cascade = [&](const double* input) -> int {
        launch(p, k_ocean_init, G, B, n, (const double*)maxdep, input, (const uint8_t*)sink, marvol, tmpa, vdep);
        GS_LAUNCH();
        double sum = 0.0;
        GS_TRY(ocean_sum(p, tmpa, sres, &sum));
        const double threshold = std::max(1.0, 1.0e-6 * sum);
        // the loop control lives on the device (stop flag, pass count):
        // passes are queued eight at a time and those after the stop only
        // carry the volumes over, so the host synchronises once per eight
        {
            const int h0[2] = {(sum > threshold) ? 0 : 1, 0};
            GS_CUDA(cudaMemcpyAsync(stop, h0, sizeof(int) * 2, cudaMemcpyHostToDevice, p->stream));
            GS_CUDA(cudaMemcpyAsync(dthr, &threshold, sizeof(double), cudaMemcpyHostToDevice, p->stream));
        }
        double* cur = tmpa;
        double* nxt = tmpb;
        int hs[2] = {(sum > threshold) ? 0 : 1, 0};
        while (!hs[0]) {
            for (int q = 0; q < 8; q++) {
                launch(p, k_ocean_step, G, B, n, p->flat, (const int*)p->nbr, (const int8_t*)p->nnb,
                       (const int8_t*)p->rev, (const unsigned long long*)p->sorder, (const unsigned short*)cand,
                       (const double*)wgt, (const uint8_t*)sink, (const uint8_t*)p->outlet, (const double*)cur, nxt,
                       marvol, vdep, (const int*)stop);
                launch(p, k_ocean_sum, SUM_NB, 256, n, (const double*)nxt, p->red, (const int*)stop);
                launch(p, k_ocean_sum_final, 1, 256, (const double*)p->red, sres, stop, dpass, (const double*)dthr);
                std::swap(cur, nxt);
            }
            GS_LAUNCH();
            GS_CUDA(cudaMemcpyAsync(hs, stop, sizeof(int) * 2, cudaMemcpyDeviceToHost, p->stream));
            GS_CUDA(cudaStreamSynchronize(p->stream));
        }
        step = hs[1];
        // what is still in transit stays where it is
        launch(p, k_ocean_rest, G, B, n, p->flat, (const uint8_t*)p->outlet, (const double*)cur, vdep);
        GS_LAUNCH();
        return GS_OK;
    };
    GS_TRY(cascade(sedflux));

    // 4b. the coupled marine system (Gmar > 0 on spheres, seaplex.py:240-402):
    // its deposit, negatives dropped, goes down the cascade again
    int gm_applies = 0;
    if (!p->flat && gmar > 0.0) {
        double* G_ = marvol;     // G = min(gmar, 0.99) below sea level (marvol is reset by the next cascade)
        double* dd = hsm;        // the elevation change d = h_new - h
        double* r0 = zsurf;
        double* t1 = tmpa;
        double* t2 = tmpb;
        launch(p, k_marine_g, G, B, n, (const double*)hl, sealevel, gmar, G_);
        GS_LAUNCH();
        GS_TRY(flow_order(p, fz, p->order));
        // r0 = G dt/A S[dep / dt]
        launch(p, k_marine_scale, G, B, n, 1.0 / dt, (const double*)vdep, (const double*)nullptr, t1);
        GS_LAUNCH();
        GS_TRY(sweep_marine(p, cand, wgt, p->order, t1, t2));
        launch(p, k_marine_gsq, G, B, n, (const double*)G_, dt, (const double*)p->larea, (const double*)t2,
               (const double*)nullptr, r0);
        GS_CUDA(cudaMemsetAsync(dd, 0, sizeof(double) * N, p->stream));
        GS_LAUNCH();
        MarineSystem op(p, n, G_, dt, cand, wgt, t1, t2);
        double relres = 0.0;
        const int gst = gmres_solve(p, op, r0, dd, 1.0e-13, 400, &gm_applies, &relres);
        if (gst == GS_EMAXITER) {
            set_error(GS_EMAXITER, "seaChange: the coupled marine system did not converge");
            return GS_EMAXITER;
        }
        GS_TRY(gst);
        // volDep = max(d A, 0), the input of the second cascade
        launch(p, k_marine_voldep, G, B, n, (const double*)dd, (const double*)p->larea, sedflux);
        GS_LAUNCH();
        GS_TRY(cascade(sedflux));
    }

    // 5. thickness, Picard diffusion over the sea cells, updates
    double* zb = tmpb;     // free once the cascade has deposited what was in transit
    double* hcur = hsm;
    double* cd = zsurf;
    double* hstart = marvol;
    launch(p, k_marine_dh, G, B, n, (const double*)vdep, (const double*)p->larea, (const double*)h, zb, hcur);
    GS_LAUNCH();
    GS_TRY(picard_diffuse(p, sea, zb, hcur, nlk, dt, cd, hstart));
    launch(p, k_marine_apply, G, B, n, (const double*)hcur, (const double*)zb, dt, h, cum_ed, eb);
    GS_LAUNCH();
    if (st) {
        st->cascade_passes = step;
        st->fill_rounds = passes;
        st->npits = m;
        st->cg_iters = gm_applies;
        st->flat_rounds = smooth_iters;
    }
    return GS_OK;
}

}  // namespace gs
