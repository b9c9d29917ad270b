// Continental sediment routing and deposition in depressions: goSPL's
// SEDMesh.sedChange (gospl/sed/sedplex.py:1061-1086) for a landscape (or an
// ensemble of landscapes) with a single lithology and no provenance tracers.
//
//   1. _getSedFlux (sedplex.py:103-188): vSed = (I - W^T)^-1 (-Eb * area) over
//      the snapshot receivers of the preceding flow accumulation (fMati), one
//      ordered flow sweep.
//   2. fillElevation(sed=True): depressions of the eroded surface filled with
//      sediment (marine depressions included, pits labelled above the fill
//      level, volumes of the unclipped surface).
//   3. _distributeSediment / _moveDownstream (sedplex.py:190-522): per pass,
//      the sediment volume reaching each depression through its sink cells;
//      depressions that overflow are filled to their spill level (sedFilled),
//      their excess leaves through the spill node, the flow graph is rebuilt
//      on sedFilled (pit-flat routing, down=True) when a depression filled,
//      and the excess is routed downstream by an ordered flow sweep; flux on
//      cells not under a filled lake adds to vSed.  Terminal cells that are
//      not a depression keep their sediment on closed domains.  Ensemble
//      members (gs_plan_set_members) each run their own loop.
//   4. _updateSinks (sedplex.py:982-1059) paths 1 and 2: each depression that
//      received sediment gets a horizontal deposit surface at the level whose
//      filled volume matches the deposit (np.interp over its five-level
//      depth-volume table, restated below), tilted by 1e-6 m/m towards its
//      spill point (_addPitMicroTilt, sedplex.py:561-644).  Path 3 (partly
//      filled depressions of at least nlPitVolume and nlPitDepth, smoothed by
//      non-linear diffusion) is reported as an error.
#include <cub/cub.cuh>

#include <string>
#include <vector>

#include "gs_plan.cuh"

namespace gs {

// member helpers of the flow cascade (gs_flow.cu)
__global__ void k_pit_member(int np1, const int* __restrict__ seg_start, const int* __restrict__ seg_count,
                             const int* __restrict__ cells, const int* __restrict__ vmember, int* pmember);
__global__ void k_chunk_sum(const int* __restrict__ lo, const double* __restrict__ x, double* part);
__global__ void k_member_sum(int nmem, const int* __restrict__ m0, const double* __restrict__ part, double* out);
__global__ void k_lsink_keep(int n, const int* __restrict__ vmember, const uint8_t* __restrict__ mbig,
                             const uint8_t* __restrict__ prev, uint8_t* lsink);
__global__ void k_rhs_members(int n, const int* __restrict__ vmember, const uint8_t* __restrict__ msolve,
                              double* b);

namespace {

enum { S_POS = 1, S_BIG = 4 };

__global__ void k_sed_rhs(int n, const double* __restrict__ eb, const double* __restrict__ larea, double* b) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (-eb[i]) * larea[i];
}

__global__ void k_sed_init(int n, const double* __restrict__ vsed, const double* __restrict__ h, double dt,
                           double* vol, double* hl, double* sfill, double* closed) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    vol[i] = vsed[i] * dt;
    hl[i] = h[i];
    sfill[i] = h[i];
    closed[i] = 0.0;
}

__global__ void k_sed_pitvol(int np1, const double* __restrict__ params, double* vol) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < np1) vol[p] = params[3 * p];
}

// flow-terminal cells that are no depression: their sediment leaves the
// routed flux (kept in place on a closed domain)
__global__ void k_sed_csink(int n, const uint8_t* __restrict__ lsink, const int* __restrict__ pit,
                            const uint8_t* __restrict__ mout, const int* __restrict__ vmember,
                            const uint8_t* __restrict__ mact, double* vol, double* closed) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !lsink[i] || pit[i] >= 0) return;
    const int m = vmember[i];
    if (!mact[m]) return;
    if (!mout[m]) closed[i] = closed[i] + vol[i];
    vol[i] = 0.0;
}

__global__ void k_fill_int_s(int n, int* a, int v) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

// per-pit decisions of one _moveDownstream pass (sedplex.py:290-330); the
// pits of members whose loop has ended are not touched
__global__ void k_sed_pits(int np1, const double* __restrict__ inV, double* vol, const int* __restrict__ info,
                           const int* __restrict__ pmember, const uint8_t* __restrict__ mact, double* ev,
                           uint8_t* state, int* win, int* mflags) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np1) return;
    const int mem = pmember[p];
    if (!mact[mem]) {
        state[p] = 0;
        return;
    }
    const double in = inV[p];
    const double e = in - vol[p];
    ev[p] = e;
    uint8_t s = 0;
    int f = 0;
    if (e > 0.0) {
        f |= S_POS;
        s = 1;
        vol[p] = 0.0;
        // nvSed[spill] = eV: with a spill node shared by several pits the
        // highest pit id is written last
        if (info[2 * p + 1] == 0) atomicMax(&win[info[2 * p]], p);
    }
    if (e < 0.0) {
        double v = vol[p] - in;
        vol[p] = v < 0.0 ? 0.0 : v;
    }
    if (e > 1.0e-3) f |= S_BIG;
    state[p] = s;
    if (f) atomicOr(&mflags[mem], f);
}

__global__ void k_sed_spill(int np1, const double* __restrict__ ev, const uint8_t* __restrict__ state,
                            const int* __restrict__ info, const int* __restrict__ win, double* nv) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np1) return;
    if (state[p] == 1 && info[2 * p + 1] == 0 && win[info[2 * p]] == p) nv[info[2 * p]] = ev[p];
}

__global__ void k_sed_cells(int n, const int* __restrict__ pit, const uint8_t* __restrict__ state,
                            const double* __restrict__ lfill, double* sfill) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = pit[i];
    if (p >= 0 && state[p] == 1) sfill[i] = lfill[i];
}

// routed excess: next pass's volumes, and the flux outside filled lakes added
// to vSed (sedplex.py:443-451)
__global__ void k_sed_accum(int n, const double* __restrict__ routed, const double* __restrict__ hl,
                            const double* __restrict__ sfill, const uint8_t* __restrict__ outlet, double dt,
                            const int* __restrict__ vmember, const uint8_t* __restrict__ msolve, double* vol,
                            double* vsed) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !msolve[vmember[i]]) return;
    const double v = routed[i];
    const double keep = (hl[i] < sfill[i]) ? 0.0 : v;
    vsed[i] = vsed[i] + keep / dt;
    vol[i] = outlet[i] ? 0.0 : v;
}

// np.interp(x, xp, fp) for one scalar x and six increasing abscissae, as
// numpy's arr_interp evaluates it: outside the range the end values, at an
// abscissa its value, else slope * (x - xp[j]) + fp[j] with j the last
// abscissa <= x.
__device__ double interp6(double x, const double* xp, const double* fp) {
    if (x > xp[5]) return fp[5];
    if (x < xp[0]) return fp[0];
    int j = 0;
    for (int k = 1; k < 6; k++)
        if (xp[k] <= x) j = k;
    if (j == 5) return fp[5];
    if (xp[j] == x) return fp[j];
    const double slope = __ddiv_rn(__dsub_rn(fp[j + 1], fp[j]), __dsub_rn(xp[j + 1], xp[j]));
    double r = __dadd_rn(__dmul_rn(slope, __dsub_rn(x, xp[j])), fp[j]);
    if (r != r) {
        r = __dadd_rn(__dmul_rn(slope, __dsub_rn(x, xp[j + 1])), fp[j + 1]);
        if (r != r && fp[j] == fp[j + 1]) r = fp[j];
    }
    return r;
}

// _updateSinks path selection and _bottomUpDelta's lake level per pit
// (sedplex.py:524-559, 1000-1014)
__global__ void k_sed_depo(int np1, const double* __restrict__ params, const double* __restrict__ vol,
                           const double* __restrict__ fvol, const double* __restrict__ flvl, double nlv,
                           double nld, uint8_t* sel, double* target, double* pdepo, int* ndiffuse) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np1) return;
    const double pv = params[3 * p], pd = params[3 * p + 2];
    double depo = pv - vol[p];
    if (depo < 0.0) depo = 0.0;
    pdepo[p] = depo;
    const bool active = depo > 0.0;
    const bool full = active && depo >= pv - 1.0e-6;
    const bool partial = active && !full;
    const bool large = pv >= nlv && pd >= nld;
    const bool diffuse = partial && large;
    if (diffuse) atomicAdd(ndiffuse, 1);
    const bool bottomup = full || (partial && !large);
    // 1: bottom-up (paths 1, 2); 2: non-linear diffusion (path 3)
    sel[p] = bottomup ? 1 : (diffuse ? 2 : 0);
    double t = -INFINITY;
    if ((bottomup || diffuse) && depo > 0.0) {
        double xp[6], fp[6];
        xp[0] = 0.0;
        fp[0] = params[3 * p + 1] - params[3 * p + 2];
        for (int k = 0; k < 5; k++) {
            xp[k + 1] = fvol[5 * p + k];
            fp[k + 1] = flvl[5 * p + k];
        }
        t = interp6(depo, xp, fp);
    }
    target[p] = t;
}

__global__ void k_sed_closed(int n, const double* __restrict__ closed, const double* __restrict__ larea, double* h,
                             double* cum) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double c = closed[i];
    if (c > 0.0) {
        const double d = c / larea[i];
        cum[i] = cum[i] + d;
        h[i] = h[i] + d;
    }
}

// bottom-up deposit, and for the micro-tilt the distance of every deposit
// cell to its pit's spill point (sedplex.py:550-556, 601-608)
__global__ void k_sed_delta(int n, const int* __restrict__ pit, const uint8_t* __restrict__ sel,
                            const double* __restrict__ target, const double* __restrict__ lfill,
                            const double* __restrict__ hl, const double* __restrict__ xyz,
                            const int* __restrict__ info, double* delta, double* dist, uint8_t* tmask) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = pit[i];
    double d = 0.0;
    if (p >= 0 && sel[p] == 1) {
        const double t = target[p], f = lfill[i];
        const double surf = t < f ? t : f;
        const double v = __dsub_rn(surf, hl[i]);
        d = v > 0.0 ? v : 0.0;
    }
    delta[i] = d;
    const bool m = p >= 0 && sel[p] == 1 && d > 0.0;
    tmask[i] = m ? 1 : 0;
    double ds = 0.0;
    if (m) {
        double sx = 0.0, sy = 0.0, sz = 0.0;
        const int sp = info[2 * p];
        if (info[2 * p + 1] == 0 && sp >= 0) {
            sx = xyz[3 * (size_t)sp];
            sy = xyz[3 * (size_t)sp + 1];
            sz = xyz[3 * (size_t)sp + 2];
        }
        const double dx = __dsub_rn(xyz[3 * (size_t)i], sx);
        const double dy = __dsub_rn(xyz[3 * (size_t)i + 1], sy);
        const double dz = __dsub_rn(xyz[3 * (size_t)i + 2], sz);
        ds = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
    }
    dist[i] = ds;
}

// members with a draining outlet (sedplex.py:45-47, _domainHasOutlet per landscape)
__global__ void k_sed_moutlet(int nout, const int* __restrict__ outlet_ids, const int* __restrict__ vmember,
                              uint8_t* mout) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nout) mout[vmember[outlet_ids[t]]] = 1;
}

__global__ void k_sed_ones(int n, double* a) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = 1.0;
}

// tilt towards the spill with the per-pit mean distance removed, then the
// deposit joins h and cumED (sedplex.py:620-644, 1038-1043)
__global__ void k_sed_apply(int n, const int* __restrict__ pit, const uint8_t* __restrict__ tmask,
                            const double* __restrict__ dist, const double* __restrict__ dsum,
                            const double* __restrict__ dcnt, int tilt, const double* __restrict__ delta,
                            const double* __restrict__ ddiff, double* h, double* cum) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = delta[i];
    if (tilt && tmask[i]) {
        const int p = pit[i];
        const double c = dcnt[p];
        const double mean = c > 0.0 ? dsum[p] / (c > 1.0 ? c : 1.0) : 0.0;
        const double t = __dmul_rn(1.0e-6, __dsub_rn(dist[i], mean));
        d = __dadd_rn(d, t);
        if (d < 0.0) d = 0.0;
    }
    if (ddiff) d = __dadd_rn(d, ddiff[i]);
    cum[i] = cum[i] + d;
    h[i] = h[i] + d;
}

// ---- path 3: lake deposits smoothed by non-linear diffusion
// (_diffuseLargePit sedplex.py:679-858 with _diffuseImplicitPicard
// hillslope.py:988-1076)

// cells of path-3 pits, and the inlets among them: cells receiving flow
// (snapshot receivers) from a donor outside their pit (sedplex.py:646-677)
__global__ void k_lake_cells(int n, const int* __restrict__ pit, const uint8_t* __restrict__ sel, uint8_t* lmask,
                             uint8_t* inlet) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = pit[i];
    lmask[i] = (p >= 0 && sel[p] == 2) ? 1 : 0;
    inlet[i] = 0;
}

__global__ void k_lake_inlets(int n, int R, const int* __restrict__ pit, const uint8_t* __restrict__ sel,
                              const int* __restrict__ rcv, uint8_t* inlet) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int pi = pit[i];
    for (int k = 0; k < R; k++) {
        const int r = rcv[(size_t)k * n + i];
        if (r == i) continue;
        const int pr = pit[r];
        if (pr >= 0 && pr != pi && sel[pr] == 2) inlet[r] = 1;
    }
}

// pits without an inlet pile their inlet share on their highest cell (the
// first in id order among equals, as np.argmax)
__global__ void __launch_bounds__(256) k_lake_top(int np1, const int* __restrict__ start,
                                                  const int* __restrict__ counts, const int* __restrict__ cells,
                                                  const uint8_t* __restrict__ sel, const double* __restrict__ hl,
                                                  double* pcnt, uint8_t* inlet) {
    __shared__ double sv[256];
    __shared__ int si[256];
    const int p = blockIdx.x;
    if (p >= np1 || sel[p] != 2 || pcnt[p] > 0.0) return;
    const int s0 = start[p], c = counts[p];
    double bv = -INFINITY;
    int bi = INT_MAX;
    for (int t = threadIdx.x; t < c; t += 256) {
        const double v = hl[cells[s0 + t]];
        if (v > bv || (v == bv && t < bi)) { bv = v; bi = t; }
    }
    sv[threadIdx.x] = bv;
    si[threadIdx.x] = bi;
    __syncthreads();
    for (int s2 = 128; s2 > 0; s2 >>= 1) {
        if (threadIdx.x < s2) {
            const double v = sv[threadIdx.x + s2];
            const int i2 = si[threadIdx.x + s2];
            if (v > sv[threadIdx.x] || (v == sv[threadIdx.x] && i2 < si[threadIdx.x])) {
                sv[threadIdx.x] = v;
                si[threadIdx.x] = i2;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && si[0] != INT_MAX) {
        inlet[cells[s0 + si[0]]] = 1;
        pcnt[p] = 1.0;
    }
}

// water depth under the deposit level and its area-weighted volume terms
__global__ void k_lake_depth(int n, const int* __restrict__ pit, const uint8_t* __restrict__ lmask,
                             const double* __restrict__ target, const double* __restrict__ hl,
                             const double* __restrict__ larea, double* wd, double* wda) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double w = 0.0;
    if (lmask[i]) {
        const double v = __dsub_rn(target[pit[i]], hl[i]);
        w = v > 0.0 ? v : 0.0;
    }
    wd[i] = w;
    wda[i] = __dmul_rn(w, larea[i]);
}

// initial deposit: bathymetric share plus the inlet pile (sedplex.py:812-838)
__global__ void k_lake_init(int n, const int* __restrict__ pit, const uint8_t* __restrict__ lmask,
                            const uint8_t* __restrict__ inlet, const double* __restrict__ wd,
                            const double* __restrict__ denom, const double* __restrict__ pcnt,
                            const double* __restrict__ depo, const double* __restrict__ larea, double bias,
                            const double* __restrict__ zb, double* hcur) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = 0.0;
    const int p = pit[i];
    if (lmask[i]) {
        const double dn = denom[p];
        if (dn > 0.0) d = __ddiv_rn(__dmul_rn(__dmul_rn(1.0 - bias, depo[p]), wd[i]), dn > 1e-30 ? dn : 1e-30);
        if (inlet[i] && pcnt[p] > 0.0) {
            const double b = dn > 0.0 ? bias : 1.0;
            d = __dadd_rn(d, __ddiv_rn(__dmul_rn(b, depo[p]), __dmul_rn(pcnt[p], larea[i])));
        }
    }
    hcur[i] = __dadd_rn(d, zb[i]);
}

// diffusivity of the deposit: C_d = minDiff + K (1 - exp(-dexp dh)), dh below
// 0.1 m counted as 0, on the lake cells only (hillslope.py:1046-1051)
__global__ void k_lake_cd(int n, const uint8_t* __restrict__ lmask, const double* __restrict__ hcur,
                          const double* __restrict__ zb, double K, double dexp, double mind, double* cd) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double c = 0.0;
    if (lmask[i]) {
        double dd = __dsub_rn(hcur[i], zb[i]);
        if (dd < 0.1) dd = 0.0;
        c = __dadd_rn(mind, __dmul_rn(K, __dsub_rn(1.0, exp(__dmul_rn(-dexp, dd)))));
    }
    cd[i] = c;
}

// the lake cells as a sub-mesh: faces to other cells carry no diffusivity,
// so the rows outside are the identity and the solve decouples
__global__ void k_lake_flag(int n, const uint8_t* __restrict__ lmask, int* flag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = lmask[i] ? 1 : 0;
}

__global__ void k_lake_list(int n, const uint8_t* __restrict__ lmask, const int* __restrict__ lid, int* cell) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && lmask[i]) cell[lid[i]] = i;
}

__global__ void k_lake_submesh(int m, int n, int W, const int* __restrict__ cell, const int* __restrict__ lid,
                               const uint8_t* __restrict__ lmask, const int* __restrict__ nbr,
                               const int8_t* __restrict__ nnb, const double* __restrict__ farea, int* nbr_c,
                               int8_t* nnb_c, double* farea_c, uint8_t* fix_c) {
    int li = blockIdx.x * blockDim.x + threadIdx.x;
    if (li >= m) return;
    const int i = cell[li];
    nnb_c[li] = nnb[i];
    farea_c[li] = farea[i];
    fix_c[li] = farea[i] > 0.0 ? 0 : 1;
    for (int s = 0; s < W; s++) {
        const int j = nbr[(size_t)s * n + i];
        nbr_c[(size_t)s * m + li] = (j >= 0 && lmask[j]) ? lid[j] : -1;
    }
}

// rows of I + dt_sub L(C_d) for the lake cells: jacobiancoeff with Kp = 0
// (functions.F90:1423-1467), faces closed where either side has no
// diffusivity
__global__ void k_lake_rows_c(int m, int n, int W, const int* __restrict__ cell, const int* __restrict__ nbr,
                              const int8_t* __restrict__ nnb, const double* __restrict__ elen,
                              const double* __restrict__ vdist, const double* __restrict__ farea,
                              const double* __restrict__ cd, double dts, const double* __restrict__ hstart,
                              double* coef_c, double* rhs_c) {
    int li = blockIdx.x * blockDim.x + threadIdx.x;
    if (li >= m) return;
    const int k = cell[li];
    for (int s = 0; s < W; s++) coef_c[(size_t)(s + 1) * m + li] = 0.0;
    double dg = 0.0;
    const double ak = farea[k];
    if (ak > 0.0) {
        const double ck = cd[k];
        for (int s = 0; s < nnb[k]; s++) {
            const double vd = vdist[(size_t)s * n + k];
            if (!(vd > 0.0)) continue;
            const int j = nbr[(size_t)s * n + k];
            const double cn = cd[j];
            if (ck > 0.0 && cn > 0.0) {
                const double c = __ddiv_rn(__dmul_rn(0.5, __dadd_rn(ck, cn)), ak);
                const double v = __ddiv_rn(__dmul_rn(c, vd), elen[(size_t)s * n + k]);
                dg = __dadd_rn(dg, v);
                coef_c[(size_t)(s + 1) * m + li] = __dmul_rn(dts, -v);
            }
        }
    }
    coef_c[li] = __dadd_rn(__dmul_rn(dts, dg), 1.0);
    rhs_c[li] = hstart[k];
}

__global__ void k_lake_scatter(int m, const int* __restrict__ cell, const double* __restrict__ x_c, double* hcur) {
    int li = blockIdx.x * blockDim.x + threadIdx.x;
    if (li < m) hcur[cell[li]] = x_c[li];
}

// smoothed deposit (clipped at 0) and its area-weighted volume terms
__global__ void k_lake_depo(int n, const uint8_t* __restrict__ lmask, const double* __restrict__ hcur,
                            const double* __restrict__ zb, const double* __restrict__ larea, double* nd, double* nda) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = __dsub_rn(hcur[i], zb[i]);
    if (v < 0.0) v = 0.0;
    nd[i] = v;
    nda[i] = lmask[i] ? __dmul_rn(v, larea[i]) : 0.0;
}

// per-pit rescale to the deposited volume (sedplex.py:842-857)
__global__ void k_lake_scale(int n, const int* __restrict__ pit, const uint8_t* __restrict__ lmask,
                             const double* __restrict__ nd, const double* __restrict__ actual,
                             const double* __restrict__ depo, double* ddiff) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = 0.0;
    if (lmask[i]) {
        const int p = pit[i];
        const double a = actual[p];
        const double sc = a > 0.0 ? __ddiv_rn(depo[p], a > 1e-30 ? a : 1e-30) : 1.0;
        d = __dmul_rn(nd[i], sc);
    }
    ddiff[i] = d;
}

// --- sediment budget (gs_sed_budget) -------------------------------------
// Each reduction runs on LED_NB blocks whatever n is: a block walks a fixed
// strided set of indices, sums per thread in index order, then a fixed warp
// butterfly and warp order; k_led_final adds the block sums in block order.
// The result therefore depends on the data and n only.
constexpr int LED_NB = 296;
constexpr int LED_T = 256;

template <int C>
__device__ __forceinline__ void led_block(const double (&v)[C], double* part) {
    __shared__ double sh[C][LED_T / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < C; c++) {
        const double t = warp_sum(v[c]);
        if (lane == 0) sh[c][w] = t;
    }
    __syncthreads();
    if (threadIdx.x < C) {
        double t = 0.0;
        for (int k = 0; k < LED_T / 32; k++) t += sh[threadIdx.x][k];
        part[threadIdx.x * LED_NB + blockIdx.x] = t;
    }
}

// volumes u at the terminal cells of the graph wgt ([R][n], every weight 0),
// by kind: depression sinks, stray sinks kept (member without outlet), stray
// sinks dropped, open outlets, other terminal cells (sea)
__global__ void __launch_bounds__(LED_T) k_led_cells(int n, int R, const double* __restrict__ u,
                                                     const double* __restrict__ wgt, const uint8_t* __restrict__ lsink,
                                                     const int* __restrict__ pit, const uint8_t* __restrict__ outlet,
                                                     const uint8_t* __restrict__ mout, const int* __restrict__ vmember,
                                                     double* part) {
    double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int i = blockIdx.x * LED_T + threadIdx.x; i < n; i += LED_NB * LED_T) {
        bool term = true;
        for (int k = 0; k < R; k++)
            if (wgt[(size_t)k * n + i] != 0.0) term = false;
        if (!term) continue;
        const double x = u[i];
        if (outlet[i]) v[3] += x;
        else if (lsink[i]) {
            if (pit[i] >= 0) v[0] += x;
            else if (mout[vmember[i]]) v[2] += x;
            else v[1] += x;
        } else v[4] += x;
    }
    led_block<5>(v, part);
}

// one pass's split of the depressions' inflow, read before k_sed_pits
// updates pitVol: retained, excess (eV > 0), inflow with eV == 0, inflow
__global__ void __launch_bounds__(LED_T) k_led_pits(int np1, const double* __restrict__ inV,
                                                    const double* __restrict__ vol, const int* __restrict__ pmember,
                                                    const uint8_t* __restrict__ mact, double* part) {
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int q = blockIdx.x * LED_T + threadIdx.x; q < np1; q += LED_NB * LED_T) {
        if (!mact[pmember[q]]) continue;
        const double in = inV[q];
        const double e = in - vol[q];
        if (e > 0.0) {
            v[0] += vol[q];
            v[1] += e;
        } else if (e < 0.0) v[0] += in;
        else v[2] += in;
        v[3] += in;
    }
    led_block<4>(v, part);
}

// sum(x * scale), or sum((x - y) * scale) when y is given
__global__ void __launch_bounds__(LED_T) k_led_sum(int n, const double* __restrict__ x, const double* __restrict__ y,
                                                   const double* __restrict__ scale_v, double scale, double* part) {
    double v[1] = {0.0};
    for (int i = blockIdx.x * LED_T + threadIdx.x; i < n; i += LED_NB * LED_T) {
        double a = y ? (x[i] - y[i]) : x[i];
        a = scale_v ? a * scale_v[i] : a * scale;
        v[0] += a;
    }
    led_block<1>(v, part);
}

// led[slot + c] += sum of the block sums of category c, c < C, block order
__global__ void __launch_bounds__(LED_T) k_led_final(int C, const double* __restrict__ part, double* led, int slot) {
    __shared__ double sh[LED_T / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int c = 0; c < C; c++) {
        double t = 0.0;
        for (int b = threadIdx.x; b < LED_NB; b += LED_T) t += part[c * LED_NB + b];
        t = warp_sum(t);
        if (lane == 0) sh[w] = t;
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = 0.0;
            for (int k = 0; k < LED_T / 32; k++) a += sh[k];
            led[slot + c] += a;
        }
        __syncthreads();
    }
}

__global__ void k_sed_pitfinal(int np1, const double* __restrict__ vol, double* params) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < np1) params[3 * p] = vol[p];
}

}  // namespace

static int led_cells(gs_plan* p, const double* u, const double* wgt, const uint8_t* lsink, const int* pit,
                     const uint8_t* mout) {
    launch(p, k_led_cells, LED_NB, LED_T, (int)p->n, p->R, u, wgt, lsink, pit, (const uint8_t*)p->outlet, mout,
           (const int*)p->vmember, p->led_part);
    launch(p, k_led_final, 1, LED_T, 5, (const double*)p->led_part, p->led, (int)GS_LED_PIT_SINKS);
    GS_LAUNCH();
    return GS_OK;
}

static int led_sum(gs_plan* p, int n, const double* x, const double* y, const double* scale_v, double scale,
                   int slot) {
    launch(p, k_led_sum, LED_NB, LED_T, n, x, y, scale_v, scale, p->led_part);
    launch(p, k_led_final, 1, LED_T, 1, (const double*)p->led_part, p->led, slot);
    GS_LAUNCH();
    return GS_OK;
}

int sed_budget(gs_plan* p, double* out16) {
    GS_CUDA(cudaMemcpyAsync(out16, p->led, sizeof(double) * 16, cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    return GS_OK;
}

// picardSub x picardIts lagged-diffusivity backward-Euler solves of
// (I + dt_sub L(C_d(h))) h = h_start over the cells of lmask, faces to the
// other cells closed (_diffuseImplicitPicard, hillslope.py:988-1076, with
// C_d = 1e-4 + K (1 - exp(-0.05 (h - zb)))): hcur holds the start surface on
// entry and the result on return; cd and hstart are [n] scratch.  The cells
// of lmask form a sub-mesh of m rows, each solve is the cooperative CG on it.
int picard_diffuse(gs_plan* p, const uint8_t* lmask, const double* zb, double* hcur, double K, double dt,
                   double* cd, double* hstart) {
    const int n = (int)p->n;
    const int B = 256, G = grid_for(n, B);
    // the lake cells as a sub-mesh of m rows
    const int W = p->W;
    if (!p->sed_coef) GS_CUDA(cudaMalloc((void**)&p->sed_coef, sizeof(double) * (size_t)n * (size_t)(W + 1)));
    if (!p->lake_i) {
        GS_CUDA(cudaMalloc((void**)&p->lake_i, sizeof(int) * (size_t)n * (size_t)(W + 1)));
        GS_CUDA(cudaMalloc((void**)&p->lake_d, sizeof(double) * (size_t)n * 3));
        GS_CUDA(cudaMalloc((void**)&p->lake_u8, (size_t)n * 2));
    }
    int* cell = p->lake_i;
    int* nbr_c = cell + n;
    double* farea_c = p->lake_d;
    double* rhs_c = farea_c + n;
    double* x_c = rhs_c + n;
    int8_t* nnb_c = (int8_t*)p->lake_u8;
    uint8_t* fix_c = p->lake_u8 + n;
    launch(p, k_lake_flag, G, B, n, (const uint8_t*)lmask, p->flagbuf);
    GS_LAUNCH();
    {
        size_t bytes = p->cub_bytes;
        GS_CUDA(cub::DeviceScan::ExclusiveSum(p->cub_tmp, bytes, (const int*)p->flagbuf, p->scanbuf, n, p->stream));
        p->launches++;
    }
    int last[2];
    GS_CUDA(cudaMemcpyAsync(&last[0], p->scanbuf + n - 1, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaMemcpyAsync(&last[1], p->flagbuf + n - 1, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    const int m = last[0] + last[1];
    if (m == 0) return GS_OK;   // no cell to diffuse over: the surface stays
    launch(p, k_lake_list, G, B, n, (const uint8_t*)lmask, (const int*)p->scanbuf, cell);
    GS_LAUNCH();
    launch(p, k_lake_submesh, grid_for(m, B), B, m, n, W, (const int*)cell, (const int*)p->scanbuf,
           (const uint8_t*)lmask, (const int*)p->nbr, (const int8_t*)p->nnb, (const double*)p->farea, nbr_c, nnb_c,
           farea_c, fix_c);
    GS_LAUNCH();
    const double dts = dt / p->lake_nsub;
    // the solves' residuals are checked once, after the last one (they feed
    // only the device): no host round trip between two Picard iterations
    double* worst = p->d_scalar + 2;
    GS_CUDA(cudaMemsetAsync(worst, 0, sizeof(double), p->stream));
    for (int sub = 0; sub < p->lake_nsub; sub++) {
        GS_CUDA(cudaMemcpyAsync(hstart, hcur, sizeof(double) * n, cudaMemcpyDeviceToDevice, p->stream));
        for (int it = 0; it < p->lake_npic; it++) {
            launch(p, k_lake_cd, G, B, n, (const uint8_t*)lmask, (const double*)hcur, zb, K, 0.05, 1.0e-4,
                   cd);
            launch(p, k_lake_rows_c, grid_for(m, B), B, m, n, W, (const int*)cell, (const int*)p->nbr,
                   (const int8_t*)p->nnb, (const double*)p->elen, (const double*)p->vdist, (const double*)p->farea,
                   (const double*)cd, dts, (const double*)hstart, p->sed_coef, rhs_c);
            GS_LAUNCH();
            GS_TRY(diffusion_solve_on(p, m, nbr_c, nnb_c, farea_c, fix_c, 0, nullptr, p->sed_coef, rhs_c, x_c,
                                      1.0e-13, 5000, nullptr, nullptr, worst));
            launch(p, k_lake_scatter, grid_for(m, B), B, m, (const int*)cell, (const double*)x_c, hcur);
            GS_LAUNCH();
        }
    }
    double w = 0.0;
    GS_CUDA(cudaMemcpyAsync(&w, worst, sizeof(double), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    if (!(w == w)) {
        set_error(GS_ENONFINITE, "diffusion CG produced a non-finite residual");
        return GS_ENONFINITE;
    }
    if (w > 1.0e-13) {
        set_error(GS_EMAXITER, "diffusion CG reached max_iter");
        return GS_EMAXITER;
    }
    return GS_OK;
}

int sed_change(gs_plan* p, double* h, double* cum_ed, const double* eb, const double* xyz, double sealevel,
               double ofill, double dt, double nl_pit_volume, double nl_pit_depth, double* lfill, int* pit_ids,
               int* flat_dirs, const int* rcv_i, const double* wgt_i, uint8_t* lsink, uint8_t* sea,
               double* vsed, gs_stats* st) {
    const int n = (int)p->n;
    if (n == 0) return GS_OK;
    const int B = 256, G = grid_for(n, B);
    if (!p->sed_buf) GS_CUDA(cudaMalloc((void**)&p->sed_buf, sizeof(double) * (size_t)n * 10));
    if (!p->sed_mask) GS_CUDA(cudaMalloc((void**)&p->sed_mask, (size_t)n * 5));
    double* vol = p->sed_buf;
    double* nv = vol + n;
    double* routed = nv + n;
    double* closed = routed + n;
    double* hl = closed + n;
    double* sfill = hl + n;
    double* delta = sfill + n;
    double* dist = delta + n;
    double* sed_extra = dist + n;   // [2][n]
    uint8_t* sea_s = p->sed_mask;
    uint8_t* tmask = sea_s + n;
    uint8_t* mout = tmask + n;   // [nmem] (nmem <= n)
    if (!p->led) GS_CUDA(cudaMalloc((void**)&p->led, sizeof(double) * 16));
    if (!p->led_part) GS_CUDA(cudaMalloc((void**)&p->led_part, sizeof(double) * 5 * LED_NB));
    GS_CUDA(cudaMemsetAsync(p->led, 0, sizeof(double) * 16, p->stream));
    GS_CUDA(cudaMemsetAsync(mout, 0, (size_t)p->nmem, p->stream));
    if (p->n_outlet > 0)
        launch(p, k_sed_moutlet, grid_for(p->n_outlet, B), B, p->n_outlet, (const int*)p->outlet_ids,
               (const int*)p->vmember, mout);

    // 2. depressions of the eroded surface, filled with sediment (the flat
    // directions and the open-sea reset of lFill are joined inside)
    GS_TRY(fill_elevation(p, h, sealevel, ofill, lfill, pit_ids, flat_dirs, st, true, nullptr, true));
    const int P = p->npits, np1 = P + 1;

    // 1. sediment flux over the snapshot graph of the last flow accumulation
    int cyc = 0, total_cycles = 0;
    launch(p, k_sed_rhs, G, B, n, eb, (const double*)p->larea, p->q2);
    GS_LAUNCH();
    GS_TRY(flow_prepare(p, rcv_i, wgt_i, p->rslot_i, vsed, p->order_i, p->h_pinned + 3));
    GS_TRY(flow_run(p, rcv_i, wgt_i, p->rslot_i, p->q2, vsed, &cyc, p->order_i, p->order_i_valid, nullptr));
    total_cycles += cyc;
    // lsinki: sinks of the snapshot graph (flowplex.py:785-791)
    GS_TRY(sink_mask(p, wgt_i, sea, lsink));
    launch(p, k_sed_init, G, B, n, (const double*)vsed, (const double*)h, dt, vol, hl, sfill, closed);
    GS_LAUNCH();
    // budget: the eroded volume, and where the snapshot solve delivers it
    GS_TRY(led_sum(p, n, p->q2, nullptr, nullptr, dt, GS_LED_ERODED));
    GS_TRY(led_cells(p, vol, wgt_i, lsink, pit_ids, mout));

    launch(p, k_sed_pitvol, grid_for(np1, B), B, np1, (const double*)p->pit_params, p->pit_vol);
    GS_LAUNCH();

    // 3. cascade over the depressions.  Every member runs its own
    // _distributeSediment loop (sedplex.py:430-453): it leaves when it has no
    // excess left, and the pits, cells and sinks of members that left are not
    // touched by later passes of the others.
    const int nm = p->nmem;
    launch(p, k_pit_member, grid_for(np1, B), B, np1, (const int*)p->seg_start, (const int*)p->seg_count,
           (const int*)p->seg_vals2, (const int*)p->vmember, p->pmember);
    GS_LAUNCH();
    std::vector<uint8_t> act(nm, 1), big(nm), rebuild(nm), solve(nm);
    auto any = [](const std::vector<uint8_t>& v) {
        for (uint8_t x : v)
            if (x) return true;
        return false;
    };
    auto all = [](const std::vector<uint8_t>& v) {
        for (uint8_t x : v)
            if (!x) return false;
        return true;
    };
    int step = 0, solves = 0;
    bool rebuilt = false;
    while (any(act) && step < 5000) {
        GS_CUDA(cudaMemcpyAsync(p->mact, act.data(), nm, cudaMemcpyHostToDevice, p->stream));
        launch(p, k_sed_csink, G, B, n, (const uint8_t*)lsink, (const int*)pit_ids, (const uint8_t*)mout,
               (const int*)p->vmember, (const uint8_t*)p->mact, vol, closed);
        GS_LAUNCH();
        GS_TRY(group_sum_by_pit(p, pit_ids, lsink, vol, p->pit_in, P));
        GS_CUDA(cudaMemsetAsync(p->mflags, 0, sizeof(int) * nm, p->stream));
        launch(p, k_fill_int_s, G, B, n, p->pit_win, -1);
        launch(p, k_led_pits, LED_NB, LED_T, np1, (const double*)p->pit_in, (const double*)p->pit_vol,
               (const int*)p->pmember, (const uint8_t*)p->mact, p->led_part);
        launch(p, k_led_final, 1, LED_T, 4, (const double*)p->led_part, p->led, (int)GS_LED_RETAINED);
        launch(p, k_sed_pits, grid_for(np1, B), B, np1, (const double*)p->pit_in, p->pit_vol,
               (const int*)p->pit_info, (const int*)p->pmember, (const uint8_t*)p->mact, p->pit_ev, p->pit_state,
               p->pit_win, p->mflags);
        GS_LAUNCH();
        GS_CUDA(cudaMemcpyAsync(p->h_mflags, p->mflags, sizeof(int) * nm, cudaMemcpyDeviceToHost, p->stream));
        GS_CUDA(cudaStreamSynchronize(p->stream));
        int anyf = 0;
        for (int m = 0; m < nm; m++) {
            const int f = act[m] ? p->h_mflags[m] : 0;
            anyf |= f;
            big[m] = (f & S_BIG) ? 1 : 0;
            rebuild[m] = (big[m] && ((f & S_POS) || step == 0 || step == 100)) ? 1 : 0;
            solve[m] = 0;
        }
        GS_CUDA(cudaMemsetAsync(nv, 0, sizeof(double) * n, p->stream));
        if (anyf & S_POS) {
            launch(p, k_sed_spill, grid_for(np1, B), B, np1, (const double*)p->pit_ev, (const uint8_t*)p->pit_state,
                   (const int*)p->pit_info, (const int*)p->pit_win, nv);
            launch(p, k_sed_cells, G, B, n, (const int*)pit_ids, (const uint8_t*)p->pit_state, (const double*)lfill,
                   sfill);
            GS_LAUNCH();
            GS_TRY(led_sum(p, n, nv, nullptr, nullptr, 1.0, GS_LED_PLACED));
        }
        if (any(big)) {
            if (any(rebuild)) {
                // flow graph of the sediment-filled surface (down=True); the
                // sinks of members that do not rebuild are kept
                const bool every = all(rebuild);
                if (!every) {
                    GS_CUDA(cudaMemcpyAsync(p->lsink_prev, lsink, n, cudaMemcpyDeviceToDevice, p->stream));
                    GS_CUDA(cudaMemcpyAsync(p->mbig, rebuild.data(), nm, cudaMemcpyHostToDevice, p->stream));
                }
                const double* surf = (step == 100) ? lfill : sfill;
                rebuilt = true;
                GS_TRY(receivers(p, p->R, 1.1, surf, sealevel, p->gid, p->rcv, p->dist, p->wgt, p->rslot));
                GS_TRY(flow_order_from(p, surf, hl, p->order_i, p->order));
                GS_TRY(flow_order_ties_prepare(p));
                GS_TRY(fill_join(p, st));
                GS_TRY(flow_direction_post(p, surf, true, lfill, pit_ids, flat_dirs, sealevel, p->rcv, p->dist,
                                           p->wgt, p->rslot, lsink, sea_s));
                if (!every)
                    launch(p, k_lsink_keep, G, B, n, (const int*)p->vmember, (const uint8_t*)p->mbig,
                           (const uint8_t*)p->lsink_prev, lsink);
                GS_TRY(flow_order_ties(p, p->pdir, p->order));
            }
            // excess of each member (tmp.sum() > 0.5 maxarea, sedplex.py:349)
            launch(p, k_chunk_sum, p->nchunk, 256, (const int*)p->chunk_lo, (const double*)nv, p->chunk_part);
            launch(p, k_member_sum, grid_for(nm, 128), 128, nm, (const int*)p->mchunk0, (const double*)p->chunk_part,
                   p->mresid);
            GS_LAUNCH();
            GS_CUDA(cudaMemcpyAsync(p->h_mresid, p->mresid, sizeof(double) * nm, cudaMemcpyDeviceToHost, p->stream));
            GS_CUDA(cudaStreamSynchronize(p->stream));
            for (int m = 0; m < nm; m++) solve[m] = (big[m] && p->h_mresid[m] > 0.5 * p->mmaxarea[m]) ? 1 : 0;
            if (any(solve)) {
                GS_CUDA(cudaMemcpyAsync(p->msolve, solve.data(), nm, cudaMemcpyHostToDevice, p->stream));
                if (!all(solve))
                    launch(p, k_rhs_members, G, B, n, (const int*)p->vmember, (const uint8_t*)p->msolve, nv);
                GS_TRY(flow_prepare(p, p->rcv, p->wgt, p->rslot, routed, p->order, p->h_pinned));
                GS_CUDA(cudaStreamSynchronize(p->stream));
                const int ok = p->h_pinned[0] ? 0 : 1;
                GS_TRY(flow_run(p, p->rcv, p->wgt, p->rslot, nv, routed, &cyc, p->order, ok, nullptr));
                total_cycles += cyc;
                GS_TRY(led_sum(p, n, nv, nullptr, nullptr, 1.0, GS_LED_ROUTED));
                GS_TRY(led_cells(p, routed, p->wgt, lsink, pit_ids, mout));
                launch(p, k_sed_accum, G, B, n, (const double*)routed, (const double*)hl, (const double*)sfill,
                       (const uint8_t*)p->outlet, dt, (const int*)p->vmember, (const uint8_t*)p->msolve, vol, vsed);
                GS_LAUNCH();
                solves++;
            }
        }
        for (int m = 0; m < nm; m++) act[m] = solve[m];
        step++;
    }
    GS_TRY(fill_join(p, st));
    // a rebuild of the flow graph set goSPL's seaID (_buildFlowDirection,
    // flowplex.py:494): the caller's live sea mask follows it
    if (rebuilt) GS_CUDA(cudaMemcpyAsync(sea, sea_s, (size_t)n, cudaMemcpyDeviceToDevice, p->stream));

    // 4. deposits in the depressions
    if (!p->sed_pit) GS_CUDA(cudaMalloc((void**)&p->sed_pit, sizeof(double) * ((size_t)n + 1) * 2));
    double* pdepo = p->sed_pit;
    double* pcnt = pdepo + (n + 1);
    GS_CUDA(cudaMemsetAsync(p->i_scalar + 11, 0, sizeof(int), p->stream));
    launch(p, k_sed_depo, grid_for(np1, B), B, np1, (const double*)p->pit_params, (const double*)p->pit_vol,
           (const double*)p->filled_vol, (const double*)p->filled_lvl, nl_pit_volume, nl_pit_depth, p->pit_state,
           p->pit_lvl, pdepo, p->i_scalar + 11);
    GS_LAUNCH();
    int ndiff = 0;
    GS_CUDA(cudaMemcpyAsync(&ndiff, p->i_scalar + 11, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    if (st) {
        st->npits = P;
        st->cascade_passes = step;
        st->cascade_solves = solves;
        st->cycle_nodes = total_cycles;
        st->status = ndiff;
    }
    if (ndiff > 0 && !p->lake_on) {
        set_error(GS_EINVAL, "sedChange: " + std::to_string(ndiff) +
                                 " partly filled depressions reach nlPitVolume and nlPitDepth (deposit smoothed "
                                 "by non-linear diffusion): built for marineSolver picard only");
        return GS_EINVAL;
    }
    // sediment kept at closed terminal sinks (sedplex.py:486-500)
    GS_TRY(led_sum(p, n, closed, nullptr, nullptr, 1.0, GS_LED_KEPT_DEP));
    launch(p, k_sed_closed, G, B, n, (const double*)closed, (const double*)p->larea, h, cum_ed);
    launch(p, k_sed_ones, G, B, n, routed);
    GS_LAUNCH();
    double* ddiff = nullptr;
    if (ndiff > 0) {
        // path 3 on the surface after the closed-sink deposits (zb = h)
        uint8_t* lmask = mout + n;
        uint8_t* inlet = lmask + n;
        double* hcur = vol;
        double* hstart = nv;
        double* cd = closed;
        double* wd = sfill;
        double* wda = sed_extra;
        ddiff = sed_extra + n;
        const double* zb = h;
        if (!p->sed_coef)
            GS_CUDA(cudaMalloc((void**)&p->sed_coef, sizeof(double) * (size_t)n * (size_t)(p->W + 1)));
        launch(p, k_lake_cells, G, B, n, (const int*)pit_ids, (const uint8_t*)p->pit_state, lmask, inlet);
        launch(p, k_lake_inlets, G, B, n, p->R, (const int*)pit_ids, (const uint8_t*)p->pit_state, rcv_i, inlet);
        GS_LAUNCH();
        GS_TRY(group_sum_by_pit(p, pit_ids, inlet, routed, pcnt, P));
        launch(p, k_lake_top, np1, 256, np1, (const int*)p->seg_start, (const int*)p->seg_count,
               (const int*)p->seg_vals2, (const uint8_t*)p->pit_state, (const double*)hl, pcnt, inlet);
        launch(p, k_lake_depth, G, B, n, (const int*)pit_ids, (const uint8_t*)lmask, (const double*)p->pit_lvl,
               (const double*)hl, (const double*)p->larea, wd, wda);
        GS_LAUNCH();
        GS_TRY(group_sum_by_pit(p, pit_ids, lmask, wda, p->pit_in, P));
        launch(p, k_lake_init, G, B, n, (const int*)pit_ids, (const uint8_t*)lmask, (const uint8_t*)inlet,
               (const double*)wd, (const double*)p->pit_in, (const double*)pcnt, (const double*)pdepo,
               (const double*)p->larea, p->lake_bias, zb, hcur);
        GS_LAUNCH();
        GS_TRY(picard_diffuse(p, lmask, zb, hcur, p->lake_K, dt, cd, hstart));
        launch(p, k_lake_depo, G, B, n, (const uint8_t*)lmask, (const double*)hcur, zb, (const double*)p->larea, wd,
               wda);
        GS_LAUNCH();
        GS_TRY(group_sum_by_pit(p, pit_ids, lmask, wda, p->pit_ev, P));
        launch(p, k_lake_scale, G, B, n, (const int*)pit_ids, (const uint8_t*)lmask, (const double*)wd,
               (const double*)p->pit_ev, (const double*)pdepo, ddiff);
        GS_LAUNCH();
    }
    launch(p, k_sed_delta, G, B, n, (const int*)pit_ids, (const uint8_t*)p->pit_state, (const double*)p->pit_lvl,
           (const double*)lfill, (const double*)hl, xyz, (const int*)p->pit_info, delta, dist, tmask);
    GS_LAUNCH();
    GS_TRY(group_sum_by_pit(p, pit_ids, tmask, dist, p->pit_in, P));
    GS_TRY(group_sum_by_pit(p, pit_ids, tmask, routed, p->pit_ev, P));
    launch(p, k_sed_apply, G, B, n, (const int*)pit_ids, (const uint8_t*)tmask, (const double*)dist,
           (const double*)p->pit_in, (const double*)p->pit_ev, 1, (const double*)delta, (const double*)ddiff, h,
           cum_ed);
    launch(p, k_sed_pitfinal, grid_for(np1, B), B, np1, (const double*)p->pit_vol, p->pit_params);
    GS_LAUNCH();
    GS_TRY(led_sum(p, n, h, hl, (const double*)p->larea, 0.0, GS_LED_REALISED));
    return GS_OK;
}

}  // namespace gs
