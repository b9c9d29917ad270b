// Implicit linear stream-power erosion, n = 1, G = 0:
// SPL._eroMats (gospl/eroder/SPL.py:45-114), _getEroDepRate (260-366) and
// erodepSPL (402-454).  The PETSc KSP solve of SPL.py:297 is replaced by the
// exact receivers-first dataflow sweep (gs_sweep.cu).
#include "gs_plan.cuh"

namespace gs {

// numpy's array ** scalar fast paths (exponent -1, 0, 0.5, 1, 2), else pow
__device__ __forceinline__ double np_scalar_pow(double x, double e) {
    if (e == 0.0) return 1.0;
    if (e == 0.5) return sqrt(x);
    if (e == 1.0) return x;
    if (e == 2.0) return x * x;
    if (e == -1.0) return 1.0 / x;
    return pow(x, e);
}

__global__ void k_spl_coef(int n, int R, const double* __restrict__ hold, const double* __restrict__ fal,
                           const double* __restrict__ rain, double k_scalar,
                           const double* __restrict__ k_field, double d, double m, double dt,
                           const int* __restrict__ rcv, const double* __restrict__ dist,
                           const double* __restrict__ wgt, const uint8_t* __restrict__ sea, double* c) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double K = k_field ? k_field[i] : k_scalar;
    double kbr = K * np_scalar_pow(rain[i], d);
    kbr = kbr * (dt * np_scalar_pow(fal[i], m));
    const bool s = sea[i] != 0;
    if (s) kbr = 0.0;
    const double hi = hold[i];
    for (int k = 0; k < R; k++) {
        int r = rcv[(size_t)k * n + i];
        double w = s ? 0.0 : wgt[(size_t)k * n + i];
        double dh = hi - hold[r];
        double lim = (dh != 0.0) ? dh / (dh + 1.0e-2) : 0.0;
        double ds = dist[(size_t)k * n + i];
        double data = (ds != 0.0) ? (kbr * lim) / ds : 0.0;
        double ck = data * w;
        if (r == i) ck = 0.0;
        c[(size_t)k * n + i] = ck;
    }
}

__global__ void k_spl_update(int n, int flat, const uint8_t* __restrict__ outlet,
                             const uint8_t* __restrict__ lsink, const double* __restrict__ hold,
                             const double* __restrict__ s, double dt, double* h, double* cum_ed,
                             double* eb) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double E = (s[i] - hold[i]) / dt;
    if (flat && outlet[i]) E = 0.0;
    if (lsink[i]) E = 0.0;
    double dz = E * dt;
    cum_ed[i] = cum_ed[i] + dz;
    h[i] = hold[i] + dz;
    eb[i] = dz / dt;
}

__global__ void k_copy_d(int n, const double* __restrict__ a, double* b) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i];
}

int erodep_spl(gs_plan* p, double* h, double* cum_ed, double* eb, const double* fal,
               const double* rain, double k_scalar, const double* k_field, double d, double m,
               double dt, const int* rcv_i, const double* dist_i, const double* wgt_i,
               const uint8_t* lsink, const uint8_t* sea, gs_stats* st) {
    const int n = (int)p->n;
    if (n == 0) return GS_OK;
    const int B = 256, G = grid_for(n, B);
    double* hold = p->hl;
    launch(p, k_copy_d, G, B, n, (const double*)h, hold);
    launch(p, k_spl_coef, G, B, n, p->R, (const double*)hold, fal, rain, k_scalar, k_field, d, m, dt,
           rcv_i, dist_i, wgt_i, sea, p->c);
    GS_LAUNCH();
    int cyc = 0;
    GS_TRY(spl_sweep(p, rcv_i, p->c, p->rslot_i, hold, p->q3, &cyc, true));
    GS_TRY(rec_spl(p, p->q3, lsink));
    launch(p, k_spl_update, G, B, n, p->flat, (const uint8_t*)p->outlet, lsink, (const double*)hold,
           (const double*)p->q3, dt, h, cum_ed, eb);
    GS_LAUNCH();
    (void)st;
    return GS_OK;
}

// ---------------------------------------------------------------------------
// Adjoint of erodepSPL for fixed receivers and masks.  Forward: c_ik =
// (Kbr_i lim_ik / ds_ik) w_ik, Kbr_i = K_i rain_i^d dt FAL_i^m, lim = dh /
// (dh + 0.01), dh = hOld_i - hOld_r; M(c) s = hOld; h = s except at flat
// outlets and live sinks (h = hOld).  Given y = M^-T (dJ/ds) this kernel
// forms, per vertex and receiver edge, dJ/dc = -y_i (s_i - s_r) and its
// chain: dJ/dK (accumulated), dJ/dFAL (written), dJ/drain (accumulated),
// dJ/dw (written, [R][n]), and the lim part of dJ/dhOld: own vertex
// (ghs, written) and receiver ([R][n] ghr, written, gathered later).
__global__ void k_spl_adj(int n, int R, const double* __restrict__ hold, const double* __restrict__ s,
                          const double* __restrict__ y, const double* __restrict__ fal,
                          const double* __restrict__ rain, double k_scalar, const double* __restrict__ k_field,
                          double d, double m, double dt, const int* __restrict__ rcv,
                          const double* __restrict__ dist, const double* __restrict__ wgt,
                          const uint8_t* __restrict__ sea, double* gK, double* gfal, double* grain, double* gw,
                          double* ghs, double* ghr) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = 0; k < R; k++) {
        gw[(size_t)k * n + i] = 0.0;
        ghr[(size_t)k * n + i] = 0.0;
    }
    ghs[i] = 0.0;
    gfal[i] = 0.0;
    if (sea[i]) return;   // Kbr = 0 and w = 0 on open sea: no dependence
    const double K = k_field ? k_field[i] : k_scalar;
    const double rd = np_scalar_pow(rain[i], d);
    const double fm = np_scalar_pow(fal[i], m);
    const double kbr = (K * rd) * (dt * fm);
    const double hi = hold[i], si = s[i], yi = y[i];
    double gkbr = 0.0, gself = 0.0;
    for (int k = 0; k < R; k++) {
        int r = rcv[(size_t)k * n + i];
        if (r == i) continue;
        double w = wgt[(size_t)k * n + i];
        double dh = hi - hold[r];
        double lim = (dh != 0.0) ? dh / (dh + 1.0e-2) : 0.0;
        double dlim = 1.0e-2 / ((dh + 1.0e-2) * (dh + 1.0e-2));
        double ds = dist[(size_t)k * n + i];
        if (ds == 0.0) continue;
        double gc = -yi * (si - s[r]);
        double data = (kbr * lim) / ds;
        gkbr += gc * (lim / ds) * w;
        double glim = gc * (kbr / ds) * w;
        gw[(size_t)k * n + i] = gc * data;
        gself += glim * dlim;
        ghr[(size_t)k * n + i] = -glim * dlim;
    }
    ghs[i] = gself;
    if (gK) gK[i] += gkbr * rd * (dt * fm);
    if (fal[i] > 0.0 && m != 0.0) gfal[i] = gkbr * K * rd * dt * m * pow(fal[i], m - 1.0);
    if (grain && d != 0.0 && rain[i] > 0.0) grain[i] += gkbr * K * d * pow(rain[i], d - 1.0) * dt * fm;
}

// dJ/dhOld = y + (dJ/dh at masked vertices) + lim terms (own + from donors)
__global__ void k_spl_adj_hold(int n, const int* __restrict__ nbr, const uint32_t* __restrict__ mask,
                               const unsigned long long* __restrict__ dk, const unsigned long long* __restrict__ sorder,
                               const double* __restrict__ y, const double* __restrict__ ghs,
                               const double* __restrict__ ghr, const double* __restrict__ direct, double* out) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    double acc = y[v] + direct[v] + ghs[v];
    uint32_t mm = mask[v];
    unsigned long long kk = dk[v], ord = sorder[v];
    for (int q = 0; q < MAXW && mm; q++) {
        int t = (int)(ord & 15ULL);
        ord >>= 4;
        if (!(mm & (1u << t))) continue;
        mm &= ~(1u << t);
        int j = nbr[(size_t)t * n + v];
        int k = (int)((kk >> (4 * t)) & 15ULL);
        acc += ghr[(size_t)k * n + j];
    }
    out[v] = acc;
}

// split dJ/dh after SPL into the part through s (unmasked) and the direct
// part to hOld (masked vertices keep hOld)
__global__ void k_spl_adj_split(int n, int flat, const uint8_t* __restrict__ outlet, const uint8_t* __restrict__ lsink,
                                const double* __restrict__ lam, double* gs, double* direct) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool masked = (flat && outlet[i]) || lsink[i];
    gs[i] = masked ? 0.0 : lam[i];
    direct[i] = masked ? lam[i] : 0.0;
}

// Adjoint of erodep_spl.  lam: dJ/dh after SPL on entry, dJ/dhOld on return.
// gw_out [R][n]: dJ/dw of the snapshot receivers (written).  gfal: dJ/dFAL.
int spl_adjoint(gs_plan* p, const double* hold, const double* s, const double* fal, const double* rain,
                double k_scalar, const double* k_field, double d, double m, double dt, const int* rcv,
                const double* dist, const double* wgt, const int8_t* rslot, const int* order, const uint8_t* lsink,
                const uint8_t* sea, double* lam, double* gK, double* grain, double* gfal, double* gw_out) {
    const int n = (int)p->n;
    if (n == 0) return GS_OK;
    const int B = 256, G = grid_for(n, B);
    double* gs_ = p->cg_r;
    double* direct = p->cg_z;
    double* y = p->cg_p;
    double* ghs = p->cg_ap;
    launch(p, k_spl_adj_split, G, B, n, p->flat, (const uint8_t*)p->outlet, lsink, (const double*)lam, gs_, direct);
    launch(p, k_spl_coef, G, B, n, p->R, hold, fal, rain, k_scalar, k_field, d, m, dt, rcv, dist, wgt, sea, p->c);
    GS_LAUNCH();
    GS_TRY(sweep_spl_adjoint(p, rcv, wgt, rslot, (const double*)p->c, order, (const double*)gs_, y));
    launch(p, k_spl_adj, G, B, n, p->R, hold, s, (const double*)y, fal, rain, k_scalar, k_field, d, m, dt, rcv, dist,
           wgt, sea, gK, gfal, grain, gw_out, ghs, p->adj_er);
    launch(p, k_spl_adj_hold, G, B, n, (const int*)p->nbr, (const uint32_t*)p->don_mask,
           (const unsigned long long*)p->don_k, (const unsigned long long*)p->sorder, (const double*)y,
           (const double*)ghs, (const double*)p->adj_er, (const double*)direct, lam);
    GS_LAUNCH();
    return GS_OK;
}

}  // namespace gs
