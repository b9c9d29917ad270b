// Implicit linear stream-power erosion, n = 1, G = 0:
// SPL._eroMats (gospl/eroder/SPL.py:45-114), _getEroDepRate (260-366) and
// erodepSPL (402-454).  The PETSc KSP solve of SPL.py:297 is replaced by the
// exact receivers-first dataflow sweep (gs_sweep.cu).
#include <algorithm>
#include <cmath>

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

// ---------------------------------------------------------------------------
// Transport-limited SPL (G > 0): _getEroDepRate's coupled branch
// (SPL.py:305-336) and _coupledEDSystem (SPL.py:116-258).  Eliminating the
// sediment flux q from the nested system
//     [eMat - diag(f)      -diag(f dt / A)] [h]   [(1 - f) hOld ]
//     [diag(A / dt)         (I - W)^T     ] [q] = [hOld A / dt  ]
// gives (I + B) h = a with B = M^-1 diag(f dt / A) W^T (I - W^T)^-1 diag(A / dt)
// (M = eMat, W^T (I - W^T)^-1 = (I - W^T)^-1 - I) and a = M^-1 hOld + B hOld.
// B is applied with one flow sweep (donors first) and one SPL sweep
// (receivers first); the system is solved by BiCGSTAB in FP64 from the
// detachment-limited solution.  f = G A / max(FAL, G A / 0.99), 0 where
// FAL = 0, at sea and at flat-model outlets, capped at 0.99.
__global__ void k_fdep(int n, double G, const double* __restrict__ larea, const double* __restrict__ fal,
                       const uint8_t* __restrict__ sea, const uint8_t* __restrict__ outlet, int flat, double* f) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double num = G * larea[i];
    const double floor_ = num / 0.99;
    const double pa = fal[i];
    double v = (pa != 0.0) ? num / (pa > floor_ ? pa : floor_) : 0.0;
    if (sea[i]) v = 0.0;
    if (v > 0.99) v = 0.99;
    if (flat && outlet[i]) v = 0.0;
    f[i] = v;
}

__global__ void k_ed_scale(int n, const double* __restrict__ larea, double dt, const double* __restrict__ x,
                           double* t) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) t[i] = larea[i] / dt * x[i];
}

// w = f dt / A (u - t): deposition source from the upstream sediment flux
__global__ void k_ed_dep(int n, const double* __restrict__ f, const double* __restrict__ larea, double dt,
                         const double* __restrict__ u, const double* __restrict__ t, double* w) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) w[i] = f[i] * dt / larea[i] * (u[i] - t[i]);
}

__global__ void k_ed_axpby(int n, double a, const double* __restrict__ x, double b, const double* __restrict__ y,
                           double* z) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) z[i] = a * x[i] + b * y[i];
}

__global__ void k_ed_dot_part(int n, const double* __restrict__ a, const double* __restrict__ b, double* part) {
    __shared__ double sh[256];
    double acc = 0.0;
    int per = (n + gridDim.x - 1) / gridDim.x;
    int lo = blockIdx.x * per, hi = lo + per < n ? lo + per : n;
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) acc += a[i] * b[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s2 = blockDim.x / 2; s2 > 0; s2 >>= 1) {
        if (threadIdx.x < s2) sh[threadIdx.x] += sh[threadIdx.x + s2];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_ed_dot_final(int parts, const double* __restrict__ part, double* out) {
    __shared__ double sh[1024];
    double acc = 0.0;
    for (int i = threadIdx.x; i < parts; i += blockDim.x) acc += part[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s2 = blockDim.x / 2; s2 > 0; s2 >>= 1) {
        if (threadIdx.x < s2) sh[threadIdx.x] += sh[threadIdx.x + s2];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

struct EdSolve {
    gs_plan* p;
    int n;
    const int* rcv;
    const double* wgt;
    const double* c;
    const double* f;
    double dt;
    double* t1;
    double* u;
    double* w;
    double* y2;
    // y = (I + B) x
    int apply(const double* x, double* y) {
        const int B = 256, G = grid_for(n, B);
        launch(p, k_ed_scale, G, B, n, (const double*)p->larea, dt, x, t1);
        GS_LAUNCH();
        GS_TRY(sweep_flow_rhs(p, wgt, p->order_i, t1, u));
        launch(p, k_ed_dep, G, B, n, f, (const double*)p->larea, dt, (const double*)u, (const double*)t1, w);
        GS_LAUNCH();
        GS_TRY(sweep_spl_rhs(p, rcv, c, p->order2, w, y2));
        launch(p, k_ed_axpby, G, B, n, 1.0, x, 1.0, (const double*)y2, y);
        GS_LAUNCH();
        return GS_OK;
    }
    int dot(const double* a, const double* b, double* out) {
        const int PARTS = 512;
        launch(p, k_ed_dot_part, PARTS, 256, n, a, b, p->red);
        launch(p, k_ed_dot_final, 1, 1024, PARTS, (const double*)p->red, p->red + 4200);
        GS_LAUNCH();
        GS_CUDA(cudaMemcpyAsync(out, p->red + 4200, sizeof(double), cudaMemcpyDeviceToHost, p->stream));
        GS_CUDA(cudaStreamSynchronize(p->stream));
        return GS_OK;
    }
};

static int coupled_ed(gs_plan* p, const double* hold, const double* fal, const uint8_t* sea, double dt,
                      const int* rcv_i, const double* wgt_i, double* x) {
    const int n = (int)p->n;
    const int B = 256, G = grid_for(n, B);
    if (!p->order_i_valid) {
        set_error(GS_EINVAL, "transport-limited SPL needs a topological order of the receiver graph");
        return GS_EINVAL;
    }
    if (!p->ed_buf) GS_CUDA(cudaMalloc((void**)&p->ed_buf, sizeof(double) * (size_t)std::max(n, 1) * 6));
    double* f = p->ed_buf;
    double* t1 = f + n;
    double* u = t1 + n;
    double* w = u + n;
    double* y2 = w + n;
    double* a = y2 + n;
    double *r = p->cg_r, *r0 = p->cg_b, *pp = p->cg_p, *v = p->cg_ap, *sv = p->cg_z, *tv = p->cg_x;
    launch(p, k_fdep, G, B, n, p->fdepa, (const double*)p->larea, fal, sea, (const uint8_t*)p->outlet, p->flat, f);
    GS_LAUNCH();
    GS_TRY(build_donors(p, rcv_i, wgt_i, p->rslot_i));
    GS_TRY(spl_order(p));
    EdSolve op{p, n, rcv_i, wgt_i, (const double*)p->c, (const double*)f, dt, t1, u, w, y2};
    // x0 = M^-1 hOld (detachment-limited), a = x0 + B hOld
    GS_TRY(sweep_spl_rhs(p, rcv_i, p->c, p->order2, hold, x));
    GS_TRY(op.apply(hold, a));                                        // a = hOld + B hOld
    launch(p, k_ed_axpby, G, B, n, 1.0, (const double*)a, -1.0, hold, a);
    launch(p, k_ed_axpby, G, B, n, 1.0, (const double*)a, 1.0, (const double*)x, a);
    GS_LAUNCH();
    // BiCGSTAB on (I + B) x = a
    GS_TRY(op.apply(x, v));
    launch(p, k_ed_axpby, G, B, n, 1.0, (const double*)a, -1.0, (const double*)v, r);
    launch(p, k_ed_axpby, G, B, n, 1.0, (const double*)r, 0.0, (const double*)r, r0);
    GS_CUDA(cudaMemsetAsync(pp, 0, sizeof(double) * n, p->stream));
    GS_CUDA(cudaMemsetAsync(v, 0, sizeof(double) * n, p->stream));
    GS_LAUNCH();
    double an = 0.0, rn = 0.0;
    GS_TRY(op.dot(a, a, &an));
    GS_TRY(op.dot(r, r, &rn));
    const double anorm = sqrt(an);
    const double tol = 1.0e-13;
    double rho = 1.0, alpha = 1.0, omega = 1.0;
    int it = 0;
    for (; it < 200 && anorm > 0.0 && sqrt(rn) > tol * anorm; it++) {
        double rho1 = 0.0;
        GS_TRY(op.dot(r0, r, &rho1));
        const double beta = (rho1 / rho) * (alpha / omega);
        // p = r + beta (p - omega v)
        launch(p, k_ed_axpby, G, B, n, 1.0, (const double*)pp, -omega, (const double*)v, pp);
        launch(p, k_ed_axpby, G, B, n, 1.0, (const double*)r, beta, (const double*)pp, pp);
        GS_LAUNCH();
        GS_TRY(op.apply(pp, v));
        double r0v = 0.0;
        GS_TRY(op.dot(r0, v, &r0v));
        alpha = rho1 / r0v;
        launch(p, k_ed_axpby, G, B, n, 1.0, (const double*)r, -alpha, (const double*)v, sv);
        GS_LAUNCH();
        double sn = 0.0;
        GS_TRY(op.dot(sv, sv, &sn));
        if (sqrt(sn) <= tol * anorm) {
            launch(p, k_ed_axpby, G, B, n, 1.0, (const double*)x, alpha, (const double*)pp, x);
            GS_LAUNCH();
            rn = sn;
            it++;
            break;
        }
        GS_TRY(op.apply(sv, tv));
        double ts = 0.0, tt = 0.0;
        GS_TRY(op.dot(tv, sv, &ts));
        GS_TRY(op.dot(tv, tv, &tt));
        omega = ts / tt;
        launch(p, k_ed_axpby, G, B, n, 1.0, (const double*)x, alpha, (const double*)pp, x);
        launch(p, k_ed_axpby, G, B, n, 1.0, (const double*)x, omega, (const double*)sv, x);
        launch(p, k_ed_axpby, G, B, n, 1.0, (const double*)sv, -omega, (const double*)tv, r);
        GS_LAUNCH();
        GS_TRY(op.dot(r, r, &rn));
        rho = rho1;
        if (!(rn == rn)) break;
    }
    p->ed_iters = it;
    p->ed_relres = anorm > 0.0 ? sqrt(rn) / anorm : 0.0;
    if (!(rn == rn) || sqrt(rn) > tol * anorm * 1.0e3) {
        set_error(GS_EMAXITER, "transport-limited SPL: BiCGSTAB did not converge");
        return GS_EMAXITER;
    }
    return GS_OK;
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
    if (p->fdepa > 0.0) GS_TRY(coupled_ed(p, hold, fal, sea, dt, rcv_i, wgt_i, p->q3));
    GS_TRY(rec_spl(p, p->q3, lsink));
    launch(p, k_spl_update, G, B, n, p->flat, (const uint8_t*)p->outlet, lsink, (const double*)hold,
           (const double*)p->q3, dt, h, cum_ed, eb);
    GS_LAUNCH();
    if (st) {
        st->cg_iters = p->fdepa > 0.0 ? p->ed_iters : 0;
        st->cg_relres = p->fdepa > 0.0 ? p->ed_relres : 0.0;
    }
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
