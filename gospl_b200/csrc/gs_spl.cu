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
    launch(p, k_spl_update, G, B, n, p->flat, (const uint8_t*)p->outlet, lsink, (const double*)hold,
           (const double*)p->q3, dt, h, cum_ed, eb);
    GS_LAUNCH();
    (void)st;
    return GS_OK;
}

}  // namespace gs
