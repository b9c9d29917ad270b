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
// (receivers first); the system is solved by restarted GMRES in FP64 from the
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

constexpr int GMRES_M1 = 31;   // GMRES restart length + 1

// fixed-order dot product (block partials, then one block), read on the host
static int gm_dot(gs_plan* p, int n, const double* a, const double* b, double* out) {
    const int PARTS = 512;
    launch(p, k_ed_dot_part, PARTS, 256, n, a, b, p->red);
    launch(p, k_ed_dot_final, 1, 1024, PARTS, (const double*)p->red, p->red + 4200);
    GS_LAUNCH();
    GS_CUDA(cudaMemcpyAsync(out, p->red + 4200, sizeof(double), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    return GS_OK;
}

struct EdSolve : LinOp {
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
    EdSolve(gs_plan* p_, int n_, const int* rcv_, const double* wgt_, const double* c_, const double* f_,
            double dt_, double* t1_, double* u_, double* w_, double* y2_)
        : p(p_), n(n_), rcv(rcv_), wgt(wgt_), c(c_), f(f_), dt(dt_), t1(t1_), u(u_), w(w_), y2(y2_) {}
    // y = (I + B) x
    int apply(const double* x, double* y) override {
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
};

// GMRES kernels: block partial dot products of w with the first k basis
// vectors, their fixed-order totals, and w -= sum_j h_j V_j
__global__ void k_mdot_part(int n, int k, const double* __restrict__ V, const double* __restrict__ w,
                            double* part) {
    __shared__ double sh[4][256];
    const int per = (n + gridDim.x - 1) / gridDim.x;
    const int lo = blockIdx.x * per, hi = lo + per < n ? lo + per : n;
    for (int jb = 0; jb < k; jb += 4) {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            const double wi = w[i];
#pragma unroll
            for (int u = 0; u < 4; u++)
                if (jb + u < k) acc[u] += V[(size_t)(jb + u) * n + i] * wi;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) sh[u][threadIdx.x] = acc[u];
        __syncthreads();
        for (int s2 = blockDim.x / 2; s2 > 0; s2 >>= 1) {
            if (threadIdx.x < s2)
#pragma unroll
                for (int u = 0; u < 4; u++) sh[u][threadIdx.x] += sh[u][threadIdx.x + s2];
            __syncthreads();
        }
        if (threadIdx.x < 4 && jb + threadIdx.x < k)
            part[(size_t)blockIdx.x * GMRES_M1 + jb + threadIdx.x] = sh[threadIdx.x][0];
        __syncthreads();
    }
}

// one block per basis vector: the block partials summed in a fixed order
__global__ void k_mdot_final(int parts, int k, const double* __restrict__ part, double* out) {
    __shared__ double sh[256];
    const int j = blockIdx.x;
    if (j >= k) return;
    double acc = 0.0;
    for (int b = threadIdx.x; b < parts; b += blockDim.x) acc += part[(size_t)b * GMRES_M1 + j];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s2 = blockDim.x / 2; s2 > 0; s2 >>= 1) {
        if (threadIdx.x < s2) sh[threadIdx.x] += sh[threadIdx.x + s2];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[j] = sh[0];
}

__global__ void k_mupdate(int n, int k, const double* __restrict__ V, const double* __restrict__ h, double* w) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = w[i];
    for (int j = 0; j < k; j++) s -= h[j] * V[(size_t)j * n + i];
    w[i] = s;
}

// Restarted GMRES(30) in FP64 on op x = a from the given x: Arnoldi with
// classical Gram-Schmidt applied twice (fixed-order block dot products of the
// new vector with the basis, k_mdot_part / k_mdot_final / k_mupdate), Givens
// rotations of the Hessenberg matrix on the host, one synchronisation per
// step; stops at |a - op x| <= tol |a| or after max_applies applications.
int gmres_solve(gs_plan* p, LinOp& op, const double* a, double* x, double tol, int max_applies, int* applies_out,
                double* relres_out) {
    const int n = (int)p->n;
    const int B = 256, G = grid_for(n, B);
    constexpr int M = GMRES_M1 - 1;   // restart length
    const int PARTS = p->sm_count * 8;
    if (!p->ed_basis)
        GS_CUDA(cudaMalloc((void**)&p->ed_basis,
                           sizeof(double) * ((size_t)std::max(n, 1) * GMRES_M1 + (size_t)PARTS * GMRES_M1 + 4 * GMRES_M1)));
    // (PARTS depends only on the SM count, fixed for the plan's device)
    double* V = p->ed_basis;
    double* part = V + (size_t)n * GMRES_M1;
    double* hd = part + (size_t)PARTS * GMRES_M1;    // [0, M1): pass 1, [M1, 2 M1): pass 2, 2 M1: norm^2
    double* r = p->cg_r;
    double an = 0.0;
    GS_TRY(gm_dot(p, n, a, a, &an));
    const double anorm = sqrt(an);
    std::vector<double> H((size_t)(M + 1) * M), cs(M), sn(M), g(M + 1), y(M), hh(2 * GMRES_M1 + 1);
    int applies = 0;
    double res = 0.0;
    bool conv = anorm == 0.0;
    while (!conv && applies < max_applies) {
        // r = a - op x, V_0 = r / |r|
        GS_TRY(op.apply(x, r));
        applies++;
        launch(p, k_ed_axpby, G, B, n, 1.0, a, -1.0, (const double*)r, r);
        GS_LAUNCH();
        double rn2 = 0.0;
        GS_TRY(gm_dot(p, n, r, r, &rn2));
        const double beta = sqrt(rn2);
        res = beta;
        if (!(beta == beta)) break;
        if (beta <= tol * anorm) { conv = true; break; }
        launch(p, k_ed_axpby, G, B, n, 1.0 / beta, (const double*)r, 0.0, (const double*)r, V);
        GS_LAUNCH();
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int k = 0;
        for (; k < M && applies < max_applies; k++) {
            double* vk1 = V + (size_t)(k + 1) * n;
            GS_TRY(op.apply(V + (size_t)k * n, vk1));
            applies++;
            for (int pass = 0; pass < 2; pass++) {
                launch(p, k_mdot_part, PARTS, 256, n, k + 1, (const double*)V, (const double*)vk1, part);
                launch(p, k_mdot_final, k + 1, 256, PARTS, k + 1, (const double*)part, hd + pass * GMRES_M1);
                launch(p, k_mupdate, G, B, n, k + 1, (const double*)V, (const double*)(hd + pass * GMRES_M1), vk1);
                GS_LAUNCH();
            }
            launch(p, k_ed_dot_part, 512, 256, n, (const double*)vk1, (const double*)vk1, p->red);
            launch(p, k_ed_dot_final, 1, 1024, 512, (const double*)p->red, hd + 2 * GMRES_M1);
            GS_LAUNCH();
            GS_CUDA(cudaMemcpyAsync(hh.data(), hd, sizeof(double) * (2 * GMRES_M1 + 1), cudaMemcpyDeviceToHost,
                                    p->stream));
            GS_CUDA(cudaStreamSynchronize(p->stream));
            double* col = &H[(size_t)k * (M + 1)];
            for (int j = 0; j <= k; j++) col[j] = hh[j] + hh[GMRES_M1 + j];
            const double hn = sqrt(hh[2 * GMRES_M1]);
            col[k + 1] = hn;
            for (int j = 0; j < k; j++) {
                const double t = cs[j] * col[j] + sn[j] * col[j + 1];
                col[j + 1] = -sn[j] * col[j] + cs[j] * col[j + 1];
                col[j] = t;
            }
            const double den = std::hypot(col[k], col[k + 1]);
            cs[k] = den > 0.0 ? col[k] / den : 1.0;
            sn[k] = den > 0.0 ? col[k + 1] / den : 0.0;
            col[k] = den;
            col[k + 1] = 0.0;
            g[k + 1] = -sn[k] * g[k];
            g[k] = cs[k] * g[k];
            res = std::fabs(g[k + 1]);
            if (!(res == res)) break;
            if (res <= tol * anorm || hn == 0.0) { k++; conv = true; break; }
            launch(p, k_ed_axpby, G, B, n, 1.0 / hn, (const double*)vk1, 0.0, (const double*)vk1, vk1);
            GS_LAUNCH();
        }
        // x += V y, H y = g (upper triangular, k columns)
        for (int i = k - 1; i >= 0; i--) {
            double s2 = g[i];
            for (int j = i + 1; j < k; j++) s2 -= H[(size_t)j * (M + 1) + i] * y[j];
            y[i] = s2 / H[(size_t)i * (M + 1) + i];
        }
        for (int i = 0; i < k; i++) y[i] = -y[i];
        GS_CUDA(cudaMemcpyAsync(hd, y.data(), sizeof(double) * k, cudaMemcpyHostToDevice, p->stream));
        launch(p, k_mupdate, G, B, n, k, (const double*)V, (const double*)hd, x);
        GS_LAUNCH();
        GS_CUDA(cudaStreamSynchronize(p->stream));
        if (!(res == res)) break;
    }
    if (applies_out) *applies_out = applies;
    if (relres_out) *relres_out = anorm > 0.0 ? res / anorm : 0.0;
    return conv ? GS_OK : GS_EMAXITER;
}

// x = y (device copy through the GMRES axpby kernel)
int gm_axpby(gs_plan* p, int n, double a, const double* x, double b, const double* y, double* z) {
    launch(p, k_ed_axpby, grid_for(n, 256), 256, n, a, x, b, y, z);
    GS_LAUNCH();
    return GS_OK;
}

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
    launch(p, k_fdep, G, B, n, p->fdepa, (const double*)p->larea, fal, sea, (const uint8_t*)p->outlet, p->flat, f);
    GS_LAUNCH();
    GS_TRY(build_donors(p, rcv_i, wgt_i, p->rslot_i));
    GS_TRY(spl_order(p));
    EdSolve op(p, n, rcv_i, wgt_i, (const double*)p->c, (const double*)f, dt, t1, u, w, y2);
    // x0 = M^-1 hOld (detachment-limited), a = x0 + B hOld
    GS_TRY(sweep_spl_rhs(p, rcv_i, p->c, p->order2, hold, x));
    GS_TRY(op.apply(hold, a));                                        // a = hOld + B hOld
    launch(p, k_ed_axpby, G, B, n, 1.0, (const double*)a, -1.0, hold, a);
    launch(p, k_ed_axpby, G, B, n, 1.0, (const double*)a, 1.0, (const double*)x, a);
    GS_LAUNCH();
    // GMRES(30) on (I + B) x = a to 1e-13 of |a|, at most 200 applications
    int applies = 0;
    double relres = 0.0;
    const int st = gmres_solve(p, op, a, x, 1.0e-13, 200, &applies, &relres);
    p->ed_iters = applies;
    p->ed_relres = relres;
    if (st == GS_EMAXITER) {
        set_error(GS_EMAXITER, "transport-limited SPL: GMRES did not converge");
        return GS_EMAXITER;
    }
    return st;
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
