// Linear hillslope diffusion: hillSLP.getHillslope -> _hillSlope(smooth=0)
// (gospl/sed/hillslope.py:90-233, 614-649) with the finite-volume stencil of
// sethillslopecoeff (fortran/functions.F90:901-938) and the outlet identity
// rows of _buildDiffMat (hillslope.py:235-257).
//
// Row k of (I + L):  diag 1 + sum_p v_kp,  off -v_kp,
//     v_kp = 0.5 (Kd_k + Kd_p) / A_k * vDist_kp / eLgt_kp.
// Multiplying row k by A_k gives a symmetric positive-definite operator
// (vDist and eLgt are per-edge), so the system is solved with
// Jacobi-preconditioned CG on  A (I + L) h = A hOld,  outlet rows (and rows of
// zero area, which carry no equation) held at hOld.  The matrix is rebuilt only
// when the land/sea mask changes, like the reference's cached operator.
#include <cooperative_groups.h>

#include <algorithm>

#include "gs_plan.cuh"

namespace cg = cooperative_groups;

namespace gs {

// row k of (I + L) for the land/sea mask `sea` (sea: Cd = cdm, land: cda)
__device__ __forceinline__ void diff_row_build(int k, int n, int W, int flat, const uint8_t* sea, double cda,
                                               double cdm, double dt, const int* nbr, const int8_t* nnb,
                                               const double* elen, const double* vdist, const double* farea,
                                               const uint8_t* outlet, double* coef) {
    const double ck = (sea[k] ? cdm : cda) * dt;
    double diag = 0.0;
    for (int s = 0; s < W; s++) coef[(size_t)(s + 1) * n + k] = 0.0;
    if (farea[k] > 0) {
        double s1 = 0.0;
        const double ak = farea[k];
        for (int s = 0; s < nnb[k]; s++) {
            double vd = vdist[(size_t)s * n + k];
            if (vd > 0.0) {
                int j = nbr[(size_t)s * n + k];
                double cn = (sea[j] ? cdm : cda) * dt;
                double c = 0.5 * (ck + cn) / ak;
                double v = c * vd / elen[(size_t)s * n + k];
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

__global__ void k_sea_of(int n, const double* __restrict__ h, double sl, uint8_t* sea) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) sea[k] = h[k] <= sl ? 1 : 0;
}

// all rows for the mask `sea`
__global__ void k_diff_rows(int n, int W, int flat, const uint8_t* __restrict__ sea, double cda, double cdm,
                            double dt, const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                            const double* __restrict__ elen, const double* __restrict__ vdist,
                            const double* __restrict__ farea, const uint8_t* __restrict__ outlet, double* coef) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) diff_row_build(k, n, W, flat, sea, cda, cdm, dt, nbr, nnb, elen, vdist, farea, outlet, coef);
}

// only the rows whose own or a neighbour's mask changed from `old` to `sea`
__global__ void k_diff_rows_dirty(int n, int W, int flat, const uint8_t* __restrict__ sea,
                                  const uint8_t* __restrict__ old, double cda, double cdm, double dt,
                                  const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                                  const double* __restrict__ elen, const double* __restrict__ vdist,
                                  const double* __restrict__ farea, const uint8_t* __restrict__ outlet,
                                  double* coef) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    bool dirty = sea[k] != old[k];
    for (int s = 0; s < nnb[k] && !dirty; s++) {
        int j = nbr[(size_t)s * n + k];
        if (j >= 0 && sea[j] != old[j]) dirty = true;
    }
    if (dirty) diff_row_build(k, n, W, flat, sea, cda, cdm, dt, nbr, nnb, elen, vdist, farea, outlet, coef);
}

__global__ void k_diff_coef(int n, int W, int flat, const double* __restrict__ h, double sl,
                            double cda, double cdm, double dt, const int* __restrict__ nbr,
                            const int8_t* __restrict__ nnb, const double* __restrict__ elen,
                            const double* __restrict__ vdist, const double* __restrict__ farea,
                            const uint8_t* __restrict__ outlet, double* coef, uint8_t* dsea) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double ck = ((h[k] <= sl) ? cdm : cda) * dt;
    dsea[k] = h[k] <= sl ? 1 : 0;
    double diag = 0.0;
    for (int s = 0; s < W; s++) coef[(size_t)(s + 1) * n + k] = 0.0;
    if (farea[k] > 0) {
        double s1 = 0.0;
        const double ak = farea[k];
        for (int s = 0; s < nnb[k]; s++) {
            double vd = vdist[(size_t)s * n + k];
            if (vd > 0.0) {
                int j = nbr[(size_t)s * n + k];
                double cn = ((h[j] <= sl) ? cdm : cda) * dt;
                double c = 0.5 * (ck + cn) / ak;
                double v = c * vd / elen[(size_t)s * n + k];
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

__device__ __forceinline__ bool diff_fixed(int k, int flat, const uint8_t* outlet, const double* farea) {
    return (flat && outlet[k]) || !(farea[k] > 0);
}

// y = A_k * ((I+L) x)_k over free rows; fixed rows and fixed columns excluded
__device__ __forceinline__ double diff_row(int k, int n, int W, const int* nbr, const int8_t* nnb,
                                           const double* coef, const double* farea, const uint8_t* outlet,
                                           int flat, const double* x, bool free_cols_only) {
    double y = coef[k] * x[k];
    for (int s = 0; s < nnb[k]; s++) {
        double o = coef[(size_t)(s + 1) * n + k];
        if (o == 0.0) continue;
        int j = nbr[(size_t)s * n + k];
        if (free_cols_only && diff_fixed(j, flat, outlet, farea)) continue;
        y = y + o * x[j];
    }
    return farea[k] * y;
}

__global__ void k_cg_init(int n, int W, int flat, const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                          const double* __restrict__ coef, const double* __restrict__ farea,
                          const uint8_t* __restrict__ outlet, const double* __restrict__ hold, double* x,
                          double* b, double* r, double* z, double* pp) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    x[k] = hold[k];
    if (diff_fixed(k, flat, outlet, farea)) {
        b[k] = 0.0; r[k] = 0.0; z[k] = 0.0; pp[k] = 0.0;
        return;
    }
    // right-hand side A_k hOld_k minus known (fixed) columns
    double bk = hold[k];
    for (int s = 0; s < nnb[k]; s++) {
        double o = coef[(size_t)(s + 1) * n + k];
        if (o == 0.0) continue;
        int j = nbr[(size_t)s * n + k];
        if (diff_fixed(j, flat, outlet, farea)) bk = bk - o * hold[j];
    }
    bk = farea[k] * bk;
    b[k] = bk;
    double ax = diff_row(k, n, W, nbr, nnb, coef, farea, outlet, flat, hold, true);
    double rk = bk - ax;
    r[k] = rk;
    double zk = rk / (farea[k] * coef[k]);
    z[k] = zk;
    pp[k] = zk;
}

__global__ void k_cg_spmv(int n, int W, int flat, const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                          const double* __restrict__ coef, const double* __restrict__ farea,
                          const uint8_t* __restrict__ outlet, const double* __restrict__ pp, double* ap) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    ap[k] = diff_fixed(k, flat, outlet, farea) ? 0.0
                                               : diff_row(k, n, W, nbr, nnb, coef, farea, outlet, flat, pp, true);
}

// fixed-shape block partial dot products (deterministic)
template <int NV>
__global__ void k_dots(int n, const double* __restrict__ a0, const double* __restrict__ b0,
                       const double* __restrict__ a1, const double* __restrict__ b1, double* part) {
    __shared__ double sh[NV][256];
    double acc[NV];
    for (int v = 0; v < NV; v++) acc[v] = 0.0;
    int per = (n + gridDim.x - 1) / gridDim.x;
    int lo = blockIdx.x * per, hi = lo + per < n ? lo + per : n;
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        acc[0] += a0[i] * b0[i];
        if (NV > 1) acc[NV - 1] += a1[i] * b1[i];
    }
    for (int v = 0; v < NV; v++) sh[v][threadIdx.x] = acc[v];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int v = 0; v < NV; v++) sh[v][threadIdx.x] += sh[v][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int v = 0; v < NV; v++) part[v * gridDim.x + blockIdx.x] = sh[v][0];
}

__global__ void k_dots_final(int parts, int nv, const double* __restrict__ part, double* out) {
    __shared__ double sh[1024];
    for (int v = 0; v < nv; v++) {
        double acc = 0.0;
        for (int i = threadIdx.x; i < parts; i += blockDim.x) acc += part[v * parts + i];
        sh[threadIdx.x] = acc;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[v] = sh[0];
        __syncthreads();
    }
}

// x += alpha p ; r -= alpha Ap ; z = r / diag  with alpha = rz / pAp (device scalars)
__global__ void k_cg_update(int n, int flat, const uint8_t* __restrict__ outlet, const double* __restrict__ farea,
                            const double* __restrict__ coef, const double* __restrict__ sc, double* x,
                            double* r, double* z, const double* __restrict__ pp, const double* __restrict__ ap) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (diff_fixed(k, flat, outlet, farea)) return;
    const double alpha = sc[0] / sc[1];
    x[k] = x[k] + alpha * pp[k];
    double rk = r[k] - alpha * ap[k];
    r[k] = rk;
    z[k] = rk / (farea[k] * coef[k]);
}

// p = z + beta p, beta = rz_new / rz_old; rotate rz
__global__ void k_cg_dir(int n, const double* __restrict__ sc_new, double* sc, const double* __restrict__ z,
                         double* pp) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    const double beta = sc_new[0] / sc[0];
    if (k < n) pp[k] = z[k] + beta * pp[k];
}

__global__ void k_cg_rotate(const double* __restrict__ sc_new, double* sc) {
    sc[0] = sc_new[0];
}

// slot of the CG's final residual in the reduction scratch (8192 doubles),
// beyond the block partials of the cooperative CG (7 per block, at most 4 blocks
// per SM) and the scalars at 4096..4103
constexpr int RES_SLOT = 8190;

__global__ void k_hill_apply(int n, const double* __restrict__ hold, const double* __restrict__ x, double dt,
                             double* h, double* cum_ed, double* eb, double* dz_out) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double dz = x[k] - hold[k];
    cum_ed[k] = cum_ed[k] + dz;
    h[k] = x[k];
    eb[k] = eb[k] + dz / dt;
    if (dz_out) dz_out[k] = dz;
}

// start of the hillslope CG: this step's elevation plus the previous step's
// diffusion change (fixed rows keep their elevation)
__global__ void k_hill_guess(int n, const double* __restrict__ hold, const double* __restrict__ dprev,
                             const uint8_t* __restrict__ fix, double* g) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    g[k] = fix[k] ? hold[k] : hold[k] + dprev[k];
}

__global__ void k_copy_d2(int n, const double* __restrict__ a, double* b) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i];
}

__global__ void k_mask_changed(int n, const double* __restrict__ h, double sl, const uint8_t* __restrict__ dsea,
                               int* flag) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n && (uint8_t)(h[k] <= sl) != dsea[k]) *flag = 1;
}

// ---------------------------------------------------------------------------
// The whole CG loop in one cooperative launch: three grid barriers per
// iteration (after A p and its dot, after the update and its dots, after the
// new direction), convergence decided on the device.  Dot products are block
// partials in a fixed order; every block sums the partials of all blocks in
// the same order (one warp, lane-strided, then a shuffle-down tree), so all
// threads hold bitwise the same scalars and leave the loop together.
__device__ __forceinline__ void block_sum2(double a, double b, double* out_a, double* out_b) {
    __shared__ double sa[256], sb[256];
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            sa[threadIdx.x] += sa[threadIdx.x + s];
            sb[threadIdx.x] += sb[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *out_a = sa[0];
        *out_b = sb[0];
    }
    __syncthreads();
}

// sum over blocks of part[i * stride + off], identical in every block
__device__ __forceinline__ double grid_total(const double* part, int stride, int off, int nb) {
    __shared__ double tot;
    if (threadIdx.x < 32) {
        double acc = 0.0;
        for (int i = threadIdx.x; i < nb; i += 32) acc += ((volatile const double*)part)[(size_t)i * stride + off];
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (threadIdx.x == 0) tot = acc;
    }
    __syncthreads();
    double t = tot;
    __syncthreads();
    return t;
}

// Jacobi-PCG on the area-weighted symmetric form S = A (I + L) of the
// hillslope system, in one cooperative launch:
//   start x = x0; free rows b = A_k (x0_k - sum over fixed columns o x0_j),
//   r = b - S x (free columns), z = r / (A_k c_k), p = z;
//   per iteration  Sp and p.Sp  | grid barrier |  x += a p, r -= a Sp,
//   z = r / diag, r.z and r.r  | grid barrier |,
// and the direction update p' = z + b p of the next iteration is made inside
// its product: each thread forms p'_j = z_j + b p_j of the neighbours it
// gathers (the same operations as a separate update pass, so the same bits)
// and writes its own p'_k to the other buffer.  Two barriers per iteration;
// block partial sums are added in block order by every block.  Fixed rows
// (flat outlets, no area) keep x = x0.  Slots are unrolled to MAXW so the
// gathers of a row issue together; <= 64 registers for four 256-thread
// blocks per SM.
__global__ void __launch_bounds__(256, 4) k_cg_coop(int n, const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                                                    const double* __restrict__ coef, const double* __restrict__ farea,
                                                    const uint8_t* __restrict__ fix, const double* __restrict__ x0,
                                                    double* x, double* b, double* r, double* z, double* p0, double* p1,
                                                    double* ap, double* part, double rtol, int max_iter, int* it_out,
                                                    double* res_out, const double* __restrict__ guess) {
    cg::grid_group grid = cg::this_grid();
    const int nb = gridDim.x, blk = blockIdx.x;
    const int gtid = blk * blockDim.x + threadIdx.x, gsz = nb * blockDim.x;
    double* pc = part;             // initial dots [3 nb]
    double* pa = part + 3 * nb;    // p.Ap [2 nb]
    double* pb = part + 5 * nb;    // r.z, r.r [2 nb]
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int k = gtid; k < n; k += gsz) {
        const double x0k = x0[k];
        if (fix[k]) {
            x[k] = x0k;
            b[k] = 0.0;
            r[k] = 0.0;
            z[k] = 0.0;
            p0[k] = 0.0;
            continue;
        }
        // the start: x0 (the right-hand side), or the guess on free rows
        const double xk = guess ? guess[k] : x0k;
        x[k] = xk;
        const int deg = nnb[k];
        const double ck = coef[k];
        double bk = x0k;
        double y = ck * xk;
#pragma unroll
        for (int s = 0; s < MAXW; s++) {
            if (s < deg) {
                const double o = coef[(size_t)(s + 1) * n + k];
                const int j = nbr[(size_t)s * n + k];
                if (o != 0.0 && j >= 0) {
                    const double xj = x0[j];
                    const double gj = guess ? guess[j] : xj;
                    if (fix[j]) bk = bk - o * xj;
                    else y = y + o * gj;
                }
            }
        }
        const double fa = farea[k];
        bk = fa * bk;
        b[k] = bk;
        const double rk = bk - fa * y;
        r[k] = rk;
        const double zk = rk / (fa * ck);
        z[k] = zk;
        p0[k] = zk;
        a0 += rk * zk;
        a1 += rk * rk;
        a2 += bk * bk;
    }
    block_sum2(a0, a1, &pc[3 * blk], &pc[3 * blk + 1]);
    block_sum2(a2, 0.0, &pc[3 * blk + 2], &pa[2 * blk + 1]);
    grid.sync();
    double rz = grid_total(pc, 3, 0, nb);
    const double rr0 = grid_total(pc, 3, 1, nb);
    const double bnorm = sqrt(grid_total(pc, 3, 2, nb));
    double relres = bnorm > 0.0 ? sqrt(rr0) / bnorm : 0.0;
    int it = 0;
    double beta = 0.0;
    double* pcur = p0;     // direction of the previous iteration
    double* pnew = p1;
    while (bnorm > 0.0 && relres > rtol && it < max_iter) {
        // p' = z + beta p (it > 0), its product and p'.Sp'
        double acc = 0.0;
        for (int k = gtid; k < n; k += gsz) {
            const double pk = it ? z[k] + beta * pcur[k] : pcur[k];
            double y = 0.0;
            if (!fix[k]) {
                const int deg = nnb[k];
                y = coef[k] * pk;
#pragma unroll
                for (int s = 0; s < MAXW; s++) {
                    if (s < deg) {
                        const double o = coef[(size_t)(s + 1) * n + k];
                        const int j = nbr[(size_t)s * n + k];
                        if (o != 0.0 && j >= 0) {
                            // the fixed flag and the values are loaded together
                            // (not the values after the flag): one round trip
                            const bool fj = fix[j] != 0;
                            const double zj = it ? z[j] : 0.0;
                            const double qj = pcur[j];
                            if (!fj) {
                                const double pj = it ? zj + beta * qj : qj;
                                y = y + o * pj;
                            }
                        }
                    }
                }
                y = farea[k] * y;
            }
            if (it) pnew[k] = pk;
            ap[k] = y;
            acc += pk * y;
        }
        if (it) {
            double* t = pcur;
            pcur = pnew;
            pnew = t;
        }
        block_sum2(acc, 0.0, &pa[2 * blk], &pa[2 * blk + 1]);
        grid.sync();
        const double pap = grid_total(pa, 2, 0, nb);
        const double alpha = (pap != 0.0) ? rz / pap : 0.0;
        double c0 = 0.0, c1 = 0.0;
        for (int k = gtid; k < n; k += gsz) {
            if (fix[k]) continue;
            x[k] = x[k] + alpha * pcur[k];
            const double rk = r[k] - alpha * ap[k];
            r[k] = rk;
            const double zk = rk / (farea[k] * coef[k]);
            z[k] = zk;
            c0 += rk * zk;
            c1 += rk * rk;
        }
        block_sum2(c0, c1, &pb[2 * blk], &pb[2 * blk + 1]);
        grid.sync();
        const double rzn = grid_total(pb, 2, 0, nb);
        const double rr = grid_total(pb, 2, 1, nb);
        beta = (rz != 0.0) ? rzn / rz : 0.0;
        rz = rzn;
        relres = sqrt(rr) / bnorm;
        it++;
        if (!(relres == relres) || relres <= rtol || it >= max_iter) break;
    }
    if (gtid == 0) {
        *it_out = it;
        *res_out = relres;
    }
}

// FP32 CG (precision form): S d = rhs from d = 0 with FP32 vectors and FP32
// arithmetic (coefficients rounded on load), dot products accumulated in FP64;
// the same barrier structure as k_cg_coop.
__global__ void __launch_bounds__(256) k_cg_coop32(int n, const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                                                   const double* __restrict__ coef, const double* __restrict__ farea,
                                                   const uint8_t* __restrict__ fix, const double* __restrict__ rhs,
                                                   float* x, float* r, float* z, float* pp, float* ap, double* part,
                                                   double rtol, int max_iter, int* it_out, double* res_out) {
    cg::grid_group grid = cg::this_grid();
    const int nb = gridDim.x, blk = blockIdx.x;
    const int gtid = blk * blockDim.x + threadIdx.x, gsz = nb * blockDim.x;
    double* pc = part;
    double* pa = part + 3 * nb;
    double* pb = part + 5 * nb;
    double a0 = 0.0, a1 = 0.0;
    for (int k = gtid; k < n; k += gsz) {
        x[k] = 0.0f;
        if (fix[k]) {
            r[k] = z[k] = pp[k] = 0.0f;
            continue;
        }
        const float rk = (float)rhs[k];
        const float zk = rk / (float)(farea[k] * coef[k]);
        r[k] = rk;
        z[k] = zk;
        pp[k] = zk;
        a0 += (double)rk * (double)zk;
        a1 += (double)rk * (double)rk;
    }
    block_sum2(a0, a1, &pc[3 * blk], &pc[3 * blk + 1]);
    grid.sync();
    double rz = grid_total(pc, 3, 0, nb);
    const double bnorm = sqrt(grid_total(pc, 3, 1, nb));
    double relres = bnorm > 0.0 ? 1.0 : 0.0;
    int it = 0;
    while (bnorm > 0.0 && relres > rtol && it < max_iter) {
        double acc = 0.0;
        for (int k = gtid; k < n; k += gsz) {
            float y = 0.0f;
            if (!fix[k]) {
                y = (float)coef[k] * pp[k];
                for (int s = 0; s < nnb[k]; s++) {
                    double o = coef[(size_t)(s + 1) * n + k];
                    if (o == 0.0) continue;
                    int j = nbr[(size_t)s * n + k];
                    if (fix[j]) continue;
                    y = y + (float)o * pp[j];
                }
                y = (float)farea[k] * y;
            }
            ap[k] = y;
            acc += (double)pp[k] * (double)y;
        }
        block_sum2(acc, 0.0, &pa[2 * blk], &pa[2 * blk + 1]);
        grid.sync();
        const double pap = grid_total(pa, 2, 0, nb);
        const float alpha = (float)((pap != 0.0) ? rz / pap : 0.0);
        double c0 = 0.0, c1 = 0.0;
        for (int k = gtid; k < n; k += gsz) {
            if (fix[k]) continue;
            x[k] = x[k] + alpha * pp[k];
            const float rk = r[k] - alpha * ap[k];
            r[k] = rk;
            const float zk = rk / (float)(farea[k] * coef[k]);
            z[k] = zk;
            c0 += (double)rk * (double)zk;
            c1 += (double)rk * (double)rk;
        }
        block_sum2(c0, c1, &pb[2 * blk], &pb[2 * blk + 1]);
        grid.sync();
        const double rzn = grid_total(pb, 2, 0, nb);
        const double rr = grid_total(pb, 2, 1, nb);
        const float beta = (float)((rz != 0.0) ? rzn / rz : 0.0);
        rz = rzn;
        relres = sqrt(rr) / bnorm;
        it++;
        if (!(relres == relres) || relres <= rtol || it >= max_iter) break;
        for (int k = gtid; k < n; k += gsz) pp[k] = z[k] + beta * pp[k];
        grid.sync();
    }
    if (gtid == 0) {
        *it_out = it;
        *res_out = relres;
    }
}

__global__ void k_add_f32_d(int n, const float* __restrict__ d, double* x) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = x[i] + (double)d[i];
}

// r = b - S x on free rows (FP64), 0 on fixed rows
__global__ void k_cg_resid(int n, int W, int flat, const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                           const double* __restrict__ coef, const double* __restrict__ farea,
                           const uint8_t* __restrict__ outlet, const double* __restrict__ b,
                           const double* __restrict__ x, double* r) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    r[k] = diff_fixed(k, flat, outlet, farea) ? 0.0
                                              : b[k] - diff_row(k, n, W, nbr, nnb, coef, farea, outlet, flat, x, true);
}

// the second direction buffer of k_cg_coop, allocated on first use
static int cg_second_direction(gs_plan* p) {
    if (!p->cg_p2) GS_CUDA(cudaMalloc((void**)&p->cg_p2, sizeof(double) * (size_t)std::max<int64_t>(p->n, 1)));
    return GS_OK;
}

static int cg_launch(gs_plan* p, const void* fn, void** args) {
    cudaEvent_t stop = nullptr;
    if (p->profiling) prof_begin(p, fn, &stop);
    GS_CUDA(cudaLaunchCooperativeKernel(fn, p->coop_blocks, 256, args, 0, p->stream));
    if (stop) cudaEventRecord(stop, p->stream);
    p->launches++;
    return GS_OK;
}

// precision form of the solve: FP32 CG corrections of an FP64 iterate, FP64
// residuals, until |r| <= tol |b| (2-norms)
static int hillslope_refine32(gs_plan* p, double tol, int max_iter, int* outer, double* relres_out) {
    const int n = (int)p->n;
    const int B = 256, G = grid_for(n, B), PARTS = 512;
    GS_TRY(precision_buffers(p));
    const size_t N = (size_t)std::max(n, 1);
    float** bufs[] = {&p->f32b, &p->f32c, &p->f32d, &p->f32e};
    for (float** q : bufs)
        if (!*q) GS_CUDA(cudaMalloc((void**)q, sizeof(float) * N));
    double* sc = p->red + 4096;
    launch(p, k_dots<2>, PARTS, 256, n, (const double*)p->cg_b, (const double*)p->cg_b,
           (const double*)p->cg_r, (const double*)p->cg_r, p->red);
    launch(p, k_dots_final, 1, 1024, PARTS, 2, (const double*)p->red, sc + 5);
    GS_LAUNCH();
    double hs[2];
    GS_CUDA(cudaMemcpyAsync(hs, sc + 5, 2 * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    const double bnorm = sqrt(hs[0]);
    double relres = bnorm > 0.0 ? sqrt(hs[1]) / bnorm : 0.0;
    int it = 0;
    int* it_d = p->i_scalar + 12;
    double* res_d = p->red + RES_SLOT;
    for (; it < 10 && relres > tol; it++) {
        int nn = n, mi = max_iter;
        double rt = 1.0e-5;
        void* args[] = {(void*)&nn, (void*)&p->nbr, (void*)&p->nnb, (void*)&p->dcoef, (void*)&p->farea,
                        (void*)&p->dfix, (void*)&p->cg_r, (void*)&p->f32a, (void*)&p->f32b, (void*)&p->f32c,
                        (void*)&p->f32d, (void*)&p->f32e, (void*)&p->red, (void*)&rt, (void*)&mi, (void*)&it_d,
                        (void*)&res_d};
        GS_TRY(cg_launch(p, (const void*)k_cg_coop32, args));
        launch(p, k_add_f32_d, G, B, n, (const float*)p->f32a, p->cg_x);
        launch(p, k_cg_resid, G, B, n, p->W, p->flat, (const int*)p->nbr, (const int8_t*)p->nnb,
               (const double*)p->dcoef, (const double*)p->farea, (const uint8_t*)p->outlet, (const double*)p->cg_b,
               (const double*)p->cg_x, p->cg_r);
        launch(p, k_dots<1>, PARTS, 256, n, (const double*)p->cg_r, (const double*)p->cg_r, (const double*)nullptr,
               (const double*)nullptr, p->red);
        launch(p, k_dots_final, 1, 1024, PARTS, 1, (const double*)p->red, sc + 3);
        GS_LAUNCH();
        GS_CUDA(cudaMemcpyAsync(hs, sc + 3, sizeof(double), cudaMemcpyDeviceToHost, p->stream));
        GS_CUDA(cudaStreamSynchronize(p->stream));
        relres = bnorm > 0.0 ? sqrt(hs[0]) / bnorm : 0.0;
        if (!(relres == relres)) break;
    }
    p->refine_iters += it;
    *outer = it;
    *relres_out = relres;
    return GS_OK;
}

int hillslope(gs_plan* p, double* h, double* cum_ed, double* eb, double sealevel, double cda,
              double cdm, double dt, double rtol, int max_iter, gs_stats* st) {
    const int n = (int)p->n;
    GS_TRY(rec_hill(p, h));
    if (n == 0) return GS_OK;
    const int B = 256, G = grid_for(n, B);
    if (cda == 0.0 && cdm == 0.0) {
        // no diffusion; the step's land/sea mask (hillslope.py:620) is still kept
        launch(p, k_sea_of, G, B, n, (const double*)h, sealevel, p->dsea);
        GS_LAUNCH();
        p->dvalid = 0;
        p->hill_sea = 1;
        return GS_OK;
    }
    // operator for the current land/sea mask: every row when the parameters
    // changed, else only the rows next to a coastline that moved
    const bool fresh = !(p->dvalid && p->dvalid_dt == dt && p->dvalid_cda == cda && p->dvalid_cdm == cdm);
    launch(p, k_sea_of, G, B, n, (const double*)h, sealevel, p->dsea2);
    if (fresh)
        launch(p, k_diff_rows, G, B, n, p->W, p->flat, (const uint8_t*)p->dsea2, cda, cdm, dt, (const int*)p->nbr,
               (const int8_t*)p->nnb, (const double*)p->elen, (const double*)p->vdist, (const double*)p->farea,
               (const uint8_t*)p->outlet, p->dcoef);
    else
        launch(p, k_diff_rows_dirty, G, B, n, p->W, p->flat, (const uint8_t*)p->dsea2, (const uint8_t*)p->dsea, cda,
               cdm, dt, (const int*)p->nbr, (const int8_t*)p->nnb, (const double*)p->elen,
               (const double*)p->vdist, (const double*)p->farea, (const uint8_t*)p->outlet, p->dcoef);
    GS_LAUNCH();
    std::swap(p->dsea, p->dsea2);
    p->dvalid = 1;
    p->hill_sea = 1;
    p->dvalid_dt = dt;
    p->dvalid_cda = cda;
    p->dvalid_cdm = cdm;
    double* hold = p->hl;
    launch(p, k_copy_d2, G, B, n, (const double*)h, hold);
    GS_LAUNCH();
    if (p->fp32) {
        launch(p, k_cg_init, G, B, n, p->W, p->flat, (const int*)p->nbr, (const int8_t*)p->nnb,
               (const double*)p->dcoef, (const double*)p->farea, (const uint8_t*)p->outlet, (const double*)hold,
               p->cg_x, p->cg_b, p->cg_r, p->cg_z, p->cg_p);
        GS_LAUNCH();
        int outer = 0;
        double relres = 0.0;
        const double tol = std::max(rtol, p->refine_tol);
        GS_TRY(hillslope_refine32(p, tol, max_iter, &outer, &relres));
        launch(p, k_hill_apply, G, B, n, (const double*)hold, (const double*)p->cg_x, dt, h, cum_ed, eb,
               (double*)nullptr);
        GS_LAUNCH();
        if (st) {
            st->cg_iters = outer;
            st->cg_relres = relres;
        }
        if (!(relres == relres)) {
            set_error(GS_ENONFINITE, "hillslope FP32 CG produced a non-finite residual");
            return GS_ENONFINITE;
        }
        if (relres > tol) {
            set_error(GS_EMAXITER, "hillslope FP32 refinement did not reach its tolerance");
            return GS_EMAXITER;
        }
        return GS_OK;
    }
    int* it_d = p->i_scalar + 12;
    double* res_d = p->red + RES_SLOT;
    GS_TRY(cg_second_direction(p));
    // The CG starts from h plus the last step's diffusion change: the change
    // varies slowly from step to step, so the start residual is a fraction of
    // the change's own and one iteration fewer reaches the tolerance.  The
    // solution is the same to the solver tolerance.
    if (!p->hill_dprev) {
        GS_CUDA(cudaMalloc((void**)&p->hill_dprev, sizeof(double) * (size_t)n));
        p->hill_dprev_ok = 0;
    }
    const double* guess = nullptr;
    if (p->hill_dprev_ok && p->warm_start) {
        launch(p, k_hill_guess, G, B, n, (const double*)hold, (const double*)p->hill_dprev,
               (const uint8_t*)p->dfix, p->cg_x);
        GS_LAUNCH();
        guess = p->cg_x;   // read before written, row by row, with equal values
    }
    {
        int nn = n, mi = max_iter;
        double rt = rtol;
        const double* x0 = hold;
        void* args[] = {(void*)&nn, (void*)&p->nbr, (void*)&p->nnb, (void*)&p->dcoef, (void*)&p->farea,
                        (void*)&p->dfix, (void*)&x0, (void*)&p->cg_x, (void*)&p->cg_b, (void*)&p->cg_r,
                        (void*)&p->cg_z, (void*)&p->cg_p, (void*)&p->cg_p2, (void*)&p->cg_ap, (void*)&p->red,
                        (void*)&rt, (void*)&mi, (void*)&it_d, (void*)&res_d, (void*)&guess};
        cudaEvent_t stop = nullptr;
        if (p->profiling) prof_begin(p, (const void*)k_cg_coop, &stop);
        GS_CUDA(cudaLaunchCooperativeKernel((const void*)k_cg_coop, p->coop_blocks, 256, args, 0, p->stream));
        if (stop) cudaEventRecord(stop, p->stream);
        p->launches++;
    }
    launch(p, k_hill_apply, G, B, n, (const double*)hold, (const double*)p->cg_x, dt, h, cum_ed, eb,
           p->hill_dprev);
    GS_LAUNCH();
    p->hill_dprev_ok = p->warm_start;
    int it = 0;
    double relres = 0.0;
    GS_CUDA(cudaMemcpyAsync(&it, it_d, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaMemcpyAsync(&relres, res_d, sizeof(double), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    if (st) {
        st->cg_iters = it;
        st->cg_relres = relres;
    }
    if (!(relres == relres)) {
        set_error(GS_ENONFINITE, "hillslope CG produced a non-finite residual");
        return GS_ENONFINITE;
    }
    if (relres > rtol) {
        set_error(GS_EMAXITER, "hillslope CG reached max_iter");
        return GS_EMAXITER;
    }
    return GS_OK;
}

// Solve (I + L) x = rhs on a sub-mesh of m rows given as rows (diag, then
// one coefficient per neighbour slot, [W+1][m], the hillslope layout; slot-major
// [W][m] neighbours, -1 or a zero coefficient where a neighbour lies outside),
// rows without area held fixed as in the hillslope solve; the cooperative CG on
// the area-weighted symmetric form.  Used by the non-linear lake diffusion of
// the sediment step.
// the worst relative residual of a run of solves (NaN wins), for one check at its end
__global__ void k_cg_fold(const double* __restrict__ res, double* worst) {
    const double r = *res, w = *worst;
    if (!(r == r) || r > w) *worst = r;
}

int diffusion_solve_on(gs_plan* p, int m, const int* nbr, const int8_t* nnb, const double* farea, const uint8_t* fix,
                       int flat, const uint8_t* outlet, const double* coef, const double* rhs, double* x, double rtol,
                       int max_iter, int* iters, const double* guess, double* worst) {
    const int n = m;
    if (n == 0) return GS_OK;
    const int B = 256, G = grid_for(n, B);
    (void)flat;
    (void)outlet;
    int* it_d = p->i_scalar + 12;
    double* res_d = p->red + RES_SLOT;
    GS_TRY(cg_second_direction(p));
    {
        int nn = n, mi = max_iter;
        double rt = rtol;
        const double* cf = coef;
        void* args[] = {(void*)&nn, (void*)&nbr, (void*)&nnb, (void*)&cf, (void*)&farea,
                        (void*)&fix, (void*)&rhs, (void*)&p->cg_x, (void*)&p->cg_b, (void*)&p->cg_r,
                        (void*)&p->cg_z, (void*)&p->cg_p, (void*)&p->cg_p2, (void*)&p->cg_ap, (void*)&p->red,
                        (void*)&rt, (void*)&mi, (void*)&it_d, (void*)&res_d, (void*)&guess};
        // a small sub-mesh (a few lakes) takes about four rows per thread and
        // no fewer blocks than SMs: fewer blocks meet at each grid barrier
        const int nb = std::min(p->coop_blocks, std::max(p->sm_count, (n + 4 * B - 1) / (4 * B)));
        cudaEvent_t stop = nullptr;
        if (p->profiling) prof_begin(p, (const void*)k_cg_coop, &stop);
        GS_CUDA(cudaLaunchCooperativeKernel((const void*)k_cg_coop, nb, 256, args, 0, p->stream));
        if (stop) cudaEventRecord(stop, p->stream);
        p->launches++;
    }
    launch(p, k_copy_d2, G, B, n, (const double*)p->cg_x, x);
    GS_LAUNCH();
    if (worst) {
        // the caller checks the worst residual of its solves once, at its end
        launch(p, k_cg_fold, 1, 1, (const double*)res_d, worst);
        GS_LAUNCH();
        if (iters) *iters = 0;
        return GS_OK;
    }
    int it = 0;
    double relres = 0.0;
    GS_CUDA(cudaMemcpyAsync(&it, it_d, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaMemcpyAsync(&relres, res_d, sizeof(double), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    if (iters) *iters = it;
    if (!(relres == relres)) {
        set_error(GS_ENONFINITE, "diffusion CG produced a non-finite residual");
        return GS_ENONFINITE;
    }
    if (relres > rtol) {
        set_error(GS_EMAXITER, "diffusion CG reached max_iter");
        return GS_EMAXITER;
    }
    return GS_OK;
}

// ---------------------------------------------------------------------------
// Adjoint of hillslope().  Forward: fixed rows F^c (flat outlets, zero area)
// keep x = h; free rows solve S_FF x_F = A_F h_F - S_FX h_X with S = A (I+L)
// symmetric.  Given lam = dJ/dx: nu = S_FF^-1 lam_F (same operator and CG),
// dJ/dh_F = A_F nu, dJ/dh_X = lam_X - sum_{free j next to X} A_j o_jX nu_j.

// warm start x0 = rhs / A (exact when L = 0: the diffusion of one step is a
// small perturbation of the identity), 0 on fixed rows
__global__ void k_cg_x0(int n, int flat, const uint8_t* __restrict__ outlet, const double* __restrict__ farea,
                        const double* __restrict__ rhs, double* x, double* b) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const bool fx = diff_fixed(k, flat, outlet, farea);
    x[k] = fx ? 0.0 : rhs[k] / farea[k];
    b[k] = fx ? 0.0 : rhs[k];
}

__global__ void k_cg_init_rhs(int n, int W, int flat, const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                              const double* __restrict__ coef, const double* __restrict__ farea,
                              const uint8_t* __restrict__ outlet, const double* __restrict__ x,
                              const double* __restrict__ b, double* r, double* z, double* pp) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (diff_fixed(k, flat, outlet, farea)) {
        r[k] = 0.0; z[k] = 0.0; pp[k] = 0.0;
        return;
    }
    const double rk = b[k] - diff_row(k, n, W, nbr, nnb, coef, farea, outlet, flat, x, true);
    r[k] = rk;
    const double zk = rk / (farea[k] * coef[k]);
    z[k] = zk;
    pp[k] = zk;
}

__global__ void k_hill_adj_out(int n, int flat, const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                               const int8_t* __restrict__ rev, const double* __restrict__ coef,
                               const double* __restrict__ farea, const uint8_t* __restrict__ outlet,
                               const double* __restrict__ nu, double* lam) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (!diff_fixed(k, flat, outlet, farea)) {
        lam[k] = farea[k] * nu[k];
        return;
    }
    double acc = lam[k];
    for (int t = 0; t < nnb[k]; t++) {
        int j = nbr[(size_t)t * n + k];
        if (j < 0 || diff_fixed(j, flat, outlet, farea)) continue;
        int s = rev[(size_t)t * n + k];
        if (s < 0) continue;
        double o = coef[(size_t)(s + 1) * n + j];
        acc = acc - farea[j] * o * nu[j];
    }
    lam[k] = acc;
}

// lam: dJ/dx (h after diffusion) on entry, dJ/dh (before) on return.  h_in
// is the elevation the forward diffused (its sea mask sets the operator).
int hillslope_adjoint(gs_plan* p, const double* h_in, double* lam, double sealevel, double cda, double cdm,
                      double dt, double rtol, int max_iter, int* iters) {
    const int n = (int)p->n;
    if (iters) *iters = 0;
    if (n == 0 || (cda == 0.0 && cdm == 0.0)) return GS_OK;
    const int B = 256, G = grid_for(n, B);
    const int PARTS = 512;
    launch(p, k_diff_coef, G, B, n, p->W, p->flat, h_in, sealevel, cda, cdm, dt, (const int*)p->nbr,
           (const int8_t*)p->nnb, (const double*)p->elen, (const double*)p->vdist, (const double*)p->farea,
           (const uint8_t*)p->outlet, p->dcoef, p->dsea);
    GS_LAUNCH();
    p->dvalid = 0;   // the forward's cached operator was overwritten
    p->hill_sea = 0;
    launch(p, k_cg_x0, G, B, n, p->flat, (const uint8_t*)p->outlet, (const double*)p->farea, (const double*)lam,
           p->cg_x, p->cg_b);
    launch(p, k_cg_init_rhs, G, B, n, p->W, p->flat, (const int*)p->nbr, (const int8_t*)p->nnb,
           (const double*)p->dcoef, (const double*)p->farea, (const uint8_t*)p->outlet, (const double*)p->cg_x,
           (const double*)p->cg_b, p->cg_r, p->cg_z, p->cg_p);
    double* sc = p->red + 4096;
    launch(p, k_dots<2>, PARTS, 256, n, (const double*)p->cg_r, (const double*)p->cg_z,
           (const double*)p->cg_b, (const double*)p->cg_b, p->red);
    launch(p, k_dots_final, 1, 1024, PARTS, 2, (const double*)p->red, sc + 5);
    launch(p, k_dots<1>, PARTS, 256, n, (const double*)p->cg_r, (const double*)p->cg_r,
           (const double*)nullptr, (const double*)nullptr, p->red);
    launch(p, k_dots_final, 1, 1024, PARTS, 1, (const double*)p->red, sc + 3);
    GS_LAUNCH();
    double hs[8];
    // sc[3] = rr, sc[5] = rz, sc[6] = bb
    GS_CUDA(cudaMemcpyAsync(hs, sc + 3, 4 * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
    GS_CUDA(cudaStreamSynchronize(p->stream));
    const double bnorm = sqrt(hs[3]);
    GS_CUDA(cudaMemcpyAsync(sc, sc + 5, sizeof(double), cudaMemcpyDeviceToDevice, p->stream));
    int it = 0;
    double relres = bnorm > 0.0 ? sqrt(hs[0]) / bnorm : 0.0;
    while (bnorm > 0.0 && relres > rtol && it < max_iter) {
        launch(p, k_cg_spmv, G, B, n, p->W, p->flat, (const int*)p->nbr, (const int8_t*)p->nnb,
               (const double*)p->dcoef, (const double*)p->farea, (const uint8_t*)p->outlet,
               (const double*)p->cg_p, p->cg_ap);
        launch(p, k_dots<1>, PARTS, 256, n, (const double*)p->cg_p, (const double*)p->cg_ap,
               (const double*)nullptr, (const double*)nullptr, p->red);
        launch(p, k_dots_final, 1, 1024, PARTS, 1, (const double*)p->red, sc + 1);
        launch(p, k_cg_update, G, B, n, p->flat, (const uint8_t*)p->outlet, (const double*)p->farea,
               (const double*)p->dcoef, (const double*)sc, p->cg_x, p->cg_r, p->cg_z,
               (const double*)p->cg_p, (const double*)p->cg_ap);
        launch(p, k_dots<2>, PARTS, 256, n, (const double*)p->cg_r, (const double*)p->cg_z,
               (const double*)p->cg_r, (const double*)p->cg_r, p->red);
        launch(p, k_dots_final, 1, 1024, PARTS, 2, (const double*)p->red, sc + 2);
        launch(p, k_cg_dir, G, B, n, (const double*)(sc + 2), sc, (const double*)p->cg_z, p->cg_p);
        launch(p, k_cg_rotate, 1, 1, (const double*)(sc + 2), sc);
        GS_LAUNCH();
        GS_CUDA(cudaMemcpyAsync(hs, sc + 3, sizeof(double), cudaMemcpyDeviceToHost, p->stream));
        GS_CUDA(cudaStreamSynchronize(p->stream));
        relres = sqrt(hs[0]) / bnorm;
        it++;
        if (!(relres == relres)) {
            set_error(GS_ENONFINITE, "hillslope adjoint CG produced a non-finite residual");
            return GS_ENONFINITE;
        }
    }
    if (iters) *iters = it;
    launch(p, k_hill_adj_out, G, B, n, p->flat, (const int*)p->nbr, (const int8_t*)p->nnb, (const int8_t*)p->rev,
           (const double*)p->dcoef, (const double*)p->farea, (const uint8_t*)p->outlet, (const double*)p->cg_x, lam);
    GS_LAUNCH();
    if (relres > rtol) {
        set_error(GS_EMAXITER, "hillslope adjoint CG reached max_iter");
        return GS_EMAXITER;
    }
    return GS_OK;
}

}  // namespace gs
