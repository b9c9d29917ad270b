// Multiple-flow-direction receivers and the flow-direction post-processing.
//
// k_mfd_receivers restates fortran/functions.F90:1544-1671 (mfdreceivers):
// one thread per vertex over the slot-major neighbour arrays, adaptive
// exponent, gid-keyed 1e-15 tie perturbation, top-R selection.  The top-R
// order for distinct slopes is the descending order the reference's quicksort
// produces; when two candidate slopes are exactly equal the reference
// quicksort/split pair (functions.F90:683-762) is replayed literally so tie
// order matches.  As in the reference, the distance of output receiver o is
// the edge length of candidate kk-1-o in candidate order (the sort permutes
// slopes and ids but not distances).
//
// k_flow_direction_post restates flowplex.py:480-540: flat routing on filled
// pits when down=True, self-sink outlets on flat models, the lsink mask.
#include "gs_plan.cuh"

namespace gs {

// --- literal replay of the reference quicksort on <=12 candidates ----------
__device__ void dev_split(double* a, int low, int high, int* mid, int* ix) {
    int left = low, right = high;
    double pivot = a[low - 1];
    int ipivot = ix[low - 1];
    for (;;) {
        if (left >= right) break;
        for (;;) {
            if (left >= right || a[right - 1] < pivot) break;
            right = right - 1;
        }
        for (;;) {
            if (left > 12) break;
            if (a[left - 1] > pivot) break;
            left = left + 1;
        }
        if (left < right) {
            double sw = a[left - 1]; a[left - 1] = a[right - 1]; a[right - 1] = sw;
            int is = ix[left - 1]; ix[left - 1] = ix[right - 1]; ix[right - 1] = is;
        }
    }
    a[low - 1] = a[right - 1];
    a[right - 1] = pivot;
    *mid = right;
    ix[low - 1] = ix[right - 1];
    ix[right - 1] = ipivot;
}

__device__ void dev_quicksort(double* a, int first, int last, int* ix) {
    // explicit stack replaying the recursion order (left part first)
    int stf[32], stl[32];
    int sp = 0;
    stf[sp] = first; stl[sp] = last; sp++;
    while (sp > 0) {
        sp--;
        int f = stf[sp], l = stl[sp];
        if (f < l) {
            int mid;
            dev_split(a, f, l, &mid, ix);
            // recursion: quicksort(first, mid-1) then quicksort(mid+1, last)
            stf[sp] = mid + 1; stl[sp] = l; sp++;
            stf[sp] = f; stl[sp] = mid - 1; sp++;
        }
    }
}

// One vertex of mfdreceivers with its candidates in arrays: any R, and the
// literal quicksort replay when candidate slopes tie exactly.  Not inlined:
// it is the only code here that needs a stack frame, and the register form
// below calls it for tied vertices only.
__device__ __noinline__ void mfd_vertex_general(int k, int n, int R, double expo, const double* __restrict__ elev,
                                                double sl, const int* __restrict__ gid, const int* __restrict__ nbr,
                                                const double* __restrict__ elen, const int8_t* __restrict__ nnb,
                                                int* __restrict__ rcv, double* __restrict__ dist,
                                                double* __restrict__ wgt, int8_t* __restrict__ rslot) {
    const double hk = elev[k];
    for (int o = 0; o < R; o++) {
        rcv[(size_t)o * n + k] = k;
        dist[(size_t)o * n + k] = 0.0;
        wgt[(size_t)o * n + k] = 0.0;
        if (rslot) rslot[(size_t)o * n + k] = -1;
    }
    if (hk <= sl) return;
    const int deg = nnb[k];
    double e = 0.0;
    for (int s = 0; s < deg; s++) {
        int nb = nbr[(size_t)s * n + k];
        double L = elen[(size_t)s * n + k];
        if (nb >= 0 && L > 0.0) {
            double val = (hk - elev[nb]) / L;
            e = (val > e) ? val : e;
        }
    }
    double fexp;
    if (e > 0) {
        double me = (e < 1.0) ? e : 1.0;
        fexp = 5.0 * me + expo;
    } else {
        fexp = 1.0;
    }
    const bool fexp_int = (fexp == floor(fexp));
    double slp[12], dst[12];
    int cid[12], cs[12];
    int kk = 0;
    for (int s = 0; s < deg; s++) {
        int nb = nbr[(size_t)s * n + k];
        double L = elen[(size_t)s * n + k];
        if (nb >= 0 && L > 0.0) {
            double d = hk - elev[nb];
            double val;
            if (d > 0.0) val = pow(d, fexp) / L;
            else if (d == 0.0) val = 0.0;
            else val = fexp_int ? pow(d, fexp) / L : -1.0;   // non-integer power of a
                                                             // negative base is NaN: no receiver
            if (val > 0.0) {
                slp[kk] = val * (1.0 - 1.0e-15 * (double)(gid ? gid[nb] : nb));
                cid[kk] = nb;
                cs[kk] = s;
                dst[kk] = L;
                kk++;
            }
        }
    }
    if (kk == 0) return;
    if (kk <= R) {
        double val = 0.0;
        for (int p = 0; p < kk; p++) {
            rcv[(size_t)p * n + k] = cid[p];
            dist[(size_t)p * n + k] = dst[p];
            if (rslot) rslot[(size_t)p * n + k] = (int8_t)cs[p];
            val = val + slp[p];
        }
        for (int p = 0; p < kk; p++) wgt[(size_t)p * n + k] = slp[p] / val;
        return;
    }
    // kk > R: top-R in descending slope order
    int top[12];
    bool tie = false;
    for (int a = 0; a < kk && !tie; a++)
        for (int b = a + 1; b < kk; b++)
            if (slp[a] == slp[b]) { tie = true; break; }
    if (!tie) {
        unsigned used = 0;
        for (int o = 0; o < R; o++) {
            int best = -1;
            for (int a = 0; a < kk; a++) {
                if (used & (1u << a)) continue;
                if (best < 0 || slp[a] > slp[best]) best = a;
            }
            used |= 1u << best;
            top[o] = best;
        }
    } else {
        double sa[12];
        int ix[12];
        for (int a = 0; a < 12; a++) { sa[a] = (a < kk) ? slp[a] : 0.0; ix[a] = a; }
        dev_quicksort(sa, 1, kk, ix);
        for (int o = 0; o < R; o++) top[o] = ix[kk - 1 - o];
    }
    double val = 0.0;
    double slope[12];
    for (int o = 0; o < R; o++) {
        int a = top[o];
        slope[o] = slp[a];
        rcv[(size_t)o * n + k] = cid[a];
        dist[(size_t)o * n + k] = dst[kk - 1 - o];
        if (rslot) rslot[(size_t)o * n + k] = (int8_t)cs[a];
        val = val + slp[a];
    }
    for (int o = 0; o < R; o++) wgt[(size_t)o * n + k] = slope[o] / val;
}

__global__ void k_mfd_receivers(int n, int W, int R, double expo, const double* __restrict__ elev,
                                double sl, const int* __restrict__ gid, const int* __restrict__ nbr,
                                const double* __restrict__ elen, const int8_t* __restrict__ nnb,
                                int* __restrict__ rcv, double* __restrict__ dist,
                                double* __restrict__ wgt, int8_t* __restrict__ rslot) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) mfd_vertex_general(k, n, R, expo, elev, sl, gid, nbr, elen, nnb, rcv, dist, wgt, rslot);
}

// Register form for R = RM <= 4 (the configurations' flowDir is 3), in two
// passes over the neighbour slots so that no per-slot array is held: the
// first finds the steepest gradient (the exponent), the second forms every
// candidate slope, sums them in slot order and keeps the RM + 1 steepest by
// insertion.  The second pass re-reads the slot's id, edge length and the
// neighbour's elevation (L1/L2 hits) instead of keeping 12 of each in
// registers, which keeps the kernel near 64 registers and the SMs full of
// warps for the gathers.  Without exact ties among the kept candidates the
// descending order is the one the reference quicksort leaves, so the result
// is bit-identical to the general form; a vertex whose new candidate equals a
// kept one goes to mfd_vertex_general (literal replay).  gid == nullptr means
// the identity numbering (one partition).
template <int RM>
__global__ void __launch_bounds__(128) k_mfd_receivers_r(int n, double expo, const double* __restrict__ elev,
                                                          double sl, const int* __restrict__ gid,
                                                          const int* __restrict__ nbr, const double* __restrict__ elen,
                                                          const int8_t* __restrict__ nnb, int* __restrict__ rcv,
                                                          double* __restrict__ dist, double* __restrict__ wgt,
                                                          int8_t* __restrict__ rslot) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double hk = elev[k];
    if (!(hk > sl)) {
#pragma unroll
        for (int o = 0; o < RM; o++) {
            rcv[(size_t)o * n + k] = k;
            dist[(size_t)o * n + k] = 0.0;
            wgt[(size_t)o * n + k] = 0.0;
            if (rslot) rslot[(size_t)o * n + k] = -1;
        }
        return;
    }
    const int deg = nnb[k];
    double e = 0.0;
    for (int s = 0; s < deg; s++) {
        const int c = nbr[(size_t)s * n + k];
        const double l = elen[(size_t)s * n + k];
        if (c >= 0 && l > 0.0) {
            const double g = (hk - elev[c]) / l;
            e = (g > e) ? g : e;
        }
    }
    double fexp;
    if (e > 0) {
        const double me = (e < 1.0) ? e : 1.0;
        fexp = 5.0 * me + expo;
    } else {
        fexp = 1.0;
    }
    const bool fexp_int = (fexp == floor(fexp));
    // candidates: slope (scaled by the global-id tie-break), kept descending;
    // strict > keeps the earlier slot ahead of an equal value
    double tv[RM + 1];
    int ts[RM + 1], tid[RM + 1];
#pragma unroll
    for (int j = 0; j <= RM; j++) {
        tv[j] = -1.0;
        ts[j] = -1;
        tid[j] = -1;
    }
    unsigned mask = 0u;
    int kk = 0;
    double tot_all = 0.0;
    bool tie = false;
    for (int s = 0; s < deg; s++) {
        const int c = nbr[(size_t)s * n + k];
        const double l = elen[(size_t)s * n + k];
        if (c < 0 || !(l > 0.0)) continue;
        const double d = hk - elev[c];
        double val;
        if (d > 0.0) val = pow(d, fexp) / l;
        else if (d == 0.0) val = 0.0;
        else val = fexp_int ? pow(d, fexp) / l : -1.0;   // non-integer power of a negative base is NaN
        if (!(val > 0.0)) continue;
        double x = val * (1.0 - 1.0e-15 * (double)(gid ? gid[c] : c));
        mask |= 1u << s;
        kk++;
        tot_all = tot_all + x;
        int xs = s, xi = c;
#pragma unroll
        for (int j = 0; j <= RM; j++) tie |= (x == tv[j]);
#pragma unroll
        for (int j = 0; j <= RM; j++) {
            if (x > tv[j]) {
                const double t = tv[j];
                const int a = ts[j], b = tid[j];
                tv[j] = x;
                ts[j] = xs;
                tid[j] = xi;
                x = t;
                xs = a;
                xi = b;
            }
        }
    }
    if (kk <= RM) {
        // every candidate is kept: receivers in slot order, weights over the
        // sum of all candidates taken in slot order
#pragma unroll
        for (int j = 0; j < RM; j++) {
            if (j < kk) {
                int o = 0;
#pragma unroll
                for (int i = 0; i < RM; i++) o += (i < kk && ts[i] < ts[j]) ? 1 : 0;
                rcv[(size_t)o * n + k] = tid[j];
                dist[(size_t)o * n + k] = elen[(size_t)ts[j] * n + k];
                wgt[(size_t)o * n + k] = tv[j] / tot_all;
                if (rslot) rslot[(size_t)o * n + k] = (int8_t)ts[j];
            } else {
                rcv[(size_t)j * n + k] = k;
                dist[(size_t)j * n + k] = 0.0;
                wgt[(size_t)j * n + k] = 0.0;
                if (rslot) rslot[(size_t)j * n + k] = -1;
            }
        }
        return;
    }
    if (tie) {
        mfd_vertex_general(k, n, RM, expo, elev, sl, gid, nbr, elen, nnb, rcv, dist, wgt, rslot);
        return;
    }
    // reference quirk: receiver o takes the edge length of candidate kk-1-o
    // in slot order (the sort permutes slopes and ids, not distances), i.e.
    // of the (o+1)-th highest candidate slot
    double tot = 0.0;
#pragma unroll
    for (int o = 0; o < RM; o++) tot = tot + tv[o];
    unsigned m = mask;
#pragma unroll
    for (int o = 0; o < RM; o++) {
        const int hs = 31 - __clz(m);
        m &= ~(1u << hs);
        rcv[(size_t)o * n + k] = tid[o];
        dist[(size_t)o * n + k] = elen[(size_t)hs * n + k];
        wgt[(size_t)o * n + k] = tv[o] / tot;
        if (rslot) rslot[(size_t)o * n + k] = (int8_t)ts[o];
    }
}

__global__ void k_flow_direction_post(int n, int W, int R, int flat, const double* __restrict__ h,
                                      int down, const double* __restrict__ lfill,
                                      const int* __restrict__ pit, const int* __restrict__ fdir,
                                      double sl, const uint8_t* __restrict__ outlet,
                                      const int* __restrict__ nbr, int* rcv, double* dist,
                                      double* wgt, int8_t* rslot, uint8_t* lsink, uint8_t* sea) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (down) {
        double sw = 0.0;
        for (int k = 0; k < R; k++) sw = sw + wgt[(size_t)k * n + i];
        if (h[i] == lfill[i] && pit[i] > -1 && fdir[i] > -1 && sw == 0.0) {
            int f = fdir[i];
            int slot = -1;
            if (f != i)
                for (int s = 0; s < W; s++)
                    if (nbr[(size_t)s * n + i] == f) { slot = s; break; }
            for (int k = 0; k < R; k++) {
                rcv[(size_t)k * n + i] = (k == 0) ? f : i;
                wgt[(size_t)k * n + i] = (k == 0) ? 1.0 : 0.0;
                rslot[(size_t)k * n + i] = (k == 0) ? (int8_t)slot : (int8_t)-1;
            }
        }
    }
    if (flat && outlet[i]) {
        for (int k = 0; k < R; k++) {
            rcv[(size_t)k * n + i] = i;
            dist[(size_t)k * n + i] = 0.0;
            wgt[(size_t)k * n + i] = 0.0;
            rslot[(size_t)k * n + i] = -1;
        }
    }
    if (!lsink) return;  // graph only: the masks are set by k_sink_mask once lFill exists
    const bool is_sea = lfill[i] <= sl;
    double sw = 0.0;
    for (int k = 0; k < R; k++) sw = sw + wgt[(size_t)k * n + i];
    lsink[i] = (sw == 0.0 && !outlet[i] && !is_sea) ? 1 : 0;
    sea[i] = is_sea ? 1 : 0;
}

// seaID (lFill <= sea level, flowplex.py:493) as a mask
__global__ void k_sea_mask(int n, const double* __restrict__ lfill, double sl, uint8_t* sea) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) sea[i] = lfill[i] <= sl ? 1 : 0;
}

// lsink (flowplex.py:531-540) from the weights and a precomputed sea mask
__global__ void k_sink_mask(int n, int R, const double* __restrict__ wgt, const uint8_t* __restrict__ outlet,
                            const uint8_t* __restrict__ sea, uint8_t* lsink) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double sw = 0.0;
    for (int k = 0; k < R; k++) sw = sw + wgt[(size_t)k * n + i];
    lsink[i] = (sw == 0.0 && !outlet[i] && !sea[i]) ? 1 : 0;
}

int sea_mask(gs_plan* p, const double* lfill, double sl, uint8_t* sea) {
    if (p->n == 0) return GS_OK;
    launch(p, k_sea_mask, grid_for(p->n, 256), 256, (int)p->n, lfill, sl, sea);
    GS_LAUNCH();
    return GS_OK;
}

int sink_mask(gs_plan* p, const double* wgt, const uint8_t* sea, uint8_t* lsink) {
    if (p->n == 0) return GS_OK;
    launch(p, k_sink_mask, grid_for(p->n, 256), 256, (int)p->n, p->R, wgt, (const uint8_t*)p->outlet, sea,
           lsink);
    GS_LAUNCH();
    return GS_OK;
}

int receivers(gs_plan* p, int nrcv, double exp, const double* elev, double sl, const int* gid,
              int* rcv, double* dist, double* wgt, int8_t* rslot) {
    if (nrcv < 1 || nrcv > 12) {
        set_error(GS_EINVAL, "mfdreceivers: nrcv must be in 1..12");
        return GS_EINVAL;
    }
    if (p->n == 0) return GS_OK;
    const int* g = gid == p->gid ? nullptr : gid;   // the plan's own numbering is the identity
    const int G = grid_for(p->n, 128), n = (int)p->n;
    switch (nrcv) {
        case 1: launch(p, k_mfd_receivers_r<1>, G, 128, n, exp, elev, sl, g, p->nbr, p->elen, p->nnb, rcv, dist, wgt, rslot); break;
        case 2: launch(p, k_mfd_receivers_r<2>, G, 128, n, exp, elev, sl, g, p->nbr, p->elen, p->nnb, rcv, dist, wgt, rslot); break;
        case 3: launch(p, k_mfd_receivers_r<3>, G, 128, n, exp, elev, sl, g, p->nbr, p->elen, p->nnb, rcv, dist, wgt, rslot); break;
        case 4: launch(p, k_mfd_receivers_r<4>, G, 128, n, exp, elev, sl, g, p->nbr, p->elen, p->nnb, rcv, dist, wgt, rslot); break;
        default:
            launch(p, k_mfd_receivers, G, 128, n, p->W, nrcv, exp, elev, sl, g, p->nbr, p->elen, p->nnb, rcv, dist,
                   wgt, rslot);
    }
    GS_LAUNCH();
    return GS_OK;
}

int flow_direction(gs_plan* p, const double* h, bool down, const double* lfill, const int* pit_ids,
                   const int* flat_dirs, double sealevel, int* rcv, double* dist, double* wgt,
                   int8_t* rslot, uint8_t* lsink, uint8_t* sea) {
    GS_TRY(receivers(p, p->R, 1.1, h, sealevel, p->gid, rcv, dist, wgt, rslot));
    return flow_direction_post(p, h, down, lfill, pit_ids, flat_dirs, sealevel, rcv, dist, wgt, rslot, lsink, sea);
}

int flow_direction_post(gs_plan* p, const double* h, bool down, const double* lfill, const int* pit_ids,
                        const int* flat_dirs, double sealevel, int* rcv, double* dist, double* wgt,
                        int8_t* rslot, uint8_t* lsink, uint8_t* sea) {
    if (p->n == 0) return GS_OK;
    launch(p, k_flow_direction_post, grid_for(p->n, 256), 256, (int)p->n, p->W, p->R, p->flat, h,
           down ? 1 : 0, lfill, pit_ids, flat_dirs, sealevel, p->outlet, p->nbr, rcv, dist, wgt,
           rslot, lsink, sea);
    GS_LAUNCH();
    return GS_OK;
}

}  // namespace gs

namespace gs {

// Reverse of the slope-weight computation of k_mfd_receivers with the
// receiver choice held fixed (the slots in rslot): given gw[o][k] = dJ/dw_ok,
// writes dJ/dz_k to gself[k] and dJ/dz of the neighbour in slot s to
// gnb[s][k].  The weights are w_o = slp_o / sum(slp), slp_o = (z_k - z_o)^f /
// L_o (1 - 1e-15 gid_o), and the adaptive exponent f = 5 min(e, 1) + expo
// with e the steepest descent (z_k - z_a) / L_a.  Cells without MFD receivers
// (sea, outlets, flat-routed cells) carry no derivative.
__global__ void k_mfd_weights_adj(int n, int W, int R, double expo, const double* __restrict__ z, double sl,
                                  const int* __restrict__ gid, const int* __restrict__ nbr,
                                  const double* __restrict__ elen, const int8_t* __restrict__ nnb,
                                  const int8_t* __restrict__ rslot, const double* __restrict__ gw,
                                  double* gself, double* gnb) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    for (int s = 0; s < W; s++) gnb[(size_t)s * n + k] = 0.0;
    gself[k] = 0.0;
    const double hk = z[k];
    if (hk <= sl) return;
    int so[MAXR];
    int nsel = 0;
    for (int o = 0; o < R; o++) {
        int s = rslot[(size_t)o * n + k];
        so[o] = s;
        if (s >= 0) nsel++;
    }
    if (nsel == 0) return;
    const int deg = nnb[k];
    double e = 0.0;
    int a = -1;
    for (int s = 0; s < deg; s++) {
        int nb = nbr[(size_t)s * n + k];
        double L = elen[(size_t)s * n + k];
        if (nb >= 0 && L > 0.0) {
            double val = (hk - z[nb]) / L;
            if (val > e) { e = val; a = s; }
        }
    }
    double fexp, dfe = 0.0;
    if (e > 0) {
        double me = (e < 1.0) ? e : 1.0;
        fexp = 5.0 * me + expo;
        if (e < 1.0) dfe = 5.0;
    } else {
        fexp = 1.0;
    }
    double slp[MAXR], dval[MAXR], fval[MAXR], gfac[MAXR];
    double V = 0.0;
    for (int o = 0; o < R; o++) {
        slp[o] = 0.0;
        int s = so[o];
        if (s < 0) continue;
        int nb = nbr[(size_t)s * n + k];
        double L = elen[(size_t)s * n + k];
        double d = hk - z[nb];
        if (!(d > 0.0) || !(L > 0.0)) return;   // not an MFD receiver (flat routing): no derivative
        double val = pow(d, fexp) / L;
        gfac[o] = 1.0 - 1.0e-15 * (double)gid[nb];
        slp[o] = val * gfac[o];
        dval[o] = fexp * pow(d, fexp - 1.0) / L;
        fval[o] = val * log(d);
        V = V + slp[o];
    }
    if (!(V > 0.0)) return;
    double sw = 0.0;
    for (int o = 0; o < R; o++)
        if (so[o] >= 0) sw += gw[(size_t)o * n + k] * (slp[o] / V);
    double gs_ = 0.0, gf = 0.0;
    for (int o = 0; o < R; o++) {
        int s = so[o];
        if (s < 0) continue;
        double gslp = (gw[(size_t)o * n + k] - sw) / V;
        double gval = gslp * gfac[o];
        double gd = gval * dval[o];
        gf += gval * fval[o];
        gs_ += gd;
        gnb[(size_t)s * n + k] -= gd;
    }
    if (dfe != 0.0 && a >= 0) {
        double La = elen[(size_t)a * n + k];
        double ge = gf * dfe / La;
        gs_ += ge;
        gnb[(size_t)a * n + k] -= ge;
    }
    gself[k] = gs_;
}

// gz[v] += gself[v] + sum over the cells k that have v as neighbour of gnb[slot of v at k][k]
__global__ void k_nb_gather(int n, const int* __restrict__ nbr, const int8_t* __restrict__ nnb,
                            const int8_t* __restrict__ rev, const double* __restrict__ gself,
                            const double* __restrict__ gnb, double* gz) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    double acc = gself[v];
    for (int t = 0; t < nnb[v]; t++) {
        int k = nbr[(size_t)t * n + v];
        if (k < 0) continue;
        int s = rev[(size_t)t * n + v];
        if (s >= 0) acc += gnb[(size_t)s * n + k];
    }
    gz[v] += acc;
}

// dJ/dz of the surface the receivers were built on, accumulated into gz,
// from dJ/dw (gw, receiver-major [R][n]); gself/gnb are [n] / [W][n] scratch.
int receivers_adjoint(gs_plan* p, const double* z, double sl, const int8_t* rslot, const double* gw, double* gself,
                      double* gnb, double* gz) {
    const int n = (int)p->n;
    if (n == 0) return GS_OK;
    launch(p, k_mfd_weights_adj, grid_for(n, 128), 128, n, p->W, p->R, 1.1, z, sl, (const int*)p->gid,
           (const int*)p->nbr, (const double*)p->elen, (const int8_t*)p->nnb, rslot, gw, gself, gnb);
    launch(p, k_nb_gather, grid_for(n, 256), 256, n, (const int*)p->nbr, (const int8_t*)p->nnb,
           (const int8_t*)p->rev, (const double*)gself, (const double*)gnb, gz);
    GS_LAUNCH();
    return GS_OK;
}

}  // namespace gs
