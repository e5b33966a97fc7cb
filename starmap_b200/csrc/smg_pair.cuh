// smg_pair.cuh -- device code of the pair kernel's work item (shared by the
// plain per-phase launch and the batched persistent kernel).
#pragma once
#include "smg_device.cuh"

namespace smg {

// ---------------------------------------------------------------------------
// Pair kernel: destination-centric, one thread per two adjacent points of a
// row (x = 2t, 2t+1), a CTA per (group of destinations, row).  Each coupling
// term is formed from the source values at the stencil neighbours (128-bit
// loads of the neighbouring rows for y/z differences, 64-bit loads for the x
// difference), divided exactly by h (sdiv), multiplied by M_d(j,i) and folded
// in sumcell order; the update runs in registers and the pair is stored once.
// A destination's couplings come in at most three runs (its x-, y- and
// z-lists); within a run the stencil offsets, h and the division are fixed,
// so they are selected once per run.  No shared memory and no barriers.
// DIV: the division mode of the launch (tdiv); REC: adjoint recording of the
// coupling sums and pre-phase values (wrec/prec).
// ---------------------------------------------------------------------------
// Loads of the state U.  NC: the read-only (non-coherent) path, valid when U
// is not written during the launch by another CTA that this CTA could read
// after (one launch per phase).  Otherwise (persistent batched kernel, which
// reads in phase p+1 what other CTAs wrote in phase p after a grid barrier)
// ordinary loads, which observe those writes after the barrier's acquire.
template <bool NC>
__device__ __forceinline__ double ldU(const double* p) {
    if (NC) return __ldg(p);
    return *p;
}
template <bool NC>
__device__ __forceinline__ double2 ldU2(const double* p) {
    if (NC) return __ldg(reinterpret_cast<const double2*>(p));
    return *reinterpret_cast<const double2*>(p);
}


__device__ __forceinline__ void pair_coef(const PairDest& dj, int k, const double* Fbase_unused, long long pt,
                                          bool v1, double& c0, double& c1) {
    const double* p = dj.fp[k];
    if (p) {
        if (v1) {
            const double2 f = __ldg(reinterpret_cast<const double2*>(p + pt));
            c0 = f.x;
            c1 = f.y;
        } else {
            c0 = __ldg(p + pt);
            c1 = 0.0;
        }
    } else {
        c0 = c1 = dj.sc[k];
    }
}

// One work item of the pair kernel: destinations [grp*group, ...) of row `row`,
// points of chunk `chunk` (bdim threads, two points each).  Shared by the
// plain launch (one item per CTA) and the batched persistent kernel.
template <int MODE, int DIV, int UNROLL, bool NC = true, bool REC = false>
__device__ __forceinline__ void pair_item(const PairArgs& a, int kf, int grp, int chunk, int row, int tid, int bdim) {
    const int y = row % a.g.B[1];
    const int z = row / a.g.B[1];
    const int t = chunk * bdim + tid;
    const int x0 = 2 * t;
    if (x0 >= a.g.B[0]) return;
    const int x1 = x0 + 1;
    const long long pt = (long long)z * a.g.s2 + (long long)y * a.g.s1 + x0;
    const double* Upt = a.U + pt;
    // stencil offsets (elements, relative to x0) for both source grid types
    int oh0[2], ol0[2], oh1[2], ol1[2], ry[4];   // ry: axis 1 (hi, lo) per g2
    int rz[4];                                    // axis 2 (hi, lo) per g2
#pragma unroll
    for (int g2 = 0; g2 < 2; ++g2) {
        int hi, lo;
        stencil(x0, a.g.n[0], a.g.bc[0], g2, hi, lo);
        oh0[g2] = hi - x0;
        ol0[g2] = lo - x0;
        stencil(x1, a.g.n[0], a.g.bc[0], g2, hi, lo);
        oh1[g2] = hi - x0;
        ol1[g2] = lo - x0;
        stencil(y, a.g.n[1], a.g.bc[1], g2, hi, lo);
        ry[2 * g2] = (hi - y) * (int)a.g.s1;
        ry[2 * g2 + 1] = (lo - y) * (int)a.g.s1;
        stencil(z, a.g.n[2], a.g.bc[2], g2, hi, lo);
        rz[2 * g2] = (hi - z) * (int)a.g.s2;
        rz[2 * g2 + 1] = (lo - z) * (int)a.g.s2;
    }
    const int d0 = grp * a.group;
    const int d1 = min(d0 + a.group, a.ndest);
    for (int di = d0; di < d1; ++di) {
        const PairDest& dj = a.dests[di];
        const int ex0 = dj.ext[0];
        if (y >= dj.ext[1] || z >= dj.ext[2] || x0 >= ex0) continue;
        const bool v1 = x1 < ex0;
        double* Uj = a.U + pt + dj.off;
        double u0, u1;
        if (v1) {
            const double2 u = *reinterpret_cast<const double2*>(Uj);
            u0 = u.x;
            u1 = u.y;
        } else {
            u0 = *Uj;
            u1 = 0.0;
        }
        double q0, q1, s0, s1, E0, E1;
        pair_coef(dj, kCoefQ, nullptr, pt, v1, q0, q1);
        pair_coef(dj, kCoefS, nullptr, pt, v1, s0, s1);
        pair_coef(dj, kCoefE, nullptr, pt, v1, E0, E1);
        double SA = 0.0, SB = 0.0;
        bool first = true;
        for (int r = 0; r < kPairRuns; ++r) {
            const int cb = dj.run[r], ce = dj.run[r + 1];
            if (cb == ce) continue;
            const int code = dj.code[r];
            const int ax = code >> 1, g2 = code & 1;
            const double hh = ax == 0 ? a.g.h[0] : (ax == 1 ? a.g.h[1] : a.g.h[2]);
            const double rr = ax == 0 ? a.rh[0] : (ax == 1 ? a.rh[1] : a.rh[2]);
            const int ee = ax == 0 ? a.exact_recip[0] : (ax == 1 ? a.exact_recip[1] : a.exact_recip[2]);
            if (ax == 0) {
                // x difference: four 64-bit loads per coupling (both points)
                const int ha = g2 ? oh0[1] : oh0[0], la = g2 ? ol0[1] : ol0[0];
                const int hb = v1 ? (g2 ? oh1[1] : oh1[0]) : 0, lb = v1 ? (g2 ? ol1[1] : ol1[0]) : 0;
                int c = cb;
                if (UNROLL >= 2) {
                    for (; c + 1 < ce; c += 2) {
                        const int o0 = a.coff[c], o1 = a.coff[c + 1];
                        const double w0 = a.cw[c], w1 = a.cw[c + 1];
                        const double a0 = ldU<NC>(Upt + (o0 + ha)), b0 = ldU<NC>(Upt + (o0 + la));
                        const double c0 = ldU<NC>(Upt + (o0 + hb)), e0 = ldU<NC>(Upt + (o0 + lb));
                        const double a1 = ldU<NC>(Upt + (o1 + ha)), b1 = ldU<NC>(Upt + (o1 + la));
                        const double c1 = ldU<NC>(Upt + (o1 + hb)), e1 = ldU<NC>(Upt + (o1 + lb));
                        const double tA0 = __dmul_rn(tdiv<DIV>(__dsub_rn(a0, b0), hh, rr, ee), w0);
                        const double tB0 = __dmul_rn(tdiv<DIV>(__dsub_rn(c0, e0), hh, rr, ee), w0);
                        const double tA1 = __dmul_rn(tdiv<DIV>(__dsub_rn(a1, b1), hh, rr, ee), w1);
                        const double tB1 = __dmul_rn(tdiv<DIV>(__dsub_rn(c1, e1), hh, rr, ee), w1);
                        if (first) { SA = tA0; SB = tB0; first = false; }
                        else { SA = __dadd_rn(SA, tA0); SB = __dadd_rn(SB, tB0); }
                        SA = __dadd_rn(SA, tA1);
                        SB = __dadd_rn(SB, tB1);
                    }
                }
                for (; c < ce; ++c) {
                    const int o = a.coff[c];
                    const double w = a.cw[c];
                    const double dA = tdiv<DIV>(__dsub_rn(ldU<NC>(Upt + (o + ha)), ldU<NC>(Upt + (o + la))), hh, rr, ee);
                    const double dB = tdiv<DIV>(__dsub_rn(ldU<NC>(Upt + (o + hb)), ldU<NC>(Upt + (o + lb))), hh, rr, ee);
                    const double tA = __dmul_rn(dA, w), tB = __dmul_rn(dB, w);
                    if (first) { SA = tA; SB = tB; first = false; }
                    else { SA = __dadd_rn(SA, tA); SB = __dadd_rn(SB, tB); }
                }
            } else {
                // y or z difference: two 128-bit loads per coupling (both points)
                const int oh = ax == 1 ? (g2 ? ry[2] : ry[0]) : (g2 ? rz[2] : rz[0]);
                const int ol = ax == 1 ? (g2 ? ry[3] : ry[1]) : (g2 ? rz[3] : rz[1]);
                int c = cb;
                if (UNROLL >= 2) {
                    // two couplings per iteration: all four row loads issued first
                    for (; c + 1 < ce; c += 2) {
                        const int o0 = a.coff[c], o1 = a.coff[c + 1];
                        const double w0 = a.cw[c], w1 = a.cw[c + 1];
                        const double2 hv0 = ldU2<NC>(Upt + (o0 + oh));
                        const double2 lv0 = ldU2<NC>(Upt + (o0 + ol));
                        const double2 hv1 = ldU2<NC>(Upt + (o1 + oh));
                        const double2 lv1 = ldU2<NC>(Upt + (o1 + ol));
                        const double tA0 = __dmul_rn(tdiv<DIV>(__dsub_rn(hv0.x, lv0.x), hh, rr, ee), w0);
                        const double tB0 = __dmul_rn(tdiv<DIV>(__dsub_rn(hv0.y, lv0.y), hh, rr, ee), w0);
                        const double tA1 = __dmul_rn(tdiv<DIV>(__dsub_rn(hv1.x, lv1.x), hh, rr, ee), w1);
                        const double tB1 = __dmul_rn(tdiv<DIV>(__dsub_rn(hv1.y, lv1.y), hh, rr, ee), w1);
                        if (first) { SA = tA0; SB = tB0; first = false; }
                        else { SA = __dadd_rn(SA, tA0); SB = __dadd_rn(SB, tB0); }
                        SA = __dadd_rn(SA, tA1);
                        SB = __dadd_rn(SB, tB1);
                    }
                }
                for (; c < ce; ++c) {
                    const int o = a.coff[c];
                    const double w = a.cw[c];
                    const double2 hv = ldU2<NC>(Upt + (o + oh));
                    const double2 lv = ldU2<NC>(Upt + (o + ol));
                    const double tA = __dmul_rn(tdiv<DIV>(__dsub_rn(hv.x, lv.x), hh, rr, ee), w);
                    const double tB = __dmul_rn(tdiv<DIV>(__dsub_rn(hv.y, lv.y), hh, rr, ee), w);
                    if (first) { SA = tA; SB = tB; first = false; }
                    else { SA = __dadd_rn(SA, tA); SB = __dadd_rn(SB, tB); }
                }
            }
        }
        const double WA = -SA, WB = -SB;
        if (REC) {   // adjoint recording of the coupling sum and the values before the phase
            double* wp = a.wrec + (long long)di * a.g.cs + pt;
            double* pp = a.prec + (long long)di * a.g.cs + pt;
            wp[0] = WA;
            pp[0] = u0;
            if (v1) {
                wp[1] = WB;
                pp[1] = u1;
            }
        }
        if (MODE == 0) {
            u0 = upd(u0, WA, q0, s0, E0, a.hdt);
            u1 = upd(u1, WB, q1, s1, E1, a.hdt);
            if (a.filter_substep) {
                double f0, f1;
                pair_coef(dj, kf == 1 ? kCoefF1 : kCoefF2, nullptr, pt, v1, f0, f1);
                u0 = __dmul_rn(u0, f0);
                u1 = __dmul_rn(u1, f1);
            }
        } else {
            double f0 = 1.0, f1 = 1.0, g0 = 1.0, g1 = 1.0;   // first / second substep filter
            if (a.filter_substep) {
                pair_coef(dj, MODE == 2 ? kCoefF2 : kCoefF1, nullptr, pt, v1, f0, f1);
                pair_coef(dj, MODE == 2 ? kCoefF1 : kCoefF2, nullptr, pt, v1, g0, g1);
            }
            u0 = upd(u0, WA, q0, s0, E0, a.hdt);
            u1 = upd(u1, WB, q1, s1, E1, a.hdt);
            if (a.filter_substep) { u0 = __dmul_rn(u0, f0); u1 = __dmul_rn(u1, f1); }
            u0 = upd(u0, WA, q0, s0, E0, a.hdt);
            u1 = upd(u1, WB, q1, s1, E1, a.hdt);
            if (a.filter_substep) { u0 = __dmul_rn(u0, g0); u1 = __dmul_rn(u1, g1); }
        }
        if (v1) *reinterpret_cast<double2*>(Uj) = make_double2(u0, u1);
        else *Uj = u0;
    }
}

}  // namespace smg
