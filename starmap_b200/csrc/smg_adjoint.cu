// smg_adjoint.cu -- discrete adjoint of the time loop.
//
// Forward: smg_forward runs the Strang loop from the current state and keeps
// a copy of the state every `ckpt_every` steps.  Backward: for each segment,
// last to first, the state is recomputed from its checkpoint with one launch
// per phase (A k=1, B, A k=2 -- the fused A-A form of smg_run computes the
// same numbers but does not expose the state between the two A phases),
// recording the state before every phase and every destination's coupling sum
//   W_j = -sum_c M_d(j,i_c) * D_c U_{i_c}.
// Then the phases are walked backwards.  A phase updates each destination j
// pointwise, U'_j = f(U_j, W_j; s_j, E_j, Q_j, F) (one or two dt/2 substeps of
// starmap_solver.m:352-357, 401-411), where E = expm1div(-s*dt/2).  With
// lambda' the adjoint after the phase:
//   k_adj_point  (per destination point)
//       lambda_j  = (dU'/dU)  lambda'_j
//       v_j       = (dU'/dW)  lambda'_j
//       grad_s   += (dU'/ds)  lambda'_j     (through E as well)
//       grad_Q   += (dU'/dQ)  lambda'_j
//   k_adj_transpose  (per source point)
//       lambda_i += - sum_{j,c: i_c = i} M_d(j,i) (D_c^T v_j)
// i.e. the transposed stencil and coupling.  The seed is the misfit
// J = 1/2 sum (U_1(T) - obs)^2 on the zeroth moment (smg_misfit) or any
// adjoint state (smg_adjoint_seed); after all phases lambda = dJ/dU(0).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <string>
#include <vector>

#include "../../include/starmap_gpu.h"
#include "smg_internal.h"
#include "smg_pair.cuh"

namespace smg {

struct AdjCoef {       // resolved coefficient of one destination in one phase
    const double* p;   // array slot, or nullptr -> scalar s
    double s;
};

struct AdjDest {
    int comp;          // component index
    int ext[3];
    AdjCoef sg, E, dE, Q, F1, F2;   // sigma, decay, d(decay)/d(sigma), source, substep filters
    double* gs;        // gradient slot of sigma's field (nullptr: not tracked)
    double* gq;        // gradient slot of the source field (nullptr: none)
};

struct TCoup {         // transposed coupling: source i <- destination slot v
    int vslot;         // index of the destination in the phase's destination list
    int code;          // axis*2 + (grid type of source i along axis == 2)
    int vcomp;         // component index of that destination
    int pad;
    double w;          // M_d(j,i)
};

struct AdjSrc {
    int comp;
    int ext[3];
    int tbeg, tend;
    int pslot;         // index of this component in the other phase type's destination list
};

struct AdjData {
    int64_t nsteps = 0, K = 0, nseg = 0;
    std::vector<double*> ckpt;
    double* work = nullptr;
    double* lam = nullptr;
    double* V = nullptr;
    double* rec_state = nullptr;   // [2K+1][maxdest*cs]: destination values before each phase
    double* rec_w = nullptr;       // [2K+1][maxdest*cs]: destination coupling sums
    // second recording (and work state) when there are several segments: the
    // next segment is recomputed on rstream while the adjoint of the current
    // one runs on the handle's stream
    double* rec_state2 = nullptr;
    double* rec_w2 = nullptr;
    double* work2 = nullptr;
    cudaStream_t rstream = nullptr;
    cudaStream_t sstream = nullptr;            // the sweep's stream at the highest priority (SMG_TUNE_ADJ_PRIORITY 2)
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    cudaEvent_t ev_rec[2] = {nullptr, nullptr};    // recording into buffer b complete
    cudaEvent_t ev_free[2] = {nullptr, nullptr};   // adjoint done reading buffer b
    int maxdest = 0;
    std::vector<double*> gfield;   // per user field: gradient slot (cs) or nullptr
    std::vector<double*> dEslot;   // per sigma field: d(decay)/d(sigma) slot (arrays)
    std::vector<double> dEscalar;  // per sigma field: scalar derivative
    // per phase (0 = A, 1 = B): destination and source tables, host and device
    std::vector<AdjDest> dests[2];
    std::vector<AdjSrc> srcs[2];
    std::vector<TCoup> tcoup[2];
    AdjDest* d_dests[2] = {nullptr, nullptr};
    AdjSrc* d_srcs[2] = {nullptr, nullptr};
    TCoup* d_tcoup[2] = {nullptr, nullptr};
    bool ready = false, seeded = false;
    bool tail_valid = false;       // the recording holds the last segment (written by smg_forward)
    DevField* dDE = nullptr;       // per field: d(decay)/d(sigma) (array slot or scalar), generated kernels
    double** dG = nullptr;         // per field: gradient slot or nullptr, generated kernels
    size_t bytes = 0;
    // generated recording and sweep: the recording holds each destination's
    // sigma-gradient factor per phase (rec_w) and no values before the phase
    // (rec_state stays unallocated); the precompiled kernels record both
    bool ds = false;
};

// phi'(x) for phi(x) = (exp(x)-1)/x with the reference's Taylor branch
// (starmap_solver.m:531-535): the derivative of 1 + x/2 + x^2/6 where that
// branch is taken, the series sum_k k x^(k-1)/(k+1)! for moderate |x| (the
// closed form cancels there), and (exp(x)*(x-1) + 1)/x^2 otherwise.
__host__ __device__ inline double dphi(double x) {
    if (fabs(x) <= 2e-4) return 0.5 + x / 3.0;
    if (fabs(x) < 0.25) {
        double term = 0.5, sum = 0.5;   // k = 1: 1/2!
        double f = 2.0;                  // (k+1)!
        double xp = 1.0;
        for (int k = 2; k <= 16; ++k) {
            xp *= x;
            f *= (k + 1);
            term = k * xp / f;
            sum += term;
        }
        return sum;
    }
    return (exp(x) * (x - 1.0) + 1.0) / (x * x);
}

__global__ void k_dphi(double* out, const double* sigma, long long n, double hdt) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // E = phi(-sigma*dt/2)  ->  dE/dsigma = -dt/2 * phi'(-sigma*dt/2)
    const double x = -sigma[i] * hdt;
    out[i] = -hdt * dphi(x);
}

__device__ __forceinline__ double cval(const AdjCoef& c, long long pt) { return c.p ? c.p[pt] : c.s; }

// MODE 0: phase A, one substep with filter F1 (= filter k of that A phase);
// MODE 1: phase B, two substeps (filters F1 then F2).
template <int MODE>
__global__ void __launch_bounds__(256) k_adj_point(DevGrid g, const AdjDest* dests, const double* __restrict__ pre,
                                                   const double* __restrict__ W, double* lam, double* V, double hdt) {
    const long long npts = g.s2 * g.B[2];
    const long long pt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int di = blockIdx.y;
    if (pt >= npts) return;
    const AdjDest d = dests[di];
    const int x = (int)(pt % g.s1);
    const int y = (int)((pt / g.s1) % g.B[1]);
    const int z = (int)(pt / g.s2);
    if (x >= d.ext[0] || y >= d.ext[1] || z >= d.ext[2]) return;
    const long long jo = (long long)d.comp * g.cs + pt;
    const double lp = lam[jo];
    const double u = pre[(long long)di * g.cs + pt];
    const double w = W[(long long)di * g.cs + pt];
    const double s = cval(d.sg, pt), E = cval(d.E, pt), dE = cval(d.dE, pt), q = cval(d.Q, pt);
    const double F1 = cval(d.F1, pt);
    const double r = 1.0 - hdt * s * E;          // d(substep)/dU before the filter
    double dU, dW, ds;
    if (MODE == 0) {
        const double G = w + q - s * u;
        dU = F1 * r;
        dW = F1 * hdt * E;
        ds = F1 * hdt * (-u * E + G * dE);
    } else {
        const double F2 = cval(d.F2, pt);
        const double G0 = w + q - s * u;
        const double V1 = F1 * (u + hdt * G0 * E);
        const double G1 = w + q - s * V1;
        dU = F2 * r * F1 * r;
        dW = F2 * (r * F1 * hdt * E + hdt * E);
        ds = F2 * (r * F1 * hdt * (-u * E + G0 * dE) + hdt * (-V1 * E + G1 * dE));
    }
    lam[jo] = dU * lp;
    V[(long long)di * g.cs + pt] = dW * lp;
    if (d.gs) atomicAdd(d.gs + pt, ds * lp);
    if (d.gq) atomicAdd(d.gq + pt, dW * lp);   // dU'/dQ = dU'/dW
}

// lambda_i += -sum M_d(j,i) (D^T v_j): D^T of the staggered difference of a
// source on grid type g2 along one axis (preimages of hi and lo under the
// stencil of starmap_solver.m:127-132).
__device__ __forceinline__ double dT(const double* v, int q, int n, int bc, int g2, long long st) {
    // v points at the destination slot at this source point's linear index
    if (!g2) {
        if (bc) {
            double a = v[0];
            if (q == n - 1) a += v[st];           // hi(p=n) = n-1
            double b = v[st];                      // lo(p=q+1) = q
            if (q == 0) b += v[0];                 // lo(p=0) = 0
            return a - b;
        }
        const long long om = (q == 0) ? (long long)(n - 1) * st : -st;   // p = (q-1) mod n
        return v[om] - v[0];
    }
    if (bc) {
        const double a = q >= 1 ? v[-st] : 0.0;    // hi(p=q-1) = q
        const double b = q <= n - 1 ? v[0] : 0.0;  // lo(p=q) = q
        return a - b;
    }
    const long long op = (q == n - 1) ? -(long long)(n - 1) * st : st;    // p = (q+1) mod n
    return v[0] - v[op];
}

__global__ void __launch_bounds__(256) k_adj_transpose(DevGrid g, const AdjSrc* srcs, const TCoup* tc,
                                                       const double* __restrict__ V, double* lam) {
    const long long npts = g.s2 * g.B[2];
    const long long pt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int si = blockIdx.y;
    if (pt >= npts) return;
    const AdjSrc S = srcs[si];
    const int x = (int)(pt % g.s1);
    const int y = (int)((pt / g.s1) % g.B[1]);
    const int z = (int)(pt / g.s2);
    if (x >= S.ext[0] || y >= S.ext[1] || z >= S.ext[2]) return;
    double acc = 0.0;
    for (int c = S.tbeg; c < S.tend; ++c) {
        const TCoup t = tc[c];
        const int ax = t.code >> 1;
        const int q = ax == 0 ? x : (ax == 1 ? y : z);
        const long long st = ax == 0 ? 1 : (ax == 1 ? g.s1 : g.s2);
        const double* v = V + (long long)t.vslot * g.cs + pt;
        acc += t.w * dT(v, q, g.n[ax], g.bc[ax], t.code & 1, st) / g.h[ax];
    }
    lam[(long long)S.comp * g.cs + pt] -= acc;
}

// Row form of dT for axes 1/2: both points of a pair share q, so every
// preimage is a row offset and one 128-bit load serves both points.
__device__ __forceinline__ double2 ld2(const double* p) { return *reinterpret_cast<const double2*>(p); }
__device__ __forceinline__ double2 sub2(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 add2(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

__device__ __forceinline__ double2 dT_row(const double* v, int q, int n, int bc, int g2, long long st) {
    const double2 z = make_double2(0.0, 0.0);
    if (!g2) {
        if (bc) {
            double2 a = ld2(v);
            if (q == n - 1) a = add2(a, ld2(v + st));
            double2 b = ld2(v + st);
            if (q == 0) b = add2(b, ld2(v));
            return sub2(a, b);
        }
        const long long om = (q == 0) ? (long long)(n - 1) * st : -st;
        return sub2(ld2(v + om), ld2(v));
    }
    if (bc) {
        const double2 a = q >= 1 ? ld2(v - st) : z;
        const double2 b = q <= n - 1 ? ld2(v) : z;
        return sub2(a, b);
    }
    const long long op = (q == n - 1) ? -(long long)(n - 1) * st : st;
    return sub2(ld2(v), ld2(v + op));
}

// Two adjacent points per thread (x = 2t, 2t+1): 128-bit loads for the y/z
// preimages, per-point loads for x.
__global__ void __launch_bounds__(128) k_adj_transpose2(DevGrid g, const AdjSrc* srcs, const TCoup* tc,
                                                        const double* __restrict__ V, double* lam) {
    const int tpr = (g.B[0] + 1) / 2;
    const long long rows = (long long)g.B[1] * g.B[2];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int si = blockIdx.y;
    if (t >= (long long)tpr * rows) return;
    const int x0 = 2 * (int)(t % tpr);
    const long long row = t / tpr;
    const int y = (int)(row % g.B[1]);
    const int z = (int)(row / g.B[1]);
    const AdjSrc S = srcs[si];
    if (x0 >= S.ext[0] || y >= S.ext[1] || z >= S.ext[2]) return;
    const bool v1 = x0 + 1 < S.ext[0];
    const long long pt = (long long)z * g.s2 + (long long)y * g.s1 + x0;
    double a0 = 0.0, a1 = 0.0;
    for (int c = S.tbeg; c < S.tend; ++c) {
        const TCoup tcp = tc[c];
        const int ax = tcp.code >> 1, g2 = tcp.code & 1;
        const double* v = V + (long long)tcp.vslot * g.cs + pt;
        const double f = tcp.w / g.h[ax];
        if (ax == 0) {
            a0 += f * dT(v, x0, g.n[0], g.bc[0], g2, 1);
            if (v1) a1 += f * dT(v + 1, x0 + 1, g.n[0], g.bc[0], g2, 1);
        } else {
            const int q = ax == 1 ? y : z;
            const long long st = ax == 1 ? g.s1 : g.s2;
            const double2 d = dT_row(v, q, g.n[ax], g.bc[ax], g2, st);
            a0 += f * d.x;
            a1 += f * d.y;
        }
    }
    double* L = lam + (long long)S.comp * g.cs + pt;
    L[0] -= a0;
    if (v1) L[1] -= a1;
}

// ---------------------------------------------------------------------------
// Fused backward phase.  The adjoint of destination j is kept scaled by the
// derivative of its phase's update with respect to its coupling sum,
//   Y_j = v_j = (dU'/dW)_j lambda'_j,
// because that is what the transposed coupling of that phase consumes; its
// own pointwise part lambda_j = (dU'/dU)_j lambda'_j is applied when j is
// next a target, through rho = (dU'/dU)/(dU'/dW), in which the filter of the
// last substep cancels and nothing is divided by zero: dU'/dW = F_2 (dt/2) E
// (r F_1 + 1) with E = expm1div(-s dt/2) > 0 and r = 1 - (dt/2) s E =
// exp(-s dt/2) > 0 (one substep: F_1 (dt/2) E).  With that, one launch per
// phase r, over the sources i of the phase (the destinations of phases r-1
// and r+1), does
//   lambda_i  = rho_{r+1,i} Y_i           (phase r+1's pointwise part; PM)
//   grads    += (d/ds, d/dQ of phase r+1 at i) lambda'_i
//   lambda_i -= sum_j M_d(j,i) D^T Y_j     (phase r's transposed coupling)
//   Y_i       = (dU'/dW)_{r-1,i} lambda_i  (scaled for phase r-1; NM)
// and reads/writes disjoint components (sources i, destinations j).
// PM / NM: 0 none, 1 one substep, 2 two substeps.
// ---------------------------------------------------------------------------
template <int M>
__device__ __forceinline__ double dWdU_scale(const AdjDest& d, long long pt, double hdt) {
    // dU'/dW of destination d at point pt (M = 1: one substep, 2: two)
    const double s = cval(d.sg, pt), E = cval(d.E, pt), F1 = cval(d.F1, pt);
    if (M == 1) return F1 * hdt * E;
    const double F2 = cval(d.F2, pt);
    const double r = 1.0 - hdt * s * E;
    return F2 * hdt * E * (r * F1 + 1.0);
}

// phase's pointwise adjoint from Y = (dU'/dW) lambda' at one point, with the
// gradient contributions; u, w: the destination value before the phase and
// its coupling sum (recorded)
template <int M>
__device__ __forceinline__ double pend_point(const AdjDest& d, long long pt, double u, double w, double Y,
                                             double hdt) {
    const double s = cval(d.sg, pt), E = cval(d.E, pt), q = cval(d.Q, pt), F1 = cval(d.F1, pt);
    const double r = 1.0 - hdt * s * E;
    double rho, dsdw = 0.0;
    if (M == 1) {
        rho = r / (hdt * E);
        if (d.gs) {
            const double dE = cval(d.dE, pt);
            const double G = w + q - s * u;
            dsdw = (-u * E + G * dE) / E;
        }
    } else {
        const double den = 1.0 / (hdt * E * (r * F1 + 1.0));
        rho = F1 * r * r * den;
        if (d.gs) {
            const double dE = cval(d.dE, pt);
            const double G0 = w + q - s * u;
            const double V1 = F1 * (u + hdt * G0 * E);
            const double G1 = w + q - s * V1;
            dsdw = (r * F1 * hdt * (-u * E + G0 * dE) + hdt * (-V1 * E + G1 * dE)) * den;
        }
    }
    if (d.gs) atomicAdd(d.gs + pt, dsdw * Y);
    if (d.gq) atomicAdd(d.gq + pt, Y);   // dU'/dQ = dU'/dW
    return rho * Y;
}

template <int PM, int NM>
__global__ void __launch_bounds__(128) k_adj_fused(DevGrid g, const AdjSrc* srcs, const TCoup* tc, int coup,
                                                   const AdjDest* pend, const double* __restrict__ pre,
                                                   const double* __restrict__ W, const AdjDest* next, double* Y,
                                                   double hdt) {
    const int tpr = (g.B[0] + 1) / 2;
    const long long rows = (long long)g.B[1] * g.B[2];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int si = blockIdx.y;
    if (t >= (long long)tpr * rows) return;
    const int x0 = 2 * (int)(t % tpr);
    const long long row = t / tpr;
    const int y = (int)(row % g.B[1]);
    const int z = (int)(row / g.B[1]);
    const AdjSrc S = srcs[si];
    if (x0 >= S.ext[0] || y >= S.ext[1] || z >= S.ext[2]) return;
    const bool v1 = x0 + 1 < S.ext[0];
    const long long pt = (long long)z * g.s2 + (long long)y * g.s1 + x0;
    double* Yi = Y + (long long)S.comp * g.cs + pt;
    double l0, l1 = 0.0;
    if (v1) {
        const double2 v = ld2(Yi);
        l0 = v.x;
        l1 = v.y;
    } else {
        l0 = Yi[0];
    }
    if (PM) {
        const AdjDest& d = pend[S.pslot];
        const long long rp = (long long)S.pslot * g.cs + pt;
        l0 = pend_point<PM>(d, pt, pre[rp], W[rp], l0, hdt);
        if (v1) l1 = pend_point<PM>(d, pt + 1, pre[rp + 1], W[rp + 1], l1, hdt);
    }
    if (coup) {
        double a0 = 0.0, a1 = 0.0;
        for (int c = S.tbeg; c < S.tend; ++c) {
            const TCoup tcp = tc[c];
            const int ax = tcp.code >> 1, g2 = tcp.code & 1;
            const double* v = Y + (long long)tcp.vcomp * g.cs + pt;
            const double f = tcp.w / g.h[ax];
            if (ax == 0) {
                a0 += f * dT(v, x0, g.n[0], g.bc[0], g2, 1);
                if (v1) a1 += f * dT(v + 1, x0 + 1, g.n[0], g.bc[0], g2, 1);
            } else {
                const int q = ax == 1 ? y : z;
                const long long st = ax == 1 ? g.s1 : g.s2;
                const double2 d = dT_row(v, q, g.n[ax], g.bc[ax], g2, st);
                a0 += f * d.x;
                a1 += f * d.y;
            }
        }
        l0 -= a0;
        l1 -= a1;
    }
    if (NM) {
        const AdjDest& n = next[S.pslot];
        l0 *= dWdU_scale<NM>(n, pt, hdt);
        if (v1) l1 *= dWdU_scale<NM>(n, pt + 1, hdt);
    }
    if (v1) *reinterpret_cast<double2*>(Yi) = make_double2(l0, l1);
    else Yi[0] = l0;
}

template <int MODE, int DIV>
__global__ void __launch_bounds__(256, 4) k_pair_rec(PairArgs a, int kf) {
    const int bid = blockIdx.x;
    pair_item<MODE, DIV, 1, true, true>(a, kf, bid % a.ngroups, (bid / a.ngroups) % a.nchunks,
                                    bid / a.ngroups / a.nchunks, threadIdx.x, blockDim.x);
}

}  // namespace smg

using smg::AdjData;

namespace {

int afail(smg_handle* h, int code, const std::string& m) {
    h->err = m;
    return code;
}

int acuda(smg_handle* h, cudaError_t e, const char* what) {
    return afail(h, e == cudaErrorMemoryAllocation ? SMG_ENOMEM : SMG_ECUDA,
                 std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

#define A_CUDA(h, expr)                                         \
    do {                                                        \
        cudaError_t e_ = (expr);                                \
        if (e_ != cudaSuccess) return acuda((h), e_, #expr);    \
    } while (0)

size_t state_bytes(const smg_handle* h) { return (size_t)h->g.cs * h->n_sys * sizeof(double); }

// pair-kernel arguments of one phase on an arbitrary state buffer
smg::PairArgs rec_args(const smg_handle* h, int phase, double* U, double* wrec, double* prec) {
    smg::PairArgs a{};
    const auto& P = h->pair[phase];
    a.g = h->g;
    a.U = U;
    a.dests = P.d_dests;
    a.coff = P.d_coff;
    a.cw = P.d_cw;
    a.ndest = P.ndest;
    a.group = 8;
    a.ngroups = (P.ndest + a.group - 1) / a.group;
    const int tpr = (h->g.B[0] + 1) / 2;
    a.nchunks = (tpr + 63) / 64;
    a.hdt = h->hdt;
    for (int k = 0; k < 3; ++k) {
        a.rh[k] = h->rh[k];
        a.exact_recip[k] = h->exact_recip[k];
    }
    a.filter_substep = h->filter_mode == SMG_FILTER_SUBSTEP;
    a.wrec = wrec;
    a.prec = prec;
    return a;
}

cudaError_t launch_rec(const smg_handle* h, int mode, int kf, double* U, double* wrec, double* prec, int dsm, int dsw,
                       cudaStream_t st) {
    if (h->adj && h->adj->ds) return smg::launch_jit_rec(h, mode, kf, U, wrec, prec, h->adj->dDE, dsm, dsw, st);
    const int phase = mode == 1 ? 1 : 0;
    const smg::PairArgs a = rec_args(h, phase, U, wrec, prec);
    if (a.ndest == 0) return cudaSuccess;
    const unsigned nb = (unsigned)((long long)a.ngroups * a.nchunks * h->g.B[1] * h->g.B[2]);
    const int div = std::min(a.exact_recip[0], std::min(a.exact_recip[1], a.exact_recip[2]));
#define SMG_REC(D)                                                                          \
    if (mode == 1) smg::k_pair_rec<1, D><<<nb, 64, 0, st>>>(a, kf);                        \
    else if (mode == 2) smg::k_pair_rec<2, D><<<nb, 64, 0, st>>>(a, kf);                   \
    else smg::k_pair_rec<0, D><<<nb, 64, 0, st>>>(a, kf);
    if (div == 2) { SMG_REC(2) }
    else if (div == 1) { SMG_REC(1) }
    else { SMG_REC(0) }
#undef SMG_REC
    return cudaGetLastError();
}

// One segment of ks steps from state U with recording, in smg_run's phase
// order: A(k=1), then per step B and the fused A(k=2)A(k=1) -- A(k=2) alone
// after the last step.  Phase r records into slot r (2ks+1 slots).  The
// sweep reads each slot as the phase kind it has there, which the
// sigma-gradient factor recorded by the generated kernels must follow: one
// substep for the first A(k=1) and for the run's final A(k=2) (last segment),
// two for B, for the fused A-A and for a segment's closing A(k=2), which the
// sweep fuses with the next segment's A(k=1); first filter k=2 for the A
// phases after the first.
cudaError_t record_segment(smg_handle* h, int64_t ks, double* U, double* rec_w, double* rec_state, cudaStream_t st,
                           bool last) {
    const AdjData* A = h->adj;
    const size_t vb = (size_t)h->g.cs * std::max(A->maxdest, 1) * sizeof(double);
    for (int64_t r = 0; r <= 2 * ks; ++r) {
        const int kind = r == 0 ? 0 : (r & 1 ? 1 : (r < 2 * ks ? 2 : 3));
        const int mode = kind == 1 ? 1 : (kind == 2 ? 2 : 0);
        const int kf = kind == 3 ? 2 : 1;
        const int dsm = (kind == 1 || kind == 2 || (kind == 3 && !last)) ? 2 : 1;
        const int dsw = (kind == 2 || kind == 3) ? 1 : 0;
        const cudaError_t e = launch_rec(h, mode, kf, U, (double*)((char*)rec_w + vb * r),
                                         rec_state ? (double*)((char*)rec_state + vb * r) : nullptr, dsm, dsw, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

void free_adj(smg_handle* h) {
    AdjData* A = h->adj;
    if (!A) return;
    for (double* p : A->ckpt) cudaFree(p);
    cudaFree(A->work);
    cudaFree(A->lam);
    cudaFree(A->V);
    cudaFree(A->rec_state);
    cudaFree(A->rec_w);
    cudaFree(A->rec_state2);
    cudaFree(A->rec_w2);
    cudaFree(A->work2);
    if (A->rstream) cudaStreamDestroy(A->rstream);
    if (A->sstream) cudaStreamDestroy(A->sstream);
    if (A->ev_in) cudaEventDestroy(A->ev_in);
    if (A->ev_out) cudaEventDestroy(A->ev_out);
    for (int b = 0; b < 2; ++b) {
        if (A->ev_rec[b]) cudaEventDestroy(A->ev_rec[b]);
        if (A->ev_free[b]) cudaEventDestroy(A->ev_free[b]);
    }
    for (double* p : A->gfield) cudaFree(p);
    for (double* p : A->dEslot) cudaFree(p);
    cudaFree(A->dDE);
    cudaFree(A->dG);
    for (int l = 0; l < 2; ++l) {
        cudaFree(A->d_dests[l]);
        cudaFree(A->d_srcs[l]);
        cudaFree(A->d_tcoup[l]);
    }
    delete A;
    h->adj = nullptr;
}

smg::AdjCoef coef_of(const smg_handle* h, int f) {
    const smg::DevField& F = h->fields_host[f];
    return smg::AdjCoef{F.p, F.p ? 0.0 : F.s};
}

// Destination/source tables of both phases (call after dE slots exist).
int build_tables(smg_handle* h) {
    AdjData* A = h->adj;
    const int one = h->field_one;
    // destinations of each phase type in the pair table's order: the recorded
    // W / pre-values and the scratch V use that index as their slot
    std::vector<int> Dl[2];
    std::map<int, int> slot_in[2];
    for (int l = 0; l < 2; ++l)
        for (const auto& pd : h->pair[l].dests) {
            const int j = (int)((long long)pd.off / h->g.cs);
            slot_in[l][j] = (int)Dl[l].size();
            Dl[l].push_back(j);
        }
    for (int l = 0; l < 2; ++l) {
        const std::vector<int>& D = Dl[l];
        const std::vector<int>& Sset = l == 0 ? h->destB : h->destA;   // sources of the phase
        A->dests[l].clear();
        A->srcs[l].clear();
        A->tcoup[l].clear();
        std::map<int, int> slot_of;
        // phase A has three tables: single substep with filter k=1, single
        // substep with filter k=2, and the fused pair A(k=2) A(k=1) as a
        // two-substep phase (filters in that order)
        for (int rep = 0; rep < (l == 0 ? 3 : 1); ++rep)
            for (int k = 0; k < (int)D.size(); ++k) {
                const int j = D[k];
                slot_of[j] = k;
                const smg::DevComp& c = h->comps[j];
                smg::AdjDest d{};
                d.comp = j;
                for (int a = 0; a < 3; ++a) d.ext[a] = c.ext[a];
                int fs, fe;
                if (l == 1 && j == 0) {
                    fs = h->sigma_a;
                    fe = h->decay_a >= 0 ? h->decay_a : h->derived_decay_a;
                    d.F1 = d.F2 = coef_of(h, one);
                } else {
                    fs = c.sT;
                    fe = c.ET;
                    d.F1 = coef_of(h, rep == 0 ? c.F1 : c.F2);
                    d.F2 = coef_of(h, rep == 2 ? c.F1 : c.F2);
                }
                d.sg = coef_of(h, fs);
                d.E = coef_of(h, fe);
                d.dE = smg::AdjCoef{A->dEslot[fs], A->dEslot[fs] ? 0.0 : A->dEscalar[fs]};
                d.Q = coef_of(h, c.Q);
                d.gs = fs < (int)A->gfield.size() ? A->gfield[fs] : nullptr;
                d.gq = c.Q < (int)A->gfield.size() ? A->gfield[c.Q] : nullptr;
                A->dests[l].push_back(d);
            }
        // transposed couplings: for each source, every (destination, code, w) naming it
        std::map<int, std::vector<smg::TCoup>> bysrc;
        for (int j : D)
            for (int q = h->comps[j].cbeg; q < h->comps[j].cend; ++q)
                bysrc[h->coups[q].src].push_back(smg::TCoup{slot_of[j], h->coups[q].code, j, 0, h->coups[q].w});
        for (int i : Sset) {
            smg::AdjSrc s{};
            s.comp = i;
            for (int a = 0; a < 3; ++a) s.ext[a] = h->comps[i].ext[a];
            s.tbeg = (int)A->tcoup[l].size();
            for (const auto& t : bysrc[i]) A->tcoup[l].push_back(t);
            s.tend = (int)A->tcoup[l].size();
            const auto it = slot_in[1 - l].find(i);
            s.pslot = it == slot_in[1 - l].end() ? -1 : it->second;
            A->srcs[l].push_back(s);
        }
        cudaFree(A->d_dests[l]);
        cudaFree(A->d_srcs[l]);
        cudaFree(A->d_tcoup[l]);
        A->d_dests[l] = nullptr;
        A->d_srcs[l] = nullptr;
        A->d_tcoup[l] = nullptr;
        A_CUDA(h, cudaMalloc(&A->d_dests[l], sizeof(smg::AdjDest) * std::max<size_t>(1, A->dests[l].size())));
        A_CUDA(h, cudaMalloc(&A->d_srcs[l], sizeof(smg::AdjSrc) * std::max<size_t>(1, A->srcs[l].size())));
        A_CUDA(h, cudaMalloc(&A->d_tcoup[l], sizeof(smg::TCoup) * std::max<size_t>(1, A->tcoup[l].size())));
        if (!A->dests[l].empty())
            A_CUDA(h, cudaMemcpyAsync(A->d_dests[l], A->dests[l].data(), sizeof(smg::AdjDest) * A->dests[l].size(),
                                      cudaMemcpyHostToDevice, h->stream));
        if (!A->srcs[l].empty())
            A_CUDA(h, cudaMemcpyAsync(A->d_srcs[l], A->srcs[l].data(), sizeof(smg::AdjSrc) * A->srcs[l].size(),
                                      cudaMemcpyHostToDevice, h->stream));
        if (!A->tcoup[l].empty())
            A_CUDA(h, cudaMemcpyAsync(A->d_tcoup[l], A->tcoup[l].data(), sizeof(smg::TCoup) * A->tcoup[l].size(),
                                      cudaMemcpyHostToDevice, h->stream));
    }
    A_CUDA(h, cudaStreamSynchronize(h->stream));
    return SMG_OK;
}

void grid_ext(const smg_handle* h, int f, int e[3]) {
    const int gt = h->field_grid[f];
    for (int a = 0; a < 3; ++a) {
        const int d = h->sd[a];
        const int g = 1 + ((gt >> d) & 1);
        e[a] = (g == 2 && h->g.bc[a] == 1) ? h->g.n[a] + 1 : h->g.n[a];
    }
}

}  // namespace

namespace {

// Two kernels per phase: k_adj_point over the destinations, then
// k_adj_transpose2 over the sources.  Segments are walked last to first,
// each recomputed from its checkpoint (the last one is still recorded from
// smg_forward).
cudaError_t backward_split(smg_handle* h, int64_t* launches) {
    AdjData* A = h->adj;
    const size_t sb = state_bytes(h);
    const size_t vb = (size_t)h->g.cs * std::max(A->maxdest, 1) * sizeof(double);
    const long long npts = h->g.s2 * h->g.B[2];
    const unsigned nbx = (unsigned)((npts + 255) / 256);
    const int tpr = (h->g.B[0] + 1) / 2;
    const unsigned nbp = (unsigned)(((long long)tpr * h->g.B[1] * h->g.B[2] + 127) / 128);
    const size_t nA = A->dests[0].size() / 3;
    for (int64_t s = A->nseg - 1; s >= 0; --s) {
        const int64_t ks = std::min<int64_t>(A->K, A->nsteps - s * A->K);
        if (!(s == A->nseg - 1 && A->tail_valid)) {
            cudaError_t e = cudaMemcpyAsync(A->work, A->ckpt[s], sb, cudaMemcpyDeviceToDevice, h->stream);
            if (e != cudaSuccess) return e;
            e = record_segment(h, ks, A->work, A->rec_w, A->rec_state, h->stream, s == A->nseg - 1);
            if (e != cudaSuccess) return e;
            *launches += 2 * ks + 1;
        }
        for (int64_t r = 2 * ks; r >= 0; --r) {
            const int kind = r == 0 ? 0 : (r & 1 ? 1 : (r < 2 * ks ? 2 : 3));
            const int l = kind == 1 ? 1 : 0;
            const double* pre = (const double*)((const char*)A->rec_state + vb * r);
            const double* W = (const double*)((const char*)A->rec_w + vb * r);
            if (l == 1 && !A->dests[1].empty()) {
                const dim3 g1(nbx, (unsigned)A->dests[1].size());
                smg::k_adj_point<1><<<g1, 256, 0, h->stream>>>(h->g, A->d_dests[1], pre, W, A->lam, A->V, h->hdt);
                ++*launches;
            } else if (l == 0 && nA) {
                const dim3 g1(nbx, (unsigned)nA);
                if (kind == 0)
                    smg::k_adj_point<0><<<g1, 256, 0, h->stream>>>(h->g, A->d_dests[0], pre, W, A->lam, A->V, h->hdt);
                else if (kind == 3)
                    smg::k_adj_point<0><<<g1, 256, 0, h->stream>>>(h->g, A->d_dests[0] + nA, pre, W, A->lam, A->V,
                                                                   h->hdt);
                else
                    smg::k_adj_point<1><<<g1, 256, 0, h->stream>>>(h->g, A->d_dests[0] + 2 * nA, pre, W, A->lam, A->V,
                                                                   h->hdt);
                ++*launches;
            }
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return e;
            if (!A->srcs[l].empty()) {
                const dim3 g2(nbp, (unsigned)A->srcs[l].size());
                smg::k_adj_transpose2<<<g2, 128, 0, h->stream>>>(h->g, A->d_srcs[l], A->d_tcoup[l], A->V, A->lam);
                ++*launches;
                e = cudaGetLastError();
                if (e != cudaSuccess) return e;
            }
        }
    }
    return cudaSuccess;
}

// One k_adj_fused launch per phase.  The backward sees the phases of one
// smg_run over all steps: A(k=1), (B, A(k=2)A(k=1))*, B, A(k=2); the A(k=2)
// ending a segment and the A(k=1) starting the next one form one fused A-A
// phase (same sources, same W; its values before are those recorded before
// the segment's A(k=2)), so destinations and sources alternate strictly.
// Phase kinds: 0 A(k=1), 1 B, 2 fused A-A, 3 A(k=2).
cudaError_t backward_fused(smg_handle* h, int64_t* launches) {
    AdjData* A = h->adj;
    const size_t sb = state_bytes(h);
    const size_t vb = (size_t)h->g.cs * std::max(A->maxdest, 1) * sizeof(double);
    const int tpr = (h->g.B[0] + 1) / 2;
    const unsigned nbp = (unsigned)(((long long)tpr * h->g.B[1] * h->g.B[2] + 127) / 128);
    const size_t nA = A->dests[0].size() / 3;
    auto table = [&](int kind) -> const smg::AdjDest* {
        if (kind < 0) return nullptr;
        if (kind == 1) return A->d_dests[1];
        return A->d_dests[0] + (kind == 0 ? 0 : (kind == 3 ? nA : 2 * nA));
    };
    auto substeps = [](int kind) { return kind < 0 ? 0 : (kind == 1 || kind == 2 ? 2 : 1); };
    // the sweep's stream: the handle's, or one of the highest priority joined to it
    cudaStream_t ss = A->sstream ? A->sstream : h->stream;
    if (A->sstream) {
        cudaError_t r = cudaEventRecord(A->ev_in, h->stream);
        if (r == cudaSuccess) r = cudaStreamWaitEvent(ss, A->ev_in, 0);
        if (r != cudaSuccess) return r;
    }
    // targets l: 0 = sources of an A phase (B destinations), 1 = sources of a B phase
    auto launch = [&](int l, int coup, int pkind, const double* pre, const double* W, int nkind) -> cudaError_t {
        if (A->srcs[l].empty()) return cudaSuccess;
        if (A->ds) {
            // kind -> (substeps, filters in k=2, k=1 order)
            auto swap = [](int kind) { return kind == 2 || kind == 3 ? 1 : 0; };
            *launches += smg::jit_adj_launches(h, l);
            return smg::launch_jit_adj(h, l, coup, substeps(pkind), swap(pkind), substeps(nkind), swap(nkind), A->lam,
                                       A->dDE, A->dG, pre, W, ss);
        }
        const dim3 grid(nbp, (unsigned)A->srcs[l].size());
        const int PM = substeps(pkind), NM = substeps(nkind);
        const smg::AdjDest* pt = table(pkind);
        const smg::AdjDest* nt = table(nkind);
#define SMG_FUSED(P, N)                                                                                 \
    if (PM == P && NM == N)                                                                             \
        smg::k_adj_fused<P, N><<<grid, 128, 0, ss>>>(h->g, A->d_srcs[l], A->d_tcoup[l], coup, pt, pre, W, \
                                                            nt, A->lam, h->hdt);
        SMG_FUSED(0, 0) SMG_FUSED(0, 1) SMG_FUSED(0, 2) SMG_FUSED(1, 0) SMG_FUSED(1, 1) SMG_FUSED(1, 2)
        SMG_FUSED(2, 0) SMG_FUSED(2, 1) SMG_FUSED(2, 2)
#undef SMG_FUSED
        ++*launches;
        return cudaGetLastError();
    };
    auto slot = [&](const double* base, int64_t r) {
        return base ? (const double*)((const char*)base + vb * r) : nullptr;
    };
    // recording buffer of segment s (the last segment uses the first, which
    // smg_forward filled); with one buffer everything runs on the handle's stream
    const bool dbl = A->rec_w2 != nullptr;
    auto buf = [&](int64_t s) { return dbl ? (int)((A->nseg - 1 - s) & 1) : 0; };
    double* RW[2] = {A->rec_w, A->rec_w2};
    double* RS[2] = {A->rec_state, A->rec_state2};
    double* WK[2] = {A->work, A->work2};
    cudaError_t e;
    auto recompute = [&](int64_t s) -> cudaError_t {
        const int b = buf(s);
        const int64_t ks = std::min<int64_t>(A->K, A->nsteps - s * A->K);
        cudaStream_t st = dbl ? A->rstream : ss;
        cudaError_t r;
        if (dbl && (r = cudaStreamWaitEvent(st, A->ev_free[b], 0)) != cudaSuccess) return r;
        if ((r = cudaMemcpyAsync(WK[b], A->ckpt[s], sb, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return r;
        if ((r = record_segment(h, ks, WK[b], RW[b], RS[b], st, s == A->nseg - 1)) != cudaSuccess) return r;
        *launches += 2 * ks + 1;
        if (dbl && (r = cudaEventRecord(A->ev_rec[b], st)) != cudaSuccess) return r;
        return cudaSuccess;
    };
    if (dbl) {
        // the recompute stream starts after the work already queued on the handle's stream
        if ((e = cudaEventRecord(A->ev_free[1], ss)) != cudaSuccess) return e;
        if ((e = cudaEventRecord(A->ev_free[0], ss)) != cudaSuccess) return e;
    }
    if (!A->tail_valid && (e = recompute(A->nseg - 1)) != cudaSuccess) return e;
    // the adjoint seed of the last phase's (A(k=2)) destinations, scaled
    e = launch(1, 0, -1, nullptr, nullptr, 3);
    if (e != cudaSuccess) return e;
    for (int64_t s = A->nseg - 1; s >= 0; --s) {
        const int64_t ks = std::min<int64_t>(A->K, A->nsteps - s * A->K);
        const bool last = s == A->nseg - 1;
        const int b = buf(s);
        if (s >= 1 && (e = recompute(s - 1)) != cudaSuccess) return e;   // overlaps this segment's sweep
        if (dbl && !(last && A->tail_valid) && (e = cudaStreamWaitEvent(ss, A->ev_rec[b], 0)) != cudaSuccess)
            return e;
        for (int64_t l = last ? 2 * ks : 2 * ks - 1; l >= 0; --l) {
            const int64_t p = l + 1;   // the phase after l (its pointwise part is pending)
            int pkind = -1;
            if (p <= 2 * ks) pkind = (p & 1) ? 1 : (p < 2 * ks ? 2 : (last ? 3 : 2));
            int nkind = -1;            // the phase before l (the targets' destination phase)
            if (l >= 1) nkind = ((l - 1) & 1) ? 1 : (l - 1 >= 2 ? 2 : (s == 0 ? 0 : 2));
            else if (s > 0) nkind = 1;
            e = launch((l & 1) ? 1 : 0, 1, pkind, pkind < 0 ? nullptr : slot(RS[b], p),
                       pkind < 0 ? nullptr : slot(RW[b], p), nkind);
            if (e != cudaSuccess) return e;
        }
        if (dbl && s >= 1 && (e = cudaEventRecord(A->ev_free[b], ss)) != cudaSuccess) return e;
    }
    // the first phase's (A(k=1)) pointwise part on its destinations
    if ((e = launch(1, 0, 0, slot(RS[buf(0)], 0), slot(RW[buf(0)], 0), -1)) != cudaSuccess) return e;
    if (A->sstream) {
        if ((e = cudaEventRecord(A->ev_out, ss)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(h->stream, A->ev_out, 0)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

void smg_adjoint_free(smg_handle* h) { free_adj(h); }

extern "C" {

int smg_forward(smg_handle* h, int64_t nsteps, int64_t ckpt_every) {
    SMG_TRY
    if (!h) return SMG_EINVAL;
    if (nsteps < 1 || ckpt_every < 0)
        return afail(h, SMG_EINVAL, "smg_forward: nsteps must be >= 1 and ckpt_every >= 0");
    if (!h->dt_set || !h->state_set) return afail(h, SMG_ESTATE, "smg_forward: set the state and dt first");
    if (h->filter_mode == SMG_FILTER_FULL)
        return afail(h, SMG_EINVAL, "smg_forward: the adjoint supports f_position '' and 'substep'");
    if (!(h->pair[0].ok && h->pair[1].ok)) return afail(h, SMG_EINVAL, "smg_forward: pair tables unavailable");
    if (!h->src_expr.empty() || h->mat.on || !h->filt.f1.empty())
        return afail(h, SMG_EINVAL,
                     "smg_forward: the adjoint covers autonomous problems (no device-evaluated sources or materials)");
    const size_t sb = state_bytes(h);
    const int maxdest = (int)std::max(h->destA.size(), h->destB.size());
    const size_t vb = (size_t)h->g.cs * std::max(maxdest, 1) * sizeof(double);
    int64_t K = std::min<int64_t>(ckpt_every, nsteps);
    if (ckpt_every == 0) {
        // the largest K (fewest recomputed steps) whose checkpoints and
        // recording fit in 70% of the free memory (the buffers this handle
        // already holds count as free)
        size_t fr = 0, tot = 0;
        A_CUDA(h, cudaMemGetInfo(&fr, &tot));
        const double held = h->adj ? (double)h->adj->bytes : 0.0;
        const double budget = 0.7 * ((double)fr + held) - 4.0 * (double)sb;
        K = 1;
        for (int64_t k = nsteps; k >= 1; --k) {
            const int64_t ns = (nsteps + k - 1) / k;
            const double rec = 2.0 * (double)vb * (2 * k + 1) * (ns > 1 ? 2 : 1) + (ns > 1 ? (double)sb : 0.0);
            if ((double)sb * (ns + 2) + rec <= budget) {
                K = k;
                break;
            }
        }
    }
    const int64_t nseg = (nsteps + K - 1) / K;
    AdjData* A = h->adj;
    if (!A || A->K != K || A->nseg != nseg) {
        // (re)allocate: checkpoints, work/adjoint/scratch states and the
        // recording of one segment (2K+1 phases); kept for later calls
        free_adj(h);
        A = new AdjData();
        h->adj = A;
        A->K = K;
        A->nseg = nseg;
        A->maxdest = maxdest;
        A->ckpt.assign(nseg, nullptr);
        for (auto& p : A->ckpt) A_CUDA(h, cudaMalloc(&p, sb));
        A_CUDA(h, cudaMalloc(&A->work, sb));
        A_CUDA(h, cudaMalloc(&A->lam, sb));
        A_CUDA(h, cudaMalloc(&A->V, vb));
        A_CUDA(h, cudaMalloc(&A->rec_w, vb * (2 * K + 1)));
        A_CUDA(h, cudaMemsetAsync(A->V, 0, vb, h->stream));
        A_CUDA(h, cudaMemsetAsync(A->rec_w, 0, vb * (2 * K + 1), h->stream));
        A->bytes = sb * (nseg + 2) + vb * (2 * K + 2);
        if (nseg > 1) {   // second recording: recompute overlapped with the sweep
            A_CUDA(h, cudaMalloc(&A->rec_w2, vb * (2 * K + 1)));
            A_CUDA(h, cudaMalloc(&A->work2, sb));
            int least = 0, greatest = 0;
            A_CUDA(h, cudaDeviceGetStreamPriorityRange(&least, &greatest));
            A_CUDA(h, cudaStreamCreateWithPriority(&A->rstream, cudaStreamNonBlocking,
                                                   h->adj_priority == 1 ? greatest : least));
            if (h->adj_priority == 2) {   // the sweep above the recompute
                A_CUDA(h, cudaStreamCreateWithPriority(&A->sstream, cudaStreamNonBlocking, greatest));
                A_CUDA(h, cudaEventCreateWithFlags(&A->ev_in, cudaEventDisableTiming));
                A_CUDA(h, cudaEventCreateWithFlags(&A->ev_out, cudaEventDisableTiming));
            }
            for (int b = 0; b < 2; ++b) {
                A_CUDA(h, cudaEventCreateWithFlags(&A->ev_rec[b], cudaEventDisableTiming));
                A_CUDA(h, cudaEventCreateWithFlags(&A->ev_free[b], cudaEventDisableTiming));
            }
            A->bytes += sb + vb * (2 * K + 1);
        }
    } else {
        for (double* p : A->gfield) cudaFree(p);
        for (double* p : A->dEslot) cudaFree(p);
        A->bytes = sb * (nseg + 2) + vb * (2 * K + 2) + (nseg > 1 ? sb + vb * (2 * K + 1) : 0) +
                   (A->rec_state ? vb * (2 * K + 1) * (nseg > 1 ? 2 : 1) : 0);
    }
    A->nsteps = nsteps;
    A->ready = false;
    A->tail_valid = false;
    // gradient slots for sigma and source fields; d(decay)/d(sigma) per sigma field
    const int nf = (int)h->field_grid.size();
    A->gfield.assign(nf, nullptr);
    A->dEslot.assign(nf, nullptr);
    A->dEscalar.assign(nf, 0.0);
    std::vector<char> is_sigma(nf, 0), is_q(nf, 0);
    for (int j = 1; j < h->n_sys; ++j) is_sigma[h->comps[j].sT] = 1;
    is_sigma[h->sigma_a] = 1;
    for (int j = 0; j < h->n_sys; ++j)
        if (h->comps[j].Q != h->field_zero) is_q[h->comps[j].Q] = 1;
    for (int f = 0; f < nf; ++f) {
        if (!(is_sigma[f] || is_q[f])) continue;
        A_CUDA(h, cudaMalloc(&A->gfield[f], (size_t)h->g.cs * sizeof(double)));
        A_CUDA(h, cudaMemsetAsync(A->gfield[f], 0, (size_t)h->g.cs * sizeof(double), h->stream));
        A->bytes += (size_t)h->g.cs * sizeof(double);
        if (!is_sigma[f]) continue;
        const smg::DevField& F = h->fields_host[f];
        if (F.p) {
            A_CUDA(h, cudaMalloc(&A->dEslot[f], (size_t)h->g.cs * sizeof(double)));
            A->bytes += (size_t)h->g.cs * sizeof(double);
            smg::k_dphi<<<(unsigned)((h->g.cs + 255) / 256), 256, 0, h->stream>>>(A->dEslot[f], F.p, h->g.cs, h->hdt);
            A_CUDA(h, cudaGetLastError());
        } else {
            A->dEscalar[f] = -h->hdt * smg::dphi(-F.s * h->hdt);
        }
    }
    int rc = build_tables(h);
    if (rc != SMG_OK) return rc;
    {   // per-field tables of the generated backward kernels
        const int nft = (int)h->fields_host.size();
        std::vector<smg::DevField> de(nft, smg::DevField{nullptr, 0.0});
        std::vector<double*> gt(nft, nullptr);
        for (int f = 0; f < nf; ++f) {
            de[f] = smg::DevField{A->dEslot[f], A->dEscalar[f]};
            gt[f] = A->gfield[f];
        }
        cudaFree(A->dDE);
        cudaFree(A->dG);
        A->dDE = nullptr;
        A->dG = nullptr;
        A_CUDA(h, cudaMalloc(&A->dDE, sizeof(smg::DevField) * nft));
        A_CUDA(h, cudaMalloc(&A->dG, sizeof(double*) * nft));
        A_CUDA(h, cudaMemcpyAsync(A->dDE, de.data(), sizeof(smg::DevField) * nft, cudaMemcpyHostToDevice, h->stream));
        A_CUDA(h, cudaMemcpyAsync(A->dG, gt.data(), sizeof(double*) * nft, cudaMemcpyHostToDevice, h->stream));
        A_CUDA(h, cudaStreamSynchronize(h->stream));
    }
    // recording and backward kernels: the generated ones where the handle runs
    // the generated kernels (AUTO or JIT), else the precompiled ones
    if ((h->variant == SMG_VARIANT_AUTO || h->variant == SMG_VARIANT_JIT) && !h->jit_failed) {
        std::string why;
        if (smg::jit_build_rec(h, why) != SMG_OK || smg::jit_build_adj(h, why) != SMG_OK) {
            h->jit_failed = true;
            h->jit_err = why;
        }
    }
    // the generated recording and fused sweep keep one value per destination
    // and phase; the precompiled kernels (and the split sweep) need the values
    // before each phase as well
    A->ds = (h->variant == SMG_VARIANT_AUTO || h->variant == SMG_VARIANT_JIT) && !h->jit_failed && h->jit_rec &&
            h->jit_adj && h->adj_fused && !h->jit_calls;
    if (!A->ds && !A->rec_state) {
        A_CUDA(h, cudaMalloc(&A->rec_state, vb * (2 * A->K + 1)));
        A_CUDA(h, cudaMemsetAsync(A->rec_state, 0, vb * (2 * A->K + 1), h->stream));
        A->bytes += vb * (2 * A->K + 1);
        if (A->nseg > 1) {
            A_CUDA(h, cudaMalloc(&A->rec_state2, vb * (2 * A->K + 1)));
            A_CUDA(h, cudaMemsetAsync(A->rec_state2, 0, vb * (2 * A->K + 1), h->stream));
            A->bytes += vb * (2 * A->K + 1);
        }
    }
    for (int l = 0; l < 2; ++l)
        for (const auto& sr : A->srcs[l])
            if (sr.pslot < 0) return afail(h, SMG_EINVAL, "smg_forward: a component is no phase's destination");
    // forward: checkpoint at the start of every segment; every segment but the
    // last as smg_run, the last one recorded for the backward sweep
    A_CUDA(h, cudaEventRecord(h->ev0, h->stream));
    h->last_launches = 0;
    for (int64_t s = 0; s < A->nseg; ++s) {
        A_CUDA(h, cudaMemcpyAsync(A->ckpt[s], h->dU, sb, cudaMemcpyDeviceToDevice, h->stream));
        const int64_t ks = std::min<int64_t>(A->K, nsteps - s * A->K);
        if (s + 1 < A->nseg) {
            rc = smg::run_steps(h, ks, false);
            if (rc != SMG_OK) return rc;
        } else {
            A_CUDA(h, record_segment(h, ks, h->dU, A->rec_w, A->rec_state, h->stream, true));
            h->last_launches += 2 * ks + 1;
        }
    }
    A_CUDA(h, cudaEventRecord(h->ev1, h->stream));
    A_CUDA(h, cudaStreamSynchronize(h->stream));
    A->ready = true;
    A->seeded = false;
    A->tail_valid = true;
    return SMG_OK;
    SMG_CATCH(h ? &h->err : nullptr)
}

int smg_misfit(smg_handle* h, const double* obs, double* J) {
    SMG_TRY
    if (!h || !obs) return SMG_EINVAL;
    AdjData* A = h->adj;
    if (!A || !A->ready) return afail(h, SMG_ESTATE, "smg_misfit: call smg_forward first");
    const int* e = h->comps[0].ext;
    const size_t n = (size_t)e[0] * e[1] * e[2];
    std::vector<double> u(n), lam0(n);
    std::vector<double*> all(h->n_sys, nullptr);
    all[0] = u.data();
    int rc = smg_get_state(h, all.data());
    if (rc != SMG_OK) return rc;
    double sum = 0.0;
    for (size_t i = 0; i < n; ++i) {
        lam0[i] = u[i] - obs[i];
        sum += lam0[i] * lam0[i];
    }
    if (J) *J = 0.5 * sum;
    const size_t sb = state_bytes(h);
    A_CUDA(h, cudaMemsetAsync(A->lam, 0, sb, h->stream));
    cudaMemcpy3DParms p{};
    p.srcPtr = make_cudaPitchedPtr(lam0.data(), (size_t)e[0] * 8, (size_t)e[0], (size_t)e[1]);
    p.dstPtr = make_cudaPitchedPtr(A->lam, (size_t)h->g.s1 * 8, (size_t)h->g.s1, (size_t)h->g.B[1]);
    p.extent = make_cudaExtent((size_t)e[0] * 8, (size_t)e[1], (size_t)e[2]);
    p.kind = cudaMemcpyHostToDevice;
    A_CUDA(h, cudaMemcpy3DAsync(&p, h->stream));
    A_CUDA(h, cudaStreamSynchronize(h->stream));
    A->seeded = true;
    return SMG_OK;
    SMG_CATCH(h ? &h->err : nullptr)
}

int smg_adjoint_seed(smg_handle* h, const double* const* lam) {
    SMG_TRY
    if (!h || !lam) return SMG_EINVAL;
    AdjData* A = h->adj;
    if (!A || !A->ready) return afail(h, SMG_ESTATE, "smg_adjoint_seed: call smg_forward first");
    A_CUDA(h, cudaMemsetAsync(A->lam, 0, state_bytes(h), h->stream));
    for (int j = 0; j < h->n_sys; ++j) {
        if (!lam[j]) continue;
        const int* e = h->comps[j].ext;
        cudaMemcpy3DParms p{};
        p.srcPtr = make_cudaPitchedPtr((void*)lam[j], (size_t)e[0] * 8, (size_t)e[0], (size_t)e[1]);
        p.dstPtr = make_cudaPitchedPtr(A->lam + (size_t)j * h->g.cs, (size_t)h->g.s1 * 8, (size_t)h->g.s1,
                                       (size_t)h->g.B[1]);
        p.extent = make_cudaExtent((size_t)e[0] * 8, (size_t)e[1], (size_t)e[2]);
        p.kind = cudaMemcpyHostToDevice;
        A_CUDA(h, cudaMemcpy3DAsync(&p, h->stream));
    }
    A_CUDA(h, cudaStreamSynchronize(h->stream));
    A->seeded = true;
    return SMG_OK;
    SMG_CATCH(h ? &h->err : nullptr)
}

int smg_backward(smg_handle* h, double* const* grad_U0, double* const* grad_fields) {
    SMG_TRY
    if (!h) return SMG_EINVAL;
    AdjData* A = h->adj;
    if (!A || !A->ready) return afail(h, SMG_ESTATE, "smg_backward: call smg_forward first");
    if (!A->seeded) return afail(h, SMG_ESTATE, "smg_backward: seed the adjoint (smg_misfit or smg_adjoint_seed)");
    for (double* g : A->gfield)
        if (g) A_CUDA(h, cudaMemsetAsync(g, 0, (size_t)h->g.cs * sizeof(double), h->stream));
    A_CUDA(h, cudaEventRecord(h->ev0, h->stream));
    int64_t launches = 0;
    // a forward recorded for the generated fused sweep is swept by it
    const cudaError_t e = (A->ds || h->adj_fused) ? backward_fused(h, &launches) : backward_split(h, &launches);
    if (e != cudaSuccess) return acuda(h, e, "smg_backward");
    A_CUDA(h, cudaEventRecord(h->ev1, h->stream));
    h->last_launches = launches;
    A->seeded = false;               // lambda now holds dJ/dU(0)
    A->tail_valid = A->nseg == 1;    // the recording now holds segment 0
    A_CUDA(h, cudaStreamSynchronize(h->stream));
    if (grad_U0) {
        for (int j = 0; j < h->n_sys; ++j) {
            if (!grad_U0[j]) continue;
            const int* e = h->comps[j].ext;
            cudaMemcpy3DParms p{};
            p.srcPtr = make_cudaPitchedPtr(A->lam + (size_t)j * h->g.cs, (size_t)h->g.s1 * 8, (size_t)h->g.s1,
                                           (size_t)h->g.B[1]);
            p.dstPtr = make_cudaPitchedPtr(grad_U0[j], (size_t)e[0] * 8, (size_t)e[0], (size_t)e[1]);
            p.extent = make_cudaExtent((size_t)e[0] * 8, (size_t)e[1], (size_t)e[2]);
            p.kind = cudaMemcpyDeviceToHost;
            A_CUDA(h, cudaMemcpy3DAsync(&p, h->stream));
        }
    }
    if (grad_fields) {
        const int nf = h->field_one;   // user fields only
        std::vector<double> tmp((size_t)h->g.cs);
        for (int f = 0; f < nf; ++f) {
            if (!grad_fields[f]) continue;
            if (!A->gfield[f]) {
                int e[3];
                grid_ext(h, f, e);
                const size_t n = h->fields_host[f].p ? (size_t)e[0] * e[1] * e[2] : 1;
                std::fill(grad_fields[f], grad_fields[f] + n, 0.0);
                continue;
            }
            if (h->fields_host[f].p) {
                int e[3];
                grid_ext(h, f, e);
                cudaMemcpy3DParms p{};
                p.srcPtr = make_cudaPitchedPtr(A->gfield[f], (size_t)h->g.s1 * 8, (size_t)h->g.s1, (size_t)h->g.B[1]);
                p.dstPtr = make_cudaPitchedPtr(grad_fields[f], (size_t)e[0] * 8, (size_t)e[0], (size_t)e[1]);
                p.extent = make_cudaExtent((size_t)e[0] * 8, (size_t)e[1], (size_t)e[2]);
                p.kind = cudaMemcpyDeviceToHost;
                A_CUDA(h, cudaMemcpy3DAsync(&p, h->stream));
            } else {
                // scalar coefficient: the derivative is the sum over every point it acts on
                A_CUDA(h, cudaMemcpyAsync(tmp.data(), A->gfield[f], tmp.size() * sizeof(double),
                                          cudaMemcpyDeviceToHost, h->stream));
                A_CUDA(h, cudaStreamSynchronize(h->stream));
                double sum = 0.0;
                for (double v : tmp) sum += v;
                grad_fields[f][0] = sum;
            }
        }
    }
    A_CUDA(h, cudaStreamSynchronize(h->stream));
    return SMG_OK;
    SMG_CATCH(h ? &h->err : nullptr)
}

int smg_adjoint_bytes(const smg_handle* h, int64_t* bytes) {
    SMG_TRY
    if (!h || !bytes) return SMG_EINVAL;
    *bytes = h->adj ? (int64_t)h->adj->bytes : 0;
    return SMG_OK;
    SMG_CATCH(h ? &const_cast<smg_handle*>(h)->err : nullptr)
}

int smg_adjoint_info(const smg_handle* h, int64_t* K, int64_t* nseg) {
    SMG_TRY
    if (!h) return SMG_EINVAL;
    if (K) *K = h->adj ? h->adj->K : 0;
    if (nseg) *nseg = h->adj ? h->adj->nseg : 0;
    return SMG_OK;
    SMG_CATCH(h ? &const_cast<smg_handle*>(h)->err : nullptr)
}

}  // extern "C"
