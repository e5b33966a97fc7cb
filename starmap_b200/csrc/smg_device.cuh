// smg_device.cuh -- device-side data structures and arithmetic of the
// staggered-grid moment update (StaRMAP starmap_solver.m:307-421).
//
// Layout in HBM: every component (and every coefficient field) occupies one
// slot of `cs` doubles, a padded box of B[0] x B[1] x B[2] points with row
// pitch s1 (>= B[0], a multiple of 8 doubles) and plane pitch s2 = s1*B[1].
// Kernel axis 0 is the first non-singleton solver dimension, so the padded box
// keeps MATLAB's column-major order of each component.  A component on a grid
// with a smaller extent simply leaves the last row/plane of its slot unused.
//
// Arithmetic: the update is written with explicit round-to-nearest intrinsics
// (no FMA contraction) in the order MATLAB/Octave evaluates the reference's
// array expressions, so that with identical decay/filter factors the GPU
// reproduces the CPU restatement bit for bit.
#pragma once
#include <cstdint>

namespace smg {

constexpr int kMaxDims = 3;

struct DevGrid {
    int n[3];          // cells per kernel axis
    int bc[3];         // boundary condition per kernel axis
    int B[3];          // box extents per kernel axis
    long long s1;      // row pitch (elements)
    long long s2;      // plane pitch (elements)
    long long cs;      // component slot stride (elements)
    double h[3];       // grid spacing per kernel axis
};

struct DevField {      // coefficient: array slot (p != nullptr) or scalar s
    const double* p;
    double s;
};

struct DevComp {
    int ext[3];        // extents of this component's grid per kernel axis
    int cbeg, cend;    // range in the coupling table
    int sT, ET, Q, F1, F2;   // field indices
    int order;         // moment order (ordering helper; not used by arithmetic)
};

// One term of W_j = -sum_i M_d(j,i) * d_d U_i, in sumcell order.
// code = axis*2 + (source grid type along that axis == 2 ? 1 : 0)
struct DevCoup {
    int src;
    int code;
    double w;
};

struct DevArgs {
    DevGrid g;
    double* U;                 // state, n_sys slots
    const DevComp* comps;
    const DevCoup* coups;
    const DevField* fields;
    const int* dest;           // component list updated by this phase
    int ndest;
    int group;                 // destinations per CTA
    int sA, EA;                // fields of component 0 in phase B
    double hdt;                // dt/2
    int filter_substep;        // 1 if f_position == 'substep'
};

// ---------------------------------------------------------------------------
// Strip kernels: a CTA owns 32 consecutive points of one grid row and sweeps a
// host-built schedule of stages.  A stage first computes derivative slots
// (one staggered difference of one source component along one axis for the
// 32 points) into shared memory, then updates destination components whose
// coupling terms read those slots.  A slot is computed once per phase and
// freed after its last use; the host assigns ring positions.
// ---------------------------------------------------------------------------
struct SlotJob {
    int src;           // source component
    int code;          // axis*2 + (source grid type along axis == 2)
    int slot;          // shared-memory slot
    int ext[3];        // extents of the difference's output grid
};

// Coefficients of a destination are resolved on the host: each of sigma_t,
// decay, source, filter k=1, filter k=2 is either a row of the CTA's
// shared-memory field cache (row >= 0) or the scalar sc[].
enum { kCoefS = 0, kCoefE = 1, kCoefQ = 2, kCoefF1 = 3, kCoefF2 = 4, kNumCoef = 5 };

struct DestJob {
    int comp;
    int cbeg, cend;    // range in the SCoup table (sumcell order)
    int ext[3];        // extents of the destination's grid
    int row[kNumCoef];
    int pad;
    double sc[kNumCoef];
};

struct SCoup {
    int slot;
    int pad;
    double w;
};

struct Stage {
    int jbeg, jend;    // slot jobs
    int dbeg, dend;    // destinations
};

struct StripSched {
    const Stage* stages;
    const SlotJob* jobs;
    const DestJob* dests;
    const SCoup* coups;
    const int* frows;  // field index of each cached row
    int nstages;
    int nslots;
    int jcap;          // staging rows (slot jobs) of the largest stage
    int nfrows;        // cached coefficient rows
};

struct StripArgs {
    DevGrid g;
    double* U;
    const DevComp* comps;
    const DevField* fields;
    StripSched s;
    int sA, EA;
    double hdt;
    double rh[3];      // RN(1/h) per axis
    int exact_recip[3];  // 1 if the reciprocal correction is exact for this axis
    int filter_substep;
};

// Pair kernel tables: destinations with resolved coefficients (array pointer
// or scalar) and couplings with the source's slot offset.
constexpr int kPairRuns = 6;   // coupling runs per destination (x/y/z lists, split by source grid)

struct PairDest {
    int off;           // component slot offset (elements)
    int ext[3];
    int run[kPairRuns + 1];   // runs [run[r], run[r+1]) of equal source code, in sumcell order
    int code[kPairRuns];      // source grid code of each run: axis*2 + (grid type == 2)
    const double* fp[kNumCoef];   // array coefficient, or nullptr -> sc
    double sc[kNumCoef];
};

struct PairArgs {
    DevGrid g;
    double* U;
    const PairDest* dests;
    const int* coff;           // source slot offset (elements) per coupling
    const double* cw;          // M_d(j,i) per coupling
    int ndest, group, ngroups, nchunks;
    double hdt;
    double rh[3];
    int exact_recip[3];
    int filter_substep;
    double* wrec;      // adjoint recording: W of destination di stored at wrec + di*cs (or nullptr)
    double* prec;      // adjoint recording: destination values before the phase, same slots
};

// (a - b) / h correctly rounded, from the precomputed reciprocal y = RN(1/h)
// (P. Markstein, IBM J. Res. Dev. 34(1), 1990; Muller et al., Handbook of
// Floating-Point Arithmetic, "Markstein's theorem": if y is within half an
// ulp of 1/h and q within one ulp of d/h, then r = d - q*h is exact in one FMA
// and RN(q + r*y) is the correctly rounded quotient).  exact_recip, set per
// axis on the host:
//   2: |y*h - 1| < 2^-54, so q = RN(d*y) is already within one ulp: one
//      correction step (3 FP64 operations);
//   1: h and y normal: a first correction brings q within one ulp (its error
//      is ~|y*h-1| times the first error plus one rounding), the second is
//      the Markstein step (5 operations);
//   0: IEEE division.
__device__ __forceinline__ double recip_div(double d, double h, double y, int mode) {
    double q = __dmul_rn(d, y);
    if (mode == 1) {
        const double r0 = __fma_rn(-q, h, d);
        q = __fma_rn(r0, y, q);
    }
    const double r = __fma_rn(-q, h, d);
    return __fma_rn(r, y, q);
}

__device__ __forceinline__ double sdiv(double d, double h, double rh, int exact_recip) {
    if (exact_recip) return recip_div(d, h, rh, exact_recip);
    return __ddiv_rn(d, h);
}

// Division with the mode fixed at compile time for every axis of a launch
// (DIV = the smallest per-axis mode; the two-step form is exact wherever the
// one-step form is).  DIV 0 keeps the per-axis choice at run time.
template <int DIV>
__device__ __forceinline__ double tdiv(double d, double h, double rh, int exact_recip) {
    if (DIV == 2) {
        const double q = __dmul_rn(d, rh);
        const double r = __fma_rn(-q, h, d);
        return __fma_rn(r, rh, q);
    }
    if (DIV == 1) {
        double q = __dmul_rn(d, rh);
        const double r0 = __fma_rn(-q, h, d);
        q = __fma_rn(r0, rh, q);
        const double r = __fma_rn(-q, h, d);
        return __fma_rn(r, rh, q);
    }
    return sdiv(d, h, rh, exact_recip);
}

__device__ __forceinline__ double fld(const DevField* f, int i, long long pt) {
    const DevField F = f[i];
    return F.p ? __ldg(F.p + pt) : F.s;
}

// U + (dt/2)*(W + Q - s.*U).*E  with MATLAB's evaluation order
// (starmap_solver.m:352-354, 402, 404-406).
__device__ __forceinline__ double upd(double u, double W, double q, double s, double E, double hdt) {
    const double t1 = __dadd_rn(W, q);
    const double t2 = __dmul_rn(s, u);
    const double t3 = __dsub_rn(t1, t2);
    const double t4 = __dmul_rn(hdt, t3);
    const double t5 = __dmul_rn(t4, E);
    return __dadd_rn(u, t5);
}

// Neighbour indices of the staggered difference along one axis, expressed as
// the reference's diff over the extension vectors (starmap_solver.m:127-132):
//   source on centres (g = 1) -> value on staggered points
//     bc 0: U[(p+1) mod n] - U[p]           bc 1: U[min(p,n-1)] - U[max(p-1,0)]
//   source on staggered points (g = 2) -> value on centres
//     bc 0: U[p] - U[(p-1) mod n]           bc 1: U[p+1] - U[p]
__device__ __forceinline__ void stencil(int p, int n, int bc, int g2, int& hi, int& lo) {
    if (!g2) {
        if (bc) { hi = p < n - 1 ? p : n - 1; lo = p > 0 ? p - 1 : 0; }
        else    { hi = (p + 1 == n) ? 0 : p + 1; lo = p; }
    } else {
        if (bc) { hi = p + 1; lo = p; }
        else    { hi = p; lo = (p == 0) ? n - 1 : p - 1; }
    }
}

}  // namespace smg
