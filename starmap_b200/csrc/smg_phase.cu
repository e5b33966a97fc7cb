// smg_phase.cu -- the fused staggered half-step kernels.
//
// One launch = one phase of the Strang splitting (starmap_solver.m:310-416):
//   phase A (case 1): destinations are the outer set c211,c121,c112,c222,
//                     sources the inner set; one dt/2 update, substep filter k.
//   phase B (case 2): destinations are the inner set c111,c221,c212,c122,
//                     sources the outer set; two dt/2 updates with the same W,
//                     component 0 decays by absorption only and is not filtered.
// Each thread owns one point of the padded box and walks the destinations of
// its CTA's group; for each destination it folds the coupling terms in sumcell
// order (x-list, y-list, z-list, ascending source index), each term being the
// staggered difference (U_i[hi]-U_i[lo])/h times M_d(j,i), then applies the
// exponential update in registers and stores once.  Sources and destinations
// are disjoint sets, so the update is in place without a race.
#include <cuda_runtime.h>

#include "smg_internal.h"

namespace smg {

template <int PHASE>
__global__ void __launch_bounds__(256) k_phase_generic(DevArgs a, int kf) {
    const long long npts = a.g.s2 * a.g.B[2];
    const int ngroups = (a.ndest + a.group - 1) / a.group;
    const int grp = blockIdx.x % ngroups;
    const long long tile = blockIdx.x / ngroups;
    const long long pt = tile * blockDim.x + threadIdx.x;
    if (pt >= npts) return;
    const int x = (int)(pt % a.g.s1);
    const int y = (int)((pt / a.g.s1) % a.g.B[1]);
    const int z = (int)(pt / a.g.s2);
    if (x >= a.g.B[0]) return;

    const int d0 = grp * a.group;
    const int d1 = min(d0 + a.group, a.ndest);
    for (int di = d0; di < d1; ++di) {
        const int j = __ldg(a.dest + di);
        const DevComp cj = a.comps[j];
        if (x >= cj.ext[0] || y >= cj.ext[1] || z >= cj.ext[2]) continue;
        double S = 0.0;
        for (int q = cj.cbeg; q < cj.cend; ++q) {
            const DevCoup cp = a.coups[q];
            const int ax = cp.code >> 1;
            const int pc = ax == 0 ? x : (ax == 1 ? y : z);
            const long long st = ax == 0 ? 1 : (ax == 1 ? a.g.s1 : a.g.s2);
            int hi, lo;
            stencil(pc, a.g.n[ax], a.g.bc[ax], cp.code & 1, hi, lo);
            const double* Us = a.U + (long long)cp.src * a.g.cs + pt;
            const double du = __ddiv_rn(__dsub_rn(__ldg(Us + (hi - pc) * st),
                                                  __ldg(Us + (lo - pc) * st)),
                                        a.g.h[ax]);
            const double term = __dmul_rn(du, cp.w);
            S = (q == cj.cbeg) ? term : __dadd_rn(S, term);
        }
        const double W = -S;
        double* Uj = a.U + (long long)j * a.g.cs + pt;
        double u = *Uj;
        const double qv = fld(a.fields, cj.Q, pt);
        if (PHASE == 0) {
            u = upd(u, W, qv, fld(a.fields, cj.sT, pt), fld(a.fields, cj.ET, pt), a.hdt);
            if (a.filter_substep) u = __dmul_rn(u, fld(a.fields, kf == 1 ? cj.F1 : cj.F2, pt));
        } else if (j == 0) {
            const double s = fld(a.fields, a.sA, pt), E = fld(a.fields, a.EA, pt);
            u = upd(u, W, qv, s, E, a.hdt);
            u = upd(u, W, qv, s, E, a.hdt);
        } else {
            const double s = fld(a.fields, cj.sT, pt), E = fld(a.fields, cj.ET, pt);
            u = upd(u, W, qv, s, E, a.hdt);
            if (a.filter_substep) u = __dmul_rn(u, fld(a.fields, cj.F1, pt));
            u = upd(u, W, qv, s, E, a.hdt);
            if (a.filter_substep) u = __dmul_rn(u, fld(a.fields, cj.F2, pt));
        }
        *Uj = u;
    }
}

// Strip kernel (see smg_device.cuh).  MODE 0: phase A with substep filter kf;
// MODE 1: phase B; MODE 2: phase A of the end of one step fused with phase A
// of the start of the next (the inner set is unchanged in between, so the
// differences are the same and the update is applied twice: filter k=2 then
// k=1, exactly the sequence of two separate launches).
template <int MODE>
__global__ void __launch_bounds__(32 * kStripWarps) k_phase_strip(StripArgs a, int kf) {
    extern __shared__ double sl[];   // [nslots][32]
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nxs = (a.g.B[0] + 31) >> 5;
    const long long strip = blockIdx.x;
    const int xs = (int)(strip % nxs);
    const long long row = strip / nxs;
    const int y = (int)(row % a.g.B[1]);
    const int z = (int)(row / a.g.B[1]);
    const int x = xs * 32 + lane;
    const long long pt = (long long)z * a.g.s2 + (long long)y * a.g.s1 + x;
    const StripSched S = a.s;
    for (int s = 0; s < S.nstages; ++s) {
        const Stage st = S.stages[s];
        for (int q = st.jbeg + warp; q < st.jend; q += kStripWarps) {
            const SlotJob jb = S.jobs[q];
            double v = 0.0;
            if (x < jb.ext[0] && y < jb.ext[1] && z < jb.ext[2]) {
                const int ax = jb.code >> 1;
                const int pc = ax == 0 ? x : (ax == 1 ? y : z);
                const long long stv = ax == 0 ? 1 : (ax == 1 ? a.g.s1 : a.g.s2);
                int hi, lo;
                stencil(pc, a.g.n[ax], a.g.bc[ax], jb.code & 1, hi, lo);
                const double* Us = a.U + (long long)jb.src * a.g.cs + pt;
                const double d = __dsub_rn(__ldg(Us + (hi - pc) * stv), __ldg(Us + (lo - pc) * stv));
                v = sdiv(d, a.g.h[ax], a.rh[ax], a.exact_recip[ax]);
            }
            sl[jb.slot * 32 + lane] = v;
        }
        __syncthreads();
        for (int q = st.dbeg + warp; q < st.dend; q += kStripWarps) {
            const DestJob dj = S.dests[q];
            const int j = dj.comp;
            const DevComp cj = a.comps[j];
            if (!(x < cj.ext[0] && y < cj.ext[1] && z < cj.ext[2])) continue;
            double* Uj = a.U + (long long)j * a.g.cs + pt;
            double u = *Uj;
            const double qv = fld(a.fields, cj.Q, pt);
            double Ssum = 0.0;
            for (int c = dj.cbeg; c < dj.cend; ++c) {
                const SCoup cp = S.coups[c];
                const double term = __dmul_rn(sl[cp.slot * 32 + lane], cp.w);
                Ssum = (c == dj.cbeg) ? term : __dadd_rn(Ssum, term);
            }
            const double W = -Ssum;
            if (MODE == 0) {
                u = upd(u, W, qv, fld(a.fields, cj.sT, pt), fld(a.fields, cj.ET, pt), a.hdt);
                if (a.filter_substep) u = __dmul_rn(u, fld(a.fields, kf == 1 ? cj.F1 : cj.F2, pt));
            } else if (MODE == 2) {
                const double s = fld(a.fields, cj.sT, pt), E = fld(a.fields, cj.ET, pt);
                u = upd(u, W, qv, s, E, a.hdt);
                if (a.filter_substep) u = __dmul_rn(u, fld(a.fields, cj.F2, pt));
                u = upd(u, W, qv, s, E, a.hdt);
                if (a.filter_substep) u = __dmul_rn(u, fld(a.fields, cj.F1, pt));
            } else if (j == 0) {
                const double s = fld(a.fields, a.sA, pt), E = fld(a.fields, a.EA, pt);
                u = upd(u, W, qv, s, E, a.hdt);
                u = upd(u, W, qv, s, E, a.hdt);
            } else {
                const double s = fld(a.fields, cj.sT, pt), E = fld(a.fields, cj.ET, pt);
                u = upd(u, W, qv, s, E, a.hdt);
                if (a.filter_substep) u = __dmul_rn(u, fld(a.fields, cj.F1, pt));
                u = upd(u, W, qv, s, E, a.hdt);
                if (a.filter_substep) u = __dmul_rn(u, fld(a.fields, cj.F2, pt));
            }
            *Uj = u;
        }
        __syncthreads();
    }
}

// Full filter at the end of a step: U{j} .*= filterTerm for j = 2..n_sys
// (starmap_solver.m:417-421).
__global__ void __launch_bounds__(256) k_full_filter(DevArgs a, int n_sys) {
    const long long npts = a.g.s2 * a.g.B[2];
    const long long pt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    if (pt >= npts || j >= n_sys) return;
    const int x = (int)(pt % a.g.s1);
    const int y = (int)((pt / a.g.s1) % a.g.B[1]);
    const int z = (int)(pt / a.g.s2);
    const DevComp cj = a.comps[j];
    if (x >= cj.ext[0] || y >= cj.ext[1] || z >= cj.ext[2]) return;
    double* Uj = a.U + (long long)j * a.g.cs + pt;
    *Uj = __dmul_rn(*Uj, fld(a.fields, cj.F1, pt));
}

// expm1div(-sigma*dt/2) elementwise (starmap_solver.m:269-272, 531-535).
__global__ void k_decay(double* out, const double* sigma, long long n, double dt) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = __dmul_rn(__dmul_rn(-sigma[i], dt), 0.5);
    double y = __dadd_rn(__dadd_rn(1.0, __dmul_rn(x, 0.5)), __ddiv_rn(__dmul_rn(x, x), 6.0));
    if (fabs(x) > 2e-4) y = __ddiv_rn(__dsub_rn(exp(x), 1.0), x);
    out[i] = y;
}

__global__ void k_finite(const double* U, long long n, int* flag) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long stride = (long long)gridDim.x * blockDim.x;
    int bad = 0;
    for (; i < n; i += stride) bad |= !isfinite(U[i]);
    if (bad) atomicOr(flag, 1);
}

static DevArgs make_args(const smg_handle* h, int phase) {
    DevArgs a{};
    a.g = h->g;
    a.U = h->dU;
    a.comps = h->dComps;
    a.coups = h->dCoups;
    a.fields = h->dFieldTab;
    a.dest = h->dDest + (phase == 0 ? 0 : (int)h->destA.size());
    a.ndest = (int)(phase == 0 ? h->destA.size() : h->destB.size());
    a.group = 4;
    a.sA = h->sigma_a;
    a.EA = h->decay_a >= 0 ? h->decay_a : h->derived_decay_a;
    a.hdt = h->hdt;
    a.filter_substep = h->filter_mode == 1;
    return a;
}

cudaError_t launch_phase(const smg_handle* h, int phase, int kfilter, cudaStream_t s) {
    DevArgs a = make_args(h, phase);
    if (a.ndest == 0) return cudaSuccess;
    const long long npts = h->g.s2 * h->g.B[2];
    const long long tiles = (npts + 255) / 256;
    const long long ngroups = (a.ndest + a.group - 1) / a.group;
    const long long blocks = tiles * ngroups;
    if (phase == 0)
        k_phase_generic<0><<<(unsigned)blocks, 256, 0, s>>>(a, kfilter);
    else
        k_phase_generic<1><<<(unsigned)blocks, 256, 0, s>>>(a, kfilter);
    return cudaGetLastError();
}

int strip_smem_bytes(const smg_handle* h, int phase) { return h->sched[phase].nslots * 32 * 8; }

// Opt the strip kernels into the dynamic shared memory the schedules need
// (called once at handle creation, outside any stream capture).
cudaError_t strip_init(const smg_handle* h) {
    const int smem = max(strip_smem_bytes(h, 0), strip_smem_bytes(h, 1));
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_phase_strip<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_phase_strip<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_phase_strip<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

cudaError_t launch_strip(const smg_handle* h, int mode, int kfilter, cudaStream_t s) {
    const int phase = mode == 1 ? 1 : 0;
    const auto& hs = h->sched[phase];
    if (hs.view.nstages == 0) return cudaSuccess;
    StripArgs a{};
    a.g = h->g;
    a.U = h->dU;
    a.comps = h->dComps;
    a.fields = h->dFieldTab;
    a.s = hs.view;
    a.sA = h->sigma_a;
    a.EA = h->decay_a >= 0 ? h->decay_a : h->derived_decay_a;
    a.hdt = h->hdt;
    for (int k = 0; k < 3; ++k) {
        a.rh[k] = h->rh[k];
        a.exact_recip[k] = h->exact_recip[k];
    }
    a.filter_substep = h->filter_mode == 1;
    const long long blocks = (long long)h->nxs * h->g.B[1] * h->g.B[2];
    const int smem = strip_smem_bytes(h, phase);
    const dim3 block(32 * kStripWarps);
    switch (mode) {
        case 0:
            k_phase_strip<0><<<(unsigned)blocks, block, smem, s>>>(a, kfilter);
            break;
        case 1:
            k_phase_strip<1><<<(unsigned)blocks, block, smem, s>>>(a, kfilter);
            break;
        default:
            k_phase_strip<2><<<(unsigned)blocks, block, smem, s>>>(a, kfilter);
            break;
    }
    return cudaGetLastError();
}

cudaError_t launch_full_filter(const smg_handle* h, cudaStream_t s) {
    if (h->n_sys < 2) return cudaSuccess;
    DevArgs a = make_args(h, 0);
    const long long npts = h->g.s2 * h->g.B[2];
    dim3 grid((unsigned)((npts + 255) / 256), (unsigned)(h->n_sys - 1));
    k_full_filter<<<grid, 256, 0, s>>>(a, h->n_sys);
    return cudaGetLastError();
}

cudaError_t launch_decay(double* out, const double* sigma, long long n, double dt, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_decay<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, sigma, n, dt);
    return cudaGetLastError();
}

cudaError_t launch_finite(const smg_handle* h, int* flag, cudaStream_t s) {
    const long long n = h->g.cs * h->n_sys;
    k_finite<<<148 * 8, 256, 0, s>>>(h->dU, n, flag);
    return cudaGetLastError();
}


}  // namespace smg
