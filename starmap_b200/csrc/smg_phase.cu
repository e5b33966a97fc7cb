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

#include <algorithm>

#include "smg_internal.h"
#include "smg_pair.cuh"

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
//
// Shared memory: [nslots][32] derivative slots, (STAGED only) [jcap][2][32]
// staged raw values of the next stage's slot jobs, [nfrows][32] coefficient
// rows of this strip (loaded once; coefficients are constant in a launch).
// Per stage s:
//   (STAGED) wait for the asynchronous copies of stage s;  barrier
//   load this warp's destination values of stage s into registers
//   slot jobs of stage s -> (hi-lo)/h -> shared slot: from the staged copies
//     (STAGED), or from global loads issued kJobBatch jobs at a time
//   barrier
//   (STAGED) issue cp.async (8 B per lane, zero-filled outside the
//     difference's extent) of stage s+1's raw values
//   destinations of stage s: fold the slots, exponential update, store
constexpr int kDestBatch = 4;   // destinations per warp whose loads are batched
constexpr int kJobBatch = 4;    // slot jobs per warp whose loads are batched
constexpr int kMaxUnrolledCoup = 8;

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Addresses of U_src[hi] and U_src[lo] for this lane's point (base of the
// component when the point lies outside the difference's extent).
__device__ __forceinline__ bool job_addr(const StripArgs& a, const SlotJob& jb, int x, int y, int z, long long pt,
                                         const double*& ph, const double*& pl) {
    const bool valid = x < jb.ext[0] && y < jb.ext[1] && z < jb.ext[2];
    const double* base = a.U + (long long)jb.src * a.g.cs;
    ph = base;
    pl = base;
    if (valid) {
        const int ax = jb.code >> 1;
        const int pc = ax == 0 ? x : (ax == 1 ? y : z);
        const long long stv = ax == 0 ? 1 : (ax == 1 ? a.g.s1 : a.g.s2);
        int hi, lo;
        stencil(pc, a.g.n[ax], a.g.bc[ax], jb.code & 1, hi, lo);
        ph = base + pt + (hi - pc) * stv;
        pl = base + pt + (lo - pc) * stv;
    }
    return valid;
}

__device__ __forceinline__ void stage_jobs(const StripArgs& a, int jbeg, int jend, double* stg, int warp,
                                           int lane, int x, int y, int z, long long pt) {
    for (int q = jbeg + warp; q < jend; q += kStripWarps) {
        const SlotJob jb = a.s.jobs[q];
        const double *ph, *pl;
        const bool valid = job_addr(a, jb, x, y, z, pt, ph, pl);
        double* d = stg + (q - jbeg) * 64;
        cp_async8(d + lane, ph, valid);
        cp_async8(d + 32 + lane, pl, valid);
    }
    cp_async_commit();
}

__device__ __forceinline__ double coef(const DestJob& dj, int k, const double* frow, int lane) {
    return dj.row[k] >= 0 ? frow[dj.row[k] * 32 + lane] : dj.sc[k];
}

template <int MODE, bool STAGED>
__global__ void __launch_bounds__(32 * kStripWarps, 3) k_phase_strip(StripArgs a, int kf) {
    extern __shared__ double smem[];
    const StripSched& S = a.s;
    double* sl = smem;                                       // derivative slots
    double* stg = smem + S.nslots * 32;                      // staged raw values
    double* frow = stg + (STAGED ? S.jcap * 64 : 0);         // coefficient rows
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
    if (STAGED && S.nstages > 0) {
        const Stage st0 = S.stages[0];
        stage_jobs(a, st0.jbeg, st0.jend, stg, warp, lane, x, y, z, pt);
    }
    for (int r = warp; r < S.nfrows; r += kStripWarps) {
        const DevField F = a.fields[S.frows[r]];
        frow[r * 32 + lane] = (x < a.g.B[0]) ? __ldg(F.p + pt) : 0.0;
    }
    for (int s = 0; s < S.nstages; ++s) {
        const Stage st = S.stages[s];
        if (STAGED) cp_async_wait_all();
        __syncthreads();
        // destination loads of this stage, issued before the slot-job math
        double uv[kDestBatch];
        const int nd = st.dend - st.dbeg;
#pragma unroll
        for (int k = 0; k < kDestBatch; ++k) {
            uv[k] = 0.0;
            const int q = warp + k * kStripWarps;
            if (q < nd) {
                const DestJob& dj = S.dests[st.dbeg + q];
                const int comp = dj.comp;
                if (x < dj.ext[0] && y < dj.ext[1] && z < dj.ext[2]) uv[k] = a.U[(long long)comp * a.g.cs + pt];
            }
        }
        if (STAGED) {
            for (int q = st.jbeg + warp; q < st.jend; q += kStripWarps) {
                const SlotJob jb = S.jobs[q];
                const double* d = stg + (q - st.jbeg) * 64;
                const int ax = jb.code >> 1;
                sl[jb.slot * 32 + lane] =
                    sdiv(__dsub_rn(d[lane], d[32 + lane]), a.g.h[ax], a.rh[ax], a.exact_recip[ax]);
            }
        } else {
            for (int q0 = st.jbeg + warp; q0 < st.jend; q0 += kJobBatch * kStripWarps) {
                double hv[kJobBatch], lv[kJobBatch];
                int slot[kJobBatch], axv[kJobBatch];
#pragma unroll
                for (int k = 0; k < kJobBatch; ++k) {
                    const int q = q0 + k * kStripWarps;
                    hv[k] = lv[k] = 0.0;
                    slot[k] = -1;
                    axv[k] = 0;
                    if (q < st.jend) {
                        const SlotJob jb = S.jobs[q];
                        const double *ph, *pl;
                        if (job_addr(a, jb, x, y, z, pt, ph, pl)) {
                            hv[k] = __ldg(ph);
                            lv[k] = __ldg(pl);
                        }
                        slot[k] = jb.slot;
                        axv[k] = jb.code >> 1;
                    }
                }
#pragma unroll
                for (int k = 0; k < kJobBatch; ++k) {
                    if (slot[k] < 0) continue;
                    const int ax = axv[k];
                    sl[slot[k] * 32 + lane] = sdiv(__dsub_rn(hv[k], lv[k]), a.g.h[ax], a.rh[ax], a.exact_recip[ax]);
                }
            }
        }
        __syncthreads();
        if (STAGED && s + 1 < S.nstages) {
            const Stage sn = S.stages[s + 1];
            stage_jobs(a, sn.jbeg, sn.jend, stg, warp, lane, x, y, z, pt);
        }
        for (int k = 0; k * kStripWarps + warp < nd; ++k) {
            const DestJob dj = S.dests[st.dbeg + warp + k * kStripWarps];
            if (!(x < dj.ext[0] && y < dj.ext[1] && z < dj.ext[2])) continue;
            double* Uj = a.U + (long long)dj.comp * a.g.cs + pt;
            double u = 0.0;
#pragma unroll
            for (int kk = 0; kk < kDestBatch; ++kk)
                if (kk == k) u = uv[kk];
            if (k >= kDestBatch) u = *Uj;
            const double qv = coef(dj, kCoefQ, frow, lane);
            const double sv = coef(dj, kCoefS, frow, lane);
            const double E = coef(dj, kCoefE, frow, lane);
            double Ssum = 0.0;
            const int cb = dj.cbeg, nc = dj.cend - dj.cbeg;
            if (nc <= kMaxUnrolledCoup) {
                // all coupling descriptors and slot values are loaded before the fold
                double tv[kMaxUnrolledCoup], wv[kMaxUnrolledCoup];
#pragma unroll
                for (int c = 0; c < kMaxUnrolledCoup; ++c) {
                    if (c < nc) {
                        const SCoup cp = S.coups[cb + c];
                        tv[c] = sl[cp.slot * 32 + lane];
                        wv[c] = cp.w;
                    }
                }
#pragma unroll
                for (int c = 0; c < kMaxUnrolledCoup; ++c) {
                    if (c < nc) {
                        const double term = __dmul_rn(tv[c], wv[c]);
                        Ssum = c == 0 ? term : __dadd_rn(Ssum, term);
                    }
                }
            } else {
                for (int c = 0; c < nc; ++c) {
                    const SCoup cp = S.coups[cb + c];
                    const double term = __dmul_rn(sl[cp.slot * 32 + lane], cp.w);
                    Ssum = c == 0 ? term : __dadd_rn(Ssum, term);
                }
            }
            const double W = -Ssum;
            if (MODE == 0) {
                u = upd(u, W, qv, sv, E, a.hdt);
                if (a.filter_substep) u = __dmul_rn(u, coef(dj, kf == 1 ? kCoefF1 : kCoefF2, frow, lane));
            } else if (MODE == 2) {
                u = upd(u, W, qv, sv, E, a.hdt);
                if (a.filter_substep) u = __dmul_rn(u, coef(dj, kCoefF2, frow, lane));
                u = upd(u, W, qv, sv, E, a.hdt);
                if (a.filter_substep) u = __dmul_rn(u, coef(dj, kCoefF1, frow, lane));
            } else {
                // phase B: component 0 carries sA/EA and unit filters (resolved on the host)
                u = upd(u, W, qv, sv, E, a.hdt);
                if (a.filter_substep) u = __dmul_rn(u, coef(dj, kCoefF1, frow, lane));
                u = upd(u, W, qv, sv, E, a.hdt);
                if (a.filter_substep) u = __dmul_rn(u, coef(dj, kCoefF2, frow, lane));
            }
            *Uj = u;
        }
    }
    if (STAGED) cp_async_wait_all();
}

template <int MODE, int DIV, int UNROLL, int MINB>
__global__ void __launch_bounds__(256, MINB) k_phase_pair(PairArgs a, int kf) {
    const int bid = blockIdx.x;
    const int grp = bid % a.ngroups;
    const int rest = bid / a.ngroups;
    pair_item<MODE, DIV, UNROLL>(a, kf, grp, rest % a.nchunks, rest / a.nchunks, threadIdx.x, blockDim.x);
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

int strip_smem_bytes(const smg_handle* h, int phase) {
    const auto& S = h->sched[phase];
    const int staging = h->strip_staged ? S.jcap * 64 : 0;
    return (S.nslots * 32 + staging + (int)S.frows.size() * 32) * 8;
}

// Opt the strip kernels into the dynamic shared memory the schedules need
// (called once at handle creation, outside any stream capture).
cudaError_t strip_init(const smg_handle* h) {
    const int smem = max(strip_smem_bytes(h, 0), strip_smem_bytes(h, 1));
    const int smem_st = max((h->sched[0].nslots * 32 + h->sched[0].jcap * 64 + (int)h->sched[0].frows.size() * 32) * 8,
                            (h->sched[1].nslots * 32 + h->sched[1].jcap * 64 + (int)h->sched[1].frows.size() * 32) * 8);
    const int big = max(smem, smem_st);
    cudaError_t e;
#define SMG_ATTR(M, ST)                                                                                       \
    if ((e = cudaFuncSetAttribute(k_phase_strip<M, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, big)) != \
        cudaSuccess)                                                                                          \
        return e;
    SMG_ATTR(0, false) SMG_ATTR(1, false) SMG_ATTR(2, false) SMG_ATTR(0, true) SMG_ATTR(1, true) SMG_ATTR(2, true)
#undef SMG_ATTR
    return cudaSuccess;
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
    const unsigned nb = (unsigned)blocks;
    if (h->strip_staged) {
        if (mode == 0) k_phase_strip<0, true><<<nb, block, smem, s>>>(a, kfilter);
        else if (mode == 1) k_phase_strip<1, true><<<nb, block, smem, s>>>(a, kfilter);
        else k_phase_strip<2, true><<<nb, block, smem, s>>>(a, kfilter);
    } else {
        if (mode == 0) k_phase_strip<0, false><<<nb, block, smem, s>>>(a, kfilter);
        else if (mode == 1) k_phase_strip<1, false><<<nb, block, smem, s>>>(a, kfilter);
        else k_phase_strip<2, false><<<nb, block, smem, s>>>(a, kfilter);
    }
    return cudaGetLastError();
}

cudaError_t launch_pair(const smg_handle* h, int mode, int kfilter, cudaStream_t s) {
    const int phase = mode == 1 ? 1 : 0;
    const auto& P = h->pair[phase];
    if (P.ndest == 0) return cudaSuccess;
    PairArgs a{};
    a.g = h->g;
    a.U = h->dU;
    a.dests = P.d_dests;
    a.coff = P.d_coff;
    a.cw = P.d_cw;
    a.ndest = P.ndest;
    a.group = h->pair_group;
    a.ngroups = (P.ndest + a.group - 1) / a.group;
    const int tpr = (h->g.B[0] + 1) / 2;   // threads per row
    const int bs = std::min(h->pair_block, (tpr + 31) / 32 * 32);
    a.nchunks = (tpr + bs - 1) / bs;
    a.hdt = h->hdt;
    for (int k = 0; k < 3; ++k) {
        a.rh[k] = h->rh[k];
        a.exact_recip[k] = h->exact_recip[k];
    }
    a.filter_substep = h->filter_mode == 1;
    const long long blocks = (long long)a.ngroups * a.nchunks * h->g.B[1] * h->g.B[2];
    const int div = std::min(h->exact_recip[0], std::min(h->exact_recip[1], h->exact_recip[2]));
    const unsigned nb = (unsigned)blocks;
    const int cfg = div | (h->pair_unroll >= 2 ? 4 : 0) | (h->pair_minb >= 4 ? 8 : 0);
#define SMG_PAIR(D, U, M)                                                                \
    case D | (U == 2 ? 4 : 0) | (M == 4 ? 8 : 0):                                        \
        if (mode == 0) k_phase_pair<0, D, U, M><<<nb, bs, 0, s>>>(a, kfilter);          \
        else if (mode == 1) k_phase_pair<1, D, U, M><<<nb, bs, 0, s>>>(a, kfilter);     \
        else k_phase_pair<2, D, U, M><<<nb, bs, 0, s>>>(a, kfilter);                    \
        break;
    switch (cfg) {
        SMG_PAIR(2, 1, 3) SMG_PAIR(2, 2, 3) SMG_PAIR(2, 1, 4) SMG_PAIR(2, 2, 4)
        SMG_PAIR(1, 1, 3) SMG_PAIR(1, 2, 3) SMG_PAIR(1, 1, 4) SMG_PAIR(1, 2, 4)
        SMG_PAIR(0, 1, 3) SMG_PAIR(0, 2, 3) SMG_PAIR(0, 1, 4) SMG_PAIR(0, 2, 4)
    }
#undef SMG_PAIR
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
