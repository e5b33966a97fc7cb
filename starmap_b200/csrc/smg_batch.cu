// smg_batch.cu -- many problems in one persistent launch.
//
// Each instance is an ordinary handle (smg_create): its state, coefficient
// fields and pair-kernel tables live in its own device buffers.  The batch
// adds a work list per phase -- one item per (instance, row, chunk of
// 2*block points, group of destinations) -- and a cooperative persistent
// kernel that walks the items of a phase, meets the other CTAs at a grid
// barrier and moves to the next phase.  One launch advances every instance by
// `steps_per_launch` Strang steps (phase A, then B and fused A-A pairs, then
// the last A: A B [AA B]... A), each instance with its own dt.  The host loop
// over launches is captured in a CUDA graph.
//
// The grid barrier is a bounded spin: a CTA that waits longer than the spin
// limit sets the error flag and returns, every CTA checks the flag after the
// barrier, and the host reports SMG_ETIMEOUT.  Nothing waits without limit.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/starmap_gpu.h"
#include "smg_internal.h"
#include "smg_pair.cuh"

namespace {

struct BatchItem {
    int inst;
    int grp;
    int chunk;
    int row;
};

struct BarrierState {
    unsigned count;
    unsigned gen;
    int err;        // 1: a barrier wait ran out of its spin limit
    int pad;
};

struct BatchArgs {
    const smg::PairArgs* args;   // [n_inst][2]: phase A tables, phase B tables
    const BatchItem* items[2];
    int nitems[2];
    int steps;                   // Strang steps in this launch
    BarrierState* bar;
    long long spin_limit;        // polls before a barrier wait gives up
    unsigned expected;           // CTAs that must arrive (gridDim.x in normal use)
};

__device__ bool grid_barrier(const BatchArgs& B, int* s_flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vgen = &B.bar->gen;
        const unsigned g = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(&B.bar->count, 1u);
        int ok = 1;
        if (arrived == B.expected - 1) {
            atomicExch(&B.bar->count, 0u);
            __threadfence();
            atomicAdd(&B.bar->gen, 1u);
        } else {
            long long it = 0;
            while (*vgen == g) {
                if (++it > B.spin_limit) {
                    atomicExch(&B.bar->err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        if (*(volatile int*)&B.bar->err) ok = 0;
        *s_flag = ok;
    }
    __syncthreads();
    return *s_flag != 0;
}

template <int MODE>
__device__ __forceinline__ void run_item(const smg::PairArgs& a, int kf, const BatchItem& it) {
    const int div = min(a.exact_recip[0], min(a.exact_recip[1], a.exact_recip[2]));
    if (div == 2) smg::pair_item<MODE, 2, 1, false>(a, kf, it.grp, it.chunk, it.row, threadIdx.x, blockDim.x);
    else if (div == 1) smg::pair_item<MODE, 1, 1, false>(a, kf, it.grp, it.chunk, it.row, threadIdx.x, blockDim.x);
    else smg::pair_item<MODE, 0, 1, false>(a, kf, it.grp, it.chunk, it.row, threadIdx.x, blockDim.x);
}

__global__ void __launch_bounds__(256, 4) k_batch(BatchArgs B) {
    __shared__ smg::PairArgs sa;
    __shared__ int s_flag;
    const int nph = 2 * B.steps + 1;   // A, (B, AA)*(steps-1), B, A
    for (int ph = 0; ph < nph; ++ph) {
        int mode, kf;
        if (ph == 0) { mode = 0; kf = 1; }
        else if (ph == nph - 1) { mode = 0; kf = 2; }
        else if (ph & 1) { mode = 1; kf = 0; }
        else { mode = 2; kf = 0; }
        const int list = mode == 1 ? 1 : 0;
        for (int w = blockIdx.x; w < B.nitems[list]; w += gridDim.x) {
            const BatchItem it = B.items[list][w];
            __syncthreads();
            {
                const int* src = reinterpret_cast<const int*>(B.args + 2 * it.inst + list);
                int* dst = reinterpret_cast<int*>(&sa);
                for (int k = threadIdx.x; k < (int)(sizeof(smg::PairArgs) / 4); k += blockDim.x) dst[k] = src[k];
            }
            __syncthreads();
            if (mode == 0) run_item<0>(sa, kf, it);
            else if (mode == 1) run_item<1>(sa, kf, it);
            else run_item<2>(sa, kf, it);
        }
        if (!grid_barrier(B, &s_flag)) return;
    }
}

// Non-persistent form: one launch per phase, one work item per CTA (the
// read-only load path is valid because a phase never reads what it writes).
template <int MODE>
__global__ void __launch_bounds__(256, 4) k_batch_phase(const smg::PairArgs* args, const BatchItem* items, int list,
                                                         int kf) {
    __shared__ smg::PairArgs sa;
    const BatchItem it = items[blockIdx.x];
    {
        const int* src = reinterpret_cast<const int*>(args + 2 * it.inst + list);
        int* dst = reinterpret_cast<int*>(&sa);
        for (int k = threadIdx.x; k < (int)(sizeof(smg::PairArgs) / 4); k += blockDim.x) dst[k] = src[k];
    }
    __syncthreads();
    const int div = min(sa.exact_recip[0], min(sa.exact_recip[1], sa.exact_recip[2]));
    if (div == 2) smg::pair_item<MODE, 2, 1, true>(sa, kf, it.grp, it.chunk, it.row, threadIdx.x, blockDim.x);
    else if (div == 1) smg::pair_item<MODE, 1, 1, true>(sa, kf, it.grp, it.chunk, it.row, threadIdx.x, blockDim.x);
    else smg::pair_item<MODE, 0, 1, true>(sa, kf, it.grp, it.chunk, it.row, threadIdx.x, blockDim.x);
}

}  // namespace

struct smg_batch {
    std::vector<smg_handle*> inst;
    std::vector<double> dt;
    std::vector<smg::PairArgs> args;
    smg::PairArgs* d_args = nullptr;
    std::vector<BatchItem> items[2];
    BatchItem* d_items[2] = {nullptr, nullptr};
    BarrierState* d_bar = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraphExec_t graph = nullptr;
    int64_t graph_steps = -1;
    int block = 64, group = 8, steps_per_launch = 8;
    int grid = 0;
    long long spin_limit = 1LL << 25;   // ~2 s of polling
    int barrier_extra = 0;
    bool use_graph = true;
    bool persistent = true;          // one cooperative launch per block of steps
    double last_ms = 0;
    int64_t last_launches = 0;
    std::string err;
    // generated family kernels (default): instances with the same structure
    // share kernels, geometry from a per-instance table
    int jit = 1;
    smg::JitFamilySet* fam = nullptr;
    bool fam_failed = false;
    std::string fam_err;
    bool graph_jit = false;
    int64_t graph_launch_count = 0;
};

namespace {

thread_local std::string g_batch_err;   // message of smg_batch_last_error(NULL), per host thread

std::string* batch_err(const smg_batch* b) { return b ? &const_cast<smg_batch*>(b)->err : &g_batch_err; }

int bfail(smg_batch* b, int code, const std::string& m) {
    if (b) b->err = m;
    else g_batch_err = m;
    return code;
}

int bcuda(smg_batch* b, cudaError_t e, const char* what) {
    return bfail(b, e == cudaErrorMemoryAllocation ? SMG_ENOMEM : SMG_ECUDA,
                 std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

#define B_CUDA(b, expr)                                          \
    do {                                                         \
        cudaError_t e_ = (expr);                                 \
        if (e_ != cudaSuccess) return bcuda((b), e_, #expr);     \
    } while (0)

smg::PairArgs phase_args(const smg_handle* h, int phase, int block, int group) {
    smg::PairArgs a{};
    const auto& P = h->pair[phase];
    a.g = h->g;
    a.U = h->dU;
    a.dests = P.d_dests;
    a.coff = P.d_coff;
    a.cw = P.d_cw;
    a.ndest = P.ndest;
    a.group = group;
    a.ngroups = (P.ndest + group - 1) / group;
    const int tpr = (h->g.B[0] + 1) / 2;
    a.nchunks = (tpr + block - 1) / block;
    a.hdt = h->hdt;
    for (int k = 0; k < 3; ++k) {
        a.rh[k] = h->rh[k];
        a.exact_recip[k] = h->exact_recip[k];
    }
    a.filter_substep = h->filter_mode == 1;
    return a;
}

void free_items(smg_batch* b) {
    for (int l = 0; l < 2; ++l) {
        cudaFree(b->d_items[l]);
        b->d_items[l] = nullptr;
    }
    cudaFree(b->d_args);
    b->d_args = nullptr;
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_steps = -1;
}

// Rebuild argument tables and work lists for the current block/group.
int build_items(smg_batch* b) {
    free_items(b);
    const int n = (int)b->inst.size();
    b->args.assign(2 * n, smg::PairArgs{});
    for (int l = 0; l < 2; ++l) b->items[l].clear();
    for (int i = 0; i < n; ++i) {
        const smg_handle* h = b->inst[i];
        for (int l = 0; l < 2; ++l) {
            const smg::PairArgs a = phase_args(h, l, b->block, b->group);
            b->args[2 * i + l] = a;
            if (a.ndest == 0) continue;
            const int rows = h->g.B[1] * h->g.B[2];
            for (int r = 0; r < rows; ++r)
                for (int c = 0; c < a.nchunks; ++c)
                    for (int g = 0; g < a.ngroups; ++g) b->items[l].push_back(BatchItem{i, g, c, r});
        }
    }
    B_CUDA(b, cudaMalloc(&b->d_args, sizeof(smg::PairArgs) * b->args.size()));
    B_CUDA(b, cudaMemcpyAsync(b->d_args, b->args.data(), sizeof(smg::PairArgs) * b->args.size(),
                              cudaMemcpyHostToDevice, b->stream));
    for (int l = 0; l < 2; ++l) {
        const size_t nb = std::max<size_t>(b->items[l].size(), 1) * sizeof(BatchItem);
        B_CUDA(b, cudaMalloc(&b->d_items[l], nb));
        if (!b->items[l].empty())
            B_CUDA(b, cudaMemcpyAsync(b->d_items[l], b->items[l].data(), b->items[l].size() * sizeof(BatchItem),
                                      cudaMemcpyHostToDevice, b->stream));
    }
    int per_sm = 0, nsm = 0, dev = 0;
    B_CUDA(b, cudaGetDevice(&dev));
    B_CUDA(b, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    B_CUDA(b, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch, b->block, 0));
    if (per_sm < 1) return bfail(b, SMG_EINVAL, "batch kernel cannot be resident with this block size");
    b->grid = per_sm * nsm;
    B_CUDA(b, cudaStreamSynchronize(b->stream));
    return SMG_OK;
}

cudaError_t launch_block(smg_batch* b, int steps) {
    BatchArgs A{};
    A.args = b->d_args;
    for (int l = 0; l < 2; ++l) {
        A.items[l] = b->d_items[l];
        A.nitems[l] = (int)b->items[l].size();
    }
    A.steps = steps;
    A.bar = b->d_bar;
    A.spin_limit = b->spin_limit;
    A.expected = (unsigned)b->grid + (unsigned)b->barrier_extra;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)b->grid);
    cfg.blockDim = dim3((unsigned)b->block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = b->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_batch, A);
}

cudaError_t launch_phase_batch(smg_batch* b, int mode, int kf) {
    const int list = mode == 1 ? 1 : 0;
    const unsigned n = (unsigned)b->items[list].size();
    if (n == 0) return cudaSuccess;
    if (mode == 0) k_batch_phase<0><<<n, b->block, 0, b->stream>>>(b->d_args, b->d_items[list], list, kf);
    else if (mode == 1) k_batch_phase<1><<<n, b->block, 0, b->stream>>>(b->d_args, b->d_items[list], list, kf);
    else k_batch_phase<2><<<n, b->block, 0, b->stream>>>(b->d_args, b->d_items[list], list, kf);
    return cudaGetLastError();
}

// the generated family kernels are built once (on the first run that wants
// them); without NVRTC the batch keeps the precompiled kernels
void ensure_fam(smg_batch* b) {
    if (!b->jit || b->fam || b->fam_failed) return;
    const smg_handle* h0 = b->inst[0];
    std::string why;
    if (smg::jit_family_build(b->inst, h0->jit_block, h0->jit_group, h0->jit_split > 0 ? h0->jit_split : 16,
                              h0->jit_regs, b->fam, why) != SMG_OK) {
        b->fam_failed = true;
        b->fam_err = why;
        b->fam = nullptr;
    }
}

bool use_fam(const smg_batch* b) { return b->jit && b->fam; }

cudaError_t enqueue_run(smg_batch* b, int64_t nsteps, int64_t* launches) {
    int64_t L = 0;
    if (use_fam(b)) {
        // A(k=1) [B AA]... B A(k=2), every phase one set of concurrent family kernels
        if (nsteps > 0) {
            cudaError_t e;
            if ((e = smg::jit_family_phase(b->fam, 0, 1, b->stream, &L)) != cudaSuccess) return e;
            for (int64_t k = 0; k < nsteps; ++k) {
                if ((e = smg::jit_family_phase(b->fam, 1, 0, b->stream, &L)) != cudaSuccess) return e;
                if ((e = smg::jit_family_phase(b->fam, k + 1 < nsteps ? 2 : 0, 2, b->stream, &L)) != cudaSuccess)
                    return e;
            }
        }
        if (launches) *launches = L;
        return cudaSuccess;
    }
    if (!b->persistent) {
        // A(k=1) [B AA]... B A(k=2): the fused sequence of the plain solver
        if (nsteps > 0) {
            cudaError_t e;
            if ((e = launch_phase_batch(b, 0, 1)) != cudaSuccess) return e;
            ++L;
            for (int64_t k = 0; k < nsteps; ++k) {
                if ((e = launch_phase_batch(b, 1, 0)) != cudaSuccess) return e;
                if ((e = launch_phase_batch(b, k + 1 < nsteps ? 2 : 0, 2)) != cudaSuccess) return e;
                L += 2;
            }
        }
        if (launches) *launches = L;
        return cudaSuccess;
    }
    for (int64_t done = 0; done < nsteps;) {
        const int s = (int)std::min<int64_t>(b->steps_per_launch, nsteps - done);
        cudaError_t e = launch_block(b, s);
        if (e != cudaSuccess) return e;
        ++L;
        done += s;
    }
    if (launches) *launches = L;
    return cudaSuccess;
}

}  // namespace

extern "C" {

int smg_batch_create(int32_t n_inst, const smg_problem* const* probs, smg_batch** out) {
    SMG_TRY
    if (!out || n_inst < 1 || !probs) return bfail(nullptr, SMG_EINVAL, "smg_batch_create: bad arguments");
    *out = nullptr;
    // the batch kernels apply no full-step filter (f_position 'full',
    // starmap_solver.m:417-421): refuse such instances rather than skip it
    for (int i = 0; i < n_inst; ++i)
        if (!probs[i] || probs[i]->filter_mode == SMG_FILTER_FULL)
            return bfail(nullptr, SMG_EINVAL,
                         "smg_batch_create: instance " + std::to_string(i) +
                             (probs[i] ? " uses f_position 'full', which the batched solver does not apply"
                                       : " is NULL"));
    smg_batch* b = new smg_batch();
    for (int i = 0; i < n_inst; ++i) {
        smg_handle* h = nullptr;
        const int rc = smg_create(probs[i], &h);
        if (rc != SMG_OK) {
            std::string m = std::string("instance ") + std::to_string(i) + ": " + smg_last_error(nullptr);
            smg_batch_destroy(b);
            return bfail(nullptr, rc, m);
        }
        b->inst.push_back(h);
        if (!(h->pair[0].ok && h->pair[1].ok)) {
            smg_batch_destroy(b);
            return bfail(nullptr, SMG_EINVAL, "instance " + std::to_string(i) + " has no pair-kernel tables");
        }
    }
    b->dt.assign(n_inst, 0.0);
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&b->ev0)) != cudaSuccess || (e = cudaEventCreate(&b->ev1)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_bar, sizeof(BarrierState))) != cudaSuccess ||
        (e = cudaMemset(b->d_bar, 0, sizeof(BarrierState))) != cudaSuccess) {
        const int rc = bcuda(nullptr, e, "smg_batch_create");
        smg_batch_destroy(b);
        return rc;
    }
    const int rc = build_items(b);
    if (rc != SMG_OK) {
        g_batch_err = b->err;
        smg_batch_destroy(b);
        return rc;
    }
    *out = b;
    return SMG_OK;
    SMG_CATCH(batch_err(nullptr))
}

void smg_batch_destroy(smg_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    free_items(b);
    smg::jit_family_free(b->fam);
    cudaFree(b->d_bar);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    for (smg_handle* h : b->inst) smg_destroy(h);
    delete b;
}

const char* smg_batch_last_error(const smg_batch* b) { return b ? b->err.c_str() : g_batch_err.c_str(); }

smg_handle* smg_batch_instance(smg_batch* b, int32_t i) {
    if (!b || i < 0 || i >= (int)b->inst.size()) return nullptr;
    return b->inst[i];
}

int smg_batch_set_dt(smg_batch* b, const double* dt) {
    SMG_TRY
    if (!b || !dt) return bfail(b, SMG_EINVAL, "smg_batch_set_dt: NULL argument");
    for (size_t i = 0; i < b->inst.size(); ++i) {
        const int rc = smg_set_dt(b->inst[i], dt[i]);
        if (rc != SMG_OK) return bfail(b, rc, "instance " + std::to_string(i) + ": " + smg_last_error(b->inst[i]));
        b->dt[i] = dt[i];
    }
    return build_items(b);   // hdt and refreshed coefficient tables enter the argument table
    SMG_CATCH(batch_err(b))
}

int smg_batch_run(smg_batch* b, int64_t nsteps) {
    SMG_TRY
    if (!b) return bfail(b, SMG_EINVAL, "smg_batch_run: NULL batch");
    if (nsteps < 0) return bfail(b, SMG_EINVAL, "smg_batch_run: nsteps must be >= 0");
    for (size_t i = 0; i < b->inst.size(); ++i) {
        if (!b->inst[i]->dt_set) return bfail(b, SMG_ESTATE, "smg_batch_run: dt not set");
        if (!b->inst[i]->state_set) return bfail(b, SMG_ESTATE, "smg_batch_run: state not set");
        const smg_handle* h = b->inst[i];
        if (!h->src_expr.empty() || h->mat.on || !h->filt.f1.empty())
            return bfail(b, SMG_EINVAL,
                         "smg_batch_run: device-evaluated sources, materials or filters are not supported in a batch");
        B_CUDA(b, cudaStreamSynchronize(b->inst[i]->stream));
    }
    B_CUDA(b, cudaMemsetAsync(b->d_bar, 0, sizeof(BarrierState), b->stream));
    ensure_fam(b);
    if (use_fam(b)) B_CUDA(b, smg::jit_family_geometry(b->fam, b->inst, b->stream));
    int64_t launches = 0;
    bool graphed = false;
    if (b->use_graph && nsteps > 0) {
        if (!b->graph || b->graph_steps != nsteps || b->graph_jit != use_fam(b)) {
            if (b->graph) cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
            cudaGraph_t gr;
            cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                cudaError_t e1 = enqueue_run(b, nsteps, &launches);
                cudaError_t e2 = cudaStreamEndCapture(b->stream, &gr);
                if (e1 == cudaSuccess && e2 == cudaSuccess) {
                    e = cudaGraphInstantiate(&b->graph, gr, 0);
                    cudaGraphDestroy(gr);
                    if (e == cudaSuccess) {
                        b->graph_steps = nsteps;
                        b->graph_jit = use_fam(b);
                        b->graph_launch_count = launches;
                    } else {
                        b->graph = nullptr;
                    }
                }
            }
            cudaGetLastError();   // a capture that is not supported falls back to direct launches
        }
        if (b->graph) {
            B_CUDA(b, cudaEventRecord(b->ev0, b->stream));
            B_CUDA(b, cudaGraphLaunch(b->graph, b->stream));
            B_CUDA(b, cudaEventRecord(b->ev1, b->stream));
            launches = b->graph_launch_count;
            graphed = true;
        }
    }
    if (!graphed) {
        B_CUDA(b, cudaEventRecord(b->ev0, b->stream));
        B_CUDA(b, enqueue_run(b, nsteps, &launches));
        B_CUDA(b, cudaEventRecord(b->ev1, b->stream));
    }
    b->last_launches = launches;
    BarrierState st{};
    B_CUDA(b, cudaMemcpyAsync(&st, b->d_bar, sizeof(st), cudaMemcpyDeviceToHost, b->stream));
    B_CUDA(b, cudaStreamSynchronize(b->stream));
    float ms = 0.f;
    B_CUDA(b, cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    b->last_ms = ms;
    if (st.err) return bfail(b, SMG_ETIMEOUT, "batch grid barrier wait exceeded its spin limit");
    return SMG_OK;
    SMG_CATCH(batch_err(b))
}

int smg_batch_last_run_stats(smg_batch* b, double* ms, int64_t* launches) {
    SMG_TRY
    if (!b) return bfail(b, SMG_EINVAL, "smg_batch_last_run_stats: NULL batch");
    if (ms) *ms = b->last_ms;
    if (launches) *launches = b->last_launches;
    return SMG_OK;
    SMG_CATCH(batch_err(b))
}

int smg_batch_tune(smg_batch* b, int32_t key, int64_t value) {
    SMG_TRY
    if (!b) return bfail(b, SMG_EINVAL, "smg_batch_tune: NULL batch");
    switch (key) {
        case SMG_BATCH_BLOCK:
            if (value < 32 || value > 256 || value % 32) return bfail(b, SMG_EINVAL, "block must be 32..256, x32");
            b->block = (int)value;
            break;
        case SMG_BATCH_GROUP:
            if (value < 1 || value > 256) return bfail(b, SMG_EINVAL, "group must be 1..256");
            b->group = (int)value;
            break;
        case SMG_BATCH_STEPS_PER_LAUNCH:
            if (value < 1 || value > 4096) return bfail(b, SMG_EINVAL, "steps per launch must be 1..4096");
            b->steps_per_launch = (int)value;
            break;
        case SMG_BATCH_SPIN_LIMIT:
            if (value < 1) return bfail(b, SMG_EINVAL, "spin limit must be >= 1");
            b->spin_limit = value;
            break;
        case SMG_BATCH_BARRIER_EXTRA:
            if (value < 0 || value > 1) return bfail(b, SMG_EINVAL, "barrier extra must be 0 or 1");
            b->barrier_extra = (int)value;
            break;
        case SMG_BATCH_USE_GRAPH:
            b->use_graph = value != 0;
            break;
        case SMG_BATCH_PERSISTENT:
            b->persistent = value != 0;
            break;
        case SMG_BATCH_JIT:
            if (value != 0 && value != 1) return bfail(b, SMG_EINVAL, "jit must be 0 or 1");
            b->jit = (int)value;
            break;
        default:
            return bfail(b, SMG_EINVAL, "smg_batch_tune: unknown key");
    }
    return build_items(b);
    SMG_CATCH(batch_err(b))
}

int smg_batch_info(const smg_batch* b, int64_t* jit_active, int64_t* families) {
    SMG_TRY
    if (!b) return bfail(nullptr, SMG_EINVAL, "smg_batch_info: NULL batch");
    if (jit_active) *jit_active = use_fam(b) ? 1 : 0;
    if (families) *families = smg::jit_family_count(b->fam);
    return SMG_OK;
    SMG_CATCH(batch_err(b))
}

int smg_batch_config(const smg_batch* b, int64_t out[4]) {
    SMG_TRY
    if (!b || !out) return bfail(nullptr, SMG_EINVAL, "smg_batch_config: NULL argument");
    out[0] = b->block;
    out[1] = b->group;
    out[2] = b->steps_per_launch;
    out[3] = b->persistent ? b->grid : 0;
    return SMG_OK;
    SMG_CATCH(batch_err(b))
}

int smg_batch_autotune(smg_batch* b, int64_t probe_steps, double* best_ms) {
    SMG_TRY
    if (!b || probe_steps < 1) return bfail(b, SMG_EINVAL, "smg_batch_autotune: bad arguments");
    // snapshot every instance's state; the probes advance it
    std::vector<double*> save(b->inst.size(), nullptr);
    for (size_t i = 0; i < b->inst.size(); ++i) {
        const size_t bytes = (size_t)b->inst[i]->g.cs * b->inst[i]->n_sys * 8;
        B_CUDA(b, cudaMalloc(&save[i], bytes));
        B_CUDA(b, cudaMemcpyAsync(save[i], b->inst[i]->dU, bytes, cudaMemcpyDeviceToDevice, b->stream));
    }
    const int blocks[] = {64, 128};
    const int groups[] = {4, 8, 16};
    const int spls[] = {0, 4, 8, 16};   // 0: one launch per phase
    double best = 1e300;
    int bb = b->block, bg = b->group, bs = b->steps_per_launch;
    bool bp = b->persistent;
    int bj = 0;
    int rc = SMG_OK;
    // the generated family kernels first (when they can be built), then the
    // precompiled configurations
    b->jit = 1;
    ensure_fam(b);
    if (b->fam) {
        if ((rc = smg_batch_run(b, probe_steps)) != SMG_OK) goto done;
        best = b->last_ms;
        bj = 1;
    }
    b->jit = 0;
    for (int blk : blocks)
        for (int grp : groups)
            for (int spl : spls) {
                b->block = blk;
                b->group = grp;
                b->persistent = spl > 0;
                if (spl > 0) b->steps_per_launch = spl;
                if ((rc = build_items(b)) != SMG_OK) goto done;
                if ((rc = smg_batch_run(b, probe_steps)) != SMG_OK) goto done;
                if (b->last_ms < best) {
                    best = b->last_ms;
                    bb = blk;
                    bg = grp;
                    bs = b->steps_per_launch;
                    bp = b->persistent;
                    bj = 0;
                }
            }
done:
    b->block = bb;
    b->group = bg;
    b->steps_per_launch = bs;
    b->persistent = bp;
    b->jit = bj;
    for (size_t i = 0; i < b->inst.size(); ++i) {
        const size_t bytes = (size_t)b->inst[i]->g.cs * b->inst[i]->n_sys * 8;
        cudaMemcpyAsync(b->inst[i]->dU, save[i], bytes, cudaMemcpyDeviceToDevice, b->stream);
    }
    cudaStreamSynchronize(b->stream);
    for (double* p : save) cudaFree(p);
    if (rc != SMG_OK) return rc;
    if (best_ms) *best_ms = best;
    return build_items(b);
    SMG_CATCH(batch_err(b))
}

}  // extern "C"
