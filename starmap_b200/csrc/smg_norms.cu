// smg_norms.cu -- per-component sums of squares of the state.
//
// The squared discrete L2 norm of every moment component, the quantity the
// reference's energy example monitors over time (starmap_2d_ex_l2norm.m:61-99,
// there with staggered trapezoid weights applied by the caller) and the
// denominator of per-moment relative L2 parity checks.  Two passes with a
// fixed reduction order, so the result is reproducible bit for bit:
//   pass 1: kSumsqBlocks CTAs per component, each thread sums x^2 over a
//           fixed strided subset of the component's slot, a CTA tree
//           reduction writes one partial per (component, CTA) to scratch;
//   pass 2: one thread per component adds its kSumsqBlocks partials in order.
// Padding points of a slot hold zeros, so the whole slot is summed.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/starmap_gpu.h"
#include "smg_internal.h"

namespace smg {

__global__ void __launch_bounds__(kSumsqThreads) k_sumsq_partial(const double* __restrict__ x, long long stride,
                                                                  long long len, double* __restrict__ partial) {
    __shared__ double red[kSumsqThreads];
    const int c = blockIdx.y;
    const double* xc = x + (long long)c * stride;
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * kSumsqThreads + threadIdx.x; i < len;
         i += (long long)kSumsqBlocks * kSumsqThreads) {
        const double v = __ldg(xc + i);
        s = __fma_rn(v, v, s);
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = kSumsqThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] = __dadd_rn(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[(long long)c * kSumsqBlocks + blockIdx.x] = red[0];
}

__global__ void k_sumsq_final(const double* __restrict__ partial, int ncomp, double* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncomp) return;
    double s = 0.0;
    for (int b = 0; b < kSumsqBlocks; ++b) s = __dadd_rn(s, partial[(long long)c * kSumsqBlocks + b]);
    out[c] = s;
}

cudaError_t launch_sumsq(const double* x, int ncomp, long long stride, long long len, double* partial, double* out,
                         cudaStream_t s) {
    if (ncomp <= 0) return cudaSuccess;
    k_sumsq_partial<<<dim3(kSumsqBlocks, (unsigned)ncomp), kSumsqThreads, 0, s>>>(x, stride, len, partial);
    k_sumsq_final<<<(ncomp + 127) / 128, 128, 0, s>>>(partial, ncomp, out);
    return cudaGetLastError();
}

}  // namespace smg

extern "C" int smg_state_sumsq(smg_handle* h, double* sumsq) {
    SMG_TRY
    if (!h || !sumsq) return SMG_EINVAL;
    if (!h->dSumsq) {
        h->err = "smg_state_sumsq: no reduction buffer";
        return SMG_ESTATE;
    }
    double* partial = h->dSumsq;
    double* out = h->dSumsq + (size_t)h->n_sys * smg::kSumsqBlocks;
    cudaError_t e = smg::launch_sumsq(h->dU, h->n_sys, h->g.cs, h->g.cs, partial, out, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(sumsq, out, sizeof(double) * h->n_sys, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        h->err = std::string("smg_state_sumsq: ") + cudaGetErrorString(e);
        return SMG_ECUDA;
    }
    return SMG_OK;
    SMG_CATCH(h ? &h->err : nullptr)
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the reduction above.
//
// Some hosts of this library must not allocate GPU memory themselves: a MEX
// gateway running inside MATLAB works with gpuArray buffers that MATLAB's own
// allocator owns and may not want a second allocator on the device; callers
// that work under a fixed memory budget cannot afford an allocation (or the
// synchronisation a cudaMalloc/cudaFree implies) per reduction.  For them the
// partial sums go to a fixed array that is part of the library image: every
// GPU that loads the library holds it (256 KB) until the process exits.
// ---------------------------------------------------------------------------
namespace {

constexpr long long kNoAllocScratch = 32768;   // doubles: 1024 components x 32 partials
static __device__ __align__(256) double g_sumsq_scratch[kNoAllocScratch];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
// per device: the array's address and the context it belongs to.  A device
// reset (cudaDeviceReset, MATLAB's reset(gpuDevice)) destroys the context and
// unloads the module; the next context loads it again, possibly at another
// address, so the address is looked up again whenever the context changes.
double* g_scratch_addr[kMaxDevices] = {nullptr};
unsigned long long g_scratch_ctx[kMaxDevices] = {0};

int noalloc_fail(int code, const std::string& m) {
    smg::set_global_error(m);   // read back with smg_last_error(NULL)
    return code;
}

// Unique id of the calling thread's current context (cuCtxGetId, reached
// through the runtime's driver entry points, so the library needs no link to
// libcuda); 0 when there is none yet or the driver lacks the call.
using CtxGetCurrentFn = int (*)(void**);
using CtxGetIdFn = int (*)(void*, unsigned long long*);

unsigned long long current_ctx_id() {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static bool looked = false;
    if (!looked) {   // under g_scratch_mu
        looked = true;
        cudaDriverEntryPointQueryResult q1, q2;
        void* f1 = nullptr;
        void* f2 = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000, cudaEnableDefault, &q1) == cudaSuccess &&
            cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess) {
            get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
            get_id = reinterpret_cast<CtxGetIdFn>(f2);
        }
    }
    if (!get_current || !get_id) return 0;
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != 0 || !ctx) return 0;
    if (get_id(ctx, &id) != 0) return 0;
    return id;
}

}  // namespace

extern "C" int smg_sumsq_noalloc(const double* d_x, int32_t ncomp, int64_t stride, int64_t len, double* d_out,
                                 void* stream) {
    SMG_TRY
    if (!d_x || !d_out) return noalloc_fail(SMG_EINVAL, "smg_sumsq_noalloc: NULL device pointer");
    if (ncomp < 1 || len < 1 || stride < len)
        return noalloc_fail(SMG_EINVAL, "smg_sumsq_noalloc: need ncomp >= 1, len >= 1 and stride >= len");
    if ((long long)ncomp * smg::kSumsqBlocks > kNoAllocScratch)
        return noalloc_fail(SMG_EINVAL, "smg_sumsq_noalloc: " + std::to_string(ncomp) +
                                            " components exceed the fixed scratch (at most " +
                                            std::to_string(kNoAllocScratch / smg::kSumsqBlocks) + ")");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(SMG_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(SMG_EINVAL, "smg_sumsq_noalloc: device index too large");
    double* scratch;
    {
        // first call on this device, or in a new context of it (with it
        // current): look up the device address of the static array; host code
        // cannot use the symbol itself.  Without a context id (no current
        // context yet, or a driver without cuCtxGetId) it is looked up on
        // every call.
        std::lock_guard<std::mutex> lk(g_scratch_mu);
        const unsigned long long ctx = current_ctx_id();
        if (!g_scratch_addr[dev] || ctx == 0 || ctx != g_scratch_ctx[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_sumsq_scratch);
            if (e != cudaSuccess)
                return noalloc_fail(SMG_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_scratch_addr[dev] = static_cast<double*>(p);
            g_scratch_ctx[dev] = ctx ? ctx : current_ctx_id();   // the lookup may have created the context
        }
        scratch = g_scratch_addr[dev];
    }
    // every partial a launch reads is written by the same launch first, so the
    // contents left by an earlier call need no clearing
    e = smg::launch_sumsq(d_x, ncomp, stride, len, scratch, d_out, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return noalloc_fail(SMG_ECUDA, std::string("smg_sumsq_noalloc: ") + cudaGetErrorString(e));
    return SMG_OK;
    SMG_CATCH(nullptr)
}
