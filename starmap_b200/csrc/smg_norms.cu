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
}
