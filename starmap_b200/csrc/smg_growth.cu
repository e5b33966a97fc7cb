// smg_growth.cu -- spectral radius of the full-step growth matrix on the GPU.
//
// The reference's parabolic time step (par.timestep 1 or 2) searches the
// largest stable dt by bracketing and bisection; every trial evaluates
// growth_factor (starmap_solver.m:506-514): the von Neumann growth matrix of
// one step, G_o G_e G_e G_o, with G_e / G_o the identity in the rows of the
// phase-A / phase-B components and I + G in the others, and its largest
// eigenvalue modulus.  With hundreds of moments this is the host's dominant
// cost (dense complex eigenvalues of an n_sys x n_sys matrix, about 15 per
// search).  Here the three products run with cuBLAS (ZGEMM) and the
// eigenvalues with cuSOLVER's general eigensolver (cusolverDnXgeev, no
// eigenvectors); both libraries are opened with dlopen on the first call, so
// the library keeps no link-time dependency on them.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>
#include <dlfcn.h>

#include <cmath>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/starmap_gpu.h"
#include "smg_internal.h"

namespace {

struct LinalgApi {
    bool ok = false;
    std::string why;
    decltype(&cublasCreate_v2) blasCreate = nullptr;
    decltype(&cublasSetStream_v2) blasSetStream = nullptr;
    decltype(&cublasZgemm_v2) zgemm = nullptr;
    decltype(&cusolverDnCreate) solverCreate = nullptr;
    decltype(&cusolverDnSetStream) solverSetStream = nullptr;
    decltype(&cusolverDnCreateParams) createParams = nullptr;
    decltype(&cusolverDnXgeev_bufferSize) geevBuffer = nullptr;
    decltype(&cusolverDnXgeev) geev = nullptr;
};

// The toolkit's copy by absolute path first: a process may hold another
// release under the same name (PyTorch bundles its own).
void* open_lib(const char* name) {
    const char* roots[] = {std::getenv("CUDA_HOME"), "/usr/local/cuda"};
    for (const char* root : roots) {
        if (!root || !*root) continue;
        const std::string path = std::string(root) + "/lib64/" + name;
        if (void* p = dlopen(path.c_str(), RTLD_NOW | RTLD_LOCAL)) return p;
    }
    return dlopen(name, RTLD_NOW | RTLD_LOCAL);
}

template <typename F>
bool sym(void* lib, const char* name, F& f) {
    f = reinterpret_cast<F>(dlsym(lib, name));
    return f != nullptr;
}

LinalgApi& linalg() {
    static LinalgApi a;
    static std::once_flag once;
    std::call_once(once, [] {
        void* bl = open_lib("libcublas.so.12");
        void* so = open_lib("libcusolver.so.11");
        if (!bl || !so) {
            a.why = !bl ? "cuBLAS (libcublas.so.12) not found" : "cuSOLVER (libcusolver.so.11) not found";
            return;
        }
        a.ok = sym(bl, "cublasCreate_v2", a.blasCreate) && sym(bl, "cublasSetStream_v2", a.blasSetStream) &&
               sym(bl, "cublasZgemm_v2", a.zgemm) && sym(so, "cusolverDnCreate", a.solverCreate) &&
               sym(so, "cusolverDnSetStream", a.solverSetStream) &&
               sym(so, "cusolverDnCreateParams", a.createParams) &&
               sym(so, "cusolverDnXgeev_bufferSize", a.geevBuffer) && sym(so, "cusolverDnXgeev", a.geev);
        if (!a.ok) a.why = "cuBLAS / cuSOLVER entry points missing (cusolverDnXgeev needs CUDA 12.6 or later)";
    });
    return a;
}

// per device: library handles, a stream and device buffers for the largest n seen
struct Workspace {
    bool init = false;
    cudaStream_t stream = nullptr;
    cublasHandle_t blas = nullptr;
    cusolverDnHandle_t solver = nullptr;
    cusolverDnParams_t params = nullptr;
    int64_t n = 0;
    cuDoubleComplex *G = nullptr, *Ge = nullptr, *Go = nullptr, *T = nullptr, *P = nullptr, *W = nullptr;
    int* odd = nullptr;
    int* info = nullptr;
    void* dwork = nullptr;
    size_t dwork_bytes = 0;
    std::vector<char> hwork;
};

std::mutex g_ws_mu;
Workspace g_ws[64];

// Ge = I + G with the phase-A rows (odd) replaced by identity rows; Go the
// same with the phase-B rows replaced (column-major, one thread per element)
__global__ void k_halves(const cuDoubleComplex* __restrict__ G, const int* __restrict__ odd, int64_t n,
                         cuDoubleComplex* __restrict__ Ge, cuDoubleComplex* __restrict__ Go) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n * n) return;
    const int64_t i = k % n, j = k / n;
    const cuDoubleComplex g = G[k];
    const double d = i == j ? 1.0 : 0.0;
    const cuDoubleComplex gi = make_cuDoubleComplex(g.x + d, g.y);
    const cuDoubleComplex id = make_cuDoubleComplex(d, 0.0);
    Ge[k] = odd[i] ? id : gi;
    Go[k] = odd[i] ? gi : id;
}

int fail(int code, const std::string& m) {
    smg::set_global_error(m);
    return code;
}

}  // namespace

extern "C" int smg_growth_radius(int32_t n, const double* G, const int32_t* odd, double* la) {
    SMG_TRY
    if (n < 1 || !G || !odd || !la) return fail(SMG_EINVAL, "smg_growth_radius: need n >= 1 and non-NULL arrays");
    LinalgApi& a = linalg();
    if (!a.ok) return fail(SMG_EINVAL, "smg_growth_radius: " + a.why);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64)
        return fail(SMG_ECUDA, std::string("smg_growth_radius: cudaGetDevice: ") + cudaGetErrorString(e));
    std::lock_guard<std::mutex> lk(g_ws_mu);
    Workspace& w = g_ws[dev];
#define GR_CUDA(expr)                                                                                       \
    do {                                                                                                    \
        cudaError_t e_ = (expr);                                                                            \
        if (e_ != cudaSuccess) return fail(SMG_ECUDA, std::string("smg_growth_radius: " #expr ": ") + cudaGetErrorString(e_)); \
    } while (0)
#define GR_LIB(expr)                                                                                        \
    do {                                                                                                    \
        const int s_ = (int)(expr);                                                                         \
        if (s_ != 0) return fail(SMG_ECUDA, "smg_growth_radius: " #expr " returned " + std::to_string(s_)); \
    } while (0)
    if (!w.init) {
        GR_CUDA(cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking));
        GR_LIB(a.blasCreate(&w.blas));
        GR_LIB(a.blasSetStream(w.blas, w.stream));
        GR_LIB(a.solverCreate(&w.solver));
        GR_LIB(a.solverSetStream(w.solver, w.stream));
        GR_LIB(a.createParams(&w.params));
        w.init = true;
    }
    const int64_t N = n;
    const size_t mat = sizeof(cuDoubleComplex) * (size_t)N * (size_t)N;
    if (N > w.n) {
        cudaFree(w.G); cudaFree(w.Ge); cudaFree(w.Go); cudaFree(w.T); cudaFree(w.P); cudaFree(w.W);
        cudaFree(w.odd); cudaFree(w.info);
        w.G = w.Ge = w.Go = w.T = w.P = w.W = nullptr;
        w.odd = w.info = nullptr;
        w.n = 0;
        GR_CUDA(cudaMalloc(&w.G, mat));
        GR_CUDA(cudaMalloc(&w.Ge, mat));
        GR_CUDA(cudaMalloc(&w.Go, mat));
        GR_CUDA(cudaMalloc(&w.T, mat));
        GR_CUDA(cudaMalloc(&w.P, mat));
        GR_CUDA(cudaMalloc(&w.W, sizeof(cuDoubleComplex) * (size_t)N));
        GR_CUDA(cudaMalloc(&w.odd, sizeof(int) * (size_t)N));
        GR_CUDA(cudaMalloc(&w.info, sizeof(int)));
        w.n = N;
    }
    std::vector<int> oddv(odd, odd + N);
    GR_CUDA(cudaMemcpyAsync(w.G, G, mat, cudaMemcpyHostToDevice, w.stream));
    GR_CUDA(cudaMemcpyAsync(w.odd, oddv.data(), sizeof(int) * (size_t)N, cudaMemcpyHostToDevice, w.stream));
    const unsigned nb = (unsigned)((N * N + 255) / 256);
    k_halves<<<nb, 256, 0, w.stream>>>(w.G, w.odd, N, w.Ge, w.Go);
    GR_CUDA(cudaGetLastError());
    // P = ((Go Ge) Ge) Go, the reference's left-to-right product
    const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
    GR_LIB(a.zgemm(w.blas, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, w.Go, n, w.Ge, n, &zero, w.T, n));
    GR_LIB(a.zgemm(w.blas, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, w.T, n, w.Ge, n, &zero, w.P, n));
    GR_LIB(a.zgemm(w.blas, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, w.P, n, w.Go, n, &zero, w.T, n));
    size_t dbytes = 0, hbytes = 0;
    GR_LIB(a.geevBuffer(w.solver, w.params, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_NOVECTOR, N, CUDA_C_64F,
                        w.T, N, CUDA_C_64F, w.W, CUDA_C_64F, nullptr, 1, CUDA_C_64F, nullptr, 1, CUDA_C_64F, &dbytes,
                        &hbytes));
    if (dbytes > w.dwork_bytes) {
        cudaFree(w.dwork);
        w.dwork = nullptr;
        w.dwork_bytes = 0;
        GR_CUDA(cudaMalloc(&w.dwork, dbytes));
        w.dwork_bytes = dbytes;
    }
    if (hbytes > w.hwork.size()) w.hwork.resize(hbytes);
    GR_LIB(a.geev(w.solver, w.params, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_NOVECTOR, N, CUDA_C_64F, w.T, N,
                  CUDA_C_64F, w.W, CUDA_C_64F, nullptr, 1, CUDA_C_64F, nullptr, 1, CUDA_C_64F, w.dwork, dbytes,
                  hbytes ? w.hwork.data() : nullptr, hbytes, w.info));
    std::vector<cuDoubleComplex> ev((size_t)N);
    int info = 0;
    GR_CUDA(cudaMemcpyAsync(ev.data(), w.W, sizeof(cuDoubleComplex) * (size_t)N, cudaMemcpyDeviceToHost, w.stream));
    GR_CUDA(cudaMemcpyAsync(&info, w.info, sizeof(int), cudaMemcpyDeviceToHost, w.stream));
    GR_CUDA(cudaStreamSynchronize(w.stream));
#undef GR_CUDA
#undef GR_LIB
    if (info != 0) return fail(SMG_ECUDA, "smg_growth_radius: cusolverDnXgeev info " + std::to_string(info));
    double m = 0.0;
    for (const cuDoubleComplex& v : ev) m = std::fmax(m, std::hypot(v.x, v.y));
    *la = m;
    return SMG_OK;
    SMG_CATCH(nullptr)
}
