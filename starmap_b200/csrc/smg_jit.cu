// smg_jit.cu -- phase kernels specialised to one problem, generated as CUDA
// C++ source and compiled at run time with NVRTC for sm_100a.
//
// The pair kernel (smg_pair.cuh) reads, for every destination and thread, the
// destination's record (extents, coupling runs, coefficient pointers), the
// coupling table (source offset, weight) and selects stencil offsets, h and
// the division mode per run.  For the P_N systems these records cost more
// instructions than the arithmetic: a destination has only about four
// couplings.  Everything in those records is fixed when the handle is created
// (couplings and weights M_d(j,i), extents, grid spacing, division mode per
// axis, which field every coefficient comes from and whether it is an array),
// so the generator writes one straight-line block per destination with all of
// it as constants:
//
//   per coupling (two points of a row): two 128-bit loads of the neighbouring
//   source rows (y/z) or four 64-bit loads (x), the difference, the exact
//   division by h, the product with M_d(j,i), the fold in sumcell order (the
//   first term initialises the sum);
//
//   per destination: its two values, the coefficient values (read at run time
//   from the handle's field table, so smg_set_field and smg_set_dt keep
//   working), the one or two substep updates with filters, one store.
//
// Arithmetic and evaluation order are those of the pair kernel and the
// reference (starmap_solver.m:307-421): results are bit-identical.
//
// Structure: destinations are cut into groups; each group is one device
// function, compiled as relocatable code in its own small NVRTC program (the
// compilers' time grows faster than linearly with function size, so one
// program per few groups, compiled on all host threads, keeps the build to
// seconds even for 820 moments); a dispatch kernel per phase type maps a CTA
// to (group, row, chunk of the row) and calls the group's function; nvJitLink
// links everything into one cubin.  One launch per phase, as for the pair
// kernel.
//
// NVRTC, nvJitLink and the driver API are loaded with dlopen on first use, so
// the library has no link-time dependency on them; without them the handle
// keeps the precompiled kernels.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <atomic>
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <functional>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/starmap_gpu.h"
#include "smg_internal.h"

namespace {

// ---- dynamically loaded NVRTC, nvJitLink and driver entry points -------------
typedef int nvrtcResult_t;
typedef struct _nvrtcProgram* nvrtcProgram_t;
typedef int nvJitLinkResult_t;
typedef struct nvJitLink* nvJitLinkHandle_t;
typedef int CUresult_t;
typedef struct CUmod_st* CUmodule_t;
typedef struct CUfunc_st* CUfunction_t;
constexpr int kJitLinkInputCubin = 1;   // NVJITLINK_INPUT_CUBIN

struct Api {
    bool ok = false;
    std::string why;
    nvrtcResult_t (*CreateProgram)(nvrtcProgram_t*, const char*, const char*, int, const char* const*,
                                   const char* const*) = nullptr;
    nvrtcResult_t (*CompileProgram)(nvrtcProgram_t, int, const char* const*) = nullptr;
    nvrtcResult_t (*GetProgramLogSize)(nvrtcProgram_t, size_t*) = nullptr;
    nvrtcResult_t (*GetProgramLog)(nvrtcProgram_t, char*) = nullptr;
    nvrtcResult_t (*GetCUBINSize)(nvrtcProgram_t, size_t*) = nullptr;
    nvrtcResult_t (*GetCUBIN)(nvrtcProgram_t, char*) = nullptr;
    nvrtcResult_t (*DestroyProgram)(nvrtcProgram_t*) = nullptr;
    const char* (*GetErrorString)(nvrtcResult_t) = nullptr;
    nvrtcResult_t (*Version)(int*, int*) = nullptr;
    bool link_ok = false;
    std::string link_why;
    nvJitLinkResult_t (*LinkCreate)(nvJitLinkHandle_t*, uint32_t, const char**) = nullptr;
    nvJitLinkResult_t (*LinkDestroy)(nvJitLinkHandle_t*) = nullptr;
    nvJitLinkResult_t (*LinkAddData)(nvJitLinkHandle_t, int, const void*, size_t, const char*) = nullptr;
    nvJitLinkResult_t (*LinkComplete)(nvJitLinkHandle_t) = nullptr;
    nvJitLinkResult_t (*LinkedCubinSize)(nvJitLinkHandle_t, size_t*) = nullptr;
    nvJitLinkResult_t (*LinkedCubin)(nvJitLinkHandle_t, void*) = nullptr;
    nvJitLinkResult_t (*LinkErrorLogSize)(nvJitLinkHandle_t, size_t*) = nullptr;
    nvJitLinkResult_t (*LinkErrorLog)(nvJitLinkHandle_t, char*) = nullptr;
    bool cu_ok = false;
    std::string cu_why;
    CUresult_t (*ModuleLoadData)(CUmodule_t*, const void*) = nullptr;
    CUresult_t (*ModuleUnload)(CUmodule_t) = nullptr;
    CUresult_t (*ModuleGetFunction)(CUfunction_t*, CUmodule_t, const char*) = nullptr;
    CUresult_t (*LaunchKernel)(CUfunction_t, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                               cudaStream_t, void**, void**) = nullptr;
    CUresult_t (*FuncSetAttribute)(CUfunction_t, int, int) = nullptr;
    CUresult_t (*CtxGetCurrent)(void**) = nullptr;          // optional: module sharing between handles
    CUresult_t (*CtxGetId)(void*, unsigned long long*) = nullptr;
};
constexpr int kFuncAttrMaxDynamicSmem = 8;   // CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES

Api g_api;
std::once_flag g_api_once;

template <typename F>
bool sym(void* lib, const char* name, F& f) {
    f = reinterpret_cast<F>(dlsym(lib, name));
    return f != nullptr;
}

void* open_first(std::initializer_list<const char*> names) {
    for (const char* n : names) {
        void* p = dlopen(n, RTLD_NOW | RTLD_LOCAL);
        if (p) return p;
    }
    return nullptr;
}

// The CUDA toolkit's copy of a library by absolute path ($CUDA_HOME, then
// /usr/local/cuda), before the bare name: a process may already hold another
// release under the same name (PyTorch bundles its own NVRTC and nvJitLink),
// which dlopen by name would return.
void* open_toolkit(const char* lib, std::initializer_list<const char*> names) {
    const char* roots[] = {std::getenv("CUDA_HOME"), "/usr/local/cuda"};
    for (const char* root : roots) {
        if (!root || !*root) continue;
        const std::string path = std::string(root) + "/lib64/" + lib;
        if (void* p = dlopen(path.c_str(), RTLD_NOW | RTLD_LOCAL)) return p;
    }
    return open_first(names);
}

void load_api() {
    Api& a = g_api;
    void* nv = open_toolkit("libnvrtc.so.12", {"libnvrtc.so.12", "libnvrtc.so"});
    if (!nv) {
        a.why = "NVRTC (libnvrtc.so.12) not found";
    } else if (sym(nv, "nvrtcCreateProgram", a.CreateProgram) && sym(nv, "nvrtcCompileProgram", a.CompileProgram) &&
               sym(nv, "nvrtcGetProgramLogSize", a.GetProgramLogSize) &&
               sym(nv, "nvrtcGetProgramLog", a.GetProgramLog) && sym(nv, "nvrtcGetCUBINSize", a.GetCUBINSize) &&
               sym(nv, "nvrtcGetCUBIN", a.GetCUBIN) && sym(nv, "nvrtcDestroyProgram", a.DestroyProgram) &&
               sym(nv, "nvrtcGetErrorString", a.GetErrorString) && sym(nv, "nvrtcVersion", a.Version)) {
        a.ok = true;
    } else {
        a.why = "NVRTC entry points missing";
    }
    // nvJitLink exports versioned names (nvJitLink.h maps the API onto them)
    void* jl = open_toolkit("libnvJitLink.so.12", {"libnvJitLink.so.12", "libnvJitLink.so"});
    if (!jl) {
        a.link_why = "nvJitLink (libnvJitLink.so.12) not found";
    } else if (sym(jl, "__nvJitLinkCreate_12_9", a.LinkCreate) && sym(jl, "__nvJitLinkDestroy_12_9", a.LinkDestroy) &&
               sym(jl, "__nvJitLinkAddData_12_9", a.LinkAddData) &&
               sym(jl, "__nvJitLinkComplete_12_9", a.LinkComplete) &&
               sym(jl, "__nvJitLinkGetLinkedCubinSize_12_9", a.LinkedCubinSize) &&
               sym(jl, "__nvJitLinkGetLinkedCubin_12_9", a.LinkedCubin) &&
               sym(jl, "__nvJitLinkGetErrorLogSize_12_9", a.LinkErrorLogSize) &&
               sym(jl, "__nvJitLinkGetErrorLog_12_9", a.LinkErrorLog)) {
        a.link_ok = true;
    } else {
        a.link_why = "nvJitLink 12.9 entry points missing";
    }
    void* cu = dlopen("libcuda.so.1", RTLD_NOW | RTLD_LOCAL);
    if (!cu) {
        a.cu_why = "CUDA driver library (libcuda.so.1) not found";
    } else if (sym(cu, "cuModuleLoadData", a.ModuleLoadData) && sym(cu, "cuModuleUnload", a.ModuleUnload) &&
               sym(cu, "cuModuleGetFunction", a.ModuleGetFunction) && sym(cu, "cuLaunchKernel", a.LaunchKernel) &&
               sym(cu, "cuFuncSetAttribute", a.FuncSetAttribute)) {
        a.cu_ok = true;
        if (!sym(cu, "cuCtxGetCurrent", a.CtxGetCurrent) || !sym(cu, "cuCtxGetId", a.CtxGetId))
            a.CtxGetCurrent = nullptr, a.CtxGetId = nullptr;
    } else {
        a.cu_why = "CUDA driver entry points missing";
    }
}

Api& api() {
    std::call_once(g_api_once, load_api);
    return g_api;
}

// Loaded modules shared between the handles of a process: handles of the
// same problem (a second starmap_solver call, the instances of an ensemble)
// run identical generated code, and loading it again costs milliseconds per
// program.  Keyed by the context and the cubin's size and two hashes;
// reference-counted, unloaded with the last user.
struct ModEntry {
    CUmodule_t mod;
    int refs;
};
std::map<std::tuple<unsigned long long, size_t, unsigned long long, unsigned long long>, ModEntry> g_mods;
std::mutex g_mods_mu;

// Word-at-a-time multiply-xorshift hash of a cubin (megabytes for hundreds of
// moments: a byte-serial hash would cost milliseconds per new handle).
unsigned long long bytes_hash(const std::vector<char>& v, unsigned long long h, unsigned long long mul) {
    const size_t nw = v.size() / 8;
    for (size_t i = 0; i < nw; ++i) {
        unsigned long long w;
        std::memcpy(&w, v.data() + 8 * i, 8);
        h = (h ^ w) * mul;
        h ^= h >> 29;
    }
    for (size_t i = 8 * nw; i < v.size(); ++i) h = (h ^ (unsigned char)v[i]) * mul;
    return h;
}

int load_module(const std::vector<char>& cubin, CUmodule_t* m) {
    Api& a = api();
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (!a.CtxGetCurrent || a.CtxGetCurrent(&ctx) != 0 || !ctx || a.CtxGetId(ctx, &id) != 0)
        return a.ModuleLoadData(m, cubin.data()) == 0 ? 0 : -1;   // no context id: not shared
    const auto key = std::make_tuple(id, cubin.size(), bytes_hash(cubin, 1469598103934665603ull, 0x9e3779b97f4a7c15ull),
                                     bytes_hash(cubin, 0x243f6a8885a308d3ull, 0xff51afd7ed558ccdull));
    std::lock_guard<std::mutex> lk(g_mods_mu);
    auto it = g_mods.find(key);
    if (it != g_mods.end()) {
        ++it->second.refs;
        *m = it->second.mod;
        return 0;
    }
    if (a.ModuleLoadData(m, cubin.data()) != 0) return -1;
    g_mods[key] = ModEntry{*m, 1};
    return 0;
}

void release_module(CUmodule_t m) {
    {
        std::lock_guard<std::mutex> lk(g_mods_mu);
        for (auto it = g_mods.begin(); it != g_mods.end(); ++it)
            if (it->second.mod == m) {
                if (--it->second.refs == 0) {
                    api().ModuleUnload(m);
                    g_mods.erase(it);
                }
                return;
            }
    }
    api().ModuleUnload(m);   // loaded without sharing
}

// ---- source generation -------------------------------------------------------
const char* kPrelude = R"(
struct DevField { const double* p; double s; };
struct FamGeom { double* U; const DevField* F; int n[4]; long long s1, s2, cs; double h[3]; double rh[3]; double hdt; };
static __device__ __forceinline__ double ld1(const double* p) { return __ldg(p); }
static __device__ __forceinline__ double2 ld2(const double* p) { return __ldg(reinterpret_cast<const double2*>(p)); }
// correctly rounded d/h from y = RN(1/h): one or two Markstein correction
// steps (the mode is chosen per axis on the host), or IEEE division
static __device__ __forceinline__ double div2(double d, double h, double y) {
    const double q = __dmul_rn(d, y);
    const double r = __fma_rn(-q, h, d);
    return __fma_rn(r, y, q);
}
static __device__ __forceinline__ double div1(double d, double h, double y) {
    double q = __dmul_rn(d, y);
    const double r0 = __fma_rn(-q, h, d);
    q = __fma_rn(r0, y, q);
    const double r = __fma_rn(-q, h, d);
    return __fma_rn(r, y, q);
}
static __device__ __forceinline__ double div0(double d, double h, double y) { return __ddiv_rn(d, h); }
// U + (dt/2)*(W + Q - s.*U).*E in MATLAB's evaluation order
static __device__ __forceinline__ double upd(double u, double W, double q, double s, double E, double hdt) {
    const double t1 = __dadd_rn(W, q);
    const double t2 = __dmul_rn(s, u);
    const double t3 = __dsub_rn(t1, t2);
    const double t4 = __dmul_rn(hdt, t3);
    const double t5 = __dmul_rn(t4, E);
    return __dadd_rn(u, t5);
}
static __device__ __forceinline__ void stencil(int p, int n, int bc, int g2, int& hi, int& lo) {
    if (!g2) {
        if (bc) { hi = p < n - 1 ? p : n - 1; lo = p > 0 ? p - 1 : 0; }
        else    { hi = (p + 1 == n) ? 0 : p + 1; lo = p; }
    } else {
        if (bc) { hi = p + 1; lo = p; }
        else    { hi = p; lo = (p == 0) ? n - 1 : p - 1; }
    }
}
static __device__ __forceinline__ const double* fp(const DevField* F, int i) {
    return reinterpret_cast<const double*>(__ldg(reinterpret_cast<const unsigned long long*>(&F[i].p)));
}
static __device__ __forceinline__ double fs(const DevField* F, int i) { return __ldg(&F[i].s); }
// request a line into L2 ahead of its load (no register, no wait)
static __device__ __forceinline__ void pf(const void* p) { asm volatile("prefetch.global.L2 [%0];" :: "l"(p)); }
// request a contiguous range into L2 with the bulk copy engine (16-byte
// aligned, a multiple of 16 bytes; no register, no shared memory, no wait)
static __device__ __forceinline__ void l2pf(const double* p, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(p), "r"(bytes) : "memory");
}
// the numerator of the sigma-gradient factor of a destination's phase (one
// substep: M = 1, two: M = 2, F1 the first substep's filter) from its value
// before the phase u and coupling sum w: the adjoint sweep divides it by E
// (M = 1) or multiplies it by its own den (M = 2) and adds factor * Y to
// dJ/dsigma -- the expressions of the sweep's evaluation from recorded u and w
static __device__ __forceinline__ double dsdw(int M, double u, double w, double s, double E, double q, double F1,
                                              double dE, double hdt) {
    if (M == 1) return -u * E + (w + q - s * u) * dE;
    const double r = 1.0 - hdt * s * E;
    const double G0 = w + q - s * u;
    const double V1 = F1 * (u + hdt * G0 * E);
    const double G1 = w + q - s * V1;
    return r * F1 * hdt * (-u * E + G0 * dE) + hdt * (-V1 * E + G1 * dE);
}
)";

// Helpers of the generated adjoint kernels: D^T of a staggered difference
// (preimages of hi and lo under the stencil of starmap_solver.m:127-132), per
// point (x) and for a row pair (y/z, one 128-bit load serves both points).
const char* kAdjPrelude = R"(
static __device__ __forceinline__ double dT(const double* v, int q, int n, int bc, int g2, long long st) {
    if (!g2) {
        if (bc) {
            double a = v[0];
            if (q == n - 1) a += v[st];
            double b = v[st];
            if (q == 0) b += v[0];
            return a - b;
        }
        const long long om = (q == 0) ? (long long)(n - 1) * st : -st;
        return v[om] - v[0];
    }
    if (bc) {
        const double a = q >= 1 ? v[-st] : 0.0;
        const double b = q <= n - 1 ? v[0] : 0.0;
        return a - b;
    }
    const long long op = (q == n - 1) ? -(long long)(n - 1) * st : st;
    return v[0] - v[op];
}
static __device__ __forceinline__ double2 L2(const double* p) { return *reinterpret_cast<const double2*>(p); }
static __device__ __forceinline__ double2 S2(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
static __device__ __forceinline__ double2 A2(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
static __device__ __forceinline__ double2 dT_row(const double* v, int q, int n, int bc, int g2, long long st) {
    const double2 z = make_double2(0.0, 0.0);
    if (!g2) {
        if (bc) {
            double2 a = L2(v);
            if (q == n - 1) a = A2(a, L2(v + st));
            double2 b = L2(v + st);
            if (q == 0) b = A2(b, L2(v));
            return S2(a, b);
        }
        const long long om = (q == 0) ? (long long)(n - 1) * st : -st;
        return S2(L2(v + om), L2(v));
    }
    if (bc) {
        const double2 a = q >= 1 ? L2(v - st) : z;
        const double2 b = q <= n - 1 ? L2(v) : z;
        return S2(a, b);
    }
    const long long op = (q == n - 1) ? -(long long)(n - 1) * st : st;
    return S2(L2(v), L2(v + op));
}
// phase's pointwise adjoint from Y = (dU'/dW) lambda' (one substep: M = 1,
// two: M = 2; F1 the first substep's filter): returns lambda = (dU'/dU)
// lambda', adds the sigma-gradient contribution to ds and the source
// gradient to gq (dU'/dQ = dU'/dW)
static __device__ __forceinline__ double pend(int M, double u, double w, double Y, double s, double E, double q,
                                              double F1, double dE, double& ds, double* gq, int pt, double hdt) {
    const double r = 1.0 - hdt * s * E;
    double rho, dsdw;
    if (M == 1) {
        rho = r / (hdt * E);
        dsdw = (-u * E + (w + q - s * u) * dE) / E;
    } else {
        const double den = 1.0 / (hdt * E * (r * F1 + 1.0));
        rho = F1 * r * r * den;
        const double G0 = w + q - s * u;
        const double V1 = F1 * (u + hdt * G0 * E);
        const double G1 = w + q - s * V1;
        dsdw = (r * F1 * hdt * (-u * E + G0 * dE) + hdt * (-V1 * E + G1 * dE)) * den;
    }
    ds += dsdw * Y;
    if (gq) atomicAdd(gq + pt, Y);
    return rho * Y;
}
// the same with the numerator N of the sigma-gradient factor recorded by the
// forward (dsdw)
static __device__ __forceinline__ double pend_ds(int M, double N, double Y, double s, double E, double F1, double& ds,
                                                 double* gq, int pt, double hdt) {
    const double r = 1.0 - hdt * s * E;
    double rho, D;
    if (M == 1) {
        rho = r / (hdt * E);
        D = N / E;
    } else {
        const double den = 1.0 / (hdt * E * (r * F1 + 1.0));
        rho = F1 * r * r * den;
        D = N * den;
    }
    ds += D * Y;
    if (gq) atomicAdd(gq + pt, Y);
    return rho * Y;
}
// dU'/dW of a destination (F1 first, F2 last substep filter)
static __device__ __forceinline__ double dwdu(int M, double s, double E, double F1, double F2, double hdt) {
    if (M == 1) return F1 * hdt * E;
    const double r = 1.0 - hdt * s * E;
    return F2 * hdt * E * (r * F1 + 1.0);
}
)";

// Helpers of the bulk-staged kernels: mbarriers in shared memory, the bulk
// copy engine (cp.async.bulk, global -> this CTA's shared memory, completion
// counted in bytes on an mbarrier; no cluster multicast), and bounded waits.
const char* kStagePrelude = R"(
static __device__ __forceinline__ unsigned sa(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
static __device__ __forceinline__ void mb_init(unsigned long long* b, unsigned n) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(sa(b)), "r"(n) : "memory");
}
static __device__ __forceinline__ void mb_expect(unsigned long long* b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(sa(b)), "r"(bytes) : "memory");
}
static __device__ __forceinline__ void mb_arrive(unsigned long long* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(sa(b)) : "memory");
}
static __device__ __forceinline__ bool mb_try(unsigned long long* b, unsigned parity) {
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok) : "r"(sa(b)), "r"(parity) : "memory");
    return ok != 0;
}
static __device__ __forceinline__ unsigned long long gtime() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// wait for the phase of parity `parity` to complete; false after 4 s (the
// caller records the failure in the error flag and stops)
static __device__ __forceinline__ bool mb_wait(unsigned long long* b, unsigned parity) {
    if (mb_try(b, parity)) return true;
    const unsigned long long t0 = gtime();
    for (unsigned n = 1;; ++n) {
        if (mb_try(b, parity)) return true;
        if ((n & 255u) == 0 && gtime() - t0 > 4000000000ull) return false;
    }
}
static __device__ __forceinline__ void bulk_ld(double* dst, const double* src, unsigned bytes, unsigned long long* b) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(sa(dst)), "l"(src), "r"(bytes), "r"(sa(b)) : "memory");
}
static __device__ __forceinline__ double2 lds2(const double* p) { return *reinterpret_cast<const double2*>(p); }
// 16-byte asynchronous copy global -> shared (cached in L2 only), its group
// commit and the wait for all but the newest N groups of this thread
static __device__ __forceinline__ void cpa(double* dst, const double* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(sa(dst)), "l"(src) : "memory");
}
static __device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// the same, cached in L1 as well, 16 or 8 bytes
static __device__ __forceinline__ void cpa16(double2* dst, const double* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" :: "r"(sa(dst)), "l"(src) : "memory");
}
static __device__ __forceinline__ void cpa8(double* dst, const double* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" :: "r"(sa(dst)), "l"(src) : "memory");
}
template <int N> static __device__ __forceinline__ void cpa_wait() {
    asm volatile("cp.async.wait_group %0;" :: "n"(N) : "memory");
}
// the four values of an x difference for a point pair: from two aligned
// 128-bit shared loads in the interior (pattern A: stencil (p, p-1), B:
// (p+1, p)), from shared memory at the stencil offsets where the stencil
// clamps, or from global memory where it wraps out of the staged window
static __device__ __forceinline__ void xvals(int patA, const double* s, const double* g, bool xf, bool xw, int h0,
                                             int l0, int h1, int l1, double& a0, double& b0, double& a1, double& b1) {
    if (xf) {
        const double2 P = lds2(s);
        if (patA) { const double2 Q = lds2(s - 2); a0 = P.x; b0 = Q.y; a1 = P.y; b1 = P.x; }
        else { const double2 R = lds2(s + 2); a0 = P.y; b0 = P.x; a1 = R.x; b1 = P.y; }
    } else if (xw) {
        a0 = s[h0]; b0 = s[l0]; a1 = s[h1]; b1 = s[l1];
    } else {
        a0 = __ldg(g + h0); b0 = __ldg(g + l0); a1 = __ldg(g + h1); b1 = __ldg(g + l1);
    }
}
)";

std::string lit(double v) {
    // exact value as a C++17 hexadecimal floating literal
    char buf[64];
    if (v == 0.0) return std::signbit(v) ? "(-0.0)" : "0.0";
    std::snprintf(buf, sizeof buf, "(%a)", v);
    return buf;
}

// Constant table of the program being emitted (null: literals in the code).
// With a table, coupling weights and grid constants are read from
// __constant__ memory, which the FP64 instructions take as an operand,
// instead of being built in registers from immediates.
struct ConstTable {
    std::vector<double> v;
    std::map<unsigned long long, int> at;
};
thread_local ConstTable* g_ctab = nullptr;

std::string clit(double v) {
    if (!g_ctab) return lit(v);
    unsigned long long bits;
    std::memcpy(&bits, &v, sizeof bits);
    auto it = g_ctab->at.find(bits);
    int i;
    if (it != g_ctab->at.end()) i = it->second;
    else {
        i = (int)g_ctab->v.size();
        g_ctab->v.push_back(v);
        g_ctab->at[bits] = i;
    }
    return "kC[" + std::to_string(i) + "]";
}

std::string ctab_decl(const ConstTable& t) {
    if (t.v.empty()) return "";
    std::string o = "__constant__ double kC[" + std::to_string(t.v.size()) + "] = {";
    for (size_t i = 0; i < t.v.size(); ++i) o += (i ? ", " : "") + lit(t.v[i]);
    return o + "};\n";
}

struct Coefs {
    int q, s, E, F1, F2;
};

Coefs coefs_of(const smg_handle* h, int phase, int j) {
    const smg::DevComp& c = h->comps[j];
    Coefs f;
    if (phase == 1 && j == 0) {
        f.s = h->sigma_a;
        f.E = h->decay_a >= 0 ? h->decay_a : h->derived_decay_a;
        f.F1 = f.F2 = h->field_one;
    } else {
        f.s = c.sT;
        f.E = c.ET;
        f.F1 = c.F1;
        f.F2 = c.F2;
    }
    f.q = c.Q;
    return f;
}

// whether field f is an array (fixed at smg_create: smg_set_field cannot
// change it); the values themselves are read at run time
bool is_array(const smg_handle* h, int f) {
    if (f == h->field_one || f == h->field_zero) return false;
    if (f < h->field_one) return h->field_is_array[f] != 0;
    // device-derived decay of a sigma field: an array when its sigma is
    for (size_t k = 0; k < h->derived_decay.size(); ++k)
        if (h->derived_decay[k] == f) return h->field_is_array[k] != 0;
    return false;
}

// declaration of the values of field f at the two points
std::string coef_decl(const smg_handle* h, int f, const char* n) {
    char b[256];
    if (is_array(h, f))
        std::snprintf(b, sizeof b, "const double2 %s = ld2(fp(F, %d) + pt); ", n, f);
    else
        std::snprintf(b, sizeof b, "const double %s = fs(F, %d); ", n, f);
    return b;
}
std::string cx(const smg_handle* h, int f, const char* n) { return is_array(h, f) ? std::string(n) + ".x" : n; }
std::string cy(const smg_handle* h, int f, const char* n) { return is_array(h, f) ? std::string(n) + ".y" : n; }

// Interior form of the x stencil for a source of grid type g2 (1 or 2 along
// x): pattern A is (hi, lo) = (p, p-1), pattern B (p+1, p).
bool xpattern_a(int g2, int bc) { return g2 == 0 ? bc == 1 : bc == 0; }

// Thread condition under which both points of the pair follow the interior
// form and the extra 128-bit load stays inside the padded row:
//   g2=0 bc=1 (A): 1 <= p <= n-1 for both points, load at x0-2 >= 0
//   g2=1 bc=0 (A): p >= 1, load at x0-2 >= 0
//   g2=0 bc=0 (B): p+1 <= n-1 for both points, load up to x0+3 < s1
//   g2=1 bc=1 (B): every p; load up to x0+3 < s1
// (a second point outside the destination's extent is computed but unused)
std::string xfast_cond(const smg_handle* h, int g2) {
    const int n = h->g.n[0], bc = h->g.bc[0];
    const long long s1 = h->g.s1;
    char b[160];
    if (g2 == 0 && bc == 1) std::snprintf(b, sizeof b, "(x0 >= 2 && x0 + 1 <= %d)", n - 1);
    else if (g2 == 1 && bc == 0) std::snprintf(b, sizeof b, "(x0 >= 2)");
    else if (g2 == 0 && bc == 0) std::snprintf(b, sizeof b, "(x0 + 2 <= %d && x0 + 3 < %lld)", n - 1, s1);
    else std::snprintf(b, sizeof b, "(x0 + 3 < %lld)", s1);
    return b;
}

// One destination's block.  Update modes: 0 one substep with filter kf;
// 1 two substeps (phase B: F1 then F2); 2 fused A(k=2) A(k=1) (F2 then F1).
// Phase A blocks carry modes 0 and 2 (chosen by `mode` at run time), phase B
// blocks mode 1.  Loads of the second point are unconditional: the row pitch
// is a multiple of 8 doubles, so x0+1 lies inside the padded row even where
// the component's extent ends at x0 (that value is unused and not stored).
// rec: also store the coupling sum W and the values before the update into
// slot di of the recording buffers WR / PR (adjoint recording, smg_forward)
void emit_dest(std::string& o, const smg_handle* h, int phase, int j, int di, bool rec) {
    const smg::DevComp& c = h->comps[j];
    const smg::DevGrid& g = h->g;
    char b[4096];
    std::string cond;
    const char* ax[3] = {"x0", "y", "z"};
    for (int a = 0; a < 3; ++a)
        if (c.ext[a] < g.B[a]) {
            if (!cond.empty()) cond += " && ";
            cond += std::string(ax[a]) + " < " + std::to_string(c.ext[a]);
        }
    o += cond.empty() ? "    {\n" : "    if (" + cond + ") {\n";
    const bool v1_always = c.ext[0] % 2 == 0;
    std::snprintf(b, sizeof b,
                      "        double* Uj = U + pt + %lld;\n        const double2 u = *reinterpret_cast<const double2*>(Uj);\n",
                      (long long)j * g.cs);
    o += b;
    // the x stencil of the second point is evaluated only inside the extent
    if (!v1_always)
        o += "        const bool v1 = x1 < " + std::to_string(c.ext[0]) + ";\n";
    const Coefs f = coefs_of(h, phase, j);
    const bool filt = h->filter_mode == SMG_FILTER_SUBSTEP;
    o += "        " + coef_decl(h, f.q, "q") + coef_decl(h, f.s, "s") + coef_decl(h, f.E, "E") + "\n";
    if (filt) o += "        " + coef_decl(h, f.F1, "fk1") + coef_decl(h, f.F2, "fk2") + "\n";
    o += "        double SA = 0.0, SB = 0.0;\n";
    bool first = true;
    for (int q = c.cbeg; q < c.cend; ++q) {
        const smg::DevCoup& cp = h->coups[q];
        const int a = cp.code >> 1, g2 = cp.code & 1;
        const long long so = (long long)cp.src * g.cs;
        const int mode_div = h->exact_recip[a];
        const std::string H = lit(g.h[a]), RH = lit(h->rh[a]), W = lit(cp.w);
        const char* dv = mode_div == 2 ? "div2" : (mode_div == 1 ? "div1" : "div0");
        const char* fold = first ? "SA = tA; SB = tB;" : "SA = __dadd_rn(SA, tA); SB = __dadd_rn(SB, tB);";
        first = false;
        if (a == 0 && !h->jit_xpair) {
            // four 64-bit loads at the thread's stencil offsets
            std::snprintf(b, sizeof b,
                          "        { const double* S = Up + %lld;\n"
                          "          const double a0 = ld1(S + hx0_%d), b0 = ld1(S + lx0_%d), a1 = ld1(S + (%shx1_%d%s)), "
                          "b1 = ld1(S + (%slx1_%d%s));\n"
                          "          const double tA = __dmul_rn(%s(__dsub_rn(a0, b0), %s, %s), %s);\n"
                          "          const double tB = __dmul_rn(%s(__dsub_rn(a1, b1), %s, %s), %s);\n"
                          "          %s }\n",
                          so, g2, g2, v1_always ? "" : "v1 ? ", g2, v1_always ? "" : " : 0", v1_always ? "" : "v1 ? ",
                          g2, v1_always ? "" : " : 0", dv, H.c_str(), RH.c_str(), W.c_str(), dv, H.c_str(), RH.c_str(),
                          W.c_str(), fold);
        } else if (a == 0) {
            // interior: the three values a point pair needs from two aligned
            // 128-bit loads (pattern A: p-1, p, p+1 -> loads at x0-2 and x0;
            // pattern B: x0, x0+1, x0+2 -> loads at x0 and x0+2); threads
            // where the stencil is not the interior one (xf_g2 false) use it
            const bool patA = xpattern_a(g2, g.bc[0]);
            const std::string fast = patA
                ? "const double2 P = ld2(S), Q = ld2(S - 2); a0 = P.x; b0 = Q.y; a1 = P.y; b1 = P.x;"
                : "const double2 P = ld2(S), R = ld2(S + 2); a0 = P.y; b0 = P.x; a1 = R.x; b1 = P.y;";
            std::snprintf(b, sizeof b,
                          "        { const double* S = Up + %lld; double a0, b0, a1, b1;\n"
                          "          if (xf_%d) { %s }\n"
                          "          else { int hi, lo; stencil(x0, %d, %d, %d, hi, lo); a0 = ld1(S + (hi - x0)); "
                          "b0 = ld1(S + (lo - x0));\n"
                          "                 if (%s) { stencil(x1, %d, %d, %d, hi, lo); a1 = ld1(S + (hi - x0)); "
                          "b1 = ld1(S + (lo - x0)); } else { a1 = b1 = 0.0; } }\n"
                          "          const double tA = __dmul_rn(%s(__dsub_rn(a0, b0), %s, %s), %s);\n"
                          "          const double tB = __dmul_rn(%s(__dsub_rn(a1, b1), %s, %s), %s);\n"
                          "          %s }\n",
                          so, g2, fast.c_str(), g.n[0], g.bc[0], g2, v1_always ? "true" : "v1", g.n[0], g.bc[0], g2,
                          dv, H.c_str(), RH.c_str(), W.c_str(), dv, H.c_str(), RH.c_str(), W.c_str(), fold);
        } else {
            const char* n = a == 1 ? "y" : "z";
            std::snprintf(b, sizeof b,
                          "        { const double* S = Up + %lld;\n"
                          "          const double2 hv = ld2(S + h%s_%d), lv = ld2(S + l%s_%d);\n"
                          "          const double tA = __dmul_rn(%s(__dsub_rn(hv.x, lv.x), %s, %s), %s);\n"
                          "          const double tB = __dmul_rn(%s(__dsub_rn(hv.y, lv.y), %s, %s), %s);\n"
                          "          %s }\n",
                          so, n, g2, n, g2, dv, H.c_str(), RH.c_str(), W.c_str(), dv, H.c_str(), RH.c_str(),
                          W.c_str(), fold);
        }
        o += b;
    }
    const std::string q0 = cx(h, f.q, "q"), q1 = cy(h, f.q, "q"), s0 = cx(h, f.s, "s"), s1 = cy(h, f.s, "s"),
                      E0 = cx(h, f.E, "E"), E1 = cy(h, f.E, "E");
    const std::string k10 = cx(h, f.F1, "fk1"), k11 = cy(h, f.F1, "fk1"), k20 = cx(h, f.F2, "fk2"),
                      k21 = cy(h, f.F2, "fk2");
    auto substep = [&]() {
        std::snprintf(b, sizeof b, "u0 = upd(u0, -SA, %s, %s, %s, hdt); u1 = upd(u1, -SB, %s, %s, %s, hdt);",
                      q0.c_str(), s0.c_str(), E0.c_str(), q1.c_str(), s1.c_str(), E1.c_str());
        return std::string(b);
    };
    auto filter = [&](const std::string& a0, const std::string& a1) {
        return filt ? " u0 = __dmul_rn(u0, " + a0 + "); u1 = __dmul_rn(u1, " + a1 + ");" : std::string();
    };
    o += "        double u0 = u.x, u1 = u.y;\n";
    if (rec) {
        const long long so = (long long)di * g.cs;
        std::snprintf(b, sizeof b,
                      "        { double* wp = WR + pt + %lld; double* pp = PR + pt + %lld;\n"
                      "          if (%s) { *reinterpret_cast<double2*>(wp) = make_double2(-SA, -SB); "
                      "*reinterpret_cast<double2*>(pp) = u; } else { wp[0] = -SA; pp[0] = u.x; } }\n",
                      so, so, v1_always ? "true" : "v1");
        o += b;
    }
    if (phase == 0) {
        const std::string one = "        " + substep() +
                                (filt ? " u0 = __dmul_rn(u0, kf == 1 ? " + k10 + " : " + k20 +
                                            "); u1 = __dmul_rn(u1, kf == 1 ? " + k11 + " : " + k21 + ");"
                                      : std::string()) +
                                "\n";
        const std::string two = "        " + substep() + filter(k20, k21) + "\n        " + substep() +
                                filter(k10, k11) + "\n";
        if (h->filter_mode == SMG_FILTER_FULL) o += one;
        else o += "        if (mode == 0) {\n" + one + "        } else {\n" + two + "        }\n";
    } else {
        o += "        " + substep() + filter(k10, k11) + "\n        " + substep() + filter(k20, k21) + "\n";
    }
    if (v1_always) o += "        *reinterpret_cast<double2*>(Uj) = make_double2(u0, u1);\n";
    else o += "        if (v1) *reinterpret_cast<double2*>(Uj) = make_double2(u0, u1); else *Uj = u0;\n";
    o += "    }\n";
}

// __launch_bounds__ arguments: the CTA size and, with a register limit per
// thread (regs > 0), the resident CTAs per SM that this limit allows (the
// bound takes precedence over --maxrregcount for kernels)
std::string bounds(int block, int regs) {
    if (regs <= 0) return std::to_string(block);
    return std::to_string(block) + ", " + std::to_string(std::max(1, 65536 / (block * regs)));
}

std::string group_name(int phase, int k) { return "smg_g" + std::to_string(phase) + "_" + std::to_string(k); }
// U and R are the same state pointer: the destinations are read and written
// through U, the sources only read through R.  A phase never writes its
// sources, so the two restrict-qualified names never touch one object that is
// modified, and the compiler may move a later destination's source loads
// above an earlier destination's store.
std::string group_args(bool rec) {
    return std::string("(double* __restrict__ U, const double* __restrict__ R, const DevField* __restrict__ F, double hdt, "
                       "int kf, int mode, int x0, "
                       "int y, int z, bool act") +
           (rec ? ", double* __restrict__ WR, double* __restrict__ PR, const DevField* __restrict__ DE, int dsm, "
                  "int dsw)"
                : ")");
}

// device function of one group: the thread's stencil offsets, then the blocks
// (inl: a function inlined into the dispatch kernel of the same program;
// otherwise an external function called from it)
void emit_group(std::string& o, const smg_handle* h, int phase, int k, const std::vector<int>& D, int group, bool inl,
                bool rec) {
    const smg::DevGrid& g = h->g;
    char b[1024];
    const int d0 = k * group, d1 = std::min<int>((k + 1) * group, (int)D.size());
    o += std::string(inl ? "static __device__ __forceinline__ void " : "extern \"C\" __device__ __noinline__ void ") +
         group_name(phase, k) + group_args(rec) + " {\n";
    std::snprintf(b, sizeof b,
                  "    const int x1 = x0 + 1;\n"
                  "    const int pt = z * %lld + y * %lld + x0;\n"
                  "    const double* Up = R + pt;\n"
                  "    (void)x1; (void)kf; (void)mode; (void)hdt; (void)Up; (void)act;\n",
                  (long long)g.s2, (long long)g.s1);
    o += b;
    bool used[3] = {false, false, false};
    for (int i = d0; i < d1; ++i)
        for (int q = h->comps[D[i]].cbeg; q < h->comps[D[i]].cend; ++q) used[h->coups[q].code >> 1] = true;
    if (used[0] && h->jit_xpair)
        for (int g2 = 0; g2 < 2; ++g2) o += "    const bool xf_" + std::to_string(g2) + " = " + xfast_cond(h, g2) + ";\n";
    if (used[0] && !h->jit_xpair)
        for (int g2 = 0; g2 < 2; ++g2) {
            std::snprintf(b, sizeof b,
                          "    int hx0_%d, lx0_%d, hx1_%d, lx1_%d;\n"
                          "    { int hi, lo; stencil(x0, %d, %d, %d, hi, lo); hx0_%d = hi - x0; lx0_%d = lo - x0;\n"
                          "      stencil(x1, %d, %d, %d, hi, lo); hx1_%d = hi - x0; lx1_%d = lo - x0; }\n",
                          g2, g2, g2, g2, g.n[0], g.bc[0], g2, g2, g2, g.n[0], g.bc[0], g2, g2, g2);
            o += b;
        }
    const char* an[3] = {"x", "y", "z"};
    for (int a = 1; a < 3; ++a) {
        if (!used[a]) continue;
        const long long st = a == 1 ? g.s1 : g.s2;
        const char* p = a == 1 ? "y" : "z";
        for (int g2 = 0; g2 < 2; ++g2) {
            std::snprintf(b, sizeof b,
                          "    int h%s_%d, l%s_%d;\n"
                          "    { int hi, lo; stencil(%s, %d, %d, %d, hi, lo); h%s_%d = (hi - %s) * %lld; "
                          "l%s_%d = (lo - %s) * %lld; }\n",
                          an[a], g2, an[a], g2, p, g.n[a], g.bc[a], g2, an[a], g2, p, st, an[a], g2, p, st);
            o += b;
        }
    }
    for (int i = d0; i < d1; ++i) emit_dest(o, h, phase, D[i], i, rec);
    o += "}\n";
}

// kernel over groups [k0, k1) of one phase type: CTA -> (group, row, chunk),
// then the group's code (inlined, or a call when the groups are compiled
// separately)
// Rows per band of the CTA order (0: group-major).  By default group-major
// order, in which each group streams its sources over the whole grid, is
// kept while a component slot is under 4 MB: the groups that run at the same
// time then reuse shared sources in L2.  With larger slots (3D grids) a
// group's sources no longer stay in L2 for the next group, so the CTAs go
// band by band, the band sized so that all components' rows of a band take
// about 48 MB (0.4 of the L2).
int band_rows(const smg_handle* h) {
    if (h->jit_band >= 0) return h->jit_band;
    const double slot = (double)h->g.cs * 8;
    if (slot < 4.0 * (1 << 20)) return 0;
    const long long rows = (long long)h->g.B[1] * h->g.B[2];
    const double row_all = (double)h->n_sys * h->g.s1 * 8;
    return (int)std::max(1LL, std::min(rows, (long long)(48.0 * (1 << 20) / row_all)));
}

void emit_dispatch(std::string& o, const smg_handle* h, int phase, int k0, int k1, int block, bool inl,
                   const std::string& name, bool rec) {
    const smg::DevGrid& g = h->g;
    const int tpr = (g.B[0] + 1) / 2;
    const int nchunks = (tpr + block - 1) / block;
    const long long per = (long long)nchunks * g.B[1] * g.B[2];
    char b[1024];
    if (!inl)
        for (int k = k0; k < k1; ++k) o += "extern \"C\" __device__ void " + group_name(phase, k) + group_args(rec) + ";\n";
    // CTA order: group-major (every row of a group, then the next group), or,
    // with bands of R rows, band-major (every group of the kernel on R rows,
    // then the next band), so that the source rows a band needs stay in L2
    // while all groups use them
    const int R = inl ? band_rows(h) : 0;
    const long long rows = (long long)g.B[1] * g.B[2];
    std::string map;
    if (R > 0) {
        const long long per_band = (long long)(k1 - k0) * R * nchunks;
        std::snprintf(b, sizeof b,
                      "    const int band = bid / %lld, r0 = bid - band * %lld;\n"
                      "    const int grp = %d + r0 / %d, r1 = r0 %% %d;\n"
                      "    const int row = band * %d + r1 / %d, chunk = r1 %% %d;\n"
                      "    if (row >= %lld) return;\n",
                      per_band, per_band, k0, R * nchunks, R * nchunks, R, nchunks, nchunks, rows);
    } else {
        std::snprintf(b, sizeof b,
                      "    const int grp = %d + bid / %lld;\n"
                      "    const int rest = bid %% %lld;\n"
                      "    const int row = rest / %d, chunk = rest - row * %d;\n",
                      k0, per, per, nchunks, nchunks);
    }
    map = b;
    std::snprintf(b, sizeof b,
                  "extern \"C\" __global__ void __launch_bounds__(%s) %s(double* __restrict__ U, "
                  "const DevField* __restrict__ F, double hdt, int kf, int mode%s) {\n"
                  "    const int bid = blockIdx.x;\n"
                  "%s"
                  "    const int y = row %% %d, z = row / %d;\n"
                  "    int x0 = 2 * (chunk * %d + (int)threadIdx.x);\n"
                  "    const bool act = x0 < %d;\n"
                  "    %s\n"
                  "    switch (grp) {\n",
                  bounds(block, h->jit_regs).c_str(), name.c_str(),
                  rec ? ", double* __restrict__ WR, double* __restrict__ PR, const DevField* __restrict__ DE, int dsm, "
                        "int dsw"
                      : "",
                  map.c_str(), g.B[1], g.B[1],
                  block, g.B[0],
                  // with x differences from lane shuffles every lane of a warp takes part:
                  // lanes past the row compute on the last pair and store nothing
                  (h->jit_xpair == 2 && inl) ? ("if (!act) x0 = " + std::to_string((g.B[0] - 1) & ~1) + ";").c_str()
                                             : "if (!act) return;");
    o += b;
    for (int k = k0; k < k1; ++k)
        o += "    case " + std::to_string(k) + ": " + group_name(phase, k) + "(U, U, F, hdt, kf, mode, x0, y, z, act" +
             (rec ? ", WR, PR, DE, dsm, dsw" : "") + "); break;\n";
    o += "    default: break;\n    }\n}\n";
}

// destinations of a phase in the pair tables' order (breadth-first levels)
std::vector<int> phase_dests(const smg_handle* h, int phase) {
    std::vector<int> D;
    for (const auto& d : h->pair[phase].dests) D.push_back((int)((long long)d.off / h->g.cs));
    if (D.empty()) D = phase == 0 ? h->destA : h->destB;
    return D;
}

// ---- groups that share loads (the inline layout) ----------------------------
// Destinations of one phase are grouped by grid type (one extent condition per
// group) and, within a grid type, greedily by the (axis, source) pairs of
// their couplings, so that the destinations of a group read many of the same
// source rows.  The group's code loads every distinct source value and
// coefficient once, at its first use, and later destinations reuse the
// register: a phase never writes its sources, so a value loaded before an
// earlier destination's store is still current.
std::vector<std::vector<int>> shared_groups(const smg_handle* h, int phase, int group) {
    const std::vector<int> D = phase_dests(h, phase);
    // the distinct (axis, source) keys of each destination, as ids axis*n_sys+src
    std::vector<std::vector<int>> K(D.size());
    std::map<std::vector<int>, std::vector<int>> by_ext;   // extents -> positions in D
    std::vector<std::vector<int>> order;
    for (size_t p = 0; p < D.size(); ++p) {
        const smg::DevComp& c = h->comps[D[p]];
        for (int q = c.cbeg; q < c.cend; ++q) K[p].push_back((h->coups[q].code >> 1) * h->n_sys + h->coups[q].src);
        std::sort(K[p].begin(), K[p].end());
        K[p].erase(std::unique(K[p].begin(), K[p].end()), K[p].end());
        std::vector<int> e(c.ext, c.ext + 3);
        if (!by_ext.count(e)) order.push_back(e);
        by_ext[e].push_back((int)p);
    }
    std::vector<std::vector<int>> G;
    std::vector<char> in(3 * (size_t)h->n_sys, 0);   // keys of the group being built
    for (const auto& e : order) {
        std::vector<int> left = by_ext[e];
        while (!left.empty()) {
            std::vector<int> g{left.front()};
            left.erase(left.begin());
            std::fill(in.begin(), in.end(), 0);
            for (int k : K[g[0]]) in[k] = 1;
            while ((int)g.size() < group && !left.empty()) {
                size_t best = 0;
                int bestn = -1;
                for (size_t i = 0; i < left.size(); ++i) {
                    int n = 0;
                    for (int k : K[left[i]]) n += in[k];
                    if (n > bestn) {
                        bestn = n;
                        best = i;
                    }
                }
                g.push_back(left[best]);
                for (int k : K[left[best]]) in[k] = 1;
                left.erase(left.begin() + best);
            }
            G.push_back(std::move(g));
        }
    }
    // groups in the order of their destinations' coupling-graph levels (the
    // destination list is level-sorted), so that groups running at the same
    // time, in one kernel or in the concurrent kernels of the phase, read
    // overlapping sources while these are in L2
    std::stable_sort(G.begin(), G.end(), [](const std::vector<int>& a, const std::vector<int>& b) {
        long long sa = 0, sb = 0;
        for (int p : a) sa += p;
        for (int p : b) sb += p;
        return sa * (long long)b.size() < sb * (long long)a.size();
    });
    return G;
}

// one group's device function (inline layout): positions P into the phase's
// destination list (the position is the destination's recording slot)
void emit_shared_group(std::string& o, const smg_handle* h, int phase, int k, const std::vector<int>& P, bool rec,
                       bool fam = false, const std::vector<int>* nextP = nullptr) {
    const smg::DevGrid& g = h->g;
    const std::vector<int> D = phase_dests(h, phase);
    char b[4096];
    if (fam) {
        // family form: the geometry (extents, pitches, spacings, component
        // stride, coefficient table) comes from the instance's FamGeom
        rec = false;
        o += "static __device__ __forceinline__ void " + group_name(phase, k) +
             "(const FamGeom& G, int kf, int mode, int x0, int y, int z) {\n"
             "    double* U = G.U; const DevField* F = G.F; const double hdt = G.hdt;\n"
             "    const int N0 = G.n[0], N1 = G.n[1], N2 = G.n[2];\n"
             "    const long long S1 = G.s1, S2 = G.s2, CS = G.cs;\n"
             "    const double H0 = G.h[0], H1 = G.h[1], H2 = G.h[2], RH0 = G.rh[0], RH1 = G.rh[1], RH2 = G.rh[2];\n"
             "    (void)N0; (void)N1; (void)N2; (void)S1; (void)S2; (void)H0; (void)H1; (void)H2; (void)RH0; (void)RH1; "
             "(void)RH2;\n"
             "    const int x1 = x0 + 1;\n"
             "    const long long pt = z * S2 + y * S1 + x0;\n"
             "    const double* Up = U + pt;\n"
             "    (void)x1; (void)kf; (void)mode; (void)Up;\n";
    } else {
        o += "static __device__ __forceinline__ void " + group_name(phase, k) + group_args(rec) + " {\n";
        std::snprintf(b, sizeof b,
                      "    const int x1 = x0 + 1;\n"
                      "    const int pt = z * %lld + y * %lld + x0;\n"
                      "    const double* Up = R + pt;\n"
                      "    (void)x1; (void)kf; (void)mode; (void)hdt; (void)Up; (void)act;\n",
                      (long long)g.s2, (long long)g.s1);
        o += b;
    }
    // extents, pitches and component offsets: literals, or the family's
    // run-time values
    auto N = [&](int a) { return fam ? "N" + std::to_string(a) : std::to_string(g.n[a]); };
    auto off = [&](int comp) {
        return fam ? "(long long)" + std::to_string(comp) + " * CS" : std::to_string((long long)comp * g.cs);
    };
    bool used[3] = {false, false, false};
    for (int p : P)
        for (int q = h->comps[D[p]].cbeg; q < h->comps[D[p]].cend; ++q) used[h->coups[q].code >> 1] = true;
    if (used[0])
        for (int g2 = 0; g2 < 2; ++g2) {
            std::snprintf(b, sizeof b,
                          "    int hx0_%d, lx0_%d, hx1_%d, lx1_%d;\n"
                          "    { int hi, lo; stencil(x0, %s, %d, %d, hi, lo); hx0_%d = hi - x0; lx0_%d = lo - x0;\n"
                          "      stencil(x1, %s, %d, %d, hi, lo); hx1_%d = hi - x0; lx1_%d = lo - x0; }\n",
                          g2, g2, g2, g2, N(0).c_str(), g.bc[0], g2, g2, g2, N(0).c_str(), g.bc[0], g2, g2, g2);
            o += b;
        }
    const char* an[3] = {"x", "y", "z"};
    for (int a = 1; a < 3; ++a) {
        if (!used[a]) continue;
        const std::string st = fam ? (a == 1 ? "S1" : "S2") : std::to_string(a == 1 ? g.s1 : g.s2);
        const char* pp = a == 1 ? "y" : "z";
        for (int g2 = 0; g2 < 2; ++g2) {
            std::snprintf(b, sizeof b,
                          "    int h%s_%d, l%s_%d;\n"
                          "    { int hi, lo; stencil(%s, %s, %d, %d, hi, lo); h%s_%d = (int)((hi - %s) * %s); "
                          "l%s_%d = (int)((lo - %s) * %s); }\n",
                          an[a], g2, an[a], g2, pp, N(a).c_str(), g.bc[a], g2, an[a], g2, pp, st.c_str(), an[a], g2,
                          pp, st.c_str());
            o += b;
        }
    }
    // the group's extent condition (all its destinations share a grid); with
    // x differences from lane shuffles the x part only guards the stores, so
    // that every lane of a warp runs the shuffles
    const bool shfl = !fam && h->jit_xpair == 2;
    const smg::DevComp& c0 = h->comps[D[P[0]]];
    std::string cond;
    const char* ax[3] = {"x0", "y", "z"};
    for (int a = shfl ? 1 : 0; a < 3; ++a)
        if (c0.ext[a] < g.B[a]) {
            if (!cond.empty()) cond += " && ";
            cond += std::string(ax[a]) + " < " +
                    (fam ? N(a) + " + " + std::to_string(c0.ext[a] - g.n[a]) : std::to_string(c0.ext[a]));
        }
    o += cond.empty() ? "    {\n" : "    if (" + cond + ") {\n";
    const bool v1_always = !fam && c0.ext[0] % 2 == 0;
    const std::string v1 = v1_always ? "true" : "v1";
    if (!v1_always)
        o += "    const bool v1 = x1 < " +
             (fam ? "N0 + " + std::to_string(c0.ext[0] - g.n[0]) : std::to_string(c0.ext[0])) + ";\n";
    const std::string stx = !shfl ? "true"
                                  : (c0.ext[0] < g.B[0] ? "(act && x0 < " + std::to_string(c0.ext[0]) + ")" : "act");
    if (shfl && used[0])
        std::snprintf(b, sizeof b,
                      "    const int lane = (int)(threadIdx.x & 31);\n"
                      "    const bool xedge = x0 == 0 || x1 + 2 >= %d;\n", g.B[0]);
    else b[0] = 0;
    o += b;
    const std::string sel1 = v1_always ? "" : "v1 ? ", sel2 = v1_always ? "" : " : 0";
    const bool filt = h->filter_mode == SMG_FILTER_SUBSTEP;
    std::set<int> coef_done;
    std::set<std::pair<int, int>> val_done;
    auto coef = [&](int f) {
        const std::string n = "C" + std::to_string(f);
        if (coef_done.insert(f).second) {
            if (is_array(h, f)) std::snprintf(b, sizeof b, "    const double2 %s = ld2(fp(F, %d) + pt);\n", n.c_str(), f);
            else std::snprintf(b, sizeof b, "    const double %s = fs(F, %d);\n", n.c_str(), f);
            o += b;
        }
        return std::make_pair(is_array(h, f) ? n + ".x" : n, is_array(h, f) ? n + ".y" : n);
    };
    if (nextP && !fam) {
        // SMG_TUNE_JIT_PREFETCH 2, 3: thread 0 of the CTA (x0 = the chunk's
        // first point) requests into L2 the row segments that a later group
        // of this kernel reads at this row chunk -- its destinations, array
        // coefficients, x sources and both rows of every y/z source -- one
        // bulk prefetch per segment, so that the later group's loads find
        // them in L2
        const std::vector<int>& NP = *nextP;
        std::snprintf(b, sizeof b,
                      "    if (threadIdx.x == 0) {\n"
                      "        const unsigned nb = (unsigned)((x0 + %d < %lld ? %d : %lld - x0) * 8);\n",
                      2 * h->jit_block, (long long)g.s1, 2 * h->jit_block, (long long)g.s1);
        o += b;
        bool nused[3][2] = {{false, false}, {false, false}, {false, false}};
        for (int p : NP)
            for (int q = h->comps[D[p]].cbeg; q < h->comps[D[p]].cend; ++q)
                nused[h->coups[q].code >> 1][h->coups[q].code & 1] = true;
        for (int a = 1; a < 3; ++a)
            for (int g2 = 0; g2 < 2; ++g2) {
                if (!nused[a][g2]) continue;
                const long long stv = a == 1 ? g.s1 : g.s2;
                const char* pv = a == 1 ? "y" : "z";
                std::snprintf(b, sizeof b,
                              "        int nh%s_%d, nl%s_%d;\n"
                              "        { int hi, lo; stencil(%s, %d, %d, %d, hi, lo); nh%s_%d = (int)((hi - %s) * %lld); "
                              "nl%s_%d = (int)((lo - %s) * %lld); }\n",
                              an[a], g2, an[a], g2, pv, g.n[a], g.bc[a], g2, an[a], g2, pv, stv, an[a], g2, pv, stv);
                o += b;
            }
        std::set<int> fdone;
        std::set<std::pair<int, int>> sdone;
        const bool nfilt = h->filter_mode == SMG_FILTER_SUBSTEP;
        for (int p : NP) {
            const int j = D[p];
            const smg::DevComp& c = h->comps[j];
            std::snprintf(b, sizeof b, "        l2pf(Up + %lld, nb);\n", (long long)j * g.cs);
            o += b;
            const Coefs f = coefs_of(h, phase, j);
            std::vector<int> fl = {f.q, f.s, f.E};
            if (nfilt) fl.insert(fl.end(), {f.F1, f.F2});
            for (int fi : fl)
                if (is_array(h, fi) && fdone.insert(fi).second) {
                    std::snprintf(b, sizeof b, "        l2pf(fp(F, %d) + pt, nb);\n", fi);
                    o += b;
                }
            for (int qq = c.cbeg; qq < c.cend; ++qq) {
                const smg::DevCoup& cp = h->coups[qq];
                const int a = cp.code >> 1, g2 = cp.code & 1;
                if (!sdone.insert({a, cp.src}).second) continue;
                const long long so = (long long)cp.src * g.cs;
                if (a == 0) std::snprintf(b, sizeof b, "        l2pf(Up + %lld, nb);\n", so);
                else std::snprintf(b, sizeof b, "        l2pf(Up + %lld + nh%s_%d, nb); l2pf(Up + %lld + nl%s_%d, nb);\n",
                                   so, an[a], g2, so, an[a], g2);
                o += b;
            }
        }
        o += "    }\n";
    }
    if (h->jit_prefetch == 1 && !fam) {
        // every row the group reads, requested into L2 up front: the loads
        // below then wait for L2 rather than DRAM
        std::set<std::pair<int, int>> seen;
        for (int p : P) {
            const int j = D[p];
            const smg::DevComp& c = h->comps[j];
            std::snprintf(b, sizeof b, "    pf(U + pt + %lld);\n", (long long)j * g.cs);
            o += b;
            for (int qq = c.cbeg; qq < c.cend; ++qq) {
                const smg::DevCoup& cp = h->coups[qq];
                const int a = cp.code >> 1, g2 = cp.code & 1;
                if (!seen.insert({a, cp.src}).second) continue;
                const long long so = (long long)cp.src * g.cs;
                if (a == 0) std::snprintf(b, sizeof b, "    pf(Up + %lld);\n", so);
                else std::snprintf(b, sizeof b, "    pf(Up + %lld + h%s_%d); pf(Up + %lld + l%s_%d);\n", so, an[a], g2, so,
                                   an[a], g2);
                o += b;
            }
        }
    }
    for (int p : P) {
        const int j = D[p];
        const smg::DevComp& c = h->comps[j];
        const Coefs f = coefs_of(h, phase, j);
        const auto q = coef(f.q), sv = coef(f.s), E = coef(f.E);
        std::pair<std::string, std::string> k1{"1.0", "1.0"}, k2{"1.0", "1.0"};
        if (filt) {
            k1 = coef(f.F1);
            k2 = coef(f.F2);
        }
        // source values of this destination's couplings not loaded yet
        for (int qq = c.cbeg; qq < c.cend; ++qq) {
            const smg::DevCoup& cp = h->coups[qq];
            const int a = cp.code >> 1, g2 = cp.code & 1;
            if (!val_done.insert({a, cp.src}).second) continue;
            const long long so = (long long)cp.src * g.cs;
            const std::string sos = off(cp.src);
            if (a == 0 && shfl) {
                // one 128-bit load of the pair; the third value from the
                // neighbouring lane (lane 0 / 31 load it); pairs at the row
                // edges (xedge) use the stencil offsets
                const int n = cp.src;
                if (xpattern_a(g2, g.bc[0]))
                    std::snprintf(b, sizeof b,
                                  "    const double2 P%d = ld2(Up + %lld);\n"
                                  "    double X%d_b0 = __shfl_up_sync(0xffffffffu, P%d.y, 1);\n"
                                  "    if (lane == 0) X%d_b0 = ld1(Up + %lld + (x0 > 0 ? -1 : 0));\n"
                                  "    double X%d_a0 = P%d.x, X%d_a1 = P%d.y, X%d_b1 = P%d.x;\n",
                                  n, so, n, n, n, so, n, n, n, n, n, n);
                else
                    std::snprintf(b, sizeof b,
                                  "    const double2 P%d = ld2(Up + %lld);\n"
                                  "    double X%d_a1 = __shfl_down_sync(0xffffffffu, P%d.x, 1);\n"
                                  "    if (lane == 31) X%d_a1 = ld1(Up + %lld + (x1 + 1 < %d ? 2 : 0));\n"
                                  "    double X%d_a0 = P%d.y, X%d_b0 = P%d.x, X%d_b1 = P%d.y;\n",
                                  n, so, n, n, n, so, g.B[0], n, n, n, n, n, n);
                o += b;
                std::snprintf(b, sizeof b,
                              "    if (xedge) { X%d_a0 = ld1(Up + %lld + hx0_%d); X%d_b0 = ld1(Up + %lld + lx0_%d); "
                              "X%d_a1 = ld1(Up + %lld + (%shx1_%d%s)); X%d_b1 = ld1(Up + %lld + (%slx1_%d%s)); }\n",
                              n, so, g2, n, so, g2, n, so, sel1.c_str(), g2, sel2.c_str(), n, so, sel1.c_str(), g2,
                              sel2.c_str());
            } else if (a == 0)
                std::snprintf(b, sizeof b,
                              "    const double X%d_a0 = ld1(Up + %s + hx0_%d), X%d_b0 = ld1(Up + %s + lx0_%d), "
                              "X%d_a1 = ld1(Up + %s + (%shx1_%d%s)), X%d_b1 = ld1(Up + %s + (%slx1_%d%s));\n",
                              cp.src, sos.c_str(), g2, cp.src, sos.c_str(), g2, cp.src, sos.c_str(), sel1.c_str(), g2,
                              sel2.c_str(), cp.src, sos.c_str(), sel1.c_str(), g2, sel2.c_str());
            else
                std::snprintf(b, sizeof b,
                              "    const double2 %c%d_h = ld2(Up + %s + h%s_%d), %c%d_l = ld2(Up + %s + l%s_%d);\n",
                              a == 1 ? 'Y' : 'Z', cp.src, sos.c_str(), an[a], g2, a == 1 ? 'Y' : 'Z', cp.src, sos.c_str(),
                              an[a], g2);
            o += b;
        }
        std::snprintf(b, sizeof b,
                      "    {\n        double* Uj = U + pt + %s;\n"
                      "        const double2 u = *reinterpret_cast<const double2*>(Uj);\n"
                      "        double SA = 0.0, SB = 0.0;\n",
                      off(j).c_str());
        o += b;
        bool first = true;
        for (int qq = c.cbeg; qq < c.cend; ++qq) {
            const smg::DevCoup& cp = h->coups[qq];
            const int a = cp.code >> 1;
            const int mode_div = h->exact_recip[a];
            // the family form divides with two correction steps: exact for
            // every normal spacing, so its instances need not share one
            const std::string H = fam ? "H" + std::to_string(a) : clit(g.h[a]),
                              RH = fam ? "RH" + std::to_string(a) : clit(h->rh[a]), W = clit(cp.w);
            const char* dv = fam ? "div1" : (mode_div == 2 ? "div2" : (mode_div == 1 ? "div1" : "div0"));
            const char* fold = first ? "SA = tA; SB = tB;" : "SA = __dadd_rn(SA, tA); SB = __dadd_rn(SB, tB);";
            first = false;
            std::string dA, dB;
            if (a == 0) {
                dA = "__dsub_rn(X" + std::to_string(cp.src) + "_a0, X" + std::to_string(cp.src) + "_b0)";
                dB = "__dsub_rn(X" + std::to_string(cp.src) + "_a1, X" + std::to_string(cp.src) + "_b1)";
            } else {
                const std::string n = std::string(1, a == 1 ? 'Y' : 'Z') + std::to_string(cp.src);
                dA = "__dsub_rn(" + n + "_h.x, " + n + "_l.x)";
                dB = "__dsub_rn(" + n + "_h.y, " + n + "_l.y)";
            }
            std::snprintf(b, sizeof b,
                          "        { const double tA = __dmul_rn(%s(%s, %s, %s), %s);\n"
                          "          const double tB = __dmul_rn(%s(%s, %s, %s), %s);\n"
                          "          %s }\n",
                          dv, dA.c_str(), H.c_str(), RH.c_str(), W.c_str(), dv, dB.c_str(), H.c_str(), RH.c_str(),
                          W.c_str(), fold);
            o += b;
        }
        o += "        double u0 = u.x, u1 = u.y;\n";
        if (rec) {
            // the sigma-gradient factor of this phase for the adjoint sweep
            // (phase kind dsm substeps, first filter k=2 when dsw), from the
            // values before the phase and the coupling sum, in W's slot
            const long long so = (long long)p * g.cs;
            std::string de0, de1;
            if (is_array(h, f.s)) {
                std::snprintf(b, sizeof b, "        const double2 DEv = ld2(fp(DE, %d) + pt);\n", f.s);
                de0 = "DEv.x";
                de1 = "DEv.y";
            } else {
                std::snprintf(b, sizeof b, "        const double DEv = fs(DE, %d);\n", f.s);
                de0 = de1 = "DEv";
            }
            o += b;
            std::snprintf(b, sizeof b,
                          "        if (%s) { double* wp = WR + pt + %lld;\n"
                          "          const double D0 = dsdw(dsm, u.x, -SA, %s, %s, %s, dsw ? %s : %s, %s, hdt);\n"
                          "          if (%s) *reinterpret_cast<double2*>(wp) = make_double2(D0, "
                          "dsdw(dsm, u.y, -SB, %s, %s, %s, dsw ? %s : %s, %s, hdt)); else wp[0] = D0; }\n",
                          stx.c_str(), so, sv.first.c_str(), E.first.c_str(), q.first.c_str(), k2.first.c_str(),
                          k1.first.c_str(), de0.c_str(), v1.c_str(), sv.second.c_str(), E.second.c_str(),
                          q.second.c_str(), k2.second.c_str(), k1.second.c_str(), de1.c_str());
            o += b;
        }
        auto sub = [&]() {
            std::snprintf(b, sizeof b, "u0 = upd(u0, -SA, %s, %s, %s, hdt); u1 = upd(u1, -SB, %s, %s, %s, hdt);",
                          q.first.c_str(), sv.first.c_str(), E.first.c_str(), q.second.c_str(), sv.second.c_str(),
                          E.second.c_str());
            return std::string(b);
        };
        auto fl = [&](const std::pair<std::string, std::string>& F) {
            return filt ? " u0 = __dmul_rn(u0, " + F.first + "); u1 = __dmul_rn(u1, " + F.second + ");" : std::string();
        };
        if (phase == 0) {
            const std::string one =
                "        " + sub() +
                (filt ? " u0 = __dmul_rn(u0, kf == 1 ? " + k1.first + " : " + k2.first + "); u1 = __dmul_rn(u1, kf == 1 ? " +
                            k1.second + " : " + k2.second + ");"
                      : std::string()) +
                "\n";
            const std::string two = "        " + sub() + fl(k2) + "\n        " + sub() + fl(k1) + "\n";
            if (h->filter_mode == SMG_FILTER_FULL) o += one;
            else o += "        if (mode == 0) {\n" + one + "        } else {\n" + two + "        }\n";
        } else {
            o += "        " + sub() + fl(k1) + "\n        " + sub() + fl(k2) + "\n";
        }
        const std::string guard = stx == "true" ? "" : "if (" + stx + ") ";
        if (v1_always) o += "        " + guard + "*reinterpret_cast<double2*>(Uj) = make_double2(u0, u1);\n    }\n";
        else
            o += "        " + guard + "{ if (v1) *reinterpret_cast<double2*>(Uj) = make_double2(u0, u1); else *Uj = u0; }\n    }\n";
    }
    o += "    }\n}\n";
}

// ---- bulk-staged kernels -----------------------------------------------------
// The register form above loads every source value with a global load at its
// first use, so each warp waits on DRAM several times per group and the loads
// in flight are bounded by the registers that hold them.  In the staged form a
// CTA owns one group, a 64-point chunk of a row and a band of rows; one
// producer thread copies, for each row of the band, every row segment the
// group reads (its destinations, the array coefficients, the x sources with
// two points either side, both neighbouring rows of every y/z source) into a
// ring of shared-memory stages with the bulk copy engine (cp.async.bulk,
// completion counted in bytes on an mbarrier), up to `stages` rows ahead of
// the consumers; consumer warps (the group's destinations split into slices,
// one warp per slice, a lane per point pair) fold the couplings from shared
// memory with the register form's arithmetic and store their destinations.
// Copies are in flight without holding registers, and the register budget is
// no longer split with the loads.  All waits are bounded (4 s): a wait that
// runs out sets the kernel's error flag and ends the CTA.
constexpr int kStW = 64;      // points of a row per CTA: 32 lanes x 2
constexpr int kStSlot = 68;   // doubles per staged row segment: the chunk and 2 points either side

struct StagedRows {
    std::vector<int> coefs;                     // array fields read by the group
    std::vector<std::pair<int, int>> xs;        // (source, g2) of x differences
    std::vector<std::tuple<int, int, int>> yz;  // (axis, source, g2): two slots (hi row, lo row)
    int nd = 0;                                 // destinations (slots 0..nd-1)
    int slot_coef(int f) const { return nd + (int)(std::find(coefs.begin(), coefs.end(), f) - coefs.begin()); }
    int slot_x(int src) const {
        for (size_t i = 0; i < xs.size(); ++i)
            if (xs[i].first == src) return nd + (int)coefs.size() + (int)i;
        return -1;
    }
    int slot_yz(int a, int src) const {
        for (size_t i = 0; i < yz.size(); ++i)
            if (std::get<0>(yz[i]) == a && std::get<1>(yz[i]) == src)
                return nd + (int)coefs.size() + (int)xs.size() + 2 * (int)i;
        return -1;
    }
    int nslots() const { return nd + (int)coefs.size() + (int)xs.size() + 2 * (int)yz.size(); }
};

StagedRows staged_rows(const smg_handle* h, int phase, const std::vector<int>& D, const std::vector<int>& P) {
    StagedRows R;
    R.nd = (int)P.size();
    const bool filt = h->filter_mode == SMG_FILTER_SUBSTEP;
    for (int p : P) {
        const Coefs f = coefs_of(h, phase, D[p]);
        std::vector<int> fl = {f.q, f.s, f.E};
        if (filt) fl.insert(fl.end(), {f.F1, f.F2});
        for (int fi : fl)
            if (is_array(h, fi) && std::find(R.coefs.begin(), R.coefs.end(), fi) == R.coefs.end())
                R.coefs.push_back(fi);
    }
    for (int p : P) {
        const smg::DevComp& c = h->comps[D[p]];
        for (int q = c.cbeg; q < c.cend; ++q) {
            const smg::DevCoup& cp = h->coups[q];
            const int a = cp.code >> 1, g2 = cp.code & 1;
            if (a == 0) {
                if (R.slot_x(cp.src) < 0) R.xs.push_back({cp.src, g2});
            } else if (R.slot_yz(a, cp.src) < 0) {
                R.yz.push_back(std::make_tuple(a, cp.src, g2));
            }
        }
    }
    return R;
}

std::string staged_group_name(int phase, int k) { return "smg_s" + std::to_string(phase) + "_" + std::to_string(k); }

// One group of the staged form over the rows of the CTA's band.  P:
// positions into the phase's destination list; ns consumer warps (slices); st
// ring stages of `stage` doubles; rb rows per band.  loader 1: a producer
// thread issues bulk copies completing on mbarriers; loader 2: the consumer
// warps copy the segments themselves with 16-byte asynchronous copies (one
// warp instruction per 64-point segment), `st - 1` rows ahead, with one CTA
// barrier per row and no spin waits.
void emit_staged_group(std::string& o, const smg_handle* h, int phase, int k, const std::vector<int>& P, int ns,
                       int st, int rb, long long stage, int loader) {
    const smg::DevGrid& g = h->g;
    const std::vector<int> D = phase_dests(h, phase);
    const StagedRows R = staged_rows(h, phase, D, P);
    const smg::DevComp& c0 = h->comps[D[P[0]]];
    const int E0 = c0.ext[0], E1 = c0.ext[1], E2 = c0.ext[2];
    const long long nrows = (long long)E1 * E2;
    const bool filt = h->filter_mode == SMG_FILTER_SUBSTEP;
    const char* an[3] = {"x", "y", "z"};
    char b[4096];
    bool used_g2[3][2] = {{false, false}, {false, false}, {false, false}};
    for (int p : P)
        for (int q = h->comps[D[p]].cbeg; q < h->comps[D[p]].cend; ++q)
            used_g2[h->coups[q].code >> 1][h->coups[q].code & 1] = true;
    std::snprintf(b, sizeof b,
                  "static __device__ __forceinline__ void %s(double* __restrict__ U, const DevField* __restrict__ F, "
                  "double hdt, int kf, int mode, int* err, double* smem, int chunk, int band) {\n"
                  "    (void)hdt; (void)kf; (void)mode; (void)F;\n"
                  "    const int c0 = chunk * %d;\n"
                  "    if (c0 >= %d) return;\n"
                  "    const int q0 = band * %d;\n"
                  "    if (q0 >= %lld) return;\n"
                  "    const int q1 = q0 + %d < %lld ? q0 + %d : %lld;\n"
                  "    double* sm = smem + 16;\n"
                  "    const int warp = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31);\n",
                  staged_group_name(phase, k).c_str(), kStW, E0, rb, nrows, rb, nrows, rb, nrows);
    o += b;
    if (loader == 1) {
        std::snprintf(b, sizeof b,
                      "    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem);\n"
                      "    if (threadIdx.x == 0) {\n"
                      "        for (int s = 0; s < %d; ++s) { mb_init(&bar[s], 1); mb_init(&bar[%d + s], %d); }\n"
                      "        asm volatile(\"fence.mbarrier_init.release.cluster;\" ::: \"memory\");\n"
                      "        asm volatile(\"fence.proxy.async.shared::cta;\" ::: \"memory\");\n"
                      "    }\n"
                      "    __syncthreads();\n",
                      st, st, ns);
        o += b;
    } else {
        o += "    (void)err;\n";
    }
    // ---- producer: one thread (loader 1)
    const int nx = (int)R.xs.size();
    if (loader == 1) {
    const int nother = R.nd + (int)R.coefs.size() + 2 * (int)R.yz.size();
    std::snprintf(b, sizeof b,
                  "    if (warp == %d) {\n"
                  "        if (lane != 0) return;\n"
                  "        const int xl = c0 - 2 < 0 ? 0 : c0 - 2, xr = c0 + %d < %lld ? c0 + %d : %lld;\n"
                  "        const unsigned xb = (unsigned)(xr - xl) * 8u;\n"
                  "        const int xo = xl - (c0 - 2);\n"
                  "        const unsigned db = (unsigned)((c0 + %d < %lld ? c0 + %d : %lld) - c0) * 8u;\n"
                  "        const unsigned tx = %du * xb + %du * db;\n"
                  "        (void)xo; (void)xb;\n"
                  "        for (int q = q0, it = 0; q < q1; ++q, ++it) {\n"
                  "            const int s = it %% %d;\n"
                  "            if (it >= %d && !mb_wait(&bar[%d + s], ((it / %d) & 1) ^ 1)) { atomicExch(err, 1); return; }\n"
                  "            const int y = q %% %d, z = q / %d;\n"
                  "            const double* Ur = U + ((long long)z * %lld + (long long)y * %lld);\n"
                  "            double* stg = sm + (long long)s * %lld;\n",
                  ns, kStW + 2, (long long)g.s1, kStW + 2, (long long)g.s1, kStW, (long long)g.s1, kStW,
                  (long long)g.s1, nx, nother, st, st, st, st, E1, E1, (long long)g.s2, (long long)g.s1, stage);
    o += b;
    for (int a = 1; a < 3; ++a)
        for (int g2 = 0; g2 < 2; ++g2) {
            if (!used_g2[a][g2]) continue;
            const long long stv = a == 1 ? g.s1 : g.s2;
            const char* pv = a == 1 ? "y" : "z";
            std::snprintf(b, sizeof b,
                          "            long long h%s_%d, l%s_%d;\n"
                          "            { int hi, lo; stencil(%s, %d, %d, %d, hi, lo); h%s_%d = (long long)(hi - %s) * %lld; "
                          "l%s_%d = (long long)(lo - %s) * %lld; }\n",
                          an[a], g2, an[a], g2, pv, g.n[a], g.bc[a], g2, an[a], g2, pv, stv, an[a], g2, pv, stv);
            o += b;
        }
    o += "            mb_expect(&bar[s], tx);\n";
    for (int i = 0; i < R.nd; ++i) {
        std::snprintf(b, sizeof b, "            bulk_ld(stg + %d, Ur + %lld + c0, db, &bar[s]);\n", i * kStSlot + 2,
                      (long long)D[P[i]] * g.cs);
        o += b;
    }
    for (size_t i = 0; i < R.coefs.size(); ++i) {
        std::snprintf(b, sizeof b, "            bulk_ld(stg + %d, fp(F, %d) + (Ur - U) + c0, db, &bar[s]);\n",
                      R.slot_coef(R.coefs[i]) * kStSlot + 2, R.coefs[i]);
        o += b;
    }
    for (const auto& xsrc : R.xs) {
        std::snprintf(b, sizeof b, "            bulk_ld(stg + %d + xo, Ur + %lld + xl, xb, &bar[s]);\n",
                      R.slot_x(xsrc.first) * kStSlot, (long long)xsrc.first * g.cs);
        o += b;
    }
    for (const auto& t : R.yz) {
        const int a = std::get<0>(t), src = std::get<1>(t), g2 = std::get<2>(t);
        const int sl = R.slot_yz(a, src);
        std::snprintf(b, sizeof b,
                      "            bulk_ld(stg + %d, Ur + %lld + h%s_%d + c0, db, &bar[s]);\n"
                      "            bulk_ld(stg + %d, Ur + %lld + l%s_%d + c0, db, &bar[s]);\n",
                      sl * kStSlot + 2, (long long)src * g.cs, an[a], g2, (sl + 1) * kStSlot + 2,
                      (long long)src * g.cs, an[a], g2);
        o += b;
    }
    o += "        }\n        return;\n    }\n";
    }
    // ---- consumers: per-thread x stencil offsets, fixed over the band
    std::snprintf(b, sizeof b,
                  "    const int x0 = c0 + 2 * lane, x1 = x0 + 1;\n"
                  "    const bool act = x0 < %d, v1 = x1 < %d;\n"
                  "    (void)v1;\n",
                  E0, E0);
    o += b;
    for (int g2 = 0; g2 < 2; ++g2) {
        if (!used_g2[0][g2]) continue;
        const bool pa = xpattern_a(g2, g.bc[0]);
        std::snprintf(b, sizeof b,
                      "    int hx0_%d = 0, lx0_%d = 0, hx1_%d = 0, lx1_%d = 0;\n"
                      "    if (act) {\n"
                      "        int hi, lo; stencil(x0, %d, %d, %d, hi, lo); hx0_%d = hi - x0; lx0_%d = lo - x0;\n"
                      "        if (v1) { stencil(x1, %d, %d, %d, hi, lo); hx1_%d = hi - x0; lx1_%d = lo - x0; }\n"
                      "    }\n"
                      "    const bool xf_%d = act && v1 && hx0_%d == %d && lx0_%d == %d && hx1_%d == %d && lx1_%d == %d;\n"
                      "    const bool xw_%d = hx0_%d >= -2 && hx0_%d <= 3 && lx0_%d >= -2 && lx0_%d <= 3 && "
                      "hx1_%d >= -2 && hx1_%d <= 3 && lx1_%d >= -2 && lx1_%d <= 3;\n",
                      g2, g2, g2, g2, g.n[0], g.bc[0], g2, g2, g2, g.n[0], g.bc[0], g2, g2, g2, g2, g2, pa ? 0 : 1, g2,
                      pa ? -1 : 0, g2, pa ? 1 : 2, g2, pa ? 0 : 1, g2, g2, g2, g2, g2, g2, g2, g2, g2);
        o += b;
    }
    if (loader == 2) {
        // the copies of one row: main 64-point segments (a warp instruction
        // each, lane l the 16 bytes at c0 + 2l) spread over the warps, and
        // the two 2-point halos of every x source (lanes 0 and 1)
        std::vector<std::pair<int, std::string>> cp;   // (slot, source row pointer expression)
        for (int i = 0; i < R.nd; ++i) cp.push_back({i, "Ur + " + std::to_string((long long)D[P[i]] * g.cs)});
        for (int f : R.coefs) cp.push_back({R.slot_coef(f), "fp(F, " + std::to_string(f) + ") + (Ur - U)"});
        for (const auto& xsrc : R.xs) cp.push_back({R.slot_x(xsrc.first), "Ur + " + std::to_string((long long)xsrc.first * g.cs)});
        for (const auto& t : R.yz) {
            const int a = std::get<0>(t), src = std::get<1>(t), g2 = std::get<2>(t);
            const int sl = R.slot_yz(a, src);
            const std::string base = "Ur + " + std::to_string((long long)src * g.cs) + " + ";
            cp.push_back({sl, base + "h" + an[a] + "_" + std::to_string(g2)});
            cp.push_back({sl + 1, base + "l" + an[a] + "_" + std::to_string(g2)});
        }
        std::snprintf(b, sizeof b,
                      "    auto issue = [&](int i) {\n"
                      "        const int qq = q0 + i;\n"
                      "        if (qq >= q1) return;\n"
                      "        const int y = qq %% %d, z = qq / %d;\n"
                      "        const double* Ur = U + ((long long)z * %lld + (long long)y * %lld);\n"
                      "        double* stg = sm + (long long)(i %% %d) * %lld;\n",
                      E1, E1, (long long)g.s2, (long long)g.s1, st, stage);
        o += b;
        for (int a = 1; a < 3; ++a)
            for (int g2 = 0; g2 < 2; ++g2) {
                if (!used_g2[a][g2]) continue;
                const long long stv = a == 1 ? g.s1 : g.s2;
                const char* pv = a == 1 ? "y" : "z";
                std::snprintf(b, sizeof b,
                              "        long long h%s_%d, l%s_%d;\n"
                              "        { int hi, lo; stencil(%s, %d, %d, %d, hi, lo); h%s_%d = (long long)(hi - %s) * %lld; "
                              "l%s_%d = (long long)(lo - %s) * %lld; }\n",
                              an[a], g2, an[a], g2, pv, g.n[a], g.bc[a], g2, an[a], g2, pv, stv, an[a], g2, pv, stv);
                o += b;
            }
        std::snprintf(b, sizeof b, "        const int xo = c0 + 2 * lane;\n        if (xo < %lld) {\n        switch (warp) {\n",
                      (long long)g.s1);
        o += b;
        for (int w = 0; w < ns; ++w) {
            std::string body;
            for (size_t c = w; c < cp.size(); c += ns)
                body += "            cpa(stg + " + std::to_string(cp[c].first * kStSlot + 2) + " + 2 * lane, " +
                        cp[c].second + " + xo);\n";
            if (!body.empty()) o += "        case " + std::to_string(w) + ":\n" + body + "            break;\n";
        }
        o += "        default: break;\n        }\n        }\n";
        if (!R.xs.empty()) {
            std::snprintf(b, sizeof b,
                          "        if (lane < 2) {\n"
                          "            const int hx = lane == 0 ? c0 - 2 : c0 + %d;\n"
                          "            if (hx >= 0 && hx + 2 <= %lld) {\n"
                          "            double* hd = stg + (lane == 0 ? 0 : %d);\n"
                          "            switch (warp) {\n",
                          kStW, (long long)g.s1, kStW + 2);
            o += b;
            for (int w = 0; w < ns; ++w) {
                std::string body;
                for (size_t c = w; c < R.xs.size(); c += ns)
                    body += "                cpa(hd + " + std::to_string(R.slot_x(R.xs[c].first) * kStSlot) + ", Ur + " +
                            std::to_string((long long)R.xs[c].first * g.cs) + " + hx);\n";
                if (!body.empty()) o += "            case " + std::to_string(w) + ":\n" + body + "                break;\n";
            }
            o += "            default: break;\n            }\n            }\n        }\n";
        }
        o += "    };\n";
        std::snprintf(b, sizeof b, "    for (int i = 0; i < %d; ++i) { issue(i); cpa_commit(); }\n", st - 1);
        o += b;
    }
    if (loader == 1)
        std::snprintf(b, sizeof b,
                      "    for (int q = q0, it = 0; q < q1; ++q, ++it) {\n"
                      "        const int s = it %% %d;\n"
                      "        if (!mb_wait(&bar[s], (it / %d) & 1)) { atomicExch(err, 1); return; }\n",
                      st, st);
    else
        std::snprintf(b, sizeof b,
                      "    for (int q = q0, it = 0; q < q1; ++q, ++it) {\n"
                      "        const int s = it %% %d;\n"
                      "        cpa_wait<%d>();\n"
                      "        __syncthreads();\n"
                      "        issue(it + %d);\n"
                      "        cpa_commit();\n",
                      st, st - 2, st - 1);
    o += b;
    std::snprintf(b, sizeof b,
                  "        const int y = q %% %d, z = q / %d;\n"
                  "        const int pt = z * %lld + y * %lld + x0;\n"
                  "        const double* st = sm + (long long)s * %lld + 2 + 2 * lane;\n"
                  "        (void)pt;\n"
                  "        if (act) {\n"
                  "        switch (warp) {\n",
                  E1, E1, (long long)g.s2, (long long)g.s1, stage);
    o += b;
    // slices: contiguous runs of the group's destinations (the group order
    // puts destinations that share sources next to each other)
    const int G = (int)P.size();
    for (int w = 0; w < ns; ++w) {
        const int p0 = (int)((long long)G * w / ns), p1 = (int)((long long)G * (w + 1) / ns);
        if (p0 >= p1) continue;
        o += "        case " + std::to_string(w) + ": {\n";
        std::set<int> coef_done;
        std::set<std::pair<int, int>> val_done;
        auto coef = [&](int f) {
            const std::string n = "C" + std::to_string(f);
            if (coef_done.insert(f).second) {
                if (is_array(h, f)) std::snprintf(b, sizeof b, "            const double2 %s = lds2(st + %d);\n", n.c_str(),
                                                  R.slot_coef(f) * kStSlot);
                else std::snprintf(b, sizeof b, "            const double %s = fs(F, %d);\n", n.c_str(), f);
                o += b;
            }
            return std::make_pair(is_array(h, f) ? n + ".x" : n, is_array(h, f) ? n + ".y" : n);
        };
        for (int pi = p0; pi < p1; ++pi) {
            const int j = D[P[pi]];
            const smg::DevComp& c = h->comps[j];
            const Coefs f = coefs_of(h, phase, j);
            const auto q = coef(f.q), sv = coef(f.s), E = coef(f.E);
            std::pair<std::string, std::string> k1{"1.0", "1.0"}, k2{"1.0", "1.0"};
            if (filt) {
                k1 = coef(f.F1);
                k2 = coef(f.F2);
            }
            for (int qq = c.cbeg; qq < c.cend; ++qq) {
                const smg::DevCoup& cp = h->coups[qq];
                const int a = cp.code >> 1, g2 = cp.code & 1;
                if (!val_done.insert({a, cp.src}).second) continue;
                if (a == 0)
                    std::snprintf(b, sizeof b,
                                  "            double X%d_a0, X%d_b0, X%d_a1, X%d_b1;\n"
                                  "            xvals(%d, st + %d, U + pt + %lld, xf_%d, xw_%d, hx0_%d, lx0_%d, hx1_%d, "
                                  "lx1_%d, X%d_a0, X%d_b0, X%d_a1, X%d_b1);\n",
                                  cp.src, cp.src, cp.src, cp.src, xpattern_a(g2, g.bc[0]) ? 1 : 0,
                                  R.slot_x(cp.src) * kStSlot, (long long)cp.src * g.cs, g2, g2, g2, g2, g2, g2, cp.src,
                                  cp.src, cp.src, cp.src);
                else
                    std::snprintf(b, sizeof b, "            const double2 %c%d_h = lds2(st + %d), %c%d_l = lds2(st + %d);\n",
                                  a == 1 ? 'Y' : 'Z', cp.src, R.slot_yz(a, cp.src) * kStSlot, a == 1 ? 'Y' : 'Z', cp.src,
                                  (R.slot_yz(a, cp.src) + 1) * kStSlot);
                o += b;
            }
            std::snprintf(b, sizeof b,
                          "            {\n"
                          "                const double2 u = lds2(st + %d);\n"
                          "                double SA = 0.0, SB = 0.0;\n",
                          pi * kStSlot);
            o += b;
            bool first = true;
            for (int qq = c.cbeg; qq < c.cend; ++qq) {
                const smg::DevCoup& cp = h->coups[qq];
                const int a = cp.code >> 1;
                const int mode_div = h->exact_recip[a];
                const std::string H = clit(g.h[a]), RH = clit(h->rh[a]), W = clit(cp.w);
                const char* dv = mode_div == 2 ? "div2" : (mode_div == 1 ? "div1" : "div0");
                const char* fold = first ? "SA = tA; SB = tB;" : "SA = __dadd_rn(SA, tA); SB = __dadd_rn(SB, tB);";
                first = false;
                std::string dA, dB;
                if (a == 0) {
                    dA = "__dsub_rn(X" + std::to_string(cp.src) + "_a0, X" + std::to_string(cp.src) + "_b0)";
                    dB = "__dsub_rn(X" + std::to_string(cp.src) + "_a1, X" + std::to_string(cp.src) + "_b1)";
                } else {
                    const std::string n = std::string(1, a == 1 ? 'Y' : 'Z') + std::to_string(cp.src);
                    dA = "__dsub_rn(" + n + "_h.x, " + n + "_l.x)";
                    dB = "__dsub_rn(" + n + "_h.y, " + n + "_l.y)";
                }
                std::snprintf(b, sizeof b,
                              "                { const double tA = __dmul_rn(%s(%s, %s, %s), %s);\n"
                              "                  const double tB = __dmul_rn(%s(%s, %s, %s), %s);\n"
                              "                  %s }\n",
                              dv, dA.c_str(), H.c_str(), RH.c_str(), W.c_str(), dv, dB.c_str(), H.c_str(), RH.c_str(),
                              W.c_str(), fold);
                o += b;
            }
            o += "                double u0 = u.x, u1 = u.y;\n";
            auto sub = [&]() {
                std::snprintf(b, sizeof b, "u0 = upd(u0, -SA, %s, %s, %s, hdt); u1 = upd(u1, -SB, %s, %s, %s, hdt);",
                              q.first.c_str(), sv.first.c_str(), E.first.c_str(), q.second.c_str(), sv.second.c_str(),
                              E.second.c_str());
                return std::string(b);
            };
            auto fl = [&](const std::pair<std::string, std::string>& Fp) {
                return filt ? " u0 = __dmul_rn(u0, " + Fp.first + "); u1 = __dmul_rn(u1, " + Fp.second + ");"
                            : std::string();
            };
            if (phase == 0) {
                const std::string one =
                    "                " + sub() +
                    (filt ? " u0 = __dmul_rn(u0, kf == 1 ? " + k1.first + " : " + k2.first +
                                "); u1 = __dmul_rn(u1, kf == 1 ? " + k1.second + " : " + k2.second + ");"
                          : std::string()) +
                    "\n";
                const std::string two = "                " + sub() + fl(k2) + "\n                " + sub() + fl(k1) + "\n";
                if (h->filter_mode == SMG_FILTER_FULL) o += one;
                else o += "                if (mode == 0) {\n" + one + "                } else {\n" + two + "                }\n";
            } else {
                o += "                " + sub() + fl(k1) + "\n                " + sub() + fl(k2) + "\n";
            }
            std::snprintf(b, sizeof b,
                          "                double* Uj = U + pt + %lld;\n"
                          "                if (v1) *reinterpret_cast<double2*>(Uj) = make_double2(u0, u1); else *Uj = u0;\n"
                          "            }\n",
                          (long long)j * g.cs);
            o += b;
        }
        o += "        } break;\n";
    }
    o += "        default: break;\n        }\n        }\n";
    if (loader == 1)
        o += "        __syncwarp();\n"
             "        if (lane == 0) mb_arrive(&bar[" + std::to_string(st) + " + s]);\n"
             "    }\n}\n";
    else
        o += "    }\n    cpa_wait<0>();\n}\n";
}


// ---- register form with a per-thread prefetch ring (SMG_TUNE_JIT_STAGED 3) ----
// The register form's CTA mapping and straight-line group code, but every
// value a destination reads from global memory for the first time is copied
// by the thread itself (cp.async, 8 or 16 bytes) into its own column of a
// small shared ring one destination ahead: while destination d computes, the
// copies of destination d+1 are in flight without holding registers.  Each
// thread reads only what it copied itself, so no barrier is needed.
struct PfItem {
    int kind;    // 0 array coefficient, 1 x source (four 8-byte values), 2 y/z source (two rows), 3 destination
    int id;      // field, source component or destination
    int a, g2;   // axis and grid flag of a source
    int slot[2];
};

std::vector<std::vector<PfItem>> prefetch_items(const smg_handle* h, int phase, const std::vector<int>& D,
                                                const std::vector<int>& P) {
    const bool filt = h->filter_mode == SMG_FILTER_SUBSTEP;
    std::vector<std::vector<PfItem>> items(P.size());
    std::set<int> coef_done;
    std::set<std::pair<int, int>> val_done;
    for (size_t pi = 0; pi < P.size(); ++pi) {
        const int j = D[P[pi]];
        const smg::DevComp& c = h->comps[j];
        const Coefs f = coefs_of(h, phase, j);
        std::vector<int> fl = {f.q, f.s, f.E};
        if (filt) fl.insert(fl.end(), {f.F1, f.F2});
        for (int fi : fl)
            if (is_array(h, fi) && coef_done.insert(fi).second) items[pi].push_back({0, fi, 0, 0, {-1, -1}});
        for (int qq = c.cbeg; qq < c.cend; ++qq) {
            const smg::DevCoup& cp = h->coups[qq];
            const int a = cp.code >> 1, g2 = cp.code & 1;
            if (!val_done.insert({a, cp.src}).second) continue;
            items[pi].push_back({a == 0 ? 1 : 2, cp.src, a, g2, {-1, -1}});
        }
        items[pi].push_back({3, j, 0, 0, {-1, -1}});
    }
    return items;
}

int item_slots(const PfItem& it) { return it.kind == 1 || it.kind == 2 ? 2 : 1; }

// ring slots one destination ahead needs: the largest sum over two consecutive destinations
int prefetch_ring(const std::vector<std::vector<PfItem>>& items) {
    int best = 1;
    for (size_t d = 0; d < items.size(); ++d) {
        int n = 0;
        for (size_t e = d; e < std::min(items.size(), d + 2); ++e)
            for (const PfItem& it : items[e]) n += item_slots(it);
        best = std::max(best, n);
    }
    return best;
}

void emit_prefetch_group(std::string& o, const smg_handle* h, int phase, int k, const std::vector<int>& P, int ring,
                         int block) {
    const smg::DevGrid& g = h->g;
    const std::vector<int> D = phase_dests(h, phase);
    std::vector<std::vector<PfItem>> items = prefetch_items(h, phase, D, P);
    int next = 0;
    for (auto& v : items)
        for (PfItem& it : v)
            for (int q = 0; q < item_slots(it); ++q) {
                it.slot[q] = next;
                next = (next + 1) % ring;
            }
    const bool filt = h->filter_mode == SMG_FILTER_SUBSTEP;
    const char* an[3] = {"x", "y", "z"};
    char b[4096];
    o += "static __device__ __forceinline__ void " + group_name(phase, k) + group_args(false) + " {\n";
    std::snprintf(b, sizeof b,
                  "    const int x1 = x0 + 1;\n"
                  "    const int pt = z * %lld + y * %lld + x0;\n"
                  "    const double* Up = R + pt;\n"
                  "    (void)x1; (void)kf; (void)mode; (void)hdt; (void)Up; (void)act;\n",
                  (long long)g.s2, (long long)g.s1);
    o += b;
    bool used[3] = {false, false, false};
    for (int p : P)
        for (int q = h->comps[D[p]].cbeg; q < h->comps[D[p]].cend; ++q) used[h->coups[q].code >> 1] = true;
    if (used[0])
        for (int g2 = 0; g2 < 2; ++g2) {
            std::snprintf(b, sizeof b,
                          "    int hx0_%d, lx0_%d, hx1_%d, lx1_%d;\n"
                          "    { int hi, lo; stencil(x0, %d, %d, %d, hi, lo); hx0_%d = hi - x0; lx0_%d = lo - x0;\n"
                          "      stencil(x1, %d, %d, %d, hi, lo); hx1_%d = hi - x0; lx1_%d = lo - x0; }\n",
                          g2, g2, g2, g2, g.n[0], g.bc[0], g2, g2, g2, g.n[0], g.bc[0], g2, g2, g2);
            o += b;
        }
    for (int a = 1; a < 3; ++a) {
        if (!used[a]) continue;
        const long long st = a == 1 ? g.s1 : g.s2;
        const char* pp = a == 1 ? "y" : "z";
        for (int g2 = 0; g2 < 2; ++g2) {
            std::snprintf(b, sizeof b,
                          "    int h%s_%d, l%s_%d;\n"
                          "    { int hi, lo; stencil(%s, %d, %d, %d, hi, lo); h%s_%d = (int)((hi - %s) * %lld); "
                          "l%s_%d = (int)((lo - %s) * %lld); }\n",
                          an[a], g2, an[a], g2, pp, g.n[a], g.bc[a], g2, an[a], g2, pp, st, an[a], g2, pp, st);
            o += b;
        }
    }
    const smg::DevComp& c0 = h->comps[D[P[0]]];
    std::string cond;
    const char* ax[3] = {"x0", "y", "z"};
    for (int a = 0; a < 3; ++a)
        if (c0.ext[a] < g.B[a]) {
            if (!cond.empty()) cond += " && ";
            cond += std::string(ax[a]) + " < " + std::to_string(c0.ext[a]);
        }
    o += cond.empty() ? "    {\n" : "    if (" + cond + ") {\n";
    const bool v1_always = c0.ext[0] % 2 == 0;
    if (!v1_always) o += "    const bool v1 = x1 < " + std::to_string(c0.ext[0]) + ";\n";
    const std::string sel1 = v1_always ? "" : "v1 ? ", sel2 = v1_always ? "" : " : 0";
    o += "    double2* R = smg_ring + threadIdx.x;\n";
    auto slot = [&](int s) { return "R[" + std::to_string(s * block) + "]"; };
    auto issue = [&](const std::vector<PfItem>& v) {
        for (const PfItem& it : v) {
            if (it.kind == 0) {
                std::snprintf(b, sizeof b, "    cpa16(&%s, fp(F, %d) + pt);\n", slot(it.slot[0]).c_str(), it.id);
            } else if (it.kind == 1) {
                const long long so = (long long)it.id * g.cs;
                const int g2 = it.g2;
                std::snprintf(b, sizeof b,
                              "    cpa8(&%s.x, Up + %lld + hx0_%d); cpa8(&%s.y, Up + %lld + lx0_%d);\n"
                              "    cpa8(&%s.x, Up + %lld + (%shx1_%d%s)); cpa8(&%s.y, Up + %lld + (%slx1_%d%s));\n",
                              slot(it.slot[0]).c_str(), so, g2, slot(it.slot[0]).c_str(), so, g2,
                              slot(it.slot[1]).c_str(), so, sel1.c_str(), g2, sel2.c_str(), slot(it.slot[1]).c_str(), so,
                              sel1.c_str(), g2, sel2.c_str());
            } else if (it.kind == 2) {
                const long long so = (long long)it.id * g.cs;
                std::snprintf(b, sizeof b, "    cpa16(&%s, Up + %lld + h%s_%d); cpa16(&%s, Up + %lld + l%s_%d);\n",
                              slot(it.slot[0]).c_str(), so, an[it.a], it.g2, slot(it.slot[1]).c_str(), so, an[it.a],
                              it.g2);
            } else {
                std::snprintf(b, sizeof b, "    cpa16(&%s, Up + %lld);\n", slot(it.slot[0]).c_str(),
                              (long long)it.id * g.cs);
            }
            o += b;
        }
        o += "    cpa_commit();\n";
    };
    issue(items[0]);
    std::set<int> scal_done;
    for (size_t pi = 0; pi < P.size(); ++pi) {
        if (pi + 1 < P.size()) {
            issue(items[pi + 1]);
            o += "    cpa_wait<1>();\n";
        } else {
            o += "    cpa_wait<0>();\n";
        }
        const int j = D[P[pi]];
        const smg::DevComp& c = h->comps[j];
        const Coefs f = coefs_of(h, phase, j);
        int uslot = -1;
        for (const PfItem& it : items[pi]) {
            if (it.kind == 0)
                std::snprintf(b, sizeof b, "    const double2 C%d = %s;\n", it.id, slot(it.slot[0]).c_str());
            else if (it.kind == 1)
                std::snprintf(b, sizeof b,
                              "    const double X%d_a0 = %s.x, X%d_b0 = %s.y, X%d_a1 = %s.x, X%d_b1 = %s.y;\n", it.id,
                              slot(it.slot[0]).c_str(), it.id, slot(it.slot[0]).c_str(), it.id, slot(it.slot[1]).c_str(),
                              it.id, slot(it.slot[1]).c_str());
            else if (it.kind == 2)
                std::snprintf(b, sizeof b, "    const double2 %c%d_h = %s, %c%d_l = %s;\n", it.a == 1 ? 'Y' : 'Z', it.id,
                              slot(it.slot[0]).c_str(), it.a == 1 ? 'Y' : 'Z', it.id, slot(it.slot[1]).c_str());
            else {
                uslot = it.slot[0];
                b[0] = 0;
            }
            o += b;
        }
        auto coef = [&](int fi) {
            const std::string n = "C" + std::to_string(fi);
            if (!is_array(h, fi) && scal_done.insert(fi).second) {
                std::snprintf(b, sizeof b, "    const double %s = fs(F, %d);\n", n.c_str(), fi);
                o += b;
            }
            return std::make_pair(is_array(h, fi) ? n + ".x" : n, is_array(h, fi) ? n + ".y" : n);
        };
        const auto q = coef(f.q), sv = coef(f.s), E = coef(f.E);
        std::pair<std::string, std::string> k1{"1.0", "1.0"}, k2{"1.0", "1.0"};
        if (filt) {
            k1 = coef(f.F1);
            k2 = coef(f.F2);
        }
        std::snprintf(b, sizeof b,
                      "    {\n        double* Uj = U + pt + %lld;\n"
                      "        const double2 u = %s;\n"
                      "        double SA = 0.0, SB = 0.0;\n",
                      (long long)j * g.cs, slot(uslot).c_str());
        o += b;
        bool first = true;
        for (int qq = c.cbeg; qq < c.cend; ++qq) {
            const smg::DevCoup& cp = h->coups[qq];
            const int a = cp.code >> 1;
            const int mode_div = h->exact_recip[a];
            const std::string H = clit(g.h[a]), RH = clit(h->rh[a]), W = clit(cp.w);
            const char* dv = mode_div == 2 ? "div2" : (mode_div == 1 ? "div1" : "div0");
            const char* fold = first ? "SA = tA; SB = tB;" : "SA = __dadd_rn(SA, tA); SB = __dadd_rn(SB, tB);";
            first = false;
            std::string dA, dB;
            if (a == 0) {
                dA = "__dsub_rn(X" + std::to_string(cp.src) + "_a0, X" + std::to_string(cp.src) + "_b0)";
                dB = "__dsub_rn(X" + std::to_string(cp.src) + "_a1, X" + std::to_string(cp.src) + "_b1)";
            } else {
                const std::string n = std::string(1, a == 1 ? 'Y' : 'Z') + std::to_string(cp.src);
                dA = "__dsub_rn(" + n + "_h.x, " + n + "_l.x)";
                dB = "__dsub_rn(" + n + "_h.y, " + n + "_l.y)";
            }
            std::snprintf(b, sizeof b,
                          "        { const double tA = __dmul_rn(%s(%s, %s, %s), %s);\n"
                          "          const double tB = __dmul_rn(%s(%s, %s, %s), %s);\n"
                          "          %s }\n",
                          dv, dA.c_str(), H.c_str(), RH.c_str(), W.c_str(), dv, dB.c_str(), H.c_str(), RH.c_str(),
                          W.c_str(), fold);
            o += b;
        }
        o += "        double u0 = u.x, u1 = u.y;\n";
        auto sub = [&]() {
            std::snprintf(b, sizeof b, "u0 = upd(u0, -SA, %s, %s, %s, hdt); u1 = upd(u1, -SB, %s, %s, %s, hdt);",
                          q.first.c_str(), sv.first.c_str(), E.first.c_str(), q.second.c_str(), sv.second.c_str(),
                          E.second.c_str());
            return std::string(b);
        };
        auto fl = [&](const std::pair<std::string, std::string>& Fp) {
            return filt ? " u0 = __dmul_rn(u0, " + Fp.first + "); u1 = __dmul_rn(u1, " + Fp.second + ");"
                        : std::string();
        };
        if (phase == 0) {
            const std::string one =
                "        " + sub() +
                (filt ? " u0 = __dmul_rn(u0, kf == 1 ? " + k1.first + " : " + k2.first +
                            "); u1 = __dmul_rn(u1, kf == 1 ? " + k1.second + " : " + k2.second + ");"
                      : std::string()) +
                "\n";
            const std::string two = "        " + sub() + fl(k2) + "\n        " + sub() + fl(k1) + "\n";
            if (h->filter_mode == SMG_FILTER_FULL) o += one;
            else o += "        if (mode == 0) {\n" + one + "        } else {\n" + two + "        }\n";
        } else {
            o += "        " + sub() + fl(k1) + "\n        " + sub() + fl(k2) + "\n";
        }
        if (v1_always) o += "        *reinterpret_cast<double2*>(Uj) = make_double2(u0, u1);\n    }\n";
        else o += "        if (v1) *reinterpret_cast<double2*>(Uj) = make_double2(u0, u1); else *Uj = u0;\n    }\n";
    }
    o += "    }\n}\n";
}

// Shape of the staged kernels of a handle.
struct StagedShape {
    int ns, st, nch, rb;
    long long nb;
};

StagedShape staged_shape(const smg_handle* h, int ngroups_phase) {
    const smg::DevGrid& g = h->g;
    StagedShape S;
    S.ns = h->jit_slices;
    S.st = h->jit_stages;
    S.nch = (g.B[0] + kStW - 1) / kStW;
    const long long rows = (long long)g.B[1] * g.B[2];
    if (h->jit_rows > 0) {
        S.rb = (int)std::min<long long>(h->jit_rows, rows);
    } else {
        // about eight waves of two CTAs per SM over the phase's (group, chunk) columns
        const long long cols = std::max(1LL, (long long)ngroups_phase * S.nch);
        S.rb = (int)std::max(1LL, std::min(rows, (rows * cols + 2367) / 2368));
    }
    S.nb = (rows + S.rb - 1) / S.rb;
    return S;
}

// The loader of the plain kernels' staged form (0: none): SMG_TUNE_JIT_STAGED
// 1 (bulk copies) or 2 (asynchronous copies by the consumer warps); never
// with separately compiled groups, and only when every group's ring fits in
// one CTA's shared memory.
int staged_form(const smg_handle* h) {
    const int want = h->jit_staged;
    if (want == 0 || want == 3 || h->jit_calls) return 0;
    for (int phase = 0; phase < 2; ++phase) {
        const std::vector<int> D = phase_dests(h, phase);
        if (D.empty()) continue;
        for (const auto& P : shared_groups(h, phase, h->jit_group)) {
            const long long smem = (16 + (long long)h->jit_stages * staged_rows(h, phase, D, P).nslots() * kStSlot) * 8;
            if (smem > 227LL * 1024) return 0;
        }
    }
    return want;
}

// Kernel over staged groups [k0, k1) of one phase: CTA -> (band, group,
// chunk), band-major, so that the CTAs running at one time cover the same
// rows of every group and the sources they share are read from L2; or
// (group_major) CTA -> (group, band, chunk), every band of a group together.
void emit_staged_dispatch(std::string& o, int phase, int k0, int k1, const StagedShape& S, int minb,
                          const std::string& name, int loader, bool group_major) {
    char b[1024];
    const int ngk = k1 - k0;
    std::string map;
    if (group_major)
        std::snprintf(b, sizeof b,
                      "    const int grp = %d + bid / %lld, rest = bid %% %lld;\n"
                      "    const int band = rest / %d, chunk = rest %% %d;\n",
                      k0, S.nb * S.nch, S.nb * S.nch, S.nch, S.nch);
    else
        std::snprintf(b, sizeof b,
                      "    const int band = bid / %d, rest = bid - band * %d;\n"
                      "    const int grp = %d + rest / %d, chunk = rest %% %d;\n",
                      ngk * S.nch, ngk * S.nch, k0, S.nch, S.nch);
    map = b;
    std::snprintf(b, sizeof b,
                  "extern \"C\" __global__ void __launch_bounds__(%d, %d) %s(double* __restrict__ U, "
                  "const DevField* __restrict__ F, double hdt, int kf, int mode, double* WR, double* PR, int* err) {\n"
                  "    extern __shared__ __align__(128) double smem_st[];\n"
                  "    (void)WR; (void)PR;\n"
                  "    const int bid = (int)blockIdx.x;\n"
                  "%s"
                  "    switch (grp) {\n",
                  32 * (S.ns + (loader == 1 ? 1 : 0)), minb, name.c_str(), map.c_str());
    o += b;
    for (int k = k0; k < k1; ++k)
        o += "    case " + std::to_string(k) + ": " + staged_group_name(phase, k) +
             "(U, F, hdt, kf, mode, err, smem_st, chunk, band); break;\n";
    o += "    default: break;\n    }\n}\n";
}

// One generated kernel: its program, phase type, name, CTA count and, for the
// staged form, CTA size and dynamic shared memory (0: the register form's).
struct KernelSrc {
    std::string src, name;
    int phase;
    long long grid;
    int block = 0;
    int smem = 0;
    int form = 0;   // 0 register form, 1 staged by bulk copies, 2 staged by asynchronous copies, 3 prefetch ring
};

// The generated code of one handle.
//   calls: [0] one dispatch kernel per phase type, then the group functions,
//          `per` groups per program, compiled as relocatable code and linked
//          (one launch per phase; each group is entered by a call);
//   inline (calls false): `per` groups per program (0: all of the phase),
//          each program one kernel over its groups with their code inlined;
//          the kernels of a phase run concurrently.
// Starts up to n helper threads running `work`.  A thread that cannot be
// started (no memory for its stack, a thread limit) is not an error: the
// threads already running and the caller share the work, and no joinable
// thread is left to an unwinding vector (which would end the process).
template <typename F>
void start_workers(std::vector<std::thread>& th, size_t n, F& work) {
    try {
        th.reserve(n);
        for (size_t t = 0; t < n; ++t) th.emplace_back(work);
    } catch (...) {
    }
}

// Runs the generators on up to 16 threads; the programs keep their order.
// An exception in a generator (out of memory) is passed on to the caller.
std::vector<KernelSrc> run_jobs(const std::vector<std::function<KernelSrc()>>& jobs) {
    if (jobs.empty()) return {};
    std::vector<KernelSrc> out(jobs.size());
    std::vector<std::exception_ptr> ex(jobs.size());
    std::atomic<size_t> next(0);
    auto work = [&]() {
        for (size_t i = next++; i < jobs.size(); i = next++) {
            try {
                out[i] = jobs[i]();
            } catch (...) {
                ex[i] = std::current_exception();
            }
        }
    };
    const size_t nt = std::min<size_t>(jobs.size(), std::max(1u, std::min(std::thread::hardware_concurrency(), 16u)));
    std::vector<std::thread> th;
    start_workers(th, nt - 1, work);
    work();
    for (auto& t : th) t.join();
    for (const auto& e : ex)
        if (e) std::rethrow_exception(e);
    return out;
}

std::vector<KernelSrc> programs(const smg_handle* h, int block, int group, int per, bool calls, bool rec = false) {
    const std::string sfx = rec ? "_r" : "";
    const smg::DevGrid& g = h->g;
    const int tpr = (g.B[0] + 1) / 2;
    const long long cta_per_group = (long long)((tpr + block - 1) / block) * g.B[1] * g.B[2];
    std::vector<KernelSrc> P;
    if (calls) {
        KernelSrc disp{kPrelude, "", -1, 0};
        std::vector<std::string> fns;
        for (int phase = 0; phase < 2; ++phase) {
            const std::vector<int> D = phase_dests(h, phase);
            if (D.empty()) continue;
            const int ng = ((int)D.size() + group - 1) / group;
            for (int k = 0; k < ng; ++k) {
                std::string s;
                emit_group(s, h, phase, k, D, group, false, rec);
                fns.push_back(std::move(s));
            }
            emit_dispatch(disp.src, h, phase, 0, ng, block, false, "smg_jit_p" + std::to_string(phase) + sfx, rec);
        }
        P.push_back(std::move(disp));
        const size_t step = per > 0 ? (size_t)per : fns.size();
        for (size_t i = 0; i < fns.size(); i += step) {
            KernelSrc k{kPrelude, "", -1, 0};
            for (size_t j = i; j < std::min(fns.size(), i + step); ++j) k.src += fns[j];
            P.push_back(std::move(k));
        }
        return P;
    }
    // Each program's source depends only on the (read-only) handle, so the
    // programs are generated concurrently: for hundreds of moments the text
    // runs to megabytes and would otherwise add tens of milliseconds to every
    // new handle of a problem whose kernels are already compiled.
    std::vector<int> Ds[2];
    std::vector<std::vector<int>> Gs[2];
    std::vector<std::function<KernelSrc()>> jobs;
    for (int phase = 0; phase < 2; ++phase) {
        Ds[phase] = phase_dests(h, phase);
        if (Ds[phase].empty()) continue;
        Gs[phase] = shared_groups(h, phase, group);
        const std::vector<int>& D = Ds[phase];
        const std::vector<std::vector<int>>& G = Gs[phase];
        const int ng = (int)G.size();
        const int step = per > 0 ? per : ng;
        const int loader = rec ? 0 : staged_form(h);
        if (loader) {
            const StagedShape S = staged_shape(h, ng);
            for (int k0 = 0; k0 < ng; k0 += step) {
                const int k1 = std::min(ng, k0 + step);
                jobs.push_back([h, phase, k0, k1, loader, S, &D, &G]() {
                    int slots = 1;
                    for (int j = k0; j < k1; ++j) slots = std::max(slots, staged_rows(h, phase, D, G[j]).nslots());
                    const long long stage = (long long)slots * kStSlot;
                    const long long smem = (16 + S.st * stage) * 8;
                    const int minb = (int)std::max(1LL, std::min(4LL, (227LL * 1024) / (smem + 1024)));
                    KernelSrc k{std::string(kPrelude) + kStagePrelude,
                                "smg_jit_p" + std::to_string(phase) + "_" + std::to_string(k0), phase,
                                S.nb * (k1 - k0) * S.nch};
                    k.block = 32 * (S.ns + (loader == 1 ? 1 : 0));
                    k.smem = (int)smem;
                    k.form = loader;
                    ConstTable tab;
                    std::string body;
                    g_ctab = h->jit_const ? &tab : nullptr;
                    for (int j = k0; j < k1; ++j)
                        emit_staged_group(body, h, phase, j, G[j], S.ns, S.st, S.rb, stage, loader);
                    g_ctab = nullptr;
                    k.src += ctab_decl(tab) + body;
                    emit_staged_dispatch(k.src, phase, k0, k1, S, minb, k.name, loader, h->jit_band == 0);
                    return k;
                });
            }
            continue;
        }
        for (int k0 = 0; k0 < ng; k0 += step) {
            const int k1 = std::min(ng, k0 + step);
            jobs.push_back([h, phase, k0, k1, block, rec, cta_per_group, &sfx, &D, &G]() {
                const smg::DevGrid& g = h->g;
                const int R = band_rows(h);
                const long long rows = (long long)g.B[1] * g.B[2];
                const long long ctas = R > 0 ? (long long)(k1 - k0) * ((rows + R - 1) / R) * R * (cta_per_group / rows)
                                             : (long long)(k1 - k0) * cta_per_group;
                KernelSrc k{kPrelude, "smg_jit_p" + std::to_string(phase) + "_" + std::to_string(k0) + sfx, phase, ctas};
                ConstTable tab;
                std::string body;
                g_ctab = h->jit_const ? &tab : nullptr;
                int ring = 0;
                if (!rec && h->jit_staged == 3 && !h->jit_xpair && !h->jit_prefetch) {
                    for (int j = k0; j < k1; ++j) ring = std::max(ring, prefetch_ring(prefetch_items(h, phase, D, G[j])));
                    if ((long long)ring * block * 16 > 48 * 1024) ring = 0;   // static shared memory limit
                }
                if (ring > 0) {
                    k.src += kStagePrelude;
                    k.form = 3;
                    body = "__shared__ double2 smg_ring[" + std::to_string(ring * block) + "];\n";
                    for (int j = k0; j < k1; ++j) emit_prefetch_group(body, h, phase, j, G[j], ring, block);
                } else {
                    for (int j = k0; j < k1; ++j) {
                        const int ahead = h->jit_prefetch >= 2 && !rec ? h->jit_prefetch - 1 : 0;
                        const std::vector<int>* nx = (ahead && j + ahead < k1) ? &G[j + ahead] : nullptr;
                        emit_shared_group(body, h, phase, j, G[j], rec, false, nx);
                    }
                }
                g_ctab = nullptr;
                k.src += ctab_decl(tab) + body;
                emit_dispatch(k.src, h, phase, k0, k1, block, true, k.name, rec);
                return k;
            });
        }
    }
    return run_jobs(jobs);
}

// regs > 0: register limit per thread of every function (--maxrregcount);
// the linked kernel's count is the maximum over its call graph
int compile_one(const std::string& src, int regs, bool rdc, std::vector<char>& cubin, std::string& err) {
    Api& a = api();
    nvrtcProgram_t prog = nullptr;
    nvrtcResult_t r = a.CreateProgram(&prog, src.c_str(), "smg_jit.cu", 0, nullptr, nullptr);
    if (r != 0) {
        err = std::string("nvrtcCreateProgram: ") + a.GetErrorString(r);
        return SMG_ECUDA;
    }
    const std::string rr = "--maxrregcount=" + std::to_string(regs);
    const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "--fmad=false",
                          rdc ? "--relocatable-device-code=true" : "--relocatable-device-code=false", rr.c_str()};
    r = a.CompileProgram(prog, regs > 0 ? 5 : 4, opts);
    if (r != 0) {
        size_t n = 0;
        a.GetProgramLogSize(prog, &n);
        std::string log(n, '\0');
        if (n) a.GetProgramLog(prog, &log[0]);
        err = std::string("nvrtcCompileProgram: ") + a.GetErrorString(r) + ": " + log.substr(0, 2000);
        a.DestroyProgram(&prog);
        return SMG_ECUDA;
    }
    size_t n = 0;
    a.GetCUBINSize(prog, &n);
    cubin.assign(n, 0);
    a.GetCUBIN(prog, cubin.data());
    a.DestroyProgram(&prog);
    return SMG_OK;
}

// ---- adjoint kernels -------------------------------------------------------
// One launch set per backward phase r over the sources i of the phase (the
// destinations of the neighbouring phases), with the adjoint kept scaled as
// Y_j = (dU'/dW)_j lambda'_j (see smg_adjoint.cu).  Per target i and point pair:
//   pm:   lambda_i = rho Y_i and the gradient contributions of the pending
//         phase r+1 (i is one of its destinations, slot pslot in the recording)
//   coup: lambda_i -= sum_j M_d(j,i) D_d^T Y_j over phase r's destinations j
//   nm:   Y_i = (dU'/dW)_{r-1,i} lambda_i for the phase before
// The kinds of r+1 and r-1 arrive at run time as (number of substeps, filter
// order swapped); everything else is a constant.


// transposed-coupling terms of target i in phase type l: (destination j,
// axis, grid flag of i along the axis, M_d(j,i)/h), in the fold order of
// smg_adjoint.cu's tables (destination order, then sumcell order)
std::vector<std::tuple<int, int, int, double>> adj_terms(const smg_handle* h, int l, int i) {
    std::vector<std::tuple<int, int, int, double>> T;
    for (int j : phase_dests(h, l))
        for (int q = h->comps[j].cbeg; q < h->comps[j].cend; ++q) {
            const smg::DevCoup& cp = h->coups[q];
            if (cp.src != i) continue;
            const int a = cp.code >> 1;
            T.emplace_back(j, a, cp.code & 1, cp.w / h->g.h[a]);
        }
    return T;
}

// Targets of the backward phases of type l grouped by grid type (one extent
// condition per group), then greedily by the (axis, destination) pairs whose
// transposed differences they read.
std::vector<std::vector<int>> adj_groups(const smg_handle* h, int l, int group) {
    const std::vector<int> T = l == 0 ? h->destB : h->destA;
    std::map<std::vector<int>, std::vector<int>> by_ext;
    std::vector<std::vector<int>> order;
    std::map<int, std::set<std::pair<int, int>>> K;
    for (int i : T) {
        for (const auto& t : adj_terms(h, l, i)) K[i].insert({std::get<1>(t), std::get<0>(t)});
        std::vector<int> e(h->comps[i].ext, h->comps[i].ext + 3);
        if (!by_ext.count(e)) order.push_back(e);
        by_ext[e].push_back(i);
    }
    std::vector<std::vector<int>> G;
    for (const auto& e : order) {
        std::vector<int> left = by_ext[e];
        while (!left.empty()) {
            std::vector<int> g{left.front()};
            left.erase(left.begin());
            std::set<std::pair<int, int>> ks = K[g[0]];
            while ((int)g.size() < group && !left.empty()) {
                size_t best = 0;
                int bestn = -1;
                for (size_t x = 0; x < left.size(); ++x) {
                    int n = 0;
                    for (const auto& k : K[left[x]]) n += (int)ks.count(k);
                    if (n > bestn) {
                        bestn = n;
                        best = x;
                    }
                }
                g.push_back(left[best]);
                ks.insert(K[left[best]].begin(), K[left[best]].end());
                left.erase(left.begin() + best);
            }
            G.push_back(std::move(g));
        }
    }
    // groups in the coupling-graph level order of their targets (their slots in
    // the other phase's level-sorted destination list): concurrent groups
    // share the rows they read while these are in L2
    std::map<int, int> lvl;
    const std::vector<int> Dother = phase_dests(h, 1 - l);
    for (size_t k = 0; k < Dother.size(); ++k) lvl[Dother[k]] = (int)k;
    std::stable_sort(G.begin(), G.end(), [&](const std::vector<int>& x, const std::vector<int>& y) {
        long long sx = 0, sy = 0;
        for (int i : x) sx += lvl[i];
        for (int i : y) sy += lvl[i];
        return sx * (long long)y.size() < sy * (long long)x.size();
    });
    return G;
}

// One group of targets (all on one grid).  Shared at group level: every
// coefficient value and every transposed difference D^T Y_j (per destination
// and axis; it does not depend on the target); per target: Y_i, the pending
// pointwise part (pm), the fold of its terms (coup), the rescaling (nm), the
// store.  Sigma-gradient contributions are summed per field and added once.
void emit_adj_group(std::string& o, const smg_handle* h, int l, const std::vector<int>& tg) {
    const smg::DevGrid& g = h->g;
    char b[4096];
    const std::vector<int> Dother = phase_dests(h, 1 - l);
    const bool filt = h->filter_mode == SMG_FILTER_SUBSTEP;
    const smg::DevComp& c0 = h->comps[tg[0]];
    std::string cond;
    const char* ax[3] = {"x0", "y", "z"};
    for (int a = 0; a < 3; ++a)
        if (c0.ext[a] < g.B[a]) {
            if (!cond.empty()) cond += " && ";
            cond += std::string(ax[a]) + " < " + std::to_string(c0.ext[a]);
        }
    // gradient accumulators per sigma field of the group
    std::map<int, int> fields;
    for (int i : tg) fields.emplace(coefs_of(h, 1 - l, i).s, i);
    for (const auto& fe : fields) {
        std::snprintf(b, sizeof b, "    double gs%d_0 = 0.0, gs%d_1 = 0.0;\n", fe.first, fe.first);
        o += b;
    }
    o += cond.empty() ? "    {\n" : "    if (" + cond + ") {\n";
    const bool v1_always = c0.ext[0] % 2 == 0;
    o += std::string("    const bool v1 = ") + (v1_always ? "true" : ("x1 < " + std::to_string(c0.ext[0])).c_str()) +
         ";\n";
    std::set<int> cdone;
    auto coef = [&](int f) {
        const std::string n = "C" + std::to_string(f);
        if (cdone.insert(f).second) {
            if (is_array(h, f)) std::snprintf(b, sizeof b, "    const double2 %s = L2(fp(F, %d) + pt);\n", n.c_str(), f);
            else std::snprintf(b, sizeof b, "    const double %s = fs(F, %d);\n", n.c_str(), f);
            o += b;
        }
        return std::make_pair(is_array(h, f) ? n + ".x" : n, is_array(h, f) ? n + ".y" : n);
    };
    std::set<std::pair<int, int>> tdone;
    auto tval = [&](int j, int a, int g2) {   // D^T Y_j along axis a at the point pair
        const std::string n = "T" + std::to_string(a) + "_" + std::to_string(j);
        if (tdone.insert({a, j}).second) {
            if (a == 0)
                std::snprintf(b, sizeof b,
                              "    const double %s_0 = dT(Y + pt + %lld, x0, %d, %d, %d, 1), "
                              "%s_1 = v1 ? dT(Y + pt + %lld + 1, x1, %d, %d, %d, 1) : 0.0;\n",
                              n.c_str(), (long long)j * g.cs, g.n[0], g.bc[0], g2, n.c_str(), (long long)j * g.cs,
                              g.n[0], g.bc[0], g2);
            else
                std::snprintf(b, sizeof b, "    const double2 %s = dT_row(Y + pt + %lld, %s, %d, %d, %d, %lld);\n",
                              n.c_str(), (long long)j * g.cs, a == 1 ? "y" : "z", g.n[a], g.bc[a], g2,
                              a == 1 ? (long long)g.s1 : (long long)g.s2);
            o += b;
        }
        return a == 0 ? std::make_pair(n + "_0", n + "_1") : std::make_pair(n + ".x", n + ".y");
    };
    for (int i : tg) {
        int pslot = -1;
        for (size_t k = 0; k < Dother.size(); ++k)
            if (Dother[k] == i) pslot = (int)k;
        const Coefs f = coefs_of(h, 1 - l, i);
        const auto sv = coef(f.s), E = coef(f.E);
        std::pair<std::string, std::string> k1{"1.0", "1.0"}, k2{"1.0", "1.0"};
        if (filt) {
            k1 = coef(f.F1);
            k2 = coef(f.F2);
        }
        const auto terms = adj_terms(h, l, i);
        std::vector<std::pair<double, std::pair<std::string, std::string>>> tv;
        if (!terms.empty()) {
            // the transposed differences at group scope (shared with later targets)
            for (const auto& t : terms) tv.push_back({std::get<3>(t), tval(std::get<0>(t), std::get<1>(t), std::get<2>(t))});
            o += "    double ta0_" + std::to_string(i) + " = 0.0, ta1_" + std::to_string(i) + " = 0.0;\n";
            o += "    if (coup) {\n";
            for (const auto& t : tv) {
                std::snprintf(b, sizeof b, "      ta0_%d += %s * %s; ta1_%d += %s * %s;\n", i, lit(t.first).c_str(),
                              t.second.first.c_str(), i, lit(t.first).c_str(), t.second.second.c_str());
                o += b;
            }
            o += "    }\n";
        }
        std::snprintf(b, sizeof b, "    {\n        double* Yi = Y + pt + %lld;\n"
                                   "        const double2 yv = L2(Yi); double l0 = yv.x, l1 = yv.y;\n",
                      (long long)i * g.cs);
        o += b;
        if (pslot >= 0) {
            const std::string F0 = filt ? "(pm_swap ? " + k2.first + " : " + k1.first + ")" : "1.0";
            const std::string F1 = filt ? "(pm_swap ? " + k2.second + " : " + k1.second + ")" : "1.0";
            std::snprintf(b, sizeof b,
                          "        if (pm) {\n"
                          "          double* gq = %s;\n"
                          "          const long long rp = %lld + pt;\n"
                          "          l0 = pend_ds(pm, WR[rp], l0, %s, %s, %s, gs%d_0, gq, pt, hdt);\n"
                          "          if (v1) l1 = pend_ds(pm, WR[rp + 1], l1, %s, %s, %s, gs%d_1, gq, pt + 1, hdt);\n"
                          "        }\n",
                          f.q == h->field_zero ? "nullptr" : ("Gt[" + std::to_string(f.q) + "]").c_str(),
                          (long long)pslot * g.cs, sv.first.c_str(), E.first.c_str(), F0.c_str(), f.s,
                          sv.second.c_str(), E.second.c_str(), F1.c_str(), f.s);
            o += b;
        }
        if (!terms.empty()) {
            std::snprintf(b, sizeof b, "        l0 -= ta0_%d; l1 -= ta1_%d;\n", i, i);
            o += b;
        }
        if (pslot >= 0) {
            const std::string a0 = filt ? "(nm_swap ? " + k2.first + " : " + k1.first + ")" : "1.0";
            const std::string a1 = filt ? "(nm_swap ? " + k2.second + " : " + k1.second + ")" : "1.0";
            const std::string z0 = filt ? "(nm_swap ? " + k1.first + " : " + k2.first + ")" : "1.0";
            const std::string z1 = filt ? "(nm_swap ? " + k1.second + " : " + k2.second + ")" : "1.0";
            std::snprintf(b, sizeof b,
                          "        if (nm) { l0 *= dwdu(nm, %s, %s, %s, %s, hdt); l1 *= dwdu(nm, %s, %s, %s, %s, hdt); }\n",
                          sv.first.c_str(), E.first.c_str(), a0.c_str(), z0.c_str(), sv.second.c_str(),
                          E.second.c_str(), a1.c_str(), z1.c_str());
            o += b;
        }
        o += "        if (v1) *reinterpret_cast<double2*>(Yi) = make_double2(l0, l1); else Yi[0] = l0;\n    }\n";
    }
    o += "    }\n";
    for (const auto& fe : fields) {
        std::string c2 = "pm";
        for (int a = 0; a < 3; ++a)
            if (c0.ext[a] < g.B[a]) c2 += std::string(" && ") + ax[a] + " < " + std::to_string(c0.ext[a]);
        std::snprintf(b, sizeof b,
                      "    if (%s) { double* gp = Gt[%d]; if (gp) { atomicAdd(gp + pt, gs%d_0); "
                      "if (x1 < %d) atomicAdd(gp + pt + 1, gs%d_1); } }\n",
                      c2.c_str(), fe.first, fe.first, c0.ext[0], fe.first);
        o += b;
    }
}

const char* kAdjArgs =
    "(double* __restrict__ Y, const DevField* __restrict__ F, const DevField* __restrict__ DE, "
    "double* const* __restrict__ Gt, const double* __restrict__ PRE, const double* __restrict__ WR, int pm_a, "
    "int pm_swap_a, int nm_a, int nm_swap_a, int coup_a, double hdt";

// kernels over the targets of backward phases of type l (l = 0: A phases,
// whose sources are the B destinations; l = 1: B phases)
std::vector<KernelSrc> adj_programs(const smg_handle* h, int block, int group, int per) {
    const smg::DevGrid& g = h->g;
    const int tpr = (g.B[0] + 1) / 2;
    const int nchunks = (tpr + block - 1) / block;
    const long long cta_per_group = (long long)nchunks * g.B[1] * g.B[2];
    std::vector<KernelSrc> P;
    for (int l = 0; l < 2; ++l) {
        const std::vector<std::vector<int>> G = adj_groups(h, l, group);
        if (G.empty()) continue;
        const int ng = (int)G.size();
        const int step = per > 0 ? per : ng;
        // two forms of every kernel: the general one takes the kinds of the
        // phases before and after at run time; the steady one has them fixed to
        // the interior of a run (both neighbours two-substep phases: fused
        // A-A around a B phase, B around an A phase), with far less code
        for (int form = 0; form < 2; ++form)
        for (int k0 = 0; k0 < ng; k0 += step) {
            const int k1 = std::min(ng, k0 + step);
            const std::string tag = form ? "s" : "p";
            KernelSrc K{std::string(kPrelude) + kAdjPrelude,
                        "smg_adj_" + tag + std::to_string(l) + "_" + std::to_string(k0), l + 2 * form,
                        (long long)(k1 - k0) * cta_per_group};
            for (int k = k0; k < k1; ++k) {
                K.src += "static __device__ __forceinline__ void smg_ag" + std::to_string(l) + "_" + std::to_string(k) +
                         std::string(kAdjArgs) + ", int x0, int y, int z) {\n"
                         "    const int x1 = x0 + 1; (void)x1;\n";
                if (form)
                    K.src += "    constexpr int pm = 2, nm = 2, coup = 1, pm_swap = " + std::to_string(l) +
                             ", nm_swap = " + std::to_string(l) + ";\n";
                else
                    K.src += "    const int pm = pm_a, nm = nm_a, coup = coup_a, pm_swap = pm_swap_a, nm_swap = nm_swap_a;\n";
                K.src += "    (void)pm; (void)nm; (void)coup; (void)pm_swap; (void)nm_swap;\n";
                char b[512];
                std::snprintf(b, sizeof b, "    const int pt = z * %lld + y * %lld + x0;\n", (long long)g.s2,
                              (long long)g.s1);
                K.src += b;
                emit_adj_group(K.src, h, l, G[k]);
                K.src += "}\n";
            }
            char b[1024];
            std::snprintf(b, sizeof b,
                          "extern \"C\" __global__ void __launch_bounds__(%s) %s%s) {\n"
                          "    const int bid = blockIdx.x;\n"
                          "    const int grp = %d + bid / %lld;\n"
                          "    const int rest = bid %% %lld;\n"
                          "    const int row = rest / %d, chunk = rest - row * %d;\n"
                          "    const int y = row %% %d, z = row / %d;\n"
                          "    const int x0 = 2 * (chunk * %d + (int)threadIdx.x);\n"
                          "    if (x0 >= %d) return;\n"
                          "    switch (grp) {\n",
                          bounds(block, h->jit_regs).c_str(), K.name.c_str(), kAdjArgs, k0, cta_per_group,
                          cta_per_group, nchunks, nchunks, g.B[1], g.B[1], block, g.B[0]);
            K.src += b;
            for (int k = k0; k < k1; ++k)
                K.src += "    case " + std::to_string(k) + ": smg_ag" + std::to_string(l) + "_" + std::to_string(k) +
                         "(Y, F, DE, Gt, PRE, WR, pm_a, pm_swap_a, nm_a, nm_swap_a, coup_a, hdt, x0, y, z); break;\n";
            K.src += "    default: break;\n    }\n}\n";
            P.push_back(std::move(K));
        }
    }
    return P;
}

// ---- family kernels for the batched solver ---------------------------------
// Instances whose generated code would be equal apart from the grid (same
// closure and order, dimensions, boundary conditions, which coefficients are
// arrays, filter mode) form a family and share kernels; the grid sizes,
// strides, spacing and dt/2 of each instance come from a FamGeom table.  The
// groups are the plain kernels' shared-load groups in level order, emitted
// in the family form of emit_shared_group.  A CTA takes one (instance,
// group, chunk, row) item from its kernel's list.
std::vector<KernelSrc> fam_programs(const smg_handle* h, int block, int group, int per) {
    const smg::DevGrid& g = h->g;
    std::vector<KernelSrc> P;
    const int e0 = g.B[0] - g.n[0], e1 = g.B[1] - g.n[1];   // box extent beyond n (0 or 1)
    for (int phase = 0; phase < 2; ++phase) {
        const std::vector<int> D = phase_dests(h, phase);
        if (D.empty()) continue;
        // the plain kernels' shared-load groups, in coupling-level order
        const std::vector<std::vector<int>> G = shared_groups(h, phase, group);
        const int ng = (int)G.size();
        const int step = per > 0 ? per : ng;
        for (int k0 = 0; k0 < ng; k0 += step) {
            const int k1 = std::min(ng, k0 + step);
            // grid: the group count (the work items are built per batch)
            KernelSrc K{kPrelude, "smg_fam_p" + std::to_string(phase) + "_" + std::to_string(k0), phase, k1 - k0};
            ConstTable tab;
            std::string body;
            g_ctab = h->jit_const ? &tab : nullptr;
            for (int k = k0; k < k1; ++k) emit_shared_group(body, h, phase, k, G[k], false, true);
            g_ctab = nullptr;
            K.src += ctab_decl(tab) + body;
            char b[1024];
            std::snprintf(b, sizeof b,
                          "extern \"C\" __global__ void __launch_bounds__(%s) %s(const FamGeom* __restrict__ geo, "
                          "const int4* __restrict__ items, int kf, int mode) {\n"
                          "    const int4 it = items[blockIdx.x];\n"
                          "    const FamGeom& G = geo[it.x];\n"
                          "    const int B1 = G.n[1] + %d;\n"
                          "    const int y = it.w %% B1, z = it.w / B1;\n"
                          "    const int x0 = 2 * (it.z * %d + (int)threadIdx.x);\n"
                          "    if (x0 >= G.n[0] + %d) return;\n"
                          "    switch (it.y) {\n",
                          bounds(block, h->jit_regs).c_str(), K.name.c_str(), e1, block, e0);
            K.src += b;
            for (int k = k0; k < k1; ++k)
                K.src += "    case " + std::to_string(k) + ": " + group_name(phase, k) + "(G, kf, mode, x0, y, z); break;\n";
            K.src += "    default: break;\n    }\n}\n";
            P.push_back(std::move(K));
        }
    }
    return P;
}

std::map<std::string, std::vector<std::vector<char>>> g_cubins;   // sources -> cubins, process-wide
std::mutex g_cubin_mu;
std::atomic<long long> g_programs_compiled(0), g_programs_from_disk(0);

// ---- on-disk cache of compiled kernels ----------------------------------------
// A process's first compilation of a problem's kernels takes seconds (NVRTC on
// all host threads); a MATLAB session calling starmap_solver would pay it on
// every first call.  The cubins are therefore also kept on disk, one file per
// (sources, options, NVRTC version, library version), named by two 64-bit
// FNV-1a hashes of that key and holding the key's length for a check.
// Directory: $SMG_JIT_CACHE_DIR, else $XDG_CACHE_HOME/starmap_b200, else
// $HOME/.cache/starmap_b200; SMG_JIT_CACHE=0 turns the cache off.  Files are
// written to a temporary name and renamed, so concurrent processes see whole
// files only.
unsigned long long fnv1a(const std::string& s, unsigned long long h) {
    for (unsigned char c : s) {
        h ^= c;
        h *= 1099511628211ull;
    }
    return h;
}

std::string cache_dir() {
    const char* off = std::getenv("SMG_JIT_CACHE");
    if (off && std::string(off) == "0") return "";
    if (const char* d = std::getenv("SMG_JIT_CACHE_DIR")) return *d ? std::string(d) : "";
    if (const char* x = std::getenv("XDG_CACHE_HOME"))
        if (*x) return std::string(x) + "/starmap_b200";
    if (const char* hm = std::getenv("HOME"))
        if (*hm) return std::string(hm) + "/.cache/starmap_b200";
    return "";
}

// mkdir -p
bool make_dirs(const std::string& d) {
    for (size_t i = 1; i <= d.size(); ++i)
        if (i == d.size() || d[i] == '/') {
            const std::string p = d.substr(0, i);
            if (mkdir(p.c_str(), 0755) != 0 && errno != EEXIST) return false;
        }
    return true;
}

std::string cache_file(const std::string& key) {
    const std::string d = cache_dir();
    if (d.empty()) return "";
    char name[64];
    std::snprintf(name, sizeof name, "/%016llx%016llx.cubins", fnv1a(key, 1469598103934665603ull),
                  fnv1a(key, 0x9e3779b97f4a7c15ull));
    return d + name;
}

// File format: "SMGCUB2\n", the key's length and bytes (the whole source
// with the options, compared in full on load: a file is used only for
// exactly its own key), the number of cubins, each cubin's size and bytes,
// and a checksum over the cubins.  A file that does not hold `count` cubins
// or whose checksum differs (truncated, corrupted) is ignored.
unsigned long long cubins_checksum(const std::vector<std::vector<char>>& v) {
    unsigned long long h = 0x6a09e667f3bcc909ull;
    for (const auto& c : v) h = bytes_hash(c, h ^ c.size(), 0x9e3779b97f4a7c15ull);
    return h;
}

bool cache_load(const std::string& key, size_t count, std::vector<std::vector<char>>& out) {
    const std::string f = cache_file(key);
    if (f.empty()) return false;
    FILE* fp = std::fopen(f.c_str(), "rb");
    if (!fp) return false;
    char magic[8] = {0};
    unsigned long long klen = 0, n = 0, sum = 0;
    bool ok = std::fread(magic, 1, 8, fp) == 8 && std::memcmp(magic, "SMGCUB2\n", 8) == 0 &&
              std::fread(&klen, sizeof klen, 1, fp) == 1 && klen == key.size();
    if (ok) {
        std::string k(key.size(), '\0');
        ok = std::fread(&k[0], 1, k.size(), fp) == k.size() && k == key;
    }
    ok = ok && std::fread(&n, sizeof n, 1, fp) == 1 && n == count;
    std::vector<std::vector<char>> v;
    for (unsigned long long i = 0; ok && i < n; ++i) {
        unsigned long long sz = 0;
        ok = std::fread(&sz, sizeof sz, 1, fp) == 1 && sz > 0 && sz < (1ull << 31);
        if (!ok) break;
        v.emplace_back(sz);
        ok = std::fread(v.back().data(), 1, sz, fp) == sz;
    }
    ok = ok && std::fread(&sum, sizeof sum, 1, fp) == 1 && sum == cubins_checksum(v);
    std::fclose(fp);
    if (!ok) return false;
    out = std::move(v);
    return true;
}

void cache_store(const std::string& key, const std::vector<std::vector<char>>& cub) {
    const std::string f = cache_file(key);
    if (f.empty() || !make_dirs(cache_dir())) return;
    const std::string tmp = f + "." + std::to_string((long long)getpid()) + ".tmp";
    FILE* fp = std::fopen(tmp.c_str(), "wb");
    if (!fp) return;
    const unsigned long long klen = key.size(), n = cub.size(), sum = cubins_checksum(cub);
    bool ok = std::fwrite("SMGCUB2\n", 1, 8, fp) == 8 && std::fwrite(&klen, sizeof klen, 1, fp) == 1 &&
              std::fwrite(key.data(), 1, key.size(), fp) == key.size() && std::fwrite(&n, sizeof n, 1, fp) == 1;
    for (const auto& c : cub) {
        const unsigned long long sz = c.size();
        ok = ok && std::fwrite(&sz, sizeof sz, 1, fp) == 1 && std::fwrite(c.data(), 1, sz, fp) == sz;
    }
    ok = ok && std::fwrite(&sum, sizeof sum, 1, fp) == 1;
    ok = std::fclose(fp) == 0 && ok;
    if (ok) ok = std::rename(tmp.c_str(), f.c_str()) == 0;
    if (!ok) std::remove(tmp.c_str());
}

// Compile the programs on all host threads; for the calls layout link them
// into one cubin, for the inline layout keep one cubin per program.  Cached
// per process by source text and options.
int compile_programs(const std::vector<KernelSrc>& P, int regs, bool calls, std::vector<std::vector<char>>& out,
                     std::string& err) {
    Api& a = api();
    std::string key = "regs " + std::to_string(regs) + (calls ? " calls\n" : " inline\n");
    {
        int major = 0, minor = 0;
        if (a.ok) a.Version(&major, &minor);
        key += "nvrtc " + std::to_string(major) + "." + std::to_string(minor) + " " + smg_version() + "\n";
    }
    for (const auto& k : P) key += k.src;
    {
        std::lock_guard<std::mutex> lk(g_cubin_mu);
        auto it = g_cubins.find(key);
        if (it != g_cubins.end()) {
            out = it->second;
            return SMG_OK;
        }
    }
    const bool link = calls && P.size() > 1;
    if (a.ok && cache_load(key, link ? 1 : P.size(), out)) {
        g_programs_from_disk += (long long)P.size();
        std::lock_guard<std::mutex> lk(g_cubin_mu);
        g_cubins[key] = out;
        return SMG_OK;
    }
    if (!a.ok) {
        err = a.why;
        return SMG_EINVAL;
    }
    if (link && !a.link_ok) {
        err = a.link_why;
        return SMG_EINVAL;
    }
    std::vector<std::vector<char>> obj(P.size());
    std::vector<std::string> errs(P.size());
    std::vector<int> rcs(P.size(), SMG_OK);
    std::atomic<size_t> next(0);
    const unsigned nt = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), 64));
    auto work = [&]() {
        for (size_t i = next++; i < P.size(); i = next++) rcs[i] = compile_one(P[i].src, regs, link, obj[i], errs[i]);
    };
    std::vector<std::thread> th;
    if (!P.empty()) start_workers(th, std::min<size_t>(nt, P.size()) - 1, work);
    work();
    for (auto& t : th) t.join();
    for (size_t i = 0; i < P.size(); ++i)
        if (rcs[i] != SMG_OK) {
            err = errs[i];
            return rcs[i];
        }
    if (!link) {
        out = std::move(obj);
    } else {
        nvJitLinkHandle_t L = nullptr;
        const char* lopts[] = {"-arch=sm_100a"};
        if (a.LinkCreate(&L, 1, lopts) != 0) {
            err = "nvJitLinkCreate failed";
            return SMG_ECUDA;
        }
        int rc = SMG_OK;
        for (size_t i = 0; i < P.size() && rc == SMG_OK; ++i) {
            const std::string name = "smg_jit_" + std::to_string(i) + ".cubin";
            if (a.LinkAddData(L, kJitLinkInputCubin, obj[i].data(), obj[i].size(), name.c_str()) != 0) rc = SMG_ECUDA;
        }
        if (rc == SMG_OK && a.LinkComplete(L) != 0) rc = SMG_ECUDA;
        if (rc != SMG_OK) {
            size_t n = 0;
            a.LinkErrorLogSize(L, &n);
            std::string log(n, '\0');
            if (n) a.LinkErrorLog(L, &log[0]);
            err = "nvJitLink: " + log.substr(0, 2000);
            a.LinkDestroy(&L);
            return rc;
        }
        size_t n = 0;
        a.LinkedCubinSize(L, &n);
        out.assign(1, std::vector<char>(n, 0));
        a.LinkedCubin(L, out[0].data());
        a.LinkDestroy(&L);
    }
    g_programs_compiled += (long long)P.size();
    cache_store(key, out);
    std::lock_guard<std::mutex> lk(g_cubin_mu);
    g_cubins[key] = out;
    return SMG_OK;
}

}  // namespace

namespace smg {

struct JitKernel {
    CUfunction_t fn = nullptr;
    long long grid = 0;
    int block = 0;   // CTA size (0: the state's)
    int smem = 0;    // dynamic shared memory (staged form)
    int form = 0;    // as KernelSrc::form
};

struct JitState {
    std::vector<CUmodule_t> mods;
    std::vector<JitKernel> k[4];           // kernels of each phase type (adjoint: 2, 3 the steady forms)
    int block = 64;
    int* dErr = nullptr;                   // error flag of the staged kernels (a bounded wait ran out)
    std::vector<cudaStream_t> side;        // concurrent kernels of a phase (inline layout)
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
};

std::string jit_source(const smg_handle* h, int block, int group) {
    std::string o;
    int i = 0;
    for (const KernelSrc& k : programs(h, block, group, h->jit_split, h->jit_calls))
        o += "// ---- program " + std::to_string(i++) + (k.name.empty() ? "" : " (" + k.name + ")") + "\n" + k.src;
    return o;
}

int jit_compile(const smg_handle* h, int block, int group, std::string& err) {
    std::vector<std::vector<char>> cubins;
    return compile_programs(programs(h, block, group, h->jit_split, h->jit_calls), 64, h->jit_calls, cubins, err);
}

void free_state(JitState*& J) {
    if (!J) return;
    for (cudaStream_t st : J->side) cudaStreamDestroy(st);
    if (J->fork) cudaEventDestroy(J->fork);
    for (cudaEvent_t e : J->join) cudaEventDestroy(e);
    if (J->dErr) cudaFree(J->dErr);
    if (api().cu_ok)
        for (CUmodule_t m : J->mods) release_module(m);
    delete J;
    J = nullptr;
}

void jit_free(smg_handle* h) {
    free_state(h->jit);
    free_state(h->jit_rec);
    free_state(h->jit_adj);
}

namespace {

// Generate, compile and load one form of the kernels (plain or recording).
// Generated programs and their cubins per generator input, shared by the
// handles of a process: a second handle of the same problem (a new
// starmap_solver call, the instances of an ensemble) skips writing the
// sources again (megabytes of text for hundreds of moments) and the lookup
// of their cubins by source text.  The key holds every handle field the
// generator reads, so equal keys give equal programs.  At most 8 entries,
// the least recently used dropped.
struct Built {
    std::vector<KernelSrc> P;
    std::vector<std::vector<char>> cubins;
};
std::mutex g_built_mu;
std::list<std::pair<std::string, std::shared_ptr<const Built>>> g_built;   // most recent first
constexpr size_t kBuiltMax = 8;
static_assert(sizeof(smg::DevComp) == 11 * sizeof(int), "DevComp is all ints (serialised as bytes)");

std::string generator_key(const smg_handle* h, int block, int group, int per, bool calls, bool rec) {
    std::string k;
    k.reserve(64 + h->comps.size() * 48 + h->coups.size() * 24);
    auto put = [&](const void* p, size_t n) { k.append(static_cast<const char*>(p), n); };
    auto i64 = [&](long long v) { put(&v, sizeof v); };
    auto f64 = [&](double v) { put(&v, sizeof v); };
    for (long long v : {(long long)block, (long long)group, (long long)per, (long long)calls, (long long)rec,
                        (long long)h->n_sys, (long long)h->filter_mode, (long long)h->field_one,
                        (long long)h->field_zero, (long long)h->sigma_a, (long long)h->decay_a,
                        (long long)h->derived_decay_a, (long long)h->jit_block, (long long)h->jit_group,
                        (long long)h->jit_split, (long long)h->jit_calls, (long long)h->jit_xpair,
                        (long long)h->jit_prefetch, (long long)h->jit_band, (long long)h->jit_const,
                        (long long)h->jit_regs, (long long)h->jit_staged, (long long)h->jit_slices,
                        (long long)h->jit_stages, (long long)h->jit_rows})
        i64(v);
    const smg::DevGrid& g = h->g;
    for (int a = 0; a < 3; ++a) {
        i64(g.n[a]);
        i64(g.bc[a]);
        i64(g.B[a]);
        f64(g.h[a]);
        f64(h->rh[a]);
        i64(h->exact_recip[a]);
    }
    i64(g.s1);
    i64(g.s2);
    i64(g.cs);
    i64((long long)h->comps.size());
    put(h->comps.data(), h->comps.size() * sizeof(smg::DevComp));
    i64((long long)h->coups.size());
    for (const smg::DevCoup& c : h->coups) {
        i64(c.src);
        i64(c.code);
        f64(c.w);
    }
    for (const std::vector<int>* v : {&h->destA, &h->destB, &h->derived_decay}) {
        i64((long long)v->size());
        for (int x : *v) i64(x);
    }
    for (int ph = 0; ph < 2; ++ph) {
        i64(h->pair[ph].ok);
        i64((long long)h->pair[ph].dests.size());
        for (const auto& d : h->pair[ph].dests) i64(d.off);
    }
    i64((long long)h->field_is_array.size());
    put(h->field_is_array.data(), h->field_is_array.size());
    return k;
}

std::shared_ptr<const Built> built_find(const std::string& key) {
    std::lock_guard<std::mutex> lk(g_built_mu);
    for (auto it = g_built.begin(); it != g_built.end(); ++it)
        if (it->first == key) {
            g_built.splice(g_built.begin(), g_built, it);
            return g_built.front().second;
        }
    return nullptr;
}

void built_store(const std::string& key, std::shared_ptr<const Built> b) {
    std::lock_guard<std::mutex> lk(g_built_mu);
    g_built.emplace_front(key, std::move(b));
    while (g_built.size() > kBuiltMax) g_built.pop_back();
}

int build_state(smg_handle* h, bool rec, JitState*& out, std::string& err) {
    if (!(h->pair[0].ok && h->pair[1].ok)) {
        err = "the problem exceeds 32-bit element offsets";
        return SMG_EINVAL;
    }
    Api& a = api();
    if (!a.cu_ok) {
        err = a.cu_why;
        return SMG_EINVAL;
    }
    const int block = h->jit_block, group = h->jit_group;
    const bool calls = h->jit_calls != 0;
    const std::string gkey = generator_key(h, block, group, h->jit_split, calls, rec);
    std::shared_ptr<const Built> B = built_find(gkey);
    if (!B) {
        auto nb = std::make_shared<Built>();
        nb->P = programs(h, block, group, h->jit_split, calls, rec);
        const int rc = compile_programs(nb->P, h->jit_regs, calls, nb->cubins, err);
        if (rc != SMG_OK) return rc;
        built_store(gkey, nb);
        B = nb;
    }
    const std::vector<KernelSrc>& P = B->P;
    const std::vector<std::vector<char>>& cubins = B->cubins;
    JitState* J = new JitState();
    J->block = block;
    auto fail = [&](const std::string& m) {
        err = m;
        free_state(J);
        return SMG_ECUDA;
    };
    for (const auto& c : cubins) {
        CUmodule_t m = nullptr;
        if (load_module(c, &m) != 0) return fail("cuModuleLoadData failed");
        J->mods.push_back(m);
    }
    if (calls) {
        const int tpr = (h->g.B[0] + 1) / 2;
        const long long per = (long long)((tpr + block - 1) / block) * h->g.B[1] * h->g.B[2];
        for (int phase = 0; phase < 2; ++phase) {
            const std::vector<int> D = phase_dests(h, phase);
            if (D.empty()) continue;
            JitKernel k;
            k.grid = ((long long)D.size() + group - 1) / group * per;
            const std::string name = "smg_jit_p" + std::to_string(phase) + (rec ? "_r" : "");
            if (a.ModuleGetFunction(&k.fn, J->mods[0], name.c_str()) != 0) return fail("cuModuleGetFunction " + name);
            J->k[phase].push_back(k);
        }
    } else {
        for (size_t i = 0; i < P.size(); ++i) {
            JitKernel k;
            k.grid = P[i].grid;
            k.block = P[i].block;
            k.smem = P[i].smem;
            k.form = P[i].form;
            if (a.ModuleGetFunction(&k.fn, J->mods[i], P[i].name.c_str()) != 0)
                return fail("cuModuleGetFunction " + P[i].name);
            if (k.smem > 48 * 1024 && a.FuncSetAttribute(k.fn, kFuncAttrMaxDynamicSmem, k.smem) != 0)
                return fail("cuFuncSetAttribute " + P[i].name + " (" + std::to_string(k.smem) + " bytes of shared memory)");
            if (k.form == 1 && !J->dErr) {
                if (cudaMalloc(&J->dErr, sizeof(int)) != cudaSuccess) return fail("cudaMalloc (staged kernels' flag)");
                if (cudaMemset(J->dErr, 0, sizeof(int)) != cudaSuccess) return fail("cudaMemset");
            }
            J->k[P[i].phase].push_back(k);
        }
    }
    const size_t nk = std::max(std::max(J->k[0].size(), J->k[1].size()), std::max(J->k[2].size(), J->k[3].size()));
    if (nk > 1) {
        if (cudaEventCreateWithFlags(&J->fork, cudaEventDisableTiming) != cudaSuccess) return fail("cudaEventCreate");
        for (size_t i = 0; i < nk; ++i) {
            cudaStream_t st = nullptr;
            cudaEvent_t ev = nullptr;
            if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return fail("cudaStreamCreate");
            J->side.push_back(st);
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return fail("cudaEventCreate");
            J->join.push_back(ev);
        }
    }
    out = J;
    return SMG_OK;
}

// One phase of state J: its kernel, or its kernels forked onto the side
// streams after the work already queued on s and joined back into s (inside
// a stream capture this becomes parallel branches of the graph).
cudaError_t launch_state(const smg_handle* h, JitState* J, double* U, int mode, int kfilter, double* wrec,
                         double* prec, cudaStream_t s, const DevField* DE = nullptr, int dsm = 1, int dsw = 0) {
    const int phase = mode == 1 ? 1 : 0;
    const std::vector<JitKernel>& K = J->k[phase];
    if (K.empty()) return cudaSuccess;
    const DevField* F = h->dFieldTab;
    double hdt = h->hdt;
    int kf = kfilter;
    int md = mode;
    int* err = J->dErr;
    // plain kernels: (U, F, hdt, kf, mode[, -, -, err]); recording kernels:
    // (U, F, hdt, kf, mode, WR, PR, DE, dsm, dsw)
    void* args_plain[] = {&U, &F, &hdt, &kf, &md, &wrec, &prec, &err};
    void* args_rec[] = {&U, &F, &hdt, &kf, &md, &wrec, &prec, &DE, &dsm, &dsw};
    void** args = wrec ? args_rec : args_plain;
    auto go = [&](const JitKernel& k, cudaStream_t st) {
        const unsigned blk = (unsigned)(k.block > 0 ? k.block : J->block);
        return api().LaunchKernel(k.fn, (unsigned)k.grid, 1, 1, blk, 1, 1, (unsigned)k.smem, st, args, nullptr) == 0
                   ? cudaSuccess
                   : cudaErrorLaunchFailure;
    };
    if (K.size() == 1) return go(K[0], s);
    // at most `lanes` kernels at a time: kernel i runs on side stream i mod
    // lanes, after kernel i - lanes
    const size_t lanes = h->jit_lanes > 0 ? std::min<size_t>((size_t)h->jit_lanes, K.size()) : K.size();
    cudaError_t e = cudaEventRecord(J->fork, s);
    if (e != cudaSuccess) return e;
    for (size_t i = 0; i < lanes; ++i)
        if ((e = cudaStreamWaitEvent(J->side[i], J->fork, 0)) != cudaSuccess) return e;
    for (size_t i = 0; i < K.size(); ++i)
        if ((e = go(K[i], J->side[i % lanes])) != cudaSuccess) return e;
    for (size_t i = 0; i < lanes; ++i) {
        if ((e = cudaEventRecord(J->join[i], J->side[i])) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s, J->join[i], 0)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

int jit_build(smg_handle* h, std::string& err) {
    if (h->jit) return SMG_OK;
    return build_state(h, false, h->jit, err);
}

int jit_build_rec(smg_handle* h, std::string& err) {
    if (h->jit_rec) return SMG_OK;
    return build_state(h, true, h->jit_rec, err);
}

cudaError_t launch_jit(const smg_handle* h, int mode, int kfilter, cudaStream_t s) {
    return launch_state(h, h->jit, h->dU, mode, kfilter, nullptr, nullptr, s);
}

cudaError_t launch_jit_rec(const smg_handle* h, int mode, int kfilter, double* U, double* wrec, double* prec,
                           const DevField* DE, int dsm, int dsw, cudaStream_t s) {
    return launch_state(h, h->jit_rec, U, mode, kfilter, wrec, prec, s, DE, dsm, dsw);
}

int jit_launches(const smg_handle* h, int phase) { return h->jit ? (int)h->jit->k[phase].size() : 0; }

// SMG_ETIMEOUT when a staged kernel's bounded wait ran out since the last
// check (the flag is cleared); call after the handle's stream is idle.
int jit_status(smg_handle* h) {
    if (!h->jit || !h->jit->dErr) return SMG_OK;
    int v = 0;
    if (cudaMemcpy(&v, h->jit->dErr, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return SMG_ECUDA;
    if (!v) return SMG_OK;
    cudaMemset(h->jit->dErr, 0, sizeof(int));
    return SMG_ETIMEOUT;
}

int jit_form(const smg_handle* h) {
    if (!h->jit) return 0;
    for (int p = 0; p < 2; ++p)
        for (const JitKernel& k : h->jit->k[p])
            if (k.form) return k.form;
    return 0;
}

// ---- sources evaluated on the device --------------------------------------
// One kernel per registered expression writes Q_j at every point of the
// component's grid: x, y, z are the point's coordinates in the solver
// dimensions (the reference's hook arguments, starmap_solver.m:278-282),
// t the evaluation time, k the 1-based component number.
void src_free(smg_handle* h, bool coords) {
    if (h->src_mod) api().ModuleUnload(static_cast<CUmodule_t>(h->src_mod));
    h->src_mod = nullptr;
    for (auto& e : h->src_expr) {
        e.fn = nullptr;
        if (coords) {
            cudaFree(e.dC);
            e.dC = nullptr;
        }
    }
    h->mat.fn.clear();
    h->filt.fn.clear();
    if (coords) {
        cudaFree(h->xyz.dC);
        cudaFree(h->mat.dOld);
        h->xyz.dC = nullptr;
        h->mat.dOld = nullptr;
        h->mat.on = false;
        h->mat.init = false;
        h->filt = smg_handle::FiltExpr{};
    }
}

namespace {
// Per sigma_t row r of the handle's material expressions (and r = rows for
// sigma_a on grid 111): the new values at t, the average with the previous
// ones into the field, its decay factor expm1div(-s*dt/2) and the new values
// kept for the next step (starmap_solver.m:214-252, 267-274); with init only
// the values at t are stored.
void emit_mat_kernel(std::string& o, const smg_handle* h, int r) {
    const auto& M = h->mat;
    const bool is_a = r == (int)M.sT.size();
    const int f = is_a ? M.sA : M.sT[r];
    const int fg = h->field_grid[f];
    const int gs[3] = {1 + (fg & 1), 1 + ((fg >> 1) & 1), 1 + ((fg >> 2) & 1)};   // solver dimensions
    int E[3], axis_of[3];
    for (int a = 0; a < 3; ++a) {
        const int d = h->sd[a];
        E[a] = (gs[d] == 2 && h->g.bc[a] == 1) ? h->g.n[a] + 1 : h->g.n[a];
        axis_of[d] = a;
    }
    char b[2048];
    std::snprintf(b, sizeof b,
                  "extern \"C\" __global__ void smg_mat_%d(double* __restrict__ S1, double* __restrict__ D, "
                  "double* __restrict__ old, const double* __restrict__ C, double t, double dt, int init) {\n"
                  "    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;\n"
                  "    if (i0 >= %d) return;\n"
                  "    for (int rr = blockIdx.y; rr < %d; rr += gridDim.y) {\n"
                  "        const int i1 = rr %% %d, i2 = rr / %d;\n"
                  "        const int ia[3] = {i0, i1, i2};\n"
                  "        const double x = C[%d + ia[%d]], y = C[%d + ia[%d]], z = C[%d + ia[%d]];\n"
                  "        const int m = %d;\n"
                  "        (void)x; (void)y; (void)z; (void)m; (void)t;\n"
                  "        const long long p = (long long)i2 * %lld + (long long)i1 * %lld + i0;\n",
                  r, E[0], E[1] * E[2], E[1], E[1], h->xyz.off[0][gs[0] - 1], axis_of[0], h->xyz.off[1][gs[1] - 1], axis_of[1],
                  h->xyz.off[2][gs[2] - 1], axis_of[2], is_a ? 0 : M.m[r], (long long)h->g.s2, (long long)h->g.s1);
    o += b;
    if (is_a) o += "        const double v = (double)(\n" + M.a + "\n        );\n";
    else {
        o += "        const double sa = (double)(\n" + M.a + "\n        );\n";
        o += "        double ss = (double)(\n" + M.s0 + "\n        );\n";
        if (!M.sm.empty()) o += "        ss = __dsub_rn(ss, (double)(\n" + M.sm + "\n        ));\n";
        o += "        const double v = __dadd_rn(sa, ss);\n";
    }
    o += "        if (init) { old[p] = v; continue; }\n"
         "        const double s1 = __dmul_rn(__dadd_rn(old[p], v), 0.5);\n"
         "        const double xx = __dmul_rn(__dmul_rn(-s1, dt), 0.5);\n"
         "        double e = __dadd_rn(__dadd_rn(1.0, __dmul_rn(xx, 0.5)), __ddiv_rn(__dmul_rn(xx, xx), 6.0));\n"
         "        if (fabs(xx) > 2e-4) e = __ddiv_rn(__dsub_rn(exp(xx), 1.0), xx);\n"
         "        S1[p] = s1; D[p] = e; old[p] = v;\n"
         "    }\n}\n";
}

// Filter row r (smg_set_filter_expr): the filter of the row's (grid type,
// order k) at t - dt/2 into field f1 and at t into f2 ('substep'), or at t
// into f1 ('full') (starmap_solver.m:283-305).  The coordinates are the
// material expressions' table.
void emit_filt_kernel(std::string& o, const smg_handle* h, int r) {
    const auto& Fl = h->filt;
    const int fg = h->field_grid[Fl.f1[r]];
    const int gs[3] = {1 + (fg & 1), 1 + ((fg >> 1) & 1), 1 + ((fg >> 2) & 1)};
    int E[3], axis_of[3];
    for (int a = 0; a < 3; ++a) {
        const int d = h->sd[a];
        E[a] = (gs[d] == 2 && h->g.bc[a] == 1) ? h->g.n[a] + 1 : h->g.n[a];
        axis_of[d] = a;
    }
    const bool two = Fl.f2[r] >= 0;
    char b[2048];
    std::snprintf(b, sizeof b,
                  "extern \"C\" __global__ void smg_filt_%d(double* __restrict__ F1, double* __restrict__ F2, "
                  "const double* __restrict__ C, double tq, double dt) {\n"
                  "    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;\n"
                  "    if (i0 >= %d) return;\n"
                  "    for (int rr = blockIdx.y; rr < %d; rr += gridDim.y) {\n"
                  "        const int i1 = rr %% %d, i2 = rr / %d;\n"
                  "        const int ia[3] = {i0, i1, i2};\n"
                  "        const double x = C[%d + ia[%d]], y = C[%d + ia[%d]], z = C[%d + ia[%d]];\n"
                  "        const int k = %d;\n"
                  "        (void)x; (void)y; (void)z; (void)k;\n"
                  "        const long long p = (long long)i2 * %lld + (long long)i1 * %lld + i0;\n",
                  r, E[0], E[1] * E[2], E[1], E[1], h->xyz.off[0][gs[0] - 1], axis_of[0], h->xyz.off[1][gs[1] - 1], axis_of[1],
                  h->xyz.off[2][gs[2] - 1], axis_of[2], Fl.k[r], (long long)h->g.s2, (long long)h->g.s1);
    o += b;
    if (two)
        o += "        { const double t = tq - dt / 2; F1[p] = (double)(\n" + Fl.expr + "\n        ); }\n"
             "        { const double t = tq; F2[p] = (double)(\n" + Fl.expr + "\n        ); }\n";
    else
        o += "        { const double t = tq; F1[p] = (double)(\n" + Fl.expr + "\n        ); }\n";
    o += "        (void)F2;\n    }\n}\n";
}
}  // namespace

int src_build(smg_handle* h, std::string& err) {
    Api& a = api();
    if (!a.cu_ok) {
        err = a.cu_why;
        return SMG_EINVAL;
    }
    src_free(h, false);
    int axis_of[3];
    for (int ax = 0; ax < 3; ++ax) axis_of[h->sd[ax]] = ax;
    std::string src;
    char b[1024];
    for (size_t i = 0; i < h->src_expr.size(); ++i) {
        const auto& e = h->src_expr[i];
        const int* E = h->comps[e.comp].ext;
        std::snprintf(b, sizeof b,
                      "extern \"C\" __global__ void smg_src_%d(double* __restrict__ Q, const double* __restrict__ C, "
                      "double t) {\n"
                      "    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;\n"
                      "    if (i0 >= %d) return;\n"
                      "    for (int r = blockIdx.y; r < %d; r += gridDim.y) {\n"
                      "        const int i1 = r %% %d, i2 = r / %d;\n"
                      "        const double a0 = C[i0], a1 = C[%d + i1], a2 = C[%d + i2];\n"
                      "        const double x = a%d, y = a%d, z = a%d;\n"
                      "        const int k = %d;\n"
                      "        (void)x; (void)y; (void)z; (void)k; (void)t;\n"
                      "        Q[(long long)i2 * %lld + (long long)i1 * %lld + i0] = (double)(\n",
                      (int)i, E[0], E[1] * E[2], E[1], E[1], E[0], E[0] + E[1], axis_of[0], axis_of[1], axis_of[2],
                      e.comp + 1, (long long)h->g.s2, (long long)h->g.s1);
        src += b;
        src += e.expr + "\n        );\n    }\n}\n";
    }
    const int nmat = h->mat.on ? (int)h->mat.sT.size() + 1 : 0;
    for (int r = 0; r < nmat; ++r) emit_mat_kernel(src, h, r);
    const int nfilt = (int)h->filt.f1.size();
    for (int r = 0; r < nfilt; ++r) emit_filt_kernel(src, h, r);
    std::vector<char> cubin;
    int rc = compile_one(src, 0, false, cubin, err);
    if (rc != SMG_OK) return rc;
    CUmodule_t m = nullptr;
    if (a.ModuleLoadData(&m, cubin.data()) != 0) {
        err = "cuModuleLoadData failed (source and material expressions)";
        return SMG_ECUDA;
    }
    h->src_mod = m;
    for (int r = 0; r < nmat; ++r) {
        CUfunction_t f = nullptr;
        const std::string name = "smg_mat_" + std::to_string(r);
        if (a.ModuleGetFunction(&f, m, name.c_str()) != 0) {
            err = "cuModuleGetFunction " + name;
            src_free(h, false);
            return SMG_ECUDA;
        }
        h->mat.fn.push_back(f);
    }
    for (int r = 0; r < nfilt; ++r) {
        CUfunction_t f = nullptr;
        const std::string name = "smg_filt_" + std::to_string(r);
        if (a.ModuleGetFunction(&f, m, name.c_str()) != 0) {
            err = "cuModuleGetFunction " + name;
            src_free(h, false);
            return SMG_ECUDA;
        }
        h->filt.fn.push_back(f);
    }
    for (size_t i = 0; i < h->src_expr.size(); ++i) {
        CUfunction_t f = nullptr;
        const std::string name = "smg_src_" + std::to_string(i);
        if (a.ModuleGetFunction(&f, m, name.c_str()) != 0) {
            err = "cuModuleGetFunction " + name;
            src_free(h, false);
            return SMG_ECUDA;
        }
        h->src_expr[i].fn = f;
    }
    return SMG_OK;
}

cudaError_t launch_mat(smg_handle* h, double t, double dt, bool init, cudaStream_t s) {
    auto& M = h->mat;
    const int rows = (int)M.sT.size();
    for (int r = 0; r <= rows; ++r) {
        const int f = r == rows ? M.sA : M.sT[r], fd = r == rows ? M.EA : M.ET[r];
        const int fg = h->field_grid[f];
        int E[3];
        for (int a = 0; a < 3; ++a) {
            const int gd = 1 + ((fg >> h->sd[a]) & 1);
            E[a] = (gd == 2 && h->g.bc[a] == 1) ? h->g.n[a] + 1 : h->g.n[a];
        }
        double* S1 = const_cast<double*>(h->fields_host[f].p);
        double* D = const_cast<double*>(h->fields_host[fd].p);
        double* old = M.dOld + (size_t)r * h->g.cs;
        const double* C = h->xyz.dC;
        double tt = t, dd = dt;
        int in = init ? 1 : 0;
        void* args[] = {&S1, &D, &old, &C, &tt, &dd, &in};
        const unsigned gx = (unsigned)((E[0] + 127) / 128), gy = (unsigned)std::min(E[1] * E[2], 4096);
        if (api().LaunchKernel(static_cast<CUfunction_t>(M.fn[r]), gx, gy, 1, 128, 1, 1, 0, s, args, nullptr) != 0)
            return cudaErrorLaunchFailure;
    }
    if (init) M.init = true;
    return cudaSuccess;
}

cudaError_t launch_filt(const smg_handle* h, double t, double dt, cudaStream_t s) {
    const auto& Fl = h->filt;
    for (size_t r = 0; r < Fl.f1.size(); ++r) {
        const int fg = h->field_grid[Fl.f1[r]];
        int E[3];
        for (int a = 0; a < 3; ++a) {
            const int gd = 1 + ((fg >> h->sd[a]) & 1);
            E[a] = (gd == 2 && h->g.bc[a] == 1) ? h->g.n[a] + 1 : h->g.n[a];
        }
        double* F1 = const_cast<double*>(h->fields_host[Fl.f1[r]].p);
        double* F2 = Fl.f2[r] >= 0 ? const_cast<double*>(h->fields_host[Fl.f2[r]].p) : F1;
        const double* C = h->xyz.dC;
        double tt = t, dd = dt;
        void* args[] = {&F1, &F2, &C, &tt, &dd};
        const unsigned gx = (unsigned)((E[0] + 127) / 128), gy = (unsigned)std::min(E[1] * E[2], 4096);
        if (api().LaunchKernel(static_cast<CUfunction_t>(Fl.fn[r]), gx, gy, 1, 128, 1, 1, 0, s, args, nullptr) != 0)
            return cudaErrorLaunchFailure;
    }
    return cudaSuccess;
}

cudaError_t launch_src(const smg_handle* h, double t, cudaStream_t s) {
    for (const auto& e : h->src_expr) {
        const int* E = h->comps[e.comp].ext;
        double* Q = const_cast<double*>(h->fields_host[h->comps[e.comp].Q].p);
        const double* C = e.dC;
        double tt = t;
        void* args[] = {&Q, &C, &tt};
        const unsigned gx = (unsigned)((E[0] + 127) / 128), gy = (unsigned)std::min(E[1] * E[2], 4096);
        if (api().LaunchKernel(static_cast<CUfunction_t>(e.fn), gx, gy, 1, 128, 1, 1, 0, s, args, nullptr) != 0)
            return cudaErrorLaunchFailure;
    }
    return cudaSuccess;
}

// Generated adjoint kernels (compiled like the forward ones, inline layout).
int jit_build_adj(smg_handle* h, std::string& err) {
    if (h->jit_adj) return SMG_OK;
    Api& a = api();
    if (!a.cu_ok) {
        err = a.cu_why;
        return SMG_EINVAL;
    }
    const int block = h->jit_block, group = h->jit_group;
    const std::vector<KernelSrc> P = adj_programs(h, block, group, h->jit_split > 0 ? h->jit_split : 16);
    std::vector<std::vector<char>> cubins;
    int rc = compile_programs(P, h->jit_regs, false, cubins, err);
    if (rc != SMG_OK) return rc;
    JitState* J = new JitState();
    J->block = block;
    for (size_t i = 0; i < cubins.size(); ++i) {
        CUmodule_t m = nullptr;
        JitKernel k;
        k.grid = P[i].grid;
        if (load_module(cubins[i], &m) != 0 ||
            (J->mods.push_back(m), a.ModuleGetFunction(&k.fn, m, P[i].name.c_str()) != 0)) {
            err = "loading the generated adjoint kernels failed";
            free_state(J);
            return SMG_ECUDA;
        }
        J->k[P[i].phase].push_back(k);
    }
    const size_t nk = std::max(std::max(J->k[0].size(), J->k[1].size()), std::max(J->k[2].size(), J->k[3].size()));
    if (nk > 1) {
        if (cudaEventCreateWithFlags(&J->fork, cudaEventDisableTiming) != cudaSuccess) {
            free_state(J);
            err = "cudaEventCreate";
            return SMG_ECUDA;
        }
        for (size_t i = 0; i < nk; ++i) {
            cudaStream_t st = nullptr;
            cudaEvent_t ev = nullptr;
            if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
                if (st) cudaStreamDestroy(st);
                free_state(J);
                err = "cudaStreamCreate";
                return SMG_ECUDA;
            }
            J->side.push_back(st);
            J->join.push_back(ev);
        }
    }
    h->jit_adj = J;
    return SMG_OK;
}

// One backward phase over the sources of a phase of type l (see adj_programs).
cudaError_t launch_jit_adj(const smg_handle* h, int l, int coup, int pm, int pm_swap, int nm, int nm_swap,
                           double* Y, const DevField* DE, double* const* Gt, const double* pre, const double* W,
                           cudaStream_t s) {
    JitState* J = h->jit_adj;
    const bool steady = coup == 1 && pm == 2 && nm == 2 && pm_swap == l && nm_swap == l;
    const std::vector<JitKernel>& K = J->k[l + (steady ? 2 : 0)];
    if (K.empty()) return cudaSuccess;
    const DevField* F = h->dFieldTab;
    double hdt = h->hdt;
    void* args[] = {&Y, &F, &DE, &Gt, &pre, &W, &pm, &pm_swap, &nm, &nm_swap, &coup, &hdt};
    auto go = [&](const JitKernel& k, cudaStream_t st) {
        return api().LaunchKernel(k.fn, (unsigned)k.grid, 1, 1, (unsigned)J->block, 1, 1, 0, st, args, nullptr) == 0
                   ? cudaSuccess
                   : cudaErrorLaunchFailure;
    };
    if (K.size() == 1) return go(K[0], s);
    // at most `lanes` kernels at a time: kernel i runs on side stream i mod
    // lanes, after kernel i - lanes
    const size_t lanes = h->jit_lanes > 0 ? std::min<size_t>((size_t)h->jit_lanes, K.size()) : K.size();
    cudaError_t e = cudaEventRecord(J->fork, s);
    if (e != cudaSuccess) return e;
    for (size_t i = 0; i < lanes; ++i)
        if ((e = cudaStreamWaitEvent(J->side[i], J->fork, 0)) != cudaSuccess) return e;
    for (size_t i = 0; i < K.size(); ++i)
        if ((e = go(K[i], J->side[i % lanes])) != cudaSuccess) return e;
    for (size_t i = 0; i < lanes; ++i) {
        if ((e = cudaEventRecord(J->join[i], J->side[i])) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s, J->join[i], 0)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int jit_adj_launches(const smg_handle* h, int l) { return h->jit_adj ? (int)h->jit_adj->k[l].size() : 0; }

// ---- family kernels of a batch ---------------------------------------------
struct FamKernel {
    CUfunction_t fn = nullptr;
    int phase = 0, fam = 0;
    int4* d_items = nullptr;
    long long nitems = 0;
};

struct JitFamilySet {
    std::vector<CUmodule_t> mods;
    std::vector<FamKernel> kernels;
    std::vector<std::vector<int>> members;   // family -> batch instance indices
    std::vector<FamGeom*> d_geo;             // family -> geometry table (one row per member)
    int block = 64;
    int nk[2] = {0, 0};
    std::vector<cudaStream_t> side;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
};

void jit_family_free(JitFamilySet*& S) {
    if (!S) return;
    for (auto& k : S->kernels) cudaFree(k.d_items);
    for (FamGeom* g : S->d_geo) cudaFree(g);
    for (cudaStream_t st : S->side) cudaStreamDestroy(st);
    if (S->fork) cudaEventDestroy(S->fork);
    for (cudaEvent_t e : S->join) cudaEventDestroy(e);
    if (api().cu_ok)
        for (CUmodule_t m : S->mods) api().ModuleUnload(m);
    delete S;
    S = nullptr;
}

int jit_family_build(const std::vector<smg_handle*>& inst, int block, int group, int split, int regs,
                     JitFamilySet*& out, std::string& err) {
    Api& a = api();
    if (!a.cu_ok) {
        err = a.cu_why;
        return SMG_EINVAL;
    }
    for (const smg_handle* h : inst)
        if (!(h->pair[0].ok && h->pair[1].ok) || std::min(h->exact_recip[0], std::min(h->exact_recip[1], h->exact_recip[2])) < 1) {
            err = "an instance exceeds 32-bit offsets or has a subnormal grid spacing";
            return SMG_EINVAL;
        }
    // families: instances whose generated code is the same text
    std::map<std::string, int> fam_of;
    std::vector<std::vector<KernelSrc>> fam_src;
    JitFamilySet* S = new JitFamilySet();
    S->block = block;
    for (size_t i = 0; i < inst.size(); ++i) {
        std::vector<KernelSrc> P = fam_programs(inst[i], block, group, split);
        std::string key;
        for (const auto& k : P) key += k.src;
        auto it = fam_of.find(key);
        if (it == fam_of.end()) {
            it = fam_of.emplace(key, (int)fam_src.size()).first;
            fam_src.push_back(std::move(P));
            S->members.emplace_back();
        }
        S->members[it->second].push_back((int)i);
    }
    std::vector<KernelSrc> all;
    std::vector<int> fam_idx;
    for (size_t f = 0; f < fam_src.size(); ++f)
        for (const auto& k : fam_src[f]) {
            all.push_back(k);
            fam_idx.push_back((int)f);
        }
    std::vector<std::vector<char>> cubins;
    int rc = compile_programs(all, regs, false, cubins, err);
    if (rc != SMG_OK) {
        delete S;
        return rc;
    }
    auto fail = [&](const std::string& m) {
        err = m;
        jit_family_free(S);
        return SMG_ECUDA;
    };
    for (size_t i = 0; i < all.size(); ++i) {
        CUmodule_t m = nullptr;
        FamKernel K;
        if (a.ModuleLoadData(&m, cubins[i].data()) != 0) return fail("cuModuleLoadData failed");
        S->mods.push_back(m);
        if (a.ModuleGetFunction(&K.fn, m, all[i].name.c_str()) != 0) return fail("cuModuleGetFunction " + all[i].name);
        K.phase = all[i].phase;
        K.fam = fam_idx[i];
        // work items of the kernel's groups over the family's instances:
        // (member, group, chunk, row), instance by instance and within an
        // instance group by group: the CTAs running at the same time share
        // a group's code, and the groups of one instance reuse its sources
        // in L2 (group-major over all members streamed every group's sources
        // through L2 once per group)
        const int k0 = std::stoi(all[i].name.substr(all[i].name.rfind('_') + 1));
        const int k1 = k0 + (int)all[i].grid;
        std::vector<int4> items;
        const std::vector<int>& mem = S->members[K.fam];
        for (size_t li = 0; li < mem.size(); ++li)
            for (int grp = k0; grp < k1; ++grp) {
                const smg_handle* h = inst[mem[li]];
                const int tpr = (h->g.B[0] + 1) / 2;
                const int nch = (tpr + block - 1) / block;
                const int rows = h->g.B[1] * h->g.B[2];
                for (int r = 0; r < rows; ++r)
                    for (int c = 0; c < nch; ++c) items.push_back(make_int4((int)li, grp, c, r));
            }
        K.nitems = (long long)items.size();
        if (cudaMalloc(&K.d_items, sizeof(int4) * std::max<size_t>(items.size(), 1)) != cudaSuccess)
            return fail("cudaMalloc (batch items)");
        if (!items.empty() &&
            cudaMemcpy(K.d_items, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            return fail("cudaMemcpy (batch items)");
        S->nk[K.phase]++;
        S->kernels.push_back(K);
    }
    for (size_t f = 0; f < S->members.size(); ++f) {
        FamGeom* g = nullptr;
        if (cudaMalloc(&g, sizeof(FamGeom) * S->members[f].size()) != cudaSuccess) return fail("cudaMalloc (geometry)");
        S->d_geo.push_back(g);
    }
    const int nk = std::max(S->nk[0], S->nk[1]);
    if (nk > 1) {
        if (cudaEventCreateWithFlags(&S->fork, cudaEventDisableTiming) != cudaSuccess) return fail("cudaEventCreate");
        for (int i = 0; i < nk; ++i) {
            cudaStream_t st = nullptr;
            cudaEvent_t ev = nullptr;
            if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return fail("cudaStreamCreate");
            S->side.push_back(st);
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return fail("cudaEventCreate");
            S->join.push_back(ev);
        }
    }
    out = S;
    return SMG_OK;
}

// Geometry tables from the instances' current state (dt/2 follows smg_batch_set_dt).
cudaError_t jit_family_geometry(JitFamilySet* S, const std::vector<smg_handle*>& inst, cudaStream_t s) {
    for (size_t f = 0; f < S->members.size(); ++f) {
        std::vector<FamGeom> G;
        for (int i : S->members[f]) {
            const smg_handle* h = inst[i];
            FamGeom g{};
            g.U = h->dU;
            g.F = h->dFieldTab;
            for (int a = 0; a < 3; ++a) {
                g.n[a] = h->g.n[a];
                g.h[a] = h->g.h[a];
                g.rh[a] = h->rh[a];
            }
            g.s1 = h->g.s1;
            g.s2 = h->g.s2;
            g.cs = h->g.cs;
            g.hdt = h->hdt;
            G.push_back(g);
        }
        cudaError_t e = cudaMemcpyAsync(S->d_geo[f], G.data(), sizeof(FamGeom) * G.size(), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return e;
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;   // G is a host temporary
    }
    return cudaSuccess;
}

// One phase of every instance: the family kernels of the phase type, concurrent.
cudaError_t jit_family_phase(JitFamilySet* S, int mode, int kfilter, cudaStream_t s, int64_t* launches) {
    const int phase = mode == 1 ? 1 : 0;
    int kf = kfilter, md = mode;
    std::vector<const FamKernel*> K;
    for (const auto& k : S->kernels)
        if (k.phase == phase && k.nitems > 0) K.push_back(&k);
    if (K.empty()) return cudaSuccess;
    *launches += (int64_t)K.size();
    auto go = [&](const FamKernel* k, cudaStream_t st) {
        const FamGeom* geo = S->d_geo[k->fam];
        const int4* items = k->d_items;
        void* args[] = {&geo, &items, &kf, &md};
        return api().LaunchKernel(k->fn, (unsigned)k->nitems, 1, 1, (unsigned)S->block, 1, 1, 0, st, args, nullptr) == 0
                   ? cudaSuccess
                   : cudaErrorLaunchFailure;
    };
    if (K.size() == 1) return go(K[0], s);
    cudaError_t e = cudaEventRecord(S->fork, s);
    if (e != cudaSuccess) return e;
    for (size_t i = 0; i < K.size(); ++i) {
        if ((e = cudaStreamWaitEvent(S->side[i], S->fork, 0)) != cudaSuccess) return e;
        if ((e = go(K[i], S->side[i])) != cudaSuccess) return e;
        if ((e = cudaEventRecord(S->join[i], S->side[i])) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s, S->join[i], 0)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int jit_family_count(const JitFamilySet* S) { return S ? (int)S->members.size() : 0; }

}  // namespace smg

static size_t adj_count(const std::vector<KernelSrc>& v) {
    size_t n = 0;
    for (const auto& k : v)
        if (k.name.rfind("smg_adj_", 0) == 0) ++n;
    return n;
}

extern "C" int smg_jit_source(const smg_problem* p, const int32_t* keys, const int32_t* values, int32_t ntune,
                              int32_t compile, char* buf, int64_t cap, int64_t* len) {
    SMG_TRY
    if (!p || ntune < 0 || (ntune > 0 && (!keys || !values))) {
        smg::set_global_error("smg_jit_source: bad arguments");
        return SMG_EINVAL;
    }
    smg_handle* h = nullptr;
    int rc = smg::create_host(p, &h);
    if (rc != SMG_OK) return rc;
    if (!(h->pair[0].ok && h->pair[1].ok)) {   // the generator reads the pair tables
        delete h;
        smg::set_global_error("smg_jit_source: the problem exceeds 32-bit element offsets");
        return SMG_EINVAL;
    }
    for (int i = 0; i < ntune; ++i) {
        if (keys[i] < SMG_TUNE_JIT_BLOCK) {
            rc = SMG_EINVAL;
            smg::set_global_error("smg_jit_source: only SMG_TUNE_JIT_* keys apply");
        } else if ((rc = smg_tune(h, keys[i], values[i])) != SMG_OK) {
            smg::set_global_error("smg_jit_source: " + h->err);
        }
        if (rc != SMG_OK) {
            delete h;
            return rc;
        }
    }
    std::string s = smg::jit_source(h, h->jit_block, h->jit_group);
    std::vector<KernelSrc> extra;
    if (compile == 2) {   // also the recording and the backward-phase kernels of the adjoint
        extra = programs(h, h->jit_block, h->jit_group, h->jit_split, h->jit_calls, true);
        const std::vector<KernelSrc> adj = adj_programs(h, h->jit_block, h->jit_group, h->jit_split > 0 ? h->jit_split : 16);
        extra.insert(extra.end(), adj.begin(), adj.end());
        for (const KernelSrc& k : extra) s += "// ---- program (" + k.name + ")\n" + k.src;
    }
    std::vector<KernelSrc> fam;
    if (compile == 3) {   // also the batched solver's family kernels
        fam = fam_programs(h, h->jit_block, h->jit_group, h->jit_split > 0 ? h->jit_split : 16);
        for (const KernelSrc& k : fam) s += "// ---- program (" + k.name + ")\n" + k.src;
    }
    if (len) *len = (int64_t)s.size();
    if (buf && cap > 0) {
        const size_t n = std::min<size_t>((size_t)cap - 1, s.size());
        std::memcpy(buf, s.data(), n);
        buf[n] = '\0';
    }
    if (compile) {
        std::string err;
        rc = smg::jit_compile(h, h->jit_block, h->jit_group, err);
        if (rc == SMG_OK && !extra.empty()) {
            std::vector<std::vector<char>> cubins;
            std::vector<KernelSrc> rec(extra.begin(), extra.begin() + (extra.size() - adj_count(extra)));
            std::vector<KernelSrc> adj(extra.end() - adj_count(extra), extra.end());
            rc = compile_programs(rec, 64, h->jit_calls != 0, cubins, err);
            if (rc == SMG_OK) rc = compile_programs(adj, 64, false, cubins, err);
        }
        if (rc == SMG_OK && !fam.empty()) {
            std::vector<std::vector<char>> cubins;
            rc = compile_programs(fam, h->jit_regs, false, cubins, err);
        }
        if (rc != SMG_OK) smg::set_global_error("smg_jit_source: " + err);
    }
    delete h;
    return rc;
    SMG_CATCH(nullptr)
}

extern "C" int smg_jit_stats(int64_t* compiled, int64_t* from_disk) {
    SMG_TRY
    if (compiled) *compiled = g_programs_compiled.load();
    if (from_disk) *from_disk = g_programs_from_disk.load();
    return SMG_OK;
    SMG_CATCH(nullptr)
}
