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

#include <algorithm>
#include <atomic>
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
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
};

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

void load_api() {
    Api& a = g_api;
    void* nv = open_first({"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"});
    if (!nv) {
        a.why = "NVRTC (libnvrtc.so.12) not found";
    } else if (sym(nv, "nvrtcCreateProgram", a.CreateProgram) && sym(nv, "nvrtcCompileProgram", a.CompileProgram) &&
               sym(nv, "nvrtcGetProgramLogSize", a.GetProgramLogSize) &&
               sym(nv, "nvrtcGetProgramLog", a.GetProgramLog) && sym(nv, "nvrtcGetCUBINSize", a.GetCUBINSize) &&
               sym(nv, "nvrtcGetCUBIN", a.GetCUBIN) && sym(nv, "nvrtcDestroyProgram", a.DestroyProgram) &&
               sym(nv, "nvrtcGetErrorString", a.GetErrorString)) {
        a.ok = true;
    } else {
        a.why = "NVRTC entry points missing";
    }
    // nvJitLink exports versioned names (nvJitLink.h maps the API onto them)
    void* jl = open_first({"libnvJitLink.so.12", "libnvJitLink.so", "/usr/local/cuda/lib64/libnvJitLink.so.12"});
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
               sym(cu, "cuModuleGetFunction", a.ModuleGetFunction) && sym(cu, "cuLaunchKernel", a.LaunchKernel)) {
        a.cu_ok = true;
    } else {
        a.cu_why = "CUDA driver entry points missing";
    }
}

Api& api() {
    std::call_once(g_api_once, load_api);
    return g_api;
}

// ---- source generation -------------------------------------------------------
const char* kPrelude = R"(
struct DevField { const double* p; double s; };
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
)";

std::string lit(double v) {
    // exact value as a C++17 hexadecimal floating literal
    char buf[64];
    if (v == 0.0) return std::signbit(v) ? "(-0.0)" : "0.0";
    std::snprintf(buf, sizeof buf, "(%a)", v);
    return buf;
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

// One destination's block.  Update modes: 0 one substep with filter kf;
// 1 two substeps (phase B: F1 then F2); 2 fused A(k=2) A(k=1) (F2 then F1).
// Phase A blocks carry modes 0 and 2 (chosen by `mode` at run time), phase B
// blocks mode 1.  Loads of the second point are unconditional: the row pitch
// is a multiple of 8 doubles, so x0+1 lies inside the padded row even where
// the component's extent ends at x0 (that value is unused and not stored).
void emit_dest(std::string& o, const smg_handle* h, int phase, int j) {
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
    if (!v1_always) o += "        const bool v1 = x1 < " + std::to_string(c.ext[0]) + ";\n";
    const std::string sel1 = v1_always ? "" : "v1 ? ", sel2 = v1_always ? "" : " : 0";
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
        if (a == 0) {
            std::snprintf(b, sizeof b,
                          "        { const double* S = Up + %lld;\n"
                          "          const double a0 = ld1(S + hx0_%d), b0 = ld1(S + lx0_%d), a1 = ld1(S + (%shx1_%d%s)), "
                          "b1 = ld1(S + (%slx1_%d%s));\n"
                          "          const double tA = __dmul_rn(%s(__dsub_rn(a0, b0), %s, %s), %s);\n"
                          "          const double tB = __dmul_rn(%s(__dsub_rn(a1, b1), %s, %s), %s);\n"
                          "          %s }\n",
                          so, g2, g2, sel1.c_str(), g2, sel2.c_str(), sel1.c_str(), g2, sel2.c_str(), dv, H.c_str(),
                          RH.c_str(), W.c_str(), dv, H.c_str(), RH.c_str(), W.c_str(), fold);
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

std::string group_name(int phase, int k) { return "smg_g" + std::to_string(phase) + "_" + std::to_string(k); }
const char* kGroupArgs =
    "(double* __restrict__ U, const DevField* __restrict__ F, double hdt, int kf, int mode, int x0, int y, int z)";

// device function of one group: the thread's stencil offsets, then the blocks
void emit_group(std::string& o, const smg_handle* h, int phase, int k, const std::vector<int>& D, int group) {
    const smg::DevGrid& g = h->g;
    char b[1024];
    const int d0 = k * group, d1 = std::min<int>((k + 1) * group, (int)D.size());
    o += "extern \"C\" __device__ __noinline__ void " + group_name(phase, k) + kGroupArgs + " {\n";
    std::snprintf(b, sizeof b,
                  "    const int x1 = x0 + 1;\n"
                  "    const int pt = z * %lld + y * %lld + x0;\n"
                  "    const double* Up = U + pt;\n"
                  "    (void)x1; (void)kf; (void)mode; (void)hdt; (void)Up;\n",
                  (long long)g.s2, (long long)g.s1);
    o += b;
    bool used[3] = {false, false, false};
    for (int i = d0; i < d1; ++i)
        for (int q = h->comps[D[i]].cbeg; q < h->comps[D[i]].cend; ++q) used[h->coups[q].code >> 1] = true;
    if (used[0])
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
    for (int i = d0; i < d1; ++i) emit_dest(o, h, phase, D[i]);
    o += "}\n";
}

// dispatch kernel of one phase type: CTA -> (group, row, chunk); calls the group
void emit_dispatch(std::string& o, const smg_handle* h, int phase, int ngroups, int block) {
    const smg::DevGrid& g = h->g;
    const int tpr = (g.B[0] + 1) / 2;
    const int nchunks = (tpr + block - 1) / block;
    const long long per = (long long)nchunks * g.B[1] * g.B[2];
    char b[1024];
    for (int k = 0; k < ngroups; ++k) o += "extern \"C\" __device__ void " + group_name(phase, k) + kGroupArgs + ";\n";
    std::snprintf(b, sizeof b,
                  "extern \"C\" __global__ void __launch_bounds__(%d) smg_jit_p%d(double* __restrict__ U, "
                  "const DevField* __restrict__ F, double hdt, int kf, int mode) {\n"
                  "    const int bid = blockIdx.x;\n"
                  "    const int grp = bid / %lld;\n"
                  "    const int rest = bid - grp * %lld;\n"
                  "    const int row = rest / %d, chunk = rest - row * %d;\n"
                  "    const int y = row %% %d, z = row / %d;\n"
                  "    const int x0 = 2 * (chunk * %d + (int)threadIdx.x);\n"
                  "    if (x0 >= %d) return;\n"
                  "    switch (grp) {\n",
                  block, phase, per, per, nchunks, nchunks, g.B[1], g.B[1], block, g.B[0]);
    o += b;
    for (int k = 0; k < ngroups; ++k)
        o += "    case " + std::to_string(k) + ": " + group_name(phase, k) + "(U, F, hdt, kf, mode, x0, y, z); break;\n";
    o += "    default: break;\n    }\n}\n";
}

// destinations of a phase in the pair tables' order (breadth-first levels)
std::vector<int> phase_dests(const smg_handle* h, int phase) {
    std::vector<int> D;
    for (const auto& d : h->pair[phase].dests) D.push_back((int)((long long)d.off / h->g.cs));
    if (D.empty()) D = phase == 0 ? h->destA : h->destB;
    return D;
}

// The programs of one handle: [0] the dispatch kernels, then the group
// functions, `per` groups per program.
std::vector<std::string> programs(const smg_handle* h, int block, int group, int per) {
    std::vector<std::string> P;
    std::string disp = kPrelude;
    std::vector<std::string> fns;
    for (int phase = 0; phase < 2; ++phase) {
        const std::vector<int> D = phase_dests(h, phase);
        if (D.empty()) continue;
        const int ng = ((int)D.size() + group - 1) / group;
        emit_dispatch(disp, h, phase, ng, block);
        for (int k = 0; k < ng; ++k) {
            std::string s;
            emit_group(s, h, phase, k, D, group);
            fns.push_back(std::move(s));
        }
    }
    P.push_back(std::move(disp));
    for (size_t i = 0; i < fns.size(); i += per) {
        std::string s = kPrelude;
        for (size_t k = i; k < std::min(fns.size(), i + per); ++k) s += fns[k];
        P.push_back(std::move(s));
    }
    return P;
}

// regs > 0: register limit per thread of every function (--maxrregcount);
// the linked kernel's count is the maximum over its call graph
int compile_one(const std::string& src, int regs, std::vector<char>& cubin, std::string& err) {
    Api& a = api();
    nvrtcProgram_t prog = nullptr;
    nvrtcResult_t r = a.CreateProgram(&prog, src.c_str(), "smg_jit.cu", 0, nullptr, nullptr);
    if (r != 0) {
        err = std::string("nvrtcCreateProgram: ") + a.GetErrorString(r);
        return SMG_ECUDA;
    }
    const std::string rr = "--maxrregcount=" + std::to_string(regs);
    const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "--fmad=false", "--relocatable-device-code=true",
                          rr.c_str()};
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

std::map<std::string, std::vector<char>> g_cubins;   // joined sources -> linked cubin, process-wide
std::mutex g_cubin_mu;

}  // namespace

namespace smg {

struct JitState {
    CUmodule_t mod = nullptr;
    CUfunction_t fn[2] = {nullptr, nullptr};   // dispatch kernel per phase type
    int block = 64, group = 8;
    long long grid[2] = {0, 0};
};

std::string jit_source(const smg_handle* h, int block, int group) {
    std::string o;
    int i = 0;
    for (const std::string& s : programs(h, block, group, 4)) o += "// ---- program " + std::to_string(i++) + "\n" + s;
    return o;
}

// Compile the programs on all host threads and link them into one sm_100a
// cubin (cached per process by source text).
int jit_compile_link(const std::vector<std::string>& P, int regs, std::vector<char>& cubin, std::string& err) {
    std::string key = "regs " + std::to_string(regs) + "\n";
    for (const auto& s : P) key += s;
    {
        std::lock_guard<std::mutex> lk(g_cubin_mu);
        auto it = g_cubins.find(key);
        if (it != g_cubins.end()) {
            cubin = it->second;
            return SMG_OK;
        }
    }
    Api& a = api();
    if (!a.ok) {
        err = a.why;
        return SMG_EINVAL;
    }
    if (!a.link_ok) {
        err = a.link_why;
        return SMG_EINVAL;
    }
    std::vector<std::vector<char>> obj(P.size());
    std::vector<std::string> errs(P.size());
    std::vector<int> rcs(P.size(), SMG_OK);
    std::atomic<size_t> next(0);
    const unsigned nt = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), 64));
    auto work = [&]() {
        for (size_t i = next++; i < P.size(); i = next++) rcs[i] = compile_one(P[i], regs, obj[i], errs[i]);
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < std::min<size_t>(nt, P.size()); ++t) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();
    for (size_t i = 0; i < P.size(); ++i)
        if (rcs[i] != SMG_OK) {
            err = errs[i];
            return rcs[i];
        }
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
    cubin.assign(n, 0);
    a.LinkedCubin(L, cubin.data());
    a.LinkDestroy(&L);
    std::lock_guard<std::mutex> lk(g_cubin_mu);
    g_cubins[key] = cubin;
    return SMG_OK;
}

int jit_build(smg_handle* h, std::string& err) {
    if (h->jit) return SMG_OK;
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
    std::vector<char> cubin;
    int rc = jit_compile_link(programs(h, block, group, 4), h->jit_regs, cubin, err);
    if (rc != SMG_OK) return rc;
    JitState* J = new JitState();
    J->block = block;
    J->group = group;
    if (a.ModuleLoadData(&J->mod, cubin.data()) != 0) {
        err = "cuModuleLoadData failed";
        delete J;
        return SMG_ECUDA;
    }
    const int tpr = (h->g.B[0] + 1) / 2;
    const long long nchunks = (tpr + block - 1) / block;
    const long long rows = (long long)h->g.B[1] * h->g.B[2];
    for (int phase = 0; phase < 2; ++phase) {
        const std::vector<int> D = phase_dests(h, phase);
        J->grid[phase] = ((long long)D.size() + group - 1) / group * nchunks * rows;
        if (D.empty()) continue;
        const std::string name = "smg_jit_p" + std::to_string(phase);
        if (a.ModuleGetFunction(&J->fn[phase], J->mod, name.c_str()) != 0) {
            err = "cuModuleGetFunction " + name;
            a.ModuleUnload(J->mod);
            delete J;
            return SMG_ECUDA;
        }
    }
    h->jit = J;
    return SMG_OK;
}

void jit_free(smg_handle* h) {
    if (!h->jit) return;
    if (h->jit->mod && api().cu_ok) api().ModuleUnload(h->jit->mod);
    delete h->jit;
    h->jit = nullptr;
}

cudaError_t launch_jit(const smg_handle* h, int mode, int kfilter, cudaStream_t s) {
    const int phase = mode == 1 ? 1 : 0;
    const JitState* J = h->jit;
    CUfunction_t f = J->fn[phase];
    if (!f || J->grid[phase] == 0) return cudaSuccess;
    double* U = h->dU;
    const DevField* F = h->dFieldTab;
    double hdt = h->hdt;
    int kf = kfilter;
    int md = mode;
    void* args[] = {&U, &F, &hdt, &kf, &md};
    const CUresult_t r =
        api().LaunchKernel(f, (unsigned)J->grid[phase], 1, 1, (unsigned)J->block, 1, 1, 0, s, args, nullptr);
    return r == 0 ? cudaSuccess : cudaErrorLaunchFailure;
}

}  // namespace smg

extern "C" int smg_jit_source(const smg_problem* p, int32_t block, int32_t group, int32_t compile, char* buf,
                              int64_t cap, int64_t* len) {
    if (!p) return SMG_EINVAL;
    if (block < 32 || block > 256 || block % 32 || group < 1 || group > 256) {
        smg::set_global_error("smg_jit_source: block must be 32..256 (x32), group 1..256");
        return SMG_EINVAL;
    }
    smg_handle* h = nullptr;
    int rc = smg::create_host(p, &h);
    if (rc != SMG_OK) return rc;
    const std::string s = smg::jit_source(h, block, group);
    std::vector<std::string> P;
    if (compile) P = programs(h, block, group, 4);
    delete h;
    if (len) *len = (int64_t)s.size();
    if (buf && cap > 0) {
        const size_t n = std::min<size_t>((size_t)cap - 1, s.size());
        std::memcpy(buf, s.data(), n);
        buf[n] = '\0';
    }
    if (compile) {
        std::vector<char> cubin;
        std::string err;
        rc = smg::jit_compile_link(P, 64, cubin, err);
        if (rc != SMG_OK) smg::set_global_error("smg_jit_source: " + err);
        return rc;
    }
    return SMG_OK;
}
