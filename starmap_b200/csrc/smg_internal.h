// smg_internal.h -- host-side structures shared by the library's translation
// units (not part of the public ABI).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "smg_device.cuh"

#define SMG_TRY try {
#define SMG_CATCH(err)                                   \
    }                                                    \
    catch (...) {                                        \
        return smg::exception_status((err), __func__);   \
    }

struct smg_problem;

namespace smg {
struct AdjData;
struct JitState;
struct JitFamilySet;
// per-instance geometry of the batched family kernels (layout shared with the
// generated code)
struct FamGeom {
    double* U;
    const DevField* F;
    int n[4];
    long long s1, s2, cs;
    double h[3];
    double rh[3];
    double hdt;
};
}

struct smg_handle {
    // problem
    int n_sys = 0;
    int sd[3] = {0, 1, 2};           // solver dimension of each kernel axis
    smg::DevGrid g{};
    std::vector<smg::DevComp> comps;
    std::vector<smg::DevCoup> coups;
    std::vector<int> destA, destB;   // outer set (phase A), inner set (phase B)
    std::vector<smg::DevField> fields_host;  // device view of the field table
    std::vector<int> field_grid;     // packed grid type of each field (for uploads)
    std::vector<char> field_is_array;  // per user field: array (1) or scalar (0), fixed at creation
    std::vector<int> sigma_t_field, decay_t_field;   // per component
    std::vector<int> derived_decay;  // field index -> decay field computed on device (or -1)
    int sigma_a = -1, decay_a = -1, derived_decay_a = -1;
    int filter_mode = 0;
    int field_one = -1, field_zero = -1;
    // device memory
    double* dU = nullptr;
    double* dStage = nullptr;        // staging for state transfers (linear copies, then a scatter kernel)
    double* dSnap = nullptr;         // copy of the state for output-time interpolation (smg_snapshot)
    bool snap_set = false;
    size_t stage_bytes = 0;
    double* dFields = nullptr;       // slots for array fields
    smg::DevComp* dComps = nullptr;
    smg::DevCoup* dCoups = nullptr;
    smg::DevField* dFieldTab = nullptr;
    int* dDest = nullptr;            // destA followed by destB
    int* dFlag = nullptr;            // device status word (finite check)
    double* dSumsq = nullptr;        // reduction scratch: n_sys*kSumsqBlocks partials + n_sys results
    size_t bytes = 0;
    int nslots = 0;
    // run state
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // staged transfers: copy stream and the events that pass the two halves
    // of the staging buffer between it and `stream` (created on first use)
    cudaStream_t xstream = nullptr;
    cudaEvent_t xev_fork = nullptr, xev_join = nullptr, xev_full[2] = {nullptr, nullptr},
                xev_free[2] = {nullptr, nullptr};
    double dt = 0.0, hdt = 0.0;
    bool dt_set = false, state_set = false;
    double last_ms = 0.0;
    int64_t last_launches = 0;
    // CUDA graph of a block of steps
    cudaGraphExec_t graph = nullptr;
    int64_t graph_steps = 0;
    int64_t graph_launches = 0;
    int graph_block = -1;            // steps per captured graph (0: direct launches; -1: by step size)
    std::string err;
    // sources evaluated on the device every step (smg_set_source_expr)
    struct SrcExpr {
        int comp = -1;
        std::string expr;                // C++ expression in x, y, z (solver dimensions), t, k
        double* dC = nullptr;            // coordinates per kernel axis, concatenated
        void* fn = nullptr;              // CUfunction once built
    };
    std::vector<SrcExpr> src_expr;
    // grid coordinates of the material and filter expressions: per solver
    // dimension, grid types 1 and 2 (offsets into dC)
    struct Coords {
        double* dC = nullptr;
        int off[3][2] = {{0, 0}, {0, 0}, {0, 0}};
    } xyz;
    // materials evaluated on the device every step (smg_set_material_expr)
    struct MatExpr {
        bool on = false;
        std::string a, s0, sm;           // sigma_a, sigma_s0, sigma_sm (sm empty: isotropic)
        std::vector<int> sT, ET, m;      // per sigma_t field: its decay field and moment order
        int sA = -1, EA = -1;
        double* dOld = nullptr;          // the values at the previous time (sT rows, then sigma_a)
        std::vector<void*> fn;           // CUfunction per sigma_t row, then sigma_a
        bool init = false;               // dOld holds the values at h->t
    } mat;
    // filters evaluated on the device every step (smg_set_filter_expr)
    struct FiltExpr {
        std::string expr;                // in x, y, z, t, dt and the order k
        std::vector<int> f1, f2, k;      // per row: fields at t - dt/2 and t (substep; f2 = -1 for 'full')
        std::vector<void*> fn;
    } filt;
    void* src_mod = nullptr;             // CUmodule of the source, material and filter kernels
    double t = 0.0;                      // time of the current state (smg_set_time)
    // strip-kernel schedules (phase 0 = A, 1 = B); empty if not usable
    struct HostSched {
        std::vector<smg::Stage> stages;
        std::vector<smg::SlotJob> jobs;
        std::vector<smg::DestJob> dests;
        std::vector<smg::SCoup> coups;
        int nslots = 0;
        int jcap = 0;                // most slot jobs of one stage (staging rows)
        std::vector<int> frows;      // field index of each cached coefficient row
        bool ok = false;
        void* dmem = nullptr;        // device copy of the four tables
        smg::StripSched view{};
    } sched[2];
    struct PairTables {
        std::vector<smg::PairDest> dests;
        std::vector<int> coff;
        std::vector<double> cw;
        smg::PairDest* d_dests = nullptr;
        int* d_coff = nullptr;
        double* d_cw = nullptr;
        int ndest = 0;
        bool ok = false;
    } pair[2];
    int pair_group = 8;              // destinations per pair-kernel CTA
    int pair_block = 64;             // threads per pair-kernel CTA (upper bound)
    int pair_unroll = 1;             // couplings per inner iteration
    int pair_minb = 4;               // resident CTAs the register budget targets
    int variant = 0;                 // SMG_VARIANT_*
    double rh[3] = {0, 0, 0};
    int exact_recip[3] = {0, 0, 0};
    int nxs = 0;                     // 32-point strips per row
    bool strip_staged = false;       // stage slot-job loads with cp.async
    smg::AdjData* adj = nullptr;     // adjoint checkpoints and buffers (smg_forward)
    int adj_fused = 1;               // smg_backward kernel form (SMG_TUNE_ADJ_FUSED)
    int adj_priority = 0;            // recompute stream at the highest priority (SMG_TUNE_ADJ_PRIORITY)
    smg::JitState* jit = nullptr;    // problem-specialised kernels (SMG_VARIANT_JIT)
    smg::JitState* jit_rec = nullptr;  // the same with adjoint recording (smg_forward / smg_backward)
    smg::JitState* jit_adj = nullptr;  // generated backward-phase kernels (smg_backward)
    int jit_block = 64, jit_group = 8, jit_regs = 80;
    int jit_split = 16;              // groups per NVRTC program (0: one program per phase)
    int jit_calls = 0;               // 1: one kernel per phase calling separately compiled groups
    int jit_xpair = 0;               // x differences from aligned 128-bit pairs (1) or 64-bit loads (0)
    int jit_prefetch = 0;            // L2 prefetch of a group's rows before its loads
    int jit_const = 1;               // coupling weights and grid constants from a __constant__ table
    int jit_band = -1;               // rows per band of the CTA order (0: group-major; -1: by slot size)
    int jit_lanes = 0;               // kernels of a phase at the same time, 0 = all (SMG_TUNE_JIT_LANES)
    int direct_xfer = 1;             // page-locked host arrays are moved by one kernel without staging
    int jit_staged = 0;              // 0 register form, 1 staged by bulk copies, 2 by async copies, 3 prefetch ring
    int jit_slices = 4;              // consumer warps (destination slices) per staged CTA
    int jit_stages = 3;              // shared-memory ring stages of the staged kernels
    int jit_rows = 0;                // rows per staged CTA (0: about eight waves per phase)
    bool jit_failed = false;         // AUTO tried the JIT and it was unavailable
    std::string jit_err;
};

void smg_adjoint_free(smg_handle* h);   // smg_adjoint.cu

namespace smg {
// kernels (smg_phase.cu)
cudaError_t launch_phase(const smg_handle* h, int phase, int kfilter, cudaStream_t s);
// strip kernels: mode 0 = phase A with filter k, 1 = phase B, 2 = fused A(k=2) A(k=1)
cudaError_t launch_strip(const smg_handle* h, int mode, int kfilter, cudaStream_t s);
cudaError_t launch_pair(const smg_handle* h, int mode, int kfilter, cudaStream_t s);
int strip_smem_bytes(const smg_handle* h, int phase);
cudaError_t strip_init(const smg_handle* h);
constexpr int kStripWarps = 8;
constexpr int kSumsqBlocks = 32;     // CTAs per component in the sum-of-squares reduction
constexpr int kSumsqThreads = 256;
void set_global_error(const std::string& msg);   // message of smg_last_error(NULL)
// No C++ exception reaches a caller of the C ABI: every entry point's body
// sits between SMG_TRY and SMG_CATCH(err), and an exception that escapes it
// (host memory exhausted, a thread that cannot be started) becomes SMG_ENOMEM
// or SMG_EINVAL with "<entry point>: <what>" in *err (the handle's message),
// or in the handle-less message when err is NULL.  Called only from a catch
// handler.
int exception_status(std::string* err, const char* fn) noexcept;
int run_steps(smg_handle* h, int64_t nsteps, bool events);   // smg_run without argument checks
int jit_build(smg_handle* h, std::string& err);             // generate, compile, load (SMG_OK or error)
void jit_free(smg_handle* h);
cudaError_t launch_jit(const smg_handle* h, int mode, int kfilter, cudaStream_t s);
int jit_build_rec(smg_handle* h, std::string& err);
int jit_build_adj(smg_handle* h, std::string& err);
cudaError_t launch_jit_adj(const smg_handle* h, int l, int coup, int pm, int pm_swap, int nm, int nm_swap, double* Y,
                           const DevField* DE, double* const* Gt, const double* pre, const double* W, cudaStream_t s);
int jit_adj_launches(const smg_handle* h, int l);
int jit_family_build(const std::vector<smg_handle*>& inst, int block, int group, int split, int regs,
                     JitFamilySet*& out, std::string& err);
void jit_family_free(JitFamilySet*& S);
cudaError_t jit_family_geometry(JitFamilySet* S, const std::vector<smg_handle*>& inst, cudaStream_t s);
cudaError_t jit_family_phase(JitFamilySet* S, int mode, int kfilter, cudaStream_t s, int64_t* launches);
int jit_family_count(const JitFamilySet* S);
// generated recording kernels: each destination's sigma-gradient factor for a phase of dsm substeps whose
// first filter is k=2 when dsw, into wrec (prec unused)
cudaError_t launch_jit_rec(const smg_handle* h, int mode, int kfilter, double* U, double* wrec, double* prec,
                           const DevField* DE, int dsm, int dsw, cudaStream_t s);
std::string jit_source(const smg_handle* h, int block, int group);
int jit_compile(const smg_handle* h, int block, int group, std::string& err);   // compile only (no device)
int jit_launches(const smg_handle* h, int phase);                                 // kernels per phase
int jit_status(smg_handle* h);              // SMG_ETIMEOUT if a staged kernel's bounded wait ran out (clears it)
int jit_form(const smg_handle* h);   // form of the loaded plain kernels: 0 register, 1/2 staged (bulk / async copies)
int src_build(smg_handle* h, std::string& err);       // compile the smg_set_source_expr kernels
void src_free(smg_handle* h, bool coords);            // unload them (and free their coordinates)
cudaError_t launch_src(const smg_handle* h, double t, cudaStream_t s);
cudaError_t launch_mat(smg_handle* h, double t, double dt, bool init, cudaStream_t s);
cudaError_t launch_filt(const smg_handle* h, double t, double dt, cudaStream_t s);
int create_host(const smg_problem* p, smg_handle** out);   // host tables only (no CUDA call)
cudaError_t launch_sumsq(const double* x, int ncomp, long long stride, long long len, double* partial, double* out,
                         cudaStream_t s);
constexpr int kMaxStripSmem = 200 * 1024;
constexpr int kJobCap = 48;          // slot jobs per stage; larger stages are split
constexpr int kMaxFieldRows = 64;    // coefficient rows cached per strip
cudaError_t launch_full_filter(const smg_handle* h, cudaStream_t s);
cudaError_t launch_decay(double* out, const double* sigma, long long n, double dt, cudaStream_t s);
cudaError_t launch_finite(const smg_handle* h, int* flag, cudaStream_t s);
}  // namespace smg
