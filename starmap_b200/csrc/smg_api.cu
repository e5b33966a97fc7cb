// smg_api.cu -- C ABI entry points of libstarmap_gpu (include/starmap_gpu.h).
//
// Host runtime: descriptor validation, kernel-axis layout, the coupling lists
// of the reference (Ix/Iy/Iz, starmap_solver.m:77-79, folded in sumcell order,
// starmap_solver.m:350-351, 516-519), coefficient upload, the step loop
// (starmap_solver.m:310-421) replayed from a captured CUDA graph, and state
// transfer in MATLAB's column-major component layout.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/starmap_gpu.h"
#include "smg_internal.h"

using smg::DevComp;
using smg::DevCoup;
using smg::DevField;

namespace {

// last handle-less failure of the calling thread: smg_last_error(NULL)
// returns a pointer into it that stays valid until that thread's next
// handle-less failure, whatever other threads do meanwhile
thread_local std::string g_err;

int fail(smg_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    else g_err = msg;
    return code;
}

int cuda_fail(smg_handle* h, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    if (e == cudaErrorMemoryAllocation) return fail(h, SMG_ENOMEM, m);
    return fail(h, SMG_ECUDA, m);
}

#define SMG_CUDA(h, expr)                                      \
    do {                                                       \
        cudaError_t e_ = (expr);                               \
        if (e_ != cudaSuccess) return cuda_fail((h), e_, #expr); \
    } while (0)

// expm1div of the reference (starmap_solver.m:531-535) for scalar fields.
double expm1div_host(double x) {
    double y = 1 + x * .5 + x * x / 6;
    if (std::fabs(x) > 2e-4) y = (std::exp(x) - 1) / x;
    return y;
}

int extent(int n, int bc, int g) { return (g == 2 && bc == 1) ? n + 1 : n; }

void resolve_pair(smg_handle* h, int phase);
cudaError_t upload_pair(smg_handle* h, int phase, bool alloc);
int create_impl(const smg_problem* p, smg_handle** out, bool device);

void free_device(smg_handle* h) {
    smg_adjoint_free(h);
    smg::jit_free(h);
    smg::src_free(h, true);
    if (h->graph) cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
    cudaFree(h->dU);
    cudaFree(h->dSnap);
    h->dSnap = nullptr;
    h->snap_set = false;
    cudaFree(h->dStage);
    h->dStage = nullptr;
    h->stage_bytes = 0;
    cudaFree(h->dFields);
    cudaFree(h->dComps);
    cudaFree(h->dCoups);
    cudaFree(h->dFieldTab);
    cudaFree(h->dDest);
    cudaFree(h->dFlag);
    cudaFree(h->dSumsq);
    h->dSumsq = nullptr;
    for (auto& sc : h->sched) {
        cudaFree(sc.dmem);
        sc.dmem = nullptr;
    }
    for (auto& pr : h->pair) {
        cudaFree(pr.d_dests);
        cudaFree(pr.d_coff);
        cudaFree(pr.d_cw);
        pr.d_dests = nullptr;
        pr.d_coff = nullptr;
        pr.d_cw = nullptr;
    }
    h->dU = h->dFields = nullptr;
    h->dComps = nullptr;
    h->dCoups = nullptr;
    h->dFieldTab = nullptr;
    h->dDest = h->dFlag = nullptr;
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    for (cudaEvent_t* ev : {&h->xev_fork, &h->xev_join, &h->xev_full[0], &h->xev_full[1], &h->xev_free[0],
                            &h->xev_free[1]}) {
        if (*ev) cudaEventDestroy(*ev);
        *ev = nullptr;
    }
    if (h->xstream) cudaStreamDestroy(h->xstream);
    h->xstream = nullptr;
    if (h->stream) cudaStreamDestroy(h->stream);
    h->ev0 = h->ev1 = nullptr;
    h->stream = nullptr;
}

// State transfers go through a staging buffer: each component (in pieces of
// whole rows where it exceeds the buffer) is one linear copy -- the copy
// engines move padded rows of a few KB several times slower than contiguous
// data -- and one kernel scatters a chunk into (or gathers it from) the
// padded slots.
constexpr size_t kStageBytes = 64u << 20;
constexpr int kXferMax = 64;   // components per chunk (kernel parameter space)

struct XferChunk {
    int n;
    int e0[kXferMax], e1[kXferMax], row0[kXferMax], rows[kXferMax];
    long long stage_off[kXferMax], slot_off[kXferMax];
};

// Entry k of a chunk: rows row0 .. row0+rows-1 (row = y + e1*z) of one
// component, compact in the staging buffer.  to_slots: stage -> padded
// slots; else slots -> stage, or with snap the interpolation
// wa*snap + wb*U (the output-time interpolation, starmap_solver.m:425-473).
// blockIdx.z is the entry, x runs along rows, blockIdx.y strides over rows.
__global__ void k_xfer(XferChunk c, double* __restrict__ stage, double* __restrict__ U,
                       const double* __restrict__ snap, double wa, double wb, long long s1, long long s2,
                       int to_slots) {
    const int k = blockIdx.z;
    if (k >= c.n) return;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int e0 = c.e0[k], e1 = c.e1[k];
    if (x >= e0) return;
    double* st = stage + c.stage_off[k];
    double* sl = U + c.slot_off[k];
    for (int r = blockIdx.y; r < c.rows[k]; r += gridDim.y) {
        const int row = c.row0[k] + r;
        const long long d = (long long)(row / e1) * s2 + (long long)(row % e1) * s1 + x;
        const long long q = (long long)r * e0 + x;
        if (to_slots) sl[d] = st[q];
        else if (snap) st[q] = __dadd_rn(__dmul_rn(wa, snap[c.slot_off[k] + d]), __dmul_rn(wb, sl[d]));
        else st[q] = sl[d];
    }
}

cudaError_t xfer_launch(const smg_handle* h, const XferChunk& c, double* stage, bool to_slots,
                        const double* snap = nullptr, double wa = 0.0, double wb = 0.0) {
    int e0max = 1, rows_max = 1;
    for (int k = 0; k < c.n; ++k) {
        e0max = std::max(e0max, c.e0[k]);
        rows_max = std::max(rows_max, c.rows[k]);
    }
    dim3 grid((unsigned)((e0max + 127) / 128), (unsigned)std::min(rows_max, 4096), (unsigned)c.n);
    k_xfer<<<grid, 128, 0, h->stream>>>(c, stage, h->dU, snap, wa, wb, h->g.s1, h->g.s2, to_slots ? 1 : 0);
    return cudaGetLastError();
}

// Direct transfer: up to kXferMax whole components whose host arrays are
// page-locked, so that the kernel reads (upload) or writes (download) them
// in place through their device addresses (unified addressing); entry k is
// component slot slot_off[k] with host array hp[k] of e0 x rows points.
struct XferDirect {
    int n;
    int e0[kXferMax], e1[kXferMax], rows[kXferMax];
    double* hp[kXferMax];
    long long slot_off[kXferMax];
};

__global__ void k_xfer_direct(XferDirect c, double* __restrict__ U, const double* __restrict__ snap, double wa,
                              double wb, long long s1, long long s2, int to_slots) {
    const int k = blockIdx.z;
    if (k >= c.n) return;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int e0 = c.e0[k], e1 = c.e1[k];
    if (x >= e0) return;
    double* hp = c.hp[k];
    double* sl = U + c.slot_off[k];
    for (int r = blockIdx.y; r < c.rows[k]; r += gridDim.y) {
        const long long d = (long long)(r / e1) * s2 + (long long)(r % e1) * s1 + x;
        const long long q = (long long)r * e0 + x;
        if (to_slots) sl[d] = hp[q];
        else if (snap) hp[q] = __dadd_rn(__dmul_rn(wa, snap[c.slot_off[k] + d]), __dmul_rn(wb, sl[d]));
        else hp[q] = sl[d];
    }
}

// Device address of one page-locked host byte, or NULL (pageable memory).
char* host_byte_view(const void* q) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, q) != cudaSuccess) {
        cudaGetLastError();   // clear the error of an unregistered pointer
        return nullptr;
    }
    return a.type == cudaMemoryTypeHost ? static_cast<char*>(a.devicePointer) : nullptr;
}

// Device address of the page-locked host range [p, p + bytes), or NULL when
// its first or last byte is not page-locked or the two are not mapped as one
// contiguous range (an array only partly registered goes through staging:
// the direct kernel must never touch an unmapped host page).
double* device_view(const void* p, size_t bytes) {
    if (bytes == 0) return nullptr;
    char* first = host_byte_view(p);
    if (!first) return nullptr;
    char* last = host_byte_view(static_cast<const char*>(p) + (bytes - 1));
    return last == first + (bytes - 1) ? reinterpret_cast<double*>(first) : nullptr;
}

// Transfer of the components with non-NULL host pointers.  When every one of
// them is page-locked, one kernel per kXferMax components moves them between
// the host arrays and the padded slots directly (no staging copies);
// otherwise the staged form below.
int direct_transfer(smg_handle* h, bool upload, const std::vector<double*>& hp, const double* snap, double wa,
                    double wb) {
    XferDirect c;
    c.n = 0;
    int e0max = 1, rows_max = 1;
    auto flush = [&]() -> cudaError_t {
        if (!c.n) return cudaSuccess;
        dim3 grid((unsigned)((e0max + 127) / 128), (unsigned)std::min(rows_max, 2048), (unsigned)c.n);
        k_xfer_direct<<<grid, 128, 0, h->stream>>>(c, h->dU, snap, wa, wb, h->g.s1, h->g.s2, upload ? 1 : 0);
        c.n = 0;
        e0max = rows_max = 1;
        return cudaGetLastError();
    };
    for (int j = 0; j < h->n_sys; ++j) {
        if (!hp[j]) continue;
        const int* e = h->comps[j].ext;
        if (c.n == kXferMax) SMG_CUDA(h, flush());
        c.e0[c.n] = e[0];
        c.e1[c.n] = e[1];
        c.rows[c.n] = e[1] * e[2];
        c.hp[c.n] = hp[j];
        c.slot_off[c.n] = (long long)j * h->g.cs;
        e0max = std::max(e0max, e[0]);
        rows_max = std::max(rows_max, e[1] * e[2]);
        ++c.n;
    }
    SMG_CUDA(h, flush());
    SMG_CUDA(h, cudaStreamSynchronize(h->stream));
    return SMG_OK;
}

// The staged transfer of the components with non-NULL host pointers: each
// component in pieces of whole rows that fit the staging buffer (a piece is
// one contiguous range of the column-major host array), up to kXferMax
// pieces per kernel launch.  Upload: copy the pieces in, then scatter.
// Download: gather (or interpolate with snap), then copy the pieces out.
// Page-locked host arrays go through direct_transfer instead.
int staged_transfer(smg_handle* h, bool upload, const double* const* Uin, double* const* Uout,
                    const double* snap, double wa, double wb) {
    // page-lock state of every host array: whole (its device address), none,
    // or only in part (its first byte locked, the rest not all)
    const int ns = h->n_sys;
    std::vector<char*> host(ns, nullptr);
    std::vector<double*> lockdev(ns, nullptr);
    std::vector<char> partly(ns, 0);
    std::vector<size_t> nbytes(ns, 0);
    int arrays = 0, runs = 0, locked = 0;
    std::vector<std::pair<int, int>> run_span;   // first and last array of each host-contiguous run
    const char* end = nullptr;
    for (int j = 0; j < ns; ++j) {
        host[j] = upload ? const_cast<char*>(reinterpret_cast<const char*>(Uin[j])) : reinterpret_cast<char*>(Uout[j]);
        if (!host[j]) continue;
        const int* e = h->comps[j].ext;
        nbytes[j] = (size_t)e[0] * e[1] * e[2] * sizeof(double);
        ++arrays;
        if (host[j] != end) {
            ++runs;
            run_span.push_back({j, j});
        }
        run_span.back().second = j;
        end = host[j] + nbytes[j];
    }
    // one query pair per run when the run is page-locked and mapped as one
    // range (arrays carved from one block), else per array
    for (const auto& rs : run_span) {
        const size_t span = (size_t)(host[rs.second] + nbytes[rs.second] - host[rs.first]);
        if (double* dv = rs.first < rs.second ? device_view(host[rs.first], span) : nullptr) {
            for (int j = rs.first; j <= rs.second; ++j)
                if (host[j]) lockdev[j] = reinterpret_cast<double*>(reinterpret_cast<char*>(dv) + (host[j] - host[rs.first]));
            continue;
        }
        for (int j = rs.first; j <= rs.second; ++j) {
            if (!host[j]) continue;
            lockdev[j] = device_view(host[j], nbytes[j]);
            partly[j] = !lockdev[j] && host_byte_view(host[j]) != nullptr;
        }
    }
    for (int j = 0; j < ns; ++j) locked += lockdev[j] != nullptr;
    // every array page-locked: in place, unless the arrays are carved in
    // order from one host block (a few contiguous runs), which large
    // copy-engine copies through the staging buffer move faster (about 43
    // against 37 GB/s measured; separate arrays are faster in place)
    if (h->direct_xfer && arrays > 0 && locked == arrays && runs * 8 > arrays)
        return direct_transfer(h, upload, lockdev, snap, wa, wb);
    // An array page-locked only in part cannot be the range of one copy (the
    // driver takes the range for page-locked memory and refuses it past the
    // registration): it goes through a pageable host bounce buffer.
    std::vector<std::vector<double>> bounce(ns);
    for (int j = 0; j < ns; ++j) {
        if (!partly[j]) continue;
        bounce[j].resize(nbytes[j] / sizeof(double));
        if (upload) std::memcpy(bounce[j].data(), host[j], nbytes[j]);
    }
    // Staged form.  The pieces of a chunk are packed into one half of the
    // staging buffer while the other half is scattered into the slots
    // (upload) or copied out to the host (download): the linear copies run on
    // a copy stream, the kernels on the handle's stream, and events pass each
    // half between the two, so the copy engine runs back to back.  Pieces
    // whose host bytes follow each other (component arrays carved in order
    // from one host block) are moved by one copy.  A problem whose rows do
    // not fit half the buffer uses it whole, one chunk at a time.
    if (!h->xstream) {
        SMG_CUDA(h, cudaStreamCreateWithFlags(&h->xstream, cudaStreamNonBlocking));
        for (cudaEvent_t* ev : {&h->xev_fork, &h->xev_join, &h->xev_full[0], &h->xev_full[1], &h->xev_free[0],
                                &h->xev_free[1]})
            SMG_CUDA(h, cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
    }
    size_t row_max = 0;
    for (int j = 0; j < h->n_sys; ++j)
        if (upload ? Uin[j] : Uout[j]) row_max = std::max(row_max, (size_t)h->comps[j].ext[0] * 8);
    const size_t half = h->stage_bytes / 2 / 256 * 256;
    const int nbuf = half >= row_max && half > 0 ? 2 : 1;
    const size_t cap = nbuf == 2 ? half : h->stage_bytes;
    if (row_max > cap) return fail(h, SMG_EINVAL, "state transfer: a row exceeds the staging buffer");
    auto base = [&](int b) { return reinterpret_cast<char*>(h->dStage) + (size_t)b * cap; };
    // the copy stream starts after all work queued on the handle's stream
    SMG_CUDA(h, cudaEventRecord(h->xev_fork, h->stream));
    SMG_CUDA(h, cudaStreamWaitEvent(h->xstream, h->xev_fork, 0));
    int buf = 0;
    XferChunk c;
    c.n = 0;
    size_t used = 0;
    // dev: the piece's device address when its array is page-locked whole
    struct Piece { char* host; char* dev; size_t stage_off, bytes; };
    std::vector<Piece> pend;
    // the chunk's linear copies, host-adjacent pieces merged (they are
    // adjacent in the stage too) while the merged range stays one kind of
    // memory for the driver: a run that starts in pageable memory takes any
    // adjacent piece; a page-locked run only pieces that continue its device
    // mapping
    auto copies = [&]() -> cudaError_t {
        for (size_t i = 0; i < pend.size();) {
            size_t k = i + 1, bytes = pend[i].bytes;
            while (k < pend.size() && pend[k].host == pend[i].host + bytes &&
                   (!pend[i].dev || pend[k].dev == pend[i].dev + bytes))
                bytes += pend[k++].bytes;
            const cudaError_t e =
                upload ? cudaMemcpyAsync(base(buf) + pend[i].stage_off, pend[i].host, bytes, cudaMemcpyHostToDevice,
                                         h->xstream)
                       : cudaMemcpyAsync(pend[i].host, base(buf) + pend[i].stage_off, bytes, cudaMemcpyDeviceToHost,
                                         h->xstream);
            if (e != cudaSuccess) return e;
            i = k;
        }
        return cudaSuccess;
    };
    auto flush = [&]() -> cudaError_t {
        if (!c.n) return cudaSuccess;
        cudaError_t e = cudaSuccess;
        double* stage = reinterpret_cast<double*>(base(buf));
        if (upload) {
            // copy into the half once its previous scatter is done, then scatter it
            if ((e = cudaStreamWaitEvent(h->xstream, h->xev_free[buf], 0)) != cudaSuccess ||
                (e = copies()) != cudaSuccess || (e = cudaEventRecord(h->xev_full[buf], h->xstream)) != cudaSuccess ||
                (e = cudaStreamWaitEvent(h->stream, h->xev_full[buf], 0)) != cudaSuccess ||
                (e = xfer_launch(h, c, stage, true)) != cudaSuccess ||
                (e = cudaEventRecord(h->xev_free[buf], h->stream)) != cudaSuccess)
                return e;
        } else {
            // gather into the half once its previous copies out are done, then copy it out
            if ((e = cudaStreamWaitEvent(h->stream, h->xev_free[buf], 0)) != cudaSuccess ||
                (e = xfer_launch(h, c, stage, false, snap, wa, wb)) != cudaSuccess ||
                (e = cudaEventRecord(h->xev_full[buf], h->stream)) != cudaSuccess ||
                (e = cudaStreamWaitEvent(h->xstream, h->xev_full[buf], 0)) != cudaSuccess ||
                (e = copies()) != cudaSuccess || (e = cudaEventRecord(h->xev_free[buf], h->xstream)) != cudaSuccess)
                return e;
        }
        c.n = 0;
        used = 0;
        pend.clear();
        buf = (buf + 1) % nbuf;
        return cudaSuccess;
    };
    for (int j = 0; j < ns; ++j) {
        if (!host[j]) continue;
        char* src = partly[j] ? reinterpret_cast<char*>(bounce[j].data()) : host[j];
        char* dev = reinterpret_cast<char*>(lockdev[j]);
        const int* e = h->comps[j].ext;
        const size_t row_bytes = (size_t)e[0] * 8;
        const int rows = e[1] * e[2];
        const int max_rows = (int)std::max<size_t>(1, cap / row_bytes);
        for (int r0 = 0; r0 < rows; r0 += max_rows) {
            const int nr = std::min(max_rows, rows - r0);
            const size_t bytes = (size_t)nr * row_bytes;
            if (c.n == kXferMax || used + bytes > cap) SMG_CUDA(h, flush());
            c.e0[c.n] = e[0];
            c.e1[c.n] = e[1];
            c.row0[c.n] = r0;
            c.rows[c.n] = nr;
            c.stage_off[c.n] = (long long)(used / 8);
            c.slot_off[c.n] = (long long)j * h->g.cs;
            ++c.n;
            pend.push_back({src + (size_t)r0 * row_bytes, dev ? dev + (size_t)r0 * row_bytes : nullptr, used, bytes});
            used += bytes;
        }
    }
    SMG_CUDA(h, flush());
    // everything of this transfer is ordered before later work on the handle's stream
    SMG_CUDA(h, cudaEventRecord(h->xev_join, h->xstream));
    SMG_CUDA(h, cudaStreamWaitEvent(h->stream, h->xev_join, 0));
    SMG_CUDA(h, cudaStreamSynchronize(h->stream));
    if (!upload)
        for (int j = 0; j < ns; ++j)
            if (partly[j]) std::memcpy(host[j], bounce[j].data(), nbytes[j]);
    return SMG_OK;
}

// Copy a column-major host array with extents e[] (kernel axes) into a
// padded device slot (field uploads).
cudaError_t put_slot(const smg_handle* h, double* dst, const double* src, const int e[3]) {
    cudaMemcpy3DParms p{};
    p.srcPtr = make_cudaPitchedPtr((void*)src, (size_t)e[0] * 8, (size_t)e[0], (size_t)e[1]);
    p.dstPtr = make_cudaPitchedPtr(dst, (size_t)h->g.s1 * 8, (size_t)h->g.s1, (size_t)h->g.B[1]);
    p.extent = make_cudaExtent((size_t)e[0] * 8, (size_t)e[1], (size_t)e[2]);
    p.kind = cudaMemcpyHostToDevice;
    return cudaMemcpy3DAsync(&p, h->stream);
}

void grid_extents(const smg_handle* h, const int gt_solver[3], int e[3]) {
    for (int a = 0; a < 3; ++a) {
        const int d = h->sd[a];
        e[a] = extent(h->g.n[a], h->g.bc[a], gt_solver[d]);
    }
}

// Strip schedule of one phase.  Destinations are grouped into stages by their
// breadth-first level in the coupling graph rooted at component 0 (for P_N and
// SP_N this level is the moment order, and a destination of order m only
// reads sources of orders m-1 and m+1).  Each derivative (source, axis) is
// computed in the stage of its first use and its shared-memory slot is
// released after its last use, so at most two source orders are live.
void build_schedule(smg_handle* h, int phase, const std::vector<int>& level) {
    using smg::DestJob;
    using smg::SCoup;
    using smg::SlotJob;
    using smg::Stage;
    auto& S = h->sched[phase];
    S = smg_handle::HostSched{};
    const std::vector<int>& D = phase == 0 ? h->destA : h->destB;
    if (D.empty()) {
        S.ok = true;
        return;
    }
    std::map<int, std::vector<int>> bylev;
    for (int j : D) bylev[level[j]].push_back(j);
    std::vector<std::vector<int>> groups;
    for (auto& kv : bylev) groups.push_back(kv.second);
    typedef std::pair<int, int> Key;   // (src, code)
    std::map<Key, std::pair<int, int>> use;   // first, last stage
    for (int s = 0; s < (int)groups.size(); ++s)
        for (int j : groups[s])
            for (int q = h->comps[j].cbeg; q < h->comps[j].cend; ++q) {
                const Key k(h->coups[q].src, h->coups[q].code);
                auto it = use.find(k);
                if (it == use.end()) use[k] = std::make_pair(s, s);
                else it->second.second = s;
            }
    std::vector<int> freelist;
    std::map<Key, int> slot_of;
    int nslots = 0;
    for (int s = 0; s < (int)groups.size(); ++s) {
        Stage st{};
        st.jbeg = (int)S.jobs.size();
        for (auto& kv : use) {
            if (kv.second.first != s) continue;
            int slot;
            if (!freelist.empty()) { slot = freelist.back(); freelist.pop_back(); }
            else slot = nslots++;
            slot_of[kv.first] = slot;
            SlotJob jb{};
            jb.src = kv.first.first;
            jb.code = kv.first.second;
            jb.slot = slot;
            const int ax = jb.code >> 1;
            for (int a = 0; a < 3; ++a) jb.ext[a] = h->comps[jb.src].ext[a];
            jb.ext[ax] = (jb.code & 1) ? h->g.n[ax] : h->g.n[ax] + h->g.bc[ax];
            S.jobs.push_back(jb);
        }
        st.jend = (int)S.jobs.size();
        // a stage with more slot jobs than the staging buffer holds is split
        // into job-only stages followed by the stage that updates destinations
        while (st.jend - st.jbeg > smg::kJobCap) {
            Stage pre{};
            pre.jbeg = st.jbeg;
            pre.jend = st.jbeg + smg::kJobCap;
            pre.dbeg = pre.dend = (int)S.dests.size();
            S.stages.push_back(pre);
            st.jbeg = pre.jend;
        }
        S.jcap = std::max(S.jcap, st.jend - st.jbeg);
        st.dbeg = (int)S.dests.size();
        for (int j : groups[s]) {
            DestJob dj{};
            dj.comp = j;
            for (int a = 0; a < 3; ++a) dj.ext[a] = h->comps[j].ext[a];
            dj.cbeg = (int)S.coups.size();
            for (int q = h->comps[j].cbeg; q < h->comps[j].cend; ++q)
                S.coups.push_back(SCoup{slot_of[Key(h->coups[q].src, h->coups[q].code)], 0, h->coups[q].w});
            dj.cend = (int)S.coups.size();
            S.dests.push_back(dj);
        }
        st.dend = (int)S.dests.size();
        S.stages.push_back(st);
        for (auto& kv : use)
            if (kv.second.second == s) freelist.push_back(slot_of[kv.first]);
    }
    S.nslots = std::max(nslots, 1);
    S.ok = (S.nslots * 32 + S.jcap * 64) * 8 <= smg::kMaxStripSmem;
}

// Resolve the coefficients of every destination of a schedule: arrays become
// rows of the strip's shared-memory cache, scalars are stored in the job.
// Called at creation and whenever a scalar coefficient changes.
void resolve_coefs(smg_handle* h, int phase) {
    auto& S = h->sched[phase];
    std::map<int, int> row_of;
    S.frows.clear();
    for (auto& dj : S.dests) {
        const smg::DevComp& c = h->comps[dj.comp];
        int f[smg::kNumCoef];
        if (phase == 1 && dj.comp == 0) {
            f[smg::kCoefS] = h->sigma_a;
            f[smg::kCoefE] = h->decay_a >= 0 ? h->decay_a : h->derived_decay_a;
            f[smg::kCoefF1] = f[smg::kCoefF2] = h->field_one;
        } else {
            f[smg::kCoefS] = c.sT;
            f[smg::kCoefE] = c.ET;
            f[smg::kCoefF1] = c.F1;
            f[smg::kCoefF2] = c.F2;
        }
        f[smg::kCoefQ] = c.Q;
        for (int k = 0; k < smg::kNumCoef; ++k) {
            const smg::DevField& F = h->fields_host[f[k]];
            if (F.p) {
                auto it = row_of.find(f[k]);
                if (it == row_of.end()) {
                    it = row_of.emplace(f[k], (int)S.frows.size()).first;
                    S.frows.push_back(f[k]);
                }
                dj.row[k] = it->second;
                dj.sc[k] = 0.0;
            } else {
                dj.row[k] = -1;
                dj.sc[k] = F.s;
            }
        }
    }
}

cudaError_t upload_schedule(smg_handle* h, int phase) {
    auto& S = h->sched[phase];
    S.view = smg::StripSched{};
    if (!S.ok || S.stages.empty()) return cudaSuccess;
    const size_t b0 = S.stages.size() * sizeof(smg::Stage);
    const size_t b1 = S.jobs.size() * sizeof(smg::SlotJob);
    const size_t b2 = S.dests.size() * sizeof(smg::DestJob);
    const size_t b3 = S.coups.size() * sizeof(smg::SCoup);
    const size_t b4 = S.frows.size() * sizeof(int);
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t tot = al(b0) + al(b1) + al(b2) + al(b3) + al(b4) + 256;
    cudaError_t e = cudaMalloc(&S.dmem, tot);
    if (e != cudaSuccess) return e;
    h->bytes += tot;
    char* p = (char*)S.dmem;
    char* p0 = p; p += al(b0);
    char* p1 = p; p += al(b1);
    char* p2 = p; p += al(b2);
    char* p3 = p; p += al(b3);
    char* p4 = p;
    if ((e = cudaMemcpyAsync(p0, S.stages.data(), b0, cudaMemcpyHostToDevice, h->stream)) != cudaSuccess) return e;
    if (b1 && (e = cudaMemcpyAsync(p1, S.jobs.data(), b1, cudaMemcpyHostToDevice, h->stream)) != cudaSuccess) return e;
    if (b2 && (e = cudaMemcpyAsync(p2, S.dests.data(), b2, cudaMemcpyHostToDevice, h->stream)) != cudaSuccess) return e;
    if (b3 && (e = cudaMemcpyAsync(p3, S.coups.data(), b3, cudaMemcpyHostToDevice, h->stream)) != cudaSuccess) return e;
    if (b4 && (e = cudaMemcpyAsync(p4, S.frows.data(), b4, cudaMemcpyHostToDevice, h->stream)) != cudaSuccess) return e;
    S.view.stages = (const smg::Stage*)p0;
    S.view.jobs = (const smg::SlotJob*)p1;
    S.view.dests = (const smg::DestJob*)p2;
    S.view.coups = (const smg::SCoup*)p3;
    S.view.frows = (const int*)p4;
    S.view.nstages = (int)S.stages.size();
    S.view.nslots = S.nslots;
    S.view.jcap = S.jcap;
    S.view.nfrows = (int)S.frows.size();
    return cudaSuccess;
}

// Re-resolve scalar coefficients of both schedules and refresh the device copy
// of the destination tables (same sizes, so the graph stays valid).
cudaError_t refresh_coefs(smg_handle* h) {
    for (int ph = 0; ph < 2; ++ph) {
        if (h->pair[ph].d_dests) {
            resolve_pair(h, ph);
            cudaError_t e = upload_pair(h, ph, false);
            if (e != cudaSuccess) return e;
        }
    }
    for (int ph = 0; ph < 2; ++ph) {
        auto& S = h->sched[ph];
        if (!S.ok || S.stages.empty() || !S.view.dests) continue;
        resolve_coefs(h, ph);
        cudaError_t e = cudaMemcpyAsync((void*)S.view.dests, S.dests.data(), S.dests.size() * sizeof(smg::DestJob),
                                        cudaMemcpyHostToDevice, h->stream);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Pair-kernel tables of one phase: destinations ordered by coupling-graph
// level (neighbouring CTAs then share sources in L1/L2), couplings in sumcell
// order with the source slot offset, coefficients resolved to a device array
// pointer or a scalar.
void build_pair(smg_handle* h, int phase, const std::vector<int>& level) {
    auto& P = h->pair[phase];
    P.dests.clear();
    P.coff.clear();
    P.cw.clear();
    P.ok = (long long)h->n_sys * h->g.cs < (1LL << 31);   // 32-bit element offsets
    std::vector<int> D = phase == 0 ? h->destA : h->destB;
    std::stable_sort(D.begin(), D.end(), [&](int a, int b) { return level[a] < level[b]; });
    for (int j : D) {
        smg::PairDest d{};
        d.off = (int)((long long)j * h->g.cs);
        for (int k = 0; k < 3; ++k) d.ext[k] = h->comps[j].ext[k];
        int nr = 0;
        int prev = -1;
        for (int q = h->comps[j].cbeg; q < h->comps[j].cend; ++q) {
            const int code = h->coups[q].code;
            if (code != prev) {
                if (nr == smg::kPairRuns) { P.ok = false; break; }
                d.run[nr] = (int)P.coff.size();
                d.code[nr] = code;
                ++nr;
                prev = code;
            }
            P.coff.push_back((int)((long long)h->coups[q].src * h->g.cs));
            P.cw.push_back(h->coups[q].w);
        }
        for (int r = nr; r <= smg::kPairRuns; ++r) d.run[r] = (int)P.coff.size();
        for (int r = nr; r < smg::kPairRuns; ++r) d.code[r] = 0;
        P.dests.push_back(d);
    }
    P.ndest = (int)P.dests.size();
}

void resolve_pair(smg_handle* h, int phase) {
    auto& P = h->pair[phase];
    for (auto& d : P.dests) {
        const int j = (int)((long long)d.off / h->g.cs);
        const smg::DevComp& c = h->comps[j];
        int f[smg::kNumCoef];
        if (phase == 1 && j == 0) {
            f[smg::kCoefS] = h->sigma_a;
            f[smg::kCoefE] = h->decay_a >= 0 ? h->decay_a : h->derived_decay_a;
            f[smg::kCoefF1] = f[smg::kCoefF2] = h->field_one;
        } else {
            f[smg::kCoefS] = c.sT;
            f[smg::kCoefE] = c.ET;
            f[smg::kCoefF1] = c.F1;
            f[smg::kCoefF2] = c.F2;
        }
        f[smg::kCoefQ] = c.Q;
        for (int k = 0; k < smg::kNumCoef; ++k) {
            const smg::DevField& F = h->fields_host[f[k]];
            d.fp[k] = F.p;
            d.sc[k] = F.p ? 0.0 : F.s;
        }
    }
}

cudaError_t upload_pair(smg_handle* h, int phase, bool alloc) {
    auto& P = h->pair[phase];
    if (P.ndest == 0 || !P.ok) return cudaSuccess;
    cudaError_t e;
    if (alloc) {
        const size_t nc = std::max<size_t>(P.coff.size(), 1);
        if ((e = cudaMalloc(&P.d_dests, sizeof(smg::PairDest) * P.dests.size())) != cudaSuccess) return e;
        if ((e = cudaMalloc(&P.d_coff, sizeof(int) * nc)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&P.d_cw, sizeof(double) * nc)) != cudaSuccess) return e;
        h->bytes += sizeof(smg::PairDest) * P.dests.size() + (sizeof(int) + sizeof(double)) * nc;
        if (!P.coff.empty()) {
            if ((e = cudaMemcpyAsync(P.d_coff, P.coff.data(), sizeof(int) * P.coff.size(), cudaMemcpyHostToDevice,
                                     h->stream)) != cudaSuccess)
                return e;
            if ((e = cudaMemcpyAsync(P.d_cw, P.cw.data(), sizeof(double) * P.cw.size(), cudaMemcpyHostToDevice,
                                     h->stream)) != cudaSuccess)
                return e;
        }
    }
    return cudaMemcpyAsync(P.d_dests, P.dests.data(), sizeof(smg::PairDest) * P.dests.size(),
                           cudaMemcpyHostToDevice, h->stream);
}

// RN(1/h) per axis and the division mode of recip_div (smg_device.cuh):
// 2 when |RN(1/h)*h - 1| < 2^-54, 1 for other normal h, 0 otherwise.
void reciprocals(smg_handle* h) {
    bool used[3] = {false, false, false};
    for (const auto& c : h->coups) used[c.code >> 1] = true;
    for (int a = 0; a < 3; ++a) {
        const double hv = h->g.h[a];
        const double r = 1.0 / hv;
        const double e = std::fma(r, hv, -1.0);
        h->rh[a] = r;
        int mode = 0;
        if (std::isnormal(hv) && std::isnormal(r)) mode = std::fabs(e) < std::ldexp(1.0, -54) ? 2 : 1;
        // an axis without differences never divides; it does not restrict the kernels
        h->exact_recip[a] = used[a] ? mode : 2;
    }
}

// Expressions evaluated on the device are spliced into generated kernels, so
// they are held to a small grammar that cannot reach memory or leave the
// expression: numbers, the variables of the expression's kind, the math
// functions below, + - * / % < > <= >= == != && || ! ?: ( ) and commas.  No
// brackets, braces, semicolons, assignments, address or pointer syntax, type
// names or string/char literals.  Returns "" when the expression is
// acceptable, else why not.
std::string expr_problem(const char* expr, int kind) {
    static const std::set<std::string> fns = {
        "sin",   "cos",   "tan",   "asin",  "acos",     "atan",      "atan2", "sinh",  "cosh",   "tanh",
        "asinh", "acosh", "atanh", "exp",   "exp2",     "exp10",     "expm1", "log",   "log2",   "log10",
        "log1p", "pow",   "sqrt",  "rsqrt", "cbrt",     "hypot",     "fabs",  "abs",   "fmin",   "fmax",
        "min",   "max",   "fmod",  "remainder", "floor", "ceil",     "round", "rint",  "trunc",  "copysign",
        "erf",   "erfc",  "tgamma", "lgamma", "sinpi",  "cospi",     "fdim",  "nearbyint", "true", "false"};
    static const char* vars[3][6] = {{"x", "y", "z", "t", "k", nullptr},
                                     {"x", "y", "z", "t", "m", nullptr},
                                     {"x", "y", "z", "t", "dt", "k"}};
    if (kind < 0 || kind > 2) return "unknown expression kind";
    if (!expr) return "NULL expression";
    const size_t n = std::strlen(expr);
    if (n == 0 || n > 65536) return "expression empty or over 64 KB";
    auto is_var = [&](const std::string& w) {
        for (const char* v : vars[kind])
            if (v && w == v) return true;
        return false;
    };
    int depth = 0;
    for (size_t i = 0; i < n;) {
        const unsigned char c = (unsigned char)expr[i];
        if (std::isspace(c)) {
            ++i;
        } else if (std::isdigit(c) || (c == '.' && i + 1 < n && std::isdigit((unsigned char)expr[i + 1]))) {
            // a decimal or hexadecimal floating literal with an optional exponent and suffix
            size_t j = i + 1;
            const bool hex = c == '0' && j < n && (expr[j] == 'x' || expr[j] == 'X');
            if (hex) ++j;
            while (j < n) {
                const char d = expr[j];
                const bool expo = hex ? (d == 'p' || d == 'P') : (d == 'e' || d == 'E');
                if (expo && j + 1 < n && (expr[j + 1] == '+' || expr[j + 1] == '-')) j += 2;
                else if (std::isxdigit((unsigned char)d) || d == '.' || expo) ++j;
                else break;
            }
            while (j < n && std::strchr("fFlLuU", expr[j])) ++j;
            if (j < n && (std::isalnum((unsigned char)expr[j]) || expr[j] == '_'))
                return "malformed number at offset " + std::to_string(i);
            i = j;
        } else if (std::isalpha(c) || c == '_') {
            size_t j = i;
            while (j < n && (std::isalnum((unsigned char)expr[j]) || expr[j] == '_')) ++j;
            const std::string w(expr + i, j - i);
            if (!is_var(w) && !fns.count(w))
                return "'" + w + "' is neither a variable of this expression nor an allowed math function";
            i = j;
        } else {
            static const char* ops2[] = {"<=", ">=", "==", "!=", "&&", "||"};
            bool two = false;
            for (const char* o : ops2)
                if (i + 1 < n && expr[i] == o[0] && expr[i + 1] == o[1]) two = true;
            if (two) {
                i += 2;
            } else if (std::strchr("+-*/%<>!?:(),", c)) {
                if (c == '(') ++depth;
                if (c == ')' && --depth < 0) return "unbalanced ')' at offset " + std::to_string(i);
                ++i;
            } else {
                return std::string("character '") + (char)c + "' at offset " + std::to_string(i) + " is not allowed";
            }
        }
    }
    if (depth != 0) return "unbalanced parentheses";
    return "";
}

bool strip_usable(const smg_handle* h) {
    return h->sched[0].ok && h->sched[1].ok && h->variant != SMG_VARIANT_GENERIC;
}

}  // namespace

void smg::set_global_error(const std::string& msg) { fail(nullptr, 0, msg); }

int smg::exception_status(std::string* err, const char* fn) noexcept {
    int code = SMG_EINVAL;
    const char* what = "unknown exception";
    try {
        throw;
    } catch (const std::bad_alloc&) {
        code = SMG_ENOMEM;
        what = "out of host memory";
    } catch (const std::length_error& e) {
        code = SMG_ENOMEM;
        what = e.what();
    } catch (const std::exception& e) {
        what = e.what();
    } catch (...) {
    }
    try {
        const std::string m = std::string(fn) + ": " + what;
        if (err) *err = m;
        else set_global_error(m);
    } catch (...) {   // no memory left for the message either
    }
    return code;
}
int smg::create_host(const smg_problem* p, smg_handle** out) { return create_impl(p, out, false); }

extern "C" {

const char* smg_version(void) { return "starmap_b200 0.1 (sm_100a, fp64)"; }

const char* smg_last_error(const smg_handle* h) {
    if (h) return h->err.c_str();
    return g_err.c_str();
}

int smg_device_count(void) {
    SMG_TRY
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return 0;
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaGetDeviceCount");
    return n;
    SMG_CATCH(nullptr)
}

int smg_set_device(int32_t device) {
    SMG_TRY
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaSetDevice");
    return SMG_OK;
    SMG_CATCH(nullptr)
}

int smg_classify(int32_t n_sys, const double* Mx, const double* My, const double* Mz, int32_t* gt_out) {
    SMG_TRY
    if (n_sys < 1 || !Mx || !My || !Mz || !gt_out) return fail(nullptr, SMG_EINVAL, "smg_classify: bad arguments");
    const double* M[3] = {Mx, My, Mz};
    // I[d][j]: sorted columns i with M_d(j,i) != 0 (starmap_solver.m:77-79)
    std::vector<std::vector<int>> I[3];
    // (one pass in memory order: column i outer, so each row's list ascends)
    for (int d = 0; d < 3; ++d) {
        I[d].resize(n_sys);
        for (int i = 0; i < n_sys; ++i) {
            const double* col = M[d] + (size_t)i * n_sys;
            for (int j = 0; j < n_sys; ++j)
                if (col[j] != 0.0) I[d][j].push_back(i);
        }
    }
    // class index = (gx-1) + 2(gy-1) + 4(gz-1); membership flags
    std::vector<int> cls(n_sys, -1);
    cls[0] = 0;
    int assigned = 1;
    // Fixed-point propagation: a component reached from class (gx,gy,gz) via
    // direction d lies on the class with that axis flipped (starmap_solver.m:82-91).
    for (int iter = 0; iter < 4 * n_sys + 8 && assigned < n_sys; ++iter) {
        bool changed = false;
        for (int j = 0; j < n_sys; ++j) {
            if (cls[j] < 0) continue;
            for (int d = 0; d < 3; ++d)
                for (int i : I[d][j]) {
                    const int c = cls[j] ^ (1 << d);
                    if (cls[i] < 0) { cls[i] = c; ++assigned; changed = true; }
                }
        }
        if (!changed) break;
    }
    if (assigned < n_sys)
        return fail(nullptr, SMG_EINVAL, "smg_classify: components not connected to component 1");
    // every coupling along d must join grids that differ in axis d alone; the
    // reference's set unions would put such a component on two grids at once
    for (int j = 0; j < n_sys; ++j)
        for (int d = 0; d < 3; ++d)
            for (int i : I[d][j])
                if (cls[i] != (cls[j] ^ (1 << d))) {
                    char buf[160];
                    std::snprintf(buf, sizeof buf,
                                  "smg_classify: M%c(%d,%d) couples components that admit no staggered grid types",
                                  "xyz"[d], j + 1, i + 1);
                    return fail(nullptr, SMG_EINVAL, buf);
                }
    for (int j = 0; j < n_sys; ++j)
        for (int d = 0; d < 3; ++d) gt_out[3 * j + d] = 1 + ((cls[j] >> d) & 1);
    return SMG_OK;
    SMG_CATCH(nullptr)
}

int smg_check_expr(int32_t kind, const char* expr) {
    SMG_TRY
    const std::string why = expr_problem(expr, kind);
    if (!why.empty()) return fail(nullptr, SMG_EINVAL, "smg_check_expr: " + why);
    return SMG_OK;
    SMG_CATCH(nullptr)
}

int smg_create(const smg_problem* p, smg_handle** out) { SMG_TRY return create_impl(p, out, true); SMG_CATCH(nullptr) }

}  // extern "C"

namespace {

// Breadth-first level of every component in the coupling graph from
// component 0 (unreached components after the last level).
std::vector<int> coupling_levels(const smg_handle* h) {
    const int ns = h->n_sys;
    std::vector<int> level(ns, -1), queue(1, 0);
    level[0] = 0;
    for (size_t qi = 0; qi < queue.size(); ++qi) {
        const int j = queue[qi];
        for (int q = h->comps[j].cbeg; q < h->comps[j].cend; ++q) {
            const int i = h->coups[q].src;
            if (level[i] < 0) { level[i] = level[j] + 1; queue.push_back(i); }
        }
    }
    int maxl = 0;
    for (int j = 0; j < ns; ++j) maxl = std::max(maxl, level[j]);
    for (int j = 0; j < ns; ++j) if (level[j] < 0) level[j] = maxl + 1;
    return level;
}

// smg_create; with device == false only the host tables (no CUDA call), for
// smg_jit_source on machines without a GPU
int create_impl(const smg_problem* p, smg_handle** out, bool device) {
    if (!p || !out) return fail(nullptr, SMG_EINVAL, "smg_create: NULL argument");
    *out = nullptr;
    const int ns = p->n_sys;
    if (ns < 1) return fail(nullptr, SMG_EINVAL, "n_sys must be >= 1");
    if (!p->gt || !p->Mx || !p->My || !p->Mz) return fail(nullptr, SMG_EINVAL, "gt/Mx/My/Mz must be given");
    if (!p->sigma_t || !p->source) return fail(nullptr, SMG_EINVAL, "sigma_t/source tables must be given");
    if (p->n_fields < 0 || (p->n_fields > 0 && !p->fields)) return fail(nullptr, SMG_EINVAL, "bad field table");
    if (p->filter_mode < 0 || p->filter_mode > 2) return fail(nullptr, SMG_EINVAL, "filter_mode must be 0, 1 or 2");
    if (p->filter_mode != 0 && !p->filter1) return fail(nullptr, SMG_EINVAL, "filter1 table required");
    if (p->filter_mode == 1 && !p->filter2) return fail(nullptr, SMG_EINVAL, "filter2 table required for substep");
    for (int d = 0; d < 3; ++d) {
        if (p->n[d] < 1 || p->n[d] > (1 << 30)) return fail(nullptr, SMG_EINVAL, "n[d] must be in [1, 2^30]");
        if (p->bc[d] != 0 && p->bc[d] != 1) return fail(nullptr, SMG_EINVAL, "bc[d] must be 0 or 1");
        if (!(p->h[d] > 0.0) || !std::isfinite(p->h[d])) return fail(nullptr, SMG_EINVAL, "h[d] must be finite and > 0");
    }
    for (int j = 0; j < ns; ++j)
        for (int d = 0; d < 3; ++d)
            if (p->gt[3 * j + d] != 1 && p->gt[3 * j + d] != 2) return fail(nullptr, SMG_EINVAL, "gt entries must be 1 or 2");
    auto bad_field = [&](int f, bool allow_none) {
        return allow_none ? (f < -1 || f >= p->n_fields) : (f < 0 || f >= p->n_fields);
    };
    for (int f = 0; f < p->n_fields; ++f)
        for (int d = 0; d < 3; ++d)
            if (p->fields[f].grid[d] != 1 && p->fields[f].grid[d] != 2)
                return fail(nullptr, SMG_EINVAL, "field grid types must be 1 or 2");
    if (bad_field(p->sigma_a, false)) return fail(nullptr, SMG_EINVAL, "sigma_a field index out of range");
    if (bad_field(p->decay_a, true)) return fail(nullptr, SMG_EINVAL, "decay_a field index out of range");
    for (int j = 1; j < ns; ++j) {
        if (bad_field(p->sigma_t[j], false)) return fail(nullptr, SMG_EINVAL, "sigma_t field index out of range");
        if (p->decay_t && bad_field(p->decay_t[j], false)) return fail(nullptr, SMG_EINVAL, "decay_t field index out of range");
    }
    for (int j = 0; j < ns; ++j) {
        if (bad_field(p->source[j], true)) return fail(nullptr, SMG_EINVAL, "source field index out of range");
        if (p->filter_mode != 0 && bad_field(p->filter1[j], true)) return fail(nullptr, SMG_EINVAL, "filter1 index out of range");
        if (p->filter_mode == 1 && bad_field(p->filter2[j], true)) return fail(nullptr, SMG_EINVAL, "filter2 index out of range");
    }

    smg_handle* h = new smg_handle();
    h->n_sys = ns;
    // kernel axes: non-singleton solver dimensions first, in solver order
    int gt2[3] = {0, 0, 0};
    for (int j = 0; j < ns; ++j)
        for (int d = 0; d < 3; ++d) gt2[d] |= (p->gt[3 * j + d] == 2);
    bool active[3];
    for (int d = 0; d < 3; ++d) active[d] = p->n[d] > 1 || (p->bc[d] == 1 && gt2[d]);
    int a = 0;
    for (int d = 0; d < 3; ++d) if (active[d]) h->sd[a++] = d;
    for (int d = 0; d < 3; ++d) if (!active[d]) h->sd[a++] = d;
    int axis_of[3];
    for (int k = 0; k < 3; ++k) axis_of[h->sd[k]] = k;
    for (int k = 0; k < 3; ++k) {
        const int d = h->sd[k];
        h->g.n[k] = p->n[d];
        h->g.bc[k] = p->bc[d];
        h->g.h[k] = p->h[d];
        h->g.B[k] = p->n[d] + ((p->bc[d] == 1 && gt2[d]) ? 1 : 0);
    }
    // the kernels index a point inside one component with 32-bit integers
    if (std::ceil(h->g.B[0] / 8.0) * 8.0 * h->g.B[1] * h->g.B[2] + 31.0 >= 2147483648.0) {
        delete h;
        return fail(nullptr, SMG_EINVAL, "grid too large: one component must hold fewer than 2^31 padded points");
    }
    h->g.s1 = ((long long)h->g.B[0] + 7) / 8 * 8;
    h->g.s2 = h->g.s1 * h->g.B[1];
    h->g.cs = (h->g.s2 * h->g.B[2] + 31) / 32 * 32;
    // CTA size of the generated kernels (two points per thread): of 64 and 96
    // threads the one that covers a row with the fewest idle points, 96 on
    // ties (fewer CTAs per row; 350-point rows: 96, measured 1-2% faster than
    // 64; 128 threads measured slower there)
    {
        long long best_idle = -1;
        for (int blk : {64, 96}) {
            const long long per = 2LL * blk, idle = (h->g.B[0] + per - 1) / per * per - h->g.B[0];
            if (best_idle < 0 || idle <= best_idle) {
                best_idle = idle;
                h->jit_block = blk;
            }
        }
    }

    // components and couplings in sumcell order.  The nonzeros of every row
    // are collected in one pass over each column-major matrix in memory order
    // (column i outer, so each row's list ascends in i); a row-by-row scan
    // strides by n_sys doubles and costs milliseconds for hundreds of moments.
    h->comps.resize(ns);
    const double* M[3] = {p->Mx, p->My, p->Mz};
    std::vector<std::vector<std::pair<int, double>>> rownz[3];
    for (int d = 0; d < 3; ++d) {
        rownz[d].resize(ns);
        for (int i = 0; i < ns; ++i) {
            const double* col = M[d] + (size_t)i * ns;
            for (int j = 0; j < ns; ++j)
                if (col[j] != 0.0) rownz[d][j].push_back({i, col[j]});
        }
    }
    for (int j = 0; j < ns; ++j) {
        DevComp& c = h->comps[j];
        grid_extents(h, &p->gt[3 * j], c.ext);
        c.cbeg = (int)h->coups.size();
        for (int d = 0; d < 3; ++d) {
            for (const auto& iw : rownz[d][j]) {
                const int i = iw.first;
                const double w = iw.second;
                const int gi = p->gt[3 * i + d];
                // the staggered difference of component i along d lives on the
                // grid of i with axis d flipped; MATLAB adds it elementwise to
                // W_j, so the extents must agree (else the reference errors).
                int eD[3];
                int gflip[3] = {p->gt[3 * i], p->gt[3 * i + 1], p->gt[3 * i + 2]};
                gflip[d] = 3 - gi;
                if (gflip[0] != p->gt[3 * j] || gflip[1] != p->gt[3 * j + 1] || gflip[2] != p->gt[3 * j + 2]) {
                    delete h;
                    char buf[160];
                    std::snprintf(buf, sizeof buf, "gt: coupling M%c(%d,%d) needs grids that differ in axis %c alone",
                                  "xyz"[d], j + 1, i + 1, "xyz"[d]);
                    return fail(nullptr, SMG_EINVAL, buf);
                }
                grid_extents(h, gflip, eD);
                if (eD[0] != c.ext[0] || eD[1] != c.ext[1] || eD[2] != c.ext[2]) {
                    delete h;
                    char buf[160];
                    std::snprintf(buf, sizeof buf, "coupling M%c(%d,%d) joins grids of different extents", "xyz"[d], j + 1, i + 1);
                    return fail(nullptr, SMG_EINVAL, buf);
                }
                h->coups.push_back(DevCoup{i, axis_of[d] * 2 + (gi == 2 ? 1 : 0), w});
            }
        }
        c.cend = (int)h->coups.size();
        int ntwo = (p->gt[3 * j] == 2) + (p->gt[3 * j + 1] == 2) + (p->gt[3 * j + 2] == 2);
        c.order = 0;
        (ntwo % 2 ? h->destA : h->destB).push_back(j);
    }
    if (h->destB.empty() || h->destB[0] != 0) {
        delete h;
        return fail(nullptr, SMG_EINVAL, "component 1 must lie on grid (1,1,1)");
    }

    // field table: user fields, then constants ONE and ZERO, then device-derived decays
    const int nf = p->n_fields;
    h->field_one = nf;
    h->field_zero = nf + 1;
    int nfields = nf + 2;
    h->derived_decay.assign(nf, -1);
    h->sigma_t_field.assign(ns, -1);
    h->decay_t_field.assign(ns, -1);
    h->sigma_a = p->sigma_a;
    h->decay_a = p->decay_a;
    h->filter_mode = p->filter_mode;
    auto need_derived = [&](int sf) {
        if (h->derived_decay[sf] < 0) h->derived_decay[sf] = nfields++;
        return h->derived_decay[sf];
    };
    for (int j = 1; j < ns; ++j) {
        h->sigma_t_field[j] = p->sigma_t[j];
        h->decay_t_field[j] = p->decay_t ? p->decay_t[j] : need_derived(p->sigma_t[j]);
    }
    if (p->decay_a < 0) h->derived_decay_a = need_derived(p->sigma_a);
    h->fields_host.assign(nfields, DevField{nullptr, 0.0});
    h->field_grid.assign(nfields, 0);
    // slots for array fields
    std::vector<int> slot(nfields, -1);
    int nslots = 0;
    h->field_is_array.assign(nf, 0);
    for (int f = 0; f < nf; ++f) {
        h->field_is_array[f] = p->fields[f].data != nullptr;
        h->field_grid[f] = (p->fields[f].grid[0] - 1) | ((p->fields[f].grid[1] - 1) << 1) | ((p->fields[f].grid[2] - 1) << 2);
        if (p->fields[f].data) slot[f] = nslots++;
        h->fields_host[f].s = p->fields[f].scalar;
    }
    h->fields_host[h->field_one].s = 1.0;
    h->fields_host[h->field_zero].s = 0.0;
    for (int f = 0; f < nf; ++f) {
        const int df = h->derived_decay[f];
        if (df >= 0) {
            h->field_grid[df] = h->field_grid[f];
            if (p->fields[f].data) slot[df] = nslots++;
        }
    }
    h->nslots = nslots;
    for (int j = 0; j < ns; ++j) {
        DevComp& c = h->comps[j];
        c.sT = j ? h->sigma_t_field[j] : h->field_zero;
        c.ET = j ? h->decay_t_field[j] : h->field_one;
        c.Q = p->source[j] >= 0 ? p->source[j] : h->field_zero;
        c.F1 = (p->filter_mode != 0 && p->filter1[j] >= 0) ? p->filter1[j] : h->field_one;
        c.F2 = (p->filter_mode == 1 && p->filter2[j] >= 0) ? p->filter2[j] : h->field_one;
    }

    if (!device) {
        const std::vector<int> level = coupling_levels(h);
        reciprocals(h);
        for (int ph = 0; ph < 2; ++ph) build_pair(h, ph, level);
        *out = h;
        return SMG_OK;
    }
    // device allocations
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess) {
        int r = cuda_fail(nullptr, e, "cudaStreamCreate");
        delete h;
        return r;
    }
    auto alloc = [&](void** ptr, size_t bytes) -> cudaError_t {
        if (bytes == 0) bytes = 16;
        cudaError_t r = cudaMalloc(ptr, bytes);
        if (r == cudaSuccess) h->bytes += bytes;
        return r;
    };
    const size_t slot_bytes = (size_t)h->g.cs * 8;
    h->stage_bytes = std::min<size_t>(kStageBytes, slot_bytes * ns);
    if ((e = alloc((void**)&h->dU, slot_bytes * ns)) != cudaSuccess ||
        (e = alloc((void**)&h->dStage, h->stage_bytes)) != cudaSuccess ||
        (e = alloc((void**)&h->dFields, slot_bytes * (size_t)std::max(nslots, 1))) != cudaSuccess ||
        (e = alloc((void**)&h->dComps, sizeof(DevComp) * ns)) != cudaSuccess ||
        (e = alloc((void**)&h->dCoups, sizeof(DevCoup) * std::max<size_t>(h->coups.size(), 1))) != cudaSuccess ||
        (e = alloc((void**)&h->dFieldTab, sizeof(DevField) * nfields)) != cudaSuccess ||
        (e = alloc((void**)&h->dDest, sizeof(int) * ns)) != cudaSuccess ||
        (e = alloc((void**)&h->dFlag, sizeof(int))) != cudaSuccess ||
        (e = alloc((void**)&h->dSumsq, sizeof(double) * (size_t)ns * (smg::kSumsqBlocks + 1))) != cudaSuccess) {
        int r = cuda_fail(nullptr, e, "cudaMalloc");
        free_device(h);
        delete h;
        return r;
    }
    for (int f = 0; f < nfields; ++f)
        if (slot[f] >= 0) h->fields_host[f].p = h->dFields + (size_t)slot[f] * h->g.cs;
    std::vector<int> dest(h->destA);
    dest.insert(dest.end(), h->destB.begin(), h->destB.end());
#define CREATE_CUDA(expr)                                   \
    do {                                                    \
        cudaError_t e_ = (expr);                            \
        if (e_ != cudaSuccess) {                            \
            int r_ = cuda_fail(nullptr, e_, #expr);         \
            free_device(h);                                 \
            delete h;                                       \
            return r_;                                      \
        }                                                   \
    } while (0)
    CREATE_CUDA(cudaMemsetAsync(h->dU, 0, slot_bytes * ns, h->stream));
    CREATE_CUDA(cudaMemsetAsync(h->dFields, 0, slot_bytes * (size_t)std::max(nslots, 1), h->stream));
    CREATE_CUDA(cudaMemcpyAsync(h->dComps, h->comps.data(), sizeof(DevComp) * ns, cudaMemcpyHostToDevice, h->stream));
    if (!h->coups.empty())
        CREATE_CUDA(cudaMemcpyAsync(h->dCoups, h->coups.data(), sizeof(DevCoup) * h->coups.size(), cudaMemcpyHostToDevice, h->stream));
    CREATE_CUDA(cudaMemcpyAsync(h->dDest, dest.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, h->stream));
    for (int f = 0; f < nf; ++f) {
        if (!p->fields[f].data) continue;
        int e3[3];
        grid_extents(h, p->fields[f].grid, e3);
        CREATE_CUDA(put_slot(h, const_cast<double*>(h->fields_host[f].p), p->fields[f].data, e3));
    }
    CREATE_CUDA(cudaMemcpyAsync(h->dFieldTab, h->fields_host.data(), sizeof(DevField) * nfields, cudaMemcpyHostToDevice, h->stream));
    // strip-kernel schedules: stage = breadth-first level of the coupling graph
    {
        const std::vector<int> level = coupling_levels(h);
        build_schedule(h, 0, level);
        build_schedule(h, 1, level);
        for (int ph = 0; ph < 2; ++ph) {
            auto& S = h->sched[ph];
            resolve_coefs(h, ph);
            S.ok = S.ok && (int)S.frows.size() <= smg::kMaxFieldRows &&
                   (S.nslots * 32 + S.jcap * 64 + (int)S.frows.size() * 32) * 8 <= smg::kMaxStripSmem;
        }
        reciprocals(h);
        h->nxs = (h->g.B[0] + 31) / 32;
        CREATE_CUDA(upload_schedule(h, 0));
        CREATE_CUDA(upload_schedule(h, 1));
        for (int ph = 0; ph < 2; ++ph) {
            build_pair(h, ph, level);
            resolve_pair(h, ph);
            CREATE_CUDA(upload_pair(h, ph, true));
        }
        if (h->sched[0].ok && h->sched[1].ok) CREATE_CUDA(smg::strip_init(h));
    }
    CREATE_CUDA(cudaEventCreate(&h->ev0));
    CREATE_CUDA(cudaEventCreate(&h->ev1));
    CREATE_CUDA(cudaStreamSynchronize(h->stream));
#undef CREATE_CUDA
    *out = h;
    return SMG_OK;
}

}  // namespace

extern "C" {

void smg_destroy(smg_handle* h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_device(h);
    delete h;
}

int smg_set_state(smg_handle* h, const double* const* U) {
    SMG_TRY
    if (!h || !U) return fail(h, SMG_EINVAL, "smg_set_state: NULL argument");
    for (int j = 0; j < h->n_sys; ++j)
        if (!U[j]) return fail(h, SMG_EINVAL, "smg_set_state: NULL component pointer");
    const int rc = staged_transfer(h, true, U, nullptr, nullptr, 0.0, 0.0);
    if (rc != SMG_OK) return rc;
    h->state_set = true;
    return SMG_OK;
    SMG_CATCH(h ? &h->err : nullptr)
}

int smg_get_state(smg_handle* h, double* const* U) {
    SMG_TRY
    if (!h || !U) return fail(h, SMG_EINVAL, "smg_get_state: NULL argument");
    const int rc = staged_transfer(h, false, nullptr, U, nullptr, 0.0, 0.0);
    if (rc == SMG_OK && smg::jit_status(h) == SMG_ETIMEOUT)
        return fail(h, SMG_ETIMEOUT,
                    "smg_get_state: a staged kernel's shared-memory pipeline wait ran out (state undefined)");
    return rc;
    SMG_CATCH(h ? &h->err : nullptr)
}

int smg_snapshot(smg_handle* h) {
    SMG_TRY
    if (!h) return fail(h, SMG_EINVAL, "smg_snapshot: NULL handle");
    if (!h->state_set) return fail(h, SMG_ESTATE, "smg_snapshot: smg_set_state has not been called");
    const size_t bytes = (size_t)h->g.cs * h->n_sys * sizeof(double);
    if (!h->dSnap) {
        SMG_CUDA(h, cudaMalloc(&h->dSnap, bytes));
        h->bytes += bytes;
    }
    SMG_CUDA(h, cudaMemcpyAsync(h->dSnap, h->dU, bytes, cudaMemcpyDeviceToDevice, h->stream));
    h->snap_set = true;
    return SMG_OK;
    SMG_CATCH(h ? &h->err : nullptr)
}

int smg_get_interp(smg_handle* h, double lambda, double* const* U) {
    SMG_TRY
    if (!h || !U) return fail(h, SMG_EINVAL, "smg_get_interp: NULL argument");
    if (!h->snap_set) return fail(h, SMG_ESTATE, "smg_get_interp: smg_snapshot has not been called");
    if (!std::isfinite(lambda)) return fail(h, SMG_EINVAL, "smg_get_interp: lambda must be finite");
    return staged_transfer(h, false, nullptr, U, h->dSnap, 1.0 - lambda, lambda);
    SMG_CATCH(h ? &h->err : nullptr)
}

int smg_set_field(smg_handle* h, int32_t f, const double* data, double scalar) {
    SMG_TRY
    if (!h) return fail(h, SMG_EINVAL, "smg_set_field: NULL handle");
    if (f < 0 || f >= h->field_one) return fail(h, SMG_EINVAL, "smg_set_field: field index out of range");
    DevField& F = h->fields_host[f];
    if ((F.p == nullptr) != (data == nullptr))
        return fail(h, SMG_EINVAL, "smg_set_field: a field cannot change between scalar and array");
    if (data) {
        int gts[3] = {1 + (h->field_grid[f] & 1), 1 + ((h->field_grid[f] >> 1) & 1), 1 + ((h->field_grid[f] >> 2) & 1)};
        int e3[3];
        grid_extents(h, gts, e3);
        SMG_CUDA(h, put_slot(h, const_cast<double*>(F.p), data, e3));
    } else {
        F.s = scalar;
        SMG_CUDA(h, cudaMemcpyAsync(h->dFieldTab + f, &F, sizeof(DevField), cudaMemcpyHostToDevice, h->stream));
        SMG_CUDA(h, refresh_coefs(h));
    }
    SMG_CUDA(h, cudaStreamSynchronize(h->stream));
    if (h->dt_set) return smg_set_dt(h, h->dt);   // refresh derived decays
    return SMG_OK;
    SMG_CATCH(h ? &h->err : nullptr)
}

int smg_set_time(smg_handle* h, double t) {
    SMG_TRY
    if (!h) return fail(h, SMG_EINVAL, "smg_set_time: NULL handle");
    if (!std::isfinite(t)) return fail(h, SMG_EINVAL, "smg_set_time: t must be finite");
    h->t = t;
    h->mat.init = false;   // materials re-evaluated at t before the next step
    return SMG_OK;
    SMG_CATCH(h ? &h->err : nullptr)
}

// The coordinate table of the material and filter expressions: per solver
// dimension d the coordinates of grid types 1 and 2 (coords[2d], coords[2d+1]).
static int set_coords(smg_handle* h, const double* const* coords, const char* who) {
    std::vector<double> c;
    smg_handle::Coords X;
    for (int d = 0; d < 3; ++d) {
        int a = 0;
        while (h->sd[a] != d) ++a;
        for (int gt = 1; gt <= 2; ++gt) {
            if (!coords[2 * d + gt - 1]) return fail(h, SMG_EINVAL, std::string(who) + ": NULL coordinate vector");
            const int len = (gt == 2 && h->g.bc[a] == 1) ? h->g.n[a] + 1 : h->g.n[a];
            X.off[d][gt - 1] = (int)c.size();
            c.insert(c.end(), coords[2 * d + gt - 1], coords[2 * d + gt - 1] + len);
        }
    }
    SMG_CUDA(h, cudaMalloc(&X.dC, c.size() * sizeof(double)));
    const cudaError_t e = cudaMemcpy(X.dC, c.data(), c.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(X.dC);
        return cuda_fail(h, e, (std::string(who) + ": coordinates").c_str());
    }
    cudaFree(h->xyz.dC);
    h->xyz = X;
    return SMG_OK;
}

static bool array_field(const smg_handle* h, int f) {
    return f >= 0 && f < (int)h->fields_host.size() && h->fields_host[f].p;
}

int smg_set_material_expr(smg_handle* h, const char* expr_a, const char* expr_s0, const char* expr_sm, int32_t nrows,
                          const int32_t* rows, int32_t sA_field, int32_t EA_field, const double* const* coords) {
    SMG_TRY
    if (!h) return fail(h, SMG_EINVAL, "smg_set_material_expr: NULL handle");
    smg::src_free(h, false);
    cudaFree(h->mat.dOld);
    h->mat = smg_handle::MatExpr{};
    if (!expr_a) return SMG_OK;   // back to uploaded values
    if (!expr_s0 || nrows < 0 || (nrows > 0 && !rows) || !coords)
        return fail(h, SMG_EINVAL, "smg_set_material_expr: NULL argument");
    for (const char* e : {expr_a, expr_s0, expr_sm}) {
        if (!e) continue;
        const std::string why = expr_problem(e, SMG_EXPR_MATERIAL);
        if (!why.empty()) return fail(h, SMG_EINVAL, "smg_set_material_expr: " + why);
    }
    smg_handle::MatExpr M;
    for (int r = 0; r < nrows; ++r) {
        if (!array_field(h, rows[3 * r]) || !array_field(h, rows[3 * r + 1]))
            return fail(h, SMG_EINVAL, "smg_set_material_expr: sigma_t and decay fields must be array fields");
        M.sT.push_back(rows[3 * r]);
        M.ET.push_back(rows[3 * r + 1]);
        M.m.push_back(rows[3 * r + 2]);
    }
    if (!array_field(h, sA_field) || !array_field(h, EA_field))
        return fail(h, SMG_EINVAL, "smg_set_material_expr: sigma_a and its decay field must be array fields");
    M.sA = sA_field;
    M.EA = EA_field;
    M.a = expr_a;
    M.s0 = expr_s0;
    M.sm = expr_sm ? expr_sm : "";
    const int rc = set_coords(h, coords, "smg_set_material_expr");
    if (rc != SMG_OK) return rc;
    SMG_CUDA(h, cudaMalloc(&M.dOld, (size_t)(nrows + 1) * h->g.cs * sizeof(double)));
    M.on = true;
    M.init = false;
    h->mat = M;
    return SMG_OK;
    SMG_CATCH(h ? &h->err : nullptr)
}

int smg_set_filter_expr(smg_handle* h, const char* expr, int32_t nrows, const int32_t* rows,
                        const double* const* coords) {
    SMG_TRY
    if (!h) return fail(h, SMG_EINVAL, "smg_set_filter_expr: NULL handle");
    smg::src_free(h, false);
    h->filt = smg_handle::FiltExpr{};
    if (!expr) return SMG_OK;   // back to uploaded values
    if (nrows < 1 || !rows || !coords) return fail(h, SMG_EINVAL, "smg_set_filter_expr: NULL argument or no rows");
    {
        const std::string why = expr_problem(expr, SMG_EXPR_FILTER);
        if (!why.empty()) return fail(h, SMG_EINVAL, "smg_set_filter_expr: " + why);
    }
    smg_handle::FiltExpr F;
    F.expr = expr;
    for (int r = 0; r < nrows; ++r) {
        const int f1 = rows[3 * r], f2 = rows[3 * r + 1];
        if (!array_field(h, f1) || (f2 >= 0 && !array_field(h, f2)))
            return fail(h, SMG_EINVAL, "smg_set_filter_expr: filter fields must be array fields");
        if (f2 >= 0 && h->field_grid[f2] != h->field_grid[f1])
            return fail(h, SMG_EINVAL, "smg_set_filter_expr: a row's two fields must share a grid");
        F.f1.push_back(f1);
        F.f2.push_back(f2);
        F.k.push_back(rows[3 * r + 2]);
    }
    const int rc = set_coords(h, coords, "smg_set_filter_expr");
    if (rc != SMG_OK) return rc;
    h->filt = F;
    return SMG_OK;
    SMG_CATCH(h ? &h->err : nullptr)
}

int smg_set_source_expr(smg_handle* h, int32_t comp, const char* expr, const double* x, const double* y,
                        const double* z) {
    SMG_TRY
    if (!h) return fail(h, SMG_EINVAL, "smg_set_source_expr: NULL handle");
    if (comp < 0 || comp >= h->n_sys) return fail(h, SMG_EINVAL, "smg_set_source_expr: component out of range");
    const int f = h->comps[comp].Q;
    size_t at = 0;
    while (at < h->src_expr.size() && h->src_expr[at].comp != comp) ++at;
    smg::src_free(h, false);   // the kernels are rebuilt at the next smg_run
    if (!expr) {   // back to the field's uploaded values
        if (at < h->src_expr.size()) {
            cudaFree(h->src_expr[at].dC);
            h->src_expr.erase(h->src_expr.begin() + at);
        }
        return SMG_OK;
    }
    if (f < 0 || f >= (int)h->fields_host.size() || !h->fields_host[f].p)
        return fail(h, SMG_EINVAL, "smg_set_source_expr: the component's source must be an array field");
    for (int j = 0; j < h->n_sys; ++j)
        if (j != comp && h->comps[j].Q == f)
            return fail(h, SMG_EINVAL, "smg_set_source_expr: the source field is shared with another component");
    if (!x || !y || !z) return fail(h, SMG_EINVAL, "smg_set_source_expr: NULL coordinate vector");
    {
        const std::string why = expr_problem(expr, SMG_EXPR_SOURCE);
        if (!why.empty()) return fail(h, SMG_EINVAL, "smg_set_source_expr: " + why);
    }
    // coordinates of the component's grid per kernel axis, from the
    // per-solver-dimension vectors
    const int* E = h->comps[comp].ext;
    const double* solver[3] = {x, y, z};
    std::vector<double> c;
    for (int a = 0; a < 3; ++a) c.insert(c.end(), solver[h->sd[a]], solver[h->sd[a]] + E[a]);
    double* d = nullptr;
    SMG_CUDA(h, cudaMalloc(&d, c.size() * sizeof(double)));
    cudaError_t e = cudaMemcpy(d, c.data(), c.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(d);
        return cuda_fail(h, e, "smg_set_source_expr: coordinates");
    }
    if (at == h->src_expr.size()) h->src_expr.emplace_back();
    else cudaFree(h->src_expr[at].dC);
    h->src_expr[at].comp = comp;
    h->src_expr[at].expr = expr;
    h->src_expr[at].dC = d;
    return SMG_OK;
    SMG_CATCH(h ? &h->err : nullptr)
}

int smg_set_dt(smg_handle* h, double dt) {
    SMG_TRY
    if (!h) return fail(h, SMG_EINVAL, "smg_set_dt: NULL handle");
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(h, SMG_EINVAL, "smg_set_dt: dt must be finite and > 0");
    h->dt = dt;
    h->hdt = dt / 2;
    for (int f = 0; f < (int)h->derived_decay.size(); ++f) {
        const int df = h->derived_decay[f];
        if (df < 0) continue;
        DevField& S = h->fields_host[f];
        DevField& D = h->fields_host[df];
        if (S.p) {
            SMG_CUDA(h, smg::launch_decay(const_cast<double*>(D.p), S.p, h->g.cs, dt, h->stream));
        } else {
            D.s = expm1div_host(-S.s * dt / 2);
        }
    }
    SMG_CUDA(h, cudaMemcpyAsync(h->dFieldTab, h->fields_host.data(), sizeof(DevField) * h->fields_host.size(),
                                cudaMemcpyHostToDevice, h->stream));
    SMG_CUDA(h, refresh_coefs(h));
    SMG_CUDA(h, cudaStreamSynchronize(h->stream));
    if (h->graph) {   // kernel arguments (dt/2) are baked into the graph
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
        h->graph_steps = 0;
    }
    h->dt_set = true;
    return SMG_OK;
    SMG_CATCH(h ? &h->err : nullptr)
}

// Enqueue `nsteps` Strang steps; *launches receives the kernel count.
// With the strip kernels and no full filter, phase A at the end of a step and
// phase A at the start of the next are one launch (same sources, the inner
// set does not change between them): A(k1) B [AA B]... A(k2).
static cudaError_t enqueue_steps(smg_handle* h, int64_t nsteps, cudaStream_t s, int64_t* launches) {
    cudaError_t e;
    int64_t L = 0;
    // AUTO runs the pair kernel when its tables exist (measured fastest on the
    // 820-moment lattice workload), else the strip kernel, else the generic one
    const bool jit = h->jit && (h->variant == SMG_VARIANT_JIT || h->variant == SMG_VARIANT_AUTO);
    const bool pair = !jit && (h->variant == SMG_VARIANT_PAIR || h->variant == SMG_VARIANT_AUTO) && h->pair[0].ok &&
                      h->pair[1].ok;
    const bool strip = !jit && !pair && strip_usable(h);
    const bool fuse = ((strip && (h->variant == SMG_VARIANT_AUTO || h->variant == SMG_VARIANT_STAGED)) || pair || jit) &&
                      h->filter_mode != SMG_FILTER_FULL;
    const bool hasA = !h->destA.empty();
    // one phase; L counts its kernels (the generated code may use several)
    auto ph = [&](int mode, int kf) {
        if (jit) {
            L += smg::jit_launches(h, mode == 1 ? 1 : 0);
            return smg::launch_jit(h, mode, kf, s);
        }
        ++L;
        return pair ? smg::launch_pair(h, mode, kf, s) : smg::launch_strip(h, mode, kf, s);
    };
    if (fuse && nsteps >= 1) {
        if (hasA) { if ((e = ph(0, 1)) != cudaSuccess) return e; }
        for (int64_t k = 0; k < nsteps; ++k) {
            if ((e = ph(1, 0)) != cudaSuccess) return e;
            if (!hasA) continue;
            if (k + 1 < nsteps) e = ph(2, 0);
            else e = ph(0, 2);
            if (e != cudaSuccess) return e;
        }
        if (launches) *launches = L;
        return cudaSuccess;
    }
    for (int64_t k = 0; k < nsteps; ++k) {
        if (jit) {
            if (hasA) { if ((e = ph(0, 1)) != cudaSuccess) return e; }
            if ((e = ph(1, 0)) != cudaSuccess) return e;
            if (hasA) { if ((e = ph(0, 2)) != cudaSuccess) return e; }
        } else if (strip) {
            if (hasA) { if ((e = smg::launch_strip(h, 0, 1, s)) != cudaSuccess) return e; ++L; }
            if ((e = smg::launch_strip(h, 1, 0, s)) != cudaSuccess) return e;
            ++L;
            if (hasA) { if ((e = smg::launch_strip(h, 0, 2, s)) != cudaSuccess) return e; ++L; }
        } else {
            if (hasA) { if ((e = smg::launch_phase(h, 0, 1, s)) != cudaSuccess) return e; ++L; }
            if ((e = smg::launch_phase(h, 1, 0, s)) != cudaSuccess) return e;
            ++L;
            if (hasA) { if ((e = smg::launch_phase(h, 0, 2, s)) != cudaSuccess) return e; ++L; }
        }
        if (h->filter_mode == SMG_FILTER_FULL && h->n_sys > 1) {
            if ((e = smg::launch_full_filter(h, s)) != cudaSuccess) return e;
            ++L;
        }
    }
    if (launches) *launches = L;
    return cudaSuccess;
}

int smg_run(smg_handle* h, int64_t nsteps) {
    SMG_TRY
    if (!h) return fail(h, SMG_EINVAL, "smg_run: NULL handle");
    if (nsteps < 0) return fail(h, SMG_EINVAL, "smg_run: nsteps must be >= 0");
    if (!h->dt_set) return fail(h, SMG_ESTATE, "smg_run: smg_set_dt has not been called");
    if (!h->state_set) return fail(h, SMG_ESTATE, "smg_run: smg_set_state has not been called");
    return smg::run_steps(h, nsteps, true);
    SMG_CATCH(h ? &h->err : nullptr)
}

}  // extern "C"

// nsteps steps on the handle's stream; with `events`, bracketed by the
// handle's timing events (smg_last_run_stats)
int smg::run_steps(smg_handle* h, int64_t nsteps, bool events) {
    // steps per captured graph (0: none).  By default a step that moves a
    // gigabyte or more (about 24 bytes per moment-cell update) runs as
    // direct launches: the host enqueues a step far faster than the GPU runs
    // it, and a fresh handle then pays no graph capture; lighter steps are
    // replayed from 64-step graphs
    int64_t kBlock = h->graph_block;
    if (kBlock < 0) {
        const double step_bytes = 24.0 * (double)h->g.B[0] * h->g.B[1] * h->g.B[2] * h->n_sys;
        kBlock = step_bytes >= 1e9 ? 0 : 64;
    }
    if (h->variant == SMG_VARIANT_AUTO && !h->jit && !h->jit_failed && nsteps > 0) {
        // first run: generate and compile the specialised kernels; without
        // NVRTC (or for tables beyond 32-bit offsets) AUTO keeps the pair kernel
        std::string why;
        if (smg::jit_build(h, why) != SMG_OK) {
            h->jit_failed = true;
            h->jit_err = why;
        } else if (h->graph) {
            cudaGraphExecDestroy(h->graph);
            h->graph = nullptr;
            h->graph_steps = 0;
        }
    }
    int64_t left = nsteps;
    int64_t launches = 0, rem = 0;
    if (!h->src_expr.empty() || h->mat.on || !h->filt.f1.empty()) {
        // sources and materials evaluated on the device: before every step
        // the materials at t + dt averaged with those at t (and their decay
        // factors), Q at t + dt/2 (starmap_solver.m:214-282), then one
        // unfused step (the two phase-A passes around a step boundary see
        // different coefficients); the time advances as the host loop does
        if ((!h->src_expr.empty() && !h->src_expr[0].fn) || (h->mat.on && h->mat.fn.empty()) ||
            (!h->filt.f1.empty() && h->filt.fn.empty())) {
            std::string why;
            const int rc = smg::src_build(h, why);
            if (rc != SMG_OK) return fail(h, rc, "source and material expressions: " + why);
        }
        if (h->mat.on && !h->mat.init) SMG_CUDA(h, smg::launch_mat(h, h->t, h->dt, true, h->stream));
        if (events) SMG_CUDA(h, cudaEventRecord(h->ev0, h->stream));
        for (int64_t k = 0; k < nsteps; ++k) {
            const double t_end = h->t + h->dt;
            if (h->mat.on) {
                SMG_CUDA(h, smg::launch_mat(h, t_end, h->dt, false, h->stream));
                launches += (int64_t)h->mat.sT.size() + 1;
            }
            SMG_CUDA(h, smg::launch_src(h, t_end - h->dt / 2, h->stream));
            SMG_CUDA(h, smg::launch_filt(h, t_end, h->dt, h->stream));
            launches += (int64_t)h->filt.f1.size();
            SMG_CUDA(h, enqueue_steps(h, 1, h->stream, &rem));
            launches += rem + (int64_t)h->src_expr.size();
            h->t = t_end;
        }
        if (events) SMG_CUDA(h, cudaEventRecord(h->ev1, h->stream));
        h->last_launches = events ? launches : h->last_launches + launches;
        return SMG_OK;
    }
    if (events) SMG_CUDA(h, cudaEventRecord(h->ev0, h->stream));
    if (kBlock > 0 && left >= kBlock && (!h->graph || h->graph_steps != kBlock)) {
        // the first block goes to the stream as direct launches, so that the
        // GPU runs it while the graph for the following blocks is captured
        SMG_CUDA(h, enqueue_steps(h, kBlock, h->stream, &rem));
        launches += rem;
        left -= kBlock;
    }
    if (kBlock > 0 && left >= kBlock) {
        if (!h->graph || h->graph_steps != kBlock) {
            if (h->graph) cudaGraphExecDestroy(h->graph);
            h->graph = nullptr;
            cudaGraph_t gr;
            SMG_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t e = enqueue_steps(h, kBlock, h->stream, &h->graph_launches);
            cudaError_t e2 = cudaStreamEndCapture(h->stream, &gr);
            if (e != cudaSuccess) return cuda_fail(h, e, "capture step block");
            if (e2 != cudaSuccess) return cuda_fail(h, e2, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&h->graph, gr, 0);
            cudaGraphDestroy(gr);
            if (e != cudaSuccess) return cuda_fail(h, e, "cudaGraphInstantiate");
            h->graph_steps = kBlock;
        }
    }
    for (; kBlock > 0 && left >= kBlock; left -= kBlock) {
        SMG_CUDA(h, cudaGraphLaunch(h->graph, h->stream));
        launches += h->graph_launches;
    }
    SMG_CUDA(h, enqueue_steps(h, left, h->stream, &rem));
    if (events) SMG_CUDA(h, cudaEventRecord(h->ev1, h->stream));
    h->last_launches = events ? launches + rem : h->last_launches + launches + rem;
    return SMG_OK;
}

extern "C" {

int smg_tune(smg_handle* h, int32_t key, int32_t value) {
    SMG_TRY
    if (!h) return fail(h, SMG_EINVAL, "smg_tune: NULL handle");
    switch (key) {
        case SMG_TUNE_PAIR_GROUP:
            if (value < 1 || value > 256) return fail(h, SMG_EINVAL, "smg_tune: group must be 1..256");
            h->pair_group = value;
            break;
        case SMG_TUNE_PAIR_BLOCK:
            if (value < 32 || value > 256 || value % 32) return fail(h, SMG_EINVAL, "smg_tune: block must be 32..256, x32");
            h->pair_block = value;
            break;
        case SMG_TUNE_PAIR_UNROLL:
            if (value != 1 && value != 2) return fail(h, SMG_EINVAL, "smg_tune: unroll must be 1 or 2");
            h->pair_unroll = value;
            break;
        case SMG_TUNE_PAIR_MINB:
            if (value != 3 && value != 4) return fail(h, SMG_EINVAL, "smg_tune: minb must be 3 or 4");
            h->pair_minb = value;
            break;
        case SMG_TUNE_JIT_BLOCK:
            if (value < 32 || value > 256 || value % 32) return fail(h, SMG_EINVAL, "smg_tune: jit block must be 32..256, x32");
            h->jit_block = value;
            smg::jit_free(h);
            h->jit_failed = false;
            break;
        case SMG_TUNE_JIT_GROUP:
            if (value < 1 || value > 256) return fail(h, SMG_EINVAL, "smg_tune: jit group must be 1..256");
            h->jit_group = value;
            smg::jit_free(h);
            h->jit_failed = false;
            break;
        case SMG_TUNE_JIT_REGS:
            if (value != 0 && (value < 32 || value > 255)) return fail(h, SMG_EINVAL, "smg_tune: jit regs must be 0 or 32..255");
            h->jit_regs = value;
            smg::jit_free(h);
            h->jit_failed = false;
            break;
        case SMG_TUNE_JIT_SPLIT:
            if (value < 0 || value > 64) return fail(h, SMG_EINVAL, "smg_tune: jit split must be 0..64");
            h->jit_split = value;
            smg::jit_free(h);
            h->jit_failed = false;
            break;
        case SMG_TUNE_JIT_CALLS:
            if (value != 0 && value != 1) return fail(h, SMG_EINVAL, "smg_tune: jit calls must be 0 or 1");
            h->jit_calls = value;
            smg::jit_free(h);
            h->jit_failed = false;
            break;
        case SMG_TUNE_JIT_XPAIR:
            if (value < 0 || value > 2) return fail(h, SMG_EINVAL, "smg_tune: jit xpair must be 0, 1 or 2");
            h->jit_xpair = value;
            smg::jit_free(h);
            h->jit_failed = false;
            break;
        case SMG_TUNE_JIT_PREFETCH:
            if (value < 0 || value > 3) return fail(h, SMG_EINVAL, "smg_tune: jit prefetch must be 0..3");
            h->jit_prefetch = value;
            smg::jit_free(h);
            h->jit_failed = false;
            break;
        case SMG_TUNE_JIT_CONST:
            if (value != 0 && value != 1) return fail(h, SMG_EINVAL, "smg_tune: jit const must be 0 or 1");
            h->jit_const = value;
            smg::jit_free(h);
            h->jit_failed = false;
            break;
        case SMG_TUNE_JIT_BAND:
            if (value < -1 || value > (1 << 20)) return fail(h, SMG_EINVAL, "smg_tune: jit band must be -1..2^20");
            h->jit_band = value;
            smg::jit_free(h);
            h->jit_failed = false;
            break;
        case SMG_TUNE_JIT_STAGED:
            if (value < 0 || value > 3) return fail(h, SMG_EINVAL, "smg_tune: jit staged must be 0..3");
            h->jit_staged = value;
            smg::jit_free(h);
            h->jit_failed = false;
            break;
        case SMG_TUNE_JIT_SLICES:
            if (value < 1 || value > 16) return fail(h, SMG_EINVAL, "smg_tune: jit slices must be 1..16");
            h->jit_slices = value;
            smg::jit_free(h);
            h->jit_failed = false;
            break;
        case SMG_TUNE_JIT_STAGES:
            if (value < 2 || value > 6) return fail(h, SMG_EINVAL, "smg_tune: jit stages must be 2..6");
            h->jit_stages = value;
            smg::jit_free(h);
            h->jit_failed = false;
            break;
        case SMG_TUNE_JIT_ROWS:
            if (value < 0 || value > (1 << 30)) return fail(h, SMG_EINVAL, "smg_tune: jit rows must be 0..2^30");
            h->jit_rows = value;
            smg::jit_free(h);
            h->jit_failed = false;
            break;
        case SMG_TUNE_GRAPH_STEPS:
            if (value < -1 || value > 4096) return fail(h, SMG_EINVAL, "smg_tune: graph steps must be -1..4096");
            h->graph_block = value;
            break;
        case SMG_TUNE_JIT_LANES:
            if (value < 0 || value > 64) return fail(h, SMG_EINVAL, "smg_tune: jit lanes must be 0..64");
            h->jit_lanes = value;
            break;
        case SMG_TUNE_DIRECT_XFER:
            if (value != 0 && value != 1) return fail(h, SMG_EINVAL, "smg_tune: direct xfer must be 0 or 1");
            h->direct_xfer = value;
            return SMG_OK;
        case SMG_TUNE_ADJ_PRIORITY:
            if (value < 0 || value > 2) return fail(h, SMG_EINVAL, "smg_tune: adj priority must be 0, 1 or 2");
            h->adj_priority = value;
            return SMG_OK;
        case SMG_TUNE_ADJ_FUSED:
            if (value != 0 && value != 1) return fail(h, SMG_EINVAL, "smg_tune: adj_fused must be 0 or 1");
            h->adj_fused = value;
            return SMG_OK;
        default:
            return fail(h, SMG_EINVAL, "smg_tune: unknown key");
    }
    if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
        h->graph_steps = 0;
    }
    return SMG_OK;
    SMG_CATCH(h ? &h->err : nullptr)
}

int smg_active_variant(smg_handle* h, int32_t* variant, char* why, int64_t cap) {
    SMG_TRY
    if (!h || !variant) return fail(h, SMG_EINVAL, "smg_active_variant: NULL argument");
    int v;
    if (h->jit && (h->variant == SMG_VARIANT_JIT || h->variant == SMG_VARIANT_AUTO)) v = SMG_VARIANT_JIT;
    else if ((h->variant == SMG_VARIANT_PAIR || h->variant == SMG_VARIANT_AUTO) && h->pair[0].ok && h->pair[1].ok)
        v = SMG_VARIANT_PAIR;
    else if (strip_usable(h)) v = h->strip_staged ? SMG_VARIANT_STAGED : SMG_VARIANT_STRIP;
    else v = SMG_VARIANT_GENERIC;
    *variant = v;
    if (why && cap > 0) {
        // with the generated kernels active: their form; otherwise why AUTO could not use them
        const std::string m = v == SMG_VARIANT_JIT
                                  ? std::string(smg::jit_form(h) == 1   ? "bulk-staged"
                                                : smg::jit_form(h) == 2 ? "async-staged"
                                                : smg::jit_form(h) == 3 ? "prefetch-ring"
                                                                        : "register")
                                  : h->jit_err;
        const size_t n = std::min<size_t>((size_t)cap - 1, m.size());
        std::memcpy(why, m.data(), n);
        why[n] = '\0';
    }
    return SMG_OK;
    SMG_CATCH(h ? &h->err : nullptr)
}

int smg_set_variant(smg_handle* h, int32_t variant) {
    SMG_TRY
    if (!h) return fail(h, SMG_EINVAL, "smg_set_variant: NULL handle");
    if (variant < SMG_VARIANT_AUTO || variant > SMG_VARIANT_JIT)
        return fail(h, SMG_EINVAL, "smg_set_variant: unknown variant");
    if (variant == SMG_VARIANT_JIT && !h->jit) {
        std::string why;
        const int rc = smg::jit_build(h, why);
        if (rc != SMG_OK) return fail(h, rc, "smg_set_variant: specialised kernels unavailable: " + why);
    }
    if ((variant == SMG_VARIANT_STRIP || variant == SMG_VARIANT_STAGED) && !(h->sched[0].ok && h->sched[1].ok))
        return fail(h, SMG_EINVAL, "smg_set_variant: strip schedule does not fit in shared memory");
    if (variant == SMG_VARIANT_PAIR && !(h->pair[0].ok && h->pair[1].ok))
        return fail(h, SMG_EINVAL, "smg_set_variant: pair tables unavailable for this problem");
    h->variant = variant;
    h->strip_staged = variant == SMG_VARIANT_STAGED;
    if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
        h->graph_steps = 0;
    }
    return SMG_OK;
    SMG_CATCH(h ? &h->err : nullptr)
}

int smg_sync(smg_handle* h) {
    SMG_TRY
    if (!h) return fail(h, SMG_EINVAL, "smg_sync: NULL handle");
    SMG_CUDA(h, cudaStreamSynchronize(h->stream));
    if (smg::jit_status(h) == SMG_ETIMEOUT)
        return fail(h, SMG_ETIMEOUT, "smg_sync: a staged kernel's shared-memory pipeline wait ran out (state undefined)");
    return SMG_OK;
    SMG_CATCH(h ? &h->err : nullptr)
}

int smg_last_run_stats(smg_handle* h, double* ms, int64_t* launches) {
    SMG_TRY
    if (!h) return fail(h, SMG_EINVAL, "smg_last_run_stats: NULL handle");
    SMG_CUDA(h, cudaEventSynchronize(h->ev1));
    float f = 0.f;
    SMG_CUDA(h, cudaEventElapsedTime(&f, h->ev0, h->ev1));
    if (ms) *ms = f;
    if (launches) *launches = h->last_launches;
    return SMG_OK;
    SMG_CATCH(h ? &h->err : nullptr)
}

int smg_layout(const smg_handle* h, int64_t* bytes, int64_t dims_out[4]) {
    SMG_TRY
    if (!h) return fail(nullptr, SMG_EINVAL, "smg_layout: NULL handle");
    if (bytes) *bytes = (int64_t)h->bytes;
    if (dims_out) {
        dims_out[0] = h->g.s1;
        dims_out[1] = h->g.B[1];
        dims_out[2] = h->g.B[2];
        dims_out[3] = h->g.cs;
    }
    return SMG_OK;
    SMG_CATCH(h ? &const_cast<smg_handle*>(h)->err : nullptr)
}

int smg_check_finite(smg_handle* h) {
    SMG_TRY
    if (!h) return fail(h, SMG_EINVAL, "smg_check_finite: NULL handle");
    int flag = 0;
    SMG_CUDA(h, cudaMemsetAsync(h->dFlag, 0, sizeof(int), h->stream));
    SMG_CUDA(h, smg::launch_finite(h, h->dFlag, h->stream));
    SMG_CUDA(h, cudaMemcpyAsync(&flag, h->dFlag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    SMG_CUDA(h, cudaStreamSynchronize(h->stream));
    if (flag) return fail(h, SMG_ENONFINITE, "state holds NaN or Inf");
    return SMG_OK;
    SMG_CATCH(h ? &h->err : nullptr)
}

}  // extern "C"
