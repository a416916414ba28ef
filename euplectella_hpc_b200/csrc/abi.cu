// C ABI entry points (include/eup.h): handle life cycle, state transfer in the
// reference's haloed layout, the time-step sequence and diagnostics.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "../../include/eup.h"
#include "geometry.h"
#include "internal.h"

using namespace eup;

struct eup_handle {
    eup_config cfg{};
    Geo g{};
    cudaStream_t stream = nullptr;
    int prec = EUP_FP32;
    size_t sbytes = 4, rbytes = 4;
    int64_t Nq = 0;
    void* lat[2] = {nullptr, nullptr};
    void* ghost = nullptr;
    void* xface = nullptr;        // x = 1 / x = l columns, [2][18][m*n] arithmetic type
    int64_t* d_itime = nullptr;   // device copy of the step counter (series slot of the drag)
    cudaGraphExec_t graph[2] = {nullptr, nullptr};  // one time step, source lattice 0 or 1
    int cur = 0;
    uint32_t* bits = nullptr;
    int wpr = 0;
    int32_t* blist = nullptr;
    uint64_t* blinks = nullptr;   // neighbour classification of each boundary-solid voxel
    int64_t nblist = 0;
    int64_t nsolid = 0;           // solid voxels of the installed mask
    double* partials = nullptr;
    unsigned int* counter = nullptr;
    double* series = nullptr;
    int64_t cap = 0;
    double* dscratch = nullptr;  // 64 doubles
    unsigned int* d_bad = nullptr;  // upload check: bit q set when population q had a non-finite value
    unsigned int* bc_bar = nullptr; // grid barrier of the single-launch halo kernel: arrivals, generation, timeouts
    void* staging = nullptr;
    size_t staging_bytes = 0;
    // state transfers: a second staging buffer and a copy stream, so that the host copy of
    // one population overlaps the scatter (gather) of the previous one; events 0/1: copy of
    // buffer 0/1 done, 2/3: kernel on buffer 0/1 done
    void* staging2 = nullptr;
    size_t staging2_bytes = 0;
    cudaStream_t xfer = nullptr;
    cudaEvent_t xev[4] = {nullptr, nullptr, nullptr, nullptr};
    int64_t itime = 0, series_first = 0;
    bool has_state = false;
    double scale = 1.0;
    int variant = 0;  // EUP_STEP_VARIANT: bit 0/2 16/8-byte vector stream-collide, bit 1 no CUDA graphs
    bool pbb = false;             // partial-bounce-back model active (solid fraction set)
    void* ns = nullptr;           // solid fraction n_s per interior node, arithmetic type
    int32_t* ns_list = nullptr;   // interior linear indices with n_s > 0, ascending
    int64_t ns_count = 0;
    int64_t launches = 0;  // kernels launched by the step calls (split steps and plane pack/unpack too)
    bool mid_step = false;  // eup_step_boundaries done, eup_step_stream pending
    bool interior_done = false;  // eup_step_stream_interior done, eup_step_stream_faces pending
    int launches_per_step = 0;
    std::string err;
};

bool eup_internal_read_record(FILE* f, void* dst, int64_t want, std::string* why);
bool eup_internal_write_record(FILE* f, const void* src, int64_t bytes);

namespace {

thread_local std::string g_err;

int fail(eup_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    else g_err = msg;
    return code;
}

int cuda_fail(eup_handle* h, cudaError_t e, const char* what) {
    return fail(h, e == cudaErrorMemoryAllocation ? EUP_ERR_OOM : EUP_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

#define CK(h, call)                                      \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, #call); \
    } while (0)

bool face_flag_ok(int face, int f) {
    switch (face) {
        case EUP_FRONT: return f == 0 || f == 1 || f == 5 || f == EUP_BC_EXCHANGE;
        case EUP_REAR: return f == 0 || f == 1 || f == 4 || f == EUP_BC_EXCHANGE;
        case EUP_UP: return f == 0 || f == 1 || f == 2 || f == 3;
        default: return f == 0 || f == 1 || f == 3;
    }
}

// Population q of a lattice buffer: Nq elements per population, the node
// values starting kPopPad elements in.  16-bit storage shifts population q by
// cx_q elements, so that the pull a_q(x - c_q) of an even x reads an aligned
// pair in every population (see the two-node stream-collide kernel); the
// node-indexed view every kernel uses is unchanged.
constexpr int64_t kPopPad = 64;

template <typename S>
S* pop_ptr(const eup_handle* h, void* base, int q) {
    const int64_t shift = (DevStore<S>::value && q < 18) ? cx_of(q) : 0;
    return static_cast<S*>(base) + (q * h->Nq + kPopPad + shift);
}

template <typename S, typename R>
Lat<S, R> make_lat(const eup_handle* h, int which) {
    Lat<S, R> L;
    for (int q = 0; q < Q; ++q) L.pop[q] = pop_ptr<S>(h, h->lat[which], q);
    L.ghost = static_cast<R*>(h->ghost);
    L.xface = static_cast<R*>(h->xface);
    L.scale = (R)h->scale;
    L.inv_scale = (R)(1.0 / h->scale);
    return L;
}

template <typename R>
Phys<R> make_phys(const eup_handle* h) {
    // CODE/SRC/hencol.F90:30-39: svisc and u0 are real(mykind); omega from a
    // double expression; fgrad = 4.0*u0*svisc/(5.0*real(n)*real(n)) in mykind.
    Phys<R> ph;
    const R sv = (R)h->cfg.svisc, u0 = (R)h->cfg.u0;
    ph.omega = (R)(2.0 / (6.0 * (double)sv + 1.0));
    ph.omega1 = R(1) - ph.omega;
    ph.fgrad = R(4) * u0 * sv / (R(5) * (R)h->g.n * (R)h->g.n);
    ph.u_inflow = (R)h->cfg.u_inflow;
    ph.force = (R)((R)h->cfg.u00 / R(6));
    return ph;
}

Mask make_mask(const eup_handle* h) { return Mask{h->bits, h->wpr}; }

// The halo kernels' grid barrier when they run as one cooperative launch (EUP_STEP_VARIANT
// bit 12; measured slower than one launch per block, the default), else none.
unsigned int* bc_bar(const eup_handle* h) { return (h->variant & 4096) ? h->bc_bar : nullptr; }
Reduce make_reduce(const eup_handle* h) { return Reduce{h->partials, h->counter, kReduceMaxBlocks}; }

template <typename S, typename R>
void enqueue_drag_only(eup_handle* h) {
    const int bc[6] = {h->cfg.bc[0], h->cfg.bc[1], h->cfg.bc[2], h->cfg.bc[3], h->cfg.bc[4], h->cfg.bc[5]};
    launch_bounce_drag<S, R>(make_lat<S, R>(h, h->cur), h->g, bc, h->blist, h->blinks, h->nblist, false,
                             make_reduce(h), h->series, h->cap, h->d_itime, false, h->stream);
}

// Events bracketing the phases of each step when profiling: ev[4*s + p].
struct PhaseEvents {
    std::vector<cudaEvent_t> ev;
    void mark(size_t idx, cudaStream_t st) {
        if (idx < ev.size()) cudaEventRecord(ev[idx], st);
    }
};

// One time step from lattice `src_idx`: bounce-back + drag (advances the device
// step counter), halo planes in the reference's order, stream-collide.
// Returns the number of kernels launched.
template <typename S, typename R>
int enqueue_one_step(eup_handle* h, int src_idx, PhaseEvents* pe, size_t s) {
    const Phys<R> ph = make_phys<R>(h);
    const int bc[6] = {h->cfg.bc[0], h->cfg.bc[1], h->cfg.bc[2], h->cfg.bc[3], h->cfg.bc[4], h->cfg.bc[5]};
    const Lat<S, R> src = make_lat<S, R>(h, src_idx), dst = make_lat<S, R>(h, src_idx ^ 1);
    int n = 0;
    if (pe) pe->mark(4 * s + 0, h->stream);
    if (h->pbb) {  // partial bounce-back: halo planes, stream-collide, mixing and force of the step
        if (pe) pe->mark(4 * s + 1, h->stream);
        n += launch_bc<S, R>(src, h->g, bc, ph, h->stream, bc_bar(h));
        if (pe) pe->mark(4 * s + 2, h->stream);
        launch_pbb_step<S, R>(src, dst, h->g, ph, static_cast<const R*>(h->ns), h->ns_list, h->ns_count,
                              make_reduce(h), h->series, h->cap, h->d_itime, h->stream);
        if (pe) pe->mark(4 * s + 3, h->stream);
        return n + 2;
    }
    // boundaries: bounce-back then halo planes (CODE/SRC/boundaries.F90:36-49,235-248)
    launch_bounce_drag<S, R>(src, h->g, bc, h->blist, h->blinks, h->nblist, true, make_reduce(h), h->series,
                             h->cap, h->d_itime, true, h->stream);
    n += 1;
    if (pe) pe->mark(4 * s + 1, h->stream);
    n += launch_bc<S, R>(src, h->g, bc, ph, h->stream, bc_bar(h));
    if (pe) pe->mark(4 * s + 2, h->stream);
    // propagation + collision (CODE/SRC/bgk3d.F90:133-138)
    launch_stream_collide<S, R>(src, dst, h->g, ph, h->variant, h->stream);
    n += 1;
    if (pe) pe->mark(4 * s + 3, h->stream);
    return n;
}

// The two halves of a step of an x-slab lattice (the plane exchange goes between).
// Bit 0: the x = 0 face (column x = 1, side 0) is an exchange face; bit 1: the x = l+1 face.
int exchange_sides(const eup_handle* h) {
    return (h->cfg.bc[EUP_REAR] == EUP_BC_EXCHANGE ? 1 : 0) | (h->cfg.bc[EUP_FRONT] == EUP_BC_EXCHANGE ? 2 : 0);
}

template <typename S, typename R>
void enqueue_boundaries(eup_handle* h) {
    const Phys<R> ph = make_phys<R>(h);
    const int bc[6] = {h->cfg.bc[0], h->cfg.bc[1], h->cfg.bc[2], h->cfg.bc[3], h->cfg.bc[4], h->cfg.bc[5]};
    const Lat<S, R> src = make_lat<S, R>(h, h->cur);
    launch_bounce_drag<S, R>(src, h->g, bc, h->blist, h->blinks, h->nblist, true, make_reduce(h), h->series,
                             h->cap, h->d_itime, true, h->stream);
    h->launches += 1 + launch_bc<S, R>(src, h->g, bc, ph, h->stream, bc_bar(h));
    if (const int xs = exchange_sides(h)) {  // the plane messages' halo rows, after the halo kernels
        launch_pack_x_rim<S, R>(src, h->g, xs, h->stream);
        h->launches += 1;
    }
}

template <typename S, typename R>
void enqueue_stream(eup_handle* h, int part) {
    const Phys<R> ph = make_phys<R>(h);
    launch_stream_collide<S, R>(make_lat<S, R>(h, h->cur), make_lat<S, R>(h, h->cur ^ 1), h->g, ph, h->variant,
                                h->stream, part);
    h->launches += 1;
    if (part == kStreamInterior) return;
    h->cur ^= 1;
    h->itime += 1;
    enqueue_drag_only<S, R>(h);  // the force of the state reached, as eup_step leaves it
    h->launches += 1;
}

template <typename S, typename R>
void pack_x_dispatch(eup_handle* h, int side, void* dst) {
    launch_pack_x<S, R>(make_lat<S, R>(h, h->cur), h->g, side, static_cast<R*>(dst), h->stream);
    h->launches += 1;
}

template <typename S, typename R>
void unpack_x_dispatch(eup_handle* h, int side, const void* src) {
    launch_unpack_x<S, R>(make_lat<S, R>(h, h->cur), h->g, side, static_cast<const R*>(src), h->stream);
    h->launches += 1;
}

template <typename S, typename R>
void unpack_x_view_dispatch(eup_handle* h, int side, const void* src) {
    launch_unpack_x_view<S, R>(make_lat<S, R>(h, h->cur), h->g, side, static_cast<const R*>(src), h->stream);
    h->launches += 1;
}

template <typename S, typename R>
cudaError_t capture_graphs(eup_handle* h, int* per_step) {
    for (int p = 0; p < 2; ++p) {
        if (h->graph[p]) continue;
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        *per_step = enqueue_one_step<S, R>(h, p, nullptr, 0);
        e = cudaStreamEndCapture(h->stream, &graph);
        if (e != cudaSuccess) return e;
        e = cudaGraphInstantiate(&h->graph[p], graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

void drop_graphs(eup_handle* h) {
    for (auto& g : h->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

template <typename S, typename R>
cudaError_t enqueue_steps(eup_handle* h, int32_t nsteps, PhaseEvents* pe = nullptr) {
    if (pe || (h->variant & 2)) {  // profiled, or graphs disabled (EUP_STEP_VARIANT bit 1)
        for (int32_t s = 0; s < nsteps; ++s) {
            h->launches += enqueue_one_step<S, R>(h, h->cur, pe, (size_t)s);
            h->cur ^= 1;
            h->itime += 1;
        }
    } else {
        int per_step = 0;
        cudaError_t e = capture_graphs<S, R>(h, &per_step);
        if (e != cudaSuccess) return e;
        if (per_step == 0) per_step = h->launches_per_step;
        h->launches_per_step = per_step;
        for (int32_t s = 0; s < nsteps; ++s) {
            e = cudaGraphLaunch(h->graph[h->cur], h->stream);
            if (e != cudaSuccess) return e;
            h->launches += per_step;
            h->cur ^= 1;
            h->itime += 1;
        }
    }
    if (!h->pbb) {  // the partial-bounce-back step records its force itself
        enqueue_drag_only<S, R>(h);
        h->launches += 1;
    }
    return cudaSuccess;
}

#define DISPATCH(h, FN, ...)                                                   \
    do {                                                                       \
        switch ((h)->prec) {                                                   \
            case EUP_FP32: FN<float, float>(__VA_ARGS__); break;               \
            case EUP_FP64: FN<double, double>(__VA_ARGS__); break;             \
            case EUP_FP16_DEV: FN<__half, float>(__VA_ARGS__); break;          \
            default: FN<__nv_bfloat16, float>(__VA_ARGS__); break;             \
        }                                                                      \
    } while (0)

#define DISPATCH_RET(h, OUT, FN, ...)                                          \
    do {                                                                       \
        switch ((h)->prec) {                                                   \
            case EUP_FP32: OUT = FN<float, float>(__VA_ARGS__); break;         \
            case EUP_FP64: OUT = FN<double, double>(__VA_ARGS__); break;       \
            case EUP_FP16_DEV: OUT = FN<__half, float>(__VA_ARGS__); break;    \
            default: OUT = FN<__nv_bfloat16, float>(__VA_ARGS__); break;       \
        }                                                                      \
    } while (0)

template <typename S, typename R>
void fill_xface_dispatch(eup_handle* h) {
    launch_fill_xface<S, R>(make_lat<S, R>(h, h->cur), h->g, h->stream);
}

template <typename S, typename R, typename T>
void enqueue_upload_q(eup_handle* h, int q, const void* buf) {
    launch_scatter<S, R, T>(make_lat<S, R>(h, h->cur), h->g, q, static_cast<const T*>(buf), h->d_bad, h->stream);
}
template <typename S, typename R, typename T>
void enqueue_download_q(eup_handle* h, int q, void* buf) {
    launch_gather<S, R, T>(make_lat<S, R>(h, h->cur), h->g, q, static_cast<T*>(buf), h->stream);
}
template <typename S, typename R>
void upload_q(eup_handle* h, int q, int eb, const void* buf) {
    if (eb == 4) enqueue_upload_q<S, R, float>(h, q, buf);
    else enqueue_upload_q<S, R, double>(h, q, buf);
}
template <typename S, typename R>
void download_q(eup_handle* h, int q, int eb, void* buf) {
    if (eb == 4) enqueue_download_q<S, R, float>(h, q, buf);
    else enqueue_download_q<S, R, double>(h, q, buf);
}
template <typename S, typename R>
void monitor_dispatch(eup_handle* h) {
    launch_monitor<S, R>(make_lat<S, R>(h, h->cur), h->g, make_mask(h), make_reduce(h), h->dscratch, h->stream);
}
template <typename S, typename R>
void line_dispatch(eup_handle* h, int axis, int c1, int c2, double* d_out) {
    launch_line<S, R>(make_lat<S, R>(h, h->cur), h->g, axis, c1, c2, d_out, h->stream);
}
template <typename S, typename R>
void plane_dispatch(eup_handle* h, int axis, double* d_out) {
    launch_plane_means<S, R>(make_lat<S, R>(h, h->cur), h->g, axis, d_out, h->stream);
}
template <typename S, typename R>
void cv_dispatch(eup_handle* h, const int* box) {
    launch_cv_drag<S, R>(make_lat<S, R>(h, h->cur), h->g, box, make_phys<R>(h).omega, make_reduce(h), h->dscratch,
                         h->stream);
}
template <typename S, typename R>
void region_dispatch(eup_handle* h, const uint8_t* d_region) {
    launch_region_sums<S, R>(make_lat<S, R>(h, h->cur), h->g, make_mask(h), d_region, make_reduce(h), h->dscratch,
                             h->stream);
}
template <typename S, typename R>
void probes_dispatch(eup_handle* h, int npts, const int32_t* d_ijk, double* d_out) {
    launch_probes<S, R>(make_lat<S, R>(h, h->cur), h->g, npts, d_ijk, d_out, h->stream);
}

// After the 19 populations of a new state are on the device: step counter,
// x-face copy, and the force of the state (CODE/SRC/bgk3d.F90 records the drag
// of every state reached, the initial one included).
int finish_state(eup_handle* h, int64_t itime) {
    CK(h, cudaMemcpyAsync(h->d_itime, &itime, sizeof(int64_t), cudaMemcpyHostToDevice, h->stream));
    DISPATCH(h, fill_xface_dispatch, h);
    h->itime = itime;
    h->series_first = itime;
    h->has_state = true;
    h->mid_step = false;
    h->interior_done = false;
    if (h->pbb) CK(h, cudaMemsetAsync(h->series + 3 * (itime % h->cap), 0, 3 * sizeof(double), h->stream));
    else DISPATCH(h, enqueue_drag_only, h);
    CK(h, cudaGetLastError());
    CK(h, cudaStreamSynchronize(h->stream));
    return EUP_OK;
}

// The copy stream, its events and the second staging buffer of the state transfers.
int ensure_xfer(eup_handle* h, size_t bytes) {
    if (!h->xfer) {  // all or nothing: the handle keeps no half-made set
        cudaStream_t s = nullptr;
        cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
        cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        for (auto& x : ev)
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            for (auto& x : ev)
                if (x) cudaEventDestroy(x);
            if (s) cudaStreamDestroy(s);
            return cuda_fail(h, e, "state transfer stream");
        }
        h->xfer = s;
        for (int i = 0; i < 4; ++i) h->xev[i] = ev[i];
    }
    if (h->staging2_bytes >= bytes) return EUP_OK;
    if (h->staging2) {
        CK(h, cudaStreamSynchronize(h->xfer));
        cudaFree(h->staging2);
    }
    h->staging2 = nullptr;
    h->staging2_bytes = 0;
    CK(h, cudaMalloc(&h->staging2, bytes));
    h->staging2_bytes = bytes;
    return EUP_OK;
}

// End of a double-buffered state transfer: both streams drained whatever happened, so that
// no copy touches the caller's host arrays after the call returns; the first error wins.
int end_transfer(eup_handle* h, cudaError_t e, const char* who) {
    if (e == cudaSuccess) e = cudaGetLastError();
    const cudaError_t ex = cudaStreamSynchronize(h->xfer);
    const cudaError_t es = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess) e = ex != cudaSuccess ? ex : es;
    return e == cudaSuccess ? EUP_OK : cuda_fail(h, e, who);
}

int ensure_staging(eup_handle* h, size_t bytes) {
    if (h->staging_bytes >= bytes) return EUP_OK;
    if (h->staging) cudaFree(h->staging);
    h->staging = nullptr;
    h->staging_bytes = 0;
    CK(h, cudaMalloc(&h->staging, bytes));
    h->staging_bytes = bytes;
    return EUP_OK;
}

// Start / end of a state transfer into the device: the scatter sets bit q of d_bad for a
// population that held a value that is not finite.  A rejected state leaves the handle
// without a state (the lattice holds part of it).
int begin_upload_check(eup_handle* h) {
    CK(h, cudaMemsetAsync(h->d_bad, 0, sizeof(unsigned int), h->stream));
    return EUP_OK;
}
int end_upload_check(eup_handle* h, const char* who) {
    unsigned int bad = 0;
    CK(h, cudaMemcpyAsync(&bad, h->d_bad, sizeof(bad), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    if (bad == 0) return EUP_OK;
    h->has_state = false;
    std::string qs;
    for (int q = 0; q < Q; ++q)
        if (bad & (1u << q)) qs += (qs.empty() ? "" : ",") + std::to_string(q + 1);
    return fail(h, EUP_ERR_INVALID_ARG,
                std::string(who) + ": non-finite value (NaN or Inf) in population(s) a" + qs +
                    "; the state was rejected and the handle holds no state");
}

bool has_exchange_face(const eup_handle* h) {
    return h->cfg.bc[EUP_FRONT] == EUP_BC_EXCHANGE || h->cfg.bc[EUP_REAR] == EUP_BC_EXCHANGE;
}

// After a synchronisation: a bounded wait of the staged stream-collide kernel that ran out
// left a step incomplete.
int check_kernel_waits(eup_handle* h, const char* who) {
    unsigned int n = 0;
    CK(h, staged_wait_timeouts(&n));
    if (n != 0)
        return fail(h, EUP_ERR_CUDA,
                    std::string(who) + ": " + std::to_string(n) +
                        " bulk copies of the staged stream-collide kernel did not complete within 2 s; "
                        "the steps since are incomplete");
    unsigned int bar[3] = {0, 0, 0};
    CK(h, cudaMemcpy(bar, h->bc_bar, sizeof(bar), cudaMemcpyDeviceToHost));
    if (bar[2] != 0) {
        cudaMemset(h->bc_bar, 0, sizeof(bar));  // a barrier that gave up leaves its counter behind
        return fail(h, EUP_ERR_CUDA,
                    std::string(who) + ": " + std::to_string(bar[2]) +
                        " grid-barrier waits of the halo kernel gave up after 1 s; the steps since are incomplete");
    }
    return EUP_OK;
}

int check_handle(eup_handle* h) {
    if (!h) return fail(nullptr, EUP_ERR_INVALID_ARG, "null handle");
    cudaError_t e = cudaSetDevice(h->cfg.device);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaSetDevice");
    return EUP_OK;
}

}  // namespace

void eup_internal_set_error(const std::string& msg) { g_err = msg; }

extern "C" {

int32_t eup_abi_version(void) { return EUP_ABI_VERSION; }

int32_t eup_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

const char* eup_last_error(const eup_handle* h) { return h ? h->err.c_str() : g_err.c_str(); }

int eup_create(const eup_config* cfg, eup_handle** out) {
    if (!cfg || !out) return fail(nullptr, EUP_ERR_INVALID_ARG, "eup_create: null argument");
    *out = nullptr;
    if (cfg->lx < 1 || cfg->ly < 1 || cfg->lz < 1)
        return fail(nullptr, EUP_ERR_INVALID_ARG, "eup_create: lattice sizes must be >= 1");
    const int64_t N = (int64_t)cfg->lx * cfg->ly * cfg->lz;
    if (N > 2147483647LL)
        return fail(nullptr, EUP_ERR_UNSUPPORTED, "eup_create: more than 2^31-1 nodes on one GPU");
    for (int f = 0; f < 6; ++f)
        if (!face_flag_ok(f, cfg->bc[f]))
            return fail(nullptr, EUP_ERR_UNSUPPORTED,
                        "eup_create: boundary flag " + std::to_string(cfg->bc[f]) + " not defined for face " +
                            std::to_string(f) + " (CODE/SRC/bcond.bc.F90 has no such block)");
    if (cfg->precision < EUP_FP32 || cfg->precision > EUP_BF16_DEV)
        return fail(nullptr, EUP_ERR_INVALID_ARG, "eup_create: unknown precision");
    if (!(cfg->svisc > 0.0)) return fail(nullptr, EUP_ERR_INVALID_ARG, "eup_create: svisc must be > 0");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(nullptr, EUP_ERR_NO_DEVICE, "eup_create: no CUDA device");
    }
    if (cfg->device < 0 || cfg->device >= ndev)
        return fail(nullptr, EUP_ERR_INVALID_ARG, "eup_create: device ordinal out of range");

    eup_handle* h = new eup_handle();
    h->cfg = *cfg;
    h->g.init(cfg->lx, cfg->ly, cfg->lz);
    h->prec = cfg->precision;
    h->sbytes = (h->prec == EUP_FP32) ? 4 : (h->prec == EUP_FP64) ? 8 : 2;
    h->rbytes = (h->prec == EUP_FP64) ? 8 : 4;
    h->scale = (h->prec == EUP_FP16_DEV || h->prec == EUP_BF16_DEV) ? (cfg->dev_scale > 0 ? cfg->dev_scale : 4096.0) : 1.0;
    h->cap = cfg->series_capacity > 0 ? cfg->series_capacity : (int64_t)1 << 20;
    h->Nq = (N + 2 * kPopPad + 127) / 128 * 128;
    if (const char* v = std::getenv("EUP_STEP_VARIANT")) h->variant = std::atoi(v);

    auto cleanup_fail = [&](int code) {
        std::string m = h->err;
        eup_destroy(h);
        g_err = m;
        return code;
    };
    cudaError_t e = cudaSetDevice(cfg->device);
    if (e != cudaSuccess) return cleanup_fail(cuda_fail(h, e, "cudaSetDevice"));
    if ((e = prepare_stream_collide()) != cudaSuccess)
        return cleanup_fail(cuda_fail(h, e, "stream-collide kernel attributes"));
    if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return cleanup_fail(cuda_fail(h, e, "cudaStreamCreate"));
    const size_t lat_bytes = (size_t)Q * h->Nq * h->sbytes;
    for (int w = 0; w < 2; ++w) {
        if ((e = cudaMalloc(&h->lat[w], lat_bytes)) != cudaSuccess)
            return cleanup_fail(cuda_fail(h, e, "cudaMalloc(lattice)"));
        cudaMemsetAsync(h->lat[w], 0, lat_bytes, h->stream);
    }
    const size_t ghost_bytes = (size_t)Q * h->g.G * h->rbytes;
    if ((e = cudaMalloc(&h->ghost, ghost_bytes)) != cudaSuccess) return cleanup_fail(cuda_fail(h, e, "cudaMalloc(halo shell)"));
    cudaMemsetAsync(h->ghost, 0, ghost_bytes, h->stream);
    if ((e = cudaMalloc(&h->partials, sizeof(double) * kReduceMaxBlocks * kReduceWidth)) != cudaSuccess)
        return cleanup_fail(cuda_fail(h, e, "cudaMalloc(partials)"));
    if ((e = cudaMalloc(&h->counter, sizeof(unsigned int))) != cudaSuccess)
        return cleanup_fail(cuda_fail(h, e, "cudaMalloc(counter)"));
    cudaMemsetAsync(h->counter, 0, sizeof(unsigned int), h->stream);
    if ((e = cudaMalloc(&h->series, sizeof(double) * 3 * h->cap)) != cudaSuccess)
        return cleanup_fail(cuda_fail(h, e, "cudaMalloc(force series)"));
    cudaMemsetAsync(h->series, 0, sizeof(double) * 3 * h->cap, h->stream);
    if ((e = cudaMalloc(&h->dscratch, sizeof(double) * 64)) != cudaSuccess)
        return cleanup_fail(cuda_fail(h, e, "cudaMalloc(scratch)"));
    if ((e = cudaMalloc(&h->d_bad, sizeof(unsigned int))) != cudaSuccess)
        return cleanup_fail(cuda_fail(h, e, "cudaMalloc(upload check)"));
    if ((e = cudaMalloc(&h->bc_bar, 3 * sizeof(unsigned int))) != cudaSuccess)
        return cleanup_fail(cuda_fail(h, e, "cudaMalloc(halo barrier)"));
    if ((e = cudaMemset(h->bc_bar, 0, 3 * sizeof(unsigned int))) != cudaSuccess)
        return cleanup_fail(cuda_fail(h, e, "cudaMemset(halo barrier)"));
    if ((h->variant & 4096) && (e = prepare_bc_fused(h->bc_bar)) != cudaSuccess)
        return cleanup_fail(cuda_fail(h, e, "halo kernel set-up"));
    const size_t xface_bytes = (size_t)xface_elems(h->g) * h->rbytes;
    if ((e = cudaMalloc(&h->xface, xface_bytes)) != cudaSuccess)
        return cleanup_fail(cuda_fail(h, e, "cudaMalloc(x-face copy)"));
    cudaMemsetAsync(h->xface, 0, xface_bytes, h->stream);
    if ((e = cudaMalloc(&h->d_itime, sizeof(int64_t))) != cudaSuccess)
        return cleanup_fail(cuda_fail(h, e, "cudaMalloc(step counter)"));
    cudaMemsetAsync(h->d_itime, 0, sizeof(int64_t), h->stream);
    if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return cleanup_fail(cuda_fail(h, e, "create"));
    *out = h;
    return EUP_OK;
}

int eup_destroy(eup_handle* h) {
    if (!h) return EUP_OK;
    cudaSetDevice(h->cfg.device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->xfer) cudaStreamSynchronize(h->xfer);
    drop_graphs(h);
    void* ptrs[] = {h->lat[0], h->lat[1], h->ghost, h->bits, h->blist, h->blinks, h->partials, h->counter,
                    h->series, h->dscratch, h->staging, h->xface, h->d_itime, h->ns, h->d_bad, h->ns_list,
                    h->bc_bar, h->staging2};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (cudaEvent_t e : h->xev)
        if (e) cudaEventDestroy(e);
    if (h->xfer) cudaStreamDestroy(h->xfer);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return EUP_OK;
}

}  // extern "C"

namespace {

// The checks eup_set_obstacles and eup_build_obstacles share, from the number of solid
// voxels and of those on the columns i = 1 and i = l.
int check_obstacles(eup_handle* h, const char* who, int64_t nsolid, int64_t on_first, int64_t on_last) {
    if (nsolid > 0 && h->pbb)
        return fail(h, EUP_ERR_UNSUPPORTED,
                    std::string(who) + ": a solid-fraction field is set; the partial-bounce-back model takes no "
                    "halfway-bounce-back voxels (fold them into the field as n_s = 1)");
    if (h->cfg.bc[EUP_FRONT] == EUP_BC_OUTFLOW && on_last > 0)
        return fail(h, EUP_ERR_UNSUPPORTED,
                    std::string(who) + ": solid voxel on the outflow plane i=l; the reference's outflow "
                    "there reads values whose order its bounce-back loop leaves undefined");
    if ((h->cfg.bc[EUP_REAR] == EUP_BC_EXCHANGE && on_first > 0) ||
        (h->cfg.bc[EUP_FRONT] == EUP_BC_EXCHANGE && on_last > 0))
        return fail(h, EUP_ERR_UNSUPPORTED,
                    std::string(who) + ": solid voxel on a column next to an x-slab exchange face; move the "
                    "slab boundary (bounce-back there would read the neighbour's previous state)");
    return EUP_OK;
}

// Installs `bits` (m*n*wpr words, owned by the handle from here on; null or
// nsolid == 0: no solids) in place of the current mask: the list of boundary
// solids, their link words, and the drag of the current state.  Every buffer is
// allocated before the current mask is released, so a failed allocation leaves
// the handle as it was.
int install_mask(eup_handle* h, uint32_t* bits, int64_t nsolid) {
    const Geo& g = h->g;
    if (nsolid <= 0 && bits) { cudaFree(bits); bits = nullptr; }
    uint8_t* d_flags = nullptr;
    int32_t* blist = nullptr;
    uint64_t* blinks = nullptr;
    if (nsolid > 0) {
        cudaError_t e = cudaMalloc(&d_flags, g.N);
        if (e == cudaSuccess) e = cudaMalloc(&blist, sizeof(int32_t) * (size_t)nsolid);
        if (e == cudaSuccess) e = cudaMalloc(&blinks, sizeof(uint64_t) * (size_t)nsolid);
        if (e != cudaSuccess) {
            cudaFree(d_flags);
            cudaFree(blist);
            cudaFree(blinks);
            cudaFree(bits);
            return cuda_fail(h, e, "install obstacles");
        }
    }
    drop_graphs(h);  // the captured steps hold the old mask and list pointers
    if (h->bits) cudaFree(h->bits);
    if (h->blist) cudaFree(h->blist);
    if (h->blinks) cudaFree(h->blinks);
    h->bits = bits;
    h->blist = blist;
    h->blinks = blinks;
    h->nblist = 0;
    h->nsolid = nsolid > 0 ? nsolid : 0;
    if (nsolid > 0) {
        launch_flag_boundary_solid(g, make_mask(h), d_flags, h->stream);
        cudaError_t e;
        const int64_t cnt = compact_flags(d_flags, g.N, h->blist, h->stream, &e);
        cudaFree(d_flags);
        if (e != cudaSuccess) return cuda_fail(h, e, "compact boundary solid list");
        h->nblist = cnt;  // cnt <= nsolid: the boundary solids are solids
        const int bc[6] = {h->cfg.bc[0], h->cfg.bc[1], h->cfg.bc[2], h->cfg.bc[3], h->cfg.bc[4], h->cfg.bc[5]};
        launch_bsolid_links(g, make_mask(h), bc, h->blist, cnt, h->blinks, h->stream);
    }
    if (h->has_state && !h->pbb) DISPATCH(h, enqueue_drag_only, h);
    CK(h, cudaGetLastError());
    CK(h, cudaStreamSynchronize(h->stream));
    return EUP_OK;
}

}  // namespace

extern "C" {

int eup_set_obstacles(eup_handle* h, const int32_t* obs) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!obs) return fail(h, EUP_ERR_INVALID_ARG, "eup_set_obstacles: null obs");
    const Geo& g = h->g;
    int64_t nsolid = 0, on_first = 0, on_last = 0;
    for (int64_t t = 0; t < g.N; ++t) nsolid += (obs[t] == 1);
    for (int64_t r = 0; r < (int64_t)g.m * g.n; ++r) {
        on_first += (obs[r * g.l] == 1);
        on_last += (obs[r * g.l + (g.l - 1)] == 1);
    }
    if ((rc = check_obstacles(h, "eup_set_obstacles", nsolid, on_first, on_last))) return rc;
    CK(h, cudaStreamSynchronize(h->stream));
    h->wpr = (g.l + 31) / 32;
    uint32_t* bits = nullptr;
    if (nsolid > 0) {
        int32_t* d_obs = nullptr;
        CK(h, cudaMalloc(&d_obs, sizeof(int32_t) * g.N));
        cudaError_t e = cudaMemcpyAsync(d_obs, obs, sizeof(int32_t) * g.N, cudaMemcpyHostToDevice, h->stream);
        if (e == cudaSuccess) e = cudaMalloc(&bits, sizeof(uint32_t) * (size_t)g.m * g.n * h->wpr);
        if (e == cudaSuccess) launch_build_mask(d_obs, g, bits, h->wpr, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        cudaFree(d_obs);
        if (e != cudaSuccess) {
            if (bits) cudaFree(bits);
            return cuda_fail(h, e, "eup_set_obstacles: mask");
        }
    }
    return install_mask(h, bits, nsolid);
}

int eup_build_obstacles(eup_handle* h, const eup_geometry* geo) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!geo) return fail(h, EUP_ERR_INVALID_ARG, "eup_build_obstacles: null geometry");
    VoxShape S;
    std::vector<double> pores;
    std::string why;
    if (!prepare_shape(*geo, &S, &pores, &why)) return fail(h, EUP_ERR_INVALID_ARG, "eup_build_obstacles: " + why);
    const Geo& g = h->g;
    CK(h, cudaStreamSynchronize(h->stream));
    const int wpr = (g.l + 31) / 32;
    uint32_t* bits = nullptr;
    double* d_pores = nullptr;
    unsigned long long* d_cnt = nullptr;
    unsigned long long cnt[3] = {0, 0, 0};
    cudaError_t e = cudaMalloc(&bits, sizeof(uint32_t) * (size_t)g.m * g.n * wpr);
    if (e == cudaSuccess) e = cudaMalloc(&d_cnt, sizeof(cnt));
    if (e == cudaSuccess && !pores.empty()) {
        e = cudaMalloc(&d_pores, sizeof(double) * pores.size());
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_pores, pores.data(), sizeof(double) * pores.size(), cudaMemcpyHostToDevice, h->stream);
    }
    S.ridge.pores = d_pores;
    if (e == cudaSuccess) {
        launch_voxelise(g, S, bits, wpr, h->stream);
        launch_mask_counts(bits, g, wpr, d_cnt, h->stream);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(cnt, d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (d_pores) cudaFree(d_pores);
    if (d_cnt) cudaFree(d_cnt);
    if (e != cudaSuccess) {
        if (bits) cudaFree(bits);
        return cuda_fail(h, e, "eup_build_obstacles");
    }
    if ((rc = check_obstacles(h, "eup_build_obstacles", (int64_t)cnt[0], (int64_t)cnt[1], (int64_t)cnt[2]))) {
        cudaFree(bits);
        return rc;
    }
    h->wpr = wpr;
    return install_mask(h, bits, (int64_t)cnt[0]);
}

int eup_get_obstacles(eup_handle* h, int32_t* obs, int64_t* nobs) {
    int rc = check_handle(h);
    if (rc) return rc;
    const Geo& g = h->g;
    if (nobs) *nobs = h->nsolid;
    if (!obs) return EUP_OK;
    if (!h->bits) {
        std::memset(obs, 0, sizeof(int32_t) * (size_t)g.N);
        return EUP_OK;
    }
    const int64_t rows = (int64_t)g.m * g.n;
    std::vector<uint32_t> bits((size_t)(rows * h->wpr));
    CK(h, cudaMemcpyAsync(bits.data(), h->bits, sizeof(uint32_t) * bits.size(), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    const int wpr = h->wpr, l = g.l;
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < rows; ++r)
        for (int i = 0; i < l; ++i) obs[r * l + i] = (int32_t)((bits[(size_t)(r * wpr + (i >> 5))] >> (i & 31)) & 1u);
    return EUP_OK;
}

int eup_write_obstacles(eup_handle* h, const char* path) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!path) return fail(h, EUP_ERR_INVALID_ARG, "eup_write_obstacles: null path");
    const int64_t n = h->nsolid;
    if (n > 2147483647LL) return fail(h, EUP_ERR_UNSUPPORTED, "eup_write_obstacles: more than 2^31-1 obstacles");
    CK(h, cudaStreamSynchronize(h->stream));
    int32_t* d_rec = nullptr;
    int32_t* rec = nullptr;
    const size_t bytes = sizeof(int32_t) * 5 * (size_t)n;
    cudaError_t e = cudaSuccess;
    if (n > 0) {
        e = cudaMalloc(&d_rec, bytes);
        if (e == cudaSuccess) e = cudaMallocHost(&rec, bytes);
        if (e == cudaSuccess) e = obstacle_records(h->g, make_mask(h), n, d_rec, h->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(rec, d_rec, bytes, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    }
    int out = EUP_OK;
    if (e != cudaSuccess) {
        out = cuda_fail(h, e, "eup_write_obstacles");
    } else {
        FILE* f = std::fopen(path, "wb");
        const int32_t c32 = (int32_t)n;
        if (!f) out = fail(h, EUP_ERR_IO, std::string("eup_write_obstacles: cannot create ") + path);
        else if (!eup_internal_write_record(f, &c32, 4) || (n > 0 && std::fwrite(rec, 1, bytes, f) != bytes))
            out = fail(h, EUP_ERR_IO, "eup_write_obstacles: write failed");
        if (f && std::fclose(f) != 0 && out == EUP_OK) out = fail(h, EUP_ERR_IO, "eup_write_obstacles: close failed");
    }
    if (d_rec) cudaFree(d_rec);
    if (rec) cudaFreeHost(rec);
    return out;
}

int eup_upload(eup_handle* h, const void* const pops[19], int32_t elem_bytes, int64_t itime) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!pops || (elem_bytes != 4 && elem_bytes != 8))
        return fail(h, EUP_ERR_INVALID_ARG, "eup_upload: pops must be 19 arrays of 4- or 8-byte reals");
    for (int q = 0; q < Q; ++q)
        if (!pops[q]) return fail(h, EUP_ERR_INVALID_ARG, "eup_upload: null population array");
    const Geo& g = h->g;
    const size_t bytes = (size_t)(g.l + 2) * (g.m + 2) * (g.n + 2) * elem_bytes;
    if ((rc = ensure_staging(h, bytes)) || (rc = ensure_xfer(h, bytes))) return rc;
    if ((rc = begin_upload_check(h))) return rc;
    void* buf[2] = {h->staging, h->staging2};
    // earlier work on the stream may use the buffers
    cudaError_t e = cudaEventRecord(h->xev[2], h->stream);
    if (e == cudaSuccess) e = cudaEventRecord(h->xev[3], h->stream);
    for (int q = 0; q < Q && e == cudaSuccess; ++q) {  // copy of q (copy stream) beside the scatter of q - 1
        const int b = q & 1;
        e = cudaStreamWaitEvent(h->xfer, h->xev[2 + b], 0);
        if (e == cudaSuccess) e = cudaMemcpyAsync(buf[b], pops[q], bytes, cudaMemcpyHostToDevice, h->xfer);
        if (e == cudaSuccess) e = cudaEventRecord(h->xev[b], h->xfer);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(h->stream, h->xev[b], 0);
        if (e == cudaSuccess) {
            DISPATCH(h, upload_q, h, q, elem_bytes, buf[b]);
            e = cudaEventRecord(h->xev[2 + b], h->stream);
        }
    }
    if ((rc = end_transfer(h, e, "eup_upload"))) return rc;
    if ((rc = end_upload_check(h, "eup_upload"))) return rc;
    return finish_state(h, itime);
}

int eup_init_state(eup_handle* h, double u_in, double amp, uint64_t seed, int64_t itime) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!std::isfinite(u_in) || !std::isfinite(amp)) return fail(h, EUP_ERR_INVALID_ARG, "eup_init_state: bad velocity");
    const Geo& g = h->g;
    const int eb = (h->prec == EUP_FP64) ? 8 : 4;  // what eup_init_equilibrium would hand to eup_upload
    const size_t bytes = (size_t)(g.l + 2) * (g.m + 2) * (g.n + 2) * eb;
    if ((rc = ensure_staging(h, bytes))) return rc;
    if ((rc = begin_upload_check(h))) return rc;
    for (int q = 0; q < Q; ++q) {
        if (eb == 8) launch_init_population<double>(static_cast<double*>(h->staging), g, q, u_in, amp, seed, h->stream);
        else launch_init_population<float>(static_cast<float*>(h->staging), g, q, u_in, amp, seed, h->stream);
        DISPATCH(h, upload_q, h, q, eb, h->staging);
    }
    if ((rc = end_upload_check(h, "eup_init_state"))) return rc;
    return finish_state(h, itime);
}

int eup_save_state(eup_handle* h, const char* path, int32_t elem_bytes) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!path || (elem_bytes != 4 && elem_bytes != 8))
        return fail(h, EUP_ERR_INVALID_ARG, "eup_save_state: need a path and elem_bytes 4 or 8");
    if (!h->has_state) return fail(h, EUP_ERR_INVALID_ARG, "eup_save_state: no state uploaded");
    if (h->itime > 2147483647LL) return fail(h, EUP_ERR_UNSUPPORTED, "eup_save_state: itime beyond int32");
    const Geo& g = h->g;
    const size_t bytes = (size_t)(g.l + 2) * (g.m + 2) * (g.n + 2) * elem_bytes;
    if ((rc = ensure_staging(h, bytes))) return rc;
    void* pinned = nullptr;
    CK(h, cudaMallocHost(&pinned, bytes));
    FILE* f = std::fopen(path, "wb");
    int out = EUP_OK;
    const int32_t it = (int32_t)h->itime;
    if (!f) out = fail(h, EUP_ERR_IO, std::string("eup_save_state: cannot create ") + path);
    else if (!eup_internal_write_record(f, &it, 4)) out = fail(h, EUP_ERR_IO, "eup_save_state: write failed");
    for (int q = 0; q < Q && out == EUP_OK; ++q) {
        DISPATCH(h, download_q, h, q, elem_bytes, h->staging);
        cudaError_t e = cudaMemcpyAsync(pinned, h->staging, bytes, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) out = cuda_fail(h, e, "eup_save_state");
        else if (!eup_internal_write_record(f, pinned, (int64_t)bytes))
            out = fail(h, EUP_ERR_IO, "eup_save_state: write failed (records over 2 GiB are not supported)");
    }
    if (f) std::fclose(f);
    cudaFreeHost(pinned);
    return out;
}

int eup_restore_state(eup_handle* h, const char* path, int32_t elem_bytes) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!path || (elem_bytes != 4 && elem_bytes != 8))
        return fail(h, EUP_ERR_INVALID_ARG, "eup_restore_state: need a path and elem_bytes 4 or 8");
    const Geo& g = h->g;
    const size_t bytes = (size_t)(g.l + 2) * (g.m + 2) * (g.n + 2) * elem_bytes;
    if ((rc = ensure_staging(h, bytes))) return rc;
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(h, EUP_ERR_IO, std::string("eup_restore_state: cannot open ") + path);
    void* pinned = nullptr;
    cudaError_t e = cudaMallocHost(&pinned, bytes);
    if (e != cudaSuccess) {
        std::fclose(f);
        return cuda_fail(h, e, "cudaMallocHost");
    }
    int out = begin_upload_check(h);
    int32_t it = 0;
    std::string why;
    if (out == EUP_OK && !eup_internal_read_record(f, &it, 4, &why)) out = fail(h, EUP_ERR_IO, "eup_restore_state: itime: " + why);
    for (int q = 0; q < Q && out == EUP_OK; ++q) {
        if (!eup_internal_read_record(f, pinned, (int64_t)bytes, &why)) {
            out = fail(h, EUP_ERR_IO, "eup_restore_state: population " + std::to_string(q + 1) + ": " + why);
            break;
        }
        e = cudaMemcpyAsync(h->staging, pinned, bytes, cudaMemcpyHostToDevice, h->stream);
        if (e == cudaSuccess) {
            DISPATCH(h, upload_q, h, q, elem_bytes, h->staging);
            e = cudaStreamSynchronize(h->stream);  // the pinned buffer is refilled next
        }
        if (e != cudaSuccess) out = cuda_fail(h, e, "eup_restore_state");
    }
    std::fclose(f);
    cudaFreeHost(pinned);
    if (out != EUP_OK) return out;
    if ((out = end_upload_check(h, "eup_restore_state"))) return out;
    return finish_state(h, it);
}

int eup_download(eup_handle* h, void* const pops[19], int32_t elem_bytes) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!h->has_state) return fail(h, EUP_ERR_INVALID_ARG, "eup_download: no state uploaded");
    if (!pops || (elem_bytes != 4 && elem_bytes != 8))
        return fail(h, EUP_ERR_INVALID_ARG, "eup_download: pops must be 19 arrays of 4- or 8-byte reals");
    for (int q = 0; q < Q; ++q)
        if (!pops[q]) return fail(h, EUP_ERR_INVALID_ARG, "eup_download: null population array");
    const Geo& g = h->g;
    const size_t bytes = (size_t)(g.l + 2) * (g.m + 2) * (g.n + 2) * elem_bytes;
    if ((rc = ensure_staging(h, bytes)) || (rc = ensure_xfer(h, bytes))) return rc;
    void* buf[2] = {h->staging, h->staging2};
    // earlier copies may still read the buffers
    cudaError_t e = cudaEventRecord(h->xev[0], h->xfer);
    if (e == cudaSuccess) e = cudaEventRecord(h->xev[1], h->xfer);
    for (int q = 0; q < Q && e == cudaSuccess; ++q) {  // gather of q beside the copy of q - 1 (copy stream)
        const int b = q & 1;
        e = cudaStreamWaitEvent(h->stream, h->xev[b], 0);
        if (e == cudaSuccess) {
            DISPATCH(h, download_q, h, q, elem_bytes, buf[b]);
            e = cudaEventRecord(h->xev[2 + b], h->stream);
        }
        if (e == cudaSuccess) e = cudaStreamWaitEvent(h->xfer, h->xev[2 + b], 0);
        if (e == cudaSuccess) e = cudaMemcpyAsync(pops[q], buf[b], bytes, cudaMemcpyDeviceToHost, h->xfer);
        if (e == cudaSuccess) e = cudaEventRecord(h->xev[b], h->xfer);
    }
    return end_transfer(h, e, "eup_download");
}

int eup_step(eup_handle* h, int32_t nsteps) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!h->has_state) return fail(h, EUP_ERR_INVALID_ARG, "eup_step: no state uploaded");
    if (nsteps < 0) return fail(h, EUP_ERR_INVALID_ARG, "eup_step: nsteps < 0");
    if (has_exchange_face(h))
        return fail(h, EUP_ERR_INVALID_ARG,
                    "eup_step: an x-slab lattice steps with eup_step_boundaries / eup_step_stream around the "
                    "plane exchange");
    if (nsteps == 0) return EUP_OK;
    cudaError_t e = cudaSuccess;
    DISPATCH_RET(h, e, enqueue_steps, h, nsteps);
    if (e != cudaSuccess) return cuda_fail(h, e, "eup_step");
    CK(h, cudaGetLastError());
    return EUP_OK;
}

int eup_step_boundaries(eup_handle* h) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!h->has_state) return fail(h, EUP_ERR_INVALID_ARG, "eup_step_boundaries: no state uploaded");
    if (h->pbb) return fail(h, EUP_ERR_UNSUPPORTED, "eup_step_boundaries: not for the partial-bounce-back model");
    if (h->mid_step) return fail(h, EUP_ERR_INVALID_ARG, "eup_step_boundaries: eup_step_stream is due first");
    DISPATCH(h, enqueue_boundaries, h);
    CK(h, cudaGetLastError());
    h->mid_step = true;
    return EUP_OK;
}

int eup_step_stream(eup_handle* h) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!h->mid_step || h->interior_done)
        return fail(h, EUP_ERR_INVALID_ARG, "eup_step_stream: eup_step_boundaries (alone) is due first");
    DISPATCH(h, enqueue_stream, h, (int)kStreamAll);
    CK(h, cudaGetLastError());
    h->mid_step = false;
    return EUP_OK;
}

int eup_step_stream_interior(eup_handle* h) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!h->mid_step || h->interior_done)
        return fail(h, EUP_ERR_INVALID_ARG, "eup_step_stream_interior: eup_step_boundaries (alone) is due first");
    DISPATCH(h, enqueue_stream, h, (int)kStreamInterior);
    CK(h, cudaGetLastError());
    h->interior_done = true;
    return EUP_OK;
}

int eup_step_stream_faces(eup_handle* h) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!h->mid_step || !h->interior_done)
        return fail(h, EUP_ERR_INVALID_ARG, "eup_step_stream_faces: eup_step_stream_interior is due first");
    DISPATCH(h, enqueue_stream, h, (int)kStreamFaces);
    CK(h, cudaGetLastError());
    h->interior_done = false;
    h->mid_step = false;
    return EUP_OK;
}

int eup_get_x_planes(eup_handle* h, int32_t side, void* dst) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!dst || (side != 0 && side != 1)) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_x_planes: bad side or null");
    if (!h->has_state) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_x_planes: no state uploaded");
    DISPATCH(h, pack_x_dispatch, h, side, dst);
    CK(h, cudaGetLastError());
    return EUP_OK;
}

int eup_set_x_planes(eup_handle* h, int32_t side, const void* src) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!src || (side != 0 && side != 1)) return fail(h, EUP_ERR_INVALID_ARG, "eup_set_x_planes: bad side or null");
    if (h->cfg.bc[side == 0 ? EUP_REAR : EUP_FRONT] != EUP_BC_EXCHANGE)
        return fail(h, EUP_ERR_INVALID_ARG, "eup_set_x_planes: that face is not an exchange face");
    DISPATCH(h, unpack_x_dispatch, h, side, src);
    CK(h, cudaGetLastError());
    return EUP_OK;
}

int eup_get_x_planes_view(eup_handle* h, int32_t side, const void** dev) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!dev || (side != 0 && side != 1))
        return fail(h, EUP_ERR_INVALID_ARG, "eup_get_x_planes_view: bad side or null");
    if (!((exchange_sides(h) >> side) & 1))
        return fail(h, EUP_ERR_INVALID_ARG, "eup_get_x_planes_view: that face is not an exchange face");
    *dev = static_cast<const char*>(h->xface) + (size_t)xface_send_offset(h->g, side) * h->rbytes;
    return EUP_OK;
}

int eup_set_x_planes_view(eup_handle* h, int32_t side, const void* src) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!src || (side != 0 && side != 1))
        return fail(h, EUP_ERR_INVALID_ARG, "eup_set_x_planes_view: bad side or null");
    if (!((exchange_sides(h) >> side) & 1))
        return fail(h, EUP_ERR_INVALID_ARG, "eup_set_x_planes_view: that face is not an exchange face");
    DISPATCH(h, unpack_x_view_dispatch, h, side, src);
    CK(h, cudaGetLastError());
    return EUP_OK;
}

int eup_step_profiled(eup_handle* h, int32_t nsteps, double ms[4]) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!ms) return fail(h, EUP_ERR_INVALID_ARG, "eup_step_profiled: null ms");
    if (!h->has_state) return fail(h, EUP_ERR_INVALID_ARG, "eup_step_profiled: no state uploaded");
    if (nsteps < 1) return fail(h, EUP_ERR_INVALID_ARG, "eup_step_profiled: nsteps < 1");
    if (has_exchange_face(h))
        return fail(h, EUP_ERR_INVALID_ARG, "eup_step_profiled: not for an x-slab lattice");
    PhaseEvents pe;
    pe.ev.resize(4 * (size_t)nsteps + 1);
    for (auto& e : pe.ev) CK(h, cudaEventCreate(&e));
    cudaError_t e = cudaSuccess;
    DISPATCH_RET(h, e, enqueue_steps, h, nsteps, &pe);
    pe.mark(pe.ev.size() - 1, h->stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess) {
        for (int32_t s = 0; s < nsteps; ++s)
            for (int p = 0; p < 3; ++p) {
                float t = 0.f;
                cudaEventElapsedTime(&t, pe.ev[4 * (size_t)s + p], pe.ev[4 * (size_t)s + p + 1]);
                ms[p] += t;
            }
        float tot = 0.f;
        cudaEventElapsedTime(&tot, pe.ev[0], pe.ev.back());
        ms[3] = tot;
    }
    for (auto& ev : pe.ev) cudaEventDestroy(ev);
    if (e != cudaSuccess) return cuda_fail(h, e, "eup_step_profiled");
    return EUP_OK;
}

int eup_synchronize(eup_handle* h) {
    int rc = check_handle(h);
    if (rc) return rc;
    CK(h, cudaStreamSynchronize(h->stream));
    return check_kernel_waits(h, "eup_synchronize");
}

int eup_get_launch_count(eup_handle* h, int64_t* launches) {
    if (!h || !launches) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_launch_count: null argument");
    *launches = h->launches;
    return EUP_OK;
}

int eup_get_stream(eup_handle* h, void** stream) {
    if (!h || !stream) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_stream: null argument");
    *stream = (void*)h->stream;
    return EUP_OK;
}

int eup_get_itime(eup_handle* h, int64_t* itime) {
    if (!h || !itime) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_itime: null argument");
    *itime = h->itime;
    return EUP_OK;
}

int eup_get_forces(eup_handle* h, double fxyz[3]) { return eup_get_force_series(h, h ? h->itime : 0, 1, fxyz); }

int eup_get_force_series(eup_handle* h, int64_t first_step, int32_t count, double* fxyz) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!fxyz || count < 0) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_force_series: bad argument");
    if (!h->has_state) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_force_series: no state uploaded");
    const int64_t lo = std::max(h->series_first, h->itime - h->cap + 1);
    if (first_step < lo || first_step + count - 1 > h->itime)
        return fail(h, EUP_ERR_INVALID_ARG,
                    "eup_get_force_series: steps " + std::to_string(first_step) + ".." +
                        std::to_string(first_step + count - 1) + " outside the recorded range " +
                        std::to_string(lo) + ".." + std::to_string(h->itime));
    CK(h, cudaStreamSynchronize(h->stream));
    if ((rc = check_kernel_waits(h, "eup_get_force_series"))) return rc;
    for (int32_t c = 0; c < count;) {
        const int64_t t = first_step + c;
        const int64_t pos = t % h->cap;
        const int32_t run = (int32_t)std::min<int64_t>(count - c, h->cap - pos);
        CK(h, cudaMemcpy(fxyz + 3 * (int64_t)c, h->series + 3 * pos, sizeof(double) * 3 * run, cudaMemcpyDeviceToHost));
        c += run;
    }
    for (int64_t t = 0; t < 3 * (int64_t)count; ++t)
        if (!std::isfinite(fxyz[t]))
            return fail(h, EUP_ERR_DIVERGED,
                        "eup_get_force_series: non-finite FP64 force at step " + std::to_string(first_step + t / 3) +
                            " (run diverged)");
    return EUP_OK;
}

int eup_get_cd_series(eup_handle* h, int64_t first_step, int32_t count, double* cd) {
    if (!cd || count < 0) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_cd_series: bad argument");
    if (h && !(h->cfg.cd_rho0 > 0 && h->cfg.cd_uref != 0 && h->cfg.cd_length > 0 && h->cfg.cd_span > 0))
        return fail(h, EUP_ERR_INVALID_ARG, "eup_get_cd_series: drag normalisation not set in eup_config");
    std::vector<double> f((size_t)3 * count);
    int rc = eup_get_force_series(h, first_step, count, f.data());
    if (rc) return rc;
    const double den = 0.5 * h->cfg.cd_rho0 * h->cfg.cd_uref * h->cfg.cd_uref * h->cfg.cd_length * h->cfg.cd_span;
    for (int32_t c = 0; c < count; ++c) cd[c] = f[3 * (size_t)c] / den;
    return EUP_OK;
}

int eup_get_monitor(eup_handle* h, double out[5]) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!out) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_monitor: null out");
    if (!h->has_state) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_monitor: no state uploaded");
    DISPATCH(h, monitor_dispatch, h);
    CK(h, cudaGetLastError());
    CK(h, cudaMemcpyAsync(out, h->dscratch, sizeof(double) * 5, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    for (int c = 0; c < 5; ++c)
        if (!std::isfinite(out[c])) return fail(h, EUP_ERR_DIVERGED, "eup_get_monitor: non-finite FP64 sum (run diverged)");
    return EUP_OK;
}

int eup_get_line(eup_handle* h, int32_t axis, int32_t c1, int32_t c2, double* out) {
    int rc = check_handle(h);
    if (rc) return rc;
    const Geo& g = h->g;
    if (!out || axis < 0 || axis > 2) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_line: bad axis or null out");
    const int e1 = axis == 0 ? g.m : g.l, e2 = axis == 2 ? g.m : g.n;
    if (c1 < 1 || c1 > e1 || c2 < 1 || c2 > e2)
        return fail(h, EUP_ERR_INVALID_ARG, "eup_get_line: line outside the interior");
    if (!h->has_state) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_line: no state uploaded");
    const int len = axis == 0 ? g.l : (axis == 1 ? g.m : g.n);
    if ((rc = ensure_staging(h, sizeof(double) * 4 * (size_t)len))) return rc;
    DISPATCH(h, line_dispatch, h, axis, c1, c2, static_cast<double*>(h->staging));
    CK(h, cudaGetLastError());
    CK(h, cudaMemcpyAsync(out, h->staging, sizeof(double) * 4 * (size_t)len, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return EUP_OK;
}

int eup_get_plane_means(eup_handle* h, int32_t axis, double* out) {
    int rc = check_handle(h);
    if (rc) return rc;
    const Geo& g = h->g;
    if (!out || axis < 0 || axis > 2) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_plane_means: bad axis or null out");
    if (!h->has_state) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_plane_means: no state uploaded");
    const int len = axis == 0 ? g.l : (axis == 1 ? g.m : g.n);
    if ((rc = ensure_staging(h, sizeof(double) * 4 * (size_t)len))) return rc;
    DISPATCH(h, plane_dispatch, h, axis, static_cast<double*>(h->staging));
    CK(h, cudaGetLastError());
    CK(h, cudaMemcpyAsync(out, h->staging, sizeof(double) * 4 * (size_t)len, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return EUP_OK;
}

int eup_get_cv_drag(eup_handle* h, const int32_t box[6], double out[2]) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!box || !out) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_cv_drag: null argument");
    if (!h->has_state) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_cv_drag: no state uploaded");
    // clipping and face weights of CODE/SRC/flux_X.F90:56-156 with the serial offsets 0
    const int ext[3] = {h->g.l, h->g.m, h->g.n};
    int lo[3], hi[3], w[3][2];
    out[0] = out[1] = 0.0;
    for (int d = 0; d < 3; ++d) {
        const int s0 = box[2 * d], s1 = box[2 * d + 1];
        if (s0 > s1) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_cv_drag: box start after stop");
        w[d][0] = w[d][1] = 1;
        if (s0 > ext[d] || s1 < 0) return EUP_OK;  // box misses the lattice
        if (s0 > 0 && s1 <= ext[d]) { lo[d] = s0; hi[d] = s1; }
        else if (s0 > 0) { lo[d] = s0; hi[d] = ext[d]; w[d][1] = 0; }
        else if (s1 <= ext[d]) { lo[d] = 1; hi[d] = s1; w[d][0] = 0; }
        else return EUP_OK;  // box around the whole lattice: no face inside
    }
    const int clipped[6] = {lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]};
    DISPATCH(h, cv_dispatch, h, clipped);
    CK(h, cudaGetLastError());
    double f[4];
    CK(h, cudaMemcpyAsync(f, h->dscratch, sizeof(double) * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    out[0] = -f[0] * w[0][0] + f[1] * w[0][1];
    out[1] = f[2] * w[1][0] + f[3] * w[1][1];
    return EUP_OK;
}

int eup_get_region_sums(eup_handle* h, const uint8_t* region, double out[6]) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!region || !out) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_region_sums: null argument");
    if (!h->has_state) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_region_sums: no state uploaded");
    uint8_t* d_region = nullptr;
    CK(h, cudaMalloc(&d_region, (size_t)h->g.N));
    cudaError_t e = cudaMemcpyAsync(d_region, region, (size_t)h->g.N, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        DISPATCH(h, region_dispatch, h, d_region);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, h->dscratch, sizeof(double) * 6, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(d_region);
    if (e != cudaSuccess) return cuda_fail(h, e, "eup_get_region_sums");
    for (int c = 0; c < 6; ++c)
        if (!std::isfinite(out[c])) return fail(h, EUP_ERR_DIVERGED, "eup_get_region_sums: non-finite FP64 sum");
    return EUP_OK;
}

int eup_get_probes(eup_handle* h, int32_t npts, const int32_t* ijk, double* rho_u) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (npts < 0 || (npts > 0 && (!ijk || !rho_u))) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_probes: bad argument");
    if (!h->has_state) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_probes: no state uploaded");
    for (int32_t p = 0; p < npts; ++p)
        if (!h->g.interior(ijk[3 * p], ijk[3 * p + 1], ijk[3 * p + 2]))
            return fail(h, EUP_ERR_INVALID_ARG, "eup_get_probes: probe outside the interior");
    if (npts == 0) return EUP_OK;
    int32_t* d_ijk = nullptr;
    double* d_out = nullptr;
    CK(h, cudaMalloc(&d_ijk, sizeof(int32_t) * 3 * npts));
    CK(h, cudaMalloc(&d_out, sizeof(double) * 4 * npts));
    CK(h, cudaMemcpyAsync(d_ijk, ijk, sizeof(int32_t) * 3 * npts, cudaMemcpyHostToDevice, h->stream));
    DISPATCH(h, probes_dispatch, h, npts, d_ijk, d_out);
    cudaMemcpyAsync(rho_u, d_out, sizeof(double) * 4 * npts, cudaMemcpyDeviceToHost, h->stream);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    cudaFree(d_ijk);
    cudaFree(d_out);
    if (e != cudaSuccess) return cuda_fail(h, e, "eup_get_probes");
    return EUP_OK;
}

int eup_get_links(eup_handle* h, uint32_t* links) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!links) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_links: null out");
    uint32_t* d = nullptr;
    CK(h, cudaMalloc(&d, sizeof(uint32_t) * h->g.N));
    launch_links(h->g, make_mask(h), d, h->stream);
    cudaMemcpyAsync(links, d, sizeof(uint32_t) * h->g.N, cudaMemcpyDeviceToHost, h->stream);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(h, e, "eup_get_links");
    return EUP_OK;
}

int eup_get_boundary_solid(eup_handle* h, int64_t* list, int64_t cap, int64_t* count) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!count || cap < 0 || (cap > 0 && !list)) return fail(h, EUP_ERR_INVALID_ARG, "eup_get_boundary_solid: bad argument");
    *count = h->nblist;
    const int64_t n = std::min(cap, h->nblist);
    if (n > 0) {
        std::vector<int32_t> tmp((size_t)n);
        CK(h, cudaMemcpy(tmp.data(), h->blist, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
        for (int64_t t = 0; t < n; ++t) list[t] = tmp[(size_t)t];
    }
    return EUP_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Partial bounce-back and the checkpointed discrete adjoint
// ---------------------------------------------------------------------------
namespace {

template <typename T>
struct DevBuf {
    T* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, sizeof(T) * (n > 0 ? n : 1)); }
};

template <typename T>
cudaError_t upload_vec(DevBuf<T>& b, const std::vector<T>& v) {
    cudaError_t e = b.alloc(v.size());
    if (e == cudaSuccess && !v.empty()) e = cudaMemcpy(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice);
    return e;
}

// Lattice view of an arbitrary state buffer laid out like the handle's lattices.
template <typename S, typename R>
Lat<S, R> lat_at(const eup_handle* h, S* base, R* shell = nullptr) {
    Lat<S, R> L = make_lat<S, R>(h, 0);
    for (int q = 0; q < Q; ++q) L.pop[q] = pop_ptr<S>(h, base, q);
    if (shell) L.ghost = shell;
    return L;
}

// ---- binomial checkpointing ---------------------------------------------------------
// Reversing n steps from a stored state with c snapshot slots (the stored state's own
// included) needs at least t(n, c) = r n - C(c + r, r - 1) forward steps, r the smallest
// repetition number with C(c + r, c) >= n (t = 0 for n <= 1, n(n-1)/2 for c = 1):
// A. Griewank, "Achieving logarithmic growth of temporal and spatial complexity in reverse
// automatic differentiation", Optim. Methods Softw. 1 (1992); A. Griewank and A. Walther,
// ACM TOMS 26 (2000), "revolve".  The schedule below splits each range at the step that
// minimises m + t(m, c) + t(n - m, c - 1) (scanned with the closed form), which attains
// t(n, c).

// C(a, b), saturating far above any step count
int64_t binom_sat(int64_t a, int64_t b) {
    if (b < 0 || b > a) return 0;
    if (b > a - b) b = a - b;
    const int64_t cap = (int64_t)1 << 50;
    int64_t v = 1;
    for (int64_t i = 1; i <= b; ++i) {
        v = v * (a - b + i) / i;  // exact: the product of i consecutive integers divides by i!
        if (v > cap) return cap;
    }
    return v;
}

int64_t revolve_cost(int64_t n, int64_t c) {
    if (n <= 1) return 0;
    if (c <= 1) return n * (n - 1) / 2;
    int64_t r = 0;
    while (binom_sat(c + r, c) < n) ++r;
    return r * n - binom_sat(c + r, r - 1);
}

// smallest r with C(c + r, c) >= n
int revolve_repetition(int64_t n, int64_t c) {
    if (n <= 1) return 0;
    if (c <= 1) return (int)(n - 1);
    int r = 0;
    while (binom_sat(c + r, c) < n) ++r;
    return r;
}

enum : int { kActAdvance = 0, kActSnapshot = 1, kActRestore = 2, kActAdjoint = 3 };

// CUDA graphs of the launch sequences an adjoint run repeats (a forward step between two given
// buffers, an adjoint step from a given buffer), captured the first time a key is met and
// launched from then on: a reverse sweep uses a few hundred distinct sequences thousands of
// times.  With use == false the sequence is launched directly.
struct GraphCache {
    std::unordered_map<uint64_t, cudaGraphExec_t> exec;
    ~GraphCache() {
        for (auto& kv : exec) cudaGraphExecDestroy(kv.second);
    }
    // Captures (on st, which may hold pending work) and instantiates the sequence of key.
    template <typename F>
    cudaError_t prepare(uint64_t key, cudaStream_t st, F&& enqueue) {
        if (exec.count(key)) return cudaSuccess;
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        enqueue();
        e = cudaStreamEndCapture(st, &graph);
        if (e != cudaSuccess) return e;
        cudaGraphExec_t ge = nullptr;
        // kernels keep the priority of the stream they were captured from
        e = cudaGraphInstantiate(&ge, graph, cudaGraphInstantiateFlagUseNodePriority);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return e;
        exec.emplace(key, ge);
        return cudaSuccess;
    }
    template <typename F>
    cudaError_t run(uint64_t key, cudaStream_t st, bool use, F&& enqueue) {
        if (!use) {
            enqueue();
            return cudaGetLastError();
        }
        const cudaError_t e = prepare(key, st, enqueue);
        if (e != cudaSuccess) return e;
        return cudaGraphLaunch(exec.find(key)->second, st);
    }
};
struct RevAct {
    int kind, arg;  // advance: steps; snapshot/restore: slot; adjoint: the step t reversed (from state t-1)
};

// A high-priority second stream and two events: an adjoint step forks its boundary part
// (halo kernels, boundary-plane nodes, halo transposes) onto it, beside the interior kernel.
struct SideStream {
    cudaStream_t s = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    SideStream() = default;
    SideStream(const SideStream&) = delete;
    SideStream& operator=(const SideStream&) = delete;
    ~SideStream() {
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
        if (s) cudaStreamDestroy(s);
    }
    cudaError_t create() {
        int least = 0, greatest = 0;
        cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
        if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, greatest);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join, cudaEventDisableTiming);
        return e;
    }
};

// Reverse steps a+1 .. b with the working state at a (also held in slot_a) and `free` slots.
void revolve_schedule(int a, int b, int slot_a, std::vector<int>& free, std::vector<RevAct>& acts) {
    const int n = b - a;
    if (n == 1) {
        acts.push_back({kActAdjoint, b});
        return;
    }
    if (free.empty()) {  // no slot left: recompute from a for every step
        for (int t = b; t > a; --t) {
            if (t != b) acts.push_back({kActRestore, slot_a});
            if (t - 1 - a > 0) acts.push_back({kActAdvance, t - 1 - a});
            acts.push_back({kActAdjoint, t});
        }
        return;
    }
    const int64_t c = (int64_t)free.size() + 1;
    int best_m = 1;
    int64_t best = -1;
    for (int m = 1; m < n; ++m) {
        const int64_t v = m + revolve_cost(m, c) + revolve_cost(n - m, c - 1);
        if (best < 0 || v < best) {
            best = v;
            best_m = m;
        }
    }
    const int k = free.back();
    free.pop_back();
    acts.push_back({kActAdvance, best_m});
    acts.push_back({kActSnapshot, k});
    revolve_schedule(a + best_m, b, k, free, acts);
    free.push_back(k);
    acts.push_back({kActRestore, slot_a});
    revolve_schedule(a, a + best_m, slot_a, free, acts);
}

// T partial-bounce-back steps forward, then the adjoint back, with `slots` stored states
// (binomial checkpointing).  The plain forward sweep on the handle's own lattices records
// every step's force and, as it passes them, copies the states the schedule stores on its
// first descent (state 0 included) into their slots and state T-1 into the working
// buffer; the rest of the schedule then runs on two working buffers: restores, forward
// steps without force, stores, and adjoint steps in the order T, T-1, ..., 1.  Before each
// forward or adjoint step the halo blocks run on the working state (its halo follows from
// it: configurations whose halo holds older values are refused), writing a working halo
// shell that starts as a copy of the handle's (its never-written slots are constant).
template <typename S, typename R>
int adjoint_run(eup_handle* h, const eup_adjoint_config* ac, double* objective, double* grad_out, double* stats) {
    const Geo& g = h->g;
    const int T = ac->nsteps, A = ac->avg_steps;
    int slots = ac->checkpoints > 0 ? ac->checkpoints : 64;
    if (slots > T) slots = T;
    const int bc[6] = {h->cfg.bc[0], h->cfg.bc[1], h->cfg.bc[2], h->cfg.bc[3], h->cfg.bc[4], h->cfg.bc[5]};
    const double norm = 0.5 * h->cfg.cd_rho0 * h->cfg.cd_uref * h->cfg.cd_uref * h->cfg.cd_length * h->cfg.cd_span;
    const double gamma = 1.0 / ((double)A * norm);
    const Phys<R> ph = make_phys<R>(h);
    const R* ns = static_cast<const R*>(h->ns);
    cudaStream_t st = h->stream;
    // EUP_STEP_VARIANT bit 18: every adjoint step in one stream (the reference order of its
    // kernels, against which the forked step is tested bit for bit)
    const bool serial = (h->variant & 262144) != 0;
    SideStream side;
    if (!serial) CK(h, side.create());

    HaloAdjointTables tab;
    std::string why;
    if (build_halo_adjoint_tables(g, bc, &tab, &why) != EUP_OK) return fail(h, EUP_ERR_UNSUPPORTED, "eup_adjoint_run: " + why);
    DevBuf<int64_t> d_ckey, d_cslot, d_oslot;
    DevBuf<int32_t> d_cstart, d_ojk, d_ostart;
    DevBuf<int8_t> d_oq;
    CK(h, upload_vec(d_ckey, tab.copy_key));
    CK(h, upload_vec(d_cstart, tab.copy_start));
    CK(h, upload_vec(d_cslot, tab.copy_slot));
    CK(h, upload_vec(d_ojk, tab.out_jk));
    CK(h, upload_vec(d_ostart, tab.out_start));
    CK(h, upload_vec(d_oslot, tab.out_slot));
    CK(h, upload_vec(d_oq, tab.out_q));
    HaloAdjointDevice td;
    td.copy_key = d_ckey.p; td.copy_start = d_cstart.p; td.copy_slot = d_cslot.p; td.ncopy = (int64_t)tab.copy_key.size();
    td.out_jk = d_ojk.p; td.out_start = d_ostart.p; td.out_slot = d_oslot.p; td.out_q = d_oq.p;
    td.nout = (int64_t)tab.out_jk.size();

    // the schedule, and the states its first descent stores
    std::vector<RevAct> acts;
    {
        std::vector<int> free;
        for (int k = slots - 1; k >= 1; --k) free.push_back(k);
        acts.push_back({kActSnapshot, 0});
        revolve_schedule(0, T, 0, free, acts);
    }
    std::vector<int> store_at((size_t)T, -1);  // forward-sweep state -> slot
    size_t first_adj = 0;
    {
        int state = 0;
        for (; first_adj < acts.size() && acts[first_adj].kind != kActAdjoint; ++first_adj) {
            if (acts[first_adj].kind == kActAdvance) state += acts[first_adj].arg;
            else if (acts[first_adj].kind == kActSnapshot) store_at[(size_t)state] = acts[first_adj].arg;
        }
        if (state != T - 1) return fail(h, EUP_ERR_INVALID_ARG, "eup_adjoint_run: internal schedule error");
    }

    // state buffers: the slots, then two working buffers; each with its own x-face copy
    // (the columns x = 1 and x = l the halo blocks read), so a state is never copied to be
    // read: a restore only makes a slot the working state, and the forward step that ends
    // where the schedule stores a state writes it into the slot directly
    const size_t state = (size_t)Q * h->Nq;
    const size_t shell = (size_t)Q * g.G;
    const size_t xfs = (size_t)xface_elems(g);
    const int nbuf = slots + 2;
    DevBuf<S> bufs;
    DevBuf<R> xfaces, lam, gmu, wshell;
    DevBuf<double> grad;
    CK(h, bufs.alloc(state * nbuf));
    CK(h, xfaces.alloc(xfs * nbuf));
    CK(h, lam.alloc(state * 2));
    CK(h, gmu.alloc(shell));
    CK(h, wshell.alloc(shell));
    CK(h, grad.alloc(g.N));
    CK(h, cudaMemsetAsync(grad.p, 0, sizeof(double) * g.N, st));
    CK(h, cudaMemsetAsync(lam.p, 0, sizeof(R) * state * 2, st));
    const Reduce red = make_reduce(h);
    auto buf_lat = [&](int b) {
        Lat<S, R> L = lat_at<S, R>(h, bufs.p + state * b, wshell.p);
        L.xface = xfaces.p + xfs * b;
        return L;
    };
    auto keep = [&](int b) -> cudaError_t {  // the handle's current state (and x-face copy) into buffer b
        cudaError_t e = cudaMemcpyAsync(bufs.p + state * b, h->lat[h->cur], sizeof(S) * state,
                                        cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(xfaces.p + xfs * b, h->xface, sizeof(R) * xfs, cudaMemcpyDeviceToDevice, st);
        return e;
    };

    cudaEvent_t ev[3];
    for (auto& e : ev) CK(h, cudaEventCreate(&e));
    // ---- forward sweep (the handle's own state, force series recorded) ----
    const int64_t t0 = h->itime;
    const int w0 = slots, w1 = slots + 1;  // the working buffers
    // every step as a CUDA graph (EUP_STEP_VARIANT bit 1: plain launches): the forward sweep
    // uses the handle's own step graphs, the reverse sweep the cache below
    const bool graphs = !(h->variant & 2);
    int per_step = 0;
    if (graphs) {
        const cudaError_t e_cap = capture_graphs<S, R>(h, &per_step);
        CK(h, e_cap);
    }
    GraphCache cache;
    CK(h, cudaEventRecord(ev[0], st));
    for (int s = 0; s < T; ++s) {
        if (store_at[(size_t)s] >= 0) CK(h, keep(store_at[(size_t)s]));
        if (s == T - 1) CK(h, keep(w0));
        if (graphs) {
            CK(h, cudaGraphLaunch(h->graph[h->cur], st));
        } else {
            const Lat<S, R> src = make_lat<S, R>(h, h->cur), dst = make_lat<S, R>(h, h->cur ^ 1);
            launch_bc<S, R>(src, g, bc, ph, st, bc_bar(h));
            launch_pbb_step<S, R>(src, dst, g, ph, ns, h->ns_list, h->ns_count, red, h->series, h->cap, h->d_itime,
                                  st);
        }
        h->cur ^= 1;
        h->itime += 1;
    }
    CK(h, cudaMemcpyAsync(wshell.p, h->ghost, sizeof(R) * shell, cudaMemcpyDeviceToDevice, st));
    CK(h, cudaEventRecord(ev[1], st));
    CK(h, cudaGetLastError());

    // ---- reverse sweep: the rest of the schedule ----
    // Walked twice: first without launching, capturing and instantiating every distinct step
    // graph while the device still runs the forward sweep, then enqueueing the steps behind it.
    // The sweep needs nothing from the host's reading of the objective, which comes after.
    int64_t recomputed = 0;
    auto reverse = [&](bool dry) -> int {
        int cur = w0;           // buffer holding the working state (state T-1 now)
        int cur_lam = 0;        // lam[cur_lam] = adjoint of the state after the step being reversed
        auto step = [&](uint64_t key, auto&& enqueue) -> cudaError_t {
            if (!dry) return cache.run(key, st, graphs, enqueue);
            return graphs ? cache.prepare(key, st, enqueue) : cudaSuccess;
        };
        for (size_t a = first_adj; a < acts.size(); ++a) {
            const RevAct act = acts[a];
            if (act.kind == kActAdvance) {
                // the last step goes straight into the slot the next action stores
                const int target =
                    (a + 1 < acts.size() && acts[a + 1].kind == kActSnapshot) ? acts[a + 1].arg : -1;
                for (int s = 0; s < act.arg; ++s) {
                    const int next = (s + 1 == act.arg && target >= 0) ? target : (cur == w0 ? w1 : w0);
                    const Lat<S, R> src = buf_lat(cur), dst = buf_lat(next);
                    const uint64_t key = ((uint64_t)1 << 60) | ((uint64_t)cur << 24) | (uint64_t)next;
                    const cudaError_t e_run = step(key, [&] {
                        launch_bc<S, R>(src, g, bc, ph, st, bc_bar(h));
                        launch_pbb_step<S, R>(src, dst, g, ph, ns, h->ns_list, h->ns_count, red, nullptr, 0, nullptr,
                                              st);
                    });
                    CK(h, e_run);
                    cur = next;
                    if (!dry) ++recomputed;
                }
                if (target >= 0) ++a;  // the store is done
            } else if (act.kind == kActSnapshot) {
                if (cur != act.arg) {  // not reached in these schedules: a store always follows a forward step
                    if (!dry) {
                        CK(h, cudaMemcpyAsync(bufs.p + state * act.arg, bufs.p + state * cur, sizeof(S) * state,
                                              cudaMemcpyDeviceToDevice, st));
                        CK(h, cudaMemcpyAsync(xfaces.p + xfs * act.arg, xfaces.p + xfs * cur, sizeof(R) * xfs,
                                              cudaMemcpyDeviceToDevice, st));
                    }
                    cur = act.arg;
                }
            } else if (act.kind == kActRestore) {
                cur = act.arg;  // read in place; forward steps write elsewhere
            } else {  // adjoint of step t from state t-1
                const int t = act.arg;
                const Lat<S, R> f = buf_lat(cur);
                const Lat<R, R> lin_ = lat_at<R, R>(h, lam.p + state * cur_lam),
                                lout = lat_at<R, R>(h, lam.p + state * (cur_lam ^ 1));
                const bool in_window = t > T - A;
                const R gam = in_window ? (R)gamma : R(0);
                const uint64_t key = ((uint64_t)2 << 60) | ((uint64_t)cur << 24) | ((uint64_t)cur_lam << 1) |
                                     (uint64_t)in_window;
                const cudaError_t e_run = step(key, [&] {
                    if (serial) {
                        launch_bc<S, R>(f, g, bc, ph, st, bc_bar(h));  // the halo of step t, from state t-1
                        launch_pbb_adjoint<S, R>(f, g, ph, ns, lin_, lout, gmu.p, grad.p, gam, td, st, kAdjAll);
                        return;
                    }
                    // the interior nodes read no halo value and write other slots than the
                    // boundary-plane nodes: the halo of step t (from state t-1) and the boundary-plane
                    // nodes run on the side stream beside them; the halo transposes after both
                    cudaEventRecord(side.fork, st);
                    cudaStreamWaitEvent(side.s, side.fork, 0);
                    launch_bc<S, R>(f, g, bc, ph, side.s, bc_bar(h));
                    launch_pbb_adjoint<S, R>(f, g, ph, ns, lin_, lout, gmu.p, grad.p, gam, td, side.s, kAdjFaces);
                    cudaEventRecord(side.join, side.s);
                    launch_pbb_adjoint<S, R>(f, g, ph, ns, lin_, lout, gmu.p, grad.p, gam, td, st, kAdjInterior);
                    cudaStreamWaitEvent(st, side.join, 0);
                    launch_pbb_adjoint<S, R>(f, g, ph, ns, lin_, lout, gmu.p, grad.p, gam, td, st, kAdjTransposes);
                });
                CK(h, e_run);
                cur_lam ^= 1;
            }
        }
        return EUP_OK;
    };
    int rc = reverse(true);
    if (rc == EUP_OK) rc = reverse(false);
    if (rc != EUP_OK) {
        cudaStreamSynchronize(st);
        return rc;
    }
    CK(h, cudaEventRecord(ev[2], st));
    CK(h, cudaGetLastError());
    CK(h, cudaMemcpyAsync(grad_out, grad.p, sizeof(double) * g.N, cudaMemcpyDeviceToHost, st));
    // objective: mean C_d over the last A steps (steps T-A+1 .. T), from the series the forward
    // sweep recorded (the reverse sweep records none): at most two runs of the ring buffer
    // (A <= its capacity, checked on entry)
    std::vector<double> fser((size_t)3 * A);
    {
        const int64_t first = (t0 + T - A + 1) % h->cap;
        const int64_t n1 = std::min<int64_t>(A, h->cap - first);
        CK(h, cudaMemcpyAsync(fser.data(), h->series + 3 * first, sizeof(double) * 3 * n1, cudaMemcpyDeviceToHost,
                              st));
        if (n1 < A)
            CK(h, cudaMemcpyAsync(fser.data() + 3 * n1, h->series, sizeof(double) * 3 * (A - n1),
                                  cudaMemcpyDeviceToHost, st));
    }
    CK(h, cudaStreamSynchronize(st));
    double J = 0.0;
    for (int s = 0; s < A; ++s) J += fser[3 * (size_t)s];
    J *= gamma;
    if (!std::isfinite(J)) return fail(h, EUP_ERR_DIVERGED, "eup_adjoint_run: forward run diverged");
    float fwd_ms = 0.f, rev_ms = 0.f;
    cudaEventElapsedTime(&fwd_ms, ev[0], ev[1]);
    cudaEventElapsedTime(&rev_ms, ev[1], ev[2]);
    for (auto& e : ev) cudaEventDestroy(e);
    *objective = J;
    if (stats) {
        stats[0] = fwd_ms;
        stats[1] = rev_ms;
        stats[2] = (double)recomputed;
        stats[3] = slots;
        stats[4] = revolve_repetition(T, slots);
        stats[5] = (double)(sizeof(S) * state * (size_t)nbuf + sizeof(R) * (xfs * (size_t)nbuf + state * 2 + shell * 2));
        stats[6] = T;
        stats[7] = A;
    }
    return EUP_OK;
}

}  // namespace

extern "C" {

int eup_set_solid_fraction(eup_handle* h, const double* ns) {
    int rc = check_handle(h);
    if (rc) return rc;
    CK(h, cudaStreamSynchronize(h->stream));
    drop_graphs(h);
    if (!ns) {
        if (h->ns) cudaFree(h->ns);
        if (h->ns_list) cudaFree(h->ns_list);
        h->ns = nullptr;
        h->ns_list = nullptr;
        h->ns_count = 0;
        h->pbb = false;
        return EUP_OK;
    }
    if (has_exchange_face(h))
        return fail(h, EUP_ERR_UNSUPPORTED, "eup_set_solid_fraction: not offered on an x-slab lattice");
    if (h->nblist > 0 || h->bits)
        return fail(h, EUP_ERR_UNSUPPORTED,
                    "eup_set_solid_fraction: obstacles are set; fold them into the field as n_s = 1 instead");
    const int64_t N = h->g.N;
    for (int64_t t = 0; t < N; ++t)
        if (!(ns[t] >= 0.0 && ns[t] <= 1.0))
            return fail(h, EUP_ERR_INVALID_ARG, "eup_set_solid_fraction: n_s outside [0,1] at index " + std::to_string(t));
    // the voxels the solid takes momentum from (n_s > 0 in the arithmetic type)
    std::vector<int32_t> list;
    for (int64_t t = 0; t < N; ++t)
        if ((h->prec == EUP_FP64 ? ns[t] : (double)(float)ns[t]) > 0.0) list.push_back((int32_t)t);
    if (!h->ns) CK(h, cudaMalloc(&h->ns, h->rbytes * N));
    if (h->ns_list) cudaFree(h->ns_list);
    h->ns_list = nullptr;
    h->ns_count = 0;
    CK(h, cudaMalloc(&h->ns_list, sizeof(int32_t) * (list.empty() ? 1 : list.size())));
    if (!list.empty())
        CK(h, cudaMemcpy(h->ns_list, list.data(), sizeof(int32_t) * list.size(), cudaMemcpyHostToDevice));
    h->ns_count = (int64_t)list.size();
    if (h->prec == EUP_FP64) {
        CK(h, cudaMemcpy(h->ns, ns, sizeof(double) * N, cudaMemcpyHostToDevice));
    } else {
        std::vector<float> tmp((size_t)N);
        for (int64_t t = 0; t < N; ++t) tmp[(size_t)t] = (float)ns[t];
        CK(h, cudaMemcpy(h->ns, tmp.data(), sizeof(float) * N, cudaMemcpyHostToDevice));
    }
    h->pbb = true;
    return EUP_OK;
}

int eup_adjoint_plan(int32_t nsteps, int32_t checkpoints, int64_t* forward_steps, int64_t* recomputed,
                     int32_t* repetitions) {
    if (nsteps < 1 || checkpoints < 0 || !forward_steps || !recomputed || !repetitions)
        return fail(nullptr, EUP_ERR_INVALID_ARG, "eup_adjoint_plan: need nsteps >= 1, checkpoints >= 0 and outputs");
    int slots = checkpoints > 0 ? checkpoints : 64;
    if (slots > nsteps) slots = nsteps;
    std::vector<RevAct> acts;
    std::vector<int> free;
    for (int k = slots - 1; k >= 1; --k) free.push_back(k);
    acts.push_back({kActSnapshot, 0});
    revolve_schedule(0, nsteps, 0, free, acts);
    int64_t total = 0, sweep = 0;
    bool reversing = false;
    for (const RevAct& a : acts) {
        if (a.kind == kActAdjoint) reversing = true;
        if (a.kind == kActAdvance) (reversing ? total : sweep) += a.arg;
    }
    *forward_steps = sweep + total;          // t(T, c): the first descent plus the recomputation
    *recomputed = total;                     // what the reverse sweep recomputes (eup_adjoint_run's stats[2])
    *repetitions = revolve_repetition(nsteps, slots);
    return EUP_OK;
}

int eup_adjoint_run(eup_handle* h, const eup_adjoint_config* cfg, double* objective, double* grad_ns,
                    double stats[8]) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!cfg || !objective || !grad_ns) return fail(h, EUP_ERR_INVALID_ARG, "eup_adjoint_run: null argument");
    if (!h->pbb) return fail(h, EUP_ERR_INVALID_ARG, "eup_adjoint_run: no solid-fraction field set");
    if (!h->has_state) return fail(h, EUP_ERR_INVALID_ARG, "eup_adjoint_run: no state uploaded");
    if (cfg->nsteps < 1 || cfg->avg_steps < 1 || cfg->avg_steps > cfg->nsteps || cfg->checkpoints < 0)
        return fail(h, EUP_ERR_INVALID_ARG, "eup_adjoint_run: need 1 <= avg_steps <= nsteps, checkpoints >= 0");
    if (!(h->cfg.cd_rho0 > 0 && h->cfg.cd_uref != 0 && h->cfg.cd_length > 0 && h->cfg.cd_span > 0))
        return fail(h, EUP_ERR_INVALID_ARG, "eup_adjoint_run: drag normalisation not set in eup_config");
    if (cfg->avg_steps > h->cap)
        return fail(h, EUP_ERR_INVALID_ARG, "eup_adjoint_run: avg_steps exceeds the force history capacity");
    switch (h->prec) {
        case EUP_FP64: return adjoint_run<double, double>(h, cfg, objective, grad_ns, stats);
        case EUP_FP16_DEV: return adjoint_run<__half, float>(h, cfg, objective, grad_ns, stats);
        case EUP_BF16_DEV: return adjoint_run<__nv_bfloat16, float>(h, cfg, objective, grad_ns, stats);
        default: return adjoint_run<float, float>(h, cfg, objective, grad_ns, stats);
    }
}

}  // extern "C"
