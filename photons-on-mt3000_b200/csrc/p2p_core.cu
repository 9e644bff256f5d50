// libphotons_p2p: host side of the B200 P2P pass and its C ABI
// (include/photons_p2p.h). See p2p_kernels.cuh for the device code.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <tuple>
#include <string>
#include <vector>

#include "photons_p2p.h"
#include "p2p_internal.h"
#include "p2p_fit.h"
#include "p2p_args.h"
#include "p2p_launch.h"
#include "p2p_host_shared.h"
#include "p2p_pass_kernels.cuh"
#include "p2p_walk_kernels.cuh"

namespace p2p {
#include "p2p_csr.h"
}  // namespace p2p

#define P2P_API extern "C" __attribute__((visibility("default")))

namespace p2p {
namespace {

thread_local std::string g_last_error;
std::atomic<int64_t> g_launches{0};

int fail(int status, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return status;
}

#define CUDA_TRY(expr)                                                                   \
    do {                                                                                 \
        cudaError_t _e = (expr);                                                         \
        if (_e != cudaSuccess)                                                           \
            return fail(P2P_ERR_CUDA, "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e), \
                        __FILE__, __LINE__);                                             \
    } while (0)

#define P2P_TRY(expr)              \
    do {                           \
        int _s = (expr);           \
        if (_s != P2P_OK) return _s; \
    } while (0)

// Grow-only device buffer.
struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
};

}  // namespace
}  // namespace p2p

using namespace p2p;

struct p2p_session {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_begin = nullptr, ev_end = nullptr, ev_k0 = nullptr, ev_k1 = nullptr;
    // pipelined host submits: list pieces uploaded on copy_stream into two
    // buffer pairs while the previous piece computes on stream
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t piece_ready[2] = {nullptr, nullptr}, piece_free[2] = {nullptr, nullptr};
    bool kernel_timed = false;
    bool dry_run = false;  // dispatch without launching (fills the occupancy cache)
    int last_blocks = 0;
    std::map<std::tuple<const void *, int, size_t>, int> occupancy;
    p2p_params params{};
    PolyFit fit;
    // device buffers
    DevBuf task_t2, task_s2;  // second buffer pair of pipelined submits
    DevBuf pos, mass, leaf_ip, leaf_np, task_t, task_s, meta, pos4, counts, fill, row_off,
        row_src, tile_sums, acc, status, queue, pairs, skipped, evaluated, probe;
    DevBuf keys_a, keys_b, vals_b, hist, hoffs, hsums;  // radix sort of the list
    std::vector<DevBuf> scratch;  // grow-only temporaries of p2p_dtree_build, by request order
    DevBuf walk_slab;             // the walk's first pass keeps short rows here (p2p_pass_submit_walk)
    // pass state
    bool in_pass = false;
    int npart = 0, nleaf = 0;
    // particles whose host positions the pos buffer holds from the last
    // p2p_pass_begin / p2p_pass_begin_update (-1: none); p2p_pass_begin_update
    // uploads only the changed chunks over them
    int pos_held = -1;
    const double *d_pos = nullptr, *d_mass = nullptr;
    const int *d_ip = nullptr, *d_np = nullptr;
    // graph cache for p2p_pass_run_device
    cudaGraphExec_t gexec = nullptr;
    int graph_kernels = 0;
    struct Key {
        const void *p[6];
        int64_t n[3];
        int version;
    } gkey{};
    int version = 0;
};

namespace {

int ensure(p2p_session *s, DevBuf &b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.cap >= bytes) return P2P_OK;
    size_t want = std::max(bytes + bytes / 4, (size_t)256);
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (b.p) CUDA_TRY(cudaFree(b.p));
    b.p = nullptr;
    b.cap = 0;
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        return fail(P2P_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
    }
    b.cap = want;
    if (s->gexec) {  // cached graph refers to the old buffer
        cudaGraphExecDestroy(s->gexec);
        s->gexec = nullptr;
    }
    return P2P_OK;
}

bool is_fp32_form(int form) { return form != P2P_FORM_PLAIN_FP64; }

// The device walk's slab of short rows: up to kWalkSlabMax ids per leaf (a
// power of two, halved down to kWalkSlabMin while it exceeds kWalkSlabBytes).
constexpr int kWalkSlabMax = 2048;
constexpr int kWalkSlabMin = 64;
constexpr size_t kWalkSlabBytes = (size_t)8 << 30;

// Host list submits longer than 2 * kPipePieceMin entries are uploaded and
// computed in about kPipePieces pieces of at least kPipePieceMin entries.
constexpr int64_t kPipePieceMin = (int64_t)1 << 25;
constexpr int64_t kPipePieces = 8;

int validate_params(const p2p_params *p) {
    if (p->form < P2P_FORM_PLAIN_FP64 || p->form > P2P_FORM_KAHAN_FP32)
        return fail(P2P_ERR_ARG, "unknown form %d", p->form);
    if (p->soft_mode != P2P_SOFT_CLAMP && p->soft_mode != P2P_SOFT_PLUMMER)
        return fail(P2P_ERR_ARG, "unknown soft_mode %d", p->soft_mode);
    if (!(p->soften > 0.0) || !std::isfinite(p->soften))
        return fail(P2P_ERR_ARG, "soften must be positive and finite");
    if (!(p->split_radius > 0.0) || !std::isfinite(p->split_radius))
        return fail(P2P_ERR_ARG, "split_radius must be positive and finite");
    if (!std::isfinite(p->x_cut) || !std::isfinite(p->mass))
        return fail(P2P_ERR_ARG, "x_cut and mass must be finite");
    if (!(p->poly_tol >= 0.0) || !std::isfinite(p->poly_tol))
        return fail(P2P_ERR_ARG, "poly_tol must be >= 0");
    if (p->warps_per_block < 0 || p->warps_per_block > 8)
        return fail(P2P_ERR_ARG, "warps_per_block must be in [0, 8]");
    if (p->stage_sources < 0 || p->stage_sources > 1024 || (p->stage_sources % 32))
        return fail(P2P_ERR_ARG, "stage_sources must be a multiple of 32 in [0, 1024]");
    if (p->blocks_per_sm < 0 || p->blocks_per_sm > 32)
        return fail(P2P_ERR_ARG, "blocks_per_sm must be in [0, 32]");
    if (p->warps_per_leaf != 0 && p->warps_per_leaf != 1 && p->warps_per_leaf != 2 && p->warps_per_leaf != 4)
        return fail(P2P_ERR_ARG, "warps_per_leaf must be 0, 1, 2 or 4");
    if (p->kernel_variant < P2P_VARIANT_AUTO || p->kernel_variant > P2P_VARIANT_SINK_REGS8)
        return fail(P2P_ERR_ARG, "unknown kernel_variant %d", p->kernel_variant);
    if (p->form != P2P_FORM_PLAIN_FP64 && p->kernel_variant != P2P_VARIANT_SINK_LANES &&
        p->warps_per_block > 4)
        return fail(P2P_ERR_ARG, "the source-lane kernel runs at most 4 warps per block");
    {
        const int w = p->warps_per_block ? p->warps_per_block : 4;
        const int st = p->stage_sources ? p->stage_sources : (p->form == P2P_FORM_PLAIN_FP64 ? 128 : 256);
        const size_t smem = p->form == P2P_FORM_PLAIN_FP64 ? pair_smem_plain(w, st)
                            : std::max(std::max(std::max(pair_smem_x2(w, st), pair_smem_sx2(w, st)),
                                                pair_smem_split(w, st, true)),
                                       pair_smem_sreg(w, st, 8));
        if (smem > (size_t)227 * 1024)
            return fail(P2P_ERR_ARG, "warps_per_block * stage_sources needs %zu B of shared memory (> 227 KB)", smem);
    }
    return P2P_OK;
}

int launch_count(int n) {
    g_launches += n;
    return P2P_OK;
}

bool source_lanes(const p2p_params &p) {
    return p.form != P2P_FORM_PLAIN_FP64 && p.kernel_variant != P2P_VARIANT_SINK_LANES;
}

bool packed_lanes(const p2p_params &p) {
    return p.form != P2P_FORM_PLAIN_FP64 &&
           (p.kernel_variant == P2P_VARIANT_SOURCE_LANES_X2 ||
            p.kernel_variant == P2P_VARIANT_SOURCE_LANES_X2_S16);
}

// Whether the pair kernel counts the pairs it evaluates on the device (the
// sink-register kernel, which also drops single source particles).
bool sink_regs(const p2p_params &p) {
    return is_fp32_form(p.form) &&
           (p.kernel_variant == P2P_VARIANT_SINK_REGS || p.kernel_variant == P2P_VARIANT_SINK_REGS8 ||
            p.kernel_variant == P2P_VARIANT_AUTO);
}
bool counts_evaluated(const p2p_params &p) { return sink_regs(p); }

int default_stage(const p2p_params &p) {
    return p.stage_sources ? p.stage_sources : (p.form == P2P_FORM_PLAIN_FP64 ? 128 : 256);
}

// Dispatch to the lane mapping's launcher (p2p_pair_*.cu).
int launch_pair(p2p_session *s, const PairArgs &a) {
    const p2p_params &p = s->params;
    PairLaunch L;
    L.stream = s->stream;
    L.sm_count = s->sm_count;
    L.soft_mode = p.soft_mode == P2P_SOFT_CLAMP ? SOFT_CLAMP : SOFT_PLUMMER;
    L.masses = a.mass != nullptr;
    L.acc = p.form == P2P_FORM_KAHAN_FP32 ? ACC_KAHAN : (p.form == P2P_FORM_NAIVE_FP32 ? ACC_F32 : ACC_F64);
    L.ncoef = s->fit.ncoef_kernel;
    L.warps = p.warps_per_block ? p.warps_per_block : 4;
    L.stage = default_stage(p);
    L.blocks_per_sm = p.blocks_per_sm;
    L.dry_run = s->dry_run;
    L.occ = &s->occupancy;
    L.sink_pairs = p.kernel_variant == P2P_VARIANT_SOURCE_LANES_X2_S16 ? 8 : 16;
    L.sreg_spl = p.kernel_variant == P2P_VARIANT_SINK_REGS8 ? 8 : 4;
    PairLaunchResult r;
    if (p.form == P2P_FORM_PLAIN_FP64)
        r = launch_pair_plain(L, a);
    else if (p.kernel_variant == P2P_VARIANT_SINK_LANES_X2)
        r = launch_pair_sink_lanes_x2(L, a);
    else if (sink_regs(p))
        r = launch_pair_sink_regs(L, a);
    else if (packed_lanes(p))
        r = launch_pair_source_lanes_x2(L, a);
    else if (source_lanes(p))
        r = launch_pair_source_lanes(L, a);
    else
        r = launch_pair_sink_lanes(L, a);
    if (!r.fits) return fail(P2P_ERR_ARG, "pair kernel does not fit on an SM with this launch shape");
    if (r.cuda != cudaSuccess)
        return fail(P2P_ERR_CUDA, "pair kernel launch: %s", cudaGetErrorString(r.cuda));
    if (s->dry_run) return P2P_OK;
    s->last_blocks = r.blocks;
    return launch_count(1);
}

cudaError_t allow_smem_all() {
    cudaError_t e = allow_smem_sink_lanes();
    if (e == cudaSuccess) e = allow_smem_source_lanes();
    if (e == cudaSuccess) e = allow_smem_source_lanes_x2();
    if (e == cudaSuccess) e = allow_smem_sink_lanes_x2();
    if (e == cudaSuccess) e = allow_smem_sink_regs();
    if (e == cudaSuccess) e = allow_smem_plain();
    return e;
}

int grid_for(int64_t n, int threads, int cap_blocks) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap_blocks) b = cap_blocks;
    return (int)b;
}

// Frame/coordinate preparation for the current pass inputs (stream-ordered).
int enqueue_prep(p2p_session *s) {
    const int nleaf = s->nleaf, npart = s->npart;
    const int form = s->params.form;
    LeafMeta *meta = (LeafMeta *)s->meta.p;
    if (nleaf == 0) return P2P_OK;
    const int threads = 256;
    if (form == P2P_FORM_PLAIN_FP64) {
        prep_plain_kernel<<<grid_for(nleaf, threads, 65535), threads, 0, s->stream>>>(
            s->d_ip, s->d_np, npart, nleaf, meta, (int *)s->status.p);
    } else {
        const int blocks = grid_for((int64_t)nleaf * 32, threads, 65535);
        const double c = 0.5 / s->params.split_radius;
        if (form == P2P_FORM_NAIVE_FP32)
            prep_split_kernel<false><<<blocks, threads, 0, s->stream>>>(
                s->d_pos, s->d_mass, s->d_ip, s->d_np, npart, nleaf, c, meta, (float4 *)s->pos4.p,
                (int *)s->status.p);
        else
            prep_split_kernel<true><<<blocks, threads, 0, s->stream>>>(
                s->d_pos, s->d_mass, s->d_ip, s->d_np, npart, nleaf, c, meta, (float4 *)s->pos4.p,
                (int *)s->status.p);
    }
    CUDA_TRY(cudaGetLastError());
    return launch_count(1);
}

PairArgs make_args(p2p_session *s) {
    PairArgs a;
    std::memset(&a, 0, sizeof(a));
    const p2p_params &p = s->params;
    a.leaf = (const LeafMeta *)s->meta.p;
    a.row_off = (const int64_t *)s->row_off.p;
    a.row_src = (const int *)s->row_src.p;
    a.pos4 = (const float4 *)s->pos4.p;
    a.pos = s->d_pos;
    a.mass = s->d_mass;
    a.acc = (double *)s->acc.p;
    a.queue = (int *)s->queue.p;
    a.evaluated = counts_evaluated(p) ? (unsigned long long *)s->evaluated.p : nullptr;
    a.npart = s->npart;
    a.nleaf = s->nleaf;
    fill_pass_scalars(a, p, s->fit, s->d_mass != nullptr);
    return a;
}

int size_radix_buffers(p2p_session *s, int64_t ntask) {
    const size_t n = (size_t)std::max<int64_t>(ntask, 1);
    P2P_TRY(ensure(s, s->row_src, sizeof(int) * n));
    P2P_TRY(ensure(s, s->keys_a, sizeof(int) * n));
    P2P_TRY(ensure(s, s->keys_b, sizeof(int) * n));
    P2P_TRY(ensure(s, s->vals_b, sizeof(int) * n));
    P2P_TRY(ensure(s, s->hist, sizeof(int) * csr_hist_len(ntask)));
    P2P_TRY(ensure(s, s->hoffs, sizeof(int64_t) * (csr_hist_len(ntask) + 1)));
    P2P_TRY(ensure(s, s->hsums, sizeof(int64_t) * csr_hsum_len(ntask)));
    return P2P_OK;
}

int enqueue_pairs(p2p_session *s, bool timed);

// Whether the pair kernel of these parameters skips entries wholly beyond the
// cutoff (their pairs are then counted apart, for the evaluated-pair count).
bool skips_outside(const p2p_session *s) {
    return packed_lanes(s->params) ||
           (is_fp32_form(s->params.form) && s->params.kernel_variant == P2P_VARIANT_SINK_LANES_X2);
}


// CSR build + pair kernel for one list chunk already on the device.
int enqueue_chunk(p2p_session *s, int64_t ntask, const int *d_t, const int *d_s, bool timed,
                  cudaEvent_t lists_read = nullptr) {
    if (ntask <= 0 || s->nleaf <= 0) return P2P_OK;
    CsrBufs b;
    b.counts = (int *)s->counts.p;
    b.row_off = (int64_t *)s->row_off.p;
    b.tile_sums = (int64_t *)s->tile_sums.p;
    b.row_src = (int *)s->row_src.p;
    b.keys_a = (int *)s->keys_a.p;
    b.keys_b = (int *)s->keys_b.p;
    b.vals_b = (int *)s->vals_b.p;
    b.hist = (int *)s->hist.p;
    b.hoffs = (int64_t *)s->hoffs.p;
    b.hsums = (int64_t *)s->hsums.p;
    b.pairs = (unsigned long long *)s->pairs.p;
    if (skips_outside(s)) {
        // the packed kernels skip entries wholly beyond the cutoff; count their pairs
        b.skipped = (unsigned long long *)s->skipped.p;
        b.cscale = 0.5 / s->params.split_radius;
        b.uout = (float)(s->fit.umax * (1.0 + kCutBand) * (1.0 + kOutsideMargin));
    }
    b.status = (int *)s->status.p;
    int launched = 0;
    CUDA_TRY(enqueue_csr_build(s->stream, ntask, d_t, d_s, s->nleaf, (const LeafMeta *)s->meta.p, b,
                               &launched));
    launch_count(launched);
    if (lists_read) CUDA_TRY(cudaEventRecord(lists_read, s->stream));  // d_t / d_s may be reused
    return enqueue_pairs(s, timed);
}

// The pair kernel over the session's CSR rows (row_off, row_src).
int enqueue_pairs(p2p_session *s, bool timed) {
    CUDA_TRY(cudaMemsetAsync(s->queue.p, 0, sizeof(int), s->stream));
    PairArgs a = make_args(s);
    // Inside a stream capture the kernel's events become external event-record
    // nodes of the graph; outside it they are ordinary records.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CUDA_TRY(cudaStreamIsCapturing(s->stream, &cap));
    const unsigned evflags = cap == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : 0u;
    if (timed) CUDA_TRY(cudaEventRecordWithFlags(s->ev_k0, s->stream, evflags));
    P2P_TRY(launch_pair(s, a));
    if (timed) CUDA_TRY(cudaEventRecordWithFlags(s->ev_k1, s->stream, evflags));
    s->kernel_timed = timed;
    return P2P_OK;
}

int size_pass_buffers(p2p_session *s, int npart, int nleaf, bool host_inputs, bool masses) {
    const size_t n3 = 3 * (size_t)npart;
    if (host_inputs) {
        P2P_TRY(ensure(s, s->pos, sizeof(double) * n3));
        if (masses) P2P_TRY(ensure(s, s->mass, sizeof(double) * (size_t)npart));
        P2P_TRY(ensure(s, s->leaf_ip, sizeof(int) * (size_t)nleaf));
        P2P_TRY(ensure(s, s->leaf_np, sizeof(int) * (size_t)nleaf));
    }
    P2P_TRY(ensure(s, s->acc, sizeof(double) * n3));
    P2P_TRY(ensure(s, s->meta, sizeof(LeafMeta) * (size_t)nleaf));
    if (is_fp32_form(s->params.form)) P2P_TRY(ensure(s, s->pos4, sizeof(float4) * (size_t)npart));
    P2P_TRY(ensure(s, s->counts, sizeof(int) * (size_t)nleaf));
    P2P_TRY(ensure(s, s->fill, sizeof(int) * (size_t)nleaf));
    P2P_TRY(ensure(s, s->row_off, sizeof(int64_t) * ((size_t)nleaf + 1)));
    P2P_TRY(ensure(s, s->tile_sums, sizeof(int64_t) * csr_tile_sums(nleaf)));
    P2P_TRY(ensure(s, s->status, sizeof(int)));
    P2P_TRY(ensure(s, s->queue, sizeof(int)));
    P2P_TRY(ensure(s, s->pairs, sizeof(unsigned long long)));
    P2P_TRY(ensure(s, s->skipped, sizeof(unsigned long long)));
    P2P_TRY(ensure(s, s->evaluated, sizeof(unsigned long long)));
    return P2P_OK;
}

int begin_common(p2p_session *s) {
    CUDA_TRY(cudaMemsetAsync(s->acc.p, 0, sizeof(double) * 3 * (size_t)s->npart, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->status.p, 0, sizeof(int), s->stream));
    CUDA_TRY(cudaMemsetAsync(s->pairs.p, 0, sizeof(unsigned long long), s->stream));
    CUDA_TRY(cudaMemsetAsync(s->skipped.p, 0, sizeof(unsigned long long), s->stream));
    CUDA_TRY(cudaMemsetAsync(s->evaluated.p, 0, sizeof(unsigned long long), s->stream));
    return enqueue_prep(s);
}

int check_session(p2p_session *s) {
    if (!s) return fail(P2P_ERR_ARG, "null session");
    CUDA_TRY(cudaSetDevice(s->device));
    return P2P_OK;
}

}  // namespace

// Host-side services shared with the server's translation unit
// (p2p_host_shared.h).
namespace p2p {
int report_error(int status, const char *msg) {
    g_last_error = msg;
    return status;
}
int check_params(const p2p_params *p) { return validate_params(p); }
void count_launches(int n) { g_launches += n; }
cudaError_t allow_large_smem() { return allow_smem_all(); }
int session_device(const p2p_session *s) { return s ? s->device : 0; }

void *session_scratch(p2p_session *s, int slot, size_t bytes) {
    if (!s || slot < 0) return nullptr;
    if ((size_t)slot >= s->scratch.size()) s->scratch.resize((size_t)slot + 1);
    if (ensure(s, s->scratch[(size_t)slot], bytes) != P2P_OK) return nullptr;
    return s->scratch[(size_t)slot].p;
}
}  // namespace p2p

// ------------------------------------------------------------------ ABI ---

P2P_API void p2p_params_default(p2p_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->form = P2P_FORM_PLAIN_FP64;
    p->soft_mode = P2P_SOFT_CLAMP;
    p->soften = 1.0;
    p->split_radius = 1.0;
    p->x_cut = 2.8125;
    p->mass = 1.0;
}

P2P_API const char *p2p_status_string(int status) {
    switch (status) {
        case P2P_OK: return "ok";
        case P2P_ERR_ARG: return "invalid argument";
        case P2P_ERR_CUDA: return "CUDA error";
        case P2P_ERR_STATE: return "call out of order";
        case P2P_ERR_NOMEM: return "out of device memory";
        case P2P_ERR_RANGE: return "input index out of range";
        case P2P_ERR_CAPACITY: return "input exceeds fixed capacity";
        default: return "unknown status";
    }
}

P2P_API const char *p2p_last_error(void) { return g_last_error.c_str(); }

P2P_API int p2p_version(void) { return 10000; }

P2P_API int p2p_device_count(int *count) {
    if (!count) return fail(P2P_ERR_ARG, "null argument");
    *count = 0;
    cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *count = 0;
        if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return P2P_OK;
        return fail(P2P_ERR_CUDA, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
    }
    return P2P_OK;
}

P2P_API int p2p_session_create(int device, p2p_session **out) {
    if (!out) return fail(P2P_ERR_ARG, "null out");
    *out = nullptr;
    int ndev = 0;
    CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(P2P_ERR_ARG, "device %d of %d", device, ndev);
    CUDA_TRY(cudaSetDevice(device));
    p2p_session *s = new p2p_session();
    s->device = device;
    cudaError_t e = cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev_begin);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev_end);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev_k0);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev_k1);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking);
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
        e = cudaEventCreateWithFlags(&s->piece_ready[k], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->piece_free[k], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = allow_smem_all();
    if (e != cudaSuccess) {
        delete s;
        return fail(P2P_ERR_CUDA, "session setup: %s", cudaGetErrorString(e));
    }
    p2p_params_default(&s->params);
    *out = s;
    return P2P_OK;
}

P2P_API int p2p_session_destroy(p2p_session *s) {
    if (!s) return P2P_OK;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->gexec) cudaGraphExecDestroy(s->gexec);
    DevBuf *bufs[] = {&s->pos, &s->mass, &s->leaf_ip, &s->leaf_np, &s->task_t, &s->task_s,
                      &s->meta, &s->pos4, &s->counts, &s->fill, &s->row_off, &s->row_src,
                      &s->tile_sums, &s->acc, &s->status, &s->queue, &s->pairs, &s->skipped, &s->evaluated, &s->probe,
                      &s->keys_a, &s->keys_b, &s->vals_b, &s->hist, &s->hoffs, &s->hsums,
                      &s->task_t2, &s->task_s2, &s->walk_slab};
    if (s->copy_stream) cudaStreamSynchronize(s->copy_stream);
    for (DevBuf *b : bufs)
        if (b->p) cudaFree(b->p);
    for (DevBuf &b : s->scratch)
        if (b.p) cudaFree(b.p);
    cudaEvent_t evs[] = {s->ev_begin, s->ev_end, s->ev_k0, s->ev_k1, s->piece_ready[0], s->piece_ready[1],
                         s->piece_free[0], s->piece_free[1]};
    for (cudaEvent_t ev : evs)
        if (ev) cudaEventDestroy(ev);
    if (s->stream) cudaStreamDestroy(s->stream);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
    delete s;
    return P2P_OK;
}

P2P_API int p2p_session_set_params(p2p_session *s, const p2p_params *params) {
    if (!s || !params) return fail(P2P_ERR_ARG, "null argument");
    if (s->in_pass) return fail(P2P_ERR_STATE, "cannot change parameters inside a pass");
    P2P_TRY(validate_params(params));
    s->params = *params;
    if (is_fp32_form(params->form)) {
        s->fit = fit_h(fit_umax(params->x_cut), params->poly_tol > 0.0 ? params->poly_tol : kDefaultPolyTol);
    } else {
        s->fit = PolyFit();
    }
    s->version++;
    if (s->gexec) {
        cudaGraphExecDestroy(s->gexec);
        s->gexec = nullptr;
    }
    return P2P_OK;
}

P2P_API int p2p_session_get_params(const p2p_session *s, p2p_params *params) {
    if (!s || !params) return fail(P2P_ERR_ARG, "null argument");
    *params = s->params;
    return P2P_OK;
}

P2P_API void *p2p_session_stream(p2p_session *s) { return s ? (void *)s->stream : nullptr; }

P2P_API int p2p_session_poly_degree(const p2p_session *s) { return s ? s->fit.degree : 0; }

P2P_API double p2p_session_poly_error(const p2p_session *s) { return s ? s->fit.max_err : 0.0; }

namespace {
int check_host_begin(p2p_session *s, int npart, const double *pos, int nleaf, const int *leaf_ipart,
                     const int *leaf_npart) {
    P2P_TRY(check_session(s));
    if (s->in_pass) return fail(P2P_ERR_STATE, "pass already open");
    if (npart < 0 || nleaf < 0) return fail(P2P_ERR_ARG, "negative size");
    if ((npart > 0 && !pos) || (nleaf > 0 && (!leaf_ipart || !leaf_npart)))
        return fail(P2P_ERR_ARG, "null input");
    for (int l = 0; l < nleaf; ++l) {
        const int64_t ip = leaf_ipart[l], np = leaf_npart[l];
        if (ip < 0 || np < 0 || ip + np > npart)
            return fail(P2P_ERR_RANGE, "leaf %d covers [%lld, %lld) outside [0, %d)", l,
                        (long long)ip, (long long)(ip + np), npart);
    }
    return P2P_OK;
}

// The leaf table upload and the pass state after the positions are queued.
int finish_host_begin(p2p_session *s, int npart, const double *masses, int nleaf, const int *leaf_ipart,
                      const int *leaf_npart) {
    if (masses && npart)
        CUDA_TRY(cudaMemcpyAsync(s->mass.p, masses, sizeof(double) * (size_t)npart, cudaMemcpyHostToDevice, s->stream));
    if (nleaf) {
        CUDA_TRY(cudaMemcpyAsync(s->leaf_ip.p, leaf_ipart, sizeof(int) * (size_t)nleaf, cudaMemcpyHostToDevice, s->stream));
        CUDA_TRY(cudaMemcpyAsync(s->leaf_np.p, leaf_npart, sizeof(int) * (size_t)nleaf, cudaMemcpyHostToDevice, s->stream));
    }
    s->pos_held = npart;
    s->d_pos = (const double *)s->pos.p;
    s->d_mass = masses ? (const double *)s->mass.p : nullptr;
    s->d_ip = (const int *)s->leaf_ip.p;
    s->d_np = (const int *)s->leaf_np.p;
    P2P_TRY(begin_common(s));
    s->in_pass = true;
    s->kernel_timed = false;
    return P2P_OK;
}
}  // namespace

P2P_API int p2p_pass_begin(p2p_session *s, int npart, const double *pos, const double *masses,
                           int nleaf, const int *leaf_ipart, const int *leaf_npart) {
    P2P_TRY(check_host_begin(s, npart, pos, nleaf, leaf_ipart, leaf_npart));
    s->pos_held = -1;
    P2P_TRY(size_pass_buffers(s, npart, nleaf, true, masses != nullptr));
    s->npart = npart;
    s->nleaf = nleaf;
    CUDA_TRY(cudaEventRecord(s->ev_begin, s->stream));
    if (npart) CUDA_TRY(cudaMemcpyAsync(s->pos.p, pos, sizeof(double) * 3 * (size_t)npart, cudaMemcpyHostToDevice, s->stream));
    return finish_host_begin(s, npart, masses, nleaf, leaf_ipart, leaf_npart);
}

P2P_API int p2p_pass_begin_update(p2p_session *s, int npart, const double *pos, int nleaf, const int *leaf_ipart,
                                  const int *leaf_npart, const unsigned char *dirty, int64_t chunk,
                                  int64_t *uploaded_bytes) {
    P2P_TRY(check_host_begin(s, npart, pos, nleaf, leaf_ipart, leaf_npart));
    if (dirty && chunk <= 0) return fail(P2P_ERR_ARG, "chunk must be positive");
    const void *before = s->pos.p;
    const bool held = s->pos_held == npart;
    s->pos_held = -1;
    P2P_TRY(size_pass_buffers(s, npart, nleaf, true, false));
    s->npart = npart;
    s->nleaf = nleaf;
    CUDA_TRY(cudaEventRecord(s->ev_begin, s->stream));
    const size_t n = (size_t)npart;
    double *dst = (double *)s->pos.p;
    int64_t bytes = 0;
    if (!dirty || !held || s->pos.p != before) {
        if (npart) CUDA_TRY(cudaMemcpyAsync(dst, pos, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s->stream));
        bytes = (int64_t)(sizeof(double) * 3 * n);
    } else {
        // runs of changed chunks, one copy per coordinate row and run
        const int64_t nchunk = (npart + chunk - 1) / chunk;
        for (int64_t c = 0; c < nchunk;) {
            if (!dirty[c]) {
                ++c;
                continue;
            }
            int64_t e = c;
            while (e < nchunk && dirty[e]) ++e;
            const size_t a = (size_t)(c * chunk), b = std::min(n, (size_t)(e * chunk));
            for (int d = 0; d < 3; ++d)
                CUDA_TRY(cudaMemcpyAsync(dst + d * n + a, pos + d * n + a, sizeof(double) * (b - a),
                                         cudaMemcpyHostToDevice, s->stream));
            bytes += (int64_t)(3 * sizeof(double) * (b - a));
            c = e;
        }
    }
    if (uploaded_bytes) *uploaded_bytes = bytes;
    return finish_host_begin(s, npart, nullptr, nleaf, leaf_ipart, leaf_npart);
}

P2P_API int p2p_pass_begin_device(p2p_session *s, int npart, const double *d_pos,
                                  const double *d_masses, int nleaf, const int *d_leaf_ipart,
                                  const int *d_leaf_npart) {
    P2P_TRY(check_session(s));
    if (s->in_pass) return fail(P2P_ERR_STATE, "pass already open");
    if (npart < 0 || nleaf < 0) return fail(P2P_ERR_ARG, "negative size");
    if ((npart > 0 && !d_pos) || (nleaf > 0 && (!d_leaf_ipart || !d_leaf_npart)))
        return fail(P2P_ERR_ARG, "null input");
    P2P_TRY(size_pass_buffers(s, npart, nleaf, false, false));
    s->npart = npart;
    s->nleaf = nleaf;
    s->d_pos = d_pos;
    s->d_mass = d_masses;
    s->d_ip = d_leaf_ipart;
    s->d_np = d_leaf_npart;
    CUDA_TRY(cudaEventRecord(s->ev_begin, s->stream));
    P2P_TRY(begin_common(s));
    s->in_pass = true;
    s->kernel_timed = false;
    return P2P_OK;
}

P2P_API int p2p_pass_submit(p2p_session *s, int64_t ntask, const int *task_t, const int *task_s) {
    P2P_TRY(check_session(s));
    if (!s->in_pass) return fail(P2P_ERR_STATE, "no open pass");
    if (ntask < 0) return fail(P2P_ERR_ARG, "negative ntask");
    if (ntask == 0) return P2P_OK;
    if (!task_t || !task_s) return fail(P2P_ERR_ARG, "null task list");
    if (ntask > 2 * kPipePieceMin && is_fp32_form(s->params.form)) {
        // Large lists (FP32 forms): upload in pieces on the copy stream while
        // the previous piece's CSR build and pair kernel run (each piece is a
        // list chunk, as the reference's LEN_TASK chunks are). The FP64 form
        // keeps one chunk: its slowest rows would stretch every piece's tail.
        const int64_t piece = std::max<int64_t>(kPipePieceMin, (ntask + kPipePieces - 1) / kPipePieces);
        P2P_TRY(ensure(s, s->task_t, sizeof(int) * (size_t)piece));
        P2P_TRY(ensure(s, s->task_s, sizeof(int) * (size_t)piece));
        P2P_TRY(ensure(s, s->task_t2, sizeof(int) * (size_t)piece));
        P2P_TRY(ensure(s, s->task_s2, sizeof(int) * (size_t)piece));
        P2P_TRY(size_radix_buffers(s, piece));
        DevBuf *bt[2] = {&s->task_t, &s->task_t2}, *bs[2] = {&s->task_s, &s->task_s2};
        // the copy stream starts after everything queued so far (begin's uploads)
        CUDA_TRY(cudaEventRecord(s->piece_ready[0], s->stream));
        CUDA_TRY(cudaStreamWaitEvent(s->copy_stream, s->piece_ready[0], 0));
        bool used[2] = {false, false};
        for (int64_t i0 = 0, k = 0; i0 < ntask; i0 += piece, k ^= 1) {
            const int64_t n = std::min(piece, ntask - i0);
            if (used[k]) CUDA_TRY(cudaStreamWaitEvent(s->copy_stream, s->piece_free[k], 0));
            CUDA_TRY(cudaMemcpyAsync(bt[k]->p, task_t + i0, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice,
                                     s->copy_stream));
            CUDA_TRY(cudaMemcpyAsync(bs[k]->p, task_s + i0, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice,
                                     s->copy_stream));
            CUDA_TRY(cudaEventRecord(s->piece_ready[k], s->copy_stream));
            CUDA_TRY(cudaStreamWaitEvent(s->stream, s->piece_ready[k], 0));
            P2P_TRY(enqueue_chunk(s, n, (const int *)bt[k]->p, (const int *)bs[k]->p, i0 + n >= ntask,
                                  s->piece_free[k]));
            used[k] = true;
        }
        return P2P_OK;
    }
    P2P_TRY(ensure(s, s->task_t, sizeof(int) * (size_t)ntask));
    P2P_TRY(ensure(s, s->task_s, sizeof(int) * (size_t)ntask));
    P2P_TRY(size_radix_buffers(s, ntask));
    CUDA_TRY(cudaMemcpyAsync(s->task_t.p, task_t, sizeof(int) * (size_t)ntask, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->task_s.p, task_s, sizeof(int) * (size_t)ntask, cudaMemcpyHostToDevice, s->stream));
    return enqueue_chunk(s, ntask, (const int *)s->task_t.p, (const int *)s->task_s.p, true);
}

P2P_API int p2p_pass_submit_device(p2p_session *s, int64_t ntask, const int *d_task_t,
                                   const int *d_task_s) {
    P2P_TRY(check_session(s));
    if (!s->in_pass) return fail(P2P_ERR_STATE, "no open pass");
    if (ntask < 0) return fail(P2P_ERR_ARG, "negative ntask");
    if (ntask == 0) return P2P_OK;
    if (!d_task_t || !d_task_s) return fail(P2P_ERR_ARG, "null task list");
    P2P_TRY(size_radix_buffers(s, ntask));
    return enqueue_chunk(s, ntask, d_task_t, d_task_s, true);
}

P2P_API int p2p_pass_end(p2p_session *s, double *gpu_seconds) {
    P2P_TRY(check_session(s));
    if (!s->in_pass) return fail(P2P_ERR_STATE, "no open pass");
    s->in_pass = false;
    CUDA_TRY(cudaEventRecord(s->ev_end, s->stream));
    CUDA_TRY(cudaEventSynchronize(s->ev_end));
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, s->ev_begin, s->ev_end));
    if (gpu_seconds) *gpu_seconds = ms * 1e-3;
    int status = 0;
    CUDA_TRY(cudaMemcpy(&status, s->status.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (status & ST_LEAF_RANGE) return fail(P2P_ERR_RANGE, "a leaf range lies outside the particles");
    if (status & ST_TASK_RANGE) return fail(P2P_ERR_RANGE, "a task entry names a leaf outside [0, nleaf)");
    if (status & ST_WALK_TREE) return fail(P2P_ERR_ARG, "walk: a child code outside the tree");
    if (status & (ST_WALK_STACK | ST_WALK_ROW)) return fail(P2P_ERR_CAPACITY, "walk: a sink's walk exceeded its stack");
    return P2P_OK;
}

P2P_API int p2p_pass_submit_walk(p2p_session *s, const p2p_walk_tree *t, double cutoff, double open_angle,
                                 int64_t *ntask) {
    P2P_TRY(check_session(s));
    if (!s->in_pass) return fail(P2P_ERR_STATE, "no open pass");
    if (!t) return fail(P2P_ERR_ARG, "null tree");
    if (t->nleaf != s->nleaf) return fail(P2P_ERR_ARG, "tree has %d leaves, the pass %d", t->nleaf, s->nleaf);
    if (t->nnode < 0) return fail(P2P_ERR_ARG, "negative size");
    if ((t->nnode > 0 && (!t->son || !t->node_first || !t->node_center || !t->node_width)) ||
        (t->nleaf > 0 && (!t->leaf_center || !t->leaf_width || !t->leaf_active)))
        return fail(P2P_ERR_ARG, "null tree array");
    if (!(cutoff >= 0.0) || !(open_angle >= 0.0)) return fail(P2P_ERR_ARG, "bad cutoff or open angle");
    if (ntask) *ntask = 0;
    const int nleaf = s->nleaf;
    if (nleaf == 0 || t->nnode == 0) return P2P_OK;
    WalkArgs w;
    w.nnode = t->nnode;
    w.nleaf = nleaf;
    w.son = t->son;
    w.node_first = t->node_first;
    w.leaf_active = t->leaf_active;
    w.node_center = t->node_center;
    w.node_width = t->node_width;
    w.leaf_center = t->leaf_center;
    w.leaf_width = t->leaf_width;
    w.cutoff = cutoff;
    w.open_angle = open_angle;
    const int threads = kWalkWarps * 32;
    const int grid = grid_for(nleaf, kWalkWarps, s->sm_count * 32);
    int *status = (int *)s->status.p;
    // The first pass keeps each row's first slab_cap entries in a slab of
    // slab_cap ids per leaf (at most kWalkSlabBytes), from which the rows are
    // gathered; only rows longer than that are walked a second time.
    int slab_cap = kWalkSlabMax;
    while (slab_cap > kWalkSlabMin && (size_t)nleaf * slab_cap * sizeof(int) > kWalkSlabBytes) slab_cap >>= 1;
    if ((size_t)nleaf * slab_cap * sizeof(int) > kWalkSlabBytes) slab_cap = 0;  // two walks
    int *slab = nullptr;
    if (slab_cap > 0) {
        P2P_TRY(ensure(s, s->walk_slab, sizeof(int) * (size_t)nleaf * slab_cap));
        slab = (int *)s->walk_slab.p;
    }
    // pass 1: row lengths (and the slab), then the row offsets
    walk_rows_kernel<false><<<grid, threads, 0, s->stream>>>(w, (int *)s->counts.p, nullptr, nullptr, nullptr,
                                                               nullptr, 0.0, 0.f, nullptr, nullptr, status, slab,
                                                               slab_cap);
    const int ntiles = (int)((nleaf + (int64_t)kScanTile - 1) / kScanTile);
    int64_t *row_off = (int64_t *)s->row_off.p;
    scan_tiles_kernel<<<ntiles, kScanThreads, 0, s->stream>>>((const int *)s->counts.p, nleaf, row_off,
                                                               (int64_t *)s->tile_sums.p);
    scan_sums_kernel<<<1, kScanThreads, 0, s->stream>>>((int64_t *)s->tile_sums.p, ntiles, row_off + nleaf);
    scan_add_kernel<<<grid_for(nleaf, 256, 1 << 30), 256, 0, s->stream>>>(row_off, nleaf, (int64_t *)s->tile_sums.p);
    CUDA_TRY(cudaGetLastError());
    launch_count(4);
    int64_t total = 0;
    int st = 0;
    CUDA_TRY(cudaMemcpyAsync(&total, row_off + nleaf, sizeof(total), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaMemcpyAsync(&st, status, sizeof(st), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (st & ST_WALK_TREE) return fail(P2P_ERR_ARG, "walk: a child code outside the tree");
    if (st & ST_WALK_STACK) return fail(P2P_ERR_CAPACITY, "walk: a sink's walk exceeded its stack");
    if (ntask) *ntask = total;
    if (total == 0) return P2P_OK;
    // pass 2: the rows' source ids, pair counts (short rows from the slab,
    // long rows walked again); then the pair kernel
    P2P_TRY(ensure(s, s->row_src, sizeof(int) * (size_t)total));
    const bool skip = skips_outside(s);
    const double cscale = 0.5 / s->params.split_radius;
    const float uout = (float)(s->fit.umax * (1.0 + kCutBand) * (1.0 + kOutsideMargin));
    unsigned long long *d_skipped = skip ? (unsigned long long *)s->skipped.p : nullptr;
    if (slab)
        walk_gather_kernel<<<grid_for(nleaf, 8, s->sm_count * 16), 256, 0, s->stream>>>(
            (const int *)s->counts.p, row_off, nleaf, slab, slab_cap, (int *)s->row_src.p, s->d_np,
            (const LeafMeta *)s->meta.p, cscale, uout, (unsigned long long *)s->pairs.p, d_skipped, status);
    walk_rows_kernel<true><<<grid, threads, 0, s->stream>>>(
        w, (int *)s->counts.p, row_off, (int *)s->row_src.p, s->d_np, (const LeafMeta *)s->meta.p, cscale, uout,
        (unsigned long long *)s->pairs.p, d_skipped, status, nullptr, slab_cap);
    // each row ascending by source leaf id: the serial walk's order for that sink
    int *rs = (int *)s->row_src.p;
    csr_sort_rows_warp_kernel<1, kSortWarpMax><<<grid_for(nleaf, 4, s->sm_count * 8), 128, 0, s->stream>>>(
        row_off, nleaf, rs);
    csr_sort_rows_warp_kernel<kSortWarpMax, kSortWarpMax2><<<grid_for(nleaf, 4, s->sm_count * 8), 128, 0, s->stream>>>(
        row_off, nleaf, rs);
    csr_sort_rows_block_kernel<<<grid_for(nleaf, 1, s->sm_count * 4), kSortBlockThreads, 0, s->stream>>>(
        row_off, nleaf, rs);
    csr_sort_rows_global_kernel<<<grid_for(nleaf, 1, s->sm_count), kSortBlockThreads, 0, s->stream>>>(
        row_off, nleaf, rs);
    CUDA_TRY(cudaGetLastError());
    launch_count(slab ? 6 : 5);
    return enqueue_pairs(s, true);
}

P2P_API int p2p_pass_rows(p2p_session *s, int64_t *row_off, int *row_src) {
    P2P_TRY(check_session(s));
    if (s->in_pass) return fail(P2P_ERR_STATE, "pass still open; call p2p_pass_end first");
    if (!row_off) return fail(P2P_ERR_ARG, "null argument");
    const size_t nl = (size_t)s->nleaf + 1;
    CUDA_TRY(cudaMemcpy(row_off, s->row_off.p, sizeof(int64_t) * nl, cudaMemcpyDeviceToHost));
    const int64_t total = row_off[s->nleaf];
    if (total > 0 && row_src)
        CUDA_TRY(cudaMemcpy(row_src, s->row_src.p, sizeof(int) * (size_t)total, cudaMemcpyDeviceToHost));
    return P2P_OK;
}

P2P_API int p2p_pass_accumulate(p2p_session *s, double *acc) {
    P2P_TRY(check_session(s));
    if (s->in_pass) return fail(P2P_ERR_STATE, "pass still open; call p2p_pass_end first");
    if (!acc && s->npart) return fail(P2P_ERR_ARG, "null acc");
    const size_t n3 = 3 * (size_t)s->npart;
    std::vector<double> buf(n3);
    if (n3) CUDA_TRY(cudaMemcpy(buf.data(), s->acc.p, sizeof(double) * n3, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n3; ++i) acc[i] += buf[i];
    return P2P_OK;
}

P2P_API int p2p_pass_result(p2p_session *s, double *out) {
    P2P_TRY(check_session(s));
    if (s->in_pass) return fail(P2P_ERR_STATE, "pass still open; call p2p_pass_end first");
    if (!out && s->npart) return fail(P2P_ERR_ARG, "null out");
    const size_t n3 = 3 * (size_t)s->npart;
    if (n3) CUDA_TRY(cudaMemcpy(out, s->acc.p, sizeof(double) * n3, cudaMemcpyDeviceToHost));
    return P2P_OK;
}

P2P_API int p2p_session_synchronize(p2p_session *s) {
    P2P_TRY(check_session(s));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return P2P_OK;
}

P2P_API int p2p_pass_result_device(p2p_session *s, const double **d_acc) {
    if (!s || !d_acc) return fail(P2P_ERR_ARG, "null argument");
    *d_acc = (const double *)s->acc.p;
    return P2P_OK;
}

P2P_API int p2p_pass_evaluated_pairs(p2p_session *s, int64_t *pairs) {
    P2P_TRY(check_session(s));
    if (!pairs) return fail(P2P_ERR_ARG, "null argument");
    unsigned long long v = 0, k = 0;
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (counts_evaluated(s->params)) {
        CUDA_TRY(cudaMemcpy(&v, s->evaluated.p, sizeof(v), cudaMemcpyDeviceToHost));
        *pairs = (int64_t)v;
        return P2P_OK;
    }
    CUDA_TRY(cudaMemcpy(&v, s->pairs.p, sizeof(v), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(&k, s->skipped.p, sizeof(k), cudaMemcpyDeviceToHost));
    *pairs = (int64_t)(v - k);
    return P2P_OK;
}

P2P_API int p2p_pass_pair_count(p2p_session *s, int64_t *pairs) {
    P2P_TRY(check_session(s));
    if (!pairs) return fail(P2P_ERR_ARG, "null argument");
    unsigned long long v = 0;
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    CUDA_TRY(cudaMemcpy(&v, s->pairs.p, sizeof(v), cudaMemcpyDeviceToHost));
    *pairs = (int64_t)v;
    return P2P_OK;
}

P2P_API int p2p_pass_run_device(p2p_session *s, int npart, const double *d_pos,
                                const double *d_masses, int nleaf, const int *d_leaf_ipart,
                                const int *d_leaf_npart, int64_t ntask, const int *d_task_t,
                                const int *d_task_s) {
    P2P_TRY(check_session(s));
    if (s->in_pass) return fail(P2P_ERR_STATE, "pass already open");
    if (npart < 0 || nleaf < 0 || ntask < 0) return fail(P2P_ERR_ARG, "negative size");
    if ((npart > 0 && !d_pos) || (nleaf > 0 && (!d_leaf_ipart || !d_leaf_npart)) ||
        (ntask > 0 && (!d_task_t || !d_task_s)))
        return fail(P2P_ERR_ARG, "null input");
    p2p_session::Key key{};
    key.p[0] = d_pos; key.p[1] = d_masses; key.p[2] = d_leaf_ipart; key.p[3] = d_leaf_npart;
    key.p[4] = d_task_t; key.p[5] = d_task_s;
    key.n[0] = npart; key.n[1] = nleaf; key.n[2] = ntask;
    key.version = s->version;
    // sizing may drop a cached graph (buffers moved)
    P2P_TRY(size_pass_buffers(s, npart, nleaf, false, false));
    P2P_TRY(size_radix_buffers(s, ntask));
    s->npart = npart;
    s->nleaf = nleaf;
    s->d_pos = d_pos;
    s->d_mass = d_masses;
    s->d_ip = d_leaf_ipart;
    s->d_np = d_leaf_npart;
    const bool hit = s->gexec && std::memcmp(&key, &s->gkey, sizeof(key)) == 0;
    if (!hit) {
        if (s->gexec) {
            cudaGraphExecDestroy(s->gexec);
            s->gexec = nullptr;
        }
        {   // resolve launch shapes (occupancy queries) before capturing
            s->dry_run = true;
            const int st = launch_pair(s, make_args(s));
            s->dry_run = false;
            if (st != P2P_OK) return st;
        }
        cudaGraph_t graph = nullptr;
        CUDA_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        const int64_t before = g_launches.load();
        int st = begin_common(s);
        if (st == P2P_OK) st = enqueue_chunk(s, ntask, d_task_t, d_task_s, true);
        cudaError_t ce = cudaStreamEndCapture(s->stream, &graph);
        const int64_t captured = g_launches.load() - before;
        g_launches -= captured;  // capture does not launch; replays are counted below
        if (st != P2P_OK) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        if (ce != cudaSuccess) return fail(P2P_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
        cudaError_t ie = cudaGraphInstantiate(&s->gexec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) {
            s->gexec = nullptr;
            return fail(P2P_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ie));
        }
        s->graph_kernels = (int)captured;
        s->gkey = key;
    }
    CUDA_TRY(cudaEventRecord(s->ev_begin, s->stream));
    CUDA_TRY(cudaGraphLaunch(s->gexec, s->stream));
    g_launches += s->graph_kernels;
    s->kernel_timed = ntask > 0 && nleaf > 0;
    s->in_pass = true;
    return P2P_OK;
}

P2P_API int64_t p2p_kernel_launch_count(void) { return g_launches.load(); }

P2P_API int p2p_session_last_kernel_ms(p2p_session *s, float *ms) {
    if (!s || !ms) return fail(P2P_ERR_ARG, "null argument");
    *ms = 0.f;
    if (!s->kernel_timed) return P2P_OK;
    CUDA_TRY(cudaEventSynchronize(s->ev_k1));
    CUDA_TRY(cudaEventElapsedTime(ms, s->ev_k0, s->ev_k1));
    return P2P_OK;
}

P2P_API int p2p_measure_fp32_peak(p2p_session *s, double *tflops) {
    P2P_TRY(check_session(s));
    if (!tflops) return fail(P2P_ERR_ARG, "null argument");
    const int threads = 256, blocks = s->sm_count * 8, iters = 4096;
    P2P_TRY(ensure(s, s->probe, sizeof(float) * (size_t)threads * blocks));
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        CUDA_TRY(cudaEventRecord(s->ev_k0, s->stream));
        fma_probe_kernel<<<blocks, threads, 0, s->stream>>>((float *)s->probe.p, iters, 0.9999999f, 1e-7f);
        CUDA_TRY(cudaGetLastError());
        launch_count(1);
        CUDA_TRY(cudaEventRecord(s->ev_k1, s->stream));
        CUDA_TRY(cudaEventSynchronize(s->ev_k1));
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, s->ev_k0, s->ev_k1));
        best = std::min(best, ms);
    }
    const double flops = 2.0 * 8 * 8 * (double)iters * threads * blocks;
    *tflops = flops / (best * 1e-3) / 1e12;
    s->kernel_timed = false;
    return P2P_OK;
}

P2P_API int p2p_measure_fp64_peak(p2p_session *s, double *tflops) {
    P2P_TRY(check_session(s));
    if (!tflops) return fail(P2P_ERR_ARG, "null argument");
    const int threads = 256, blocks = s->sm_count * 8, iters = 1024;
    P2P_TRY(ensure(s, s->probe, sizeof(double) * (size_t)threads * blocks));
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        CUDA_TRY(cudaEventRecord(s->ev_k0, s->stream));
        dfma_probe_kernel<<<blocks, threads, 0, s->stream>>>((double *)s->probe.p, iters, 0.9999999999,
                                                             1e-12);
        CUDA_TRY(cudaGetLastError());
        launch_count(1);
        CUDA_TRY(cudaEventRecord(s->ev_k1, s->stream));
        CUDA_TRY(cudaEventSynchronize(s->ev_k1));
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, s->ev_k0, s->ev_k1));
        best = std::min(best, ms);
    }
    const double flops = 2.0 * 8 * 8 * (double)iters * threads * blocks;
    *tflops = flops / (best * 1e-3) / 1e12;
    s->kernel_timed = false;
    return P2P_OK;
}
