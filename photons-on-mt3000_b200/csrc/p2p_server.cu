// p2p_server: force passes for an ensemble of independent periodic boxes
// with continuous batching (C ABI in include/photons_p2p.h).
//
// Device memory is one arena of fixed size split into three index spaces,
// each with a first-fit range allocator:
//   particles  pos (FP64 SoA, stride = particle capacity), pos4 (FP32 leaf
//              frames), acc (FP64 SoA, kept zero between requests)
//   leaves     LeafMeta + row offsets (nleaf + 1 per box)
//   rows       CSR source ids
// A resident box owns one range in each. Its positions are stored in the
// shared kernel units (times length_scale) and its leaf / row ids are
// arena-global, so any set of resident boxes forms one pass over the arena:
// a packed launch only lists each box's leaf range as a segment of its work
// queue (PairArgs::seg_*), and a row is computed the same way whatever else
// is packed with it.
//
// One dispatcher thread owns every CUDA object. It moves submitted requests
// to a pending queue, makes their boxes resident (upload, frame prep, CSR
// build on a build stream, evicting least recently used idle boxes when the
// arena is full), packs pending requests of distinct idle boxes into one
// persistent launch per free slot (stream), and retires slots when their
// completion callback fires. A launch is: reset the work counter, pair
// kernel, finalize kernel (scale to box units, write to the caller's mapped
// host buffer, clear the arena's acc), host callback.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "photons_p2p.h"
#include "p2p_args.h"
#include "p2p_fit.h"
#include "p2p_host_shared.h"
#include "p2p_internal.h"
#include "p2p_launch.h"

// This file's own instance of the pass kernels (private namespace, so its
// non-template kernels do not collide with the session path's at link time).
namespace p2p_server_kernels {
using namespace ::p2p;
#include "p2p_pass_kernels.cuh"
namespace p2p {
#include "p2p_csr.h"

// Box positions into the arena in kernel units.
__global__ void scale_positions_kernel(const double *__restrict__ in, int n, double scale,
                                       double *__restrict__ out, int64_t stride) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * (int64_t)n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t d = i / n, k = i - d * n;
        out[d * stride + k] = in[i] * scale;
    }
}

__global__ void add_offset_kernel(int *__restrict__ v, int64_t n, int off) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        v[i] += off;
}

__global__ void iota_kernel(int *__restrict__ v, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

__global__ void add_offset64_kernel(int64_t *__restrict__ v, int64_t n, int64_t off) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        v[i] += off;
}

// One box of a launch, for the clear and gather kernels.
struct OutSeg {
    int64_t p0;      // arena particle base
    int n;           // particles
    int nres;        // returned particles
    int64_t off;     // offset of the box's results in the staging buffer (doubles)
    double scale;    // kernel units -> box units (length_scale^2 * mass)
};
struct OutArgs {
    int nseg;
    int64_t stride;     // particle capacity
    double *acc;
    const int *rmap;    // per box: box-local slot of each returned particle
    double *stage;      // results, SoA per box: 3 * nres doubles
    OutSeg seg[kMaxSeg];
};

// Zeroes the launch's boxes' accumulators (the pair kernel adds into them).
__global__ void clear_acc_kernel(const __grid_constant__ OutArgs f) {
    const OutSeg &s = f.seg[blockIdx.y];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * (int64_t)s.n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t d = i / s.n, k = i - d * s.n;
        f.acc[d * f.stride + s.p0 + k] = 0.0;
    }
}

// Returned particles' accelerations, in box units, into the staging buffer.
__global__ void gather_results_kernel(const __grid_constant__ OutArgs f) {
    const OutSeg &s = f.seg[blockIdx.y];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * (int64_t)s.nres;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t d = i / s.nres, r = i - d * s.nres;
        const int slot = f.rmap[s.p0 + r];
        f.stage[s.off + i] = f.acc[d * f.stride + s.p0 + slot] * s.scale;
    }
}
}  // namespace p2p
}  // namespace p2p_server_kernels

#define P2P_API extern "C" __attribute__((visibility("default")))

namespace {

using namespace ::p2p;
using namespace ::p2p_server_kernels::p2p;
using Clock = std::chrono::steady_clock;

int fail(int status, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return report_error(status, buf);
}

#define CUDA_TRY(expr)                                                                   \
    do {                                                                                 \
        cudaError_t _e = (expr);                                                         \
        if (_e != cudaSuccess)                                                           \
            return fail(P2P_ERR_CUDA, "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e), \
                        __FILE__, __LINE__);                                             \
    } while (0)

#define P2P_TRY(expr)                \
    do {                             \
        int _s = (expr);             \
        if (_s != P2P_OK) return _s; \
    } while (0)

// First-fit allocator of index ranges in [0, cap).
struct RangeAlloc {
    int64_t cap = 0, used = 0;
    std::map<int64_t, int64_t> free_;  // start -> length
    void reset(int64_t c) {
        cap = c;
        used = 0;
        free_.clear();
        if (c > 0) free_[0] = c;
    }
    bool alloc(int64_t n, int64_t *start) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                *start = it->first;
                const int64_t rest = it->second - n, s = it->first + n;
                free_.erase(it);
                if (rest > 0) free_[s] = rest;
                used += n;
                return true;
            }
        }
        return false;
    }
    void release(int64_t start, int64_t n) {
        if (n <= 0) return;
        used -= n;
        auto next = free_.lower_bound(start);
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == start) {
                start = prev->first;
                n += prev->second;
                free_.erase(prev);
            }
        }
        next = free_.lower_bound(start);
        if (next != free_.end() && start + n == next->first) {
            n += next->second;
            free_.erase(next);
        }
        free_[start] = n;
    }
};

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
};

struct Box {
    double length_scale = 1.0, mass = 1.0;
    int npart = 0, nleaf = 0, nres = 0;
    const int *res_slots = nullptr;  // null: every particle, in slot order
    int64_t ntask = 0;
    const double *pos = nullptr;
    const int *ip = nullptr, *np = nullptr, *tt = nullptr, *ts = nullptr;
    bool resident = false, busy = false;
    bool pinned = false;          // preloaded: never evicted
    int64_t P = 0, L = 0, R = 0;  // arena bases
    int pending = 0;              // queued requests
    uint64_t last_use = 0;
    cudaEvent_t ready = nullptr;  // residency build done
    int64_t pairs = 0;            // pair interactions of one pass
};

constexpr int kMaxBoxes = 1 << 16;

struct Request {
    int box = -1;
    double *out = nullptr;
    Clock::time_point t_submit, t_done;
    bool done = false;
    int status = P2P_OK;
};

// A request as the dispatcher sees it.
struct Job {
    int64_t ticket;
    int box;
    double *out;   // page-locked host buffer
    bool preload;  // make the box resident and pinned; no pass
    std::chrono::steady_clock::time_point t_submit;
};

// A launch slot: its compute stream and the copy stream that drains its
// results while the next launch computes. Staging is double-buffered.
struct Slot {
    cudaStream_t stream = nullptr, copy = nullptr;
    cudaEvent_t k0 = nullptr, k1 = nullptr, staged = nullptr;
    cudaEvent_t copied[2] = {nullptr, nullptr};
    bool copied_used[2] = {false, false};
    DevBuf stage[2];
    int cur = 0;
    int *d_queue = nullptr;
    bool busy = false;
};

struct Launch {
    struct p2p_server *srv = nullptr;
    Slot *slot = nullptr;
    std::vector<Job> jobs;
    bool kernel_done = false, kernel_seen = false;  // pair + gather finished / processed
    bool copy_done = false;                         // results are in the callers' buffers
    Clock::time_point t_copy;
};

}  // namespace

struct p2p_server {
    int device = 0, sm_count = 0;
    p2p_params shape{};
    PolyFit fit;
    p2p_server_config cfg{};
    bool fp32 = true;
    // arena
    int64_t Pcap = 0, Lcap = 0, Rcap = 0;
    void *arena = nullptr;
    size_t arena_bytes = 0;
    double *pos = nullptr, *acc = nullptr;
    float4 *pos4 = nullptr;
    LeafMeta *meta = nullptr;
    int64_t *row_off = nullptr;
    int *row_src = nullptr;
    int *rmap = nullptr;             // particle space: returned particles' box-local slots
    RangeAlloc pa, la, ra;
    // build
    cudaStream_t build_stream = nullptr;
    cudaEvent_t b0 = nullptr, b1 = nullptr;
    DevBuf st_pos, st_ip, st_np, st_t, st_s, counts, tile_sums, keys_a, keys_b, vals_b, hist, hoffs,
        hsums, ctrl;
    int64_t *h_pairs = nullptr;  // pinned: pair count and status of the last build
    OccupancyCache occ;
    std::vector<Slot> slots;
    std::vector<Launch *> launches;  // in flight (dispatcher-owned; flags under mu)
    // Boxes: reserved for kMaxBoxes so elements never move; the dispatcher
    // sees the first nbox_seen of them and owns their residency fields.
    std::vector<Box> boxes;
    int nbox_seen = 0;
    // Requests (guarded by mu) and the dispatcher's queue of them.
    std::deque<Request> reqs;
    std::deque<Job> incoming;      // submitted, not yet seen by the dispatcher
    std::deque<Job> pending;       // dispatcher-owned
    uint64_t use_clock = 0;
    // synchronisation
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    uint64_t epoch = 0;            // bumped by completions
    bool stop = false;
    // batching window: the dispatcher sleeps at most until here; flush: the
    // server is stopping, launch without waiting (both dispatcher-owned)
    std::chrono::steady_clock::time_point hold_until = std::chrono::steady_clock::time_point::max();
    bool flush = false;
    double set_window_ms = -1.0, set_min_pairs = 0.0;  // p2p_server_set_batching (mu)
    int error = P2P_OK;
    std::string error_msg;
    int64_t submitted = 0, finished = 0;
    p2p_server_stats stats{};      // published copy (mu)
    p2p_server_stats ds{};         // the dispatcher's own
    std::thread thread;
};

namespace {

int ensure(DevBuf &b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.cap >= bytes) return P2P_OK;
    const size_t want = std::max(bytes + bytes / 4, (size_t)256);
    if (b.p) CUDA_TRY(cudaFree(b.p));
    b.p = nullptr;
    b.cap = 0;
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        return fail(P2P_ERR_NOMEM, "server scratch cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
    }
    b.cap = want;
    return P2P_OK;
}

size_t particle_bytes(bool fp32) { return fp32 ? 68 : 52; }

size_t box_bytes(const p2p_server *S, const Box &b) {
    return particle_bytes(S->fp32) * (size_t)b.npart + 56 * ((size_t)b.nleaf + 1) + 4 * (size_t)b.ntask;
}

int grid_of(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 32));
}

// ---- residency ---------------------------------------------------------

void release_box(p2p_server *S, Box &b) {
    S->pa.release(b.P, b.npart);
    S->la.release(b.L, (int64_t)b.nleaf + 1);
    S->ra.release(b.R, b.ntask);
    b.resident = false;
    S->ds.resident_boxes--;
    S->ds.resident_bytes -= box_bytes(S, b);
}

bool try_alloc(p2p_server *S, Box &b) {
    int64_t P, L, R = 0;
    if (!S->pa.alloc(b.npart, &P)) return false;
    if (!S->la.alloc((int64_t)b.nleaf + 1, &L)) {
        S->pa.release(P, b.npart);
        return false;
    }
    if (b.ntask > 0 && !S->ra.alloc(b.ntask, &R)) {
        S->pa.release(P, b.npart);
        S->la.release(L, (int64_t)b.nleaf + 1);
        return false;
    }
    b.P = P;
    b.L = L;
    b.R = R;
    return true;
}

// Arena ranges for box id, evicting least recently used idle boxes that have
// no queued request. false: it does not fit now (retry after completions).
bool admit(p2p_server *S, int id) {
    Box &b = S->boxes[id];
    while (!try_alloc(S, b)) {
        int victim = -1;
        for (int k = 0; k < S->nbox_seen; ++k) {
            const Box &c = S->boxes[k];
            if (k == id || !c.resident || c.busy || c.pinned || c.pending > 0) continue;
            if (victim < 0 || c.last_use < S->boxes[victim].last_use) victim = k;
        }
        if (victim < 0) return false;
        release_box(S, S->boxes[victim]);
        S->ds.evictions++;
    }
    return true;
}

// Uploads and prepares box id into its arena ranges (build stream).
int build_box(p2p_server *S, int id) {
    Box &b = S->boxes[id];
    cudaStream_t st = S->build_stream;
    const int n = b.npart, nl = b.nleaf;
    const int64_t nt = b.ntask;
    P2P_TRY(ensure(S->st_pos, sizeof(double) * 3 * (size_t)n));
    P2P_TRY(ensure(S->st_ip, sizeof(int) * (size_t)nl));
    P2P_TRY(ensure(S->st_np, sizeof(int) * (size_t)nl));
    P2P_TRY(ensure(S->st_t, sizeof(int) * (size_t)std::max<int64_t>(nt, 1)));
    P2P_TRY(ensure(S->st_s, sizeof(int) * (size_t)std::max<int64_t>(nt, 1)));
    P2P_TRY(ensure(S->counts, sizeof(int) * (size_t)nl));
    P2P_TRY(ensure(S->tile_sums, sizeof(int64_t) * csr_tile_sums(nl)));
    P2P_TRY(ensure(S->keys_a, sizeof(int) * (size_t)std::max<int64_t>(nt, 1)));
    P2P_TRY(ensure(S->keys_b, sizeof(int) * (size_t)std::max<int64_t>(nt, 1)));
    P2P_TRY(ensure(S->vals_b, sizeof(int) * (size_t)std::max<int64_t>(nt, 1)));
    P2P_TRY(ensure(S->hist, sizeof(int) * csr_hist_len(nt)));
    P2P_TRY(ensure(S->hoffs, sizeof(int64_t) * (csr_hist_len(nt) + 1)));
    P2P_TRY(ensure(S->hsums, sizeof(int64_t) * csr_hsum_len(nt)));
    int launches = 0;
    CUDA_TRY(cudaEventRecord(S->b0, st));
    // positions, in kernel units
    CUDA_TRY(cudaMemcpyAsync(S->st_pos.p, b.pos, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice, st));
    scale_positions_kernel<<<grid_of(3 * (int64_t)n, 256), 256, 0, st>>>(
        (const double *)S->st_pos.p, n, b.length_scale, S->pos + b.P, S->Pcap);
    // leaf ranges, arena-global
    CUDA_TRY(cudaMemcpyAsync(S->st_ip.p, b.ip, sizeof(int) * (size_t)nl, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(S->st_np.p, b.np, sizeof(int) * (size_t)nl, cudaMemcpyHostToDevice, st));
    add_offset_kernel<<<grid_of(nl, 256), 256, 0, st>>>((int *)S->st_ip.p, nl, (int)b.P);
    int *status = (int *)S->ctrl.p;
    unsigned long long *pairs = (unsigned long long *)((char *)S->ctrl.p + 8);
    CUDA_TRY(cudaMemsetAsync(S->ctrl.p, 0, 16, st));
    const int wblocks = grid_of((int64_t)nl * 32, 256);
    const double c = 0.5 / S->shape.split_radius;
    if (!S->fp32)
        prep_plain_kernel<<<grid_of(nl, 256), 256, 0, st>>>((const int *)S->st_ip.p, (const int *)S->st_np.p,
                                                            (int)S->Pcap, nl, S->meta + b.L, status);
    else if (S->shape.form == P2P_FORM_NAIVE_FP32)
        prep_split_kernel<false><<<wblocks, 256, 0, st>>>(S->pos, nullptr, (const int *)S->st_ip.p,
                                                          (const int *)S->st_np.p, (int)S->Pcap, nl, c,
                                                          S->meta + b.L, S->pos4, status);
    else
        prep_split_kernel<true><<<wblocks, 256, 0, st>>>(S->pos, nullptr, (const int *)S->st_ip.p,
                                                         (const int *)S->st_np.p, (int)S->Pcap, nl, c,
                                                         S->meta + b.L, S->pos4, status);
    launches += 3;
    // CSR: box-local row offsets and source ids, then made arena-global
    if (nt > 0) {
        CUDA_TRY(cudaMemcpyAsync(S->st_t.p, b.tt, sizeof(int) * (size_t)nt, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(S->st_s.p, b.ts, sizeof(int) * (size_t)nt, cudaMemcpyHostToDevice, st));
        CsrBufs cb;
        cb.counts = (int *)S->counts.p;
        cb.row_off = S->row_off + b.L;
        cb.tile_sums = (int64_t *)S->tile_sums.p;
        cb.row_src = S->row_src + b.R;
        cb.keys_a = (int *)S->keys_a.p;
        cb.keys_b = (int *)S->keys_b.p;
        cb.vals_b = (int *)S->vals_b.p;
        cb.hist = (int *)S->hist.p;
        cb.hoffs = (int64_t *)S->hoffs.p;
        cb.hsums = (int64_t *)S->hsums.p;
        cb.pairs = pairs;
        cb.status = status;
        CUDA_TRY(enqueue_csr_build(st, nt, (const int *)S->st_t.p, (const int *)S->st_s.p, nl, S->meta + b.L,
                                   cb, &launches));
        add_offset64_kernel<<<grid_of((int64_t)nl + 1, 256), 256, 0, st>>>(S->row_off + b.L, (int64_t)nl + 1,
                                                                          b.R);
        add_offset_kernel<<<grid_of(nt, 256), 256, 0, st>>>(S->row_src + b.R, nt, (int)b.L);
        launches += 2;
    } else {
        CUDA_TRY(cudaMemsetAsync(S->row_off + b.L, 0, sizeof(int64_t) * ((size_t)nl + 1), st));
    }
    CUDA_TRY(cudaGetLastError());
    // returned particles (box-local slots), or every particle in slot order
    if (b.res_slots) {
        CUDA_TRY(cudaMemcpyAsync(S->rmap + b.P, b.res_slots, sizeof(int) * (size_t)b.nres, cudaMemcpyHostToDevice, st));
    } else {
        iota_kernel<<<grid_of(n, 256), 256, 0, st>>>(S->rmap + b.P, n);
        launches += 1;
    }
    CUDA_TRY(cudaMemcpyAsync(S->h_pairs, S->ctrl.p, 16, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaEventRecord(S->b1, st));
    CUDA_TRY(cudaEventRecord(b.ready, st));
    count_launches(launches);
    // The build's pair count is needed for the statistics and its status
    // for the input check: wait for it here (the dispatcher has nothing
    // else to issue for this box before it is ready).
    CUDA_TRY(cudaEventSynchronize(S->b1));
    const int st_bits = (int)(S->h_pairs[0] & 0xffffffff);
    if (st_bits) return fail(P2P_ERR_RANGE, "box %d: device check of leaf / list ranges failed (0x%x)", id, st_bits);
    b.pairs = S->h_pairs[1];
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, S->b0, S->b1));
    S->ds.build_ms += ms;
    S->ds.builds++;
    b.resident = true;
    S->ds.resident_boxes++;
    S->ds.resident_bytes += box_bytes(S, b);
    return P2P_OK;
}

// ---- launches ----------------------------------------------------------

void CUDART_CB on_kernel_done(void *p) {
    Launch *L = (Launch *)p;
    p2p_server *S = L->srv;
    {
        std::lock_guard<std::mutex> g(S->mu);
        L->kernel_done = true;
        S->epoch++;
    }
    S->cv_work.notify_all();
}

void CUDART_CB on_copy_done(void *p) {
    Launch *L = (Launch *)p;
    p2p_server *S = L->srv;
    {
        std::lock_guard<std::mutex> g(S->mu);
        L->copy_done = true;
        L->t_copy = Clock::now();
        S->epoch++;
    }
    S->cv_work.notify_all();
}

PairLaunchResult dispatch_pair(const p2p_params &p, const PairLaunch &L, const PairArgs &a) {
    if (p.form == P2P_FORM_PLAIN_FP64) return launch_pair_plain(L, a);
    if (p.kernel_variant == P2P_VARIANT_SINK_LANES) return launch_pair_sink_lanes(L, a);
    if (p.kernel_variant == P2P_VARIANT_SINK_LANES_X2) return launch_pair_sink_lanes_x2(L, a);
    // the default mapping is the sink-register kernel (28% more saturation
    // throughput than the source-lane kernel on the serving ensemble)
    if (p.kernel_variant == P2P_VARIANT_SINK_REGS || p.kernel_variant == P2P_VARIANT_SINK_REGS8 ||
        p.kernel_variant == P2P_VARIANT_AUTO) {
        PairLaunch L8 = L;
        L8.sreg_spl = p.kernel_variant == P2P_VARIANT_SINK_REGS8 ? 8 : 4;
        return launch_pair_sink_regs(L8, a);
    }
    if (p.kernel_variant == P2P_VARIANT_SOURCE_LANES) return launch_pair_source_lanes(L, a);
    return launch_pair_source_lanes_x2(L, a);
}

// One packed launch on slot sl: clear the boxes' accumulators, the pair
// kernel over their leaf ranges, gather the returned particles into the
// slot's staging buffer; the copy stream then moves each box's results to
// its caller's buffer.
int launch_pack(p2p_server *S, Slot &sl, const std::vector<Job> &jobs) {
    const p2p_params &p = S->shape;
    PairArgs a;
    std::memset(&a, 0, sizeof(a));
    fill_pass_scalars(a, p, S->fit, false);
    a.out_scale = (0.5 / p.split_radius) * (0.5 / p.split_radius);  // the box's mass comes in the gather
    a.leaf = S->meta;
    a.row_off = S->row_off;
    a.row_src = S->row_src;
    a.pos4 = S->pos4;
    a.pos = S->pos;
    a.mass = nullptr;
    a.acc = S->acc;
    a.queue = sl.d_queue;
    a.npart = (int)S->Pcap;
    OutArgs f;
    std::memset(&f, 0, sizeof(f));
    f.stride = S->Pcap;
    f.acc = S->acc;
    f.rmap = S->rmap;
    int items = 0, k = 0, maxn = 0, maxr = 0;
    int64_t pairs = 0, off = 0;
    for (const Job &j : jobs) {
        Box &b = S->boxes[j.box];
        CUDA_TRY(cudaStreamWaitEvent(sl.stream, b.ready, 0));
        a.seg_item[k] = items;
        a.seg_leaf[k] = (int)b.L;
        items += b.nleaf;
        f.seg[k].p0 = b.P;
        f.seg[k].n = b.npart;
        f.seg[k].nres = b.nres;
        f.seg[k].off = off;
        f.seg[k].scale = b.length_scale * b.length_scale * b.mass;
        off += 3 * (int64_t)b.nres;
        maxn = std::max(maxn, b.npart);
        maxr = std::max(maxr, b.nres);
        pairs += b.pairs;
        ++k;
    }
    a.nseg = k;
    a.seg_item[k] = items;
    a.nleaf = items;
    f.nseg = k;
    const int cur = sl.cur;
    P2P_TRY(ensure(sl.stage[cur], sizeof(double) * (size_t)std::max<int64_t>(off, 1)));
    f.stage = (double *)sl.stage[cur].p;
    PairLaunch L;
    L.stream = sl.stream;
    L.sm_count = S->sm_count;
    L.soft_mode = p.soft_mode == P2P_SOFT_CLAMP ? SOFT_CLAMP : SOFT_PLUMMER;
    L.masses = false;
    L.acc = p.form == P2P_FORM_KAHAN_FP32 ? ACC_KAHAN : (p.form == P2P_FORM_NAIVE_FP32 ? ACC_F32 : ACC_F64);
    L.ncoef = S->fit.ncoef_kernel;
    L.warps = p.warps_per_block ? p.warps_per_block : 4;
    L.stage = p.stage_sources ? p.stage_sources : (p.form == P2P_FORM_PLAIN_FP64 ? 128 : 256);
    L.blocks_per_sm = p.blocks_per_sm;
    L.dry_run = false;
    L.occ = &S->occ;
    L.max_blocks = 0;
    L.sink_pairs = p.kernel_variant == P2P_VARIANT_SOURCE_LANES_X2_S16 ? 8 : 16;
    if (!S->cfg.full_grid && S->cfg.slots > 1) {
        // a share of the resident blocks (the occupancy query runs once, dry)
        PairLaunch D = L;
        D.dry_run = true;
        const PairLaunchResult r0 = dispatch_pair(p, D, a);
        if (!r0.fits) return fail(P2P_ERR_ARG, "pair kernel does not fit on an SM with this launch shape");
        L.max_blocks = std::max(S->sm_count, r0.blocks / S->cfg.slots);
    }
    CUDA_TRY(cudaMemsetAsync(sl.d_queue, 0, sizeof(int), sl.stream));
    const dim3 cg((unsigned)std::min<int64_t>(std::max<int64_t>((3 * (int64_t)maxn + 255) / 256, 1), 128), k);
    clear_acc_kernel<<<cg, 256, 0, sl.stream>>>(f);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(sl.k0, sl.stream));
    const PairLaunchResult r = dispatch_pair(p, L, a);
    if (!r.fits) return fail(P2P_ERR_ARG, "pair kernel does not fit on an SM with this launch shape");
    if (r.cuda != cudaSuccess) return fail(P2P_ERR_CUDA, "pair kernel launch: %s", cudaGetErrorString(r.cuda));
    CUDA_TRY(cudaEventRecord(sl.k1, sl.stream));
    // the staging buffer's previous results must have left it
    if (sl.copied_used[cur]) CUDA_TRY(cudaStreamWaitEvent(sl.stream, sl.copied[cur], 0));
    const dim3 gg((unsigned)std::min<int64_t>(std::max<int64_t>((3 * (int64_t)maxr + 255) / 256, 1), 128), k);
    gather_results_kernel<<<gg, 256, 0, sl.stream>>>(f);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(sl.staged, sl.stream));
    Launch *rec = new Launch();
    rec->srv = S;
    rec->slot = &sl;
    rec->jobs = jobs;
    S->launches.push_back(rec);
    CUDA_TRY(cudaLaunchHostFunc(sl.stream, on_kernel_done, rec));
    CUDA_TRY(cudaStreamWaitEvent(sl.copy, sl.staged, 0));
    for (int q = 0; q < k; ++q)
        CUDA_TRY(cudaMemcpyAsync(jobs[q].out, f.stage + f.seg[q].off, sizeof(double) * 3 * (size_t)f.seg[q].nres,
                                 cudaMemcpyDeviceToHost, sl.copy));
    CUDA_TRY(cudaEventRecord(sl.copied[cur], sl.copy));
    sl.copied_used[cur] = true;
    CUDA_TRY(cudaLaunchHostFunc(sl.copy, on_copy_done, rec));
    count_launches(3);
    sl.cur ^= 1;
    sl.busy = true;
    S->ds.launches++;
    S->ds.boxes_launched += k;
    S->ds.pairs += pairs;
    return P2P_OK;
}

// Pair kernel and gather of a launch finished: its boxes and slot are free.
int retire_kernel(p2p_server *S, Launch &L) {
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, L.slot->k0, L.slot->k1));
    S->ds.kernel_ms += ms;
    for (const Job &j : L.jobs) S->boxes[j.box].busy = false;
    L.slot->busy = false;
    return P2P_OK;
}

// Results of a launch are in the callers' buffers: its requests are done.
void retire_copy(p2p_server *S, Launch &L) {
    {
        std::lock_guard<std::mutex> g(S->mu);
        for (const Job &j : L.jobs) {
            Request &r = S->reqs[j.ticket];
            r.t_done = L.t_copy;
            r.done = true;
            S->finished++;
        }
        S->ds.requests_done += (int64_t)L.jobs.size();
        S->stats = S->ds;
    }
    S->cv_done.notify_all();
}

void complete_request(p2p_server *S, int64_t ticket, int status) {
    {
        std::lock_guard<std::mutex> g(S->mu);
        Request &r = S->reqs[ticket];
        r.t_done = Clock::now();
        r.status = status;
        r.done = true;
        S->finished++;
    }
    S->cv_done.notify_all();
}

bool any_slot_busy(const p2p_server *S) {
    for (const Slot &sl : S->slots)
        if (sl.busy) return true;
    return false;
}

// Preload requests: resident and pinned, no pass. One that cannot be
// admitted waits for completions while launches are in flight.
int handle_preloads(p2p_server *S) {
    for (auto it = S->pending.begin(); it != S->pending.end();) {
        if (!it->preload) {
            ++it;
            continue;
        }
        Box &b = S->boxes[it->box];
        int st = P2P_OK;
        if (!b.resident) {
            if (!admit(S, it->box)) {
                if (any_slot_busy(S)) {
                    ++it;
                    continue;
                }
                st = fail(P2P_ERR_CAPACITY, "box %d does not fit beside the pinned and queued boxes", it->box);
            } else {
                P2P_TRY(build_box(S, it->box));
            }
        }
        if (st == P2P_OK) b.pinned = true;
        b.pending--;
        complete_request(S, it->ticket, st);
        it = S->pending.erase(it);
    }
    return P2P_OK;
}

// Batching window (cfg.batch_window_ms > 0): a pack launches at once when it
// would hold max_pack boxes or cfg.min_pack_pairs pair interactions, or when
// its oldest request has waited the window; until then the requests wait for
// others to share the launch, and hold_until tells the dispatcher when to
// look again. A box not yet built has no pair count and launches at once.
bool hold_for_window(p2p_server *S) {
    if (S->cfg.batch_window_ms <= 0.0 || S->flush) return false;
    std::vector<char> seen(S->nbox_seen, 0);
    int count = 0;
    double work = 0.0;
    Clock::time_point oldest = Clock::time_point::max();
    for (const Job &j : S->pending) {
        if (j.preload || S->boxes[j.box].busy || seen[j.box]) continue;
        seen[j.box] = 1;
        const Box &b = S->boxes[j.box];
        if (b.pairs <= 0) return false;
        work += (double)b.pairs;
        oldest = std::min(oldest, j.t_submit);
        if (++count >= S->cfg.max_pack) return false;
    }
    if (count == 0) return false;
    if (S->cfg.min_pack_pairs > 0.0 && work >= S->cfg.min_pack_pairs) return false;
    const auto until = oldest + std::chrono::duration_cast<Clock::duration>(
                                    std::chrono::duration<double, std::milli>(S->cfg.batch_window_ms));
    if (Clock::now() >= until) return false;
    S->hold_until = std::min(S->hold_until, until);
    return true;
}

// One scheduling round: admit and pack pending requests into free slots.
int schedule(p2p_server *S) {
    P2P_TRY(handle_preloads(S));
    S->hold_until = Clock::time_point::max();
    bool held = false;
    for (Slot &sl : S->slots) {
        if (sl.busy) continue;
        if ((held = hold_for_window(S))) break;
        std::vector<Job> pack;
        std::vector<char> taken(S->nbox_seen, 0);
        bool blocked = false;  // the oldest non-resident box did not fit: admit no later one
        for (auto it = S->pending.begin(); it != S->pending.end() && (int)pack.size() < S->cfg.max_pack;) {
            const Job j = *it;
            const int id = j.box;
            Box &b = S->boxes[id];
            if (j.preload || b.busy || taken[id]) {
                ++it;
                continue;
            }
            if (!b.resident) {
                if (blocked || !admit(S, id)) {
                    blocked = true;
                    ++it;
                    continue;
                }
                P2P_TRY(build_box(S, id));
            }
            taken[id] = 1;
            b.busy = true;
            b.pending--;
            b.last_use = ++S->use_clock;
            pack.push_back(j);
            it = S->pending.erase(it);
        }
        if (pack.empty()) break;
        P2P_TRY(launch_pack(S, sl, pack));
    }
    // Nothing in flight and nothing launched or held: the oldest request's box
    // cannot be admitted even with every evictable box gone.
    if (!held && !any_slot_busy(S)) {
        for (auto it = S->pending.begin(); it != S->pending.end(); ++it) {
            if (it->preload) continue;
            S->boxes[it->box].pending--;
            complete_request(S, it->ticket,
                             fail(P2P_ERR_CAPACITY, "box %d does not fit beside the pinned and queued boxes",
                                  it->box));
            S->pending.erase(it);
            break;
        }
    }
    return P2P_OK;
}

void dispatcher(p2p_server *S) {
    cudaSetDevice(S->device);
    uint64_t seen = 0;
    for (;;) {
        std::vector<Launch *> kdone, cdone;
        bool stopping;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            auto ready = [&] { return S->stop || !S->incoming.empty() || S->epoch != seen; };
            if (S->hold_until == Clock::time_point::max())
                S->cv_work.wait(lk, ready);
            else
                S->cv_work.wait_until(lk, S->hold_until, ready);
            seen = S->epoch;
            S->nbox_seen = (int)S->boxes.size();
            while (!S->incoming.empty()) {
                const Job j = S->incoming.front();
                S->incoming.pop_front();
                S->pending.push_back(j);
                S->boxes[j.box].pending++;
            }
            for (Launch *L : S->launches) {
                if (L->kernel_done && !L->kernel_seen) {
                    L->kernel_seen = true;
                    kdone.push_back(L);
                }
                if (L->kernel_seen && L->copy_done) cdone.push_back(L);
            }
            stopping = S->stop;
            if (S->set_window_ms >= 0.0) {
                S->cfg.batch_window_ms = S->set_window_ms;
                S->cfg.min_pack_pairs = S->set_min_pairs;
                S->set_window_ms = -1.0;
            }
        }
        S->flush = stopping;
        int st = P2P_OK;
        for (Launch *L : kdone)
            if (st == P2P_OK) st = retire_kernel(S, *L);
        for (Launch *L : cdone) {
            retire_copy(S, *L);
            S->launches.erase(std::find(S->launches.begin(), S->launches.end(), L));
            delete L;
        }
        if (st == P2P_OK && S->error == P2P_OK) st = schedule(S);
        if (st != P2P_OK) {
            std::lock_guard<std::mutex> g(S->mu);
            if (S->error == P2P_OK) {
                S->error = st;
                S->error_msg = p2p_last_error();
            }
            // fail every request that can no longer finish
            for (const Job &j : S->pending) {
                S->reqs[j.ticket].done = true;
                S->finished++;
            }
            S->pending.clear();
        }
        {
            std::lock_guard<std::mutex> g(S->mu);
            S->stats = S->ds;
        }
        if (S->error != P2P_OK) S->cv_done.notify_all();
        if (stopping && S->launches.empty() && S->pending.empty()) {
            std::lock_guard<std::mutex> g(S->mu);
            if (S->incoming.empty()) break;
        }
        if (stopping && S->error != P2P_OK) break;
    }
}

int check_server(p2p_server *S) {
    if (!S) return fail(P2P_ERR_ARG, "null server");
    CUDA_TRY(cudaSetDevice(S->device));
    return P2P_OK;
}

void free_server(p2p_server *S) {
    for (Slot &sl : S->slots) {
        if (sl.stream) cudaStreamDestroy(sl.stream);
        if (sl.copy) cudaStreamDestroy(sl.copy);
        cudaEvent_t evs[] = {sl.k0, sl.k1, sl.staged, sl.copied[0], sl.copied[1]};
        for (cudaEvent_t e : evs)
            if (e) cudaEventDestroy(e);
        for (DevBuf &b : sl.stage)
            if (b.p) cudaFree(b.p);
        if (sl.d_queue) cudaFree(sl.d_queue);
    }
    for (Launch *L : S->launches) delete L;
    for (Box &b : S->boxes)
        if (b.ready) cudaEventDestroy(b.ready);
    DevBuf *bufs[] = {&S->st_pos, &S->st_ip, &S->st_np, &S->st_t, &S->st_s, &S->counts, &S->tile_sums,
                      &S->keys_a, &S->keys_b, &S->vals_b, &S->hist, &S->hoffs, &S->hsums, &S->ctrl};
    for (DevBuf *b : bufs)
        if (b->p) cudaFree(b->p);
    if (S->arena) cudaFree(S->arena);
    if (S->h_pairs) cudaFreeHost(S->h_pairs);
    if (S->build_stream) cudaStreamDestroy(S->build_stream);
    if (S->b0) cudaEventDestroy(S->b0);
    if (S->b1) cudaEventDestroy(S->b1);
    delete S;
}

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace

// ------------------------------------------------------------------ ABI ---

P2P_API void p2p_server_config_default(p2p_server_config *cfg) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->slots = 1;
    cfg->max_pack = kMaxSeg;
    cfg->full_grid = 1;
    cfg->hbm_bytes = 0;
    cfg->rows_per_particle = 24.0;
    cfg->particles_per_leaf = 16.0;
}

P2P_API int p2p_server_create(int device, const p2p_params *shape, const p2p_server_config *cfg,
                              p2p_server **out) {
    if (!out || !shape) return fail(P2P_ERR_ARG, "null argument");
    *out = nullptr;
    P2P_TRY(check_params(shape));
    int ndev = 0;
    CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(P2P_ERR_ARG, "device %d of %d", device, ndev);
    CUDA_TRY(cudaSetDevice(device));
    p2p_server_config c;
    p2p_server_config_default(&c);
    if (cfg) {
        if (cfg->slots < 0 || cfg->slots > 16) return fail(P2P_ERR_ARG, "slots must be in [0, 16]");
        if (cfg->max_pack < 0 || cfg->max_pack > kMaxSeg) return fail(P2P_ERR_ARG, "max_pack must be in [0, %d]", kMaxSeg);
        if (cfg->rows_per_particle < 0 || cfg->particles_per_leaf < 0) return fail(P2P_ERR_ARG, "negative sizing hint");
        if (cfg->slots) c.slots = cfg->slots;
        if (cfg->max_pack) c.max_pack = cfg->max_pack;
        c.full_grid = cfg->full_grid;
        c.hbm_bytes = cfg->hbm_bytes;
        if (cfg->rows_per_particle > 0) c.rows_per_particle = cfg->rows_per_particle;
        if (!(cfg->batch_window_ms >= 0.0) || !(cfg->min_pack_pairs >= 0.0) || cfg->batch_window_ms > 1e4)
            return fail(P2P_ERR_ARG, "batch_window_ms must be in [0, 1e4] and min_pack_pairs >= 0");
        c.batch_window_ms = cfg->batch_window_ms;
        c.min_pack_pairs = cfg->min_pack_pairs;
        if (cfg->particles_per_leaf > 0) c.particles_per_leaf = std::max(1.0, cfg->particles_per_leaf);
    }
    p2p_server *S = new p2p_server();
    S->device = device;
    S->shape = *shape;
    S->shape.mass = 1.0;
    S->cfg = c;
    S->fp32 = shape->form != P2P_FORM_PLAIN_FP64;
    if (S->fp32)
        S->fit = fit_h(fit_umax(shape->x_cut), shape->poly_tol > 0.0 ? shape->poly_tol : kDefaultPolyTol);
    auto cleanup = [&](int st) {
        free_server(S);
        return st;
    };
    cudaError_t e = cudaDeviceGetAttribute(&S->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = allow_large_smem();
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->build_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&S->b0);
    if (e == cudaSuccess) e = cudaEventCreate(&S->b1);
    if (e == cudaSuccess) e = cudaHostAlloc((void **)&S->h_pairs, 16, cudaHostAllocDefault);
    if (e != cudaSuccess) return cleanup(fail(P2P_ERR_CUDA, "server setup: %s", cudaGetErrorString(e)));
    // arena
    size_t budget = c.hbm_bytes;
    if (!budget) {
        size_t fr = 0, tot = 0;
        e = cudaMemGetInfo(&fr, &tot);
        if (e != cudaSuccess) return cleanup(fail(P2P_ERR_CUDA, "cudaMemGetInfo: %s", cudaGetErrorString(e)));
        budget = fr / 2;
    }
    const double per_particle = (double)particle_bytes(S->fp32) + 56.0 / c.particles_per_leaf +
                                4.0 * c.rows_per_particle;
    S->Pcap = std::min<int64_t>((int64_t)((double)budget / per_particle), (int64_t)1 << 30);
    S->Lcap = std::min<int64_t>((int64_t)((double)S->Pcap / c.particles_per_leaf) + 4096, (int64_t)1 << 30);
    S->Rcap = std::min<int64_t>((int64_t)((double)S->Pcap * c.rows_per_particle), (int64_t)1 << 38);
    if (S->Pcap < 1024) return cleanup(fail(P2P_ERR_ARG, "hbm_bytes %zu is too small", budget));
    const size_t o_pos = 0;
    const size_t o_acc = o_pos + align256(sizeof(double) * 3 * (size_t)S->Pcap);
    const size_t o_pos4 = o_acc + align256(sizeof(double) * 3 * (size_t)S->Pcap);
    const size_t o_meta = o_pos4 + (S->fp32 ? align256(sizeof(float4) * (size_t)S->Pcap) : 0);
    const size_t o_roff = o_meta + align256(sizeof(LeafMeta) * (size_t)S->Lcap);
    const size_t o_rsrc = o_roff + align256(sizeof(int64_t) * (size_t)S->Lcap);
    const size_t o_rmap = o_rsrc + align256(sizeof(int) * (size_t)S->Rcap);
    S->arena_bytes = o_rmap + align256(sizeof(int) * (size_t)S->Pcap);
    e = cudaMalloc(&S->arena, S->arena_bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        S->arena = nullptr;
        return cleanup(fail(P2P_ERR_NOMEM, "arena cudaMalloc(%zu) failed: %s", S->arena_bytes, cudaGetErrorString(e)));
    }
    char *base = (char *)S->arena;
    S->pos = (double *)(base + o_pos);
    S->acc = (double *)(base + o_acc);
    S->pos4 = S->fp32 ? (float4 *)(base + o_pos4) : nullptr;
    S->meta = (LeafMeta *)(base + o_meta);
    S->row_off = (int64_t *)(base + o_roff);
    S->row_src = (int *)(base + o_rsrc);
    S->rmap = (int *)(base + o_rmap);
    S->pa.reset(S->Pcap);
    S->la.reset(S->Lcap);
    S->ra.reset(S->Rcap);
    S->ds.capacity_bytes = S->arena_bytes;
    S->stats = S->ds;
    S->boxes.reserve(kMaxBoxes);
    if (ensure(S->ctrl, 16) != P2P_OK) return cleanup(P2P_ERR_NOMEM);
    S->slots.resize(c.slots);
    for (Slot &sl : S->slots) {
        e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sl.copy, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreate(&sl.k0);
        if (e == cudaSuccess) e = cudaEventCreate(&sl.k1);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.staged, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.copied[0], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.copied[1], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMalloc(&sl.d_queue, 256);
        if (e != cudaSuccess) return cleanup(fail(P2P_ERR_CUDA, "slot setup: %s", cudaGetErrorString(e)));
    }
    S->thread = std::thread(dispatcher, S);
    *out = S;
    return P2P_OK;
}

P2P_API int p2p_server_destroy(p2p_server *S) {
    if (!S) return P2P_OK;
    {
        std::lock_guard<std::mutex> g(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    if (S->thread.joinable()) S->thread.join();
    cudaSetDevice(S->device);
    for (Slot &sl : S->slots) {
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        if (sl.copy) cudaStreamSynchronize(sl.copy);
    }
    if (S->build_stream) cudaStreamSynchronize(S->build_stream);
    free_server(S);
    return P2P_OK;
}

P2P_API int p2p_server_add_box(p2p_server *S, double length_scale, double mass, int npart,
                               const double *pos, int nleaf, const int *leaf_ipart,
                               const int *leaf_npart, int64_t ntask, const int *task_t,
                               const int *task_s, int nresult, const int *result_slots,
                               int *box_id) {
    P2P_TRY(check_server(S));
    if (!box_id) return fail(P2P_ERR_ARG, "null box_id");
    if (npart <= 0 || nleaf <= 0 || ntask < 0) return fail(P2P_ERR_ARG, "box needs particles and leaves");
    if (!pos || !leaf_ipart || !leaf_npart || (ntask > 0 && (!task_t || !task_s)))
        return fail(P2P_ERR_ARG, "null input array");
    if (!(length_scale > 0.0) || !std::isfinite(length_scale) || !std::isfinite(mass))
        return fail(P2P_ERR_ARG, "length_scale must be positive and mass finite");
    for (int l = 0; l < nleaf; ++l) {
        const int64_t ip = leaf_ipart[l], np = leaf_npart[l];
        if (ip < 0 || np < 0 || ip + np > npart)
            return fail(P2P_ERR_RANGE, "leaf %d: particle range [%lld, %lld) outside [0, %d)", l, (long long)ip,
                        (long long)(ip + np), npart);
    }
    for (int64_t e = 0; e < ntask; ++e)
        if (task_t[e] < 0 || task_t[e] >= nleaf || task_s[e] < 0 || task_s[e] >= nleaf)
            return fail(P2P_ERR_RANGE, "list entry %lld names a leaf outside [0, %d)", (long long)e, nleaf);
    if (result_slots) {
        if (nresult < 0 || nresult > npart) return fail(P2P_ERR_ARG, "nresult must be in [0, npart]");
        for (int r = 0; r < nresult; ++r)
            if (result_slots[r] < 0 || result_slots[r] >= npart)
                return fail(P2P_ERR_RANGE, "result %d names particle slot %d outside [0, %d)", r, result_slots[r], npart);
    }
    if (npart > S->Pcap || (int64_t)nleaf + 1 > S->Lcap || ntask > S->Rcap)
        return fail(P2P_ERR_CAPACITY,
                    "box (%d particles, %d leaves, %lld entries) exceeds the arena (%lld, %lld, %lld)", npart,
                    nleaf, (long long)ntask, (long long)S->Pcap, (long long)S->Lcap, (long long)S->Rcap);
    Box b;
    b.length_scale = length_scale;
    b.mass = mass;
    b.npart = npart;
    b.nleaf = nleaf;
    b.ntask = ntask;
    b.pos = pos;
    b.ip = leaf_ipart;
    b.np = leaf_npart;
    b.tt = task_t;
    b.ts = task_s;
    b.res_slots = result_slots;
    b.nres = result_slots ? nresult : npart;
    CUDA_TRY(cudaEventCreateWithFlags(&b.ready, cudaEventDisableTiming));
    std::lock_guard<std::mutex> g(S->mu);
    if ((int)S->boxes.size() >= kMaxBoxes) {
        cudaEventDestroy(b.ready);
        return fail(P2P_ERR_CAPACITY, "a server holds at most %d boxes", kMaxBoxes);
    }
    *box_id = (int)S->boxes.size();
    S->boxes.push_back(b);
    return P2P_OK;
}

P2P_API int p2p_server_box_bytes(p2p_server *S, int box_id, size_t *bytes) {
    if (!S || !bytes) return fail(P2P_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(S->mu);
    if (box_id < 0 || box_id >= (int)S->boxes.size()) return fail(P2P_ERR_ARG, "unknown box %d", box_id);
    *bytes = box_bytes(S, S->boxes[box_id]);
    return P2P_OK;
}

P2P_API int p2p_server_submit(p2p_server *S, int box_id, double *out, int64_t *ticket) {
    P2P_TRY(check_server(S));
    if (!out || !ticket) return fail(P2P_ERR_ARG, "null argument");
    cudaPointerAttributes attr;
    CUDA_TRY(cudaPointerGetAttributes(&attr, out));
    if (attr.type != cudaMemoryTypeHost)
        return fail(P2P_ERR_ARG, "out must be page-locked host memory (p2p_host_alloc)");
    const auto now = Clock::now();
    {
        std::lock_guard<std::mutex> g(S->mu);
        if (S->error != P2P_OK) return fail(S->error, "server failed earlier: %s", S->error_msg.c_str());
        if (box_id < 0 || box_id >= (int)S->boxes.size()) return fail(P2P_ERR_ARG, "unknown box %d", box_id);
        Request r;
        r.box = box_id;
        r.out = out;
        r.t_submit = now;
        *ticket = (int64_t)S->reqs.size();
        S->reqs.push_back(r);
        S->incoming.push_back(Job{*ticket, box_id, out, false, now});
        S->submitted++;
    }
    S->cv_work.notify_all();
    return P2P_OK;
}

P2P_API int p2p_server_preload(p2p_server *S, int box_id) {
    P2P_TRY(check_server(S));
    int64_t ticket;
    {
        std::lock_guard<std::mutex> g(S->mu);
        if (S->error != P2P_OK) return fail(S->error, "server failed earlier: %s", S->error_msg.c_str());
        if (box_id < 0 || box_id >= (int)S->boxes.size()) return fail(P2P_ERR_ARG, "unknown box %d", box_id);
        Request r;
        r.box = box_id;
        r.t_submit = Clock::now();
        ticket = (int64_t)S->reqs.size();
        S->reqs.push_back(r);
        S->incoming.push_back(Job{ticket, box_id, nullptr, true, r.t_submit});
        S->submitted++;
    }
    S->cv_work.notify_all();
    return p2p_server_wait(S, ticket, nullptr);
}

P2P_API int p2p_server_query(p2p_server *S, int64_t ticket, int *done, double *latency_s) {
    if (!S || !done) return fail(P2P_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(S->mu);
    if (ticket < 0 || ticket >= (int64_t)S->reqs.size()) return fail(P2P_ERR_ARG, "unknown ticket");
    const Request &r = S->reqs[ticket];
    *done = r.done ? 1 : 0;
    if (r.done && S->error != P2P_OK && r.t_done == Clock::time_point())
        return fail(S->error, "server failed: %s", S->error_msg.c_str());
    if (r.done && r.status != P2P_OK) return fail(r.status, "request %lld failed", (long long)ticket);
    if (latency_s) *latency_s = r.done ? std::chrono::duration<double>(r.t_done - r.t_submit).count() : 0.0;
    return P2P_OK;
}

P2P_API int p2p_server_wait(p2p_server *S, int64_t ticket, double *latency_s) {
    if (!S) return fail(P2P_ERR_ARG, "null server");
    std::unique_lock<std::mutex> lk(S->mu);
    if (ticket < 0 || ticket >= (int64_t)S->reqs.size()) return fail(P2P_ERR_ARG, "unknown ticket");
    S->cv_done.wait(lk, [&] { return S->reqs[ticket].done || S->error != P2P_OK; });
    const Request &r = S->reqs[ticket];
    if (!r.done || r.t_done == Clock::time_point())
        return fail(S->error, "server failed: %s", S->error_msg.c_str());
    if (r.status != P2P_OK) return fail(r.status, "request %lld: box does not fit in the arena", (long long)ticket);
    if (latency_s) *latency_s = std::chrono::duration<double>(r.t_done - r.t_submit).count();
    return P2P_OK;
}

P2P_API int p2p_server_set_batching(p2p_server *S, double batch_window_ms, double min_pack_pairs) {
    if (!S) return fail(P2P_ERR_ARG, "null server");
    if (!(batch_window_ms >= 0.0) || batch_window_ms > 1e4 || !(min_pack_pairs >= 0.0))
        return fail(P2P_ERR_ARG, "batch_window_ms must be in [0, 1e4] and min_pack_pairs >= 0");
    {
        std::lock_guard<std::mutex> g(S->mu);
        S->set_window_ms = batch_window_ms;
        S->set_min_pairs = min_pack_pairs;
        S->epoch++;
    }
    S->cv_work.notify_all();
    return P2P_OK;
}

P2P_API int p2p_server_drain(p2p_server *S) {
    if (!S) return fail(P2P_ERR_ARG, "null server");
    std::unique_lock<std::mutex> lk(S->mu);
    S->cv_done.wait(lk, [&] { return S->finished >= S->submitted || S->error != P2P_OK; });
    if (S->error != P2P_OK) return fail(S->error, "server failed: %s", S->error_msg.c_str());
    return P2P_OK;
}

P2P_API int p2p_server_get_stats(p2p_server *S, p2p_server_stats *stats) {
    if (!S || !stats) return fail(P2P_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(S->mu);
    *stats = S->stats;
    return P2P_OK;
}

P2P_API int p2p_host_alloc(size_t bytes, void **ptr) {
    if (!ptr) return fail(P2P_ERR_ARG, "null ptr");
    *ptr = nullptr;
    CUDA_TRY(cudaHostAlloc(ptr, bytes ? bytes : 16, cudaHostAllocMapped | cudaHostAllocPortable));
    return P2P_OK;
}

P2P_API int p2p_host_free(void *ptr) {
    if (ptr) CUDA_TRY(cudaFreeHost(ptr));
    return P2P_OK;
}
