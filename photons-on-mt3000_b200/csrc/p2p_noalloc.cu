// p2p_pass_noalloc: the whole P2P force pass without any device allocation.
//
// Who needs it: host codes that cannot let a library call cudaMalloc or
// cudaFree while they run. Examples are a simulation that reserves nearly all
// of the GPU's memory for its own pool at start-up (a library allocation
// then fails, or fragments the pool), a process held to a fixed device-memory
// quota on a shared GPU, and a code that runs other work on its own streams
// meanwhile (cudaFree synchronises the whole device and would stall those
// streams; this call waits for its own stream only). For them
// the scratch this pass needs lives in one file-scope __device__ array of a
// fixed size, P2P_NOALLOC_SCRATCH_BYTES, that every GPU loading the library
// holds until the process exits. The caller passes inputs and the output.
//
// The same kernels as the session path run here (frame prep, CSR build with
// sorted rows, pair kernel); this file only lays the scratch out in the
// static array and launches them on the caller's stream.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "photons_p2p.h"
#include "p2p_fit.h"
#include "p2p_args.h"
#include "p2p_internal.h"

// This file's own instance of the pass kernels: the header is compiled into
// a private namespace so its non-template kernels do not collide with the
// session path's copies at link time.
namespace p2p_noalloc_kernels {
using namespace ::p2p;
#include "p2p_kernels.cuh"
}  // namespace p2p_noalloc_kernels

#define P2P_API extern "C" __attribute__((visibility("default")))

namespace p2p {
namespace {

using namespace ::p2p_noalloc_kernels::p2p;

constexpr int kMaxDevices = 64;

// The scratch. Host code must not use this symbol as a device address: it
// is a host-side stand-in. The device address is obtained once per device
// with cudaGetSymbolAddress (noalloc_setup).
static __device__ __align__(256) unsigned char g_noalloc_scratch[P2P_NOALLOC_SCRATCH_BYTES];

std::mutex g_setup_mutex;
unsigned char *g_scratch_addr[kMaxDevices] = {nullptr};

// Last polynomial fit, reused while x_cut and the tolerance stay the same
// (no allocation).
std::mutex g_fit_mutex;
double g_fit_xcut = -1.0, g_fit_tol = -1.0;
PolyFit g_fit;

constexpr size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

struct Layout {
    size_t meta, pos4, counts, fill, row_off, tile_sums, row_src, ctrl, total;
};

// Offsets of every scratch piece; total is what the pass needs.
Layout layout(bool fp32, int npart, int nleaf, int64_t ntask) {
    Layout L;
    size_t off = 0;
    const size_t ntiles = ((size_t)nleaf + kScanTile - 1) / kScanTile + 1;
    L.meta = off;      off += align256(sizeof(LeafMeta) * (size_t)nleaf);
    L.pos4 = off;      off += fp32 ? align256(sizeof(float4) * (size_t)npart) : 0;
    L.counts = off;    off += align256(sizeof(int) * (size_t)nleaf);
    L.fill = off;      off += align256(sizeof(int) * (size_t)nleaf);
    L.row_off = off;   off += align256(sizeof(int64_t) * ((size_t)nleaf + 1));
    L.tile_sums = off; off += align256(sizeof(int64_t) * ntiles);
    L.row_src = off;   off += align256(sizeof(int) * (size_t)(ntask > 0 ? ntask : 1));
    L.ctrl = off;      off += 256;  // status (int), queue (int), pairs (u64)
    L.total = off;
    return L;
}

template <int SOFT, int NC>
cudaError_t allow_smem() {
    cudaError_t e = cudaFuncSetAttribute((const void *)pair_split_src2_kernel<SOFT, false, ACC_F64, NC>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    return e;
}

// Once per device, with that device current: resolve the scratch address and
// opt the pair kernels of this file into large dynamic shared memory.
int noalloc_setup(int dev, unsigned char **addr) {
    if (dev < 0 || dev >= kMaxDevices) return P2P_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return P2P_ERR_CUDA;
        }
        cudaError_t e = cudaSuccess;
        const void *plain[] = {(const void *)pair_plain_kernel<SOFT_CLAMP, false>,
                               (const void *)pair_plain_kernel<SOFT_PLUMMER, false>};
        for (const void *k : plain)
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
#define P2P_ALLOW(NCV)                                                         \
    if (e == cudaSuccess) e = allow_smem<SOFT_CLAMP, NCV>();                   \
    if (e == cudaSuccess) e = allow_smem<SOFT_PLUMMER, NCV>();
        P2P_ALLOW(9) P2P_ALLOW(11) P2P_ALLOW(13) P2P_ALLOW(15) P2P_ALLOW(17) P2P_ALLOW(21)
#undef P2P_ALLOW
        if (e != cudaSuccess) {
            cudaGetLastError();
            return P2P_ERR_CUDA;
        }
        g_scratch_addr[dev] = (unsigned char *)p;
    }
    *addr = g_scratch_addr[dev];
    return P2P_OK;
}

int grid_cap(int64_t n, int threads, int cap) {
    int64_t b = (n + threads - 1) / threads;
    return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

// The persistent pair kernel's launch: with blocks == 0 it only resolves the
// grid (resident blocks per SM times SMs) into *blocks; otherwise it launches.
template <class K>
int launch_persistent(K kernel, int sms, int warps, size_t smem, cudaStream_t st,
                      const PairArgs &a, int stage, int *blocks) {
    if (*blocks == 0) {
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, warps * 32, smem) != cudaSuccess ||
            per_sm < 1) {
            cudaGetLastError();
            return P2P_ERR_ARG;
        }
        *blocks = per_sm * sms;
        return P2P_OK;
    }
    kernel<<<*blocks, warps * 32, smem, st>>>(a, stage);
    return cudaGetLastError() == cudaSuccess ? P2P_OK : P2P_ERR_CUDA;
}

template <int SOFT>
int launch_split(int nc, int sms, int warps, size_t smem, cudaStream_t st, const PairArgs &a,
                 int stage, int *blocks) {
    switch (nc) {
        case 9: return launch_persistent(pair_split_src2_kernel<SOFT, false, ACC_F64, 9>, sms, warps, smem, st, a, stage, blocks);
        case 11: return launch_persistent(pair_split_src2_kernel<SOFT, false, ACC_F64, 11>, sms, warps, smem, st, a, stage, blocks);
        case 13: return launch_persistent(pair_split_src2_kernel<SOFT, false, ACC_F64, 13>, sms, warps, smem, st, a, stage, blocks);
        case 15: return launch_persistent(pair_split_src2_kernel<SOFT, false, ACC_F64, 15>, sms, warps, smem, st, a, stage, blocks);
        case 17: return launch_persistent(pair_split_src2_kernel<SOFT, false, ACC_F64, 17>, sms, warps, smem, st, a, stage, blocks);
        case 21: return launch_persistent(pair_split_src2_kernel<SOFT, false, ACC_F64, 21>, sms, warps, smem, st, a, stage, blocks);
        default: return P2P_ERR_STATE;
    }
}

// The pair kernel of these parameters (blocks == 0: resolve the grid only).
int launch_pair_kernel(bool fp32, const p2p_params &p, int nc, int sms, int warps, size_t smem, cudaStream_t s,
                       const PairArgs &a, int stage, int *blocks) {
    if (fp32)
        return p.soft_mode == P2P_SOFT_CLAMP ? launch_split<SOFT_CLAMP>(nc, sms, warps, smem, s, a, stage, blocks)
                                             : launch_split<SOFT_PLUMMER>(nc, sms, warps, smem, s, a, stage, blocks);
    return p.soft_mode == P2P_SOFT_CLAMP
               ? launch_persistent(pair_plain_kernel<SOFT_CLAMP, false>, sms, warps, smem, s, a, stage, blocks)
               : launch_persistent(pair_plain_kernel<SOFT_PLUMMER, false>, sms, warps, smem, s, a, stage, blocks);
}

// An error after work was queued: the call still returns only once that work
// (which writes the shared scratch) has finished on the stream.
int fail_after_queue(cudaStream_t s, int status) {
    cudaGetLastError();
    cudaStreamSynchronize(s);
    cudaGetLastError();
    return status;
}

}  // namespace
}  // namespace p2p

using namespace p2p;

// See include/photons_p2p.h for the contract.
P2P_API int p2p_pass_noalloc(const p2p_params *params, int npart, const double *d_pos, int nleaf,
                             const int *d_leaf_ipart, const int *d_leaf_npart, int64_t ntask,
                             const int *d_task_t, const int *d_task_s, double *d_acc,
                             void *stream) {
    if (!params) return P2P_ERR_ARG;
    const p2p_params &p = *params;
    if (p.form != P2P_FORM_SPLIT && p.form != P2P_FORM_PLAIN_FP64) return P2P_ERR_ARG;
    if (p.soft_mode != P2P_SOFT_CLAMP && p.soft_mode != P2P_SOFT_PLUMMER) return P2P_ERR_ARG;
    // the session's checks of the numeric fields (p2p_session_set_params)
    if (!(p.soften > 0.0) || !std::isfinite(p.soften)) return P2P_ERR_ARG;
    if (!(p.split_radius > 0.0) || !std::isfinite(p.split_radius)) return P2P_ERR_ARG;
    if (!std::isfinite(p.x_cut) || !std::isfinite(p.mass)) return P2P_ERR_ARG;
    if (!(p.poly_tol >= 0.0) || !std::isfinite(p.poly_tol)) return P2P_ERR_ARG;
    if (npart < 0 || nleaf < 0 || ntask < 0) return P2P_ERR_ARG;
    if ((npart > 0 && (!d_pos || !d_acc)) || (nleaf > 0 && (!d_leaf_ipart || !d_leaf_npart)) ||
        (ntask > 0 && (!d_task_t || !d_task_s)))
        return P2P_ERR_ARG;
    const bool fp32 = p.form == P2P_FORM_SPLIT;
    const Layout L = layout(fp32, npart, nleaf, ntask);
    if (L.total > (size_t)P2P_NOALLOC_SCRATCH_BYTES) return P2P_ERR_CAPACITY;
    const int warps = 4;
    const int stage = p.stage_sources ? p.stage_sources : (fp32 ? 256 : 128);
    if (stage % 32 || stage > 1024) return P2P_ERR_ARG;
    const size_t smem = fp32 ? (size_t)warps * (stage + 64 + stage / 4) * sizeof(float4)
                             : (size_t)warps * stage * sizeof(double4);
    if (smem > (size_t)227 * 1024) return P2P_ERR_ARG;

    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return P2P_ERR_CUDA;
    }
    unsigned char *base = nullptr;
    int st = noalloc_setup(dev, &base);
    if (st != P2P_OK) return st;

    PolyFit fit;
    if (fp32) {
        std::lock_guard<std::mutex> lock(g_fit_mutex);
        const double tol = p.poly_tol > 0.0 ? p.poly_tol : kDefaultPolyTol;
        if (g_fit_xcut != p.x_cut || g_fit_tol != tol) {
            g_fit = fit_h(fit_umax(p.x_cut), tol);
            g_fit_xcut = p.x_cut;
            g_fit_tol = tol;
        }
        fit = g_fit;
    }

    cudaStream_t s = (cudaStream_t)stream;
    // the pair kernel's grid, and that the fit has an instantiated degree,
    // before anything is queued
    int blocks = 0;
    {
        PairArgs probe;
        memset(&probe, 0, sizeof(probe));
        st = launch_pair_kernel(fp32, p, fit.ncoef_kernel, sms, warps, smem, s, probe, stage, &blocks);
        if (st != P2P_OK) return st;
    }
    LeafMeta *meta = (LeafMeta *)(base + L.meta);
    float4 *pos4 = (float4 *)(base + L.pos4);
    int *counts = (int *)(base + L.counts);
    int *fill = (int *)(base + L.fill);
    int64_t *row_off = (int64_t *)(base + L.row_off);
    int64_t *tiles = (int64_t *)(base + L.tile_sums);
    int *row_src = (int *)(base + L.row_src);
    int *status = (int *)(base + L.ctrl);
    int *queue = status + 1;
    unsigned long long *pairs = (unsigned long long *)(base + L.ctrl + 8);

    // Every call shares the scratch: clear what must start at zero.
    bool ok = cudaMemsetAsync(base + L.ctrl, 0, 16, s) == cudaSuccess;
    if (npart) ok = ok && cudaMemsetAsync(d_acc, 0, sizeof(double) * 3 * (size_t)npart, s) == cudaSuccess;
    if (nleaf) {
        ok = ok && cudaMemsetAsync(counts, 0, sizeof(int) * (size_t)nleaf, s) == cudaSuccess;
        ok = ok && cudaMemsetAsync(fill, 0, sizeof(int) * (size_t)nleaf, s) == cudaSuccess;
    }
    if (!ok) return fail_after_queue(s, P2P_ERR_CUDA);
    if (nleaf == 0 || ntask == 0) {
        // nothing to sum: the zeroed output is the result
        return cudaStreamSynchronize(s) == cudaSuccess ? P2P_OK : fail_after_queue(s, P2P_ERR_CUDA);
    }
    const double c = 0.5 / p.split_radius;
    const int threads = 256;
    if (fp32)
        prep_split_kernel<true><<<grid_cap((int64_t)nleaf * 32, threads, 65535), threads, 0, s>>>(
            d_pos, nullptr, d_leaf_ipart, d_leaf_npart, npart, nleaf, c, meta, pos4, status);
    else
        prep_plain_kernel<<<grid_cap(nleaf, threads, 65535), threads, 0, s>>>(
            d_leaf_ipart, d_leaf_npart, npart, nleaf, meta, status);
    const int eblocks = grid_cap(ntask, threads, sms * 16);
    csr_count_kernel<<<eblocks, threads, 0, s>>>(d_task_t, d_task_s, ntask, nleaf, meta, counts,
                                                 pairs, status, nullptr, 1.0, 0.f);
    const int ntiles = (int)((nleaf + (int64_t)kScanTile - 1) / kScanTile);
    scan_tiles_kernel<<<ntiles, kScanThreads, 0, s>>>(counts, nleaf, row_off, tiles);
    scan_sums_kernel<<<1, kScanThreads, 0, s>>>(tiles, ntiles, row_off + nleaf);
    scan_add_kernel<<<grid_cap(nleaf, threads, 1 << 30), threads, 0, s>>>(row_off, nleaf, tiles);
    csr_scatter_kernel<<<eblocks, threads, 0, s>>>(d_task_t, d_task_s, ntask, nleaf, row_off, fill,
                                                   row_src);
    csr_sort_rows_warp_kernel<1, kSortWarpMax><<<grid_cap(nleaf, 4, sms * 8), 128, 0, s>>>(row_off, nleaf, row_src);
    csr_sort_rows_warp_kernel<kSortWarpMax, kSortWarpMax2><<<grid_cap(nleaf, 4, sms * 8), 128, 0, s>>>(row_off, nleaf,
                                                                                                   row_src);
    csr_sort_rows_block_kernel<<<grid_cap(nleaf, 1, sms * 4), kSortBlockThreads, 0, s>>>(row_off, nleaf, row_src);
    csr_sort_rows_global_kernel<<<grid_cap(nleaf, 1, sms), kSortBlockThreads, 0, s>>>(row_off, nleaf, row_src);
    if (cudaGetLastError() != cudaSuccess) return fail_after_queue(s, P2P_ERR_CUDA);

    PairArgs a;
    memset(&a, 0, sizeof(a));
    a.leaf = meta;
    a.row_off = row_off;
    a.row_src = row_src;
    a.pos4 = pos4;
    a.pos = d_pos;
    a.mass = nullptr;
    a.acc = d_acc;
    a.queue = queue;
    a.npart = npart;
    a.nleaf = nleaf;
    fill_pass_scalars(a, p, fit, false);
    st = launch_pair_kernel(fp32, p, fit.ncoef_kernel, sms, warps, smem, s, a, stage, &blocks);
    if (st != P2P_OK) return fail_after_queue(s, st);
    // the status word read on the caller's stream, behind the pass; the call
    // returns once that stream has reached it
    int flags = 0;
    if (cudaMemcpyAsync(&flags, status, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return fail_after_queue(s, P2P_ERR_CUDA);
    if (cudaStreamSynchronize(s) != cudaSuccess) return fail_after_queue(s, P2P_ERR_CUDA);
    return flags ? P2P_ERR_RANGE : P2P_OK;
}
