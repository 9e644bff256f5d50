// Launch interface of the pair kernels. Each lane mapping lives in its own
// translation unit (p2p_pair_*.cu) so the many template instances compile in
// parallel; the session code (p2p_core.cu) calls them through this header.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <map>
#include <tuple>

#include "p2p_internal.h"

namespace p2p {

using OccupancyCache = std::map<std::tuple<const void *, int, size_t>, int>;

struct PairLaunch {
    cudaStream_t stream;
    int sm_count;
    int soft_mode;      // SOFT_CLAMP / SOFT_PLUMMER
    bool masses;        // per-particle masses staged in .w
    int acc;            // ACC_F64 / ACC_KAHAN / ACC_F32 (FP32 forms)
    int ncoef;          // polynomial coefficients (FP32 forms)
    int warps, stage;   // block shape (resolved, non-zero)
    int blocks_per_sm;  // 0: as many as fit
    bool dry_run;       // resolve the launch shape only
    OccupancyCache *occ;
    int max_blocks = 0; // > 0: cap on the persistent grid (a share of the GPU)
    int sink_pairs = 16; // packed source-lane kernel: sink pairs per slice (16 or 8)
    int sreg_spl = 4;    // sink-register kernel: sinks per lane (4: 32-sink slices, 8: 64)
};

struct PairLaunchResult {
    cudaError_t cuda = cudaSuccess;
    int blocks = 0;
    bool fits = true;  // false: the block shape does not fit on an SM
};

// Dynamic shared memory of one block of each mapping.
inline size_t pair_smem_split(int warps, int stage, bool source_lanes) {
    return (size_t)warps * (stage + (source_lanes ? 32 : 0)) * 16;
}
inline size_t pair_smem_plain(int warps, int stage) { return (size_t)warps * stage * 32; }
// packed source-lane kernel: sink pairs, band corrections, staged sources + their indices
inline size_t pair_smem_x2(int warps, int stage) { return (size_t)warps * (stage + 64 + stage / 4) * 16; }
// packed sink-lane kernel: staged sources as two float4 + index, 32 padding slots
inline size_t pair_smem_sx2(int warps, int stage) { return (size_t)warps * (stage + 32) * 36; }
// sink-register kernel: staged sources (pre-duplicated, with their indices) + lane
// accumulators + staging context; its stage holds at least kSregMinStage sources (one staging group)
constexpr int kSregMinStage = 128;
inline int sreg_stage(int stage) { return stage < kSregMinStage ? kSregMinStage : stage; }
inline size_t pair_smem_sreg(int warps, int stage, int spl = 4) {
    return (size_t)warps * ((size_t)sreg_stage(stage) * 32 + 3 * (size_t)spl * 32 * 8 + 1024);
}

// Persistent grid for `kernel`: blocks_per_sm, or as many as registers and
// shared memory let reside (queried once and cached).
template <class K>
bool persistent_blocks(const PairLaunch &L, K kernel, size_t smem, PairLaunchResult &r) {
    int per_sm = L.blocks_per_sm;
    if (!per_sm) {
        const auto key = std::make_tuple((const void *)kernel, L.warps, smem);
        auto it = L.occ->find(key);
        if (it == L.occ->end()) {
            r.cuda = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, L.warps * 32, smem);
            if (r.cuda != cudaSuccess) return false;
            (*L.occ)[key] = per_sm;
        } else {
            per_sm = it->second;
        }
    }
    if (per_sm < 1) {
        r.fits = false;
        return false;
    }
    r.blocks = per_sm * L.sm_count;
    if (L.max_blocks > 0 && r.blocks > L.max_blocks) r.blocks = L.max_blocks;
    return true;
}

template <class K>
PairLaunchResult launch_persistent(const PairLaunch &L, K kernel, size_t smem, const PairArgs &a) {
    PairLaunchResult r;
    if (!persistent_blocks(L, kernel, smem, r)) return r;
    if (L.dry_run) return r;
    kernel<<<r.blocks, L.warps * 32, smem, L.stream>>>(a, L.stage);
    r.cuda = cudaGetLastError();
    return r;
}

// FP32 forms. Returns cudaErrorInvalidValue in .cuda for an unsupported
// coefficient count.
PairLaunchResult launch_pair_sink_lanes(const PairLaunch &L, const PairArgs &a);
PairLaunchResult launch_pair_source_lanes(const PairLaunch &L, const PairArgs &a);
PairLaunchResult launch_pair_source_lanes_x2(const PairLaunch &L, const PairArgs &a);
PairLaunchResult launch_pair_sink_lanes_x2(const PairLaunch &L, const PairArgs &a);
PairLaunchResult launch_pair_sink_regs(const PairLaunch &L, const PairArgs &a);
// FP64 form.
PairLaunchResult launch_pair_plain(const PairLaunch &L, const PairArgs &a);

// Opt each mapping's kernels into large dynamic shared memory (per device).
cudaError_t allow_smem_sink_lanes();
cudaError_t allow_smem_source_lanes();
cudaError_t allow_smem_source_lanes_x2();
cudaError_t allow_smem_sink_lanes_x2();
cudaError_t allow_smem_sink_regs();
cudaError_t allow_smem_plain();

}  // namespace p2p
