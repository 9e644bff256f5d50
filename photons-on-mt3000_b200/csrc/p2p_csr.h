// CSR build of one interaction list on explicit device buffers: the sink
// histogram and pair count (csr_count_kernel), its exclusive scan into row
// offsets, and the stable LSD radix sort of the list by sink id whose last
// pass writes the rows' source ids (the reference's stable sort_by_key,
// src/gpu_entry.cu:132-138). Shared by the session path and the server.
// Include after p2p_pass_kernels.cuh, in the namespace that holds the kernels.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

struct CsrBufs {
    int *counts = nullptr;              // nleaf
    int64_t *row_off = nullptr;         // nleaf + 1 (output)
    int64_t *tile_sums = nullptr;       // csr_tile_sums(nleaf)
    int *row_src = nullptr;             // ntask (output)
    int *keys_a = nullptr, *keys_b = nullptr, *vals_b = nullptr;  // ntask each
    int *hist = nullptr;                // csr_hist_len(ntask)
    int64_t *hoffs = nullptr;           // csr_hist_len(ntask) + 1
    int64_t *hsums = nullptr;           // csr_hsum_len(ntask)
    unsigned long long *pairs = nullptr;  // += pair count
    int *status = nullptr;              // |= ST_* bits
    unsigned long long *skipped = nullptr;  // += pairs of entries wholly beyond the cutoff (nullable)
    double cscale = 1.0;                // frame scale and bound used for skipped
    float uout = 0.f;
};

inline int csr_grid(int64_t n, int threads, int cap_blocks) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap_blocks) b = cap_blocks;
    return (int)b;
}
inline size_t csr_tile_sums(int64_t nleaf) { return (size_t)(nleaf + kScanTile - 1) / kScanTile + 1; }
inline size_t csr_hist_len(int64_t ntask) {
    const int64_t n = std::max<int64_t>(ntask, 1);
    return (size_t)kRadixBins * (size_t)((n + kRadixTile - 1) / kRadixTile);
}
inline size_t csr_hsum_len(int64_t ntask) {  // chunk sums of the histogram's column scan
    const int64_t n = std::max<int64_t>(ntask, 1);
    const int64_t rtiles = (n + kRadixTile - 1) / kRadixTile;
    return (size_t)kRadixBins * (size_t)((rtiles + kColTiles - 1) / kColTiles) + 1;
}

// Enqueues the build on `st`; *launches += kernels launched.
inline cudaError_t enqueue_csr_build(cudaStream_t st, int64_t ntask, const int *d_t, const int *d_s,
                                     int nleaf, const LeafMeta *meta, const CsrBufs &b,
                                     int *launches) {
    if (ntask <= 0 || nleaf <= 0) return cudaSuccess;
    const int threads = 256;
    cudaError_t e = cudaMemsetAsync(b.counts, 0, sizeof(int) * (size_t)nleaf, st);
    if (e != cudaSuccess) return e;
    csr_count_kernel<<<csr_grid(ntask, threads, 148 * 16), threads, 0, st>>>(
        d_t, d_s, ntask, nleaf, meta, b.counts, b.pairs, b.status, b.skipped, b.cscale, b.uout);
    const int ntiles = (int)((nleaf + (int64_t)kScanTile - 1) / kScanTile);
    scan_tiles_kernel<<<ntiles, kScanThreads, 0, st>>>(b.counts, nleaf, b.row_off, b.tile_sums);
    scan_sums_kernel<<<1, kScanThreads, 0, st>>>(b.tile_sums, ntiles, b.row_off + nleaf);
    scan_add_kernel<<<csr_grid(nleaf, threads, 1 << 30), threads, 0, st>>>(b.row_off, nleaf, b.tile_sums);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    *launches += 4;
    // radix passes over keys in [0, nleaf]: 8-bit digits, or two 10-bit
    // digits for 17-20 key bits (one pass fewer)
    int bits = 1;
    while (bits < 31 && ((int64_t)1 << bits) <= (int64_t)nleaf) ++bits;
    const int rtiles = (int)((ntask + kRadixTile - 1) / kRadixTile);
    // (10-bit digits up to 2^20 tiles: 4 GB of histogram and 8 GB of offsets there)
    const int digit = (bits > 16 && bits <= 20 && rtiles <= (1 << 20)) ? 10 : 8;
    const int passes = (bits + digit - 1) / digit;
    const int nchunks = (rtiles + kColTiles - 1) / kColTiles;
    int *kbuf[2] = {b.keys_a, b.keys_b};
    int *vbuf[2] = {b.row_src, b.vals_b};
    const int *kin = nullptr, *vin = nullptr;
    for (int pass = 0; pass < passes; ++pass) {
        const int shift = digit * pass;
        const int o = (passes - 1 - pass) & 1;  // the last pass lands in row_src
        int *kout = pass == passes - 1 ? nullptr : kbuf[o];
        int *vout = vbuf[o];
        if (digit == 10) {
            if (pass == 0)
                radix_hist_kernel<10, true><<<rtiles, kRadixWarps * 32, 0, st>>>(kin, d_t, d_s, nleaf, ntask,
                                                                                 shift, b.hist, rtiles);
            else
                radix_hist_kernel<10, false><<<rtiles, kRadixWarps * 32, 0, st>>>(kin, d_t, d_s, nleaf, ntask,
                                                                                  shift, b.hist, rtiles);
        } else {
            if (pass == 0)
                radix_hist_kernel<8, true><<<rtiles, kRadixWarps * 32, 0, st>>>(kin, d_t, d_s, nleaf, ntask,
                                                                                shift, b.hist, rtiles);
            else
                radix_hist_kernel<8, false><<<rtiles, kRadixWarps * 32, 0, st>>>(kin, d_t, d_s, nleaf, ntask,
                                                                                 shift, b.hist, rtiles);
        }
        if (digit == 10) {
            radix_colsum_kernel<1024><<<nchunks, 1024, 0, st>>>(b.hist, rtiles, b.hsums);
            radix_colscan_kernel<1024><<<1, 1024, 0, st>>>(b.hsums, nchunks);
            radix_offs_kernel<1024><<<nchunks, 1024, 0, st>>>(b.hist, rtiles, b.hsums, b.hoffs);
        } else {
            radix_colsum_kernel<256><<<nchunks, 256, 0, st>>>(b.hist, rtiles, b.hsums);
            radix_colscan_kernel<256><<<1, 256, 0, st>>>(b.hsums, nchunks);
            radix_offs_kernel<256><<<nchunks, 256, 0, st>>>(b.hist, rtiles, b.hsums, b.hoffs);
        }
        if (digit == 10) {
            if (pass == 0)
                radix_scatter_kernel<10, true><<<rtiles, kRadixWarps * 32, 0, st>>>(
                    kin, vin, d_t, d_s, nleaf, ntask, shift, b.hoffs, rtiles, kout, vout);
            else
                radix_scatter_kernel<10, false><<<rtiles, kRadixWarps * 32, 0, st>>>(
                    kin, vin, d_t, d_s, nleaf, ntask, shift, b.hoffs, rtiles, kout, vout);
        } else {
            if (pass == 0)
                radix_scatter_kernel<8, true><<<rtiles, kRadixWarps * 32, 0, st>>>(
                    kin, vin, d_t, d_s, nleaf, ntask, shift, b.hoffs, rtiles, kout, vout);
            else
                radix_scatter_kernel<8, false><<<rtiles, kRadixWarps * 32, 0, st>>>(
                    kin, vin, d_t, d_s, nleaf, ntask, shift, b.hoffs, rtiles, kout, vout);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        *launches += 5;
        kin = kout;
        vin = vout;
    }
    return cudaSuccess;
}
