// Pass kernels: frame preparation, CSR build (count, scan, scatter, row
// sort) and the FP32 throughput probe. Non-template kernels: a translation
// unit that includes this header defines them.
#pragma once

#include "p2p_device_common.cuh"

namespace p2p {

// ---------------------------------------------------------------- prep ----

// FP32 forms: frame centres and scaled FP32 coordinates. LOCAL = false puts
// every leaf's frame at the origin (global FP32 coordinates, the naive form).
template <bool LOCAL>
__global__ void prep_split_kernel(const double *__restrict__ pos, const double *__restrict__ mass,
                                  const int *__restrict__ leaf_ip, const int *__restrict__ leaf_np,
                                  int npart, int nleaf, double cscale, LeafMeta *__restrict__ meta,
                                  float4 *__restrict__ pos4, int *__restrict__ status) {
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int l = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; l < nleaf; l += nwarps) {
        const int ip = leaf_ip[l], np = leaf_np[l];
        const bool ok = ip >= 0 && np >= 0 && (int64_t)ip + np <= npart;
        if (!ok) {
            if (lane == 0) {
                atomicOr(status, ST_LEAF_RANGE);
                LeafMeta m;
                m.cx = m.cy = m.cz = 0.0;
                m.ipart = 0;
                m.npart = 0;
                m.hx = m.hy = m.hz = m.pad = 0.f;
                meta[l] = m;
            }
            continue;
        }
        const double *X = pos, *Y = pos + npart, *Z = pos + 2 * (size_t)npart;
        double c0 = 0.0, c1 = 0.0, c2 = 0.0;
        float e0 = 0.f, e1 = 0.f, e2 = 0.f;
        if (LOCAL && np > 0) {
            double lo0 = 1e300, lo1 = 1e300, lo2 = 1e300, hi0 = -1e300, hi1 = -1e300, hi2 = -1e300;
            for (int q = lane; q < np; q += 32) {
                const double x = X[ip + q], y = Y[ip + q], z = Z[ip + q];
                lo0 = fmin(lo0, x); hi0 = fmax(hi0, x);
                lo1 = fmin(lo1, y); hi1 = fmax(hi1, y);
                lo2 = fmin(lo2, z); hi2 = fmax(hi2, z);
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                lo0 = fmin(lo0, __shfl_xor_sync(kFull, lo0, off));
                lo1 = fmin(lo1, __shfl_xor_sync(kFull, lo1, off));
                lo2 = fmin(lo2, __shfl_xor_sync(kFull, lo2, off));
                hi0 = fmax(hi0, __shfl_xor_sync(kFull, hi0, off));
                hi1 = fmax(hi1, __shfl_xor_sync(kFull, hi1, off));
                hi2 = fmax(hi2, __shfl_xor_sync(kFull, hi2, off));
            }
            c0 = 0.5 * (lo0 + hi0);
            c1 = 0.5 * (lo1 + hi1);
            c2 = 0.5 * (lo2 + hi2);
            // half-extents, rounded up: a bound, never an underestimate
            e0 = __double2float_ru(0.5 * (hi0 - lo0) * cscale * (1.0 + 1e-6));
            e1 = __double2float_ru(0.5 * (hi1 - lo1) * cscale * (1.0 + 1e-6));
            e2 = __double2float_ru(0.5 * (hi2 - lo2) * cscale * (1.0 + 1e-6));
        }
        if (lane == 0) {
            LeafMeta m;
            m.cx = c0;
            m.cy = c1;
            m.cz = c2;
            m.ipart = ip;
            m.npart = np;
            m.hx = LOCAL ? e0 : 1e30f;  // global frames: never claim an entry fully inside
            m.hy = LOCAL ? e1 : 1e30f;
            m.hz = LOCAL ? e2 : 1e30f;
            m.pad = 0.f;
            meta[l] = m;
        }
        for (int q = lane; q < np; q += 32) {
            const int i = ip + q;
            pos4[i] = make_float4((float)((X[i] - c0) * cscale), (float)((Y[i] - c1) * cscale),
                                  (float)((Z[i] - c2) * cscale), mass ? (float)mass[i] : 1.0f);
        }
    }
}

// FP64 form: leaf table only (positions stay FP64 SoA).
__global__ void prep_plain_kernel(const int *__restrict__ leaf_ip, const int *__restrict__ leaf_np,
                                  int npart, int nleaf, LeafMeta *__restrict__ meta,
                                  int *__restrict__ status) {
    for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < nleaf; l += gridDim.x * blockDim.x) {
        int ip = leaf_ip[l], np = leaf_np[l];
        if (!(ip >= 0 && np >= 0 && (int64_t)ip + np <= npart)) {
            atomicOr(status, ST_LEAF_RANGE);
            ip = 0;
            np = 0;
        }
        LeafMeta m;
        m.cx = m.cy = m.cz = 0.0;
        m.ipart = ip;
        m.npart = np;
        m.hx = m.hy = m.hz = m.pad = 0.f;
        meta[l] = m;
    }
}

// ----------------------------------------------------------------- CSR ----

// skipped (nullable): += pairs of entries the FP32 pair kernels skip as lying
// wholly beyond the cutoff (lower bound on u above uout, frames scaled by cscale).
__global__ void csr_count_kernel(const int *__restrict__ tt, const int *__restrict__ ts, int64_t n,
                                 int nleaf, const LeafMeta *__restrict__ meta,
                                 int *__restrict__ counts, unsigned long long *__restrict__ pairs,
                                 int *__restrict__ status, unsigned long long *__restrict__ skipped,
                                 double cscale, float uout) {
    __shared__ unsigned long long block_pairs, block_skip;
    if (threadIdx.x == 0) block_pairs = block_skip = 0;
    __syncthreads();
    unsigned long long local = 0, lskip = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
        const int t = tt[e], s = ts[e];
        if ((unsigned)t >= (unsigned)nleaf || (unsigned)s >= (unsigned)nleaf) {
            atomicOr(status, ST_TASK_RANGE);
            continue;
        }
        atomicAdd(&counts[t], 1);
        const LeafMeta mt = meta[t], ms = meta[s];
        const unsigned long long np = (unsigned long long)mt.npart * (unsigned long long)ms.npart;
        local += np;
        if (skipped) {
            float ox, oy, oz;
            entry_offset(ms, mt, cscale, ox, oy, oz);
            if (entry_u_min(ms, mt, ox, oy, oz) > uout) lskip += np;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        local += __shfl_xor_sync(kFull, local, off);
        lskip += __shfl_xor_sync(kFull, lskip, off);
    }
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(&block_pairs, local);
    if ((threadIdx.x & 31) == 0 && lskip) atomicAdd(&block_skip, lskip);
    __syncthreads();
    if (threadIdx.x == 0 && block_pairs) atomicAdd(pairs, block_pairs);
    if (threadIdx.x == 0 && block_skip) atomicAdd(skipped, block_skip);
}

__global__ void csr_scatter_kernel(const int *__restrict__ tt, const int *__restrict__ ts, int64_t n,
                                   int nleaf, const int64_t *__restrict__ row_off,
                                   int *__restrict__ fill, int *__restrict__ row_src) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
        const int t = tt[e], s = ts[e];
        if ((unsigned)t >= (unsigned)nleaf || (unsigned)s >= (unsigned)nleaf) continue;
        const int k = atomicAdd(&fill[t], 1);
        row_src[row_off[t] + k] = s;
    }
}

// Rows are sorted by source leaf id after the scatter, so the order in which
// a row's sources are summed does not depend on the order the atomics
// placed them in: results are bit-for-bit repeatable.
//
// Sorting network: bitonic with "flip" merges, every comparator putting the
// smaller key at the lower index. Padding a row of length L to the next power
// of two with +inf keys then never moves a padded key below L, so comparators
// whose upper index is >= L are simply skipped and no padding is stored.
// Block sizes and strides are powers of two, so comparator indices are
// formed with shifts and masks of their logarithms (a division by a run-time
// value would cost a multi-instruction sequence per comparator).
template <class Sync>
__device__ __forceinline__ void flip_bitonic_sort(int *v, int len, int tid, int nthreads,
                                                  Sync sync) {
    int lgP = 0;
    while ((1 << lgP) < len) ++lgP;
    const int half_n = (1 << lgP) >> 1;  // comparators per round
    for (int lgs = 1; lgs <= lgP; ++lgs) {  // merge blocks of 2^lgs keys
        const int lgh = lgs - 1, hmask = (1 << lgh) - 1, size = 1 << lgs;
        for (int i = tid; i < half_n; i += nthreads) {
            const int base = (i >> lgh) << lgs, off = i & hmask;
            const int lo = base + off, hi = base + size - 1 - off;
            if (hi < len) {
                const int a = v[lo], b = v[hi];
                if (a > b) { v[lo] = b; v[hi] = a; }
            }
        }
        sync();
        for (int lgst = lgh - 1; lgst >= 0; --lgst) {  // then strides 2^lgst down to 1
            const int smask = (1 << lgst) - 1;
            for (int i = tid; i < half_n; i += nthreads) {
                const int lo = ((i >> lgst) << (lgst + 1)) + (i & smask), hi = lo + (1 << lgst);
                if (hi < len) {
                    const int a = v[lo], b = v[hi];
                    if (a > b) { v[lo] = b; v[hi] = a; }
                }
            }
            sync();
        }
    }
}

constexpr int kSortWarpMax = 1024;   // rows up to this length: one warp, shared memory
constexpr int kSortWarpMax2 = 2048;  // rows up to this length: one warp, a larger buffer
constexpr int kSortBlockMax = 8192;  // rows up to this length: one block, shared memory
constexpr int kSortBlockThreads = 512;

// Rows of length LO+1..HI (and at least 2), one warp per row (4 warps per
// block): <1, kSortWarpMax> and <kSortWarpMax, kSortWarpMax2>, so the short
// rows keep a small buffer and many resident warps.
template <int LO, int HI>
__global__ void __launch_bounds__(128)
csr_sort_rows_warp_kernel(const int64_t *__restrict__ row_off, int nleaf, int *__restrict__ row_src) {
    __shared__ int buf[4][HI];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int *v = buf[w];
    const int nw = gridDim.x * 4;
    for (int r = blockIdx.x * 4 + w; r < nleaf; r += nw) {
        const int64_t b = row_off[r];
        const int len = (int)(row_off[r + 1] - b);
        if (len < 2 || len <= LO || len > HI) continue;
        for (int i = lane; i < len; i += 32) v[i] = row_src[b + i];
        __syncwarp();
        flip_bitonic_sort(v, len, lane, 32, []() { __syncwarp(); });
        for (int i = lane; i < len; i += 32) row_src[b + i] = v[i];
        __syncwarp();
    }
}

// Rows of length kSortWarpMax2+1..kSortBlockMax, one block per row.
__global__ void __launch_bounds__(kSortBlockThreads)
csr_sort_rows_block_kernel(const int64_t *__restrict__ row_off, int nleaf, int *__restrict__ row_src) {
    __shared__ int v[kSortBlockMax];
    for (int r = blockIdx.x; r < nleaf; r += gridDim.x) {
        const int64_t b = row_off[r];
        const int len = (int)(row_off[r + 1] - b);
        if (len <= kSortWarpMax2 || len > kSortBlockMax) continue;
        for (int i = threadIdx.x; i < len; i += blockDim.x) v[i] = row_src[b + i];
        __syncthreads();
        flip_bitonic_sort(v, len, threadIdx.x, blockDim.x, []() { __syncthreads(); });
        for (int i = threadIdx.x; i < len; i += blockDim.x) row_src[b + i] = v[i];
        __syncthreads();
    }
}

// Longer rows, one block per row, sorted in place in global memory.
__global__ void __launch_bounds__(kSortBlockThreads)
csr_sort_rows_global_kernel(const int64_t *__restrict__ row_off, int nleaf, int *__restrict__ row_src) {
    for (int r = blockIdx.x; r < nleaf; r += gridDim.x) {
        const int64_t b = row_off[r];
        const int64_t len = row_off[r + 1] - b;
        if (len <= kSortBlockMax) continue;
        __syncthreads();
        flip_bitonic_sort(row_src + b, (int)len, threadIdx.x, blockDim.x,
                          []() { __threadfence_block(); __syncthreads(); });
    }
}

// Stable LSD radix sort of the list by sink id (8- or 10-bit digits), the CSR
// build: within a row, entries keep list order - the order the reference's
// stable thrust::sort_by_key gives (src/gpu_entry.cu:132) - so the pair
// kernels sum every row in a fixed order and results repeat bit for bit.
//
// Per digit pass: radix_hist_kernel (per-tile histogram, stored tile-major:
// row t holds tile t's counts), the output offset of every (tile, digit) -
// the digit's start plus the counts of that digit in earlier tiles - from a
// column scan of the histogram (radix_colsum_kernel, radix_colscan_kernel,
// radix_offs_kernel; every access a whole row), and radix_scatter_kernel: the
// stable rank of each entry within its tile by digit (warp-private counts and
// __match_any_sync), the tile reordered by digit in shared memory, then
// written out so consecutive threads store consecutive entries of a digit's
// run (a few sectors per warp store instead of one per entry). Entries with
// an out-of-range sink or source get key nleaf and sort past the rows.
constexpr int kRadixBins = 1024;  // most bins of a digit (10 bits); histograms are sized for it
constexpr int kRadixWarps = 8;
constexpr int kRadixRounds = 16;
constexpr int kRadixTile = kRadixWarps * kRadixRounds * 32;  // 4096 entries

// RAW (first pass): the key comes from the raw (t, s) list, else from keys.
template <bool RAW>
__device__ __forceinline__ unsigned radix_key(const int *keys, const int *raw_t, const int *raw_s,
                                              int nleaf, int64_t i) {
    if (!RAW) return (unsigned)keys[i];
    const int t = raw_t[i], s = raw_s[i];
    return ((unsigned)t < (unsigned)nleaf && (unsigned)s < (unsigned)nleaf) ? (unsigned)t : (unsigned)nleaf;
}

// RAW: first pass, keys computed from the raw (t, s) list (keys unused).
// BITS: digit width (8 or 10).
template <int BITS, bool RAW>
__global__ void __launch_bounds__(kRadixWarps * 32)
radix_hist_kernel(const int *__restrict__ keys, const int *__restrict__ raw_t,
                  const int *__restrict__ raw_s, int nleaf, int64_t n, int shift,
                  int *__restrict__ hist, int ntiles) {
    constexpr int NB = 1 << BITS;
    constexpr unsigned MASK = NB - 1u;
    __shared__ int h[kRadixWarps][NB];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int b = threadIdx.x; b < kRadixWarps * NB; b += blockDim.x) (&h[0][0])[b] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kRadixTile + (int64_t)w * kRadixRounds * 32;
    // all rounds' loads first (in flight together), then the counts
    unsigned key[kRadixRounds];
#pragma unroll
    for (int r = 0; r < kRadixRounds; ++r) {
        const int64_t i = base + r * 32 + lane;
        key[r] = i < n ? radix_key<RAW>(keys, raw_t, raw_s, nleaf, i) : 0xffffffffu;
    }
#pragma unroll
    for (int r = 0; r < kRadixRounds; ++r)
        if (key[r] != 0xffffffffu) atomicAdd(&h[w][(key[r] >> shift) & MASK], 1);
    __syncthreads();
    for (int b = threadIdx.x; b < NB; b += blockDim.x) {
        int tot = 0;
#pragma unroll
        for (int q = 0; q < kRadixWarps; ++q) tot += h[q][b];
        hist[(int64_t)blockIdx.x * NB + b] = tot;
    }
}

template <int BITS, bool RAW>
__global__ void __launch_bounds__(kRadixWarps * 32)
radix_scatter_kernel(const int *__restrict__ keys, const int *__restrict__ vals,
                     const int *__restrict__ raw_t, const int *__restrict__ raw_s, int nleaf,
                     int64_t n, int shift, const int64_t *__restrict__ offs, int ntiles,
                     int *__restrict__ keys_out, int *__restrict__ vals_out) {
    constexpr int NB = 1 << BITS;
    constexpr unsigned MASK = NB - 1u;
    constexpr int NT = kRadixWarps * 32;
    constexpr int BPT = NB / NT;  // bins per thread in the bin scans
    static_assert(NB % NT == 0, "bins must split evenly over the block");
    constexpr int POOL = kRadixWarps * NB > 2 * kRadixTile ? kRadixWarps * NB : 2 * kRadixTile;
    // the warp counts (warp q, digit b at pool[q * NB + b]), then, once every
    // entry's tile position is known, the tile's keys and values in digit order
    __shared__ int pool[POOL];
    __shared__ int bin_start[NB];      // exclusive start of each digit within the tile
    __shared__ int64_t gdelta[NB];     // output offset of the digit's run minus its start in the tile
    __shared__ int wsum[kRadixWarps];
    int(*cnt)[NB] = reinterpret_cast<int(*)[NB]>(pool);
    int *tkeys = pool;
    int *tvals = pool + kRadixTile;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    int64_t goff[BPT];  // this thread's digits' output offsets, loaded early
#pragma unroll
    for (int k = 0; k < BPT; ++k) goff[k] = offs[(int64_t)blockIdx.x * NB + threadIdx.x * BPT + k];
    const int64_t tile0 = (int64_t)blockIdx.x * kRadixTile;
    const int64_t base = tile0 + (int64_t)w * kRadixRounds * 32;
    unsigned key[kRadixRounds];
    int val[kRadixRounds];
    unsigned peers[kRadixRounds];
    // all rounds' loads first (in flight together), then the ranks
#pragma unroll
    for (int r = 0; r < kRadixRounds; ++r) {
        const int64_t i = base + r * 32 + lane;
        const bool ok = i < n;
        key[r] = ok ? radix_key<RAW>(keys, raw_t, raw_s, nleaf, i) : 0xffffffffu;
        val[r] = ok ? (RAW ? raw_s[i] : vals[i]) : 0;
    }
    for (int b = threadIdx.x; b < kRadixWarps * NB; b += NT) pool[b] = 0;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRadixRounds; ++r) {
        const bool ok = base + r * 32 + lane < n;
        const int d = ok ? (int)((key[r] >> shift) & MASK) : NB + lane;  // tail lanes: own group
        peers[r] = __match_any_sync(kFull, d);
        if (ok && lane == __ffs(peers[r]) - 1) cnt[w][d] += __popc(peers[r]);
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive base of every warp within the digit's run, the
    // run's length, then the runs' starts (a block scan over the digits)
    int tot[BPT];
    int run_sum = 0;
#pragma unroll
    for (int k = 0; k < BPT; ++k) {
        const int b = threadIdx.x * BPT + k;
        int run = 0;
#pragma unroll
        for (int q = 0; q < kRadixWarps; ++q) {
            const int c = cnt[q][b];
            cnt[q][b] = run;
            run += c;
        }
        tot[k] = run;
        run_sum += run;
    }
    int incl = run_sum;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int v = __shfl_up_sync(kFull, incl, off);
        if (lane >= off) incl += v;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    int start = incl - run_sum;
    for (int q = 0; q < w; ++q) start += wsum[q];
#pragma unroll
    for (int k = 0; k < BPT; ++k) {
        const int b = threadIdx.x * BPT + k;
        bin_start[b] = start;
        gdelta[b] = goff[k] - start;
        start += tot[k];
    }
    __syncthreads();
    // each entry's position within the tile (digit order, list order within a digit)
    int lp[kRadixRounds];
#pragma unroll
    for (int r = 0; r < kRadixRounds; ++r) {
        const bool ok = base + r * 32 + lane < n;
        const int d = ok ? (int)((key[r] >> shift) & MASK) : 0;
        const int before = ok ? cnt[w][d] : 0;
        __syncwarp();
        lp[r] = ok ? bin_start[d] + before + __popc(peers[r] & lt) : -1;
        if (ok && lane == __ffs(peers[r]) - 1) cnt[w][d] = before + __popc(peers[r]);
        __syncwarp();
    }
    __syncthreads();  // the warp counts are dead: the tile is staged over them
#pragma unroll
    for (int r = 0; r < kRadixRounds; ++r) {
        if (lp[r] >= 0) {
            tkeys[lp[r]] = (int)key[r];
            tvals[lp[r]] = val[r];
        }
    }
    __syncthreads();
    // consecutive threads write consecutive entries of a digit's run
    const int tn = (int)min((int64_t)kRadixTile, n - tile0);
    for (int j = threadIdx.x; j < tn; j += NT) {
        const unsigned k = (unsigned)tkeys[j];
        const int64_t pos = gdelta[(k >> shift) & MASK] + j;
        if (keys_out) keys_out[pos] = (int)k;
        vals_out[pos] = tvals[j];
    }
}

// Column scan of the tile-major histogram in chunks of kColTiles tiles:
// csum[c * NB + d] = count of digit d in chunk c (radix_colsum_kernel), then
// in place the exclusive prefix over chunks plus digit d's start in the
// output (radix_colscan_kernel, one block), then offs[t * NB + d], tile t's
// output offset for digit d (radix_offs_kernel). One thread per digit; the
// threads of a block read and write whole rows.
constexpr int kColTiles = 128;

template <int NB>
__global__ void __launch_bounds__(NB)
radix_colsum_kernel(const int *__restrict__ hist, int ntiles, int64_t *__restrict__ csum) {
    const int d = threadIdx.x;
    const int t0 = blockIdx.x * kColTiles, t1 = min(ntiles, t0 + kColTiles);
    int64_t s = 0;
#pragma unroll 8
    for (int t = t0; t < t1; ++t) s += hist[(int64_t)t * NB + d];
    csum[(int64_t)blockIdx.x * NB + d] = s;
}

template <int NB>
__global__ void __launch_bounds__(NB)
radix_colscan_kernel(int64_t *__restrict__ csum, int nchunks) {
    constexpr int NW = NB / 32;
    __shared__ int64_t wsum[NW];
    const int d = threadIdx.x, lane = d & 31, w = d >> 5;
    int64_t tot = 0;
#pragma unroll 8
    for (int c = 0; c < nchunks; ++c) tot += csum[(int64_t)c * NB + d];
    // digit starts: exclusive scan of the totals over the digits
    int64_t x = tot;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int64_t y = __shfl_up_sync(kFull, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        int64_t v = lane < NW ? wsum[lane] : 0;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int64_t y = __shfl_up_sync(kFull, v, off);
            if (lane >= off) v += y;
        }
        if (lane < NW) wsum[lane] = v;
    }
    __syncthreads();
    int64_t run = x - tot + (w > 0 ? wsum[w - 1] : 0);
    for (int c = 0; c < nchunks; ++c) {
        const int64_t i = (int64_t)c * NB + d;
        const int64_t v = csum[i];
        csum[i] = run;
        run += v;
    }
}

template <int NB>
__global__ void __launch_bounds__(NB)
radix_offs_kernel(const int *__restrict__ hist, int ntiles, const int64_t *__restrict__ csum,
                  int64_t *__restrict__ offs) {
    const int d = threadIdx.x;
    const int t0 = blockIdx.x * kColTiles, t1 = min(ntiles, t0 + kColTiles);
    int64_t run = csum[(int64_t)blockIdx.x * NB + d];
    for (int k0 = t0; k0 < t1; k0 += 8) {
        int h[8];  // eight rows' loads in flight
#pragma unroll
        for (int k = 0; k < 8; ++k) h[k] = k0 + k < t1 ? hist[(int64_t)(k0 + k) * NB + d] : 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (k0 + k < t1) offs[(int64_t)(k0 + k) * NB + d] = run;
            run += h[k];
        }
    }
}

// Exclusive scan int32 -> int64 in three kernels. kScanTile elements per block.
constexpr int kScanThreads = 256;
constexpr int kScanPer = 8;
constexpr int kScanTile = kScanThreads * kScanPer;

__device__ __forceinline__ int64_t block_exclusive_scan(int64_t v, int64_t *warp_sums,
                                                        int64_t *total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int64_t x = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int64_t y = __shfl_up_sync(kFull, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
        int64_t ws = lane < (kScanThreads / 32) ? warp_sums[lane] : 0;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int64_t y = __shfl_up_sync(kFull, ws, off);
            if (lane >= off) ws += y;
        }
        if (lane < (kScanThreads / 32)) warp_sums[lane] = ws;
    }
    __syncthreads();
    const int64_t before = (w > 0 ? warp_sums[w - 1] : 0) + x - v;
    if (total) *total = warp_sums[kScanThreads / 32 - 1];
    return before;
}

__global__ void __launch_bounds__(kScanThreads)
scan_tiles_kernel(const int *__restrict__ in, int n, int64_t *__restrict__ out,
                  int64_t *__restrict__ tile_sums) {
    __shared__ int64_t warp_sums[kScanThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanPer;
    int64_t v[kScanPer];
    int64_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        const int64_t i = base + k;
        v[k] = i < n ? in[i] : 0;
        s += v[k];
    }
    int64_t total;
    int64_t run = block_exclusive_scan(s, warp_sums, &total);
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        const int64_t i = base + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads)
scan_sums_kernel(int64_t *__restrict__ tile_sums, int ntiles, int64_t *__restrict__ grand_total) {
    __shared__ int64_t warp_sums[kScanThreads / 32];
    int64_t carry = 0;
    for (int b0 = 0; b0 < ntiles; b0 += kScanThreads) {
        const int i = b0 + threadIdx.x;
        const int64_t v = i < ntiles ? tile_sums[i] : 0;
        int64_t total;
        const int64_t ex = block_exclusive_scan(v, warp_sums, &total);
        if (i < ntiles) tile_sums[i] = carry + ex;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *grand_total = carry;
}

__global__ void scan_add_kernel(int64_t *__restrict__ out, int n,
                                const int64_t *__restrict__ tile_sums) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += tile_sums[i / kScanTile];
}

// --------------------------------------------------------------- probes ---

// FP32 FFMA throughput: 8 independent dependent chains per thread.
__global__ void __launch_bounds__(256) fma_probe_kernel(float *out, int iters, float m, float b) {
    float x0 = threadIdx.x * 1e-7f, x1 = x0 + 1.f, x2 = x0 + 2.f, x3 = x0 + 3.f;
    float x4 = x0 + 4.f, x5 = x0 + 5.f, x6 = x0 + 6.f, x7 = x0 + 7.f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            x0 = fmaf(x0, m, b); x1 = fmaf(x1, m, b); x2 = fmaf(x2, m, b); x3 = fmaf(x3, m, b);
            x4 = fmaf(x4, m, b); x5 = fmaf(x5, m, b); x6 = fmaf(x6, m, b); x7 = fmaf(x7, m, b);
        }
    }
    const float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// FP64 DFMA throughput: the same chains in double precision.
__global__ void __launch_bounds__(256) dfma_probe_kernel(double *out, int iters, double m, double b) {
    double x0 = threadIdx.x * 1e-7, x1 = x0 + 1.0, x2 = x0 + 2.0, x3 = x0 + 3.0;
    double x4 = x0 + 4.0, x5 = x0 + 5.0, x6 = x0 + 6.0, x7 = x0 + 7.0;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            x0 = fma(x0, m, b); x1 = fma(x1, m, b); x2 = fma(x2, m, b); x3 = fma(x3, m, b);
            x4 = fma(x4, m, b); x5 = fma(x5, m, b); x6 = fma(x6, m, b); x7 = fma(x7, m, b);
        }
    }
    const double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 1234.5) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace p2p
