// Device interaction-list walk: the P2P lists of PhotoNs' dual-tree walk
// (walk_task_p2p, src/fmm.c:656-792, with the LONGSHORT acceptance test of
// src/fmm.c:409-479) computed per sink leaf on the GPU, straight into CSR rows.
//
// The serial walk recurses over leaf/node pairs (A, B) from (root, root). An
// entry (L, S) is emitted when the recursion reaches two leaves. For a fixed
// sink leaf L the pairs it visits on the way to L's entries have A on L's
// ancestor path, and which child of A the recursion takes is fixed by L (the
// child whose subtree holds L); how a pair expands depends on the pair alone.
// So one warp per sink leaf expands that part of the recursion, its lanes
// taking up to 32 pending pairs at a time from a shared-memory stack. The
// serial walk emits a sink's sources in pre-order of the source side, i.e. in
// increasing leaf id (leaves are numbered in pre-order and son[0]'s subtree is
// walked before son[1]'s); sorting each row ascending afterwards therefore
// gives the serial order, the row a stable sort of the serial list by sink
// gives: the rows equal those the list path builds, entry for entry.
//
// The acceptance arithmetic is written with explicitly rounded FP64
// operations (no contraction), the ISO C evaluation of the reference's code.
#pragma once

#include "p2p_device_common.cuh"

namespace p2p {

struct WalkArgs {
    int nnode, nleaf;
    const int *son;           // 2 * nnode encoded children: leaf l -> 2l, node k -> 2k + 1
    const int *node_first;    // nnode: smallest leaf id in the node's subtree
    const int *leaf_active;   // nleaf: >= 0 for leaves holding a local particle (sinks)
    const double *node_center, *node_width;  // 3 * nnode
    const double *leaf_center, *leaf_width;  // 3 * nleaf
    double cutoff, open_angle;
};

enum : int {
    ST_WALK_STACK = 4,    // a sink's pending pairs exceeded the walk's stack (its row is cut short)
    ST_WALK_ROW = 8,      // the fill pass found more entries than the count pass
    ST_WALK_TREE = 16,    // a child code outside the tree, or a walk longer than any tree allows
};

__device__ __forceinline__ const double *walk_center(const WalkArgs &w, int c) {
    return (c & 1) ? w.node_center + 3 * (size_t)(c >> 1) : w.leaf_center + 3 * (size_t)(c >> 1);
}
__device__ __forceinline__ const double *walk_width(const WalkArgs &w, int c) {
    return (c & 1) ? w.node_width + 3 * (size_t)(c >> 1) : w.leaf_width + 3 * (size_t)(c >> 1);
}

// acceptance (LONGSHORT), src/fmm.c:409-479: 0 open, 1 accept (M2L), -1 drop.
__device__ __forceinline__ int walk_acceptance(const double *wi, const double *wj, const double *ci,
                                               const double *cj, double cutoff, double open_angle) {
    double dist[3], w[3], mn[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        dist[d] = __dsub_rn(ci[d], cj[d]);
        w[d] = __dmul_rn(__dadd_rn(wi[d], wj[d]), 0.5);
    }
    const double dd2 = __dadd_rn(__dadd_rn(__dmul_rn(dist[0], dist[0]), __dmul_rn(dist[1], dist[1])),
                                 __dmul_rn(dist[2], dist[2]));
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double m = dist[d] < 0.0 ? -dist[d] : dist[d];
        m = __dsub_rn(m, w[d]);
        mn[d] = m <= 0.0 ? 0.0 : m;
    }
    if (__dadd_rn(__dadd_rn(mn[0], mn[1]), mn[2]) < 1.0e-15) return 0;
    const double dm2 = __dadd_rn(__dadd_rn(__dmul_rn(mn[0], mn[0]), __dmul_rn(mn[1], mn[1])),
                                 __dmul_rn(mn[2], mn[2]));
    if (dm2 > __dmul_rn(cutoff, cutoff)) return -1;
    double wmax = w[0];
    if (w[1] > wmax) wmax = w[1];
    if (w[2] > wmax) wmax = w[2];
    wmax = fabs(wmax);
    wmax = __dmul_rn(wmax, 2.0);
    if (__dmul_rn(wmax, wmax) < __dmul_rn(__dmul_rn(open_angle, open_angle), dd2)) return 1;
    return 0;
}

__device__ __forceinline__ bool walk_valid(const WalkArgs &w, int c) {
    return c >= 0 && ((c & 1) ? (c >> 1) < w.nnode : (c >> 1) < w.nleaf);
}

// The child of node code A whose subtree holds leaf L (pre-order leaf ids:
// son[0]'s leaves precede son[1]'s); -1 for a child code outside the tree.
__device__ __forceinline__ int walk_child_toward(const WalkArgs &w, int A, int L) {
    const int k = A >> 1;
    const int s1 = w.son[2 * k + 1];
    if (!walk_valid(w, s1)) return -1;
    const int f1 = (s1 & 1) ? w.node_first[s1 >> 1] : (s1 >> 1);
    return L < f1 ? w.son[2 * k] : s1;
}

constexpr int kWalkWarps = 4;         // warps (sink leaves in flight) per block
constexpr int kWalkWarpStack = 1024;  // pending pairs per warp (shared memory)

// One warp per sink leaf. FILL = false: row lengths into counts[L]; with a
// slab, also the row's first slab_cap source ids into slab[L * slab_cap ...]
// (walk_gather_kernel moves them into the rows). FILL = true: the row's
// source ids into row_src[row_off[L] ...] (in the order the warp finds them;
// the rows are sorted afterwards), the row's pair count (and, with skipped,
// the pairs of entries wholly beyond the FP32 forms' cutoff) added into
// *pairs / *skipped; with slab_cap > 0 only for the rows longer than
// slab_cap (counts[L] from the first pass), the others having been gathered.
template <bool FILL>
__global__ void __launch_bounds__(kWalkWarps * 32)
walk_rows_kernel(const WalkArgs w, int *__restrict__ counts, const int64_t *__restrict__ row_off,
                 int *__restrict__ row_src, const int *__restrict__ leaf_npart,
                 const LeafMeta *__restrict__ meta, double cscale, float uout,
                 unsigned long long *__restrict__ pairs, unsigned long long *__restrict__ skipped,
                 int *__restrict__ status, int *__restrict__ slab, int slab_cap) {
    __shared__ int2 stacks[kWalkWarps][kWalkWarpStack];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    int2 *stk = stacks[wid];
    unsigned long long my_pairs = 0, my_skip = 0;
    for (int L = blockIdx.x * kWalkWarps + wid; L < w.nleaf; L += gridDim.x * kWalkWarps) {
        if (w.leaf_active[L] < 0 || w.nnode <= 0) {  // warp-uniform
            if (!FILL && lane == 0) counts[L] = 0;
            continue;
        }
        if (FILL && slab_cap > 0 && counts[L] <= slab_cap) continue;  // gathered from the slab (warp-uniform)
        if (lane == 0) stk[0] = make_int2(1, 1);  // (root, root): node 0
        __syncwarp();
        int sp = 1, n = 0, bad = 0;
        int64_t base = 0, cap = 0;
        LeafMeta mt{};
        long long np_t = 0;
        if (FILL) {
            base = row_off[L];
            cap = row_off[L + 1] - base;
            np_t = leaf_npart[L];
            if (skipped) mt = meta[L];
        }
        // every pair is visited at most once per sink: a longer walk means a
        // malformed tree
        long long budget = 64LL * ((long long)w.nnode + w.nleaf) + 16;
        while (sp > 0) {
            const int take = min(32, sp);
            sp -= take;
            budget -= take;
            int2 p = make_int2(0, 0);
            if (lane < take) p = stk[sp + lane];
            __syncwarp();  // the batch is read before children overwrite it
            const int A = p.x, B = p.y;
            int nchild = 0, c0 = 0, c1 = 0, fault = 0;
            bool emit = false;
            if (lane < take) {
                const bool a_node = A & 1, b_node = B & 1;
                if ((A == B && !a_node) || (!a_node && !b_node)) {
                    emit = true;
                } else if (A == B) {
                    const int c = walk_child_toward(w, A, L);
                    const int k = A >> 1;
                    c0 = c;  // the pairs (c, son[0]) and (c, son[1]): second codes below
                    nchild = 2;
                    p = make_int2(w.son[2 * k], w.son[2 * k + 1]);
                } else {
                    const double *wa = walk_width(w, A), *wb = walk_width(w, B);
                    if (walk_acceptance(wa, wb, walk_center(w, A), walk_center(w, B), w.cutoff,
                                        w.open_angle) == 0) {
                        bool split_a = a_node && !b_node;
                        if (a_node && b_node)
                            split_a = __dadd_rn(__dadd_rn(wa[0], wa[1]), wa[2]) >
                                      __dadd_rn(__dadd_rn(wb[0], wb[1]), wb[2]);
                        if (split_a) {
                            c0 = walk_child_toward(w, A, L);
                            c1 = B;
                            nchild = 1;
                        } else {
                            const int k = B >> 1;
                            c0 = A;
                            nchild = 2;
                            p = make_int2(w.son[2 * k], w.son[2 * k + 1]);
                        }
                    }
                }
            }
            // children as (first, second) codes: nchild 1 -> (c0, c1);
            // nchild 2 -> (c0, p.x), (c0, p.y)
            int2 ch0 = nchild == 1 ? make_int2(c0, c1) : make_int2(c0, p.x);
            int2 ch1 = make_int2(c0, p.y);
            if (nchild >= 1 && (!walk_valid(w, ch0.x) || !walk_valid(w, ch0.y))) fault = ST_WALK_TREE;
            if (nchild == 2 && !walk_valid(w, ch1.y)) fault = ST_WALK_TREE;
            if (fault) nchild = 0;
            int incl = nchild;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const int v = __shfl_up_sync(kFull, incl, off);
                if (lane >= off) incl += v;
            }
            const int total = __shfl_sync(kFull, incl, 31);
            bad |= __reduce_or_sync(kFull, fault);
            if (sp + total > kWalkWarpStack) {
                bad |= ST_WALK_STACK;
            } else {
                const int at = sp + incl - nchild;
                if (nchild >= 1) stk[at] = ch0;
                if (nchild == 2) stk[at + 1] = ch1;
                sp += total;
            }
            const unsigned em = __ballot_sync(kFull, emit);
            if (emit) {
                const int slot = n + __popc(em & lt);
                const int S = B >> 1;
                if (!FILL && slab && slot < slab_cap) slab[(int64_t)L * slab_cap + slot] = S;
                if (FILL) {
                    if (slot < cap) {
                        row_src[base + slot] = S;
                        const unsigned long long np = (unsigned long long)(np_t * (long long)leaf_npart[S]);
                        my_pairs += np;
                        if (skipped) {
                            const LeafMeta ms = meta[S];
                            float ox, oy, oz;
                            entry_offset(ms, mt, cscale, ox, oy, oz);
                            if (entry_u_min(ms, mt, ox, oy, oz) > uout) my_skip += np;
                        }
                    }
                }
            }
            n += __popc(em);
            if (FILL && n > cap) bad |= ST_WALK_ROW;
            if (budget < 0) bad |= ST_WALK_TREE;
            __syncwarp();
            if (bad) break;  // warp-uniform
        }
        if (lane == 0) {
            if (!FILL) counts[L] = n;
            if (bad) atomicOr(status, bad);
        }
    }
    if (FILL) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            my_pairs += __shfl_xor_sync(kFull, my_pairs, off);
            my_skip += __shfl_xor_sync(kFull, my_skip, off);
        }
        if (lane == 0) {
            if (my_pairs) atomicAdd(pairs, my_pairs);
            if (skipped && my_skip) atomicAdd(skipped, my_skip);
        }
    }
}

// Rows of at most slab_cap entries, from the first pass's slab into their
// CSR rows (in the order the walk found them; the row sort follows), with the
// pair counts the fill pass would add. One warp per sink leaf; a row whose
// offsets disagree with its length, or an id outside the leaves, sets
// ST_WALK_ROW and is skipped.
__global__ void __launch_bounds__(256)
walk_gather_kernel(const int *__restrict__ counts, const int64_t *__restrict__ row_off, int nleaf,
                   const int *__restrict__ slab, int slab_cap, int *__restrict__ row_src,
                   const int *__restrict__ leaf_npart, const LeafMeta *__restrict__ meta, double cscale,
                   float uout, unsigned long long *__restrict__ pairs, unsigned long long *__restrict__ skipped,
                   int *__restrict__ status) {
    const int lane = threadIdx.x & 31;
    const int nw = (int)(((int64_t)gridDim.x * blockDim.x) >> 5);
    unsigned long long my_pairs = 0, my_skip = 0;
    int bad = 0;
    for (int L = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5); L < nleaf; L += nw) {
        const int n = counts[L];
        if (n <= 0 || n > slab_cap) continue;  // warp-uniform
        const int64_t base = row_off[L];
        if (row_off[L + 1] - base != n) {
            bad = ST_WALK_ROW;
            continue;
        }
        const long long np_t = leaf_npart[L];
        LeafMeta mt{};
        if (skipped) mt = meta[L];
        for (int i = lane; i < n; i += 32) {
            const int S = slab[(int64_t)L * slab_cap + i];
            if ((unsigned)S >= (unsigned)nleaf) {
                bad = ST_WALK_ROW;
                continue;
            }
            row_src[base + i] = S;
            const unsigned long long np = (unsigned long long)(np_t * (long long)leaf_npart[S]);
            my_pairs += np;
            if (skipped) {
                const LeafMeta ms = meta[S];
                float ox, oy, oz;
                entry_offset(ms, mt, cscale, ox, oy, oz);
                if (entry_u_min(ms, mt, ox, oy, oz) > uout) my_skip += np;
            }
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        my_pairs += __shfl_xor_sync(kFull, my_pairs, off);
        my_skip += __shfl_xor_sync(kFull, my_skip, off);
    }
    if (lane == 0) {
        if (my_pairs) atomicAdd(pairs, my_pairs);
        if (skipped && my_skip) atomicAdd(skipped, my_skip);
    }
    if (bad) atomicOr(status, bad);
}

}  // namespace p2p
