// Device interaction-list walk: the P2P lists of PhotoNs' dual-tree walk
// (walk_task_p2p, src/fmm.c:656-792, with the LONGSHORT acceptance test of
// src/fmm.c:409-479) computed per sink leaf on the GPU, straight into CSR rows.
//
// The serial walk recurses over leaf/node pairs (A, B) from (root, root). An
// entry (L, S) is emitted when the recursion reaches two leaves. For a fixed
// sink leaf L the pairs it visits on the way to its entries have A on L's
// ancestor path, and which child of A the recursion takes is fixed by L; so
// one thread per sink leaf replays exactly the part of the recursion whose
// sink side contains L, depth first with the children in the serial order.
// Its entries come out in the order the serial walk emits them for that sink,
// which is the row order a stable sort of the serial list by sink gives: the
// rows equal those the list path builds, entry for entry.
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

constexpr int kWalkStack = 192;  // pending (A, B) pairs per sink leaf

enum : int {
    ST_WALK_STACK = 4,    // a sink's pending pairs exceeded kWalkStack (its row is cut short)
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

// One thread per sink leaf. FILL = false: row lengths into counts[L].
// FILL = true: the row's source ids into row_src[row_off[L] ...], the row's
// pair count (and, with skipped, the pairs of entries wholly beyond the
// FP32 forms' cutoff) added into *pairs / *skipped.
template <bool FILL>
__global__ void __launch_bounds__(128)
walk_rows_kernel(const WalkArgs w, int *__restrict__ counts, const int64_t *__restrict__ row_off,
                 int *__restrict__ row_src, const int *__restrict__ leaf_npart,
                 const LeafMeta *__restrict__ meta, double cscale, float uout,
                 unsigned long long *__restrict__ pairs, unsigned long long *__restrict__ skipped,
                 int *__restrict__ status) {
    unsigned long long my_pairs = 0, my_skip = 0;
    const int stride = gridDim.x * blockDim.x;
    for (int L = blockIdx.x * blockDim.x + threadIdx.x; L < w.nleaf; L += stride) {
        if (w.leaf_active[L] < 0 || w.nnode <= 0) {
            if (!FILL) counts[L] = 0;
            continue;
        }
        int2 stack[kWalkStack];
        int sp = 0;
        stack[sp++] = make_int2(1, 1);  // (root, root): node 0
        int n = 0;
        int64_t base = 0, cap = 0;
        LeafMeta mt{};
        long long np_t = 0;
        if (FILL) {
            base = row_off[L];
            cap = row_off[L + 1] - base;
            np_t = leaf_npart[L];
            if (skipped) mt = meta[L];
        }
        int bad = 0;
        // a pair (A, B) is visited at most once per sink, A on the sink's
        // ancestor path: any longer walk means a malformed tree
        long long budget = 64LL * ((long long)w.nnode + w.nleaf) + 16;
        auto emit = [&](int B) {
            const int S = B >> 1;
            if (FILL) {
                if (n >= cap) {
                    bad = ST_WALK_ROW;
                    return;
                }
                row_src[base + n] = S;
                const unsigned long long np = (unsigned long long)(np_t * (long long)leaf_npart[S]);
                my_pairs += np;
                if (skipped) {
                    const LeafMeta ms = meta[S];
                    float ox, oy, oz;
                    entry_offset(ms, mt, cscale, ox, oy, oz);
                    if (entry_u_min(ms, mt, ox, oy, oz) > uout) my_skip += np;
                }
            }
            ++n;
        };
        auto push = [&](int A, int B) {
            if (!walk_valid(w, A) || !walk_valid(w, B)) bad = ST_WALK_TREE;
            else if (sp < kWalkStack) stack[sp++] = make_int2(A, B);
            else bad = ST_WALK_STACK;
        };
        while (sp > 0 && !bad) {
            if (--budget < 0) {
                bad = ST_WALK_TREE;
                break;
            }
            const int2 p = stack[--sp];
            const int A = p.x, B = p.y;
            if (A == B) {
                if (!(A & 1)) {
                    emit(B);
                } else {
                    const int c = walk_child_toward(w, A, L);
                    const int k = A >> 1;
                    push(c, w.son[2 * k + 1]);
                    push(c, w.son[2 * k]);
                }
                continue;
            }
            const bool a_node = A & 1, b_node = B & 1;
            if (!a_node && !b_node) {
                emit(B);
                continue;
            }
            // (the reference passes the leaf's width first in the node-leaf
            // case; the sum of the two widths is the same either way)
            const double *wa = walk_width(w, A), *wb = walk_width(w, B);
            if (walk_acceptance(wa, wb, walk_center(w, A), walk_center(w, B), w.cutoff, w.open_angle) != 0)
                continue;
            if (!a_node) {  // leaf - node: both children of B, son[0] first
                const int k = B >> 1;
                push(A, w.son[2 * k + 1]);
                push(A, w.son[2 * k]);
            } else if (!b_node) {  // node - leaf: the child of A toward L
                push(walk_child_toward(w, A, L), B);
            } else {
                const double sa = __dadd_rn(__dadd_rn(wa[0], wa[1]), wa[2]);
                const double sb = __dadd_rn(__dadd_rn(wb[0], wb[1]), wb[2]);
                if (sa > sb) {
                    push(walk_child_toward(w, A, L), B);
                } else {
                    const int k = B >> 1;
                    push(A, w.son[2 * k + 1]);
                    push(A, w.son[2 * k]);
                }
            }
        }
        if (bad) atomicOr(status, bad);
        if (!FILL) counts[L] = n;
    }
    if (FILL) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            my_pairs += __shfl_xor_sync(kFull, my_pairs, off);
            my_skip += __shfl_xor_sync(kFull, my_skip, off);
        }
        if ((threadIdx.x & 31) == 0) {
            if (my_pairs) atomicAdd(pairs, my_pairs);
            if (skipped && my_skip) atomicAdd(skipped, my_skip);
        }
    }
}

}  // namespace p2p
