// Device kd-tree build (C ABI p2p_dtree_*; kernels in p2p_tree_kernels.cuh).
//
// Replaces the caller's build_kdtree / center_kdtree (src/fmm.c:69-122,
// 231-327) plus the leaf.active marking (src/fmm.c:1226-1236) on the GPU,
// producing the same tree: nodes and leaves in the reference's pre-order
// numbering, the same particle order, node and leaf boxes, active flags.
// The result feeds p2p_pass_begin_device (positions in tree order, leaf
// ranges) and p2p_pass_submit_walk (the node and leaf tables) directly.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "photons_p2p.h"
#include "p2p_host_shared.h"
#include "p2p_tree_kernels.cuh"

#define P2P_API extern "C" __attribute__((visibility("default")))

using namespace p2p;

struct p2p_dtree {
    int device = 0;
    int npart = 0, nleaf = 0, nnode = 0;
    double *pos = nullptr;  // SoA, tree order
    int *perm = nullptr;    // tree slot -> input index
    int *leaf_ipart = nullptr, *leaf_npart = nullptr, *leaf_active = nullptr;
    double *leaf_center = nullptr, *leaf_width = nullptr;  // AoS, 3 per leaf
    int *son = nullptr, *node_first = nullptr;
    double *node_center = nullptr, *node_width = nullptr;  // AoS, 3 per node
    float build_ms = 0.f;
    int cap_part = 0, cap_leaf = 0, cap_node = 0;  // sizes the arrays were allocated for
};

namespace {

void free_tree(p2p_dtree *t) {
    void *ptrs[] = {t->pos, t->perm, t->leaf_ipart, t->leaf_npart, t->leaf_active, t->leaf_center,
                    t->leaf_width, t->son, t->node_first, t->node_center, t->node_width};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    t->pos = t->leaf_center = t->leaf_width = t->node_center = t->node_width = nullptr;
    t->perm = t->leaf_ipart = t->leaf_npart = t->leaf_active = t->son = t->node_first = nullptr;
    t->cap_part = t->cap_leaf = t->cap_node = 0;
    t->npart = t->nleaf = t->nnode = 0;
}

// Temporaries of one build, in the session's grow-only scratch (one slot
// per request, numbered in request order): a rebuild of the same size
// allocates and frees nothing. The build returns only after its last kernel
// has finished, so the next build may reuse every slot.
struct Scratch {
    p2p_session *s;
    int next = 0;
    template <class T>
    bool get(T **out, size_t count) {
        void *p = session_scratch(s, next++, sizeof(T) * (count > 0 ? count : 1));
        if (!p) return false;
        *out = (T *)p;
        return true;
    }
};

template <class T>
bool dev_alloc(T **out, size_t count) {
    void *p = nullptr;
    if (cudaMalloc(&p, sizeof(T) * (count > 0 ? count : 1)) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    *out = (T *)p;
    return true;
}

int cuda_fail(cudaError_t e, const char *what) {
    char msg[256];
    snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
    cudaGetLastError();
    return report_error(P2P_ERR_CUDA, msg);
}

#define TREE_CUDA(expr)                                  \
    do {                                                 \
        cudaError_t _e = (expr);                         \
        if (_e != cudaSuccess) return cuda_fail(_e, #expr); \
    } while (0)

int grid(int64_t n, int threads, int cap) {
    int64_t b = (n + threads - 1) / threads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, cap));
}

}  // namespace

namespace {

int check_build_args(p2p_session *s, int npart, const double *d_pos, int maxleaf, double boxsize) {
    if (!s) return report_error(P2P_ERR_ARG, "null argument");
    if (npart <= 0 || !d_pos) return report_error(P2P_ERR_ARG, "tree build needs particles");
    if (maxleaf <= 0) return report_error(P2P_ERR_ARG, "maxleaf must be positive");
    if (!(boxsize > 0.0)) return report_error(P2P_ERR_ARG, "boxsize must be positive");
    return P2P_OK;
}

// The tree's arrays for npart particles, nleaf leaves and nnode nodes: kept
// where they are large enough, else reallocated (with an eighth to spare,
// so rebuilds whose sizes drift reallocate rarely).
bool fit_tree(p2p_dtree *tree, int n, int nleaf, int nnode) {
    auto more = [](int c) { return (int)std::min<int64_t>((int64_t)c + c / 8 + 16, INT32_MAX); };
    bool ok = true;
    if (n > tree->cap_part) {
        cudaFree(tree->pos);
        cudaFree(tree->perm);
        tree->pos = nullptr;
        tree->perm = nullptr;
        const int c = more(n);
        ok = ok && dev_alloc(&tree->pos, 3 * (size_t)c) && dev_alloc(&tree->perm, c);
        tree->cap_part = ok ? c : 0;
    }
    if (ok && nleaf > tree->cap_leaf) {
        int **iv[] = {&tree->leaf_ipart, &tree->leaf_npart, &tree->leaf_active};
        double **dv[] = {&tree->leaf_center, &tree->leaf_width};
        for (int **p : iv) { cudaFree(*p); *p = nullptr; }
        for (double **p : dv) { cudaFree(*p); *p = nullptr; }
        const int c = more(nleaf);
        for (int **p : iv) ok = ok && dev_alloc(p, c);
        for (double **p : dv) ok = ok && dev_alloc(p, 3 * (size_t)c);
        tree->cap_leaf = ok ? c : 0;
    }
    if (ok && nnode > tree->cap_node) {
        cudaFree(tree->son);
        cudaFree(tree->node_first);
        cudaFree(tree->node_center);
        cudaFree(tree->node_width);
        tree->son = tree->node_first = nullptr;
        tree->node_center = tree->node_width = nullptr;
        const int c = more(nnode);
        ok = ok && dev_alloc(&tree->son, 2 * (size_t)c) && dev_alloc(&tree->node_first, c) &&
             dev_alloc(&tree->node_center, 3 * (size_t)c) && dev_alloc(&tree->node_width, 3 * (size_t)c);
        tree->cap_node = ok ? c : 0;
    }
    return ok;
}

// Builds into tree (its arrays reused where large enough). On an error the
// caller discards the tree's contents.
int build_into(p2p_session *s, p2p_dtree *tree, int npart, const double *d_pos, const int *d_tag, int maxleaf,
               double boxsize) {
    TREE_CUDA(cudaSetDevice(session_device(s)));
    cudaStream_t st = (cudaStream_t)p2p_session_stream(s);
    cudaEvent_t e0, e1;
    TREE_CUDA(cudaEventCreate(&e0));
    TREE_CUDA(cudaEventCreate(&e1));
    struct Events {
        cudaEvent_t a, b;
        ~Events() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } evs{e0, e1};
    TREE_CUDA(cudaEventRecord(e0, st));
    int launches = 0;

    const int n = npart;
    // Nodes and leaves: a binary tree has one leaf more than nodes; leaves
    // hold up to maxleaf particles and mean splits keep most of them over
    // half full. The capacity allows 8 / maxleaf of a leaf per particle.
    const int64_t cap64 = std::min<int64_t>((int64_t)n + 1, 8LL * n / maxleaf + 1024);
    const int cap = (int)cap64;

    Scratch S{s};
    TreeParts P;
    TreeRec R;
    std::memset(&R, 0, sizeof(R));
    int *map = nullptr;
    float *blo = nullptr, *bhi = nullptr;
    const int init_blocks = grid(n, kTreeThreads, 1024);
    bool ok = S.get(&P.x, n) && S.get(&P.y, n) && S.get(&P.z, n) && S.get(&P.id, n) && S.get(&map, n) &&
              S.get(&blo, 3 * (size_t)init_blocks) && S.get(&bhi, 3 * (size_t)init_blocks) &&
              S.get(&R.split, cap) && S.get(&R.son, 2 * (size_t)cap) && S.get(&R.depth, cap) &&
              S.get(&R.nn, cap) && S.get(&R.nl, cap) && S.get(&R.pre, cap) && S.get(&R.first, cap) &&
              S.get(&R.box, 6 * (size_t)cap) && S.get(&R.lipart, cap) && S.get(&R.lnpart, cap) &&
              S.get(&R.lid, cap) && S.get(&R.counters, 4);
    if (!ok) return report_error(P2P_ERR_NOMEM, "tree build: device allocation failed");
    R.node_cap = cap;
    R.leaf_cap = cap;

    tree_init_kernel<<<init_blocks, kTreeThreads, 0, st>>>(d_pos, n, P, blo, bhi);
    tree_root_box_kernel<<<1, 32, 0, st>>>(blo, bhi, init_blocks, boxsize, R, 0);
    launches += 2;

    // ---- nodes above kTreeSmall particles, level by level (host-driven) ----
    std::vector<int> h_son, h_depth, h_lipart, h_lnpart;  // records made on the host
    std::vector<TreeTask> tasks;
    std::vector<TreeSeg> segs;
    int nnode_h = 0, nleaf_h = 0, maxdepth = 0;
    if (n <= kTreeSmall) {
        tasks.push_back(TreeTask{0, n, 0, 0, -1, 0});  // the whole tree in one block
    } else {
        h_son.assign(2, -1);
        h_depth.assign(1, 0);
        nnode_h = 1;
        segs.push_back(TreeSeg{0, n, 0, 0, 0.0, 0, 0});
    }
    TreeSeg *d_segs = nullptr;
    int *d_tile_seg = nullptr, *d_tile_off = nullptr, *d_tile_pre = nullptr, *d_tile_small = nullptr;
    size_t seg_cap = 0, tile_cap = 0;
    int level = 0;
    while (!segs.empty()) {
        if (++level > 4096) return report_error(P2P_ERR_CAPACITY, "tree build: more than 4096 levels above 2048 particles");
        const int nseg = (int)segs.size();
        std::vector<int> tile_seg, tile_off;
        for (int g = 0; g < nseg; ++g)
            for (int o = 0; o < segs[g].length; o += kTreeTile) {
                tile_seg.push_back(g);
                tile_off.push_back(o);
            }
        const int ntile = (int)tile_seg.size();
        if ((size_t)nseg > seg_cap) {
            if (!S.get(&d_segs, 2 * (size_t)nseg)) return report_error(P2P_ERR_NOMEM, "tree build: allocation");
            seg_cap = 2 * (size_t)nseg;
        }
        if ((size_t)ntile > tile_cap) {
            if (!(S.get(&d_tile_seg, 2 * (size_t)ntile) && S.get(&d_tile_off, 2 * (size_t)ntile) &&
                  S.get(&d_tile_pre, 2 * (size_t)ntile) && S.get(&d_tile_small, 2 * (size_t)ntile)))
                return report_error(P2P_ERR_NOMEM, "tree build: allocation");
            tile_cap = 2 * (size_t)ntile;
        }
        TREE_CUDA(cudaMemcpyAsync(d_segs, segs.data(), sizeof(TreeSeg) * nseg, cudaMemcpyHostToDevice, st));
        TREE_CUDA(cudaMemcpyAsync(d_tile_seg, tile_seg.data(), sizeof(int) * ntile, cudaMemcpyHostToDevice, st));
        TREE_CUDA(cudaMemcpyAsync(d_tile_off, tile_off.data(), sizeof(int) * ntile, cudaMemcpyHostToDevice, st));
        tree_seg_mean_kernel<<<nseg, kTreeThreads, 0, st>>>(d_segs, P, R);
        tree_tile_count_kernel<<<ntile, kTreeThreads, 0, st>>>(d_segs, d_tile_seg, d_tile_off, P, d_tile_small);
        launches += 2;
        std::vector<int> tsmall(ntile), tpre(ntile);
        TREE_CUDA(cudaMemcpyAsync(tsmall.data(), d_tile_small, sizeof(int) * ntile, cudaMemcpyDeviceToHost, st));
        TREE_CUDA(cudaMemcpyAsync(segs.data(), d_segs, sizeof(TreeSeg) * nseg, cudaMemcpyDeviceToHost, st));  // means
        TREE_CUDA(cudaStreamSynchronize(st));
        for (auto &g : segs) g.nsmall = 0;
        for (int t = 0; t < ntile; ++t) {
            tpre[t] = segs[tile_seg[t]].nsmall;
            segs[tile_seg[t]].nsmall += tsmall[t];
        }
        for (auto &g : segs) g.nbig = g.length - g.nsmall;
        TREE_CUDA(cudaMemcpyAsync(d_segs, segs.data(), sizeof(TreeSeg) * nseg, cudaMemcpyHostToDevice, st));
        TREE_CUDA(cudaMemcpyAsync(d_tile_pre, tpre.data(), sizeof(int) * ntile, cudaMemcpyHostToDevice, st));
        tree_tile_map_kernel<<<ntile, kTreeThreads, 0, st>>>(d_segs, d_tile_seg, d_tile_off, d_tile_pre, P, map);
        tree_tile_swap_kernel<<<ntile, kTreeThreads, 0, st>>>(d_segs, d_tile_seg, d_tile_off, d_tile_pre, P, map);
        launches += 2;
        TREE_CUDA(cudaGetLastError());
        // children: leaves, subtrees for one block, or next level's nodes
        std::vector<TreeSeg> next;
        for (const TreeSeg &g : segs) {
            const int left = g.nbig == 0 ? g.length - 1 : g.nsmall;
            const int np[2] = {left, g.length - left};
            const int ip[2] = {g.ipart, g.ipart + left};
            const int depth = h_depth[g.node] + 1;
            const int axis = (g.axis + 1) % 3;
            for (int c = 0; c < 2; ++c) {
                if (np[c] <= maxleaf) {
                    h_lipart.push_back(ip[c]);
                    h_lnpart.push_back(np[c]);
                    h_son[2 * g.node + c] = 2 * nleaf_h++;
                } else if (np[c] <= kTreeSmall) {
                    tasks.push_back(TreeTask{ip[c], np[c], axis, depth, g.node, c});
                } else {
                    const int k = nnode_h++;
                    h_son.push_back(-1);
                    h_son.push_back(-1);
                    h_depth.push_back(depth);
                    maxdepth = std::max(maxdepth, depth);
                    h_son[2 * g.node + c] = 2 * k + 1;
                    next.push_back(TreeSeg{ip[c], np[c], axis, k, 0.0, 0, 0});
                }
            }
        }
        segs.swap(next);
    }
    if (nnode_h > cap || nleaf_h > cap) return report_error(P2P_ERR_CAPACITY, "tree build: node capacity");
    // host-made records to the device, then the counters for the blocks' atomics
    if (nnode_h) {
        TREE_CUDA(cudaMemcpyAsync(R.son, h_son.data(), sizeof(int) * 2 * nnode_h, cudaMemcpyHostToDevice, st));
        TREE_CUDA(cudaMemcpyAsync(R.depth, h_depth.data(), sizeof(int) * nnode_h, cudaMemcpyHostToDevice, st));
    }
    if (nleaf_h) {
        TREE_CUDA(cudaMemcpyAsync(R.lipart, h_lipart.data(), sizeof(int) * nleaf_h, cudaMemcpyHostToDevice, st));
        TREE_CUDA(cudaMemcpyAsync(R.lnpart, h_lnpart.data(), sizeof(int) * nleaf_h, cudaMemcpyHostToDevice, st));
    }
    int hc[4] = {nnode_h, nleaf_h, 0, maxdepth};
    TREE_CUDA(cudaMemcpyAsync(R.counters, hc, sizeof(hc), cudaMemcpyHostToDevice, st));

    // ---- subtrees of at most kTreeSmall particles, one block each ----
    if (!tasks.empty()) {
        TreeTask *d_tasks = nullptr;
        if (!S.get(&d_tasks, tasks.size())) return report_error(P2P_ERR_NOMEM, "tree build: allocation");
        TREE_CUDA(cudaMemcpyAsync(d_tasks, tasks.data(), sizeof(TreeTask) * tasks.size(), cudaMemcpyHostToDevice, st));
        TREE_CUDA(cudaFuncSetAttribute(tree_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kTreeSmallSmem));
        tree_small_kernel<<<(int)tasks.size(), kTreeThreads, kTreeSmallSmem, st>>>(d_tasks, P, R, maxleaf);
        launches += 1;
        TREE_CUDA(cudaGetLastError());
    }
    TREE_CUDA(cudaMemcpyAsync(hc, R.counters, sizeof(hc), cudaMemcpyDeviceToHost, st));
    TREE_CUDA(cudaStreamSynchronize(st));
    if (hc[2] & (TB_NODE_CAP | TB_LEAF_CAP))
        return report_error(P2P_ERR_CAPACITY, "tree build: more nodes or leaves than the build's capacity");
    const int nnode = hc[0], nleaf = hc[1];
    maxdepth = hc[3];

    // ---- pre-order numbering and boxes, by depth ----
    const int gn = grid(nnode, 256, 4096);
    for (int d = maxdepth; d >= 0; --d) tree_count_kernel<<<gn, 256, 0, st>>>(R, nnode, d);
    TREE_CUDA(cudaMemsetAsync(R.pre, 0, sizeof(int), st));    // the root (build id 0): pre-order id 0
    TREE_CUDA(cudaMemsetAsync(R.first, 0, sizeof(int), st));  // its first leaf: 0
    for (int d = 0; d <= maxdepth; ++d) tree_order_kernel<<<gn, 256, 0, st>>>(R, nnode, d);
    launches += 2 * (maxdepth + 1);

    p2p_dtree *t = tree;
    t->device = session_device(s);
    if (!fit_tree(t, n, nleaf, nnode)) return report_error(P2P_ERR_NOMEM, "tree build: device allocation failed");
    t->npart = n;
    t->nleaf = nleaf;
    t->nnode = nnode;
    tree_emit_kernel<<<gn, 256, 0, st>>>(R, nnode, nleaf, t->son, t->node_first, t->node_center, t->node_width,
                                         t->leaf_ipart, t->leaf_npart, t->leaf_center, t->leaf_width);
    {   // the numbering is consistent before the leaf tables are read
        int status = 0;
        cudaError_t ce = cudaMemcpyAsync(&status, R.counters + 2, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
        if (ce != cudaSuccess || (status & TB_NUMBERING)) {
            if (ce != cudaSuccess) return cuda_fail(ce, "tree build");
            return report_error(P2P_ERR_STATE, "tree build: inconsistent node records");
        }
    }
    tree_active_kernel<<<grid((int64_t)nleaf * 32, 256, 8192), 256, 0, st>>>(t->leaf_ipart, t->leaf_npart, nleaf,
                                                                            P.id, d_tag, t->leaf_active);
    tree_pos_out_kernel<<<grid(n, 256, 8192), 256, 0, st>>>(P, n, t->pos);
    launches += 3;
    cudaError_t e = cudaMemcpyAsync(t->perm, P.id, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecord(e1, st);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);  // the next build may reuse the scratch
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t->build_ms, e0, e1);
    if (e != cudaSuccess) return cuda_fail(e, "tree build");
    count_launches(launches);
    return P2P_OK;
}

}  // namespace

P2P_API int p2p_dtree_build(p2p_session *s, int npart, const double *d_pos, const int *d_tag, int maxleaf,
                            double boxsize, p2p_dtree **out) {
    if (!out) return report_error(P2P_ERR_ARG, "null argument");
    *out = nullptr;
    const int st = check_build_args(s, npart, d_pos, maxleaf, boxsize);
    if (st != P2P_OK) return st;
    p2p_dtree *t = new p2p_dtree();
    const int r = build_into(s, t, npart, d_pos, d_tag, maxleaf, boxsize);
    if (r != P2P_OK) {
        cudaSetDevice(t->device);
        free_tree(t);
        delete t;
        return r;
    }
    *out = t;
    return P2P_OK;
}

P2P_API int p2p_dtree_rebuild(p2p_session *s, p2p_dtree *t, int npart, const double *d_pos, const int *d_tag,
                              int maxleaf, double boxsize) {
    if (!t) return report_error(P2P_ERR_ARG, "null tree");
    const int st = check_build_args(s, npart, d_pos, maxleaf, boxsize);
    if (st != P2P_OK) return st;
    if ((t->pos || t->son) && t->device != session_device(s))
        return report_error(P2P_ERR_ARG, "tree and session are on different devices");
    const int r = build_into(s, t, npart, d_pos, d_tag, maxleaf, boxsize);
    if (r != P2P_OK) t->npart = t->nleaf = t->nnode = 0;  // no tree; its arrays stay for the next rebuild
    return r;
}

P2P_API int p2p_dtree_free(p2p_dtree *t) {
    if (!t) return P2P_OK;
    cudaSetDevice(t->device);
    free_tree(t);
    delete t;
    return P2P_OK;
}

P2P_API int p2p_dtree_counts(const p2p_dtree *t, int *npart, int *nleaf, int *nnode, float *build_ms) {
    if (!t) return report_error(P2P_ERR_ARG, "null tree");
    if (npart) *npart = t->npart;
    if (nleaf) *nleaf = t->nleaf;
    if (nnode) *nnode = t->nnode;
    if (build_ms) *build_ms = t->build_ms;
    return P2P_OK;
}

P2P_API int p2p_dtree_device_arrays(const p2p_dtree *t, const double **d_pos, const int **d_perm,
                                    const int **d_leaf_ipart, const int **d_leaf_npart) {
    if (!t) return report_error(P2P_ERR_ARG, "null tree");
    if (d_pos) *d_pos = t->pos;
    if (d_perm) *d_perm = t->perm;
    if (d_leaf_ipart) *d_leaf_ipart = t->leaf_ipart;
    if (d_leaf_npart) *d_leaf_npart = t->leaf_npart;
    return P2P_OK;
}

P2P_API int p2p_dtree_walk_tree(const p2p_dtree *t, p2p_walk_tree *w) {
    if (!t || !w) return report_error(P2P_ERR_ARG, "null argument");
    w->nnode = t->nnode;
    w->nleaf = t->nleaf;
    w->son = t->son;
    w->node_first = t->node_first;
    w->node_center = t->node_center;
    w->node_width = t->node_width;
    w->leaf_center = t->leaf_center;
    w->leaf_width = t->leaf_width;
    w->leaf_active = t->leaf_active;
    return P2P_OK;
}

P2P_API int p2p_dtree_unpermute(const p2p_dtree *t, p2p_session *s, const double *d_in, double *d_out) {
    if (!t || !s || !d_in || !d_out) return report_error(P2P_ERR_ARG, "null argument");
    if (d_in == d_out) return report_error(P2P_ERR_ARG, "unpermute needs distinct buffers");
    TREE_CUDA(cudaSetDevice(t->device));
    cudaStream_t st = (cudaStream_t)p2p_session_stream(s);
    tree_unpermute_kernel<<<grid(t->npart, 256, 8192), 256, 0, st>>>(d_in, t->perm, t->npart, d_out);
    TREE_CUDA(cudaGetLastError());
    count_launches(1);
    return P2P_OK;
}

P2P_API int p2p_dtree_download(const p2p_dtree *t, double *pos, int *perm, int *leaf_ipart, int *leaf_npart,
                               int *leaf_active, double *leaf_center, double *leaf_width, int *son,
                               int *node_first, double *node_center, double *node_width) {
    if (!t) return report_error(P2P_ERR_ARG, "null tree");
    TREE_CUDA(cudaSetDevice(t->device));
    struct Item {
        void *dst;
        const void *src;
        size_t bytes;
    } items[] = {{pos, t->pos, sizeof(double) * 3 * (size_t)t->npart},
                 {perm, t->perm, sizeof(int) * (size_t)t->npart},
                 {leaf_ipart, t->leaf_ipart, sizeof(int) * (size_t)t->nleaf},
                 {leaf_npart, t->leaf_npart, sizeof(int) * (size_t)t->nleaf},
                 {leaf_active, t->leaf_active, sizeof(int) * (size_t)t->nleaf},
                 {leaf_center, t->leaf_center, sizeof(double) * 3 * (size_t)t->nleaf},
                 {leaf_width, t->leaf_width, sizeof(double) * 3 * (size_t)t->nleaf},
                 {son, t->son, sizeof(int) * 2 * (size_t)t->nnode},
                 {node_first, t->node_first, sizeof(int) * (size_t)t->nnode},
                 {node_center, t->node_center, sizeof(double) * 3 * (size_t)t->nnode},
                 {node_width, t->node_width, sizeof(double) * 3 * (size_t)t->nnode}};
    for (const Item &it : items)
        if (it.dst && it.bytes) TREE_CUDA(cudaMemcpy(it.dst, it.src, it.bytes, cudaMemcpyDeviceToHost));
    return P2P_OK;
}
