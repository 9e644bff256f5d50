// Caller side of the P2P pass: the tree build and interaction-list walk that
// PhotoNs runs before it calls task_compute_p2p_gpu, restated in C++ so the
// library's tests, benchmark and serving loop can produce lists without the
// reference program. The algorithms follow the reference step for step so the
// lists are identical entry for entry (same leaves, same particle order, same
// emission order):
//   bksort_inplace       src/fmm.c:69-122   (mean split, sampled above 1e5)
//   build_kdtree         src/fmm.c:231-270  (pre-order leaf / node numbering)
//   center_kdtree        src/fmm.c:273-327  (box centres and widths)
//   leaf.active          src/fmm.c:1226-1236
//   acceptance           src/fmm.c:409-479  (LONGSHORT cutoff, open angle)
//   walk_task_p2p        src/fmm.c:656-792  (dual-tree walk, one-sided lists)
//   particle_combine     src/gravity.c:15-140 (float-rounded bounds)
//   periodic ghosts      src/boundary.c:592-680 restated for one domain
// What differs is only how the work is scheduled: the walk is cut into
// independent sub-walks at a fixed depth, run on OpenMP threads and
// concatenated in the serial order, so the output equals the serial walk.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct Node {
    int son[2];  // encoded child: leaf l -> 2*l, node k -> 2*k+1
    double split;
    double width[3];
    double center[3];
};

struct Leaf {
    int ipart, npart, active;
    double width[3];
    double center[3];
};

struct Tree {
    int npart = 0;
    std::vector<Node> nodes;
    std::vector<Leaf> leaves;
};

inline bool is_node(int c) { return c & 1; }
inline int cidx(int c) { return c >> 1; }

// Particle record moved by the partition, as the reference moves whole Body
// structs; id is the particle's original index, tag its local/ghost flag.
struct Rec {
    double pos[3];
    int id;
    int tag;
};

// bksort_inplace, src/fmm.c:69-122 (non-INTXYZ). Returns the left count and
// the split through *split.
void bksort(int D, Rec *p, int length, int npart[2], double *split) {
    npart[0] = npart[1] = 0;
    if (length < 2) {
        npart[1] = length;
        return;
    }
    if (length == 2) {
        npart[0] = npart[1] = 1;
        *split = 0.5 * (p[0].pos[D] + p[1].pos[D]);
        if (p[0].pos[D] > p[1].pos[D]) std::swap(p[0], p[1]);
        return;
    }
    double mean = 0.0;
    int mul = 1;
    if (length > 100000) mul = length / 100000;
    for (int n = 0; n < length; n += mul) mean += p[n].pos[D];
    mean /= (double)length;
    mean *= (double)mul;
    int but = length - 1;
    int n = 0;
    while (n < but) {
        if (p[n].pos[D] > mean) {
            Rec temp = p[n];
            while (p[but].pos[D] > mean && but > n) but--;
            p[n] = p[but];
            p[but] = temp;
        }
        n++;
    }
    npart[0] = but;
    npart[1] = length - npart[0];
    *split = mean;
}

// A subtree built with local numbering; merged into the global pre-order
// numbering afterwards.
struct SubTree {
    std::vector<Node> nodes;   // nodes[0] is the subtree root
    std::vector<Leaf> leaves;
};

void build_serial(SubTree &st, Rec *part, int direct, int ipart, int length, int inode,
                  int maxleaf) {
    // build_kdtree, src/fmm.c:231-270: pre-order numbering, son 0 first.
    Rec *p = part + ipart;
    int np[2];
    double split = 0.0;
    bksort(direct, p, length, np, &split);
    st.nodes[inode].split = split;
    int ip = ipart;
    int nd = (direct + 1) % 3;
    for (int n = 0; n < 2; ++n) {
        if (np[n] <= maxleaf) {
            Leaf lf{};
            lf.ipart = ip;
            lf.npart = np[n];
            st.leaves.push_back(lf);
            st.nodes[inode].son[n] = 2 * (int)(st.leaves.size() - 1);
        } else {
            st.nodes.push_back(Node{});
            int k = (int)st.nodes.size() - 1;
            st.nodes[inode].son[n] = 2 * k + 1;
            build_serial(st, part, nd, ip, np[n], k, maxleaf);
        }
        ip += np[n];
    }
}

// Top part of the tree, split in parallel down to subtrees of at most
// `grain` particles (or depth limit); those are built as independent tasks.
struct TopItem {
    // Either an internal top node (children given) or a frontier subtree.
    bool frontier;
    int direct, ipart, length;
    int son_item[2];      // for top nodes: child items (or -1 when the child is a leaf)
    int leaf_npart[2];    // for top nodes whose child is a leaf
    double split;
};

int top_split(std::vector<TopItem> &items, Rec *part, int direct, int ipart, int length,
              int maxleaf, int grain, int depth) {
    int me = (int)items.size();
    items.push_back(TopItem{});
    items[me].direct = direct;
    items[me].ipart = ipart;
    items[me].length = length;
    if (length <= grain || depth >= 24) {
        items[me].frontier = true;
        return me;
    }
    items[me].frontier = false;
    int np[2];
    double split = 0.0;
    bksort(direct, part + ipart, length, np, &split);
    items[me].split = split;
    int ip = ipart;
    int nd = (direct + 1) % 3;
    for (int n = 0; n < 2; ++n) {
        if (np[n] <= maxleaf) {
            items[me].son_item[n] = -1;
            items[me].leaf_npart[n] = np[n];
        } else {
            int c = top_split(items, part, nd, ip, np[n], maxleaf, grain, depth + 1);
            items[me].son_item[n] = c;
        }
        ip += np[n];
    }
    return me;
}

// Assign global pre-order ids: walk the top skeleton in the serial order,
// splicing in frontier subtrees.
void splice(Tree &T, const std::vector<TopItem> &items, std::vector<SubTree> &subs,
            const std::vector<int> &sub_of_item, int item, int gnode) {
    const TopItem &it = items[item];
    if (it.frontier) {
        // Subtree root is gnode; its other nodes follow in local order.
        SubTree &st = subs[sub_of_item[item]];
        int node_base = gnode;        // local node k -> node_base + k
        int leaf_base = (int)T.leaves.size();
        // nodes were reserved by the caller for the root only; append the rest
        for (size_t k = 1; k < st.nodes.size(); ++k) T.nodes.push_back(Node{});
        for (size_t k = 0; k < st.nodes.size(); ++k) {
            Node nd = st.nodes[k];
            for (int n = 0; n < 2; ++n) {
                int c = nd.son[n];
                nd.son[n] = is_node(c) ? 2 * (node_base + cidx(c)) + 1 : 2 * (leaf_base + cidx(c));
            }
            T.nodes[node_base + k] = nd;
        }
        for (auto &lf : st.leaves) T.leaves.push_back(lf);
        return;
    }
    T.nodes[gnode].split = it.split;
    int ip = it.ipart;
    for (int n = 0; n < 2; ++n) {
        if (it.son_item[n] < 0) {
            Leaf lf{};
            lf.ipart = ip;
            lf.npart = it.leaf_npart[n];
            T.leaves.push_back(lf);
            T.nodes[gnode].son[n] = 2 * (int)(T.leaves.size() - 1);
            ip += it.leaf_npart[n];
        } else {
            T.nodes.push_back(Node{});
            int k = (int)T.nodes.size() - 1;
            T.nodes[gnode].son[n] = 2 * k + 1;
            splice(T, items, subs, sub_of_item, it.son_item[n], k);
            ip += items[it.son_item[n]].length;
        }
    }
}

// center_kdtree, src/fmm.c:273-327.
void center_tree(Tree &T, int direct, int inode, double left[3], double right[3]) {
    Node &nd = T.nodes[inode];
    for (int d = 0; d < 3; ++d) {
        nd.width[d] = right[d] - left[d];
        nd.center[d] = 0.5 * (right[d] + left[d]);
    }
    int newd = (direct + 1) % 3;
    for (int n = 0; n < 2; ++n) {
        int c = nd.son[n];
        if (!is_node(c)) {
            Leaf &lf = T.leaves[cidx(c)];
            for (int d = 0; d < 3; ++d) {
                lf.width[d] = nd.width[d];
                lf.center[d] = nd.center[d];
            }
            if (n == 0) {
                lf.width[direct] = nd.split - left[direct];
                lf.center[direct] = 0.5 * (left[direct] + nd.split);
            } else {
                lf.width[direct] = right[direct] - nd.split;
                lf.center[direct] = 0.5 * (right[direct] + nd.split);
            }
        } else {
            double tmp;
            if (n == 0) {
                tmp = right[direct];
                right[direct] = nd.split;
                center_tree(T, newd, cidx(c), left, right);
                right[direct] = tmp;
            } else {
                tmp = left[direct];
                left[direct] = nd.split;
                center_tree(T, newd, cidx(c), left, right);
                left[direct] = tmp;
            }
        }
    }
}

// acceptance, src/fmm.c:409-479 with LONGSHORT: 0 open, 1 accept (M2L), -1 drop.
inline int acceptance(const double wi[3], const double wj[3], const double dist[3],
                      double cutoff, double open_angle) {
    double mn[3], w[3];
    w[0] = (wi[0] + wj[0]) * 0.5;
    w[1] = (wi[1] + wj[1]) * 0.5;
    w[2] = (wi[2] + wj[2]) * 0.5;
    mn[0] = dist[0];
    mn[1] = dist[1];
    mn[2] = dist[2];
    double dd2 = dist[0] * dist[0] + dist[1] * dist[1] + dist[2] * dist[2];
    for (int d = 0; d < 3; ++d) {
        if (mn[d] < 0.0) mn[d] = -mn[d];
        mn[d] -= w[d];
        if (mn[d] <= 0.0) mn[d] = 0.0;
    }
    if (mn[0] + mn[1] + mn[2] < 1.0e-15) return 0;
    double dm2 = mn[0] * mn[0] + mn[1] * mn[1] + mn[2] * mn[2];
    double c2 = cutoff * cutoff;
    if (dm2 > c2) return -1;
    double wmax = w[0];
    if (w[1] > wmax) wmax = w[1];
    if (w[2] > wmax) wmax = w[2];
    wmax = std::fabs(wmax);
    wmax *= 2;
    if (wmax * wmax < open_angle * open_angle * dd2) return 1;
    return 0;
}

struct Walker {
    const Tree &T;
    double cutoff, open_angle;
    const std::vector<char> *node_has_sink;  // null: no pruning
    int defer_depth;                 // < 0: never defer
    std::vector<int> *out_t, *out_s; // emitted (sink, source) leaf ids
    std::vector<int64_t> *deferred;  // packed (im, jm) deferred calls, in order
    std::vector<int64_t> *seq;       // sequence: >=0 deferred index, <0 inline emit slot

    void emit(int im, int jm) {
        if (T.leaves[cidx(im)].active < 0) return;
        if (seq) seq->push_back(-(int64_t)out_t->size() - 1);
        out_t->push_back(cidx(im));
        out_s->push_back(cidx(jm));
    }
    const double *ctr(int c) const {
        return is_node(c) ? T.nodes[cidx(c)].center : T.leaves[cidx(c)].center;
    }
    const double *wid(int c) const {
        return is_node(c) ? T.nodes[cidx(c)].width : T.leaves[cidx(c)].width;
    }
    // walk_task_p2p, src/fmm.c:656-792.
    void walk(int im, int jm, int depth) {
        // a sink-side subtree without an active leaf emits nothing: skip it
        if (node_has_sink && is_node(im) && !(*node_has_sink)[cidx(im)]) return;
        if (defer_depth >= 0 && depth >= defer_depth && (is_node(im) || is_node(jm))) {
            seq->push_back((int64_t)deferred->size());
            deferred->push_back(((int64_t)im << 32) | (uint32_t)jm);
            return;
        }
        if (im == jm) {
            if (!is_node(im)) {
                emit(im, jm);
            } else {
                const Node &a = T.nodes[cidx(im)];
                walk(a.son[0], a.son[0], depth + 1);
                walk(a.son[0], a.son[1], depth + 1);
                walk(a.son[1], a.son[0], depth + 1);
                walk(a.son[1], a.son[1], depth + 1);
            }
            return;
        }
        if (!is_node(im) && !is_node(jm)) {
            emit(im, jm);
            return;
        }
        const double *ci = ctr(im), *cj = ctr(jm);
        double dist[3] = {ci[0] - cj[0], ci[1] - cj[1], ci[2] - cj[2]};
        if (!is_node(im)) {  // leaf - node
            int flag = acceptance(wid(im), wid(jm), dist, cutoff, open_angle);
            if (flag == 0) {
                const Node &b = T.nodes[cidx(jm)];
                walk(im, b.son[0], depth + 1);
                walk(im, b.son[1], depth + 1);
            }
            return;
        }
        if (!is_node(jm)) {  // node - leaf
            int flag = acceptance(wid(jm), wid(im), dist, cutoff, open_angle);
            if (flag == 0) {
                const Node &a = T.nodes[cidx(im)];
                walk(a.son[0], jm, depth + 1);
                walk(a.son[1], jm, depth + 1);
            }
            return;
        }
        int flag = acceptance(wid(im), wid(jm), dist, cutoff, open_angle);
        if (flag == 0) {
            const Node &a = T.nodes[cidx(im)], &b = T.nodes[cidx(jm)];
            if (a.width[0] + a.width[1] + a.width[2] > b.width[0] + b.width[1] + b.width[2]) {
                walk(a.son[0], jm, depth + 1);
                walk(a.son[1], jm, depth + 1);
            } else {
                walk(im, b.son[0], depth + 1);
                walk(im, b.son[1], depth + 1);
            }
        }
    }
};

}  // namespace

extern "C" {

struct p2p_tree_s {
    Tree T;
    std::vector<int> task_t, task_s;
};
typedef struct p2p_tree_s p2p_tree;

// Periodic ghost images for one domain [origin, origin + box)^3: every image
// x + s*box (s in {-1,0,1}^3, s != 0) that lies strictly within `width` of
// the domain on every axis. Images are written particle by particle, shifts
// in lexicographic order. With out_pos == NULL only the count is returned.
int64_t p2p_make_ghosts(int n, const double *pos, double origin, double box, double width,
                        double *out_pos, int64_t out_cap, int *out_src) {
    const double lo = origin - width, hi = origin + box + width;
    std::vector<int64_t> cnt((size_t)n + 1, 0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        int c = 0;
        for (int sx = -1; sx <= 1; ++sx)
            for (int sy = -1; sy <= 1; ++sy)
                for (int sz = -1; sz <= 1; ++sz) {
                    if (!sx && !sy && !sz) continue;
                    double q[3] = {pos[i] + sx * box, pos[(size_t)n + i] + sy * box,
                                   pos[2 * (size_t)n + i] + sz * box};
                    if (q[0] > lo && q[0] < hi && q[1] > lo && q[1] < hi && q[2] > lo && q[2] < hi) c++;
                }
        cnt[i + 1] = c;
    }
    for (int i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
    int64_t total = cnt[n];
    if (!out_pos) return total;
    if (total > out_cap) return -1;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        int64_t k = cnt[i];
        for (int sx = -1; sx <= 1; ++sx)
            for (int sy = -1; sy <= 1; ++sy)
                for (int sz = -1; sz <= 1; ++sz) {
                    if (!sx && !sy && !sz) continue;
                    double q[3] = {pos[i] + sx * box, pos[(size_t)n + i] + sy * box,
                                   pos[2 * (size_t)n + i] + sz * box};
                    if (q[0] > lo && q[0] < hi && q[1] > lo && q[1] < hi && q[2] > lo && q[2] < hi) {
                        out_pos[k] = q[0];
                        out_pos[(size_t)out_cap + k] = q[1];
                        out_pos[2 * (size_t)out_cap + k] = q[2];
                        if (out_src) out_src[k] = i;
                        k++;
                    }
                }
    }
    return total;
}

// Builds the kd-tree over npart particles (SoA pos, tag 1 local / 0 ghost).
// boxsize is BOXSIZE (enters the bounds margin of particle_combine). On
// return pos is permuted into tree order and perm[i] holds the original index
// of tree slot i. Returns a handle, or NULL.
p2p_tree *p2p_tree_build(int npart, double *pos, const int *tag, int maxleaf, double boxsize,
                         int *perm) {
    if (npart <= 0 || maxleaf <= 0) return nullptr;
    p2p_tree *h = new p2p_tree();
    Tree &T = h->T;
    T.npart = npart;
    std::vector<Rec> part((size_t)npart);
    double boxL[3] = {boxsize, boxsize, boxsize}, boxH[3] = {0.0, 0.0, 0.0};
    for (int n = 0; n < npart; ++n) {
        Rec &r = part[n];
        r.id = n;
        r.tag = tag ? tag[n] : 1;
        for (int d = 0; d < 3; ++d) r.pos[d] = pos[(size_t)d * npart + n];
        float fp[3] = {(float)r.pos[0], (float)r.pos[1], (float)r.pos[2]};
        for (int d = 0; d < 3; ++d) {
            if (boxL[d] > fp[d]) boxL[d] = fp[d];
            if (boxH[d] < fp[d]) boxH[d] = fp[d];
        }
    }
    for (int d = 0; d < 3; ++d) {
        boxL[d] -= 0.000001 * boxsize;
        boxH[d] += 0.000001 * boxsize;
    }
    // Top skeleton in parallel, frontier subtrees as tasks.
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
#endif
    int grain = std::max(4 * maxleaf, npart / (64 * nthreads));
    std::vector<TopItem> items;
    if (npart <= maxleaf) {
        // The reference splits the root even when it would fit one leaf.
        grain = 0;
    }
    top_split(items, part.data(), 0, 0, npart, maxleaf, grain, 0);
    std::vector<int> sub_of_item(items.size(), -1);
    std::vector<int> frontier;
    for (size_t i = 0; i < items.size(); ++i)
        if (items[i].frontier) {
            sub_of_item[i] = (int)frontier.size();
            frontier.push_back((int)i);
        }
    std::vector<SubTree> subs(frontier.size());
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t f = 0; f < frontier.size(); ++f) {
        const TopItem &it = items[frontier[f]];
        SubTree &st = subs[f];
        st.nodes.push_back(Node{});
        build_serial(st, part.data(), it.direct, it.ipart, it.length, 0, maxleaf);
    }
    T.nodes.push_back(Node{});
    splice(T, items, subs, sub_of_item, 0, 0);
    center_tree(T, 0, 0, boxL, boxH);
    for (auto &lf : T.leaves) {
        lf.active = -1;
        for (int i = 0; i < lf.npart; ++i)
            if (part[lf.ipart + i].tag == 1) {
                lf.active = 0;
                break;
            }
    }
    for (int n = 0; n < npart; ++n) {
        perm[n] = part[n].id;
        for (int d = 0; d < 3; ++d) pos[(size_t)d * npart + n] = part[n].pos[d];
    }
    return h;
}

void p2p_tree_free(p2p_tree *h) { delete h; }

int p2p_tree_nleaf(const p2p_tree *h) { return (int)h->T.leaves.size(); }
int p2p_tree_nnode(const p2p_tree *h) { return (int)h->T.nodes.size(); }

// Leaf table in leaf-id order: ipart, npart, active, centre and width (AoS).
void p2p_tree_leaves(const p2p_tree *h, int *ipart, int *npart, int *active, double *center,
                     double *width) {
    const Tree &T = h->T;
    for (size_t l = 0; l < T.leaves.size(); ++l) {
        const Leaf &lf = T.leaves[l];
        if (ipart) ipart[l] = lf.ipart;
        if (npart) npart[l] = lf.npart;
        if (active) active[l] = lf.active;
        for (int d = 0; d < 3; ++d) {
            if (center) center[3 * l + d] = lf.center[d];
            if (width) width[3 * l + d] = lf.width[d];
        }
    }
}

// Node table in node-id order for the device walk: child codes (2 per
// node), the smallest leaf id of each subtree, centre and width (AoS).
void p2p_tree_nodes(const p2p_tree *h, int *son, int *first_leaf, double *center, double *width) {
    const Tree &T = h->T;
    const int nn = (int)T.nodes.size();
    if (first_leaf) {
        // children have larger pre-order ids than their parent: fill bottom-up
        for (int k = nn - 1; k >= 0; --k) {
            const int c = T.nodes[k].son[0];
            first_leaf[k] = is_node(c) ? first_leaf[cidx(c)] : cidx(c);
        }
    }
    for (int k = 0; k < nn; ++k) {
        const Node &nd = T.nodes[k];
        if (son) {
            son[2 * k] = nd.son[0];
            son[2 * k + 1] = nd.son[1];
        }
        for (int d = 0; d < 3; ++d) {
            if (center) center[3 * k + d] = nd.center[d];
            if (width) width[3 * k + d] = nd.width[d];
        }
    }
}

namespace {
// has_sink[node] = the subtree holds a leaf with active >= 0
char mark_sinks(const Tree &T, int c, std::vector<char> &has) {
    if (!is_node(c)) return T.leaves[cidx(c)].active >= 0;
    const Node &n = T.nodes[cidx(c)];
    const char a = mark_sinks(T, n.son[0], has);
    const char b = mark_sinks(T, n.son[1], has);
    return has[cidx(c)] = (char)(a || b);
}
int64_t walk_impl(p2p_tree *h, double cutoff, double open_angle, const std::vector<char> *prune);
}  // namespace

// Runs the P2P walk from (root, root). Returns the number of list entries
// kept inside the handle (fetch them with p2p_tree_tasks).
int64_t p2p_tree_walk(p2p_tree *h, double cutoff, double open_angle) {
    return walk_impl(h, cutoff, open_angle, nullptr);
}

// The walk restricted to the sink leaves with sink_mask[leaf] != 0 (others
// are treated as inactive sinks, like ghost-only leaves). The emitted entries
// are exactly the unrestricted walk's entries whose sink is kept, in the
// same order; subtrees without a kept sink are not descended into.
int64_t p2p_tree_walk_masked(p2p_tree *h, double cutoff, double open_angle,
                             const unsigned char *sink_mask) {
    Tree &T = h->T;
    std::vector<int> saved(T.leaves.size());
    for (size_t l = 0; l < T.leaves.size(); ++l) {
        saved[l] = T.leaves[l].active;
        if (!sink_mask[l]) T.leaves[l].active = -1;
    }
    std::vector<char> has(T.nodes.size(), 0);
    mark_sinks(T, 1, has);
    const int64_t n = walk_impl(h, cutoff, open_angle, &has);
    for (size_t l = 0; l < T.leaves.size(); ++l) T.leaves[l].active = saved[l];
    return n;
}

namespace {
int64_t walk_impl(p2p_tree *h, double cutoff, double open_angle, const std::vector<char> *prune) {
    const Tree &T = h->T;
    h->task_t.clear();
    h->task_s.clear();
    const int root = 1;  // node 0, encoded
    std::vector<int> top_t, top_s;
    std::vector<int64_t> deferred, seq;
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
#endif
    int depth = 12;
    if (nthreads > 1) depth = 16;
    {
        Walker w{T, cutoff, open_angle, prune, depth, &top_t, &top_s, &deferred, &seq};
        w.walk(root, root, 0);
    }
    std::vector<std::vector<int>> dt(deferred.size()), ds(deferred.size());
#pragma omp parallel for schedule(dynamic, 4)
    for (size_t k = 0; k < deferred.size(); ++k) {
        int im = (int)(deferred[k] >> 32), jm = (int)(uint32_t)deferred[k];
        Walker w{T, cutoff, open_angle, prune, -1, &dt[k], &ds[k], nullptr, nullptr};
        w.walk(im, jm, 0);
    }
    // Concatenate in serial order.
    std::vector<int64_t> off(seq.size() + 1, 0);
    for (size_t q = 0; q < seq.size(); ++q)
        off[q + 1] = off[q] + (seq[q] >= 0 ? (int64_t)dt[(size_t)seq[q]].size() : 1);
    int64_t total = off[seq.size()];
    h->task_t.resize((size_t)total);
    h->task_s.resize((size_t)total);
#pragma omp parallel for schedule(dynamic, 64)
    for (size_t q = 0; q < seq.size(); ++q) {
        int64_t o = off[q];
        if (seq[q] >= 0) {
            const auto &a = dt[(size_t)seq[q]];
            const auto &b = ds[(size_t)seq[q]];
            std::memcpy(&h->task_t[(size_t)o], a.data(), sizeof(int) * a.size());
            std::memcpy(&h->task_s[(size_t)o], b.data(), sizeof(int) * b.size());
        } else {
            int64_t e = -seq[q] - 1;
            h->task_t[(size_t)o] = top_t[(size_t)e];
            h->task_s[(size_t)o] = top_s[(size_t)e];
        }
    }
    return total;
}
}  // namespace

void p2p_tree_tasks(const p2p_tree *h, int *task_t, int *task_s) {
    std::memcpy(task_t, h->task_t.data(), sizeof(int) * h->task_t.size());
    std::memcpy(task_s, h->task_s.data(), sizeof(int) * h->task_s.size());
}

int p2p_lists_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
