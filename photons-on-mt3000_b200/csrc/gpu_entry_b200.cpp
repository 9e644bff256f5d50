// PhotoNs gpu_entry boundary served by the B200 library (the drop-in for
// src/gpu_entry.cu + src/gpu_func.impl.h). Compiled inside a PhotoNs source
// tree, against its photoNs.h, with its -D flags:
//   CPU_DP / INTXYZ   layout of Body (inc/typedef.h:24-46), as in PhotoNs
//   GPU_DP            selects the plain FP64 form (default: the FP32/FP64
//                     split form); PHOTONS_P2P_FORM=plain|split overrides
//   GPUCUTOFF         pair cutoff x > 2.8125 (src/gpu_kernel.impl.h:192-196)
// The functions read the same globals the reference's versions read and keep
// its call protocol, ownership and print-and-exit error behaviour; the
// declarations are listed in include/photons_gpu_entry.h.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

extern "C" {
#include "photoNs.h"
}
#include "photons_p2p.h"

namespace {

p2p_session *g_sess = nullptr;
int g_call_cnt = 0;
long long g_tot_tasks = 0;
bool g_pass_open = false;
double *g_out = nullptr;  // h_part_buf of the reference
int g_out_n = 0;
int64_t g_uploaded = 0;   // position bytes the last pass uploaded

void check(const char *where, int status);

// Page-locked staging the module owns (grow-only, freed by devfree): the
// packed positions and leaf table of the open pass, and the rebased lists
// of p2ppack_compute_gpu. Copies from them are asynchronous, so they stay
// untouched until the pass has ended (get_last_kntime) or the next begins.
struct Pinned {
    void *p = nullptr;
    size_t cap = 0;
    void *get(size_t bytes) {
        if (bytes > cap) {
            if (p) p2p_host_free(p);
            p = nullptr;
            cap = 0;
            const size_t want = bytes + bytes / 8;
            check("p2p_host_alloc", p2p_host_alloc(want, &p));
            cap = want;
        }
        return p;
    }
    void release() {
        if (p) p2p_host_free(p);
        p = nullptr;
        cap = 0;
    }
};
Pinned g_pin_pos, g_pin_leaf, g_pin_tasks, g_pin_out;
// Particles whose packed positions g_pin_pos holds from the previous pass
// (-1: none): the next pass compares while packing and uploads only the
// chunks that changed (p2p_pass_begin_update).
int g_pin_pos_n = -1;
constexpr int kDirtyChunk = 1 << 16;

[[noreturn]] void die(const char *where, int status) {
    // checkDevErrors, src/gpu_func.impl.h:70-86
    fprintf(stderr, "Device runtime error in %s: %s (%s)\n", where, p2p_status_string(status),
            p2p_last_error());
    exit(EXIT_FAILURE);
}

void check(const char *where, int status) {
    if (status != P2P_OK) die(where, status);
}

int choose_form() {
    const char *env = getenv("PHOTONS_P2P_FORM");
    if (env && !strcmp(env, "plain")) return P2P_FORM_PLAIN_FP64;
    if (env && !strcmp(env, "split")) return P2P_FORM_SPLIT;
#ifdef GPU_DP
    return P2P_FORM_PLAIN_FP64;
#else
    return P2P_FORM_SPLIT;
#endif
}

// initGPU (src/gpu_func.impl.h:428-454, non-INTRA_LB): ranks share devices.
void init_device() {
    if (g_sess) return;
    int ndev = 0;
    check("p2p_device_count", p2p_device_count(&ndev));
    if (ndev <= 0) {
        printf("No available device\n");
        exit(0);
    }
    int dev;
    if (PROC_SIZE / ndev == 0)
        dev = PROC_RANK;
    else
        dev = (PROC_RANK % PROC_SIZE) / (PROC_SIZE / ndev);
    if (dev >= ndev) dev = dev % ndev;
    check("p2p_session_create", p2p_session_create(dev, &g_sess));
}

void set_pass_params() {
    p2p_params p;
    p2p_params_default(&p);
    p.form = choose_form();
    p.soft_mode = P2P_SOFT_CLAMP;  // P2P_kernel3 calls P2P_core_lite
    p.soften = SoftenScale;
    p.split_radius = splitRadius;
#ifdef GPUCUTOFF
    p.x_cut = 2.8125;
#else
    p.x_cut = 0.0;
#endif
    p.mass = MASSPART;
    check("p2p_session_set_params", p2p_session_set_params(g_sess, &p));
}

// SoA pack of the particle positions (src/gpu_entry.cu:85-105) and the leaf
// table (:108-111), then the first-call upload (devMemcpyHD_part). The pack
// goes into the module's page-locked staging, which keeps the previous
// pass's positions: each chunk of 65536 particles is compared (bit for bit)
// while it is packed, and only chunks that changed are uploaded over the
// copy the session keeps on the device.
void begin_pass() {
    init_device();
    set_pass_params();
    const int n = NPART;
    const int nleaf = last_leaf - first_leaf;
    const void *before = g_pin_pos.p;
    double *pos = (double *)g_pin_pos.get(sizeof(double) * 3 * (size_t)(n > 0 ? n : 1));
    const bool have_old = g_pin_pos_n == n && pos == before;
    const int nchunk = (n + kDirtyChunk - 1) / kDirtyChunk;
    std::vector<unsigned char> dirty((size_t)(nchunk > 0 ? nchunk : 1), have_old ? 0 : 1);
    // (the reference packs on one thread; the chunks are independent)
#pragma omp parallel for schedule(static)
    for (int c = 0; c < nchunk; ++c) {
        const int i1 = (c + 1) * kDirtyChunk < n ? (c + 1) * kDirtyChunk : n;
        unsigned char changed = 0;
        for (int i = c * kDirtyChunk; i < i1; ++i) {
            for (int d = 0; d < 3; ++d) {
#ifndef INTXYZ
                const double v = part[i].pos[d];
#else
                const double v = INT2POS * (part[i].posi[d] - domain_center_i[d]);
#endif
                double &slot = pos[(size_t)d * n + i];
                if (have_old) {
                    uint64_t a, b;
                    std::memcpy(&a, &slot, 8);
                    std::memcpy(&b, &v, 8);
                    changed |= (unsigned char)(a != b);
                }
                slot = v;
            }
        }
        if (have_old) dirty[(size_t)c] = changed;
    }
    g_pin_pos_n = -1;
    int *ip = (int *)g_pin_leaf.get(sizeof(int) * 2 * (size_t)(nleaf > 0 ? nleaf : 1));
    int *np = ip + nleaf;
    for (int l = 0; l < nleaf; ++l) {
        ip[l] = leaf[l + first_leaf].ipart;
        np[l] = leaf[l + first_leaf].npart;
    }
    check("p2p_pass_begin_update",
          p2p_pass_begin_update(g_sess, n, pos, nleaf, ip, np, dirty.data(), kDirtyChunk, &g_uploaded));
    g_pin_pos_n = n;
    g_pass_open = true;
}

// Active-level passes (hierarchical time steps). The particles such a pass
// changes: the reference's download adds a result where level == -1 or
// (level != 0 and act == level) (updateAcc_fromHostBuff,
// src/gpu_func.impl.h:644-653); built with ACT_OPT, the kernel of
// task_compute_p2p_act_gpu also leaves a sink at zero unless its act, as a
// byte, equals the level as a byte (P2P_kernel, src/gpu_kernel.impl.h:392-396),
// so a result it adds there is zero.
bool act_updates(int act, int level, bool kernel_filter) {
    if (kernel_filter && (unsigned char)act != (unsigned char)level) return false;
    return level == -1 || (level != 0 && act == level);
}

#ifdef ACT_OPT
constexpr bool kActKernelFilter = true;
#else
constexpr bool kActKernelFilter = false;
#endif

// Per leaf of the pass (0-based): 1 if it holds a particle the active-level
// pass changes. Only the rows of those sink leaves are submitted: every other
// row's results the reference computes and then does not add (or adds as
// zeros), so the sums are the same with less work.
std::vector<unsigned char> g_leaf_live;
std::vector<int> g_act_tasks;  // the kept entries of a chunk (pageable: staged by the submit)

void mark_live_leaves(int level, bool kernel_filter) {
    const int nleaf = last_leaf - first_leaf;
    g_leaf_live.assign((size_t)(nleaf > 0 ? nleaf : 1), 0);
#pragma omp parallel for schedule(static)
    for (int l = 0; l < nleaf; ++l) {
        const int a = leaf[l + first_leaf].ipart, b = a + leaf[l + first_leaf].npart;
        unsigned char live = 0;
        for (int j = a; j < b && !live; ++j) live = act_updates(part[j].act, level, kernel_filter) ? 1 : 0;
        g_leaf_live[(size_t)l] = live;
    }
}

// Copies the entries whose sink leaf is live to t / s as 0-based leaf ids
// (tin / sin hold ids base-based; t / s must not overlap them), keeping their
// order; returns how many. Blocks are counted, then filled, in parallel.
int64_t keep_live_rows(int64_t m, const int *tin, const int *sin, int base, int *t, int *s) {
    constexpr int kBlocks = 256;
    int64_t cnt[kBlocks + 1];
    const int nleaf = last_leaf - first_leaf;
    auto live = [&](int64_t j) {
        const int l = tin[j] - base;
        return l >= 0 && l < nleaf && g_leaf_live[(size_t)l];
    };
#pragma omp parallel for schedule(static)
    for (int b = 0; b < kBlocks; ++b) {
        int64_t c = 0;
        for (int64_t j = m * b / kBlocks; j < m * (b + 1) / kBlocks; ++j) c += live(j) ? 1 : 0;
        cnt[b + 1] = c;
    }
    cnt[0] = 0;
    for (int b = 0; b < kBlocks; ++b) cnt[b + 1] += cnt[b];
#pragma omp parallel for schedule(static)
    for (int b = 0; b < kBlocks; ++b) {
        int64_t o = cnt[b];
        for (int64_t j = m * b / kBlocks; j < m * (b + 1) / kBlocks; ++j)
            if (live(j)) {
                t[o] = tin[j] - base;
                s[o] = sin[j] - base;
                ++o;
            }
    }
    return cnt[kBlocks];
}

// Each pack's list rebased to 0-based leaf ids into the module's page-locked
// task staging and submitted to the open pass; with live, only the rows of
// live sink leaves.
void submit_packs(P2PPack *packs, int npack, bool live) {
    size_t total = 0;
    for (int n = 0; n < npack; ++n) total += (size_t)(packs[n].ntask > 0 ? packs[n].ntask : 0);
    int *buf = (int *)g_pin_tasks.get(sizeof(int) * 2 * (total > 0 ? total : 1));
    size_t off = 0;
    for (int n = 0; n < npack; ++n) {
        if (packs[n].ntask <= 0) continue;
        packs[n].rankid = 0;
        const int m = packs[n].ntask;
        int *t = buf + 2 * off, *s = t + m;
        int64_t k = m;
        if (live) {
            k = keep_live_rows(m, packs[n].task_t, packs[n].task_s, first_leaf, t, s);
        } else {
#pragma omp parallel for schedule(static)
            for (int j = 0; j < m; ++j) {
                t[j] = packs[n].task_t[j] - first_leaf;
                s[j] = packs[n].task_s[j] - first_leaf;
            }
        }
        if (k > 0) check("p2p_pass_submit", p2p_pass_submit(g_sess, k, t, s));
        off += (size_t)m;
    }
}

void update_acc(P2PPack *packs, int npack, int active_level, bool kernel_filter);

}  // namespace

extern "C" {

double get_last_kntime(int proc_rank);
void hostmalloc_out(int npart);
void hostfree_out(void);

void *task_compute_p2p_gpu(int ntask, int *ltask_t, int *ltask_s, int last_time) {
    const bool first_time = (g_call_cnt == 0);
    g_tot_tasks += ntask;
    g_call_cnt++;
    P2PPack *pack = packlist;
    pack->ntask = ntask;
    pack->task_t = ltask_t;
    pack->task_s = ltask_s;
    pack->ileaf = first_leaf;
    pack->nleaf = last_leaf - first_leaf;
    pack->ipart = 0;
    pack->npart = NPART;
    pack->rankid = 0;
    if (first_time) {
        NPACK++;
        begin_pass();
    }
    if (ntask > 0) {
        // devMemcpyHD_task rebases the caller's arrays in place (src/gpu_func.impl.h:704-713)
#pragma omp parallel for schedule(static)
        for (int j = 0; j < ntask; ++j) {
            ltask_t[j] -= first_leaf;
            ltask_s[j] -= first_leaf;
        }
        check("p2p_pass_submit", p2p_pass_submit(g_sess, ntask, ltask_t, ltask_s));
    }
    if (last_time) {
        g_tot_tasks = 0;
        g_call_cnt = 0;
    }
    return NULL;
}

// Every pack of the pass on the one device (the reference spreads packs over
// devices and gives each its own leaf and particle slices, src/gpu_entry.cu:211-386,
// src/gpu_func.impl.h:588-618): here the whole local tree is resident, so each
// pack's list, rebased to 0-based leaf ids, is one submit of the same pass.
// The reference rebases the caller's arrays in place by the pack's first leaf
// (devMemcpyHD_task, src/gpu_func.impl.h:704-713) and the caller does not
// read them again; this copy leaves them as they are.
void *p2ppack_compute_gpu(P2PPack *packs, int npack) {
    if (npack == 0) return NULL;
    begin_pass();
    submit_packs(packs, npack, false);
    return NULL;
}

// Active-level chunked pass: as task_compute_p2p_gpu, but only the particles
// of the level receive forces, and the last chunk also ends the pass and adds
// the result (get_last_kntime, hostmalloc_out, devMemcpyDH_updateAcc and
// hostfree_out inside the call). Replaces task_compute_p2p_act_gpu,
// src/gpu_active.impl.h:1-153. Like the reference, it rebases the caller's
// arrays in place; the rows of sink leaves without a particle of the level
// are not submitted.
void *task_compute_p2p_act_gpu(int ntask, int *ltask_t, int *ltask_s, int last_time, int active_level) {
    const bool first_time = (g_call_cnt == 0);
    g_tot_tasks += ntask;
    g_call_cnt++;
    P2PPack *pack = packlist;
    pack->ntask = ntask;
    pack->task_t = ltask_t;
    pack->task_s = ltask_s;
    pack->ileaf = first_leaf;
    pack->nleaf = last_leaf - first_leaf;
    pack->ipart = 0;
    pack->npart = NPART;
    pack->rankid = 0;
    if (first_time) {
        NPACK++;
        begin_pass();
        mark_live_leaves(active_level, kActKernelFilter);
    }
    if (ntask > 0) {
#pragma omp parallel for schedule(static)
        for (int j = 0; j < ntask; ++j) {
            ltask_t[j] -= first_leaf;
            ltask_s[j] -= first_leaf;
        }
        if (g_act_tasks.size() < 2 * (size_t)ntask) g_act_tasks.resize(2 * (size_t)ntask);
        int *t = g_act_tasks.data(), *s = t + ntask;
        const int64_t k = keep_live_rows(ntask, ltask_t, ltask_s, 0, t, s);
        if (k > 0) check("p2p_pass_submit", p2p_pass_submit(g_sess, k, t, s));
    }
    if (last_time) {
        g_tot_tasks = 0;
        g_call_cnt = 0;
        get_last_kntime(PROC_RANK);
        hostmalloc_out(NPART);
        update_acc(pack, NPACK, active_level, kActKernelFilter);
        hostfree_out();
    }
    return NULL;
}

// Multi-pack active-level pass: as p2ppack_compute_gpu, then the pass is
// ended and its result added for the particles of the level (here the
// reference's kernel computes every sink; only its download filters).
// Replaces p2ppack_compute_act_gpu, src/gpu_active.impl.h:155-321. The rows
// of sink leaves without a particle of the level are not submitted.
void *p2ppack_compute_act_gpu(P2PPack *packs, int npack, int active_level) {
    if (npack == 0) return NULL;
    begin_pass();
    mark_live_leaves(active_level, false);
    submit_packs(packs, npack, true);
    get_last_kntime(PROC_RANK);
    hostmalloc_out(NPART);
    update_acc(packs, NPACK, active_level, false);
    hostfree_out();
    return NULL;
}

void hostmalloc_task(int len) {
    task_s = (int *)mymalloc(sizeof(int) * (size_t)len, 58);
    task_t = (int *)mymalloc(sizeof(int) * (size_t)len, 59);
}

void hostrealloc_task(int len) {
    task_s = (int *)myrealloc(task_s, sizeof(int) * (size_t)len, 58);
    task_t = (int *)myrealloc(task_t, sizeof(int) * (size_t)len, 59);
}

void hostfree_task(void) {
    myfree(task_s, 58);
    myfree(task_t, 59);
}

double get_last_kntime(int proc_rank) {
    (void)proc_rank;
    if (!g_pass_open) return 0.0;
    double sec = 0.0;
    check("p2p_pass_end", p2p_pass_end(g_sess, &sec));
    g_pass_open = false;
    return sec;
}

// The result buffer is the module's page-locked staging (grow-only, kept
// until devfree), so the D2H is one pinned copy and no allocation per pass;
// these two only mark it reserved, as the reference's malloc / free did.
void hostmalloc_out(int npart) {
    g_out = (double *)g_pin_out.get(sizeof(double) * 3 * (size_t)(npart > 0 ? npart : 1));
    g_out_n = npart;
}

void hostfree_out(void) {
    g_out = nullptr;
    g_out_n = 0;
}

// D2H of the result, then acc[d][j] += buf over the particles of the packs
// (updateAcc_fromHostBuff, src/gpu_func.impl.h:644-681). The reference keeps
// one result slice per pack and adds each over its pack's particle range;
// here the pass leaves one total per particle, so it is added once for every
// particle that some pack covers (pack ranges may overlap: the walk's
// inter-subtree pack spans the others, src/fmm_LB.c:25-49,215-228).
void devMemcpyDH_updateAcc(P2PPack *packs, int npack, int active_level) {
    update_acc(packs, npack, active_level, false);
}

}  // extern "C"

namespace {

// devMemcpyDH_updateAcc; kernel_filter adds the ACT_OPT sink test of the
// active-level pass (act_updates).
void update_acc(P2PPack *packs, int npack, int active_level, bool kernel_filter) {
    if (!g_sess) return;
    bool any = false;
    for (int n = 0; n < npack; ++n) any = any || packs[n].ntask != 0;
    if (!any) return;
    if (!g_out || g_out_n < NPART) {
        fprintf(stderr, "devMemcpyDH_updateAcc: hostmalloc_out(%d) missing\n", NPART);
        exit(EXIT_FAILURE);
    }
    check("p2p_pass_result", p2p_pass_result(g_sess, g_out));
    const int n = NPART;
    // the union of the packs' particle ranges, as sorted disjoint intervals
    int *lo = (int *)malloc(sizeof(int) * 2 * (size_t)(npack > 0 ? npack : 1));
    int *hi = lo + npack;
    int nr = 0;
    for (int p = 0; p < npack; ++p) {
        if (packs[p].ntask == 0 || packs[p].npart <= 0) continue;
        int a = packs[p].ipart, b = packs[p].ipart + packs[p].npart, k = nr++;
        while (k > 0 && lo[k - 1] > a) {  // insertion by start
            lo[k] = lo[k - 1];
            hi[k] = hi[k - 1];
            --k;
        }
        lo[k] = a;
        hi[k] = b;
    }
    int m = 0;
    for (int k = 0; k < nr; ++k) {
        if (m > 0 && lo[k] <= hi[m - 1]) {
            if (hi[k] > hi[m - 1]) hi[m - 1] = hi[k];
        } else {
            lo[m] = lo[k];
            hi[m] = hi[k];
            ++m;
        }
    }
    for (int r = 0; r < m; ++r) {
        const int a = lo[r] < 0 ? 0 : lo[r], b = hi[r] > n ? n : hi[r];
#pragma omp parallel for schedule(static)
        for (int j = a; j < b; ++j) {
            if (act_updates(part[j].act, active_level, kernel_filter)) {
                acc[0][j] += g_out[j];
                acc[1][j] += g_out[(size_t)n + j];
                acc[2][j] += g_out[2 * (size_t)n + j];
            }
        }
    }
    free(lo);
}

}  // namespace

extern "C" {

void devfree(void) {
    if (g_sess) p2p_session_destroy(g_sess);
    g_sess = nullptr;
    g_pin_pos.release();
    g_pin_leaf.release();
    g_pin_tasks.release();
    g_pin_out.release();
    std::vector<unsigned char>().swap(g_leaf_live);
    std::vector<int>().swap(g_act_tasks);
    g_pin_pos_n = -1;
    g_out = nullptr;
    g_out_n = 0;
    g_pass_open = false;
    g_call_cnt = 0;
    g_tot_tasks = 0;
}

void dinfofree(void) {}

int64_t p2p_dropin_last_upload_bytes(void) { return g_uploaded; }

void sync_with_dev(void) {
    if (g_sess) check("p2p_session_synchronize", p2p_session_synchronize(g_sess));
}

}  // extern "C"
