/*
 * TEST INFRASTRUCTURE ONLY: drives the multi-pack entry point
 * p2ppack_compute_gpu of the B200 drop-in the way the reference's
 * load-balanced walk does (src/fmm.c:1245-1250 under INTRA_LB, packs made by
 * add_one_p2ppack, src/fmm_LB.c:25-49), then collects the result the way
 * gravity_fmm_pm_kick does (get_last_kntime, hostmalloc_out,
 * devMemcpyDH_updateAcc, hostfree_out; src/gravity.c:440-449). The tree is
 * given (particles in tree order and the leaf table); the reference's globals
 * come from its src/global.c, linked beside this file by oracle/build_ref.sh
 * into libref_dropin_{dp,sp,act}.so only.
 *
 * ref_act_run drives the active-level entry points the same way:
 * p2ppack_compute_act_gpu (src/gpu_active.impl.h:155-321) with the packs, or
 * task_compute_p2p_act_gpu (:1-153) over the concatenated list in chunks of
 * `chunk` entries, the last with last_time = 1, as turn2compute_p2p_act's
 * commented-out call would (src/fmm.c:1016-1025). Both add the result
 * themselves.
 */
#include <stdlib.h>
#include <string.h>
#include <mpi.h>
#include "photoNs.h"

void *p2ppack_compute_gpu(P2PPack *packs, int npack);
double get_last_kntime(int proc_rank);
void hostmalloc_out(int npart);
void hostfree_out(void);
void devMemcpyDH_updateAcc(P2PPack *packs, int npack, int active_level);
void *p2ppack_compute_act_gpu(P2PPack *packs, int npack, int active_level);
void *task_compute_p2p_act_gpu(int ntask, int *ltask_t, int *ltask_s, int last_time, int active_level);

static int run(int npart, const double *pos, int nleaf, const int *leaf_ipart, const int *leaf_npart,
               int leaf_base, double split_radius, double soften, double mass, int npack, const int *pack_ntask,
               const int *pack_ileaf, const int *pack_nleaf, const int *pack_ipart, const int *pack_npart,
               const int *task_t, const int *task_s, double *acc_out, double *kernel_seconds, const int *act,
               int mode, int active_level, int chunk);

/*
 * pos: SoA doubles of npart particles in tree order; leaf_ipart/leaf_npart:
 * nleaf leaves, stored from leaf id leaf_base on (the reference's biased
 * leaf pointer, first_leaf = leaf_base). Pack k holds pack_ntask[k] entries
 * of task_t/task_s (absolute leaf ids, concatenated in pack order) and the
 * ranges pack_ileaf/nleaf/ipart/npart. acc_out: SoA doubles, += result.
 */
int ref_pack_run(int npart, const double *pos, int nleaf, const int *leaf_ipart, const int *leaf_npart,
                 int leaf_base, double split_radius, double soften, double mass, int npack,
                 const int *pack_ntask, const int *pack_ileaf, const int *pack_nleaf, const int *pack_ipart,
                 const int *pack_npart, const int *task_t, const int *task_s, double *acc_out,
                 double *kernel_seconds) {
    return run(npart, pos, nleaf, leaf_ipart, leaf_npart, leaf_base, split_radius, soften, mass, npack, pack_ntask,
               pack_ileaf, pack_nleaf, pack_ipart, pack_npart, task_t, task_s, acc_out, kernel_seconds, NULL, 0, -1,
               0);
}

/* act: npart levels (part[i].act); mode 1: p2ppack_compute_act_gpu, mode 2:
 * task_compute_p2p_act_gpu in chunks of `chunk` entries. */
int ref_act_run(int npart, const double *pos, int nleaf, const int *leaf_ipart, const int *leaf_npart, int leaf_base,
                double split_radius, double soften, double mass, int npack, const int *pack_ntask,
                const int *pack_ileaf, const int *pack_nleaf, const int *pack_ipart, const int *pack_npart,
                const int *task_t, const int *task_s, double *acc_out, const int *act, int mode, int active_level,
                int chunk) {
    if ((mode != 1 && mode != 2) || (mode == 2 && (chunk <= 0 || npack < 1))) return -2;
    return run(npart, pos, nleaf, leaf_ipart, leaf_npart, leaf_base, split_radius, soften, mass, npack, pack_ntask,
               pack_ileaf, pack_nleaf, pack_ipart, pack_npart, task_t, task_s, acc_out, NULL, act, mode,
               active_level, chunk);
}

static int run(int npart, const double *pos, int nleaf, const int *leaf_ipart, const int *leaf_npart,
               int leaf_base, double split_radius, double soften, double mass, int npack, const int *pack_ntask,
               const int *pack_ileaf, const int *pack_nleaf, const int *pack_ipart, const int *pack_npart,
               const int *task_t, const int *task_s, double *acc_out, double *kernel_seconds, const int *act,
               int mode, int active_level, int chunk) {
    PROC_RANK = 0;
    PROC_SIZE = 1;
    splitRadius = split_radius;
    SoftenScale = soften;
    MASSPART = mass;
    NPART = npart;
    part = (Body *)calloc((size_t)(npart > 0 ? npart : 1), sizeof(Body));
    Pack *leaves = (Pack *)calloc((size_t)(nleaf > 0 ? nleaf : 1), sizeof(Pack));
    if (!part || !leaves) return -1;
    for (int i = 0; i < npart; ++i) {
        part[i].tag = 1;
        part[i].act = act ? act[i] : 0;
        for (int d = 0; d < 3; ++d) part[i].pos[d] = pos[(size_t)d * npart + i];
    }
    for (int l = 0; l < nleaf; ++l) {
        leaves[l].ipart = leaf_ipart[l];
        leaves[l].npart = leaf_npart[l];
    }
    leaf = leaves - leaf_base;
    first_leaf = leaf_base;
    last_leaf = leaf_base + nleaf;
    for (int d = 0; d < 3; ++d) {
        acc[d] = (cpuType *)malloc(sizeof(cpuType) * (size_t)(npart > 0 ? npart : 1));
        for (int i = 0; i < npart; ++i) acc[d][i] = acc_out[(size_t)d * npart + i];
    }
    MAXNPACK = npack;
    NPACK = npack;
    packlist = (P2PPack *)calloc((size_t)(npack > 0 ? npack : 1), sizeof(P2PPack));
    long long off = 0;
    for (int k = 0; k < npack; ++k) {
        P2PPack *p = &packlist[k];
        p->ntask = pack_ntask[k];
        p->task_t = (int *)malloc(sizeof(int) * (size_t)(p->ntask > 0 ? p->ntask : 1));
        p->task_s = (int *)malloc(sizeof(int) * (size_t)(p->ntask > 0 ? p->ntask : 1));
        memcpy(p->task_t, task_t + off, sizeof(int) * (size_t)p->ntask);
        memcpy(p->task_s, task_s + off, sizeof(int) * (size_t)p->ntask);
        off += p->ntask;
        p->ileaf = pack_ileaf[k];
        p->nleaf = pack_nleaf[k];
        p->ipart = pack_ipart[k];
        p->npart = pack_npart[k];
        p->rankid = -1;
    }
    if (mode == 0) {
        p2ppack_compute_gpu(packlist, NPACK);
        const double ksec = get_last_kntime(PROC_RANK);
        hostmalloc_out(NPART);
        devMemcpyDH_updateAcc(packlist, NPACK, -1);
        hostfree_out();
        if (kernel_seconds) *kernel_seconds = ksec;
    } else if (mode == 1) {
        p2ppack_compute_act_gpu(packlist, NPACK, active_level);
    } else {
        /* the walk's task buffers: one chunk at a time, rebased in place by the callee */
        long long total = 0;
        for (int k = 0; k < npack; ++k) total += pack_ntask[k];
        int *tt = (int *)malloc(sizeof(int) * (size_t)chunk);
        int *ts = (int *)malloc(sizeof(int) * (size_t)chunk);
        int *own_t = packlist[0].task_t, *own_s = packlist[0].task_s; /* the callee repoints pack 0 */
        NPACK = 0; /* the first chunk counts the pack, as the reference's does */
        long long done = 0;
        do {
            const int m = total - done < chunk ? (int)(total - done) : chunk;
            memcpy(tt, task_t + done, sizeof(int) * (size_t)m);
            memcpy(ts, task_s + done, sizeof(int) * (size_t)m);
            done += m;
            task_compute_p2p_act_gpu(m, tt, ts, done == total, active_level);
        } while (done < total);
        free(tt);
        free(ts);
        packlist[0].task_t = own_t;
        packlist[0].task_s = own_s;
    }
    for (int d = 0; d < 3; ++d) {
        for (int i = 0; i < npart; ++i) acc_out[(size_t)d * npart + i] = acc[d][i];
        free(acc[d]);
        acc[d] = NULL;
    }
    for (int k = 0; k < npack; ++k) {
        free(packlist[k].task_t);
        free(packlist[k].task_s);
    }
    free(packlist);
    packlist = NULL;
    NPACK = 0;
    free(leaves);
    leaf = NULL;
    free(part);
    part = NULL;
    return 0;
}
