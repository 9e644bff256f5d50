/*
 * TEST INFRASTRUCTURE ONLY: drives the reference's own tree build and P2P
 * interaction-list walk (src/fmm.c fmm_prepare :962-998 and fmm_task
 * :1221-1300, compiled unchanged from the reference tree by
 * oracle/build_ref.sh) on one periodic domain, the way
 * gravity_fmm_pm_kick (src/gravity.c:326-449) does:
 *   particle_combine bounds  (src/gravity.c:15-140, restated below)
 *   fmm_prepare(0, bdl, bdr)
 *   p2ppack_init              (src/gravity.c:188-194, restated below)
 *   fmm_task()                -> task_compute_p2p_gpu(...) chunks
 *   get_last_kntime, hostmalloc_out, devMemcpyDH_updateAcc, hostfree_out
 *                              (src/gravity.c:440-449)
 * ref_harness_fmm runs the same with the far field of the short-range force
 * (p2m, m2m, the M2L walk and m2l, l2l, l2p of src/operator.c) and returns
 * the reference's multipoles, locals and far-field accelerations.
 * The gpu_entry symbols come from whichever object is linked beside it:
 * oracle/ref_entry_record.c (records the lists) or the B200 drop-in
 * photons-on-mt3000_b200/csrc/gpu_entry_b200.cpp (runs the pass on the GPU).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <mpi.h>
#include "photoNs.h"
#include "operator.h"

/* gpu_entry boundary (inc/gpu_kernel.h:27-42) and fmm.c helpers; declared
 * here because inc/gpu_kernel.h also defines host buffers. */
double get_last_kntime(int proc_rank);
void hostmalloc_out(int npart);
void hostfree_out(void);
void devMemcpyDH_updateAcc(P2PPack *packs, int npack, int active_level);
void fmm_deconstruct(void);

/* PhotoNs' main program provides print_msg (src/fmm.c:485 calls it); the
 * harness stands in for the main program. */
int print_msg(void) { return 0; }

/* Reset by each run; the reference keeps these as process globals. */
static void restate_p2ppack_init(void) {
    NPACK = 0;
    MAXNPACK = 9; /* pow(2, packLevel) + 1 with packLevel = 3, src/setparam.c:53 */
    packlist = (P2PPack *)calloc((size_t)MAXNPACK, sizeof(P2PPack));
}

static void restate_p2ppack_cln(void) {
    free(packlist);
    packlist = NULL;
    NPACK = 0;
}

/* The globals of one run and the particles with their particle_combine
 * bounds (src/gravity.c:15-140); returns 0, or -1 when out of memory. */
static int harness_setup(int npart, const double *pos, const int *tag, int maxleaf, double boxsize,
                         double split_radius, double cutoff_radius, double soften, double mass,
                         double open_angle_in, int len_task, int alloc_acc, cpuType *boxL, cpuType *boxH) {
    PROC_RANK = 0;
    PROC_SIZE = 1;
    BOXSIZE = boxsize;
    MAXLEAF = maxleaf;
    splitRadius = split_radius;
    cutoffRadius = cutoff_radius;
    SoftenScale = soften;
    MASSPART = mass;
    PIisq = 1.0 / sqrt(M_PI); /* src/setparam.c:59 */
    open_angle = open_angle_in;
    LEN_TASK = len_task;
    NPART = npart;

    part = (Body *)malloc(sizeof(Body) * (size_t)npart);
    if (!part) return -1;
    memset(part, 0, sizeof(Body) * (size_t)npart);
    for (int d = 0; d < 3; ++d) {
        boxL[d] = BOXSIZE;
        boxH[d] = 0.0;
    }
    for (int n = 0; n < npart; ++n) {
        part[n].tag = tag[n];
        part[n].act = 0;
        part[n].id = (unsigned long)n;
        for (int d = 0; d < 3; ++d) part[n].pos[d] = pos[(size_t)d * npart + n];
        /* particle_combine takes the bounds on float copies (src/gravity.c:69-121) */
        float fp[3] = {(float)part[n].pos[0], (float)part[n].pos[1], (float)part[n].pos[2]};
        for (int d = 0; d < 3; ++d) {
            if (boxL[d] > fp[d]) boxL[d] = fp[d];
            if (boxH[d] < fp[d]) boxH[d] = fp[d];
        }
    }
    for (int d = 0; d < 3; ++d) {
        boxL[d] -= 0.000001 * BOXSIZE;
        boxH[d] += 0.000001 * BOXSIZE;
    }
    if (alloc_acc) {
        for (int d = 0; d < 3; ++d) {
            acc[d] = (cpuType *)malloc(sizeof(cpuType) * (size_t)npart);
            for (int n = 0; n < npart; ++n) acc[d][n] = 0.0;
        }
    }
    return 0;
}

/* Tree order and the leaf table, rebased to 0; returns the leaf count. */
static int harness_leaves(int npart, int *perm, int *leaf_ipart, int *leaf_npart, double *leaf_center,
                          double *leaf_width, int *leaf_active) {
    int nleaf = last_leaf - first_leaf;
    for (int i = 0; i < npart; ++i) perm[i] = (int)part[i].id;
    for (int l = 0; l < nleaf; ++l) {
        Pack *lf = &leaf[first_leaf + l];
        leaf_ipart[l] = lf->ipart;
        leaf_npart[l] = lf->npart;
        leaf_active[l] = lf->active;
        for (int d = 0; d < 3; ++d) {
            leaf_center[3 * l + d] = lf->center[d];
            leaf_width[3 * l + d] = lf->width[d];
        }
    }
    return nleaf;
}

/*
 * pos: SoA doubles of all npart particles (locals then ghosts, any order),
 * tag: 1 for local particles, 0 for ghost images (src/gravity.c:70-122).
 * Outputs (arrays sized by the caller: perm npart, leaf_* npart + 1 entries,
 * leaf_center/leaf_width 3 * (npart + 1) as AoS):
 *   perm[i]       original index of the particle in tree slot i
 *   leaf_*        leaves first_leaf..last_leaf-1, rebased to 0
 *   acc (nullable) SoA doubles in tree order, filled when collect_acc != 0
 * Returns the number of leaves, or -1.
 */
int ref_harness_run(int npart, const double *pos, const int *tag, int maxleaf,
                    double boxsize, double split_radius, double cutoff_radius,
                    double soften, double mass, double open_angle_in, int len_task,
                    int collect_acc, int *perm, int *leaf_ipart, int *leaf_npart,
                    double *leaf_center, double *leaf_width, int *leaf_active,
                    double *acc_out, double *kernel_seconds) {
    cpuType boxL[3], boxH[3];
    if (harness_setup(npart, pos, tag, maxleaf, boxsize, split_radius, cutoff_radius, soften, mass,
                      open_angle_in, len_task, collect_acc, boxL, boxH))
        return -1;

    fmm_prepare(0, boxL, boxH);
    restate_p2ppack_init();
    fmm_task();

    double ksec = 0.0;
    if (collect_acc) {
        ksec = get_last_kntime(PROC_RANK);
        hostmalloc_out(NPART);
        devMemcpyDH_updateAcc(packlist, NPACK, -1);
        hostfree_out();
    }
    restate_p2ppack_cln();
    if (kernel_seconds) *kernel_seconds = ksec;

    int nleaf = harness_leaves(npart, perm, leaf_ipart, leaf_npart, leaf_center, leaf_width, leaf_active);
    if (collect_acc) {
        for (int d = 0; d < 3; ++d) {
            if (acc_out)
                for (int n = 0; n < npart; ++n) acc_out[(size_t)d * npart + n] = acc[d][n];
            free(acc[d]);
            acc[d] = NULL;
        }
    }
    fmm_deconstruct();
    free(part);
    part = NULL;
    return nleaf;
}

/*
 * The reference's far field of the short-range force on one periodic domain:
 * fmm_prepare (p2m on every leaf and walk_m2m, src/fmm.c:962-998), fmm_task
 * (walk_task_m2l + task_compute_m2l + walk_l2l, src/fmm.c:1221-1300; its P2P
 * lists go to the recording stub), then l2p on every leaf holding a local
 * particle into zeroed accelerations (src/gravity.c:417-428). Outputs as
 * ref_harness_run, plus (all in tree order, leaves rebased to 0):
 *   leaf_M, leaf_L   20 doubles per leaf: multipoles after p2m, locals after
 *                    walk_l2l (the M2L sums plus the parents' shifted locals)
 *   acc_out          SoA far-field accelerations of the l2p
 *   counts           [0] M2L tasks (idxM2L), [1] m2l calls, [2] nodes
 *   times            [0] seconds of task_compute_m2l (the reference's own
 *                    dtime_m2l), [1] seconds of the l2p loop
 * Returns the number of leaves, or -1.
 */
int ref_harness_fmm(int npart, const double *pos, const int *tag, int maxleaf, double boxsize,
                    double split_radius, double cutoff_radius, double soften, double mass, double open_angle_in,
                    int *perm, int *leaf_ipart, int *leaf_npart, double *leaf_center, double *leaf_width,
                    int *leaf_active, double *leaf_M, double *leaf_L, double *acc_out, long long *counts,
                    double *times) {
    cpuType boxL[3], boxH[3];
    if (harness_setup(npart, pos, tag, maxleaf, boxsize, split_radius, cutoff_radius, soften, mass,
                      open_angle_in, 1 << 24, 1, boxL, boxH))
        return -1;
    walk_m2l_count = 0;
    fmm_prepare(0, boxL, boxH);
    int nleaf = last_leaf - first_leaf;
    for (int l = 0; l < nleaf; ++l)
        for (int k = 0; k < NMULTI; ++k) leaf_M[(size_t)NMULTI * l + k] = leaf[first_leaf + l].M[k];
    restate_p2ppack_init();
    fmm_task();
    restate_p2ppack_cln();
    for (int d = 0; d < 3; ++d)
        for (int n = 0; n < npart; ++n) acc[d][n] = 0.0;
    const double t_l2p = dtime();
    for (int n = first_leaf; n < last_leaf; ++n)
        if (leaf[n].active >= 0) l2p(n);
    times[0] = dtime_m2l;  /* the reference's own timer of task_compute_m2l (src/fmm.c:1188-1217) */
    times[1] = dtime() - t_l2p;
    for (int l = 0; l < nleaf; ++l)
        for (int k = 0; k < NMULTI; ++k) leaf_L[(size_t)NMULTI * l + k] = leaf[first_leaf + l].L[k];
    counts[0] = idxM2L;
    counts[1] = walk_m2l_count;
    counts[2] = last_node - first_node + 1;
    harness_leaves(npart, perm, leaf_ipart, leaf_npart, leaf_center, leaf_width, leaf_active);
    for (int d = 0; d < 3; ++d) {
        for (int n = 0; n < npart; ++n) acc_out[(size_t)d * npart + n] = acc[d][n];
        free(acc[d]);
        acc[d] = NULL;
    }
    fmm_deconstruct();
    free(part);
    part = NULL;
    return nleaf;
}
