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
    cpuType boxL[3] = {BOXSIZE, BOXSIZE, BOXSIZE}, boxH[3] = {0.0, 0.0, 0.0};
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
    if (collect_acc) {
        for (int d = 0; d < 3; ++d) {
            acc[d] = (cpuType *)malloc(sizeof(cpuType) * (size_t)npart);
            for (int n = 0; n < npart; ++n) acc[d][n] = 0.0;
        }
    }

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
