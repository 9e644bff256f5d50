/*
 * photons_gpu_entry.h - the PhotoNs gpu_entry boundary, served by the B200
 * library. These are the symbols the reference's src/fmm.c and src/gravity.c
 * call for the P2P pass; photons-on-mt3000_b200/csrc/gpu_entry_b200.cpp
 * implements them over photons_p2p.h. They read and write the reference's
 * globals (part, NPART, leaf, first_leaf, last_leaf, MASSPART, SoftenScale,
 * splitRadius, packlist, NPACK, acc, task_t, task_s ...) exactly as the
 * reference's src/gpu_entry.cu and src/gpu_func.impl.h do, so the file is
 * compiled inside a PhotoNs source tree (it includes photoNs.h) with the same
 * -D flags (CPU_DP / INTXYZ / GPU_DP / GPUCUTOFF) and linked with
 * -lphotons_p2p in place of gpu_entry.cu.
 *
 * Errors keep the reference behaviour: a message on stderr and exit
 * (src/gpu_func.impl.h:70-86).
 */
#ifndef PHOTONS_GPU_ENTRY_H
#define PHOTONS_GPU_ENTRY_H

#ifdef __cplusplus
extern "C" {
#endif

/* packs arguments point to the reference's P2PPack array (inc/typedef.h:
 * 109-119); they are typed void* here so this header needs no PhotoNs type.
 * The implementation is compiled against photoNs.h and does not include this
 * header (C linkage makes the two declarations the same symbol). */

/* One chunk of the P2P list of the current pass; the first call of a pass
 * uploads particles and leaves, last_time = 1 marks the final chunk.
 * Replaces task_compute_p2p_gpu, src/gpu_entry.cu:32-209 (declared at
 * inc/gpu_kernel.h:27; called from src/fmm.c:504, :1275, :1348). */
void *task_compute_p2p_gpu(int ntask, int *ltask_t, int *ltask_s, int last_time);

/* Multi-pack pass (INTRA_LB): every pack's list in one pass on one device.
 * Replaces p2ppack_compute_gpu, src/gpu_entry.cu:211-386 (called from
 * src/fmm.c:1250, :1334). The argument is the reference's P2PPack array. */
void *p2ppack_compute_gpu(void *packs, int npack);

/* Active-level passes (hierarchical time steps): only the particles of
 * active_level receive forces (acc[d][j] += result where active_level == -1
 * or (active_level != 0 and part[j].act == active_level); built with
 * ACT_OPT, the chunked form also requires (unsigned char) part[j].act ==
 * (unsigned char) active_level). The call that ends the pass (last_time = 1;
 * every call of the multi-pack form) also waits for it and adds the result,
 * as get_last_kntime + hostmalloc_out + devMemcpyDH_updateAcc + hostfree_out
 * would. Rows whose sink leaf holds no such particle are not computed.
 * Replace task_compute_p2p_act_gpu, src/gpu_active.impl.h:1-153, and
 * p2ppack_compute_act_gpu, :155-321 (compiled into src/gpu_entry.cu:388; the
 * chunked form's one call site, src/fmm.c:1020, is commented out there). */
void *task_compute_p2p_act_gpu(int ntask, int *ltask_t, int *ltask_s, int last_time, int active_level);
void *p2ppack_compute_act_gpu(void *packs, int npack, int active_level);

/* Host task buffers the walk writes into (the globals task_t / task_s of
 * src/global.c:128-129). Replace src/gpu_func.impl.h:184-197. */
void hostmalloc_task(int len_task);
void hostrealloc_task(int len_task);
void hostfree_task(void);

/* Completion barrier of the pass; returns its GPU seconds.
 * Replaces get_last_kntime, src/gpu_func.impl.h:715-730 (src/gravity.c:315, :442). */
double get_last_kntime(int proc_rank);

/* Result staging and acc[d][i] += result for the particles of the packs
 * (active_level -1: all). Replace src/gpu_func.impl.h:264-275, :644-681
 * (src/gravity.c:317-319, :444-446). packs is the reference's P2PPack array.
 * The staging is the module's page-locked buffer, kept between passes (one
 * pinned D2H per pass, no allocation); hostfree_out only releases the
 * reservation, devfree the memory. */
void hostmalloc_out(int npart);
void devMemcpyDH_updateAcc(void *packs, int npack, int active_level);
void hostfree_out(void);

/* Release device buffers / device bookkeeping.
 * Replace devfree src/gpu_func.impl.h:396-400 and dinfofree :229-257
 * (src/photoNs.c:383-384). */
void devfree(void);
void dinfofree(void);

/* Waits for all queued device work. Replaces sync_with_dev,
 * src/gpu_func.impl.h:133-135. */
void sync_with_dev(void);

/* Position bytes the last pass uploaded (no counterpart in the reference).
 * The module keeps the previous pass's packed positions in its page-locked
 * staging and on the device; a pass uploads only the 65536-particle chunks
 * whose positions changed, so a pass over unmoved particles uploads none. */
#include <stdint.h>
int64_t p2p_dropin_last_upload_bytes(void);

#ifdef __cplusplus
}
#endif

#endif /* PHOTONS_GPU_ENTRY_H */
