/*
 * TEST INFRASTRUCTURE ONLY: a recording stand-in for the reference's
 * gpu_entry boundary (the symbols src/fmm.c and src/gravity.c call,
 * inc/gpu_kernel.h:27-42). It keeps every (sink, source) leaf pair the walk
 * hands to task_compute_p2p_gpu, rebased by first_leaf the way
 * devMemcpyHD_task does (src/gpu_func.impl.h:704-713), plus the chunk
 * boundaries of the successive calls (src/fmm.c:500-515, :1275).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <mpi.h>
#include "photoNs.h"

static int *rec_t, *rec_s;
static long long rec_n, rec_cap;
static long long *rec_chunk_end;
static int rec_nchunk, rec_chunk_cap;

static void rec_push_chunk(long long end) {
    if (rec_nchunk == rec_chunk_cap) {
        rec_chunk_cap = rec_chunk_cap ? 2 * rec_chunk_cap : 64;
        rec_chunk_end = (long long *)realloc(rec_chunk_end, sizeof(long long) * (size_t)rec_chunk_cap);
    }
    rec_chunk_end[rec_nchunk++] = end;
}

void *task_compute_p2p_gpu(int ntask, int *ltask_t, int *ltask_s, int last_time) {
    if (rec_n + ntask > rec_cap) {
        long long cap = rec_cap ? rec_cap : 1 << 16;
        while (cap < rec_n + ntask) cap *= 2;
        rec_t = (int *)realloc(rec_t, sizeof(int) * (size_t)cap);
        rec_s = (int *)realloc(rec_s, sizeof(int) * (size_t)cap);
        rec_cap = cap;
    }
    for (int i = 0; i < ntask; ++i) {
        rec_t[rec_n + i] = ltask_t[i] - first_leaf;
        rec_s[rec_n + i] = ltask_s[i] - first_leaf;
    }
    rec_n += ntask;
    if (ntask > 0 || last_time) rec_push_chunk(rec_n);
    return NULL;
}

void hostmalloc_task(int len) {
    task_s = (int *)malloc(sizeof(int) * (size_t)len);
    task_t = (int *)malloc(sizeof(int) * (size_t)len);
}
void hostrealloc_task(int len) {
    task_s = (int *)realloc(task_s, sizeof(int) * (size_t)len);
    task_t = (int *)realloc(task_t, sizeof(int) * (size_t)len);
}
void hostfree_task(void) {
    free(task_s);
    free(task_t);
    task_s = task_t = NULL;
}
double get_last_kntime(int proc_rank) { (void)proc_rank; return 0.0; }
void hostmalloc_out(int n) { (void)n; }
void hostfree_out(void) {}
void devMemcpyDH_updateAcc(P2PPack *packs, int npack, int active_level) {
    (void)packs; (void)npack; (void)active_level;
}

void ref_record_reset(void) {
    rec_n = 0;
    rec_nchunk = 0;
}
long long ref_record_count(void) { return rec_n; }
int ref_record_nchunk(void) { return rec_nchunk; }
void ref_record_copy(int *t, int *s, long long *chunk_end) {
    memcpy(t, rec_t, sizeof(int) * (size_t)rec_n);
    memcpy(s, rec_s, sizeof(int) * (size_t)rec_n);
    memcpy(chunk_end, rec_chunk_end, sizeof(long long) * (size_t)rec_nchunk);
}
