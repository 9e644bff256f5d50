/*
 * TEST INFRASTRUCTURE ONLY: a host stand-in for the pass protocol of
 * libphotons_p2p (the calls photons-on-mt3000_b200/csrc/gpu_entry_b200.cpp
 * makes), linked by oracle/build_ref.sh into libref_dropin_host{,act}.so so
 * the CPU tests can drive the drop-in's host logic (pack protocol, list
 * rebasing, active-level row selection, result update over the packs'
 * particles) with no GPU. It computes no gravity: every submitted entry
 * (t, s) adds, to each particle j of sink leaf t,
 *   acc[0][j] += npart of leaf s,  acc[1][j] += s + 1,  acc[2][j] += 1,
 * so the result tells which rows were submitted, and it counts the entries.
 * Never part of the product library.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "photons_p2p.h"

struct p2p_session {
    int npart, nleaf, in_pass;
    double *acc;
    int *ip, *np;
};

static char g_err[256];
static long long g_entries;  /* entries submitted since the last stub_reset */
static long long g_passes;   /* passes begun since the last stub_reset */

static int fail(int status, const char *msg) {
    snprintf(g_err, sizeof g_err, "%s", msg);
    return status;
}

long long stub_submitted_entries(void) { return g_entries; }
long long stub_passes(void) { return g_passes; }
void stub_reset(void) { g_entries = 0; g_passes = 0; }

const char *p2p_status_string(int status) { return status == P2P_OK ? "ok" : "error"; }
const char *p2p_last_error(void) { return g_err; }
int p2p_device_count(int *count) {
    *count = 1;
    return P2P_OK;
}

void p2p_params_default(p2p_params *p) { memset(p, 0, sizeof *p); }

int p2p_session_create(int device, p2p_session **out) {
    (void)device;
    *out = (p2p_session *)calloc(1, sizeof(p2p_session));
    return *out ? P2P_OK : fail(P2P_ERR_NOMEM, "calloc");
}

int p2p_session_destroy(p2p_session *s) {
    if (!s) return P2P_OK;
    free(s->acc);
    free(s->ip);
    free(s->np);
    free(s);
    return P2P_OK;
}

int p2p_session_set_params(p2p_session *s, const p2p_params *params) {
    return s && params ? P2P_OK : fail(P2P_ERR_ARG, "null argument");
}

int p2p_session_synchronize(p2p_session *s) { return s ? P2P_OK : fail(P2P_ERR_ARG, "null session"); }

int p2p_host_alloc(size_t bytes, void **ptr) {
    *ptr = malloc(bytes ? bytes : 1);
    return *ptr ? P2P_OK : fail(P2P_ERR_NOMEM, "malloc");
}

int p2p_host_free(void *ptr) {
    free(ptr);
    return P2P_OK;
}

int p2p_pass_begin_update(p2p_session *s, int npart, const double *pos, int nleaf, const int *leaf_ipart,
                          const int *leaf_npart, const unsigned char *dirty, int64_t chunk,
                          int64_t *uploaded_bytes) {
    if (!s || (npart > 0 && !pos) || (nleaf > 0 && (!leaf_ipart || !leaf_npart)) || chunk <= 0)
        return fail(P2P_ERR_ARG, "bad begin");
    if (s->in_pass) return fail(P2P_ERR_STATE, "pass already open");
    free(s->acc);
    free(s->ip);
    free(s->np);
    s->acc = (double *)calloc(3 * (size_t)(npart > 0 ? npart : 1), sizeof(double));
    s->ip = (int *)malloc(sizeof(int) * (size_t)(nleaf > 0 ? nleaf : 1));
    s->np = (int *)malloc(sizeof(int) * (size_t)(nleaf > 0 ? nleaf : 1));
    if (!s->acc || !s->ip || !s->np) return fail(P2P_ERR_NOMEM, "alloc");
    memcpy(s->ip, leaf_ipart, sizeof(int) * (size_t)nleaf);
    memcpy(s->np, leaf_npart, sizeof(int) * (size_t)nleaf);
    for (int l = 0; l < nleaf; ++l)
        if (s->ip[l] < 0 || s->np[l] < 0 || s->ip[l] + s->np[l] > npart) return fail(P2P_ERR_RANGE, "leaf range");
    int64_t bytes = 0;
    for (int64_t c = 0; c * chunk < npart; ++c) {
        const int64_t a = c * chunk, b = a + chunk < npart ? a + chunk : npart;
        if (!dirty || dirty[c]) bytes += 24 * (b - a);
    }
    if (uploaded_bytes) *uploaded_bytes = bytes;
    s->npart = npart;
    s->nleaf = nleaf;
    s->in_pass = 1;
    ++g_passes;
    return P2P_OK;
}

int p2p_pass_submit(p2p_session *s, int64_t ntask, const int *task_t, const int *task_s) {
    if (!s) return fail(P2P_ERR_ARG, "null session");
    if (!s->in_pass) return fail(P2P_ERR_STATE, "no open pass");
    if (ntask < 0 || (ntask > 0 && (!task_t || !task_s))) return fail(P2P_ERR_ARG, "bad list");
    for (int64_t e = 0; e < ntask; ++e) {
        const int t = task_t[e], src = task_s[e];
        if (t < 0 || t >= s->nleaf || src < 0 || src >= s->nleaf) return fail(P2P_ERR_RANGE, "leaf id");
        for (int j = s->ip[t]; j < s->ip[t] + s->np[t]; ++j) {
            s->acc[j] += s->np[src];
            s->acc[(size_t)s->npart + j] += src + 1;
            s->acc[2 * (size_t)s->npart + j] += 1;
        }
    }
    g_entries += ntask;
    return P2P_OK;
}

int p2p_pass_end(p2p_session *s, double *gpu_seconds) {
    if (!s) return fail(P2P_ERR_ARG, "null session");
    if (!s->in_pass) return fail(P2P_ERR_STATE, "no open pass");
    s->in_pass = 0;
    if (gpu_seconds) *gpu_seconds = 1e-6;
    return P2P_OK;
}

int p2p_pass_result(p2p_session *s, double *out) {
    if (!s) return fail(P2P_ERR_ARG, "null session");
    if (s->in_pass) return fail(P2P_ERR_STATE, "pass still open");
    memcpy(out, s->acc, sizeof(double) * 3 * (size_t)s->npart);
    return P2P_OK;
}
