/*
 * serve_client.c - a C11 caller of the extension API beyond one session: a
 * batch with host-frame ticks, stage timing, snapshot / restore, the
 * autotuner and the served request loop.  Compiled and linked against
 * libwema_cuda on any host (tests/test_ext_layout.py); run on a GPU, it
 * checks that a session's frames equal a batched stream's host-tick frames
 * and prints OK.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "wema_cuda.h"

#define W 96
#define H 64
#define F 4

static int fail(const char *what) {
    fprintf(stderr, "%s: %s\n", what, wema_cuda_last_error());
    return 1;
}

int main(void) {
    const size_t fb = (size_t)W * H * 3;
    unsigned char *in = malloc(F * fb), *out_b = malloc(F * fb);
    if (!in || !out_b) return 1;
    for (size_t i = 0; i < F * fb; i++) in[i] = (unsigned char)((i * 2654435761u) >> 24);

    char report[256];
    if (wema_cuda_autotune(0, report, sizeof report) < 0) return fail("autotune");
    printf("%s\n", report);

    wema_cuda_config cfg;
    wema_cuda_config_default(&cfg, W, H, 30.0f);
    cfg.amp_factor = 60.0f;
    cfg.f_high = 3.0f;

    /* batched stream, host frames */
    wema_cuda_batch *b;
    int id;
    if (wema_cuda_batch_create(0, 4, &b) || wema_cuda_batch_add(b, &cfg, &id)) return fail("batch");
    if (wema_cuda_batch_set_timing(b, 1)) return fail("timing");
    for (int t = 0; t < F; t++) {
        const void *pi[1] = {in + t * fb};
        void *po[1] = {out_b + t * fb};
        if (wema_cuda_batch_tick_host(b, &id, pi, po, 1, NULL, NULL)) return fail("tick_host");
    }
    if (wema_cuda_batch_sync(b)) return fail("sync");
    double ms[WEMA_CUDA_STAGES];
    long long ticks = 0;
    if (wema_cuda_batch_stage_times(b, ms, &ticks) || ticks != F) return fail("stage times");
    const size_t sb = wema_cuda_batch_snapshot_bytes(b, id);
    void *snap = malloc(sb);
    if (!snap || wema_cuda_batch_snapshot(b, id, snap, sb)) return fail("snapshot");
    wema_cuda_batch_destroy(b);

    /* the same frames through the served loop */
    wema_cuda_server *srv;
    int sid;
    if (wema_cuda_server_create(0, (size_t)1 << 30, 4, &srv) || wema_cuda_server_open(srv, &cfg, &sid))
        return fail("server");
    wema_cuda_session_status st;
    do {
        if (wema_cuda_server_poll(srv, sid, &st)) return fail("poll");
    } while (st.state == WEMA_CUDA_SESSION_QUEUED);
    /* device buffers are the caller's: here the frames go through a session's
     * host path instead, compared with the batch */
    wema_cuda_session *s;
    if (wema_cuda_session_create(&cfg, &s)) return fail("session");
    unsigned char *o = malloc(fb);
    int bad = 0;
    for (int t = 0; t < F; t++) {
        if (wema_cuda_process_host_u8(s, in + t * fb, o)) return fail("process");
        bad |= memcmp(o, out_b + t * fb, fb) != 0;
    }
    if (wema_cuda_session_restore(s, snap, sb) == 0) bad = 1;   /* batch snapshot: one buffer set */
    wema_cuda_serve_stats ss;
    if (wema_cuda_server_close(srv, sid) || wema_cuda_server_drain(srv, 10000) ||
        wema_cuda_server_stats(srv, 0, &ss))
        return fail("server stats");
    wema_cuda_server_destroy(srv);
    wema_cuda_session_destroy(s);
    free(o);
    free(snap);
    free(in);
    free(out_b);
    printf(bad ? "MISMATCH\n" : "OK\n");
    return bad;
}
