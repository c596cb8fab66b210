/*
 * refdrv.c -- multi-threaded driver for timing the REFERENCE CPU verify.
 *
 * TEST / BASELINE INFRASTRUCTURE ONLY (loaded by the cpu_baseline and
 * --impl reference legs of bench.py).  It dlopen()s the reference library
 * compiled by oracle/Makefile (oracle/_ref/libufsecp_ref.so) and calls its C ABI
 * exactly as a reference user would: one ufsecp_ctx per thread
 * (include/ufsecp/ufsecp.h: contexts are single-thread), each thread verifying
 * a static slice with ufsecp_ecdsa_verify(ctx, msg32, sig64, pubkey33)
 * (src/cpu/src/impl/ufsecp_ecdsa.cpp:244) or ufsecp_schnorr_verify(ctx, msg32,
 * sig64, pubkey_x32) (:992).  Verdict = return code == UFSECP_OK.
 */
#include <dlfcn.h>
#include <limits.h>
#include <unistd.h>
#include <pthread.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>

typedef int (*ctx_create_fn)(void **);
typedef void (*ctx_destroy_fn)(void *);
typedef int (*verify_fn)(void *, const uint8_t *, const uint8_t *, const uint8_t *);

static void *g_lib;
static ctx_create_fn g_create;
static ctx_destroy_fn g_destroy;
static verify_fn g_ecdsa, g_schnorr;

/* Returns 0 on success. */
int refdrv_open(const char *path, const char *cache_dir) {
    if (g_lib) return 0;
    g_lib = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!g_lib) { fprintf(stderr, "refdrv: %s\n", dlerror()); return 1; }
    g_create = (ctx_create_fn)dlsym(g_lib, "ufsecp_ctx_create");
    g_destroy = (ctx_destroy_fn)dlsym(g_lib, "ufsecp_ctx_destroy");
    g_ecdsa = (verify_fn)dlsym(g_lib, "ufsecp_ecdsa_verify");
    g_schnorr = (verify_fn)dlsym(g_lib, "ufsecp_schnorr_verify");
    /* the library's generator cache goes where the caller says (ufsecp_set_cache_dir,
     * include/ufsecp/ufsecp.h:136), not into the working directory */
    int (*set_dir)(const char *) = (int (*)(const char *))dlsym(g_lib, "ufsecp_set_cache_dir");
    if (set_dir && cache_dir) set_dir(cache_dir);
    /* The first generator multiplication builds the library's fixed-base tables
     * and saves them to the working directory when the cache dir has no copy yet
     * (src/cpu/src/precompute.cpp:2235-2256), so do that once from the cache dir. */
    typedef int (*pk_fn)(void *, const uint8_t *, uint8_t *);
    pk_fn pk = (pk_fn)dlsym(g_lib, "ufsecp_pubkey_create");
    char cwd[PATH_MAX];
    if (pk && cache_dir && g_create && getcwd(cwd, sizeof cwd) && chdir(cache_dir) == 0) {
        void *ctx = NULL;
        uint8_t sk[32] = {0}, pub[33];
        sk[31] = 1;
        if (g_create(&ctx) == 0) {
            pk(ctx, sk, pub);
            g_destroy(ctx);
        }
        if (chdir(cwd) != 0) return 4;
    }
    return (g_create && g_destroy && g_ecdsa && g_schnorr) ? 0 : 2;
}

typedef struct {
    int kind;
    const uint8_t *msgs, *pubs, *sigs;
    uint8_t *out;
    size_t lo, hi;
    int rc;
} job_t;

static void *worker(void *arg) {
    job_t *j = (job_t *)arg;
    void *ctx = NULL;
    if (g_create(&ctx) != 0) { j->rc = 1; return NULL; }
    const size_t ps = j->kind == 0 ? 33 : 32;
    verify_fn fn = j->kind == 0 ? g_ecdsa : g_schnorr;
    for (size_t i = j->lo; i < j->hi; ++i)
        j->out[i] = fn(ctx, j->msgs + 32 * i, j->sigs + 64 * i, j->pubs + ps * i) == 0;
    g_destroy(ctx);
    j->rc = 0;
    return NULL;
}

/* kind 0 = ECDSA (33-byte keys), 1 = BIP-340 (32-byte x-only keys). */
int refdrv_verify(int kind, const uint8_t *msgs, const uint8_t *pubs, const uint8_t *sigs, size_t n,
                  uint8_t *out, int threads) {
    if (!g_lib) return 3;
    if (threads < 1) threads = 1;
    if (threads > 512) threads = 512;
    if ((size_t)threads > n) threads = n ? (int)n : 1;
    pthread_t th[512];
    job_t jobs[512];
    for (int t = 0; t < threads; ++t) {
        jobs[t] = (job_t){kind, msgs, pubs, sigs, out, n * t / threads, n * (t + 1) / threads, 0};
        if (t) pthread_create(&th[t], NULL, worker, &jobs[t]);
    }
    worker(&jobs[0]);
    int rc = jobs[0].rc;
    for (int t = 1; t < threads; ++t) {
        pthread_join(th[t], NULL);
        rc |= jobs[t].rc;
    }
    return rc;
}

/* Corpus generation with the reference's own signers (for the reference arm):
 * kind 0: ufsecp_pubkey_create + ufsecp_ecdsa_sign; kind 1: ufsecp_pubkey_xonly +
 * ufsecp_schnorr_sign(msg, sk, aux).  ok[i] = 1 when both calls returned UFSECP_OK. */
typedef int (*pub_fn)(void *, const uint8_t *, uint8_t *);
typedef int (*esign_fn)(void *, const uint8_t *, const uint8_t *, uint8_t *);
typedef int (*ssign_fn)(void *, const uint8_t *, const uint8_t *, const uint8_t *, uint8_t *);

typedef struct {
    int kind;
    const uint8_t *msgs, *sks, *auxs;
    uint8_t *pubs, *sigs, *ok;
    size_t lo, hi;
} sjob_t;

static void *sign_worker(void *arg) {
    sjob_t *j = (sjob_t *)arg;
    void *ctx = NULL;
    if (g_create(&ctx) != 0) return NULL;
    pub_fn pc = (pub_fn)dlsym(g_lib, j->kind == 0 ? "ufsecp_pubkey_create" : "ufsecp_pubkey_xonly");
    esign_fn es = (esign_fn)dlsym(g_lib, "ufsecp_ecdsa_sign");
    ssign_fn ss = (ssign_fn)dlsym(g_lib, "ufsecp_schnorr_sign");
    const size_t ps = j->kind == 0 ? 33 : 32;
    for (size_t i = j->lo; i < j->hi; ++i) {
        int a = pc(ctx, j->sks + 32 * i, j->pubs + ps * i);
        int b = j->kind == 0 ? es(ctx, j->msgs + 32 * i, j->sks + 32 * i, j->sigs + 64 * i)
                             : ss(ctx, j->msgs + 32 * i, j->sks + 32 * i, j->auxs + 32 * i, j->sigs + 64 * i);
        j->ok[i] = (a == 0 && b == 0);
    }
    g_destroy(ctx);
    return NULL;
}

int refdrv_sign(int kind, const uint8_t *msgs, const uint8_t *sks, const uint8_t *auxs, size_t n,
                uint8_t *pubs, uint8_t *sigs, uint8_t *ok, int threads) {
    if (!g_lib) return 3;
    if (threads < 1) threads = 1;
    if (threads > 512) threads = 512;
    if ((size_t)threads > n) threads = n ? (int)n : 1;
    pthread_t th[512];
    sjob_t jobs[512];
    for (int t = 0; t < threads; ++t) {
        jobs[t] = (sjob_t){kind, msgs, sks, auxs, pubs, sigs, ok, n * t / threads, n * (t + 1) / threads};
        if (t) pthread_create(&th[t], NULL, sign_worker, &jobs[t]);
    }
    sign_worker(&jobs[0]);
    for (int t = 1; t < threads; ++t) pthread_join(th[t], NULL);
    return 0;
}
