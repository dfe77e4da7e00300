/*
 * w2w_oracle.c -- CPU oracle for the Gaussian rasterizer hot path.
 *
 * TEST INFRASTRUCTURE ONLY (tests/, __graft_entry__.smoke(), bench.py's CPU
 * baseline).  The product never links or calls this library.
 *
 * Restates the reference extension cudaForwardBackwardRenderer:
 *   projection.cu, ADRculling.cu, gaussianForwardPass.cu (SH colour),
 *   gaussianRasterizer.cu:77-117 (inclusive scan), prepareSort.cu (key
 *   emission and the stable 64-bit radix sort), gaussianTiles.cu (tile
 *   ranges), pixelGaussiansFull.cu / pixelGaussiansDev.cuh / gaussEval.h
 *   (blend), backward.cu / gradientPass.cu (backward).
 * The per-element arithmetic lives in raster_core.h, instantiated for float
 * (bit-level restatement) and double (fp64 re-evaluation).
 *
 * Build: gcc -O2 -ffp-contract=off -fno-fast-math -pthread -fPIC -shared (see Makefile).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

typedef struct {
    int W, H;          /* image size */
    int degree, M;     /* SH degree used, coefficients stored per Gaussian */
    int compat_spill;  /* 1: reference key-emission rectangle (see orc_emit) */
    float focal_x;
    float view[16];    /* viewmatrix as passed (device reads it column-major) */
    float proj[16];    /* projmatrix as passed */
    float campos[3];
    float bg[3];
} orc_cfg;

/* fusion-pattern selectors, one per expression instance (see raster_core.h) */
enum {
    V_RQ = 0,                 /* 9: rotation entries, column-major          */
    V_SIGMA = V_RQ + 9,       /* 6: stored Sigma entries                    */
    V_VIEW_A = V_SIGMA + 6,   /* 4: view rows, (m0 x + m1 y)                */
    V_VIEW_B = V_VIEW_A + 4,  /* 4: view rows, (m2 z + m3)                  */
    V_RAYR2 = V_VIEW_B + 4,   /* 1 */
    V_DPROJ = V_RAYR2 + 1,    /* 6: jx[0..2], jy[0..2]                      */
    V_SIGV = V_DPROJ + 6,     /* 6: Sigma*jx rows, Sigma*jy rows            */
    V_DOT3 = V_SIGV + 6,      /* 3: cxx, cxy, cyy                           */
    V_DET = V_DOT3 + 3,       /* 1 */
    V_PROJ_A = V_DET + 1,     /* 4 */
    V_PROJ_B = V_PROJ_A + 4,  /* 4 */
    V_PIX = V_PROJ_B + 4,     /* 2 */
    V_ADR_DELTA = V_PIX + 2,  /* 1 */
    V_BL_DET, V_BL_TX, V_BL_TY, V_BL_NUM, V_BL_DEPTH, V_SH_DOT, V_SH_ACC,
    V_SH2A, V_SH2B, V_SH3A, V_SH3B, V_SH3C, V_SH3D, V_SH3E,
    V_COUNT
};
static int orc_var[V_COUNT];

/* Threads of the per-pixel and per-Gaussian loops (1 = serial, the default:
 * the tests' results are then independent of the machine).  Only the timed
 * CPU baseline raises it. */
static int orc_threads = 1;
void orc_set_threads(int n) { orc_threads = n > 1 ? (n < 1024 ? n : 1024) : 1; }
int orc_get_threads(void) { return orc_threads; }

/* Parallel loop over [0, n): workers take `chunk` indices at a time from a
 * shared counter and call fn(ctx, lo, hi, worker).  Worker 0 is the calling
 * thread; if a thread cannot be started its share is taken by the others. */
typedef void (*orc_part_fn)(void* ctx, long long lo, long long hi, int tid);
typedef struct {
    orc_part_fn fn;
    void* ctx;
    long long n, chunk, next;
} orc_job;
typedef struct {
    orc_job* job;
    int tid;
} orc_worker_arg;

static void* orc_worker(void* p) {
    orc_worker_arg* w = (orc_worker_arg*)p;
    orc_job* j = w->job;
    for (;;) {
        const long long lo = __atomic_fetch_add(&j->next, j->chunk, __ATOMIC_RELAXED);
        if (lo >= j->n) break;
        const long long hi = lo + j->chunk < j->n ? lo + j->chunk : j->n;
        j->fn(j->ctx, lo, hi, w->tid);
    }
    return NULL;
}

static void orc_parallel_for(long long n, long long chunk, orc_part_fn fn, void* ctx) {
    const int nt = orc_threads;
    if (nt <= 1 || n <= chunk) {
        if (n > 0) fn(ctx, 0, n, 0);
        return;
    }
    orc_job job = {fn, ctx, n, chunk, 0};
    pthread_t th[1024];
    orc_worker_arg arg[1024];
    int started[1024];
    for (int t = 0; t < nt; ++t) { arg[t].job = &job; arg[t].tid = t; started[t] = 0; }
    for (int t = 1; t < nt; ++t) started[t] = pthread_create(&th[t], NULL, orc_worker, &arg[t]) == 0;
    orc_worker(&arg[0]);
    for (int t = 1; t < nt; ++t)
        if (started[t]) pthread_join(th[t], NULL);
}

void orc_set_variant(int k, int v) { if (k >= 0 && k < V_COUNT) orc_var[k] = v; }
int orc_get_variant(int k) { return (k >= 0 && k < V_COUNT) ? orc_var[k] : -1; }
int orc_variant_count(void) { return V_COUNT; }

#define RABS(x) ((x) < 0 ? -(x) : (x))

/* ---- fp32 restatement ---- */
#define REAL float
#define SFX(n) n##_f32
#define RFMA fmaf
#define REXP expf
#define RLOG logf
#define RSQRT sqrtf
#define RCEIL ceilf
#define RFLOOR floorf
#include "raster_core.h"
#undef REAL
#undef SFX
#undef RFMA
#undef REXP
#undef RLOG
#undef RSQRT
#undef RCEIL
#undef RFLOOR

/* ---- fp64 re-evaluation ---- */
#define REAL double
#define SFX(n) n##_f64
#define RFMA fma
#define REXP exp
#define RLOG log
#define RSQRT sqrt
#define RCEIL ceil
#define RFLOOR floor
#include "raster_core.h"

/* ---- integer stages (precision independent) ---- */

/* inclusive scan of tiles-touched (gaussianRasterizer.cu:77-117) */
void orc_inclusive_scan_u32(const uint32_t* in, uint32_t* out, long long n) {
    uint32_t acc = 0;
    for (long long i = 0; i < n; ++i) { acc += in[i]; out[i] = acc; }
}

/* Stable sort of (key, value) pairs by the 64-bit key: LSD radix, 8-bit
 * digits, digit passes on which every key agrees are skipped.  Same result
 * as the reference's 32-pass 2-bit LSD sort (prepareSort.cu:303-360): both
 * are stable, so ties keep their input order. */
void orc_sort_pairs_u64(uint64_t* keys, uint32_t* vals, long long n) {
    if (n <= 1) return;
    uint64_t* k2 = (uint64_t*)malloc((size_t)n * 8);
    uint32_t* v2 = (uint32_t*)malloc((size_t)n * 4);
    uint64_t* ka = keys; uint32_t* va = vals; uint64_t* kb = k2; uint32_t* vb = v2;
    for (int shift = 0; shift < 64; shift += 8) {
        long long cnt[257];
        memset(cnt, 0, sizeof(cnt));
        for (long long i = 0; i < n; ++i) cnt[((ka[i] >> shift) & 255) + 1]++;
        int uniform = 0;
        for (int d = 1; d <= 256; ++d) if (cnt[d] == n) uniform = 1;
        if (uniform) continue;
        for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
        for (long long i = 0; i < n; ++i) {
            long long p = cnt[(ka[i] >> shift) & 255]++;
            kb[p] = ka[i]; vb[p] = va[i];
        }
        uint64_t* tk = ka; ka = kb; kb = tk;
        uint32_t* tv = va; va = vb; vb = tv;
    }
    if (ka != keys) { memcpy(keys, ka, (size_t)n * 8); memcpy(vals, va, (size_t)n * 4); }
    free(k2); free(v2);
}

/* per-tile [start, end) from sorted keys (gaussianTiles.cu:6-33); ranges of
 * tiles without entries stay (0, 0) */
void orc_tile_ranges(const uint64_t* keys, long long n, uint32_t* ranges, int num_tiles) {
    memset(ranges, 0, (size_t)num_tiles * 2 * sizeof(uint32_t));
    for (long long i = 0; i < n; ++i) {
        uint32_t t = (uint32_t)(keys[i] >> 32);
        if ((int)t >= num_tiles) continue;
        if (i == 0 || (uint32_t)(keys[i - 1] >> 32) != t) ranges[2 * t] = (uint32_t)i;
        if (i == n - 1 || (uint32_t)(keys[i + 1] >> 32) != t) ranges[2 * t + 1] = (uint32_t)(i + 1);
    }
}
