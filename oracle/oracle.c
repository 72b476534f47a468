/*
 * oracle.c -- CPU restatement of the prime-gap search path (TEST INFRASTRUCTURE).
 *
 * This file is the checker, not the product.  Only tests/, the smoke check in
 * __graft_entry__.py and the cpu_baseline / reference arm of bench.py load it.
 * The CUDA library under prime-gap-gpu_b200/ never links or calls it.
 *
 * What it restates (file:line in sethtroisi/prime-gap-gpu):
 *   K = P#/d, log K ............ gap_common.cpp:44-65 (init_K, _log)
 *   m coprime to d ............. gap_search_gpu.cpp:263-304 (is_coprime_and_valid_m)
 *   sieve, one row per X ....... gap_search_gpu.cpp:586-689 (d-wheel, small and large
 *                                primes), with the two documented bugs fixed: 64-bit
 *                                products everywhere (the reference wraps
 *                                X * neg_inv_K in 32 bits at :659/:679) and the
 *                                halving of the start index in the large branch
 *                                (missing at :683-685).  Both signs of X are sieved.
 *   sieve, one row per m ....... the same residue test transposed (m outer, p inner)
 *   strong PRP ................. miller_rabin.h:216-248 (bases = first `rounds`
 *                                primes, generate_primes miller_rabin.h:272-289;
 *                                result = number of bases passed)
 *   finishing past SL .......... overflow.cpp:145-160 (mpz_nextprime / mpz_prevprime)
 *   ground truth ............... GMP mpz_nextprime / mpz_prevprime from the centre
 *
 * Conventions shared with the CUDA path:
 *   N = m*K + X, X = 2*Y, Y in [-SLY, SLY] with SLY = floor(SL/2).  d must be even,
 *   so K is odd and every m coprime to d is odd; odd X are never prime.
 *   Per m the sieve is a bitmap of 2*SLY+1 bits, bit (Y + SLY) set = composite,
 *   rows of ceil((2*SLY+1)/32) little-endian uint32 words.
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gmp_shim.h"

typedef unsigned __int128 u128;

#define OR_MAX_THREADS 256

/* ------------------------------------------------------------------------- */
/* small helpers                                                             */
/* ------------------------------------------------------------------------- */

static uint64_t gcd_u64(uint64_t a, uint64_t b) {
    while (b) { uint64_t t = a % b; a = b; b = t; }
    return a;
}

/* a^-1 mod p by the extended Euclidean algorithm (gap_search_gpu.cpp:436-458
 * restated with 64-bit signed state so primes above 2^31 work). */
static uint64_t inv_mod(uint64_t a, uint64_t p) {
    int64_t t = 0, nt = 1;
    int64_t r = (int64_t)p, nr = (int64_t)(a % p);
    while (nr != 0) {
        int64_t q = r / nr;
        int64_t tmp = t - q * nt; t = nt; nt = tmp;
        tmp = r - q * nr; r = nr; nr = tmp;
    }
    if (t < 0) t += (int64_t)p;
    return (uint64_t)t;
}

static int is_prime_u64(uint64_t n) {
    if (n < 2) return 0;
    for (uint64_t q = 2; q * q <= n; q++)
        if (n % q == 0) return 0;
    return 1;
}

/* ------------------------------------------------------------------------- */
/* primes: segmented sieve of Eratosthenes (replaces primesieve::iterator,    */
/* gap_search_gpu.cpp:480-500; the small sieve follows gap_common.cpp:256-278) */
/* ------------------------------------------------------------------------- */

static uint32_t *small_primes(uint32_t n, size_t *count) {
    uint8_t *comp = calloc(n + 1, 1);
    size_t cap = 1024, k = 0;
    uint32_t *out = malloc(cap * sizeof(uint32_t));
    for (uint64_t i = 2; i <= n; i++) {
        if (comp[i]) continue;
        if (k == cap) { cap *= 2; out = realloc(out, cap * sizeof(uint32_t)); }
        out[k++] = (uint32_t)i;
        for (uint64_t j = i * i; j <= n; j += i) comp[j] = 1;
    }
    free(comp);
    *count = k;
    return out;
}

typedef struct {
    uint64_t lo, hi;          /* odd primes in [lo, hi] */
    const uint32_t *base; size_t nbase;
    uint64_t *out; size_t n, cap;
} seg_task;

static void *seg_worker(void *arg) {
    seg_task *t = (seg_task *)arg;
    const uint64_t SEG = 1u << 21;   /* odd numbers per segment */
    uint8_t *comp = malloc(SEG);
    t->n = 0; t->cap = 1 << 16;
    t->out = malloc(t->cap * sizeof(uint64_t));
    uint64_t lo = t->lo | 1;
    for (uint64_t s = lo; s <= t->hi; s += 2 * SEG) {
        uint64_t e = s + 2 * SEG - 2;            /* last odd in segment */
        if (e > t->hi) e = t->hi;
        uint64_t cnt = (e - s) / 2 + 1;
        memset(comp, 0, cnt);
        for (size_t i = 1; i < t->nbase; i++) {  /* skip 2 */
            uint64_t q = t->base[i];
            if (q * q > e) break;
            uint64_t st = q * q;
            if (st < s) st = ((s + q - 1) / q) * q;
            if ((st & 1) == 0) st += q;
            for (uint64_t v = st; v <= e; v += 2 * q) comp[(v - s) / 2] = 1;
        }
        for (uint64_t i = 0; i < cnt; i++) {
            if (comp[i]) continue;
            uint64_t v = s + 2 * i;
            if (v < 3) continue;
            if (t->n == t->cap) { t->cap *= 2; t->out = realloc(t->out, t->cap * sizeof(uint64_t)); }
            t->out[t->n++] = v;
        }
    }
    free(comp);
    return NULL;
}

/* All odd primes in [lo, hi], ascending.  Caller frees. */
uint64_t *or_primes(uint64_t lo, uint64_t hi, size_t *count, int threads) {
    if (lo < 3) lo = 3;
    *count = 0;
    if (hi < lo) return malloc(8);
    uint32_t root = (uint32_t)sqrt((double)hi) + 2;
    size_t nbase;
    uint32_t *base = small_primes(root, &nbase);
    if (threads < 1) threads = 1;
    if (threads > OR_MAX_THREADS) threads = OR_MAX_THREADS;
    uint64_t span = hi - lo + 1;
    if (span < (uint64_t)threads * 4096) threads = 1;
    seg_task tasks[OR_MAX_THREADS];
    pthread_t th[OR_MAX_THREADS];
    uint64_t per = (span / threads + 1) & ~(uint64_t)1;
    for (int i = 0; i < threads; i++) {
        tasks[i].lo = lo + per * i;
        tasks[i].hi = (i == threads - 1) ? hi : lo + per * (i + 1) - 1;
        tasks[i].base = base; tasks[i].nbase = nbase;
        pthread_create(&th[i], NULL, seg_worker, &tasks[i]);
    }
    size_t total = 0;
    for (int i = 0; i < threads; i++) { pthread_join(th[i], NULL); total += tasks[i].n; }
    uint64_t *out = malloc((total + 1) * sizeof(uint64_t));
    size_t k = 0;
    for (int i = 0; i < threads; i++) {
        memcpy(out + k, tasks[i].out, tasks[i].n * sizeof(uint64_t));
        k += tasks[i].n;
        free(tasks[i].out);
    }
    free(base);
    *count = total;
    return out;
}

/* ------------------------------------------------------------------------- */
/* job: K, tables                                                            */
/* ------------------------------------------------------------------------- */

typedef struct {
    uint32_t P, d, sl, sly;
    uint64_t limit;
    mpz_t K;
    double K_log;
    /* K-primes: odd q <= P with q not dividing d (q | K). */
    uint32_t *kprimes; size_t nk;
    /* sieve primes: odd d-primes, then every prime in (P, limit]; with
     * c = K mod p and cinv = K^-1 mod p. */
    uint64_t *sp; uint64_t *sc; uint64_t *scinv; size_t ns;
} or_job;

/* K = P#/d (gap_common.cpp:60-65).  Returns 0 on success. */
static int make_K(uint32_t P, uint32_t d, mpz_t K) {
    mpz_init(K);
    mpz_primorial_ui(K, P);
    unsigned long r = mpz_tdiv_q_ui(K, K, d);
    if (r != 0) return -1;
    if (mpz_cmp_ui(K, 1) <= 0) return -2;
    return 0;
}

/* log(K) as in _log (gap_common.cpp:44-48). */
static double log_mpz(mpz_srcptr z) {
    long e;
    double mant = mpz_get_d_2exp(&e, z);
    return log(mant) + log(2.0) * (double)e;
}

typedef struct { or_job *j; size_t lo, hi; } tab_task;

static void *tab_worker(void *arg) {
    tab_task *t = (tab_task *)arg;
    for (size_t i = t->lo; i < t->hi; i++) {
        uint64_t p = t->j->sp[i];
        uint64_t c = mpz_fdiv_ui(t->j->K, p);
        t->j->sc[i] = c;
        t->j->scinv[i] = c ? inv_mod(c, p) : 0;
    }
    return NULL;
}

void or_job_free(or_job *j) {
    if (!j) return;
    mpz_clear(j->K);
    free(j->kprimes); free(j->sp); free(j->sc); free(j->scinv);
    free(j);
}

/* Builds K and the prime tables.  Returns NULL (and *err < 0) on bad input:
 * -1 d does not divide P#, -2 K <= 1, -3 d odd, -4 P not prime,
 * -5 K too small for the sieve limit / search radius. */
or_job *or_job_create(uint32_t P, uint32_t d, uint32_t sl, uint64_t limit, int threads, int *err) {
    *err = 0;
    if (!is_prime_u64(P)) { *err = -4; return NULL; }
    if (d % 2 != 0) { *err = -3; return NULL; }
    or_job *j = calloc(1, sizeof(or_job));
    j->P = P; j->d = d; j->sl = sl; j->sly = sl / 2; j->limit = limit;
    int e = make_K(P, d, j->K);
    if (e) { *err = e; mpz_clear(j->K); free(j); return NULL; }
    j->K_log = log_mpz(j->K);
    /* every candidate must exceed the sieve limit so that "divisible" means composite */
    if (mpz_sizeinbase(j->K, 2) < 70) {
        mpz_t t; mpz_init(t);
        mpz_set_ui(t, limit); mpz_add_ui(t, t, (unsigned long)sl + 2);
        int bad = mpz_cmp(j->K, t) <= 0;
        mpz_clear(t);
        if (bad) { *err = -5; or_job_free(j); return NULL; }
    }
    size_t nsmall;
    uint32_t *sm = small_primes(P, &nsmall);
    j->kprimes = malloc((nsmall + 1) * sizeof(uint32_t));
    size_t ndp = 0;
    uint64_t dps[64];
    for (size_t i = 0; i < nsmall; i++) {
        uint32_t q = sm[i];
        if (q == 2) continue;
        if (d % q == 0) dps[ndp++] = q;
        else j->kprimes[j->nk++] = q;
    }
    free(sm);
    size_t nbig = 0;
    uint64_t *big = or_primes((uint64_t)P + 1, limit, &nbig, threads);
    j->ns = ndp + nbig;
    j->sp = malloc((j->ns + 1) * sizeof(uint64_t));
    j->sc = malloc((j->ns + 1) * sizeof(uint64_t));
    j->scinv = malloc((j->ns + 1) * sizeof(uint64_t));
    for (size_t i = 0; i < ndp; i++) j->sp[i] = dps[i];
    memcpy(j->sp + ndp, big, nbig * sizeof(uint64_t));
    free(big);
    if (threads < 1) threads = 1;
    if (threads > OR_MAX_THREADS) threads = OR_MAX_THREADS;
    tab_task tt[OR_MAX_THREADS];
    pthread_t th[OR_MAX_THREADS];
    size_t per = j->ns / threads + 1;
    for (int i = 0; i < threads; i++) {
        tt[i].j = j;
        tt[i].lo = per * i < j->ns ? per * i : j->ns;
        tt[i].hi = per * (i + 1) < j->ns ? per * (i + 1) : j->ns;
        pthread_create(&th[i], NULL, tab_worker, &tt[i]);
    }
    for (int i = 0; i < threads; i++) pthread_join(th[i], NULL);
    return j;
}

double or_job_K_log(const or_job *j) { return j->K_log; }
size_t or_job_num_sieve_primes(const or_job *j) { return j->ns; }

/* K as little-endian uint32 words; returns the word count (or the needed
 * count if it exceeds max_words, without writing). */
int or_job_K_words(const or_job *j, uint32_t *out, int max_words) {
    size_t bits = mpz_sizeinbase(j->K, 2);
    int nw = (int)((bits + 31) / 32);
    if (nw > max_words) return nw;
    size_t cnt = 0;
    mpz_export(out, &cnt, -1, 4, 0, 0, j->K);
    for (int i = (int)cnt; i < nw; i++) out[i] = 0;
    return nw;
}

/* ------------------------------------------------------------------------- */
/* m coprime to d in [m_start, m_start + m_inc) (gap_search_gpu.cpp:263-304)  */
/* ------------------------------------------------------------------------- */

size_t or_coprime_ms(uint64_t m_start, uint64_t m_inc, uint32_t d, uint64_t *out, size_t cap) {
    size_t k = 0;
    for (uint64_t m = m_start; m < m_start + m_inc; m++) {
        if (gcd_u64(m, d) != 1) continue;
        if (out && k < cap) out[k] = m;
        k++;
    }
    return k;
}

/* ------------------------------------------------------------------------- */
/* sieve, one row per m                                                      */
/* ------------------------------------------------------------------------- */

static inline void set_bit(uint32_t *row, uint64_t idx) { row[idx >> 5] |= 1u << (idx & 31); }

uint32_t or_words_per_m(uint32_t sl) { return ((sl / 2) * 2 + 1 + 31) / 32; }

static void sieve_one_m(const or_job *j, uint64_t m, uint32_t *row) {
    const uint64_t sly = j->sly, nbits = 2 * sly + 1;
    memset(row, 0, or_words_per_m(j->sl) * sizeof(uint32_t));
    set_bit(row, sly);                                   /* X = 0: m*K */
    for (size_t i = 0; i < j->nk; i++) {                 /* q | K: q | Y */
        uint64_t q = j->kprimes[i];
        for (uint64_t idx = sly % q; idx < nbits; idx += q) set_bit(row, idx);
    }
    for (size_t i = 0; i < j->ns; i++) {                 /* q !| K */
        uint64_t p = j->sp[i];
        uint64_t r = (uint64_t)((u128)(m % p) * j->sc[i] % p);      /* m*K mod p */
        uint64_t inv2 = (p + 1) / 2;
        uint64_t y0 = (uint64_t)((u128)((p - r) % p) * inv2 % p);   /* Y = -m*K/2 */
        uint64_t idx = (y0 + sly) % p;
        for (; idx < nbits; idx += p) set_bit(row, idx);
    }
}

typedef struct { const or_job *j; const uint64_t *ms; size_t lo, hi; uint32_t *bitmaps; } sm_task;

static void *sieve_m_worker(void *arg) {
    sm_task *t = (sm_task *)arg;
    uint32_t w = or_words_per_m(t->j->sl);
    for (size_t i = t->lo; i < t->hi; i++) sieve_one_m(t->j, t->ms[i], t->bitmaps + i * w);
    return NULL;
}

static int clamp_threads(int threads, size_t work) {
    if (threads < 1) threads = 1;
    if (threads > OR_MAX_THREADS) threads = OR_MAX_THREADS;
    if ((size_t)threads > work) threads = work ? (int)work : 1;
    return threads;
}

void or_sieve_m(const or_job *j, const uint64_t *ms, size_t nm, uint32_t *bitmaps, int threads) {
    threads = clamp_threads(threads, nm);
    sm_task tt[OR_MAX_THREADS];
    pthread_t th[OR_MAX_THREADS];
    size_t per = nm / threads + 1;
    for (int i = 0; i < threads; i++) {
        tt[i] = (sm_task){j, ms, per * i < nm ? per * i : nm, per * (i + 1) < nm ? per * (i + 1) : nm, bitmaps};
        pthread_create(&th[i], NULL, sieve_m_worker, &tt[i]);
    }
    for (int i = 0; i < threads; i++) pthread_join(th[i], NULL);
}

/* ------------------------------------------------------------------------- */
/* sieve, one row per X across all odd m (the reference's loop structure,     */
/* gap_search_gpu.cpp:586-689, corrected), written into per-m bitmaps        */
/* ------------------------------------------------------------------------- */

typedef struct {
    const or_job *j; uint64_t m0; uint64_t nodd; const int64_t *rank;
    uint32_t w_lo, w_hi;   /* word range of the per-m rows handled */
    uint32_t *bitmaps; uint8_t *rowbuf;
} sx_task;

static void *sieve_x_worker(void *arg) {
    sx_task *t = (sx_task *)arg;
    const or_job *j = t->j;
    const int64_t sly = j->sly;
    const uint32_t W = or_words_per_m(j->sl);
    uint8_t *comp = t->rowbuf;                    /* one byte per odd m of the window */
    for (uint64_t idx = (uint64_t)t->w_lo * 32; idx < (uint64_t)t->w_hi * 32 && idx <= (uint64_t)(2 * sly); idx++) {
        int64_t Y = (int64_t)idx - sly;
        int all = (Y == 0);
        for (size_t i = 0; i < j->nk && !all; i++)
            if (Y % (int64_t)j->kprimes[i] == 0) all = 1;
        if (all) {
            for (uint64_t jj = 0; jj < t->nodd; jj++)
                if (t->rank[jj] >= 0) t->bitmaps[(uint64_t)t->rank[jj] * W + (idx >> 5)] |= 1u << (idx & 31);
            continue;
        }
        memset(comp, 0, t->nodd);
        for (size_t i = 0; i < j->ns; i++) {
            uint64_t p = j->sp[i];
            /* m = m0 + 2*jj with (m*K + 2Y) = 0 mod p  ->  jj = (-2Y*K^-1 - m0) / 2 mod p */
            uint64_t x = (uint64_t)((Y % (int64_t)p + (int64_t)p) % (int64_t)p);
            uint64_t mneg = (uint64_t)((u128)((2 * x) % p) * t->j->scinv[i] % p);   /* 2Y*K^-1 */
            uint64_t m_res = (2 * p - mneg - t->m0 % p) % p;                        /* -2Y/K - m0 */
            uint64_t j0 = (uint64_t)((u128)m_res * ((p + 1) / 2) % p);
            for (uint64_t jj = j0; jj < t->nodd; jj += p) comp[jj] = 1;
        }
        for (uint64_t jj = 0; jj < t->nodd; jj++)
            if (comp[jj] && t->rank[jj] >= 0)
                t->bitmaps[(uint64_t)t->rank[jj] * W + (idx >> 5)] |= 1u << (idx & 31);
    }
    return NULL;
}

/* Sieve the window [m_start, m_start+m_inc) one X row at a time for the row
 * words [w_lo, w_hi) (pass 0, UINT32_MAX for all).  Output rows are for the
 * coprime m in ascending order (as or_coprime_ms), zero-initialised by the
 * caller.  Returns the number of coprime m. */
size_t or_sieve_x(const or_job *j, uint64_t m_start, uint64_t m_inc, uint32_t w_lo, uint32_t w_hi,
                  uint32_t *bitmaps, int threads) {
    const uint32_t W = or_words_per_m(j->sl);
    if (w_hi > W) w_hi = W;
    uint64_t m0 = m_start | 1;
    uint64_t nodd = (m_start + m_inc > m0) ? (m_start + m_inc - m0 + 1) / 2 : 0;
    int64_t *rank = malloc((nodd + 1) * sizeof(int64_t));
    int64_t r = 0;
    for (uint64_t jj = 0; jj < nodd; jj++) rank[jj] = gcd_u64(m0 + 2 * jj, j->d) == 1 ? r++ : -1;
    threads = clamp_threads(threads, w_hi > w_lo ? w_hi - w_lo : 1);
    sx_task tt[OR_MAX_THREADS];
    pthread_t th[OR_MAX_THREADS];
    uint32_t span = w_hi > w_lo ? w_hi - w_lo : 0;
    for (int i = 0; i < threads; i++) {
        tt[i].j = j; tt[i].m0 = m0; tt[i].nodd = nodd; tt[i].rank = rank; tt[i].bitmaps = bitmaps;
        tt[i].w_lo = w_lo + (uint32_t)((uint64_t)span * i / threads);
        tt[i].w_hi = w_lo + (uint32_t)((uint64_t)span * (i + 1) / threads);
        tt[i].rowbuf = malloc(nodd + 1);
        pthread_create(&th[i], NULL, sieve_x_worker, &tt[i]);
    }
    for (int i = 0; i < threads; i++) { pthread_join(th[i], NULL); free(tt[i].rowbuf); }
    free(rank);
    return (size_t)r;
}

/* The same per-X loop for an explicit list of rows (Y values); the rows are
 * split across threads and written with atomic ORs.  Used to time a bounded
 * sample of the reference's CPU sieve. */
typedef struct {
    const or_job *j; uint64_t m0; uint64_t nodd; const int64_t *rank;
    const int64_t *ys; size_t lo, hi; uint32_t *bitmaps;
} sxr_task;

static void *sieve_rows_worker(void *arg) {
    sxr_task *t = (sxr_task *)arg;
    const or_job *j = t->j;
    const int64_t sly = j->sly;
    const uint32_t W = or_words_per_m(j->sl);
    uint8_t *comp = malloc(t->nodd + 1);
    for (size_t r = t->lo; r < t->hi; r++) {
        int64_t Y = t->ys[r];
        uint64_t idx = (uint64_t)(Y + sly);
        memset(comp, 0, t->nodd);
        int all = (Y == 0);
        for (size_t i = 0; i < j->nk && !all; i++)
            if (Y % (int64_t)j->kprimes[i] == 0) all = 1;
        if (all) memset(comp, 1, t->nodd);
        else
            for (size_t i = 0; i < j->ns; i++) {
                uint64_t p = j->sp[i];
                uint64_t x = (uint64_t)((Y % (int64_t)p + (int64_t)p) % (int64_t)p);
                uint64_t mneg = (uint64_t)((u128)((2 * x) % p) * j->scinv[i] % p);
                uint64_t m_res = (2 * p - mneg - t->m0 % p) % p;
                uint64_t j0 = (uint64_t)((u128)m_res * ((p + 1) / 2) % p);
                for (uint64_t jj = j0; jj < t->nodd; jj += p) comp[jj] = 1;
            }
        for (uint64_t jj = 0; jj < t->nodd; jj++)
            if (comp[jj] && t->rank[jj] >= 0)
                __atomic_fetch_or(&t->bitmaps[(uint64_t)t->rank[jj] * W + (idx >> 5)], 1u << (idx & 31),
                                  __ATOMIC_RELAXED);
    }
    free(comp);
    return NULL;
}

size_t or_sieve_x_rows(const or_job *j, uint64_t m_start, uint64_t m_inc, const int64_t *ys, size_t nys,
                       uint32_t *bitmaps, int threads) {
    uint64_t m0 = m_start | 1;
    uint64_t nodd = (m_start + m_inc > m0) ? (m_start + m_inc - m0 + 1) / 2 : 0;
    int64_t *rank = malloc((nodd + 1) * sizeof(int64_t));
    int64_t r = 0;
    for (uint64_t jj = 0; jj < nodd; jj++) rank[jj] = gcd_u64(m0 + 2 * jj, j->d) == 1 ? r++ : -1;
    threads = clamp_threads(threads, nys);
    sxr_task tt[OR_MAX_THREADS];
    pthread_t th[OR_MAX_THREADS];
    for (int i = 0; i < threads; i++) {
        tt[i] = (sxr_task){j, m0, nodd, rank, ys, nys * i / threads, nys * (i + 1) / threads, bitmaps};
        pthread_create(&th[i], NULL, sieve_rows_worker, &tt[i]);
    }
    for (int i = 0; i < threads; i++) pthread_join(th[i], NULL);
    free(rank);
    return (size_t)r;
}

/* ------------------------------------------------------------------------- */
/* strong probable-prime test (miller_rabin.h:216-248)                        */
/* ------------------------------------------------------------------------- */

static const uint32_t MR_BASES[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53};

/* number of bases (2, 3, 5, ... in order) passed before the first failure */
static int prp_mpz(mpz_srcptr n, int rounds) {
    if (mpz_cmp_ui(n, 3) < 0 || !mpz_odd_p(n)) return 0;
    mpz_t n1, dd, x, b;
    mpz_init(n1); mpz_init(dd); mpz_init(x); mpz_init(b);
    mpz_sub_ui(n1, n, 1);
    unsigned long s = mpz_scan1(n1, 0);
    mpz_tdiv_q_2exp(dd, n1, s);
    int k;
    for (k = 0; k < rounds && k < 16; k++) {
        mpz_set_ui(b, MR_BASES[k]);
        if (mpz_cmp(b, n1) >= 0) continue;     /* tiny n: base >= n-1 proves nothing */
        mpz_powm(x, b, dd, n);
        if (mpz_cmp_ui(x, 1) == 0 || mpz_cmp(x, n1) == 0) continue;
        int ok = 0;
        for (unsigned long i = 1; i < s; i++) {
            mpz_powm_ui(x, x, 2, n);
            if (mpz_cmp(x, n1) == 0) { ok = 1; break; }
            if (mpz_cmp_ui(x, 1) == 0) break;
        }
        if (!ok) break;
    }
    mpz_clear(n1); mpz_clear(dd); mpz_clear(x); mpz_clear(b);
    return k;
}

int or_prp(const uint32_t *words, int nwords, int rounds) {
    mpz_t n; mpz_init(n);
    mpz_import(n, (size_t)nwords, -1, 4, 0, 0, words);
    int r = prp_mpz(n, rounds);
    mpz_clear(n);
    return r;
}

typedef struct { const uint32_t *w; int nw; size_t lo, hi; int rounds; int32_t *out; } prp_task;

static void *prp_worker(void *arg) {
    prp_task *t = (prp_task *)arg;
    mpz_t n; mpz_init(n);
    for (size_t i = t->lo; i < t->hi; i++) {
        mpz_import(n, (size_t)t->nw, -1, 4, 0, 0, t->w + i * (size_t)t->nw);
        t->out[i] = prp_mpz(n, t->rounds);
    }
    mpz_clear(n);
    return NULL;
}

/* prp of n numbers of nwords words each, on `threads` threads */
void or_prp_batch(const uint32_t *words, size_t n, int nwords, int rounds, int32_t *out, int threads) {
    threads = clamp_threads(threads, n);
    prp_task tt[OR_MAX_THREADS];
    pthread_t th[OR_MAX_THREADS];
    for (int i = 0; i < threads; i++) {
        tt[i] = (prp_task){words, nwords, n * i / threads, n * (i + 1) / threads, rounds, out};
        pthread_create(&th[i], NULL, prp_worker, &tt[i]);
    }
    for (int i = 0; i < threads; i++) pthread_join(th[i], NULL);
}

int or_probab_prime(const uint32_t *words, int nwords, int reps) {
    mpz_t n; mpz_init(n);
    mpz_import(n, (size_t)nwords, -1, 4, 0, 0, words);
    int r = mpz_probab_prime_p(n, reps);
    mpz_clear(n);
    return r;
}

/* N = m*K + X as little-endian uint32 words; returns the word count. */
int or_candidate_words(const or_job *j, uint64_t m, int64_t X, uint32_t *out, int max_words) {
    mpz_t n, t; mpz_init(n); mpz_init(t);
    mpz_set_ui(t, (unsigned long)m);
    mpz_mul(n, j->K, t);
    if (X >= 0) mpz_add_ui(n, n, (unsigned long)X); else mpz_sub_ui(n, n, (unsigned long)(-X));
    int nw = (int)((mpz_sizeinbase(n, 2) + 31) / 32);
    if (nw <= max_words) {
        size_t cnt = 0;
        mpz_export(out, &cnt, -1, 4, 0, 0, n);
        for (int i = (int)cnt; i < nw; i++) out[i] = 0;
    }
    mpz_clear(n); mpz_clear(t);
    return nw;
}

/* ------------------------------------------------------------------------- */
/* search: sieve + PRP outward from X = 0, finishing past SL with GMP         */
/* ------------------------------------------------------------------------- */

typedef struct {
    const or_job *j; const uint64_t *ms; size_t lo, hi; int rounds;
    uint32_t *prev_gap, *next_gap; uint64_t tests; uint32_t *overflow;
} search_task;

static void *search_worker(void *arg) {
    search_task *t = (search_task *)arg;
    const or_job *j = t->j;
    const uint64_t sly = j->sly;
    uint32_t W = or_words_per_m(j->sl);
    uint32_t *row = malloc(W * sizeof(uint32_t));
    mpz_t center, n, mm;
    mpz_init(center); mpz_init(n); mpz_init(mm);
    t->tests = 0;
    for (size_t i = t->lo; i < t->hi; i++) {
        uint64_t m = t->ms[i];
        sieve_one_m(j, m, row);
        mpz_set_ui(mm, (unsigned long)m);
        mpz_mul(center, j->K, mm);
        for (int side = 0; side < 2; side++) {          /* 0 = next, 1 = prev */
            uint64_t gap = 0;
            for (uint64_t y = 1; y <= sly; y++) {
                uint64_t idx = side == 0 ? sly + y : sly - y;
                if (row[idx >> 5] >> (idx & 31) & 1) continue;
                if (side == 0) mpz_add_ui(n, center, 2 * y); else mpz_sub_ui(n, center, 2 * y);
                t->tests++;
                if (prp_mpz(n, t->rounds) == t->rounds) { gap = 2 * y; break; }
            }
            if (gap == 0) {                              /* past SL: overflow.cpp:145-160 */
                if (t->overflow) t->overflow[i] |= 1u << side;
                if (side == 0) {
                    mpz_add_ui(n, center, 2 * sly);
                    mpz_nextprime(n, n);
                    mpz_sub(n, n, center);
                } else {
                    mpz_sub_ui(n, center, 2 * sly);
                    mpz_prevprime(n, n);
                    mpz_sub(n, center, n);
                }
                gap = mpz_get_ui(n);
            }
            if (side == 0) t->next_gap[i] = (uint32_t)gap; else t->prev_gap[i] = (uint32_t)gap;
        }
    }
    mpz_clear(center); mpz_clear(n); mpz_clear(mm);
    free(row);
    return NULL;
}

/* Returns the number of strong-PRP tests executed (sum over threads). */
uint64_t or_search(const or_job *j, const uint64_t *ms, size_t nm, int rounds,
                   uint32_t *prev_gap, uint32_t *next_gap, uint32_t *overflow, int threads) {
    threads = clamp_threads(threads, nm);
    search_task tt[OR_MAX_THREADS];
    pthread_t th[OR_MAX_THREADS];
    size_t per = nm / threads + 1;
    for (int i = 0; i < threads; i++) {
        tt[i] = (search_task){j, ms, per * i < nm ? per * i : nm, per * (i + 1) < nm ? per * (i + 1) : nm,
                              rounds, prev_gap, next_gap, 0, overflow};
        pthread_create(&th[i], NULL, search_worker, &tt[i]);
    }
    uint64_t tests = 0;
    for (int i = 0; i < threads; i++) { pthread_join(th[i], NULL); tests += tt[i].tests; }
    return tests;
}

/* ------------------------------------------------------------------------- */
/* ground truth straight from GMP                                            */
/* ------------------------------------------------------------------------- */

typedef struct { const or_job *j; const uint64_t *ms; size_t lo, hi; uint32_t *prev_gap, *next_gap; } gt_task;

static void *gmp_gap_worker(void *arg) {
    gt_task *t = (gt_task *)arg;
    mpz_t center, n, mm;
    mpz_init(center); mpz_init(n); mpz_init(mm);
    for (size_t i = t->lo; i < t->hi; i++) {
        mpz_set_ui(mm, (unsigned long)t->ms[i]);
        mpz_mul(center, t->j->K, mm);
        mpz_nextprime(n, center);
        mpz_sub(n, n, center);
        t->next_gap[i] = (uint32_t)mpz_get_ui(n);
        mpz_prevprime(n, center);
        mpz_sub(n, center, n);
        t->prev_gap[i] = (uint32_t)mpz_get_ui(n);
    }
    mpz_clear(center); mpz_clear(n); mpz_clear(mm);
    return NULL;
}

void or_gmp_gaps(const or_job *j, const uint64_t *ms, size_t nm, uint32_t *prev_gap, uint32_t *next_gap, int threads) {
    threads = clamp_threads(threads, nm);
    gt_task tt[OR_MAX_THREADS];
    pthread_t th[OR_MAX_THREADS];
    size_t per = nm / threads + 1;
    for (int i = 0; i < threads; i++) {
        tt[i] = (gt_task){j, ms, per * i < nm ? per * i : nm, per * (i + 1) < nm ? per * (i + 1) : nm, prev_gap, next_gap};
        pthread_create(&th[i], NULL, gmp_gap_worker, &tt[i]);
    }
    for (int i = 0; i < threads; i++) pthread_join(th[i], NULL);
}

/* GMP library version string (gmp_version is an exported variable). */
extern const char *const __gmp_version;
const char *or_gmp_version(void) { return __gmp_version; }
