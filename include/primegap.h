/*
 * primegap.h -- C ABI of the B200 prime-gap search library (libprimegap.so).
 *
 * The library finds, for every m coprime to d in a window, the previous and
 * next prime around the centre m*K, K = P#/d, and the merit of the gap
 * between them.  It replaces the data plane of sethtroisi/prime-gap-gpu:
 *
 *   reference                                       replaced by
 *   ----------------------------------------------  ------------------------------
 *   test_runner_t ctor/dtor (miller_rabin.h:322-362)  pg_ctx_create / pg_ctx_destroy
 *   test_runner_t::run_test (miller_rabin.h:364-408)  pg_prp_batch (host buffers)
 *                                                     pg_prp_batch_device (device)
 *   init_K + sieve prework (gap_common.cpp:60-65,     pg_job_create
 *     gap_search_gpu.cpp:471-501)
 *   per-X sieve pass (gap_search_gpu.cpp:570-755),    pg_sieve_interval
 *     GPUSieve::run (sieve_small.h:40)
 *   GPU batches + CPU overflow finishing              pg_search
 *     (gpu_testing.cu:203-350, overflow.cpp:61-227)
 *
 * Conventions
 *   - Every function returns PG_OK (0) or a negative PG_ERR_* code; nothing
 *     calls exit().  pg_last_error() describes the last failure of the
 *     calling thread.
 *   - Numbers are little-endian arrays of uint32 words (the mpz_export order
 *     -1 of miller_rabin.h:39-54).
 *   - d must be even (gap_search_gpu.cpp:240, :269), so every m searched is
 *     odd and every candidate N = m*K + X has X even.
 *   - A context owns one CUDA stream on one device.  Use one context per host
 *     thread; calls on the same context are serialised by the caller.
 */
#ifndef PRIMEGAP_H
#define PRIMEGAP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PG_OK 0
#define PG_ERR_ARG (-1)         /* invalid argument */
#define PG_ERR_CUDA (-2)        /* CUDA runtime error */
#define PG_ERR_UNSUPPORTED (-3) /* size outside the compiled kernels */
#define PG_ERR_NOMEM (-4)       /* device or host allocation failed */
#define PG_ERR_TIMEOUT (-5)     /* a bounded device wait gave up */
#define PG_ERR_STATE (-6)       /* call made in the wrong state */

/* largest operand, in 32-bit words, the PRP kernels accept */
#define PG_MAX_WORDS 160

typedef struct pg_ctx pg_ctx;
typedef struct pg_job pg_job;

/* ---------------------------------------------------------------- context */

/* Creates a context on CUDA device `device` with its own stream.
 * Replaces the resources test_runner_t allocates (miller_rabin.h:322-349). */
int pg_ctx_create(int device, pg_ctx **out);
int pg_ctx_destroy(pg_ctx *ctx);

/* The context's cudaStream_t (as void *): every kernel of the context's
 * calls is enqueued on it, so callers can time them with CUDA events. */
void *pg_ctx_stream(pg_ctx *ctx);

/* Text of the last error on this thread ("" if none). */
const char *pg_last_error(void);

/* Measured throughput of independent 32-bit integer multiply-adds on the
 * context's device (instructions per second, whole GPU), from a register-only
 * microbenchmark kernel.  No counterpart in the reference: it is the
 * denominator of the PRP kernel's roofline.  Synchronous. */
int pg_measure_imad_peak(pg_ctx *ctx, double *imad_per_second);

/* Version string of the library. */
const char *pg_version(void);

/* ------------------------------------------------------------------- PRP */

/* Strong probable-prime test of n numbers, each `words` LE uint32 words, in
 * host memory; bases are the first `rounds` primes (2, 3, 5, ...).
 * passed[i] = number of bases passed before the first failure, exactly the
 * `passed` field of the reference (miller_rabin.h:216-270); the number is a
 * probable prime iff passed[i] == rounds.  Even numbers and numbers < 3
 * give 0.  Synchronous, like test_runner_t::run_test (miller_rabin.h:364). */
int pg_prp_batch(pg_ctx *ctx, const uint32_t *limbs, uint32_t n, uint32_t words,
                 uint32_t rounds, int32_t *passed);

/* Same on device buffers, enqueued on `stream` (a cudaStream_t, or NULL for
 * the context's stream); returns without waiting. */
int pg_prp_batch_device(pg_ctx *ctx, const uint32_t *d_limbs, uint32_t n, uint32_t words,
                        uint32_t rounds, int32_t *d_passed, void *stream);

/* ------------------------------------------------------------------- jobs */

typedef struct {
    uint32_t p;            /* P of P# (-p), prime */
    uint32_t d;            /* divisor (-d), even, divides P# */
    uint32_t sl;           /* search radius: candidates X in [-sl, sl] are sieved */
    uint64_t max_prime;    /* sieve limit: every prime <= max_prime (--max-prime * 1e6) */
    uint64_t max_m_inc;    /* largest window later passed to pg_search / pg_sieve_interval */
    uint64_t max_m;        /* largest m that will be searched (sizes the limbs) */
    uint32_t rounds;       /* strong-PRP bases per accepted prime: 1 = base 2 only
                              (the reference's ROUNDS, gpu_testing.cu:62); r > 1 confirms
                              every base-2 probable prime with bases 3, 5, ... */
    uint32_t small_limit;  /* primes <= small_limit are sieved per m in shared memory;
                              0 = default (65536) */
    uint32_t ext_window;   /* extension positions past sl tried in the first pass; 0 = 64 */
    uint32_t flags;        /* PG_JOB_* */
    uint32_t search_hits;  /* 0 = every large prime above 2*sl+1 is sieved by modular search
                              (default); n > 0 keeps primes expecting >= n hits per window on
                              the kernel that steps every X */
    uint32_t tpi;          /* threads per number of the PRP kernels: 0 = automatic (one
                              thread up to 48 words, then groups), 1, or a group size 4 / 8 / 16 */
    double confirm_merit;  /* record confirmation (the double-check of overflow.cpp:164-177):
                              for every m whose gap has merit > confirm_merit, both primes
                              must pass confirm_rounds strong bases (2, 3, 5, ...) before the
                              search returns; a side whose prime fails one is searched on
                              from its next candidate, so the gap stays exact.  The bulk
                              search still runs `rounds` bases.  0 = no record confirmation */
    uint32_t confirm_rounds; /* bases of the record confirmation, 2..16; 0 = 16 */
    uint32_t pad;
} pg_job_params;

/* large-prime sieve: 0 = automatic, else force one method */
#define PG_JOB_LARGE_STEP   0x1u   /* step every X for every prime */
#define PG_JOB_LARGE_SEARCH 0x2u   /* modular search for the next hit */
#define PG_JOB_NO_GRAPH     0x4u   /* launch the persistent form's kernels one by one
                                      instead of as one CUDA graph per window; pg_job_create
                                      then returns without waiting for the device (the job's
                                      launches wait for its set-up on their own streams) */
#define PG_JOB_COMPACT_WALK 0x8u   /* keep the large-prime sieve's walk steps (8 B per prime below
                                      2^32, computed at job creation: 0.8 GB at 2e9) only for the
                                      primes expecting >= 64 hits per window; the others find each
                                      hit after the first by another modular search.  For short-lived
                                      jobs (the server sets it for its jobs) */

typedef struct {
    uint32_t k_bits;          /* bits of K */
    uint32_t limbs;           /* 32-bit words of the PRP operands */
    uint32_t tpi;             /* threads per number of the PRP kernels */
    uint32_t words_per_m;     /* uint32 words of one sieve row */
    uint32_t side_capacity;   /* longest possible survivor list of one side */
    uint64_t num_primes;      /* primes in (P, max_prime] */
    uint64_t num_small;       /* of them (plus odd d-primes) sieved per m */
    double k_log;             /* log(K), as _log (gap_common.cpp:44-48) */
    double setup_seconds;     /* wall time of pg_job_create (small when the tables were shared) */
    uint64_t device_bytes;    /* device memory the job uses: its slots and wheel, and the prime
                                 tables it shares with the context's jobs of the same
                                 (p, d, max_prime, small_limit) */
} pg_job_info;

int pg_job_create(pg_ctx *ctx, const pg_job_params *params, pg_job **out);
int pg_job_destroy(pg_job *job);
int pg_job_get_info(const pg_job *job, pg_job_info *info);
/* K as LE words; *nwords receives the count (call with out = NULL to size). */
int pg_job_k_words(const pg_job *job, uint32_t *out, uint32_t *nwords);

/* Number of m coprime to d in [m_start, m_start + m_inc). */
uint64_t pg_count_m(uint64_t m_start, uint64_t m_inc, uint32_t d);

/* Sieve of the window: for each m coprime to d in [m_start, m_start+m_inc)
 * (ascending, written to ms) one row of words_per_m uint32, bit (Y + sl/2)
 * set when m*K + 2Y has a prime factor <= max_prime.  Host buffers of
 * pg_count_m(...) entries / rows.  This is sieve_interval_cpu's contract
 * with both signs of X (the reference sieves X > 0 only). */
int pg_sieve_interval(pg_job *job, uint64_t m_start, uint64_t m_inc, uint64_t *ms, uint32_t *bitmaps);

/* Search forms */
#define PG_SEARCH_PERSISTENT 0  /* one persistent kernel per window, device work queue */
#define PG_SEARCH_PLAIN 1       /* one PRP launch per pass, host loop (the reference's shape) */

typedef struct {
    uint64_t m_count;         /* m searched */
    uint64_t prp_tests;       /* strong base-2 tests executed */
    uint64_t confirm_tests;   /* extra-base tests executed */
    uint64_t extended_sides;  /* sides whose prime lay past sl */
    uint32_t passes;          /* PRP launches (plain: one per pass) */
    uint32_t relaunches;      /* continuation / re-search launches */
    double sieve_ms;          /* device time of the sieve kernels */
    double prp_ms;            /* device time of the PRP kernels, finalize and continuation */
    double total_ms;          /* device time of the whole call, inputs already on the device */
    double search_kernel_ms;  /* device time of the first PRP search launch(es) alone */
    uint64_t kernel_launches; /* kernels of this library launched by the call */
    uint64_t h2d_bytes;       /* host-to-device bytes copied by the call */
    uint64_t d2h_bytes;       /* device-to-host bytes copied by the call */
    uint32_t graph_launches;  /* CUDA graph launches (the persistent form's window is one graph) */
    uint32_t pad;
    uint64_t survivors;       /* candidates the sieve left in [-sl, sl], both sides of every m */
} pg_search_stats;

/* Searches the window: for each m coprime to d (ascending; ms may be NULL)
 * writes prev_gap[i] = m*K - prevprime(m*K) and next_gap[i] =
 * nextprime(m*K) - m*K.  Host arrays of pg_count_m(...) entries.  Primes
 * past sl are found on the device (no CPU fallback). */
int pg_search(pg_job *job, uint64_t m_start, uint64_t m_inc, int form,
              uint64_t *ms, uint32_t *prev_gap, uint32_t *next_gap, pg_search_stats *stats);

/* ------------------------------------------------------ allocation-free */

/* Largest batch of pg_next_prime_noalloc. */
#define PG_NOALLOC_MAX_N 65536

/* Next probable prime without allocating device memory.  No counterpart in
 * the reference.  It is for callers that cannot call cudaMalloc: code whose
 * device memory is owned by another allocator (a framework's caching pool, a
 * budget fixed at start-up) and code that must not stall a running pipeline
 * on an allocation, which can synchronise the device.
 *
 * For each of the n numbers at d_numbers (n rows of `words` LE uint32, device
 * memory) writes to d_steps[i] the smallest k < max_steps such that
 * d_numbers[i] + 2k passes the strong base-2 test, or 0xFFFFFFFF if none
 * does (even numbers and numbers below 3 give 0xFFFFFFFF).  Every candidate
 * d_numbers[i] + 2k is tested at full width for words < 48; for words = 48 a
 * candidate that no longer fits in 48 words (d_numbers[i] within 2*max_steps
 * of 2^1536) is skipped, never reported.  Enqueued on
 * `stream` (a cudaStream_t; NULL = the legacy default stream) of the current
 * device; returns without waiting.
 *
 * Its only working memory is a file-scope device array of
 * PG_NOALLOC_MAX_N + 64 uint32 (257 KB), which every GPU that loads the
 * library holds until the process exits.  The first call on each device
 * looks up that array's device address (cudaGetSymbolAddress) with the
 * device current: make the first call on a device before any stream capture.
 * The address is kept for the life of the process: after cudaDeviceReset (or
 * any teardown of the device's primary context) the module may load elsewhere,
 * so do not call this function on that device again in the same process.
 * n above PG_NOALLOC_MAX_N is rejected (PG_ERR_ARG), words above 48
 * (PG_ERR_UNSUPPORTED).  Every call shares the array and clears it before
 * use, so calls that can overlap on the GPU (other streams, other host
 * threads) race and must be serialised by the caller. */
int pg_next_prime_noalloc(const uint32_t *d_numbers, uint32_t n, uint32_t words, uint32_t max_steps,
                          uint32_t *d_steps, void *stream);

/* Pipelined search: a job has PG_SEARCH_SLOTS window slots (own stream and
 * buffers each), so PG_SEARCH_SLOTS windows can be in flight and overlap on
 * the device -- the reference keeps GPU_BATCHES batches in flight
 * (gpu_testing.cu:57) for the same reason.  pg_search_submit enqueues the
 * search of one window and returns a ticket (tickets count up from 0; ticket
 * t uses slot t % PG_SEARCH_SLOTS, which must not hold an un-waited ticket,
 * else PG_ERR_STATE).  pg_search_wait(ticket) blocks until that window is
 * done and fills the outputs like pg_search.  flags: PG_SUBMIT_DRAIN lets
 * the PRP kernel's warps leave once fewer than D lanes per unresolved side
 * would remain busy, handing their SMs to the next window (for callers that
 * keep another window submitted; a lone window finishes later with it);
 * D = (flags >> 8) & 0xff, 0 = 4.  PG_SUBMIT_WARPS_PER_SM(w) caps the PRP
 * kernel at w resident warps per SM (0 = as many as fit), leaving room for
 * the next window's kernels to run beside it.  pg_search() is submit + wait. */
#define PG_SEARCH_SLOTS 2
#define PG_SUBMIT_DRAIN 0x1u
#define PG_SUBMIT_DRAIN_LANES(d) (((uint32_t)(d) & 0xffu) << 8)
#define PG_SUBMIT_WARPS_PER_SM(w) (((uint32_t)(w) & 0xffu) << 16)
int pg_search_submit(pg_job *job, uint64_t m_start, uint64_t m_inc, int form, uint32_t flags, uint64_t *ticket);
int pg_search_wait(pg_job *job, uint64_t ticket, uint64_t *ms, uint32_t *prev_gap, uint32_t *next_gap,
                   pg_search_stats *stats);
/* cudaStream_t of window slot `slot` (for CUDA-event timing by callers). */
void *pg_job_stream(pg_job *job, int slot);

/* Autotuner (no counterpart in the reference, which fixes these at compile
 * time, gpu_testing.cu:44-62).  Starting from *base, times searches of the
 * sample window [m_start, m_start + m_inc) and writes to *best the fastest
 * small_limit (the prime bound of the per-m shared-memory sieve tile, tried
 * 16384 / 65536 / 262144) and then threads per number (tpi 1, 4, 8 where a
 * compiled layout fits the operand width; the limb count follows), and to
 * *best_ms its device time per window.  Builds one job per candidate. */
int pg_autotune(pg_ctx *ctx, const pg_job_params *base, uint64_t m_start, uint64_t m_inc, pg_job_params *best,
                double *best_ms);

/* The wider autotuner: the knobs the reference fixes at compile time
 * (THREADS_PER_INSTANCE, WINDOW_BITS, GPU_BATCH_SIZE, GPU_BATCHES,
 * gpu_testing.cu:50-62) and their counterparts here, timed on the sample
 * window [m_start, m_start + m_inc) with PG_SEARCH_SLOTS windows in flight
 * (the pipelined form callers run), one knob after the other:
 *   1. threads per number: tpi 0 (automatic), 1, 4, 8, 16 where a compiled
 *      layout fits;
 *   2. the small-prime bound of the shared-memory sieve tile: 16384, 65536,
 *      262144;
 *   3. the PRP kernel's warps per SM (PG_SUBMIT_WARPS_PER_SM): 0 (all that
 *      fit), 4, 6, 8, 10, 12, each over max(2 x reps, 8) passes (a short
 *      sample favours full occupancy), then the two fastest once more, and
 *      the mean of their two timings decides;
 *   4. with PG_TUNE_WINDOW, the m per window: m_inc, m_inc / 2, m_inc / 4.
 * The exponentiation window has no knob: the base-2 test multiplies by
 * doublings, never by a table entry.  Each setting runs one warm-up pass and
 * then `reps` passes (0 = 4) over the sample; m/s is their m over the wall
 * time.  out->params is *base with the chosen small_limit and tpi. */
#define PG_TUNE_WINDOW 0x1u
typedef struct {
    pg_job_params params;   /* the chosen job parameters */
    uint32_t warps_per_sm;  /* the chosen PG_SUBMIT_WARPS_PER_SM cap (0 = as many as fit) */
    uint32_t settings;      /* settings timed */
    uint64_t window_m;      /* the chosen m per window */
    double m_per_sec;       /* the chosen setting's m/s, PG_SEARCH_SLOTS windows in flight (from
                               the longer re-timing of the caps, unless a window size won after it) */
    double first_m_per_sec; /* m/s of the first setting timed (tpi 0 with base's knobs, no cap) */
} pg_tune_result;
int pg_autotune_ex(pg_ctx *ctx, const pg_job_params *base, uint64_t m_start, uint64_t m_inc, uint32_t flags,
                   uint32_t reps, pg_tune_result *out);

/* ---------------------------------------------------------------- serving
 *
 * A server takes gap-search requests (any P, d, sl, sieve limit and m range)
 * from any host thread and runs them on one device with continuous batching:
 * a worker thread cuts each request's m range into windows, and packs windows
 * of every admitted request whose operands share a layout into one search
 * launch (one persistent PRP kernel over all their sides), two launches in
 * flight.  Prime tables depend on (P, d, max_prime, small_limit) only and are
 * shared by every request with that key, whatever its sl or m range.  A
 * request is admitted once its tables are resident; tables that would not fit
 * the device-memory budget wait until idle tables can be evicted (least
 * recently used first).  The reference runs one (P, d, sl, range) per process
 * (gap_search_gpu.cpp:106-135) and has no counterpart. */
typedef struct pg_server pg_server;

typedef struct {
    uint64_t hbm_budget;   /* device bytes for tables and batch buffers; 0 = 3/4 of the free memory */
    uint32_t batch_m;      /* coprime m per search launch (all its windows); 0 = 65536 */
    uint32_t window_m;     /* requests are cut into windows of at most this many m; 0 = 65536 */
    uint32_t max_windows;  /* windows per search launch; 0 = 64 */
    uint32_t max_sl;       /* largest sl accepted; 0 = 20000 */
    uint32_t small_limit;  /* as pg_job_params (0 = default) */
    uint32_t ext_window;   /* as pg_job_params (0 = default) */
    uint32_t tpi;          /* as pg_job_params (0 = automatic) */
    uint32_t warps_per_sm; /* cap on each launch's PRP warps per SM (PG_SUBMIT_WARPS_PER_SM), so the
                              launches in flight share the SMs; 0 = as many as fit */
    uint32_t slots;        /* launch slots (own stream and buffers each); 0 = 2 (4 with preemption:
                              two run, the others hold stopped launches), at most 8 */
    uint32_t preempt_us;   /* preemption of running launches: 0 = off.  Otherwise launches are
                              scheduled by operand width, narrowest first, and at most
                              min(slots - 1, 2) run;
                              once narrower windows have waited preempt_us microseconds, every
                              running launch of wider operands is told to stop (its warps leave after
                              the tests in hand), its slot holds the search's state, the narrower
                              windows run, and the stopped search resumes from its queue head when
                              no narrower work runs or waits.  A request waiting max(2 s,
                              100 x preempt_us) goes first whatever its width.  Results do not
                              change; a short request need not wait for a long launch to end */
} pg_server_params;

typedef struct {
    uint32_t p, d, sl;     /* as pg_job_params */
    uint32_t rounds;       /* as pg_job_params (0 = 1) */
    uint64_t max_prime;    /* sieve limit */
    uint64_t m_start;      /* the m range [m_start, m_start + m_inc) */
    uint64_t m_inc;
} pg_request;

typedef struct {
    uint64_t m_count;      /* m searched: pg_count_m(m_start, m_inc, d) */
    double k_log;          /* log(K) of the request's K = P#/d */
    double submit_s;       /* server clock (seconds since pg_server_create): submitted */
    double start_s;        /* first window launched */
    double done_s;         /* last window finished */
    uint32_t windows;      /* windows the range was cut into */
    int32_t status;        /* PG_OK, or the error that failed the request */
} pg_request_info;

typedef struct {
    uint64_t requests_done;  /* completed (or failed) requests */
    uint64_t m_done;         /* m searched */
    uint64_t prp_tests;      /* strong base-2 tests */
    uint64_t launches;       /* search launches (batches) */
    uint64_t windows;        /* windows run */
    uint64_t tables_built;   /* prime-table builds */
    uint64_t tables_evicted; /* prime tables dropped to admit others */
    uint64_t resident_bytes; /* device bytes held now */
    uint64_t peak_bytes;     /* most device bytes held */
    double sieve_ms;         /* device time of the sieves, summed over launches */
    double prp_ms;           /* device time of the searches, summed over launches */
    double busy_s;           /* wall time with at least one launch in flight */
    uint64_t preemptions;    /* launches stopped to let waiting windows run (resumed later) */
} pg_server_stats;

/* Starts a server (and its worker thread) on CUDA device `device`. */
int pg_server_create(int device, const pg_server_params *params, pg_server **out);
/* Queues a request and returns at once with its id.  Argument errors are
 * returned here; errors found later (d does not divide P#, tables larger than
 * the budget, CUDA errors) fail the request and come back from wait. */
int pg_server_submit(pg_server *srv, const pg_request *rq, uint64_t *id);
/* Waits up to timeout_s seconds (< 0 = for ever) for request id, then copies
 * its results (arrays of info->m_count = pg_count_m(...) entries, ascending
 * m; any may be NULL) and forgets the request.  PG_ERR_TIMEOUT if it is not
 * done yet (it stays queued); the request's own error if it failed;
 * PG_ERR_ARG for an unknown id or one another waiter has already returned. */
int pg_server_wait(pg_server *srv, uint64_t id, double timeout_s, uint64_t *ms, uint32_t *prev_gap,
                   uint32_t *next_gap, pg_request_info *info);
/* Id of a finished request not yet returned by this call, oldest first;
 * PG_ERR_TIMEOUT when none finishes within timeout_s. */
int pg_server_next_done(pg_server *srv, double timeout_s, uint64_t *id);
int pg_server_get_stats(pg_server *srv, pg_server_stats *stats);
/* Seconds since pg_server_create on the server clock. */
double pg_server_clock(const pg_server *srv);
/* Finishes the launches in flight, fails the requests not yet run
 * (PG_ERR_STATE), stops the worker and frees the device memory. */
int pg_server_destroy(pg_server *srv);

/* Merit of a gap as overflow.cpp:162: gap / (k_log + log(m)). */
double pg_merit(double k_log, uint64_t m, uint64_t gap);

/* Record line of overflow.cpp:180-182: "{gap} {merit:.3f} {m} * {P}# / {D} - {prev}".
 * Returns the length written (excluding NUL), or a negative error. */
int pg_format_record(char *buf, size_t buflen, uint64_t gap, double merit, uint64_t m,
                     uint32_t p, uint32_t d, uint64_t prev_gap);

#ifdef __cplusplus
}
#endif

#endif /* PRIMEGAP_H */
