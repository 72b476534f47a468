// pg_internal.h -- declarations shared by the kernels (pg_kernels.cu) and the
// host side of the C ABI (pg_api.cu).  Not part of the public interface.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "../../include/primegap.h"

namespace pg {

constexpr uint32_t NOT_FOUND = 0xffffffffu;
constexpr uint32_t TRIAL_PRIMES = 256;  // odd primes tried on positions past sl
// The persistent search kernels run one warp per block, so a warp that
// retires while a launch drains hands its registers back at once (a block's
// resources are released only when all of its warps have exited) and the
// next window's kernels can start on them.
constexpr int PERSIST_THREADS = 32;

// One window of a search launch: the constants of the job it belongs to.  A
// launch may carry windows of several jobs that share an operand layout; side
// s (m index s >> 1) belongs to window wid[s >> 1], or window 0 when wid is
// NULL.
struct WinInfo {
    uint32_t K[PG_MAX_WORDS];          // K = P#/d, zero above kwords
    uint32_t trial_r[TRIAL_PRIMES];    // (-(K mod q)/2) mod q for the trial primes
    uint32_t kwords;
    uint32_t sly;                      // sl / 2; positions Y in [-sly, sly], X = 2Y
    uint32_t rounds;                   // confirmation of every accepted prime: total bases
    uint32_t confirm_rounds;           // record confirmation: total bases (< 2 = off)
    double k_log;                      // log(K), as the merit's denominator uses it
    double confirm_merit;              // m whose merit exceeds this get both primes confirmed
};

// A gap is confirmed when its approximate merit on the device exceeds
// confirm_merit - CONFIRM_MARGIN: the device log() and the host's differ by a
// few ulps at most, so every gap the host then finds above confirm_merit has
// been confirmed.
constexpr double CONFIRM_MARGIN = 1e-6;

// Arguments of the search kernels (one launch over the sides of one or more
// windows; the per-side arrays are indexed by the launch's side index).
struct SearchArgs {
    const WinInfo *win;      // [windows]
    const uint16_t *wid;     // [M] window of each m index, NULL = all window 0
    uint32_t cap;            // list stride per side
    uint32_t n_act;          // active sides in this launch
    uint32_t kspan;          // items per active side in this launch
    uint32_t ext_max;        // extension positions allowed past sly (absolute)
    uint32_t ntrial;         // trial primes for extension positions
    const uint64_t *ms;      // m of each m index
    const uint16_t *lists;   // [2M][cap] |Y| of the survivors, nearest first
    const uint32_t *counts;  // [2M] survivors per side
    const uint32_t *act;     // active side ids
    const uint32_t *k_start; // [2M] first item of each side
    const uint32_t *max_count;  // device scalar: longest list (bounds the queue)
    uint32_t *found_k;       // [2M] item index of the first probable prime
    unsigned long long *next_item;  // work-queue head
    unsigned long long *tests;      // PRP tests executed
    const uint32_t *trial_q;   // [TRIAL_PRIMES] 3, 5, 7, ...
    // draining: a warp with no work in hand retires when more than
    // drain_lanes lanes per unresolved side are active (0 = never retire)
    uint32_t *unresolved;      // sides of this launch without a probable prime yet
    uint32_t *active_warps;    // warps of this launch still pulling work
    uint32_t drain_lanes;
    uint32_t min_warps;        // never retire below this many warps
    // preemption (the server's launches): while *stop is nonzero warps take
    // no new items and leave once their items in hand are tested; a warp that
    // leaves with items still queued sets *stopped, finalize then writes
    // nothing, and a relaunch with the same arguments resumes at the queue head
    const volatile uint32_t *stop;  // NULL = never stop
    uint32_t *stopped;
};

// Device scalars of one window slot.
struct Scalars {
    unsigned long long next_item;
    unsigned long long tests;
    unsigned long long confirm;
    unsigned long long survivors;  // list entries the sieve wrote (both sides of every m)
    uint32_t n_redo;
    uint32_t n_out;
    uint32_t max_count;
    uint32_t unresolved;
    uint32_t active_warps;
    uint32_t stopped;  // the search left items queued (preempted)
};

// Arguments of the sieve kernels for one window.
struct SieveArgs {
    uint32_t sly;
    uint32_t words;          // words per row
    uint32_t cap;
    uint64_t m0;             // first odd m of the window
    uint64_t nodd;           // odd m in the window
    uint32_t nm;             // coprime m in the window
    const uint64_t *ms;      // [nm]
    const int32_t *rank;     // [nodd] index among coprime m, -1 if gcd(m, d) > 1
    uint32_t *bitmaps;       // [nm][words]
    const uint32_t *wheel;   // [words] Y = 0 and q | Y for q | K
    // small primes sieved per m: q, r = (-(K mod q)/2) mod q, floor(2^64/q)
    const uint32_t *sq;
    const uint32_t *sr;
    const uint64_t *sbar;
    uint32_t nsmall;
    uint32_t n32, n256;      // the first n32 small primes are below 32, the first n256 below 256
    uint16_t *lists;
    uint32_t *counts;
    uint32_t *max_count;
    unsigned long long *survivors;
};

struct WalkC;

struct LargeArgs {
    uint32_t sly;
    uint32_t words;
    uint64_t m0;
    uint64_t nodd;
    const int32_t *rank;
    uint32_t *bitmaps;
    uint64_t np;
    const void *p;      // uint32 or uint64 primes
    const void *cinv;   // K^-1 mod p, same type
    const void *c;      // K mod p, same type
    const uint32_t *wheel;  // [words] positions composite in every row (Y = 0, q | Y for q | K)
    const struct WalkC *walk;  // walk steps of the primes [walk_first, walk_end), NULL = none
    uint64_t walk_first, walk_end;
};

// The three-distance walk of one prime below 2^32: the step counts sa (the
// first step whose shift A*sa mod p = alpha lands in [0, W]) and sb (the
// first whose shift lands in [p - W, p), i.e. -beta); alpha = A*sa mod p and
// beta = p - A*sb mod p follow with two modular products.  They depend on p,
// K mod p and the window width W only, so a job computes them once.
struct WalkC {
    uint32_t sa, sb;
};

// Primes of the large-prime table processed by the segmented kernel in one
// launch: [first, first + count), each split into nseg segments of seg_len
// odd m (thread = prime x segment).
struct SegBand {
    uint64_t first, count;
    uint32_t nseg, seg_len;
};
constexpr int MAX_SEG_BANDS = 24;
// expected hits per (prime, segment) item the bands aim at
constexpr uint32_t SEG_HITS = 64;

// --- launchers (pg_kernels.cu); all enqueue on `st` and return cudaError_t
cudaError_t launch_prime_count(uint64_t v_first, uint64_t limit, const uint32_t *base, uint32_t nbase,
                               uint32_t nseg, uint32_t *seg_counts, cudaStream_t st);
cudaError_t launch_prime_write(uint64_t v_first, uint64_t limit, const uint32_t *base, uint32_t nbase,
                               uint32_t nseg, const uint64_t *seg_offsets, void *out, bool wide, cudaStream_t st);
cudaError_t launch_prime_tables(const uint32_t *K, uint32_t kwords, uint64_t np, const void *p, void *c,
                                void *cinv, bool wide, cudaStream_t st);
// orders the primes of every segment by the modular search's Euclid depth
// (into op / oc / oci; depth: np bytes of scratch)
cudaError_t launch_prime_reorder(uint64_t np, uint32_t nseg, const uint64_t *seg_off, const void *p, const void *c,
                                 const void *ci, void *op, void *oc, void *oci, uint8_t *depth, bool wide,
                                 cudaStream_t st);
// Large-prime sieve of one window: primes [0, split) step every Y; the bands
// run the segmented walk (the walk steps of a.walk); primes [search_first,
// np) one thread each (modular search for the first hit, then the walk).
cudaError_t launch_sieve_large(const LargeArgs &a, bool wide, uint64_t split, const SegBand *bands, int nbands,
                               uint64_t search_first, cudaStream_t st);
// walk constants of the primes [first, first + count) (all < 2^32) for width W
cudaError_t launch_walk_consts(const void *p, const void *c, const void *ci, bool wide, uint64_t first,
                               uint64_t count, uint32_t W, WalkC *out, cudaStream_t st);
cudaError_t launch_sieve_small(const SieveArgs &a, bool compact, cudaStream_t st);
cudaError_t launch_prp_batch(uint32_t L, const uint32_t *cand, uint32_t words, uint32_t n, uint32_t rounds,
                             int32_t *out, cudaStream_t st);
cudaError_t launch_search_persistent(uint32_t L, const SearchArgs &a, int grid, cudaStream_t st);
cudaError_t launch_search_plain(uint32_t L, const SearchArgs &a, uint32_t *k_next, cudaStream_t st);
cudaError_t launch_compact_active(const uint32_t *act_in, uint32_t n_in, const uint32_t *found_k,
                                  const uint32_t *k_next, const uint32_t *counts, uint32_t ext_max,
                                  uint32_t *act_out, uint32_t *n_out, cudaStream_t st);
cudaError_t launch_finalize(uint32_t L, const SearchArgs &a, uint32_t nsides, uint32_t *gaps,
                            uint32_t *redo, uint32_t *n_redo, unsigned long long *confirm_tests,
                            uint32_t *k_start_rw, cudaStream_t st);
// Record confirmation over the sides a.act[0 .. a.n_act): sides of gaps whose
// merit exceeds their window's confirm_merit, not yet confirmed at their
// current k (conf[s]), are tested with bases 3, 5, ... up to confirm_rounds
// bases in all; failures are reset and queued in redo for another search.
cudaError_t launch_confirm(uint32_t L, const SearchArgs &a, uint32_t *gaps, uint32_t *conf, uint32_t *redo,
                           uint32_t *n_redo, unsigned long long *confirm_tests, uint32_t *k_start_rw,
                           cudaStream_t st);
cudaError_t launch_iota(uint32_t *out, uint32_t n, cudaStream_t st);
// found_k = NOT_FOUND, k_start = 0, act = 0..S-1, conf = NOT_FOUND for S
// sides; the scalars' queue head and counters = 0, unresolved = S,
// active_warps = warps
cudaError_t launch_init_search(uint32_t S, uint32_t *found_k, uint32_t *k_start, uint32_t *act, uint32_t *conf,
                               Scalars *sc, uint32_t warps, cudaStream_t st);
cudaError_t launch_imad_peak(int grid, uint32_t iters, uint32_t *sink, cudaStream_t st);
// records the calling thread's pg_last_error() text (pg_api.cu)
void set_error(const char *msg);
int search_grid(uint32_t L, int device);
bool supported_limbs(uint32_t L);
uint32_t pick_limbs(uint32_t words);  // layout for operands of `words` words, 0 if none
// layout for operands of `bits` bits: tpi 0 = automatic, 1 = one thread per
// number, T = groups of T lanes; 0 if none is compiled
uint32_t pick_layout(uint32_t bits, uint32_t tpi);
uint32_t layout_words(uint32_t layout);  // total words of a layout

}  // namespace pg
