// pg_host.h -- host objects shared by the job API (pg_api.cu) and the
// serving loop (pg_server.cu).  Not part of the public interface.
//
//   pg_ctx  -- device, default stream, PRP staging, and a cache of the prime
//              tables of the jobs alive on it
//   Tables  -- everything that depends only on K = P#/d, the sieve limit and
//              the small-prime bound: small-prime residues, trial residues
//              and the large-prime table (p, K mod p, K^-1 mod p).  Shared by
//              every job with the same key, whatever its sl.
//   pg_job  -- one (Tables, sl, rounds, operand layout): the wheel row, the
//              per-window constants (WinInfo) and two window slots
//   Slot    -- buffers, stream and in-flight state of one search launch over
//              one or more windows (of one or several jobs) that share an
//              operand layout
#pragma once

#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "pg_internal.h"

namespace pg {

constexpr int SLOT_FULL = 1;
constexpr int SLOT_STOPPED = 2;  // slot_finish: the search was preempted; slot_resume continues it
constexpr int SLOT_PENDING = 3;  // slot_finish(wait = false): another round is queued; call again when idle

// records the calling thread's error text and returns code
int fail(int code, const char *fmt, ...);

#define PG_CUDA(call)                                                                                        \
    do {                                                                                                     \
        cudaError_t e_ = (call);                                                                             \
        if (e_ != cudaSuccess)                                                                               \
            return ::pg::fail(e_ == cudaErrorMemoryAllocation ? PG_ERR_NOMEM : PG_ERR_CUDA, "%s: %s (%s:%d)", \
                              #call, cudaGetErrorString(e_), __FILE__, __LINE__);                            \
    } while (0)

cudaError_t record_ev(cudaEvent_t e, cudaStream_t st);
uint64_t gcd64(uint64_t a, uint64_t b);

typedef std::vector<uint32_t> Big;  // little-endian words, no leading zeros

struct Tables {
    int device = 0;
    uint32_t p = 0, d = 0, q1 = 0;  // small primes are <= q1
    uint64_t max_prime = 0;
    Big K;
    uint32_t kbits = 0;
    double k_log = 0;
    std::vector<uint32_t> kprimes;  // odd primes dividing K
    uint32_t *d_sq = nullptr, *d_sr = nullptr;
    uint64_t *d_sbar = nullptr;
    uint32_t nsmall = 0;
    uint32_t n32 = 0, n256 = 0;  // small primes (ascending) below 32 and below 256
    uint32_t *d_tq = nullptr;   // trial primes 3, 5, 7, ...
    std::vector<uint32_t> tr;   // their residues (-(K mod q)/2) mod q
    void *d_lp = nullptr, *d_lc = nullptr, *d_lcinv = nullptr;
    uint64_t np = 0;
    bool wide = false;
    // prime-table index of each sieve segment (segment s starts at value seg_v0 + s * seg_span)
    std::vector<uint64_t> seg_off;
    uint64_t seg_v0 = 0, seg_span = 0;
    uint64_t bytes = 0;
    double setup_s = 0;
    ~Tables();
};

// The tables of (p, d, max_prime, small_limit) on ctx: a live copy shared with
// other jobs, else a new build.
int tables_get(pg_ctx *c, const pg_job_params &p, std::shared_ptr<Tables> &out);
// Device bytes a build of those tables would take (an upper estimate).
uint64_t tables_bytes_estimate(const pg_job_params &p);

// One window of a slot.
struct WinPart {
    pg_job *job = nullptr;
    uint64_t m0 = 0, nodd = 0;  // first odd m, odd m in the window
    uint32_t nm = 0;            // coprime m
    uint32_t m_off = 0;         // first m index of the window in the slot
    uint64_t odd_off = 0;       // first odd-m rank entry of the window in the slot
};

struct Slot {
    // capacities
    uint64_t nm_cap = 0, nodd_cap = 0, bm_cap = 0, list_cap = 0;  // m, odd m, bitmap words, list entries
    uint32_t win_cap = 0;
    // device
    cudaStream_t st = nullptr;
    uint64_t *d_ms = nullptr;
    uint16_t *d_wid = nullptr;
    int32_t *d_rank = nullptr;
    uint32_t *d_bitmaps = nullptr;
    uint16_t *d_lists = nullptr;
    uint32_t *d_counts = nullptr, *d_found = nullptr, *d_kstart = nullptr, *d_knext = nullptr, *d_gaps = nullptr;
    uint32_t *d_act0 = nullptr, *d_act1 = nullptr, *d_redo = nullptr;
    uint32_t *d_conf = nullptr;  // per side: the k whose prime passed the record confirmation
    Scalars *d_sc = nullptr;
    WinInfo *d_win = nullptr;
    // pinned host staging
    Scalars *h_sc = nullptr;
    uint64_t *h_ms = nullptr;
    uint16_t *h_wid = nullptr;
    int32_t *h_rank = nullptr;
    uint32_t *h_gaps = nullptr;
    WinInfo *h_win = nullptr;
    cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    cudaGraphExec_t gexec = nullptr;  // the persistent form's window graph
    uint64_t bytes = 0;
    // contents and in-flight state
    std::vector<WinPart> parts;
    uint32_t nm = 0;       // m in the slot
    uint64_t nodd = 0;     // odd m in the slot
    uint32_t L = 0;        // operand layout of every window
    uint32_t stride = 0;   // list stride (largest job capacity)
    uint32_t ext_window = 0;
    bool confirm = false;  // a window of the slot confirms the primes of its large gaps
    // preemption (serving): stop flag in mapped pinned host memory, read by the
    // persistent search; the search's arguments are kept for the resume
    volatile uint32_t *h_stop = nullptr;
    uint32_t *d_stop = nullptr;
    SearchArgs search{};
    // slot_finish's place between calls: after a finalize (0) or a record
    // confirmation (1); continuation rounds so far; extension positions done
    bool fin_active = false;
    int fin_phase = 0;
    uint32_t fin_round = 0, fin_ext = 0;
    int grid = 0;
    bool busy = false;
    uint64_t ticket = 0;
    pg_search_stats sst{};
};

int slot_alloc(Slot &s, uint64_t nm_cap, uint64_t nodd_cap, uint64_t bm_cap, uint64_t list_cap, uint32_t win_cap);
void slot_free(Slot &s);
// empties an idle slot (its stream must have no work on the staging buffers)
void slot_reset(Slot &s);
// Appends the window [m_start, m_start + m_inc) of job j: its coprime m, odd-m
// ranks and constants go into the pinned staging.  Returns SLOT_FULL when the
// slot has no room for it (the slot is unchanged).
int slot_add(Slot &s, pg_job *j, uint64_t m_start, uint64_t m_inc);
// Room left for a window of job j with nm coprime and nodd odd m.
bool slot_fits(const Slot &s, const pg_job *j, uint64_t nm, uint64_t nodd);
// Enqueues the device work of all windows on the slot's stream: uploads,
// sieves, the search (persistent or plain) and finalize.  graph: capture the
// persistent form as one CUDA graph.
int slot_enqueue(Slot &s, int form, uint32_t flags, bool graph);
// Waits for the queued work, continues unresolved sides past sl, and fills
// the slot's stats.  Gaps are then in h_gaps (next side 2i, prev side 2i+1).
// With wait = false it returns SLOT_PENDING after queueing each further round
// (record confirmation or continuation) instead of waiting for it: call it
// again once the slot's stream is idle.
int slot_finish(Slot &s, bool wait = true);
// Gives the slot a stop flag: its persistent searches can be preempted.
int slot_enable_preempt(Slot &s);
// Raises the stop flag of the slot's running search (host write, no call into
// the device); its warps leave after the items in hand.
void slot_preempt(Slot &s);
// Continues a search whose slot_finish returned SLOT_STOPPED: relaunches the
// persistent search from its queue head and finalize, on the slot's stream.
int slot_resume(Slot &s);

int job_create(pg_ctx *c, const pg_job_params &p, pg_job **out);

}  // namespace pg

struct pg_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t up = nullptr;  // host-to-device copies only: never queued behind a kernel
    int sms = 0;
    // PRP batch staging
    uint32_t *d_cand = nullptr;
    int32_t *d_res = nullptr;
    size_t cand_cap = 0, res_cap = 0;
    // prime tables of the jobs alive on this context
    std::mutex tables_mu;
    std::vector<std::weak_ptr<pg::Tables>> tables;
};

struct pg_job {
    pg_ctx *ctx = nullptr;
    // walk constants of the many-hit primes [walk_first, walk_first + walk_count)
    // of the table for this job's window width (segmented large-prime sieve)
    pg::WalkC *d_walk = nullptr;
    uint64_t walk_first = 0, walk_count = 0;
    pg_job_params prm{};
    std::shared_ptr<pg::Tables> T;
    uint32_t L = 0, sly = 0, W = 0, cap = 0;
    uint32_t *d_wheel = nullptr;
    // jobs built without waiting on the device (PG_JOB_NO_GRAPH): the wheel
    // and the walk table are in place once this event completes
    cudaEvent_t ready = nullptr;
    pg::WinInfo win{};  // K, trial residues, sly, rounds
    std::vector<uint8_t> coprime;       // [d] gcd(r, d) == 1
    uint64_t nm_cap = 0, nodd_cap = 0;  // one window of max_m_inc
    pg::Slot slot[PG_SEARCH_SLOTS];     // allocated on first use
    bool slots_ready = false;
    uint64_t next_ticket = 0;
    uint64_t own_bytes = 0;
    double setup_s = 0;
};
