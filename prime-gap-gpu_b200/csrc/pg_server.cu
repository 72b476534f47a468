// pg_server.cu -- the serving loop of include/primegap.h (pg_server_*).
//
// One worker thread owns the device work.  Clients only touch the request
// table under the server mutex: submit queues a request, wait / next_done
// sleep on a condition variable until the worker marks it done.
//
// Worker cycle:
//   1. admit queued requests in arrival order: their prime tables (keyed by
//      P, d, max_prime, small_limit) must be resident; a missing set is
//      built if it fits the budget, after evicting idle sets (no admitted
//      request uses them) least recently used first; a request whose tables
//      cannot fit waits, or fails when nothing else holds memory.
//   2. fill every idle slot with one search launch: the operand layout of
//      the oldest admitted request with windows left (with preemption: of the
//      cheapest class with windows left), then windows of every
//      admitted request of that layout in arrival order until the slot is
//      full (coprime m, windows, list space).  Windows of different requests
//      (different K, sl, rounds) share the launch; the kernels read each
//      side's constants from its window's WinInfo.
//   3. finish the oldest launch in flight whose stream is idle: queue its
//      next continuation or confirmation round if it needs one (it stays in
//      flight), else scatter its gaps to the requests; a request is done
//      when its last window is.
// Two slots (pg_server_params.slots) keep one launch queued behind the running
// one, so the host work of step 2 overlaps the device; the worker polls the
// running launch's stream so requests that arrive meanwhile go into a free
// slot at once.
//
// Preemption (pg_server_params.preempt_us): launches are scheduled by
// operand class (words per number; a test costs ~ words^2 x bits), cheapest
// first, and one slot is kept free of running launches.  A persistent launch
// holds every SM it fits on until its queue drains, so once cheaper windows
// have waited preempt_us (or a cheaper launch has been in flight that long),
// every running launch of a costlier class is told to stop (a flag in mapped
// host memory the warps read between test rounds); its warps leave after the
// tests in hand, finalize skips the launch, and the slot keeps the search's
// device state (SUSPENDED).  A suspended launch resumes from its queue head
// (the same kernel, same arguments) when fewer than min(slots - 1, 2)
// launches run and no cheaper work runs or waits; the slots beyond those hold
// stopped launches (default 4: two running, one stopped per class overtaken).  A request that has waited
// max(2 s, 100 x preempt_us) is placed first whatever its class.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "pg_host.h"

using namespace pg;

namespace {

struct TableKey {
    uint32_t p, d, q1;
    uint64_t max_prime;
    bool operator<(const TableKey &o) const {
        return std::tie(p, d, q1, max_prime) < std::tie(o.p, o.d, o.q1, o.max_prime);
    }
};

// Jobs of one table set: one per (sl, rounds, operand bound), created on demand.
struct TableEntry {
    std::shared_ptr<Tables> T;
    std::map<std::tuple<uint32_t, uint32_t, uint32_t>, pg_job *> jobs;
    uint64_t job_bytes = 0;
    uint32_t users = 0;     // admitted requests not yet done
    uint64_t last_use = 0;  // admission counter of the last user
};

enum class St { QUEUED, ADMITTED, DONE };

struct Request {
    uint64_t id = 0;
    pg_request rq{};
    St state = St::QUEUED;
    int status = PG_OK;
    std::string error;
    TableKey key{};
    pg_job *job = nullptr;
    uint64_t next_m = 0;    // first m not yet in a window
    uint64_t m_end = 0;
    uint64_t nm_assigned = 0;
    uint32_t windows = 0, windows_done = 0;
    std::vector<uint64_t> ms;
    std::vector<uint32_t> prev, next;
    double t_submit = 0, t_start = -1, t_done = 0;
    double k_log = 0;
};

// a window of a request placed in a slot
struct Placed {
    uint64_t id;
    uint32_t m_off;   // first m index in the slot
    uint32_t nm;
    uint64_t out_off; // first result index in the request
};

struct SlotState {
    Slot s;
    std::vector<Placed> placed;
    std::vector<const Tables *> tabs;  // table sets the launch reads
    bool inflight = false;   // work enqueued on the slot's stream
    bool stopping = false;   // its stop flag is raised
    bool suspended = false;  // its search stopped with items queued: resumed later
    double t_run = 0;        // when the launch (or its resume) was enqueued
    double t_wait = 0;       // submit time of the oldest request with windows in the launch
    uint64_t seq = 0;
};

uint32_t small_bound_of(const pg_request &r, uint32_t small_limit) {
    uint64_t q1 = std::max<uint64_t>(small_limit ? small_limit : 65536u, r.p);
    q1 = std::min<uint64_t>(q1, r.max_prime);
    return (uint32_t)std::max<uint64_t>(q1, r.p);
}

uint32_t bitlen(uint64_t v) { return v ? 64 - __builtin_clzll(v) : 0; }

bool prime_u32(uint32_t n) {
    if (n < 2) return false;
    for (uint64_t q = 2; q * q <= n; q++)
        if (n % q == 0) return false;
    return true;
}

}  // namespace

struct pg_server {
    pg_ctx *ctx = nullptr;
    pg_server_params prm{};
    std::chrono::steady_clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread worker;
    bool stop = false;
    uint64_t next_id = 1;
    std::map<uint64_t, Request> reqs;   // every request not yet waited for
    std::deque<uint64_t> order;         // queued / admitted ids in arrival order
    double aging_s = 0;                 // with preemption: a request waiting this long goes first
    std::deque<uint64_t> done_ids;      // finished, not yet returned by next_done
    std::map<TableKey, TableEntry> tables;
    uint64_t admissions = 0;
    std::vector<SlotState> slot;  // launch slots (pg_server_params.slots)
    uint64_t slot_bytes = 0;
    uint64_t launch_seq = 0;
    pg_server_stats st{};

    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }

    uint64_t resident() const {
        uint64_t b = slot_bytes;
        for (const auto &kv : tables) b += kv.second.T->bytes + kv.second.job_bytes;
        return b;
    }

    void note_bytes() {
        st.resident_bytes = resident();
        st.peak_bytes = std::max(st.peak_bytes, st.resident_bytes);
    }

    // ---------------------------------------------------------- requests

    void finish(Request &r, int status, const std::string &err) {
        if (r.state == St::DONE) return;
        if (r.state == St::ADMITTED) {
            auto it = tables.find(r.key);
            if (it != tables.end() && it->second.users) it->second.users--;
        }
        r.state = St::DONE;
        r.status = status;
        r.error = err;
        r.t_done = now();
        st.requests_done++;
        if (status == PG_OK) st.m_done += r.ms.size();
        order.erase(std::remove(order.begin(), order.end(), r.id), order.end());
        done_ids.push_back(r.id);
        cv_done.notify_all();
    }

    // A launch in flight may still read a table set whose requests are all
    // done (one failed while another of its windows was running): such a
    // set is not evicted until the launch has finished.
    bool read_in_flight(const Tables *T) const {
        for (const auto &ss : slot)
            if ((ss.inflight || ss.suspended) && std::find(ss.tabs.begin(), ss.tabs.end(), T) != ss.tabs.end())
                return true;
        return false;
    }

    void evict(std::map<TableKey, TableEntry>::iterator it) {
        for (auto &kv : it->second.jobs) pg_job_destroy(kv.second);
        tables.erase(it);  // the last reference frees the device tables
        st.tables_evicted++;
    }

    // Builds (or finds) the job of an admitted request; called without the lock.
    int job_for(TableEntry &e, const pg_request &rq, pg_job **out) {
        const uint32_t mbits = bitlen(rq.m_start + rq.m_inc);
        const auto jk = std::make_tuple(rq.sl, rq.rounds, mbits);
        auto it = e.jobs.find(jk);
        if (it != e.jobs.end()) {
            *out = it->second;
            return PG_OK;
        }
        pg_job_params p{};
        p.p = rq.p;
        p.d = rq.d;
        p.sl = rq.sl;
        p.max_prime = rq.max_prime;
        p.max_m_inc = prm.window_m;
        p.max_m = mbits >= 64 ? ~0ull : (1ull << mbits) - 1;
        p.rounds = rq.rounds;
        p.small_limit = prm.small_limit;
        p.ext_window = prm.ext_window;
        p.tpi = prm.tpi;
        p.flags = PG_JOB_NO_GRAPH | PG_JOB_COMPACT_WALK;  // jobs come and go with requests
        pg_job *j = nullptr;
        int rc = job_create(ctx, p, &j);
        if (rc) return rc;
        e.jobs[jk] = j;
        e.job_bytes += j->own_bytes;
        *out = j;
        return PG_OK;
    }

    // Admits queued requests in arrival order (step 1).  Holds the lock
    // except around table and job builds.
    void admit(std::unique_lock<std::mutex> &lk) {
        for (size_t oi = 0; oi < order.size(); oi++) {
            Request &r = reqs.at(order[oi]);
            if (r.state != St::QUEUED) continue;
            pg_job_params tp{};
            tp.p = r.rq.p;
            tp.d = r.rq.d;
            tp.max_prime = r.rq.max_prime;
            tp.small_limit = prm.small_limit;
            r.key = TableKey{r.rq.p, r.rq.d, small_bound_of(r.rq, prm.small_limit), r.rq.max_prime};
            auto it = tables.find(r.key);
            if (it == tables.end()) {
                const uint64_t need = tables_bytes_estimate(tp);
                while (resident() + need > prm.hbm_budget) {  // evict idle sets, oldest use first
                    auto victim = tables.end();
                    for (auto t = tables.begin(); t != tables.end(); ++t)
                        if (t->second.users == 0 && !read_in_flight(t->second.T.get()) &&
                            (victim == tables.end() || t->second.last_use < victim->second.last_use))
                            victim = t;
                    if (victim == tables.end()) break;
                    evict(victim);
                }
                if (resident() + need > prm.hbm_budget) {
                    bool others = false;
                    for (const auto &kv : tables) others |= kv.second.users > 0;
                    if (!others && tables.empty()) {
                        char buf[160];
                        snprintf(buf, sizeof buf, "prime tables of ~%llu bytes exceed the budget of %llu bytes",
                                 (unsigned long long)need, (unsigned long long)prm.hbm_budget);
                        finish(r, PG_ERR_NOMEM, buf);
                        oi--;  // finish removed it from order
                    }
                    continue;  // wait for memory
                }
                std::shared_ptr<Tables> T;
                lk.unlock();
                int rc = tables_get(ctx, tp, T);
                std::string err = rc ? pg_last_error() : "";
                lk.lock();
                if (rc) {
                    finish(r, rc, err);
                    oi--;
                    continue;
                }
                TableEntry e;
                e.T = T;
                it = tables.emplace(r.key, std::move(e)).first;
                st.tables_built++;
            }
            TableEntry &e = it->second;
            pg_job *j = nullptr;
            lk.unlock();
            int rc = job_for(e, r.rq, &j);
            std::string err = rc ? pg_last_error() : "";
            lk.lock();
            if (rc) {
                finish(r, rc, err);
                oi--;
                continue;
            }
            e.users++;
            e.last_use = ++admissions;
            r.job = j;
            r.k_log = e.T->k_log;
            r.state = St::ADMITTED;
            r.next_m = r.rq.m_start;
            r.m_end = r.rq.m_start + r.rq.m_inc;
            const uint64_t nm = pg_count_m(r.rq.m_start, r.rq.m_inc, r.rq.d);
            r.ms.assign(nm, 0);
            r.prev.assign(nm, 0);
            r.next.assign(nm, 0);
            if (nm == 0) {
                finish(r, PG_OK, "");
                oi--;
            }
            note_bytes();
        }
    }

    // Scheduling class of an operand layout: its words (a test costs ~ words^2 x bits).
    static uint32_t cls(uint32_t layout) { return layout_words(layout); }

    // The layout the next launch packs (0: no windows wait) and the submit
    // time of its oldest waiting request.  Without preemption: the oldest
    // waiting request's.  With it: the cheapest class with windows waiting,
    // so short requests overtake long ones, unless the oldest waiting request
    // has waited aging_s, which then goes first.
    uint32_t next_layout(double *since = nullptr) const {
        uint32_t best = 0;
        double t_best = -1;
        bool first = true;
        for (uint64_t id : order) {
            const Request &r = reqs.at(id);
            if (r.state != St::ADMITTED || r.next_m >= r.m_end) continue;
            if (first && (!prm.preempt_us || now() - r.t_submit >= aging_s)) {
                best = r.job->L;
                t_best = r.t_submit;
                break;
            }
            first = false;
            if (!best || cls(r.job->L) < cls(best)) {
                best = r.job->L;
                t_best = r.t_submit;
            }
        }
        if (since) *since = t_best;
        return best;
    }

    // Packs windows into an idle slot (step 2); false when there is no work.
    bool fill(SlotState &ss) {
        Slot &s = ss.s;
        slot_reset(s);
        ss.placed.clear();
        ss.tabs.clear();
        const uint32_t layout = next_layout();
        if (!layout) return false;
        ss.t_wait = now();
        std::vector<std::pair<uint64_t, std::pair<int, std::string>>> failed;
        for (uint64_t id : order) {
            Request &r = reqs.at(id);
            if (r.state != St::ADMITTED || r.job->L != layout) continue;
            bool full = false;
            while (r.next_m < r.m_end) {
                const uint64_t inc = std::min<uint64_t>(r.m_end - r.next_m, prm.window_m);
                const uint32_t m_off = s.nm;
                const int rc = slot_add(s, r.job, r.next_m, inc);
                if (rc == SLOT_FULL) {
                    full = true;
                    break;
                }
                if (rc) {  // an argument error of this request
                    failed.push_back({r.id, {rc, pg_last_error()}});
                    r.next_m = r.m_end;
                    break;
                }
                const uint32_t nm = s.nm - m_off;
                ss.placed.push_back(Placed{r.id, m_off, nm, r.nm_assigned});
                if (std::find(ss.tabs.begin(), ss.tabs.end(), r.job->T.get()) == ss.tabs.end())
                    ss.tabs.push_back(r.job->T.get());
                r.nm_assigned += nm;
                r.next_m += inc;
                r.windows++;
                if (r.t_start < 0) r.t_start = now();
                ss.t_wait = std::min(ss.t_wait, r.t_submit);
            }
            if (full) break;
        }
        for (auto &f : failed) finish(reqs.at(f.first), f.second.first, f.second.second);
        if (ss.placed.empty()) {
            // the first window did not fit an empty slot: cannot happen with
            // the capacities of create(); fail the request rather than spin
            for (uint64_t id : order) {
                Request &r = reqs.at(id);
                if (r.state == St::ADMITTED && r.job->L == layout && r.next_m < r.m_end) {
                    finish(r, PG_ERR_UNSUPPORTED, "window larger than a search launch");
                    break;
                }
            }
            return false;
        }
        return true;
    }

    // Fails the requests of a launch that hit an error; whatever of it was
    // enqueued has finished before the slot counts as idle.  The server lock
    // is released while the stream drains, so submit / wait / next_done
    // callers do not block on device time; only this worker thread touches
    // the slot meanwhile.
    void fail_launch(std::unique_lock<std::mutex> &lk, SlotState &ss, int rc, std::string err) {
        lk.unlock();
        const cudaError_t es = cudaStreamSynchronize(ss.s.st);
        const cudaError_t el = cudaGetLastError();
        lk.lock();
        const cudaError_t extra = es != cudaSuccess ? es : el;
        if (extra != cudaSuccess) {
            err += "; draining the launch: ";
            err += cudaGetErrorString(extra);
        }
        for (const Placed &pl : ss.placed) {
            auto it = reqs.find(pl.id);
            if (it != reqs.end()) finish(it->second, rc, err);
        }
        ss.placed.clear();
        ss.inflight = false;
        ss.stopping = false;
        ss.suspended = false;
    }

    // Scatters a finished launch's gaps (step 3).
    void deliver(SlotState &ss) {
        const Slot &s = ss.s;
        for (const Placed &pl : ss.placed) {
            auto it = reqs.find(pl.id);
            if (it == reqs.end() || it->second.state == St::DONE) continue;
            Request &r = it->second;
            for (uint32_t i = 0; i < pl.nm; i++) {
                const uint32_t src = pl.m_off + i;
                r.ms[pl.out_off + i] = s.h_ms[src];
                r.next[pl.out_off + i] = s.h_gaps[2 * src];
                r.prev[pl.out_off + i] = s.h_gaps[2 * src + 1];
            }
            r.windows_done++;
            if (r.next_m >= r.m_end && r.windows_done == r.windows) finish(r, PG_OK, "");
        }
        st.launches++;
        st.windows += s.parts.size();
        st.prp_tests += s.sst.prp_tests;
        st.sieve_ms += s.sst.sieve_ms;
        st.prp_ms += s.sst.prp_ms;
        ss.placed.clear();
        ss.inflight = false;
    }

    // launches occupying the device (running or being stopped)
    size_t running() const {
        size_t n = 0;
        for (const auto &ss : slot) n += ss.inflight;
        return n;
    }

    // With preemption: a persistent launch holds every SM it fits on until its
    // queue drains, so cheaper work would wait behind it.  Once a launch of a
    // cheaper class has been in flight preempt_us, or the next launch's
    // windows (next_layout) have waited preempt_us with a slot free for them,
    // raise the stop flag of every running launch of a costlier class.
    void maybe_preempt() {
        if (!prm.preempt_us) return;
        const double limit = prm.preempt_us * 1e-6, t = now();
        uint32_t c = UINT32_MAX;  // cheapest class that has waited long enough
        bool idle = false;
        for (const auto &ss : slot) {
            idle |= !ss.inflight && !ss.suspended;
            if (ss.inflight && !ss.stopping && t - ss.t_wait >= limit) c = std::min(c, cls(ss.s.L));
        }
        double since = -1;
        const uint32_t L = next_layout(&since);
        if (L && idle && t - since >= limit) c = std::min(c, cls(L));
        if (c == UINT32_MAX) return;
        for (auto &ss : slot) {
            if (!ss.inflight || ss.stopping || cls(ss.s.L) <= c) continue;
            slot_preempt(ss.s);
            ss.stopping = true;
            st.preemptions++;
        }
    }

    // A stopped launch resumes when no launch of a cheaper class runs and,
    // unless the server is stopping, no windows of a cheaper class wait.
    bool may_resume(const SlotState &x) const {
        for (const auto &ss : slot)
            if (ss.inflight && cls(ss.s.L) < cls(x.s.L)) return false;
        if (stop) return true;
        const uint32_t L = next_layout();
        return !L || cls(L) >= cls(x.s.L);
    }

    // An idle slot takes new windows unless a stopped launch of the same or a
    // cheaper class waits to resume (it goes first).
    bool may_fill() const {
        const uint32_t L = next_layout();
        if (!L) return false;
        for (const auto &ss : slot)
            if (ss.suspended && cls(ss.s.L) <= cls(L)) return false;
        return true;
    }

    void run() {
        cudaSetDevice(ctx->device);
        std::unique_lock<std::mutex> lk(mu);
        double busy_since = -1;
        // with preemption the slots beyond two hold stopped launches: one per
        // operand class that was overtaken, and one is kept free
        const size_t run_limit = prm.preempt_us ? std::min<size_t>(slot.size() - 1, 2) : slot.size();
        while (true) {
            if (!stop) admit(lk);
            // resume stopped launches, oldest first, while there is room
            while (running() < run_limit) {
                SlotState *next = nullptr;
                for (auto &ss : slot)
                    if (ss.suspended && may_resume(ss) && (!next || ss.seq < next->seq)) next = &ss;
                if (!next) break;
                next->suspended = false;
                next->t_run = now();
                const int rc = slot_resume(next->s);
                if (rc) {
                    fail_launch(lk, *next, rc, pg_last_error());
                    continue;
                }
                next->inflight = true;
                if (busy_since < 0) busy_since = now();
            }
            // step 2: idle slots get launches while fewer than run_limit run
            for (auto &ss : slot) {
                if (ss.inflight || ss.suspended || stop) continue;
                if (running() >= run_limit || !may_fill()) break;
                if (!fill(ss)) break;
                ss.seq = ++launch_seq;
                ss.t_run = now();
                int rc = slot_enqueue(ss.s, PG_SEARCH_PERSISTENT, PG_SUBMIT_WARPS_PER_SM(prm.warps_per_sm), false);
                if (rc) {
                    fail_launch(lk, ss, rc, pg_last_error());
                    continue;
                }
                ss.inflight = true;
                if (busy_since < 0) busy_since = now();
            }
            if (!stop) maybe_preempt();
            // step 3: finish a launch whose stream is idle (oldest first); until
            // then keep admitting and filling as requests arrive
            SlotState *ready = nullptr;
            bool any_inflight = false;
            for (auto &ss : slot) {
                if (!ss.inflight) continue;
                any_inflight = true;
                if (ready && ss.seq > ready->seq) continue;
                const cudaError_t q = cudaStreamQuery(ss.s.st);
                if (q == cudaErrorNotReady) {
                    if (cudaPeekAtLastError() == cudaErrorNotReady) cudaGetLastError();
                    continue;
                }
                ready = &ss;
            }
            if (ready) {
                lk.unlock();
                // one step: a launch needing a continuation or confirmation
                // round gets it queued and stays in flight, so the worker
                // never waits on the device here
                const int rc = slot_finish(ready->s, false);
                const std::string err = rc < 0 ? pg_last_error() : "";
                lk.lock();
                if (rc == SLOT_PENDING) continue;
                ready->inflight = false;
                ready->stopping = false;
                if (rc == SLOT_STOPPED) {
                    ready->suspended = true;  // holds its state until resumed
                } else if (rc) {
                    ready->inflight = true;   // fail_launch drains the stream and frees the slot
                    fail_launch(lk, *ready, rc, err);
                } else {
                    deliver(*ready);
                }
                bool any = false;
                for (auto &ss : slot) any |= ss.inflight || ss.suspended;
                if (!any && busy_since >= 0) {
                    st.busy_s += now() - busy_since;
                    busy_since = -1;
                }
                note_bytes();
                continue;
            }
            if (any_inflight) {
                cv_work.wait_for(lk, std::chrono::microseconds(200));
                continue;
            }
            bool suspended = false;
            for (auto &ss : slot) suspended |= ss.suspended;
            if (suspended) continue;  // resumed above on the next pass
            if (stop) break;
            bool work = false;
            for (uint64_t id : order) {
                const Request &r = reqs.at(id);
                work |= r.state == St::ADMITTED && r.next_m < r.m_end;
            }
            if (!work) cv_work.wait_for(lk, std::chrono::milliseconds(20));
        }
        // stopping: nothing in flight; fail what never ran
        std::vector<uint64_t> left(order.begin(), order.end());
        for (uint64_t id : left) finish(reqs.at(id), PG_ERR_STATE, "server destroyed before the request ran");
    }
};

extern "C" int pg_server_create(int device, const pg_server_params *params, pg_server **out) {
    if (!out) return fail(PG_ERR_ARG, "pg_server_create: out is NULL");
    *out = nullptr;
    pg_server_params p = params ? *params : pg_server_params{};
    if (!p.batch_m) p.batch_m = 65536;
    if (!p.window_m) p.window_m = 65536;
    if (!p.max_windows) p.max_windows = 64;
    if (!p.max_sl) p.max_sl = 20000;
    if (!p.ext_window) p.ext_window = 64;
    if (p.max_windows > 65535) return fail(PG_ERR_ARG, "max_windows=%u > 65535", p.max_windows);
    if (p.max_sl / 2 > 65535) return fail(PG_ERR_ARG, "max_sl=%u > 131071", p.max_sl);
    if (!p.slots) p.slots = p.preempt_us ? 4 : 2;
    if (p.slots > 8) return fail(PG_ERR_ARG, "slots=%u > 8", p.slots);
    if (p.preempt_us && p.slots < 2) return fail(PG_ERR_ARG, "preemption needs at least 2 slots");
    pg_ctx *c = nullptr;
    int rc = pg_ctx_create(device, &c);
    if (rc) return rc;
    if (!p.hbm_budget) {
        size_t free_b = 0, total_b = 0;
        const cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
        if (e != cudaSuccess) {
            pg_ctx_destroy(c);
            return fail(PG_ERR_CUDA, "pg_server_create: cudaMemGetInfo: %s", cudaGetErrorString(e));
        }
        p.hbm_budget = free_b / 4 * 3;
    }
    pg_server *srv = new pg_server();
    srv->ctx = c;
    srv->prm = p;
    srv->t0 = std::chrono::steady_clock::now();
    srv->slot.resize(p.slots);
    srv->aging_s = std::max(2.0, 1e-4 * p.preempt_us);
    // launch capacities: batch_m coprime m over at most max_windows windows
    // of window_m m; lists at most half of each side's positions
    const uint64_t nodd_w = p.window_m / 2 + 1;
    const uint64_t nm_cap = p.batch_m;
    const uint64_t nodd_cap = std::min<uint64_t>((uint64_t)p.max_windows * nodd_w, 8 * nm_cap + 2 * nodd_w);
    const uint64_t W = (p.max_sl / 2 * 2 + 1 + 31) / 32;
    const uint64_t bm_cap = std::min<uint64_t>(nodd_w, nm_cap) * W;
    const uint64_t list_cap = nm_cap * std::max<uint64_t>(p.max_sl / 2, 1);
    for (auto &ss : srv->slot) {
        rc = slot_alloc(ss.s, nm_cap, nodd_cap, bm_cap, list_cap, p.max_windows);
        if (rc) {
            std::string keep = pg_last_error();
            for (auto &s2 : srv->slot) slot_free(s2.s);
            pg_ctx_destroy(c);
            delete srv;
            return fail(rc, "%s", keep.c_str());
        }
        srv->slot_bytes += ss.s.bytes;
        if (p.preempt_us && !rc) rc = slot_enable_preempt(ss.s);
        if (rc) {
            std::string keep = pg_last_error();
            for (auto &s2 : srv->slot) slot_free(s2.s);
            pg_ctx_destroy(c);
            delete srv;
            return fail(rc, "%s", keep.c_str());
        }
    }
    if (srv->slot_bytes > p.hbm_budget) {
        for (auto &ss : srv->slot) slot_free(ss.s);
        pg_ctx_destroy(c);
        const uint64_t sb = srv->slot_bytes;
        delete srv;
        return fail(PG_ERR_NOMEM, "launch buffers of %llu bytes exceed the budget of %llu bytes",
                    (unsigned long long)sb, (unsigned long long)p.hbm_budget);
    }
    srv->note_bytes();
    srv->worker = std::thread([srv] { srv->run(); });
    *out = srv;
    return PG_OK;
}

extern "C" int pg_server_submit(pg_server *srv, const pg_request *rq, uint64_t *id) {
    if (!srv || !rq || !id) return fail(PG_ERR_ARG, "pg_server_submit: NULL argument");
    pg_request r = *rq;
    if (!r.rounds) r.rounds = 1;
    if (!prime_u32(r.p)) return fail(PG_ERR_ARG, "p=%u is not prime", r.p);
    if (r.d == 0 || r.d % 2) return fail(PG_ERR_ARG, "d=%u must be even", r.d);
    if (r.sl < 2 || r.sl > srv->prm.max_sl) return fail(PG_ERR_ARG, "sl=%u outside [2, %u]", r.sl, srv->prm.max_sl);
    if (r.rounds > 16) return fail(PG_ERR_ARG, "rounds=%u (1..16)", r.rounds);
    if (r.max_prime >= (1ull << 40)) return fail(PG_ERR_ARG, "max_prime must be < 2^40");
    if (r.m_start == 0 || r.m_inc == 0) return fail(PG_ERR_ARG, "empty or zero m range");
    if (r.m_start + r.m_inc < r.m_start) return fail(PG_ERR_ARG, "m range overflows");
    std::lock_guard<std::mutex> lk(srv->mu);
    if (srv->stop) return fail(PG_ERR_STATE, "server is stopping");
    Request q;
    q.id = srv->next_id++;
    q.rq = r;
    q.t_submit = srv->now();
    srv->order.push_back(q.id);
    *id = q.id;
    srv->reqs.emplace(q.id, std::move(q));
    srv->cv_work.notify_one();
    return PG_OK;
}

template <class Pred>
static bool wait_on(std::condition_variable &cv, std::unique_lock<std::mutex> &lk, double timeout_s, Pred pred) {
    if (timeout_s < 0) {
        cv.wait(lk, pred);
        return true;
    }
    return cv.wait_for(lk, std::chrono::duration<double>(timeout_s), pred);
}

extern "C" int pg_server_wait(pg_server *srv, uint64_t id, double timeout_s, uint64_t *ms, uint32_t *prev_gap,
                              uint32_t *next_gap, pg_request_info *info) {
    if (!srv) return fail(PG_ERR_ARG, "pg_server_wait: server is NULL");
    std::unique_lock<std::mutex> lk(srv->mu);
    if (srv->reqs.find(id) == srv->reqs.end())
        return fail(PG_ERR_ARG, "pg_server_wait: no request %llu", (unsigned long long)id);
    // looked up again after every wake-up: another waiter of the same id may
    // have returned it (and erased it) meanwhile
    auto done_or_gone = [&] {
        auto f = srv->reqs.find(id);
        return f == srv->reqs.end() || f->second.state == St::DONE;
    };
    if (!wait_on(srv->cv_done, lk, timeout_s, done_or_gone))
        return fail(PG_ERR_TIMEOUT, "request %llu not done", (unsigned long long)id);
    auto it = srv->reqs.find(id);
    if (it == srv->reqs.end())
        return fail(PG_ERR_ARG, "pg_server_wait: request %llu was returned to another waiter", (unsigned long long)id);
    Request &r = it->second;
    const size_t n = r.ms.size();
    if (info) {
        info->m_count = r.status == PG_OK ? n : 0;
        info->k_log = r.k_log;
        info->submit_s = r.t_submit;
        info->start_s = r.t_start;
        info->done_s = r.t_done;
        info->windows = r.windows;
        info->status = r.status;
    }
    const int status = r.status;
    if (status == PG_OK) {
        if (ms && n) std::memcpy(ms, r.ms.data(), n * 8);
        if (prev_gap && n) std::memcpy(prev_gap, r.prev.data(), n * 4);
        if (next_gap && n) std::memcpy(next_gap, r.next.data(), n * 4);
    } else {
        fail(status, "%s", r.error.c_str());
    }
    srv->done_ids.erase(std::remove(srv->done_ids.begin(), srv->done_ids.end(), id), srv->done_ids.end());
    srv->reqs.erase(it);
    return status;
}

extern "C" int pg_server_next_done(pg_server *srv, double timeout_s, uint64_t *id) {
    if (!srv || !id) return fail(PG_ERR_ARG, "pg_server_next_done: NULL argument");
    std::unique_lock<std::mutex> lk(srv->mu);
    if (!wait_on(srv->cv_done, lk, timeout_s, [&] { return !srv->done_ids.empty(); }))
        return fail(PG_ERR_TIMEOUT, "no request finished");
    *id = srv->done_ids.front();
    srv->done_ids.pop_front();
    return PG_OK;
}

extern "C" int pg_server_get_stats(pg_server *srv, pg_server_stats *stats) {
    if (!srv || !stats) return fail(PG_ERR_ARG, "pg_server_get_stats: NULL argument");
    std::lock_guard<std::mutex> lk(srv->mu);
    *stats = srv->st;
    return PG_OK;
}

extern "C" double pg_server_clock(const pg_server *srv) { return srv ? srv->now() : 0.0; }

extern "C" int pg_server_destroy(pg_server *srv) {
    if (!srv) return PG_OK;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stop = true;
    }
    srv->cv_work.notify_all();
    if (srv->worker.joinable()) srv->worker.join();
    cudaSetDevice(srv->ctx->device);
    for (auto &ss : srv->slot) slot_free(ss.s);
    while (!srv->tables.empty()) {
        for (auto &kv : srv->tables.begin()->second.jobs) pg_job_destroy(kv.second);
        srv->tables.erase(srv->tables.begin());
    }
    pg_ctx_destroy(srv->ctx);
    delete srv;
    return PG_OK;
}
