// pg_api.cu -- host side of the C ABI (include/primegap.h).
//
// Job set-up builds K = P#/d with a small host bignum (gap_common.cpp:60-65),
// the small-prime tables on the host, and the large prime table (every prime
// in (small_limit, max_prime] with K mod p and K^-1 mod p) on the device.
// These tables depend on (P, d, max_prime, small_limit) only; jobs on one
// context with the same key share one copy whatever their sl.  A job adds
// its K-prime wheel row and PG_SEARCH_SLOTS window slots, each with its own
// stream and buffers, so consecutive windows overlap on the device.  A slot
// runs one search launch over one or more windows on its stream:
//   per window: large-prime sieve -> small-prime sieve + survivor lists
//   then: PRP search (persistent or plain) -> finalize/confirm
//   [-> continuation launches]
// No function exits the process; errors come back as PG_ERR_* with a message
// in pg_last_error().
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pg_host.h"

using namespace pg;

// ============================================================== errors

static thread_local std::string g_last_error;

int pg::fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

extern "C" const char *pg_last_error(void) { return g_last_error.c_str(); }

void pg::set_error(const char *msg) { g_last_error = msg; }

// Timing events are recorded as external event nodes when the stream is
// being captured, so they keep their timestamps inside a window's graph.
cudaError_t pg::record_ev(cudaEvent_t e, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t err = cudaStreamIsCapturing(st, &cs);
    if (err != cudaSuccess) return err;
    return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(e, st, cudaEventRecordExternal)
                                               : cudaEventRecord(e, st);
}

extern "C" const char *pg_version(void) { return "primegap-b200 0.2 (sm_100a)"; }

// ======================================================= host bignum (K)


static void big_trim(Big &a) {
    while (!a.empty() && a.back() == 0) a.pop_back();
}
static void big_mul_u32(Big &a, uint32_t m) {
    uint64_t c = 0;
    for (auto &w : a) {
        c += (uint64_t)w * m;
        w = (uint32_t)c;
        c >>= 32;
    }
    if (c) a.push_back((uint32_t)c);
}
static uint32_t big_divmod_u32(Big &a, uint32_t d) {
    uint64_t r = 0;
    for (size_t i = a.size(); i-- > 0;) {
        const uint64_t cur = (r << 32) | a[i];
        a[i] = (uint32_t)(cur / d);
        r = cur % d;
    }
    big_trim(a);
    return (uint32_t)r;
}
static uint32_t big_mod_u32(const Big &a, uint32_t d) {
    uint64_t r = 0;
    for (size_t i = a.size(); i-- > 0;) r = ((r << 32) | a[i]) % d;
    return (uint32_t)r;
}
static uint32_t big_bits(const Big &a) {
    if (a.empty()) return 0;
    return 32 * (uint32_t)(a.size() - 1) + (32 - __builtin_clz(a.back()));
}

// log(K) computed as _log (gap_common.cpp:44-48): mpz_get_d_2exp truncates
// the mantissa to 53 bits, then log(mantissa) + log(2) * exp.
static double big_log(const Big &a) {
    const uint32_t bits = big_bits(a);
    uint64_t top = 0;  // the top min(bits, 64) bits
    for (int b = 0; b < 64 && b < (int)bits; b++) {
        const uint32_t pos = bits - 1 - b;
        top = (top << 1) | ((a[pos >> 5] >> (pos & 31)) & 1u);
    }
    const int have = bits < 64 ? (int)bits : 64;
    const uint64_t mant53 = have > 53 ? top >> (have - 53) : top << (53 - have);
    const double d = (double)mant53 / 9007199254740992.0;  // / 2^53, in [0.5, 1)
    return std::log(d) + std::log(2.0) * (double)bits;
}

static std::vector<uint32_t> host_primes(uint32_t n) {  // all primes <= n
    std::vector<uint8_t> comp(n + 1, 0);
    std::vector<uint32_t> out;
    for (uint64_t i = 2; i <= n; i++) {
        if (comp[i]) continue;
        out.push_back((uint32_t)i);
        for (uint64_t j = i * i; j <= n; j += i) comp[j] = 1;
    }
    return out;
}

static bool is_prime_u32(uint32_t n) {
    if (n < 2) return false;
    for (uint64_t q = 2; q * q <= n; q++)
        if (n % q == 0) return false;
    return true;
}

uint64_t pg::gcd64(uint64_t a, uint64_t b) {
    while (b) {
        uint64_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}

// ============================================================== context

extern "C" int pg_ctx_create(int device, pg_ctx **out) {
    if (!out) return fail(PG_ERR_ARG, "pg_ctx_create: out is NULL");
    *out = nullptr;
    int n = 0;
    PG_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) return fail(PG_ERR_ARG, "pg_ctx_create: device %d of %d", device, n);
    PG_CUDA(cudaSetDevice(device));
    pg_ctx *c = new pg_ctx();
    c->device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->up, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        if (c->stream) cudaStreamDestroy(c->stream);
        delete c;
        return fail(PG_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
    }
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
    *out = c;
    return PG_OK;
}

extern "C" void *pg_ctx_stream(pg_ctx *c) { return c ? (void *)c->stream : nullptr; }

extern "C" int pg_measure_imad_peak(pg_ctx *c, double *imad_per_second) {
    if (!c || !imad_per_second) return fail(PG_ERR_ARG, "pg_measure_imad_peak: NULL argument");
    PG_CUDA(cudaSetDevice(c->device));
    uint32_t *sink = nullptr;
    cudaEvent_t e0, e1;
    PG_CUDA(cudaMalloc((void **)&sink, 4));
    PG_CUDA(cudaEventCreate(&e0));
    PG_CUDA(cudaEventCreate(&e1));
    const int grid = c->sms * 8;  // 2048 threads per SM
    const uint32_t iters = 4096;
    PG_CUDA(launch_imad_peak(grid, 64, sink, c->stream));  // warm-up
    double best = 0;
    for (int rep = 0; rep < 3; rep++) {
        PG_CUDA(cudaEventRecord(e0, c->stream));
        PG_CUDA(launch_imad_peak(grid, iters, sink, c->stream));
        PG_CUDA(cudaEventRecord(e1, c->stream));
        PG_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        PG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        const double ops = (double)grid * 256.0 * iters * 16.0 * 8.0;
        best = std::max(best, ops / (ms * 1e-3));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    *imad_per_second = best;
    return PG_OK;
}

extern "C" int pg_ctx_destroy(pg_ctx *c) {
    if (!c) return PG_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    cudaFree(c->d_cand);
    cudaFree(c->d_res);
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->up) {
        cudaStreamSynchronize(c->up);
        cudaStreamDestroy(c->up);
    }
    delete c;
    return PG_OK;
}

// ================================================================== PRP

extern "C" int pg_prp_batch_device(pg_ctx *c, const uint32_t *d_limbs, uint32_t n, uint32_t words, uint32_t rounds,
                                   int32_t *d_passed, void *stream) {
    if (!c) return fail(PG_ERR_ARG, "pg_prp_batch_device: ctx is NULL");
    if (n == 0) return PG_OK;
    if (!d_limbs || !d_passed) return fail(PG_ERR_ARG, "pg_prp_batch_device: NULL buffer");
    if (words == 0 || words > PG_MAX_WORDS) return fail(PG_ERR_ARG, "pg_prp_batch_device: words=%u", words);
    if (rounds < 1 || rounds > 16) return fail(PG_ERR_ARG, "pg_prp_batch_device: rounds=%u (1..16)", rounds);
    const uint32_t L = pick_limbs(words);
    if (!L) return fail(PG_ERR_UNSUPPORTED, "pg_prp_batch_device: %u words above the compiled limit", words);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    PG_CUDA(cudaSetDevice(c->device));
    PG_CUDA(launch_prp_batch(L, d_limbs, words, n, rounds, d_passed, st));
    return PG_OK;
}

extern "C" int pg_prp_batch(pg_ctx *c, const uint32_t *limbs, uint32_t n, uint32_t words, uint32_t rounds,
                            int32_t *passed) {
    if (!c) return fail(PG_ERR_ARG, "pg_prp_batch: ctx is NULL");
    if (n == 0) return PG_OK;
    if (!limbs || !passed) return fail(PG_ERR_ARG, "pg_prp_batch: NULL buffer");
    if (words == 0 || words > PG_MAX_WORDS) return fail(PG_ERR_ARG, "pg_prp_batch: words=%u", words);
    PG_CUDA(cudaSetDevice(c->device));
    const size_t cb = (size_t)n * words * sizeof(uint32_t), rb = (size_t)n * sizeof(int32_t);
    if (cb > c->cand_cap) {
        cudaFree(c->d_cand);
        c->d_cand = nullptr;
        c->cand_cap = 0;
        PG_CUDA(cudaMalloc((void **)&c->d_cand, cb));
        c->cand_cap = cb;
    }
    if (rb > c->res_cap) {
        cudaFree(c->d_res);
        c->d_res = nullptr;
        c->res_cap = 0;
        PG_CUDA(cudaMalloc((void **)&c->d_res, rb));
        c->res_cap = rb;
    }
    PG_CUDA(cudaMemcpyAsync(c->d_cand, limbs, cb, cudaMemcpyHostToDevice, c->stream));
    int rc = pg_prp_batch_device(c, c->d_cand, n, words, rounds, c->d_res, c->stream);
    if (rc) return rc;
    PG_CUDA(cudaMemcpyAsync(passed, c->d_res, rb, cudaMemcpyDeviceToHost, c->stream));
    PG_CUDA(cudaStreamSynchronize(c->stream));
    return PG_OK;
}

// ================================================================ tables

template <typename T>
static int dalloc(uint64_t &acct, T **p, size_t count) {
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = cudaMalloc((void **)p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? PG_ERR_NOMEM : PG_ERR_CUDA, "cudaMalloc(%zu): %s", bytes,
                    cudaGetErrorString(e));
    }
    acct += bytes;
    return PG_OK;
}

pg::Tables::~Tables() {
    cudaSetDevice(device);
    void *ptrs[] = {d_sq, d_sr, d_sbar, d_tq, d_lp, d_lc, d_lcinv};
    for (void *p : ptrs) cudaFree(p);
}

static uint32_t bitlen64(uint64_t v) { return v ? 64 - __builtin_clzll(v) : 0; }

// small primes are <= q1: max(small_limit, P), capped at the sieve limit
static uint32_t small_bound(const pg_job_params &p) {
    uint32_t q1 = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(p.small_limit ? p.small_limit : 65536u, p.p),
                                               p.max_prime);
    return std::max(q1, p.p);
}

uint64_t pg::tables_bytes_estimate(const pg_job_params &p) {
    const double x = (double)std::max<uint64_t>(p.max_prime, 17);
    const double pi_hi = 1.26 * x / std::log(x);  // pi(x) < 1.25506 x / ln x
    const double esz = p.max_prime >= (1ull << 32) ? 8.0 : 4.0;
    const double q1 = small_bound(p);
    return (uint64_t)(3.0 * esz * pi_hi + 16.0 * q1 + (1u << 20));
}

static int tables_build(pg::Tables &T, const pg_job_params &p, cudaStream_t st) {
    // ---- K = P#/d
    std::vector<uint32_t> upto_p = host_primes(p.p);
    T.K.assign(1, 1);
    for (uint32_t q : upto_p) big_mul_u32(T.K, q);
    if (big_divmod_u32(T.K, p.d) != 0) return fail(PG_ERR_ARG, "d=%u does not divide %u#", p.d, p.p);
    if (big_bits(T.K) < 2) return fail(PG_ERR_ARG, "K = %u#/%u <= 1", p.p, p.d);
    T.kbits = big_bits(T.K);
    if (T.K.size() > PG_MAX_WORDS - 4) return fail(PG_ERR_UNSUPPORTED, "K has %u bits", T.kbits);
    T.k_log = big_log(T.K);
    // ---- small primes, trial primes, K-primes
    const uint32_t host_lim = std::max<uint32_t>(T.q1, 1700);  // >= TRIAL_PRIMES odd primes
    std::vector<uint32_t> sp = host_primes(host_lim);
    std::vector<uint32_t> sq, sr, tq;
    std::vector<uint64_t> sbar;
    for (uint32_t q : sp) {
        if (q == 2) continue;
        const uint32_t c = big_mod_u32(T.K, q);
        const uint32_t inv2 = (q + 1) / 2;
        const uint32_t r = (uint32_t)((uint64_t)((q - c) % q) * inv2 % q);  // -(K mod q)/2 mod q
        if (tq.size() < TRIAL_PRIMES) {
            tq.push_back(q);
            T.tr.push_back(r);
        }
        if (q <= p.p && c == 0) {
            T.kprimes.push_back(q);
            continue;
        }
        if (q <= T.q1 && q <= p.max_prime) {  // odd d-primes and (P, q1]
            sq.push_back(q);
            sr.push_back(r);
            sbar.push_back(~0ull / q);
        }
    }
    T.nsmall = (uint32_t)sq.size();
    for (uint32_t q : sq) {
        T.n32 += q < 32;
        T.n256 += q < 256;
    }
    int rc;
    if ((rc = dalloc(T.bytes, &T.d_sq, sq.size())) || (rc = dalloc(T.bytes, &T.d_sr, sr.size())) ||
        (rc = dalloc(T.bytes, &T.d_sbar, sbar.size())) || (rc = dalloc(T.bytes, &T.d_tq, TRIAL_PRIMES)))
        return rc;
    if (!sq.empty()) {
        PG_CUDA(cudaMemcpyAsync(T.d_sq, sq.data(), sq.size() * 4, cudaMemcpyHostToDevice, st));
        PG_CUDA(cudaMemcpyAsync(T.d_sr, sr.data(), sr.size() * 4, cudaMemcpyHostToDevice, st));
        PG_CUDA(cudaMemcpyAsync(T.d_sbar, sbar.data(), sbar.size() * 8, cudaMemcpyHostToDevice, st));
    }
    PG_CUDA(cudaMemcpyAsync(T.d_tq, tq.data(), tq.size() * 4, cudaMemcpyHostToDevice, st));
    PG_CUDA(cudaStreamSynchronize(st));  // host vectors die at return
    // ---- large primes (q1, max_prime] on the device
    T.np = 0;
    if (p.max_prime > T.q1) {
        T.wide = p.max_prime >= (1ull << 32);
        const uint32_t root = (uint32_t)std::sqrt((double)p.max_prime) + 2;
        std::vector<uint32_t> base;
        for (uint32_t q : host_primes(root))
            if (q != 2) base.push_back(q);
        const uint64_t v_first = ((uint64_t)T.q1 + 1) | 1ull;
        const uint64_t seg_span = 2ull * (1u << 18);
        const uint64_t nseg64 = (p.max_prime - v_first) / seg_span + 1;
        if (nseg64 > 0x7fffffff) return fail(PG_ERR_UNSUPPORTED, "max_prime too large");
        const uint32_t nseg = (uint32_t)nseg64;
        uint32_t *d_base = nullptr, *d_cnt = nullptr, *d_K = nullptr;
        uint64_t *d_off = nullptr;
        uint64_t scratch = 0;
        auto free_scratch = [&]() {
            cudaStreamSynchronize(st);
            cudaFree(d_base);
            cudaFree(d_cnt);
            cudaFree(d_off);
            cudaFree(d_K);
        };
        if ((rc = dalloc(scratch, &d_base, base.size())) || (rc = dalloc(scratch, &d_cnt, nseg)) ||
            (rc = dalloc(scratch, &d_off, nseg)) || (rc = dalloc(scratch, &d_K, T.K.size()))) {
            free_scratch();
            return rc;
        }
        cudaError_t e = cudaMemcpyAsync(d_base, base.data(), base.size() * 4, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = launch_prime_count(v_first, p.max_prime, d_base, (uint32_t)base.size(), nseg, d_cnt, st);
        std::vector<uint32_t> cnt(nseg);
        std::vector<uint64_t> off(nseg);
        if (e == cudaSuccess) e = cudaMemcpyAsync(cnt.data(), d_cnt, (size_t)nseg * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            free_scratch();
            return fail(PG_ERR_CUDA, "prime count: %s", cudaGetErrorString(e));
        }
        uint64_t acc = 0;
        for (uint32_t i = 0; i < nseg; i++) {
            off[i] = acc;
            acc += cnt[i];
        }
        T.np = acc;
        T.seg_off = off;
        T.seg_v0 = v_first;
        T.seg_span = seg_span;
        const size_t esz = T.wide ? 8 : 4;
        uint8_t *lp = nullptr, *lc = nullptr, *lci = nullptr;
        if ((rc = dalloc(T.bytes, &lp, acc * esz)) || (rc = dalloc(T.bytes, &lc, acc * esz)) ||
            (rc = dalloc(T.bytes, &lci, acc * esz))) {
            cudaFree(lp);
            cudaFree(lc);
            cudaFree(lci);
            free_scratch();
            return fail(PG_ERR_NOMEM, "prime table of %llu primes", (unsigned long long)acc);
        }
        T.d_lp = lp;
        T.d_lc = lc;
        T.d_lcinv = lci;
        e = cudaMemcpyAsync(d_off, off.data(), (size_t)nseg * 8, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = launch_prime_write(v_first, p.max_prime, d_base, (uint32_t)base.size(), nseg, d_off, T.d_lp, T.wide, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_K, T.K.data(), T.K.size() * 4, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = launch_prime_tables(d_K, (uint32_t)T.K.size(), T.np, T.d_lp, T.d_lc, T.d_lcinv, T.wide, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        // order each segment's primes by the modular search's Euclid depth (the
        // table is used unordered if the extra copy does not fit)
        if (e == cudaSuccess) {
            uint8_t *op = nullptr, *oc = nullptr, *oci = nullptr, *dep = nullptr;
            uint64_t extra = 0;
            if (!dalloc(extra, &op, acc * esz) && !dalloc(extra, &oc, acc * esz) && !dalloc(extra, &oci, acc * esz) &&
                !dalloc(extra, &dep, acc)) {
                e = launch_prime_reorder(acc, nseg, d_off, T.d_lp, T.d_lc, T.d_lcinv, op, oc, oci, dep, T.wide, st);
                if (e == cudaSuccess) e = cudaStreamSynchronize(st);
                if (e == cudaSuccess) {  // keep the ordered copies, free the others below
                    void *old[3] = {T.d_lp, T.d_lc, T.d_lcinv};
                    T.d_lp = op;
                    T.d_lc = oc;
                    T.d_lcinv = oci;
                    op = (uint8_t *)old[0];
                    oc = (uint8_t *)old[1];
                    oci = (uint8_t *)old[2];
                }
            }
            g_last_error.clear();
            cudaFree(op);  // the unordered copies (or the unused new ones)
            cudaFree(oc);
            cudaFree(oci);
            cudaFree(dep);
        }
        free_scratch();
        if (e != cudaSuccess) return fail(PG_ERR_CUDA, "prime tables: %s", cudaGetErrorString(e));
    }
    return PG_OK;
}

int pg::tables_get(pg_ctx *c, const pg_job_params &p, std::shared_ptr<Tables> &out) {
    const uint32_t q1 = small_bound(p);
    std::lock_guard<std::mutex> lock(c->tables_mu);
    auto &v = c->tables;
    v.erase(std::remove_if(v.begin(), v.end(), [](const std::weak_ptr<Tables> &w) { return w.expired(); }), v.end());
    for (auto &w : v) {
        std::shared_ptr<Tables> t = w.lock();
        if (t && t->p == p.p && t->d == p.d && t->max_prime == p.max_prime && t->q1 == q1) {
            out = t;
            return PG_OK;
        }
    }
    const auto t0 = std::chrono::steady_clock::now();
    auto t = std::make_shared<Tables>();
    t->device = c->device;
    t->p = p.p;
    t->d = p.d;
    t->max_prime = p.max_prime;
    t->q1 = q1;
    int rc = tables_build(*t, p, c->stream);
    if (rc) return rc;  // t frees what it holds
    t->setup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    v.push_back(t);
    out = t;
    return PG_OK;
}

// ================================================================ slots

int pg::slot_alloc(Slot &s, uint64_t nm_cap, uint64_t nodd_cap, uint64_t bm_cap, uint64_t list_cap,
                   uint32_t win_cap) {
    s.nm_cap = nm_cap;
    s.nodd_cap = nodd_cap;
    s.bm_cap = bm_cap;
    s.list_cap = list_cap;
    s.win_cap = win_cap;
    const uint64_t S = 2 * nm_cap;
    uint64_t &b = s.bytes;
    int rc;
    if ((rc = dalloc(b, &s.d_ms, nm_cap)) || (rc = dalloc(b, &s.d_wid, nm_cap)) ||
        (rc = dalloc(b, &s.d_rank, nodd_cap)) || (rc = dalloc(b, &s.d_bitmaps, bm_cap)) ||
        (rc = dalloc(b, &s.d_lists, list_cap)) || (rc = dalloc(b, &s.d_counts, S)) || (rc = dalloc(b, &s.d_found, S)) ||
        (rc = dalloc(b, &s.d_kstart, S)) || (rc = dalloc(b, &s.d_knext, S)) || (rc = dalloc(b, &s.d_gaps, S)) ||
        (rc = dalloc(b, &s.d_act0, S)) || (rc = dalloc(b, &s.d_act1, S)) || (rc = dalloc(b, &s.d_redo, S)) ||
        (rc = dalloc(b, &s.d_conf, S)) ||
        (rc = dalloc(b, &s.d_sc, 1)) || (rc = dalloc(b, &s.d_win, win_cap)))
        return rc;
    PG_CUDA(cudaMallocHost((void **)&s.h_sc, sizeof(Scalars)));
    PG_CUDA(cudaMallocHost((void **)&s.h_ms, std::max<uint64_t>(nm_cap, 1) * 8));
    PG_CUDA(cudaMallocHost((void **)&s.h_wid, std::max<uint64_t>(nm_cap, 1) * 2));
    PG_CUDA(cudaMallocHost((void **)&s.h_rank, std::max<uint64_t>(nodd_cap, 1) * 4));
    PG_CUDA(cudaMallocHost((void **)&s.h_gaps, std::max<uint64_t>(S, 1) * 4));
    PG_CUDA(cudaMallocHost((void **)&s.h_win, (size_t)std::max<uint32_t>(win_cap, 1) * sizeof(WinInfo)));
    for (auto &e : s.ev) PG_CUDA(cudaEventCreate(&e));
    PG_CUDA(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
    return PG_OK;
}

void pg::slot_free(Slot &s) {
    if (s.st) cudaStreamSynchronize(s.st);
    void *ptrs[] = {s.d_ms,   s.d_wid,  s.d_rank, s.d_bitmaps, s.d_lists, s.d_counts, s.d_found, s.d_kstart,
                    s.d_knext, s.d_gaps, s.d_act0, s.d_act1,    s.d_redo,  s.d_conf,   s.d_sc,     s.d_win};
    for (void *p : ptrs) cudaFree(p);
    void *hptrs[] = {s.h_sc, s.h_ms, s.h_wid, s.h_rank, s.h_gaps, s.h_win, (void *)s.h_stop};
    for (void *p : hptrs) cudaFreeHost(p);
    for (auto &e : s.ev)
        if (e) cudaEventDestroy(e);
    if (s.gexec) cudaGraphExecDestroy(s.gexec);
    if (s.st) cudaStreamDestroy(s.st);
    s = Slot();
}

void pg::slot_reset(Slot &s) {
    s.parts.clear();
    s.nm = 0;
    s.nodd = 0;
    s.L = 0;
    s.stride = 0;
    s.ext_window = 0;
    s.confirm = false;
    s.fin_active = false;
    s.sst = pg_search_stats{};
}

bool pg::slot_fits(const Slot &s, const pg_job *j, uint64_t nm, uint64_t nodd) {
    if (s.parts.size() >= s.win_cap) return false;
    if (!s.parts.empty() && (j->L != s.L || j->prm.ext_window != s.ext_window)) return false;
    if (s.nm + nm > s.nm_cap || s.nodd + nodd > s.nodd_cap) return false;
    if (nm * j->W > s.bm_cap) return false;
    const uint64_t stride = std::max(s.stride, j->cap);
    return 2 * (s.nm + nm) * stride <= s.list_cap;
}

int pg::slot_add(Slot &s, pg_job *j, uint64_t m_start, uint64_t m_inc) {
    const pg_job_params &p = j->prm;
    if (m_inc == 0) return fail(PG_ERR_ARG, "m_inc must be > 0");
    if (m_start == 0) return fail(PG_ERR_ARG, "m_start must be > 0");
    if (m_start + m_inc - 1 > p.max_m) return fail(PG_ERR_ARG, "m beyond max_m");
    WinPart w;
    w.job = j;
    w.m0 = m_start | 1ull;
    const uint64_t end = m_start + m_inc;
    w.nodd = end > w.m0 ? (end - w.m0 + 1) / 2 : 0;
    w.m_off = s.nm;
    w.odd_off = s.nodd;
    if (s.parts.size() >= s.win_cap || s.nodd + w.nodd > s.nodd_cap) return SLOT_FULL;
    const uint16_t wid = (uint16_t)s.parts.size();
    // m coprime to d: odd m stepping by 2 walk the residues mod d
    const uint8_t *cop = j->coprime.data();
    uint32_t rm = (uint32_t)(w.m0 % p.d), r = 0;
    int32_t *rank = s.h_rank + w.odd_off;
    for (uint64_t jj = 0; jj < w.nodd; jj++) {
        if (cop[rm]) {
            if (s.nm + r >= s.nm_cap) return SLOT_FULL;
            s.h_ms[s.nm + r] = w.m0 + 2 * jj;
            s.h_wid[s.nm + r] = wid;
            rank[jj] = (int32_t)r++;
        } else {
            rank[jj] = -1;
        }
        rm += 2;
        if (rm >= p.d) rm -= p.d;
    }
    w.nm = r;
    if (!slot_fits(s, j, w.nm, w.nodd)) return SLOT_FULL;
    s.h_win[wid] = j->win;
    if (s.parts.empty()) {
        s.L = j->L;
        s.ext_window = p.ext_window;
    }
    s.stride = std::max(s.stride, j->cap);
    s.confirm = s.confirm || j->win.confirm_rounds >= 2;
    s.nm += w.nm;
    s.nodd += w.nodd;
    s.parts.push_back(w);
    return PG_OK;
}

// prime-table index of the first segment starting at or above value v
static uint64_t table_index_at(const pg::Tables &T, double v) {
    if (v <= (double)T.seg_v0) return 0;
    const double s = std::ceil((v - (double)T.seg_v0) / (double)T.seg_span);
    if (s >= (double)T.seg_off.size()) return T.np;
    return T.seg_off[(size_t)s];
}

// First prime-table index sieved by modular search rather than by stepping
// every Y.  The search needs p > 2 sly + 1 (one hit per m); by default every
// such prime is searched (with the hit walk, stepping is slower at any split
// on the P=503 window); search_hits > 0 keeps primes expecting at least that
// many hits, nodd * (2 sly + 1) / p, on the stepping kernel.
static uint64_t large_split(const pg_job *j, uint64_t nodd) {
    const pg::Tables &T = *j->T;
    if (T.np == 0) return 0;
    const uint64_t min_split = table_index_at(T, 2.0 * j->sly + 2);
    if (j->prm.flags & PG_JOB_LARGE_STEP) return T.np;
    if ((j->prm.flags & PG_JOB_LARGE_SEARCH) || j->prm.search_hits == 0) return min_split;
    const double hits = (double)j->prm.search_hits;
    return std::max(min_split, table_index_at(T, (double)nodd * (2.0 * j->sly + 1) / hits));
}

// Bands of the segmented large-prime kernel for a window of nodd odd m: the
// primes with walk steps from max(split, walk_first) up to those expecting
// about SEG_HITS hits in the window, table segment by table segment (primes
// of one segment lie within 2^19 of each other), each cut into the power of
// two of segments that leaves about SEG_HITS expected hits per (prime,
// segment) item at the segment's smallest prime; neighbouring segments with
// the same count share a band (all bands of a window run in one launch).
// Returns the first prime index left to the one-thread-per-prime kernel.
static uint64_t seg_bands(const pg_job *j, uint64_t split, uint64_t nodd, SegBand *bands, int *nb) {
    *nb = 0;
    const pg::Tables &T = *j->T;
    const double width = 2.0 * j->sly + 1;
    const uint64_t lo = std::max(split, j->walk_first);
    const uint64_t hi = std::min(j->walk_first + j->walk_count, table_index_at(T, (double)nodd * width / SEG_HITS));
    if (!j->walk_count || lo >= hi) return split;
    const size_t nseg_tab = T.seg_off.size();
    for (size_t s = 0; s < nseg_tab; s++) {
        const uint64_t a = std::max<uint64_t>(lo, T.seg_off[s]);
        const uint64_t b = std::min<uint64_t>(hi, s + 1 < nseg_tab ? T.seg_off[s + 1] : T.np);
        if (a >= b) continue;
        const double pmin = std::max((double)T.seg_v0 + (double)s * (double)T.seg_span, (double)T.q1 + 1);
        const double hits = (double)nodd * width / pmin;
        uint32_t nseg = 1;
        while (nseg < 32768 && 2.0 * nseg * SEG_HITS <= hits) nseg *= 2;
        const uint32_t seg_len = (uint32_t)((nodd + nseg - 1) / nseg);
        SegBand *last = *nb ? &bands[*nb - 1] : nullptr;
        if (last && last->first + last->count == a && (last->nseg == nseg || *nb == MAX_SEG_BANDS)) {
            last->count = b - last->first;  // extends the band (a full list keeps its segment count)
            continue;
        }
        bands[(*nb)++] = SegBand{a, b - a, nseg, seg_len};
    }
    return hi;
}

// sieve of one window of the slot into its rows of lists (compact) or into
// the bitmap rows (the slot's first window only)
static int run_sieve(Slot &s, const WinPart &w, bool compact) {
    const pg_job *j = w.job;
    const pg::Tables &T = *j->T;
    if (j->ready) PG_CUDA(cudaStreamWaitEvent(s.st, j->ready, 0));
    PG_CUDA(cudaMemsetAsync(s.d_bitmaps, 0, (size_t)w.nm * j->W * 4, s.st));
    LargeArgs la{};
    la.sly = j->sly;
    la.words = j->W;
    la.m0 = w.m0;
    la.nodd = w.nodd;
    la.rank = s.d_rank + w.odd_off;
    la.bitmaps = s.d_bitmaps;
    la.np = T.np;
    la.p = T.d_lp;
    la.cinv = T.d_lcinv;
    la.c = T.d_lc;
    la.wheel = j->d_wheel;
    la.walk = j->d_walk;
    la.walk_first = j->walk_first;
    la.walk_end = j->walk_first + j->walk_count;
    const uint64_t split = large_split(j, w.nodd);
    SegBand bands[MAX_SEG_BANDS];
    int nb = 0;
    const uint64_t search_first = seg_bands(j, split, w.nodd, bands, &nb);
    PG_CUDA(launch_sieve_large(la, T.wide, split, bands, nb, search_first, s.st));
    s.sst.kernel_launches += (split > 0) + (nb > 0) + (search_first < T.np);
    SieveArgs sa{};
    sa.sly = j->sly;
    sa.words = j->W;
    sa.cap = s.stride;
    sa.m0 = w.m0;
    sa.nodd = w.nodd;
    sa.nm = w.nm;
    sa.ms = s.d_ms + w.m_off;
    sa.rank = s.d_rank + w.odd_off;
    sa.bitmaps = s.d_bitmaps;
    sa.wheel = j->d_wheel;
    sa.sq = T.d_sq;
    sa.sr = T.d_sr;
    sa.sbar = T.d_sbar;
    sa.nsmall = T.nsmall;
    sa.n32 = T.n32;
    sa.n256 = T.n256;
    sa.lists = s.d_lists + (size_t)2 * w.m_off * s.stride;
    sa.counts = s.d_counts + (size_t)2 * w.m_off;
    sa.max_count = &s.d_sc->max_count;
    sa.survivors = &s.d_sc->survivors;
    PG_CUDA(launch_sieve_small(sa, compact, s.st));
    s.sst.kernel_launches++;
    return PG_OK;
}

static int slot_upload(Slot &s) {
    if (s.nm) PG_CUDA(cudaMemcpyAsync(s.d_ms, s.h_ms, (size_t)s.nm * 8, cudaMemcpyHostToDevice, s.st));
    if (s.nm && s.parts.size() > 1)
        PG_CUDA(cudaMemcpyAsync(s.d_wid, s.h_wid, (size_t)s.nm * 2, cudaMemcpyHostToDevice, s.st));
    if (s.nodd) PG_CUDA(cudaMemcpyAsync(s.d_rank, s.h_rank, (size_t)s.nodd * 4, cudaMemcpyHostToDevice, s.st));
    PG_CUDA(cudaMemcpyAsync(s.d_win, s.h_win, s.parts.size() * sizeof(WinInfo), cudaMemcpyHostToDevice, s.st));
    return PG_OK;
}

static SearchArgs base_args(Slot &s) {
    SearchArgs a{};
    a.win = s.d_win;
    a.wid = s.parts.size() > 1 ? s.d_wid : nullptr;
    a.cap = s.stride;
    a.ntrial = TRIAL_PRIMES;
    a.ms = s.d_ms;
    a.lists = s.d_lists;
    a.counts = s.d_counts;
    a.k_start = s.d_kstart;
    a.found_k = s.d_found;
    a.next_item = &s.d_sc->next_item;
    a.tests = &s.d_sc->tests;
    a.trial_q = s.parts[0].job->T->d_tq;
    return a;
}

// Finalize all sides and queue the copies back; the host reads n_redo in
// slot_finish.
static int enqueue_finalize(Slot &s, SearchArgs &a, uint32_t S) {
    PG_CUDA(cudaMemsetAsync(&s.d_sc->n_redo, 0, 4, s.st));
    PG_CUDA(launch_finalize(s.L, a, S, s.d_gaps, s.d_redo, &s.d_sc->n_redo, &s.d_sc->confirm, s.d_kstart, s.st));
    s.sst.kernel_launches++;
    PG_CUDA(record_ev(s.ev[2], s.st));  // end of the device work (before the copies back)
    PG_CUDA(cudaMemcpyAsync(s.h_gaps, s.d_gaps, (size_t)S * 4, cudaMemcpyDeviceToHost, s.st));
    PG_CUDA(cudaMemcpyAsync(s.h_sc, s.d_sc, sizeof(Scalars), cudaMemcpyDeviceToHost, s.st));
    return PG_OK;
}

// The device work of all windows on the slot's stream (capturable for the
// persistent form; the plain form reads counts back and is not).
static int enqueue_windows(Slot &s, int form, uint32_t flags) {
    int rc;
    const uint32_t S = 2 * s.nm;
    if ((rc = slot_upload(s))) return rc;
    PG_CUDA(record_ev(s.ev[0], s.st));
    PG_CUDA(cudaMemsetAsync(&s.d_sc->max_count, 0, 4, s.st));
    PG_CUDA(cudaMemsetAsync(&s.d_sc->survivors, 0, 8, s.st));
    for (const WinPart &w : s.parts)
        if ((rc = run_sieve(s, w, true))) return rc;
    PG_CUDA(record_ev(s.ev[1], s.st));
    const uint32_t warps = (uint32_t)s.grid * (PERSIST_THREADS / 32);
    PG_CUDA(launch_init_search(S, s.d_found, s.d_kstart, s.d_act0, s.d_conf, s.d_sc, warps, s.st));
    s.sst.kernel_launches++;
    SearchArgs a = base_args(s);
    a.act = s.d_act0;
    a.n_act = S;
    a.ext_max = s.ext_window;
    if (form == PG_SEARCH_PERSISTENT) {
        a.kspan = s.stride + a.ext_max;
        a.max_count = &s.d_sc->max_count;
        a.unresolved = &s.d_sc->unresolved;
        a.active_warps = &s.d_sc->active_warps;
        if (flags & PG_SUBMIT_DRAIN) {
            int sms = 0;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s.parts[0].job->ctx->device);
            const uint32_t d = (flags >> 8) & 0xffu;
            a.drain_lanes = d ? d : 4;
            a.min_warps = (uint32_t)sms;
        }
        if (s.d_stop) {
            *s.h_stop = 0;
            a.stop = s.d_stop;
            a.stopped = &s.d_sc->stopped;
        }
        s.search = a;
        PG_CUDA(record_ev(s.ev[3], s.st));
        PG_CUDA(launch_search_persistent(s.L, a, s.grid, s.st));
        PG_CUDA(record_ev(s.ev[4], s.st));
        s.sst.kernel_launches++;
        s.sst.passes = 1;
    } else {  // one launch per pass, the active-side count read back after each
        PG_CUDA(cudaMemsetAsync(s.d_knext, 0, (size_t)S * 4, s.st));
        uint32_t n_act = S;
        uint32_t *cur = s.d_act0, *nxt = s.d_act1;
        PG_CUDA(record_ev(s.ev[3], s.st));
        while (n_act > 0) {
            a.act = cur;
            a.n_act = n_act;
            PG_CUDA(launch_search_plain(s.L, a, s.d_knext, s.st));
            s.sst.passes++;
            PG_CUDA(cudaMemsetAsync(&s.d_sc->n_out, 0, 4, s.st));
            PG_CUDA(launch_compact_active(cur, n_act, s.d_found, s.d_knext, s.d_counts, a.ext_max, nxt,
                                          &s.d_sc->n_out, s.st));
            s.sst.kernel_launches += 2;
            s.sst.d2h_bytes += 4;
            PG_CUDA(cudaMemcpyAsync(&s.h_sc->n_out, &s.d_sc->n_out, 4, cudaMemcpyDeviceToHost, s.st));
            PG_CUDA(cudaStreamSynchronize(s.st));
            n_act = s.h_sc->n_out;
            std::swap(cur, nxt);
        }
        PG_CUDA(record_ev(s.ev[4], s.st));
        PG_CUDA(launch_iota(s.d_act0, S, s.st));
        s.sst.kernel_launches++;
    }
    a.act = s.d_act0;
    a.n_act = S;
    a.max_count = nullptr;
    a.stop = nullptr;  // finalize reads `stopped` only
    return enqueue_finalize(s, a, S);
}

int pg::slot_enable_preempt(Slot &s) {
    if (s.h_stop) return PG_OK;
    uint32_t *h = nullptr;
    PG_CUDA(cudaHostAlloc((void **)&h, sizeof(uint32_t), cudaHostAllocMapped));
    *h = 0;
    s.h_stop = h;
    PG_CUDA(cudaHostGetDevicePointer((void **)&s.d_stop, h, 0));
    return PG_OK;
}

void pg::slot_preempt(Slot &s) {
    if (s.h_stop) *s.h_stop = 1;
}

int pg::slot_resume(Slot &s) {
    if (!s.d_stop) return fail(PG_ERR_STATE, "slot_resume: the slot has no stop flag");
    *s.h_stop = 0;
    s.fin_active = false;
    const uint32_t S = 2 * s.nm;
    PG_CUDA(cudaMemsetAsync(&s.d_sc->stopped, 0, 4, s.st));
    PG_CUDA(launch_search_persistent(s.L, s.search, s.grid, s.st));
    s.sst.kernel_launches++;
    s.sst.relaunches++;
    SearchArgs a = s.search;
    a.act = s.d_act0;
    a.n_act = S;
    a.max_count = nullptr;
    a.stop = nullptr;
    return enqueue_finalize(s, a, S);
}

int pg::slot_enqueue(Slot &s, int form, uint32_t flags, bool graph) {
    s.fin_active = false;
    s.sst.m_count = s.nm;
    s.sst.h2d_bytes = (uint64_t)s.nm * 8 + (uint64_t)s.nodd * 4 + s.parts.size() * sizeof(WinInfo) +
                      (s.parts.size() > 1 ? (uint64_t)s.nm * 2 : 0);
    if (s.nm == 0) return PG_OK;
    s.grid = search_grid(s.L, s.parts[0].job->ctx->device);
    const uint32_t wps = (flags >> 16) & 0xffu;  // warps per SM cap
    if (wps) s.grid = std::min(s.grid, s.parts[0].job->ctx->sms * (int)wps * 32 / PERSIST_THREADS);
    if (form == PG_SEARCH_PLAIN || !graph) return enqueue_windows(s, form, flags);
    // The persistent form's whole window (upload, sieves, search, finalize,
    // copies back) is captured as one CUDA graph and launched once; the slot
    // keeps the instantiated graph and updates it in place for the next window.
    PG_CUDA(cudaStreamBeginCapture(s.st, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_windows(s, form, flags);
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(s.st, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (ec != cudaSuccess) return fail(PG_ERR_CUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(ec));
    if (s.gexec) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(s.gexec, g, &info) != cudaSuccess) {
            cudaGetLastError();
            cudaGraphExecDestroy(s.gexec);
            s.gexec = nullptr;
        }
    }
    cudaError_t ei = cudaSuccess;
    if (!s.gexec) ei = cudaGraphInstantiate(&s.gexec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return fail(PG_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(ei));
    PG_CUDA(cudaGraphLaunch(s.gexec, s.st));
    s.sst.graph_launches = 1;
    return PG_OK;
}

// Continues sides without a prime within sl + ext_window on the device with
// 4x larger extension windows; once every side has a prime, confirms the
// primes of large gaps (windows with confirm_rounds >= 2) and continues the
// sides whose prime failed from their next candidate.  Then reads the timings.
// Each round is queued on the slot's stream; its results (n_redo, gaps) come
// back with the Scalars copy, read after the stream is idle.
int pg::slot_finish(Slot &s, bool wait) {
    const uint32_t S = 2 * s.nm;
    while (true) {
        PG_CUDA(cudaStreamSynchronize(s.st));  // no wait when the caller saw the stream idle
        if (s.nm == 0) return PG_OK;
        if (!s.fin_active) {
            if (s.h_sc->stopped) return SLOT_STOPPED;  // preempted before its queue ran out: slot_resume
            s.fin_active = true;
            s.fin_phase = 0;
            s.fin_round = 0;
            s.fin_ext = s.ext_window;
        }
        const uint32_t n_redo = s.h_sc->n_redo;
        if (n_redo == 0 && s.fin_phase == 0 && s.confirm) {  // every side resolved: confirm the large gaps
            SearchArgs c = base_args(s);
            c.act = s.d_act0;  // 0 .. S-1
            c.n_act = S;
            PG_CUDA(cudaMemsetAsync(&s.d_sc->n_redo, 0, 4, s.st));
            PG_CUDA(launch_confirm(s.L, c, s.d_gaps, s.d_conf, s.d_redo, &s.d_sc->n_redo, &s.d_sc->confirm,
                                   s.d_kstart, s.st));
            s.sst.kernel_launches++;
            PG_CUDA(record_ev(s.ev[2], s.st));
            PG_CUDA(cudaMemcpyAsync(s.h_gaps, s.d_gaps, (size_t)S * 4, cudaMemcpyDeviceToHost, s.st));
            PG_CUDA(cudaMemcpyAsync(s.h_sc, s.d_sc, sizeof(Scalars), cudaMemcpyDeviceToHost, s.st));
            s.sst.d2h_bytes += 4;
            s.fin_phase = 1;
            if (!wait) return SLOT_PENDING;
            continue;
        }
        if (n_redo == 0) break;
        if (s.fin_round >= 24) {
            s.fin_active = false;
            return fail(PG_ERR_STATE, "pg_search: %u sides unresolved after %u extension positions", n_redo,
                        s.fin_ext);
        }
        SearchArgs a = base_args(s);
        PG_CUDA(cudaMemcpyAsync(s.d_act1, s.d_redo, (size_t)n_redo * 4, cudaMemcpyDeviceToDevice, s.st));
        const uint32_t ext_new = std::min<uint32_t>(s.fin_ext * 4, 1u << 26);
        a.act = s.d_act1;
        a.n_act = n_redo;
        a.ext_max = ext_new;
        a.kspan = s.stride + ext_new;
        a.max_count = nullptr;
        PG_CUDA(cudaMemsetAsync(&s.d_sc->next_item, 0, 8, s.st));
        PG_CUDA(launch_search_persistent(s.L, a, s.grid, s.st));
        s.sst.kernel_launches++;
        s.sst.relaunches++;
        s.sst.extended_sides += n_redo;
        s.fin_ext = ext_new;
        s.fin_round++;
        // finalize the continued sides only (their gaps and a new redo list)
        PG_CUDA(cudaMemsetAsync(&s.d_sc->n_redo, 0, 4, s.st));
        PG_CUDA(launch_finalize(s.L, a, S, s.d_gaps, s.d_redo, &s.d_sc->n_redo, &s.d_sc->confirm, s.d_kstart, s.st));
        s.sst.kernel_launches++;
        PG_CUDA(record_ev(s.ev[2], s.st));
        PG_CUDA(cudaMemcpyAsync(s.h_gaps, s.d_gaps, (size_t)S * 4, cudaMemcpyDeviceToHost, s.st));
        PG_CUDA(cudaMemcpyAsync(s.h_sc, s.d_sc, sizeof(Scalars), cudaMemcpyDeviceToHost, s.st));
        s.sst.d2h_bytes += 4;
        s.fin_phase = 0;
        if (!wait) return SLOT_PENDING;
    }
    s.fin_active = false;
    s.sst.d2h_bytes += (uint64_t)S * 4 + sizeof(Scalars);
    float t_sieve = 0, t_prp = 0, t_kernel = 0;
    if (cudaEventElapsedTime(&t_sieve, s.ev[0], s.ev[1]) != cudaSuccess) t_sieve = 0;
    if (cudaEventElapsedTime(&t_prp, s.ev[1], s.ev[2]) != cudaSuccess) t_prp = 0;
    if (cudaEventElapsedTime(&t_kernel, s.ev[3], s.ev[4]) != cudaSuccess) t_kernel = 0;
    cudaGetLastError();  // a failed timing read must not surface in a later call
    s.sst.search_kernel_ms = t_kernel;
    s.sst.sieve_ms = t_sieve;
    s.sst.prp_ms = t_prp;
    s.sst.total_ms = t_sieve + t_prp;
    s.sst.prp_tests = s.h_sc->tests;
    s.sst.confirm_tests = s.h_sc->confirm;
    s.sst.survivors = s.h_sc->survivors;
    return PG_OK;
}

// ================================================================= jobs

extern "C" uint64_t pg_count_m(uint64_t m_start, uint64_t m_inc, uint32_t d) {
    uint64_t c = 0;
    for (uint64_t m = m_start; m < m_start + m_inc; m++) c += gcd64(m, d) == 1;
    return c;
}

static void job_free(pg_job *j) {
    if (!j) return;
    cudaSetDevice(j->ctx->device);
    cudaStreamSynchronize(j->ctx->stream);
    if (j->ready) {
        cudaEventSynchronize(j->ready);
        cudaEventDestroy(j->ready);
    }
    for (auto &s : j->slot) slot_free(s);
    cudaFree(j->d_wheel);
    cudaFree(j->d_walk);
    delete j;  // drops this job's reference to the shared tables
}

extern "C" int pg_job_destroy(pg_job *j) {
    job_free(j);
    return PG_OK;
}

static int job_build(pg_job *j) {
    const pg_job_params &p = j->prm;
    int rc = tables_get(j->ctx, p, j->T);
    if (rc) return rc;
    const pg::Tables &T = *j->T;
    // every candidate must exceed max_prime (divisible then means composite)
    if (T.kbits <= 64) {
        uint64_t kv = 0;
        for (size_t i = T.K.size(); i-- > 0;) kv = (kv << 32) | T.K[i];
        if (kv <= p.max_prime + 2ull * p.sl + 2) return fail(PG_ERR_ARG, "K too small for max_prime and sl");
    }
    // ---- limbs of the PRP operands: N < K * (max_m + 1)
    const uint32_t nbits = T.kbits + bitlen64(p.max_m + 1);
    j->L = pick_layout(nbits, p.tpi);
    if (!j->L)
        return fail(PG_ERR_UNSUPPORTED, "operands of %u bits with tpi=%u are outside the compiled layouts", nbits,
                    p.tpi);
    // ---- geometry, wheel, capacity
    j->sly = p.sl / 2;
    j->W = (2 * j->sly + 1 + 31) / 32;
    std::vector<uint32_t> wheel(j->W, 0);
    auto setb = [&](uint32_t idx) { wheel[idx >> 5] |= 1u << (idx & 31); };
    setb(j->sly);
    for (uint32_t q : T.kprimes)
        for (uint32_t idx = j->sly % q; idx <= 2 * j->sly; idx += q) setb(idx);
    j->cap = 0;
    for (uint32_t y = 1; y <= j->sly; y++) j->cap += !((wheel[(j->sly + y) >> 5] >> ((j->sly + y) & 31)) & 1u);
    if (j->cap == 0) j->cap = 1;
    if ((rc = dalloc(j->own_bytes, &j->d_wheel, j->W))) return rc;
    // Jobs launched without graphs (the server's, created while other launches
    // hold the SMs) do not wait for the device: the wheel goes up on the
    // context's copy-only stream (a pageable copy returns once it is staged),
    // the walk kernel queues behind it on the context's stream, and every
    // launch of the job waits for j->ready on its own stream first.
    const bool async = p.flags & PG_JOB_NO_GRAPH;
    if (async) {
        PG_CUDA(cudaEventCreateWithFlags(&j->ready, cudaEventDisableTiming));
        PG_CUDA(cudaMemcpyAsync(j->d_wheel, wheel.data(), wheel.size() * 4, cudaMemcpyHostToDevice, j->ctx->up));
        PG_CUDA(cudaEventRecord(j->ready, j->ctx->up));
        PG_CUDA(cudaStreamWaitEvent(j->ctx->stream, j->ready, 0));
    } else {
        PG_CUDA(cudaMemcpyAsync(j->d_wheel, wheel.data(), wheel.size() * 4, cudaMemcpyHostToDevice,
                                j->ctx->stream));
        PG_CUDA(cudaStreamSynchronize(j->ctx->stream));
    }
    // ---- per-window constants
    std::memset(&j->win, 0, sizeof j->win);
    std::memcpy(j->win.K, T.K.data(), T.K.size() * 4);
    std::memcpy(j->win.trial_r, T.tr.data(), std::min<size_t>(T.tr.size(), TRIAL_PRIMES) * 4);
    j->win.kwords = (uint32_t)T.K.size();
    j->win.sly = j->sly;
    j->win.rounds = p.rounds;
    j->win.k_log = T.k_log;
    j->win.confirm_merit = p.confirm_merit;
    j->win.confirm_rounds = p.confirm_merit > 0 ? (p.confirm_rounds ? p.confirm_rounds : 16u) : 0u;
    j->coprime.assign(p.d, 0);
    for (uint32_t r = 0; r < p.d; r++) j->coprime[r] = gcd64(r, p.d) == 1;
    // ---- window capacity
    const uint64_t mi = std::max<uint64_t>(p.max_m_inc, 2);
    j->nodd_cap = mi / 2 + 1;
    uint64_t phi = 0;
    for (uint64_t r = 1; r <= p.d; r++) phi += gcd64(r, p.d) == 1;
    j->nm_cap = std::min<uint64_t>(j->nodd_cap, (mi / p.d + 1) * phi);
    if (2 * j->nm_cap >= 0xffffffffull) return fail(PG_ERR_UNSUPPORTED, "max_m_inc too large");
    // ---- walk steps of the large primes below 2^32 for this job's window width
    // (with PG_JOB_COMPACT_WALK only of those expecting >= SEG_HITS hits in the
    // largest window, which the segmented kernel needs)
    if (T.np && !(p.flags & PG_JOB_LARGE_STEP)) {
        const uint64_t first = table_index_at(T, 2.0 * j->sly + 2);
        double pmax = (p.flags & PG_JOB_COMPACT_WALK) ? (double)j->nodd_cap * (2.0 * j->sly + 1) / SEG_HITS
                                                      : 4294967296.0;
        // table_index_at keeps the whole segment holding pmax: with primes above
        // 2^32 in the table, stop a segment early so every kept prime is below 2^32
        if (T.wide) pmax = std::min(pmax, 4294967296.0 - (double)T.seg_span);
        const uint64_t end = table_index_at(T, pmax);
        if (end > first) {
            j->walk_first = first;
            j->walk_count = end - first;
            if ((rc = dalloc(j->own_bytes, &j->d_walk, j->walk_count))) return rc;
            PG_CUDA(launch_walk_consts(T.d_lp, T.d_lc, T.d_lcinv, T.wide, first, j->walk_count, 2 * j->sly,
                                       j->d_walk, j->ctx->stream));
            if (!async) PG_CUDA(cudaStreamSynchronize(j->ctx->stream));
        }
    }
    if (async) PG_CUDA(cudaEventRecord(j->ready, j->ctx->stream));  // after the wheel copy and the walk kernel
    return PG_OK;
}

static int job_slots(pg_job *j) {
    if (j->slots_ready) return PG_OK;
    for (auto &s : j->slot) {
        int rc = slot_alloc(s, j->nm_cap, j->nodd_cap, j->nm_cap * j->W, 2 * j->nm_cap * j->cap, 1);
        if (rc) return rc;
    }
    j->slots_ready = true;
    return PG_OK;
}

int pg::job_create(pg_ctx *c, const pg_job_params &p, pg_job **out) {
    *out = nullptr;
    if (!is_prime_u32(p.p)) return fail(PG_ERR_ARG, "p=%u is not prime", p.p);
    if (p.d == 0 || p.d % 2) return fail(PG_ERR_ARG, "d=%u must be even", p.d);
    if (p.sl < 2 || p.sl / 2 > 65535) return fail(PG_ERR_ARG, "sl=%u outside [2, 131071]", p.sl);
    if (p.max_prime >= (1ull << 40)) return fail(PG_ERR_ARG, "max_prime must be < 2^40");
    if (p.max_m == 0) return fail(PG_ERR_ARG, "max_m must be set");
    if (p.rounds < 1 || p.rounds > 16) return fail(PG_ERR_ARG, "rounds=%u (1..16)", p.rounds);
    if (p.confirm_merit < 0 || !(p.confirm_merit == p.confirm_merit))
        return fail(PG_ERR_ARG, "confirm_merit must be >= 0");
    if (p.confirm_rounds == 1 || p.confirm_rounds > 16)
        return fail(PG_ERR_ARG, "confirm_rounds=%u (2..16, 0 = 16)", p.confirm_rounds);
    PG_CUDA(cudaSetDevice(c->device));
    const auto t0 = std::chrono::steady_clock::now();
    pg_job *j = new pg_job();
    j->ctx = c;
    j->prm = p;
    if (!j->prm.ext_window) j->prm.ext_window = 64;
    int rc = job_build(j);
    if (rc) {
        std::string keep = g_last_error;
        job_free(j);
        g_last_error = keep;
        return rc;
    }
    j->setup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = j;
    return PG_OK;
}

extern "C" int pg_job_create(pg_ctx *c, const pg_job_params *params, pg_job **out) {
    if (!c || !params || !out) return fail(PG_ERR_ARG, "pg_job_create: NULL argument");
    pg_job *j = nullptr;
    int rc = job_create(c, *params, &j);
    if (rc) return rc;
    const auto t0 = std::chrono::steady_clock::now();
    if ((rc = job_slots(j))) {
        std::string keep = g_last_error;
        job_free(j);
        g_last_error = keep;
        return rc;
    }
    j->setup_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = j;
    return PG_OK;
}

extern "C" int pg_job_get_info(const pg_job *j, pg_job_info *info) {
    if (!j || !info) return fail(PG_ERR_ARG, "pg_job_get_info: NULL argument");
    info->k_bits = j->T->kbits;
    info->limbs = layout_words(j->L);
    info->tpi = j->L >> 16 ? j->L >> 16 : 1;
    info->words_per_m = j->W;
    info->side_capacity = j->cap;
    info->num_primes = j->T->np;
    info->num_small = j->T->nsmall;
    info->k_log = j->T->k_log;
    info->setup_seconds = j->setup_s;
    uint64_t b = j->own_bytes + j->T->bytes;
    for (const auto &s : j->slot) b += s.bytes;
    info->device_bytes = b;
    return PG_OK;
}

extern "C" int pg_job_k_words(const pg_job *j, uint32_t *out, uint32_t *nwords) {
    if (!j || !nwords) return fail(PG_ERR_ARG, "pg_job_k_words: NULL argument");
    if (out) std::memcpy(out, j->T->K.data(), j->T->K.size() * 4);
    *nwords = (uint32_t)j->T->K.size();
    return PG_OK;
}

extern "C" void *pg_job_stream(pg_job *j, int slot) {
    if (!j || slot < 0 || slot >= PG_SEARCH_SLOTS) return nullptr;
    return (void *)j->slot[slot].st;
}

// ============================================================== windows

static int slot_idle(Slot &s, const char *who) {
    if (s.busy)
        return fail(PG_ERR_STATE, "%s: window slot holds ticket %llu; pg_search_wait it first", who,
                    (unsigned long long)s.ticket);
    return PG_OK;
}

// the job's window [m_start, m_start + m_inc) alone in slot s
static int job_window(pg_job *j, Slot &s, uint64_t m_start, uint64_t m_inc) {
    if (m_inc == 0) return fail(PG_ERR_ARG, "m_inc must be > 0");
    if (m_inc > std::max<uint64_t>(j->prm.max_m_inc, 2))
        return fail(PG_ERR_ARG, "m_inc=%llu > max_m_inc=%llu", (unsigned long long)m_inc,
                    (unsigned long long)j->prm.max_m_inc);
    slot_reset(s);
    int rc = slot_add(s, j, m_start, m_inc);
    if (rc == SLOT_FULL) return fail(PG_ERR_STATE, "window does not fit its slot");
    return rc;
}

extern "C" int pg_sieve_interval(pg_job *j, uint64_t m_start, uint64_t m_inc, uint64_t *ms, uint32_t *bitmaps) {
    if (!j) return fail(PG_ERR_ARG, "pg_sieve_interval: job is NULL");
    PG_CUDA(cudaSetDevice(j->ctx->device));
    int rc = job_slots(j);
    if (rc) return rc;
    Slot &s = j->slot[0];
    if ((rc = slot_idle(s, "pg_sieve_interval"))) return rc;
    PG_CUDA(cudaStreamSynchronize(s.st));  // pinned staging is reused
    if ((rc = job_window(j, s, m_start, m_inc))) return rc;
    if (s.nm == 0) return PG_OK;
    if ((rc = slot_upload(s))) return rc;
    if ((rc = run_sieve(s, s.parts[0], false))) return rc;
    if (bitmaps) PG_CUDA(cudaMemcpyAsync(bitmaps, s.d_bitmaps, (size_t)s.nm * j->W * 4, cudaMemcpyDeviceToHost, s.st));
    PG_CUDA(cudaStreamSynchronize(s.st));
    if (ms) std::memcpy(ms, s.h_ms, (size_t)s.nm * 8);
    return PG_OK;
}

extern "C" int pg_search_submit(pg_job *j, uint64_t m_start, uint64_t m_inc, int form, uint32_t flags,
                                uint64_t *ticket) {
    if (!j || !ticket) return fail(PG_ERR_ARG, "pg_search_submit: NULL argument");
    if (form != PG_SEARCH_PERSISTENT && form != PG_SEARCH_PLAIN)
        return fail(PG_ERR_ARG, "pg_search_submit: form=%d", form);
    PG_CUDA(cudaSetDevice(j->ctx->device));
    int rc = job_slots(j);
    if (rc) return rc;
    Slot &s = j->slot[j->next_ticket % PG_SEARCH_SLOTS];
    if ((rc = slot_idle(s, "pg_search_submit"))) return rc;
    PG_CUDA(cudaStreamSynchronize(s.st));  // the slot's pinned staging is reused
    if ((rc = job_window(j, s, m_start, m_inc))) return rc;
    s.ticket = j->next_ticket++;
    s.busy = true;
    *ticket = s.ticket;
    rc = slot_enqueue(s, form, flags, !(j->prm.flags & PG_JOB_NO_GRAPH));
    if (rc) s.busy = false;
    return rc;
}

extern "C" int pg_search_wait(pg_job *j, uint64_t ticket, uint64_t *ms, uint32_t *prev_gap, uint32_t *next_gap,
                              pg_search_stats *stats) {
    if (!j) return fail(PG_ERR_ARG, "pg_search_wait: job is NULL");
    PG_CUDA(cudaSetDevice(j->ctx->device));
    Slot &s = j->slot[ticket % PG_SEARCH_SLOTS];
    if (!s.busy || s.ticket != ticket)
        return fail(PG_ERR_STATE, "pg_search_wait: ticket %llu is not in flight", (unsigned long long)ticket);
    s.busy = false;
    int rc = slot_finish(s);
    if (rc) return rc;
    for (uint32_t r = 0; r < s.nm; r++) {
        if (next_gap) next_gap[r] = s.h_gaps[2 * r];
        if (prev_gap) prev_gap[r] = s.h_gaps[2 * r + 1];
    }
    if (ms) std::memcpy(ms, s.h_ms, (size_t)s.nm * 8);
    if (stats) *stats = s.sst;
    return PG_OK;
}

extern "C" int pg_search(pg_job *j, uint64_t m_start, uint64_t m_inc, int form, uint64_t *ms, uint32_t *prev_gap,
                         uint32_t *next_gap, pg_search_stats *stats) {
    uint64_t t = 0;
    int rc = pg_search_submit(j, m_start, m_inc, form, 0, &t);
    if (rc) return rc;
    return pg_search_wait(j, t, ms, prev_gap, next_gap, stats);
}

// ============================================================ autotune

// device time of one search of the window with params p (a warm-up search first)
static int time_params(pg_ctx *c, const pg_job_params &p, uint64_t m_start, uint64_t m_inc, double *ms) {
    pg_job *j = nullptr;
    int rc = pg_job_create(c, &p, &j);
    if (rc) return rc;
    pg_search_stats st{};
    double best = 1e300;
    for (int rep = 0; rep < 3 && rc == PG_OK; rep++) {
        rc = pg_search(j, m_start, m_inc, PG_SEARCH_PERSISTENT, nullptr, nullptr, nullptr, &st);
        if (rep > 0) best = std::min(best, st.total_ms);
    }
    pg_job_destroy(j);
    *ms = best;
    return rc;
}

extern "C" int pg_autotune(pg_ctx *c, const pg_job_params *base, uint64_t m_start, uint64_t m_inc, pg_job_params *best,
                           double *best_ms) {
    if (!c || !base || !best) return fail(PG_ERR_ARG, "pg_autotune: NULL argument");
    pg_job_params p = *base;
    p.max_m_inc = std::max<uint64_t>(p.max_m_inc, m_inc);
    p.max_m = std::max<uint64_t>(p.max_m, m_start + m_inc);
    double top = 1e300;
    pg_job_params winner = p;
    // 1. the shared-memory sieve's prime bound
    const uint32_t smalls[] = {16384, 65536, 262144};
    for (uint32_t v : smalls) {
        if (v > p.max_prime && v != smalls[0]) continue;
        pg_job_params q = p;
        q.small_limit = v;
        double ms = 0;
        int rc = time_params(c, q, m_start, m_inc, &ms);
        if (rc == PG_ERR_UNSUPPORTED) continue;
        if (rc) return rc;
        if (ms < top) {
            top = ms;
            winner = q;
        }
    }
    // 2. threads per number (the operand layout)
    const uint32_t tpis[] = {1, 4, 8};
    const uint32_t keep_tpi = winner.tpi;
    for (uint32_t t : tpis) {
        pg_job_params q = winner;
        q.tpi = t;
        if (t == keep_tpi) continue;
        double ms = 0;
        int rc = time_params(c, q, m_start, m_inc, &ms);
        if (rc == PG_ERR_UNSUPPORTED) continue;  // no layout of that width fits
        if (rc) return rc;
        if (ms < top) {
            top = ms;
            winner = q;
        }
    }
    g_last_error.clear();
    *best = winner;
    if (best_ms) *best_ms = top;
    return PG_OK;
}

// m/s of `reps` passes over [m_start, m_start + m_inc) in windows of `window`
// m, PG_SEARCH_SLOTS in flight, after one warm-up pass (wall clock: the
// windows are device bound)
static int time_pipelined(pg_job *j, uint64_t m_start, uint64_t m_inc, uint64_t window, uint32_t flags,
                          uint32_t reps, double *m_per_sec) {
    const uint64_t nwin = (m_inc + window - 1) / window;
    uint64_t m_done = 0;
    bool timing = false;
    auto t0 = std::chrono::steady_clock::now();
    std::vector<uint64_t> pending;
    int rc = PG_OK;
    auto drain_one = [&]() {
        pg_search_stats st{};
        const int r = pg_search_wait(j, pending.front(), nullptr, nullptr, nullptr, &st);
        pending.erase(pending.begin());
        if (r == PG_OK && timing) m_done += st.m_count;
        return r;
    };
    for (uint32_t it = 0; it < 1 + reps && rc == PG_OK; it++) {
        if (it == 1) {  // the warm-up pass is done: start the clock
            while (!pending.empty() && rc == PG_OK) rc = drain_one();
            if (rc) break;
            timing = true;
            t0 = std::chrono::steady_clock::now();
        }
        for (uint64_t w = 0; w < nwin && rc == PG_OK; w++) {
            if (pending.size() == PG_SEARCH_SLOTS) rc = drain_one();
            if (rc) break;
            uint64_t t = 0;
            const uint64_t inc = std::min(window, m_inc - w * window);
            rc = pg_search_submit(j, m_start + w * window, inc, PG_SEARCH_PERSISTENT, flags, &t);
            if (rc == PG_OK) pending.push_back(t);
        }
    }
    while (!pending.empty()) {
        const int r = drain_one();
        if (rc == PG_OK) rc = r;
    }
    if (rc) return rc;
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *m_per_sec = m_done / std::max(secs, 1e-9);
    return PG_OK;
}

extern "C" int pg_autotune_ex(pg_ctx *c, const pg_job_params *base, uint64_t m_start, uint64_t m_inc, uint32_t flags,
                              uint32_t reps, pg_tune_result *out) {
    if (!c || !base || !out) return fail(PG_ERR_ARG, "pg_autotune_ex: NULL argument");
    if (m_inc == 0) return fail(PG_ERR_ARG, "pg_autotune_ex: m_inc must be > 0");
    if (!reps) reps = 4;
    pg_job_params p = *base;
    p.max_m_inc = std::max<uint64_t>(p.max_m_inc, m_inc);
    p.max_m = std::max<uint64_t>(p.max_m, m_start + m_inc);
    pg_tune_result best{};
    best.params = p;
    best.window_m = m_inc;
    uint32_t settings = 0;
    // times job parameters q with warps cap w and window size win; keeps the best
    auto trial = [&](const pg_job_params &q, uint32_t w, uint64_t win) -> int {
        pg_job *j = nullptr;
        int rc = pg_job_create(c, &q, &j);
        if (rc) return rc;
        double v = 0;
        rc = time_pipelined(j, m_start, m_inc, win, PG_SUBMIT_WARPS_PER_SM(w), reps, &v);
        pg_job_destroy(j);
        if (rc) return rc;
        if (settings++ == 0) best.first_m_per_sec = v;
        if (v > best.m_per_sec) {
            best.m_per_sec = v;
            best.params = q;
            best.warps_per_sm = w;
            best.window_m = win;
        }
        return PG_OK;
    };
    // 1. threads per number
    const uint32_t tpis[] = {0, 1, 4, 8, 16};
    for (uint32_t t : tpis) {
        pg_job_params q = p;
        q.tpi = t;
        const int rc = trial(q, 0, m_inc);
        if (rc == PG_ERR_UNSUPPORTED) continue;  // no layout of that width for this tpi
        if (rc) return rc;
    }
    if (settings == 0) return fail(PG_ERR_UNSUPPORTED, "pg_autotune_ex: no compiled layout fits");
    // 2. the sieve tile's small-prime bound
    const uint32_t smalls[] = {16384, 65536, 262144};
    const pg_job_params after_tpi = best.params;
    for (uint32_t v : smalls) {
        if (v > p.max_prime && v != smalls[0]) continue;
        pg_job_params q = after_tpi;
        if (q.small_limit == v || (q.small_limit == 0 && v == 65536)) continue;  // timed already
        q.small_limit = v;
        const int rc = trial(q, 0, m_inc);
        if (rc == PG_ERR_UNSUPPORTED) continue;
        if (rc) return rc;
    }
    // 3. PRP warps per SM, two windows in flight.  The caps differ by a few
    // per cent, and a sample of one or two windows favours full occupancy
    // (its windows start side by side and end alone), so every cap is timed
    // over at least 8 windows on one job, then the two best once more, and
    // the mean of their two timings decides.
    const uint32_t caps[] = {0, 4, 6, 8, 10, 12};
    const pg_job_params tuned = best.params;
    {
        pg_job *j = nullptr;
        int rc = pg_job_create(c, &tuned, &j);
        if (rc) return rc;
        const uint32_t passes = std::max(2 * reps, 8u);
        std::vector<std::pair<double, uint32_t>> by_cap;
        for (uint32_t w : caps) {
            double v = 0;
            if ((rc = time_pipelined(j, m_start, m_inc, m_inc, PG_SUBMIT_WARPS_PER_SM(w), passes, &v))) break;
            by_cap.push_back({v, w});
            settings++;
        }
        std::sort(by_cap.rbegin(), by_cap.rend());
        for (size_t k = 0; k < 2 && !rc; k++) {
            double v = 0;
            rc = time_pipelined(j, m_start, m_inc, m_inc, PG_SUBMIT_WARPS_PER_SM(by_cap[k].second), passes, &v);
            by_cap[k].first = (by_cap[k].first + v) / 2;
            settings++;
        }
        pg_job_destroy(j);
        if (rc) return rc;
        const size_t k = by_cap[1].first > by_cap[0].first ? 1 : 0;
        best.params = tuned;
        best.warps_per_sm = by_cap[k].second;
        best.m_per_sec = by_cap[k].first;
        best.window_m = m_inc;
    }
    // 4. window size
    if (flags & PG_TUNE_WINDOW) {
        const uint32_t cap = best.warps_per_sm;
        for (uint64_t div : {2ull, 4ull}) {
            if (m_inc / div < 2) break;
            const int rc = trial(tuned, cap, (m_inc + div - 1) / div);
            if (rc) return rc;
        }
    }
    g_last_error.clear();
    best.settings = settings;
    *out = best;
    return PG_OK;
}

// ============================================================= records

extern "C" double pg_merit(double k_log, uint64_t m, uint64_t gap) { return (double)gap / (k_log + std::log((double)m)); }

extern "C" int pg_format_record(char *buf, size_t buflen, uint64_t gap, double merit, uint64_t m, uint32_t p,
                                uint32_t d, uint64_t prev_gap) {
    if (!buf || buflen == 0) return fail(PG_ERR_ARG, "pg_format_record: no buffer");
    const int n = snprintf(buf, buflen, "%llu %.3f %llu * %u# / %u - %llu", (unsigned long long)gap, merit,
                           (unsigned long long)m, p, d, (unsigned long long)prev_gap);
    if (n < 0 || (size_t)n >= buflen) return fail(PG_ERR_ARG, "pg_format_record: buffer too small");
    return n;
}
