// pg_api.cu -- host side of the C ABI (include/primegap.h).
//
// Job set-up builds K = P#/d with a small host bignum (gap_common.cpp:60-65),
// the K-prime wheel and the small-prime tables on the host, and the large
// prime table (every prime in (small_limit, max_prime] with K mod p and
// K^-1 mod p) on the device.  A job has PG_SEARCH_SLOTS window slots, each
// with its own stream and buffers, so consecutive windows overlap on the
// device.  A search of one window runs on its slot's stream:
//   large-prime sieve -> small-prime sieve + survivor lists -> PRP search
//   (persistent or plain) -> finalize/confirm [-> continuation launches]
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

#include "pg_internal.h"

using namespace pg;

// ============================================================== errors

static thread_local std::string g_last_error;

static int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define PG_CUDA(call)                                                                                    \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            return fail(e_ == cudaErrorMemoryAllocation ? PG_ERR_NOMEM : PG_ERR_CUDA, "%s: %s (%s:%d)", \
                        #call, cudaGetErrorString(e_), __FILE__, __LINE__);                              \
    } while (0)

extern "C" const char *pg_last_error(void) { return g_last_error.c_str(); }

void pg::set_error(const char *msg) { g_last_error = msg; }

// Timing events are recorded as external event nodes when the stream is
// being captured, so they keep their timestamps inside a window's graph.
static cudaError_t record_ev(cudaEvent_t e, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t err = cudaStreamIsCapturing(st, &cs);
    if (err != cudaSuccess) return err;
    return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(e, st, cudaEventRecordExternal)
                                               : cudaEventRecord(e, st);
}

extern "C" const char *pg_version(void) { return "primegap-b200 0.2 (sm_100a)"; }

// ======================================================= host bignum (K)

typedef std::vector<uint32_t> Big;  // little-endian words, no leading zeros

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

static uint64_t gcd64(uint64_t a, uint64_t b) {
    while (b) {
        uint64_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}

// ============================================================== objects

struct pg_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    int sms = 0;
    // PRP batch staging
    uint32_t *d_cand = nullptr;
    int32_t *d_res = nullptr;
    size_t cand_cap = 0, res_cap = 0;
};

// One window in flight: its buffers, stream, events and the host state
// needed to finish it.
struct WinSlot {
    cudaStream_t st = nullptr;
    uint64_t *d_ms = nullptr;
    int32_t *d_rank = nullptr;
    uint32_t *d_bitmaps = nullptr;
    uint16_t *d_lists = nullptr;
    uint32_t *d_counts = nullptr, *d_found = nullptr, *d_kstart = nullptr, *d_knext = nullptr, *d_gaps = nullptr;
    uint32_t *d_act0 = nullptr, *d_act1 = nullptr, *d_redo = nullptr;
    Scalars *d_sc = nullptr;
    Scalars *h_sc = nullptr;    // pinned
    uint64_t *h_ms = nullptr;   // pinned
    int32_t *h_rank = nullptr;  // pinned
    uint32_t *h_gaps = nullptr; // pinned
    cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    cudaGraphExec_t gexec = nullptr;  // the persistent form's window graph
    // in-flight state
    bool busy = false;
    uint64_t ticket = 0;
    uint64_t m0 = 0, nodd = 0;
    uint32_t nm = 0;
    pg_search_stats sst{};
};

struct pg_job {
    pg_ctx *ctx = nullptr;
    pg_job_params prm{};
    Big K;
    uint32_t kbits = 0, L = 0, sly = 0, W = 0, cap = 0;
    double k_log = 0, setup_s = 0;
    uint32_t q1 = 0;  // small/large split: small primes are <= q1
    // tables
    uint32_t *d_wheel = nullptr;
    uint32_t *d_sq = nullptr, *d_sr = nullptr;
    uint64_t *d_sbar = nullptr;
    uint32_t nsmall = 0;
    uint32_t *d_tq = nullptr, *d_tr = nullptr;
    void *d_lp = nullptr, *d_lc = nullptr, *d_lcinv = nullptr;
    uint64_t np = 0;
    bool wide = false;
    // prime table index of each sieve segment (segment s starts at value seg_v0 + s * seg_span)
    std::vector<uint64_t> seg_off;
    uint64_t seg_v0 = 0, seg_span = 0;
    // window slots
    uint64_t nm_cap = 0, nodd_cap = 0;
    WinSlot slot[PG_SEARCH_SLOTS];
    uint64_t next_ticket = 0;
    uint64_t dev_bytes = 0;
    int grid = 0;
};

template <typename T>
static int dalloc(pg_job *j, T **p, size_t count) {
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = cudaMalloc((void **)p, bytes);
    if (e != cudaSuccess)
        return fail(e == cudaErrorMemoryAllocation ? PG_ERR_NOMEM : PG_ERR_CUDA, "cudaMalloc(%zu): %s", bytes,
                    cudaGetErrorString(e));
    j->dev_bytes += bytes;
    return PG_OK;
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
    if (e != cudaSuccess) {
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

// ================================================================= jobs

extern "C" uint64_t pg_count_m(uint64_t m_start, uint64_t m_inc, uint32_t d) {
    uint64_t c = 0;
    for (uint64_t m = m_start; m < m_start + m_inc; m++) c += gcd64(m, d) == 1;
    return c;
}

static void slot_free(WinSlot &s) {
    if (s.st) cudaStreamSynchronize(s.st);
    void *ptrs[] = {s.d_ms,   s.d_rank,   s.d_bitmaps, s.d_lists, s.d_counts, s.d_found, s.d_kstart,
                    s.d_knext, s.d_gaps,  s.d_act0,    s.d_act1,  s.d_redo,   s.d_sc};
    for (void *p : ptrs) cudaFree(p);
    cudaFreeHost(s.h_sc);
    cudaFreeHost(s.h_ms);
    cudaFreeHost(s.h_rank);
    cudaFreeHost(s.h_gaps);
    for (auto &e : s.ev)
        if (e) cudaEventDestroy(e);
    if (s.gexec) cudaGraphExecDestroy(s.gexec);
    if (s.st) cudaStreamDestroy(s.st);
}

static void job_free(pg_job *j) {
    if (!j) return;
    cudaSetDevice(j->ctx->device);
    cudaStreamSynchronize(j->ctx->stream);
    for (auto &s : j->slot) slot_free(s);
    void *ptrs[] = {j->d_wheel, j->d_sq, j->d_sr, j->d_sbar, j->d_tq, j->d_tr, j->d_lp, j->d_lc, j->d_lcinv};
    for (void *p : ptrs) cudaFree(p);
    delete j;
}

extern "C" int pg_job_destroy(pg_job *j) {
    job_free(j);
    return PG_OK;
}

static uint32_t bitlen64(uint64_t v) { return v ? 64 - __builtin_clzll(v) : 0; }

static int slot_alloc(pg_job *j, WinSlot &s) {
    const uint64_t S = 2 * j->nm_cap;
    int rc;
    if ((rc = dalloc(j, &s.d_ms, j->nm_cap)) || (rc = dalloc(j, &s.d_rank, j->nodd_cap)) ||
        (rc = dalloc(j, &s.d_bitmaps, j->nm_cap * j->W)) || (rc = dalloc(j, &s.d_lists, S * j->cap)) ||
        (rc = dalloc(j, &s.d_counts, S)) || (rc = dalloc(j, &s.d_found, S)) || (rc = dalloc(j, &s.d_kstart, S)) ||
        (rc = dalloc(j, &s.d_knext, S)) || (rc = dalloc(j, &s.d_gaps, S)) || (rc = dalloc(j, &s.d_act0, S)) ||
        (rc = dalloc(j, &s.d_act1, S)) || (rc = dalloc(j, &s.d_redo, S)) || (rc = dalloc(j, &s.d_sc, 1)))
        return rc;
    PG_CUDA(cudaMallocHost((void **)&s.h_sc, sizeof(Scalars)));
    PG_CUDA(cudaMallocHost((void **)&s.h_ms, j->nm_cap * 8));
    PG_CUDA(cudaMallocHost((void **)&s.h_rank, j->nodd_cap * 4));
    PG_CUDA(cudaMallocHost((void **)&s.h_gaps, S * 4));
    for (auto &e : s.ev) PG_CUDA(cudaEventCreate(&e));
    PG_CUDA(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
    return PG_OK;
}

static int job_build(pg_job *j) {
    const pg_job_params &p = j->prm;
    cudaStream_t st = j->ctx->stream;
    // ---- K = P#/d
    std::vector<uint32_t> upto_p = host_primes(p.p);
    j->K.assign(1, 1);
    for (uint32_t q : upto_p) big_mul_u32(j->K, q);
    if (big_divmod_u32(j->K, p.d) != 0) return fail(PG_ERR_ARG, "d=%u does not divide %u#", p.d, p.p);
    if (big_bits(j->K) < 2) return fail(PG_ERR_ARG, "K = %u#/%u <= 1", p.p, p.d);
    j->kbits = big_bits(j->K);
    if (j->K.size() > PG_MAX_WORDS - 4) return fail(PG_ERR_UNSUPPORTED, "K has %u bits", j->kbits);
    j->k_log = big_log(j->K);
    // every candidate must exceed max_prime (divisible then means composite)
    if (j->kbits <= 64) {
        uint64_t kv = 0;
        for (size_t i = j->K.size(); i-- > 0;) kv = (kv << 32) | j->K[i];
        if (kv <= p.max_prime + 2ull * p.sl + 2) return fail(PG_ERR_ARG, "K too small for max_prime and sl");
    }
    // ---- limbs of the PRP operands: N < K * (max_m + 1)
    const uint32_t nbits = j->kbits + bitlen64(p.max_m + 1);
    j->L = pick_layout(nbits, p.tpi);
    if (!j->L)
        return fail(PG_ERR_UNSUPPORTED, "operands of %u bits with tpi=%u are outside the compiled layouts", nbits,
                    p.tpi);
    // ---- geometry
    j->sly = p.sl / 2;
    j->W = (2 * j->sly + 1 + 31) / 32;
    // ---- small primes, wheel, capacity
    j->q1 = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(p.small_limit ? p.small_limit : 65536u, p.p), p.max_prime);
    if (j->q1 < p.p) j->q1 = p.p;
    const uint32_t host_lim = std::max<uint32_t>(j->q1, 1700);  // >= TRIAL_PRIMES odd primes
    std::vector<uint32_t> sp = host_primes(host_lim);
    std::vector<uint32_t> kprimes, sq, sr, tq, tr;
    std::vector<uint64_t> sbar;
    for (uint32_t q : sp) {
        if (q == 2) continue;
        const uint32_t c = big_mod_u32(j->K, q);
        const uint32_t inv2 = (q + 1) / 2;
        const uint32_t r = (uint32_t)((uint64_t)((q - c) % q) * inv2 % q);  // -(K mod q)/2 mod q
        if (tq.size() < TRIAL_PRIMES) {
            tq.push_back(q);
            tr.push_back(r);
        }
        if (q <= p.p && c == 0) {
            kprimes.push_back(q);
            continue;
        }
        if (q <= j->q1 && q <= p.max_prime) {  // odd d-primes and (P, q1]
            sq.push_back(q);
            sr.push_back(r);
            sbar.push_back(~0ull / q);
        }
    }
    j->nsmall = (uint32_t)sq.size();
    std::vector<uint32_t> wheel(j->W, 0);
    auto setb = [&](uint32_t idx) { wheel[idx >> 5] |= 1u << (idx & 31); };
    setb(j->sly);
    for (uint32_t q : kprimes)
        for (uint32_t idx = j->sly % q; idx <= 2 * j->sly; idx += q) setb(idx);
    j->cap = 0;
    for (uint32_t y = 1; y <= j->sly; y++) j->cap += !((wheel[(j->sly + y) >> 5] >> ((j->sly + y) & 31)) & 1u);
    if (j->cap == 0) j->cap = 1;
    // ---- device copies of the host tables
    int rc;
    if ((rc = dalloc(j, &j->d_wheel, j->W)) || (rc = dalloc(j, &j->d_sq, sq.size())) ||
        (rc = dalloc(j, &j->d_sr, sr.size())) || (rc = dalloc(j, &j->d_sbar, sbar.size())) ||
        (rc = dalloc(j, &j->d_tq, TRIAL_PRIMES)) || (rc = dalloc(j, &j->d_tr, TRIAL_PRIMES)))
        return rc;
    PG_CUDA(cudaMemcpyAsync(j->d_wheel, wheel.data(), wheel.size() * 4, cudaMemcpyHostToDevice, st));
    if (!sq.empty()) {
        PG_CUDA(cudaMemcpyAsync(j->d_sq, sq.data(), sq.size() * 4, cudaMemcpyHostToDevice, st));
        PG_CUDA(cudaMemcpyAsync(j->d_sr, sr.data(), sr.size() * 4, cudaMemcpyHostToDevice, st));
        PG_CUDA(cudaMemcpyAsync(j->d_sbar, sbar.data(), sbar.size() * 8, cudaMemcpyHostToDevice, st));
    }
    PG_CUDA(cudaMemcpyAsync(j->d_tq, tq.data(), tq.size() * 4, cudaMemcpyHostToDevice, st));
    PG_CUDA(cudaMemcpyAsync(j->d_tr, tr.data(), tr.size() * 4, cudaMemcpyHostToDevice, st));
    PG_CUDA(cudaStreamSynchronize(st));  // host vectors die at return
    // ---- large primes (q1, max_prime] on the device
    j->np = 0;
    if (p.max_prime > j->q1) {
        j->wide = p.max_prime >= (1ull << 32);
        const uint32_t root = (uint32_t)std::sqrt((double)p.max_prime) + 2;
        std::vector<uint32_t> base;
        for (uint32_t q : host_primes(root))
            if (q != 2) base.push_back(q);
        const uint64_t v_first = ((uint64_t)j->q1 + 1) | 1ull;
        const uint64_t seg_span = 2ull * (1u << 18);
        const uint64_t nseg64 = (p.max_prime - v_first) / seg_span + 1;
        if (nseg64 > 0x7fffffff) return fail(PG_ERR_UNSUPPORTED, "max_prime too large");
        const uint32_t nseg = (uint32_t)nseg64;
        uint32_t *d_base = nullptr, *d_cnt = nullptr;
        uint64_t *d_off = nullptr;
        PG_CUDA(cudaMalloc((void **)&d_base, base.size() * 4));
        PG_CUDA(cudaMalloc((void **)&d_cnt, (size_t)nseg * 4));
        PG_CUDA(cudaMalloc((void **)&d_off, (size_t)nseg * 8));
        PG_CUDA(cudaMemcpyAsync(d_base, base.data(), base.size() * 4, cudaMemcpyHostToDevice, st));
        PG_CUDA(launch_prime_count(v_first, p.max_prime, d_base, (uint32_t)base.size(), nseg, d_cnt, st));
        std::vector<uint32_t> cnt(nseg);
        std::vector<uint64_t> off(nseg);
        PG_CUDA(cudaMemcpyAsync(cnt.data(), d_cnt, (size_t)nseg * 4, cudaMemcpyDeviceToHost, st));
        PG_CUDA(cudaStreamSynchronize(st));
        uint64_t acc = 0;
        for (uint32_t i = 0; i < nseg; i++) {
            off[i] = acc;
            acc += cnt[i];
        }
        j->np = acc;
        j->seg_off = off;
        j->seg_v0 = v_first;
        j->seg_span = seg_span;
        const size_t esz = j->wide ? 8 : 4;
        void *lp = nullptr, *lc = nullptr, *lci = nullptr;
        cudaError_t e1 = cudaMalloc(&lp, std::max<uint64_t>(acc, 1) * esz);
        cudaError_t e2 = cudaMalloc(&lc, std::max<uint64_t>(acc, 1) * esz);
        cudaError_t e3 = cudaMalloc(&lci, std::max<uint64_t>(acc, 1) * esz);
        j->d_lp = lp;
        j->d_lc = lc;
        j->d_lcinv = lci;
        if (e1 || e2 || e3) {
            cudaFree(d_base);
            cudaFree(d_cnt);
            cudaFree(d_off);
            return fail(PG_ERR_NOMEM, "prime table of %llu primes", (unsigned long long)acc);
        }
        j->dev_bytes += 3 * std::max<uint64_t>(acc, 1) * esz;
        PG_CUDA(cudaMemcpyAsync(d_off, off.data(), (size_t)nseg * 8, cudaMemcpyHostToDevice, st));
        PG_CUDA(launch_prime_write(v_first, p.max_prime, d_base, (uint32_t)base.size(), nseg, d_off, j->d_lp, j->wide,
                                   st));
        uint32_t *d_K = nullptr;
        PG_CUDA(cudaMalloc((void **)&d_K, j->K.size() * 4));
        PG_CUDA(cudaMemcpyAsync(d_K, j->K.data(), j->K.size() * 4, cudaMemcpyHostToDevice, st));
        PG_CUDA(launch_prime_tables(d_K, (uint32_t)j->K.size(), j->np, j->d_lp, j->d_lc, j->d_lcinv, j->wide, st));
        PG_CUDA(cudaStreamSynchronize(st));
        cudaFree(d_K);
        cudaFree(d_base);
        cudaFree(d_cnt);
        cudaFree(d_off);
    }
    // ---- window slots
    const uint64_t mi = std::max<uint64_t>(p.max_m_inc, 2);
    j->nodd_cap = mi / 2 + 1;
    uint64_t phi = 0;
    for (uint64_t r = 1; r <= p.d; r++) phi += gcd64(r, p.d) == 1;
    j->nm_cap = std::min<uint64_t>(j->nodd_cap, (mi / p.d + 1) * phi);
    if (2 * j->nm_cap >= 0xffffffffull) return fail(PG_ERR_UNSUPPORTED, "max_m_inc too large");
    for (auto &s : j->slot)
        if ((rc = slot_alloc(j, s))) return rc;
    j->grid = search_grid(j->L, j->ctx->device);
    return PG_OK;
}

extern "C" int pg_job_create(pg_ctx *c, const pg_job_params *params, pg_job **out) {
    if (!c || !params || !out) return fail(PG_ERR_ARG, "pg_job_create: NULL argument");
    *out = nullptr;
    const pg_job_params &p = *params;
    if (!is_prime_u32(p.p)) return fail(PG_ERR_ARG, "p=%u is not prime", p.p);
    if (p.d == 0 || p.d % 2) return fail(PG_ERR_ARG, "d=%u must be even", p.d);
    if (p.sl < 2 || p.sl / 2 > 65535) return fail(PG_ERR_ARG, "sl=%u outside [2, 131071]", p.sl);
    if (p.max_prime >= (1ull << 40)) return fail(PG_ERR_ARG, "max_prime must be < 2^40");
    if (p.max_m == 0) return fail(PG_ERR_ARG, "max_m must be set");
    if (p.rounds < 1 || p.rounds > 16) return fail(PG_ERR_ARG, "rounds=%u (1..16)", p.rounds);
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

extern "C" int pg_job_get_info(const pg_job *j, pg_job_info *info) {
    if (!j || !info) return fail(PG_ERR_ARG, "pg_job_get_info: NULL argument");
    info->k_bits = j->kbits;
    info->limbs = layout_words(j->L);
    info->tpi = j->L >> 16 ? j->L >> 16 : 1;
    info->words_per_m = j->W;
    info->side_capacity = j->cap;
    info->num_primes = j->np;
    info->num_small = j->nsmall;
    info->k_log = j->k_log;
    info->setup_seconds = j->setup_s;
    info->device_bytes = j->dev_bytes;
    return PG_OK;
}

extern "C" int pg_job_k_words(const pg_job *j, uint32_t *out, uint32_t *nwords) {
    if (!j || !nwords) return fail(PG_ERR_ARG, "pg_job_k_words: NULL argument");
    if (out) std::memcpy(out, j->K.data(), j->K.size() * 4);
    *nwords = (uint32_t)j->K.size();
    return PG_OK;
}

extern "C" void *pg_job_stream(pg_job *j, int slot) {
    if (!j || slot < 0 || slot >= PG_SEARCH_SLOTS) return nullptr;
    return (void *)j->slot[slot].st;
}

// ============================================================== windows

// Computes the coprime m and the odd-m rank table of a window into the
// slot's pinned staging (host work only).
static int window_tables(pg_job *j, WinSlot &s, uint64_t m_start, uint64_t m_inc) {
    const pg_job_params &p = j->prm;
    if (m_inc == 0) return fail(PG_ERR_ARG, "m_inc must be > 0");
    if (m_inc > std::max<uint64_t>(p.max_m_inc, 2))
        return fail(PG_ERR_ARG, "m_inc=%llu > max_m_inc=%llu", (unsigned long long)m_inc,
                    (unsigned long long)p.max_m_inc);
    if (m_start == 0) return fail(PG_ERR_ARG, "m_start must be > 0");
    if (m_start + m_inc - 1 > p.max_m) return fail(PG_ERR_ARG, "m beyond max_m");
    s.m0 = m_start | 1ull;
    const uint64_t end = m_start + m_inc;
    s.nodd = end > s.m0 ? (end - s.m0 + 1) / 2 : 0;
    uint32_t r = 0;
    for (uint64_t jj = 0; jj < s.nodd; jj++) {
        const uint64_t m = s.m0 + 2 * jj;
        if (gcd64(m, p.d) == 1) {
            s.h_ms[r] = m;
            s.h_rank[jj] = (int32_t)r++;
        } else {
            s.h_rank[jj] = -1;
        }
    }
    s.nm = r;
    return PG_OK;
}

// Uploads the window tables on the slot's stream.
static int window_upload(WinSlot &s) {
    if (s.nm) PG_CUDA(cudaMemcpyAsync(s.d_ms, s.h_ms, (size_t)s.nm * 8, cudaMemcpyHostToDevice, s.st));
    if (s.nodd) PG_CUDA(cudaMemcpyAsync(s.d_rank, s.h_rank, (size_t)s.nodd * 4, cudaMemcpyHostToDevice, s.st));
    return PG_OK;
}

static int window_setup(pg_job *j, WinSlot &s, uint64_t m_start, uint64_t m_inc) {
    int rc = window_tables(j, s, m_start, m_inc);
    return rc ? rc : window_upload(s);
}

// prime-table index of the first segment starting at or above value v
static uint64_t table_index_at(const pg_job *j, double v) {
    if (v <= (double)j->seg_v0) return 0;
    const double s = std::ceil((v - (double)j->seg_v0) / (double)j->seg_span);
    if (s >= (double)j->seg_off.size()) return j->np;
    return j->seg_off[(size_t)s];
}

// First prime-table index sieved by modular search rather than by stepping
// every Y.  The search needs p > 2 sly + 1 (one hit per m); by default every
// such prime is searched (with the hit walk, stepping is slower at any split
// on the P=503 window); search_hits > 0 keeps primes expecting at least that
// many hits, nodd * (2 sly + 1) / p, on the stepping kernel.
static uint64_t large_split(const pg_job *j, uint64_t nodd) {
    if (j->np == 0) return 0;
    const uint64_t min_split = table_index_at(j, 2.0 * j->sly + 2);
    if (j->prm.flags & PG_JOB_LARGE_STEP) return j->np;
    if ((j->prm.flags & PG_JOB_LARGE_SEARCH) || j->prm.search_hits == 0) return min_split;
    const double hits = (double)j->prm.search_hits;
    return std::max(min_split, table_index_at(j, (double)nodd * (2.0 * j->sly + 1) / hits));
}

static int run_sieve(pg_job *j, WinSlot &s, bool compact) {
    PG_CUDA(cudaMemsetAsync(s.d_bitmaps, 0, (size_t)s.nm * j->W * 4, s.st));
    PG_CUDA(cudaMemsetAsync(&s.d_sc->max_count, 0, 4, s.st));
    LargeArgs la{};
    la.sly = j->sly;
    la.words = j->W;
    la.m0 = s.m0;
    la.nodd = s.nodd;
    la.rank = s.d_rank;
    la.bitmaps = s.d_bitmaps;
    la.np = j->np;
    la.p = j->d_lp;
    la.cinv = j->d_lcinv;
    la.c = j->d_lc;
    const uint64_t split = large_split(j, s.nodd);
    PG_CUDA(launch_sieve_large(la, j->wide, split, s.st));
    s.sst.kernel_launches += (split > 0) + (split < j->np);
    SieveArgs sa{};
    sa.sly = j->sly;
    sa.words = j->W;
    sa.cap = j->cap;
    sa.m0 = s.m0;
    sa.nodd = s.nodd;
    sa.nm = s.nm;
    sa.ms = s.d_ms;
    sa.rank = s.d_rank;
    sa.bitmaps = s.d_bitmaps;
    sa.wheel = j->d_wheel;
    sa.sq = j->d_sq;
    sa.sr = j->d_sr;
    sa.sbar = j->d_sbar;
    sa.nsmall = j->nsmall;
    sa.lists = s.d_lists;
    sa.counts = s.d_counts;
    sa.max_count = &s.d_sc->max_count;
    PG_CUDA(launch_sieve_small(sa, compact, s.st));
    s.sst.kernel_launches++;
    return PG_OK;
}

static int slot_idle(pg_job *j, WinSlot &s, const char *who) {
    if (s.busy)
        return fail(PG_ERR_STATE, "%s: window slot holds ticket %llu; pg_search_wait it first", who,
                    (unsigned long long)s.ticket);
    (void)j;
    return PG_OK;
}

extern "C" int pg_sieve_interval(pg_job *j, uint64_t m_start, uint64_t m_inc, uint64_t *ms, uint32_t *bitmaps) {
    if (!j) return fail(PG_ERR_ARG, "pg_sieve_interval: job is NULL");
    PG_CUDA(cudaSetDevice(j->ctx->device));
    WinSlot &s = j->slot[0];
    int rc = slot_idle(j, s, "pg_sieve_interval");
    if (rc) return rc;
    PG_CUDA(cudaStreamSynchronize(s.st));  // pinned staging is reused
    if ((rc = window_setup(j, s, m_start, m_inc))) return rc;
    if ((rc = run_sieve(j, s, false))) return rc;
    if (bitmaps && s.nm)
        PG_CUDA(cudaMemcpyAsync(bitmaps, s.d_bitmaps, (size_t)s.nm * j->W * 4, cudaMemcpyDeviceToHost, s.st));
    PG_CUDA(cudaStreamSynchronize(s.st));
    if (ms) std::memcpy(ms, s.h_ms, (size_t)s.nm * 8);
    return PG_OK;
}

static SearchArgs base_args(pg_job *j, WinSlot &s) {
    SearchArgs a{};
    std::memset(a.K, 0, sizeof a.K);
    std::memcpy(a.K, j->K.data(), j->K.size() * 4);
    a.kwords = (uint32_t)j->K.size();
    a.sly = j->sly;
    a.cap = j->cap;
    a.ntrial = TRIAL_PRIMES;
    a.rounds = j->prm.rounds;
    a.ms = s.d_ms;
    a.lists = s.d_lists;
    a.counts = s.d_counts;
    a.k_start = s.d_kstart;
    a.found_k = s.d_found;
    a.next_item = &s.d_sc->next_item;
    a.tests = &s.d_sc->tests;
    a.trial_q = j->d_tq;
    a.trial_r = j->d_tr;
    return a;
}

// Finalize all sides and queue the copies back; the host reads n_redo in
// slot_finish.
static int enqueue_finalize(pg_job *j, WinSlot &s, SearchArgs &a, uint32_t S) {
    PG_CUDA(cudaMemsetAsync(&s.d_sc->n_redo, 0, 4, s.st));
    PG_CUDA(launch_finalize(j->L, a, S, s.d_gaps, s.d_redo, &s.d_sc->n_redo, &s.d_sc->confirm, s.d_kstart, s.st));
    s.sst.kernel_launches++;
    PG_CUDA(record_ev(s.ev[2], s.st));  // end of the device work (before the copies back)
    PG_CUDA(cudaMemcpyAsync(s.h_gaps, s.d_gaps, (size_t)S * 4, cudaMemcpyDeviceToHost, s.st));
    PG_CUDA(cudaMemcpyAsync(s.h_sc, s.d_sc, sizeof(Scalars), cudaMemcpyDeviceToHost, s.st));
    return PG_OK;
}

static int enqueue_window(pg_job *j, WinSlot &s, int form, uint32_t flags);

extern "C" int pg_search_submit(pg_job *j, uint64_t m_start, uint64_t m_inc, int form, uint32_t flags,
                                uint64_t *ticket) {
    if (!j || !ticket) return fail(PG_ERR_ARG, "pg_search_submit: NULL argument");
    if (form != PG_SEARCH_PERSISTENT && form != PG_SEARCH_PLAIN)
        return fail(PG_ERR_ARG, "pg_search_submit: form=%d", form);
    PG_CUDA(cudaSetDevice(j->ctx->device));
    WinSlot &s = j->slot[j->next_ticket % PG_SEARCH_SLOTS];
    int rc = slot_idle(j, s, "pg_search_submit");
    if (rc) return rc;
    PG_CUDA(cudaStreamSynchronize(s.st));  // the slot's pinned staging is reused
    s.sst = pg_search_stats{};
    if ((rc = window_tables(j, s, m_start, m_inc))) return rc;
    s.sst.m_count = s.nm;
    s.sst.h2d_bytes = (uint64_t)s.nm * 8 + (uint64_t)s.nodd * 4;
    s.ticket = j->next_ticket++;
    s.busy = true;
    *ticket = s.ticket;
    if (s.nm == 0) return PG_OK;
    if (form == PG_SEARCH_PLAIN || (j->prm.flags & PG_JOB_NO_GRAPH)) return enqueue_window(j, s, form, flags);
    // The persistent form's whole window (upload, sieves, search, finalize,
    // copies back) is captured as one CUDA graph and launched once; the slot
    // keeps the instantiated graph and updates it in place for the next window.
    PG_CUDA(cudaStreamBeginCapture(s.st, cudaStreamCaptureModeThreadLocal));
    rc = enqueue_window(j, s, form, flags);
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

// Enqueues one window's device work on the slot's stream (capturable for the
// persistent form; the plain form reads counts back and is not).
static int enqueue_window(pg_job *j, WinSlot &s, int form, uint32_t flags) {
    int rc;
    const uint32_t S = 2 * s.nm;
    if ((rc = window_upload(s))) return rc;
    PG_CUDA(record_ev(s.ev[0], s.st));
    if ((rc = run_sieve(j, s, true))) return rc;
    PG_CUDA(record_ev(s.ev[1], s.st));
    const uint32_t warps = (uint32_t)j->grid * 4;
    PG_CUDA(launch_init_search(S, s.d_found, s.d_kstart, s.d_act0, s.d_sc, warps, s.st));
    s.sst.kernel_launches++;
    SearchArgs a = base_args(j, s);
    a.act = s.d_act0;
    a.n_act = S;
    a.ext_max = j->prm.ext_window;
    if (form == PG_SEARCH_PERSISTENT) {
        a.kspan = j->cap + a.ext_max;
        a.max_count = &s.d_sc->max_count;
        a.unresolved = &s.d_sc->unresolved;
        a.active_warps = &s.d_sc->active_warps;
        if (flags & PG_SUBMIT_DRAIN) {
            a.drain_lanes = 4;
            a.min_warps = (uint32_t)j->ctx->sms;
        }
        PG_CUDA(record_ev(s.ev[3], s.st));
        PG_CUDA(launch_search_persistent(j->L, a, j->grid, s.st));
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
            PG_CUDA(launch_search_plain(j->L, a, s.d_knext, s.st));
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
    return enqueue_finalize(j, s, a, S);
}

// Waits for the slot's queued work; continues sides without a prime within
// sl + ext_window on the device with 4x larger extension windows.
static int slot_finish(pg_job *j, WinSlot &s) {
    PG_CUDA(cudaStreamSynchronize(s.st));
    const uint32_t S = 2 * s.nm;
    SearchArgs a = base_args(j, s);
    uint32_t ext_done = j->prm.ext_window;
    for (int round = 0;; round++) {
        const uint32_t n_redo = s.h_sc->n_redo;
        if (n_redo == 0) break;
        if (round >= 24)
            return fail(PG_ERR_STATE, "pg_search: %u sides unresolved after %u extension positions", n_redo, ext_done);
        PG_CUDA(cudaMemcpyAsync(s.d_act1, s.d_redo, (size_t)n_redo * 4, cudaMemcpyDeviceToDevice, s.st));
        const uint32_t ext_new = std::min<uint32_t>(ext_done * 4, 1u << 26);
        a.act = s.d_act1;
        a.n_act = n_redo;
        a.ext_max = ext_new;
        a.kspan = j->cap + ext_new;
        a.max_count = nullptr;
        PG_CUDA(cudaMemsetAsync(&s.d_sc->next_item, 0, 8, s.st));
        PG_CUDA(launch_search_persistent(j->L, a, j->grid, s.st));
        s.sst.kernel_launches++;
        s.sst.relaunches++;
        s.sst.extended_sides += n_redo;
        ext_done = ext_new;
        // finalize the continued sides only (their gaps and a new redo list)
        PG_CUDA(cudaMemsetAsync(&s.d_sc->n_redo, 0, 4, s.st));
        PG_CUDA(launch_finalize(j->L, a, S, s.d_gaps, s.d_redo, &s.d_sc->n_redo, &s.d_sc->confirm, s.d_kstart, s.st));
        s.sst.kernel_launches++;
        PG_CUDA(record_ev(s.ev[2], s.st));
        PG_CUDA(cudaMemcpyAsync(s.h_gaps, s.d_gaps, (size_t)S * 4, cudaMemcpyDeviceToHost, s.st));
        PG_CUDA(cudaMemcpyAsync(s.h_sc, s.d_sc, sizeof(Scalars), cudaMemcpyDeviceToHost, s.st));
        s.sst.d2h_bytes += 4;
        PG_CUDA(cudaStreamSynchronize(s.st));
    }
    return PG_OK;
}

extern "C" int pg_search_wait(pg_job *j, uint64_t ticket, uint64_t *ms, uint32_t *prev_gap, uint32_t *next_gap,
                              pg_search_stats *stats) {
    if (!j) return fail(PG_ERR_ARG, "pg_search_wait: job is NULL");
    PG_CUDA(cudaSetDevice(j->ctx->device));
    WinSlot &s = j->slot[ticket % PG_SEARCH_SLOTS];
    if (!s.busy || s.ticket != ticket)
        return fail(PG_ERR_STATE, "pg_search_wait: ticket %llu is not in flight", (unsigned long long)ticket);
    s.busy = false;
    if (s.nm == 0) {
        if (stats) *stats = s.sst;
        return PG_OK;
    }
    int rc = slot_finish(j, s);
    if (rc) return rc;
    for (uint32_t r = 0; r < s.nm; r++) {
        if (next_gap) next_gap[r] = s.h_gaps[2 * r];
        if (prev_gap) prev_gap[r] = s.h_gaps[2 * r + 1];
    }
    if (ms) std::memcpy(ms, s.h_ms, (size_t)s.nm * 8);
    s.sst.d2h_bytes += (uint64_t)2 * s.nm * 4 + sizeof(Scalars);
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
