// gap_search_gpu -- command line of the prime-gap search on the B200 library.
//
// Keeps the reference's flags and output (gap_common.cpp:313-492,
// gap_search_gpu.cpp:106-175, overflow.cpp:179-188):
//   -p P -d D --mstart M --minc I --max-prime MILLIONS --min-merit F
//   --cpu-fraction F --cpu-threads N   (accepted; there is no CPU finishing)
//   --hide-timing --testing -q -v -h
// and adds:
//   --sl X        search radius: X in [-sl, sl] is sieved (default 8*ln(N), even)
//   --ranges R    windows of --minc m to search; 0 = until Ctrl-C (the reference's only mode)
//   --chunk C     m per device call (default min(minc, 1,000,000))
//   --form persistent|plain   --rounds R   --device N
//   --warps-per-sm W   cap on each window's PRP warps per SM (default 6 for one-thread operands,
//                      none for lane-group operands; 0 = all that fit): two windows are in flight
//                      and share the SMs
//   --resume FILE      after every finished range write "P D MINC NEXT_MSTART RANGES_DONE" to FILE;
//                      when FILE exists at start (same P, D, MINC), continue from it
//   --devices A,B,...  one worker per listed CUDA device, each searching whole ranges (the m ranges
//                      shard with no exchange); records are printed in range order
//   --confirm-rounds R both primes of every gap with merit > --min-merit pass R strong bases
//                      (2, 3, 5, ...) on the device before it is printed (default 16; 0 = off):
//                      the double-check of overflow.cpp:164-177
//   --spot-check N     GMP re-tests both primes of N m per window with mpz_probab_prime_p(n, 20), as
//                      the reference spot-checks GPU primes (gpu_testing.cu:125-129, overflow.cpp:117-135);
//                      libgmp.so.10 is loaded at run time (default 1; 0 = off; skipped with a notice
//                      when the library is absent)
// Record lines "{gap} {merit:.3f} {m} * {P}# / {D} - {prev}" go to stdout and
// are appended to records_{P}.txt.  Ctrl-C once: finish the current window;
// twice: stop after the current device call; three times: exit(2)
// (gap_search_gpu.cpp:1050-1069).
#include <dlfcn.h>
#include <getopt.h>

#include <atomic>
#include <chrono>
#include <cmath>
#include <csignal>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/primegap.h"

struct Config {
    int valid = 1;
    uint32_t p = 0, d = 0;
    uint64_t m_start = 0, m_inc = 0;
    float min_merit = 18;
    uint64_t max_prime = 0;
    float cpu_fraction = 0.005f;
    int cpu_threads = 3;
    int verbose = 1;
    bool show_timing = true;
    bool testing = false;
    // additions
    uint32_t sl = 0;
    uint64_t ranges = 0;
    uint64_t chunk = 0;
    int form = PG_SEARCH_PERSISTENT;
    uint32_t rounds = 1;
    int device = 0;
    int warps_per_sm = -1;  // -1: 6 for one-thread layouts, no cap for lane groups
    std::string resume;
    std::vector<int> devices;  // --devices; empty = {device}
    uint32_t confirm_rounds = 16;
    uint32_t spot_check = 1;
};

static void show_usage(const char *name) {
    printf("Usage: %s\n[REQUIRED]\n  -p <p>\n  -d <p>\n  --mstart <start>\n  --minc   <int>\n\n", name);
    printf("[OPTIONALLY]\n  --min-merit <min_merit>\n    only display prime gaps with merit >= min_merit\n");
    printf("  --max-prime\n    use primes <= max-prime (in millions) for checking composite\n\n");
    printf("  --cpu-fraction <fraction>   (accepted for compatibility; no CPU finishing)\n");
    printf("  --cpu-threads <n>           (accepted for compatibility; no CPU finishing)\n");
    printf("  --sl <X>        sieve X in [-sl, sl] around m*K (default 8*ln(m*K))\n");
    printf("  --ranges <R>    search R windows of minc m, 0 = until Ctrl-C (default 0)\n");
    printf("  --chunk <C>     m per device call (default min(minc, 1000000))\n");
    printf("  --form persistent|plain   --rounds <bases>   --device <n>\n");
    printf("  --warps-per-sm <W>  PRP warps per SM of each of the two windows in flight\n");
    printf("                      (default 6, or all for lane-group operands; 0 = as many as fit)\n");
    printf("  --resume <file>     progress file: written after every finished range, read at start\n");
    printf("  --devices <a,b,..>  search on these CUDA devices, one range per device at a time\n");
    printf("  --confirm-rounds <R> strong bases both primes of a record pass (default 16, 0 = off)\n");
    printf("  --spot-check <N>    m per window whose primes GMP re-tests (default 1, 0 = off)\n\n");
    printf("[OPTIONAL]\n  -q, --quiet\n  -v, --verbose\n  -h, --help\n");
}

static bool is_prime(uint64_t n) {
    if (n < 2) return false;
    for (uint64_t t = 2; t * t <= n; t++)
        if (n % t == 0) return false;
    return true;
}

static Config argparse(int argc, char **argv) {
    static struct option long_options[] = {
        {"p", required_argument, 0, 'p'},         {"d", required_argument, 0, 'd'},
        {"mstart", required_argument, 0, 1},      {"minc", required_argument, 0, 2},
        {"min-merit", required_argument, 0, 4},   {"max-prime", required_argument, 0, 5},
        {"cpu-fraction", required_argument, 0, 7}, {"cpu-threads", required_argument, 0, 8},
        {"hide-timing", no_argument, 0, 11},      {"testing", no_argument, 0, 12},
        {"sl", required_argument, 0, 20},         {"ranges", required_argument, 0, 21},
        {"chunk", required_argument, 0, 22},      {"form", required_argument, 0, 23},
        {"rounds", required_argument, 0, 24},     {"device", required_argument, 0, 25},
        {"warps-per-sm", required_argument, 0, 26}, {"resume", required_argument, 0, 27},
        {"devices", required_argument, 0, 28},     {"confirm-rounds", required_argument, 0, 29},
        {"spot-check", required_argument, 0, 30},
        {"quiet", no_argument, 0, 'q'},           {"verbose", no_argument, 0, 'v'},
        {"help", no_argument, 0, 'h'},            {0, 0, 0, 0}};
    Config c;
    int idx = 0, ch;
    while ((ch = getopt_long(argc, argv, "qvhp:d:", long_options, &idx)) >= 0) {
        switch (ch) {
            case 'h': show_usage(argv[0]); exit(0);
            case 'q': c.verbose--; break;
            case 'v': c.verbose++; break;
            case 'p': c.p = (uint32_t)atoi(optarg); break;
            case 'd': c.d = (uint32_t)atoi(optarg); break;
            case 1: c.m_start = strtoull(optarg, nullptr, 10); break;
            case 2: c.m_inc = strtoull(optarg, nullptr, 10); break;
            case 4: c.min_merit = (float)atof(optarg); break;
            case 5: c.max_prime = strtoull(optarg, nullptr, 10) * 1000000ull; break;
            case 7: c.cpu_fraction = (float)atof(optarg); break;
            case 8: c.cpu_threads = atoi(optarg); break;
            case 11: c.show_timing = false; break;
            case 12: c.testing = true; break;
            case 20: c.sl = (uint32_t)strtoul(optarg, nullptr, 10); break;
            case 21: c.ranges = strtoull(optarg, nullptr, 10); break;
            case 22: c.chunk = strtoull(optarg, nullptr, 10); break;
            case 23:
                if (!strcmp(optarg, "persistent")) c.form = PG_SEARCH_PERSISTENT;
                else if (!strcmp(optarg, "plain")) c.form = PG_SEARCH_PLAIN;
                else c.valid = 0;
                break;
            case 24: c.rounds = (uint32_t)atoi(optarg); break;
            case 25: c.device = atoi(optarg); break;
            case 26: c.warps_per_sm = atoi(optarg); break;
            case 27: c.resume = optarg; break;
            case 28:
                for (const char *q = optarg; *q;) {
                    char *end = nullptr;
                    const long v = strtol(q, &end, 10);
                    if (end == q || v < 0 || (*end && *end != ',')) {
                        c.valid = 0;
                        break;
                    }
                    c.devices.push_back((int)v);
                    q = *end == ',' ? end + 1 : end;
                }
                break;
            case 29: c.confirm_rounds = (uint32_t)atoi(optarg); break;
            case 30: c.spot_check = (uint32_t)atoi(optarg); break;
            default: c.valid = 0;
        }
    }
    if (optind < argc) {
        c.valid = 0;
        printf("unknown positional argument: ");
        while (optind < argc) printf("%s ", argv[optind++]);
        printf("\n");
    }
    // validation (gap_common.cpp:416-490; the m parity, 2e9 prime and BITS limits are lifted)
    if (c.m_start == 0) { c.valid = 0; printf("mstart must be greater than 0\n"); }
    if (c.m_inc == 0) { c.valid = 0; printf("m_inc must be greater than 0\n"); }
    if (c.max_prime < 1000) { c.valid = 0; printf("max_prime must be set\n"); }
    if (c.max_prime >= (1ull << 40)) { c.valid = 0; printf("max_prime must be below 2^40\n"); }
    if (!is_prime(c.p) || c.p >= 10000000) { printf("p# not prime (p=%u)\n", c.p); exit(1); }
    if (c.d == 0 || c.d % 2) { c.valid = 0; printf("d must be even and greater than 0: %u\n", c.d); }
    if (c.cpu_fraction < .00001f || c.cpu_fraction > .1f) { c.valid = 0; printf("cpu-fraction must be between .00001 and .1\n"); }
    if (c.cpu_threads < 1 || c.cpu_threads > 159) { c.valid = 0; printf("cpu-threads must be between 1 and 159\n"); }
    if (c.rounds < 1 || c.rounds > 16) { c.valid = 0; printf("rounds must be in 1..16\n"); }
    if (c.confirm_rounds == 1 || c.confirm_rounds > 16) { c.valid = 0; printf("confirm-rounds must be 0 or in 2..16\n"); }
    return c;
}

static std::atomic<int> g_stop{0};
static void on_sigint(int) {
    const int n = ++g_stop;
    if (n == 1) printf("\nCaught CTRL+C stopping, winding down work.\n\n");
    else if (n == 2) printf("\nCaught 2nd CTRL+C, stopping after the current device call\n");
    else { printf("\nCaught 3nd CTRL+C, exit(2) now.\n"); exit(2); }
}

#define CHECK(call)                                                              \
    do {                                                                         \
        int rc_ = (call);                                                        \
        if (rc_ != PG_OK) {                                                      \
            fprintf(stderr, "ERROR %s: %s\n", #call, pg_last_error());           \
            return 1;                                                            \
        }                                                                        \
    } while (0)

// GMP spot checks of found primes (the reference re-tests GPU primes with
// mpz_probab_prime_p(n, 20), gpu_testing.cu:125-129, overflow.cpp:117-135).
// libgmp is opened at run time so the tool runs without it; only the four
// public mpz entry points used are declared (GMP exports mpz_xxx as __gmpz_xxx,
// and an mpz_t is {int alloc; int size; limb *d}).
struct GmpCheck {
    struct Mpz {
        int alloc, size;
        void *d;
    };
    void (*init)(Mpz *) = nullptr;
    void (*clear)(Mpz *) = nullptr;
    void (*import_)(Mpz *, size_t, int, size_t, int, size_t, const void *) = nullptr;
    int (*probab_prime_p)(const Mpz *, int) = nullptr;
    void *h = nullptr;
    bool open() {
        for (const char *name : {"libgmp.so.10", "libgmp.so"}) {
            h = dlopen(name, RTLD_NOW | RTLD_LOCAL);
            if (h) break;
        }
        if (!h) return false;
        init = (void (*)(Mpz *))dlsym(h, "__gmpz_init");
        clear = (void (*)(Mpz *))dlsym(h, "__gmpz_clear");
        import_ = (void (*)(Mpz *, size_t, int, size_t, int, size_t, const void *))dlsym(h, "__gmpz_import");
        probab_prime_p = (int (*)(const Mpz *, int))dlsym(h, "__gmpz_probab_prime_p");
        return init && clear && import_ && probab_prime_p;
    }
    // m*K + x (x may be negative) as LE words, then GMP's verdict (> 0: probably prime)
    int verdict(const std::vector<uint32_t> &K, uint64_t m, int64_t x) const {
        std::vector<uint32_t> n(K.size() + 3, 0);
        uint64_t carry = 0;
        for (size_t i = 0; i < K.size() + 2; i++) {  // n = K * m (m < 2^64: two words)
            const uint64_t kw = i < K.size() ? K[i] : 0;
            const unsigned __int128 t = (unsigned __int128)kw * m + carry;
            n[i] = (uint32_t)t;
            carry = (uint64_t)(t >> 32);
        }
        const uint64_t ax = (uint64_t)(x < 0 ? -x : x);
        if (x >= 0) {
            uint64_t c = ax;
            for (size_t i = 0; i < n.size() && c; i++) {
                const uint64_t t = (uint64_t)n[i] + (c & 0xffffffffu);
                n[i] = (uint32_t)t;
                c = (c >> 32) + (t >> 32);
            }
        } else {
            uint64_t b = ax;
            for (size_t i = 0; i < n.size() && b; i++) {
                const uint64_t sub = b & 0xffffffffu;
                const uint64_t cur = n[i];
                n[i] = (uint32_t)(cur - sub);
                b = (b >> 32) + (cur < sub ? 1 : 0);
            }
        }
        Mpz z;
        init(&z);
        import_(&z, n.size(), -1, 4, 0, 0, n.data());
        const int v = probab_prime_p(&z, 20);
        clear(&z);
        return v;
    }
};

// One device's context and job, with the host buffers of its PG_SEARCH_SLOTS
// windows in flight.
struct Engine {
    Engine() = default;
    Engine(const Engine &) = delete;
    Engine &operator=(const Engine &) = delete;
    pg_ctx *ctx = nullptr;
    pg_job *job = nullptr;
    pg_job_info info{};
    std::vector<uint32_t> K;      // K = P#/d, LE words (spot checks)
    const GmpCheck *gmp = nullptr;
    uint64_t spot_seq = 0;        // windows finished (picks the spot-checked m)
    std::vector<uint64_t> ms[PG_SEARCH_SLOTS];
    std::vector<uint32_t> prev[PG_SEARCH_SLOTS], next[PG_SEARCH_SLOTS];
    ~Engine() {
        if (job) pg_job_destroy(job);
        if (ctx) pg_ctx_destroy(ctx);
    }
};

// The records and counts of one range of --minc m.
struct RangeOut {
    std::vector<std::string> lines;
    uint64_t m = 0, tests = 0, ext = 0, batches = 0, confirm = 0, spot = 0;
    double dev_ms = 0;  // device time of the range's calls
    bool whole = true;  // false when a second Ctrl-C stopped it part-way
    bool done = false;
};

static int make_engine(Engine &e, int device, const pg_job_params &prm, uint64_t chunk) {
    CHECK(pg_ctx_create(device, &e.ctx));
    CHECK(pg_job_create(e.ctx, &prm, &e.job));
    pg_job_get_info(e.job, &e.info);
    uint32_t nk = 0;
    CHECK(pg_job_k_words(e.job, nullptr, &nk));
    e.K.resize(nk);
    CHECK(pg_job_k_words(e.job, e.K.data(), &nk));
    for (int k = 0; k < PG_SEARCH_SLOTS; k++) {
        e.ms[k].resize(chunk);
        e.prev[k].resize(chunk);
        e.next[k].resize(chunk);
    }
    return 0;
}

// Searches [m_start, m_start + m_inc) in chunks with PG_SEARCH_SLOTS windows in
// flight: while one window's gaps are read, the next runs on the device.
static int search_range(Engine &e, const Config &c, uint64_t chunk, uint64_t m_start, RangeOut &out) {
    struct Pending {
        uint64_t ticket;
        int buf;
    };
    // default cap: two one-thread windows in flight share the SMs best at 6 warps per SM each; the lane
    // groups' carry chains need all the warps their registers allow to hide their latency
    const uint32_t wps = c.warps_per_sm >= 0 ? (uint32_t)c.warps_per_sm : (e.info.tpi > 1 ? 0u : 6u);
    const uint32_t flags = c.form == PG_SEARCH_PERSISTENT ? PG_SUBMIT_WARPS_PER_SM(wps) : 0u;
    std::vector<Pending> pending;
    auto finish_one = [&]() {
        const Pending pd = pending.front();
        pending.erase(pending.begin());
        pg_search_stats st{};
        CHECK(pg_search_wait(e.job, pd.ticket, e.ms[pd.buf].data(), e.prev[pd.buf].data(), e.next[pd.buf].data(),
                             &st));
        out.m += st.m_count;
        out.tests += st.prp_tests;
        out.confirm += st.confirm_tests;
        out.ext += st.extended_sides;
        out.batches++;
        out.dev_ms += st.total_ms;
        // GMP spot checks: both primes of spot_check m spread over the window
        if (e.gmp && st.m_count) {
            for (uint32_t q = 0; q < c.spot_check; q++) {
                const uint64_t i = (e.spot_seq * 7919u + q * 104729u) % st.m_count;
                const uint64_t m = e.ms[pd.buf][i];
                const int64_t ends[2] = {(int64_t)e.next[pd.buf][i], -(int64_t)e.prev[pd.buf][i]};
                for (int64_t x : ends) {
                    out.spot++;
                    if (e.gmp->verdict(e.K, m, x) <= 0) {
                        fprintf(stderr, "\n\nSPOT CHECK FAILED: %llu * %u# / %u %+lld is not prime!\n\n",
                                (unsigned long long)m, c.p, c.d, (long long)x);
                        exit(1);
                    }
                }
            }
            e.spot_seq++;
        }
        for (uint64_t i = 0; i < st.m_count; i++) {
            const uint64_t gap = (uint64_t)e.prev[pd.buf][i] + e.next[pd.buf][i];
            const double merit = pg_merit(e.info.k_log, e.ms[pd.buf][i], gap);
            if (merit > c.min_merit) {
                char line[160];
                pg_format_record(line, sizeof line, gap, merit, e.ms[pd.buf][i], c.p, c.d, e.prev[pd.buf][i]);
                out.lines.push_back(line);
            }
        }
        return 0;
    };
    int next_buf = 0;
    for (uint64_t off = 0; off < c.m_inc; off += chunk) {
        if (g_stop >= 2) {
            out.whole = false;
            break;
        }
        const uint64_t inc = std::min(chunk, c.m_inc - off);
        if ((int)pending.size() == PG_SEARCH_SLOTS && finish_one()) return 1;
        uint64_t ticket = 0;
        CHECK(pg_search_submit(e.job, m_start + off, inc, c.form, flags, &ticket));
        pending.push_back({ticket, next_buf});
        next_buf = (next_buf + 1) % PG_SEARCH_SLOTS;
    }
    while (!pending.empty())
        if (finish_one()) return 1;
    return 0;
}

int main(int argc, char **argv) {
    Config c = argparse(argc, argv);
    if (!c.valid) {
        show_usage(argv[0]);
        return 1;
    }
    if (c.verbose >= 0) printf("\nTesting m * %u#/%u\n", c.p, c.d);
    // progress file: continue after the last finished range of the same search
    uint64_t ranges_done = 0;
    if (!c.resume.empty()) {
        if (FILE *f = fopen(c.resume.c_str(), "r")) {
            unsigned long long fp = 0, fd = 0, finc = 0, fnext = 0, fdone = 0;
            const int got = fscanf(f, "%llu %llu %llu %llu %llu", &fp, &fd, &finc, &fnext, &fdone);
            fclose(f);
            if (got != 5 || fp != c.p || fd != c.d || finc != c.m_inc) {
                fprintf(stderr, "ERROR %s does not hold the progress of -p %u -d %u --minc %llu\n", c.resume.c_str(),
                        c.p, c.d, (unsigned long long)c.m_inc);
                return 1;
            }
            c.m_start = fnext;
            ranges_done = fdone;
            if (c.verbose >= 0)
                printf("resuming at m = %llu after %llu ranges\n", (unsigned long long)fnext, (unsigned long long)fdone);
        }
    }
    if (c.ranges && ranges_done >= c.ranges) return 0;
    const uint64_t chunk = c.chunk ? c.chunk : std::min<uint64_t>(c.m_inc, 1000000);
    const uint64_t last_m =
        c.ranges ? c.m_start + (c.ranges - ranges_done) * c.m_inc : c.m_start + 1000 * c.m_inc;
    if (c.devices.empty()) c.devices.push_back(c.device);
    // default radius: 8 * ln(N), even (the serving configuration's SL)
    uint32_t sl = c.sl;
    pg_job_params prm{};
    prm.p = c.p;
    prm.d = c.d;
    prm.max_prime = c.max_prime;
    prm.max_m_inc = chunk;
    prm.max_m = last_m;
    prm.rounds = c.rounds;
    // records are confirmed on the device before they are printed
    prm.confirm_merit = c.confirm_rounds ? std::max(c.min_merit, 1e-9f) : 0.0;
    prm.confirm_rounds = c.confirm_rounds;
    if (!sl) {
        // log(K) first from a throw-away job with a tiny radius
        pg_ctx *pctx = nullptr;
        CHECK(pg_ctx_create(c.devices[0], &pctx));
        pg_job *probe = nullptr;
        pg_job_params pp = prm;
        pp.sl = 2;
        pp.max_prime = std::min<uint64_t>(c.max_prime, 1000);
        pp.max_m_inc = 2;
        CHECK(pg_job_create(pctx, &pp, &probe));
        pg_job_info pi{};
        pg_job_get_info(probe, &pi);
        pg_job_destroy(probe);
        pg_ctx_destroy(pctx);
        sl = 2 * (uint32_t)std::lround(4.0 * (pi.k_log + std::log((double)c.m_start)));
    }
    prm.sl = sl;
    const size_t ndev = c.devices.size();
    GmpCheck gmp;
    const bool have_gmp = c.spot_check && gmp.open();
    if (c.spot_check && !have_gmp && c.verbose >= 0) printf("spot checks skipped: libgmp.so.10 not found\n");
    std::vector<Engine> eng(ndev);
    for (size_t k = 0; k < ndev; k++) {
        if (make_engine(eng[k], c.devices[k], prm, chunk)) return 1;
        eng[k].gmp = have_gmp ? &gmp : nullptr;
    }
    const pg_job_info &info = eng[0].info;
    if (c.verbose >= 1) {
        printf("K = %u bits, log(K) = %.2f\n", info.k_bits, info.k_log);
        printf("sieve: %llu primes <= %llu, X in [-%u, %u], %u-word operands\n",
               (unsigned long long)info.num_primes + info.num_small, (unsigned long long)c.max_prime, sl, sl,
               info.limbs);
        if (ndev > 1) printf("devices: %zu, each searching whole ranges of %llu m\n", ndev, (unsigned long long)c.m_inc);
        if (c.show_timing) printf("\tSetup took %.1f seconds\n", info.setup_seconds);
        printf("Min Gap ~= %d (for merit > %.1f)\n", (int)(c.min_merit * (info.k_log + std::log((double)c.m_inc))),
               c.min_merit);
    }
    std::signal(SIGINT, on_sigint);
    char fname[64];
    snprintf(fname, sizeof fname, "records_%u.txt", c.p);
    FILE *rec = fopen(fname, "a");
    uint64_t total_m = 0, total_tests = 0, total_primes = 0, total_ext = 0, total_batches = 0, total_confirm = 0,
             total_spot = 0;
    double total_dev_s = 0;
    const auto t0 = std::chrono::steady_clock::now();
    // Ranges are handed to the devices in order; each range's records are
    // printed, and the progress file advanced, in range order.
    std::mutex mu;
    std::condition_variable cv;
    std::map<uint64_t, RangeOut> finished;
    std::atomic<uint64_t> next_range{ranges_done};
    std::atomic<int> failed{0};
    std::atomic<size_t> stopped{0};  // workers that have exited
    auto worker = [&](size_t k) {
        while (g_stop == 0 && !failed) {
            const uint64_t r = next_range++;
            if (c.ranges && r >= c.ranges) break;
            RangeOut out;
            if (search_range(eng[k], c, chunk, c.m_start + (r - ranges_done) * c.m_inc, out)) {
                failed = 1;
                break;
            }
            std::lock_guard<std::mutex> lk(mu);
            finished[r] = std::move(out);
            cv.notify_all();
        }
        std::lock_guard<std::mutex> lk(mu);
        stopped++;
        cv.notify_all();
    };
    std::vector<std::thread> threads;
    for (size_t k = 0; k < ndev; k++) threads.emplace_back(worker, k);
    // print the ranges in order as they finish
    bool contiguous = true;  // every range so far searched whole: the progress file may advance
    for (uint64_t r = ranges_done;; r++) {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return finished.count(r) || stopped == ndev; });
        auto it = finished.find(r);
        if (it == finished.end()) break;  // every worker has stopped and range r never ran
        RangeOut out = std::move(it->second);
        finished.erase(it);
        lk.unlock();
        for (const auto &line : out.lines) {
            printf("%s\n", line.c_str());
            if (rec) fprintf(rec, "%s\n", line.c_str());
        }
        if (rec) fflush(rec);
        total_m += out.m;
        total_tests += out.tests;
        total_primes += 2 * out.m;
        total_ext += out.ext;
        total_batches += out.batches;
        total_confirm += out.confirm;
        total_spot += out.spot;
        total_dev_s += out.dev_ms / 1e3;
        contiguous = contiguous && out.whole;
        if (contiguous && !c.resume.empty()) {  // the range is done: record where the next one starts
            const std::string tmp = c.resume + ".tmp";
            if (FILE *f = fopen(tmp.c_str(), "w")) {
                fprintf(f, "%u %u %llu %llu %llu\n", c.p, c.d, (unsigned long long)c.m_inc,
                        (unsigned long long)(c.m_start + (r + 1 - ranges_done) * c.m_inc),
                        (unsigned long long)(r + 1));
                fclose(f);
                std::rename(tmp.c_str(), c.resume.c_str());
            }
        }
        if (c.verbose >= 1) {
            const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            printf("\nGPU Timings (%.0f seconds):\n", c.show_timing ? secs : 0.0);
            // the field names of the reference's print_stats (gap_search_gpu.cpp:138-175); its CPU
            // pipeline's fields (waiting 4 sieve, filling batches, results, batch fill) have no
            // counterpart here, and overflowed sides continue on the device
            printf("\tm               : %llu (%.0f/sec)\n", (unsigned long long)total_m, total_m / secs);
            printf("\tm processed     : %llu (%.0f/sec)\n", (unsigned long long)total_m, total_m / secs);
            printf("\ttotal tests     : %llu (%.1f%% prime) (%.0f/sec)\n", (unsigned long long)total_tests,
                   total_tests ? 100.0 * total_primes / total_tests : 0.0, total_tests / secs);
            printf("\ttotal batches   : %llu (%.5f secs/batch)\n", (unsigned long long)total_batches,
                   total_batches ? secs / total_batches : 0.0);
            printf("\trunning on gpu  : %.1f seconds (%.1f%%)\n", total_dev_s,
                   secs > 0 ? 100.0 * total_dev_s / (secs * ndev) : 0.0);
            printf("\toverflowed      : %llu (%.1f%% of sides, continued on the device)\n",
                   (unsigned long long)total_ext, total_m ? 100.0 * total_ext / (2.0 * total_m) : 0.0);
            printf("\tconfirm tests   : %llu (record primes, %u bases each)\n", (unsigned long long)total_confirm,
                   c.confirm_rounds);
            printf("\tspot checked    : %llu (GMP mpz_probab_prime_p)\n\n", (unsigned long long)total_spot);
        }
    }
    for (auto &t : threads) t.join();
    if (rec) fclose(rec);
    return failed ? 1 : 0;
}
