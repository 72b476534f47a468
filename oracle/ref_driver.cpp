// ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.  A command-line driver around the
// reference's own, unmodified gap_common.cpp and overflow.cpp, compiled where
// they lie (oracle/Makefile, target ref, output oracle/_ref/ref_tool).  It
// produces the values the tests pin the oracle and the product against:
//
//   k P D                 K = P#/D in hex and its bit count (init_K, gap_common.cpp:60-65),
//                         K_log as a hex double (calc_log_K, gap_common.cpp:51-57, via _log :44-48)
//   count MS MI D         count_num_m (gap_common.cpp:170-206)
//   primes N              count, sum and last of get_sieve_primes(N) (gap_common.cpp:256-278)
//   overflow P D MINC MIN_MERIT M...
//                         runs run_cpu_overflow_thread (overflow.cpp:61-227) on the listed m,
//                         each queued with min_x = 1, so the reference's GMP next/prev prime,
//                         merit, record double-check and record line (overflow.cpp:145-188)
//                         print every record line it finds on stdout (and append them to
//                         records_P.txt in the working directory, as the reference does)
//   argparse ARGS...      Args::argparse (gap_common.cpp:313-492); prints the parsed Config
//
// The reference's globals that overflow.cpp uses are defined here; they live in
// gap_search_gpu.cpp, which needs primesieve and CUDA and is not built.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <string>
#include <utility>
#include <vector>

#include "gap_common.h"
#include "gap_search_gpu.h"
#include "gap_stats.h"
#include "overflow.h"

std::atomic<bool> is_running{true};
std::atomic<uint8_t> stop_queue{0};
std::mutex overflow_mtx;
deque<std::pair<uint64_t, uint32_t>> overflowed;
deque<std::pair<uint64_t, uint32_t>> spot_check;
std::condition_variable overflow_cv;

static Config config_of(uint32_t p, uint32_t d) {
    Config c;
    c.p = p;
    c.d = d;
    c.verbose = -1;
    return c;
}

static int cmd_k(uint32_t p, uint32_t d) {
    Config c = config_of(p, d);
    mpz_t K;
    init_K(c, K);
    char *hex = mpz_get_str(nullptr, 16, K);
    const double k_log = calc_log_K(c);
    printf("bits %zu\nhex %s\nk_log %a\n", mpz_sizeinbase(K, 2), hex, k_log);
    free(hex);
    mpz_clear(K);
    return 0;
}

static int cmd_overflow(int argc, char **argv) {
    Config c = config_of((uint32_t)atoi(argv[0]), (uint32_t)atoi(argv[1]));
    c.m_inc = strtoull(argv[2], nullptr, 10);
    c.min_merit = (float)atof(argv[3]);
    c.m_start = 1;
    mpz_t K;
    init_K(c, K);
    for (int i = 4; i < argc; i++) overflowed.push_back({strtoull(argv[i], nullptr, 10), 1u});
    stop_queue = 2;  // finish the queue, then return
    TestingStats stats;
    run_cpu_overflow_thread(0, c, K, stats);
    fprintf(stderr, "tested %lu prev %lu skipped_prev %lu over_min %lu mismatches %lu\n",
            (unsigned long)stats.tested.load(), (unsigned long)stats.tested_prev.load(),
            (unsigned long)stats.skipped_prev.load(), (unsigned long)stats.greater_than_min_merit.load(),
            (unsigned long)stats.mismatches.load());
    mpz_clear(K);
    return overflowed.empty() ? 0 : 1;
}

static int cmd_argparse(int argc, char **argv) {
    std::vector<char *> av;
    static char name[] = "gap_search_gpu";
    av.push_back(name);
    for (int i = 0; i < argc; i++) av.push_back(argv[i]);
    av.push_back(nullptr);
    Config c = Args::argparse((int)av.size() - 1, av.data(), Args::Pr::SEARCH_GPU);
    printf("\nCONFIG valid %d p %u d %u m_start %lu m_inc %lu min_merit %a max_prime %lu cpu_fraction %a "
           "cpu_threads %d verbose %d show_timing %d testing %d\n",
           c.valid, c.p, c.d, (unsigned long)c.m_start, (unsigned long)c.m_inc, (double)c.min_merit,
           (unsigned long)c.max_prime, (double)c.cpu_fraction, c.cpu_threads, c.verbose, (int)c.show_timing,
           (int)c.testing);
    return 0;
}

int main(int argc, char **argv) {
    if (argc < 2) {
        fprintf(stderr, "usage: ref_tool k|count|primes|overflow|argparse ...\n");
        return 2;
    }
    const std::string cmd = argv[1];
    if (cmd == "k" && argc == 4) return cmd_k((uint32_t)atoi(argv[2]), (uint32_t)atoi(argv[3]));
    if (cmd == "count" && argc == 5) {
        printf("%zu\n", count_num_m(atol(argv[2]), atol(argv[3]), strtoull(argv[4], nullptr, 10)));
        return 0;
    }
    if (cmd == "primes" && argc == 3) {
        const vector<uint32_t> ps = get_sieve_primes((uint32_t)atol(argv[2]));
        unsigned long long sum = 0;
        for (uint32_t q : ps) sum += q;
        printf("count %zu sum %llu last %u\n", ps.size(), sum, ps.empty() ? 0u : ps.back());
        return 0;
    }
    if (cmd == "overflow" && argc >= 6) return cmd_overflow(argc - 2, argv + 2);
    if (cmd == "argparse") return cmd_argparse(argc - 2, argv + 2);
    fprintf(stderr, "ref_tool: bad arguments\n");
    return 2;
}
