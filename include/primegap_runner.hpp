// primegap_runner.hpp -- C++ drop-in for the reference's PRP runner.
//
// Replaces miller_rabin.h for its callers: mr_params_t<tpi, bits, window>
// (miller_rabin.h:117-130) and test_runner_t<params> with the constructor
// test_runner_t(n, rounds) (miller_rabin.h:322) and
// run_test(active, tests, results) (miller_rabin.h:364-408) keep their names,
// argument meaning and results, so gpu_testing.cu:217-218 and :274 compile
// unchanged when they include this header instead of miller_rabin.h.
//
// Differences, all on error paths: a batch larger than n, a number wider than
// params::BITS, or a CUDA failure throws std::runtime_error instead of
// calling exit(1); results past `active` are 0 instead of stale.
//
// Requires <gmp.h> (the caller's, as the reference) and links libprimegap.so.
#pragma once

#include <gmp.h>

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "primegap.h"

template <uint32_t tpi, uint32_t bits, uint32_t window_bits>
class mr_params_t {
   public:
    static const uint32_t TPB = 0;
    static const uint32_t MAX_ROTATION = 4;
    static const uint32_t SHM_LIMIT = 0;
    static const bool CONSTANT_TIME = false;
    static const uint32_t TPI = tpi;                  // advisory: the library picks its own layout
    static const uint32_t BITS = bits;                // operand width (multiple of 32)
    static const uint32_t WINDOW_BITS = window_bits;  // advisory
};

template <class params>
class test_runner_t {
   public:
    const size_t n;       // largest batch
    const size_t rounds;  // strong-PRP bases (2, 3, 5, ...); 1 = base 2 only

    test_runner_t(size_t n, size_t rounds, int device = 0) : n(n), rounds(rounds), words_(params::BITS / 32) {
        static_assert(params::BITS % 32 == 0, "BITS must be a multiple of 32");
        check(pg_ctx_create(device, &ctx_), "pg_ctx_create");
        limbs_.resize(n * words_);
        passed_.resize(n);
    }
    ~test_runner_t() { pg_ctx_destroy(ctx_); }
    test_runner_t(const test_runner_t &) = delete;
    test_runner_t &operator=(const test_runner_t &) = delete;

    // results[i] = 1 if *tests[i] passed all `rounds` bases (i < active), else 0.
    void run_test(const size_t active, const std::vector<mpz_t *> &tests, std::vector<int> &results) {
        if (tests.size() == 0) return;
        if (tests.size() > n) throw std::runtime_error("tests(" + std::to_string(tests.size()) + ") > n");
        const size_t to_run = std::min(active, tests.size());
        for (size_t i = 0; i < to_run; i++) {
            if (mpz_sizeinbase(*tests[i], 2) > params::BITS)
                throw std::runtime_error("candidate wider than params::BITS");
            size_t count = 0;
            uint32_t *dst = limbs_.data() + i * words_;
            mpz_export(dst, &count, -1, sizeof(uint32_t), 0, 0, *tests[i]);
            std::fill(dst + count, dst + words_, 0u);
        }
        if (to_run) check(pg_prp_batch(ctx_, limbs_.data(), (uint32_t)to_run, (uint32_t)words_, (uint32_t)rounds,
                                       passed_.data()),
                          "pg_prp_batch");
        for (size_t i = 0; i < tests.size(); i++) results[i] = i < to_run && passed_[i] == (int32_t)rounds;
    }

   private:
    static void check(int rc, const char *what) {
        if (rc != PG_OK) throw std::runtime_error(std::string(what) + ": " + pg_last_error());
    }
    pg_ctx *ctx_ = nullptr;
    const size_t words_;
    std::vector<uint32_t> limbs_;
    std::vector<int32_t> passed_;
};
