// Uses include/primegap_runner.hpp exactly as gpu_testing.cu:217-218 and :274
// use miller_rabin.h: typedef mr_params_t<TPI, BITS, WINDOW>, construct
// test_runner_t<params>(batch, rounds), call run_test(active, z, results).
// Prints one line per candidate: "<index> <result>".
#include <cstdio>
#include <vector>

#include "primegap_runner.hpp"

int main() {
    typedef mr_params_t<8, 1024, 5> params;
    test_runner_t<params> runner(8, 1);
    const char *nums[] = {
        "6864797660130609714981900799081393217269435300143305409394463459185543183397656052122559640661454554977296311391480858037121987999716643812574028291115057151",  // 2^521-1
        "6864797660130609714981900799081393217269435300143305409394463459185543183397656052122559640661454554977296311391480858037121987999716643812574028291115057153",  // 2^521+1
        "2047",   // strong base-2 pseudoprime: passes like in the reference
        "101",
        "170141183460469231731687303715884105727",  // 2^127-1
        "170141183460469231731687303715884105729"};
    const size_t n = sizeof(nums) / sizeof(nums[0]);
    mpz_t *z = new mpz_t[n];
    std::vector<mpz_t *> tests;
    for (size_t i = 0; i < n; i++) {
        mpz_init(z[i]);
        mpz_set_str(z[i], nums[i], 10);
        tests.push_back(&z[i]);
    }
    std::vector<int> results(8, -1);
    runner.run_test(5, tests, results);
    for (size_t i = 0; i < n; i++) printf("%zu %d\n", i, results[i]);
    for (size_t i = 0; i < n; i++) mpz_clear(z[i]);
    delete[] z;
    return 0;
}
