// pg_dispatch.cu -- maps a runtime limb count to its compiled instantiation.
#include "pg_limbs.h"
#include "pg_search.cuh"

namespace pg {

#define PG_DECL(n) PG_DECLARE_LIMBS(n)
PG_LIMB_LIST(PG_DECL)
#undef PG_DECL

bool supported_limbs(uint32_t L) {
#define PG_CASE(n) \
    if (L == n) return true;
    PG_LIMB_LIST(PG_CASE)
#undef PG_CASE
    return false;
}

uint32_t pick_limbs(uint32_t words) {
    uint32_t best = 0;
#define PG_CASE(n) \
    if (best == 0 && (uint32_t)n >= words) best = n;
    PG_LIMB_LIST(PG_CASE)
#undef PG_CASE
    return best;
}

cudaError_t launch_prp_batch(uint32_t L, const uint32_t *cand, uint32_t words, uint32_t n, uint32_t rounds,
                             int32_t *out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
#define PG_CASE(nl) \
    if (L == nl) return launch_prp_batch_t<nl>(cand, words, n, rounds, out, st);
    PG_LIMB_LIST(PG_CASE)
#undef PG_CASE
    return cudaErrorInvalidValue;
}

int search_grid(uint32_t L, int device) {
    int sms = 0, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
#define PG_CASE(nl) \
    if (L == nl) per = search_occupancy_t<nl>();
    PG_LIMB_LIST(PG_CASE)
#undef PG_CASE
    if (per < 1) per = 1;
    return sms * per;
}

cudaError_t launch_search_persistent(uint32_t L, const SearchArgs &a, int grid, cudaStream_t st) {
    if (a.n_act == 0) return cudaSuccess;
#define PG_CASE(nl) \
    if (L == nl) return launch_search_persistent_t<nl>(a, grid, st);
    PG_LIMB_LIST(PG_CASE)
#undef PG_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_search_plain(uint32_t L, const SearchArgs &a, uint32_t *k_next, cudaStream_t st) {
    if (a.n_act == 0) return cudaSuccess;
#define PG_CASE(nl) \
    if (L == nl) return launch_search_plain_t<nl>(a, k_next, st);
    PG_LIMB_LIST(PG_CASE)
#undef PG_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_finalize(uint32_t L, const SearchArgs &a, uint32_t nsides, uint32_t *gaps, uint32_t *redo,
                            uint32_t *n_redo, unsigned long long *confirm_tests, uint32_t *k_start_rw,
                            cudaStream_t st) {
    if (a.n_act == 0) return cudaSuccess;
#define PG_CASE(nl) \
    if (L == nl) return launch_finalize_t<nl>(a, nsides, gaps, redo, n_redo, confirm_tests, k_start_rw, st);
    PG_LIMB_LIST(PG_CASE)
#undef PG_CASE
    return cudaErrorInvalidValue;
}

}  // namespace pg
