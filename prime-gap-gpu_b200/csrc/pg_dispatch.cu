// pg_dispatch.cu -- maps a runtime operand layout to its compiled kernels.
//
// A layout code is L (one thread per number, L words) or (T << 16) | L (a
// group of T lanes per number, L/T words per lane); see pg_limbs.h.
#include "pg_limbs.h"
#include "pg_search.cuh"
#include "pg_search_group.cuh"

namespace pg {

#define PG_DECL(n) PG_DECLARE_LIMBS(n)
PG_LIMB_LIST(PG_DECL)
#undef PG_DECL
#define PG_GDECL(t, lt) PG_GDECLARE(t, lt)
PG_GROUP_LIST(PG_GDECL)
#undef PG_GDECL

bool supported_limbs(uint32_t L) {
#define PG_CASE(n) \
    if (L == n) return true;
    PG_LIMB_LIST(PG_CASE)
#undef PG_CASE
#define PG_GCASE(t, lt) \
    if (L == PG_LAYOUT_GROUP(t, (t) * (lt))) return true;
    PG_GROUP_LIST(PG_GCASE)
#undef PG_GCASE
    return false;
}

uint32_t pick_layout(uint32_t bits, uint32_t tpi) {
    uint32_t best = 0;
    if (tpi <= 1) {
#define PG_CASE(n) \
    if (best == 0 && 32u * (n) >= bits) best = n;
        PG_LIMB_LIST(PG_CASE)
#undef PG_CASE
        if (best || tpi == 1) return best;
    }
    uint32_t bestL = 0;
#define PG_GCASE(t, lt)                                                                                 \
    if ((tpi == 0 || tpi == (uint32_t)(t)) && 32u * (t) * (lt) >= bits + 2 &&                           \
        (bestL == 0 || (uint32_t)((t) * (lt)) < bestL)) {                                               \
        bestL = (t) * (lt);                                                                             \
        best = PG_LAYOUT_GROUP(t, (t) * (lt));                                                          \
    }
    PG_GROUP_LIST(PG_GCASE)
#undef PG_GCASE
    return best;
}

uint32_t pick_limbs(uint32_t words) { return pick_layout(32 * words, 0); }

uint32_t layout_words(uint32_t layout) { return layout & 0xffffu; }

cudaError_t launch_prp_batch(uint32_t L, const uint32_t *cand, uint32_t words, uint32_t n, uint32_t rounds,
                             int32_t *out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
#define PG_CASE(nl) \
    if (L == nl) return launch_prp_batch_t<nl>(cand, words, n, rounds, out, st);
    PG_LIMB_LIST(PG_CASE)
#undef PG_CASE
#define PG_GCASE(t, lt) \
    if (L == PG_LAYOUT_GROUP(t, (t) * (lt))) return glaunch_prp_batch<t, lt>(cand, words, n, rounds, out, st);
    PG_GROUP_LIST(PG_GCASE)
#undef PG_GCASE
    return cudaErrorInvalidValue;
}

int search_grid(uint32_t L, int device) {
    int sms = 0, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
#define PG_CASE(nl) \
    if (L == nl) per = search_occupancy_t<nl>();
    PG_LIMB_LIST(PG_CASE)
#undef PG_CASE
#define PG_GCASE(t, lt) \
    if (L == PG_LAYOUT_GROUP(t, (t) * (lt))) per = gsearch_occupancy<t, lt>();
    PG_GROUP_LIST(PG_GCASE)
#undef PG_GCASE
    if (per < 1) per = 1;
    return sms * per;
}

cudaError_t launch_search_persistent(uint32_t L, const SearchArgs &a, int grid, cudaStream_t st) {
    if (a.n_act == 0) return cudaSuccess;
#define PG_CASE(nl) \
    if (L == nl) return launch_search_persistent_t<nl>(a, grid, st);
    PG_LIMB_LIST(PG_CASE)
#undef PG_CASE
#define PG_GCASE(t, lt) \
    if (L == PG_LAYOUT_GROUP(t, (t) * (lt))) return glaunch_search_persistent<t, lt>(a, grid, st);
    PG_GROUP_LIST(PG_GCASE)
#undef PG_GCASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_search_plain(uint32_t L, const SearchArgs &a, uint32_t *k_next, cudaStream_t st) {
    if (a.n_act == 0) return cudaSuccess;
#define PG_CASE(nl) \
    if (L == nl) return launch_search_plain_t<nl>(a, k_next, st);
    PG_LIMB_LIST(PG_CASE)
#undef PG_CASE
#define PG_GCASE(t, lt) \
    if (L == PG_LAYOUT_GROUP(t, (t) * (lt))) return glaunch_search_plain<t, lt>(a, k_next, st);
    PG_GROUP_LIST(PG_GCASE)
#undef PG_GCASE
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
#define PG_GCASE(t, lt)                                                                                    \
    if (L == PG_LAYOUT_GROUP(t, (t) * (lt)))                                                               \
        return glaunch_finalize<t, lt>(a, nsides, gaps, redo, n_redo, confirm_tests, k_start_rw, st);
    PG_GROUP_LIST(PG_GCASE)
#undef PG_GCASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_confirm(uint32_t L, const SearchArgs &a, uint32_t *gaps, uint32_t *conf, uint32_t *redo,
                           uint32_t *n_redo, unsigned long long *confirm_tests, uint32_t *k_start_rw,
                           cudaStream_t st) {
    if (a.n_act == 0) return cudaSuccess;
#define PG_CASE(nl) \
    if (L == nl) return launch_confirm_t<nl>(a, gaps, conf, redo, n_redo, confirm_tests, k_start_rw, st);
    PG_LIMB_LIST(PG_CASE)
#undef PG_CASE
#define PG_GCASE(t, lt)                                                                                    \
    if (L == PG_LAYOUT_GROUP(t, (t) * (lt)))                                                               \
        return glaunch_confirm<t, lt>(a, gaps, conf, redo, n_redo, confirm_tests, k_start_rw, st);
    PG_GROUP_LIST(PG_GCASE)
#undef PG_GCASE
    return cudaErrorInvalidValue;
}

}  // namespace pg
