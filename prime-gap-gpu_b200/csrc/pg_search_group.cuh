// pg_search_group.cuh -- the PRP kernels of pg_search.cuh for operands spread
// over a group of T lanes (pg_group.cuh): the same work items, queue, refill
// and first-prime rule, with a group instead of a lane holding an item.
//
// Each (T, LT) is instantiated in its own translation unit (pg_ginst.cu with
// -DPG_GT=T -DPG_GLT=LT); pg_dispatch.cu maps a job's operand width to one.
#pragma once

#include "pg_group.cuh"
#include "pg_search.cuh"

namespace pg {

// the group's slice of m*K + 2Y (next side) or m*K - 2Y (prev side)
template <int T, int LT>
__device__ __forceinline__ void gbuild_candidate(const Group<T> &G, const uint32_t *__restrict__ K, uint64_t m,
                                                 uint32_t Y, bool prev, uint32_t (&x)[LT]) {
    const uint32_t ml = (uint32_t)m, mh = (uint32_t)(m >> 32);
    uint32_t ks[LT], kh[LT];
#pragma unroll
    for (int k = 0; k < LT; k++) {
        const int wi = (int)(G.gl * LT) + k;
        ks[k] = __ldg(K + wi);
        kh[k] = wi > 0 ? __ldg(K + wi - 1) : 0u;  // K shifted up one word, for the high half of m
    }
#pragma unroll
    for (int k = 0; k < LT; k++) x[k] = 0;
    uint64_t spill = 0;
    row_mac<LT>(x, spill, ml, ks);
    if (mh) row_mac<LT>(x, spill, mh, kh);
    const uint32_t lo = __shfl_up_sync(G.gmask, (uint32_t)spill, 1);
    const uint32_t hi = __shfl_up_sync(G.gmask, (uint32_t)(spill >> 32), 1);
    resolve_in<T, LT>(G, x, G.gl == 0 ? 0ull : ((uint64_t)hi << 32 | lo));
    const uint32_t X = 2 * Y;
    if (!prev) {
        resolve_in<T, LT>(G, x, G.gl == 0 ? (uint64_t)X : 0ull);
    } else {
        uint32_t xs[LT];
#pragma unroll
        for (int k = 0; k < LT; k++) xs[k] = (G.gl == 0 && k == 0) ? X : 0u;
        uint32_t d[LT];
        group_sub<T, LT>(G, d, x, xs);
#pragma unroll
        for (int k = 0; k < LT; k++) x[k] = d[k];
    }
}

// bases passed (2, 3, 5, ...) of the group-held odd n
template <int T, int LT>
__device__ __forceinline__ int gprp_rounds(const Group<T> &G, const uint32_t (&n)[LT], int rounds) {
    const uint32_t bases[16] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53};
    uint32_t hi = 0;
#pragma unroll
    for (int k = 0; k < LT; k++) hi |= (G.gl == 0 && k == 0) ? 0u : n[k];
    const bool big = G.field(__ballot_sync(G.gmask, hi != 0)) != 0;
    const uint32_t n0 = __shfl_sync(G.gmask, n[0], G.gb);
    if ((n0 & 1u) == 0 || (!big && n0 < 3)) return 0;
    int passed = 0;
    for (int r = 0; r < rounds && r < 16; r++) {
        const bool tiny = !big && n0 - 1 <= bases[r];
        if (!tiny && !gstrong_prp<T, LT>(G, n, bases[r])) break;
        passed++;
    }
    return passed;
}

template <int T, int LT>
__global__ void __launch_bounds__(128) k_prp_batch_g(const uint32_t *__restrict__ cand, uint32_t words, uint32_t n,
                                                     uint32_t rounds, int32_t *__restrict__ out) {
    const Group<T> G;
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) / T;
    if (i >= n) return;  // whole groups leave together
    uint32_t x[LT];
#pragma unroll
    for (int k = 0; k < LT; k++) {
        const uint32_t wi = G.gl * LT + k;
        x[k] = wi < words ? cand[(size_t)i * words + wi] : 0u;
    }
    const int passed = gprp_rounds<T, LT>(G, x, (int)rounds);
    if (G.gl == 0) out[i] = passed;
}

// Persistent search with one item per group (see k_search_persistent).
template <int T, int LT>
__global__ void __launch_bounds__(PERSIST_THREADS) k_search_persistent_g(const __grid_constant__ SearchArgs a) {
    const unsigned FULL = 0xffffffffu;
    const Group<T> G;
    uint32_t kspan = a.kspan;
    if (a.max_count) kspan = min(kspan, *a.max_count + a.ext_max);
    const unsigned long long total = (unsigned long long)a.n_act * kspan;
    bool have = false, exhausted = false;
    uint32_t s = 0, k = 0, Y = 0;
    unsigned long long ntests = 0;
    while (true) {
        __syncwarp();
        if (a.stop && !exhausted) stop_check(a, total, exhausted);
        if (a.drain_lanes && !exhausted) {
            int retire = 0;
            if (G.lane == 0) {
                const uint32_t u = *(volatile const uint32_t *)a.unresolved;
                const uint32_t w = *(volatile const uint32_t *)a.active_warps;
                if ((unsigned long long)u * a.drain_lanes < (unsigned long long)w * (32 / T) &&
                    w > a.min_warps) {
                    if (atomicSub(a.active_warps, 1u) > a.min_warps)
                        retire = 1;
                    else
                        atomicAdd(a.active_warps, 1u);
                }
            }
            if (__shfl_sync(FULL, retire, 0)) break;
        }
        while (!exhausted) {
            const unsigned need = __ballot_sync(FULL, !have && G.gl == 0);  // group leaders without work
            if (need == 0) break;
            const int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if ((int)G.lane == leader) base = atomicAdd(a.next_item, (unsigned long long)__popc(need));
            base = __shfl_sync(FULL, base, leader);
            if (base >= total) {
                exhausted = true;
                break;
            }
            if (!have) {
                const unsigned long long t = base + __popc(need & ((1u << G.gb) - 1));
                if (t < total) {
                    const uint32_t kk = (uint32_t)(t / a.n_act);
                    const uint32_t i = (uint32_t)(t - (unsigned long long)kk * a.n_act);
                    s = a.act[i];
                    k = a.k_start[s] + kk;
                    have = pick_item(a, s, k, Y);
                }
            }
        }
        if (!__any_sync(FULL, have)) break;
        if (have) {
            uint32_t x[LT];
            gbuild_candidate<T, LT>(G, win_of(a, s).K, a.ms[s >> 1], Y, s & 1, x);
            const bool pr = gstrong_prp<T, LT>(G, x, 2);
            if (G.gl == 0) {
                ntests++;
                if (pr && atomicMin(&a.found_k[s], k) == NOT_FOUND && a.unresolved) atomicSub(a.unresolved, 1u);
            }
            have = false;
        }
    }
    __syncwarp();
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ntests += __shfl_down_sync(FULL, ntests, o);
    if (G.lane == 0 && ntests) atomicAdd(a.tests, ntests);
}

// Plain form: one group per active side tests that side's next candidate.
template <int T, int LT>
__global__ void __launch_bounds__(128) k_search_plain_g(const __grid_constant__ SearchArgs a, uint32_t *k_next) {
    const Group<T> G;
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) / T;
    if (i >= a.n_act) return;
    const uint32_t s = a.act[i];
    uint32_t k = k_next[s], Y = 0;
    const uint32_t lim = a.counts[s] + a.ext_max;
    while (true) {
        if (k >= lim) {
            __syncwarp(G.gmask);
            if (G.gl == 0) k_next[s] = k;
            return;
        }
        if (pick_item(a, s, k, Y)) break;
        k++;
    }
    uint32_t x[LT];
    gbuild_candidate<T, LT>(G, win_of(a, s).K, a.ms[s >> 1], Y, s & 1, x);
    const bool pr = gstrong_prp<T, LT>(G, x, 2);
    if (G.gl == 0) {
        if (pr) a.found_k[s] = k;
        k_next[s] = k + 1;
        atomicAdd(a.tests, 1ull);
    }
}

template <int T, int LT>
__global__ void __launch_bounds__(128) k_finalize_g(const __grid_constant__ SearchArgs a, uint32_t nsides,
                                                    uint32_t *gaps, uint32_t *redo, uint32_t *n_redo,
                                                    unsigned long long *confirm_tests, uint32_t *k_start_rw) {
    const Group<T> G;
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) / T;
    if (i >= a.n_act) return;
    if (a.stopped && *(volatile const uint32_t *)a.stopped) return;  // preempted: resumed later
    (void)nsides;
    const uint32_t s = a.act[i];
    const uint32_t k = a.found_k[s];
    if (k == NOT_FOUND) {
        if (G.gl == 0) {
            gaps[s] = 0;
            k_start_rw[s] = a.counts[s] + a.ext_max;
            redo[atomicAdd(n_redo, 1u)] = s;
        }
        return;
    }
    const uint32_t Y = item_y(a, s, k);
    const WinInfo &w = win_of(a, s);
    if (w.rounds > 1) {
        const uint32_t bases[16] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53};
        uint32_t x[LT];
        gbuild_candidate<T, LT>(G, w.K, a.ms[s >> 1], Y, s & 1, x);
        bool ok = true;
        for (uint32_t r = 1; r < w.rounds && r < 16; r++) {
            if (G.gl == 0) atomicAdd(confirm_tests, 1ull);
            if (!gstrong_prp<T, LT>(G, x, bases[r])) {
                ok = false;
                break;
            }
        }
        if (!ok) {
            if (G.gl == 0) {
                a.found_k[s] = NOT_FOUND;
                gaps[s] = 0;
                k_start_rw[s] = k + 1;
                redo[atomicAdd(n_redo, 1u)] = s;
            }
            return;
        }
    }
    if (G.gl == 0) gaps[s] = 2 * Y;
}

// Record confirmation (k_confirm) for lane-group operands: one warp per side,
// its 32/T groups taking the extra bases in turn.
template <int T, int LT>
__global__ void __launch_bounds__(128) k_confirm_g(const __grid_constant__ SearchArgs a, uint32_t *gaps,
                                                   uint32_t *conf, uint32_t *redo, uint32_t *n_redo,
                                                   unsigned long long *confirm_tests, uint32_t *k_start_rw) {
    const Group<T> G;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= a.n_act) return;
    const uint32_t s = a.act[warp];
    const WinInfo &w = win_of(a, s);
    const uint32_t k = a.found_k[s];
    if (w.confirm_rounds < 2 || k == NOT_FOUND || conf[s] == k) return;
    const uint32_t g = gaps[s], g2 = gaps[s ^ 1u];
    if (g == 0 || g2 == 0) return;
    const uint64_t m = a.ms[s >> 1];
    const double merit = (double)(g + g2) / (w.k_log + log((double)m));
    if (!(merit > w.confirm_merit - CONFIRM_MARGIN)) return;
    const uint32_t bases[16] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53};
    const uint32_t extra = min(w.confirm_rounds, 16u) - 1;
    uint32_t x[LT];
    gbuild_candidate<T, LT>(G, w.K, m, g >> 1, s & 1, x);
    bool ok = true;
    for (uint32_t b = G.gb / T; b < extra; b += 32 / T)
        if (!gstrong_prp<T, LT>(G, x, bases[b + 1])) ok = false;
    const bool all = __all_sync(0xffffffffu, ok);
    if (G.lane == 0) {
        atomicAdd(confirm_tests, (unsigned long long)extra);
        if (all) {
            conf[s] = k;
        } else {
            a.found_k[s] = NOT_FOUND;
            gaps[s] = 0;
            k_start_rw[s] = k + 1;
            redo[atomicAdd(n_redo, 1u)] = s;
        }
    }
}

// ------------------------------------------------------------ launchers

template <int T, int LT>
cudaError_t glaunch_prp_batch(const uint32_t *cand, uint32_t words, uint32_t n, uint32_t rounds, int32_t *out,
                              cudaStream_t st) {
    const uint64_t threads = (uint64_t)n * T;
    k_prp_batch_g<T, LT><<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(cand, words, n, rounds, out);
    return cudaGetLastError();
}

template <int T, int LT>
int gsearch_occupancy() {
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_search_persistent_g<T, LT>, PERSIST_THREADS, 0);
    return per;
}

template <int T, int LT>
cudaError_t glaunch_search_persistent(const SearchArgs &a, int grid, cudaStream_t st) {
    k_search_persistent_g<T, LT><<<grid, PERSIST_THREADS, 0, st>>>(a);
    return cudaGetLastError();
}

template <int T, int LT>
cudaError_t glaunch_search_plain(const SearchArgs &a, uint32_t *k_next, cudaStream_t st) {
    const uint64_t threads = (uint64_t)a.n_act * T;
    k_search_plain_g<T, LT><<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(a, k_next);
    return cudaGetLastError();
}

template <int T, int LT>
cudaError_t glaunch_finalize(const SearchArgs &a, uint32_t nsides, uint32_t *gaps, uint32_t *redo, uint32_t *n_redo,
                             unsigned long long *confirm_tests, uint32_t *k_start_rw, cudaStream_t st) {
    const uint64_t threads = (uint64_t)a.n_act * T;
    k_finalize_g<T, LT><<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(a, nsides, gaps, redo, n_redo,
                                                                          confirm_tests, k_start_rw);
    return cudaGetLastError();
}

template <int T, int LT>
cudaError_t glaunch_confirm(const SearchArgs &a, uint32_t *gaps, uint32_t *conf, uint32_t *redo, uint32_t *n_redo,
                            unsigned long long *confirm_tests, uint32_t *k_start_rw, cudaStream_t st) {
    const uint64_t threads = (uint64_t)a.n_act * 32;
    k_confirm_g<T, LT><<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(a, gaps, conf, redo, n_redo,
                                                                          confirm_tests, k_start_rw);
    return cudaGetLastError();
}

#define PG_GDECLARE(T, LT)                                                                                        \
    extern template cudaError_t glaunch_prp_batch<T, LT>(const uint32_t *, uint32_t, uint32_t, uint32_t,         \
                                                         int32_t *, cudaStream_t);                               \
    extern template int gsearch_occupancy<T, LT>();                                                               \
    extern template cudaError_t glaunch_search_persistent<T, LT>(const SearchArgs &, int, cudaStream_t);         \
    extern template cudaError_t glaunch_search_plain<T, LT>(const SearchArgs &, uint32_t *, cudaStream_t);       \
    extern template cudaError_t glaunch_finalize<T, LT>(const SearchArgs &, uint32_t, uint32_t *, uint32_t *,    \
                                                        uint32_t *, unsigned long long *, uint32_t *, cudaStream_t); \
    extern template cudaError_t glaunch_confirm<T, LT>(const SearchArgs &, uint32_t *, uint32_t *, uint32_t *,   \
                                                       uint32_t *, unsigned long long *, uint32_t *, cudaStream_t);

#define PG_GINSTANTIATE(T, LT)                                                                                    \
    template cudaError_t glaunch_prp_batch<T, LT>(const uint32_t *, uint32_t, uint32_t, uint32_t, int32_t *,     \
                                                  cudaStream_t);                                                  \
    template int gsearch_occupancy<T, LT>();                                                                      \
    template cudaError_t glaunch_search_persistent<T, LT>(const SearchArgs &, int, cudaStream_t);                \
    template cudaError_t glaunch_search_plain<T, LT>(const SearchArgs &, uint32_t *, cudaStream_t);              \
    template cudaError_t glaunch_finalize<T, LT>(const SearchArgs &, uint32_t, uint32_t *, uint32_t *,           \
                                                 uint32_t *, unsigned long long *, uint32_t *, cudaStream_t);    \
    template cudaError_t glaunch_confirm<T, LT>(const SearchArgs &, uint32_t *, uint32_t *, uint32_t *,          \
                                                uint32_t *, unsigned long long *, uint32_t *, cudaStream_t);

}  // namespace pg
