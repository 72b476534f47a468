// pg_search.cuh -- PRP kernels templated on the limb count L.
//
//   k_prp_batch          strong PRP of a batch (miller_rabin.h:252-270)
//   k_search_persistent  persistent PRP search with a device work queue
//                        (replaces gpu_testing.cu:203-350 and the CPU overflow
//                        threads of overflow.cpp:61-227)
//   k_search_plain       one PRP per active side per launch
//   k_finalize           gaps, confirmation bases, continuation list
//
// Each L is instantiated in its own translation unit (pg_inst.cu compiled
// with -DPG_LIMBS=L) so the fully unrolled kernels build in parallel;
// pg_dispatch.cu maps a runtime L to the instantiation.
#pragma once

#include "pg_internal.h"
#include "pg_mont.cuh"

// minimum resident one-warp blocks per SM requested from ptxas for the
// persistent search (caps its registers); 1 leaves the choice to ptxas
#ifndef PG_PERSIST_MIN_BLOCKS
#define PG_PERSIST_MIN_BLOCKS 1
#endif

namespace pg {

// ================================================================= PRP

template <int L>
__global__ void __launch_bounds__(128) k_prp_batch(const uint32_t *__restrict__ cand, uint32_t words, uint32_t n,
                                                   uint32_t rounds, int32_t *__restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t x[L];
#pragma unroll
    for (int k = 0; k < L; k++) x[k] = ((uint32_t)k < words) ? cand[(size_t)i * words + k] : 0u;
    out[i] = prp_rounds<L>(x, (int)rounds);
}

// ------------------------------------------------------------ search core

// the window of side s
__device__ __forceinline__ const WinInfo &win_of(const SearchArgs &a, uint32_t s) {
    return a.win[a.wid ? a.wid[s >> 1] : 0u];
}

// m*K + 2Y (next side) or m*K - 2Y (prev side); K has at least L words
template <int L>
__device__ __forceinline__ void build_candidate(const uint32_t *__restrict__ K, uint64_t m, uint32_t Y, bool prev,
                                                uint32_t (&x)[L]) {
    uint32_t kw[L];
#pragma unroll
    for (int k = 0; k < L; k++) kw[k] = __ldg(K + k);
    const uint32_t ml = (uint32_t)m, mh = (uint32_t)(m >> 32);
    uint32_t carry = 0;
#pragma unroll
    for (int k = 0; k < L; k++) {
        const uint64_t p = (uint64_t)kw[k] * ml + carry;
        x[k] = (uint32_t)p;
        carry = (uint32_t)(p >> 32);
    }
    if (mh) {
        carry = 0;
#pragma unroll
        for (int k = 1; k < L; k++) {
            const uint64_t p = (uint64_t)kw[k - 1] * mh + x[k] + carry;
            x[k] = (uint32_t)p;
            carry = (uint32_t)(p >> 32);
        }
    }
    const uint32_t X = 2 * Y;
    if (!prev) {
        x[0] = add_cc(x[0], X);
#pragma unroll
        for (int k = 1; k < L; k++) x[k] = (k + 1 < L) ? addc_cc(x[k], 0u) : addc(x[k], 0u);
    } else {
        x[0] = sub_cc(x[0], X);
#pragma unroll
        for (int k = 1; k < L; k++) x[k] = (k + 1 < L) ? subc_cc(x[k], 0u) : subc(x[k], 0u);
    }
}

__device__ __forceinline__ uint32_t load_found(const uint32_t *p) { return *(volatile const uint32_t *)p; }

// Preemption check of a persistent search warp (a.stop set), called by the
// whole warp: once the flag is raised the warp takes no more items
// (exhausted); if items are still queued the launch is marked stopped, so
// finalize skips it and the host resumes it.  Lane 0 reads the flags.
__device__ __forceinline__ void stop_check(const SearchArgs &a, unsigned long long total, bool &exhausted) {
    const bool lead = (threadIdx.x & 31) == 0;
    uint32_t st = 0;
    if (lead) st = *a.stop;
    if (__shfl_sync(0xffffffffu, st, 0)) {
        exhausted = true;
        if (lead && *(volatile unsigned long long *)a.next_item < total) atomicExch(a.stopped, 1u);
    }
}

// Resolves work item (side s, k-th candidate) to its position Y, or returns
// false when the item needs no test: the side already has a probable prime
// at a smaller k, the item lies past this launch's extension window, or an
// extension position (past sl, where there is no sieve row) has a factor
// among the trial primes.
__device__ __forceinline__ bool pick_item(const SearchArgs &a, uint32_t s, uint32_t k, uint32_t &Y) {
    if (load_found(&a.found_k[s]) < k) return false;
    const uint32_t cnt = a.counts[s];
    if (k < cnt) {
        Y = a.lists[(size_t)s * a.cap + k];
        return true;
    }
    const uint32_t ext = k - cnt;
    if (ext >= a.ext_max) return false;
    const WinInfo &w = win_of(a, s);
    Y = w.sly + 1 + ext;
    const uint64_t m = a.ms[s >> 1];
    const bool prev = s & 1;
    for (uint32_t i = 0; i < a.ntrial; i++) {
        const uint32_t q = a.trial_q[i];
        const uint32_t y0 = (uint32_t)(((m % q) * w.trial_r[i]) % q);
        const uint32_t yq = Y % q;
        const uint32_t ys = prev ? (yq ? q - yq : 0u) : yq;
        if (ys == y0) return false;
    }
    return true;
}

__device__ __forceinline__ uint32_t item_y(const SearchArgs &a, uint32_t s, uint32_t k) {
    const uint32_t cnt = a.counts[s];
    return k < cnt ? (uint32_t)a.lists[(size_t)s * a.cap + k] : win_of(a, s).sly + 1 + (k - cnt);
}

// Persistent search.  Items t = kk * n_act + i stand for the kk-th candidate
// (after k_start) of active side i, so the queue hands out the nearest
// untested candidate of every side first.  Each lane of a warp holds one
// item; lanes whose item is resolved or composite by trial division are
// refilled from the queue before the warp runs its next round of tests, so
// the 32 lanes stay busy while survivor counts and prime distances differ.
// A side is resolved by the smallest k with a probable prime: every smaller
// k is tested because items are only skipped behind a smaller found k.
template <int L>
__global__ void __launch_bounds__(PERSIST_THREADS, PG_PERSIST_MIN_BLOCKS) k_search_persistent(const __grid_constant__ SearchArgs a) {
    const unsigned FULL = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31;
    uint32_t kspan = a.kspan;
    if (a.max_count) kspan = min(kspan, *a.max_count + a.ext_max);
    const unsigned long long total = (unsigned long long)a.n_act * kspan;
    bool have = false, exhausted = false;
    uint32_t s = 0, k = 0, Y = 0;
    unsigned long long ntests = 0;
    while (true) {
        if (a.stop && !exhausted) stop_check(a, total, exhausted);
        // Draining: once the unresolved sides are few, extra lanes would only
        // test candidates beyond a prime about to be found; such a warp leaves
        // (with no item in hand) so its SM slot can run other work.  The last
        // min_warps warps never leave, so every item is still handed out.
        if (a.drain_lanes && !exhausted) {
            int retire = 0;
            if (lane == 0) {
                const uint32_t u = *(volatile const uint32_t *)a.unresolved;
                const uint32_t w = *(volatile const uint32_t *)a.active_warps;
                if ((unsigned long long)u * a.drain_lanes < (unsigned long long)w * 32 && w > a.min_warps) {
                    if (atomicSub(a.active_warps, 1u) > a.min_warps)
                        retire = 1;
                    else
                        atomicAdd(a.active_warps, 1u);
                }
            }
            if (__shfl_sync(FULL, retire, 0)) break;
        }
        while (!exhausted) {
            const unsigned need = __ballot_sync(FULL, !have);
            if (need == 0) break;
            const int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) base = atomicAdd(a.next_item, (unsigned long long)__popc(need));
            base = __shfl_sync(FULL, base, leader);
            if (base >= total) {
                exhausted = true;
                break;
            }
            if (!have) {
                const unsigned long long t = base + __popc(need & ((1u << lane) - 1));
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
            uint32_t x[L];
            build_candidate<L>(win_of(a, s).K, a.ms[s >> 1], Y, s & 1, x);
            const bool pr = strong_prp<L>(x, 2);
            ntests++;
            if (pr && atomicMin(&a.found_k[s], k) == NOT_FOUND && a.unresolved) atomicSub(a.unresolved, 1u);
            have = false;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ntests += __shfl_down_sync(FULL, ntests, o);
    if (lane == 0 && ntests) atomicAdd(a.tests, ntests);
}

// Plain form: one thread per active side tests that side's next candidate.
template <int L>
__global__ void __launch_bounds__(128) k_search_plain(const __grid_constant__ SearchArgs a, uint32_t *k_next) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_act) return;
    const uint32_t s = a.act[i];
    uint32_t k = k_next[s], Y = 0;
    const uint32_t lim = a.counts[s] + a.ext_max;
    while (true) {
        if (k >= lim) {
            k_next[s] = k;
            return;
        }
        if (pick_item(a, s, k, Y)) break;
        k++;
    }
    uint32_t x[L];
    build_candidate<L>(win_of(a, s).K, a.ms[s >> 1], Y, s & 1, x);
    if (strong_prp<L>(x, 2)) a.found_k[s] = k;
    k_next[s] = k + 1;
    atomicAdd(a.tests, 1ull);
}

// gaps of resolved sides; extra-base confirmation; continuation list
template <int L>
__global__ void __launch_bounds__(128) k_finalize(const __grid_constant__ SearchArgs a, uint32_t nsides,
                                                  uint32_t *gaps, uint32_t *redo, uint32_t *n_redo,
                                                  unsigned long long *confirm_tests, uint32_t *k_start_rw) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_act) return;
    if (a.stopped && *(volatile const uint32_t *)a.stopped) return;  // preempted: resumed later
    const uint32_t s = a.act[i];
    (void)nsides;
    const uint32_t k = a.found_k[s];
    if (k == NOT_FOUND) {
        gaps[s] = 0;
        k_start_rw[s] = a.counts[s] + a.ext_max;  // continue past the window just searched
        redo[atomicAdd(n_redo, 1u)] = s;
        return;
    }
    const uint32_t Y = item_y(a, s, k);
    const WinInfo &w = win_of(a, s);
    if (w.rounds > 1) {
        const uint32_t bases[16] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53};
        uint32_t x[L];
        build_candidate<L>(w.K, a.ms[s >> 1], Y, s & 1, x);
        bool ok = true;
        for (uint32_t r = 1; r < w.rounds && r < 16; r++) {
            atomicAdd(confirm_tests, 1ull);
            if (!strong_prp<L>(x, bases[r])) {
                ok = false;
                break;
            }
        }
        if (!ok) {  // base-2 pseudoprime: search again from the next candidate
            a.found_k[s] = NOT_FOUND;
            gaps[s] = 0;
            k_start_rw[s] = k + 1;
            redo[atomicAdd(n_redo, 1u)] = s;
            return;
        }
    }
    gaps[s] = 2 * Y;
}

// Record confirmation, one warp per side (the double-check of overflow.cpp:
// 164-177 done on the device).  The search accepts a prime on one strong
// base-2 test; a composite that passes it (a base-2 pseudoprime) would end a
// gap early, while no prime is ever rejected (a prime passes every base and
// the sieve removes only multiples of its primes).  So a gap is exact once
// its two ends pass more bases: a side whose gap and partner gap are both
// known, with merit (prev + next) / (k_log + log m) above its window's
// confirm_merit, has its prime tested with bases 3, 5, ... (confirm_rounds in
// all, one base per lane).  A failure resets the side to search again from
// its next candidate; conf[s] keeps the k confirmed, so a later pass re-tests
// only sides whose prime changed.
template <int L>
__global__ void __launch_bounds__(128) k_confirm(const __grid_constant__ SearchArgs a, uint32_t *gaps, uint32_t *conf,
                                                 uint32_t *redo, uint32_t *n_redo,
                                                 unsigned long long *confirm_tests, uint32_t *k_start_rw) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= a.n_act) return;
    const uint32_t s = a.act[warp];
    const WinInfo &w = win_of(a, s);
    const uint32_t k = a.found_k[s];
    if (w.confirm_rounds < 2 || k == NOT_FOUND || conf[s] == k) return;
    const uint32_t g = gaps[s], g2 = gaps[s ^ 1u];
    if (g == 0 || g2 == 0) return;  // the other side is still open: a later pass decides
    const uint64_t m = a.ms[s >> 1];
    const double merit = (double)(g + g2) / (w.k_log + log((double)m));
    if (!(merit > w.confirm_merit - CONFIRM_MARGIN)) return;
    const uint32_t bases[16] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53};
    const uint32_t extra = min(w.confirm_rounds, 16u) - 1;
    bool ok = true;
    if (lane < extra) {
        uint32_t x[L];
        build_candidate<L>(w.K, m, g >> 1, s & 1, x);
        ok = strong_prp<L>(x, bases[lane + 1]);
    }
    const bool all = __all_sync(0xffffffffu, ok);
    if (lane == 0) {
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

template <int L>
cudaError_t launch_prp_batch_t(const uint32_t *cand, uint32_t words, uint32_t n, uint32_t rounds, int32_t *out,
                               cudaStream_t st) {
    const uint32_t threads = 128, blocks = (n + threads - 1) / threads;
    k_prp_batch<L><<<blocks, threads, 0, st>>>(cand, words, n, rounds, out);
    return cudaGetLastError();
}

template <int L>
int search_occupancy_t() {
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_search_persistent<L>, PERSIST_THREADS, 0);
    return per;
}

template <int L>
cudaError_t launch_search_persistent_t(const SearchArgs &a, int grid, cudaStream_t st) {
    k_search_persistent<L><<<grid, PERSIST_THREADS, 0, st>>>(a);
    return cudaGetLastError();
}

template <int L>
cudaError_t launch_search_plain_t(const SearchArgs &a, uint32_t *k_next, cudaStream_t st) {
    const uint32_t threads = 128, blocks = (a.n_act + threads - 1) / threads;
    k_search_plain<L><<<blocks, threads, 0, st>>>(a, k_next);
    return cudaGetLastError();
}

template <int L>
cudaError_t launch_finalize_t(const SearchArgs &a, uint32_t nsides, uint32_t *gaps, uint32_t *redo, uint32_t *n_redo,
                              unsigned long long *confirm_tests, uint32_t *k_start_rw, cudaStream_t st) {
    const uint32_t threads = 128, blocks = (a.n_act + threads - 1) / threads;
    k_finalize<L><<<blocks, threads, 0, st>>>(a, nsides, gaps, redo, n_redo, confirm_tests, k_start_rw);
    return cudaGetLastError();
}

template <int L>
cudaError_t launch_confirm_t(const SearchArgs &a, uint32_t *gaps, uint32_t *conf, uint32_t *redo, uint32_t *n_redo,
                             unsigned long long *confirm_tests, uint32_t *k_start_rw, cudaStream_t st) {
    const uint64_t threads = (uint64_t)a.n_act * 32;
    k_confirm<L><<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(a, gaps, conf, redo, n_redo, confirm_tests,
                                                                    k_start_rw);
    return cudaGetLastError();
}

#define PG_DECLARE_LIMBS(L)                                                                                       \
    extern template cudaError_t launch_prp_batch_t<L>(const uint32_t *, uint32_t, uint32_t, uint32_t, int32_t *,  \
                                                      cudaStream_t);                                              \
    extern template int search_occupancy_t<L>();                                                                  \
    extern template cudaError_t launch_search_persistent_t<L>(const SearchArgs &, int, cudaStream_t);            \
    extern template cudaError_t launch_search_plain_t<L>(const SearchArgs &, uint32_t *, cudaStream_t);          \
    extern template cudaError_t launch_finalize_t<L>(const SearchArgs &, uint32_t, uint32_t *, uint32_t *,       \
                                                     uint32_t *, unsigned long long *, uint32_t *, cudaStream_t); \
    extern template cudaError_t launch_confirm_t<L>(const SearchArgs &, uint32_t *, uint32_t *, uint32_t *,      \
                                                    uint32_t *, unsigned long long *, uint32_t *, cudaStream_t);

#define PG_INSTANTIATE_LIMBS(L)                                                                                   \
    template cudaError_t launch_prp_batch_t<L>(const uint32_t *, uint32_t, uint32_t, uint32_t, int32_t *,         \
                                               cudaStream_t);                                                     \
    template int search_occupancy_t<L>();                                                                         \
    template cudaError_t launch_search_persistent_t<L>(const SearchArgs &, int, cudaStream_t);                   \
    template cudaError_t launch_search_plain_t<L>(const SearchArgs &, uint32_t *, cudaStream_t);                 \
    template cudaError_t launch_finalize_t<L>(const SearchArgs &, uint32_t, uint32_t *, uint32_t *, uint32_t *,  \
                                              unsigned long long *, uint32_t *, cudaStream_t);                  \
    template cudaError_t launch_confirm_t<L>(const SearchArgs &, uint32_t *, uint32_t *, uint32_t *, uint32_t *,  \
                                             unsigned long long *, uint32_t *, cudaStream_t);

}  // namespace pg
