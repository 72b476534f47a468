// pg_kernels.cu -- sm_100a kernels of the prime-gap search path.
//
//   k_prime_count / k_prime_write  segmented sieve of Eratosthenes in shared
//                                  memory: every prime in (P, max_prime]
//                                  (replaces primesieve, gap_search_gpu.cpp:480-500)
//   k_prime_tables                 K mod p and K^-1 mod p per prime
//                                  (mpz_fdiv_ui + _invert, gap_search_gpu.cpp:489-493)
//   k_sieve_large_step             large primes, one thread per prime, stepping
//                                  the residue through every X of the window
//                                  (the per-X loop of gap_search_gpu.cpp:651-689,
//                                  transposed so each prime is read once)
//   k_sieve_small                  small primes per m on a bit-packed shared
//                                  memory row, then ballot/popc compaction of
//                                  the survivors into per-side lists
//                                  (gap_search_gpu.cpp:586-639 and 710-755)
//   k_compact_active               active-side list of the plain form
// The PRP kernels, templated on the limb count, are in pg_search.cuh.
#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>

#include "pg_internal.h"

namespace pg {

// ================================================================ helpers

__device__ __forceinline__ uint64_t mod_u64(uint64_t x, uint64_t q) { return x % q; }

// a*b mod p for a, b < p < 2^40 without 128-bit arithmetic
__device__ __forceinline__ uint64_t mulmod40(uint64_t a, uint64_t b, uint64_t p) {
    if (p < (1ull << 32)) return (a * b) % p;
    const uint64_t bh = b >> 20, bl = b & 0xFFFFFull;
    uint64_t r = ((a * bh) % p << 20) % p;
    return (r + (a * bl) % p) % p;
}

// a^-1 mod p (gcd(a, p) = 1), extended Euclid on signed 64-bit state
__device__ __forceinline__ uint64_t invmod64(uint64_t a, uint64_t p) {
    int64_t t = 0, nt = 1, r = (int64_t)p, nr = (int64_t)(a % p);
    while (nr != 0) {
        const int64_t q = r / nr;
        int64_t tmp = t - q * nt;
        t = nt;
        nt = tmp;
        tmp = r - q * nr;
        r = nr;
        nr = tmp;
    }
    if (t < 0) t += (int64_t)p;
    return (uint64_t)t;
}

// x mod q with bar = floor((2^64-1)/q)
__device__ __forceinline__ uint32_t barrett64(uint64_t x, uint32_t q, uint64_t bar) {
    uint64_t r = x - __umul64hi(x, bar) * q;
    while (r >= q) r -= q;
    return (uint32_t)r;
}

// ======================================================= prime generation

constexpr uint32_t SEG_ODDS = 1u << 18;          // odd numbers per segment
constexpr uint32_t SEG_WORDS = SEG_ODDS / 32;    // 32 KB of shared memory
constexpr int SEG_THREADS = 512;
constexpr uint32_t COOP_LIMIT = 4096;            // base primes below this mark cooperatively

// Marks the odd composites of segment [v_lo, v_lo + 2*SEG_ODDS) in bm.
__device__ void segment_sieve(uint64_t v_lo, const uint32_t *base, uint32_t nbase, uint32_t *bm) {
    for (uint32_t w = threadIdx.x; w < SEG_WORDS; w += blockDim.x) bm[w] = 0;
    __syncthreads();
    const uint64_t v_end = v_lo + 2ull * (SEG_ODDS - 1);
    // cooperative marking for small base primes (many multiples each)
    for (uint32_t i = 0; i < nbase; i++) {
        const uint64_t q = base[i];
        if (q >= COOP_LIMIT || q * q > v_end) break;
        uint64_t st = q * q;
        if (st < v_lo) st = ((v_lo + q - 1) / q) * q;
        if ((st & 1) == 0) st += q;
        if (st > v_end) continue;
        const uint32_t idx0 = (uint32_t)((st - v_lo) >> 1);
        const uint32_t cnt = (SEG_ODDS - 1 - idx0) / (uint32_t)q + 1;
        for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x) {
            const uint32_t idx = idx0 + k * (uint32_t)q;
            atomicOr(&bm[idx >> 5], 1u << (idx & 31));
        }
    }
    // one thread per larger base prime
    for (uint32_t i = threadIdx.x; i < nbase; i += blockDim.x) {
        const uint64_t q = base[i];
        if (q < COOP_LIMIT) continue;
        if (q * q > v_end) break;
        uint64_t st = q * q;
        if (st < v_lo) st = ((v_lo + q - 1) / q) * q;
        if ((st & 1) == 0) st += q;
        for (uint64_t v = st; v <= v_end; v += 2 * q) {
            const uint32_t idx = (uint32_t)((v - v_lo) >> 1);
            atomicOr(&bm[idx >> 5], 1u << (idx & 31));
        }
    }
    __syncthreads();
}

// survivors (primes) of word w of a segment, restricted to v <= limit
__device__ __forceinline__ uint32_t segment_word(const uint32_t *bm, uint32_t w, uint64_t v_lo, uint64_t limit) {
    uint32_t bits = ~bm[w];
    const uint64_t v0 = v_lo + 64ull * w;  // value of bit 0
    if (v0 > limit) return 0;
    const uint64_t last = v0 + 62;
    if (last > limit) {
        const uint32_t keep = (uint32_t)((limit - v0) >> 1) + 1;  // bits 0 .. keep-1
        bits &= keep >= 32 ? 0xffffffffu : ((1u << keep) - 1);
    }
    return bits;
}

__global__ void __launch_bounds__(SEG_THREADS) k_prime_count(uint64_t v_first, uint64_t limit, const uint32_t *base,
                                                             uint32_t nbase, uint32_t *seg_counts) {
    __shared__ uint32_t bm[SEG_WORDS];
    const uint64_t v_lo = v_first + 2ull * SEG_ODDS * blockIdx.x;
    segment_sieve(v_lo, base, nbase, bm);
    uint32_t c = 0;
    for (uint32_t w = threadIdx.x; w < SEG_WORDS; w += blockDim.x) c += __popc(segment_word(bm, w, v_lo, limit));
    typedef cub::BlockReduce<uint32_t, SEG_THREADS> Reduce;
    __shared__ typename Reduce::TempStorage tmp;
    const uint32_t total = Reduce(tmp).Sum(c);
    if (threadIdx.x == 0) seg_counts[blockIdx.x] = total;
}

template <typename T>
__global__ void __launch_bounds__(SEG_THREADS) k_prime_write(uint64_t v_first, uint64_t limit, const uint32_t *base,
                                                             uint32_t nbase, const uint64_t *seg_offsets, T *out) {
    __shared__ uint32_t bm[SEG_WORDS];
    const uint64_t v_lo = v_first + 2ull * SEG_ODDS * blockIdx.x;
    segment_sieve(v_lo, base, nbase, bm);
    constexpr uint32_t PER = SEG_WORDS / SEG_THREADS;  // consecutive words per thread
    const uint32_t w0 = threadIdx.x * PER;
    uint32_t c = 0;
#pragma unroll
    for (uint32_t k = 0; k < PER; k++) c += __popc(segment_word(bm, w0 + k, v_lo, limit));
    typedef cub::BlockScan<uint32_t, SEG_THREADS> Scan;
    __shared__ typename Scan::TempStorage tmp;
    uint32_t off;
    Scan(tmp).ExclusiveSum(c, off);
    uint64_t pos = seg_offsets[blockIdx.x] + off;
    for (uint32_t k = 0; k < PER; k++) {
        uint32_t bits = segment_word(bm, w0 + k, v_lo, limit);
        while (bits) {
            const uint32_t b = __ffs(bits) - 1;
            bits &= bits - 1;
            out[pos++] = (T)(v_lo + 64ull * (w0 + k) + 2ull * b);
        }
    }
}

cudaError_t launch_prime_count(uint64_t v_first, uint64_t limit, const uint32_t *base, uint32_t nbase, uint32_t nseg,
                               uint32_t *seg_counts, cudaStream_t st) {
    if (nseg == 0) return cudaSuccess;
    k_prime_count<<<nseg, SEG_THREADS, 0, st>>>(v_first, limit, base, nbase, seg_counts);
    return cudaGetLastError();
}

cudaError_t launch_prime_write(uint64_t v_first, uint64_t limit, const uint32_t *base, uint32_t nbase, uint32_t nseg,
                               const uint64_t *seg_offsets, void *out, bool wide, cudaStream_t st) {
    if (nseg == 0) return cudaSuccess;
    if (wide)
        k_prime_write<uint64_t><<<nseg, SEG_THREADS, 0, st>>>(v_first, limit, base, nbase, seg_offsets, (uint64_t *)out);
    else
        k_prime_write<uint32_t><<<nseg, SEG_THREADS, 0, st>>>(v_first, limit, base, nbase, seg_offsets, (uint32_t *)out);
    return cudaGetLastError();
}

// ============================================================ prime tables

template <typename T>
__global__ void k_prime_tables(const uint32_t *K, uint32_t kwords, uint64_t np, const T *p, T *c, T *cinv) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const uint64_t q = p[i];
    uint64_t r = 0;
    if (q < (1ull << 32)) {
        for (int w = (int)kwords - 1; w >= 0; w--) r = ((r << 32) | K[w]) % q;
    } else {
        for (int w = (int)kwords - 1; w >= 0; w--) {
            r = ((r << 16) | (K[w] >> 16)) % q;
            r = ((r << 16) | (K[w] & 0xffffu)) % q;
        }
    }
    c[i] = (T)r;
    cinv[i] = (T)(r ? invmod64(r, q) : 0);
}

cudaError_t launch_prime_tables(const uint32_t *K, uint32_t kwords, uint64_t np, const void *p, void *c, void *cinv,
                                bool wide, cudaStream_t st) {
    if (np == 0) return cudaSuccess;
    const uint32_t threads = 256;
    const uint64_t blocks = (np + threads - 1) / threads;
    if (wide)
        k_prime_tables<uint64_t><<<(unsigned)blocks, threads, 0, st>>>(K, kwords, np, (const uint64_t *)p,
                                                                       (uint64_t *)c, (uint64_t *)cinv);
    else
        k_prime_tables<uint32_t><<<(unsigned)blocks, threads, 0, st>>>(K, kwords, np, (const uint32_t *)p,
                                                                       (uint32_t *)c, (uint32_t *)cinv);
    return cudaGetLastError();
}

// ========================================================= depth ordering

// The modular search's Euclid depth for a prime depends on p and K mod p
// (and on the window width), not on the window.  Ordering the primes of each
// sieve segment by that depth gives the threads of a warp equal trip counts;
// segments keep their order, so prime-table indices of segment boundaries
// still split the table by value.
constexpr uint32_t DEPTH_W = 8192;  // reference window width (2 * sly) for the ordering
constexpr int DEPTH_BINS = 64;

template <typename T>
__global__ void k_prime_depth(uint64_t np, const T *p, const T *c, uint8_t *depth) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    uint64_t M = p[i], A = M - c[i];  // A = -K mod p, c in [1, p)
    int d = 0;
    while (A > DEPTH_W + 1 && d < DEPTH_BINS - 1) {
        const uint64_t r = M % A;
        M = A;
        A = r;
        d++;
    }
    depth[i] = (uint8_t)d;
}

// One block per segment: counting sort of the segment's primes by depth.
template <typename T>
__global__ void __launch_bounds__(1024) k_prime_reorder(const uint64_t *seg_off, uint32_t nseg, uint64_t np,
                                                        const uint8_t *depth, const T *p, const T *c, const T *ci,
                                                        T *op, T *oc, T *oci) {
    __shared__ uint32_t hist[DEPTH_BINS];
    const uint64_t lo = seg_off[blockIdx.x];
    const uint64_t hi = blockIdx.x + 1 < nseg ? seg_off[blockIdx.x + 1] : np;
    if (threadIdx.x < DEPTH_BINS) hist[threadIdx.x] = 0;
    __syncthreads();
    for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) atomicAdd(&hist[depth[i]], 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (int b = 0; b < DEPTH_BINS; b++) {
            const uint32_t v = hist[b];
            hist[b] = acc;
            acc += v;
        }
    }
    __syncthreads();
    for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const uint64_t pos = lo + atomicAdd(&hist[depth[i]], 1u);
        op[pos] = p[i];
        oc[pos] = c[i];
        oci[pos] = ci[i];
    }
}

cudaError_t launch_prime_reorder(uint64_t np, uint32_t nseg, const uint64_t *seg_off, const void *p, const void *c,
                                 const void *ci, void *op, void *oc, void *oci, uint8_t *depth, bool wide,
                                 cudaStream_t st) {
    if (np == 0 || nseg == 0) return cudaSuccess;
    const uint32_t threads = 256;
    const uint64_t blocks = (np + threads - 1) / threads;
    if (wide) {
        k_prime_depth<uint64_t><<<(unsigned)blocks, threads, 0, st>>>(np, (const uint64_t *)p, (const uint64_t *)c,
                                                                      depth);
        k_prime_reorder<uint64_t><<<nseg, 1024, 0, st>>>(seg_off, nseg, np, depth, (const uint64_t *)p,
                                                         (const uint64_t *)c, (const uint64_t *)ci, (uint64_t *)op,
                                                         (uint64_t *)oc, (uint64_t *)oci);
    } else {
        k_prime_depth<uint32_t><<<(unsigned)blocks, threads, 0, st>>>(np, (const uint32_t *)p, (const uint32_t *)c,
                                                                      depth);
        k_prime_reorder<uint32_t><<<nseg, 1024, 0, st>>>(seg_off, nseg, np, depth, (const uint32_t *)p,
                                                         (const uint32_t *)c, (const uint32_t *)ci, (uint32_t *)op,
                                                         (uint32_t *)oc, (uint32_t *)oci);
    }
    return cudaGetLastError();
}

// ====================================================== large-prime sieve

__device__ __forceinline__ void mark_hit(const LargeArgs &a, uint64_t j, uint32_t idx) {
    const int32_t r = a.rank[j];
    if (r >= 0) atomicOr(&a.bitmaps[(size_t)r * a.words + (idx >> 5)], 1u << (idx & 31));
}

// The same, skipping positions the K-prime wheel already marks in every row
// (about two thirds of them at P = 503: Y = 0 and every Y with a factor
// q | K); the small-prime kernel ORs the wheel into each row, so the rows
// come out the same with a third of the atomics and rank loads.
__device__ __forceinline__ void mark_hit(const LargeArgs &a, const uint32_t *s_wheel, uint64_t j, uint32_t idx) {
    if ((s_wheel[idx >> 5] >> (idx & 31)) & 1u) return;
    mark_hit(a, j, idx);
}

// One thread per prime p.  For the odd m = m0 + 2j of the window,
// p | m*K + 2Y  <=>  j = -Y*K^-1 - m0/2 (mod p), so the residue j(Y) drops
// by K^-1 each time Y grows by one; every j(Y) inside the window is a hit.
template <typename T>
__global__ void __launch_bounds__(256) k_sieve_large_step(const __grid_constant__ LargeArgs a) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.np) return;
    const uint64_t p = ((const T *)a.p)[i];
    const uint64_t ci = ((const T *)a.cinv)[i];
    const uint64_t inv2 = (p + 1) >> 1;
    const uint64_t t1 = mulmod40(a.sly % p, ci, p);
    const uint64_t t2 = mulmod40(a.m0 % p, inv2, p);
    uint64_t j = t1 >= t2 ? t1 - t2 : t1 + p - t2;  // j at Y = -sly (idx 0)
    const uint32_t nb = 2 * a.sly + 1;
    if (p < (1ull << 32)) {
        uint32_t j32 = (uint32_t)j;
        const uint32_t p32 = (uint32_t)p, c32 = (uint32_t)ci;
        const uint32_t nodd32 = a.nodd < 0xffffffffull ? (uint32_t)a.nodd : 0xffffffffu;
        for (uint32_t idx = 0; idx < nb; idx++) {
            if (j32 < nodd32)
                for (uint64_t jj = j32; jj < a.nodd; jj += p32) mark_hit(a, jj, idx);
            j32 = (j32 >= c32) ? j32 - c32 : j32 + (p32 - c32);
        }
    } else {
        for (uint32_t idx = 0; idx < nb; idx++) {
            if (j < a.nodd)
                for (uint64_t jj = j; jj < a.nodd; jj += p) mark_hit(a, jj, idx);
            j = (j >= ci) ? j - ci : j + (p - ci);
        }
    }
}

// ------------------------------------------------------ modular search

// x mod A for one divisor A >= 1 and several x.  32-bit operands use the
// integer remainder.  64-bit operands (x < 2^40) use a double-precision
// reciprocal: x is exact as a double, 1/A and the product x * (1/A) are each
// rounded once (relative error 2^-53 each), so the quotient estimate
// trunc(x * (1/A)) is within one of floor(x / A) (x / A < 2^40, absolute
// error below 2^-12), and the remainder x - q*A, exact in signed 64-bit
// arithmetic, needs at most one correction either way.
template <typename U>
struct DivBy {
    U A;
    __device__ __forceinline__ explicit DivBy(U a) : A(a) {}
    __device__ __forceinline__ U rem(U x) const { return x % A; }
};
template <>
struct DivBy<uint64_t> {
    uint64_t A;
    double inv;
    __device__ __forceinline__ explicit DivBy(uint64_t a) : A(a), inv(1.0 / (double)a) {}
    __device__ __forceinline__ uint64_t rem(uint64_t x) const {
        const uint64_t q = (uint64_t)((double)x * inv);
        int64_t r = (int64_t)(x - q * A);
        if (r < 0) r += (int64_t)A;
        if (r >= (int64_t)A) r -= (int64_t)A;
        return (uint64_t)r;
    }
};

// x mod A for 32-bit x and a divisor A >= 2^13, with one single-precision
// reciprocal shared by every x.  Each step rounds toward zero (A up, x and
// the products down) and the reciprocal is scaled by 1 - 2^-20, so the
// quotient estimate never exceeds floor(x / A); the relative shortfall is
// below 2^-19.3 (rcp.approx is within one ulp, each rounding within one
// ulp), so with x / A < 2^19 it falls short by at most one.  The remainder
// x - q*A then lies in [0, 2A) and is at most x, so it is exact in 32 bits
// and one conditional subtraction finishes it.
struct DivByF32 {
    uint32_t A;
    float inv;
    __device__ __forceinline__ explicit DivByF32(uint32_t a) : A(a) {
        float af, r;
        asm("cvt.rp.f32.u32 %0, %1;" : "=f"(af) : "r"(a));
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(af));
        asm("mul.rm.ftz.f32 %0, %1, %2;" : "=f"(inv) : "f"(r), "f"(1.0f - 0x1p-20f));
    }
    __device__ __forceinline__ uint32_t rem(uint32_t x) const {
        float xf, e;
        uint32_t q;
        asm("cvt.rm.f32.u32 %0, %1;" : "=f"(xf) : "r"(x));
        asm("mul.rm.ftz.f32 %0, %1, %2;" : "=f"(e) : "f"(xf), "f"(inv));
        asm("cvt.rzi.u32.f32 %0, %1;" : "=r"(q) : "f"(e));
        const uint32_t r = x - q * A;
        return r >= A ? r - A : r;
    }
};

// Windows at least this wide (W = 2*sly) let the 32-bit levels of the
// modular search use DivByF32: every level that does not end has A > W + 1
// (and A > W for the walk search over W - 1).
constexpr uint32_t F32_MIN_W = 1u << 13;

// For 0 < A < M, B < M, W < M - 1 and gcd(A, M) = 1, the value
// u = (A*x + B) mod M at the smallest x >= 0 with (A*x + B) mod M <= W.
// If B <= W, x = 0 and u = B.  If W + 1 >= A the first wrap already lands in
// [0, W]: u = A*ceil((M-B)/A) - (M-B).  Otherwise the wrap count y whose
// interval [M*y - B, M*y - B + W] first holds a multiple of A solves, after
// the reflection z -> W - z, the same problem for (M mod A, ., A, W): a
// Euclid step, so the depth is O(log M).  The landing value of each level
// is W minus the landing value of the level below, so no state is kept on
// the way down and nothing is rebuilt on the way back; the caller recovers
// x = (u - B) * A^-1 mod M with one modular product.
//
// One level: true with u set when the search ends here, else the next
// level's (A, B, M) in place (the caller flips the reflection parity).
// F (32-bit values, W >= F32_MIN_W only): the remainders of a level that
// does not end use DivByF32.
template <typename U, bool F>
__device__ __forceinline__ bool modsearch_level(U &A, U &B, U &M, U W, U &u) {
    if (B <= W) {
        u = B;
        return true;
    }
    if (W + 1 >= A) {
        const U t = DivBy<U>(A).rem(M - B);
        u = t ? A - t : 0;
        return true;
    }
    U r, b1;
    if constexpr (F) {
        static_assert(sizeof(U) == 4, "DivByF32 takes 32-bit values");
        const DivByF32 by(A);
        r = by.rem(M);
        b1 = by.rem(B);
    } else {
        const DivBy<U> by(A);
        r = by.rem(M);
        b1 = by.rem(B);
    }
    b1 = b1 >= r ? b1 - r : b1 + (A - r);  // (B - M) mod A
    B = W >= b1 ? W - b1 : W + (A - b1);   // reflected
    M = A;
    A = r;
    return false;
}

// M * J <= M0 without overflow (M < 2^40, J < 2^32).
__device__ __forceinline__ bool prod_le(uint32_t M, uint64_t J, uint32_t M0) { return (uint64_t)M * J <= M0; }
__device__ __forceinline__ bool prod_le(uint64_t M, uint64_t J, uint64_t M0) {
    return __umul64hi(M, J) == 0 && M * J <= M0;
}

// The search restricted to x < J (E set): false when the first hit lies at
// x >= J.  Bound: a level whose value B is above W has no hit at x = 0, so
// its own x_k >= 1; the level above it lands its hit at
// x = ceil(((x_k + 1) * M - B) / A) > x_k * M / A, and M of the level below
// is that A, so over the levels x_0 >= x_k * M_0 / M_k.  So at the first
// level with M_k * J <= M_0 the search ends: with B_k > W its hit lies at
// x_0 >= J, otherwise B_k <= W is the hit; the levels between M_0 / J and
// about W are skipped.  The test costs a product and a compare per level,
// so callers set E only where it saves many levels (primes expecting well
// under one hit).  Values of 64 bits run their levels in 32-bit arithmetic
// once they fit.
template <typename U, bool F, bool E>
__device__ __forceinline__ bool modsearch_within(U A, U B, U M, U W, uint64_t J, U &u_out) {
    const U M0 = M;
    uint32_t flips = 0;
    U u;
    if constexpr (sizeof(U) == 8) {
        while (M >> 32) {
            if (E && B > W && prod_le(M, J, M0)) return false;
            if (modsearch_level<uint64_t, false>(A, B, M, W, u)) {
                u_out = flips ? W - u : u;
                return true;
            }
            flips ^= 1u;
        }
        uint32_t A32 = (uint32_t)A, B32 = (uint32_t)B, M32 = (uint32_t)M, u32;
        const uint32_t W32 = (uint32_t)W;
        while (true) {  // M32 * J < 2^64: J < 2^32
            if (E && B32 > W32 && (uint64_t)M32 * J <= M0) return false;
            if (modsearch_level<uint32_t, F>(A32, B32, M32, W32, u32)) break;
            flips ^= 1u;
        }
        u_out = flips ? W - u32 : u32;
        return true;
    } else {
        while (true) {
            if (E && B > W && prod_le(M, J, M0)) return false;
            if (modsearch_level<U, F>(A, B, M, W, u)) break;
            flips ^= 1u;
        }
        u_out = flips ? W - u : u;
        return true;
    }
}

// The search without a bound on x.
template <typename U, bool F = false>
__device__ __forceinline__ U modsearch_value(U A, U B, U M, U W) {
    U u;
    modsearch_within<U, F, false>(A, B, M, W, 0, u);
    return u;
}

// Arithmetic mod a prime p < 2^32 with a double-precision reciprocal: the
// quotient estimate floor(v * (1/p)) is within one of floor(v / p) for
// every v < 2^64 and p >= 2^14 (relative error of three roundings, 3 * 2^-53,
// times v/p <= 2^50), and the remainder is corrected in signed arithmetic.
// Smaller p (a small-prime bound set below 2^14) take the integer remainder.
struct Mod32 {
    uint32_t p;
    double inv;
    __device__ __forceinline__ explicit Mod32(uint32_t q) : p(q), inv(1.0 / (double)q) {}
    __device__ __forceinline__ uint32_t red(uint64_t v) const {
        if (p < (1u << 14)) return (uint32_t)(v % p);
        const uint64_t q = (uint64_t)((double)v * inv);
        int64_t r = (int64_t)(v - q * p);
        if (r < 0) r += p;
        if (r < 0) r += p;
        if (r >= (int64_t)p) r -= p;
        if (r >= (int64_t)p) r -= p;
        return (uint32_t)r;
    }
    __device__ __forceinline__ uint32_t mul(uint32_t a, uint32_t b) const { return red((uint64_t)a * b); }
    __device__ __forceinline__ uint32_t sub(uint32_t a, uint32_t b) const { return a >= b ? a - b : a + (p - b); }
};

// The same for primes in [2^32, 2^40).  For v < 2^64 the estimate
// trunc(v * (1/p)) is within one of floor(v / p) (quotient below 2^32,
// relative error 3 * 2^-53); for a, b < p the estimate of floor(a*b / p)
// from the double product a*b (rounded) times 1/p is within one too
// (quotient below 2^40, absolute error below 2^-11).  The remainder is the
// low 64 bits of v - q*p (or a*b - q*p), exact as a signed value in
// (-p, 2p), corrected once either way.
struct Mod40 {
    uint64_t p;
    double inv;
    __device__ __forceinline__ explicit Mod40(uint64_t q) : p(q), inv(1.0 / (double)q) {}
    __device__ __forceinline__ uint64_t fix(uint64_t x, uint64_t q) const {
        int64_t r = (int64_t)(x - q * p);
        if (r < 0) r += (int64_t)p;
        if (r >= (int64_t)p) r -= (int64_t)p;
        return (uint64_t)r;
    }
    __device__ __forceinline__ uint64_t red(uint64_t v) const { return fix(v, (uint64_t)((double)v * inv)); }
    __device__ __forceinline__ uint64_t mul(uint64_t a, uint64_t b) const {
        return fix(a * b, (uint64_t)((double)a * (double)b * inv));
    }
    __device__ __forceinline__ uint64_t sub(uint64_t a, uint64_t b) const { return a >= b ? a - b : a + (p - b); }
};

// Marks every hit of a prime's walk from the hit (j, v) (inclusive) up to
// j_end: the hit after v is v + alpha (step sa) if that is <= W, else
// v - beta (step sb) if v >= beta, else v + alpha - beta (step sa + sb).
// WALK_BATCH hits at a time: their steps (selects, no branches) come first,
// then the batch's rank loads are issued together so their latencies
// overlap, then its marks; hits at or past j_end are masked.  The walk is
// bound by the integer ALU pipe, so walk_from counts j in 32 bits whenever
// j_end + sa + sb < 2^32 (no step from j < j_end can then wrap).
constexpr int WALK_BATCH = 4;

template <typename U, typename J>
__device__ __forceinline__ void walk_marks(const LargeArgs &a, const uint32_t *s_wheel, J j, U v, J j_end, U alpha,
                                           U beta, U W, J sa, J sb) {
    while (j < j_end) {
        J jj[WALK_BATCH];
        uint32_t vv[WALK_BATCH];
#pragma unroll
        for (int k = 0; k < WALK_BATCH; k++) {
            jj[k] = j;
            vv[k] = (uint32_t)v;
            const bool up = v + alpha <= W, down = v >= beta;
            j += up ? sa : (down ? sb : sa + sb);
            v = up ? v + alpha : (down ? v - beta : v + alpha - beta);
        }
        int32_t r[WALK_BATCH];
#pragma unroll
        for (int k = 0; k < WALK_BATCH; k++) {
            const bool skip = jj[k] >= j_end || ((s_wheel[vv[k] >> 5] >> (vv[k] & 31)) & 1u);
            r[k] = skip ? -1 : a.rank[jj[k]];
        }
#pragma unroll
        for (int k = 0; k < WALK_BATCH; k++)
            if (r[k] >= 0) atomicOr(&a.bitmaps[(size_t)r[k] * a.words + (vv[k] >> 5)], 1u << (vv[k] & 31));
    }
}

template <typename U>
__device__ __forceinline__ void walk_from(const LargeArgs &a, const uint32_t *s_wheel, uint64_t j, U v,
                                          uint64_t j_end, U alpha, U beta, U W, uint64_t sa, uint64_t sb) {
    if (j >= j_end) return;
    if (j_end + sa + sb < (1ull << 32))
        walk_marks<U, uint32_t>(a, s_wheel, (uint32_t)j, v, (uint32_t)j_end, alpha, beta, W, (uint32_t)sa,
                                (uint32_t)sb);
    else
        walk_marks<U, uint64_t>(a, s_wheel, j, v, j_end, alpha, beta, W, sa, sb);
}

// Sieve of one prime p > 2*sly + 1 over the window.  With X = 2Y and the
// odd m = m0 + 2j, p | m*K + X  <=>  u = Y + sly = (A*j + B) mod p with
// A = -K mod p and B = sly - m0*K/2 mod p; every j of the window with
// u <= W = 2*sly is a hit (one per j, since p > W).  The first hit is found
// by modsearch_value in O(log p).  When more hits are expected, the
// three-distance structure of the sequence gives every later hit in O(1):
// with a = the first step whose shift A*a mod p = alpha lands in [0, W] and
// b = the first step whose shift lands in [p-W, p) (i.e. -beta), the hit
// after u is u + alpha (step a) if that is <= W, else u - beta (step b) if
// u >= beta, else u + alpha - beta (step a + b).  Otherwise each next hit is
// one more search.
//
// With the job's walk steps (wk != NULL: sa, sb precomputed, alpha and beta
// two modular products away) every hit after the first is one walk step,
// whatever the number of hits.  F: 32-bit search levels with DivByF32
// (W >= F32_MIN_W); E: searches stop once their hit provably lies past the
// window.
template <typename U, typename Mod, bool F, bool E>
__device__ __forceinline__ void sieve_prime(const LargeArgs &a, const uint32_t *s_wheel, const Mod &md, U c, U ci,
                                            const WalkC *wk) {
    const U p = md.p;
    const U W = (U)(2u * a.sly);
    const U c2 = (c & 1) ? (U)((c + (uint64_t)p) >> 1) : c >> 1;  // K/2 mod p
    const U t = md.mul(md.red(a.m0), c2);
    U B = md.sub((U)a.sly, t);
    const U A = p - c;     // c in [1, p)
    const U Ainv = p - ci; // (-K)^-1
    uint64_t j = 0;
    while (true) {
        U u;
        if (!modsearch_within<U, F, E>(A, B, p, W, a.nodd - j, u)) return;
        j += md.mul(md.sub(u, B), Ainv);
        if (j >= a.nodd) return;
        if (wk || (a.nodd - j - 1) * (uint64_t)(W + 1) >= 2ull * p) {  // steps known, or 2+ hits expected: walk
            U alpha, beta;
            uint64_t sa, sb;
            if (wk) {
                sa = wk->sa;
                sb = wk->sb;
                alpha = md.mul(A, (U)sa);
                beta = p - md.mul(A, (U)sb);
            } else {
                alpha = modsearch_value<U, F>(A, A, p, W);
                sa = 1 + (uint64_t)md.mul(md.sub(alpha, A), Ainv);
                const U aw = A + W >= p ? A + W - p : A + W;
                const U ub = modsearch_value<U, F>(A, aw, p, W - 1);
                beta = W - ub;
                sb = 1 + (uint64_t)md.mul(md.sub(ub, aw), Ainv);
            }
            walk_from<U>(a, s_wheel, j, u, a.nodd, alpha, beta, W, sa, sb);
            return;
        }
        mark_hit(a, s_wheel, j, (uint32_t)u);
        B = u + A >= p ? u + A - p : u + A;  // residue of j + 1
        j++;
    }
}

// One thread per prime of [first, first + count); the block keeps the wheel
// row in shared memory.  A warp whose 32 primes all expect under 1/64 hit in
// the window (p > 64 * nodd * (W + 1)) bounds its searches by the window
// (modsearch_within): they end near the level where the Euclid values fall
// to p / nodd > 64 (W + 1), about four or more levels (a factor ~3.3 each)
// before the values reach W.  Where primes expect more hits
// the per-level test costs more than the few levels it saves (measured with
// the bound on every warp expecting under one hit per prime).
template <typename T, bool F>
__global__ void __launch_bounds__(256) k_sieve_large_search(const __grid_constant__ LargeArgs a, uint64_t first,
                                                            uint64_t count) {
    extern __shared__ uint32_t s_wheel[];
    for (uint32_t w = threadIdx.x; w < a.words; w += blockDim.x) s_wheel[w] = a.wheel[w];
    __syncthreads();
    const uint64_t i = first + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < first + count;
    const uint64_t p = valid ? (uint64_t)((const T *)a.p)[i] : 0;
    const bool sparse = __all_sync(0xffffffffu, !valid || a.nodd * (2ull * a.sly + 1) * 64 < p);
    if (!valid) return;
    const uint64_t c = ((const T *)a.c)[i];
    const uint64_t ci = ((const T *)a.cinv)[i];
    const bool walk = a.walk && i >= a.walk_first && i < a.walk_end;  // walk steps are kept below 2^32 only
    WalkC wk;
    if (walk) wk = a.walk[i - a.walk_first];
    if (p < (1ull << 32)) {
        const Mod32 md((uint32_t)p);
        if (sparse)
            sieve_prime<uint32_t, Mod32, F, true>(a, s_wheel, md, (uint32_t)c, (uint32_t)ci, walk ? &wk : nullptr);
        else
            sieve_prime<uint32_t, Mod32, F, false>(a, s_wheel, md, (uint32_t)c, (uint32_t)ci, walk ? &wk : nullptr);
    } else {
        const Mod40 md(p);
        if (sparse)
            sieve_prime<uint64_t, Mod40, F, true>(a, s_wheel, md, c, ci, nullptr);
        else
            sieve_prime<uint64_t, Mod40, F, false>(a, s_wheel, md, c, ci, nullptr);
    }
}

// Walk constants (alpha, sa, beta, sb of sieve_prime) of the primes
// [first, first + count), all below 2^32, for the window width W.
template <typename T>
__global__ void __launch_bounds__(256) k_walk_consts(const T *pt, const T *ct, const T *cit, uint64_t first,
                                                     uint64_t count, uint32_t W, WalkC *out) {
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const uint32_t p = (uint32_t)pt[first + k], c = (uint32_t)ct[first + k];
    const Mod32 md(p);
    const uint32_t A = p - c, Ainv = p - (uint32_t)cit[first + k];  // -K and (-K)^-1
    const uint32_t alpha = modsearch_value<uint32_t>(A, A, p, W);
    const uint32_t aw = A + W >= p ? A + W - p : A + W;
    const uint32_t ub = modsearch_value<uint32_t>(A, aw, p, W - 1);
    WalkC w;
    w.sa = 1 + md.mul(md.sub(alpha, A), Ainv);
    w.sb = 1 + md.mul(md.sub(ub, aw), Ainv);
    out[k] = w;
}

cudaError_t launch_walk_consts(const void *p, const void *c, const void *ci, bool wide, uint64_t first,
                               uint64_t count, uint32_t W, WalkC *out, cudaStream_t st) {
    if (count == 0) return cudaSuccess;
    const uint64_t blocks = (count + 255) / 256;
    if (wide)
        k_walk_consts<uint64_t><<<(unsigned)blocks, 256, 0, st>>>((const uint64_t *)p, (const uint64_t *)c,
                                                                   (const uint64_t *)ci, first, count, W, out);
    else
        k_walk_consts<uint32_t><<<(unsigned)blocks, 256, 0, st>>>((const uint32_t *)p, (const uint32_t *)c,
                                                                   (const uint32_t *)ci, first, count, W, out);
    return cudaGetLastError();
}

// Segmented sieve of the many-hit primes (below 2^32): thread (prime i,
// segment blockIdx.y) covers the odd m j in [j0, j1) of its segment.  The
// first hit at j >= j0 comes from one modular search from the residue at j0,
// (A*j0 + B) mod p; every later hit of the segment from the prime's walk
// constants.  A prime expecting thousands of hits per window is thus spread
// over many threads of similar work instead of one long serial walk.
//
// Every band of a window (its own segment count) runs in this one launch:
// block b belongs to the first band whose cumulative block count exceeds b,
// and inside the band to segment (b' / prime blocks), prime block
// (b' mod prime blocks).  Bands of a few thousand blocks, each too short to
// fill the SMs through its tail, so overlap.
struct SegGrid {
    SegBand band[MAX_SEG_BANDS];
    uint32_t block_end[MAX_SEG_BANDS];  // blocks of bands 0 .. b
    uint32_t pblocks[MAX_SEG_BANDS];    // blocks of 256 primes in band b
    int nbands;
};

template <typename T>
__global__ void __launch_bounds__(256) k_sieve_large_seg(const __grid_constant__ LargeArgs a,
                                                         const __grid_constant__ SegGrid g) {
    extern __shared__ uint32_t s_wheel[];
    for (uint32_t w = threadIdx.x; w < a.words; w += blockDim.x) s_wheel[w] = a.wheel[w];
    __syncthreads();
    int b = 0;
    while (b + 1 < g.nbands && blockIdx.x >= g.block_end[b]) b++;
    const uint32_t local = blockIdx.x - (b ? g.block_end[b - 1] : 0u);
    const uint32_t seg = local / g.pblocks[b];
    const SegBand &bd = g.band[b];
    const uint64_t i = bd.first + (uint64_t)(local - seg * g.pblocks[b]) * blockDim.x + threadIdx.x;
    const uint64_t j0 = (uint64_t)seg * bd.seg_len;
    if (i >= bd.first + bd.count || j0 >= a.nodd) return;
    const uint64_t j1 = min(a.nodd, j0 + bd.seg_len);
    const uint32_t p = (uint32_t)((const T *)a.p)[i];
    const uint32_t c = (uint32_t)((const T *)a.c)[i];
    const uint32_t ci = (uint32_t)((const T *)a.cinv)[i];
    const WalkC wk = a.walk[i - a.walk_first];
    const Mod32 md(p);
    const uint32_t W = 2u * a.sly;
    const uint32_t c2 = (c & 1) ? (uint32_t)((c + (uint64_t)p) >> 1) : c >> 1;  // K/2 mod p
    const uint32_t A = p - c, Ainv = p - ci;
    const uint32_t alpha = md.mul(A, wk.sa), beta = p - md.mul(A, wk.sb);
    const uint32_t B0 = md.sub(a.sly % p, md.mul(md.red(a.m0), c2));
    const uint32_t B = md.red((uint64_t)md.mul(A, md.red(j0)) + B0);  // residue at j0
    const uint32_t u = W >= F32_MIN_W ? modsearch_value<uint32_t, true>(A, B, p, W)
                                      : modsearch_value<uint32_t, false>(A, B, p, W);
    walk_from<uint32_t>(a, s_wheel, j0 + md.mul(md.sub(u, B), Ainv), u, j1, alpha, beta, W, wk.sa, wk.sb);
}

cudaError_t launch_sieve_large(const LargeArgs &a, bool wide, uint64_t split, const SegBand *bands, int nbands,
                               uint64_t search_first, cudaStream_t st) {
    if (a.np == 0) return cudaSuccess;
    const uint32_t threads = 256;
    const size_t smem = (size_t)a.words * sizeof(uint32_t);
    if (split > a.np) split = a.np;
    SegGrid g{};
    uint64_t blocks = 0;
    for (int b = 0; b < nbands && b < MAX_SEG_BANDS; b++) {
        const SegBand &bd = bands[b];
        if (bd.count == 0 || bd.nseg == 0) continue;
        const uint64_t pb = (bd.count + threads - 1) / threads;
        blocks += pb * bd.nseg;
        if (blocks >= (1ull << 31)) return cudaErrorInvalidConfiguration;
        g.band[g.nbands] = bd;
        g.pblocks[g.nbands] = (uint32_t)pb;
        g.block_end[g.nbands] = (uint32_t)blocks;
        g.nbands++;
    }
    if (blocks) {
        if (wide)
            k_sieve_large_seg<uint64_t><<<(unsigned)blocks, threads, smem, st>>>(a, g);
        else
            k_sieve_large_seg<uint32_t><<<(unsigned)blocks, threads, smem, st>>>(a, g);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (search_first < split) search_first = split;
    if (split > 0) {  // primes with many hits per window: step every Y
        LargeArgs s = a;
        s.np = split;
        const uint64_t blocks = (split + threads - 1) / threads;
        if (wide)
            k_sieve_large_step<uint64_t><<<(unsigned)blocks, threads, 0, st>>>(s);
        else
            k_sieve_large_step<uint32_t><<<(unsigned)blocks, threads, 0, st>>>(s);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (search_first < a.np) {  // the rest: modular search for each hit
        const uint64_t count = a.np - search_first;
        const uint64_t blocks = (count + threads - 1) / threads;
        const bool f32 = 2ull * a.sly >= F32_MIN_W;  // every 32-bit level that does not end has A >= 2^13
        if (wide && f32)
            k_sieve_large_search<uint64_t, true><<<(unsigned)blocks, threads, smem, st>>>(a, search_first, count);
        else if (wide)
            k_sieve_large_search<uint64_t, false><<<(unsigned)blocks, threads, smem, st>>>(a, search_first, count);
        else if (f32)
            k_sieve_large_search<uint32_t, true><<<(unsigned)blocks, threads, smem, st>>>(a, search_first, count);
        else
            k_sieve_large_search<uint32_t, false><<<(unsigned)blocks, threads, smem, st>>>(a, search_first, count);
    }
    return cudaGetLastError();
}

// ================================================ small-prime sieve + lists

constexpr int SMALL_THREADS = 256;

// First marked position of small prime i in the row of m: p | m*K + 2Y
// <=> Y = (m mod q) * r_q (mod q), position idx = Y + sly.
__device__ __forceinline__ uint32_t small_first(const SieveArgs &a, uint32_t i, uint64_t m) {
    const uint32_t q = a.sq[i];
    const uint64_t bar = a.sbar[i];
    const uint32_t mq = barrett64(m, q, bar);
    const uint32_t y0 = barrett64((uint64_t)mq * a.sr[i], q, bar);
    uint32_t idx = y0 + barrett64(a.sly, q, bar);
    return idx >= q ? idx - q : idx;
}

// One block per m.  The row starts as the K-prime wheel OR the large-prime
// hits, the small primes are struck out in shared memory, then the survivors
// of each side are compacted, nearest first, into that side's list.  Primes
// below 32 (odd d-primes such as 3 and 5 hit a third and a fifth of the row)
// are laid on whole words by the thread that owns the word, as it loads the
// row; primes below 256 are marked by all threads of the block, each taking
// every blockDim-th hit; the rest one prime per thread.  A row's work is thus
// spread over the block instead of waiting on the thread of q = 3.
__global__ void __launch_bounds__(SMALL_THREADS) k_sieve_small(const __grid_constant__ SieveArgs a, int compact) {
    extern __shared__ uint32_t bm[];
    __shared__ uint32_t s_first[64];  // first positions of the primes below 32 (at most 10 of them)
    const uint32_t r = blockIdx.x;
    const uint64_t m = a.ms[r];
    const uint32_t W = a.words, sly = a.sly, nb = 2 * sly + 1;
    uint32_t *grow = a.bitmaps + (size_t)r * W;
    if (threadIdx.x < a.n32) s_first[threadIdx.x] = small_first(a, threadIdx.x, m);
    __syncthreads();
    for (uint32_t w = threadIdx.x; w < W; w += blockDim.x) {
        uint32_t pm = 0;
        for (uint32_t i = 0; i < a.n32; i++) {  // bits 32w + b with b = first - 32w (mod q), stride q
            const uint32_t q = a.sq[i];
            const uint32_t base = (32u * w) % q;
            uint32_t b = s_first[i] >= base ? s_first[i] - base : s_first[i] + q - base;
            for (; b < 32; b += q) pm |= 1u << b;
        }
        if (32u * w + 32u > nb) pm &= (1u << (nb - 32u * w)) - 1u;  // no marks past position 2 sly
        bm[w] = a.wheel[w] | grow[w] | pm;
    }
    __syncthreads();
    for (uint32_t i = a.n32; i < a.n256; i++) {  // all threads stride over the hits of each prime below 256
        const uint32_t q = a.sq[i];
        for (uint32_t idx = small_first(a, i, m) + threadIdx.x * q; idx < nb; idx += blockDim.x * q)
            atomicOr(&bm[idx >> 5], 1u << (idx & 31));
    }
    for (uint32_t i = a.n256 + threadIdx.x; i < a.nsmall; i += blockDim.x) {
        const uint32_t q = a.sq[i];
        const uint64_t bar = a.sbar[i];
        const uint32_t mq = barrett64(m, q, bar);
        const uint32_t y0 = barrett64((uint64_t)mq * a.sr[i], q, bar);
        uint32_t idx = y0 + barrett64(sly, q, bar);
        if (idx >= q) idx -= q;
        for (; idx < nb; idx += q) atomicOr(&bm[idx >> 5], 1u << (idx & 31));
    }
    __syncthreads();
    if (!compact) {
        for (uint32_t w = threadIdx.x; w < W; w += blockDim.x) grow[w] = bm[w];
        return;
    }
    typedef cub::BlockScan<uint32_t, SMALL_THREADS> Scan;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ uint32_t s_count[2];
    // next side: idx sly+1 .. 2 sly ascending, Y = idx - sly
    {
        uint16_t *out = a.lists + (size_t)(2 * r) * a.cap;
        const uint32_t lo = sly + 1, hi = 2 * sly;
        const uint32_t w_lo = lo >> 5, w_hi = hi >> 5;
        uint32_t base = 0;
        for (uint32_t c0 = w_lo; c0 <= w_hi; c0 += blockDim.x) {
            const uint32_t w = c0 + threadIdx.x;
            uint32_t bits = 0;
            if (w <= w_hi) {
                bits = ~bm[w];
                if (w == w_lo) bits &= 0xffffffffu << (lo & 31);
                if (w == w_hi) bits &= (hi & 31) == 31 ? 0xffffffffu : ((2u << (hi & 31)) - 1);
            }
            uint32_t off, total;
            Scan(tmp).ExclusiveSum((uint32_t)__popc(bits), off, total);
            uint32_t pos = base + off;
            while (bits) {
                const uint32_t b = __ffs(bits) - 1;
                bits &= bits - 1;
                out[pos++] = (uint16_t)(w * 32 + b - sly);
            }
            base += total;
            __syncthreads();
        }
        if (threadIdx.x == 0) s_count[0] = base;
    }
    // prev side: idx sly-1 .. 0 descending, |Y| = sly - idx
    {
        uint16_t *out = a.lists + (size_t)(2 * r + 1) * a.cap;
        const uint32_t hi = sly - 1;
        const uint32_t w_hi = hi >> 5;
        uint32_t base = 0;
        for (uint32_t c0 = 0; c0 <= w_hi; c0 += blockDim.x) {
            const uint32_t k = c0 + threadIdx.x;
            uint32_t bits = 0, w = 0;
            if (k <= w_hi) {
                w = w_hi - k;
                bits = ~bm[w];
                if (w == w_hi) bits &= (hi & 31) == 31 ? 0xffffffffu : ((2u << (hi & 31)) - 1);
            }
            uint32_t off, total;
            Scan(tmp).ExclusiveSum((uint32_t)__popc(bits), off, total);
            uint32_t pos = base + off;
            while (bits) {
                const uint32_t b = 31 - __clz(bits);
                bits &= ~(1u << b);
                out[pos++] = (uint16_t)(sly - (w * 32 + b));
            }
            base += total;
            __syncthreads();
        }
        if (threadIdx.x == 0) s_count[1] = base;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        a.counts[2 * r] = s_count[0];
        a.counts[2 * r + 1] = s_count[1];
        atomicMax(a.max_count, max(s_count[0], s_count[1]));
        atomicAdd(a.survivors, (unsigned long long)(s_count[0] + s_count[1]));
    }
}

cudaError_t launch_sieve_small(const SieveArgs &a, bool compact, cudaStream_t st) {
    if (a.nm == 0) return cudaSuccess;
    const size_t smem = (size_t)a.words * sizeof(uint32_t);
    k_sieve_small<<<a.nm, SMALL_THREADS, smem, st>>>(a, compact ? 1 : 0);
    return cudaGetLastError();
}

// ================================================ IMAD throughput probe

// Eight independent multiply-add chains per thread (each instruction depends
// only on its own chain), enough warps per SM to hide the latency: measures
// how many 32-bit integer multiply-adds the SMs retire per second.
__global__ void __launch_bounds__(256) k_imad_peak(uint32_t iters, uint32_t seed, uint32_t *sink) {
    uint32_t a0 = seed + threadIdx.x, a1 = a0 ^ 0x9e3779b9u, a2 = a0 * 3u, a3 = a0 + 7u;
    uint32_t a4 = a0 ^ 0x85ebca6bu, a5 = a0 * 5u, a6 = a0 + 11u, a7 = a0 ^ 0xc2b2ae35u;
    const uint32_t m = seed | 1u, c = seed >> 3;
    for (uint32_t i = 0; i < iters; i++) {
#pragma unroll
        for (int r = 0; r < 16; r++) {
            asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a0) : "r"(m), "r"(c));
            asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a1) : "r"(m), "r"(c));
            asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a2) : "r"(m), "r"(c));
            asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a3) : "r"(m), "r"(c));
            asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a4) : "r"(m), "r"(c));
            asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a5) : "r"(m), "r"(c));
            asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a6) : "r"(m), "r"(c));
            asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a7) : "r"(m), "r"(c));
        }
    }
    const uint32_t v = a0 ^ a1 ^ a2 ^ a3 ^ a4 ^ a5 ^ a6 ^ a7;
    if (v == 0x12345678u) sink[0] = v;  // keeps the chains alive
}

cudaError_t launch_imad_peak(int grid, uint32_t iters, uint32_t *sink, cudaStream_t st) {
    k_imad_peak<<<grid, 256, 0, st>>>(iters, 0x2545F491u, sink);
    return cudaGetLastError();
}

__global__ void k_iota(uint32_t *out, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = i;
}

__global__ void k_init_search(uint32_t S, uint32_t *found_k, uint32_t *k_start, uint32_t *act, uint32_t *conf,
                              Scalars *sc, uint32_t warps) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < S) {
        found_k[i] = NOT_FOUND;
        k_start[i] = 0;
        act[i] = i;
        conf[i] = NOT_FOUND;
    }
    if (i == 0) {
        sc->next_item = 0;
        sc->tests = 0;
        sc->confirm = 0;
        sc->n_redo = 0;
        sc->n_out = 0;
        sc->unresolved = S;
        sc->active_warps = warps;
        sc->stopped = 0;
    }
}

cudaError_t launch_init_search(uint32_t S, uint32_t *found_k, uint32_t *k_start, uint32_t *act, uint32_t *conf,
                               Scalars *sc, uint32_t warps, cudaStream_t st) {
    k_init_search<<<(S + 255) / 256 + 1, 256, 0, st>>>(S, found_k, k_start, act, conf, sc, warps);
    return cudaGetLastError();
}

cudaError_t launch_iota(uint32_t *out, uint32_t n, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_iota<<<(n + 255) / 256, 256, 0, st>>>(out, n);
    return cudaGetLastError();
}

// keeps the sides that are unresolved and still have candidates
__global__ void k_compact_active(const uint32_t *act_in, uint32_t n_in, const uint32_t *found_k, const uint32_t *k_next,
                                 const uint32_t *counts, uint32_t ext_max, uint32_t *act_out, uint32_t *n_out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_in) return;
    const uint32_t s = act_in[i];
    if (found_k[s] != NOT_FOUND || k_next[s] >= counts[s] + ext_max) return;
    act_out[atomicAdd(n_out, 1u)] = s;
}

cudaError_t launch_compact_active(const uint32_t *act_in, uint32_t n_in, const uint32_t *found_k,
                                  const uint32_t *k_next, const uint32_t *counts, uint32_t ext_max,
                                  uint32_t *act_out, uint32_t *n_out, cudaStream_t st) {
    if (n_in == 0) return cudaSuccess;
    const uint32_t threads = 256, blocks = (n_in + threads - 1) / threads;
    k_compact_active<<<blocks, threads, 0, st>>>(act_in, n_in, found_k, k_next, counts, ext_max, act_out, n_out);
    return cudaGetLastError();
}

}  // namespace pg
