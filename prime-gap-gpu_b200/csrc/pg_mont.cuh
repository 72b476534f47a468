// pg_mont.cuh -- multi-precision Montgomery arithmetic for the strong PRP test.
//
// One thread owns one L-word number: the operand, the modulus and the 2L+1
// word double-width accumulator all live in registers (the loops below are
// fully unrolled over the compile-time L, so every array index is a
// constant).  Products use PTX multiply-add carry chains (mad.lo.cc /
// madc.hi.cc), i.e. integer multiply-add only -- no floating point and no
// tensor cores: this is exact multi-precision integer arithmetic.
//
// The reference computes the same test with CGBN (miller_rabin.h:160-248):
// a fixed-window Montgomery powm followed by a squaring chain.  Here the
// base-2 test never multiplies by a table entry: in Montgomery form a
// multiplication by 2 is a shift and one conditional subtraction, so the
// exponentiation is B squarings plus O(L) work per set bit.
#pragma once

#include <cstdint>

namespace pg {

// ---------------------------------------------------------------- PTX ops
__device__ __forceinline__ uint32_t mad_lo_cc(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t r;
    asm volatile("mad.lo.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
    return r;
}
__device__ __forceinline__ uint32_t madc_lo_cc(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t r;
    asm volatile("madc.lo.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
    return r;
}
__device__ __forceinline__ uint32_t madc_hi_cc(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t r;
    asm volatile("madc.hi.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
    return r;
}
__device__ __forceinline__ uint32_t mad_hi_cc(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t r;
    asm volatile("mad.hi.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
    return r;
}
__device__ __forceinline__ uint32_t madc_hi(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t r;
    asm volatile("madc.hi.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
    return r;
}
__device__ __forceinline__ uint32_t add_cc(uint32_t a, uint32_t b) {
    uint32_t r;
    asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t addc_cc(uint32_t a, uint32_t b) {
    uint32_t r;
    asm volatile("addc.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t addc(uint32_t a, uint32_t b) {
    uint32_t r;
    asm volatile("addc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t sub_cc(uint32_t a, uint32_t b) {
    uint32_t r;
    asm volatile("sub.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t subc_cc(uint32_t a, uint32_t b) {
    uint32_t r;
    asm volatile("subc.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t subc(uint32_t a, uint32_t b) {
    uint32_t r;
    asm volatile("subc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}

// -n^-1 mod 2^32 for odd n0 (Newton iteration, 3 -> 6 -> 12 -> 24 -> 48 bits)
__device__ __forceinline__ uint32_t neg_inv32(uint32_t n0) {
    uint32_t x = n0;
#pragma unroll
    for (int i = 0; i < 4; i++) x *= 2u - n0 * x;
    return 0u - x;
}

// ------------------------------------------------------------ Montgomery
// REDC of the 2L+1 word value t (< n*R): returns t * R^-1 mod n in x (< n).
template <int L>
__device__ __forceinline__ void mont_redc(uint32_t (&t)[2 * L + 1], const uint32_t (&n)[L], uint32_t ninv,
                                          uint32_t (&x)[L]) {
    uint32_t pend = 0;  // carry pending into t[i + L]
#pragma unroll
    for (int i = 0; i < L; i++) {
        const uint32_t q = t[i] * ninv;
        // The chain that ends at word i+L-1 ("short") runs first, then the
        // pending carry and its carry go into t[i+L], then the chain that
        // ends at word i+L ("long").  Even j: lo at i+j, hi at i+j+1.
        if ((L & 1) == 0) {
            // short = even j (last even j = L-2 -> hi at i+L-1)
            t[i] = mad_lo_cc(q, n[0], t[i]);
            t[i + 1] = madc_hi_cc(q, n[0], t[i + 1]);
#pragma unroll
            for (int j = 2; j < L; j += 2) {
                t[i + j] = madc_lo_cc(q, n[j], t[i + j]);
                t[i + j + 1] = madc_hi_cc(q, n[j], t[i + j + 1]);
            }
            t[i + L] = addc_cc(t[i + L], pend);
            uint32_t c1 = addc(0u, 0u);
            // long = odd j (last odd j = L-1 -> hi at i+L)
            t[i + 1] = mad_lo_cc(q, n[1], t[i + 1]);
            t[i + 2] = madc_hi_cc(q, n[1], t[i + 2]);
#pragma unroll
            for (int j = 3; j < L; j += 2) {
                t[i + j] = madc_lo_cc(q, n[j], t[i + j]);
                t[i + j + 1] = madc_hi_cc(q, n[j], t[i + j + 1]);
            }
            pend = addc(c1, 0u);
        } else {
            // short = odd j (last odd j = L-2 -> hi at i+L-1)
            if (L > 1) {
                t[i + 1] = mad_lo_cc(q, n[1 < L ? 1 : 0], t[i + 1]);
                t[i + 2] = madc_hi_cc(q, n[1 < L ? 1 : 0], t[i + 2]);
#pragma unroll
                for (int j = 3; j < L; j += 2) {
                    t[i + j] = madc_lo_cc(q, n[j], t[i + j]);
                    t[i + j + 1] = madc_hi_cc(q, n[j], t[i + j + 1]);
                }
                t[i + L] = addc_cc(t[i + L], pend);
            } else {
                t[i + L] = add_cc(t[i + L], pend);
            }
            uint32_t c1 = addc(0u, 0u);
            // long = even j (last even j = L-1 -> hi at i+L)
            t[i] = mad_lo_cc(q, n[0], t[i]);
            t[i + 1] = madc_hi_cc(q, n[0], t[i + 1]);
#pragma unroll
            for (int j = 2; j < L; j += 2) {
                t[i + j] = madc_lo_cc(q, n[j], t[i + j]);
                t[i + j + 1] = madc_hi_cc(q, n[j], t[i + j + 1]);
            }
            pend = addc(c1, 0u);
        }
    }
    t[2 * L] += pend;
    // u = t[L .. 2L] < 2n; x = u - n if u >= n else u
    uint32_t d[L];
    d[0] = sub_cc(t[L], n[0]);
#pragma unroll
    for (int j = 1; j < L; j++) d[j] = subc_cc(t[L + j], n[j]);
    const uint32_t top = subc(t[2 * L], 0u);  // 0 if u >= n, 0xffffffff on borrow
    const bool keep = top != 0;
#pragma unroll
    for (int j = 0; j < L; j++) x[j] = keep ? t[L + j] : d[j];
}

// x = x^2 * R^-1 mod n (x < n in and out).  Squaring by cross products,
// doubling, and the diagonal squares, then REDC.
template <int L>
__device__ __forceinline__ void mont_sqr(uint32_t (&x)[L], const uint32_t (&n)[L], uint32_t ninv) {
    uint32_t t[2 * L + 1];
#pragma unroll
    for (int i = 0; i < 2 * L + 1; i++) t[i] = 0;
    // cross products: row i adds x_i * x[i+1 .. L-1] at words 2i+1 .. i+L;
    // the running sum stays below 2^(32(i+L+1)) so nothing leaves word i+L.
#pragma unroll
    for (int i = 0; i < L - 1; i++) {
        const int N = L - 1 - i;
        const int off = 2 * i + 1;
        const uint32_t a = x[i];
        // even chain: jj = 0, 2, ... (product a * x[i+1+jj]: lo at off+jj, hi at off+jj+1)
        t[off] = mad_lo_cc(a, x[i + 1], t[off]);
        if (N > 1) {
            t[off + 1] = madc_hi_cc(a, x[i + 1], t[off + 1]);
#pragma unroll
            for (int jj = 2; jj < N; jj += 2) {
                t[off + jj] = madc_lo_cc(a, x[i + 1 + jj], t[off + jj]);
                if (jj + 1 < N || (N & 1) == 0)
                    t[off + jj + 1] = madc_hi_cc(a, x[i + 1 + jj], t[off + jj + 1]);
                else
                    t[off + jj + 1] = madc_hi(a, x[i + 1 + jj], t[off + jj + 1]);  // ends at the top word
            }
            if ((N & 1) == 0) t[off + N] = addc(t[off + N], 0u);  // even chain ended at off+N-1
            // odd chain: jj = 1, 3, ...
            t[off + 1] = mad_lo_cc(a, x[i + 2], t[off + 1]);
#pragma unroll
            for (int jj = 1; jj < N; jj += 2) {
                if (jj > 1) t[off + jj] = madc_lo_cc(a, x[i + 1 + jj], t[off + jj]);
                if (jj + 2 < N || (N & 1) == 1)
                    t[off + jj + 1] = madc_hi_cc(a, x[i + 1 + jj], t[off + jj + 1]);
                else
                    t[off + jj + 1] = madc_hi(a, x[i + 1 + jj], t[off + jj + 1]);  // ends at the top word
            }
            if ((N & 1) == 1) t[off + N] = addc(t[off + N], 0u);  // odd chain ended at off+N-1
        } else {
            t[off + 1] = madc_hi(a, x[i + 1], t[off + 1]);  // single product, hi is the top word
        }
    }
    // double (the cross sum is < 2^(64L-1), so no bit leaves word 2L-1)
#pragma unroll
    for (int k = 2 * L - 1; k >= 1; k--) t[k] = __funnelshift_l(t[k - 1], t[k], 1);
    t[0] = t[0] << 1;
    // diagonal squares x_i^2 at words 2i, 2i+1, one carry chain
    t[0] = mad_lo_cc(x[0], x[0], t[0]);
    t[1] = madc_hi_cc(x[0], x[0], t[1]);
#pragma unroll
    for (int i = 1; i < L; i++) {
        t[2 * i] = madc_lo_cc(x[i], x[i], t[2 * i]);
        if (i + 1 < L)
            t[2 * i + 1] = madc_hi_cc(x[i], x[i], t[2 * i + 1]);
        else
            t[2 * i + 1] = madc_hi(x[i], x[i], t[2 * i + 1]);
    }
    mont_redc<L>(t, n, ninv, x);
}

// x = 2x mod n (x < n)
template <int L>
__device__ __forceinline__ void mod_dbl(uint32_t (&x)[L], const uint32_t (&n)[L]) {
    uint32_t y[L];
    const uint32_t carry = x[L - 1] >> 31;
#pragma unroll
    for (int k = L - 1; k >= 1; k--) y[k] = __funnelshift_l(x[k - 1], x[k], 1);
    y[0] = x[0] << 1;
    uint32_t d[L];
    d[0] = sub_cc(y[0], n[0]);
#pragma unroll
    for (int k = 1; k < L; k++) d[k] = subc_cc(y[k], n[k]);
    const uint32_t borrow = subc(carry, 0u);  // nonzero iff 2x < n
#pragma unroll
    for (int k = 0; k < L; k++) x[k] = borrow ? y[k] : d[k];
}

// x = a*x mod n for a small a (x < n); a - 1 conditional subtractions at most
template <int L>
__device__ __forceinline__ void mod_mul_small(uint32_t (&x)[L], const uint32_t (&n)[L], uint32_t a) {
    uint32_t y[L + 1];
    y[0] = x[0] * a;
    uint32_t hi = __umulhi(x[0], a);
#pragma unroll
    for (int k = 1; k < L; k++) {
        uint64_t p = (uint64_t)x[k] * a + hi;
        y[k] = (uint32_t)p;
        hi = (uint32_t)(p >> 32);
    }
    y[L] = hi;
    for (uint32_t it = 0; it < a; it++) {
        uint32_t d[L + 1];
        d[0] = sub_cc(y[0], n[0]);
#pragma unroll
        for (int k = 1; k < L; k++) d[k] = subc_cc(y[k], n[k]);
        d[L] = subc_cc(y[L], 0u);
        const uint32_t borrow = subc(0u, 0u);
        if (borrow) break;
#pragma unroll
        for (int k = 0; k <= L; k++) y[k] = d[k];
    }
#pragma unroll
    for (int k = 0; k < L; k++) x[k] = y[k];
}

template <int L>
__device__ __forceinline__ bool eq_words(const uint32_t (&a)[L], const uint32_t (&b)[L]) {
    uint32_t acc = 0;
#pragma unroll
    for (int k = 0; k < L; k++) acc |= a[k] ^ b[k];
    return acc == 0;
}

// bit length of n (0 for n == 0)
template <int L>
__device__ __forceinline__ int bit_length(const uint32_t (&n)[L]) {
    int b = 0;
#pragma unroll
    for (int k = 0; k < L; k++)
        if (n[k]) b = 32 * k + 32 - __clz(n[k]);
    return b;
}

// Strong probable-prime test of odd n > base+1 to the given base
// (miller_rabin.h:216-248 for one base).  Returns true if n passes.
// One loop walks the bits of n-1 from the top: above bit s it squares and
// multiplies by the base; from bit s-1 down it is the squaring chain of the
// strong test, checked against 1 and n-1 after leaving Montgomery form.
template <int L>
__device__ __forceinline__ bool strong_prp(const uint32_t (&n)[L], uint32_t base) {
    const uint32_t ninv = neg_inv32(n[0]);
    const int B = bit_length<L>(n);
    // s = ctz(n - 1); n is odd so n - 1 = n with bit 0 cleared
    int s = 0;
    {
        bool found = false;
#pragma unroll
        for (int k = 0; k < L; k++) {
            const uint32_t w = (k == 0) ? (n[0] & ~1u) : n[k];
            if (!found && w) {
                s = 32 * k + __ffs(w) - 1;
                found = true;
            }
        }
    }
    // x = R mod n: 2^(B-1) < n doubled 32L - B + 1 times
    uint32_t x[L];
    {
        const int b = B - 1;
#pragma unroll
        for (int k = 0; k < L; k++) x[k] = (k == (b >> 5)) ? (1u << (b & 31)) : 0u;
        for (int i = 0; i < 32 * L - B + 1; i++) mod_dbl<L>(x, n);
    }
    // x = Mont(base): accounts for the top bit B-1 of n-1
    if (base == 2)
        mod_dbl<L>(x, n);
    else
        mod_mul_small<L>(x, n, base);
    uint32_t e[L];  // exponent words, indexed by a runtime bit position
#pragma unroll
    for (int k = 0; k < L; k++) e[k] = n[k];
    for (int b = B - 2;; b--) {
        if (b < s) {
            uint32_t t[2 * L + 1];
#pragma unroll
            for (int k = 0; k < 2 * L + 1; k++) t[k] = (k < L) ? x[k] : 0u;
            uint32_t y[L];
            mont_redc<L>(t, n, ninv, y);
            uint32_t d1 = y[0] ^ 1u, dm = y[0] ^ (n[0] & ~1u);
#pragma unroll
            for (int k = 1; k < L; k++) {
                d1 |= y[k];
                dm |= y[k] ^ n[k];
            }
            if (dm == 0) return true;             // base^(d 2^i) = -1
            if (d1 == 0) return b == s - 1;       // = 1: pass only for i = 0
            if (b == 0) return false;
        }
        mont_sqr<L>(x, n, ninv);
        if (b >= s && ((e[b >> 5] >> (b & 31)) & 1u)) {
            if (base == 2)
                mod_dbl<L>(x, n);
            else
                mod_mul_small<L>(x, n, base);
        }
    }
}

// true if n is odd and small enough that `base` proves nothing (n - 1 <= base):
// such n count as passing, as the oracle does.
template <int L>
__device__ __forceinline__ bool tiny_pass(const uint32_t (&n)[L], uint32_t base) {
    uint32_t hi = 0;
#pragma unroll
    for (int k = 1; k < L; k++) hi |= n[k];
    return hi == 0 && n[0] - 1 <= base;
}

// number of bases (2, 3, 5, ...) passed before the first failure
template <int L>
__device__ __forceinline__ int prp_rounds(const uint32_t (&n)[L], int rounds) {
    const uint32_t bases[16] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53};
    uint32_t hi = 0;
#pragma unroll
    for (int k = 1; k < L; k++) hi |= n[k];
    if ((n[0] & 1u) == 0 || (hi == 0 && n[0] < 3)) return 0;
    int passed = 0;
    for (int r = 0; r < rounds && r < 16; r++) {
        if (!tiny_pass<L>(n, bases[r]) && !strong_prp<L>(n, bases[r])) break;
        passed++;
    }
    return passed;
}

}  // namespace pg
