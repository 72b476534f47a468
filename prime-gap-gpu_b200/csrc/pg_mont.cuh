// pg_mont.cuh -- multi-precision Montgomery arithmetic for the strong PRP test.
//
// One thread owns one L-word number: the operand, the modulus and the
// double-width accumulator (two arrays, see "Register layout" below) all live
// in registers (the loops below are fully unrolled over the compile-time L,
// so every array index is a constant).  Products use PTX multiply-add carry
// chains (mad.lo.cc / madc.hi.cc, fused by ptxas into one 64-bit multiply-add
// per limb product), i.e. integer multiply-add only -- no floating point and
// no tensor cores: this is exact multi-precision integer arithmetic.
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
//
// Register layout.  The fused 32x32+64 multiply-add writes a 64-bit pair of
// registers that must be aligned, so a single accumulator array whose chains
// start at both even and odd word positions costs register moves on every
// product of the odd-aligned chains.  Instead the running value is kept as
//     E + F*B + C*B^L          (B = 2^32)
// with products whose low word lands at an even position accumulated in E
// (pairs E[p], E[p+1]) and those landing at an odd position in F (F[k] holds
// position k+1, pairs F[p-1], F[p]): every multiply-add of every chain works
// on an aligned pair.  C counts the carries out of the reduction's chains
// (positions L .. 2L) so they never ripple.  The sums that resolve a word
// from E, F and the carry below are written as PTX carry chains too: left to
// the compiler they interleave with the multiply chains and force the carry
// flag through general registers.

// (lo, hi) += a*b as one link of a carry chain (FIRST: no carry in)
template <bool FIRST>
__device__ __forceinline__ void mad_link(uint32_t &lo, uint32_t &hi, uint32_t a, uint32_t b) {
    lo = FIRST ? mad_lo_cc(a, b, lo) : madc_lo_cc(a, b, lo);
    hi = madc_hi_cc(a, b, hi);
}

// x = (E + F*B) * R^-1 mod n for E + F*B < n*R (x < n), R = B^L.
template <int L>
__device__ __forceinline__ void mont_redc_ef(uint32_t (&E)[2 * L + 2], uint32_t (&F)[2 * L + 2],
                                             const uint32_t (&n)[L], uint32_t ninv, uint32_t (&x)[L]) {
    uint32_t C[L + 2];
#pragma unroll
    for (int k = 0; k < L + 2; k++) C[k] = 0;
    uint32_t cin = 0;  // carry into position i from the resolved positions below
#pragma unroll
    for (int i = 0; i < L; i++) {
        uint32_t w = E[i];  // word i of the running value
        if (i) {
            w = add_cc(E[i], F[i - 1]);
            w = add_cc(w, cin);
        }
        const uint32_t q = w * ninv;
        // chain over E (j with i + j even) and chain over F (i + j odd); each
        // chain's carry out is counted in C at its position (>= L)
#pragma unroll
        for (int par = 0; par < 2; par++) {
            const int j0 = (i + par) & 1;
            int jl = j0;
#pragma unroll
            for (int j = j0; j < L; j += 2) jl = j;
#pragma unroll
            for (int j = j0; j < L; j += 2) {
                const int p = i + j;
                if (par == 0) {
                    if (j == j0) mad_link<true>(E[p], E[p + 1], q, n[j]);
                    else mad_link<false>(E[p], E[p + 1], q, n[j]);
                } else {
                    if (j == j0) mad_link<true>(F[p - 1], F[p], q, n[j]);
                    else mad_link<false>(F[p - 1], F[p], q, n[j]);
                }
            }
            const int cp = i + jl + 2;
            if (cp <= 2 * L) C[cp - L] = addc(C[cp - L], 0u);
        }
        // position i now sums to a multiple of B (the REDC identity); its carry
        // (0..2) moves up.  At i = 0 the carry went up inside the pair add.
        if (i) {
            const uint32_t z = add_cc(E[i], F[i - 1]);
            const uint32_t k1 = addc(0u, 0u);
            (void)add_cc(z, cin);
            cin = addc(k1, 0u);
        }
    }
    // u = positions L .. 2L of the sum (u < 2n), then x = u mod n
    C[0] += cin;
    uint32_t A[L + 1], u[L + 1];
    A[0] = add_cc(E[L], F[L - 1]);
#pragma unroll
    for (int k = 1; k < L; k++) A[k] = addc_cc(E[L + k], F[L + k - 1]);
    A[L] = addc(E[2 * L], F[2 * L - 1]);
    u[0] = add_cc(A[0], C[0]);
#pragma unroll
    for (int k = 1; k < L; k++) u[k] = addc_cc(A[k], C[k]);
    u[L] = addc(A[L], C[L]);
    uint32_t d[L];
    d[0] = sub_cc(u[0], n[0]);
#pragma unroll
    for (int k = 1; k < L; k++) d[k] = subc_cc(u[k], n[k]);
    const uint32_t top = subc(u[L], 0u);  // 0 if u >= n, 0xffffffff on borrow
    const bool keep = top != 0;
#pragma unroll
    for (int k = 0; k < L; k++) x[k] = keep ? u[k] : d[k];
}

// REDC of the 2L+1 word value t (< n*R): returns t * R^-1 mod n in x (< n).
template <int L>
__device__ __forceinline__ void mont_redc(uint32_t (&t)[2 * L + 1], const uint32_t (&n)[L], uint32_t ninv,
                                          uint32_t (&x)[L]) {
    uint32_t E[2 * L + 2], F[2 * L + 2];
#pragma unroll
    for (int k = 0; k < 2 * L + 2; k++) {
        E[k] = k < 2 * L + 1 ? t[k] : 0u;
        F[k] = 0;
    }
    mont_redc_ef<L>(E, F, n, ninv, x);
}

// x = x^2 * R^-1 mod n (x < n in and out).  Cross products once, doubled,
// diagonal squares added, then REDC.
template <int L>
__device__ __forceinline__ void mont_sqr(uint32_t (&x)[L], const uint32_t (&n)[L], uint32_t ninv) {
    uint32_t E[2 * L + 2], F[2 * L + 2];
#pragma unroll
    for (int k = 0; k < 2 * L + 2; k++) E[k] = F[k] = 0;
    // cross products x_i * x_j (j > i) at position i + j, row i in two chains
    // (j - i odd, j - i even).  Each array stays below B^(i+L+1) after row i,
    // so a chain's carry out stops in the word above its top pair, and the
    // chain that ends at j = L - 1 (top pair at i+L-1, i+L) has none at all.
#pragma unroll
    for (int i = 0; i < L - 1; i++) {
        const uint32_t a = x[i];
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const int j0 = i + 1 + c;
            if (j0 >= L) continue;
            const int jl = j0 + ((L - 1 - j0) / 2) * 2;
            const bool top = jl == L - 1;
#pragma unroll
            for (int j = j0; j < L; j += 2) {
                const int p = i + j;
                uint32_t &lo = (p & 1) == 0 ? E[p] : F[p - 1];
                uint32_t &hi = (p & 1) == 0 ? E[p + 1] : F[p];
                lo = j == j0 ? mad_lo_cc(a, x[j], lo) : madc_lo_cc(a, x[j], lo);
                hi = (j == jl && top) ? madc_hi(a, x[j], hi) : madc_hi_cc(a, x[j], hi);
            }
            if (!top) {
                const int cp = i + jl + 2;
                if ((cp & 1) == 0)
                    E[cp] = addc(E[cp], 0u);
                else
                    F[cp - 1] = addc(F[cp - 1], 0u);
            }
        }
    }
    // double both arrays (each holds less than half of B^(2L))
#pragma unroll
    for (int k = 2 * L - 1; k >= 1; k--) E[k] = __funnelshift_l(E[k - 1], E[k], 1);
    E[0] <<= 1;
#pragma unroll
    for (int k = 2 * L - 1; k >= 1; k--) F[k] = __funnelshift_l(F[k - 1], F[k], 1);
    F[0] <<= 1;
    // diagonal squares x_i^2 at the even positions 2i, one chain into E
    mad_link<true>(E[0], E[1], x[0], x[0]);
#pragma unroll
    for (int i = 1; i < L; i++) {
        E[2 * i] = madc_lo_cc(x[i], x[i], E[2 * i]);
        if (i + 1 < L)
            E[2 * i + 1] = madc_hi_cc(x[i], x[i], E[2 * i + 1]);
        else
            E[2 * i + 1] = madc_hi(x[i], x[i], E[2 * i + 1]);
    }
    mont_redc_ef<L>(E, F, n, ninv, x);
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
