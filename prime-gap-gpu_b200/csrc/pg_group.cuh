// pg_group.cuh -- multi-precision Montgomery arithmetic with one number spread
// over a group of T lanes (T in {4, 8, 16, 32}), LT words per lane, L = T*LT.
//
// For operands too wide for one thread's registers (P = 3001: 4 248-bit N,
// 136 words).  Lane g of a group holds words [g*LT, (g+1)*LT) of every value.
// Multiplication is CIOS, row by row: the row's word of `a` is broadcast by a
// warp shuffle, every lane multiplies its slice, lane 0 of the group derives
// the Montgomery factor q and broadcasts it, and each lane hands the word
// leaving its bottom to the lane below.  Carries leaving a lane's slice are
// not passed on at once: they stay in the top words of the lane's window
// (they belong to the next lane's lowest words), so a row has no serial carry
// chain across lanes.  What remains at the end is resolved in one step by
// carry lookahead over warp ballots (generate / propagate bits per lane,
// added as integers).
//
// Every shuffle and ballot names only the group's lanes, so the groups of a
// warp may diverge (one idle, another still squaring).
//
// Values are kept in [0, 2n) ("almost Montgomery"): with 4n < R = 2^(32L),
// a product of two values below 2n is again below 2n, so no conditional
// subtraction is needed per multiplication.  Callers pick L with at least two
// spare bits above the bit length of n.
#pragma once

#include <cstdint>

#include "pg_mont.cuh"

namespace pg {

template <int T>
struct Group {
    static_assert(T == 2 || T == 4 || T == 8 || T == 16 || T == 32, "group size");
    uint32_t lane, gl, gb;  // lane in warp, lane in group, first lane of the group
    uint32_t gmask;         // the group's lanes as a bit mask
    __device__ __forceinline__ Group() {
        lane = threadIdx.x & 31;
        gl = lane & (T - 1);
        gb = lane - gl;
        gmask = (T == 32) ? 0xffffffffu : (((1u << T) - 1) << gb);
    }
    // the group's T bits of a warp ballot, lane gb at bit 0
    __device__ __forceinline__ uint32_t field(uint32_t ballot) const {
        return (T == 32) ? ballot : ((ballot >> gb) & ((1u << T) - 1));
    }
};

// Carry-in of this lane when every lane has a carry-out bit g (generate) and
// a slice that would pass an incoming carry on (p, all ones): the carries of
// a ripple through the group, found by adding (g|p) + g as T-bit integers.
// Returns the lane's carry-in; *out receives the group's final carry-out.
template <int T>
__device__ __forceinline__ uint32_t lookahead(const Group<T> &G, bool g, bool p, uint32_t *out) {
    const uint64_t gf = G.field(__ballot_sync(G.gmask, g));
    const uint64_t pf = G.field(__ballot_sync(G.gmask, p));
    const uint64_t a = gf | pf;
    const uint64_t c = (a + gf) ^ a ^ gf;  // bit i = carry into lane i (bit T = out of the group)
    if (out) *out = (uint32_t)((c >> T) & 1u);
    return (uint32_t)((c >> G.gl) & 1u);
}

// x (slice) += cin (0 or 1) through the LT words
template <int LT>
__device__ __forceinline__ void slice_add_bit(uint32_t (&x)[LT], uint32_t cin) {
    x[0] = add_cc(x[0], cin);
#pragma unroll
    for (int k = 1; k < LT; k++) x[k] = (k + 1 < LT) ? addc_cc(x[k], 0u) : addc(x[k], 0u);
}

// Adds the pending 64-bit value `in` (which belongs at this lane's lowest
// word) and resolves all carries across the group.  Returns the group's final
// carry-out (identical in every lane).
template <int T, int LT>
__device__ __forceinline__ uint32_t resolve_in(const Group<T> &G, uint32_t (&x)[LT], uint64_t in) {
    static_assert(LT >= 2, "a lane holds at least two words");
    x[0] = add_cc(x[0], (uint32_t)in);
    if (LT > 1) {
        x[1 < LT ? 1 : 0] = addc_cc(x[1 < LT ? 1 : 0], (uint32_t)(in >> 32));
#pragma unroll
        for (int k = 2; k < LT; k++) x[k] = addc_cc(x[k], 0u);
    }
    const uint32_t g = addc(0u, 0u) | (LT == 1 ? (uint32_t)(in >> 32) : 0u);
    uint32_t all1 = 0xffffffffu;
#pragma unroll
    for (int k = 0; k < LT; k++) all1 &= x[k];
    uint32_t out;
    const uint32_t cin = lookahead<T>(G, g != 0, all1 == 0xffffffffu, &out);
    slice_add_bit<LT>(x, cin);
    return out;
}

// d = x - y across the group; returns 1 when x < y (a borrow leaves the top)
template <int T, int LT>
__device__ __forceinline__ uint32_t group_sub(const Group<T> &G, uint32_t (&d)[LT], const uint32_t (&x)[LT],
                                              const uint32_t (&y)[LT]) {
    d[0] = sub_cc(x[0], y[0]);
#pragma unroll
    for (int k = 1; k < LT; k++) d[k] = subc_cc(x[k], y[k]);
    const uint32_t bout = subc(0u, 0u) & 1u;  // borrow out of the slice
    uint32_t all0 = 0;
#pragma unroll
    for (int k = 0; k < LT; k++) all0 |= d[k];
    uint32_t out;
    const uint32_t bin = lookahead<T>(G, bout != 0, all0 == 0, &out);
    // subtract the incoming borrow
    d[0] = sub_cc(d[0], bin);
#pragma unroll
    for (int k = 1; k < LT; k++) d[k] = (k + 1 < LT) ? subc_cc(d[k], 0u) : subc(d[k], 0u);
    return out;
}

template <int T, int LT>
__device__ __forceinline__ bool group_eq(const uint32_t (&x)[LT], const uint32_t (&y)[LT]) {
    uint32_t acc = 0;
#pragma unroll
    for (int k = 0; k < LT; k++) acc |= x[k] ^ y[k];
    const Group<T> G;
    return G.field(__ballot_sync(G.gmask, acc != 0)) == 0;
}

// acc (slice) + spill += ai * b (slice): lo products chain over the slice, hi
// products one word up; what leaves the slice is added to the spill.  One row
// only (building a candidate m*K), so the two chains are left unfused.
template <int LT>
__device__ __forceinline__ void row_mac(uint32_t (&acc)[LT], uint64_t &spill, uint32_t ai, const uint32_t (&b)[LT]) {
    acc[0] = mad_lo_cc(ai, b[0], acc[0]);
#pragma unroll
    for (int k = 1; k < LT; k++) acc[k] = madc_lo_cc(ai, b[k], acc[k]);
    const uint32_t c1 = addc(0u, 0u);
    uint32_t h;
    if (LT > 1) {
        acc[1 < LT ? 1 : 0] = mad_hi_cc(ai, b[0], acc[1 < LT ? 1 : 0]);
#pragma unroll
        for (int k = 1; k < LT - 1; k++) acc[k + 1] = madc_hi_cc(ai, b[k], acc[k + 1]);
        h = madc_hi(ai, b[LT - 1], c1);
    } else {
        h = __umulhi(ai, b[0]) + c1;
    }
    spill += h;
}

// Products m*v[k] of one row, k < LT, added at positions S + k of the lane's
// window (S is a constant once the caller's row loop is unrolled): products
// whose low word lands at an even position go to E (pairs E[P], E[P+1]), at an
// odd position to H (pairs H[P], H[P+1]), so every link is one fused
// multiply-add on an aligned register pair.  Each chain's carry out is added
// two words up (the top words only gather carries and cannot overflow).
template <int LT, int PH>
__device__ __forceinline__ void gmac_row(uint32_t (&E)[PH], uint32_t (&H)[PH], int S, uint32_t m,
                                         const uint32_t (&v)[LT]) {
#pragma unroll
    for (int par = 0; par < 2; par++) {  // par 0: even positions (E), 1: odd (H)
        const int k0 = ((S & 1) == par) ? 0 : 1;
        if (k0 >= LT) continue;
        const int kl = k0 + ((LT - 1 - k0) / 2) * 2;
#pragma unroll
        for (int k = k0; k < LT; k += 2) {
            const int P = S + k;
            if (par == 0) {
                if (k == k0) mad_link<true>(E[P], E[P + 1], m, v[k]);
                else mad_link<false>(E[P], E[P + 1], m, v[k]);
            } else {
                if (k == k0) mad_link<true>(H[P], H[P + 1], m, v[k]);
                else mad_link<false>(H[P], H[P + 1], m, v[k]);
            }
        }
        const int C = S + kl + 2;
        if (par == 0) {
            E[C] = addc_cc(E[C], 0u);
            E[C + 1] = addc(E[C + 1], 0u);
        } else {
            H[C] = addc_cc(H[C], 0u);
            H[C + 1] = addc(H[C + 1], 0u);
        }
    }
}

// r = a * b * R^-1 mod n, inputs and output in [0, 2n), 4n < R.  CIOS, row by
// row: the row's word of a is broadcast by a shuffle, every lane multiplies
// its slice, lane 0 derives the Montgomery factor q and broadcasts it.  The
// accumulator is kept as two arrays (E, H) in a window that moves up one word
// per row instead of being shifted down (a shift would change the register
// pairing of every word and cost moves on every product): row w
// of a source lane's LT rows works at offset w, so every index is a
// compile-time constant and every product is one fused 64-bit multiply-add;
// after the LT rows the window is moved back by LT words.  The word leaving a
// lane's bottom is E + H plus the carry kept from the previous bottom word;
// its low 32 bits go to the lane below, which adds them LT words up, and its
// carry (one bit) stays in the lane, in c0, for its next bottom word (the
// same position, so one shuffle per row carries the hand-down).  In lane 0
// the low word is 0 mod 2^32 (the Montgomery step) and only the carry stays.
template <int T, int LT>
__device__ __forceinline__ void gmont_mul(const Group<T> &G, uint32_t (&r)[LT], const uint32_t (&a)[LT],
                                           const uint32_t (&b)[LT], const uint32_t (&n)[LT], uint32_t ninv) {
    constexpr int PH = 2 * LT + 4;
    uint32_t E[PH], H[PH];
#pragma unroll
    for (int k = 0; k < PH; k++) E[k] = H[k] = 0;
    uint32_t c0 = 0;  // carry into the lane's bottom word
    const bool bottom = G.gl == 0, top = G.gl == T - 1;
#pragma unroll 1
    for (int src = 0; src < T; src++) {
#pragma unroll
        for (int w = 0; w < LT; w++) {
            const uint32_t ai = __shfl_sync(G.gmask, a[w], G.gb + src);
            gmac_row<LT, PH>(E, H, w, ai, b);
            // Montgomery factor from lane 0's bottom word
            uint32_t q = add_cc(E[w], H[w]);
            q = add_cc(q, c0);
            q = __shfl_sync(G.gmask, q * ninv, G.gb);
            gmac_row<LT, PH>(E, H, w, q, n);
            // the bottom word leaves: 0 mod 2^32 in lane 0 (its carry stays),
            // handed to the lane below elsewhere
            uint32_t lo = add_cc(E[w], H[w]);
            const uint32_t hi = addc(0u, 0u);
            lo = add_cc(lo, c0);
            c0 = addc(hi, 0u);
            uint32_t rlo = __shfl_down_sync(G.gmask, lo, 1);
            if (top) rlo = 0;
            const int P = w + LT;
            if ((P & 1) == 0) {
                E[P] = add_cc(E[P], rlo);
                E[P + 1] = addc_cc(E[P + 1], 0u);
                E[P + 2] = addc(E[P + 2], 0u);
            } else {
                H[P] = add_cc(H[P], rlo);
                H[P + 1] = addc_cc(H[P + 1], 0u);
                H[P + 2] = addc(H[P + 2], 0u);
            }
        }
        // move the window back by LT words
#pragma unroll
        for (int k = 0; k < PH; k++) {
            E[k] = k + LT < PH ? E[k + LT] : 0u;
            H[k] = k + LT < PH ? H[k + LT] : 0u;
        }
    }
    // the slice (positions 0 .. LT-1) and what lies above it (LT, LT+1), plus
    // the lane's last bottom carry at position 0
    uint32_t R[LT + 2];
    R[0] = add_cc(E[0], H[0]);
#pragma unroll
    for (int k = 1; k < LT + 2; k++) R[k] = (k + 1 < LT + 2) ? addc_cc(E[k], H[k]) : addc(E[k], H[k]);
    R[0] = add_cc(R[0], c0);
#pragma unroll
    for (int k = 1; k < LT + 2; k++) R[k] = (k + 1 < LT + 2) ? addc_cc(R[k], 0u) : addc(R[k], 0u);
    const uint64_t spill = ((uint64_t)R[LT + 1] << 32) | R[LT];
    const uint32_t slo = __shfl_up_sync(G.gmask, (uint32_t)spill, 1);
    const uint32_t shi = __shfl_up_sync(G.gmask, (uint32_t)(spill >> 32), 1);
    const uint64_t in = bottom ? 0ull : ((uint64_t)shi << 32 | slo);
    uint32_t acc[LT];
#pragma unroll
    for (int k = 0; k < LT; k++) acc[k] = R[k];
    resolve_in<T, LT>(G, acc, in);
#pragma unroll
    for (int k = 0; k < LT; k++) r[k] = acc[k];
}

// x = 2x mod 2n for x in [0, 2n): shift left one bit across the group, then
// subtract 2n (n2) unless that borrows
template <int T, int LT>
__device__ __forceinline__ void gdbl(const Group<T> &G, uint32_t (&x)[LT], const uint32_t (&n2)[LT]) {
    uint32_t y[LT];
    const uint32_t topbit = x[LT - 1] >> 31;
    uint32_t in = __shfl_up_sync(G.gmask, topbit, 1);
    if (G.gl == 0) in = 0;
#pragma unroll
    for (int k = LT - 1; k >= 1; k--) y[k] = __funnelshift_l(x[k - 1], x[k], 1);
    y[0] = (x[0] << 1) | in;
    uint32_t d[LT];
    const uint32_t borrow = group_sub<T, LT>(G, d, y, n2);
#pragma unroll
    for (int k = 0; k < LT; k++) x[k] = borrow ? y[k] : d[k];
}

// Strong probable-prime test of the odd group-held n (> base + 1) to `base`
// (miller_rabin.h:216-248 for one base).  bits(n) <= 32*L - 2 is required.
template <int T, int LT>
__device__ __forceinline__ bool gstrong_prp(const Group<T> &G, const uint32_t (&n)[LT], uint32_t base) {
    // ninv from the lowest word (lane 0), B and s = ctz(n-1) over the group
    const uint32_t n0 = __shfl_sync(G.gmask, n[0], G.gb);
    const uint32_t ninv = neg_inv32(n0);
    int myB = 0, myS = 1 << 30;
#pragma unroll
    for (int k = 0; k < LT; k++) {
        const int wi = G.gl * LT + k;
        if (n[k]) myB = 32 * wi + 32 - __clz(n[k]);
        const uint32_t w = (wi == 0) ? (n[k] & ~1u) : n[k];
        if (w && myS == (1 << 30)) myS = 32 * wi + __ffs(w) - 1;
    }
#pragma unroll
    for (int o = 1; o < T; o <<= 1) {
        myB = max(myB, __shfl_xor_sync(G.gmask, myB, o));
        myS = min(myS, __shfl_xor_sync(G.gmask, myS, o));
    }
    const int B = myB, s = myS;
    // n2 = 2n
    uint32_t n2[LT];
    {
        const uint32_t topbit = n[LT - 1] >> 31;
        uint32_t in = __shfl_up_sync(G.gmask, topbit, 1);
        if (G.gl == 0) in = 0;
#pragma unroll
        for (int k = LT - 1; k >= 1; k--) n2[k] = __funnelshift_l(n[k - 1], n[k], 1);
        n2[0] = (n[0] << 1) | in;
    }
    // one = R mod 2n (a value below 2n congruent to R): 2^(B-1) doubled 32L - B + 1 times
    uint32_t one[LT];
    {
        const int b = B - 1;
#pragma unroll
        for (int k = 0; k < LT; k++) one[k] = (G.gl * LT + k == (b >> 5)) ? (1u << (b & 31)) : 0u;
        for (int i = 0; i < 32 * T * LT - B + 1; i++) gdbl<T, LT>(G, one, n2);
    }
    // x = Mont(base): base * R, by doubling (base 2) or repeated addition
    uint32_t x[LT], bm[LT];
#pragma unroll
    for (int k = 0; k < LT; k++) x[k] = one[k];
    if (base == 2) {
        gdbl<T, LT>(G, x, n2);
    } else {
        for (uint32_t t = 1; t < base; t++) {  // x = x + one mod 2n
            uint32_t y[LT];
            y[0] = add_cc(x[0], one[0]);
#pragma unroll
            for (int k = 1; k < LT; k++) y[k] = addc_cc(x[k], one[k]);
            const uint32_t c = addc(0u, 0u);  // belongs to the next lane's lowest word
            const uint32_t cin = __shfl_up_sync(G.gmask, c, 1);
            resolve_in<T, LT>(G, y, G.gl == 0 ? 0ull : (uint64_t)cin);
            uint32_t d[LT];
            const uint32_t borrow = group_sub<T, LT>(G, d, y, n2);
#pragma unroll
            for (int k = 0; k < LT; k++) x[k] = borrow ? y[k] : d[k];
        }
    }
#pragma unroll
    for (int k = 0; k < LT; k++) bm[k] = x[k];
    // exponent words (n with bit 0 cleared), read by a runtime bit index
    uint32_t e[LT];
#pragma unroll
    for (int k = 0; k < LT; k++) e[k] = n[k];
    uint32_t unit[LT];  // the plain number 1
#pragma unroll
    for (int k = 0; k < LT; k++) unit[k] = (G.gl == 0 && k == 0) ? 1u : 0u;
    uint32_t nm1[LT];
#pragma unroll
    for (int k = 0; k < LT; k++) nm1[k] = (G.gl == 0 && k == 0) ? (n[0] & ~1u) : n[k];
    for (int b = B - 2;; b--) {
        if (b < s) {
            uint32_t y[LT];
            gmont_mul<T, LT>(G, y, x, unit, n, ninv);  // leave Montgomery form: y in [0, n]
            const bool is1 = group_eq<T, LT>(y, unit);
            const bool ism1 = group_eq<T, LT>(y, nm1);
            if (ism1) return true;
            if (is1) return b == s - 1;
            if (b == 0) return false;
        }
        gmont_mul<T, LT>(G, x, x, x, n, ninv);
        if (b >= s) {
            const int w = b >> 5;
            const uint32_t owner = (uint32_t)(w / LT);
            const int idx = w - (int)(G.gl * LT);
            const uint32_t mine = (idx >= 0 && idx < LT) ? e[idx] : 0u;
            const uint32_t word = __shfl_sync(G.gmask, mine, G.gb + owner);
            if ((word >> (b & 31)) & 1u) {
                if (base == 2)
                    gdbl<T, LT>(G, x, n2);
                else
                    gmont_mul<T, LT>(G, x, x, bm, n, ninv);
            }
        }
    }
}

}  // namespace pg
