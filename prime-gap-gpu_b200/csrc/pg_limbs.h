// pg_limbs.h -- the operand layouts the library is compiled for.
//
// PG_LIMB_LIST: one thread per number, L words in its registers.  An operand
// of w words runs on the smallest listed L >= w.
// PG_GROUP_LIST: one number spread over a group of T lanes, LT words per lane
// (L = T*LT words, used with two spare bits: bits(N) <= 32*L - 2).
// The build script reads both lists to compile one object per entry.
#pragma once

#define PG_LIMB_LIST(X) X(4) X(8) X(12) X(15) X(16) X(20) X(22) X(23) X(24) X(28) X(32) X(36) X(40) X(44) X(48)

#define PG_GROUP_LIST(X) \
    X(8, 3) X(4, 6) X(4, 8) X(4, 10) X(4, 12) X(8, 8) X(8, 12) X(8, 17) X(8, 20) X(16, 2) X(16, 3) X(16, 9)

// layout codes: L for one thread per number, (T << 16) | L for groups of T lanes
#define PG_LAYOUT_GROUP(T, L) (((uint32_t)(T) << 16) | (uint32_t)(L))
