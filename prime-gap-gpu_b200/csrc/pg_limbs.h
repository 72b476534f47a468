// pg_limbs.h -- the limb counts (32-bit words per PRP operand) the library
// is compiled for.  An operand of w words runs on the smallest listed L >= w.
// The build script reads this list to compile one pg_inst.cu object per L.
#pragma once

#define PG_LIMB_LIST(X) X(4) X(8) X(12) X(15) X(16) X(20) X(22) X(23) X(24) X(28) X(32) X(36) X(40) X(44) X(48)
