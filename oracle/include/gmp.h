/* TEST INFRASTRUCTURE ONLY: <gmp.h> for compiling the reference's own
 * gap_common.cpp and overflow.cpp into oracle/_ref (gmp.h is not installed
 * here; the GMP 6.3.0 runtime is).  Forwards to the hand-written
 * declarations of the public mpz ABI. */
#include "../gmp_shim.h"
