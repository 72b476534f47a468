/* Test-only stand-in for the absent gmp.h: forwards to the oracle's
 * hand-written declarations of the GMP runtime's public mpz ABI. */
#include "../../../oracle/gmp_shim.h"
