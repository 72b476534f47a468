// pg_inst.cu -- one limb count of the PRP kernels (built once per L with
// -DPG_LIMBS=L; see pg_search.cuh).
#include "pg_search.cuh"

#ifndef PG_LIMBS
#error "compile with -DPG_LIMBS=<limb count>"
#endif

namespace pg {
PG_INSTANTIATE_LIMBS(PG_LIMBS)
}  // namespace pg
