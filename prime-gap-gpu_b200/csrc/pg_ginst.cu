// pg_ginst.cu -- one group layout of the PRP kernels (built once per entry of
// PG_GROUP_LIST with -DPG_GT=T -DPG_GLT=LT; see pg_search_group.cuh).
#include "pg_search_group.cuh"

#if !defined(PG_GT) || !defined(PG_GLT)
#error "compile with -DPG_GT=<lanes per number> -DPG_GLT=<words per lane>"
#endif

namespace pg {
PG_GINSTANTIATE(PG_GT, PG_GLT)
}  // namespace pg
