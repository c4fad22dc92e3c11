// Split-BF16 tensor-core density solver: placeholder until the tcgen05 GEMMs land.
#include "poisson_internal.h"

namespace gpl {

cudaError_t tc_plan_init(PoissonPlan *, const BasisHost &) { return cudaErrorNotSupported; }
void tc_plan_free(PoissonPlan *) {}
cudaError_t tc_solve(PoissonPlan *, float *, float *, cudaStream_t) { return cudaErrorNotSupported; }
int tc_launches(const PoissonPlan *) { return 0; }

}  // namespace gpl
