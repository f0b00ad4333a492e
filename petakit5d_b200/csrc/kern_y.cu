// Instantiation of the register-packing y pass kernels (pass_yreg.cuh) for the 256-point plan.
#include "pass_yreg.cuh"

void pk_fill_yreg(pkpass::YregTable& t) { pkpass::RegisterYreg<pkpass::kYregPlan, 0>::fill(t); }
