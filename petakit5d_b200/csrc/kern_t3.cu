// Instantiation of the persistent TMA x / z pass kernels for plans [36, kNumPlans) (split across files so
// nvcc builds them in parallel).
#include "pass_tma.cuh"

void pk_fill_tma_3(pkpass::TmaTable& t) { pkpass::RegisterTma<36, kNumPlans>::fill(t); }
