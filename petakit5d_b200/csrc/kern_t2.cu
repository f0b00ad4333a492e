// Instantiation of the persistent TMA x / z pass kernels for plans [24, 36) (split across files so
// nvcc builds them in parallel).
#include "pass_tma.cuh"

void pk_fill_tma_2(pkpass::TmaTable& t) { pkpass::RegisterTma<24, 36>::fill(t); }
