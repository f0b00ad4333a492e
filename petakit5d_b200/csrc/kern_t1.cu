// Instantiation of the persistent TMA x / z pass kernels for plans [12, 24) (split across files so
// nvcc builds them in parallel).
#include "pass_tma.cuh"

void pk_fill_tma_1(pkpass::TmaTable& t) { pkpass::RegisterTma<12, 24>::fill(t); }
