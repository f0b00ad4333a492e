// Instantiation of the persistent TMA x / z pass kernels for plans [0, 12) (split across files so
// nvcc builds them in parallel).
#include "pass_tma.cuh"

void pk_fill_tma_0(pkpass::TmaTable& t) { pkpass::RegisterTma<0, 12>::fill(t); }
