// Instantiation of the pass kernels for plans [24, 36) (split across files so nvcc builds them in parallel).
#include "pass_kernels.cuh"

void pk_fill_kernels_c(pkpass::KernelTable& t) { pkpass::Register<24, 36>::fill(t); }
