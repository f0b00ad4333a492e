// Instantiation of the pass kernels for plans [30, 36) (split across files so nvcc builds them in parallel).
#include "pass_kernels.cuh"

void pk_fill_kernels_g(pkpass::KernelTable& t) { pkpass::Register<30, 36>::fill(t); }
