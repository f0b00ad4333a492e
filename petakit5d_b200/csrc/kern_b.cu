// Instantiation of the pass kernels for plans [3, 9) (split across files so nvcc builds them in parallel).
#include "pass_kernels.cuh"

void pk_fill_kernels_b(pkpass::KernelTable& t) { pkpass::Register<3, 9>::fill(t); }
