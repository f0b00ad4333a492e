// Instantiation of the pass kernels for plans [18, 24) (split across files so nvcc builds them in parallel).
#include "pass_kernels.cuh"

void pk_fill_kernels_e(pkpass::KernelTable& t) { pkpass::Register<18, 24>::fill(t); }
