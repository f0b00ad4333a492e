// Instantiation of the pass kernels for plans [41, 46) (split across files so nvcc builds them in parallel).
#include "pass_kernels.cuh"

void pk_fill_kernels_i(pkpass::KernelTable& t) { pkpass::Register<41, kNumPlans>::fill(t); }
