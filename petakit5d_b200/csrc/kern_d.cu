// Instantiation of the pass kernels for plans [36, kNumPlans) (split across files so nvcc builds them in parallel).
#include "pass_kernels.cuh"

void pk_fill_kernels_d(pkpass::KernelTable& t) { pkpass::Register<36, kNumPlans>::fill(t); }
