// Instantiation of the pass kernels for plans [9, 12) (split across files so nvcc builds them in parallel).
#include "pass_kernels.cuh"

void pk_fill_kernels_c(pkpass::KernelTable& t) { pkpass::Register<9, 12>::fill(t); }
