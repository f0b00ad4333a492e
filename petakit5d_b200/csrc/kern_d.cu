// Instantiation of the pass kernels for plans [12, 18) (split across files so nvcc builds them in parallel).
#include "pass_kernels.cuh"

void pk_fill_kernels_d(pkpass::KernelTable& t) { pkpass::Register<12, 18>::fill(t); }
