// Instantiation of the pass kernels for plans [0, 3) (split across files so nvcc builds them in parallel).
#include "pass_kernels.cuh"

void pk_fill_kernels_a(pkpass::KernelTable& t) { pkpass::Register<0, 3>::fill(t); }
