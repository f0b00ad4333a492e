// Instantiation of the pass kernels for plans [36, 41) (split across files so nvcc builds them in parallel).
#include "pass_kernels.cuh"

void pk_fill_kernels_h(pkpass::KernelTable& t) { pkpass::Register<36, 41>::fill(t); }
