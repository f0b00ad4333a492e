// Instantiation of the pass kernels for plans [24, 30) (split across files so nvcc builds them in parallel).
#include "pass_kernels.cuh"

void pk_fill_kernels_f(pkpass::KernelTable& t) { pkpass::Register<24, 30>::fill(t); }
