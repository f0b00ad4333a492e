// Instantiation of the fused x-z-x convolution kernels (pass_conv3.cuh) for the (x, z) length pairs
// built: 512 x 256, 256 x 512, 512 x 512 and 256 x 256 on 16-column tiles with two buffers and 8
// compute warps (at 12 or 16 compute warps the register cap of one CTA per SM makes them spill).
#include "pass_conv3.cuh"

void pk_fill_conv3(std::vector<pkpass::Conv3Entry>& v) {
    v.push_back(pkpass::conv3_entry<10, 9, 16, 2, 256>());
    v.push_back(pkpass::conv3_entry<9, 10, 16, 2, 256>());
    v.push_back(pkpass::conv3_entry<10, 10, 16, 2, 256>());
    v.push_back(pkpass::conv3_entry<9, 9, 16, 2, 256>());
}
