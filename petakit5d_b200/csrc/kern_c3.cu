// Instantiation of the fused x-z-x convolution kernels (pass_conv3.cuh) for the (x, z) length pairs
// built, on 16-column tiles with 16 compute warps plus the loader and storer warps (96 registers a
// thread at one CTA per SM): 512 x 256 and 256 x 256 with three buffers that each carry a z item's
// OTF tile, 256 x 512 and 512 x 512 with two buffers and one OTF buffer.
#include "pass_conv3.cuh"

void pk_fill_conv3(std::vector<pkpass::Conv3Entry>& v) {
    v.push_back(pkpass::conv3_entry<10, 9, 16, 3, 512>());
    v.push_back(pkpass::conv3_entry<9, 10, 16, 2, 512>());
    v.push_back(pkpass::conv3_entry<10, 10, 16, 2, 512>());
    v.push_back(pkpass::conv3_entry<9, 9, 16, 3, 512>());
}
