// sets_small.cu — kernel sets of the small single-CTA sizes (N = 16 ... 128).
#include "kernel_sets.cuh"

namespace dns2d {

const KernelSet *kernel_sets_small(int N)
{
    static const KernelSet sets[] = {
        Launch<16>::make(),
        Launch<32>::make(),
        Launch<64>::make(),
        Launch<128>::make(),
    };
    for (const KernelSet &k : sets)
        if (k.N == N) return &k;
    return nullptr;
}

}  // namespace dns2d
