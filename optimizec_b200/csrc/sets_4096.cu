// sets_4096.cu — kernel set of N = 4096.
#include "kernel_sets.cuh"

namespace dns2d {

const KernelSet *kernel_sets_4096(int N)
{
    static const KernelSet sets[] = {
        Launch<4096>::make(),
    };
    for (const KernelSet &k : sets)
        if (k.N == N) return &k;
    return nullptr;
}

}  // namespace dns2d
