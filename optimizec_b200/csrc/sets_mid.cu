// sets_mid.cu — kernel sets of N = 1024 and 2048.
#include "kernel_sets.cuh"

namespace dns2d {

const KernelSet *kernel_sets_mid(int N)
{
    static const KernelSet sets[] = {
        Launch<1024>::make(),
        Launch<2048>::make(),
    };
    for (const KernelSet &k : sets)
        if (k.N == N) return &k;
    return nullptr;
}

}  // namespace dns2d
