// sets_16384.cu — kernel set of the cluster size N = 16384.
#include "kernel_sets.cuh"

namespace dns2d {

const KernelSet *kernel_sets_16384(int N)
{
    static const KernelSet sets[] = {
        LaunchC<16384>::make(),
    };
    for (const KernelSet &k : sets)
        if (k.N == N) return &k;
    return nullptr;
}

}  // namespace dns2d
