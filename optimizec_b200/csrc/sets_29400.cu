// sets_29400.cu — kernel set of the cluster size N = 29400.
#include "kernel_sets.cuh"

namespace dns2d {

const KernelSet *kernel_sets_29400(int N)
{
    static const KernelSet sets[] = {
        LaunchC<29400>::make(),
    };
    for (const KernelSet &k : sets)
        if (k.N == N) return &k;
    return nullptr;
}

}  // namespace dns2d
