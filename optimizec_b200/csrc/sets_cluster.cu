// sets_cluster.cu — kernel sets of the cluster sizes N = 840, 8192 and 9216.
#include "kernel_sets.cuh"

namespace dns2d {

const KernelSet *kernel_sets_cluster(int N)
{
    static const KernelSet sets[] = {
        LaunchC<840>::make(),
        LaunchC<8192>::make(),
        LaunchC<9216>::make(),
    };
    for (const KernelSet &k : sets)
        if (k.N == N) return &k;
    return nullptr;
}

}  // namespace dns2d
