// sets_256.cu — kernel sets of N = 256 and 512 (three radix plans each, rows per CTA variants).
#include "kernel_sets.cuh"

namespace dns2d {

const KernelSet *kernel_sets_256(int N)
{
    static const KernelSet sets[] = {
        Launch<256>::make(),
        Launch<512>::make(),
    };
    for (const KernelSet &k : sets)
        if (k.N == N) return &k;
    return nullptr;
}

}  // namespace dns2d
