// gpufft-b200: one-kernel FP32 split products for transform lengths 2^10..2^12
// (rings N = 2^11..2^13); a separate translation unit so that the
// kernel instantiations compile in parallel.
#include "gf_split.cuh"

namespace gfb
{
int launch_split_single_hi(int L, const SplitArgs& a, long long ctas, cudaStream_t s)
{
    return dispatch_int<10, 12>(L, [&]<int LL>() {
        return dispatch_int<1, SPLIT_SINGLE_MAX_LIMBS>(a.k, [&]<int KK>() { return launch_mid_k<LL, true, KK>(a, ctas, s); });
    });
}
} // namespace gfb
