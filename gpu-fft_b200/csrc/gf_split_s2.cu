// gpufft-b200: one-kernel FP32 split products for transform lengths 2^7..2^9
// (rings N = 2^8..2^10); a separate translation unit so that the
// kernel instantiations compile in parallel.
#include "gf_split.cuh"

namespace gfb
{
int launch_split_single_mid(int L, const SplitArgs& a, long long ctas, cudaStream_t s)
{
    return dispatch_int<7, 9>(L, [&]<int LL>() {
        return dispatch_int<1, SPLIT_SINGLE_MAX_LIMBS>(a.k, [&]<int KK>() { return launch_mid_k<LL, true, KK>(a, ctas, s); });
    });
}
} // namespace gfb
