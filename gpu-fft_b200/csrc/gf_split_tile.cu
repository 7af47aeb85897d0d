// gpufft-b200: launcher and C ABI of the split product's shared-memory tile
// kernel (gf_split_tile.cuh), in a translation unit of its own.
#include "gf_split_tile.cuh"

namespace gfb
{
template <int K> static int launch_tile_k(const SplitArgs& a, long long tiles, cudaStream_t s)
{
    static int done[64] = {0};
    const size_t smem = stile::smem_bytes(K);
    int st = ensure_smem(split_tile_kernel<K>, smem, done);
    if (st) return st;
    const long long grid = tiles < (long long)sm_count() ? tiles : (long long)sm_count();
    // 2k limb tiles in, 2k-1 group tiles out
    GF_TRACE(tr, (double)tiles * stile::P * sizeof(float2) * (4 * K - 1), s, "split_tile<k%d>", K);
    return launch_k(split_tile_kernel<K>, dim3((unsigned)grid), dim3(stile::NTT), smem, s, a, tiles);
}

int launch_split_tile(int k, const SplitArgs& a, long long tiles, cudaStream_t s)
{
    if (tiles <= 0) return GPUFFT_SUCCESS;
    return dispatch_int<1, SPLIT_TILE_MAXK>(k, [&]<int KK>() { return launch_tile_k<KK>(a, tiles, s); });
}
} // namespace gfb

extern "C" int gpufft_split_wait_timeouts(unsigned* count, int clear)
{
    if (!count) return GPUFFT_ERROR_INVALID_VALUE;
    cudaError_t e = cudaMemcpyFromSymbol(count, gfb::g_split_wait_timeouts, sizeof(unsigned));
    if (e != cudaSuccess) return gfb::set_cuda_error(e);
    if (clear)
    {
        const unsigned zero = 0;
        e = cudaMemcpyToSymbol(gfb::g_split_wait_timeouts, &zero, sizeof(unsigned));
        if (e != cudaSuccess) return gfb::set_cuda_error(e);
    }
    return GPUFFT_SUCCESS;
}
