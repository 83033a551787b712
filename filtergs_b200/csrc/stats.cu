// OGFS key/value-pair statistics on the device (the reference copies the
// K-sized per-pair arrays to the host and loops over them on the CPU,
// antialias/cuda_rasterizer/rasterizer_impl.cu:479-556).
//
// One CTA per tile walks the tile's pairs: per-pair KPC bin (edges
// rasterizer_impl.cu:60-73), used/unused counts, and the per-tile alpha sum,
// used ratio (KPC_USED_THRESH) and pair count that define bar_g_tile.
#include "fgs_common.cuh"
#include "fgs_internal.h"

namespace fgs {

namespace {

constexpr int kBins = 11;

__global__ void __launch_bounds__(128) kpc_kernel(const uint2* __restrict__ ranges, const float* __restrict__ kv_sum,
                                                  const uint32_t* __restrict__ kv_cnt, float used_thresh,
                                                  double* __restrict__ out /* gtc, used, unused, bins[11] */,
                                                  double* __restrict__ tile_ratio, double* __restrict__ tile_total,
                                                  int num_tiles)
{
    const float edges[kBins] = {0.01f, 0.05f, 0.10f, 0.15f, 0.20f, 0.25f, 0.30f, 0.35f, 0.40f, 0.45f, 0.50f};
    __shared__ unsigned long long s_cnt[kBins + 3];  // bins, used, unused, used_in_tile
    __shared__ double s_sum;
    const int t = blockIdx.x;
    if (threadIdx.x < kBins + 3) s_cnt[threadIdx.x] = 0;
    if (threadIdx.x == 0) s_sum = 0.0;
    __syncthreads();
    const uint2 r = ranges[t];
    unsigned long long bins[kBins] = {0}, used = 0, unused = 0, used_tile = 0;
    double sum = 0.0;
    for (uint32_t k = r.x + threadIdx.x; k < r.y; k += blockDim.x) {
        const float v = kv_sum[k];
        const uint32_t c = kv_cnt[k];
        sum += (double)v;
        if (c > 0 && v >= used_thresh) used_tile++;
        if (c == 0) {
            unused++;
            continue;
        }
        int bin = 0;
        while (bin < kBins && v > edges[bin]) bin++;
        if (bin >= kBins) continue;  // above the last edge: neither used nor unused
        bins[bin]++;
        used++;
    }
#pragma unroll
    for (int b = 0; b < kBins; b++)
        if (bins[b]) atomicAdd(&s_cnt[b], bins[b]);
    if (used) atomicAdd(&s_cnt[kBins], used);
    if (unused) atomicAdd(&s_cnt[kBins + 1], unused);
    if (used_tile) atomicAdd(&s_cnt[kBins + 2], used_tile);
    if (sum != 0.0) atomicAdd(&s_sum, sum);
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t n = r.y > r.x ? r.y - r.x : 0;
        tile_total[t] = (double)n;
        tile_ratio[t] = n ? (double)s_cnt[kBins + 2] / (double)n : 0.0;
        if (n) atomicAdd(&out[0], s_sum / (double)n);
        if (s_cnt[kBins]) atomicAdd(&out[1], (double)s_cnt[kBins]);
        if (s_cnt[kBins + 1]) atomicAdd(&out[2], (double)s_cnt[kBins + 1]);
        for (int b = 0; b < kBins; b++)
            if (s_cnt[b]) atomicAdd(&out[3 + b], (double)s_cnt[b]);
    }
}

}  // namespace

// dev_out: [3 + 11 + 2 * num_tiles] doubles, zeroed here.
void launch_kpc_stats(const BinState& b, const ImageState& im, int num_tiles, float used_thresh, double* dev_out,
                      cudaStream_t s)
{
    cudaMemsetAsync(dev_out, 0, sizeof(double) * (3 + kBins + 2 * (size_t)num_tiles), s);
    if (num_tiles <= 0) return;
    kpc_kernel<<<num_tiles, 128, 0, s>>>(im.ranges, b.kv_sum, b.kv_cnt, used_thresh, dev_out, dev_out + 3 + kBins,
                                         dev_out + 3 + kBins + num_tiles, num_tiles);
    note_launches(1);
}

}  // namespace fgs
