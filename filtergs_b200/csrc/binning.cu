// Binning: depth ordering, duplicateWithKeys, onesweep radix sort by tile,
// tile ranges (antialias/cuda_rasterizer/rasterizer_impl.cu:113-194,363-445).
//
// The reference stably sorts 64-bit (tile << 32 | depth bits) keys of all K
// pairs with a 6-pass LSD radix sort.  An LSD sort's first four passes only
// look at the depth bits, and every pair of a Gaussian carries the same
// depth, so the same permutation is obtained by (1) stably sorting the P
// Gaussians by depth bits, (2) emitting each Gaussian's pairs in that order
// (rect y-major, x-minor, as the reference does), and (3) stably sorting the
// pairs by tile id only.  The result -- sorted order, keys, ranges -- is
// identical, and the K-sized passes drop from 6 to ceil(tile_bits / 8).
//
// Every sort pass is one onesweep kernel (Adinets & Merrill 2022): chunks
// take ascending indices from an atomic counter, rank their keys with
// warp-level match/ballot, and learn their global offsets per digit from a
// decoupled look-back over the preceding chunks (fgs_scan.cuh: windowed,
// bounded; on timeout the kernel records FGS_ERR_TIMEOUT and moves on).
#include "fgs_common.cuh"
#include "fgs_internal.h"
#include "fgs_scan.cuh"

namespace fgs {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;                        // keys per thread, at most
constexpr int kSortItemsMin = 8;                      // keys per thread, at least
constexpr int kSortTile = kSortThreads * kSortItems;  // largest chunk
constexpr int kSortTileMin = kSortThreads * kSortItemsMin;
constexpr int kRadix = 256;
// Exclusive scan of one value per thread over a 256-thread block.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* s_warp /*[8]*/, uint32_t* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    uint32_t wpre = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; w++) {
        const uint32_t c = s_warp[w];
        if (w < warp) wpre += c;
        tot += c;
    }
    __syncthreads();
    if (total) *total = tot;
    return wpre + x - v;
}

// One onesweep pass over `n` 32-bit keys with 32-bit values.
//   vals_in == nullptr: values are the element indices.
//   rec_out != nullptr (last tile pass): also gathers the per-Gaussian render
//   record of each value into sorted position.
//   n_dev != nullptr: the live count is min(n, *n_dev) (the grid covers n).
// Persistent: each CTA takes chunks from the counter until none is left, so a
// grid sized for a bound costs nothing for the chunks that are not live.  Per
// chunk: rank the keys (warp match), publish the digit counts at once, sort the
// chunk locally in shared memory (which needs no global offsets), and only
// then walk back for the global offsets -- the registers that held the keys
// are free by then, so the walk keeps 32 status loads in flight per digit
// (64 registers, 4 CTAs per SM).
__global__ void __launch_bounds__(kSortThreads, 4)
    onesweep_kernel(const uint32_t* __restrict__ keys_in, uint32_t* __restrict__ keys_out,
                    const uint32_t* __restrict__ vals_in, uint32_t* __restrict__ vals_out, uint32_t n, int shift,
                    int nbits, const uint32_t* __restrict__ pass_hist, uint32_t* status, uint32_t* chunk_counter,
                    unsigned* err, const PairRecord* __restrict__ grec, PairRecord* __restrict__ rec_out,
                    const unsigned long long* __restrict__ n_dev, const int2* __restrict__ erow, int gx,
                    unsigned long long wait_ns = kWaitLimitNs, uint32_t skip_chunk = 0xffffffffu)
{
    __shared__ uint32_t s_hist[kSortWarps][kRadix];
    __shared__ uint32_t s_keys[kSortTile];
    __shared__ uint32_t s_vals[kSortTile];
    __shared__ uint32_t s_start[kRadix];
    __shared__ uint32_t s_gbase[kRadix];
    __shared__ uint32_t s_warp[kSortWarps];
    __shared__ uint32_t s_chunk;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (n_dev) n = (uint32_t)min((unsigned long long)n, *n_dev);
    // Keys per thread from the live count: about one chunk per resident CTA, between
    // kSortItemsMin and kSortItems (a small sort gets more, shorter chunks; a large one
    // fewer chunks and a shorter look-back chain).  The same on every CTA.
    const uint32_t per_cta = (n + gridDim.x - 1) / gridDim.x;
    const int items = (int)min((uint32_t)kSortItems,
                               max((uint32_t)kSortItemsMin, (per_cta + kSortThreads - 1) / kSortThreads));
    const uint32_t tile = (uint32_t)items * kSortThreads;
    const uint32_t live = (n + tile - 1) / tile;
    if (blockIdx.x >= live) return;
    const uint32_t dmask = (1u << nbits) - 1u;
    // global start of every digit in this pass (the same for all chunks)
    const uint32_t gh = (uint32_t)tid <= dmask ? __ldg(pass_hist + tid) : 0u;
    const uint32_t gofs = block_excl_scan(gh, s_warp, nullptr);
    const unsigned lt = (1u << lane) - 1u;

    for (;;) {
        if (tid == 0) s_chunk = atomicAdd(chunk_counter, 1u);
#pragma unroll
        for (int w = 0; w < kSortWarps; w++) s_hist[w][tid] = 0;
        __syncthreads();
        const uint32_t chunk = s_chunk;
        if (chunk >= live) break;
        const uint32_t base = chunk * tile;
        const uint32_t count = min(tile, n - base);

        uint32_t key[kSortItems], rank[kSortItems];
#pragma unroll
        for (int i = 0; i < kSortItems; i++) {
            if (i >= items) break;
            const uint32_t pos = warp * (items * 32) + i * 32 + lane;
            const bool valid = pos < count;
            key[i] = valid ? __ldg(keys_in + base + pos) : 0xffffffffu;
            const uint32_t dg = valid ? ((key[i] >> shift) & dmask) : kRadix;
            const unsigned peers = __match_any_sync(0xffffffffu, dg);
            const int leader = __ffs(peers) - 1;
            uint32_t old = 0;
            if (lane == leader && dg < kRadix) {
                old = s_hist[warp][dg];
                s_hist[warp][dg] = old + __popc(peers);
            }
            old = __shfl_sync(0xffffffffu, old, leader);
            rank[i] = old + __popc(peers & lt);
            __syncwarp();
        }
        __syncthreads();
        // per digit (thread d): exclusive prefix over warps, chunk total, published at once
        uint32_t tot = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; w++) {
            const uint32_t c = s_hist[w][tid];
            s_hist[w][tid] = tot;
            tot += c;
        }
        // skip_chunk (a test hook) never publishes: its successors wait until wait_ns runs out
        const bool publish = chunk != skip_chunk;
        if (publish) lookback_publish(status + tid, chunk, kRadix, tot);
        s_start[tid] = block_excl_scan(tot, s_warp, nullptr);
        __syncthreads();
        // local sort of the chunk by digit
#pragma unroll
        for (int i = 0; i < kSortItems; i++) {
            if (i >= items) break;
            const uint32_t pos = warp * (items * 32) + i * 32 + lane;
            if (pos < count) {
                const uint32_t dg = (key[i] >> shift) & dmask;
                const uint32_t lp = s_start[dg] + s_hist[warp][dg] + rank[i];
                s_keys[lp] = key[i];
                s_vals[lp] = vals_in ? __ldg(vals_in + base + pos) : base + pos;
            }
        }
        // global offset of this chunk's digit run
        s_gbase[tid] = gofs + thread_lookback_walk<32>(status + tid, chunk, kRadix, tot, err, wait_ns, publish);
        __syncthreads();
        for (uint32_t p = tid; p < count; p += kSortThreads) {
            const uint32_t k = s_keys[p];
            const uint32_t dg = (k >> shift) & dmask;
            const uint32_t gp = s_gbase[dg] + (p - s_start[dg]);
            const uint32_t v = s_vals[p];
            if (gp >= n) {  // cannot happen with consistent histograms; never write out of bounds
                set_error(err, FGS_ERR_OVERFLOW);
                continue;
            }
            if (keys_out) keys_out[gp] = k;
            vals_out[gp] = v;
            if (rec_out) {
                // The record also carries the pair's emission index: the Gaussian's first
                // pair plus this tile's row-major place in its tile rectangle (the order in
                // which duplicate_kernel emitted them), from the row base and width that
                // duplicate_kernel left per Gaussian.  The backward writes the pair's
                // gradients there, so each Gaussian's pairs are contiguous and are summed
                // in a fixed order.
                PairRecord r = grec[v];
                const int2 er = __ldg(erow + v);
                const uint32_t ty = k / (uint32_t)gx, tx = k - ty * (uint32_t)gx;
                r.c.w = __uint_as_float((uint32_t)er.x + ty * (uint32_t)er.y + tx);
                rec_out[gp] = r;
            }
        }
        __syncthreads();  // shared buffers are reused by the next chunk
    }
}

// Histograms of the 4 depth-key bytes (one read of the keys).
__global__ void depth_hist_kernel(const uint32_t* __restrict__ keys, uint32_t n,
                                  const unsigned long long* __restrict__ n_dev, uint32_t* __restrict__ hist)
{
    __shared__ uint32_t s[4][kRadix];
    n = (uint32_t)min((unsigned long long)n, *n_dev);
    for (int i = threadIdx.x; i < 4 * kRadix; i += blockDim.x) (&s[0][0])[i] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = __ldg(keys + i);
#pragma unroll
        for (int b = 0; b < 4; b++) atomicAdd(&s[b][(k >> (8 * b)) & 255u], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * kRadix; i += blockDim.x) {
        const uint32_t c = (&s[0][0])[i];
        if (c) atomicAdd(hist + i, c);
    }
}

// duplicateWithKeys over the depth-ordered Gaussians, with the prefix sum of
// tiles_touched fused in (decoupled look-back over 256-Gaussian chunks, taken
// by persistent CTAs; the tile histograms leave each CTA once) and
// warp-aggregated pair emission: the pairs of a warp's 32 Gaussians are
// spread evenly over its lanes, so a large splat does not serialise on one
// thread.  Also builds the per-pass tile digit histograms for the tile sort.
__global__ void __launch_bounds__(256)
    duplicate_kernel(const uint32_t* __restrict__ sorted_ids, const uint32_t* __restrict__ tiles,
                     const PairRecord* __restrict__ grec, const int* __restrict__ radii, uint32_t V, int gx,
                     int gy, uint32_t* __restrict__ tile_out, uint32_t* __restrict__ val_out, uint32_t K,
                     uint32_t* status, uint32_t* chunk_counter, uint32_t* __restrict__ tile_hist, int tile_passes,
                     const unsigned long long* __restrict__ V_dev, uint32_t* __restrict__ pair_off,
                     int2* __restrict__ erow, unsigned* err)
{
    __shared__ uint32_t s_hist[4][kRadix];
    __shared__ uint32_t s_warp[8];
    __shared__ uint32_t s_chunk, s_prefix;
    const int tid = threadIdx.x, lane = tid & 31;
    // persistent over chunks of 256 Gaussians (the grid covers a bound on V)
    V = (uint32_t)min((unsigned long long)V, *V_dev);
    const uint32_t live = (V + 255) / 256;
    if (blockIdx.x >= live) return;
    for (int i = tid; i < 4 * kRadix; i += 256) (&s_hist[0][0])[i] = 0;
    for (;;) {
        if (tid == 0) s_chunk = atomicAdd(chunk_counter, 1u);
        __syncthreads();
        const uint32_t chunk = s_chunk;
        if (chunk >= live) break;
        const uint32_t j = chunk * 256 + tid;
        uint32_t id = 0, cnt = 0;
        int x0 = 0, y0 = 0, w = 1;
        if (j < V) {
            id = __ldg(sorted_ids + j);
            cnt = __ldg(tiles + id);
            const float4 a = grec[id].a;
            int x1, y1;
            tile_rect(a.x, a.y, __ldg(radii + id), gx, gy, kTileX, kTileY, x0, y0, x1, y1);
            w = max(1, x1 - x0);
        }
        uint32_t block_total;
        const uint32_t local = block_excl_scan(cnt, s_warp, &block_total);
        if (tid < 32) {
            const uint32_t e = warp_lookback(status, chunk, 1, block_total, err);
            if (tid == 0) s_prefix = e;
        }
        __syncthreads();
        const uint32_t off = s_prefix + local;
        if (cnt) {
            // first emitted pair (by depth rank j: Gaussian j's pairs are
            // [pair_off[j], pair_off[j + 1])), and the emission index of tile
            // (tx, ty) as erow.x + ty * erow.y + tx (unsigned wrap-around)
            pair_off[j] = off;
            erow[id] = make_int2((int)(off - (uint32_t)y0 * (uint32_t)w - (uint32_t)x0), w);
        }
        // warp-local exclusive prefix of cnt
        uint32_t wx = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, wx, o);
            if (lane >= o) wx += y;
        }
        const uint32_t wtotal = __shfl_sync(0xffffffffu, wx, 31);
        wx -= cnt;  // exclusive
        for (uint32_t pb = 0; pb < wtotal; pb += 32) {
            const uint32_t p = pb + lane;
            // owner lane: last lane g with wx[g] <= p (lanes with no pairs never win)
            int lo = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const int probe = lo + step;
                const uint32_t e = __shfl_sync(0xffffffffu, wx, probe);
                if (e <= p) lo = probe;
            }
            const uint32_t owx = __shfl_sync(0xffffffffu, wx, lo);
            const uint32_t ooff = __shfl_sync(0xffffffffu, off, lo);
            const uint32_t oid = __shfl_sync(0xffffffffu, id, lo);
            const int ox0 = __shfl_sync(0xffffffffu, x0, lo);
            const int oy0 = __shfl_sync(0xffffffffu, y0, lo);
            const int ow = __shfl_sync(0xffffffffu, w, lo);
            if (p < wtotal) {
                const uint32_t t = p - owx;
                if (ooff + t >= K) {  // K and tiles_touched come from the same kernel; guard anyway
                    set_error(err, FGS_ERR_OVERFLOW);
                    continue;
                }
                const uint32_t ty = t / (uint32_t)ow, tx = t - ty * (uint32_t)ow;
                const uint32_t tile = (uint32_t)(oy0 + ty) * (uint32_t)gx + (uint32_t)(ox0 + tx);
                tile_out[ooff + t] = tile;
                val_out[ooff + t] = oid;
                for (int b = 0; b < tile_passes; b++) atomicAdd(&s_hist[b][(tile >> (8 * b)) & 255u], 1u);
            }
        }
        __syncthreads();  // s_chunk / s_prefix / s_warp are reused by the next chunk
    }
    for (int i = tid; i < tile_passes * kRadix; i += 256) {
        const uint32_t c = (&s_hist[0][0])[i];
        if (c) atomicAdd(tile_hist + i, c);
    }
}

// identifyTileRanges (rasterizer_impl.cu:172-194) over the sorted tile ids.
__global__ void ranges_kernel(const uint32_t* __restrict__ tile, uint32_t K, uint2* __restrict__ ranges,
                              const unsigned long long* __restrict__ n_dev)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (n_dev) K = (uint32_t)min((unsigned long long)K, *n_dev);
    if (i >= K) return;
    const uint32_t t = tile[i];
    if (i == 0 || tile[i - 1] != t) ranges[t].x = i;
    if (i == K - 1 || tile[i + 1] != t) ranges[t].y = i + 1;
}

inline uint32_t chunks_of(long long n, int tile) { return (uint32_t)((n + tile - 1) / tile); }

// Test hook of the first depth-sort pass (fgs_debug_lookback_fault): the chunk
// that never publishes its counts and the wait limit of that pass.
unsigned long long g_fault_wait_ns = kWaitLimitNs;
uint32_t g_fault_skip_chunk = 0xffffffffu;

}  // namespace

void set_lookback_fault(uint32_t skip_chunk, unsigned long long wait_ns)
{
    g_fault_skip_chunk = skip_chunk;
    g_fault_wait_ns = wait_ns ? wait_ns : kWaitLimitNs;
}

int sort_chunk_size() { return kSortTileMin; }  // the smallest chunk: sizes the status words

void launch_depth_sort(const GeomState& g, int P, cudaStream_t s)
{
    // the V visible Gaussians (count on the device, bound P): keys depth_key[0..V), ids sort_ids_b[0..V)
    if (P <= 0) return;
    const uint32_t n = (uint32_t)P;
    const unsigned long long* V = g.total + 1;
    const uint32_t nch = chunks_of(n, kSortTileMin);
    const uint32_t hb0 = (n + 1023) / 1024;
    const int hb = (int)(hb0 < 1184u ? hb0 : 1184u);
    depth_hist_kernel<<<hb, 256, 0, s>>>(g.depth_key, n, V, g.hist);
    const uint32_t grid = min(nch, resident_ctas(onesweep_kernel, kSortThreads));
    note_launches(5);
    // ping-pong: depth_key -> sort_keys_b -> depth_key -> sort_keys_b ; ids b -> a -> b -> a -> b
    const uint32_t* kin[4] = {g.depth_key, g.sort_keys_b, g.depth_key, g.sort_keys_b};
    uint32_t* kout[4] = {g.sort_keys_b, g.depth_key, g.sort_keys_b, nullptr};
    const uint32_t* vin[4] = {g.sort_ids_b, g.sort_ids_a, g.sort_ids_b, g.sort_ids_a};
    uint32_t* vout[4] = {g.sort_ids_a, g.sort_ids_b, g.sort_ids_a, g.sort_ids_b};
    for (int pass = 0; pass < 4; pass++) {
        onesweep_kernel<<<grid, kSortThreads, 0, s>>>(kin[pass], kout[pass], vin[pass], vout[pass], n, 8 * pass, 8,
                                                     g.hist + pass * kRadix, g.status + (size_t)pass * nch * kRadix,
                                                     g.counters + pass, g.err, nullptr, nullptr, V, nullptr, 1,
                                                     pass ? kWaitLimitNs : g_fault_wait_ns,
                                                     pass ? 0xffffffffu : g_fault_skip_chunk);
    }
}

void launch_duplicate(const GeomState& g, const BinState& b, uint32_t V, uint32_t K, int W, int H, int tile_bits,
                      cudaStream_t s)
{
    if (V == 0) return;
    const int gx = (W + kTileX - 1) / kTileX, gy = (H + kTileY - 1) / kTileY;
    const int passes = (tile_bits + 7) / 8;
    // The tile sort ping-pongs between the a/b buffers and must end in b:
    // with an odd number of passes it starts from a, with an even one from b.
    uint32_t* tout = (passes & 1) ? b.tile_a : b.tile_b;
    uint32_t* vout = (passes & 1) ? b.val_a : b.val_b;
    const uint32_t grid = min(chunks_of(V, 256), resident_ctas(duplicate_kernel, 256));
    duplicate_kernel<<<grid, 256, 0, s>>>(g.sort_ids_b, g.tiles, g.grec, g.radii, V, gx, gy, tout,
                                                       vout, K, b.scan_status, g.counters + 8, g.hist + 4 * kRadix,
                                                       passes, g.total + 1, g.pair_off, g.erow, g.err);
    note_launches(1);
}

void launch_tile_sort(const GeomState& g, const BinState& b, long long K, int tile_bits, int W, int H, cudaStream_t s,
                      const unsigned long long* n_dev)
{
    if (K <= 0) return;
    const int gx = (W + kTileX - 1) / kTileX;  // tile ids are row-major over gx columns
    (void)H;
    const uint32_t n = (uint32_t)K;
    const uint32_t nch = chunks_of(n, kSortTileMin);
    const uint32_t grid = min(nch, resident_ctas(onesweep_kernel, kSortThreads));
    const int passes = (tile_bits + 7) / 8;
    const uint32_t* ki = (passes & 1) ? b.tile_a : b.tile_b;
    const uint32_t* vi = (passes & 1) ? b.val_a : b.val_b;
    for (int pass = 0; pass < passes; pass++) {
        const bool last = pass == passes - 1;
        const int nbits = min(8, tile_bits - 8 * pass);
        uint32_t* ko = (ki == b.tile_a) ? b.tile_b : b.tile_a;
        uint32_t* vo = (vi == b.val_a) ? b.val_b : b.val_a;
        onesweep_kernel<<<grid, kSortThreads, 0, s>>>(ki, ko, vi, vo, n, 8 * pass, nbits, g.hist + (4 + pass) * kRadix,
                                                     b.status + (size_t)pass * nch * kRadix, g.counters + 4 + pass,
                                                     g.err, last ? g.grec : nullptr, last ? b.rec : nullptr, n_dev,
                                                     g.erow, gx);
        ki = ko;
        vi = vo;
    }
    note_launches(passes);
}

void launch_ranges(const BinState& b, const ImageState& im, long long K, int num_tiles, cudaStream_t s,
                   const unsigned long long* n_dev)
{
    cudaMemsetAsync(im.ranges, 0, sizeof(uint2) * (size_t)num_tiles, s);
    if (K <= 0) return;
    ranges_kernel<<<chunks_of(K, 256), 256, 0, s>>>(b.tile_b, (uint32_t)K, im.ranges, n_dev);
    note_launches(1);
}

}  // namespace fgs
