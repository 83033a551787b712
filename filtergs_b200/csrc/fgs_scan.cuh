// Decoupled look-back primitives shared by the single-pass scans (pair
// emission, onesweep radix passes, ordered compaction).
//
// Each chunk of a scan owns a 32-bit status word: 2 flag bits (aggregate
// published / inclusive prefix published) and a 30-bit value.  A chunk
// publishes its aggregate as soon as it is known, walks back over its
// predecessors summing aggregates until it meets an inclusive prefix, then
// publishes its own inclusive prefix.  Chunk ids come from an atomic
// counter, so every predecessor of a running chunk is already running and
// the walk always ends; each wait is still bounded (kWaitLimitNs, or a
// caller's shorter limit) and a timeout is recorded as FGS_ERR_TIMEOUT
// instead of spinning forever.
//
// The walk is the scan's critical path: with all chunks resident at once a
// chunk may find dozens of predecessors that have only published their
// aggregate.  Both walks here keep many status loads in flight per round
// trip -- 32 predecessors per warp-wide step in warp_lookback, kWindow per
// thread in thread_lookback_walk -- instead of one.
#pragma once

#include "fgs_common.cuh"

namespace fgs {

constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kValMask = (1u << 30) - 1;

__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v)
{
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint32_t sat_value(unsigned long long v, bool& saturated)
{
    saturated = v > kValMask;
    return saturated ? kValMask : (uint32_t)v;
}

// Warp-cooperative look-back: all 32 lanes of one warp call it with the same
// arguments; status words are `stride` apart.  Lane l polls predecessor
// j - l, so one round trip covers 32 predecessors.  Returns the exclusive
// prefix on every lane.  A sum past the 30-bit value range saturates and
// records FGS_ERR_OVERFLOW.
__device__ __forceinline__ uint32_t warp_lookback(uint32_t* status, uint32_t chunk, int stride, uint32_t agg,
                                                  unsigned* err)
{
    const int lane = threadIdx.x & 31;
    uint32_t* mine = status + (size_t)chunk * stride;
    if (chunk == 0) {
        if (lane == 0) st_relaxed(mine, kFlagPrefix | agg);
        return 0;
    }
    if (lane == 0) st_relaxed(mine, kFlagAgg | agg);
    unsigned long long excl = 0;
    long long j = (long long)chunk - 1;
    WaitBound wb;
    while (true) {
        const long long q = j - lane;
        const uint32_t s = q >= 0 ? ld_relaxed(status + (size_t)q * stride) : kFlagPrefix;
        const uint32_t flag = s & ~kValMask;
        const unsigned pref = __ballot_sync(0xffffffffu, flag == kFlagPrefix);
        const unsigned empty = __ballot_sync(0xffffffffu, flag == 0);
        const int fp = pref ? __ffs(pref) - 1 : 31;           // nearest inclusive prefix (or the window)
        const unsigned upto = fp == 31 ? 0xffffffffu : ((2u << fp) - 1u);
        int take = fp + 1;                                      // lanes [0, take) are summed
        if (empty & upto) take = __ffs(empty & upto) - 1;       // stop before an unpublished word
        uint32_t v = lane < take ? (s & kValMask) : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        excl += v;
        if (take == fp + 1 && pref) break;                      // reached an inclusive prefix
        // take is warp-uniform; lane 0's clock decides for the whole warp, so every
        // lane leaves the loop (and its ballots) on the same iteration
        if (take == 0 && __shfl_sync(0xffffffffu, (int)wb.expired(kWaitLimitNs), 0)) {
            if (lane == 0) set_error(err, FGS_ERR_TIMEOUT);
            break;
        }
        j -= take;
    }
    bool sat = false;
    const uint32_t incl = sat_value(excl + agg, sat);
    if (lane == 0) {
        st_relaxed(mine, kFlagPrefix | incl);
        if (sat) set_error(err, FGS_ERR_OVERFLOW);
    }
    return excl > kValMask ? kValMask : (uint32_t)excl;
}

// Per-thread look-back (one thread per independent scan, e.g. one radix digit
// per thread); status words `stride` apart.  Split in two so a caller can
// publish its aggregate as early as possible and walk later:
// lookback_publish() first, then thread_lookback_walk<W>(), which polls W
// predecessors per round trip, returns the exclusive prefix and publishes
// the inclusive one (unless `publish` is false: a test hook that leaves the
// chunk's successors waiting until their limit runs out).
__device__ __forceinline__ void lookback_publish(uint32_t* status, uint32_t chunk, int stride, uint32_t agg)
{
    st_relaxed(status + (size_t)chunk * stride, (chunk == 0 ? kFlagPrefix : kFlagAgg) | agg);
}

template <int kWindow>
__device__ __forceinline__ uint32_t thread_lookback_walk(uint32_t* status, uint32_t chunk, int stride, uint32_t agg,
                                                         unsigned* err,
                                                         unsigned long long limit_ns = kWaitLimitNs,
                                                         bool publish = true)
{
    if (chunk == 0) return 0;
    unsigned long long excl = 0;
    long long j = (long long)chunk - 1;
    WaitBound wb;
    while (true) {
        uint32_t s[kWindow];
#pragma unroll
        for (int i = 0; i < kWindow; i++)
            s[i] = (j - i >= 0) ? ld_relaxed(status + (size_t)(j - i) * stride) : kFlagPrefix;
        int take = 0;
        bool done = false;
#pragma unroll
        for (int i = 0; i < kWindow; i++) {
            const uint32_t flag = s[i] & ~kValMask;
            if (!done && take == i && flag != 0) {
                excl += s[i] & kValMask;
                take = i + 1;
                done = flag == kFlagPrefix;
            }
        }
        if (done) break;
        if (take == 0 && wb.expired(limit_ns)) {
            set_error(err, FGS_ERR_TIMEOUT);
            break;
        }
        j -= take;
    }
    bool sat = false;
    const uint32_t incl = sat_value(excl + agg, sat);
    if (publish) st_relaxed(status + (size_t)chunk * stride, kFlagPrefix | incl);
    if (sat) set_error(err, FGS_ERR_OVERFLOW);
    return excl > kValMask ? kValMask : (uint32_t)excl;
}

}  // namespace fgs
