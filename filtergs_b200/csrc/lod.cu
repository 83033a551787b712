// LoD selection and the per-view glue in front of the rasterizer.
//
//   gather_attributes   FilterGS/cuda/gather_attributes_kernel.cu:6-66 (row gather by int64 index)
//   compact_mask        torch.nonzero(mask) of FilterGS/filtergs.py:64 as one ordered
//                       stream compaction (decoupled look-back), count left on the device
//   gather_activate     FilterGS get_all (filtergs.py:98-134): gather + LoG/model/activation.py:36-43
//                       (exp scale, sigmoid opacity, normalised quaternion, SH2RGB(dc) + eval_sh_wobase)
//   log_cut             LoG/model/tensor_tree.py:133-187 (TensorTree.traverse) as a level-synchronous
//                       frontier on the device: per level one kernel reads the frontier size from
//                       device memory, so the whole traversal is launched without host syncs
//   cull                the redundancy culling of the cut (drop radius < min_px or
//                       sigmoid(opacity) < 1/255), order preserving
#include "fgs_common.cuh"
#include "fgs_internal.h"
#include "fgs_scan.cuh"

namespace fgs {

namespace {

// Ordered exclusive prefix of a per-thread count over a 256-thread chunk plus
// a decoupled look-back over earlier chunks.  Returns the global exclusive
// offset of this thread's items; *chunk_total receives the chunk's sum.
__device__ __forceinline__ uint32_t chunk_offset(uint32_t cnt, uint32_t chunk, uint32_t* status, unsigned* err)
{
    __shared__ uint32_t s_warp[8];
    __shared__ uint32_t s_prefix;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    uint32_t wpre = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < 8; w++) {
        const uint32_t c = s_warp[w];
        if (w < warp) wpre += c;
        tot += c;
    }
    if (threadIdx.x < 32) {
        const uint32_t excl = warp_lookback(status, chunk, 1, tot, err);
        if (threadIdx.x == 0) s_prefix = excl;
    }
    __syncthreads();
    const uint32_t r = s_prefix + wpre + x - cnt;
    __syncthreads();
    return r;
}

// Ordered compaction, kCompactItems items per thread (a chunk of 4096 per CTA):
// a thread's items are consecutive, so its survivors are written as one run at
// its exclusive offset, and one look-back per 4096 items orders the chunks.
constexpr int kCompactItems = 16;
constexpr uint32_t kCompactChunk = 256u * kCompactItems;

// Writes the indices base + k of the set bits k of `bits` at out[off...] in order.
__device__ __forceinline__ void write_run(uint32_t bits, uint32_t base, uint32_t off, int64_t* __restrict__ out)
{
    while (bits) {
        const int k = __ffs(bits) - 1;
        bits &= bits - 1;
        out[off++] = (int64_t)(base + (uint32_t)k);
    }
}

// mask[n] (bytes) -> ordered indices (int64) of the nonzero entries; count to *count.
__global__ void __launch_bounds__(256) compact_kernel(const uint8_t* __restrict__ mask, uint32_t n, int vec,
                                                      int64_t* __restrict__ out, unsigned long long* count,
                                                      uint32_t* status, uint32_t* counter, unsigned* err)
{
    __shared__ uint32_t s_chunk;
    if (threadIdx.x == 0) s_chunk = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t chunk = s_chunk;
    const uint32_t base = chunk * kCompactChunk + threadIdx.x * kCompactItems;
    uint32_t bits = 0;
    if (vec && base + kCompactItems <= n) {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(mask + base));
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int q = 0; q < 4; q++)
#pragma unroll
            for (int b = 0; b < 4; b++)
                if ((w[q] >> (8 * b)) & 0xffu) bits |= 1u << (4 * q + b);
    } else {
        for (int k = 0; k < kCompactItems; k++)
            if (base + k < n && mask[base + k]) bits |= 1u << k;
    }
    const uint32_t cnt = __popc(bits);
    const uint32_t off = chunk_offset(cnt, chunk, status, err);
    write_run(bits, base, off, out);
    if (chunk == gridDim.x - 1 && threadIdx.x == 255) *count = off + cnt;  // the last chunk knows the total
}

__global__ void gather_kernel(const int64_t* __restrict__ index, long long N, const float* __restrict__ xyz,
                              const float* __restrict__ scaling, const float* __restrict__ rotation,
                              const float* __restrict__ opacity, const float* __restrict__ colors,
                              const float* __restrict__ shs, int sh_floats, float* __restrict__ o_xyz,
                              float* __restrict__ o_scaling, float* __restrict__ o_rotation,
                              float* __restrict__ o_opacity, float* __restrict__ o_colors, float* __restrict__ o_shs)
{
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const long long s = index[n];
#pragma unroll
    for (int k = 0; k < 3; k++) o_xyz[3 * n + k] = xyz[3 * s + k];
#pragma unroll
    for (int k = 0; k < 3; k++) o_scaling[3 * n + k] = scaling[3 * s + k];
    *reinterpret_cast<float4*>(o_rotation + 4 * n) = *reinterpret_cast<const float4*>(rotation + 4 * s);
    o_opacity[n] = opacity[s];
#pragma unroll
    for (int k = 0; k < 3; k++) o_colors[3 * n + k] = colors[3 * s + k];
    if (shs && o_shs)
        for (int f = 0; f < sh_floats; f++) o_shs[n * sh_floats + f] = shs[s * sh_floats + f];
}

// eval_sh_wobase (LoG/model/sh_utils.py:31-68) for one channel of the rest
// coefficients rest[k*3 + c], k = 0 .. (deg+1)^2 - 2.  The reference evaluates it
// as a chain of torch element-wise ops, each rounded on its own (a Python scalar
// becomes a float operand): the same ops in the same order here, with
// round-to-nearest intrinsics so that no multiply-add is fused.
__device__ __forceinline__ float sh_wobase(int deg, const float* rest, int c, float x, float y, float z)
{
    auto R = [&](int k) { return rest[k * 3 + c]; };
    auto M = [](float a, float b) { return __fmul_rn(a, b); };
    auto P = [](float a, float b) { return __fadd_rn(a, b); };
    auto D = [](float a, float b) { return __fsub_rn(a, b); };
    // - C1 * y * sh0 + C1 * z * sh1 - C1 * x * sh2
    float r = D(P(M(M(-kSH_C1, y), R(0)), M(M(kSH_C1, z), R(1))), M(M(kSH_C1, x), R(2)));
    if (deg > 1) {
        const float xx = M(x, x), yy = M(y, y), zz = M(z, z), xy = M(x, y), yz = M(y, z), xz = M(x, z);
        r = P(r, M(M(kSH_C2_0, xy), R(3)));
        r = P(r, M(M(kSH_C2_1, yz), R(4)));
        r = P(r, M(M(kSH_C2_2, D(D(M(2.0f, zz), xx), yy)), R(5)));
        r = P(r, M(M(kSH_C2_3, xz), R(6)));
        r = P(r, M(M(kSH_C2_4, D(xx, yy)), R(7)));
        if (deg > 2) {
            r = P(r, M(M(M(kSH_C3_0, y), D(M(3.0f, xx), yy)), R(8)));
            r = P(r, M(M(M(kSH_C3_1, xy), z), R(9)));
            r = P(r, M(M(M(kSH_C3_2, y), D(D(M(4.0f, zz), xx), yy)), R(10)));
            r = P(r, M(M(M(kSH_C3_3, z), D(D(M(2.0f, zz), M(3.0f, xx)), M(3.0f, yy))), R(11)));
            r = P(r, M(M(M(kSH_C3_4, x), D(D(M(4.0f, zz), xx), yy)), R(12)));
            r = P(r, M(M(M(kSH_C3_5, z), D(xx, yy)), R(13)));
            r = P(r, M(M(M(kSH_C3_6, x), D(xx, M(3.0f, yy))), R(14)));
        }
    }
    return r;
}

__global__ void gather_activate_kernel(const int64_t* __restrict__ index, const unsigned long long* __restrict__ count,
                                       long long N_cap, const float* __restrict__ xyz,
                                       const float* __restrict__ log_scale, const float* __restrict__ rot,
                                       const float* __restrict__ opac_raw, const float* __restrict__ dc,
                                       const float* __restrict__ rest, int deg, int rest_coeffs,
                                       const float* __restrict__ campos, float* __restrict__ o_xyz,
                                       float* __restrict__ o_scale, float* __restrict__ o_rot,
                                       float* __restrict__ o_opac, float* __restrict__ o_rgb)
{
    const long long N = count ? (long long)min((unsigned long long)N_cap, *count) : N_cap;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < N;
         n += (long long)gridDim.x * blockDim.x) {
        const long long s = index[n];
        const float px = xyz[3 * s], py = xyz[3 * s + 1], pz = xyz[3 * s + 2];
        o_xyz[3 * n] = px; o_xyz[3 * n + 1] = py; o_xyz[3 * n + 2] = pz;
#pragma unroll
        for (int k = 0; k < 3; k++) o_scale[3 * n + k] = expf(log_scale[3 * s + k]);
        // torch.nn.functional.normalize: x / max(|x|, 1e-12), where torch's norm over the
        // last dim of 4 adds the rounded squares as (x0^2 + x2^2) + (x1^2 + x3^2) (and
        // over 3 as (x0^2 + x2^2) + x1^2), matched bit for bit against torch on the GPU
        const float4 q = *reinterpret_cast<const float4*>(rot + 4 * s);
        const float q2 = __fadd_rn(__fadd_rn(__fmul_rn(q.x, q.x), __fmul_rn(q.z, q.z)),
                                   __fadd_rn(__fmul_rn(q.y, q.y), __fmul_rn(q.w, q.w)));
        const float nr = fmaxf(__fsqrt_rn(q2), 1e-12f);
        *reinterpret_cast<float4*>(o_rot + 4 * n) =
            make_float4(__fdiv_rn(q.x, nr), __fdiv_rn(q.y, nr), __fdiv_rn(q.z, nr), __fdiv_rn(q.w, nr));
        o_opac[n] = __fdiv_rn(1.0f, __fadd_rn(1.0f, expf(-opac_raw[s])));
        // dir_pp = xyz - camera_center; dir_pp / torch.norm(dir_pp, dim=-1) (activation.py:36-43)
        float dx = __fsub_rn(px, campos[0]), dy = __fsub_rn(py, campos[1]), dz = __fsub_rn(pz, campos[2]);
        const float dl = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dz, dz)), __fmul_rn(dy, dy)));
        dx = __fdiv_rn(dx, dl); dy = __fdiv_rn(dy, dl); dz = __fdiv_rn(dz, dl);
        const float* rs = rest ? rest + (size_t)s * rest_coeffs * 3 : nullptr;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            // SH2RGB (sh_utils.py:78): two torch ops, then the add of activation.py:40
            float col = __fadd_rn(__fmul_rn(dc[3 * s + c], kSH_C0), 0.5f);
            if (deg > 0 && rs) col = __fadd_rn(col, sh_wobase(deg, rs, c, dx, dy, dz));
            o_rgb[3 * n + c] = col;
        }
    }
}

// One LoG traversal level.  frontier[0..*fsize) are expanded nodes; their
// children (frontier-major, child-slot-minor) are either kept (appended to
// out at *out_count) or expanded (written to next[] in order).  Chunks of 4096
// items (16 consecutive per thread) come from an atomic counter; two look-backs
// give ordered positions.
__global__ void __launch_bounds__(256)
    log_level_kernel(const int32_t* __restrict__ frontier, const uint32_t* __restrict__ fsize,
                     const int32_t* __restrict__ node_index, const int32_t* __restrict__ tree, int max_child,
                     const float* __restrict__ radius, float min_res, int32_t* __restrict__ out,
                     const uint32_t* __restrict__ count_in, uint32_t* __restrict__ count_out,
                     int32_t* __restrict__ next, uint32_t* __restrict__ next_size, uint32_t* status_keep,
                     uint32_t* status_next, uint32_t* counter, uint32_t max_items, unsigned* err)
{
    // Sizes of this level are read from slots the previous level wrote and
    // results go to the other slots, so no block reads a value this launch changes.
    __shared__ uint32_t s_chunk;
    __shared__ uint32_t s_base;
    const uint32_t items = min(*fsize * (uint32_t)max_child, max_items);
    const uint32_t nchunks = (items + kCompactChunk - 1) / kCompactChunk;
    if (threadIdx.x == 0) s_base = *count_in;
    if (nchunks == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            *count_out = *count_in;
            *next_size = 0;
        }
        return;
    }
    for (;;) {
        if (threadIdx.x == 0) s_chunk = atomicAdd(counter, 1u);
        __syncthreads();
        const uint32_t chunk = s_chunk;
        if (chunk >= nchunks) break;
        const uint32_t base = chunk * kCompactChunk + threadIdx.x * kCompactItems;
        int32_t ch[kCompactItems];
#pragma unroll
        for (int k = 0; k < kCompactItems; k++) {
            const uint32_t it = base + k;
            ch[k] = -1;
            if (it < items) {
                const int32_t ni = __ldg(node_index + __ldg(frontier + it / max_child));
                if (ni >= 0) ch[k] = __ldg(tree + (size_t)ni * max_child + it % max_child);
            }
        }
        uint32_t kbits = 0, xbits = 0;
#pragma unroll
        for (int k = 0; k < kCompactItems; k++) {
            if (ch[k] < 0) continue;
            const bool keep = __ldg(radius + ch[k]) < min_res || __ldg(node_index + ch[k]) == -1;
            if (keep) kbits |= 1u << k;
            else xbits |= 1u << k;
        }
        const uint32_t kc = __popc(kbits), xc = __popc(xbits);
        const uint32_t ok = chunk_offset(kc, chunk, status_keep, err);
        const uint32_t ox = chunk_offset(xc, chunk, status_next, err);
        uint32_t o = s_base + ok, q = ox;
#pragma unroll
        for (int k = 0; k < kCompactItems; k++) {
            if ((kbits >> k) & 1u) out[o++] = ch[k];
            if ((xbits >> k) & 1u) next[q++] = ch[k];
        }
        if (chunk == nchunks - 1 && threadIdx.x == 255) {
            *next_size = ox + xc;
            *count_out = s_base + ok + kc;
        }
        __syncthreads();
    }
}

// roots -> kept roots appended to out, expanded roots to the first frontier.
__global__ void __launch_bounds__(256)
    log_roots_kernel(const int32_t* __restrict__ roots, uint32_t nroots, const int32_t* __restrict__ node_index,
                     const float* __restrict__ radius, float min_res, int32_t* __restrict__ out,
                     uint32_t* __restrict__ out_count, int32_t* __restrict__ next, uint32_t* __restrict__ next_size,
                     uint32_t* status_keep, uint32_t* status_next, uint32_t* counter, unsigned* err)
{
    __shared__ uint32_t s_chunk;
    if (threadIdx.x == 0) s_chunk = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t chunk = s_chunk;
    const uint32_t i = chunk * 256 + threadIdx.x;
    uint32_t k = 0, x = 0;
    int32_t id = -1;
    if (i < nroots) {
        id = roots[i];
        const bool keep = radius[id] < min_res || node_index[id] == -1;
        k = keep;
        x = !keep;
    }
    const uint32_t ok = chunk_offset(k, chunk, status_keep, err);
    const uint32_t ox = chunk_offset(x, chunk, status_next, err);
    if (k) out[ok] = id;
    if (x) next[ox] = id;
    if (chunk == gridDim.x - 1 && threadIdx.x == 255) {
        *out_count = ok + k;
        *next_size = ox + x;
    }
}

// Order-preserving filter of a node list: keep radius >= min_px and sigmoid(opacity) >= 1/255.
// Chunks of 4096 ids; CTAs past the live count leave at once.
__global__ void __launch_bounds__(256)
    cull_kernel(const int32_t* __restrict__ in, const uint32_t* __restrict__ n_in, uint32_t cap,
                const float* __restrict__ radius, const float* __restrict__ opac_raw, float min_px,
                int64_t* __restrict__ out, unsigned long long* __restrict__ n_out, uint32_t* status, uint32_t* counter,
                unsigned* err)
{
    __shared__ uint32_t s_chunk;
    const uint32_t n = min(*n_in, cap);
    const uint32_t nchunks = (n + kCompactChunk - 1) / kCompactChunk;
    if (threadIdx.x == 0) s_chunk = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t chunk = s_chunk;
    if (chunk >= nchunks) {
        if (chunk == 0 && threadIdx.x == 0) *n_out = 0;  // n == 0
        return;
    }
    const uint32_t base = chunk * kCompactChunk + threadIdx.x * kCompactItems;
    int32_t id[kCompactItems];
    uint32_t bits = 0;
#pragma unroll
    for (int k = 0; k < kCompactItems; k++) id[k] = base + k < n ? __ldg(in + base + k) : -1;
#pragma unroll
    for (int k = 0; k < kCompactItems; k++) {
        if (id[k] < 0) continue;
        const float o = 1.0f / (1.0f + expf(-__ldg(opac_raw + id[k])));
        if (__ldg(radius + id[k]) >= min_px && o >= 1.0f / 255.0f) bits |= 1u << k;
    }
    const uint32_t cnt = __popc(bits);
    const uint32_t off = chunk_offset(cnt, chunk, status, err);
    uint32_t o = off;
    while (bits) {
        const int k = __ffs(bits) - 1;
        bits &= bits - 1;
        out[o++] = (int64_t)id[k];
    }
    if (chunk == nchunks - 1 && threadIdx.x == 255) *n_out = off + cnt;
}

// v2 3-sigma radius on raw parameters: exp(log scale) and normalised quaternion in-kernel
// (the LoG radius of LoG/model/level_of_gaussian.py:66-88 without the torch activations).
__global__ void radius_raw_kernel(int P, const float* __restrict__ means, const float* __restrict__ lscales,
                                  const float* __restrict__ rots, const float* __restrict__ view,
                                  const float* __restrict__ proj, float fx, float fy, float tanx, float tany,
                                  float* __restrict__ radius)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= P) return;
    radius[idx] = 0;
    const float3 p_orig = {means[3 * idx], means[3 * idx + 1], means[3 * idx + 2]};
    const float4 p_hom = xform_point4x4(p_orig, proj);
    const float p_w = 1.0f / (p_hom.w + 0.0000001f);
    const float3 p_proj = {p_hom.x * p_w, p_hom.y * p_w, p_hom.z * p_w};
    if (p_proj.x < -1.3 || p_proj.x > 1.3 || p_proj.y < -1.3 || p_proj.y > 1.3) return;
    float4 q = {rots[4 * idx], rots[4 * idx + 1], rots[4 * idx + 2], rots[4 * idx + 3]};
    const float nr = fmaxf(sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w), 1e-12f);
    q = {q.x / nr, q.y / nr, q.z / nr, q.w / nr};
    float cov3D[6];
    cov3d_from_scale_rot(expf(lscales[3 * idx]), expf(lscales[3 * idx + 1]), expf(lscales[3 * idx + 2]), 1.f, q,
                         cov3D);
    float3 cov = ewa_cov2d(p_orig, fx, fy, tanx, tany, cov3D, view);
    cov.x = dilate_max(cov.x);
    cov.z = dilate_max(cov.z);
    const float det = (cov.x * cov.z - cov.y * cov.y);
    if (det == 0.0f) return;
    const float mid = 0.5f * (cov.x + cov.z);
    const float lambda1 = mid + sqrtf(fmaxf(0.1f, mid * mid - det));
    const float lambda2 = mid - sqrtf(fmaxf(0.1f, mid * mid - det));
    radius[idx] = 3.f * sqrtf(fmaxf(lambda1, lambda2));
}

// rebuild_ancestor_path (apps/ancestor.py:21-73) without its level loop.  The
// reference visits depths 1..max in order and, for each node i at depth d with
// a parent p >= 0, copies row(p) as it stands at that moment and sets column
// d-1 to p (a node with p < 0 keeps a row of -1).  row(p) is final when
// 1 <= depth(p) < d, and still all -1 otherwise (not yet visited, or visited in
// the same level, whose gather precedes its scatter).  So row(i) is the chain
// i -> p -> ... followed while depths strictly decrease and stay >= 1, each
// step writing its own column: one thread per node walks it (at most L steps;
// the -1 fill is a memset).  The reference raises on a parent id >= P and on a
// column d-1 >= L; both are reported through err.
__global__ void __launch_bounds__(256) ancestor_path_kernel(int P, const int32_t* __restrict__ parent,
                                                            const int32_t* __restrict__ depth, int L,
                                                            int32_t* __restrict__ out, unsigned* err)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P; i += gridDim.x * blockDim.x) {
        int cur = i, dc = __ldg(depth + i);
        int32_t* row = out + (size_t)i * L;
        while (dc >= 1) {
            const int p = __ldg(parent + cur);
            if (p < 0) break;  // orphan: its row is all -1
            if (p >= P || dc - 1 >= L) {
                set_error(err, FGS_ERR_ARG);
                break;
            }
            row[dc - 1] = p;
            const int dp = __ldg(depth + p);
            if (dp >= dc) break;  // the parent's row is still -1 when this level is visited
            cur = p;
            dc = dp;
        }
    }
}

}  // namespace

// ---------------------------------------------------------------- launchers

void launch_compact(const uint8_t* mask, uint32_t n, int64_t* out, unsigned long long* count, uint32_t* scratch,
                    unsigned* err, cudaStream_t s)
{
    // scratch: [1 counter][one status word per chunk], zeroed here
    const uint32_t nch = (n + kCompactChunk - 1) / kCompactChunk;
    cudaMemsetAsync(scratch, 0, sizeof(uint32_t) * (1 + nch), s);
    if (n == 0) {
        cudaMemsetAsync(count, 0, sizeof(unsigned long long), s);
        return;
    }
    const int vec = (reinterpret_cast<uintptr_t>(mask) & 15u) == 0;
    compact_kernel<<<nch, 256, 0, s>>>(mask, n, vec, out, count, scratch + 1, scratch, err);
    note_launches(1);
}

void launch_gather(const int64_t* index, long long N, const float* xyz, const float* scaling, const float* rotation,
                   const float* opacity, const float* colors, const float* shs, int sh_floats, float* o_xyz,
                   float* o_scaling, float* o_rotation, float* o_opacity, float* o_colors, float* o_shs,
                   cudaStream_t s)
{
    if (N <= 0) return;
    gather_kernel<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(index, N, xyz, scaling, rotation, opacity, colors, shs,
                                                              sh_floats, o_xyz, o_scaling, o_rotation, o_opacity,
                                                              o_colors, o_shs);
    note_launches(1);
}

namespace {
// FilterGS/filtergs.py:159-172: a gathered, activated row is rendered only when xyz,
// scaling, rotation, opacity and colour are all finite, the smallest scale is > 0 and
// the opacity is > 0.  Writes keep[n] (1 = render) and counts the rows dropped.
__global__ void rows_valid_kernel(long long N, const float* __restrict__ xyz, const float* __restrict__ sc,
                                  const float* __restrict__ rot, const float* __restrict__ opac,
                                  const float* __restrict__ col, uint8_t* __restrict__ keep,
                                  unsigned long long* __restrict__ dropped)
{
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += (long long)gridDim.x * blockDim.x) {
        bool ok = isfinite(opac[n]) && opac[n] > 0.f;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            ok = ok && isfinite(xyz[3 * n + k]) && isfinite(col[3 * n + k]) && isfinite(sc[3 * n + k]);
        }
        ok = ok && fminf(fminf(sc[3 * n], sc[3 * n + 1]), sc[3 * n + 2]) > 0.f;
#pragma unroll
        for (int k = 0; k < 4; k++) ok = ok && isfinite(rot[4 * n + k]);
        keep[n] = ok ? 1 : 0;
        if (!ok) atomicAdd(dropped, 1ull);
    }
}
}  // namespace

void launch_gather_activate(const int64_t* index, const unsigned long long* count, long long N_cap, const float* xyz,
                            const float* log_scale, const float* rot, const float* opac_raw, const float* dc,
                            const float* rest, int deg, int rest_coeffs, const float* campos, float* o_xyz,
                            float* o_scale, float* o_rot, float* o_opac, float* o_rgb, cudaStream_t s)
{
    if (N_cap <= 0) return;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long want = (N_cap + 255) / 256;
    const int blocks = (int)(want < sms * 8 ? want : sms * 8);
    gather_activate_kernel<<<blocks, 256, 0, s>>>(index, count, N_cap, xyz, log_scale, rot, opac_raw, dc, rest, deg,
                                                  rest_coeffs, campos, o_xyz, o_scale, o_rot, o_opac, o_rgb);
    note_launches(1);
}

void launch_radius_raw(int P, const float* means, const float* lscales, const float* rots, const float* view,
                       const float* proj, float fx, float fy, float tanx, float tany, float* radius, cudaStream_t s)
{
    if (P <= 0) return;
    radius_raw_kernel<<<(P + 255) / 256, 256, 0, s>>>(P, means, lscales, rots, view, proj, fx, fy, tanx, tany,
                                                      radius);
    note_launches(1);
}

// workspace layout (uint32 words): [0,1] output-count slots, [2,3] frontier-size slots,
// [8 .. 8+levels+2) chunk counters, then 2 status arrays per level, then frontiers A and B.
// After `levels` levels the output count is in slot (levels & 1).
// look-back status words per level: 4096-item chunks of the children, 256-root chunks of the roots
size_t log_cut_chunks(int P, int nroots, int max_child)
{
    return ((size_t)P * (size_t)max(1, max_child) + kCompactChunk - 1) / kCompactChunk + ((size_t)nroots + 255) / 256 +
           1;
}

size_t log_cut_scratch_words(int P, int nroots, int max_child, int levels)
{
    const size_t chunks = log_cut_chunks(P, nroots, max_child);
    return 8 + (size_t)levels + 2 + (size_t)(levels + 2) * 2 * chunks + 2 * (size_t)P;
}

void launch_log_cut(int P, const int32_t* roots, int nroots, const int32_t* node_index, const int32_t* tree,
                    int max_child, const float* radius, float min_res, int levels, int32_t* out, uint32_t* scratch,
                    unsigned* err, cudaStream_t s)
{
    const size_t words = log_cut_scratch_words(P, nroots, max_child, levels);
    cudaMemsetAsync(scratch, 0, sizeof(uint32_t) * (words - 2 * (size_t)P), s);
    if (nroots <= 0) return;
    const size_t chunks = log_cut_chunks(P, nroots, max_child);
    uint32_t* count = scratch;       // [2]
    uint32_t* fsize = scratch + 2;   // [2]
    uint32_t* counters = scratch + 8;
    uint32_t* status = counters + levels + 2;
    int32_t* fr[2];
    fr[0] = reinterpret_cast<int32_t*>(status + (size_t)(levels + 2) * 2 * chunks);
    fr[1] = fr[0] + P;
    log_roots_kernel<<<(nroots + 255) / 256, 256, 0, s>>>(roots, (uint32_t)nroots, node_index, radius, min_res, out,
                                                          count, fr[0], fsize, status, status + chunks, counters,
                                                          err);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    for (int l = 0; l < levels; l++) {
        const int a = l & 1, b = a ^ 1;
        uint32_t* st = status + (size_t)(l + 1) * 2 * chunks;
        log_level_kernel<<<sms * 4, 256, 0, s>>>(fr[a], fsize + a, node_index, tree, max_child, radius, min_res, out,
                                                count + a, count + b, fr[b], fsize + b, st, st + chunks,
                                                counters + 1 + l, (uint32_t)(chunks * kCompactChunk), err);
    }
    note_launches(1 + levels);
}

void launch_cull(const int32_t* in, const uint32_t* n_in, uint32_t cap, const float* radius, const float* opac_raw,
                 float min_px, int64_t* out, unsigned long long* n_out, uint32_t* scratch, unsigned* err,
                 cudaStream_t s)
{
    // one CTA per possible chunk of the capacity; those past the live count leave at once
    const uint32_t nch = (cap + kCompactChunk - 1) / kCompactChunk + 1;
    cudaMemsetAsync(scratch, 0, sizeof(uint32_t) * (1 + nch), s);
    cudaMemsetAsync(n_out, 0, sizeof(unsigned long long), s);
    cull_kernel<<<nch, 256, 0, s>>>(in, n_in, cap, radius, opac_raw, min_px, out, n_out, scratch + 1, scratch, err);
    note_launches(1);
}

void launch_ancestor_path(int P, const int32_t* parent, const int32_t* depth, int L, int32_t* out, unsigned* err,
                          cudaStream_t s)
{
    cudaMemsetAsync(out, 0xff, sizeof(int32_t) * (size_t)P * (size_t)L, s);  // -1 everywhere
    const uint32_t want = ((uint32_t)P + 255) / 256;
    const uint32_t grid = min(want, 8 * resident_ctas(ancestor_path_kernel, 256));
    ancestor_path_kernel<<<grid, 256, 0, s>>>(P, parent, depth, L, out, err);
    note_launches(1);
}

}  // namespace fgs

using namespace fgs;

namespace {
bool a16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }
int launch_status() { return cudaGetLastError() == cudaSuccess ? FGS_OK : FGS_ERR_CUDA; }
}  // namespace

extern "C" {

int fgs_gather_attributes(long long N, const int64_t* index, const float* xyz, const float* scaling,
                          const float* rotation, const float* opacity, const float* colors, const float* shs,
                          int sh_coeffs, int sh_channels, float* o_xyz, float* o_scaling, float* o_rotation,
                          float* o_opacity, float* o_colors, float* o_shs, void* stream)
{
    if (N < 0 || sh_coeffs < 0 || sh_channels < 0) return FGS_ERR_ARG;
    if (N == 0) return FGS_OK;
    if (!index || !xyz || !scaling || !rotation || !opacity || !colors || !o_xyz || !o_scaling || !o_rotation ||
        !o_opacity || !o_colors || (shs && !o_shs))
        return FGS_ERR_ARG;
    if (!a16(rotation) || !a16(o_rotation)) return FGS_ERR_ARG;
    launch_gather(index, N, xyz, scaling, rotation, opacity, colors, shs, sh_coeffs * sh_channels, o_xyz, o_scaling,
                  o_rotation, o_opacity, o_colors, shs ? o_shs : nullptr, static_cast<cudaStream_t>(stream));
    return launch_status();
}

size_t fgs_compact_scratch_bytes(int n) { return n < 0 ? 0 : sizeof(uint32_t) * (size_t)(2 + (n + 255) / 256 + 8); }

int fgs_compact_mask(int n, const uint8_t* mask, int64_t* out_index, unsigned long long* count, void* scratch,
                     void* stream)
{
    if (n < 0 || (n > 0 && (!mask || !out_index)) || !count || !scratch) return FGS_ERR_ARG;
    uint32_t* sc = static_cast<uint32_t*>(scratch);
    unsigned* err = reinterpret_cast<unsigned*>(sc + 2 + (n + 255) / 256);
    cudaMemsetAsync(err, 0, sizeof(unsigned), static_cast<cudaStream_t>(stream));
    launch_compact(mask, (uint32_t)n, out_index, count, sc, err, static_cast<cudaStream_t>(stream));
    return launch_status();
}

int fgs_rows_valid(long long N, const float* xyz, const float* scaling, const float* rotation, const float* opacity,
                   const float* colors, uint8_t* keep, unsigned long long* dropped, void* stream)
{
    if (N < 0 || !dropped) return FGS_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaMemsetAsync(dropped, 0, sizeof(unsigned long long), s);
    if (N == 0) return launch_status();
    if (!xyz || !scaling || !rotation || !opacity || !colors || !keep) return FGS_ERR_ARG;
    const long long want = (N + 255) / 256;
    rows_valid_kernel<<<(int)(want < 1184 ? want : 1184), 256, 0, s>>>(N, xyz, scaling, rotation, opacity, colors,
                                                                    keep, dropped);
    note_launches(1);
    return launch_status();
}

int fgs_gather_activate(long long N_cap, const int64_t* index, const unsigned long long* count_dev,
                        const float* xyz, const float* log_scale, const float* rotation, const float* opacity_raw,
                        const float* features_dc, const float* shs_rest, int sh_degree, int rest_coeffs,
                        const float* campos, float* o_xyz, float* o_scaling, float* o_rotation, float* o_opacity,
                        float* o_colors, void* stream)
{
    if (N_cap < 0 || sh_degree < 0 || sh_degree > 3) return FGS_ERR_ARG;
    if (N_cap == 0) return FGS_OK;
    if (!index || !xyz || !log_scale || !rotation || !opacity_raw || !features_dc || !campos || !o_xyz ||
        !o_scaling || !o_rotation || !o_opacity || !o_colors)
        return FGS_ERR_ARG;
    if (sh_degree > 0 && (!shs_rest || rest_coeffs < (sh_degree + 1) * (sh_degree + 1) - 1)) return FGS_ERR_ARG;
    if (!a16(rotation) || !a16(o_rotation)) return FGS_ERR_ARG;
    launch_gather_activate(index, count_dev, N_cap, xyz, log_scale, rotation, opacity_raw, features_dc,
                           sh_degree > 0 ? shs_rest : nullptr, sh_degree, rest_coeffs, campos, o_xyz, o_scaling,
                           o_rotation, o_opacity, o_colors, static_cast<cudaStream_t>(stream));
    return launch_status();
}

int fgs_radius_raw(int P, const float* means3D, const float* log_scales, const float* rotations,
                   const float* viewmatrix, const float* projmatrix, float focal_x, float focal_y, float tan_fovx,
                   float tan_fovy, float* radius, void* stream)
{
    if (P < 0 || (P > 0 && (!means3D || !log_scales || !rotations || !viewmatrix || !projmatrix || !radius)))
        return FGS_ERR_ARG;
    launch_radius_raw(P, means3D, log_scales, rotations, viewmatrix, projmatrix, focal_x, focal_y, tan_fovx, tan_fovy,
                      radius, static_cast<cudaStream_t>(stream));
    return launch_status();
}

size_t fgs_log_cut_scratch_bytes(int P, int num_roots, int max_child, int levels)
{
    if (P < 0 || num_roots < 0 || max_child < 1 || levels < 0) return 0;
    return sizeof(uint32_t) * (log_cut_scratch_words(P, num_roots, max_child, levels) + 8);
}

int fgs_log_cut(int P, const int32_t* roots, int num_roots, const int32_t* node_index, const int32_t* tree,
                int max_child, const float* radius, float min_resolution_pixel, int levels, int32_t* out,
                uint32_t* out_count_dev, void* scratch, void* stream)
{
    if (P < 0 || num_roots < 0 || num_roots > P || max_child < 1 || levels < 0 || levels > 64) return FGS_ERR_ARG;
    if (P > 0 && (!roots || !node_index || !tree || !radius || !out || !out_count_dev || !scratch))
        return FGS_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t* sc = static_cast<uint32_t*>(scratch);
    const size_t words = log_cut_scratch_words(P, num_roots, max_child, levels);
    unsigned* err = reinterpret_cast<unsigned*>(sc + words);
    cudaMemsetAsync(err, 0, sizeof(unsigned), s);
    if (P == 0 || num_roots == 0) {
        cudaMemsetAsync(out_count_dev, 0, sizeof(uint32_t), s);
        return launch_status();
    }
    launch_log_cut(P, roots, num_roots, node_index, tree, max_child, radius, min_resolution_pixel, levels, out, sc,
                   err, s);
    cudaMemcpyAsync(out_count_dev, sc + (levels & 1), sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    return launch_status();
}

int fgs_ancestor_path(int P, const int32_t* index_parent, const int32_t* depth, int L, int32_t* out,
                      unsigned* err_dev, void* stream)
{
    if (P < 0 || L < 0 || !err_dev || (P > 0 && L > 0 && (!index_parent || !depth || !out))) return FGS_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaMemsetAsync(err_dev, 0, sizeof(unsigned), s);
    // an empty table (L == 0) is returned as is, without the level loop (apps/ancestor.py:51-55)
    if (P > 0 && L > 0) launch_ancestor_path(P, index_parent, depth, L, out, err_dev, s);
    return launch_status();
}

int fgs_cull(const int32_t* ids, const uint32_t* count_dev, int cap, const float* radius, const float* opacity_raw,
             float min_px, int64_t* out, unsigned long long* out_count_dev, void* scratch, void* stream)
{
    if (cap < 0 || !count_dev || !out_count_dev || !scratch || (cap > 0 && (!ids || !radius || !opacity_raw || !out)))
        return FGS_ERR_ARG;
    uint32_t* sc = static_cast<uint32_t*>(scratch);
    unsigned* err = reinterpret_cast<unsigned*>(sc + 2 + (cap + 255) / 256 + 1);
    cudaMemsetAsync(err, 0, sizeof(unsigned), static_cast<cudaStream_t>(stream));
    launch_cull(ids, count_dev, (uint32_t)cap, radius, opacity_raw, min_px, out, out_count_dev, sc, err,
                static_cast<cudaStream_t>(stream));
    return launch_status();
}

}  // extern "C"
