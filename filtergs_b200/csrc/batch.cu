// Many views of one Gaussian set in one stream-ordered, host-sync-free
// sequence (the batched path; the reference renders one view per call).
//
// fgs_batch_create carves a caller-owned workspace into per-view state with
// fixed pair capacities and uploads the per-view tile descriptors once; after
// that fgs_batch_forward / fgs_batch_backward only enqueue kernels and
// memsets on the caller's stream -- no host synchronisation, no allocation --
// so the pair can be captured into a CUDA graph and replayed.  Per view the
// front end (preprocess, depth sort, pair emission, tile sort, ranges) runs
// with the pair count kept on the device, the views spread over eight streams
// forked from the caller's stream and joined before compositing (those kernels
// are latency-bound, so views overlap); compositing, forward and backward,
// is ONE persistent launch per direction over the tiles of all views, fed by a
// global work queue.  Backward then gathers each view's screen-space gradients
// (views on the same streams) and sums every view's gradients per Gaussian in
// view order in one pass, writing each shared gradient row once.
// A view whose pairs exceed its capacity is truncated and FGS_ERR_OVERFLOW is
// recorded; fgs_batch_check reports it (the caller re-plans with a larger
// capacity, outside any captured graph).
#include <cstring>
#include <new>
#include <vector>

#include "fgs_common.cuh"
#include "fgs_internal.h"

namespace fgs {
namespace {

constexpr size_t kAlign = 256;
inline size_t align_up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

struct ViewState {
    PreParams pre;
    int num_tiles, tile_bits;
    long long cap;
    GeomState g;
    ImageState im;
    BinState b;
    char* geom_base;
    size_t geom_bytes_v;
    float *dmean2D, *dconic, *dopac, *dcolor;  // screen-space gradients of this view
    int* radii_out;
};

constexpr int kFrontStreams = 8;  // views whose front ends run concurrently

struct Batch {
    int P, V, consistent;
    // fork/join of the per-view front ends over auxiliary streams (graph-capturable)
    std::vector<cudaStream_t> aux;
    std::vector<cudaEvent_t> joined;
    cudaEvent_t forked = nullptr;
    ~Batch()
    {
        for (cudaStream_t x : aux) cudaStreamDestroy(x);
        for (cudaEvent_t e : joined) cudaEventDestroy(e);
        if (forked) cudaEventDestroy(forked);
    }
    std::vector<ViewState> views;
    TileArgs* d_args_fwd;
    TileArgs* d_args_bwd;
    std::vector<TileArgs> h_args;  // host copy of d_args_fwd ++ d_args_bwd (sources of pointer updates)
    uint32_t* d_begin;
    uint32_t* d_queue;
    uint32_t* d_long;  // long-tile bins [32][total_tiles], then their 34 counters
    unsigned* d_err;
    uint32_t total_tiles;
    const float* background;
    float *g_means3D, *g_opacity, *g_sh, *g_scales, *g_rot;
    FoldView* d_fold;  // [V] per-view backward descriptors
    FoldView h_fold0;  // host copy of view 0's (the inputs all views share)
    uint32_t* d_vis;   // [(V + 31) / 32][P] views that saw each Gaussian (set by the gathers)
    unsigned long long* d_seen_count;
    uint32_t* d_seen;  // [P] the Gaussians some view saw (count in d_seen_count)
    int vis_words;
    DensifyStats dens{nullptr, nullptr, nullptr};  // optional (fgs_batch_set_densify)
    int M;
    bool has_sr;
    float4* packed;  // [3][P] (PreParams::packed), refreshed by every forward
};

struct Layout {
    size_t total;
    std::vector<size_t> geom_off, img_off, bin_off, grad_off;
    size_t args_off, begin_off, misc_off, vis_off, list_off, fold_off, long_off, packed_off;
};

// Zero every view's per-Gaussian maximum weight (out_point_weight, when the view has one)
// before the forward compositing takes its maxima; the pointers are read from the device
// descriptors, so a captured graph follows fgs_batch_set_view_outputs.
__global__ void zero_point_weight_kernel(const TileArgs* __restrict__ views, int P)
{
    float* pw = views[blockIdx.y].out_point_weight;
    if (!pw) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P; i += gridDim.x * blockDim.x) pw[i] = 0.f;
}

Layout plan(int P, int V, const fgs_view_args* views)
{
    Layout L;
    size_t off = 0;
    for (int v = 0; v < V; v++) {
        L.geom_off.push_back(off);
        off = align_up(off + geom_bytes(P));
        L.img_off.push_back(off);
        off = align_up(off + image_bytes(views[v].width, views[v].height));
        L.bin_off.push_back(off);
        off = align_up(off + bin_bytes(views[v].pair_capacity, P));
        L.grad_off.push_back(off);
        off = align_up(off + sizeof(float) * 11 * (size_t)P);
    }
    L.args_off = off;
    off = align_up(off + 2 * sizeof(TileArgs) * (size_t)V);
    L.begin_off = off;
    off = align_up(off + sizeof(uint32_t) * (size_t)(V + 1));
    L.misc_off = off;
    off = align_up(off + 64);
    L.vis_off = off;
    off = align_up(off + sizeof(uint32_t) * (size_t)((V + 31) / 32) * P);
    L.list_off = off;  // count (8 bytes, padded to 16), then [P] ids
    off = align_up(off + 16 + sizeof(uint32_t) * (size_t)P);
    L.fold_off = off;
    off = align_up(off + sizeof(FoldView) * (size_t)V);
    size_t tiles = 0;
    for (int v = 0; v < V; v++)
        tiles += (size_t)((views[v].width + kTileX - 1) / kTileX) * ((views[v].height + kTileY - 1) / kTileY);
    L.long_off = off;  // long-tile bins [32][tiles] + 34 counters
    off = align_up(off + sizeof(uint32_t) * (32 * tiles + 34));
    L.packed_off = off;  // the Gaussians' packed float4 planes, shared by the views' preprocess
    off = align_up(off + 3 * sizeof(float4) * (size_t)P);
    L.total = off;
    return L;
}

int tile_bits_of(int num_tiles)
{
    int bits = 1;
    while (bits < 31 && (1u << bits) < (unsigned)num_tiles) bits++;
    return bits;
}

}  // namespace
}  // namespace fgs

using namespace fgs;

extern "C" {

size_t fgs_batch_workspace_bytes(int P, int nviews, const fgs_view_args* views)
{
    if (P < 0 || nviews <= 0 || !views) return 0;
    for (int v = 0; v < nviews; v++)
        if (views[v].width <= 0 || views[v].height <= 0 || views[v].pair_capacity < 0) return 0;
    return plan(P, nviews, views).total;
}

void* fgs_batch_create(const fgs_raster_args* shared, int nviews, const fgs_view_args* views, void* workspace,
                       size_t workspace_bytes, int backward_mode, float* dL_dmeans3D, float* dL_dopacity,
                       float* dL_dsh, float* dL_dscales, float* dL_drotations, int* status, void* stream)
{
    auto fail = [&](int st) -> void* {
        if (status) *status = st;
        return nullptr;
    };
    if (!shared || nviews <= 0 || !views || !workspace) return fail(FGS_ERR_ARG);
    if (backward_mode != FGS_BACKWARD_REF_COMPAT && backward_mode != FGS_BACKWARD_CONSISTENT) return fail(FGS_ERR_ARG);
    const int P = shared->P;
    if (P <= 0) return fail(FGS_ERR_ARG);
    const Layout L = plan(P, nviews, views);
    if (workspace_bytes < L.total) return fail(FGS_ERR_ARG);
    if ((reinterpret_cast<uintptr_t>(workspace) & (kAlign - 1)) != 0) return fail(FGS_ERR_ARG);
    Batch* B = new (std::nothrow) Batch();
    if (!B) return fail(FGS_ERR_CUDA);
    B->P = P;
    B->V = nviews;
    B->consistent = backward_mode == FGS_BACKWARD_CONSISTENT;
    {
        const int ns = nviews < kFrontStreams ? nviews : kFrontStreams;
        bool ok = cudaEventCreateWithFlags(&B->forked, cudaEventDisableTiming) == cudaSuccess;
        for (int i = 0; ok && i < ns; i++) {
            cudaStream_t x = nullptr;
            cudaEvent_t e = nullptr;
            ok = cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking) == cudaSuccess;
            if (ok) B->aux.push_back(x);
            ok = ok && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess;
            if (ok) B->joined.push_back(e);
        }
        if (!ok) {
            delete B;
            return fail(FGS_ERR_CUDA);
        }
    }
    B->background = shared->background;
    B->g_means3D = dL_dmeans3D;
    B->g_opacity = dL_dopacity;
    B->g_sh = dL_dsh;
    B->g_scales = dL_dscales;
    B->g_rot = dL_drotations;
    char* base = static_cast<char*>(workspace);
    B->d_vis = reinterpret_cast<uint32_t*>(base + L.vis_off);
    B->d_seen_count = reinterpret_cast<unsigned long long*>(base + L.list_off);
    B->d_seen = reinterpret_cast<uint32_t*>(base + L.list_off + 16);
    B->vis_words = (nviews + 31) / 32;
    B->d_fold = reinterpret_cast<FoldView*>(base + L.fold_off);
    B->packed = reinterpret_cast<float4*>(base + L.packed_off);
    std::vector<TileArgs> fa(nviews), ba(nviews);
    std::vector<uint32_t> begin(nviews + 1, 0);
    for (int v = 0; v < nviews; v++) {
        const fgs_view_args& va = views[v];
        fgs_raster_args a = *shared;
        a.width = va.width;
        a.height = va.height;
        a.viewmatrix = va.viewmatrix;
        a.projmatrix = va.projmatrix;
        a.campos = va.campos;
        a.tan_fovx = va.tan_fovx;
        a.tan_fovy = va.tan_fovy;
        a.ogfs_enable_stats = 0;
        ViewState s{};
        int st = make_params(&a, s.pre);
        if (st || !va.out_color || va.pair_capacity >= (1ll << 30)) {
            delete B;
            return fail(st ? st : FGS_ERR_ARG);
        }
        s.pre.packed = B->packed;  // every view's preprocess reads the packed copy
        const int gx = (va.width + kTileX - 1) / kTileX, gy = (va.height + kTileY - 1) / kTileY;
        s.num_tiles = gx * gy;
        s.tile_bits = tile_bits_of(s.num_tiles);
        s.cap = va.pair_capacity;
        s.geom_base = base + L.geom_off[v];
        s.geom_bytes_v = geom_bytes(P);
        s.g = geom_views(s.geom_base, P);
        s.im = image_views(base + L.img_off[v], va.width, va.height);
        s.b = bin_views(base + L.bin_off[v], s.cap, P);
        float* gr = reinterpret_cast<float*>(base + L.grad_off[v]);
        s.dmean2D = gr;
        s.dconic = gr + 3 * (size_t)P;
        s.dopac = gr + 7 * (size_t)P;
        s.dcolor = gr + 8 * (size_t)P;
        s.radii_out = va.out_radii;
        B->M = s.pre.M;
        B->has_sr = s.pre.scales != nullptr;
        TileArgs f{};
        f.ranges = s.im.ranges; f.recs = s.b.rec; f.W = va.width; f.H = va.height; f.bg = shared->background;
        f.out_color = va.out_color; f.final_T = s.im.final_T; f.n_contrib = s.im.n_contrib;
        TileArgs bk = f;
        bk.out_color = nullptr;
        bk.dL_dpix = va.dL_dout_color;
        bk.pgrad = s.b.pgrad;
        fa[v] = f;
        ba[v] = bk;
        begin[v + 1] = begin[v] + (uint32_t)s.num_tiles;
        B->views.push_back(s);
    }
    B->total_tiles = begin[nviews];
    std::vector<FoldView> fold(nviews);
    for (int v = 0; v < nviews; v++) {
        const ViewState& s = B->views[v];
        fold[v] = FoldView{s.pre, s.dmean2D, s.dmean2D, s.dconic, s.dopac, s.dcolor, s.g.clamped};
    }
    B->h_fold0 = fold[0];
    B->h_args = fa;
    B->h_args.insert(B->h_args.end(), ba.begin(), ba.end());
    B->d_args_fwd = reinterpret_cast<TileArgs*>(base + L.args_off);
    B->d_args_bwd = B->d_args_fwd + nviews;
    B->d_begin = reinterpret_cast<uint32_t*>(base + L.begin_off);
    B->d_queue = reinterpret_cast<uint32_t*>(base + L.misc_off);
    B->d_err = reinterpret_cast<unsigned*>(base + L.misc_off + 16);
    B->d_long = reinterpret_cast<uint32_t*>(base + L.long_off);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cudaMemcpyAsync(B->d_args_fwd, fa.data(), sizeof(TileArgs) * nviews, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(B->d_args_bwd, ba.data(), sizeof(TileArgs) * nviews, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(B->d_begin, begin.data(), sizeof(uint32_t) * (nviews + 1), cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaMemcpyAsync(B->d_fold, fold.data(), sizeof(FoldView) * nviews, cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaMemsetAsync(B->d_queue, 0, 64, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
        delete B;
        return fail(FGS_ERR_CUDA);
    }
    if (status) *status = FGS_OK;
    return B;
}

void fgs_batch_destroy(void* handle) { delete static_cast<Batch*>(handle); }

int fgs_batch_set_view_io(void* handle, int count, const int* view_ids, float* const* out_color,
                          const float* const* dL_dout_color, void* stream)
{
    Batch* B = static_cast<Batch*>(handle);
    if (!B || count < 0 || (count > 0 && (!view_ids || !out_color))) return FGS_ERR_ARG;
    for (int i = 0; i < count; i++)
        if (view_ids[i] < 0 || view_ids[i] >= B->V || !out_color[i]) return FGS_ERR_ARG;
    for (int i = 0; i < count; i++) {
        B->h_args[view_ids[i]].out_color = out_color[i];
        if (dL_dout_color && dL_dout_color[i]) B->h_args[B->V + view_ids[i]].dL_dpix = dL_dout_color[i];
    }
    // one copy of the whole descriptor table (forward ++ backward are contiguous); the source is
    // pageable, so it is staged before the call returns and later updates cannot race it
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cudaMemcpyAsync(B->d_args_fwd, B->h_args.data(), sizeof(TileArgs) * B->h_args.size(), cudaMemcpyHostToDevice,
                        s) != cudaSuccess)
        return FGS_ERR_CUDA;
    return FGS_OK;
}

int fgs_batch_set_view_outputs(void* handle, int count, const int* view_ids, int* const* out_point_id,
                               float* const* out_point_weight_pixel, float* const* out_point_weight, void* stream)
{
    Batch* B = static_cast<Batch*>(handle);
    if (!B || count < 0 || (count > 0 && !view_ids)) return FGS_ERR_ARG;
    for (int i = 0; i < count; i++)
        if (view_ids[i] < 0 || view_ids[i] >= B->V) return FGS_ERR_ARG;
    for (int i = 0; i < count; i++) {
        TileArgs& f = B->h_args[view_ids[i]];
        f.out_point_id = out_point_id ? out_point_id[i] : nullptr;
        f.out_pw_pixel = out_point_weight_pixel ? out_point_weight_pixel[i] : nullptr;
        f.out_point_weight = out_point_weight ? out_point_weight[i] : nullptr;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cudaMemcpyAsync(B->d_args_fwd, B->h_args.data(), sizeof(TileArgs) * B->h_args.size(), cudaMemcpyHostToDevice,
                        s) != cudaSuccess)
        return FGS_ERR_CUDA;
    return FGS_OK;
}

int fgs_batch_forward(void* handle, void* stream)
{
    Batch* B = static_cast<Batch*>(handle);
    if (!B) return FGS_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // The per-view front ends are independent and mostly latency-bound (scans with
    // look-back, small sorts): they run on kFrontStreams streams forked from `s`
    // and joined back before the one compositing launch over all views.
    const int ns = (int)B->aux.size();
    {
        // one structure-of-arrays copy of the Gaussians per forward, read by every view
        StageTimer t(FGS_STAGE_PREPROCESS, s);
        const PreParams& p0 = B->views[0].pre;
        launch_pack_gaussians(B->P, p0.means, p0.opac, p0.scales, p0.rots, B->packed, s);
    }
    if (cudaEventRecord(B->forked, s) != cudaSuccess) return FGS_ERR_CUDA;
    for (int i = 0; i < ns; i++) cudaStreamWaitEvent(B->aux[i], B->forked, 0);
    for (int vi = 0; vi < B->V; vi++) {
        ViewState& v = B->views[vi];
        cudaStream_t vs = B->aux[vi % ns];
        {
            StageTimer t(FGS_STAGE_PREPROCESS, vs);
            char* zero_begin = reinterpret_cast<char*>(v.g.hist);
            cudaMemsetAsync(zero_begin, 0, (size_t)(v.geom_base + v.geom_bytes_v - zero_begin), vs);
            launch_preprocess(v.pre, v.g, v.radii_out, vs);
        }
        {
            StageTimer t(FGS_STAGE_DEPTH_SORT, vs);
            launch_depth_sort(v.g, B->P, vs);
        }
        if (v.cap > 0) {
            {
                StageTimer t(FGS_STAGE_DUPLICATE, vs);
                cudaMemsetAsync(v.b.status, 0, sizeof(uint32_t) * (v.b.status_words + v.b.scan_words), vs);
                launch_duplicate(v.g, v.b, (uint32_t)B->P, (uint32_t)v.cap, v.pre.W, v.pre.H, v.tile_bits, vs);
            }
            StageTimer t(FGS_STAGE_TILE_SORT, vs);
            launch_tile_sort(v.g, v.b, v.cap, v.tile_bits, v.pre.W, v.pre.H, vs, v.g.total);
        }
        StageTimer t(FGS_STAGE_RANGES, vs);
        launch_ranges(v.b, v.im, v.cap, v.num_tiles, vs, v.g.total);
    }
    for (int i = 0; i < ns; i++) {
        cudaEventRecord(B->joined[i], B->aux[i]);
        cudaStreamWaitEvent(s, B->joined[i], 0);
    }
    StageTimer t(FGS_STAGE_RENDER_FWD, s);
    zero_point_weight_kernel<<<dim3((unsigned)((B->P + 255) / 256 < 592 ? (B->P + 255) / 256 : 592), (unsigned)B->V),
                               256, 0, s>>>(B->d_args_fwd, B->P);
    note_launches(1);
    launch_render_fwd_multi(B->d_args_fwd, B->d_begin, B->V, B->total_tiles, B->d_queue, B->d_long,
                            B->d_long + 32 * (size_t)B->total_tiles, B->d_err, s);
    return cudaGetLastError() == cudaSuccess ? FGS_OK : FGS_ERR_CUDA;
}

int fgs_batch_backward(void* handle, void* stream)
{
    Batch* B = static_cast<Batch*>(handle);
    if (!B) return FGS_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t P = (size_t)B->P;
    if (!B->g_means3D || !B->g_opacity) return FGS_ERR_ARG;
    {
        StageTimer t(FGS_STAGE_RENDER_BWD, s);
        launch_render_bwd_multi(B->d_args_bwd, B->d_begin, B->V, B->total_tiles, B->d_queue + 1, B->consistent,
                                B->d_err, s);
    }
    StageTimer t(FGS_STAGE_PREPROCESS_BWD, s);
    // Each view's screen-space gradients (the sums of its per-pair rows) and the
    // views that saw each Gaussian, the views spread over the front-end streams;
    // then one pass per Gaussian over all views writes every gradient row once.
    cudaMemsetAsync(B->d_vis, 0, sizeof(uint32_t) * (size_t)B->vis_words * P, s);
    const int ns = (int)B->aux.size();
    if (cudaEventRecord(B->forked, s) != cudaSuccess) return FGS_ERR_CUDA;
    for (int i = 0; i < ns; i++) cudaStreamWaitEvent(B->aux[i], B->forked, 0);
    // the shared outputs are zeroed while the gathers run (the fold writes the rows of
    // the Gaussians some view saw)
    const bool sh = B->views[0].pre.shs && B->g_sh;
    cudaMemsetAsync(B->g_means3D, 0, sizeof(float) * 3 * P, s);
    cudaMemsetAsync(B->g_opacity, 0, sizeof(float) * P, s);
    if (sh) cudaMemsetAsync(B->g_sh, 0, sizeof(float) * 3 * (size_t)B->M * P, s);
    if (B->has_sr && B->g_scales) cudaMemsetAsync(B->g_scales, 0, sizeof(float) * 3 * P, s);
    if (B->has_sr && B->g_rot) cudaMemsetAsync(B->g_rot, 0, sizeof(float) * 4 * P, s);
    for (int vi = 0; vi < B->V; vi++) {
        ViewState& v = B->views[vi];
        launch_pair_grad_gather(v.g, v.b.pgrad, v.cap, v.dmean2D, v.dconic, v.dcolor, v.dopac,
                                B->d_vis + (size_t)(vi >> 5) * P, 1u << (vi & 31), B->P, B->aux[vi % ns]);
    }
    for (int i = 0; i < ns; i++) {
        cudaEventRecord(B->joined[i], B->aux[i]);
        cudaStreamWaitEvent(s, B->joined[i], 0);
    }
    launch_fold_bwd(B->d_fold, B->V, B->P, B->d_vis, B->d_seen, B->d_seen_count, B->consistent, sh, B->g_means3D,
                    B->g_opacity, sh ? B->g_sh : nullptr, B->has_sr ? B->g_scales : nullptr,
                    B->has_sr ? B->g_rot : nullptr, B->dens.grad_sum ? &B->dens : nullptr, B->h_fold0, s);
    return cudaGetLastError() == cudaSuccess ? FGS_OK : FGS_ERR_CUDA;
}

int fgs_batch_set_densify(void* handle, float* grad_sum, int* vis_count, unsigned char* flag)
{
    Batch* B = static_cast<Batch*>(handle);
    if (!B) return FGS_ERR_ARG;
    if ((grad_sum == nullptr) != (vis_count == nullptr) || (grad_sum == nullptr) != (flag == nullptr))
        return FGS_ERR_ARG;
    B->dens = DensifyStats{grad_sum, vis_count, flag};
    return FGS_OK;
}

int fgs_batch_pair_counts(void* handle, long long* counts, void* stream)
{
    Batch* B = static_cast<Batch*>(handle);
    if (!B || !counts) return FGS_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    std::vector<unsigned long long> tot(2 * B->V);
    for (int v = 0; v < B->V; v++)
        cudaMemcpyAsync(&tot[2 * v], B->views[v].g.total, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return FGS_ERR_CUDA;
    for (int v = 0; v < B->V; v++) counts[v] = (long long)tot[2 * v];
    return FGS_OK;
}

int fgs_batch_check(void* handle, void* stream)
{
    Batch* B = static_cast<Batch*>(handle);
    if (!B) return FGS_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    std::vector<unsigned> errs(B->V + 1, 0);
    for (int v = 0; v < B->V; v++)
        cudaMemcpyAsync(&errs[v], B->views[v].g.err, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&errs[B->V], B->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) return FGS_ERR_CUDA;
    unsigned all = 0;
    for (unsigned e : errs) all |= e;
    for (int c = 1; c < 32; c++)
        if (all & (1u << c)) return c;
    return FGS_OK;
}

}  // extern "C"
