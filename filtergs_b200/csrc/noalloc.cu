// Forward rendering without any device allocation by the library or its caller.
//
// Some callers cannot allocate device memory while they render: a viewer or
// game engine that submits a frame from its render thread and must not hit the
// device-wide synchronisation and possible stall of cudaMalloc, a plugin that
// runs inside a host application which owns every device allocation, or a
// process running under a fixed device-memory budget.  They still own their
// inputs and outputs, but have nowhere to put the rasterizer's three scratch
// workspaces (per-Gaussian state, per-pixel state, tile/Gaussian pairs).
//
// fgs_forward_noalloc keeps those workspaces in one file-scope device array of
// kNoAllocScratchBytes (32 MiB), which every GPU that loads this library holds
// until the process exits.  The array's host-side name is not a device
// address; each call looks up its device address on the current device with
// cudaGetSymbolAddress (a table lookup once the module is loaded), so a device
// reset or a new primary context between calls leaves no stale address.  The
// first call on a device loads the library's device code there, so it should
// come before any stream capture.
//
// Every call shares the array and finds the previous call's contents in it;
// all state that must start at zero is cleared on the stream at the start of
// each call.  Two calls whose work overlaps on the GPU (different streams, or
// different host threads) race on the array: callers must serialise them.
#include "fgs_common.cuh"
#include "fgs_internal.h"

namespace fgs {

namespace {

constexpr size_t kNoAllocScratchBytes = 32ull << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of the scratch array in the current device's context, looked
// up on every call (never cached: a reset device reloads the module elsewhere).
int noalloc_scratch(void** out)
{
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return FGS_ERR_CUDA;
    *out = p;
    return FGS_OK;
}

int first_error(unsigned bits)
{
    for (int c = 1; c < 32; c++)
        if (bits & (1u << c)) return c;
    return FGS_OK;
}

}  // namespace

}  // namespace fgs

using namespace fgs;

extern "C" {

size_t fgs_noalloc_capacity_bytes(void) { return kNoAllocScratchBytes; }

int fgs_forward_noalloc(const fgs_raster_args* a, int* radii, float* out_color, int* out_point_id,
                        float* out_point_weight_pixel, float* out_point_weight, long long* num_rendered,
                        void* stream)
{
    PreParams p;
    int st = make_params(a, p);
    if (st) return st;
    if (a->ogfs_enable_stats) return FGS_ERR_ARG;  // the statistics need workspace this entry point does not have
    if (!radii || !out_color || !out_point_id || !out_point_weight_pixel || !out_point_weight || !num_rendered)
        return FGS_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (p.P == 0) {  // nothing to draw: the reference's all-zero outputs
        const size_t N = (size_t)p.W * p.H;
        cudaMemsetAsync(out_color, 0, sizeof(float) * 3 * N, s);
        cudaMemsetAsync(out_point_id, 0, sizeof(int) * N, s);
        cudaMemsetAsync(out_point_weight_pixel, 0, sizeof(float) * N, s);
        *num_rendered = 0;
        return cudaGetLastError() == cudaSuccess ? FGS_OK : FGS_ERR_CUDA;
    }
    const size_t gb = geom_bytes(p.P), ib = image_bytes(p.W, p.H);
    if (gb + ib > kNoAllocScratchBytes) return FGS_ERR_CAPACITY;
    void* scratch = nullptr;
    if ((st = noalloc_scratch(&scratch))) return st;
    char* base = static_cast<char*>(scratch);
    char* geom = base;
    char* image = base + gb;
    GeomState g = geom_views(geom, p.P);
    ImageState im = image_views(image, p.W, p.H);
    // everything from the radix histograms to the end of the geometry workspace starts at zero
    char* zero_begin = reinterpret_cast<char*>(g.hist);
    cudaMemsetAsync(zero_begin, 0, (size_t)(geom + gb - zero_begin), s);
    launch_preprocess(p, g, radii, s);
    launch_depth_sort(g, p.P, s);
    unsigned long long tot[2] = {0, 0};
    unsigned err = 0;
    cudaMemcpyAsync(tot, g.total, sizeof(tot), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&err, g.err, sizeof(err), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) return FGS_ERR_CUDA;
    if (err) return first_error(err);
    if (tot[0] >= (1ull << 30)) return FGS_ERR_OVERFLOW;
    const long long K = (long long)tot[0];
    const size_t bb = bin_bytes_forward(K, p.P);
    if (gb + ib + bb > kNoAllocScratchBytes) return FGS_ERR_CAPACITY;
    BinState b = bin_views(base + gb + ib, K, p.P);
    const int gx = (p.W + kTileX - 1) / kTileX, gy = (p.H + kTileY - 1) / kTileY;
    const int num_tiles = gx * gy;
    const int tbits = tile_bits_for(num_tiles);
    cudaMemsetAsync(out_point_weight, 0, sizeof(float) * (size_t)p.P, s);
    if (K > 0) {
        cudaMemsetAsync(b.status, 0, sizeof(uint32_t) * (b.status_words + b.scan_words), s);
        launch_duplicate(g, b, (uint32_t)p.P, (uint32_t)K, p.W, p.H, tbits, s);
        launch_tile_sort(g, b, K, tbits, p.W, p.H, s);
    }
    launch_ranges(b, im, K, num_tiles, s);
    launch_render_fwd(p.W, p.H, im, b, K, a->background, out_color, out_point_id, out_point_weight_pixel,
                      out_point_weight, false, g.err, s);
    cudaMemcpyAsync(&err, g.err, sizeof(err), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) return FGS_ERR_CUDA;
    if (err) return first_error(err);
    *num_rendered = K;
    return FGS_OK;
}

}  // extern "C"
