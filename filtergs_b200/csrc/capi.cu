// extern "C" entry points (include/filtergs_b200.h): argument checks,
// workspace carving, kernel sequencing on the caller's stream.
#include <atomic>
#include <cerrno>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "fgs_common.cuh"
#include "fgs_internal.h"

namespace fgs {

namespace {

constexpr size_t kAlign = 256;
inline size_t align_up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

struct Carver {
    char* base;
    size_t off = 0;
    template <typename T>
    T* take(size_t count)
    {
        T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
        off = align_up(off + count * sizeof(T));
        return p;
    }
};

inline uint32_t sort_chunks(long long n) { return (uint32_t)((n + sort_chunk_size() - 1) / sort_chunk_size()); }

struct GeomCarve {
    GeomState g;
    char* zero_begin;
    size_t zero_bytes;
    size_t total;
};

GeomCarve carve_geom(void* base, int P)
{
    Carver c{static_cast<char*>(base)};
    GeomCarve r{};
    r.g.grec = c.take<PairRecord>(P);
    r.g.radii = c.take<int>(P);
    r.g.tiles = c.take<uint32_t>(P);
    r.g.clamped = c.take<uint8_t>(P);
    r.g.depth_key = c.take<uint32_t>(P);
    r.g.sort_ids_a = c.take<uint32_t>(P);
    r.g.sort_ids_b = c.take<uint32_t>(P);
    r.g.sort_keys_b = c.take<uint32_t>(P);
    r.g.pair_off = r.g.sort_keys_b;
    r.g.erow = c.take<int2>(P);
    r.g.cand_ids = c.take<uint32_t>(P);
    const size_t zero_off = c.off;
    r.g.hist = c.take<uint32_t>(8 * 256);
    r.g.counters = c.take<uint32_t>(16);
    r.g.total = c.take<unsigned long long>(4);
    r.g.err = c.take<unsigned int>(1);
    r.g.status_words = (size_t)4 * sort_chunks(P) * 256;
    r.g.status = c.take<uint32_t>(r.g.status_words);
    r.g.chunk_counts = c.take<uint32_t>(2 * (((size_t)P + 255) / 256));
    r.zero_begin = base ? static_cast<char*>(base) + zero_off : nullptr;
    r.zero_bytes = c.off - zero_off;
    r.total = c.off;
    return r;
}

struct BinCarve {
    BinState b;
    size_t total;
};

BinCarve carve_bin(void* base, long long K, int P, bool with_grad = true)
{
    Carver c{static_cast<char*>(base)};
    BinCarve r{};
    r.b.tile_a = c.take<uint32_t>(K);
    r.b.tile_b = c.take<uint32_t>(K);
    r.b.val_a = c.take<uint32_t>(K);
    r.b.val_b = c.take<uint32_t>(K);
    r.b.rec = c.take<PairRecord>(K);
    r.b.status_words = (size_t)4 * sort_chunks(K) * 256;
    r.b.status = c.take<uint32_t>(r.b.status_words);
    r.b.scan_words = (size_t)(P + 255) / 256 + 1;
    r.b.scan_status = c.take<uint32_t>(r.b.scan_words);
    // Statistics reuse the sort's scratch buffers, dead once the last pass ran.
    r.b.kv_sum = reinterpret_cast<float*>(r.b.tile_a);
    r.b.kv_cnt = r.b.val_a;
    r.b.pgrad = with_grad ? c.take<float>((size_t)9 * K) : nullptr;
    r.total = c.off;
    return r;
}

// Device errors recorded after a launch are read back lazily through this
// pinned word (checked at the next synchronisation point on the host).
unsigned int* pinned_words()
{
    static unsigned int* w = nullptr;
    if (!w) {
        if (cudaHostAlloc(reinterpret_cast<void**>(&w), 64, cudaHostAllocDefault) != cudaSuccess) w = nullptr;
        if (w) memset(w, 0, 64);
    }
    return w;
}

int err_code_from_bits(unsigned bits)
{
    for (int c = 1; c < 32; c++)
        if (bits & (1u << c)) return c;
    return FGS_OK;
}

int cuda_status(cudaError_t e) { return e == cudaSuccess ? FGS_OK : FGS_ERR_CUDA; }

int check_launch()
{
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FGS_OK : FGS_ERR_CUDA;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

int tile_bits_for(int num_tiles)
{
    int bits = 1;
    while (bits < 31 && (1u << bits) < (unsigned)num_tiles) bits++;
    return bits;
}

int make_params(const fgs_raster_args* a, PreParams& p, bool backward)
{
    if (!a) return FGS_ERR_ARG;
    // P < 2^30: visible counts travel in the 30-bit values of the look-back status words
    if (a->P < 0 || a->P >= (1 << 30) || a->width <= 0 || a->height <= 0) return FGS_ERR_ARG;
    if (a->P > 0 && (!a->means3D || (!backward && !a->opacities))) return FGS_ERR_ARG;
    if (!a->viewmatrix || !a->projmatrix || !a->background) return FGS_ERR_ARG;
    const bool has_sr = a->scales && a->rotations;
    if (a->P > 0 && !has_sr && !a->cov3D_precomp) return FGS_ERR_ARG;
    if (a->P > 0 && !a->colors_precomp && !a->shs) return FGS_ERR_ARG;
    if (a->shs && (a->M <= 0 || a->D < 0 || a->D > 3 || (a->D + 1) * (a->D + 1) > a->M)) return FGS_ERR_ARG;
    if (a->shs && !a->colors_precomp && !a->campos) return FGS_ERR_ARG;
    if (a->filter3d_scale < 0.f) return FGS_ERR_ARG;
    p.P = a->P;
    p.D = a->D;
    p.M = a->shs ? a->M : 0;
    p.W = a->width;
    p.H = a->height;
    p.means = a->means3D;
    p.scales = has_sr ? a->scales : nullptr;
    p.rots = has_sr ? a->rotations : nullptr;
    p.opac = a->opacities;
    p.shs = a->colors_precomp ? nullptr : a->shs;
    p.cov3D = a->cov3D_precomp;
    p.colors = a->colors_precomp;
    p.view = a->viewmatrix;
    p.proj = a->projmatrix;
    p.campos = a->campos;
    p.scale_mod = a->scale_modifier;
    p.tanx = a->tan_fovx;
    p.tany = a->tan_fovy;
    // rasterizer_impl.cu:283-284
    p.fy = a->height / (2.0f * a->tan_fovy);
    p.fx = a->width / (2.0f * a->tan_fovx);
    p.prefiltered = a->prefiltered;
    p.use_filter = a->use_filter;
    p.eps_scale = a->ogfs_epsilon_scale;
    p.eps_max = a->ogfs_epsilon_max;
    p.energy_floor = a->ogfs_energy_floor;
    p.ratio_min = a->ogfs_radius_ratio_min;
    p.filter3d = a->filter3d_scale;
    p.packed = nullptr;
    p.aligned = aligned16(p.means) && (!p.opac || aligned16(p.opac)) && (!p.scales || aligned16(p.scales)) &&
                (!p.rots || aligned16(p.rots)) && (!p.shs || aligned16(p.shs));
    return FGS_OK;
}

namespace {

// rasterizer_impl.cu:44-55
float kpc_used_thresh()
{
    const char* env = std::getenv("KPC_USED_THRESH");
    if (!env || env[0] == '\0') return 1e-4f;
    char* end = nullptr;
    errno = 0;
    const float v = std::strtof(env, &end);
    if (errno != 0 || end == env || v <= 0.0f) return 1e-4f;
    return v;
}

__global__ void sorted_keys_kernel(const uint32_t* __restrict__ tile, const uint32_t* __restrict__ val,
                                   const PairRecord* __restrict__ grec, uint32_t K, uint64_t* __restrict__ keys,
                                   uint32_t* __restrict__ vals)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= K) return;
    const uint32_t v = val[i];
    if (keys) keys[i] = ((uint64_t)tile[i] << 32) | __float_as_uint(grec[v].c.z);
    if (vals) vals[i] = v;
}

__global__ void pre_outputs_kernel(const PairRecord* __restrict__ grec, const uint32_t* __restrict__ tiles, int P,
                                   float* means2D, float* depths, float* conic_o, float* rgb, uint32_t* tt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const PairRecord r = grec[i];
    if (means2D) { means2D[2 * i] = r.a.x; means2D[2 * i + 1] = r.a.y; }
    if (depths) depths[i] = r.c.z;
    if (conic_o) {
        conic_o[4 * i] = r.a.z; conic_o[4 * i + 1] = r.a.w; conic_o[4 * i + 2] = r.b.x; conic_o[4 * i + 3] = r.b.y;
    }
    if (rgb) { rgb[3 * i] = r.b.z; rgb[3 * i + 1] = r.b.w; rgb[3 * i + 2] = r.c.x; }
    if (tt) tt[i] = tiles[i];
}

}  // namespace

// ---------------------------------------------------------------- profiling
namespace {
struct EventPair {
    int stage;
    cudaEvent_t a, b;
};
std::atomic<long long> g_launches{0};
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<EventPair> g_prof_live;
std::vector<cudaEvent_t> g_prof_pool;

cudaEvent_t pool_event()
{
    if (!g_prof_pool.empty()) {
        cudaEvent_t e = g_prof_pool.back();
        g_prof_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}
}  // namespace

void note_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

uint32_t resident_ctas_query(const void* kernel, int threads)
{
    struct Entry {
        const void* k;
        int threads, dev;
        uint32_t ctas;
    };
    static std::mutex mu;
    static std::vector<Entry> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    for (const Entry& e : cache)
        if (e.k == kernel && e.threads == threads && e.dev == dev) return e.ctas;
    int sms = 148, per = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, 0);
    const uint32_t r = (uint32_t)(sms * (per > 0 ? per : 1));
    cache.push_back(Entry{kernel, threads, dev, r});
    return r;
}

StageTimer::StageTimer(int st, cudaStream_t s) : stage(st), stream(s), slot(nullptr)
{
    std::lock_guard<std::mutex> lk(g_prof_mu);
    if (!g_prof_on) return;
    // launches captured into a CUDA graph are not timed (their events would only fire at replay)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
    EventPair* ep = new EventPair{st, pool_event(), pool_event()};
    cudaEventRecord(ep->a, s);
    slot = ep;
}

StageTimer::~StageTimer()
{
    if (!slot) return;
    EventPair* ep = static_cast<EventPair*>(slot);
    cudaEventRecord(ep->b, stream);
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_prof_live.push_back(*ep);
    delete ep;
}

GeomState geom_views(void* base, int P) { return carve_geom(base, P).g; }
size_t geom_bytes(int P) { return carve_geom(nullptr, P).total; }

ImageState image_views(void* base, int W, int H)
{
    Carver c{static_cast<char*>(base)};
    ImageState s;
    const size_t N = (size_t)W * H;
    const size_t T = (size_t)((W + kTileX - 1) / kTileX) * ((H + kTileY - 1) / kTileY);
    s.final_T = c.take<float>(N);
    s.n_contrib = c.take<uint32_t>(N);
    s.ranges = c.take<uint2>(T);
    s.long_list = c.take<uint32_t>(32 * T);
    s.long_ctr = c.take<uint32_t>(2 + 32);
    return s;
}
size_t image_bytes(int W, int H)
{
    Carver c{nullptr};
    const size_t N = (size_t)W * H;
    const size_t T = (size_t)((W + kTileX - 1) / kTileX) * ((H + kTileY - 1) / kTileY);
    c.take<float>(N);
    c.take<uint32_t>(N);
    c.take<uint2>(T);
    c.take<uint32_t>(32 * T);
    c.take<uint32_t>(2 + 32);
    return c.off;
}
BinState bin_views(void* base, long long K, int P) { return carve_bin(base, K, P).b; }
size_t bin_bytes(long long K, int P) { return carve_bin(nullptr, K, P).total; }
size_t bin_bytes_forward(long long K, int P) { return carve_bin(nullptr, K, P, false).total; }

}  // namespace fgs

using namespace fgs;

extern "C" {

const char* fgs_version(void) { return "filtergs_b200 0.1 (sm_100a)"; }

const char* fgs_status_string(int status)
{
    switch (status) {
    case FGS_OK: return "ok";
    case FGS_ERR_ARG: return "invalid argument";
    case FGS_ERR_CUDA: return "CUDA runtime error";
    case FGS_ERR_TIMEOUT: return "a bounded device-side wait timed out";
    case FGS_ERR_PREFILTERED: return "a Gaussian failed the near-plane test although prefiltered was set";
    case FGS_ERR_CAPACITY: return "preallocated capacity exceeded";
    case FGS_ERR_OVERFLOW: return "too many tile/Gaussian pairs (limit 2^30)";
    default: return "unknown status";
    }
}

size_t fgs_geom_bytes(int P) { return P < 0 ? 0 : geom_bytes(P); }
size_t fgs_image_bytes(int width, int height)
{
    return (width <= 0 || height <= 0) ? 0 : image_bytes(width, height);
}
size_t fgs_binning_bytes(long long num_rendered, int P)
{
    return (num_rendered < 0 || P < 0) ? 0 : bin_bytes(num_rendered, P);
}

int fgs_forward_preprocess(const fgs_raster_args* a, void* geom, void* image, int* radii, long long* num_rendered,
                           void* stream)
{
    PreParams p;
    int st = make_params(a, p);
    if (st) return st;
    if (!geom || !num_rendered || (!image)) return FGS_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned int* pin = pinned_words();
    if (!pin) return FGS_ERR_CUDA;
    // an error recorded by an earlier call on this stream surfaces now
    st = cuda_status(cudaStreamSynchronize(s));
    if (st) return st;
    if (pin[4]) {
        const int prev = err_code_from_bits(pin[4]);
        pin[4] = 0;
        return prev;
    }
    GeomCarve gc = carve_geom(geom, p.P);
    cudaMemsetAsync(gc.zero_begin, 0, gc.zero_bytes, s);
    {
        StageTimer t(FGS_STAGE_PREPROCESS, s);
        launch_preprocess(p, gc.g, radii, s);
    }
    {
        StageTimer t(FGS_STAGE_DEPTH_SORT, s);
        launch_depth_sort(gc.g, p.P, s);
    }
    if ((st = check_launch())) return st;
    unsigned long long* tot = reinterpret_cast<unsigned long long*>(pin + 8);
    cudaMemcpyAsync(tot, gc.g.total, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(pin, gc.g.err, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    st = cuda_status(cudaStreamSynchronize(s));
    if (st) return st;
    if (pin[0]) return err_code_from_bits(pin[0]);
    if (tot[0] >= (1ull << 30)) return FGS_ERR_OVERFLOW;
    *num_rendered = (long long)tot[0];
    return FGS_OK;
}

int fgs_forward_render(const fgs_raster_args* a, void* geom, void* image, void* binning, long long num_rendered,
                       const int* radii, float* out_color, int* out_point_id, float* out_point_weight_pixel,
                       float* out_point_weight, double* stats_host, int stats_len, void* stream)
{
    (void)radii;
    PreParams p;
    int st = make_params(a, p);
    if (st) return st;
    if (!geom || !image || (num_rendered > 0 && !binning)) return FGS_ERR_ARG;
    if (!out_color || !out_point_id || !out_point_weight_pixel || (p.P > 0 && !out_point_weight)) return FGS_ERR_ARG;
    if (num_rendered < 0 || num_rendered >= (1ll << 30)) return FGS_ERR_OVERFLOW;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int W = p.W, H = p.H;
    const int gx = (W + kTileX - 1) / kTileX, gy = (H + kTileY - 1) / kTileY;
    const int num_tiles = gx * gy;
    const int tbits = tile_bits_for(num_tiles);
    const long long K = num_rendered;
    GeomState g = geom_views(geom, p.P);
    ImageState im = image_views(image, W, H);
    BinCarve bc = carve_bin(binning, K, p.P);
    const bool stats = a->ogfs_enable_stats != 0;
    if (stats && stats_host && stats_len < 9 + 2 * FGS_STATS_SLOTS) return FGS_ERR_ARG;
    if (p.P > 0) cudaMemsetAsync(out_point_weight, 0, sizeof(float) * (size_t)p.P, s);
    if (K > 0) {
        cudaMemsetAsync(bc.b.status, 0, sizeof(uint32_t) * (bc.b.status_words + bc.b.scan_words), s);
        // V lives on the device (g.total[1]); every Gaussian beyond it has no pairs.
        {
            StageTimer t(FGS_STAGE_DUPLICATE, s);
            launch_duplicate(g, bc.b, (uint32_t)p.P, (uint32_t)K, W, H, tbits, s);
        }
        StageTimer t(FGS_STAGE_TILE_SORT, s);
        launch_tile_sort(g, bc.b, K, tbits, W, H, s);
    }
    {
        StageTimer t(FGS_STAGE_RANGES, s);
        launch_ranges(bc.b, im, K, num_tiles, s);
    }
    {
        StageTimer t_render(FGS_STAGE_RENDER_FWD, s);
        launch_render_fwd(W, H, im, bc.b, K, a->background, out_color, out_point_id, out_point_weight_pixel,
                          out_point_weight, stats && K > 0, g.err, s);
    }
    if ((st = check_launch())) return st;
    unsigned int* pin = pinned_words();
    if (stats && stats_host) {
        // rasterize_points.cu:138-177
        const int slots = FGS_STATS_SLOTS;
        const bool tiles_out = K > 0;
        const int need = 9 + 2 * slots + (tiles_out ? 2 * num_tiles : 0);
        if (stats_len < need) return FGS_ERR_ARG;
        double* dev = nullptr;
        const size_t nd = 3 + 11 + 2 * (size_t)num_tiles;
        if (K > 0) {
            // device scratch for the statistics: the tail of the pair-record buffer is free
            // only when it is large enough; otherwise use a temporary allocation.
            if (cudaMallocAsync(reinterpret_cast<void**>(&dev), nd * sizeof(double), s) != cudaSuccess) return FGS_ERR_CUDA;
            StageTimer t(FGS_STAGE_STATS, s);
            launch_kpc_stats(bc.b, im, num_tiles, kpc_used_thresh(), dev, s);
        }
        double* host = static_cast<double*>(std::malloc(nd * sizeof(double)));
        if (!host) return FGS_ERR_CUDA;
        memset(host, 0, nd * sizeof(double));
        if (K > 0) {
            cudaMemcpyAsync(host, dev, nd * sizeof(double), cudaMemcpyDeviceToHost, s);
            cudaFreeAsync(dev, s);
        }
        cudaMemcpyAsync(pin, g.err, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
        st = cuda_status(cudaStreamSynchronize(s));
        if (st) { std::free(host); return st; }
        for (int i = 0; i < stats_len; i++) stats_host[i] = 0.0;
        stats_host[0] = K > 0 ? host[0] / (double)num_tiles : 0.0;
        stats_host[1] = p.P > 0 ? (double)K / (double)p.P : 0.0;
        stats_host[2] = num_tiles > 0 ? (double)K / (double)num_tiles : 0.0;
        stats_host[3] = (double)K;
        stats_host[4] = (double)num_tiles;
        stats_host[5] = (double)p.P;
        stats_host[6] = K > 0 ? host[1] : 0.0;
        stats_host[7] = K > 0 ? host[2] : 0.0;
        stats_host[8] = K > 0 ? 11.0 : 0.0;
        if (K > 0) {
            const double edges[11] = {0.01f, 0.05f, 0.10f, 0.15f, 0.20f, 0.25f, 0.30f, 0.35f, 0.40f, 0.45f, 0.50f};
            for (int b = 0; b < 11; b++) {
                stats_host[9 + b] = edges[b];
                stats_host[9 + slots + b] = host[3 + b];
            }
            for (int t = 0; t < num_tiles; t++) {
                stats_host[9 + 2 * slots + t] = host[14 + t];
                stats_host[9 + 2 * slots + num_tiles + t] = host[14 + num_tiles + t];
            }
        }
        std::free(host);
        if (pin[0]) return err_code_from_bits(pin[0]);
    } else if (stats_host) {
        for (int i = 0; i < stats_len; i++) stats_host[i] = 0.0;
        stats_host[1] = p.P > 0 ? (double)K / (double)p.P : 0.0;
        stats_host[2] = num_tiles > 0 ? (double)K / (double)num_tiles : 0.0;
        stats_host[3] = (double)K;
        stats_host[4] = (double)num_tiles;
        stats_host[5] = (double)p.P;
        cudaMemcpyAsync(pin + 4, g.err, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    } else {
        cudaMemcpyAsync(pin + 4, g.err, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    }
    return FGS_OK;
}

int fgs_backward(const fgs_raster_args* a, const void* geom, const void* image, const void* binning,
                 long long num_rendered, const int* radii, const float* dL_dout_color, float* dL_dmeans2D,
                 float* dL_dconic, float* dL_dopacity, float* dL_dcolors, float* dL_dmeans3D, float* dL_dcov3D,
                 float* dL_dsh, float* dL_dscales, float* dL_drotations, int backward_mode, void* stream)
{
    PreParams p;
    int st = make_params(a, p, true);
    if (st) return st;
    if (backward_mode != FGS_BACKWARD_REF_COMPAT && backward_mode != FGS_BACKWARD_CONSISTENT) return FGS_ERR_ARG;
    if (!geom || !image || (num_rendered > 0 && !binning) || !dL_dout_color) return FGS_ERR_ARG;
    if (p.P > 0 && (!dL_dmeans2D || !dL_dconic || !dL_dopacity || !dL_dcolors || !dL_dmeans3D || !dL_dcov3D))
        return FGS_ERR_ARG;
    if (p.shs && !dL_dsh) return FGS_ERR_ARG;
    if (p.scales && (!dL_dscales || !dL_drotations)) return FGS_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (p.P == 0) return FGS_OK;
    GeomState g = geom_views(const_cast<void*>(geom), p.P);
    ImageState im = image_views(const_cast<void*>(image), p.W, p.H);
    BinState b = bin_views(const_cast<void*>(binning), num_rendered, p.P);
    (void)radii;  // the forward's visible list (radii > 0) is in geom
    cudaMemsetAsync(dL_dmeans2D, 0, sizeof(float) * 3 * (size_t)p.P, s);
    cudaMemsetAsync(dL_dconic, 0, sizeof(float) * 4 * (size_t)p.P, s);
    cudaMemsetAsync(dL_dopacity, 0, sizeof(float) * (size_t)p.P, s);
    cudaMemsetAsync(dL_dcolors, 0, sizeof(float) * 3 * (size_t)p.P, s);
    if (!p.scales) {
        if (dL_dscales) cudaMemsetAsync(dL_dscales, 0, sizeof(float) * 3 * (size_t)p.P, s);
        if (dL_drotations) cudaMemsetAsync(dL_drotations, 0, sizeof(float) * 4 * (size_t)p.P, s);
    }
    if (!p.shs && dL_dsh && a->M > 0) cudaMemsetAsync(dL_dsh, 0, sizeof(float) * 3 * (size_t)a->M * p.P, s);
    const int consistent = backward_mode == FGS_BACKWARD_CONSISTENT;
    if (num_rendered > 0) {
        StageTimer t(FGS_STAGE_RENDER_BWD, s);
        launch_render_bwd(p.W, p.H, im, b, a->background, dL_dout_color, consistent, g.err, s);
    }
    {
        StageTimer t_pb(FGS_STAGE_PREPROCESS_BWD, s);
        launch_preprocess_bwd(p, g, b.pgrad, dL_dmeans2D, dL_dconic, dL_dcolors, dL_dopacity, dL_dmeans3D,
                              dL_dcov3D, p.shs ? dL_dsh : nullptr, p.scales ? dL_dscales : nullptr,
                              p.scales ? dL_drotations : nullptr, consistent, s);
    }
    if ((st = check_launch())) return st;
    unsigned int* pin = pinned_words();
    cudaMemcpyAsync(pin + 4, g.err, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    return FGS_OK;
}

int fgs_check(const void* geom, void* stream)
{
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int st = cuda_status(cudaStreamSynchronize(s));
    if (st) return st;
    if ((st = check_launch())) return st;
    unsigned int* pin = pinned_words();
    if (!pin) return FGS_ERR_CUDA;
    if (pin[4]) {
        const int prev = err_code_from_bits(pin[4]);
        pin[4] = 0;
        return prev;
    }
    (void)geom;
    return FGS_OK;
}

int fgs_mark_visible(int P, const float* means3D, const float* viewmatrix, const float* projmatrix,
                     uint8_t* present, void* stream)
{
    (void)projmatrix;
    if (P < 0 || (P > 0 && (!means3D || !viewmatrix || !present))) return FGS_ERR_ARG;
    launch_mark_visible(P, means3D, viewmatrix, present, static_cast<cudaStream_t>(stream));
    return check_launch();
}

int fgs_compute_radius(int P, int height, int width, const float* means3D, const float* scales,
                       const float* rotations, const float* viewmatrix, const float* projmatrix, float tan_fovx,
                       float tan_fovy, float* radii, void* stream)
{
    if (P < 0 || (P > 0 && (!means3D || !scales || !rotations || !viewmatrix || !projmatrix || !radii)))
        return FGS_ERR_ARG;
    // forward.cu:580-581
    const float fy = height / (2.0f * tan_fovy);
    const float fx = width / (2.0f * tan_fovx);
    launch_compute_radius(0, P, means3D, scales, rotations, viewmatrix, projmatrix, fx, fy, tan_fovx, tan_fovy, radii,
                          static_cast<cudaStream_t>(stream));
    return check_launch();
}

int fgs_compute_radius_v2(int P, const float* means3D, const float* scales, const float* rotations,
                          const float* projmatrix, const float* viewmatrix, float focal_x, float focal_y,
                          float tan_fovx, float tan_fovy, float* radii, void* stream)
{
    if (P < 0 || (P > 0 && (!means3D || !scales || !rotations || !viewmatrix || !projmatrix || !radii)))
        return FGS_ERR_ARG;
    launch_compute_radius(1, P, means3D, scales, rotations, viewmatrix, projmatrix, focal_x, focal_y, tan_fovx,
                          tan_fovy, radii, static_cast<cudaStream_t>(stream));
    return check_launch();
}

int fgs_visibility_radius(int P, const float* means3D, const float* log_scales, const float* rotations,
                          const float* projmatrix, const float* viewmatrix, const int32_t* tree_node_index,
                          const int32_t* ancestor_path, int max_level, float focal_x, float focal_y, float tan_fovx,
                          float tan_fovy, float padding, float radius_max, float radius_filter_threshold,
                          uint8_t* mask, float* radius2d, float* depth, void* stream)
{
    if (P < 0 || max_level < 0) return FGS_ERR_ARG;
    if (P > 0 && (!means3D || !log_scales || !rotations || !projmatrix || !viewmatrix || !tree_node_index ||
                  (max_level > 0 && !ancestor_path) || !mask || !radius2d || !depth))
        return FGS_ERR_ARG;
    launch_visibility_radius(P, means3D, log_scales, rotations, projmatrix, viewmatrix, tree_node_index,
                             ancestor_path, max_level, focal_x, focal_y, tan_fovx, tan_fovy, padding, radius_max,
                             radius_filter_threshold, mask, radius2d, depth, static_cast<cudaStream_t>(stream));
    return check_launch();
}

int fgs_sorted_pairs(const void* geom, const void* binning, int P, long long num_rendered, uint64_t* keys,
                     uint32_t* vals, void* stream)
{
    if (!geom || num_rendered < 0 || (num_rendered > 0 && !binning)) return FGS_ERR_ARG;
    if (num_rendered == 0) return FGS_OK;
    GeomState g = geom_views(const_cast<void*>(geom), P);
    BinState b = bin_views(const_cast<void*>(binning), num_rendered, P);
    const uint32_t K = (uint32_t)num_rendered;
    sorted_keys_kernel<<<(K + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(b.tile_b, b.val_b, g.grec, K,
                                                                                      keys, vals);
    return check_launch();
}

int fgs_preprocess_outputs(const void* geom, int P, float* means2D, float* depths, float* conic_opacity, float* rgb,
                           uint32_t* tiles_touched, void* stream)
{
    if (!geom || P < 0) return FGS_ERR_ARG;
    if (P == 0) return FGS_OK;
    GeomState g = geom_views(const_cast<void*>(geom), P);
    pre_outputs_kernel<<<(P + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        g.grec, g.tiles, P, means2D, depths, conic_opacity, rgb, tiles_touched);
    return check_launch();
}

int fgs_image_outputs(const void* image, int width, int height, float* final_T, uint32_t* n_contrib,
                      uint32_t* ranges, void* stream)
{
    if (!image || width <= 0 || height <= 0) return FGS_ERR_ARG;
    ImageState im = image_views(const_cast<void*>(image), width, height);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t N = (size_t)width * height;
    const size_t T = (size_t)((width + kTileX - 1) / kTileX) * ((height + kTileY - 1) / kTileY);
    if (final_T) cudaMemcpyAsync(final_T, im.final_T, N * sizeof(float), cudaMemcpyDeviceToDevice, s);
    if (n_contrib) cudaMemcpyAsync(n_contrib, im.n_contrib, N * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    if (ranges) cudaMemcpyAsync(ranges, im.ranges, T * sizeof(uint2), cudaMemcpyDeviceToDevice, s);
    return check_launch();
}

int fgs_profile_enable(int on)
{
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_prof_on = on != 0;
    return FGS_OK;
}

int fgs_profile_read(double* ms, long long* calls, int reset)
{
    std::vector<EventPair> live;
    {
        std::lock_guard<std::mutex> lk(g_prof_mu);
        live = g_prof_live;
        if (reset) g_prof_live.clear();
    }
    for (int i = 0; i < FGS_NUM_STAGES; i++) {
        if (ms) ms[i] = 0.0;
        if (calls) calls[i] = 0;
    }
    int st = FGS_OK;
    for (const EventPair& e : live) {
        if (cudaEventSynchronize(e.b) != cudaSuccess) st = FGS_ERR_CUDA;
        float t = 0.f;
        if (cudaEventElapsedTime(&t, e.a, e.b) != cudaSuccess) st = FGS_ERR_CUDA;
        if (e.stage >= 0 && e.stage < FGS_NUM_STAGES) {
            if (ms) ms[e.stage] += t;
            if (calls) calls[e.stage] += 1;
        }
    }
    if (reset) {
        std::lock_guard<std::mutex> lk(g_prof_mu);
        for (const EventPair& e : live) {
            g_prof_pool.push_back(e.a);
            g_prof_pool.push_back(e.b);
        }
    }
    return st;
}

long long fgs_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int fgs_debug_lookback_fault(unsigned int skip_chunk, unsigned long long wait_ns)
{
    set_lookback_fault(skip_chunk, wait_ns);
    return FGS_OK;
}

int fgs_set_render_config(int fwd_ppt, int fwd_batch, int bwd_ppt, int bwd_batch)
{
    const RenderConfig cur = get_render_config();
    const RenderConfig c{fwd_ppt, fwd_batch, bwd_ppt, bwd_batch, cur.fwd_split, cur.fwd_band};
    if (!valid_render_config(c)) return FGS_ERR_ARG;
    set_render_config(c);
    return FGS_OK;
}

int fgs_set_render_split(int min_records, int band_shape)
{
    RenderConfig c = get_render_config();
    c.fwd_split = min_records;
    c.fwd_band = band_shape;
    if (!valid_render_config(c)) return FGS_ERR_ARG;
    set_render_config(c);
    return FGS_OK;
}

int fgs_get_render_split(int* cfg)
{
    if (!cfg) return FGS_ERR_ARG;
    const RenderConfig c = get_render_config();
    cfg[0] = c.fwd_split;
    cfg[1] = c.fwd_band;
    return FGS_OK;
}

int fgs_get_render_config(int* cfg)
{
    if (!cfg) return FGS_ERR_ARG;
    const RenderConfig c = get_render_config();
    cfg[0] = c.fwd_ppt; cfg[1] = c.fwd_batch; cfg[2] = c.bwd_ppt; cfg[3] = c.bwd_batch;
    return FGS_OK;
}

}  // extern "C"
