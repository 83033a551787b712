// Internal host-side declarations shared by the .cu translation units.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/filtergs_b200.h"

namespace fgs {

struct PairRecord;

// Per-call forward parameters after validation (device pointers).
struct PreParams {
    int P, D, M, W, H;
    const float* means;       // [P,3]
    const float* scales;      // [P,3] or null
    const float* rots;        // [P,4] or null
    const float* opac;        // [P]
    const float* shs;         // [P,M,3] or null
    const float* cov3D;       // [P,6] or null (precomputed)
    const float* colors;      // [P,3] or null (precomputed)
    const float* view;        // [16]
    const float* proj;        // [16]
    const float* campos;      // [3]
    float scale_mod, tanx, tany, fx, fy;
    int prefiltered, use_filter;
    float eps_scale, eps_max, energy_floor, ratio_min;
    float filter3d;
    int aligned;              // means/scales/rots/opac 16-byte aligned: stage with float4 loads
    // Optional structure-of-arrays copy of the per-Gaussian inputs the preprocess reads
    // ([3][P] float4: {mean, opacity}, {scale, 0}, rotation), one coalesced float4 load
    // each; null: the reference's AoS tensors above are read instead.
    const float4* packed;
};
// Writes the packed copy (PreParams::packed) of P Gaussians' means, opacities,
// scales and rotations (the last two planes only when scales/rots are given).
void launch_pack_gaussians(int P, const float* means, const float* opac, const float* scales, const float* rots,
                           float4* packed, cudaStream_t s);

// Geometry workspace views (per-Gaussian state kept from forward to backward).
struct GeomState {
    PairRecord* grec;          // [P] render record per Gaussian
    int* radii;                // [P] internal radii (when the caller passes none)
    uint32_t* tiles;           // [P] tiles touched
    uint8_t* clamped;          // [P] SH clamp bits
    uint32_t* depth_key;       // [V] depth bits of the visible Gaussians (index order, then sort ping)
    uint32_t* sort_ids_a;      // [V] depth-sorted ids (ping)
    uint32_t* sort_ids_b;      // [V] visible ids in index order, then depth-sorted (pong)
    uint32_t* sort_keys_b;     // [P]
    uint32_t* pair_off;        // [V] first emitted pair of the visible Gaussian of depth rank j (aliases
                               //     sort_keys_b, dead once the depth sort is done)
    int2* erow;                // [P] emission index of tile (tx, ty) = erow.x + ty * erow.y + tx
    uint32_t* hist;            // [8][256] radix histograms: 4 depth passes + up to 4 tile passes
    uint32_t* status;          // lookback status words, depth passes
    uint32_t* chunk_counts;    // [2][ceil(P/256)] preprocess chunk counts: visible (scanned in place), pairs
    uint32_t* cand_ids;        // [P] Gaussians that passed the preprocess tile bound (count in counters[12])
    uint32_t* counters;        // [16] chunk counters: 0-3 depth passes, 4-7 tile passes, 8 pairs, 12 candidates
    unsigned long long* total; // [4]: 0 = K (pairs), 1 = V (visible count)
    unsigned int* err;         // error bit set
    size_t status_words;
};
GeomState geom_views(void* base, int P);
size_t geom_bytes(int P);

struct ImageState {
    float* final_T;     // [N]
    uint32_t* n_contrib; // [N]
    uint2* ranges;      // [tiles]
    uint32_t* long_list; // [32][tiles] tiles rendered in bands, binned by log2(records) (render.cu)
    uint32_t* long_ctr;  // [34] 0: long tiles, 1: band queue, 2 + b: tiles in bin b
};
ImageState image_views(void* base, int W, int H);
size_t image_bytes(int W, int H);

struct BinState {
    uint32_t* tile_a;   // [K]
    uint32_t* tile_b;   // [K]
    uint32_t* val_a;    // [K]
    uint32_t* val_b;    // [K] final point list
    PairRecord* rec;    // [K] (c.w: the pair's emission index)
    float* pgrad;       // [K][9] per-pair gradients at the emission index (null in forward-only layouts)
    uint32_t* status;   // lookback words, tile passes
    uint32_t* scan_status; // lookback words of the fused scan
    float* kv_sum;      // [K] (stats)
    uint32_t* kv_cnt;   // [K] (stats)
    size_t status_words, scan_words;
};
BinState bin_views(void* base, long long K, int P);
size_t bin_bytes(long long K, int P);
size_t bin_bytes_forward(long long K, int P);  // without the per-pair gradients
// Key bits of the tile index (the reference's getHigherMsb, rasterizer_impl.cu:78-93).
int tile_bits_for(int num_tiles);

// ---------------------------------------------------------------- launchers
// Resident CTAs of a kernel on this device (persistent grids never exceed it).
// Cached per (kernel, block size, device): kernels of the same signature have
// their own entries.
uint32_t resident_ctas_query(const void* kernel, int threads);
template <typename Kern>
inline uint32_t resident_ctas(Kern k, int threads)
{
    return resident_ctas_query(reinterpret_cast<const void*>(k), threads);
}

void launch_preprocess(const PreParams& p, const GeomState& g, int* radii, cudaStream_t s);
void launch_depth_sort(const GeomState& g, int P, cudaStream_t s);
// Test hook: chunk skip_chunk of the first depth-sort pass never publishes its
// look-back counts, and that pass waits at most wait_ns (0: the default limit).
void set_lookback_fault(uint32_t skip_chunk, unsigned long long wait_ns);
void launch_duplicate(const GeomState& g, const BinState& b, uint32_t V, uint32_t K, int W, int H, int tile_bits,
                      cudaStream_t s);
int sort_chunk_size();
// K is the pair count, or the capacity when n_dev (device-side count) is given.
void launch_tile_sort(const GeomState& g, const BinState& b, long long K, int tile_bits, int W, int H, cudaStream_t s,
                      const unsigned long long* n_dev = nullptr);
void launch_ranges(const BinState& b, const ImageState& im, long long K, int num_tiles, cudaStream_t s,
                   const unsigned long long* n_dev = nullptr);
// K: the pair count (or capacity) of b, for the statistics' zeroing when long tiles are split.
void launch_render_fwd(int W, int H, const ImageState& im, const BinState& b, long long K, const float* bg,
                       float* out_color, int* point_id, float* pw_pixel, float* point_weight, bool stats,
                       unsigned* err, cudaStream_t s);
void launch_render_bwd(int W, int H, const ImageState& im, const BinState& b, const float* bg,
                       const float* dL_dpix, int consistent, unsigned* err, cudaStream_t s);
// Densification statistics a training step keeps per Gaussian (null pointers: off).
struct DensifyStats {
    float* grad_sum;   // += |dL/dmean2D[:2]| per view that sees the Gaussian
    int* count;        // += 1 per such view
    uint8_t* flag;     // = 1 (visible in this step)
};
// Per-Gaussian backward of one view.  Screen-space gradients come from the
// per-pair gradients (pgrad, at the emission index), summed per Gaussian in
// emission order: dmean2D / dconic / dcolor / dopac are the dense screen-space
// outputs (rows of visible Gaussians written; the caller zeroes them), the rest are
// written densely.  The Gaussians the forward found visible (radii > 0) receive
// gradients.
void launch_preprocess_bwd(const PreParams& p, const GeomState& g, const float* pgrad, float* dmean2D,
                           float* dconic, float* dcolor, float* dopac, float* dmean3D, float* dcov3D, float* dsh,
                           float* dscale, float* drot, int consistent, cudaStream_t s);
// Batched backward (backward.cu): per-view screen-space gradient gathers (pgrad holds
// `rows` pair rows: the view's pair capacity), each also setting the view's bit
// (vis_bit) in vis[idx] for every Gaussian it sees, then one pass per Gaussian over
// all views.
struct FoldView {
    PreParams p;              // the view's preprocess parameters (camera, shared inputs)
    float* dm_geo;            // [P,3] the view's geometric dL/dmean3D between the two passes (with SH)
    const float* dmean2D;     // [P,3] the view's screen-space gradients (gather outputs)
    const float* dconic;      // [P,4]
    const float* dopac;       // [P]
    const float* dcolor;      // [P,3]
    const uint8_t* clamped;   // [P] SH clamp bits of the view's forward
};
void launch_pair_grad_gather(const GeomState& g, const float* pgrad, long long rows, float* dmean2D, float* dconic,
                             float* dcolor, float* dopac, uint32_t* vis, uint32_t vis_bit, int P, cudaStream_t s);
// views: device table of nviews descriptors; shared: any one of them (its inputs shared by all views);
// list [P] and count: scratch for the Gaussians some view saw.  The caller zeroes dmean3D, dopac,
// dsh, dscale and drot first (rows no view saw stay zero).
void launch_fold_bwd(const FoldView* views, int nviews, int P, const uint32_t* vis, uint32_t* list,
                     unsigned long long* count, int consistent, bool sh, float* dmean3D, float* dopac, float* dsh,
                     float* dscale, float* drot, const DensifyStats* dens, const FoldView& shared, cudaStream_t s);
void launch_kpc_stats(const BinState& b, const ImageState& im, int num_tiles, float used_thresh, double* dev_out,
                      cudaStream_t s);

// radius / visibility helpers
void launch_compute_radius(int variant, int P, const float* means, const float* scales, const float* rots,
                           const float* view, const float* proj, float fx, float fy, float tanx, float tany,
                           float* radius, cudaStream_t s);
void launch_mark_visible(int P, const float* means, const float* view, uint8_t* present, cudaStream_t s);
void launch_visibility_radius(int P, const float* means, const float* lscales, const float* rots,
                              const float* proj, const float* view, const int32_t* node_index,
                              const int32_t* ancestors, int L, float fx, float fy, float tanx, float tany,
                              float padding, float radius_max, float radius_filter, uint8_t* mask, float* radius2d,
                              float* depth, cudaStream_t s);

// Validate a fgs_raster_args and derive the kernel parameters (opacities may
// be absent in backward).
int make_params(const fgs_raster_args* a, PreParams& p, bool backward = false);

// ---------------------------------------------------------------- render views
// Everything one tile needs, for the plain launch (one view, one tile per CTA)
// and the persistent multi-view launch (CTAs pop (view, tile) work items).
struct TileArgs {
    const uint2* ranges;
    const PairRecord* recs;
    int W, H;
    const float* bg;
    // forward outputs
    float* out_color;
    float* final_T;
    uint32_t* n_contrib;
    int* out_point_id;
    float* out_pw_pixel;
    float* out_point_weight;
    float* kv_sum;
    uint32_t* kv_cnt;
    // backward input / output
    const float* dL_dpix;
    float* pgrad;  // [K][9] per-pair gradients, indexed by the record's emission index
};

// Persistent multi-view compositing over the tiles of `nviews` views; begin[v]
// is the first work item of view v (begin[nviews] == total_tiles); queue is a
// device counter (zeroed here).
// long_list: [32 * total_tiles] scratch, long_ctr: [34] scratch (bands of long tiles; statistics must be off).
void launch_render_fwd_multi(const TileArgs* views, const uint32_t* begin, int nviews, uint32_t total_tiles,
                             uint32_t* queue, uint32_t* long_list, uint32_t* long_ctr, unsigned* err, cudaStream_t s);
void launch_render_bwd_multi(const TileArgs* views, const uint32_t* begin, int nviews, uint32_t total_tiles,
                             uint32_t* queue, int consistent, unsigned* err, cudaStream_t s);

// Render kernel shape: pixels per thread {1,2,4} and records per shared-memory batch {64,128,256}.
struct RenderConfig {
    int fwd_ppt, fwd_batch, bwd_ppt, bwd_batch;
    int fwd_split;  // forward: tiles with at least this many records are rendered in bands (0: never)
    int fwd_band;   // band shape: 0 = 16x2, 1 = 8x4, 2 = 4x4, 3 = 4x2 pixels per warp
};
bool valid_render_config(const RenderConfig& c);
void set_render_config(const RenderConfig& c);
RenderConfig get_render_config();

// LoD selection and gather (lod.cu)
void launch_compact(const uint8_t* mask, uint32_t n, int64_t* out, unsigned long long* count, uint32_t* scratch,
                    unsigned* err, cudaStream_t s);
void launch_gather(const int64_t* index, long long N, const float* xyz, const float* scaling, const float* rotation,
                   const float* opacity, const float* colors, const float* shs, int sh_floats, float* o_xyz,
                   float* o_scaling, float* o_rotation, float* o_opacity, float* o_colors, float* o_shs,
                   cudaStream_t s);
void launch_gather_activate(const int64_t* index, const unsigned long long* count, long long N_cap, const float* xyz,
                            const float* log_scale, const float* rot, const float* opac_raw, const float* dc,
                            const float* rest, int deg, int rest_coeffs, const float* campos, float* o_xyz,
                            float* o_scale, float* o_rot, float* o_opac, float* o_rgb, cudaStream_t s);
void launch_radius_raw(int P, const float* means, const float* lscales, const float* rots, const float* view,
                       const float* proj, float fx, float fy, float tanx, float tany, float* radius, cudaStream_t s);
size_t log_cut_scratch_words(int P, int nroots, int max_child, int levels);
void launch_log_cut(int P, const int32_t* roots, int nroots, const int32_t* node_index, const int32_t* tree,
                    int max_child, const float* radius, float min_res, int levels, int32_t* out, uint32_t* scratch,
                    unsigned* err, cudaStream_t s);
void launch_cull(const int32_t* in, const uint32_t* n_in, uint32_t cap, const float* radius, const float* opac_raw,
                 float min_px, int64_t* out, unsigned long long* n_out, uint32_t* scratch, unsigned* err,
                 cudaStream_t s);
void launch_ancestor_path(int P, const int32_t* parent, const int32_t* depth, int L, int32_t* out, unsigned* err,
                          cudaStream_t s);

// Kernel-launch accounting (fgs_launch_count) and per-stage event timing.
void note_launches(int n);
struct StageTimer {
    StageTimer(int stage, cudaStream_t s);
    ~StageTimer();
    int stage;
    cudaStream_t stream;
    void* slot;
};

}  // namespace fgs
