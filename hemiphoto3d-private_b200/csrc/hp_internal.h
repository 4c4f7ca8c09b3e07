// Internal types shared by the engine's host code and kernels.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/hpmvs.h"

namespace hp {

// Pixel tile one CTA covers: TILE_W x TILE_H pixels, 256 threads (the FP16
// kernels also run TILE_W x 4 tiles with 128 threads).  In a
// red-black half-pass each thread owns one pixel of the active color (a warp
// covers one 64-pixel row segment); the full-map kernels give each thread the
// two horizontally adjacent pixels of its pair.
constexpr int TILE_W = 64;
constexpr int TILE_H = 8;
constexpr int CTA_THREADS = 256;

struct FilterStage;

// Per-view descriptor, resident in device memory for the duration of a solve.
// Hypotheses are packed (depth, nx, ny, nz) so one 16-byte load fetches a
// pixel's plane; cost is a separate float plane.
struct ViewDesc {
    const float* ref;                 // FP32 reference image, row pitch ref_pitch floats
    const __half* ref16;              // FP16 reference image, row pitch ref16_pitch halves
    cudaTextureObject_t src_tex[HP_MAX_SOURCES];    // FP32 sources, linear filter
    cudaTextureObject_t src_tex16[HP_MAX_SOURCES];  // FP16 sources, linear filter
    const uint2* src_quad[HP_MAX_SOURCES];          // FP16 sources, block-tiled software-sampler quads
    float kinv[9];
    alignas(16) float ab[HP_MAX_SOURCES][12];  // A (9), b (3) per source; 16-byte aligned rows
    float4* hyp;                      // H*W
    float* cost;                      // H*W
    int ref_pitch, ref16_pitch;
    int W, H, S;
    int tiles_x, tiles_y;
    int tile_h;                       // rows of a tile (a CTA has tile_h warps, one per row)
    float dmin, dmax;
    uint32_t seed_lo, seed_hi, view_id;
    int iterations;
    // Persistent schedule only: per-tile completed-stage flags (tiles_x *
    // tiles_y, -1 before stage 0) and, when set, the device maps the final
    // stage unpacks into (depth H*W, normal H*W*3 camera frame, cost H*W).
    int* done;
    float* out_depth;
    float* out_normal;
    float* out_cost;
    float* out_conf;  // may be null: confidence 1 - cost / 2 per pixel
    // Geometric-consistency stage after the last half-pass (null: none).
    const FilterStage* filter;
    // SfM seeding (null when the job has none): per pixel the index of the
    // seed whose plane replaces the random initial one, -1 for none.
    const int* seed_map;
    const hp_seed* seeds;
};

// Solver constants for one launch.
// SolveConsts::soft_mask bit 31 (tests only): no corner-test shortcuts in the
// FP16 cost, every window through the per-tap checked form.
constexpr unsigned SOFT_MASK_CHECKED = 1u << 31;

struct SolveConsts {
    int radius, stride, top_k, refine_steps;
    float iter_decay, step_decay;
    unsigned soft_mask;  // FP16 path: sources sampled in software (bit per source); SOFT_MASK_CHECKED
    int tile_h;          // rows of a CTA's tile (TILE_W x tile_h pixels, tile_h warps): 8, or 4 (FP16 path)
    int staging;         // FP16 path: quad loads in flight per window row, 4 or 8
};

// A batch launch covers the tiles of several views: view k owns flattened
// tile indices [tile_prefix[k], tile_prefix[k+1]).
struct BatchList {
    const ViewDesc* views;      // all views of the solve
    const int* active;          // indices of the views in this launch
    const int* tile_prefix;     // n_active + 1 entries
    int n_active;
    int total_tiles;
};

// Persistent launch.  A view's work is a sequence of stages, each covering
// all its tiles: stage 0 initialises the hypotheses and scores them, stage
// 1 + 2*it + color is red-black half-pass (it, color), and stage
// 2*iterations + 1, present when the view has output maps, unpacks its state
// into them.  Tickets number (view, stage, tile) stage-major - every tile of
// every view's stage k precedes any of stage k + 1 - and entry e of the
// schedule is the run of tickets [entry_ticket[e], entry_ticket[e + 1]) of
// view entry_info[e].x at stage entry_info[e].y.  A CTA takes tickets from an
// atomic counter and, before running a stage k >= 1 tile, waits until that
// tile and its four neighbour tiles have finished stage k - 1 (the half-pass
// reads one pixel of halo).  Every ticket waited on is smaller than the
// waiter's, so it is held by a CTA that is already running: progress needs no
// co-residency guarantee.  The waiting thread's acquire load followed by the
// CTA barrier orders the neighbours' earlier stores before every thread's
// later plain loads (PTX memory model: release/acquire at gpu scope, then
// bar.sync), so the stage bodies read state with ordinary loads.  Waits are
// bounded by wait_limit_ns; a wait that
// runs out records SCHED_TIMEOUT in status[0] and its ticket in status[2] and
// raises the abort flag, and every CTA then stops taking tickets.  The abort
// flag is status[1] unless the launcher gives another word: the server shares
// one between its launches, so the launches queued behind one that gave up
// stop at their first claim (SCHED_ABORTED) instead of each waiting out the
// limit on the state the first left unfinished.
constexpr int SCHED_OK = 0;
constexpr int SCHED_TIMEOUT = 1;
constexpr int SCHED_ABORTED = 2;
struct Schedule {
    const ViewDesc* views;
    const int* entry_ticket;      // n_entries + 1 (the last is the ticket total)
    const int2* entry_info;       // (view, stage)
    int n_entries;
    int total;
    unsigned* counter;            // next ticket
    int* status;                  // [0] SCHED_* code, [1] abort flag, [2] ticket whose wait ran out
    int* abort;                   // abort flag (null: status + 1; the launchers fill it in)
    unsigned long long wait_limit_ns;
    int stall_view, stall_tile;   // this tile never reports completion (bounded-wait test); -1 = none
    SolveConsts sc;
    // Filter stages (null when the schedule has none): tickets below
    // main_total are the solve proper; every one of them must have finished
    // (main_done counts them) before a filter stage starts.
    unsigned* main_done;
    int main_total;
};

// Geometric-consistency check of one reference view against its solved
// sources (the rule of geometric_consistency_filter_kernel,
// src/dense_recon/patchmatch_mvs.cu:668-781).  Each source's transform is
// composed in FP64 on the host from the two cameras and cast once: a
// reference pixel (x, y) at depth d lands at source pixel p.xy / p.z with
// p = d A (x, y, 1) + b (A = K_s R_rel K_ref^-1, b = K_s t_rel: the
// homography setup's coefficients) at source-camera depth
// z = d m.(x, y, 1) + cz (m = the third row of R_rel K_ref^-1, cz = t_rel.z),
// and a camera-frame normal n maps to R_rel n in the source's frame, so the
// world-frame normal test is (R_rel n_ref) . n_src.
struct FilterSource {
    float A[9];
    float b[3];
    float m[3];
    float cz;
    float Rn[9];
    int view;  // fused stage: index of the source's ViewDesc in the solve
};
struct FilterStage {
    FilterSource src[HP_MAX_SOURCES];
    int n;                // sources checked (views of the same size that were solved too)
    int min_consistent;   // fewer agreeing sources: depth 0 and cost 2 (confidence 0)
    float depth_tol;      // relative depth tolerance
    float normal_cos;     // minimum cosine between the two world-frame normals
    // Persistent schedule only: the filtered view before this one in the
    // sequential order (-1 for the first) and a count of this view's tiles
    // that finished the stage; a view's filter starts after its predecessor's
    // has finished everywhere, so each view sees the earlier views filtered
    // and the later ones not, as the reference's view-by-view loop does.
    int prev;
    int* tiles_done;
};
// External maps (hp_geometric_filter): the same check on caller maps.
struct FilterMaps {
    FilterStage f;
    const float* src_depth[HP_MAX_SOURCES];
    const float* src_normal[HP_MAX_SOURCES];  // AoS, camera frame
    int W, H;
};

// Depth-map fusion (hp_fuse_depth_maps): one view's device maps and its
// camera cast to FP32 (kinv is the FP64 inverse of K, then cast).
struct FuseView {
    const float* depth;
    const float* normal;
    const float* conf;  // may be null
    const float* gray;  // may be null
    float K[9], kinv[9], R[9], t[3];
    int W, H;
    int nb_begin, nb_count;  // this view's slice of FuseArgs::neighbors
};
struct FuseArgs {
    const FuseView* views;  // device, n_views
    const int* neighbors;   // device
    const int* view_block;  // device, n_views + 1: first CTA of each view's pixels
    int n_views;
    int min_views;
    float min_conf, max_depth_rel, max_reproj_sq, min_normal_cos;
};
constexpr int FUSE_THREADS = 256;  // pixels per CTA of the fusion kernels

}  // namespace hp

// Kernel launchers (defined in the .cu files), all on the given stream.
namespace hp {
// Initialisation of a batch whose views have tiles of tile_h rows.
cudaError_t launch_init(const BatchList& bl, int tile_h, cudaStream_t st);
cudaError_t launch_cost_f32(const BatchList& bl, const SolveConsts& sc, cudaStream_t st);
cudaError_t launch_propagate_f32(const BatchList& bl, const SolveConsts& sc, int iteration, int color,
                                 cudaStream_t st);
cudaError_t launch_cost_f16(const BatchList& bl, const SolveConsts& sc, cudaStream_t st);
cudaError_t launch_persistent_f32(const Schedule& s, int grid, cudaStream_t st);
cudaError_t launch_persistent_f16(const Schedule& s, int grid, cudaStream_t st);
// Resident CTAs per SM of the persistent kernel for (radius, stride).
cudaError_t persistent_occupancy_f32(int radius, int stride, int* blocks_per_sm);
cudaError_t persistent_occupancy_f16(const SolveConsts& sc, int* blocks_per_sm);
cudaError_t launch_propagate_f16(const BatchList& bl, const SolveConsts& sc, int iteration, int color,
                                 cudaStream_t st);
// FP16 plane -> block-tiled software-sampler quad plane (see hpx::QuadPlane).
cudaError_t launch_quads(const __half* src16, int pitch16, int W, int H, uint2* quads, cudaStream_t st);
// SfM seed index map of a W x H view: per pixel the last-listed of the (device) seeds whose
// (2 radius + 1)^2 square covers it, -1 for none.
cudaError_t launch_seed_map(const hp_seed* seeds, int num_seeds, int radius, int W, int H, int* map,
                            cudaStream_t st);
cudaError_t launch_unpack(const ViewDesc* views_host_copy, int view, float* depth, float* normal, float* cost,
                          float* conf, cudaStream_t st);
cudaError_t launch_pack(const ViewDesc* views_host_copy, int view, const float* depth, const float* normal,
                        const float* cost, cudaStream_t st);
// The filter stage of view `view` (views: device descriptors; tiles: its tile
// count), in place on its packed state; with write_out it also writes the
// view's out_* maps (the final unpack, fused).
cudaError_t launch_filter_view(const ViewDesc* views, int view, int tiles, int tile_h, bool write_out,
                               cudaStream_t st);
// The same check on caller maps: depth and confidence updated in place.
cudaError_t launch_filter_maps(const FilterMaps& a, float* depth, const float* normal, float* conf,
                               cudaStream_t st);
cudaError_t launch_to_f32(const void* src, int dtype, int W, int H, float* dst, int dst_pitch, __half* dst16,
                          int dst16_pitch, cudaStream_t st);
// Fusion: per-CTA counts of emitted points, their exclusive prefix (and the
// total), then the points written at their offsets (index < capacity only).
cudaError_t launch_fuse_count(const FuseArgs& a, int blocks, int* block_counts, cudaStream_t st);
cudaError_t launch_fuse_scan(const int* block_counts, int blocks, long long* block_offsets, long long* total,
                             cudaStream_t st);
cudaError_t launch_fuse_write(const FuseArgs& a, int blocks, const long long* block_offsets, float* positions,
                              float* normals, float* colors, long long capacity, cudaStream_t st);
}  // namespace hp
