// Internal launcher declarations shared by the engine's translation units.
#pragma once

#include "rg_common.cuh"

namespace rg {

struct BvhBuffers {
    unsigned long long* keys_in = nullptr;
    unsigned long long* keys_out = nullptr;
    int* vals_in = nullptr;
    int* leaf_gid = nullptr;      // leaf -> Gaussian
    int* rank = nullptr;          // Gaussian -> leaf
    LeafRec* leaf_rec = nullptr;  // leaf-ordered records
    LeafIS* leaf_is = nullptr;    // leaf-ordered reference conics (parity intersection test)
    float4* leaf_ext = nullptr;   // leaf-ordered {scale.xyz, 0}, {quaternion}
    float4* leaf_lo = nullptr;
    float4* leaf_hi = nullptr;
    Node* nodes = nullptr;
    int* depth = nullptr;         // per binary node: depth below the root
    int* wide_cnt = nullptr;      // per binary node: wide children (0 unless a wide node)
    int2* wide_tab = nullptr;     // per binary node: {first slot, slot count} of its wide node
    WideSlot* slots = nullptr;    // wide-node children (at most 2n slots)
    int* leaf_parent = nullptr;
    int* node_parent = nullptr;
    unsigned* refit_cnt = nullptr;
    float* root_box = nullptr;
    void* sort_temp = nullptr;
    size_t sort_temp_bytes = 0;
};

struct RenderArgs {
    const rg_camera* cams;
    const ViewTable* views;
    const LeafRec* rec;
    const LeafIS* is_rec;
    const float4* ext;
    const float4* rgb;            // (n_views, n_leaves) leaf order
    const int2* wide_tab;         // wide node of binary node i: {first slot, slot count} (root: entry 0)
    const WideSlot* slots;        // wide-node children
    int n_leaves;
    const int* scene_ord;
    int white_bg, jitter, rnd_sample, max_prim_slice;
    unsigned iteration;
    int chunk_slabs;
    // forward outputs
    float* ray_colors;
    float* final_T;
    // backward inputs / outputs
    const float* ray_colors_in;
    const float* dL;
    float4* gacc_geo;             // (n_leaves, 3): ddens, dpos.xyz, dscale.xyz, dquat.xyzw, pad (the
                                  // render kernel accumulates moments there; launch_moment_grads converts)
    float4* gacc_rgb;             // (n_leaves, n_views): {drgb.xyz, 0}, a leaf's views contiguous
    int n_views = 0;              // views of the launch (the gacc_rgb row length)
    int* work_counter;
    DevStatus* st;
    // hit-list record: the forward appends each warp chunk's leaf ids to the arena (chunk records
    // linked per tile); the backward replays them instead of traversing.  Null arena: no record.
    unsigned* rec_arena;
    unsigned long long* rec_top;  // words used (reset before every recording forward)
    unsigned rec_cap;             // arena words
    unsigned* rec_tile;           // first chunk record of each tile (kNoRecord: none)
    int rec_tiles;                // entries of rec_tile
    int replay;                   // backward: replay the records
    // inference launch (the reference's cuda_test programs): slab query without the box-exit clip,
    // conic-space sample stepping (parity arithmetic), optional Gaussians per ray
    int infer;
    int* counts;
    int diag;                  // 1: count the fine-grained traversal/list statistics (rg_tuning.diagnostics)
};

cudaError_t launch_prepass(const rg_gaussians* g, GaussRec* rec, float* aabb, int* scene_ord, DevStatus* st,
                           cudaStream_t s);
cudaError_t launch_scene_out(const int* scene_ord, float* out, cudaStream_t s);
size_t sort_temp_bytes(long long n);
cudaError_t launch_build(long long n, const float* aabb, const int* scene_ord, const GaussRec* rec,
                         const rg_gaussians* g, BvhBuffers& b, cudaStream_t s);
cudaError_t launch_refit(long long n, const float* aabb, const GaussRec* rec, const rg_gaussians* g,
                         BvhBuffers& b, cudaStream_t s);

cudaError_t launch_moment_grads(int n, const LeafRec* rec, const float4* ext, float4* acc, cudaStream_t s);
cudaError_t launch_setup_views(const rg_camera* cams, int n_cams, ViewTable* vt, int* work_counter,
                               cudaStream_t s);
cudaError_t launch_color_forward(const rg_gaussians* g, const rg_camera* cams, int n_cams, const int* rank,
                                 float4* rgb_leaf, float* rgb_out, cudaStream_t s);
cudaError_t launch_color_backward(const rg_gaussians* g, const rg_camera* cams, int n_cams, const int* rank,
                                  const float4* gacc_geo, const float4* gacc_rgb, int sh_quirk,
                                  const rg_gradients* out, cudaStream_t s);

// mode: RG_MODE_PARITY / RG_MODE_FAST; cap: 64/128
cudaError_t launch_render(bool backward, int mode, int cap, int grid, const RenderArgs& a, cudaStream_t s);
int render_occupancy(bool backward, int mode, int cap);

// Copies a device status block read back to the host into the public struct (record_words is left
// to the caller).
void export_status(const DevStatus& h, rg_status* out);

}  // namespace rg
