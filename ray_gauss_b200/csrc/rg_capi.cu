// C ABI of the engine (include/raygauss_b200.h): argument validation, scratch ownership and the
// stream-ordered launch sequences of the reference's forward and backward.
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <new>

#include "rg_common.cuh"
#include "rg_kernels.h"

struct rg_engine {
    int device = 0;
    int num_sms = 148;
    long long cap_n = 0;
    int cap_views = 0;
    long long cap_rays = 0;
    rg::GaussRec* rec = nullptr;     // Gaussian order
    float* aabb = nullptr;           // (N,6)
    int* scene_ord = nullptr;        // 6 ordered ints
    rg::BvhBuffers bvh;
    float4* rgb_leaf = nullptr;      // (views, N)
    float4* gacc_geo = nullptr;      // (N, 3)
    float4* gacc_rgb = nullptr;      // (N, views)
    rg::ViewTable* vt = nullptr;
    int* work_counter = nullptr;
    rg::DevStatus* st = nullptr;
    long long n_bbox = -1;           // N of the last rg_ellipsoids_bbox
    long long n_built = -1;          // N of the last rg_bvh_build
    int colors_views = 0;            // views in the colour table
    rg_gaussians g_bbox{};           // parameters of the last rg_ellipsoids_bbox (borrowed pointers)
    // hit-list record of the last forward (replayed by the backward of the same launch)
    unsigned* rec_arena = nullptr;
    unsigned long long* rec_top = nullptr;
    unsigned rec_cap = 0;            // arena words
    unsigned* rec_tile = nullptr;
    int rec_tiles = 0;
    bool rec_valid = false;          // the arena holds the record of the launch described below
    const rg_camera* rec_cams = nullptr;
    int rec_n_cams = 0;
    rg_settings rec_settings{};
    rg_tuning tuning{64, 0, 64, 1, 0};
    unsigned long long launches = 0;
    char last_err[256] = {0};
};

namespace {

int cuda_fail(rg_engine* e, cudaError_t err, const char* where) {
    if (err == cudaSuccess) return RG_OK;
    if (e) std::snprintf(e->last_err, sizeof(e->last_err), "%s: %s", where, cudaGetErrorString(err));
    return err == cudaErrorMemoryAllocation ? RG_ERR_OOM : RG_ERR_CUDA;
}

#define RG_CUDA(call, where)                            \
    do {                                                \
        cudaError_t _e = (call);                        \
        if (_e != cudaSuccess) return cuda_fail(e, _e, where); \
    } while (0)

template <typename T>
int grow(rg_engine* e, T*& p, size_t count) {
    if (p) cudaFree(p);
    p = nullptr;
    if (count == 0) return RG_OK;
    cudaError_t err = cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * count);
    return cuda_fail(e, err, "cudaMalloc");
}

int ensure_n(rg_engine* e, long long n) {
    if (n <= e->cap_n) return RG_OK;
    int rc;
    size_t N = (size_t)n;
    if ((rc = grow(e, e->rec, N))) return rc;
    if ((rc = grow(e, e->aabb, N * 6))) return rc;
    if ((rc = grow(e, e->bvh.keys_in, N))) return rc;
    if ((rc = grow(e, e->bvh.keys_out, N))) return rc;
    if ((rc = grow(e, e->bvh.vals_in, N))) return rc;
    if ((rc = grow(e, e->bvh.leaf_gid, N))) return rc;
    if ((rc = grow(e, e->bvh.rank, N))) return rc;
    if ((rc = grow(e, e->bvh.leaf_rec, N))) return rc;
    if ((rc = grow(e, e->bvh.leaf_is, N))) return rc;
    if ((rc = grow(e, e->bvh.leaf_ext, N * 2))) return rc;
    if ((rc = grow(e, e->bvh.leaf_lo, N))) return rc;
    if ((rc = grow(e, e->bvh.leaf_hi, N))) return rc;
    if ((rc = grow(e, e->bvh.nodes, N > 1 ? N - 1 : 1))) return rc;
    if ((rc = grow(e, e->bvh.depth, N > 1 ? N - 1 : 1))) return rc;
    if ((rc = grow(e, e->bvh.wide_cnt, N > 1 ? N - 1 : 1))) return rc;
    if ((rc = grow(e, e->bvh.wide_tab, N > 1 ? N - 1 : 1))) return rc;
    if ((rc = grow(e, e->bvh.slots, 2 * N))) return rc;
    if ((rc = grow(e, e->bvh.leaf_parent, N))) return rc;
    if ((rc = grow(e, e->bvh.node_parent, N > 1 ? N - 1 : 1))) return rc;
    if ((rc = grow(e, e->bvh.refit_cnt, N > 1 ? N - 1 : 1))) return rc;
    if ((rc = grow(e, e->gacc_geo, N * 3))) return rc;
    size_t tb = rg::sort_temp_bytes(n);
    unsigned char* tmp = nullptr;
    if ((rc = grow(e, tmp, tb))) return rc;
    e->bvh.sort_temp = tmp;
    e->bvh.sort_temp_bytes = tb;
    e->cap_n = n;
    // per-view tables depend on N
    if (e->cap_views > 0) {
        if ((rc = grow(e, e->rgb_leaf, N * (size_t)e->cap_views))) return rc;
        if ((rc = grow(e, e->gacc_rgb, N * (size_t)e->cap_views))) return rc;
    }
    e->n_built = -1;
    e->n_bbox = -1;
    return RG_OK;
}

int ensure_views(rg_engine* e, int views) {
    if (views <= e->cap_views) return RG_OK;
    int rc;
    size_t N = (size_t)(e->cap_n > 0 ? e->cap_n : 1);
    if ((rc = grow(e, e->rgb_leaf, N * (size_t)views))) return rc;
    if ((rc = grow(e, e->gacc_rgb, N * (size_t)views))) return rc;
    e->cap_views = views;
    e->colors_views = 0;
    return RG_OK;
}

constexpr long long kRecordWordsPerRay = 24;
constexpr long long kRecordBaseWords = 4096;

// Hit-list record storage for launches of up to n_rays rays (tiles <= rays).
int ensure_record(rg_engine* e, long long n_rays) {
    long long words = std::min(n_rays * kRecordWordsPerRay + kRecordBaseWords, (long long)0xfffffff0ll);
    long long tiles = std::min(n_rays, (long long)INT_MAX);
    int rc;
    if (!e->rec_top && (rc = grow(e, e->rec_top, 1))) return rc;
    if (words > (long long)e->rec_cap) {
        e->rec_cap = 0;
        if ((rc = grow(e, e->rec_arena, (size_t)words))) return rc;
        e->rec_cap = (unsigned)words;
    }
    if (tiles > e->rec_tiles) {
        e->rec_tiles = 0;
        if ((rc = grow(e, e->rec_tile, (size_t)tiles))) return rc;
        e->rec_tiles = (int)tiles;
    }
    e->rec_valid = false;
    return RG_OK;
}

int check_gaussians(const rg_gaussians* g) {
    if (!g || !g->positions || !g->scales || !g->quaternions || !g->densities || !g->color_features) return RG_ERR_INVALID_ARG;
    if (g->n <= 0 || g->n > rg::kMaxGaussians) return RG_ERR_INVALID_ARG;   // wide-node slot ids: 2^25
    if (g->sh_degree < 0 || g->sh_degree > 3) return RG_ERR_INVALID_ARG;
    if (g->num_sph_gauss < 0 || g->num_sph_gauss > RG_MAX_SG) return RG_ERR_INVALID_ARG;
    if (g->num_sph_gauss > 0 && (!g->sph_gauss_features || !g->bandwidth_sharpness || !g->lobe_axis))
        return RG_ERR_INVALID_ARG;
    if (g->storage != RG_STORAGE_F32 && g->storage != RG_STORAGE_BF16) return RG_ERR_INVALID_ARG;
    if (reinterpret_cast<uintptr_t>(g->quaternions) % 16 != 0) return RG_ERR_INVALID_ARG;
    return RG_OK;
}

int check_views(const rg_camera* cams, int n_cams) {
    if (!cams || n_cams <= 0 || n_cams > rg::kMaxViews) return RG_ERR_INVALID_ARG;
    return RG_OK;
}

// The per-(view, leaf) colour and gradient tables are indexed with 32-bit offsets.
int check_table(long long n, int n_cams) {
    return (long long)n_cams * n >= (long long)INT_MAX ? RG_ERR_INVALID_ARG : RG_OK;
}

cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Makes the engine's device current for one entry point and restores the caller's current device
// when the entry point returns, so a call on an engine of another device leaves the caller's (and
// torch's) notion of the current device unchanged.
struct DeviceScope {
    int prev = -1;
    bool switched = false;
    int enter(rg_engine* e) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != e->device) {
            RG_CUDA(cudaSetDevice(e->device), "cudaSetDevice");
            switched = prev >= 0;
        }
        return RG_OK;
    }
    ~DeviceScope() {
        if (switched) cudaSetDevice(prev);
    }
};

// The fast kernels run only without random sample offsets (launch_render picks the same way).
int kernel_mode(const rg_settings* s) {
    return (s->mode == RG_MODE_FAST && s->rnd_sample == 0) ? RG_MODE_FAST : RG_MODE_PARITY;
}

int render_grid(rg_engine* e, bool bwd, int mode) {
    int per_sm = e->tuning.blocks_per_sm;
    int occ = rg::render_occupancy(bwd, mode, e->tuning.list_capacity);
    if (per_sm <= 0 || per_sm > occ) per_sm = occ > 0 ? occ : 1;
    return e->num_sms * per_sm;
}

int fill_args(rg_engine* e, const rg_camera* cams, const rg_settings* s, rg::RenderArgs& a) {
    std::memset(&a, 0, sizeof(a));
    a.cams = cams;
    a.views = e->vt;
    a.rec = e->bvh.leaf_rec;
    a.is_rec = e->bvh.leaf_is;
    a.ext = e->bvh.leaf_ext;
    a.rgb = e->rgb_leaf;
    a.wide_tab = e->bvh.wide_tab;
    a.slots = e->bvh.slots;
    a.n_leaves = (int)e->n_built;
    a.scene_ord = e->scene_ord;
    a.white_bg = s->white_background;
    a.jitter = s->jitter;
    a.rnd_sample = s->rnd_sample;
    a.max_prim_slice = s->max_prim_slice > 0 ? s->max_prim_slice : 1024;
    a.iteration = s->iteration;
    a.chunk_slabs = e->tuning.chunk_slabs;
    a.diag = e->tuning.diagnostics;
    a.work_counter = e->work_counter;
    a.st = e->st;
    return RG_OK;
}

}  // namespace

void rg::export_status(const DevStatus& h, rg_status* out) {
    out->hit_pairs = h.hit_pairs;
    out->slabs = h.slabs;
    out->slab_cap_exceeded = h.slab_cap_exceeded;
    out->list_passes = h.list_passes;
    out->chunk_splits = h.chunk_splits;
    out->stack_overflows = h.stack_overflows;
    out->watchdog_trips = h.watchdog_trips;
    out->nonfinite_inputs = h.nonfinite_inputs;
    out->traversals = h.traversals;
    out->node_visits = h.node_visits;
    out->leaf_tests = h.leaf_tests;
    out->list_entries = h.list_entries;
    out->slab_steps = h.slab_steps;
    out->entry_slabs = h.entry_slabs;
    out->replayed_chunks = h.replayed_chunks;
    out->record_overflows = h.record_overflows;
    out->record_words = 0;
}

extern "C" {

int rg_abi_version(void) { return RG_ABI_VERSION; }

const char* rg_error_string(int code) {
    switch (code) {
        case RG_OK: return "ok";
        case RG_ERR_INVALID_ARG: return "invalid argument";
        case RG_ERR_CUDA: return "CUDA error";
        case RG_ERR_OOM: return "out of device memory";
        case RG_ERR_STATE: return "call order violated (bbox/bvh/colour missing or stale)";
        case RG_ERR_CAPACITY: return "request exceeds the entry point's fixed capacity";
        default: return "unknown error";
    }
}

const char* rg_last_cuda_error(const rg_engine* e) { return e ? e->last_err : ""; }
uint64_t rg_kernel_launches(const rg_engine* e) { return e ? e->launches : 0; }

int rg_create(rg_engine** out, int device) {
    if (!out) return RG_ERR_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return RG_ERR_INVALID_ARG;
    rg_engine* e = new (std::nothrow) rg_engine();
    if (!e) return RG_ERR_OOM;
    e->device = device;
    DeviceScope dev_scope;
    int rc = dev_scope.enter(e);
    if (rc) { delete e; return rc; }
    cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, device);
    if ((rc = grow(e, e->scene_ord, 6)) || (rc = grow(e, e->vt, 1)) || (rc = grow(e, e->work_counter, 4)) ||
        (rc = grow(e, e->st, 1)) || (rc = grow(e, e->bvh.root_box, 6))) {
        rg_destroy(e);
        return rc;
    }
    cudaMemset(e->st, 0, sizeof(rg::DevStatus));
    *out = e;
    return RG_OK;
}

int rg_destroy(rg_engine* e) {
    if (!e) return RG_OK;
    DeviceScope dev_scope;
    dev_scope.enter(e);
    void* ptrs[] = {e->rec, e->aabb, e->scene_ord, e->bvh.keys_in, e->bvh.keys_out, e->bvh.vals_in, e->bvh.leaf_gid,
                    e->bvh.rank, e->bvh.leaf_rec, e->bvh.leaf_is, e->bvh.leaf_ext, e->bvh.leaf_lo, e->bvh.leaf_hi, e->bvh.nodes,
                    e->bvh.depth, e->bvh.wide_cnt, e->bvh.wide_tab, e->bvh.slots,
                    e->bvh.leaf_parent, e->bvh.node_parent, e->bvh.refit_cnt, e->bvh.root_box, e->bvh.sort_temp,
                    e->rgb_leaf, e->gacc_geo, e->gacc_rgb, e->vt, e->work_counter, e->st, e->rec_arena,
                    e->rec_top, e->rec_tile};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete e;
    return RG_OK;
}

int rg_reserve(rg_engine* e, int64_t n, int32_t n_views, int64_t n_rays) {
    if (!e || n < 0 || n_views < 0 || n_views > rg::kMaxViews) return RG_ERR_INVALID_ARG;
    DeviceScope dev_scope;
    int rc = dev_scope.enter(e);
    if (rc) return rc;
    if (n > 0 && (rc = ensure_n(e, n))) return rc;
    if (n_views > 0 && (rc = ensure_views(e, n_views))) return rc;
    if (n_rays > e->cap_rays) {
        if ((rc = ensure_record(e, n_rays))) return rc;
        e->cap_rays = n_rays;
    }
    return RG_OK;
}

int rg_set_tuning(rg_engine* e, const rg_tuning* t) {
    if (!e || !t) return RG_ERR_INVALID_ARG;
    if (t->chunk_slabs < 0 || t->chunk_slabs > rg::kMaxChunk) return RG_ERR_INVALID_ARG;
    if (t->list_capacity != 0 && t->list_capacity != 64 && t->list_capacity != 128)
        return RG_ERR_INVALID_ARG;
    if (t->blocks_per_sm < 0) return RG_ERR_INVALID_ARG;
    if (t->record_hits < -1 || t->record_hits > 1) return RG_ERR_INVALID_ARG;
    if (t->diagnostics < 0 || t->diagnostics > 1) return RG_ERR_INVALID_ARG;
    if (t->chunk_slabs) e->tuning.chunk_slabs = t->chunk_slabs;
    if (t->list_capacity) e->tuning.list_capacity = t->list_capacity;
    if (t->record_hits) e->tuning.record_hits = t->record_hits;
    e->tuning.blocks_per_sm = t->blocks_per_sm;
    e->tuning.diagnostics = t->diagnostics;
    e->rec_valid = false;
    return RG_OK;
}

int rg_get_tuning(const rg_engine* e, rg_tuning* t) {
    if (!e || !t) return RG_ERR_INVALID_ARG;
    *t = e->tuning;
    return RG_OK;
}

int rg_ellipsoids_bbox(rg_engine* e, const rg_gaussians* g, float* aabb_out, float* scene_box_out, void* stream) {
    if (!e) return RG_ERR_INVALID_ARG;
    int rc = check_gaussians(g);
    if (rc) return rc;
    DeviceScope dev_scope;
    if ((rc = dev_scope.enter(e))) return rc;
    if ((rc = ensure_n(e, g->n))) return rc;
    RG_CUDA(rg::launch_prepass(g, e->rec, e->aabb, e->scene_ord, e->st, S(stream)), "prepass");
    e->launches += 2;
    if (aabb_out) {
        RG_CUDA(cudaMemcpyAsync(aabb_out, e->aabb, sizeof(float) * 6 * (size_t)g->n, cudaMemcpyDeviceToDevice, S(stream)),
                "copy aabb");
    }
    if (scene_box_out) {
        RG_CUDA(rg::launch_scene_out(e->scene_ord, scene_box_out, S(stream)), "scene box");
        e->launches += 1;
    }
    e->n_bbox = g->n;
    e->g_bbox = *g;
    e->rec_valid = false;
    return RG_OK;
}

// Build and refit read the scales and quaternions of the last rg_ellipsoids_bbox call (kept as
// borrowed pointers) for the leaf extension records used by the adjoint.
int rg_bvh_build(rg_engine* e, void* stream) {
    if (!e || e->n_bbox <= 0) return RG_ERR_STATE;
    const rg_gaussians* g = &e->g_bbox;
    DeviceScope dev_scope;
    int rc = dev_scope.enter(e);
    if (rc) return rc;
    RG_CUDA(rg::launch_build(e->n_bbox, e->aabb, e->scene_ord, e->rec, g, e->bvh, S(stream)), "bvh build");
    e->launches += 6;
    e->n_built = e->n_bbox;
    e->colors_views = 0;
    e->rec_valid = false;
    return RG_OK;
}

int rg_bvh_refit(rg_engine* e, void* stream) {
    if (!e || e->n_bbox <= 0 || e->n_built != e->n_bbox) return RG_ERR_STATE;
    const rg_gaussians* g = &e->g_bbox;
    DeviceScope dev_scope;
    int rc = dev_scope.enter(e);
    if (rc) return rc;
    RG_CUDA(rg::launch_refit(e->n_built, e->aabb, e->rec, g, e->bvh, S(stream)), "bvh refit");
    e->launches += 2;
    e->colors_views = 0;
    e->rec_valid = false;
    return RG_OK;
}


int rg_forward_sh(rg_engine* e, const rg_gaussians* g, const rg_camera* cams, int32_t n_cams, float* rgb_out,
                  void* stream) {
    if (!e) return RG_ERR_INVALID_ARG;
    int rc = check_gaussians(g);
    if (rc || (rc = check_views(cams, n_cams))) return rc;
    if (e->n_built != g->n) return RG_ERR_STATE;
    if ((rc = check_table(g->n, n_cams))) return rc;
    DeviceScope dev_scope;
    if ((rc = dev_scope.enter(e)) || (rc = ensure_views(e, n_cams))) return rc;
    RG_CUDA(rg::launch_color_forward(g, cams, n_cams, e->bvh.rank, e->rgb_leaf, rgb_out, S(stream)), "forward_sh");
    e->launches += 1;
    e->colors_views = n_cams;
    e->rec_valid = false;
    return RG_OK;
}

int rg_launch_forward(rg_engine* e, const rg_camera* cams, int32_t n_cams, const rg_settings* s, float* ray_colors,
                      float* final_T, void* stream) {
    if (!e || !s || !ray_colors) return RG_ERR_INVALID_ARG;
    int rc = check_views(cams, n_cams);
    if (rc) return rc;
    if (e->n_built <= 0 || e->colors_views < n_cams) return RG_ERR_STATE;
    DeviceScope dev_scope;
    if ((rc = dev_scope.enter(e))) return rc;
    RG_CUDA(rg::launch_setup_views(cams, n_cams, e->vt, e->work_counter, S(stream)), "setup views");
    rg::RenderArgs a;
    fill_args(e, cams, s, a);
    a.ray_colors = ray_colors;
    a.final_T = final_T;
    const bool record = e->tuning.record_hits == 1 && e->rec_arena != nullptr;
    e->rec_valid = false;
    if (record) {
        RG_CUDA(cudaMemsetAsync(e->rec_top, 0, sizeof(unsigned long long), S(stream)), "reset record");
        a.rec_arena = e->rec_arena;
        a.rec_top = e->rec_top;
        a.rec_cap = e->rec_cap;
        a.rec_tile = e->rec_tile;
        a.rec_tiles = e->rec_tiles;
    }
    int grid = render_grid(e, false, kernel_mode(s));
    RG_CUDA(rg::launch_render(false, s->mode, e->tuning.list_capacity, grid, a, S(stream)), "render forward");
    e->launches += 2;
    if (record) {
        e->rec_valid = true;
        e->rec_cams = cams;
        e->rec_n_cams = n_cams;
        e->rec_settings = *s;
    }
    return RG_OK;
}

int rg_launch_inference(rg_engine* e, const rg_camera* cams, int32_t n_cams, const rg_settings* s,
                        float* ray_colors, int32_t* gaussians_per_ray, void* stream) {
    if (!e || !s || !ray_colors) return RG_ERR_INVALID_ARG;
    int rc = check_views(cams, n_cams);
    if (rc) return rc;
    if (e->n_built <= 0 || e->colors_views < n_cams) return RG_ERR_STATE;
    DeviceScope dev_scope;
    if ((rc = dev_scope.enter(e))) return rc;
    // the inference programs sample without jitter or random offsets
    rg_settings si = *s;
    si.jitter = 0;
    si.rnd_sample = 0;
    RG_CUDA(rg::launch_setup_views(cams, n_cams, e->vt, e->work_counter, S(stream)), "setup views");
    rg::RenderArgs a;
    fill_args(e, cams, &si, a);
    a.ray_colors = ray_colors;
    a.infer = 1;
    a.counts = gaussians_per_ray;
    int grid = render_grid(e, false, kernel_mode(&si));
    RG_CUDA(rg::launch_render(false, si.mode, e->tuning.list_capacity, grid, a, S(stream)), "render inference");
    e->launches += 2;
    return RG_OK;
}

int rg_render_inference(rg_engine* e, const rg_gaussians* g, const rg_camera* cams, int32_t n_cams,
                        const rg_settings* s, int32_t refit, float* ray_colors, int32_t* gaussians_per_ray,
                        float* rgb_out, void* stream) {
    int rc = rg_ellipsoids_bbox(e, g, nullptr, nullptr, stream);
    if (rc) return rc;
    if (refit && e->n_built == g->n) rc = rg_bvh_refit(e, stream);
    else rc = rg_bvh_build(e, stream);
    if (rc) return rc;
    if ((rc = rg_forward_sh(e, g, cams, n_cams, rgb_out, stream))) return rc;
    return rg_launch_inference(e, cams, n_cams, s, ray_colors, gaussians_per_ray, stream);
}

int rg_launch_backward(rg_engine* e, const rg_camera* cams, int32_t n_cams, const rg_settings* s,
                       const float* ray_colors, const float* dloss_dray_colors, void* stream) {
    if (!e || !s || !ray_colors || !dloss_dray_colors) return RG_ERR_INVALID_ARG;
    int rc = check_views(cams, n_cams);
    if (rc) return rc;
    if (e->n_built <= 0 || e->colors_views < n_cams) return RG_ERR_STATE;
    DeviceScope dev_scope;
    if ((rc = dev_scope.enter(e))) return rc;
    size_t N = (size_t)e->n_built;
    RG_CUDA(cudaMemsetAsync(e->gacc_geo, 0, sizeof(float4) * 3 * N, S(stream)), "zero grads");
    RG_CUDA(cudaMemsetAsync(e->gacc_rgb, 0, sizeof(float4) * N * (size_t)n_cams, S(stream)), "zero grads");
    RG_CUDA(rg::launch_setup_views(cams, n_cams, e->vt, e->work_counter, S(stream)), "setup views");
    rg::RenderArgs a;
    fill_args(e, cams, s, a);
    a.ray_colors_in = ray_colors;
    a.dL = dloss_dray_colors;
    a.gacc_geo = e->gacc_geo;
    a.gacc_rgb = e->gacc_rgb;
    a.n_views = n_cams;
    // Replay the last forward's hit lists when nothing changed the engine state since that forward
    // (bbox, BVH, colour and tuning calls invalidate the record) and this backward uses the same
    // camera table, view count and settings: the chunk sequence is then the forward's.
    if (e->rec_valid && e->tuning.record_hits == 1 && e->rec_cams == cams && e->rec_n_cams == n_cams &&
        std::memcmp(&e->rec_settings, s, sizeof(rg_settings)) == 0) {
        a.rec_arena = e->rec_arena;
        a.rec_cap = e->rec_cap;
        a.rec_tile = e->rec_tile;
        a.rec_tiles = e->rec_tiles;
        a.replay = 1;
    }
    int grid = render_grid(e, true, kernel_mode(s));
    RG_CUDA(rg::launch_render(true, s->mode, e->tuning.list_capacity, grid, a, S(stream)), "render backward");
    RG_CUDA(rg::launch_moment_grads((int)N, e->bvh.leaf_rec, e->bvh.leaf_ext, e->gacc_geo, S(stream)), "moments");
    e->launches += 3;
    return RG_OK;
}

int rg_backward_sh(rg_engine* e, const rg_gaussians* g, const rg_camera* cams, int32_t n_cams, const rg_settings* s,
                   const rg_gradients* out, void* stream) {
    if (!e || !s || !out) return RG_ERR_INVALID_ARG;
    int rc = check_gaussians(g);
    if (rc || (rc = check_views(cams, n_cams))) return rc;
    if (!out->positions || !out->scales || !out->quaternions || !out->densities || !out->color_features)
        return RG_ERR_INVALID_ARG;
    if (g->num_sph_gauss > 0 && (!out->sph_gauss_features || !out->bandwidth_sharpness || !out->lobe_axis))
        return RG_ERR_INVALID_ARG;
    if (e->n_built != g->n) return RG_ERR_STATE;
    DeviceScope dev_scope;
    if ((rc = dev_scope.enter(e))) return rc;
    RG_CUDA(rg::launch_color_backward(g, cams, n_cams, e->bvh.rank, e->gacc_geo, e->gacc_rgb, s->sh_quirk, out,
                                      S(stream)),
            "backward_sh");
    e->launches += 1;
    return RG_OK;
}

int rg_render_forward(rg_engine* e, const rg_gaussians* g, const rg_camera* cams, int32_t n_cams,
                      const rg_settings* s, int32_t refit, float* ray_colors, float* final_T, float* rgb_out,
                      void* stream) {
    int rc = rg_ellipsoids_bbox(e, g, nullptr, nullptr, stream);
    if (rc) return rc;
    if (refit && e->n_built == g->n) rc = rg_bvh_refit(e, stream);
    else rc = rg_bvh_build(e, stream);
    if (rc) return rc;
    if ((rc = rg_forward_sh(e, g, cams, n_cams, rgb_out, stream))) return rc;
    return rg_launch_forward(e, cams, n_cams, s, ray_colors, final_T, stream);
}

int rg_render_backward(rg_engine* e, const rg_gaussians* g, const rg_camera* cams, int32_t n_cams,
                       const rg_settings* s, const float* ray_colors, const float* dloss_dray_colors,
                       const rg_gradients* out, void* stream) {
    int rc = rg_launch_backward(e, cams, n_cams, s, ray_colors, dloss_dray_colors, stream);
    if (rc) return rc;
    return rg_backward_sh(e, g, cams, n_cams, s, out, stream);
}

int rg_leaf_order(rg_engine* e, int32_t* leaf_gid_out, void* stream) {
    if (!e || !leaf_gid_out) return RG_ERR_INVALID_ARG;
    if (e->n_built <= 0) return RG_ERR_STATE;
    DeviceScope dev_scope;
    int rc = dev_scope.enter(e);
    if (rc) return rc;
    RG_CUDA(cudaMemcpyAsync(leaf_gid_out, e->bvh.leaf_gid, sizeof(int32_t) * (size_t)e->n_built,
                            cudaMemcpyDeviceToDevice, S(stream)),
            "copy leaf order");
    return RG_OK;
}

int rg_get_status(rg_engine* e, rg_status* out, int32_t reset, void* stream) {
    if (!e || !out) return RG_ERR_INVALID_ARG;
    DeviceScope dev_scope;
    int rc = dev_scope.enter(e);
    if (rc) return rc;
    RG_CUDA(cudaStreamSynchronize(S(stream)), "sync");
    rg::DevStatus h;
    RG_CUDA(cudaMemcpy(&h, e->st, sizeof(h), cudaMemcpyDeviceToHost), "read status");
    rg::export_status(h, out);
    if (e->rec_top) {
        unsigned long long w = 0;
        RG_CUDA(cudaMemcpy(&w, e->rec_top, sizeof(w), cudaMemcpyDeviceToHost), "read record size");
        out->record_words = w;
    }
    if (reset) RG_CUDA(cudaMemset(e->st, 0, sizeof(rg::DevStatus)), "reset status");
    return RG_OK;
}

}  // extern "C"
