// Allocation-free forward render: rg_render_forward_noalloc.
//
// Some callers cannot call cudaMalloc: code that runs while a CUDA graph is being captured in a
// mode that forbids allocation, hosts that hand the library a fixed device-memory budget up front,
// or plugins loaded into a process whose allocator must not be touched.  This entry point runs
// the same pre-pass, LBVH build, colour pass and forward launch as rg_render_forward without an
// engine and without allocating: all of its scratch lives in one file-scope device array of
// kNoAllocScratchBytes (about 10 MB), which every GPU that loads this library holds until the
// process exits.  The caller still passes the Gaussians, cameras and output buffers.
//
// Limits: at most kNoAllocMaxGaussians (16384) Gaussians and kNoAllocMaxViews (4) views per call;
// larger requests return RG_ERR_CAPACITY before touching the device.  Every call shares the one
// array and leaves the previous call's contents in it; each call clears what must start at zero
// (scene box, refit counters, work counter, status block) on its stream, so calls that overlap on
// the GPU (different streams, or different host threads without ordering) race on the array.
// rg_noalloc_get_status reads the device counters of the latest call on the current device
// (non-finite inputs, watchdog trips, stack overflows and the rest of rg_status), allocating
// nothing either: it synchronises the given stream and copies the array's status block.
// The first call on a device looks up the array's device address with cudaGetSymbolAddress and
// caches it; make that first call before any stream capture.
#include <cstring>
#include <mutex>

#include "rg_common.cuh"
#include "rg_kernels.h"

namespace {

constexpr long long kNoAllocMaxGaussians = 16384;
constexpr int kNoAllocMaxViews = 4;
constexpr size_t kSortReserve = 1u << 20;  // radix-sort temporary storage (checked at set-up)

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Byte offsets of every scratch buffer inside the array.
struct NoAllocLayout {
    size_t rec, aabb, scene, keys_in, keys_out, vals_in, leaf_gid, rank, leaf_rec, leaf_is, leaf_ext, leaf_lo,
        leaf_hi, nodes, depth, wide_cnt, wide_tab, slots, leaf_parent, node_parent, refit_cnt, root_box, rgb_leaf, vt,
        work, status, sort, total;
};

constexpr NoAllocLayout make_layout() {
    const size_t N = (size_t)kNoAllocMaxGaussians;
    NoAllocLayout L{};
    size_t o = 0;
    auto take = [&o](size_t bytes) {
        size_t at = o;
        o += align256(bytes);
        return at;
    };
    L.rec = take(sizeof(rg::GaussRec) * N);
    L.aabb = take(sizeof(float) * 6 * N);
    L.scene = take(sizeof(int) * 6);
    L.keys_in = take(sizeof(unsigned long long) * N);
    L.keys_out = take(sizeof(unsigned long long) * N);
    L.vals_in = take(sizeof(int) * N);
    L.leaf_gid = take(sizeof(int) * N);
    L.rank = take(sizeof(int) * N);
    L.leaf_rec = take(sizeof(rg::LeafRec) * N);
    L.leaf_is = take(sizeof(rg::LeafIS) * N);
    L.leaf_ext = take(sizeof(float4) * 2 * N);
    L.leaf_lo = take(sizeof(float4) * N);
    L.leaf_hi = take(sizeof(float4) * N);
    L.nodes = take(sizeof(rg::Node) * N);
    L.depth = take(sizeof(int) * N);
    L.wide_cnt = take(sizeof(int) * N);
    L.wide_tab = take(sizeof(int2) * N);
    L.slots = take(sizeof(rg::WideSlot) * 2 * N);
    L.leaf_parent = take(sizeof(int) * N);
    L.node_parent = take(sizeof(int) * N);
    L.refit_cnt = take(sizeof(unsigned) * N);
    L.root_box = take(sizeof(float) * 6);
    L.rgb_leaf = take(sizeof(float4) * N * kNoAllocMaxViews);
    L.vt = take(sizeof(rg::ViewTable));
    L.work = take(sizeof(int) * 4);
    L.status = take(sizeof(rg::DevStatus));
    L.sort = take(kSortReserve);
    L.total = o;
    return L;
}

constexpr NoAllocLayout kLayout = make_layout();
constexpr size_t kNoAllocScratchBytes = kLayout.total;

}  // namespace

// The scratch array (one per device that loads the library).
static __device__ __align__(256) unsigned char g_rg_noalloc_scratch[kNoAllocScratchBytes];

namespace {

constexpr int kMaxDevices = 64;

struct DeviceSetup {
    bool ready = false;
    unsigned char* base = nullptr;  // device address of g_rg_noalloc_scratch on this device
    int num_sms = 0;
};

std::mutex g_setup_mutex;
DeviceSetup g_setup[kMaxDevices];

// Once per device, with that device current: resolve the array's device address (the host-side
// symbol is only a stand-in and must never be passed to a kernel) and check the sort reserve.
int setup_device(int dev, DeviceSetup** out) {
    if (dev < 0 || dev >= kMaxDevices) return RG_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceSetup& d = g_setup[dev];
    if (!d.ready) {
        void* ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, g_rg_noalloc_scratch) != cudaSuccess || ptr == nullptr) return RG_ERR_CUDA;
        if (rg::sort_temp_bytes(kNoAllocMaxGaussians) > kSortReserve) return RG_ERR_CAPACITY;
        if (cudaDeviceGetAttribute(&d.num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return RG_ERR_CUDA;
        d.base = static_cast<unsigned char*>(ptr);
        d.ready = true;
    }
    *out = &d;
    return RG_OK;
}

template <typename T>
T* at(unsigned char* base, size_t off) {
    return reinterpret_cast<T*>(base + off);
}

}  // namespace

extern "C" RG_API int rg_render_forward_noalloc(const rg_gaussians* g, const rg_camera* cams, int32_t n_cams,
                                                const rg_settings* s, float* ray_colors, float* final_T,
                                                void* stream) {
    if (!g || !s || !ray_colors || !cams || n_cams <= 0) return RG_ERR_INVALID_ARG;
    if (!g->positions || !g->scales || !g->quaternions || !g->densities || !g->color_features)
        return RG_ERR_INVALID_ARG;
    if (g->n <= 0 || g->sh_degree < 0 || g->sh_degree > 3 || g->num_sph_gauss < 0 || g->num_sph_gauss > RG_MAX_SG)
        return RG_ERR_INVALID_ARG;
    if (g->num_sph_gauss > 0 && (!g->sph_gauss_features || !g->bandwidth_sharpness || !g->lobe_axis))
        return RG_ERR_INVALID_ARG;
    if (g->storage != RG_STORAGE_F32 && g->storage != RG_STORAGE_BF16) return RG_ERR_INVALID_ARG;
    if (reinterpret_cast<uintptr_t>(g->quaternions) % 16 != 0) return RG_ERR_INVALID_ARG;
    if (g->n > kNoAllocMaxGaussians || n_cams > kNoAllocMaxViews) return RG_ERR_CAPACITY;

    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return RG_ERR_CUDA;
    DeviceSetup* d = nullptr;
    int rc = setup_device(dev, &d);
    if (rc) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    unsigned char* b = d->base;
    const long long n = g->n;

    rg::GaussRec* rec = at<rg::GaussRec>(b, kLayout.rec);
    float* aabb = at<float>(b, kLayout.aabb);
    int* scene_ord = at<int>(b, kLayout.scene);
    rg::DevStatus* status = at<rg::DevStatus>(b, kLayout.status);
    rg::BvhBuffers bvh;
    bvh.keys_in = at<unsigned long long>(b, kLayout.keys_in);
    bvh.keys_out = at<unsigned long long>(b, kLayout.keys_out);
    bvh.vals_in = at<int>(b, kLayout.vals_in);
    bvh.leaf_gid = at<int>(b, kLayout.leaf_gid);
    bvh.rank = at<int>(b, kLayout.rank);
    bvh.leaf_rec = at<rg::LeafRec>(b, kLayout.leaf_rec);
    bvh.leaf_is = at<rg::LeafIS>(b, kLayout.leaf_is);
    bvh.leaf_ext = at<float4>(b, kLayout.leaf_ext);
    bvh.leaf_lo = at<float4>(b, kLayout.leaf_lo);
    bvh.leaf_hi = at<float4>(b, kLayout.leaf_hi);
    bvh.nodes = at<rg::Node>(b, kLayout.nodes);
    bvh.depth = at<int>(b, kLayout.depth);
    bvh.wide_cnt = at<int>(b, kLayout.wide_cnt);
    bvh.wide_tab = at<int2>(b, kLayout.wide_tab);
    bvh.slots = at<rg::WideSlot>(b, kLayout.slots);
    bvh.leaf_parent = at<int>(b, kLayout.leaf_parent);
    bvh.node_parent = at<int>(b, kLayout.node_parent);
    bvh.refit_cnt = at<unsigned>(b, kLayout.refit_cnt);
    bvh.root_box = at<float>(b, kLayout.root_box);
    bvh.sort_temp = at<unsigned char>(b, kLayout.sort);
    bvh.sort_temp_bytes = kSortReserve;
    float4* rgb_leaf = at<float4>(b, kLayout.rgb_leaf);
    rg::ViewTable* vt = at<rg::ViewTable>(b, kLayout.vt);
    int* work = at<int>(b, kLayout.work);

    // the status block is the only buffer no kernel below re-initialises
    if (cudaMemsetAsync(status, 0, sizeof(rg::DevStatus), st) != cudaSuccess) return RG_ERR_CUDA;
    if (rg::launch_prepass(g, rec, aabb, scene_ord, status, st) != cudaSuccess) return RG_ERR_CUDA;
    if (rg::launch_build(n, aabb, scene_ord, rec, g, bvh, st) != cudaSuccess) return RG_ERR_CUDA;
    if (rg::launch_color_forward(g, cams, n_cams, bvh.rank, rgb_leaf, nullptr, st) != cudaSuccess) return RG_ERR_CUDA;
    if (rg::launch_setup_views(cams, n_cams, vt, work, st) != cudaSuccess) return RG_ERR_CUDA;

    rg::RenderArgs a;
    std::memset(&a, 0, sizeof(a));
    a.cams = cams;
    a.views = vt;
    a.rec = bvh.leaf_rec;
    a.is_rec = bvh.leaf_is;
    a.ext = bvh.leaf_ext;
    a.rgb = rgb_leaf;
    a.wide_tab = bvh.wide_tab;
    a.slots = bvh.slots;
    a.n_leaves = (int)n;
    a.scene_ord = scene_ord;
    a.white_bg = s->white_background;
    a.jitter = s->jitter;
    a.rnd_sample = s->rnd_sample;
    a.max_prim_slice = s->max_prim_slice > 0 ? s->max_prim_slice : 1024;
    a.iteration = s->iteration;
    a.chunk_slabs = 64;  // the engine's default tuning: 64-slab chunks, list capacity 64
    a.work_counter = work;
    a.st = status;
    a.ray_colors = ray_colors;
    a.final_T = final_T;
    const int cap = 64;
    // random sample offsets run the parity kernel in either mode (launch_render picks it): size the
    // grid for the kernel that runs
    const int run_mode = (s->mode == RG_MODE_FAST && s->rnd_sample == 0) ? RG_MODE_FAST : RG_MODE_PARITY;
    int per_sm = rg::render_occupancy(false, run_mode, cap);
    int grid = d->num_sms * (per_sm > 0 ? per_sm : 1);
    if (rg::launch_render(false, s->mode, cap, grid, a, st) != cudaSuccess) return RG_ERR_CUDA;
    return RG_OK;
}

extern "C" RG_API int rg_noalloc_get_status(rg_status* out, void* stream) {
    if (!out) return RG_ERR_INVALID_ARG;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return RG_ERR_CUDA;
    DeviceSetup* d = nullptr;
    int rc = setup_device(dev, &d);
    if (rc) return rc;
    if (cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess) return RG_ERR_CUDA;
    rg::DevStatus h;
    if (cudaMemcpy(&h, d->base + kLayout.status, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) return RG_ERR_CUDA;
    rg::export_status(h, out);
    return RG_OK;
}
