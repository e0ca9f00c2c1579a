/*
 * Runs the reference's own device programs on the CPU — TEST INFRASTRUCTURE ONLY.
 * oracle/Makefile compiles this file four times against sources in the reference tree
 * (REF_STAGE 1: cuda_train/forward/gaussians_aabb.cu, 2: cuda_train/backward/gaussians_aabb.cu,
 * 3: vec_math.h + utils/sh_utils.cu, 4: cuda_test/gaussians_aabb.cu, the inference programs),
 * with ref_shim/optix.h standing in for the OptiX device API.  The outputs (oracle/_ref/*.so)
 * pin the C restatement in rg_oracle_impl.h.
 */
#include <cstring>
#include <cstdlib>
#include <cmath>

#if REF_STAGE == 1 || REF_STAGE == 2
#include REF_SOURCE
thread_local RgEmulRay rg_emul;
RgEmulScene rg_emul_scene;
/* trace calls find their primitives through the grid (1) or a per-ray scan of all AABBs (0) */
static bool rg_use_grid = true;
extern "C" void ref_set_grid(int on) { rg_use_grid = on != 0; }

static void set_common(int n, const float* pos, const float* scl, const float* quat, const float* dens,
                       const float* rgb, const float* scene_box, const float* cam, int W, int H,
                       int max_prim_slice, int jitter, int rnd_sample, unsigned iteration, int* hit_buf) {
    params.iteration = iteration;
    params.jitter = (unsigned)jitter;
    params.rnd_sample = (unsigned)rnd_sample;
    params.max_prim_slice = (unsigned)max_prim_slice;
    params.bbox_min = make_float3(scene_box[0], scene_box[1], scene_box[2]);
    params.bbox_max = make_float3(scene_box[3], scene_box[4], scene_box[5]);
    params.image_width = (unsigned)W;
    params.image_height = (unsigned)H;
    params.cam_eye = make_float3(cam[0], cam[1], cam[2]);
    params.cam_u = make_float3(cam[3], cam[4], cam[5]);
    params.cam_v = make_float3(cam[6], cam[7], cam[8]);
    params.cam_w = make_float3(cam[9], cam[10], cam[11]);
    params.cam_tan_half_fovx = cam[12];
    params.cam_tan_half_fovy = cam[13];
    params.densities = const_cast<float*>(dens);
    params.color_features = const_cast<float*>(rgb);
    params.positions = (float3*)pos;
    params.scales = (float3*)scl;
    params.quaternions = (float4*)quat;
    params.hit_prim_idx = hit_buf;
    (void)n;
}

static sphere::SphereHitGroupData g_sbt;

/* Launch the ray-generation program for rays ids[0..n_ids) (all W*H rays when ids is null). */
static void run_rays(int W, int H, const int* ids, int n_ids) {
    const int n_rays = ids ? n_ids : W * H;
#pragma omp parallel for schedule(dynamic, 8)
    for (int r = 0; r < n_rays; ++r) {
        rg_emul.launch_idx = make_uint3((unsigned)(ids ? ids[r] : r), 0u, 0u);
        rg_emul.launch_dim = make_uint3((unsigned)(W * H), 1u, 1u);
        rg_emul.have_cands = false;
        __raygen__rg();
    }
}
#endif

#if REF_STAGE == 1
extern "C" int ref_forward(int n, const float* pos, const float* scl, const float* quat, const float* dens,
                           const float* rgb, const float* aabb, const float* scene_box, const float* cam,
                           int W, int H, int white_bg, int max_prim_slice, int jitter, int rnd_sample,
                           unsigned iteration, const int* ids, int n_ids, float* out_colors, int* overflow) {
    /* W*H*max_prim_slice slots as the reference allocates them (scripts/train.py:38-39); only the
     * pages of launched rays are touched */
    int* hit_buf = (int*)std::calloc((size_t)W * H * (size_t)max_prim_slice, sizeof(int));
    if (!hit_buf) return -1;
    set_common(n, pos, scl, quat, dens, rgb, scene_box, cam, W, H, max_prim_slice, jitter, rnd_sample,
               iteration, hit_buf);
    params.ray_colors = (float3*)out_colors;
    params.handle = 0;
    *overflow = 0;
    params.max_gaussians_exceeded = overflow;
    params.white_background = (unsigned)white_bg;
    g_sbt.positions = (float3*)pos; g_sbt.scales = (float3*)scl; g_sbt.quaternions = (float4*)quat;
    rg_emul_bind(aabb, n, scene_box, &g_sbt, rg_use_grid);
    run_rays(W, H, ids, n_ids);
    rg_emul_unbind();
    std::free(hit_buf);
    return 0;
}
#elif REF_STAGE == 2
extern "C" int ref_backward(int n, const float* pos, const float* scl, const float* quat, const float* dens,
                            const float* rgb, const float* aabb, const float* scene_box, const float* cam,
                            int W, int H, int max_prim_slice, int jitter, int rnd_sample, unsigned iteration,
                            const int* ids, int n_ids, const float* ray_colors, const float* dL, float* d_dens,
                            float* d_rgb, float* d_pos, float* d_scl, float* d_quat) {
    int* hit_buf = (int*)std::calloc((size_t)W * H * (size_t)max_prim_slice, sizeof(int));
    if (!hit_buf) return -1;
    set_common(n, pos, scl, quat, dens, rgb, scene_box, cam, W, H, max_prim_slice, jitter, rnd_sample,
               iteration, hit_buf);
    params.ray_colors = (float3*)ray_colors;
    params.dloss_dray_colors = (float3*)dL;
    params.densities_grad = d_dens;
    params.color_features_grad = (float3*)d_rgb;
    params.positions_grad = (float3*)d_pos;
    params.scales_grad = (float3*)d_scl;
    params.quaternions_grad = (float4*)d_quat;
    params.handle = 0;
    g_sbt.positions = (float3*)pos; g_sbt.scales = (float3*)scl; g_sbt.quaternions = (float4*)quat;
    rg_emul_bind(aabb, n, scene_box, &g_sbt, rg_use_grid);
    run_rays(W, H, ids, n_ids);
    rg_emul_unbind();
    std::free(hit_buf);
    return 0;
}
#elif REF_STAGE == 4
#include REF_SOURCE
thread_local RgEmulRay rg_emul;
RgEmulScene rg_emul_scene;
/* trace calls find their primitives through the grid (1) or a per-ray scan of all AABBs (0) */
static bool rg_use_grid = true;
extern "C" void ref_set_grid(int on) { rg_use_grid = on != 0; }
static sphere::SphereHitGroupData g_sbt;

/* optix_utils.py:302-373: inference launch; colours (R,3) and Gaussians per ray (R) */
extern "C" int ref_inference(int n, const float* pos, const float* scl, const float* quat, const float* dens,
                             const float* rgb, const float* aabb, const float* scene_box, const float* cam,
                             int W, int H, int white_bg, int max_prim_slice, const int* ids, int n_ids,
                             float* out_colors, int* out_counts) {
    params.rnd_sample = 0u;
    params.max_prim_slice = (unsigned)max_prim_slice;
    params.bbox_min = make_float3(scene_box[0], scene_box[1], scene_box[2]);
    params.bbox_max = make_float3(scene_box[3], scene_box[4], scene_box[5]);
    params.image_width = (unsigned)W;
    params.image_height = (unsigned)H;
    params.cam_eye = make_float3(cam[0], cam[1], cam[2]);
    params.cam_u = make_float3(cam[3], cam[4], cam[5]);
    params.cam_v = make_float3(cam[6], cam[7], cam[8]);
    params.cam_w = make_float3(cam[9], cam[10], cam[11]);
    params.cam_tan_half_fovx = cam[12];
    params.cam_tan_half_fovy = cam[13];
    params.densities = const_cast<float*>(dens);
    params.color_features = const_cast<float*>(rgb);
    params.positions = (float3*)pos;
    params.scales = (float3*)scl;
    params.quaternions = (float4*)quat;
    /* the program writes colours and adds counts at launch indices: full-size buffers */
    float* colors = (float*)std::calloc((size_t)W * H * 3, sizeof(float));
    int* counts = (int*)std::calloc((size_t)W * H, sizeof(int));
    if (!colors || !counts) { std::free(colors); std::free(counts); return -1; }
    params.ray_colors = (float3*)colors;
    params.number_of_gaussians_per_ray = counts;
    params.number_of_gaussians_per_slab = nullptr;
    params.handle = 0;
    params.white_background = (unsigned)white_bg;
    g_sbt.positions = (float3*)pos; g_sbt.scales = (float3*)scl; g_sbt.quaternions = (float4*)quat;
    rg_emul_bind(aabb, n, scene_box, &g_sbt, rg_use_grid);
    const int n_rays = ids ? n_ids : W * H;
#pragma omp parallel for schedule(dynamic, 8)
    for (int r = 0; r < n_rays; ++r) {
        rg_emul.launch_idx = make_uint3((unsigned)(ids ? ids[r] : r), 0u, 0u);
        rg_emul.launch_dim = make_uint3((unsigned)(W * H), 1u, 1u);
        rg_emul.have_cands = false;
        __raygen__rg();
    }
    rg_emul_unbind();
    for (int r = 0; r < n_rays; ++r) {
        const int k = ids ? ids[r] : r;
        for (int c = 0; c < 3; ++c) out_colors[3 * r + c] = colors[3 * k + c];
        out_counts[r] = counts[k];
    }
    std::free(colors);
    std::free(counts);
    return 0;
}
#elif REF_STAGE == 3
#include <vector_types.h>
static thread_local uint3 threadIdx;
static thread_local uint3 blockIdx;
static thread_local dim3 blockDim;
#include REF_VECMATH
#include REF_SOURCE

extern "C" void ref_forward_sh(const float* campos, const float* pos, const float* sh, const float* sg,
                               const float* kappa, const float* axis, unsigned nsg, int deg, int n, float* rgb) {
    blockDim = dim3(128, 1, 1);
    for (int i = 0; i < n; ++i) {
        blockIdx = make_uint3((unsigned)(i / 128), 0, 0);
        threadIdx = make_uint3((unsigned)(i % 128), 0, 0);
        forward_sh(const_cast<float*>(campos), (float3*)pos, const_cast<float*>(sh), const_cast<float*>(sg),
                   const_cast<float*>(kappa), const_cast<float*>(axis), nsg, deg, n, rgb);
    }
}

extern "C" void ref_backward_sh(const float* campos, const float* pos, const float* sh, const float* sg,
                                const float* kappa, const float* axis, unsigned nsg, int deg, int n,
                                const float* drgb, float* dsh, float* dpos, float* dsg, float* dkappa,
                                float* daxis) {
    blockDim = dim3(128, 1, 1);
    for (int i = 0; i < n; ++i) {
        blockIdx = make_uint3((unsigned)(i / 128), 0, 0);
        threadIdx = make_uint3((unsigned)(i % 128), 0, 0);
        backward_sh(const_cast<float*>(campos), (float3*)pos, const_cast<float*>(sh), const_cast<float*>(sg),
                    const_cast<float*>(kappa), const_cast<float*>(axis), nsg, deg, n, (float3*)drgb, dsh,
                    (float3*)dpos, dsg, dkappa, daxis);
    }
}
#endif
