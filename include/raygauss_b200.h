/*
 * raygauss_b200 — C ABI of the B200 (sm_100a) engine for RayGauss's differentiable volumetric
 * Gaussian ray caster.
 *
 * Plain C: pointers, sizes and POD structs only.  Descriptor structs (rg_gaussians, rg_settings,
 * rg_train_tail, rg_densify, field and tensor lists ...) live in host memory; the arrays they and
 * the arguments point to are device memory unless stated otherwise, and the kernels cannot tell a
 * host pointer from a device one (the Python layer checks the tensors' devices; C callers must).
 * Every device pointer is borrowed (the caller owns it); the engine owns only its scratch (BVH,
 * leaf records, per-view colours, gradient accumulators, work counters).  Every call is ordered on
 * the CUDA stream passed as `stream` (a cudaStream_t, 0 = legacy default stream) and returns RG_OK
 * or an RG_ERR_* code; it performs no host synchronisation and no allocation once the engine has
 * been sized for the scene (rg_reserve), except where an entry point says so (rg_densify_plan
 * reads its counts back).  Device-side conditions (hit-list passes, stack overflow, watchdog,
 * non-finite input) are counted in a device status block read by rg_get_status().
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   rg_ellipsoids_bbox  optix_raycasting/optix_utils.py:34-66 (quaternion_to_rotation,
 *                       compute_ellipsoids_bbox) + render_optix.py:105-106 (scene box min/max)
 *   rg_bvh_build        optix_raycasting/optix_utils.py:68-71 (create_acceleration_structure)
 *   rg_bvh_refit        optix_raycasting/optix_utils.py:73-75 (update_acceleration_structure)
 *   rg_forward_sh       utils/sh_utils.cu:25-119 (forward_sh) via render_optix.py:19-32
 *                       (compute_cupy_rgb)
 *   rg_launch_forward   optix_raycasting/optix_utils.py:128-209 (launch_pipeline_forward) and the
 *                       programs of cuda_train/forward/gaussians_aabb.cu:324-641
 *   rg_launch_backward  optix_raycasting/optix_utils.py:213-299 (launch_pipeline_backward) and the
 *                       programs of cuda_train/backward/gaussians_aabb.cu:405-802
 *   rg_backward_sh      utils/sh_utils.cu:121-315 (backward_sh) via render_optix.py:34-52
 *                       (compute_cupy_sh_grad) and the gradient assembly of render_optix.py:170-190
 *   rg_render_forward   RenderOptixFunction.forward, optix_raycasting/render_optix.py:92-132
 *   rg_render_backward  RenderOptixFunction.backward, optix_raycasting/render_optix.py:136-190
 *   rg_launch_inference optix_raycasting/optix_utils.py:302-373 (launch_pipeline_test) and the
 *                       programs of cuda_test/gaussians_aabb.cu:236-470
 *   rg_render_inference the inference render of scripts/test.py:42-132 (bbox, GAS, colour, launch)
 *   rg_train_tail_step  the step tail of scripts/train.py:121-181 (statistics, the optimizer
 *                       managers' Adam steps of classes/optimizer.py:13-21, parameter clamps)
 *   rg_densify_plan /   densify_and_prune, classes/point_cloud.py:1068-1143, with the optimizer
 *   rg_densify_apply    state surgery of classes/optimizer.py:54-83
 *   rg_records_to_columns  the field extraction of scripts/ply.py:85-146 (read_ply) and of the
 *                       loaders classes/point_cloud.py:298-394, 396-495
 *   rg_compute_3d_filter   PointCloud.compute_3D_filter, classes/point_cloud.py:1153-1215
 *   rg_knn_mean_dist    distCUDA2 of the simple-knn extension (submodules/simple-knn/spatial.cu:14-25),
 *                       used by classes/point_cloud.py:374-378 for point clouds without scales
 */
#ifndef RAYGAUSS_B200_H
#define RAYGAUSS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RG_ABI_VERSION 3

#if defined(__GNUC__)
#define RG_API __attribute__((visibility("default")))
#else
#define RG_API
#endif

enum rg_result {
    RG_OK = 0,
    RG_ERR_INVALID_ARG = 1,   /* null pointer, bad size, unsupported degree, misaligned buffer */
    RG_ERR_CUDA = 2,          /* a CUDA runtime call failed (see rg_last_cuda_error) */
    RG_ERR_OOM = 3,           /* scratch allocation failed */
    RG_ERR_STATE = 4,         /* call order violated (e.g. render before bbox/bvh) */
    RG_ERR_CAPACITY = 5       /* request exceeds a fixed capacity of the entry point */
};

/* Storage type of densities, colour features and SG amplitudes. */
enum rg_storage { RG_STORAGE_F32 = 0, RG_STORAGE_BF16 = 1 };

/* Sample arithmetic of the render kernels.
 * RG_MODE_PARITY: the reference's per-sample arithmetic (drop-in; image max-abs <= 1e-4).
 * RG_MODE_FAST: incremental per-slab sample evaluation and moment-form adjoint (same sample
 * grid, masks and early exit; accuracy reported as PSNR against the FP64 oracle). */
enum rg_mode { RG_MODE_PARITY = 0, RG_MODE_FAST = 1 };

/* Pinhole camera: the launch-parameter record of optix_utils.py:166-177.  u, v, w are the camera
 * x (right), y (down) and z (forward) axes in world space, i.e. world_view_transform[:3,0..2];
 * width/height are the ray grid (image size times supersampling). 64 bytes. */
typedef struct rg_camera {
    float eye[3];
    float u[3];
    float v[3];
    float w[3];
    float tan_half_fovx;
    float tan_half_fovy;
    int32_t width;
    int32_t height;
} rg_camera;

/* Gaussian parameters in the layout of PointCloud.get_data (classes/point_cloud.py:729-739).
 * All pointers are device pointers, contiguous, 4-byte aligned (16-byte for quaternions). */
typedef struct rg_gaussians {
    const float* positions;            /* (N,3) */
    const float* scales;               /* (N,3), already exp(log_scale) */
    const float* quaternions;          /* (N,4), (w,x,y,z), used as passed (not normalised) */
    const void* densities;             /* (N,) raw, f32 or bf16 per `storage` */
    const void* color_features;        /* (N,3,(deg+1)^2) channel-major, f32 or bf16 */
    const void* sph_gauss_features;    /* (N,3,nsg), f32 or bf16; may be NULL when nsg == 0 */
    const float* bandwidth_sharpness;  /* (N,nsg) after softplus; may be NULL when nsg == 0 */
    const float* lobe_axis;            /* (N,nsg,3) unit axes; may be NULL when nsg == 0 */
    int64_t n;                         /* 1 .. 2^25 (33,554,432) Gaussians per engine */
    int32_t sh_degree;                 /* 0..3 */
    int32_t num_sph_gauss;             /* 0..RG_MAX_SG */
    int32_t storage;                   /* enum rg_storage */
    int32_t reserved;
} rg_gaussians;

#define RG_MAX_SG 16

/* Per-call settings: the RenderOptixSettings fields that reach the device
 * (render_optix.py:67-87; configs/base.yml training.max_prim_slice/jitter/rnd_sample). */
typedef struct rg_settings {
    int32_t white_background;
    int32_t jitter;
    int32_t rnd_sample;
    int32_t max_prim_slice;            /* reference per-slab hit cap (counted, never truncated) */
    uint32_t iteration;                /* RNG seed component (tea<4>(iteration, ray)) */
    int32_t mode;                      /* enum rg_mode */
    int32_t sh_quirk;                  /* 1: reproduce the reference SH basis-9 y-derivative */
    int32_t reserved;
} rg_settings;

/* Output gradients (device, f32, fully overwritten — no accumulation, no zero-fill needed).
 * sph_gauss_features / bandwidth_sharpness / lobe_axis may be NULL when nsg == 0. */
typedef struct rg_gradients {
    float* positions;                  /* (N,3) geometric + view-direction terms */
    float* scales;                     /* (N,3) */
    float* quaternions;                /* (N,4) */
    float* densities;                  /* (N,) */
    float* color_features;             /* (N,3,(deg+1)^2) */
    float* sph_gauss_features;         /* (N,3,nsg) */
    float* bandwidth_sharpness;        /* (N,nsg) */
    float* lobe_axis;                  /* (N,nsg,3) */
} rg_gradients;

/* Device counters accumulated since the last reset. */
typedef struct rg_status {
    uint64_t hit_pairs;                /* (ray, slab, Gaussian) pairs evaluated */
    uint64_t slabs;                    /* (ray, slab) pairs marched */
    uint64_t slab_cap_exceeded;        /* slabs with more hits than max_prim_slice (reference truncates) */
    uint64_t list_passes;              /* extra traversal passes caused by a full warp hit list */
    uint64_t chunk_splits;             /* chunk-length reductions caused by a full warp hit list */
    uint64_t stack_overflows;          /* traversal stack overflows (result incomplete) */
    uint64_t watchdog_trips;           /* work items abandoned by the iteration limit */
    uint64_t nonfinite_inputs;         /* Gaussians with a non-finite parameter (skipped) */
    uint64_t traversals;               /* warp-level BVH traversals (one per chunk and pass) */
    uint64_t node_visits;              /* warp-level internal-node visits */
    uint64_t leaf_tests;               /* warp-level leaf (exact ellipsoid) tests */
    uint64_t list_entries;             /* warp hit-list entries appended */
    uint64_t slab_steps;               /* warp-level slab iterations with at least one entry */
    uint64_t entry_slabs;              /* warp-level (entry, slab) evaluations */
    uint64_t replayed_chunks;          /* backward chunks replayed from the forward's hit-list record */
    uint64_t record_overflows;         /* tiles whose hit-list record did not fit (backward traverses) */
    uint64_t record_words;             /* 4-byte words of the last forward's hit-list record */
} rg_status;

/* Kernel tuning knobs (rg_autotune picks them; 0 = keep the current value). */
typedef struct rg_tuning {
    int32_t chunk_slabs;               /* longest traversal chunk in slabs, 1..255 */
    int32_t blocks_per_sm;             /* resident render CTAs per SM */
    int32_t list_capacity;             /* 64 or 128: fast-arithmetic warp hit lists hold 4x this
                                          many entries; parity lists always hold 128 */
    int32_t record_hits;               /* 1: the forward records its hit lists and the backward
                                          replays them (default); -1: the backward traverses */
    int32_t diagnostics;               /* 1: the render kernels also count node visits, leaf tests,
                                          list entries, slab steps and entry-slabs (rg_status);
                                          0 (default): those stay 0 and the kernels hold fewer
                                          registers */
} rg_tuning;

typedef struct rg_engine rg_engine;

/* Engine lifetime (no reference counterpart beyond create_context, optix_utils.py:77-81). */
RG_API int rg_create(rg_engine** out, int device);
RG_API int rg_destroy(rg_engine* e);
/* Size the engine's scratch for n Gaussians, up to n_views views and n_rays rays per call.
 * Calls made afterwards with sizes within these bounds allocate nothing.  n_rays also sizes the
 * hit-list record (96 B per ray); without it the backward traverses the BVH again. */
RG_API int rg_reserve(rg_engine* e, int64_t n, int32_t n_views, int64_t n_rays);
RG_API int rg_set_tuning(rg_engine* e, const rg_tuning* t);
RG_API int rg_get_tuning(const rg_engine* e, rg_tuning* t);

/* optix_utils.py:34-66 + render_optix.py:105-106.  Computes the per-Gaussian threshold-ellipsoid
 * AABBs, the scene box and the leaf records used by the BVH and the render kernels.
 * aabb_out (N,6) and scene_box_out (6) are optional device outputs (NULL to skip). */
RG_API int rg_ellipsoids_bbox(rg_engine* e, const rg_gaussians* g, float* aabb_out, float* scene_box_out,
                       void* stream);
/* optix_utils.py:68-71: full LBVH build (Morton codes, radix sort, Karras hierarchy, refit). */
RG_API int rg_bvh_build(rg_engine* e, void* stream);
/* optix_utils.py:73-75: keep the leaf order and topology of the last build, refit the boxes to
 * the current parameters (rg_ellipsoids_bbox must have run on the new parameters). */
RG_API int rg_bvh_refit(rg_engine* e, void* stream);

/* utils/sh_utils.cu:25-119 for n_cams views at once.  cams is a DEVICE array of rg_camera.
 * rgb_out (n_cams,N,3) is an optional device output in Gaussian order.  n_cams * N < 2^31. */
RG_API int rg_forward_sh(rg_engine* e, const rg_gaussians* g, const rg_camera* cams, int32_t n_cams,
                  float* rgb_out, void* stream);

/* optix_utils.py:128-209 for n_cams views in one persistent launch.  ray_colors (R,3) with the
 * views' rays packed in order, ray y*W+x within a view; final_T (R,) optional. */
RG_API int rg_launch_forward(rg_engine* e, const rg_camera* cams, int32_t n_cams, const rg_settings* s,
                      float* ray_colors, float* final_T, void* stream);
/* optix_utils.py:302-373 (launch_pipeline_test) with the inference programs of
 * optix_raycasting/cuda_test/gaussians_aabb.cu:236-470: a forward render without jitter or random
 * sample offsets whose slab query is not clipped at the scene-box exit and whose samples step
 * through the conic space (parity arithmetic).  gaussians_per_ray (R,) int32 is optional: the
 * per-slab hit counts summed over the ray, each capped at max_prim_slice (exact in the parity
 * arithmetic; the fast arithmetic counts every list entry whose chunk interval covers the lane). */
RG_API int rg_launch_inference(rg_engine* e, const rg_camera* cams, int32_t n_cams, const rg_settings* s,
                        float* ray_colors, int32_t* gaussians_per_ray, void* stream);
/* bbox -> BVH build (or refit) -> colour -> rg_launch_inference, as rg_render_forward. */
RG_API int rg_render_inference(rg_engine* e, const rg_gaussians* g, const rg_camera* cams, int32_t n_cams,
                        const rg_settings* s, int32_t refit, float* ray_colors, int32_t* gaussians_per_ray,
                        float* rgb_out, void* stream);
/* optix_utils.py:213-299: recompute the forward's slabs and scatter per-Gaussian gradients into
 * the engine's accumulators (zeroed by this call).  ray_colors are the forward outputs.  When no
 * bbox/BVH/colour/tuning call came after the last rg_launch_forward and cams, n_cams and *s are
 * that forward's, its recorded warp hit lists are replayed instead of traversing the BVH again. */
RG_API int rg_launch_backward(rg_engine* e, const rg_camera* cams, int32_t n_cams, const rg_settings* s,
                       const float* ray_colors, const float* dloss_dray_colors, void* stream);
/* utils/sh_utils.cu:121-315 + render_optix.py:170-190: SH/SG backward for every view and the
 * final gradient assembly into `out`. */
RG_API int rg_backward_sh(rg_engine* e, const rg_gaussians* g, const rg_camera* cams, int32_t n_cams,
                   const rg_settings* s, const rg_gradients* out, void* stream);

/* RenderOptixFunction.forward (render_optix.py:92-132): bbox -> BVH (build, or refit when
 * `refit` != 0 and a build of the same N exists) -> colour -> march.  rgb_out optional. */
RG_API int rg_render_forward(rg_engine* e, const rg_gaussians* g, const rg_camera* cams, int32_t n_cams,
                      const rg_settings* s, int32_t refit, float* ray_colors, float* final_T,
                      float* rgb_out, void* stream);
/* RenderOptixFunction.backward (render_optix.py:136-190) on the BVH and colours of the last
 * rg_render_forward with the same parameters. */
RG_API int rg_render_backward(rg_engine* e, const rg_gaussians* g, const rg_camera* cams, int32_t n_cams,
                       const rg_settings* s, const float* ray_colors, const float* dloss_dray_colors,
                       const rg_gradients* out, void* stream);

/* Leaf order of the last BVH build: leaf_gid_out[l] = index of the Gaussian in leaf l (N int32,
 * device).  Hits of a slab are accumulated in increasing leaf order; the reference's order is
 * its (unspecified) traversal order.  No reference counterpart (introspection of the BVH). */
RG_API int rg_leaf_order(rg_engine* e, int32_t* leaf_gid_out, void* stream);
/* Allocation-free forward render for callers that cannot call cudaMalloc (allocation-free graph
 * capture, fixed device-memory budgets, plugins that must not touch the process allocator).  No
 * counterpart in the reference.  Same pre-pass, LBVH build, colour pass and forward launch as
 * rg_render_forward (default tuning), without an engine: all scratch lives in one static device
 * array of about 10 MB that every GPU loading this library keeps until exit.  At most 16384
 * Gaussians and 4 views per call (RG_ERR_CAPACITY beyond).  Calls share that array, so calls that
 * overlap on the GPU race; the first call on a device resolves the array's address and should
 * come before any stream capture.  cams, ray_colors and final_T are device pointers as in
 * rg_launch_forward; final_T may be NULL. */
RG_API int rg_render_forward_noalloc(const rg_gaussians* g, const rg_camera* cams, int32_t n_cams,
                                     const rg_settings* s, float* ray_colors, float* final_T, void* stream);
/* Device counters of the latest rg_render_forward_noalloc call on the current device (each call
 * clears them when it starts): synchronises `stream`, then copies the counters out of the static
 * array, allocating nothing.  record_words is always 0 (the call keeps no hit-list record).  No
 * counterpart in the reference. */
RG_API int rg_noalloc_get_status(rg_status* out, void* stream);
/* Read (and optionally reset) the device counters; synchronises the engine's last stream. */
RG_API int rg_get_status(rg_engine* e, rg_status* out, int32_t reset, void* stream);
/* Number of kernels launched by this engine since creation (for launch accounting). */
RG_API uint64_t rg_kernel_launches(const rg_engine* e);
RG_API const char* rg_error_string(int code);
RG_API const char* rg_last_cuda_error(const rg_engine* e);
RG_API int rg_abi_version(void);

/* ---- Fused training-step tail (scripts/train.py:121-181) ----------------------------------------
 * One launch over the Gaussians: the densification statistics of the position gradient
 * (classes/point_cloud.py:633-640), one Adam step on every listed tensor (classes/optimizer.py:13-21,
 * torch.optim.Adam arithmetic with the learning rate and bias corrections of this step from the
 * host), then densities < 0 -> 0, optional quaternion and lobe-axis normalisation and the log-scale
 * clamp to [min_scale (filter_3D), max_scale] (scripts/train.py:166-181).  Tensors are FP32 with
 * `width` floats per Gaussian (e.g. positions 3, SH 45); an inactive tensor or one without a gradient
 * is left as it is, like a torch parameter whose .grad is None. */
#define RG_TAIL_MAX_TENSORS 12
typedef struct rg_adam_tensor {
    float* param;
    const float* grad;
    float* exp_avg;
    float* exp_avg_sq;
    int32_t width;                     /* floats per Gaussian */
    int32_t active;                    /* 0: skip this tensor at this step */
    float lr, beta1, beta2, eps;
    float one_minus_beta1;             /* 1 - beta1 and 1 - beta2, rounded once from the host's */
    float one_minus_beta2;             /* values (as torch does with its Python scalars) */
    float bias1;                       /* 1 - beta1^t */
    float bias2_sqrt;                  /* sqrt(1 - beta2^t) */
} rg_adam_tensor;

typedef struct rg_train_tail {
    int64_t n;                         /* Gaussians */
    int32_t n_tensors;
    int32_t idx_positions, idx_densities, idx_scales, idx_quaternions, idx_lobe_axis;  /* -1: absent */
    int32_t normalize_quaternions, normalize_lobe_axis;
    float max_scale;                   /* upper clamp of the log scales (+inf: none) */
    const float* min_scale;            /* (N,) lower clamp of the log scales (filter_3D), NULL: none */
    float* grad_norm_accum;            /* (N,) += |dL/dposition|, NULL: skip */
    float* num_accum;                  /* (N,) += 1 where the position gradient is non-zero, NULL: skip */
    float* num_accum_gnv;              /* (N,) same, the not-visible statistic, NULL: skip */
    /* NULL, or a DEVICE array [n_tensors][4] = {active, lr, bias1, bias2_sqrt} read by the kernel in
     * place of those host fields (tensors[i].active must still be set for a tensor that may step):
     * the launch can then be captured in a CUDA graph and each replay's scalars written beforehand. */
    const float* step_scalars;
    rg_adam_tensor tensors[RG_TAIL_MAX_TENSORS];
} rg_train_tail;

RG_API int rg_train_tail_step(const rg_train_tail* d, void* stream);

/* ---- Densification (classes/point_cloud.py:1068-1143) -------------------------------------------
 * densify_and_prune(max_grad, min_density, extent): Gaussians whose mean position gradient
 * (grad_accum / num_accum, NaN -> 0) is >= grad_threshold are cloned when max(exp(log_scales)) <=
 * scale_threshold (0.01 * extent; the original and the clone get half the density) and split into
 * n_split copies otherwise (positions mu + R(q) (z * exp(s)) with z the caller's standard normals,
 * log scales log(exp(s) * split_scale_mul), half the density; the original is removed); then every
 * Gaussian with density <= min_density is removed.  Output order as the reference's: surviving
 * originals, clones, split copy 0 of every split Gaussian, copy 1, ...
 *   rg_densify_plan   classifies and counts; reads the counts back (synchronises `stream`) and
 *                     fills n_out and the other counts
 *   rg_densify_apply  writes every listed tensor at the new size (dst holds n_out rows); draws
 *                     nothing: split_normals is (n_split * n_split_sel, 3), row c * n_split_sel + k
 *                     for copy c of the k-th split Gaussian (torch.normal's sample order)
 * workspace: rg_densify_workspace_bytes(n, n_split) device bytes, kept from plan to apply. */
#define RG_DENSIFY_MAX_TENSORS 48
enum rg_densify_kind {
    RG_DENSIFY_COPY = 0,        /* every output row copies its source row (parameters, filter_3D) */
    RG_DENSIFY_OLD_ONLY = 1,    /* rows of kept originals move, new rows are 0 (Adam moments, num_accum_gnv) */
    RG_DENSIFY_ZERO = 2,        /* all rows 0 (the reset gradient statistics); src unused */
    RG_DENSIFY_DENSITIES = 3,   /* width 1: halved for clones, their originals and split copies */
    RG_DENSIFY_LOG_SCALES = 4,  /* width 3: split copies get log(exp(s) * split_scale_mul) */
    RG_DENSIFY_POSITIONS = 5    /* width 3: split copies get mu + R(q) (z * exp(s)) */
};
typedef struct rg_densify_tensor {
    const float* src;                  /* (n, width) */
    float* dst;                        /* (n_out, width) */
    int32_t width;
    int32_t kind;                      /* rg_densify_kind */
} rg_densify_tensor;

typedef struct rg_densify {
    int64_t n;
    const float* grad_accum;           /* (n,) xyz_gradient_accum_norm */
    const float* num_accum;            /* (n,) */
    const float* log_scales;           /* (n, 3) */
    const float* quaternions;          /* (n, 4), 16-byte aligned (split rotations) */
    const float* densities;            /* (n,) */
    float grad_threshold;              /* densify_grad_threshold */
    float scale_threshold;             /* 0.01 * scene extent, rounded to float */
    float min_density;                 /* SIGMA_THRESHOLD: densities <= it are removed */
    float split_scale_mul;             /* 1 / (0.8 * n_split), rounded to float */
    int32_t n_split;                   /* copies per split Gaussian (reference: 2), 1..8 */
    int32_t planned;                   /* set by rg_densify_plan */
    void* workspace;
    /* written by rg_densify_plan */
    int64_t n_clone, n_split_sel;      /* selected for cloning / splitting */
    int64_t n_out;                     /* Gaussians after densify and prune */
    int64_t n_kept, kept_clones, kept_splits;  /* surviving originals, clones, copies per split copy */
} rg_densify;

/* ---- PLY vertex records -> FP32 columns (scripts/ply.py:85-146) ------------------------------------
 * `records` is the device copy of a binary PLY vertex block: n records of record_bytes bytes.  Each
 * field reads `type` at byte `offset` of every record (big_endian: the file's byte order), converts
 * it to double, optionally applies ((v / div) + add) * mul_a * mul_b in double (the reference's
 * colour initialisation, classes/point_cloud.py:326-329), and writes it rounded to float to
 * dst[i * dst_stride].  record_bytes <= 36864; up to RG_RECORD_MAX_FIELDS fields per call. */
#define RG_RECORD_MAX_FIELDS 1024
enum rg_field_type {
    RG_FIELD_I8 = 0, RG_FIELD_U8 = 1, RG_FIELD_I16 = 2, RG_FIELD_U16 = 3,
    RG_FIELD_I32 = 4, RG_FIELD_U32 = 5, RG_FIELD_F32 = 6, RG_FIELD_F64 = 7
};
typedef struct rg_record_field {
    int32_t offset;                    /* byte offset in the record */
    int32_t type;                      /* rg_field_type */
    int32_t big_endian;
    int32_t affine;                    /* 0: plain conversion */
    float* dst;
    int64_t dst_stride;                /* floats between consecutive records' values */
    double div, add, mul_a, mul_b;
} rg_record_field;

RG_API int rg_records_to_columns(const void* records, int64_t n, int32_t record_bytes, const rg_record_field* fields,
                                 int32_t n_fields, void* stream);

/* ---- 3D minimum-size filter (classes/point_cloud.py:1153-1215) -----------------------------------
 * filter_out[i] = log(0.5 * depth_i / focal) with depth_i the smallest camera-space depth over the
 * cameras that see Gaussian i (depth > 0.2, projection inside the image widened by 15 % per side),
 * or the largest such depth of all Gaussians when no camera sees it (-inf when no Gaussian is seen
 * at all; the reference raises).  Each camera holds the reference's per-camera values rounded to
 * float on the host: R (world_view_transform[:3,:3], row-major), T (world_view_transform[3,:3]),
 * focal_x, focal_y, W / 2, H / 2 and the window bounds -0.15 W, 1.15 W, -0.15 H, 1.15 H.
 * inv_focal = 1 / (largest focal length), rounded to float.  depth_scratch: n floats and
 * max_scratch: one word of device memory. */
typedef struct rg_filter_camera {
    float R[9];
    float T[3];
    float focal_x, focal_y, cx, cy;
    float x_lo, x_hi, y_lo, y_hi;
} rg_filter_camera;

RG_API int rg_compute_3d_filter(const float* positions, int64_t n, const rg_filter_camera* cameras, int32_t n_cams,
                                float inv_focal, float* depth_scratch, uint32_t* max_scratch, float* filter_out,
                                void* stream);

/* ---- Mean squared distance to the 3 nearest neighbours (simple-knn distCUDA2) --------------------
 * mean_dist[i] = (d0 + d1 + d2) / 3 with d0 <= d1 <= d2 the three smallest squared distances from
 * point i to the other points (exact; missing neighbours count as FLT_MAX, so two neighbours give
 * about FLT_MAX / 3 and one or none +inf, as the extension).  points: (n, 3)
 * device floats; workspace: rg_knn_workspace_bytes(n) device bytes. */
RG_API int rg_knn_workspace_bytes(int64_t n, uint64_t* bytes);
RG_API int rg_knn_mean_dist(const float* points, int64_t n, float* mean_dist, void* workspace, void* stream);

RG_API int rg_densify_workspace_bytes(int64_t n, int32_t n_split, uint64_t* bytes);
RG_API int rg_densify_plan(rg_densify* d, void* stream);
RG_API int rg_densify_apply(const rg_densify* d, const float* split_normals, const rg_densify_tensor* tensors,
                            int32_t n_tensors, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* RAYGAUSS_B200_H */
