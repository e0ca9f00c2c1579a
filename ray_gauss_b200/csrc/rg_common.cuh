// Shared device definitions of the B200 ray-caster engine.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "raygauss_b200.h"

namespace rg {

// Reference constants (optix_raycasting/cuda_train/forward/gaussians_aabb.h:2-5).
constexpr int kBuf = 8;                 // samples per slab
constexpr float kDt = 0.0025f;          // sample spacing
constexpr float kSlab = kDt * kBuf;     // slab length (0.02)
constexpr float kTeps = 0.003f;         // early-exit transmittance
constexpr float kSigThr = 0.1f;         // per-sample density threshold

constexpr int kWarp = 32;
constexpr int kTileW = 8;               // a warp renders an 8x4 pixel tile
constexpr int kTileH = 4;
constexpr int kMaxChunk = 255;          // slabs per traversal chunk (slab ranges are bytes)
constexpr int kStack = 192;             // warp traversal stack depth (up to 31 pushes per wide node)

// Device status block (mirrors rg_status) + work counters.
struct DevStatus {
    unsigned long long hit_pairs;
    unsigned long long slabs;
    unsigned long long slab_cap_exceeded;
    unsigned long long list_passes;
    unsigned long long chunk_splits;
    unsigned long long stack_overflows;
    unsigned long long watchdog_trips;
    unsigned long long nonfinite_inputs;
    unsigned long long traversals;        // warp-level BVH traversals
    unsigned long long node_visits;       // warp-level internal-node visits
    unsigned long long leaf_tests;        // warp-level leaf (ellipsoid) tests
    unsigned long long list_entries;      // hit-list entries appended
    unsigned long long slab_steps;        // warp-level slab iterations with at least one entry
    unsigned long long entry_slabs;       // warp-level (entry, slab) evaluations
    unsigned long long replayed_chunks;   // backward chunks whose list came from the forward record
    unsigned long long record_overflows;  // tiles whose record did not fit the arena
};

// Per-launch view table computed on the device from the camera array (no host sync).
struct ViewTable {
    int n_views;
    int total_tiles;
    long long total_rays;
    int tile_prefix[65];
    long long ray_prefix[65];
};
constexpr int kMaxViews = 64;

// ---- small float3 helpers (own definitions) -------------------------------------------------
__host__ __device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Ordered-int encoding so that float min/max can use integer atomics.
__device__ __forceinline__ int f2ord(float f) {
    int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__host__ __device__ __forceinline__ float ord2f(int i) {
#ifdef __CUDA_ARCH__
    return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff);
#else
    union { int i; float f; } u;
    u.i = i >= 0 ? i : i ^ 0x7fffffff;
    return u.f;
#endif
}

__device__ __forceinline__ float load_param(const void* p, long long i, int storage) {
    if (storage == RG_STORAGE_BF16) return __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(p)[i]);
    return reinterpret_cast<const float*>(p)[i];
}

// 2^x with the SFU (one MUFU.EX2); inputs here are <= 0 and the result may flush to zero.
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// Three-input min / max (one instruction on sm_100)
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
// SFU base-2 logarithm (x <= 0 gives -inf / NaN, which fail every threshold comparison)
__device__ __forceinline__ float lg2_approx(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// tea<4>(v0, v1) seeding and LCG draws of the reference RNG (forward/gaussians_aabb.h:63-94).
__device__ __forceinline__ unsigned tea4(unsigned v0, unsigned v1) {
    unsigned s0 = 0;
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        s0 += 0x9e3779b9u;
        v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + s0) ^ ((v1 >> 5) + 0xc8013ea4u);
        v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + s0) ^ ((v0 >> 5) + 0x7e95761eu);
    }
    return v0;
}
__device__ __forceinline__ float lcg_rnd(unsigned& prev) {
    prev = 1664525u * prev + 1013904223u;
    return (float)(prev & 0x00FFFFFFu) / (float)0x01000000;
}

// Leaf record (leaf order), 64 bytes: {mu.xyz, density}, {M row 0, k}, {M row 1, log2(density)},
// {M row 2, 1 / density} where m = M (x - mu) = S^-1 R^T (x - mu) and k = 1/sqrt(log((density/0.1)^2))
// scales M to the threshold ellipsoid (forward/gaussians_aabb.cu:341-357); the log and reciprocal
// (SFU approximations) serve the fast sample arithmetic.
struct __align__(16) LeafRec {
    float4 a, r0, r1, r2;
};

// Threshold-ellipsoid conic of a leaf in the reference's arithmetic, 48 bytes: the rotation columns
// scaled by 1/(s_j sqrt(log((density/0.1)^2))) (forward/gaussians_aabb.cu:341-357), used by the
// exact ray/ellipsoid interval test of the parity arithmetic; u.w holds sqrt(log((density/0.1)^2)),
// the factor the inference programs scale their sample conic back with.
struct __align__(16) LeafIS {
    float4 u, v, w;
};

// Per-Gaussian pre-pass output in Gaussian order (gathered into leaf order by the BVH build).
struct __align__(16) GaussRec {
    LeafRec s;
    LeafIS is;
};

// Wide traversal nodes.  Every binary node at a depth that is a multiple of kWideLevels owns the
// frontier of its subtree kWideLevels levels down (binary nodes there, or leaves reached earlier):
// at most kWideSlots children, stored as consecutive slots in leaf order.  A slot holds the child's
// box, its id and the last leaf of its subtree (the multi-pass cursor test).  The id of a leaf
// child is ~leaf (< 0); that of a wide child holds the child's own slots, first slot | (count - 1)
// << kWideCountShift (>= 0), so a visit needs no other load.  32 bytes, one 256-bit load per lane.
constexpr int kWideLevels = 5;
constexpr int kWideSlots = 1 << kWideLevels;
constexpr int kWideCountShift = 26;                       // first slot < 2^26: at most 2^25 Gaussians
constexpr long long kMaxGaussians = 1ll << 25;
__host__ __device__ __forceinline__ int wide_pack(int first, int count) {
    return first | ((count - 1) << kWideCountShift);
}
struct __align__(32) WideSlot {
    float lo[3], hi[3];
    int id;
    int range_hi;
};

// BVH internal node, 64 bytes: child boxes, child ids (>= 0 internal, < 0 leaf ~id),
// split position and last leaf of the node's range.
struct __align__(32) Node {   // 32-byte aligned for 256-bit loads
    float4 n0;  // lbox lo.xyz, lbox hi.x
    float4 n1;  // lbox hi.yz, rbox lo.xy
    float4 n2;  // rbox lo.z, rbox hi.xyz
    int4 n3;    // left, right, split, range_hi
};

}  // namespace rg
