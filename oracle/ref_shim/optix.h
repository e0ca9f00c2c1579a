/*
 * Host-side emulation of the OptiX 7 device API calls that the reference's programs make
 * (optix_raycasting/cuda_train/{forward,backward}/gaussians_aabb.cu and the inference programs
 * optix_raycasting/cuda_test/gaussians_aabb.cu) — TEST
 * INFRASTRUCTURE ONLY.  It lets oracle/ref_harness.cpp compile those programs, unmodified,
 * as plain C++ on the CPU so that their own intersection, any-hit, sampling, compositing and
 * adjoint code produce reference outputs for small scenes.
 *
 * Only the traversal is emulated: optixTrace() visits, in primitive-index order, every primitive
 * whose AABB overlaps [tmin, tmax], calls __intersection__gaussian(), and on a reported
 * intersection calls __anyhit__ah(), honouring optixTerminateRay().  The primitives are found
 * through a nested uniform grid over the AABBs (../orc_grid.h) when the scene is bound with one,
 * else from a per-ray scan of all AABBs; both give the same primitives in the same order.  OptiX
 * itself (a closed library) is not used.
 */
#pragma once
#include <vector_types.h>
#include <vector_functions.h>
#include <cmath>
#include <vector>
#include <cstdio>
#include <cstring>
#include <algorithm>

#include "../orc_grid.h"

typedef unsigned long long OptixTraversableHandle;
typedef unsigned int OptixVisibilityMask;
enum { OPTIX_RAY_FLAG_NONE = 0 };

extern "C" void __intersection__gaussian();
extern "C" void __anyhit__ah();

struct RgEmulRay {
    uint3 launch_idx;
    uint3 launch_dim;
    unsigned payload0;
    unsigned payload1, payload2;
    unsigned attr[6];
    unsigned prim;
    float3 o, d;
    float tmin, tmax;
    bool reported;
    bool terminated;
    bool have_cands;
    std::vector<int> cands;
    std::vector<unsigned char> mark;   /* grid query scratch */
    std::vector<int> ids;
    std::vector<long long> key;
};

struct RgEmulScene {
    const float* aabb;  /* (n,6) lo.xyz hi.xyz */
    int n;
    void* sbt_data;
    orc_grid* grid;     /* candidate prefilter (null: scan every AABB per ray) */
    double* box;        /* the AABBs in double for the grid */
};

extern thread_local RgEmulRay rg_emul;
extern RgEmulScene rg_emul_scene;

static inline uint3 optixGetLaunchIndex() { return rg_emul.launch_idx; }
static inline uint3 optixGetLaunchDimensions() { return rg_emul.launch_dim; }
static inline unsigned optixGetPayload_0() { return rg_emul.payload0; }
static inline void optixSetPayload_0(unsigned v) { rg_emul.payload0 = v; }
static inline unsigned optixGetPrimitiveIndex() { return rg_emul.prim; }
static inline float3 optixGetWorldRayOrigin() { return rg_emul.o; }
static inline float3 optixGetWorldRayDirection() { return rg_emul.d; }
static inline float optixGetRayTmin() { return rg_emul.tmin; }
static inline float optixGetRayTmax() { return rg_emul.tmax; }
static inline void* optixGetSbtDataPointer() { return rg_emul_scene.sbt_data; }
static inline bool optixReportIntersection(float t, unsigned /*kind*/) {
    if (t >= rg_emul.tmin && t <= rg_emul.tmax) { rg_emul.reported = true; return true; }
    return false;
}
/* report with six 32-bit attributes (read back by the any-hit program) */
static inline bool optixReportIntersection(float t, unsigned kind, unsigned a0, unsigned a1, unsigned a2,
                                           unsigned a3, unsigned a4, unsigned a5) {
    rg_emul.attr[0] = a0; rg_emul.attr[1] = a1; rg_emul.attr[2] = a2;
    rg_emul.attr[3] = a3; rg_emul.attr[4] = a4; rg_emul.attr[5] = a5;
    return optixReportIntersection(t, kind);
}
static inline unsigned optixGetAttribute_0() { return rg_emul.attr[0]; }
static inline unsigned optixGetAttribute_1() { return rg_emul.attr[1]; }
static inline unsigned optixGetAttribute_2() { return rg_emul.attr[2]; }
static inline unsigned optixGetAttribute_3() { return rg_emul.attr[3]; }
static inline unsigned optixGetAttribute_4() { return rg_emul.attr[4]; }
static inline unsigned optixGetAttribute_5() { return rg_emul.attr[5]; }
static inline unsigned optixGetPayload_1() { return rg_emul.payload1; }
static inline unsigned optixGetPayload_2() { return rg_emul.payload2; }
#ifndef __CUDACC__
static inline unsigned __float_as_uint(float f) { unsigned u; std::memcpy(&u, &f, sizeof u); return u; }
static inline float __uint_as_float(unsigned u) { float f; std::memcpy(&f, &u, sizeof f); return f; }
#endif
static inline void optixTerminateRay() { rg_emul.terminated = true; }
static inline void optixIgnoreIntersection() {}

/* conservative ray/AABB overlap on [tmin, tmax] with a small relative margin */
static inline bool rg_emul_box(const float* bb, float3 o, float3 d, float tmin, float tmax) {
    double tn = tmin, tf = tmax;
    double oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
    for (int a = 0; a < 3; ++a) {
        double ext = 1e-5 * (std::fabs((double)bb[a]) + std::fabs((double)bb[3 + a])) + 1e-7;
        double lo = (double)bb[a] - ext, hi = (double)bb[3 + a] + ext;
        if (dd[a] == 0.0) { if (oo[a] < lo || oo[a] > hi) return false; continue; }
        double t0 = (lo - oo[a]) / dd[a], t1 = (hi - oo[a]) / dd[a];
        if (t0 > t1) { double tt = t0; t0 = t1; t1 = tt; }
        if (t0 > tn) tn = t0;
        if (t1 < tf) tf = t1;
        if (tn > tf) return false;
    }
    return true;
}

/* Binds the scene of one launch: the AABBs, the hit-group record and, with use_grid, a grid over
 * the AABBs inside the scene box. */
static inline void rg_emul_bind(const float* aabb, int n, const float* scene_box, void* sbt, bool use_grid) {
    rg_emul_scene.aabb = aabb;
    rg_emul_scene.n = n;
    rg_emul_scene.sbt_data = sbt;
    rg_emul_scene.grid = nullptr;
    rg_emul_scene.box = nullptr;
    if (!use_grid || n <= 0) return;
    rg_emul_scene.box = (double*)std::malloc(sizeof(double) * 6 * (size_t)n);
    for (long long i = 0; i < 6 * (long long)n; ++i) rg_emul_scene.box[i] = (double)aabb[i];
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = scene_box[a];
        hi[a] = scene_box[3 + a];
        if (!std::isfinite(lo[a]) || !std::isfinite(hi[a]) || !(hi[a] >= lo[a])) { lo[a] = -1.0; hi[a] = 1.0; }
    }
    rg_emul_scene.grid = (orc_grid*)std::malloc(sizeof(orc_grid));
    orc_grid_build(rg_emul_scene.grid, rg_emul_scene.box, n, lo, hi);
}

static inline void rg_emul_unbind() {
    if (rg_emul_scene.grid) {
        orc_grid_free(rg_emul_scene.grid);
        std::free(rg_emul_scene.grid);
        std::free(rg_emul_scene.box);
    }
    rg_emul_scene.grid = nullptr;
    rg_emul_scene.box = nullptr;
}

/* The primitives of one trace call through the grid, in index order. */
static inline void rg_emul_grid_cands(float3 o, float3 d, float tmin, float tmax) {
    const size_t n = (size_t)rg_emul_scene.n;
    if (rg_emul.mark.size() < n) {
        rg_emul.mark.assign(n, 0);
        rg_emul.ids.resize(n);
        rg_emul.key.resize(n);
    }
    double oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
    double t1 = std::isfinite(tmax) ? (double)tmax : 1e300;
    double span = 1e-6 * (std::fabs((double)tmin) + std::fabs(std::isfinite(tmax) ? (double)tmax : 0.0)) + 1e-9;
    int k = orc_grid_query(rg_emul_scene.grid, oo, dd, (double)tmin - span, t1 + span, rg_emul.mark.data(),
                           rg_emul.ids.data());
    orc_grid_unmark(rg_emul.mark.data(), rg_emul.ids.data(), k);
    orc_grid_sort(rg_emul.ids.data(), k, nullptr, rg_emul.key.data());
    rg_emul.cands.assign(rg_emul.ids.begin(), rg_emul.ids.begin() + k);
}

static inline void optixTrace(OptixTraversableHandle, float3 o, float3 d, float tmin, float tmax, float,
                              OptixVisibilityMask, unsigned, unsigned, unsigned, unsigned, unsigned& p0) {
    if (rg_emul_scene.grid) {
        rg_emul_grid_cands(o, d, tmin, tmax);
    } else if (!rg_emul.have_cands) {
        rg_emul.cands.clear();
        for (int g = 0; g < rg_emul_scene.n; ++g)
            if (rg_emul_box(rg_emul_scene.aabb + 6 * g, o, d, 0.0f, INFINITY)) rg_emul.cands.push_back(g);
        rg_emul.have_cands = true;
    }
    rg_emul.o = o; rg_emul.d = d; rg_emul.tmin = tmin; rg_emul.tmax = tmax;
    rg_emul.payload0 = p0;
    rg_emul.terminated = false;
    for (int g : rg_emul.cands) {
        if (!rg_emul_box(rg_emul_scene.aabb + 6 * g, o, d, tmin, tmax)) continue;
        rg_emul.prim = (unsigned)g;
        rg_emul.reported = false;
        __intersection__gaussian();
        if (rg_emul.reported) {
            __anyhit__ah();
            if (rg_emul.terminated) break;
        }
    }
    p0 = rg_emul.payload0;
}

/* three-payload form (payloads 1 and 2 carry a pointer to the caller's sample buffer) */
static inline void optixTrace(OptixTraversableHandle h, float3 o, float3 d, float tmin, float tmax, float rt,
                              OptixVisibilityMask m, unsigned f, unsigned a, unsigned b, unsigned c, unsigned& p0,
                              unsigned& p1, unsigned& p2) {
    rg_emul.payload1 = p1;
    rg_emul.payload2 = p2;
    optixTrace(h, o, d, tmin, tmax, rt, m, f, a, b, c, p0);
}

/* device atomics used by the programs, made thread-safe for the OpenMP ray loop */
static inline int atomicAdd(int* a, int v) { int old; _Pragma("omp atomic capture") { old = *a; *a += v; } return old; }
static inline float atomicAdd(float* a, float v) { float old; _Pragma("omp atomic capture") { old = *a; *a += v; } return old; }
