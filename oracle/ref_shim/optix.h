/*
 * Host-side emulation of the OptiX 7 device API calls that the reference's programs make
 * (optix_raycasting/cuda_train/{forward,backward}/gaussians_aabb.cu and the inference programs
 * optix_raycasting/cuda_test/gaussians_aabb.cu) — TEST
 * INFRASTRUCTURE ONLY.  It lets oracle/ref_harness.cpp compile those programs, unmodified,
 * as plain C++ on the CPU so that their own intersection, any-hit, sampling, compositing and
 * adjoint code produce reference outputs for small scenes.
 *
 * Only the traversal is emulated: optixTrace() visits every primitive of a per-ray candidate
 * list whose AABB overlaps [tmin, tmax], calls __intersection__gaussian(), and on a reported
 * intersection calls __anyhit__ah(), honouring optixTerminateRay().  OptiX itself (a closed
 * library) is not used.
 */
#pragma once
#include <vector_types.h>
#include <vector_functions.h>
#include <cmath>
#include <vector>
#include <cstdio>
#include <cstring>

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
};

struct RgEmulScene {
    const float* aabb;  /* (n,6) lo.xyz hi.xyz */
    int n;
    void* sbt_data;
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

static inline void optixTrace(OptixTraversableHandle, float3 o, float3 d, float tmin, float tmax, float,
                              OptixVisibilityMask, unsigned, unsigned, unsigned, unsigned, unsigned& p0) {
    if (!rg_emul.have_cands) {
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
