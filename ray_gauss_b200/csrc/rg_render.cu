// Persistent, warp-cooperative ray-casting kernels: forward (density/colour sampling, alpha
// compositing, early termination) and the recompute-based adjoint.
//
// Reference semantics (paths inside the reference project):
//   ray generation            optix_raycasting/cuda_train/forward/gaussians_aabb.cu:405-434
//   scene-box clip, slab loop :521-612 (slab = 8 samples x 0.0025 starting at the box entry,
//                             per-slab early-exit test T > 0.003, samples past the box exit in the
//                             last slab are still evaluated)
//   exact ellipsoid test      :324-402 (including its root-order behaviour for b <= 0)
//   sample buffers            :437-498, compositing :500-519
//   adjoint                   optix_raycasting/cuda_train/backward/gaussians_aabb.cu:505-775
//
// Design.  A warp owns an 8x4 pixel tile (tiles of all views are pulled from one atomic work
// counter).  Each lane marches its own ray with the reference's slab sequence (tb += 0.02 in
// FP32); the warp advances in chunks of K slabs per lane (K adapts between 1 and 255: it grows
// while hits are sparse and halves when the hit list overflows).  For a chunk the warp traverses
// the wide BVH once for the packet of its lanes' segments (one child slot per lane, tested with
// interval arithmetic over the lanes' directions) with a warp-uniform stack, runs the exact
// ellipsoid test per lane at the leaves
// and appends every leaf that any lane hits to a shared hit
// list with, per lane, the range of the chunk's slabs its interval covers (exact for K <= 8; one
// slab of margin on each side for longer chunks, where the extra slabs' samples fall outside the
// threshold ellipsoid and are masked out).  The list is consumed slab by slab: each lane evaluates
// only entries whose range holds the slab, reading the leaf record with a warp-uniform (broadcast)
// load.  A full list for a single slab is consumed in several passes (a leaf-index cursor skips
// the leaves already taken; DFS order visits leaves in increasing index), so no hit is dropped.
// The adjoint recomputes each slab's sample buffers, folds the compositing adjoint into three
// scalars per sample, evaluates each Gaussian's gradient per lane, reduces it across the warp with
// a transposed shuffle reduction (16 shuffles for 14 values) and issues one atomic per value.
//
// Sample arithmetic.  RG_MODE_PARITY evaluates samples, ray generation and compositing in the
// reference's operation order with IEEE round-to-nearest operations (no FMA contraction); when a
// sample's density*weight lies within a few ulps of the 0.1 threshold the weight is re-evaluated
// with a correctly rounded exponential so the threshold decision matches the FP32 reference
// arithmetic.  RG_MODE_FAST evaluates the 8 samples of a slab from the quadratic form of the
// Mahalanobis distance along the ray with the SFU exponential and accumulates the adjoint in
// moment form.
#include <cstddef>

#include "rg_common.cuh"
#include "rg_kernels.h"

namespace rg {

constexpr int kWarpsPerBlock = 4;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxRounds = 1 << 20;        // chunk rounds per tile before the watchdog trips
constexpr float kNegHalfLog2e = -0.72134752044448170f;
constexpr float kLog2SigThr = -3.3219280948873623f;   // log2(0.1): per-sample density threshold
constexpr float kInvSlab = 50.0f;          // 1 / 0.02
constexpr int kExactChunk = 8;             // chunks up to this length use exact slab ranges
constexpr int kCounters = 9;
#ifndef RG_DIRECT_ATOMIC_LANES
#define RG_DIRECT_ATOMIC_LANES 24  // up to this many contributing lanes add with float4 atomics directly
#endif               // per-warp counters: the WarpStats fields, hit pairs, slabs
constexpr unsigned kNoRecord = 0xffffffffu;     // hit-list record: no (next) chunk record
constexpr unsigned kRecordMulti = 0x80000000u;  // chunk consumed in several traversal passes
constexpr unsigned kRecordFailed = 0xfffffffeu; // the tile's record did not fit the arena

// Warp hit-list layout.  Parity arithmetic keeps, per entry and lane, the exact range of the
// chunk's slabs the lane's interval covers (64 B per entry); the fast arithmetic keeps only the mask
// of lanes whose interval overlaps the chunk (4 B per entry) and lets those lanes evaluate every
// slab of the entry's union range (samples outside the lane's interval fall outside the threshold
// ellipsoid and are masked out), which allows 4x longer lists and so 4x longer chunks in dense
// regions.
template <bool FAST, int CAP>
struct WarpSmem {
    static constexpr int MB = FAST ? 4 : 2;         // slabs per entry-mask block
    static constexpr int NB = 64;                   // entry-mask blocks
    static constexpr int KM = FAST ? 255 : 128;     // longest chunk (MB * NB, slab ranges are bytes)
    int ids[CAP];
    unsigned urng[CAP];                              // union of the lanes' slab ranges: lo | hi << 16
    unsigned lmask[FAST ? CAP : 1];                  // fast: lanes whose interval overlaps the chunk
    unsigned short lrng[FAST ? 1 : CAP][32];         // parity: per lane lo | hi << 8 (lo > hi: no hit)
    unsigned smask[NB][CAP / 32];                    // entries whose union range meets block k / MB
    unsigned long long occ[4];                       // slabs holding any entry (union occupancy)
    __align__(16) float packet[24];                  // the chunk's ray packet (set_packet), read as float4
    int stack[kStack];
    // hit-list record of the warp's current tile (written by lane 0)
    unsigned rec_first, rec_prev;                    // forward: first / last chunk record
    unsigned rec_cur;                                // backward: next chunk record to replay
    unsigned long long cnt[kCounters];               // activity counters of the warp (lane 0)
};

// Warp-uniform activity counters of one tile (32-bit; added to the warp's shared-memory totals at
// the end of the tile so that few registers stay live through the traversal and slab loops).
struct WarpStats {
    unsigned traversals = 0, node_visits = 0, leaf_tests = 0, entries = 0, slab_steps = 0, entry_slabs = 0,
             replays = 0;
};

struct RayState {
    float3 o, d;
    float tenter, texit;
    float tb;
    float T;
    float3 C;     // forward: accumulated colour
    float3 g;     // backward: dL/dcolour of the ray
    float gR;     // backward: g . R, R the colour still to come (the adjoint needs only this product)
    unsigned seed;
    bool alive;
};

// ---- IEEE-ordered helpers (no contraction) for the parity arithmetic ----------------------------
__device__ __forceinline__ float dot_rn(float3 a, float3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ float3 rows_rn(float3 r0, float3 r1, float3 r2, float3 v) {
    return f3(dot_rn(r0, v), dot_rn(r1, v), dot_rn(r2, v));
}

// One wide-node child slot (32 bytes) in one 256-bit read-only load.
__device__ __forceinline__ void load_slot(const WideSlot* p, float3& lo, float3& hi, int& id, int& range_hi) {
    float f[6];
    int u[2];
    asm("ld.global.nc.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(f[0]), "=f"(f[1]), "=f"(f[2]), "=f"(f[3]), "=f"(f[4]), "=f"(f[5]), "=r"(u[0]), "=r"(u[1])
        : "l"(p));
    lo = f3(f[0], f[1], f[2]);
    hi = f3(f[3], f[4], f[5]);
    id = u[0];
    range_hi = u[1];
}

// The chunk's ray packet for the wide-node test (interval arithmetic).  All rays start at the eye;
// over the active lanes, per axis the direction component lies in [dmin, dmax] and the ray
// parameter of the chunk segments in [tmin, tmax].  For a box, a ray's entry and exit parameters
// along axis a are the smaller and larger of (lo_a - o_a) / d_a and (hi_a - o_a) / d_a, linear in
// 1 / d_a: over the packet they lie between the products at the ends of the 1 / d interval, so the
// box can meet a segment only if the largest of the smallest entries (and tmin) does not exceed
// the smallest of the largest exits (and tmax).  Exact for one ray, conservative for a packet, tight
// for the nearly parallel rays of a tile.  An axis whose direction interval holds 0 gives no bound
// there; the box of the packet's segments (o + t d over the t and d intervals) bounds every axis.
// Stored per axis {1/dmax, 1/dmin, -o/dmax, -o/dmin}, then {tmin - slack, tmax + slack}, then the
// segments' box {lo.xyz, -}, {hi.xyz, -} widened by a position slack.  The
// products round like the per-ray slab test's t = b/d - o/d: a few ulps of |o| in position, far
// inside the leaf boxes' 1e-5 inflation, so the bound needs no slack of its own; a small one in t
// covers the ends of the segments.  (A slack that grows with 1/|d| would stretch the packets of
// rays nearly parallel to a coordinate plane over most of their length.)
template <bool FAST, int CAP>
__device__ __forceinline__ void set_packet(WarpSmem<FAST, CAP>& sm, const RayState& r, bool on, float seg_hi,
                                           int lane) {
    float dmin[3], dmax[3];
    const float dv[3] = {r.d.x, r.d.y, r.d.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        dmin[a] = ord2f(__reduce_min_sync(kFull, on ? f2ord(dv[a]) : 0x7fffffff));
        dmax[a] = ord2f(__reduce_max_sync(kFull, on ? f2ord(dv[a]) : (int)0x80000000));
    }
    const float tmin = __uint_as_float(__reduce_min_sync(kFull, on ? __float_as_uint(fmaxf(r.tb, 0.f)) : 0x7f800000u));
    const float tmax = __uint_as_float(__reduce_max_sync(kFull, on ? __float_as_uint(fmaxf(seg_hi, 0.f)) : 0u));
    if (lane == 0) {
        const float ov[3] = {r.o.x, r.o.y, r.o.z};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            float4 q;
            if (!(dmin[a] > 0.f) && !(dmax[a] < 0.f)) {
                q = make_float4(0.f, 0.f, -INFINITY, INFINITY);   // the interval holds 0: no bound
            } else {
                const float rA = 1.f / dmax[a], rB = 1.f / dmin[a];
                q = make_float4(rA, rB, -ov[a] * rA, -ov[a] * rB);
            }
            *reinterpret_cast<float4*>(sm.packet + 4 * a) = q;
        }
        const float slack = 1e-6f * (tmax + 1.f);
        *reinterpret_cast<float4*>(sm.packet + 12) = make_float4(tmin - slack, tmax + slack, 0.f, 0.f);
        const float pslack = 1e-6f * (fabsf(ov[0]) + fabsf(ov[1]) + fabsf(ov[2]) + tmax + 1.f);
        float bl[3], bh[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float e0 = tmin * dmin[a], e1 = tmin * dmax[a], e2 = tmax * dmin[a], e3 = tmax * dmax[a];
            bl[a] = ov[a] + fminf(fminf(e0, e1), fminf(e2, e3)) - pslack;
            bh[a] = ov[a] + fmaxf(fmaxf(e0, e1), fmaxf(e2, e3)) + pslack;
        }
        *reinterpret_cast<float4*>(sm.packet + 16) = make_float4(bl[0], bl[1], bl[2], 0.f);
        *reinterpret_cast<float4*>(sm.packet + 20) = make_float4(bh[0], bh[1], bh[2], 0.f);
    }
    __syncwarp();
}

__device__ __forceinline__ void packet_axis(float4 q, float lo, float hi, float& tin, float& tout) {
    const float p1 = fmaf(lo, q.x, q.z), p2 = fmaf(lo, q.y, q.w), p3 = fmaf(hi, q.x, q.z), p4 = fmaf(hi, q.y, q.w);
    tin = fminf(fminf(p1, p2), fminf(p3, p4));
    tout = fmaxf(fmaxf(p1, p2), fmaxf(p3, p4));
}

// Whether a box may meet a segment of the packet (see set_packet).
__device__ __forceinline__ bool packet_hit(const float* F, float3 lo, float3 hi) {
    const float4 qx = *reinterpret_cast<const float4*>(F), qy = *reinterpret_cast<const float4*>(F + 4),
                 qz = *reinterpret_cast<const float4*>(F + 8), qt = *reinterpret_cast<const float4*>(F + 12);
    const float4 bl = *reinterpret_cast<const float4*>(F + 16), bh = *reinterpret_cast<const float4*>(F + 20);
    float ix, ox, iy, oy, iz, oz;
    packet_axis(qx, lo.x, hi.x, ix, ox);
    packet_axis(qy, lo.y, hi.y, iy, oy);
    packet_axis(qz, lo.z, hi.z, iz, oz);
    const bool in_box = lo.x <= bh.x && hi.x >= bl.x && lo.y <= bh.y && hi.y >= bl.y && lo.z <= bh.z && hi.z >= bl.z;
    return in_box && fmaxf(max3f(ix, iy, iz), qt.x) <= fminf(min3f(ox, oy, oz), qt.y);
}

__device__ __forceinline__ LeafRec load_rec(const LeafRec* p, int i) {
    const float4* q = reinterpret_cast<const float4*>(p + i);
    LeafRec r;
    r.a = __ldg(q);
    r.r0 = __ldg(q + 1);
    r.r1 = __ldg(q + 2);
    r.r2 = __ldg(q + 3);
    return r;
}

// Ray/ellipsoid interval in the reference intersection program's arithmetic
// (forward/gaussians_aabb.cu:359-381): IEEE operations in source order on the precomputed
// threshold-scaled conic.  Returns false when disc <= 1e-7 (no report).
__device__ __forceinline__ bool roots_exact(const LeafIS& s, float3 mu, const RayState& r, float& root1,
                                            float& root2) {
    float3 U = f3(s.u.x, s.u.y, s.u.z), V = f3(s.v.x, s.v.y, s.v.z), W = f3(s.w.x, s.w.y, s.w.z);
    float3 O = f3(__fsub_rn(r.o.x, mu.x), __fsub_rn(r.o.y, mu.y), __fsub_rn(r.o.z, mu.z));
    float3 Oe = f3(dot_rn(U, O), dot_rn(V, O), dot_rn(W, O));
    float3 De = f3(dot_rn(U, r.d), dot_rn(V, r.d), dot_rn(W, r.d));
    float l = __fdiv_rn(1.f, __fsqrt_rn(dot_rn(De, De)));
    float3 D = f3(__fmul_rn(De.x, l), __fmul_rn(De.y, l), __fmul_rn(De.z, l));
    float b = -dot_rn(Oe, D);
    float c = __fsub_rn(dot_rn(Oe, Oe), 1.f);
    float3 p = f3(__fadd_rn(Oe.x, __fmul_rn(D.x, b)), __fadd_rn(Oe.y, __fmul_rn(D.y, b)),
                  __fadd_rn(Oe.z, __fmul_rn(D.z, b)));
    float disc = __fsub_rn(1.f, dot_rn(p, p));
    if (!(disc > 1e-7f)) return false;
    float sd = __fsqrt_rn(disc);
    float q = __fadd_rn(b, b > 0.f ? sd : -sd);
    root1 = __fmul_rn(__fdiv_rn(c, q), l);
    root2 = __fmul_rn(q, l);
    return true;
}

// The same interval from the sampling conic scaled by the threshold factor k (fast arithmetic).
__device__ __forceinline__ bool roots_fast(const LeafRec& rec, const RayState& r, float& root1, float& root2) {
    float3 O = r.o - f3(rec.a.x, rec.a.y, rec.a.z);
    float k = rec.r0.w;
    float3 r0 = f3(rec.r0.x, rec.r0.y, rec.r0.z), r1 = f3(rec.r1.x, rec.r1.y, rec.r1.z),
           r2 = f3(rec.r2.x, rec.r2.y, rec.r2.z);
    float3 Oe = f3(dot3(r0, O) * k, dot3(r1, O) * k, dot3(r2, O) * k);
    float3 De = f3(dot3(r0, r.d) * k, dot3(r1, r.d) * k, dot3(r2, r.d) * k);
    // SFU reciprocal square roots and a fast division (the fast arithmetic's interval ends move by
    // ulps; the forward and the backward's replay run this same test)
    float l = rsqrtf(dot3(De, De));
    float3 Dn = De * l;
    float b = -dot3(Oe, Dn);
    float c = dot3(Oe, Oe) - 1.f;
    float3 p = Oe + Dn * b;
    float disc = 1.f - dot3(p, p);
    if (!(disc > 1e-7f)) return false;
    float sd = disc * rsqrtf(disc);
    float q = b + (b > 0.f ? sd : -sd);   // |q| >= sd > 3e-4
    root1 = __fdividef(c, q) * l;
    root2 = q * l;
    return true;
}

__device__ __forceinline__ LeafIS load_is(const LeafIS* p, int i) {
    const float4* q = reinterpret_cast<const float4*>(p + i);
    LeafIS s;
    s.u = __ldg(q);
    s.v = __ldg(q + 1);
    s.w = __ldg(q + 2);
    return s;
}

// Slab range [lo, hi] of the chunk (K slabs from r.tb) hit by the interval [root1, root2].
// Slab k of the chunk against the interval, in slab units from tb (a, b: interval ends, e: box
// exit) with tb_k = k up to the margin m: 1 certain hit, -1 certain miss, 0 undecided.  Slab k is
// hit iff root1 <= min(texit, tb_k + 0.02), tb_k <= root2 and root1 <= root2.
__device__ __forceinline__ int classify_slab(int k, float a, float b, float e, float m) {
    const float kf = (float)k;
    if (a > b || a > kf + 1.f + m || a > e + m || kf - m > b) return -1;
    if (a <= kf + 1.f - m && a <= e - m && kf + m <= b) return 1;
    return 0;
}

// The reference's test for slab k of the chunk, tb_k by k repeated FP32 additions from tb.
__device__ __noinline__ bool slab_k_hit(float tb, float tenter, float texit, int k, float root1, float root2) {
    float t = tb;
    for (int j = 0; j < k; ++j) t = t + kSlab;
    const float th = fminf(texit, t + kSlab);
    return th > tenter && fmaxf(t, root1) <= fminf(th, root2);
}

// Longer chunks map the interval arithmetically.  Slab k starts at tb_k, tb plus k slabs by repeated
// FP32 addition, and is hit iff root1 <= tb_k + 0.02 and tb_k <= root2.  The range keeps a margin
// that covers the drift of the repeated addition, so it holds every hit slab and at most one extra
// slab at each end: the parity arithmetic settles the ends exactly here, the fast arithmetic
// evaluates them (their samples fall outside the threshold ellipsoid).
template <bool FAST>
__device__ __forceinline__ void slab_range(const RayState& r, int K, int nv, float seg_hi, float tclip, float root1,
                                           float root2, int& lo, int& hi) {
    lo = 255;
    hi = -1;
    if (K <= kExactChunk) {
        // exact: the reference's per-slab test max(tmin, root1) <= min(tmax, root2)
        float t = r.tb;
#pragma unroll
        for (int kk = 0; kk < kExactChunk; ++kk) {
            if (kk < nv) {
                float tn = t + kSlab;
                float th = fminf(tclip, tn);
                if (th > r.tenter && fmaxf(t, root1) <= fminf(th, root2)) {
                    lo = min(lo, kk);
                    hi = kk;
                }
                t = tn;
            }
        }
    } else if (fmaxf(r.tb, root1) <= fminf(seg_hi, root2)) {
        float a = fmaxf((root1 - r.tb) * kInvSlab, -1.f);
        float b = fminf((root2 - r.tb) * kInvSlab, 4096.f);
        // drift of tb_k in slab units: (K + 1) ulps of |tb| + K slabs, 2^-23 relative each (four
        // times the bound of round-to-nearest additions)
        const float m = (float)(K + 1) * (fabsf(r.tb) + (float)K * kSlab) * (kInvSlab * 2.4e-7f) + 1e-4f;
        lo = max(0, (int)ceilf(a - 1.f - m));
        hi = min(K - 1, (int)floorf(b + m));
        if (!FAST) {
            // Parity: settle both ends exactly.  A slab whose hit or miss the margins cannot decide
            // gets the reference's per-slab test (rare: its interval end lies within the margin
            // of a slab edge or of the box exit).
            const float e = fminf((tclip - r.tb) * kInvSlab, 4096.f);
            while (lo <= hi) {
                const int c = classify_slab(lo, a, b, e, m);
                if (c > 0 || (c == 0 && slab_k_hit(r.tb, r.tenter, tclip, lo, root1, root2))) break;
                ++lo;
            }
            while (hi >= lo) {
                const int c = classify_slab(hi, a, b, e, m);
                if (c > 0 || (c == 0 && slab_k_hit(r.tb, r.tenter, tclip, hi, root1, root2))) break;
                --hi;
            }
        }
        if (lo > hi) { lo = 255; hi = -1; }
    }
}

// 32-entry mask words holding `count` list entries.
__device__ __forceinline__ int nwords(int count) { return (count + 31) >> 5; }

// Union occupancy of the chunk's slabs (256 bits): bit k set when some lane has a hit in slab k.
__device__ __forceinline__ void occ_set(unsigned long long* occ, int lo, int hi) {
#pragma unroll
    for (int w = 0; w < 4; ++w) {
        int a0 = max(lo, 64 * w), b0 = min(hi, 64 * w + 63);
        if (a0 <= b0) {
            int n = b0 - a0 + 1;
            unsigned long long m = (n == 64) ? ~0ull : (((1ull << n) - 1ull) << (a0 - 64 * w));
            occ[w] |= m;
        }
    }
}
__device__ __forceinline__ bool occ_test(const unsigned long long* occ, int k) {
    return (occ[k >> 6] >> (k & 63)) & 1ull;
}
// first occupied slab >= k (K when none)
__device__ __forceinline__ int occ_next(const unsigned long long* occ, int k, int K) {
    for (int w = k >> 6; w < 4 && 64 * w < K; ++w) {
        unsigned long long m = occ[w];
        if (w == (k >> 6)) m &= (~0ull) << (k & 63);
        if (m) return min(K, 64 * w + __ffsll((long long)m) - 1);
    }
    return K;
}

template <bool FAST, int CAP>
__device__ __forceinline__ void clear_occ(WarpSmem<FAST, CAP>& sm, int lane) {
    if (lane == 0) {
#pragma unroll
        for (int w = 0; w < 4; ++w) sm.occ[w] = 0ull;
    }
}

// Adds the tile's counters to the warp's totals and resets them.
template <bool FAST, int CAP, bool DIAG>
__device__ __forceinline__ void flush_stats(WarpSmem<FAST, CAP>& sm, WarpStats& ws, unsigned hits, unsigned slabs,
                                            int lane) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        hits += __shfl_xor_sync(kFull, hits, o);
        slabs += __shfl_xor_sync(kFull, slabs, o);
    }
    if (lane == 0) {
        sm.cnt[0] += ws.traversals;
        if (DIAG) {
            sm.cnt[1] += ws.node_visits;
            sm.cnt[2] += ws.leaf_tests;
            sm.cnt[3] += ws.entries;
            sm.cnt[4] += ws.slab_steps;
            sm.cnt[5] += ws.entry_slabs;
        }
        sm.cnt[6] += ws.replays;
        sm.cnt[7] += hits;
        sm.cnt[8] += slabs;
    }
    ws = WarpStats();
}

// Exact leaf test of every active lane for the chunk [tb, seg_hi]: appends the leaf to the warp
// list when any lane's interval meets one of the chunk's slabs.  Returns false (leaf not taken)
// when the list is already full.
template <bool FAST, int CAP, bool DIAG>
__device__ __forceinline__ bool leaf_entry(WarpSmem<FAST, CAP>& sm, const RenderArgs& a, const RayState& r, bool on,
                                           float seg_hi, int K, int nv, int leaf, int& count, int lane,
                                           WarpStats& ws, bool infer) {
    if (DIAG) ++ws.leaf_tests;
    int lo = 255, hi = -1;
    if (on) {
        float root1, root2;
        bool ok;
        if (FAST) {
            ok = roots_fast(load_rec(a.rec, leaf), r, root1, root2);
        } else {
            float4 m4 = __ldg(reinterpret_cast<const float4*>(a.rec + leaf));
            ok = roots_exact(load_is(a.is_rec, leaf), f3(m4.x, m4.y, m4.z), r, root1, root2);
        }
        // the slab query ends at the box exit in training launches and at the slab end in
        // inference launches (cuda_test/gaussians_aabb.cu:408-409)
        const float tclip = infer ? INFINITY : r.texit;
        if (ok) slab_range<FAST>(r, K, nv, seg_hi, tclip, root1, root2, lo, hi);
    }
    unsigned any = __ballot_sync(kFull, lo <= hi);
    if (!any) return true;
    if (count == CAP) return false;
    int ulo = (int)__reduce_min_sync(kFull, (unsigned)lo);
    int uhi = (int)__reduce_max_sync(kFull, (unsigned)(hi + 1)) - 1;
    if (FAST) {
        if (lane == 0) sm.lmask[count] = any;
    } else {
        sm.lrng[count][lane] = (unsigned short)((lo & 0xff) | ((hi & 0xff) << 8));
    }
    if (lane == 0) {
        sm.ids[count] = leaf;
        sm.urng[count] = (unsigned)ulo | ((unsigned)uhi << 16);
        occ_set(sm.occ, ulo, uhi);
    }
    ++count;
    return true;
}

// Publishes the chunk list: occupancy bits and the entry masks per block of MB slabs.
template <bool FAST, int CAP, bool DIAG>
__device__ __forceinline__ void finish_list(WarpSmem<FAST, CAP>& sm, int count, int K, int lane, WarpStats& ws) {
    __syncwarp();
    if (DIAG) ws.entries += count;
    // lane l fills blocks l, l+32
    constexpr int MB = WarpSmem<FAST, CAP>::MB;
    const int nblk = (K + MB - 1) / MB;
    const int nw = nwords(count);
    for (int bk = lane; bk < nblk; bk += 32) {
        const int k0 = bk * MB, k1 = k0 + MB - 1;
#pragma unroll 1
        for (int w = 0; w < nw; ++w) {
            unsigned mw = 0u;
            const int e0 = 32 * w, e1 = min(count, e0 + 32);
#pragma unroll 1
            for (int e = e0; e < e1; ++e) {
                unsigned u = sm.urng[e];
                if (k1 >= (int)(u & 0xffff) && k0 <= (int)(u >> 16)) mw |= 1u << (e - e0);
            }
            sm.smask[bk][w] = mw;
        }
    }
    __syncwarp();
}

// Warp-cooperative traversal for the chunk [tb, seg_hi] of every active lane (the packet set by
// set_packet).  At a wide node lane k tests child slot k against the packet; the first hit child is
// visited next and the others wait on the stack, the lowest index on top, so leaves are reached in
// increasing index (the multi-pass cursor relies on it).  Appends hit leaves with index > cursor to
// the warp list; returns the entry count.  `ovf` is set when the list filled up before the
// traversal finished.
template <bool FAST, int CAP, bool DIAG>
__device__ int traverse(WarpSmem<FAST, CAP>& sm, const RenderArgs& a, const RayState& r, bool on, float seg_hi,
                        int K, int nv, int cursor, bool& ovf, int lane, WarpStats& ws, bool infer) {
    int count = 0;
    ++ws.traversals;
    ovf = false;
    clear_occ(sm, lane);
    int sp = 0;
    int cur = ~0;   // one Gaussian: the root is a leaf
    if (a.n_leaves > 1) {
        const int2 root = __ldg(a.wide_tab);
        cur = wide_pack(root.x, root.y);
    }
    unsigned guard = 0, visits = 0;
    const unsigned guard_max = 2u * (unsigned)a.n_leaves + 64u;
    while (true) {
        if (++guard > guard_max) {
            if (lane == 0) atomicAdd(&a.st->watchdog_trips, 1ull);
            break;
        }
        if (cur >= 0) {
            if (DIAG) ++visits;
            const int first = cur & ((1 << kWideCountShift) - 1), count = (cur >> kWideCountShift) + 1;
            bool hit = false;
            int cid = 0;
            if (lane < count) {
                float3 lo, hi;
                int range_hi;
                load_slot(a.slots + first + lane, lo, hi, cid, range_hi);
                hit = (range_hi > cursor) && packet_hit(sm.packet, lo, hi);
            }
            const unsigned hm = __ballot_sync(kFull, hit);
            if (hm) {
                // continue with the first hit child; the later ones go on the stack in reverse order
                // (the hit child k at the position of the hit children above it), lowest on top
                const int f = __ffs(hm) - 1;
                const unsigned rest = hm & (hm - 1u);
                const int np = __popc(rest);
                if (sp + np <= kStack) {
                    if ((rest >> lane) & 1u) sm.stack[sp + __popc(rest >> lane) - 1] = cid;
                    sp += np;
                } else if (lane == 0) {
                    atomicAdd(&a.st->stack_overflows, 1ull);
                }
                cur = __shfl_sync(kFull, cid, f);
                __syncwarp();
                continue;
            }
        } else {
            int leaf = ~cur;
            if (leaf > cursor && !leaf_entry<FAST, CAP, DIAG>(sm, a, r, on, seg_hi, K, nv, leaf, count, lane, ws, infer)) {
                ovf = true;
                break;
            }
        }
        if (sp == 0) break;
        cur = sm.stack[--sp];
    }
    if (DIAG) ws.node_visits += visits;
    finish_list<FAST, CAP, DIAG>(sm, count, K, lane, ws);
    return count;
}

// The chunk list from the forward's record: the recorded leaves (at most the list capacity) get
// the same exact leaf test as in a traversal, without the traversal.
template <bool FAST, int CAP, bool DIAG>
__device__ int replay_list(WarpSmem<FAST, CAP>& sm, const RenderArgs& a, const RayState& r, bool on, float seg_hi,
                           int K, int nv, const unsigned* ids, int n, int lane, WarpStats& ws) {
    int count = 0;
    clear_occ(sm, lane);
    n = min(n, CAP);
    for (int base = 0; base < n; base += 32) {
        const int m = min(32, n - base);
        const int mine = lane < m ? (int)ids[base + lane] : 0;
#pragma unroll 1
        for (int j = 0; j < m; ++j) {
            const int leaf = __shfl_sync(kFull, mine, j);
            if (leaf >= 0 && leaf < a.n_leaves)
                leaf_entry<FAST, CAP, DIAG>(sm, a, r, on, seg_hi, K, nv, leaf, count, lane, ws, false);
        }
    }
    finish_list<FAST, CAP, DIAG>(sm, count, K, lane, ws);
    return count;
}

// Per-slab sample offsets beyond i*dt (rnd_sample 1: random; 2+: half step).  Returns the seed
// after the slab's draws (used only when the slab had hits).
__device__ __forceinline__ unsigned slab_offsets(int rnd_sample, unsigned seed, float* roff) {
    if (rnd_sample == 1) {
#pragma unroll
        for (int i = 0; i < kBuf; ++i) roff[i] = lcg_rnd(seed) * kDt;
    } else {
#pragma unroll
        for (int i = 0; i < kBuf; ++i) roff[i] = (rnd_sample == 0) ? 0.f : 0.5f * kDt;
    }
    return seed;
}

// Exponent -|M (o + t d - mu)|^2 / 2 of a sample in the reference's operation order.
__device__ __forceinline__ float parity_power(float3 o, float3 d, float t, float3 mu, float3 r0, float3 r1,
                                              float3 r2) {
    const float3 x = f3(__fadd_rn(o.x, __fmul_rn(d.x, t)), __fadd_rn(o.y, __fmul_rn(d.y, t)),
                        __fadd_rn(o.z, __fmul_rn(d.z, t)));
    const float3 v = f3(__fsub_rn(x.x, mu.x), __fsub_rn(x.y, mu.y), __fsub_rn(x.z, mu.z));
    const float3 m = rows_rn(r0, r1, r2, v);
    return __fmul_rn(-0.5f, dot_rn(m, m));
}

__device__ __forceinline__ float parity_time(float tb, int i, int rnd_sample, const float* roff) {
    float t = __fadd_rn(tb, __fmul_rn((float)i, kDt));
    if (rnd_sample) t = __fadd_rn(t, roff[i]);
    return t;
}

// Reference-order weights w[i] of the 8 samples of a slab for one Gaussian, and the mask of the
// samples whose density * weight exceeds 0.1.  The eight weights are computed first, without
// branches, so their dependency chains interleave; a sample whose density * weight lies within the
// exponential's error of 0.1 is then re-evaluated with a correctly rounded weight, so that the
// threshold decision is the one of the FP32 reference arithmetic.
__device__ __forceinline__ unsigned parity_weights(const RayState& r, int rnd_sample, const float* roff, float3 mu,
                                                   float3 r0, float3 r1, float3 r2, float dn, float* w) {
    unsigned near = 0u;
#pragma unroll
    for (int i = 0; i < kBuf; ++i) {
        w[i] = expf(parity_power(r.o, r.d, parity_time(r.tb, i, rnd_sample, roff), mu, r0, r1, r2));
        near |= (fabsf(__fmul_rn(dn, w[i]) - kSigThr) < 4e-8f ? 1u : 0u) << i;
    }
    if (near) {
#pragma unroll
        for (int i = 0; i < kBuf; ++i) {
            if ((near >> i) & 1u)
                w[i] = (float)exp((double)parity_power(r.o, r.d, parity_time(r.tb, i, rnd_sample, roff), mu, r0, r1,
                                                       r2));
        }
    }
    unsigned in = 0u;
#pragma unroll
    for (int i = 0; i < kBuf; ++i) in |= (__fmul_rn(dn, w[i]) > kSigThr ? 1u : 0u) << i;
    return in;
}

__device__ __forceinline__ bool in_range(unsigned short rg, int k) {
    return k >= (int)(rg & 0xff) && k <= (int)(rg >> 8);
}
__device__ __forceinline__ bool in_urange(unsigned u, int k) {
    return k >= (int)(u & 0xffff) && k <= (int)(u >> 16);
}

// Whether the lane holds list entry e in slab k: the fast lists keep the lanes whose interval meets
// the chunk, the parity lists each lane's exact slab range.
template <bool FAST, int CAP>
__device__ __forceinline__ bool lane_has_entry(const WarpSmem<FAST, CAP>& sm, const RenderArgs& a, int e, int k, int K,
                                               int leaf, const RayState& r, int lane) {
    if (FAST) return (sm.lmask[e] >> lane) & 1u;
    const unsigned short rg = sm.lrng[e][lane];
    return k >= (int)(rg & 0xff) && k <= (int)(rg >> 8);
}

// Sample buffers of slab k: sum of density and density-weighted colour of the lane's hits.  The
// backward (GDOT) needs the colour only through g . C, so it accumulates that scalar in gC instead.
template <bool FAST, int CAP, bool GDOT, bool DIAG>
__device__ __forceinline__ int slab_buffers(const WarpSmem<FAST, CAP>& sm, int k, int K, bool has, const RayState& r,
                                            const RenderArgs& a, int rgb_base, const float* roff,
                                            float* sig, float3* C, float* gC, int nw, int lane, WarpStats& ws) {
    int nh = 0;
#pragma unroll 1
    for (int w = 0; w < nw; ++w) {
        unsigned mw = sm.smask[k / WarpSmem<FAST, CAP>::MB][w];
        while (mw) {
            const int e = 32 * w + __ffs(mw) - 1;
            mw &= mw - 1u;
            if (!in_urange(sm.urng[e], k)) continue;
            if (DIAG) ++ws.entry_slabs;
            if (!has) continue;
            const int leaf = sm.ids[e];
            if (!lane_has_entry<FAST, CAP>(sm, a, e, k, K, leaf, r, lane)) continue;
            LeafRec rec = load_rec(a.rec, leaf);
            float4 col4 = __ldg(a.rgb + rgb_base + leaf);
            float3 mu = f3(rec.a.x, rec.a.y, rec.a.z);
            float dn = rec.a.w;
            float3 r0 = f3(rec.r0.x, rec.r0.y, rec.r0.z), r1 = f3(rec.r1.x, rec.r1.y, rec.r1.z),
                   r2 = f3(rec.r2.x, rec.r2.y, rec.r2.z);
            ++nh;
            if (FAST) {
                // log2(dens * w_i) = log2(dens) - q_i log2(e) / 2, q_i quadratic in the sample index
                float3 v0 = (r.o + r.d * r.tb) - mu;
                float3 vb = r.d * kDt;
                float3 m0 = f3(dot3(r0, v0), dot3(r1, v0), dot3(r2, v0));
                float3 mb = f3(dot3(r0, vb), dot3(r1, vb), dot3(r2, vb));
                float A = fmaf(kNegHalfLog2e, dot3(m0, m0), rec.r1.w);   // r1.w = log2(dens)
                float B2 = (2.f * kNegHalfLog2e) * dot3(m0, mb), Cq = kNegHalfLog2e * dot3(mb, mb);
                float3 col = f3(col4.x, col4.y, col4.z);
                const float gcol = GDOT ? dot3(r.g, col) : 0.f;
#pragma unroll
                for (int i = 0; i < kBuf; ++i) {
                    float fi = (float)i;
                    float e = fmaf(fi, fmaf(fi, Cq, B2), A);
                    if (e > kLog2SigThr) {
                        float dw = ex2_approx(e);
                        sig[i] += dw;
                        if (GDOT) gC[i] = fmaf(gcol, dw, gC[i]);
                        else C[i] = C[i] + col * dw;
                    }
                }
            } else if (!GDOT && a.infer) {
                // Inference programs (cuda_test/gaussians_aabb.cu:282-295, :501-515): the samples step
                // through the scaled conic space from the slab start, m_{i+1} = m_i + dt * M d, and
                // weight * density multiplies the colour.  Reference operation order.
                const LeafIS is = load_is(a.is_rec, leaf);
                const float kf = is.u.w;   // sqrt(log(ratio^2)) of the Gaussian
                const float3 U = f3(is.u.x, is.u.y, is.u.z), V = f3(is.v.x, is.v.y, is.v.z),
                             W = f3(is.w.x, is.w.y, is.w.z);
                const float3 xg = f3(__fsub_rn(__fadd_rn(r.o.x, __fmul_rn(r.tb, r.d.x)), mu.x),
                                     __fsub_rn(__fadd_rn(r.o.y, __fmul_rn(r.tb, r.d.y)), mu.y),
                                     __fsub_rn(__fadd_rn(r.o.z, __fmul_rn(r.tb, r.d.z)), mu.z));
                float3 m = f3(__fmul_rn(dot_rn(U, xg), kf), __fmul_rn(dot_rn(V, xg), kf),
                              __fmul_rn(dot_rn(W, xg), kf));
                const float3 mdt = f3(__fmul_rn(__fmul_rn(dot_rn(U, r.d), kf), kDt),
                                      __fmul_rn(__fmul_rn(dot_rn(V, r.d), kf), kDt),
                                      __fmul_rn(__fmul_rn(dot_rn(W, r.d), kf), kDt));
#pragma unroll
                for (int i = 0; i < kBuf; ++i) {
                    const float power = __fmul_rn(-0.5f, dot_rn(m, m));
                    float w = expf(power);
                    float wd = __fmul_rn(w, dn);
                    if (fabsf(wd - kSigThr) < 4e-8f) wd = __fmul_rn((float)exp((double)power), dn);
                    if (wd > kSigThr) {
                        sig[i] = __fadd_rn(sig[i], wd);
                        C[i] = f3(__fadd_rn(C[i].x, __fmul_rn(col4.x, wd)), __fadd_rn(C[i].y, __fmul_rn(col4.y, wd)),
                                  __fadd_rn(C[i].z, __fmul_rn(col4.z, wd)));
                    }
                    m = f3(__fadd_rn(m.x, mdt.x), __fadd_rn(m.y, mdt.y), __fadd_rn(m.z, mdt.z));
                }
            } else {
                float ws[kBuf];
                const unsigned in_mask = parity_weights(r, a.rnd_sample, roff, mu, r0, r1, r2, dn, ws);
#pragma unroll
                for (int i = 0; i < kBuf; ++i) {
                    const float w = ws[i];
                    if ((in_mask >> i) & 1u) {
                        sig[i] = __fadd_rn(sig[i], __fmul_rn(dn, w));
                        if (GDOT) {
                            gC[i] += (r.g.x * col4.x + r.g.y * col4.y + r.g.z * col4.z) * (w * dn);
                        } else {
                            C[i] = f3(__fadd_rn(C[i].x, __fmul_rn(__fmul_rn(col4.x, w), dn)),
                                      __fadd_rn(C[i].y, __fmul_rn(__fmul_rn(col4.y, w), dn)),
                                      __fadd_rn(C[i].z, __fmul_rn(__fmul_rn(col4.z, w), dn)));
                        }
                    }
                }
            }
        }
    }
    return nh;
}

template <bool FAST>
__device__ __forceinline__ float exp_neg(float x) {
    return FAST ? ex2_approx(-x * 1.4426950408889634f) : (float)exp(-(double)x);
}

__device__ __forceinline__ bool any_density(const float* sig) {
    bool any = false;
#pragma unroll
    for (int i = 0; i < kBuf; ++i) any |= sig[i] > 0.f;
    return any;
}

// Alpha compositing of one slab's 8 samples (forward/gaussians_aabb.cu:500-519).  A slab whose
// samples all fell under the threshold composites to exactly nothing (alpha = 1 - exp(0) = 0).
template <bool FAST>
__device__ __forceinline__ void composite(RayState& r, const float* sig, const float3* C) {
    if (!any_density(sig)) return;
    float ex[kBuf];
    if (!FAST) {
        // the eight exponentials are independent of the transmittance chain: evaluate them first
#pragma unroll
        for (int i = 0; i < kBuf; ++i) ex[i] = exp_neg<false>(__fmul_rn(sig[i], kDt));
    }
#pragma unroll
    for (int i = 0; i < kBuf; ++i) {
        if (FAST) {
            // C[i] is zero wherever sig[i] is (both sum the same above-threshold samples)
            float alpha = 1.f - exp_neg<true>(sig[i] * kDt);
            float s = sig[i] > 0.f ? __fdividef(r.T * alpha, sig[i]) : 0.f;
            r.C = r.C + C[i] * s;
            r.T *= 1.f - alpha;
        } else {
            float alpha = __fsub_rn(1.f, ex[i]);
            float3 c = C[i];
            if (sig[i] > 0.f) {
                float inv = __fdiv_rn(1.f, sig[i]);
                c = f3(__fmul_rn(c.x, inv), __fmul_rn(c.y, inv), __fmul_rn(c.z, inv));
            }
            float ta = __fmul_rn(r.T, alpha);
            r.C = f3(__fadd_rn(r.C.x, __fmul_rn(c.x, ta)), __fadd_rn(r.C.y, __fmul_rn(c.y, ta)),
                     __fadd_rn(r.C.z, __fmul_rn(c.z, ta)));
            r.T = __fmul_rn(r.T, __fsub_rn(1.f, alpha));
        }
    }
}

__device__ __forceinline__ float4 quat_grad(float4 q, float3 d1, float3 d2, float3 d3) {
    // derivative of the (not normalised) polynomial rotation columns w.r.t. (r, i, j, k)
    float r = q.x, i = q.y, j = q.z, k = q.w;
    float4 o;
    o.x = 2.f * (k * d1.y - j * d1.z - k * d2.x + i * d2.z + j * d3.x - i * d3.y);
    o.y = 2.f * (j * d1.y + k * d1.z + j * d2.x - 2.f * i * d2.y + r * d2.z + k * d3.x - r * d3.y - 2.f * i * d3.z);
    o.z = 2.f * (-2.f * j * d1.x + i * d1.y - r * d1.z + i * d2.x + k * d2.z + r * d3.x + k * d3.y - 2.f * j * d3.z);
    o.w = 2.f * (-2.f * k * d1.x + r * d1.y + i * d1.z - r * d2.x - 2.f * k * d2.y + j * d2.z + i * d3.x + j * d3.y);
    return o;
}

// Transposed warp reduction of 16 values: afterwards lane l holds the warp sum of value
// 8*b4 + 4*b3 + 2*b2 + b1 (b_i = bit i of l); lanes l and l^1 hold the same value.
__device__ __forceinline__ float transpose_reduce16(float* v, int lane) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        bool up = lane & 16;
        float send = up ? v[i] : v[i + 8];
        float keep = up ? v[i + 8] : v[i];
        v[i] = keep + __shfl_xor_sync(kFull, send, 16);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        bool up = lane & 8;
        float send = up ? v[i] : v[i + 4];
        float keep = up ? v[i + 4] : v[i];
        v[i] = keep + __shfl_xor_sync(kFull, send, 8);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        bool up = lane & 4;
        float send = up ? v[i] : v[i + 2];
        float keep = up ? v[i + 2] : v[i];
        v[i] = keep + __shfl_xor_sync(kFull, send, 4);
    }
    {
        bool up = lane & 2;
        float send = up ? v[0] : v[1];
        float keep = up ? v[1] : v[0];
        v[0] = keep + __shfl_xor_sync(kFull, send, 2);
    }
    v[0] += __shfl_xor_sync(kFull, v[0], 1);
    return v[0];
}

// Adjoint of slab k for all list entries: per-lane gradient of each hit Gaussian, warp reduction,
// one atomic per value.  Value order: ddens, S1.xyz, M2 (xx yy zz xy xz yz), 0, drgb.xyz.
template <bool FAST, int CAP, bool DIAG>
__device__ __forceinline__ void slab_adjoint(const WarpSmem<FAST, CAP>& sm, int k, int K, bool has, const RayState& r,
                                             const RenderArgs& a, int rgb_base, const float* roff,
                                             const float* H, const float* F, int nw, int lane,
                                             WarpStats& ws, int view) {
    const int vid = ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
#pragma unroll 1
    for (int w = 0; w < nw; ++w) {
      unsigned mw = sm.smask[k / WarpSmem<FAST, CAP>::MB][w];
      while (mw) {
        const int e = 32 * w + __ffs(mw) - 1;
        mw &= mw - 1u;
        if (!in_urange(sm.urng[e], k)) continue;
        const int leaf = sm.ids[e];
        if (DIAG) ++ws.entry_slabs;
        bool act = has && lane_has_entry<FAST, CAP>(sm, a, e, k, K, leaf, r, lane);
        unsigned am = __ballot_sync(kFull, act);
        if (am == 0u) continue;
        float v[16];
#pragma unroll
        for (int z = 0; z < 16; ++z) v[z] = 0.f;
        if (act) {
            LeafRec rec = load_rec(a.rec, leaf);
            float4 col4 = __ldg(a.rgb + rgb_base + leaf);
            float3 mu = f3(rec.a.x, rec.a.y, rec.a.z);
            float dn = rec.a.w;
            float3 r0 = f3(rec.r0.x, rec.r0.y, rec.r0.z), r1 = f3(rec.r1.x, rec.r1.y, rec.r1.z),
                   r2 = f3(rec.r2.x, rec.r2.y, rec.r2.z);
            float gcol = r.g.x * col4.x + r.g.y * col4.y + r.g.z * col4.z;
            float gc = 0.f, dd = 0.f;
            // Moment form.  With the sample offsets from the Gaussian v_i = v0 + x_i vb, every
            // geometric gradient of this (ray, Gaussian, slab) is linear in the ray-independent
            // moments S1 = sum_i u_i v_i and M2 = sum_i u_i v_i v_i^T (u_i = dens * h_i * w_i), which
            // follow from U_k = sum_i u_i x_i^k (k = 0, 1, 2).  The moments of all rays and slabs are
            // summed per Gaussian and turned into position/scale/rotation gradients once per
            // Gaussian afterwards (k_moment_grads).  Fast arithmetic: x_i = i, vb = dt * dir.  Parity:
            // x_i = t_i - tb, vb = dir (random sample offsets included), the reference's weights and
            // threshold decisions.
            const float3 v0 = (r.o + r.d * r.tb) - mu;
            const float3 vb = FAST ? r.d * kDt : r.d;
            float U0 = 0.f, U1 = 0.f, U2 = 0.f;
            if (FAST) {
                // dw_i = dens * w_i in the exponent domain (as in the forward); accumulates
                // sum dw F, sum dw h and the moments of u = dw h, then divides by dens once
                const float3 m0 = f3(dot3(r0, v0), dot3(r1, v0), dot3(r2, v0));
                const float3 mb = f3(dot3(r0, vb), dot3(r1, vb), dot3(r2, vb));
                float A = fmaf(kNegHalfLog2e, dot3(m0, m0), rec.r1.w);   // r1.w = log2(dens)
                float B2 = (2.f * kNegHalfLog2e) * dot3(m0, mb), Cq = kNegHalfLog2e * dot3(mb, mb);
#pragma unroll
                for (int i = 0; i < kBuf; ++i) {
                    float fi = (float)i;
                    float e = fmaf(fi, fmaf(fi, Cq, B2), A);
                    if (e > kLog2SigThr) {
                        float dw = ex2_approx(e);
                        float u = fmaf(F[i], gcol, H[i]) * dw;
                        gc = fmaf(dw, F[i], gc);
                        U0 += u;
                        U1 = fmaf(fi, u, U1);
                        U2 = fmaf(fi * fi, u, U2);
                    }
                }
                dd = (U0 != 0.f) ? U0 * rec.r2.w : 0.f;                   // r2.w = 1 / dens
            } else {
                float ws[kBuf];
                const unsigned in_mask = parity_weights(r, a.rnd_sample, roff, mu, r0, r1, r2, dn, ws);
#pragma unroll
                for (int i = 0; i < kBuf; ++i) {
                    if ((in_mask >> i) & 1u) {
                        const float wt = ws[i];
                        const float t = parity_time(r.tb, i, a.rnd_sample, roff);
                        float h = fmaf(F[i], gcol, H[i]);
                        gc += wt * F[i];
                        dd += wt * h;
                        float u = h * wt;
                        float x = t - r.tb;
                        U0 += u;
                        U1 += x * u;
                        U2 += x * x * u;
                    }
                }
                gc *= dn;
                U0 *= dn; U1 *= dn; U2 *= dn;
            }
            // S1 = v0 U0 + vb U1; M2 = v0 v0^T U0 + (v0 vb^T + vb v0^T) U1 + vb vb^T U2
            const float3 p = v0 * U0 + vb * U1;     // sum u v
            const float3 q = v0 * U1 + vb * U2;     // sum u x v
            v[0] = dd;
            v[1] = p.x; v[2] = p.y; v[3] = p.z;
            v[4] = v0.x * p.x + vb.x * q.x;         // xx
            v[5] = v0.y * p.y + vb.y * q.y;         // yy
            v[6] = v0.z * p.z + vb.z * q.z;         // zz
            v[7] = v0.x * p.y + vb.x * q.y;         // xy
            v[8] = v0.x * p.z + vb.x * q.z;         // xz
            v[9] = v0.y * p.z + vb.y * q.z;         // yz
            v[11] = r.g.x * gc; v[12] = r.g.y * gc; v[13] = r.g.z * gc;
        }
        float* gg = reinterpret_cast<float*>(a.gacc_geo + 3 * (long long)leaf);
        float* gr = reinterpret_cast<float*>(a.gacc_rgb + (long long)leaf * a.n_views + view);
        // lanes whose samples all fell under the threshold contribute nothing
        const bool nz = act && (v[0] != 0.f || v[1] != 0.f || v[2] != 0.f || v[3] != 0.f || v[11] != 0.f ||
                                v[12] != 0.f || v[13] != 0.f);
        const unsigned zm = __ballot_sync(kFull, nz);
        if (zm == 0u) continue;
        if (__popc(zm) <= RG_DIRECT_ATOMIC_LANES) {
            if (nz) {
                float4* g4 = reinterpret_cast<float4*>(gg);
                atomicAdd(g4, make_float4(v[0], v[1], v[2], v[3]));
                atomicAdd(g4 + 1, make_float4(v[4], v[5], v[6], v[7]));
                atomicAdd(g4 + 2, make_float4(v[8], v[9], v[10], 0.f));
                atomicAdd(reinterpret_cast<float4*>(gr), make_float4(v[11], v[12], v[13], 0.f));
            }
        } else {
            float s = transpose_reduce16(v, lane);
            if (!(lane & 1) && vid < 14) {
                if (vid < 11) atomicAdd(gg + vid, s);
                else atomicAdd(gr + (vid - 11), s);
            }
        }
      }
    }
}

// Per-sample compositing adjoint scalars of one slab (reference backward :675-730): with
// E = g.((T c - R) dt), F = T alpha / sigma and G = g.c, a Gaussian of colour col and weight w
// at the sample has dL/d(sigma-share) h = E + F (g.col - G) = F g.col + H, H = E - F G.  Only
// g.C (gC, C the colour sum of the sample) and g.R (r.gR) enter: with gc = g.C / sigma,
// E = dt (T gc - g.R), H = E - F gc, and g.R drops by gc T alpha per sample.
// Returns H and F; advances T and g.R over the slab.
template <bool FAST>
__device__ __forceinline__ void slab_adjoint_scalars(const RayState& r, const float* sig, const float* gC, float* H,
                                                     float* F, float& Ta, float& gRa) {
    Ta = r.T;
    gRa = r.gR;
    float ex[kBuf];
    if (!FAST) {
#pragma unroll
        for (int i = 0; i < kBuf; ++i) ex[i] = exp_neg<false>(__fmul_rn(sig[i], kDt));
    }
#pragma unroll
    for (int i = 0; i < kBuf; ++i) {
        const float cd = sig[i];
        float inv = 0.f;
        if (cd > 0.f) inv = FAST ? __fdividef(1.f, cd) : 1.f / cd;
        const float gc = gC[i] * inv;
        const float alpha = FAST ? 1.f - exp_neg<true>(cd * kDt) : __fsub_rn(1.f, ex[i]);
        const float ta = Ta * alpha;
        F[i] = ta * inv;
        H[i] = kDt * (Ta * gc - gRa) - F[i] * gc;
        gRa -= gc * ta;
        Ta = FAST ? Ta * (1.f - alpha) : __fmul_rn(Ta, __fsub_rn(1.f, alpha));
    }
}

// Resident blocks per SM each kernel is compiled for (0: the compiler's choice).  The defaults
// fit the shared memory of the 64-entry tuning (256-entry fast lists) and were measured best on
// 1M Gaussians x 16 views.
#ifndef RG_FAST_FWD_MIN_BLOCKS
#define RG_FAST_FWD_MIN_BLOCKS 7
#endif
#ifndef RG_FAST_BWD_MIN_BLOCKS
#define RG_FAST_BWD_MIN_BLOCKS 7
#endif
#ifndef RG_PAR_FWD_MIN_BLOCKS
#define RG_PAR_FWD_MIN_BLOCKS 4
#endif
#ifndef RG_PAR_BWD_MIN_BLOCKS
#define RG_PAR_BWD_MIN_BLOCKS 4
#endif
template <bool BWD, bool FAST>
constexpr int min_blocks() {
    return FAST ? (BWD ? RG_FAST_BWD_MIN_BLOCKS : RG_FAST_FWD_MIN_BLOCKS)
                : (BWD ? RG_PAR_BWD_MIN_BLOCKS : RG_PAR_FWD_MIN_BLOCKS);
}

// DIAG: also count node visits, leaf tests, list entries, slab steps and entry-slabs (rg_status);
// without it those counters compile away and the kernel holds fewer live registers.
template <bool BWD, bool FAST, int CAP, bool DIAG>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, min_blocks<BWD, FAST>()) k_render(RenderArgs a) {
    __shared__ WarpSmem<FAST, CAP> smem[kWarpsPerBlock];
    const int lane = threadIdx.x & 31;
    WarpSmem<FAST, CAP>& sm = smem[threadIdx.x >> 5];
    const ViewTable* vt = a.views;
    const float bg = a.white_bg ? 1.f : 0.f;
    if (lane == 0) {
#pragma unroll
        for (int c = 0; c < kCounters; ++c) sm.cnt[c] = 0ull;
    }
    const int kmax =
        min((a.rnd_sample == 1) ? min(a.chunk_slabs, kExactChunk) : a.chunk_slabs, WarpSmem<FAST, CAP>::KM);

    while (true) {
        int tile = 0;
        if (lane == 0) tile = atomicAdd(a.work_counter, 1);
        tile = __shfl_sync(kFull, tile, 0);
        if (tile >= vt->total_tiles) break;
        // view of this tile (binary search over the tile prefix)
        int lo = 0, hi = vt->n_views - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (vt->tile_prefix[mid] <= tile) lo = mid; else hi = mid - 1;
        }
        const int view = lo;
        const rg_camera cam = a.cams[view];
        const int W = cam.width, H = cam.height;
        const int tiles_x = (W + kTileW - 1) / kTileW;
        const int local = tile - vt->tile_prefix[view];
        const int px = (local % tiles_x) * kTileW + (lane & (kTileW - 1));
        const int py = (local / tiles_x) * kTileH + (lane / kTileW);
        const bool valid = px < W && py < H;
        const unsigned ray_l = (unsigned)(py * W + px);
        const int rgb_base = view * a.n_leaves;   // views x leaves < 2^31 (checked by the host)

        RayState r;
        WarpStats ws;
        unsigned hits_acc = 0, slabs_acc = 0;   // this lane's (slab, Gaussian) pairs and slabs
        r.seed = tea4(a.iteration, ray_l);
        {
            // computeRay (forward/gaussians_aabb.cu:405-434) in IEEE operation order
            float ix, iy;
            if (a.jitter == 1) {
                float jx = lcg_rnd(r.seed) * 0.333333f;
                float jy = lcg_rnd(r.seed) * 0.333333f;
                ix = __fdiv_rn(__fadd_rn(__fadd_rn((float)(ray_l % (unsigned)W), 0.333333f), jx), (float)W);
                iy = __fdiv_rn(__fadd_rn(__fadd_rn((float)(ray_l / (unsigned)W), 0.333333f), jy), (float)H);
            } else {
                ix = __fdiv_rn(__fadd_rn((float)(ray_l % (unsigned)W), 0.5f), (float)W);
                iy = __fdiv_rn(__fadd_rn((float)(ray_l / (unsigned)W), 0.5f), (float)H);
            }
            float dx = __fmul_rn(__fsub_rn(__fmul_rn(2.f, ix), 1.f), cam.tan_half_fovx);
            float dy = __fmul_rn(__fsub_rn(__fmul_rn(2.f, iy), 1.f), cam.tan_half_fovy);
            float3 dir = f3(__fadd_rn(__fadd_rn(__fmul_rn(cam.u[0], dx), __fmul_rn(cam.v[0], dy)), cam.w[0]),
                            __fadd_rn(__fadd_rn(__fmul_rn(cam.u[1], dx), __fmul_rn(cam.v[1], dy)), cam.w[1]),
                            __fadd_rn(__fadd_rn(__fmul_rn(cam.u[2], dx), __fmul_rn(cam.v[2], dy)), cam.w[2]));
            float inv = __fdiv_rn(1.f, __fsqrt_rn(dot_rn(dir, dir)));
            r.d = f3(__fmul_rn(dir.x, inv), __fmul_rn(dir.y, inv), __fmul_rn(dir.z, inv));
            r.o = f3(cam.eye[0], cam.eye[1], cam.eye[2]);
        }
        {
            float scene[6];   // scene box, read per tile (not kept live through the tile's loops)
#pragma unroll
            for (int z = 0; z < 6; ++z) scene[z] = ord2f(__ldg(a.scene_ord + z));
            float t0x = __fdiv_rn(scene[0] - r.o.x, r.d.x), t1x = __fdiv_rn(scene[3] - r.o.x, r.d.x);
            float t0y = __fdiv_rn(scene[1] - r.o.y, r.d.y), t1y = __fdiv_rn(scene[4] - r.o.y, r.d.y);
            float t0z = __fdiv_rn(scene[2] - r.o.z, r.d.z), t1z = __fdiv_rn(scene[5] - r.o.z, r.d.z);
            r.tenter = fmaxf(0.f, fmaxf(fminf(t0x, t1x), fmaxf(fminf(t0y, t1y), fminf(t0z, t1z))));
            r.texit = fminf(fmaxf(t0x, t1x), fminf(fmaxf(t0y, t1y), fmaxf(t0z, t1z)));
        }
        r.alive = valid && (r.tenter < r.texit);
        r.tb = r.tenter;
        r.T = 1.f;
        r.C = f3(0.f, 0.f, 0.f);
        r.g = f3(0.f, 0.f, 0.f);
        r.gR = 0.f;
        if (BWD && valid) {
            const long long ray_g = vt->ray_prefix[view] + (long long)ray_l;
            r.g = f3(a.dL[3 * ray_g], a.dL[3 * ray_g + 1], a.dL[3 * ray_g + 2]);
            r.gR = r.g.x * a.ray_colors_in[3 * ray_g] + r.g.y * a.ray_colors_in[3 * ray_g + 1] +
                   r.g.z * a.ray_colors_in[3 * ray_g + 2];
        }

        int K = min(kExactChunk, kmax);
        int rounds = 0;
        // end of the searched range: an inference launch queries the last slab in full
        const bool infer = !BWD && a.infer;
        const float t_end = infer ? r.texit + kSlab : r.texit;
        // hit-list record of this tile: the forward appends chunk records, the backward replays them
        const bool rec_here = a.rec_arena != nullptr && tile < a.rec_tiles;
        if (lane == 0) {
            sm.rec_first = kNoRecord;
            sm.rec_prev = kNoRecord;
            sm.rec_cur = (BWD && rec_here && a.replay) ? a.rec_tile[tile] : kNoRecord;
        }
        __syncwarp();
        while (true) {
            bool on = r.alive;
            if (!__any_sync(kFull, on)) break;
            if (++rounds > kMaxRounds) {
                if (lane == 0) atomicAdd(&a.st->watchdog_trips, 1ull);
                break;
            }
            unsigned rec_hdr = 0u;
            unsigned rec_cur = BWD ? sm.rec_cur : kNoRecord;
            if (BWD && rec_cur != kNoRecord) {
                if (rec_cur + 2u > a.rec_cap) {
                    rec_cur = kNoRecord;   // malformed link: traverse from here on
                } else {
                    rec_hdr = a.rec_arena[rec_cur];
                    K = max(1, min(kmax, (int)((rec_hdr >> 16) & 0xffu)));
                }
            }
            // slabs of this chunk: slab k is marched iff tb_k < texit (tb_k by repeated addition)
            int nv = 0;
            float seg_hi = r.tb;
            if (on) {
                if (K <= kExactChunk) {
                    float t = r.tb;
                    for (int kk = 0; kk < K; ++kk) {
                        if (t < r.texit) { nv = kk + 1; t = t + kSlab; } else break;
                    }
                    seg_hi = fminf(t_end, t);
                } else {
                    nv = K;
                    seg_hi = fminf(t_end, r.tb + (float)(K + 1) * kSlab);
                }
                // a slab step that no longer changes tb (|t| beyond ~2^19) would march forever
                if (!(r.tb < r.texit) || r.tb + kSlab == r.tb) { r.alive = false; on = false; nv = 0; }
            }
            bool ovf = false;
            int count;
            const bool replayed = BWD && rec_cur != kNoRecord && !(rec_hdr & kRecordMulti);
            if (!replayed) set_packet<FAST, CAP>(sm, r, on, seg_hi, lane);
            if (replayed) {
                const unsigned n_ids = min(rec_hdr & 0xffffu, a.rec_cap - rec_cur - 2u);
                count = replay_list<FAST, CAP, DIAG>(sm, a, r, on, seg_hi, K, nv, a.rec_arena + rec_cur + 2, (int)n_ids,
                                               lane, ws);
                ++ws.replays;
            } else {
                count = traverse<FAST, CAP, DIAG>(sm, a, r, on, seg_hi, K, nv, -1, ovf, lane, ws, infer);
            }
            const unsigned long long* occ = sm.occ;
            if (ovf && K > 1) {
                K = max(1, K >> 1);
                if (lane == 0) atomicAdd(&a.st->chunk_splits, 1ull);
                continue;
            }
            if (!BWD && rec_here && sm.rec_first != kRecordFailed) {
                // chunk record: header (multi-pass flag | K << 16 | id count), next record, ids
                const unsigned n_ids = ovf ? 0u : (unsigned)count;
                const unsigned words = 2u + n_ids;
                unsigned off = kNoRecord;
                if (lane == 0) {
                    unsigned long long o = atomicAdd(a.rec_top, (unsigned long long)words);
                    if (o + words <= (unsigned long long)a.rec_cap) {
                        off = (unsigned)o;
                        a.rec_arena[off] = (ovf ? kRecordMulti : 0u) | ((unsigned)K << 16) | n_ids;
                        a.rec_arena[off + 1] = kNoRecord;
                        if (sm.rec_prev != kNoRecord) a.rec_arena[sm.rec_prev + 1] = off;
                        if (sm.rec_first == kNoRecord) sm.rec_first = off;
                        sm.rec_prev = off;
                    } else {
                        sm.rec_first = kRecordFailed;
                        atomicAdd(&a.st->record_overflows, 1ull);
                    }
                }
                off = __shfl_sync(kFull, off, 0);
                if (off != kNoRecord)
                    for (unsigned e = lane; e < n_ids; e += 32) a.rec_arena[off + 2 + e] = (unsigned)sm.ids[e];
                __syncwarp();
            }
            if (!ovf) {
                for (int k = 0; k < K; ++k) {
                    bool has = on && r.tb < r.texit && r.T > kTeps;
                    if (!__any_sync(kFull, has)) break;
                    if (!occ_test(occ, k)) {
                        // no lane has a hit in slabs [k, k2): march them (tb only; T is unchanged)
                        int k2 = occ_next(occ, k, K);
                        if (has) {
                            for (int j = k; j < k2 && r.tb < r.texit; ++j) {
                                r.tb = r.tb + kSlab;
                                ++slabs_acc;
                            }
                        }
                        k = k2 - 1;
                        continue;
                    }
                    if (DIAG) ++ws.slab_steps;
                    float roff[kBuf];
                    unsigned seed_next = slab_offsets(a.rnd_sample, r.seed, roff);
                    float sig[kBuf];
                    float3 Cb[BWD ? 1 : kBuf];
                    float gC[BWD ? kBuf : 1];
#pragma unroll
                    for (int i = 0; i < kBuf; ++i) {
                        sig[i] = 0.f;
                        if (BWD) gC[i] = 0.f;
                        else Cb[i] = f3(0.f, 0.f, 0.f);
                    }
                    int nh = slab_buffers<FAST, CAP, BWD, DIAG>(sm, k, K, has, r, a, rgb_base, roff, sig, Cb, gC,
                                                          nwords(count), lane, ws);
                    if (has) {
                        ++slabs_acc;
                        hits_acc += (!BWD && a.counts) ? min(nh, a.max_prim_slice) : nh;
                        if (nh > a.max_prim_slice) atomicAdd(&a.st->slab_cap_exceeded, 1ull);
                    }
                    if (!BWD) {
                        if (has && nh > 0) {
                            composite<FAST>(r, sig, Cb);
                            r.seed = seed_next;
                        }
                    } else {
                        float H[kBuf], F[kBuf], Ta, gRa;
                        slab_adjoint_scalars<FAST>(r, sig, gC, H, F, Ta, gRa);
                        bool act = has && nh > 0 && any_density(sig);
                        slab_adjoint<FAST, CAP, DIAG>(sm, k, K, act, r, a, rgb_base, roff, H, F, nwords(count), lane, ws,
                                                      view);
                        if (has && nh > 0) {
                            r.T = Ta;
                            r.gR = gRa;
                            r.seed = seed_next;
                        }
                    }
                    if (has) r.tb = r.tb + kSlab;
                }
                // next chunk length: aim at half a list, grow at most 2x per chunk
                {
                    int target = count > 0 ? (K * (CAP / 2)) / count : kmax;
                    K = max(1, min(kmax, min(2 * K, target)));
                }
            } else {
                // K == 1 and more hits than the list holds: consume the slab in several passes
                bool has = on && nv > 0 && r.T > kTeps;
                float roff[kBuf];
                unsigned seed_next = slab_offsets(a.rnd_sample, r.seed, roff);
                float sig[kBuf];
                float3 Cb[BWD ? 1 : kBuf];
                float gC[BWD ? kBuf : 1];
#pragma unroll
                for (int i = 0; i < kBuf; ++i) {
                    sig[i] = 0.f;
                    if (BWD) gC[i] = 0.f;
                    else Cb[i] = f3(0.f, 0.f, 0.f);
                }
                int nh = slab_buffers<FAST, CAP, BWD, DIAG>(sm, 0, 1, has, r, a, rgb_base, roff, sig, Cb, gC, nwords(count),
                                                      lane, ws);
                bool more = ovf;
                while (more) {
                    int cursor = sm.ids[count - 1];
                    __syncwarp();
                    if (lane == 0) atomicAdd(&a.st->list_passes, 1ull);
                    count = traverse<FAST, CAP, DIAG>(sm, a, r, on, seg_hi, 1, nv, cursor, more, lane, ws, infer);
                    nh += slab_buffers<FAST, CAP, BWD, DIAG>(sm, 0, 1, has, r, a, rgb_base, roff, sig, Cb, gC,
                                                       nwords(count), lane, ws);
                }
                if (has) {
                    ++slabs_acc;
                    hits_acc += (!BWD && a.counts) ? min(nh, a.max_prim_slice) : nh;
                    if (nh > a.max_prim_slice) atomicAdd(&a.st->slab_cap_exceeded, 1ull);
                }
                if (!BWD) {
                    if (has && nh > 0) {
                        composite<FAST>(r, sig, Cb);
                        r.seed = seed_next;
                    }
                } else {
                    float H[kBuf], F[kBuf], Ta, gRa;
                    slab_adjoint_scalars<FAST>(r, sig, gC, H, F, Ta, gRa);
                    bool act = has && nh > 0 && any_density(sig);
                    int cursor = -1;
                    bool more2 = true;
                    while (more2) {
                        count = traverse<FAST, CAP, DIAG>(sm, a, r, on, seg_hi, 1, nv, cursor, more2, lane, ws, infer);
                        slab_adjoint<FAST, CAP, DIAG>(sm, 0, 1, act, r, a, rgb_base, roff, H, F, nwords(count), lane, ws,
                                                      view);
                        if (more2) cursor = sm.ids[count - 1];
                        __syncwarp();
                    }
                    if (has && nh > 0) {
                        r.T = Ta;
                        r.gR = gRa;
                        r.seed = seed_next;
                    }
                }
                if (has) r.tb = r.tb + kSlab;
            }
            if (on) r.alive = r.alive && (r.T > kTeps) && (r.tb < r.texit);
            if (BWD && lane == 0) sm.rec_cur = (rec_cur != kNoRecord) ? a.rec_arena[rec_cur + 1] : kNoRecord;
            __syncwarp();
        }
        if (!BWD && rec_here && lane == 0)
            a.rec_tile[tile] = (sm.rec_first == kRecordFailed) ? kNoRecord : sm.rec_first;
        flush_stats<FAST, CAP, DIAG>(sm, ws, hits_acc, slabs_acc, lane);
        if (!BWD && valid) {
            const long long ray_g = vt->ray_prefix[view] + (long long)ray_l;
            a.ray_colors[3 * ray_g] = __fadd_rn(r.C.x, __fmul_rn(r.T, bg));
            a.ray_colors[3 * ray_g + 1] = __fadd_rn(r.C.y, __fmul_rn(r.T, bg));
            a.ray_colors[3 * ray_g + 2] = __fadd_rn(r.C.z, __fmul_rn(r.T, bg));
            if (a.final_T) a.final_T[ray_g] = r.T;
            // Gaussians per ray (inference launches): the per-slab hit counts, each capped at
            // max_prim_slice like the reference any-hit program (cuda_test/gaussians_aabb.cu:438)
            if (a.counts) a.counts[ray_g] = (int)hits_acc;
        }
    }
    // counters: one atomic per warp and counter
    __syncwarp();
    if (lane == 0) {
        atomicAdd(&a.st->traversals, sm.cnt[0]);
        atomicAdd(&a.st->node_visits, sm.cnt[1]);
        atomicAdd(&a.st->leaf_tests, sm.cnt[2]);
        atomicAdd(&a.st->list_entries, sm.cnt[3]);
        atomicAdd(&a.st->slab_steps, sm.cnt[4]);
        atomicAdd(&a.st->entry_slabs, sm.cnt[5]);
        if (BWD) atomicAdd(&a.st->replayed_chunks, sm.cnt[6]);
        atomicAdd(&a.st->hit_pairs, sm.cnt[7]);
        atomicAdd(&a.st->slabs, sm.cnt[8]);
    }
}

// Per-leaf conversion of the summed adjoint moments into gradients (one thread per leaf):
//   in  [dens grad, S1.xyz, M2 xx yy zz xy xz yz, 0, 0]
//   out [dens grad, dpos.xyz, dscale.xyz, dquat.xyzw, 0]
// with m = M v (rows of M = R^T / s): dpos = M^T M S1, dscale_j = r_j^T M2 r_j / s_j and, for the
// rotation, P_j = M2 r_j enters the quaternion derivative as -P_j / s_j.
__global__ void k_moment_grads(int n, const LeafRec* __restrict__ rec, const float4* __restrict__ ext,
                               float4* __restrict__ acc) {
    int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n) return;
    const float4 a0 = acc[3 * (long long)l], a1 = acc[3 * (long long)l + 1], a2 = acc[3 * (long long)l + 2];
    const LeafRec rr = rec[l];
    const float4 s4 = ext[2 * (long long)l], q4 = ext[2 * (long long)l + 1];
    const float3 r0 = f3(rr.r0.x, rr.r0.y, rr.r0.z), r1 = f3(rr.r1.x, rr.r1.y, rr.r1.z),
                 r2 = f3(rr.r2.x, rr.r2.y, rr.r2.z);
    const float3 S1 = f3(a0.y, a0.z, a0.w);
    const float xx = a1.x, yy = a1.y, zz = a1.z, xy = a1.w, xz = a2.x, yz = a2.y;
    auto m2 = [&](float3 w) {
        return f3(xx * w.x + xy * w.y + xz * w.z, xy * w.x + yy * w.y + yz * w.z, xz * w.x + yz * w.y + zz * w.z);
    };
    const float3 Sm = f3(dot3(r0, S1), dot3(r1, S1), dot3(r2, S1));
    const float3 dp = r0 * Sm.x + r1 * Sm.y + r2 * Sm.z;
    const float3 P0 = m2(r0), P1 = m2(r1), P2 = m2(r2);
    const float3 is = f3(1.f / s4.x, 1.f / s4.y, 1.f / s4.z);
    const float3 dsc = f3(dot3(r0, P0) * is.x, dot3(r1, P1) * is.y, dot3(r2, P2) * is.z);
    const float4 dq = quat_grad(q4, P0 * (-is.x), P1 * (-is.y), P2 * (-is.z));
    acc[3 * (long long)l] = make_float4(a0.x, dp.x, dp.y, dp.z);
    acc[3 * (long long)l + 1] = make_float4(dsc.x, dsc.y, dsc.z, dq.x);
    acc[3 * (long long)l + 2] = make_float4(dq.y, dq.z, dq.w, 0.f);
}

cudaError_t launch_moment_grads(int n, const LeafRec* rec, const float4* ext, float4* acc, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_moment_grads<<<(n + 255) / 256, 256, 0, s>>>(n, rec, ext, acc);
    return cudaGetLastError();
}

// List capacity per arithmetic: 4x the tuning value (64 or 128) for the fast lists; 128 for the
// parity lists at either value (their per-lane slab ranges make an entry 64 B; shorter lists turn
// dense slabs into multi-pass traversals, which the backward cannot replay).
static_assert(sizeof(WarpSmem<false, 128>) * kWarpsPerBlock <= 48 * 1024, "static shared memory limit");
// the packet is read as float4: 16-byte aligned in every warp's slice of the block's array
using ParitySmem = WarpSmem<false, 128>;
using FastSmem256 = WarpSmem<true, 256>;
using FastSmem512 = WarpSmem<true, 512>;
static_assert(offsetof(ParitySmem, packet) % 16 == 0 && sizeof(ParitySmem) % 16 == 0, "packet alignment");
static_assert(offsetof(FastSmem256, packet) % 16 == 0 && sizeof(FastSmem256) % 16 == 0, "packet alignment");
static_assert(offsetof(FastSmem512, packet) % 16 == 0 && sizeof(FastSmem512) % 16 == 0, "packet alignment");
static_assert(sizeof(WarpSmem<true, 512>) * kWarpsPerBlock <= 48 * 1024, "static shared memory limit");

template <bool BWD, bool FAST>
static cudaError_t launch_cap(int cap, int grid, const RenderArgs& a, cudaStream_t s) {
    const int threads = kWarpsPerBlock * 32;
    if constexpr (FAST) {
        if (cap <= 64) {
            if (a.diag) k_render<BWD, FAST, 256, true><<<grid, threads, 0, s>>>(a);
            else k_render<BWD, FAST, 256, false><<<grid, threads, 0, s>>>(a);
        } else {
            if (a.diag) k_render<BWD, FAST, 512, true><<<grid, threads, 0, s>>>(a);
            else k_render<BWD, FAST, 512, false><<<grid, threads, 0, s>>>(a);
        }
    } else {
        if (a.diag) k_render<BWD, FAST, 128, true><<<grid, threads, 0, s>>>(a);
        else k_render<BWD, FAST, 128, false><<<grid, threads, 0, s>>>(a);
    }
    return cudaGetLastError();
}

template <bool BWD, bool FAST>
static int occ_cap(int cap) {
    int nb = 0;
    const int threads = kWarpsPerBlock * 32;
    if constexpr (FAST) {
        if (cap <= 64) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_render<BWD, FAST, 256, false>, threads, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_render<BWD, FAST, 512, false>, threads, 0);
    } else {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_render<BWD, FAST, 128, false>, threads, 0);
    }
    return nb;
}

int render_occupancy(bool backward, int mode, int cap) {
    bool fast = mode == RG_MODE_FAST;
    if (backward) return fast ? occ_cap<true, true>(cap) : occ_cap<true, false>(cap);
    return fast ? occ_cap<false, true>(cap) : occ_cap<false, false>(cap);
}

cudaError_t launch_render(bool backward, int mode, int cap, int grid, const RenderArgs& a, cudaStream_t s) {
    bool fast = (mode == RG_MODE_FAST) && a.rnd_sample == 0;
    if (backward) return fast ? launch_cap<true, true>(cap, grid, a, s) : launch_cap<true, false>(cap, grid, a, s);
    return fast ? launch_cap<false, true>(cap, grid, a, s) : launch_cap<false, false>(cap, grid, a, s);
}

}  // namespace rg
