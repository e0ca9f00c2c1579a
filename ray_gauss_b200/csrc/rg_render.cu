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
// counter).  Each lane marches its own ray; the warp advances in chunks of up to 8 slabs per
// lane.  For a chunk the warp traverses the LBVH once for the union of its lanes' segments with a
// warp-uniform stack, runs the exact ellipsoid test per lane at the leaves and appends every leaf
// that any lane hits to a shared hit list together with one 32-bit lane mask per slab.  The list
// is then consumed slab by slab: every lane evaluates only the entries whose mask bit it owns,
// reading the leaf record with a warp-uniform (broadcast) load.  A full list halves the chunk;
// a full list for a single slab is consumed in several passes (a leaf-index cursor skips the
// leaves already taken; DFS order visits leaves in increasing index), so no hit is ever dropped.
// The adjoint recomputes each slab's sample buffers, folds the per-sample compositing adjoint
// into three scalars per sample, evaluates each Gaussian's gradient per lane, reduces it across
// the warp with shuffles and issues vector atomics (float4) into leaf-ordered accumulators.
#include "rg_common.cuh"
#include "rg_kernels.h"

namespace rg {

constexpr int kWarpsPerBlock = 4;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxRounds = 1 << 20;        // chunk rounds per tile before the watchdog trips
constexpr float kNegHalfLog2e = -0.72134752044448170f;

template <int CAP>
struct WarpSmem {
    int ids[CAP];
    unsigned mask[kMaxChunk][CAP];
    int stack[kStack];
};

struct RayState {
    float3 o, d, invd;
    float tenter, texit;
    float tb;
    float T;
    float3 C;     // forward: accumulated colour; backward: remaining colour R
    float3 g;     // backward: dL/dcolour of the ray
    unsigned seed;
    bool alive;
};

__device__ __forceinline__ bool box_hit(const float* bx, const RayState& r, float lo, float hi) {
    float tx0 = (bx[0] - r.o.x) * r.invd.x, tx1 = (bx[3] - r.o.x) * r.invd.x;
    float ty0 = (bx[1] - r.o.y) * r.invd.y, ty1 = (bx[4] - r.o.y) * r.invd.y;
    float tz0 = (bx[2] - r.o.z) * r.invd.z, tz1 = (bx[5] - r.o.z) * r.invd.z;
    float tn = fmaxf(fmaxf(lo, fminf(tx0, tx1)), fmaxf(fminf(ty0, ty1), fminf(tz0, tz1)));
    float tf = fminf(fminf(hi, fmaxf(tx0, tx1)), fminf(fmaxf(ty0, ty1), fmaxf(tz0, tz1)));
    return tn <= tf;
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

// Warp-cooperative traversal for the chunk [tb, seg_hi] of every active lane.  Appends hit leaves
// with index > cursor to the warp list; returns the entry count.  `ovf` is set when the list
// filled up before the traversal finished.
template <int CAP>
__device__ int traverse(WarpSmem<CAP>& sm, const RenderArgs& a, const RayState& r, bool on, float seg_hi,
                        int K, int nv, int cursor, bool& ovf, int lane) {
    int count = 0;
    ovf = false;
    int sp = 0;
    int cur = (a.n_leaves == 1) ? ~0 : 0;
    long long guard = 0;
    const long long guard_max = 4ll * a.n_leaves + 64;
    while (true) {
        if (++guard > guard_max) {
            if (lane == 0) atomicAdd(&a.st->watchdog_trips, 1ull);
            break;
        }
        if (cur >= 0) {
            const float4* np = reinterpret_cast<const float4*>(a.nodes + cur);
            float4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2);
            int4 n3 = __ldg(reinterpret_cast<const int4*>(np + 3));
            float lb[6] = {n0.x, n0.y, n0.z, n0.w, n1.x, n1.y};
            float rb[6] = {n1.z, n1.w, n2.x, n2.y, n2.z, n2.w};
            bool hl = on && n3.z > cursor && box_hit(lb, r, r.tb, seg_hi);
            bool hr = on && n3.w > cursor && box_hit(rb, r, r.tb, seg_hi);
            unsigned bl = __ballot_sync(kFull, hl), br = __ballot_sync(kFull, hr);
            if (bl && br) {
                if (sp < kStack) {
                    if (lane == 0) sm.stack[sp] = n3.y;
                    ++sp;
                } else if (lane == 0) {
                    atomicAdd(&a.st->stack_overflows, 1ull);
                }
                __syncwarp();
                cur = n3.x;
                continue;
            }
            if (bl) { cur = n3.x; continue; }
            if (br) { cur = n3.y; continue; }
        } else {
            int leaf = ~cur;
            if (leaf > cursor) {
                LeafRec rec = load_rec(a.rec, leaf);
                unsigned m = 0;
                if (on) {
                    // exact interval against the threshold ellipsoid (reference IS program)
                    float3 O = r.o - f3(rec.a.x, rec.a.y, rec.a.z);
                    float k = rec.r0.w;
                    float3 r0 = f3(rec.r0.x, rec.r0.y, rec.r0.z), r1 = f3(rec.r1.x, rec.r1.y, rec.r1.z),
                           r2 = f3(rec.r2.x, rec.r2.y, rec.r2.z);
                    float3 Oe = f3(dot3(r0, O) * k, dot3(r1, O) * k, dot3(r2, O) * k);
                    float3 De = f3(dot3(r0, r.d) * k, dot3(r1, r.d) * k, dot3(r2, r.d) * k);
                    float l = 1.f / sqrtf(dot3(De, De));
                    float3 Dn = De * l;
                    float b = -dot3(Oe, Dn);
                    float c = dot3(Oe, Oe) - 1.f;
                    float3 p = Oe + Dn * b;
                    float disc = 1.f - dot3(p, p);
                    if (disc > 1e-7f) {
                        float sd = sqrtf(disc);
                        float q = b + (b > 0.f ? sd : -sd);
                        float root1 = (c / q) * l, root2 = q * l;
                        float t = r.tb;
#pragma unroll
                        for (int kk = 0; kk < kMaxChunk; ++kk) {
                            if (kk < nv) {
                                float tn = t + kSlab;
                                float hi = fminf(r.texit, tn);
                                if (hi > r.tenter && fmaxf(t, root1) <= fminf(hi, root2)) m |= 1u << kk;
                                t = tn;
                            }
                        }
                    }
                }
                unsigned any = __ballot_sync(kFull, m != 0u);
                if (any) {
                    if (count == CAP) {
                        ovf = true;
                        break;
                    }
                    if (lane == 0) sm.ids[count] = leaf;
                    for (int kk = 0; kk < K; ++kk) {
                        unsigned wk = __ballot_sync(kFull, (m >> kk) & 1u);
                        if (lane == kk) sm.mask[kk][count] = wk;
                    }
                    ++count;
                }
            }
        }
        if (sp == 0) break;
        __syncwarp();
        cur = sm.stack[--sp];
    }
    __syncwarp();
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

// Sample buffers of slab k: sum of density and density-weighted colour of the lane's hits.
template <bool FAST, int CAP>
__device__ __forceinline__ int slab_buffers(const WarpSmem<CAP>& sm, int count, int k, bool has, const RayState& r,
                                            const RenderArgs& a, long long rgb_base, const float* roff,
                                            float* sig, float3* C, int lane) {
    int nh = 0;
    const unsigned bit = 1u << lane;
    for (int e = 0; e < count; ++e) {
        unsigned w = sm.mask[k][e];
        if (w == 0u) continue;
        if (has && (w & bit)) {
            int leaf = sm.ids[e];
            LeafRec rec = load_rec(a.rec, leaf);
            float4 col4 = __ldg(a.rgb + rgb_base + leaf);
            float3 mu = f3(rec.a.x, rec.a.y, rec.a.z);
            float dn = rec.a.w;
            float3 r0 = f3(rec.r0.x, rec.r0.y, rec.r0.z), r1 = f3(rec.r1.x, rec.r1.y, rec.r1.z),
                   r2 = f3(rec.r2.x, rec.r2.y, rec.r2.z);
            float3 col = f3(col4.x, col4.y, col4.z);
            ++nh;
            if (FAST) {
                float3 v0 = (r.o + r.d * r.tb) - mu;
                float3 vb = r.d * kDt;
                float3 m0 = f3(dot3(r0, v0), dot3(r1, v0), dot3(r2, v0));
                float3 mb = f3(dot3(r0, vb), dot3(r1, vb), dot3(r2, vb));
                float A = dot3(m0, m0), B2 = 2.f * dot3(m0, mb), Cq = dot3(mb, mb);
#pragma unroll
                for (int i = 0; i < kBuf; ++i) {
                    float fi = (float)i;
                    float qv = fmaf(fi, fmaf(fi, Cq, B2), A);
                    float dw = dn * ex2_approx(kNegHalfLog2e * qv);
                    if (dw > kSigThr) {
                        sig[i] += dw;
                        C[i] = C[i] + col * dw;
                    }
                }
            } else {
#pragma unroll
                for (int i = 0; i < kBuf; ++i) {
                    float t = r.tb + (float)i * kDt;
                    if (a.rnd_sample) t += roff[i];
                    float3 v = (r.o + r.d * t) - mu;
                    float3 m = f3(dot3(r0, v), dot3(r1, v), dot3(r2, v));
                    float w = expf(-0.5f * dot3(m, m));
                    if (dn * w > kSigThr) {
                        sig[i] += dn * w;
                        C[i] = C[i] + (col * w) * dn;
                    }
                }
            }
        }
    }
    return nh;
}

template <bool FAST>
__device__ __forceinline__ float exp_neg(float x) {
    // exp(-x) for the compositing alpha
    return FAST ? ex2_approx(-x * 1.4426950408889634f) : expf(-x);
}

template <bool FAST>
__device__ __forceinline__ void composite(RayState& r, const float* sig, const float3* C) {
#pragma unroll
    for (int i = 0; i < kBuf; ++i) {
        float alpha = 1.f - exp_neg<FAST>(sig[i] * kDt);
        float3 c = C[i];
        if (sig[i] > 0.f) c = c * (1.f / sig[i]);
        r.C = r.C + c * (r.T * alpha);
        r.T *= 1.f - alpha;
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

// Adjoint of slab k for all list entries: per-lane gradient of each hit Gaussian, warp reduction,
// one set of vector atomics per entry.
template <bool FAST, int CAP>
__device__ __forceinline__ void slab_adjoint(const WarpSmem<CAP>& sm, int count, int k, bool has, const RayState& r,
                                             const RenderArgs& a, int view, long long rgb_base, const float* roff,
                                             const float* E, const float* F, const float* G, int lane) {
    const unsigned bit = 1u << lane;
    for (int e = 0; e < count; ++e) {
        unsigned w = sm.mask[k][e];
        if (w == 0u) continue;
        bool act = has && (w & bit);
        unsigned am = __ballot_sync(kFull, act);
        if (am == 0u) continue;
        int leaf = sm.ids[e];
        float v[14];
#pragma unroll
        for (int z = 0; z < 14; ++z) v[z] = 0.f;
        if (act) {
            LeafRec rec = load_rec(a.rec, leaf);
            float4 col4 = __ldg(a.rgb + rgb_base + leaf);
            float4 s4 = __ldg(a.ext + 2 * (long long)leaf);
            float4 q4 = __ldg(a.ext + 2 * (long long)leaf + 1);
            float3 mu = f3(rec.a.x, rec.a.y, rec.a.z);
            float dn = rec.a.w;
            float3 r0 = f3(rec.r0.x, rec.r0.y, rec.r0.z), r1 = f3(rec.r1.x, rec.r1.y, rec.r1.z),
                   r2 = f3(rec.r2.x, rec.r2.y, rec.r2.z);
            float gcol = r.g.x * col4.x + r.g.y * col4.y + r.g.z * col4.z;
            float gc = 0.f, dd = 0.f;
            float3 dsc = f3(0.f, 0.f, 0.f), dp = f3(0.f, 0.f, 0.f);
            float3 d1 = f3(0.f, 0.f, 0.f), d2 = f3(0.f, 0.f, 0.f), d3 = f3(0.f, 0.f, 0.f);
            if (FAST) {
                float3 v0 = (r.o + r.d * r.tb) - mu;
                float3 vb = r.d * kDt;
                float3 m0 = f3(dot3(r0, v0), dot3(r1, v0), dot3(r2, v0));
                float3 mb = f3(dot3(r0, vb), dot3(r1, vb), dot3(r2, vb));
                float A = dot3(m0, m0), B2 = 2.f * dot3(m0, mb), Cq = dot3(mb, mb);
                float U0 = 0.f, U1 = 0.f, U2 = 0.f;
#pragma unroll
                for (int i = 0; i < kBuf; ++i) {
                    float fi = (float)i;
                    float qv = fmaf(fi, fmaf(fi, Cq, B2), A);
                    float wt = ex2_approx(kNegHalfLog2e * qv);
                    if (dn * wt > kSigThr) {
                        float h = E[i] + F[i] * (gcol - G[i]);
                        gc += wt * F[i];
                        dd += wt * h;
                        float u = h * wt;
                        U0 += u;
                        U1 += fi * u;
                        U2 += fi * fi * u;
                    }
                }
                gc *= dn;
                U0 *= dn; U1 *= dn; U2 *= dn;
                float3 Sm = m0 * U0 + mb * U1;
                float3 Smm = f3(m0.x * m0.x * U0 + 2.f * m0.x * mb.x * U1 + mb.x * mb.x * U2,
                                m0.y * m0.y * U0 + 2.f * m0.y * mb.y * U1 + mb.y * mb.y * U2,
                                m0.z * m0.z * U0 + 2.f * m0.z * mb.z * U1 + mb.z * mb.z * U2);
                dsc = f3(Smm.x / s4.x, Smm.y / s4.y, Smm.z / s4.z);
                dp = f3(r0.x * Sm.x + r1.x * Sm.y + r2.x * Sm.z, r0.y * Sm.x + r1.y * Sm.y + r2.y * Sm.z,
                        r0.z * Sm.x + r1.z * Sm.y + r2.z * Sm.z);
                // P[:, j] = sum_i u_i v_i m_ij with v_i = v0 + i vb, m_i = m0 + i mb
                float3 P0 = v0 * (m0.x * U0 + mb.x * U1) + vb * (m0.x * U1 + mb.x * U2);
                float3 P1 = v0 * (m0.y * U0 + mb.y * U1) + vb * (m0.y * U1 + mb.y * U2);
                float3 P2 = v0 * (m0.z * U0 + mb.z * U1) + vb * (m0.z * U1 + mb.z * U2);
                d1 = P0 * (-1.f / s4.x);
                d2 = P1 * (-1.f / s4.y);
                d3 = P2 * (-1.f / s4.z);
            } else {
#pragma unroll
                for (int i = 0; i < kBuf; ++i) {
                    float t = r.tb + (float)i * kDt;
                    if (a.rnd_sample) t += roff[i];
                    float3 vv = (r.o + r.d * t) - mu;
                    float3 m = f3(dot3(r0, vv), dot3(r1, vv), dot3(r2, vv));
                    float wt = expf(-0.5f * dot3(m, m));
                    if (dn * wt > kSigThr) {
                        float h = E[i] + F[i] * (gcol - G[i]);
                        gc += wt * dn * F[i];
                        dd += wt * h;
                        float u = dn * h * wt;
                        dsc.x += u * (m.x * m.x) / s4.x;
                        dsc.y += u * (m.y * m.y) / s4.y;
                        dsc.z += u * (m.z * m.z) / s4.z;
                        dp.x += u * (r0.x * m.x + r1.x * m.y + r2.x * m.z);
                        dp.y += u * (r0.y * m.x + r1.y * m.y + r2.y * m.z);
                        dp.z += u * (r0.z * m.x + r1.z * m.y + r2.z * m.z);
                        d1 = d1 - vv * (u * m.x / s4.x);
                        d2 = d2 - vv * (u * m.y / s4.y);
                        d3 = d3 - vv * (u * m.z / s4.z);
                    }
                }
            }
            float4 dq = quat_grad(q4, d1, d2, d3);
            v[0] = dd; v[1] = dp.x; v[2] = dp.y; v[3] = dp.z;
            v[4] = dsc.x; v[5] = dsc.y; v[6] = dsc.z;
            v[7] = dq.x; v[8] = dq.y; v[9] = dq.z; v[10] = dq.w;
            v[11] = r.g.x * gc; v[12] = r.g.y * gc; v[13] = r.g.z * gc;
        }
        int leader = __ffs(am) - 1;
        if (__popc(am) > 1) {
#pragma unroll
            for (int z = 0; z < 14; ++z) {
#pragma unroll
                for (int o = 16; o; o >>= 1) v[z] += __shfl_xor_sync(kFull, v[z], o);
            }
        }
        if (lane == leader) {
            float4* gg = a.gacc_geo + 3 * (long long)leaf;
            atomicAdd(gg, make_float4(v[0], v[1], v[2], v[3]));
            atomicAdd(gg + 1, make_float4(v[4], v[5], v[6], 0.f));
            atomicAdd(gg + 2, make_float4(v[7], v[8], v[9], v[10]));
            atomicAdd(a.gacc_rgb + rgb_base + leaf, make_float4(v[11], v[12], v[13], 0.f));
        }
    }
}

template <bool BWD, bool FAST, int CAP>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) k_render(RenderArgs a) {
    __shared__ WarpSmem<CAP> smem[kWarpsPerBlock];
    const int lane = threadIdx.x & 31;
    WarpSmem<CAP>& sm = smem[threadIdx.x >> 5];
    const ViewTable* vt = a.views;
    const float bg = a.white_bg ? 1.f : 0.f;
    float scene[6];
#pragma unroll
    for (int z = 0; z < 6; ++z) scene[z] = ord2f(a.scene_ord[z]);
    unsigned long long hits_acc = 0, slabs_acc = 0;

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
        const long long ray_g = vt->ray_prefix[view] + (long long)ray_l;
        const long long rgb_base = (long long)view * a.n_leaves;

        RayState r;
        r.seed = tea4(a.iteration, ray_l);
        {
            float ix, iy;
            if (a.jitter == 1) {
                float jx = lcg_rnd(r.seed) * 0.333333f;
                float jy = lcg_rnd(r.seed) * 0.333333f;
                ix = ((float)(ray_l % (unsigned)W) + 0.333333f + jx) / (float)W;
                iy = ((float)(ray_l / (unsigned)W) + 0.333333f + jy) / (float)H;
            } else {
                ix = ((float)(ray_l % (unsigned)W) + 0.5f) / (float)W;
                iy = ((float)(ray_l / (unsigned)W) + 0.5f) / (float)H;
            }
            float dx = (2.f * ix - 1.f) * cam.tan_half_fovx;
            float dy = (2.f * iy - 1.f) * cam.tan_half_fovy;
            float3 dir = f3(dx * cam.u[0] + dy * cam.v[0] + cam.w[0], dx * cam.u[1] + dy * cam.v[1] + cam.w[1],
                            dx * cam.u[2] + dy * cam.v[2] + cam.w[2]);
            float inv = 1.f / sqrtf(dot3(dir, dir));
            r.d = dir * inv;
            r.o = f3(cam.eye[0], cam.eye[1], cam.eye[2]);
        }
        {
            float t0x = (scene[0] - r.o.x) / r.d.x, t1x = (scene[3] - r.o.x) / r.d.x;
            float t0y = (scene[1] - r.o.y) / r.d.y, t1y = (scene[4] - r.o.y) / r.d.y;
            float t0z = (scene[2] - r.o.z) / r.d.z, t1z = (scene[5] - r.o.z) / r.d.z;
            r.tenter = fmaxf(0.f, fmaxf(fminf(t0x, t1x), fmaxf(fminf(t0y, t1y), fminf(t0z, t1z))));
            r.texit = fminf(fmaxf(t0x, t1x), fminf(fmaxf(t0y, t1y), fmaxf(t0z, t1z)));
        }
        {
            const float tiny = 1e-20f;
            r.invd = f3(1.f / (fabsf(r.d.x) > tiny ? r.d.x : copysignf(tiny, r.d.x)),
                        1.f / (fabsf(r.d.y) > tiny ? r.d.y : copysignf(tiny, r.d.y)),
                        1.f / (fabsf(r.d.z) > tiny ? r.d.z : copysignf(tiny, r.d.z)));
        }
        r.alive = valid && (r.tenter < r.texit);
        r.tb = r.tenter;
        r.T = 1.f;
        if (BWD) {
            if (valid) {
                r.C = f3(a.ray_colors_in[3 * ray_g], a.ray_colors_in[3 * ray_g + 1], a.ray_colors_in[3 * ray_g + 2]);
                r.g = f3(a.dL[3 * ray_g], a.dL[3 * ray_g + 1], a.dL[3 * ray_g + 2]);
            } else {
                r.C = f3(0.f, 0.f, 0.f);
                r.g = f3(0.f, 0.f, 0.f);
            }
        } else {
            r.C = f3(0.f, 0.f, 0.f);
            r.g = f3(0.f, 0.f, 0.f);
        }

        int K = a.chunk_slabs;
        int rounds = 0;
        while (true) {
            bool on = r.alive;
            if (!__any_sync(kFull, on)) break;
            if (++rounds > kMaxRounds) {
                if (lane == 0) atomicAdd(&a.st->watchdog_trips, 1ull);
                break;
            }
            // slabs of this chunk: slab k is marched iff tb_k < texit (tb_k by repeated addition)
            int nv = 0;
            float seg_hi = r.tb;
            if (on) {
                float t = r.tb;
                for (int kk = 0; kk < K; ++kk) {
                    if (t < r.texit) { nv = kk + 1; t = t + kSlab; } else break;
                }
                seg_hi = fminf(r.texit, t);
                // a slab step that no longer changes tb (|t| beyond ~2^19) would march forever
                if (nv == 0 || r.tb + kSlab == r.tb) { r.alive = false; on = false; nv = 0; }
            }
            bool ovf;
            int count = traverse<CAP>(sm, a, r, on, seg_hi, K, nv, -1, ovf, lane);
            if (ovf && K > 1) {
                K = max(1, K >> 1);
                if (lane == 0) atomicAdd(&a.st->chunk_splits, 1ull);
                continue;
            }
            if (!ovf) {
                for (int k = 0; k < K; ++k) {
                    bool has = on && k < nv && r.T > kTeps;
                    float roff[kBuf];
                    unsigned seed_next = slab_offsets(a.rnd_sample, r.seed, roff);
                    float sig[kBuf];
                    float3 Cb[kBuf];
#pragma unroll
                    for (int i = 0; i < kBuf; ++i) { sig[i] = 0.f; Cb[i] = f3(0.f, 0.f, 0.f); }
                    int nh = slab_buffers<FAST, CAP>(sm, count, k, has, r, a, rgb_base, roff, sig, Cb, lane);
                    if (has) {
                        ++slabs_acc;
                        hits_acc += nh;
                        if (nh > a.max_prim_slice) atomicAdd(&a.st->slab_cap_exceeded, 1ull);
                    }
                    if (!BWD) {
                        if (has && nh > 0) {
                            composite<FAST>(r, sig, Cb);
                            r.seed = seed_next;
                        }
                    } else {
                        float E[kBuf], F[kBuf], G[kBuf];
                        float Ta = r.T;
                        float3 Ra = r.C;
#pragma unroll
                        for (int i = 0; i < kBuf; ++i) {
                            float cd = sig[i];
                            float3 cc = Cb[i];
                            if (cd > 0.f) cc = cc * (1.f / cd);
                            float alpha = 1.f - exp_neg<FAST>(cd * kDt);
                            float3 aux = (cc * Ta - Ra) * kDt;
                            E[i] = dot3(r.g, aux);
                            F[i] = cd > 0.f ? Ta * alpha / cd : 0.f;
                            G[i] = dot3(r.g, cc);
                            Ra = Ra - cc * (Ta * alpha);
                            Ta *= 1.f - alpha;
                        }
                        bool act = has && nh > 0;
                        slab_adjoint<FAST, CAP>(sm, count, k, act, r, a, view, rgb_base, roff, E, F, G, lane);
                        if (act) {
                            r.T = Ta;
                            r.C = Ra;
                            r.seed = seed_next;
                        }
                    }
                    if (has) r.tb = r.tb + kSlab;
                }
                if (count < CAP / 4 && K < a.chunk_slabs) K = min(a.chunk_slabs, K << 1);
            } else {
                // K == 1 and more hits than the list holds: consume the slab in several passes
                bool has = on && nv > 0 && r.T > kTeps;
                float roff[kBuf];
                unsigned seed_next = slab_offsets(a.rnd_sample, r.seed, roff);
                float sig[kBuf];
                float3 Cb[kBuf];
#pragma unroll
                for (int i = 0; i < kBuf; ++i) { sig[i] = 0.f; Cb[i] = f3(0.f, 0.f, 0.f); }
                int nh = slab_buffers<FAST, CAP>(sm, count, 0, has, r, a, rgb_base, roff, sig, Cb, lane);
                bool more = ovf;
                while (more) {
                    int cursor = sm.ids[count - 1];
                    __syncwarp();
                    if (lane == 0) atomicAdd(&a.st->list_passes, 1ull);
                    count = traverse<CAP>(sm, a, r, on, seg_hi, 1, nv, cursor, more, lane);
                    nh += slab_buffers<FAST, CAP>(sm, count, 0, has, r, a, rgb_base, roff, sig, Cb, lane);
                }
                if (has) {
                    ++slabs_acc;
                    hits_acc += nh;
                    if (nh > a.max_prim_slice) atomicAdd(&a.st->slab_cap_exceeded, 1ull);
                }
                if (!BWD) {
                    if (has && nh > 0) {
                        composite<FAST>(r, sig, Cb);
                        r.seed = seed_next;
                    }
                } else {
                    float E[kBuf], F[kBuf], G[kBuf];
                    float Ta = r.T;
                    float3 Ra = r.C;
#pragma unroll
                    for (int i = 0; i < kBuf; ++i) {
                        float cd = sig[i];
                        float3 cc = Cb[i];
                        if (cd > 0.f) cc = cc * (1.f / cd);
                        float alpha = 1.f - exp_neg<FAST>(cd * kDt);
                        float3 aux = (cc * Ta - Ra) * kDt;
                        E[i] = dot3(r.g, aux);
                        F[i] = cd > 0.f ? Ta * alpha / cd : 0.f;
                        G[i] = dot3(r.g, cc);
                        Ra = Ra - cc * (Ta * alpha);
                        Ta *= 1.f - alpha;
                    }
                    bool act = has && nh > 0;
                    int cursor = -1;
                    bool more2 = true;
                    while (more2) {
                        count = traverse<CAP>(sm, a, r, on, seg_hi, 1, nv, cursor, more2, lane);
                        slab_adjoint<FAST, CAP>(sm, count, 0, act, r, a, view, rgb_base, roff, E, F, G, lane);
                        if (more2) cursor = sm.ids[count - 1];
                        __syncwarp();
                    }
                    if (act) {
                        r.T = Ta;
                        r.C = Ra;
                        r.seed = seed_next;
                    }
                }
                if (has) r.tb = r.tb + kSlab;
            }
            if (on) r.alive = r.alive && (r.T > kTeps) && (r.tb < r.texit);
        }
        if (!BWD && valid) {
            a.ray_colors[3 * ray_g] = r.C.x + r.T * bg;
            a.ray_colors[3 * ray_g + 1] = r.C.y + r.T * bg;
            a.ray_colors[3 * ray_g + 2] = r.C.z + r.T * bg;
            if (a.final_T) a.final_T[ray_g] = r.T;
        }
    }
    // counters: warp reduction, one atomic per warp
    for (int o = 16; o; o >>= 1) {
        hits_acc += __shfl_xor_sync(kFull, hits_acc, o);
        slabs_acc += __shfl_xor_sync(kFull, slabs_acc, o);
    }
    if (lane == 0) {
        atomicAdd(&a.st->hit_pairs, hits_acc);
        atomicAdd(&a.st->slabs, slabs_acc);
    }
}

int render_block_threads() { return kWarpsPerBlock * 32; }

size_t render_smem_bytes(bool, int cap) {
    if (cap <= 64) return sizeof(WarpSmem<64>) * kWarpsPerBlock;
    if (cap <= 128) return sizeof(WarpSmem<128>) * kWarpsPerBlock;
    return sizeof(WarpSmem<256>) * kWarpsPerBlock;
}

template <bool BWD, bool FAST>
static cudaError_t launch_cap(int cap, int grid, const RenderArgs& a, cudaStream_t s) {
    const int threads = kWarpsPerBlock * 32;
    if (cap <= 64) k_render<BWD, FAST, 64><<<grid, threads, 0, s>>>(a);
    else if (cap <= 128) k_render<BWD, FAST, 128><<<grid, threads, 0, s>>>(a);
    else k_render<BWD, FAST, 256><<<grid, threads, 0, s>>>(a);
    return cudaGetLastError();
}

template <bool BWD, bool FAST>
static int occ_cap(int cap) {
    int nb = 0;
    const int threads = kWarpsPerBlock * 32;
    if (cap <= 64) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_render<BWD, FAST, 64>, threads, 0);
    else if (cap <= 128) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_render<BWD, FAST, 128>, threads, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_render<BWD, FAST, 256>, threads, 0);
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
