// Per-Gaussian pre-pass (threshold-ellipsoid AABB, scene box, leaf records) and the LBVH:
// 63-bit Morton codes, radix sort, Karras (2012) hierarchy, bottom-up refit.
//
// Reference: the AABB formula is optix_raycasting/optix_utils.py:34-66 and the scene box
// render_optix.py:105-106; the BVH replaces the OptiX GAS built by optix_utils.py:68-75.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <climits>

#include "rg_common.cuh"
#include "rg_kernels.h"

namespace rg {

__global__ void k_reset_box(int* scene_ord) {
    int t = threadIdx.x;
    if (t < 3) scene_ord[t] = f2ord(INFINITY);
    else if (t < 6) scene_ord[t] = f2ord(-INFINITY);
}

// One thread per Gaussian: AABB of the ellipsoid where density*exp(-r^2/2) > 0.1, the leaf record
// (mu, density, M = S^-1 R^T rows, threshold factor k) in Gaussian order, and a block-reduced
// contribution to the scene box.
__global__ void __launch_bounds__(256) k_prepass(long long n, const float* __restrict__ pos,
                                                 const float* __restrict__ scl, const float4* __restrict__ quat,
                                                 const void* __restrict__ dens, int storage,
                                                 GaussRec* __restrict__ rec, float* __restrict__ aabb,
                                                 int* __restrict__ scene_ord, DevStatus* st) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    if (g < n) {
        float px = pos[3 * g], py = pos[3 * g + 1], pz = pos[3 * g + 2];
        float sx = scl[3 * g], sy = scl[3 * g + 1], sz = scl[3 * g + 2];
        float4 q = quat[g];
        float d = load_param(dens, g, storage);
        bool finite = isfinite(px) && isfinite(py) && isfinite(pz) && isfinite(sx) && isfinite(sy) &&
                      isfinite(sz) && isfinite(q.x) && isfinite(q.y) && isfinite(q.z) && isfinite(q.w) &&
                      isfinite(d);
        float w = q.x, x = q.y, y = q.z, z = q.w;
        // Rotation matrix R of the (w,x,y,z) polynomial (optix_utils.py:34-46), the threshold scale
        // and the AABB, in IEEE operation order (no contraction) so that the scene box, the slab grid
        // anchored on it and the sample positions reproduce the FP32 reference arithmetic.
#define MUL __fmul_rn
#define ADD __fadd_rn
#define SUB __fsub_rn
        float R00 = SUB(1.f, MUL(2.f, ADD(MUL(y, y), MUL(z, z)))), R01 = MUL(2.f, SUB(MUL(x, y), MUL(w, z)));
        float R02 = MUL(2.f, ADD(MUL(x, z), MUL(w, y))), R10 = MUL(2.f, ADD(MUL(x, y), MUL(w, z)));
        float R11 = SUB(1.f, MUL(2.f, ADD(MUL(x, x), MUL(z, z)))), R12 = MUL(2.f, SUB(MUL(y, z), MUL(w, x)));
        float R20 = MUL(2.f, SUB(MUL(x, z), MUL(w, y))), R21 = MUL(2.f, ADD(MUL(y, z), MUL(w, x)));
        float R22 = SUB(1.f, MUL(2.f, ADD(MUL(x, x), MUL(y, y))));
        float ratio = __fdiv_rn(d, 0.1f);
        float lg = (float)log((double)MUL(ratio, ratio));   // correctly rounded log
        float delta = __fsqrt_rn(fmaxf(lg, 0.f));
        float ds0 = MUL(delta, sx), ds1 = MUL(delta, sy), ds2 = MUL(delta, sz);
        float e00 = MUL(ds0, R00), e01 = MUL(ds1, R01), e02 = MUL(ds2, R02);
        float e10 = MUL(ds0, R10), e11 = MUL(ds1, R11), e12 = MUL(ds2, R12);
        float e20 = MUL(ds0, R20), e21 = MUL(ds1, R21), e22 = MUL(ds2, R22);
        float e0 = __fsqrt_rn(ADD(ADD(MUL(e00, e00), MUL(e01, e01)), MUL(e02, e02)));
        float e1 = __fsqrt_rn(ADD(ADD(MUL(e10, e10), MUL(e11, e11)), MUL(e12, e12)));
        float e2 = __fsqrt_rn(ADD(ADD(MUL(e20, e20), MUL(e21, e21)), MUL(e22, e22)));
        float ix = __fdiv_rn(1.f, sx), iy = __fdiv_rn(1.f, sy), iz = __fdiv_rn(1.f, sz);
        LeafRec r;
        // m_j = (column j of R) . (x - mu) / s_j
        r.a = make_float4(px, py, pz, d);
        r.r0 = make_float4(MUL(R00, ix), MUL(R10, ix), MUL(R20, ix), 1.f / sqrtf(lg));
        // .w: log2(density) and 1 / density for the fast sample arithmetic (per Gaussian, not per sample)
        r.r1 = make_float4(MUL(R01, iy), MUL(R11, iy), MUL(R21, iy), lg2_approx(d));
        r.r2 = make_float4(MUL(R02, iz), MUL(R12, iz), MUL(R22, iz), __fdividef(1.f, d));
        float b[6] = {SUB(px, e0), SUB(py, e1), SUB(pz, e2), ADD(px, e0), ADD(py, e1), ADD(pz, e2)};
        // reference intersection-program conic: s' = s sqrt(log(ratio^2)) (NaN below the threshold)
        float dl_is = __fsqrt_rn(lg);
        float jx = __fdiv_rn(1.f, MUL(sx, dl_is)), jy = __fdiv_rn(1.f, MUL(sy, dl_is)),
              jz = __fdiv_rn(1.f, MUL(sz, dl_is));
        LeafIS is;
        is.u = make_float4(MUL(R00, jx), MUL(R10, jx), MUL(R20, jx), dl_is);   // .w: inference conic scale
        is.v = make_float4(MUL(R01, jy), MUL(R11, jy), MUL(R21, jy), 0.f);
        is.w = make_float4(MUL(R02, jz), MUL(R12, jz), MUL(R22, jz), 0.f);
#undef MUL
#undef ADD
#undef SUB
        if (!finite) {
            atomicAdd(&st->nonfinite_inputs, 1ull);
            r.a = make_float4(0.f, 0.f, 0.f, 0.f);
            r.r0.w = __int_as_float(0x7fc00000);  // NaN threshold factor: never hit
            is.u.x = __int_as_float(0x7fc00000);
        }
        rec[g].s = r;
        rec[g].is = is;
        if (aabb) {
            for (int a = 0; a < 6; ++a) aabb[6 * g + a] = finite ? b[a] : (a < 3 ? INFINITY : -INFINITY);
        }
        if (finite) {
            lo[0] = b[0]; lo[1] = b[1]; lo[2] = b[2];
            hi[0] = b[3]; hi[1] = b[4]; hi[2] = b[5];
        }
    }
    // warp then block reduction of the scene box
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        for (int o = 16; o; o >>= 1) {
            lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    }
    __shared__ float sb[8][6];
    int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        for (int a = 0; a < 3; ++a) { sb[wid][a] = lo[a]; sb[wid][3 + a] = hi[a]; }
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        int a = threadIdx.x;
        float v = sb[0][a];
        int nw = blockDim.x >> 5;
        for (int w2 = 1; w2 < nw; ++w2) v = (a < 3) ? fminf(v, sb[w2][a]) : fmaxf(v, sb[w2][a]);
        if (a < 3) {
            if (v < INFINITY) atomicMin(&scene_ord[a], f2ord(v));
        } else {
            if (v > -INFINITY) atomicMax(&scene_ord[a], f2ord(v));
        }
    }
}

__global__ void k_scene_out(const int* scene_ord, float* out) {
    int t = threadIdx.x;
    if (t < 6) out[t] = ord2f(scene_ord[t]);
}

// Spread the low 21 bits of v so that bit i lands at bit 3i.
__device__ __forceinline__ unsigned long long spread3(unsigned long long v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

__global__ void k_morton(long long n, const float* __restrict__ aabb, const int* __restrict__ scene_ord,
                         unsigned long long* __restrict__ keys, int* __restrict__ vals) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    float c[3];
    for (int a = 0; a < 3; ++a) {
        float l = aabb[6 * g + a], h = aabb[6 * g + 3 + a];
        float slo = ord2f(scene_ord[a]), shi = ord2f(scene_ord[3 + a]);
        float ctr = (l <= h) ? 0.5f * (l + h) : slo;
        float ext = shi - slo;
        float u = ext > 0.f ? (ctr - slo) / ext : 0.f;
        c[a] = fminf(fmaxf(u, 0.f), 1.f);
    }
    const float scale = 2097152.0f;  // 2^21
    unsigned long long qx = (unsigned long long)fminf(c[0] * scale, 2097151.f);
    unsigned long long qy = (unsigned long long)fminf(c[1] * scale, 2097151.f);
    unsigned long long qz = (unsigned long long)fminf(c[2] * scale, 2097151.f);
    keys[g] = (spread3(qx) << 2) | (spread3(qy) << 1) | spread3(qz);
    vals[g] = (int)g;
}

// Leaf-ordered records and slightly inflated leaf boxes (the exact test decides; the boxes only
// need to be conservative), plus the Gaussian -> leaf rank.
__global__ void k_leaves(long long n, const int* __restrict__ leaf_gid, const GaussRec* __restrict__ rec,
                         const float* __restrict__ aabb, const float* __restrict__ scl,
                         const float4* __restrict__ quat, LeafRec* __restrict__ leaf_rec, LeafIS* __restrict__ leaf_is,
                         float4* __restrict__ leaf_ext, float4* __restrict__ leaf_lo, float4* __restrict__ leaf_hi,
                         int* __restrict__ rank) {
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n) return;
    int g = leaf_gid[l];
    leaf_rec[l] = rec[g].s;
    leaf_is[l] = rec[g].is;
    rank[g] = (int)l;
    leaf_ext[2 * l] = make_float4(scl[3 * (long long)g], scl[3 * (long long)g + 1], scl[3 * (long long)g + 2], 0.f);
    leaf_ext[2 * l + 1] = quat[g];
    float b[6];
    for (int a = 0; a < 6; ++a) b[a] = aabb[6 * (long long)g + a];
    float lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        float m = 1e-5f * (fabsf(b[a]) + fabsf(b[3 + a])) + 1e-7f;
        lo[a] = b[a] - m;
        hi[a] = b[3 + a] + m;
    }
    leaf_lo[l] = make_float4(lo[0], lo[1], lo[2], 0.f);
    leaf_hi[l] = make_float4(hi[0], hi[1], hi[2], 0.f);
}

__device__ __forceinline__ int kdelta(const unsigned long long* keys, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    unsigned long long a = keys[i], b = keys[j];
    if (a == b) return 64 + __clz(i ^ j);
    return __clzll(a ^ b);
}

// Karras 2012: one thread per internal node i in [0, n-2].
__global__ void k_karras(int n, const unsigned long long* __restrict__ keys, Node* __restrict__ nodes,
                         int* __restrict__ leaf_parent, int* __restrict__ node_parent) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d = (kdelta(keys, n, i, i + 1) - kdelta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = kdelta(keys, n, i, i - d);
    int lmax = 2;
    while (kdelta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (kdelta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = kdelta(keys, n, i, j);
    int s = 0;
    int t = l;
    do {
        t = (t + 1) >> 1;
        if (kdelta(keys, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    int gamma = i + s * d + min(d, 0);
    int lo = min(i, j), hi = max(i, j);
    int left = (lo == gamma) ? ~gamma : gamma;
    int right = (hi == gamma + 1) ? ~(gamma + 1) : gamma + 1;
    nodes[i].n3 = make_int4(left, right, gamma, hi);
    if (left < 0) leaf_parent[~left] = i; else node_parent[left] = i;
    if (right < 0) leaf_parent[~right] = i; else node_parent[right] = i;
    if (i == 0) node_parent[0] = -1;
}

// Bottom-up refit: the second thread to reach a node merges its two child boxes and carries the
// union to the node's slot in its parent.
__global__ void k_refit(int n, const float4* __restrict__ leaf_lo, const float4* __restrict__ leaf_hi,
                        Node* nodes, const int* __restrict__ leaf_parent, const int* __restrict__ node_parent,
                        unsigned* cnt, float* root_box) {
    int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n) return;
    float4 a = leaf_lo[l], b = leaf_hi[l];
    float lo[3] = {a.x, a.y, a.z}, hi[3] = {b.x, b.y, b.z};
    if (n == 1) {
        for (int k = 0; k < 3; ++k) { root_box[k] = lo[k]; root_box[3 + k] = hi[k]; }
        return;
    }
    int child = ~l;
    int p = leaf_parent[l];
    for (int level = 0; level < 4096; ++level) {
        float* f = reinterpret_cast<float*>(&nodes[p]);
        int left = nodes[p].n3.x;
        float* slot = (left == child) ? f : f + 6;
        for (int k = 0; k < 3; ++k) { slot[k] = lo[k]; slot[3 + k] = hi[k]; }
        __threadfence();
        unsigned old = atomicAdd(&cnt[p], 1u);
        if (old == 0) return;
        __threadfence();
        volatile float* vf = f;
        for (int k = 0; k < 3; ++k) {
            lo[k] = fminf(vf[k], vf[6 + k]);
            hi[k] = fmaxf(vf[3 + k], vf[9 + k]);
        }
        child = p;
        p = node_parent[p];
        if (p < 0) {
            for (int k = 0; k < 3; ++k) { root_box[k] = lo[k]; root_box[3 + k] = hi[k]; }
            return;
        }
    }
}

// Depth of every binary node below the root (walk to the root; a few dozen steps).
__global__ void k_depth(int n, const int* __restrict__ node_parent, int* __restrict__ depth) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d = 0;
    for (int p = node_parent[i]; p >= 0 && d < 4096; p = node_parent[p]) ++d;
    depth[i] = d;
}

// Frontier of the wide node at binary node i, in leaf order (depth-first, left child first): every
// binary descendant kWideLevels levels down and every leaf reached before.  Calls emit(k, id, box)
// for the k-th child; the box of a child is the one its binary parent stores for it.
template <typename Emit>
__device__ __forceinline__ int wide_frontier(const Node* __restrict__ nodes, int i, Emit emit) {
    struct Entry { int id, level; float b[6]; };
    Entry st[kWideLevels + 2];
    int sp = 0, k = 0;
    auto push_children = [&](int p, int level) {
        const Node nd = nodes[p];
        const float* f = reinterpret_cast<const float*>(&nd);
        Entry r{nd.n3.y, level, {f[6], f[7], f[8], f[9], f[10], f[11]}};
        Entry l{nd.n3.x, level, {f[0], f[1], f[2], f[3], f[4], f[5]}};
        st[sp++] = r;
        st[sp++] = l;
    };
    push_children(i, 1);
    while (sp > 0) {
        const Entry e = st[--sp];
        if (e.id < 0 || e.level == kWideLevels) {
            emit(k, e.id, e.b);
            ++k;
        } else {
            push_children(e.id, e.level + 1);
        }
    }
    return k;
}

// Children of every wide node (binary nodes at depths that are multiples of kWideLevels).
__global__ void k_wide_count(int n, const Node* __restrict__ nodes, const int* __restrict__ depth,
                             int* __restrict__ cnt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    cnt[i] = (depth[i] % kWideLevels == 0) ? wide_frontier(nodes, i, [](int, int, const float*) {}) : 0;
}

__global__ void k_wide_table(int n, const int* __restrict__ cnt, const int* __restrict__ begin,
                             int2* __restrict__ tab) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    tab[i] = make_int2(begin[i], cnt[i]);
}

// Slots of every wide node from the refitted binary boxes (after every build and refit).
__global__ void k_wide_fill(int n, const Node* __restrict__ nodes, const int2* __restrict__ tab,
                            WideSlot* __restrict__ slots) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int2 t = tab[i];
    if (t.y == 0) return;
    WideSlot* out = slots + t.x;
    wide_frontier(nodes, i, [&](int k, int id, const float* b) {
        WideSlot sl;
        for (int a = 0; a < 3; ++a) { sl.lo[a] = b[a]; sl.hi[a] = b[3 + a]; }
        if (id < 0) {
            sl.id = id;
            sl.range_hi = ~id;
        } else {
            const int2 c = tab[id];
            sl.id = wide_pack(c.x, c.y);
            sl.range_hi = nodes[id].n3.w;
        }
        out[k] = sl;
    });
}

// ---- host launchers --------------------------------------------------------------------------

cudaError_t launch_prepass(const rg_gaussians* g, GaussRec* rec, float* aabb, int* scene_ord, DevStatus* st,
                           cudaStream_t s) {
    k_reset_box<<<1, 32, 0, s>>>(scene_ord);
    long long n = g->n;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 0)
        k_prepass<<<blocks, 256, 0, s>>>(n, g->positions, g->scales, reinterpret_cast<const float4*>(g->quaternions),
                                         g->densities, g->storage, rec, aabb, scene_ord, st);
    return cudaGetLastError();
}

cudaError_t launch_scene_out(const int* scene_ord, float* out, cudaStream_t s) {
    k_scene_out<<<1, 32, 0, s>>>(scene_ord, out);
    return cudaGetLastError();
}

// Temporary storage of the radix sort and of the wide-node slot scan (they run one after the other).
size_t sort_temp_bytes(long long n) {
    size_t bytes = 0, scan = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const unsigned long long*)nullptr,
                                    (unsigned long long*)nullptr, (const int*)nullptr, (int*)nullptr, (int)n, 0,
                                    63);
    cub::DeviceScan::ExclusiveSum(nullptr, scan, (const int*)nullptr, (int*)nullptr, (int)(n > 1 ? n - 1 : 1));
    return bytes > scan ? bytes : scan;
}

cudaError_t launch_refit_only(long long n, BvhBuffers& b, cudaStream_t s);

cudaError_t launch_build(long long n, const float* aabb, const int* scene_ord, const GaussRec* rec,
                         const rg_gaussians* g, BvhBuffers& b, cudaStream_t s) {
    int blocks = (int)((n + 255) / 256);
    k_morton<<<blocks, 256, 0, s>>>(n, aabb, scene_ord, b.keys_in, b.vals_in);
    size_t bytes = b.sort_temp_bytes;
    cudaError_t err = cub::DeviceRadixSort::SortPairs(b.sort_temp, bytes, b.keys_in, b.keys_out, b.vals_in,
                                                      b.leaf_gid, (int)n, 0, 63, s);
    if (err != cudaSuccess) return err;
    k_leaves<<<blocks, 256, 0, s>>>(n, b.leaf_gid, rec, aabb, g->scales, reinterpret_cast<const float4*>(g->quaternions),
                                    b.leaf_rec, b.leaf_is, b.leaf_ext, b.leaf_lo, b.leaf_hi, b.rank);
    if (n > 1) {
        int ib = (int)((n - 1 + 255) / 256);
        k_karras<<<ib, 256, 0, s>>>((int)n, b.keys_out, b.nodes, b.leaf_parent, b.node_parent);
        // wide-node layout (topology only): depths, children per wide node, first slots
        k_depth<<<ib, 256, 0, s>>>((int)n, b.node_parent, b.depth);
        k_wide_count<<<ib, 256, 0, s>>>((int)n, b.nodes, b.depth, b.wide_cnt);
        size_t sbytes = b.sort_temp_bytes;
        err = cub::DeviceScan::ExclusiveSum(b.sort_temp, sbytes, b.wide_cnt, b.depth, (int)(n - 1), s);
        if (err != cudaSuccess) return err;
        // the scan overwrote the depths with the first slots; the table keeps {first slot, count}
        k_wide_table<<<ib, 256, 0, s>>>((int)n, b.wide_cnt, b.depth, b.wide_tab);
    }
    return launch_refit_only(n, b, s);
}

cudaError_t launch_refit_only(long long n, BvhBuffers& b, cudaStream_t s) {
    if (n > 1) {
        // the refit counters must start at zero (the allocation-free path's array keeps old contents)
        const cudaError_t err = cudaMemsetAsync(b.refit_cnt, 0, sizeof(unsigned) * (size_t)(n - 1), s);
        if (err != cudaSuccess) return err;
    }
    int blocks = (int)((n + 255) / 256);
    k_refit<<<blocks, 256, 0, s>>>((int)n, b.leaf_lo, b.leaf_hi, b.nodes, b.leaf_parent, b.node_parent, b.refit_cnt,
                                   b.root_box);
    if (n > 1) {
        int ib = (int)((n - 1 + 255) / 256);
        k_wide_fill<<<ib, 256, 0, s>>>((int)n, b.nodes, b.wide_tab, b.slots);
    }
    return cudaGetLastError();
}

cudaError_t launch_refit(long long n, const float* aabb, const GaussRec* rec, const rg_gaussians* g, BvhBuffers& b,
                         cudaStream_t s) {
    int blocks = (int)((n + 255) / 256);
    k_leaves<<<blocks, 256, 0, s>>>(n, b.leaf_gid, rec, aabb, g->scales, reinterpret_cast<const float4*>(g->quaternions),
                                    b.leaf_rec, b.leaf_is, b.leaf_ext, b.leaf_lo, b.leaf_hi, b.rank);
    return launch_refit_only(n, b, s);
}

}  // namespace rg
