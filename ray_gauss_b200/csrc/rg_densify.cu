// Densification: clone, split and prune of the Gaussians with their Adam moments and statistics,
// as the reference's densify_and_prune (classes/point_cloud.py:1068-1143) with the optimizer-state
// surgery of classes/optimizer.py:54-83 (_prune_optimizer / _cat_tensor: moments of new rows are
// zero, moments of kept rows move with them).
//
// The reference's result, in order: the original Gaussians that survive, then the clones, then
// split copy 0 of every split Gaussian, then split copy 1, ... each segment in Gaussian order and
// with the Gaussians whose density is <= min_density removed.  Clone and split selections are
// disjoint (max scale <= vs > the threshold), so every output row is (source Gaussian, kind) with
// kind 0 = original, 1 = clone, 2 + c = split copy c.
//
//   rg_densify_plan   k_dens_classify  per Gaussian: mean gradient, selections, survival flags and
//                                      per-block counts of the four scanned predicates
//                     k_dens_scan_blocks  exclusive scan of the block counts (one block)
//                     -> the counts are read back on the host (the output size)
//   rg_densify_apply  k_dens_index     block-local ranks -> the source map of every output row
//                     k_dens_gather    one thread per output float of every tensor: copy, zero, or
//                                      the transform of its role (halved densities, split positions
//                                      and log scales)
// Arithmetic follows the torch expressions of the reference operation by operation (no contraction):
// grads = accum / num (NaN -> 0); max(exp(scales)) against 0.01 * extent; densities * 0.5;
// build_rotation (utils/general_utils.py:466-487) of the normalised quaternion; samples = z * std;
// new position = R sample + mu; new log scale = log(exp(s) * (1 / (0.8 n_split))).
#include <cmath>
#include <cstdint>
#include <cstring>

#include "rg_common.cuh"

namespace {

constexpr int kDensThreads = 1024;
constexpr int kDensCols = 5;           // keep_orig, keep_clone, keep_split, split_sel, clone_sel
constexpr int kMaxSplit = 8;

enum : unsigned char { F_KEEP_ORIG = 1, F_CLONE = 2, F_KEEP_CLONE = 4, F_SPLIT = 8, F_KEEP_SPLIT = 16 };

struct Workspace {
    unsigned char* flags;   // (N)
    int* blk_cnt;           // (nblk, 5)
    int* blk_off;           // (nblk, 5)
    long long* totals;      // 8
    int* split_rank;        // (N)
    int2* map;              // (N * (1 + max(1, n_split)))
};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

long long n_blocks(long long n) { return (n + kDensThreads - 1) / kDensThreads; }

long long max_out(long long n, int n_split) { return n * (1 + (n_split > 1 ? n_split : 1)); }

size_t workspace_bytes(long long n, int n_split) {
    const long long nb = n_blocks(n);
    return align256(n) + 2 * align256(sizeof(int) * kDensCols * nb) + align256(8 * sizeof(long long)) +
           align256(sizeof(int) * n) + align256(sizeof(int2) * max_out(n, n_split)) + 256;
}

Workspace carve(void* base, long long n, int n_split) {
    uintptr_t p = (reinterpret_cast<uintptr_t>(base) + 255) & ~uintptr_t(255);
    const long long nb = n_blocks(n);
    Workspace w;
    w.flags = reinterpret_cast<unsigned char*>(p);
    p += align256(n);
    w.blk_cnt = reinterpret_cast<int*>(p);
    p += align256(sizeof(int) * kDensCols * nb);
    w.blk_off = reinterpret_cast<int*>(p);
    p += align256(sizeof(int) * kDensCols * nb);
    w.totals = reinterpret_cast<long long*>(p);
    p += align256(8 * sizeof(long long));
    w.split_rank = reinterpret_cast<int*>(p);
    p += align256(sizeof(int) * n);
    w.map = reinterpret_cast<int2*>(p);
    (void)n_split;
    return w;
}

__global__ void __launch_bounds__(kDensThreads) k_dens_classify(long long n, const float* __restrict__ accum,
                                                                const float* __restrict__ num,
                                                                const float* __restrict__ log_scales,
                                                                const float* __restrict__ dens, float grad_thr,
                                                                float scale_thr, float min_density, Workspace w) {
    const long long i = (long long)blockIdx.x * kDensThreads + threadIdx.x;
    unsigned char f = 0;
    if (i < n) {
        float g = __fdiv_rn(accum[i], num[i]);
        if (isnan(g)) g = 0.f;                          // grads[grads.isnan()] = 0.0
        const bool big = g >= grad_thr;
        const float s0 = expf(log_scales[3 * i]), s1 = expf(log_scales[3 * i + 1]),
                    s2 = expf(log_scales[3 * i + 2]);
        // torch.max over the row propagates NaN
        const float smax = (isnan(s0) || isnan(s1) || isnan(s2)) ? s0 + s1 + s2 : fmaxf(fmaxf(s0, s1), s2);
        const bool clone = big && smax <= scale_thr;
        const bool split = big && smax > scale_thr;
        const float d = dens[i];
        const float half = __fmul_rn(d, 0.5f);
        const float d_orig = clone ? half : d;       // the clone step halves the original too
        if (!split && !(d_orig <= min_density)) f |= F_KEEP_ORIG;
        if (clone) f |= F_CLONE;
        if (clone && !(half <= min_density)) f |= F_KEEP_CLONE;
        if (split) f |= F_SPLIT;
        if (split && !(half <= min_density)) f |= F_KEEP_SPLIT;
        w.flags[i] = f;
    }
    const int c0 = __syncthreads_count(f & F_KEEP_ORIG);
    const int c1 = __syncthreads_count(f & F_KEEP_CLONE);
    const int c2 = __syncthreads_count(f & F_KEEP_SPLIT);
    const int c3 = __syncthreads_count(f & F_SPLIT);
    const int c4 = __syncthreads_count(f & F_CLONE);
    if (threadIdx.x == 0) {
        int* o = w.blk_cnt + (long long)kDensCols * blockIdx.x;
        o[0] = c0; o[1] = c1; o[2] = c2; o[3] = c3; o[4] = c4;
    }
}

// Exclusive scan of the per-block counts, one column per pass, in chunks of kDensThreads blocks.
__global__ void __launch_bounds__(kDensThreads) k_dens_scan_blocks(long long nb, Workspace w) {
    __shared__ int warp_sum[32];
    __shared__ long long carry;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int col = 0; col < kDensCols; ++col) {
        if (threadIdx.x == 0) carry = 0;
        __syncthreads();
        for (long long base = 0; base < nb; base += kDensThreads) {
            const long long b = base + threadIdx.x;
            const int v = b < nb ? w.blk_cnt[kDensCols * b + col] : 0;
            int x = v;  // inclusive warp scan
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (lane == 31) warp_sum[wid] = x;
            __syncthreads();
            if (wid == 0) {
                int s = warp_sum[lane];
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, s, o);
                    if (lane >= o) s += y;
                }
                warp_sum[lane] = s;  // inclusive over warps
            }
            __syncthreads();
            const long long excl = carry + (wid ? warp_sum[wid - 1] : 0) + (x - v);
            if (b < nb) w.blk_off[kDensCols * b + col] = (int)excl;
            __syncthreads();
            if (threadIdx.x == 0) carry += warp_sum[31];
            __syncthreads();
        }
        if (threadIdx.x == 0) w.totals[col] = carry;
        __syncthreads();
    }
}

// Block-local exclusive ranks of the four scanned predicates; each Gaussian writes the map entries
// of its output rows and its split rank (the row of its standard normals).
__global__ void __launch_bounds__(kDensThreads) k_dens_index(long long n, int n_split, long long k_orig,
                                                             long long k_clone, long long k_split, Workspace w) {
    __shared__ int wsum[4][32];
    const long long i = (long long)blockIdx.x * kDensThreads + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned char f = i < n ? w.flags[i] : 0;
    const bool pred[4] = {(f & F_KEEP_ORIG) != 0, (f & F_KEEP_CLONE) != 0, (f & F_KEEP_SPLIT) != 0,
                          (f & F_SPLIT) != 0};
    int rank[4];
    const unsigned lower = (1u << lane) - 1u;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const unsigned b = __ballot_sync(0xffffffffu, pred[j]);
        rank[j] = __popc(b & lower);
        if (lane == 0) wsum[j][wid] = __popc(b);
    }
    __syncthreads();
    if (wid < 4) {
        int s = wsum[wid][lane];
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        wsum[wid][lane] = s - wsum[wid][lane];  // exclusive over the block's warps
    }
    __syncthreads();
    if (i >= n) return;
    const int* off = w.blk_off + (long long)kDensCols * blockIdx.x;
    long long r[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) r[j] = (long long)off[j] + wsum[j][wid] + rank[j];
    const int src = (int)i;
    if (pred[0]) w.map[r[0]] = make_int2(src, 0);
    if (pred[1]) w.map[k_orig + r[1]] = make_int2(src, 1);
    if (pred[2]) {
        for (int c = 0; c < n_split; ++c) w.map[k_orig + k_clone + c * k_split + r[2]] = make_int2(src, 2 + c);
    }
    if (pred[3]) w.split_rank[i] = (int)r[3];
}

struct GatherArgs {
    rg_densify_tensor t[RG_DENSIFY_MAX_TENSORS];
    int n_tensors;
    long long n_out;
    long long n_split_sel;
    float split_mul;
    const float* log_scales;
    const float* quaternions;
    const float* normals;
    Workspace w;
};

// (R sample) row c of build_rotation(q) applied to z * exp(log_scale), in the reference's operation
// order (torch elementwise ops: each product and sum rounded; the 3x3 product as an fma chain).
__device__ float split_offset(const GatherArgs& a, int s, int copy, int c) {
    const float4 q4 = reinterpret_cast<const float4*>(a.quaternions)[s];
    const float nq = __fsqrt_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(q4.x, q4.x), __fmul_rn(q4.y, q4.y)),
                                                    __fmul_rn(q4.z, q4.z)),
                                          __fmul_rn(q4.w, q4.w)));
    const float r = __fdiv_rn(q4.x, nq), x = __fdiv_rn(q4.y, nq), y = __fdiv_rn(q4.z, nq), z = __fdiv_rn(q4.w, nq);
    float R0, R1, R2;
    if (c == 0) {
        R0 = __fsub_rn(1.f, __fmul_rn(2.f, __fadd_rn(__fmul_rn(y, y), __fmul_rn(z, z))));
        R1 = __fmul_rn(2.f, __fsub_rn(__fmul_rn(x, y), __fmul_rn(r, z)));
        R2 = __fmul_rn(2.f, __fadd_rn(__fmul_rn(x, z), __fmul_rn(r, y)));
    } else if (c == 1) {
        R0 = __fmul_rn(2.f, __fadd_rn(__fmul_rn(x, y), __fmul_rn(r, z)));
        R1 = __fsub_rn(1.f, __fmul_rn(2.f, __fadd_rn(__fmul_rn(x, x), __fmul_rn(z, z))));
        R2 = __fmul_rn(2.f, __fsub_rn(__fmul_rn(y, z), __fmul_rn(r, x)));
    } else {
        R0 = __fmul_rn(2.f, __fsub_rn(__fmul_rn(x, z), __fmul_rn(r, y)));
        R1 = __fmul_rn(2.f, __fadd_rn(__fmul_rn(y, z), __fmul_rn(r, x)));
        R2 = __fsub_rn(1.f, __fmul_rn(2.f, __fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y))));
    }
    const long long row = (long long)copy * a.n_split_sel + a.w.split_rank[s];
    const float* zr = a.normals + 3 * row;
    const float* ls = a.log_scales + 3 * (long long)s;
    const float v0 = __fmul_rn(zr[0], expf(ls[0])), v1 = __fmul_rn(zr[1], expf(ls[1])),
                v2 = __fmul_rn(zr[2], expf(ls[2]));
    return __fmaf_rn(R2, v2, __fmaf_rn(R1, v1, __fmul_rn(R0, v0)));
}

// One output element of a tensor of kind K: copy, zero, or the role's transform.
template <int K, typename Idx>
__device__ __forceinline__ float dens_value(const GatherArgs& a, const rg_densify_tensor& t, Idx e, Idx w) {
    if (K == RG_DENSIFY_ZERO) return 0.f;
    const Idx o = e / w;
    const int c = (int)(e - o * w);
    const int2 m = a.w.map[o];
    const long long si = (long long)m.x * w + c;
    if (K == RG_DENSIFY_OLD_ONLY) return m.y == 0 ? t.src[si] : 0.f;
    float v = t.src[si];
    if (K == RG_DENSIFY_DENSITIES) {
        if (m.y != 0 || (a.w.flags[m.x] & F_CLONE)) v = __fmul_rn(v, 0.5f);
    } else if (K == RG_DENSIFY_LOG_SCALES) {
        if (m.y >= 2) v = logf(__fmul_rn(expf(v), a.split_mul));
    } else if (K == RG_DENSIFY_POSITIONS) {
        if (m.y >= 2) v = __fadd_rn(split_offset(a, m.x, m.y - 2, c), v);
    }
    return v;
}

// Grid-stride over the tensor's output floats, kUnroll independent elements per thread per pass so
// that several loads are in flight before the first store.
constexpr int kUnroll = 4;

template <int K, typename Idx>
__device__ __forceinline__ void dens_gather_tensor(const GatherArgs& a, const rg_densify_tensor& t) {
    const Idx w = (Idx)t.width;
    const Idx total = (Idx)a.n_out * w;
    const Idx stride = (Idx)gridDim.x * blockDim.x;
    for (Idx base = (Idx)blockIdx.x * blockDim.x + threadIdx.x; base < total; base += kUnroll * stride) {
        float v[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const Idx e = base + u * stride;
            v[u] = e < total ? dens_value<K>(a, t, e, w) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const Idx e = base + u * stride;
            if (e < total) t.dst[e] = v[u];
        }
    }
}

// blockIdx.y selects the tensor.  Index type: 32-bit when every tensor's output fits (the row/column
// split is then a 32-bit divide).
template <typename Idx>
__global__ void __launch_bounds__(256) k_dens_gather(const GatherArgs a) {
    const rg_densify_tensor& t = a.t[blockIdx.y];
    switch (t.kind) {
        case RG_DENSIFY_ZERO: dens_gather_tensor<RG_DENSIFY_ZERO, Idx>(a, t); break;
        case RG_DENSIFY_OLD_ONLY: dens_gather_tensor<RG_DENSIFY_OLD_ONLY, Idx>(a, t); break;
        case RG_DENSIFY_DENSITIES: dens_gather_tensor<RG_DENSIFY_DENSITIES, Idx>(a, t); break;
        case RG_DENSIFY_LOG_SCALES: dens_gather_tensor<RG_DENSIFY_LOG_SCALES, Idx>(a, t); break;
        case RG_DENSIFY_POSITIONS: dens_gather_tensor<RG_DENSIFY_POSITIONS, Idx>(a, t); break;
        default: dens_gather_tensor<RG_DENSIFY_COPY, Idx>(a, t); break;
    }
}

int check_plan(const rg_densify* d) {
    if (!d || d->n < 0 || d->n > (long long)INT32_MAX / (1 + kMaxSplit)) return RG_ERR_INVALID_ARG;
    if (d->n_split < 1 || d->n_split > kMaxSplit) return RG_ERR_INVALID_ARG;
    if (d->n > 0 && (!d->grad_accum || !d->num_accum || !d->log_scales || !d->densities || !d->workspace))
        return RG_ERR_INVALID_ARG;
    return RG_OK;
}

}  // namespace

extern "C" {

int rg_densify_workspace_bytes(int64_t n, int32_t n_split, uint64_t* bytes) {
    if (!bytes || n < 0 || n_split < 1 || n_split > kMaxSplit) return RG_ERR_INVALID_ARG;
    *bytes = workspace_bytes(n, n_split);
    return RG_OK;
}

int rg_densify_plan(rg_densify* d, void* stream) {
    int rc = check_plan(d);
    if (rc) return rc;
    d->planned = 0;
    d->n_clone = d->n_split_sel = d->n_out = d->n_kept = 0;
    if (d->n == 0) {
        d->planned = 1;
        return RG_OK;
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const Workspace w = carve(d->workspace, d->n, d->n_split);
    const long long nb = n_blocks(d->n);
    k_dens_classify<<<(unsigned)nb, kDensThreads, 0, s>>>(d->n, d->grad_accum, d->num_accum, d->log_scales,
                                                          d->densities, d->grad_threshold, d->scale_threshold,
                                                          d->min_density, w);
    k_dens_scan_blocks<<<1, kDensThreads, 0, s>>>(nb, w);
    long long tot[kDensCols];
    if (cudaMemcpyAsync(tot, w.totals, sizeof(tot), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return RG_ERR_CUDA;
    d->n_kept = tot[0];
    d->n_split_sel = tot[3];
    d->n_clone = tot[4];
    d->n_out = tot[0] + tot[1] + (long long)d->n_split * tot[2];
    d->kept_clones = tot[1];
    d->kept_splits = tot[2];
    d->planned = 1;
    return RG_OK;
}

int rg_densify_apply(const rg_densify* d, const float* split_normals, const rg_densify_tensor* tensors,
                     int32_t n_tensors, void* stream) {
    int rc = check_plan(d);
    if (rc) return rc;
    if (!d->planned || n_tensors < 0 || n_tensors > RG_DENSIFY_MAX_TENSORS || (n_tensors && !tensors))
        return RG_ERR_INVALID_ARG;
    bool need_quat = false;
    for (int i = 0; i < n_tensors; ++i) {
        const rg_densify_tensor& t = tensors[i];
        if (t.width <= 0 || t.kind < RG_DENSIFY_COPY || t.kind > RG_DENSIFY_POSITIONS) return RG_ERR_INVALID_ARG;
        if (d->n_out > 0 && !t.dst) return RG_ERR_INVALID_ARG;
        if (t.kind != RG_DENSIFY_ZERO && d->n > 0 && !t.src) return RG_ERR_INVALID_ARG;
        if ((t.kind == RG_DENSIFY_POSITIONS || t.kind == RG_DENSIFY_LOG_SCALES) && t.width != 3)
            return RG_ERR_INVALID_ARG;
        if (t.kind == RG_DENSIFY_DENSITIES && t.width != 1) return RG_ERR_INVALID_ARG;
        if (t.kind == RG_DENSIFY_POSITIONS) need_quat = true;
    }
    if (need_quat && d->n_split_sel > 0 &&
        (!d->quaternions || !split_normals || ((uintptr_t)d->quaternions & 15) != 0))
        return RG_ERR_INVALID_ARG;
    if (d->n == 0 || d->n_out == 0 || n_tensors == 0) return RG_OK;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    GatherArgs a;
    std::memset(&a, 0, sizeof(a));
    a.w = carve(d->workspace, d->n, d->n_split);
    const long long nb = n_blocks(d->n);
    k_dens_index<<<(unsigned)nb, kDensThreads, 0, s>>>(d->n, d->n_split, d->n_kept, d->kept_clones, d->kept_splits,
                                                       a.w);
    std::memcpy(a.t, tensors, sizeof(rg_densify_tensor) * n_tensors);
    a.n_tensors = n_tensors;
    a.n_out = d->n_out;
    a.n_split_sel = d->n_split_sel;
    a.split_mul = d->split_scale_mul;
    a.log_scales = d->log_scales;
    a.quaternions = d->quaternions;
    a.normals = split_normals;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    long long maxw = 1;
    for (int i = 0; i < n_tensors; ++i) maxw = tensors[i].width > maxw ? tensors[i].width : maxw;
    long long want = (d->n_out * maxw + 255) / 256;
    const long long cap = (long long)sms * 8;
    const unsigned gx = (unsigned)(want < cap ? (want > 0 ? want : 1) : cap);
    if (d->n_out * maxw + (long long)kUnroll * gx * 256 < (long long)UINT32_MAX)
        k_dens_gather<unsigned><<<dim3(gx, (unsigned)n_tensors), 256, 0, s>>>(a);
    else
        k_dens_gather<unsigned long long><<<dim3(gx, (unsigned)n_tensors), 256, 0, s>>>(a);
    return cudaGetLastError() == cudaSuccess ? RG_OK : RG_ERR_CUDA;
}

}  // extern "C"
