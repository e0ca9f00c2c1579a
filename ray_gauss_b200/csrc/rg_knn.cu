// Mean squared distance to the 3 nearest neighbours of every point: the initial scale of a point
// cloud without scales (classes/point_cloud.py:374-378 -> distCUDA2 of the simple-knn extension,
// submodules/simple-knn/spatial.cu:14-25 and simple_knn.cu:126-221).
//
// The extension's result is exact: for point i, (d0 + d1 + d2) / 3 with d0 <= d1 <= d2 the three
// smallest squared distances |p_j - p_i|^2 (j != i), each evaluated as dx*dx + dy*dy + dz*dz with
// the multiply-adds contracted, the sum left to right; fewer than three other points leave FLT_MAX
// entries (two neighbours: about FLT_MAX / 3; one or none: +inf).  Its Morton boxes only prune the
// search.
//
// This engine's search: points sorted by a 30-bit Morton code (k_knn_bounds, k_knn_morton, CUB
// radix sort), boxes of kBox consecutive sorted points (k_knn_boxes), then one warp per 32
// consecutive sorted points (k_knn_query): the warp's own box and its neighbours first, then every
// other box whose distance to the warp's query box is at most the warp's largest third-best
// distance; a surviving box's points are loaded once and broadcast by shuffle to all 32 queries.
#include <cfloat>
#include <cstdint>

#include <cub/device/device_radix_sort.cuh>

#include "rg_common.cuh"

namespace {

using rg::f2ord;
using rg::ord2f;

constexpr int kBox = 64;          // sorted points per box: two per lane
constexpr int kNear = 2;          // boxes on each side of the warp's own box scanned first

struct KnnWs {
    int* bounds;                  // 6 ordered ints: scene min, max
    unsigned* keys_in;
    unsigned* keys_out;
    int* vals_in;
    int* vals_out;                // sorted point ids
    float4* box_lo;
    float4* box_hi;
    void* sort_temp;
    size_t sort_bytes;
};

size_t a256(size_t x) { return (x + 255) & ~size_t(255); }

size_t sort_bytes(long long n) {
    size_t b = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, b, (const unsigned*)nullptr, (unsigned*)nullptr, (const int*)nullptr,
                                    (int*)nullptr, (int)n, 0, 30);
    return b;
}

size_t ws_bytes(long long n) {
    const long long nb = (n + kBox - 1) / kBox;
    return 256 + a256(6 * sizeof(int)) + 4 * a256(sizeof(int) * n) + 2 * a256(sizeof(float4) * nb) +
           a256(sort_bytes(n));
}

KnnWs carve(void* base, long long n) {
    uintptr_t p = (reinterpret_cast<uintptr_t>(base) + 255) & ~uintptr_t(255);
    const long long nb = (n + kBox - 1) / kBox;
    KnnWs w;
    w.bounds = reinterpret_cast<int*>(p); p += a256(6 * sizeof(int));
    w.keys_in = reinterpret_cast<unsigned*>(p); p += a256(sizeof(int) * n);
    w.keys_out = reinterpret_cast<unsigned*>(p); p += a256(sizeof(int) * n);
    w.vals_in = reinterpret_cast<int*>(p); p += a256(sizeof(int) * n);
    w.vals_out = reinterpret_cast<int*>(p); p += a256(sizeof(int) * n);
    w.box_lo = reinterpret_cast<float4*>(p); p += a256(sizeof(float4) * nb);
    w.box_hi = reinterpret_cast<float4*>(p); p += a256(sizeof(float4) * nb);
    w.sort_temp = reinterpret_cast<void*>(p);
    w.sort_bytes = sort_bytes(n);
    return w;
}

__global__ void k_knn_init_bounds(int* b) {
    if (threadIdx.x < 3) b[threadIdx.x] = f2ord(INFINITY);
    else if (threadIdx.x < 6) b[threadIdx.x] = f2ord(-INFINITY);
}

__global__ void __launch_bounds__(256) k_knn_bounds(long long n, const float* __restrict__ p, int* __restrict__ b) {
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    if (i < n) {
        for (int a = 0; a < 3; ++a) lo[a] = hi[a] = p[3 * i + a];
    }
    for (int a = 0; a < 3; ++a) {
        for (int o = 16; o; o >>= 1) {
            lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int a = 0; a < 3; ++a) {
            atomicMin(b + a, f2ord(lo[a]));
            atomicMax(b + 3 + a, f2ord(hi[a]));
        }
    }
}

__device__ __forceinline__ unsigned spread10(unsigned v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__global__ void __launch_bounds__(256) k_knn_morton(long long n, const float* __restrict__ p,
                                                    const int* __restrict__ b, unsigned* __restrict__ keys,
                                                    int* __restrict__ vals) {
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
    unsigned q[3];
    for (int a = 0; a < 3; ++a) {
        const float lo = ord2f(b[a]), hi = ord2f(b[3 + a]);
        const float u = hi > lo ? (p[3 * i + a] - lo) / (hi - lo) : 0.f;
        q[a] = (unsigned)fminf(fmaxf(u * 1023.f, 0.f), 1023.f);
    }
    keys[i] = spread10(q[0]) | (spread10(q[1]) << 1) | (spread10(q[2]) << 2);
    vals[i] = (int)i;
}

__global__ void __launch_bounds__(kBox) k_knn_boxes(long long n, const float* __restrict__ p,
                                                    const int* __restrict__ sorted, float4* __restrict__ blo,
                                                    float4* __restrict__ bhi) {
    const long long i = (long long)blockIdx.x * kBox + threadIdx.x;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    if (i < n) {
        const long long s = sorted[i];
        for (int a = 0; a < 3; ++a) lo[a] = hi[a] = p[3 * s + a];
    }
    __shared__ float red[2][3][kBox / 32];
    for (int a = 0; a < 3; ++a) {
        for (int o = 16; o; o >>= 1) {
            lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
        if ((threadIdx.x & 31) == 0) {
            red[0][a][threadIdx.x >> 5] = lo[a];
            red[1][a][threadIdx.x >> 5] = hi[a];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float l[3], h[3];
        for (int a = 0; a < 3; ++a) {
            l[a] = red[0][a][0];
            h[a] = red[1][a][0];
            for (int w = 1; w < kBox / 32; ++w) {
                l[a] = fminf(l[a], red[0][a][w]);
                h[a] = fmaxf(h[a], red[1][a][w]);
            }
        }
        blo[blockIdx.x] = make_float4(l[0], l[1], l[2], 0.f);
        bhi[blockIdx.x] = make_float4(h[0], h[1], h[2], 0.f);
    }
}

__device__ __forceinline__ void insert3(float d, float (&best)[3]) {
    // updateKBest<3>: keep the three smallest in ascending order
    for (int j = 0; j < 3; ++j) {
        if (best[j] > d) {
            const float t = best[j];
            best[j] = d;
            d = t;
        }
    }
}

// The distances from this lane's query to the kBox points of box `bx` (two loaded per lane,
// broadcast by shuffle).
__device__ __forceinline__ void scan_box(long long n, const float* __restrict__ p, const int* __restrict__ sorted,
                                         long long bx, long long me, float3 q, bool active, float (&best)[3],
                                         int lane) {
    float3 v[2];
    long long idx[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        idx[h] = bx * kBox + h * 32 + lane;
        if (idx[h] < n) {
            const long long s = sorted[idx[h]];
            v[h] = make_float3(p[3 * s], p[3 * s + 1], p[3 * s + 2]);
        } else {
            v[h] = make_float3(0.f, 0.f, 0.f);
        }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const long long base = bx * kBox + h * 32;
        const int m = (int)min(32ll, n - base);
        for (int j = 0; j < m; ++j) {
            const float px = __shfl_sync(0xffffffffu, v[h].x, j);
            const float py = __shfl_sync(0xffffffffu, v[h].y, j);
            const float pz = __shfl_sync(0xffffffffu, v[h].z, j);
            if (active && base + j != me) {
                const float dx = px - q.x, dy = py - q.y, dz = pz - q.z;
                insert3(__fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx))), best);
            }
        }
    }
}

__global__ void __launch_bounds__(128) k_knn_query(long long n, const float* __restrict__ p,
                                                   const int* __restrict__ sorted, const float4* __restrict__ blo,
                                                   const float4* __restrict__ bhi, float* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long me = warp * 32 + lane;
    if (warp * 32 >= n) return;                       // whole warp past the end
    const bool active = me < n;
    const long long nb = (n + kBox - 1) / kBox;
    float3 q = make_float3(0.f, 0.f, 0.f);
    if (active) {
        const long long s = sorted[me];
        q = make_float3(p[3 * s], p[3 * s + 1], p[3 * s + 2]);
    }
    // the warp's query box
    float ql[3] = {active ? q.x : INFINITY, active ? q.y : INFINITY, active ? q.z : INFINITY};
    float qh[3] = {active ? q.x : -INFINITY, active ? q.y : -INFINITY, active ? q.z : -INFINITY};
    for (int a = 0; a < 3; ++a) {
        for (int o = 16; o; o >>= 1) {
            ql[a] = fminf(ql[a], __shfl_xor_sync(0xffffffffu, ql[a], o));
            qh[a] = fmaxf(qh[a], __shfl_xor_sync(0xffffffffu, qh[a], o));
        }
    }
    float best[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    const long long own = (warp * 32) / kBox;
    const long long n0 = own - kNear > 0 ? own - kNear : 0;
    const long long n1 = own + kNear < nb - 1 ? own + kNear : nb - 1;
    for (long long bx = n0; bx <= n1; ++bx) scan_box(n, p, sorted, bx, me, q, active, best, lane);
    // every other box within the warp's largest third-best distance of the query box
    for (long long b0 = 0; b0 < nb; b0 += 32) {
        const unsigned lim = __reduce_max_sync(0xffffffffu, active ? __float_as_uint(best[2]) : 0u);
        const float limf = __uint_as_float(lim);
        const long long bx = b0 + lane;
        bool need = false;
        if (bx < nb && (bx < n0 || bx > n1)) {
            const float4 l = blo[bx], h = bhi[bx];
            const float gx = fmaxf(0.f, fmaxf(l.x - qh[0], ql[0] - h.x));
            const float gy = fmaxf(0.f, fmaxf(l.y - qh[1], ql[1] - h.y));
            const float gz = fmaxf(0.f, fmaxf(l.z - qh[2], ql[2] - h.z));
            // skipped only when clearly farther than every lane's third best (a relative margin
            // keeps rounding of the gap from dropping a point at the tie distance)
            need = !(__fmul_rn(gx * gx + gy * gy + gz * gz, 0.999999f) > limf);
        }
        unsigned m = __ballot_sync(0xffffffffu, need);
        while (m) {
            const int j = __ffs(m) - 1;
            m &= m - 1;
            // the box passed the warp test; scan it only when some lane's own point is close enough
            const float4 l = blo[b0 + j], h = bhi[b0 + j];
            const float gx = fmaxf(0.f, fmaxf(l.x - q.x, q.x - h.x));
            const float gy = fmaxf(0.f, fmaxf(l.y - q.y, q.y - h.y));
            const float gz = fmaxf(0.f, fmaxf(l.z - q.z, q.z - h.z));
            const bool mine = active && !(__fmul_rn(gx * gx + gy * gy + gz * gz, 0.999999f) > best[2]);
            if (__any_sync(0xffffffffu, mine)) scan_box(n, p, sorted, b0 + j, me, q, active, best, lane);
        }
    }
    if (active) out[sorted[me]] = __fdiv_rn(__fadd_rn(__fadd_rn(best[0], best[1]), best[2]), 3.0f);
}

}  // namespace

extern "C" {

int rg_knn_workspace_bytes(int64_t n, uint64_t* bytes) {
    if (!bytes || n < 0 || n > INT32_MAX) return RG_ERR_INVALID_ARG;
    *bytes = ws_bytes(n);
    return RG_OK;
}

int rg_knn_mean_dist(const float* points, int64_t n, float* mean_dist, void* workspace, void* stream) {
    if (n < 0 || n > INT32_MAX || (n > 0 && (!points || !mean_dist || !workspace))) return RG_ERR_INVALID_ARG;
    if (n == 0) return RG_OK;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    KnnWs w = carve(workspace, n);
    const unsigned blocks = (unsigned)((n + 255) / 256);
    k_knn_init_bounds<<<1, 32, 0, s>>>(w.bounds);
    k_knn_bounds<<<blocks, 256, 0, s>>>(n, points, w.bounds);
    k_knn_morton<<<blocks, 256, 0, s>>>(n, points, w.bounds, w.keys_in, w.vals_in);
    size_t bytes = w.sort_bytes;
    if (cub::DeviceRadixSort::SortPairs(w.sort_temp, bytes, w.keys_in, w.keys_out, w.vals_in, w.vals_out, (int)n, 0,
                                        30, s) != cudaSuccess)
        return RG_ERR_CUDA;
    const long long nb = (n + kBox - 1) / kBox;
    k_knn_boxes<<<(unsigned)nb, kBox, 0, s>>>(n, points, w.vals_out, w.box_lo, w.box_hi);
    const long long warps = (n + 31) / 32;
    k_knn_query<<<(unsigned)((warps + 3) / 4), 128, 0, s>>>(n, points, w.vals_out, w.box_lo, w.box_hi, mean_dist);
    return cudaGetLastError() == cudaSuccess ? RG_OK : RG_ERR_CUDA;
}

}  // extern "C"
