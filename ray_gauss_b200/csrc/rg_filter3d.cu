// The 3D minimum-size filter of the training loop (classes/point_cloud.py:1153-1215,
// compute_3D_filter, run every 100 iterations by scripts/train.py:163-164), fused.
//
// The reference loops over the training cameras in Python, about fifteen torch launches per
// camera: project every Gaussian, keep it when its depth is > 0.2 and its projection falls inside
// the image widened by 15 % on each side, and take the smallest such depth per Gaussian; Gaussians
// no camera sees get the largest depth of those seen; filter_3D = log(0.5 * depth / focal) with
// focal the largest focal length of the cameras.
//
// Here k_filter_depth runs one thread per Gaussian over all cameras staged in shared memory, with
// the same float operations per camera (xyz R + T as an FMA chain, depth clamp at 0.001,
// x / z * f + W / 2, the window tests against the float-rounded bounds), and a block-reduced
// atomic max of the seen depths; k_filter_finish substitutes that maximum for unseen Gaussians and
// writes log((depth * 0.5) * (1 / focal)).
#include <cmath>
#include <cstdint>

#include "rg_common.cuh"

namespace {

constexpr int kFilterThreads = 256;
constexpr int kCamFloats = 20;          // rg_filter_camera in floats
constexpr int kCamsPerStage = 512;      // 40 KB of shared memory per stage

static_assert(sizeof(rg_filter_camera) == kCamFloats * sizeof(float), "rg_filter_camera layout");

__global__ void __launch_bounds__(kFilterThreads) k_filter_depth(long long n, const float* __restrict__ pos,
                                                                 const rg_filter_camera* __restrict__ cams,
                                                                 int n_cams, float* __restrict__ depth,
                                                                 unsigned* __restrict__ max_bits) {
    __shared__ float cs[kCamsPerStage * kCamFloats];
    const long long g = (long long)blockIdx.x * kFilterThreads + threadIdx.x;
    float px = 0.f, py = 0.f, pz = 0.f;
    if (g < n) {
        px = pos[3 * g];
        py = pos[3 * g + 1];
        pz = pos[3 * g + 2];
    }
    float dist = 100000.0f;
    bool seen = false;
    for (int c0 = 0; c0 < n_cams; c0 += kCamsPerStage) {
        const int nc = min(kCamsPerStage, n_cams - c0);
        __syncthreads();
        const float* src = reinterpret_cast<const float*>(cams + c0);
        for (int i = threadIdx.x; i < nc * kCamFloats; i += kFilterThreads) cs[i] = src[i];
        __syncthreads();
        if (g < n) {
            for (int c = 0; c < nc; ++c) {
                const float* k = cs + c * kCamFloats;
                // xyz_cam = xyz @ R + T (row vector times R)
                const float x = __fadd_rn(__fmaf_rn(pz, k[6], __fmaf_rn(py, k[3], __fmul_rn(px, k[0]))), k[9]);
                const float y = __fadd_rn(__fmaf_rn(pz, k[7], __fmaf_rn(py, k[4], __fmul_rn(px, k[1]))), k[10]);
                const float zr = __fadd_rn(__fmaf_rn(pz, k[8], __fmaf_rn(py, k[5], __fmul_rn(px, k[2]))), k[11]);
                const bool front = zr > 0.2f;
                const float z = fmaxf(zr, 0.001f);
                const float sx = __fadd_rn(__fmul_rn(__fdiv_rn(x, z), k[12]), k[14]);
                const float sy = __fadd_rn(__fmul_rn(__fdiv_rn(y, z), k[13]), k[15]);
                const bool inside = sx >= k[16] && sx <= k[17] && sy >= k[18] && sy <= k[19];
                if (front && inside) {
                    dist = fminf(dist, z);
                    seen = true;
                }
            }
        }
    }
    if (g < n) depth[g] = seen ? dist : -1.f;       // -1: seen by no camera
    // block max of the seen depths (positive floats order like their bit patterns)
    float m = seen ? dist : 0.f;
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ float wm[kFilterThreads / 32];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        float b = 0.f;
        for (int w = 0; w < kFilterThreads / 32; ++w) b = fmaxf(b, wm[w]);
        if (b > 0.f) atomicMax(max_bits, __float_as_uint(b));
    }
}

__global__ void __launch_bounds__(kFilterThreads) k_filter_finish(long long n, const float* __restrict__ depth,
                                                                  const unsigned* __restrict__ max_bits,
                                                                  float inv_focal, float* __restrict__ out) {
    const long long g = (long long)blockIdx.x * kFilterThreads + threadIdx.x;
    if (g >= n) return;
    float d = depth[g];
    if (d < 0.f) d = __uint_as_float(*max_bits);
    out[g] = logf(__fmul_rn(__fmul_rn(d, 0.5f), inv_focal));
}

}  // namespace

extern "C" {

int rg_compute_3d_filter(const float* positions, int64_t n, const rg_filter_camera* cameras, int32_t n_cams,
                         float inv_focal, float* depth_scratch, uint32_t* max_scratch, float* filter_out,
                         void* stream) {
    if (n < 0 || n_cams < 0 || (n > 0 && (!positions || !depth_scratch || !max_scratch || !filter_out)) ||
        (n_cams > 0 && !cameras))
        return RG_ERR_INVALID_ARG;
    if (n == 0) return RG_OK;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(max_scratch, 0, sizeof(uint32_t), s) != cudaSuccess) return RG_ERR_CUDA;
    const unsigned blocks = (unsigned)((n + kFilterThreads - 1) / kFilterThreads);
    k_filter_depth<<<blocks, kFilterThreads, 0, s>>>(n, positions, cameras, n_cams, depth_scratch, max_scratch);
    k_filter_finish<<<blocks, kFilterThreads, 0, s>>>(n, depth_scratch, max_scratch, inv_focal, filter_out);
    return cudaGetLastError() == cudaSuccess ? RG_OK : RG_ERR_CUDA;
}

}  // extern "C"
