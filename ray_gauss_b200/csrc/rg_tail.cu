// Fused training-step tail: Adam on every parameter tensor of the Gaussians, the densification
// statistics and the parameter clamps in one launch.
//
// Reference semantics (paths inside the reference project):
//   statistics   scripts/train.py:121-123 -> classes/point_cloud.py:633-640 (accumulate_gradient,
//                accumulate_gradient_gaussians_not_visible: |dL/dposition| summed, visible counts)
//   Adam         classes/optimizer.py:13-21, 203-218 (one torch.optim.Adam per tensor, eps 1e-15,
//                default betas; learning rates and step counts come from the host)
//   clamps       scripts/train.py:166-181 (densities < 0 -> 0, quaternion and lobe-axis
//                normalisation, log scales clamped to [filter_3D, max_scale]) with
//                classes/point_cloud.py:703-727 (zero-norm quaternion -> (1,0,0,0), zero-norm
//                axis -> (0,0,1))
// Adam per element, as torch.optim.Adam:  m += (1 - beta1) (g - m);  v = beta2 v + (1 - beta2) g^2;
// p -= (lr / (1 - beta1^t)) * m / (sqrt(v) / sqrt(1 - beta2^t) + eps).
//
// Layout: a block owns kTailGaussians consecutive Gaussians.  For each tensor it streams the block's
// contiguous element range [g0 * width, g1 * width) with coalesced float4 accesses (scalar when a
// pointer is not 16-byte aligned), then, after a block barrier, one thread per Gaussian applies the
// statistics and the clamps to the values the block has just written.  Every byte is read and
// written once: HBM-bound at 28 bytes per parameter float (param, m, v read and written, grad read).
#include <cmath>
#include <cstdint>
#include <cstring>

#include "rg_common.cuh"

namespace {

constexpr int kTailMaxTensors = RG_TAIL_MAX_TENSORS;
constexpr int kTailThreads = 256;
constexpr int kTailGaussians = 256;

struct TailArgs {
    rg_train_tail d;
};

struct AdamStep {
    float w1, w2, beta2, eps, step_size, bias2_sqrt;
};

__device__ __forceinline__ void adam1(float& p, float g, float& m, float& v, const AdamStep& s) {
    m = m + s.w1 * (g - m);
    v = s.beta2 * v + s.w2 * g * g;
    p -= s.step_size * (m / (sqrtf(v) / s.bias2_sqrt + s.eps));
}

__device__ void adam_range(const rg_adam_tensor& t, const AdamStep& s, long long e0, long long e1) {
    const bool vec = (((uintptr_t)t.param | (uintptr_t)t.grad | (uintptr_t)t.exp_avg | (uintptr_t)t.exp_avg_sq) &
                      15) == 0 && (e0 & 3) == 0;
    long long e = e0;
    if (vec) {
        const long long nv = (e1 - e0) >> 2;
        float4* P = reinterpret_cast<float4*>(t.param + e0);
        const float4* G = reinterpret_cast<const float4*>(t.grad + e0);
        float4* M = reinterpret_cast<float4*>(t.exp_avg + e0);
        float4* V = reinterpret_cast<float4*>(t.exp_avg_sq + e0);
        for (long long j = threadIdx.x; j < nv; j += kTailThreads) {
            float4 p = P[j], m = M[j], v = V[j];
            const float4 g = __ldcs(G + j);
            adam1(p.x, g.x, m.x, v.x, s);
            adam1(p.y, g.y, m.y, v.y, s);
            adam1(p.z, g.z, m.z, v.z, s);
            adam1(p.w, g.w, m.w, v.w, s);
            P[j] = p;
            M[j] = m;
            V[j] = v;
        }
        e = e0 + 4 * nv;
    }
    for (long long j = e + threadIdx.x; j < e1; j += kTailThreads) {
        float p = t.param[j], m = t.exp_avg[j], v = t.exp_avg_sq[j];
        adam1(p, t.grad[j], m, v, s);
        t.param[j] = p;
        t.exp_avg[j] = m;
        t.exp_avg_sq[j] = v;
    }
}

__global__ void __launch_bounds__(kTailThreads) k_train_tail(const TailArgs args) {
    const rg_train_tail& d = args.d;
    const long long g0 = (long long)blockIdx.x * kTailGaussians;
    const long long g1 = g0 + kTailGaussians < d.n ? g0 + kTailGaussians : d.n;
    for (int i = 0; i < d.n_tensors && i < kTailMaxTensors; ++i) {
        const rg_adam_tensor& t = d.tensors[i];
        if (!t.active || !t.grad || !t.param || t.width <= 0) continue;
        float lr = t.lr, bias1 = t.bias1, bias2_sqrt = t.bias2_sqrt;
        if (d.step_scalars) {
            const float* sc = d.step_scalars + 4 * i;
            if (sc[0] == 0.f) continue;
            lr = sc[1];
            bias1 = sc[2];
            bias2_sqrt = sc[3];
        }
        const AdamStep s{t.one_minus_beta1, t.one_minus_beta2, t.beta2, t.eps, lr / bias1, bias2_sqrt};
        adam_range(t, s, g0 * t.width, g1 * t.width);
    }
    __syncthreads();  // the clamps below read parameters that other threads of the block stepped
    const long long g = g0 + threadIdx.x;
    if (g >= g1) return;
    // densification statistics from the position gradient
    if (d.idx_positions >= 0 && d.tensors[d.idx_positions].grad &&
        (d.grad_norm_accum || d.num_accum || d.num_accum_gnv)) {
        const float* gp = d.tensors[d.idx_positions].grad + 3 * g;
        const float gn = sqrtf(gp[0] * gp[0] + gp[1] * gp[1] + gp[2] * gp[2]);
        if (d.grad_norm_accum) d.grad_norm_accum[g] += gn;
        if (d.num_accum && gn > 0.f) d.num_accum[g] += 1.f;
        if (d.num_accum_gnv && gn > 0.f) d.num_accum_gnv[g] += 1.f;
    }
    // clamps after the step
    if (d.idx_densities >= 0) {
        float* p = d.tensors[d.idx_densities].param + g;
        if (*p < 0.f) *p = 0.f;
    }
    if (d.normalize_quaternions && d.idx_quaternions >= 0) {
        float4* qp = reinterpret_cast<float4*>(d.tensors[d.idx_quaternions].param) + g;
        float4 q = *qp;
        float nn = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
        if (nn == 0.f) { q = make_float4(1.f, 0.f, 0.f, 0.f); nn = 1.f; }
        *qp = make_float4(q.x / nn, q.y / nn, q.z / nn, q.w / nn);
    }
    if (d.normalize_lobe_axis && d.idx_lobe_axis >= 0 && d.tensors[d.idx_lobe_axis].width > 0) {
        const rg_adam_tensor& t = d.tensors[d.idx_lobe_axis];
        for (int l = 0; l < t.width / 3; ++l) {
            float* ax = t.param + g * t.width + 3 * l;
            float nn = sqrtf(ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2]);
            if (nn == 0.f) { ax[0] = 0.f; ax[1] = 0.f; ax[2] = 1.f; nn = 1.f; }
            for (int k = 0; k < 3; ++k) ax[k] /= nn;
        }
    }
    if (d.idx_scales >= 0) {
        float* s = d.tensors[d.idx_scales].param + 3 * g;
        const float lo = d.min_scale ? d.min_scale[g] : -INFINITY;
        for (int k = 0; k < 3; ++k) {
            float v = s[k];
            if (v < lo) v = lo;
            if (v > d.max_scale) v = d.max_scale;
            s[k] = v;
        }
    }
}

int check_tail(const rg_train_tail* d) {
    if (!d || d->n < 0 || d->n_tensors < 0 || d->n_tensors > kTailMaxTensors) return RG_ERR_INVALID_ARG;
    const int idx[5] = {d->idx_positions, d->idx_densities, d->idx_scales, d->idx_quaternions, d->idx_lobe_axis};
    const int width[5] = {3, 1, 3, 4, -1};
    for (int j = 0; j < 5; ++j) {
        if (idx[j] < -1 || idx[j] >= d->n_tensors) return RG_ERR_INVALID_ARG;
        if (idx[j] >= 0) {
            const rg_adam_tensor& t = d->tensors[idx[j]];
            // a lobe-axis tensor may have zero width (no SG lobes unlocked yet)
            if ((!t.param && t.width != 0) || (width[j] > 0 && t.width != width[j]) ||
                (width[j] < 0 && t.width % 3 != 0))
                return RG_ERR_INVALID_ARG;
        }
    }
    // the quaternion clamp reads and writes float4 rows
    if (d->normalize_quaternions && d->idx_quaternions >= 0 &&
        ((uintptr_t)d->tensors[d->idx_quaternions].param & 15) != 0)
        return RG_ERR_INVALID_ARG;
    for (int i = 0; i < d->n_tensors; ++i) {
        const rg_adam_tensor& t = d->tensors[i];
        if (!t.active) continue;
        if (!t.param || !t.exp_avg || !t.exp_avg_sq || t.width <= 0) return RG_ERR_INVALID_ARG;
        if (!d->step_scalars && (!(t.bias1 > 0.f) || !(t.bias2_sqrt > 0.f))) return RG_ERR_INVALID_ARG;
    }
    return RG_OK;
}

}  // namespace

extern "C" {

int rg_train_tail_step(const rg_train_tail* d, void* stream) {
    int rc = check_tail(d);
    if (rc) return rc;
    if (d->n == 0) return RG_OK;
    TailArgs a;
    std::memcpy(&a.d, d, sizeof(rg_train_tail));
    const long long blocks = (d->n + kTailGaussians - 1) / kTailGaussians;
    k_train_tail<<<(unsigned)blocks, kTailThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(a);
    return cudaGetLastError() == cudaSuccess ? RG_OK : RG_ERR_CUDA;
}

}  // extern "C"
