// View-dependent colour of every Gaussian for a batch of views (SH degree <= 3 + spherical
// Gaussians) and its backward, fused with the final gradient assembly.
//
// Reference: utils/sh_utils.cu:25-119 (forward_sh), :121-315 (backward_sh), and the gradient
// assembly of optix_raycasting/render_optix.py:170-190.  Coefficients are read once per Gaussian
// and evaluated for all views of the batch; results go to the leaf-ordered colour table that the
// render kernels read.
#include "rg_common.cuh"
#include "rg_kernels.h"

namespace rg {

// Real SH constants (degree 0..3), the standard values used by the reference.
__constant__ float cSH0 = 0.28209479177387814f;
__constant__ float cSH1 = 0.4886025119029199f;
__constant__ float cSH2[5] = {1.0925484305920792f, -1.0925484305920792f, 0.31539156525252005f,
                              -1.0925484305920792f, 0.5462742152960396f};
__constant__ float cSH3[7] = {-0.5900435899266435f, 2.890611442640554f, -0.4570457994644658f,
                              0.3731763325901154f, -0.4570457994644658f, 1.445305721320277f,
                              -0.5900435899266435f};

__device__ __forceinline__ void sh_basis(float x, float y, float z, int deg, float* B) {
    B[0] = cSH0;
    if (deg < 1) return;
    B[1] = -cSH1 * y;
    B[2] = cSH1 * z;
    B[3] = -cSH1 * x;
    if (deg < 2) return;
    float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
    B[4] = cSH2[0] * xy;
    B[5] = cSH2[1] * yz;
    B[6] = cSH2[2] * (2.f * zz - xx - yy);
    B[7] = cSH2[3] * xz;
    B[8] = cSH2[4] * (xx - yy);
    if (deg < 3) return;
    B[9] = cSH3[0] * y * (3.f * xx - yy);
    B[10] = cSH3[1] * xy * z;
    B[11] = cSH3[2] * y * (4.f * zz - xx - yy);
    B[12] = cSH3[3] * z * (2.f * zz - 3.f * xx - 3.f * yy);
    B[13] = cSH3[4] * x * (4.f * zz - xx - yy);
    B[14] = cSH3[5] * z * (xx - yy);
    B[15] = cSH3[6] * x * (xx - 3.f * yy);
}

__global__ void k_setup_views(const rg_camera* __restrict__ cams, int n, ViewTable* vt, int* work_counter) {
    if (threadIdx.x != 0) return;
    int tiles = 0;
    long long rays = 0;
    for (int v = 0; v < n; ++v) {
        vt->tile_prefix[v] = tiles;
        vt->ray_prefix[v] = rays;
        int w = cams[v].width, h = cams[v].height;
        tiles += ((w + kTileW - 1) / kTileW) * ((h + kTileH - 1) / kTileH);
        rays += (long long)w * h;
    }
    vt->tile_prefix[n] = tiles;
    vt->ray_prefix[n] = rays;
    vt->n_views = n;
    vt->total_tiles = tiles;
    vt->total_rays = rays;
    work_counter[0] = 0;
    work_counter[1] = 0;
}

// One thread per Gaussian: rgb for every view (+0.5 offset, no clamp) into the leaf-ordered table.
__global__ void __launch_bounds__(128) k_color_fwd(long long n, const float* __restrict__ pos,
                                                   const void* __restrict__ sh, const void* __restrict__ sg,
                                                   const float* __restrict__ kappa, const float* __restrict__ axis,
                                                   int deg, int nsg, int storage, const rg_camera* __restrict__ cams,
                                                   int n_cams, const int* __restrict__ rank,
                                                   float4* __restrict__ rgb_leaf, float* __restrict__ rgb_out) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const int nsh = (deg + 1) * (deg + 1);
    float coef[3][16];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = 0; k < 16; ++k)
            coef[c][k] = (k < nsh) ? load_param(sh, (g * 3 + c) * nsh + k, storage) : 0.f;
    float px = pos[3 * g], py = pos[3 * g + 1], pz = pos[3 * g + 2];
    int leaf = rank ? rank[g] : (int)g;
    for (int v = 0; v < n_cams; ++v) {
        float dx = px - cams[v].eye[0], dy = py - cams[v].eye[1], dz = pz - cams[v].eye[2];
        float inv = 1.f / sqrtf(dx * dx + dy * dy + dz * dz);
        float x = dx * inv, y = dy * inv, z = dz * inv;
        float res[3] = {0.f, 0.f, 0.f};
        for (int l = 0; l < nsg; ++l) {
            long long b = g * nsg + l;
            float wgt = expf(kappa[b] * ((x * axis[3 * b] + y * axis[3 * b + 1] + z * axis[3 * b + 2]) - 1.f));
#pragma unroll
            for (int c = 0; c < 3; ++c) res[c] += load_param(sg, (g * 3 + c) * nsg + l, storage) * wgt;
        }
        float B[16];
        sh_basis(x, y, z, deg, B);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
#pragma unroll
            for (int k = 0; k < 16; ++k)
                if (k < nsh) res[c] += B[k] * coef[c][k];
            res[c] += 0.5f;
        }
        rgb_leaf[(long long)v * n + leaf] = make_float4(res[0], res[1], res[2], 0.f);
        if (rgb_out) {
            float* o = rgb_out + ((long long)v * n + g) * 3;
            o[0] = res[0]; o[1] = res[1]; o[2] = res[2];
        }
    }
}

// One thread per Gaussian: gather the leaf-ordered accumulators, run the SH backward for every view,
// add its view-direction term to the position gradient and write the geometry, density and SH
// gradients.  The spherical Gaussians follow in k_color_bwd_sg.
__global__ void __launch_bounds__(128) k_color_bwd(long long n, const float* __restrict__ pos,
                                                   const void* __restrict__ sh, const void* __restrict__ sg,
                                                   const float* __restrict__ kappa, const float* __restrict__ axis,
                                                   int deg, int nsg, int storage, const rg_camera* __restrict__ cams,
                                                   int n_cams, const int* __restrict__ rank,
                                                   const float4* __restrict__ gacc_geo,
                                                   const float4* __restrict__ gacc_rgb, int sh_quirk,
                                                   rg_gradients out) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const int nsh = (deg + 1) * (deg + 1);
    int leaf = rank[g];
    // accumulator layout (12 floats): ddens, dpos.xyz, dscale.xyz, dquat.xyzw, pad
    float4 a0 = gacc_geo[3 * (long long)leaf], a1 = gacc_geo[3 * (long long)leaf + 1],
           a2 = gacc_geo[3 * (long long)leaf + 2];
    float dpos[3] = {a0.y, a0.z, a0.w};
    out.densities[g] = a0.x;
    out.scales[3 * g] = a1.x; out.scales[3 * g + 1] = a1.y; out.scales[3 * g + 2] = a1.z;
    out.quaternions[4 * g] = a1.w; out.quaternions[4 * g + 1] = a2.x;
    out.quaternions[4 * g + 2] = a2.y; out.quaternions[4 * g + 3] = a2.z;

    float coef[3][16];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = 0; k < 16; ++k)
            coef[c][k] = (k < nsh) ? load_param(sh, (g * 3 + c) * nsh + k, storage) : 0.f;
    float dsh[3][16];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = 0; k < 16; ++k) dsh[c][k] = 0.f;
    float px = pos[3 * g], py = pos[3 * g + 1], pz = pos[3 * g + 2];
    for (int v = 0; v < n_cams; ++v) {
        float4 gr4 = gacc_rgb[(long long)leaf * n_cams + v];
        float gr[3] = {gr4.x, gr4.y, gr4.z};
        if (gr[0] == 0.f && gr[1] == 0.f && gr[2] == 0.f) continue;
        float dx = px - cams[v].eye[0], dy = py - cams[v].eye[1], dz = pz - cams[v].eye[2];
        float s2 = dx * dx + dy * dy + dz * dz;
        float inv = 1.f / sqrtf(s2);
        float x = dx * inv, y = dy * inv, z = dz * inv;
        float B[16];
        sh_basis(x, y, z, deg, B);
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int k = 0; k < 16; ++k)
                if (k < nsh) dsh[c][k] += B[k] * gr[c];
        // derivative of each basis function along x, y, z
        float bx[16], by[16], bz[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) { bx[k] = 0.f; by[k] = 0.f; bz[k] = 0.f; }
        if (deg >= 1) { by[1] = -cSH1; bz[2] = cSH1; bx[3] = -cSH1; }
        if (deg >= 2) {
            bx[4] = cSH2[0] * y; by[4] = cSH2[0] * x;
            by[5] = cSH2[1] * z; bz[5] = cSH2[1] * y;
            bx[6] = -2.f * cSH2[2] * x; by[6] = -2.f * cSH2[2] * y; bz[6] = 4.f * cSH2[2] * z;
            bx[7] = cSH2[3] * z; bz[7] = cSH2[3] * x;
            bx[8] = 2.f * cSH2[4] * x; by[8] = -2.f * cSH2[4] * y;
        }
        if (deg >= 3) {
            float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
            bx[9] = 6.f * cSH3[0] * xy;
            // d/dy of y(3x^2-y^2) is 3(x^2-y^2); the reference kernel computes (3x^2-y^2)
            // (utils/sh_utils.cu:270), reproduced when sh_quirk is set.
            by[9] = sh_quirk ? cSH3[0] * (3.f * xx - yy) : 3.f * cSH3[0] * (xx - yy);
            bx[10] = cSH3[1] * yz; by[10] = cSH3[1] * xz; bz[10] = cSH3[1] * xy;
            bx[11] = -2.f * cSH3[2] * xy; by[11] = cSH3[2] * (-3.f * yy + 4.f * zz - xx); bz[11] = 8.f * cSH3[2] * yz;
            bx[12] = -6.f * cSH3[3] * xz; by[12] = -6.f * cSH3[3] * yz;
            bz[12] = 3.f * cSH3[3] * (2.f * zz - xx - yy);
            bx[13] = cSH3[4] * (-3.f * xx + 4.f * zz - yy); by[13] = -2.f * cSH3[4] * xy; bz[13] = 8.f * cSH3[4] * xz;
            bx[14] = 2.f * cSH3[5] * xz; by[14] = -2.f * cSH3[5] * yz; bz[14] = cSH3[5] * (xx - yy);
            bx[15] = 3.f * cSH3[6] * (xx - yy); by[15] = -6.f * cSH3[6] * xy;
        }
        float ddir[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll
            for (int k = 1; k < 16; ++k)
                if (k < nsh) { sx += bx[k] * coef[c][k]; sy += by[k] * coef[c][k]; sz += bz[k] * coef[c][k]; }
            ddir[0] += gr[c] * sx; ddir[1] += gr[c] * sy; ddir[2] += gr[c] * sz;
        }
        // d(v/|v|)/dv applied to dL/ddir
        float inv3 = inv * inv * inv;
        float dv[3] = {dx, dy, dz};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            float acc = 0.f;
#pragma unroll
            for (int b = 0; b < 3; ++b) acc += ((a == b ? s2 : 0.f) - dv[a] * dv[b]) * ddir[b];
            dpos[a] += acc * inv3;
        }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = 0; k < 16; ++k)
            if (k < nsh) out.color_features[(g * 3 + c) * nsh + k] = dsh[c][k];
    out.positions[3 * g] = dpos[0];
    out.positions[3 * g + 1] = dpos[1];
    out.positions[3 * g + 2] = dpos[2];
}

// The spherical-Gaussian part of the colour backward (utils/sh_utils.cu:121-315), one thread per
// Gaussian, lobes outer and views inner: a lobe's amplitude, sharpness and axis gradients stay in
// registers across the views and are written once; its view-direction term is added to the
// position gradient k_color_bwd wrote.
__global__ void __launch_bounds__(128) k_color_bwd_sg(long long n, const float* __restrict__ pos,
                                                      const void* __restrict__ sg, const float* __restrict__ kappa,
                                                      const float* __restrict__ axis, int nsg, int storage,
                                                      const rg_camera* __restrict__ cams, int n_cams,
                                                      const int* __restrict__ rank,
                                                      const float4* __restrict__ gacc_rgb, rg_gradients out) {
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const int leaf = rank[g];
    const float px = pos[3 * g], py = pos[3 * g + 1], pz = pos[3 * g + 2];
    float dpos[3] = {0.f, 0.f, 0.f};
    for (int l = 0; l < nsg; ++l) {
        const long long b = g * nsg + l;
        const float ax = axis[3 * b], ay = axis[3 * b + 1], az = axis[3 * b + 2];
        const float kap = kappa[b];
        float amp[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) amp[c] = load_param(sg, (g * 3 + c) * nsg + l, storage);
        float damp[3] = {0.f, 0.f, 0.f}, dax[3] = {0.f, 0.f, 0.f}, dkap = 0.f;
        for (int v = 0; v < n_cams; ++v) {
            const float4 gr4 = gacc_rgb[(long long)leaf * n_cams + v];
            if (gr4.x == 0.f && gr4.y == 0.f && gr4.z == 0.f) continue;
            const float dx = px - cams[v].eye[0], dy = py - cams[v].eye[1], dz = pz - cams[v].eye[2];
            const float s2 = dx * dx + dy * dy + dz * dz;
            const float inv = 1.f / sqrtf(s2);
            const float x = dx * inv, y = dy * inv, z = dz * inv;
            const float cosm1 = (x * ax + y * ay + z * az) - 1.f;
            const float wgt = expf(cosm1 * kap);
            const float dldw = gr4.x * amp[0] + gr4.y * amp[1] + gr4.z * amp[2];
            damp[0] += gr4.x * wgt; damp[1] += gr4.y * wgt; damp[2] += gr4.z * wgt;
            dax[0] += dldw * kap * x * wgt;
            dax[1] += dldw * kap * y * wgt;
            dax[2] += dldw * kap * z * wgt;
            dkap += dldw * cosm1 * wgt;
            // d(v/|v|)/dv applied to this lobe's dL/ddir
            const float ddir[3] = {dldw * kap * wgt * ax, dldw * kap * wgt * ay, dldw * kap * wgt * az};
            const float inv3 = inv * inv * inv;
            const float dv[3] = {dx, dy, dz};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                float acc = 0.f;
#pragma unroll
                for (int c = 0; c < 3; ++c) acc += ((a == c ? s2 : 0.f) - dv[a] * dv[c]) * ddir[c];
                dpos[a] += acc * inv3;
            }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) out.sph_gauss_features[(g * 3 + c) * nsg + l] = damp[c];
        out.bandwidth_sharpness[b] = dkap;
        out.lobe_axis[3 * b] = dax[0]; out.lobe_axis[3 * b + 1] = dax[1]; out.lobe_axis[3 * b + 2] = dax[2];
    }
    out.positions[3 * g] += dpos[0];
    out.positions[3 * g + 1] += dpos[1];
    out.positions[3 * g + 2] += dpos[2];
}

cudaError_t launch_setup_views(const rg_camera* cams, int n_cams, ViewTable* vt, int* work_counter, cudaStream_t s) {
    k_setup_views<<<1, 32, 0, s>>>(cams, n_cams, vt, work_counter);
    return cudaGetLastError();
}

cudaError_t launch_color_forward(const rg_gaussians* g, const rg_camera* cams, int n_cams, const int* rank,
                                 float4* rgb_leaf, float* rgb_out, cudaStream_t s) {
    long long n = g->n;
    int blocks = (int)((n + 127) / 128);
    k_color_fwd<<<blocks, 128, 0, s>>>(n, g->positions, g->color_features, g->sph_gauss_features,
                                       g->bandwidth_sharpness, g->lobe_axis, g->sh_degree, g->num_sph_gauss,
                                       g->storage, cams, n_cams, rank, rgb_leaf, rgb_out);
    return cudaGetLastError();
}

cudaError_t launch_color_backward(const rg_gaussians* g, const rg_camera* cams, int n_cams, const int* rank,
                                  const float4* gacc_geo, const float4* gacc_rgb, int sh_quirk,
                                  const rg_gradients* out, cudaStream_t s) {
    long long n = g->n;
    int blocks = (int)((n + 127) / 128);
    k_color_bwd<<<blocks, 128, 0, s>>>(n, g->positions, g->color_features, g->sph_gauss_features,
                                       g->bandwidth_sharpness, g->lobe_axis, g->sh_degree, g->num_sph_gauss,
                                       g->storage, cams, n_cams, rank, gacc_geo, gacc_rgb, sh_quirk, *out);
    if (g->num_sph_gauss > 0) {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        k_color_bwd_sg<<<blocks, 128, 0, s>>>(n, g->positions, g->sph_gauss_features, g->bandwidth_sharpness,
                                              g->lobe_axis, g->num_sph_gauss, g->storage, cams, n_cams, rank,
                                              gacc_rgb, *out);
    }
    return cudaGetLastError();
}

}  // namespace rg
