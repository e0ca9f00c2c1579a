/*
 * CPU oracle for the RayGauss differentiable ray caster — TEST INFRASTRUCTURE ONLY.
 *
 * This header is instantiated twice by rg_oracle.c: once with REAL=float (suffix _f32, the
 * literal FP32 restatement used for max-abs parity) and once with REAL=double (suffix _f64,
 * the FP64 oracle used for PSNR and gradient error).  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg may load it; the product path never does.
 *
 * Every function restates one piece of the reference algorithm (paths relative to the
 * reference project):
 *   orc_bbox            optix_raycasting/optix_utils.py:34-66  (quaternion_to_rotation,
 *                       compute_ellipsoids_bbox) and render_optix.py:105-106 (scene box)
 *   orc_forward_sh      utils/sh_utils.cu:25-119   (forward_sh)
 *   orc_backward_sh     utils/sh_utils.cu:121-315  (backward_sh)
 *   orc_render_forward  optix_raycasting/cuda_train/forward/gaussians_aabb.cu:324-402
 *                       (__intersection__gaussian), :405-434 (computeRay), :437-498
 *                       (computeBufferForward), :500-519 (colorBlending), :521-612
 *                       (__raygen__rg), :621-641 (__anyhit__ah cap semantics)
 *   orc_render_backward optix_raycasting/cuda_train/backward/gaussians_aabb.cu:505-775
 *   orc_render_inference optix_raycasting/cuda_test/gaussians_aabb.cu:236-470 (inference
 *                       programs launched by optix_utils.py:302-373)
 * Reference quirks reproduced on request: the sign-dependent root order of the ellipsoid test
 * (camera inside, centre behind: never hit) is always reproduced; the SH degree-3 y-derivative
 * of basis 9 is reproduced when ref_quirks=1.
 * Constants: forward/gaussians_aabb.h:2-5 (BUFFER_SIZE 8, DT 0.0025, TRANSMITTANCE_EPSILON
 * 0.003, SIGMA_THRESHOLD 0.1).  RNG: forward/gaussians_aabb.h:63-94.
 *
 * The traversal (OptiX BVH in the reference) is replaced by a candidate list per ray, prefiltered
 * by a nested uniform grid over the AABBs (orc_grid.h) and equal to that of a scan over all
 * Gaussians: every Gaussian whose exact ellipsoid interval overlaps the ray's scene-box interval, in
 * Gaussian index order or in a given order (e.g. a BVH leaf order, so that FP32 sums of a slab's
 * hits associate the same way as in an engine that visits hits in that order).
 * The per-slab hit decision then uses the reference's exact interval test verbatim, so the set
 * of hits per slab is the reference's set (ordered by Gaussian index; the reference's order is
 * unspecified).  Gradients are accumulated in double in both instantiations.
 */

#include "orc_grid.h"

#define ORC_CAT2(a, b) a##b
#define ORC_CAT(a, b) ORC_CAT2(a, b)
#define ORC_FN(name) ORC_CAT(name, SFX)

typedef struct { REAL x, y, z; } ORC_FN(v3_);
#define V3 ORC_FN(v3_)

static inline V3 ORC_FN(mk)(REAL x, REAL y, REAL z) { V3 r = {x, y, z}; return r; }
static inline V3 ORC_FN(add)(V3 a, V3 b) { return ORC_FN(mk)(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 ORC_FN(sub)(V3 a, V3 b) { return ORC_FN(mk)(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 ORC_FN(scl)(V3 a, REAL s) { return ORC_FN(mk)(a.x * s, a.y * s, a.z * s); }
static inline REAL ORC_FN(dot)(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
/* vector / scalar is multiplication by the reciprocal, as in the reference's float3 helpers */
static inline V3 ORC_FN(divs)(V3 a, REAL s) { REAL inv = (REAL)1 / s; return ORC_FN(scl)(a, inv); }

#define MK ORC_FN(mk)
#define ADD ORC_FN(add)
#define SUB ORC_FN(sub)
#define SCL ORC_FN(scl)
#define DOT ORC_FN(dot)
#define DIVS ORC_FN(divs)

/* correctly rounded exponential: double exp rounded to REAL (for REAL=float this is expf rounded to nearest) */
static inline REAL ORC_FN(r_exp)(REAL x) { return (REAL)exp((double)x); }
static inline REAL ORC_FN(r_log)(REAL x) { return (REAL)log((double)x); }
static inline REAL ORC_FN(r_sqrt)(REAL x) { return (sizeof(REAL) == 4) ? (REAL)sqrtf((float)x) : (REAL)sqrt((double)x); }
#define REXP ORC_FN(r_exp)
#define RLOG ORC_FN(r_log)
#define RSQRT ORC_FN(r_sqrt)

/* Columns of the rotation matrix of a (w,x,y,z) quaternion, not normalised
 * (forward/gaussians_aabb.cu:296-310; same polynomial as optix_utils.py:34-46). */
static void ORC_FN(rot_cols)(const REAL* q, V3* c0, V3* c1, V3* c2) {
    REAL r = q[0], i = q[1], j = q[2], k = q[3];
    *c0 = MK((REAL)1 - (REAL)2 * (j * j + k * k), (REAL)2 * (i * j + r * k), (REAL)2 * (i * k - r * j));
    *c1 = MK((REAL)2 * (i * j - r * k), (REAL)1 - (REAL)2 * (i * i + k * k), (REAL)2 * (j * k + r * i));
    *c2 = MK((REAL)2 * (i * k + r * j), (REAL)2 * (j * k - r * i), (REAL)1 - (REAL)2 * (i * i + j * j));
}

/* Rows M1,M2,M3 of M = (R S^-1)^T given per-axis inverse scales; m = M1*v.x + M2*v.y + M3*v.z. */
static void ORC_FN(conic_rows)(const REAL* q, V3 inv, V3* M1, V3* M2, V3* M3) {
    V3 U, V, W;
    ORC_FN(rot_cols)(q, &U, &V, &W);
    U = SCL(U, inv.x); V = SCL(V, inv.y); W = SCL(W, inv.z);
    *M1 = MK(U.x, V.x, W.x);
    *M2 = MK(U.y, V.y, W.y);
    *M3 = MK(U.z, V.z, W.z);
}

static inline V3 ORC_FN(apply)(V3 M1, V3 M2, V3 M3, V3 v) {
    return ADD(ADD(SCL(M1, v.x), SCL(M2, v.y)), SCL(M3, v.z));
}

/* ------------------------------------------------------------------------------------------ */
/* Ellipsoid AABB at the density threshold + scene box (optix_utils.py:54-66, render_optix.py:105-106) */
void ORC_FN(orc_bbox)(int n, const REAL* pos, const REAL* scl, const REAL* quat, const REAL* dens,
                      REAL* aabb, REAL* scene) {
    REAL lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int g = 0; g < n; ++g) {
        REAL ratio = dens[g] / (REAL)0.1;
        REAL delta = RLOG(ratio * ratio);
        if (delta < 0) delta = 0;
        delta = RSQRT(delta);
        const REAL* q = quat + 4 * g;
        REAL w = q[0], x = q[1], y = q[2], z = q[3];
        REAL L[3][3] = {
            {(REAL)1 - (REAL)2 * (y * y + z * z), (REAL)2 * (x * y - w * z), (REAL)2 * (x * z + w * y)},
            {(REAL)2 * (x * y + w * z), (REAL)1 - (REAL)2 * (x * x + z * z), (REAL)2 * (y * z - w * x)},
            {(REAL)2 * (x * z - w * y), (REAL)2 * (y * z + w * x), (REAL)1 - (REAL)2 * (x * x + y * y)}};
        for (int a = 0; a < 3; ++a) {
            REAL ss = 0;
            for (int c = 0; c < 3; ++c) {
                REAL e = delta * scl[3 * g + c] * L[a][c];
                ss += e * e;
            }
            REAL ext = RSQRT(ss);
            aabb[6 * g + a] = pos[3 * g + a] - ext;
            aabb[6 * g + 3 + a] = pos[3 * g + a] + ext;
            if (aabb[6 * g + a] < lo[a]) lo[a] = aabb[6 * g + a];
            if (aabb[6 * g + 3 + a] > hi[a]) hi[a] = aabb[6 * g + 3 + a];
        }
    }
    for (int a = 0; a < 3; ++a) { scene[a] = lo[a]; scene[3 + a] = hi[a]; }
}

/* ------------------------------------------------------------------------------------------ */
/* SH (degree <= 3) + spherical-Gaussian colour (utils/sh_utils.cu:25-119).  Channel-major
 * coefficient layout (N,3,(deg+1)^2); SG amplitudes (N,3,nsg); sharpness (N,nsg); axes (N,nsg,3). */
#ifndef ORC_SH_CONSTS
#define ORC_SH_CONSTS
static const double ORC_SH_C0 = 0.28209479177387814;
static const double ORC_SH_C1 = 0.4886025119029199;
static const double ORC_SH_C2[5] = {1.0925484305920792, -1.0925484305920792, 0.31539156525252005,
                                    -1.0925484305920792, 0.5462742152960396};
static const double ORC_SH_C3[7] = {-0.5900435899266435, 2.890611442640554, -0.4570457994644658,
                                    0.3731763325901154, -0.4570457994644658, 1.445305721320277,
                                    -0.5900435899266435};
#endif

/* The 16 real SH basis values at direction (x,y,z), in the reference's coefficient order. */
static void ORC_FN(sh_basis)(REAL x, REAL y, REAL z, int deg, REAL* B) {
    B[0] = (REAL)ORC_SH_C0;
    if (deg < 1) return;
    B[1] = -(REAL)ORC_SH_C1 * y;
    B[2] = (REAL)ORC_SH_C1 * z;
    B[3] = -(REAL)ORC_SH_C1 * x;
    if (deg < 2) return;
    REAL xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
    B[4] = (REAL)ORC_SH_C2[0] * xy;
    B[5] = (REAL)ORC_SH_C2[1] * yz;
    B[6] = (REAL)ORC_SH_C2[2] * (REAL)((double)2 * zz - xx - yy);
    B[7] = (REAL)ORC_SH_C2[3] * xz;
    B[8] = (REAL)ORC_SH_C2[4] * (xx - yy);
    if (deg < 3) return;
    B[9] = (REAL)ORC_SH_C3[0] * y * (REAL)(3.0 * xx - yy);
    B[10] = (REAL)ORC_SH_C3[1] * xy * z;
    B[11] = (REAL)ORC_SH_C3[2] * y * (REAL)(4.0 * zz - xx - yy);
    B[12] = (REAL)ORC_SH_C3[3] * z * (REAL)(2.0 * zz - 3.0 * xx - 3.0 * yy);
    B[13] = (REAL)ORC_SH_C3[4] * x * (REAL)(4.0 * zz - xx - yy);
    B[14] = (REAL)ORC_SH_C3[5] * z * (xx - yy);
    B[15] = (REAL)ORC_SH_C3[6] * x * (REAL)(xx - 3.0 * yy);
}

void ORC_FN(orc_forward_sh)(int n, const REAL* campos, const REAL* pos, const REAL* sh, int deg,
                            const REAL* sg, const REAL* kappa, const REAL* axis, int nsg, REAL* rgb) {
    int nsh = (deg + 1) * (deg + 1);
    for (int g = 0; g < n; ++g) {
        V3 dor = MK(pos[3 * g] - campos[0], pos[3 * g + 1] - campos[1], pos[3 * g + 2] - campos[2]);
        V3 dir = DIVS(dor, RSQRT(DOT(dor, dor)));
        REAL res[3] = {0, 0, 0};
        for (int l = 0; l < nsg; ++l) {
            V3 ax = MK(axis[(g * nsg + l) * 3], axis[(g * nsg + l) * 3 + 1], axis[(g * nsg + l) * 3 + 2]);
            REAL wgt = REXP(kappa[g * nsg + l] * (DOT(dir, ax) - (REAL)1));
            for (int c = 0; c < 3; ++c) res[c] += sg[(g * 3 + c) * nsg + l] * wgt;
        }
        REAL B[16];
        ORC_FN(sh_basis)(dir.x, dir.y, dir.z, deg, B);
        for (int c = 0; c < 3; ++c) {
            const REAL* s = sh + (size_t)(g * 3 + c) * nsh;
            for (int k = 0; k < nsh; ++k) res[c] += B[k] * s[k];
            rgb[3 * g + c] = res[c] + (REAL)0.5;
        }
    }
}

/* utils/sh_utils.cu:121-315: dL/dSH, dL/dSG amplitude, dL/dsharpness, dL/daxis and dL/dpos
 * through the view direction.  Gaussians with an all-zero colour gradient get zero outputs. */
void ORC_FN(orc_backward_sh)(int n, const REAL* campos, const REAL* pos, const REAL* sh, int deg,
                             const REAL* sg, const REAL* kappa, const REAL* axis, int nsg,
                             const REAL* drgb, REAL* dsh, REAL* dpos, REAL* dsg, REAL* dkappa, REAL* daxis,
                             int ref_quirks) {
    int nsh = (deg + 1) * (deg + 1);
    for (int g = 0; g < n; ++g) {
        REAL gr[3] = {drgb[3 * g], drgb[3 * g + 1], drgb[3 * g + 2]};
        for (int k = 0; k < 3 * nsh; ++k) dsh[(size_t)g * 3 * nsh + k] = 0;
        for (int k = 0; k < 3 * nsg; ++k) dsg[(size_t)g * 3 * nsg + k] = 0;
        for (int k = 0; k < nsg; ++k) dkappa[(size_t)g * nsg + k] = 0;
        for (int k = 0; k < 3 * nsg; ++k) daxis[(size_t)g * 3 * nsg + k] = 0;
        dpos[3 * g] = dpos[3 * g + 1] = dpos[3 * g + 2] = 0;
        if (gr[0] == 0 && gr[1] == 0 && gr[2] == 0) continue;
        V3 dor = MK(pos[3 * g] - campos[0], pos[3 * g + 1] - campos[1], pos[3 * g + 2] - campos[2]);
        V3 dir = DIVS(dor, RSQRT(DOT(dor, dor)));
        REAL x = dir.x, y = dir.y, z = dir.z;
        REAL B[16];
        ORC_FN(sh_basis)(x, y, z, deg, B);
        for (int c = 0; c < 3; ++c)
            for (int k = 0; k < nsh; ++k) dsh[(size_t)(g * 3 + c) * nsh + k] = B[k] * gr[c];
        /* d(colour)/d(direction), per channel: derivative of each basis function */
        REAL dBx[16] = {0}, dBy[16] = {0}, dBz[16] = {0};
        if (deg >= 1) {
            dBy[1] = -(REAL)ORC_SH_C1; dBz[2] = (REAL)ORC_SH_C1; dBx[3] = -(REAL)ORC_SH_C1;
        }
        if (deg >= 2) {
            dBx[4] = (REAL)ORC_SH_C2[0] * y; dBy[4] = (REAL)ORC_SH_C2[0] * x;
            dBy[5] = (REAL)ORC_SH_C2[1] * z; dBz[5] = (REAL)ORC_SH_C2[1] * y;
            dBx[6] = (REAL)ORC_SH_C2[2] * (REAL)-2 * x; dBy[6] = (REAL)ORC_SH_C2[2] * (REAL)-2 * y;
            dBz[6] = (REAL)ORC_SH_C2[2] * (REAL)4 * z;
            dBx[7] = (REAL)ORC_SH_C2[3] * z; dBz[7] = (REAL)ORC_SH_C2[3] * x;
            dBx[8] = (REAL)ORC_SH_C2[4] * (REAL)2 * x; dBy[8] = (REAL)ORC_SH_C2[4] * (REAL)-2 * y;
        }
        if (deg >= 3) {
            REAL xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
            dBx[9] = (REAL)ORC_SH_C3[0] * (REAL)6 * xy;
            /* d/dy of y(3x^2-y^2) is 3(x^2-y^2); the reference kernel uses (3x^2-y^2)
             * (utils/sh_utils.cu:270).  ref_quirks=1 reproduces it. */
            dBy[9] = ref_quirks ? (REAL)ORC_SH_C3[0] * ((REAL)3 * xx - yy)
                                : (REAL)ORC_SH_C3[0] * (REAL)3 * (xx - yy);
            dBx[10] = (REAL)ORC_SH_C3[1] * yz; dBy[10] = (REAL)ORC_SH_C3[1] * xz; dBz[10] = (REAL)ORC_SH_C3[1] * xy;
            dBx[11] = (REAL)ORC_SH_C3[2] * (REAL)-2 * xy;
            dBy[11] = (REAL)ORC_SH_C3[2] * ((REAL)-3 * yy + (REAL)4 * zz - xx);
            dBz[11] = (REAL)ORC_SH_C3[2] * (REAL)8 * yz;
            dBx[12] = (REAL)ORC_SH_C3[3] * (REAL)-6 * xz;
            dBy[12] = (REAL)ORC_SH_C3[3] * (REAL)-6 * yz;
            dBz[12] = (REAL)ORC_SH_C3[3] * (REAL)3 * ((REAL)2 * zz - xx - yy);
            dBx[13] = (REAL)ORC_SH_C3[4] * ((REAL)-3 * xx + (REAL)4 * zz - yy);
            dBy[13] = (REAL)ORC_SH_C3[4] * (REAL)-2 * xy;
            dBz[13] = (REAL)ORC_SH_C3[4] * (REAL)8 * xz;
            dBx[14] = (REAL)ORC_SH_C3[5] * (REAL)2 * xz;
            dBy[14] = (REAL)ORC_SH_C3[5] * (REAL)-2 * yz;
            dBz[14] = (REAL)ORC_SH_C3[5] * (xx - yy);
            dBx[15] = (REAL)ORC_SH_C3[6] * (REAL)3 * (xx - yy);
            dBy[15] = (REAL)ORC_SH_C3[6] * (REAL)-6 * xy;
        }
        REAL ddir[3] = {0, 0, 0};
        for (int c = 0; c < 3; ++c) {
            const REAL* s = sh + (size_t)(g * 3 + c) * nsh;
            REAL dx = 0, dy = 0, dz = 0;
            for (int k = 1; k < nsh; ++k) { dx += dBx[k] * s[k]; dy += dBy[k] * s[k]; dz += dBz[k] * s[k]; }
            ddir[0] += gr[c] * dx; ddir[1] += gr[c] * dy; ddir[2] += gr[c] * dz;
        }
        for (int l = 0; l < nsg; ++l) {
            V3 ax = MK(axis[(g * nsg + l) * 3], axis[(g * nsg + l) * 3 + 1], axis[(g * nsg + l) * 3 + 2]);
            REAL kap = kappa[g * nsg + l];
            REAL cosm1 = DOT(dir, ax) - (REAL)1;
            REAL wgt = REXP(cosm1 * kap);
            REAL dldw = 0;
            for (int c = 0; c < 3; ++c) {
                dsg[(size_t)(g * 3 + c) * nsg + l] = gr[c] * wgt;
                dldw += gr[c] * sg[(g * 3 + c) * nsg + l];
            }
            daxis[(size_t)(g * nsg + l) * 3 + 0] = dldw * kap * x * wgt;
            daxis[(size_t)(g * nsg + l) * 3 + 1] = dldw * kap * y * wgt;
            daxis[(size_t)(g * nsg + l) * 3 + 2] = dldw * kap * z * wgt;
            dkappa[(size_t)g * nsg + l] = dldw * cosm1 * wgt;
            ddir[0] += dldw * kap * wgt * ax.x;
            ddir[1] += dldw * kap * wgt * ax.y;
            ddir[2] += dldw * kap * wgt * ax.z;
        }
        /* Jacobian of v/|v| applied to dL/ddir */
        REAL s2 = DOT(dor, dor);
        REAL inv32 = (REAL)1 / RSQRT(s2 * s2 * s2);
        REAL v[3] = {dor.x, dor.y, dor.z};
        for (int a = 0; a < 3; ++a) {
            REAL acc = 0;
            for (int b = 0; b < 3; ++b) acc += ((a == b ? s2 : (REAL)0) - v[a] * v[b]) * ddir[b];
            dpos[3 * g + a] = acc * inv32;
        }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Ray generation, scene-box clip and the reference's exact ray/ellipsoid interval test. */

typedef struct {
    const REAL* pos; const REAL* scl; const REAL* quat; const REAL* dens; const REAL* rgb;
    int n;
    const orc_grid* grid;   /* candidate prefilter over the AABBs */
    const int* rank;        /* position of each Gaussian in the candidate order (NULL: index order) */
} ORC_FN(scene_);
#define SCENE ORC_FN(scene_)

typedef struct { int g; REAL r1, r2; } ORC_FN(cand_);
#define CAND ORC_FN(cand_)

typedef struct { REAL r1; int k; } ORC_FN(r1key_);
#define R1KEY ORC_FN(r1key_)

/* Per-thread scratch of the candidate gathering and the slab sweep. */
typedef struct { unsigned char* mark; int* ids; long long* key; R1KEY* by_r1; int* active; CAND* tmp; } ORC_FN(gscratch_);
#define GSCRATCH ORC_FN(gscratch_)


/* tea<4> seeding and LCG draws (forward/gaussians_aabb.h:63-94, a published TEA variant) */
static unsigned ORC_FN(tea4)(unsigned v0, unsigned v1) {
    unsigned s0 = 0;
    for (int n = 0; n < 4; ++n) {
        s0 += 0x9e3779b9u;
        v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + s0) ^ ((v1 >> 5) + 0xc8013ea4u);
        v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + s0) ^ ((v0 >> 5) + 0x7e95761eu);
    }
    return v0;
}
static REAL ORC_FN(rnd)(unsigned* prev) {
    *prev = 1664525u * *prev + 1013904223u;
    return (REAL)((float)(*prev & 0x00FFFFFFu) / (float)0x01000000);
}

/* cam: eye[3], u[3], v[3], w[3], tan_half_fovx, tan_half_fovy  (optix_utils.py:166-177) */
static void ORC_FN(make_ray)(const REAL* cam, int W, int H, unsigned idx, int jitter, unsigned* seed,
                             V3* o, V3* d) {
    REAL ix, iy;
    if (jitter == 1) {
        REAL jx = ORC_FN(rnd)(seed) * (REAL)0.333333f;
        REAL jy = ORC_FN(rnd)(seed) * (REAL)0.333333f;
        ix = ((REAL)(idx % (unsigned)W) + (REAL)0.333333f + jx) / (REAL)W;
        iy = ((REAL)(idx / (unsigned)W) + (REAL)0.333333f + jy) / (REAL)H;
    } else {
        ix = ((REAL)(idx % (unsigned)W) + (REAL)0.5) / (REAL)W;
        iy = ((REAL)(idx / (unsigned)W) + (REAL)0.5) / (REAL)H;
    }
    REAL px = (REAL)2 * ix - (REAL)1, py = (REAL)2 * iy - (REAL)1;
    REAL dx = px * cam[12], dy = py * cam[13];
    V3 U = MK(cam[3], cam[4], cam[5]), Vv = MK(cam[6], cam[7], cam[8]), Wv = MK(cam[9], cam[10], cam[11]);
    V3 dir = ADD(ADD(SCL(U, dx), SCL(Vv, dy)), Wv);
    REAL inv = (REAL)1 / RSQRT(DOT(dir, dir));
    *d = SCL(dir, inv);
    *o = MK(cam[0], cam[1], cam[2]);
}

static REAL ORC_FN(fmn)(REAL a, REAL b) { return (sizeof(REAL) == 4) ? (REAL)fminf((float)a, (float)b) : fmin(a, b); }
static REAL ORC_FN(fmx)(REAL a, REAL b) { return (sizeof(REAL) == 4) ? (REAL)fmaxf((float)a, (float)b) : fmax(a, b); }
#define FMN ORC_FN(fmn)
#define FMX ORC_FN(fmx)

static void ORC_FN(scene_clip)(const REAL* box, V3 o, V3 d, REAL* tenter, REAL* texit) {
    REAL t0x = (box[0] - o.x) / d.x, t0y = (box[1] - o.y) / d.y, t0z = (box[2] - o.z) / d.z;
    REAL t1x = (box[3] - o.x) / d.x, t1y = (box[4] - o.y) / d.y, t1z = (box[5] - o.z) / d.z;
    REAL mnx = FMN(t0x, t1x), mny = FMN(t0y, t1y), mnz = FMN(t0z, t1z);
    REAL mxx = FMX(t0x, t1x), mxy = FMX(t0y, t1y), mxz = FMX(t0z, t1z);
    *tenter = FMX((REAL)0, FMX(mnx, FMX(mny, mnz)));
    *texit = FMN(mxx, FMN(mxy, mxz));
}

/* Exact interval of the ray against the threshold ellipsoid d*exp(-r^2/2) = 0.1
 * (forward/gaussians_aabb.cu:324-402).  Returns 0 when disc <= 1e-7.  For b <= 0 the two roots
 * come back in reversed order, which makes the slab test below fail: the reference never
 * reports such Gaussians (camera inside the ellipsoid with the centre behind it). */
static int ORC_FN(ellipsoid_roots)(const SCENE* S, int g, V3 o, V3 d, REAL* r1, REAL* r2) {
    V3 mu = MK(S->pos[3 * g], S->pos[3 * g + 1], S->pos[3 * g + 2]);
    V3 s = MK(S->scl[3 * g], S->scl[3 * g + 1], S->scl[3 * g + 2]);
    REAL ratio = S->dens[g] / (REAL)0.1;
    s = SCL(s, RSQRT(RLOG(ratio * ratio)));
    V3 inv = MK((REAL)1 / s.x, (REAL)1 / s.y, (REAL)1 / s.z);
    V3 M1, M2, M3;
    ORC_FN(conic_rows)(S->quat + 4 * g, inv, &M1, &M2, &M3);
    V3 O = SUB(o, mu);
    V3 Oe = ORC_FN(apply)(M1, M2, M3, O);
    V3 De = ORC_FN(apply)(M1, M2, M3, d);
    REAL l = (REAL)1 / RSQRT(DOT(De, De));
    V3 Dn = SCL(De, l);
    REAL b = -DOT(Oe, Dn);
    REAL c = DOT(Oe, Oe) - (REAL)1;
    V3 p = ADD(Oe, SCL(Dn, b));
    REAL disc = (REAL)1 - DOT(p, p);
    if (!(disc > (REAL)1e-7f)) return 0;
    REAL sd = RSQRT(disc);
    REAL sb = (b > 0) ? (REAL)1 : (REAL)-1;
    REAL qq = b + sb * sd;
    *r1 = (c / qq) * l;
    *r2 = qq * l;
    return 1;
}

static inline int ORC_FN(slab_hit)(REAL lo, REAL hi, REAL r1, REAL r2) {
    return FMX(lo, r1) <= FMN(hi, r2);
}

/* One candidate: an AABB prefilter with a generous margin (it only skips work), then the exact
 * interval must overlap [tenter, texit]. */
static int ORC_FN(cand_test)(const SCENE* S, const REAL* aabb, int g, V3 o, V3 d, V3 invd, REAL tenter, REAL texit,
                             CAND* out) {
    const REAL* bb = aabb + 6 * g;
    double tn = tenter, tf = texit;
    double oo[3] = {o.x, o.y, o.z}, id[3] = {invd.x, invd.y, invd.z};
    for (int a = 0; a < 3; ++a) {
        double ext = 1e-4 * (fabs((double)bb[a]) + fabs((double)bb[3 + a])) + 1e-6;
        double lo = (double)bb[a] - ext, hi = (double)bb[3 + a] + ext;
        double t0 = (lo - oo[a]) * id[a], t1 = (hi - oo[a]) * id[a];
        if (isnan(t0) || isnan(t1)) continue;
        double a0 = t0 < t1 ? t0 : t1, a1 = t0 < t1 ? t1 : t0;
        if (a0 > tn) tn = a0;
        if (a1 < tf) tf = a1;
        if (tn > tf) return 0;
    }
    REAL r1, r2;
    if (!ORC_FN(ellipsoid_roots)(S, g, o, d, &r1, &r2)) return 0;
    if (!ORC_FN(slab_hit)(tenter, texit, r1, r2)) return 0;
    out->g = g; out->r1 = r1; out->r2 = r2;
    return 1;
}

/* All Gaussians whose exact interval overlaps [tenter, texit], in candidate order (Gaussian index,
 * or the given order).  With a grid, only the Gaussians registered in the cells along the ray are
 * tested, sorted back into candidate order: the list equals that of testing every Gaussian. */
static int ORC_FN(gather_cands)(const SCENE* S, const REAL* aabb, V3 o, V3 d, REAL tenter, REAL texit,
                                const int* order, CAND* out, GSCRATCH* gs) {
    int m = 0;
    V3 invd = MK((REAL)1 / d.x, (REAL)1 / d.y, (REAL)1 / d.z);
    if (S->grid) {
        double oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
        double span = 1e-6 * (fabs((double)tenter) + fabs((double)texit)) + 1e-9;
        int k = orc_grid_query(S->grid, oo, dd, (double)tenter - span, (double)texit + span, gs->mark, gs->ids);
        orc_grid_unmark(gs->mark, gs->ids, k);
        /* test first, then sort the (few) passing candidates into candidate order */
        for (int j = 0; j < k; ++j) m += ORC_FN(cand_test)(S, aabb, gs->ids[j], o, d, invd, tenter, texit, out + m);
        for (int j = 0; j < m; ++j) gs->ids[j] = j;
        for (int j = 0; j < m; ++j)
            gs->key[j] = ((long long)(S->rank ? S->rank[out[j].g] : out[j].g) << 32) | (unsigned)j;
        qsort(gs->key, (size_t)m, sizeof(long long), orc_grid_cmp_ll);
        for (int j = 0; j < m; ++j) gs->tmp[j] = out[(int)(gs->key[j] & 0xffffffffLL)];
        memcpy(out, gs->tmp, sizeof(CAND) * (size_t)m);
        return m;
    }
    for (int li = 0; li < S->n; ++li) {
        int g = order ? order[li] : li;
        m += ORC_FN(cand_test)(S, aabb, g, o, d, invd, tenter, texit, out + m);
    }
    return m;
}

/* Grid over the AABBs (and the rank of each Gaussian in `order`) for one render call. */
typedef struct { orc_grid grid; double* box; int* rank; } ORC_FN(gridset_);
#define GRIDSET ORC_FN(gridset_)

static void ORC_FN(gridset_build)(GRIDSET* G, const REAL* aabb, const REAL* scene_box, int n, const int* order) {
    memset(G, 0, sizeof(*G));
    if (!orc_grid_enabled) return;
    G->box = (double*)malloc(sizeof(double) * 6 * (size_t)(n > 0 ? n : 1));
    for (long long i = 0; i < 6 * (long long)n; ++i) G->box[i] = (double)aabb[i];
    double lo[3] = {scene_box[0], scene_box[1], scene_box[2]}, hi[3] = {scene_box[3], scene_box[4], scene_box[5]};
    for (int a = 0; a < 3; ++a) {
        if (!isfinite(lo[a]) || !isfinite(hi[a]) || !(hi[a] >= lo[a])) { lo[a] = -1.0; hi[a] = 1.0; }
    }
    orc_grid_build(&G->grid, G->box, n, lo, hi);
    G->rank = NULL;
    if (order) {
        G->rank = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
        for (int li = 0; li < n; ++li) G->rank[order[li]] = li;
    }
}

static void ORC_FN(gridset_free)(GRIDSET* G) {
    if (G->box) orc_grid_free(&G->grid);
    free(G->box);
    free(G->rank);
}

static void ORC_FN(gscratch_alloc)(GSCRATCH* gs, int n) {
    size_t m = (size_t)(n > 0 ? n : 1);
    gs->mark = (unsigned char*)calloc(m, 1);
    gs->ids = (int*)malloc(sizeof(int) * m);
    gs->key = (long long*)malloc(sizeof(long long) * m);
    gs->by_r1 = (R1KEY*)malloc(sizeof(R1KEY) * m);
    gs->tmp = (CAND*)malloc(sizeof(CAND) * m);
    gs->active = (int*)malloc(sizeof(int) * m);
}

static void ORC_FN(gscratch_free)(GSCRATCH* gs) {
    free(gs->mark);
    free(gs->ids);
    free(gs->key);
    free(gs->by_r1);
    free(gs->tmp);
    free(gs->active);
}

#define ORC_BUF 8
#define ORC_DT ((REAL)0.0025f)
#define ORC_TEPS ((REAL)0.003f)
#define ORC_STHR ((REAL)0.1f)

typedef struct {
    V3 M1, M2, M3; V3 mu; V3 s; V3 col; REAL dens; const REAL* q;
} ORC_FN(gauss_);
#define GAUSS ORC_FN(gauss_)

static void ORC_FN(load_gauss)(const SCENE* S, int g, GAUSS* G) {
    G->mu = MK(S->pos[3 * g], S->pos[3 * g + 1], S->pos[3 * g + 2]);
    G->s = MK(S->scl[3 * g], S->scl[3 * g + 1], S->scl[3 * g + 2]);
    V3 inv = MK((REAL)1 / G->s.x, (REAL)1 / G->s.y, (REAL)1 / G->s.z);
    G->q = S->quat + 4 * g;
    ORC_FN(conic_rows)(G->q, inv, &G->M1, &G->M2, &G->M3);
    G->col = MK(S->rgb[3 * g], S->rgb[3 * g + 1], S->rgb[3 * g + 2]);
    G->dens = S->dens[g];
}

/* sample time of buffer slot i (rnd_sample 0: grid; 1: random offset; otherwise midpoint) */
static inline REAL ORC_FN(sample_t)(REAL tb, int i, int rnd_sample, unsigned* cs) {
    if (rnd_sample == 0) return tb + (REAL)i * ORC_DT;
    if (rnd_sample == 1) return tb + (REAL)i * ORC_DT + ORC_FN(rnd)(cs) * ORC_DT;
    return tb + (REAL)i * ORC_DT + (REAL)0.5f * ORC_DT;
}

/* Sample buffers of one slab: summed density and density-weighted colour at the 8 samples
 * (forward/gaussians_aabb.cu:437-498; backward :570-627). */
static void ORC_FN(slab_buffers)(const SCENE* S, const int* hits, int nh, REAL tb, V3 o, V3 d,
                                 int rnd_sample, unsigned* seed, REAL* sig, V3* C) {
    for (int i = 0; i < ORC_BUF; ++i) { sig[i] = 0; C[i] = MK(0, 0, 0); }
    unsigned cs = *seed;
    for (int h = 0; h < nh; ++h) {
        GAUSS G;
        ORC_FN(load_gauss)(S, hits[h], &G);
        cs = *seed;
        for (int i = 0; i < ORC_BUF; ++i) {
            REAL t = ORC_FN(sample_t)(tb, i, rnd_sample, &cs);
            V3 x = ADD(o, SCL(d, t));
            V3 xd = SUB(x, G.mu);
            V3 m = ORC_FN(apply)(G.M1, G.M2, G.M3, xd);
            REAL w = REXP((REAL)-0.5f * DOT(m, m));
            if (G.dens * w > ORC_STHR) {
                sig[i] += G.dens * w;
                C[i] = ADD(C[i], SCL(SCL(G.col, w), G.dens));
            }
        }
    }
    if (nh > 0) *seed = cs;
}

/* Per-slab hit list with the reference's cap semantics (forward/gaussians_aabb.cu:621-641):
 * at most max_prim_slice hits are kept; every further hit counts one overflow. */
/* The hits of one slab query [lo, hi] among a ray's candidates, in candidate order, at most `cap`
 * (the any-hit cap, forward/gaussians_aabb.cu:621-641).  The queries of a ray move forward (lo and
 * hi never decrease), so a sweep keeps an active list in candidate order: a candidate enters when
 * r1 <= hi and leaves once r2 < lo, after which the exact test can no longer pass.  The active
 * entries get the exact test, so the result is that of testing every candidate (the scan below,
 * used when the prefilters are switched off). */
typedef struct {
    const CAND* cands; int nc;
    R1KEY* by_r1; int next;          /* candidates by increasing r1 (ties: candidate order) */
    int* active; int n_active;       /* candidate positions, increasing */
    int sweep;
} ORC_FN(sweep_);
#define SWEEP ORC_FN(sweep_)

static int ORC_FN(r1key_cmp)(const void* a, const void* b) {
    const R1KEY* x = (const R1KEY*)a;
    const R1KEY* y = (const R1KEY*)b;
    if (x->r1 < y->r1) return -1;
    if (x->r1 > y->r1) return 1;
    return x->k - y->k;
}

static void ORC_FN(sweep_init)(SWEEP* sw, const CAND* cands, int nc, R1KEY* by_r1, int* active) {
    sw->cands = cands; sw->nc = nc; sw->by_r1 = by_r1; sw->active = active;
    sw->next = 0; sw->n_active = 0;
    sw->sweep = orc_grid_enabled;
    if (!sw->sweep) return;
    for (int k = 0; k < nc; ++k) { by_r1[k].r1 = cands[k].r1; by_r1[k].k = k; }
    qsort(by_r1, (size_t)nc, sizeof(R1KEY), ORC_FN(r1key_cmp));
}

static int ORC_FN(slab_hits)(SWEEP* sw, REAL lo, REAL hi, int cap, int* hits, long long* overflow) {
    const CAND* cands = sw->cands;
    int nh = 0;
    if (!sw->sweep) {
        for (int k = 0; k < sw->nc; ++k) {
            if (!ORC_FN(slab_hit)(lo, hi, cands[k].r1, cands[k].r2)) continue;
            if (nh >= cap) { ++*overflow; break; }
            hits[nh++] = cands[k].g;
        }
        return nh;
    }
    while (sw->next < sw->nc && sw->by_r1[sw->next].r1 <= hi) {
        int k = sw->by_r1[sw->next++].k, j = sw->n_active++;
        while (j > 0 && sw->active[j - 1] > k) { sw->active[j] = sw->active[j - 1]; --j; }
        sw->active[j] = k;
    }
    int keep = 0;
    for (int j = 0; j < sw->n_active; ++j) {
        int k = sw->active[j];
        if (cands[k].r2 < lo) continue;     /* behind the ray's queries from here on */
        sw->active[keep++] = k;
    }
    sw->n_active = keep;
    for (int j = 0; j < sw->n_active; ++j) {
        int k = sw->active[j];
        if (!ORC_FN(slab_hit)(lo, hi, cands[k].r1, cands[k].r2)) continue;
        if (nh >= cap) { ++*overflow; break; }
        hits[nh++] = cands[k].g;
    }
    return nh;
}

/* stats: [0] hit-list overflows, [1] (ray, slab, hit) pairs, [2] slabs visited */
int ORC_FN(orc_render_forward)(int n, const REAL* pos, const REAL* scl, const REAL* quat, const REAL* dens,
                               const REAL* rgb, const REAL* aabb, const REAL* scene_box, const REAL* cam,
                               int W, int H, int white_bg, int max_prim_slice, int jitter, int rnd_sample,
                               unsigned iteration, const int* ray_ids, int n_rays, const int* order, REAL* out,
                               REAL* out_T, long long* stats) {
    GRIDSET GS;
    ORC_FN(gridset_build)(&GS, aabb, scene_box, n, order);
    SCENE S = {pos, scl, quat, dens, rgb, n, GS.box ? &GS.grid : NULL, GS.rank};
    long long st0 = 0, st1 = 0, st2 = 0;
    int cap = max_prim_slice > 0 ? max_prim_slice : 1024;
#pragma omp parallel reduction(+ : st0, st1, st2)
    {
        CAND* cands = (CAND*)malloc(sizeof(CAND) * (size_t)(n > 0 ? n : 1));
        int* hits = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
        GSCRATCH gs;
        ORC_FN(gscratch_alloc)(&gs, n);
#pragma omp for schedule(dynamic, 16)
        for (int rr = 0; rr < n_rays; ++rr) {
            unsigned idx = ray_ids ? (unsigned)ray_ids[rr] : (unsigned)rr;
            unsigned seed = ORC_FN(tea4)(iteration, idx);
            V3 o, d;
            ORC_FN(make_ray)(cam, W, H, idx, jitter, &seed, &o, &d);
            REAL tenter, texit;
            ORC_FN(scene_clip)(scene_box, o, d, &tenter, &texit);
            REAL bg = white_bg ? (REAL)1 : (REAL)0;
            REAL T = 1;
            V3 col = MK(0, 0, 0);
            if (tenter < texit) {
                int nc = ORC_FN(gather_cands)(&S, aabb, o, d, tenter, texit, order, cands, &gs);
                SWEEP sw;
                ORC_FN(sweep_init)(&sw, cands, nc, gs.by_r1, gs.active);
                const REAL slab = ORC_DT * (REAL)ORC_BUF;
                REAL tb = tenter;
                while (tb < texit && T > ORC_TEPS) {
                    REAL lo = FMX(tenter, tb), hi = FMN(texit, tb + slab);
                    if (hi > tenter) {
                        ++st2;
                        int nh = ORC_FN(slab_hits)(&sw, lo, hi, cap, hits, &st0);
                        if (nh > 0) {
                            st1 += nh;
                            REAL sig[ORC_BUF]; V3 C[ORC_BUF];
                            ORC_FN(slab_buffers)(&S, hits, nh, tb, o, d, rnd_sample, &seed, sig, C);
                            for (int i = 0; i < ORC_BUF; ++i) {
                                REAL alpha = (REAL)1 - REXP(-sig[i] * ORC_DT);
                                V3 c = C[i];
                                if (sig[i] > 0) c = DIVS(c, sig[i]);
                                col = ADD(col, SCL(c, T * alpha));
                                T *= (REAL)1 - alpha;
                            }
                        }
                    }
                    tb += slab;
                }
            }
            out[3 * rr + 0] = col.x + T * bg;
            out[3 * rr + 1] = col.y + T * bg;
            out[3 * rr + 2] = col.z + T * bg;
            if (out_T) out_T[rr] = T;
        }
        free(cands);
        free(hits);
        ORC_FN(gscratch_free)(&gs);
    }
    ORC_FN(gridset_free)(&GS);
    if (stats) { stats[0] = st0; stats[1] = st1; stats[2] = st2; }
    return 0;
}

/* Inference render (optix_raycasting/cuda_test/gaussians_aabb.cu:236-470, launched by
 * optix_utils.py:302-373).  Differs from the training forward in three ways:
 *  - the slab query is [tb, tb + 0.02] without the box-exit clip (:408-409);
 *  - the samples of a hit step through the conic space from the slab start: m_0 is the scaled
 *    conic applied to (o + tb d - mu) times sqrt(log(ratio^2)), m_{i+1} = m_i + dt M d (:282-295,
 *    :501-515), weight_density = exp(-|m|^2 / 2) * density and colour * weight_density;
 *  - counts[ray] sums the per-slab hit counts (capped at max_prim_slice like the any-hit, :438;
 *    count_cap > 0 caps the counts alone, for an engine that keeps every hit but counts the same).
 * No jitter and no random sample offsets.  Colours, background and blending as the training
 * forward. */
static void ORC_FN(slab_buffers_inf)(const SCENE* S, const int* hits, int nh, REAL tb, V3 o, V3 d, REAL* sig,
                                     V3* C) {
    for (int i = 0; i < ORC_BUF; ++i) { sig[i] = 0; C[i] = MK(0, 0, 0); }
    for (int h = 0; h < nh; ++h) {
        const int g = hits[h];
        V3 mu = MK(S->pos[3 * g], S->pos[3 * g + 1], S->pos[3 * g + 2]);
        V3 s = MK(S->scl[3 * g], S->scl[3 * g + 1], S->scl[3 * g + 2]);
        REAL dens = S->dens[g];
        REAL ratio = dens / (REAL)0.1;
        REAL kf = RSQRT(RLOG(ratio * ratio));
        s = SCL(s, kf);
        V3 inv = MK((REAL)1 / s.x, (REAL)1 / s.y, (REAL)1 / s.z);
        V3 M1, M2, M3;
        ORC_FN(conic_rows)(S->quat + 4 * g, inv, &M1, &M2, &M3);
        V3 hit = ADD(o, SCL(d, tb));
        V3 m = SCL(ORC_FN(apply)(M1, M2, M3, SUB(hit, mu)), kf);
        V3 mdt = SCL(SCL(ORC_FN(apply)(M1, M2, M3, d), kf), ORC_DT);
        V3 col = MK(S->rgb[3 * g], S->rgb[3 * g + 1], S->rgb[3 * g + 2]);
        for (int i = 0; i < ORC_BUF; ++i) {
            REAL wd = REXP((REAL)-0.5f * DOT(m, m)) * dens;
            if (wd > ORC_STHR) {
                sig[i] += wd;
                C[i] = ADD(C[i], SCL(col, wd));
            }
            m = ADD(m, mdt);
        }
    }
}

int ORC_FN(orc_render_inference)(int n, const REAL* pos, const REAL* scl, const REAL* quat, const REAL* dens,
                                 const REAL* rgb, const REAL* aabb, const REAL* scene_box, const REAL* cam,
                                 int W, int H, int white_bg, int max_prim_slice, int count_cap, const int* ray_ids,
                                 int n_rays, const int* order, REAL* out, int* counts, long long* stats) {
    GRIDSET GS;
    ORC_FN(gridset_build)(&GS, aabb, scene_box, n, order);
    SCENE S = {pos, scl, quat, dens, rgb, n, GS.box ? &GS.grid : NULL, GS.rank};
    long long st0 = 0, st1 = 0;
    int cap = max_prim_slice > 0 ? max_prim_slice : 1024;
    int ccap = count_cap > 0 ? count_cap : cap;   /* per-slab cap of the counts alone (0: the hit cap) */
#pragma omp parallel reduction(+ : st0, st1)
    {
        CAND* cands = (CAND*)malloc(sizeof(CAND) * (size_t)(n > 0 ? n : 1));
        int* hits = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
        GSCRATCH gs;
        ORC_FN(gscratch_alloc)(&gs, n);
#pragma omp for schedule(dynamic, 16)
        for (int rr = 0; rr < n_rays; ++rr) {
            unsigned idx = ray_ids ? (unsigned)ray_ids[rr] : (unsigned)rr;
            unsigned seed = 0;
            V3 o, d;
            ORC_FN(make_ray)(cam, W, H, idx, 0, &seed, &o, &d);
            REAL tenter, texit;
            ORC_FN(scene_clip)(scene_box, o, d, &tenter, &texit);
            REAL bg = white_bg ? (REAL)1 : (REAL)0;
            REAL T = 1;
            V3 col = MK(0, 0, 0);
            int cnt = 0;
            if (tenter < texit) {
                const REAL slab = ORC_DT * (REAL)ORC_BUF;
                /* candidates over the whole marched range: the last slab reaches past texit */
                int nc = ORC_FN(gather_cands)(&S, aabb, o, d, tenter, texit + slab, order, cands, &gs);
                SWEEP sw;
                ORC_FN(sweep_init)(&sw, cands, nc, gs.by_r1, gs.active);
                REAL tb = tenter;
                while (tb < texit && T > ORC_TEPS) {
                    REAL lo = tb, hi = tb + slab;
                    if (hi > tenter) {
                        int nh = ORC_FN(slab_hits)(&sw, lo, hi, cap, hits, &st0);
                        if (nh > 0) {
                            st1 += nh;
                            cnt += nh < ccap ? nh : ccap;
                            REAL sig[ORC_BUF]; V3 C[ORC_BUF];
                            ORC_FN(slab_buffers_inf)(&S, hits, nh, tb, o, d, sig, C);
                            for (int i = 0; i < ORC_BUF; ++i) {
                                REAL alpha = (REAL)1 - REXP(-sig[i] * ORC_DT);
                                V3 c = C[i];
                                if (sig[i] > 0) c = DIVS(c, sig[i]);
                                col = ADD(col, SCL(c, T * alpha));
                                T *= (REAL)1 - alpha;
                            }
                        }
                    }
                    tb += slab;
                }
            }
            out[3 * rr + 0] = col.x + T * bg;
            out[3 * rr + 1] = col.y + T * bg;
            out[3 * rr + 2] = col.z + T * bg;
            if (counts) counts[rr] = cnt;
        }
        free(cands);
        free(hits);
        ORC_FN(gscratch_free)(&gs);
    }
    ORC_FN(gridset_free)(&GS);
    if (stats) { stats[0] = st0; stats[1] = st1; }
    return 0;
}

/* Hand adjoint (backward/gaussians_aabb.cu:505-775).  grads (double, accumulated): drgb (n,3),
 * ddens (n), dpos (n,3), dscl (n,3), dquat (n,4).  The quaternion gradient is the derivative of
 * the polynomial rotation with respect to the quaternion as passed (not normalised). */
int ORC_FN(orc_render_backward)(int n, const REAL* pos, const REAL* scl, const REAL* quat, const REAL* dens,
                                const REAL* rgb, const REAL* aabb, const REAL* scene_box, const REAL* cam,
                                int W, int H, int max_prim_slice, int jitter, int rnd_sample,
                                unsigned iteration, const int* ray_ids, int n_rays, const int* order,
                                const REAL* ray_colors, const REAL* dL,
                                double* drgb, double* ddens, double* dpos, double* dscl, double* dquat,
                                long long* stats) {
    GRIDSET GS;
    ORC_FN(gridset_build)(&GS, aabb, scene_box, n, order);
    SCENE S = {pos, scl, quat, dens, rgb, n, GS.box ? &GS.grid : NULL, GS.rank};
    long long st0 = 0, st1 = 0;
    int cap = max_prim_slice > 0 ? max_prim_slice : 1024;
#pragma omp parallel reduction(+ : st0, st1)
    {
        CAND* cands = (CAND*)malloc(sizeof(CAND) * (size_t)(n > 0 ? n : 1));
        int* hits = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
        GSCRATCH gs;
        ORC_FN(gscratch_alloc)(&gs, n);
#pragma omp for schedule(dynamic, 16)
        for (int rr = 0; rr < n_rays; ++rr) {
            unsigned idx = ray_ids ? (unsigned)ray_ids[rr] : (unsigned)rr;
            unsigned seed = ORC_FN(tea4)(iteration, idx);
            V3 o, d;
            ORC_FN(make_ray)(cam, W, H, idx, jitter, &seed, &o, &d);
            REAL tenter, texit;
            ORC_FN(scene_clip)(scene_box, o, d, &tenter, &texit);
            if (!(tenter < texit)) continue;
            int nc = ORC_FN(gather_cands)(&S, aabb, o, d, tenter, texit, order, cands, &gs);
            SWEEP sw;
            ORC_FN(sweep_init)(&sw, cands, nc, gs.by_r1, gs.active);
            const REAL slab = ORC_DT * (REAL)ORC_BUF;
            REAL tb = tenter;
            REAL Tb = 1;
            V3 Rb = MK(ray_colors[3 * rr], ray_colors[3 * rr + 1], ray_colors[3 * rr + 2]);
            V3 gr = MK(dL[3 * rr], dL[3 * rr + 1], dL[3 * rr + 2]);
            while (tb < texit && Tb > ORC_TEPS) {
                REAL lo = FMX(tenter, tb), hi = FMN(texit, tb + slab);
                if (hi > tenter) {
                    int nh = ORC_FN(slab_hits)(&sw, lo, hi, cap, hits, &st0);
                    if (nh == 0) { tb += slab; continue; }
                    st1 += nh;
                    REAL sig[ORC_BUF]; V3 C[ORC_BUF];
                    unsigned seed_b = seed;
                    ORC_FN(slab_buffers)(&S, hits, nh, tb, o, d, rnd_sample, &seed_b, sig, C);
                    unsigned cs = seed;
                    REAL Tn = Tb; V3 Rn = Rb;
                    for (int h = 0; h < nh; ++h) {
                        int g = hits[h];
                        GAUSS G;
                        ORC_FN(load_gauss)(&S, g, &G);
                        cs = seed;
                        REAL Ta = Tb; V3 Ra = Rb;
                        REAL gcol = 0;
                        V3 dcds = MK(0, 0, 0), dsc = MK(0, 0, 0), dp = MK(0, 0, 0);
                        V3 dr1 = MK(0, 0, 0), dr2 = MK(0, 0, 0), dr3 = MK(0, 0, 0);
                        for (int i = 0; i < ORC_BUF; ++i) {
                            REAL cd = sig[i];
                            V3 cc = C[i];
                            if (cd > 0) cc = DIVS(cc, cd);
                            REAL alpha = (REAL)1 - REXP(-cd * ORC_DT);
                            REAL t = ORC_FN(sample_t)(tb, i, rnd_sample, &cs);
                            V3 x = ADD(o, SCL(d, t));
                            V3 xd = SUB(x, G.mu);
                            V3 m = ORC_FN(apply)(G.M1, G.M2, G.M3, xd);
                            REAL w = REXP((REAL)-0.5f * DOT(m, m));
                            if (G.dens * w > ORC_STHR) {
                                REAL wn = w * G.dens;
                                if (cd > 0) wn /= cd;
                                gcol += wn * alpha * Ta;
                                V3 aux = SCL(SUB(SCL(cc, Ta), Ra), ORC_DT);
                                dcds = ADD(dcds, SCL(aux, w));
                                V3 dcdw = SCL(aux, G.dens);
                                if (cd > 0) {
                                    V3 dc = DIVS(SUB(G.col, cc), cd);
                                    dcdw = ADD(dcdw, SCL(SCL(dc, Ta * alpha), G.dens));
                                    dcds = ADD(dcds, SCL(SCL(dc, Ta * alpha), w));
                                }
                                REAL dldw = DOT(gr, dcdw);
                                REAL u = dldw * w;
                                dsc.x += u * (m.x * m.x) / G.s.x;
                                dsc.y += u * (m.y * m.y) / G.s.y;
                                dsc.z += u * (m.z * m.z) / G.s.z;
                                dp.x += u * DOT(G.M1, m);
                                dp.y += u * DOT(G.M2, m);
                                dp.z += u * DOT(G.M3, m);
                                dr1 = SUB(dr1, SCL(SCL(xd, u), m.x / G.s.x));
                                dr2 = SUB(dr2, SCL(SCL(xd, u), m.y / G.s.y));
                                dr3 = SUB(dr3, SCL(SCL(xd, u), m.z / G.s.z));
                            }
                            Ra = SUB(Ra, SCL(cc, Ta * alpha));
                            Ta *= (REAL)1 - alpha;
                        }
                        /* dL/dq from dL/d(columns of R): d col_j / d q as in the polynomial rotation */
                        const REAL* q = G.q;
                        REAL r = q[0], qi = q[1], qj = q[2], qk = q[3];
                        double gq[4];
                        gq[0] = 2.0 * (double)(qk * dr1.y - qj * dr1.z - qk * dr2.x + qi * dr2.z + qj * dr3.x - qi * dr3.y);
                        gq[1] = 2.0 * (double)(qj * dr1.y + qk * dr1.z + qj * dr2.x - (REAL)2 * qi * dr2.y + r * dr2.z
                                               + qk * dr3.x - r * dr3.y - (REAL)2 * qi * dr3.z);
                        gq[2] = 2.0 * (double)(-(REAL)2 * qj * dr1.x + qi * dr1.y - r * dr1.z + qi * dr2.x + qk * dr2.z
                                               + r * dr3.x + qk * dr3.y - (REAL)2 * qj * dr3.z);
                        gq[3] = 2.0 * (double)(-(REAL)2 * qk * dr1.x + r * dr1.y + qi * dr1.z - r * dr2.x
                                               - (REAL)2 * qk * dr2.y + qj * dr2.z + qi * dr3.x + qj * dr3.y);
#pragma omp atomic
                        drgb[3 * g + 0] += (double)(gr.x * gcol);
#pragma omp atomic
                        drgb[3 * g + 1] += (double)(gr.y * gcol);
#pragma omp atomic
                        drgb[3 * g + 2] += (double)(gr.z * gcol);
#pragma omp atomic
                        ddens[g] += (double)(gr.x * dcds.x + gr.y * dcds.y + gr.z * dcds.z);
#pragma omp atomic
                        dscl[3 * g + 0] += (double)dsc.x;
#pragma omp atomic
                        dscl[3 * g + 1] += (double)dsc.y;
#pragma omp atomic
                        dscl[3 * g + 2] += (double)dsc.z;
#pragma omp atomic
                        dpos[3 * g + 0] += (double)dp.x;
#pragma omp atomic
                        dpos[3 * g + 1] += (double)dp.y;
#pragma omp atomic
                        dpos[3 * g + 2] += (double)dp.z;
                        for (int a = 0; a < 4; ++a) {
#pragma omp atomic
                            dquat[4 * g + a] += gq[a];
                        }
                        if (h == nh - 1) { Tn = Ta; Rn = Ra; }
                    }
                    Tb = Tn; Rb = Rn; seed = cs;
                }
                tb += slab;
            }
        }
        free(cands);
        free(hits);
        ORC_FN(gscratch_free)(&gs);
    }
    ORC_FN(gridset_free)(&GS);
    if (stats) { stats[0] = st0; stats[1] = st1; }
    return 0;
}

#undef V3
#undef MK
#undef ADD
#undef SUB
#undef SCL
#undef DOT
#undef DIVS
#undef REXP
#undef RLOG
#undef RSQRT
#undef FMN
#undef FMX
#undef SCENE
#undef CAND
#undef GSCRATCH
#undef GRIDSET
#undef SWEEP
#undef R1KEY
#undef GAUSS
#undef ORC_BUF
#undef ORC_DT
#undef ORC_TEPS
#undef ORC_STHR
