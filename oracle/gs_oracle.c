/* CPU oracle for the gamesplat per-frame splatting path (test infrastructure).
 *
 * Restates, in reference operand order, shaders/cull.glsl, shaders/sort.glsl,
 * shaders/splat.glsl (+ the GL blend state of src/renderer.cpp:266-320),
 * shaders/gps.glsl and shaders/accum.glsl.  See gs_oracle.h for the parity
 * status.  Build with -ffp-contract=off (oracle/Makefile): every expression
 * below is evaluated one IEEE single-precision operation at a time.
 */
#include "gs_oracle.h"
#include <math.h>
#include <string.h>
#include <stdlib.h>

static inline float fbits(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline uint32_t ubits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

/* GLSL built-ins with their specified definitions (GLSL 4.50 §8.3). */
static inline float g_min(float x, float y) { return (y < x) ? y : x; }
static inline float g_max(float x, float y) { return (x < y) ? y : x; }
static inline float g_clamp(float x, float lo, float hi) { return g_min(g_max(x, lo), hi); }
static inline float g_mix(float x, float y, float a) { return x * (1.0f - a) + y * a; }
static inline float g_fract(float x) { return x - floorf(x); }
/* float -> uint conversion that saturates like the GPU's cvt.rzi.u32.f32. */
static inline uint32_t g_f2u_sat(float x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)x;
}

/* ------------------------------------------------------------------------ */
/* Deterministic transcendental functions.                                   */
/*                                                                           */
/* log: x = m * 2^e with m in [sqrt(1/2), sqrt(2)];                          */
/*      ln m = 2 atanh(s), s = (m-1)/(m+1), atanh by its Taylor series      */
/*      s + s^3/3 + s^5/5 + s^7/7 + s^9/9 (|s| <= 0.172, truncation < 1e-9); */
/*      ln 2 split in a 15-bit head (e * head exact) and a tail.            */
/* exp: Cody-Waite reduction x = n ln2 + r, |r| <= 0.35, e^r by its Taylor   */
/*      series to degree 7, then scaling by 2^n through the exponent field. */
/* sin/cos: reduction by pi/2 (17-bit head + tail), Taylor series to        */
/*      degree 9 (sin) and 10 (cos) on |r| <= pi/4, quadrant selection.     */
/* Only +,-,*,/ and exact bit manipulation are used, so a CUDA device       */
/* function doing the same operations in the same order (with _rn          */
/* intrinsics) returns identical bits.                                      */
/* ------------------------------------------------------------------------ */
#define OC_LN2_HI   0.693145751953125f      /* 22713 / 32768 */
#define OC_LN2_LO   1.428606765330187e-06f   /* ln 2 - OC_LN2_HI */
#define OC_INV_LN2  1.4426950216293335f
#define OC_PIO2_HI  1.5707855224609375f      /* floor(pi/2 * 2^16) / 2^16 */
#define OC_PIO2_LO  1.0804334124259185e-05f  /* pi/2 - OC_PIO2_HI */
#define OC_2_OVER_PI 0.6366197466850281f

float oc_logf(float x) {
    if (x != x) return x;
    if (x < 0.0f) return NAN;
    if (x == 0.0f) return -INFINITY;
    if (x == INFINITY) return x;
    uint32_t ix = ubits(x);
    int e = 0;
    if (ix < 0x00800000u) { x = x * 16777216.0f; ix = ubits(x); e = -24; }
    e += (int)(ix >> 23) - 127;
    float m = fbits((ix & 0x007fffffu) | 0x3f800000u);
    if (m > 1.41421354f) { m = m * 0.5f; e += 1; }
    float f = m - 1.0f;
    float s = f / (m + 1.0f);
    float z = s * s;
    float p = ((((z * 0.1111111119389534f) + 0.1428571492433548f) * z + 0.20000000298023224f) * z
               + 0.3333333432674408f) * z;
    float two_s = s + s;
    float lm = two_s + two_s * p;
    float ef = (float)e;
    return ef * OC_LN2_HI + (lm + ef * OC_LN2_LO);
}

float oc_expf(float x) {
    if (x != x) return x;
    if (x > 88.72283f) return INFINITY;
    if (x < -103.97208f) return 0.0f;
    float n = rintf(x * OC_INV_LN2);
    float r = (x - n * OC_LN2_HI) - n * OC_LN2_LO;
    float p = 1.0f + r * (1.0f + r * (0.5f + r * (0.1666666716337204f + r * (0.0416666679084301f
              + r * (0.008333333767950535f + r * (0.0013888889225199819f
              + r * 0.00019841270113829523f))))));
    int k = (int)n;
    if (k > 127) { p = p * 2.0f; k -= 1; }
    if (k < -126) { p = p * 5.421010862427522e-20f; k += 64; }
    return p * fbits((uint32_t)(k + 127) << 23);
}

void oc_sincosf(float x, float* s_out, float* c_out) {
    float n = rintf(x * OC_2_OVER_PI);
    float r = (x - n * OC_PIO2_HI) - n * OC_PIO2_LO;
    float z = r * r;
    float sr = r + (r * z) * (-0.1666666716337204f + z * (0.008333333767950535f
               + z * (-0.00019841270113829523f + z * 2.7557318844628753e-06f)));
    float cr = 1.0f + z * (-0.5f + z * (0.0416666679084301f + z * (-0.0013888889225199819f
               + z * (2.4801587642286904e-05f + z * -2.755731998149713e-07f))));
    int q = ((int)n) & 3;
    switch (q) {
        case 0: *s_out = sr;  *c_out = cr;  break;
        case 1: *s_out = cr;  *c_out = -sr; break;
        case 2: *s_out = -sr; *c_out = -cr; break;
        default: *s_out = -cr; *c_out = sr; break;
    }
}

/* shaders/cull.glsl:116-123 (also shaders/gps.glsl:102-109). */
float oc_dilog(float x) {
    float s = 1.0f - x;
    float y = (((((((-1.068681974f * x + 3.334685126f) * x - 4.173996483f) * x +
                   2.567860600f) * x - 0.884150470f) * x - 0.123550674f) * x +
                   1.992765336f) * x + 6.74195669e-05f);
    y += (s > 0.0f) ? (s * oc_logf(s)) : 0.0f;
    return y;
}

/* shaders/gps.glsl:225-230. */
float oc_inv_dilog(float x) {
    return ((((((((((-0.322192871f * x + 2.562830719f) * x - 8.669815892f) * x +
                   16.243561492f) * x - 18.394710417f) * x + 12.891925084f) * x -
                   5.501796628f) * x + 1.361194673f) * x - 0.417517201f) * x +
                   1.008071981f) * x - 6.39879974e-05f);
}

/* ------------------------------------------------------------------------ */
/* Cull / project / SH (shaders/cull.glsl:166-424).                          */
/* ------------------------------------------------------------------------ */
#define SH_C0   0.28209479177387814f
#define SH_C1   0.4886025119029199f
#define SH_C2_0 1.0925484305920792f
#define SH_C2_1 (-1.0925484305920792f)
#define SH_C2_2 0.31539156525252005f
#define SH_C2_3 (-1.0925484305920792f)
#define SH_C2_4 0.5462742152960396f
#define SH_C3_0 (-0.5900435899266435f)
#define SH_C3_1 2.890611442640554f
#define SH_C3_2 (-0.4570457994644658f)
#define SH_C3_3 0.3731763325901154f
#define SH_C3_4 (-0.4570457994644658f)
#define SH_C3_5 1.445305721320277f
#define SH_C3_6 (-0.5900435899266435f)

static inline void sh_add(float* res, float w, const float* sh) {
    res[0] = res[0] + w * sh[0];
    res[1] = res[1] + w * sh[1];
    res[2] = res[2] + w * sh[2];
}

/* gsanim int8 appearance deltas (shaders/cull.glsl:125-164): state 0 is the
 * base row; state s >= 1 adds q * scale[j] with q the int8 at
 * ((s-1) * N + row) * 48 + j, j = 0..2 for the DC slots 12..14 and
 * 3 + channel*15 + k for the SH slot 16 + 3k + channel. */
typedef struct oc_anim {
    const int8_t* deltas;
    uint32_t count;           /* rows per state (N) */
    const float* scales;      /* 48 */
    int state_a, state_b;
    float weight;
} oc_anim;

static inline float anim_coeff(const oc_anim* a, float base, uint32_t row, int j, int state) {
    if (state == 0) return base;
    uint64_t off = ((uint64_t)(state - 1) * a->count + row) * 48u + (uint64_t)j;
    int q = (int)a->deltas[off];
    return base + (float)q * a->scales[j];
}

static void anim_row(const oc_anim* a, uint32_t row, const float* in, float* out) {
    memcpy(out, in, 64 * sizeof(float));
    for (int slot = 12; slot < 61; ++slot) {
        if (slot == 15) continue;
        int j = slot < 15 ? slot - 12 : 3 + ((slot - 16) % 3) * 15 + (slot - 16) / 3;
        float v = anim_coeff(a, in[slot], row, j, a->state_a);
        if (a->weight > 0.0f) {
            float b = anim_coeff(a, in[slot], row, j, a->state_b);
            v = (1.0f - a->weight) * v + a->weight * b;
        }
        out[slot] = v;
    }
}

/* gsanim 0.3 appearance layers (shaders/cull.glsl:141-148, 354-416): layer
 * l's 48 half coefficients of a row replace its DC and SH slots; each layer's
 * colour is evaluated without the +0.5 bias, clamped at 0, weighted per
 * channel and summed. */
typedef struct oc_layers {
    const uint16_t* halves;  /* [(l * n + row) * 48 + j], j = DC 0..2, then 3 + c*15 + k */
    uint32_t n;
    int count;
    const float* weights;    /* [l * 3 + c] */
} oc_layers;

static void layer_row(const oc_layers* L, int l, uint32_t row, const float* in, float* out) {
    for (int k = 0; k < 64; ++k) out[k] = in[k];
    const uint16_t* h = L->halves + ((size_t)l * L->n + row) * 48u;
    for (int j = 0; j < 3; ++j) out[12 + j] = oc_half_to_float(h[j]);
    for (int slot = 16; slot < 61; ++slot)
        out[slot] = oc_half_to_float(h[3 + ((slot - 16) % 3) * 15 + (slot - 16) / 3]);
}

/* SH colour before the bias (shaders/cull.glsl:355-408): DC at r[12..14],
 * SH(k) at r[16 + 3k .. 18 + 3k]. */
static void sh_eval(const float* r, float x, float y, float z, int eff_degree, float* res) {
    res[0] = SH_C0 * r[12];
    res[1] = SH_C0 * r[13];
    res[2] = SH_C0 * r[14];
    const float* sh = r + 16;  /* SH(k) = sh + 3k */
    if (eff_degree >= 1) {
        sh_add(res, -SH_C1 * y, sh + 0);
        sh_add(res, SH_C1 * z, sh + 3);
        sh_add(res, -SH_C1 * x, sh + 6);
        if (eff_degree >= 2) {
            float xx = x * x, yy = y * y, zz = z * z;
            float xy = x * y, yz = y * z, xz = z * x;
            sh_add(res, SH_C2_0 * xy, sh + 9);
            sh_add(res, SH_C2_1 * yz, sh + 12);
            sh_add(res, SH_C2_2 * ((2.0f * zz - xx) - yy), sh + 15);
            sh_add(res, SH_C2_3 * xz, sh + 18);
            sh_add(res, SH_C2_4 * (xx - yy), sh + 21);
            if (eff_degree >= 3) {
                sh_add(res, (SH_C3_0 * y) * (3.0f * xx - yy), sh + 24);
                sh_add(res, (SH_C3_1 * xy) * z, sh + 27);
                sh_add(res, (SH_C3_2 * y) * ((4.0f * zz - xx) - yy), sh + 30);
                sh_add(res, (SH_C3_3 * z) * ((2.0f * zz - 3.0f * xx) - 3.0f * yy), sh + 33);
                sh_add(res, (SH_C3_4 * x) * ((4.0f * zz - xx) - yy), sh + 36);
                sh_add(res, (SH_C3_5 * z) * (xx - yy), sh + 39);
                sh_add(res, (SH_C3_6 * x) * (xx - 3.0f * yy), sh + 42);
            }
        }
    }
}

static void cull_one(const float* r, uint32_t idx, const oc_camera* cam, int sh_degree,
                     float sh_lod_distance, int collect_stats, const oc_layers* layers, uint32_t* ids,
                     uint32_t* keys, float* out, uint32_t* visible_count, uint32_t* diag) {
    const float* V = cam->view;
    const float* P = cam->proj;
    float px = r[0], py = r[1], pz = r[2], opacity = r[3];
    float sx = r[4], sy = r[5], sz = r[6];
    float qw = r[8], qx = r[9], qy = r[10], qz = r[11];

    /* p_view = view * vec4(position, 1.0)  (:209-210) */
    float vx = ((V[0] * px + V[4] * py) + V[8] * pz) + V[12];
    float vy = ((V[1] * px + V[5] * py) + V[9] * pz) + V[13];
    float vz = ((V[2] * px + V[6] * py) + V[10] * pz) + V[14];

    float t = cam->orthographic;
    int visible = vz <= -0.2f;                                   /* :212 */
    if (visible) {
        float inv_z = -1.0f / vz;
        float ndc_x = ((P[0] * vx) * inv_z) * (1.0f - t) + (P[0] * vx) * t;
        float ndc_y = ((P[5] * vy) * inv_z) * (1.0f - t) + (P[5] * vy) * t;
        visible = fabsf(ndc_x) <= 1.3f && fabsf(ndc_y) <= 1.3f;  /* :219 */
    }
    if (!visible) {                                              /* :222-228 */
        out[0] = out[1] = out[2] = out[3] = 0.0f;
        out[4] = out[5] = out[6] = out[7] = 0.0f;
        out[8] = 1.0f; out[9] = 0.0f; out[10] = 1.0f; out[11] = 1.0f;
        out[12] = out[13] = out[14] = out[15] = 0.0f;
        return;
    }
    (*visible_count)++;                                          /* :230-232 */
    ids[idx] = idx;
    keys[idx] = 0xFFFFFFFFu - ubits(g_max(-vz, 0.0f));

    /* R (column-major mat3 constructor, :235-247); M = R * S; cov = M M^T */
    float R[3][3];
    R[0][0] = 1.0f - 2.0f * (qy * qy + qz * qz);
    R[0][1] = 2.0f * (qx * qy + qw * qz);
    R[0][2] = 2.0f * (qx * qz - qw * qy);
    R[1][0] = 2.0f * (qx * qy - qw * qz);
    R[1][1] = 1.0f - 2.0f * (qx * qx + qz * qz);
    R[1][2] = 2.0f * (qy * qz + qw * qx);
    R[2][0] = 2.0f * (qx * qz + qw * qy);
    R[2][1] = 2.0f * (qy * qz - qw * qx);
    R[2][2] = 1.0f - 2.0f * (qx * qx + qy * qy);
    float s3[3] = {sx, sy, sz};
    float M[3][3];
    for (int c = 0; c < 3; ++c)
        for (int rr = 0; rr < 3; ++rr) M[c][rr] = R[c][rr] * s3[c];
    float cov[3][3];
    for (int c = 0; c < 3; ++c)
        for (int rr = 0; rr < 3; ++rr)
            cov[c][rr] = (M[0][rr] * M[0][c] + M[1][rr] * M[1][c]) + M[2][rr] * M[2][c];

    float fx_p = cam->persp_focal, fy_p = cam->persp_focal;
    float fx_o = cam->ortho_focal, fy_o = cam->ortho_focal;
    float J00 = g_mix(fx_p / vz, -fx_o, t);                      /* :261-264 */
    float J11 = g_mix(fy_p / vz, -fy_o, t);
    float J02 = g_mix((-fx_p * vx) / (vz * vz), 0.0f, t);
    float J12 = g_mix((-fy_p * vy) / (vz * vz), 0.0f, t);

    /* W cov W^T evaluated as (W * cov) * transpose(W) (:266-267) */
    float W[3][3];
    for (int c = 0; c < 3; ++c)
        for (int rr = 0; rr < 3; ++rr) W[c][rr] = V[c * 4 + rr];
    float A[3][3], B[3][3];
    for (int c = 0; c < 3; ++c)
        for (int rr = 0; rr < 3; ++rr)
            A[c][rr] = (W[0][rr] * cov[c][0] + W[1][rr] * cov[c][1]) + W[2][rr] * cov[c][2];
    for (int c = 0; c < 3; ++c)
        for (int rr = 0; rr < 3; ++rr)
            B[c][rr] = (A[0][rr] * W[0][c] + A[1][rr] * W[1][c]) + A[2][rr] * W[2][c];

    float a = ((J00 * J00) * B[0][0] + ((2.0f * J00) * J02) * B[0][2]) + (J02 * J02) * B[2][2];
    float b = (((J00 * J11) * B[0][1] + (J00 * J12) * B[0][2]) + (J02 * J11) * B[1][2])
              + (J02 * J12) * B[2][2];
    float c = ((J11 * J11) * B[1][1] + ((2.0f * J11) * J12) * B[1][2]) + (J12 * J12) * B[2][2];
    a += 0.3f;                                                   /* :272-273 */
    c += 0.3f;
    float det = a * c - b * b;                                   /* :275-277 */
    if (det < 1e-6f) det = 1e-6f;
    float conic_x = c / det, conic_y = -b / det, conic_z = a / det;

    float vpx = cam->viewport[0], vpy = cam->viewport[1];      /* :279-291 */
    float pcx = (fx_p * vx) / vz + vpx * 0.5f;
    float pcy = vpy * 0.5f + (fy_p * vy) / vz;
    float ocx = -fx_o * vx + vpx * 0.5f;
    float ocy = vpy * 0.5f - fy_o * vy;
    float cx = g_mix(pcx, ocx, t), cy = g_mix(pcy, ocy, t);
    float y_flip = (1.0f - cam->clip_y_sign) * 0.5f;
    float rcy = g_mix(cy, vpy - cy, y_flip);
    float rconic_y = conic_y * cam->clip_y_sign;

    float radius_x = ceilf(3.0f * sqrtf(a));                    /* :293-294 */
    float radius_y = ceilf(3.0f * sqrtf(c));

    if (collect_stats) {                                         /* :296-318 */
        float quad_area = g_max(0.0f, (4.0f * radius_x) * radius_y);
        uint32_t qa = g_f2u_sat(g_min(quad_area, 4294967295.0f));
        diag[0] += (uint32_t)(qa + 1023u) >> 10u;
        if (qa > diag[1]) diag[1] = qa;
        if (qa > 1024u) diag[2] += 1u;
        if (qa > 16384u) diag[3] += 1u;
        float gps_points = (6.28318530718f * sqrtf(g_max(det, 0.0f))) * oc_dilog(g_clamp(opacity, 0.0f, 1.0f));
        uint32_t gp = g_f2u_sat(g_min(ceilf(gps_points), 4294967295.0f));
        diag[4] += (uint32_t)(gp + 1023u) >> 10u;
        if (gp > diag[5]) diag[5] = gp;
        if (gp > 1024u) diag[6] += 1u;
        if (gp > 16384u) diag[7] += 1u;
    }

    float ndc_z = (P[10] * vz + P[14]) / (-vz);                 /* :320-321 */
    ndc_z = g_mix(ndc_z, ndc_z * 0.5f + 0.5f, cam->clip_z_01);

    /* cam_pos_world = -transpose(W) * view[3].xyz; dir = normalize(pos - cam) */
    float cam_w[3];
    for (int rr = 0; rr < 3; ++rr)
        cam_w[rr] = -((W[rr][0] * V[12] + W[rr][1] * V[13]) + W[rr][2] * V[14]);
    float dx = px - cam_w[0], dy = py - cam_w[1], dz = pz - cam_w[2];
    float len = sqrtf((dx * dx + dy * dy) + dz * dz);
    float x = dx / len, y = dy / len, z = dz / len;

    int eff_degree = sh_degree;                                  /* :348-351 */
    if (sh_lod_distance > 0.0f && (-vz) > sh_lod_distance) eff_degree = 0;

    float res[3];                                                /* :353-417 */
    if (layers && layers->count > 0) {
        float tmp[64], r3[3];
        res[0] = res[1] = res[2] = 0.0f;
        for (int l = 0; l < layers->count; ++l) {
            layer_row(layers, l, idx, r, tmp);
            sh_eval(tmp, x, y, z, eff_degree, r3);
            for (int k = 0; k < 3; ++k) res[k] = res[k] + g_max(r3[k], 0.0f) * layers->weights[l * 3 + k];
        }
    } else {
        sh_eval(r, x, y, z, eff_degree, res);
        for (int k = 0; k < 3; ++k) res[k] = g_max(res[k] + 0.5f, 0.0f);
    }

    out[0] = res[0]; out[1] = res[1]; out[2] = res[2]; out[3] = opacity;   /* :420-423 */
    out[4] = cx; out[5] = rcy; out[6] = radius_x; out[7] = radius_y;
    out[8] = conic_x; out[9] = rconic_y; out[10] = conic_z; out[11] = ndc_z;
    out[12] = a; out[13] = b * cam->clip_y_sign; out[14] = c; out[15] = det;
}

void oc_cull_anim(const float* rows, uint32_t n, const oc_camera* cam, int sh_degree,
                  float sh_lod_distance, int collect_stats, const int8_t* deltas, const float* scales,
                  int state_a, int state_b, float weight, uint32_t* ids, uint32_t* keys,
                  float* projected, uint32_t* visible_count, uint32_t* diag) {
    *visible_count = 0;
    for (int k = 0; k < 8; ++k) diag[k] = 0;
    for (uint32_t i = 0; i < n; ++i) { ids[i] = OC_SENTINEL; keys[i] = OC_SENTINEL; }
    oc_anim a = {deltas, n, scales, state_a, state_b, weight};
    /* shaders/cull.glsl:155-160 blends whenever the weight is positive, also
     * between two keys of state 0 (gsanim_sample returns {0, 0, w} there,
     * src/gaussian_loader_gsanim.cpp:495-508): (1 - w) x + w x need not be x */
    const int animated = deltas != NULL && (state_a != 0 || weight > 0.0f);
    float tmp[64];
    for (uint32_t i = 0; i < n; ++i) {
        const float* row = rows + (size_t)i * 64;
        if (animated) {
            anim_row(&a, i, row, tmp);
            row = tmp;
        }
        cull_one(row, i, cam, sh_degree, sh_lod_distance, collect_stats, NULL, ids, keys,
                 projected + (size_t)i * 16, visible_count, diag);
    }
}

void oc_cull_layers(const float* rows, uint32_t n, const oc_camera* cam, int sh_degree,
                    float sh_lod_distance, int collect_stats, const uint16_t* halves, int layer_count,
                    const float* weights, uint32_t* ids, uint32_t* keys, float* projected,
                    uint32_t* visible_count, uint32_t* diag) {
    *visible_count = 0;
    for (int k = 0; k < 8; ++k) diag[k] = 0;
    for (uint32_t i = 0; i < n; ++i) { ids[i] = OC_SENTINEL; keys[i] = OC_SENTINEL; }
    oc_layers L = {halves, n, layer_count, weights};
    for (uint32_t i = 0; i < n; ++i)
        cull_one(rows + (size_t)i * 64, i, cam, sh_degree, sh_lod_distance, collect_stats, &L, ids, keys,
                 projected + (size_t)i * 16, visible_count, diag);
}

void oc_cull(const float* rows, uint32_t n, const oc_camera* cam, int sh_degree,
             float sh_lod_distance, int collect_stats, uint32_t* ids, uint32_t* keys,
             float* projected, uint32_t* visible_count, uint32_t* diag) {
    oc_cull_anim(rows, n, cam, sh_degree, sh_lod_distance, collect_stats, NULL, NULL, 0, 0, 0.0f, ids, keys,
                 projected, visible_count, diag);
}

/* ------------------------------------------------------------------------ */
/* Radix sort (shaders/sort.glsl): 4 stable counting passes over 8-bit      */
/* digits, ascending, ties kept in input order.                             */
/* ------------------------------------------------------------------------ */
void oc_sort_pairs(const uint32_t* keys_in, const uint32_t* ids_in, uint32_t n,
                   uint32_t* keys_out, uint32_t* ids_out) {
    uint32_t* ka = (uint32_t*)malloc((size_t)n * 4 + 4);
    uint32_t* ia = (uint32_t*)malloc((size_t)n * 4 + 4);
    memcpy(keys_out, keys_in, (size_t)n * 4);
    memcpy(ids_out, ids_in, (size_t)n * 4);
    uint32_t *src_k = keys_out, *src_i = ids_out, *dst_k = ka, *dst_i = ia;
    for (int pass = 0; pass < 4; ++pass) {
        int shift = pass * 8;
        uint32_t count[256];
        memset(count, 0, sizeof(count));
        for (uint32_t i = 0; i < n; ++i) count[(src_k[i] >> shift) & 255u]++;
        uint32_t total = 0;
        for (int b = 0; b < 256; ++b) { uint32_t c = count[b]; count[b] = total; total += c; }
        for (uint32_t i = 0; i < n; ++i) {
            uint32_t d = count[(src_k[i] >> shift) & 255u]++;
            dst_k[d] = src_k[i];
            dst_i[d] = src_i[i];
        }
        uint32_t* t;
        t = src_k; src_k = dst_k; dst_k = t;
        t = src_i; src_i = dst_i; dst_i = t;
    }
    /* After an even number of passes the data is back in keys_out/ids_out. */
    free(ka);
    free(ia);
}

/* ------------------------------------------------------------------------ */
/* Quad coverage: shaders/splat.glsl:61-67 corners, NDC, viewport transform */
/* x_w = ndc * (w/2) + w/2, snapping to 1/256 pixel, pixel centres at       */
/* k + 0.5.  Fill rule: left and top edges inclusive (top = larger GL y).   */
/* ------------------------------------------------------------------------ */
static inline int64_t floor_div256(int64_t a) { return (a >= 0) ? (a / 256) : -((-a + 255) / 256); }
static inline int64_t ceil_div256(int64_t a) { return -floor_div256(-a); }
static inline int64_t snap256(float w) {
    float s = w * 256.0f;
    if (s > 1.0e15f) s = 1.0e15f;
    if (s < -1.0e15f) s = -1.0e15f;
    return (int64_t)rintf(s);
}

int oc_quad_rect(const float* p16, float jx, float jy, float vp_w, float vp_h, float clip_y_sign,
                 int width, int height, int32_t rect[4]) {
    rect[0] = rect[1] = rect[2] = rect[3] = 0;
    float ndc_z = p16[11];
    if (!(ndc_z >= -1.0f && ndc_z <= 1.0f)) return 0;
    float cx = p16[4], cy = p16[5], rx = p16[6], ry = p16[7];
    float hw = (float)width * 0.5f, hh = (float)height * 0.5f;
    float xa = (cx + -rx) + jx, xb = (cx + rx) + jx;
    float ya = (cy + -ry) + jy, yb = (cy + ry) + jy;
    float nxa = (2.0f * xa) / vp_w - 1.0f, nxb = (2.0f * xb) / vp_w - 1.0f;
    float nya = ((2.0f * ya) / vp_h - 1.0f) * clip_y_sign, nyb = ((2.0f * yb) / vp_h - 1.0f) * clip_y_sign;
    int64_t Xa = snap256(nxa * hw + hw), Xb = snap256(nxb * hw + hw);
    int64_t Ya = snap256(nya * hh + hh), Yb = snap256(nyb * hh + hh);
    int64_t X0 = Xa < Xb ? Xa : Xb, X1 = Xa < Xb ? Xb : Xa;
    int64_t Y0 = Ya < Yb ? Ya : Yb, Y1 = Ya < Yb ? Yb : Ya;
    int64_t i0 = ceil_div256(X0 - 128), i1 = ceil_div256(X1 - 128);
    int64_t j0 = floor_div256(Y0 - 128) + 1, j1 = floor_div256(Y1 - 128) + 1;
    if (i0 < 0) i0 = 0;
    if (j0 < 0) j0 = 0;
    if (i1 > width) i1 = width;
    if (j1 > height) j1 = height;
    if (i1 <= i0 || j1 <= j0) return 0;
    rect[0] = (int32_t)i0; rect[1] = (int32_t)i1; rect[2] = (int32_t)j0; rect[3] = (int32_t)j1;
    return 1;
}

/* The per-fragment Gaussian of shaders/splat.glsl:88-104. Returns 1 if kept. */
static inline int splat_power(const float* p16, float fcx, float fcy, float jx, float jy, float* power_out) {
    float ccx = p16[4] + jx, ccy = p16[5] + jy;
    float dx = fcx - ccx, dy = fcy - ccy;
    float power = -0.5f * (((p16[8] * dx) * dx + ((2.0f * p16[9]) * dx) * dy) + (p16[10] * dy) * dy);
    *power_out = power;
    return power <= 0.0f;
}

static inline float alpha_cutoff(float opacity) {
    return oc_logf((1.0f / 255.0f) / g_max(opacity, 1.0e-8f));
}

#ifdef __FLT16_MAX__
static inline float round_f16(float v) { return (float)(_Float16)v; }
#else
#error "the oracle needs _Float16"
#endif

uint64_t oc_composite_alpha(const uint32_t* sorted_ids, uint32_t count, const float* projected,
                            int width, int height, float vp_w, float vp_h, float clip_y_sign,
                            float bg, float jx, float jy, int fp16_per_blend, float* out) {
    size_t npix = (size_t)width * (size_t)height;
    /* GL-order (row 0 = bottom) working image. */
    float* img = (float*)malloc(npix * 4 * sizeof(float));
    for (size_t p = 0; p < npix; ++p) {
        img[p * 4 + 0] = bg; img[p * 4 + 1] = bg; img[p * 4 + 2] = bg; img[p * 4 + 3] = 0.0f;
    }
    uint64_t frags = 0;
    int bands = 64;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : frags)
    for (int band = 0; band < bands; ++band) {
        int rows_per = (height + bands - 1) / bands;
        int jb0 = band * rows_per, jb1 = jb0 + rows_per;
        if (jb1 > height) jb1 = height;
        if (jb0 >= jb1) continue;
        for (uint32_t s = 0; s < count; ++s) {
            uint32_t id = sorted_ids[s];
            if (id == OC_SENTINEL) continue;
            const float* p16 = projected + (size_t)id * 16;
            int32_t rc[4];
            if (!oc_quad_rect(p16, jx, jy, vp_w, vp_h, clip_y_sign, width, height, rc)) continue;
            int j0 = rc[2] > jb0 ? rc[2] : jb0, j1 = rc[3] < jb1 ? rc[3] : jb1;
            if (j0 >= j1) continue;
            float opacity = p16[3];
            float cutoff = alpha_cutoff(opacity);
            for (int j = j0; j < j1; ++j) {
                float fcy = (float)j + 0.5f;
                for (int i = rc[0]; i < rc[1]; ++i) {
                    float power;
                    if (!splat_power(p16, (float)i + 0.5f, fcy, jx, jy, &power)) continue;
                    if (power < cutoff) continue;
                    float alpha = g_min(opacity * expf(power), 0.99f);
                    float om = 1.0f - alpha;
                    float* d = img + ((size_t)j * width + i) * 4;
                    for (int k = 0; k < 3; ++k) {
                        float v = p16[k] * alpha + om * d[k];
                        d[k] = fp16_per_blend ? round_f16(v) : v;
                    }
                    float va = alpha + om * d[3];
                    d[3] = fp16_per_blend ? round_f16(va) : va;
                    frags++;
                }
            }
        }
    }
    for (int j = 0; j < height; ++j)
        memcpy(out + (size_t)(height - 1 - j) * width * 4, img + (size_t)j * width * 4,
               (size_t)width * 4 * sizeof(float));
    free(img);
    return frags;
}

/* ------------------------------------------------------------------------ */
/* Stochastic sample (shaders/splat.glsl:121-145, depth LESS + write).      */
/* ------------------------------------------------------------------------ */
static inline float hash13(float p0, float p1, float p2) {
    p0 = g_fract(p0 * 0.1031f);
    p1 = g_fract(p1 * 0.1031f);
    p2 = g_fract(p2 * 0.1031f);
    float d = (p0 * (p1 + 33.33f) + p1 * (p2 + 33.33f)) + p2 * (p0 + 33.33f);
    p0 = p0 + d; p1 = p1 + d; p2 = p2 + d;
    return g_fract((p0 + p1) * p2);
}

static inline uint32_t depth24(float ndc_z) {
    float zw = ndc_z * 0.5f + 0.5f;
    return (uint32_t)rintf(g_clamp(zw, 0.0f, 1.0f) * 16777215.0f);
}

uint64_t oc_stochastic_sample(const uint32_t* ids, uint32_t count, const float* projected,
                              int width, int height, float vp_w, float vp_h, float clip_y_sign,
                              float bg, float jx, float jy, float frame_seed, int rgba8,
                              float* out_rgba, float* out_depth) {
    size_t npix = (size_t)width * (size_t)height;
    uint32_t* zbuf = (uint32_t*)malloc(npix * sizeof(uint32_t));
    uint32_t* win = (uint32_t*)malloc(npix * sizeof(uint32_t));
    for (size_t p = 0; p < npix; ++p) { zbuf[p] = 16777215u; win[p] = OC_SENTINEL; }
    uint64_t kept = 0;
    int bands = 64;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : kept)
    for (int band = 0; band < bands; ++band) {
        int rows_per = (height + bands - 1) / bands;
        int jb0 = band * rows_per, jb1 = jb0 + rows_per;
        if (jb1 > height) jb1 = height;
        if (jb0 >= jb1) continue;
        for (uint32_t s = 0; s < count; ++s) {
            uint32_t id = ids[s];
            if (id == OC_SENTINEL) continue;
            const float* p16 = projected + (size_t)id * 16;
            int32_t rc[4];
            if (!oc_quad_rect(p16, jx, jy, vp_w, vp_h, clip_y_sign, width, height, rc)) continue;
            int j0 = rc[2] > jb0 ? rc[2] : jb0, j1 = rc[3] < jb1 ? rc[3] : jb1;
            if (j0 >= j1) continue;
            float opacity = p16[3];
            float cutoff = alpha_cutoff(opacity);
            uint32_t z24 = depth24(p16[11]);
            float hz = (float)id + frame_seed;
            for (int j = j0; j < j1; ++j) {
                float fcy = (float)j + 0.5f;
                for (int i = rc[0]; i < rc[1]; ++i) {
                    size_t pix = (size_t)j * width + i;
                    if (!(z24 < zbuf[pix])) continue;  /* early depth test, same outcome */
                    float power;
                    float fcx = (float)i + 0.5f;
                    if (!splat_power(p16, fcx, fcy, jx, jy, &power)) continue;
                    if (power < cutoff) continue;
                    float alpha = g_min(opacity * oc_expf(power), 0.99f);
                    float rnd = hash13(fcx, fcy, hz);
                    if (rnd >= alpha) continue;
                    zbuf[pix] = z24;
                    win[pix] = id;
                    kept++;
                }
            }
        }
    }
    for (int j = 0; j < height; ++j) {
        for (int i = 0; i < width; ++i) {
            size_t pix = (size_t)j * width + i;
            size_t o = (size_t)(height - 1 - j) * width + i;
            float* c = out_rgba + o * 4;
            if (win[pix] == OC_SENTINEL) {
                c[0] = bg; c[1] = bg; c[2] = bg; c[3] = 0.0f;
            } else {
                const float* p16 = projected + (size_t)win[pix] * 16;
                c[0] = p16[0]; c[1] = p16[1]; c[2] = p16[2]; c[3] = 1.0f;
            }
            if (rgba8)
                for (int k = 0; k < 4; ++k) c[k] = rintf(g_clamp(c[k], 0.0f, 1.0f) * 255.0f) / 255.0f;
            out_depth[o] = (float)zbuf[pix] / 16777215.0f;
        }
    }
    free(zbuf);
    free(win);
    return kept;
}

/* ------------------------------------------------------------------------ */
/* Gaussian Point Splatting (shaders/gps.glsl).                              */
/* ------------------------------------------------------------------------ */
static inline float hash01(uint32_t x) {                       /* gps.glsl:111-118 */
    x ^= x >> 16u;
    x *= 0x7feb352du;
    x ^= x >> 15u;
    x *= 0x846ca68bu;
    x ^= x >> 16u;
    return (float)x * (1.0f / 4294967296.0f);
}

typedef struct { float mean_x, mean_y, l00, l10, l11, alpha, dilog_alpha; uint32_t depth_key, color, splat_id; } gps_prep;

void oc_gps_frame(const uint32_t* ids, uint32_t count, const float* projected, int width,
                  int height, int supersample, uint32_t max_work_items, float clip_z_01,
                  int linear_color, float frame_seed, float bg, float* out_rgba, float* out_depth,
                  uint32_t* work_stats) {
    if (supersample < 1) supersample = 1;
    if (supersample > 4) supersample = 4;
    if (max_work_items < 1u) max_work_items = 1u;
    uint32_t gw = (uint32_t)width * supersample, gh = (uint32_t)height * supersample;
    size_t gpix = (size_t)gw * gh;
    uint64_t* buf = (uint64_t*)malloc(gpix * sizeof(uint64_t));
    for (size_t p = 0; p < gpix; ++p) buf[p] = 0xFFFFFFFF00000000ull;           /* gps_clear */
    gps_prep* prep = (gps_prep*)calloc(count ? count : 1, sizeof(gps_prep));
    uint32_t* work = (uint32_t*)malloc((size_t)max_work_items * 2 * sizeof(uint32_t));
    uint32_t work_count = 0, overflow = 0;
    float ss = (float)supersample;

    for (uint32_t idx = 0; idx < count; ++idx) {                                  /* gps_expand */
        uint32_t splat_id = ids[idx];
        if (splat_id == OC_SENTINEL) continue;
        const float* p16 = projected + (size_t)splat_id * 16;
        float ssf = g_max(ss, 1.0f);
        float cov_a = p16[12] + 0.3f, cov_b = p16[13], cov_c = p16[14] + 0.3f;
        float det = cov_a * cov_c - cov_b * cov_b;
        float expected = (((ssf * ssf) * 6.28318530718f) * sqrtf(g_max(det, 0.0f)))
                         * oc_dilog(g_clamp(p16[3], 0.0f, 1.0f));
        float ppw = g_max(ssf * ssf, 1.0f);
        float scaled = g_max(expected / ppw, 0.0f);
        uint32_t wic = g_f2u_sat(g_clamp(floorf(scaled), 0.0f, 4294967295.0f));
        if (hash01(splat_id + 0x9e3779b9u) < g_fract(scaled) && wic < 0xFFFFFFFFu) wic += 1u;
        if (wic == 0u) continue;
        uint32_t base = work_count;
        work_count += wic;
        uint32_t capacity = max_work_items;
        if (base >= capacity || wic > capacity - base) overflow = 1u;
        if (base >= capacity) continue;
        uint32_t write_count = wic < capacity - base ? wic : capacity - base;
        gps_prep* pr = &prep[idx];
        pr->mean_x = p16[4]; pr->mean_y = p16[5];
        pr->l00 = sqrtf(g_max(cov_a, 1.0e-5f));
        pr->l10 = cov_b / pr->l00;
        pr->l11 = sqrtf(g_max(cov_c - pr->l10 * pr->l10, 1.0e-5f));
        pr->alpha = g_clamp(p16[3], 1.0e-6f, 1.0f);
        pr->dilog_alpha = oc_dilog(pr->alpha);
        float ndc = p16[11];
        float z = g_mix(ndc * 0.5f + 0.5f, ndc, clip_z_01);
        pr->depth_key = g_f2u_sat(g_clamp(z, 0.0f, 1.0f) * 4294967294.0f);
        uint32_t rgb[3];
        for (int k = 0; k < 3; ++k) rgb[k] = (uint32_t)rintf(g_clamp(p16[k], 0.0f, 1.0f) * 255.0f);
        pr->color = rgb[0] | (rgb[1] << 8u) | (rgb[2] << 16u) | 0xFF000000u;
        if (linear_color) pr->color = splat_id;
        pr->splat_id = splat_id;
        for (uint32_t i = 0; i < write_count; ++i) { work[(size_t)(base + i) * 2] = idx; work[(size_t)(base + i) * 2 + 1] = i; }
    }

    uint32_t actual = work_count < max_work_items ? work_count : max_work_items;  /* gps_splat */
    int ppw_i = (int)rintf(ss * ss);
    if (ppw_i < 1) ppw_i = 1;
    uint32_t fseed = g_f2u_sat(frame_seed);
    for (uint32_t w = 0; w < actual; ++w) {
        uint32_t idx = work[(size_t)w * 2], sample_idx = work[(size_t)w * 2 + 1];
        const gps_prep* pr = &prep[idx];
        uint32_t seed_x = pr->splat_id * 747796405u + fseed * 2891336453u;
        uint32_t seed_y = pr->splat_id * 277803737u + 0x9E3779B9u;
        for (int p = 0; p < ppw_i; ++p) {
            uint32_t sx = seed_x + (sample_idx * (uint32_t)ppw_i + (uint32_t)p) * 374761393u, sy = seed_y;
            sx = 1664525u * sx + 1013904223u;
            sy = 1664525u * sy + 1013904223u;
            sx += 1664525u * sy;
            sy += 1664525u * sx;
            sx ^= sx >> 16u; sy ^= sy >> 16u;
            sx += 1664525u * sy;
            sy += 1664525u * sx;
            sx ^= sx >> 16u; sy ^= sy >> 16u;
            float r0 = (float)sx * 2.32830643654e-10f, r1 = (float)sy * 2.32830643654e-10f;
            float arg = oc_inv_dilog((1.0f - r0) * pr->dilog_alpha) / pr->alpha;
            arg = g_clamp(arg, 1.0e-7f, 1.0f);
            float radius = sqrtf(-2.0f * oc_logf(arg));
            float az = 6.28318530718f * r1;
            float sn, cs;
            oc_sincosf(az, &sn, &cs);
            float lx = cs * radius, ly = sn * radius;
            float ptx = (pr->mean_x + pr->l00 * lx) * g_max(ss, 1.0f);
            float pty = (pr->mean_y + (pr->l10 * lx + pr->l11 * ly)) * g_max(ss, 1.0f);
            float fx = floorf(ptx + 0.5f), fy = floorf(pty + 0.5f);
            if (fx >= 0.0f && fy >= 0.0f && fx < (float)gw && fy < (float)gh) {
                size_t pix = (size_t)fy * gw + (size_t)fx;
                uint64_t v = ((uint64_t)pr->depth_key << 32) | pr->color;
                if (v < buf[pix]) buf[pix] = v;
            }
        }
    }

    for (int y = 0; y < height; ++y) {                                           /* gps_resolve */
        for (int x = 0; x < width; ++x) {
            float sum[3] = {0.0f, 0.0f, 0.0f}, cov = 0.0f;
            uint32_t min_key = 0xFFFFFFFFu;
            for (int yy = 0; yy < supersample; ++yy) {
                for (int xx = 0; xx < supersample; ++xx) {
                    uint32_t sxp = (uint32_t)(x * supersample + xx), syp = (uint32_t)(y * supersample + yy);
                    if (sxp >= gw || syp >= gh) continue;
                    uint64_t v = buf[(size_t)syp * gw + sxp];
                    uint32_t key = (uint32_t)(v >> 32), payload = (uint32_t)v;
                    if (key != 0xFFFFFFFFu) {
                        if (linear_color) {
                            const float* q = projected + (size_t)payload * 16;
                            sum[0] = sum[0] + q[0]; sum[1] = sum[1] + q[1]; sum[2] = sum[2] + q[2];
                        } else {
                            sum[0] = sum[0] + (float)(payload & 255u) / 255.0f;
                            sum[1] = sum[1] + (float)((payload >> 8u) & 255u) / 255.0f;
                            sum[2] = sum[2] + (float)((payload >> 16u) & 255u) / 255.0f;
                        }
                        cov = cov + 1.0f;
                        if (key < min_key) min_key = key;
                    }
                }
            }
            size_t o = (size_t)(height - 1 - y) * width + x;
            float* c = out_rgba + o * 4;
            if (cov <= 0.0f) {
                c[0] = bg; c[1] = bg; c[2] = bg; c[3] = 0.0f;
                out_depth[o] = 1.0f;
            } else {
                float spc = (float)(supersample * supersample);
                c[0] = sum[0] / spc; c[1] = sum[1] / spc; c[2] = sum[2] / spc; c[3] = cov / spc;
                out_depth[o] = (float)min_key / 4294967294.0f;
            }
        }
    }
    work_stats[0] = work_count;
    work_stats[1] = overflow;
    free(buf);
    free(prep);
    free(work);
}

/* ------------------------------------------------------------------------ */
/* Accumulation (shaders/accum.glsl).                                        */
/* ------------------------------------------------------------------------ */
void oc_accum(const float* sample, const float* history, float sample_count, uint64_t count4,
              float* out) {
    float n = g_max(sample_count, 1.0f);
    for (uint64_t k = 0; k < count4; ++k) out[k] = history[k] + (sample[k] - history[k]) / n;
}

/* Texel (x, y) in GL orientation of a top-first image. */
static inline const float* texel(const float* img, int w, int h, int x, int y, int ch) {
    return img + ((size_t)(h - 1 - y) * w + x) * ch;
}

static void bilinear4(const float* img, int w, int h, float u, float v, float out[4]) {
    float px = u * (float)w - 0.5f, py = v * (float)h - 0.5f;
    float flx = floorf(px), fly = floorf(py);
    int x0 = (int)flx, y0 = (int)fly, x1 = x0 + 1, y1 = y0 + 1;
    float fx = g_fract(px), fy = g_fract(py);
    int cx0 = x0 < 0 ? 0 : (x0 > w - 1 ? w - 1 : x0), cx1 = x1 < 0 ? 0 : (x1 > w - 1 ? w - 1 : x1);
    int cy0 = y0 < 0 ? 0 : (y0 > h - 1 ? h - 1 : y0), cy1 = y1 < 0 ? 0 : (y1 > h - 1 ? h - 1 : y1);
    const float* c00 = texel(img, w, h, cx0, cy0, 4);
    const float* c10 = texel(img, w, h, cx1, cy0, 4);
    const float* c01 = texel(img, w, h, cx0, cy1, 4);
    const float* c11 = texel(img, w, h, cx1, cy1, 4);
    for (int k = 0; k < 4; ++k) out[k] = g_mix(g_mix(c00[k], c10[k], fx), g_mix(c01[k], c11[k], fx), fy);
}

void oc_taa(const float* cur_color, const float* cur_depth, const float* hist_color,
            const float* hist_xyz, int width, int height, const float* inv_view,
            const float* prev_view, const float* vo, const float* fc, const float* pfc,
            const float* proj_z, float history_valid, float view_changed, float* out_color,
            float* out_xyz) {
    for (int y = 0; y < height; ++y) {
        for (int x = 0; x < width; ++x) {
            float u = ((float)x + 0.5f) / (float)width, v = ((float)y + 0.5f) / (float)height;
            const float* cc = texel(cur_color, width, height, x, y, 4);
            float depth = *texel(cur_depth, width, height, x, y, 1);
            /* reconstruct_view_pos (:82-94) */
            float z_ndc = depth * 2.0f - 1.0f;
            float view_z = -proj_z[1] / (z_ndc + proj_z[0]);
            float pxx = u * vo[0], pxy = v * vo[1];
            float unflip = (1.0f - fc[2]) * 0.5f;
            pxy = g_mix(pxy, vo[1] - pxy, unflip);
            float cex = pxx - vo[0] * 0.5f, cey = pxy - vo[1] * 0.5f;
            float denom = g_mix(fc[0] / view_z, -fc[1], vo[2]);
            float vp3[3] = {cex / denom, cey / denom, view_z};
            float world[3];
            for (int rr = 0; rr < 3; ++rr)
                world[rr] = ((inv_view[rr] * vp3[0] + inv_view[4 + rr] * vp3[1]) + inv_view[8 + rr] * vp3[2])
                            + inv_view[12 + rr];
            /* project_prev_uv (:96-114) */
            float pv[3];
            for (int rr = 0; rr < 3; ++rr)
                pv[rr] = ((prev_view[rr] * world[0] + prev_view[4 + rr] * world[1]) + prev_view[8 + rr] * world[2])
                         + prev_view[12 + rr];
            float puv_x = -1.0f, puv_y = -1.0f;
            if (!(pv[2] >= -0.001f)) {
                float t = vo[3];
                float ppx = (pfc[0] * pv[0]) / pv[2] + vo[0] * 0.5f;
                float ppy = vo[1] * 0.5f + (pfc[0] * pv[1]) / pv[2];
                float opx = -pfc[1] * pv[0] + vo[0] * 0.5f;
                float opy = vo[1] * 0.5f - pfc[1] * pv[1];
                float qx = g_mix(ppx, opx, t), qy = g_mix(ppy, opy, t);
                float y_flip = (1.0f - pfc[2]) * 0.5f;
                qy = g_mix(qy, vo[1] - qy, y_flip);
                puv_x = qx / vo[0];
                puv_y = qy / vo[1];
            }
            int valid = history_valid != 0.0f && puv_x >= 0.0f && puv_x <= 1.0f && puv_y >= 0.0f && puv_y <= 1.0f;
            float hc[4] = {0, 0, 0, 0}, hx[4] = {0, 0, 0, 0};
            if (valid) {
                bilinear4(hist_color, width, height, puv_x, puv_y, hc);
                bilinear4(hist_xyz, width, height, puv_x, puv_y, hx);
                float ddx = world[0] - hx[0], ddy = world[1] - hx[1], ddz = world[2] - hx[2];
                float len = sqrtf((ddx * ddx + ddy * ddy) + ddz * ddz);
                valid = hc[3] > 0.0f && (view_changed == 0.0f || len < 100.0f);
            }
            size_t o = ((size_t)(height - 1 - y) * width + x) * 4;
            if (valid) {
                float n = g_min(hc[3], 128.0f);
                for (int k = 0; k < 3; ++k) out_color[o + k] = (hc[k] * n + cc[k]) / (n + 1.0f);
                out_color[o + 3] = g_min(n + 1.0f, 128.0f);
                for (int k = 0; k < 3; ++k) out_xyz[o + k] = (hx[k] * n + world[k]) / (n + 1.0f);
                out_xyz[o + 3] = 1.0f;
            } else {
                for (int k = 0; k < 3; ++k) out_color[o + k] = cc[k];
                out_color[o + 3] = 1.0f;
                for (int k = 0; k < 3; ++k) out_xyz[o + k] = world[k];
                out_xyz[o + 3] = 1.0f;
            }
        }
    }
}

/* The TAA's inverse view matrix as the reference computes it
 * (src/renderer.cpp:86-206): the adjugate by cofactor expansion divided by
 * the determinant, returning 0 when |det| <= 1e-8.  Entry k = 4c + r of the
 * column-major result is (-1)^(c+r) times the 3x3 determinant over rows != c
 * and columns != r of m, summed as six triple products left to right: the
 * first factor's column a runs over the remaining columns in order at the
 * first remaining row, the other two columns take the other two rows in
 * order, then swapped (sign pattern + - - + + -). */
int oc_mat4_inverse(const float* m, float* out) {
    float inv[16];
    for (int k = 0; k < 16; ++k) {
        int c = k >> 2, r = k & 3, R[3], Q[3], n = 0;
        for (int i = 0; i < 4; ++i) if (i != c) R[n++] = i;
        n = 0;
        for (int i = 0; i < 4; ++i) if (i != r) Q[n++] = i;
        int flip = (c + r) & 1;
        float acc = 0.0f;
        for (int t = 0; t < 6; ++t) {
            int ai = t >> 1, sw = t & 1;
            int a = Q[ai], b = Q[ai == 0 ? 1 : 0], d = Q[ai == 2 ? 1 : 2];
            float p = (m[a * 4 + R[0]] * m[b * 4 + (sw ? R[2] : R[1])]) * m[d * 4 + (sw ? R[1] : R[2])];
            int minus = ((ai == 1) ^ sw) ^ flip;
            acc = t == 0 ? (minus ? -p : p) : (minus ? acc - p : acc + p);
        }
        inv[k] = acc;
    }
    float det = ((m[0] * inv[0] + m[1] * inv[4]) + m[2] * inv[8]) + m[3] * inv[12];
    if (fabsf(det) <= 1.0e-8f) return 0;
    det = 1.0f / det;
    for (int i = 0; i < 16; ++i) out[i] = inv[i] * det;
    return 1;
}

float oc_halton(uint32_t index, uint32_t base) {              /* src/renderer.cpp:246-255 */
    float f = 1.0f, r = 0.0f;
    while (index > 0) {
        f /= (float)base;
        r += f * (float)(index % base);
        index /= base;
    }
    return r;
}

/* ------------------------------------------------------------------------ */
/* Display transform (shaders/accum.glsl:201-240; blit :181-192).            */
/* ------------------------------------------------------------------------ */
float oc_half_to_float(uint16_t h) {
    uint32_t sign = (uint32_t)(h >> 15) << 31, e = (h >> 10) & 31u, m = h & 1023u;
    if (e == 31u) return fbits(sign | 0x7f800000u | (m << 13));
    if (e == 0u) {
        if (m == 0u) return fbits(sign);
        float v = (float)m * 5.9604644775390625e-08f;   /* m * 2^-24, exact */
        return sign ? -v : v;
    }
    return fbits(sign | ((e + 112u) << 23) | (m << 13));
}

static float oc_exp2f_det(float x) { return oc_expf(x * 0.6931471805599453f); }
static float oc_log2f_det(float x) { return oc_logf(x) * 1.4426950216293335f; }

static float lut_entry(const uint16_t* lut, int n, int x, int y, int z, int c) {
    int i = ((z * n + y) * n + x) * 3 + c;                    /* shaders/accum.glsl:216-224 */
    return (float)lut[i] / 65535.0f;
}

void oc_display(const uint16_t* in_half, int width, int height, const uint16_t* lut, int lut_size,
                float log2_min, float log2_max, float exposure_ev, float* out_rgba) {
    size_t npix = (size_t)width * (size_t)height;
    float gain = oc_exp2f_det(exposure_ev);
    float lo_clamp = oc_exp2f_det(log2_min);
    float range = log2_max - log2_min;
    float top = (float)(lut_size - 1);
    for (size_t i = 0; i < npix; ++i) {
        float px[4];
        for (int c = 0; c < 4; ++c) px[c] = oc_half_to_float(in_half[i * 4 + c]);
        float* o = out_rgba + i * 4;
        if (!lut) { for (int c = 0; c < 4; ++c) o[c] = px[c]; continue; }
        int lo[3], hi[3];
        float f[3];
        for (int c = 0; c < 3; ++c) {                          /* :226-232 */
            float rad = px[c] * gain;
            float s = g_clamp((oc_log2f_det(g_max(rad, lo_clamp)) - log2_min) / range, 0.0f, 1.0f);
            if (s != s) s = 0.0f;                              /* NaN input: first lattice entry */
            float p = s * top;
            float fl = floorf(p);
            lo[c] = (int)fl;
            hi[c] = lo[c] + 1 < lut_size - 1 ? lo[c] + 1 : lut_size - 1;
            f[c] = p - fl;
        }
        for (int c = 0; c < 3; ++c) {                          /* :233-238 */
            int n = lut_size;
            float a = g_mix(g_mix(lut_entry(lut, n, lo[0], lo[1], lo[2], c), lut_entry(lut, n, hi[0], lo[1], lo[2], c), f[0]),
                            g_mix(lut_entry(lut, n, lo[0], hi[1], lo[2], c), lut_entry(lut, n, hi[0], hi[1], lo[2], c), f[0]),
                            f[1]);
            float b = g_mix(g_mix(lut_entry(lut, n, lo[0], lo[1], hi[2], c), lut_entry(lut, n, hi[0], lo[1], hi[2], c), f[0]),
                            g_mix(lut_entry(lut, n, lo[0], hi[1], hi[2], c), lut_entry(lut, n, hi[0], hi[1], hi[2], c), f[0]),
                            f[1]);
            o[c] = g_mix(a, b, f[2]);
        }
        o[3] = 1.0f;
    }
}
