// Learned path guiding: device side shared by the renderer and the training kernels.
//
// A small MLP maps a surface point to a proposal distribution over incident directions:
//   input  (80)  12-band frequency encoding sin/cos(2^k pi x) of the position normalised to
//                the scene bounds (3 x 12 x 2 = 72), the normal facing the viewer (3), the
//                hero wavelength mapped to [0, 1] (1), a constant 1 that acts as the first
//                layer's bias (1), and 3 zeros
//   hidden       4 layers of width 64 with ReLU, no biases
//   head   (41)  8 von Mises-Fisher lobes: mixture logits (8), unnormalised mean directions
//                (8 x 3), log concentrations (8); and the logit of the point's selection
//                probability c (used when the guide learns it, fl_guide_config.learn_select)
// Weights are FP16 (row-major [out][in], packed layer after layer, 20,032 values) and every
// product accumulates in FP32 on the tensor cores (mma.sync m16n8k16, operands staged in
// shared memory and loaded with ldmatrix). One warp evaluates 16 points at a time; the
// output of one layer stays in registers as the A operand of the next.
//
// The renderer samples the continuation at Lambert vertices from this mixture with
// probability c and from the BSDF otherwise (one-sample MIS): the path weight uses the
// mixture density c q(w) + (1 - c) p_bsdf(w), which is positive wherever the BSDF is,
// so the estimator stays unbiased whatever the network outputs. The network is new code:
// the reference has no guiding.
#pragma once

#include <cuda_fp16.h>

#include "fl_device.cuh"

namespace fl {

constexpr int kGuideIn = 80;
constexpr int kGuideHidden = 64;
constexpr int kGuideOut = 41;
constexpr int kGuideLobes = 8;
constexpr int kGuideParams = 64 * 80 + 3 * 64 * 64 + 41 * 64;  // 20,032
constexpr int kGuideLayers = 5;
// shared-memory copy of the weights: rows padded to 88 (layer 1) or 72 halves so that the
// eight rows read by one ldmatrix fall into distinct banks; the head gets 8 zero rows so
// that its transpose can be the B operand of a K = 48 product
constexpr int kLdIn = 88, kLdH = 72, kHeadRowsPad = 48;
constexpr int kSmWHalves = 64 * 88 + 3 * 64 * 72 + 48 * 72;  // 22,912
constexpr int kHeadLd = 44;                                  // floats per head row in shared memory
// log concentration = min + (max - min) * sigmoid(s - shift): bounded, with a gradient
// everywhere (a clamp would freeze a lobe that overshoots), about 0.4 at s = 0
constexpr float kLogKappaMin = -2.f, kLogKappaMax = 7.f, kLogKappaShift = 2.f;
// per path slot: pi[8], mu[8][3], kappa[8], log(pi * vMF normalisation)[8], c, 3 unused
constexpr int kMixFloats = 52;
constexpr int kMixSelect = 48;
// learned selection probability c = min + (max - min) * sigmoid(s): kept inside (0, 1), so
// both techniques of the one-sample MIS keep a positive density; the upper bound also bounds
// the weight of radiance the BSDF part finds where the mixture is sharp (1 / (1 - max))
// (measured on the 1024^2 caustic: bounds [0.05, 0.95] made the equal-time error 3.7x
// worse than a fixed c = 0.5, [0.2, 0.7] 1.13x better)
#ifndef FL_SELECT_MIN
#define FL_SELECT_MIN 0.2f
#endif
#ifndef FL_SELECT_MAX
#define FL_SELECT_MAX 0.7f
#endif
constexpr float kSelectMin = FL_SELECT_MIN, kSelectMax = FL_SELECT_MAX;
constexpr int kRecFloats = 20;  // training record, see GuideArgs
constexpr uint32_t kNoRecord = 0xffffffffu;

__host__ __device__ constexpr int guide_in(int l) { return l == 0 ? 80 : 64; }
__host__ __device__ constexpr int guide_out(int l) { return l == 4 ? 41 : 64; }
__host__ __device__ constexpr int guide_woff(int l) { return l == 0 ? 0 : 5120 + (l - 1) * 4096; }
__host__ __device__ constexpr int guide_sm_off(int l) { return l == 0 ? 0 : 5632 + (l - 1) * 4608; }
__host__ __device__ constexpr int guide_sm_ld(int l) { return l == 0 ? kLdIn : kLdH; }

// Guiding state seen by the render kernels (all null / zero when guiding is off).
// Training record (kRecFloats floats): 0-2 position, 3-5 normal facing the viewer,
// 6 hero wavelength, 7-9 sampled direction, 10 its sampling density, 11 incident radiance
// estimate along it (written when the path ends), 12-15 path throughput after the vertex
// (per hero wavelength, before Russian roulette), 16-19 radiance gathered before it.
struct GuideArgs {
    const __half *w;      // packed FP16 weights
    float *mix;           // kMixFloats per path slot (see kMixFloats); pi[0] < 0 = unusable
    uint32_t *rec_idx;    // 2 x cap open records per path (kNoRecord = none)
    float *rec;           // records
    uint32_t *rec_count;  // records written this wave
    uint32_t rec_cap;
    float select;         // c: probability of sampling the mixture at a Lambert vertex (0: guiding off)
    int learned_select;   // take c from the network's output per point instead of `select`
    int record;           // write training records
    float bmin[3], binv[3];  // position normalisation to [0, 1]^3
};

// --------------------------------------------------------------------------- tensor-core primitives

__device__ __forceinline__ void mma16816(float c[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void ldsm_x4(uint32_t r[4], const void *p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p))
                 : "memory");
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t r[4], const void *p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p))
                 : "memory");
}
__device__ __forceinline__ void ldsm_x2(uint32_t r[2], const void *p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];\n"
                 : "=r"(r[0]), "=r"(r[1])
                 : "r"(smem_u32(p))
                 : "memory");
}
__device__ __forceinline__ void ldsm_x2_t(uint32_t r[2], const void *p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n"
                 : "=r"(r[0]), "=r"(r[1])
                 : "r"(smem_u32(p))
                 : "memory");
}
// two floats -> packed half2, clamped to the FP16 range (and through ReLU when asked)
__device__ __forceinline__ uint32_t pack_h2(float x, float y, bool relu) {
    if (relu) {
        x = fmaxf(x, 0.f);
        y = fmaxf(y, 0.f);
    }
    x = fminf(fmaxf(x, -65000.f), 65000.f);
    y = fminf(fmaxf(y, -65000.f), 65000.f);
    __half2 h = __floats2half2_rn(x, y);
    return *reinterpret_cast<uint32_t *>(&h);
}

// Copies the packed weights into the padded shared-memory layout (all threads of the block).
__device__ inline void guide_stage_weights(__half *sw, const __half *__restrict__ w) {
    uint32_t *z = reinterpret_cast<uint32_t *>(sw);
    for (int i = threadIdx.x; i < kSmWHalves / 2; i += blockDim.x) z[i] = 0u;
    __syncthreads();
#pragma unroll
    for (int l = 0; l < kGuideLayers; ++l) {
        const int in = guide_in(l), out = guide_out(l), ld = guide_sm_ld(l);
        const int per_row = in / 8;
        for (int i = threadIdx.x; i < out * per_row; i += blockDim.x) {
            const int r = i / per_row, c8 = i % per_row;
            const uint4 v = *reinterpret_cast<const uint4 *>(w + guide_woff(l) + r * in + c8 * 8);
            *reinterpret_cast<uint4 *>(sw + guide_sm_off(l) + r * ld + c8 * 8) = v;
        }
    }
    __syncthreads();
}

// --------------------------------------------------------------------------- input encoding

// Half of one point's 80 features (part 0: features 0..39, part 1: 40..79) as FP16, written
// to `row` + 40 * part. pn is the position normalised to [0, 1]^3. Feature 2 (12 a + k) + {0, 1}
// is sin / cos(2^k pi pn[a]); both halves of a warp run the same loop over their 20
// (axis, band) pairs, so the two parts do not serialise.
__device__ inline void guide_encode_pairs(const float pn[3], const float nf[3], float lam01, int part, uint32_t h[20]) {
#pragma unroll
    for (int i = 0; i < 20; ++i) {
        const int pair = 20 * part + i;  // (axis, band) = (pair / 12, pair % 12); pairs >= 36 are not sines
        const int a = pair < 36 ? pair / 12 : 0, k = pair < 36 ? pair % 12 : 0;
        const float x = a == 0 ? pn[0] : (a == 1 ? pn[1] : pn[2]);
        float sv, cv;
        sincospif(x * __int_as_float((127 + k) << 23), &sv, &cv);
        h[i] = pack_h2(sv, cv, false);
    }
    if (part == 1) {
        // features 72..79
        h[16] = pack_h2(nf[0], nf[1], false);
        h[17] = pack_h2(nf[2], lam01, false);
        h[18] = pack_h2(1.f, 0.f, false);
        h[19] = 0u;
    }
}
__device__ inline void guide_encode_part(const float pn[3], const float nf[3], float lam01, int part, __half *row) {
    uint32_t h[20];  // feature pairs as packed FP16
    guide_encode_pairs(pn, nf, lam01, part, h);
    uint4 *dst = reinterpret_cast<uint4 *>(row + 40 * part);
#pragma unroll
    for (int q = 0; q < 5; ++q) dst[q] = make_uint4(h[4 * q], h[4 * q + 1], h[4 * q + 2], h[4 * q + 3]);
}

__device__ inline void guide_normalise(const float bmin[3], const float binv[3], v3 p, float pn[3]) {
    pn[0] = fminf(fmaxf((p.x - bmin[0]) * binv[0], 0.f), 1.f);
    pn[1] = fminf(fmaxf((p.y - bmin[1]) * binv[1], 0.f), 1.f);
    pn[2] = fminf(fmaxf((p.z - bmin[2]) * binv[2], 0.f), 1.f);
}

// The features of a training record (position, normal, wavelength) into `row`, part 0 or 1.
__device__ inline void guide_encode_record(const float *R, const float bmin[3], const float binv[3], int part,
                                           __half *row) {
    float pn[3];
    guide_normalise(bmin, binv, mk(R[0], R[1], R[2]), pn);
    const float nf[3] = {R[3], R[4], R[5]};
    guide_encode_part(pn, nf, (R[6] - 380.f) * (1.f / 340.f), part, row);
}

// --------------------------------------------------------------------------- forward pass

// One warp: the network on 16 points whose features are rows 0..15 of X (ld kLdIn); X is
// read only by the first layer, so `head` may alias it.
// When `act` is set, the four post-ReLU hidden layers are also stored to act + l * act_stride
// (rows 0..15, ld kLdH) for the backward pass. The head goes to `head` (16 x kHeadLd floats).
__device__ inline void guide_forward_warp(const __half *sw, const __half *X, __half *act, int act_stride,
                                          float *head) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    // B operand rows (output features) and column half picked by this lane for x4 loads of two n-tiles
    const int brow = (lane & 7) + ((lane >> 4) << 3), bcol = ((lane >> 3) & 1) * 8;
    uint32_t h[4][4];
    // layer 1 (K = 80): one A tile of the features at a time
    {
        float acc[8][4];
#pragma unroll
        for (int n = 0; n < 8; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
        const __half *W = sw + guide_sm_off(0);
#pragma unroll
        for (int kt = 0; kt < 5; ++kt) {
            uint32_t a[4];
            ldsm_x4(a, X + (lane & 15) * kLdIn + kt * 16 + (lane >> 4) * 8);
#pragma unroll
            for (int np = 0; np < 4; ++np) {
                uint32_t b[4];
                ldsm_x4(b, W + (np * 16 + brow) * kLdIn + kt * 16 + bcol);
                mma16816(acc[2 * np], a, b[0], b[1]);
                mma16816(acc[2 * np + 1], a, b[2], b[3]);
            }
        }
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
            h[kt][0] = pack_h2(acc[2 * kt][0], acc[2 * kt][1], true);
            h[kt][1] = pack_h2(acc[2 * kt][2], acc[2 * kt][3], true);
            h[kt][2] = pack_h2(acc[2 * kt + 1][0], acc[2 * kt + 1][1], true);
            h[kt][3] = pack_h2(acc[2 * kt + 1][2], acc[2 * kt + 1][3], true);
        }
    }
    // hidden layers 2..4 (K = 64)
#pragma unroll
    for (int l = 1; l < 4; ++l) {
        if (act) {
            __half *A = act + (l - 1) * act_stride;
#pragma unroll
            for (int kt = 0; kt < 4; ++kt) {
                *reinterpret_cast<uint32_t *>(A + g * kLdH + kt * 16 + 2 * t) = h[kt][0];
                *reinterpret_cast<uint32_t *>(A + (g + 8) * kLdH + kt * 16 + 2 * t) = h[kt][1];
                *reinterpret_cast<uint32_t *>(A + g * kLdH + kt * 16 + 8 + 2 * t) = h[kt][2];
                *reinterpret_cast<uint32_t *>(A + (g + 8) * kLdH + kt * 16 + 8 + 2 * t) = h[kt][3];
            }
        }
        float acc[8][4];
#pragma unroll
        for (int n = 0; n < 8; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
        const __half *W = sw + guide_sm_off(l);
#pragma unroll
        for (int np = 0; np < 4; ++np)
#pragma unroll
            for (int kt = 0; kt < 4; ++kt) {
                uint32_t b[4];
                ldsm_x4(b, W + (np * 16 + brow) * kLdH + kt * 16 + bcol);
                mma16816(acc[2 * np], h[kt], b[0], b[1]);
                mma16816(acc[2 * np + 1], h[kt], b[2], b[3]);
            }
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
            h[kt][0] = pack_h2(acc[2 * kt][0], acc[2 * kt][1], true);
            h[kt][1] = pack_h2(acc[2 * kt][2], acc[2 * kt][3], true);
            h[kt][2] = pack_h2(acc[2 * kt + 1][0], acc[2 * kt + 1][1], true);
            h[kt][3] = pack_h2(acc[2 * kt + 1][2], acc[2 * kt + 1][3], true);
        }
    }
    if (act) {
        __half *A = act + 3 * act_stride;
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
            *reinterpret_cast<uint32_t *>(A + g * kLdH + kt * 16 + 2 * t) = h[kt][0];
            *reinterpret_cast<uint32_t *>(A + (g + 8) * kLdH + kt * 16 + 2 * t) = h[kt][1];
            *reinterpret_cast<uint32_t *>(A + g * kLdH + kt * 16 + 8 + 2 * t) = h[kt][2];
            *reinterpret_cast<uint32_t *>(A + (g + 8) * kLdH + kt * 16 + 8 + 2 * t) = h[kt][3];
        }
    }
    // head (N = 41: n-tiles 0..5, the last holding output 40 and seven zero rows), linear
    {
        float acc[6][4];
#pragma unroll
        for (int n = 0; n < 6; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
        const __half *W = sw + guide_sm_off(4);
#pragma unroll
        for (int np = 0; np < 3; ++np)
#pragma unroll
            for (int kt = 0; kt < 4; ++kt) {
                uint32_t b[4];
                ldsm_x4(b, W + (np * 16 + brow) * kLdH + kt * 16 + bcol);
                mma16816(acc[2 * np], h[kt], b[0], b[1]);
                mma16816(acc[2 * np + 1], h[kt], b[2], b[3]);
            }
#pragma unroll
        for (int n = 0; n < 5; ++n) {
            head[g * kHeadLd + n * 8 + 2 * t] = acc[n][0];
            head[g * kHeadLd + n * 8 + 2 * t + 1] = acc[n][1];
            head[(g + 8) * kHeadLd + n * 8 + 2 * t] = acc[n][2];
            head[(g + 8) * kHeadLd + n * 8 + 2 * t + 1] = acc[n][3];
        }
        if (t < 2) {  // columns 40..43 of the 44 a head row holds
            head[g * kHeadLd + 40 + 2 * t] = acc[5][0];
            head[g * kHeadLd + 41 + 2 * t] = acc[5][1];
            head[(g + 8) * kHeadLd + 40 + 2 * t] = acc[5][2];
            head[(g + 8) * kHeadLd + 41 + 2 * t] = acc[5][3];
        }
    }
}

// --------------------------------------------------------------------------- vMF mixture

__device__ inline float guide_sigmoid(float s) { return 1.f / (1.f + expf(-(s - kLogKappaShift))); }
__device__ inline float guide_log_kappa(float s) { return kLogKappaMin + (kLogKappaMax - kLogKappaMin) * guide_sigmoid(s); }
__device__ inline float guide_kappa(float s) { return expf(guide_log_kappa(s)); }
// log of the vMF normalisation kappa / (2 pi (1 - exp(-2 kappa)))
__device__ inline float vmf_log_norm(float k) { return logf(k) - 1.8378770664f - logf(-expm1f(-2.f * k)); }
__device__ inline float vmf_log_norm2(float k, float logk) { return logk - 1.8378770664f - log1pf(-expf(-2.f * k)); }

__device__ inline float guide_select(float s) { return kSelectMin + (kSelectMax - kSelectMin) / (1.f + expf(-s)); }

// Mixture parameters of one point from its 41 head outputs: pi (softmax), mu (unit), kappa
// and the selection probability c (out[40]); with `lognorm` (the per-slot layout of
// kMixFloats) log(pi_j * C(kappa_j)) goes to out[40..47] and c to out[kMixSelect].
// Returns false (and marks pi[0] = -1) when the outputs are not finite.
__device__ inline bool guide_mixture(const float *h, float *out, bool lognorm = false) {
    float mx = h[0];
#pragma unroll
    for (int j = 1; j < 8; ++j) mx = fmaxf(mx, h[j]);
    float pi[8], sum = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        pi[j] = expf(h[j] - mx);
        sum += pi[j];
    }
    bool ok = isfinite(sum) && sum > 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        out[j] = pi[j] / sum;
        const float x = h[8 + 3 * j], y = h[9 + 3 * j], z = h[10 + 3 * j];
        const float len = sqrtf(x * x + y * y + z * z);
        const float il = 1.f / fmaxf(len, 1e-6f);
        out[8 + 3 * j] = x * il;
        out[9 + 3 * j] = y * il;
        out[10 + 3 * j] = z * il;
        const float lk = guide_log_kappa(h[32 + j]);
        out[32 + j] = expf(lk);
        if (lognorm) out[40 + j] = (h[j] - mx) - logf(sum) + vmf_log_norm2(out[32 + j], lk);
        ok = ok && isfinite(len) && len > 1e-6f && isfinite(h[32 + j]);
    }
    out[lognorm ? kMixSelect : 40] = guide_select(h[40]);
    ok = ok && isfinite(h[40]);
    if (!ok) out[0] = -1.f;
    return ok;
}

// density of a mixture laid out by guide_mixture(.., lognorm = true)
__device__ inline float guide_mixture_pdf(const float *__restrict__ m, v3 w) {
    float q = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const float c = m[8 + 3 * j] * w.x + m[9 + 3 * j] * w.y + m[10 + 3 * j] * w.z;
        q += expf(m[40 + j] + m[32 + j] * (c - 1.f));
    }
    return q;
}

// Samples the mixture: lobe by u_lobe, then the vMF lobe by (u1, u2) (Wenzel Jakob, "Numerically
// stable sampling of the von Mises Fisher distribution on S^2", 2012).
__device__ inline v3 guide_mixture_sample(const float *__restrict__ m, float u_lobe, float u1, float u2) {
    int j = 0;
    float acc = m[0];
    while (j < 7 && u_lobe >= acc) {
        ++j;
        acc += m[j];
    }
    const float k = m[32 + j];
    const v3 mu = mk(m[8 + 3 * j], m[9 + 3 * j], m[10 + 3 * j]);
    float wz = 1.f + logf(u1 + (1.f - u1) * expf(-2.f * k)) / k;
    wz = fminf(fmaxf(wz, -1.f), 1.f);
    const float st = sqrtf(fmaxf(0.f, 1.f - wz * wz));
    float sp, cp;
    sincospif(2.f * u2, &sp, &cp);
    v3 s, t;
    coordinate_system(mu, &s, &t);
    s = normalize(s);
    t = normalize(cross(mu, s));
    const v3 w = mk(wz * mu.x + st * (cp * s.x + sp * t.x), wz * mu.y + st * (cp * s.y + sp * t.y),
                    wz * mu.z + st * (cp * s.z + sp * t.z));
    return normalize(w);
}

}  // namespace fl
