// Learned path guiding: training kernels (forward + backward + Adam on the tensor cores),
// the guided wave loop and the fl_guide_* entry points of include/filianore_gpu.h.
//
// Training minimises the radiance-weighted KL divergence between the normalised incident
// radiance (times the cosine) and the guide's mixture q, estimated from the renderer's own
// samples: loss = mean_i w_i * -log q(w_i | x_i), w_i = L_i cos_i / p_i / mean(w)
// (p_i: the density the direction was sampled with). During rendering the minibatches are
// drawn from the wave's records with probability proportional to w_i (stratified, by
// inverse CDF over a prefix sum) and weighted 1: the same expected gradient, but the rare
// records that carry most of the weight (caustic paths) are in every batch instead of in
// one batch out of many. fl_guide_gradient evaluates the weighted loss over the given
// records in order instead. One CTA of 8 warps takes 128 records:
// each warp runs the forward pass of 16 records with the activations kept in shared
// memory, the head gradient is computed per record in FP32, and the backward pass goes
// layer by layer, the weight gradients dW^T = A^T dZ as tensor-core products over the
// CTA's 128 records (ldmatrix.trans operands), added to an FP32 gradient with one atomic
// per element and CTA. Per-record head gradients are scaled by kLossScale before the FP16
// backward pass; Adam divides it out.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <mutex>
#include <vector>

#include <cub/device/device_scan.cuh>

#include "fl_render.cuh"

namespace fl {

CamDev camera_basis_of(const fl_camera &c);

constexpr int kTrainWarps = 8;
constexpr int kTrainRows = 16 * kTrainWarps;  // 128 records per CTA
constexpr float kLossScale = 1.f / 64.f;
constexpr float kWeightClamp = 4096.f;        // normalised record weights are clamped here
constexpr size_t kTrainSmem = (size_t)kSmWHalves * 2 + (size_t)kTrainRows * kLdIn * 2 +
                              4 * (size_t)kTrainRows * kLdH * 2 + 2 * (size_t)kTrainRows * kLdH * 2 +
                              (size_t)kTrainRows * kHeadLd * 4;

struct TrainArgs {
    const __half *w;
    float *grad;               // FL_GUIDE_PARAMS, FP32, scaled by kLossScale
    const float *rec;
    const uint32_t *rec_count;
    uint32_t rec_cap;
    uint32_t batch_begin, batch_size;
    const float *wstat;        // [0] sum of record weights, [1] number of records
    float *loss;               // [0] += sum of weighted losses of the batch
    float bmin[3], binv[3];
    const float *cdf;          // resampling: inclusive prefix sum of the record weights (null: in order)
    uint32_t seed;             // resampling: stratification jitter of this batch
    int learned;               // fit the selection probability with the mixture (loss -log f)
    int *err;                  // counts tensor-core products that did not complete (nullable)
};

__device__ inline float hash01(uint32_t a, uint32_t b) {
    uint32_t h = a * 0x9e3779b1u ^ (b + 0x7f4a7c15u) * 0x85ebca77u;
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    h *= 0x846ca68bu;
    h ^= h >> 16;
    return (float)(h >> 8) * (1.f / 16777216.f);
}

// record weight L cos / p (0 when the record cannot be learnt from)
__device__ inline float record_weight(const float *R) {
    const float c = R[3] * R[7] + R[4] * R[8] + R[5] * R[9];
    const float p = R[10], li = R[11];
    if (!(p > 0.f) || !(li > 0.f) || !(c > 0.f) || !isfinite(li)) return 0.f;
    const float w = li * c / p;
    return isfinite(w) ? w : 0.f;
}

// d(loss)/d(head) for one point (FP32); returns the loss. Without a learned selection the
// loss is -log q(w). With it (learned = true) the loss is -log f(w) of the one-sample MIS
// density f = c q + (1 - c) pb, c = guide_select(h[40]) and pb the BSDF's density of w: the
// mixture and c are fitted together, so c grows where the guide explains the incident
// radiance better than the BSDF does and shrinks where it does not.
__device__ inline float guide_head_grad(const float *h, v3 w, float *dh, float pb, bool learned) {
    float mx = h[0];
#pragma unroll
    for (int j = 1; j < 8; ++j) mx = fmaxf(mx, h[j]);
    float se = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) se += expf(h[j] - mx);
    const float lse_pi = mx + logf(se);
    float lq[8], mu[8][3], len[8], kap[8], dp[8];
    float lmax = -INFINITY;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const float x = h[8 + 3 * j], y = h[9 + 3 * j], z = h[10 + 3 * j];
        len[j] = fmaxf(sqrtf(x * x + y * y + z * z), 1e-6f);
        mu[j][0] = x / len[j];
        mu[j][1] = y / len[j];
        mu[j][2] = z / len[j];
        kap[j] = guide_kappa(h[32 + j]);
        dp[j] = mu[j][0] * w.x + mu[j][1] * w.y + mu[j][2] * w.z;
        lq[j] = (h[j] - lse_pi) + vmf_log_norm(kap[j]) + kap[j] * (dp[j] - 1.f);
        lmax = fmaxf(lmax, lq[j]);
    }
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += expf(lq[j] - lmax);
    const float lse = lmax + logf(s);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const float r = expf(lq[j] - lse);
        const float pi = expf(h[j] - lse_pi);
        dh[j] = -(r - pi);
        // mean direction through the normalisation: (I - mu mu^T) / |v| * d/dmu
        const float gx = -r * kap[j] * w.x, gy = -r * kap[j] * w.y, gz = -r * kap[j] * w.z;
        const float mg = mu[j][0] * gx + mu[j][1] * gy + mu[j][2] * gz;
        dh[8 + 3 * j] = (gx - mu[j][0] * mg) / len[j];
        dh[9 + 3 * j] = (gy - mu[j][1] * mg) / len[j];
        dh[10 + 3 * j] = (gz - mu[j][2] * mg) / len[j];
        // concentration: d log q_j / d log kappa = 1 - 2 kappa / expm1(2 kappa) + kappa (mu.w - 1),
        // d log kappa / ds = (max - min) sigmoid' (s - shift)
        const float sg = guide_sigmoid(h[32 + j]);
        const float k = kap[j];
        dh[32 + j] = -r * (1.f - 2.f * k / expm1f(2.f * k) + k * (dp[j] - 1.f)) *
                     (kLogKappaMax - kLogKappaMin) * sg * (1.f - sg);
    }
    dh[40] = 0.f;
    if (!learned) return -lse;
    // f = c q + (1 - c) pb in logs: d(-log f)/dh_k = (c q / f) d(-log q)/dh_k for the mixture
    // outputs, and d(-log f)/ds = -(q - pb) / f dc/ds for the selection logit s = h[40]
    const float sg = 1.f / (1.f + expf(-h[40]));
    const float c = kSelectMin + (kSelectMax - kSelectMin) * sg;
    const float a = logf(c) + lse;                                   // log(c q)
    const float b = pb > 0.f ? logf((1.f - c) * pb) : -INFINITY;     // log((1 - c) pb)
    const float m = fmaxf(a, b);
    const float lf = m + logf(expf(a - m) + expf(b - m));            // log f
    const float rq = expf(a - lf);                                   // c q / f
#pragma unroll
    for (int k = 0; k < 40; ++k) dh[k] *= rq;
    dh[40] = -(expf(lse - lf) - pb * expf(-lf)) * (kSelectMax - kSelectMin) * sg * (1.f - sg);
    return -lf;
}

// the Lambert BSDF's density of a record's direction (normal facing the viewer): cos / pi
__device__ inline float record_bsdf_pdf(const float *R) {
    const float c = R[3] * R[7] + R[4] * R[8] + R[5] * R[9];
    return c > 0.f ? c * kInvPi : 0.f;
}

// dW^T (in x out) += S^T D over the CTA's 128 rows: S rows = records (ld ldS, Mt 16-col
// tiles of inputs), D rows = records (ld kLdH, Nt 8-col tiles of outputs). Tiles are
// spread over the warps; each ends with one atomic per gradient element.
__device__ inline void guide_dw(const __half *S, int ldS, int Mt, const __half *D, int Nt, float *grad, int in_dim,
                                int out_valid) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int tile = warp; tile < Mt * Nt; tile += kTrainWarps) {
        const int m0 = (tile / Nt) * 16, n0 = (tile % Nt) * 8;
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int k0 = 0; k0 < kTrainRows; k0 += 16) {
            uint32_t a[4], b[2];
            ldsm_x4_t(a, S + (k0 + (lane & 7) + ((lane >> 4) << 3)) * ldS + m0 + ((lane >> 3) & 1) * 8);
            ldsm_x2_t(b, D + (k0 + (lane & 15)) * kLdH + n0);
            mma16816(acc, a, b[0], b[1]);
        }
        const int o = n0 + 2 * t, i = m0 + g;
        if (o < out_valid) {
            atomicAdd(&grad[o * in_dim + i], acc[0]);
            atomicAdd(&grad[o * in_dim + i + 8], acc[2]);
        }
        if (o + 1 < out_valid) {
            atomicAdd(&grad[(o + 1) * in_dim + i], acc[1]);
            atomicAdd(&grad[(o + 1) * in_dim + i + 8], acc[3]);
        }
    }
}

// One warp, its 16 rows: Dnext = (Dcur W) * [Act > 0], Dcur with Kt 16-col tiles of the
// layer's outputs, W the layer's [out][in] weights in shared memory (in = 64).
__device__ inline void guide_back_warp(const __half *Dcur, int Kt, const __half *W, const __half *Act, __half *Dnext) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    uint32_t a[4][4];
#pragma unroll
    for (int kt = 0; kt < 4; ++kt)
        if (kt < Kt) ldsm_x4(a[kt], Dcur + (lane & 15) * kLdH + kt * 16 + (lane >> 4) * 8);
    float acc[8][4];
#pragma unroll
    for (int n = 0; n < 8; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
#pragma unroll
    for (int np = 0; np < 4; ++np)
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
            if (kt >= Kt) continue;
            uint32_t b[4];
            ldsm_x4_t(b, W + (kt * 16 + (lane & 15)) * kLdH + np * 16 + (lane >> 4) * 8);
            mma16816(acc[2 * np], a[kt], b[0], b[1]);
            mma16816(acc[2 * np + 1], a[kt], b[2], b[3]);
        }
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        const int col = n * 8 + 2 * t;
        const float2 a0 = __half22float2(*reinterpret_cast<const __half2 *>(Act + g * kLdH + col));
        const float2 a1 = __half22float2(*reinterpret_cast<const __half2 *>(Act + (g + 8) * kLdH + col));
        *reinterpret_cast<uint32_t *>(Dnext + g * kLdH + col) =
            pack_h2(a0.x > 0.f ? acc[n][0] : 0.f, a0.y > 0.f ? acc[n][1] : 0.f, false);
        *reinterpret_cast<uint32_t *>(Dnext + (g + 8) * kLdH + col) =
            pack_h2(a1.x > 0.f ? acc[n][2] : 0.f, a1.y > 0.f ? acc[n][3] : 0.f, false);
    }
}

__global__ void __launch_bounds__(256, 1) k_guide_train(TrainArgs T) {
    extern __shared__ __align__(16) unsigned char tsm[];
    const uint32_t n_total = min(*T.rec_count, T.rec_cap);
    const uint32_t begin = T.cdf ? blockIdx.x * kTrainRows : T.batch_begin + blockIdx.x * kTrainRows;
    const uint32_t end = T.cdf ? (n_total ? T.batch_size : 0u) : min(T.batch_begin + T.batch_size, n_total);
    if (begin >= end || !(T.wstat[0] > 0.f)) return;
    const float total = T.cdf ? T.cdf[n_total - 1] : 0.f;
    if (T.cdf && !(total > 0.f)) return;
    __half *sw = reinterpret_cast<__half *>(tsm);
    __half *X = sw + kSmWHalves;
    __half *Act = X + kTrainRows * kLdIn;
    __half *DzA = Act + 4 * kTrainRows * kLdH;
    __half *DzB = DzA + kTrainRows * kLdH;
    float *Head = reinterpret_cast<float *>(DzB + kTrainRows * kLdH);
    const int actS = kTrainRows * kLdH;
    guide_stage_weights(sw, T.w);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r0 = warp * 16;
    uint32_t i = begin + r0 + (lane & 15);
    const bool valid = i < end;
    if (T.cdf && valid) {
        // stratified draw proportional to the record weights: first record whose
        // inclusive prefix sum exceeds u
        const float u = ((float)i + hash01(T.seed, i)) / (float)T.batch_size * total;
        uint32_t lo = 0, hi = n_total - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (T.cdf[mid] > u) hi = mid;
            else lo = mid + 1;
        }
        i = lo;
    }
    const float *R = T.rec + (size_t)(valid ? i : 0) * kRecFloats;
    // features of this warp's 16 records (two lanes per record)
    {
        __half *row = X + (r0 + (lane & 15)) * kLdIn;
        if (valid) {
            guide_encode_record(R, T.bmin, T.binv, lane >> 4, row);
        } else {
            uint4 *d = reinterpret_cast<uint4 *>(row + 40 * (lane >> 4));
#pragma unroll
            for (int k = 0; k < 5; ++k) d[k] = make_uint4(0, 0, 0, 0);
        }
    }
    __syncwarp();
    guide_forward_warp(sw, X + r0 * kLdIn, Act + r0 * kLdH, actS, Head + r0 * kHeadLd);
    __syncwarp();
    // head gradient of the weighted loss, one lane per record, scaled into FP16 range
    if (lane < 16) {
        float dh[kGuideOut + 1];  // even count: written as FP16 pairs
#pragma unroll
        for (int k = 0; k <= kGuideOut; ++k) dh[k] = 0.f;
        float loss = 0.f;
        if (valid) {
            const float wmean = T.wstat[0] / fmaxf(T.wstat[1], 1.f);
            const float wr = record_weight(R);
            const float wn = T.cdf ? (wr > 0.f ? 1.f : 0.f) : fminf(wr / wmean, kWeightClamp);
            if (wn > 0.f) {
                const float nl = guide_head_grad(Head + (r0 + lane) * kHeadLd, mk(R[7], R[8], R[9]), dh,
                                                 record_bsdf_pdf(R), T.learned != 0);
                loss = wn * nl;
#pragma unroll
                for (int k = 0; k < kGuideOut; ++k) dh[k] *= wn * kLossScale;
            }
        }
        __half *drow = DzA + (r0 + lane) * kLdH;
#pragma unroll
        for (int k = 0; k < kGuideOut; k += 2) *reinterpret_cast<uint32_t *>(drow + k) = pack_h2(dh[k], dh[k + 1], false);
#pragma unroll
        for (int k = kGuideOut + 1; k < kHeadRowsPad; k += 2) *reinterpret_cast<uint32_t *>(drow + k) = 0u;
        // batch loss (one atomic per warp)
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) loss += __shfl_down_sync(0x0000ffffu, loss, o, 16);
        if (lane == 0 && loss != 0.f) atomicAdd(T.loss, loss);
    }
    __syncthreads();
    // head: dW^T = Act4^T dZ, then dZ of hidden layer 4
    guide_dw(Act + 3 * actS, kLdH, 4, DzA, 6, T.grad + guide_woff(4), 64, kGuideOut);
    guide_back_warp(DzA + r0 * kLdH, 3, sw + guide_sm_off(4), Act + 3 * actS + r0 * kLdH, DzB + r0 * kLdH);
    __syncthreads();
    guide_dw(Act + 2 * actS, kLdH, 4, DzB, 8, T.grad + guide_woff(3), 64, 64);
    guide_back_warp(DzB + r0 * kLdH, 4, sw + guide_sm_off(3), Act + 2 * actS + r0 * kLdH, DzA + r0 * kLdH);
    __syncthreads();
    guide_dw(Act + 1 * actS, kLdH, 4, DzA, 8, T.grad + guide_woff(2), 64, 64);
    guide_back_warp(DzA + r0 * kLdH, 4, sw + guide_sm_off(2), Act + 1 * actS + r0 * kLdH, DzB + r0 * kLdH);
    __syncthreads();
    guide_dw(Act, kLdH, 4, DzB, 8, T.grad + guide_woff(1), 64, 64);
    guide_back_warp(DzB + r0 * kLdH, 4, sw + guide_sm_off(1), Act + r0 * kLdH, DzA + r0 * kLdH);
    __syncthreads();
    guide_dw(X, kLdIn, 5, DzA, 8, T.grad + guide_woff(0), 80, 64);
}


// ----------------------------------------------------------------- tcgen05 training kernel
//
// The same step as k_guide_train with its nine 128-row products on the 5th-generation tensor
// cores: the forward layers (X W0^T, ..., A4 Wh^T) and the backward products dZ W of the
// layers past the first run as tcgen05.mma (M = 128 records, N = 64 or 48, K = 16 per
// instruction) from shared memory into a 64-column TMEM accumulator, issued by one thread
// and completed through an mbarrier; the epilogues read the accumulator back with
// tcgen05.ld (each warp its 32 TMEM lanes, a warp pair splitting the columns), apply ReLU or
// the ReLU mask and write FP16 operands for the next product. The weight gradients (64 or 80
// input rows, summed over the records) stay on mma.sync and overlap the tensor-core product
// of the same level. Operands use the canonical K-major layout without swizzle: 8-row x 16-byte
// core matrices, the next one along K 128 bytes on, the next 8 rows K x 16 bytes on.

// element (r, k) of an R x K operand in the canonical layout, in halves
__device__ __forceinline__ int tc_canon(int r, int k, int K) { return (r >> 3) * (K * 8) + (k >> 3) * 64 + (r & 7) * 8 + (k & 7); }
__device__ __forceinline__ uint64_t tc_sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    // start, leading and stride byte offsets, descriptor version 1, no swizzle
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// FP32 accumulator, FP16 A and B, A K-major, B K-major or (b_mn) MN-major, M = 128
__host__ __device__ constexpr uint32_t tc_idesc(int n, bool b_mn) {
    return (1u << 4) | (b_mn ? 1u << 16 : 0u) | ((uint32_t)(n >> 3) << 17) | ((128u >> 4) << 24);
}

// D (TMEM) = A (128 x K, K-major) * B, one thread issues, the mbarrier receives the commit.
// B is W (N rows x K, K-major) for the forward products, or, for the backward ones, the same
// forward copy of W read as an MN-major K x N operand (its 8-row groups along K 16 * Kw
// bytes apart, Kw its own row length), which makes dZ W without a transposed copy.
__device__ inline void tc_gemm(uint32_t tmem, const __half *A, const __half *B, int K, int n, bool b_mn, int Kw,
                               uint64_t *mbar) {
    const uint32_t a0 = smem_u32(A), b0 = smem_u32(B), sbo = (uint32_t)K * 16u, idesc = tc_idesc(n, b_mn);
    const uint32_t b_lbo = b_mn ? (uint32_t)Kw * 16u : 128u, b_sbo = b_mn ? 128u : sbo;
    const uint32_t b_step = b_mn ? 2u * (uint32_t)Kw * 16u : 256u;  // bytes per 16 of K
    for (int s = 0; s < K / 16; ++s) {
        const uint64_t da = tc_sdesc(a0 + 256u * s, 128u, sbo), db = tc_sdesc(b0 + b_step * s, b_lbo, b_sbo);
        const uint32_t acc = s > 0 ? 1u : 0u;
        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                     "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                     "l"(da), "l"(db), "r"(idesc), "r"(acc));
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}
// every writer of an operand calls this before the barrier that precedes the product
__device__ __forceinline__ void tc_operands_written() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
// bounded wait for the product's commit (phase `ph`); false if it did not arrive
__device__ inline bool tc_wait(uint64_t *mbar, uint32_t ph) {
    uint32_t done = 0;
    for (int it = 0; it < (1 << 24) && !done; ++it)
        asm volatile("{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\tselp.b32 %0, 1, 0, P1;\n\t}\n"
                     : "=r"(done)
                     : "r"(smem_u32(mbar)), "r"(ph));
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    return done != 0;
}
// 16 / 32 consecutive accumulator columns of this thread's TMEM lane
__device__ inline void tc_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ inline void tc_ld32(uint32_t taddr, float v[32]) {
    tc_ld16(taddr, v);
    tc_ld16(taddr + 16u, v + 16);
}
// 32 accumulator columns of row m (from c0) through ReLU, or through the mask of the
// activations `mask` (same layout), into the 64-wide canonical operand `out`
__device__ inline void tc_store_row32(const float v[32], int m, int c0, __half *out, const __half *mask) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint32_t h[4];
        const int c = c0 + 8 * q;
        uint4 mk4 = make_uint4(0, 0, 0, 0);
        if (mask) mk4 = *reinterpret_cast<const uint4 *>(mask + tc_canon(m, c, 64));
        const uint32_t mw[4] = {mk4.x, mk4.y, mk4.z, mk4.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float a = v[8 * q + 2 * j], b = v[8 * q + 2 * j + 1];
            if (mask) {
                const float2 am = __half22float2(*reinterpret_cast<const __half2 *>(&mw[j]));
                a = am.x > 0.f ? a : 0.f;
                b = am.y > 0.f ? b : 0.f;
            }
            h[j] = pack_h2(a, b, mask == nullptr);
        }
        *reinterpret_cast<uint4 *>(out + tc_canon(m, c, 64)) = make_uint4(h[0], h[1], h[2], h[3]);
    }
}
// weight gradient of one layer, as guide_dw, from canonical operands: S (records x in, Ks
// wide) and D (records x out, Kd wide)
__device__ inline void tc_dw(const __half *S, int Ks, int Mt, const __half *D, int Kd, int Nt, float *grad, int in_dim,
                             int out_valid) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int tile = warp; tile < Mt * Nt; tile += kTrainWarps) {
        const int m0 = (tile / Nt) * 16, n0 = (tile % Nt) * 8;
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int k0 = 0; k0 < kTrainRows; k0 += 16) {
            uint32_t a[4], b[2];
            ldsm_x4_t(a, S + tc_canon(k0 + (lane & 7) + ((lane >> 4) << 3), m0 + ((lane >> 3) & 1) * 8, Ks));
            ldsm_x2_t(b, D + tc_canon(k0 + (lane & 15), n0, Kd));
            mma16816(acc, a, b[0], b[1]);
        }
        const int o = n0 + 2 * t, i = m0 + g;
        if (o < out_valid) {
            atomicAdd(&grad[o * in_dim + i], acc[0]);
            atomicAdd(&grad[o * in_dim + i + 8], acc[2]);
        }
        if (o + 1 < out_valid) {
            atomicAdd(&grad[(o + 1) * in_dim + i], acc[1]);
            atomicAdd(&grad[(o + 1) * in_dim + i + 8], acc[3]);
        }
    }
}

// shared memory of k_guide_train_tc (byte offsets)
constexpr int kTcW0 = 0, kTcW1 = 10240, kTcWh = 34816, kTcX = 40960, kTcAct = 61440, kTcDzA = 126976,
              kTcDzB = 143360, kTcMisc = 159744;
constexpr size_t kTrainSmemTc = (size_t)kTcMisc + 1024;

__global__ void __launch_bounds__(256, 1) k_guide_train_tc(TrainArgs T) {
    extern __shared__ __align__(16) unsigned char tsm[];  // every operand offset is a multiple of 1024
    const uint32_t n_total = min(*T.rec_count, T.rec_cap);
    const uint32_t begin = T.cdf ? blockIdx.x * kTrainRows : T.batch_begin + blockIdx.x * kTrainRows;
    const uint32_t end = T.cdf ? (n_total ? T.batch_size : 0u) : min(T.batch_begin + T.batch_size, n_total);
    if (begin >= end || !(T.wstat[0] > 0.f)) return;
    const float total = T.cdf ? T.cdf[n_total - 1] : 0.f;
    if (T.cdf && !(total > 0.f)) return;
    __half *Wc[4] = {reinterpret_cast<__half *>(tsm + kTcW0), reinterpret_cast<__half *>(tsm + kTcW1),
                     reinterpret_cast<__half *>(tsm + kTcW1 + 8192), reinterpret_cast<__half *>(tsm + kTcW1 + 16384)};
    __half *Wch = reinterpret_cast<__half *>(tsm + kTcWh);
    __half *Xc = reinterpret_cast<__half *>(tsm + kTcX);
    __half *Act[4] = {reinterpret_cast<__half *>(tsm + kTcAct), reinterpret_cast<__half *>(tsm + kTcAct + 16384),
                      reinterpret_cast<__half *>(tsm + kTcAct + 32768), reinterpret_cast<__half *>(tsm + kTcAct + 49152)};
    __half *DzA = reinterpret_cast<__half *>(tsm + kTcDzA);
    __half *DzB = reinterpret_cast<__half *>(tsm + kTcDzB);
    uint64_t *mbar = reinterpret_cast<uint64_t *>(tsm + kTcMisc);
    uint32_t *taddr_s = reinterpret_cast<uint32_t *>(tsm + kTcMisc + 8);
    uint32_t *rid = reinterpret_cast<uint32_t *>(tsm + kTcMisc + 64);  // record of each row (~0u: none)
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // TMEM: 64 columns for the accumulator (warp 0 allocates and frees)
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(taddr_s)), "r"(64));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::);
    }
    // weights W_l [out][in], canonical K-major (rows = outputs), 8 halves per copy; the head's
    // rows 41..47 are zero
    for (int l = 0; l < kGuideLayers; ++l) {
        const int in = guide_in(l), out = guide_out(l), rows = l == 4 ? kHeadRowsPad : out, per_row = in / 8;
        const __half *w = T.w + guide_woff(l);
        __half *F = l == 4 ? Wch : Wc[l];
        for (int e = tid; e < rows * per_row; e += blockDim.x) {
            const int o = e / per_row, c8 = e % per_row;
            const uint4 v = o < out ? *reinterpret_cast<const uint4 *>(w + o * in + 8 * c8) : make_uint4(0, 0, 0, 0);
            *reinterpret_cast<uint4 *>(F + tc_canon(o, 8 * c8, in)) = v;
        }
    }
    // the rows' records (stratified resampling as k_guide_train), then their features
    if (tid < kTrainRows) {
        uint32_t i = begin + tid;
        const bool valid = i < end;
        if (T.cdf && valid) {
            const float u = ((float)i + hash01(T.seed, i)) / (float)T.batch_size * total;
            uint32_t lo = 0, hi = n_total - 1;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (T.cdf[mid] > u) hi = mid;
                else lo = mid + 1;
            }
            i = lo;
        }
        rid[tid] = valid ? i : ~0u;
    }
    __syncthreads();
    {
        const int m = tid >> 1, part = tid & 1;
        uint32_t h[20];
        if (rid[m] != ~0u) {
            const float *R = T.rec + (size_t)rid[m] * kRecFloats;
            float pn[3];
            guide_normalise(T.bmin, T.binv, mk(R[0], R[1], R[2]), pn);
            const float nf[3] = {R[3], R[4], R[5]};
            guide_encode_pairs(pn, nf, (R[6] - 380.f) * (1.f / 340.f), part, h);
        } else {
#pragma unroll
            for (int k = 0; k < 20; ++k) h[k] = 0u;
        }
#pragma unroll
        for (int q = 0; q < 5; ++q)
            *reinterpret_cast<uint4 *>(Xc + tc_canon(m, 40 * part + 8 * q, kGuideIn)) =
                make_uint4(h[4 * q], h[4 * q + 1], h[4 * q + 2], h[4 * q + 3]);
    }
    tc_operands_written();
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *taddr_s;
    const int q4 = warp & 3, chalf = warp >> 2;       // TMEM lane quarter and column half of this warp
    const int row = 32 * q4 + lane;                     // the accumulator row (record) this thread reads
    const uint32_t tl = tmem + ((uint32_t)(32 * q4) << 16);
    uint32_t ph = 0;
    bool ok = true;
    // forward: 4 hidden layers (ReLU) and the head
    for (int l = 0; l < 5; ++l) {
        if (tid == 0) tc_gemm(tmem, l == 0 ? Xc : Act[l - 1], l == 4 ? Wch : Wc[l], l == 0 ? kGuideIn : 64,
                              l == 4 ? kHeadRowsPad : 64, false, 0, mbar);
        ok = tc_wait(mbar, ph) && ok;
        ph ^= 1u;
        if (l < 4) {
            float v[32];
            tc_ld32(tl + 32u * chalf, v);
            tc_store_row32(v, row, 32 * chalf, Act[l], nullptr);
        } else if (warp < 4) {
            // head gradient of the weighted loss, one thread per record, scaled into FP16 range
            float hrow[kHeadRowsPad];
            tc_ld32(tl, hrow);
            tc_ld16(tl + 32u, hrow + 32);
            float dh[kHeadRowsPad];
#pragma unroll
            for (int k = 0; k < kHeadRowsPad; ++k) dh[k] = 0.f;
            float loss = 0.f;
            if (rid[row] != ~0u) {
                const float *R = T.rec + (size_t)rid[row] * kRecFloats;
                const float wmean = T.wstat[0] / fmaxf(T.wstat[1], 1.f);
                const float wr = record_weight(R);
                const float wn = T.cdf ? (wr > 0.f ? 1.f : 0.f) : fminf(wr / wmean, kWeightClamp);
                if (wn > 0.f) {
                    const float nl = guide_head_grad(hrow, mk(R[7], R[8], R[9]), dh, record_bsdf_pdf(R), T.learned != 0);
                    loss = wn * nl;
#pragma unroll
                    for (int k = 0; k < kGuideOut; ++k) dh[k] *= wn * kLossScale;
                }
            }
#pragma unroll
            for (int q = 0; q < kHeadRowsPad / 8; ++q) {
                uint32_t h[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int k = 8 * q + 2 * j;
                    h[j] = k < kGuideOut + 1 ? pack_h2(dh[k], dh[k + 1], false) : 0u;
                }
                *reinterpret_cast<uint4 *>(DzA + tc_canon(row, 8 * q, kHeadRowsPad)) = make_uint4(h[0], h[1], h[2], h[3]);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) loss += __shfl_down_sync(0xffffffffu, loss, o);
            if (lane == 0 && loss != 0.f) atomicAdd(T.loss, loss);
        }
        tc_operands_written();
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    // backward: per level, the product dZ W on the tensor cores (issued first) and the
    // weight gradient on mma.sync meanwhile; then the masked dZ of the layer below
    const __half *dz = DzA;
    __half *dzn = DzB;
    for (int l = 4; l >= 1; --l) {
        const int kz = l == 4 ? kHeadRowsPad : 64;  // width of this level's dZ
        if (tid == 0) tc_gemm(tmem, dz, l == 4 ? Wch : Wc[l], kz, 64, true, 64, mbar);
        tc_dw(Act[l - 1], 64, 4, dz, kz, l == 4 ? 6 : 8, T.grad + guide_woff(l), 64, guide_out(l));
        ok = tc_wait(mbar, ph) && ok;
        ph ^= 1u;
        float v[32];
        tc_ld32(tl + 32u * chalf, v);
        tc_store_row32(v, row, 32 * chalf, dzn, Act[l - 1]);
        tc_operands_written();
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const __half *t2 = dzn;
        dzn = const_cast<__half *>(dz);
        dz = t2;
    }
    tc_dw(Xc, kGuideIn, 5, dz, 64, 8, T.grad + guide_woff(0), kGuideIn, 64);
    if (!ok && tid == 0 && T.err) atomicAdd(T.err, 1);
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64));
}

// one training step's forward + backward over the records of T, on the kernel the guide's
// configuration names (fl_guide_config.train_kernel)
static void launch_train(const TrainArgs &T, uint32_t blocks, cudaStream_t st, int kernel) {
    if (kernel == FL_GUIDE_TRAIN_TCGEN05) k_guide_train_tc<<<blocks, 32 * kTrainWarps, kTrainSmemTc, st>>>(T);
    else k_guide_train<<<blocks, 32 * kTrainWarps, kTrainSmem, st>>>(T);
}

// sum and count of the record weights of this wave (and the weights themselves, when asked)
__global__ void k_guide_stats(const float *rec, const uint32_t *rec_count, uint32_t rec_cap, float *wstat,
                              float *weights) {
    const uint32_t n = min(*rec_count, rec_cap);
    float s = 0.f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float w = record_weight(rec + (size_t)i * kRecFloats);
        if (weights) weights[i] = w;
        s += w;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && s != 0.f) atomicAdd(&wstat[0], s);
    if (blockIdx.x == 0 && threadIdx.x == 0) wstat[1] = (float)n;
}

struct AdamArgs {
    float *w32, *m, *v, *grad;
    __half *w16;
    float *wavg;       // weight average (null: off), its decay and bias correction
    __half *w16avg;
    float beta, bc_avg;
    const uint32_t *rec_count;
    uint32_t rec_cap, batch_begin, batch_size;
    const float *wstat;
    float lr, bc1, bc2;  // step size and the bias corrections 1 - beta^t
    int resampled;       // batches drawn by weight: always batch_size records
};

// Adam (beta1 0.9, beta2 0.999, eps 1e-8) on the mean gradient of the batch; clears the gradient.
__global__ void k_guide_adam(AdamArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kGuideParams) return;
    const uint32_t n = min(*a.rec_count, a.rec_cap);
    const bool step = (a.resampled ? n > 0 : a.batch_begin < n) && a.wstat[0] > 0.f;
    if (step) {
        const float cnt = a.resampled ? (float)a.batch_size : (float)min(a.batch_size, n - a.batch_begin);
        float g = a.grad[i] / (kLossScale * cnt);
        if (!isfinite(g)) g = 0.f;
        const float m = 0.9f * a.m[i] + 0.1f * g;
        const float v = 0.999f * a.v[i] + 0.001f * g * g;
        a.m[i] = m;
        a.v[i] = v;
        float w = a.w32[i] - a.lr * (m / a.bc1) / (sqrtf(v / a.bc2) + 1e-8f);
        w = fminf(fmaxf(w, -60000.f), 60000.f);
        a.w32[i] = w;
        a.w16[i] = __float2half_rn(w);
        if (a.wavg) {
            const float e = a.beta * a.wavg[i] + (1.f - a.beta) * w;
            a.wavg[i] = e;
            a.w16avg[i] = __float2half_rn(e / a.bc_avg);
        }
    }
    a.grad[i] = 0.f;
}

// mixture parameters for host-given records (fl_guide_eval)
__global__ void __launch_bounds__(32 * kInferWarps) k_guide_eval(const __half *w, const float *rec, uint32_t n, float b0,
                                                                 float b1, float b2, float i0, float i1, float i2,
                                                                 float *out) {
    extern __shared__ __align__(16) unsigned char gsm[];
    __half *sw = reinterpret_cast<__half *>(gsm);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __half *X = reinterpret_cast<__half *>(gsm + kSmWHalves * 2) + warp * 16 * kLdIn;
    float *head = reinterpret_cast<float *>(X);
    guide_stage_weights(sw, w);
    const float bmin[3] = {b0, b1, b2}, binv[3] = {i0, i1, i2};
    for (uint32_t chunk = blockIdx.x * kInferWarps + warp; chunk * 16 < n; chunk += gridDim.x * kInferWarps) {
        const uint32_t i = chunk * 16 + (lane & 15);
        __half *row = X + (lane & 15) * kLdIn;
        if (i < n) {
            guide_encode_record(rec + (size_t)i * kRecFloats, bmin, binv, lane >> 4, row);
        } else {
            uint4 *d = reinterpret_cast<uint4 *>(row + 40 * (lane >> 4));
#pragma unroll
            for (int k = 0; k < 5; ++k) d[k] = make_uint4(0, 0, 0, 0);
        }
        __syncwarp();
        guide_forward_warp(sw, X, nullptr, 0, head);
        __syncwarp();
        if (i < n && lane < 16) guide_mixture(head + lane * kHeadLd, out + (size_t)i * kGuideOut);
        __syncwarp();
    }
}

// ------------------------------------------------------------------------------ host side

struct Guide {
    Context *ctx = nullptr;
    fl_guide_config cfg{};
    void *mem = nullptr;  // weights, Adam state, gradient, statistics
    __half *w16 = nullptr;
    float *w32 = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr, *wstat = nullptr, *loss = nullptr;
    // rendering weights: w16, or with weight_average > 0 the FP16 copy of the bias-corrected
    // moving average wavg of the Adam iterates (avg_steps of them since the last upload)
    float *wavg = nullptr;
    __half *w16avg = nullptr;
    int64_t avg_steps = 0;
    const __half *render_weights() const { return cfg.weight_average > 0.f ? w16avg : w16; }
    uint32_t *rec_count = nullptr;
    float *rec = nullptr;
    float *mix = nullptr;
    uint32_t *rec_idx = nullptr;
    size_t slot_cap = 0;
    float *wts = nullptr, *cdf = nullptr;  // per-record weights and their prefix sum
    void *scan_tmp = nullptr;
    size_t scan_bytes = 0;
    uint32_t *h_count = nullptr;  // pinned
    float *h_loss = nullptr;      // pinned
    int64_t steps = 0;
    float last_loss = 0.f;
};

// He-uniform hidden layers, Xavier-uniform head, from a PCG32 stream
static void guide_init_weights(uint64_t seed, std::vector<float> &w) {
    w.assign(kGuideParams, 0.f);
    Pcg32 r;
    r.seed(seed, 0x9e3779b97f4a7c15ull);
    for (int l = 0; l < kGuideLayers; ++l) {
        const int in = guide_in(l), out = guide_out(l);
        const float lim = l < 4 ? sqrtf(6.f / (float)in) : sqrtf(6.f / (float)(in + out));
        for (int k = 0; k < in * out; ++k) w[guide_woff(l) + k] = (2.f * r.nextf() - 1.f) * lim;
    }
}

static fl_status guide_upload_weights(Guide *G, const std::vector<float> &w) {
    Context *ctx = G->ctx;
    std::vector<__half> h(kGuideParams);
    for (int i = 0; i < kGuideParams; ++i) h[i] = __float2half_rn(w[i]);
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(G->w32, w.data(), sizeof(float) * kGuideParams, cudaMemcpyHostToDevice, ctx->stream));
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(G->w16, h.data(), sizeof(__half) * kGuideParams, cudaMemcpyHostToDevice, ctx->stream));
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(G->w16avg, h.data(), sizeof(__half) * kGuideParams, cudaMemcpyHostToDevice,
                                     ctx->stream));
    FL_CUDA_TRY(ctx, cudaMemsetAsync(G->wavg, 0, sizeof(float) * kGuideParams, ctx->stream));
    G->avg_steps = 0;
    FL_CUDA_TRY(ctx, cudaMemsetAsync(G->m, 0, sizeof(float) * kGuideParams, ctx->stream));
    FL_CUDA_TRY(ctx, cudaMemsetAsync(G->v, 0, sizeof(float) * kGuideParams, ctx->stream));
    FL_CUDA_TRY(ctx, cudaMemsetAsync(G->grad, 0, sizeof(float) * kGuideParams, ctx->stream));
    FL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    G->steps = 0;
    return FL_OK;
}

static fl_status guide_slots(Guide *G, size_t cap) {
    if (cap <= G->slot_cap) return FL_OK;
    Context *ctx = G->ctx;
    cudaFree(G->mix);
    cudaFree(G->rec_idx);
    G->mix = nullptr;
    G->rec_idx = nullptr;
    G->slot_cap = 0;
    FL_CUDA_TRY(ctx, cudaMalloc(&G->mix, cap * kMixFloats * sizeof(float)));
    FL_CUDA_TRY(ctx, cudaMalloc(&G->rec_idx, cap * 2 * sizeof(uint32_t)));
    G->slot_cap = cap;
    return FL_OK;
}

static void bounds_of(const float bmin[3], const float bmax[3], float binv[3]) {
    for (int a = 0; a < 3; ++a) {
        const float e = bmax[a] - bmin[a];
        binv[a] = e > 0.f ? 1.f / e : 0.f;
    }
}

// Adam steps on the records of the last wave (n of them): stream-ordered
static fl_status guide_train(Guide *G, uint32_t n, const float bmin[3], const float binv[3], cudaStream_t st) {
    Context *ctx = G->ctx;
    if (n == 0) return FL_OK;
    FL_CUDA_TRY(ctx, cudaMemsetAsync(G->wstat, 0, 2 * sizeof(float), st));
    FL_CUDA_TRY(ctx, cudaMemsetAsync(G->loss, 0, sizeof(float), st));
    const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
    k_guide_stats<<<std::min<uint32_t>((n + 255) / 256, (uint32_t)sms * 4), 256, 0, st>>>(
        G->rec, G->rec_count, G->cfg.max_records, G->wstat, G->wts);
    size_t tmp = G->scan_bytes;
    FL_CUDA_TRY(ctx, cub::DeviceScan::InclusiveSum(G->scan_tmp, tmp, G->wts, G->cdf, (int)n, st));
    const uint32_t B = (uint32_t)G->cfg.batch;
    const uint32_t n_steps = std::min<uint32_t>((n + B - 1) / B, (uint32_t)G->cfg.steps_per_wave);
    for (uint32_t k = 0; k < n_steps; ++k) {
        TrainArgs T{};
        T.w = G->w16;
        T.grad = G->grad;
        T.rec = G->rec;
        T.rec_count = G->rec_count;
        T.rec_cap = (uint32_t)G->cfg.max_records;
        T.batch_begin = k * B;
        T.batch_size = B;
        T.wstat = G->wstat;
        T.loss = G->loss;
        for (int a = 0; a < 3; ++a) {
            T.bmin[a] = bmin[a];
            T.binv[a] = binv[a];
        }
        T.cdf = G->cdf;
        T.seed = (uint32_t)G->steps;
        T.learned = G->cfg.learn_select;
        T.err = ctx->d_error;
        launch_train(T, (B + kTrainRows - 1) / kTrainRows, st, G->cfg.train_kernel);
        G->steps += 1;
        AdamArgs a{};
        a.w32 = G->w32;
        a.m = G->m;
        a.v = G->v;
        a.grad = G->grad;
        a.w16 = G->w16;
        a.rec_count = G->rec_count;
        a.rec_cap = (uint32_t)G->cfg.max_records;
        a.batch_begin = k * B;
        a.batch_size = B;
        a.wstat = G->wstat;
        a.lr = G->cfg.learning_rate;
        a.bc1 = 1.f - powf(0.9f, (float)G->steps);
        a.bc2 = 1.f - powf(0.999f, (float)G->steps);
        a.resampled = 1;
        if (G->cfg.weight_average > 0.f) {
            G->avg_steps += 1;
            a.wavg = G->wavg;
            a.w16avg = G->w16avg;
            a.beta = G->cfg.weight_average;
            a.bc_avg = 1.f - powf(a.beta, (float)G->avg_steps);
        }
        k_guide_adam<<<(kGuideParams + 255) / 256, 256, 0, st>>>(a);
    }
    FL_CUDA_TRY(ctx, cudaGetLastError());
    return FL_OK;
}

// One guided pass: all samples of params into d_film (FP64 XYZ sums, added to).
static fl_status guide_pass(Guide *G, Scene *s, const CamDev &cam, const fl_render_params &p, int flags,
                            double *d_film, WaveCounters *h_cnt) {
    Context *ctx = s->ctx;
    cudaStream_t st = ctx->stream;
    const unsigned long long n_pix = (unsigned long long)cam.W * (unsigned long long)cam.H;
    const unsigned long long total = n_pix * (unsigned long long)p.spp;
    size_t cap_req = p.wave_paths > 0 ? (size_t)p.wave_paths : (size_t)1 << 21;
    cap_req = std::min<size_t>(cap_req, (size_t)total);
    WaveBuffers W;
    fl_status rc = wave_buffers(ctx, 4, (int)s->n_lights, cap_req, nullptr, 0, W);
    if (rc) return rc;
    rc = guide_slots(G, W.cap);
    if (rc) return rc;
    const bool train = (flags & FL_GUIDE_TRAIN) != 0;
    float binv[3];
    bounds_of(s->bmin, s->bmax, binv);
    for (int a = 0; a < 3; ++a) binv[a] *= G->cfg.position_scale;
    GuideArgs &ga = W.A.g;
    ga.w = G->render_weights();
    ga.mix = G->mix;
    ga.rec_idx = train ? G->rec_idx : nullptr;
    ga.rec = G->rec;
    ga.rec_count = G->rec_count;
    ga.rec_cap = (uint32_t)G->cfg.max_records;
    ga.select = (flags & FL_GUIDE_SAMPLE) ? G->cfg.select_prob : 0.f;
    ga.learned_select = G->cfg.learn_select;
    ga.record = train ? 1 : 0;
    for (int a = 0; a < 3; ++a) {
        ga.bmin[a] = s->bmin[a];
        ga.binv[a] = binv[a];
    }
    const JobDev j = job_of(s, cam, p, d_film);
    W.A.job0 = W.d_jobs;  // one job: every path's scene is job 0's
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(W.d_jobs, &j, sizeof(JobDev), cudaMemcpyHostToDevice, st));
    FL_CUDA_TRY(ctx, cudaMemsetAsync(W.A.cnt, 0, sizeof(WaveCounters), st));
    const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
    const size_t desc_bytes = offsetof(WaveDesc, seg) + sizeof(WaveSeg);
    RenderProfile prof;
    if (!train) {
        // sampling only: streaming waves, as fl_render's (no records to close per wave)
        W.A.slot_free = W.slot_free;
        W.A.free_count = W.free_count;
        W.A.free_off = W.free_off;
        for (unsigned long long wb = 0; wb < total; wb += kStreamDescPaths) {
            WaveDesc d;
            d.n_wave = (uint32_t)std::min<unsigned long long>(kStreamDescPaths, total - wb);
            d.n_seg = 1;
            d.seg[0] = WaveSeg{0u, 0u, d.n_wave, 0u, wb, 0ull};
            FL_CUDA_TRY(ctx, cudaMemcpyAsync(W.d_wave, &d, desc_bytes, cudaMemcpyHostToDevice, st));
            k_stream_init<<<std::min<uint32_t>(((uint32_t)W.cap + 127) / 128, (uint32_t)sms * 8), 128, 0, st>>>(W.A);
            const unsigned long long max_iters =
                ((unsigned long long)d.n_wave / W.cap + 2ull) * (unsigned long long)(j.bounce_cap + 2);
            for (unsigned long long it = 0;; it += kStreamIters) {
                if (it > max_iters) {
                    set_error(ctx, "streaming wave did not drain within its iteration bound");
                    return FL_ERR_TRAVERSAL;
                }
                enqueue_bounces<4, true>(W, 0, kStreamIters, false, &prof, sms, st, s->ext_kernels, true);
                FL_CUDA_TRY(ctx, cudaGetLastError());
                FL_CUDA_TRY(ctx, cudaMemcpyAsync(h_cnt, W.A.cnt, sizeof(WaveCounters), cudaMemcpyDeviceToHost, st));
                FL_CUDA_TRY(ctx, cudaStreamSynchronize(st));
                if (h_cnt->n_next == 0 && h_cnt->next_path >= d.n_wave) break;
            }
        }
        return FL_OK;
    }
    // Training: fixed waves, so that every path of a wave has ended, and closed its records,
    // when they train the guide after the wave.
    for (unsigned long long wb = 0; wb < total; wb += W.cap) {
        WaveDesc d;
        d.n_wave = (uint32_t)std::min<unsigned long long>(W.cap, total - wb);
        d.n_seg = 1;
        d.seg[0] = WaveSeg{0u, 0u, d.n_wave, 0u, wb, 0ull};
        FL_CUDA_TRY(ctx, cudaMemcpyAsync(W.d_wave, &d, desc_bytes, cudaMemcpyHostToDevice, st));
        if (train) FL_CUDA_TRY(ctx, cudaMemsetAsync(G->rec_count, 0, sizeof(uint32_t), st));
        enqueue_wave<4, true>(W, deepest_depth(p), false, &prof, sms, st, s->ext_kernels);
        FL_CUDA_TRY(ctx, cudaGetLastError());
        if (!depths_equal(p)) {
            rc = run_tail<4, true>(ctx, W, deepest_depth(p) + 1, false, &prof, sms, st, s->ext_kernels);
            if (rc) return rc;
        }
        if (train) {
            FL_CUDA_TRY(ctx, cudaMemcpyAsync(G->h_count, G->rec_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
            FL_CUDA_TRY(ctx, cudaStreamSynchronize(st));
            const uint32_t n = std::min<uint32_t>(*G->h_count, (uint32_t)G->cfg.max_records);
            rc = guide_train(G, n, s->bmin, binv, st);
            if (rc) return rc;
            FL_CUDA_TRY(ctx, cudaMemcpyAsync(G->h_loss, G->loss, sizeof(float), cudaMemcpyDeviceToHost, st));
        }
    }
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(h_cnt, W.A.cnt, sizeof(WaveCounters), cudaMemcpyDeviceToHost, st));
    return FL_OK;
}

static fl_status check_render_args(Context *ctx, Scene *s, const fl_camera *camera, const fl_render_params *params,
                                   void *film_rgb, int32_t memory) {
    if (!camera || !params || !film_rgb) {
        set_error(ctx, "null camera, parameters or film");
        return FL_ERR_INVALID;
    }
    const fl_render_params &p = *params;
    if (!camera_ok(*camera) || p.spp <= 0 || !depths_ok(p) || p.spectral_mode != FL_SPECTRAL_HERO4 ||
        (memory != FL_MEM_HOST && memory != FL_MEM_DEVICE)) {
        set_error(ctx, "invalid guided render parameters (hero wavelengths only)");
        return FL_ERR_INVALID;
    }
    if (s->n_lights > 64) {
        set_error(ctx, "more than 64 lights");
        return FL_ERR_INVALID;
    }
    return FL_OK;
}

// film scratch + resolve + copies shared by the two render calls
struct FilmOut {
    double *d_xyz = nullptr;
    float *d_rgb = nullptr;
    size_t n_pix = 0;
};
static fl_status film_begin(Context *ctx, const fl_camera *camera, float *film_rgb, double *film_xyz64,
                            int32_t memory, FilmOut &F) {
    F.n_pix = (size_t)camera->width * camera->height;
    const bool own_xyz = !(film_xyz64 && memory == FL_MEM_DEVICE);
    const size_t xyz_bytes = (F.n_pix * 3 * sizeof(double) + 255) & ~(size_t)255;
    void *fs = nullptr;
    fl_status rc = ensure_film_scratch(ctx, xyz_bytes + F.n_pix * 3 * sizeof(float), &fs);
    if (rc) return rc;
    F.d_xyz = own_xyz ? static_cast<double *>(fs) : film_xyz64;
    F.d_rgb = memory == FL_MEM_DEVICE ? film_rgb : reinterpret_cast<float *>(static_cast<char *>(fs) + xyz_bytes);
    FL_CUDA_TRY(ctx, cudaMemsetAsync(F.d_xyz, 0, F.n_pix * 3 * sizeof(double), ctx->stream));
    return FL_OK;
}
static fl_status film_end(Context *ctx, const FilmOut &F, double inv_spp, float *film_rgb, double *film_xyz64,
                          int32_t memory) {
    cudaStream_t st = ctx->stream;
    k_resolve<<<std::min<size_t>((F.n_pix + 255) / 256, (size_t)ctx->sm_count * 8), 256, 0, st>>>(
        F.d_xyz, (uint32_t)F.n_pix, inv_spp, F.d_rgb);
    FL_CUDA_TRY(ctx, cudaGetLastError());
    if (memory == FL_MEM_HOST) {
        FL_CUDA_TRY(ctx, cudaMemcpyAsync(film_rgb, F.d_rgb, F.n_pix * 3 * sizeof(float), cudaMemcpyDeviceToHost, st));
        if (film_xyz64)
            FL_CUDA_TRY(ctx, cudaMemcpyAsync(film_xyz64, F.d_xyz, F.n_pix * 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    FL_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return FL_OK;
}

static void add_stats(fl_render_stats *stats, const WaveCounters &hc) {
    stats->paths += hc.paths;
    stats->rays += hc.rays;
    stats->shadow_rays += hc.shadow_rays;
    stats->bounces += hc.bounces;
    stats->traversal_errors += (uint32_t)hc.err;
    stats->paths_cut += hc.cut;
}

}  // namespace fl

using namespace fl;

extern "C" fl_status fl_guide_create(fl_context *ctx_h, const fl_guide_config *cfg, fl_guide **out) {
    Context *ctx = reinterpret_cast<Context *>(ctx_h);
    if (!ctx || !cfg || !out) return FL_ERR_INVALID;
    *out = nullptr;
    std::lock_guard<std::mutex> lock(ctx->mu);
    const fl_guide_config c = *cfg;
    if (!(c.learning_rate > 0.f) || !(c.select_prob >= 0.f && c.select_prob < 1.f) || c.batch < 128 ||
        c.batch > 65536 || c.batch % 128 != 0 || c.max_records < c.batch || c.max_records > (1 << 26) ||
        c.steps_per_wave < 1 || !(c.position_scale >= 0.f && c.position_scale <= 1.f) ||
        !(c.weight_average >= 0.f && c.weight_average < 1.f) || (c.learn_select != 0 && c.learn_select != 1) ||
        (c.train_kernel != FL_GUIDE_TRAIN_MMA_SYNC && c.train_kernel != FL_GUIDE_TRAIN_TCGEN05)) {
        set_error(ctx, "invalid guide configuration");
        return FL_ERR_INVALID;
    }
    FL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    FL_CUDA_TRY(ctx, cudaFuncSetAttribute(k_guide_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem));
    FL_CUDA_TRY(ctx, cudaFuncSetAttribute(k_guide_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmemTc));
    FL_CUDA_TRY(ctx, cudaFuncSetAttribute(k_guide_infer<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)guide_infer_smem_bytes()));
    FL_CUDA_TRY(ctx, cudaFuncSetAttribute(k_guide_eval, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)guide_infer_smem_bytes()));
    Guide *G = new Guide();
    G->ctx = ctx;
    G->cfg = c;
    if (G->cfg.position_scale == 0.f) G->cfg.position_scale = 1.f;
    const size_t P = align_up(kGuideParams * sizeof(float));
    const size_t bytes = 2 * align_up(kGuideParams * sizeof(__half)) + 5 * P + 256 + 256 + 256;
    auto fail = [&](cudaError_t e, const char *what) {
        cudaFree(G->mem);
        cudaFree(G->rec);
        cudaFree(G->wts);
        cudaFreeHost(G->h_count);
        cudaFreeHost(G->h_loss);
        delete G;
        return cuda_status(ctx, e, what);
    };
    cudaError_t e = cudaMalloc(&G->mem, bytes);
    if (e) return fail(e, "guide state");
    e = cudaMalloc(&G->rec, (size_t)c.max_records * kRecFloats * sizeof(float));
    if (e) return fail(e, "guide records");
    e = cub::DeviceScan::InclusiveSum(nullptr, G->scan_bytes, (const float *)nullptr, (float *)nullptr,
                                      c.max_records, ctx->stream);
    if (e) return fail(e, "guide scan size");
    e = cudaMalloc(&G->wts, align_up((size_t)c.max_records * sizeof(float)) * 2 + G->scan_bytes);
    if (e) return fail(e, "guide record weights");
    G->cdf = reinterpret_cast<float *>(reinterpret_cast<char *>(G->wts) + align_up((size_t)c.max_records * sizeof(float)));
    G->scan_tmp = reinterpret_cast<char *>(G->cdf) + align_up((size_t)c.max_records * sizeof(float));
    e = cudaMallocHost(&G->h_count, sizeof(uint32_t));
    if (e) return fail(e, "guide pinned counter");
    e = cudaMallocHost(&G->h_loss, sizeof(float));
    if (e) return fail(e, "guide pinned loss");
    char *B = static_cast<char *>(G->mem);
    G->w16 = reinterpret_cast<__half *>(B);
    B += align_up(kGuideParams * sizeof(__half));
    G->w32 = reinterpret_cast<float *>(B);
    G->m = reinterpret_cast<float *>(B + P);
    G->v = reinterpret_cast<float *>(B + 2 * P);
    G->grad = reinterpret_cast<float *>(B + 3 * P);
    G->wstat = reinterpret_cast<float *>(B + 4 * P);
    G->loss = reinterpret_cast<float *>(B + 4 * P + 256);
    G->rec_count = reinterpret_cast<uint32_t *>(B + 4 * P + 512);
    G->wavg = reinterpret_cast<float *>(B + 4 * P + 768);
    G->w16avg = reinterpret_cast<__half *>(B + 5 * P + 768);
    e = cudaMemsetAsync(G->rec_count, 0, sizeof(uint32_t), ctx->stream);
    if (e) return fail(e, "guide counter");
    std::vector<float> w;
    guide_init_weights(c.seed, w);
    fl_status rc = guide_upload_weights(G, w);
    if (rc) {
        cudaFree(G->mem);
        cudaFree(G->rec);
        cudaFree(G->wts);
        cudaFreeHost(G->h_count);
        cudaFreeHost(G->h_loss);
        delete G;
        return rc;
    }
    ctx->children++;
    *out = reinterpret_cast<fl_guide *>(G);
    return FL_OK;
}

extern "C" fl_status fl_guide_destroy(fl_guide *g_h) {
    Guide *G = reinterpret_cast<Guide *>(g_h);
    if (!G) return FL_OK;
    Context *ctx = G->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaFree(G->mem);
    cudaFree(G->rec);
    cudaFree(G->wts);
    cudaFree(G->mix);
    cudaFree(G->rec_idx);
    cudaFreeHost(G->h_count);
    cudaFreeHost(G->h_loss);
    ctx->children--;
    delete G;
    return FL_OK;
}

extern "C" fl_status fl_guide_render(fl_guide *g_h, fl_scene *scene_h, const fl_camera *camera,
                                     const fl_render_params *params, int32_t flags, float *film_rgb,
                                     double *film_xyz64, int32_t memory, fl_render_stats *stats) {
    Guide *G = reinterpret_cast<Guide *>(g_h);
    Scene *s = reinterpret_cast<Scene *>(scene_h);
    if (!G || !s || G->ctx != s->ctx) return FL_ERR_INVALID;
    Context *ctx = s->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    fl_status rc = check_render_args(ctx, s, camera, params, film_rgb, memory);
    if (rc) return rc;
    FL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    const auto t0 = std::chrono::steady_clock::now();
    FilmOut F;
    rc = film_begin(ctx, camera, film_rgb, film_xyz64, memory, F);
    if (rc) return rc;
    WaveCounters hc{};
    rc = guide_pass(G, s, camera_basis_of(*camera), *params, flags, F.d_xyz, &hc);
    if (rc) return rc;
    rc = film_end(ctx, F, 1.0 / (double)params->spp, film_rgb, film_xyz64, memory);
    if (rc) return rc;
    if (flags & FL_GUIDE_TRAIN) G->last_loss = *G->h_loss;
    if (stats) {
        *stats = fl_render_stats{};
        add_stats(stats, hc);
        stats->ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return render_bounds_status(ctx, hc);
}

extern "C" fl_status fl_guide_render_timed(fl_guide *g_h, fl_scene *scene_h, const fl_camera *camera,
                                           const fl_render_params *params, double budget_ms, double train_fraction,
                                           float *film_rgb, double *film_xyz64, int32_t memory,
                                           fl_render_stats *stats) {
    Guide *G = reinterpret_cast<Guide *>(g_h);
    Scene *s = reinterpret_cast<Scene *>(scene_h);
    if (!G || !s || G->ctx != s->ctx) return FL_ERR_INVALID;
    Context *ctx = s->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    fl_status rc = check_render_args(ctx, s, camera, params, film_rgb, memory);
    if (rc) return rc;
    if (!(budget_ms > 0.0) || !(train_fraction >= 0.0 && train_fraction <= 1.0)) {
        set_error(ctx, "invalid time budget");
        return FL_ERR_INVALID;
    }
    FL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    const auto t0 = std::chrono::steady_clock::now();
    auto elapsed = [&] { return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(); };
    FilmOut F;
    rc = film_begin(ctx, camera, film_rgb, film_xyz64, memory, F);
    if (rc) return rc;
    const CamDev cam = camera_basis_of(*camera);
    fl_render_params p = *params;
    fl_render_stats acc{};
    uint32_t passes = 0;
    while (passes == 0 || elapsed() < budget_ms) {
        const bool train = elapsed() < train_fraction * budget_ms;
        const int flags = (train ? FL_GUIDE_TRAIN : 0) | (G->steps > 0 ? FL_GUIDE_SAMPLE : 0);
        p.sample_offset = params->sample_offset + passes * (uint32_t)params->spp;
        WaveCounters hc{};
        rc = guide_pass(G, s, cam, p, flags, F.d_xyz, &hc);
        if (rc) return rc;
        FL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        add_stats(&acc, hc);
        if (train) G->last_loss = *G->h_loss;
        ++passes;
    }
    rc = film_end(ctx, F, 1.0 / ((double)params->spp * passes), film_rgb, film_xyz64, memory);
    if (rc) return rc;
    if (stats) {
        *stats = acc;
        stats->ms = elapsed();
    }
    WaveCounters total{};
    total.err = (int)acc.traversal_errors;
    total.cut = (uint32_t)acc.paths_cut;
    return render_bounds_status(ctx, total);
}

extern "C" fl_status fl_guide_get_weights(fl_guide *g_h, float *weights) {
    Guide *G = reinterpret_cast<Guide *>(g_h);
    if (!G || !weights) return FL_ERR_INVALID;
    Context *ctx = G->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    FL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(weights, G->w32, sizeof(float) * kGuideParams, cudaMemcpyDeviceToHost, ctx->stream));
    FL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return FL_OK;
}

extern "C" fl_status fl_guide_set_weights(fl_guide *g_h, const float *weights) {
    Guide *G = reinterpret_cast<Guide *>(g_h);
    if (!G || !weights) return FL_ERR_INVALID;
    Context *ctx = G->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    FL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    std::vector<float> w(weights, weights + kGuideParams);
    for (float x : w)
        if (!std::isfinite(x)) {
            set_error(ctx, "non-finite guide weight");
            return FL_ERR_INVALID;
        }
    return guide_upload_weights(G, w);
}

extern "C" fl_status fl_guide_get_info(fl_guide *g_h, int64_t *adam_steps, float *last_loss) {
    Guide *G = reinterpret_cast<Guide *>(g_h);
    if (!G) return FL_ERR_INVALID;
    std::lock_guard<std::mutex> lock(G->ctx->mu);
    if (adam_steps) *adam_steps = G->steps;
    if (last_loss) *last_loss = G->last_loss;
    return FL_OK;
}

extern "C" fl_status fl_guide_gradient(fl_guide *g_h, const float *records, uint32_t n, const float bmin[3],
                                       const float bmax[3], float *grad, float *loss) {
    Guide *G = reinterpret_cast<Guide *>(g_h);
    if (!G || !records || !grad || !bmin || !bmax) return FL_ERR_INVALID;
    Context *ctx = G->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (n == 0 || n > (uint32_t)G->cfg.max_records) {
        set_error(ctx, "record count must be in [1, max_records]");
        return FL_ERR_INVALID;
    }
    FL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    float binv[3];
    bounds_of(bmin, bmax, binv);
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(G->rec, records, (size_t)n * kRecFloats * sizeof(float), cudaMemcpyHostToDevice, st));
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(G->rec_count, &n, sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    FL_CUDA_TRY(ctx, cudaMemsetAsync(G->wstat, 0, 2 * sizeof(float), st));
    FL_CUDA_TRY(ctx, cudaMemsetAsync(G->loss, 0, sizeof(float), st));
    FL_CUDA_TRY(ctx, cudaMemsetAsync(G->grad, 0, sizeof(float) * kGuideParams, st));
    const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
    k_guide_stats<<<std::min<uint32_t>((n + 255) / 256, (uint32_t)sms * 4), 256, 0, st>>>(
        G->rec, G->rec_count, G->cfg.max_records, G->wstat, nullptr);
    TrainArgs T{};
    T.w = G->w16;
    T.grad = G->grad;
    T.rec = G->rec;
    T.rec_count = G->rec_count;
    T.rec_cap = (uint32_t)G->cfg.max_records;
    T.batch_begin = 0;
    T.batch_size = n;
    T.wstat = G->wstat;
    T.loss = G->loss;
    T.learned = G->cfg.learn_select;
    for (int a = 0; a < 3; ++a) {
        T.bmin[a] = bmin[a];
        T.binv[a] = binv[a];
    }
    T.err = ctx->d_error;
    launch_train(T, (n + kTrainRows - 1) / kTrainRows, st, G->cfg.train_kernel);
    FL_CUDA_TRY(ctx, cudaGetLastError());
    std::vector<float> g(kGuideParams);
    float l = 0.f;
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(g.data(), G->grad, sizeof(float) * kGuideParams, cudaMemcpyDeviceToHost, st));
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(&l, G->loss, sizeof(float), cudaMemcpyDeviceToHost, st));
    FL_CUDA_TRY(ctx, cudaMemsetAsync(G->grad, 0, sizeof(float) * kGuideParams, st));
    FL_CUDA_TRY(ctx, cudaMemsetAsync(G->rec_count, 0, sizeof(uint32_t), st));
    FL_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    for (int i = 0; i < kGuideParams; ++i) grad[i] = g[i] / (kLossScale * (float)n);
    if (loss) *loss = l / (float)n;
    return FL_OK;
}

extern "C" fl_status fl_guide_get_records(fl_guide *g_h, float *records, uint32_t max_n, uint32_t *n) {
    Guide *G = reinterpret_cast<Guide *>(g_h);
    if (!G || !n || (max_n && !records)) return FL_ERR_INVALID;
    Context *ctx = G->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    FL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    uint32_t cnt = 0;
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(&cnt, G->rec_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    FL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    cnt = std::min<uint32_t>(cnt, (uint32_t)G->cfg.max_records);
    const uint32_t m = std::min(cnt, max_n);
    if (m)
        FL_CUDA_TRY(ctx, cudaMemcpyAsync(records, G->rec, (size_t)m * kRecFloats * sizeof(float), cudaMemcpyDeviceToHost,
                                         ctx->stream));
    FL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    *n = m;
    return FL_OK;
}

extern "C" fl_status fl_guide_eval(fl_guide *g_h, const float *records, uint32_t n, const float bmin[3],
                                   const float bmax[3], float *mixture) {
    Guide *G = reinterpret_cast<Guide *>(g_h);
    if (!G || !records || !mixture || !bmin || !bmax) return FL_ERR_INVALID;
    Context *ctx = G->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (n == 0 || n > (uint32_t)G->cfg.max_records) {
        set_error(ctx, "record count must be in [1, max_records]");
        return FL_ERR_INVALID;
    }
    FL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    float binv[3];
    bounds_of(bmin, bmax, binv);
    // records in, mixtures out: the record buffer holds both (mixtures after the records)
    const size_t rec_bytes = align_up((size_t)n * kRecFloats * sizeof(float));
    if (rec_bytes + (size_t)n * kGuideOut * sizeof(float) > (size_t)G->cfg.max_records * kRecFloats * sizeof(float)) {
        set_error(ctx, "too many records for one evaluation");
        return FL_ERR_CAPACITY;
    }
    float *d_rec = G->rec;
    float *d_out = reinterpret_cast<float *>(reinterpret_cast<char *>(G->rec) + rec_bytes);
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(d_rec, records, (size_t)n * kRecFloats * sizeof(float), cudaMemcpyHostToDevice, st));
    const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
    k_guide_eval<<<std::min<uint32_t>((n + 16 * kInferWarps - 1) / (16 * kInferWarps), (uint32_t)sms * 3),
                   32 * kInferWarps, guide_infer_smem_bytes(), st>>>(
        G->w16, d_rec, n, bmin[0], bmin[1], bmin[2], binv[0], binv[1], binv[2], d_out);
    FL_CUDA_TRY(ctx, cudaGetLastError());
    FL_CUDA_TRY(ctx, cudaMemcpyAsync(mixture, d_out, (size_t)n * kGuideOut * sizeof(float), cudaMemcpyDeviceToHost, st));
    FL_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return FL_OK;
}
