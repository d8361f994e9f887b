/*
 * ORACLE — test infrastructure only (see oracle.h). CPU restatement of the learned
 * path-guiding network of filianore-core_b200 (csrc/fl_guide.cuh, csrc/fl_guide.cu):
 * feature encoding, forward pass, vMF mixture, and the gradient of the radiance-weighted
 * training loss. The reference has no guiding; this oracle pins the GPU kernels to the
 * mathematics they implement. It rounds where the GPU rounds (FP16 weights, features,
 * post-ReLU activations and back-propagated gradients) and accumulates in double where
 * the GPU accumulates in FP32 on the tensor cores, so the two agree to FP32 summation
 * order plus the rare FP16 rounding tie.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "oracle.h"

#define G_IN 80
#define G_H 64
#define G_OUT 41
#define G_PARAMS 20032
#define G_REC 20
#define G_LOSS_SCALE (1.0 / 64.0)
#define G_WCLAMP 4096.0
#define G_LKMIN -2.0
#define G_LKMAX 7.0
#define G_LKSHIFT 2.0
#define G_SELMIN 0.2
#define G_SELMAX 0.7

static int g_exact = 0; /* 1: no FP16 rounding (finite-difference checks of the gradient) */
void orc_guide_set_exact(int on) { g_exact = on; }

static float h16(double x) {
    if (g_exact) return (float)x;
    if (x > 65000.0) x = 65000.0;
    if (x < -65000.0) x = -65000.0;
    return (float)(_Float16)(float)x;
}
static int w_in(int l) { return l == 0 ? 80 : 64; }
static int w_out(int l) { return l == 4 ? 41 : 64; }
static int w_off(int l) { return l == 0 ? 0 : 5120 + (l - 1) * 4096; }

/* features of a record: sin/cos(2^k pi x) per axis and band, normal, wavelength, 1, zeros */
static void features(const float *R, const float bmin[3], const float binv[3], float x[G_IN]) {
    double pn[3];
    for (int a = 0; a < 3; ++a) {
        float v = (R[a] - bmin[a]) * binv[a];
        v = v < 0.f ? 0.f : (v > 1.f ? 1.f : v);
        pn[a] = v;
    }
    for (int a = 0; a < 3; ++a)
        for (int k = 0; k < 12; ++k) {
            const double arg = M_PI * pn[a] * (double)(1 << k);
            x[24 * a + 2 * k] = h16(sin(arg));
            x[24 * a + 2 * k + 1] = h16(cos(arg));
        }
    x[72] = h16(R[3]);
    x[73] = h16(R[4]);
    x[74] = h16(R[5]);
    x[75] = h16((R[6] - 380.f) * (1.f / 340.f));
    x[76] = 1.f;
    x[77] = x[78] = x[79] = 0.f;
}

/* forward pass; acts[l] = post-ReLU output of hidden layer l (FP16 values), head in double */
static void forward(const float *w, const float x[G_IN], float acts[4][G_H], double head[G_OUT]) {
    const float *in = x;
    for (int l = 0; l < 4; ++l) {
        for (int o = 0; o < G_H; ++o) {
            double s = 0.0;
            for (int i = 0; i < w_in(l); ++i) s += (double)w[w_off(l) + o * w_in(l) + i] * in[i];
            acts[l][o] = h16(s > 0.0 ? s : 0.0);
        }
        in = acts[l];
    }
    for (int o = 0; o < G_OUT; ++o) {
        double s = 0.0;
        for (int i = 0; i < G_H; ++i) s += (double)w[w_off(4) + o * G_H + i] * in[i];
        head[o] = s;
    }
}

/* log kappa = min + (max - min) * sigmoid(s - shift) */
static double sigm(double s) { return 1.0 / (1.0 + exp(-(s - G_LKSHIFT))); }
static double kappa_of(double s) { return exp(G_LKMIN + (G_LKMAX - G_LKMIN) * sigm(s)); }
static double vmf_log_norm(double k) { return log(k) - log(2.0 * M_PI) - log(-expm1(-2.0 * k)); }

static double select_of(double s) { return G_SELMIN + (G_SELMAX - G_SELMIN) / (1.0 + exp(-s)); }

/* d(loss)/d(head); returns the loss: -log q(d), or with a learned selection -log f(d) of the
 * one-sample MIS density f = c q + (1 - c) pb, c = select_of(h[40]) */
static double head_grad(const double h[G_OUT], const double d[3], double dh[G_OUT], double pb, int learned) {
    double mx = h[0];
    for (int j = 1; j < 8; ++j) mx = h[j] > mx ? h[j] : mx;
    double se = 0.0;
    for (int j = 0; j < 8; ++j) se += exp(h[j] - mx);
    const double lse_pi = mx + log(se);
    double lq[8], mu[8][3], len[8], kap[8], dp[8], lmax = -INFINITY;
    for (int j = 0; j < 8; ++j) {
        const double x = h[8 + 3 * j], y = h[9 + 3 * j], z = h[10 + 3 * j];
        len[j] = sqrt(x * x + y * y + z * z);
        if (len[j] < 1e-6) len[j] = 1e-6;
        mu[j][0] = x / len[j];
        mu[j][1] = y / len[j];
        mu[j][2] = z / len[j];
        kap[j] = kappa_of(h[32 + j]);
        dp[j] = mu[j][0] * d[0] + mu[j][1] * d[1] + mu[j][2] * d[2];
        lq[j] = (h[j] - lse_pi) + vmf_log_norm(kap[j]) + kap[j] * (dp[j] - 1.0);
        if (lq[j] > lmax) lmax = lq[j];
    }
    double s = 0.0;
    for (int j = 0; j < 8; ++j) s += exp(lq[j] - lmax);
    const double lse = lmax + log(s);
    for (int j = 0; j < 8; ++j) {
        const double r = exp(lq[j] - lse), pi = exp(h[j] - lse_pi);
        dh[j] = -(r - pi);
        double g[3], mg = 0.0;
        for (int a = 0; a < 3; ++a) {
            g[a] = -r * kap[j] * d[a];
            mg += mu[j][a] * g[a];
        }
        for (int a = 0; a < 3; ++a) dh[8 + 3 * j + a] = (g[a] - mu[j][a] * mg) / len[j];
        const double sg = sigm(h[32 + j]), k = kap[j];
        dh[32 + j] = -r * (1.0 - 2.0 * k / expm1(2.0 * k) + k * (dp[j] - 1.0)) * (G_LKMAX - G_LKMIN) * sg * (1.0 - sg);
    }
    dh[40] = 0.0;
    if (!learned) return -lse;
    const double sg = 1.0 / (1.0 + exp(-h[40]));
    const double c = G_SELMIN + (G_SELMAX - G_SELMIN) * sg;
    const double q = exp(lse);
    const double f = c * q + (1.0 - c) * pb;
    for (int k = 0; k < 40; ++k) dh[k] *= c * q / f;
    dh[40] = -(q - pb) / f * (G_SELMAX - G_SELMIN) * sg * (1.0 - sg);
    return -log(f);
}

/* the Lambert BSDF's density of a record's direction (normal facing the viewer) */
static double record_bsdf_pdf(const float *R) {
    const double c = (double)R[3] * R[7] + (double)R[4] * R[8] + (double)R[5] * R[9];
    return c > 0.0 ? c / M_PI : 0.0;
}

static double record_weight(const float *R) {
    const double c = (double)R[3] * R[7] + (double)R[4] * R[8] + (double)R[5] * R[9];
    const double p = R[10], li = R[11];
    if (!(p > 0.0) || !(li > 0.0) || !(c > 0.0) || !isfinite(li)) return 0.0;
    return li * c / p;
}

static void round_weights(const float *w32, float *w16) {
    for (int i = 0; i < G_PARAMS; ++i) w16[i] = h16(w32[i]);
}

static void binv_of(const float bmin[3], const float bmax[3], float binv[3]) {
    for (int a = 0; a < 3; ++a) {
        const float e = bmax[a] - bmin[a];
        binv[a] = e > 0.f ? 1.f / e : 0.f;
    }
}

void orc_guide_eval(const float *w32, const float *rec, uint32_t n, const float bmin[3], const float bmax[3],
                    float *mix) {
    static float w[G_PARAMS];
    round_weights(w32, w);
    float binv[3];
    binv_of(bmin, bmax, binv);
    for (uint32_t r = 0; r < n; ++r) {
        float x[G_IN], acts[4][G_H];
        double h[G_OUT];
        features(rec + (size_t)r * G_REC, bmin, binv, x);
        forward(w, x, acts, h);
        float *m = mix + (size_t)r * G_OUT;
        double mx = h[0], s = 0.0;
        for (int j = 1; j < 8; ++j) mx = h[j] > mx ? h[j] : mx;
        for (int j = 0; j < 8; ++j) s += exp(h[j] - mx);
        for (int j = 0; j < 8; ++j) {
            m[j] = (float)(exp(h[j] - mx) / s);
            double len = sqrt(h[8 + 3 * j] * h[8 + 3 * j] + h[9 + 3 * j] * h[9 + 3 * j] + h[10 + 3 * j] * h[10 + 3 * j]);
            if (len < 1e-6) len = 1e-6;
            for (int a = 0; a < 3; ++a) m[8 + 3 * j + a] = (float)(h[8 + 3 * j + a] / len);
            m[32 + j] = (float)kappa_of(h[32 + j]);
        }
        m[40] = (float)select_of(h[40]);
    }
}

/* grad = d/dw of mean_r wn_r * loss_r, wn = min(w / mean(w), clamp), loss_r = -log q_r (or, with
 * learned != 0, -log of the one-sample MIS density); returns the mean loss */
float orc_guide_gradient(const float *w32, const float *rec, uint32_t n, const float bmin[3], const float bmax[3],
                         float *grad, int learned) {
    static float w[G_PARAMS];
    static double gacc[G_PARAMS];
    round_weights(w32, w);
    memset(gacc, 0, sizeof(gacc));
    float binv[3];
    binv_of(bmin, bmax, binv);
    double wsum = 0.0;
    for (uint32_t r = 0; r < n; ++r) wsum += (float)record_weight(rec + (size_t)r * G_REC);
    const double wmean = wsum / (double)n;
    double loss = 0.0;
    for (uint32_t r = 0; r < n && wsum > 0.0; ++r) {
        const float *R = rec + (size_t)r * G_REC;
        double wn = (float)record_weight(R) / wmean;
        if (wn > G_WCLAMP) wn = G_WCLAMP;
        if (!(wn > 0.0)) continue;
        float x[G_IN], acts[4][G_H];
        double h[G_OUT], dh[G_OUT];
        features(R, bmin, binv, x);
        forward(w, x, acts, h);
        const double d[3] = {R[7], R[8], R[9]};
        loss += wn * head_grad(h, d, dh, record_bsdf_pdf(R), learned);
        /* back-propagation with the GPU's FP16 roundings */
        float dz[G_H], dprev[G_H];
        for (int o = 0; o < G_OUT; ++o) dz[o] = h16(dh[o] * wn * G_LOSS_SCALE);
        for (int l = 4; l >= 0; --l) {
            const int in = w_in(l), out = w_out(l);
            const float *a_in = l == 0 ? x : acts[l - 1];
            for (int o = 0; o < out; ++o)
                for (int i = 0; i < in; ++i) gacc[w_off(l) + o * in + i] += (double)dz[o] * a_in[i];
            if (l == 0) break;
            for (int i = 0; i < in; ++i) {
                double s = 0.0;
                for (int o = 0; o < out; ++o) s += (double)dz[o] * w[w_off(l) + o * in + i];
                dprev[i] = acts[l - 1][i] > 0.f ? h16(s) : 0.f;
            }
            memcpy(dz, dprev, sizeof(dz));
        }
    }
    for (int i = 0; i < G_PARAMS; ++i) grad[i] = (float)(gacc[i] / (G_LOSS_SCALE * (double)n));
    return (float)(loss / (double)n);
}
