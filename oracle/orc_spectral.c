/*
 * ORACLE — test infrastructure only.
 *
 * PCG32 (src/ext/pcg32.h:40-163, O'Neill's PCG-XSH-RR 64/32 generator), the spectral
 * table binning of InitializeSpectrals (src/filianore/color/spectruminits.cpp:6-64),
 * RGB->spectrum upsampling (from_reflectance_rgb, color/spectrumoperations.cpp:113-147)
 * and spectrum->XYZ (to_xyz, color/spectrumoperations.cpp:193-207), restated in C.
 * Float/double mixing follows the reference exactly (the `0.5 *` double product in
 * average_spectrum_samples, the float `.94` scale).
 */
#include "oracle.h"

#include <stdlib.h>

#define PCG_MULT 0x5851f42d4c957f2dULL

uint32_t orc_pcg32_next(orc_pcg32 *r) {
    uint64_t old = r->state;
    r->state = old * PCG_MULT + r->inc;
    uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((~rot + 1u) & 31));
}

void orc_pcg32_seed(orc_pcg32 *r, uint64_t initstate, uint64_t initseq) {
    r->state = 0u;
    r->inc = (initseq << 1u) | 1u;
    orc_pcg32_next(r);
    r->state += initstate;
    orc_pcg32_next(r);
}

float orc_pcg32_nextf(orc_pcg32 *r) {
    uint32_t u = (orc_pcg32_next(r) >> 9) | 0x3f800000u;
    return orc_u2f(u) - 1.0f;
}

/* Brown's arbitrary-stride LCG jump, pcg32.h:142-163 */
void orc_pcg32_advance(orc_pcg32 *r, int64_t delta_) {
    uint64_t cur_mult = PCG_MULT, cur_plus = r->inc, acc_mult = 1u, acc_plus = 0u;
    uint64_t delta = (uint64_t)delta_;
    while (delta > 0) {
        if (delta & 1) {
            acc_mult *= cur_mult;
            acc_plus = acc_plus * cur_mult + cur_plus;
        }
        cur_plus = (cur_mult + 1) * cur_plus;
        cur_mult *= cur_mult;
        delta /= 2;
    }
    r->state = acc_mult * r->state + acc_plus;
}

void orc_pcg32_sequence(uint64_t initstate, uint64_t initseq, int64_t adv, uint32_t n, uint32_t *out) {
    orc_pcg32 r;
    orc_pcg32_seed(&r, initstate, initseq);
    if (adv) orc_pcg32_advance(&r, adv);
    for (uint32_t i = 0; i < n; ++i) out[i] = orc_pcg32_next(&r);
}

/* ---------------------------------------------------------------- tables */

static float lerpf_ref(float t, float v1, float v2) { return (1.f - t) * v1 + t * v2; }

float orc_average_spectrum_samples(const float *wl, const float *vals, int n, float ws, float we) {
    if (we <= wl[0]) return vals[0];
    if (ws >= wl[n - 1]) return vals[n - 1];
    if (n == 1) return vals[0];
    float sum = 0;
    if (ws < wl[0]) sum += vals[0] * (wl[0] - ws);
    if (we > wl[n - 1]) sum += vals[n - 1] * (we - wl[n - 1]);
    int i = 0;
    while (ws > wl[i + 1]) ++i;
    for (; i + 1 < n && we >= wl[i]; ++i) {
        float ss = ws > wl[i] ? ws : wl[i];
        float se = we < wl[i + 1] ? we : wl[i + 1];
        float ia = lerpf_ref((ss - wl[i]) / (wl[i + 1] - wl[i]), vals[i], vals[i + 1]);
        float ib = lerpf_ref((se - wl[i]) / (wl[i + 1] - wl[i]), vals[i], vals[i + 1]);
        sum = (float)((double)sum + 0.5 * (double)(ia + ib) * (double)(se - ss));
    }
    return sum / (we - ws);
}

int orc_tables_init(orc_tables *t, const fl_spectral_tables *s) {
    if (!s || s->n_cie <= 1 || s->n_cie > 512 || s->n_rgb2spec <= 1 || s->n_rgb2spec > 64) return -1;
    if (s->n_metals != 0 && s->n_metals != 9) return -1;
    for (int m = 0; m < s->n_metals; ++m)
        if (s->metal_n[m] < 1 || !s->metal_lambda[m] || !s->metal_eta[m] || !s->metal_k[m]) return -1;
    memset(t, 0, sizeof(*t));
    t->n_cie = s->n_cie;
    t->n_rgb = s->n_rgb2spec;
    t->cie_y_integral = s->cie_y_integral;
    memcpy(t->cie_lambda, s->cie_lambda, sizeof(float) * s->n_cie);
    memcpy(t->cie_x, s->cie_x, sizeof(float) * s->n_cie);
    memcpy(t->cie_y, s->cie_y, sizeof(float) * s->n_cie);
    memcpy(t->cie_z, s->cie_z, sizeof(float) * s->n_cie);
    memcpy(t->rgb_lambda, s->rgb2spec_lambda, sizeof(float) * s->n_rgb2spec);
    for (int b = 0; b < 7; ++b) {
        memcpy(t->refl[b], s->refl[b], sizeof(float) * s->n_rgb2spec);
        memcpy(t->illum[b], s->illum[b], sizeof(float) * s->n_rgb2spec);
    }
    for (int i = 0; i < ORC_NBINS; ++i) {
        float wl0 = lerpf_ref((float)i / (float)ORC_NBINS, 400.f, 700.f);
        float wl1 = lerpf_ref((float)(i + 1) / (float)ORC_NBINS, 400.f, 700.f);
        t->X[i] = orc_average_spectrum_samples(t->cie_lambda, t->cie_x, t->n_cie, wl0, wl1);
        t->Y[i] = orc_average_spectrum_samples(t->cie_lambda, t->cie_y, t->n_cie, wl0, wl1);
        t->Z[i] = orc_average_spectrum_samples(t->cie_lambda, t->cie_z, t->n_cie, wl0, wl1);
        for (int b = 0; b < 7; ++b) {
            t->brefl[b][i] = orc_average_spectrum_samples(t->rgb_lambda, t->refl[b], t->n_rgb, wl0, wl1);
            t->billum[b][i] = orc_average_spectrum_samples(t->rgb_lambda, t->illum[b], t->n_rgb, wl0, wl1);
        }
        for (int m = 0; m < s->n_metals && m < 9; ++m) {
            t->metal[m][0][i] = orc_average_spectrum_samples(s->metal_lambda[m], s->metal_eta[m], s->metal_n[m], wl0, wl1);
            t->metal[m][1][i] = orc_average_spectrum_samples(s->metal_lambda[m], s->metal_k[m], s->metal_n[m], wl0, wl1);
        }
    }
    return 0;
}

void orc_tables_metals(const orc_tables *t, float *out) { memcpy(out, t->metal, sizeof(t->metal)); }

void orc_tables_binned(const orc_tables *t, float *out) {
    memcpy(out, t->X, sizeof(float) * ORC_NBINS);
    memcpy(out + 60, t->Y, sizeof(float) * ORC_NBINS);
    memcpy(out + 120, t->Z, sizeof(float) * ORC_NBINS);
    for (int b = 0; b < 7; ++b) memcpy(out + 180 + 60 * b, t->brefl[b], sizeof(float) * ORC_NBINS);
    for (int b = 0; b < 7; ++b) memcpy(out + 600 + 60 * b, t->billum[b], sizeof(float) * ORC_NBINS);
}

/* ---------------------------------------------------------------- upsampling */

enum { B_WHITE = 0, B_CYAN, B_MAGENTA, B_YELLOW, B_RED, B_GREEN, B_BLUE };

/* The three (basis, weight) terms from_reflectance_rgb adds, in its order (:113-147). */
static void smits_terms(const float rgb[3], int basis[3], float w[3]) {
    if (rgb[0] <= rgb[1] && rgb[0] <= rgb[2]) {
        basis[0] = B_WHITE; w[0] = rgb[0];
        if (rgb[1] <= rgb[2]) {
            basis[1] = B_CYAN; w[1] = rgb[1] - rgb[0];
            basis[2] = B_BLUE; w[2] = rgb[2] - rgb[1];
        } else {
            basis[1] = B_CYAN; w[1] = rgb[2] - rgb[0];
            basis[2] = B_GREEN; w[2] = rgb[1] - rgb[2];
        }
    } else if (rgb[1] <= rgb[0] && rgb[1] <= rgb[2]) {
        basis[0] = B_WHITE; w[0] = rgb[1];
        if (rgb[0] <= rgb[2]) {
            basis[1] = B_MAGENTA; w[1] = rgb[0] - rgb[1];
            basis[2] = B_BLUE; w[2] = rgb[2] - rgb[0];
        } else {
            basis[1] = B_MAGENTA; w[1] = rgb[2] - rgb[1];
            basis[2] = B_RED; w[2] = rgb[0] - rgb[2];
        }
    } else {
        basis[0] = B_WHITE; w[0] = rgb[2];
        if (rgb[0] <= rgb[1]) {
            basis[1] = B_YELLOW; w[1] = rgb[0] - rgb[2];
            basis[2] = B_GREEN; w[2] = rgb[1] - rgb[0];
        } else {
            basis[1] = B_YELLOW; w[1] = rgb[1] - rgb[2];
            basis[2] = B_RED; w[2] = rgb[0] - rgb[1];
        }
    }
}

/* linear interpolation of a table sampled uniformly between lambda[0] and lambda[n-1] */
static float table_at(const float *lambda, const float *vals, int n, float l) {
    float x = (l - lambda[0]) / (lambda[n - 1] - lambda[0]) * (float)(n - 1);
    if (x <= 0.f) return vals[0];
    if (x >= (float)(n - 1)) return vals[n - 1];
    int j = (int)x;
    if (j > n - 2) j = n - 2;
    float f = x - (float)j;
    return vals[j] * (1.f - f) + vals[j + 1] * f;
}

void orc_reflectance(const orc_tables *t, const float rgb[3], int mode, const float *lambda, float *out) {
    int basis[3];
    float w[3];
    smits_terms(rgb, basis, w);
    int n = mode == FL_SPECTRAL_BINS60 ? ORC_NBINS : 4;
    for (int i = 0; i < n; ++i) {
        float r = 0.f;
        for (int k = 0; k < 3; ++k) {
            float b = mode == FL_SPECTRAL_BINS60 ? t->brefl[basis[k]][i]
                                                 : table_at(t->rgb_lambda, t->refl[basis[k]], t->n_rgb, lambda[i]);
            r += b * w[k];
        }
        r *= 0.94f;
        out[i] = r < 0.f ? 0.f : r;
    }
}

static float cie_at(const orc_tables *t, const float *tab, float l) {
    float x = l - t->cie_lambda[0];
    if (x <= 0.f) return tab[0];
    if (x >= (float)(t->n_cie - 1)) return tab[t->n_cie - 1];
    int j = (int)x;
    float f = x - (float)j;
    return tab[j] * (1.f - f) + tab[j + 1] * f;
}

void orc_xyz_from_spectrum(const orc_tables *t, int mode, const float *lambda, const float *L, double *xyz) {
    if (mode == FL_SPECTRAL_BINS60) {
        /* to_xyz, color/spectrumoperations.cpp:193-207 */
        float x = 0.f, y = 0.f, z = 0.f;
        for (int i = 0; i < ORC_NBINS; ++i) {
            x += t->X[i] * L[i];
            y += t->Y[i] * L[i];
            z += t->Z[i] * L[i];
        }
        float scale = (float)(700 - 400) / (float)(t->cie_y_integral * ORC_NBINS);
        xyz[0] = x * scale; xyz[1] = y * scale; xyz[2] = z * scale;
    } else {
        /* hero estimator of the same integral over 380..720 nm: pdf(lambda) = 1/340 */
        float x = 0.f, y = 0.f, z = 0.f;
        for (int k = 0; k < 4; ++k) {
            x += cie_at(t, t->cie_x, lambda[k]) * L[k];
            y += cie_at(t, t->cie_y, lambda[k]) * L[k];
            z += cie_at(t, t->cie_z, lambda[k]) * L[k];
        }
        float scale = 340.f / (4.f * t->cie_y_integral);
        xyz[0] = x * scale; xyz[1] = y * scale; xyz[2] = z * scale;
    }
}
