/*
 * Host utilities of the B200 engine library: the reference's host-side input
 * preparation that a caller without the reference driver needs, restated in C
 * with the reference's float/double arithmetic (built with -ffp-contract=off,
 * no -march, so the values match the reference's own build).
 *   ifosb_cpml_coeff : CPML_coeff.c:87-324
 *   ifosb_wavelet    : wavelet.c:29-99 (shapes 1, 2, 4, 5)
 *   ifosb_moduli     : readmod.c:48-65, 106-129 (the arithmetic, not the file IO)
 *   ifosb_steplength : steplength.c:26-91, in double
 */
#include "../../include/ifos_b200.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define PI_REF (3.141592653589793) /* fd.h:39 */

/* One direction of CPML_coeff. K, a, b, Kh, ah, bh are 1-based arrays of 2*FW+2.
 * zero_a_on_small_d: the array the reference clears when (int)d == 0 — a_x for the
 * x and the y loops (CPML_coeff.c:146-147, :200-201), none for z. */
static void pml_profile(int FW, float vppml, float fpml, float dt, float dh, float *K, float *a, float *b, float *Kh,
                        float *ah, float *bh, float *zero_a_on_small_d) {
    const float npower = 3, k_max_PML = 2.0;
    const float alpha_max_PML = 2.0 * PI_REF * (fpml / 2.0);
    const float Rcoef = 0.0008;
    const float pa = 0.25, pb = 0.75, pc = 0.0;
    const float d0 = -(npower + 1) * vppml * log(Rcoef) / (2.0 * FW * dh);
    for (int i = 1; i <= FW + 1; i++) {
        float pos = (FW - i + 1) * dh;
        float norm = pos / (FW * dh);
        float d = d0 * (pa * norm + pb * pow(norm, npower) + pc * pow(norm, (4)));
        K[i] = 1.0 + (k_max_PML - 1.0) * pow(norm, npower);
        float alpha = alpha_max_PML * (1.0 - norm);
        b[i] = exp(-(d / K[i] + alpha) * dt);
        int big = abs((int)d) > 1.0e-6; /* the reference applies integer abs() to a float */
        if (big) a[i] = d * (b[i] - 1.0) / (K[i] * (d + K[i] * alpha));
        else if (zero_a_on_small_d) zero_a_on_small_d[i] = 0.0;
        if (i <= FW) {
            float posh = (FW - i + 0.5) * dh;
            float normh = posh / (FW * dh);
            float dhf = d0 * (pa * normh + pb * pow(normh, npower) + pc * pow(normh, (4)));
            Kh[i] = 1.0 + (k_max_PML - 1.0) * pow(normh, npower);
            float alphah = alpha_max_PML * (1.0 - normh);
            bh[i] = exp(-(dhf / Kh[i] + alphah) * dt);
            if (abs((int)dhf) > 1.0e-6) ah[i] = dhf * (bh[i] - 1.0) / (Kh[i] * (dhf + Kh[i] * alphah));
            int l = 2 * FW - i + 1; /* the far face mirrors the near one */
            if (i > 1) {
                K[l + 1] = K[i];
                b[l + 1] = b[i];
                if (big) a[l + 1] = a[i];
            }
            Kh[l] = Kh[i];
            bh[l] = bh[i];
            if (big) ah[l] = ah[i];
        }
    }
}

int ifosb_cpml_coeff(const ifosb_params *p, float vppml, float fpml, float *coeff) {
    if (!p || !coeff || p->fw < 1) return IFOSB_EARG;
    const int n2 = 2 * p->fw, w = n2 + 2;
    float *t = calloc((size_t)18 * w, sizeof(float));
    if (!t) return IFOSB_ENOMEM;
    const float dh[3] = {p->dx, p->dy, p->dz};
    float *a_x = t + w;
    for (int d = 0; d < 3; d++) {
        float *r = t + (size_t)d * 6 * w;
        pml_profile(p->fw, vppml, fpml, p->dt, dh[d], r, r + w, r + 2 * w, r + 3 * w, r + 4 * w, r + 5 * w,
                    d < 2 ? a_x : NULL);
    }
    for (int r = 0; r < 18; r++)
        for (int h = 1; h <= n2; h++) coeff[(size_t)r * n2 + h - 1] = t[(size_t)r * w + h];
    free(t);
    return IFOSB_OK;
}

int ifosb_wavelet(const ifosb_params *p, int shape, int nsrc, const float *srcpos, float *signals) {
    if (!p || nsrc < 0 || (nsrc > 0 && (!srcpos || !signals))) return IFOSB_EARG;
    if (shape != 1 && shape != 2 && shape != 4 && shape != 5) return IFOSB_EARG;
    for (int nt = 1; nt <= p->nt; nt++) {
        float t = (float)nt * p->dt;
        for (int k = 0; k < nsrc; k++) {
            const float tshift = srcpos[k * 7 + 3], fc = srcpos[k * 7 + 4], a = srcpos[k * 7 + 5];
            const float ts = 1.0 / fc;
            float amp = 0.0f, tau;
            if (shape == 1) {
                tau = PI_REF * (t - 1.5 * ts - tshift) / (ts); /* Ricker */
                amp = (((1.0 - 2.0 * tau * tau) * exp(-tau * tau)));
            } else if (shape == 2) {
                if ((t < tshift) || (t > (tshift + ts))) amp = 0.0;
                else amp = ((sin(2.0 * PI_REF * (t - tshift) * fc) - 0.5 * sin(4.0 * PI_REF * (t - tshift) * fc)));
            } else if (shape == 4) {
                if ((t < tshift) || (t > (tshift + ts))) amp = 0.0; /* sin^3 */
                else amp = (0.75 * PI_REF / ts) * (pow(sin(PI_REF * (t - tshift) / ts), 3.0));
            } else {
                amp = (t < tshift) ? 0.0f : 1.0f;
            }
            signals[(size_t)k * p->nt + nt - 1] = amp * a;
        }
    }
    return IFOSB_OK;
}

int ifosb_moduli(const ifosb_params *p, long long n, const float *vp, const float *vs, const float *rho, float tau,
                 const float *fl, float *pi, float *u, float *taus, float *taup, float *eta) {
    if (!p || n < 0 || !vp || !vs || !rho || !pi || !u || p->nmech < 0 || p->nmech > 16) return IFOSB_EARG;
    const int L = p->nmech;
    if (L > 0 && (!fl || !taus || !taup || !eta)) return IFOSB_EARG;
    float pts[17], sumu = 0.0f, sumpi = 0.0f;
    const float ts = tau, tp = tau;
    for (int l = 1; l <= L; l++) {
        pts[l] = 1.0 / (2.0 * PI_REF * fl[l - 1]);
        eta[l - 1] = p->dt / pts[l];
    }
    if (L > 0) {
        const float ws = 2.0 * PI_REF * fl[0];
        for (int l = 1; l <= L; l++) {
            sumu = sumu + ((ws * ws * pts[l] * pts[l] * ts) / (1.0 + ws * ws * pts[l] * pts[l]));
            sumpi = sumpi + ((ws * ws * pts[l] * pts[l] * tp) / (1.0 + ws * ws * pts[l] * pts[l]));
        }
    }
    for (long long o = 0; o < n; o++) {
        const float muv = vs[o] * vs[o] * rho[o] / (1.0 + sumu);
        const float piv = vp[o] * vp[o] * rho[o] / (1.0 + sumpi);
        u[o] = muv;
        pi[o] = piv;
        if (L) { taus[o] = ts; taup[o] = tp; }
    }
    return IFOSB_OK;
}

/* steplength (steplength.c:26-91) with every quantity in double: the parabola
 * through (step[i], L2[i]), i = 0..2, its minimum step[3] limited as the
 * reference limits it, the parabola's value L2[3] there, and the next test
 * step step[4]. */
int ifosb_steplength(double *L2, double *step, int lbfgs, int it_group, double teststep, double *abc) {
    if (!L2 || !step) return IFOSB_EARG;
    const double s0 = step[0], s1 = step[1], s2 = step[2];
    const double a = ((s0 - s1) * (L2[0] - L2[2]) - (s0 - s2) * (L2[0] - L2[1])) /
                     (s0 * s2 * (s0 - s2) + s0 * s1 * (s1 - s0) + s1 * s2 * (s2 - s1));
    double b = (L2[0] - L2[1]) / (s0 - s1);
    b = b - a * (s0 + s1);
    const double c = L2[0] - a * s0 * s0 - b * s0;
    step[3] = 0.0;
    if (a > 0) step[3] = -b / (2 * a);
    if (a < 0) {
        if (L2[0] < L2[1] && L2[0] < L2[2]) step[3] = 0.1 * s1;
        if (L2[1] < L2[0] && L2[1] < L2[2]) step[3] = s1;
        if (L2[2] < L2[0] && L2[2] < L2[1]) step[3] = s2;
    }
    if (step[3] > 2.5 * step[4]) step[3] = 2.5 * step[4];
    if (lbfgs && it_group > 1 && step[3] > 1.0) step[3] = 1.0;
    if (step[3] <= 0) step[3] = 0.1 * s1;
    if (step[3] < 0.1 * s1) step[3] = 0.1 * s1;
    L2[3] = a * step[3] * step[3] + b * step[3] + c;
    step[4] = step[3] / 2;
    if (step[4] < 0.2 * teststep) step[4] = 0.2 * teststep;
    if (step[4] > teststep) step[4] = teststep;
    if (lbfgs && it_group > 1) step[4] = 0.5;
    if (abc) { abc[0] = a; abc[1] = b; abc[2] = c; }
    return IFOSB_OK;
}
