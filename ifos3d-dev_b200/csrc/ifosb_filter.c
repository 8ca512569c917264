/* ifosb_filter.c — the time-domain Butterworth filter of the multiscale stages
 * (FILT = 1): src/filt_seis.c:27-77 applies it to the source signals and the
 * observed seismograms of a stage, with the stage's highest frequency as corner.
 *
 * The filter is the recursive Butterworth of E. Wielandt's SEIFE (which the
 * reference links as libcseife): an order-m low- or high-pass is a cascade of one
 * first-order section (m odd) and m/2 second-order sections with damping
 * h_j = sin(pi (2j - 1) / (2m)). Each section is the bilinear transform of its
 * analog prototype at eps = 2 pi / T0 (T0 = corner period in samples):
 *   first order   g1 = (2 - eps) / (2 + eps);  low-pass f0 = f1 = eps / (2 + eps);
 *                 high-pass f0 = 2 / (2 + eps), f1 = -f0
 *   second order  a = 1 - eps h + eps^2/4, b = -2 + eps^2/2, c = 1 + eps h + eps^2/4,
 *                 g1 = -b/c, g2 = -a/c;  low-pass f0 = eps^2/4/c, f1 = 2 f0, f2 = f0;
 *                 high-pass f0 = 1/c, f1 = -2 f0, f2 = f0
 *   y[n] = f0 x[n] + f1 x[n-1] + f2 x[n-2] + g1 y[n-1] + g2 y[n-2]  (zero initial state)
 * evaluated in double in that operation order, so results are the reference's
 * bits. A high-pass first subtracts the first sample from the trace.
 *
 * filt_seis passes its 1-based sample vector to the 0-based filter, so the filter
 * runs over (0, s_1, ..., s_{ns-1}) and the last sample s_ns stays unfiltered. The
 * leading zero leaves a zero state, so s_1..s_{ns-1} come out as a plain filter of
 * the trace; this keeps both properties.
 */
#include "../../include/ifos_b200.h"

#include <math.h>
#include <stdlib.h>

typedef struct {
    double f0, f1, f2, g1, g2;
} section_t;

enum { LP1, HP1, LP2, HP2 };

static section_t design(int kind, double t0, double h) {
    const double eps = 8.0 * atan(1.0) / t0;
    section_t s = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (kind == LP1 || kind == HP1) {
        s.g1 = (2.0 - eps) / (2.0 + eps);
        if (kind == LP1) {
            s.f0 = eps / (2.0 + eps);
            s.f1 = s.f0;
        } else {
            s.f0 = 2.0 / (2.0 + eps);
            s.f1 = -(s.f0);
        }
    } else {
        const double e2 = eps * eps;
        const double a = 1.0 - eps * h + e2 / 4.0, b = -2.0 + e2 / 2.0, c = 1.0 + eps * h + e2 / 4.0;
        s.g1 = -b / c;
        s.g2 = -a / c;
        if (kind == LP2) {
            s.f0 = e2 / 4.0 / c;
            s.f1 = s.f0 + s.f0;
            s.f2 = s.f0;
        } else {
            s.f0 = 1.0 / c;
            s.f1 = -(s.f0) - s.f0;
            s.f2 = s.f0;
        }
    }
    return s;
}

static void apply(double *x, int n, section_t s) {
    double xa = 0.0, xaa = 0.0, ya = 0.0, yaa = 0.0;
    for (int j = 0; j < n; ++j) {
        const double xn = x[j];
        const double y = s.f0 * xn + s.f1 * xa + s.f2 * xaa + s.g1 * ya + s.g2 * yaa;
        x[j] = y;
        xaa = xa;
        xa = xn;
        yaa = ya;
        ya = y;
    }
}

/* Order-m Butterworth over x[0..n-1]; t0 = corner period in samples. */
static void butterworth(double *x, int n, double t0, int m, int highpass) {
    if (highpass) {
        const double x0 = x[0];
        for (int i = 0; i < n; ++i) x[i] -= x0;
    }
    const int mm = m / 2;
    if (m > 2 * mm) apply(x, n, design(highpass ? HP1 : LP1, t0, 0.0));
    const double pih = 2.0 * atan(1.0);
    for (int j = 1; j <= mm; ++j) {
        const double h = sin(pih * (2 * j - 1) / m);
        apply(x, n, design(highpass ? HP2 : LP2, t0, h));
    }
}

int ifosb_filt_seis(float *data, int ntr, int ns, float finv, float dt, int order, int highpass) {
    if (ntr < 0 || ns < 1 || order < 1 || !(finv > 0.0f) || !(dt > 0.0f) || (ntr > 0 && !data))
        return IFOSB_EARG;
    double *s = (double *)malloc(sizeof(double) * (size_t)(ns + 1));
    if (!s) return IFOSB_ENOMEM;
    const double T0 = 1.0 / finv;
    const double t0 = T0 / (double)dt;
    for (int t = 0; t < ntr; ++t) {
        float *d = data + (size_t)t * ns;
        /* s[0] is filt_seis's unused element 0 (zero), s[1..ns] the samples */
        s[0] = 0.0;
        for (int j = 0; j < ns; ++j) s[j + 1] = (double)d[j];
        butterworth(s, ns, t0, order, highpass);
        for (int j = 0; j < ns; ++j) d[j] = (float)s[j + 1];
    }
    free(s);
    return IFOSB_OK;
}
