/*
 * CPU ORACLE — plain-C restatement of the IFOS3D wavefield path.
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py, never by the CUDA product.
 *
 * Restates, per grid cell instead of per loop nest, the arithmetic of:
 *   update_v_ssg.c:92-130 (+ forces :474-522), update_v_ssg_CPML.c:30-403,
 *   update_s_ssg_elastic.c:95-147, update_s_ssg_CPML_elastic.c:30-505,
 *   update_s_ssg.c:139-232 and update_s_ssg_CPML.c (viscoelastic, generalised
 *   from one to L relaxation mechanisms the way the memory-variable sums of
 *   update_s_ssg.c:88-96 / :123-138 are written), surface_ssg_elastic.c:69-111,
 *   surface_ssg.c:117-160, psource.c:26-54, seismo_ssg.c:43-50,
 *   disc_fourier.c:28-61, gradient_F.c:30-171, residual.c:27-60, av_mat.c:28-80,
 *   matcopy.c (one rank: periodic ghost wrap), CPML_coeff.c:87-324,
 *   CPML_ini_elastic.c:26-71, readmod.c:28-139, wavelet.c:29-99.
 * Every expression keeps the reference's operand order and float/double
 * promotions, so at L<=1 its results are bit-identical to the reference built
 * with the same compiler flags (pinned by tests/test_oracle_pin.py).
 *
 * Parity: pinned against the reference itself (oracle/_ref/libifos_ref.so) and
 * against the committed fixtures in tests/golden/ that the reference produced.
 */
#include "ifos_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <unistd.h>

/* Threads of the cell loops (1 unless ifo_set_threads says otherwise). Every
 * cell of a parallel loop reads only fields that the loop does not write and
 * writes only its own entries, so the results do not depend on the count. */
#define MAX_THREADS 256
static int g_threads = 1;

void ifo_set_threads(int n) {
    if (n <= 0) n = (int)sysconf(_SC_NPROCESSORS_ONLN);
    g_threads = n < 1 ? 1 : (n > MAX_THREADS ? MAX_THREADS : n);
}

/* rows lo..hi of a loop, split into contiguous blocks over the threads */
typedef void (*rows_fn)(void *ctx, int lo, int hi);
typedef struct {
    rows_fn fn;
    void *ctx;
    int lo, hi;
} par_job;

static void *par_body(void *a) {
    par_job *q = a;
    q->fn(q->ctx, q->lo, q->hi);
    return NULL;
}

static void par_rows(int lo, int hi, rows_fn fn, void *ctx) {
    const int n = hi - lo + 1, T = g_threads < n ? g_threads : n;
    if (T <= 1) {
        fn(ctx, lo, hi);
        return;
    }
    pthread_t th[MAX_THREADS];
    par_job jb[MAX_THREADS];
    int ok[MAX_THREADS];
    for (int t = 0; t < T; t++) {
        jb[t].fn = fn;
        jb[t].ctx = ctx;
        jb[t].lo = lo + (int)((long long)n * t / T);
        jb[t].hi = lo + (int)((long long)n * (t + 1) / T) - 1;
    }
    for (int t = 1; t < T; t++) ok[t] = pthread_create(&th[t], NULL, par_body, &jb[t]) == 0;
    par_body(&jb[0]);
    for (int t = 1; t < T; t++) {
        if (ok[t]) pthread_join(th[t], NULL);
        else par_body(&jb[t]); /* no thread: run the block here */
    }
}

#define PI_REF (3.141592653589793) /* fd.h:39 */
#define MAXMECH 8

typedef struct {
    int nx, ny, nz, fw;
    size_t WX, WY, WZ, wn;
} geo_t;

static geo_t mkgeo(const ifo_params *p) {
    geo_t g;
    g.nx = p->nx; g.ny = p->ny; g.nz = p->nz; g.fw = p->fw;
    g.WX = (size_t)p->nx + 4; g.WY = (size_t)p->ny + 5; g.WZ = (size_t)p->nz + 4;
    g.wn = g.WX * g.WY * g.WZ;
    return g;
}
/* wavefield cell (j,i,k), j=-2..NY+2, i=-1..NX+2, k=-1..NZ+2 */
#define W(j, i, k) ((((size_t)((j) + 2)) * G.WX + (size_t)((i) + 1)) * G.WZ + (size_t)((k) + 1))
/* interior cell, 1-based */
#define M(j, i, k) ((((size_t)((j) - 1)) * (size_t)G.nx + (size_t)((i) - 1)) * (size_t)G.nz + (size_t)((k) - 1))
/* ghosted model cell, j=0..NY+1 */
#define MG(j, i, k) ((((size_t)(j)) * (size_t)(G.nx + 2) + (size_t)(i)) * (size_t)(G.nz + 2) + (size_t)(k))

int ifo_nsamples(const ifo_params *p) {
    if (p->ndtshift > p->nt) return 0;
    return (int)ceil((float)(p->nt - p->ndtshift) / (float)p->ndt); /* ifos3d.c:178-179 */
}

static void fd_coeffs(const ifo_params *p, float *b1, float *b2) {
    *b1 = 9.0 / 8.0; *b2 = -1.0 / 24.0;           /* Taylor, update_v_ssg.c:97 */
    if (p->fdcoeff == 2) { *b1 = 1.1382; *b2 = -0.046414; } /* Holberg, :98-100 */
}

/* ------------------------------------------------------------------------- */
/* readmod.c:28-139: relaxed-modulus scaling of the elastic moduli.           */
int ifo_readmod(const ifo_params *p, const ifo_velmodel *vm, float *rho, float *pi, float *u,
                float *taus, float *taup, float *eta) {
    int L = p->nmech;
    float pts[MAXMECH + 1], ts = vm->tau, tp = vm->tau, ws, sumu = 0.0f, sumpi = 0.0f;
    if (L > MAXMECH) return 1;
    for (int l = 1; l <= L; l++) {
        pts[l] = 1.0 / (2.0 * PI_REF * vm->fl[l - 1]);
        eta[l - 1] = p->dt / pts[l];
    }
    if (L > 0) {
        ws = 2.0 * PI_REF * vm->fl[0];
        for (int l = 1; l <= L; l++) {
            sumu = sumu + ((ws * ws * pts[l] * pts[l] * ts) / (1.0 + ws * ws * pts[l] * pts[l]));
            sumpi = sumpi + ((ws * ws * pts[l] * pts[l] * tp) / (1.0 + ws * ws * pts[l] * pts[l]));
        }
    }
    size_t n = (size_t)p->nx * p->ny * p->nz;
    for (size_t o = 0; o < n; o++) {
        float vp = vm->vp[o], vs = vm->vs[o], rhov = vm->rho[o];
        float muv = vs * vs * rhov / (1.0 + sumu);
        float piv = vp * vp * rhov / (1.0 + sumpi);
        u[o] = muv; rho[o] = rhov; pi[o] = piv;
        if (L) { taus[o] = ts; taup[o] = tp; }
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* CPML_coeff.c:87-324 (one direction; the three are identical in form).     */
/* else_a: the array the reference zeroes when d < 1 (a_x for both the x and the
 * y loop, CPML_coeff.c:146-147 and :200-201; nothing for z). */
static void cpml_dir(const ifo_params *p, float dh, float *K, float *a, float *b, float *Kh, float *ah, float *bh,
                     float *else_a) {
    const int FW = p->fw;
    const float npower = 3, k_max_PML = 2.0;
    const float alpha_max_PML = 2.0 * PI_REF * (p->fpml / 2.0);
    const float Rcoef = 0.0008;
    const float ca = 0.25, cb = 0.75, cc = 0.0;
    /* 1-based work arrays of length 2*FW (+1 for the i=FW+1 point) */
    float *d = calloc((size_t)2 * FW + 2, sizeof(float)), *dh_ = calloc((size_t)2 * FW + 2, sizeof(float));
    float *alpha = calloc((size_t)2 * FW + 2, sizeof(float)), *alphah = calloc((size_t)2 * FW + 2, sizeof(float));
    float d0 = -(npower + 1) * p->vppml * log(Rcoef) / (2.0 * FW * dh);
    for (int i = 1; i <= FW + 1; i++) {
        float pos = (FW - i + 1) * dh;
        float norm = pos / (FW * dh);
        d[i] = d0 * (ca * norm + cb * pow(norm, npower) + cc * pow(norm, (4)));
        K[i] = 1.0 + (k_max_PML - 1.0) * pow(norm, npower);
        alpha[i] = alpha_max_PML * (1.0 - norm);
        b[i] = exp(-(d[i] / K[i] + alpha[i]) * p->dt);
        /* integer abs() of a float as in the reference (CPML_coeff.c:146) */
        if (abs((int)d[i]) > 1.0e-6) a[i] = d[i] * (b[i] - 1.0) / (K[i] * (d[i] + K[i] * alpha[i]));
        else if (else_a) else_a[i] = 0.0;
        if (i <= FW) {
            float posh = (FW - i + 0.5) * dh;
            float normh = posh / (FW * dh);
            dh_[i] = d0 * (ca * normh + cb * pow(normh, npower) + cc * pow(normh, (4)));
            Kh[i] = 1.0 + (k_max_PML - 1.0) * pow(normh, npower);
            alphah[i] = alpha_max_PML * (1.0 - normh);
            bh[i] = exp(-(dh_[i] / Kh[i] + alphah[i]) * p->dt);
            if (abs((int)dh_[i]) > 1.0e-6) ah[i] = dh_[i] * (bh[i] - 1.0) / (Kh[i] * (dh_[i] + Kh[i] * alphah[i]));
            int l = 2 * FW - i + 1;
            if (i > 1) {
                K[l + 1] = K[i];
                b[l + 1] = b[i];
                if (abs((int)d[i]) > 1.0e-6) a[l + 1] = a[i];
            }
            Kh[l] = Kh[i];
            bh[l] = bh[i];
            if (abs((int)d[i]) > 1.0e-6) ah[l] = ah[i];
        }
    }
    free(d); free(dh_); free(alpha); free(alphah);
}

int ifo_cpml_coeff(const ifo_params *p, float *flat) {
    const int n2 = 2 * p->fw;
    float *w = calloc((size_t)18 * (n2 + 2), sizeof(float));
    float dhs[3] = {p->dx, p->dy, p->dz};
    float *a_x = w + (n2 + 2);
    for (int d = 0; d < 3; d++) {
        float *base = w + (size_t)d * 6 * (n2 + 2);
        cpml_dir(p, dhs[d], base, base + (n2 + 2), base + 2 * (n2 + 2), base + 3 * (n2 + 2),
                 base + 4 * (n2 + 2), base + 5 * (n2 + 2), d < 2 ? a_x : NULL);
    }
    for (int r = 0; r < 18; r++)
        for (int h = 1; h <= n2; h++) flat[(size_t)r * n2 + h - 1] = w[(size_t)r * (n2 + 2) + h];
    free(w);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* wavelet.c:29-99 (shapes 1 Ricker, 2 fumue, 4 sin^3, 5 step).               */
int ifo_wavelet(const ifo_params *p, int nsrc, const float *srcpos, float *signals) {
    for (int nt = 1; nt <= p->nt; nt++) {
        float t = (float)nt * p->dt;
        for (int k = 0; k < nsrc; k++) {
            float tshift = srcpos[k * 7 + 3], fc = srcpos[k * 7 + 4], a = srcpos[k * 7 + 5];
            float ts = 1.0 / fc, amp = 0.0f, tau;
            switch (p->source_shape) {
            case 1:
                tau = PI_REF * (t - 1.5 * ts - tshift) / (ts);
                amp = (((1.0 - 2.0 * tau * tau) * exp(-tau * tau)));
                break;
            case 2:
                if ((t < tshift) || (t > (tshift + ts))) amp = 0.0;
                else amp = ((sin(2.0 * PI_REF * (t - tshift) * fc) - 0.5 * sin(4.0 * PI_REF * (t - tshift) * fc)));
                break;
            case 4:
                if ((t < tshift) || (t > (tshift + ts))) amp = 0.0;
                else amp = (0.75 * PI_REF / ts) * (pow(sin(PI_REF * (t - tshift) / ts), 3.0));
                break;
            case 5:
                amp = (t < tshift) ? 0.0f : 1.0f;
                break;
            default:
                return 1;
            }
            signals[(size_t)k * p->nt + nt - 1] = amp * a;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Model with ghosts: one-rank matcopy.c leaves every ghost layer holding the  */
/* opposite face, i.e. a periodic wrap (the MPI_PROC_NULL receives are no-ops).*/
static float *ghosted(const ifo_params *p, const float *m) {
    geo_t G = mkgeo(p);
    float *gm = malloc(sizeof(float) * (size_t)(G.nx + 2) * (G.ny + 2) * (G.nz + 2));
    for (int j = 0; j <= G.ny + 1; j++) {
        int jj = j == 0 ? G.ny : (j == G.ny + 1 ? 1 : j);
        for (int i = 0; i <= G.nx + 1; i++) {
            int ii = i == 0 ? G.nx : (i == G.nx + 1 ? 1 : i);
            for (int k = 0; k <= G.nz + 1; k++) {
                int kk = k == 0 ? G.nz : (k == G.nz + 1 ? 1 : k);
                gm[MG(j, i, k)] = m[M(jj, ii, kk)];
            }
        }
    }
    return gm;
}

/* av_mat.c:45-69 */
static void av_mat_g(const ifo_params *p, const float *rho, const float *u, const float *taus, float *avg9) {
    geo_t G = mkgeo(p);
    size_t n = (size_t)G.nx * G.ny * G.nz;
    for (int j = 1; j <= G.ny; j++)
        for (int i = 1; i <= G.nx; i++)
            for (int k = 1; k <= G.nz; k++) {
                size_t o = M(j, i, k);
                avg9[0 * n + o] = 4.0 / ((1.0 / u[MG(j, i, k)]) + (1.0 / u[MG(j, i + 1, k)]) +
                                         (1.0 / u[MG(j + 1, i + 1, k)]) + (1.0 / u[MG(j + 1, i, k)]));
                avg9[1 * n + o] = 4.0 / ((1.0 / u[MG(j, i, k)]) + (1.0 / u[MG(j, i, k + 1)]) +
                                         (1.0 / u[MG(j + 1, i, k + 1)]) + (1.0 / u[MG(j + 1, i, k)]));
                avg9[2 * n + o] = 4.0 / ((1.0 / u[MG(j, i, k)]) + (1.0 / u[MG(j, i, k + 1)]) +
                                         (1.0 / u[MG(j, i + 1, k + 1)]) + (1.0 / u[MG(j, i + 1, k)]));
                if (taus) {
                    avg9[6 * n + o] = 0.25 * (taus[MG(j, i, k)] + taus[MG(j, i + 1, k)] + taus[MG(j + 1, i + 1, k)] +
                                              taus[MG(j + 1, i, k)]);
                    avg9[7 * n + o] = 0.25 * (taus[MG(j, i, k)] + taus[MG(j + 1, i, k)] + taus[MG(j + 1, i, k + 1)] +
                                              taus[MG(j, i, k + 1)]);
                    avg9[8 * n + o] = 0.25 * (taus[MG(j, i, k)] + taus[MG(j, i + 1, k)] + taus[MG(j, i + 1, k + 1)] +
                                              taus[MG(j, i, k + 1)]);
                } else {
                    avg9[6 * n + o] = avg9[7 * n + o] = avg9[8 * n + o] = 0.0f;
                }
                avg9[4 * n + o] = 0.5 * (rho[MG(j, i, k)] + rho[MG(j + 1, i, k)]); /* rjp */
                avg9[5 * n + o] = 0.5 * (rho[MG(j, i, k)] + rho[MG(j, i, k + 1)]); /* rkp */
                avg9[3 * n + o] = 0.5 * (rho[MG(j, i, k)] + rho[MG(j, i + 1, k)]); /* rip */
            }
}

int ifo_av_mat(const ifo_params *p, const float *rho, const float *pi, const float *u,
               const float *taus, const float *taup, float *avg9) {
    float *gr = ghosted(p, rho), *gu = ghosted(p, u), *gt = (p->nmech && taus) ? ghosted(p, taus) : NULL;
    av_mat_g(p, gr, gu, gt, avg9);
    free(gr); free(gu); free(gt);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Propagation state and one time step.                                       */
typedef struct {
    const ifo_params *p;
    geo_t G;
    float b1, b2;
    /* model */
    const float *pi, *u, *taus, *taup; /* interior [NY][NX][NZ] */
    float eta[MAXMECH];
    float *avg9;                       /* uipjp, ujpkp, uipkp, rip, rjp, rkp, tausipjp, tausjpkp, tausipkp */
    const float *cp;                   /* cpml [18][2FW] */
    /* wavefield */
    float *vx, *vy, *vz, *sxx, *syy, *szz, *sxy, *syz, *sxz;
    float *r[MAXMECH][6];              /* rxx, ryy, rzz, rxy, ryz, rxz per mechanism, interior layout */
    float *ps[9], *pv[9];
} orc_t;

enum { K_X, A_X, B_X, KH_X, AH_X, BH_X, K_Y, A_Y, B_Y, KH_Y, AH_Y, BH_Y, K_Z, A_Z, B_Z, KH_Z, AH_Z, BH_Z };
#define CP(row, h) (o->cp[(size_t)(row) * 2 * o->p->fw + (h) - 1])

/* CPML face membership (CPML_ini_elastic.c:26-71, the face loops of
 * update_v_ssg_CPML.c); returns the 1-based slab index or 0. */
static int face_x(const orc_t *o, int i) {
    int FW = o->p->fw;
    if (i <= FW) return i;
    if (i >= o->G.nx - FW + 1) return i - o->G.nx + 2 * FW;
    return 0;
}
static int face_y(const orc_t *o, int j) {
    int FW = o->p->fw;
    if (!o->p->free_surf && j <= FW) return j;
    if (j >= o->G.ny - FW + 1) return j - o->G.ny + 2 * FW;
    return 0;
}
static int face_z(const orc_t *o, int k) {
    int FW = o->p->fw;
    if (k <= FW) return k;
    if (k >= o->G.nz - FW + 1) return k - o->G.nz + 2 * FW;
    return 0;
}
/* slab storage: x [NY][2FW][NZ], y [2FW][NX][NZ], z [NY][NX][2FW] */
static size_t sx_idx(const orc_t *o, int j, int h, int k) { return ((size_t)(j - 1) * 2 * o->p->fw + (h - 1)) * o->G.nz + (k - 1); }
static size_t sy_idx(const orc_t *o, int h, int i, int k) { return ((size_t)(h - 1) * o->G.nx + (i - 1)) * o->G.nz + (k - 1); }
static size_t sz_idx(const orc_t *o, int j, int i, int h) { return ((size_t)(j - 1) * o->G.nx + (i - 1)) * 2 * o->p->fw + (h - 1); }

typedef struct { int i, j, k, kind; } pt_t; /* kind: stype 1..5 (forward) or 6 adjoint */

/* Velocity update of one cell: update_v_ssg.c:102-127 interior expressions, the
 * CPML psi recursions of update_v_ssg_CPML.c, and point forces in the
 * reference's order (interior: update then force; CPML frame: force, update,
 * force again for the adjoint). */
static void v_cell(orc_t *o, int j, int i, int k, int nt, int back, int npt, const pt_t *pts,
                   const float *sigx, const float *sigy, const float *sigz) {
    const geo_t G = o->G;
    const ifo_params *p = o->p;
    const float b1 = o->b1, b2 = o->b2;
    float dx = p->dt / p->dx, dy = p->dt / p->dy, dz = p->dt / p->dz;
    const float *sxx = o->sxx, *syy = o->syy, *szz = o->szz, *sxy = o->sxy, *syz = o->syz, *sxz = o->sxz;
    float sxx_x = dx * (b1 * (sxx[W(j, i + 1, k)] - sxx[W(j, i, k)]) + b2 * (sxx[W(j, i + 2, k)] - sxx[W(j, i - 1, k)]));
    float sxy_y = dy * (b1 * (sxy[W(j, i, k)] - sxy[W(j - 1, i, k)]) + b2 * (sxy[W(j + 1, i, k)] - sxy[W(j - 2, i, k)]));
    float sxz_z = dz * (b1 * (sxz[W(j, i, k)] - sxz[W(j, i, k - 1)]) + b2 * (sxz[W(j, i, k + 1)] - sxz[W(j, i, k - 2)]));
    float syy_y = dy * (b1 * (syy[W(j + 1, i, k)] - syy[W(j, i, k)]) + b2 * (syy[W(j + 2, i, k)] - syy[W(j - 1, i, k)]));
    float sxy_x = dx * (b1 * (sxy[W(j, i, k)] - sxy[W(j, i - 1, k)]) + b2 * (sxy[W(j, i + 1, k)] - sxy[W(j, i - 2, k)]));
    float syz_z = dz * (b1 * (syz[W(j, i, k)] - syz[W(j, i, k - 1)]) + b2 * (syz[W(j, i, k + 1)] - syz[W(j, i, k - 2)]));
    float szz_z = dz * (b1 * (szz[W(j, i, k + 1)] - szz[W(j, i, k)]) + b2 * (szz[W(j, i, k + 2)] - szz[W(j, i, k - 1)]));
    float sxz_x = dx * (b1 * (sxz[W(j, i, k)] - sxz[W(j, i - 1, k)]) + b2 * (sxz[W(j, i + 1, k)] - sxz[W(j, i - 2, k)]));
    float syz_y = dy * (b1 * (syz[W(j, i, k)] - syz[W(j - 1, i, k)]) + b2 * (syz[W(j + 1, i, k)] - syz[W(j - 2, i, k)]));

    int hx = face_x(o, i), hy = face_y(o, j), hz = face_z(o, k);
    int cpml = hx || hy || hz;
    if (hx) {
        float *pxx = &o->ps[0][sx_idx(o, j, hx, k)], *pxy = &o->ps[1][sx_idx(o, j, hx, k)], *pxz = &o->ps[2][sx_idx(o, j, hx, k)];
        *pxx = CP(BH_X, hx) * *pxx + CP(AH_X, hx) * sxx_x; sxx_x = sxx_x / CP(KH_X, hx) + *pxx;
        *pxy = CP(B_X, hx) * *pxy + CP(A_X, hx) * sxy_x;   sxy_x = sxy_x / CP(K_X, hx) + *pxy;
        *pxz = CP(B_X, hx) * *pxz + CP(A_X, hx) * sxz_x;   sxz_x = sxz_x / CP(K_X, hx) + *pxz;
    }
    if (hy) {
        float *pxy = &o->ps[3][sy_idx(o, hy, i, k)], *pyy = &o->ps[4][sy_idx(o, hy, i, k)], *pyz = &o->ps[5][sy_idx(o, hy, i, k)];
        *pxy = CP(B_Y, hy) * *pxy + CP(A_Y, hy) * sxy_y;   sxy_y = sxy_y / CP(K_Y, hy) + *pxy;
        *pyy = CP(BH_Y, hy) * *pyy + CP(AH_Y, hy) * syy_y; syy_y = syy_y / CP(KH_Y, hy) + *pyy;
        *pyz = CP(B_Y, hy) * *pyz + CP(A_Y, hy) * syz_y;   syz_y = syz_y / CP(K_Y, hy) + *pyz;
    }
    if (hz) {
        float *pxz = &o->ps[6][sz_idx(o, j, i, hz)], *pyz = &o->ps[7][sz_idx(o, j, i, hz)], *pzz = &o->ps[8][sz_idx(o, j, i, hz)];
        *pxz = CP(B_Z, hz) * *pxz + CP(A_Z, hz) * sxz_z;   sxz_z = sxz_z / CP(K_Z, hz) + *pxz;
        *pyz = CP(B_Z, hz) * *pyz + CP(A_Z, hz) * syz_z;   syz_z = syz_z / CP(K_Z, hz) + *pyz;
        *pzz = CP(BH_Z, hz) * *pzz + CP(AH_Z, hz) * szz_z; szz_z = szz_z / CP(KH_Z, hz) + *pzz;
    }
    size_t c = W(j, i, k), m = M(j, i, k), n = (size_t)G.nx * G.ny * G.nz;
    const float *rip = o->avg9 + 3 * n, *rjp = o->avg9 + 4 * n, *rkp = o->avg9 + 5 * n;

    /* point forces located in this cell, in list order */
    float amp0 = 0.0f;
    (void)amp0;
    if (cpml) { /* update_v forces run before update_v_CPML touches the frame */
        for (int l = 0; l < npt; l++) {
            if (pts[l].i != i || pts[l].j != j || pts[l].k != k) continue;
            if (back) {
                o->vx[c] += sigx[(size_t)l * p->nt + nt - 1];
                o->vz[c] += sigz[(size_t)l * p->nt + nt - 1];
                o->vy[c] += sigy[(size_t)l * p->nt + nt - 1];
            } else {
                float amp = p->dt * sigx[(size_t)l * p->nt + nt - 1] / (p->dx * p->dy * p->dz);
                switch (pts[l].kind) {
                case 2: o->vx[c] += amp * rip[m]; break;
                case 3: o->vz[c] += amp * rjp[m]; break;
                case 4: o->vy[c] += amp * rkp[m]; break;
                case 5: {
                    float alpha_rad = p->alpha * PI_REF / 180, beta_rad = p->beta * PI_REF / 180;
                    o->vx[c] += cos(beta_rad) * cos(alpha_rad) * amp;
                    o->vy[c] += sin(alpha_rad) * amp;
                    o->vz[c] += sin(beta_rad) * cos(alpha_rad) * amp;
                } break;
                default: break;
                }
            }
        }
    }
    o->vx[c] += (sxx_x + sxy_y + sxz_z) / rip[m];
    o->vy[c] += (syy_y + sxy_x + syz_z) / rjp[m];
    o->vz[c] += (szz_z + sxz_x + syz_y) / rkp[m];
    /* interior: update_v forces after the update; CPML frame: second adjoint injection */
    int passes = cpml ? (back ? 1 : 0) : (back ? 2 : 1);
    for (int pass = 0; pass < passes; pass++) {
        for (int l = 0; l < npt; l++) {
            if (pts[l].i != i || pts[l].j != j || pts[l].k != k) continue;
            if (back) {
                o->vx[c] += sigx[(size_t)l * p->nt + nt - 1];
                o->vz[c] += sigz[(size_t)l * p->nt + nt - 1];
                o->vy[c] += sigy[(size_t)l * p->nt + nt - 1];
            } else {
                float amp = p->dt * sigx[(size_t)l * p->nt + nt - 1] / (p->dx * p->dy * p->dz);
                switch (pts[l].kind) {
                case 2: o->vx[c] += amp * rip[m]; break;
                case 3: o->vz[c] += amp * rjp[m]; break;
                case 4: o->vy[c] += amp * rkp[m]; break;
                case 5: {
                    float alpha_rad = p->alpha * PI_REF / 180, beta_rad = p->beta * PI_REF / 180;
                    o->vx[c] += cos(beta_rad) * cos(alpha_rad) * amp;
                    o->vy[c] += sin(alpha_rad) * amp;
                    o->vz[c] += sin(beta_rad) * cos(alpha_rad) * amp;
                } break;
                default: break;
                }
            }
        }
    }
}

/* Stress update of one cell: update_s_ssg_elastic.c:106-140 (L=0) or
 * update_s_ssg.c:150-230 generalised to L mechanisms, with the CPML psi
 * recursions of update_s_ssg_CPML_elastic.c (including its use of K_y for the
 * front z face, :104-108). */
static void s_cell(orc_t *o, int j, int i, int k) {
    const geo_t G = o->G;
    const ifo_params *p = o->p;
    const float b1 = o->b1, b2 = o->b2;
    const float DX = p->dx, DY = p->dy, DZ = p->dz, DT = p->dt;
    const float *vx = o->vx, *vy = o->vy, *vz = o->vz;
    float vxx = (b1 * (vx[W(j, i, k)] - vx[W(j, i - 1, k)]) + b2 * (vx[W(j, i + 1, k)] - vx[W(j, i - 2, k)])) / DX;
    float vxy = (b1 * (vx[W(j + 1, i, k)] - vx[W(j, i, k)]) + b2 * (vx[W(j + 2, i, k)] - vx[W(j - 1, i, k)])) / DY;
    float vxz = (b1 * (vx[W(j, i, k + 1)] - vx[W(j, i, k)]) + b2 * (vx[W(j, i, k + 2)] - vx[W(j, i, k - 1)])) / DZ;
    float vyx = (b1 * (vy[W(j, i + 1, k)] - vy[W(j, i, k)]) + b2 * (vy[W(j, i + 2, k)] - vy[W(j, i - 1, k)])) / DX;
    float vyy = (b1 * (vy[W(j, i, k)] - vy[W(j - 1, i, k)]) + b2 * (vy[W(j + 1, i, k)] - vy[W(j - 2, i, k)])) / DY;
    float vyz = (b1 * (vy[W(j, i, k + 1)] - vy[W(j, i, k)]) + b2 * (vy[W(j, i, k + 2)] - vy[W(j, i, k - 1)])) / DZ;
    float vzx = (b1 * (vz[W(j, i + 1, k)] - vz[W(j, i, k)]) + b2 * (vz[W(j, i + 2, k)] - vz[W(j, i - 1, k)])) / DX;
    float vzy = (b1 * (vz[W(j + 1, i, k)] - vz[W(j, i, k)]) + b2 * (vz[W(j + 2, i, k)] - vz[W(j - 1, i, k)])) / DY;
    float vzz = (b1 * (vz[W(j, i, k)] - vz[W(j, i, k - 1)]) + b2 * (vz[W(j, i, k + 1)] - vz[W(j, i, k - 2)])) / DZ;

    int hx = face_x(o, i), hy = face_y(o, j), hz = face_z(o, k);
    if (hx) {
        float *a = &o->pv[0][sx_idx(o, j, hx, k)], *b = &o->pv[1][sx_idx(o, j, hx, k)], *c = &o->pv[2][sx_idx(o, j, hx, k)];
        *a = CP(B_X, hx) * *a + CP(A_X, hx) * vxx;   vxx = vxx / CP(K_X, hx) + *a;
        *b = CP(BH_X, hx) * *b + CP(AH_X, hx) * vyx; vyx = vyx / CP(KH_X, hx) + *b;
        *c = CP(BH_X, hx) * *c + CP(AH_X, hx) * vzx; vzx = vzx / CP(KH_X, hx) + *c;
    }
    if (hy) {
        float *a = &o->pv[3][sy_idx(o, hy, i, k)], *b = &o->pv[4][sy_idx(o, hy, i, k)], *c = &o->pv[5][sy_idx(o, hy, i, k)];
        *a = CP(BH_Y, hy) * *a + CP(AH_Y, hy) * vxy; vxy = vxy / CP(KH_Y, hy) + *a;
        *b = CP(B_Y, hy) * *b + CP(A_Y, hy) * vyy;   vyy = vyy / CP(K_Y, hy) + *b;
        *c = CP(BH_Y, hy) * *c + CP(AH_Y, hy) * vzy; vzy = vzy / CP(KH_Y, hy) + *c;
    }
    if (hz) {
        int front = k <= p->fw;
        float *a = &o->pv[6][sz_idx(o, j, i, hz)], *b = &o->pv[7][sz_idx(o, j, i, hz)], *c = &o->pv[8][sz_idx(o, j, i, hz)];
        float kh = front ? CP(KH_Y, hz) : CP(KH_Z, hz), kf = front ? CP(K_Y, hz) : CP(K_Z, hz);
        *a = CP(BH_Z, hz) * *a + CP(AH_Z, hz) * vxz; vxz = vxz / kh + *a;
        *b = CP(BH_Z, hz) * *b + CP(AH_Z, hz) * vyz; vyz = vyz / kh + *b;
        *c = CP(B_Z, hz) * *c + CP(A_Z, hz) * vzz;   vzz = vzz / kf + *c;
    }
    size_t c = W(j, i, k), m = M(j, i, k), n = (size_t)G.nx * G.ny * G.nz;
    const float uipjp = o->avg9[0 * n + m], ujpkp = o->avg9[1 * n + m], uipkp = o->avg9[2 * n + m];
    float vxyyx = vxy + vyx, vyzzy = vyz + vzy, vxzzx = vxz + vzx;
    float vxxyyzz = vxx + vyy + vzz, vyyzz = vyy + vzz, vxxzz = vxx + vzz, vxxyy = vxx + vyy;
    const int L = p->nmech;
    if (L == 0) {
        float fipjp = uipjp * DT, fjpkp = ujpkp * DT, fipkp = uipkp * DT;
        float g = o->pi[m], f = 2.0 * o->u[m];
        o->sxy[c] += (fipjp * vxyyx);
        o->syz[c] += (fjpkp * vyzzy);
        o->sxz[c] += (fipkp * vxzzx);
        o->sxx[c] += DT * ((g * vxxyyzz) - (f * vyyzz));
        o->syy[c] += DT * ((g * vxxyyzz) - (f * vxxzz));
        o->szz[c] += DT * ((g * vxxyyzz) - (f * vxxyy));
        return;
    }
    const float tausipjp = o->avg9[6 * n + m], tausjpkp = o->avg9[7 * n + m], tausipkp = o->avg9[8 * n + m];
    const float taus = o->taus[m], taup = o->taup[m], pim = o->pi[m], um = o->u[m];
    float dthalbe = DT / 2.0;
    /* memory-variable sums (update_s_ssg.c:157-162 for one mechanism) */
    float sr[6];
    for (int q = 0; q < 6; q++) {
        sr[q] = o->r[0][q][m];
        for (int l = 1; l < L; l++) sr[q] += o->r[l][q][m];
    }
    float fipjp = uipjp * DT * (1.0 + L * tausipjp);
    float fjpkp = ujpkp * DT * (1.0 + L * tausjpkp);
    float fipkp = uipkp * DT * (1.0 + L * tausipkp);
    float g = pim * (1.0 + L * taup);
    float f = 2.0 * um * (1.0 + L * taus);
    /* r order: 0 rxx, 1 ryy, 2 rzz, 3 rxy, 4 ryz, 5 rxz */
    o->sxy[c] += (fipjp * vxyyx) + (dthalbe * sr[3]);
    o->syz[c] += (fjpkp * vyzzy) + (dthalbe * sr[4]);
    o->sxz[c] += (fipkp * vxzzx) + (dthalbe * sr[5]);
    o->sxx[c] += DT * ((g * vxxyyzz) - (f * vyyzz)) + (dthalbe * sr[0]);
    o->syy[c] += DT * ((g * vxxyyzz) - (f * vxxzz)) + (dthalbe * sr[1]);
    o->szz[c] += DT * ((g * vxxyyzz) - (f * vxxyy)) + (dthalbe * sr[2]);
    for (int l = 0; l < L; l++) {
        float eta = o->eta[l];
        float b = 1.0 / (1.0 + (eta * 0.5));
        float cc = 1.0 - (eta * 0.5);
        float dipjp = uipjp * eta * tausipjp, djpkp = ujpkp * eta * tausjpkp, dipkp = uipkp * eta * tausipkp;
        float d = 2.0 * um * eta * taus;
        float e = pim * eta * taup;
        float *r = NULL;
        r = &o->r[l][3][m]; *r = b * (*r * cc - (dipjp * vxyyx));
        r = &o->r[l][4][m]; *r = b * (*r * cc - (djpkp * vyzzy));
        r = &o->r[l][5][m]; *r = b * (*r * cc - (dipkp * vxzzx));
        r = &o->r[l][0][m]; *r = b * (*r * cc - (e * vxxyyzz) + (d * vyyzz));
        r = &o->r[l][1][m]; *r = b * (*r * cc - (e * vxxyyzz) + (d * vxxzz));
        r = &o->r[l][2][m]; *r = b * (*r * cc - (e * vxxyyzz) + (d * vxxyy));
    }
    for (int q = 0; q < 6; q++) {
        sr[q] = o->r[0][q][m];
        for (int l = 1; l < L; l++) sr[q] += o->r[l][q][m];
    }
    o->sxy[c] += (dthalbe * sr[3]);
    o->syz[c] += (dthalbe * sr[4]);
    o->sxz[c] += (dthalbe * sr[5]);
    o->sxx[c] += (dthalbe * sr[0]);
    o->syy[c] += (dthalbe * sr[1]);
    o->szz[c] += (dthalbe * sr[2]);
}

/* Free surface at j=1: surface_ssg_elastic.c:69-111 / surface_ssg.c:117-160. */
static void surface_cell(orc_t *o, int i, int k) {
    const geo_t G = o->G;
    const ifo_params *p = o->p;
    const float b1 = o->b1, b2 = o->b2;
    const float DX = p->dx, DY = p->dy, DZ = p->dz, DT = p->dt;
    const int j = 1;
    size_t c = W(j, i, k), m = M(j, i, k);
    o->syy[c] = 0.0;
    for (int q = 0; q < p->nmech; q++) o->r[q][1][m] = 0.0;
    for (int mm = 1; mm <= 2; mm++) {
        o->syy[W(j - mm, i, k)] = -o->syy[W(j + mm, i, k)];
        o->sxy[W(j - mm, i, k)] = -o->sxy[W(j + mm - 1, i, k)];
        o->syz[W(j - mm, i, k)] = -o->syz[W(j + mm - 1, i, k)];
    }
    const float *vx = o->vx, *vy = o->vy, *vz = o->vz;
    float vxx = (b1 * (vx[W(j, i, k)] - vx[W(j, i - 1, k)]) + b2 * (vx[W(j, i + 1, k)] - vx[W(j, i - 2, k)])) / DX;
    float vyy = (b1 * (vy[W(j, i, k)] - vy[W(j - 1, i, k)]) + b2 * (vy[W(j + 1, i, k)] - vy[W(j - 2, i, k)])) / DY;
    float vzz = (b1 * (vz[W(j, i, k)] - vz[W(j, i, k - 1)]) + b2 * (vz[W(j, i, k + 1)] - vz[W(j, i, k - 2)])) / DZ;
    const int L = p->nmech;
    if (L == 0) {
        float f = o->u[m] * 2.0, g = o->pi[m];
        float h = -(DT * (g - f) * (g - f) * (vxx + vzz) / g) - (DT * (g - f) * vyy);
        o->sxx[c] += h;
        o->szz[c] += h;
        return;
    }
    float dthalbe = DT / 2.0;
    float taus = o->taus[m], taup = o->taup[m], um = o->u[m], pim = o->pi[m];
    float f = um * 2.0 * (1.0 + L * taus);
    float g = pim * (1.0 + L * taup);
    float h = -(DT * (g - f) * (g - f) * (vxx + vzz) / g) - (DT * (g - f) * vyy);
    float srx = o->r[0][0][m], srz = o->r[0][2][m];
    for (int l = 1; l < L; l++) { srx += o->r[l][0][m]; srz += o->r[l][2][m]; }
    o->sxx[c] += h - (dthalbe * srx);
    o->szz[c] += h - (dthalbe * srz);
    for (int l = 0; l < L; l++) {
        float b = o->eta[l] / (1.0 + (o->eta[l] * 0.5));
        float d = 2.0 * um * taus;
        float e = pim * taup;
        float hh = b * (((d - e) * ((f / g) - 1.0) * (vxx + vzz)) - ((d - e) * vyy));
        o->r[l][0][m] += hh;
        o->r[l][2][m] += hh;
    }
    srx = o->r[0][0][m]; srz = o->r[0][2][m];
    for (int l = 1; l < L; l++) { srx += o->r[l][0][m]; srz += o->r[l][2][m]; }
    o->sxx[c] += (dthalbe * srx);
    o->szz[c] += (dthalbe * srz);
}

static int orc_init(orc_t *o, const ifo_params *p, const float *rho, const float *pi, const float *u,
                    const float *taus, const float *taup, const float *eta, const float *cpml) {
    memset(o, 0, sizeof *o);
    if (p->nmech > MAXMECH || p->nmech < 0) return 2;
    if (p->nx < 2 * p->fw + 1 || p->ny < 2 * p->fw + 1 || p->nz < 2 * p->fw + 1) return 1;
    o->p = p;
    o->G = mkgeo(p);
    fd_coeffs(p, &o->b1, &o->b2);
    geo_t G = o->G;
    size_t n = (size_t)G.nx * G.ny * G.nz;
    o->pi = pi; o->u = u; o->taus = taus; o->taup = taup; o->cp = cpml;
    for (int l = 0; l < p->nmech; l++) o->eta[l] = eta[l];
    o->avg9 = calloc(9 * n, sizeof(float));
    ifo_av_mat(p, rho, pi, u, taus, taup, o->avg9);
    float **f9[9] = {&o->vx, &o->vy, &o->vz, &o->sxx, &o->syy, &o->szz, &o->sxy, &o->syz, &o->sxz};
    for (int q = 0; q < 9; q++) *f9[q] = calloc(G.wn, sizeof(float));
    for (int l = 0; l < p->nmech; l++)
        for (int q = 0; q < 6; q++) o->r[l][q] = calloc(n, sizeof(float));
    size_t nsx = (size_t)G.ny * 2 * p->fw * G.nz, nsy = (size_t)2 * p->fw * G.nx * G.nz, nsz = (size_t)G.ny * G.nx * 2 * p->fw;
    for (int q = 0; q < 3; q++) {
        o->ps[q] = calloc(nsx, sizeof(float)); o->pv[q] = calloc(nsx, sizeof(float));
        o->ps[q + 3] = calloc(nsy, sizeof(float)); o->pv[q + 3] = calloc(nsy, sizeof(float));
        o->ps[q + 6] = calloc(nsz, sizeof(float)); o->pv[q + 6] = calloc(nsz, sizeof(float));
    }
    return 0;
}

static void orc_free(orc_t *o) {
    float *f9[9] = {o->vx, o->vy, o->vz, o->sxx, o->syy, o->szz, o->sxy, o->syz, o->sxz};
    for (int q = 0; q < 9; q++) free(f9[q]);
    for (int l = 0; l < MAXMECH; l++)
        for (int q = 0; q < 6; q++) free(o->r[l][q]);
    for (int q = 0; q < 9; q++) { free(o->ps[q]); free(o->pv[q]); }
    free(o->avg9);
}

static void orc_state_out(orc_t *o, float *state9) {
    if (!state9) return;
    float *f9[9] = {o->vx, o->vy, o->vz, o->sxx, o->syy, o->szz, o->sxy, o->syz, o->sxz};
    for (int q = 0; q < 9; q++) memcpy(state9 + q * o->G.wn, f9[q], sizeof(float) * o->G.wn);
}

/* disc_fourier.c:28-61 */
typedef struct {
    orc_t *o;
    float *F[6];
    double trig1, trig2;
} dft_ctx;

static void dft_rows(void *vc, int j0, int j1) {
    dft_ctx *d = vc;
    orc_t *o = d->o;
    const geo_t G = o->G;
    for (int j = j0; j <= j1; j++)
        for (int i = 1; i <= G.nx; i++)
            for (int k = 1; k <= G.nz; k++) {
                size_t c = W(j, i, k);
                d->F[0][c] += o->vx[c] * d->trig1;
                d->F[1][c] += o->vy[c] * d->trig1;
                d->F[2][c] += o->vz[c] * d->trig1;
                d->F[3][c] += o->vx[c] * d->trig2;
                d->F[4][c] += o->vy[c] * d->trig2;
                d->F[5][c] += o->vz[c] * d->trig2;
            }
}

static void dft_step(orc_t *o, int nt, int back, int nf, const float *finv, int ntast, float *dft) {
    const geo_t G = o->G;
    const ifo_params *p = o->p;
    float t = 0.0;
    if (back == 0) t = nt * p->dt;
    if (back == 1) t = p->time - nt * p->dt;
    for (int l = 0; l < nf; l++) {
        dft_ctx d;
        d.o = o;
        d.trig1 = cos(2.0 * t * finv[l] * M_PI) * p->dt * ntast;
        d.trig2 = sin(2.0 * t * finv[l] * M_PI) * p->dt * ntast;
        for (int q = 0; q < 6; q++) d.F[q] = dft + ((size_t)q * nf + l) * G.wn;
        par_rows(1, G.ny, dft_rows, &d);
    }
}

/* psource.c:38-52: explosive source amplitude at step nt */
static float psource_amp(const ifo_params *p, const float *s, int nt) {
    float amp = 0.0;
    if (nt == 1) amp = s[nt + 1 - 1] / (2.0 * p->dx * p->dy * p->dz);
    if ((nt > 1) && (nt < p->nt)) amp = (s[nt + 1 - 1] - s[nt - 1 - 1]) / (2.0 * p->dx * p->dy * p->dz);
    if (nt == p->nt) amp = -s[nt - 1 - 1] / (2.0 * p->dx * p->dy * p->dz);
    return amp;
}

typedef struct {
    orc_t *o;
    int nt, back, npt;
    const pt_t *pts;
    const float *sigx, *sigy, *sigz;
} vrow_ctx;

static void v_rows(void *vc, int j0, int j1) {
    vrow_ctx *v = vc;
    const geo_t G = v->o->G;
    for (int j = j0; j <= j1; j++)
        for (int i = 1; i <= G.nx; i++)
            for (int k = 1; k <= G.nz; k++) v_cell(v->o, j, i, k, v->nt, v->back, v->npt, v->pts, v->sigx, v->sigy, v->sigz);
}

static void s_rows(void *vc, int j0, int j1) {
    orc_t *o = vc;
    const geo_t G = o->G;
    for (int j = j0; j <= j1; j++)
        for (int i = 1; i <= G.nx; i++)
            for (int k = 1; k <= G.nz; k++) s_cell(o, j, i, k);
}

static void surface_cols(void *vc, int k0, int k1) {
    orc_t *o = vc;
    for (int k = k0; k <= k1; k++)
        for (int i = 1; i <= o->G.nx; i++) surface_cell(o, i, k);
}

static void run_loop(orc_t *o, int back, int npt, const pt_t *pts, const float *sigx, const float *sigy,
                     const float *sigz, int ntr, const int *recpos, float *sections,
                     int nf, const float *finv, int ntast, float *dft) {
    const geo_t G = o->G;
    const ifo_params *p = o->p;
    int ns = ifo_nsamples(p), lsamp = p->ndtshift + 1, nlsamp = 1;
    for (int nt = 1; nt <= p->nt; nt++) {
        vrow_ctx vc = {o, nt, back, npt, pts, sigx, sigy, sigz};
        par_rows(1, G.ny, v_rows, &vc);
        par_rows(1, G.ny, s_rows, o);
        if (!back)
            for (int l = 0; l < npt; l++)
                if (pts[l].kind == 1) {
                    float amp = psource_amp(p, sigx + (size_t)l * p->nt, nt);
                    size_t c = W(pts[l].j, pts[l].i, pts[l].k);
                    o->sxx[c] += amp; o->syy[c] += amp; o->szz[c] += amp;
                }
        if (nf > 0 && nt % ntast == 0) dft_step(o, nt, back, nf, finv, ntast, dft);
        if (p->free_surf) par_rows(1, G.nz, surface_cols, o);
        if (ntr > 0 && nt == lsamp) {
            if (sections && nlsamp <= ns)
                for (int t = 0; t < ntr; t++) {
                    size_t c = W(recpos[t * 3 + 1], recpos[t * 3 + 0], recpos[t * 3 + 2]);
                    sections[((size_t)0 * ntr + t) * ns + nlsamp - 1] = o->vx[c];
                    sections[((size_t)1 * ntr + t) * ns + nlsamp - 1] = o->vy[c];
                    sections[((size_t)2 * ntr + t) * ns + nlsamp - 1] = o->vz[c];
                }
            nlsamp++;
            lsamp += p->ndt;
        }
    }
}

int ifo_forward(const ifo_params *p, const float *rho, const float *pi, const float *u,
                const float *taus, const float *taup, const float *eta, const float *cpml,
                int nsrc, const float *srcpos, const float *signals,
                int ntr, const int *recpos, int nf, const float *finv, int ntast,
                float *sections, float *dft, float *state9) {
    orc_t o;
    int rc = orc_init(&o, p, rho, pi, u, taus, taup, eta, cpml);
    if (rc) return rc;
    pt_t *pts = malloc(sizeof(pt_t) * (size_t)(nsrc > 0 ? nsrc : 1));
    for (int l = 0; l < nsrc; l++) {
        pts[l].i = (int)srcpos[l * 7 + 0];
        pts[l].j = (int)srcpos[l * 7 + 1];
        pts[l].k = (int)srcpos[l * 7 + 2];
        pts[l].kind = (int)srcpos[l * 7 + 6];
    }
    float *F = NULL;
    if (nf > 0) F = dft ? dft : calloc((size_t)6 * nf * o.G.wn, sizeof(float));
    if (F && F == dft) memset(F, 0, sizeof(float) * (size_t)6 * nf * o.G.wn);
    run_loop(&o, 0, nsrc, pts, signals, signals, signals, ntr, recpos, sections, nf, finv, ntast, F);
    if (F && F != dft) free(F);
    orc_state_out(&o, state9);
    free(pts);
    orc_free(&o);
    return 0;
}

/* residual.c:35-60 */
int ifo_residual(const ifo_params *p, int ntr, const float *obs, const float *syn, float *diff, float *l2) {
    int ns = ifo_nsamples(p);
    float L2 = *l2;
    for (int c = 0; c < 3; c++)
        for (int t = 0; t < ntr; t++) {
            const float *d = obs + ((size_t)c * ntr + t) * ns, *s = syn + ((size_t)c * ntr + t) * ns;
            float *o = diff + ((size_t)c * ntr + t) * ns;
            float vdiff = 0.0;
            for (int j = 1; j <= ns; j++) {
                vdiff += s[j - 1] - d[j - 1];
                o[ns - j] = p->dt * vdiff;
                L2 += fabs(o[ns - j] * o[ns - j]);
            }
        }
    *l2 = L2;
    return 0;
}

int ifo_adjoint(const ifo_params *p, const float *rho, const float *pi, const float *u,
                const float *taus, const float *taup, const float *eta, const float *cpml,
                int ntr, const int *recpos, const float *diff,
                int nf, const float *finv, int ntast, float *dft_back, float *state9) {
    if (p->ndt != 1 || p->ndtshift != 0) return 3;
    orc_t o;
    int rc = orc_init(&o, p, rho, pi, u, taus, taup, eta, cpml);
    if (rc) return rc;
    int ns = ifo_nsamples(p);
    pt_t *pts = malloc(sizeof(pt_t) * (size_t)(ntr > 0 ? ntr : 1));
    for (int t = 0; t < ntr; t++) {
        pts[t].i = recpos[t * 3 + 0]; pts[t].j = recpos[t * 3 + 1]; pts[t].k = recpos[t * 3 + 2];
        pts[t].kind = 6;
    }
    const float *dx = diff, *dy = diff + (size_t)ntr * ns, *dz = diff + (size_t)2 * ntr * ns;
    float *F = NULL;
    if (nf > 0) F = dft_back ? dft_back : calloc((size_t)6 * nf * o.G.wn, sizeof(float));
    if (F && F == dft_back) memset(F, 0, sizeof(float) * (size_t)6 * nf * o.G.wn);
    run_loop(&o, 1, ntr, pts, dx, dy, dz, 0, recpos, NULL, nf, finv, ntast, F);
    if (F && F != dft_back) free(F);
    orc_state_out(&o, state9);
    free(pts);
    orc_free(&o);
    return 0;
}

/* gradient_F.c:62-139 */
/* gradient_F.c:30-171 for one frequency, rows j0..j1 */
typedef struct {
    const ifo_params *p;
    geo_t G;
    float b1, b2, fdummy;
    const float *f[6], *bk[6];
    const float *rho, *pi, *u;
    float *grad;
} grad_ctx;

static void grad_rows(void *vc, int j0, int j1) {
    const grad_ctx *q = vc;
    const geo_t G = q->G;
    const float b1 = q->b1, b2 = q->b2, fdummy = q->fdummy;
    const float DX = q->p->dx, DY = q->p->dy, DZ = q->p->dz;
    const float *const *f = q->f, *const *bk = q->bk;
    const float *rho = q->rho, *pi = q->pi, *u = q->u;
    float *grad = q->grad;
    const size_t n = (size_t)G.nx * G.ny * G.nz;
    for (int j = j0; j <= j1; j++)
        for (int i = 1; i <= G.nx; i++)
            for (int k = 1; k <= G.nz; k++) {
                float d[4][9]; /* fwd re, back re, fwd im, back im; xx xy xz yx yy yz zx zy zz */
                const float *src[4][3] = {{f[0], f[1], f[2]}, {bk[0], bk[1], bk[2]}, {f[3], f[4], f[5]}, {bk[3], bk[4], bk[5]}};
                for (int s = 0; s < 4; s++) {
                    const float *X = src[s][0], *Y = src[s][1], *Z = src[s][2];
                    d[s][0] = (b1 * (X[W(j, i, k)] - X[W(j, i - 1, k)]) + b2 * (X[W(j, i + 1, k)] - X[W(j, i - 2, k)])) / DX;
                    d[s][1] = (b1 * (X[W(j + 1, i, k)] - X[W(j, i, k)]) + b2 * (X[W(j + 2, i, k)] - X[W(j - 1, i, k)])) / DY;
                    d[s][2] = (b1 * (X[W(j, i, k + 1)] - X[W(j, i, k)]) + b2 * (X[W(j, i, k + 2)] - X[W(j, i, k - 1)])) / DZ;
                    d[s][3] = (b1 * (Y[W(j, i + 1, k)] - Y[W(j, i, k)]) + b2 * (Y[W(j, i + 2, k)] - Y[W(j, i - 1, k)])) / DX;
                    d[s][4] = (b1 * (Y[W(j, i, k)] - Y[W(j - 1, i, k)]) + b2 * (Y[W(j + 1, i, k)] - Y[W(j - 2, i, k)])) / DY;
                    d[s][5] = (b1 * (Y[W(j, i, k + 1)] - Y[W(j, i, k)]) + b2 * (Y[W(j, i, k + 2)] - Y[W(j, i, k - 1)])) / DZ;
                    d[s][6] = (b1 * (Z[W(j, i + 1, k)] - Z[W(j, i, k)]) + b2 * (Z[W(j, i + 2, k)] - Z[W(j, i - 1, k)])) / DX;
                    d[s][7] = (b1 * (Z[W(j + 1, i, k)] - Z[W(j, i, k)]) + b2 * (Z[W(j + 2, i, k)] - Z[W(j - 1, i, k)])) / DY;
                    d[s][8] = (b1 * (Z[W(j, i, k)] - Z[W(j, i, k - 1)]) + b2 * (Z[W(j, i, k + 1)] - Z[W(j, i, k - 2)])) / DZ;
                }
                float *fv = d[0], *bv = d[1], *fi = d[2], *bi = d[3];
                float gradlam = 0.0, gradmu = 0.0, gradrho = 0.0;
                gradlam = (fv[0] + fv[4] + fv[8]) * (bv[0] + bv[4] + bv[8]) + (fi[0] + fi[4] + fi[8]) * (bi[0] + bi[4] + bi[8]);
                gradlam = -gradlam * fdummy;
                gradmu = 2 * fv[0] * bv[0] + 2 * fv[4] * bv[4] + 2 * fv[8] * bv[8] + 2 * fi[0] * bi[0] + 2 * fi[4] * bi[4] +
                         2 * fi[8] * bi[8] + (fv[1] + fv[3]) * (bv[1] + bv[3]) + (fi[1] + fi[3]) * (bi[1] + bi[3]) +
                         (fv[2] + fv[6]) * (bv[2] + bv[6]) + (fi[2] + fi[6]) * (bi[2] + bi[6]) +
                         (fv[5] + fv[7]) * (bv[5] + bv[7]) + (fi[5] + fi[7]) * (bi[5] + bi[7]);
                gradmu = -gradmu * fdummy;
                size_t c = W(j, i, k), m = M(j, i, k);
                gradrho = (f[0][c] * bk[0][c] + f[1][c] * bk[1][c] + f[2][c] * bk[2][c]) +
                          (f[3][c] * bk[3][c] + f[4][c] * bk[4][c] + f[5][c] * bk[5][c]);
                float r = rho[m], pp = pi[m], uu = u[m];
                grad[0 * n + m] += sqrt(r * pp) * 2 * gradlam;
                grad[1 * n + m] += -4 * sqrt(r * uu) * gradlam + 2 * sqrt(r * uu) * gradmu;
                grad[2 * n + m] += gradrho + uu / r * gradmu + (pp - 2 * uu) / r * gradlam;
            }
}

int ifo_gradient(const ifo_params *p, const float *rho, const float *pi, const float *u,
                 int nf, const float *finv, const float *dft_fwd, const float *dft_back, float *grad) {
    grad_ctx q;
    q.p = p;
    q.G = mkgeo(p);
    fd_coeffs(p, &q.b1, &q.b2);
    q.rho = rho;
    q.pi = pi;
    q.u = u;
    q.grad = grad;
    for (int l = 0; l < nf; l++) {
        float fdummy = 0.0;
        fdummy = 2.0 * 2.0 * finv[l] * finv[l] * M_PI * M_PI;
        fdummy = 1 / fdummy;
        q.fdummy = fdummy;
        for (int c = 0; c < 6; c++) {
            q.f[c] = dft_fwd + ((size_t)c * nf + l) * q.G.wn;
            q.bk[c] = dft_back + ((size_t)c * nf + l) * q.G.wn;
        }
        par_rows(1, q.G.ny, grad_rows, &q);
    }
    return 0;
}
