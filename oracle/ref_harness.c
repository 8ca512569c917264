/*
 * Reference harness — TEST INFRASTRUCTURE ONLY (the CPU oracle).
 *
 * Drives the UNMODIFIED reference functions (compiled from the reference's
 * src/ by oracle/Makefile, with the one-rank MPI of ifos3d-dev_b200/host/mpi1)
 * through flat arrays, in the call order of the reference driver:
 *   forward   : src/ifos3d.c:738-814  (zero_wavefield, zero_invers, NT loop of
 *               update_v, update_v_CPML, update_s_elastic, update_s_CPML_elastic,
 *               psource, discfourier, surface_elastic, seismo)
 *   residual  : src/ifos3d.c:837-858
 *   adjoint   : src/ifos3d.c:882-960  (residual injected at receivers, back=1)
 *   gradient  : src/ifos3d.c:974       (gradient_F)
 * With nmech==1 the stress update switches to the viscoelastic functions
 * update_s / update_s_CPML / surface, whose calls the reference driver keeps
 * commented out (src/ifos3d.c:773, 777, 796); the reference supports L<=1 only.
 *
 * This file is compiled against the reference headers (fd.h, globvar.h), so the
 * globals it sets are the reference's own.
 */
#include "fd.h"
#include "globvar.h"
#include "ifos_oracle.h"

#include <stdint.h>
#include <unistd.h>

float readdsk(FILE *fp_in, int format);

static FILE *g_null = NULL;

static void set_globals(const ifo_params *p) {
    if (!g_null) g_null = fopen("/dev/null", "w");
    FP = g_null;
    FI = g_null;
    NX = NXG = IENDX = p->nx;
    NY = NYG = IENDY = p->ny;
    NZ = NZG = IENDZ = p->nz;
    DX = p->dx; DY = p->dy; DZ = p->dz;
    DT = p->dt; NT = p->nt; TIME = p->time;
    FDORDER = 4; FDCOEFF = p->fdcoeff;
    FREE_SURF = p->free_surf; FW = p->fw; L = p->nmech;
    ABS_TYPE = 1; SEISMO = 1;
    NDT = p->ndt; NDTSHIFT = p->ndtshift;
    VPPML = p->vppml; FPML = p->fpml;
    ALPHA = p->alpha; BETA = p->beta;
    SOURCE_SHAPE = p->source_shape;
    POS[1] = POS[2] = POS[3] = 0;
    NPROCX = NPROCY = NPROCZ = NPROC = NP = 1;
    MYID = 0; VERBOSE = 0; METHOD = 1; F_INV = 0.0f;
    for (int i = 0; i < 7; i++) INDEX[i] = MPI_PROC_NULL;
}

int ifo_nsamples(const ifo_params *p) {
    if (p->ndtshift > p->nt) return 0;
    return (int)ceil((float)(p->nt - p->ndtshift) / (float)p->ndt); /* src/ifos3d.c:178-179 */
}

/* ---- flat <-> NR tensor helpers ------------------------------------------ */
#define WY (p->ny + 5)
#define WX (p->nx + 4)
#define WZ (p->nz + 4)

static float ***alloc_w(const ifo_params *p, int jlo) {
    return f3tensor(jlo, p->ny + 2, -1, p->nx + 2, -1, p->nz + 2);
}
static void free_w(const ifo_params *p, float ***t, int jlo) {
    free_f3tensor(t, jlo, p->ny + 2, -1, p->nx + 2, -1, p->nz + 2);
}
/* copy tensor allocated from plane jlo into a flat W array starting at j=-2 */
static void w_out(const ifo_params *p, float ***t, int jlo, float *dst) {
    size_t plane = (size_t)WX * WZ;
    memset(dst, 0, sizeof(float) * plane * WY);
    memcpy(dst + (size_t)(jlo + 2) * plane, &t[jlo][-1][-1],
           sizeof(float) * plane * (size_t)(p->ny + 2 - jlo + 1));
}
static float ***alloc_m(const ifo_params *p) {
    return f3tensor(0, p->ny + 1, 0, p->nx + 1, 0, p->nz + 1);
}
static void m_in(const ifo_params *p, float ***t, const float *src) {
    for (int j = 1; j <= p->ny; j++)
        for (int i = 1; i <= p->nx; i++)
            memcpy(&t[j][i][1], src + ((size_t)(j - 1) * p->nx + (i - 1)) * p->nz, sizeof(float) * p->nz);
}
static float ***alloc_g(const ifo_params *p) { return f3tensor(1, p->ny, 1, p->nx, 1, p->nz); }
static void free_g(const ifo_params *p, float ***t) { free_f3tensor(t, 1, p->ny, 1, p->nx, 1, p->nz); }
static void g_out(const ifo_params *p, float ***t, float *dst) {
    memcpy(dst, &t[1][1][1], sizeof(float) * (size_t)p->nx * p->ny * p->nz);
}
static void g_in(const ifo_params *p, float ***t, const float *src) {
    memcpy(&t[1][1][1], src, sizeof(float) * (size_t)p->nx * p->ny * p->nz);
}
static float ****alloc_f(const ifo_params *p, int nf) {
    return f4tensor(1, nf, -2, p->ny + 2, -1, p->nx + 2, -1, p->nz + 2);
}
static void free_f(const ifo_params *p, float ****t, int nf) {
    free_f4tensor(t, 1, nf, -2, p->ny + 2, -1, p->nx + 2, -1, p->nz + 2);
}
static size_t wsize(const ifo_params *p) { return (size_t)WX * WY * WZ; }

/* ---- model & CPML ---------------------------------------------------------- */
typedef struct {
    float ***rho, ***pi, ***u, ***taus, ***taup, *eta;
    float ***uipjp, ***ujpkp, ***uipkp, ***tausipjp, ***tausjpkp, ***tausipkp, ***rip, ***rjp, ***rkp;
} refmodel;

static void model_setup(const ifo_params *p, refmodel *m, const float *rho, const float *pi, const float *u,
                        const float *taus, const float *taup, const float *eta) {
    m->rho = alloc_m(p); m->pi = alloc_m(p); m->u = alloc_m(p);
    m_in(p, m->rho, rho); m_in(p, m->pi, pi); m_in(p, m->u, u);
    m->taus = m->taup = NULL; m->eta = NULL;
    m->tausipjp = m->tausjpkp = m->tausipkp = NULL;
    if (p->nmech) {
        m->taus = alloc_m(p); m->taup = alloc_m(p);
        m_in(p, m->taus, taus); m_in(p, m->taup, taup);
        m->eta = vector(1, p->nmech);
        for (int l = 1; l <= p->nmech; l++) m->eta[l] = eta ? eta[l - 1] : 0.0f;
        m->tausipjp = alloc_g(p); m->tausjpkp = alloc_g(p); m->tausipkp = alloc_g(p);
    }
    m->uipjp = alloc_g(p); m->ujpkp = alloc_g(p); m->uipkp = alloc_g(p);
    m->rip = alloc_g(p); m->rjp = alloc_g(p); m->rkp = alloc_g(p);
    matcopy(m->rho, m->pi, m->u, m->taus, m->taup);                        /* src/ifos3d.c:681 */
    av_mat(m->rho, m->pi, m->u, m->taus, m->taup, m->uipjp, m->ujpkp, m->uipkp,
           m->tausipjp, m->tausjpkp, m->tausipkp, m->rjp, m->rkp, m->rip);  /* src/ifos3d.c:683 */
}

static void model_free(const ifo_params *p, refmodel *m) {
    free_f3tensor(m->rho, 0, p->ny + 1, 0, p->nx + 1, 0, p->nz + 1);
    free_f3tensor(m->pi, 0, p->ny + 1, 0, p->nx + 1, 0, p->nz + 1);
    free_f3tensor(m->u, 0, p->ny + 1, 0, p->nx + 1, 0, p->nz + 1);
    if (p->nmech) {
        free_f3tensor(m->taus, 0, p->ny + 1, 0, p->nx + 1, 0, p->nz + 1);
        free_f3tensor(m->taup, 0, p->ny + 1, 0, p->nx + 1, 0, p->nz + 1);
        free_vector(m->eta, 1, p->nmech);
        free_g(p, m->tausipjp); free_g(p, m->tausjpkp); free_g(p, m->tausipkp);
    }
    free_g(p, m->uipjp); free_g(p, m->ujpkp); free_g(p, m->uipkp);
    free_g(p, m->rip); free_g(p, m->rjp); free_g(p, m->rkp);
}

typedef struct { float *v[24]; } refcpml; /* K,alpha',a,b x2 (full, half) per direction, CPML_coeff order */

static void cpml_alloc(const ifo_params *p, refcpml *c) {
    for (int n = 0; n < 24; n++) c->v[n] = vector(1, 2 * p->fw);
}
static void cpml_free(const ifo_params *p, refcpml *c) {
    for (int n = 0; n < 24; n++) free_vector(c->v[n], 1, 2 * p->fw);
}
/* CPML_coeff argument order: K, alpha', a, b, K_half, alpha'_half, a_half, b_half per direction.
 * Flat order (ifos_oracle.h): K, a, b, K_half, a_half, b_half per direction. */
static const int cpml_map[18] = {0, 2, 3, 4, 6, 7, 8, 10, 11, 12, 14, 15, 16, 18, 19, 20, 22, 23};
static void cpml_load(const ifo_params *p, refcpml *c, const float *flat) {
    for (int n = 0; n < 18; n++)
        for (int h = 1; h <= 2 * p->fw; h++) c->v[cpml_map[n]][h] = flat[(size_t)n * 2 * p->fw + h - 1];
}

int ifo_cpml_coeff(const ifo_params *p, float *flat) {
    set_globals(p);
    refcpml c; cpml_alloc(p, &c);
    CPML_coeff(c.v[0], c.v[1], c.v[2], c.v[3], c.v[4], c.v[5], c.v[6], c.v[7],
               c.v[8], c.v[9], c.v[10], c.v[11], c.v[12], c.v[13], c.v[14], c.v[15],
               c.v[16], c.v[17], c.v[18], c.v[19], c.v[20], c.v[21], c.v[22], c.v[23]);
    for (int n = 0; n < 18; n++)
        for (int h = 1; h <= 2 * p->fw; h++) flat[(size_t)n * 2 * p->fw + h - 1] = c.v[cpml_map[n]][h];
    cpml_free(p, &c);
    return 0;
}

static float **srcpos_matrix(int nsrc, const float *srcpos) {
    float **s = fmatrix(1, 7, 1, nsrc > 0 ? nsrc : 1);
    for (int l = 1; l <= nsrc; l++)
        for (int r = 1; r <= 7; r++) s[r][l] = srcpos[(size_t)(l - 1) * 7 + r - 1];
    return s;
}

int ifo_wavelet(const ifo_params *p, int nsrc, const float *srcpos, float *signals) {
    set_globals(p);
    float **s = srcpos_matrix(nsrc, srcpos);
    float **sig = fmatrix(1, nsrc, 1, p->nt);
    wavelet(s, nsrc, p->source_shape, sig);
    for (int l = 1; l <= nsrc; l++) memcpy(signals + (size_t)(l - 1) * p->nt, &sig[l][1], sizeof(float) * p->nt);
    free_matrix(sig, 1, nsrc, 1, p->nt);
    free_matrix(s, 1, 7, 1, nsrc > 0 ? nsrc : 1);
    return 0;
}

int ifo_readmod(const ifo_params *p, const ifo_velmodel *vm, float *rho, float *pi, float *u,
                float *taus, float *taup, float *eta) {
    set_globals(p);
    /* write the three model files in the reference's binary layout [z][x][y] (readmod.c:99-105) */
    char base[] = "/tmp/ifoXXXXXX";
    int fd = mkstemp(base);
    if (fd < 0) return 1;
    close(fd);
    const char *ext[3] = {"vp", "vs", "rho"};
    const float *src[3] = {vm->vp, vm->vs, vm->rho};
    for (int f = 0; f < 3; f++) {
        char name[128];
        snprintf(name, sizeof name, "%s.%s", base, ext[f]);
        FILE *fp = fopen(name, "wb");
        if (!fp) return 1;
        for (int k = 0; k < p->nz; k++)
            for (int i = 0; i < p->nx; i++)
                for (int j = 0; j < p->ny; j++)
                    fwrite(src[f] + ((size_t)j * p->nx + i) * p->nz + k, sizeof(float), 1, fp);
        fclose(fp);
    }
    snprintf(MFILE, STRING_SIZE, "%s", base);
    int lv = p->nmech > 0 ? p->nmech : 1;
    FL = vector(1, lv);
    for (int l = 1; l <= p->nmech; l++) FL[l] = vm->fl[l - 1];
    TAU = vm->tau;
    float ***r = alloc_m(p), ***pp = alloc_m(p), ***uu = alloc_m(p), ***ts = NULL, ***tp = NULL;
    float *e = vector(1, lv);
    if (p->nmech) { ts = alloc_m(p); tp = alloc_m(p); }
    readmod(r, pp, uu, ts, tp, e);
    for (int j = 1; j <= p->ny; j++)
        for (int i = 1; i <= p->nx; i++)
            for (int k = 1; k <= p->nz; k++) {
                size_t o = ((size_t)(j - 1) * p->nx + (i - 1)) * p->nz + (k - 1);
                rho[o] = r[j][i][k]; pi[o] = pp[j][i][k]; u[o] = uu[j][i][k];
                if (p->nmech) { taus[o] = ts[j][i][k]; taup[o] = tp[j][i][k]; }
            }
    for (int l = 1; l <= p->nmech; l++) eta[l - 1] = e[l];
    for (int f = 0; f < 3; f++) {
        char name[128];
        snprintf(name, sizeof name, "%s.%s", base, ext[f]);
        unlink(name);
    }
    unlink(base);
    free_vector(FL, 1, lv); free_vector(e, 1, lv);
    free_f3tensor(r, 0, p->ny + 1, 0, p->nx + 1, 0, p->nz + 1);
    free_f3tensor(pp, 0, p->ny + 1, 0, p->nx + 1, 0, p->nz + 1);
    free_f3tensor(uu, 0, p->ny + 1, 0, p->nx + 1, 0, p->nz + 1);
    if (p->nmech) {
        free_f3tensor(ts, 0, p->ny + 1, 0, p->nx + 1, 0, p->nz + 1);
        free_f3tensor(tp, 0, p->ny + 1, 0, p->nx + 1, 0, p->nz + 1);
    }
    return 0;
}

int ifo_av_mat(const ifo_params *p, const float *rho, const float *pi, const float *u,
               const float *taus, const float *taup, float *avg9) {
    set_globals(p);
    refmodel m;
    model_setup(p, &m, rho, pi, u, taus, taup, NULL);
    size_t n = (size_t)p->nx * p->ny * p->nz;
    float ***a[9] = {m.uipjp, m.ujpkp, m.uipkp, m.rip, m.rjp, m.rkp, m.tausipjp, m.tausjpkp, m.tausipkp};
    for (int q = 0; q < 9; q++) {
        if (a[q]) g_out(p, a[q], avg9 + q * n);
        else memset(avg9 + q * n, 0, sizeof(float) * n);
    }
    model_free(p, &m);
    return 0;
}

/* ---- the propagation state (src/ifos3d.c:294-442) ---------------------------- */
typedef struct {
    float ***vx, ***vy, ***vz, ***sxy, ***syz;   /* from j=-2 */
    float ***sxx, ***syy, ***szz, ***sxz;         /* from j=-1 */
    float ***rxx, ***ryy, ***rzz, ***rxy, ***ryz, ***rxz;
    float ***psx[9];  /* psi_sxx_x, psi_sxy_x, psi_sxz_x, psi_sxy_y, psi_syy_y, psi_syz_y, psi_sxz_z, psi_syz_z, psi_szz_z */
    float ***pv[9];   /* psi_vxx, psi_vyx, psi_vzx, psi_vxy, psi_vyy, psi_vzy, psi_vxz, psi_vyz, psi_vzz */
    float ***absorb;
    int xb[2], yb[2], zb[2];
} refstate;

static void state_alloc(const ifo_params *p, refstate *s) {
    s->vx = alloc_w(p, -2); s->vy = alloc_w(p, -2); s->vz = alloc_w(p, -2);
    s->sxy = alloc_w(p, -2); s->syz = alloc_w(p, -2);
    s->sxz = alloc_w(p, -1); s->sxx = alloc_w(p, -1); s->syy = alloc_w(p, -1); s->szz = alloc_w(p, -1);
    s->rxx = s->ryy = s->rzz = s->rxy = s->ryz = s->rxz = NULL;
    if (p->nmech) {
        s->rxy = alloc_g(p); s->ryz = alloc_g(p); s->rxz = alloc_g(p);
        s->rxx = alloc_g(p); s->ryy = alloc_g(p); s->rzz = alloc_g(p);
    }
    int NYv = p->ny, NXv = p->nx, NZv = p->nz, fw2 = 2 * p->fw;
    /* x slabs [NY][2FW][NZ], y slabs [2FW][NX][NZ], z slabs [NY][NX][2FW] (src/ifos3d.c:421-440) */
    s->psx[0] = f3tensor(1, NYv, 1, fw2, 1, NZv); s->psx[1] = f3tensor(1, NYv, 1, fw2, 1, NZv);
    s->psx[2] = f3tensor(1, NYv, 1, fw2, 1, NZv);
    s->psx[3] = f3tensor(1, fw2, 1, NXv, 1, NZv); s->psx[4] = f3tensor(1, fw2, 1, NXv, 1, NZv);
    s->psx[5] = f3tensor(1, fw2, 1, NXv, 1, NZv);
    s->psx[6] = f3tensor(1, NYv, 1, NXv, 1, fw2); s->psx[7] = f3tensor(1, NYv, 1, NXv, 1, fw2);
    s->psx[8] = f3tensor(1, NYv, 1, NXv, 1, fw2);
    s->pv[0] = f3tensor(1, NYv, 1, fw2, 1, NZv); s->pv[1] = f3tensor(1, NYv, 1, fw2, 1, NZv);
    s->pv[2] = f3tensor(1, NYv, 1, fw2, 1, NZv);
    s->pv[3] = f3tensor(1, fw2, 1, NXv, 1, NZv); s->pv[4] = f3tensor(1, fw2, 1, NXv, 1, NZv);
    s->pv[5] = f3tensor(1, fw2, 1, NXv, 1, NZv);
    s->pv[6] = f3tensor(1, NYv, 1, NXv, 1, fw2); s->pv[7] = f3tensor(1, NYv, 1, NXv, 1, fw2);
    s->pv[8] = f3tensor(1, NYv, 1, NXv, 1, fw2);
    s->absorb = alloc_g(p);
    CPML_ini_elastic(s->xb, s->yb, s->zb);
}

static void state_free(const ifo_params *p, refstate *s) {
    free_w(p, s->vx, -2); free_w(p, s->vy, -2); free_w(p, s->vz, -2);
    free_w(p, s->sxy, -2); free_w(p, s->syz, -2);
    free_w(p, s->sxz, -1); free_w(p, s->sxx, -1); free_w(p, s->syy, -1); free_w(p, s->szz, -1);
    if (p->nmech) {
        free_g(p, s->rxy); free_g(p, s->ryz); free_g(p, s->rxz);
        free_g(p, s->rxx); free_g(p, s->ryy); free_g(p, s->rzz);
    }
    int fw2 = 2 * p->fw;
    for (int q = 0; q < 3; q++) {
        free_f3tensor(s->psx[q], 1, p->ny, 1, fw2, 1, p->nz);
        free_f3tensor(s->pv[q], 1, p->ny, 1, fw2, 1, p->nz);
        free_f3tensor(s->psx[q + 3], 1, fw2, 1, p->nx, 1, p->nz);
        free_f3tensor(s->pv[q + 3], 1, fw2, 1, p->nx, 1, p->nz);
        free_f3tensor(s->psx[q + 6], 1, p->ny, 1, p->nx, 1, fw2);
        free_f3tensor(s->pv[q + 6], 1, p->ny, 1, p->nx, 1, fw2);
    }
    free_g(p, s->absorb);
}

static void state_out(const ifo_params *p, refstate *s, float *state9) {
    if (!state9) return;
    size_t n = wsize(p);
    w_out(p, s->vx, -2, state9 + 0 * n); w_out(p, s->vy, -2, state9 + 1 * n); w_out(p, s->vz, -2, state9 + 2 * n);
    w_out(p, s->sxx, -1, state9 + 3 * n); w_out(p, s->syy, -1, state9 + 4 * n); w_out(p, s->szz, -1, state9 + 5 * n);
    w_out(p, s->sxy, -2, state9 + 6 * n); w_out(p, s->syz, -2, state9 + 7 * n); w_out(p, s->sxz, -1, state9 + 8 * n);
}

static void zero_state(refstate *s) {
    zero_wavefield(NX, NY, NZ, s->vx, s->vy, s->vz, s->sxx, s->syy, s->szz, s->sxy, s->syz, s->sxz,
                   s->rxx, s->ryy, s->rzz, s->rxy, s->ryz, s->rxz,
                   s->psx[0], s->psx[1], s->psx[2], s->psx[3], s->psx[4], s->psx[5], s->psx[6], s->psx[7], s->psx[8],
                   s->pv[0], s->pv[1], s->pv[2], s->pv[3], s->pv[4], s->pv[5], s->pv[6], s->pv[7], s->pv[8]);
}

/* One time step in the order of src/ifos3d.c:761-804 (forward) / 916-955 (adjoint). */
static void time_step(const ifo_params *p, refstate *s, refmodel *m, refcpml *c, int nt,
                      float **srcpos, float **sigx, float **sigy, float **sigz, int nsrc, int back,
                      float **psrc_signals, int npsrc,
                      float ****F[6], float *finv, int nf, int ntast,
                      int ntr, int **recpos, float **sx, float **sy, float **sz, float **sdum, int *lsamp, int *nlsamp,
                      float **sdiv, float **scurl, float **sp) {
    float **v = c->v;
    if (isnan(s->vy[NY / 2][NX / 2][NZ / 2])) err(" Simulation is unstable !");
    update_v(s->xb[0], s->xb[1], s->yb[0], s->yb[1], s->zb[0], s->zb[1], nt, s->vx, s->vy, s->vz,
             s->sxx, s->syy, s->szz, s->sxy, s->syz, s->sxz, m->rho, m->rjp, m->rkp, m->rip,
             srcpos, sigx, sigy, sigz, nsrc, s->absorb, back);
    update_v_CPML(s->xb[0], s->xb[1], s->yb[0], s->yb[1], s->zb[0], s->zb[1], nt, s->vx, s->vy, s->vz,
                  s->sxx, s->syy, s->szz, s->sxy, s->syz, s->sxz, m->rho, m->rjp, m->rkp, m->rip,
                  srcpos, sigx, sigy, sigz, nsrc, s->absorb, back,
                  v[0], v[2], v[3], v[4], v[6], v[7], v[8], v[10], v[11], v[12], v[14], v[15],
                  v[16], v[18], v[19], v[20], v[22], v[23],
                  s->psx[0], s->psx[1], s->psx[2], s->psx[3], s->psx[4], s->psx[5], s->psx[6], s->psx[7], s->psx[8]);
    if (p->nmech == 0) {
        update_s_elastic(s->xb[0], s->xb[1], s->yb[0], s->yb[1], s->zb[0], s->zb[1], s->vx, s->vy, s->vz,
                         s->sxx, s->syy, s->szz, s->sxy, s->syz, s->sxz, m->pi, m->u, m->uipjp, m->ujpkp, m->uipkp);
        update_s_CPML_elastic(s->xb[0], s->xb[1], s->yb[0], s->yb[1], s->zb[0], s->zb[1], s->vx, s->vy, s->vz,
                              s->sxx, s->syy, s->szz, s->sxy, s->syz, s->sxz, m->pi, m->u, m->uipjp, m->ujpkp, m->uipkp,
                              v[0], v[2], v[3], v[4], v[6], v[7], v[8], v[10], v[11], v[12], v[14], v[15],
                              v[16], v[18], v[19], v[20], v[22], v[23],
                              s->pv[0], s->pv[1], s->pv[2], s->pv[3], s->pv[4], s->pv[5], s->pv[6], s->pv[7], s->pv[8]);
    } else {
        update_s(s->xb[0], s->xb[1], s->yb[0], s->yb[1], s->zb[0], s->zb[1], s->vx, s->vy, s->vz,
                 s->sxx, s->syy, s->szz, s->sxy, s->syz, s->sxz, s->rxx, s->ryy, s->rzz, s->rxy, s->ryz, s->rxz,
                 m->pi, m->u, m->uipjp, m->ujpkp, m->uipkp, m->taus, m->tausipjp, m->tausjpkp, m->tausipkp, m->taup, m->eta);
        update_s_CPML(s->xb[0], s->xb[1], s->yb[0], s->yb[1], s->zb[0], s->zb[1], s->vx, s->vy, s->vz,
                      s->sxx, s->syy, s->szz, s->sxy, s->syz, s->sxz, s->rxx, s->ryy, s->rzz, s->rxy, s->ryz, s->rxz,
                      m->pi, m->u, m->uipjp, m->ujpkp, m->uipkp, m->taus, m->tausipjp, m->tausjpkp, m->tausipkp, m->taup, m->eta,
                      v[0], v[2], v[3], v[4], v[6], v[7], v[8], v[10], v[11], v[12], v[14], v[15],
                      v[16], v[18], v[19], v[20], v[22], v[23],
                      s->pv[0], s->pv[1], s->pv[2], s->pv[3], s->pv[4], s->pv[5], s->pv[6], s->pv[7], s->pv[8]);
    }
    if (!back) psource(nt, s->sxx, s->syy, s->szz, srcpos, psrc_signals, npsrc);
    if (nf > 0 && nt % ntast == 0)
        discfourier(1, NX, 1, NY, 1, NZ, nt, s->vx, s->vy, s->vz, F[0], F[1], F[2], F[3], F[4], F[5],
                    finv, nf, ntast, 0, back);
    if (FREE_SURF) {
        if (p->nmech == 0) surface_elastic(1, m->u, m->pi, s->sxx, s->syy, s->szz, s->sxy, s->syz, s->vx, s->vy, s->vz);
        else surface(1, m->u, m->pi, m->taus, m->taup, m->eta, s->sxx, s->syy, s->szz, s->sxy, s->syz,
                     s->rxx, s->ryy, s->rzz, s->vx, s->vy, s->vz);
    }
    if (ntr > 0 && nt == *lsamp) {
        seismo(*nlsamp, ntr, recpos, sx, sy, sz, sdiv ? sdiv : sdum, scurl ? scurl : sdum, sp ? sp : sdum, s->vx, s->vy,
               s->vz, s->sxx, s->syy, s->szz, m->pi, m->u);
        (*nlsamp)++;
        *lsamp += NDT;
    }
}

static int **recpos_matrix(int ntr, const int *recpos) {
    int **r = imatrix(1, 4, 1, ntr > 0 ? ntr : 1);
    for (int t = 1; t <= ntr; t++) {
        r[1][t] = recpos[(t - 1) * 3 + 0];
        r[2][t] = recpos[(t - 1) * 3 + 1];
        r[3][t] = recpos[(t - 1) * 3 + 2];
        r[4][t] = 0;
    }
    return r;
}

static void sections_out(int ntr, int ns, float **sx, float **sy, float **sz, float *dst) {
    for (int t = 1; t <= ntr; t++) {
        memcpy(dst + ((size_t)0 * ntr + t - 1) * ns, &sx[t][1], sizeof(float) * ns);
        memcpy(dst + ((size_t)1 * ntr + t - 1) * ns, &sy[t][1], sizeof(float) * ns);
        memcpy(dst + ((size_t)2 * ntr + t - 1) * ns, &sz[t][1], sizeof(float) * ns);
    }
}

static void dft_out(const ifo_params *p, float ****F[6], int nf, float *dst) {
    size_t n = wsize(p);
    for (int c = 0; c < 6; c++)
        for (int l = 1; l <= nf; l++)
            memcpy(dst + ((size_t)c * nf + (l - 1)) * n, &F[c][l][-2][-1][-1], sizeof(float) * n);
}

static int check_params(const ifo_params *p) {
    if (p->nmech > 1) return 2; /* the reference is limited to one mechanism (src/read_par_json.c:269-283) */
    if (p->nx < 2 * p->fw + 1 || p->ny < 2 * p->fw + 1 || p->nz < 2 * p->fw + 1) return 1;
    return 0;
}

static int forward_impl(const ifo_params *p, const float *rho, const float *pi, const float *u,
                        const float *taus, const float *taup, const float *eta, const float *cpml,
                        int nsrc, const float *srcpos, const float *signals,
                        int ntr, const int *recpos, int nf, const float *finv, int ntast,
                        float *sections, float *dft, float *state9, int seismo, float *pdc);

int ifo_forward(const ifo_params *p, const float *rho, const float *pi, const float *u,
                const float *taus, const float *taup, const float *eta, const float *cpml,
                int nsrc, const float *srcpos, const float *signals,
                int ntr, const int *recpos, int nf, const float *finv, int ntast,
                float *sections, float *dft, float *state9) {
    return forward_impl(p, rho, pi, u, taus, taup, eta, cpml, nsrc, srcpos, signals, ntr, recpos, nf, finv, ntast,
                        sections, dft, state9, 1, NULL);
}

/* The forward with SEISMO = seismo (1-4): sections [3][ntr][ns] vx, vy, vz (zero
 * unless SEISMO is 1 or 4, as seismo() leaves them) and pdc [3][ntr][ns] p, div,
 * curl (reference build only). */
int ifo_forward_seismo(const ifo_params *p, const float *rho, const float *pi, const float *u,
                       const float *taus, const float *taup, const float *eta, const float *cpml,
                       int nsrc, const float *srcpos, const float *signals, int ntr, const int *recpos,
                       int seismo, float *sections, float *pdc) {
    return forward_impl(p, rho, pi, u, taus, taup, eta, cpml, nsrc, srcpos, signals, ntr, recpos, 0, NULL, 1,
                        sections, NULL, NULL, seismo, pdc);
}

static int forward_impl(const ifo_params *p, const float *rho, const float *pi, const float *u,
                        const float *taus, const float *taup, const float *eta, const float *cpml,
                        int nsrc, const float *srcpos, const float *signals,
                        int ntr, const int *recpos, int nf, const float *finv, int ntast,
                        float *sections, float *dft, float *state9, int seismo, float *pdc) {
    int rc = check_params(p);
    if (rc) return rc;
    set_globals(p);
    SEISMO = seismo;
    int ns = ifo_nsamples(p);
    refmodel m; model_setup(p, &m, rho, pi, u, taus, taup, eta);
    refcpml c; cpml_alloc(p, &c); cpml_load(p, &c, cpml);
    refstate s; state_alloc(p, &s);
    float **sp = srcpos_matrix(nsrc, srcpos);
    float **sig = fmatrix(1, nsrc > 0 ? nsrc : 1, 1, p->nt);
    for (int l = 1; l <= nsrc; l++) memcpy(&sig[l][1], signals + (size_t)(l - 1) * p->nt, sizeof(float) * p->nt);
    int **rp = recpos_matrix(ntr, recpos);
    int ntr1 = ntr > 0 ? ntr : 1, ns1 = ns > 0 ? ns : 1;
    float **sx = fmatrix(1, ntr1, 1, ns1), **sy = fmatrix(1, ntr1, 1, ns1), **sz = fmatrix(1, ntr1, 1, ns1);
    float **sdum = fmatrix(1, ntr1, 1, ns1);
    float ****F[6] = {NULL, NULL, NULL, NULL, NULL, NULL};
    float *fv = NULL;
    if (nf > 0) {
        for (int q = 0; q < 6; q++) F[q] = alloc_f(p, nf);
        fv = vector(0, nf - 1);
        for (int l = 0; l < nf; l++) fv[l] = finv[l];
    }
    zero_state(&s);
    int lsamp = NDTSHIFT + 1, nlsamp = 1;
    float **xd = fmatrix(1, ntr1, 1, ns1), **xc = fmatrix(1, ntr1, 1, ns1), **xp = fmatrix(1, ntr1, 1, ns1);
    for (int nt = 1; nt <= NT; nt++)
        time_step(p, &s, &m, &c, nt, sp, sig, sig, sig, nsrc, 0, sig, nsrc, F, fv, nf, ntast,
                  ntr, rp, sx, sy, sz, sdum, &lsamp, &nlsamp, xd, xc, xp);
    SEISMO = 1;
    if (sections && ntr > 0) sections_out(ntr, ns, sx, sy, sz, sections);
    if (pdc && ntr > 0) sections_out(ntr, ns, xp, xd, xc, pdc);
    free_matrix(xd, 1, ntr1, 1, ns1); free_matrix(xc, 1, ntr1, 1, ns1); free_matrix(xp, 1, ntr1, 1, ns1);
    if (dft && nf > 0) dft_out(p, F, nf, dft);
    state_out(p, &s, state9);
    if (nf > 0) {
        for (int q = 0; q < 6; q++) free_f(p, F[q], nf);
        free_vector(fv, 0, nf - 1);
    }
    free_matrix(sx, 1, ntr1, 1, ns1); free_matrix(sy, 1, ntr1, 1, ns1); free_matrix(sz, 1, ntr1, 1, ns1);
    free_matrix(sdum, 1, ntr1, 1, ns1);
    free_imatrix(rp, 1, 4, 1, ntr1);
    free_matrix(sig, 1, nsrc > 0 ? nsrc : 1, 1, p->nt);
    free_matrix(sp, 1, 7, 1, nsrc > 0 ? nsrc : 1);
    state_free(p, &s); cpml_free(p, &c); model_free(p, &m);
    return 0;
}

int ifo_residual(const ifo_params *p, int ntr, const float *obs, const float *syn, float *diff, float *l2) {
    set_globals(p);
    int ns = ifo_nsamples(p);
    float **d = fmatrix(1, ntr, 1, ns), **df = fmatrix(1, ntr, 1, ns), **sy = fmatrix(1, ntr, 1, ns),
          **sd = fmatrix(1, ntr, 1, ns);
    float L2 = *l2, L2f = 0.0f;
    for (int c = 0; c < 3; c++) {
        for (int t = 1; t <= ntr; t++) {
            memcpy(&d[t][1], obs + ((size_t)c * ntr + t - 1) * ns, sizeof(float) * ns);
            memcpy(&sy[t][1], syn + ((size_t)c * ntr + t - 1) * ns, sizeof(float) * ns);
        }
        residual(d, df, sy, sd, ntr, ns, &L2, &L2f);
        for (int t = 1; t <= ntr; t++) memcpy(diff + ((size_t)c * ntr + t - 1) * ns, &sd[t][1], sizeof(float) * ns);
    }
    *l2 = L2;
    free_matrix(d, 1, ntr, 1, ns); free_matrix(df, 1, ntr, 1, ns);
    free_matrix(sy, 1, ntr, 1, ns); free_matrix(sd, 1, ntr, 1, ns);
    return 0;
}

int ifo_adjoint(const ifo_params *p, const float *rho, const float *pi, const float *u,
                const float *taus, const float *taup, const float *eta, const float *cpml,
                int ntr, const int *recpos, const float *diff,
                int nf, const float *finv, int ntast, float *dft_back, float *state9) {
    int rc = check_params(p);
    if (rc) return rc;
    if (p->ndt != 1 || p->ndtshift != 0) return 3; /* the injection indexes the residual by step (update_v_ssg.c:518) */
    set_globals(p);
    int ns = ifo_nsamples(p);
    refmodel m; model_setup(p, &m, rho, pi, u, taus, taup, eta);
    refcpml c; cpml_alloc(p, &c); cpml_load(p, &c, cpml);
    refstate s; state_alloc(p, &s);
    int ntr1 = ntr > 0 ? ntr : 1;
    float **back = fmatrix(1, 7, 1, ntr1);
    for (int t = 1; t <= ntr; t++) {
        back[1][t] = (float)recpos[(t - 1) * 3 + 0];
        back[2][t] = (float)recpos[(t - 1) * 3 + 1];
        back[3][t] = (float)recpos[(t - 1) * 3 + 2];
    }
    float **dx = fmatrix(1, ntr1, 1, p->nt), **dy = fmatrix(1, ntr1, 1, p->nt), **dz = fmatrix(1, ntr1, 1, p->nt);
    for (int t = 1; t <= ntr; t++) {
        memcpy(&dx[t][1], diff + ((size_t)0 * ntr + t - 1) * ns, sizeof(float) * ns);
        memcpy(&dy[t][1], diff + ((size_t)1 * ntr + t - 1) * ns, sizeof(float) * ns);
        memcpy(&dz[t][1], diff + ((size_t)2 * ntr + t - 1) * ns, sizeof(float) * ns);
    }
    int **rp = recpos_matrix(ntr, recpos);
    float **sx = fmatrix(1, ntr1, 1, ns), **sy = fmatrix(1, ntr1, 1, ns), **sz = fmatrix(1, ntr1, 1, ns);
    float **sdum = fmatrix(1, ntr1, 1, ns);
    float ****F[6] = {NULL, NULL, NULL, NULL, NULL, NULL};
    float *fv = NULL;
    if (nf > 0) {
        for (int q = 0; q < 6; q++) F[q] = alloc_f(p, nf);
        fv = vector(0, nf - 1);
        for (int l = 0; l < nf; l++) fv[l] = finv[l];
    }
    zero_state(&s);
    int lsamp = NDTSHIFT + 1, nlsamp = 1;
    for (int nt = 1; nt <= NT; nt++)
        time_step(p, &s, &m, &c, nt, back, dx, dy, dz, ntr, 1, NULL, 0, F, fv, nf, ntast,
                  ntr, rp, sx, sy, sz, sdum, &lsamp, &nlsamp, NULL, NULL, NULL);
    if (dft_back && nf > 0) dft_out(p, F, nf, dft_back);
    state_out(p, &s, state9);
    if (nf > 0) {
        for (int q = 0; q < 6; q++) free_f(p, F[q], nf);
        free_vector(fv, 0, nf - 1);
    }
    free_matrix(sx, 1, ntr1, 1, ns); free_matrix(sy, 1, ntr1, 1, ns); free_matrix(sz, 1, ntr1, 1, ns);
    free_matrix(sdum, 1, ntr1, 1, ns);
    free_imatrix(rp, 1, 4, 1, ntr1);
    free_matrix(dx, 1, ntr1, 1, p->nt); free_matrix(dy, 1, ntr1, 1, p->nt); free_matrix(dz, 1, ntr1, 1, p->nt);
    free_matrix(back, 1, 7, 1, ntr1);
    state_free(p, &s); cpml_free(p, &c); model_free(p, &m);
    return 0;
}

int ifo_gradient(const ifo_params *p, const float *rho, const float *pi, const float *u,
                 int nf, const float *finv, const float *dft_fwd, const float *dft_back, float *grad) {
    ifo_params q = *p;
    q.nmech = 0; /* gradient_F reads rho, pi, u only */
    p = &q;
    set_globals(p);
    refmodel m; model_setup(p, &m, rho, pi, u, NULL, NULL, NULL);
    size_t n = wsize(p);
    float ****F[6], ****B[6];
    for (int q = 0; q < 6; q++) {
        F[q] = alloc_f(p, nf); B[q] = alloc_f(p, nf);
        for (int l = 1; l <= nf; l++) {
            memcpy(&F[q][l][-2][-1][-1], dft_fwd + ((size_t)q * nf + l - 1) * n, sizeof(float) * n);
            memcpy(&B[q][l][-2][-1][-1], dft_back + ((size_t)q * nf + l - 1) * n, sizeof(float) * n);
        }
    }
    float *fv = vector(0, nf - 1);
    for (int l = 0; l < nf; l++) fv[l] = finv[l];
    size_t g = (size_t)p->nx * p->ny * p->nz;
    float ***g1 = alloc_g(p), ***g2 = alloc_g(p), ***g3 = alloc_g(p);
    g_in(p, g1, grad); g_in(p, g2, grad + g); g_in(p, g3, grad + 2 * g);
    gradient_F(NX, NY, NZ, F[0], F[1], F[2], F[3], F[4], F[5], B[0], B[1], B[2], B[3], B[4], B[5],
               g1, g2, g3, NT, m.rho, m.pi, m.u, fv, nf, 1);
    g_out(p, g1, grad); g_out(p, g2, grad + g); g_out(p, g3, grad + 2 * g);
    free_g(p, g1); free_g(p, g2); free_g(p, g3);
    free_vector(fv, 0, nf - 1);
    for (int q = 0; q < 6; q++) { free_f(p, F[q], nf); free_f(p, B[q], nf); }
    model_free(p, &m);
    return 0;
}

/* hess_F (src/hess_F.c) for one shot: forward DFT [6][nf][W] against ngreen
 * receivers' DFT fields [ngreen][6][nf][W], added to hess [3][ny][nx][nz].
 * Receiver n (1-based) sits at the reference's backward index n*nf + l. */
int ifo_hessian(const ifo_params *p, const float *rho, const float *pi, const float *u, int nf, const float *finv,
                const float *dft_fwd, int ngreen, const float *dft_green, float *hess) {
    ifo_params q = *p;
    q.nmech = 0;
    p = &q;
    set_globals(p);
    refmodel m; model_setup(p, &m, rho, pi, u, NULL, NULL, NULL);
    size_t n = wsize(p);
    const int nb = nf * (ngreen + 1);
    float ****F[6], ****B[6];
    for (int c = 0; c < 6; c++) {
        F[c] = alloc_f(p, nf); B[c] = alloc_f(p, nb);
        for (int l = 1; l <= nf; l++)
            memcpy(&F[c][l][-2][-1][-1], dft_fwd + ((size_t)c * nf + l - 1) * n, sizeof(float) * n);
        for (int r = 1; r <= ngreen; r++)
            for (int l = 1; l <= nf; l++)
                memcpy(&B[c][r * nf + l][-2][-1][-1], dft_green + (((size_t)(r - 1) * 6 + c) * nf + l - 1) * n,
                       sizeof(float) * n);
    }
    float *fv = vector(0, nf - 1);
    for (int l = 0; l < nf; l++) fv[l] = finv[l];
    size_t g = (size_t)p->nx * p->ny * p->nz;
    float ***h1 = alloc_g(p), ***h2 = alloc_g(p), ***h3 = alloc_g(p);
    g_in(p, h1, hess); g_in(p, h2, hess + g); g_in(p, h3, hess + 2 * g);
    hess_F(NX, NY, NZ, F[0], F[1], F[2], F[3], F[4], F[5], B[0], B[1], B[2], B[3], B[4], B[5],
           h1, h2, h3, NT, m.rho, m.pi, m.u, fv, nf, ngreen);
    g_out(p, h1, hess); g_out(p, h2, hess + g); g_out(p, h3, hess + 2 * g);
    free_g(p, h1); free_g(p, h2); free_g(p, h3);
    free_vector(fv, 0, nf - 1);
    for (int c = 0; c < 6; c++) { free_f(p, F[c], nf); free_f(p, B[c], nb); }
    model_free(p, &m);
    return 0;
}
