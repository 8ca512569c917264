/*
 * Reference optimiser harness — TEST INFRASTRUCTURE ONLY (the CPU oracle).
 *
 * Drives the UNMODIFIED reference functions conjugate (src/conjugategrad.c),
 * lbfgs (src/lbfgs.c), lbfgs_savegrad (src/lbfgs_save.c), steplength
 * (src/steplength.c) and modelupdate (src/modelupdate.c), compiled from the
 * reference's src/ by oracle/Makefile with the one-rank MPI stub, through flat
 * arrays: gradients [3][ny][nx][nz], CG priors [6][ny][nx][nz], L-BFGS
 * matrices [bfgsnum][numpar*n] (row w-1 = the reference's row w), models
 * ghosted [ny+2][nx+2][nz+2].
 */
#include "fd.h"

#include <stdio.h>
#include <string.h>

extern FILE *FP, *FI;
extern int NX, NY, NZ, MYID, LBFGS, NUMPAR, BFGSNUM;
extern float TESTSTEP, VP0, VS0, RHO0, WEIGHT[3];

static void quiet(void) {
    static FILE *null = NULL;
    if (!null) null = fopen("/dev/null", "w");
    FP = FI = null;
    MYID = 0;
}

static float ***g_alloc(int nx, int ny, int nz, const float *src) {
    float ***t = f3tensor(1, ny, 1, nx, 1, nz);
    if (src) memcpy(&t[1][1][1], src, sizeof(float) * (size_t)nx * ny * nz);
    return t;
}
static void g_free(int nx, int ny, int nz, float ***t, float *dst) {
    if (dst) memcpy(dst, &t[1][1][1], sizeof(float) * (size_t)nx * ny * nz);
    free_f3tensor(t, 1, ny, 1, nx, 1, nz);
}

int ifo_ref_conjugate(int nx, int ny, int nz, float *grad, float *prior, int cdf, float *beta) {
    quiet();
    NX = nx; NY = ny; NZ = nz;
    const size_t n = (size_t)nx * ny * nz;
    float ***g[3], ***p[6];
    for (int c = 0; c < 3; c++) g[c] = g_alloc(nx, ny, nz, grad + c * n);
    for (int c = 0; c < 6; c++) p[c] = g_alloc(nx, ny, nz, prior + c * n);
    conjugate(nx, ny, nz, g[0], g[1], g[2], p[0], p[1], p[2], p[3], p[4], p[5], beta, 0, cdf);
    for (int c = 0; c < 3; c++) g_free(nx, ny, nz, g[c], grad + c * n);
    for (int c = 0; c < 6; c++) g_free(nx, ny, nz, p[c], prior + c * n);
    return 0;
}

static float **m_alloc(int rows, int cols, const float *src) {
    float **m = fmatrix(1, rows, 1, cols);
    for (int r = 1; r <= rows; r++) memcpy(&m[r][1], src + (size_t)(r - 1) * cols, sizeof(float) * cols);
    return m;
}
static void m_free(int rows, int cols, float **m, float *dst) {
    for (int r = 1; r <= rows; r++) memcpy(dst + (size_t)(r - 1) * cols, &m[r][1], sizeof(float) * cols);
    free_matrix(m, 1, rows, 1, cols);
}

/* lbfgs (it_group >= 2) or lbfgs_savegrad (it_group == 1), as src/ifos3d.c:1007-1014. */
int ifo_ref_lbfgs(int nx, int ny, int nz, int numpar, int bfgsnum, float *grad, float *scale, float *mod,
                  float *bgrad, int it_group) {
    quiet();
    NX = nx; NY = ny; NZ = nz; NUMPAR = numpar; BFGSNUM = bfgsnum; LBFGS = 1;
    const size_t n = (size_t)nx * ny * nz;
    const int cols = numpar * (int)n;
    float ***g[3];
    for (int c = 0; c < 3; c++) g[c] = g_alloc(nx, ny, nz, grad + c * n);
    float **M = m_alloc(bfgsnum, cols, mod), **G = m_alloc(bfgsnum, cols, bgrad);
    float *S = vector(1, bfgsnum);
    memcpy(&S[1], scale, sizeof(float) * bfgsnum);
    if (it_group > 1) lbfgs(g[0], g[1], g[2], S, M, G, it_group);
    else lbfgs_savegrad(g[0], g[1], g[2], G);
    memcpy(scale, &S[1], sizeof(float) * bfgsnum);
    free_vector(S, 1, bfgsnum);
    m_free(bfgsnum, cols, M, mod);
    m_free(bfgsnum, cols, G, bgrad);
    for (int c = 0; c < 3; c++) g_free(nx, ny, nz, g[c], grad + c * n);
    return 0;
}

int ifo_ref_steplength(float *L2, float *step, int lbfgs_on, int it_group, float teststep) {
    quiet();
    LBFGS = lbfgs_on;
    TESTSTEP = teststep;
    steplength(L2, step, 0, it_group);
    return 0;
}

int ifo_ref_modelupdate(int nx, int ny, int nz, float *grad, float *rho, float *pi, float *u, float *mod,
                        int numpar, int bfgsnum, float step, const float *weight, float vp0, float vs0, float rho0,
                        int lbfgs_on, int it_group) {
    quiet();
    NX = nx; NY = ny; NZ = nz; NUMPAR = numpar; BFGSNUM = bfgsnum; LBFGS = lbfgs_on;
    VP0 = vp0; VS0 = vs0; RHO0 = rho0;
    WEIGHT[0] = weight[0]; WEIGHT[1] = weight[1]; WEIGHT[2] = weight[2];
    const size_t n = (size_t)nx * ny * nz, mg = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    float ***g[3];
    for (int c = 0; c < 3; c++) g[c] = g_alloc(nx, ny, nz, grad + c * n);
    float ***m[3];
    float *src[3] = {rho, pi, u};
    for (int c = 0; c < 3; c++) {
        m[c] = f3tensor(0, ny + 1, 0, nx + 1, 0, nz + 1);
        memcpy(&m[c][0][0][0], src[c], sizeof(float) * mg);
    }
    const int cols = numpar * (int)n;
    float **M = (lbfgs_on && bfgsnum > 0) ? m_alloc(bfgsnum, cols, mod) : NULL;
    float beta[3] = {0, 0, 0};
    modelupdate(nx, ny, nz, g[0], g[1], g[2], m[0], m[1], m[2], M, step, beta, it_group);
    if (M) m_free(bfgsnum, cols, M, mod);
    for (int c = 0; c < 3; c++) {
        memcpy(src[c], &m[c][0][0][0], sizeof(float) * mg);
        free_f3tensor(m[c], 0, ny + 1, 0, nx + 1, 0, nz + 1);
    }
    for (int c = 0; c < 3; c++) g_free(nx, ny, nz, g[c], grad + c * n);
    return 0;
}

extern int DAMPTYPE, FREE_SURF, FW, NXG, NYG, NZG, POS[4], NPROCX, NPROCY, NPROCZ;
extern float DX, DY, DZ;

/* precon_grad with DAMPTYPE, FREE_SURF, FW as given; srcpos [nsrc][3] metres,
 * recpos [ntr][3] grid indices (the reference's srcpos[1..3][l], recpos[1..3][n]). */
int ifo_ref_precon_grad(int nx, int ny, int nz, float *grad, int damptype, int free_surf, int fw, float dx, float dy,
                        float dz, int nsrc, const float *srcpos, int ntr, const int *recpos) {
    quiet();
    NX = NXG = nx; NY = NYG = ny; NZ = NZG = nz;
    DAMPTYPE = damptype; FREE_SURF = free_surf; FW = fw; DX = dx; DY = dy; DZ = dz;
    POS[1] = POS[2] = POS[3] = 0;
    const size_t n = (size_t)nx * ny * nz;
    float ***g[3];
    for (int c = 0; c < 3; c++) g[c] = g_alloc(nx, ny, nz, grad + c * n);
    float **S = fmatrix(1, 7, 1, nsrc > 0 ? nsrc : 1);
    for (int l = 1; l <= nsrc; l++)
        for (int c = 1; c <= 3; c++) S[c][l] = srcpos[3 * (l - 1) + c - 1];
    int **R = imatrix(1, 3, 1, ntr > 0 ? ntr : 1);
    for (int t = 1; t <= ntr; t++)
        for (int c = 1; c <= 3; c++) R[c][t] = recpos[3 * (t - 1) + c - 1];
    precon_grad(nx, ny, nz, g[0], g[1], g[2], nsrc, S, ntr, R, 0.0f, 1, 0);
    free_matrix(S, 1, 7, 1, nsrc > 0 ? nsrc : 1);
    free_imatrix(R, 1, 3, 1, ntr > 0 ? ntr : 1);
    for (int c = 0; c < 3; c++) g_free(nx, ny, nz, g[c], grad + c * n);
    return 0;
}

/* constant_boundary on ghosted models [ny+2][nx+2][nz+2] with the one-rank
 * interior bounds of CPML_ini_elastic (xb = FW+1..NX-FW, zb = FW+1..NZ-FW). */
int ifo_ref_constant_boundary(int nx, int ny, int nz, int fw, float *rho, float *pi, float *u) {
    quiet();
    NX = nx; NY = ny; NZ = nz; FW = fw;
    POS[1] = POS[2] = POS[3] = 0;
    NPROCX = NPROCY = NPROCZ = 1;
    const size_t mg = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    float *src[3] = {rho, pi, u};
    float ***m[3];
    for (int c = 0; c < 3; c++) {
        m[c] = f3tensor(0, ny + 1, 0, nx + 1, 0, nz + 1);
        memcpy(&m[c][0][0][0], src[c], sizeof(float) * mg);
    }
    constant_boundary(fw + 1, nx - fw, 1, ny, fw + 1, nz - fw, m[1], m[2], m[0]);
    for (int c = 0; c < 3; c++) {
        memcpy(src[c], &m[c][0][0][0], sizeof(float) * mg);
        free_f3tensor(m[c], 0, ny + 1, 0, nx + 1, 0, nz + 1);
    }
    return 0;
}
