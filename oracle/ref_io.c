/*
 * Reference IO harness — TEST INFRASTRUCTURE ONLY (the CPU oracle).
 *
 * Drives the UNMODIFIED reference writers and readers, compiled from the
 * reference's src/ by oracle/Makefile with the one-rank MPI stub: outseis
 * (src/outseis.c), saveseis (src/saveseis.c), outmod + mergemod (src/outmod.c,
 * src/mergemod.c), outgrad (src/outgrad.c), readseis (src/readseis.c) and
 * readseis_split (src/readseis_split.c). Arrays are flat: sections [ntr][ns],
 * receiver positions [ntr][3] (grid indices), models [ny+2][nx+2][nz+2] ghosted,
 * gradients [3][ny][nx][nz].
 */
#include "fd.h"

#include <stdio.h>
#include <string.h>

extern FILE *FP, *FI;
extern int NX, NY, NZ, MYID, NDT, LITTLEBIG, SEISMO, SEIS_FORMAT, RUN_MULTIPLE_SHOTS, NPROC, METHOD;
extern int NPROCX, NPROCY, NPROCZ, IDX, IDY, IDZ, POS[4], VERBOSE;
extern float DX, DY, DZ, TIME, DT, REFREC[4];
extern char SEIS_FILE[STRING_SIZE], SEIS_OBS_FILE[STRING_SIZE], MOD_OUT_FILE[STRING_SIZE];

static void quiet(void) {
    static FILE *null = NULL;
    if (!null) null = fopen("/dev/null", "w");
    FP = FI = null;
    MYID = 0;
    NPROC = NPROCX = NPROCY = NPROCZ = 1;
    POS[1] = POS[2] = POS[3] = 0;
    VERBOSE = 0;
}

/* recpos [1..3][1..ntr] from rec [ntr][3]; recpos_loc[4][t] = trace_no[t-1]
 * (the global trace number), recpos_loc[1..3] the same positions. */
static void rec_mats(int ntr, const int *rec, const int *trace_no, int ***R, int ***RL) {
    const int n = ntr > 0 ? ntr : 1;
    int ntot = 0;
    for (int t = 0; t < ntr; ++t) ntot = trace_no[t] > ntot ? trace_no[t] : ntot;
    if (ntot < 1) ntot = 1;
    *R = imatrix(1, 3, 1, ntot);
    *RL = imatrix(1, 4, 1, n);
    for (int t = 1; t <= ntr; ++t) {
        for (int c = 1; c <= 3; ++c) {
            (*R)[c][trace_no[t - 1]] = rec[3 * (t - 1) + c - 1];
            (*RL)[c][t] = rec[3 * (t - 1) + c - 1];
        }
        (*RL)[4][t] = trace_no[t - 1];
    }
}

static float **sec_mat(int ntr, int ns, const float *sec) {
    float **S = fmatrix(1, ntr > 0 ? ntr : 1, 1, ns);
    for (int t = 1; t <= ntr; ++t) memcpy(&S[t][1], sec + (size_t)(t - 1) * ns, sizeof(float) * ns);
    return S;
}

static void set_common(float dx, float dy, float dz, int ndt, float dt, int littlebig) {
    DX = dx; DY = dy; DZ = dz; NDT = ndt; DT = dt; LITTLEBIG = littlebig;
    TIME = dt * 1000.0f;
    REFREC[1] = REFREC[2] = REFREC[3] = 0.0f;
}

int ifo_ref_outseis(const char *path, int comp, const float *sec, int ntr, int ns, const int *rec,
                    const int *trace_no, const float *src, float dx, float dy, float dz, int ndt, float dt, int fmt,
                    int littlebig) {
    quiet();
    set_common(dx, dy, dz, ndt, dt, littlebig);
    int **R, **RL;
    rec_mats(ntr, rec, trace_no, &R, &RL);
    float **S = sec_mat(ntr, ns, sec);
    float **P = fmatrix(1, 3, 1, 1);
    for (int c = 1; c <= 3; ++c) P[c][1] = src[c - 1];
    outseis(FP, fopen(path, "w"), comp, S, R, RL, ntr, P, 1, ns, fmt);
    free_matrix(P, 1, 3, 1, 1);
    free_matrix(S, 1, ntr > 0 ? ntr : 1, 1, ns);
    return 0;
}

/* saveseis with SEISMO = 1 on one rank: writes the rank file and the merged file
 * of vx, vy, vz (and removes the rank files when iteration > 0, METHOD and !obs).
 * secs: [3][ntr][ns]; srcpos: [nshot][3] metres. */
int ifo_ref_saveseis(const char *seis_file, const char *obs_file, const float *secs, int ntr, int ns, const int *rec,
                     const int *trace_no, const float *srcpos, int nshot, int ishot, int obs, int iteration, int fmt,
                     int multiple, int method, float dx, float dy, float dz, int ndt, float dt) {
    quiet();
    set_common(dx, dy, dz, ndt, dt, 0);
    snprintf(SEIS_FILE, STRING_SIZE, "%s", seis_file);
    snprintf(SEIS_OBS_FILE, STRING_SIZE, "%s", obs_file);
    SEISMO = 1;
    SEIS_FORMAT = fmt;
    RUN_MULTIPLE_SHOTS = multiple;
    METHOD = method;
    int **R, **RL;
    rec_mats(ntr, rec, trace_no, &R, &RL);
    const size_t n = (size_t)ntr * ns;
    float **S[3];
    for (int c = 0; c < 3; ++c) S[c] = sec_mat(ntr, ns, secs + c * n);
    float **P = fmatrix(1, 7, 1, nshot);
    for (int l = 1; l <= nshot; ++l) {
        for (int c = 1; c <= 3; ++c) P[c][l] = srcpos[3 * (l - 1) + c - 1];
        for (int c = 4; c <= 7; ++c) P[c][l] = 0.0f;
    }
    saveseis(FP, S[0], S[1], S[2], NULL, NULL, NULL, R, RL, ntr, P, ishot, ns, obs, iteration);
    free_matrix(P, 1, 7, 1, nshot);
    for (int c = 0; c < 3; ++c) free_matrix(S[c], 1, ntr > 0 ? ntr : 1, 1, ns);
    return 0;
}

int ifo_ref_readseis(const char *obs_file, int ishot, float *sec, int ntr, int ns, int comp, int multiple) {
    quiet();
    snprintf(SEIS_OBS_FILE, STRING_SIZE, "%s", obs_file);
    RUN_MULTIPLE_SHOTS = multiple;
    float **S = fmatrix(1, ntr > 0 ? ntr : 1, 1, ns);
    readseis(ishot, S, NULL, ntr, ns, comp);
    for (int t = 1; t <= ntr; ++t) memcpy(sec + (size_t)(t - 1) * ns, &S[t][1], sizeof(float) * ns);
    free_matrix(S, 1, ntr > 0 ? ntr : 1, 1, ns);
    return 0;
}

int ifo_ref_readseis_split(const char *obs_file, int ishot, float *sec, int ntr, const int *keep, int ns, int comp) {
    quiet();
    snprintf(SEIS_OBS_FILE, STRING_SIZE, "%s", obs_file);
    float **S = fmatrix(1, ntr > 0 ? ntr : 1, 1, ns);
    int *rn = ivector(1, ntr > 0 ? ntr : 1);
    for (int t = 1; t <= ntr; ++t) rn[t] = keep[t - 1];
    readseis_split(ishot, S, ntr, rn, ns, comp);
    int k = 0;
    for (int t = 1; t <= ntr; ++t)
        if (keep[t - 1] == 1) { ++k; memcpy(sec + (size_t)(k - 1) * ns, &S[k][1], sizeof(float) * ns); }
    free_ivector(rn, 1, ntr > 0 ? ntr : 1);
    free_matrix(S, 1, ntr > 0 ? ntr : 1, 1, ns);
    return k;
}

static float ***ghosted(int nx, int ny, int nz, const float *src) {
    float ***t = f3tensor(0, ny + 1, 0, nx + 1, 0, nz + 1);
    memcpy(&t[0][0][0], src, sizeof(float) * (size_t)(nx + 2) * (ny + 2) * (nz + 2));
    return t;
}

int ifo_ref_outmod(const char *base, int iteration, int nx, int ny, int nz, const float *rho, const float *pi,
                   const float *u, int idx, int idy, int idz) {
    quiet();
    NX = nx; NY = ny; NZ = nz; IDX = idx; IDY = idy; IDZ = idz;
    snprintf(MOD_OUT_FILE, STRING_SIZE, "%s", base);
    float ***R = ghosted(nx, ny, nz, rho), ***P = ghosted(nx, ny, nz, pi), ***U = ghosted(nx, ny, nz, u);
    outmod(nx, ny, nz, R, P, U, iteration);
    free_f3tensor(R, 0, ny + 1, 0, nx + 1, 0, nz + 1);
    free_f3tensor(P, 0, ny + 1, 0, nx + 1, 0, nz + 1);
    free_f3tensor(U, 0, ny + 1, 0, nx + 1, 0, nz + 1);
    return 0;
}

int ifo_ref_outgrad(const char *base, float finv, int iteration, int nx, int ny, int nz, const float *grad, int idx,
                    int idy, int idz) {
    quiet();
    NX = nx; NY = ny; NZ = nz; IDX = idx; IDY = idy; IDZ = idz;
    const size_t n = (size_t)nx * ny * nz;
    float ***G[3];
    for (int c = 0; c < 3; ++c) {
        G[c] = f3tensor(1, ny, 1, nx, 1, nz);
        memcpy(&G[c][1][1][1], grad + c * n, sizeof(float) * n);
    }
    char b[STRING_SIZE];
    snprintf(b, STRING_SIZE, "%s", base);
    outgrad(nx, ny, nz, G[0], G[1], G[2], finv, iteration, b);
    for (int c = 0; c < 3; ++c) free_f3tensor(G[c], 1, ny, 1, nx, 1, nz);
    return 0;
}

/* filt_seis (src/filt_seis.c) on data [ntr][ns] in place: FILT's Butterworth
 * low-pass of order 4 through libcseife's seife_lpb. */
extern float DT;
int ifo_ref_filt_seis(float *data, int ntr, int ns, float finv, float dt) {
    quiet();
    DT = dt;
    float **S = sec_mat(ntr, ns, data);
    filt_seis(S, ntr, ns, finv);
    for (int t = 1; t <= ntr; ++t) memcpy(data + (size_t)(t - 1) * ns, &S[t][1], sizeof(float) * ns);
    free_matrix(S, 1, ntr > 0 ? ntr : 1, 1, ns);
    return 0;
}

/* readinv (src/readinv.c) for stage `groupnum`: finv[nfmax], *nf, it[2]. */
extern char INV_FILE[STRING_SIZE];
int ifo_ref_readinv(const char *path, int groupnum, float *finv, int *nf, int *it, int nfmax) {
    quiet();
    snprintf(INV_FILE, STRING_SIZE, "%s", path);
    int g = groupnum - 1;
    readinv(finv, nf, &g, it, nfmax);
    return g;
}

/* hess_apply (src/hess_apply.c) on grad, hess [3][ny][nx][nz] (grad in place). */
extern float WATER_HESS[3], VP0, VS0, RHO0;
extern int LBFGS, NXG, NYG, NZG, FW;
int ifo_ref_hess_apply(int nx, int ny, int nz, float *grad, const float *hess, const float *water, int lbfgs,
                       float vp0, float vs0, float rho0) {
    quiet();
    NX = NXG = nx; NY = NYG = ny; NZ = NZG = nz; FW = 1;
    for (int c = 0; c < 3; ++c) WATER_HESS[c] = water[c];
    LBFGS = lbfgs; VP0 = vp0; VS0 = vs0; RHO0 = rho0;
    const size_t n = (size_t)nx * ny * nz;
    float ***G[3], ***H[3];
    for (int c = 0; c < 3; ++c) {
        G[c] = f3tensor(1, ny, 1, nx, 1, nz); memcpy(&G[c][1][1][1], grad + c * n, sizeof(float) * n);
        H[c] = f3tensor(1, ny, 1, nx, 1, nz); memcpy(&H[c][1][1][1], hess + c * n, sizeof(float) * n);
    }
    hess_apply(1, nx, 1, ny, 1, nz, G[0], G[1], G[2], H[0], H[1], H[2], 0.0f, 1);
    for (int c = 0; c < 3; ++c) {
        memcpy(grad + c * n, &G[c][1][1][1], sizeof(float) * n);
        free_f3tensor(G[c], 1, ny, 1, nx, 1, nz);
        free_f3tensor(H[c], 1, ny, 1, nx, 1, nz);
    }
    return 0;
}

/* readhess (src/readhess.c) into hess [3][ny][nx][nz]. */
extern char HESS_FILE[STRING_SIZE];
int ifo_ref_readhess(const char *base, float finv, int iteration, int nx, int ny, int nz, float vp0, float vs0,
                     float rho0, float *hess) {
    quiet();
    NX = NXG = nx; NY = NYG = ny; NZ = NZG = nz;
    VP0 = vp0; VS0 = vs0; RHO0 = rho0;
    snprintf(HESS_FILE, STRING_SIZE, "%s", base);
    const size_t n = (size_t)nx * ny * nz;
    float ***H[3];
    for (int c = 0; c < 3; ++c) H[c] = f3tensor(1, ny, 1, nx, 1, nz);
    readhess(nx, ny, nz, H[0], H[1], H[2], finv, iteration);
    for (int c = 0; c < 3; ++c) {
        memcpy(hess + c * n, &H[c][1][1][1], sizeof(float) * n);
        free_f3tensor(H[c], 1, ny, 1, nx, 1, nz);
    }
    return 0;
}
