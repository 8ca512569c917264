/*
 * b200_glue.c — the reference driver's time loops served by the B200 engine.
 *
 * The drop-in host is the reference's own program: src/ifos3d.c and its host
 * files, compiled unmodified except that b200_hooks.h renames, inside
 * ifos3d.c, the calls of the three time loops and of the functions that read
 * their results. This file implements those renamed calls on top of the C ABI
 * in include/ifos_b200.h:
 *
 *  - the per-step calls (update_v, update_v_CPML, update_s_elastic,
 *    update_s_CPML_elastic, psource, exchange_v/s, discfourier,
 *    surface_elastic, seismo; src/ifos3d.c:754-814, 909-960, 1070-1103) only
 *    record what the loop asks for — which sources or residuals are injected,
 *    whether the DFT runs, where the traces go;
 *  - the first call that needs the loop's results (saveseis, residual,
 *    exchange_Fv, gradient_F, or the next zero_wavefield) runs the whole loop
 *    on the GPU at once: ifosb_forward for a forward loop (traces copied into
 *    the driver's section arrays), ifosb_adjoint with the driver's residual
 *    arrays for a back-propagation;
 *  - av_mat uploads the driver's current (or test) model with ifosb_set_model;
 *    zero_grad zeroes the device gradient; gradient_F runs gradient_F on the
 *    device and copies the accumulated gradient into grad1..3, in the
 *    reference's shot order and arithmetic (the same bits);
 *  - the halo exchanges are no-ops: one rank holds the whole grid.
 *
 * The host's wavefield arrays (vx, sxx, ...) are allocated by the driver but
 * never filled: the wavefield lives on the device, and the driver's NaN probe
 * (src/ifos3d.c:761) is replaced by the engine's, which reports through the
 * reference's own err(). Not served: snapshots (SNAP) and the approximate
 * Hessian (HESS), which need host wavefields or per-receiver loops; a run that
 * asks for them stops with err(). Viscoelastic propagation follows the
 * reference driver, which calls the elastic updates (its update_s calls are
 * commented out); IFOSB_HOST_VISCO=1 runs the L-mechanism update instead.
 */
#include "b200_hooks.h"
#include "fd.h"
#undef av_mat
#undef saveseis
#undef residual

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/ifos_b200.h"

/* the reference functions the hooks still call */
void saveseis(FILE *fp, float **sectionvx, float **sectionvy, float **sectionvz, float **sectionp,
              float **sectioncurl, float **sectiondiv, int **recpos, int **recpos_loc, int ntr, float **srcpos,
              int nsrc, int ns, int obs, int iteration);
void residual(float **sectiondata, float **sectiondataf, float **section, float **sectiondiff, int ntr, int ns,
              float *L2, float *L2f);

extern int NX, NY, NZ, NT, FDORDER, FDCOEFF, FREE_SURF, ABS_TYPE, FW, L, NDT, NDTSHIFT, SEISMO, SNAP, HESS,
    METHOD, NFMAX, NP;
extern float DX, DY, DZ, DT, TIME, ALPHA, BETA, *FL;

enum { PASS_NONE = 0, PASS_FWD = 1, PASS_ADJ = 2 };

/* what the driver's current time loop asked for */
static struct {
    int kind;
    float **srcpos;  /* srcpos_loc[1..7][1..npt] (forward) or srcpos_loc_back (adjoint) */
    float **sigx, **sigy, **sigz;
    int npt;
    int dft, nf, ntast;
    const float *finv;
    float ***surf_u, ***surf_pi;
} P;

static ifosb_engine *E;
static int g_cpml_set, g_rec_ntr = -1, g_nf = -1, g_ntast = 0, g_surface_alt;
static float g_finv[64];
static float ***g_u, ***g_pi;    /* the model last uploaded */
static float **g_sec[6];         /* the driver's trace arrays: vx vy vz div curl p */
static int **g_recpos, g_ntr;
static int g_visco;

static void engine_fail(int rc, const char *what) {
    char msg[512];
    if (rc == IFOSB_EUNSTABLE) err(" Simulation is unstable !");
    snprintf(msg, sizeof msg, " B200 engine: %s failed (%d): %s", what, rc, E ? ifosb_last_error(E) : "");
    err(msg);
}

static void check(int rc, const char *what) {
    if (rc != IFOSB_OK) engine_fail(rc, what);
}

static void ensure_engine(void) {
    if (E) return;
    if (NP != 1) err(" B200 engine: the drop-in host runs on one rank (NPROCX = NPROCY = NPROCZ = 1)");
    if (SNAP) err(" B200 engine: snapshots (SNAP) need host wavefields and are not produced");
    if (HESS) err(" B200 engine: the approximate Hessian (HESS) is not served by the drop-in host");
    if (ABS_TYPE != 1) err(" B200 engine: only ABS_TYPE = 1 (CPML) is implemented");
    const char *v = getenv("IFOSB_HOST_VISCO");
    g_visco = v && v[0] == '1' && L > 0;
    ifosb_params p;
    memset(&p, 0, sizeof p);
    p.nx = NX; p.ny = NY; p.nz = NZ;
    p.dx = DX; p.dy = DY; p.dz = DZ;
    p.dt = DT; p.nt = NT; p.time = TIME;
    p.fdorder = FDORDER; p.fdcoeff = FDCOEFF;
    p.free_surf = FREE_SURF; p.abs_type = ABS_TYPE; p.fw = FW;
    p.nmech = g_visco ? L : 0;
    p.ndt = NDT; p.ndtshift = NDTSHIFT;
    p.alpha = ALPHA; p.beta = BETA;
    check(ifosb_create(&p, 1, METHOD ? NFMAX : 0, &E), "ifosb_create");
    if (SEISMO) check(ifosb_set_seismo(E, SEISMO), "ifosb_set_seismo");
}

/* receivers from the driver's recpos_loc[1..3][1..ntr] (seen by the seismo hook) */
static void ensure_receivers(void) {
    if (g_rec_ntr == g_ntr || !g_recpos) return;
    int *rec = malloc(sizeof(int) * 3 * (size_t)(g_ntr > 0 ? g_ntr : 1));
    for (int t = 0; t < g_ntr; ++t)
        for (int c = 0; c < 3; ++c) rec[3 * t + c] = g_recpos[c + 1][t + 1];
    check(ifosb_set_receivers(E, g_ntr, rec), "ifosb_set_receivers");
    free(rec);
    g_rec_ntr = g_ntr;
}

static void set_frequencies(int dft) {
    const int nf = dft ? P.nf : 0;
    int same = nf == g_nf && (!nf || P.ntast == g_ntast);
    for (int l = 0; same && l < nf; ++l) same = P.finv[l] == g_finv[l];
    if (same) return;
    if (nf > 64) err(" B200 engine: more than 64 frequencies per stage");
    check(ifosb_set_frequencies(E, nf, nf ? P.finv : NULL, nf ? P.ntast : 1), "ifosb_set_frequencies");
    for (int l = 0; l < nf; ++l) g_finv[l] = P.finv[l];
    g_nf = nf;
    g_ntast = P.ntast;
}

static void run_forward(void) {
    const int ns = ifosb_nsamples(&(ifosb_params){.nt = NT, .ndt = NDT, .ndtshift = NDTSHIFT});
    float *srcpos = malloc(sizeof(float) * 7 * (size_t)(P.npt > 0 ? P.npt : 1));
    for (int l = 0; l < P.npt; ++l)
        for (int q = 0; q < 7; ++q) srcpos[7 * l + q] = P.srcpos[q + 1][l + 1];
    ifosb_shot shot = {P.npt, srcpos, P.npt ? &P.sigx[1][1] : NULL};
    /* the step-length forwards give surface_elastic the current model's u and pi while
       they propagate in the test model (src/ifos3d.c:1087-1090) */
    if (FREE_SURF && !g_visco && P.surf_u && (P.surf_u != g_u || P.surf_pi != g_pi)) {
        check(ifosb_set_surface_moduli(E, &P.surf_pi[0][0][0], &P.surf_u[0][0][0]), "ifosb_set_surface_moduli");
        g_surface_alt = 1;
    } else if (g_surface_alt) {
        check(ifosb_set_surface_moduli(E, NULL, NULL), "ifosb_set_surface_moduli");
        g_surface_alt = 0;
    }
    static const int ncomp_of[5] = {0, 3, 1, 2, 6};
    /* ifosb_forward's components in saveseis order (vx vy vz p div curl) -> g_sec slots */
    static const int slot_of[5][6] = {{0}, {0, 1, 2}, {5}, {3, 4}, {0, 1, 2, 5, 3, 4}};
    const int ncomp = SEISMO ? ncomp_of[SEISMO] : 0;
    float *sec = NULL;
    if (ncomp && g_ntr > 0) sec = malloc(sizeof(float) * (size_t)ncomp * g_ntr * ns);
    check(ifosb_forward(E, 1, &shot, sec), "ifosb_forward");
    for (int c = 0; sec && c < ncomp; ++c) {
        float **dst = g_sec[slot_of[SEISMO][c]];
        if (dst) memcpy(&dst[1][1], sec + (size_t)c * g_ntr * ns, sizeof(float) * (size_t)g_ntr * ns);
    }
    free(sec);
    free(srcpos);
}

static void run_adjoint(void) {
    const int ns = ifosb_nsamples(&(ifosb_params){.nt = NT, .ndt = NDT, .ndtshift = NDTSHIFT});
    /* the injection points are the receivers (srcpos_loc_back = recpos_loc, src/ifos3d.c:708-710) */
    if (P.npt != g_ntr) err(" B200 engine: the back-propagation injects at other points than the receivers");
    for (int t = 0; t < P.npt; ++t)
        for (int c = 0; c < 3; ++c)
            if ((int)P.srcpos[c + 1][t + 1] != g_recpos[c + 1][t + 1])
                err(" B200 engine: the back-propagation injects at other points than the receivers");
    float *diff = malloc(sizeof(float) * 3 * (size_t)(g_ntr > 0 ? g_ntr : 1) * ns);
    float **comp[3] = {P.sigx, P.sigy, P.sigz};
    for (int c = 0; c < 3; ++c)
        if (g_ntr > 0) memcpy(diff + (size_t)c * g_ntr * ns, &comp[c][1][1], sizeof(float) * (size_t)g_ntr * ns);
    check(ifosb_adjoint(E, diff), "ifosb_adjoint");
    free(diff);
}

/* run the recorded time loop, if one is pending */
static void flush(void) {
    if (P.kind == PASS_NONE) return;
    ensure_engine();
    ensure_receivers();
    set_frequencies(P.dft);
    if (P.kind == PASS_FWD) run_forward();
    else run_adjoint();
    P.kind = PASS_NONE;
}

/* ---- model and resets -------------------------------------------------- */

void b200_av_mat(float ***rho, float ***pi, float ***u, float ***taus, float ***taup, float ***uipjp, float ***ujpkp,
                 float ***uipkp, float ***tausipjp, float ***tausjpkp, float ***tausipkp, float ***rjp, float ***rkp,
                 float ***rip) {
    (void)uipjp; (void)ujpkp; (void)uipkp; (void)tausipjp; (void)tausjpkp; (void)tausipkp;
    (void)rjp; (void)rkp; (void)rip;
    flush();
    ensure_engine();
    float eta[8] = {0};
    if (g_visco) {
        if (L > 8) err(" B200 engine: at most 8 relaxation mechanisms");
        /* readmod's eta[l] = DT / (1 / (2 pi FL[l])) (src/readmod.c:48-52) */
        for (int l = 1; l <= L; ++l) {
            const float pts = 1.0 / (2.0 * PI * FL[l]);
            eta[l - 1] = DT / pts;
        }
    }
    check(ifosb_set_model(E, &rho[0][0][0], &pi[0][0][0], &u[0][0][0], g_visco ? &taus[0][0][0] : NULL,
                          g_visco ? &taup[0][0][0] : NULL, g_visco ? eta : NULL),
          "ifosb_set_model");
    g_u = u;
    g_pi = pi;
}

void b200_zero_wavefield(int nx, int ny, int nz, float ***vx, float ***vy, float ***vz, float ***sxx, float ***syy,
                         float ***szz, float ***sxy, float ***syz, float ***sxz, float ***rxx, float ***ryy,
                         float ***rzz, float ***rxy, float ***ryz, float ***rxz, float ***psi_sxx_x,
                         float ***psi_sxy_x, float ***psi_sxz_x, float ***psi_sxy_y, float ***psi_syy_y,
                         float ***psi_syz_y, float ***psi_sxz_z, float ***psi_syz_z, float ***psi_szz_z,
                         float ***psi_vxx, float ***psi_vyx, float ***psi_vzx, float ***psi_vxy, float ***psi_vyy,
                         float ***psi_vzy, float ***psi_vxz, float ***psi_vyz, float ***psi_vzz) {
    (void)nx; (void)ny; (void)nz; (void)vx; (void)vy; (void)vz; (void)sxx; (void)syy; (void)szz; (void)sxy;
    (void)syz; (void)sxz; (void)rxx; (void)ryy; (void)rzz; (void)rxy; (void)ryz; (void)rxz; (void)psi_sxx_x;
    (void)psi_sxy_x; (void)psi_sxz_x; (void)psi_sxy_y; (void)psi_syy_y; (void)psi_syz_y; (void)psi_sxz_z;
    (void)psi_syz_z; (void)psi_szz_z; (void)psi_vxx; (void)psi_vyx; (void)psi_vzx; (void)psi_vxy; (void)psi_vyy;
    (void)psi_vzy; (void)psi_vxz; (void)psi_vyz; (void)psi_vzz;
    flush();  /* the device zeroes its own wavefield at the start of every loop */
}

void b200_zero_invers(int nx, int ny, int nz, float ****Ffvx, float ****Ffvy, float ****Ffvz, float ****Ffivx,
                      float ****Ffivy, float ****Ffivz, float ****Fbvx, float ****Fbvy, float ****Fbvz,
                      float ****Fbivx, float ****Fbivy, float ****Fbivz, int nfmax, int ntr_hess) {
    (void)nx; (void)ny; (void)nz; (void)Ffvx; (void)Ffvy; (void)Ffvz; (void)Ffivx; (void)Ffivy; (void)Ffivz;
    (void)Fbvx; (void)Fbvy; (void)Fbvz; (void)Fbivx; (void)Fbivy; (void)Fbivz; (void)nfmax; (void)ntr_hess;
    flush();  /* DFT accumulators live on the device, zeroed with each loop */
}

void b200_zero_grad(int nx, int ny, int nz, float ***grad1, float ***grad2, float ***grad3) {
    flush();
    ensure_engine();
    check(ifosb_zero_gradient(E), "ifosb_zero_gradient");
    const size_t n = (size_t)nx * ny * nz;
    memset(&grad1[1][1][1], 0, n * sizeof(float));
    memset(&grad2[1][1][1], 0, n * sizeof(float));
    memset(&grad3[1][1][1], 0, n * sizeof(float));
}

/* ---- one time step: record only ---------------------------------------- */

double b200_update_v(int nx1, int nx2, int ny1, int ny2, int nz1, int nz2, int nt, float ***vx, float ***vy,
                     float ***vz, float ***sxx, float ***syy, float ***szz, float ***sxy, float ***syz, float ***sxz,
                     float ***rho, float ***rjp, float ***rkp, float ***rip, float **srcpos_loc, float **signals,
                     float **signaly, float **signalz, int nsrc, float ***absorb_coeff, int back) {
    (void)nx1; (void)nx2; (void)ny1; (void)ny2; (void)nz1; (void)nz2; (void)vx; (void)vy; (void)vz; (void)sxx;
    (void)syy; (void)szz; (void)sxy; (void)syz; (void)sxz; (void)rho; (void)rjp; (void)rkp; (void)rip;
    (void)absorb_coeff;
    if (nt == 1) {
        flush();
        P.kind = back ? PASS_ADJ : PASS_FWD;
        P.dft = 0;
        P.surf_u = P.surf_pi = NULL;
    }
    P.srcpos = srcpos_loc;
    P.sigx = signals;
    P.sigy = signaly;
    P.sigz = signalz;
    P.npt = nsrc;
    return 0.0;
}

double b200_update_v_CPML(int nx1, int nx2, int ny1, int ny2, int nz1, int nz2, int nt, float ***vx, float ***vy,
                          float ***vz, float ***sxx, float ***syy, float ***szz, float ***sxy, float ***syz,
                          float ***sxz, float ***rho, float ***rjp, float ***rkp, float ***rip, float **srcpos_loc,
                          float **signals, float **signaly, float **signalz, int nsrc, float ***absorb_coeff,
                          int back, float *K_x, float *a_x, float *b_x, float *K_x_half, float *a_x_half,
                          float *b_x_half, float *K_y, float *a_y, float *b_y, float *K_y_half, float *a_y_half,
                          float *b_y_half, float *K_z, float *a_z, float *b_z, float *K_z_half, float *a_z_half,
                          float *b_z_half, float ***psi_sxx_x, float ***psi_sxy_x, float ***psi_sxz_x,
                          float ***psi_sxy_y, float ***psi_syy_y, float ***psi_syz_y, float ***psi_sxz_z,
                          float ***psi_syz_z, float ***psi_szz_z) {
    (void)nx1; (void)nx2; (void)ny1; (void)ny2; (void)nz1; (void)nz2; (void)nt; (void)vx; (void)vy; (void)vz;
    (void)sxx; (void)syy; (void)szz; (void)sxy; (void)syz; (void)sxz; (void)rho; (void)rjp; (void)rkp; (void)rip;
    (void)srcpos_loc; (void)signals; (void)signaly; (void)signalz; (void)nsrc; (void)absorb_coeff; (void)back;
    (void)psi_sxx_x; (void)psi_sxy_x; (void)psi_sxz_x; (void)psi_sxy_y; (void)psi_syy_y; (void)psi_syz_y;
    (void)psi_sxz_z; (void)psi_syz_z; (void)psi_szz_z;
    if (g_cpml_set) return 0.0;
    /* CPML_coeff's profiles (src/ifos3d.c:626), fixed for the run: rows K, a, b, K_half,
       a_half, b_half of x, y, z; element h is the reference's index h + 1 */
    ensure_engine();
    const float *rows[18] = {K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y,
                             K_y_half, a_y_half, b_y_half, K_z, a_z, b_z, K_z_half, a_z_half, b_z_half};
    const int n2 = 2 * FW;
    float *coeff = malloc(sizeof(float) * 18 * (size_t)n2);
    for (int r = 0; r < 18; ++r)
        for (int h = 0; h < n2; ++h) coeff[(size_t)r * n2 + h] = rows[r][h + 1];
    check(ifosb_set_cpml(E, coeff), "ifosb_set_cpml");
    free(coeff);
    g_cpml_set = 1;
    return 0.0;
}

double b200_update_s(int nx1, int nx2, int ny1, int ny2, int nz1, int nz2, float ***vx, float ***vy, float ***vz,
                     float ***sxx, float ***syy, float ***szz, float ***sxy, float ***syz, float ***sxz, float ***rxx,
                     float ***ryy, float ***rzz, float ***rxy, float ***ryz, float ***rxz, float ***pi, float ***u,
                     float ***uipjp, float ***ujpkp, float ***uipkp, float ***taus, float ***tausipjp,
                     float ***tausjpkp, float ***tausipkp, float ***taup, float *eta) {
    (void)nx1; (void)nx2; (void)ny1; (void)ny2; (void)nz1; (void)nz2; (void)vx; (void)vy; (void)vz; (void)sxx;
    (void)syy; (void)szz; (void)sxy; (void)syz; (void)sxz; (void)rxx; (void)ryy; (void)rzz; (void)rxy; (void)ryz;
    (void)rxz; (void)pi; (void)u; (void)uipjp; (void)ujpkp; (void)uipkp; (void)taus; (void)tausipjp;
    (void)tausjpkp; (void)tausipkp; (void)taup; (void)eta;
    return 0.0;
}

double b200_update_s_CPML(int nx1, int nx2, int ny1, int ny2, int nz1, int nz2, float ***vx, float ***vy,
                          float ***vz, float ***sxx, float ***syy, float ***szz, float ***sxy, float ***syz,
                          float ***sxz, float ***rxx, float ***ryy, float ***rzz, float ***rxy, float ***ryz,
                          float ***rxz, float ***pi, float ***u, float ***uipjp, float ***ujpkp, float ***uipkp,
                          float ***taus, float ***tausipjp, float ***tausjpkp, float ***tausipkp, float ***taup,
                          float *eta, float *K_x, float *a_x, float *b_x, float *K_x_half, float *a_x_half,
                          float *b_x_half, float *K_y, float *a_y, float *b_y, float *K_y_half, float *a_y_half,
                          float *b_y_half, float *K_z, float *a_z, float *b_z, float *K_z_half, float *a_z_half,
                          float *b_z_half, float ***psi_vxx, float ***psi_vyx, float ***psi_vzx, float ***psi_vxy,
                          float ***psi_vyy, float ***psi_vzy, float ***psi_vxz, float ***psi_vyz, float ***psi_vzz) {
    (void)nx1; (void)nx2; (void)ny1; (void)ny2; (void)nz1; (void)nz2; (void)vx; (void)vy; (void)vz; (void)sxx;
    (void)syy; (void)szz; (void)sxy; (void)syz; (void)sxz; (void)rxx; (void)ryy; (void)rzz; (void)rxy; (void)ryz;
    (void)rxz; (void)pi; (void)u; (void)uipjp; (void)ujpkp; (void)uipkp; (void)taus; (void)tausipjp;
    (void)tausjpkp; (void)tausipkp; (void)taup; (void)eta; (void)K_x; (void)a_x; (void)b_x; (void)K_x_half;
    (void)a_x_half; (void)b_x_half; (void)K_y; (void)a_y; (void)b_y; (void)K_y_half; (void)a_y_half;
    (void)b_y_half; (void)K_z; (void)a_z; (void)b_z; (void)K_z_half; (void)a_z_half; (void)b_z_half;
    (void)psi_vxx; (void)psi_vyx; (void)psi_vzx; (void)psi_vxy; (void)psi_vyy; (void)psi_vzy; (void)psi_vxz;
    (void)psi_vyz; (void)psi_vzz;
    return 0.0;
}

double b200_update_s_elastic(int nx1, int nx2, int ny1, int ny2, int nz1, int nz2, float ***vx, float ***vy,
                             float ***vz, float ***sxx, float ***syy, float ***szz, float ***sxy, float ***syz,
                             float ***sxz, float ***pi, float ***u, float ***uipjp, float ***ujpkp, float ***uipkp) {
    (void)nx1; (void)nx2; (void)ny1; (void)ny2; (void)nz1; (void)nz2; (void)vx; (void)vy; (void)vz; (void)sxx;
    (void)syy; (void)szz; (void)sxy; (void)syz; (void)sxz; (void)pi; (void)u; (void)uipjp; (void)ujpkp;
    (void)uipkp;
    return 0.0;
}

double b200_update_s_CPML_elastic(int nx1, int nx2, int ny1, int ny2, int nz1, int nz2, float ***vx, float ***vy,
                                  float ***vz, float ***sxx, float ***syy, float ***szz, float ***sxy, float ***syz,
                                  float ***sxz, float ***pi, float ***u, float ***uipjp, float ***ujpkp,
                                  float ***uipkp, float *K_x, float *a_x, float *b_x, float *K_x_half,
                                  float *a_x_half, float *b_x_half, float *K_y, float *a_y, float *b_y,
                                  float *K_y_half, float *a_y_half, float *b_y_half, float *K_z, float *a_z,
                                  float *b_z, float *K_z_half, float *a_z_half, float *b_z_half, float ***psi_vxx,
                                  float ***psi_vyx, float ***psi_vzx, float ***psi_vxy, float ***psi_vyy,
                                  float ***psi_vzy, float ***psi_vxz, float ***psi_vyz, float ***psi_vzz) {
    (void)nx1; (void)nx2; (void)ny1; (void)ny2; (void)nz1; (void)nz2; (void)vx; (void)vy; (void)vz; (void)sxx;
    (void)syy; (void)szz; (void)sxy; (void)syz; (void)sxz; (void)pi; (void)u; (void)uipjp; (void)ujpkp;
    (void)uipkp; (void)K_x; (void)a_x; (void)b_x; (void)K_x_half; (void)a_x_half; (void)b_x_half; (void)K_y;
    (void)a_y; (void)b_y; (void)K_y_half; (void)a_y_half; (void)b_y_half; (void)K_z; (void)a_z; (void)b_z;
    (void)K_z_half; (void)a_z_half; (void)b_z_half; (void)psi_vxx; (void)psi_vyx; (void)psi_vzx; (void)psi_vxy;
    (void)psi_vyy; (void)psi_vzy; (void)psi_vxz; (void)psi_vyz; (void)psi_vzz;
    return 0.0;
}

void b200_psource(int nt, float ***sxx, float ***syy, float ***szz, float **srcpos_loc, float **signals, int nsrc) {
    (void)nt; (void)sxx; (void)syy; (void)szz; (void)srcpos_loc; (void)signals; (void)nsrc;
}

void b200_surface(int ndepth, float ***u, float ***pi, float ***taus, float ***taup, float *eta, float ***sxx,
                  float ***syy, float ***szz, float ***sxy, float ***syz, float ***rxx, float ***ryy, float ***rzz,
                  float ***vx, float ***vy, float ***vz) {
    (void)ndepth; (void)taus; (void)taup; (void)eta; (void)sxx; (void)syy; (void)szz; (void)sxy; (void)syz;
    (void)rxx; (void)ryy; (void)rzz; (void)vx; (void)vy; (void)vz;
    P.surf_u = u;
    P.surf_pi = pi;
}

void b200_surface_elastic(int ndepth, float ***u, float ***pi, float ***sxx, float ***syy, float ***szz,
                          float ***sxy, float ***syz, float ***vx, float ***vy, float ***vz) {
    (void)ndepth; (void)sxx; (void)syy; (void)szz; (void)sxy; (void)syz; (void)vx; (void)vy; (void)vz;
    P.surf_u = u;
    P.surf_pi = pi;
}

void b200_discfourier(int nx1, int nx2, int ny1, int ny2, int nz1, int nz2, int nt, float ***vx, float ***vy,
                      float ***vz, float ****Fvx, float ****Fvy, float ****Fvz, float ****Fvxi, float ****Fvyi,
                      float ****Fvzi, float *finv, int nf, int ntast, int pshot, int back) {
    (void)nx1; (void)nx2; (void)ny1; (void)ny2; (void)nz1; (void)nz2; (void)nt; (void)vx; (void)vy; (void)vz;
    (void)Fvx; (void)Fvy; (void)Fvz; (void)Fvxi; (void)Fvyi; (void)Fvzi; (void)pshot; (void)back;
    P.dft = 1;
    P.finv = finv;
    P.nf = nf;
    P.ntast = ntast;
}

void b200_seismo(int lsamp, int ntr, int **recpos, float **sectionvx, float **sectionvy, float **sectionvz,
                 float **sectiondiv, float **sectioncurl, float **sectionp, float ***vx, float ***vy, float ***vz,
                 float ***sxx, float ***syy, float ***szz, float ***pi, float ***u) {
    (void)lsamp; (void)vx; (void)vy; (void)vz; (void)sxx; (void)syy; (void)szz; (void)pi; (void)u;
    /* only the forward loops' traces are read back (the driver discards the
       back-propagation's, src/ifos3d.c:963-964) */
    if (P.kind != PASS_FWD) return;
    g_recpos = recpos;
    g_ntr = ntr;
    g_sec[0] = sectionvx; g_sec[1] = sectionvy; g_sec[2] = sectionvz;
    g_sec[3] = sectiondiv; g_sec[4] = sectioncurl; g_sec[5] = sectionp;
}

void b200_snap(FILE *fp, int nt, int nsnap, int format, int type, float ***vx, float ***vy, float ***vz,
               float ***sxx, float ***syy, float ***szz, float ***u, float ***pi, int idx, int idy, int idz, int nx1,
               int ny1, int nz1, int nx2, int ny2, int nz2) {
    (void)fp; (void)nt; (void)nsnap; (void)format; (void)type; (void)vx; (void)vy; (void)vz; (void)sxx; (void)syy;
    (void)szz; (void)u; (void)pi; (void)idx; (void)idy; (void)idz; (void)nx1; (void)ny1; (void)nz1; (void)nx2;
    (void)ny2; (void)nz2;
    err(" B200 engine: snapshots (SNAP) need host wavefields and are not produced");
}

/* ---- halo exchanges: one rank, nothing to exchange ----------------------- */

double b200_exchange_v(float ***vx, float ***vy, float ***vz, float ***bufferlef_to_rig, float ***bufferrig_to_lef,
                       float ***buffertop_to_bot, float ***bufferbot_to_top, float ***bufferfro_to_bac,
                       float ***bufferbac_to_fro, MPI_Request *req_send, MPI_Request *req_rec) {
    (void)vx; (void)vy; (void)vz; (void)bufferlef_to_rig; (void)bufferrig_to_lef; (void)buffertop_to_bot;
    (void)bufferbot_to_top; (void)bufferfro_to_bac; (void)bufferbac_to_fro; (void)req_send; (void)req_rec;
    return 0.0;
}

double b200_exchange_s(float ***sxx, float ***syy, float ***szz, float ***sxy, float ***syz, float ***sxz,
                       float ***bufferlef_to_rig, float ***bufferrig_to_lef, float ***buffertop_to_bot,
                       float ***bufferbot_to_top, float ***bufferfro_to_bac, float ***bufferbac_to_fro,
                       MPI_Request *req_send, MPI_Request *req_rec) {
    (void)sxx; (void)syy; (void)szz; (void)sxy; (void)syz; (void)sxz; (void)bufferlef_to_rig;
    (void)bufferrig_to_lef; (void)buffertop_to_bot; (void)bufferbot_to_top; (void)bufferfro_to_bac;
    (void)bufferbac_to_fro; (void)req_send; (void)req_rec;
    return 0.0;
}

double b200_exchange_Fv(float ****vx, float ****vy, float ****vz, int nf, float ***bufferlef_to_rig,
                        float ***bufferrig_to_lef, float ***buffertop_to_bot, float ***bufferbot_to_top,
                        float ***bufferfro_to_bac, float ***bufferbac_to_fro, MPI_Request *req_send,
                        MPI_Request *req_rec, int ntr_hess) {
    (void)vx; (void)vy; (void)vz; (void)nf; (void)bufferlef_to_rig; (void)bufferrig_to_lef;
    (void)buffertop_to_bot; (void)bufferbot_to_top; (void)bufferfro_to_bac; (void)bufferbac_to_fro;
    (void)req_send; (void)req_rec; (void)ntr_hess;
    flush();
    return 0.0;
}

/* ---- consumers of a loop's results ----------------------------------------- */

void b200_saveseis(FILE *fp, float **sectionvx, float **sectionvy, float **sectionvz, float **sectionp,
                   float **sectioncurl, float **sectiondiv, int **recpos, int **recpos_loc, int ntr, float **srcpos,
                   int nsrc, int ns, int obs, int iteration) {
    flush();
    saveseis(fp, sectionvx, sectionvy, sectionvz, sectionp, sectioncurl, sectiondiv, recpos, recpos_loc, ntr, srcpos,
             nsrc, ns, obs, iteration);
}

void b200_residual(float **sectiondata, float **sectiondataf, float **section, float **sectiondiff, int ntr, int ns,
                   float *L2, float *L2f) {
    flush();
    residual(sectiondata, sectiondataf, section, sectiondiff, ntr, ns, L2, L2f);
}

void b200_gradient_F(int nx, int ny, int nz, float ****fvx, float ****fvy, float ****fvz, float ****fivx,
                     float ****fivy, float ****fivz, float ****bvx, float ****bvy, float ****bvz, float ****bivx,
                     float ****bivy, float ****bivz, float ***gradlam, float ***gradmu, float ***gradrho, int nt,
                     float ***rho, float ***pi, float ***u, float *finv, int nf, int iteration) {
    (void)fvx; (void)fvy; (void)fvz; (void)fivx; (void)fivy; (void)fivz; (void)bvx; (void)bvy; (void)bvz;
    (void)bivx; (void)bivy; (void)bivz; (void)nt; (void)rho; (void)pi; (void)u; (void)finv; (void)nf;
    (void)iteration;
    flush();
    check(ifosb_gradient(E), "ifosb_gradient");
    const size_t n = (size_t)nx * ny * nz;
    float *g = malloc(sizeof(float) * 3 * n);
    check(ifosb_get_gradient(E, g, NULL), "ifosb_get_gradient");
    memcpy(&gradlam[1][1][1], g, n * sizeof(float));
    memcpy(&gradmu[1][1][1], g + n, n * sizeof(float));
    memcpy(&gradrho[1][1][1], g + 2 * n, n * sizeof(float));
    free(g);
}

void b200_hess_F(int nx, int ny, int nz, float ****fvx, float ****fvy, float ****fvz, float ****fivx, float ****fivy,
                 float ****fivz, float ****bvx, float ****bvy, float ****bvz, float ****bivx, float ****bivy,
                 float ****bivz, float ***hess1, float ***hess2, float ***hess3, int nt, float ***rho, float ***pi,
                 float ***u, float *finv, int nf, int pshot) {
    (void)nx; (void)ny; (void)nz; (void)fvx; (void)fvy; (void)fvz; (void)fivx; (void)fivy; (void)fivz; (void)bvx;
    (void)bvy; (void)bvz; (void)bivx; (void)bivy; (void)bivz; (void)hess1; (void)hess2; (void)hess3; (void)nt;
    (void)rho; (void)pi; (void)u; (void)finv; (void)nf; (void)pshot;
    err(" B200 engine: the approximate Hessian (HESS) is not served by the drop-in host");
}
