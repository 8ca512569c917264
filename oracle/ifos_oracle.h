/*
 * CPU ORACLE interface — TEST INFRASTRUCTURE ONLY.
 *
 * Two implementations export exactly these symbols:
 *   - oracle/_ref/libifos_ref.so : the reference IFOS3D sources themselves
 *     (src/update_v_ssg.c, update_s_ssg*.c, surface_ssg*.c, psource.c,
 *     seismo_ssg.c, disc_fourier.c, gradient_F.c, residual.c, av_mat.c,
 *     matcopy.c, CPML_coeff.c, wavelet.c, util.c, zero_*.c) compiled with a
 *     one-rank MPI stub and driven by oracle/ref_harness.c in the call order
 *     of src/ifos3d.c:738-974;
 *   - oracle/lib/libifos_oracle.so : oracle/ifos_oracle.c, a plain-C
 *     restatement of the same algorithm that also covers L>1 relaxation
 *     mechanisms (the reference stops at L=1, src/update_s_ssg.c:75-76).
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load either library. Neither is part of the CUDA product.
 *
 * Layout conventions (identical to the reference's NR tensors, flattened):
 *   wavefield W : [NY+5][NX+4][NZ+4]  indices j=-2..NY+2, i=-1..NX+2, k=-1..NZ+2
 *                 (src/ifos3d.c:294-337 allocation ranges for POS[2]==0, FDORDER=4)
 *   model     M : [NY][NX][NZ] interior values (ghost layers are filled inside by
 *                 the one-rank matcopy wrap, src/matcopy.c:31-327)
 *   grad      G : [NY][NX][NZ]
 *   sections    : [3][ntr][ns]  components vx, vy, vz (src/seismo_ssg.c:43-50)
 *   dft         : [6][nf] W-shaped fields, order Re vx,vy,vz then Im vx,vy,vz
 *   cpml        : [18][2*FW]  K_x,a_x,b_x,K_x_half,a_x_half,b_x_half, then y, then z
 *                 (element h of a row is the reference's vector index h+1)
 *   srcpos      : [nsrc][7]   x-index, y-index, z-index (grid points), tshift, fc, amp, stype
 *                 (the reference's srcpos_loc[1..7][l] rows, src/sources.c:44-66)
 *   recpos      : [ntr][3]    x-, y-, z-index (recpos_loc[1..3][itr])
 */
#ifndef IFOS_ORACLE_H
#define IFOS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int nx, ny, nz;        /* NX, NY, NZ (one rank: local == global) */
    float dx, dy, dz;      /* DX, DY, DZ */
    float dt;              /* DT */
    int nt;                /* NT */
    float time;            /* TIME after TIME=(NT-1)*DT (src/ifos3d.c:177) */
    int fdcoeff;           /* FDCOEFF: 1 Taylor, 2 Holberg */
    int free_surf;         /* FREE_SURF */
    int fw;                /* FW, CPML width */
    int nmech;             /* L relaxation mechanisms, 0 = elastic */
    int ndt, ndtshift;     /* NDT, NDTSHIFT seismogram sampling */
    float vppml, fpml;     /* VPPML, FPML (src/CPML_coeff.c:111-114) */
    float alpha, beta;     /* ALPHA, BETA custom force angles (src/update_v_ssg.c:498-503) */
    int source_shape;      /* SOURCE_SHAPE for wavelet() */
} ifo_params;

typedef struct {
    const float *vp, *vs, *rho;   /* [NY][NX][NZ] as read by readmod.c */
    float tau;                    /* TAU */
    const float *fl;              /* FL[1..L] relaxation frequencies, [nmech] */
} ifo_velmodel;

/* Number of samples per trace, src/ifos3d.c:178-179. */
int ifo_nsamples(const ifo_params *p);

/* readmod.c:28-139 arithmetic: vp/vs/rho -> rho, pi, u (+ taus, taup, eta). */
int ifo_readmod(const ifo_params *p, const ifo_velmodel *vm, float *rho, float *pi, float *u,
                float *taus, float *taup, float *eta);

/* CPML_coeff.c:87-324 into cpml[18][2*FW]. */
int ifo_cpml_coeff(const ifo_params *p, float *cpml);

/* wavelet.c:29-99 into signals[nsrc][NT]. */
int ifo_wavelet(const ifo_params *p, int nsrc, const float *srcpos, float *signals);

/* matcopy (one rank) + av_mat: model [NY][NX][NZ] in, averaged arrays out
 * ([NY][NX][NZ] each): uipjp, ujpkp, uipkp, rip, rjp, rkp, tausipjp, tausjpkp, tausipkp. */
int ifo_av_mat(const ifo_params *p, const float *rho, const float *pi, const float *u,
               const float *taus, const float *taup, float *avg9);

/* Forward time loop (src/ifos3d.c:738-814).
 * nf==0 runs METHOD=0 (no DFT). Outputs may be NULL. state9 = vx,vy,vz,sxx,syy,szz,sxy,syz,sxz (W each). */
int ifo_forward(const ifo_params *p, const float *rho, const float *pi, const float *u,
                const float *taus, const float *taup, const float *eta, const float *cpml,
                int nsrc, const float *srcpos, const float *signals,
                int ntr, const int *recpos, int nf, const float *finv, int ntast,
                float *sections, float *dft, float *state9);

/* residual() for the three components (src/ifos3d.c:837-858, src/residual.c:27-60).
 * obs, syn, diff: [3][ntr][ns]. *l2 accumulates exactly like the reference's float L2. */
int ifo_residual(const ifo_params *p, int ntr, const float *obs, const float *syn, float *diff, float *l2);

/* Back-propagation time loop (src/ifos3d.c:882-960): residual injected at the
 * receivers (twice with CPML), backward DFT with t = TIME - nt*DT. */
int ifo_adjoint(const ifo_params *p, const float *rho, const float *pi, const float *u,
                const float *taus, const float *taup, const float *eta, const float *cpml,
                int ntr, const int *recpos, const float *diff,
                int nf, const float *finv, int ntast, float *dft_back, float *state9);

/* gradient_F (src/gradient_F.c:30-171): grad[3][NY][NX][NZ] += contribution. */
int ifo_gradient(const ifo_params *p, const float *rho, const float *pi, const float *u,
                 int nf, const float *finv, const float *dft_fwd, const float *dft_back, float *grad);
/* hess_F for one shot against ngreen receivers' DFT fields (reference build only). */
int ifo_hessian(const ifo_params *p, const float *rho, const float *pi, const float *u, int nf, const float *finv,
                const float *dft_fwd, int ngreen, const float *dft_green, float *hess);
/* The forward with SEISMO 1-4 (reference build only): sections [3][ntr][ns],
 * pdc [3][ntr][ns] = p, div, curl. */
int ifo_forward_seismo(const ifo_params *p, const float *rho, const float *pi, const float *u,
                       const float *taus, const float *taup, const float *eta, const float *cpml,
                       int nsrc, const float *srcpos, const float *signals, int ntr, const int *recpos,
                       int seismo, float *sections, float *pdc);

#ifdef __cplusplus
}
#endif
#endif
