/*
 * ifos_b200.h — C ABI of the B200 (sm_100a) wavefield engine for IFOS3D.
 *
 * The engine replaces the three time loops of the reference driver
 * (src/ifos3d.c:754-814 forward, :909-960 back-propagation, :1070-1103
 * step-length forwards) and the per-shot kernels they call, plus
 * residual() and gradient_F(). The host program keeps its own JSON input,
 * model/gradient/SU file handling and optimiser; it calls these entry points
 * with the arrays it already owns. All device memory is owned by the library;
 * host buffers belong to the caller. Every entry point is synchronous at
 * return and returns an int status (IFOSB_OK == 0); a non-zero status is what
 * the reference turns into err() (src/util.c:30-40).
 *
 * Index conventions are the reference's: y (index j) is depth, arrays are
 * [j][i][k] with k (z) contiguous; grid indices are 1-based like the
 * reference's loops (cells 1..NX, 1..NY, 1..NZ).
 */
#ifndef IFOS_B200_H
#define IFOS_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define IFOSB_OK 0
#define IFOSB_EARG 1          /* invalid argument or unsupported parameter        */
#define IFOSB_ECUDA 2         /* CUDA runtime/launch error                        */
#define IFOSB_ENOMEM 3        /* device allocation failed                         */
#define IFOSB_EUNSTABLE 4     /* NaN probe fired (src/ifos3d.c:761, :916, :1075) */
#define IFOSB_ESTATE 5        /* call order violated (e.g. adjoint before residual) */
#define IFOSB_ENODEV 6        /* no CUDA device                                   */

/* Parameters, taken from the reference's globals (src/globvar.h). One rank:
 * NX, NY, NZ are the whole grid. */
typedef struct ifosb_params {
    int nx, ny, nz;         /* NX, NY, NZ                                          */
    float dx, dy, dz;       /* DX, DY, DZ                                          */
    float dt;               /* DT                                                  */
    int nt;                 /* NT = ceil(TIME/DT)            (src/ifos3d.c:176)    */
    float time;             /* TIME after TIME=(NT-1)*DT     (src/ifos3d.c:177)    */
    int fdorder;            /* FDORDER; only 4 is implemented                     */
    int fdcoeff;            /* FDCOEFF: 1 Taylor, 2 Holberg                       */
    int free_surf;          /* FREE_SURF (free surface at j=1)                    */
    int abs_type;           /* ABS_TYPE; only 1 (CPML) is implemented             */
    int fw;                 /* FW, CPML width in cells                            */
    int nmech;              /* L relaxation mechanisms; 0 = elastic               */
    int ndt, ndtshift;      /* NDT, NDTSHIFT seismogram sampling                  */
    float alpha, beta;      /* ALPHA, BETA (custom-force source type 5)           */
} ifosb_params;

/* One shot: the sources the reference keeps in srcpos_loc[1..7][l] and the
 * wavelets in signals[l][1..NT] (src/ifos3d.c:712-732). */
typedef struct ifosb_shot {
    int nsrc;
    const float *srcpos;   /* [nsrc][7]: x-index, y-index, z-index, tshift, fc, amp, stype */
    const float *signals;  /* [nsrc][NT] */
} ifosb_shot;

typedef struct ifosb_engine ifosb_engine;

/* Field ids for ifosb_get_field (diagnostics and parity tests). */
#define IFOSB_F_VX 0
#define IFOSB_F_VY 1
#define IFOSB_F_VZ 2
#define IFOSB_F_SXX 3
#define IFOSB_F_SYY 4
#define IFOSB_F_SZZ 5
#define IFOSB_F_SXY 6
#define IFOSB_F_SYZ 7
#define IFOSB_F_SXZ 8
#define IFOSB_F_DFT_FWD 100   /* + comp*nf + l, comp 0..5 = Re vx,vy,vz, Im vx,vy,vz */
#define IFOSB_F_DFT_BACK 200  /* + comp*nf + l */

/* ---- lifecycle ---------------------------------------------------------- */

/* Creates an engine on the current CUDA device for up to max_shots shots per
 * batch and up to max_nf DFT frequencies (0 = forward modelling only). */
int ifosb_create(const ifosb_params *p, int max_shots, int max_nf, ifosb_engine **out);
void ifosb_destroy(ifosb_engine *e);
const char *ifosb_last_error(const ifosb_engine *e);
/* Device bytes the engine holds (state, PML, DFT, model, gradient, traces). */
long long ifosb_device_bytes(const ifosb_engine *e);

/* ---- static inputs ------------------------------------------------------ */

/* CPML profiles as CPML_coeff() returns them (src/CPML_coeff.c:87-324):
 * coeff[18][2*FW], rows K_x,a_x,b_x,K_x_half,a_x_half,b_x_half, then _y, then _z;
 * element h of a row is the reference's vector index h+1 (&K_x[1] etc.). */
int ifosb_set_cpml(ifosb_engine *e, const float *coeff);

/* Model after the host's matcopy (src/ifos3d.c:681): rho, pi (=lambda+2mu), u (=mu)
 * and, when nmech>0, taus, taup as the reference allocates them,
 * f3tensor(0,NY+1,0,NX+1,0,NZ+1) — pass &rho[0][0][0]. eta[nmech] as readmod()
 * returns it (eta[l-1] = the reference's eta[l]). The staggered averages of
 * av_mat() (src/av_mat.c:28-80) are formed on the device. */
int ifosb_set_model(ifosb_engine *e, const float *rho, const float *pi, const float *u,
                    const float *taus, const float *taup, const float *eta);

/* The moduli the elastic free surface uses at j = 1, when they are not the
 * propagation model's: the reference's step-length forwards propagate in the test
 * model but call surface_elastic with the current model's u and pi
 * (src/ifos3d.c:1087-1090, src/surface_ssg_elastic.c:102-103). pi, u: ghosted
 * [NY+2][NX+2][NZ+2] arrays as for ifosb_set_model (plane j = 1 is read);
 * NULL, NULL = the propagation model's (the default). Elastic engines only. */
int ifosb_set_surface_moduli(ifosb_engine *e, const float *pi, const float *u);

/* Receivers (recpos_loc[1..3][itr], src/ifos3d.c:197-204): recpos[ntr][3] x, y, z index. */
int ifosb_set_receivers(ifosb_engine *e, int ntr, const int *recpos);

/* Monochromatic frequencies of the current stage (finv[0..nf-1], readinv.c) and the
 * DFT sampling interval ntast (src/ifos3d.c:745-749). nf=0 = forward modelling (METHOD=0). */
int ifosb_set_frequencies(ifosb_engine *e, int nf, const float *finv, int ntast);

/* ---- the time loops ----------------------------------------------------- */

/* Forward propagation of nshots shots in one batch (src/ifos3d.c:738-814 per shot):
 * zeroes the wavefield, runs NT steps of update_v/_CPML, update_s(_elastic)/_CPML,
 * psource, discfourier (if nf>0), surface, seismo. sections (optional, host):
 * [nshots][3][ntr][ns] vx, vy, vz traces, or the SEISMO components set by
 * ifosb_set_seismo. DFT fields stay on the device. */
int ifosb_forward(ifosb_engine *e, int nshots, const ifosb_shot *shots, float *sections);

/* residual() for every shot of the last forward batch (src/ifos3d.c:837-858):
 * obs [nshots][3][ntr][ns] observed traces (host memory, or device memory of the
 * engine's GPU for traces already resident there). Forms the time-reversed
 * displacement residual on the device. misfit_fp64 (optional, [nshots]) gets
 * sum(residual^2) reduced in FP64; l2_ref (optional, [nshots]) gets the same
 * sum in the reference's float accumulation order. */
int ifosb_residual(ifosb_engine *e, const float *obs, double *misfit_fp64, float *l2_ref);

/* Back-propagation (src/ifos3d.c:882-960): the residual of the last
 * ifosb_residual (or, if diff != NULL, the caller's [nshots][3][ntr][ns] residual)
 * is injected at the receivers, twice per step as the reference does with CPML,
 * and the backward DFT is accumulated with t = TIME - nt*DT. */
int ifosb_adjoint(ifosb_engine *e, const float *diff);

/* gradient_F (src/gradient_F.c:30-171) of the last forward/adjoint batch,
 * accumulated into the engine's gradient in shot order (the reference's shot
 * loop): FP32 exactly as the reference, and a parallel FP64 accumulation. */
int ifosb_gradient(ifosb_engine *e);

/* Time-domain gradient kernels of the last forward batch and its residual, with
 * checkpointing instead of the DFT: the forward is run again saving its state
 * every `interval` steps (unless that forward saved them itself, see
 * ifosb_set_td_checkpoints, or an earlier call for it did), the residual is
 * back-propagated, and each forward step
 * is recomputed from the nearest checkpoint, one segment at a time, when its
 * zero-lag adjoint step (n + m = TIME/DT, the pairing of discfourier's phases,
 * src/disc_fourier.c:36-37) is reached. kernels[4][NY][NX][NZ] (FP64, summed over
 * the batch's shots): rho  sum_t v_f . v_b;  lambda  sum_t div U_f div U_b;
 * mu  sum_t (2 sum_i e_ii,f e_ii,b + sum_i<j (e_ij+e_ji)_f (e_ij+e_ji)_b), with U
 * the running sum of v DT and e the gradient_F stencils of U; dc  U_f(NT) . U_b(NT).
 * With frequencies f_l = l / (2 NT DT) the rho kernel equals (by Parseval)
 * (dc + 2 sum_{l=1}^{NT-1} gradrho_l + gradrho_NT) / (2 NT DT^2), gradrho_l being
 * gradient_F's rho term. Elastic or viscoelastic (the checkpoints carry the memory
 * variables with the rest of the state; the kernels are the same correlations that
 * gradient_F forms at its frequencies), NDT 1, NDTSHIFT 0. Device memory:
 * ceil((TIME/DT - 1)/interval) checkpoints of the batch state plus `interval` steps
 * of six fields per shot. The DFT fields, traces and residual stay as they were;
 * the wavefield state (ifosb_get_field) is the time-domain adjoint's last step. */
int ifosb_gradient_td(ifosb_engine *e, int interval, double *kernels);

/* interval > 0: every following ifosb_forward also keeps the time-domain
 * checkpoints of that interval (the running sums U and a state every `interval`
 * steps, in the time-domain block) so that ifosb_gradient_td with the same
 * interval skips its re-run of the forward; 0 turns it off. Costs the block's
 * device memory and one extra pass over v per forward step. */
int ifosb_set_td_checkpoints(ifosb_engine *e, int interval);

/* Viscoelastic engines (nmech > 0): the accumulated FP64 gradients with respect
 * to the model's taup and taus (gradq[2][NY][NX][NZ]), summed like grad64 by
 * ifosb_gradient and zeroed by ifosb_zero_gradient. The reference has no Q
 * gradient; this one follows from its memory-variable update
 * (src/update_s_ssg.c:108-122): in the frequency domain of discfourier a modulus
 * M acts as M (1 + tau Phi(w)), Phi = sum_l s t_l / (1 + s t_l), s = -i w,
 * t_l = DT / eta_l, so with gradient_F's lambda and mu correlations taken complex
 * (C = F conj(B), real parts = gradlam, gradmu):
 *   d/dtaup = pi sum_f Re[Phi C_lambda],  d/dtaus = u sum_f Re[Phi (C_mu - 2 C_lambda)],
 * with gradient_F's sign (minus the misfit gradient). With tau proportional to
 * 1/Q (the tau method), d/dQ = -(taup d/dtaup + taus d/dtaus) / Q. */
int ifosb_get_gradient_q(ifosb_engine *e, double *gradq);

/* The exact discrete vector-Jacobian product of the misfit (no counterpart in the
 * reference, whose gradient_F correlates a back-propagation with the forward operator,
 * src/ifos3d.c:882-975 — an approximation of the derivative). For each shot of the last
 * forward batch: the time loop in FP64 (the engine's expressions without float
 * rounding: elastic, or L relaxation mechanisms with their memory variables) with a
 * checkpoint every `interval` steps; the misfit misfit[s] = sum D^2,
 * D = DT * cumsum(syn - obs) over every trace of the shot (the residual of
 * residual.c:35-60; obs are the last ifosb_residual's observed traces); then the
 * transposed time steps in reverse — the CPML memory recursions, the memory-variable
 * recursions, the free-surface update and its image rows, the stress and velocity
 * stencils — each segment of forward states recomputed from its checkpoint.
 * grad (optional, [5][NY][NX][NZ] FP64): the derivative of the batch's summed misfit
 * with respect to the raw model ifosb_set_model received — rho, pi, u, taus, taup of
 * each interior cell (taus, taup zero for L = 0) — through av_mat's averages
 * (src/av_mat.c:45-69, the taus means at :57-59) and the model's ghost layers taken as
 * matcopy's periodic copies on one rank. NULL grad: the misfits only. Explosive
 * sources, NDT 1, NDTSHIFT 0. Device memory: ceil(NT/interval) + interval + 2 FP64
 * states of one shot (fields, 6 L memory variables, PML memory). */
int ifosb_vjp_exact_moduli(ifosb_engine *e, int interval, double *grad, double *misfit);

/* The same for elastic engines (nmech 0) with grad [3][NY][NX][NZ] with respect to
 * vp, vs, rho: the moduli gradient through pi = rho vp^2, u = rho vs^2 (readmod.c with
 * L = 0). EARG for L > 0, whose velocities depend on the reference frequency the
 * engine does not hold: take the moduli form there. */
int ifosb_vjp_exact(ifosb_engine *e, int interval, double *grad, double *misfit);

/* Zero the accumulated gradients (zero_grad, src/zero_grad.c). */
int ifosb_zero_gradient(ifosb_engine *e);

/* Copy the accumulated gradient out: grad[3][NY][NX][NZ] (vp, vs, rho; the layout of
 * grad1..3 interior) and/or the FP64 accumulation grad64[3][NY][NX][NZ]. Either may
 * be host memory or device memory (e.g. a buffer for a device-side all-reduce). */
int ifosb_get_gradient(ifosb_engine *e, float *grad, double *grad64);

/* forward + residual + adjoint + gradient for a batch: the per-shot body of
 * src/ifos3d.c:712-975 for nshots shots at once. obs as for ifosb_residual (host or
 * device memory); misfit (optional): [nshots] FP64, host. */
int ifosb_shot_gradient(ifosb_engine *e, int nshots, const ifosb_shot *shots,
                        const float *obs, double *misfit);

/* Copy one field of one shot of the last batch in the reference's wavefield
 * layout [NY+5][NX+4][NZ+4] (j=-2..NY+2, i=-1..NX+2, k=-1..NZ+2). */
int ifosb_get_field(ifosb_engine *e, int shot, int field, float *out);

/* Synchronous launch mode: 0 = the time loop is captured once into a CUDA graph
 * and replayed (default); 1 = plain stream launches, one per kernel. */
int ifosb_set_launch_mode(ifosb_engine *e, int mode);

/* Failure-path test of the bounded waits (no counterpart in the reference, whose
 * failures end in err(), src/util.c:30-40). Every mbarrier wait of the TMA time-step
 * kernels gives up after wait_ns (default and maximum 1e9 = 1 s, minimum 1000);
 * the call then returns IFOSB_ECUDA and the engine stays usable. With kernel = 1
 * (velocity) or 2 (stress) and stop_plane >= 0, that kernel's producer warp stops
 * issuing loads at iteration stop_plane of each CTA's y chunk, waits for the boxes
 * it has issued and returns, so the consumers' waits for the rest run out: the
 * path from an expired wait to the error status, made to run without a GPU fault.
 * kernel = 0 (and stop_plane = -1) restores normal launches. For tests only. */
int ifosb_set_wait_test(ifosb_engine *e, long long wait_ns, int kernel, int stop_plane);

/* Kernels launched by the last forward/adjoint call (per-step kernels x steps). */
long long ifosb_last_launch_count(const ifosb_engine *e);

/* Time-loop CUDA graphs captured so far: a call with the same batch shape and
 * inputs as an earlier one replays its graph instead of capturing a new one. */
long long ifosb_graph_captures(const ifosb_engine *e);

/* Kernel timing: with profile=1 the time loops launch kernel by kernel with a
 * CUDA event pair around every launch on the engine's stream; after a forward
 * or adjoint call ifosb_kernel_times returns the summed device milliseconds of
 * the velocity and the stress kernels and the number of steps timed. */
int ifosb_set_profiling(ifosb_engine *e, int profile);
int ifosb_kernel_times(const ifosb_engine *e, double *vel_ms, double *str_ms, int *steps);

/* Autotuner: times `steps` forward time steps of this batch (the same shots a
 * later ifosb_forward / ifosb_shot_gradient will use) for each launch shape —
 * y planes per CTA chunk (2 to 64, and the built-in choice) and the L2 prefetch
 * distance of the TMA kernels (0-3 planes) — and keeps, for each of the two
 * time-step kernels, its fastest shape for every later call with nshots shots.
 * Results do not depend on the shape (bit-identical). The batch's wavefield is
 * undefined afterwards. shape (optional, int[4]) gets the choice: velocity
 * kernel planes per chunk and prefetch distance, then the stress kernel's. */
int ifosb_autotune(ifosb_engine *e, int nshots, const ifosb_shot *shots, int steps, int *shape);

/* Sets the launch shapes for batches of nshots shots directly (the int[4] that
 * ifosb_autotune reports), e.g. a shape tuned in an earlier run. */
int ifosb_set_launch_shape(ifosb_engine *e, int nshots, const int *shape);

/* Run the engine's work on the caller's CUDA stream (a cudaStream_t passed as
 * void*; NULL = the engine's own stream). Calls stay synchronous at return. */
int ifosb_set_stream(ifosb_engine *e, void *stream);

/* SEISMO (seismo_ssg.c:27-129): 1 (default) records vx, vy, vz; 2 the pressure
 * p = -(sxx+syy+szz); 3 the divergence and curl (one-sided velocity differences,
 * scaled by sqrt(pi) and sqrt(u) as the reference does); 4 all six. ifosb_forward's
 * sections are then [nshots][ncomp][ntr][ns] with ncomp = 3, 1, 2, 6 in saveseis's
 * order (vx vy vz p div curl). The residual and adjoint use vx, vy, vz. */
int ifosb_set_seismo(ifosb_engine *e, int seismo);

/* ---- approximate Hessian (HESS; src/hess_F.c, src/ifos3d.c:882-986) --------
 * Elastic models only (the reference propagates its Hessian wavefields with
 * update_s_elastic), NDT = 1, NDTSHIFT = 0, frequencies set.
 *
 * ifosb_hessian_green: the Hessian wavefields of the reference's pshot loop
 * (ifos3d.c:887-938) for receivers rec_ids[0..nrec-1] (indices into the
 * receiver list): each is a y-velocity injection of its row of signals
 * [nrec][NT] at the receiver, propagated in adjoint mode with the backward DFT
 * (discfourier, back = 1). The reference's row is wavelet(..., 5, ...) of the
 * receiver's recpos_loc column with amplitude 1 (a step at t = row 4), low-passed
 * when FILT. They are kept on the
 * device until the model, receivers or frequencies change. Destroys the current
 * wavefield state (call before a batch's forward).
 * ifosb_hessian: replaces hess_F (hess_F.c:25-160) for the shots of the last
 * forward batch, adding to the device Hessian in the reference's order (shots,
 * receivers, frequencies), FP32, the same bits.
 * ifosb_zero_hessian / ifosb_get_hessian: hess [3][NY][NX][NZ] (vp, vs, rho). */
int ifosb_hessian_green(ifosb_engine *e, int nrec, const int *rec_ids, const float *signals);
int ifosb_hessian(ifosb_engine *e);
int ifosb_zero_hessian(ifosb_engine *e);
int ifosb_get_hessian(ifosb_engine *e, float *hess);

/* ---- host utilities (restated reference host code) ---------------------- */

/* CPML_coeff (src/CPML_coeff.c:87-324) with VPPML, FPML into coeff[18][2*FW]. */
int ifosb_cpml_coeff(const ifosb_params *p, float vppml, float fpml, float *coeff);

/* wavelet (src/wavelet.c:29-99) for source shapes 1, 2, 4, 5: signals[nsrc][NT]. */
int ifosb_wavelet(const ifosb_params *p, int shape, int nsrc, const float *srcpos, float *signals);

/* readmod (src/readmod.c:28-139) without the file reading: vp, vs, rho [n] ->
 * rho stays, pi = vp^2 rho/(1+sumpi), u = vs^2 rho/(1+sumu) (relaxed moduli at
 * ws = 2 pi FL[1]), taus = taup = TAU, eta[l] = DT/tau_sigma_l. fl[nmech] = FL[1..L]. */
int ifosb_moduli(const ifosb_params *p, long long n, const float *vp, const float *vs, const float *rho, float tau,
                 const float *fl, float *pi, float *u, float *taus, float *taup, float *eta);

/* Number of samples per trace ns (src/ifos3d.c:178-179). */
int ifosb_nsamples(const ifosb_params *p);

/* ---- inversion-loop updates (src/ifos3d.c:1005-1138) -------------------- */

/* The model-space state of the reference's optimiser on the device: the CG
 * priors gradprior1..6 and the L-BFGS history bfgsmod/bfgsgrad/bfgsscale.
 * Dot products and the L-BFGS work vector are FP64 (the reference: float and
 * MPI_FLOAT), reduced in a fixed order. Gradient and model pointers may be
 * host or device memory. n = NX*NY*NZ; gradients are grad[3][NY][NX][NZ]
 * (vp, vs, rho: grad1..3 interior); models are the ghosted
 * [NY+2][NX+2][NZ+2] arrays of ifosb_set_model (interior updated). */
typedef struct ifosb_optim ifosb_optim;

/* numpar = NUMPAR (1: vp, 2: vp and vs in L-BFGS), bfgsnum = BFGSNUM (0: CG only). */
int ifosb_optim_create(int nx, int ny, int nz, int numpar, int bfgsnum, ifosb_optim **out);
void ifosb_optim_destroy(ifosb_optim *o);
const char *ifosb_optim_last_error(const ifosb_optim *o);

/* conjugate (src/conjugategrad.c:27-110): cdf=1 starts a new sequence (grad
 * unchanged); otherwise Mora's beta with FP64 sums, the reference's clamp of
 * beta[0] to [0, 0.5] (beta[1], beta[2] are not clamped there), and
 * grad = prior*beta + grad in place. beta (optional) gets the three betas. */
int ifosb_conjugate(ifosb_optim *o, float *grad, int cdf, double *beta);

/* lbfgs_savegrad (src/lbfgs_save.c:25-56): the first iteration's gradient. */
int ifosb_lbfgs_savegrad(ifosb_optim *o, const float *grad);

/* lbfgs (src/lbfgs.c:26-181) for it_group >= 2: the two-loop recursion over
 * the last BFGSNUM pairs in FP64; grad (vp[, vs]) is replaced by the direction. */
int ifosb_lbfgs(ifosb_optim *o, float *grad, int it_group);

/* modelupdate (src/modelupdate.c:26-160): without L-BFGS the gradients are first
 * normalised by their maxima (in place, as the reference does); then
 * vp, vs, rho += step*WEIGHT*grad*(VP0, VS0, RHO0) with the reference's float
 * arithmetic (bit-identical) and rho, pi, u rewritten. With L-BFGS the model
 * difference of slot it_group%BFGSNUM is recorded in FP64. weight[3] = WEIGHT. */
int ifosb_modelupdate(ifosb_optim *o, float *grad, float *rho, float *pi, float *u, float step,
                      const float *weight, float vp0, float vs0, float rho0, int lbfgs, int it_group);

/* precon_grad (src/precongrad.c:28-336): damping of grad[3][NY][NX][NZ] in place
 * around sources (damptype 2), receivers (1, 2) and towards the model edges, as
 * DAMPTYPE selects, with the reference's float results (the factors come from
 * its double expressions, tabulated on the host). Quirks kept: with free_surf
 * the y factor at the top is 0, so types 0-2 zero the gradient; types 0 and 3
 * evaluate their edge factors at index 0 (the loop variables they read are
 * never set). srcpos[nsrc][3]: source x, y, z in metres (srcpos[1..3][l]);
 * recpos[ntr][3]: receiver grid indices (recpos[1..3][n]). */
int ifosb_precon_grad(ifosb_optim *o, float *grad, int damptype, int free_surf, int fw, float dx, float dy, float dz,
                      int nsrc, const float *srcpos, int ntr, const int *recpos);

/* constant_boundary (src/constant_boundary.c:27-222), one rank, on the ghosted
 * model rho, pi, u [NY+2][NX+2][NZ+2] in place: the model in the x and z CPML
 * frames (and 4 cells more) replaced by copies and 6-point averages of the
 * cells just inside, in the reference's order (later faces read cells earlier
 * faces rewrote), with its double averages. The driver calls it after a model
 * update when FREE_SURF (src/ifos3d.c:682, :1035). */
int ifosb_constant_boundary(ifosb_optim *o, float *rho, float *pi, float *u, int fw);

/* The L-BFGS history for inspection: s, y [BFGSNUM][NUMPAR*n], scale [BFGSNUM]. */
int ifosb_lbfgs_history(const ifosb_optim *o, double *s, double *y, double *scale);

/* steplength (src/steplength.c:26-91) in FP64: L2[0..2] misfits at step[0..2]
 * (step[0] = 0), step[4] the test step; writes step[3] (the parabola's minimum
 * with the reference's limits), L2[3] and the next test step step[4].
 * abc (optional) gets the parabola coefficients a, b, c. Scalar work: it runs
 * on the host in FP64. */
int ifosb_steplength(double *L2, double *step, int lbfgs, int it_group, double teststep, double *abc);

/* hess_apply (src/hess_apply.c:25-79, called at src/ifos3d.c:1002): grad [3][ny][nx][nz]
 * (host or device pointer) divided by hess + water[c] (WATER_HESS), after scaling by
 * VP0, VS0, RHO0 when lbfgs; the same bits as the reference. */
int ifosb_hess_apply(ifosb_optim *o, float *grad, const float *hess, const float *water, int lbfgs, float vp0,
                     float vs0, float rho0);

/* ---- residual without allocation ---------------------------------------- */

/* No counterpart in the reference (its residual() works on host arrays).
 *
 * ifosb_residual_noalloc computes what ifosb_residual computes — the
 * time-integrated, time-reversed residual of residual() (src/residual.c:35-60)
 * and the per-shot FP64 misfit, the same bits — for traces that already sit in
 * the caller's device memory, without an engine and without allocating: no
 * cudaMalloc/cudaFree and no allocating library call. It is for callers that
 * cannot allocate at that point: a shot planner that has filled HBM with
 * wavefield batches and has no room left; a pipeline that evaluates misfits on
 * one stream while propagation runs on another, where cudaMalloc/cudaFree would
 * synchronise the device; a host whose device memory all comes from its own pool.
 *
 * d_syn, d_obs, d_diff: device [nshots][3][ntr][ns] float (synthetic, observed,
 * residual out); d_misfit: device [nshots] double. d_diff must not overlap d_syn
 * or d_obs (the residual is written time-reversed while the inputs are read
 * forward): an overlapping call returns IFOSB_EARG. The work is enqueued on
 * `stream` (a cudaStream_t as void*, NULL = the legacy default stream) and the
 * call returns without waiting for it — unlike the other entry points. A CUDA
 * error already pending on the calling thread is left in place and the call
 * returns IFOSB_ECUDA without launching.
 *
 * The per-trace partial sums live in a fixed device array of
 * IFOSB_NOALLOC_MAX_TRACES doubles (512 KiB) per device; nothing in it has to be
 * zero at the start of a call. Limit: nshots*3*ntr <= IFOSB_NOALLOC_MAX_TRACES,
 * else IFOSB_ETOOBIG and nothing is launched. The first call on each device
 * looks up that array's address (cudaGetSymbolAddress), and so does the first
 * call after the device's context changed (e.g. after cudaDeviceReset); make
 * those calls before any stream capture. Calls on one stream run in order; calls
 * that overlap in time on the same device (two streams, two host threads) share
 * the array and race. */
#define IFOSB_ETOOBIG 7
#define IFOSB_NOALLOC_MAX_TRACES 65536
int ifosb_residual_noalloc(int nshots, int ntr, int ns, float dt, const float *d_syn, const float *d_obs,
                           float *d_diff, double *d_misfit, void *stream);

/* ---- on-disk formats (host; the files IFOS3D writes and reads) ------------
 * No engine and no GPU: plain C file IO in the host's byte order.
 * Return IFOSB_OK, IFOSB_EARG (bad argument, or a file name longer than 4095
 * bytes), IFOSB_ENOMEM (host allocation) or IFOSB_EIO (file cannot be opened,
 * read or written). */
#define IFOSB_EIO 8

/* One component's seismograms in the reference's format, replacing outseis()
 * (src/outseis.c:30-276; called from src/saveseis.c:76-81).
 * section: [ntr][ns] float. rec: [ntr][3] global receiver grid indices (x, y, z),
 * i.e. recpos[1..3][recpos_loc[4][t]]. trace_no: [ntr] trace numbers written to
 * tracl (recpos_loc[4][t]); NULL = 1..ntr. src: the shot's source position in
 * metres (x, y, z) or NULL = 0, as for nsrc != 1. comp is accepted for the
 * reference's signature; it does not reach the file. fmt = SEIS_FORMAT: 0 or 1 SU
 * (240-byte trace header + ns floats per trace), 2 ASCII (%e, one column per
 * trace), 3 raw floats, byte-swapped when littlebig != 0 (LITTLEBIG). Header
 * fields outseis() leaves unassigned (cdp, selev, swdep, trailing pad) are zero. */
int ifosb_write_seis(const char *path, int comp, const float *section, int ntr, int ns, const int *rec,
                     const int *trace_no, const float *src, float dx, float dy, float dz, int ndt, float dt, int fmt,
                     int littlebig);

/* Rank 0's merge of the ranks' SU files into one (src/saveseis.c:86-229): the
 * whole traces (240 + 4 ns bytes each) of inputs[0..nin-1] in order; a missing
 * input is skipped, an input whose size is not a whole number of traces
 * contributes nothing. *ntr_out (may be NULL) = traces written. */
int ifosb_merge_seis(const char *out, int nin, const char *const *inputs, int ns, int *ntr_out);

/* Observed seismograms, replacing readseis() (src/readseis.c:25-69): ntr traces,
 * each a 240-byte header (skipped) and ns floats, into section [ntr][ns]; samples
 * past the end of the file read as 0. A missing file is IFOSB_EIO. */
int ifosb_read_seis(const char *path, float *section, int ntr, int ns);

/* readseis_split() (src/readseis_split.c:25-65): the traces t with keep[t] == 1
 * (rnum_loc), packed in file order into section [count][ns]. */
int ifosb_read_seis_split(const char *path, float *section, int ntr, const int *keep, int ns);

/* Model files of outmod() + mergemod() for one rank (src/outmod.c:25-84,
 * src/mergemod.c:25-80): "<base>.vp_it<iteration>", ".vs_it", ".rho_it", each
 * [z][x][y] floats (y fastest), vp = sqrt(pi/rho), vs = sqrt(u/rho). rho, pi, u:
 * [ny][nx][nz] (ghost = 0) or the reference's ghosted [ny+2][nx+2][nz+2]
 * (ghost = 1). idx, idy, idz = IDX, IDY, IDZ: mergemod keeps the first
 * ceil(NZ/IDZ)*ceil(NX/IDX)*ceil(NY/IDY) values of the full-resolution file,
 * and so does this. */
int ifosb_write_model(const char *base, int iteration, int nx, int ny, int nz, const float *rho, const float *pi,
                      const float *u, int ghost, int idx, int idy, int idz);

/* Gradient files of outgrad() + mergemod() (src/outgrad.c:25-85):
 * "<base>.vp_<finv %4.2f>Hz_it<iteration>", ".vs_...", ".rho_..." from grad =
 * [3][ny][nx][nz] (ghost = 0) or [3][ny+2][nx+2][nz+2] (ghost = 1). */
int ifosb_write_gradient(const char *base, float finv, int iteration, int nx, int ny, int nz, const float *grad,
                         int ghost, int idx, int idy, int idz);

/* Hessian files written by outgrad (HESS_FILE) read back as readhess() does
 * (src/readhess.c:25-95): hess [3][ny][nx][nz] = file value * VP0^2, VS0^2, RHO0^2. */
int ifosb_read_hessian(const char *base, float finv, int iteration, int nx, int ny, int nz, float vp0, float vs0,
                       float rho0, float *hess);

/* ---- multiscale stages (host) ---------------------------------------------
 * Time-domain Butterworth filter of FILT = 1, replacing filt_seis()
 * (src/filt_seis.c:27-77, which calls libcseife's seife_lpb / seife_hpb): each of
 * the ntr traces of data [ntr][ns] is filtered in place in double precision,
 * corner frequency finv (the stage's highest frequency), sample interval dt,
 * order `order` (the reference uses 4), low-pass (highpass = 0, the reference's
 * method 1) or high-pass. As in the reference, the last sample of each trace
 * is left unfiltered. */
int ifosb_filt_seis(float *data, int ntr, int ns, float finv, float dt, int order, int highpass);

/* Model resampling between multiscale grids (the reference has none): src
 * [ny][nx][nz] with spacing dx, dy, dz onto dst [my][mx][mz] with spacing ex, ey,
 * ez, by trilinear interpolation at the cell positions (i*dx etc.), constant
 * outside the source grid, in double, rounded once. Host or device pointers; runs
 * on the current CUDA device. */
int ifosb_resample(const float *src, int nx, int ny, int nz, float dx, float dy, float dz, float *dst, int mx, int my,
                   int mz, float ex, float ey, float ez);

#ifdef __cplusplus
}
#endif
#endif
