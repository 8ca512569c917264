/*
 * b200_hooks.h — force-included (gcc -include) ahead of the reference's
 * src/ifos3d.c when the drop-in host is built. It renames, in that one file,
 * the per-step and per-shot calls of the three time loops
 * (src/ifos3d.c:754-814 forward, :909-960 back-propagation, :1070-1103
 * step-length forwards) and the calls that consume their results, so that
 * src/fd.h declares them under b200_ names with the reference's own
 * prototypes and ifos3d.c calls the B200 engine's glue (b200_glue.c) instead.
 * Everything else in ifos3d.c — JSON input, model and file IO, the residual
 * arithmetic, preconditioning, CG/L-BFGS, step length, model update — stays
 * the reference's code.
 */
#ifndef IFOSB_B200_HOOKS_H
#define IFOSB_B200_HOOKS_H

/* model and state resets */
#define av_mat b200_av_mat
#define zero_wavefield b200_zero_wavefield
#define zero_invers b200_zero_invers
#define zero_grad b200_zero_grad
/* the time step: recorded, then run as a whole time loop on the device */
#define update_v b200_update_v
#define update_v_CPML b200_update_v_CPML
#define update_s b200_update_s
#define update_s_CPML b200_update_s_CPML
#define update_s_elastic b200_update_s_elastic
#define update_s_CPML_elastic b200_update_s_CPML_elastic
#define psource b200_psource
#define surface b200_surface
#define surface_elastic b200_surface_elastic
#define discfourier b200_discfourier
#define seismo b200_seismo
#define snap b200_snap
/* halo exchanges: no-ops on one device */
#define exchange_v b200_exchange_v
#define exchange_s b200_exchange_s
#define exchange_Fv b200_exchange_Fv
/* consumers of a time loop's results */
#define saveseis b200_saveseis
#define residual b200_residual
#define gradient_F b200_gradient_F
#define hess_F b200_hess_F

#endif
