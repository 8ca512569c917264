// Exact discrete vector-Jacobian product of the elastic time loop (FP64).
//
// The reference's gradient (gradient_F.c:30-171 over the discfourier fields of a
// forward and a back-propagation driven by the time-reversed residual) is an
// approximation of the misfit's derivative: the back-propagation uses the
// forward operator, not its transpose, and the CPML recursions, the doubled
// injection (update_v_ssg_CPML.c:384-393) and the free-surface mirror are not
// transposed. This file holds the transpose itself, for a gradient that a
// finite-difference check can hold to rounding.
//
// One time step n of the elastic forward (update_v + update_v_CPML, then
// update_s_elastic + update_s_CPML_elastic, psource, surface_elastic and its
// mirror rows; seismo samples v after the step) is linear in the state
// x = (v, sigma, psi_sigma, psi_v):
//   A: v^n = v^{n-1} + T(sigma^{n-1}, psi_sigma) / rho_avg          (velocity)
//   B: sigma^n = sigma^{n-1} + DT C(model) E(v^n, psi_v) (+ sources, surface)
// where T and E are the 4th-order staggered derivatives with their CPML memory
// recursions psi' = b psi + a d, d_eff = d / K + psi'. The kernels below run the
// forward in FP64 (same expressions, no float rounding) and the transposed step
//   lambda^{n-1} = A^T B^T lambda^n,
// accumulating d misfit / d (pi, u, uipjp, ujpkp, uipkp, rip, rjp, rkp) per cell
// from lambda^n and the forward states x^{n-1}, x^n. The host folds those through
// av_mat's averages (av_mat.c:45-69) and the ghost wrap of matcopy onto the raw
// model, then onto vp, vs, rho.
//
// The misfit is the engine's: J = sum over shots, components, traces and samples of
// D[n]^2, D = DT * cumsum(syn - obs) (residual.c:35-60, the sum of squares does not
// depend on the time reversal), whose derivative with respect to the sample syn[k]
// is 2 DT sum_{n >= k} D[n]: the adjoint source injected at the receivers.
//
// Layout: the engine's padded fields ([slot][field], slots vx vy vz syy sxy syz sxx
// szz sxz) and PML slabs, in double. Plain kernels, one thread per cell.
#pragma once

namespace ifosb {

struct Vjp64 {
    Geo g;
    Slabs sl;
    const double *md;   // [N64][field]: pi, u, uipjp, ujpkp, uipkp, rip, rjp, rkp, taus, taup, tausipjp, tausjpkp, tausipkp
    const float *cpg;   // CPML rows [18][2*MAXFW] (float, as the engine's)
    double b1, b2, dx, dy, dz, rdx, rdy, rdz, dt;  // dx = DT/DX (velocity update), rdx = DX
    int nsrc;
    const int *src;     // [nsrc][3] j, i, k of explosive sources
    const double *amp;  // [nsrc][NT] psource amplitudes
    int nt_total;
    // L relaxation mechanisms (0 = elastic): eta_l = DT/tau_l and the update's
    // 1/(1+eta/2), 1-eta/2 and the surface's eta/(1+eta/2) (update_s_ssg.c:123-124,
    // surface_ssg.c:152)
    int nmech;
    double eta[MAXMECH], bb[MAXMECH], cc[MAXMECH], msb[MAXMECH];
};

enum {
    M64_PI = 0, M64_U, M64_UIPJP, M64_UJPKP, M64_UIPKP, M64_RIP, M64_RJP, M64_RKP,
    M64_TAUS, M64_TAUP, M64_TSIPJP, M64_TSJPKP, M64_TSIPKP, N64
};

__device__ __forceinline__ double cp64(const float *cpg, int row, int h) { return (double)cpg[row * 2 * MAXFW + h - 1]; }

// the averaged model in double from the raw ghosted model ([NY+2][NX+2][NZ+2] floats):
// the expressions of av_mat (av_mat.c:45-69) without their float rounding
__global__ void k64_model(Geo g, const float *rho, const float *pi, const float *u, const float *taus,
                          const float *taup, double *md) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1, i = blockIdx.y + 1, j = blockIdx.z + 1;
    if (k > g.nz) return;
    const long long F = g.field, c = widx(g, j, i, k);
    const int GX = g.nx + 2, GZ = g.nz + 2;
    auto G = [&](const float *a, int jj, int ii, int kk) { return (double)a[((long long)jj * GX + ii) * GZ + kk]; };
    md[M64_PI * F + c] = G(pi, j, i, k);
    md[M64_U * F + c] = G(u, j, i, k);
    md[M64_UIPJP * F + c] = 4.0 / (1.0 / G(u, j, i, k) + 1.0 / G(u, j, i + 1, k) + 1.0 / G(u, j + 1, i + 1, k) + 1.0 / G(u, j + 1, i, k));
    md[M64_UJPKP * F + c] = 4.0 / (1.0 / G(u, j, i, k) + 1.0 / G(u, j, i, k + 1) + 1.0 / G(u, j + 1, i, k + 1) + 1.0 / G(u, j + 1, i, k));
    md[M64_UIPKP * F + c] = 4.0 / (1.0 / G(u, j, i, k) + 1.0 / G(u, j, i, k + 1) + 1.0 / G(u, j, i + 1, k + 1) + 1.0 / G(u, j, i + 1, k));
    md[M64_RIP * F + c] = 0.5 * (G(rho, j, i, k) + G(rho, j, i + 1, k));
    md[M64_RJP * F + c] = 0.5 * (G(rho, j, i, k) + G(rho, j + 1, i, k));
    md[M64_RKP * F + c] = 0.5 * (G(rho, j, i, k) + G(rho, j, i, k + 1));
    if (taus) {
        md[M64_TAUS * F + c] = G(taus, j, i, k);
        md[M64_TAUP * F + c] = G(taup, j, i, k);
        md[M64_TSIPJP * F + c] = 0.25 * (G(taus, j, i, k) + G(taus, j, i + 1, k) + G(taus, j + 1, i + 1, k) + G(taus, j + 1, i, k));
        md[M64_TSJPKP * F + c] = 0.25 * (G(taus, j, i, k) + G(taus, j + 1, i, k) + G(taus, j + 1, i, k + 1) + G(taus, j, i, k + 1));
        md[M64_TSIPKP * F + c] = 0.25 * (G(taus, j, i, k) + G(taus, j, i + 1, k) + G(taus, j, i + 1, k + 1) + G(taus, j, i, k + 1));
    }
}

// 4th-order differences: "up" reads f[c+1] - f[c] (and f[c+2] - f[c-1]),
// "dn" reads f[c] - f[c-1] (and f[c+1] - f[c-2]); o = the axis stride
__device__ __forceinline__ double dup(const double *f, long long c, long long o, double b1, double b2) {
    return b1 * (f[c + o] - f[c]) + b2 * (f[c + 2 * o] - f[c - o]);
}
__device__ __forceinline__ double ddn(const double *f, long long c, long long o, double b1, double b2) {
    return b1 * (f[c] - f[c - o]) + b2 * (f[c + o] - f[c - 2 * o]);
}
// their transposes, gathered at the cell the difference reads: for d = dup(f), the
// adjoint of f at c' is b1 (l[c'-o] - l[c']) + b2 (l[c'-2o] - l[c'+o]); for d = ddn(f),
// b1 (l[c'] - l[c'+o]) + b2 (l[c'-o] - l[c'+2o])
__device__ __forceinline__ double tup(const double *l, long long c, long long o, double b1, double b2) {
    return b1 * (l[c - o] - l[c]) + b2 * (l[c - 2 * o] - l[c + o]);
}
__device__ __forceinline__ double tdn(const double *l, long long c, long long o, double b1, double b2) {
    return b1 * (l[c] - l[c + o]) + b2 * (l[c - o] - l[c + 2 * o]);
}

// CPML recursion of one derivative: psi' = b psi + a d, returns d / K + psi'
__device__ __forceinline__ double cpml_fwd(double d, double &psi, double K, double a, double b) {
    psi = b * psi + a * d;
    return d / K + psi;
}
// its transpose: W = adjoint of the output, L = adjoint of psi' carried from the
// next step; returns the adjoint of d and leaves the adjoint of the old psi in L
__device__ __forceinline__ double cpml_adj(double W, double &L, double K, double a, double b) {
    const double Lp = L + W;
    L = b * Lp;
    return W / K + a * Lp;
}

// ---- forward (FP64) -------------------------------------------------------

// velocity update of the interior cells (update_v_ssg.c:102-127 with update_v_ssg_CPML.c)
__global__ void k64_vel(Vjp64 a, double *st, double *ps) {
    const Geo &g = a.g;
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1, i = blockIdx.y + 1, j = blockIdx.z + 1;
    if (k > g.nz) return;
    const long long F = g.field, c = widx(g, j, i, k), dI = g.pz, dJ = g.plane;
    const double *sxx = st + SXX * F, *syy = st + SYY * F, *szz = st + SZZ * F;
    const double *sxy = st + SXY * F, *syz = st + SYZ * F, *sxz = st + SXZ * F;
    const double b1 = a.b1, b2 = a.b2;
    double sxx_x = a.dx * dup(sxx, c, dI, b1, b2), sxy_y = a.dy * ddn(sxy, c, dJ, b1, b2), sxz_z = a.dz * ddn(sxz, c, 1, b1, b2);
    double syy_y = a.dy * dup(syy, c, dJ, b1, b2), sxy_x = a.dx * ddn(sxy, c, dI, b1, b2), syz_z = a.dz * ddn(syz, c, 1, b1, b2);
    double szz_z = a.dz * dup(szz, c, 1, b1, b2), sxz_x = a.dx * ddn(sxz, c, dI, b1, b2), syz_y = a.dy * ddn(syz, c, dJ, b1, b2);
    const int hx = face_x(g, i), hy = face_y(g, j), hz = face_z(g, k);
    const float *cg = a.cpg;
    if (hx) {
        double *p = ps + sxi(g, j, hx, k);
        const long long o = a.sl.sx;
        sxx_x = cpml_fwd(sxx_x, p[0], cp64(cg, KH_X, hx), cp64(cg, AH_X, hx), cp64(cg, BH_X, hx));
        sxy_x = cpml_fwd(sxy_x, p[o], cp64(cg, K_X, hx), cp64(cg, A_X, hx), cp64(cg, B_X, hx));
        sxz_x = cpml_fwd(sxz_x, p[2 * o], cp64(cg, K_X, hx), cp64(cg, A_X, hx), cp64(cg, B_X, hx));
    }
    if (hy) {
        double *p = ps + 3 * a.sl.sx + syi(g, hy, i, k);
        const long long o = a.sl.sy;
        sxy_y = cpml_fwd(sxy_y, p[0], cp64(cg, K_Y, hy), cp64(cg, A_Y, hy), cp64(cg, B_Y, hy));
        syy_y = cpml_fwd(syy_y, p[o], cp64(cg, KH_Y, hy), cp64(cg, AH_Y, hy), cp64(cg, BH_Y, hy));
        syz_y = cpml_fwd(syz_y, p[2 * o], cp64(cg, K_Y, hy), cp64(cg, A_Y, hy), cp64(cg, B_Y, hy));
    }
    if (hz) {
        double *p = ps + 3 * a.sl.sx + 3 * a.sl.sy + szi(g, j, i, hz);
        const long long o = a.sl.sz;
        sxz_z = cpml_fwd(sxz_z, p[0], cp64(cg, K_Z, hz), cp64(cg, A_Z, hz), cp64(cg, B_Z, hz));
        syz_z = cpml_fwd(syz_z, p[o], cp64(cg, K_Z, hz), cp64(cg, A_Z, hz), cp64(cg, B_Z, hz));
        szz_z = cpml_fwd(szz_z, p[2 * o], cp64(cg, KH_Z, hz), cp64(cg, AH_Z, hz), cp64(cg, BH_Z, hz));
    }
    st[VX * F + c] += (sxx_x + sxy_y + sxz_z) / a.md[M64_RIP * F + c];
    st[VY * F + c] += (syy_y + sxy_x + syz_z) / a.md[M64_RJP * F + c];
    st[VZ * F + c] += (szz_z + sxz_x + syz_y) / a.md[M64_RKP * F + c];
}

// the nine velocity derivatives of the stress update at a cell (plain, then with
// their CPML recursions; the front z face divides by K_y as the reference does,
// update_s_ssg_CPML_elastic.c:104-108). ps null: read the old psi without updating.
struct VDer {
    double d[9];  // plain: xx xy xz yx yy yz zx zy zz
    double e[9];  // effective (CPML applied)
};
__device__ __forceinline__ void vel_derivs(const Vjp64 &a, const double *st, double *ps, int j, int i, int k, VDer &o) {
    const Geo &g = a.g;
    const long long F = g.field, c = widx(g, j, i, k), dI = g.pz, dJ = g.plane;
    const double *vx = st + VX * F, *vy = st + VY * F, *vz = st + VZ * F;
    const double b1 = a.b1, b2 = a.b2;
    o.d[0] = ddn(vx, c, dI, b1, b2) / a.rdx;
    o.d[1] = dup(vx, c, dJ, b1, b2) / a.rdy;
    o.d[2] = dup(vx, c, 1, b1, b2) / a.rdz;
    o.d[3] = dup(vy, c, dI, b1, b2) / a.rdx;
    o.d[4] = ddn(vy, c, dJ, b1, b2) / a.rdy;
    o.d[5] = dup(vy, c, 1, b1, b2) / a.rdz;
    o.d[6] = dup(vz, c, dI, b1, b2) / a.rdx;
    o.d[7] = dup(vz, c, dJ, b1, b2) / a.rdy;
    o.d[8] = ddn(vz, c, 1, b1, b2) / a.rdz;
    for (int q = 0; q < 9; ++q) o.e[q] = o.d[q];
    const int hx = face_x(g, i), hy = face_y(g, j), hz = face_z(g, k);
    const float *cg = a.cpg;
    double tmp;
    if (hx) {
        double *p = ps + sxi(g, j, hx, k);
        const long long s = a.sl.sx;
        tmp = p[0]; o.e[0] = cpml_fwd(o.d[0], tmp, cp64(cg, K_X, hx), cp64(cg, A_X, hx), cp64(cg, B_X, hx)); p[0] = tmp;
        tmp = p[s]; o.e[3] = cpml_fwd(o.d[3], tmp, cp64(cg, KH_X, hx), cp64(cg, AH_X, hx), cp64(cg, BH_X, hx)); p[s] = tmp;
        tmp = p[2 * s]; o.e[6] = cpml_fwd(o.d[6], tmp, cp64(cg, KH_X, hx), cp64(cg, AH_X, hx), cp64(cg, BH_X, hx)); p[2 * s] = tmp;
    }
    if (hy) {
        double *p = ps + 3 * a.sl.sx + syi(g, hy, i, k);
        const long long s = a.sl.sy;
        tmp = p[0]; o.e[1] = cpml_fwd(o.d[1], tmp, cp64(cg, KH_Y, hy), cp64(cg, AH_Y, hy), cp64(cg, BH_Y, hy)); p[0] = tmp;
        tmp = p[s]; o.e[4] = cpml_fwd(o.d[4], tmp, cp64(cg, K_Y, hy), cp64(cg, A_Y, hy), cp64(cg, B_Y, hy)); p[s] = tmp;
        tmp = p[2 * s]; o.e[7] = cpml_fwd(o.d[7], tmp, cp64(cg, KH_Y, hy), cp64(cg, AH_Y, hy), cp64(cg, BH_Y, hy)); p[2 * s] = tmp;
    }
    if (hz) {
        const bool zfront = k <= g.fw;
        double *p = ps + 3 * a.sl.sx + 3 * a.sl.sy + szi(g, j, i, hz);
        const long long s = a.sl.sz;
        const double kh = zfront ? cp64(cg, KH_Y, hz) : cp64(cg, KH_Z, hz);
        const double kf = zfront ? cp64(cg, K_Y, hz) : cp64(cg, K_Z, hz);
        tmp = p[0]; o.e[2] = cpml_fwd(o.d[2], tmp, kh, cp64(cg, AH_Z, hz), cp64(cg, BH_Z, hz)); p[0] = tmp;
        tmp = p[s]; o.e[5] = cpml_fwd(o.d[5], tmp, kh, cp64(cg, AH_Z, hz), cp64(cg, BH_Z, hz)); p[s] = tmp;
        tmp = p[2 * s]; o.e[8] = cpml_fwd(o.d[8], tmp, kf, cp64(cg, A_Z, hz), cp64(cg, B_Z, hz)); p[2 * s] = tmp;
    }
}

// stress update with L memory-variable mechanisms, explosive sources, free
// surface and its mirror rows (update_s_ssg_elastic.c:106-140 for L = 0,
// update_s_ssg.c:108-140 generalised to L mechanisms, psource.c:38-52,
// surface_ssg_elastic.c:69-111 and surface_ssg.c:117-160). With
// gg = pi (1 + L taup), f = 2u (1 + L taus), f_xy = DT uipjp (1 + L tausipjp) ...:
//   sigma' = sigma + DT C(gg, f, f_xy..) e + DT/2 (sum_l r_l + sum_l r_l')
//   r_l'   = bb_l (cc_l r_l - D_l(e)),  D_l with E_l = pi eta_l taup, D_l = 2u eta_l taus
//            (normal) and uipjp eta_l tausipjp ... (shear)
// At the surface (j = 1): syy = 0, r_yy = 0, sxx and szz gain h + DT/2 sum_l hh_l and
// r_xx, r_zz gain hh_l, hh_l = msb_l ((dd - ee)(f/gg - 1)(dxx + dzz) - (dd - ee) dyy),
// dd = 2u taus, ee = pi taup, on the plain derivatives.
struct Mod64 {
    double pim, um, uipjp, ujpkp, uipkp, taus, taup, tsipjp, tsjpkp, tsipkp;
};
__device__ __forceinline__ Mod64 mod64(const Vjp64 &a, long long c) {
    const long long F = a.g.field;
    const double *md = a.md;
    Mod64 m;
    m.pim = md[M64_PI * F + c]; m.um = md[M64_U * F + c];
    m.uipjp = md[M64_UIPJP * F + c]; m.ujpkp = md[M64_UJPKP * F + c]; m.uipkp = md[M64_UIPKP * F + c];
    if (a.nmech) {
        m.taus = md[M64_TAUS * F + c]; m.taup = md[M64_TAUP * F + c];
        m.tsipjp = md[M64_TSIPJP * F + c]; m.tsjpkp = md[M64_TSJPKP * F + c]; m.tsipkp = md[M64_TSIPKP * F + c];
    } else {
        m.taus = m.taup = m.tsipjp = m.tsjpkp = m.tsipkp = 0.0;
    }
    return m;
}

__global__ void k64_str(Vjp64 a, double *st, double *ps, int nt) {
    const Geo &g = a.g;
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1, i = blockIdx.y + 1, j = blockIdx.z + 1;
    if (k > g.nz) return;
    const long long F = g.field, c = widx(g, j, i, k), dJ = g.plane;
    VDer v;
    vel_derivs(a, st, ps + 3 * (a.sl.sx + a.sl.sy + a.sl.sz), j, i, k, v);
    const Mod64 m = mod64(a, c);
    const int L = a.nmech;
    const double DT = a.dt, h = 0.5 * DT, Lf = L;
    const double *e = v.e;
    const double gg = m.pim * (1.0 + Lf * m.taup), f = 2.0 * m.um * (1.0 + Lf * m.taus);
    const double fxy = DT * m.uipjp * (1.0 + Lf * m.tsipjp), fyz = DT * m.ujpkp * (1.0 + Lf * m.tsjpkp),
                 fxz = DT * m.uipkp * (1.0 + Lf * m.tsipkp);
    const double exy = e[1] + e[3], eyz = e[5] + e[7], exz = e[2] + e[6];
    const double div = e[0] + e[4] + e[8], syz_ = e[4] + e[8], sxz_ = e[0] + e[8], sxy_ = e[0] + e[4];
    double *S = st + c;
    // sigma slots in the order xx yy zz xy yz xz of the memory variables
    double sg[6] = {S[SXX * F], S[SYY * F], S[SZZ * F], S[SXY * F], S[SYZ * F], S[SXZ * F]};
    sg[0] += DT * (gg * div - f * syz_);
    sg[1] += DT * (gg * div - f * sxz_);
    sg[2] += DT * (gg * div - f * sxy_);
    sg[3] += fxy * exy;
    sg[4] += fyz * eyz;
    sg[5] += fxz * exz;
    double rn[MAXMECH][6];
    for (int l = 0; l < L; ++l) {
        double *R = st + (NEL + 6 * l) * F + c;
        const double El = m.pim * a.eta[l] * m.taup, Dl = 2.0 * m.um * a.eta[l] * m.taus;
        const double drive[6] = {El * div - Dl * syz_, El * div - Dl * sxz_, El * div - Dl * sxy_,
                                 m.uipjp * a.eta[l] * m.tsipjp * exy, m.ujpkp * a.eta[l] * m.tsjpkp * eyz,
                                 m.uipkp * a.eta[l] * m.tsipkp * exz};
        for (int q = 0; q < 6; ++q) {
            const double ro = R[q * F];
            rn[l][q] = a.bb[l] * (a.cc[l] * ro - drive[q]);
            sg[q] += h * (ro + rn[l][q]);
        }
    }
    for (int q = 0; q < a.nsrc; ++q)
        if (a.src[3 * q] == j && a.src[3 * q + 1] == i && a.src[3 * q + 2] == k) {
            const double am = a.amp[(long long)q * a.nt_total + nt - 1];
            sg[0] += am; sg[1] += am; sg[2] += am;
        }
    if (g.free_surf && j == 1) {
        sg[1] = 0.0;
        const double X = v.d[0] + v.d[8], Y = v.d[4];
        const double hs = -(DT * (gg - f) * (gg - f) * X / gg) - (DT * (gg - f) * Y);
        sg[0] += hs;
        sg[2] += hs;
        const double dd = 2.0 * m.um * m.taus, ee = m.pim * m.taup;
        for (int l = 0; l < L; ++l) {
            const double hh = a.msb[l] * ((dd - ee) * (f / gg - 1.0) * X - (dd - ee) * Y);
            rn[l][1] = 0.0;
            rn[l][0] += hh;
            rn[l][2] += hh;
            sg[0] += h * hh;
            sg[2] += h * hh;
        }
    }
    S[SXX * F] = sg[0]; S[SYY * F] = sg[1]; S[SZZ * F] = sg[2]; S[SXY * F] = sg[3]; S[SYZ * F] = sg[4]; S[SXZ * F] = sg[5];
    for (int l = 0; l < L; ++l)
        for (int q = 0; q < 6; ++q) st[(NEL + 6 * l + q) * F + c] = rn[l][q];
    if (g.free_surf && j <= 3) {
        if (j == 1) { S[SXY * F - dJ] = -sg[3]; S[SYZ * F - dJ] = -sg[4]; }
        if (j == 2) { S[SYY * F - 2 * dJ] = -sg[1]; S[SXY * F - 3 * dJ] = -sg[3]; S[SYZ * F - 3 * dJ] = -sg[4]; }
        if (j == 3) { S[SYY * F - 4 * dJ] = -sg[1]; }
    }
}

// v at the receivers after a step: traces [3][ntr][ns], sample s
__global__ void k64_sample(Geo g, const double *st, const int *rec, int ntr, int ns, int s, double *tr) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntr) return;
    const long long F = g.field, c = widx(g, rec[3 * t + 1], rec[3 * t], rec[3 * t + 2]);
    for (int q = 0; q < 3; ++q) tr[((long long)q * ntr + t) * ns + s] = st[q * F + c];
}

// ---- transpose (FP64) -------------------------------------------------------

// the adjoint source of sample s at the receivers: lambda_v += src[comp][t][s]
__global__ void k64_inject(Geo g, double *lam, const int *rec, int ntr, int ns, int s, const double *src) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntr) return;
    const long long F = g.field, c = widx(g, rec[3 * t + 1], rec[3 * t], rec[3 * t + 2]);
    for (int q = 0; q < 3; ++q) atomicAdd(lam + q * F + c, src[((long long)q * ntr + t) * ns + s]);
}

// the mirror rows of the free surface: what the velocity update read from the
// image rows goes back to the interior stresses they were copied from, negated
__global__ void k64_mirror_T(Geo g, double *lam) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1, i = blockIdx.y + 1;
    if (k > g.nz) return;
    const long long F = g.field, dJ = g.plane;
    double *syy = lam + SYY * F, *sxy = lam + SXY * F, *syz = lam + SYZ * F;
    const long long c0 = widx(g, 0, i, k), cm = widx(g, -1, i, k);
    sxy[c0 + dJ] -= sxy[c0]; syz[c0 + dJ] -= syz[c0];          // sxy(0) = -sxy(1)
    sxy[c0 + 2 * dJ] -= sxy[cm]; syz[c0 + 2 * dJ] -= syz[cm];  // sxy(-1) = -sxy(2)
    syy[c0 + 2 * dJ] -= syy[c0];                               // syy(0) = -syy(2)
    syy[c0 + 3 * dJ] -= syy[cm];                               // syy(-1) = -syy(3)
    sxy[c0] = sxy[cm] = syz[c0] = syz[cm] = syy[c0] = syy[cm] = 0.0;
}

// parameter-gradient accumulators, compact [NY][NX][NZ]
struct Grad64 {
    double *q[N64];
};

// B^T at one interior cell: the adjoints of the nine velocity derivatives (ld),
// the velocity-derivative PML memories (lps, one step back), the stresses' and
// memory variables' adjoints one step back, and the gradients of the cell's
// coefficients. cur = x^n (v^n), prev_ps = the PML memory of x^{n-1}.
__global__ void k64_str_T(Vjp64 a, double *lam, double *lps, double *ld, const double *cur, const double *prev_ps,
                          Grad64 gr) {
    const Geo &g = a.g;
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1, i = blockIdx.y + 1, j = blockIdx.z + 1;
    if (k > g.nz) return;
    const long long F = g.field, c = widx(g, j, i, k);
    const long long mm = ((long long)(j - 1) * g.nx + (i - 1)) * g.nz + (k - 1);
    const long long poff = 3 * (a.sl.sx + a.sl.sy + a.sl.sz);
    const int hx = face_x(g, i), hy = face_y(g, j), hz = face_z(g, k);
    const float *cg = a.cpg;
    // the forward derivatives of step n: v^n with the old psi_v, whose recursion runs
    // in registers (the stored forward state stays as it is)
    VDer v;
    {
        const double *st = cur;
        const long long dI = g.pz, dJ = g.plane;
        const double *vx = st + VX * F, *vy = st + VY * F, *vz = st + VZ * F;
        const double b1 = a.b1, b2 = a.b2;
        v.d[0] = ddn(vx, c, dI, b1, b2) / a.rdx;
        v.d[1] = dup(vx, c, dJ, b1, b2) / a.rdy;
        v.d[2] = dup(vx, c, 1, b1, b2) / a.rdz;
        v.d[3] = dup(vy, c, dI, b1, b2) / a.rdx;
        v.d[4] = ddn(vy, c, dJ, b1, b2) / a.rdy;
        v.d[5] = dup(vy, c, 1, b1, b2) / a.rdz;
        v.d[6] = dup(vz, c, dI, b1, b2) / a.rdx;
        v.d[7] = dup(vz, c, dJ, b1, b2) / a.rdy;
        v.d[8] = ddn(vz, c, 1, b1, b2) / a.rdz;
        for (int q = 0; q < 9; ++q) v.e[q] = v.d[q];
        const double *P = prev_ps + poff;
        if (hx) {
            const long long o = sxi(g, j, hx, k), s = a.sl.sx;
            double t0 = P[o], t1 = P[o + s], t2 = P[o + 2 * s];
            v.e[0] = cpml_fwd(v.d[0], t0, cp64(cg, K_X, hx), cp64(cg, A_X, hx), cp64(cg, B_X, hx));
            v.e[3] = cpml_fwd(v.d[3], t1, cp64(cg, KH_X, hx), cp64(cg, AH_X, hx), cp64(cg, BH_X, hx));
            v.e[6] = cpml_fwd(v.d[6], t2, cp64(cg, KH_X, hx), cp64(cg, AH_X, hx), cp64(cg, BH_X, hx));
        }
        if (hy) {
            const long long o = 3 * a.sl.sx + syi(g, hy, i, k), s = a.sl.sy;
            double t0 = P[o], t1 = P[o + s], t2 = P[o + 2 * s];
            v.e[1] = cpml_fwd(v.d[1], t0, cp64(cg, KH_Y, hy), cp64(cg, AH_Y, hy), cp64(cg, BH_Y, hy));
            v.e[4] = cpml_fwd(v.d[4], t1, cp64(cg, K_Y, hy), cp64(cg, A_Y, hy), cp64(cg, B_Y, hy));
            v.e[7] = cpml_fwd(v.d[7], t2, cp64(cg, KH_Y, hy), cp64(cg, AH_Y, hy), cp64(cg, BH_Y, hy));
        }
        if (hz) {
            const bool zfront = k <= g.fw;
            const long long o = 3 * a.sl.sx + 3 * a.sl.sy + szi(g, j, i, hz), s = a.sl.sz;
            const double kh = zfront ? cp64(cg, KH_Y, hz) : cp64(cg, KH_Z, hz);
            const double kf = zfront ? cp64(cg, K_Y, hz) : cp64(cg, K_Z, hz);
            double t0 = P[o], t1 = P[o + s], t2 = P[o + 2 * s];
            v.e[2] = cpml_fwd(v.d[2], t0, kh, cp64(cg, AH_Z, hz), cp64(cg, BH_Z, hz));
            v.e[5] = cpml_fwd(v.d[5], t1, kh, cp64(cg, AH_Z, hz), cp64(cg, BH_Z, hz));
            v.e[8] = cpml_fwd(v.d[8], t2, kf, cp64(cg, A_Z, hz), cp64(cg, B_Z, hz));
        }
    }
    const Mod64 m = mod64(a, c);
    const int L = a.nmech;
    const double DT = a.dt, h = 0.5 * DT, Lf = L;
    const double *e = v.e;
    const double gg = m.pim * (1.0 + Lf * m.taup), f = 2.0 * m.um * (1.0 + Lf * m.taus);
    const double fxy = DT * m.uipjp * (1.0 + Lf * m.tsipjp), fyz = DT * m.ujpkp * (1.0 + Lf * m.tsjpkp),
                 fxz = DT * m.uipkp * (1.0 + Lf * m.tsipkp);
    const double exy = e[1] + e[3], eyz = e[5] + e[7], exz = e[2] + e[6];
    const double div = e[0] + e[4] + e[8], syz_ = e[4] + e[8], sxz_ = e[0] + e[8], sxy_ = e[0] + e[4];
    static constexpr int sslot[6] = {SXX, SYY, SZZ, SXY, SYZ, SXZ};
    double Ls[6], Lr[MAXMECH][6];
    for (int q = 0; q < 6; ++q) Ls[q] = lam[sslot[q] * F + c];
    for (int l = 0; l < L; ++l)
        for (int q = 0; q < 6; ++q) Lr[l][q] = lam[(NEL + 6 * l + q) * F + c];
    double g_gg = 0.0, g_f = 0.0, g_dd = 0.0, g_ee = 0.0;
    double Wd[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // adjoints of the plain derivatives (surface terms)
    const bool surf = g.free_surf && j == 1;
    if (surf) {
        const double X = v.d[0] + v.d[8], Y = v.d[4], gf = gg - f;
        const double lhs = Ls[0] + Ls[2];
        const double dd = 2.0 * m.um * m.taus, ee = m.pim * m.taup, B = dd - ee;
        g_gg += lhs * (-DT * X * (2.0 * gf * gg - gf * gf) / (gg * gg) - DT * Y);
        g_f += lhs * (DT * 2.0 * gf * X / gg + DT * Y);
        Wd[0] += lhs * (-(DT * gf * gf / gg));
        Wd[8] += lhs * (-(DT * gf * gf / gg));
        Wd[4] += lhs * (-(DT * gf));
        for (int l = 0; l < L; ++l) {
            const double lhh = h * lhs + Lr[l][0] + Lr[l][2];
            const double dhdB = a.msb[l] * ((f / gg - 1.0) * X - Y);
            g_dd += lhh * dhdB;
            g_ee -= lhh * dhdB;
            g_f += lhh * a.msb[l] * B * X / gg;
            g_gg += lhh * (-a.msb[l] * B * f * X / (gg * gg));
            Wd[0] += lhh * a.msb[l] * B * (f / gg - 1.0);
            Wd[8] += lhh * a.msb[l] * B * (f / gg - 1.0);
            Wd[4] += lhh * (-a.msb[l] * B);
            Lr[l][1] = 0.0;  // r_yy = 0 after the update
        }
        Ls[1] = 0.0;  // syy = 0 after the update
    }
    // the update: sigma' = sigma + M e + h (sum r + sum r'), r' = bb (cc r - D(e))
    double W[9];
    W[0] = DT * (gg * Ls[0] + (gg - f) * (Ls[1] + Ls[2]));
    W[4] = DT * (gg * Ls[1] + (gg - f) * (Ls[0] + Ls[2]));
    W[8] = DT * (gg * Ls[2] + (gg - f) * (Ls[0] + Ls[1]));
    W[1] = W[3] = fxy * Ls[3];
    W[5] = W[7] = fyz * Ls[4];
    W[2] = W[6] = fxz * Ls[5];
    g_gg += DT * div * (Ls[0] + Ls[1] + Ls[2]);
    g_f += -DT * (syz_ * Ls[0] + sxz_ * Ls[1] + sxy_ * Ls[2]);
    double g_fxy = exy * Ls[3], g_fyz = eyz * Ls[4], g_fxz = exz * Ls[5];
    double g_pi_r = 0.0, g_u_r = 0.0, g_tp_r = 0.0, g_ts_r = 0.0;
    double g_uxy_r = 0.0, g_uyz_r = 0.0, g_uxz_r = 0.0, g_txy_r = 0.0, g_tyz_r = 0.0, g_txz_r = 0.0;
    for (int l = 0; l < L; ++l) {
        double Lrn[6];
        for (int q = 0; q < 6; ++q) Lrn[q] = Lr[l][q] + h * Ls[q];  // adjoint of r' (before the surface terms)
        const double eta = a.eta[l], bb = a.bb[l];
        const double El = m.pim * eta * m.taup, Dl = 2.0 * m.um * eta * m.taus;
        const double sn = Lrn[0] + Lrn[1] + Lrn[2];
        W[0] += -bb * (El * sn - Dl * (Lrn[1] + Lrn[2]));
        W[4] += -bb * (El * sn - Dl * (Lrn[0] + Lrn[2]));
        W[8] += -bb * (El * sn - Dl * (Lrn[0] + Lrn[1]));
        const double dxy = m.uipjp * eta * m.tsipjp, dyz = m.ujpkp * eta * m.tsjpkp, dxz = m.uipkp * eta * m.tsipkp;
        W[1] += -bb * dxy * Lrn[3]; W[3] += -bb * dxy * Lrn[3];
        W[5] += -bb * dyz * Lrn[4]; W[7] += -bb * dyz * Lrn[4];
        W[2] += -bb * dxz * Lrn[5]; W[6] += -bb * dxz * Lrn[5];
        const double gE = -bb * div * sn, gD = bb * (syz_ * Lrn[0] + sxz_ * Lrn[1] + sxy_ * Lrn[2]);
        g_pi_r += gE * eta * m.taup; g_tp_r += gE * m.pim * eta;
        g_u_r += gD * 2.0 * eta * m.taus; g_ts_r += gD * 2.0 * m.um * eta;
        const double gxy = -bb * exy * Lrn[3], gyz = -bb * eyz * Lrn[4], gxz = -bb * exz * Lrn[5];
        g_uxy_r += gxy * eta * m.tsipjp; g_txy_r += gxy * m.uipjp * eta;
        g_uyz_r += gyz * eta * m.tsjpkp; g_tyz_r += gyz * m.ujpkp * eta;
        g_uxz_r += gxz * eta * m.tsipkp; g_txz_r += gxz * m.uipkp * eta;
        // the memory variable one step back: r' reads cc r, sigma' reads h r
        for (int q = 0; q < 6; ++q) lam[(NEL + 6 * l + q) * F + c] = bb * a.cc[l] * Lrn[q] + h * Ls[q];
    }
    for (int q = 0; q < 6; ++q) lam[sslot[q] * F + c] = Ls[q];
    // the coefficients' gradients, onto the cell's model values
    gr.q[M64_PI][mm] += g_gg * (1.0 + Lf * m.taup) + g_pi_r + g_ee * m.taup;
    gr.q[M64_U][mm] += g_f * 2.0 * (1.0 + Lf * m.taus) + g_u_r + g_dd * 2.0 * m.taus;
    gr.q[M64_UIPJP][mm] += g_fxy * DT * (1.0 + Lf * m.tsipjp) + g_uxy_r;
    gr.q[M64_UJPKP][mm] += g_fyz * DT * (1.0 + Lf * m.tsjpkp) + g_uyz_r;
    gr.q[M64_UIPKP][mm] += g_fxz * DT * (1.0 + Lf * m.tsipkp) + g_uxz_r;
    if (L) {
        gr.q[M64_TAUP][mm] += g_gg * Lf * m.pim + g_tp_r + g_ee * m.pim;
        gr.q[M64_TAUS][mm] += g_f * 2.0 * m.um * Lf + g_ts_r + g_dd * 2.0 * m.um;
        gr.q[M64_TSIPJP][mm] += g_fxy * DT * m.uipjp * Lf + g_txy_r;
        gr.q[M64_TSJPKP][mm] += g_fyz * DT * m.ujpkp * Lf + g_tyz_r;
        gr.q[M64_TSIPKP][mm] += g_fxz * DT * m.uipkp * Lf + g_txz_r;
    }
    // through the CPML recursions (the adjoint memory steps back one step)
    double Ld[9];
    for (int q = 0; q < 9; ++q) Ld[q] = W[q];
    double *P = lps + poff;
    if (hx) {
        const long long o = sxi(g, j, hx, k), s = a.sl.sx;
        Ld[0] = cpml_adj(W[0], P[o], cp64(cg, K_X, hx), cp64(cg, A_X, hx), cp64(cg, B_X, hx));
        Ld[3] = cpml_adj(W[3], P[o + s], cp64(cg, KH_X, hx), cp64(cg, AH_X, hx), cp64(cg, BH_X, hx));
        Ld[6] = cpml_adj(W[6], P[o + 2 * s], cp64(cg, KH_X, hx), cp64(cg, AH_X, hx), cp64(cg, BH_X, hx));
    }
    if (hy) {
        const long long o = 3 * a.sl.sx + syi(g, hy, i, k), s = a.sl.sy;
        Ld[1] = cpml_adj(W[1], P[o], cp64(cg, KH_Y, hy), cp64(cg, AH_Y, hy), cp64(cg, BH_Y, hy));
        Ld[4] = cpml_adj(W[4], P[o + s], cp64(cg, K_Y, hy), cp64(cg, A_Y, hy), cp64(cg, B_Y, hy));
        Ld[7] = cpml_adj(W[7], P[o + 2 * s], cp64(cg, KH_Y, hy), cp64(cg, AH_Y, hy), cp64(cg, BH_Y, hy));
    }
    if (hz) {
        const bool zfront = k <= g.fw;
        const long long o = 3 * a.sl.sx + 3 * a.sl.sy + szi(g, j, i, hz), s = a.sl.sz;
        const double kh = zfront ? cp64(cg, KH_Y, hz) : cp64(cg, KH_Z, hz);
        const double kf = zfront ? cp64(cg, K_Y, hz) : cp64(cg, K_Z, hz);
        Ld[2] = cpml_adj(W[2], P[o], kh, cp64(cg, AH_Z, hz), cp64(cg, BH_Z, hz));
        Ld[5] = cpml_adj(W[5], P[o + s], kh, cp64(cg, AH_Z, hz), cp64(cg, BH_Z, hz));
        Ld[8] = cpml_adj(W[8], P[o + 2 * s], kf, cp64(cg, A_Z, hz), cp64(cg, B_Z, hz));
    }
    for (int q = 0; q < 9; ++q) ld[q * F + c] = Ld[q] + Wd[q];
}

// velocity adjoint from the derivative adjoints: lambda_v += E^T ld
__global__ void k64_str_T_gather(Vjp64 a, double *lam, const double *ld) {
    const Geo &g = a.g;
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1, i = blockIdx.y + 1, j = blockIdx.z + 1;
    if (k > g.nz) return;
    const long long F = g.field, c = widx(g, j, i, k), dI = g.pz, dJ = g.plane;
    const double b1 = a.b1, b2 = a.b2;
    lam[VX * F + c] += tdn(ld + 0 * F, c, dI, b1, b2) / a.rdx + tup(ld + 1 * F, c, dJ, b1, b2) / a.rdy +
                       tup(ld + 2 * F, c, 1, b1, b2) / a.rdz;
    lam[VY * F + c] += tup(ld + 3 * F, c, dI, b1, b2) / a.rdx + tdn(ld + 4 * F, c, dJ, b1, b2) / a.rdy +
                       tup(ld + 5 * F, c, 1, b1, b2) / a.rdz;
    lam[VZ * F + c] += tup(ld + 6 * F, c, dI, b1, b2) / a.rdx + tup(ld + 7 * F, c, dJ, b1, b2) / a.rdy +
                       tdn(ld + 8 * F, c, 1, b1, b2) / a.rdz;
}

// A^T at one interior cell: adjoints of the nine scaled stress derivatives (ls),
// the stress-derivative PML memories (lps, one step back), and the gradients of
// the averaged densities from v^n - v^{n-1} = T / rho_avg.
__global__ void k64_vel_T(Vjp64 a, const double *lam, double *lps, double *ls, const double *cur, const double *prev,
                          Grad64 gr) {
    const Geo &g = a.g;
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1, i = blockIdx.y + 1, j = blockIdx.z + 1;
    if (k > g.nz) return;
    const long long F = g.field, c = widx(g, j, i, k);
    const long long m = ((long long)(j - 1) * g.nx + (i - 1)) * g.nz + (k - 1);
    const double *md = a.md;
    const double rip = md[M64_RIP * F + c], rjp = md[M64_RJP * F + c], rkp = md[M64_RKP * F + c];
    const double lx = lam[VX * F + c], ly = lam[VY * F + c], lz = lam[VZ * F + c];
    gr.q[M64_RIP][m] += -lx * (cur[VX * F + c] - prev[VX * F + c]) / rip;
    gr.q[M64_RJP][m] += -ly * (cur[VY * F + c] - prev[VY * F + c]) / rjp;
    gr.q[M64_RKP][m] += -lz * (cur[VZ * F + c] - prev[VZ * F + c]) / rkp;
    const double Ux = lx / rip, Uy = ly / rjp, Uz = lz / rkp;
    // order: sxx_x sxy_y sxz_z | syy_y sxy_x syz_z | szz_z sxz_x syz_y
    double Ls[9] = {Ux, Ux, Ux, Uy, Uy, Uy, Uz, Uz, Uz};
    const int hx = face_x(g, i), hy = face_y(g, j), hz = face_z(g, k);
    const float *cg = a.cpg;
    if (hx) {
        const long long o = sxi(g, j, hx, k), s = a.sl.sx;
        Ls[0] = cpml_adj(Ux, lps[o], cp64(cg, KH_X, hx), cp64(cg, AH_X, hx), cp64(cg, BH_X, hx));     // sxx_x
        Ls[4] = cpml_adj(Uy, lps[o + s], cp64(cg, K_X, hx), cp64(cg, A_X, hx), cp64(cg, B_X, hx));    // sxy_x
        Ls[7] = cpml_adj(Uz, lps[o + 2 * s], cp64(cg, K_X, hx), cp64(cg, A_X, hx), cp64(cg, B_X, hx));  // sxz_x
    }
    if (hy) {
        const long long o = 3 * a.sl.sx + syi(g, hy, i, k), s = a.sl.sy;
        Ls[1] = cpml_adj(Ux, lps[o], cp64(cg, K_Y, hy), cp64(cg, A_Y, hy), cp64(cg, B_Y, hy));       // sxy_y
        Ls[3] = cpml_adj(Uy, lps[o + s], cp64(cg, KH_Y, hy), cp64(cg, AH_Y, hy), cp64(cg, BH_Y, hy));  // syy_y
        Ls[8] = cpml_adj(Uz, lps[o + 2 * s], cp64(cg, K_Y, hy), cp64(cg, A_Y, hy), cp64(cg, B_Y, hy));  // syz_y
    }
    if (hz) {
        const long long o = 3 * a.sl.sx + 3 * a.sl.sy + szi(g, j, i, hz), s = a.sl.sz;
        Ls[2] = cpml_adj(Ux, lps[o], cp64(cg, K_Z, hz), cp64(cg, A_Z, hz), cp64(cg, B_Z, hz));         // sxz_z
        Ls[5] = cpml_adj(Uy, lps[o + s], cp64(cg, K_Z, hz), cp64(cg, A_Z, hz), cp64(cg, B_Z, hz));     // syz_z
        Ls[6] = cpml_adj(Uz, lps[o + 2 * s], cp64(cg, KH_Z, hz), cp64(cg, AH_Z, hz), cp64(cg, BH_Z, hz));  // szz_z
    }
    for (int q = 0; q < 9; ++q) ls[q * F + c] = Ls[q];
}

// stress adjoint from the scaled-derivative adjoints: lambda_sigma += T^T ls, at the
// interior cells and (free surface) the image rows j = 0, -1 the velocity update read
__global__ void k64_vel_T_gather(Vjp64 a, double *lam, const double *ls, int jlo) {
    const Geo &g = a.g;
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1, i = blockIdx.y + 1, j = blockIdx.z + jlo;
    if (k > g.nz) return;
    const long long F = g.field, c = widx(g, j, i, k), dI = g.pz, dJ = g.plane;
    const double b1 = a.b1, b2 = a.b2;
    const double *Lxx_x = ls, *Lxy_y = ls + F, *Lxz_z = ls + 2 * F, *Lyy_y = ls + 3 * F, *Lxy_x = ls + 4 * F;
    const double *Lyz_z = ls + 5 * F, *Lzz_z = ls + 6 * F, *Lxz_x = ls + 7 * F, *Lyz_y = ls + 8 * F;
    lam[SYY * F + c] += a.dy * tup(Lyy_y, c, dJ, b1, b2);
    lam[SXY * F + c] += a.dy * tdn(Lxy_y, c, dJ, b1, b2) + a.dx * tdn(Lxy_x, c, dI, b1, b2);
    lam[SYZ * F + c] += a.dz * tdn(Lyz_z, c, 1, b1, b2) + a.dy * tdn(Lyz_y, c, dJ, b1, b2);
    if (j >= 1) {  // the in-plane stresses have no image rows
        lam[SXX * F + c] += a.dx * tup(Lxx_x, c, dI, b1, b2);
        lam[SZZ * F + c] += a.dz * tup(Lzz_z, c, 1, b1, b2);
        lam[SXZ * F + c] += a.dz * tdn(Lxz_z, c, 1, b1, b2) + a.dx * tdn(Lxz_x, c, dI, b1, b2);
    }
}

}  // namespace ifosb
