// Device kernels of the B200 wavefield engine.
//
// Arithmetic contract: every floating-point expression keeps the operand order
// and the float/double promotions of the reference C code it restates, and the
// library is compiled with --fmad=false (no FMA contraction), IEEE division and
// square root, and denormals preserved. On the same inputs the results are
// therefore bit-identical to the reference built with gcc -O3 on x86-64.
//
// Layout in HBM (per shot, per field): the reference's halo ranges
// j=-2..NY+2, i=-1..NX+2, k=-1..NZ+2, with the z row padded to a pitch that is a
// multiple of 8 floats and k=1 placed at a 32-byte boundary. Fields of a shot are
// contiguous ([shot][field][y][x][z]); the model is one copy shared by all shots.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ifosb {

constexpr int MAXFW = 64;
constexpr int MAXMECH = 4;
constexpr int MAXNF = 16;
constexpr int BX = 32;  // threads along z (contiguous)
#ifndef IFOSB_BY
#define IFOSB_BY 8
#endif
constexpr int BY = IFOSB_BY;  // threads along x

// state field slots of a shot. The stresses with a y derivative in the velocity
// update (syy, sxy, syz) come first, then the in-plane ones (sxx, szz, sxz), then
// the memory variables, so each group is one contiguous TMA box.
enum { VX = 0, VY, VZ, SYY, SXY, SYZ, SXX, SZZ, SXZ, NEL };
// memory variables: slot NEL + 6*l + q, q: 0 rxx, 1 ryy, 2 rzz, 3 rxy, 4 ryz, 5 rxz
// model slots (one copy shared by every shot): the stress update's coefficients
// first (5, or 10 with non-uniform relaxation times), then the velocity update's.
enum { MD_PI = 0, MD_U, MD_UIPJP, MD_UJPKP, MD_UIPKP, MD_TAUS, MD_TAUP, MD_TSIPJP, MD_TSJPKP, MD_TSIPKP, MD_RIP, MD_RJP, MD_RKP, NMODEL };
// CPML coefficient rows
enum { K_X = 0, A_X, B_X, KH_X, AH_X, BH_X, K_Y, A_Y, B_Y, KH_Y, AH_Y, BH_Y, K_Z, A_Z, B_Z, KH_Z, AH_Z, BH_Z };

struct Geo {
    int nx, ny, nz, fw, free_surf, nmech;
    int pz;             // z row pitch in floats
    int px;             // rows per plane (NX+4)
    long long plane;    // px*pz
    long long field;    // (NY+5)*plane
    int cy, nyc;        // y planes per block, y chunks
    int ntk, nti;       // blocks along z and x
    int by;             // rows (x) per block: the tile height of the kernels in use
};

__host__ __device__ __forceinline__ long long widx(const Geo &g, int j, int i, int k) {
    return (long long)(j + 2) * g.plane + (long long)(i + 1) * g.pz + (k + 7);
}

// A source, injection or receiver located in one cell. Lists are grouped per
// (shot, block) and keep the order in which the reference visits them.
struct Pt {
    int j, i, k, kind;  // kind: 1 explosive, 2..5 body force, 6 adjoint injection, 7 receiver
    int row;            // value-table row (forces) or trace number (receivers)
    int pad0, pad1, pad2;
};
enum { PT_EXPLOSIVE = 1, PT_ADJOINT = 6, PT_RECEIVER = 7 };

__constant__ float c_cpml[18][2 * MAXFW];

__device__ __forceinline__ float CP(int row, int h) { return c_cpml[row][h - 1]; }

// a / b rounded to nearest (IEEE), the same bits as the division operator. The
// division's range check sends a zero dividend down its slow path (three times
// the cost of a normal quotient), and a wavefield is zero ahead of its front, so
// a zero dividend is handled here: q = 2^-24 / b has the sign of b, is finite for
// every finite non-zero b (2^-24 / 2^-149 = 2^125), +-0 for b = +-inf or |b| near
// FLT_MAX, inf for b = 0 and NaN for b = NaN; a * q is then exactly 0 / b
// (+-0 with the sign of a xor b, NaN for b = 0 or NaN).
__device__ __forceinline__ float div_rn(float a, float b) {
    const bool z = a == 0.f;
    const float q = __fdiv_rn(z ? 0x1p-24f : a, b);
    return z ? __fmul_rn(a, q) : q;
}
// z-face slab indices differ between the lanes of a warp; the constant cache would
// serialise them, L1 serves them in one pass
__device__ __forceinline__ float CPG(const float *cpg, int row, int h) { return __ldg(cpg + row * 2 * MAXFW + h - 1); }

// CPML frame membership (CPML_ini_elastic.c:26-71): 1-based slab index or 0.
__device__ __forceinline__ int face_x(const Geo &g, int i) {
    return i <= g.fw ? i : (i > g.nx - g.fw ? i - g.nx + 2 * g.fw : 0);
}
__device__ __forceinline__ int face_y(const Geo &g, int j) {
    return (!g.free_surf && j <= g.fw) ? j : (j > g.ny - g.fw ? j - g.ny + 2 * g.fw : 0);
}
__device__ __forceinline__ int face_z(const Geo &g, int k) {
    return k <= g.fw ? k : (k > g.nz - g.fw ? k - g.nz + 2 * g.fw : 0);
}

// PML memory slabs of a shot: 9 for the stress derivatives (velocity update),
// then 9 for the velocity derivatives (stress update). x: [NY][2FW][NZ],
// y: [2FW][NX][NZ], z: [NY][NX][2FW] (the reference's shapes, ifos3d.c:421-440).
struct Slabs {
    long long sx, sy, sz;
};
__device__ __forceinline__ long long sxi(const Geo &g, int j, int h, int k) {
    return ((long long)(j - 1) * 2 * g.fw + (h - 1)) * g.nz + (k - 1);
}
__device__ __forceinline__ long long syi(const Geo &g, int h, int i, int k) {
    return ((long long)(h - 1) * g.nx + (i - 1)) * g.nz + (k - 1);
}
__device__ __forceinline__ long long szi(const Geo &g, int j, int i, int h) {
    return ((long long)(j - 1) * g.nx + (i - 1)) * 2 * g.fw + (h - 1);
}

struct VelArgs {
    Geo g;
    Slabs sl;
    float *st;            // state base (shot 0)
    long long st_shot;    // floats per shot
    const float *md;      // model base
    float *psi;           // PML memory base (shot 0)
    long long psi_shot;
    const int *pt_off;    // [nshots][nblocks+1] or null
    const Pt *pts;
    const float *val;     // forces: amp table [row][NT]; adjoint: residual [shot][3][ntr][ns]
    long long val_row, val_comp;
    float dxr, dyr, dzr;  // DT/DX, DT/DY, DT/DZ
    float b1, b2;
    double cf5x, cf5y, cf5z;  // type-5 force direction factors (update_v_ssg.c:498-503)
    const float *cpg;         // global copy of the CPML rows, for lane-divergent (z-face) reads
    int *err_step;        // [nshots] first step whose probe cell went NaN
    int probe_j, probe_i, probe_k;
};

struct StrArgs {
    Geo g;
    Slabs sl;
    float *st;
    long long st_shot;
    const float *md;
    float *psi;
    long long psi_shot;
    const int *pt_off;
    const Pt *pts;
    const float *amp;     // explosive amplitudes [row][NT]
    long long amp_row;
    float *sec;           // traces [shot][3][ntr][ns]
    long long sec_shot, sec_comp, sec_tr;
    float *dft;           // [shot][nf][6][field]
    long long dft_shot;
    int nf;
    const double *trig;   // [NT][nf][2]: cos, sin of 2 pi f t, times DT*ntast
    float dt, dthalbe, rdx, rdy, rdz;
    float b1, b2;
    float eta[MAXMECH], mb[MAXMECH], mc[MAXMECH], msb[MAXMECH];
    const float *cpg;     // global copy of the CPML rows, for lane-divergent (z-face) reads
    int seismo;           // SEISMO: 1 particle velocities; 2, 3, 4 add p / div, curl (sec2)
    float *sec2;          // [shot][3][ntr][ns]: p, div, curl
    float hrx, hry, hrz;  // 1.0/DX etc. in float (seismo_ssg.c:38-40)
    const float *smod;    // elastic free surface: pi, u of plane j=1 ([2][NX][NZ]) when they
                          // differ from the propagation model's, else null
};

// seismo (seismo_ssg.c:48-125), SEISMO 2-4: pressure from the cell's new
// stresses; divergence and curl from one-sided velocity differences at the cell.
// The curl's squares are formed in double as the reference's fabs() promotes them.
__device__ __forceinline__ void seismo_pdc(float vx, float vx_im, float vx_jp, float vx_kp, float vy, float vy_jm,
                                           float vy_ip, float vy_kp, float vz, float vz_km, float vz_ip, float vz_jp,
                                           float sxx, float syy, float szz, float pi, float u, float hx, float hy,
                                           float hz, float &p, float &dv, float &cu) {
    p = -sxx - syy - szz;
    const float vxy = (vx_jp - vx) * hy, vxz = (vx_kp - vx) * hz;
    const float vyx = (vy_ip - vy) * hx, vyz = (vy_kp - vy) * hz;
    const float vzx = (vz_ip - vz) * hx, vzy = (vz_jp - vz) * hy;
    const double t1 = (double)(vyz - vzy) * fabs((double)(vyz - vzy));
    const double t2 = (double)(vzx - vxz) * fabs((double)(vzx - vxz));
    const double t3 = (double)(vxy - vyx) * fabs((double)(vxy - vyx));
    const float amp = (float)((double)u * (t1 + t2 + t3));
    cu = (float)((amp < 0.0 ? -1 : 1) * sqrt(fabs((double)amp)));
    const float vxx = (vx - vx_im) * hx, vyy = (vy - vy_jm) * hy, vzz = (vz - vz_km) * hz;
    dv = (float)((double)(vxx + vyy + vzz) * sqrt((double)pi));
}

__device__ __forceinline__ void block_points(const int *pt_off, const Geo &g, int s, int yc, int &p0, int &p1) {
    p0 = p1 = 0;
    if (pt_off) {
        const int nblk = g.ntk * g.nti * g.nyc;
        const int blk = (yc * g.nti + blockIdx.y) * g.ntk + blockIdx.x;
        const int *o = pt_off + (long long)s * (nblk + 1);
        p0 = o[blk];
        p1 = o[blk + 1];
    }
}

// ---------------------------------------------------------------------------
// Velocity update: update_v_ssg.c:102-127, update_v_ssg_CPML.c, and the point
// forces of update_v_ssg.c:474-522 / update_v_ssg_CPML.c:384-393.
template <bool BACK>
__device__ __forceinline__ void vel_points(const VelArgs &a, float *st, int p0, int p1, int j, int i, int k, int nt,
                                           long long c) {
    const long long F = a.g.field;
    for (int q = p0; q < p1; ++q) {
        const Pt pt = a.pts[q];
        if (pt.j != j || pt.i != i || pt.k != k) continue;
        if (BACK) {
            const float *v = a.val + (long long)pt.row * a.val_row + (nt - 1);
            st[VX * F + c] += v[0];
            st[VZ * F + c] += v[2 * a.val_comp];
            st[VY * F + c] += v[a.val_comp];
        } else {
            const float amp = a.val[(long long)pt.row * a.val_row + (nt - 1)];
            switch (pt.kind) {
            case 2: st[VX * F + c] += amp * a.md[MD_RIP * F + c]; break;
            case 3: st[VZ * F + c] += amp * a.md[MD_RJP * F + c]; break;  // rjp for vz as in the reference
            case 4: st[VY * F + c] += amp * a.md[MD_RKP * F + c]; break;  // rkp for vy as in the reference
            case 5:
                st[VX * F + c] = (float)((double)st[VX * F + c] + a.cf5x * (double)amp);
                st[VY * F + c] = (float)((double)st[VY * F + c] + a.cf5y * (double)amp);
                st[VZ * F + c] = (float)((double)st[VZ * F + c] + a.cf5z * (double)amp);
                break;
            default: break;
            }
        }
    }
}

template <bool BACK>
__global__ void __launch_bounds__(BX *BY) k_velocity(VelArgs a, int nt) {
    const Geo &g = a.g;
    const int k = blockIdx.x * BX + threadIdx.x + 1;
    const int i = blockIdx.y * blockDim.y + threadIdx.y + 1;  // blockDim.y == g.by
    const int yc = blockIdx.z % g.nyc, s = blockIdx.z / g.nyc;
    int p0, p1;
    block_points(a.pt_off, g, s, yc, p0, p1);
    if (k > g.nz || i > g.nx) return;
    const int j0 = yc * g.cy + 1;
    const int j1 = min(j0 + g.cy - 1, g.ny);
    float *st = a.st + (long long)s * a.st_shot;
    float *ps = a.psi + (long long)s * a.psi_shot;
    const long long F = g.field;
    const float *__restrict__ sxx = st + SXX * F;
    const float *__restrict__ syy = st + SYY * F;
    const float *__restrict__ szz = st + SZZ * F;
    const float *__restrict__ sxy = st + SXY * F;
    const float *__restrict__ syz = st + SYZ * F;
    const float *__restrict__ sxz = st + SXZ * F;
    const float b1 = a.b1, b2 = a.b2, dx = a.dxr, dy = a.dyr, dz = a.dzr;
    const long long dI = g.pz, dJ = g.plane;
    const int hx = face_x(g, i), hz = face_z(g, k);
    for (int j = j0; j <= j1; ++j) {
        const long long c = widx(g, j, i, k);
        float sxx_x = dx * (b1 * (__ldg(sxx + c + dI) - __ldg(sxx + c)) + b2 * (__ldg(sxx + c + 2 * dI) - __ldg(sxx + c - dI)));
        float sxy_y = dy * (b1 * (__ldg(sxy + c) - __ldg(sxy + c - dJ)) + b2 * (__ldg(sxy + c + dJ) - __ldg(sxy + c - 2 * dJ)));
        float sxz_z = dz * (b1 * (__ldg(sxz + c) - __ldg(sxz + c - 1)) + b2 * (__ldg(sxz + c + 1) - __ldg(sxz + c - 2)));
        float syy_y = dy * (b1 * (__ldg(syy + c + dJ) - __ldg(syy + c)) + b2 * (__ldg(syy + c + 2 * dJ) - __ldg(syy + c - dJ)));
        float sxy_x = dx * (b1 * (__ldg(sxy + c) - __ldg(sxy + c - dI)) + b2 * (__ldg(sxy + c + dI) - __ldg(sxy + c - 2 * dI)));
        float syz_z = dz * (b1 * (__ldg(syz + c) - __ldg(syz + c - 1)) + b2 * (__ldg(syz + c + 1) - __ldg(syz + c - 2)));
        float szz_z = dz * (b1 * (__ldg(szz + c + 1) - __ldg(szz + c)) + b2 * (__ldg(szz + c + 2) - __ldg(szz + c - 1)));
        float sxz_x = dx * (b1 * (__ldg(sxz + c) - __ldg(sxz + c - dI)) + b2 * (__ldg(sxz + c + dI) - __ldg(sxz + c - 2 * dI)));
        float syz_y = dy * (b1 * (__ldg(syz + c) - __ldg(syz + c - dJ)) + b2 * (__ldg(syz + c + dJ) - __ldg(syz + c - 2 * dJ)));
        const int hy = face_y(g, j);
        const bool frame = hx || hy || hz;
        if (hx) {
            float *p = ps + sxi(g, j, hx, k);
            const long long o = a.sl.sx;
            float v0 = CP(BH_X, hx) * p[0] + CP(AH_X, hx) * sxx_x; p[0] = v0; sxx_x = sxx_x / CP(KH_X, hx) + v0;
            float v1 = CP(B_X, hx) * p[o] + CP(A_X, hx) * sxy_x; p[o] = v1; sxy_x = sxy_x / CP(K_X, hx) + v1;
            float v2 = CP(B_X, hx) * p[2 * o] + CP(A_X, hx) * sxz_x; p[2 * o] = v2; sxz_x = sxz_x / CP(K_X, hx) + v2;
        }
        if (hy) {
            float *p = ps + 3 * a.sl.sx + syi(g, hy, i, k);
            const long long o = a.sl.sy;
            float v0 = CP(B_Y, hy) * p[0] + CP(A_Y, hy) * sxy_y; p[0] = v0; sxy_y = sxy_y / CP(K_Y, hy) + v0;
            float v1 = CP(BH_Y, hy) * p[o] + CP(AH_Y, hy) * syy_y; p[o] = v1; syy_y = syy_y / CP(KH_Y, hy) + v1;
            float v2 = CP(B_Y, hy) * p[2 * o] + CP(A_Y, hy) * syz_y; p[2 * o] = v2; syz_y = syz_y / CP(K_Y, hy) + v2;
        }
        if (hz) {
            float *p = ps + 3 * a.sl.sx + 3 * a.sl.sy + szi(g, j, i, hz);
            const long long o = a.sl.sz;
            float v0 = CP(B_Z, hz) * p[0] + CP(A_Z, hz) * sxz_z; p[0] = v0; sxz_z = sxz_z / CP(K_Z, hz) + v0;
            float v1 = CP(B_Z, hz) * p[o] + CP(A_Z, hz) * syz_z; p[o] = v1; syz_z = syz_z / CP(K_Z, hz) + v1;
            float v2 = CP(BH_Z, hz) * p[2 * o] + CP(AH_Z, hz) * szz_z; p[2 * o] = v2; szz_z = szz_z / CP(KH_Z, hz) + v2;
        }
        // CPML frame: update_v() applies its point forces before update_v_CPML() updates the frame
        if (frame && p1 > p0) vel_points<BACK>(a, st, p0, p1, j, i, k, nt, c);
        st[VX * F + c] += (sxx_x + sxy_y + sxz_z) / a.md[MD_RIP * F + c];
        st[VY * F + c] += (syy_y + sxy_x + syz_z) / a.md[MD_RJP * F + c];
        st[VZ * F + c] += (szz_z + sxz_x + syz_y) / a.md[MD_RKP * F + c];
        if (p1 > p0) {
            // interior: forces after the update (the adjoint injects twice);
            // frame: only the adjoint's second injection (update_v_ssg_CPML.c:384-393)
            const int passes = frame ? (BACK ? 1 : 0) : (BACK ? 2 : 1);
            for (int pass = 0; pass < passes; ++pass) vel_points<BACK>(a, st, p0, p1, j, i, k, nt, c);
        }
        if (j == a.probe_j && i == a.probe_i && k == a.probe_k) {
            if (isnan(st[VY * F + c])) atomicMin(a.err_step + s, nt);
        }
    }
}

// ---------------------------------------------------------------------------
// Stress update and the rest of the time step, per cell, in the reference's order:
//   1. update_s_elastic / update_s (L mechanisms) with the CPML psi recursions
//      (update_s_ssg_elastic.c:106-140, update_s_ssg.c:150-230,
//       update_s_ssg_CPML(_elastic).c)
//   2. psource (psource.c:38-52)
//   3. discfourier (disc_fourier.c:36-57)
//   4. surface_elastic / surface at j=1 (surface_ssg_elastic.c:69-111,
//      surface_ssg.c:117-160), mirror rows j=0,-1 written by the j=1..3 cells
//   5. seismo (seismo_ssg.c:43-50)
template <int L>
__global__ void __launch_bounds__(BX *BY) k_stress(StrArgs a, int nt, int do_dft, int sample) {
    const Geo &g = a.g;
    const int k = blockIdx.x * BX + threadIdx.x + 1;
    const int i = blockIdx.y * blockDim.y + threadIdx.y + 1;  // blockDim.y == g.by
    const int yc = blockIdx.z % g.nyc, s = blockIdx.z / g.nyc;
    int p0, p1;
    block_points(a.pt_off, g, s, yc, p0, p1);
    if (k > g.nz || i > g.nx) return;
    const int j0 = yc * g.cy + 1;
    const int j1 = min(j0 + g.cy - 1, g.ny);
    float *st = a.st + (long long)s * a.st_shot;
    float *ps = a.psi + (long long)s * a.psi_shot + 3 * (a.sl.sx + a.sl.sy + a.sl.sz);
    const long long F = g.field;
    const float *__restrict__ vx = st + VX * F;
    const float *__restrict__ vy = st + VY * F;
    const float *__restrict__ vz = st + VZ * F;
    const float b1 = a.b1, b2 = a.b2, DX = a.rdx, DY = a.rdy, DZ = a.rdz, DT = a.dt;
    const long long dI = g.pz, dJ = g.plane;
    const int hx = face_x(g, i), hz = face_z(g, k);
    const bool zfront = k <= g.fw;
    for (int j = j0; j <= j1; ++j) {
        const long long c = widx(g, j, i, k);
        const float vx0 = __ldg(vx + c), vy0 = __ldg(vy + c), vz0 = __ldg(vz + c);
        float vxx = (b1 * (vx0 - __ldg(vx + c - dI)) + b2 * (__ldg(vx + c + dI) - __ldg(vx + c - 2 * dI))) / DX;
        float vxy = (b1 * (__ldg(vx + c + dJ) - vx0) + b2 * (__ldg(vx + c + 2 * dJ) - __ldg(vx + c - dJ))) / DY;
        float vxz = (b1 * (__ldg(vx + c + 1) - vx0) + b2 * (__ldg(vx + c + 2) - __ldg(vx + c - 1))) / DZ;
        float vyx = (b1 * (__ldg(vy + c + dI) - vy0) + b2 * (__ldg(vy + c + 2 * dI) - __ldg(vy + c - dI))) / DX;
        float vyy = (b1 * (vy0 - __ldg(vy + c - dJ)) + b2 * (__ldg(vy + c + dJ) - __ldg(vy + c - 2 * dJ))) / DY;
        float vyz = (b1 * (__ldg(vy + c + 1) - vy0) + b2 * (__ldg(vy + c + 2) - __ldg(vy + c - 1))) / DZ;
        float vzx = (b1 * (__ldg(vz + c + dI) - vz0) + b2 * (__ldg(vz + c + 2 * dI) - __ldg(vz + c - dI))) / DX;
        float vzy = (b1 * (__ldg(vz + c + dJ) - vz0) + b2 * (__ldg(vz + c + 2 * dJ) - __ldg(vz + c - dJ))) / DY;
        float vzz = (b1 * (vz0 - __ldg(vz + c - 1)) + b2 * (__ldg(vz + c + 1) - __ldg(vz + c - 2))) / DZ;
        // the free surface works on the plain derivatives (surface_ssg_elastic.c:91-93)
        const float svxx = vxx, svyy = vyy, svzz = vzz;
        const int hy = face_y(g, j);
        if (hx) {
            float *p = ps + sxi(g, j, hx, k);
            const long long o = a.sl.sx;
            float v0 = CP(B_X, hx) * p[0] + CP(A_X, hx) * vxx; p[0] = v0; vxx = vxx / CP(K_X, hx) + v0;
            float v1 = CP(BH_X, hx) * p[o] + CP(AH_X, hx) * vyx; p[o] = v1; vyx = vyx / CP(KH_X, hx) + v1;
            float v2 = CP(BH_X, hx) * p[2 * o] + CP(AH_X, hx) * vzx; p[2 * o] = v2; vzx = vzx / CP(KH_X, hx) + v2;
        }
        if (hy) {
            float *p = ps + 3 * a.sl.sx + syi(g, hy, i, k);
            const long long o = a.sl.sy;
            float v0 = CP(BH_Y, hy) * p[0] + CP(AH_Y, hy) * vxy; p[0] = v0; vxy = vxy / CP(KH_Y, hy) + v0;
            float v1 = CP(B_Y, hy) * p[o] + CP(A_Y, hy) * vyy; p[o] = v1; vyy = vyy / CP(K_Y, hy) + v1;
            float v2 = CP(BH_Y, hy) * p[2 * o] + CP(AH_Y, hy) * vzy; p[2 * o] = v2; vzy = vzy / CP(KH_Y, hy) + v2;
        }
        if (hz) {
            // the reference divides by K_y on the front z face (update_s_ssg_CPML_elastic.c:104-108)
            float *p = ps + 3 * a.sl.sx + 3 * a.sl.sy + szi(g, j, i, hz);
            const long long o = a.sl.sz;
            const float kh = zfront ? CP(KH_Y, hz) : CP(KH_Z, hz);
            const float kf = zfront ? CP(K_Y, hz) : CP(K_Z, hz);
            float v0 = CP(BH_Z, hz) * p[0] + CP(AH_Z, hz) * vxz; p[0] = v0; vxz = vxz / kh + v0;
            float v1 = CP(BH_Z, hz) * p[o] + CP(AH_Z, hz) * vyz; p[o] = v1; vyz = vyz / kh + v1;
            float v2 = CP(B_Z, hz) * p[2 * o] + CP(A_Z, hz) * vzz; p[2 * o] = v2; vzz = vzz / kf + v2;
        }
        const float *md = a.md;
        const float uipjp = md[MD_UIPJP * F + c], ujpkp = md[MD_UJPKP * F + c], uipkp = md[MD_UIPKP * F + c];
        const float pim = md[MD_PI * F + c], um = md[MD_U * F + c];
        const float vxyyx = vxy + vyx, vyzzy = vyz + vzy, vxzzx = vxz + vzx;
        const float vxxyyzz = vxx + vyy + vzz, vyyzz = vyy + vzz, vxxzz = vxx + vzz, vxxyy = vxx + vyy;
        float *S = st + c;
        float sxx = S[SXX * F], syy = S[SYY * F], szz = S[SZZ * F], sxy = S[SXY * F], syz = S[SYZ * F], sxz = S[SXZ * F];
        // ---- 1. stress (and memory variables) -----------------------------------
        float rv[L > 0 ? L : 1][6];
        float taus = 0.f, taup = 0.f;
        if constexpr (L == 0) {
            const float fipjp = uipjp * DT, fjpkp = ujpkp * DT, fipkp = uipkp * DT;
            const float gg = pim, f = (float)(2.0 * (double)um);
            sxy += (fipjp * vxyyx);
            syz += (fjpkp * vyzzy);
            sxz += (fipkp * vxzzx);
            sxx += DT * ((gg * vxxyyzz) - (f * vyyzz));
            syy += DT * ((gg * vxxyyzz) - (f * vxxzz));
            szz += DT * ((gg * vxxyyzz) - (f * vxxyy));
        } else {
            const float tausipjp = md[MD_TSIPJP * F + c], tausjpkp = md[MD_TSJPKP * F + c], tausipkp = md[MD_TSIPKP * F + c];
            taus = md[MD_TAUS * F + c];
            taup = md[MD_TAUP * F + c];
            const float Lf = (float)L, dthalbe = a.dthalbe;
            const float *r = st + NEL * F + c;
            float sr[6];
#pragma unroll
            for (int l = 0; l < L; ++l)
#pragma unroll
                for (int q = 0; q < 6; ++q) rv[l][q] = r[(6 * l + q) * F];
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                sr[q] = rv[0][q];
#pragma unroll
                for (int l = 1; l < L; ++l) sr[q] += rv[l][q];
            }
            const float fipjp = (float)((double)(uipjp * DT) * (1.0 + (double)(Lf * tausipjp)));
            const float fjpkp = (float)((double)(ujpkp * DT) * (1.0 + (double)(Lf * tausjpkp)));
            const float fipkp = (float)((double)(uipkp * DT) * (1.0 + (double)(Lf * tausipkp)));
            const float gg = (float)((double)pim * (1.0 + (double)(Lf * taup)));
            const float f = (float)((2.0 * (double)um) * (1.0 + (double)(Lf * taus)));
            sxy += (fipjp * vxyyx) + (dthalbe * sr[3]);
            syz += (fjpkp * vyzzy) + (dthalbe * sr[4]);
            sxz += (fipkp * vxzzx) + (dthalbe * sr[5]);
            sxx += DT * ((gg * vxxyyzz) - (f * vyyzz)) + (dthalbe * sr[0]);
            syy += DT * ((gg * vxxyyzz) - (f * vxxzz)) + (dthalbe * sr[1]);
            szz += DT * ((gg * vxxyyzz) - (f * vxxyy)) + (dthalbe * sr[2]);
#pragma unroll
            for (int l = 0; l < L; ++l) {
                const float eta = a.eta[l], bb = a.mb[l], cc = a.mc[l];
                const float dipjp = uipjp * eta * tausipjp, djpkp = ujpkp * eta * tausjpkp, dipkp = uipkp * eta * tausipkp;
                const float d = (float)(((2.0 * (double)um) * (double)eta) * (double)taus);
                const float e = pim * eta * taup;
                rv[l][3] = bb * (rv[l][3] * cc - (dipjp * vxyyx));
                rv[l][4] = bb * (rv[l][4] * cc - (djpkp * vyzzy));
                rv[l][5] = bb * (rv[l][5] * cc - (dipkp * vxzzx));
                rv[l][0] = bb * (rv[l][0] * cc - (e * vxxyyzz) + (d * vyyzz));
                rv[l][1] = bb * (rv[l][1] * cc - (e * vxxyyzz) + (d * vxxzz));
                rv[l][2] = bb * (rv[l][2] * cc - (e * vxxyyzz) + (d * vxxyy));
            }
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                sr[q] = rv[0][q];
#pragma unroll
                for (int l = 1; l < L; ++l) sr[q] += rv[l][q];
            }
            sxy += (dthalbe * sr[3]);
            syz += (dthalbe * sr[4]);
            sxz += (dthalbe * sr[5]);
            sxx += (dthalbe * sr[0]);
            syy += (dthalbe * sr[1]);
            szz += (dthalbe * sr[2]);
        }
        // ---- 2. explosive sources ------------------------------------------------
        for (int q = p0; q < p1; ++q) {
            const Pt pt = a.pts[q];
            if (pt.kind == PT_EXPLOSIVE && pt.j == j && pt.i == i && pt.k == k) {
                const float amp = a.amp[(long long)pt.row * a.amp_row + (nt - 1)];
                sxx += amp; syy += amp; szz += amp;
            }
        }
        // ---- 3. on-the-fly DFT of the velocities ----------------------------------
        if (do_dft) {
            float *Fd = a.dft + (long long)s * a.dft_shot + c;
            const double *tr = a.trig + (long long)(nt - 1) * a.nf * 2;
            for (int l = 0; l < a.nf; ++l) {
                const double t1 = tr[2 * l], t2 = tr[2 * l + 1];
                float *Fl = Fd + (long long)l * 6 * F;
                Fl[0 * F] = (float)((double)Fl[0 * F] + (double)vx0 * t1);
                Fl[1 * F] = (float)((double)Fl[1 * F] + (double)vy0 * t1);
                Fl[2 * F] = (float)((double)Fl[2 * F] + (double)vz0 * t1);
                Fl[3 * F] = (float)((double)Fl[3 * F] + (double)vx0 * t2);
                Fl[4 * F] = (float)((double)Fl[4 * F] + (double)vy0 * t2);
                Fl[5 * F] = (float)((double)Fl[5 * F] + (double)vz0 * t2);
            }
        }
        // ---- 4. free surface ---------------------------------------------------
        if (g.free_surf && j == 1) {
            syy = 0.0f;
            if constexpr (L == 0) {
                float spi = pim, su = um;
                if (a.smod) {
                    const long long q = (long long)(i - 1) * g.nz + (k - 1);
                    spi = a.smod[q];
                    su = a.smod[(long long)g.nx * g.nz + q];
                }
                const float f = (float)((double)su * 2.0), gg = spi;
                const float h = -(DT * (gg - f) * (gg - f) * (svxx + svzz) / gg) - (DT * (gg - f) * svyy);
                sxx += h;
                szz += h;
            } else {
                const float Lf = (float)L, dthalbe = a.dthalbe;
#pragma unroll
                for (int l = 0; l < L; ++l) rv[l][1] = 0.0f;
                const float f = (float)(((double)um * 2.0) * (1.0 + (double)(Lf * taus)));
                const float gg = (float)((double)pim * (1.0 + (double)(Lf * taup)));
                const float h = -(DT * (gg - f) * (gg - f) * (svxx + svzz) / gg) - (DT * (gg - f) * svyy);
                float srx = rv[0][0], srz = rv[0][2];
#pragma unroll
                for (int l = 1; l < L; ++l) { srx += rv[l][0]; srz += rv[l][2]; }
                sxx += h - (dthalbe * srx);
                szz += h - (dthalbe * srz);
                const float d = (float)((2.0 * (double)um) * (double)taus);
                const float e = pim * taup;
#pragma unroll
                for (int l = 0; l < L; ++l) {
                    const float hh = (float)((double)a.msb[l] *
                                             ((((double)(d - e) * ((double)(f / gg) - 1.0)) * (double)(svxx + svzz)) -
                                              (double)((d - e) * svyy)));
                    rv[l][0] += hh;
                    rv[l][2] += hh;
                }
                srx = rv[0][0]; srz = rv[0][2];
#pragma unroll
                for (int l = 1; l < L; ++l) { srx += rv[l][0]; srz += rv[l][2]; }
                sxx += (dthalbe * srx);
                szz += (dthalbe * srz);
            }
        }
        S[SXX * F] = sxx; S[SYY * F] = syy; S[SZZ * F] = szz;
        S[SXY * F] = sxy; S[SYZ * F] = syz; S[SXZ * F] = sxz;
        if constexpr (L > 0) {
            float *r = st + NEL * F + c;
#pragma unroll
            for (int l = 0; l < L; ++l)
#pragma unroll
                for (int q = 0; q < 6; ++q) r[(6 * l + q) * F] = rv[l][q];
        }
        if (g.free_surf && j <= 3) {
            // image rows above the surface (surface_ssg_elastic.c:80-84)
            if (j == 1) { S[SXY * F - dJ] = -sxy; S[SYZ * F - dJ] = -syz; }
            if (j == 2) { S[SYY * F - 2 * dJ] = -syy; S[SXY * F - 3 * dJ] = -sxy; S[SYZ * F - 3 * dJ] = -syz; }
            if (j == 3) { S[SYY * F - 4 * dJ] = -syy; }
        }
        // ---- 5. receivers --------------------------------------------------------
        if (sample >= 0) {
            for (int q = p0; q < p1; ++q) {
                const Pt pt = a.pts[q];
                if (pt.kind == PT_RECEIVER && pt.j == j && pt.i == i && pt.k == k) {
                    float *o = a.sec + (long long)s * a.sec_shot + (long long)pt.row * a.sec_tr + sample;
                    o[0] = vx0;
                    o[a.sec_comp] = vy0;
                    o[2 * a.sec_comp] = vz0;
                    if (a.seismo >= 2) {
                        float pr, dv, cu;
                        seismo_pdc(vx0, __ldg(vx + c - dI), __ldg(vx + c + dJ), __ldg(vx + c + 1), vy0, __ldg(vy + c - dJ),
                                   __ldg(vy + c + dI), __ldg(vy + c + 1), vz0, __ldg(vz + c - 1), __ldg(vz + c + dI),
                                   __ldg(vz + c + dJ), sxx, syy, szz, a.md[MD_PI * F + c], a.md[MD_U * F + c], a.hrx,
                                   a.hry, a.hrz, pr, dv, cu);
                        float *o2 = a.sec2 + (long long)s * a.sec_shot + (long long)pt.row * a.sec_tr + sample;
                        o2[0] = pr;
                        o2[a.sec_comp] = dv;
                        o2[2 * a.sec_comp] = cu;
                    }
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// gradient_F (gradient_F.c:62-139): for every shot of the batch (in order) and
// every frequency, the 4th-order derivatives of the forward and backward DFT
// fields are multiplied into the vp, vs, rho gradients. grad is compact
// [3][NY][NX][NZ]; grad64 accumulates the same contributions in FP64.
struct GradArgs {
    Geo g;
    const float *dftf, *dftb;  // [shot][nf][6][field]
    long long dft_shot;
    int nshots, nf;
    const float *md;           // model: rho is taken from the ghosted rho slot
    const float *rho;          // rho in field layout
    float fdummy[MAXNF];       // 1/(4 pi^2 f^2) in float as gradient_F.c:70-72
    float b1, b2, rdx, rdy, rdz;
    float ihx, ihy, ihz;       // 1/DX, 1/DY, 1/DZ (exact for power-of-two spacings)
    float *grad;
    double *grad64;
    // viscoelastic only: gradients with respect to taup and taus ([2][NY][NX][NZ],
    // FP64), with Phi(omega_l) = sum_m s tau_m / (1 + s tau_m), s = -i omega_l,
    // tau_m = DT / eta_m (the memory-variable relaxation of update_s_ssg.c:108-122)
    double *gradq;
    double rphi[MAXNF], iphi[MAXNF];
};

// x / h with the division operator's bits: for a power-of-two spacing the exact
// reciprocal (x * (1/h) == x / h for h = 2^k), else div_rn (no slow path for the
// zero dividends of a field the wave has not reached)
template <bool P2>
__device__ __forceinline__ float dvh(float x, float h, float ih) {
    return P2 ? __fmul_rn(x, ih) : div_rn(x, h);
}

// d: a float[9] or a column of shared memory (SCol); DX.. the spacings, IX.. their
// reciprocals (used with P2)
template <bool P2, class D>
__device__ __forceinline__ void dft_derivs(const float *X, const float *Y, const float *Z, long long c, long long dI,
                                           long long dJ, float b1, float b2, float DX, float DY, float DZ, float IX,
                                           float IY, float IZ, D d) {
    d[0] = dvh<P2>(b1 * (X[c] - X[c - dI]) + b2 * (X[c + dI] - X[c - 2 * dI]), DX, IX);
    d[1] = dvh<P2>(b1 * (X[c + dJ] - X[c]) + b2 * (X[c + 2 * dJ] - X[c - dJ]), DY, IY);
    d[2] = dvh<P2>(b1 * (X[c + 1] - X[c]) + b2 * (X[c + 2] - X[c - 1]), DZ, IZ);
    d[3] = dvh<P2>(b1 * (Y[c + dI] - Y[c]) + b2 * (Y[c + 2 * dI] - Y[c - dI]), DX, IX);
    d[4] = dvh<P2>(b1 * (Y[c] - Y[c - dJ]) + b2 * (Y[c + dJ] - Y[c - 2 * dJ]), DY, IY);
    d[5] = dvh<P2>(b1 * (Y[c + 1] - Y[c]) + b2 * (Y[c + 2] - Y[c - 1]), DZ, IZ);
    d[6] = dvh<P2>(b1 * (Z[c + dI] - Z[c]) + b2 * (Z[c + 2 * dI] - Z[c - dI]), DX, IX);
    d[7] = dvh<P2>(b1 * (Z[c + dJ] - Z[c]) + b2 * (Z[c + 2 * dJ] - Z[c - dJ]), DY, IY);
    d[8] = dvh<P2>(b1 * (Z[c] - Z[c - 1]) + b2 * (Z[c + 1] - Z[c - 2]), DZ, IZ);
}

// The same pointer, hidden from the optimiser (an empty asm that "changes" it).
__device__ __forceinline__ const float *opaque(const float *p) {
    asm volatile("" : "+l"(p));
    return p;
}

// Nine values of one thread in shared memory, stride one block: the kernel keeps
// its 36 derivatives there instead of in registers.
struct SCol {
    float *p;
    __device__ __forceinline__ float &operator[](int q) const { return p[q * (BX * BY)]; }
};

// Q: also the viscoelastic taup / taus gradient (a.gradq). Two instances, so the
// elastic one keeps the registers of gradient_F's terms alone. The kernel is
// latency-bound on its 156 loads per cell, shot and frequency. Left to itself the
// compiler hoisted all of them (and their 64-bit addresses) and used 243-254
// registers: one block per SM, or spills that went to DRAM at lower caps. With
// the derivatives in shared memory and each stencil set's pointers opaque, four
// blocks per SM fit in 62-64 registers: 5.7 ms instead of 18.4 ms for 4 shots x
// 4 frequencies at 128^3, L=3 (0.66 instead of 2.0 ms elastic, nf=2), same bits.
#ifndef IFOSB_GRAD_MINB
#define IFOSB_GRAD_MINB 4
#endif
template <bool Q, bool P2>
__global__ void __launch_bounds__(BX *BY, IFOSB_GRAD_MINB) k_gradient(GradArgs a) {
    __shared__ float sdv[4 * 9 * BX * BY];
    const Geo &g = a.g;
    const int k = blockIdx.x * BX + threadIdx.x + 1;
    const int i = blockIdx.y * BY + threadIdx.y + 1;
    const int tid = threadIdx.y * BX + threadIdx.x;
    const SCol fv{sdv + tid}, bv{sdv + 9 * BX * BY + tid}, fi{sdv + 18 * BX * BY + tid}, bi{sdv + 27 * BX * BY + tid};
    const int yc = blockIdx.z;
    if (k > g.nz || i > g.nx) return;
    const int j0 = yc * g.cy + 1;
    const int j1 = min(j0 + g.cy - 1, g.ny);
    const long long F = g.field, dI = g.pz, dJ = g.plane;
    const long long n = (long long)g.nx * g.ny * g.nz;
    for (int j = j0; j <= j1; ++j) {
        const long long c = widx(g, j, i, k);
        const long long m = ((long long)(j - 1) * g.nx + (i - 1)) * g.nz + (k - 1);
        float g1 = a.grad[m], g2 = a.grad[n + m], g3 = a.grad[2 * n + m];
        double h1 = a.grad64[m], h2 = a.grad64[n + m], h3 = a.grad64[2 * n + m];
        double qp = 0.0, qs = 0.0;
        if (Q) {
            qp = a.gradq[m];
            qs = a.gradq[n + m];
        }
        const float r = a.rho[c], pp = a.md[MD_PI * F + c], uu = a.md[MD_U * F + c];
        const double sqp = sqrt((double)(r * pp)), squ = sqrt((double)(r * uu));
        for (int s = 0; s < a.nshots; ++s) {
            for (int l = 0; l < a.nf; ++l) {
                const float *Fb = a.dftf + (long long)s * a.dft_shot + (long long)l * 6 * F;
                const float *Bb = a.dftb + (long long)s * a.dft_shot + (long long)l * 6 * F;
                // One stencil set at a time: each set's field pointers pass through an
                // empty asm, so the compiler can neither hoist the 36 addresses of all
                // sets out of the loops nor issue the next set's loads early; the
                // 144 loads then need few registers (no spills to local memory).
                const float *Fc = Fb + c, *Bc = Bb + c;
                const float *p0 = opaque(Fc), *p1 = opaque(Fc + F), *p2 = opaque(Fc + 2 * F);
                dft_derivs<P2>(p0, p1, p2, 0, dI, dJ, a.b1, a.b2, a.rdx, a.rdy, a.rdz, a.ihx, a.ihy, a.ihz, fv);
                p0 = opaque(Bc); p1 = opaque(Bc + F); p2 = opaque(Bc + 2 * F);
                dft_derivs<P2>(p0, p1, p2, 0, dI, dJ, a.b1, a.b2, a.rdx, a.rdy, a.rdz, a.ihx, a.ihy, a.ihz, bv);
                p0 = opaque(Fc + 3 * F); p1 = opaque(Fc + 4 * F); p2 = opaque(Fc + 5 * F);
                dft_derivs<P2>(p0, p1, p2, 0, dI, dJ, a.b1, a.b2, a.rdx, a.rdy, a.rdz, a.ihx, a.ihy, a.ihz, fi);
                p0 = opaque(Bc + 3 * F); p1 = opaque(Bc + 4 * F); p2 = opaque(Bc + 5 * F);
                dft_derivs<P2>(p0, p1, p2, 0, dI, dJ, a.b1, a.b2, a.rdx, a.rdy, a.rdz, a.ihx, a.ihy, a.ihz, bi);
                const float fdummy = a.fdummy[l];
                float gradlam = (fv[0] + fv[4] + fv[8]) * (bv[0] + bv[4] + bv[8]) + (fi[0] + fi[4] + fi[8]) * (bi[0] + bi[4] + bi[8]);
                gradlam = -gradlam * fdummy;
                float gradmu = 2.0f * fv[0] * bv[0] + 2.0f * fv[4] * bv[4] + 2.0f * fv[8] * bv[8] + 2.0f * fi[0] * bi[0] +
                               2.0f * fi[4] * bi[4] + 2.0f * fi[8] * bi[8] + (fv[1] + fv[3]) * (bv[1] + bv[3]) +
                               (fi[1] + fi[3]) * (bi[1] + bi[3]) + (fv[2] + fv[6]) * (bv[2] + bv[6]) +
                               (fi[2] + fi[6]) * (bi[2] + bi[6]) + (fv[5] + fv[7]) * (bv[5] + bv[7]) +
                               (fi[5] + fi[7]) * (bi[5] + bi[7]);
                gradmu = -gradmu * fdummy;
                const float gradrho = (Fb[c] * Bb[c] + Fb[F + c] * Bb[F + c] + Fb[2 * F + c] * Bb[2 * F + c]) +
                                      (Fb[3 * F + c] * Bb[3 * F + c] + Fb[4 * F + c] * Bb[4 * F + c] + Fb[5 * F + c] * Bb[5 * F + c]);
                const double c1 = sqp * 2.0 * (double)gradlam;
                const double c2 = -4.0 * squ * (double)gradlam + 2.0 * squ * (double)gradmu;
                const float c3 = gradrho + uu / r * gradmu + (pp - 2.0f * uu) / r * gradlam;
                g1 = (float)((double)g1 + c1);
                g2 = (float)((double)g2 + c2);
                g3 = g3 + c3;
                h1 += c1;
                h2 += c2;
                h3 += (double)c3;
                if (Q) {
                    // complex correlations C = F conj(B) of the lambda and mu terms with
                    // gradient_F's factor -fdummy: its gradlam / gradmu are their real
                    // parts. A modulus M(1 + tau Phi) perturbed in tau moves the misfit
                    // by Re[M Phi C] (lambda part for taup; mu - 2 lambda for taus).
                    const double fd = -(double)fdummy;
                    const double dfr = (double)fv[0] + fv[4] + fv[8], dfi = (double)fi[0] + fi[4] + fi[8];
                    const double dbr = (double)bv[0] + bv[4] + bv[8], dbi = (double)bi[0] + bi[4] + bi[8];
                    const double rl = fd * (dfr * dbr + dfi * dbi), il = fd * (dfi * dbr - dfr * dbi);
                    double rm = 0.0, im = 0.0;
                    for (int q = 0; q < 9; q += 4) {  // xx, yy, zz
                        rm += 2.0 * ((double)fv[q] * bv[q] + (double)fi[q] * bi[q]);
                        im += 2.0 * ((double)fi[q] * bv[q] - (double)fv[q] * bi[q]);
                    }
                    const int pr[3][2] = {{1, 3}, {2, 6}, {5, 7}};  // xy, xz, yz
                    for (int q = 0; q < 3; ++q) {
                        const double fr = (double)fv[pr[q][0]] + fv[pr[q][1]], fim = (double)fi[pr[q][0]] + fi[pr[q][1]];
                        const double br = (double)bv[pr[q][0]] + bv[pr[q][1]], bim = (double)bi[pr[q][0]] + bi[pr[q][1]];
                        rm += fr * br + fim * bim;
                        im += fim * br - fr * bim;
                    }
                    rm *= fd;
                    im *= fd;
                    const double ph = a.rphi[l], qh = a.iphi[l];
                    qp += (double)pp * (ph * rl - qh * il);
                    qs += (double)uu * (ph * (rm - 2.0 * rl) - qh * (im - 2.0 * il));
                }
            }
        }
        a.grad[m] = g1; a.grad[n + m] = g2; a.grad[2 * n + m] = g3;
        a.grad64[m] = h1; a.grad64[n + m] = h2; a.grad64[2 * n + m] = h3;
        if (Q) {
            a.gradq[m] = qp;
            a.gradq[n + m] = qs;
        }
    }
}

// ---------------------------------------------------------------------------
// Time-domain gradient kernels (the optional checkpoint/recompute mode). For a
// forward step n and the adjoint step m = P - n, P = TIME / DT (TIME = (NT-1) DT
// after ifos3d.c:177), the pair whose discfourier phases agree (t_f - t_b =
// n DT - (TIME - m DT) = 0), they add
//   rho: sum_c v_f,c v_b,c                      (gradient_F's gradrho term)
//   lambda: div U_f . div U_b                   (U = running time sum of v times DT)
//   mu: 2 sum_i e_ii,f e_ii,b + sum_i<j (e_ij+e_ji)_f (e_ij+e_ji)_b
// in FP64 over the interior cells, summed over the batch's shots.
struct TdArgs {
    Geo g;
    const float *st;       // adjoint state [shot][slot][field] (v at slots 0..2)
    long long st_shot;
    const float *ub;       // adjoint running sums [shot][3][field]
    const float *seg;      // forward v and running sums of one step [shot][6][field]
    long long seg_shot;
    int nshots;
    float b1, b2, rdx, rdy, rdz;
    float ihx, ihy, ihz;   // 1/DX, 1/DY, 1/DZ (exact for power-of-two spacings)
    double *k;             // [4][NY][NX][NZ]: rho, lambda, mu, dc
};

// One thread per interior cell: blocks of BX (z) x BY (x) cells, one plane each
// (grid ceil(NZ/BX) x ceil(NX/BY) x NY). (A variant that marched 1-16 planes per
// block with the x/z neighbours staged in shared memory and the y neighbours in
// registers ran 1.5-2.2 times slower at 128^3: fewer loads, but a barrier between
// each plane's loads and its arithmetic.)
template <bool P2>
__global__ void __launch_bounds__(BX *BY, 4) k_td_corr(TdArgs a) {
    const Geo &g = a.g;
    const int k = blockIdx.x * BX + threadIdx.x + 1, i = blockIdx.y * BY + threadIdx.y + 1, j = blockIdx.z + 1;
    if (k > g.nz || i > g.nx) return;
    const long long n = (long long)g.nx * g.ny * g.nz, F = g.field, dI = g.pz, dJ = g.plane;
    {
        const long long m = ((long long)(j - 1) * g.nx + (i - 1)) * g.nz + (k - 1);
        const long long c = widx(g, j, i, k);
        double kr = 0.0, kl = 0.0, km = 0.0;
        for (int s = 0; s < a.nshots; ++s) {
            const float *vb = a.st + (long long)s * a.st_shot, *ub = a.ub + (long long)s * 3 * F;
            const float *vf = a.seg + (long long)s * a.seg_shot, *uf = vf + 3 * F;
            kr += (double)vf[c] * vb[c] + (double)vf[F + c] * vb[F + c] + (double)vf[2 * F + c] * vb[2 * F + c];
            float fu[9], bu[9];
            const float *p0 = opaque(uf + c), *p1 = opaque(uf + F + c), *p2 = opaque(uf + 2 * F + c);
            dft_derivs<P2>(p0, p1, p2, 0, dI, dJ, a.b1, a.b2, a.rdx, a.rdy, a.rdz, a.ihx, a.ihy, a.ihz, fu);
            p0 = opaque(ub + c); p1 = opaque(ub + F + c); p2 = opaque(ub + 2 * F + c);
            dft_derivs<P2>(p0, p1, p2, 0, dI, dJ, a.b1, a.b2, a.rdx, a.rdy, a.rdz, a.ihx, a.ihy, a.ihz, bu);
            kl += ((double)fu[0] + fu[4] + fu[8]) * ((double)bu[0] + bu[4] + bu[8]);
            km += 2.0 * ((double)fu[0] * bu[0] + (double)fu[4] * bu[4] + (double)fu[8] * bu[8]) +
                  ((double)fu[1] + fu[3]) * ((double)bu[1] + bu[3]) + ((double)fu[2] + fu[6]) * ((double)bu[2] + bu[6]) +
                  ((double)fu[5] + fu[7]) * ((double)bu[5] + bu[7]);
        }
        a.k[m] += kr;
        a.k[n + m] += kl;
        a.k[2 * n + m] += km;
    }
}

// The zero-frequency product of the two runs: sum_c U_f,c(NT) U_b,c(NT).
__global__ void k_td_dc(TdArgs a, const float *uf_end) {
    const Geo &g = a.g;
    const long long n = (long long)g.nx * g.ny * g.nz, F = g.field;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(m % g.nz) + 1, i = (int)((m / g.nz) % g.nx) + 1, j = (int)(m / ((long long)g.nz * g.nx)) + 1;
        const long long c = widx(g, j, i, k);
        double d = 0.0;
        for (int s = 0; s < a.nshots; ++s) {
            const float *uf = uf_end + (long long)s * 3 * F, *ub = a.ub + (long long)s * 3 * F;
            d += (double)uf[c] * ub[c] + (double)uf[F + c] * ub[F + c] + (double)uf[2 * F + c] * ub[2 * F + c];
        }
        a.k[3 * n + m] += d;
    }
}

// U += v * DT over the three velocity fields (whole padded fields) of shot
// blockIdx.y, four floats at a time (a field is a multiple of 8 floats and every
// base is 16-byte aligned), each component as the scalar u + v * dt. With seg
// set, the step's v and new U also go to the shot's segment slot
// (seg + s * seg_shot: [v 3F][U 3F]), in the same pass.
__global__ void k_td_integrate(float *u, const float *st, long long st_shot, long long F, int nshots, float dt,
                               float *seg, long long seg_shot) {
    const int s = blockIdx.y;
    if (s >= nshots) return;
    const long long n4 = 3 * F / 4;
    float4 *U = reinterpret_cast<float4 *>(u + (long long)s * 3 * F);
    const float4 *S = reinterpret_cast<const float4 *>(st + (long long)s * st_shot);
    float4 *SV = seg ? reinterpret_cast<float4 *>(seg + (long long)s * seg_shot) : nullptr;
    float4 *SU = seg ? SV + n4 : nullptr;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n4; q += (long long)gridDim.x * blockDim.x) {
        float4 x = U[q];
        const float4 v = S[q];
        x.x += v.x * dt;
        x.y += v.y * dt;
        x.z += v.z * dt;
        x.w += v.w * dt;
        U[q] = x;
        if (SV) {
            SV[q] = v;
            SU[q] = x;
        }
    }
}

// ---------------------------------------------------------------------------
// hess_F (hess_F.c:67-155): the diagonal approximate Hessian from the forward DFT
// fields of every shot of the batch (in order) and the DFT fields of the
// receivers' Green's functions (wavefields of a y-force at each receiver), for
// every frequency. hess is compact [3][NY][NX][NZ] FP32, accumulated in the
// reference's order: shots, then receivers, then frequencies.
struct HessArgs {
    Geo g;
    const float *dftf;         // [shot][nf][6][field]
    long long dft_shot;
    const float *green;        // [receiver][nf][6][field] (same per-entry stride)
    int nshots, nrec, nf;
    const float *md;           // model: pi, u slots
    const float *rho;          // rho in field layout
    float fdummy[MAXNF];       // 1/(2 pi f) in float as hess_F.c:72-74
    float b1, b2, rdx, rdy, rdz;
    float ihx, ihy, ihz;       // 1/DX, 1/DY, 1/DZ (exact for power-of-two spacings)
    float *hess;
};

// With the derivatives in shared memory and opaque stencil pointers (as in
// k_gradient), four blocks per SM fit in 62 registers without spills: 35.5 ms
// for 2 shots x 25 receivers x 2 frequencies at 128^3, against 98 ms at one
// block (236 registers) and 62 ms at two (128, with spills); same bits.
#ifndef IFOSB_HESS_MINB
#define IFOSB_HESS_MINB 4
#endif
template <bool P2>
__global__ void __launch_bounds__(BX *BY, IFOSB_HESS_MINB) k_hessian(HessArgs a) {
    __shared__ float sdv[4 * 9 * BX * BY];
    const Geo &g = a.g;
    const int k = blockIdx.x * BX + threadIdx.x + 1;
    const int i = blockIdx.y * BY + threadIdx.y + 1;
    const int tid = threadIdx.y * BX + threadIdx.x;
    const SCol fv{sdv + tid}, bv{sdv + 9 * BX * BY + tid}, fi{sdv + 18 * BX * BY + tid}, bi{sdv + 27 * BX * BY + tid};
    const int yc = blockIdx.z;
    if (k > g.nz || i > g.nx) return;
    const int j0 = yc * g.cy + 1;
    const int j1 = min(j0 + g.cy - 1, g.ny);
    const long long F = g.field, dI = g.pz, dJ = g.plane;
    const long long n = (long long)g.nx * g.ny * g.nz;
    for (int j = j0; j <= j1; ++j) {
        const long long c = widx(g, j, i, k);
        const long long m = ((long long)(j - 1) * g.nx + (i - 1)) * g.nz + (k - 1);
        float h1 = a.hess[m], h2 = a.hess[n + m], h3 = a.hess[2 * n + m];
        const float r = a.rho[c], pp = a.md[MD_PI * F + c], uu = a.md[MD_U * F + c];
        for (int s = 0; s < a.nshots; ++s) {
            for (int q = 0; q < a.nrec; ++q) {
                for (int l = 0; l < a.nf; ++l) {
                    const float *Fb = a.dftf + (long long)s * a.dft_shot + (long long)l * 6 * F;
                    const float *Bb = a.green + (long long)q * a.dft_shot + (long long)l * 6 * F;
                    // one stencil set at a time, as in k_gradient
                    const float *Fc = Fb + c, *Bc = Bb + c;
                    const float *p0 = opaque(Fc), *p1 = opaque(Fc + F), *p2 = opaque(Fc + 2 * F);
                    dft_derivs<P2>(p0, p1, p2, 0, dI, dJ, a.b1, a.b2, a.rdx, a.rdy, a.rdz, a.ihx, a.ihy, a.ihz, fv);
                    p0 = opaque(Bc); p1 = opaque(Bc + F); p2 = opaque(Bc + 2 * F);
                    dft_derivs<P2>(p0, p1, p2, 0, dI, dJ, a.b1, a.b2, a.rdx, a.rdy, a.rdz, a.ihx, a.ihy, a.ihz, bv);
                    p0 = opaque(Fc + 3 * F); p1 = opaque(Fc + 4 * F); p2 = opaque(Fc + 5 * F);
                    dft_derivs<P2>(p0, p1, p2, 0, dI, dJ, a.b1, a.b2, a.rdx, a.rdy, a.rdz, a.ihx, a.ihy, a.ihz, fi);
                    p0 = opaque(Bc + 3 * F); p1 = opaque(Bc + 4 * F); p2 = opaque(Bc + 5 * F);
                    dft_derivs<P2>(p0, p1, p2, 0, dI, dJ, a.b1, a.b2, a.rdx, a.rdy, a.rdz, a.ihx, a.ihy, a.ihz, bi);
                    const float fd = a.fdummy[l];
                    const float fdiv = fv[0] + fv[4] + fv[8], fidiv = fi[0] + fi[4] + fi[8];
                    const float bdiv = bv[0] + bv[4] + bv[8], bidiv = bi[0] + bi[4] + bi[8];
                    float relam = fidiv * bdiv + fdiv * bidiv;
                    relam = fd * relam;
                    float imlam = fidiv * bidiv - fdiv * bdiv;
                    imlam = fd * imlam;
                    float remu = 2.0f * fi[0] * bv[0] + 2.0f * fi[4] * bv[4] + 2.0f * fi[8] * bv[8] +
                                 2.0f * fv[0] * bi[0] + 2.0f * fv[4] * bi[4] + 2.0f * fv[8] * bi[8] +
                                 (fi[1] + fi[3]) * (bv[1] + bv[3]) + (fv[1] + fv[3]) * (bi[1] + bi[3]) +
                                 (fi[2] + fi[6]) * (bv[2] + bv[6]) + (fv[2] + fv[6]) * (bi[2] + bi[6]) +
                                 (fi[5] + fi[7]) * (bv[5] + bv[7]) + (fv[5] + fv[7]) * (bi[5] + bi[7]);
                    remu = fd * remu;
                    float immu = 2.0f * fi[0] * bi[0] + 2.0f * fi[4] * bi[4] + 2.0f * fi[8] * bi[8] -
                                 2.0f * fv[0] * bv[0] - 2.0f * fv[4] * bv[4] - 2.0f * fv[8] * bv[8] +
                                 (fi[1] + fi[3]) * (bi[1] + bi[3]) - (fv[1] + fv[3]) * (bv[1] + bv[3]) +
                                 (fi[2] + fi[6]) * (bi[2] + bi[6]) - (fv[2] + fv[6]) * (bv[2] + bv[6]) +
                                 (fi[5] + fi[7]) * (bi[5] + bi[7]) - (fv[5] + fv[7]) * (bv[5] + bv[7]);
                    immu = fd * immu;
                    const float rerho = (Fb[c] * Bb[c] + Fb[F + c] * Bb[F + c] + Fb[2 * F + c] * Bb[2 * F + c]) -
                                        (Fb[3 * F + c] * Bb[3 * F + c] + Fb[4 * F + c] * Bb[4 * F + c] +
                                         Fb[5 * F + c] * Bb[5 * F + c]);
                    const float imrho = (Fb[c] * Bb[3 * F + c] + Fb[F + c] * Bb[4 * F + c] + Fb[2 * F + c] * Bb[5 * F + c]) +
                                        (Fb[3 * F + c] * Bb[c] + Fb[4 * F + c] * Bb[F + c] + Fb[5 * F + c] * Bb[2 * F + c]);
                    const float revs = -2.0f * relam + remu;
                    const float imvs = -2.0f * imlam + immu;
                    const float rerho1 = rerho + relam * (pp - 2.0f * uu) / r + remu * uu / r;
                    const float imrho1 = imrho + imlam * (pp - 2.0f * uu) / r + immu * uu / r;
                    h1 += (relam * relam + imlam * imlam) * r * pp * 4.0f;
                    h2 += (revs * revs + imvs * imvs) * 4.0f * r * uu;
                    h3 += rerho1 * rerho1 + imrho1 * imrho1;
                }
            }
        }
        a.hess[m] = h1; a.hess[n + m] = h2; a.hess[2 * n + m] = h3;
    }
}

// ---------------------------------------------------------------------------
// av_mat (av_mat.c:45-69) from the ghosted model [NY+2][NX+2][NZ+2] into the
// model slots, plus the per-cell pi, u, taus, taup.
struct AvArgs {
    Geo g;
    const float *rho, *pi, *u, *taus, *taup;  // ghosted
    float *md;
    float *rho_w;                              // rho in field layout (gradient)
};

// rho in field layout over the ghosted box (j, i, k = 0..N+1): the ghost layers
// matcopy left (periodic on one rank) next to the interior, so the velocity
// kernel can form av_mat's averages rip, rjp, rkp from rho and its +1 neighbours.
__global__ void k_rho_field(AvArgs a) {
    const Geo &g = a.g;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    const int j = blockIdx.z;
    if (k > g.nz + 1 || i > g.nx + 1 || j > g.ny + 1) return;
    const long long GX = g.nx + 2, GZ = g.nz + 2;
    a.rho_w[widx(g, j, i, k)] = a.rho[((long long)j * GX + i) * GZ + k];
}

__global__ void k_av_mat(AvArgs a) {
    const Geo &g = a.g;
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int i = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int j = blockIdx.z + 1;
    if (k > g.nz || i > g.nx || j > g.ny) return;
    const long long GX = g.nx + 2, GZ = g.nz + 2;
#define GM(A, jj, ii, kk) ((double)A[((long long)(jj) * GX + (ii)) * GZ + (kk)])
#define GF(A, jj, ii, kk) (A[((long long)(jj) * GX + (ii)) * GZ + (kk)])
    const long long F = g.field, c = widx(g, j, i, k);
    const float *u = a.u, *rho = a.rho;
    a.md[MD_UIPJP * F + c] = (float)(4.0 / ((1.0 / GM(u, j, i, k)) + (1.0 / GM(u, j, i + 1, k)) + (1.0 / GM(u, j + 1, i + 1, k)) +
                                          (1.0 / GM(u, j + 1, i, k))));
    a.md[MD_UJPKP * F + c] = (float)(4.0 / ((1.0 / GM(u, j, i, k)) + (1.0 / GM(u, j, i, k + 1)) + (1.0 / GM(u, j + 1, i, k + 1)) +
                                          (1.0 / GM(u, j + 1, i, k))));
    a.md[MD_UIPKP * F + c] = (float)(4.0 / ((1.0 / GM(u, j, i, k)) + (1.0 / GM(u, j, i, k + 1)) + (1.0 / GM(u, j, i + 1, k + 1)) +
                                          (1.0 / GM(u, j, i + 1, k))));
    if (g.nmech) {
        const float *t = a.taus;
        a.md[MD_TSIPJP * F + c] = (float)(0.25 * (double)(GF(t, j, i, k) + GF(t, j, i + 1, k) + GF(t, j + 1, i + 1, k) + GF(t, j + 1, i, k)));
        a.md[MD_TSJPKP * F + c] = (float)(0.25 * (double)(GF(t, j, i, k) + GF(t, j + 1, i, k) + GF(t, j + 1, i, k + 1) + GF(t, j, i, k + 1)));
        a.md[MD_TSIPKP * F + c] = (float)(0.25 * (double)(GF(t, j, i, k) + GF(t, j, i + 1, k) + GF(t, j, i + 1, k + 1) + GF(t, j, i, k + 1)));
        a.md[MD_TAUS * F + c] = GF(a.taus, j, i, k);
        a.md[MD_TAUP * F + c] = GF(a.taup, j, i, k);
    }
    a.md[MD_RJP * F + c] = (float)(0.5 * (double)(GF(rho, j, i, k) + GF(rho, j + 1, i, k)));
    a.md[MD_RKP * F + c] = (float)(0.5 * (double)(GF(rho, j, i, k) + GF(rho, j, i, k + 1)));
    a.md[MD_RIP * F + c] = (float)(0.5 * (double)(GF(rho, j, i, k) + GF(rho, j, i + 1, k)));
    a.md[MD_PI * F + c] = GF(a.pi, j, i, k);
    a.md[MD_U * F + c] = GF(a.u, j, i, k);
    a.rho_w[c] = GF(rho, j, i, k);
#undef GM
#undef GF
}

// ---------------------------------------------------------------------------
// residual (residual.c:35-60): one thread per (shot, component, trace) runs the
// time-integrated, time-reversed difference; the FP64 sum of squares of each
// trace goes to part[] and is reduced per shot in a fixed order.
__global__ void k_residual(const float *syn, const float *obs, float *diff, double *part, int nshots, int ntr, int ns,
                           float DT) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nshots * 3 * ntr) return;
    const float *sy = syn + (long long)t * ns;
    const float *ob = obs + (long long)t * ns;
    float *o = diff + (long long)t * ns;
    float vdiff = 0.0f;
    double acc = 0.0;
    for (int j = 1; j <= ns; ++j) {
        vdiff += sy[j - 1] - ob[j - 1];
        const float d = DT * vdiff;
        o[ns - j] = d;
        acc += (double)d * (double)d;
    }
    part[t] = acc;
}

// One warp per shot: strided lane sums then a shuffle tree — a fixed order, so
// the FP64 misfit is deterministic.
__global__ void k_misfit(const double *part, double *misfit, int per_shot) {
    const int s = blockIdx.x;
    const double *p = part + (long long)s * per_shot;
    double v = 0.0;
    for (int q = threadIdx.x; q < per_shot; q += 32) v += p[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) misfit[s] = v;
}

// The reference's own float L2 (residual.c:53): a sequential sum per shot.
__global__ void k_l2_ref(const float *diff, float *l2, int nshots, int ntr, int ns) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nshots) return;
    float L2 = 0.0f;
    const float *d = diff + (long long)s * 3 * ntr * ns;
    for (int c = 0; c < 3; ++c)
        for (int t = 0; t < ntr; ++t)
            for (int j = 1; j <= ns; ++j) {
                const float x = d[((long long)c * ntr + t) * ns + (ns - j)];
                L2 = (float)((double)L2 + fabs((double)(x * x)));
            }
    l2[s] = L2;
}

}  // namespace ifosb
