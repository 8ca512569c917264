// ifosb_tma_tile.cuh — the tile-height-dependent part of the TMA-staged
// time-step kernels: ring and stage layouts, the pipeline set-up, the velocity
// and stress kernels. ifosb_tma.cuh includes it once per tile height, inside a
// namespace that defines TX (rows of a tile = consumer warps of a CTA); it has
// no include guard on purpose and is not meant to be included elsewhere.

constexpr int RX = TX + 2 * HX;              // ring rows
constexpr int RPLANE = RX * RZ;              // floats per field per ring plane
constexpr int PT = TX * TZ;                  // floats per point-wise field tile
constexpr int RSLOT = a32(3 * RPLANE);       // ring slot stride (3 stencil fields)
constexpr int VS_RHO = a32(3 * RPLANE);      // velocity stage: rho of plane j with the x/z halo
constexpr int VS_PT = VS_RHO + a32(RPLANE);  // velocity stage: offset of the v box
constexpr int VS_RJ = VS_PT + a32(3 * PT);   // velocity stage: rho of plane j + 1 (the tile)
constexpr int VS_SP = VS_RJ + a32(PT);       // velocity stage stride
static_assert(RSLOT % 32 == 0 && VS_RHO % 32 == 0 && VS_PT % 32 == 0 && VS_RJ % 32 == 0 && VS_SP % 32 == 0,
              "TMA alignment");
constexpr int NTHR = 32 * (TX + 1);          // TX consumer warps + 1 producer warp

__host__ __device__ constexpr size_t vel_tma_smem() {
    return sizeof(float) * ((size_t)VRING * RSLOT + VNSTAGE * (size_t)VS_SP) + 8 * VNBAR;
}
// Stress stage: [sigma + memory variables: nsr][model: nm][DFT: ndf] boxes of PT
// floats per field, each box start rounded up to 32 floats.
__host__ __device__ inline int str_mod_off(int nsr) { return a32(nsr * PT); }
__host__ __device__ inline int str_dft_off(int nsr, int nm) { return a32(nsr * PT) + a32(nm * PT); }
__host__ __device__ inline int str_stage(int nsr, int nm, int ndf) { return str_dft_off(nsr, nm) + a32(ndf * PT); }
__host__ __device__ inline size_t str_tma_smem(int nsr, int nm, int ndf) {
    return sizeof(float) * ((size_t)RING * RSLOT + NSTAGE * (size_t)str_stage(nsr, nm, ndf)) + 8 * NBAR;
}

// CTA start: returns false (for every thread) if an earlier CTA reported a timeout.
// NR ring slots and NS stages: barriers [full ring | empty ring | full stage | empty stage].
template <int NR, int NS>
__device__ __forceinline__ bool pipeline_start(uint64_t *bar, const int *err) {
    __shared__ int s_go;
    if (threadIdx.x == 0 && threadIdx.y == TX) {
        s_go = *(volatile const int *)err == 0;
        if (s_go) {
            for (int q = 0; q < NR; ++q) {
                mbar_init(&bar[q], 1);             // full ring slot
                mbar_init(&bar[NR + q], TX);       // empty ring slot
            }
            for (int b = 0; b < NS; ++b) {
                mbar_init(&bar[2 * NR + b], 1);        // full stage
                mbar_init(&bar[2 * NR + NS + b], TX);  // empty stage
            }
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
    }
    __syncthreads();
    return s_go != 0;
}

// Consumer side of one plane: wait for the stencil planes and the stage.
__device__ __forceinline__ bool consumer_wait(uint64_t *bar, int it, int j, int j0, int rfirst, uint64_t lim) {
    bool ok = true;
    if (it == 0) {
        for (int P = j0 - 2; P <= j0 + 2; ++P) ok = ok && mbar_wait(&bar[(P - rfirst) % RING], ((P - rfirst) / RING) & 1, lim);
    } else {
        const int r = j + 2 - rfirst;
        ok = ok && mbar_wait(&bar[r % RING], (r / RING) & 1, lim);
    }
    ok = ok && mbar_wait(&bar[2 * RING + it % NSTAGE], (it / NSTAGE) & 1, lim);
    return ok;
}

// Producer exit on a failure path (a timed-out wait, or the test stop): wait,
// bounded, for the boxes already issued, so that no copy is still landing in
// shared memory when the CTA's warps have all returned. ring_hi / stage_hi are
// the last ring plane and stage iteration issued; a slot's latest phase is the
// only one not yet known to be complete.
template <int NR, int NS>
__device__ __forceinline__ void producer_drain(uint64_t *bar, int rfirst, int ring_hi, int stage_hi, uint64_t lim) {
    for (int P = max(rfirst, ring_hi - NR + 1); P <= ring_hi; ++P)
        if (!mbar_wait(&bar[(P - rfirst) % NR], ((P - rfirst) / NR) & 1, lim)) break;
    for (int q = max(0, stage_hi - NS + 1); q <= stage_hi; ++q)
        if (!mbar_wait(&bar[2 * NR + q % NS], (q / NS) & 1, lim)) break;
}

// Consumer hands back the ring plane j-2 and/or the stage of iteration `it`.
template <int NR = RING, int NS = NSTAGE>
__device__ __forceinline__ void consumer_release(uint64_t *bar, int it, bool ring_slot, bool stage) {
    __syncwarp();
    if (threadIdx.x == 0) {
        if (ring_slot) mbar_arrive(&bar[NR + it % NR]);
        if (stage) mbar_arrive(&bar[2 * NR + NS + it % NS]);
    }
}

// Consumer side of the velocity update: warp tx computes row i0+tx of the tile
// for planes j0..j1. XZ = the tile touches an x or z PML face (or the grid
// edge); without it hx = hz = 0 and every lane is active. Ring slots, the
// slot and parity of the next wait and the cell pointer advance by one plane
// per iteration (no per-plane division or 64-bit index arithmetic).
template <bool BACK, bool XZ>
__device__ __forceinline__ void vel_rows(const VelTma &T, int nt, const float *ring, const float *stg, uint64_t *bar,
                                         int j0, int j1, int s, int ycn, int k0, int i0) {
    const VelArgs &a = T.a;
    const Geo &g = a.g;
    constexpr int SP = VS_SP;
    const int tz = threadIdx.x, tx = threadIdx.y;
    const int k = k0 + tz, i = i0 + tx;
    const bool active = XZ ? (k <= g.nz && i <= g.nx) : true;
    int p0, p1;
    block_points(a.pt_off, g, s, ycn, p0, p1);
    float *st = a.st + (long long)s * a.st_shot;
    float *ps = a.psi + (long long)s * a.psi_shot;
    const long long F = g.field;
    const float b1 = a.b1, b2 = a.b2, dx = a.dxr, dy = a.dyr, dz = a.dzr;
    const int hx = XZ ? face_x(g, i) : 0, hz = XZ ? face_z(g, k) : 0;
    const int cz = tz + HZ, cx = tx + HX;
    const int probe_j = (a.probe_i == i && a.probe_k == k) ? a.probe_j : -1;
    // ring planes j-2..j+2 sit in slots 0..4 for j = j0; the next plane enters slot 5
    const float *Rb = ring + cx * RZ + cz;
    const float *Rm2 = Rb, *Rm1 = Rb + RSLOT, *R0 = Rb + 2 * RSLOT, *Rp1 = Rb + 3 * RSLOT, *Rp2 = Rb + 4 * RSLOT;
    int nslot = 5;            // slot of the plane that becomes j+2 next
    int wslot = 5, wpar = 0;  // slot and phase parity of plane j+2 at it >= 1
    float *V = st + widx(g, j0, i, k);
    PsiPre q{};
    if (active && (hx || hz || face_y(g, j0))) psi_load(q, ps, a.sl, g, j0, i, k, hx, hz);
    for (int it = 0, j = j0; j <= j1; ++it, ++j, V += g.plane) {
        bool ok = true;
        if (it == 0) {
            for (int r = 0; r < 5; ++r) ok = ok && mbar_wait(&bar[r], 0, T.w.limit_ns);
        } else {
            ok = ok && mbar_wait(&bar[wslot], wpar, T.w.limit_ns);
            if (++wslot == VRING) { wslot = 0; wpar ^= 1; }
        }
        ok = ok && mbar_wait(&bar[2 * VRING + it % VNSTAGE], (it / VNSTAGE) & 1, T.w.limit_ns);
        if (!ok) { if (tz == 0) atomicExch(T.tma_err, 1); return; }
        // everything this row needs from the stage, so the stage can go back at once
        float sxx_x = 0.f, sxz_z = 0.f, szz_z = 0.f, sxz_x = 0.f;
        float vxo = 0.f, vyo = 0.f, vzo = 0.f, rip = 1.f, rjp = 1.f, rkp = 1.f;
        if (active) {
            const float *stage = stg + (it % VNSTAGE) * SP;
            const float *Ip = stage + cx * RZ + cz;
            // stage in-plane fields: 0 sxx, 1 szz, 2 sxz
#define IP(f, x, z) Ip[(f) * RPLANE + (x) * RZ + (z)]
            sxx_x = dx * (b1 * (IP(0, 1, 0) - IP(0, 0, 0)) + b2 * (IP(0, 2, 0) - IP(0, -1, 0)));
            sxz_z = dz * (b1 * (IP(2, 0, 0) - IP(2, 0, -1)) + b2 * (IP(2, 0, 1) - IP(2, 0, -2)));
            szz_z = dz * (b1 * (IP(1, 0, 1) - IP(1, 0, 0)) + b2 * (IP(1, 0, 2) - IP(1, 0, -1)));
            sxz_x = dx * (b1 * (IP(2, 0, 0) - IP(2, -1, 0)) + b2 * (IP(2, 1, 0) - IP(2, -2, 0)));
#undef IP
            const float *pv = stage + VS_PT + tx * TZ + tz;
            vxo = pv[0]; vyo = pv[PT]; vzo = pv[2 * PT];
            // av_mat's averaged densities (av_mat.c:63-65) from rho and its +1
            // neighbours in x, y (the next plane's tile) and z, in its arithmetic
            const float *rh = stage + VS_RHO + cx * RZ + cz;
            const float r0 = rh[0];
            rip = (float)(0.5 * (double)(r0 + rh[RZ]));
            rjp = (float)(0.5 * (double)(r0 + stage[VS_RJ + tx * TZ + tz]));
            rkp = (float)(0.5 * (double)(r0 + rh[1]));
        }
        consumer_release<VRING, VNSTAGE>(bar, it, false, true);
        if (active) {
            // ring fields: 0 syy, 1 sxy, 2 syz
#define RF(Rp, f, x, z) Rp[(f) * RPLANE + (x) * RZ + (z)]
            float sxy_y = dy * (b1 * (RF(R0, 1, 0, 0) - RF(Rm1, 1, 0, 0)) + b2 * (RF(Rp1, 1, 0, 0) - RF(Rm2, 1, 0, 0)));
            float syy_y = dy * (b1 * (RF(Rp1, 0, 0, 0) - RF(R0, 0, 0, 0)) + b2 * (RF(Rp2, 0, 0, 0) - RF(Rm1, 0, 0, 0)));
            float sxy_x = dx * (b1 * (RF(R0, 1, 0, 0) - RF(R0, 1, -1, 0)) + b2 * (RF(R0, 1, 1, 0) - RF(R0, 1, -2, 0)));
            float syz_z = dz * (b1 * (RF(R0, 2, 0, 0) - RF(R0, 2, 0, -1)) + b2 * (RF(R0, 2, 0, 1) - RF(R0, 2, 0, -2)));
            float syz_y = dy * (b1 * (RF(R0, 2, 0, 0) - RF(Rm1, 2, 0, 0)) + b2 * (RF(Rp1, 2, 0, 0) - RF(Rm2, 2, 0, 0)));
#undef RF
            const int hy = face_y(g, j);
            const bool frame = hx || hy || hz;
            if (XZ && hx) {
                float *p = ps + sxi(g, j, hx, k);
                const long long o = a.sl.sx;
                float v0 = CP(BH_X, hx) * q.x[0] + CP(AH_X, hx) * sxx_x; p[0] = v0; sxx_x = div_rn(sxx_x, CP(KH_X, hx)) + v0;
                float v1 = CP(B_X, hx) * q.x[1] + CP(A_X, hx) * sxy_x; p[o] = v1; sxy_x = div_rn(sxy_x, CP(K_X, hx)) + v1;
                float v2 = CP(B_X, hx) * q.x[2] + CP(A_X, hx) * sxz_x; p[2 * o] = v2; sxz_x = div_rn(sxz_x, CP(K_X, hx)) + v2;
            }
            if (hy) {
                float *p = ps + 3 * a.sl.sx + syi(g, hy, i, k);
                const long long o = a.sl.sy;
                float v0 = CP(B_Y, hy) * q.y[0] + CP(A_Y, hy) * sxy_y; p[0] = v0; sxy_y = div_rn(sxy_y, CP(K_Y, hy)) + v0;
                float v1 = CP(BH_Y, hy) * q.y[1] + CP(AH_Y, hy) * syy_y; p[o] = v1; syy_y = div_rn(syy_y, CP(KH_Y, hy)) + v1;
                float v2 = CP(B_Y, hy) * q.y[2] + CP(A_Y, hy) * syz_y; p[2 * o] = v2; syz_y = div_rn(syz_y, CP(K_Y, hy)) + v2;
            }
            if (XZ && hz) {
                float *p = ps + 3 * a.sl.sx + 3 * a.sl.sy + szi(g, j, i, hz);
                const long long o = a.sl.sz;
                const float *cg = a.cpg;
                float v0 = CPG(cg, B_Z, hz) * q.z[0] + CPG(cg, A_Z, hz) * sxz_z; p[0] = v0; sxz_z = div_rn(sxz_z, CPG(cg, K_Z, hz)) + v0;
                float v1 = CPG(cg, B_Z, hz) * q.z[1] + CPG(cg, A_Z, hz) * syz_z; p[o] = v1; syz_z = div_rn(syz_z, CPG(cg, K_Z, hz)) + v1;
                float v2 = CPG(cg, BH_Z, hz) * q.z[2] + CPG(cg, AH_Z, hz) * szz_z; p[2 * o] = v2; szz_z = div_rn(szz_z, CPG(cg, KH_Z, hz)) + v2;
            }
            // the next plane's PML memory, a plane ahead of its use
            if (j < j1 && (hx || hz || face_y(g, j + 1))) psi_load(q, ps, a.sl, g, j + 1, i, k, hx, hz);
            if (p1 > p0) {
                // cells of this block hold point forces: the order of update_v / update_v_CPML
                const long long c = V - st;
                V[VX * F] = vxo; V[VY * F] = vyo; V[VZ * F] = vzo;
                if (frame) vel_points<BACK>(a, st, p0, p1, j, i, k, nt, c);
                V[VX * F] = V[VX * F] + div_rn(sxx_x + sxy_y + sxz_z, rip);
                V[VY * F] = V[VY * F] + div_rn(syy_y + sxy_x + syz_z, rjp);
                V[VZ * F] = V[VZ * F] + div_rn(szz_z + sxz_x + syz_y, rkp);
                const int passes = frame ? (BACK ? 1 : 0) : (BACK ? 2 : 1);
                for (int pass = 0; pass < passes; ++pass) vel_points<BACK>(a, st, p0, p1, j, i, k, nt, c);
            } else {
                V[VX * F] = vxo + div_rn(sxx_x + sxy_y + sxz_z, rip);
                V[VY * F] = vyo + div_rn(syy_y + sxy_x + syz_z, rjp);
                V[VZ * F] = vzo + div_rn(szz_z + sxz_x + syz_y, rkp);
            }
            if (j == probe_j && isnan(V[VY * F])) atomicMin(a.err_step + s, nt);
        }
        consumer_release<VRING, VNSTAGE>(bar, it, true, false);
        // planes move down one slot; the plane loaded into slot nslot becomes j+2
        Rm2 = Rm1; Rm1 = R0; R0 = Rp1; Rp1 = Rp2; Rp2 = Rb + nslot * RSLOT;
        if (++nslot == VRING) nslot = 0;
    }
}

// ---------------------------------------------------------------------------
// Velocity update. Stage layout: [sxx|szz|sxz halo planes][rho halo plane][vx vy vz]
// [rho of the next plane]: rho (one word per cell, shared by the shots) replaces
// the three averaged densities.
template <bool BACK>
__global__ void __launch_bounds__(NTHR, 3) k_velocity_tma(const __grid_constant__ VelTma T, int nt) {
    extern __shared__ __align__(128) unsigned char smem[];
    const VelArgs &a = T.a;
    const Geo &g = a.g;
    const int tz = threadIdx.x, tx = threadIdx.y;
    const int k0 = blockIdx.x * TZ + 1, i0 = blockIdx.y * TX + 1;
    const int ycn = blockIdx.z % g.nyc, s = blockIdx.z / g.nyc;
    const int j0 = ycn * g.cy + 1, j1 = min(j0 + g.cy - 1, g.ny);
    const int n = j1 - j0 + 1;
    float *ring = reinterpret_cast<float *>(smem);
    constexpr int SP = VS_SP;
    float *stg = ring + VRING * RSLOT;
    uint64_t *bar = reinterpret_cast<uint64_t *>(stg + VNSTAGE * SP);
    const int rfirst = j0 - 2, rlast = j1 + 2;
    if (!pipeline_start<VRING, VNSTAGE>(bar, T.tma_err)) return;

    if (tx == TX) {  // ---------------- producer warp
        if (tz != 0) return;
        auto ring_load = [&](int P) {
            const int sl = (P - rfirst) % VRING;
            mbar_expect_tx(&bar[sl], 3 * RPLANE * 4);
            tma_load5(ring + sl * RSLOT, &T.m_halo, zc(k0) - HZ, xc(i0) - HX, yc_(P), SYY, s, &bar[sl]);
        };
        auto stage_load = [&](int it) {
            const int j = j0 + it, b = it % VNSTAGE;
            float *d = stg + b * SP;
            uint64_t *fb = &bar[2 * VRING + b];
            mbar_expect_tx(fb, (4 * RPLANE + 4 * PT) * 4);
            tma_load5(d, &T.m_halo, zc(k0) - HZ, xc(i0) - HX, yc_(j), SXX, s, fb);
            tma_load3(d + VS_RHO, &T.m_rho_halo, zc(k0) - HZ, xc(i0) - HX, yc_(j), fb);
            tma_load5(d + VS_PT, &T.m_pt, zc(k0), xc(i0), yc_(j), VX, s, fb);
            tma_load3(d + VS_RJ, &T.m_rho_pt, zc(k0), xc(i0), yc_(j + 1), fb);
        };
        auto stage_prefetch = [&](int it) {
            const int j = j0 + it;
            tma_prefetch5(&T.m_halo, zc(k0) - HZ, xc(i0) - HX, yc_(j), SXX, s);
            tma_prefetch3(&T.m_rho_halo, zc(k0) - HZ, xc(i0) - HX, yc_(j));
            tma_prefetch5(&T.m_pt, zc(k0), xc(i0), yc_(j), VX, s);
        };
        auto ring_prefetch = [&](int P) { tma_prefetch5(&T.m_halo, zc(k0) - HZ, xc(i0) - HX, yc_(P), SYY, s); };
        const uint64_t lim = T.w.limit_ns;
        int ring_hi = min(rfirst + VRING - 1, rlast), stage_hi = min(VNSTAGE, n) - 1;
        for (int P = rfirst; P <= ring_hi; ++P) ring_load(P);
        for (int it = 0; it <= stage_hi; ++it) stage_load(it);
        for (int q = 0; q < T.l2ahead; ++q) {
            if (VNSTAGE + q < n) stage_prefetch(VNSTAGE + q);
            if (rfirst + VRING + q <= rlast) ring_prefetch(rfirst + VRING + q);
        }
        for (int it = 0; it < n; ++it) {
            if (it == T.w.stop_it) {  // failure-path test: issue nothing more
                producer_drain<VRING, VNSTAGE>(bar, rfirst, ring_hi, stage_hi, lim);
                return;
            }
            if (rfirst + it + VRING <= rlast) {
                if (!mbar_wait(&bar[VRING + it % VRING], (it / VRING) & 1, lim)) {
                    atomicExch(T.tma_err, 1);
                    producer_drain<VRING, VNSTAGE>(bar, rfirst, ring_hi, stage_hi, lim);
                    return;
                }
                ring_load(ring_hi = rfirst + it + VRING);
                if (T.l2ahead > 0 && rfirst + it + VRING + T.l2ahead <= rlast) ring_prefetch(rfirst + it + VRING + T.l2ahead);
            }
            if (it + VNSTAGE < n) {
                if (!mbar_wait(&bar[2 * VRING + VNSTAGE + it % VNSTAGE], (it / VNSTAGE) & 1, lim)) {
                    atomicExch(T.tma_err, 1);
                    producer_drain<VRING, VNSTAGE>(bar, rfirst, ring_hi, stage_hi, lim);
                    return;
                }
                stage_load(stage_hi = it + VNSTAGE);
                if (T.l2ahead > 0 && it + VNSTAGE + T.l2ahead < n) stage_prefetch(it + VNSTAGE + T.l2ahead);
            }
        }
        return;
    }

    // ---------------- consumer warps: row tx of the tile
    // A tile that touches no x or z PML face lies wholly inside the grid: the
    // lean instance drops the x/z frame code and the bounds test.
    const bool xz = i0 <= g.fw || i0 + TX - 1 > g.nx - g.fw || k0 <= g.fw || k0 + TZ - 1 > g.nz - g.fw;
    if (xz) vel_rows<BACK, true>(T, nt, ring, stg, bar, j0, j1, s, ycn, k0, i0);
    else vel_rows<BACK, false>(T, nt, ring, stg, bar, j0, j1, s, ycn, k0, i0);
}


// Register cap of the stress kernel. An SM sub-partition holds 16,384 registers
// and a CTA's TX+1 warps spread over the 4 sub-partitions, so the cap decides how
// many CTAs share an SM. 8-row tiles (9 warps): two CTAs need 5 warps on one
// sub-partition, i.e. at most 96 registers; the elastic kernel fits that without
// spills, with memory variables 96 spills, so those keep 112 (one CTA per SM).
// 7-row tiles (8 warps): two CTAs per SM at up to 128 registers, no spills.
constexpr int STR_REGS_ELASTIC = TX == 8 ? 96 : 128;
constexpr int STR_REGS_MECH = TX == 8 ? 112 : 128;
template <int L, bool P2>
__global__ void __maxnreg__(L == 0 ? STR_REGS_ELASTIC : STR_REGS_MECH) k_stress_tma(const __grid_constant__ StrTma T, int nt, int do_dft, int sample) {
    extern __shared__ __align__(128) unsigned char smem[];
    const StrArgs &a = T.a;
    const Geo &g = a.g;
    const int tz = threadIdx.x, tx = threadIdx.y;
    const int k0 = blockIdx.x * TZ + 1, i0 = blockIdx.y * TX + 1;
    const int ycn = blockIdx.z % g.nyc, s = blockIdx.z / g.nyc;
    const int j0 = ycn * g.cy + 1, j1 = min(j0 + g.cy - 1, g.ny);
    const int n = j1 - j0 + 1;
    const int nsr = T.nsr, nm = T.nm, ndf = do_dft ? T.ndf : 0;
    const int SP = str_stage(nsr, nm, T.ndf), MOFF = str_mod_off(nsr), DOFF = str_dft_off(nsr, nm);
    float *ring = reinterpret_cast<float *>(smem);
    float *stg = ring + RING * RSLOT;
    uint64_t *bar = reinterpret_cast<uint64_t *>(stg + NSTAGE * SP);
    const int rfirst = j0 - 2, rlast = j1 + 2;
    if (!pipeline_start<RING, NSTAGE>(bar, T.tma_err)) return;

    if (tx == TX) {  // ---------------- producer warp
        if (tz != 0) return;
        const uint32_t stage_bytes = (uint32_t)(nsr + nm + ndf) * PT * 4;
        auto ring_load = [&](int P) {
            const int sl = (P - rfirst) % RING;
            mbar_expect_tx(&bar[sl], 3 * RPLANE * 4);
            tma_load5(ring + sl * RSLOT, &T.m_halo, zc(k0) - HZ, xc(i0) - HX, yc_(P), VX, s, &bar[sl]);
        };
        auto stage_load = [&](int it) {
            const int j = j0 + it, b = it % NSTAGE;
            float *d = stg + b * SP;
            uint64_t *fb = &bar[2 * RING + b];
            mbar_expect_tx(fb, stage_bytes);
            tma_load5(d, &T.m_sr, zc(k0), xc(i0), yc_(j), SYY, s, fb);
            tma_load4(d + MOFF, &T.m_mod, zc(k0), xc(i0), yc_(j), 0, fb);
            if (ndf) tma_load5(d + DOFF, &T.m_dft, zc(k0), xc(i0), yc_(j), 0, s, fb);
        };
        auto stage_prefetch = [&](int it) {
            const int j = j0 + it;
            tma_prefetch5(&T.m_sr, zc(k0), xc(i0), yc_(j), SYY, s);
            tma_prefetch4(&T.m_mod, zc(k0), xc(i0), yc_(j), 0);
            if (ndf) tma_prefetch5(&T.m_dft, zc(k0), xc(i0), yc_(j), 0, s);
        };
        auto ring_prefetch = [&](int P) { tma_prefetch5(&T.m_halo, zc(k0) - HZ, xc(i0) - HX, yc_(P), VX, s); };
        const uint64_t lim = T.w.limit_ns;
        int ring_hi = min(rfirst + RING - 1, rlast), stage_hi = min(NSTAGE, n) - 1;
        for (int P = rfirst; P <= ring_hi; ++P) ring_load(P);
        for (int it = 0; it <= stage_hi; ++it) stage_load(it);
        for (int q = 0; q < T.l2ahead; ++q) {
            if (NSTAGE + q < n) stage_prefetch(NSTAGE + q);
            if (rfirst + RING + q <= rlast) ring_prefetch(rfirst + RING + q);
        }
        for (int it = 0; it < n; ++it) {
            if (it == T.w.stop_it) {  // failure-path test: issue nothing more
                producer_drain<RING, NSTAGE>(bar, rfirst, ring_hi, stage_hi, lim);
                return;
            }
            if (rfirst + it + RING <= rlast) {
                if (!mbar_wait(&bar[RING + it % RING], (it / RING) & 1, lim)) {
                    atomicExch(T.tma_err, 1);
                    producer_drain<RING, NSTAGE>(bar, rfirst, ring_hi, stage_hi, lim);
                    return;
                }
                ring_load(ring_hi = rfirst + it + RING);
                if (T.l2ahead > 0 && rfirst + it + RING + T.l2ahead <= rlast) ring_prefetch(rfirst + it + RING + T.l2ahead);
            }
            if (it + NSTAGE < n) {
                if (!mbar_wait(&bar[2 * RING + NSTAGE + it % NSTAGE], (it / NSTAGE) & 1, lim)) {
                    atomicExch(T.tma_err, 1);
                    producer_drain<RING, NSTAGE>(bar, rfirst, ring_hi, stage_hi, lim);
                    return;
                }
                stage_load(stage_hi = it + NSTAGE);
                if (T.l2ahead > 0 && it + NSTAGE + T.l2ahead < n) stage_prefetch(it + NSTAGE + T.l2ahead);
            }
        }
        return;
    }

    // ---------------- consumer warps: row tx of the tile
    const int k = k0 + tz, i = i0 + tx;
    const bool active = k <= g.nz && i <= g.nx;
    int p0, p1;
    block_points(a.pt_off, g, s, ycn, p0, p1);
    float *st = a.st + (long long)s * a.st_shot;
    float *ps = a.psi + (long long)s * a.psi_shot + 3 * (a.sl.sx + a.sl.sy + a.sl.sz);
    const long long F = g.field, dJ = g.plane;
    const float b1 = a.b1, b2 = a.b2, DX = a.rdx, DY = a.rdy, DZ = a.rdz, DT = a.dt;
    const float iX = T.idx, iY = T.idy, iZ = T.idz;
    const int hx = face_x(g, i), hz = face_z(g, k);
    const bool zfront = k <= g.fw;
    const int cz = tz + HZ, cx = tx + HX;
    int sl = 2;
    PsiPre q{};
    if (active && (hx || hz || face_y(g, j0))) psi_load(q, ps, a.sl, g, j0, i, k, hx, hz);
    for (int it = 0, j = j0; j <= j1; ++it, ++j) {
        if (!consumer_wait(bar, it, j, j0, rfirst, T.w.limit_ns)) { if (tz == 0) atomicExch(T.tma_err, 1); return; }
        if (active) {
            const float *stage = stg + (it % NSTAGE) * SP;
            const int sm2 = sl >= 2 ? sl - 2 : sl + RING - 2, sm1 = sl >= 1 ? sl - 1 : sl + RING - 1;
            const int sp1 = sl + 1 < RING ? sl + 1 : sl + 1 - RING, sp2 = sl + 2 < RING ? sl + 2 : sl + 2 - RING;
            const float *R0 = ring + sl * RSLOT + cx * RZ + cz;
            const float *Rm2 = ring + sm2 * RSLOT + cx * RZ + cz, *Rm1 = ring + sm1 * RSLOT + cx * RZ + cz;
            const float *Rp1 = ring + sp1 * RSLOT + cx * RZ + cz, *Rp2 = ring + sp2 * RSLOT + cx * RZ + cz;
#define RF(Rp, f, x, z) Rp[(f) * RPLANE + (x) * RZ + (z)]
            const float vx0 = RF(R0, 0, 0, 0), vy0 = RF(R0, 1, 0, 0), vz0 = RF(R0, 2, 0, 0);
            float vxx = ddiv<P2>(b1 * (vx0 - RF(R0, 0, -1, 0)) + b2 * (RF(R0, 0, 1, 0) - RF(R0, 0, -2, 0)), DX, iX);
            float vxy = ddiv<P2>(b1 * (RF(Rp1, 0, 0, 0) - vx0) + b2 * (RF(Rp2, 0, 0, 0) - RF(Rm1, 0, 0, 0)), DY, iY);
            float vxz = ddiv<P2>(b1 * (RF(R0, 0, 0, 1) - vx0) + b2 * (RF(R0, 0, 0, 2) - RF(R0, 0, 0, -1)), DZ, iZ);
            float vyx = ddiv<P2>(b1 * (RF(R0, 1, 1, 0) - vy0) + b2 * (RF(R0, 1, 2, 0) - RF(R0, 1, -1, 0)), DX, iX);
            float vyy = ddiv<P2>(b1 * (vy0 - RF(Rm1, 1, 0, 0)) + b2 * (RF(Rp1, 1, 0, 0) - RF(Rm2, 1, 0, 0)), DY, iY);
            float vyz = ddiv<P2>(b1 * (RF(R0, 1, 0, 1) - vy0) + b2 * (RF(R0, 1, 0, 2) - RF(R0, 1, 0, -1)), DZ, iZ);
            float vzx = ddiv<P2>(b1 * (RF(R0, 2, 1, 0) - vz0) + b2 * (RF(R0, 2, 2, 0) - RF(R0, 2, -1, 0)), DX, iX);
            float vzy = ddiv<P2>(b1 * (RF(Rp1, 2, 0, 0) - vz0) + b2 * (RF(Rp2, 2, 0, 0) - RF(Rm1, 2, 0, 0)), DY, iY);
            float vzz = ddiv<P2>(b1 * (vz0 - RF(R0, 2, 0, -1)) + b2 * (RF(R0, 2, 0, 1) - RF(R0, 2, 0, -2)), DZ, iZ);
#undef RF
            const float svxx = vxx, svyy = vyy, svzz = vzz;  // the free surface uses the plain derivatives
            const int hy = face_y(g, j);
            if (hx) {
                float *p = ps + sxi(g, j, hx, k);
                const long long o = a.sl.sx;
                float v0 = CP(B_X, hx) * q.x[0] + CP(A_X, hx) * vxx; p[0] = v0; vxx = div_rn(vxx, CP(K_X, hx)) + v0;
                float v1 = CP(BH_X, hx) * q.x[1] + CP(AH_X, hx) * vyx; p[o] = v1; vyx = div_rn(vyx, CP(KH_X, hx)) + v1;
                float v2 = CP(BH_X, hx) * q.x[2] + CP(AH_X, hx) * vzx; p[2 * o] = v2; vzx = div_rn(vzx, CP(KH_X, hx)) + v2;
            }
            if (hy) {
                float *p = ps + 3 * a.sl.sx + syi(g, hy, i, k);
                const long long o = a.sl.sy;
                float v0 = CP(BH_Y, hy) * q.y[0] + CP(AH_Y, hy) * vxy; p[0] = v0; vxy = div_rn(vxy, CP(KH_Y, hy)) + v0;
                float v1 = CP(B_Y, hy) * q.y[1] + CP(A_Y, hy) * vyy; p[o] = v1; vyy = div_rn(vyy, CP(K_Y, hy)) + v1;
                float v2 = CP(BH_Y, hy) * q.y[2] + CP(AH_Y, hy) * vzy; p[2 * o] = v2; vzy = div_rn(vzy, CP(KH_Y, hy)) + v2;
            }
            if (hz) {
                // the reference divides by K_y on the front z face (update_s_ssg_CPML_elastic.c:104-108)
                float *p = ps + 3 * a.sl.sx + 3 * a.sl.sy + szi(g, j, i, hz);
                const long long o = a.sl.sz;
                const float *cg = a.cpg;
                const float kh = zfront ? CPG(cg, KH_Y, hz) : CPG(cg, KH_Z, hz);
                const float kf = zfront ? CPG(cg, K_Y, hz) : CPG(cg, K_Z, hz);
                float v0 = CPG(cg, BH_Z, hz) * q.z[0] + CPG(cg, AH_Z, hz) * vxz; p[0] = v0; vxz = div_rn(vxz, kh) + v0;
                float v1 = CPG(cg, BH_Z, hz) * q.z[1] + CPG(cg, AH_Z, hz) * vyz; p[o] = v1; vyz = div_rn(vyz, kh) + v1;
                float v2 = CPG(cg, B_Z, hz) * q.z[2] + CPG(cg, A_Z, hz) * vzz; p[2 * o] = v2; vzz = div_rn(vzz, kf) + v2;
            }
            // the next plane's PML memory, a plane ahead of its use
            if (j < j1 && (hx || hz || face_y(g, j + 1))) psi_load(q, ps, a.sl, g, j + 1, i, k, hx, hz);
            const float *S = stage + tx * TZ + tz;      // sigma + memory variables (old values)
            const float *Mo = S + MOFF;                 // model
            const float pim = Mo[MD_PI * PT], um = Mo[MD_U * PT];
            const float uipjp = Mo[MD_UIPJP * PT], ujpkp = Mo[MD_UJPKP * PT], uipkp = Mo[MD_UIPKP * PT];
            const float vxyyx = vxy + vyx, vyzzy = vyz + vzy, vxzzx = vxz + vzx;
            const float vxxyyzz = vxx + vyy + vzz, vyyzz = vyy + vzz, vxxzz = vxx + vzz, vxxyy = vxx + vyy;
            // stage order of sigma: syy, sxy, syz, sxx, szz, sxz (state slots 3..8)
            float syy = S[0], sxy = S[PT], syz = S[2 * PT], sxx = S[3 * PT], szz = S[4 * PT], sxz = S[5 * PT];
            const long long c = widx(g, j, i, k);
            float *O = st + c;
            const bool surf = g.free_surf && j == 1;
            float taus = 0.f, taup = 0.f, sr[6];
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
                float tausipjp, tausjpkp, tausipkp;
                if (nm == 5) {
                    taus = T.utaus; taup = T.utaup;
                    tausipjp = tausjpkp = tausipkp = T.uts_avg;
                } else {
                    taus = Mo[MD_TAUS * PT]; taup = Mo[MD_TAUP * PT];
                    tausipjp = Mo[MD_TSIPJP * PT]; tausjpkp = Mo[MD_TSJPKP * PT]; tausipkp = Mo[MD_TSIPKP * PT];
                }
                const float Lf = (float)L, dthalbe = a.dthalbe;
                const float *R = S + 6 * PT;  // r[l][q] at (6 l + q) PT
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    sr[q] = R[q * PT];
#pragma unroll
                    for (int l = 1; l < L; ++l) sr[q] += R[(6 * l + q) * PT];
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
                // memory variables, one mechanism at a time from the stage's old values
#pragma unroll
                for (int l = 0; l < L; ++l) {
                    const float eta = a.eta[l], bb = a.mb[l], cc = a.mc[l];
                    const float dipjp = uipjp * eta * tausipjp, djpkp = ujpkp * eta * tausjpkp, dipkp = uipkp * eta * tausipkp;
                    const float d = (float)(((2.0 * (double)um) * (double)eta) * (double)taus);
                    const float e = pim * eta * taup;
                    const float *Rl = R + 6 * l * PT;
                    const float nxy = bb * (Rl[3 * PT] * cc - (dipjp * vxyyx));
                    const float nyz = bb * (Rl[4 * PT] * cc - (djpkp * vyzzy));
                    const float nxz = bb * (Rl[5 * PT] * cc - (dipkp * vxzzx));
                    const float nxx = bb * (Rl[0] * cc - (e * vxxyyzz) + (d * vyyzz));
                    const float nyy = bb * (Rl[PT] * cc - (e * vxxyyzz) + (d * vxxzz));
                    const float nzz = bb * (Rl[2 * PT] * cc - (e * vxxyyzz) + (d * vxxyy));
                    if (l == 0) {
                        sr[0] = nxx; sr[1] = nyy; sr[2] = nzz; sr[3] = nxy; sr[4] = nyz; sr[5] = nxz;
                    } else {
                        sr[0] += nxx; sr[1] += nyy; sr[2] += nzz; sr[3] += nxy; sr[4] += nyz; sr[5] += nxz;
                    }
                    if (!surf) {
                        float *Ol = O + (NEL + 6 * l) * F;
                        Ol[0] = nxx; Ol[F] = nyy; Ol[2 * F] = nzz; Ol[3 * F] = nxy; Ol[4 * F] = nyz; Ol[5 * F] = nxz;
                    }
                }
                sxy += (dthalbe * sr[3]);
                syz += (dthalbe * sr[4]);
                sxz += (dthalbe * sr[5]);
                sxx += (dthalbe * sr[0]);
                syy += (dthalbe * sr[1]);
                szz += (dthalbe * sr[2]);
            }
            if (p1 > p0) {
                for (int q = p0; q < p1; ++q) {
                    const Pt pt = a.pts[q];
                    if (pt.kind == PT_EXPLOSIVE && pt.j == j && pt.i == i && pt.k == k) {
                        const float amp = a.amp[(long long)pt.row * a.amp_row + (nt - 1)];
                        sxx += amp; syy += amp; szz += amp;
                    }
                }
            }
            if (ndf) {
                const float *Fs = S + DOFF;
                float *Fd = a.dft + (long long)s * a.dft_shot + c;
                const double *tr = a.trig + (long long)(nt - 1) * a.nf * 2;
                for (int l = 0; l < a.nf; ++l) {
                    const double t1 = tr[2 * l], t2 = tr[2 * l + 1];
                    const float *Fl = Fs + l * 6 * PT;
                    float *Gl = Fd + (long long)l * 6 * F;
                    Gl[0 * F] = (float)((double)Fl[0 * PT] + (double)vx0 * t1);
                    Gl[1 * F] = (float)((double)Fl[1 * PT] + (double)vy0 * t1);
                    Gl[2 * F] = (float)((double)Fl[2 * PT] + (double)vz0 * t1);
                    Gl[3 * F] = (float)((double)Fl[3 * PT] + (double)vx0 * t2);
                    Gl[4 * F] = (float)((double)Fl[4 * PT] + (double)vy0 * t2);
                    Gl[5 * F] = (float)((double)Fl[5 * PT] + (double)vz0 * t2);
                }
            }
            if (surf) {
                // surface_ssg_elastic.c:69-111 / surface_ssg.c:117-160
                syy = 0.0f;
                if constexpr (L == 0) {
                    float spi = pim, su = um;
                    if (a.smod) {  // the surface's own moduli (the reference's step-length forwards)
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
                    const float f = (float)(((double)um * 2.0) * (1.0 + (double)(Lf * taus)));
                    const float gg = (float)((double)pim * (1.0 + (double)(Lf * taup)));
                    const float h = -(DT * (gg - f) * (gg - f) * (svxx + svzz) / gg) - (DT * (gg - f) * svyy);
                    sxx += h - (dthalbe * sr[0]);
                    szz += h - (dthalbe * sr[2]);
                    const float d = (float)((2.0 * (double)um) * (double)taus);
                    const float e = pim * taup;
                    // the memory variables of the surface row: recompute each mechanism's
                    // update (same bits), apply the surface term, then store
                    const float *R = S + 6 * PT;
                    const float tausipjp = nm == 5 ? T.uts_avg : Mo[MD_TSIPJP * PT];
                    const float tausjpkp = nm == 5 ? T.uts_avg : Mo[MD_TSJPKP * PT];
                    const float tausipkp = nm == 5 ? T.uts_avg : Mo[MD_TSIPKP * PT];
                    float srx = 0.f, srz = 0.f;
#pragma unroll
                    for (int l = 0; l < L; ++l) {
                        const float eta = a.eta[l], bb = a.mb[l], cc = a.mc[l];
                        const float dipjp = uipjp * eta * tausipjp, djpkp = ujpkp * eta * tausjpkp, dipkp = uipkp * eta * tausipkp;
                        const float dd = (float)(((2.0 * (double)um) * (double)eta) * (double)taus);
                        const float ee = pim * eta * taup;
                        const float *Rl = R + 6 * l * PT;
                        const float nxy = bb * (Rl[3 * PT] * cc - (dipjp * vxyyx));
                        const float nyz = bb * (Rl[4 * PT] * cc - (djpkp * vyzzy));
                        const float nxz = bb * (Rl[5 * PT] * cc - (dipkp * vxzzx));
                        float nxx = bb * (Rl[0] * cc - (ee * vxxyyzz) + (dd * vyyzz));
                        float nzz = bb * (Rl[2 * PT] * cc - (ee * vxxyyzz) + (dd * vxxyy));
                        const float hh = (float)((double)a.msb[l] *
                                                 ((((double)(d - e) * ((double)(f / gg) - 1.0)) * (double)(svxx + svzz)) -
                                                  (double)((d - e) * svyy)));
                        nxx += hh;
                        nzz += hh;
                        if (l == 0) { srx = nxx; srz = nzz; } else { srx += nxx; srz += nzz; }
                        float *Ol = O + (NEL + 6 * l) * F;
                        Ol[0] = nxx; Ol[F] = 0.0f; Ol[2 * F] = nzz; Ol[3 * F] = nxy; Ol[4 * F] = nyz; Ol[5 * F] = nxz;
                    }
                    sxx += (dthalbe * srx);
                    szz += (dthalbe * srz);
                }
            }
            O[SYY * F] = syy; O[SXY * F] = sxy; O[SYZ * F] = syz;
            O[SXX * F] = sxx; O[SZZ * F] = szz; O[SXZ * F] = sxz;
            if (g.free_surf && j <= 3) {
                if (j == 1) { O[SXY * F - dJ] = -sxy; O[SYZ * F - dJ] = -syz; }
                if (j == 2) { O[SYY * F - 2 * dJ] = -syy; O[SXY * F - 3 * dJ] = -sxy; O[SYZ * F - 3 * dJ] = -syz; }
                if (j == 3) { O[SYY * F - 4 * dJ] = -syy; }
            }
            if (sample >= 0 && p1 > p0) {
                for (int q = p0; q < p1; ++q) {
                    const Pt pt = a.pts[q];
                    if (pt.kind == PT_RECEIVER && pt.j == j && pt.i == i && pt.k == k) {
                        float *o = a.sec + (long long)s * a.sec_shot + (long long)pt.row * a.sec_tr + sample;
                        o[0] = vx0;
                        o[a.sec_comp] = vy0;
                        o[2 * a.sec_comp] = vz0;
                        if (a.seismo >= 2) {
#define RV(Rp, f, x, z) Rp[(f) * RPLANE + (x) * RZ + (z)]
                            const long long c = widx(g, j, i, k);
                            float pr, dv, cu;
                            seismo_pdc(vx0, RV(R0, 0, -1, 0), RV(Rp1, 0, 0, 0), RV(R0, 0, 0, 1), vy0, RV(Rm1, 1, 0, 0),
                                       RV(R0, 1, 1, 0), RV(R0, 1, 0, 1), vz0, RV(R0, 2, 0, -1), RV(R0, 2, 1, 0),
                                       RV(Rp1, 2, 0, 0), sxx, syy, szz, a.md[MD_PI * F + c], a.md[MD_U * F + c], a.hrx,
                                       a.hry, a.hrz, pr, dv, cu);
#undef RV
                            float *o2 = a.sec2 + (long long)s * a.sec_shot + (long long)pt.row * a.sec_tr + sample;
                            o2[0] = pr;
                            o2[a.sec_comp] = dv;
                            o2[2 * a.sec_comp] = cu;
                        }
                    }
                }
            }
        }
        consumer_release(bar, it, true, true);
        sl = sl + 1 < RING ? sl + 1 : 0;
    }
}
