// TMA-staged time-step kernels (sm_100a).
//
// A CTA owns an x-z tile (TZ=32 cells along z, TX=7 or 8 rows along x) of one shot and
// streams along y through a chunk of planes. Per plane, the Tensor Memory
// Accelerator brings into shared memory
//   * the stencil planes with their x/z halos into a ring of RING planes
//     (velocity kernel: syy, sxy, syz; stress kernel: vx, vy, vz), and
//   * the point-wise fields of the plane into one of two stage buffers (velocity
//     kernel: v and rip/rjp/rkp plus the in-plane stencil fields sxx, szz, sxz;
//     stress kernel: sigma and every memory variable in one 5-D box, the model
//     coefficients, and the DFT accumulators on DFT steps),
// each completing on a "full" mbarrier with the byte count of its boxes. One
// producer warp issues every TMA load; the TX consumer warps compute one row of
// the tile each and hand a ring plane or a stage back through an "empty"
// mbarrier once they have read it, so warps never wait on each other through
// CTA-wide barriers. Results go straight from registers to HBM with coalesced
// stores (consumers never write shared memory). No cluster multicast is used.
//
// Every mbarrier wait is bounded in time (1 s of %globaltimer): on expiry the
// warp sets the error flag and returns; the other warps' waits then expire in
// turn, and CTAs that start after the flag is set return at once.
//
// The per-cell arithmetic is the expression sequence of the plain kernels in
// ifosb_kernels.cuh (and of the reference), so the results are bit-identical.
// With power-of-two grid spacings the divisions by DX, DY, DZ become
// multiplications by the exact reciprocal, which gives the same bits.
#pragma once
#include <cuda.h>

#include "ifosb_kernels.cuh"

namespace ifosb {

constexpr int TZ = 32;    // tile extent along z (== BX)
#ifndef IFOSB_RING
#define IFOSB_RING 6
#endif
constexpr int RING = IFOSB_RING;  // stencil planes held: j-2..j+2 and RING-5 being loaded
static_assert(RING >= 6, "the stencil needs planes j-2..j+2 plus one in flight");
constexpr int HZ = 4;     // z halo (keeps TMA z-coordinates 16-byte aligned)
constexpr int HX = 2;     // x halo
constexpr int RZ = TZ + 2 * HZ;              // ring row length
// TMA writes shared memory only at 128-byte aligned destinations: every box
// starts on a multiple of 32 floats (padding is empty for TX = 8).
__host__ __device__ constexpr int a32(int x) { return (x + 31) & ~31; }
#ifndef IFOSB_NSTAGE
#define IFOSB_NSTAGE 2
#endif
constexpr int NSTAGE = IFOSB_NSTAGE;         // stage buffers (point-wise fields of NSTAGE planes in flight)
static_assert(NSTAGE >= 2, "two stages at least");
constexpr int NBAR = 2 * RING + 2 * NSTAGE;  // full/empty per ring slot, full/empty per stage
// The velocity kernel holds less per plane than the stress kernel, so it can
// afford a deeper ring and more stages (more loads in flight per CTA).
#ifndef IFOSB_VRING
#define IFOSB_VRING RING
#endif
#ifndef IFOSB_VNSTAGE
#define IFOSB_VNSTAGE NSTAGE
#endif
constexpr int VRING = IFOSB_VRING;
constexpr int VNSTAGE = IFOSB_VNSTAGE;
static_assert(VRING >= 6 && VNSTAGE >= 2, "velocity ring: j-2..j+2 plus one in flight; two stages at least");
constexpr int VNBAR = 2 * VRING + 2 * VNSTAGE;

__device__ __forceinline__ uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}
// IFOSB_WAIT_HINT_NS > 0 lets a waiting thread be suspended in hardware for up
// to that many nanoseconds per try (instead of returning at once and spinning).
#ifndef IFOSB_WAIT_HINT_NS
#define IFOSB_WAIT_HINT_NS 0
#endif
__device__ __forceinline__ bool mbar_try(uint64_t *b, uint32_t parity) {
    uint32_t ok;
#if IFOSB_WAIT_HINT_NS > 0
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity), "r"((uint32_t)IFOSB_WAIT_HINT_NS)
        : "memory");
#else
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity)
        : "memory");
#endif
    return ok != 0;
}
__device__ __forceinline__ uint64_t gtimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait: gives up after `limit_ns` of wall time (1 s unless a test lowers
// it; a TMA box lands in microseconds).
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity, uint64_t limit_ns) {
    if (mbar_try(b, parity)) return true;
    const uint64_t t0 = gtimer();
    while (!mbar_try(b, parity))
        if (gtimer() - t0 > limit_ns) return false;
    return true;
}
constexpr uint64_t WAIT_LIMIT_NS = 1000000000ull;
__device__ __forceinline__ void tma_load5(void *dst, const CUtensorMap *m, int c0, int c1, int c2, int c3, int c4,
                                          uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(su32(dst)),
        "l"(m), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(su32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_load4(void *dst, const CUtensorMap *m, int c0, int c1, int c2, int c3, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(su32(dst)),
        "l"(m), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(su32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load3(void *dst, const CUtensorMap *m, int c0, int c1, int c2, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(su32(dst)),
        "l"(m), "r"(c0), "r"(c1), "r"(c2), "r"(su32(bar))
        : "memory");
}

// L2 prefetch of a box (no shared memory, no completion): warms L2 for a later load.
__device__ __forceinline__ void tma_prefetch5(const CUtensorMap *m, int c0, int c1, int c2, int c3, int c4) {
    asm volatile("cp.async.bulk.prefetch.tensor.5d.L2.global.tile [%0, {%1, %2, %3, %4, %5}];" ::"l"(m), "r"(c0), "r"(c1),
                 "r"(c2), "r"(c3), "r"(c4)
                 : "memory");
}
__device__ __forceinline__ void tma_prefetch3(const CUtensorMap *m, int c0, int c1, int c2) {
    asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(m), "r"(c0), "r"(c1), "r"(c2)
                 : "memory");
}
__device__ __forceinline__ void tma_prefetch4(const CUtensorMap *m, int c0, int c1, int c2, int c3) {
    asm volatile("cp.async.bulk.prefetch.tensor.4d.L2.global.tile [%0, {%1, %2, %3, %4}];" ::"l"(m), "r"(c0), "r"(c1), "r"(c2),
                 "r"(c3)
                 : "memory");
}

// Planes are prefetched into L2 `l2ahead` iterations before their shared-memory
// load (a launch argument, 0 = no L2 prefetch; the engine's autotuner picks it).
// Untuned defaults: the distances the autotuner picked on 128^3 to 384x256x384
// grids (velocity 1-2, stress 1 every time).
constexpr int L2AHEAD_VEL_DEFAULT = 2;
constexpr int L2AHEAD_STR_DEFAULT = 1;

// Tensor-map coordinates of a cell: z index k+7, row i+1, plane j+2.
__device__ __forceinline__ int zc(int k) { return k + 7; }
__device__ __forceinline__ int xc(int i) { return i + 1; }
__device__ __forceinline__ int yc_(int j) { return j + 2; }

// Failure-path test knobs of the TMA kernels: the mbarrier wait limit, and the
// chunk iteration at which the producer warp stops issuing loads (-1 = never).
// A producer that stops waits for the boxes it has issued and returns; the
// consumers' waits for the boxes never issued then run out.
struct WaitCtl {
    uint64_t limit_ns;
    int stop_it;
};

struct VelTma {
    CUtensorMap m_halo;      // state, box {RZ, RX, 1, 3, 1}
    CUtensorMap m_pt;        // state, box {TZ, TX, 1, 3, 1}
    CUtensorMap m_rho_halo;  // rho in field layout, box {RZ, RX, 1}
    CUtensorMap m_rho_pt;    // rho in field layout, box {TZ, TX, 1}
    VelArgs a;
    int *tma_err;
    int l2ahead;
    WaitCtl w;
};

struct StrTma {
    CUtensorMap m_halo;  // state, box {RZ, RX, 1, 3, 1}
    CUtensorMap m_sr;    // state, box {TZ, TX, 1, nsr, 1}
    CUtensorMap m_mod;   // model, box {TZ, TX, 1, nm}
    CUtensorMap m_dft;   // DFT accumulators, box {TZ, TX, 1, ndf, 1}
    StrArgs a;
    int nsr, nm, ndf;
    float utaus, utaup, uts_avg;  // uniform taus, taup and their staggered averages (nm == 5)
    float idx, idy, idz;          // exact 1/DX, 1/DY, 1/DZ (power-of-two spacings)
    int *tma_err;
    int l2ahead;
    WaitCtl w;
};

// PML memory values of one cell (x, y, z slabs: three each), read one plane ahead
// so that the global-memory latency overlaps the previous plane's work.
struct PsiPre {
    float x[3], y[3], z[3];
};
__device__ __forceinline__ void psi_load(PsiPre &q, const float *ps, const Slabs &sl, const Geo &g, int j, int i, int k,
                                         int hx, int hz) {
    if (hx) {
        const float *p = ps + sxi(g, j, hx, k);
        q.x[0] = p[0]; q.x[1] = p[sl.sx]; q.x[2] = p[2 * sl.sx];
    }
    const int hy = face_y(g, j);
    if (hy) {
        const float *p = ps + 3 * sl.sx + syi(g, hy, i, k);
        q.y[0] = p[0]; q.y[1] = p[sl.sy]; q.y[2] = p[2 * sl.sy];
    }
    if (hz) {
        const float *p = ps + 3 * sl.sx + 3 * sl.sy + szi(g, j, i, hz);
        q.z[0] = p[0]; q.z[1] = p[sl.sz]; q.z[2] = p[2 * sl.sz];
    }
}

// ---------------------------------------------------------------------------
// Stress update (+ source, DFT, free surface, receivers).
// Stage layout: [sigma(6) r(6L)][model(nm)][dft(6 nf) on DFT steps].
template <bool P2>
__device__ __forceinline__ float ddiv(float a, float d, float inv) {
    if constexpr (P2) return a * inv;
    else return div_rn(a, d);
}

// The tile-height-dependent part, compiled for 8-row and 7-row tiles. The engine
// takes 7-row tiles (8-warp CTAs, two per SM) when the stress kernel carries
// memory variables and 8-row tiles otherwise, the faster choice for each.
namespace t8 {
constexpr int TX = 8;
#include "ifosb_tma_tile.cuh"
}  // namespace t8
namespace t7 {
constexpr int TX = 7;
#include "ifosb_tma_tile.cuh"
}  // namespace t7

}  // namespace ifosb
