// ifosb_optim.cu — the inversion-loop updates of the reference driver on the
// device, with every reduction in FP64:
//   conjugate()      src/conjugategrad.c:27-110  (Mora 1987 CG direction)
//   lbfgs_savegrad() src/lbfgs_save.c:25-56
//   lbfgs()          src/lbfgs.c:26-181          (two-loop recursion)
//   modelupdate()    src/modelupdate.c:26-160
// The reference accumulates its dot products in float (and sums them across
// ranks with MPI_FLOAT); here every dot product and the L-BFGS work vector are
// FP64 and the reductions run in a fixed order (fixed grid, per-block tree,
// one final block), so results are deterministic. The elementwise model update
// keeps the reference's float/double expressions and is bit-identical to it.
#include "../../include/ifos_b200.h"

#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

namespace {

constexpr int RBLK = 296;  // reduction blocks: 2 per SM on a 148-SM B200
constexpr int RTHR = 256;
constexpr int MAXSUM = 6;

#define OCU(call)                                                                \
    do {                                                                         \
        cudaError_t _e = (call);                                                 \
        if (_e != cudaSuccess) {                                                 \
            o->err = std::string(#call) + ": " + cudaGetErrorString(_e);         \
            return _e == cudaErrorMemoryAllocation ? IFOSB_ENOMEM : IFOSB_ECUDA; \
        }                                                                        \
    } while (0)

// Block-wide sum of K values per thread into part[blockIdx.x*K + q] (fixed order).
template <int K>
__device__ void block_sums(double (&v)[K], double *part) {
    __shared__ double sh[K][RTHR / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < K; ++q) {
        double x = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[q][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0.0;
        for (int w = 0; w < RTHR / 32; ++w) s += sh[threadIdx.x][w];
        part[blockIdx.x * K + threadIdx.x] = s;
    }
}

// Final fixed-order sum of the RBLK partials of K sums: out[q].
__global__ void k_final(const double *part, int K, double *out) {
    const int q = threadIdx.x;
    if (q >= K) return;
    double s = 0.0;
    for (int b = 0; b < RBLK; ++b) s += part[b * K + q];
    out[q] = s;
}

// conjugategrad.c:59-74: the six sums of Mora's beta, and prior1..3 = grad.
__global__ void k_cg_sums(const float *g, float *prior, long long n, double *part) {
    double v[6] = {0, 0, 0, 0, 0, 0};
    for (long long i = blockIdx.x * (long long)RTHR + threadIdx.x; i < n; i += (long long)RBLK * RTHR) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double gc = g[c * n + i], pc = prior[c * n + i];
            v[2 * c] += gc * (gc - pc);
            v[2 * c + 1] += pc * pc;
            prior[c * n + i] = (float)gc;
        }
    }
    block_sums<6>(v, part);
}

// conjugategrad.c:79-91: beta = num/den where den != 0; the clamps test beta[0]
// only, so beta[0] ends in [0, 0.5] and beta[1], beta[2] are not clamped.
__global__ void k_cg_beta(const double *sums, int cdf, double *beta) {
    if (threadIdx.x != 0) return;
    double b[3] = {0.0, 0.0, 0.0};
    if (cdf == 0)
        for (int c = 0; c < 3; ++c)
            if (fabs(sums[2 * c + 1]) > 0.0) b[c] = sums[2 * c] / sums[2 * c + 1];
    if (b[0] < 0) b[0] = 0.0;
    if (b[0] > 0.5) b[0] = 0.5;
    beta[0] = b[0];
    beta[1] = b[1];
    beta[2] = b[2];
}

// conjugategrad.c:94-107: grad = prior4*beta + grad; prior4 = grad.
__global__ void k_cg_dir(float *g, float *prior46, const double *beta, long long n) {
    for (long long i = blockIdx.x * (long long)RTHR + threadIdx.x; i < n; i += (long long)RBLK * RTHR) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float d = (float)((double)prior46[c * n + i] * beta[c] + (double)g[c * n + i]);
            g[c * n + i] = d;
            prior46[c * n + i] = d;
        }
    }
}

// lbfgs.c:49-72: y_w = (previous gradient) - gradient; q = gradient.
__global__ void k_lb_start(const float *g, double *y, double *q, long long nn) {
    for (long long i = blockIdx.x * (long long)RTHR + threadIdx.x; i < nn; i += (long long)RBLK * RTHR) {
        const double gv = g[i];
        y[i] = y[i] - gv;
        q[i] = gv;
    }
}

__global__ void k_dot(const double *x, const double *y, long long nn, double *part) {
    double v[1] = {0.0};
    for (long long i = blockIdx.x * (long long)RTHR + threadIdx.x; i < nn; i += (long long)RBLK * RTHR)
        v[0] += x[i] * y[i];
    block_sums<1>(v, part);
}

__global__ void k_dot2(const double *x, const double *y, long long nn, double *part) {
    double v[2] = {0.0, 0.0};
    for (long long i = blockIdx.x * (long long)RTHR + threadIdx.x; i < nn; i += (long long)RBLK * RTHR) {
        v[0] += x[i] * y[i];
        v[1] += x[i] * x[i];
    }
    block_sums<2>(v, part);
}

// Scalars of the recursion, kept on the device so no host round trip sits
// between the passes: sc[0..B-1] rho_w (bfgsscale), sc[B..2B-1] alpha_w,
// sc[2B] h0, sc[2B+1] the coefficient of the current axpy, sc[2B+2..] raw sums.
enum { OP_SCALE, OP_ALPHA, OP_BETA };
__global__ void k_lb_scalar(const double *part, int K, double *sc, int B, int w, int op) {
    if (threadIdx.x != 0) return;
    double s[2] = {0.0, 0.0};
    for (int q = 0; q < K; ++q)
        for (int b = 0; b < RBLK; ++b) s[q] += part[b * K + q];
    if (op == OP_SCALE) {  // lbfgs.c:84-87: rho_w = 1/(y.s), h0 = (y.s)/(y.y)
        sc[w] = 1.0 / s[0];
        sc[2 * B] = s[0] / s[1];
        sc[2 * B + 2] = s[0];
        sc[2 * B + 3] = s[1];
    } else if (op == OP_ALPHA) {  // lbfgs.c:100-110: alpha_w = rho_w s_w.q; q -= alpha_w y_w
        sc[B + w] = sc[w] * s[0];
        sc[2 * B + 1] = -sc[B + w];
    } else {  // lbfgs.c:146-158: beta = rho_w y_w.q; q += s_w (alpha_w - beta)
        sc[2 * B + 1] = sc[B + w] - sc[w] * s[0];
    }
}

__global__ void k_axpy(double *q, const double *x, const double *coef, long long nn) {
    const double a = *coef;
    for (long long i = blockIdx.x * (long long)RTHR + threadIdx.x; i < nn; i += (long long)RBLK * RTHR)
        q[i] += a * x[i];
}

__global__ void k_scale(double *q, const double *h0, long long nn) {
    const double a = *h0;
    for (long long i = blockIdx.x * (long long)RTHR + threadIdx.x; i < nn; i += (long long)RBLK * RTHR)
        q[i] = q[i] * a;
}

// lbfgs.c:161-181: y_w' = gradient (kept for the next call); gradient = q.
__global__ void k_lb_end(float *g, double *y, const double *q, long long nn) {
    for (long long i = blockIdx.x * (long long)RTHR + threadIdx.x; i < nn; i += (long long)RBLK * RTHR) {
        y[i] = g[i];
        g[i] = (float)q[i];
    }
}

__global__ void k_copy_f2d(double *d, const float *s, long long nn) {
    for (long long i = blockIdx.x * (long long)RTHR + threadIdx.x; i < nn; i += (long long)RBLK * RTHR) d[i] = s[i];
}

// modelupdate.c:82-102: max |grad_c| (non-negative floats order like their bits).
__global__ void k_absmax(const float *g, long long n, unsigned int *mx) {
    unsigned int m[3] = {0u, 0u, 0u};
    for (long long i = blockIdx.x * (long long)RTHR + threadIdx.x; i < n; i += (long long)RBLK * RTHR)
#pragma unroll
        for (int c = 0; c < 3; ++c) m[c] = max(m[c], __float_as_uint(fabsf(g[c * n + i])));
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m[c] = max(m[c], __shfl_down_sync(0xffffffffu, m[c], o));
        if ((threadIdx.x & 31) == 0) atomicMax(mx + c, m[c]);
    }
}

// modelupdate.c:105-117: grad_c /= max_c when max0 > 0 and max1 > 0 (max2 = 0 -> 1).
__global__ void k_normalise(float *g, long long n, const unsigned int *mx) {
    const float m0 = __uint_as_float(mx[0]), m1 = __uint_as_float(mx[1]);
    float m2 = __uint_as_float(mx[2]);
    if (m2 == 0.0f) m2 = 1.0f;
    if (!(m0 > 0.0f && m1 > 0.0f)) return;
    for (long long i = blockIdx.x * (long long)RTHR + threadIdx.x; i < n; i += (long long)RBLK * RTHR) {
        g[i] = g[i] / m0;
        g[n + i] = g[n + i] / m1;
        g[2 * n + i] = g[2 * n + i] / m2;
    }
}

struct UpdArgs {
    int nx, ny, nz;
    float step, scale1, scale2, scale3, vp0, vs0, rho0;
    int numpar;
    double *s;  // L-BFGS model difference of this iteration, or nullptr
};

// modelupdate.c:119-157 with the reference's promotions: sqrt() of the float
// ratio in double, the float product step*scale*grad*V0 added in double and the
// sum stored as float; moduli from the new values in float.
__global__ void k_modelupdate(const float *g, float *rho, float *pi, float *u, UpdArgs a) {
    const long long n = (long long)a.nx * a.ny * a.nz;
    for (long long l = blockIdx.x * (long long)RTHR + threadIdx.x; l < n; l += (long long)RBLK * RTHR) {
        const int k = (int)(l % a.nz), i = (int)((l / a.nz) % a.nx), j = (int)(l / ((long long)a.nz * a.nx));
        const long long m = ((long long)(j + 1) * (a.nx + 2) + (i + 1)) * (a.nz + 2) + (k + 1);
        const float r = rho[m], p = pi[m], mu = u[m];
        const double vp_old = sqrt((double)(p / r)), vs_old = sqrt((double)(mu / r));
        const float vpnew = (float)(vp_old + (double)(a.step * a.scale1 * g[l] * a.vp0));
        const float vsnew = (float)(vs_old + (double)(a.step * a.scale2 * g[n + l] * a.vs0));
        const float rhonew = r + a.scale3 * a.step * g[2 * n + l] * a.rho0;
        if (a.s) {
            a.s[l] = ((double)vpnew - vp_old) / (double)a.vp0;
            if (a.numpar > 1) a.s[n + l] = ((double)vsnew - vs_old) / (double)a.vs0;
        }
        u[m] = rhonew * vsnew * vsnew;
        pi[m] = rhonew * vpnew * vpnew;
        rho[m] = rhonew;
    }
}

// precongrad.c:28-336 on one cell: the source and receiver damping factors
// (functions of the integer squared distance, tabulated on the host with the
// reference's double expressions) and the per-axis edge factors, multiplied in
// the reference's order; factors that are exactly 1.0f are skipped (exact).
struct PreArgs {
    int nx, ny, nz, type;
    int nsrc, ntr, ds, dr;            // table lengths: factors beyond them are 1.0f
    const int *src, *rec;             // [nsrc][3], [ntr][3]: x, y, z grid indices
    const float *lut_s, *lut_r;       // by squared distance
    const float *ty, *tx, *tz;        // [2][ny], [2][nx], [2][nz] edge factor pairs
};
__global__ void k_precon(float *g, PreArgs a) {
    const long long n = (long long)a.nx * a.ny * a.nz;
    for (long long l = blockIdx.x * (long long)RTHR + threadIdx.x; l < n; l += (long long)RBLK * RTHR) {
        const int k = (int)(l % a.nz) + 1, i = (int)((l / a.nz) % a.nx) + 1, j = (int)(l / ((long long)a.nz * a.nx)) + 1;
        float g0 = g[l], g1 = g[n + l], g2 = g[2 * n + l];
        if (a.type == 2)
            for (int q = 0; q < a.nsrc; ++q) {
                const int ex = i - a.src[3 * q], ey = j - a.src[3 * q + 1], ez = k - a.src[3 * q + 2];
                const int d2 = ey * ey + ex * ex + ez * ez;
                if (d2 < a.ds) {
                    const float G = a.lut_s[d2];
                    g0 = g0 * G; g1 = g1 * G; g2 = g2 * G;
                }
            }
        if (a.type == 1 || a.type == 2)
            for (int q = 0; q < a.ntr; ++q) {
                const int ex = i - a.rec[3 * q], ey = j - a.rec[3 * q + 1], ez = k - a.rec[3 * q + 2];
                const int d2 = ey * ey + ex * ex + ez * ez;
                if (d2 < a.dr) {
                    const float G = a.lut_r[d2];
                    g0 = g0 * G; g1 = g1 * G; g2 = g2 * G;
                }
            }
        const float y0 = a.ty[j - 1], y1 = a.ty[a.ny + j - 1];
        g0 = g0 * y0 * y1; g1 = g1 * y0 * y1; g2 = g2 * y0 * y1;
        const float x0 = a.tx[i - 1], x1 = a.tx[a.nx + i - 1];
        g0 = g0 * x0 * x1; g1 = g1 * x0 * x1; g2 = g2 * x0 * x1;
        const float z0 = a.tz[k - 1], z1 = a.tz[a.nz + k - 1];
        g0 = g0 * z0 * z1; g1 = g1 * z0 * z1; g2 = g2 * z0 * z1;
        g[l] = g0; g[n + l] = g1; g[2 * n + l] = g2;
    }
}

// constant_boundary (constant_boundary.c:27-222): one region of one phase.
// mode 0: copy from (j, a0, k); 1: copy from (j, i, a0); 2: average around
// (j, a0, k) with (j, a1, k); 3: average around (j, i, a0) with (j, i, a1). The
// averages are the reference's double sums divided by 8.0.
struct CbPhase {
    int j0, j1, i0, i1, k0, k1, mode, a0, a1;
};
__global__ void k_cbound(float *rho, float *pi, float *u, int nx, int nz, CbPhase ph) {
    const int ni = ph.i1 - ph.i0 + 1, nk = ph.k1 - ph.k0 + 1;
    const long long n = (long long)(ph.j1 - ph.j0 + 1) * ni * nk;
    const long long sj = (long long)(nx + 2) * (nz + 2), si = nz + 2;
    float *f[3] = {u, pi, rho};
    for (long long l = blockIdx.x * (long long)RTHR + threadIdx.x; l < n; l += (long long)RBLK * RTHR) {
        const int k = ph.k0 + (int)(l % nk), i = ph.i0 + (int)((l / nk) % ni), j = ph.j0 + (int)(l / ((long long)nk * ni));
        const long long d = j * sj + i * si + k;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            float *a = f[q];
            if (ph.mode == 0) {
                a[d] = a[j * sj + ph.a0 * si + k];
            } else if (ph.mode == 1) {
                a[d] = a[j * sj + i * si + ph.a0];
            } else if (ph.mode == 2) {
                const long long c = j * sj + ph.a0 * si + k;
                a[d] = (float)((3.0 * a[c] + a[c - sj] + a[c + sj] + a[c - 1] + a[c + 1] + a[j * sj + ph.a1 * si + k]) / 8.0);
            } else {
                const long long c = j * sj + i * si + ph.a0;
                a[d] = (float)((3.0 * a[c] + a[c - sj] + a[c + sj] + a[c - si] + a[c + si] + a[j * sj + i * si + ph.a1]) / 8.0);
            }
        }
    }
}

}  // namespace

struct ifosb_optim {
    int nx = 0, ny = 0, nz = 0, numpar = 1, bfgsnum = 0;
    long long n = 0;
    float *d_grad = nullptr;    // [3][n]
    float *d_prior = nullptr;   // [6][n] gradprior1..6
    double *d_s = nullptr;      // [bfgsnum][numpar*n] bfgsmod
    double *d_y = nullptr;      // [bfgsnum][numpar*n] bfgsgrad
    double *d_q = nullptr;      // [numpar*n]
    double *d_part = nullptr;   // [RBLK*MAXSUM]
    double *d_sc = nullptr;     // scalars of the recursion
    double *d_out = nullptr;    // [MAXSUM]
    unsigned int *d_max = nullptr;
    float *d_model = nullptr;   // [3][(ny+2)(nx+2)(nz+2)] rho, pi, u
    cudaStream_t stream = nullptr;
    std::string err;
};

static int ofail(ifosb_optim *o, int code, const char *msg) {
    if (o) o->err = msg;
    return code;
}

extern "C" int ifosb_optim_create(int nx, int ny, int nz, int numpar, int bfgsnum, ifosb_optim **out) {
    if (!out || nx < 1 || ny < 1 || nz < 1 || numpar < 1 || numpar > 2 || bfgsnum < 0) return IFOSB_EARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return IFOSB_ENODEV;
    }
    ifosb_optim *o = new ifosb_optim;
    o->nx = nx;
    o->ny = ny;
    o->nz = nz;
    o->numpar = numpar;
    o->bfgsnum = bfgsnum;
    o->n = (long long)nx * ny * nz;
    const long long n = o->n, nn = (long long)numpar * n, mg = (long long)(nx + 2) * (ny + 2) * (nz + 2);
    auto alloc = [&](void **p, size_t bytes) { return cudaMalloc(p, bytes) == cudaSuccess; };
    bool ok = alloc((void **)&o->d_grad, sizeof(float) * 3 * n) && alloc((void **)&o->d_prior, sizeof(float) * 6 * n) &&
              alloc((void **)&o->d_part, sizeof(double) * RBLK * MAXSUM) &&
              alloc((void **)&o->d_sc, sizeof(double) * (2 * bfgsnum + 8)) &&
              alloc((void **)&o->d_out, sizeof(double) * MAXSUM) && alloc((void **)&o->d_max, sizeof(unsigned) * 3) &&
              alloc((void **)&o->d_model, sizeof(float) * 3 * mg);
    if (ok && bfgsnum > 0)
        ok = alloc((void **)&o->d_s, sizeof(double) * bfgsnum * nn) && alloc((void **)&o->d_y, sizeof(double) * bfgsnum * nn) &&
             alloc((void **)&o->d_q, sizeof(double) * nn);
    if (ok) ok = cudaStreamCreateWithFlags(&o->stream, cudaStreamNonBlocking) == cudaSuccess;
    if (ok) ok = cudaMemsetAsync(o->d_prior, 0, sizeof(float) * 6 * n, o->stream) == cudaSuccess &&
                 cudaMemsetAsync(o->d_sc, 0, sizeof(double) * (2 * bfgsnum + 8), o->stream) == cudaSuccess;
    if (ok && bfgsnum > 0)
        ok = cudaMemsetAsync(o->d_s, 0, sizeof(double) * bfgsnum * nn, o->stream) == cudaSuccess &&
             cudaMemsetAsync(o->d_y, 0, sizeof(double) * bfgsnum * nn, o->stream) == cudaSuccess;
    if (ok) ok = cudaStreamSynchronize(o->stream) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        ifosb_optim_destroy(o);
        return IFOSB_ENOMEM;
    }
    *out = o;
    return IFOSB_OK;
}

extern "C" void ifosb_optim_destroy(ifosb_optim *o) {
    if (!o) return;
    for (void *p : {(void *)o->d_grad, (void *)o->d_prior, (void *)o->d_s, (void *)o->d_y, (void *)o->d_q,
                    (void *)o->d_part, (void *)o->d_sc, (void *)o->d_out, (void *)o->d_max, (void *)o->d_model})
        if (p) cudaFree(p);
    if (o->stream) cudaStreamDestroy(o->stream);
    delete o;
}

extern "C" const char *ifosb_optim_last_error(const ifosb_optim *o) { return o ? o->err.c_str() : "no optimiser"; }

static int finish(ifosb_optim *o) {
    OCU(cudaGetLastError());
    OCU(cudaStreamSynchronize(o->stream));
    return IFOSB_OK;
}

extern "C" int ifosb_conjugate(ifosb_optim *o, float *grad, int cdf, double *beta) {
    if (!o || !grad) return IFOSB_EARG;
    const long long n = o->n;
    double *d_beta = o->d_sc + 2 * o->bfgsnum + 4;
    OCU(cudaMemcpyAsync(o->d_grad, grad, sizeof(float) * 3 * n, cudaMemcpyDefault, o->stream));
    if (cdf == 1) {  // conjugategrad.c:43-56: both priors start from this gradient
        OCU(cudaMemcpyAsync(o->d_prior, o->d_grad, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, o->stream));
        OCU(cudaMemcpyAsync(o->d_prior + 3 * n, o->d_grad, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, o->stream));
    } else {
        k_cg_sums<<<RBLK, RTHR, 0, o->stream>>>(o->d_grad, o->d_prior, n, o->d_part);
        k_final<<<1, 32, 0, o->stream>>>(o->d_part, 6, o->d_out);
        k_cg_beta<<<1, 32, 0, o->stream>>>(o->d_out, cdf, d_beta);
        k_cg_dir<<<RBLK, RTHR, 0, o->stream>>>(o->d_grad, o->d_prior + 3 * n, d_beta, n);
        OCU(cudaMemcpyAsync(grad, o->d_grad, sizeof(float) * 3 * n, cudaMemcpyDefault, o->stream));
    }
    int rc = finish(o);
    if (rc) return rc;
    if (beta) {
        if (cdf == 1) {
            beta[0] = beta[1] = beta[2] = 0.0;
        } else {
            OCU(cudaMemcpy(beta, d_beta, sizeof(double) * 3, cudaMemcpyDeviceToHost));
        }
    }
    return IFOSB_OK;
}

static int slot(int v, int B) {
    const int w = v % B;
    return w == 0 ? B : w;  // 1-based as the reference's bfgs matrices
}

extern "C" int ifosb_lbfgs_savegrad(ifosb_optim *o, const float *grad) {
    if (!o || !grad) return IFOSB_EARG;
    if (o->bfgsnum < 1) return ofail(o, IFOSB_ESTATE, "optimiser created without L-BFGS history");
    const long long nn = (long long)o->numpar * o->n;
    OCU(cudaMemcpyAsync(o->d_grad, grad, sizeof(float) * nn, cudaMemcpyDefault, o->stream));
    k_copy_f2d<<<RBLK, RTHR, 0, o->stream>>>(o->d_y, o->d_grad, nn);  // lbfgs_save.c:31-52: slot 1
    return finish(o);
}

extern "C" int ifosb_lbfgs(ifosb_optim *o, float *grad, int it_group) {
    if (!o || !grad || it_group < 2) return IFOSB_EARG;
    const int B = o->bfgsnum;
    if (B < 1) return ofail(o, IFOSB_ESTATE, "optimiser created without L-BFGS history");
    const long long nn = (long long)o->numpar * o->n;
    double *sc = o->d_sc;
    int m = it_group - B;
    if (m < 1) m = 1;
    auto S = [&](int w) { return o->d_s + (long long)(w - 1) * nn; };
    auto Y = [&](int w) { return o->d_y + (long long)(w - 1) * nn; };
    OCU(cudaMemcpyAsync(o->d_grad, grad, sizeof(float) * nn, cudaMemcpyDefault, o->stream));
    int w = slot(it_group - 1, B);
    k_lb_start<<<RBLK, RTHR, 0, o->stream>>>(o->d_grad, Y(w), o->d_q, nn);
    k_dot2<<<RBLK, RTHR, 0, o->stream>>>(Y(w), S(w), nn, o->d_part);
    k_lb_scalar<<<1, 32, 0, o->stream>>>(o->d_part, 2, sc, B, w - 1, OP_SCALE);
    for (int v = it_group - 1; v >= m; --v) {
        w = slot(v, B);
        k_dot<<<RBLK, RTHR, 0, o->stream>>>(S(w), o->d_q, nn, o->d_part);
        k_lb_scalar<<<1, 32, 0, o->stream>>>(o->d_part, 1, sc, B, w - 1, OP_ALPHA);
        k_axpy<<<RBLK, RTHR, 0, o->stream>>>(o->d_q, Y(w), sc + 2 * B + 1, nn);
    }
    k_scale<<<RBLK, RTHR, 0, o->stream>>>(o->d_q, sc + 2 * B, nn);
    for (int v = m; v <= it_group - 1; ++v) {
        w = slot(v, B);
        k_dot<<<RBLK, RTHR, 0, o->stream>>>(Y(w), o->d_q, nn, o->d_part);
        k_lb_scalar<<<1, 32, 0, o->stream>>>(o->d_part, 1, sc, B, w - 1, OP_BETA);
        k_axpy<<<RBLK, RTHR, 0, o->stream>>>(o->d_q, S(w), sc + 2 * B + 1, nn);
    }
    k_lb_end<<<RBLK, RTHR, 0, o->stream>>>(o->d_grad, Y(slot(it_group, B)), o->d_q, nn);
    OCU(cudaMemcpyAsync(grad, o->d_grad, sizeof(float) * nn, cudaMemcpyDefault, o->stream));
    return finish(o);
}

extern "C" int ifosb_modelupdate(ifosb_optim *o, float *grad, float *rho, float *pi, float *u, float step,
                                 const float *weight, float vp0, float vs0, float rho0, int lbfgs, int it_group) {
    if (!o || !grad || !rho || !pi || !u || !weight) return IFOSB_EARG;
    if (lbfgs && o->bfgsnum < 1) return ofail(o, IFOSB_ESTATE, "optimiser created without L-BFGS history");
    const long long n = o->n, mg = (long long)(o->nx + 2) * (o->ny + 2) * (o->nz + 2);
    float *drho = o->d_model, *dpi = o->d_model + mg, *du = o->d_model + 2 * mg;
    OCU(cudaMemcpyAsync(o->d_grad, grad, sizeof(float) * 3 * n, cudaMemcpyDefault, o->stream));
    OCU(cudaMemcpyAsync(drho, rho, sizeof(float) * mg, cudaMemcpyDefault, o->stream));
    OCU(cudaMemcpyAsync(dpi, pi, sizeof(float) * mg, cudaMemcpyDefault, o->stream));
    OCU(cudaMemcpyAsync(du, u, sizeof(float) * mg, cudaMemcpyDefault, o->stream));
    if (!lbfgs) {
        OCU(cudaMemsetAsync(o->d_max, 0, sizeof(unsigned) * 3, o->stream));
        k_absmax<<<RBLK, RTHR, 0, o->stream>>>(o->d_grad, n, o->d_max);
        k_normalise<<<RBLK, RTHR, 0, o->stream>>>(o->d_grad, n, o->d_max);
    }
    UpdArgs a;
    a.nx = o->nx;
    a.ny = o->ny;
    a.nz = o->nz;
    a.step = step;
    a.scale1 = weight[0];
    a.scale2 = weight[1];
    a.scale3 = weight[2];
    a.vp0 = vp0;
    a.vs0 = vs0;
    a.rho0 = rho0;
    a.numpar = o->numpar;
    a.s = lbfgs ? o->d_s + (long long)(slot(it_group, o->bfgsnum) - 1) * o->numpar * n : nullptr;
    k_modelupdate<<<RBLK, RTHR, 0, o->stream>>>(o->d_grad, drho, dpi, du, a);
    if (!lbfgs) OCU(cudaMemcpyAsync(grad, o->d_grad, sizeof(float) * 3 * n, cudaMemcpyDefault, o->stream));
    OCU(cudaMemcpyAsync(rho, drho, sizeof(float) * mg, cudaMemcpyDefault, o->stream));
    OCU(cudaMemcpyAsync(pi, dpi, sizeof(float) * mg, cudaMemcpyDefault, o->stream));
    OCU(cudaMemcpyAsync(u, du, sizeof(float) * mg, cudaMemcpyDefault, o->stream));
    return finish(o);
}

extern "C" int ifosb_lbfgs_history(const ifosb_optim *o, double *s, double *y, double *scale) {
    if (!o || o->bfgsnum < 1) return IFOSB_EARG;
    const size_t nn = (size_t)o->numpar * o->n * o->bfgsnum;
    if (s && cudaMemcpy(s, o->d_s, sizeof(double) * nn, cudaMemcpyDeviceToHost) != cudaSuccess) return IFOSB_ECUDA;
    if (y && cudaMemcpy(y, o->d_y, sizeof(double) * nn, cudaMemcpyDeviceToHost) != cudaSuccess) return IFOSB_ECUDA;
    if (scale && cudaMemcpy(scale, o->d_sc, sizeof(double) * o->bfgsnum, cudaMemcpyDeviceToHost) != cudaSuccess)
        return IFOSB_ECUDA;
    return IFOSB_OK;
}

// Host side of precon_grad: the factor tables, computed with the reference's
// expressions (float variables, double exp and division).
static float damp_rec(int d2) {  // precongrad.c:53-58: 1/(1+1000 exp(-0.7 r^2))
    const float r = (float)sqrt((double)d2);
    return (float)(1 / (1 + 1000 * exp(-0.7 * r * r)));
}
static float damp_src(int d2) {  // precongrad.c:133-143: 1/(1+1000 exp(-0.7 r))
    const float r = (float)sqrt((double)d2);
    return (float)(1 / (1 + 1000 * exp(-0.7 * r)));
}
static float damp_edge(int x) {  // 1/(1+2000 exp(-0.6 r)), r = x
    const float r = (float)(x * 1.0);
    return (float)(1 / (1 + 2000 * exp(-0.6 * r)));
}
// Table of f(d2) up to the first d2 from which f is exactly 1.0f (checked on to
// 4 times that length); returns the length.
static std::vector<float> damp_table(float (*f)(int)) {
    std::vector<float> t;
    int d2 = 0;
    for (; d2 < (1 << 22); ++d2) {
        const float v = f(d2);
        if (v == 1.0f) {
            bool ones = true;
            for (int q = d2; q < 4 * d2 + 64 && ones; ++q) ones = f(q) == 1.0f;
            if (ones) break;
        }
        t.push_back(v);
    }
    return t;
}

extern "C" int ifosb_precon_grad(ifosb_optim *o, float *grad, int damptype, int free_surf, int fw, float dx, float dy,
                                 float dz, int nsrc, const float *srcpos, int ntr, const int *recpos) {
    if (!o || !grad || damptype < 0 || damptype > 3 || nsrc < 0 || ntr < 0) return IFOSB_EARG;
    if ((nsrc > 0 && !srcpos) || (ntr > 0 && !recpos)) return IFOSB_EARG;
    const int NX = o->nx, NY = o->ny, NZ = o->nz;
    const long long n = o->n;
    // edge factor pairs per axis; types 0 and 3 read ii, jj, kk, which those
    // branches never assign (they stay 0, precongrad.c:34): constant tables
    std::vector<float> ty(2 * NY), tx(2 * NX), tz(2 * NZ);
    const bool pos = damptype == 1 || damptype == 2;
    for (int j = 1; j <= NY; ++j) {
        const int jj = pos ? j : 0;
        float a, b;
        if (damptype == 3) {  // precongrad.c:226-234
            const int sh = fw + 40, rh = fw + 40;
            float r = (float)((jj - sh) * 1.0);
            a = r < 0 ? 0.0f : (float)(1 / (1 + 1000 * exp(-0.7 * r * r)));
            r = (float)((NY - jj - rh) * 1.0);
            b = r < 0 ? 0.0f : (float)(1 / (1 + 1000 * exp(-0.7 * r)));
        } else {
            a = free_surf ? 0.0f : damp_edge(jj);
            b = damp_edge(NY - jj);
        }
        ty[j - 1] = a;
        ty[NY + j - 1] = b;
    }
    for (int i = 1; i <= NX; ++i) {
        const int ii = pos ? i : 0;
        tx[i - 1] = damp_edge(ii);  // r = ii >= 0, so type 3's r < 0 test never fires
        tx[NX + i - 1] = (NX - ii) < 0 ? 0.0f : damp_edge(NX - ii);
    }
    for (int k = 1; k <= NZ; ++k) {
        const int kk = pos ? k : 0;
        tz[k - 1] = damp_edge(kk);
        tz[NZ + k - 1] = (NZ - kk) < 0 ? 0.0f : damp_edge(NZ - kk);
    }
    static const std::vector<float> lut_r = damp_table(damp_rec), lut_s = damp_table(damp_src);
    std::vector<int> src(3 * (size_t)nsrc), rec(3 * (size_t)ntr);
    for (int q = 0; q < nsrc; ++q) {  // iround(srcpos/DX) (fd.h:35) of the positions in metres
        src[3 * q] = (int)floor(srcpos[3 * q] / dx + 0.5);
        src[3 * q + 1] = (int)floor(srcpos[3 * q + 1] / dy + 0.5);
        src[3 * q + 2] = (int)floor(srcpos[3 * q + 2] / dz + 0.5);
    }
    for (int q = 0; q < 3 * ntr; ++q) rec[q] = recpos[q];
    // one device block for all tables
    const size_t nf = ty.size() + tx.size() + tz.size() + lut_r.size() + lut_s.size();
    const size_t ni = src.size() + rec.size();
    float *dt = nullptr;
    int *di = nullptr;
    OCU(cudaMalloc(&dt, sizeof(float) * nf));
    if (ni) {
        cudaError_t ce = cudaMalloc(&di, sizeof(int) * ni);
        if (ce != cudaSuccess) {
            cudaFree(dt);
            OCU(ce);
        }
    }
    std::vector<float> hf;
    hf.reserve(nf);
    hf.insert(hf.end(), ty.begin(), ty.end());
    hf.insert(hf.end(), tx.begin(), tx.end());
    hf.insert(hf.end(), tz.begin(), tz.end());
    hf.insert(hf.end(), lut_r.begin(), lut_r.end());
    hf.insert(hf.end(), lut_s.begin(), lut_s.end());
    std::vector<int> hi(src);
    hi.insert(hi.end(), rec.begin(), rec.end());
    PreArgs a;
    a.nx = NX; a.ny = NY; a.nz = NZ; a.type = damptype;
    a.nsrc = nsrc; a.ntr = ntr;
    a.dr = (int)lut_r.size(); a.ds = (int)lut_s.size();
    a.ty = dt; a.tx = dt + ty.size(); a.tz = a.tx + tx.size();
    a.lut_r = a.tz + tz.size(); a.lut_s = a.lut_r + lut_r.size();
    a.src = di; a.rec = di ? di + src.size() : nullptr;
    int rc = IFOSB_OK;
    cudaError_t ce = cudaMemcpyAsync(dt, hf.data(), sizeof(float) * nf, cudaMemcpyHostToDevice, o->stream);
    if (ce == cudaSuccess && ni) ce = cudaMemcpyAsync(di, hi.data(), sizeof(int) * ni, cudaMemcpyHostToDevice, o->stream);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(o->d_grad, grad, sizeof(float) * 3 * n, cudaMemcpyDefault, o->stream);
    if (ce == cudaSuccess) {
        k_precon<<<RBLK, RTHR, 0, o->stream>>>(o->d_grad, a);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(grad, o->d_grad, sizeof(float) * 3 * n, cudaMemcpyDefault, o->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(o->stream);
    if (ce != cudaSuccess) {
        o->err = std::string("precon_grad: ") + cudaGetErrorString(ce);
        rc = IFOSB_ECUDA;
    }
    cudaFree(dt);
    if (di) cudaFree(di);
    return rc;
}

extern "C" int ifosb_constant_boundary(ifosb_optim *o, float *rho, float *pi, float *u, int fw) {
    if (!o || !rho || !pi || !u || fw < 1) return IFOSB_EARG;
    const int NX = o->nx, NY = o->ny, NZ = o->nz, dist = 4;
    if (NX < 2 * fw + dist + 2 || NZ < 2 * fw + dist + 2 || NY < 3) return ofail(o, IFOSB_EARG, "grid too small");
    // one rank: the interior bounds of CPML_ini_elastic (CPML_ini_elastic.c:28-54)
    const int nx1 = fw + 1, nx2 = NX - fw, nz1 = fw + 1, nz2 = NZ - fw;
    const int a = fw + 1 + dist, b = fw + 2 + dist, c = nx2 - dist, cz = nz2 - dist;
    // the reference's loops in their order; later faces read cells earlier ones rewrote
    const CbPhase ph[] = {
        {1, 1, 1, fw + dist, nz1, nz2, 0, a, 0},                      // x front, top row
        {NY, NY, 1, fw + dist, nz1, nz2, 0, a, 0},                    // x front, bottom row
        {2, NY - 1, 1, fw + dist, nz1, nz2, 2, a, b},                 // x front
        {1, 1, nx2 + 1 - dist, nx2 + fw, nz1, nz2, 0, c, 0},          // x back, top row
        {NY, NY, nx2 + 1 - dist, nx2 + fw, nz1, nz2, 0, c, 0},        // x back, bottom row
        {2, NY - 1, nx2 + 1 - dist, nx2 + fw, nz1, nz2, 2, c, c - 1}, // x back
        {1, 1, 1, NX, 1, fw + dist, 1, a, 0},                         // z front, top row
        {NY, NY, 1, NX, 1, fw + dist, 1, a, 0},                       // z front, bottom row
        {2, NY - 1, 1, fw + dist, 1, fw + dist, 1, a, 0},             // z front, x-front corner
        {2, NY - 1, nx2 + 1 - dist, nx2 + fw, 1, fw + dist, 1, a, 0}, // z front, x-back corner
        {2, NY - 1, nx1, nx2, 1, fw + dist, 3, a, b},                 // z front
        {1, 1, 1, NX, nz2 + 1 - dist, nz2 + fw, 1, cz, 0},            // z back, top row
        {NY, NY, 1, NX, nz2 + 1 - dist, nz2 + fw, 1, cz, 0},          // z back, bottom row
        {2, NY - 1, 1, fw + dist, nz2 + 1 - dist, nz2 + fw, 1, cz, 0},
        {2, NY - 1, nx2 + 1 - dist, nx2 + fw, nz2 + 1 - dist, nz2 + fw, 1, cz, 0},
        {2, NY - 1, nx1, nx2, nz2 + 1 - dist, nz2 + fw, 3, cz, cz - 1}, // z back
    };
    const long long mg = (long long)(NX + 2) * (NY + 2) * (NZ + 2);
    float *drho = o->d_model, *dpi = o->d_model + mg, *du = o->d_model + 2 * mg;
    OCU(cudaMemcpyAsync(drho, rho, sizeof(float) * mg, cudaMemcpyDefault, o->stream));
    OCU(cudaMemcpyAsync(dpi, pi, sizeof(float) * mg, cudaMemcpyDefault, o->stream));
    OCU(cudaMemcpyAsync(du, u, sizeof(float) * mg, cudaMemcpyDefault, o->stream));
    for (const CbPhase &q : ph) k_cbound<<<RBLK, RTHR, 0, o->stream>>>(drho, dpi, du, NX, NZ, q);
    OCU(cudaMemcpyAsync(rho, drho, sizeof(float) * mg, cudaMemcpyDefault, o->stream));
    OCU(cudaMemcpyAsync(pi, dpi, sizeof(float) * mg, cudaMemcpyDefault, o->stream));
    OCU(cudaMemcpyAsync(u, du, sizeof(float) * mg, cudaMemcpyDefault, o->stream));
    return finish(o);
}

// ---------------------------------------------------------------------------
// hess_apply (hess_apply.c:25-79): with L-BFGS the gradients are first scaled by
// VP0, VS0, RHO0; then grad_c /= (hess_c + WATER_HESS[c]). The water level the
// reference derives from the Hessian's log-average is printed there and never
// used, so it is not formed here.
__global__ void k_hess_apply(float *g, const float *h, long long n, float w0, float w1, float w2, int lbfgs, float vp0,
                             float vs0, float rho0) {
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
        float g1 = g[m], g2 = g[n + m], g3 = g[2 * n + m];
        if (lbfgs) {
            g1 = g1 * vp0;
            g2 = g2 * vs0;
            g3 = g3 * rho0;
        }
        g[m] = g1 / (h[m] + w0);
        g[n + m] = g2 / (h[n + m] + w1);
        g[2 * n + m] = g3 / (h[2 * n + m] + w2);
    }
}

extern "C" int ifosb_hess_apply(ifosb_optim *o, float *grad, const float *hess, const float *water, int lbfgs,
                                float vp0, float vs0, float rho0) {
    if (!o || !grad || !hess || !water) return IFOSB_EARG;
    const long long n = o->n;
    float *dh = nullptr;
    OCU(cudaMalloc(&dh, sizeof(float) * 3 * n));
    cudaError_t ce = cudaMemcpyAsync(dh, hess, sizeof(float) * 3 * n, cudaMemcpyDefault, o->stream);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(o->d_grad, grad, sizeof(float) * 3 * n, cudaMemcpyDefault, o->stream);
    if (ce == cudaSuccess) {
        k_hess_apply<<<RBLK, RTHR, 0, o->stream>>>(o->d_grad, dh, n, water[0], water[1], water[2], lbfgs ? 1 : 0, vp0,
                                                   vs0, rho0);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(grad, o->d_grad, sizeof(float) * 3 * n, cudaMemcpyDefault, o->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(o->stream);
    cudaFree(dh);
    if (ce != cudaSuccess) {
        o->err = std::string("hess_apply: ") + cudaGetErrorString(ce);
        return IFOSB_ECUDA;
    }
    return IFOSB_OK;
}

// ---------------------------------------------------------------------------
// Model resampling between the grids of a multiscale run (coarse to fine, e.g.
// 256x256x160 at 2 m to 512x512x320 at 1 m). The reference has no such step, so
// the rule is our own and plain: cell (i, j, k) of a grid sits at (i dx, j dy,
// k dz), as source and receiver positions do in the reference (index x spacing).
// A destination cell takes the trilinear interpolation of the source grid at its
// position, clamped to the source's first/last cell outside it (constant
// extrapolation), computed in double and rounded once to float.
struct ResampleArgs {
    const float *src;
    float *dst;
    int nx, ny, nz, mx, my, mz;
    double rx, ry, rz;  // destination spacing / source spacing, per axis
};

__device__ __forceinline__ void axis_weights(int i, double r, int n, int &i0, int &i1, double &w) {
    const double u = (double)i * r;  // position in source index units (1-based)
    if (u <= 1.0) { i0 = i1 = 1; w = 0.0; return; }
    if (u >= (double)n) { i0 = i1 = n; w = 0.0; return; }
    i0 = (int)floor(u);
    i1 = i0 + 1;
    w = u - (double)i0;
}

__global__ void k_resample(ResampleArgs a) {
    const long long total = (long long)a.mx * a.my * a.mz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(q % a.mz) + 1, i = (int)((q / a.mz) % a.mx) + 1, j = (int)(q / ((long long)a.mz * a.mx)) + 1;
        int x0, x1, y0, y1, z0, z1;
        double wx, wy, wz;
        axis_weights(i, a.rx, a.nx, x0, x1, wx);
        axis_weights(j, a.ry, a.ny, y0, y1, wy);
        axis_weights(k, a.rz, a.nz, z0, z1, wz);
        auto S = [&](int jj, int ii, int kk) {
            return (double)a.src[((long long)(jj - 1) * a.nx + (ii - 1)) * a.nz + (kk - 1)];
        };
        const double c00 = S(y0, x0, z0) * (1.0 - wz) + S(y0, x0, z1) * wz;
        const double c01 = S(y0, x1, z0) * (1.0 - wz) + S(y0, x1, z1) * wz;
        const double c10 = S(y1, x0, z0) * (1.0 - wz) + S(y1, x0, z1) * wz;
        const double c11 = S(y1, x1, z0) * (1.0 - wz) + S(y1, x1, z1) * wz;
        const double c0 = c00 * (1.0 - wx) + c01 * wx;
        const double c1 = c10 * (1.0 - wx) + c11 * wx;
        a.dst[q] = (float)(c0 * (1.0 - wy) + c1 * wy);
    }
}

extern "C" int ifosb_resample(const float *src, int nx, int ny, int nz, float dx, float dy, float dz, float *dst,
                              int mx, int my, int mz, float ex, float ey, float ez) {
    if (!src || !dst || nx < 1 || ny < 1 || nz < 1 || mx < 1 || my < 1 || mz < 1) return IFOSB_EARG;
    if (!(dx > 0.f && dy > 0.f && dz > 0.f && ex > 0.f && ey > 0.f && ez > 0.f)) return IFOSB_EARG;
    int dev = 0;
    if (cudaGetDeviceCount(&dev) != cudaSuccess || dev == 0) {
        cudaGetLastError();
        return IFOSB_ENODEV;
    }
    const size_t ns = (size_t)nx * ny * nz, nd = (size_t)mx * my * mz;
    float *ds = nullptr, *dd = nullptr;
    cudaError_t ce = cudaMalloc(&ds, ns * sizeof(float));
    if (ce == cudaSuccess) ce = cudaMalloc(&dd, nd * sizeof(float));
    if (ce == cudaSuccess) ce = cudaMemcpy(ds, src, ns * sizeof(float), cudaMemcpyDefault);
    if (ce == cudaSuccess) {
        ResampleArgs a{ds, dd, nx, ny, nz, mx, my, mz, (double)ex / (double)dx, (double)ey / (double)dy,
                       (double)ez / (double)dz};
        k_resample<<<RBLK, RTHR>>>(a);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaMemcpy(dst, dd, nd * sizeof(float), cudaMemcpyDefault);
    if (ds) cudaFree(ds);
    if (dd) cudaFree(dd);
    if (ce != cudaSuccess) {
        cudaGetLastError();
        return ce == cudaErrorMemoryAllocation ? IFOSB_ENOMEM : IFOSB_ECUDA;
    }
    return IFOSB_OK;
}
