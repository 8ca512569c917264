// C-ABI implementation of the B200 wavefield engine (include/ifos_b200.h).
//
// One engine = one device-resident problem: the model (shared by all shots),
// per-shot wavefield state, PML memory, DFT accumulators and traces for a
// batch of up to max_shots shots, and the accumulated gradient. The time loops
// run as two kernels per step (velocity; stress + source + DFT + surface +
// receivers), captured once into a CUDA graph per batch shape and direction
// and replayed on later calls.
#include "../../include/ifos_b200.h"
#include "ifosb_kernels.cuh"
#include "ifosb_tma.cuh"
#include "ifosb_vjp.cuh"

#include <cudaTypedefs.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

using namespace ifosb;

namespace {

constexpr int DEFAULT_CY = 8;

struct GraphCache {
    cudaGraphExec_t exec = nullptr;
    std::vector<unsigned char> key;
    long long used = 0;  // last use, for replacing the least recently used
};
// Time-loop graphs kept per direction: a run of batches alternates between a few
// shapes (full batches and a shorter last one), and each keeps its own graph.
constexpr int GRAPHS_PER_DIRECTION = 4;
struct GraphSet {
    GraphCache g[GRAPHS_PER_DIRECTION];
    long long tick = 0;
};

struct HostPt {
    int s, j, i, k, kind, row;
};

}  // namespace

struct ifosb_engine {
    ifosb_params p{};
    Geo g{};
    Slabs sl{};
    int max_shots = 0, max_nf = 0;
    cudaStream_t stream = nullptr;
    float b1 = 0.f, b2 = 0.f;
    float eta[MAXMECH] = {0.f, 0.f, 0.f, 0.f};
    // device memory
    float *d_state = nullptr;  long long st_shot = 0;
    float *d_psi = nullptr;    long long psi_shot = 0;
    float *d_model = nullptr;  float *d_rho_w = nullptr;
    float *d_dftf = nullptr, *d_dftb = nullptr; long long dft_shot = 0;
    float *d_grad = nullptr;   double *d_grad64 = nullptr;
    double *d_gradq = nullptr;  // viscoelastic: FP64 gradients with respect to taup and taus
    int *d_err = nullptr;
    // receivers and traces
    int ntr = 0, ns = 0;
    std::vector<int> rec;
    float *d_sec = nullptr, *d_diff = nullptr, *d_obs = nullptr;
    int seismo = 1;            // SEISMO: 1 vx, vy, vz; 2 p; 3 div, curl; 4 all six
    float *d_sec2 = nullptr;   // [max_shots][3][ntr][ns]: p, div, curl (SEISMO 2-4)
    double *d_part = nullptr, *d_misfit = nullptr;
    float *d_l2 = nullptr;
    // frequencies
    int nf = 0, ntast = 1;
    std::vector<float> finv;
    double *d_trig_f = nullptr, *d_trig_b = nullptr;
    // point lists (grow-only buffers)
    int *d_voff = nullptr, *d_soff = nullptr; size_t cap_voff = 0, cap_soff = 0;
    Pt *d_vpts = nullptr, *d_spts = nullptr;  size_t cap_vpts = 0, cap_spts = 0;
    float *d_amp = nullptr;                   size_t cap_amp = 0;
    // status
    int nshots = 0;
    bool have_model = false, have_cpml = false, fwd_ok = false, res_ok = false, adj_ok = false;
    int launch_mode = 0;
    long long launches = 0;
    long long dev_bytes = 0;
    GraphSet gfwd, gadj;
    // kernel timing
    int profile = 0;
    double t_vel_ms = 0.0, t_str_ms = 0.0;
    int t_steps = 0;
    std::vector<cudaEvent_t> events;
    cudaStream_t own_stream = nullptr;
    // launch shapes picked by ifosb_autotune per batch size: y planes per CTA chunk
    // and the L2 prefetch distance; nt_limit > 0 shortens the time loop while tuning
    struct Shape {
        int cyv, l2v, cys, l2s;  // velocity and stress kernels: y planes per chunk, L2 prefetch
    };
    std::map<int, Shape> tuned;
    int vby = 8;  // rows per tile of the velocity kernel
    int nt_limit = 0;
    long long captures = 0;  // time-loop graphs captured (a replay reuses one)
    float *d_mstage = nullptr;  // ifosb_set_model's staging of the raw model (5 ghosted fields)
    float *d_smod = nullptr;    // free-surface moduli of plane j=1 [2][NX][NZ] (ifosb_set_surface_moduli)
    bool smod_on = false;
    // approximate Hessian: receivers' Green's-function DFT fields and the accumulated diagonal
    float *d_green = nullptr; int ngreen = 0, cap_green = 0;
    float *d_gsig = nullptr;   // [max_shots][3][NT] injection traces of a Green's-function batch
    float *d_hess = nullptr;   // [3][NY][NX][NZ]
    bool hess_fwd = false;     // d_dftf holds a forward batch not yet added to the Hessian
    // time-domain gradient mode: the last forward batch's point lists (host) and
    // device copies of its own, so the recomputation never shares the adjoint's
    std::vector<HostPt> td_vp, td_sp;
    std::vector<float> td_amp;
    int *d_voff_t = nullptr, *d_soff_t = nullptr, *d_voff_a = nullptr;
    size_t cap_voff_t = 0, cap_soff_t = 0, cap_voff_a = 0;
    Pt *d_vpts_t = nullptr, *d_spts_t = nullptr, *d_vpts_a = nullptr;
    size_t cap_vpts_t = 0, cap_spts_t = 0, cap_vpts_a = 0;
    float *d_amp_t = nullptr; size_t cap_amp_t = 0;
    // time-domain mode's checkpoint/segment block and kernels, kept between calls
    float *d_td_blk = nullptr; size_t cap_td_blk = 0;
    double *d_td_k = nullptr; size_t cap_td_k = 0;
    // checkpoints the forward itself writes for the time-domain mode
    // (ifosb_set_td_checkpoints): the interval asked for, and the batch whose
    // checkpoints the block holds
    int td_arm = 0;
    bool td_ck_ok = false;
    int td_ck_K = 0, td_ck_nshots = 0;
    cudaError_t hook_err = cudaSuccess;
    GraphSet gtd;  // time-domain loops, one graph per batch shape and interval
    // TMA staging (default) and its wait-timeout flag; the failure-path test knobs
    int use_tma = 1;
    int *d_tma_err = nullptr;
    unsigned long long wait_ns = WAIT_LIMIT_NS;
    int stop_it = -1, stop_kernel = 0;  // stop_kernel: 1 velocity, 2 stress
    float *d_cpg = nullptr;  // CPML rows in global memory (lane-divergent reads)
    // uniform relaxation times: passed as scalars instead of five model fields
    bool unif_tau = false;
    float utaus = 0.f, utaup = 0.f, uts_avg = 0.f;
    std::string err;
};

// ---------------------------------------------------------------------------
// helpers

static int fail(ifosb_engine *e, int code, const std::string &msg) {
    if (e) e->err = msg;
    return code;
}

#define CU(call)                                                                                     \
    do {                                                                                             \
        cudaError_t _e = (call);                                                                     \
        if (_e != cudaSuccess)                                                                       \
            return fail(e, _e == cudaErrorMemoryAllocation ? IFOSB_ENOMEM : IFOSB_ECUDA,             \
                        std::string(#call) + ": " + cudaGetErrorString(_e));                         \
    } while (0)

template <class T>
static int dalloc(ifosb_engine *e, T **ptr, size_t count) {
    if (count == 0) count = 1;
    cudaError_t r = cudaMalloc((void **)ptr, count * sizeof(T));
    if (r != cudaSuccess) {
        *ptr = nullptr;
        cudaGetLastError();
        return fail(e, IFOSB_ENOMEM, "cudaMalloc of " + std::to_string(count * sizeof(T)) + " bytes failed");
    }
    e->dev_bytes += (long long)(count * sizeof(T));
    return IFOSB_OK;
}

template <class T>
static void dfree(ifosb_engine *e, T **ptr, size_t count) {
    if (*ptr) {
        cudaFree(*ptr);
        e->dev_bytes -= (long long)(std::max<size_t>(count, 1) * sizeof(T));
        *ptr = nullptr;
    }
}

template <class T>
static int dgrow(ifosb_engine *e, T **ptr, size_t *cap, size_t count) {
    if (count <= *cap && *ptr) return IFOSB_OK;
    dfree(e, ptr, *cap);
    *cap = 0;
    size_t want = std::max<size_t>(count, 16);
    int rc = dalloc(e, ptr, want);
    if (rc == IFOSB_OK) *cap = want;
    return rc;
}

static void fd_coeffs(int fdcoeff, float *b1, float *b2) {
    *b1 = 9.0 / 8.0; *b2 = -1.0 / 24.0;                  // Taylor (update_v_ssg.c:97)
    if (fdcoeff == 2) { *b1 = 1.1382; *b2 = -0.046414; }  // Holberg (update_v_ssg.c:98-100)
}

static int nsamples(const ifosb_params *p) {
    if (p->ndtshift > p->nt) return 0;
    return (int)ceil((float)(p->nt - p->ndtshift) / (float)p->ndt);  // ifos3d.c:178-179
}

static void release_graph(GraphCache &gc) {
    if (gc.exec) cudaGraphExecDestroy(gc.exec);
    gc.exec = nullptr;
    gc.key.clear();
}

static void release_graph(GraphSet &gs) {
    for (GraphCache &gc : gs.g) release_graph(gc);
}

static int check_launch(ifosb_engine *e, const char *what) {
    cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) return fail(e, IFOSB_ECUDA, std::string(what) + ": " + cudaGetErrorString(le));
    return IFOSB_OK;
}

static int block_of(const Geo &g, int j, int i, int k) {
    const int bx = (k - 1) / BX, by = (i - 1) / g.by, yc = (j - 1) / g.cy;
    return (yc * g.nti + by) * g.ntk + bx;
}

// Groups points per (shot, block), stable within a group (the reference's loop order).
static int upload_points(ifosb_engine *e, const Geo &g, int nshots, const std::vector<HostPt> &pts, int **d_off,
                         size_t *cap_off, Pt **d_pts, size_t *cap_pts) {
    const int nblk = g.ntk * g.nti * g.nyc;
    std::vector<int> cnt((size_t)nshots * nblk, 0);
    for (const HostPt &q : pts) cnt[(size_t)q.s * nblk + block_of(g, q.j, q.i, q.k)]++;
    std::vector<int> off((size_t)nshots * (nblk + 1), 0), pos((size_t)nshots * nblk, 0);
    int run = 0;
    for (int s = 0; s < nshots; ++s) {
        for (int b = 0; b < nblk; ++b) {
            off[(size_t)s * (nblk + 1) + b] = run;
            pos[(size_t)s * nblk + b] = run;
            run += cnt[(size_t)s * nblk + b];
        }
        off[(size_t)s * (nblk + 1) + nblk] = run;
    }
    std::vector<Pt> out(pts.size());
    for (const HostPt &q : pts) {
        Pt t{};
        t.j = q.j; t.i = q.i; t.k = q.k; t.kind = q.kind; t.row = q.row;
        out[pos[(size_t)q.s * nblk + block_of(g, q.j, q.i, q.k)]++] = t;
    }
    int rc;
    if ((rc = dgrow(e, d_off, cap_off, off.size())) || (rc = dgrow(e, d_pts, cap_pts, out.size()))) return rc;
    CU(cudaMemcpyAsync(*d_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, e->stream));
    if (!out.empty()) CU(cudaMemcpyAsync(*d_pts, out.data(), out.size() * sizeof(Pt), cudaMemcpyHostToDevice, e->stream));
    return IFOSB_OK;
}

// ---------------------------------------------------------------------------
// lifecycle

extern "C" int ifosb_nsamples(const ifosb_params *p) { return p ? nsamples(p) : 0; }

extern "C" int ifosb_create(const ifosb_params *p, int max_shots, int max_nf, ifosb_engine **out) {
    if (!p || !out) return IFOSB_EARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return IFOSB_ENODEV;
    }
    if (p->fdorder != 4 || p->abs_type != 1 || p->nmech < 0 || p->nmech > MAXMECH || p->fw < 1 || p->fw > MAXFW ||
        p->nx < 2 * p->fw + 1 || p->ny < 2 * p->fw + 1 || p->nz < 2 * p->fw + 1 || p->nt < 2 || p->ndt < 1 ||
        p->ndtshift < 0 || max_shots < 1 || max_nf < 0 || max_nf > MAXNF || !(p->dt > 0.f) || !(p->dx > 0.f) ||
        !(p->dy > 0.f) || !(p->dz > 0.f))
        return IFOSB_EARG;
    ifosb_engine *e = new ifosb_engine();
    e->p = *p;
    e->max_shots = max_shots;
    e->max_nf = max_nf;
    fd_coeffs(p->fdcoeff, &e->b1, &e->b2);
    Geo &g = e->g;
    g.nx = p->nx; g.ny = p->ny; g.nz = p->nz; g.fw = p->fw; g.free_surf = p->free_surf ? 1 : 0; g.nmech = p->nmech;
    g.pz = ((p->nz + 10) + 7) / 8 * 8;
    g.px = p->nx + 4;
    g.plane = (long long)g.px * g.pz;
    g.field = (long long)(p->ny + 5) * g.plane;
    g.cy = DEFAULT_CY;
    g.nyc = (p->ny + g.cy - 1) / g.cy;
    {
        const char *v = getenv("IFOSB_TMA");
        if (v && v[0] == '0') e->use_tma = 0;
    }
    // tile rows: 7 (8-warp CTAs, two per SM) when the stress kernel carries memory
    // variables, else 8; IFOSB_TILE_ROWS=7|8 overrides (tests, tuning experiments)
    g.by = (e->use_tma && p->nmech > 0) ? 7 : 8;
    if (const char *v = getenv("IFOSB_TILE_ROWS")) {
        const int t = atoi(v);
        if (t == 7 || t == 8) g.by = t;
    }
    if (const char *v = getenv("IFOSB_VEL_TILE_ROWS")) {
        const int t = atoi(v);
        if (t == 7 || t == 8) e->vby = t;
    }
    if (!e->use_tma) e->vby = g.by;
    g.ntk = (p->nz + BX - 1) / BX;
    g.nti = (p->nx + g.by - 1) / g.by;
    if ((long long)g.nyc * max_shots > 65535) { delete e; return IFOSB_EARG; }
    e->sl.sx = (long long)p->ny * 2 * p->fw * p->nz;
    e->sl.sy = (long long)2 * p->fw * p->nx * p->nz;
    e->sl.sz = (long long)p->ny * p->nx * 2 * p->fw;
    e->st_shot = (long long)(NEL + 6 * p->nmech) * g.field;
    e->psi_shot = 6 * (e->sl.sx + e->sl.sy + e->sl.sz);
    e->dft_shot = (long long)max_nf * 6 * g.field;
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete e;
        return IFOSB_ECUDA;
    }
    e->own_stream = e->stream;
    const long long ncell = (long long)p->nx * p->ny * p->nz;
    int rc;
    if ((rc = dalloc(e, &e->d_state, (size_t)(e->st_shot * max_shots))) ||
        (rc = dalloc(e, &e->d_psi, (size_t)(e->psi_shot * max_shots))) ||
        (rc = dalloc(e, &e->d_model, (size_t)(NMODEL * g.field))) ||
        (rc = dalloc(e, &e->d_rho_w, (size_t)g.field)) ||
        (rc = dalloc(e, &e->d_grad, (size_t)(3 * ncell))) ||
        (rc = dalloc(e, &e->d_grad64, (size_t)(3 * ncell))) ||
        (rc = dalloc(e, &e->d_err, (size_t)max_shots)) || (rc = dalloc(e, &e->d_tma_err, 1))) {
        ifosb_destroy(e);
        return rc;
    }
    if (p->nmech > 0 && (rc = dalloc(e, &e->d_gradq, (size_t)(2 * ncell)))) {
        ifosb_destroy(e);
        return rc;
    }
    if (e->d_gradq) cudaMemsetAsync(e->d_gradq, 0, sizeof(double) * 2 * ncell, e->stream);
    if (max_nf > 0) {
        if ((rc = dalloc(e, &e->d_dftf, (size_t)(e->dft_shot * max_shots))) ||
            (rc = dalloc(e, &e->d_dftb, (size_t)(e->dft_shot * max_shots)))) {
            ifosb_destroy(e);
            return rc;
        }
    }
    // halos and row padding of every field stay zero for the engine's lifetime
    cudaMemsetAsync(e->d_model, 0, sizeof(float) * NMODEL * g.field, e->stream);
    cudaMemsetAsync(e->d_rho_w, 0, sizeof(float) * g.field, e->stream);
    cudaMemsetAsync(e->d_grad, 0, sizeof(float) * 3 * ncell, e->stream);
    cudaMemsetAsync(e->d_grad64, 0, sizeof(double) * 3 * ncell, e->stream);
    if (cudaStreamSynchronize(e->stream) != cudaSuccess) {
        cudaGetLastError();
        ifosb_destroy(e);
        return IFOSB_ECUDA;
    }
    *out = e;
    return IFOSB_OK;
}

extern "C" void ifosb_destroy(ifosb_engine *e) {
    if (!e) return;
    if (e->stream) cudaStreamSynchronize(e->stream);
    release_graph(e->gfwd);
    release_graph(e->gadj);
    release_graph(e->gtd);
    void *bufs[] = {e->d_state, e->d_psi, e->d_model, e->d_rho_w, e->d_dftf, e->d_dftb, e->d_grad, e->d_grad64,
                    e->d_err, e->d_sec, e->d_diff, e->d_obs, e->d_part, e->d_misfit, e->d_l2, e->d_trig_f,
                    e->d_trig_b, e->d_voff, e->d_soff, e->d_vpts, e->d_spts, e->d_amp, e->d_tma_err, e->d_cpg,
                    e->d_mstage, e->d_green, e->d_gsig, e->d_hess, e->d_sec2, e->d_voff_t, e->d_soff_t,
                    e->d_voff_a, e->d_vpts_t, e->d_spts_t, e->d_vpts_a, e->d_amp_t, e->d_gradq, e->d_smod,
                    e->d_td_blk, e->d_td_k};
    for (void *b : bufs)
        if (b) cudaFree(b);
    for (cudaEvent_t ev : e->events) cudaEventDestroy(ev);
    if (e->own_stream) cudaStreamDestroy(e->own_stream);
    delete e;
}

extern "C" int ifosb_set_seismo(ifosb_engine *e, int seismo) {
    if (!e || seismo < 1 || seismo > 4) return IFOSB_EARG;
    if (seismo >= 2 && !e->d_sec2 && e->ntr > 0) {
        const size_t secn = (size_t)e->max_shots * 3 * e->ntr * e->ns;
        int rc;
        if ((rc = dalloc(e, &e->d_sec2, secn))) return rc;
        CU(cudaMemsetAsync(e->d_sec2, 0, secn * sizeof(float), e->stream));
        CU(cudaStreamSynchronize(e->stream));
    }
    e->seismo = seismo;
    return IFOSB_OK;
}

extern "C" int ifosb_set_profiling(ifosb_engine *e, int profile) {
    if (!e) return IFOSB_EARG;
    e->profile = profile ? 1 : 0;
    return IFOSB_OK;
}

extern "C" int ifosb_kernel_times(const ifosb_engine *e, double *vel_ms, double *str_ms, int *steps) {
    if (!e) return IFOSB_EARG;
    if (vel_ms) *vel_ms = e->t_vel_ms;
    if (str_ms) *str_ms = e->t_str_ms;
    if (steps) *steps = e->t_steps;
    return IFOSB_OK;
}

extern "C" int ifosb_set_stream(ifosb_engine *e, void *stream) {
    if (!e) return IFOSB_EARG;
    if (e->stream) cudaStreamSynchronize(e->stream);
    e->stream = stream ? (cudaStream_t)stream : e->own_stream;
    release_graph(e->gfwd);
    release_graph(e->gadj);
    release_graph(e->gtd);
    return IFOSB_OK;
}

extern "C" const char *ifosb_last_error(const ifosb_engine *e) { return e ? e->err.c_str() : "no engine"; }
extern "C" long long ifosb_device_bytes(const ifosb_engine *e) { return e ? e->dev_bytes : 0; }
extern "C" long long ifosb_last_launch_count(const ifosb_engine *e) { return e ? e->launches : 0; }
extern "C" long long ifosb_graph_captures(const ifosb_engine *e) { return e ? e->captures : 0; }

extern "C" int ifosb_set_wait_test(ifosb_engine *e, long long wait_ns, int kernel, int stop_plane) {
    if (!e || wait_ns < 1000 || wait_ns > (long long)WAIT_LIMIT_NS || kernel < 0 || kernel > 2 || stop_plane < -1)
        return IFOSB_EARG;
    e->wait_ns = (unsigned long long)wait_ns;
    e->stop_kernel = kernel;
    e->stop_it = kernel ? stop_plane : -1;
    return IFOSB_OK;
}

extern "C" int ifosb_set_launch_mode(ifosb_engine *e, int mode) {
    if (!e || (mode != 0 && mode != 1)) return IFOSB_EARG;
    e->launch_mode = mode;
    return IFOSB_OK;
}

// ---------------------------------------------------------------------------
// static inputs

extern "C" int ifosb_set_cpml(ifosb_engine *e, const float *coeff) {
    if (!e || !coeff) return IFOSB_EARG;
    std::vector<float> host((size_t)18 * 2 * MAXFW, 0.f);
    const int n2 = 2 * e->p.fw;
    for (int r = 0; r < 18; ++r)
        for (int h = 0; h < n2; ++h) host[(size_t)r * 2 * MAXFW + h] = coeff[(size_t)r * n2 + h];
    CU(cudaMemcpyToSymbol(c_cpml, host.data(), host.size() * sizeof(float)));
    if (!e->d_cpg) {
        int rc = dalloc(e, &e->d_cpg, host.size());
        if (rc) return rc;
    }
    CU(cudaMemcpy(e->d_cpg, host.data(), host.size() * sizeof(float), cudaMemcpyHostToDevice));
    e->have_cpml = true;
    return IFOSB_OK;
}

extern "C" int ifosb_set_model(ifosb_engine *e, const float *rho, const float *pi, const float *u, const float *taus,
                               const float *taup, const float *eta) {
    if (!e || !rho || !pi || !u) return IFOSB_EARG;
    const ifosb_params &p = e->p;
    if (p.nmech > 0 && (!taus || !taup || !eta)) return fail(e, IFOSB_EARG, "viscoelastic model needs taus, taup, eta");
    e->ngreen = 0;  // Green's functions belong to a model
    const size_t ng = (size_t)(p.nx + 2) * (p.ny + 2) * (p.nz + 2);
    for (size_t q = 0; q < ng; ++q)
        if (!(rho[q] > 0.f) || !(u[q] > 0.f) || !(pi[q] > 0.f) || !std::isfinite(rho[q]) || !std::isfinite(u[q]) ||
            !std::isfinite(pi[q]))
            return fail(e, IFOSB_EARG, "model value not positive and finite at ghosted index " + std::to_string(q));
    for (int l = 0; l < p.nmech; ++l)
        if (!std::isfinite(eta[l])) return fail(e, IFOSB_EARG, "eta not finite");
    if (!e->d_mstage) {  // staging for the raw model, kept for the engine's lifetime
        const int rc = dalloc(e, &e->d_mstage, ng * 5);
        if (rc) return rc;
    }
    float *tmp = e->d_mstage;
    CU(cudaMemcpyAsync(tmp, rho, ng * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    CU(cudaMemcpyAsync(tmp + ng, pi, ng * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    CU(cudaMemcpyAsync(tmp + 2 * ng, u, ng * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    if (p.nmech > 0) {
        CU(cudaMemcpyAsync(tmp + 3 * ng, taus, ng * sizeof(float), cudaMemcpyHostToDevice, e->stream));
        CU(cudaMemcpyAsync(tmp + 4 * ng, taup, ng * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    }
    AvArgs a{};
    a.g = e->g;
    a.rho = tmp; a.pi = tmp + ng; a.u = tmp + 2 * ng; a.taus = tmp + 3 * ng; a.taup = tmp + 4 * ng;
    a.md = e->d_model;
    a.rho_w = e->d_rho_w;
    dim3 blk(32, 4), grd((p.nz + 31) / 32, (p.nx + 3) / 4, p.ny);
    k_av_mat<<<grd, blk, 0, e->stream>>>(a);
    k_rho_field<<<dim3((p.nz + 2 + 31) / 32, (p.nx + 2 + 3) / 4, p.ny + 2), blk, 0, e->stream>>>(a);
    cudaError_t le = cudaGetLastError();
    cudaError_t se = cudaStreamSynchronize(e->stream);
    if (le != cudaSuccess || se != cudaSuccess)
        return fail(e, IFOSB_ECUDA, std::string("av_mat: ") + cudaGetErrorString(le != cudaSuccess ? le : se));
    for (int l = 0; l < MAXMECH; ++l) e->eta[l] = l < p.nmech ? eta[l] : 0.f;
    // readmod() gives every cell the same TAU (readmod.c:57-58, 119-120); then the
    // staggered averages are one value too and the kernels take scalars
    e->unif_tau = false;
    if (p.nmech > 0) {
        bool u = true;
        for (size_t q = 1; q < ng && u; ++q) u = taus[q] == taus[0] && taup[q] == taup[0];
        if (u) {
            const float t = taus[0];
            e->unif_tau = true;
            e->utaus = t;
            e->utaup = taup[0];
            e->uts_avg = 0.25 * (t + t + t + t);  // av_mat.c:56-58 with four equal values
        }
    }
    e->have_model = true;
    e->fwd_ok = e->res_ok = e->adj_ok = false;
    return IFOSB_OK;
}

// The elastic free surface's own moduli: the reference's step-length forwards
// propagate in the test model but call surface_elastic with the current model's
// u and pi (src/ifos3d.c:1087-1090), which matters at the plane j = 1 only.
extern "C" int ifosb_set_surface_moduli(ifosb_engine *e, const float *pi, const float *u) {
    if (!e || (!pi) != (!u)) return IFOSB_EARG;
    e->fwd_ok = e->res_ok = e->adj_ok = false;
    if (!pi) {
        e->smod_on = false;
        return IFOSB_OK;
    }
    const ifosb_params &p = e->p;
    if (p.nmech > 0) return fail(e, IFOSB_EARG, "separate surface moduli apply to the elastic free surface only");
    const size_t plane = (size_t)p.nx * p.nz;
    std::vector<float> h(2 * plane);
    for (int i = 1; i <= p.nx; ++i)
        for (int k = 1; k <= p.nz; ++k) {
            const size_t gidx = ((size_t)1 * (p.nx + 2) + i) * (p.nz + 2) + k;  // [j=1][i][k] of the ghosted array
            const size_t q = (size_t)(i - 1) * p.nz + (k - 1);
            if (!(pi[gidx] > 0.f) || !std::isfinite(pi[gidx]) || !(u[gidx] >= 0.f) || !std::isfinite(u[gidx]))
                return fail(e, IFOSB_EARG, "surface modulus not positive and finite");
            h[q] = pi[gidx];
            h[plane + q] = u[gidx];
        }
    if (!e->d_smod) {
        const int rc = dalloc(e, &e->d_smod, 2 * plane);
        if (rc) return rc;
    }
    CU(cudaMemcpyAsync(e->d_smod, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    CU(cudaStreamSynchronize(e->stream));
    e->smod_on = true;
    return IFOSB_OK;
}

extern "C" int ifosb_set_receivers(ifosb_engine *e, int ntr, const int *recpos) {
    if (!e || ntr < 0 || (ntr > 0 && !recpos)) return IFOSB_EARG;
    e->ngreen = 0;
    const ifosb_params &p = e->p;
    for (int t = 0; t < ntr; ++t) {
        const int i = recpos[3 * t], j = recpos[3 * t + 1], k = recpos[3 * t + 2];
        if (i < 1 || i > p.nx || j < 1 || j > p.ny || k < 1 || k > p.nz)
            return fail(e, IFOSB_EARG, "receiver " + std::to_string(t) + " outside the grid");
    }
    const int ns = nsamples(&p);
    const size_t secn = (size_t)e->max_shots * 3 * std::max(ntr, 1) * std::max(ns, 1);
    dfree(e, &e->d_sec, e->ntr ? (size_t)e->max_shots * 3 * e->ntr * e->ns : 0);
    dfree(e, &e->d_sec2, e->ntr ? (size_t)e->max_shots * 3 * e->ntr * e->ns : 0);
    dfree(e, &e->d_diff, e->ntr ? (size_t)e->max_shots * 3 * e->ntr * e->ns : 0);
    dfree(e, &e->d_obs, e->ntr ? (size_t)e->max_shots * 3 * e->ntr * e->ns : 0);
    dfree(e, &e->d_part, e->ntr ? (size_t)e->max_shots * 3 * e->ntr : 0);
    dfree(e, &e->d_misfit, (size_t)e->max_shots);
    dfree(e, &e->d_l2, (size_t)e->max_shots);
    e->ntr = 0;
    int rc;
    if ((rc = dalloc(e, &e->d_sec, secn)) || (rc = dalloc(e, &e->d_diff, secn)) || (rc = dalloc(e, &e->d_obs, secn)) ||
        (rc = dalloc(e, &e->d_part, (size_t)e->max_shots * 3 * std::max(ntr, 1))) ||
        (rc = dalloc(e, &e->d_misfit, (size_t)e->max_shots)) || (rc = dalloc(e, &e->d_l2, (size_t)e->max_shots)))
        return rc;
    CU(cudaMemsetAsync(e->d_sec, 0, secn * sizeof(float), e->stream));
    if (e->seismo >= 2) {
        if ((rc = dalloc(e, &e->d_sec2, secn))) return rc;
        CU(cudaMemsetAsync(e->d_sec2, 0, secn * sizeof(float), e->stream));
    }
    e->ntr = ntr;
    e->ns = ns;
    e->rec.assign(recpos, recpos + 3 * ntr);
    e->fwd_ok = e->res_ok = e->adj_ok = false;
    release_graph(e->gfwd);
    release_graph(e->gadj);
    release_graph(e->gtd);
    CU(cudaStreamSynchronize(e->stream));
    return IFOSB_OK;
}

// Trig tables of discfourier (disc_fourier.c:36-45), in double as the reference.
static void trig_table(const ifosb_params &p, int nf, const float *finv, int ntast, int back, std::vector<double> &out) {
    out.assign((size_t)p.nt * nf * 2, 0.0);
    for (int nt = 1; nt <= p.nt; ++nt) {
        float t = 0.0;
        if (back == 0) t = nt * p.dt;
        if (back == 1) t = p.time - nt * p.dt;
        for (int l = 0; l < nf; ++l) {
            out[((size_t)(nt - 1) * nf + l) * 2 + 0] = cos(2.0 * t * finv[l] * M_PI) * p.dt * ntast;
            out[((size_t)(nt - 1) * nf + l) * 2 + 1] = sin(2.0 * t * finv[l] * M_PI) * p.dt * ntast;
        }
    }
}

extern "C" int ifosb_set_frequencies(ifosb_engine *e, int nf, const float *finv, int ntast) {
    if (!e || nf < 0 || nf > e->max_nf || (nf > 0 && (!finv || ntast < 1))) return IFOSB_EARG;
    e->ngreen = 0;
    e->hess_fwd = false;
    for (int l = 0; l < nf; ++l)
        if (!(finv[l] > 0.f)) return fail(e, IFOSB_EARG, "frequency must be positive");
    const ifosb_params &p = e->p;
    dfree(e, &e->d_trig_f, (size_t)p.nt * e->nf * 2);
    dfree(e, &e->d_trig_b, (size_t)p.nt * e->nf * 2);
    e->nf = 0;
    if (nf > 0) {
        std::vector<double> tf, tb;
        trig_table(p, nf, finv, ntast, 0, tf);
        trig_table(p, nf, finv, ntast, 1, tb);
        int rc;
        if ((rc = dalloc(e, &e->d_trig_f, tf.size())) || (rc = dalloc(e, &e->d_trig_b, tb.size()))) return rc;
        CU(cudaMemcpy(e->d_trig_f, tf.data(), tf.size() * sizeof(double), cudaMemcpyHostToDevice));
        CU(cudaMemcpy(e->d_trig_b, tb.data(), tb.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    e->nf = nf;
    e->ntast = nf > 0 ? ntast : 1;
    e->finv.assign(finv, finv + nf);
    e->fwd_ok = e->res_ok = e->adj_ok = false;
    release_graph(e->gfwd);
    release_graph(e->gadj);
    release_graph(e->gtd);
    return IFOSB_OK;
}

// ---------------------------------------------------------------------------
// the time loop

static_assert(TZ == BX, "TMA tiles and plain blocks share one block geometry along z");

// Everything one forward or adjoint call launches with.
// The time-domain checkpoints an armed forward writes after its steps: the
// running sums U += v DT, a checkpoint (state, PML memory, U) after steps K, 2K,
// ..., and U at NT (K = 0: none).
struct TdHook {
    float *uf, *uf_end, *ckp;
    size_t ck, ss, ps, us, ssz, psz;
    int K, nseg;
};

struct Loop {
    Geo lg;   // launch geometry of the stress kernel (the y chunking depends on the batch size)
    Geo lgv;  // launch geometry of the velocity kernel
    VelArgs va;
    StrArgs sa;
    VelTma vt;
    StrTma stt;
    int nshots = 0;
    bool back = false;
    bool tma = false;
    bool p2 = false;  // power-of-two spacings (stress kernel multiplies by 1/DX etc.)
    size_t vel_smem = 0, str_smem = 0;
    TdHook td;
};

// The launch shape for a batch of nshots: the autotuner's for that batch size,
// else the one tuned for the nearest batch size (the larger on a tie), else null.
static const ifosb_engine::Shape *shape_for(const ifosb_engine *e, int nshots) {
    if (e->tuned.empty()) return nullptr;
    auto hi = e->tuned.lower_bound(nshots);
    if (hi != e->tuned.end() && hi->first == nshots) return &hi->second;
    if (hi == e->tuned.begin()) return &hi->second;
    auto lo = std::prev(hi);
    if (hi == e->tuned.end() || nshots - lo->first < hi->first - nshots) return &lo->second;
    return &hi->second;
}

// y planes per CTA. Untuned, with no other batch size tuned either: enough chunks
// for about four CTAs per SM over the whole batch, 8 to 16 planes each (the
// autotuner picked 3 to 32 on 128^3 to 384x256x384 grids; chunks of 64 planes ran
// a 10-shot 384x256x384 batch 60 % slower than its tuned shape).
static Geo launch_geo(const ifosb_engine *e, int nshots, bool vel) {
    Geo g = e->g;
    if (vel) {
        g.by = e->vby;
        g.nti = (g.nx + g.by - 1) / g.by;
    }
    int cy;
    if (const ifosb_engine::Shape *t = shape_for(e, nshots)) {
        cy = vel ? t->cyv : t->cys;
    } else {
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaGetLastError();
        const long long per_set = (long long)g.ntk * g.nti * nshots;
        const long long chunks = std::max<long long>(1, (4LL * sms + per_set - 1) / per_set);
        cy = (int)((g.ny + chunks - 1) / chunks);
        cy = std::min(std::max(cy, DEFAULT_CY), 16);
    }
    cy = std::min(cy, g.ny);
    while (cy < g.ny && (long long)((g.ny + cy - 1) / cy) * nshots > 65535) ++cy;  // grid.z limit
    g.cy = cy;
    g.nyc = (g.ny + cy - 1) / cy;
    return g;
}

static void fill_common(ifosb_engine *e, Loop &L) {
    const ifosb_params &p = e->p;
    VelArgs &va = L.va;
    StrArgs &sa = L.sa;
    va = VelArgs{};
    sa = StrArgs{};
    va.g = L.lgv;
    sa.g = L.lg;
    va.sl = sa.sl = e->sl;
    va.st = sa.st = e->d_state;
    va.st_shot = sa.st_shot = e->st_shot;
    va.md = sa.md = e->d_model;
    va.psi = sa.psi = e->d_psi;
    va.psi_shot = sa.psi_shot = e->psi_shot;
    va.dxr = p.dt / p.dx; va.dyr = p.dt / p.dy; va.dzr = p.dt / p.dz;
    va.b1 = sa.b1 = e->b1;
    va.b2 = sa.b2 = e->b2;
    {
        // custom force direction factors (update_v_ssg.c:498-503); the reference is C,
        // so cos/sin of its float angles run in double (C++ would pick the float overloads)
        const float alpha_rad = p.alpha * 3.141592653589793 / 180, beta_rad = p.beta * 3.141592653589793 / 180;
        const double ca = std::cos((double)alpha_rad), sa_ = std::sin((double)alpha_rad);
        const double cb = std::cos((double)beta_rad), sb = std::sin((double)beta_rad);
        va.cf5x = cb * ca;
        va.cf5y = sa_;
        va.cf5z = sb * ca;
    }
    va.err_step = e->d_err;
    va.cpg = sa.cpg = e->d_cpg;
    va.probe_j = p.ny / 2; va.probe_i = p.nx / 2; va.probe_k = p.nz / 2;  // ifos3d.c:761
    sa.dt = p.dt;
    sa.dthalbe = p.dt / 2.0;
    sa.rdx = p.dx; sa.rdy = p.dy; sa.rdz = p.dz;
    for (int l = 0; l < MAXMECH; ++l) {
        const float eta = e->eta[l];
        sa.eta[l] = eta;
        sa.mb[l] = 1.0 / (1.0 + (eta * 0.5));      // update_s_ssg.c:123
        sa.mc[l] = 1.0 - (eta * 0.5);              // update_s_ssg.c:124
        sa.msb[l] = eta / (1.0 + (eta * 0.5));     // surface_ssg.c:152
    }
    sa.sec = e->d_sec;
    sa.seismo = e->seismo;
    sa.sec2 = e->d_sec2;
    sa.hrx = (float)(1.0 / (double)e->p.dx);  // seismo_ssg.c:38-40
    sa.hry = (float)(1.0 / (double)e->p.dy);
    sa.hrz = (float)(1.0 / (double)e->p.dz);
    sa.sec_tr = e->ns;
    sa.sec_comp = (long long)e->ntr * e->ns;
    sa.sec_shot = 3 * sa.sec_comp;
    sa.nf = e->nf;
    sa.dft_shot = e->dft_shot;
    sa.smod = e->smod_on ? e->d_smod : nullptr;
}

// cuTensorMapEncodeTiled from the driver, reached through the runtime (no libcuda link).
static PFN_cuTensorMapEncodeTiled_v12000 tma_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)f;
        else
            cudaGetLastError();
    }
    return fn;
}

static bool encode(CUtensorMap *m, void *base, int rank, const cuuint64_t *dims, const cuuint64_t *strides,
                   const cuuint32_t *box) {
    auto fn = tma_encoder();
    if (!fn) return false;
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (cuuint32_t)rank, base, dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static void smem_set(const void *f, size_t bytes) {
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}
template <int M>
static void smem_attrs(int vby, int sby, size_t vel, size_t str) {
    if (vby == 7) {
        smem_set((const void *)t7::k_velocity_tma<true>, vel);
        smem_set((const void *)t7::k_velocity_tma<false>, vel);
    } else {
        smem_set((const void *)t8::k_velocity_tma<true>, vel);
        smem_set((const void *)t8::k_velocity_tma<false>, vel);
    }
    if (sby == 7) {
        smem_set((const void *)t7::k_stress_tma<M, true>, str);
        smem_set((const void *)t7::k_stress_tma<M, false>, str);
    } else {
        smem_set((const void *)t8::k_stress_tma<M, true>, str);
        smem_set((const void *)t8::k_stress_tma<M, false>, str);
    }
}

// An exact reciprocal exists for a power-of-two spacing: x/h == x*(1/h) bit for bit.
static bool pow2(float h) {
    int ex = 0;
    return h > 0.f && std::isfinite(h) && std::frexp(h, &ex) == 0.5f;
}

// Tensor maps over the state [shot][slot][y][x][z], the model [slot][y][x][z] and the
// DFT accumulators [shot][6 nf][y][x][z]; false if TMA staging cannot be used.
static bool setup_tma(ifosb_engine *e, Loop &L, float *dft) {
    const Geo &g = e->g;
    const ifosb_params &p = e->p;
    const int nslot = NEL + 6 * p.nmech;
    const int nsr = 6 + 6 * p.nmech;
    const int nm = (p.nmech == 0 || e->unif_tau) ? 5 : 10;
    const int ndf = (dft && e->nf > 0) ? 6 * e->nf : 0;
    const size_t vs = L.lgv.by == 7 ? t7::vel_tma_smem() : t8::vel_tma_smem();
    const size_t ss = L.lg.by == 7 ? t7::str_tma_smem(nsr, nm, ndf) : t8::str_tma_smem(nsr, nm, ndf);
    const cuuint32_t TXV = (cuuint32_t)L.lgv.by, RXV = TXV + 2 * HX;  // velocity tile rows, ring rows
    const cuuint32_t TX = (cuuint32_t)L.lg.by, RX = TX + 2 * HX;      // stress tile rows, ring rows
    if (vs > 227 * 1024 || ss > 227 * 1024) return false;
    const cuuint64_t sdims[5] = {(cuuint64_t)g.pz, (cuuint64_t)g.px, (cuuint64_t)(p.ny + 5), (cuuint64_t)nslot,
                                 (cuuint64_t)e->max_shots};
    const cuuint64_t sstr[4] = {(cuuint64_t)g.pz * 4, (cuuint64_t)g.plane * 4, (cuuint64_t)g.field * 4,
                                (cuuint64_t)e->st_shot * 4};
    const cuuint64_t mdims[4] = {(cuuint64_t)g.pz, (cuuint64_t)g.px, (cuuint64_t)(p.ny + 5), (cuuint64_t)NMODEL};
    const cuuint64_t mstr[3] = {(cuuint64_t)g.pz * 4, (cuuint64_t)g.plane * 4, (cuuint64_t)g.field * 4};
    const cuuint32_t bhalov[5] = {(cuuint32_t)RZ, RXV, 1, 3, 1}, bpt[5] = {(cuuint32_t)TZ, TXV, 1, 3, 1};
    const cuuint64_t rdims[3] = {(cuuint64_t)g.pz, (cuuint64_t)g.px, (cuuint64_t)(p.ny + 5)};
    const cuuint64_t rstr[2] = {(cuuint64_t)g.pz * 4, (cuuint64_t)g.plane * 4};
    const cuuint32_t brh[3] = {(cuuint32_t)RZ, RXV, 1}, brp[3] = {(cuuint32_t)TZ, TXV, 1};
    const cuuint32_t bhalo[5] = {(cuuint32_t)RZ, RX, 1, 3, 1}, bsr[5] = {(cuuint32_t)TZ, TX, 1, (cuuint32_t)nsr, 1};
    const cuuint32_t bms[4] = {(cuuint32_t)TZ, TX, 1, (cuuint32_t)nm};
    L.vt = VelTma{};
    L.stt = StrTma{};
    if (!encode(&L.vt.m_halo, e->d_state, 5, sdims, sstr, bhalov) ||
        !encode(&L.vt.m_pt, e->d_state, 5, sdims, sstr, bpt) ||
        !encode(&L.vt.m_rho_halo, e->d_rho_w, 3, rdims, rstr, brh) ||
        !encode(&L.vt.m_rho_pt, e->d_rho_w, 3, rdims, rstr, brp) ||
        !encode(&L.stt.m_halo, e->d_state, 5, sdims, sstr, bhalo) ||
        !encode(&L.stt.m_sr, e->d_state, 5, sdims, sstr, bsr) || !encode(&L.stt.m_mod, e->d_model, 4, mdims, mstr, bms))
        return false;
    if (ndf) {
        const cuuint64_t ddims[5] = {(cuuint64_t)g.pz, (cuuint64_t)g.px, (cuuint64_t)(p.ny + 5),
                                     (cuuint64_t)(6 * e->max_nf), (cuuint64_t)e->max_shots};
        const cuuint64_t dstr[4] = {(cuuint64_t)g.pz * 4, (cuuint64_t)g.plane * 4, (cuuint64_t)g.field * 4,
                                    (cuuint64_t)e->dft_shot * 4};
        const cuuint32_t bd[5] = {(cuuint32_t)TZ, TX, 1, (cuuint32_t)ndf, 1};
        if (!encode(&L.stt.m_dft, dft, 5, ddims, dstr, bd)) return false;
    }
    L.vt.a = L.va;
    L.stt.a = L.sa;
    L.vt.tma_err = L.stt.tma_err = e->d_tma_err;
    L.vt.w = WaitCtl{e->wait_ns, e->stop_kernel == 1 ? e->stop_it : -1};
    L.stt.w = WaitCtl{e->wait_ns, e->stop_kernel == 2 ? e->stop_it : -1};
    {
        const ifosb_engine::Shape *t = shape_for(e, L.nshots);
        L.vt.l2ahead = t ? t->l2v : L2AHEAD_VEL_DEFAULT;
        L.stt.l2ahead = t ? t->l2s : L2AHEAD_STR_DEFAULT;
    }
    L.stt.nsr = nsr;
    L.stt.nm = nm;
    L.stt.ndf = ndf;
    L.stt.utaus = e->utaus;
    L.stt.utaup = e->utaup;
    L.stt.uts_avg = e->uts_avg;
    L.p2 = pow2(p.dx) && pow2(p.dy) && pow2(p.dz);
    L.stt.idx = 1.0f / p.dx;
    L.stt.idy = 1.0f / p.dy;
    L.stt.idz = 1.0f / p.dz;
    L.vel_smem = vs;
    L.str_smem = ss;
    switch (p.nmech) {
    case 0: smem_attrs<0>(L.lgv.by, L.lg.by, vs, ss); break;
    case 1: smem_attrs<1>(L.lgv.by, L.lg.by, vs, ss); break;
    case 2: smem_attrs<2>(L.lgv.by, L.lg.by, vs, ss); break;
    case 3: smem_attrs<3>(L.lgv.by, L.lg.by, vs, ss); break;
    default: smem_attrs<4>(L.lgv.by, L.lg.by, vs, ss); break;
    }
    return cudaGetLastError() == cudaSuccess;
}

template <int M>
static void launch_str_m(const Loop &L, dim3 grd, cudaStream_t st, int nt, int do_dft, int sample) {
    const int by = L.lg.by;
    if (L.tma) {
        const dim3 blk(TZ, by + 1);
        if (by == 7) {
            if (L.p2) t7::k_stress_tma<M, true><<<grd, blk, L.str_smem, st>>>(L.stt, nt, do_dft, sample);
            else t7::k_stress_tma<M, false><<<grd, blk, L.str_smem, st>>>(L.stt, nt, do_dft, sample);
        } else {
            if (L.p2) t8::k_stress_tma<M, true><<<grd, blk, L.str_smem, st>>>(L.stt, nt, do_dft, sample);
            else t8::k_stress_tma<M, false><<<grd, blk, L.str_smem, st>>>(L.stt, nt, do_dft, sample);
        }
    } else {
        k_stress<M><<<grd, dim3(BX, by), 0, st>>>(L.sa, nt, do_dft, sample);
    }
}

static void launch_str(int nmech, const Loop &L, dim3 grd, cudaStream_t st, int nt, int do_dft, int sample) {
    switch (nmech) {
    case 0: launch_str_m<0>(L, grd, st, nt, do_dft, sample); break;
    case 1: launch_str_m<1>(L, grd, st, nt, do_dft, sample); break;
    case 2: launch_str_m<2>(L, grd, st, nt, do_dft, sample); break;
    case 3: launch_str_m<3>(L, grd, st, nt, do_dft, sample); break;
    default: launch_str_m<4>(L, grd, st, nt, do_dft, sample); break;
    }
}

static void launch_vel(const Loop &L, dim3 grd, cudaStream_t st, int nt) {
    const int by = L.lgv.by;
    if (L.tma) {
        const dim3 blk(TZ, by + 1);
        if (by == 7) {
            if (L.back) t7::k_velocity_tma<true><<<grd, blk, L.vel_smem, st>>>(L.vt, nt);
            else t7::k_velocity_tma<false><<<grd, blk, L.vel_smem, st>>>(L.vt, nt);
        } else {
            if (L.back) t8::k_velocity_tma<true><<<grd, blk, L.vel_smem, st>>>(L.vt, nt);
            else t8::k_velocity_tma<false><<<grd, blk, L.vel_smem, st>>>(L.vt, nt);
        }
    } else {
        const dim3 blk(BX, by);
        if (L.back) k_velocity<true><<<grd, blk, 0, st>>>(L.va, nt);
        else k_velocity<false><<<grd, blk, 0, st>>>(L.va, nt);
    }
}

// Per-step launch parameters: DFT on steps nt % ntast == 0 (ifos3d.c:788), seismogram
// sample index when nt == lsamp (ifos3d.c:799-804, forward only).
static void step_flags(const ifosb_engine *e, bool back, int nt, int &lsamp, int &nlsamp, int &do_dft, int &sample) {
    do_dft = (e->nf > 0 && nt % e->ntast == 0) ? 1 : 0;
    sample = -1;
    if (!back && nt == lsamp) {
        sample = nlsamp++;
        lsamp += e->p.ndt;
    }
}

// The time-domain block of a batch: state2 | psi2 | Uf | Ub | Uf(NT) | checkpoints
// 1..nseg-1 | segment, each sub-buffer 256-byte aligned. The adjoint's step m
// stands at time TIME - m DT (discfourier's backward phase), so forward step n
// meets it at zero lag when n + m = P = TIME / DT (nearest whole step); forward
// steps 1..P-1 pair with an adjoint step, in segments of K steps. False when P is
// out of range.
struct TdLayout {
    int P, K, last, nseg;
    size_t ssz, psz, ss, ps, us, ck, seg_shot, total;
};
static bool td_layout(const ifosb_engine *e, int nshots, int interval, TdLayout &t) {
    const ifosb_params &p = e->p;
    t.P = (int)std::lround((double)p.time / (double)p.dt);
    if (t.P < 2 || t.P > p.nt + 1) return false;
    auto al = [](size_t v) { return (v + 63) & ~(size_t)63; };
    const long long F = e->g.field;
    t.K = std::min(interval, t.P - 1);
    t.last = t.P - 1;
    t.nseg = (t.last + t.K - 1) / t.K;  // segment q covers steps q*K+1 .. min((q+1)*K, last)
    t.ssz = (size_t)e->st_shot * nshots;
    t.psz = (size_t)e->psi_shot * nshots;
    t.ss = al(t.ssz);
    t.ps = al(t.psz);
    t.us = al((size_t)3 * F * nshots);
    t.ck = t.ss + t.ps + t.us;        // one checkpoint: state, PML memory, running sums
    t.seg_shot = (size_t)6 * F;       // one step of a segment: v and running sums
    t.total = t.ss + t.ps + 3 * t.us + (size_t)(t.nseg - 1) * t.ck + (size_t)t.K * t.seg_shot * nshots;
    return true;
}

static void td_integrate(ifosb_engine *e, int nshots, float *u, const float *st, float *seg, size_t seg_shot) {
    k_td_integrate<<<dim3(2 * 148, nshots), 256, 0, e->stream>>>(u, st, e->st_shot, e->g.field, nshots, e->p.dt, seg,
                                                                 (long long)seg_shot);
}

static void hook_copy(ifosb_engine *e, void *dst, const void *src, size_t words) {
    const cudaError_t r = cudaMemcpyAsync(dst, src, words * sizeof(float), cudaMemcpyDeviceToDevice, e->stream);
    if (r != cudaSuccess && e->hook_err == cudaSuccess) e->hook_err = r;
}

// after forward step nt of an armed forward (the engine's own state)
static void td_hook(ifosb_engine *e, const Loop &L, int nt) {
    const TdHook &t = L.td;
    td_integrate(e, L.nshots, t.uf, e->d_state, nullptr, 0);
    if (nt % t.K == 0 && nt / t.K < t.nseg) {
        float *c = t.ckp + (size_t)(nt / t.K - 1) * t.ck;
        hook_copy(e, c, e->d_state, t.ssz);
        hook_copy(e, c + t.ss, e->d_psi, t.psz);
        hook_copy(e, c + t.ss + t.ps, t.uf, t.us);
    }
    if (nt == e->p.nt) hook_copy(e, t.uf_end, t.uf, t.us);
}

// Enqueue the NT steps (two kernels per step) on the engine stream.
static void enqueue_loop(ifosb_engine *e, const Loop &L) {
    const ifosb_params &p = e->p;
    const dim3 grd(L.lg.ntk, L.lg.nti, L.lg.nyc * L.nshots), grdv(L.lgv.ntk, L.lgv.nti, L.lgv.nyc * L.nshots);
    int lsamp = p.ndtshift + 1, nlsamp = 0;
    for (int nt = 1; nt <= p.nt; ++nt) {
        launch_vel(L, grdv, e->stream, nt);
        int do_dft, sample;
        step_flags(e, L.back, nt, lsamp, nlsamp, do_dft, sample);
        launch_str(p.nmech, L, grd, e->stream, nt, do_dft, sample);
        if (L.td.K) td_hook(e, L, nt);
    }
}

// Kernel-by-kernel launches with an event pair around each kernel (kernel timing).
static int run_loop_profiled(ifosb_engine *e, const Loop &L) {
    const ifosb_params &p = e->p;
    const int nsteps = e->nt_limit > 0 ? std::min(e->nt_limit, p.nt) : p.nt;  // the autotuner times a few steps
    const size_t need = (size_t)3 * nsteps;
    while (e->events.size() < need) {
        cudaEvent_t ev;
        CU(cudaEventCreate(&ev));
        e->events.push_back(ev);
    }
    const dim3 grd(L.lg.ntk, L.lg.nti, L.lg.nyc * L.nshots), grdv(L.lgv.ntk, L.lgv.nti, L.lgv.nyc * L.nshots);
    int lsamp = p.ndtshift + 1, nlsamp = 0;
    for (int nt = 1; nt <= nsteps; ++nt) {
        cudaEvent_t *ev = &e->events[(size_t)3 * (nt - 1)];
        CU(cudaEventRecord(ev[0], e->stream));
        launch_vel(L, grdv, e->stream, nt);
        CU(cudaEventRecord(ev[1], e->stream));
        int do_dft, sample;
        step_flags(e, L.back, nt, lsamp, nlsamp, do_dft, sample);
        launch_str(p.nmech, L, grd, e->stream, nt, do_dft, sample);
        CU(cudaEventRecord(ev[2], e->stream));
        if (L.td.K) td_hook(e, L, nt);
    }
    int rc = check_launch(e, "time loop");
    if (rc) return rc;
    CU(cudaStreamSynchronize(e->stream));
    double tv = 0.0, ts = 0.0;
    for (int nt = 1; nt <= nsteps; ++nt) {
        cudaEvent_t *ev = &e->events[(size_t)3 * (nt - 1)];
        float a = 0.f, b = 0.f;
        CU(cudaEventElapsedTime(&a, ev[0], ev[1]));
        CU(cudaEventElapsedTime(&b, ev[1], ev[2]));
        tv += a;
        ts += b;
    }
    e->t_vel_ms = tv;
    e->t_str_ms = ts;
    e->t_steps = nsteps;
    return IFOSB_OK;
}

// Replays the graph of `key` from the set, or captures `enqueue` into the least
// recently used slot and replays that.
template <class Fn>
static int replay_graph(ifosb_engine *e, GraphSet &gs, const std::vector<unsigned char> &key, Fn enqueue) {
    GraphCache *hit = nullptr, *lru = &gs.g[0];
    for (GraphCache &c : gs.g) {
        if (c.exec && c.key == key) hit = &c;
        if (!c.exec) { if (lru->exec) lru = &c; }
        else if (lru->exec && c.used < lru->used) lru = &c;
    }
    GraphCache &gc = hit ? *hit : *lru;
    gc.used = ++gs.tick;
    if (!hit) {
        release_graph(gc);
        cudaGraph_t graph = nullptr;
        CU(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        enqueue();
        cudaError_t ce = cudaStreamEndCapture(e->stream, &graph);
        if (ce != cudaSuccess) {
            cudaGetLastError();
            return fail(e, IFOSB_ECUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
        }
        ce = cudaGraphInstantiate(&gc.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) {
            gc.exec = nullptr;
            cudaGetLastError();
            return fail(e, IFOSB_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
        }
        gc.key = key;
        ++e->captures;
    }
    CU(cudaGraphLaunch(gc.exec, e->stream));
    return IFOSB_OK;
}

static int run_loop(ifosb_engine *e, const Loop &L) {
    GraphSet &gs = L.back ? e->gadj : e->gfwd;
    e->launches = 2LL * e->p.nt;
    if (e->profile) return run_loop_profiled(e, L);
    if (e->launch_mode == 1) {
        enqueue_loop(e, L);
        return check_launch(e, "time loop");
    }
    std::vector<unsigned char> key(sizeof(Loop));
    std::memcpy(key.data(), &L, sizeof(Loop));
    return replay_graph(e, gs, key, [&]() { enqueue_loop(e, L); });
}

static int check_unstable(ifosb_engine *e, int nshots) {
    std::vector<int> errs(nshots);
    int terr = 0;
    CU(cudaMemcpyAsync(errs.data(), e->d_err, sizeof(int) * nshots, cudaMemcpyDeviceToHost, e->stream));
    CU(cudaMemcpyAsync(&terr, e->d_tma_err, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
    CU(cudaStreamSynchronize(e->stream));
    if (terr)
        return fail(e, IFOSB_ECUDA, "a TMA stage did not arrive within " + std::to_string(e->wait_ns / 1000000ull) +
                                        " ms (mbarrier wait timed out)");
    for (int s = 0; s < nshots; ++s)
        if (errs[s] != INT_MAX)
            return fail(e, IFOSB_EUNSTABLE,
                        " Simulation is unstable ! (shot " + std::to_string(s) + ", step " + std::to_string(errs[s]) + ")");
    return IFOSB_OK;
}

static int reset_state(ifosb_engine *e, int nshots, float *dft) {
    CU(cudaMemsetAsync(e->d_state, 0, sizeof(float) * e->st_shot * nshots, e->stream));       // zero_wavefield
    CU(cudaMemsetAsync(e->d_psi, 0, sizeof(float) * e->psi_shot * nshots, e->stream));
    if (dft && e->nf > 0) CU(cudaMemsetAsync(dft, 0, sizeof(float) * e->dft_shot * nshots, e->stream));  // zero_invers
    std::vector<int> init(nshots, INT_MAX);
    CU(cudaMemcpyAsync(e->d_err, init.data(), sizeof(int) * nshots, cudaMemcpyHostToDevice, e->stream));
    CU(cudaMemsetAsync(e->d_tma_err, 0, sizeof(int), e->stream));
    CU(cudaStreamSynchronize(e->stream));  // init lives on the host stack
    return IFOSB_OK;
}

// psource.c:38-52, the explosive-source amplitude at step nt
static float psource_amp(const ifosb_params &p, const float *s, int nt) {
    float amp = 0.0;
    if (nt == 1) amp = s[nt + 1 - 1] / (2.0 * p.dx * p.dy * p.dz);
    if ((nt > 1) && (nt < p.nt)) amp = (s[nt + 1 - 1] - s[nt - 1 - 1]) / (2.0 * p.dx * p.dy * p.dz);
    if (nt == p.nt) amp = -s[nt - 1 - 1] / (2.0 * p.dx * p.dy * p.dz);
    return amp;
}

extern "C" int ifosb_forward(ifosb_engine *e, int nshots, const ifosb_shot *shots, float *sections) {
    if (!e || !shots || nshots < 1 || nshots > e->max_shots) return IFOSB_EARG;
    if (!e->have_model || !e->have_cpml) return fail(e, IFOSB_ESTATE, "set the model and the CPML profiles first");
    const ifosb_params &p = e->p;
    // point lists: forces (velocity kernel), explosive sources and receivers (stress kernel)
    std::vector<HostPt> vp, sp;
    std::vector<float> amp;
    int row = 0;
    for (int s = 0; s < nshots; ++s) {
        const ifosb_shot &sh = shots[s];
        if (sh.nsrc < 0 || (sh.nsrc > 0 && (!sh.srcpos || !sh.signals))) return IFOSB_EARG;
        for (int l = 0; l < sh.nsrc; ++l) {
            const float *sp7 = sh.srcpos + 7 * l;
            const int i = (int)sp7[0], j = (int)sp7[1], k = (int)sp7[2], kind = (int)sp7[6];
            if (i < 1 || i > p.nx || j < 1 || j > p.ny || k < 1 || k > p.nz)
                return fail(e, IFOSB_EARG, "source outside the grid");
            const float *sig = sh.signals + (size_t)l * p.nt;
            if (kind == 1) {
                for (int nt = 1; nt <= p.nt; ++nt) amp.push_back(psource_amp(p, sig, nt));
                sp.push_back({s, j, i, k, 1, row++});
            } else if (kind >= 2 && kind <= 5) {
                // update_v_ssg.c:480: amp = DT*signals[l][nt]/(DX*DY*DZ)
                for (int nt = 1; nt <= p.nt; ++nt) amp.push_back(p.dt * sig[nt - 1] / (p.dx * p.dy * p.dz));
                vp.push_back({s, j, i, k, kind, row++});
            }
        }
        for (int t = 0; t < e->ntr; ++t) sp.push_back({s, e->rec[3 * t + 1], e->rec[3 * t], e->rec[3 * t + 2], PT_RECEIVER, t});
    }
    Loop L;
    std::memset(static_cast<void *>(&L), 0, sizeof(L));  // the graph cache compares Loops bytewise, padding included
    L.nshots = nshots;
    L.back = false;
    L.lg = launch_geo(e, nshots, false);
    L.lgv = launch_geo(e, nshots, true);
    int rc;
    if ((rc = upload_points(e, L.lgv, nshots, vp, &e->d_voff, &e->cap_voff, &e->d_vpts, &e->cap_vpts)) ||
        (rc = upload_points(e, L.lg, nshots, sp, &e->d_soff, &e->cap_soff, &e->d_spts, &e->cap_spts)) ||
        (rc = dgrow(e, &e->d_amp, &e->cap_amp, amp.size())))
        return rc;
    if (!amp.empty()) CU(cudaMemcpyAsync(e->d_amp, amp.data(), amp.size() * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    e->td_vp = vp;
    e->td_sp = sp;
    e->td_amp = amp;
    if ((rc = reset_state(e, nshots, e->d_dftf))) return rc;
    fill_common(e, L);
    VelArgs &va = L.va;
    StrArgs &sa = L.sa;
    va.pt_off = vp.empty() ? nullptr : e->d_voff;
    va.pts = e->d_vpts;
    va.val = e->d_amp;
    va.val_row = p.nt;
    va.val_comp = 0;
    sa.pt_off = sp.empty() ? nullptr : e->d_soff;
    sa.pts = e->d_spts;
    sa.amp = e->d_amp;
    sa.amp_row = p.nt;
    sa.dft = e->d_dftf;
    sa.trig = e->d_trig_f;
    L.tma = e->use_tma && setup_tma(e, L, e->d_dftf);
    e->fwd_ok = e->res_ok = e->adj_ok = e->hess_fwd = false;
    e->td_ck_ok = false;
    TdLayout tl;
    if (e->td_arm > 0 && e->nt_limit == 0 && td_layout(e, nshots, e->td_arm, tl)) {
        // checkpoints for ifosb_gradient_td, written by this forward (the whole loop runs)
        if ((rc = dgrow(e, &e->d_td_blk, &e->cap_td_blk, tl.total))) return rc;
        float *uf = e->d_td_blk + tl.ss + tl.ps, *uf_end = uf + 2 * tl.us;
        L.td = TdHook{uf, uf_end, uf_end + tl.us, tl.ck, tl.ss, tl.ps, tl.us, tl.ssz, tl.psz, tl.K, tl.nseg};
        CU(cudaMemsetAsync(uf, 0, tl.us * sizeof(float), e->stream));
    }
    e->hook_err = cudaSuccess;
    if ((rc = run_loop(e, L))) return rc;
    if (e->hook_err != cudaSuccess)
        return fail(e, IFOSB_ECUDA, std::string("time-domain checkpoints: ") + cudaGetErrorString(e->hook_err));
    e->nshots = nshots;
    if ((rc = check_unstable(e, nshots))) return rc;  // a failed batch is not a forward to build on
    e->fwd_ok = true;
    if (L.td.K) {
        e->td_ck_ok = true;
        e->td_ck_K = L.td.K;
        e->td_ck_nshots = nshots;
    }
    e->hess_fwd = e->nf > 0;
    if (sections && e->ntr > 0) {
        // [shot][component][ntr][ns] in saveseis's order: vx vy vz (1), p (2), div curl (3), all six (4)
        const size_t tr = (size_t)e->ntr * e->ns;
        static const int comps[5][7] = {{0}, {3, 0, 1, 2}, {1, 3}, {2, 4, 5}, {6, 0, 1, 2, 3, 4, 5}};
        const int *cl = comps[e->seismo];
        for (int sh = 0; sh < nshots; ++sh)
            for (int q = 0; q < cl[0]; ++q) {
                const int c = cl[q + 1];
                const float *src = c < 3 ? e->d_sec + ((size_t)sh * 3 + c) * tr : e->d_sec2 + ((size_t)sh * 3 + c - 3) * tr;
                CU(cudaMemcpyAsync(sections + ((size_t)sh * cl[0] + q) * tr, src, sizeof(float) * tr,
                                   cudaMemcpyDeviceToHost, e->stream));
            }
        CU(cudaStreamSynchronize(e->stream));
    }
    return check_launch(e, "forward");
}

extern "C" int ifosb_residual(ifosb_engine *e, const float *obs, double *misfit_fp64, float *l2_ref) {
    if (!e || !obs) return IFOSB_EARG;
    if (!e->fwd_ok || e->ntr == 0) return fail(e, IFOSB_ESTATE, "residual needs a forward batch with receivers");
    const int nshots = e->nshots, ntr = e->ntr, ns = e->ns;
    const size_t n = (size_t)nshots * 3 * ntr * ns;
    // obs may be host or device memory (unified addressing picks the copy's direction)
    CU(cudaMemcpyAsync(e->d_obs, obs, n * sizeof(float), cudaMemcpyDefault, e->stream));
    const int nthr = nshots * 3 * ntr;
    k_residual<<<(nthr + 127) / 128, 128, 0, e->stream>>>(e->d_sec, e->d_obs, e->d_diff, e->d_part, nshots, ntr, ns, e->p.dt);
    k_misfit<<<nshots, 32, 0, e->stream>>>(e->d_part, e->d_misfit, 3 * ntr);
    if (l2_ref) k_l2_ref<<<(nshots + 31) / 32, 32, 0, e->stream>>>(e->d_diff, e->d_l2, nshots, ntr, ns);
    int rc = check_launch(e, "residual");
    if (rc) return rc;
    if (misfit_fp64) CU(cudaMemcpyAsync(misfit_fp64, e->d_misfit, sizeof(double) * nshots, cudaMemcpyDeviceToHost, e->stream));
    if (l2_ref) CU(cudaMemcpyAsync(l2_ref, e->d_l2, sizeof(float) * nshots, cudaMemcpyDeviceToHost, e->stream));
    CU(cudaStreamSynchronize(e->stream));
    e->res_ok = true;
    e->adj_ok = false;
    return IFOSB_OK;
}

extern "C" int ifosb_adjoint(ifosb_engine *e, const float *diff) {
    if (!e) return IFOSB_EARG;
    const ifosb_params &p = e->p;
    if (!e->fwd_ok) return fail(e, IFOSB_ESTATE, "adjoint needs a forward batch");
    if (!diff && !e->res_ok) return fail(e, IFOSB_ESTATE, "adjoint needs ifosb_residual or a caller residual");
    if (p.ndt != 1 || p.ndtshift != 0)
        return fail(e, IFOSB_EARG, "the adjoint indexes the residual by time step: NDT=1, NDTSHIFT=0 (update_v_ssg.c:518)");
    if (e->nf == 0) return fail(e, IFOSB_ESTATE, "adjoint needs DFT frequencies");
    const int nshots = e->nshots, ntr = e->ntr, ns = e->ns;
    if (diff) CU(cudaMemcpyAsync(e->d_diff, diff, sizeof(float) * (size_t)nshots * 3 * ntr * ns, cudaMemcpyHostToDevice, e->stream));
    std::vector<HostPt> vp;
    for (int s = 0; s < nshots; ++s)
        for (int t = 0; t < ntr; ++t) vp.push_back({s, e->rec[3 * t + 1], e->rec[3 * t], e->rec[3 * t + 2], PT_ADJOINT, s * 3 * ntr + t});
    Loop L;
    std::memset(static_cast<void *>(&L), 0, sizeof(L));  // the graph cache compares Loops bytewise, padding included
    L.nshots = nshots;
    L.back = true;
    L.lg = launch_geo(e, nshots, false);
    L.lgv = launch_geo(e, nshots, true);
    int rc;
    if ((rc = upload_points(e, L.lgv, nshots, vp, &e->d_voff, &e->cap_voff, &e->d_vpts, &e->cap_vpts))) return rc;
    if ((rc = reset_state(e, nshots, e->d_dftb))) return rc;
    fill_common(e, L);
    VelArgs &va = L.va;
    StrArgs &sa = L.sa;
    va.pt_off = vp.empty() ? nullptr : e->d_voff;
    va.pts = e->d_vpts;
    va.val = e->d_diff;
    va.val_row = ns;
    va.val_comp = (long long)ntr * ns;
    sa.pt_off = nullptr;
    sa.pts = nullptr;
    sa.dft = e->d_dftb;
    sa.trig = e->d_trig_b;
    L.tma = e->use_tma && setup_tma(e, L, e->d_dftb);
    if ((rc = run_loop(e, L))) return rc;
    if ((rc = check_unstable(e, nshots))) return rc;
    e->adj_ok = true;
    return check_launch(e, "adjoint");
}

extern "C" int ifosb_gradient(ifosb_engine *e) {
    if (!e) return IFOSB_EARG;
    if (!e->adj_ok) return fail(e, IFOSB_ESTATE, "gradient needs a forward and an adjoint batch");
    const ifosb_params &p = e->p;
    GradArgs a{};
    a.g = e->g;
    a.dftf = e->d_dftf;
    a.dftb = e->d_dftb;
    a.dft_shot = e->dft_shot;
    a.nshots = e->nshots;
    a.nf = e->nf;
    a.md = e->d_model;
    a.rho = e->d_rho_w;
    for (int l = 0; l < e->nf; ++l) {
        float fdummy = 0.0;
        fdummy = 2.0 * 2.0 * e->finv[l] * e->finv[l] * M_PI * M_PI;  // gradient_F.c:70-72
        fdummy = 1 / fdummy;
        a.fdummy[l] = fdummy;
    }
    a.b1 = e->b1; a.b2 = e->b2;
    a.rdx = p.dx; a.rdy = p.dy; a.rdz = p.dz;
    a.ihx = 1.0f / p.dx; a.ihy = 1.0f / p.dy; a.ihz = 1.0f / p.dz;
    const bool p2 = pow2(p.dx) && pow2(p.dy) && pow2(p.dz);
    a.grad = e->d_grad;
    a.grad64 = e->d_grad64;
    a.gradq = p.nmech > 0 ? e->d_gradq : nullptr;
    for (int l = 0; l < e->nf; ++l) {
        const double w = 2.0 * M_PI * (double)e->finv[l];
        double re = 0.0, im = 0.0;
        for (int q = 0; q < p.nmech; ++q) {
            if (!(e->eta[q] > 0.f)) {  // no relaxation: the term is 1 (the unrelaxed modulus)
                re += 1.0;
                continue;
            }
            const double ts = (double)p.dt / (double)e->eta[q], wt = w * ts, den = 1.0 + wt * wt;
            re += wt * wt / den;  // s ts / (1 + s ts) with s = -i w (discfourier's e^{+i w t})
            im -= wt / den;
        }
        a.rphi[l] = re;
        a.iphi[l] = im;
    }
    dim3 blk(BX, BY), grd(e->g.ntk, e->g.nti, e->g.nyc);
    if (a.gradq) {
        if (p2) k_gradient<true, true><<<grd, blk, 0, e->stream>>>(a);
        else k_gradient<true, false><<<grd, blk, 0, e->stream>>>(a);
    } else {
        if (p2) k_gradient<false, true><<<grd, blk, 0, e->stream>>>(a);
        else k_gradient<false, false><<<grd, blk, 0, e->stream>>>(a);
    }
    int rc = check_launch(e, "gradient");
    if (rc) return rc;
    CU(cudaStreamSynchronize(e->stream));
    e->adj_ok = false;  // one gradient contribution per adjoint batch
    return IFOSB_OK;
}

// ---------------------------------------------------------------------------
// Time-domain gradient kernels with checkpointing: the forward batch is run again
// with its state saved every `interval` steps (or the checkpoints the forward
// wrote itself, ifosb_set_td_checkpoints, are taken); the adjoint then runs
// forward in its own time, and for each adjoint step the forward step it pairs
// with is recomputed segment by segment from the nearest checkpoint (segments
// taken in reverse). Memory: one state per checkpoint plus one segment of
// velocities, instead of the whole time history. No DFT, no traces; the loops of
// a call are one CUDA graph per batch shape and interval.
static void td_step(ifosb_engine *e, const Loop &L, int nt) {
    const dim3 grd(L.lg.ntk, L.lg.nti, L.lg.nyc * L.nshots), grdv(L.lgv.ntk, L.lgv.nti, L.lgv.nyc * L.nshots);
    launch_vel(L, grdv, e->stream, nt);
    launch_str(e->p.nmech, L, grd, e->stream, nt, 0, -1);
}

extern "C" int ifosb_set_td_checkpoints(ifosb_engine *e, int interval) {
    if (!e || interval < 0) return IFOSB_EARG;
    e->td_arm = interval;
    e->td_ck_ok = false;
    return IFOSB_OK;
}

extern "C" int ifosb_gradient_td(ifosb_engine *e, int interval, double *kernels) {
    if (!e || !kernels || interval < 1) return IFOSB_EARG;
    const ifosb_params &p = e->p;
    if (!e->fwd_ok || !e->res_ok) return fail(e, IFOSB_ESTATE, "the time-domain gradient needs a forward batch and its residual");
    if (p.ndt != 1 || p.ndtshift != 0) return fail(e, IFOSB_EARG, "the adjoint indexes the residual by step: NDT=1, NDTSHIFT=0");
    const int NT = p.nt, nshots = e->nshots;
    TdLayout t;
    if (!td_layout(e, nshots, interval, t)) return fail(e, IFOSB_EARG, "TIME / DT must lie between 2 and NT + 1 steps");
    const int K = t.K, last = t.last, nseg = t.nseg;
    const long long n = (long long)p.nx * p.ny * p.nz;
    const size_t ss = t.ss, ps = t.ps, us = t.us, ck = t.ck, seg_shot = t.seg_shot;
    // the last forward's own checkpoints at this interval spare the re-run (the
    // block is grow-only: it still holds them when it is large enough)
    const bool have_ck = e->td_ck_ok && e->td_ck_K == K && e->td_ck_nshots == nshots && e->d_td_blk &&
                         e->cap_td_blk >= t.total;
    int grc;
    if ((grc = dgrow(e, &e->d_td_blk, &e->cap_td_blk, t.total)) || (grc = dgrow(e, &e->d_td_k, &e->cap_td_k, (size_t)4 * n)))
        return grc;
    float *blk = e->d_td_blk;
    double *dk = e->d_td_k;
    float *st2 = blk, *psi2 = st2 + ss, *uf = psi2 + ps, *ub = uf + us, *uf_end = ub + us, *ckp = uf_end + us;
    float *segb = ckp + (size_t)(nseg - 1) * ck;
    int rc = IFOSB_OK;
    auto run = [&]() -> int {
        // the recomputation loop: the last forward's sources on its own state
        Loop Lf;
        std::memset(static_cast<void *>(&Lf), 0, sizeof(Lf));
        Lf.nshots = nshots;
        Lf.lg = launch_geo(e, nshots, false);
        Lf.lgv = launch_geo(e, nshots, true);
        int r;
        if ((r = upload_points(e, Lf.lgv, nshots, e->td_vp, &e->d_voff_t, &e->cap_voff_t, &e->d_vpts_t, &e->cap_vpts_t)) ||
            (r = upload_points(e, Lf.lg, nshots, e->td_sp, &e->d_soff_t, &e->cap_soff_t, &e->d_spts_t, &e->cap_spts_t)) ||
            (r = dgrow(e, &e->d_amp_t, &e->cap_amp_t, e->td_amp.size())))
            return r;
        if (!e->td_amp.empty())
            CU(cudaMemcpyAsync(e->d_amp_t, e->td_amp.data(), e->td_amp.size() * sizeof(float), cudaMemcpyHostToDevice,
                               e->stream));
        std::swap(e->d_state, st2);  // fill_common and the tensor maps take the engine's state pointers
        std::swap(e->d_psi, psi2);
        fill_common(e, Lf);
        Lf.va.pt_off = e->td_vp.empty() ? nullptr : e->d_voff_t;
        Lf.va.pts = e->d_vpts_t;
        Lf.va.val = e->d_amp_t;
        Lf.va.val_row = NT;
        Lf.sa.pt_off = e->td_sp.empty() ? nullptr : e->d_soff_t;
        Lf.sa.pts = e->d_spts_t;
        Lf.sa.amp = e->d_amp_t;
        Lf.sa.amp_row = NT;
        {
            const int ms = e->max_shots;  // the tensor maps cover this batch's shots only
            e->max_shots = nshots;
            Lf.tma = e->use_tma && setup_tma(e, Lf, nullptr);
            e->max_shots = ms;
        }
        std::swap(e->d_state, st2);
        std::swap(e->d_psi, psi2);
        // the adjoint loop: the residual injected at the receivers, on the engine's state
        Loop La;
        std::memset(static_cast<void *>(&La), 0, sizeof(La));
        La.nshots = nshots;
        La.back = true;
        La.lg = launch_geo(e, nshots, false);
        La.lgv = launch_geo(e, nshots, true);
        std::vector<HostPt> va;
        for (int sh = 0; sh < nshots; ++sh)
            for (int tr = 0; tr < e->ntr; ++tr)
                va.push_back({sh, e->rec[3 * tr + 1], e->rec[3 * tr], e->rec[3 * tr + 2], PT_ADJOINT, sh * 3 * e->ntr + tr});
        if ((r = upload_points(e, La.lgv, nshots, va, &e->d_voff_a, &e->cap_voff_a, &e->d_vpts_a, &e->cap_vpts_a))) return r;
        fill_common(e, La);
        La.va.pt_off = va.empty() ? nullptr : e->d_voff_a;
        La.va.pts = e->d_vpts_a;
        La.va.val = e->d_diff;
        La.va.val_row = e->ns;
        La.va.val_comp = (long long)e->ntr * e->ns;
        La.tma = e->use_tma && setup_tma(e, La, nullptr);
        TdArgs ta;
        std::memset(static_cast<void *>(&ta), 0, sizeof(ta));  // part of the graph key, padding included
        ta.g = e->g;
        ta.st = e->d_state;
        ta.st_shot = e->st_shot;
        ta.ub = ub;
        ta.seg_shot = (long long)seg_shot;
        ta.nshots = nshots;
        ta.b1 = e->b1; ta.b2 = e->b2;
        ta.rdx = p.dx; ta.rdy = p.dy; ta.rdz = p.dz;
        ta.ihx = 1.0f / p.dx; ta.ihy = 1.0f / p.dy; ta.ihz = 1.0f / p.dz;
        const bool p2 = pow2(p.dx) && pow2(p.dy) && pow2(p.dz);
        ta.k = dk;
        {
            std::vector<int> init(nshots, INT_MAX);
            CU(cudaMemcpyAsync(e->d_err, init.data(), sizeof(int) * nshots, cudaMemcpyHostToDevice, e->stream));
            CU(cudaMemsetAsync(e->d_tma_err, 0, sizeof(int), e->stream));
            CU(cudaStreamSynchronize(e->stream));  // init lives on the host stack
        }
        const int nb = 2 * 148, tb = 256;
        const dim3 grd_c((p.nz + BX - 1) / BX, (p.nx + BY - 1) / BY, p.ny);
        auto integrate = [&](float *u, const float *st, float *seg) { td_integrate(e, nshots, u, st, seg, seg_shot); };
        auto enqueue = [&]() {
            cudaMemsetAsync(dk, 0, (size_t)4 * n * sizeof(double), e->stream);
            if (!have_ck) {
                // 1. the forward again, a checkpoint after steps K, 2K, ... and the sums at NT
                cudaMemsetAsync(st2, 0, ss * sizeof(float), e->stream);
                cudaMemsetAsync(psi2, 0, ps * sizeof(float), e->stream);
                cudaMemsetAsync(uf, 0, us * sizeof(float), e->stream);
                for (int nt = 1; nt <= NT; ++nt) {
                    td_step(e, Lf, nt);
                    integrate(uf, st2, nullptr);
                    if (nt % K == 0 && nt / K < nseg) {
                        float *c = ckp + (size_t)(nt / K - 1) * ck;
                        hook_copy(e, c, st2, ss);
                        hook_copy(e, c + ss, psi2, ps);
                        hook_copy(e, c + ss + ps, uf, us);
                    }
                }
                hook_copy(e, uf_end, uf, us);
            }
            // 2. the adjoint, with each segment of forward steps recomputed as it is reached
            cudaMemsetAsync(e->d_state, 0, t.ssz * sizeof(float), e->stream);
            cudaMemsetAsync(e->d_psi, 0, t.psz * sizeof(float), e->stream);
            cudaMemsetAsync(ub, 0, us * sizeof(float), e->stream);
            int ntb = 1;  // next adjoint step
            for (int q = nseg - 1; q >= 0; --q) {
                const int a0 = q * K + 1, a1 = std::min((q + 1) * K, last);
                if (q == 0) {
                    cudaMemsetAsync(st2, 0, ss * sizeof(float), e->stream);
                    cudaMemsetAsync(psi2, 0, ps * sizeof(float), e->stream);
                    cudaMemsetAsync(uf, 0, us * sizeof(float), e->stream);
                } else {
                    const float *c = ckp + (size_t)(q - 1) * ck;
                    hook_copy(e, st2, c, ss);
                    hook_copy(e, psi2, c + ss, ps);
                    hook_copy(e, uf, c + ss + ps, us);
                }
                for (int m = a0; m <= a1; ++m) {  // v and U of each step go to the segment in the same pass
                    td_step(e, Lf, m);
                    integrate(uf, st2, segb + (size_t)(m - a0) * seg_shot * nshots);
                }
                for (int m = a1; m >= a0; --m, ++ntb) {  // adjoint steps P-a1 .. P-a0, in order
                    td_step(e, La, ntb);
                    integrate(ub, e->d_state, nullptr);
                    ta.seg = segb + (size_t)(m - a0) * seg_shot * nshots;
                    if (p2) k_td_corr<true><<<grd_c, dim3(BX, BY), 0, e->stream>>>(ta);
                    else k_td_corr<false><<<grd_c, dim3(BX, BY), 0, e->stream>>>(ta);
                }
            }
            for (; ntb <= NT; ++ntb) {  // adjoint steps past P-1 meet forward steps before the first (zero)
                td_step(e, La, ntb);
                integrate(ub, e->d_state, nullptr);
            }
            k_td_dc<<<nb, tb, 0, e->stream>>>(ta, uf_end);
        };
        e->hook_err = cudaSuccess;
        if (e->launch_mode == 1 || e->profile) {
            enqueue();
        } else {
            // the graph key: both loops, the kernels' arguments and the schedule
            std::vector<unsigned char> key(2 * sizeof(Loop) + sizeof(TdArgs) + 64);
            unsigned char *kp = key.data();
            std::memcpy(kp, &Lf, sizeof(Loop)); kp += sizeof(Loop);
            std::memcpy(kp, &La, sizeof(Loop)); kp += sizeof(Loop);
            std::memcpy(kp, &ta, sizeof(TdArgs)); kp += sizeof(TdArgs);
            const long long sched[8] = {K, nseg, last, NT, have_ck ? 1 : 0, (long long)(uintptr_t)blk, nshots, 0};
            std::memcpy(kp, sched, sizeof(sched));
            if ((r = replay_graph(e, e->gtd, key, enqueue))) return r;
        }
        if ((r = check_launch(e, "time-domain loops"))) return r;
        if (e->hook_err != cudaSuccess)
            return fail(e, IFOSB_ECUDA, std::string("time-domain copies: ") + cudaGetErrorString(e->hook_err));
        if ((r = check_unstable(e, nshots))) return r;
        CU(cudaMemcpyAsync(kernels, dk, (size_t)4 * n * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
        CU(cudaStreamSynchronize(e->stream));
        // the checkpoints stay in the block (the segments only read them): a repeat
        // call for this forward starts from them
        e->td_ck_ok = true;
        e->td_ck_K = K;
        e->td_ck_nshots = nshots;
        return IFOSB_OK;
    };
    e->td_ck_ok = false;  // a failure below leaves the block undefined
    rc = run();
    cudaStreamSynchronize(e->stream);
    return rc;
}

// ---------------------------------------------------------------------------
// Exact discrete VJP (ifosb_vjp.cuh): the FP64 forward of each shot of the last
// batch with a checkpoint every `interval` steps, the misfit and its adjoint
// source from the residual's observed traces, then the transposed steps in
// reverse, each segment of forward states recomputed from its checkpoint. The
// gradient comes out with respect to the raw model ifosb_set_model received,
// interior cells, [5][NY*NX*NZ]: rho, pi, u, taus, taup (the last two zero for
// L = 0).
static int vjp_exact_moduli(ifosb_engine *e, int interval, double *gmod, double *misfit) {
    if (!e || !misfit || interval < 1) return IFOSB_EARG;
    const ifosb_params &p = e->p;
    if (!e->fwd_ok || !e->res_ok) return fail(e, IFOSB_ESTATE, "the exact VJP needs a forward batch and its residual");
    if (p.ndt != 1 || p.ndtshift != 0) return fail(e, IFOSB_EARG, "the exact VJP samples every step: NDT=1, NDTSHIFT=0");
    if (!e->td_vp.empty()) return fail(e, IFOSB_EARG, "the exact VJP takes explosive sources only");
    const Geo g = e->g;
    const int NT = p.nt, ns = e->ns, ntr = e->ntr, nshots = e->nshots;
    if (ntr < 1) return fail(e, IFOSB_ESTATE, "the exact VJP needs receivers");
    const int K = std::min(interval, NT), nseg = (NT + K - 1) / K;
    const long long F = g.field, n = (long long)p.nx * p.ny * p.nz;
    const int L = p.nmech, NELV = NEL + 6 * L;                       // fields, then L x 6 memory variables
    const size_t SZ = (size_t)NELV * F + (size_t)e->psi_shot;  // one FP64 state: those, then PML memory
    const size_t ntrace = (size_t)3 * ntr * ns;
    // device block: model | checkpoints | segment | adjoint state | ld | ls | gradients | traces | source
    const size_t total = (size_t)N64 * F + (size_t)nseg * SZ + (size_t)(K + 1) * SZ + SZ + 18 * (size_t)F +
                         (size_t)N64 * n + 2 * ntrace;
    double *blk = nullptr;
    int *ibuf = nullptr;
    double *damp = nullptr;
    CU(cudaMalloc(&blk, total * sizeof(double)));
    double *md = blk, *ck = md + (size_t)N64 * F, *seg = ck + (size_t)nseg * SZ, *lam = seg + (size_t)(K + 1) * SZ;
    double *ld = lam + SZ, *ls = ld + 9 * (size_t)F, *gq = ls + 9 * (size_t)F, *tr = gq + (size_t)N64 * n;
    double *asrc = tr + ntrace;
    int rc = IFOSB_OK;
    auto run = [&]() -> int {
        CU(cudaMemsetAsync(blk, 0, total * sizeof(double), e->stream));
        const size_t ng = (size_t)(p.nx + 2) * (p.ny + 2) * (p.nz + 2);
        const float *raw = e->d_mstage;  // rho, pi, u, taus, taup as ifosb_set_model received them (ghosted)
        const dim3 blk3(128), grd3((p.nz + 127) / 128, p.nx, p.ny);
        k64_model<<<grd3, blk3, 0, e->stream>>>(g, raw, raw + ng, raw + 2 * ng, L ? raw + 3 * ng : nullptr,
                                                 L ? raw + 4 * ng : nullptr, md);
        Vjp64 a{};
        a.g = g;
        a.sl = e->sl;
        a.md = md;
        a.cpg = e->d_cpg;
        a.b1 = e->b1; a.b2 = e->b2;
        a.dx = (double)p.dt / p.dx; a.dy = (double)p.dt / p.dy; a.dz = (double)p.dt / p.dz;
        a.rdx = p.dx; a.rdy = p.dy; a.rdz = p.dz; a.dt = p.dt;
        a.nt_total = NT;
        a.nmech = L;
        for (int l = 0; l < L; ++l) {  // update_s_ssg.c:123-124, surface_ssg.c:152, in double
            const double eta = e->eta[l];
            a.eta[l] = eta;
            a.bb[l] = 1.0 / (1.0 + eta * 0.5);
            a.cc[l] = 1.0 - eta * 0.5;
            a.msb[l] = eta / (1.0 + eta * 0.5);
        }
        Grad64 gr;
        for (int q = 0; q < N64; ++q) gr.q[q] = gq + (size_t)q * n;
        std::vector<int> rec(e->rec.begin(), e->rec.end());
        std::vector<float> obs((size_t)nshots * ntrace);
        CU(cudaMemcpyAsync(obs.data(), e->d_obs, obs.size() * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
        CU(cudaStreamSynchronize(e->stream));
        std::vector<double> trh(ntrace), src(ntrace);
        const double DT = p.dt;
        for (int sh = 0; sh < nshots; ++sh) {
            // explosive sources of this shot: cell and psource amplitude row
            std::vector<int> cells;
            std::vector<double> amps;
            for (const HostPt &pt : e->td_sp)
                if (pt.s == sh && pt.kind == PT_EXPLOSIVE) {
                    cells.insert(cells.end(), {pt.j, pt.i, pt.k});
                    for (int t = 0; t < NT; ++t) amps.push_back(e->td_amp[(size_t)pt.row * NT + t]);
                }
            const int nsrc = (int)cells.size() / 3;
            if (ibuf) cudaFree(ibuf);
            if (damp) cudaFree(damp);
            ibuf = nullptr;
            damp = nullptr;
            CU(cudaMalloc(&ibuf, sizeof(int) * (3 * (size_t)ntr + 3 * (size_t)std::max(nsrc, 1))));
            CU(cudaMalloc(&damp, sizeof(double) * std::max<size_t>(amps.size(), 1)));
            int *drec = ibuf, *dsrc = ibuf + 3 * ntr;
            CU(cudaMemcpyAsync(drec, rec.data(), sizeof(int) * 3 * ntr, cudaMemcpyHostToDevice, e->stream));
            if (nsrc) {
                CU(cudaMemcpyAsync(dsrc, cells.data(), sizeof(int) * cells.size(), cudaMemcpyHostToDevice, e->stream));
                CU(cudaMemcpyAsync(damp, amps.data(), sizeof(double) * amps.size(), cudaMemcpyHostToDevice, e->stream));
            }
            a.nsrc = nsrc;
            a.src = dsrc;
            a.amp = damp;
            auto step = [&](double *st, int nt) {
                double *ps = st + (size_t)NELV * F;
                k64_vel<<<grd3, blk3, 0, e->stream>>>(a, st, ps);
                k64_str<<<grd3, blk3, 0, e->stream>>>(a, st, ps, nt);
            };
            // 1. the forward from rest, checkpoints after steps 0, K, 2K, ..., the traces
            double *w = seg;
            CU(cudaMemsetAsync(w, 0, SZ * sizeof(double), e->stream));
            CU(cudaMemsetAsync(ck, 0, SZ * sizeof(double), e->stream));
            for (int nt = 1; nt <= NT; ++nt) {
                step(w, nt);
                k64_sample<<<(ntr + 127) / 128, 128, 0, e->stream>>>(g, w, drec, ntr, ns, nt - 1, tr);
                if (nt % K == 0 && nt / K < nseg)
                    CU(cudaMemcpyAsync(ck + (size_t)(nt / K) * SZ, w, SZ * sizeof(double), cudaMemcpyDeviceToDevice,
                                       e->stream));
            }
            int r;
            if ((r = check_launch(e, "exact VJP forward"))) return r;
            CU(cudaMemcpyAsync(trh.data(), tr, ntrace * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
            CU(cudaStreamSynchronize(e->stream));
            // 2. the misfit sum D^2, D = DT cumsum(syn - obs), and its derivative
            //    2 DT sum_{n >= k} D[n] with respect to each sample
            double J = 0.0;
            const float *ob = obs.data() + (size_t)sh * ntrace;
            for (size_t t = 0; t < (size_t)3 * ntr; ++t) {
                const double *sy = trh.data() + t * ns;
                const float *o = ob + t * ns;
                std::vector<double> D(ns);
                double run_sum = 0.0;
                for (int k = 0; k < ns; ++k) {
                    run_sum += sy[k] - (double)o[k];
                    D[k] = DT * run_sum;
                    J += D[k] * D[k];
                }
                double tail = 0.0;
                for (int k = ns - 1; k >= 0; --k) {
                    tail += D[k];
                    src[t * ns + k] = 2.0 * DT * tail;
                }
            }
            misfit[sh] = J;
            if (!gmod) continue;
            CU(cudaMemcpyAsync(asrc, src.data(), ntrace * sizeof(double), cudaMemcpyHostToDevice, e->stream));
            // 3. the transposed steps, last to first, each segment recomputed from its checkpoint
            CU(cudaMemsetAsync(lam, 0, SZ * sizeof(double), e->stream));
            CU(cudaMemsetAsync(ld, 0, 18 * (size_t)F * sizeof(double), e->stream));
            double *lps = lam + (size_t)NELV * F;
            const dim3 grdg((p.nz + 127) / 128, p.nx, p.ny + (g.free_surf ? 2 : 0));
            const dim3 grds((p.nz + 127) / 128, p.nx);
            for (int q = nseg - 1; q >= 0; --q) {
                const int a0 = q * K + 1, a1 = std::min((q + 1) * K, NT);
                CU(cudaMemcpyAsync(seg, ck + (size_t)q * SZ, SZ * sizeof(double), cudaMemcpyDeviceToDevice, e->stream));
                for (int nt = a0; nt <= a1; ++nt) {
                    double *cur = seg + (size_t)(nt - a0 + 1) * SZ;
                    CU(cudaMemcpyAsync(cur, cur - SZ, SZ * sizeof(double), cudaMemcpyDeviceToDevice, e->stream));
                    step(cur, nt);
                }
                for (int nt = a1; nt >= a0; --nt) {
                    const double *cur = seg + (size_t)(nt - a0 + 1) * SZ, *prev = cur - SZ;
                    k64_inject<<<(ntr + 127) / 128, 128, 0, e->stream>>>(g, lam, drec, ntr, ns, nt - 1, asrc);
                    if (g.free_surf) k64_mirror_T<<<grds, blk3, 0, e->stream>>>(g, lam);
                    k64_str_T<<<grd3, blk3, 0, e->stream>>>(a, lam, lps, ld, cur, prev + (size_t)NELV * F, gr);
                    k64_str_T_gather<<<grd3, blk3, 0, e->stream>>>(a, lam, ld);
                    k64_vel_T<<<grd3, blk3, 0, e->stream>>>(a, lam, lps, ls, cur, prev, gr);
                    k64_vel_T_gather<<<grdg, blk3, 0, e->stream>>>(a, lam, ls, g.free_surf ? -1 : 1);
                }
                if ((r = check_launch(e, "exact VJP adjoint"))) return r;
            }
        }
        if (!gmod) return IFOSB_OK;
        // 4. the averaged moduli's gradients onto the raw model (av_mat.c:45-69 and
        //    matcopy's periodic ghost layers)
        std::vector<double> gh((size_t)N64 * n);
        std::vector<float> rawh(3 * ng);
        CU(cudaMemcpyAsync(gh.data(), gq, gh.size() * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
        CU(cudaMemcpyAsync(rawh.data(), raw, rawh.size() * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
        CU(cudaStreamSynchronize(e->stream));
        const int NX = p.nx, NY = p.ny, NZ = p.nz, GX = NX + 2, GZ = NZ + 2;
        auto G = [&](int j, int i, int k) { return ((size_t)j * GX + i) * GZ + k; };
        const float *u = rawh.data() + 2 * ng;
        // ghosted accumulators in the order of the output: rho, pi, u, taus, taup
        std::vector<double> acc(5 * ng, 0.0);
        double *dr = acc.data(), *dp = dr + ng, *du = dp + ng, *dts = du + ng, *dtp = dts + ng;
        auto harm = [&](double gval, int j0, int i0, int k0, int j1, int i1, int k1, int j2, int i2, int k2, int j3,
                        int i3, int k3) {
            const size_t c[4] = {G(j0, i0, k0), G(j1, i1, k1), G(j2, i2, k2), G(j3, i3, k3)};
            double s = 0.0;
            for (size_t q : c) s += 1.0 / (double)u[q];
            const double avg = 4.0 / s;
            for (size_t q : c) du[q] += gval * avg * avg / (4.0 * (double)u[q] * (double)u[q]);
        };
        auto quarter = [&](double gval, int j0, int i0, int k0, int j1, int i1, int k1, int j2, int i2, int k2, int j3,
                           int i3, int k3) {
            dts[G(j0, i0, k0)] += 0.25 * gval; dts[G(j1, i1, k1)] += 0.25 * gval;
            dts[G(j2, i2, k2)] += 0.25 * gval; dts[G(j3, i3, k3)] += 0.25 * gval;
        };
        for (int j = 1; j <= NY; ++j)
            for (int i = 1; i <= NX; ++i)
                for (int k = 1; k <= NZ; ++k) {
                    const size_t m = ((size_t)(j - 1) * NX + (i - 1)) * NZ + (k - 1), c = G(j, i, k);
                    auto gv = [&](int q) { return gh[(size_t)q * n + m]; };
                    dp[c] += gv(M64_PI);
                    du[c] += gv(M64_U);
                    dr[c] += 0.5 * gv(M64_RIP); dr[G(j, i + 1, k)] += 0.5 * gv(M64_RIP);
                    dr[c] += 0.5 * gv(M64_RJP); dr[G(j + 1, i, k)] += 0.5 * gv(M64_RJP);
                    dr[c] += 0.5 * gv(M64_RKP); dr[G(j, i, k + 1)] += 0.5 * gv(M64_RKP);
                    harm(gv(M64_UIPJP), j, i, k, j, i + 1, k, j + 1, i + 1, k, j + 1, i, k);
                    harm(gv(M64_UJPKP), j, i, k, j, i, k + 1, j + 1, i, k + 1, j + 1, i, k);
                    harm(gv(M64_UIPKP), j, i, k, j, i, k + 1, j, i + 1, k + 1, j, i + 1, k);
                    if (L) {  // tausipjp ... are plain means of four cells (av_mat.c:57-59)
                        dts[c] += gv(M64_TAUS);
                        dtp[c] += gv(M64_TAUP);
                        quarter(gv(M64_TSIPJP), j, i, k, j, i + 1, k, j + 1, i + 1, k, j + 1, i, k);
                        quarter(gv(M64_TSJPKP), j, i, k, j + 1, i, k, j + 1, i, k + 1, j, i, k + 1);
                        quarter(gv(M64_TSIPKP), j, i, k, j, i + 1, k, j, i + 1, k + 1, j, i, k + 1);
                    }
                }
        // fold the ghost layers (matcopy on one rank: index 0 = N, N + 1 = 1)
        auto wrapi = [](int x, int N) { return x == 0 ? N : (x == N + 1 ? 1 : x); };
        std::fill(gmod, gmod + 5 * n, 0.0);
        for (int j = 0; j <= NY + 1; ++j)
            for (int i = 0; i <= NX + 1; ++i)
                for (int k = 0; k <= NZ + 1; ++k) {
                    const size_t c = G(j, i, k);
                    const size_t m = ((size_t)(wrapi(j, NY) - 1) * NX + (wrapi(i, NX) - 1)) * NZ + (wrapi(k, NZ) - 1);
                    for (int q = 0; q < 5; ++q) gmod[(size_t)q * n + m] += acc[(size_t)q * ng + c];
                }
        return IFOSB_OK;
    };
    rc = run();
    cudaStreamSynchronize(e->stream);
    cudaFree(blk);
    if (ibuf) cudaFree(ibuf);
    if (damp) cudaFree(damp);
    return rc;
}

extern "C" int ifosb_vjp_exact_moduli(ifosb_engine *e, int interval, double *grad, double *misfit) {
    return vjp_exact_moduli(e, interval, grad, misfit);
}

// The elastic form: the moduli gradient through pi = rho vp^2, u = rho vs^2
// (readmod.c with L = 0) onto vp, vs, rho, [3][NY*NX*NZ].
extern "C" int ifosb_vjp_exact(ifosb_engine *e, int interval, double *grad, double *misfit) {
    if (!e || !misfit || interval < 1) return IFOSB_EARG;
    const ifosb_params &p = e->p;
    if (p.nmech != 0)
        return fail(e, IFOSB_EARG, "the (vp, vs, rho) form is elastic; ifosb_vjp_exact_moduli takes L > 0");
    if (!grad) return vjp_exact_moduli(e, interval, nullptr, misfit);
    const size_t n = (size_t)p.nx * p.ny * p.nz, ng = (size_t)(p.nx + 2) * (p.ny + 2) * (p.nz + 2);
    std::vector<double> gm(5 * n);
    int rc = vjp_exact_moduli(e, interval, gm.data(), misfit);
    if (rc) return rc;
    std::vector<float> rawh(3 * ng);
    CU(cudaMemcpy(rawh.data(), e->d_mstage, rawh.size() * sizeof(float), cudaMemcpyDeviceToHost));
    const int NX = p.nx, NY = p.ny, NZ = p.nz, GX = NX + 2, GZ = NZ + 2;
    const float *rho = rawh.data(), *pi = rho + ng, *u = pi + ng;
    const double *fr = gm.data(), *fp = fr + n, *fu = fp + n;
    for (int j = 1; j <= NY; ++j)
        for (int i = 1; i <= NX; ++i)
            for (int k = 1; k <= NZ; ++k) {
                const size_t m = ((size_t)(j - 1) * NX + (i - 1)) * NZ + (k - 1), c = ((size_t)j * GX + i) * GZ + k;
                const double r = rho[c], vp = std::sqrt((double)pi[c] / r), vs = std::sqrt((double)u[c] / r);
                grad[m] = fp[m] * 2.0 * r * vp;
                grad[n + m] = fu[m] * 2.0 * r * vs;
                grad[2 * n + m] = fr[m] + fp[m] * vp * vp + fu[m] * vs * vs;
            }
    return IFOSB_OK;
}

// ---------------------------------------------------------------------------
// Approximate Hessian (hess_F.c, and the Hessian wavefields of ifos3d.c:882-938).
// The Green's function of receiver r is the wavefield of a y-directed velocity
// injection of `signal` at the receiver, propagated like an adjoint wavefield
// (update_v with back = 1, elastic stress update) with the backward DFT. Each
// is computed once per model and frequency set and kept on the device; a
// batch of them runs as one multi-shot adjoint launch.
extern "C" int ifosb_hessian_green(ifosb_engine *e, int nrec, const int *rec_ids, const float *signals) {
    if (!e || nrec < 1 || !rec_ids || !signals) return IFOSB_EARG;
    const ifosb_params &p = e->p;
    if (!e->have_model || !e->have_cpml) return fail(e, IFOSB_ESTATE, "Green's functions need a model and CPML");
    if (p.nmech != 0) return fail(e, IFOSB_EARG, "the Hessian wavefields are elastic (ifos3d.c:929): nmech must be 0");
    if (e->nf == 0) return fail(e, IFOSB_ESTATE, "Green's functions need DFT frequencies");
    if (p.ndt != 1 || p.ndtshift != 0)
        return fail(e, IFOSB_EARG, "the injection indexes its trace by time step: NDT=1, NDTSHIFT=0");
    for (int q = 0; q < nrec; ++q)
        if (rec_ids[q] < 0 || rec_ids[q] >= e->ntr) return fail(e, IFOSB_EARG, "receiver index out of range");
    int rc;
    if (nrec > e->cap_green) {
        dfree(e, &e->d_green, (size_t)e->dft_shot * e->cap_green);
        e->cap_green = 0;
        if ((rc = dalloc(e, &e->d_green, (size_t)e->dft_shot * nrec))) return rc;
        e->cap_green = nrec;
    }
    e->ngreen = 0;
    const int NT = p.nt, B0 = e->max_shots;
    if (!e->d_gsig && (rc = dalloc(e, &e->d_gsig, (size_t)B0 * 3 * NT))) return rc;
    std::vector<float> sig((size_t)B0 * 3 * NT, 0.0f);
    for (int q0 = 0; q0 < nrec; q0 += B0) {
        const int B = std::min(B0, nrec - q0);
        for (int b = 0; b < B; ++b)  // vx and vz stay 0, vy is the receiver's signal
            std::memcpy(&sig[((size_t)b * 3 + 1) * NT], signals + (size_t)(q0 + b) * NT, sizeof(float) * NT);
        CU(cudaMemcpyAsync(e->d_gsig, sig.data(), sizeof(float) * (size_t)B * 3 * NT, cudaMemcpyHostToDevice, e->stream));
        CU(cudaStreamSynchronize(e->stream));  // sig is reused by the next batch
        std::vector<HostPt> vp;
        for (int b = 0; b < B; ++b) {
            const int t = rec_ids[q0 + b];
            vp.push_back({b, e->rec[3 * t + 1], e->rec[3 * t], e->rec[3 * t + 2], PT_ADJOINT, b * 3});
        }
        float *dft = e->d_green + (long long)q0 * e->dft_shot;
        Loop L;
        std::memset(static_cast<void *>(&L), 0, sizeof(L));  // the graph cache compares Loops bytewise
        L.nshots = B;
        L.back = true;
        L.lg = launch_geo(e, B, false);
        L.lgv = launch_geo(e, B, true);
        if ((rc = upload_points(e, L.lgv, B, vp, &e->d_voff, &e->cap_voff, &e->d_vpts, &e->cap_vpts))) return rc;
        if ((rc = reset_state(e, B, dft))) return rc;
        fill_common(e, L);
        L.va.pt_off = e->d_voff;
        L.va.pts = e->d_vpts;
        L.va.val = e->d_gsig;  // entry b: vx, vy, vz traces at b*3*NT
        L.va.val_row = NT;
        L.va.val_comp = NT;
        L.sa.pt_off = nullptr;
        L.sa.pts = nullptr;
        L.sa.dft = dft;
        L.sa.trig = e->d_trig_b;
        L.tma = e->use_tma && setup_tma(e, L, dft);
        if ((rc = run_loop(e, L))) return rc;
        if ((rc = check_unstable(e, B))) return rc;
    }
    e->ngreen = nrec;
    e->fwd_ok = e->res_ok = e->adj_ok = false;  // the wavefield state now holds the last Green's function
    return check_launch(e, "hessian_green");
}

// hess_F for the shots of the last forward batch against every stored Green's function.
extern "C" int ifosb_hessian(ifosb_engine *e) {
    if (!e) return IFOSB_EARG;
    if (e->ngreen == 0) return fail(e, IFOSB_ESTATE, "hessian needs ifosb_hessian_green first");
    if (e->nshots < 1 || e->nf == 0 || !e->hess_fwd) return fail(e, IFOSB_ESTATE, "hessian needs a forward batch with DFT");
    const ifosb_params &p = e->p;
    int rc;
    if (!e->d_hess) {
        if ((rc = dalloc(e, &e->d_hess, (size_t)3 * p.nx * p.ny * p.nz))) return rc;
        CU(cudaMemsetAsync(e->d_hess, 0, sizeof(float) * 3 * p.nx * p.ny * p.nz, e->stream));
    }
    HessArgs a{};
    a.g = e->g;
    a.dftf = e->d_dftf;
    a.dft_shot = e->dft_shot;
    a.green = e->d_green;
    a.nshots = e->nshots;
    a.nrec = e->ngreen;
    a.nf = e->nf;
    a.md = e->d_model;
    a.rho = e->d_rho_w;
    for (int l = 0; l < e->nf; ++l) {
        float fdummy = 0.0;
        fdummy = e->finv[l] * M_PI * 2;  // hess_F.c:72-74
        fdummy = 1 / fdummy;
        a.fdummy[l] = fdummy;
    }
    a.b1 = e->b1; a.b2 = e->b2;
    a.rdx = p.dx; a.rdy = p.dy; a.rdz = p.dz;
    a.ihx = 1.0f / p.dx; a.ihy = 1.0f / p.dy; a.ihz = 1.0f / p.dz;
    a.hess = e->d_hess;
    dim3 blk(BX, BY), grd(e->g.ntk, e->g.nti, e->g.nyc);
    if (pow2(p.dx) && pow2(p.dy) && pow2(p.dz)) k_hessian<true><<<grd, blk, 0, e->stream>>>(a);
    else k_hessian<false><<<grd, blk, 0, e->stream>>>(a);
    if ((rc = check_launch(e, "hessian"))) return rc;
    CU(cudaStreamSynchronize(e->stream));
    e->hess_fwd = false;  // one contribution per forward batch
    return IFOSB_OK;
}

extern "C" int ifosb_zero_hessian(ifosb_engine *e) {
    if (!e) return IFOSB_EARG;
    const size_t n = (size_t)3 * e->p.nx * e->p.ny * e->p.nz;
    int rc;
    if (!e->d_hess && (rc = dalloc(e, &e->d_hess, n))) return rc;
    CU(cudaMemsetAsync(e->d_hess, 0, n * sizeof(float), e->stream));
    CU(cudaStreamSynchronize(e->stream));
    return IFOSB_OK;
}

extern "C" int ifosb_get_hessian(ifosb_engine *e, float *hess) {
    if (!e || !hess) return IFOSB_EARG;
    const size_t n = (size_t)3 * e->p.nx * e->p.ny * e->p.nz;
    if (!e->d_hess) {
        std::memset(hess, 0, n * sizeof(float));
        return IFOSB_OK;
    }
    CU(cudaMemcpyAsync(hess, e->d_hess, n * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
    CU(cudaStreamSynchronize(e->stream));
    return IFOSB_OK;
}

extern "C" int ifosb_zero_gradient(ifosb_engine *e) {
    if (!e) return IFOSB_EARG;
    const size_t n = (size_t)3 * e->p.nx * e->p.ny * e->p.nz;
    CU(cudaMemsetAsync(e->d_grad, 0, n * sizeof(float), e->stream));
    CU(cudaMemsetAsync(e->d_grad64, 0, n * sizeof(double), e->stream));
    if (e->d_gradq) CU(cudaMemsetAsync(e->d_gradq, 0, n / 3 * 2 * sizeof(double), e->stream));
    CU(cudaStreamSynchronize(e->stream));
    return IFOSB_OK;
}

extern "C" int ifosb_get_gradient_q(ifosb_engine *e, double *gradq) {
    if (!e || !gradq) return IFOSB_EARG;
    if (!e->d_gradq) return fail(e, IFOSB_ESTATE, "the Q gradient needs a viscoelastic engine (nmech > 0)");
    const size_t n = (size_t)2 * e->p.nx * e->p.ny * e->p.nz;
    CU(cudaMemcpyAsync(gradq, e->d_gradq, n * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    CU(cudaStreamSynchronize(e->stream));
    return IFOSB_OK;
}

extern "C" int ifosb_get_gradient(ifosb_engine *e, float *grad, double *grad64) {
    if (!e) return IFOSB_EARG;
    const size_t n = (size_t)3 * e->p.nx * e->p.ny * e->p.nz;
    // host or device destinations (unified addressing)
    if (grad) CU(cudaMemcpyAsync(grad, e->d_grad, n * sizeof(float), cudaMemcpyDefault, e->stream));
    if (grad64) CU(cudaMemcpyAsync(grad64, e->d_grad64, n * sizeof(double), cudaMemcpyDefault, e->stream));
    CU(cudaStreamSynchronize(e->stream));
    return IFOSB_OK;
}

extern "C" int ifosb_shot_gradient(ifosb_engine *e, int nshots, const ifosb_shot *shots, const float *obs, double *misfit) {
    int rc;
    if ((rc = ifosb_forward(e, nshots, shots, nullptr))) return rc;
    if ((rc = ifosb_residual(e, obs, misfit, nullptr))) return rc;
    if ((rc = ifosb_adjoint(e, nullptr))) return rc;
    return ifosb_gradient(e);
}

extern "C" int ifosb_get_field(ifosb_engine *e, int shot, int field, float *out) {
    if (!e || !out || shot < 0 || shot >= std::max(e->nshots, 1)) return IFOSB_EARG;
    const ifosb_params &p = e->p;
    const Geo &g = e->g;
    const float *src = nullptr;
    // IFOSB_F_* ids follow the reference's vx, vy, vz, sxx, syy, szz, sxy, syz, sxz
    static const int slot_of[NEL] = {VX, VY, VZ, SXX, SYY, SZZ, SXY, SYZ, SXZ};
    if (field >= 0 && field < NEL) {
        src = e->d_state + (long long)shot * e->st_shot + (long long)slot_of[field] * g.field;
    } else if (field >= IFOSB_F_DFT_FWD && field < IFOSB_F_DFT_FWD + 6 * e->nf && e->d_dftf) {
        const int q = field - IFOSB_F_DFT_FWD, comp = q / e->nf, l = q % e->nf;
        src = e->d_dftf + (long long)shot * e->dft_shot + ((long long)l * 6 + comp) * g.field;
    } else if (field >= IFOSB_F_DFT_BACK && field < IFOSB_F_DFT_BACK + 6 * e->nf && e->d_dftb) {
        const int q = field - IFOSB_F_DFT_BACK, comp = q / e->nf, l = q % e->nf;
        src = e->d_dftb + (long long)shot * e->dft_shot + ((long long)l * 6 + comp) * g.field;
    } else {
        return fail(e, IFOSB_EARG, "unknown field id");
    }
    // device rows start at k=-1 (offset 6); host rows are NZ+4 wide
    CU(cudaMemcpy2D(out, sizeof(float) * (p.nz + 4), src + 6, sizeof(float) * g.pz, sizeof(float) * (p.nz + 4),
                    (size_t)(p.ny + 5) * (p.nx + 4), cudaMemcpyDeviceToHost));
    return IFOSB_OK;
}

// ---------------------------------------------------------------------------
// ifosb_residual_noalloc: the residual and FP64 misfit of ifosb_residual on the
// caller's device buffers and stream, with the per-trace partial sums in a
// fixed file-scope device array instead of engine memory. It runs the same two
// kernels (k_residual, k_misfit) as ifosb_residual, so the results are the same
// bits. Every scratch word that k_misfit reads is written by k_residual earlier
// in the same call, so nothing has to be cleared between calls.
static __device__ __align__(256) double g_noalloc_part[IFOSB_NOALLOC_MAX_TRACES];

namespace {
constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
// Address of g_noalloc_part on each device, with the context it was looked up
// in: a module loaded into a new context (after cudaDeviceReset, say) may place
// the array elsewhere, so a changed context means a fresh lookup.
struct NoallocSlot {
    CUcontext ctx;
    double *addr;
};
NoallocSlot g_noalloc_slot[NOALLOC_MAX_DEVICES];

PFN_cuCtxGetCurrent_v4000 ctx_getter() {
    static PFN_cuCtxGetCurrent_v4000 fn = nullptr;
    if (!fn) {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuCtxGetCurrent_v4000)f;
    }
    return fn;
}

bool overlaps(const void *a, const void *b, size_t bytes) {
    const char *x = static_cast<const char *>(a), *y = static_cast<const char *>(b);
    return x < y + bytes && y < x + bytes;
}
}  // namespace

extern "C" int ifosb_residual_noalloc(int nshots, int ntr, int ns, float dt, const float *d_syn, const float *d_obs,
                                      float *d_diff, double *d_misfit, void *stream) {
    if (nshots < 1 || ntr < 1 || ns < 1 || !d_syn || !d_obs || !d_diff || !d_misfit) return IFOSB_EARG;
    if ((long long)nshots * 3 * ntr > IFOSB_NOALLOC_MAX_TRACES) return IFOSB_ETOOBIG;
    // k_residual writes diff[ns-1-t] while it reads syn[t] and obs[t] forward:
    // an output that overlaps an input would be read after it was overwritten
    const size_t bytes = (size_t)nshots * 3 * ntr * ns * sizeof(float);
    if (overlaps(d_diff, d_syn, bytes) || overlaps(d_diff, d_obs, bytes)) return IFOSB_EARG;
    // an error the caller left pending on this thread stays theirs: report it, do not clear it
    if (cudaPeekAtLastError() != cudaSuccess) return IFOSB_ECUDA;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return IFOSB_ENODEV;
    }
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return IFOSB_EARG;
    double *part;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        CUcontext ctx = nullptr;
        auto get_ctx = ctx_getter();
        if (!get_ctx || get_ctx(&ctx) != CUDA_SUCCESS) return IFOSB_ECUDA;
        NoallocSlot &slot = g_noalloc_slot[dev];
        if (!slot.addr || slot.ctx != ctx) {
            void *addr = nullptr;
            if (cudaGetSymbolAddress(&addr, g_noalloc_part) != cudaSuccess || !addr) {
                cudaGetLastError();
                slot.addr = nullptr;
                return IFOSB_ECUDA;
            }
            slot.addr = static_cast<double *>(addr);
            slot.ctx = ctx;
        }
        part = slot.addr;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int nthr = nshots * 3 * ntr;
    k_residual<<<(nthr + 127) / 128, 128, 0, s>>>(d_syn, d_obs, d_diff, part, nshots, ntr, ns, dt);
    if (cudaGetLastError() != cudaSuccess) return IFOSB_ECUDA;
    k_misfit<<<nshots, 32, 0, s>>>(part, d_misfit, 3 * ntr);
    return cudaGetLastError() == cudaSuccess ? IFOSB_OK : IFOSB_ECUDA;
}

// Autotuner: for a batch of nshots shots, times `steps` forward time steps
// (kernel-by-kernel, CUDA events) for each launch shape — y planes per CTA chunk
// and the L2 prefetch distance of the TMA kernels — and keeps the fastest for
// later calls with that batch size. The shape changes no arithmetic: results
// stay bit-identical. The wavefield of the batch is left undefined.
extern "C" int ifosb_autotune(ifosb_engine *e, int nshots, const ifosb_shot *shots, int steps, int *shape) {
    if (!e || !shots || nshots < 1 || nshots > e->max_shots || steps < 1) return IFOSB_EARG;
    const int saved_profile = e->profile;
    e->tuned.erase(nshots);
    const Geo hv = launch_geo(e, nshots, true), hs = launch_geo(e, nshots, false);  // built-in choices
    std::vector<int> cys = {2, 3, 4, 6, 8, 12, 16, 24, 32, 64, hv.cy, hs.cy};
    {
        // chunkings whose CTA count fills one or two waves at 1-4 CTAs per SM: on
        // a small grid the fixed list leaves either a nearly empty last wave or
        // chunks so short that each CTA's pipeline start-up dominates
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaGetLastError();
        for (const Geo *lg : {&hv, &hs}) {
            const long long per_set = (long long)lg->ntk * lg->nti * nshots;
            for (int per_sm = 1; per_sm <= 4; ++per_sm)
                for (int waves = 1; waves <= 2; ++waves) {
                    const long long nyc = (long long)waves * per_sm * sms / per_set;
                    if (nyc < 1) continue;
                    const int cy = (int)((e->p.ny + nyc - 1) / nyc);
                    if (cy >= 2) cys.push_back(cy);
                }
        }
    }
    std::sort(cys.begin(), cys.end());
    cys.erase(std::unique(cys.begin(), cys.end()), cys.end());
    double bv = 1e30, bs = 1e30;
    const ifosb_engine::Shape *near = shape_for(e, nshots);
    ifosb_engine::Shape pick{hv.cy, near ? near->l2v : L2AHEAD_VEL_DEFAULT, hs.cy,
                             near ? near->l2s : L2AHEAD_STR_DEFAULT};
    int rc = IFOSB_OK;
    e->profile = 1;
    e->nt_limit = steps;
    for (int cy : cys) {
        if (cy > e->p.ny || (long long)((e->p.ny + cy - 1) / cy) * nshots > 65535) continue;
        for (int l2 : {0, 1, 2, 3}) {
            e->tuned[nshots] = {cy, l2, cy, l2};
            if ((rc = ifosb_forward(e, nshots, shots, nullptr))) break;
            // the two kernels are timed separately: each keeps its own best shape
            if (e->t_vel_ms < bv) { bv = e->t_vel_ms; pick.cyv = cy; pick.l2v = l2; }
            if (e->t_str_ms < bs) { bs = e->t_str_ms; pick.cys = cy; pick.l2s = l2; }
        }
        if (rc) break;
    }
    e->nt_limit = 0;
    e->profile = saved_profile;
    e->fwd_ok = e->res_ok = e->adj_ok = false;
    if (rc) {
        e->tuned.erase(nshots);
        return rc;
    }
    e->tuned[nshots] = pick;
    release_graph(e->gfwd);
    release_graph(e->gadj);
    release_graph(e->gtd);
    if (shape) {
        shape[0] = pick.cyv;
        shape[1] = pick.l2v;
        shape[2] = pick.cys;
        shape[3] = pick.l2s;
    }
    return IFOSB_OK;
}

// Sets the launch shapes for batches of nshots shots (as ifosb_autotune leaves
// them): shape[4] = velocity kernel y planes per chunk and L2 prefetch distance,
// then the stress kernel's. Lets a caller reuse a tuned shape without re-timing.
extern "C" int ifosb_set_launch_shape(ifosb_engine *e, int nshots, const int *shape) {
    if (!e || !shape || nshots < 1 || nshots > e->max_shots) return IFOSB_EARG;
    for (int q : {0, 2})
        if (shape[q] < 1 || shape[q] > e->p.ny || (long long)((e->p.ny + shape[q] - 1) / shape[q]) * nshots > 65535)
            return fail(e, IFOSB_EARG, "y planes per chunk out of range");
    for (int q : {1, 3})
        if (shape[q] < 0 || shape[q] > 8) return fail(e, IFOSB_EARG, "L2 prefetch distance out of range (0-8)");
    e->tuned[nshots] = {shape[0], shape[1], shape[2], shape[3]};
    release_graph(e->gfwd);
    release_graph(e->gadj);
    release_graph(e->gtd);
    return IFOSB_OK;
}
