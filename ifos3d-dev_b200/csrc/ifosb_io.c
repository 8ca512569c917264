/* ifosb_io.c — the reference's on-disk formats for seismograms, models and
 * gradients, so that files written next to the GPU engine are the files IFOS3D
 * itself writes (and reads back as observed data).
 *
 *   ifosb_write_seis       outseis.c:30-276   SU (240-byte trace header + floats),
 *                                             ASCII, raw binary (optionally byte-swapped)
 *   ifosb_merge_seis       saveseis.c:86-229  rank 0 concatenates the ranks' SU files
 *   ifosb_read_seis        readseis.c:25-69   skip 240 bytes, read ns floats per trace
 *   ifosb_read_seis_split  readseis_split.c   the same, keeping flagged traces only
 *   ifosb_write_model      outmod.c + mergemod.c   vp, vs, rho as [z][x][y] floats
 *   ifosb_write_gradient   outgrad.c + mergemod.c  three gradients, same order
 *
 * Header values follow outseis.c's expressions and promotions (float products,
 * double sqrt, iround = (int)floor(x + 0.5)). Fields outseis.c never assigns
 * (cdp, selev, swdep and the 30 trailing pad bytes) hold whatever was on its stack;
 * they are written as zeros here. All files use the host's byte order, as the
 * reference's fwrite of its structs and floats does.
 */
#include "../../include/ifos_b200.h"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define SU_HDR 240
#define SU_MAXNS 65535 /* segy.h: SU_NFLTS = USHRT_MAX */

static int iround_d(double x) { return (int)floor(x + 0.5); }

/* snprintf into a path buffer; 0 when the name did not fit. */
#define PATH_FMT(buf, ...) (snprintf(buf, sizeof buf, __VA_ARGS__) < (int)sizeof buf)

static void put32(unsigned char *h, int off, int32_t v) { memcpy(h + off, &v, 4); }
static void put16(unsigned char *h, int off, int16_t v) { memcpy(h + off, &v, 2); }

/* The 240-byte SU trace header of outseis.c:66-260 (SEG-Y rev 0 positions). */
static void su_header(unsigned char *h, int tracl, float xr, float yr, float zr, float XS, float YS, float ZS, int ns,
                      int ndt, float dt) {
    const float scalefac = (float)pow(10.0, 3.0);
    memset(h, 0, SU_HDR);
    put32(h, 0, tracl);                         /* tracl */
    put16(h, 28, 1);                            /* trid: seismic */
    put32(h, 36, iround_d(sqrt((XS - xr) * (XS - xr) + (YS - yr) * (YS - yr) + (ZS - zr) * (ZS - zr)) * scalefac));
    put32(h, 40, iround_d(yr * scalefac));      /* gelev */
    put32(h, 48, iround_d(YS * scalefac));      /* sdepth */
    put16(h, 68, (int16_t)(-3));                /* scalel */
    put16(h, 70, (int16_t)(-3));                /* scalco */
    put32(h, 72, iround_d(XS * scalefac));      /* sx */
    put32(h, 76, iround_d(ZS * scalefac));      /* sy: the z source coordinate */
    put32(h, 80, iround_d(xr * scalefac));      /* gx */
    put32(h, 84, iround_d(zr * scalefac));      /* gy: the z receiver coordinate */
    put16(h, 114, (int16_t)(unsigned short)ns); /* ns */
    put16(h, 116, (int16_t)(unsigned short)iround_d(((float)ndt * dt) * 1.0e6)); /* dt in us */
}

static uint32_t bswap32(uint32_t x) {
    return ((x >> 24) & 0xffu) | ((x & 0xffu) << 24) | ((x >> 8) & 0xff00u) | ((x & 0xff00u) << 8);
}

int ifosb_write_seis(const char *path, int comp, const float *section, int ntr, int ns, const int *rec,
                     const int *trace_no, const float *src, float dx, float dy, float dz, int ndt, float dt, int fmt,
                     int littlebig) {
    (void)comp; /* outseis.c:67 stores it in ep and :98 overwrites it with 0 */
    if (!path || ntr < 0 || ns < 1 || (ntr > 0 && !section)) return IFOSB_EARG;
    if ((fmt == 0 || fmt == 1) && (ns > SU_MAXNS || (ntr > 0 && !rec))) return IFOSB_EARG;
    FILE *f = fopen(path, "wb");
    if (!f) return IFOSB_EIO;
    int rc = IFOSB_OK;
    const float XS = src ? src[0] : 0.0f, YS = src ? src[1] : 0.0f, ZS = src ? src[2] : 0.0f;
    switch (fmt) {
    case 0:
    case 1: {
        unsigned char h[SU_HDR];
        for (int t = 0; t < ntr && rc == IFOSB_OK; ++t) {
            const float xr = rec[3 * t] * dx, yr = rec[3 * t + 1] * dy, zr = rec[3 * t + 2] * dz;
            su_header(h, trace_no ? trace_no[t] : t + 1, xr, yr, zr, XS, YS, ZS, ns, ndt, dt);
            if (fwrite(h, 1, SU_HDR, f) != SU_HDR ||
                fwrite(section + (size_t)t * ns, sizeof(float), (size_t)ns, f) != (size_t)ns)
                rc = IFOSB_EIO;
        }
        break;
    }
    case 2: /* one column per trace, one row per sample */
        for (int j = 0; j < ns && rc == IFOSB_OK; ++j) {
            for (int t = 0; t < ntr; ++t)
                if (fprintf(f, "%e\t", section[(size_t)t * ns + j]) < 0) rc = IFOSB_EIO;
            if (fprintf(f, "\n") < 0) rc = IFOSB_EIO;
        }
        break;
    case 3:
        for (int t = 0; t < ntr && rc == IFOSB_OK; ++t)
            for (int j = 0; j < ns; ++j) {
                float v = section[(size_t)t * ns + j];
                if (littlebig) {
                    uint32_t u;
                    memcpy(&u, &v, 4);
                    u = bswap32(u);
                    memcpy(&v, &u, 4);
                }
                if (fwrite(&v, sizeof(float), 1, f) != 1) { rc = IFOSB_EIO; break; }
            }
        break;
    default: /* outseis.c:268-271: no output written */
        rc = IFOSB_EARG;
    }
    if (fclose(f) != 0 && rc == IFOSB_OK) rc = IFOSB_EIO;
    return rc;
}

int ifosb_merge_seis(const char *out, int nin, const char *const *inputs, int ns, int *ntr_out) {
    if (!out || nin < 0 || (nin > 0 && !inputs) || ns < 1) return IFOSB_EARG;
    FILE *fo = fopen(out, "wb");
    if (!fo) return IFOSB_EIO;
    const size_t rec = SU_HDR + 4 * (size_t)ns;
    unsigned char *buf = (unsigned char *)malloc(rec);
    int rc = buf ? IFOSB_OK : IFOSB_ENOMEM, total = 0;
    for (int r = 0; r < nin && rc == IFOSB_OK; ++r) {
        FILE *fi = inputs[r] ? fopen(inputs[r], "rb") : NULL;
        if (!fi) continue; /* saveseis.c:97: a rank without traces wrote no file */
        fseek(fi, 0, SEEK_END);
        const long k = ftell(fi);
        const long l = (k >= 0 && k % (long)rec == 0) ? k / (long)rec : 0; /* :100-104 */
        fseek(fi, 0, SEEK_SET);
        for (long m = 0; m < l; ++m) {
            if (fread(buf, 1, rec, fi) != rec || fwrite(buf, 1, rec, fo) != rec) { rc = IFOSB_EIO; break; }
            ++total;
        }
        fclose(fi);
    }
    free(buf);
    if (fclose(fo) != 0 && rc == IFOSB_OK) rc = IFOSB_EIO;
    if (ntr_out) *ntr_out = total;
    return rc;
}

/* readseis.c:49-57: a trace's samples stay 0 where the file ends early. */
static int read_traces(const char *path, float *section, int ntr, const int *keep, int ns) {
    if (!path || ntr < 0 || ns < 1 || (ntr > 0 && !section)) return IFOSB_EARG;
    if (ntr == 0) return IFOSB_OK;
    FILE *f = fopen(path, "rb");
    if (!f) return IFOSB_EIO;
    int row = 0;
    for (int t = 0; t < ntr; ++t) {
        fseek(f, SU_HDR, SEEK_CUR);
        if (keep && keep[t] != 1) {
            fseek(f, 4L * ns, SEEK_CUR);
            continue;
        }
        float *d = section + (size_t)row * ns;
        for (int j = 0; j < ns; ++j) {
            d[j] = 0.0f;
            if (fread(&d[j], sizeof(float), 1, f) != 1) d[j] = 0.0f;
        }
        ++row;
    }
    fclose(f);
    return IFOSB_OK;
}

int ifosb_read_seis(const char *path, float *section, int ntr, int ns) {
    return read_traces(path, section, ntr, NULL, ns);
}

int ifosb_read_seis_split(const char *path, float *section, int ntr, const int *keep, int ns) {
    if (!keep) return IFOSB_EARG;
    return read_traces(path, section, ntr, keep, ns);
}

/* Element (j, i, k), 1-based interior indices, of a dense [ny][nx][nz] array or of
 * a ghosted [ny+2][nx+2][nz+2] one. */
static float at(const float *a, int ghost, int nx, int nz, int j, int i, int k) {
    if (ghost) return a[((size_t)j * (nx + 2) + i) * (nz + 2) + k];
    return a[((size_t)(j - 1) * nx + (i - 1)) * nz + (k - 1)];
}

/* mergemod.c:58-65 for one rank: the merged file holds the first
 * ceil(NZ/IDZ)*ceil(NX/IDX)*ceil(NY/IDY) values of the rank file, which outmod
 * and outgrad write in [z][x][y] order at full resolution. */
static long merged_count(int nx, int ny, int nz, int idx, int idy, int idz) {
    return (long)((nz - 1) / idz + 1) * ((nx - 1) / idx + 1) * ((ny - 1) / idy + 1);
}

typedef float (*cell_fn)(const float *const *arrs, int ghost, int nx, int nz, int j, int i, int k);

static int write_zxy(const char *path, cell_fn fn, const float *const *arrs, int ghost, int nx, int ny, int nz,
                     long count) {
    FILE *f = fopen(path, "wb");
    if (!f) return IFOSB_EIO;
    int rc = IFOSB_OK;
    long n = 0;
    for (int k = 1; k <= nz && n < count && rc == IFOSB_OK; ++k)
        for (int i = 1; i <= nx && n < count && rc == IFOSB_OK; ++i)
            for (int j = 1; j <= ny && n < count; ++j, ++n) {
                const float v = fn(arrs, ghost, nx, nz, j, i, k);
                if (fwrite(&v, sizeof(float), 1, f) != 1) { rc = IFOSB_EIO; break; }
            }
    if (fclose(f) != 0 && rc == IFOSB_OK) rc = IFOSB_EIO;
    return rc;
}

/* outmod.c:54-55: vp = sqrt(pi/rho), vs = sqrt(u/rho), float quotient, double root. */
static float cell_vp(const float *const *m, int g, int nx, int nz, int j, int i, int k) {
    return (float)sqrt(at(m[1], g, nx, nz, j, i, k) / at(m[0], g, nx, nz, j, i, k));
}
static float cell_vs(const float *const *m, int g, int nx, int nz, int j, int i, int k) {
    return (float)sqrt(at(m[2], g, nx, nz, j, i, k) / at(m[0], g, nx, nz, j, i, k));
}
static float cell_0(const float *const *m, int g, int nx, int nz, int j, int i, int k) { return at(m[0], g, nx, nz, j, i, k); }

static int dims_ok(int nx, int ny, int nz, int idx, int idy, int idz) {
    return nx > 0 && ny > 0 && nz > 0 && idx > 0 && idy > 0 && idz > 0;
}

int ifosb_write_model(const char *base, int iteration, int nx, int ny, int nz, const float *rho, const float *pi,
                      const float *u, int ghost, int idx, int idy, int idz) {
    if (!base || !rho || !pi || !u || !dims_ok(nx, ny, nz, idx, idy, idz)) return IFOSB_EARG;
    const long cnt = merged_count(nx, ny, nz, idx, idy, idz);
    const float *m[3] = {rho, pi, u};
    const float *r[1] = {rho};
    char path[4096];
    int rc;
    if (!PATH_FMT(path, "%s.vp_it%d", base, iteration)) return IFOSB_EARG;
    if ((rc = write_zxy(path, cell_vp, m, ghost, nx, ny, nz, cnt)) != IFOSB_OK) return rc;
    if (!PATH_FMT(path, "%s.vs_it%d", base, iteration)) return IFOSB_EARG;
    if ((rc = write_zxy(path, cell_vs, m, ghost, nx, ny, nz, cnt)) != IFOSB_OK) return rc;
    if (!PATH_FMT(path, "%s.rho_it%d", base, iteration)) return IFOSB_EARG;
    return write_zxy(path, cell_0, r, ghost, nx, ny, nz, cnt);
}

int ifosb_write_gradient(const char *base, float finv, int iteration, int nx, int ny, int nz, const float *grad,
                         int ghost, int idx, int idy, int idz) {
    if (!base || !grad || !dims_ok(nx, ny, nz, idx, idy, idz)) return IFOSB_EARG;
    const long cnt = merged_count(nx, ny, nz, idx, idy, idz);
    const size_t n = ghost ? (size_t)(nx + 2) * (ny + 2) * (nz + 2) : (size_t)nx * ny * nz;
    static const char *name[3] = {"vp", "vs", "rho"};
    char path[4096];
    for (int c = 0; c < 3; ++c) {
        const float *a[1] = {grad + c * n};
        if (!PATH_FMT(path, "%s.%s_%4.2fHz_it%d", base, name[c], finv, iteration)) return IFOSB_EARG;
        const int rc = write_zxy(path, cell_0, a, ghost, nx, ny, nz, cnt);
        if (rc != IFOSB_OK) return rc;
    }
    return IFOSB_OK;
}

/* readhess.c:25-95 on one rank: the three "<base>.{vp,vs,rho}_<finv %4.2f>Hz_it<n>"
 * files, [z][x][y] floats, into hess [3][ny][nx][nz] scaled by VP0^2, VS0^2, RHO0^2
 * (float value times the double power, rounded to float). */
int ifosb_read_hessian(const char *base, float finv, int iteration, int nx, int ny, int nz, float vp0, float vs0,
                       float rho0, float *hess) {
    if (!base || !hess || nx < 1 || ny < 1 || nz < 1) return IFOSB_EARG;
    static const char *name[3] = {"vp", "vs", "rho"};
    const double sc[3] = {pow(vp0, 2), pow(vs0, 2), pow(rho0, 2)};
    const size_t n = (size_t)nx * ny * nz;
    char path[4096];
    for (int c = 0; c < 3; ++c) {
        if (!PATH_FMT(path, "%s.%s_%4.2fHz_it%d", base, name[c], finv, iteration)) return IFOSB_EARG;
        FILE *f = fopen(path, "rb");
        if (!f) return IFOSB_EIO;
        for (int k = 1; k <= nz; ++k)
            for (int i = 1; i <= nx; ++i)
                for (int j = 1; j <= ny; ++j) {
                    float v = 0.0f;
                    if (fread(&v, sizeof(float), 1, f) != 1) { fclose(f); return IFOSB_EIO; }
                    hess[c * n + ((size_t)(j - 1) * nx + (i - 1)) * nz + (k - 1)] = (float)(v * sc[c]);
                }
        fclose(f);
    }
    return IFOSB_OK;
}
