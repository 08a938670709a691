/*
 * pb_oracle.c -- CPU restatement of DoseCUDA's proton pencil-beam dose path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path: it
 * is built into oracle/liboracle.so (FP64 continuous math, FP32 decisions)
 * and oracle/libport32.so (the same restatement in FP32 with OpenMP, used
 * only as the timed CPU baseline).  Only tests/, the smoke check in
 * __graft_entry__.py and bench.py's CPU-baseline / reference legs may load
 * it.  The product library never links or calls it.
 *
 * Parity is pinned against the reference's own CUDA module, built from the
 * reference sources into oracle/_ref by oracle/Makefile and run on a B200;
 * its outputs are committed as fixtures under tests/golden/.
 *
 * Semantics followed (reference paths are relative to the DoseCUDA repo):
 *   beam set-up          DoseCUDA/dose_kernels/CudaClasses.cu:17-51,
 *                        dosemodule.cu:148-175 (gantry+180, iso-origin)
 *   voxel <-> mm maps    CudaClasses.cuh:84-116
 *   image <-> BEV        CudaClasses.cu:65-126
 *   WET ray trace        CudaClasses.cu:180-228 (1 mm steps, RLSP*0.1 cm,
 *                        start at -0.05 cm, texture border 0, linear filter
 *                        TextureClasses.cu:14-41)
 *   WET smoothing        IMPTClasses.cu:139-202
 *   LUT interpolation    IMPTClasses.cu:69-92, lowerBound CudaClasses.cuh:130-144
 *   sigma in air         IMPTClasses.cu:94-102
 *   nuclear halo         IMPTClasses.cu:104-121
 *   axis distance        IMPTClasses.cu:123-133
 *   pencil-beam sum      IMPTClasses.cu:204-271
 *
 * Decision arithmetic (sample positions, in-grid tests, nearest-voxel
 * rounding, loop trip counts, the 1.1*R80 cut, the LUT bracket) is done in
 * FP32 with one fixed operation order and no contraction, so that the CUDA
 * path, which uses the same order through explicit intrinsics, takes the same
 * discrete decisions.  Everything continuous (trilinear weights, integrals,
 * sigmas, halo, Gaussians, sums) is done in FP64 in liboracle.so.
 *
 * Deliberate difference from the reference: the reference samples RLSP
 * through the texture unit, whose linear-filter weights are 8-bit fixed
 * point; the oracle uses exact trilinear weights (the mathematical intent).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef PB_PORT32
typedef float real;
#define R_EXP expf
#define R_LOG logf
#define R_SQRT sqrtf
#define R_HYPOT hypotf
#define R(x) x##f
#else
typedef double real;
#define R_EXP exp
#define R_LOG log
#define R_SQRT sqrt
#define R_HYPOT hypot
#define R(x) x
#endif

#define OB_PI_F 3.141592654f
#define OB_TWO_PI 6.283185307179586

typedef struct {
    float iso[3];   /* isocentre minus grid origin, mm */
    float src[3];   /* source position relative to the isocentre, mm */
    float singa, cosga, sinta, costa;
    float vsadx, vsady;
} ob_beam;

typedef struct {
    int nx, ny, nz;  /* nx = numpy axis 2 (fastest), nz = numpy axis 0 */
    float s;         /* isotropic spacing, mm */
} ob_grid;

typedef struct {
    float x, y, mu;
    int energy_id;
} ob_spot;

typedef struct {
    int spot_start, n_spots, energy_id;
    float r80, energy;
} ob_layer;

/* ------------------------------------------------------------------ */
/* Beam geometry (dosemodule.cu:148-175, CudaClasses.cu:17-51)          */
/* ------------------------------------------------------------------ */
void ob_beam_setup(double gantry_deg, double couch_deg, double vsadx,
                   double vsady, const float *iso, const float *origin,
                   ob_beam *b)
{
    float ga = fmodf((float)(gantry_deg + 180.0), 360.0f);
    float ta = (float)couch_deg;
    float gar = ga * OB_PI_F / 180.0f;
    float tar = ta * OB_PI_F / 180.0f;
    b->singa = sinf(gar);
    b->cosga = cosf(gar);
    b->sinta = sinf(tar);
    b->costa = cosf(tar);
    b->vsadx = (float)vsadx;
    b->vsady = (float)vsady;
    float sd = (b->vsadx + b->vsady) / 2.0f;
    float xg = -sd * b->singa;
    float yg = sd * b->cosga;
    b->src[0] = xg * b->costa;
    b->src[1] = yg;
    b->src[2] = -xg * b->sinta;
    for (int d = 0; d < 3; d++)
        b->iso[d] = iso[d] - origin[d];
}

/* Six lateral smoothing directions, angle i*pi/3 (IMPTClasses.cu:173-177).
 * The reference takes them from CUDA's sincosf on the device; a caller that
 * has those values (from the GPU) sets them with ob_set_smooth_dirs, else
 * the C library's cosf/sinf of the same FP32 angle are used. */
static float g_set_c[6], g_set_s[6];
static int g_dirs_set = 0;

void ob_set_smooth_dirs(const float *c, const float *s)
{
    g_dirs_set = c && s;
    for (int i = 0; g_dirs_set && i < 6; i++) {
        g_set_c[i] = c[i];
        g_set_s[i] = s[i];
    }
}

void ob_smooth_dirs(float *c, float *s)
{
    if (g_dirs_set) {
        for (int i = 0; i < 6; i++) {
            c[i] = g_set_c[i];
            s[i] = g_set_s[i];
        }
        return;
    }
    for (int i = 0; i < 6; i++) {
        /* volatile: the values must come from the C library at run time,
         * not from compile-time folding */
        volatile float a = (float)i * OB_PI_F / 3.0f;
        c[i] = cosf(a);
        s[i] = sinf(a);
    }
}

/* i*s - iso as one fused multiply-add, as the reference's compiler
 * contracts CudaClasses.cuh:106-110. */
static inline void vox_mm(const ob_grid *g, const ob_beam *b, int i, int j,
                          int k, float *p)
{
    p[0] = fmaf((float)i, g->s, -b->iso[0]);
    p[1] = fmaf((float)j, g->s, -b->iso[1]);
    p[2] = fmaf((float)k, g->s, -b->iso[2]);
}

/* Which products of the FP32 rotation expressions are fused into a
 * multiply-add, as the reference's compiler contracts a*b + c*d: per entry
 * 0 (unfused), 1 (fma of the first product with the rounded second), 2 (of
 * the second with the rounded first).  Entries: image_to_head xt, zt, xg,
 * yg (0-3), head_to_image xg, yg, xt, zt (4-7), and the smoothing sample
 * h + dr * direction (8: 0 or 1).  Default: the reference's compiled
 * arithmetic (CudaClasses.cu:65-126, IMPTClasses.cu:180-181) -- image ->
 * head fuses the second product, head -> image the first, the sample is
 * one multiply-add -- established against the reference module's smoothed
 * WET on oblique beams. */
static const int k_fuse_ref[9] = {2, 2, 2, 2, 1, 1, 1, 1, 1};
static int g_fuse[9] = {2, 2, 2, 2, 1, 1, 1, 1, 1};

void ob_set_fuse(const int *m)
{
    for (int i = 0; i < 9; i++) g_fuse[i] = m ? m[i] : k_fuse_ref[i];
}

static inline float ab_cd(float a, float b, float c, float d, int mode)
{
    if (mode == 1) return fmaf(a, b, c * d);
    if (mode == 2) return fmaf(c, d, a * b);
    return a * b + c * d;
}

/* Image -> beam's-eye (head) frame, FP32, fixed order (CudaClasses.cu:65-95). */
static inline void image_to_head_f(const ob_beam *b, const float *p, float *h)
{
    float sx = -b->sinta, cx = b->costa;
    float xt = ab_cd(p[0], cx, p[2], sx, g_fuse[0]);
    float yt = p[1];
    float zt = ab_cd(-p[0], sx, p[2], cx, g_fuse[1]);
    sx = -b->singa;
    cx = b->cosga;
    float xg = ab_cd(xt, cx, -yt, sx, g_fuse[2]);
    float yg = ab_cd(xt, sx, yt, cx, g_fuse[3]);
    h[0] = -xg;
    h[1] = zt;
    h[2] = yg;
}

/* Head -> image frame, FP32, fixed order (CudaClasses.cu:97-126). */
static inline void head_to_image_f(const ob_beam *b, const float *h, float *p)
{
    float xz = -h[0], yz = h[2], zz = h[1];
    float sx = b->singa, cx = b->cosga;
    float xg = ab_cd(xz, cx, -yz, sx, g_fuse[4]);
    float yg = ab_cd(xz, sx, yz, cx, g_fuse[5]);
    float zg = zz;
    sx = b->sinta;
    cx = b->costa;
    p[0] = ab_cd(xg, cx, zg, sx, g_fuse[6]);
    p[1] = yg;
    p[2] = ab_cd(-xg, sx, zg, cx, g_fuse[7]);
}

/* Image -> head frame in FP64 (continuous use only). */
static inline void image_to_head_d(const ob_beam *b, const float *pf, real *h)
{
    real p0 = pf[0], p1 = pf[1], p2 = pf[2];
    real sx = -(real)b->sinta, cx = b->costa;
    real xt = p0 * cx + p2 * sx;
    real yt = p1;
    real zt = -p0 * sx + p2 * cx;
    sx = -(real)b->singa;
    cx = b->cosga;
    real xg = xt * cx - yt * sx;
    real yg = xt * sx + yt * cx;
    h[0] = -xg;
    h[1] = zt;
    h[2] = yg;
}

/* Unit vector from a voxel toward the source: FP32 difference, FP64 norm,
 * rounded once to FP32 (CudaClasses.cuh:41-52 computes the same direction). */
static inline void unit_to_source(const ob_beam *b, const float *p, float *u)
{
    float d0 = b->src[0] - p[0];
    float d1 = b->src[1] - p[1];
    float d2 = b->src[2] - p[2];
    double n2 = (double)d0 * (double)d0 + (double)d1 * (double)d1;
    n2 = n2 + (double)d2 * (double)d2;
    double inv = 1.0 / sqrt(n2);
    u[0] = (float)((double)d0 * inv);
    u[1] = (float)((double)d1 * inv);
    u[2] = (float)((double)d2 * inv);
}

/* Trilinear sample at voxel-index coordinates (x,y,z) with value 0 outside
 * the grid (texture border mode, TextureClasses.cu:22-31). */
static inline real trilinear(const float *rho, const ob_grid *g, float xb,
                             float yb, float zb)
{
    float fx = floorf(xb), fy = floorf(yb), fz = floorf(zb);
    int i0 = (int)fx, j0 = (int)fy, k0 = (int)fz;
    real ax = (real)(xb - fx), ay = (real)(yb - fy), az = (real)(zb - fz);
    real acc = 0;
    for (int dk = 0; dk < 2; dk++) {
        int k = k0 + dk;
        if (k < 0 || k >= g->nz) continue;
        real wz = dk ? az : (R(1.0) - az);
        for (int dj = 0; dj < 2; dj++) {
            int j = j0 + dj;
            if (j < 0 || j >= g->ny) continue;
            real wy = dj ? ay : (R(1.0) - ay);
            for (int di = 0; di < 2; di++) {
                int i = i0 + di;
                if (i < 0 || i >= g->nx) continue;
                real wx = di ? ax : (R(1.0) - ax);
                acc += wx * wy * wz *
                       (real)rho[(int64_t)i + (int64_t)g->nx * (j + (int64_t)g->ny * k)];
            }
        }
    }
    return acc;
}

static inline int max_ray_steps(const ob_grid *g)
{
    double diag = g->s * sqrt((double)g->nx * g->nx + (double)g->ny * g->ny +
                              (double)g->nz * g->nz);
    return (int)ceil(diag) + 2;
}

/* Raw WET (cm) of one voxel (CudaClasses.cu:180-228). */
real ob_raytrace_voxel(const float *rho, const ob_grid *g, const ob_beam *b,
                       int i, int j, int k, int *err)
{
    float p[3], u[3];
    vox_mm(g, b, i, j, k, p);
    unit_to_source(b, p, u);
    const float inv_s = 1.0f / g->s;
    const int cap = max_ray_steps(g);
    real wet = R(-0.05);
    float t = 0.0f;
    for (int n = 0;; n++) {
        float q0 = fmaf(u[0], t, p[0]);
        float q1 = fmaf(u[1], t, p[1]);
        float q2 = fmaf(u[2], t, p[2]);
        float x = fmaf(inv_s, q0 + b->iso[0], 0.5f);
        float y = fmaf(inv_s, q1 + b->iso[1], 0.5f);
        float z = fmaf(inv_s, q2 + b->iso[2], 0.5f);
        if (!(x >= 0.0f && x < (float)g->nx && y >= 0.0f &&
              y < (float)g->ny && z >= 0.0f && z < (float)g->nz))
            break;
        if (n >= cap) {
            if (err) *err = 1;
            break;
        }
        real r = trilinear(rho, g, x - 0.5f, y - 0.5f, z - 0.5f);
#ifdef PB_PORT32
        wet = fmaf(r > 0.0f ? r : 0.0f, 0.1f, wet);
#else
        wet += (r > 0.0 ? r : 0.0) * 0.1;
#endif
        t += 1.0f;
    }
    return wet;
}

/* Raw WET over a whole grid or over a voxel subset (idx != NULL). */
int ob_raytrace(const float *rho, const ob_grid *g, const ob_beam *b,
                const int64_t *idx, int64_t n_idx, real *out)
{
    int err = 0;
    int64_t nv = (int64_t)g->nx * g->ny * g->nz;
    int64_t n = idx ? n_idx : nv;
#pragma omp parallel for schedule(dynamic, 256) reduction(| : err)
    for (int64_t q = 0; q < n; q++) {
        int64_t v = idx ? idx[q] : q;
        int i = (int)(v % g->nx);
        int j = (int)((v / g->nx) % g->ny);
        int k = (int)(v / ((int64_t)g->nx * g->ny));
        int e = 0;
        out[q] = ob_raytrace_voxel(rho, g, b, i, j, k, &e);
        err |= e;
    }
    return err;
}

/* The in-grid smoothing samples of one voxel in the reference's order
 * (direction, then radius; IMPTClasses.cu:166-198), written to vals;
 * returns how many (at most 54).  raw is the full raw-WET volume in FP32
 * (cm). */
static int smooth_samples(const float *raw, const ob_grid *g, const ob_beam *b,
                          const float *dc, const float *ds, int i, int j, int k,
                          float *vals)
{
    float p[3], h[3];
    int64_t v = (int64_t)i + (int64_t)g->nx * (j + (int64_t)g->ny * k);
    float center = raw[v];
    int n = 0;
    vox_mm(g, b, i, j, k, p);
    image_to_head_f(b, p, h);
    for (int d = 0; d < 6; d++) {
        float dr = 1.0f;
        while (dr < center * 10.0f && dr < 10.0f) {
            float hc[3], pc[3];
            hc[0] = g_fuse[8] ? fmaf(dr, dc[d], h[0]) : h[0] + dr * dc[d];
            hc[1] = g_fuse[8] ? fmaf(dr, ds[d], h[1]) : h[1] + dr * ds[d];
            hc[2] = h[2];
            head_to_image_f(b, hc, pc);
            int ii = (int)roundf((pc[0] + b->iso[0]) / g->s);
            int jj = (int)roundf((pc[1] + b->iso[1]) / g->s);
            int kk = (int)roundf((pc[2] + b->iso[2]) / g->s);
            if (ii >= 0 && ii < g->nx && jj >= 0 && jj < g->ny && kk >= 0 &&
                kk < g->nz)
                vals[n++] = raw[(int64_t)ii + (int64_t)g->nx * (jj + (int64_t)g->ny * kk)];
            dr += 1.0f;
        }
    }
    return n;
}

/* Smoothed WET of one voxel: the mean of the voxel's raw WET and its
 * samples, summed in `real` (FP64 in the oracle). */
real ob_smooth_voxel(const float *raw, const ob_grid *g, const ob_beam *b,
                     const float *dc, const float *ds, int i, int j, int k)
{
    float vals[54];
    const int m = smooth_samples(raw, g, b, dc, ds, i, j, k, vals);
    real sum = raw[(int64_t)i + (int64_t)g->nx * (j + (int64_t)g->ny * k)];
    for (int q = 0; q < m; q++) sum += vals[q];
#ifdef PB_PORT32
    return sum / (float)(m + 1);
#else
    return sum / (double)(m + 1);
#endif
}

void ob_smooth(const float *raw, const ob_grid *g, const ob_beam *b,
               const int64_t *idx, int64_t n_idx, real *out)
{
    float dc[6], ds[6];
    ob_smooth_dirs(dc, ds);
    int64_t nv = (int64_t)g->nx * g->ny * g->nz;
    int64_t n = idx ? n_idx : nv;
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < n; q++) {
        int64_t v = idx ? idx[q] : q;
        int i = (int)(v % g->nx);
        int j = (int)((v / g->nx) % g->ny);
        int k = (int)(v / ((int64_t)g->nx * g->ny));
        out[q] = ob_smooth_voxel(raw, g, b, dc, ds, i, j, k);
    }
}

/* The voxel index (i, j, k) that the reference's FP32 arithmetic picks for
 * every smoothing sample of every voxel, whether or not the sample is in
 * the grid or within the voxel's radius limit: out[((v*6 + d)*9 + r)*3 + a]
 * for direction d, radius r+1 mm, axis a (IMPTClasses.cu:178-186). */
void ob_smooth_choices(const ob_grid *g, const ob_beam *b, int32_t *out)
{
    float dc[6], ds[6];
    ob_smooth_dirs(dc, ds);
    int64_t nv = (int64_t)g->nx * g->ny * g->nz;
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < nv; v++) {
        int i = (int)(v % g->nx);
        int j = (int)((v / g->nx) % g->ny);
        int k = (int)(v / ((int64_t)g->nx * g->ny));
        float p[3], h[3];
        vox_mm(g, b, i, j, k, p);
        image_to_head_f(b, p, h);
        for (int d = 0; d < 6; d++) {
            float dr = 1.0f;
            for (int r = 0; r < 9; r++) {
                float hc[3], pc[3];
                hc[0] = g_fuse[8] ? fmaf(dr, dc[d], h[0]) : h[0] + dr * dc[d];
                hc[1] = g_fuse[8] ? fmaf(dr, ds[d], h[1]) : h[1] + dr * ds[d];
                hc[2] = h[2];
                head_to_image_f(b, hc, pc);
                int32_t *o = out + ((v * 6 + d) * 9 + r) * 3;
                o[0] = (int32_t)roundf((pc[0] + b->iso[0]) / g->s);
                o[1] = (int32_t)roundf((pc[1] + b->iso[1]) / g->s);
                o[2] = (int32_t)roundf((pc[2] + b->iso[2]) / g->s);
                dr += 1.0f;
            }
        }
    }
}

/* The smoothing with the reference's own arithmetic: an FP32 sum in
 * sample order and an FP32 quotient (IMPTClasses.cu:168-198), so that a
 * kernel choosing the same voxels gives the same bits. */
void ob_smooth_f32(const float *raw, const ob_grid *g, const ob_beam *b, float *out)
{
    float dc[6], ds[6];
    ob_smooth_dirs(dc, ds);
    int64_t nv = (int64_t)g->nx * g->ny * g->nz;
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < nv; v++) {
        int i = (int)(v % g->nx);
        int j = (int)((v / g->nx) % g->ny);
        int k = (int)(v / ((int64_t)g->nx * g->ny));
        float vals[54];
        const int m = smooth_samples(raw, g, b, dc, ds, i, j, k, vals);
        float sum = raw[v];
        for (int q = 0; q < m; q++) sum += vals[q];
        out[v] = sum / (float)(m + 1);
    }
}

/* ------------------------------------------------------------------ */
/* Spot sorting and layers (dosemodule.cu:204-225, IMPTClasses.cu:29-67) */
/* ------------------------------------------------------------------ */
typedef struct { ob_spot s; int ord; } ob_tagged;

static int cmp_tagged(const void *a, const void *b)
{
    const ob_tagged *x = (const ob_tagged *)a, *y = (const ob_tagged *)b;
    if (x->s.energy_id != y->s.energy_id)
        return x->s.energy_id < y->s.energy_id ? -1 : 1;
    return x->ord < y->ord ? -1 : (x->ord > y->ord);
}

/* spot_list is N x 4 float (x, y, mu, energy_id).  Spots are sorted by
 * energy id (ties keep input order) and grouped into contiguous layers the
 * way importLayers does it.  Returns the number of layers. */
int ob_build_layers(const float *spot_list, int n, const float *dvp,
                    int dvp_len, int n_energies, ob_spot *spots,
                    ob_layer *layers)
{
    ob_tagged *t = (ob_tagged *)malloc(sizeof(ob_tagged) * (size_t)(n > 0 ? n : 1));
    for (int q = 0; q < n; q++) {
        t[q].s.x = spot_list[4 * q];
        t[q].s.y = spot_list[4 * q + 1];
        t[q].s.mu = spot_list[4 * q + 2];
        t[q].s.energy_id = (int)spot_list[4 * q + 3];
        t[q].ord = q;
    }
    qsort(t, (size_t)n, sizeof(ob_tagged), cmp_tagged);
    for (int q = 0; q < n; q++) spots[q] = t[q].s;
    free(t);

    int nl = 0, start = 0;
    for (int e = 0; e < n_energies; e++) {
        int end = start;
        while (end < n && spots[end].energy_id == e) end++;
        int cnt = end - start;
        if (!cnt) continue;
        layers[nl].spot_start = start;
        layers[nl].n_spots = cnt;
        layers[nl].energy_id = e;
        layers[nl].r80 = dvp[dvp_len * e + 1];
        layers[nl].energy = dvp[dvp_len * e];
        nl++;
        start += cnt;
    }
    return nl;
}

/* ------------------------------------------------------------------ */
/* Pencil-beam model per (voxel, layer)                                 */
/* ------------------------------------------------------------------ */
typedef struct {
    const float *dvp;     /* n_energies x dvp_len: energy, R80, A, B, C */
    const float *depths;  /* n_energies x lut_len */
    const float *sigmas;
    const float *idds;
    int dvp_len, lut_len, n_energies;
} ob_model;

typedef struct {
    real pf, hf;      /* Gaussian prefactors */
    real ps, hs;      /* exponent scales, -1/(2 sigma^2) */
    real h[3];        /* voxel in head frame */
    int active;
} ob_vl;

static inline int lower_bound_f(const float *d, int len, float key)
{
    int l = 0, r = len;
    while (l < r) {
        int m = (l + r) / 2;
        if (key <= d[m]) r = m; else l = m + 1;
    }
    return l;
}

static void ob_voxel_layer(const ob_grid *g, const ob_beam *b, const ob_model *m,
                           const ob_layer *L, float wet_cm, const float *p,
                           ob_vl *o)
{
    float wetf = wet_cm * 10.0f;
    o->active = 0;
    if (wetf > 1.1f * L->r80) return;   /* IMPTClasses.cu:222-226 */
    o->active = 1;
    const int e = L->energy_id;
    const float *dep = m->depths + (size_t)e * m->lut_len;
    const float *sig = m->sigmas + (size_t)e * m->lut_len;
    const float *idd = m->idds + (size_t)e * m->lut_len;
    int i = lower_bound_f(dep, m->lut_len, wetf);
    real wet = wetf, vidd, vsig;
    if (i == m->lut_len) { vidd = idd[i - 1]; vsig = sig[i - 1]; }
    else if (i == 0) { vidd = idd[0]; vsig = sig[0]; }
    else {
        real f = (wet - (real)dep[i - 1]) / ((real)dep[i] - (real)dep[i - 1]);
        vidd = (real)idd[i - 1] + f * ((real)idd[i] - (real)idd[i - 1]);
        vsig = (real)sig[i - 1] + f * ((real)sig[i] - (real)sig[i - 1]);
    }
    real dx = (real)b->src[0] - (real)p[0];
    real dy = (real)b->src[1] - (real)p[1];
    real dz = (real)b->src[2] - (real)p[2];
    real dist = R_SQRT(dx * dx + dy * dy + dz * dz);
    const float *c = m->dvp + (size_t)m->dvp_len * e;
    real r80 = L->r80;
    real d = dist - wet + R(0.7) * r80;
    real sair = ((real)c[2] * d + (real)c[3]) * d + (real)c[4];
    real st = sair + vsig;
    real w = wet;
    if (w < R(0.1)) w = R(0.1);
    if (w > r80 - R(0.1)) w = r80 - R(0.1);
    real a1 = w - r80 - R(5.0);
    real sh = R(2.85) + R(0.0014) * r80 * R_LOG(w + R(3.0)) + R(0.06) * w -
              R(7.4e-5) * w * w - (R(0.22) * r80) / (a1 * a1);
    real r3 = r80 + R(3.0);
    real wh = R(0.052) * R_LOG(R(1.13) + w / (R(11.2) - R(0.023) * r80)) +
              R(0.35) * (R(0.0017) * r80 * r80 - r80) / (r3 * r3 - w * w) -
              R(1.61e-9) * w * r3 * r3;
    if (sh < 0) sh = 0;
    if (wh < 0) wh = 0;
    if (wh > R(0.9)) wh = R(0.9);
    real sht = R_HYPOT(st, sh);
    o->pf = (R(1.0) - wh) * vidd / ((real)OB_TWO_PI * st * st);
    o->hf = wh * vidd / ((real)OB_TWO_PI * sht * sht);
    o->ps = st != 0 ? R(-0.5) / (st * st) : -INFINITY;
    o->hs = sht != 0 ? R(-0.5) / (sht * sht) : -INFINITY;
    image_to_head_d(b, p, o->h);
}

/* Pencil-beam kernel of one spot at one voxel (IMPTClasses.cu:123-133,
 * 255-265). */
static inline real ob_kernel(const ob_vl *o, const ob_spot *s, const ob_beam *b)
{
    real tx = (real)s->x / (real)b->vsadx;
    real ty = (real)s->y / (real)b->vsady;
    real rx = o->h[0] - (real)s->x, ry = o->h[1] - (real)s->y, rz = o->h[2];
    real t2 = tx * tx + ty * ty + R(1.0);
    real r2 = rx * rx + ry * ry + rz * rz;
    real dp = tx * rx + ty * ry - rz;
    real d2 = r2 - dp * dp / t2;
    return o->pf * R_EXP(o->ps * d2) + o->hf * R_EXP(o->hs * d2);
}

/* Dose of one beam at a whole grid or a voxel subset.  wet_cm is the
 * smoothed WET volume in cm (FP32, as passed between the two reference
 * passes).  spots/layers come from ob_build_layers. Output accumulates
 * (+=) into out. */
void ob_dose(const float *wet_cm, const ob_grid *g, const ob_beam *b,
             const ob_model *m, const ob_spot *spots, const ob_layer *layers,
             int n_layers, const int64_t *idx, int64_t n_idx, real *out)
{
    int64_t nv = (int64_t)g->nx * g->ny * g->nz;
    int64_t n = idx ? n_idx : nv;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t q = 0; q < n; q++) {
        int64_t v = idx ? idx[q] : q;
        int i = (int)(v % g->nx);
        int j = (int)((v / g->nx) % g->ny);
        int k = (int)(v / ((int64_t)g->nx * g->ny));
        float p[3];
        vox_mm(g, b, i, j, k, p);
        real acc = 0;
        for (int l = 0; l < n_layers; l++) {
            ob_vl o;
            ob_voxel_layer(g, b, m, &layers[l], wet_cm[v], p, &o);
            if (!o.active) continue;
            real dl = 0;
            const ob_spot *s = spots + layers[l].spot_start;
            for (int t = 0; t < layers[l].n_spots; t++)
                dl += (real)s[t].mu * ob_kernel(&o, &s[t], b);
            acc += dl;
        }
        out[q] += acc;
    }
}

/* Adjoint: grad[s] += sum_v w[v] * K(v, s) over the whole grid, where K is
 * the dose per unit weight of spot s at voxel v.  Spots index the sorted
 * array. */
void ob_adjoint(const float *wet_cm, const ob_grid *g, const ob_beam *b,
                const ob_model *m, const ob_spot *spots, const ob_layer *layers,
                int n_layers, const double *w, real *grad)
{
    int64_t nv = (int64_t)g->nx * g->ny * g->nz;
    for (int l = 0; l < n_layers; l++) {
        const ob_layer *L = &layers[l];
        ob_vl *vl = (ob_vl *)malloc(sizeof(ob_vl) * (size_t)nv);
#pragma omp parallel for schedule(static)
        for (int64_t v = 0; v < nv; v++) {
            int i = (int)(v % g->nx);
            int j = (int)((v / g->nx) % g->ny);
            int k = (int)(v / ((int64_t)g->nx * g->ny));
            float p[3];
            vox_mm(g, b, i, j, k, p);
            ob_voxel_layer(g, b, m, L, wet_cm[v], p, &vl[v]);
            if (w[v] == 0.0) vl[v].active = 0;
        }
#pragma omp parallel for schedule(dynamic, 1)
        for (int t = 0; t < L->n_spots; t++) {
            const ob_spot *s = &spots[L->spot_start + t];
            real acc = 0;
            for (int64_t v = 0; v < nv; v++) {
                if (!vl[v].active) continue;
                acc += (real)w[v] * ob_kernel(&vl[v], s, b);
            }
            grad[L->spot_start + t] += acc;
        }
        free(vl);
    }
}

/* Dense pair count E = sum_layers |{v : 10*WET(v) <= 1.1*R80}| * spots. */
int64_t ob_count_pairs(const float *wet_cm, int64_t nv, const ob_layer *layers,
                       int n_layers)
{
    int64_t e = 0;
    for (int l = 0; l < n_layers; l++) {
        int64_t c = 0;
        float cut = 1.1f * layers[l].r80;
#pragma omp parallel for reduction(+ : c)
        for (int64_t v = 0; v < nv; v++)
            if (!(wet_cm[v] * 10.0f > cut)) c++;
        e += c * layers[l].n_spots;
    }
    return e;
}

int ob_real_size(void) { return (int)sizeof(real); }
