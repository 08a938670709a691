// pb_wet.cu -- HU -> RLSP conversion and the water-equivalent-thickness
// (WET) pass: ray trace toward the source and lateral smoothing.
//
//   HU -> RLSP            DoseCUDA/plan_impt.py:158-168 (numpy.interp)
//   ray trace             DoseCUDA/dose_kernels/CudaClasses.cu:180-228
//   smoothing             DoseCUDA/dose_kernels/IMPTClasses.cu:139-202
//
// Layout: every volume is x-fastest; one thread per voxel; blocks are 8x4x4
// voxel bricks so that a warp covers an 8x4 patch whose rays have similar
// lengths whatever the beam direction, and each row of 8 voxels is one
// 32-byte sector.  Several beams share one launch (grid z = z-bricks x beams).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

#include "pb_internal.h"

namespace pb {

// ------------------------------------------------------------------ HU->RLSP

struct HuCurve {
    double x[PB_MAX_CURVE];
    double y[PB_MAX_CURVE];
    double slope[PB_MAX_CURVE];
    int n;
};

// numpy.interp: left of the first point -> first value, right of the last
// -> last value, on a knot -> the knot's value, else slope*(x-x_j)+y_j in
// FP64 with no contraction; the result is rounded to FP32 as np.array(...,
// dtype=single) does.
__global__ void k_rlsp(const float *__restrict__ hu, int64_t n,
                       const __grid_constant__ HuCurve c,
                       float *__restrict__ out)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
         q += (int64_t)gridDim.x * blockDim.x) {
        const double x = (double)hu[q];
        double r;
        if (x != x) {
            r = x;
        } else if (x < c.x[0]) {
            r = c.y[0];
        } else if (x > c.x[c.n - 1]) {
            r = c.y[c.n - 1];
        } else {
            int j = 0;
            while (j + 1 < c.n && c.x[j + 1] <= x) ++j;
            if (j == c.n - 1 || c.x[j] == x) {
                r = c.y[j];
            } else {
                r = __dadd_rn(__dmul_rn(c.slope[j], __dsub_rn(x, c.x[j])), c.y[j]);
            }
        }
        out[q] = __double2float_rn(r);
    }
}

PbStatus launch_rlsp(const float *hu, int64_t n, const double *xh,
                     const double *yh, int m, float *out, cudaStream_t st)
{
    HuCurve c;
    c.n = m;
    for (int i = 0; i < m; ++i) {
        c.x[i] = xh[i];
        c.y[i] = yh[i];
    }
    for (int i = 0; i + 1 < m; ++i) c.slope[i] = (yh[i + 1] - yh[i]) / (xh[i + 1] - xh[i]);
    c.slope[m - 1] = 0.0;
    if (n == 0) return PB_OK;
    int blocks = (int)((n + 255) / 256);
    const int cap = 148 * 16;
    if (blocks > cap) blocks = cap;
    k_rlsp<<<blocks, 256, 0, st>>>(hu, n, c, out);
    return check_launch("k_rlsp");
}

// ----------------------------------------------------------------- ray trace

// Trilinear sample at voxel-index coordinates with 0 outside the grid
// (the reference samples a border-0 texture with linear filtering).
__device__ __forceinline__ float trilinear(const float *__restrict__ rho,
                                           int nx, int ny, int nz, float xb,
                                           float yb, float zb)
{
    const float fx = floorf(xb), fy = floorf(yb), fz = floorf(zb);
    const int i0 = (int)fx, j0 = (int)fy, k0 = (int)fz;
    const float ax = xb - fx, ay = yb - fy, az = zb - fz;
    const int64_t sy = nx, sz = (int64_t)nx * ny;
    float c000, c100, c010, c110, c001, c101, c011, c111;
    if (i0 >= 0 && j0 >= 0 && k0 >= 0 && i0 + 1 < nx && j0 + 1 < ny && k0 + 1 < nz) {
        const float *p = rho + i0 + sy * j0 + sz * k0;
        c000 = __ldg(p);
        c100 = __ldg(p + 1);
        c010 = __ldg(p + sy);
        c110 = __ldg(p + sy + 1);
        c001 = __ldg(p + sz);
        c101 = __ldg(p + sz + 1);
        c011 = __ldg(p + sz + sy);
        c111 = __ldg(p + sz + sy + 1);
    } else {
        const bool xi0 = i0 >= 0 && i0 < nx, xi1 = i0 + 1 >= 0 && i0 + 1 < nx;
        const bool yj0 = j0 >= 0 && j0 < ny, yj1 = j0 + 1 >= 0 && j0 + 1 < ny;
        const bool zk0 = k0 >= 0 && k0 < nz, zk1 = k0 + 1 >= 0 && k0 + 1 < nz;
        auto at = [&](bool ok, int i, int j, int k) -> float {
            return ok ? __ldg(rho + i + sy * j + sz * k) : 0.0f;
        };
        c000 = at(xi0 && yj0 && zk0, i0, j0, k0);
        c100 = at(xi1 && yj0 && zk0, i0 + 1, j0, k0);
        c010 = at(xi0 && yj1 && zk0, i0, j0 + 1, k0);
        c110 = at(xi1 && yj1 && zk0, i0 + 1, j0 + 1, k0);
        c001 = at(xi0 && yj0 && zk1, i0, j0, k0 + 1);
        c101 = at(xi1 && yj0 && zk1, i0 + 1, j0, k0 + 1);
        c011 = at(xi0 && yj1 && zk1, i0, j0 + 1, k0 + 1);
        c111 = at(xi1 && yj1 && zk1, i0 + 1, j0 + 1, k0 + 1);
    }
    const float c00 = fmaf(ax, c100 - c000, c000);
    const float c10 = fmaf(ax, c110 - c010, c010);
    const float c01 = fmaf(ax, c101 - c001, c001);
    const float c11 = fmaf(ax, c111 - c011, c011);
    const float c0 = fmaf(ay, c10 - c00, c00);
    const float c1 = fmaf(ay, c11 - c01, c01);
    return fmaf(az, c1 - c0, c0);
}

// Number of leading samples t = 0, 1, ... whose texture coordinates are
// certainly inside [0, n) on every axis, so the in-grid test can be skipped
// for them.  The bound is taken on the exact (real-number) coordinates
// A + B t of the FP32 formula with a margin of 4e-3 texel; the FP32
// evaluation differs from them by less than 1e-3 texel for any grid this
// library accepts, so the skipped tests would all have passed.
__device__ __forceinline__ int safe_steps(const PbGrid &g, const PbBeamGeom &B, float inv_s,
                                          float px, float py, float pz, float ux, float uy,
                                          float uz, int cap)
{
    const double margin = 4e-3;
    const float pv[3] = {px, py, pz}, uv[3] = {ux, uy, uz};
    const int nv[3] = {g.nx, g.ny, g.nz};
    double T = (double)cap;
    for (int a = 0; a < 3; ++a) {
        const double A = (double)inv_s * ((double)pv[a] + (double)B.iso[a]) + 0.5;
        const double Bt = (double)inv_s * (double)uv[a];
        const double lo = margin, hi = (double)nv[a] - margin;
        if (A < lo || A > hi) return 0;
        if (Bt > 0.0) T = fmin(T, (hi - A) / Bt);
        else if (Bt < 0.0) T = fmin(T, (lo - A) / Bt);
    }
    if (!(T >= 0.0)) return 0;
    const double n = floor(T) + 1.0;
    return n < (double)cap ? (int)n : cap;
}

template <bool TEX>
__device__ __forceinline__ float ray_sample(const float *__restrict__ rho,
                                            cudaTextureObject_t tex, const PbGrid &g,
                                            float x, float y, float z)
{
    if (TEX) return tex3D<float>(tex, x, y, z);
    return trilinear(rho, g.nx, g.ny, g.nz, __fsub_rn(x, 0.5f), __fsub_rn(y, 0.5f),
                     __fsub_rn(z, 0.5f));
}

// Raw WET (cm) per voxel: samples every 1 mm from the voxel toward the
// source while the texture coordinate stays inside [0, n); WET = -0.05 +
// 0.1 * sum(max(RLSP, 0)).  The sum is carried in FP64 (FP32 partials of 8
// samples).  A ray that exceeds the grid-diagonal step cap stops and raises
// PB_ERR_RAY_CAP in *status.  The leading samples that are certainly inside
// the grid (safe_steps) go without the in-grid test: with cell records, as
// runs through flat cells (flat_run) and bursts of kTexBurst fetches
// elsewhere; without them, 8 fetches at a time.  Either way several
// fetches are in flight per thread.
//
// TEX = true samples RLSP through a border-0, linearly filtered 3-D texture
// and forms the ray direction with rnorm3df, as the reference does
// (CudaClasses.cuh:41-52, TextureClasses.cu:14-41), so the samples are the
// reference's own.  TEX = false interpolates with exact FP32 trilinear
// weights from global memory and forms the direction in FP64, the CPU
// oracle's arithmetic.
// floor(a) for -2^22 <= a < 2^22 on the FP32 adder: adding 1.5 * 2^23 with
// rounding toward -infinity leaves floor(a) in the low mantissa bits.
__device__ __forceinline__ int floor_small(float a)
{
    return __float_as_int(__fadd_rd(a, 12582912.0f)) - 0x4B400000;
}

__device__ __forceinline__ float floor_small_f(float a)
{
    return __fsub_rn(__fadd_rd(a, 12582912.0f), 12582912.0f);
}

// Run of samples, starting with the one at (x, y, z), whose texture values
// are certainly the flat value v of the current cell.  Every cell within
// L-infinity distance r-1 of a flat cell with distance r is flat, with the
// same value (face-adjacent flat cells share four texels).  Sample m of the
// run lies within m*dmax texels of sample 0 on each axis, so its computed
// cell (floor(x-0.5)+1) is within floor(m*dmax)+1 cells of the current one,
// and the texture unit, which quantises the coordinate before taking the
// floor, may read the cell next to that one: one more.  Hence samples with
// m*dmax <= r-3 read only cells of value v, and a flat 2x2x2 neighbourhood
// filters to exactly v.  Returns 0 where no run is certain.
__device__ __forceinline__ float flat_run(const float2 *__restrict__ rec, int cx, int cy,
                                          float x, float y, float z, float inv_dmax, float &v)
{
    const int i = floor_small(__fsub_rn(x, 0.5f)) + 1, j = floor_small(__fsub_rn(y, 0.5f)) + 1,
              k = floor_small(__fsub_rn(z, 0.5f)) + 1;
    const float2 r = __ldg(rec + i + cx * (j + cy * k));
    v = r.x;
    if (r.y < 3.0f) return 0.0f;
    // floor((r - 3) / dmax) + 1, every rounding downward so that the run
    // never exceeds the bound
    return floor_small_f(__fmul_rd(r.y - 3.0f, inv_dmax)) + 1.0f;
}

constexpr int kTexBurst = 4;   // texture samples taken per look at a non-flat record

template <bool TEX>
__device__ __forceinline__ float raytrace_voxel(const float *__restrict__ rho,
                                                cudaTextureObject_t tex,
                                                const float2 *__restrict__ rec, const PbGrid &g,
                                                const PbBeamGeom &B, int i, int j, int k,
                                                int cap, int *status)
{
    float px, py, pz, ux, uy, uz;
    vox_mm(B, g.spacing, i, j, k, px, py, pz);
    if (TEX) {
        ux = __fsub_rn(B.src[0], px);
        uy = __fsub_rn(B.src[1], py);
        uz = __fsub_rn(B.src[2], pz);
        const float nrm = rnorm3df(ux, uy, uz);
        ux = __fmul_rn(ux, nrm);
        uy = __fmul_rn(uy, nrm);
        uz = __fmul_rn(uz, nrm);
    } else {
        unit_to_source(B, px, py, pz, ux, uy, uz);
    }
    const float inv_s = __fdiv_rn(1.0f, g.spacing);
    const float fnx = (float)g.nx, fny = (float)g.ny, fnz = (float)g.nz;
    const float ix = B.iso[0], iy = B.iso[1], iz = B.iso[2];
    const int nsafe = safe_steps(g, B, inv_s, px, py, pz, ux, uy, uz, cap);
    double acc = 0.0;
    int n = 0;
    if (rec) {
        // runs through flat regions, the sampler elsewhere; the sample
        // counter is kept in FP32 (exact below 2^24).  Exact trilinear
        // weights on a flat cell also give exactly its value.
        const float dmax = fmaxf(fabsf(inv_s * ux), fmaxf(fabsf(inv_s * uy), fabsf(inv_s * uz))) +
                           1e-6f;
        const float inv_dmax = __frcp_rd(dmax);
        const float nsf = (float)nsafe;
        const int cx = g.nx + 1, cy = g.ny + 1;
        float t = 0.0f;
        while (t < nsf) {
            const float x = __fmaf_rn(inv_s, __fadd_rn(__fmaf_rn(ux, t, px), ix), 0.5f);
            const float y = __fmaf_rn(inv_s, __fadd_rn(__fmaf_rn(uy, t, py), iy), 0.5f);
            const float z = __fmaf_rn(inv_s, __fadd_rn(__fmaf_rn(uz, t, pz), iz), 0.5f);
            float v;
            const float run = flat_run(rec, cx, cy, x, y, z, inv_dmax, v);
            if (run > 0.0f) {
                const float m = fminf(run, nsf - t);
                acc += (double)(m * fmaxf(v, 0.0f));
                t += m;
            } else {
                // not flat here: the texture unit for the next few samples
                // before looking at the records again
                float part = fmaxf(ray_sample<TEX>(rho, tex, g, x, y, z), 0.0f);
                const float e = fminf(t + (float)kTexBurst, nsf);
                if constexpr (TEX) {
                    // all fetches of the burst issued together; those past
                    // e (possibly outside the grid: the border reads 0) are
                    // not added, so the sum is the loop's, bit for bit
                    // (measured 7.50 -> 7.24 ms for the whole WET)
                    float sv[kTexBurst - 1];
#pragma unroll
                    for (int q = 1; q < kTexBurst; ++q) {
                        const float tq = __fadd_rn(t, (float)q);
                        const float x = __fmaf_rn(inv_s, __fadd_rn(__fmaf_rn(ux, tq, px), ix), 0.5f);
                        const float y = __fmaf_rn(inv_s, __fadd_rn(__fmaf_rn(uy, tq, py), iy), 0.5f);
                        const float z = __fmaf_rn(inv_s, __fadd_rn(__fmaf_rn(uz, tq, pz), iz), 0.5f);
                        sv[q - 1] = fmaxf(tex3D<float>(tex, x, y, z), 0.0f);
                    }
#pragma unroll
                    for (int q = 1; q < kTexBurst; ++q)
                        part = __fadd_rn(t, (float)q) < e ? __fadd_rn(part, sv[q - 1]) : part;
                    t = fmaxf(__fadd_rn(t, 1.0f), e);
                } else {
                    for (t += 1.0f; t < e; t += 1.0f) {
                        const float x = __fmaf_rn(inv_s, __fadd_rn(__fmaf_rn(ux, t, px), ix), 0.5f);
                        const float y = __fmaf_rn(inv_s, __fadd_rn(__fmaf_rn(uy, t, py), iy), 0.5f);
                        const float z = __fmaf_rn(inv_s, __fadd_rn(__fmaf_rn(uz, t, pz), iz), 0.5f);
                        part += fmaxf(ray_sample<TEX>(rho, tex, g, x, y, z), 0.0f);
                    }
                }
                acc += (double)part;
            }
        }
        n = (int)t;
    } else {
        for (; n + 8 <= nsafe; n += 8) {
            float r[8];
#pragma unroll
            for (int m = 0; m < 8; ++m) {
                const float t = (float)(n + m);
                const float x = __fmaf_rn(inv_s, __fadd_rn(__fmaf_rn(ux, t, px), ix), 0.5f);
                const float y = __fmaf_rn(inv_s, __fadd_rn(__fmaf_rn(uy, t, py), iy), 0.5f);
                const float z = __fmaf_rn(inv_s, __fadd_rn(__fmaf_rn(uz, t, pz), iz), 0.5f);
                r[m] = ray_sample<TEX>(rho, tex, g, x, y, z);
            }
            float part = 0.0f;
#pragma unroll
            for (int m = 0; m < 8; ++m) part += fmaxf(r[m], 0.0f);
            acc += (double)part;
        }
    }
    float part = 0.0f;
    for (;; ++n) {
        const float t = (float)n;
        const float x = __fmaf_rn(inv_s, __fadd_rn(__fmaf_rn(ux, t, px), ix), 0.5f);
        const float y = __fmaf_rn(inv_s, __fadd_rn(__fmaf_rn(uy, t, py), iy), 0.5f);
        const float z = __fmaf_rn(inv_s, __fadd_rn(__fmaf_rn(uz, t, pz), iz), 0.5f);
        if (n >= nsafe &&
            !(x >= 0.0f && x < fnx && y >= 0.0f && y < fny && z >= 0.0f && z < fnz))
            break;
        if (n >= cap) {
            if (status) atomicOr(status, (int)PB_ERR_RAY_CAP);
            break;
        }
        part += fmaxf(ray_sample<TEX>(rho, tex, g, x, y, z), 0.0f);
    }
    acc += (double)part;
    return __double2float_rn(fma(0.1, acc, -0.05));
}

// Texture sampling: 12 resident blocks per SM (40 registers), more warps to
// cover the dependent record loads; measured faster than the unbounded 48
// registers.  The exact-trilinear version spills at 40 and is left unbounded.
template <bool TEX>
__global__ void __launch_bounds__(128, TEX ? 12 : 1)
k_raytrace(const float *__restrict__ rho, cudaTextureObject_t tex,
           const float2 *__restrict__ rec, PbGrid g, const __grid_constant__ BeamGeomSet bs,
           int zbricks, int cap, float *__restrict__ raw, int *status)
{
    const int b = blockIdx.z / zbricks;
    const int k = (blockIdx.z - b * zbricks) * 4 + threadIdx.z;
    const int j = blockIdx.y * 4 + threadIdx.y;
    const int i = blockIdx.x * 8 + threadIdx.x;
    if (i >= g.nx || j >= g.ny || k >= g.nz) return;
    const int64_t V = (int64_t)g.nx * g.ny * g.nz;
    const int64_t v = i + (int64_t)g.nx * (j + (int64_t)g.ny * k);
    raw[b * V + v] = raytrace_voxel<TEX>(rho, tex, rec, g, bs.b[b], i, j, k, cap, status);
}

// Per-beam table of the smoothing samples.  Sample (direction dd, radius
// dr = r + 1 mm) of voxel (i, j, k) lies, along each axis a, at index
// coordinate  m_a = i_a + dr * dm_a  up to the FP32 roundings of the
// reference's sample position (the map from head to image coordinates is
// linear and the voxel's own coordinate is an integer), where dm_a is the
// index step of 1 mm along the direction.  Where the fractional part of
// dr * dm_a is farther than the rounding bound from 0.5, roundf picks
// i_a + ro, ro = round(dr * dm_a), for every voxel of the beam.  The other
// (direction, radius, axis) triples are flagged in tmask and take the
// reference-order position per voxel, which is i_a + ro or i_a + ro + 1
// with ro = floor(dr * dm_a) there.  The table holds ro + 1/2 (hh): for a
// flagged triple, the half-integer the position is compared with.
struct SmoothBeam {
    int off[6][9];            // linear-index offset when no axis is flagged
    float hh[6][9][3];        // per-axis index offset ro + 1/2: ro = round(dr * dm_a),
                              // floor where flagged
    unsigned tmask[6];        // 3 bits (x, y, z) per radius, radius 1 lowest
    int margin[3];            // interior: margin_a <= i_a <= n_a - 1 - margin_a
    float inv_s;              // 1 / spacing in FP32
    int pow2;                 // the spacing is a power of two: inv_s is exact
};

struct SmoothSet {
    SmoothBeam b[PB_MAX_BEAMS];
};

// Which (direction, radius, axis) samples can come near a half-integer.  A
// voxel's reference-order index coordinate differs from the real-number
// i_a + dr*dm_a by at most `err` (FP32 roundings of positions no larger
// than the grid's extent plus the isocentre), so where the fractional part
// of dr*dm_a is farther than tie + 2*err + 1e-4 from 0.5, every voxel's
// sample rounds to i_a + round(dr*dm_a); elsewhere the kernel takes the
// reference-order index, which is one of the two integers around it.
// (With beams along the image axes the lateral step is exactly half a
// voxel along an axis, so every other radius of two directions is flagged.)
static void smooth_table(const PbGrid &g, const PbBeamGeom &B, const float *c, const float *sn,
                         double err, double tie, SmoothBeam &T)
{
    memset(&T, 0, sizeof(T));
    const double inv_s = 1.0 / (double)g.spacing;
    int e2;
    T.pow2 = frexp((double)g.spacing, &e2) == 0.5;
    T.inv_s = (float)inv_s;
    const double sg = B.singa, cg = B.cosga, st = B.sinta, ct = B.costa;
    // head (hx, hy, hz) -> (xz, yz, zz) = (-hx, hz, hy); gantry; couch:
    // x = (xz cg - yz sg) ct + zz st ; y = xz sg + yz cg ;
    // z = -(xz cg - yz sg) st + zz ct.  Rows: image axis; columns: hx, hy.
    const double M[3][2] = {{-cg * ct, st}, {-sg, 0.0}, {cg * st, ct}};
    const double band = tie + 2.0 * err + 1e-4;
    const int64_t sy = g.nx, sz = (int64_t)g.nx * g.ny;
    for (int dd = 0; dd < 6; ++dd) {
        double dm[3];
        for (int a = 0; a < 3; ++a)
            dm[a] = (M[a][0] * (double)c[dd] + M[a][1] * (double)sn[dd]) * inv_s;
        unsigned m = 0;
        for (int r = 0; r < 9; ++r) {
            const double dr = (double)(r + 1);
            // dr is a small integer, so the FP64 product is exact and its
            // FP32 rounding is the FP32 product
            int64_t off = 0;
            for (int a = 0; a < 3; ++a) {
                const double x = dr * dm[a];
                const bool flag = fabs((x - floor(x)) - 0.5) < band;
                if (flag) m |= 1u << (3 * r + a);
                // flagged: the lower of the two candidates (exact_steps)
                const int o = (int)(flag ? floor(x) : nearbyint(x));
                T.hh[dd][r][a] = (float)o + 0.5f;
                off += (a == 0 ? 1 : a == 1 ? sy : sz) * (int64_t)o;
                T.margin[a] = std::max(T.margin[a], (int)ceil(fabs(x)) + 1);
            }
            T.off[dd][r] = (int)off;   // used only when the grid has < 2^31 voxels
        }
        T.tmask[dd] = m;
    }
}

static void smooth_set(const PbGrid &g, const PbBeamGeom *beams, int n_beams, SmoothSet &o)
{
    float c[6], sn[6];
    smooth_dirs(c, sn);
    const double inv_s = 1.0 / (double)g.spacing;
    // Bound on |FP32 reference-order index - real index|: about 8 roundings
    // of a coordinate no larger than `ext` mm, divided by the spacing, plus
    // 2e-4; the band is twice that, at least 2e-3.
    double ext = g.spacing * (double)(g.nx > g.ny ? (g.nx > g.nz ? g.nx : g.nz)
                                                  : (g.ny > g.nz ? g.ny : g.nz));
    for (int b = 0; b < n_beams; ++b)
        for (int a = 0; a < 3; ++a) ext = fmax(ext, fabs((double)beams[b].iso[a]) + ext);
    const double err = 8.0 * ldexp(ext + 16.0, -24) * inv_s + 2e-4;
    const double tie = fmax(2e-3, 2.0 * err);
    for (int b = 0; b < n_beams; ++b) smooth_table(g, beams[b], c, sn, err, tie, o.b[b]);
}

// The correctly rounded quotient, out of line: the unrolled smoothing
// loop calls it from many places.
__device__ __noinline__ float div_rn(float q, float s) { return __fdiv_rn(q, s); }

// roundf(q / s) (CudaClasses.cuh:112-116) minus lo, for a flagged sample
// whose quotient lies within half a voxel of h = lo + 1/2: 1 when the
// quotient is above h, or equal to it and positive (roundf rounds halves
// away from zero), else 0.  The quotient is the correctly rounded one;
// with a power-of-two spacing 1/s is exact, so q * (1/s) is it.
template <bool POW2>
__device__ __forceinline__ int round_up(float q, float h, float s, float inv_s)
{
    const float m = POW2 ? __fmul_rn(q, inv_s) : div_rn(q, s);
    return (m > h || (m == h && h > 0.0f)) ? 1 : 0;
}

// Sample (dd, r) along the flagged axes: the reference's FP32 position
// (head point plus dr*(c, s, 0), rotated to the image frame, plus the
// isocentre) divided by the spacing and rounded, as 0/1 steps from the
// table's lower candidates; fi, fj, fk are the voxel's indexes as floats.
// Only the flagged axes' image coordinates are formed.
// The six smoothing directions (cos, sin of i pi/3) as the reference forms
// them on the device: the FP32 angle (float)i * pi / 3 and CUDA's sincosf
// (IMPTClasses.cu:175-177).  Ties decided by the FP32 sample positions
// depend on these exact values, so they are CUDA's, not the host library's.
__device__ __forceinline__ void smooth_dir_dev(int i, float &c, float &s)
{
    sincosf(__fdiv_rn(__fmul_rn((float)i, 3.141592654f), 3.0f), &s, &c);
}

template <bool POW2>
__device__ __forceinline__ void exact_steps(const PbBeamGeom &B, const SmoothBeam &T, float s,
                                            const float *dc, const float *ds, float hx,
                                            float hy, float hz, float fi, float fj, float fk,
                                            int dd, int r, int axes, int &ui, int &uj, int &uk)
{
    // h + dr * (cos, sin), dr = r + 1 mm, each one fused multiply-add as the
    // reference's compiled code forms it (IMPTClasses.cu:180-181)
    const float dr = (float)(r + 1);
    const float hxs = __fmaf_rn(dr, dc[dd], hx);
    const float hys = __fmaf_rn(dr, ds[dd], hy);
    float qx, qy, qz;
    if (axes & 1) {
        head_to_image_ref(B, hxs, hys, hz, qx, qy, qz);
        ui = round_up<POW2>(__fadd_rn(qx, B.iso[0]), __fadd_rn(fi, T.hh[dd][r][0]), s,
                            T.inv_s);
    }
    if (axes & 2) {
        head_to_image_ref(B, hxs, hys, hz, qx, qy, qz);
        uj = round_up<POW2>(__fadd_rn(qy, B.iso[1]), __fadd_rn(fj, T.hh[dd][r][1]), s,
                            T.inv_s);
    }
    if (axes & 4) {
        head_to_image_ref(B, hxs, hys, hz, qx, qy, qz);
        uk = round_up<POW2>(__fadd_rn(qz, B.iso[2]), __fadd_rn(fk, T.hh[dd][r][2]), s,
                            T.inv_s);
    }
}

// Smoothed WET: mean of the voxel's raw WET and the in-grid nearest-voxel
// samples at 1..9 mm along six BEV-lateral directions, taking radius dr
// while dr < 10*WET(cm) (IMPTClasses.cu:166-198), summed in FP32 in the
// reference's order (direction, then radius).  A sample is the voxel at
// a fixed offset from this one (SmoothBeam), except along flagged axes,
// where the reference's FP32 position is rounded (exact_steps); the
// chosen voxels are the reference's.  POW2: the grid spacing is a power
// of two.
template <bool POW2>
__device__ __forceinline__ float smooth_voxel(const float *__restrict__ R, const PbGrid &g,
                                              const PbBeamGeom &Bp, const SmoothBeam &T,
                                              const float *dc, const float *ds, int i, int j,
                                              int k)
{
    const int64_t v = i + (int64_t)g.nx * (j + (int64_t)g.ny * k);
    const float center = R[v];
    const float lim = __fmul_rn(center, 10.0f);
    if (!(1.0f < lim)) return center;
    // radii 1..nr: dr < lim and dr < 10
    const int nr = lim > 9.0f ? 9 : (int)ceilf(lim) - 1;
    const PbBeamGeom B = Bp;   // the rotation and isocentre in registers
    float px, py, pz, hx, hy, hz;
    vox_mm(B, g.spacing, i, j, k, px, py, pz);
    image_to_head_ref(B, px, py, pz, hx, hy, hz);
    const float s = g.spacing;
    const float fi = (float)i, fj = (float)j, fk = (float)k;
    float sum = center;
    // The radius loops run to 9 for every thread, the samples past the
    // voxel's own count masked out: the loop counters and the table reads
    // stay uniform across the warp, and whether a sample is flagged is a
    // uniform branch.
    if (i >= T.margin[0] && i <= g.nx - 1 - T.margin[0] && j >= T.margin[1] &&
        j <= g.ny - 1 - T.margin[1] && k >= T.margin[2] && k <= g.nz - 1 - T.margin[2] &&
        (int64_t)g.nx * g.ny * g.nz < ((int64_t)1 << 31)) {
        // Interior: both candidates of every sample lie inside the grid
        // (the margins), so there are no bounds tests and the indexes are
        // 32-bit.  A sample past the voxel's count is loaded and not added,
        // without a branch.
        const int vi = (int)v, sy = g.nx, sz = g.nx * g.ny;
        // The nine radii unrolled with an explicit count of 9 (the WET pass
        // of the 4-beam 256x256x160 plan: 6.79 ms, against 7.29 ms with a
        // bare "unroll", whose code came out larger, 7.31 ms unrolled by
        // three and 7.36 by two); the directions stay a loop.
        for (int dd = 0; dd < 6; ++dd) {
            const unsigned tm = T.tmask[dd];   // the same for the whole beam
#pragma unroll 9
            for (int r = 0; r < 9; ++r) {
                const int axes = (tm >> (3 * r)) & 7u;
                int idx = vi + T.off[dd][r];
                if (axes) {
                    int ui = 0, uj = 0, uk = 0;
                    exact_steps<POW2>(B, T, s, dc, ds, hx, hy, hz, fi, fj, fk, dd, r, axes, ui, uj,
                                      uk);
                    idx += ui + sy * uj + sz * uk;
                }
                const float x = __ldg(R + idx);
                sum = r < nr ? __fadd_rn(sum, x) : sum;
            }
        }
        return __fdiv_rn(sum, (float)(6 * nr + 1));
    }
    int n = 1;
    for (int dd = 0; dd < 6; ++dd) {
        unsigned tm = T.tmask[dd];
#pragma unroll 1
        for (int r = 0; r < 9; ++r, tm >>= 3) {
            int ii = i + __float2int_rd(T.hh[dd][r][0]), jj = j + __float2int_rd(T.hh[dd][r][1]),
                kk = k + __float2int_rd(T.hh[dd][r][2]);
            const int axes = tm & 7u;
            if (axes) {
                int ui = 0, uj = 0, uk = 0;
                exact_steps<POW2>(B, T, s, dc, ds, hx, hy, hz, fi, fj, fk, dd, r, axes, ui, uj,
                                  uk);
                ii += ui;
                jj += uj;
                kk += uk;
            }
            const bool take = r < nr && (unsigned)ii < (unsigned)g.nx &&
                              (unsigned)jj < (unsigned)g.ny && (unsigned)kk < (unsigned)g.nz;
            if (take) {
                sum = __fadd_rn(sum, __ldg(R + ii + (int64_t)g.nx * (jj + (int64_t)g.ny * kk)));
                n += 1;
            }
        }
    }
    return __fdiv_rn(sum, (float)n);
}

// 12 resident blocks per SM (40 registers) with a power-of-two spacing,
// measured faster; with the division call the kernel spills at 40 and is
// left unbounded.
template <bool POW2>
__global__ void __launch_bounds__(128, POW2 ? 12 : 1)
k_smooth(const float *__restrict__ raw, PbGrid g, const __grid_constant__ BeamGeomSet bs,
         const __grid_constant__ SmoothSet st, int zbricks, float *__restrict__ wet)
{
    __shared__ float s_dc[6], s_ds[6];
    const int tid = threadIdx.x + 8 * (threadIdx.y + 4 * threadIdx.z);
    if (tid < 6) smooth_dir_dev(tid, s_dc[tid], s_ds[tid]);
    __syncthreads();
    const int b = blockIdx.z / zbricks;
    const int k = (blockIdx.z - b * zbricks) * 4 + threadIdx.z;
    const int j = blockIdx.y * 4 + threadIdx.y;
    const int i = blockIdx.x * 8 + threadIdx.x;
    if (i >= g.nx || j >= g.ny || k >= g.nz) return;
    const int64_t V = (int64_t)g.nx * g.ny * g.nz;
    const int64_t v = i + (int64_t)g.nx * (j + (int64_t)g.ny * k);
    wet[b * V + v] = smooth_voxel<POW2>(raw + b * V, g, bs.b[b], st.b[b], s_dc, s_ds, i, j, k);
}

// One (plan, beam) of a batched WET pass.
struct BatchWet {
    PbGrid g;
    PbBeamGeom geom;
    const float *rlsp;
    cudaTextureObject_t tex;
    const float2 *rec;          // the texture's cell records (or null)
    float *raw;                 // this beam's unsmoothed WET (V)
    float *wet;                 // this beam's smoothed WET (V)
    SmoothBeam sm;              // this beam's smoothing samples
    int cap;
    int bx, by, bz;             // 8x4x4 bricks per axis
    long long brick_start;      // first brick of this item in the launch
};

__device__ __forceinline__ int find_wet_item(const BatchWet *__restrict__ items, int n,
                                             long long brick)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].brick_start <= brick) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Brick of 8x4x4 voxels of one (plan, beam) per block of 128 threads.
__device__ __forceinline__ bool brick_voxel(const BatchWet &W, long long brick, int &i, int &j,
                                            int &k)
{
    long long lb = brick - W.brick_start;
    const int bx = (int)(lb % W.bx);
    lb /= W.bx;
    const int by = (int)(lb % W.by);
    const int bz = (int)(lb / W.by);
    i = bx * 8 + (threadIdx.x & 7);
    j = by * 4 + ((threadIdx.x >> 3) & 3);
    k = bz * 4 + (threadIdx.x >> 5);
    return i < W.g.nx && j < W.g.ny && k < W.g.nz;
}

__global__ void __launch_bounds__(128)
k_raytrace_batch(const BatchWet *__restrict__ items, int n_items, int *status)
{
    const BatchWet &W = items[find_wet_item(items, n_items, blockIdx.x)];
    int i, j, k;
    if (!brick_voxel(W, blockIdx.x, i, j, k)) return;
    const float r =
        W.tex ? raytrace_voxel<true>(W.rlsp, W.tex, W.rec, W.g, W.geom, i, j, k, W.cap, status)
              : raytrace_voxel<false>(W.rlsp, 0, W.rec, W.g, W.geom, i, j, k, W.cap, status);
    W.raw[i + (int64_t)W.g.nx * (j + (int64_t)W.g.ny * k)] = r;
}

__global__ void __launch_bounds__(128)
k_smooth_batch(const BatchWet *__restrict__ items, int n_items)
{
    static_assert(sizeof(SmoothBeam) % 4 == 0, "the table is copied as words");
    __shared__ SmoothBeam sm;
    __shared__ float s_dc[6], s_ds[6];
    if (threadIdx.x < 6) smooth_dir_dev(threadIdx.x, s_dc[threadIdx.x], s_ds[threadIdx.x]);
    const BatchWet &W = items[find_wet_item(items, n_items, blockIdx.x)];
    // the block's sample table into shared memory (one item per block)
    const int *src = reinterpret_cast<const int *>(&W.sm);
    int *dst = reinterpret_cast<int *>(&sm);
    for (int q = threadIdx.x; q < (int)(sizeof(SmoothBeam) / 4); q += blockDim.x)
        dst[q] = __ldg(src + q);
    __syncthreads();
    int i, j, k;
    if (!brick_voxel(W, blockIdx.x, i, j, k)) return;
    float *out = W.wet + i + (int64_t)W.g.nx * (j + (int64_t)W.g.ny * k);
    *out = sm.pow2 ? smooth_voxel<true>(W.raw, W.g, W.geom, sm, s_dc, s_ds, i, j, k)
                   : smooth_voxel<false>(W.raw, W.g, W.geom, sm, s_dc, s_ds, i, j, k);
}

__device__ float g_smooth_dirs[12];

__global__ void k_smooth_dirs()
{
    if (threadIdx.x < 6)
        smooth_dir_dev(threadIdx.x, g_smooth_dirs[threadIdx.x], g_smooth_dirs[6 + threadIdx.x]);
}

PbStatus device_smooth_dirs(float *c, float *s)
{
    k_smooth_dirs<<<1, 32>>>();
    PbStatus st = check_launch("k_smooth_dirs");
    float v[12];
    if (st == PB_OK)
        st = check_cuda(cudaMemcpyFromSymbol(v, g_smooth_dirs, sizeof(v)),
                        "cudaMemcpyFromSymbol(directions)");
    if (st != PB_OK) return st;
    for (int i = 0; i < 6; ++i) {
        c[i] = v[i];
        s[i] = v[6 + i];
    }
    return PB_OK;
}

int ray_step_cap(const PbGrid &g)
{
    const double diag = g.spacing * sqrt((double)g.nx * g.nx + (double)g.ny * g.ny +
                                         (double)g.nz * g.nz);
    return (int)ceil(diag) + 2;
}

PbStatus launch_wet(const float *rlsp, cudaTextureObject_t tex, const float2 *rec,
                    const PbGrid &g, const PbBeamGeom *beams, int n_beams, float *raw,
                    float *wet, int *status, cudaStream_t st)
{
    BeamGeomSet bs;
    for (int b = 0; b < n_beams; ++b) bs.b[b] = beams[b];
    SmoothSet ss;
    smooth_set(g, beams, n_beams, ss);
    const int zb = (g.nz + 3) / 4;
    dim3 block(8, 4, 4);
    dim3 grid((g.nx + 7) / 8, (g.ny + 3) / 4, zb * n_beams);
    if (tex)
        k_raytrace<true><<<grid, block, 0, st>>>(rlsp, tex, rec, g, bs, zb, ray_step_cap(g),
                                                 raw, status);
    else
        k_raytrace<false><<<grid, block, 0, st>>>(rlsp, tex, rec, g, bs, zb,
                                                  ray_step_cap(g), raw, status);
    PbStatus s = check_launch("k_raytrace");
    if (s != PB_OK) return s;
    if (ss.b[0].pow2)
        k_smooth<true><<<grid, block, 0, st>>>(raw, g, bs, ss, zb, wet);
    else
        k_smooth<false><<<grid, block, 0, st>>>(raw, g, bs, ss, zb, wet);
    return check_launch("k_smooth");
}

void smooth_table_host(const PbGrid &g, const PbBeamGeom *beams, int n_beams, int beam,
                       int *off, float *hh, unsigned *tmask, int *margin)
{
    SmoothSet ss;
    smooth_set(g, beams, n_beams, ss);
    const SmoothBeam &T = ss.b[beam];
    memcpy(off, T.off, sizeof(T.off));
    memcpy(hh, T.hh, sizeof(T.hh));
    memcpy(tmask, T.tmask, sizeof(T.tmask));
    memcpy(margin, T.margin, sizeof(T.margin));
}

size_t batch_wet_size() { return sizeof(BatchWet); }

// Fills the batch records of one plan's beams; returns the bricks they use.
long long fill_batch_wet(void *items_host, int first, const PbGrid &g, const PbBeamGeom *beams,
                         int n_beams, const float *rlsp, cudaTextureObject_t tex,
                         const float2 *rec, float *raw, float *wet, long long brick_start)
{
    BatchWet *W = static_cast<BatchWet *>(items_host) + first;
    SmoothSet ss;
    smooth_set(g, beams, n_beams, ss);
    const int64_t V = (int64_t)g.nx * g.ny * g.nz;
    const int bx = (g.nx + 7) / 8, by = (g.ny + 3) / 4, bz = (g.nz + 3) / 4;
    const long long per = (long long)bx * by * bz;
    for (int b = 0; b < n_beams; ++b) {
        BatchWet &w = W[b];
        w.g = g;
        w.geom = beams[b];
        w.rlsp = rlsp;
        w.tex = tex;
        w.rec = rec;
        w.raw = raw + b * V;
        w.wet = wet + b * V;
        w.sm = ss.b[b];
        w.cap = ray_step_cap(g);
        w.bx = bx;
        w.by = by;
        w.bz = bz;
        w.brick_start = brick_start + per * b;
    }
    return per * n_beams;
}

PbStatus launch_wet_batch(const void *items_dev, int n_items, long long n_bricks, int *status,
                          cudaStream_t st)
{
    if (n_bricks <= 0) return PB_OK;
    if (n_bricks > 0x7fffffffLL) return set_error(PB_ERR_INVALID, "batch too large");
    const BatchWet *I = static_cast<const BatchWet *>(items_dev);
    k_raytrace_batch<<<(unsigned)n_bricks, 128, 0, st>>>(I, n_items, status);
    PbStatus s = check_launch("k_raytrace_batch");
    if (s != PB_OK) return s;
    k_smooth_batch<<<(unsigned)n_bricks, 128, 0, st>>>(I, n_items);
    return check_launch("k_smooth_batch");
}

// Cells of a volume with border 0: cell (ci, cj, ck) holds the 2x2x2
// texels with base (ci-1, cj-1, ck-1) -- the texels a linear fetch reads
// for a coordinate inside it.  A cell is flat when its eight texels are
// equal.  Two adjacent flat cells share texels, so a connected flat region
// has one value.
constexpr int kRunCap = 15;   // largest stored distance (cells)
constexpr int kFlagPad = 16;  // zero bytes before and after each row of flat flags

// Row lengths (bytes) of the distance passes' work arrays: cells padded to
// a multiple of 4, and the flat flags with kFlagPad bytes on each side.
__host__ __device__ __forceinline__ int cell_row(int nx) { return (nx + 1 + 3) & ~3; }
__host__ __device__ __forceinline__ int flag_row(int nx) { return cell_row(nx) + 2 * kFlagPad; }

// Pass 0: flat cells -> their value, else NaN; 1-D distance along x to the
// nearest non-flat cell (cells outside the cell grid count as non-flat),
// capped at kRunCap.
__global__ void __launch_bounds__(256)
k_cell_flat(const float *__restrict__ rho, PbGrid g, float *__restrict__ value,
            unsigned char *__restrict__ flag)
{
    const int cx = g.nx + 1, cy = g.ny + 1, cz = g.nz + 1;
    const int64_t n = (int64_t)cx * cy * cz;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int ci = (int)(c % cx);
        const int cj = (int)((c / cx) % cy);
        const int ck = (int)(c / ((int64_t)cx * cy));
        float v0 = 0.0f;
        bool flat = true;
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const int i = ci - 1 + (t & 1), j = cj - 1 + ((t >> 1) & 1), k = ck - 1 + (t >> 2);
            const bool in = i >= 0 && i < g.nx && j >= 0 && j < g.ny && k >= 0 && k < g.nz;
            const float v = in ? __ldg(rho + i + (int64_t)g.nx * (j + (int64_t)g.ny * k)) : 0.0f;
            if (t == 0) v0 = v;
            else flat &= (v == v0);
        }
        const bool f = flat && v0 == v0;
        value[c] = f ? v0 : __int_as_float(0x7fc00000);
        // the x distance pass's input: kRunCap where flat, in rows with
        // kFlagPad zero bytes before and after (flag_row)
        flag[(c / cx) * flag_row(g.nx) + kFlagPad + ci] = f ? (unsigned char)kRunCap : 0;
    }
}

// Separable L-infinity distance to the nearest non-flat cell, capped at
// kRunCap: min over |k| <= kRunCap of max(|k|, d(pos + k)), a cell outside
// the grid counting as non-flat (d = 0).  All three passes work on four
// cells per 32-bit word with byte-wise SIMD max/min.  The distances are
// bytes in rows padded to a multiple of 4 cells (cell_row); the x pass reads
// the flat flags (kRunCap or 0) in rows with kFlagPad zero bytes on each
// side (flag_row), so that every tap of a word is two aligned words and a
// funnel shift.
__global__ void __launch_bounds__(256, 4)
k_cell_dist_x(PbGrid g, const unsigned char *__restrict__ flag, unsigned int *__restrict__ dout)
{
    static_assert(kFlagPad > kRunCap && kFlagPad % 4 == 0, "every tap inside the padded row");
    constexpr int kWords = (kFlagPad + kRunCap) / 4 + 2;   // words w .. w + kWords - 1
    const int cy = g.ny + 1, cz = g.nz + 1, words = cell_row(g.nx) / 4, frow = flag_row(g.nx);
    const int64_t n = (int64_t)words * cy * cz;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int w = (int)(c % words);
        const int64_t line = c / words;
        // cells 4w - kRunCap .. 4w + 3 + kRunCap: flag bytes from
        // 4w + kFlagPad - kRunCap on, within the row's words from w (the last
        // word read ends at most at the row's last byte)
        const unsigned int *src =
            reinterpret_cast<const unsigned int *>(flag + line * frow + 4 * w);
        unsigned int W[kWords];
#pragma unroll
        for (int j = 0; j < kWords; ++j) W[j] = __ldg(src + j);
        unsigned int best = kRunCap * 0x01010101u;
#pragma unroll
        for (int k = -kRunCap; k <= kRunCap; ++k) {
            const int b = kFlagPad + k;   // first byte of the window
            const unsigned int d = __funnelshift_r(W[b >> 2], W[(b >> 2) + 1], 8 * (b & 3));
            const unsigned int ak = (unsigned int)(k < 0 ? -k : k) * 0x01010101u;
            best = __vminu4(best, __vmaxu4(ak, d));
        }
        dout[c] = best;
    }
}

template <int AXIS>
__global__ void __launch_bounds__(256, 4)
k_cell_dist4(PbGrid g, const unsigned int *__restrict__ din, unsigned int *__restrict__ dout)
{
    static_assert(AXIS == 1 || AXIS == 2, "y or z");
    const int cy = g.ny + 1, cz = g.nz + 1, words = cell_row(g.nx) / 4;
    const int64_t n = (int64_t)words * cy * cz;
    const int len = AXIS == 1 ? cy : cz;
    const int64_t stride = AXIS == 1 ? (int64_t)words : (int64_t)words * cy;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int pos = AXIS == 1 ? (int)((c / words) % cy) : (int)(c / ((int64_t)words * cy));
        unsigned int best = kRunCap * 0x01010101u;
#pragma unroll
        for (int k = -kRunCap; k <= kRunCap; ++k) {
            const int q = pos + k;
            const unsigned int ak = (unsigned int)(k < 0 ? -k : k) * 0x01010101u;
            // outside the grid counts as non-flat (distance 0)
            const unsigned int d = (q >= 0 && q < len) ? __ldg(din + c + k * stride) : 0u;
            best = __vminu4(best, __vmaxu4(ak, d));
        }
        dout[c] = best;
    }
}

// Record per cell: (value, distance); distance 0 for non-flat cells.
__global__ void __launch_bounds__(256)
k_cell_records(PbGrid g, const float *__restrict__ value, const unsigned char *__restrict__ dist,
               float2 *__restrict__ rec)
{
    const int cx = g.nx + 1, row = cell_row(g.nx);
    const int64_t n = (int64_t)cx * (g.ny + 1) * (g.nz + 1);
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        const float v = value[c];
        const unsigned char d = dist[(c / cx) * row + c % cx];
        rec[c] = make_float2(v == v ? v : 0.0f, v == v ? (float)d : 0.0f);
    }
}

// 3-D texture over an RLSP volume: float channel, linear filter, border 0,
// unnormalised coordinates (TextureClasses.cu:14-41), and the cell records
// the ray trace uses to take runs of samples in flat regions at once.
struct RlspTexture {
    cudaArray_t arr = nullptr;
    cudaTextureObject_t tex = 0;
    float2 *rec = nullptr;            // (nx+1)(ny+1)(nz+1) cell records
    float *value = nullptr;           // work: flat values
    unsigned char *d0 = nullptr, *d1 = nullptr;  // work: distance passes
    unsigned char *flag = nullptr;    // work: flat flags (zero-padded rows)
    int nx = 0, ny = 0, nz = 0;
};

static PbStatus texture_fill(RlspTexture *t, const float *rlsp, cudaStream_t st)
{
    cudaMemcpy3DParms p{};
    p.srcPtr = make_cudaPitchedPtr(const_cast<float *>(rlsp), sizeof(float) * (size_t)t->nx, t->nx,
                                   t->ny);
    p.dstArray = t->arr;
    p.extent = make_cudaExtent(t->nx, t->ny, t->nz);
    p.kind = cudaMemcpyDeviceToDevice;
    if (t->arr) {
        const PbStatus s = check_cuda(cudaMemcpy3DAsync(&p, st), "cudaMemcpy3DAsync");
        if (s != PB_OK) return s;
    }
    const PbGrid g{t->nx, t->ny, t->nz, 1.0f};
    const int blocks = 148 * 8;
    k_cell_flat<<<blocks, 256, 0, st>>>(rlsp, g, t->value, t->flag);
    k_cell_dist_x<<<blocks, 256, 0, st>>>(g, t->flag, reinterpret_cast<unsigned int *>(t->d0));
    k_cell_dist4<1><<<blocks, 256, 0, st>>>(g, reinterpret_cast<const unsigned int *>(t->d0),
                                            reinterpret_cast<unsigned int *>(t->d1));
    k_cell_dist4<2><<<blocks, 256, 0, st>>>(g, reinterpret_cast<const unsigned int *>(t->d1),
                                            reinterpret_cast<unsigned int *>(t->d0));
    k_cell_records<<<blocks, 256, 0, st>>>(g, t->value, t->d0, t->rec);
    return check_launch("cell records");
}

static void texture_free(RlspTexture *t)
{
    if (t->tex) cudaDestroyTextureObject(t->tex);
    if (t->arr) cudaFreeArray(t->arr);
    cudaFree(t->rec);
    cudaFree(t->value);
    cudaFree(t->d0);
    cudaFree(t->d1);
    cudaFree(t->flag);
    delete t;
}

// with_texture false: the cell records only, for exact-trilinear sampling.
PbStatus texture_create(const float *rlsp, const PbGrid &g, uint64_t *out, cudaStream_t st,
                        bool with_texture)
{
    const size_t ncell = (size_t)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
    if (ncell > (size_t)INT32_MAX)
        return set_error(PB_ERR_INVALID, "grid too large for a texture (%zu cells)", ncell);
    RlspTexture *t = new (std::nothrow) RlspTexture;
    if (!t) return set_error(PB_ERR_NOMEM, "host allocation failed");
    t->nx = g.nx;
    t->ny = g.ny;
    t->nz = g.nz;
    cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
    cudaExtent ext = make_cudaExtent(g.nx, g.ny, g.nz);
    PbStatus s = PB_OK;
    if (with_texture)
        s = check_cuda(cudaMalloc3DArray(&t->arr, &ch, ext, cudaArrayDefault),
                       "cudaMalloc3DArray");
    if (s == PB_OK) s = check_cuda(cudaMalloc(&t->rec, sizeof(float2) * ncell), "cudaMalloc");
    if (s == PB_OK) s = check_cuda(cudaMalloc(&t->value, sizeof(float) * ncell), "cudaMalloc");
    // distance passes: rows padded to 4 cells (32-bit words)
    const size_t npad = (size_t)cell_row(g.nx) * (g.ny + 1) * (g.nz + 1);
    if (s == PB_OK) s = check_cuda(cudaMalloc(&t->d0, npad), "cudaMalloc");
    if (s == PB_OK) s = check_cuda(cudaMalloc(&t->d1, npad), "cudaMalloc");
    // flat flags: the padding bytes stay zero, the cells are rewritten by
    // every fill
    const size_t nflag = (size_t)flag_row(g.nx) * (g.ny + 1) * (g.nz + 1);
    if (s == PB_OK) s = check_cuda(cudaMalloc(&t->flag, nflag), "cudaMalloc");
    if (s == PB_OK) s = check_cuda(cudaMemset(t->flag, 0, nflag), "cudaMemset");
    if (s == PB_OK && with_texture) {
        cudaResourceDesc rd{};
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = t->arr;
        cudaTextureDesc td{};
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 0;
        s = check_cuda(cudaCreateTextureObject(&t->tex, &rd, &td, nullptr),
                       "cudaCreateTextureObject");
    }
    if (s == PB_OK) s = texture_fill(t, rlsp, st);
    if (s != PB_OK) {
        texture_free(t);
        return s;
    }
    *out = reinterpret_cast<uint64_t>(t);
    return PB_OK;
}

PbStatus texture_update(uint64_t h, const float *rlsp, cudaStream_t st)
{
    return texture_fill(reinterpret_cast<RlspTexture *>(h), rlsp, st);
}

bool texture_matches(uint64_t h, const PbGrid &g)
{
    const RlspTexture *t = reinterpret_cast<const RlspTexture *>(h);
    return t && t->nx == g.nx && t->ny == g.ny && t->nz == g.nz;
}

bool texture_samples(uint64_t h)
{
    return h && reinterpret_cast<const RlspTexture *>(h)->tex != 0;
}

cudaTextureObject_t texture_object(uint64_t h)
{
    return h ? reinterpret_cast<const RlspTexture *>(h)->tex : 0;
}

const float2 *texture_cells(uint64_t h)
{
    return h ? reinterpret_cast<const RlspTexture *>(h)->rec : nullptr;
}

void texture_destroy(uint64_t h)
{
    RlspTexture *t = reinterpret_cast<RlspTexture *>(h);
    if (t) texture_free(t);
}

}  // namespace pb
