// pb_dose.cu -- forward pencil-beam dose, its adjoint (spot-weight
// gradient), the quadratic objective and the dense pair count.
//
// Physics per (voxel, layer), following DoseCUDA/dose_kernels/IMPTClasses.cu:
//   cut  10*WET > 1.1*R80 -> no dose                            (:222-226)
//   IDD, sigma_mcs from the LUT row of the layer's energy        (:69-92)
//   sigma_air = A d^2 + B d + C, d = dist_src - wet + 0.7 R80     (:94-102)
//   halo sigma / weight closed forms                             (:104-121)
//   D += mu (Pf exp(-r^2/2st^2) + Hf exp(-r^2/2sht^2))           (:204-271)
// with r the distance of the voxel from the spot's diverging axis
// (:123-133).  The axis distance is evaluated as |t x ray|^2/|t|^2, the
// same quantity as |ray|^2 - (t.ray)^2/|t|^2 without its cancellation:
//   t = (xs/VSADX, ys/VSADY, -1), ray = (X-xs, Y-ys, Z)
//   t x ray = ( Y - ys(1-Z/VSADY), -(X - xs(1-Z/VSADX)),
//               (xs/VSADX) Y - (ys/VSADY) X - xs ys (1/VSADX - 1/VSADY) ).
//
// Work decomposition: one block of 128 threads per 8x8x8 voxel tile, four
// voxels per thread; all beams and layers of the plan are looped inside the
// block, so each voxel's dose is written once, compensated (Neumaier) across
// layers and beams, with no atomics.  Per (tile, layer): a test on the
// layer's bounds (pb_layer_bounds) skips layers no spot of which can reach
// the tile; the layer's LUT row is staged in shared memory; the layer's
// spots are culled against the tile -- a Gaussian term is skipped when, at
// every voxel of the tile, it is below 2^-24 of the voxel's peak factor
// (bound from the tile's BEV box and the widest sigma in the tile), which
// leaves spots with both terms and spots with the halo term only.
// Surviving spots are compacted into shared memory (each value stored
// twice), and every thread evaluates each spot on its four voxels as two
// packed FP32x2 voxel pairs (two spot-voxel pairs per instruction) with the
// SFU's ex2.
//
// The adjoint is the same tile code (dose_tile in adjoint mode): the same
// decisions, with the voxels where dObj/dD = 0 inactive; the per-spot sums
// over a thread's voxels meet across the warp with a transposed butterfly,
// across the block in shared memory, and go to the gradient with one global
// atomic per spot per (tile, layer).
#include <climits>
#include <type_traits>
#include "pb_internal.h"

namespace pb {

constexpr float kCullLog2 = 24.0f;  // skip factors below 2^-24

struct PlanArgs {
    PbGrid g;
    int n_beams;
    int tiles_x, tiles_y, tiles_z;
    int centre[3];   // voxel holding the mean isocentre (clamped to the grid)
    const int *order;   // line-tile launches: tile of each block (raster index), or NULL
    float scale;
    PbBeam beams[PB_MAX_BEAMS];
};

// One spot, each value duplicated, for packed FP32x2 evaluation against a
// pair of voxels.
struct __align__(16) SpotRec {
    float4 a;  // (-x, -x, -y, -y)
    float4 b;  // (tx, tx, -ty, -ty)
    float4 c;  // (-cs, -cs, it2, it2)
    float4 d;  // (mu, mu, 0, 0)
};


struct TileBounds {
    float x0, x1, y0, y1, gx0, gx1, gy0, gy1;  // BEV box and divergence factors
    float d0, d1, w0, w1;                      // source distance range, least and
                                               // greatest 10*WET
};

// Slots of the per-warp reduction array: 11 for tile_bounds, 2 for block_max2.
constexpr int kRedSlots = 13;

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 lo2(const float4 &v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(const float4 &v) { return make_float2(v.z, v.w); }
__device__ __forceinline__ float2 ex2x2(float2 a) { return make_float2(ex2(a.x), ex2(a.y)); }

// Squared axis distance of two spots at one voxel, times 1/|t|^2.
__device__ __forceinline__ float2 axis_r2(float2 nx, float2 ny, float2 tx, float2 nty,
                                          float2 ncs, float2 it2, float2 X, float2 Y,
                                          float2 GX, float2 GY)
{
    const float2 ax = __ffma2_rn(nx, GX, X);
    const float2 ay = __ffma2_rn(ny, GY, Y);
    const float2 cz = __ffma2_rn(tx, Y, __ffma2_rn(nty, X, ncs));
    const float2 S = __ffma2_rn(ax, ax, __ffma2_rn(ay, ay, __fmul2_rn(cz, cz)));
    return __fmul2_rn(S, it2);
}

// Per-layer constants of the Gaussian parameters (uniform over a block).
struct LayerK {
    float r80, off;          // R80, 0.7 R80
    float ca, cb, cc;        // sigma_air = A d^2 + B d + C
    float d0, inv_step;      // depth table: first depth, 1 / (second - first)
    float c_log, c_sh;       // 0.0014 R80, 0.22 R80
    float k_wh, c_wh;        // 1 / (11.2 - 0.023 R80), 0.35 (0.0017 R80^2 - R80)
    float r3sq, c_lin;       // (R80 + 3)^2, 1.61e-9 (R80 + 3)^2
};

// A LUT row: a plain pointer (shared memory) or RowG, a row in global
// memory read through the read-only data cache.
struct RowG {
    const float *p;
    __device__ __forceinline__ float operator[](int i) const { return __ldg(p + i); }
};

template <class Row>
__device__ __forceinline__ LayerK layer_consts(float r80, const float *cabc, const Row &s_dep,
                                               int lut_len)
{
    LayerK K;
    K.r80 = r80;
    K.off = __fmul_rn(0.7f, r80);
    K.ca = __ldg(cabc);
    K.cb = __ldg(cabc + 1);
    K.cc = __ldg(cabc + 2);
    K.d0 = s_dep[0];
    const float step = lut_len > 1 ? __fsub_rn(s_dep[1], s_dep[0]) : 0.0f;
    K.inv_step = step > 0.0f ? __fdiv_rn(1.0f, step) : 0.0f;
    K.c_log = __fmul_rn(0.0014f, r80);
    K.c_sh = __fmul_rn(0.22f, r80);
    K.k_wh = __fdiv_rn(1.0f, __fsub_rn(11.2f, __fmul_rn(0.023f, r80)));
    K.c_wh = __fmul_rn(0.35f, __fsub_rn(__fmul_rn(__fmul_rn(0.0017f, r80), r80), r80));
    const float r3 = __fadd_rn(r80, 3.0f);
    K.r3sq = __fmul_rn(r3, r3);
    K.c_lin = __fmul_rn(1.61e-9f, K.r3sq);
    return K;
}

// Per-(voxel, layer) Gaussian parameters.  wet_mm is 10*WET (cm), dist the
// distance to the source (mm).  Exponent scales are pre-multiplied by
// log2(e) for ex2.
//
// The LUT row is the first depth >= wet_mm (lowerBound,
// CudaClasses.cuh:130-144): guessed from the first depth and the first step
// (exact for the uniform 1 mm tables of the beam models), then moved until
// it is that row, so any ascending depth table gives the binary search's
// row.  The halo closed forms (IMPTClasses.cu:104-121) and the Gaussian
// prefactors use the SFU's log2 and reciprocal (relative error ~1e-7).
// Every operation is an explicitly rounded intrinsic, so that no
// instantiation of the tile code contracts them differently: all kernel
// shapes give the same bits.
template <class Row>
__device__ __forceinline__ void layer_params(float wet_mm, float dist, const LayerK &K,
                                             const Row &s_dep, const Row &s_sig,
                                             const Row &s_idd, int lut_len, float &pf,
                                             float &hf, float &ps2, float &hs2)
{
    const float gs = ceilf(__fmul_rn(__fsub_rn(wet_mm, K.d0), K.inv_step));
    int lo = gs > 0.0f ? (gs < (float)lut_len ? (int)gs : lut_len) : 0;
    if (wet_mm != wet_mm) lo = lut_len;   // NaN compares false: the search ends high
    while (lo > 0 && s_dep[lo - 1] >= wet_mm) --lo;
    while (lo < lut_len && s_dep[lo] < wet_mm) ++lo;
    float idd, sms;
    if (lo == lut_len) {
        idd = s_idd[lo - 1];
        sms = s_sig[lo - 1];
    } else if (lo == 0) {
        idd = s_idd[0];
        sms = s_sig[0];
    } else {
        const float f = __fdividef(__fsub_rn(wet_mm, s_dep[lo - 1]),
                                   __fsub_rn(s_dep[lo], s_dep[lo - 1]));
        idd = __fmaf_rn(__fsub_rn(s_idd[lo], s_idd[lo - 1]), f, s_idd[lo - 1]);
        sms = __fmaf_rn(__fsub_rn(s_sig[lo], s_sig[lo - 1]), f, s_sig[lo - 1]);
    }
    const float d = __fadd_rn(__fsub_rn(dist, wet_mm), K.off);
    const float st = __fadd_rn(__fmaf_rn(__fmaf_rn(K.ca, d, K.cb), d, K.cc), sms);
    const float w = fminf(fmaxf(wet_mm, 0.1f), __fsub_rn(K.r80, 0.1f));
    const float a1 = __fsub_rn(__fsub_rn(w, K.r80), 5.0f);
    float sh = __fadd_rn(2.85f, __fmul_rn(K.c_log, __logf(__fadd_rn(w, 3.0f))));
    sh = __fadd_rn(sh, __fmul_rn(0.06f, w));
    sh = __fsub_rn(sh, __fmul_rn(__fmul_rn(7.4e-5f, w), w));
    sh = __fsub_rn(sh, __fdividef(K.c_sh, __fmul_rn(a1, a1)));
    float wh = __fmul_rn(0.052f, __logf(__fmaf_rn(w, K.k_wh, 1.13f)));
    wh = __fadd_rn(wh, __fdividef(K.c_wh, __fsub_rn(K.r3sq, __fmul_rn(w, w))));
    wh = __fsub_rn(wh, __fmul_rn(K.c_lin, w));
    sh = fmaxf(sh, 0.0f);
    wh = fminf(fmaxf(wh, 0.0f), 0.9f);
    const float st2 = __fmul_rn(st, st);
    const float sht2 = __fmaf_rn(sh, sh, st2);
    const float rp = __fdividef(1.0f, st2), rh = __fdividef(1.0f, sht2);
    const float iddn = __fmul_rn(idd, 1.0f / kTwoPi);
    pf = __fmul_rn(__fmul_rn(__fsub_rn(1.0f, wh), iddn), rp);
    hf = __fmul_rn(__fmul_rn(wh, iddn), rh);
    ps2 = st2 != 0.0f ? __fmul_rn(-0.5f * kLog2e, rp) : -INFINITY;
    hs2 = sht2 != 0.0f ? __fmul_rn(-0.5f * kLog2e, rh) : -INFINITY;
}

// Squared distance (times 1/|t|^2) from the spot's axis to the tile's BEV
// box, a lower bound over the tile's voxels of the axis_r2 value.
__device__ __forceinline__ float cull_r2(float xs, float ys, float it2, const TileBounds &tb)
{
    const float p0 = xs * tb.gx0, p1 = xs * tb.gx1;
    const float lox = tb.x0 - fmaxf(p0, p1), hix = tb.x1 - fminf(p0, p1);
    const float dx = fmaxf(0.0f, fmaxf(lox, -hix));
    const float q0 = ys * tb.gy0, q1 = ys * tb.gy1;
    const float loy = tb.y0 - fmaxf(q0, q1), hiy = tb.y1 - fminf(q0, q1);
    const float dy = fmaxf(0.0f, fmaxf(loy, -hiy));
    return __fmul_rn(__fmaf_rn(dx, dx, __fmul_rn(dy, dy)), it2);
}

// Spot classes per tile and layer: the halo term is below 2^-24 of its
// peak at every voxel of the tile (0, skipped); only the primary term is
// (1, halo only); neither (2, both terms).  nhs / nps are the smallest
// |hs2| / |ps2| among the tile's active voxels (the widest halo and primary
// Gaussians); the halo is never narrower than the primary, so nps >= nhs.
__device__ __forceinline__ int cull_class(float e, float nhs, float nps)
{
    if (e * nhs >= kCullLog2) return 0;
    return (e * nps >= kCullLog2) ? 1 : 2;
}

__device__ __forceinline__ void neumaier(float &s, float &c, float x)
{
    const float t = s + x;
    if (fabsf(s) >= fabsf(x)) c += (s - t) + x; else c += (x - t) + s;
    s = t;
}

// Block-wide min/max of the tile's BEV box over valid voxels.
// Block-wide box of the tile's valid voxels: BEV x, y and divergence
// factors (min and max), distance to the source (min and max), 10*WET (min,
// with NaN taken as -infinity).
template <int NV, int NT>
__device__ __forceinline__ TileBounds tile_bounds(const float *X, const float *Y,
                                                  const float *GX, const float *GY,
                                                  const float *D, const float *W,
                                                  const bool *valid,
                                                  float (*s_red)[kRedSlots])
{
    constexpr int kWarps = NT / 32;
    float v[12] = {INFINITY, -INFINITY, INFINITY, -INFINITY, INFINITY, -INFINITY,
                   INFINITY, -INFINITY, INFINITY, -INFINITY, INFINITY, -INFINITY};
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        if (!valid[q]) continue;
        v[0] = fminf(v[0], X[q]);  v[1] = fmaxf(v[1], X[q]);
        v[2] = fminf(v[2], Y[q]);  v[3] = fmaxf(v[3], Y[q]);
        v[4] = fminf(v[4], GX[q]); v[5] = fmaxf(v[5], GX[q]);
        v[6] = fminf(v[6], GY[q]); v[7] = fmaxf(v[7], GY[q]);
        v[8] = fminf(v[8], D[q]);  v[9] = fmaxf(v[9], D[q]);
        // a NaN depth is never skipped: it widens both depth bounds
        v[10] = fminf(v[10], W[q] == W[q] ? W[q] : -INFINITY);
        v[11] = fmaxf(v[11], W[q] == W[q] ? W[q] : INFINITY);
    }
    // slot m: odd = max, even = min
#pragma unroll
    for (int m = 0; m < 12; ++m) v[m] = (m & 1) ? warp_max(v[m]) : warp_min(v[m]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
#pragma unroll
        for (int m = 0; m < 12; ++m) s_red[warp][m] = v[m];
    }
    __syncthreads();
    float r[12];
#pragma unroll
    for (int m = 0; m < 12; ++m) r[m] = s_red[0][m];
    for (int w = 1; w < kWarps; ++w) {
#pragma unroll
        for (int m = 0; m < 12; ++m)
            r[m] = (m & 1) ? fmaxf(r[m], s_red[w][m]) : fminf(r[m], s_red[w][m]);
    }
    TileBounds tb;
    tb.x0 = r[0]; tb.x1 = r[1]; tb.y0 = r[2]; tb.y1 = r[3];
    tb.gx0 = r[4]; tb.gx1 = r[5]; tb.gy0 = r[6]; tb.gy1 = r[7];
    tb.d0 = r[8]; tb.d1 = r[9]; tb.w0 = r[10]; tb.w1 = r[11];
    return tb;
}

// Block-wide maxima of two values (slots 11 and 12 of s_red).
template <int NT>
__device__ __forceinline__ void block_max2(float a, float b, float (*s_red)[kRedSlots],
                                           float &ra, float &rb)
{
    constexpr int kWarps = NT / 32;
    a = warp_max(a);
    b = warp_max(b);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        s_red[warp][11] = a;
        s_red[warp][12] = b;
    }
    __syncthreads();
    ra = s_red[0][11];
    rb = s_red[0][12];
    for (int w = 1; w < kWarps; ++w) {
        ra = fmaxf(ra, s_red[w][11]);
        rb = fmaxf(rb, s_red[w][12]);
    }
}

// True when no spot of layer L can pass cull_class at any voxel of the
// tile, decided from the layer's bounds alone (before any per-voxel work).
// A spot's cull value is (dx^2 + dy^2) * it2 * nhs; here dx, dy are taken
// to the box of all the layer's spot axes at the tile's depths (FP32
// products are monotone, so each spot's own dx, dy are no smaller), it2 to
// its least value over that box, and nhs to 0.5 log2(e) / sigma^2 with
// sigma bounding every active voxel's total halo sigma:
//   sigma^2 <= sh_max^2 + (max |A d^2 + B d + C| + mcs_max)^2
// over d = dist - wet_mm + 0.7 R80, dist in the tile's range and wet_mm in
// [the tile's least 10*WET, 1.1 R80].  Margins (1 % on sigma^2, 0.1 % on
// it2) cover the kernels' FP32 and SFU arithmetic, so a skipped layer is
// one whose every spot the per-spot cull would drop: the dose is the same.
// An upper bound of the nuclear-halo sigma of layer_params (mm) over the
// depths w0 <= w <= w1 (10*WET, mm): with the depth clamped to
// [0.1, R80 - 0.1] as there, c_log log(w + 3) and -c_sh / (w - R80 - 5)^2
// are monotone in w (w - R80 - 5 <= -5.1 < 0), so each is largest at an
// end of the range; 0.06 w - 7.4e-5 w^2 is concave, largest at an end or
// at its vertex.  INFINITY when the range is empty or not a number.
__device__ __forceinline__ float halo_sigma_bound(float r80, float w0, float w1)
{
    const float top = r80 - 0.1f;
    const float lo = fminf(fmaxf(w0, 0.1f), top), hi = fminf(fmaxf(w1, 0.1f), top);
    if (!(lo <= hi)) return INFINITY;
    const float cl = 0.0014f * r80, cs = 0.22f * r80;
    const float l0 = cl * logf(lo + 3.0f), l1 = cl * logf(hi + 3.0f);
    const float a0 = lo - r80 - 5.0f, a1 = hi - r80 - 5.0f;
    const float q0 = -cs / (a0 * a0), q1 = -cs / (a1 * a1);
    float p = fmaxf(0.06f * lo - 7.4e-5f * lo * lo, 0.06f * hi - 7.4e-5f * hi * hi);
    const float wv = 0.06f / (2.0f * 7.4e-5f);
    if (wv > lo && wv < hi) p = fmaxf(p, 0.06f * wv - 7.4e-5f * wv * wv);
    const float b = 2.85f + fmaxf(l0, l1) + fmaxf(q0, q1) + p;
    return b != b ? INFINITY : fmaxf(b, 0.0f) * 1.001f + 1e-3f;
}

// The layer's spot box (at the isocentre plane) scaled to the tile's depth
// range by the divergence factors: the box every spot's axis crosses the
// tile in.
__device__ __forceinline__ void layer_box(const PbLayer &L, const TileBounds &tb, float &pxl,
                                          float &pxh, float &pyl, float &pyh)
{
    const float a0 = L.sx0 * tb.gx0, a1 = L.sx0 * tb.gx1, a2 = L.sx1 * tb.gx0,
                a3 = L.sx1 * tb.gx1;
    const float b0 = L.sy0 * tb.gy0, b1 = L.sy0 * tb.gy1, b2 = L.sy1 * tb.gy0,
                b3 = L.sy1 * tb.gy1;
    pxl = fminf(fminf(a0, a1), fminf(a2, a3));
    pxh = fmaxf(fmaxf(a0, a1), fmaxf(a2, a3));
    pyl = fminf(fminf(b0, b1), fminf(b2, b3));
    pyh = fmaxf(fmaxf(b0, b1), fmaxf(b2, b3));
}

// A lower bound of 1/|t|^2 over the layer's spots (it2) and an upper bound
// of the widest Gaussian's sigma^2 at the tile (sig2): sigma in air over
// the tile's source-distance range plus the LUT's largest |sigma_mcs|, and
// the halo sigma over the tile's active depths (or over every depth,
// whichever is smaller).  False when no bound applies (NaN, empty tile).
__device__ __forceinline__ bool layer_sig2(const PbLayer &L, const TileBounds &tb,
                                           const PbBeam &B, float cut, float &it2, float &sig2)
{
    const float mx = fmaxf(L.sx0 * L.sx0, L.sx1 * L.sx1) / (B.geom.vsadx * B.geom.vsadx);
    const float my = fmaxf(L.sy0 * L.sy0, L.sy1 * L.sy1) / (B.geom.vsady * B.geom.vsady);
    it2 = 0.999f / (1.0f + mx + my);
    const float *cabc = B.dvp_dev + (size_t)B.dvp_len * L.energy_id + 2;
    const float ca = __ldg(cabc), cb = __ldg(cabc + 1), cc = __ldg(cabc + 2);
    const float off = 0.7f * L.r80;
    const float dlo = tb.d0 - cut + off, dhi = tb.d1 - tb.w0 + off;
    if (!(dlo <= dhi)) return false;   // NaN or an empty tile: no decision
    float q = fmaxf(fabsf(fmaf(fmaf(ca, dlo, cb), dlo, cc)),
                    fabsf(fmaf(fmaf(ca, dhi, cb), dhi, cc)));
    if (ca != 0.0f) {
        const float dv = -cb / (2.0f * ca);
        if (dv > dlo && dv < dhi) q = fmaxf(q, fabsf(fmaf(fmaf(ca, dv, cb), dv, cc)));
    }
    const float st = q + L.mcs_max;
    const float shb = fminf(L.sh_max, halo_sigma_bound(L.r80, tb.w0, fminf(tb.w1, cut)));
    sig2 = fmaf(shb, shb, st * st) * 1.01f + 1e-2f;
    return true;
}

__device__ __forceinline__ bool layer_skip(const PbLayer &L, const TileBounds &tb,
                                           const PbBeam &B, float cut)
{
    if (!L.bound_ok) return false;
    float pxl, pxh, pyl, pyh;
    layer_box(L, tb, pxl, pxh, pyl, pyh);
    const float dx = fmaxf(0.0f, fmaxf(tb.x0 - pxh, pxl - tb.x1));
    const float dy = fmaxf(0.0f, fmaxf(tb.y0 - pyh, pyl - tb.y1));
    const float r2 = dx * dx + dy * dy;
    if (!(r2 > 0.0f)) return false;
    float it2, sig2;
    if (!layer_sig2(L, tb, B, cut, it2, sig2)) return false;
    const float e = r2 * it2 * ((0.5f * kLog2e) / sig2);
    return e >= kCullLog2;
}

// Voxels of this block's tile owned by this thread: (li, lj, lk + step*q),
// with 64 * 8/NV threads per 8x8x8 tile.
template <int NV>
__device__ __forceinline__ void tile_voxels(const PlanArgs &A, int tile, int *vi, int *vj,
                                            int *vk, bool *valid, int *vidx)
{
    int t = tile;
    const int tx = t % A.tiles_x;
    t /= A.tiles_x;
    const int ty = t % A.tiles_y;
    const int tz = t / A.tiles_y;
    constexpr int step = 8 / NV;
    const int li = threadIdx.x & 7, lj = (threadIdx.x >> 3) & 7, lk = threadIdx.x >> 6;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        vi[q] = tx * 8 + li;
        vj[q] = ty * 8 + lj;
        vk[q] = tz * 8 + lk + step * q;
        valid[q] = vi[q] < A.g.nx && vj[q] < A.g.ny && vk[q] < A.g.nz;
        vidx[q] = valid[q] ? vi[q] + A.g.nx * (vj[q] + A.g.ny * vk[q]) : 0;
    }
}

// Head-frame position of a voxel and its divergence factors.
__device__ __forceinline__ void voxel_head(const PbGrid &g, const PbBeam &B, int i, int j,
                                           int k, float &X, float &Y, float &Z, float &gx,
                                           float &gy)
{
    float px, py, pz;
    vox_mm(B.geom, g.spacing, i, j, k, px, py, pz);
    image_to_head(B.geom, px, py, pz, X, Y, Z);
    gx = 1.0f - Z / B.geom.vsadx;
    gy = 1.0f - Z / B.geom.vsady;
}

// Distance to the source, which sits at (0, 0, (VSADX+VSADY)/2) in the head
// frame (CudaClasses.cu:17-51 rotated into the nozzle frame).
__device__ __forceinline__ float source_distance(const PbBeam &B, float X, float Y, float Z)
{
    const float dz = __fsub_rn(__fmul_rn(0.5f, __fadd_rn(B.geom.vsadx, B.geom.vsady)), Z);
    return sqrtf(__fmaf_rn(X, X, __fmaf_rn(Y, Y, __fmul_rn(dz, dz))));
}

// Asynchronous 4-byte global-to-shared copies (cp.async), committed and
// waited for in groups.
__device__ __forceinline__ void cp_async4(float *dst, const float *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n"
                 :: "r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_commit()
{
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" :: "n"(N) : "memory");
}

// Starts the copy of energy e's LUT row into shared memory (one commit
// group per thread; the block waits with cp_async_wait and a barrier).
template <int NT>
__device__ __forceinline__ void stage_lut_async(const PbBeam &B, int e, float *s_dep,
                                                float *s_sig, float *s_idd)
{
    const size_t o = (size_t)e * B.lut_len;
    for (int x = threadIdx.x; x < B.lut_len; x += NT) {
        cp_async4(s_dep + x, B.depths_dev + o + x);
        cp_async4(s_sig + x, B.sigmas_dev + o + x);
        cp_async4(s_idd + x, B.idds_dev + o + x);
    }
    cp_async_commit();
}

// ------------------------------------------------------------------ forward


// What dose_tile computes: the dose, the forward's operation counts, or the
// adjoint (gradient with respect to the spot weights).
constexpr int kModeDose = 0, kModeCount = 1, kModeAdjoint = 2, kModeAdjointPos = 3;

// Shared memory of one tile.  The spot list has 8 slots past its end: the
// adjoint reads spots in groups of 8.
template <int NT, int KCULL>
struct DoseShared {
    // LUT rows, double-buffered: the next kept layer's row is copied in
    // while the current layer is processed
    float dep[2][PB_MAX_LUT_LEN], sig[2][PB_MAX_LUT_LEN], idd[2][PB_MAX_LUT_LEN];
    SpotRec spot[NT * KCULL + 8];
    float gsum[NT * KCULL + 8];   // adjoint: per-slot gradient partials
    float red[NT / 32][kRedSlots];
    int wcount[KCULL][NT / 32];
    int wcount_h[KCULL][NT / 32];
    int lcount[NT / 32];          // layers kept per warp (one chunk of NT layers)
    int lsel[NT];                 // the chunk's kept layers, in order
};

// Sum over the warp of eight per-lane values v[0..7] (one per spot) with a
// transposed butterfly (9 shuffles): on return, the lanes whose two lowest
// bits are 0 hold the total of spot `slot` (each of the 8 spots once).
__device__ __forceinline__ float warp_sum8(float (&v)[8], int lane, int &slot)
{
    const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float send = h16 ? v[i] : v[i + 4], keep = h16 ? v[i + 4] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const float send = h8 ? v[i] : v[i + 2], keep = h8 ? v[i + 2] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
    const float send = h4 ? v[0] : v[1], keep = h4 ? v[1] : v[0];
    float t = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    t += __shfl_xor_sync(0xffffffffu, t, 2);
    t += __shfl_xor_sync(0xffffffffu, t, 1);
    slot = (h16 ? 4 : 0) + (h8 ? 2 : 0) + (h4 ? 1 : 0);
    return t;
}

// Sum over the warp of N per-lane values v[0..N-1] (N = 1, 2, 4 or 8; one
// per spot): log2 N transposed butterfly levels, each halving the values a
// lane holds, then plain levels down to offset 1.  On return the lanes whose
// low log2(32 / N) bits are 0 hold the total of spot `slot`.
template <int N>
__device__ __forceinline__ float warp_sum_n(float (&v)[N], int lane, int &slot)
{
    static_assert(N == 1 || N == 2 || N == 4 || N == 8, "1, 2, 4 or 8 values");
    slot = 0;
#pragma unroll
    for (int h = N / 2, off = 16; h >= 1; h /= 2, off /= 2) {
        const bool up = lane & off;
#pragma unroll
        for (int i = 0; i < h; ++i) {
            const float send = up ? v[i] : v[i + h], keep = up ? v[i + h] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, off);
        }
        slot = 2 * slot + (up ? 1 : 0);
    }
    float t = v[0];
#pragma unroll
    for (int off = 16 / N; off >= 1; off /= 2) t += __shfl_xor_sync(0xffffffffu, t, off);
    return t;
}

// Spot-position derivatives of the adjoint sums.  With q = |t x ray|^2 *
// it2 the scaled squared axis distance (axis_r2), the spot's factor at a
// voxel is mu (Pf 2^(ps2 q) + Hf 2^(hs2 q)), so
//   d/dxs = mu ln2 (Pf ps2 e1 + Hf hs2 e2) dq/dxs,
// and from ax = X - xs gx, ay = Y - ys gy, cz = (xs/VSADX) Y - (ys/VSADY) X
// - xs ys k (k = 1/VSADX - 1/VSADY), it2 = 1/(1 + xs^2/VSADX^2 + ys^2/VSADY^2):
//   dq/dxs = 2 it2 (-ax gx + cz (Y/VSADX - ys k) - q xs/VSADX^2)
//   dq/dys = 2 it2 (-ay gy + cz (-X/VSADY - xs k) - q ys/VSADY^2).
// The voxel sums of wv (Pf ps2 e1 + Hf hs2 e2) ln2 times the bracket meet as
// in the weight adjoint; the spot's factor mu * 2 * it2 is applied when they
// go to grad_x, grad_y.  The weight gradient is formed alongside (grad may
// be NULL).
template <int NT, int NP, int KCAP>
__device__ __forceinline__ void adjoint_positions(const SpotRec *s_spot, float *gsum,
                                                  float *gsum_x, float *gsum_y, int n2, int n1,
                                                  const PbBeam &B, const float2 *XP,
                                                  const float2 *YP, const float2 *GXP,
                                                  const float2 *GYP, const float2 *PS,
                                                  const float2 *HS, const float2 *FP,
                                                  const float2 *FH, const float2 *FPd,
                                                  const float2 *FHd, int lane,
                                                  const float *__restrict__ mu,
                                                  float *__restrict__ grad,
                                                  float *__restrict__ grad_x,
                                                  float *__restrict__ grad_y)
{
    const float ivx = __fdiv_rn(1.0f, B.geom.vsadx), ivy = __fdiv_rn(1.0f, B.geom.vsady);
    const float kap = __fsub_rn(ivx, ivy);
    const float ivx2 = __fmul_rn(ivx, ivx), ivy2 = __fmul_rn(ivy, ivy);
    for (int cls = 0; cls < 2; ++cls) {
        const int lo = cls == 0 ? 0 : KCAP - n1, hi = cls == 0 ? n2 : KCAP;
        for (int c0 = lo; c0 < hi; c0 += 8) {
            float v[8], vx[8], vy[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const SpotRec r = s_spot[c0 + k];
                const float xs = -r.a.x, ys = -r.a.z;
                const float2 kx2 = f2(-__fmul_rn(xs, ivx2)), ky2 = f2(-__fmul_rn(ys, ivy2));
                const float2 ckx = f2(-__fmul_rn(ys, kap)), cky = f2(-__fmul_rn(xs, kap));
                float2 t = make_float2(0.0f, 0.0f), ux = t, uy = t;
#pragma unroll
                for (int p = 0; p < NP; ++p) {
                    const float2 ax = __ffma2_rn(lo2(r.a), GXP[p], XP[p]);
                    const float2 ay = __ffma2_rn(hi2(r.a), GYP[p], YP[p]);
                    const float2 cz = __ffma2_rn(lo2(r.b), YP[p], __ffma2_rn(hi2(r.b), XP[p],
                                                                            lo2(r.c)));
                    const float2 S = __ffma2_rn(ax, ax, __ffma2_rn(ay, ay, __fmul2_rn(cz, cz)));
                    const float2 qq = __fmul2_rn(S, hi2(r.c));
                    const float2 e2 = ex2x2(__fmul2_rn(HS[p], qq));
                    t = __ffma2_rn(FH[p], e2, t);
                    float2 u = __fmul2_rn(FHd[p], e2);
                    if (cls == 0) {
                        const float2 e1 = ex2x2(__fmul2_rn(PS[p], qq));
                        t = __ffma2_rn(FP[p], e1, t);
                        u = __ffma2_rn(FPd[p], e1, u);
                    }
                    float2 bx = __ffma2_rn(cz, __ffma2_rn(YP[p], f2(ivx), ckx),
                                           __fmul2_rn(ax, __fmul2_rn(GXP[p], f2(-1.0f))));
                    bx = __ffma2_rn(qq, kx2, bx);
                    float2 by = __ffma2_rn(cz, __ffma2_rn(XP[p], f2(-ivy), cky),
                                           __fmul2_rn(ay, __fmul2_rn(GYP[p], f2(-1.0f))));
                    by = __ffma2_rn(qq, ky2, by);
                    ux = __ffma2_rn(u, bx, ux);
                    uy = __ffma2_rn(u, by, uy);
                }
                v[k] = t.x + t.y;
                vx[k] = ux.x + ux.y;
                vy[k] = uy.x + uy.y;
            }
            int slot;
            const float sum = warp_sum8(v, lane, slot);
            const float sx = warp_sum8(vx, lane, slot);
            const float sy = warp_sum8(vy, lane, slot);
            if ((lane & 3) == 0 && c0 + slot < hi) {
                if (sum != 0.0f) atomicAdd(&gsum[c0 + slot], sum);
                if (sx != 0.0f) atomicAdd(&gsum_x[c0 + slot], sx);
                if (sy != 0.0f) atomicAdd(&gsum_y[c0 + slot], sy);
            }
        }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < n2 + n1; c += NT) {
        const int sl = c < n2 ? c : KCAP - n1 + (c - n2);
        const int si = __float_as_int(s_spot[sl].d.x);
        const float f = __fmul_rn(__fmul_rn(2.0f, s_spot[sl].c.z), __ldg(mu + si));
        if (grad && gsum[sl] != 0.0f) atomicAdd(grad + si, gsum[sl]);
        if (gsum_x[sl] != 0.0f) atomicAdd(grad_x + si, __fmul_rn(gsum_x[sl], f));
        if (gsum_y[sl] != 0.0f) atomicAdd(grad_y + si, __fmul_rn(gsum_y[sl], f));
        gsum[sl] = gsum_x[sl] = gsum_y[sl] = 0.0f;
    }
}

// One 8x8x8 tile of one plan by one block of NT threads, VPT = 512 / NT
// voxels per thread; spots are culled KCULL per thread per compaction round.
//   kModeDose     the dose (BEAM_OUT: also each beam's dose)
//   kModeCount    every decision of the forward, but instead of evaluating
//                 the surviving spots, add to count[0] the SFU exponentials
//                 and to count[1] the spot-voxel evaluations the forward
//                 issues (each surviving spot against the tile's 512 voxel
//                 slots); no dose
//   kModeAdjointPos  as kModeAdjoint (grad may be NULL), and also the
//                 derivatives with respect to the spot's position at the
//                 isocentre plane into grad_x, grad_y (see below)
//   kModeAdjoint  grad[spot] += scale * sum over the tile's voxels of
//                 wfield[v] * d dose[v] / d mu[spot], with the voxels where
//                 wfield is 0 inactive.  Each thread evaluates its voxels
//                 against the surviving spots in groups of 8; the per-spot
//                 sums meet across the warp (warp_sum8), across the warps in
//                 shared memory, then go to grad with one global atomic per
//                 spot per (tile, layer).
template <int NT, int VPT, int KCULL, bool BEAM_OUT, int MODE = kModeDose>
__device__ __forceinline__ void dose_tile(const PlanArgs &A, int tile,
                                          const float *__restrict__ wet,
                                          const PbLayer *__restrict__ layers,
                                          const float4 *__restrict__ geo,
                                          const float *__restrict__ mu, float *__restrict__ dose,
                                          float *__restrict__ beam_dose,
                                          DoseShared<NT, KCULL> &sh,
                                          unsigned long long *count = nullptr,
                                          const float *__restrict__ wfield = nullptr,
                                          float *__restrict__ grad = nullptr,
                                          float *__restrict__ grad_x = nullptr,
                                          float *__restrict__ grad_y = nullptr,
                                          float *gsum_xy = nullptr)
{
    constexpr bool POS = MODE == kModeAdjointPos;
    constexpr bool COUNT = MODE == kModeCount;
    constexpr bool ADJ = MODE == kModeAdjoint || POS;
    unsigned long long n_ex2 = 0, n_eval = 0;
    static_assert(NT * VPT == 512, "a block covers one 8x8x8 tile");
    constexpr int kVpt = VPT;
    constexpr int kThreads = NT;
    constexpr int kCull = KCULL;
    constexpr int NP = kVpt / 2;  // voxel pairs per thread
    constexpr int kWarps = kThreads / 32;
    SpotRec *s_spot = sh.spot;
    float (*s_red)[kRedSlots] = sh.red;
    int (*s_wcount)[kWarps] = sh.wcount;
    int (*s_wcount_h)[kWarps] = sh.wcount_h;

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int vidx[kVpt];
    bool valid[kVpt];
    {
        int vi[kVpt], vj[kVpt], vk[kVpt];
        tile_voxels<kVpt>(A, tile, vi, vj, vk, valid, vidx);
    }
    const int64_t V = (int64_t)A.g.nx * A.g.ny * A.g.nz;

    float tot_s[kVpt], tot_c[kVpt];
#pragma unroll
    for (int q = 0; q < kVpt; ++q) tot_s[q] = tot_c[q] = 0.0f;
    float wv[kVpt];   // adjoint: scale * dObj/dD per voxel
    if constexpr (ADJ) {
        bool anyw = false;
#pragma unroll
        for (int q = 0; q < kVpt; ++q) {
            wv[q] = valid[q] ? __ldg(wfield + vidx[q]) * A.scale : 0.0f;
            anyw |= (wv[q] != 0.0f);
        }
        if (!__syncthreads_or(anyw)) return;
        for (int c = threadIdx.x; c < kCull * kThreads + 8; c += kThreads) sh.gsum[c] = 0.0f;
        if constexpr (POS)
            for (int c = threadIdx.x; c < 2 * (kCull * kThreads + 8); c += kThreads)
                gsum_xy[c] = 0.0f;
    }
    if constexpr (COUNT) {
        // counting for the adjoint: the tiles it skips are skipped here too
        if (wfield != nullptr) {
            bool anyw = false;
#pragma unroll
            for (int q = 0; q < kVpt; ++q)
                anyw |= valid[q] && __ldg(wfield + vidx[q]) * A.scale != 0.0f;
            if (!__syncthreads_or(anyw)) return;
        }
    }

    for (int b = 0; b < A.n_beams; ++b) {
        const PbBeam &B = A.beams[b];
        // voxel geometry of this beam, kept only as packed voxel pairs
        float2 XP[NP], YP[NP], GXP[NP], GYP[NP], WP[NP];
        TileBounds tb;
        {
            float X[kVpt], Y[kVpt], GX[kVpt], GY[kVpt], W[kVpt], D[kVpt];
#pragma unroll
            for (int q = 0; q < kVpt; ++q) {
                if (valid[q]) {
                    const int i = vidx[q] % A.g.nx, jk = vidx[q] / A.g.nx;
                    float Z;
                    voxel_head(A.g, B, i, jk % A.g.ny, jk / A.g.ny, X[q], Y[q], Z, GX[q], GY[q]);
                    W[q] = __fmul_rn(__ldg(wet + b * V + vidx[q]), 10.0f);
                    D[q] = source_distance(B, X[q], Y[q], B.geom.vsadx * (1.0f - GX[q]));
                } else {
                    X[q] = Y[q] = 0.0f;
                    GX[q] = GY[q] = 1.0f;
                    W[q] = INFINITY;
                    D[q] = 0.0f;
                }
            }
            // the least depth only over voxels that can be active
            float Wa[kVpt];
#pragma unroll
            for (int q = 0; q < kVpt; ++q) Wa[q] = (ADJ && wv[q] == 0.0f) ? INFINITY : W[q];
            tb = tile_bounds<kVpt, kThreads>(X, Y, GX, GY, D, Wa, valid, s_red);
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                XP[p] = make_float2(X[2 * p], X[2 * p + 1]);
                YP[p] = make_float2(Y[2 * p], Y[2 * p + 1]);
                GXP[p] = make_float2(GX[2 * p], GX[2 * p + 1]);
                GYP[p] = make_float2(GY[2 * p], GY[2 * p + 1]);
                WP[p] = make_float2(W[2 * p], W[2 * p + 1]);
            }
        }
        float bs_s[kVpt], bs_c[kVpt];
#pragma unroll
        for (int q = 0; q < kVpt; ++q) bs_s[q] = bs_c[q] = 0.0f;

        // The layers that can reach the tile, found in parallel (one thread
        // per layer, NT layers per chunk): some voxel that can be active
        // lies within the range cut (the tile's least depth), and the
        // layer's bounds do not rule out every spot (layer_skip).
        for (int l0 = 0; l0 < B.n_layers; l0 += kThreads) {
            __syncthreads();   // the previous chunk's list has been read
            bool keep = false;
            {
                const int l = l0 + threadIdx.x;
                if (l < B.n_layers) {
                    const PbLayer L = layers[B.layer_start + l];
                    const float cut = __fmul_rn(1.1f, L.r80);
                    keep = tb.w0 <= cut && !layer_skip(L, tb, B, cut);
                }
            }
            const unsigned lm = __ballot_sync(0xffffffffu, keep);
            if (lane == 0) sh.lcount[warp] = __popc(lm);
            __syncthreads();
            int nsel = 0, lpos = 0;
            for (int w = 0; w < kWarps; ++w) {
                if (w == warp) lpos = nsel + __popc(lm & ((1u << lane) - 1u));
                nsel += sh.lcount[w];
            }
            if (keep) sh.lsel[lpos] = l0 + threadIdx.x;
            __syncthreads();
            if (nsel > 0)
                stage_lut_async<kThreads>(B, layers[B.layer_start + sh.lsel[0]].energy_id,
                                          sh.dep[0], sh.sig[0], sh.idd[0]);
            for (int li = 0; li < nsel; ++li) {
                const int l = sh.lsel[li];
                const PbLayer L = layers[B.layer_start + l];
                const float cut = __fmul_rn(1.1f, L.r80);
                bool act[kVpt];
#pragma unroll
                for (int q = 0; q < kVpt; ++q) {
                    const float w = (q & 1) ? WP[q >> 1].y : WP[q >> 1].x;
                    act[q] = valid[q] && !(w > cut);
                    if constexpr (ADJ) act[q] = act[q] && wv[q] != 0.0f;
                }
                // the next kept layer's LUT row into the other buffer; then
                // wait for this layer's
                const int buf = li & 1;
                if (li + 1 < nsel) {
                    stage_lut_async<kThreads>(
                        B, layers[B.layer_start + sh.lsel[li + 1]].energy_id, sh.dep[buf ^ 1],
                        sh.sig[buf ^ 1], sh.idd[buf ^ 1]);
                    cp_async_wait<1>();
                } else {
                    cp_async_wait<0>();
                }
                __syncthreads();
                const float *s_dep = sh.dep[buf], *s_sig = sh.sig[buf], *s_idd = sh.idd[buf];
                const LayerK K = layer_consts(
                    L.r80, B.dvp_dev + (size_t)B.dvp_len * L.energy_id + 2, s_dep, B.lut_len);
                float pf[kVpt], hf[kVpt];
                float2 PS[NP], HS[NP];
                float hmax = -INFINITY, pmax = -INFINITY;
                // every voxel's parameters without branching, so that the four
                // voxels' dependent chains overlap; inactive voxels take a
                // harmless depth and are masked out afterwards
#pragma unroll
                for (int q = 0; q < kVpt; ++q) {
                    float ps2, hs2;
                    {
                        const int p = q >> 1;
                        const float X = (q & 1) ? XP[p].y : XP[p].x;
                        const float Y = (q & 1) ? YP[p].y : YP[p].x;
                        const float gx = (q & 1) ? GXP[p].y : GXP[p].x;
                        const float w = act[q] ? ((q & 1) ? WP[p].y : WP[p].x) : 0.0f;
                        const float Z = B.geom.vsadx * (1.0f - gx);
                        layer_params(w, source_distance(B, X, Y, Z), K, s_dep, s_sig, s_idd,
                                     B.lut_len, pf[q], hf[q], ps2, hs2);
                    }
                    if (act[q]) {
                        hmax = fmaxf(hmax, hs2);
                        pmax = fmaxf(pmax, ps2);
                    } else {
                        pf[q] = hf[q] = ps2 = hs2 = 0.0f;
                    }
                    if (q & 1) {
                        PS[q >> 1].y = ps2;
                        HS[q >> 1].y = hs2;
                    } else {
                        PS[q >> 1].x = ps2;
                        HS[q >> 1].x = hs2;
                    }
                }
                float nhs, nps;
                block_max2<kThreads>(hmax, pmax, s_red, nhs, nps);
                nhs = -nhs;
                nps = -nps;
                // adjoint: the voxels' weighted prefactors as packed pairs;
                // for positions also times d(exponent)/dq = ln2 * ps2 (hs2)
                float2 FP[NP], FH[NP], FPd[NP], FHd[NP];
                if constexpr (ADJ) {
#pragma unroll
                    for (int p = 0; p < NP; ++p) {
                        FP[p] = make_float2(wv[2 * p] * pf[2 * p], wv[2 * p + 1] * pf[2 * p + 1]);
                        FH[p] = make_float2(wv[2 * p] * hf[2 * p], wv[2 * p + 1] * hf[2 * p + 1]);
                        if constexpr (POS) {
                            constexpr float kLn2 = 0.6931471805599453f;
                            FPd[p] = __fmul2_rn(__fmul2_rn(FP[p], PS[p]), f2(kLn2));
                            FHd[p] = __fmul2_rn(__fmul2_rn(FH[p], HS[p]), f2(kLn2));
                        }
                    }
                }
                float2 AP[NP], AH[NP];
#pragma unroll
                for (int p = 0; p < NP; ++p) AP[p] = AH[p] = make_float2(0.0f, 0.0f);

                // Spots with both terms are compacted to the front of s_spot,
                // halo-only spots to the back.
                constexpr int kCap = kThreads * kCull;
                const int s0 = B.spot_start + L.spot_start;
                for (int base = 0; base < L.n_spots; base += kCap) {
                    int cls[kCull];
                    float4 ga[kCull], gb[kCull];
                    unsigned m2[kCull], m1[kCull];
#pragma unroll
                    for (int c = 0; c < kCull; ++c) {
                        const int si = base + c * kThreads + threadIdx.x;
                        cls[c] = 0;
                        if (si < L.n_spots) {
                            ga[c] = __ldg(geo + 2 * (int64_t)(s0 + si));
                            cls[c] = cull_class(cull_r2(ga[c].x, ga[c].y, ga[c].z, tb), nhs, nps);
                            // the record's second half only for the kept spots
                            if (cls[c]) gb[c] = __ldg(geo + 2 * (int64_t)(s0 + si) + 1);
                        }
                        m2[c] = __ballot_sync(0xffffffffu, cls[c] == 2);
                        m1[c] = __ballot_sync(0xffffffffu, cls[c] == 1);
                        if (lane == 0) {
                            s_wcount[c][warp] = __popc(m2[c]);
                            s_wcount_h[c][warp] = __popc(m1[c]);
                        }
                    }
                    __syncthreads();
                    int n2 = 0, n1 = 0;
                    const unsigned below = (1u << lane) - 1u;
#pragma unroll
                    for (int c = 0; c < kCull; ++c) {
                        int pos2 = 0, pos1 = 0;
                        for (int w = 0; w < kWarps; ++w) {
                            if (w == warp) {
                                pos2 = n2 + __popc(m2[c] & below);
                                pos1 = n1 + __popc(m1[c] & below);
                            }
                            n2 += s_wcount[c][w];
                            n1 += s_wcount_h[c][w];
                        }
                        if (cls[c]) {
                            // the adjoint keeps the spot's index where the dose keeps its weight
                            const int si = s0 + base + c * kThreads + threadIdx.x;
                            const float w =
                                MODE == kModeDose ? __ldg(mu + si) : __int_as_float(si);
                            SpotRec r;
                            r.a = make_float4(-ga[c].x, -ga[c].x, -ga[c].y, -ga[c].y);
                            r.b = make_float4(ga[c].w, ga[c].w, -gb[c].x, -gb[c].x);
                            r.c = make_float4(-gb[c].y, -gb[c].y, ga[c].z, ga[c].z);
                            r.d = make_float4(w, w, 0.0f, 0.0f);
                            s_spot[cls[c] == 2 ? pos2 : kCap - 1 - pos1] = r;
                        }
                    }
                    __syncthreads();
                    if constexpr (COUNT) {
                        n_ex2 += 512ull * (unsigned long long)(2 * n2 + n1);
                        n_eval += 512ull * (unsigned long long)(n2 + n1);
                    } else if constexpr (POS) {
                        adjoint_positions<kThreads, NP, kCap>(
                            s_spot, sh.gsum, gsum_xy, gsum_xy + kCap + 8, n2, n1, B, XP, YP,
                            GXP, GYP, PS, HS, FP, FH, FPd, FHd, lane, mu, grad, grad_x, grad_y);
                    } else if constexpr (ADJ) {
                        // both terms: slots [0, n2); halo only: [kCap - n1, kCap);
                        // a group's slots past its class hold other records or
                        // padding, and their sums are dropped
                        for (int c0 = 0; c0 < n2; c0 += 8) {
                            float v[8];
#pragma unroll
                            for (int k = 0; k < 8; ++k) {
                                const SpotRec r = s_spot[c0 + k];
                                float2 t = make_float2(0.0f, 0.0f);
#pragma unroll
                                for (int p = 0; p < NP; ++p) {
                                    const float2 qq =
                                        axis_r2(lo2(r.a), hi2(r.a), lo2(r.b), hi2(r.b), lo2(r.c),
                                                hi2(r.c), XP[p], YP[p], GXP[p], GYP[p]);
                                    t = __ffma2_rn(FP[p], ex2x2(__fmul2_rn(PS[p], qq)), t);
                                    t = __ffma2_rn(FH[p], ex2x2(__fmul2_rn(HS[p], qq)), t);
                                }
                                v[k] = t.x + t.y;
                            }
                            int slot;
                            const float sum = warp_sum8(v, lane, slot);
                            if ((lane & 3) == 0 && c0 + slot < n2 && sum != 0.0f)
                                atomicAdd(&sh.gsum[c0 + slot], sum);
                        }
                        for (int c0 = kCap - n1; c0 < kCap; c0 += 8) {
                            float v[8];
#pragma unroll
                            for (int k = 0; k < 8; ++k) {
                                const SpotRec r = s_spot[c0 + k];
                                float2 t = make_float2(0.0f, 0.0f);
#pragma unroll
                                for (int p = 0; p < NP; ++p) {
                                    const float2 qq =
                                        axis_r2(lo2(r.a), hi2(r.a), lo2(r.b), hi2(r.b), lo2(r.c),
                                                hi2(r.c), XP[p], YP[p], GXP[p], GYP[p]);
                                    t = __ffma2_rn(FH[p], ex2x2(__fmul2_rn(HS[p], qq)), t);
                                }
                                v[k] = t.x + t.y;
                            }
                            int slot;
                            const float sum = warp_sum8(v, lane, slot);
                            if ((lane & 3) == 0 && c0 + slot < kCap && sum != 0.0f)
                                atomicAdd(&sh.gsum[c0 + slot], sum);
                        }
                        __syncthreads();
                        // each surviving spot's tile sum to its gradient
                        for (int c = threadIdx.x; c < n2 + n1; c += kThreads) {
                            const int sl = c < n2 ? c : kCap - n1 + (c - n2);
                            const float a = sh.gsum[sl];
                            if (a != 0.0f) atomicAdd(grad + __float_as_int(s_spot[sl].d.x), a);
                            sh.gsum[sl] = 0.0f;
                        }
                    } else {
                        // unrolled by 8: more independent exp2 chains in
                        // flight (measured: 8.57 -> 8.29 ms against 2)
#pragma unroll 8
                        for (int c = 0; c < n2; ++c) {
                            const SpotRec r = s_spot[c];
                            const float2 nx = lo2(r.a), ny = hi2(r.a), tx = lo2(r.b);
                            const float2 nty = hi2(r.b), ncs = lo2(r.c), it2 = hi2(r.c);
                            const float2 w = lo2(r.d);
#pragma unroll
                            for (int p = 0; p < NP; ++p) {
                                const float2 qq = axis_r2(nx, ny, tx, nty, ncs, it2, XP[p], YP[p],
                                                          GXP[p], GYP[p]);
                                AP[p] = __ffma2_rn(w, ex2x2(__fmul2_rn(PS[p], qq)), AP[p]);
                                AH[p] = __ffma2_rn(w, ex2x2(__fmul2_rn(HS[p], qq)), AH[p]);
                            }
                        }
#pragma unroll 8
                        for (int c = kCap - n1; c < kCap; ++c) {
                            const SpotRec r = s_spot[c];
                            const float2 nx = lo2(r.a), ny = hi2(r.a), tx = lo2(r.b);
                            const float2 nty = hi2(r.b), ncs = lo2(r.c), it2 = hi2(r.c);
                            const float2 w = lo2(r.d);
#pragma unroll
                            for (int p = 0; p < NP; ++p) {
                                const float2 qq = axis_r2(nx, ny, tx, nty, ncs, it2, XP[p], YP[p],
                                                          GXP[p], GYP[p]);
                                AH[p] = __ffma2_rn(w, ex2x2(__fmul2_rn(HS[p], qq)), AH[p]);
                            }
                        }
                    }
                    __syncthreads();
                }
                if constexpr (!ADJ) {
#pragma unroll
                    for (int q = 0; q < kVpt; ++q) {
                        if (act[q]) {
                            const float ap = (q & 1) ? AP[q >> 1].y : AP[q >> 1].x;
                            const float ah = (q & 1) ? AH[q >> 1].y : AH[q >> 1].x;
                            const float ld = fmaf(pf[q], ap, hf[q] * ah);
                            if (BEAM_OUT) neumaier(bs_s[q], bs_c[q], ld);
                            neumaier(tot_s[q], tot_c[q], ld);
                        }
                    }
                }
            }
        }
        if (BEAM_OUT) {
#pragma unroll
            for (int q = 0; q < kVpt; ++q)
                if (valid[q]) beam_dose[b * V + vidx[q]] = (bs_s[q] + bs_c[q]) * A.scale;
        }
        __syncthreads();  // s_red is rewritten by the next beam's tile_bounds
    }
    if constexpr (COUNT) {
        if (threadIdx.x == 0) {
            atomicAdd(count, n_ex2);
            atomicAdd(count + 1, n_eval);
        }
    } else if constexpr (!ADJ) {
#pragma unroll
        for (int q = 0; q < kVpt; ++q)
            if (valid[q]) dose[vidx[q]] = (tot_s[q] + tot_c[q]) * A.scale;
    }
}

// ------------------------------------------------------------ line tiles
//
// The forward, its operation count and the spot-weight adjoint also exist
// on tiles of 8 x TY x TZ voxels, one block of TY*TZ threads per tile, each
// thread owning one line of kLine = 8 voxels along x.  Along a line the
// voxels' head-frame coordinates, and the divergence factors, are affine in
// the voxel's offset q' = q - 3.5 from the line's centre, so the three
// components of t x ray (axis_r2) are affine in q' and the scaled squared
// axis distance of a spot is a quadratic
//     it2 |t x ray|^2 = S0 + B1 q' + C2 q'^2 .
// Per spot the block's compaction stores the spot's line-independent part
// (C2 and 2 it2 times the per-voxel step of each component, from the
// beam's constant step along x); each thread then forms S0 and B1 for its
// own line from the components at the line's centre (11 operations) and
// evaluates every voxel with two fused multiply-adds.  The per-voxel work
// is the exponent (one multiply), the SFU's ex2 and the accumulation, so
// the spot loops are bound by the SFU's exp2 rate rather than shared with
// the FMA pipe.  The LUT rows are read through the read-only data cache
// (no staging barrier).  Decisions (layer selection, the per-layer range
// cut, the spot cull) are those of the 8^3 tiles above.
//
// Shapes (template TY, TZ, KCULL): tiles of 8x8x8 (64 threads), 8x8x4 and
// 8x4x8 (32 threads), 8x16x8 and 8x8x16 (128 threads); KCULL spots culled
// per thread per compaction round.  Shapes that differ in tile or round size
// cull differently, or add a layer's spots in another order, and agree to
// rounding.

constexpr int kLine = 8;

// Line-tile record of one surviving spot: (-x, -y, x/VSADX, -y/VSADY),
// (-x y (1/VSADX - 1/VSADY), it2, C2, weight or index), and 2 it2 times the
// step of each component of t x ray per voxel along x (the last float unused).
struct LineSpot {
    float4 a, b, c;
};

// Per-voxel state that changes once per layer lives here rather than in
// registers (thread t's voxel q at [q][t]), so that the spot loops keep
// only their own values live.
template <int NT, int KCULL, bool BEAM_OUT = false, bool DOSE = true>
struct LineShared {
    static constexpr int kWarps = NT / 32;
    LineSpot spot[NT * KCULL + 8];
    float gsum[NT * KCULL + 8];      // adjoint: per-slot gradient partials
    float w[kLine][NT];              // the beam's 10*WET per voxel (INF: not valid)
    float d[kLine][NT];              // distance to the source per voxel
    float tot[2][kLine][DOSE ? NT : 1];   // dose: compensated sum over layers and beams
    float pfh[2][kLine][DOSE ? NT : 1];   // dose: the layer's prefactors Pf, Hf
    float bsum[BEAM_OUT ? 2 : 1][kLine][BEAM_OUT ? NT : 1];   // each beam's own sum
    float red[kWarps][kRedSlots];
    int wcount[KCULL][kWarps];
    int wcount_h[KCULL][kWarps];
    int lcount[kWarps];
    int lsel[NT];
};

// Offsets q - 3.5 of a line's voxel pair (2p, 2p + 1) from the line's centre
// (exact in FP32).
__device__ __forceinline__ float2 line_off2(int p)
{
    return make_float2((float)(2 * p) - 3.5f, (float)(2 * p) - 2.5f);
}

// Offset q - 3.5 of a line's voxel from the line's centre (exact in FP32).
__device__ __forceinline__ constexpr float line_off(int q) { return (float)q - 3.5f; }

// Per-thread part of a spot's quadratic on this thread's line: S0 and B1
// from the spot's axis components at the line's centre.
__device__ __forceinline__ void line_spot(const LineSpot &r, float Xc, float Yc, float gxc,
                                          float gyc, float &S0, float &B1)
{
    const float ax = __fmaf_rn(r.a.x, gxc, Xc);
    const float ay = __fmaf_rn(r.a.y, gyc, Yc);
    const float az = __fmaf_rn(r.a.z, Yc, __fmaf_rn(r.a.w, Xc, r.b.x));
    S0 = __fmul_rn(r.b.y, __fmaf_rn(ax, ax, __fmaf_rn(ay, ay, __fmul_rn(az, az))));
    B1 = __fmaf_rn(ax, r.c.x, __fmaf_rn(ay, r.c.y, __fmul_rn(az, r.c.z)));
}

template <int TY, int TZ, int KCULL, bool BEAM_OUT, int MODE = kModeDose>
__device__ __forceinline__ void line_tile(const PlanArgs &A, int tx, int ty, int tz,
                                          const float *__restrict__ wet,
                                          const PbLayer *__restrict__ layers,
                                          const float4 *__restrict__ geo,
                                          const float *__restrict__ mu,
                                          float *__restrict__ dose,
                                          float *__restrict__ beam_dose,
                                          LineShared<TY * TZ, KCULL, BEAM_OUT,
                                                     MODE == kModeDose> &sh,
                                          unsigned long long *count = nullptr,
                                          const float *__restrict__ wfield = nullptr,
                                          float *__restrict__ grad = nullptr)
{
    constexpr int NT = TY * TZ;
    constexpr int kWarps = NT / 32;
    constexpr bool COUNT = MODE == kModeCount;
    constexpr bool ADJ = MODE == kModeAdjoint;
    static_assert(NT % 32 == 0, "whole warps");
    static_assert(MODE == kModeDose || MODE == kModeCount || MODE == kModeAdjoint,
                  "line tiles: dose, count or weight adjoint");
    constexpr int kCap = NT * KCULL;
    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;

    // this thread's line: voxels (i0 + q, j, k), q < nvalid
    const int i0 = tx * kLine, j = ty * TY + t % TY, k = tz * TZ + t / TY;
    const int nvalid = (j < A.g.ny && k < A.g.nz) ? min(kLine, A.g.nx - i0) : 0;
    const int64_t vbase = i0 + (int64_t)A.g.nx * (j + (int64_t)A.g.ny * k);
    const int64_t V = (int64_t)A.g.nx * A.g.ny * A.g.nz;
    unsigned long long n_ex2 = 0, n_eval = 0;

    if constexpr (MODE == kModeDose) {
#pragma unroll
        for (int q = 0; q < kLine; ++q) sh.tot[0][q][t] = sh.tot[1][q][t] = 0.0f;
    }
    float wv[kLine];   // adjoint: scale * dObj/dD per voxel
    if constexpr (ADJ) {
        bool anyw = false;
#pragma unroll
        for (int q = 0; q < kLine; ++q) {
            wv[q] = q < nvalid ? __ldg(wfield + vbase + q) * A.scale : 0.0f;
            anyw |= (wv[q] != 0.0f);
        }
        if (!__syncthreads_or(anyw)) return;
        for (int c = t; c < kCap + 8; c += NT) sh.gsum[c] = 0.0f;
    }
    if constexpr (COUNT) {
        // counting for the adjoint: the tiles it skips are skipped here too
        if (wfield != nullptr) {
            bool anyw = false;
#pragma unroll
            for (int q = 0; q < kLine; ++q)
                anyw |= q < nvalid && __ldg(wfield + vbase + q) * A.scale != 0.0f;
            if (!__syncthreads_or(anyw)) return;
        }
    }

    for (int b = 0; b < A.n_beams; ++b) {
        const PbBeam &B = A.beams[b];
        // line geometry: head-frame centre and step per voxel along x
        float dX, dY, dZ;
        image_to_head(B.geom, A.g.spacing, 0.0f, 0.0f, dX, dY, dZ);
        const float dgx = -__fdiv_rn(dZ, B.geom.vsadx), dgy = -__fdiv_rn(dZ, B.geom.vsady);
        float Xc, Yc, Zc;
        {
            float px, py, pz, X0, Y0, Z0;
            vox_mm(B.geom, A.g.spacing, i0, j, k, px, py, pz);
            image_to_head(B.geom, px, py, pz, X0, Y0, Z0);
            Xc = __fmaf_rn(3.5f, dX, X0);
            Yc = __fmaf_rn(3.5f, dY, Y0);
            Zc = __fmaf_rn(3.5f, dZ, Z0);
        }
        const float gxc = __fsub_rn(1.0f, __fdiv_rn(Zc, B.geom.vsadx));
        const float gyc = __fsub_rn(1.0f, __fdiv_rn(Zc, B.geom.vsady));
        TileBounds tb;
        {
            // the beam's depth and source distance per voxel into shared
            // memory; the tile's box over its valid voxels
            float v[12] = {INFINITY, -INFINITY, INFINITY, -INFINITY, INFINITY, -INFINITY,
                           INFINITY, -INFINITY, INFINITY, -INFINITY, INFINITY, -INFINITY};
#pragma unroll
            for (int q = 0; q < kLine; ++q) {
                const float o = line_off(q);
                float w = INFINITY, dd = 0.0f;
                if (q < nvalid) {
                    const float X = __fmaf_rn(o, dX, Xc), Y = __fmaf_rn(o, dY, Yc);
                    const float Z = __fmaf_rn(o, dZ, Zc);
                    w = __fmul_rn(__ldg(wet + b * V + vbase + q), 10.0f);
                    dd = source_distance(B, X, Y, Z);
                    const float GX = __fmaf_rn(o, dgx, gxc), GY = __fmaf_rn(o, dgy, gyc);
                    v[0] = fminf(v[0], X);  v[1] = fmaxf(v[1], X);
                    v[2] = fminf(v[2], Y);  v[3] = fmaxf(v[3], Y);
                    v[4] = fminf(v[4], GX); v[5] = fmaxf(v[5], GX);
                    v[6] = fminf(v[6], GY); v[7] = fmaxf(v[7], GY);
                    v[8] = fminf(v[8], dd); v[9] = fmaxf(v[9], dd);
                    // the least depth over voxels that can be active; a NaN
                    // depth is never skipped
                    if (!ADJ || wv[q] != 0.0f) {
                        v[10] = fminf(v[10], w == w ? w : -INFINITY);
                        v[11] = fmaxf(v[11], w == w ? w : INFINITY);
                    }
                }
                sh.w[q][t] = w;
                sh.d[q][t] = dd;
            }
#pragma unroll
            for (int m = 0; m < 12; ++m) v[m] = (m & 1) ? warp_max(v[m]) : warp_min(v[m]);
            if (lane == 0) {
#pragma unroll
                for (int m = 0; m < 12; ++m) sh.red[warp][m] = v[m];
            }
            __syncthreads();
            float r[12];
#pragma unroll
            for (int m = 0; m < 12; ++m) r[m] = sh.red[0][m];
            for (int w = 1; w < kWarps; ++w) {
#pragma unroll
                for (int m = 0; m < 12; ++m)
                    r[m] = (m & 1) ? fmaxf(r[m], sh.red[w][m]) : fminf(r[m], sh.red[w][m]);
            }
            tb.x0 = r[0]; tb.x1 = r[1]; tb.y0 = r[2]; tb.y1 = r[3];
            tb.gx0 = r[4]; tb.gx1 = r[5]; tb.gy0 = r[6]; tb.gy1 = r[7];
            tb.d0 = r[8]; tb.d1 = r[9]; tb.w0 = r[10]; tb.w1 = r[11];
        }
        if constexpr (BEAM_OUT) {
#pragma unroll
            for (int q = 0; q < kLine; ++q) sh.bsum[0][q][t] = sh.bsum[1][q][t] = 0.0f;
        }

        for (int l0 = 0; l0 < B.n_layers; l0 += NT) {
            __syncthreads();   // the previous chunk's list and the bounds have been read
            bool keep = false;
            {
                const int l = l0 + t;
                if (l < B.n_layers) {
                    const PbLayer L = layers[B.layer_start + l];
                    const float cut = __fmul_rn(1.1f, L.r80);
                    keep = L.n_spots > 0 && tb.w0 <= cut && !layer_skip(L, tb, B, cut);
                }
            }
            const unsigned lm = __ballot_sync(0xffffffffu, keep);
            if (lane == 0) sh.lcount[warp] = __popc(lm);
            __syncthreads();
            int nsel = 0, lpos = 0;
            for (int w = 0; w < kWarps; ++w) {
                if (w == warp) lpos = nsel + __popc(lm & ((1u << lane) - 1u));
                nsel += sh.lcount[w];
            }
            if (keep) sh.lsel[lpos] = l0 + t;
            __syncthreads();
            for (int li = 0; li < nsel; ++li) {
                // every kept layer has spots, so each runs at least one
                // compaction round, whose barriers separate this layer's
                // block_max2 from the next one's
                const PbLayer L = layers[B.layer_start + sh.lsel[li]];
                const float cut = __fmul_rn(1.1f, L.r80);
                const size_t ro = (size_t)L.energy_id * B.lut_len;
                const RowG dep{B.depths_dev + ro}, sig{B.sigmas_dev + ro}, idd{B.idds_dev + ro};
                const LayerK K =
                    layer_consts(L.r80, B.dvp_dev + (size_t)B.dvp_len * L.energy_id + 2, dep,
                                 B.lut_len);
                float pf[kLine], hf[kLine];
                float2 PS[kLine / 2], HS[kLine / 2];   // voxel pairs (q, q + 1)
                bool act[kLine];
                float hmax = -INFINITY, pmax = -INFINITY;
                // every voxel's parameters without branching (inactive
                // voxels take a harmless depth and are masked afterwards)
#pragma unroll
                for (int q = 0; q < kLine; ++q) {
                    const float w = sh.w[q][t];
                    act[q] = !(w > cut) && q < nvalid;
                    if constexpr (ADJ) act[q] = act[q] && wv[q] != 0.0f;
                    float ps2, hs2;
                    layer_params(act[q] ? w : 0.0f, sh.d[q][t], K, dep, sig, idd, B.lut_len,
                                 pf[q], hf[q], ps2, hs2);
                    if (act[q]) {
                        hmax = fmaxf(hmax, hs2);
                        pmax = fmaxf(pmax, ps2);
                    } else {
                        pf[q] = hf[q] = ps2 = hs2 = 0.0f;
                    }
                    if (q & 1) {
                        PS[q >> 1].y = ps2;
                        HS[q >> 1].y = hs2;
                    } else {
                        PS[q >> 1].x = ps2;
                        HS[q >> 1].x = hs2;
                    }
                    if constexpr (MODE == kModeDose) {
                        sh.pfh[0][q][t] = pf[q];
                        sh.pfh[1][q][t] = hf[q];
                    }
                }
                float nhs, nps;
                block_max2<NT>(hmax, pmax, sh.red, nhs, nps);
                nhs = -nhs;
                nps = -nps;
                // forward: per-voxel sums; adjoint: weighted prefactors
                float2 AP[kLine / 2], AH[kLine / 2];
#pragma unroll
                for (int p = 0; p < kLine / 2; ++p) {
                    if constexpr (ADJ) {
                        AP[p] = make_float2(__fmul_rn(wv[2 * p], pf[2 * p]),
                                            __fmul_rn(wv[2 * p + 1], pf[2 * p + 1]));
                        AH[p] = make_float2(__fmul_rn(wv[2 * p], hf[2 * p]),
                                            __fmul_rn(wv[2 * p + 1], hf[2 * p + 1]));
                    } else {
                        AP[p] = AH[p] = make_float2(0.0f, 0.0f);
                    }
                }

                const int s0 = B.spot_start + L.spot_start;
                for (int base = 0; base < L.n_spots; base += kCap) {
                    int cls[KCULL];
                    float4 ga[KCULL], gb[KCULL];
                    unsigned m2[KCULL], m1[KCULL];
#pragma unroll
                    for (int c = 0; c < KCULL; ++c) {
                        const int si = base + c * NT + t;
                        cls[c] = 0;
                        if (si < L.n_spots) {
                            ga[c] = __ldg(geo + 2 * (int64_t)(s0 + si));
                            cls[c] = cull_class(cull_r2(ga[c].x, ga[c].y, ga[c].z, tb), nhs, nps);
                            if (cls[c]) gb[c] = __ldg(geo + 2 * (int64_t)(s0 + si) + 1);
                        }
                        m2[c] = __ballot_sync(0xffffffffu, cls[c] == 2);
                        m1[c] = __ballot_sync(0xffffffffu, cls[c] == 1);
                        if (lane == 0) {
                            sh.wcount[c][warp] = __popc(m2[c]);
                            sh.wcount_h[c][warp] = __popc(m1[c]);
                        }
                    }
                    __syncthreads();
                    int n2 = 0, n1 = 0;
                    const unsigned below = (1u << lane) - 1u;
#pragma unroll
                    for (int c = 0; c < KCULL; ++c) {
                        int pos2 = 0, pos1 = 0;
                        for (int w = 0; w < kWarps; ++w) {
                            if (w == warp) {
                                pos2 = n2 + __popc(m2[c] & below);
                                pos1 = n1 + __popc(m1[c] & below);
                            }
                            n2 += sh.wcount[c][w];
                            n1 += sh.wcount_h[c][w];
                        }
                        if (cls[c]) {
                            const int si = s0 + base + c * NT + t;
                            // the dose keeps the spot's weight, the adjoint its index
                            const float wgt =
                                MODE == kModeDose ? __ldg(mu + si) : __int_as_float(si);
                            const float nx = -ga[c].x, ny = -ga[c].y, txs = ga[c].w;
                            const float nty = -gb[c].x, it2 = ga[c].z;
                            // the spot's step of each component per voxel along x
                            const float sx = __fmaf_rn(nx, dgx, dX);
                            const float sy = __fmaf_rn(ny, dgy, dY);
                            const float sz = __fmaf_rn(txs, dY, __fmul_rn(nty, dX));
                            const float c2 = __fmul_rn(
                                it2, __fmaf_rn(sx, sx, __fmaf_rn(sy, sy, __fmul_rn(sz, sz))));
                            const float k2 = __fmul_rn(2.0f, it2);
                            LineSpot r;
                            r.a = make_float4(nx, ny, txs, nty);
                            r.b = make_float4(-gb[c].y, it2, c2, wgt);
                            r.c = make_float4(__fmul_rn(k2, sx), __fmul_rn(k2, sy),
                                              __fmul_rn(k2, sz), 0.0f);
                            sh.spot[cls[c] == 2 ? pos2 : kCap - 1 - pos1] = r;
                        }
                    }
                    __syncthreads();
                    if constexpr (COUNT) {
                        n_ex2 += (unsigned long long)(kLine * NT) * (2 * n2 + n1);
                        n_eval += (unsigned long long)(kLine * NT) * (n2 + n1);
                    } else if constexpr (ADJ) {
                        // both terms: slots [0, n2); halo only: [kCap - n1, kCap);
                        // a group's slots past its class hold other records or
                        // padding, and their sums are dropped
                        // (the class is a compile-time constant of each
                        // loop, so neither loop body branches on it)
                        // groups of 8 spots, the rest in groups of 4, 2 and 1,
                        // so that no padding slot is evaluated
                        auto group = [&](auto two, auto n, const int c0) {
                            constexpr int N = decltype(n)::value;
                            float v[N];
#pragma unroll
                            for (int u = 0; u < N; ++u) {
                                const LineSpot r = sh.spot[c0 + u];
                                float S0, B1;
                                line_spot(r, Xc, Yc, gxc, gyc, S0, B1);
                                const float2 s0 = f2(S0), b1 = f2(B1), c2 = f2(r.b.z);
                                float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
                                for (int p = 0; p < kLine / 2; ++p) {
                                    const float2 o = line_off2(p);
                                    const float2 S = __ffma2_rn(__ffma2_rn(c2, o, b1), o, s0);
                                    acc = __ffma2_rn(AH[p], ex2x2(__fmul2_rn(HS[p], S)), acc);
                                    if constexpr (decltype(two)::value)
                                        acc = __ffma2_rn(AP[p], ex2x2(__fmul2_rn(PS[p], S)),
                                                         acc);
                                }
                                v[u] = acc.x + acc.y;
                            }
                            int slot;
                            const float sum = warp_sum_n<N>(v, lane, slot);
                            if ((lane & (32 / N - 1)) == 0 && sum != 0.0f)
                                atomicAdd(&sh.gsum[c0 + slot], sum);
                        };
                        auto groups = [&](auto two, const int lo, const int hi) {
                            int c0 = lo;
                            for (; c0 + 8 <= hi; c0 += 8)
                                group(two, std::integral_constant<int, 8>{}, c0);
                            if (hi - c0 >= 4) {
                                group(two, std::integral_constant<int, 4>{}, c0);
                                c0 += 4;
                            }
                            if (hi - c0 >= 2) {
                                group(two, std::integral_constant<int, 2>{}, c0);
                                c0 += 2;
                            }
                            if (hi - c0 >= 1) group(two, std::integral_constant<int, 1>{}, c0);
                        };
                        groups(std::true_type{}, 0, n2);
                        groups(std::false_type{}, kCap - n1, kCap);
                        __syncthreads();
                        // each surviving spot's tile sum to its gradient
                        for (int c = t; c < n2 + n1; c += NT) {
                            const int sl = c < n2 ? c : kCap - n1 + (c - n2);
                            const float a = sh.gsum[sl];
                            if (a != 0.0f) atomicAdd(grad + __float_as_int(sh.spot[sl].b.w), a);
                            sh.gsum[sl] = 0.0f;
                        }
                    } else {
                        // both terms (unrolled by 4: the per-beam forward
                        // 6.37 against 6.49 ms, the plain one unchanged)
#pragma unroll 4
                        for (int c = 0; c < n2; ++c) {
                            const LineSpot r = sh.spot[c];
                            float S0, B1;
                            line_spot(r, Xc, Yc, gxc, gyc, S0, B1);
                            const float2 s0 = f2(S0), b1 = f2(B1), c2 = f2(r.b.z), w = f2(r.b.w);
#pragma unroll
                            for (int p = 0; p < kLine / 2; ++p) {
                                const float2 o = line_off2(p);
                                const float2 S = __ffma2_rn(__ffma2_rn(c2, o, b1), o, s0);
                                AP[p] = __ffma2_rn(w, ex2x2(__fmul2_rn(PS[p], S)), AP[p]);
                                AH[p] = __ffma2_rn(w, ex2x2(__fmul2_rn(HS[p], S)), AH[p]);
                            }
                        }
                        // halo only (unrolled by 4: 6.04 against 6.12 ms)
#pragma unroll 4
                        for (int c = kCap - n1; c < kCap; ++c) {
                            const LineSpot r = sh.spot[c];
                            float S0, B1;
                            line_spot(r, Xc, Yc, gxc, gyc, S0, B1);
                            const float2 s0 = f2(S0), b1 = f2(B1), c2 = f2(r.b.z), w = f2(r.b.w);
#pragma unroll
                            for (int p = 0; p < kLine / 2; ++p) {
                                const float2 o = line_off2(p);
                                const float2 S = __ffma2_rn(__ffma2_rn(c2, o, b1), o, s0);
                                AH[p] = __ffma2_rn(w, ex2x2(__fmul2_rn(HS[p], S)), AH[p]);
                            }
                        }
                    }
                    __syncthreads();
                }
                if constexpr (MODE == kModeDose) {
#pragma unroll
                    for (int q = 0; q < kLine; ++q) {
                        if (act[q]) {
                            const float ap = (q & 1) ? AP[q >> 1].y : AP[q >> 1].x;
                            const float ah = (q & 1) ? AH[q >> 1].y : AH[q >> 1].x;
                            const float ld = fmaf(sh.pfh[0][q][t], ap, sh.pfh[1][q][t] * ah);
                            if constexpr (BEAM_OUT) {
                                float bs = sh.bsum[0][q][t], bc = sh.bsum[1][q][t];
                                neumaier(bs, bc, ld);
                                sh.bsum[0][q][t] = bs;
                                sh.bsum[1][q][t] = bc;
                            }
                            float ts = sh.tot[0][q][t], tc = sh.tot[1][q][t];
                            neumaier(ts, tc, ld);
                            sh.tot[0][q][t] = ts;
                            sh.tot[1][q][t] = tc;
                        }
                    }
                }
            }
        }
        if (BEAM_OUT) {
#pragma unroll
            for (int q = 0; q < kLine; ++q)
                if (q < nvalid)
                    beam_dose[b * V + vbase + q] = (sh.bsum[0][q][t] + sh.bsum[1][q][t]) * A.scale;
        }
        __syncthreads();  // sh.w, sh.d and sh.red are rewritten by the next beam
    }
    if constexpr (COUNT) {
        if (t == 0) {
            atomicAdd(count, n_ex2);
            atomicAdd(count + 1, n_eval);
        }
    } else if constexpr (MODE == kModeDose) {
#pragma unroll
        for (int q = 0; q < kLine; ++q)
            if (q < nvalid) dose[vbase + q] = (sh.tot[0][q][t] + sh.tot[1][q][t]) * A.scale;
    }
}

// Resident blocks per SM the line-tile kernels are compiled for (their
// register budget): 20 of 32 threads, 10 of 64, 5 of 128.  The kernels with
// more live state per thread (the per-beam forward's extra sums, the
// adjoint's weighted prefactors and spot groups) take 4 of 128 threads (128
// registers): on the 4-beam 256x256x160 plan the adjoint went from 6.65 to
// 6.43 ms and the per-beam forward from 6.78 to 6.47 ms, while the plain
// forward is faster at 5 (6.12 against 6.25 ms).
template <int NT, bool HEAVY = false> constexpr int line_min_blocks()
{
    return NT == 32 ? 20 : (NT == 64 ? 10 : (HEAVY ? 4 : 5));
}

#ifndef PB_TILE_ORDER
#define PB_TILE_ORDER 1
#endif

// The r-th index of 0..n-1 taken outward from c: c, c+1, c-1, c+2, c-2, ...
// and, once one side is used up, the rest of the other side in order.
__device__ __forceinline__ int center_out(int r, int n, int c)
{
    const int m = min(c, n - 1 - c);
    if (r <= 2 * m) {
        const int k = (r + 1) >> 1;
        return (r & 1) ? c + k : c - k;
    }
    const int j = r - 2 * m;
    return c - m == 0 ? c + m + j : c - m - j;
}

// Tile of a linear block index over the grid's 8 x TY x TZ tiles.  Blocks
// start in launch order, so the tiles are handed out from the tile holding
// the plan's centre (the mean isocentre) outward, z slabs first: the tiles
// most beams cross, the longest ones, start early and the launch does not
// end on a few of them while the other SMs idle.
//
// With A.order (pb_tile_order: the tiles by estimated cost, most expensive
// first) block b takes tile A.order[b] instead; an entry outside the grid's
// tiles makes the block return (false) without touching anything.
template <int TY, int TZ>
__device__ __forceinline__ bool line_tile_coords(const PlanArgs &A, long long tile, int &tx,
                                                 int &ty, int &tz)
{
    const PbGrid &g = A.g;
    const int nx8 = (g.nx + kLine - 1) / kLine, nty = (g.ny + TY - 1) / TY;
    const int ntz = (g.nz + TZ - 1) / TZ;
    if (A.order != nullptr) {
        const long long o = A.order[tile];
        if (o < 0 || o >= (long long)nx8 * nty * ntz) return false;
        tx = (int)(o % nx8);
        ty = (int)((o / nx8) % nty);
        tz = (int)(o / ((long long)nx8 * nty));
        return true;
    }
    const int rx = (int)(tile % nx8);
    tile /= nx8;
    const int ry = (int)(tile % nty);
    const int rz = (int)(tile / nty);
    if (PB_TILE_ORDER == 0) {
        tx = rx;
        ty = ry;
        tz = rz;
        return true;
    }
    tx = center_out(rx, nx8, min(max(A.centre[0] / kLine, 0), nx8 - 1));
    ty = center_out(ry, nty, min(max(A.centre[1] / TY, 0), nty - 1));
    tz = center_out(rz, ntz, min(max(A.centre[2] / TZ, 0), ntz - 1));
    return true;
}

template <int TY, int TZ, int KCULL, bool BEAM_OUT>
__global__ void __launch_bounds__(TY * TZ, line_min_blocks<TY * TZ, BEAM_OUT>())
k_dose_line(const __grid_constant__ PlanArgs A, const float *__restrict__ wet,
            const PbLayer *__restrict__ layers, const float4 *__restrict__ geo,
            const float *__restrict__ mu, float *__restrict__ dose,
            float *__restrict__ beam_dose)
{
    __shared__ LineShared<TY * TZ, KCULL, BEAM_OUT> sh;
    int tx, ty, tz;
    if (!line_tile_coords<TY, TZ>(A, blockIdx.x, tx, ty, tz)) return;
    line_tile<TY, TZ, KCULL, BEAM_OUT>(A, tx, ty, tz, wet, layers, geo, mu, dose, beam_dose, sh);
}

// Forward kernel variants the autotuner chooses from.  Two families:
//   t<threads>_v<voxels per thread>_c<k>  8x8x8 tiles, each thread a set of
//       voxels evaluated one by one (dose_tile);
//   l8x<TY>x<TZ>_c<k>  8 x TY x TZ tiles, each thread a line of 8 voxels
//       along x evaluated as a quadratic (line_tile);
// k = spots each thread culls per compaction round.  `batch` marks the
// shapes the persistent batch kernel takes (tiles dividing 8x8x8 units).
struct DoseVariant {
    int line, ty, tz, nt, kcull;
    bool batch;
    const char *name;
};
constexpr DoseVariant kDoseVariants[] = {
    {1, 8, 8, 64, 2, true, "l8x8x8_c2"},    {1, 8, 8, 64, 4, true, "l8x8x8_c4"},
    {1, 8, 4, 32, 4, true, "l8x8x4_c4"},    {1, 4, 8, 32, 4, true, "l8x4x8_c4"},
    {1, 16, 8, 128, 2, false, "l8x16x8_c2"}, {1, 8, 16, 128, 2, false, "l8x8x16_c2"},
    {0, 8, 8, 128, 1, true, "t128_v4_c1"},  {0, 8, 8, 128, 2, true, "t128_v4_c2"},
    {0, 8, 8, 128, 4, true, "t128_v4_c4"},  {0, 8, 8, 256, 1, true, "t256_v2_c1"},
    {0, 8, 8, 128, 3, true, "t128_v4_c3"},
};
constexpr int kNumDoseVariants = sizeof(kDoseVariants) / sizeof(kDoseVariants[0]);

// The shape pb_dose and pb_count_evaluated use; pb_dose_adjoint runs the
// adjoint kernel of its family.
#ifndef PB_DEFAULT_DOSE_VARIANT
#define PB_DEFAULT_DOSE_VARIANT 4   // l8x16x8_c2
#endif
constexpr int kDefaultDoseVariant = PB_DEFAULT_DOSE_VARIANT;
static_assert(kDefaultDoseVariant >= 0 && kDefaultDoseVariant < kNumDoseVariants,
              "default shape");

// Line-tile shape of the counts and the adjoint (and of the per-beam
// forward): the default's when it is a line shape, else l8x8x8_c2.  On
// the 4-beam 256x256x160 plan l8x16x8_c2 measured 6.72 ms forward and
// 7.12 ms adjoint, against 6.83 and 7.55 ms for l8x8x8_c2.
constexpr int kLineShape = kDoseVariants[kDefaultDoseVariant].line ? kDefaultDoseVariant : 0;
static_assert(kDoseVariants[kLineShape].line, "a line shape");
constexpr int kLineTY = kDoseVariants[kLineShape].ty, kLineTZ = kDoseVariants[kLineShape].tz,
              kLineCull = kDoseVariants[kLineShape].kcull;

__global__ void __launch_bounds__(kLineTY * kLineTZ, line_min_blocks<kLineTY * kLineTZ>())
k_dose_count_line(const __grid_constant__ PlanArgs A, const float *__restrict__ wet,
                  const PbLayer *__restrict__ layers, const float4 *__restrict__ geo,
                  unsigned long long *count, const float *__restrict__ wfield)
{
    __shared__ LineShared<kLineTY * kLineTZ, kLineCull, false, false> sh;
    int tx, ty, tz;
    if (!line_tile_coords<kLineTY, kLineTZ>(A, blockIdx.x, tx, ty, tz)) return;
    line_tile<kLineTY, kLineTZ, kLineCull, false, kModeCount>(A, tx, ty, tz, wet, layers, geo,
                                                              nullptr, nullptr, nullptr, sh,
                                                              count, wfield);
}

__global__ void __launch_bounds__(kLineTY * kLineTZ, line_min_blocks<kLineTY * kLineTZ, true>())
k_adjoint_line(const __grid_constant__ PlanArgs A, const float *__restrict__ wet,
               const PbLayer *__restrict__ layers, const float4 *__restrict__ geo,
               const float *__restrict__ wfield, float *__restrict__ grad)
{
    __shared__ LineShared<kLineTY * kLineTZ, kLineCull, false, false> sh;
    int tx, ty, tz;
    if (!line_tile_coords<kLineTY, kLineTZ>(A, blockIdx.x, tx, ty, tz)) return;
    line_tile<kLineTY, kLineTZ, kLineCull, false, kModeAdjoint>(A, tx, ty, tz, wet, layers, geo,
                                                                nullptr, nullptr, nullptr, sh,
                                                                nullptr, wfield, grad);
}

// ------------------------------------------------------------ tile order
//
// The line tiles' work spans more than two orders of magnitude (tens of us
// for a tile no spot reaches, milliseconds for one that every beam crosses
// near the target), and blocks start in launch order, so a launch whose
// longest tiles start late ends on a few of them.  k_tile_cost estimates each
// tile's cost and k_order_* sort the tiles by it, most expensive first (a
// bucket sort on log2 of the cost); the forward and the adjoint then take
// their tiles in that order (PlanArgs::order).  The order changes when the
// work is done, not what each tile computes.

// Cost units: one spot evaluated over a tile; a kept (tile, layer) pair
// also pays its per-voxel Gaussian parameters, the cull and its barriers,
// about this many.  Measured on the 4-beam 256x256x160 plan (forward /
// adjoint): 24 -> 6.04 / 6.43 ms, 48 -> 6.03 / 6.41, 96 -> 6.02 / 6.39,
// 192 -> 6.02 / 6.38.
constexpr float kPairCost = 192.0f;
constexpr int kOrderBuckets = 1024;

// Estimated work of a kept (tile, layer) pair: kPairCost plus the layer's
// spots times the fraction of its spot box, scaled to the tile's depth, that
// lies within the cull radius of the tile's box (from the same sigma bound
// as the layer skip); 0 for a pair the dose kernels do not keep.
__device__ __forceinline__ float layer_pair_cost(const PbLayer &L, const TileBounds &tb,
                                                 const PbBeam &B)
{
    const float cut = __fmul_rn(1.1f, L.r80);
    if (!(L.n_spots > 0 && tb.w0 <= cut) || layer_skip(L, tb, B, cut)) return 0.0f;
    float frac = 1.0f;
    float pxl, pxh, pyl, pyh, it2, sig2;
    if (L.bound_ok && layer_sig2(L, tb, B, cut, it2, sig2)) {
        layer_box(L, tb, pxl, pxh, pyl, pyh);
        const float R = sqrtf(kCullLog2 * sig2 / ((0.5f * kLog2e) * it2));
        auto part = [](float lo, float hi, float a, float b) {
            const float ov = fminf(hi, b) - fmaxf(lo, a);
            const float len = hi - lo;
            if (!(ov > 0.0f)) return 0.0f;
            return len > 1e-3f ? fminf(ov / len, 1.0f) : 1.0f;
        };
        frac = part(pxl, pxh, tb.x0 - R, tb.x1 + R) * part(pyl, pyh, tb.y0 - R, tb.y1 + R);
    }
    return kPairCost + (float)L.n_spots * frac;
}

// One warp per line tile (raster index: x fastest; four tiles per block),
// each lane a quarter of the tile's lines: the tile's box and depth range
// per beam as line_tile forms them (warp reductions, no barrier), then the
// estimated cost of every layer pair it keeps.
template <int TY, int TZ>
__global__ void __launch_bounds__(128)
k_tile_cost(const __grid_constant__ PlanArgs A, const float *__restrict__ wet,
            const PbLayer *__restrict__ layers, float *__restrict__ cost, long long n_tiles)
{
    constexpr int kLinesPerLane = TY * TZ / 32;
    static_assert(TY * TZ % 32 == 0, "whole warps of lines");
    const long long tile = (long long)blockIdx.x * 4 + (threadIdx.x >> 5);
    if (tile >= n_tiles) return;   // the whole warp
    const int lane = threadIdx.x & 31;
    const int nx8 = (A.g.nx + kLine - 1) / kLine, nty = (A.g.ny + TY - 1) / TY;
    const int tx = (int)(tile % nx8), ty = (int)((tile / nx8) % nty);
    const int tz = (int)(tile / ((long long)nx8 * nty));
    const int i0 = tx * kLine;
    const int64_t V = (int64_t)A.g.nx * A.g.ny * A.g.nz;
    float c = 0.0f;
    for (int b = 0; b < A.n_beams; ++b) {
        const PbBeam &B = A.beams[b];
        float dX, dY, dZ;
        image_to_head(B.geom, A.g.spacing, 0.0f, 0.0f, dX, dY, dZ);
        const float dgx = -__fdiv_rn(dZ, B.geom.vsadx), dgy = -__fdiv_rn(dZ, B.geom.vsady);
        float v[12] = {INFINITY, -INFINITY, INFINITY, -INFINITY, INFINITY, -INFINITY,
                       INFINITY, -INFINITY, INFINITY, -INFINITY, INFINITY, -INFINITY};
#pragma unroll
        for (int m = 0; m < kLinesPerLane; ++m) {
            const int ln = lane + 32 * m;
            const int j = ty * TY + ln % TY, k = tz * TZ + ln / TY;
            const int nvalid = (j < A.g.ny && k < A.g.nz) ? min(kLine, A.g.nx - i0) : 0;
            if (nvalid <= 0) continue;
            const int64_t vbase = i0 + (int64_t)A.g.nx * (j + (int64_t)A.g.ny * k);
            float px, py, pz, X0, Y0, Z0;
            vox_mm(B.geom, A.g.spacing, i0, j, k, px, py, pz);
            image_to_head(B.geom, px, py, pz, X0, Y0, Z0);
            const float Xc = __fmaf_rn(3.5f, dX, X0), Yc = __fmaf_rn(3.5f, dY, Y0);
            const float Zc = __fmaf_rn(3.5f, dZ, Z0);
            const float gxc = __fsub_rn(1.0f, __fdiv_rn(Zc, B.geom.vsadx));
            const float gyc = __fsub_rn(1.0f, __fdiv_rn(Zc, B.geom.vsady));
#pragma unroll
            for (int q = 0; q < kLine; ++q) {
                if (q >= nvalid) continue;
                const float o = line_off(q);
                const float X = __fmaf_rn(o, dX, Xc), Y = __fmaf_rn(o, dY, Yc);
                const float Z = __fmaf_rn(o, dZ, Zc);
                const float w = __fmul_rn(__ldg(wet + b * V + vbase + q), 10.0f);
                const float dd = source_distance(B, X, Y, Z);
                const float GX = __fmaf_rn(o, dgx, gxc), GY = __fmaf_rn(o, dgy, gyc);
                v[0] = fminf(v[0], X);  v[1] = fmaxf(v[1], X);
                v[2] = fminf(v[2], Y);  v[3] = fmaxf(v[3], Y);
                v[4] = fminf(v[4], GX); v[5] = fmaxf(v[5], GX);
                v[6] = fminf(v[6], GY); v[7] = fmaxf(v[7], GY);
                v[8] = fminf(v[8], dd); v[9] = fmaxf(v[9], dd);
                v[10] = fminf(v[10], w == w ? w : -INFINITY);
                v[11] = fmaxf(v[11], w == w ? w : INFINITY);
            }
        }
#pragma unroll
        for (int m = 0; m < 12; ++m) v[m] = (m & 1) ? warp_max(v[m]) : warp_min(v[m]);
        TileBounds tb;
        tb.x0 = v[0]; tb.x1 = v[1]; tb.y0 = v[2]; tb.y1 = v[3];
        tb.gx0 = v[4]; tb.gx1 = v[5]; tb.gy0 = v[6]; tb.gy1 = v[7];
        tb.d0 = v[8]; tb.d1 = v[9]; tb.w0 = v[10]; tb.w1 = v[11];
        for (int l = lane; l < B.n_layers; l += 32)
            c += layer_pair_cost(layers[B.layer_start + l], tb, B);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) cost[tile] = c;
}

// Bucket of a cost, most expensive last: 32 buckets per octave.
__device__ __forceinline__ int order_bucket(float c)
{
    const float x = log2f(1.0f + fmaxf(c, 0.0f)) * 32.0f;
    return x < (float)(kOrderBuckets - 1) ? (int)x : kOrderBuckets - 1;
}

__global__ void k_order_hist(const float *__restrict__ cost, int n, int *__restrict__ hist)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) atomicAdd(hist + order_bucket(cost[i]), 1);
}

// Start of each bucket in the order, the most expensive bucket first (one
// block of kOrderBuckets threads; the counts are replaced by the starts).
__global__ void __launch_bounds__(kOrderBuckets) k_order_scan(int *hist)
{
    __shared__ int s[kOrderBuckets];
    const int t = threadIdx.x;
    s[t] = hist[kOrderBuckets - 1 - t];   // descending cost
    __syncthreads();
    for (int off = 1; off < kOrderBuckets; off <<= 1) {
        const int add = t >= off ? s[t - off] : 0;
        __syncthreads();
        s[t] += add;
        __syncthreads();
    }
    // exclusive start of bucket (kOrderBuckets - 1 - t)
    hist[kOrderBuckets - 1 - t] = t > 0 ? s[t - 1] : 0;
}

__global__ void k_order_scatter(const float *__restrict__ cost, int n, int *__restrict__ start,
                                int *__restrict__ order)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) order[atomicAdd(start + order_bucket(cost[i]), 1)] = i;
}

#ifndef PB_DOSE_MIN_BLOCKS
#define PB_DOSE_MIN_BLOCKS 5
#endif
// Resident blocks per SM the kernels are compiled for (their register
// budget).  Shapes of 128 threads that cull one round of 128 spots (the
// forward's default) take one more block: measured 8.28 -> 8.19 ms.  The
// adjoint (two rounds) stays at PB_DOSE_MIN_BLOCKS: one more made it
// slower (9.16 -> 9.23 ms).
template <int NT, int KCULL = 2> constexpr int dose_min_blocks()
{
    return NT == 128 ? PB_DOSE_MIN_BLOCKS + (KCULL == 1 ? 1 : 0) : 3;
}

template <int NT, int VPT, int KCULL, bool BEAM_OUT>
__global__ void __launch_bounds__(NT, dose_min_blocks<NT, KCULL>())
k_dose(const __grid_constant__ PlanArgs A, const float *__restrict__ wet,
       const PbLayer *__restrict__ layers, const float4 *__restrict__ geo,
       const float *__restrict__ mu, float *__restrict__ dose,
       float *__restrict__ beam_dose)
{
    __shared__ DoseShared<NT, KCULL> sh;
    dose_tile<NT, VPT, KCULL, BEAM_OUT>(A, blockIdx.x, wet, layers, geo, mu, dose, beam_dose, sh);
}

// The forward's SFU exponentials and spot-voxel evaluations, counted with
// its own decisions (dose_tile with COUNT); shape of pb_dose's kernel.
__global__ void __launch_bounds__(128, dose_min_blocks<128, 1>())
k_dose_count(const __grid_constant__ PlanArgs A, const float *__restrict__ wet,
             const PbLayer *__restrict__ layers, const float4 *__restrict__ geo,
             unsigned long long *count, const float *__restrict__ wfield)
{
    __shared__ DoseShared<128, 1> sh;
    dose_tile<128, 4, 1, false, kModeCount>(A, blockIdx.x, wet, layers, geo, nullptr, nullptr,
                                            nullptr, sh, count, wfield);
}

// Spot-weight gradient: dose_tile in adjoint mode, shape of pb_dose's kernel.
__global__ void __launch_bounds__(128, dose_min_blocks<128>())
k_adjoint_tile(const __grid_constant__ PlanArgs A, const float *__restrict__ wet,
               const PbLayer *__restrict__ layers, const float4 *__restrict__ geo,
               const float *__restrict__ wfield, float *__restrict__ grad)
{
    __shared__ DoseShared<128, 2> sh;
    dose_tile<128, 4, 2, false, kModeAdjoint>(A, blockIdx.x, wet, layers, geo, nullptr, nullptr,
                                              nullptr, sh, nullptr, wfield, grad);
}

// Spot-weight and spot-position gradients: dose_tile in kModeAdjointPos.
__global__ void __launch_bounds__(128, dose_min_blocks<128>())
k_adjoint_pos_tile(const __grid_constant__ PlanArgs A, const float *__restrict__ wet,
                   const PbLayer *__restrict__ layers, const float4 *__restrict__ geo,
                   const float *__restrict__ mu, const float *__restrict__ wfield,
                   float *__restrict__ grad, float *__restrict__ grad_x,
                   float *__restrict__ grad_y)
{
    __shared__ DoseShared<128, 2> sh;
    __shared__ float gsum_xy[2 * (2 * 128 + 8)];
    dose_tile<128, 4, 2, false, kModeAdjointPos>(A, blockIdx.x, wet, layers, geo, mu, nullptr,
                                                 nullptr, sh, nullptr, wfield, grad, grad_x,
                                                 grad_y, gsum_xy);
}

// SFU exp2 throughput: kEx2Chains independent chains x <- 2^(-x) per
// thread (each stays in (0.5, 1)); the result is stored only if it takes a
// value it never takes, so that nothing is removed as dead code.
constexpr int kEx2Chains = 8;
__device__ float g_ex2_sink;

__global__ void __launch_bounds__(256) k_ex2_rate(int iters)
{
    float x[kEx2Chains];
#pragma unroll
    for (int c = 0; c < kEx2Chains; ++c) x[c] = 0.5f + 0.01f * (float)(c + (threadIdx.x & 7));
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kEx2Chains; ++c) x[c] = ex2(-x[c]);
    }
    float t = 0.0f;
#pragma unroll
    for (int c = 0; c < kEx2Chains; ++c) t += x[c];
    if (t == 12345.0f) g_ex2_sink = t;
}

// One plan of a batch as the persistent kernel reads it.
struct BatchDose {
    PlanArgs A;
    const float *wet;
    const PbLayer *layers;
    const float4 *geo;
    const float *mu;
    float *dose;
    long long tile_start;   // first work item of the plan (queue order)
};

// Persistent forward over many plans: blocks take (plan, tile) items from
// one queue until it is empty.  Plans are stored in decreasing order of
// estimated cost per tile so that the expensive tiles start first.
template <int NT, int VPT, int KCULL>
__global__ void __launch_bounds__(NT, dose_min_blocks<NT, KCULL>())
k_dose_batch(const BatchDose *__restrict__ plans, int n_plans, long long n_items,
             unsigned long long *counter)
{
    __shared__ DoseShared<NT, KCULL> sh;
    __shared__ long long s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = (long long)atomicAdd(counter, 1ULL);
        __syncthreads();
        const long long it = s_item;
        __syncthreads();
        if (it >= n_items) break;
        int lo = 0, hi = n_plans - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (plans[mid].tile_start <= it) lo = mid; else hi = mid - 1;
        }
        const BatchDose &D = plans[lo];
        dose_tile<NT, VPT, KCULL, false>(D.A, (int)(it - D.tile_start), D.wet, D.layers, D.geo,
                                         D.mu, D.dose, nullptr, sh);
        __syncthreads();
    }
}

// The persistent batch on line tiles: the same queue of 8x8x8 units, each
// done as (8/TY) x (8/TZ) tiles of the kernel's shape.
template <int TY, int TZ, int KCULL>
__global__ void __launch_bounds__(TY * TZ, line_min_blocks<TY * TZ>())
k_dose_batch_line(const BatchDose *__restrict__ plans, int n_plans, long long n_items,
                  unsigned long long *counter)
{
    static_assert(8 % TY == 0 && 8 % TZ == 0, "batch units are 8x8x8 voxels");
    __shared__ LineShared<TY * TZ, KCULL> sh;
    __shared__ long long s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = (long long)atomicAdd(counter, 1ULL);
        __syncthreads();
        const long long it = s_item;
        __syncthreads();
        if (it >= n_items) break;
        int lo = 0, hi = n_plans - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (plans[mid].tile_start <= it) lo = mid; else hi = mid - 1;
        }
        const BatchDose &D = plans[lo];
        long long u = it - D.tile_start;
        const int ux = (int)(u % D.A.tiles_x);
        u /= D.A.tiles_x;
        const int uy = (int)(u % D.A.tiles_y), uz = (int)(u / D.A.tiles_y);
        for (int sz = 0; sz < 8 / TZ; ++sz)
            for (int sy = 0; sy < 8 / TY; ++sy) {
                line_tile<TY, TZ, KCULL, false>(D.A, ux, uy * (8 / TY) + sy, uz * (8 / TZ) + sz,
                                                D.wet, D.layers, D.geo, D.mu, D.dose, nullptr,
                                                sh);
                __syncthreads();
            }
    }
}

// ---------------------------------------------------------------- objective

constexpr int kObjBlocks = 148 * 4;

__global__ void __launch_bounds__(256)
k_objective(const float *__restrict__ dose, const float *__restrict__ presc,
            const float *__restrict__ weight, int64_t n, double *partial,
            float *__restrict__ resid)
{
    double acc = 0.0;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
         q += (int64_t)gridDim.x * blockDim.x) {
        const double d = (double)dose[q] - (double)presc[q];
        const double w = (double)weight[q];
        acc += w * d * d;
        if (resid) resid[q] = (float)(2.0 * w * d);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    __shared__ double s[8];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += s[w];
        partial[blockIdx.x] = t;
    }
}

__global__ void k_objective_final(const double *partial, int nb, double *obj)
{
    __shared__ double s[256];
    double a = 0.0;
    for (int i = threadIdx.x; i < nb; i += 256) a += partial[i];
    s[threadIdx.x] = a;
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) s[threadIdx.x] += s[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) obj[0] = s[0];
}

// ----------------------------------------------------------- layer bounds

struct BeamList {
    int n_beams;
    PbBeam b[PB_MAX_BEAMS];
};

constexpr int kBoundThreads = 256;
constexpr int kHaloSamples = 2048;

// sh(w), the nuclear-halo sigma before its clamp at 0 (IMPTClasses.cu:104-121),
// in FP64.
__device__ __forceinline__ double halo_sigma(double w, double r80)
{
    const double a1 = w - r80 - 5.0;
    return 2.85 + 0.0014 * r80 * log(w + 3.0) + 0.06 * w - 7.4e-5 * w * w -
           (0.22 * r80) / (a1 * a1);
}

// One block per (beam, layer): the culling bounds of PbLayer.
//   spot box     min / max of the spots' x and y
//   mcs_max      max |sigma| over the layer's LUT row (interpolation and the
//                end clamps stay within the row's values)
//   sh_max       max over the kernels' clamped depth w in [0.1, R80 - 0.1]
//                (the single point R80 - 0.1 when that is below 0.1) of
//                max(sh(w), 0): the maximum over kHaloSamples equally spaced
//                points plus Lip * h / 2, with Lip a bound on |sh'(w)| there:
//                |0.0014 R80| / (w + 3) + |0.06 - 1.48e-4 w| + 0.44 |R80| / 5.1^3
//                (|w - R80 - 5| >= 5.1 on the interval).
// bound_ok stays 0 when the layer has no spot or a value is not finite.
__global__ void __launch_bounds__(kBoundThreads)
k_layer_bounds(const __grid_constant__ BeamList A, PbLayer *layers, const float4 *geo)
{
    const PbBeam &B = A.b[blockIdx.y];
    if ((int)blockIdx.x >= B.n_layers) return;
    PbLayer *Lp = layers + B.layer_start + blockIdx.x;
    const PbLayer L = *Lp;
    __shared__ float s_v[kBoundThreads / 32][6];
    __shared__ double s_h[kBoundThreads / 32];
    __shared__ int s_bad;
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    bool bad = false;
    float x0 = INFINITY, x1 = -INFINITY, y0 = INFINITY, y1 = -INFINITY, mm = 0.0f;
    const int s0 = B.spot_start + L.spot_start;
    for (int i = threadIdx.x; i < L.n_spots; i += kBoundThreads) {
        const float4 g = geo[2 * (int64_t)(s0 + i)];
        bad |= !(isfinite(g.x) && isfinite(g.y));
        x0 = fminf(x0, g.x);
        x1 = fmaxf(x1, g.x);
        y0 = fminf(y0, g.y);
        y1 = fmaxf(y1, g.y);
    }
    const float *sig = B.sigmas_dev + (size_t)L.energy_id * B.lut_len;
    for (int i = threadIdx.x; i < B.lut_len; i += kBoundThreads) {
        const float v = sig[i];
        bad |= !isfinite(v);
        mm = fmaxf(mm, fabsf(v));
    }
    const double r80 = (double)L.r80;
    const double hi_w = (double)(L.r80 - 0.1f);
    const double lo_w = hi_w > 0.1 ? 0.1 : hi_w;
    const double h = (hi_w - lo_w) / (kHaloSamples - 1);
    double shm = 0.0;
    for (int k = threadIdx.x; k < kHaloSamples; k += kBoundThreads) {
        const double v = halo_sigma(lo_w + h * k, r80);
        shm = v > shm ? v : shm;
    }
    const double lip = fabs(0.0014 * r80) / (lo_w + 3.0) +
                       fmax(fabs(0.06 - 1.48e-4 * lo_w), fabs(0.06 - 1.48e-4 * hi_w)) +
                       0.44 * fabs(r80) / (5.1 * 5.1 * 5.1);
    x0 = warp_min(x0);
    x1 = warp_max(x1);
    y0 = warp_min(y0);
    y1 = warp_max(y1);
    mm = warp_max(mm);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) shm = fmax(shm, __shfl_xor_sync(0xffffffffu, shm, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (bad) atomicOr(&s_bad, 1);
    if (lane == 0) {
        s_v[warp][0] = x0;
        s_v[warp][1] = x1;
        s_v[warp][2] = y0;
        s_v[warp][3] = y1;
        s_v[warp][4] = mm;
        s_h[warp] = shm;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int w = 1; w < kBoundThreads / 32; ++w) {
        x0 = fminf(x0, s_v[w][0]);
        x1 = fmaxf(x1, s_v[w][1]);
        y0 = fminf(y0, s_v[w][2]);
        y1 = fmaxf(y1, s_v[w][3]);
        mm = fmaxf(mm, s_v[w][4]);
        shm = fmax(shm, s_h[w]);
    }
    shm += lip * h * 0.5;
    const bool ok = L.n_spots > 0 && !s_bad && isfinite(shm) && isfinite(r80);
    Lp->sx0 = x0;
    Lp->sx1 = x1;
    Lp->sy0 = y0;
    Lp->sy1 = y1;
    Lp->sh_max = (float)shm * 1.0001f + 1e-3f;
    Lp->mcs_max = mm;
    Lp->bound_ok = ok ? 1 : 0;
}

// --------------------------------------------------------------- pair count

__global__ void __launch_bounds__(256)
k_count(const __grid_constant__ PlanArgs A, const float *__restrict__ wet,
        const PbLayer *__restrict__ layers, unsigned long long *count)
{
    const int64_t V = (int64_t)A.g.nx * A.g.ny * A.g.nz;
    unsigned long long c = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V;
         v += (int64_t)gridDim.x * blockDim.x) {
        for (int b = 0; b < A.n_beams; ++b) {
            const float wmm = __fmul_rn(wet[b * V + v], 10.0f);
            const PbBeam &B = A.beams[b];
            for (int l = 0; l < B.n_layers; ++l) {
                const PbLayer L = layers[B.layer_start + l];
                if (!(wmm > __fmul_rn(1.1f, L.r80))) c += (unsigned long long)L.n_spots;
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(count, c);
}

// ----------------------------------------------------------------- launches

static void fill_args(PlanArgs &A, const PbGrid &g, const PbBeam *beams, int n_beams,
                      float scale)
{
    A.g = g;
    A.n_beams = n_beams;
    A.tiles_x = (g.nx + 7) / 8;
    A.tiles_y = (g.ny + 7) / 8;
    A.tiles_z = (g.nz + 7) / 8;
    A.scale = scale;
    A.order = nullptr;
    double c[3] = {0.0, 0.0, 0.0};
    for (int b = 0; b < n_beams; ++b) {
        A.beams[b] = beams[b];
        for (int a = 0; a < 3; ++a) c[a] += beams[b].geom.iso[a];
    }
    const int n[3] = {g.nx, g.ny, g.nz};
    for (int a = 0; a < 3; ++a) {
        const double v = n_beams > 0 && g.spacing > 0.0f ? c[a] / n_beams / g.spacing : 0.0;
        A.centre[a] = v != v ? 0 : (int)fmin(fmax(v, 0.0), (double)(n[a] - 1));
    }
}


int dose_variant_default() { return kDefaultDoseVariant; }
int dose_variant_count() { return kNumDoseVariants; }

static bool variant_line(int v)
{
    if (v < 0 || v >= kNumDoseVariants) v = kDefaultDoseVariant;
    return kDoseVariants[v].line != 0;
}
const char *dose_variant_name(int v)
{
    return (v >= 0 && v < kNumDoseVariants) ? kDoseVariants[v].name : "";
}
static bool dose_variant_batch(int v)
{
    return v >= 0 && v < kNumDoseVariants && kDoseVariants[v].batch;
}

static unsigned line_tiles(const PbGrid &g, int ty, int tz)
{
    return (unsigned)((long long)((g.nx + kLine - 1) / kLine) * ((g.ny + ty - 1) / ty) *
                      ((g.nz + tz - 1) / tz));
}

template <int NT, int VPT, int KCULL>
static void launch_dose_t(const PlanArgs &A, unsigned tiles, const float *wet,
                          const PbLayer *layers, const float4 *geo, const float *mu,
                          float *dose, cudaStream_t st)
{
    k_dose<NT, VPT, KCULL, false><<<tiles, NT, 0, st>>>(A, wet, layers, geo, mu, dose, nullptr);
}

template <int TY, int TZ, int KCULL>
static void launch_line_t(const PlanArgs &A, const float *wet, const PbLayer *layers,
                          const float4 *geo, const float *mu, float *dose, cudaStream_t st)
{
    k_dose_line<TY, TZ, KCULL, false><<<line_tiles(A.g, TY, TZ), TY * TZ, 0, st>>>(
        A, wet, layers, geo, mu, dose, nullptr);
}

PbStatus launch_dose(const PbGrid &g, const PbBeam *beams, int n_beams,
                     const float *wet, const PbLayer *layers, const float *geo,
                     const float *mu, float scale, float *dose, float *beam_dose,
                     cudaStream_t st, int variant, const int *order)
{
    PlanArgs A;
    fill_args(A, g, beams, n_beams, scale);
    const unsigned tiles = (unsigned)((int64_t)A.tiles_x * A.tiles_y * A.tiles_z);
    const float4 *g4 = reinterpret_cast<const float4 *>(geo);
    if (variant < 0) variant = kDefaultDoseVariant;
    // a tile order (pb_tile_order) is for the line-tile shape of the default
    A.order = (variant_line(variant) && (beam_dose || variant == kLineShape)) ? order : nullptr;
    if (beam_dose) {
        // per-beam output: the default shape of the variant's family only
        if (variant_line(variant))
            k_dose_line<kLineTY, kLineTZ, kLineCull, true>
                <<<line_tiles(g, kLineTY, kLineTZ), kLineTY * kLineTZ, 0, st>>>(
                    A, wet, layers, g4, mu, dose, beam_dose);
        else
            k_dose<128, 4, 1, true><<<tiles, 128, 0, st>>>(A, wet, layers, g4, mu, dose,
                                                           beam_dose);
        return check_launch("k_dose");
    }
    switch (variant) {
    case 1: launch_line_t<8, 8, 4>(A, wet, layers, g4, mu, dose, st); break;
    case 2: launch_line_t<8, 4, 4>(A, wet, layers, g4, mu, dose, st); break;
    case 3: launch_line_t<4, 8, 4>(A, wet, layers, g4, mu, dose, st); break;
    case 4: launch_line_t<16, 8, 2>(A, wet, layers, g4, mu, dose, st); break;
    case 5: launch_line_t<8, 16, 2>(A, wet, layers, g4, mu, dose, st); break;
    case 6: launch_dose_t<128, 4, 1>(A, tiles, wet, layers, g4, mu, dose, st); break;
    case 7: launch_dose_t<128, 4, 2>(A, tiles, wet, layers, g4, mu, dose, st); break;
    case 8: launch_dose_t<128, 4, 4>(A, tiles, wet, layers, g4, mu, dose, st); break;
    case 9: launch_dose_t<256, 2, 1>(A, tiles, wet, layers, g4, mu, dose, st); break;
    case 10: launch_dose_t<128, 4, 3>(A, tiles, wet, layers, g4, mu, dose, st); break;
    default: launch_line_t<8, 8, 2>(A, wet, layers, g4, mu, dose, st); break;
    }
    return check_launch("k_dose");
}

void fill_batch_dose(BatchDose &D, const PbGrid &g, const PbBeam *beams, int n_beams,
                     float scale, const float *wet, const PbLayer *layers, const float *geo,
                     const float *mu, float *dose, long long tile_start)
{
    fill_args(D.A, g, beams, n_beams, scale);
    D.wet = wet;
    D.layers = layers;
    D.geo = reinterpret_cast<const float4 *>(geo);
    D.mu = mu;
    D.dose = dose;
    D.tile_start = tile_start;
}

size_t batch_dose_size() { return sizeof(BatchDose); }

long long plan_tiles(const PbGrid &g)
{
    return (long long)((g.nx + 7) / 8) * ((g.ny + 7) / 8) * ((g.nz + 7) / 8);
}

PbStatus launch_dose_batch(const void *plans_dev, int n_plans, long long n_items,
                           unsigned long long *counter, int variant, int blocks,
                           cudaStream_t st)
{
    if (!dose_variant_batch(variant))
        return set_error(PB_ERR_INVALID, "variant %d (%s) is not a batch shape", variant,
                         dose_variant_name(variant));
    PbStatus s = check_cuda(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st),
                            "cudaMemsetAsync(queue)");
    if (s != PB_OK) return s;
    const BatchDose *P = static_cast<const BatchDose *>(plans_dev);
    switch (variant) {
    case 1: k_dose_batch_line<8, 8, 4><<<blocks, 64, 0, st>>>(P, n_plans, n_items, counter); break;
    case 2: k_dose_batch_line<8, 4, 4><<<blocks, 32, 0, st>>>(P, n_plans, n_items, counter); break;
    case 3: k_dose_batch_line<4, 8, 4><<<blocks, 32, 0, st>>>(P, n_plans, n_items, counter); break;
    case 6: k_dose_batch<128, 4, 1><<<blocks, 128, 0, st>>>(P, n_plans, n_items, counter); break;
    case 7: k_dose_batch<128, 4, 2><<<blocks, 128, 0, st>>>(P, n_plans, n_items, counter); break;
    case 8: k_dose_batch<128, 4, 4><<<blocks, 128, 0, st>>>(P, n_plans, n_items, counter); break;
    case 9: k_dose_batch<256, 2, 1><<<blocks, 256, 0, st>>>(P, n_plans, n_items, counter); break;
    case 10: k_dose_batch<128, 4, 3><<<blocks, 128, 0, st>>>(P, n_plans, n_items, counter); break;
    default: k_dose_batch_line<8, 8, 2><<<blocks, 64, 0, st>>>(P, n_plans, n_items, counter); break;
    }
    return check_launch("k_dose_batch");
}

int dose_variant_threads(int variant)
{
    return (variant >= 0 && variant < kNumDoseVariants) ? kDoseVariants[variant].nt : 128;
}

PbStatus launch_adjoint(const PbGrid &g, const PbBeam *beams, int n_beams,
                        const float *wet, const PbLayer *layers, const float *geo,
                        const float *w, float scale, float *grad, cudaStream_t st,
                        int variant, const int *order)
{
    PlanArgs A;
    fill_args(A, g, beams, n_beams, scale);
    A.order = variant_line(variant) ? order : nullptr;
    int total_spots = 0;
    for (int b = 0; b < n_beams; ++b) {
        const int e = beams[b].spot_start + beams[b].n_spots;
        if (e > total_spots) total_spots = e;
    }
    PbStatus s = check_cuda(cudaMemsetAsync(grad, 0, sizeof(float) * (size_t)total_spots, st),
                            "cudaMemsetAsync(grad)");
    if (s != PB_OK) return s;
    const int64_t tiles = (int64_t)A.tiles_x * A.tiles_y * A.tiles_z;
    const float4 *g4 = reinterpret_cast<const float4 *>(geo);
    if (variant_line(variant)) {
        k_adjoint_line<<<line_tiles(g, kLineTY, kLineTZ), kLineTY * kLineTZ, 0, st>>>(
            A, wet, layers, g4, w, grad);
        return check_launch("k_adjoint_line");
    }
    k_adjoint_tile<<<(unsigned)tiles, 128, 0, st>>>(A, wet, layers, g4, w, grad);
    return check_launch("k_adjoint_tile");
}

PbStatus launch_adjoint_positions(const PbGrid &g, const PbBeam *beams, int n_beams,
                                  const float *wet, const PbLayer *layers, const float *geo,
                                  const float *mu, const float *w, float scale, float *grad,
                                  float *grad_x, float *grad_y, cudaStream_t st)
{
    PlanArgs A;
    fill_args(A, g, beams, n_beams, scale);
    int total_spots = 0;
    for (int b = 0; b < n_beams; ++b) {
        const int e = beams[b].spot_start + beams[b].n_spots;
        if (e > total_spots) total_spots = e;
    }
    const size_t bytes = sizeof(float) * (size_t)total_spots;
    PbStatus s = PB_OK;
    for (float *o : {grad, grad_x, grad_y})
        if (o && s == PB_OK) s = check_cuda(cudaMemsetAsync(o, 0, bytes, st), "cudaMemsetAsync");
    if (s != PB_OK) return s;
    const int64_t tiles = (int64_t)A.tiles_x * A.tiles_y * A.tiles_z;
    k_adjoint_pos_tile<<<(unsigned)tiles, 128, 0, st>>>(A, wet, layers,
                                                        reinterpret_cast<const float4 *>(geo), mu,
                                                        w, grad, grad_x, grad_y);
    return check_launch("k_adjoint_pos_tile");
}

size_t objective_work_size() { return sizeof(double) * kObjBlocks; }

PbStatus launch_objective(const float *dose, const float *presc, const float *weight,
                          int64_t n, double *obj, float *resid, void *work,
                          cudaStream_t st)
{
    double *partial = static_cast<double *>(work);
    k_objective<<<kObjBlocks, 256, 0, st>>>(dose, presc, weight, n, partial, resid);
    PbStatus s = check_launch("k_objective");
    if (s != PB_OK) return s;
    k_objective_final<<<1, 256, 0, st>>>(partial, kObjBlocks, obj);
    return check_launch("k_objective_final");
}

PbStatus launch_layer_bounds(const PbBeam *beams, int n_beams, PbLayer *layers,
                            const float *geo, cudaStream_t st)
{
    BeamList A;
    A.n_beams = n_beams;
    int max_layers = 0;
    for (int b = 0; b < n_beams; ++b) {
        A.b[b] = beams[b];
        if (beams[b].n_layers > max_layers) max_layers = beams[b].n_layers;
    }
    if (max_layers == 0) return PB_OK;
    k_layer_bounds<<<dim3((unsigned)max_layers, (unsigned)n_beams), kBoundThreads, 0, st>>>(
        A, layers, reinterpret_cast<const float4 *>(geo));
    return check_launch("k_layer_bounds");
}

long long tile_order_count(const PbGrid &g) { return line_tiles(g, kLineTY, kLineTZ); }

void tile_order_tile(int *voxels)
{
    voxels[0] = kLine;
    voxels[1] = kLineTY;
    voxels[2] = kLineTZ;
}

size_t tile_order_work_size(const PbGrid &g)
{
    const size_t n = (size_t)tile_order_count(g);
    return ((n * sizeof(float) + 255) / 256) * 256 + kOrderBuckets * sizeof(int);
}

PbStatus launch_tile_order(const PbGrid &g, const PbBeam *beams, int n_beams, const float *wet,
                           const PbLayer *layers, void *work, int *order, cudaStream_t st)
{
    PlanArgs A;
    fill_args(A, g, beams, n_beams, 1.0f);
    const long long n = tile_order_count(g);
    if (n <= 0) return PB_OK;
    if (n > (long long)INT_MAX) return set_error(PB_ERR_INVALID, "too many tiles for an order");
    float *cost = static_cast<float *>(work);
    int *hist = reinterpret_cast<int *>(static_cast<char *>(work) +
                                        ((size_t)n * sizeof(float) + 255) / 256 * 256);
    PbStatus s = check_cuda(cudaMemsetAsync(hist, 0, kOrderBuckets * sizeof(int), st),
                            "cudaMemsetAsync(order buckets)");
    if (s != PB_OK) return s;
    k_tile_cost<kLineTY, kLineTZ><<<(unsigned)((n + 3) / 4), 128, 0, st>>>(A, wet, layers, cost,
                                                                          n);
    s = check_launch("k_tile_cost");
    if (s != PB_OK) return s;
    const unsigned blocks = (unsigned)((n + 255) / 256);
    k_order_hist<<<blocks, 256, 0, st>>>(cost, (int)n, hist);
    k_order_scan<<<1, kOrderBuckets, 0, st>>>(hist);
    k_order_scatter<<<blocks, 256, 0, st>>>(cost, (int)n, hist, order);
    return check_launch("k_order_scatter");
}

PbStatus launch_count_evaluated(const PbGrid &g, const PbBeam *beams, int n_beams,
                                const float *wet, const PbLayer *layers, const float *geo,
                                unsigned long long *count, cudaStream_t st, int variant,
                                const float *wfield, float scale)
{
    PlanArgs A;
    fill_args(A, g, beams, n_beams, scale);
    PbStatus s = check_cuda(cudaMemsetAsync(count, 0, 2 * sizeof(unsigned long long), st),
                            "cudaMemsetAsync(count)");
    if (s != PB_OK) return s;
    const int64_t tiles = (int64_t)A.tiles_x * A.tiles_y * A.tiles_z;
    const float4 *g4 = reinterpret_cast<const float4 *>(geo);
    if (variant_line(variant)) {
        k_dose_count_line<<<line_tiles(g, kLineTY, kLineTZ), kLineTY * kLineTZ, 0, st>>>(
            A, wet, layers, g4, count, wfield);
        return check_launch("k_dose_count_line");
    }
    k_dose_count<<<(unsigned)tiles, 128, 0, st>>>(A, wet, layers, g4, count, wfield);
    return check_launch("k_dose_count");
}

PbStatus measure_ex2_rate(double *ops_per_s, cudaStream_t st)
{
    int dev = 0, sms = 0;
    PbStatus s = check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    if (s == PB_OK)
        s = check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev),
                       "cudaDeviceGetAttribute");
    if (s != PB_OK) return s;
    const int blocks = sms * 8, iters = 4096;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    s = check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
    if (s == PB_OK) s = check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
    float best = 0.0f;
    for (int rep = 0; rep < 4 && s == PB_OK; ++rep) {   // the first run warms up
        s = check_cuda(cudaEventRecord(e0, st), "cudaEventRecord");
        if (s == PB_OK) {
            k_ex2_rate<<<blocks, 256, 0, st>>>(iters);
            s = check_launch("k_ex2_rate");
        }
        if (s == PB_OK) s = check_cuda(cudaEventRecord(e1, st), "cudaEventRecord");
        if (s == PB_OK) s = check_cuda(cudaEventSynchronize(e1), "cudaEventSynchronize");
        float ms = 0.0f;
        if (s == PB_OK) s = check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
        if (s == PB_OK && rep > 0 && (best == 0.0f || ms < best)) best = ms;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s != PB_OK) return s;
    *ops_per_s = (double)blocks * 256.0 * iters * kEx2Chains / (best * 1e-3);
    return PB_OK;
}

PbStatus launch_count_pairs(const PbGrid &g, const PbBeam *beams, int n_beams,
                            const float *wet, const PbLayer *layers,
                            unsigned long long *count, cudaStream_t st)
{
    PlanArgs A;
    fill_args(A, g, beams, n_beams, 1.0f);
    PbStatus s = check_cuda(cudaMemsetAsync(count, 0, sizeof(unsigned long long), st),
                            "cudaMemsetAsync(count)");
    if (s != PB_OK) return s;
    k_count<<<148 * 8, 256, 0, st>>>(A, wet, layers, count);
    return check_launch("k_count");
}

}  // namespace pb
