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
// Work decomposition: one block of 256 threads per 8x8x8 voxel tile, two
// voxels per thread; all beams and layers of the plan are looped inside
// the block, so each voxel's dose is written once, compensated (Neumaier)
// across layers and beams, with no atomics.  Per (tile, layer) the layer's
// LUT row is staged in shared memory and the layer's spots are culled
// against the tile: a spot is skipped when, for every voxel of the tile,
// its Gaussian factor is below 2^-24 of the voxel's peak factor (bound from
// the tile's BEV box and the widest halo sigma in the tile).  Surviving
// spots are compacted into shared memory and streamed by every thread.
//
// The adjoint uses the same tiles and culling; per (tile, layer) the active
// voxels (dObj/dD != 0, inside the range cut) are compacted into shared
// memory and each thread takes one surviving spot and reduces over them,
// then adds its partial to the spot's gradient with one atomic.
#include "pb_internal.h"

namespace pb {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kVpt = 2;            // voxels per thread
constexpr float kCullLog2 = 24.0f; // skip factors below 2^-24

struct PlanArgs {
    PbGrid g;
    int n_beams;
    int tiles_x, tiles_y, tiles_z;
    float scale;
    PbBeam beams[PB_MAX_BEAMS];
};

struct __align__(16) SpotRec {
    float4 a;  // (-x, -y, tx, -ty)
    float4 b;  // (-cs, it2, mu, 0)
};

struct __align__(16) VoxRec {
    float4 a;  // (X, Y, gx, gy)
    float4 b;  // (ps2, hs2, w*Pf, w*Hf)
};

struct TileBounds {
    float x0, x1, y0, y1, gx0, gx1, gy0, gy1;
};

// Per-(voxel, layer) Gaussian parameters.  wet_mm is 10*WET (cm), dist the
// distance to the source (mm).  Exponent scales are pre-multiplied by
// log2(e) for ex2.
__device__ __forceinline__ void layer_params(float wet_mm, float dist, float r80,
                                             const float *s_dep, const float *s_sig,
                                             const float *s_idd, int lut_len,
                                             float ca, float cb, float cc,
                                             float &pf, float &hf, float &ps2,
                                             float &hs2)
{
    int lo = 0, hi = lut_len;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (wet_mm <= s_dep[mid]) hi = mid; else lo = mid + 1;
    }
    float idd, sms;
    if (lo == lut_len) {
        idd = s_idd[lo - 1];
        sms = s_sig[lo - 1];
    } else if (lo == 0) {
        idd = s_idd[0];
        sms = s_sig[0];
    } else {
        const float f = (wet_mm - s_dep[lo - 1]) / (s_dep[lo] - s_dep[lo - 1]);
        idd = fmaf(s_idd[lo] - s_idd[lo - 1], f, s_idd[lo - 1]);
        sms = fmaf(s_sig[lo] - s_sig[lo - 1], f, s_sig[lo - 1]);
    }
    const float d = dist - wet_mm + 0.7f * r80;
    const float st = fmaf(fmaf(ca, d, cb), d, cc) + sms;
    const float w = fminf(fmaxf(wet_mm, 0.1f), r80 - 0.1f);
    const float a1 = w - r80 - 5.0f;
    float sh = 2.85f + 0.0014f * r80 * logf(w + 3.0f) + 0.06f * w - 7.4e-5f * w * w -
               (0.22f * r80) / (a1 * a1);
    const float r3 = r80 + 3.0f;
    float wh = 0.052f * logf(1.13f + w / (11.2f - 0.023f * r80)) +
               0.35f * (0.0017f * r80 * r80 - r80) / (r3 * r3 - w * w) -
               1.61e-9f * w * r3 * r3;
    sh = fmaxf(sh, 0.0f);
    wh = fminf(fmaxf(wh, 0.0f), 0.9f);
    const float st2 = st * st;
    const float sht2 = fmaf(sh, sh, st2);
    pf = (1.0f - wh) * idd / (kTwoPi * st2);
    hf = wh * idd / (kTwoPi * sht2);
    ps2 = st2 != 0.0f ? (-0.5f * kLog2e) / st2 : -INFINITY;
    hs2 = sht2 != 0.0f ? (-0.5f * kLog2e) / sht2 : -INFINITY;
}

// True unless every voxel of the tile is further than the cull radius from
// the spot's axis.  nhs = smallest |hs2| among the tile's active voxels.
__device__ __forceinline__ bool cull_keep(float xs, float ys, float it2,
                                          const TileBounds &tb, float nhs)
{
    const float p0 = xs * tb.gx0, p1 = xs * tb.gx1;
    const float lox = tb.x0 - fmaxf(p0, p1), hix = tb.x1 - fminf(p0, p1);
    const float dx = fmaxf(0.0f, fmaxf(lox, -hix));
    const float q0 = ys * tb.gy0, q1 = ys * tb.gy1;
    const float loy = tb.y0 - fmaxf(q0, q1), hiy = tb.y1 - fminf(q0, q1);
    const float dy = fmaxf(0.0f, fmaxf(loy, -hiy));
    const float e = (dx * dx + dy * dy) * it2 * nhs;
    return !(e >= kCullLog2);
}

__device__ __forceinline__ void neumaier(float &s, float &c, float x)
{
    const float t = s + x;
    if (fabsf(s) >= fabsf(x)) c += (s - t) + x; else c += (x - t) + s;
    s = t;
}

// Block-wide min/max of the tile's BEV box over valid voxels.
__device__ __forceinline__ TileBounds tile_bounds(const float *X, const float *Y,
                                                  const float *GX, const float *GY,
                                                  const bool *valid,
                                                  float (*s_red)[9])
{
    float v[8] = {INFINITY, -INFINITY, INFINITY, -INFINITY,
                  INFINITY, -INFINITY, INFINITY, -INFINITY};
#pragma unroll
    for (int q = 0; q < kVpt; ++q) {
        if (!valid[q]) continue;
        v[0] = fminf(v[0], X[q]);  v[1] = fmaxf(v[1], X[q]);
        v[2] = fminf(v[2], Y[q]);  v[3] = fmaxf(v[3], Y[q]);
        v[4] = fminf(v[4], GX[q]); v[5] = fmaxf(v[5], GX[q]);
        v[6] = fminf(v[6], GY[q]); v[7] = fmaxf(v[7], GY[q]);
    }
#pragma unroll
    for (int m = 0; m < 8; ++m) v[m] = (m & 1) ? warp_max(v[m]) : warp_min(v[m]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
#pragma unroll
        for (int m = 0; m < 8; ++m) s_red[warp][m] = v[m];
    }
    __syncthreads();
    TileBounds tb;
    float r[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) r[m] = s_red[0][m];
    for (int w = 1; w < kWarps; ++w) {
#pragma unroll
        for (int m = 0; m < 8; ++m) r[m] = (m & 1) ? fmaxf(r[m], s_red[w][m]) : fminf(r[m], s_red[w][m]);
    }
    tb.x0 = r[0]; tb.x1 = r[1]; tb.y0 = r[2]; tb.y1 = r[3];
    tb.gx0 = r[4]; tb.gx1 = r[5]; tb.gy0 = r[6]; tb.gy1 = r[7];
    return tb;
}

__device__ __forceinline__ float block_max_slot8(float v, float (*s_red)[9])
{
    v = warp_max(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_red[warp][8] = v;
    __syncthreads();
    float r = s_red[0][8];
    for (int w = 1; w < kWarps; ++w) r = fmaxf(r, s_red[w][8]);
    return r;
}

struct VoxelGeom {
    float X[kVpt], Y[kVpt], GX[kVpt], GY[kVpt], DIST[kVpt], WMM[kVpt];
};

__device__ __forceinline__ void beam_voxel_geom(const PbGrid &g, const PbBeam &B,
                                                const float *__restrict__ wetb,
                                                const int *vi, const int *vj,
                                                const int *vk, const bool *valid,
                                                const int64_t *vidx, VoxelGeom &o)
{
#pragma unroll
    for (int q = 0; q < kVpt; ++q) {
        if (valid[q]) {
            float px, py, pz, hx, hy, hz;
            vox_mm(B.geom, g.spacing, vi[q], vj[q], vk[q], px, py, pz);
            image_to_head(B.geom, px, py, pz, hx, hy, hz);
            o.X[q] = hx;
            o.Y[q] = hy;
            o.GX[q] = 1.0f - hz / B.geom.vsadx;
            o.GY[q] = 1.0f - hz / B.geom.vsady;
            const float dx = B.geom.src[0] - px, dy = B.geom.src[1] - py,
                        dz = B.geom.src[2] - pz;
            o.DIST[q] = sqrtf(dx * dx + dy * dy + dz * dz);
            o.WMM[q] = __fmul_rn(__ldg(wetb + vidx[q]), 10.0f);
        } else {
            o.X[q] = o.Y[q] = 0.0f;
            o.GX[q] = o.GY[q] = 1.0f;
            o.DIST[q] = 0.0f;
            o.WMM[q] = INFINITY;
        }
    }
}

__device__ __forceinline__ void tile_voxels(const PlanArgs &A, int *vi, int *vj,
                                            int *vk, bool *valid, int64_t *vidx)
{
    int t = blockIdx.x;
    const int tx = t % A.tiles_x;
    t /= A.tiles_x;
    const int ty = t % A.tiles_y;
    const int tz = t / A.tiles_y;
    const int li = threadIdx.x & 7, lj = (threadIdx.x >> 3) & 7, lk = threadIdx.x >> 6;
#pragma unroll
    for (int q = 0; q < kVpt; ++q) {
        vi[q] = tx * 8 + li;
        vj[q] = ty * 8 + lj;
        vk[q] = tz * 8 + lk + 4 * q;
        valid[q] = vi[q] < A.g.nx && vj[q] < A.g.ny && vk[q] < A.g.nz;
        vidx[q] = valid[q] ? vi[q] + (int64_t)A.g.nx * (vj[q] + (int64_t)A.g.ny * vk[q]) : 0;
    }
}

__device__ __forceinline__ void stage_lut(const PbBeam &B, int e, float *s_dep,
                                          float *s_sig, float *s_idd)
{
    const size_t o = (size_t)e * B.lut_len;
    for (int x = threadIdx.x; x < B.lut_len; x += kThreads) {
        s_dep[x] = __ldg(B.depths_dev + o + x);
        s_sig[x] = __ldg(B.sigmas_dev + o + x);
        s_idd[x] = __ldg(B.idds_dev + o + x);
    }
}

// ------------------------------------------------------------------ forward

__global__ void __launch_bounds__(kThreads, 2)
k_dose(const __grid_constant__ PlanArgs A, const float *__restrict__ wet,
       const PbLayer *__restrict__ layers, const float4 *__restrict__ geo,
       const float *__restrict__ mu, float *__restrict__ dose,
       float *__restrict__ beam_dose)
{
    __shared__ float s_dep[PB_MAX_LUT_LEN], s_sig[PB_MAX_LUT_LEN], s_idd[PB_MAX_LUT_LEN];
    __shared__ SpotRec s_spot[kThreads];
    __shared__ float s_red[kWarps][9];
    __shared__ int s_wcount[kWarps];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int vi[kVpt], vj[kVpt], vk[kVpt];
    bool valid[kVpt];
    int64_t vidx[kVpt];
    tile_voxels(A, vi, vj, vk, valid, vidx);
    const int64_t V = (int64_t)A.g.nx * A.g.ny * A.g.nz;

    float tot_s[kVpt], tot_c[kVpt];
#pragma unroll
    for (int q = 0; q < kVpt; ++q) tot_s[q] = tot_c[q] = 0.0f;

    for (int b = 0; b < A.n_beams; ++b) {
        const PbBeam &B = A.beams[b];
        VoxelGeom vg;
        beam_voxel_geom(A.g, B, wet + b * V, vi, vj, vk, valid, vidx, vg);
        const TileBounds tb = tile_bounds(vg.X, vg.Y, vg.GX, vg.GY, valid, s_red);
        float bs_s[kVpt], bs_c[kVpt];
#pragma unroll
        for (int q = 0; q < kVpt; ++q) bs_s[q] = bs_c[q] = 0.0f;

        for (int l = 0; l < B.n_layers; ++l) {
            const PbLayer L = layers[B.layer_start + l];
            const float cut = __fmul_rn(1.1f, L.r80);
            bool act[kVpt];
            bool any = false;
#pragma unroll
            for (int q = 0; q < kVpt; ++q) {
                act[q] = valid[q] && !(vg.WMM[q] > cut);
                any |= act[q];
            }
            if (!__syncthreads_or(any)) continue;
            stage_lut(B, L.energy_id, s_dep, s_sig, s_idd);
            __syncthreads();
            const float *cabc = B.dvp_dev + (size_t)B.dvp_len * L.energy_id + 2;
            const float ca = __ldg(cabc), cb = __ldg(cabc + 1), cc = __ldg(cabc + 2);
            float pf[kVpt], hf[kVpt], ps2[kVpt], hs2[kVpt];
            float hmax = -INFINITY;
#pragma unroll
            for (int q = 0; q < kVpt; ++q) {
                if (act[q]) {
                    layer_params(vg.WMM[q], vg.DIST[q], L.r80, s_dep, s_sig, s_idd,
                                 B.lut_len, ca, cb, cc, pf[q], hf[q], ps2[q], hs2[q]);
                    hmax = fmaxf(hmax, hs2[q]);
                } else {
                    pf[q] = hf[q] = ps2[q] = hs2[q] = 0.0f;
                }
            }
            const float nhs = -block_max_slot8(hmax, s_red);

            float accp[kVpt], acch[kVpt];
#pragma unroll
            for (int q = 0; q < kVpt; ++q) accp[q] = acch[q] = 0.0f;
            const int s0 = B.spot_start + L.spot_start;
            for (int base = 0; base < L.n_spots; base += kThreads) {
                const int si = base + threadIdx.x;
                bool keep = false;
                float4 ga = make_float4(0.f, 0.f, 0.f, 0.f), gb = ga;
                if (si < L.n_spots) {
                    ga = __ldg(geo + 2 * (int64_t)(s0 + si));
                    gb = __ldg(geo + 2 * (int64_t)(s0 + si) + 1);
                    keep = cull_keep(ga.x, ga.y, gb.y, tb, nhs);
                }
                const unsigned m = __ballot_sync(0xffffffffu, keep);
                if (lane == 0) s_wcount[warp] = __popc(m);
                __syncthreads();
                int off = 0, total = 0;
#pragma unroll
                for (int w = 0; w < kWarps; ++w) {
                    const int c = s_wcount[w];
                    off += (w < warp) ? c : 0;
                    total += c;
                }
                if (keep) {
                    const int pos = off + __popc(m & ((1u << lane) - 1u));
                    SpotRec r;
                    r.a = make_float4(-ga.x, -ga.y, ga.z, -ga.w);
                    r.b = make_float4(-gb.x, gb.y, __ldg(mu + s0 + si), 0.0f);
                    s_spot[pos] = r;
                }
                __syncthreads();
                for (int c = 0; c < total; ++c) {
                    const SpotRec r = s_spot[c];
#pragma unroll
                    for (int q = 0; q < kVpt; ++q) {
                        const float ax = fmaf(r.a.x, vg.GX[q], vg.X[q]);
                        const float ay = fmaf(r.a.y, vg.GY[q], vg.Y[q]);
                        const float cz = fmaf(r.a.z, vg.Y[q], fmaf(r.a.w, vg.X[q], r.b.x));
                        const float S = fmaf(ax, ax, fmaf(ay, ay, cz * cz));
                        const float qq = S * r.b.y;
                        accp[q] = fmaf(r.b.z, ex2(ps2[q] * qq), accp[q]);
                        acch[q] = fmaf(r.b.z, ex2(hs2[q] * qq), acch[q]);
                    }
                }
                __syncthreads();
            }
#pragma unroll
            for (int q = 0; q < kVpt; ++q) {
                if (act[q]) {
                    const float ld = fmaf(pf[q], accp[q], hf[q] * acch[q]);
                    neumaier(bs_s[q], bs_c[q], ld);
                    neumaier(tot_s[q], tot_c[q], ld);
                }
            }
        }
        if (beam_dose) {
#pragma unroll
            for (int q = 0; q < kVpt; ++q)
                if (valid[q]) beam_dose[b * V + vidx[q]] = (bs_s[q] + bs_c[q]) * A.scale;
        }
        __syncthreads();  // s_red is rewritten by the next beam's tile_bounds
    }
#pragma unroll
    for (int q = 0; q < kVpt; ++q)
        if (valid[q]) dose[vidx[q]] = (tot_s[q] + tot_c[q]) * A.scale;
}

// ------------------------------------------------------------------ adjoint

__global__ void __launch_bounds__(kThreads, 2)
k_adjoint(const __grid_constant__ PlanArgs A, const float *__restrict__ wet,
          const PbLayer *__restrict__ layers, const float4 *__restrict__ geo,
          const float *__restrict__ wfield, float *__restrict__ grad)
{
    __shared__ float s_dep[PB_MAX_LUT_LEN], s_sig[PB_MAX_LUT_LEN], s_idd[PB_MAX_LUT_LEN];
    __shared__ VoxRec s_vox[kThreads * kVpt];
    __shared__ SpotRec s_spot[kThreads];
    __shared__ float s_red[kWarps][9];
    __shared__ int s_wcount[kWarps * kVpt];
    __shared__ int s_scount[kWarps];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int vi[kVpt], vj[kVpt], vk[kVpt];
    bool valid[kVpt];
    int64_t vidx[kVpt];
    tile_voxels(A, vi, vj, vk, valid, vidx);
    const int64_t V = (int64_t)A.g.nx * A.g.ny * A.g.nz;
    float wv[kVpt];
    bool anyw = false;
#pragma unroll
    for (int q = 0; q < kVpt; ++q) {
        wv[q] = valid[q] ? __ldg(wfield + vidx[q]) * A.scale : 0.0f;
        anyw |= (wv[q] != 0.0f);
    }
    if (!__syncthreads_or(anyw)) return;

    for (int b = 0; b < A.n_beams; ++b) {
        const PbBeam &B = A.beams[b];
        VoxelGeom vg;
        beam_voxel_geom(A.g, B, wet + b * V, vi, vj, vk, valid, vidx, vg);
        const TileBounds tb = tile_bounds(vg.X, vg.Y, vg.GX, vg.GY, valid, s_red);

        for (int l = 0; l < B.n_layers; ++l) {
            const PbLayer L = layers[B.layer_start + l];
            const float cut = __fmul_rn(1.1f, L.r80);
            bool act[kVpt];
            bool any = false;
#pragma unroll
            for (int q = 0; q < kVpt; ++q) {
                act[q] = valid[q] && wv[q] != 0.0f && !(vg.WMM[q] > cut);
                any |= act[q];
            }
            if (!__syncthreads_or(any)) continue;
            stage_lut(B, L.energy_id, s_dep, s_sig, s_idd);
            __syncthreads();
            const float *cabc = B.dvp_dev + (size_t)B.dvp_len * L.energy_id + 2;
            const float ca = __ldg(cabc), cb = __ldg(cabc + 1), cc = __ldg(cabc + 2);
            float hmax = -INFINITY;
            unsigned mq[kVpt];
            VoxRec rec[kVpt];
#pragma unroll
            for (int q = 0; q < kVpt; ++q) {
                if (act[q]) {
                    float pf, hf, ps2, hs2;
                    layer_params(vg.WMM[q], vg.DIST[q], L.r80, s_dep, s_sig, s_idd,
                                 B.lut_len, ca, cb, cc, pf, hf, ps2, hs2);
                    hmax = fmaxf(hmax, hs2);
                    rec[q].a = make_float4(vg.X[q], vg.Y[q], vg.GX[q], vg.GY[q]);
                    rec[q].b = make_float4(ps2, hs2, wv[q] * pf, wv[q] * hf);
                }
                mq[q] = __ballot_sync(0xffffffffu, act[q]);
                if (lane == 0) s_wcount[q * kWarps + warp] = __popc(mq[q]);
            }
            const float nhs = -block_max_slot8(hmax, s_red);  // includes a barrier
            // Compact the active voxels' records: order q, warp, lane.
            int nact = 0;
#pragma unroll
            for (int q = 0; q < kVpt; ++q) {
                int pos = 0;
                for (int w = 0; w < kWarps; ++w) {
                    const int c = s_wcount[q * kWarps + w];
                    if (w == warp) pos = nact + __popc(mq[q] & ((1u << lane) - 1u));
                    nact += c;
                }
                if (act[q]) s_vox[pos] = rec[q];
            }

            const int s0 = B.spot_start + L.spot_start;
            for (int base = 0; base < L.n_spots; base += kThreads) {
                const int si = base + threadIdx.x;
                bool keep = false;
                float4 ga = make_float4(0.f, 0.f, 0.f, 0.f), gb = ga;
                if (si < L.n_spots) {
                    ga = __ldg(geo + 2 * (int64_t)(s0 + si));
                    gb = __ldg(geo + 2 * (int64_t)(s0 + si) + 1);
                    keep = cull_keep(ga.x, ga.y, gb.y, tb, nhs);
                }
                const unsigned m = __ballot_sync(0xffffffffu, keep);
                if (lane == 0) s_scount[warp] = __popc(m);
                __syncthreads();
                int off = 0, total = 0;
#pragma unroll
                for (int w = 0; w < kWarps; ++w) {
                    const int c = s_scount[w];
                    off += (w < warp) ? c : 0;
                    total += c;
                }
                if (keep) {
                    const int p = off + __popc(m & ((1u << lane) - 1u));
                    SpotRec r;
                    r.a = make_float4(-ga.x, -ga.y, ga.z, -ga.w);
                    r.b = make_float4(-gb.x, gb.y, __int_as_float(s0 + si), 0.0f);
                    s_spot[p] = r;
                }
                __syncthreads();
                if ((int)threadIdx.x < total) {
                    const SpotRec r = s_spot[threadIdx.x];
                    float acc = 0.0f;
                    for (int c = 0; c < nact; ++c) {
                        const VoxRec v = s_vox[c];
                        const float ax = fmaf(r.a.x, v.a.z, v.a.x);
                        const float ay = fmaf(r.a.y, v.a.w, v.a.y);
                        const float cz = fmaf(r.a.z, v.a.y, fmaf(r.a.w, v.a.x, r.b.x));
                        const float S = fmaf(ax, ax, fmaf(ay, ay, cz * cz));
                        const float qq = S * r.b.y;
                        acc = fmaf(v.b.z, ex2(v.b.x * qq), acc);
                        acc = fmaf(v.b.w, ex2(v.b.y * qq), acc);
                    }
                    if (acc != 0.0f) atomicAdd(grad + __float_as_int(r.b.z), acc);
                }
                __syncthreads();
            }
        }
        __syncthreads();  // s_red is rewritten by the next beam's tile_bounds
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
        const float d = dose[q] - presc[q];
        const float w = weight[q];
        acc += (double)w * (double)d * (double)d;
        if (resid) resid[q] = 2.0f * w * d;
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
    for (int b = 0; b < n_beams; ++b) A.beams[b] = beams[b];
}

PbStatus launch_dose(const PbGrid &g, const PbBeam *beams, int n_beams,
                     const float *wet, const PbLayer *layers, const float *geo,
                     const float *mu, float scale, float *dose, float *beam_dose,
                     cudaStream_t st)
{
    PlanArgs A;
    fill_args(A, g, beams, n_beams, scale);
    const int64_t tiles = (int64_t)A.tiles_x * A.tiles_y * A.tiles_z;
    k_dose<<<(unsigned)tiles, kThreads, 0, st>>>(A, wet, layers,
                                                 reinterpret_cast<const float4 *>(geo), mu,
                                                 dose, beam_dose);
    return check_launch("k_dose");
}

PbStatus launch_adjoint(const PbGrid &g, const PbBeam *beams, int n_beams,
                        const float *wet, const PbLayer *layers, const float *geo,
                        const float *w, float scale, float *grad, cudaStream_t st)
{
    PlanArgs A;
    fill_args(A, g, beams, n_beams, scale);
    int total_spots = 0;
    for (int b = 0; b < n_beams; ++b) {
        const int e = beams[b].spot_start + beams[b].n_spots;
        if (e > total_spots) total_spots = e;
    }
    PbStatus s = check_cuda(cudaMemsetAsync(grad, 0, sizeof(float) * (size_t)total_spots, st),
                            "cudaMemsetAsync(grad)");
    if (s != PB_OK) return s;
    const int64_t tiles = (int64_t)A.tiles_x * A.tiles_y * A.tiles_z;
    k_adjoint<<<(unsigned)tiles, kThreads, 0, st>>>(A, wet, layers,
                                                    reinterpret_cast<const float4 *>(geo), w,
                                                    grad);
    return check_launch("k_adjoint");
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
