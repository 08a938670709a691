// pb_device.cuh -- device helpers shared by the pencil-beam kernels.
//
// Decision arithmetic (voxel positions, sample positions, frame rotations,
// nearest-voxel rounding) is written with explicit round-to-nearest
// intrinsics so that no multiply-add is contracted: the discrete decisions
// then follow one fixed FP32 operation order, the one the CPU oracle uses.
// The operation order itself follows the reference:
//   voxel <-> mm             DoseCUDA/dose_kernels/CudaClasses.cuh:100-116
//   image -> head (BEV)      CudaClasses.cu:65-95
//   head -> image            CudaClasses.cu:97-126
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/pb_b200.h"

namespace pb {

constexpr float kLog2e = 1.4426950408889634f;
constexpr float kTwoPi = 6.283185307179586f;

// Beams of one launch, passed by value as a kernel parameter.
struct BeamGeomSet {
    PbBeamGeom b[PB_MAX_BEAMS];
};

// Voxel index -> mm relative to the isocentre, i*s - iso: the reference's
// expression (CudaClasses.cuh:106-110) as its compiler contracts it, one
// fused multiply-add.
__device__ __forceinline__ void vox_mm(const PbBeamGeom &b, float s, int i,
                                       int j, int k, float &x, float &y,
                                       float &z)
{
    x = __fmaf_rn((float)i, s, -b.iso[0]);
    y = __fmaf_rn((float)j, s, -b.iso[1]);
    z = __fmaf_rn((float)k, s, -b.iso[2]);
}

// Image frame -> beam's-eye (head) frame: couch about y, then gantry about
// z, then the axis swap to the nozzle frame (beam travels toward -z).
__device__ __forceinline__ void image_to_head(const PbBeamGeom &b, float px,
                                              float py, float pz, float &hx,
                                              float &hy, float &hz)
{
    float sx = -b.sinta, cx = b.costa;
    const float xt = __fadd_rn(__fmul_rn(px, cx), __fmul_rn(pz, sx));
    const float yt = py;
    const float zt = __fadd_rn(__fmul_rn(-px, sx), __fmul_rn(pz, cx));
    sx = -b.singa;
    cx = b.cosga;
    const float xg = __fsub_rn(__fmul_rn(xt, cx), __fmul_rn(yt, sx));
    const float yg = __fadd_rn(__fmul_rn(xt, sx), __fmul_rn(yt, cx));
    hx = -xg;
    hy = zt;
    hz = yg;
}

__device__ __forceinline__ void head_to_image(const PbBeamGeom &b, float hx,
                                              float hy, float hz, float &px,
                                              float &py, float &pz)
{
    const float xz = -hx, yz = hz, zz = hy;
    float sx = b.singa, cx = b.cosga;
    const float xg = __fsub_rn(__fmul_rn(xz, cx), __fmul_rn(yz, sx));
    const float yg = __fadd_rn(__fmul_rn(xz, sx), __fmul_rn(yz, cx));
    const float zg = zz;
    sx = b.sinta;
    cx = b.costa;
    px = __fadd_rn(__fmul_rn(xg, cx), __fmul_rn(zg, sx));
    py = yg;
    pz = __fadd_rn(__fmul_rn(-xg, sx), __fmul_rn(zg, cx));
}

// The two rotations as the reference's compiled code evaluates them
// (CudaClasses.cu:65-126): its compiler contracts each a*b + c*d into one
// fused multiply-add and a rounded product -- in the image -> head rotation
// the second product is fused, in the head -> image rotation the first.
// The smoothing's half-voxel ties depend on these last bits (established
// against the reference module's output on oblique beams).
__device__ __forceinline__ void image_to_head_ref(const PbBeamGeom &b, float px,
                                                  float py, float pz, float &hx,
                                                  float &hy, float &hz)
{
    float sx = -b.sinta, cx = b.costa;
    const float xt = __fmaf_rn(pz, sx, __fmul_rn(px, cx));
    const float yt = py;
    const float zt = __fmaf_rn(pz, cx, __fmul_rn(-px, sx));
    sx = -b.singa;
    cx = b.cosga;
    const float xg = __fmaf_rn(-yt, sx, __fmul_rn(xt, cx));
    const float yg = __fmaf_rn(yt, cx, __fmul_rn(xt, sx));
    hx = -xg;
    hy = zt;
    hz = yg;
}

__device__ __forceinline__ void head_to_image_ref(const PbBeamGeom &b, float hx,
                                                  float hy, float hz, float &px,
                                                  float &py, float &pz)
{
    const float xz = -hx, yz = hz, zz = hy;
    float sx = b.singa, cx = b.cosga;
    const float xg = __fmaf_rn(xz, cx, __fmul_rn(-yz, sx));
    const float yg = __fmaf_rn(xz, sx, __fmul_rn(yz, cx));
    const float zg = zz;
    sx = b.sinta;
    cx = b.costa;
    px = __fmaf_rn(xg, cx, __fmul_rn(zg, sx));
    py = yg;
    pz = __fmaf_rn(-xg, sx, __fmul_rn(zg, cx));
}

// Unit vector from a voxel toward the source: FP32 difference, FP64 norm,
// one rounding to FP32.
__device__ __forceinline__ void unit_to_source(const PbBeamGeom &b, float px,
                                               float py, float pz, float &ux,
                                               float &uy, float &uz)
{
    const float d0 = __fsub_rn(b.src[0], px);
    const float d1 = __fsub_rn(b.src[1], py);
    const float d2 = __fsub_rn(b.src[2], pz);
    double n2 = __dadd_rn(__dmul_rn((double)d0, (double)d0),
                          __dmul_rn((double)d1, (double)d1));
    n2 = __dadd_rn(n2, __dmul_rn((double)d2, (double)d2));
    const double inv = __ddiv_rn(1.0, __dsqrt_rn(n2));
    ux = __double2float_rn(__dmul_rn((double)d0, inv));
    uy = __double2float_rn(__dmul_rn((double)d1, inv));
    uz = __double2float_rn(__dmul_rn((double)d2, inv));
}

// 2^x on the SFU (PTX ex2.approx.ftz.f32).
__device__ __forceinline__ float ex2(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float warp_min(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ float warp_max(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

}  // namespace pb
