// Device arithmetic of the PPF registration path.
//
// Every function here restates a piece of the reference's arithmetic
// (src/cuda/kernel.cu) with the SAME floating-point operation order, because
// the integer outputs of the path (feature keys, alpha bins, cell keys) depend
// on the exact bits of intermediate floats: a one-ulp change moves a bin and
// changes the FNV hash completely.  The kernels that include this header are
// compiled with the reference's arithmetic flags
// (--ftz=true --prec-div=false --prec-sqrt=false, contraction on;
// CMakeLists.txt:71) so that `/`, `sqrtf` and a*b+c sequences round the same
// way.  Matrices are row-major float[4][4] as in the reference.
//
// Two kinds of expressions are written with explicit *_rn intrinsics:
// the float3 arithmetic that the reference performs through out-of-line
// operators in another translation unit (src/cuda/vector_ops.cu:80-103, built
// with separate compilation, so never fused with neighbouring operations).
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

namespace ppf {

// Angle quantum: 2*pi/30 formed in float exactly as include/kernel.h:15-16.
#define PPF_N_ANGLE 30
#define PPF_D_ANGLE ((2.0f * float(CUDART_PI_F)) / float(PPF_N_ANGLE))
// Rotation threshold of the clustering kernel (include/kernel.h:17).
#define PPF_ROT_THRESH (2 * PPF_D_ANGLE)
// FNV-1a offset basis and prime (include/kernel.h:22, src/cuda/kernel.cu:23-30).
#define PPF_FNV_BASIS 2166136261u
#define PPF_FNV_PRIME 16777619u

struct Mat4 {
  float m[4][4];
};

// ---------------------------------------------------------------- hashing --

// FNV-1a over raw bytes, each byte taken as a *signed* char and sign-extended
// before the xor (src/cuda/kernel.cu:23-30).
__device__ __forceinline__ uint32_t fnv1a_word(uint32_t h, uint32_t w) {
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    int8_t c = (int8_t)((w >> (8 * b)) & 0xffu);
    h ^= (uint32_t)(int32_t)c;
    h *= PPF_FNV_PRIME;
  }
  return h;
}

// Key of a discretised feature: hash of the 16 bytes of the float4
// (src/cuda/kernel.cu:460-477); 0 marks "no feature" (NaN distance).
__device__ __forceinline__ uint32_t feature_key(float4 f) {
  if (isnan(f.x)) return 0u;
  uint32_t h = PPF_FNV_BASIS;
  h = fnv1a_word(h, __float_as_uint(f.x));
  h = fnv1a_word(h, __float_as_uint(f.y));
  h = fnv1a_word(h, __float_as_uint(f.z));
  h = fnv1a_word(h, __float_as_uint(f.w));
  return h;
}

// Hash of an int3 cell index (src/cuda/kernel.cu:680,693).
__device__ __forceinline__ uint32_t cell_key(int x, int y, int z) {
  uint32_t h = PPF_FNV_BASIS;
  h = fnv1a_word(h, (uint32_t)x);
  h = fnv1a_word(h, (uint32_t)y);
  h = fnv1a_word(h, (uint32_t)z);
  return h;
}

// ------------------------------------------------------------ vector math --

__device__ __forceinline__ float dot3(float3 a, float3 b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
__device__ __forceinline__ float dot4(float4 a, float4 b) {
  return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
}
__device__ __forceinline__ float norm3(float3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ float norm4(float4 a) { return sqrtf(dot4(a, a)); }

// x rounded down to a multiple of y, as x - fmodf(x, y) (src/cuda/kernel.cu:90-92).
__device__ __forceinline__ float quant_down(float x, float y) { return x - fmodf(x, y); }

// Point pair feature (|d|, angle(n1,d), angle(n2,d), angle(n1,n2))
// (src/cuda/kernel.cu:109-122), then discretised (src/cuda/kernel.cu:94-100).
__device__ __forceinline__ float4 pair_feature(float3 p1, float3 n1, float3 p2, float3 n2,
                                               float d_dist) {
  float3 d;
  d.x = p2.x - p1.x;
  d.y = p2.y - p1.y;
  d.z = p2.z - p1.z;
  float4 f;
  f.x = norm3(d);
  f.y = acosf(dot3(n1, d) / (norm3(n1) * norm3(d)));
  f.z = acosf(dot3(n2, d) / (norm3(n2) * norm3(d)));
  f.w = acosf(dot3(n1, n2) / (norm3(n1) * norm3(n2)));
  f.x = quant_down(f.x, d_dist);
  f.y = quant_down(f.y, PPF_D_ANGLE);
  f.z = quant_down(f.z, PPF_D_ANGLE);
  f.w = quant_down(f.w, PPF_D_ANGLE);
  return f;
}

// -------------------------------------------------------- 4x4 transforms --
// Builders and products with the reference's zero-initialised layouts
// (src/cuda/kernel.cu:32-49,170-223,234-242,254-299).

__device__ __forceinline__ void mat_zero(Mat4& T) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) T.m[i][j] = 0;
}

__device__ __forceinline__ void mat_translation(float3 v, Mat4& T) {
  mat_zero(T);
  T.m[0][0] = 1;
  T.m[1][1] = 1;
  T.m[2][2] = 1;
  T.m[3][3] = 1;
  T.m[0][3] = v.x;
  T.m[1][3] = v.y;
  T.m[2][3] = v.z;
}

__device__ __forceinline__ void mat_rot_x(float th, Mat4& T) {
  mat_zero(T);
  T.m[0][0] = 1;
  T.m[1][1] = cosf(th);
  T.m[2][1] = sinf(th);
  T.m[1][2] = -1 * T.m[2][1];
  T.m[2][2] = T.m[1][1];
  T.m[3][3] = 1;
}

__device__ __forceinline__ void mat_rot_y(float th, Mat4& T) {
  mat_zero(T);
  T.m[0][0] = cosf(th);
  T.m[0][2] = sinf(th);
  T.m[1][1] = 1;
  T.m[2][0] = -1 * T.m[0][2];
  T.m[2][2] = T.m[0][0];
  T.m[3][3] = 1;
}

__device__ __forceinline__ void mat_rot_z(float th, Mat4& T) {
  mat_zero(T);
  T.m[0][0] = cosf(th);
  T.m[1][0] = sinf(th);
  T.m[0][1] = -1 * T.m[1][0];
  T.m[1][1] = T.m[0][0];
  T.m[2][2] = 1;
  T.m[3][3] = 1;
}

// C = A * B, each entry accumulated from 0 over k = 0..3.
__device__ __forceinline__ void mat_mul(const Mat4& A, const Mat4& B, Mat4& C) {
  mat_zero(C);
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int k = 0; k < 4; ++k) C.m[i][j] += A.m[i][k] * B.m[k][j];
}

__device__ __forceinline__ float4 mat_row(const Mat4& A, int i) {
  return make_float4(A.m[i][0], A.m[i][1], A.m[i][2], A.m[i][3]);
}

// Row i of A times the homogeneous point (p, 1).
__device__ __forceinline__ float row_apply(float4 row, float3 p) {
  return dot4(row, make_float4(p.x, p.y, p.z, 1));
}

// Inverse of a rigid transform [R t; 0 1] -> [R' -R't; 0 1]
// (src/cuda/kernel.cu:254-299).
__device__ __forceinline__ void mat_rigid_inverse(const Mat4& T, Mat4& Ti) {
  Ti.m[0][0] = T.m[0][0];
  Ti.m[0][1] = T.m[1][0];
  Ti.m[0][2] = T.m[2][0];
  Ti.m[1][0] = T.m[0][1];
  Ti.m[1][1] = T.m[1][1];
  Ti.m[1][2] = T.m[2][1];
  Ti.m[2][0] = T.m[0][2];
  Ti.m[2][1] = T.m[1][2];
  Ti.m[2][2] = T.m[2][2];
  float3 r0 = make_float3(-Ti.m[0][0], -Ti.m[0][1], -Ti.m[0][2]);
  float3 r1 = make_float3(-Ti.m[1][0], -Ti.m[1][1], -Ti.m[1][2]);
  float3 r2 = make_float3(-Ti.m[2][0], -Ti.m[2][1], -Ti.m[2][2]);
  float3 t = make_float3(T.m[0][3], T.m[1][3], T.m[2][3]);
  Ti.m[0][3] = dot3(r0, t);
  Ti.m[1][3] = dot3(r1, t);
  Ti.m[2][3] = dot3(r2, t);
  Ti.m[3][0] = 0;
  Ti.m[3][1] = 0;
  Ti.m[3][2] = 0;
  Ti.m[3][3] = 1;
}

// ------------------------------------------------------ reference frames --
//
// T_g = Rz(-atan2(n'.y, n'.x)) * Ry(atan2(n.z, n.x)) * Trans(-p), with
// n' = Ry * (n, 1): moves p to the origin and turns n onto the +x axis
// (src/cuda/kernel.cu:310-327).  Only rows 1 and 2 of T_g reach the alpha
// angle, because the x coordinate is zeroed there (src/cuda/kernel.cu:338-339).

struct FrameAngles {
  float roty;  // atan2(n.z, n.x)
  float rotz;  // -atan2(n'.y, n'.x)
};

// src/cuda/kernel.cu:352-369 (one half).
__device__ __forceinline__ FrameAngles frame_angles(float3 n) {
  FrameAngles a;
  Mat4 ry;
  a.roty = atan2f(n.z, n.x);
  mat_rot_y(a.roty, ry);
  float4 nt = make_float4(dot4(mat_row(ry, 0), make_float4(n.x, n.y, n.z, 1)),
                          dot4(mat_row(ry, 1), make_float4(n.x, n.y, n.z, 1)), 0.f, 0.f);
  a.rotz = -1 * atan2f(nt.y, nt.x);
  return a;
}

// Full frame transform from precomputed angles (src/cuda/kernel.cu:382-395).
__device__ __forceinline__ void frame_from_angles(float3 p, float roty, float rotz, Mat4& Tg) {
  Mat4 tr, ry, rz, tmp;
  float3 np = make_float3(-1 * p.x, -1 * p.y, -1 * p.z);
  mat_translation(np, tr);
  mat_rot_y(roty, ry);
  mat_rot_z(rotz, rz);
  mat_mul(rz, ry, tmp);
  mat_mul(tmp, tr, Tg);
}

// The frame as trans_model_scene builds it (src/cuda/kernel.cu:310-318):
// identical values to frame_from_angles(p, frame_angles(n)).
__device__ __forceinline__ void frame_of(float3 p, float3 n, Mat4& Tg) {
  Mat4 tr, ry, rz, tmp;
  float3 np = make_float3(-1 * p.x, -1 * p.y, -1 * p.z);
  mat_translation(np, tr);
  mat_rot_y(atan2f(n.z, n.x), ry);
  float4 h = make_float4(n.x, n.y, n.z, 1);
  float4 nt;
  nt.x = dot4(mat_row(ry, 0), h);
  nt.y = dot4(mat_row(ry, 1), h);
  mat_rot_z(-1 * atan2f(nt.y, nt.x), rz);
  mat_mul(rz, ry, tmp);
  mat_mul(tmp, tr, Tg);
}

// Rows 1 and 2 of a frame: what the alpha computation needs.
struct FrameYZ {
  float4 r1, r2;
};

__device__ __forceinline__ FrameYZ frame_yz(float3 p, float3 n) {
  Mat4 Tg;
  frame_of(p, n, Tg);
  FrameYZ f;
  f.r1 = mat_row(Tg, 1);
  f.r2 = mat_row(Tg, 2);
  return f;
}

// (y, z) of a point in a frame: u or v of src/cuda/kernel.cu:330-336.
__device__ __forceinline__ float2 frame_point_yz(const FrameYZ& f, float3 q) {
  return make_float2(row_apply(f.r1, q), row_apply(f.r2, q));
}

// ----------------------------------------------------------- alpha angle --
//
// alpha = atan2(cross(u,v).x, dot(u,v)) with u.x = v.x = 0, then the bin
// lrintf(quant_down(alpha + pi, D) / D) (src/cuda/kernel.cu:338-342).

__device__ __forceinline__ float alpha_angle(float2 u, float2 v) {
  float3 uu = make_float3(0, u.x, u.y);
  float3 vv = make_float3(0, v.x, v.y);
  float cx = uu.y * vv.z - uu.z * vv.y;
  return atan2f(cx, dot3(uu, vv));
}

// Exact alpha bin.  fmodf is exact, so quant_down(x, D) == fl(n*D) with
// n = trunc(x / D) taken in real arithmetic; dividing fl(n*D) by D (an
// approximate division with a few-ulp error) and rounding to the nearest
// integer gives n back for every n <= 31.  n is therefore computed directly:
// the sign of x - k*D is exact in one fma.
__device__ __forceinline__ unsigned alpha_bin_of(float alpha) {
  float x = alpha + CUDART_PI_F;
  const float D = PPF_D_ANGLE;
  int n = (int)(x * (1.0f / D));
  if (n < 0) n = 0;
  if (__fmaf_rn(-(float)n, D, x) < 0.f) --n;
  if (__fmaf_rn(-(float)(n + 1), D, x) >= 0.f) ++n;
  // x is in [0, 2pi] for every finite alpha, so n is in [0, 30]; a NaN alpha
  // (NaN normals) is kept inside the accumulator.
  n = n < 0 ? 0 : (n > PPF_N_ANGLE ? PPF_N_ANGLE : n);
  return (unsigned)n;
}

__device__ __forceinline__ unsigned alpha_bin_exact(float2 u, float2 v) {
  return alpha_bin_of(alpha_angle(u, v));
}

// 21-bit fixed-point direction angle of (y, z): round(atan2(z, y) * 2^21 / 2pi)
// mod 2^21, in units of 2pi / 2^21 (3.0e-6 rad).  Error against the exact
// angle of the float vector: 0.5 units of rounding, atan2f's few ulp of pi
// (0.23 units) and the scaling multiply (0.12 units): under 0.9 units.
__device__ __forceinline__ uint32_t angle21(float2 yz) {
  float a = atan2f(yz.y, yz.x);  // [-pi, pi]
  float s = a * (2097152.0f / (2.0f * CUDART_PI_F));
  int q = __float2int_rn(s);
  return (uint32_t)q & 0x1fffffu;
}

// Fast alpha bin from the 21-bit angles beta_m of u (model) and beta_s of v
// (scene): alpha + pi = beta_s - beta_m + 2^20 units, bin = floor(30 x /
// 2^21).  The reference's alpha + pi differs from the exact angle difference
// of the float vectors by at most ~1.5e-6 rad (0.5 units: rounding of the
// cross and dot products, atan2f's bound, the add of pi), and the two 21-bit
// angles add under 1.8 units, so a vote within PPF_BIN_MARGIN_UNITS of a bin
// edge (including the wrap at 0 / 2pi) is ambiguous and takes the exact path.
#define PPF_BIN_MARGIN_UNITS 6
#define PPF_ANGLE_BITS 21

// --------------------------------------------------------------- poses --

// Pose of a vote: T = inv(T_s_g) * Rx(bin*D - pi) * T_m_g
// (src/cuda/kernel.cu:372-401), row-major into T[16].
__device__ __forceinline__ void vote_pose(unsigned bin, float3 mr, FrameAngles ma, float3 sr,
                                          FrameAngles sa, float* out) {
  Mat4 Tm, Ts, rx, Tsi, tmp, T;
  frame_from_angles(mr, ma.roty, ma.rotz, Tm);
  frame_from_angles(sr, sa.roty, sa.rotz, Ts);
  mat_rot_x(bin * PPF_D_ANGLE - CUDART_PI_F, rx);
  mat_rigid_inverse(Ts, Tsi);
  mat_mul(Tsi, rx, tmp);
  mat_mul(tmp, Tm, T);
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) out[i * 4 + j] = T.m[i][j];
}

// Quaternion (w, x, y, z) of a rotation matrix via the copysign formula,
// normalised by sqrt(|q|) as the reference does (src/cuda/kernel.cu:128-144).
__device__ __forceinline__ float4 pose_quaternion(const float* T) {
  float t, r;
  float4 q;
  t = T[0] + T[5] + T[10];
  r = sqrtf(1 + t);
  q.x = 0.5f * r;
  q.y = copysignf(0.5f * sqrtf(1 + T[0] - T[5] - T[10]), T[9] - T[6]);
  q.z = copysignf(0.5f * sqrtf(1 - T[0] + T[5] - T[10]), T[2] - T[8]);
  q.w = copysignf(0.5f * sqrtf(1 - T[0] - T[5] + T[10]), T[4] - T[1]);
  float n = sqrtf(norm4(q));
  q.x /= n;
  q.y /= n;
  q.z /= n;
  q.w /= n;
  return q;
}

// Cell of a translation: truncation toward zero of (x - fmod(x, d)) / d
// (src/cuda/kernel.cu:675-678).
__device__ __forceinline__ int3 trans_cell(float3 t, float d) {
  float3 q;
  q.x = quant_down(t.x, d);
  q.y = quant_down(t.y, d);
  q.z = quant_down(t.z, d);
  int3 c;
  c.x = (int)(q.x / d);
  c.y = (int)(q.y / d);
  c.z = (int)(q.z / d);
  return c;
}

// float3 operators of the reference are out-of-line (no contraction with
// their neighbours); these keep each product and sum separately rounded.
__device__ __forceinline__ float3 v3_scale(float a, float3 v) {
  return make_float3(__fmul_rn(a, v.x), __fmul_rn(a, v.y), __fmul_rn(a, v.z));
}
__device__ __forceinline__ float3 v3_add(float3 a, float3 b) {
  return make_float3(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z));
}
__device__ __forceinline__ float3 v3_sub(float3 a, float3 b) {
  return make_float3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z));
}

}  // namespace ppf
