// The hex8 element matrix in its Hadamard basis: the algebra shared by the
// fine operator sweeps (kernels_hsweep.cu) and the element energy pass
// (kernels_design.cu).
//
// With H the 2x2 Hadamard matrix and T = H (x) H (x) H acting on the eight
// corners of an element (corner (cx, cy, cz), mode (px, py, pz), sign
// (-1)^(px cx + py cy + pz cz)), S = T Ke T' of an isotropic cube element has
// 45 non-zeros in a fixed pattern of eight constants, and
//   Ke u = T' S T u / 64,   u' Ke u = (T u)' S (T u) / 64.
// The host derives the constants and checks the pattern (hadamard_ke).
#pragma once

#include "gputo_internal.h"

namespace gputo {

template <typename T> struct HC {
    T a, bc, c, de, e, f, g, h;   // S constants / 64: a, b - c, c, d - e, e, f, g, h
};

// Arithmetic shared by the scalar kernels and the paired FP32 sweep, which
// runs two elements per lane as float2 (element 2l in .x, 2l + 1 in .y):
// each operation on a pair is one paired instruction with the same rounding
// as the scalar one (a - b as fma(-1, b, a) is exact before rounding).
__device__ __forceinline__ float hfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double hfma(double a, double b, double c) { return ::fma(a, b, c); }
__device__ __forceinline__ float2 hfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 operator-(float2 a, float2 b) { return __ffma2_rn(make_float2(-1.f, -1.f), b, a); }
__device__ __forceinline__ float2 operator*(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 operator-(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float hmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double hmul(double a, double b) { return __dmul_rn(a, b); }
template <typename T> __device__ __forceinline__ T hzero() { return T(0); }
template <> __device__ __forceinline__ float2 hzero<float2>() { return make_float2(0.f, 0.f); }
// A constant in the arithmetic type (both halves of a pair).
template <typename T> __device__ __forceinline__ T hconst(double v) { return (T)v; }
template <> __device__ __forceinline__ float2 hconst<float2>(double v) { return make_float2((float)v, (float)v); }
inline HC<float2> pair_hc(const HC<float> &k)
{
    auto p = [](float v) { return make_float2(v, v); };
    return HC<float2>{p(k.a), p(k.bc), p(k.c), p(k.de), p(k.e), p(k.f), p(k.g), p(k.h)};
}

// The eight constants as the kernels use them (divided by 64).
template <typename T>
inline HC<T> make_hc(const HadamardKe &hk)
{
    HC<T> hc;
    hc.a = (T)(hk.c[0] / 64.0);
    hc.bc = (T)((hk.c[1] - hk.c[2]) / 64.0);
    hc.c = (T)(hk.c[2] / 64.0);
    hc.de = (T)((hk.c[3] - hk.c[4]) / 64.0);
    hc.e = (T)(hk.c[4] / 64.0);
    hc.f = (T)(hk.c[5] / 64.0);
    hc.g = (T)(hk.c[6] / 64.0);
    hc.h = (T)(hk.c[7] / 64.0);
    return hc;
}

// Face values are stored at [c 4 + d]: corner (or mode) c = 2 cy + cz (2 py +
// pz), component d < 3; slot 3 of each group is unused.  The x and y
// components of a group sit in an aligned register pair, so FP32 code works
// on them with paired instructions.
constexpr int HF = 16;

// (y, z) butterflies of one face: corners -> modes; applied twice it
// multiplies by 4.
template <typename T>
__device__ __forceinline__ void face_h(T (&x)[HF])
{
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const T u00 = x[d], u01 = x[4 + d], u10 = x[8 + d], u11 = x[12 + d];
        const T s0 = u00 + u10, d0 = u00 - u10, s1 = u01 + u11, d1 = u01 - u11;
        x[d] = s0 + s1;
        x[4 + d] = s0 - s1;
        x[8 + d] = d0 + d1;
        x[12 + d] = d0 - d1;
    }
}

__device__ __forceinline__ float2 f2(const float (&x)[HF], int i) { return make_float2(x[i], x[i + 1]); }
__device__ __forceinline__ void f2set(float (&x)[HF], int i, float2 v)
{
    x[i] = v.x;
    x[i + 1] = v.y;
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(make_float2(-1.f, -1.f), b, a); }

// FP32: components x, y of each group with paired adds, z alone.
template <>
__device__ __forceinline__ void face_h<float>(float (&x)[HF])
{
    const float2 u00 = f2(x, 0), u01 = f2(x, 4), u10 = f2(x, 8), u11 = f2(x, 12);
    const float2 s0 = __fadd2_rn(u00, u10), d0 = sub2(u00, u10), s1 = __fadd2_rn(u01, u11), d1 = sub2(u01, u11);
    f2set(x, 0, __fadd2_rn(s0, s1));
    f2set(x, 4, sub2(s0, s1));
    f2set(x, 8, __fadd2_rn(d0, d1));
    f2set(x, 12, sub2(d0, d1));
    const float z00 = x[2], z01 = x[6], z10 = x[10], z11 = x[14];
    const float zs0 = __fadd_rn(z00, z10), zd0 = __fsub_rn(z00, z10), zs1 = __fadd_rn(z01, z11),
                zd1 = __fsub_rn(z01, z11);
    x[2] = __fadd_rn(zs0, zs1);
    x[6] = __fsub_rn(zs0, zs1);
    x[10] = __fadd_rn(zd0, zd1);
    x[14] = __fsub_rn(zd0, zd1);
}

// The S step of one element, v -> w = cx S v / 64 (the mode-(0,0,0) rows
// are zero).  Mode m = 4 px + 2 py + pz with px selecting v0 / v1 and
// (py, pz, d) the index (2 py + pz) 4 + d.
template <typename T>
__device__ __forceinline__ void element_s(const T (&v0)[HF], const T (&v1)[HF], T cx, const HC<T> &k, T (&w0)[HF],
                                          T (&w1)[HF])
{
    const T ka = k.a * cx, kbc = k.bc * cx, kc = k.c * cx, kde = k.de * cx, ke = k.e * cx, kf = k.f * cx,
            kg = k.g * cx, kh = k.h * cx;
    T t;
    w0[0] = w0[1] = w0[2] = hzero<T>();   // mode (0,0,0): rigid translation
    // a [1 1; 1 1]: {(m1,x),(m4,z)}, {(m1,y),(m2,z)}, {(m2,x),(m4,y)}
    t = ka * (v0[4] + v1[2]);
    w0[4] = t, w1[2] = t;
    t = ka * (v0[5] + v0[10]);
    w0[5] = t, w0[10] = t;
    t = ka * (v0[8] + v1[1]);
    w0[8] = t, w1[1] = t;
    // (b - c) I + c 11': {(m1,z),(m2,y),(m4,x)}
    t = kc * (v0[6] + v0[9] + v1[0]);
    w0[6] = hfma(kbc, v0[6], t);
    w0[9] = hfma(kbc, v0[9], t);
    w1[0] = hfma(kbc, v1[0], t);
    // (d - e) I + e 11': {(m3,x),(m5,y),(m6,z)}
    t = ke * (v0[12] + v1[5] + v1[10]);
    w0[12] = hfma(kde, v0[12], t);
    w1[5] = hfma(kde, v1[5], t);
    w1[10] = hfma(kde, v1[10], t);
    // [f g; g f]: {(m3,y),(m5,x)}, {(m3,z),(m6,x)}, {(m5,z),(m6,y)}
    w0[13] = hfma(kf, v0[13], kg * v1[4]);
    w1[4] = hfma(kf, v1[4], kg * v0[13]);
    w0[14] = hfma(kf, v0[14], kg * v1[8]);
    w1[8] = hfma(kf, v1[8], kg * v0[14]);
    w1[6] = hfma(kf, v1[6], kg * v1[9]);
    w1[9] = hfma(kf, v1[9], kg * v1[6]);
    // h I on mode (1,1,1)
    w1[12] = kh * v1[12];
    w1[13] = kh * v1[13];
    w1[14] = kh * v1[14];
}


// u_e' Ke u_e of one element from its transformed front (x = 0) and back
// (x = 1) faces: v = T u, w = S v / 64, energy = v . w.
template <typename T>
__device__ __forceinline__ T element_energy_h(const T (&Fp)[HF], const T (&Fn)[HF], const HC<T> &k)
{
    T v0[HF], v1[HF], w0[HF], w1[HF];
#pragma unroll
    for (int q = 0; q < HF; ++q)
        if ((q & 3) != 3) {
            v0[q] = Fp[q] + Fn[q];
            v1[q] = Fp[q] - Fn[q];
        }
    element_s(v0, v1, T(1), k, w0, w1);
    T s = T(0);
#pragma unroll
    for (int q = 0; q < HF; ++q)
        if ((q & 3) != 3) {
            s = fma(v0[q], w0[q], s);
            s = fma(v1[q], w1[q], s);
        }
    return s;
}

}  // namespace gputo
