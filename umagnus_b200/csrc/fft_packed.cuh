// fft_packed.cuh -- radix-2/4/8 butterflies in packed FP32 arithmetic.
//
// sm_100 executes two lane-wise FP32 operations per instruction
// (add/sub/mul/fma.rn.f32x2 on a 64-bit register pair).  A complex value
// (re, im) is one such pair, so a complex addition is one instruction instead
// of two.  Each lane of a packed operation is an IEEE single-precision
// operation with round-to-nearest: packed code gives the same bits wherever
// it runs, so every instantiation of a transform that uses these butterflies
// agrees bit for bit.  Multiplication by -i, which swaps the components,
// costs a register swap; it is folded into a multiply-add by (1, -1) where
// it feeds an addition.
#pragma once
#include <cuda_runtime.h>

namespace umag {

struct P2 {
    unsigned long long v;
};
__device__ __forceinline__ P2 p2(float2 a) {
    P2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a.x), "f"(a.y));
    return r;
}
__device__ __forceinline__ P2 p2(float x, float y) { return p2(make_float2(x, y)); }
__device__ __forceinline__ float2 f2(P2 a) {
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(a.v));
    return r;
}
__device__ __forceinline__ P2 padd(P2 a, P2 b) { P2 r; asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v)); return r; }
__device__ __forceinline__ P2 psub(P2 a, P2 b) { P2 r; asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v)); return r; }
__device__ __forceinline__ P2 pmul(P2 a, P2 b) { P2 r; asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v)); return r; }
__device__ __forceinline__ P2 pfma(P2 a, P2 b, P2 c) {
    P2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return r;
}
__device__ __forceinline__ P2 pswap(P2 a) {
    P2 r;
    asm("{.reg .f32 lo, hi;\n mov.b64 {lo, hi}, %1;\n mov.b64 %0, {hi, lo};}" : "=l"(r.v) : "l"(a.v));
    return r;
}

// a + (-i) d and a - (-i) d: (-i) d = (d.im, -d.re)
__device__ __forceinline__ void p_pm_mi(P2 a, P2 d, P2& plus, P2& minus) {
    const P2 ds = pswap(d);
    plus = pfma(ds, p2(1.f, -1.f), a);
    minus = pfma(ds, p2(-1.f, 1.f), a);
}
__device__ __forceinline__ void pdft2(P2* v) {
    const P2 a = v[0], b = v[1];
    v[0] = padd(a, b);
    v[1] = psub(a, b);
}
// forward DFT of 4, natural order in and out
__device__ __forceinline__ void pdft4(P2* v) {
    const P2 t0 = padd(v[0], v[2]), t1 = psub(v[0], v[2]), t2 = padd(v[1], v[3]), d = psub(v[1], v[3]);
    v[0] = padd(t0, t2);
    v[2] = psub(t0, t2);
    p_pm_mi(t1, d, v[1], v[3]);
}
// o W8 with W8 = s (1 - i): s ((re + im), (im - re))
__device__ __forceinline__ P2 pw8(P2 o) {
    const float s = 0.70710678118654752440084436210485f;
    return pmul(pfma(pswap(o), p2(1.f, -1.f), o), p2(s, s));
}
// o W8^3 with W8^3 = s (-1 - i): s ((im - re), (-re - im))
__device__ __forceinline__ P2 pw83(P2 o) {
    const float s = 0.70710678118654752440084436210485f;
    return pmul(pfma(pswap(o), p2(1.f, -1.f), pmul(o, p2(-1.f, -1.f))), p2(s, s));
}
// forward DFT of 8 (two DFT4 of the even and odd samples, combined)
__device__ __forceinline__ void pdft8(P2* v) {
    P2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    pdft4(e);
    pdft4(o);
    const P2 o1 = pw8(o[1]), o3 = pw83(o[3]);
    v[0] = padd(e[0], o[0]);
    v[4] = psub(e[0], o[0]);
    v[1] = padd(e[1], o1);
    v[5] = psub(e[1], o1);
    p_pm_mi(e[2], o[2], v[2], v[6]);
    v[3] = padd(e[3], o3);
    v[7] = psub(e[3], o3);
}
// forward DFT of 8 of (u0, u1, u2, u3, 0, 0, 0, 0): the even outputs are the
// DFT4 of u, the odd ones the DFT4 of u_n W8^n
__device__ __forceinline__ void pdft8_zhalf(P2* v) {
    const P2 a = v[0], b = v[1], c = v[2], d = v[3];
    const P2 t0 = padd(a, c), t1 = psub(a, c), t2 = padd(b, d), dd = psub(b, d);
    v[0] = padd(t0, t2);
    v[4] = psub(t0, t2);
    p_pm_mi(t1, dd, v[2], v[6]);
    const P2 b1 = pw8(b), d1 = pw83(d);
    P2 s0, s1;  // a + c W8^2 and a - c W8^2, W8^2 = -i
    p_pm_mi(a, c, s0, s1);
    const P2 s2 = padd(b1, d1), sd = psub(b1, d1);
    v[1] = padd(s0, s2);
    v[5] = psub(s0, s2);
    p_pm_mi(s1, sd, v[3], v[7]);
}
// u w for a twiddle w given as the pairs (w.re, w.re) and (-w.im, w.im):
// u (wr, wr) + swap(u) (-wi, wi)
__device__ __forceinline__ P2 pcmul(P2 u, P2 wrr, P2 wii) { return pfma(pswap(u), wii, pmul(u, wrr)); }

}  // namespace umag
