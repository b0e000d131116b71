// cellmath.cuh -- per-cell field and torque arithmetic.
//
// Every operation uses an explicit round-to-nearest intrinsic (__fadd_rn,
// __fmul_rn, ...), which the compiler never contracts into an FMA.  The
// operand order follows the reference's OpenCL kernels, so these functions
// round exactly like the reference's float32 program compiled without
// -cl-mad-enable (opencl/init.go:175): results are bit-identical to the
// reference kernels given identical inputs.
#pragma once
#include <cstdint>

namespace umag {

struct f3 {
    float x, y, z;
};

__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fd(float a, float b) { return __fdiv_rn(a, b); }

__device__ __forceinline__ float dot3(f3 a, f3 b) { return fa(fa(fm(a.x, b.x), fm(a.y, b.y)), fm(a.z, b.z)); }
__device__ __forceinline__ bool is0(f3 a) { return dot3(a, a) == 0.0f; }
__device__ __forceinline__ f3 cross3(f3 a, f3 b) {
    return f3{fs(fm(a.y, b.z), fm(a.z, b.y)), fs(fm(a.z, b.x), fm(a.x, b.z)), fs(fm(a.x, b.y), fm(a.y, b.x))};
}
__device__ __forceinline__ f3 ld3(const float* __restrict__ x, const float* __restrict__ y,
                                  const float* __restrict__ z, int i) {
    return f3{__ldg(x + i), __ldg(y + i), __ldg(z + i)};
}

// kernels_src/clh/amul.clh:5-7
__device__ __forceinline__ float amul(const float* __restrict__ arr, float mul, int i) {
    return arr == nullptr ? mul : fm(mul, __ldg(arr + i));
}
// kernels_src/clh/amul.clh:19-26
__device__ __forceinline__ float inv_msat(const float* __restrict__ Ms, float mul, int i) {
    float ms = amul(Ms, mul, i);
    return ms == 0.0f ? 0.0f : fd(1.0f, ms);
}

// kernels_src/clh/exchange.clh:5
__device__ __forceinline__ int symidx(int i, int j) {
    return (j <= i) ? ((i * (i + 1)) / 2 + j) : ((j * (j + 1)) / 2 + i);
}

// kernels_src/clh/stencil.clh:13-29: wrap (PBC) or clamp a neighbour index
__device__ __forceinline__ int lclamp(int i, int n, bool pbc) { return pbc ? ((i % n) + n) % n : (i > 0 ? i : 0); }
__device__ __forceinline__ int hclamp(int i, int n, bool pbc) { return pbc ? ((i % n) + n) % n : (i < n - 1 ? i : n - 1); }

struct Mesh3 {
    int Nx, Ny, Nz, pbc;
};

// exchange.cl:5-87 -- returns the exchange contribution before the 1/Ms factor.
__device__ __forceinline__ f3 exchange_sum(const float* __restrict__ mx, const float* __restrict__ my,
                                           const float* __restrict__ mz, const float* __restrict__ aLUT,
                                           const uint8_t* __restrict__ regions, float wx, float wy,
                                           float wz, Mesh3 g, int ix, int iy, int iz, f3 m0, int r0) {
    f3 b{0.f, 0.f, 0.f};
    int nb[6];
    nb[0] = (iz * g.Ny + iy) * g.Nx + lclamp(ix - 1, g.Nx, g.pbc & 1);
    nb[1] = (iz * g.Ny + iy) * g.Nx + hclamp(ix + 1, g.Nx, g.pbc & 1);
    nb[2] = (iz * g.Ny + lclamp(iy - 1, g.Ny, g.pbc & 2)) * g.Nx + ix;
    nb[3] = (iz * g.Ny + hclamp(iy + 1, g.Ny, g.pbc & 2)) * g.Nx + ix;
    nb[4] = (lclamp(iz - 1, g.Nz, g.pbc & 4) * g.Ny + iy) * g.Nx + ix;
    nb[5] = (hclamp(iz + 1, g.Nz, g.pbc & 4) * g.Ny + iy) * g.Nx + ix;
    const int nn = (g.Nz != 1) ? 6 : 4;
#pragma unroll
    for (int k = 0; k < 6; k++) {
        if (k >= nn) break;
        float w = k < 2 ? wx : (k < 4 ? wy : wz);
        f3 mn = ld3(mx, my, mz, nb[k]);
        if (is0(mn)) mn = m0;
        float a = __ldg(aLUT + symidx(r0, __ldg(regions + nb[k])));
        float s = fm(w, a);
        b.x = fa(b.x, fm(s, fs(mn.x, m0.x)));
        b.y = fa(b.y, fm(s, fs(mn.y, m0.y)));
        b.z = fa(b.z, fm(s, fs(mn.z, m0.z)));
    }
    return b;
}

// dmi.cl:95-235 -- exchange + interfacial DMI before the 1/Ms factor.
__device__ __forceinline__ f3 dmi_sum(const float* __restrict__ mx, const float* __restrict__ my,
                                      const float* __restrict__ mz, const float* __restrict__ aLUT,
                                      const float* __restrict__ dLUT, const uint8_t* __restrict__ regions,
                                      float cx, float cy, float cz, Mesh3 g, bool openbc, int ix, int iy,
                                      int iz, f3 m0, int r0) {
    f3 h{0.f, 0.f, 0.f};
#pragma unroll
    for (int d = 0; d < 2; d++) {
        const float c = d == 0 ? cx : cy;
#pragma unroll
        for (int side = -1; side <= 1; side += 2) {
            f3 mn{0.f, 0.f, 0.f};
            int i_;
            bool inside;
            if (d == 0) {
                int xx = side < 0 ? lclamp(ix - 1, g.Nx, g.pbc & 1) : hclamp(ix + 1, g.Nx, g.pbc & 1);
                i_ = (iz * g.Ny + iy) * g.Nx + xx;
                inside = (side < 0 ? ix - 1 >= 0 : ix + 1 < g.Nx) || (g.pbc & 1);
            } else {
                int yy = side < 0 ? lclamp(iy - 1, g.Ny, g.pbc & 2) : hclamp(iy + 1, g.Ny, g.pbc & 2);
                i_ = (iz * g.Ny + yy) * g.Nx + ix;
                inside = (side < 0 ? iy - 1 >= 0 : iy + 1 < g.Ny) || (g.pbc & 2);
            }
            if (inside) mn = ld3(mx, my, mz, i_);
            bool missing = is0(mn);
            int rn = missing ? r0 : __ldg(regions + i_);
            int si = symidx(r0, rn);
            float A = __ldg(aLUT + si);
            float D = __ldg(dLUT + si);
            if (!missing || !openbc) {
                float sc = side < 0 ? -c : c;
                if (missing) {  // Neumann extrapolation of the missing neighbour
                    float q = fm(sc, fd(fm(0.5f, D), A));
                    if (d == 0) {
                        mn.x = fs(m0.x, fm(q, m0.z));
                        mn.y = m0.y;
                        mn.z = fa(m0.z, fm(q, m0.x));
                    } else {
                        mn.x = m0.x;
                        mn.y = fs(m0.y, fm(q, m0.z));
                        mn.z = fa(m0.z, fm(q, m0.y));
                    }
                }
                float s = fd(fm(2.0f, A), fm(c, c));
                h.x = fa(h.x, fm(s, fs(mn.x, m0.x)));
                h.y = fa(h.y, fm(s, fs(mn.y, m0.y)));
                h.z = fa(h.z, fm(s, fs(mn.z, m0.z)));
                float Dc = fd(D, c);
                float tz = side < 0 ? -mn.z : mn.z;
                float tp = d == 0 ? mn.x : mn.y;
                tp = side < 0 ? -tp : tp;
                if (d == 0) h.x = fa(h.x, fm(Dc, tz));
                else h.y = fa(h.y, fm(Dc, tz));
                h.z = fs(h.z, fm(Dc, tp));
            }
        }
    }
    if (g.Nz != 1) {
#pragma unroll
        for (int side = -1; side <= 1; side += 2) {
            int zz = side < 0 ? lclamp(iz - 1, g.Nz, g.pbc & 4) : hclamp(iz + 1, g.Nz, g.pbc & 4);
            int i_ = (zz * g.Ny + iy) * g.Nx + ix;
            f3 mn = ld3(mx, my, mz, i_);
            if (is0(mn)) mn = m0;
            float A = __ldg(aLUT + symidx(r0, __ldg(regions + i_)));
            float s = fd(fm(2.0f, A), fm(cz, cz));
            h.x = fa(h.x, fm(s, fs(mn.x, m0.x)));
            h.y = fa(h.y, fm(s, fs(mn.y, m0.y)));
            h.z = fa(h.z, fm(s, fs(mn.z, m0.z)));
        }
    }
    return h;
}

// Per region-pair DMI coefficients, precomputed on the device with the same
// operations dmi_sum performs per neighbour (so results are bit-identical):
// s[d] = 2A/c_d^2, dc[d] = D/c_d, q[d] = c_d * (0.5 D / A).
struct DmiPairLut {
    const float *sx, *sy, *sz, *dcx, *dcy, *qx, *qy;
};

__device__ __forceinline__ f3 dmi_sum_lut(const float* __restrict__ mx, const float* __restrict__ my,
                                          const float* __restrict__ mz, const DmiPairLut& L,
                                          const uint8_t* __restrict__ regions, Mesh3 g, bool openbc, int ix,
                                          int iy, int iz, f3 m0, int r0) {
    f3 h{0.f, 0.f, 0.f};
#pragma unroll
    for (int d = 0; d < 2; d++) {
#pragma unroll
        for (int side = -1; side <= 1; side += 2) {
            f3 mn{0.f, 0.f, 0.f};
            int i_;
            bool inside;
            if (d == 0) {
                int xx = side < 0 ? lclamp(ix - 1, g.Nx, g.pbc & 1) : hclamp(ix + 1, g.Nx, g.pbc & 1);
                i_ = (iz * g.Ny + iy) * g.Nx + xx;
                inside = (side < 0 ? ix - 1 >= 0 : ix + 1 < g.Nx) || (g.pbc & 1);
            } else {
                int yy = side < 0 ? lclamp(iy - 1, g.Ny, g.pbc & 2) : hclamp(iy + 1, g.Ny, g.pbc & 2);
                i_ = (iz * g.Ny + yy) * g.Nx + ix;
                inside = (side < 0 ? iy - 1 >= 0 : iy + 1 < g.Ny) || (g.pbc & 2);
            }
            if (inside) mn = ld3(mx, my, mz, i_);
            bool missing = is0(mn);
            int rn = missing ? r0 : __ldg(regions + i_);
            int si = symidx(r0, rn);
            if (!missing || !openbc) {
                if (missing) {
                    float q = __ldg((d == 0 ? L.qx : L.qy) + si);
                    if (side < 0) q = -q;
                    if (d == 0) {
                        mn.x = fs(m0.x, fm(q, m0.z));
                        mn.y = m0.y;
                        mn.z = fa(m0.z, fm(q, m0.x));
                    } else {
                        mn.x = m0.x;
                        mn.y = fs(m0.y, fm(q, m0.z));
                        mn.z = fa(m0.z, fm(q, m0.y));
                    }
                }
                float s = __ldg((d == 0 ? L.sx : L.sy) + si);
                h.x = fa(h.x, fm(s, fs(mn.x, m0.x)));
                h.y = fa(h.y, fm(s, fs(mn.y, m0.y)));
                h.z = fa(h.z, fm(s, fs(mn.z, m0.z)));
                float Dc = __ldg((d == 0 ? L.dcx : L.dcy) + si);
                float tz = side < 0 ? -mn.z : mn.z;
                float tp = d == 0 ? mn.x : mn.y;
                tp = side < 0 ? -tp : tp;
                if (d == 0) h.x = fa(h.x, fm(Dc, tz));
                else h.y = fa(h.y, fm(Dc, tz));
                h.z = fs(h.z, fm(Dc, tp));
            }
        }
    }
    if (g.Nz != 1) {
#pragma unroll
        for (int side = -1; side <= 1; side += 2) {
            int zz = side < 0 ? lclamp(iz - 1, g.Nz, g.pbc & 4) : hclamp(iz + 1, g.Nz, g.pbc & 4);
            int i_ = (zz * g.Ny + iy) * g.Nx + ix;
            f3 mn = ld3(mx, my, mz, i_);
            if (is0(mn)) mn = m0;
            float s = __ldg(L.sz + symidx(r0, __ldg(regions + i_)));
            h.x = fa(h.x, fm(s, fs(mn.x, m0.x)));
            h.y = fa(h.y, fm(s, fs(mn.y, m0.y)));
            h.z = fa(h.z, fm(s, fs(mn.z, m0.z)));
        }
    }
    return h;
}

// Region-free variants (every cell in region 0): the pair coefficients are the
// (0,0) entries, passed as scalars, so no region or table loads are needed.
// Same operations, hence the same rounding, as exchange_sum / dmi_sum_lut.
struct PairCoef {
    float wax, way, waz;            // exchange: w_d * A(0,0)
    float sx, sy, sz, dcx, dcy, qx, qy;  // DMI: see DmiPairLut
};

__device__ __forceinline__ f3 exchange_sum_u(const float* __restrict__ mx, const float* __restrict__ my,
                                             const float* __restrict__ mz, const PairCoef& P, Mesh3 g, int ix,
                                             int iy, int iz, f3 m0) {
    f3 b{0.f, 0.f, 0.f};
    int nb[6];
    nb[0] = (iz * g.Ny + iy) * g.Nx + lclamp(ix - 1, g.Nx, g.pbc & 1);
    nb[1] = (iz * g.Ny + iy) * g.Nx + hclamp(ix + 1, g.Nx, g.pbc & 1);
    nb[2] = (iz * g.Ny + lclamp(iy - 1, g.Ny, g.pbc & 2)) * g.Nx + ix;
    nb[3] = (iz * g.Ny + hclamp(iy + 1, g.Ny, g.pbc & 2)) * g.Nx + ix;
    nb[4] = (lclamp(iz - 1, g.Nz, g.pbc & 4) * g.Ny + iy) * g.Nx + ix;
    nb[5] = (hclamp(iz + 1, g.Nz, g.pbc & 4) * g.Ny + iy) * g.Nx + ix;
    const int nn = (g.Nz != 1) ? 6 : 4;
#pragma unroll
    for (int k = 0; k < 6; k++) {
        if (k >= nn) break;
        const float s = k < 2 ? P.wax : (k < 4 ? P.way : P.waz);
        f3 mn = ld3(mx, my, mz, nb[k]);
        if (is0(mn)) mn = m0;
        b.x = fa(b.x, fm(s, fs(mn.x, m0.x)));
        b.y = fa(b.y, fm(s, fs(mn.y, m0.y)));
        b.z = fa(b.z, fm(s, fs(mn.z, m0.z)));
    }
    return b;
}

__device__ __forceinline__ f3 dmi_sum_u(const float* __restrict__ mx, const float* __restrict__ my,
                                        const float* __restrict__ mz, const PairCoef& P, Mesh3 g, bool openbc,
                                        int ix, int iy, int iz, f3 m0) {
    f3 h{0.f, 0.f, 0.f};
#pragma unroll
    for (int d = 0; d < 2; d++) {
#pragma unroll
        for (int side = -1; side <= 1; side += 2) {
            f3 mn{0.f, 0.f, 0.f};
            int i_;
            bool inside;
            if (d == 0) {
                int xx = side < 0 ? lclamp(ix - 1, g.Nx, g.pbc & 1) : hclamp(ix + 1, g.Nx, g.pbc & 1);
                i_ = (iz * g.Ny + iy) * g.Nx + xx;
                inside = (side < 0 ? ix - 1 >= 0 : ix + 1 < g.Nx) || (g.pbc & 1);
            } else {
                int yy = side < 0 ? lclamp(iy - 1, g.Ny, g.pbc & 2) : hclamp(iy + 1, g.Ny, g.pbc & 2);
                i_ = (iz * g.Ny + yy) * g.Nx + ix;
                inside = (side < 0 ? iy - 1 >= 0 : iy + 1 < g.Ny) || (g.pbc & 2);
            }
            if (inside) mn = ld3(mx, my, mz, i_);
            const bool missing = is0(mn);
            if (!missing || !openbc) {
                if (missing) {
                    float q = d == 0 ? P.qx : P.qy;
                    if (side < 0) q = -q;
                    if (d == 0) {
                        mn.x = fs(m0.x, fm(q, m0.z));
                        mn.y = m0.y;
                        mn.z = fa(m0.z, fm(q, m0.x));
                    } else {
                        mn.x = m0.x;
                        mn.y = fs(m0.y, fm(q, m0.z));
                        mn.z = fa(m0.z, fm(q, m0.y));
                    }
                }
                const float s = d == 0 ? P.sx : P.sy;
                h.x = fa(h.x, fm(s, fs(mn.x, m0.x)));
                h.y = fa(h.y, fm(s, fs(mn.y, m0.y)));
                h.z = fa(h.z, fm(s, fs(mn.z, m0.z)));
                const float Dc = d == 0 ? P.dcx : P.dcy;
                float tz = side < 0 ? -mn.z : mn.z;
                float tp = d == 0 ? mn.x : mn.y;
                tp = side < 0 ? -tp : tp;
                if (d == 0) h.x = fa(h.x, fm(Dc, tz));
                else h.y = fa(h.y, fm(Dc, tz));
                h.z = fs(h.z, fm(Dc, tp));
            }
        }
    }
    if (g.Nz != 1) {
#pragma unroll
        for (int side = -1; side <= 1; side += 2) {
            int zz = side < 0 ? lclamp(iz - 1, g.Nz, g.pbc & 4) : hclamp(iz + 1, g.Nz, g.pbc & 4);
            int i_ = (zz * g.Ny + iy) * g.Nx + ix;
            f3 mn = ld3(mx, my, mz, i_);
            if (is0(mn)) mn = m0;
            h.x = fa(h.x, fm(P.sz, fs(mn.x, m0.x)));
            h.y = fa(h.y, fm(P.sz, fs(mn.y, m0.y)));
            h.z = fa(h.z, fm(P.sz, fs(mn.z, m0.z)));
        }
    }
    return h;
}

struct UniaxParams {
    const float *Ms, *K1, *K2, *ux, *uy, *uz;
    float Ms_mul, K1_mul, K2_mul, ux_mul, uy_mul, uz_mul;
};

// uniaxialanisotropy2.cl:17-34 -- anisotropy field of cell i added to B
__device__ __forceinline__ void add_uniaxial(f3& B, const UniaxParams& p, f3 m, int i) {
    f3 u{amul(p.ux, p.ux_mul, i), amul(p.uy, p.uy_mul, i), amul(p.uz, p.uz_mul, i)};
    float len = __fsqrt_rn(dot3(u, u));
    float il = (len != 0.0f) ? fd(1.0f, len) : 0.0f;
    u = f3{fm(il, u.x), fm(il, u.y), fm(il, u.z)};
    float invMs = inv_msat(p.Ms, p.Ms_mul, i);
    float k1 = fm(amul(p.K1, p.K1_mul, i), invMs);
    float k2 = fm(amul(p.K2, p.K2_mul, i), invMs);
    float mu = dot3(m, u);
    float f1 = fm(fm(2.0f, k1), mu);
    float f2 = fm(fm(4.0f, k2), fm(fm(mu, mu), mu));
    B.x = fa(B.x, fa(fm(f1, u.x), fm(f2, u.x)));
    B.y = fa(B.y, fa(fm(f1, u.y), fm(f2, u.y)));
    B.z = fa(B.z, fa(fm(f1, u.z), fm(f2, u.z)));
}

// cubicanisotropy2.cl:10-58 -- cubic anisotropy field of cell i added to B
struct CubicParams {
    const float *Ms, *K1, *K2, *K3, *c1[3], *c2[3];
    float Ms_mul, K1_mul, K2_mul, K3_mul, c1_mul[3], c2_mul[3];
};
// float3.clh:18-21 normalized() of amul.clh:10-15 vmul()
__device__ __forceinline__ f3 normalized_vmul(const float* const v[3], const float mul[3], int i) {
    f3 a{amul(v[0], mul[0], i), amul(v[1], mul[1], i), amul(v[2], mul[2], i)};
    float len = __fsqrt_rn(dot3(a, a));
    float il = (len != 0.0f) ? fd(1.0f, len) : 0.0f;
    return f3{fm(il, a.x), fm(il, a.y), fm(il, a.z)};
}
__device__ __forceinline__ float pw4(float x) {  // float3.clh:36-39
    float s = fm(x, x);
    return fm(s, s);
}
__device__ __forceinline__ void add_cubic(f3& B, const CubicParams& p, f3 m, int i) {
    const float invMs = inv_msat(p.Ms, p.Ms_mul, i);
    const float k1 = fm(amul(p.K1, p.K1_mul, i), invMs);
    const float k2 = fm(amul(p.K2, p.K2_mul, i), invMs);
    const float k3 = fm(amul(p.K3, p.K3_mul, i), invMs);
    const f3 u1 = normalized_vmul(p.c1, p.c1_mul, i), u2 = normalized_vmul(p.c2, p.c2_mul, i);
    const f3 u3 = cross3(u1, u2);
    const float u1m = dot3(u1, m), u2m = dot3(u2, m), u3m = dot3(u3, m);
    const float s1 = fm(u1m, u1m), s2 = fm(u2m, u2m), s3 = fm(u3m, u3m);
    const float a1 = fa(s2, s3), a2 = fa(s1, s3), a3 = fa(s1, s2);
    const float b1 = fm(s2, s3), b2 = fm(s1, s3), b3 = fm(s1, s2);
    const float e1 = fa(pw4(u2m), pw4(u3m)), e2 = fa(pw4(u1m), pw4(u3m)), e3 = fa(pw4(u1m), pw4(u2m));
    const float p1 = fm(s1, u1m), p2 = fm(s2, u2m), p3 = fm(s3, u3m);
    const float f1 = fm(-2.0f, k1), f2 = fm(2.0f, k2), f3_ = fm(4.0f, k3);
    const float U1[3] = {u1.x, u1.y, u1.z}, U2[3] = {u2.x, u2.y, u2.z}, U3[3] = {u3.x, u3.y, u3.z};
    float out[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const float S1 = fa(fa(fm(a1, fm(u1m, U1[c])), fm(a2, fm(u2m, U2[c]))), fm(a3, fm(u3m, U3[c])));
        const float S2 = fa(fa(fm(b1, fm(u1m, U1[c])), fm(b2, fm(u2m, U2[c]))), fm(b3, fm(u3m, U3[c])));
        const float S3 = fa(fa(fm(e1, fm(p1, U1[c])), fm(e2, fm(p2, U2[c]))), fm(e3, fm(p3, U3[c])));
        out[c] = fs(fs(fm(f1, S1), fm(f2, S2)), fm(f3_, S3));
    }
    B.x = fa(B.x, out[0]);
    B.y = fa(B.y, out[1]);
    B.z = fa(B.z, out[2]);
}

// dmibulk.cl:28-228 -- exchange + bulk DMI of cell (ix, iy, iz) before the
// 1/Ms factor; missing neighbours extrapolated in all three directions
__device__ __forceinline__ f3 dmibulk_sum(const float* __restrict__ mx, const float* __restrict__ my,
                                          const float* __restrict__ mz, const float* __restrict__ aLUT,
                                          const float* __restrict__ dLUT, const uint8_t* __restrict__ regions,
                                          float cx, float cy, float cz, Mesh3 g, bool openbc, int ix, int iy,
                                          int iz, f3 m0, int r0) {
    f3 h{0.f, 0.f, 0.f};
#pragma unroll
    for (int d = 0; d < 3; d++) {
        if (d == 2 && g.Nz == 1) break;
        const float c = d == 0 ? cx : (d == 1 ? cy : cz);
#pragma unroll
        for (int side = -1; side <= 1; side += 2) {
            f3 mn{0.f, 0.f, 0.f};
            int i_;
            bool inside;
            if (d == 0) {
                const int xx = side < 0 ? lclamp(ix - 1, g.Nx, g.pbc & 1) : hclamp(ix + 1, g.Nx, g.pbc & 1);
                i_ = (iz * g.Ny + iy) * g.Nx + xx;
                inside = (side < 0 ? ix - 1 >= 0 : ix + 1 < g.Nx) || (g.pbc & 1);
            } else if (d == 1) {
                const int yy = side < 0 ? lclamp(iy - 1, g.Ny, g.pbc & 2) : hclamp(iy + 1, g.Ny, g.pbc & 2);
                i_ = (iz * g.Ny + yy) * g.Nx + ix;
                inside = (side < 0 ? iy - 1 >= 0 : iy + 1 < g.Ny) || (g.pbc & 2);
            } else {
                const int zz = side < 0 ? lclamp(iz - 1, g.Nz, g.pbc & 4) : hclamp(iz + 1, g.Nz, g.pbc & 4);
                i_ = (zz * g.Ny + iy) * g.Nx + ix;
                inside = (side < 0 ? iz - 1 >= 0 : iz + 1 < g.Nz) || (g.pbc & 4);
            }
            if (inside) mn = ld3(mx, my, mz, i_);
            const bool missing = is0(mn);
            const int si = symidx(r0, missing ? r0 : (int)__ldg(regions + i_));
            const float A = __ldg(aLUT + si), D = __ldg(dLUT + si);
            const float D_2A = fd(D, fm(2.0f, A));
            if (!missing || !openbc) {
                const float sc = side < 0 ? -c : c;
                if (missing) {
                    const float q = fm(sc, D_2A);
                    if (d == 0) {
                        mn = f3{m0.x, fs(m0.y, fm(q, m0.z)), fa(m0.z, fm(q, m0.y))};
                    } else if (d == 1) {
                        mn = f3{fa(m0.x, fm(q, m0.z)), m0.y, fs(m0.z, fm(q, m0.x))};
                    } else {
                        mn = f3{fs(m0.x, fm(q, m0.y)), fa(m0.y, fm(q, m0.x)), m0.z};
                    }
                }
                const float s = fd(fm(2.0f, A), fm(c, c));
                h.x = fa(h.x, fm(s, fs(mn.x, m0.x)));
                h.y = fa(h.y, fm(s, fs(mn.y, m0.y)));
                h.z = fa(h.z, fm(s, fs(mn.z, m0.z)));
                const float Dc = fd(D, c);
                const f3 t = side < 0 ? f3{-mn.x, -mn.y, -mn.z} : mn;
                if (d == 0) {
                    h.y = fa(h.y, fm(Dc, t.z));
                    h.z = fs(h.z, fm(Dc, t.y));
                } else if (d == 1) {
                    h.x = fs(h.x, fm(Dc, t.z));
                    h.z = fa(h.z, fm(Dc, t.x));
                } else {
                    h.x = fa(h.x, fm(Dc, t.y));
                    h.y = fs(h.y, fm(Dc, t.x));
                }
            }
        }
    }
    return h;
}

// Thermal noise.  The reference draws its normals from an OpenCL Threefry
// generator whose stream depends on the device's compute-unit count and
// work-group size (opencl/rng.go:198-205), so no other device reproduces its
// numbers; only their distribution is the contract.  Here each normal is a
// function of (seed, accepted-step index, cell, component): Philox4x32-10
// (Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as easy as
// 1, 2, 3", SC'11) of the counter (cell, step lo, step hi, 0) under the
// 64-bit seed, then Box-Muller on pairs of 24-bit uniforms in (0, 1).  A
// rejected step retries with the same numbers (the step index is unchanged),
// as the reference keeps its noise during a step (engine/temperature.go:86-97).
struct PhiloxCtr {
    uint32_t v[4];
};
__host__ __device__ __forceinline__ PhiloxCtr philox4x32_10(PhiloxCtr c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint64_t p0 = (uint64_t)0xD2511F53u * c.v[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.v[2];
        const PhiloxCtr o{{(uint32_t)(p1 >> 32) ^ c.v[1] ^ k0, (uint32_t)p1, (uint32_t)(p0 >> 32) ^ c.v[3] ^ k1,
                           (uint32_t)p0}};
        c = o;
    }
    return c;
}
// uniform in (0, 1) from the top 24 bits (exact in float32)
__device__ __forceinline__ float u24(uint32_t x) { return ((float)(x >> 8) + 0.5f) * (1.0f / 16777216.0f); }
// three standard normals for (seed, step, cell)
__device__ __forceinline__ f3 therm_normals(uint64_t seed, long long step, int cell) {
    const PhiloxCtr r = philox4x32_10(PhiloxCtr{{(uint32_t)cell, (uint32_t)(uint64_t)step,
                                                  (uint32_t)((uint64_t)step >> 32), 0u}},
                                       (uint32_t)seed, (uint32_t)(seed >> 32));
    const float a = sqrtf(-2.0f * logf(u24(r.v[0])));
    const float b = sqrtf(-2.0f * logf(u24(r.v[2])));
    float s1, c1, s2, c2;
    sincospif(2.0f * u24(r.v[1]), &s1, &c1);
    sincospif(2.0f * u24(r.v[3]), &s2, &c2);
    return f3{a * c1, a * s1, b * c2};
}
// temperature2.cl:11-17: noise * sqrt(kB2_VgammaDt * alpha * T / Ms)
__device__ __forceinline__ float therm_scale(float k2, float alpha, float temp, float invMs) {
    return __fsqrt_rn(fm(fm(fm(k2, alpha), temp), invMs));
}

// lltorque2.cl:13-23
__device__ __forceinline__ f3 lltorque(f3 m, f3 H, float alpha) {
    f3 mxH = cross3(m, H);
    float gilb = fd(-1.0f, fa(1.0f, fm(alpha, alpha)));
    f3 mmxH = cross3(m, mxH);
    return f3{fm(gilb, fa(mxH.x, fm(alpha, mmxH.x))), fm(gilb, fa(mxH.y, fm(alpha, mmxH.y))),
              fm(gilb, fa(mxH.z, fm(alpha, mmxH.z)))};
}
// llnoprecess.cl:16-17
__device__ __forceinline__ f3 llnoprecess(f3 m, f3 H) {
    f3 mxH = cross3(m, H);
    f3 r = cross3(m, mxH);
    return f3{-r.x, -r.y, -r.z};
}

// normalize2.cl:10-22 -- OpenCL normalize(v) taken as v * (1/sqrt(v.v)),
// zero for a zero vector; zero where vol == 0.
__device__ __forceinline__ f3 normalize_vol(f3 v, float w) {
    f3 V{fm(w, v.x), fm(w, v.y), fm(w, v.z)};
    float d = dot3(V, V);
    float inv = d > 0.0f ? fd(1.0f, __fsqrt_rn(d)) : 0.0f;
    if (w == 0.0f) return f3{0.f, 0.f, 0.f};
    return f3{fm(V.x, inv), fm(V.y, inv), fm(V.z, inv)};
}

// Non-negative float max via unsigned bit patterns (atomicMax on floats >= 0).
__device__ __forceinline__ void atomic_max_nonneg(unsigned int* addr, float v) {
    atomicMax(addr, __float_as_uint(v));
}

// Block-wide max of non-negative floats; NaN inputs are ignored like the
// reference's fmax (reducemaxvecnorm2.cl) and reported through *nan_flag.
template <int BLOCK>
__device__ __forceinline__ float block_max(float v, float* sh) {
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        v = (l < BLOCK / 32) ? sh[l] : 0.0f;
        for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    __syncthreads();
    return v;
}

}  // namespace umag
