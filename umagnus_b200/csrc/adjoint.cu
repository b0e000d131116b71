// adjoint.cu -- a differentiable fixed-step RK4 or Heun simulation (no
// counterpart in the reference): forward pass with checkpoints of m every K
// steps, backward pass by hand-written vector-Jacobian products.
//
// Model (the engine's field and stepper, engine/effectivefield.go,
// engine/torque.go, engine/rk4.go): B = demag(Ms m) + exchange(A)/Ms +
// uniaxial(K1, u)/Ms + B_ext, torque = LL torque with alpha, RK4 with fixed
// dt and every stage normalised, or Heun (engine/heun.go:27-43: predictor
// y1 = m + h k0 not normalised, result normalize(y1 + h/2 k1 - h/2 k0)).
// Parameters: a per-cell Ms map, uniform A,
// K1 and B_ext (the differentiable ones) and uniform alpha and easy axis, on
// an open or periodic mesh, with an optional geometry (volume fractions).
// Loss: w_probe * mean over states avg_from..nsteps of the mean m_z over a
// probe window + w_target * |<m>_final - target|^2.
//
// Backward, per RK4 step in reverse (stage states recomputed from the
// segment's checkpoint and kept): the normalisation's VJP (w - n (n.w))/|u|,
// the LL torque's VJP (cross products), and the effective field's VJP: the
// demag convolution with a real, even kernel is self-adjoint (the same plan
// applied to the cotangent; with periodic axes the same holds for the
// periodic kernel), the exchange stencil with its clamped boundary, or
// wrapped on a periodic axis, is symmetric, anisotropy and Zeeman are local.
//
// Launch structure.  Forward, per stage: the three demag passes, then one
// kernel that evaluates the field and torque of the stage state and, per
// cell, forms the next stage state (or the step's result, with the probe
// sum).  Reverse, per step: one kernel for the final combination's VJP and
// the last stage's torque VJP, then per stage the demag of the field
// cotangent and one kernel for the field VJP, the stage normalisation's VJP
// and the torque VJP of the stage before.  Each segment (K steps forward, or
// K steps recomputed and reversed) is replayed from a CUDA graph.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "cellmath.cuh"
#include "common.cuh"
#include "demag.cuh"
#include "ops.cuh"

namespace umag {

struct AdjField {
    Mesh3 g;
    int N;
    const float* Ms;   // per-cell map
    const float* vol;  // geometry (cell volume fractions) or NULL: m is zero where it is 0
    // region map (or NULL) with per-region parameters: the exchange LUT of
    // the engine (harmonic means of the regions' A, symidx layout), each
    // region's A, K1 and applied field (bext[c * 256 + r]); w_d = 2/c_d^2
    const uint8_t* regions;
    const float *aLUT, *Ar, *K1r, *bextr;
    float wx, wy, wz;
    PairCoef pc;       // exchange pair coefficients w_d * A (region (0,0)); with DMI also 2A/c^2, D/c, c D/(2A)
    int dmi;           // exchange + interfacial DMI (dmi.cl) instead of exchange (exchange.cl)
    float dq[2];       // DMI: (D/c)(c D/(2A)) = D^2/(2A) per in-plane axis, the missing neighbour's net weight
    float K1, alpha, gilb;
    float u[3];        // easy axis as given (normalised per cell like uniaxialanisotropy2.cl)
    float bext[3];
    int anis;
    int probe[4];      // x0, y0, width, height
};

// Stepper weights, each float32(c) * h as Madd takes them.  RK4
// (engine/rk4.go:35-61): stage offsets 1/2, 1/2, 1 and the final combination
// 1/6, 1/3, 1/3, 1/6.  Heun (engine/heun.go:31, :42): h for the predictor,
// 0.5h and -0.5h for the result (Madd3 rounding, madd3.cl).
struct StepFac {
    int heun;
    float st[3], fin[4];
    float h, hh, mhh;
};

__device__ __forceinline__ bool in_probe(const AdjField& a, int I) {
    if (I >= a.g.Nx * a.g.Ny) return false;  // layer 0 only
    const int x = I % a.g.Nx, y = I / a.g.Nx;
    return x >= a.probe[0] && x < a.probe[0] + a.probe[2] && y >= a.probe[1] && y < a.probe[1] + a.probe[3];
}

// B_eff and the LL torque of cell I of state m (engine/effectivefield.go:14-24
// order, the engine's per-cell arithmetic); bd = demag field or NULL
__device__ __forceinline__ void adj_field_cell(const AdjField& a, const float* __restrict__ m,
                                               const float* __restrict__ bd, int I, f3& b, f3& t) {
    const int N = a.N;
    const int ix = I % a.g.Nx, iy = (I / a.g.Nx) % a.g.Ny, iz = I / (a.g.Nx * a.g.Ny);
    const float *mx = m, *my = m + N, *mz = m + 2 * N;
    const f3 m0 = ld3(mx, my, mz, I);
    b = f3{0.f, 0.f, 0.f};
    if (bd) b = f3{bd[I], bd[N + I], bd[2 * N + I]};
    const int r0 = a.regions ? a.regions[I] : 0;
    if (!is0(m0)) {
        // with a region map, the engine's exchange stencil over its LUT
        const f3 e = a.regions ? exchange_sum(mx, my, mz, a.aLUT, a.regions, a.wx, a.wy, a.wz, a.g, ix, iy, iz, m0, r0)
                     : a.dmi   ? dmi_sum_u(mx, my, mz, a.pc, a.g, false, ix, iy, iz, m0)
                               : exchange_sum_u(mx, my, mz, a.pc, a.g, ix, iy, iz, m0);
        const float inv = inv_msat(a.Ms, 1.0f, I);
        b.x = fa(b.x, fm(e.x, inv));
        b.y = fa(b.y, fm(e.y, inv));
        b.z = fa(b.z, fm(e.z, inv));
    }
    if (a.anis) {
        const UniaxParams up{a.Ms, nullptr, nullptr, nullptr, nullptr, nullptr,
                             1.0f, a.regions ? a.K1r[r0] : a.K1, 0.0f, a.u[0], a.u[1], a.u[2]};
        add_uniaxial(b, up, m0, I);
    }
    b.x = fa(b.x, a.regions ? a.bextr[r0] : a.bext[0]);
    b.y = fa(b.y, a.regions ? a.bextr[256 + r0] : a.bext[1]);
    b.z = fa(b.z, a.regions ? a.bextr[512 + r0] : a.bext[2]);
    const f3 mxB = cross3(m0, b), mmxB = cross3(m0, mxB);
    t = f3{fm(a.gilb, fa(mxB.x, fm(a.alpha, mmxB.x))), fm(a.gilb, fa(mxB.y, fm(a.alpha, mmxB.y))),
           fm(a.gilb, fa(mxB.z, fm(a.alpha, mmxB.z)))};
}

__device__ __forceinline__ void st3(float* p, int N, int I, f3 v) {
    p[I] = v.x;
    p[N + I] = v.y;
    p[2 * N + I] = v.z;
}
__device__ __forceinline__ f3 ld3p(const float* p, int N, int I) { return f3{p[I], p[N + I], p[2 * N + I]}; }

// ---------------------------------------------------------------- forward
// Stage q of a step of state m: field and torque k_q of stage state mq
// (B_q kept if Bq), then per cell the next stage state
//   RK4 q < 3: mnext = normalize(m + st[q] k_q)
//   RK4 q = 3: mnext = normalize(m + fin0 k0 + fin1 k1 + fin2 k2 + fin3 k3)
//   Heun q = 0: mnext = m + h k0;  q = 1: mnext = normalize(mq + hh k1 + mhh k0)
// with the Madd<n> rounding order (the engine's k_stage), and for the last
// stage the probe's m_z sum of mnext added to *psum when psum != NULL.
__global__ void __launch_bounds__(256) k_adj_stage_fwd(AdjField a, StepFac f, int q, const float* __restrict__ mq,
                                                       const float* __restrict__ bd, float* Bq, float* kq,
                                                       const float* __restrict__ m, const float* k0,
                                                       const float* k1, const float* k2, float* mnext,
                                                       double* psum) {
    const int N = a.N;
    double acc = 0;
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < N; I += gridDim.x * blockDim.x) {
        f3 b, t;
        adj_field_cell(a, mq, bd, I, b, t);
        if (Bq) st3(Bq, N, I, b);
        st3(kq, N, I, t);
        const float tk[3] = {t.x, t.y, t.z};
        float v[3];
        for (int c = 0; c < 3; c++) {
            const int o = c * N + I;
            float s = fm(1.0f, m[o]);
            if (f.heun) {
                if (q == 0) s = fa(s, fm(f.h, tk[c]));                                       // y1 = m + h k0
                else s = fa(fm(1.0f, mq[o]), fa(fm(f.hh, tk[c]), fm(f.mhh, k0[o])));         // y1 + h/2 k1 - h/2 k0
            } else if (q < 3) {
                s = fa(s, fm(f.st[q], tk[c]));
            } else {
                s = fa(s, fm(f.fin[0], k0[o]));
                s = fa(s, fm(f.fin[1], k1[o]));
                s = fa(s, fm(f.fin[2], k2[o]));
                s = fa(s, fm(f.fin[3], tk[c]));
            }
            v[c] = s;
        }
        // Heun's predictor is not normalised (heun.go:31)
        const f3 r = (f.heun && q == 0) ? f3{v[0], v[1], v[2]}
                                        : normalize_vol(f3{v[0], v[1], v[2]}, a.vol ? a.vol[I] : 1.0f);
        st3(mnext, N, I, r);
        if (psum && in_probe(a, I)) acc += (double)r.z;
    }
    if (psum) {
        __shared__ double sh[8];
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += sh[w];
            if (s != 0) atomicAdd(psum, s);
        }
    }
}

// ---------------------------------------------------------------- backward
__device__ __forceinline__ f3 c3(f3 a, f3 b) {
    return f3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float d3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 sc3(float s, f3 a) { return f3{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ f3 ad3(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }

// VJP of n = u / |u|: (w - n (n.w)) / |u|
__device__ __forceinline__ f3 norm_vjp(f3 u, f3 w) {
    const float len = sqrtf(d3(u, u));
    const float il = len > 0.f ? 1.0f / len : 0.0f;
    const f3 n = sc3(il, u);
    const float nw = d3(n, w);
    return f3{(w.x - n.x * nw) * il, (w.y - n.y * nw) * il, (w.z - n.z * nw) * il};
}

// VJP of the LL torque t = g (m x B + alpha m x (m x B)), g = -1/(1+alpha^2),
// with cotangent w: gm = g [B x w + alpha ((m x B) x w + B x (w x m))],
// wB = g [w x m + alpha (w x m) x m]
__device__ __forceinline__ void torque_vjp(float alpha, float gilb, f3 m, f3 B, f3 w, f3& gm, f3& wB) {
    const f3 mxB = c3(m, B), wxm = c3(w, m);
    const f3 t1 = c3(B, w), t2 = c3(mxB, w), t3 = c3(B, wxm), t4 = c3(wxm, m);
    gm = sc3(gilb, ad3(t1, sc3(alpha, ad3(t2, t3))));
    wB = sc3(gilb, ad3(wxm, sc3(alpha, t4)));
}

// Start of the reverse of one step, per cell: u = m + sum_j fin_j k_j,
// g_u = VJP(normalize)(u; lam); lam2 = g_u; gk_j = fin_j g_u (j < 3); and the
// torque VJP of stage 3 with cotangent fin_3 g_u -> gm, wB.
__global__ void __launch_bounds__(256) k_adj_rev_start(AdjField a, StepFac f, const float* __restrict__ m,
                                                       const float* __restrict__ k0, const float* __restrict__ k1,
                                                       const float* __restrict__ k2, const float* __restrict__ k3,
                                                       const float* __restrict__ m3, const float* __restrict__ B3,
                                                       const float* __restrict__ lam, float* lam2, float* gk0,
                                                       float* gk1, float* gk2, float* gm, float* wB) {
    const int N = a.N;
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < N; I += gridDim.x * blockDim.x) {
        float u[3];
        for (int c = 0; c < 3; c++) {  // the forward's rounding order
            const int o = c * N + I;
            float s = fm(1.0f, m[o]);
            s = fa(s, fm(f.fin[0], k0[o]));
            s = fa(s, fm(f.fin[1], k1[o]));
            s = fa(s, fm(f.fin[2], k2[o]));
            s = fa(s, fm(f.fin[3], k3[o]));
            u[c] = s;
        }
        const f3 gu = norm_vjp(f3{u[0], u[1], u[2]}, ld3p(lam, N, I));
        st3(lam2, N, I, gu);
        st3(gk0, N, I, sc3(f.fin[0], gu));
        st3(gk1, N, I, sc3(f.fin[1], gu));
        st3(gk2, N, I, sc3(f.fin[2], gu));
        f3 g, w;
        torque_vjp(a.alpha, a.gilb, ld3p(m3, N, I), ld3p(B3, N, I), sc3(f.fin[3], gu), g, w);
        st3(gm, N, I, g);
        st3(wB, N, I, w);
    }
}

// Start of the reverse of one Heun step, per cell: z = y1 + hh k1 + mhh k0
// (the forward's rounding), g_z = VJP(normalize)(z; lam); lam2 = g_z (the
// part of dL/dy1 through z); gk0 = mhh g_z; and the torque VJP of stage 1
// (state y1, field B1) with cotangent hh g_z -> gm, wB.
__global__ void __launch_bounds__(256) k_adj_rev_start_heun(AdjField a, StepFac f, const float* __restrict__ y1,
                                                            const float* __restrict__ k0,
                                                            const float* __restrict__ k1,
                                                            const float* __restrict__ B1,
                                                            const float* __restrict__ lam, float* lam2, float* gk0,
                                                            float* gm, float* wB) {
    const int N = a.N;
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < N; I += gridDim.x * blockDim.x) {
        float z[3];
        for (int c = 0; c < 3; c++) {
            const int o = c * N + I;
            z[c] = fa(fm(1.0f, y1[o]), fa(fm(f.hh, k1[o]), fm(f.mhh, k0[o])));
        }
        const f3 gz = norm_vjp(f3{z[0], z[1], z[2]}, ld3p(lam, N, I));
        st3(lam2, N, I, gz);
        st3(gk0, N, I, sc3(f.mhh, gz));
        f3 g, w;
        torque_vjp(a.alpha, a.gilb, ld3p(y1, N, I), ld3p(B1, N, I), sc3(f.hh, gz), g, w);
        st3(gm, N, I, g);
        st3(wB, N, I, w);
    }
}

// Stage q of the reverse, per cell.  In: gm = torque-VJP part of dL/dm_q,
// wB = dL/dB_q (all cells: the exchange transpose reads neighbours), dw =
// mu0 K wB (demag of the cotangent) or NULL.  Field VJP:
//   dL/dm_q = gm + Ms dw + S(wB / Ms) + 2 (K1/Ms) (wB.u) u
//   acc[Ms] += m.dw - wB.e/Ms^2 - 2 K1 (m.u)(wB.u)/Ms^2,  e = S m_q
//   acc[A] += wB.e/(Ms A);  acc[K1] += 2 (m.u)(wB.u)/Ms;  acc[B] += wB
// (S: the exchange stencil with the clamped or periodic boundary,
// symmetric).  Then
//   q > 0: m_q = normalize(m + st[q-1] k_{q-1}): g_u = VJP; lam2 += g_u;
//          dL/dk_{q-1} = gk_{q-1} + st[q-1] g_u, and the torque VJP of stage
//          q-1 with it -> gm (in place), wBn
//   Heun q = 1: y1 = m + h k0 (not normalised): l = lam2 + dL/dy1 here is the
//          whole dL/dy1 (the part through z is in lam2), lam2 = l (m enters
//          y1 with weight 1), dL/dk0 = gk0 + h l, and the torque VJP of stage 0
//   q = 0: lam2 += dL/dm_0, plus the probe term wprobe (m_z in the window)
// acc: per-cell FP64 accumulators [Ms | A | K1 | Bx | By | Bz] (N each).
__global__ void __launch_bounds__(256) k_adj_rev_stage(AdjField a, StepFac f, int q, float A,
                                                       const float* __restrict__ mq, const float* __restrict__ wB,
                                                       const float* __restrict__ dw, float* gm,
                                                       const float* __restrict__ m, const float* __restrict__ kprev,
                                                       const float* __restrict__ gkprev,
                                                       const float* __restrict__ mprev,
                                                       const float* __restrict__ Bprev, float* lam2, float* wBn,
                                                       float wprobe, double* acc) {
    const int N = a.N;
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < N; I += gridDim.x * blockDim.x) {
        const int ix = I % a.g.Nx, iy = (I / a.g.Nx) % a.g.Ny, iz = I / (a.g.Nx * a.g.Ny);
        const float ms = a.Ms[I];
        const float inv = ms == 0.f ? 0.f : 1.0f / ms;
        const f3 w = ld3p(wB, N, I);
        const f3 m0 = ld3p(mq, N, I);
        f3 g = ld3p(gm, N, I);
        double gms = 0;
        // geometry: a cell outside it has m = 0, no exchange/DMI field, and
        // is a missing neighbour of the stencils (a zero m in exchange.cl and
        // dmi.cl); the demag source carries the volume fraction
        const float vI = a.vol ? a.vol[I] : 1.0f;
        auto hole = [&](int j) { return a.vol != nullptr && a.vol[j] == 0.f; };
        if (dw) {
            const f3 d = sc3(vI, ld3p(dw, N, I));
            g = ad3(g, sc3(ms, d));
            gms += (double)m0.x * d.x + (double)m0.y * d.y + (double)m0.z * d.z;
        }
        if (vI == 0.f) {
            // outside the geometry: no local field terms (the normalisation's
            // VJP zeroes this cell's cotangent)
        } else if (a.dmi) {
            // h = A E(m) + D R(m) + (D^2/2A) P(m) (dmi.cl with the missing in-plane
            // neighbours extrapolated): linear in m and symmetric, so the
            // cotangent x = wB/Ms goes through the same stencil, with the
            // missing neighbours decided by the geometry, not by zero values.
            // dh/dA = E(m) - (D^2/2A^2) P(m).
            const f3 x0 = sc3(inv, w);
            f3 lx{0.f, 0.f, 0.f}, eA{0.f, 0.f, 0.f}, pb{0.f, 0.f, 0.f};
#pragma unroll
            for (int d = 0; d < 2; d++) {
#pragma unroll
                for (int sd = -1; sd <= 1; sd += 2) {
                    // a periodic axis has every neighbour (wrapped)
                    const bool per = (a.g.pbc & (d == 0 ? 1 : 2)) != 0;
                    const int j = d == 0 ? (iz * a.g.Ny + iy) * a.g.Nx + (sd < 0 ? lclamp(ix - 1, a.g.Nx, per)
                                                                                  : hclamp(ix + 1, a.g.Nx, per))
                                         : (iz * a.g.Ny + (sd < 0 ? lclamp(iy - 1, a.g.Ny, per)
                                                                  : hclamp(iy + 1, a.g.Ny, per))) * a.g.Nx + ix;
                    const bool in = (per || (d == 0 ? (sd < 0 ? ix > 0 : ix + 1 < a.g.Nx)
                                                    : (sd < 0 ? iy > 0 : iy + 1 < a.g.Ny))) && !hole(j);
                    const float S = d == 0 ? a.pc.sx : a.pc.sy, Dc = (d == 0 ? a.pc.dcx : a.pc.dcy) * sd;
                    if (in) {
                        const float msj = a.Ms[j];
                        const float ij = msj == 0.f ? 0.f : 1.0f / msj;
                        const f3 xn{wB[j] * ij, wB[N + j] * ij, wB[2 * N + j] * ij};
                        const f3 mn{mq[j], mq[N + j], mq[2 * N + j]};
                        lx = ad3(lx, sc3(S, f3{xn.x - x0.x, xn.y - x0.y, xn.z - x0.z}));
                        eA = ad3(eA, sc3(S, f3{mn.x - m0.x, mn.y - m0.y, mn.z - m0.z}));
                        if (d == 0) { lx.x += Dc * xn.z; lx.z -= Dc * xn.x; }
                        else { lx.y += Dc * xn.z; lx.z -= Dc * xn.y; }
                    } else {
                        const float q = a.dq[d];
                        if (d == 0) { lx.x += q * x0.x; lx.z += q * x0.z; pb.x += q * m0.x; pb.z += q * m0.z; }
                        else { lx.y += q * x0.y; lx.z += q * x0.z; pb.y += q * m0.y; pb.z += q * m0.z; }
                    }
                }
            }
            if (a.g.Nz != 1) {
#pragma unroll
                for (int sd = -1; sd <= 1; sd += 2) {
                    const bool pz = (a.g.pbc & 4) != 0;
                    const int j = ((sd < 0 ? lclamp(iz - 1, a.g.Nz, pz) : hclamp(iz + 1, a.g.Nz, pz)) * a.g.Ny +
                                   iy) * a.g.Nx + ix;
                    if (hole(j)) continue;  // a zero neighbour: the term vanishes
                    const float msj = a.Ms[j];
                    const float ij = msj == 0.f ? 0.f : 1.0f / msj;
                    lx = ad3(lx, sc3(a.pc.sz, f3{wB[j] * ij - x0.x, wB[N + j] * ij - x0.y, wB[2 * N + j] * ij - x0.z}));
                    eA = ad3(eA, sc3(a.pc.sz, f3{mq[j] - m0.x, mq[N + j] - m0.y, mq[2 * N + j] - m0.z}));
                }
            }
            g = ad3(g, lx);
            // the field itself, as the forward computes it (for the Ms gradient)
            const f3 h = dmi_sum_u(mq, mq + N, mq + 2 * (size_t)N, a.pc, a.g, false, ix, iy, iz, m0);
            const double wh = (double)w.x * h.x + (double)w.y * h.y + (double)w.z * h.z;
            gms -= wh * (double)inv * (double)inv;
            const double wA = (double)w.x * (eA.x - pb.x) + (double)w.y * (eA.y - pb.y) + (double)w.z * (eA.z - pb.z);
            acc[(size_t)N + I] += wA * (double)inv / (double)A;
        } else {
            int nb[6];
            // exchange.cl's neighbours: clamped, or wrapped on a periodic axis
            const bool px = a.g.pbc & 1, py = a.g.pbc & 2, pz = a.g.pbc & 4;
            nb[0] = (iz * a.g.Ny + iy) * a.g.Nx + lclamp(ix - 1, a.g.Nx, px);
            nb[1] = (iz * a.g.Ny + iy) * a.g.Nx + hclamp(ix + 1, a.g.Nx, px);
            nb[2] = (iz * a.g.Ny + lclamp(iy - 1, a.g.Ny, py)) * a.g.Nx + ix;
            nb[3] = (iz * a.g.Ny + hclamp(iy + 1, a.g.Ny, py)) * a.g.Nx + ix;
            nb[4] = (lclamp(iz - 1, a.g.Nz, pz) * a.g.Ny + iy) * a.g.Nx + ix;
            nb[5] = (hclamp(iz + 1, a.g.Nz, pz) * a.g.Ny + iy) * a.g.Nx + ix;
            const int nn = a.g.Nz != 1 ? 6 : 4;
            f3 sx{0.f, 0.f, 0.f}, e{0.f, 0.f, 0.f};
            const f3 x0 = sc3(inv, w);
            const int ri = a.regions ? a.regions[I] : 0;
            double gA = 0;  // with regions: dL/dA of this cell's region, from its pairs
            for (int k = 0; k < nn; k++) {
                const int j = nb[k];
                if (hole(j)) continue;  // a zero neighbour: the term vanishes
                const float wd = k < 2 ? a.wx : (k < 4 ? a.wy : a.wz);
                float s;
                if (a.regions) {
                    const int rj = a.regions[j];
                    s = wd * a.aLUT[symidx(ri, rj)];
                } else {
                    s = k < 2 ? a.pc.wax : (k < 4 ? a.pc.way : a.pc.waz);
                }
                const float msj = a.Ms[j];
                const float ij = msj == 0.f ? 0.f : 1.0f / msj;
                const f3 xn{wB[j] * ij, wB[N + j] * ij, wB[2 * N + j] * ij};
                const f3 dm{mq[j] - m0.x, mq[N + j] - m0.y, mq[2 * N + j] - m0.z};
                sx = ad3(sx, sc3(s, f3{xn.x - x0.x, xn.y - x0.y, xn.z - x0.z}));
                e = ad3(e, sc3(s, dm));
                if (a.regions) {
                    // the pair coefficient a = 2/(1/A_i + 1/A_j); seen from
                    // this cell: (c_ij + c_ji) da/dA_i, c = w_d x.(m_other - m_own)
                    const double cij = (double)x0.x * dm.x + (double)x0.y * dm.y + (double)x0.z * dm.z;
                    const double cji = -((double)xn.x * dm.x + (double)xn.y * dm.y + (double)xn.z * dm.z);
                    const double ap = 2.0 / (1.0 / (double)a.Ar[ri] + 1.0 / (double)a.Ar[a.regions[j]]);
                    gA += (double)wd * (cij + cji) * ap * ap / (2.0 * (double)a.Ar[ri] * (double)a.Ar[ri]);
                }
            }
            g = ad3(g, sx);
            const double we = (double)w.x * e.x + (double)w.y * e.y + (double)w.z * e.z;
            gms -= we * (double)inv * (double)inv;
            acc[(size_t)N + I] += a.regions ? gA : we * (double)inv / (double)A;
        }
        if (a.anis) {
            f3 u{a.u[0], a.u[1], a.u[2]};
            const float len = sqrtf(d3(u, u));
            u = sc3(len > 0.f ? 1.0f / len : 0.f, u);
            const float mu = d3(m0, u), wu = d3(w, u);
            const float K1 = a.regions ? a.K1r[a.regions[I]] : a.K1;
            g = ad3(g, sc3(2.f * K1 * inv * wu, u));
            gms -= 2.0 * (double)K1 * (double)mu * (double)wu * (double)inv * (double)inv;
            acc[2 * (size_t)N + I] += 2.0 * (double)mu * (double)wu * (double)inv;
        }
        acc[I] += gms;
        acc[3 * (size_t)N + I] += w.x;
        acc[4 * (size_t)N + I] += w.y;
        acc[5 * (size_t)N + I] += w.z;
        f3 l = ld3p(lam2, N, I);
        if (q > 0 && f.heun) {
            l = ad3(l, g);
            const f3 gk = ad3(ld3p(gkprev, N, I), sc3(f.h, l));
            f3 gn, wn;
            torque_vjp(a.alpha, a.gilb, ld3p(mprev, N, I), ld3p(Bprev, N, I), gk, gn, wn);
            st3(gm, N, I, gn);
            st3(wBn, N, I, wn);
        } else if (q > 0) {
            const float c = f.st[q - 1];
            const f3 M = ld3p(m, N, I), Kp = ld3p(kprev, N, I);
            const f3 u{fa(fm(1.0f, M.x), fm(c, Kp.x)), fa(fm(1.0f, M.y), fm(c, Kp.y)), fa(fm(1.0f, M.z), fm(c, Kp.z))};
            const f3 gu = norm_vjp(u, g);
            l = ad3(l, gu);
            const f3 gk = ad3(ld3p(gkprev, N, I), sc3(c, gu));
            f3 gn, wn;
            torque_vjp(a.alpha, a.gilb, ld3p(mprev, N, I), ld3p(Bprev, N, I), gk, gn, wn);
            st3(gm, N, I, gn);
            st3(wBn, N, I, wn);
        } else {
            l = ad3(l, g);
            if (wprobe != 0.f && in_probe(a, I)) l.z += wprobe;
        }
        st3(lam2, N, I, l);
    }
}

// loss cotangent of the final state: the probe term (weight wprobe per
// window cell) and the final-average term (gx, gy, gz)
__global__ void k_adj_loss_final(AdjField a, float* lam, float wprobe, float gx, float gy, float gz) {
    const int N = a.N;
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < N; I += gridDim.x * blockDim.x) {
        f3 l{gx, gy, gz};
        if (wprobe != 0.f && in_probe(a, I)) l.z += wprobe;
        st3(lam, N, I, l);
    }
}

// dL/dm0 through the initial normalisation
// (zero outside the geometry, where the normalisation gives m = 0)
__global__ void k_adj_m0(int N, const float* __restrict__ m0, const float* __restrict__ lam, float* gm0,
                         const float* __restrict__ vol) {
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < N; I += gridDim.x * blockDim.x)
        st3(gm0, N, I, (vol && vol[I] == 0.f) ? f3{0.f, 0.f, 0.f} : norm_vjp(ld3p(m0, N, I), ld3p(lam, N, I)));
}

// per-cell accumulators -> gMs (float) and the five scalar sums, in a fixed
// order (one block of 1024 threads; deterministic)
__global__ void __launch_bounds__(1024) k_adj_reduce(int N, const double* __restrict__ acc, float* gMs, double* out) {
    __shared__ double sh[5][32];
    double s[5] = {0, 0, 0, 0, 0};
    for (int I = threadIdx.x; I < N; I += blockDim.x) {
        gMs[I] = (float)acc[I];
        for (int t = 0; t < 5; t++) s[t] += acc[(size_t)(t + 1) * N + I];
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int t = 0; t < 5; t++) {
        double v = s[t];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[t][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        double v = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += sh[threadIdx.x][w];
        out[threadIdx.x] = v;
    }
}

// per-region sums of the accumulators 1..5 (A, K1, B_x, B_y, B_z): block r
// adds the cells of region r in a fixed order (deterministic)
__global__ void __launch_bounds__(1024) k_adj_reduce_regions(int N, const double* __restrict__ acc,
                                                              const uint8_t* __restrict__ regions, double* out) {
    __shared__ double sh[5][32];
    const int r = blockIdx.x;
    double s[5] = {0, 0, 0, 0, 0};
    for (int I = threadIdx.x; I < N; I += blockDim.x)
        if (regions[I] == r)
            for (int t = 0; t < 5; t++) s[t] += acc[(size_t)(t + 1) * N + I];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int t = 0; t < 5; t++) {
        double v = s[t];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[t][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        double v = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += sh[threadIdx.x][w];
        out[(size_t)r * 5 + threadIdx.x] = v;
    }
}

// ---------------------------------------------------------------- host
// work buffers (3N floats each)
enum : int {
    W_K = 0,     // 0..3: k1..k4 (forward) / 0..2: their cotangents (reverse)
    W_MS = 4,    // 4..6: stage states m2..m4 (forward)
    W_GM = 4,    // reverse: torque-VJP part of a stage state's cotangent
    W_WB = 5,    // reverse: 5, 6: field cotangents (ping-pong)
    W_BD = 7,    // demag field / demag of the field cotangent
    W_A = 8, W_B = 9,
    W_FINAL = 10,
    W_LAM = 11, W_LAM2 = 12,
    W_NEXT = 13,
    W_M0 = 14,   // m0 as given (before the initial normalisation)
    W_COUNT = 15
};

struct AdjGraph {
    std::string key;
    cudaGraphExec_t exec;
};

struct AdjImpl {
    umag_adj_params p;
    int N = 0;
    Mesh3 g{};
    umag_demag* demag = nullptr;
    float h = 0;          // float32(dt * GammaLL)
    bool heun = false;    // Heun instead of RK4
    int nst() const { return heun ? 2 : 4; }
    float* Ms = nullptr;  // per-cell Ms of the last forward
    float A = 0, A00 = 0, D00 = 0, K1 = 0, B[3] = {0, 0, 0};
    std::vector<float*> ckpt;  // m at steps 0, K, 2K, ...
    float* seg = nullptr;      // one segment: K steps x 12 x 3N (m2..m4, B1..B4, k1..k4, start state)
    float* work = nullptr;     // W_COUNT x 3N
    double* acc = nullptr;     // per-cell FP64 gradient accumulators, 6 x N
    double* dsum = nullptr;    // 8 doubles: probe sum / scalar gradients
    // region maps (p.regions): the exchange LUT and per-region A, K1 and
    // field on the device, per-region gradient sums [nregions][5]
    float* reg_par = nullptr;  // aLUT (32896) | A (256) | K1 (256) | bext (3 x 256)
    double* reg_sum = nullptr;
    std::vector<float> hA, hK1;
    bool have_forward = false;
    double avg[3] = {0, 0, 0};
    std::vector<AdjGraph> graphs;  // segment graphs by key (parameters are baked in)
    size_t n3() const { return 3 * (size_t)N; }
    float* w(int k) const { return work + (size_t)k * n3(); }
    float* slot(int j, int q) const { return seg + ((size_t)j * 12 + q) * n3(); }
};

static cudaStream_t AS() { return ctx().stream; }
constexpr int kLutSize = 256 * 257 / 2;  // symidx LUT entries (kernels_src/clh/exchange.clh:5)

static AdjField adj_field(const AdjImpl* s) {
    AdjField a{};
    a.g = s->g;
    a.N = s->N;
    a.Ms = s->Ms;
    a.vol = s->p.vol;
    if (s->p.regions) {
        a.regions = s->p.regions;
        a.aLUT = s->reg_par;
        a.Ar = s->reg_par + kLutSize;
        a.K1r = a.Ar + 256;
        a.bextr = a.K1r + 256;
    }
    a.wx = (float)(2 / (s->p.cell[0] * s->p.cell[0]));
    a.wy = (float)(2 / (s->p.cell[1] * s->p.cell[1]));
    a.wz = (float)(2 / (s->p.cell[2] * s->p.cell[2]));
    // engine/exchange.go: w_d = 2/c_d^2 (float32), coefficient w_d * A(0,0)
    const float wx = (float)(2 / (s->p.cell[0] * s->p.cell[0])), wy = (float)(2 / (s->p.cell[1] * s->p.cell[1])),
                wz = (float)(2 / (s->p.cell[2] * s->p.cell[2]));
    a.pc.wax = wx * s->A00;
    a.pc.way = wy * s->A00;
    a.pc.waz = wz * s->A00;
    // DMI pair coefficients of region (0, 0), float32 operations as the
    // engine's k_local_consts (dmi.cl: 2A/c^2, D/c and the extrapolation
    // factor c (D/2)/A), cell sizes as float32 (opencl/dmi.go:61)
    a.dmi = s->D00 != 0.f;
    if (a.dmi) {
        const float cx = (float)s->p.cell[0], cy = (float)s->p.cell[1], cz = (float)s->p.cell[2];
        const float A = s->A00, D = s->D00;
        a.pc.sx = (2.0f * A) / (cx * cx);
        a.pc.sy = (2.0f * A) / (cy * cy);
        a.pc.sz = (2.0f * A) / (cz * cz);
        a.pc.dcx = D / cx;
        a.pc.dcy = D / cy;
        const float t = (0.5f * D) / A;
        a.pc.qx = cx * t;
        a.pc.qy = cy * t;
        a.dq[0] = a.pc.dcx * a.pc.qx;
        a.dq[1] = a.pc.dcy * a.pc.qy;
    }
    a.K1 = s->K1;
    a.alpha = s->p.alpha;
    const float aa = s->p.alpha * s->p.alpha;
    const float den = 1.0f + aa;
    a.gilb = -1.0f / den;  // lltorque2.cl:18
    for (int c = 0; c < 3; c++) { a.u[c] = s->p.anisU[c]; a.bext[c] = s->B[c]; }
    a.anis = s->K1 != 0.f;
    for (int c = 0; c < 4; c++) a.probe[c] = s->p.probe[c];
    return a;
}

static StepFac step_fac(float h, bool heun) {
    StepFac f{};
    f.heun = heun ? 1 : 0;
    f.h = (float)1. * h;       // Madd2(y, y, dy0, 1, dt)
    f.hh = (float)0.5 * h;     // Madd3(y, y, dy, dy0, 1, 0.5*dt, -0.5*dt)
    f.mhh = (float)-0.5 * h;
    f.st[0] = (float)(1. / 2.) * h;
    f.st[1] = (float)(1. / 2.) * h;
    f.st[2] = (float)1. * h;
    f.fin[0] = (float)(1. / 6.) * h;
    f.fin[1] = (float)(1. / 3.) * h;
    f.fin[2] = (float)(1. / 3.) * h;
    f.fin[3] = (float)(1. / 6.) * h;
    return f;
}

static unsigned gridN(const AdjImpl* s) { return (unsigned)grid_for(s->N, 256); }

// demag of v (3N) into out: Ms map and geometry (forward), or Ms = 1 and no
// geometry (cotangent: the reverse kernel applies Ms and vol per cell)
static int adj_demag(AdjImpl* s, const float* v, const float* Ms, float* out) {
    if (!s->demag) return UMAG_OK;
    PassArgs a{};
    fill_pass_args(s->demag, a);
    for (int c = 0; c < 3; c++) { a.m[c] = v + (size_t)c * s->N; a.B[c] = out + (size_t)c * s->N; }
    a.Ms = Ms;
    a.Ms_mul = 1.0f;
    a.vol = Ms ? s->p.vol : nullptr;
    return demag_launch(s->demag, a, AS());
}

// one step m -> mout (engine/rk4.go:35-61 or engine/heun.go:27-43 with fixed
// dt).  st (or NULL) receives the stage states after m (st[0..2]: m2..m4, or
// Heun's y1), the fields (st[3..6]) and the torques (st[7..10]); psum (or
// NULL) accumulates the probe's m_z sum of mout.
static int adj_step(AdjImpl* s, const AdjField& af, const StepFac& f, const float* m, float* mout, float* const* st,
                    double* psum) {
    const int nst = s->nst();
    float* k[4];
    float* Bs[4];
    float* next[4];
    const float* ms[4];
    for (int q = 0; q < nst; q++) {
        k[q] = st ? st[7 + q] : s->w(W_K + q);
        Bs[q] = st ? st[3 + q] : nullptr;
        next[q] = q < nst - 1 ? (st ? st[q] : s->w(W_MS + q)) : mout;
        ms[q] = q == 0 ? m : next[q - 1];
    }
    const float* bd = s->demag ? s->w(W_BD) : nullptr;
    for (int q = 0; q < nst; q++) {
        UMAG_TRY(adj_demag(s, ms[q], s->Ms, s->w(W_BD)));
        k_adj_stage_fwd<<<gridN(s), 256, 0, AS()>>>(af, f, q, ms[q], bd, Bs[q], k[q], m, k[0], nst > 1 ? k[1] : nullptr,
                                                     nst > 2 ? k[2] : nullptr, next[q],
                                                     q == nst - 1 ? psum : nullptr);
        UMAG_LAUNCH_CHECK();
    }
    return UMAG_OK;
}

// run `body` directly, or from the graph cached under `key` (captured on
// first use); the graph bakes in every pointer and parameter, so the key
// holds everything that varies between calls
template <class F>
static int adj_run(AdjImpl* s, const std::string& key, F body) {
    if (s->p.no_graph) return body();
    for (const AdjGraph& g : s->graphs)
        if (g.key == key) {
            UMAG_CUDA(cudaGraphLaunch(g.exec, AS()));
            return UMAG_OK;
        }
    cudaGraph_t graph;
    UMAG_CUDA(cudaStreamBeginCapture(AS(), cudaStreamCaptureModeThreadLocal));
    const int st = body();
    const cudaError_t e = cudaStreamEndCapture(AS(), &graph);
    if (st != UMAG_OK) {
        if (e == cudaSuccess) cudaGraphDestroy(graph);
        return st;
    }
    if (e != cudaSuccess) return set_error(UMAG_E_CUDA, "adjoint graph capture: %s", cudaGetErrorString(e));
    cudaGraphExec_t exec;
    const cudaError_t e2 = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e2 != cudaSuccess) return set_error(UMAG_E_CUDA, "adjoint graph instantiate: %s", cudaGetErrorString(e2));
    s->graphs.push_back(AdjGraph{key, exec});
    UMAG_CUDA(cudaGraphLaunch(exec, AS()));
    return UMAG_OK;
}

static void adj_drop_graphs(AdjImpl* s) {
    for (AdjGraph& g : s->graphs) cudaGraphExecDestroy(g.exec);
    s->graphs.clear();
}

// the values baked into a graph besides pointers: exchange, anisotropy, field
static std::string param_key(const AdjImpl* s) {
    char buf[128];
    if (s->p.regions)  // per-region values live in device arrays the graphs read
        snprintf(buf, sizeof buf, "/R%d", s->K1 != 0.f ? 1 : 0);
    else
        snprintf(buf, sizeof buf, "/%a/%a/%a/%a/%a/%a", s->A, s->A00, s->K1, s->B[0], s->B[1], s->B[2]);
    return buf;
}

int adj_free(umag_adj* h) {
    AdjImpl* s = reinterpret_cast<AdjImpl*>(h);
    if (!s) return UMAG_OK;
    cudaStreamSynchronize(AS());
    adj_drop_graphs(s);
    if (s->demag) demag_free(s->demag);
    cudaFree(s->Ms);
    for (float* c : s->ckpt) cudaFree(c);
    cudaFree(s->seg);
    cudaFree(s->work);
    cudaFree(s->acc);
    cudaFree(s->dsum);
    cudaFree(s->reg_par);
    cudaFree(s->reg_sum);
    delete s;
    return UMAG_OK;
}

int adj_new(const umag_adj_params* p, umag_adj** out) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(p && out, "NULL argument");
    UMAG_REQUIRE(p->N[0] > 0 && p->N[1] > 0 && p->N[2] > 0, "bad mesh");
    UMAG_REQUIRE(p->cell[0] > 0 && p->cell[1] > 0 && p->cell[2] > 0, "bad cell size");
    UMAG_REQUIRE(p->nsteps > 0 && p->K > 0 && p->dt > 0, "nsteps, K and dt must be positive");
    UMAG_REQUIRE(p->avg_from >= 1 && p->avg_from <= p->nsteps, "avg_from must lie in 1..nsteps");
    UMAG_REQUIRE(p->probe[2] > 0 && p->probe[3] > 0 && p->probe[0] >= 0 && p->probe[1] >= 0 &&
                     p->probe[0] + p->probe[2] <= p->N[0] && p->probe[1] + p->probe[3] <= p->N[1],
                 "probe window outside the mesh");
    UMAG_REQUIRE(p->solver == 0 || p->solver == 2 || p->solver == 4, "solver must be 4 (RK4) or 2 (Heun)");
    UMAG_REQUIRE(p->pbc[0] >= 0 && p->pbc[1] >= 0 && p->pbc[2] >= 0, "PBC repetitions must be non-negative");
    if (p->regions) {
        UMAG_REQUIRE(p->nregions >= 1 && p->nregions <= 256, "nregions must lie in 1..256");
        if (p->Dind != 0.f)
            return set_error(UMAG_E_UNSUPPORTED, "region maps with interfacial DMI are not supported by the adjoint");
    }
    AdjImpl* s = new AdjImpl();
    s->p = *p;
    s->N = p->N[0] * p->N[1] * p->N[2];
    // periodic axes wrap the stencils (data/mesh.go PBC_code: 1 x, 2 y, 4 z)
    s->g = Mesh3{p->N[0], p->N[1], p->N[2], (p->pbc[0] ? 1 : 0) | (p->pbc[1] ? 2 : 0) | (p->pbc[2] ? 4 : 0)};
    s->heun = p->solver == 2;
    s->h = (float)(p->dt * (p->gamma_ll > 0 ? p->gamma_ll : 1.7595e11));  // engine/torque.go:27 GammaLL
    auto fail = [&](int c) {
        adj_free(reinterpret_cast<umag_adj*>(s));
        return c;
    };
    const size_t n3 = s->n3();
    const int K = std::min(p->K, p->nsteps);
    if (cudaMalloc(&s->Ms, sizeof(float) * s->N) != cudaSuccess ||
        cudaMalloc(&s->seg, sizeof(float) * n3 * 12 * (size_t)K) != cudaSuccess ||
        cudaMalloc(&s->work, sizeof(float) * n3 * W_COUNT) != cudaSuccess ||
        cudaMalloc(&s->acc, sizeof(double) * 6 * (size_t)s->N) != cudaSuccess ||
        cudaMalloc(&s->dsum, sizeof(double) * 8) != cudaSuccess)
        return fail(set_error(UMAG_E_NOMEM, "adjoint buffers"));
    if (p->regions &&
        (cudaMalloc(&s->reg_par, sizeof(float) * (kLutSize + 5 * 256)) != cudaSuccess ||
         cudaMalloc(&s->reg_sum, sizeof(double) * 5 * 256) != cudaSuccess))
        return fail(set_error(UMAG_E_NOMEM, "adjoint region tables"));
    const int nck = (p->nsteps + p->K - 1) / p->K;  // segment starts: states 0, K, 2K, ...
    for (int i = 0; i < nck; i++) {
        float* c = nullptr;
        if (cudaMalloc(&c, sizeof(float) * n3) != cudaSuccess) return fail(set_error(UMAG_E_NOMEM, "checkpoints"));
        s->ckpt.push_back(c);
    }
    if (p->enable_demag) {
        const int* pbc = p->pbc;
        const int st = p->demag_kernel == 1
                           ? demag_new_brute(p->N[0], p->N[1], p->N[2], pbc, p->cell[0], p->cell[1], p->cell[2],
                                             p->demag_accuracy > 0 ? p->demag_accuracy : 6.0, &s->demag)
                           : demag_new_newell(p->N[0], p->N[1], p->N[2], pbc, p->cell[0], p->cell[1], p->cell[2], 32,
                                              0, &s->demag);
        if (st != UMAG_OK) return fail(st);
    }
    *out = reinterpret_cast<umag_adj*>(s);
    return UMAG_OK;
}

static int adj_forward_impl(AdjImpl* s, const float* m0, const float* Ms, double* loss);

int adj_forward(umag_adj* hd, const float* m0, const float* Ms, float A, float K1, const float Bext[3], double* loss) {
    AdjImpl* s = reinterpret_cast<AdjImpl*>(hd);
    UMAG_REQUIRE(s && m0 && Ms && Bext && loss, "NULL argument");
    UMAG_REQUIRE(!s->p.regions, "this handle has a region map: use umag_adj_forward_regions");
    UMAG_REQUIRE(A > 0, "Aex must be positive");
    s->A = A;
    s->A00 = 2.0f / (1.0f / A + 1.0f / A);  // engine/exchange.go:153-167, region 0 with itself
    const float D = s->p.Dind;
    s->D00 = D == 0.f ? 0.f : 2.0f / (1.0f / D + 1.0f / D);  // the same average for the DMI LUT
    s->K1 = K1;
    for (int c = 0; c < 3; c++) s->B[c] = Bext[c];
    return adj_forward_impl(s, m0, Ms, loss);
}

// per-region values (host arrays of nregions, B_ext as [r][3]): the engine's
// exchange LUT (engine/exchange.go:153-167: 2/(1/A_i + 1/A_j) in float32 at
// symidx(i, j); regions past nregions take A of region 0, as no cell uses
// them), A, K1 and the field per region, to the device
int adj_forward_regions(umag_adj* hd, const float* m0, const float* Ms, const float* A, const float* K1,
                        const float* Bext, double* loss) {
    AdjImpl* s = reinterpret_cast<AdjImpl*>(hd);
    UMAG_REQUIRE(s && m0 && Ms && A && K1 && Bext && loss, "NULL argument");
    UMAG_REQUIRE(s->p.regions, "this handle has no region map: use umag_adj_forward");
    const int nr = s->p.nregions;
    for (int r = 0; r < nr; r++) UMAG_REQUIRE(A[r] > 0, "Aex of region %d must be positive", r);
    std::vector<float> hp((size_t)kLutSize + 5 * 256, 0.f);
    float ex[256];
    for (int r = 0; r < 256; r++) ex[r] = A[r < nr ? r : 0];
    for (int i = 0; i < 256; i++)
        for (int j = 0; j <= i; j++) {
            const volatile float inv_i = 1.0f / ex[i], inv_j = 1.0f / ex[j];
            const volatile float sum = inv_i + inv_j;
            hp[(size_t)i * (i + 1) / 2 + j] = 2.0f / sum;
        }
    float* Ar = hp.data() + kLutSize;
    bool anis = false;
    for (int r = 0; r < nr; r++) {
        Ar[r] = A[r];
        Ar[256 + r] = K1[r];
        anis |= K1[r] != 0.f;
        for (int c = 0; c < 3; c++) Ar[512 + c * 256 + r] = Bext[3 * r + c];
    }
    UMAG_CUDA(cudaMemcpyAsync(s->reg_par, hp.data(), sizeof(float) * hp.size(), cudaMemcpyHostToDevice, AS()));
    UMAG_CUDA(cudaStreamSynchronize(AS()));  // the host table is released on return
    s->hA.assign(A, A + nr);
    s->hK1.assign(K1, K1 + nr);
    s->A = A[0];
    s->A00 = 0.f;
    s->D00 = 0.f;
    s->K1 = anis ? 1.f : 0.f;  // (the flag of the anisotropy term; the values are per region)
    for (int c = 0; c < 3; c++) s->B[c] = 0.f;
    return adj_forward_impl(s, m0, Ms, loss);
}

static int adj_forward_impl(AdjImpl* s, const float* m0, const float* Ms, double* loss) {
    const umag_adj_params& p = s->p;
    const size_t n3 = s->n3();
    s->have_forward = false;
    UMAG_CUDA(cudaMemcpyAsync(s->Ms, Ms, sizeof(float) * s->N, cudaMemcpyDeviceToDevice, AS()));
    const AdjField af = adj_field(s);
    const StepFac f = step_fac(s->h, s->heun);
    UMAG_CUDA(cudaMemcpyAsync(s->w(W_M0), m0, sizeof(float) * n3, cudaMemcpyDeviceToDevice, AS()));
    float* a0 = s->w(W_A);
    UMAG_CUDA(cudaMemcpyAsync(a0, m0, sizeof(float) * n3, cudaMemcpyDeviceToDevice, AS()));
    UMAG_TRY(normalize(a0, a0 + s->N, a0 + 2 * (size_t)s->N, s->p.vol, s->N));  // engine/magnetization.go:34
    UMAG_CUDA(cudaMemsetAsync(s->dsum, 0, sizeof(double) * 8, AS()));
    const int nseg = (p.nsteps + p.K - 1) / p.K;
    const std::string pk = param_key(s);
    for (int sg = 0; sg < nseg; sg++) {
        const int n_begin = sg * p.K, len = std::min(p.nsteps, n_begin + p.K) - n_begin;
        UMAG_CUDA(cudaMemcpyAsync(s->ckpt[sg], a0, sizeof(float) * n3, cudaMemcpyDeviceToDevice, AS()));
        // segment: len steps from W_A back into W_A, probe sums after steps n >= avg_from
        std::string key = "F" + std::to_string(len) + "/";
        for (int j = 0; j < len; j++) key += (n_begin + j + 1 >= p.avg_from && p.w_probe != 0) ? '1' : '0';
        key += pk;
        UMAG_TRY(adj_run(s, key, [&]() -> int {
            float* a = s->w(W_A);
            float* b = s->w(W_B);
            for (int j = 0; j < len; j++) {
                const int n = n_begin + j + 1;
                UMAG_TRY(adj_step(s, af, f, a, b, nullptr, (n >= p.avg_from && p.w_probe != 0) ? s->dsum : nullptr));
                std::swap(a, b);
            }
            if (a != s->w(W_A))
                UMAG_CUDA(cudaMemcpyAsync(s->w(W_A), a, sizeof(float) * n3, cudaMemcpyDeviceToDevice, AS()));
            return UMAG_OK;
        }));
    }
    UMAG_CUDA(cudaMemcpyAsync(s->w(W_FINAL), a0, sizeof(float) * n3, cudaMemcpyDeviceToDevice, AS()));
    double avg[3];
    for (int c = 0; c < 3; c++) {
        UMAG_TRY(sum_dot(a0 + (size_t)c * s->N, nullptr, s->N, &avg[c]));  // compensated FP64 sum
        avg[c] /= s->N;
    }
    double probe_sum = 0;
    UMAG_CUDA(cudaMemcpyAsync(&probe_sum, s->dsum, sizeof(double), cudaMemcpyDeviceToHost, AS()));
    UMAG_CUDA(cudaStreamSynchronize(AS()));
    const double navg = (double)(p.nsteps - p.avg_from + 1);
    const double probe_mean = probe_sum / (navg * p.probe[2] * p.probe[3]);
    double d2 = 0;
    for (int c = 0; c < 3; c++) {
        d2 += (avg[c] - p.target[c]) * (avg[c] - p.target[c]);
        s->avg[c] = avg[c];
    }
    *loss = p.w_probe * probe_mean + p.w_target * d2;
    s->have_forward = true;
    return UMAG_OK;
}

int adj_final_m(umag_adj* hd, float* m) {
    AdjImpl* s = reinterpret_cast<AdjImpl*>(hd);
    UMAG_REQUIRE(s && m, "NULL argument");
    UMAG_REQUIRE(s->have_forward, "no forward pass");
    UMAG_CUDA(cudaMemcpyAsync(m, s->w(W_FINAL), sizeof(float) * s->n3(), cudaMemcpyDeviceToDevice, AS()));
    UMAG_CUDA(cudaStreamSynchronize(AS()));
    return UMAG_OK;
}

// the reverse of one segment: recompute its steps from slot(0, 11) keeping
// every stage, then the steps in reverse with lam = dL/d(state at the
// segment's end) in W_LAM, leaving dL/d(state at its start) in W_LAM
static int adj_rev_segment(AdjImpl* s, const AdjField& af, const StepFac& f, int n_begin, int len, float wprobe) {
    const umag_adj_params& p = s->p;
    const unsigned G = gridN(s);
    const size_t n3 = s->n3();
    for (int j = 0; j < len; j++) {
        float* st[11];
        for (int q = 0; q < 11; q++) st[q] = s->slot(j, q);
        UMAG_TRY(adj_step(s, af, f, s->slot(j, 11), j + 1 < len ? s->slot(j + 1, 11) : s->w(W_NEXT), st, nullptr));
    }
    float* lam = s->w(W_LAM);
    float* lam2 = s->w(W_LAM2);
    float* gk[3] = {s->w(W_K), s->w(W_K + 1), s->w(W_K + 2)};
    float* gm = s->w(W_GM);
    float* wb[2] = {s->w(W_WB), s->w(W_WB + 1)};
    const float* dw = s->demag ? s->w(W_BD) : nullptr;
    for (int j = len - 1; j >= 0; j--) {
        const int n = n_begin + j + 1;  // the step from state n-1 to state n
        const float* m = s->slot(j, 11);
        const float* ms[4] = {m, s->slot(j, 0), s->slot(j, 1), s->slot(j, 2)};
        const float* Bs[4] = {s->slot(j, 3), s->slot(j, 4), s->slot(j, 5), s->slot(j, 6)};
        const float* ks[4] = {s->slot(j, 7), s->slot(j, 8), s->slot(j, 9), s->slot(j, 10)};
        // stage q's field cotangent lives in wb[q & 1] (the last stage: wb[1])
        const int nst = s->nst();
        if (s->heun)
            k_adj_rev_start_heun<<<G, 256, 0, AS()>>>(af, f, ms[1], ks[0], ks[1], Bs[1], lam, lam2, gk[0], gm, wb[1]);
        else
            k_adj_rev_start<<<G, 256, 0, AS()>>>(af, f, m, ks[0], ks[1], ks[2], ks[3], ms[3], Bs[3], lam, lam2,
                                                  gk[0], gk[1], gk[2], gm, wb[1]);
        UMAG_LAUNCH_CHECK();
        for (int q = nst - 1; q >= 0; q--) {
            float* wcur = wb[q & 1];
            float* wnext = wb[(q + 1) & 1];
            UMAG_TRY(adj_demag(s, wcur, nullptr, s->w(W_BD)));
            const bool probe_prev = q == 0 && n - 1 >= p.avg_from && p.w_probe != 0;
            k_adj_rev_stage<<<G, 256, 0, AS()>>>(af, f, q, s->A, ms[q], wcur, dw, gm, m, q > 0 ? ks[q - 1] : nullptr,
                                                  q > 0 ? gk[q - 1] : nullptr, q > 0 ? ms[q - 1] : nullptr,
                                                  q > 0 ? Bs[q - 1] : nullptr, lam2, wnext,
                                                  probe_prev ? wprobe : 0.f, s->acc);
            UMAG_LAUNCH_CHECK();
        }
        std::swap(lam, lam2);
    }
    if (lam != s->w(W_LAM))
        UMAG_CUDA(cudaMemcpyAsync(s->w(W_LAM), lam, sizeof(float) * n3, cudaMemcpyDeviceToDevice, AS()));
    return UMAG_OK;
}

static int adj_backward_impl(AdjImpl* s, float* gMs, float* gm0, double* hs);

int adj_backward(umag_adj* hd, float* gMs, float* gm0, double* gA, double* gK1, double gB[3]) {
    AdjImpl* s = reinterpret_cast<AdjImpl*>(hd);
    UMAG_REQUIRE(s && gMs && gA && gK1 && gB, "NULL argument");
    UMAG_REQUIRE(!s->p.regions, "this handle has a region map: use umag_adj_backward_regions");
    double hs[5];
    UMAG_TRY(adj_backward_impl(s, gMs, gm0, hs));
    *gA = hs[0];
    *gK1 = hs[1];
    for (int c = 0; c < 3; c++) gB[c] = hs[2 + c];
    return UMAG_OK;
}

// per-region gradients (host arrays of nregions; gB as [r][3])
int adj_backward_regions(umag_adj* hd, float* gMs, float* gm0, double* gA, double* gK1, double* gB) {
    AdjImpl* s = reinterpret_cast<AdjImpl*>(hd);
    UMAG_REQUIRE(s && gMs && gA && gK1 && gB, "NULL argument");
    UMAG_REQUIRE(s->p.regions, "this handle has no region map: use umag_adj_backward");
    UMAG_TRY(adj_backward_impl(s, gMs, gm0, nullptr));
    const int nr = s->p.nregions;
    k_adj_reduce_regions<<<nr, 1024, 0, AS()>>>(s->N, s->acc, s->p.regions, s->reg_sum);
    UMAG_LAUNCH_CHECK();
    std::vector<double> hs((size_t)5 * nr);
    UMAG_CUDA(cudaMemcpyAsync(hs.data(), s->reg_sum, sizeof(double) * hs.size(), cudaMemcpyDeviceToHost, AS()));
    UMAG_CUDA(cudaStreamSynchronize(AS()));
    for (int r = 0; r < nr; r++) {
        gA[r] = hs[5 * r];
        gK1[r] = hs[5 * r + 1];
        for (int c = 0; c < 3; c++) gB[3 * r + c] = hs[5 * r + 2 + c];
    }
    return UMAG_OK;
}

static int adj_backward_impl(AdjImpl* s, float* gMs, float* gm0, double* hs_out) {
    UMAG_REQUIRE(s->have_forward, "backward needs a forward pass first");
    const umag_adj_params& p = s->p;
    const int N = s->N;
    const size_t n3 = s->n3();
    const unsigned G = gridN(s);
    const StepFac f = step_fac(s->h, s->heun);
    const AdjField af = adj_field(s);
    UMAG_CUDA(cudaMemsetAsync(s->acc, 0, sizeof(double) * 6 * (size_t)N, AS()));
    const float wprobe = (float)(p.w_probe / ((double)(p.nsteps - p.avg_from + 1) * p.probe[2] * p.probe[3]));
    float gavg[3];
    for (int c = 0; c < 3; c++) gavg[c] = (float)(2.0 * p.w_target * (s->avg[c] - p.target[c]) / N);
    k_adj_loss_final<<<G, 256, 0, AS()>>>(af, s->w(W_LAM), p.w_probe != 0 ? wprobe : 0.f, gavg[0], gavg[1], gavg[2]);
    UMAG_LAUNCH_CHECK();
    const int nseg = (p.nsteps + p.K - 1) / p.K;
    const std::string pk = param_key(s);
    for (int sg = nseg - 1; sg >= 0; sg--) {
        const int n_begin = sg * p.K, len = std::min(p.nsteps, n_begin + p.K) - n_begin;
        UMAG_CUDA(cudaMemcpyAsync(s->slot(0, 11), s->ckpt[sg], sizeof(float) * n3, cudaMemcpyDeviceToDevice, AS()));
        std::string key = "R" + std::to_string(len) + "/";
        for (int j = 0; j < len; j++) key += (n_begin + j >= p.avg_from && p.w_probe != 0) ? '1' : '0';
        key += pk;
        UMAG_TRY(adj_run(s, key, [&]() { return adj_rev_segment(s, af, f, n_begin, len, wprobe); }));
    }
    if (gm0) {
        k_adj_m0<<<G, 256, 0, AS()>>>(N, s->w(W_M0), s->w(W_LAM), gm0, s->p.vol);
        UMAG_LAUNCH_CHECK();
    }
    k_adj_reduce<<<1, 1024, 0, AS()>>>(N, s->acc, gMs, s->dsum);
    UMAG_LAUNCH_CHECK();
    if (hs_out) {
        UMAG_CUDA(cudaMemcpyAsync(hs_out, s->dsum, sizeof(double) * 5, cudaMemcpyDeviceToHost, AS()));
    }
    UMAG_CUDA(cudaStreamSynchronize(AS()));
    return UMAG_OK;
}

}  // namespace umag
