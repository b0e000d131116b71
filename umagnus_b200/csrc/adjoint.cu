// adjoint.cu -- a differentiable fixed-step RK4 simulation (no counterpart in
// the reference): forward pass with checkpoints of m every K steps, backward
// pass by hand-written vector-Jacobian products.
//
// Model (the engine's field and stepper, engine/effectivefield.go,
// engine/torque.go, engine/rk4.go): B = demag(Ms m) + exchange(A)/Ms +
// uniaxial(K1, u)/Ms + B_ext, torque = LL torque with alpha, RK4 with fixed
// dt and every stage normalised.  Parameters: a per-cell Ms map, uniform A,
// K1 and B_ext (the differentiable ones) and uniform alpha and easy axis.
// Loss: w_probe * mean over steps n >= n0 of the mean m_z over a probe window
// + w_target * |<m>_final - target|^2.
//
// Backward, per RK4 step in reverse (stage states recomputed from the last
// checkpoint of the segment and kept): the normalisation's VJP
// (w - n (n.w)) / |u|, the LL torque's VJP (cross products), and the
// effective field's VJP: the demag convolution with a real, even kernel is
// self-adjoint (the same plan applied to the cotangent), the exchange stencil
// with its clamped boundary is symmetric, anisotropy and Zeeman are local.
#include <algorithm>
#include <cmath>
#include <cstring>
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
    PairCoef pc;       // exchange pair coefficients w_d * A (region (0,0))
    float K1, alpha, gilb;
    float u[3];        // easy axis as given (normalised per cell like uniaxialanisotropy2.cl)
    float bext[3];
    int anis;
};

// ---------------------------------------------------------------- forward
// B_eff and the LL torque of m (engine/effectivefield.go:14-24 order);
// bd = demag field or NULL
__global__ void k_adj_field(AdjField a, const float* __restrict__ m, const float* __restrict__ bd, float* B,
                            float* tau) {
    const int N = a.N;
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < N; I += gridDim.x * blockDim.x) {
        const int ix = I % a.g.Nx, iy = (I / a.g.Nx) % a.g.Ny, iz = I / (a.g.Nx * a.g.Ny);
        const float *mx = m, *my = m + N, *mz = m + 2 * N;
        const f3 m0 = ld3(mx, my, mz, I);
        f3 b{0.f, 0.f, 0.f};
        if (bd) b = f3{bd[I], bd[N + I], bd[2 * N + I]};
        if (!is0(m0)) {
            const f3 e = exchange_sum_u(mx, my, mz, a.pc, a.g, ix, iy, iz, m0);
            const float inv = inv_msat(a.Ms, 1.0f, I);
            b.x = fa(b.x, fm(e.x, inv));
            b.y = fa(b.y, fm(e.y, inv));
            b.z = fa(b.z, fm(e.z, inv));
        }
        if (a.anis) {
            const UniaxParams up{a.Ms, nullptr, nullptr, nullptr, nullptr, nullptr, 1.0f, a.K1, 0.0f, a.u[0], a.u[1], a.u[2]};
            add_uniaxial(b, up, m0, I);
        }
        b.x = fa(b.x, a.bext[0]);
        b.y = fa(b.y, a.bext[1]);
        b.z = fa(b.z, a.bext[2]);
        const f3 mxB = cross3(m0, b), mmxB = cross3(m0, mxB);
        const f3 t{fm(a.gilb, fa(mxB.x, fm(a.alpha, mmxB.x))), fm(a.gilb, fa(mxB.y, fm(a.alpha, mmxB.y))),
                   fm(a.gilb, fa(mxB.z, fm(a.alpha, mmxB.z)))};
        if (B) { B[I] = b.x; B[N + I] = b.y; B[2 * N + I] = b.z; }
        tau[I] = t.x; tau[N + I] = t.y; tau[2 * N + I] = t.z;
    }
}

// dst = normalize(m + sum_j f_j k_j) with the Madd<n> rounding order (the
// engine's k_stage); nk = 1 or 4
__global__ void k_adj_stage(int N, const float* __restrict__ m, const float* k0, const float* k1, const float* k2,
                            const float* k3, int nk, float f0, float f1, float f2, float f3_, float* dst) {
    const float* ks[4] = {k0, k1, k2, k3};
    const float fs_[4] = {f0, f1, f2, f3_};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        float v[3];
        for (int c = 0; c < 3; c++) {
            float acc = fm(1.0f, m[c * N + i]);
            for (int j = 0; j < nk; j++) acc = fa(acc, fm(fs_[j], ks[j][c * N + i]));
            v[c] = acc;
        }
        const f3 r = normalize_vol(f3{v[0], v[1], v[2]}, 1.0f);
        dst[i] = r.x; dst[N + i] = r.y; dst[2 * N + i] = r.z;
    }
}

// loss pieces of one state: sum over the probe window of m_z (FP64), and the
// component sums of m (FP64) for the final average
__global__ void k_adj_probe(int N, int Nx, int Ny, const float* __restrict__ m, int px, int py, int pw, int ph,
                            double* out) {
    __shared__ double sh[8];
    double acc = 0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < pw * ph; q += gridDim.x * blockDim.x) {
        const int x = px + q % pw, y = py + q / pw;
        acc += (double)m[2 * N + y * Nx + x];  // z component, layer 0
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[w];
        atomicAdd(out, t);
    }
}

// ---------------------------------------------------------------- backward
// VJP of dst = normalize(u), u = m + sum_j f_j k_j: g_u = (w - n (n.w)) / |u|;
// lam += g_u; gk_j += f_j g_u
__global__ void k_adj_norm_vjp(int N, const float* __restrict__ m, const float* k0, const float* k1, const float* k2,
                               const float* k3, int nk, float f0, float f1, float f2, float f3_,
                               const float* __restrict__ w, float* lam, float* g0, float* g1, float* g2, float* g3) {
    const float* ks[4] = {k0, k1, k2, k3};
    float* gs[4] = {g0, g1, g2, g3};
    const float fs_[4] = {f0, f1, f2, f3_};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        float u[3];
        for (int c = 0; c < 3; c++) {
            float acc = fm(1.0f, m[c * N + i]);
            for (int j = 0; j < nk; j++) acc = fa(acc, fm(fs_[j], ks[j][c * N + i]));
            u[c] = acc;
        }
        const float len = sqrtf(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        const float il = len > 0.f ? 1.0f / len : 0.0f;
        const float n[3] = {u[0] * il, u[1] * il, u[2] * il};
        const float ww[3] = {w[i], w[N + i], w[2 * N + i]};
        const float nw = n[0] * ww[0] + n[1] * ww[1] + n[2] * ww[2];
        for (int c = 0; c < 3; c++) {
            const float gu = (ww[c] - n[c] * nw) * il;
            lam[c * N + i] += gu;
            for (int j = 0; j < nk; j++) gs[j][c * N + i] += fs_[j] * gu;
        }
    }
}

// VJP of the LL torque t = g (m x B + alpha m x (m x B)), g = -1/(1+alpha^2):
// gm = g [B x w + alpha ((m x B) x w + B x (w x m))],
// wB = g [w x m + alpha (w x m) x m]
__device__ __forceinline__ f3 c3(f3 a, f3 b) { return f3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
__global__ void k_adj_torque_vjp(int N, float alpha, float gilb, const float* __restrict__ m,
                                 const float* __restrict__ B, const float* __restrict__ w, float* gm, float* wB) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const f3 mm{m[i], m[N + i], m[2 * N + i]}, b{B[i], B[N + i], B[2 * N + i]}, ww{w[i], w[N + i], w[2 * N + i]};
        const f3 mxB = c3(mm, b), wxm = c3(ww, mm);
        const f3 t1 = c3(b, ww), t2 = c3(mxB, ww), t3 = c3(b, wxm), t4 = c3(wxm, mm);
        gm[i] = gilb * (t1.x + alpha * (t2.x + t3.x));
        gm[N + i] = gilb * (t1.y + alpha * (t2.y + t3.y));
        gm[2 * N + i] = gilb * (t1.z + alpha * (t2.z + t3.z));
        wB[i] = gilb * (wxm.x + alpha * t4.x);
        wB[N + i] = gilb * (wxm.y + alpha * t4.y);
        wB[2 * N + i] = gilb * (wxm.z + alpha * t4.z);
    }
}

// VJP of B_eff(m; Ms, A, K1, B_ext) with cotangent wB at state m:
//   gm += Ms D(wB) (demag D = mu0 K, self-adjoint) + S(wB / Ms) (exchange
//   stencil S, symmetric) + 2 k1 (wB.u) u (anisotropy, k1 = K1/Ms);
//   gMs += m.D(wB) - wB.e / Ms^2 - 2 K1 (m.u)(wB.u) / Ms^2 (e = S m);
//   gA += wB.e / (Ms A); gK1 += 2 (m.u)(wB.u) / Ms; gB += wB.
// dw = D(wB) (demag of the cotangent) or NULL; sums: gA, gK1, gB[3] (FP64)
__global__ void k_adj_field_vjp(AdjField a, float A, const float* __restrict__ m, const float* __restrict__ wB,
                                const float* __restrict__ dw, float* gm, double* gMs, double* sums) {
    __shared__ double sh[5][8];
    const int N = a.N;
    double acc[5] = {0, 0, 0, 0, 0};
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < N; I += gridDim.x * blockDim.x) {
        const int ix = I % a.g.Nx, iy = (I / a.g.Nx) % a.g.Ny, iz = I / (a.g.Nx * a.g.Ny);
        const float ms = a.Ms[I];
        const float inv = ms == 0.f ? 0.f : 1.0f / ms;
        const f3 w{wB[I], wB[N + I], wB[2 * N + I]};
        const f3 m0{m[I], m[N + I], m[2 * N + I]};
        f3 g{0.f, 0.f, 0.f};
        double gms = 0;
        if (dw) {  // dw = mu0 K wB (the demag plan applied to wB with Ms = 1)
            const f3 d{dw[I], dw[N + I], dw[2 * N + I]};
            g = f3{ms * d.x, ms * d.y, ms * d.z};
            gms += (double)m0.x * d.x + (double)m0.y * d.y + (double)m0.z * d.z;
        }
        // exchange: the stencil applied to x = wB / Ms (transpose of the forward
        // stencil, which is symmetric with the clamped boundary), and e = S m
        {
            int nb[6];
            nb[0] = (iz * a.g.Ny + iy) * a.g.Nx + lclamp(ix - 1, a.g.Nx, false);
            nb[1] = (iz * a.g.Ny + iy) * a.g.Nx + hclamp(ix + 1, a.g.Nx, false);
            nb[2] = (iz * a.g.Ny + lclamp(iy - 1, a.g.Ny, false)) * a.g.Nx + ix;
            nb[3] = (iz * a.g.Ny + hclamp(iy + 1, a.g.Ny, false)) * a.g.Nx + ix;
            nb[4] = (lclamp(iz - 1, a.g.Nz, false) * a.g.Ny + iy) * a.g.Nx + ix;
            nb[5] = (hclamp(iz + 1, a.g.Nz, false) * a.g.Ny + iy) * a.g.Nx + ix;
            const int nn = a.g.Nz != 1 ? 6 : 4;
            f3 sx{0.f, 0.f, 0.f}, e{0.f, 0.f, 0.f};
            const f3 x0{w.x * inv, w.y * inv, w.z * inv};
            for (int k = 0; k < nn; k++) {
                const float s = k < 2 ? a.pc.wax : (k < 4 ? a.pc.way : a.pc.waz);
                const int j = nb[k];
                const float ij = a.Ms[j] == 0.f ? 0.f : 1.0f / a.Ms[j];
                sx.x += s * (wB[j] * ij - x0.x);
                sx.y += s * (wB[N + j] * ij - x0.y);
                sx.z += s * (wB[2 * N + j] * ij - x0.z);
                e.x += s * (m[j] - m0.x);
                e.y += s * (m[N + j] - m0.y);
                e.z += s * (m[2 * N + j] - m0.z);
            }
            g.x += sx.x; g.y += sx.y; g.z += sx.z;
            const double we = (double)(w.x * e.x + w.y * e.y + w.z * e.z);
            gms -= we * (double)inv * (double)inv;
            acc[0] += we * (double)inv / (double)A;
        }
        if (a.anis) {
            f3 u{a.u[0], a.u[1], a.u[2]};
            const float len = sqrtf(u.x * u.x + u.y * u.y + u.z * u.z);
            const float il = len > 0.f ? 1.0f / len : 0.f;
            u = f3{u.x * il, u.y * il, u.z * il};
            const float mu = m0.x * u.x + m0.y * u.y + m0.z * u.z;
            const float wu = w.x * u.x + w.y * u.y + w.z * u.z;
            const float k1 = a.K1 * inv;
            g.x += 2.f * k1 * wu * u.x;
            g.y += 2.f * k1 * wu * u.y;
            g.z += 2.f * k1 * wu * u.z;
            gms -= 2.0 * (double)a.K1 * (double)mu * (double)wu * (double)inv * (double)inv;
            acc[1] += 2.0 * (double)mu * (double)wu * (double)inv;
        }
        acc[2] += w.x;
        acc[3] += w.y;
        acc[4] += w.z;
        gm[I] += g.x; gm[N + I] += g.y; gm[2 * N + I] += g.z;
        gMs[I] += gms;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int t = 0; t < 5; t++) {
        double v = acc[t];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[t][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        double v = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) v += sh[threadIdx.x][q];
        atomicAdd(sums + threadIdx.x, v);
    }
}

// loss cotangents of one state: the probe term (m_z over the window in layer
// 0, weight wprobe per cell) and the final-average term gavg (NULL: none)
__global__ void k_adj_loss_grad(int N, int Nx, int Ny, float* lam, int px, int py, int pw, int ph, float wprobe,
                                const float* gavg) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        if (gavg)
            for (int c = 0; c < 3; c++) lam[c * N + i] += gavg[c];
        if (wprobe != 0.f && i < Nx * Ny) {
            const int x = i % Nx, y = i / Nx;
            if (x >= px && x < px + pw && y >= py && y < py + ph) lam[2 * N + i] += wprobe;
        }
    }
}

__global__ void k_adj_axpy(size_t n, const float* __restrict__ x, float* y) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] += x[i];
}

__global__ void k_adj_to_f32(int n, const double* __restrict__ x, float* y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = (float)x[i];
}

// ---------------------------------------------------------------- host
// work buffers (3N floats each)
enum : int {
    W_K = 0,      // 0..3: k1..k4 (forward) / their cotangents (backward)
    W_MS = 4,     // 4..6: stage states m2..m4 (forward)
    W_GM = 4,     // backward: cotangent of a stage state
    W_WB = 5,     // backward: cotangent of the stage's field
    W_DW = 6,     // backward: demag of that cotangent
    W_BD = 7,     // demag field
    W_A = 8, W_B = 9,
    W_FINAL = 10,
    W_LAM = 11, W_LAM2 = 12,
    W_GAVG = 13,
    W_NEXT = 14,
    W_M0 = 15,    // m0 as given (before the initial normalisation)
    W_COUNT = 16
};

struct AdjImpl {
    umag_adj_params p;
    int N = 0;
    Mesh3 g{};
    umag_demag* demag = nullptr;
    float h = 0;          // float32(dt * GammaLL)
    float* Ms = nullptr;  // per-cell Ms of the last forward
    float A = 0, A00 = 0, K1 = 0, B[3] = {0, 0, 0};
    std::vector<float*> ckpt;  // m at steps 0, K, 2K, ...
    float* seg = nullptr;      // one segment: K steps x 12 x 3N (start state, m2..m4, B1..B4, k1..k4)
    float* work = nullptr;     // W_COUNT x 3N
    double* gMs = nullptr;     // per-cell gradient (FP64)
    double* dsum = nullptr;    // 8 doubles: probe sum / gA, gK1, gB
    bool have_forward = false;
    double avg[3] = {0, 0, 0};
    size_t n3() const { return 3 * (size_t)N; }
    float* w(int k) const { return work + (size_t)k * n3(); }
};

static cudaStream_t AS() { return ctx().stream; }

static AdjField adj_field(const AdjImpl* s) {
    AdjField a{};
    a.g = s->g;
    a.N = s->N;
    a.Ms = s->Ms;
    // engine/exchange.go: w_d = 2/c_d^2 (float32), coefficient w_d * A(0,0)
    const float wx = (float)(2 / (s->p.cell[0] * s->p.cell[0])), wy = (float)(2 / (s->p.cell[1] * s->p.cell[1])),
                wz = (float)(2 / (s->p.cell[2] * s->p.cell[2]));
    a.pc.wax = wx * s->A00;
    a.pc.way = wy * s->A00;
    a.pc.waz = wz * s->A00;
    a.K1 = s->K1;
    a.alpha = s->p.alpha;
    const float aa = s->p.alpha * s->p.alpha;
    const float den = 1.0f + aa;
    a.gilb = -1.0f / den;  // lltorque2.cl:18
    for (int c = 0; c < 3; c++) { a.u[c] = s->p.anisU[c]; a.bext[c] = s->B[c]; }
    a.anis = s->K1 != 0.f;
    return a;
}

static unsigned gridN(const AdjImpl* s) { return (unsigned)grid_for(s->N, 256); }

// demag of v (3N) into out: Ms map (forward) or Ms = 1 (cotangent)
static int adj_demag(AdjImpl* s, const float* v, const float* Ms, float* out) {
    PassArgs a{};
    fill_pass_args(s->demag, a);
    for (int c = 0; c < 3; c++) { a.m[c] = v + (size_t)c * s->N; a.B[c] = out + (size_t)c * s->N; }
    a.Ms = Ms;
    a.Ms_mul = 1.0f;
    return demag_launch(s->demag, a, AS());
}

// torque (and field if B) of m
static int adj_torque(AdjImpl* s, const float* m, float* B, float* tau) {
    const float* bd = nullptr;
    if (s->demag) {
        UMAG_TRY(adj_demag(s, m, s->Ms, s->w(W_BD)));
        bd = s->w(W_BD);
    }
    k_adj_field<<<gridN(s), 256, 0, AS()>>>(adj_field(s), m, bd, B, tau);
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

// RK4 weights (engine/rk4.go:35-61): stage offsets 1/2, 1/2, 1 and the final
// combination 1/6, 1/3, 1/3, 1/6, each float32(c) * h as Madd takes them
struct Rk4Fac {
    float st[3], fin[4];
};
static Rk4Fac rk4_fac(float h) {
    Rk4Fac f;
    f.st[0] = (float)(1. / 2.) * h;
    f.st[1] = (float)(1. / 2.) * h;
    f.st[2] = (float)1. * h;
    f.fin[0] = (float)(1. / 6.) * h;
    f.fin[1] = (float)(1. / 3.) * h;
    f.fin[2] = (float)(1. / 3.) * h;
    f.fin[3] = (float)(1. / 6.) * h;
    return f;
}

// one RK4 step m -> mout with fixed h; st (or NULL) receives m2..m4 (st[0..2]),
// B1..B4 (st[3..6]) and k1..k4 (st[7..10])
static int adj_step(AdjImpl* s, const float* m, float* mout, float* const* st) {
    float* k[4];
    float* ms[3];
    float* Bs[4];
    for (int q = 0; q < 4; q++) {
        k[q] = st ? st[7 + q] : s->w(W_K + q);
        Bs[q] = st ? st[3 + q] : nullptr;
    }
    for (int q = 0; q < 3; q++) ms[q] = st ? st[q] : s->w(W_MS + q);
    const Rk4Fac f = rk4_fac(s->h);
    const unsigned G = gridN(s);
    UMAG_TRY(adj_torque(s, m, Bs[0], k[0]));
    for (int q = 0; q < 3; q++) {
        k_adj_stage<<<G, 256, 0, AS()>>>(s->N, m, k[q], nullptr, nullptr, nullptr, 1, f.st[q], 0, 0, 0, ms[q]);
        UMAG_TRY(adj_torque(s, ms[q], Bs[q + 1], k[q + 1]));
    }
    k_adj_stage<<<G, 256, 0, AS()>>>(s->N, m, k[0], k[1], k[2], k[3], 4, f.fin[0], f.fin[1], f.fin[2], f.fin[3], mout);
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

int adj_free(umag_adj* h) {
    AdjImpl* s = reinterpret_cast<AdjImpl*>(h);
    if (!s) return UMAG_OK;
    cudaStreamSynchronize(AS());
    if (s->demag) demag_free(s->demag);
    cudaFree(s->Ms);
    for (float* c : s->ckpt) cudaFree(c);
    cudaFree(s->seg);
    cudaFree(s->work);
    cudaFree(s->gMs);
    cudaFree(s->dsum);
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
    AdjImpl* s = new AdjImpl();
    s->p = *p;
    s->N = p->N[0] * p->N[1] * p->N[2];
    s->g = Mesh3{p->N[0], p->N[1], p->N[2], 0};
    s->h = (float)(p->dt * (p->gamma_ll > 0 ? p->gamma_ll : 1.7595e11));  // engine/run.go:33 GammaLL
    auto fail = [&](int c) {
        adj_free(reinterpret_cast<umag_adj*>(s));
        return c;
    };
    const size_t n3 = s->n3();
    if (cudaMalloc(&s->Ms, sizeof(float) * s->N) != cudaSuccess ||
        cudaMalloc(&s->seg, sizeof(float) * n3 * 12 * (size_t)p->K) != cudaSuccess ||
        cudaMalloc(&s->work, sizeof(float) * n3 * W_COUNT) != cudaSuccess ||
        cudaMalloc(&s->gMs, sizeof(double) * s->N) != cudaSuccess ||
        cudaMalloc(&s->dsum, sizeof(double) * 8) != cudaSuccess)
        return fail(set_error(UMAG_E_NOMEM, "adjoint buffers"));
    const int nck = (p->nsteps + p->K - 1) / p->K;  // states 0, K, ..: segment starts
    for (int i = 0; i < nck; i++) {
        float* c = nullptr;
        if (cudaMalloc(&c, sizeof(float) * n3) != cudaSuccess) return fail(set_error(UMAG_E_NOMEM, "checkpoints"));
        s->ckpt.push_back(c);
    }
    if (p->enable_demag) {
        const int pbc[3] = {0, 0, 0};
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

int adj_forward(umag_adj* hd, const float* m0, const float* Ms, float A, float K1, const float Bext[3], double* loss) {
    AdjImpl* s = reinterpret_cast<AdjImpl*>(hd);
    UMAG_REQUIRE(s && m0 && Ms && Bext && loss, "NULL argument");
    UMAG_REQUIRE(A > 0, "Aex must be positive");
    const umag_adj_params& p = s->p;
    const size_t n3 = s->n3();
    s->have_forward = false;
    UMAG_CUDA(cudaMemcpyAsync(s->Ms, Ms, sizeof(float) * s->N, cudaMemcpyDeviceToDevice, AS()));
    s->A = A;
    s->A00 = 2.0f / (1.0f / A + 1.0f / A);  // engine/exchange.go:153-167, region 0 with itself
    s->K1 = K1;
    for (int c = 0; c < 3; c++) s->B[c] = Bext[c];
    float* a = s->w(W_A);
    float* b = s->w(W_B);
    UMAG_CUDA(cudaMemcpyAsync(s->w(W_M0), m0, sizeof(float) * n3, cudaMemcpyDeviceToDevice, AS()));
    UMAG_CUDA(cudaMemcpyAsync(a, m0, sizeof(float) * n3, cudaMemcpyDeviceToDevice, AS()));
    UMAG_TRY(normalize(a, a + s->N, a + 2 * (size_t)s->N, nullptr, s->N));  // engine/magnetization.go:34
    UMAG_CUDA(cudaMemsetAsync(s->dsum, 0, sizeof(double) * 8, AS()));
    for (int n = 1; n <= p.nsteps; n++) {
        if ((n - 1) % p.K == 0)
            UMAG_CUDA(cudaMemcpyAsync(s->ckpt[(n - 1) / p.K], a, sizeof(float) * n3, cudaMemcpyDeviceToDevice, AS()));
        UMAG_TRY(adj_step(s, a, b, nullptr));
        std::swap(a, b);
        if (n >= p.avg_from && p.w_probe != 0)
            k_adj_probe<<<8, 256, 0, AS()>>>(s->N, p.N[0], p.N[1], a, p.probe[0], p.probe[1], p.probe[2],
                                              p.probe[3], s->dsum);
    }
    UMAG_LAUNCH_CHECK();
    UMAG_CUDA(cudaMemcpyAsync(s->w(W_FINAL), a, sizeof(float) * n3, cudaMemcpyDeviceToDevice, AS()));
    double avg[3];
    for (int c = 0; c < 3; c++) {
        UMAG_TRY(sum_dot(a + (size_t)c * s->N, nullptr, s->N, &avg[c]));  // compensated FP64 sum
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

int adj_backward(umag_adj* hd, float* gMs, float* gm0, double* gA, double* gK1, double gB[3]) {
    AdjImpl* s = reinterpret_cast<AdjImpl*>(hd);
    UMAG_REQUIRE(s && gMs && gA && gK1 && gB, "NULL argument");
    UMAG_REQUIRE(s->have_forward, "backward needs a forward pass first");
    const umag_adj_params& p = s->p;
    const int N = s->N;
    const size_t n3 = s->n3();
    const unsigned G = gridN(s);
    const Rk4Fac f = rk4_fac(s->h);
    const AdjField af = adj_field(s);
    UMAG_CUDA(cudaMemsetAsync(s->gMs, 0, sizeof(double) * N, AS()));
    UMAG_CUDA(cudaMemsetAsync(s->dsum, 0, sizeof(double) * 8, AS()));
    float* lam = s->w(W_LAM);    // dL/d(state n)
    float* lam2 = s->w(W_LAM2);  // dL/d(state n-1), being accumulated
    float* gk = s->w(W_K);
    float* gm = s->w(W_GM);
    float* wB = s->w(W_WB);
    float* dw = s->w(W_DW);
    const float wprobe = (float)(p.w_probe / ((double)(p.nsteps - p.avg_from + 1) * p.probe[2] * p.probe[3]));
    float gavg[3];
    for (int c = 0; c < 3; c++) gavg[c] = (float)(2.0 * p.w_target * (s->avg[c] - p.target[c]) / N);
    UMAG_CUDA(cudaMemcpyAsync(s->w(W_GAVG), gavg, sizeof(gavg), cudaMemcpyHostToDevice, AS()));
    UMAG_CUDA(cudaMemsetAsync(lam, 0, sizeof(float) * n3, AS()));
    k_adj_loss_grad<<<G, 256, 0, AS()>>>(N, p.N[0], p.N[1], lam, p.probe[0], p.probe[1], p.probe[2], p.probe[3],
                                          wprobe, s->w(W_GAVG));
    UMAG_LAUNCH_CHECK();
    const int nseg = (p.nsteps + p.K - 1) / p.K;
    for (int sg = nseg - 1; sg >= 0; sg--) {
        const int n_begin = sg * p.K, len = std::min(p.nsteps, n_begin + p.K) - n_begin;
        // recompute the segment from its checkpoint, keeping every stage
        auto slot = [&](int j, int q) { return s->seg + ((size_t)j * 12 + q) * n3; };
        UMAG_CUDA(cudaMemcpyAsync(slot(0, 11), s->ckpt[sg], sizeof(float) * n3, cudaMemcpyDeviceToDevice, AS()));
        for (int j = 0; j < len; j++) {
            float* st[11];
            for (int q = 0; q < 11; q++) st[q] = slot(j, q);
            UMAG_TRY(adj_step(s, slot(j, 11), j + 1 < len ? slot(j + 1, 11) : s->w(W_NEXT), st));
        }
        // reverse through the segment's steps
        for (int j = len - 1; j >= 0; j--) {
            const int n = n_begin + j + 1;  // the step from state n-1 to state n
            const float* m = slot(j, 11);
            const float* ms[4] = {m, slot(j, 0), slot(j, 1), slot(j, 2)};
            const float* Bs[4] = {slot(j, 3), slot(j, 4), slot(j, 5), slot(j, 6)};
            const float* ks[4] = {slot(j, 7), slot(j, 8), slot(j, 9), slot(j, 10)};
            UMAG_CUDA(cudaMemsetAsync(gk, 0, sizeof(float) * 4 * n3, AS()));
            UMAG_CUDA(cudaMemsetAsync(lam2, 0, sizeof(float) * n3, AS()));
            k_adj_norm_vjp<<<G, 256, 0, AS()>>>(N, m, ks[0], ks[1], ks[2], ks[3], 4, f.fin[0], f.fin[1], f.fin[2],
                                                 f.fin[3], lam, lam2, gk, gk + n3, gk + 2 * n3, gk + 3 * n3);
            for (int q = 3; q >= 0; q--) {
                k_adj_torque_vjp<<<G, 256, 0, AS()>>>(N, af.alpha, af.gilb, ms[q], Bs[q], gk + q * n3, gm, wB);
                if (s->demag) UMAG_TRY(adj_demag(s, wB, nullptr, dw));
                k_adj_field_vjp<<<G, 256, 0, AS()>>>(af, s->A, ms[q], wB, s->demag ? dw : nullptr, gm, s->gMs,
                                                      s->dsum);
                if (q > 0)  // m_q = normalize(m + c h k_{q-1})
                    k_adj_norm_vjp<<<G, 256, 0, AS()>>>(N, m, ks[q - 1], nullptr, nullptr, nullptr, 1, f.st[q - 1],
                                                         0, 0, 0, gm, lam2, gk + (q - 1) * n3, nullptr, nullptr,
                                                         nullptr);
                else
                    k_adj_axpy<<<G, 256, 0, AS()>>>(n3, gm, lam2);
            }
            UMAG_LAUNCH_CHECK();
            std::swap(lam, lam2);
            if (n - 1 >= p.avg_from && p.w_probe != 0)  // the probe term of state n-1
                k_adj_loss_grad<<<G, 256, 0, AS()>>>(N, p.N[0], p.N[1], lam, p.probe[0], p.probe[1], p.probe[2],
                                                      p.probe[3], wprobe, nullptr);
        }
    }
    // lam = dL/d(normalised m0); through the initial normalisation
    if (gm0) {
        UMAG_CUDA(cudaMemsetAsync(gm0, 0, sizeof(float) * n3, AS()));
        k_adj_norm_vjp<<<G, 256, 0, AS()>>>(N, s->w(W_M0), nullptr, nullptr, nullptr, nullptr, 0, 0, 0, 0, 0, lam,
                                             gm0, nullptr, nullptr, nullptr, nullptr);
    }
    k_adj_to_f32<<<G, 256, 0, AS()>>>(N, s->gMs, gMs);
    UMAG_LAUNCH_CHECK();
    double hs[8];
    UMAG_CUDA(cudaMemcpyAsync(hs, s->dsum, sizeof(hs), cudaMemcpyDeviceToHost, AS()));
    UMAG_CUDA(cudaStreamSynchronize(AS()));
    *gA = hs[0];
    *gK1 = hs[1];
    for (int c = 0; c < 3; c++) gB[c] = hs[2 + c];
    return UMAG_OK;
}

}  // namespace umag
