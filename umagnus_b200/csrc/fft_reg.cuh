// fft_reg.cuh -- register-blocked Stockham FFT for power-of-two lengths.
//
// A line of length L is held by T = L/8 threads, thread t owning the eight
// elements {t + T*m : m = 0..7} in registers.  Every Stockham stage reads
// exactly that element set (for any radix R dividing 8, butterfly
// j = t + T*i uses elements j + r*L/R = t + T*(i + r*8/R)), so a stage is:
// butterflies in registers, then -- except after the last stage -- write the
// outputs to their Stockham positions in a padded shared-memory line and read
// the thread's set back.  The last stage's outputs land on the thread's own
// set (natural order X[t + T*m]), so a pointwise operation between a forward
// and an inverse transform needs no exchange, and the inverse is the forward
// transform of the conjugate.  Loads of zero padding and stores of discarded
// outputs disappear at compile time when the caller passes literal zeros /
// ignores elements.  Radices 8, then 4 or 2 for the remaining power of two.
#pragma once
#include "fft.cuh"
#include "fft_packed.cuh"

namespace umag {

constexpr int rg_log2(int L) { return L <= 1 ? 0 : 1 + rg_log2(L / 2); }
constexpr int rg_nst(int L) { return (rg_log2(L) + 2) / 3; }
// radix of stage s: 8 except a final 4 or 2 when log2(L) is not a multiple of 3
constexpr int rg_radix(int L, int s) {
    return (s < rg_log2(L) / 3) ? 8 : (rg_log2(L) % 3 == 1 ? 2 : 4);
}
constexpr bool rg_ok(int L) { return L >= 8 && (L & (L - 1)) == 0; }
// padded shared-memory index: MU slots of padding after every 2^PS elements.
// An 8-byte access of a warp is served as two half-warps of 16 lanes, each
// one wavefront when its lanes fall in 16 different 8-byte bank pairs.  PS =
// 3 when threads of several lines share a warp; 4 for one line per warp,
// where the exchanges after the first stage (outputs spaced NS = 8, 64 ...
// apart) take MU = 2 -- the choices that make these access patterns
// conflict-free.
template <int PS, int MU = 1> __host__ __device__ constexpr int rg_pad(int i) { return i + (i >> PS) * MU; }
// exchange-line stride: padded length rounded up to 4 (mod 16) 8-byte slots,
// so lines accessed by neighbouring threads start in different banks
template <int L, int PS = 3, int MU = 1> __host__ __device__ constexpr int rg_line() {
    return ((rg_pad<PS, MU>(L - 1) + 1 + 11) / 16) * 16 + 4;
}

// Staged twiddle tables.  Stage s >= 1 multiplies element r of butterfly k
// (k < NS, the product of the earlier radices; radix R) by W_L^(r k L/(NS R)).
// Read from one length-L table, lanes with different k would share banks
// (index strides r*L/(NS R)); the staged tables hold the twiddles of stage s
// as rows k of R + 1 slots (entries r = 1..R-1 used), an odd pitch, so the
// lanes of a stage read different banks.
template <int L> struct RgTw {
    static constexpr int nst = (rg_log2(L) + 2) / 3;
    static constexpr int radix(int s) { return s < rg_log2(L) / 3 ? 8 : (rg_log2(L) % 3 == 1 ? 2 : 4); }
    static constexpr int ns(int s) { return s == 0 ? 1 : ns(s - 1) * radix(s - 1); }
    static constexpr int pitch(int s) { return radix(s) + 1; }
    static constexpr int offset(int s) { return s <= 1 ? 0 : offset(s - 1) + ns(s - 1) * pitch(s - 1); }
    static constexpr int size = nst <= 1 ? 1 : offset(nst);
};

// Fill the staged tables of RgTw<L> from tw (tw[j] = exp(-2 pi i j / L),
// j < L; any memory space) by threads tid = 0..nth-1, stage by stage with
// compile-time shapes; the caller synchronises before the transform reads
// them.
template <int L, int S = 1>
__device__ __forceinline__ void rg_tw_fill(float2* tws, const float2* __restrict__ tw, int tid, int nth) {
    using G = RgTw<L>;
    if constexpr (S < G::nst) {
        constexpr int R = G::radix(S), P = G::pitch(S), N = G::ns(S) * P, STEP = L / (G::ns(S) * R);
        constexpr int OFF = G::offset(S);
        for (int e = tid; e < N; e += nth) {
            const int k = e / P, r = e - k * P;
            tws[OFF + e] = r < R ? tw[r * k * STEP] : make_float2(0.f, 0.f);
        }
        rg_tw_fill<L, S + 1>(tws, tw, tid, nth);
    }
}

// Barrier between exchange phases: the whole CTA, or only the warp when all
// threads sharing the exchange lines belong to one warp.
template <bool WARP> __device__ __forceinline__ void rg_sync() {
    if constexpr (WARP) __syncwarp();
    else __syncthreads();
}

// One stage for NC lines held by this thread (v[c][m] = element t + T*m of
// line c).  ex + c*exs is the padded exchange line of component c; the
// exchange after stage 0 pads by rg_pad<PS>, the later ones by rg_pad<PS, MU>.
// tw: the staged twiddle tables of RgTw<L>.
template <int L, int NC, int DIR, int ST, int NS, bool WARP = false, int PS = 3, bool ZH = false, int MU = 1>
__device__ __forceinline__ void rg_stage(float2 (&v)[NC][8], int t, float2* ex, int exs,
                                         const float2* __restrict__ tw) {
    static_assert(DIR == -1, "forward transforms only (the inverse is the forward of the conjugate)");
    if constexpr (ST < rg_nst(L)) {
        constexpr int R = rg_radix(L, ST);
        constexpr int NB = 8 / R;          // butterflies per thread
        constexpr int T = L / 8;
        constexpr int U = ST == 0 ? 1 : MU;  // padding slots of this stage's exchange
        constexpr bool last = (ST + 1 == rg_nst(L));
#pragma unroll
        for (int i = 0; i < NB; i++) {
            const int j = t + T * i;
            const int k = j % NS;
            // twiddles are shared by the NC lines: read them once, as the
            // pairs (w.re, w.re) and (-w.im, w.im) of the packed product
            P2 wrr[R], wii[R];
            if constexpr (NS > 1) {
                using G = RgTw<L>;
                static_assert(G::radix(ST) == R && G::ns(ST) == NS, "staged twiddle layout");
                const float2* wk = tw + G::offset(ST) + k * G::pitch(ST);
#pragma unroll
                for (int r = 1; r < R; r++) {
                    const float2 w = wk[r];
                    wrr[r] = p2(w.x, w.x);
                    wii[r] = p2(-w.y, w.y);
                }
            }
#pragma unroll
            for (int c = 0; c < NC; c++) {
                P2 u[R];
#pragma unroll
                for (int r = 0; r < R; r++) u[r] = p2(v[c][i + r * NB]);
                if constexpr (NS > 1) {
#pragma unroll
                    for (int r = 1; r < R; r++) u[r] = pcmul(u[r], wrr[r], wii[r]);
                }
                if constexpr (R == 8 && ZH && ST == 0) pdft8_zhalf(u);
                else if constexpr (R == 2) pdft2(u);
                else if constexpr (R == 4) pdft4(u);
                else pdft8(u);
                if constexpr (last) {
#pragma unroll
                    for (int q = 0; q < R; q++) v[c][i + q * NB] = f2(u[q]);
                } else {
                    const int o = (j / NS) * NS * R + k;
                    if constexpr (NS % (1 << PS) == 0) {  // pad(o + q*NS) = pad(o) + q*pad(NS)
                        float2* base = ex + c * exs + rg_pad<PS, U>(o);
#pragma unroll
                        for (int q = 0; q < R; q++) base[q * rg_pad<PS, U>(NS)] = f2(u[q]);
                    } else {
#pragma unroll
                        for (int q = 0; q < R; q++) ex[c * exs + rg_pad<PS, U>(o + q * NS)] = f2(u[q]);
                    }
                }
            }
        }
        if constexpr (!last) {
            rg_sync<WARP>();
            if constexpr (T % (1 << PS) == 0) {  // pad(t + T*m) = pad(t) + m*pad(T)
                const float2* base = ex + rg_pad<PS, U>(t);
#pragma unroll
                for (int c = 0; c < NC; c++)
#pragma unroll
                    for (int m = 0; m < 8; m++) v[c][m] = base[c * exs + m * rg_pad<PS, U>(T)];
            } else {
#pragma unroll
                for (int c = 0; c < NC; c++)
#pragma unroll
                    for (int m = 0; m < 8; m++) v[c][m] = ex[c * exs + rg_pad<PS, U>(t + T * m)];
            }
            rg_sync<WARP>();
            rg_stage<L, NC, DIR, ST + 1, NS * R, WARP, PS, ZH, MU>(v, t, ex, exs, tw);
        }
    }
}

// dft8 (forward) of (u0, u1, u2, u3, 0, 0, 0, 0), natural order out: the
// even outputs are the DFT4 of u, the odd ones the DFT4 of u_n W8^n -- 40
// instructions instead of the 56 of dft8 (x + 0 is not folded by the
// compiler: it is not an identity for x = -0).
__device__ __forceinline__ void dft8_zhalf(float2* v) {
    const float s = 0.70710678118654752440084436210485f;
    const float2 a = v[0], b = v[1], c = v[2], d = v[3];
    const float2 t0 = cadd(a, c), t1 = csub(a, c), t2 = cadd(b, d), t3 = mul_mi(csub(b, d), -1);
    float2 w1, w3;
    w1.x = s; w1.y = -s;   // W8
    w3.x = -s; w3.y = -s;  // W8^3
    const float2 b1 = cmul(b, w1), c1 = mul_mi(c, -1), d1 = cmul(d, w3);
    const float2 s0 = cadd(a, c1), s1 = csub(a, c1), s2 = cadd(b1, d1), s3 = mul_mi(csub(b1, d1), -1);
    v[0] = cadd(t0, t2); v[2] = cadd(t1, t3); v[4] = csub(t0, t2); v[6] = csub(t1, t3);
    v[1] = cadd(s0, s2); v[3] = cadd(s1, s3); v[5] = csub(s0, s2); v[7] = csub(s1, s3);
}

// Like rg_stage, for NC lines that exchange one at a time through two
// alternating buffers (ex and ex + exs; P = the buffer of the first line):
// a line is written, the CTA synchronises once and reads it back, so a
// buffer is rewritten only after a barrier that follows every read of it.
// Two buffers instead of NC, and one barrier per line and stage.  ZH: the
// upper half of the input is zero (the first radix-8 butterfly folds it).
// The butterflies and twiddle products run in packed FP32 (fft_packed.cuh).
template <int L, int NC, int ST, int NS, int P, bool ZH>
__device__ __forceinline__ void rg_stage_seq(float2 (&v)[NC][8], int t, float2* ex, int exs,
                                             const float2* __restrict__ tw) {
    constexpr int PS = 3;
    if constexpr (ST < rg_nst(L)) {
        constexpr int R = rg_radix(L, ST);
        constexpr int NB = 8 / R;
        constexpr int T = L / 8;
        constexpr bool last = (ST + 1 == rg_nst(L));
#pragma unroll
        for (int i = 0; i < NB; i++) {
            const int k = (t + T * i) % NS;
            P2 wrr[R], wii[R];  // twiddle w as (w.re, w.re) and (-w.im, w.im)
            if constexpr (NS > 1) {
                using G = RgTw<L>;
                static_assert(G::radix(ST) == R && G::ns(ST) == NS, "staged twiddle layout");
                const float2* wk = tw + G::offset(ST) + k * G::pitch(ST);
#pragma unroll
                for (int r = 1; r < R; r++) {
                    const float2 w = wk[r];
                    wrr[r] = p2(w.x, w.x);
                    wii[r] = p2(-w.y, w.y);
                }
            }
#pragma unroll
            for (int c = 0; c < NC; c++) {
                P2 u[R];
#pragma unroll
                for (int r = 0; r < R; r++) u[r] = p2(v[c][i + r * NB]);
                if constexpr (NS > 1) {
#pragma unroll
                    for (int r = 1; r < R; r++) u[r] = pcmul(u[r], wrr[r], wii[r]);
                }
                if constexpr (R == 8 && ZH && ST == 0) pdft8_zhalf(u);
                else if constexpr (R == 2) pdft2(u);
                else if constexpr (R == 4) pdft4(u);
                else pdft8(u);
#pragma unroll
                for (int q = 0; q < R; q++) v[c][i + q * NB] = f2(u[q]);
            }
        }
        if constexpr (!last) {
#pragma unroll
            for (int c = 0; c < NC; c++) {
                float2* b = ex + ((P + c) & 1) * exs;
#pragma unroll
                for (int i = 0; i < NB; i++) {
                    const int j = t + T * i;
                    const int o = (j / NS) * NS * R + j % NS;
                    if constexpr (NS % (1 << PS) == 0) {  // pad(o + q*NS) = pad(o) + q*pad(NS)
                        float2* base = b + rg_pad<PS>(o);
#pragma unroll
                        for (int q = 0; q < R; q++) base[q * (NS + (NS >> PS))] = v[c][i + q * NB];
                    } else {
#pragma unroll
                        for (int q = 0; q < R; q++) b[rg_pad<PS>(o + q * NS)] = v[c][i + q * NB];
                    }
                }
                __syncthreads();
                if constexpr (T % (1 << PS) == 0) {  // pad(t + T*m) = pad(t) + m*pad(T)
                    const float2* base = b + rg_pad<PS>(t);
#pragma unroll
                    for (int m = 0; m < 8; m++) v[c][m] = base[m * (T + (T >> PS))];
                } else {
#pragma unroll
                    for (int m = 0; m < 8; m++) v[c][m] = b[rg_pad<PS>(t + T * m)];
                }
            }
            rg_stage_seq<L, NC, ST + 1, NS * R, (P + NC) & 1, ZH>(v, t, ex, exs, tw);
        }
    }
}

// Forward FFT of NC lines held by the whole CTA, exchanged one line at a
// time through two buffers (rg_stage_seq); ZH: zero upper half of the input;
// tw: the staged twiddle tables of RgTw<L> (rg_tw_fill).
// The caller must separate it by a barrier from any earlier use of the
// buffers.
template <int L, int NC, bool ZH>
__device__ __forceinline__ void rg_fft_fwd_seq(float2 (&v)[NC][8], int t, float2* ex, int exs,
                                               const float2* __restrict__ tw) {
    static_assert(rg_ok(L), "register FFT needs a power-of-two length >= 8");
    rg_stage_seq<L, NC, 0, 1, 0, ZH>(v, t, ex, exs, tw);
}

// Unnormalised forward FFT (DIR = -1) of NC lines.  All threads that share
// the exchange lines must call it: the whole CTA, or (WARP = true) one warp.
// ZH: the upper half of every line is zero (elements m >= 4 of each thread;
// the first radix-8 butterfly folds them).  PS, MU: exchange padding
// (rg_pad; lines of rg_line<L, PS, MU> slots).  tw: the staged twiddle
// tables of RgTw<L> (rg_tw_fill).  Packed FP32 butterflies (fft_packed.cuh).
template <int L, int NC, bool WARP = false, int PS = 3, bool ZH = false, int MU = 1>
__device__ __forceinline__ void rg_fft_fwd(float2 (&v)[NC][8], int t, float2* ex, int exs,
                                           const float2* __restrict__ tw) {
    static_assert(rg_ok(L), "register FFT needs a power-of-two length >= 8");
    static_assert(!ZH || rg_radix(L, 0) == 8, "the folded first stage is radix 8");
    rg_stage<L, NC, -1, 0, 1, WARP, PS, ZH, MU>(v, t, ex, exs, tw);
}

}  // namespace umag
