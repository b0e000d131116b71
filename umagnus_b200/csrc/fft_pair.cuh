// fft_pair.cuh -- short FFTs held entirely in one thread's registers, with
// twiddle factors that are compile-time constants.
//
// Used for the z transforms of passes A and C (length Pz = 16 or 32), which
// split each column over a pair of adjacent lanes so that no shared-memory
// exchange and no twiddle-table load is needed: the pair's arithmetic is all
// in registers and immediates.
#pragma once
#include "fft.cuh"

namespace umag {

// exp(-2 pi i e / L) evaluated at compile time (Taylor series in double,
// argument reduced to [-pi, pi]); exact enough to round correctly to float.
constexpr double kCtPi = 3.14159265358979323846264338327950288;
constexpr double ct_reduce(double x) { return x > kCtPi ? x - 2 * kCtPi : x; }
constexpr double ct_sin(double x) {
    x = ct_reduce(x);
    double t = x, s = x;
    for (int k = 1; k < 24; k++) {
        t *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
        s += t;
    }
    return s;
}
constexpr double ct_cos(double x) {
    x = ct_reduce(x);
    double t = 1.0, s = 1.0;
    for (int k = 1; k < 24; k++) {
        t *= -x * x / ((2.0 * k - 1.0) * (2.0 * k));
        s += t;
    }
    return s;
}

// v * exp(-2 pi i e / L) (forward direction), with the exact cases spelled out
template <int E, int L> __host__ __device__ __forceinline__ float2 twc(float2 v) {
    constexpr int e = ((E % L) + L) % L;
    if constexpr (e == 0) {
        return v;
    } else if constexpr (4 * e == L) {  // -i
        return make_float2(v.y, -v.x);
    } else if constexpr (2 * e == L) {  // -1
        return make_float2(-v.x, -v.y);
    } else if constexpr (4 * e == 3 * L) {  // +i
        return make_float2(-v.y, v.x);
    } else {
        constexpr float c = (float)ct_cos(2.0 * kCtPi * e / L);
        constexpr float s = -(float)ct_sin(2.0 * kCtPi * e / L);
        return make_float2(v.x * c - v.y * s, v.x * s + v.y * c);
    }
}

template <int L> __host__ __device__ __forceinline__ void reg_dft(float2 (&v)[L]);

// v[n] *= W_L^{n * S} for N <= n < NN (compile-time exponents)
template <int L, int S, int N, int NN> __host__ __device__ __forceinline__ void tw_ramp(float2 (&v)[NN]) {
    if constexpr (N < NN) {
        v[N] = twc<N * S, L>(v[N]);
        tw_ramp<L, S, N + 1, NN>(v);
    }
}

// second half of the L = 4 * B split: for k1 = K1..3, twiddle column k1 by
// W_L^{n2 k1}, DFT_B over n2, scatter to X[k1 + 4 k2]
template <int L, int B, int K1> __host__ __device__ __forceinline__ void dft_cols(float2 (&y)[4][B], float2 (&v)[L]) {
    if constexpr (K1 < 4) {
        float2 z[B];
#pragma unroll
        for (int n2 = 0; n2 < B; n2++) z[n2] = y[K1][n2];
        tw_ramp<L, K1, 0, B>(z);
        reg_dft<B>(z);
#pragma unroll
        for (int k2 = 0; k2 < B; k2++) v[K1 + 4 * k2] = z[k2];
        dft_cols<L, B, K1 + 1>(y, v);
    }
}

// Forward DFT of L in {2, 4, 8, 16, 32} values, natural order in and out.
// L = 4 * B: n = B n1 + n2, k = k1 + 4 k2:
//   X[k1 + 4 k2] = DFT_B over n2 of ( W_L^{n2 k1} * DFT_4 over n1 of x[B n1 + n2] ).
template <int L> __host__ __device__ __forceinline__ void reg_dft(float2 (&v)[L]) {
    if constexpr (L == 2) {
        dft2(v);
    } else if constexpr (L == 4) {
        dft4(v, -1);
    } else if constexpr (L == 8) {
        dft8<float>(v, -1);
    } else {
        static_assert(L == 16 || L == 32, "reg_dft: L in {2, 4, 8, 16, 32}");
        constexpr int B = L / 4;
        float2 y[4][B];  // y[k1][n2] = DFT_4 over n1 of x[B n1 + n2]
#pragma unroll
        for (int n2 = 0; n2 < B; n2++) {
            float2 q[4];
#pragma unroll
            for (int n1 = 0; n1 < 4; n1++) q[n1] = v[B * n1 + n2];
            dft4(q, -1);
#pragma unroll
            for (int k1 = 0; k1 < 4; k1++) y[k1][n2] = q[k1];
        }
        dft_cols<L, B, 0>(y, v);
    }
}

}  // namespace umag
