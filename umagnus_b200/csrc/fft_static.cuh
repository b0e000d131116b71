// fft_static.cuh -- shared-memory Stockham FFT with a compile-time plan.
//
// Same algorithm as fft.cuh (in-place Stockham stages through registers),
// but the length, radix sequence, batch size, strides, thread count and
// direction are template parameters, so every index computation is a
// constant shift/multiply, every register array is fully unrolled, and no
// code for unused radices is generated.  Used by the hot demag passes for
// the sizes the benchmarks run; other sizes use fft.cuh.
#pragma once
#include "fft.cuh"

namespace umag {

// radix plan: 8s first, then the remaining power of two as 4/4, 4 or 2,
// then 3, 5, 7 (the same factorisation as fft_factor)
constexpr int sp_twos(int L) { return (L % 2 == 0) ? 1 + sp_twos(L / 2) : 0; }
constexpr int sp_odd(int L) { return (L % 2 == 0) ? sp_odd(L / 2) : L; }
constexpr int sp_n8(int L) {
    return (sp_twos(L) % 3 == 1 && sp_twos(L) >= 4) ? sp_twos(L) / 3 - 1 : sp_twos(L) / 3;
}
constexpr int sp_n4(int L) {
    return (sp_twos(L) % 3 == 2) ? 1 : ((sp_twos(L) % 3 == 1 && sp_twos(L) >= 4) ? 2 : 0);
}
constexpr int sp_n2(int L) { return (sp_twos(L) == 1) ? 1 : 0; }
constexpr int sp_count(int m, int p) { return (m % p == 0) ? 1 + sp_count(m / p, p) : 0; }
constexpr int sp_nst(int L) {
    return sp_n8(L) + sp_n4(L) + sp_n2(L) + sp_count(sp_odd(L), 3) + sp_count(sp_odd(L), 5) +
           sp_count(sp_odd(L), 7);
}
constexpr int sp_radix(int L, int s) {
    return s < sp_n8(L) ? 8
         : s < sp_n8(L) + sp_n4(L) ? 4
         : s < sp_n8(L) + sp_n4(L) + sp_n2(L) ? 2
         : s < sp_n8(L) + sp_n4(L) + sp_n2(L) + sp_count(sp_odd(L), 3) ? 3
         : s < sp_n8(L) + sp_n4(L) + sp_n2(L) + sp_count(sp_odd(L), 3) + sp_count(sp_odd(L), 5) ? 5
         : 7;
}
constexpr int sp_rest(int m) {
    return m % 3 == 0 ? sp_rest(m / 3) : m % 5 == 0 ? sp_rest(m / 5) : m % 7 == 0 ? sp_rest(m / 7) : m;
}
constexpr bool sp_supported(int L) { return L >= 1 && sp_rest(sp_odd(L)) == 1; }
// largest divisor of n that is <= cap (>= 1)
constexpr int sp_divisor_le(int n, int cap) { return cap <= 1 ? 1 : (n % cap == 0 ? cap : sp_divisor_le(n, cap - 1)); }

template <int R, int DIR, typename C>
__device__ __forceinline__ void sp_dft(C* v, const C* __restrict__ tw, int L) {
    if constexpr (R == 2) dft2(v);
    else if constexpr (R == 4) dft4(v, DIR);
    else if constexpr (R == 8) dft8<decltype(v[0].x)>(v, DIR);
    else dftg<R>(v, DIR, tw, L);
}

// One stage; recursion over the stage index ST with NS = product of the
// radices already applied.  Requires NTR*L <= NT*fft_stage_cap(R) so every
// butterfly is held in registers across the barrier.
template <typename C, int L, int NTR, int NT, int TS, int ES, bool TFAST, int DIR, int ST, int NS>
__device__ __forceinline__ void sp_stage(C* s, const C* __restrict__ tw) {
    if constexpr (ST < sp_nst(L)) {
        constexpr int R = sp_radix(L, ST);
        constexpr int NB = L / R;
        constexpr int TOTAL = NTR * NB;
        constexpr int MB = (TOTAL + NT - 1) / NT;
        constexpr int TWS = L / (NS * R);
        static_assert(MB * R <= 32, "too many elements per thread for one stage");
        C v[MB][R];
#pragma unroll
        for (int i = 0; i < MB; i++) {
            const int b = threadIdx.x + i * NT;
            if (TOTAL % NT == 0 || b < TOTAL) {
                const int t = TFAST ? b % NTR : b / NB;
                const int j = TFAST ? b / NTR : b % NB;
                const int k = j % NS;
                const C* ln = s + t * TS;
#pragma unroll
                for (int r = 0; r < R; r++) v[i][r] = ln[(j + r * NB) * ES];
                if constexpr (NS > 1) {
#pragma unroll
                    for (int r = 1; r < R; r++) {
                        C w = tw[r * k * TWS];
                        if (DIR > 0) w.y = -w.y;
                        v[i][r] = cmul(v[i][r], w);
                    }
                }
                sp_dft<R, DIR>(v[i], tw, L);
            }
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < MB; i++) {
            const int b = threadIdx.x + i * NT;
            if (TOTAL % NT == 0 || b < TOTAL) {
                const int t = TFAST ? b % NTR : b / NB;
                const int j = TFAST ? b / NTR : b % NB;
                const int k = j % NS;
                const int o = (j / NS) * NS * R + k;
                C* ln = s + t * TS;
#pragma unroll
                for (int q = 0; q < R; q++) ln[(o + q * NS) * ES] = v[i][q];
            }
        }
        __syncthreads();
        sp_stage<C, L, NTR, NT, TS, ES, TFAST, DIR, ST + 1, NS * R>(s, tw);
    }
}

// In-place unnormalised FFT of NTR lines of length L in shared memory,
// element j of line t at s[t*TS + j*ES]; tw = exp(-2 pi i j/L), j < L.
template <typename C, int L, int NTR, int NT, int TS, int ES, bool TFAST, int DIR>
__device__ __forceinline__ void sfft(C* s, const C* __restrict__ tw) {
    sp_stage<C, L, NTR, NT, TS, ES, TFAST, DIR, 0, 1>(s, tw);
}

}  // namespace umag
