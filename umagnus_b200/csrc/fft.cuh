// fft.cuh -- in-house shared-memory FFT (Stockham autosort, mixed radix).
//
// A CTA transforms a batch of lines that live in shared memory.  Each stage
// of radix R reads R inputs per butterfly into registers, synchronises, and
// writes the R outputs back in place at their Stockham positions, so one
// buffer suffices and the result comes out in natural order.  Radices 2, 4
// and 8 have dedicated butterflies; 3, 5, 7 and other small primes use the
// line's own twiddle table.  Twiddles are exp(-2 pi i j / L), computed in
// FP64 on the host and stored in the working precision.
//
// No reference code is involved: the reference delegates its FFTs to the
// third-party VkFFT library (cl/vkFFT.h).
#pragma once
#include <cuda_runtime.h>

namespace umag {

template <typename T> struct Cplx;
template <> struct Cplx<float> { using t = float2; };
template <> struct Cplx<double> { using t = double2; };

// Rounding spelled out: on the device every product is either a separate
// correctly rounded multiply or fused into an explicit FMA, so the compiler
// cannot contract the butterflies differently in different kernel
// instantiations -- every instantiation of a transform gives the same bits.
__host__ __device__ __forceinline__ float mul_rn(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
__host__ __device__ __forceinline__ double mul_rn(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
__host__ __device__ __forceinline__ float fma_rn(float a, float b, float c) {
#ifdef __CUDA_ARCH__
    return __fmaf_rn(a, b, c);
#else
    return a * b + c;
#endif
}
__host__ __device__ __forceinline__ double fma_rn(double a, double b, double c) {
#ifdef __CUDA_ARCH__
    return __fma_rn(a, b, c);
#else
    return a * b + c;
#endif
}

template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
    C r;
    r.x = fma_rn(a.x, b.x, -mul_rn(a.y, b.y));
    r.y = fma_rn(a.x, b.y, mul_rn(a.y, b.x));
    return r;
}
template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
// multiply by -i (dir < 0, forward) or +i (dir > 0, inverse)
template <typename C> __host__ __device__ __forceinline__ C mul_mi(C a, int dir) {
    C r;
    if (dir < 0) { r.x = a.y; r.y = -a.x; }
    else { r.x = -a.y; r.y = a.x; }
    return r;
}

constexpr int kMaxStages = 16;

// One FFT length: radix list and twiddle table (device pointer).
template <typename T> struct FftLine {
    int L;
    int nst;
    int R[kMaxStages];
    const typename Cplx<T>::t* tw;  // L entries
};

// Factorisation used for all plans: as many radix-8 stages as possible, the
// remaining power of two as 4s (or one 2 when L is 2 times an odd number),
// then odd primes.
inline int fft_factor(int L, int* R) {
    int n = 0, m = L, twos = 0;
    while (m % 2 == 0) { m /= 2; twos++; }
    int n8 = twos / 3, rem = twos % 3, n4 = 0, n2 = 0;
    if (rem == 2) n4 = 1;
    else if (rem == 1) {
        if (n8 > 0) { n8--; n4 = 2; }
        else n2 = 1;
    }
    for (int i = 0; i < n8; i++) R[n++] = 8;
    for (int i = 0; i < n4; i++) R[n++] = 4;
    for (int i = 0; i < n2; i++) R[n++] = 2;
    for (int p = 3; m > 1; p += 2)
        while (m % p == 0) { R[n++] = p; m /= p; }
    return n;
}
inline int fft_max_radix_ok(const int* R, int n) {
    for (int i = 0; i < n; i++)
        if (R[i] > 13) return 0;
    return 1;
}
inline int fft_min_radix(const int* R, int n) {
    int r = 1 << 30;
    for (int i = 0; i < n; i++) r = R[i] < r ? R[i] : r;
    return n ? r : 1;
}

template <typename C> __host__ __device__ __forceinline__ void dft2(C* v) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
}
template <typename C> __host__ __device__ __forceinline__ void dft4(C* v, int dir) {
    C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    C t2 = cadd(v[1], v[3]), t3 = mul_mi(csub(v[1], v[3]), dir);
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
}
template <typename T, typename C> __host__ __device__ __forceinline__ void dft8(C* v, int dir) {
    C e[4] = {v[0], v[2], v[4], v[6]};
    C o[4] = {v[1], v[3], v[5], v[7]};
    dft4(e, dir);
    dft4(o, dir);
    const T s = (T)0.70710678118654752440084436210485;
    // w8^k, k = 1..3, for the given direction
    C w1, w3;
    w1.x = s; w1.y = dir < 0 ? -s : s;
    w3.x = -s; w3.y = dir < 0 ? -s : s;
    o[1] = cmul(o[1], w1);
    o[2] = mul_mi(o[2], dir);
    o[3] = cmul(o[3], w3);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        v[k] = cadd(e[k], o[k]);
        v[k + 4] = csub(e[k], o[k]);
    }
}
// generic small-prime DFT using the line's twiddle table (L divisible by R)
template <int R, typename C>
__device__ __forceinline__ void dftg(C* v, int dir, const C* __restrict__ tw, int L) {
    C out[R];
    const int step = L / R;
#pragma unroll
    for (int q = 0; q < R; q++) {
        C acc = v[0];
#pragma unroll
        for (int r = 1; r < R; r++) {
            C w = tw[((r * q) % R) * step];
            if (dir > 0) w.y = -w.y;
            acc = cadd(acc, cmul(v[r], w));
        }
        out[q] = acc;
    }
#pragma unroll
    for (int q = 0; q < R; q++) v[q] = out[q];
}

// Register capacity per thread (complex elements held across a stage).
constexpr int kFftCap = 24;
__host__ __device__ constexpr int fft_mb(int R) { return kFftCap / R > 0 ? kFftCap / R : 1; }
// Elements per thread one radix-R stage can hold.
__host__ __device__ constexpr int fft_stage_cap(int R) { return fft_mb(R) * R; }
// Elements per thread every stage of the line can hold: a batch of lines
// may hold at most blockDim * fft_line_cap(...) elements.
template <typename T> __host__ __device__ inline int fft_line_cap(const FftLine<T>& f) {
    int c = 1 << 30;
    for (int i = 0; i < f.nst; i++) {
        int k = fft_stage_cap(f.R[i]);
        c = k < c ? k : c;
    }
    return f.nst ? c : (1 << 30);
}

// Lines of f one batch may hold (>= 1; the host checks that one line fits).
template <typename T> __device__ __forceinline__ int fft_lines_per_batch(const FftLine<T>& f, int ntr) {
    if (f.nst == 0) return ntr > 0 ? ntr : 1;
    long c = (long)blockDim.x * fft_line_cap(f) / f.L;
    if (c < 1) c = 1;
    return c < ntr ? (int)c : (ntr > 0 ? ntr : 1);
}
// Host check: one line of length L fits a CTA of `threads` threads.
template <typename T> inline bool fft_line_fits(const FftLine<T>& f, int threads) {
    return f.nst == 0 || (long)threads * fft_line_cap(f) >= f.L;
}

// One Stockham stage of radix R over ntr lines in shared memory.
// Element j of line t is s[t*ts + j*es].  tfast selects the butterfly
// order (lines fastest, or elements fastest) so that consecutive threads
// touch consecutive addresses.  Requires ntr*L <= blockDim*fft_stage_cap(R):
// every butterfly is read into registers before any is written back.
template <typename T, int R>
__device__ __forceinline__ void fft_stage(typename Cplx<T>::t* s, int ntr, int ts, int es, int L, int Ns,
                                          const typename Cplx<T>::t* __restrict__ tw, int dir, bool tfast) {
    using C = typename Cplx<T>::t;
    constexpr int MB = fft_mb(R);
    const int nb = L / R;
    const int total = ntr * nb;
    const int twstep = L / (Ns * R);
    C v[MB][R];
#pragma unroll
    for (int i = 0; i < MB; i++) {
        int b = threadIdx.x + i * blockDim.x;
        if (b < total) {
            int t = tfast ? b % ntr : b / nb;
            int j = tfast ? b / ntr : b % nb;
            int k = j % Ns;
            C* ln = s + t * ts;
#pragma unroll
            for (int r = 0; r < R; r++) v[i][r] = ln[(j + r * nb) * es];
            if (Ns > 1) {
#pragma unroll
                for (int r = 1; r < R; r++) {
                    C w = tw[r * k * twstep];
                    if (dir > 0) w.y = -w.y;
                    v[i][r] = cmul(v[i][r], w);
                }
            }
            if constexpr (R == 2) dft2(v[i]);
            else if constexpr (R == 4) dft4(v[i], dir);
            else if constexpr (R == 8) dft8<T>(v[i], dir);
            else dftg<R>(v[i], dir, tw, L);
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < MB; i++) {
        int b = threadIdx.x + i * blockDim.x;
        if (b < total) {
            int t = tfast ? b % ntr : b / nb;
            int j = tfast ? b / ntr : b % nb;
            int k = j % Ns;
            int o = (j / Ns) * Ns * R + k;
            C* ln = s + t * ts;
#pragma unroll
            for (int q = 0; q < R; q++) ln[(o + q * Ns) * es] = v[i][q];
        }
    }
    __syncthreads();
}

// In-place unnormalised FFT of ntr lines (dir -1 forward, +1 inverse).
// Must be called by all threads of the CTA with
// ntr*f.L <= blockDim*fft_line_cap(f); ends with a barrier.
template <typename T>
__device__ void smem_fft(typename Cplx<T>::t* s, int ntr, int ts, int es, const FftLine<T>& f, int dir,
                         bool tfast) {
    int Ns = 1;
    for (int st = 0; st < f.nst; st++) {
        const int R = f.R[st];
        switch (R) {
        case 2: fft_stage<T, 2>(s, ntr, ts, es, f.L, Ns, f.tw, dir, tfast); break;
        case 3: fft_stage<T, 3>(s, ntr, ts, es, f.L, Ns, f.tw, dir, tfast); break;
        case 4: fft_stage<T, 4>(s, ntr, ts, es, f.L, Ns, f.tw, dir, tfast); break;
        case 5: fft_stage<T, 5>(s, ntr, ts, es, f.L, Ns, f.tw, dir, tfast); break;
        case 7: fft_stage<T, 7>(s, ntr, ts, es, f.L, Ns, f.tw, dir, tfast); break;
        case 8: fft_stage<T, 8>(s, ntr, ts, es, f.L, Ns, f.tw, dir, tfast); break;
        case 11: fft_stage<T, 11>(s, ntr, ts, es, f.L, Ns, f.tw, dir, tfast); break;
        case 13: fft_stage<T, 13>(s, ntr, ts, es, f.L, Ns, f.tw, dir, tfast); break;
        default: break;  // rejected at plan time
        }
        Ns *= R;
    }
    __syncthreads();
}

}  // namespace umag
