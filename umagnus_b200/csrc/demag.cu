// demag.cu -- demag convolution plan (opencl/conv_demag.go replacement).
//
// Layout in HBM (float32 path, one plan per mesh):
//   spec : complex half-spectrum of the three scaled magnetisation components,
//          [c][kz][y][kx] with kx in [0, Px/2] (row pitch Lx), kz in [0, Pz),
//          y in [0, Ny) -- only the Ny rows that carry data are stored; the
//          zero padding in y never reaches memory.
//   K    : real kernel spectrum, six float32 arrays [kz'][ky'][kx] over the
//          non-redundant (Px/2+1)(Py/2+1)(Pz/2+1) block, scaled by 1/(PxPyPz)
//          (the reference layout of kernmulrsymm3d.cl and conv_demag.go:157-164).
// Three passes per evaluation:
//   A (per y, per component): scale m by MU0*Ms*vol, real-to-complex FFT
//     along x (padded length Px, packed as a length-Px/2 complex FFT), then
//     the forward FFT along z (padded length Pz) -> spec.
//   B (per kz, per block of kx): forward FFT along y (padded length Py),
//     3x3 symmetric kernel multiply, inverse FFT along y; rows y < Ny back.
//   C (per y, per component): inverse FFT along z, keep z < Nz, complex-to-
//     real inverse along x, keep x < Nx -> B (overwritten).
// Zero padding is never materialised in HBM; the padded real buffers of the
// reference (fftRBuf, conv_demag.go:143-149) do not exist here.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "demag.cuh"
#include "fft.cuh"
#include "newell.cuh"
#include "tile.cuh"

namespace umag {

static constexpr double kMu0 = 4 * 3.1415926535897932384626433 * 1e-7;  // clh/constants.clh:5

// ------------------------------------------------------------------ twiddles
template <typename C> static std::vector<C> twiddles(int L, int count) {
    std::vector<C> t(count);
    for (int j = 0; j < count; j++) {
        double a = -2.0 * M_PI * (double)j / (double)L;
        t[j].x = (decltype(t[j].x))cos(a);
        t[j].y = (decltype(t[j].y))sin(a);
    }
    return t;
}

template <typename T>
static int make_line(int L, FftLine<T>& f, typename Cplx<T>::t** dev_tw) {
    f.L = L;
    f.nst = L > 1 ? fft_factor(L, f.R) : 0;
    if (!fft_max_radix_ok(f.R, f.nst))
        return set_error(UMAG_E_UNSUPPORTED, "FFT length %d has a prime factor above 13", L);
    auto t = twiddles<typename Cplx<T>::t>(L, L);
    UMAG_CUDA(cudaMalloc((void**)dev_tw, sizeof(t[0]) * (L > 0 ? L : 1)));
    UMAG_CUDA(cudaMemcpyAsync(*dev_tw, t.data(), sizeof(t[0]) * L, cudaMemcpyHostToDevice, ctx().stream));
    UMAG_CUDA(cudaStreamSynchronize(ctx().stream));  // t is freed on return
    f.tw = *dev_tw;
    return UMAG_OK;
}

// ================================================================== Newell (FP64)
struct NewellArgs {
    int P[3], ext[3];
    int r1[3], r2[3];  // kernelRanges (mag/demagkernel.go:339-352): the periodic images are r1..r2
    double dx, dy, dz, scale, arad2;
    int use_asym;
    newell::Expansion exx, exy, exz, eyy, eyz, ezz;
};

// first and last image index k with w + k P in [r1, r2]
__device__ __forceinline__ void image_range(int w, int P, int r1, int r2, int& k0, int& k1) {
    k0 = (int)floor((double)(r1 - w) / P);
    if (w + k0 * P < r1) k0++;
    k1 = (int)floor((double)(r2 - w) / P);
}

// One thread per octant point (x, y, z) in [0, P/2] of the padded grid
// (mag/newellDemagKernel.go:1166-1252): the tensor at every periodic image
// x + kx Px, ... inside the kernel ranges, summed in the reference's loop
// order (z, then y, then x ascending).  Without PBC the only image is k = 0.
// K order: xx yy zz yz xz xy.
__global__ void k_newell_octant(double* K0, double* K1, double* K2, double* K3, double* K4, double* K5,
                                NewellArgs a) {
    long n = (long)a.ext[0] * a.ext[1] * a.ext[2];
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int xw = (int)(i % a.ext[0]);
        const int yw = (int)((i / a.ext[0]) % a.ext[1]);
        const int zw = (int)(i / ((long)a.ext[0] * a.ext[1]));
        int kx0, kx1, ky0, ky1, kz0, kz1;
        image_range(xw, a.P[0], a.r1[0], a.r2[0], kx0, kx1);
        image_range(yw, a.P[1], a.r1[1], a.r2[1], ky0, ky1);
        image_range(zw, a.P[2], a.r1[2], a.r2[2], kz0, kz1);
        double acc[6] = {0, 0, 0, 0, 0, 0};
        for (int kz = kz0; kz <= kz1; kz++)
            for (int ky = ky0; ky <= ky1; ky++)
                for (int kx = kx0; kx <= kx1; kx++) {
                    const int x = xw + kx * a.P[0], y = yw + ky * a.P[1], z = zw + kz * a.P[2];
                    const double Rx = x * a.dx, Ry = y * a.dy, Rz = z * a.dz;
                    double v[6];
                    if (a.use_asym && Rx * Rx > a.arad2 - Rz * Rz - Ry * Ry) {
                        v[0] = -newell::expansion_eval(a.exx, Rx, Ry, Rz);
                        v[5] = -newell::expansion_eval(a.exy, Rx, Ry, Rz);
                        v[4] = -newell::expansion_eval(a.exz, Rx, Rz, Ry);
                        v[1] = -newell::expansion_eval(a.eyy, Ry, Rx, Rz);
                        v[3] = -newell::expansion_eval(a.eyz, Ry, Rz, Rx);
                        v[2] = -newell::expansion_eval(a.ezz, Rz, Ry, Rx);
                    } else {
                        v[0] = newell::sda00(Rx, Ry, Rz, a.dx, a.dy, a.dz) * a.scale;
                        v[5] = newell::sda01(Rx, Ry, Rz, a.dx, a.dy, a.dz) * a.scale;
                        v[4] = newell::sda01(Rx, Rz, Ry, a.dx, a.dz, a.dy) * a.scale;
                        v[1] = newell::sda00(Ry, Rx, Rz, a.dy, a.dx, a.dz) * a.scale;
                        v[3] = newell::sda01(Ry, Rz, Rx, a.dy, a.dz, a.dx) * a.scale;
                        v[2] = newell::sda00(Rz, Ry, Rx, a.dz, a.dy, a.dx) * a.scale;
                    }
                    for (int c = 0; c < 6; c++) acc[c] += v[c];
                }
        long I = ((long)zw * a.P[1] + yw) * a.P[0] + xw;
        K0[I] = acc[0]; K1[I] = acc[1]; K2[I] = acc[2]; K3[I] = acc[3]; K4[I] = acc[4]; K5[I] = acc[5];
    }
}

// Fill the rest of the padded grid from the octant with the mirror signs
// (mag/newellDemagKernel.go:1254-1298); Nyquist planes stay zero.
__global__ void k_newell_mirror(double* K0, double* K1, double* K2, double* K3, double* K4, double* K5,
                                int Px, int Py, int Pz) {
    long n = (long)Px * Py * Pz;
    double* K[6] = {K0, K1, K2, K3, K4, K5};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        int x = (int)(i % Px), y = (int)((i / Px) % Py), z = (int)(i / ((long)Px * Py));
        bool fx = x > Px / 2, fy = y > Py / 2, fz = z > Pz / 2;
        if (!fx && !fy && !fz) continue;
        int sx = fx ? Px - x : x, sy = fy ? Py - y : y, sz = fz ? Pz - z : z;
        long S = ((long)sz * Py + sy) * Px + sx;
        double gx = fx ? -1.0 : 1.0, gy = fy ? -1.0 : 1.0, gz = fz ? -1.0 : 1.0;
        const double sgn[6] = {1.0, 1.0, 1.0, gy * gz, gx * gz, gx * gy};
#pragma unroll
        for (int c = 0; c < 6; c++) K[c][i] = sgn[c] * K[c][S];
    }
}

// ================================================================== FP64 line FFTs
// FFT along one axis of a complex P-grid; a CTA transforms G lines.
template <typename T>
__global__ void k_fft_axis(typename Cplx<T>::t* data, FftLine<T> f, int Px, int Py, int Pz, int axis, int G,
                           int dir) {
    using C = typename Cplx<T>::t;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s = reinterpret_cast<C*>(smem_raw);
    const int L = f.L;
    long base;
    long es;  // element stride in data
    int gcount;
    if (axis == 0) {
        long row0 = (long)blockIdx.x * G;
        long rows = (long)Py * Pz;
        gcount = (int)((rows - row0) < G ? (rows - row0) : G);
        base = row0 * Px;
        es = 1;
        // s[t*L + j]
        for (int e = threadIdx.x; e < gcount * L; e += blockDim.x) s[e] = data[base + e];
        __syncthreads();
        int cap = fft_lines_per_batch(f, gcount);
        for (int t0 = 0; t0 < gcount; t0 += cap) {
            int nt = gcount - t0 < cap ? gcount - t0 : cap;
            smem_fft<T>(s + t0 * L, nt, L, 1, f, dir, false);
        }
        for (int e = threadIdx.x; e < gcount * L; e += blockDim.x) data[base + e] = s[e];
        return;
    }
    // axis 1 or 2: G consecutive x at fixed (z) or (y); s[j*G + t]
    int xg = (Px + G - 1) / G;
    int x0 = (blockIdx.x % xg) * G;
    int other = blockIdx.x / xg;
    gcount = Px - x0 < G ? Px - x0 : G;
    if (axis == 1) { base = (long)other * Py * Px + x0; es = Px; }
    else { base = (long)other * Px + x0; es = (long)Px * Py; }
    for (int e = threadIdx.x; e < L * G; e += blockDim.x) {
        int j = e / G, t = e % G;
        C v;
        v.x = 0; v.y = 0;
        if (t < gcount) v = data[base + j * es + t];
        s[e] = v;
    }
    __syncthreads();
    int cap = fft_lines_per_batch(f, G);
    for (int t0 = 0; t0 < G; t0 += cap) {
        int nt = G - t0 < cap ? G - t0 : cap;
        smem_fft<T>(s + t0, nt, 1, G, f, dir, true);
    }
    for (int e = threadIdx.x; e < L * G; e += blockDim.x) {
        int j = e / G, t = e % G;
        if (t < gcount) data[base + j * es + t] = s[e];
    }
}

__global__ void k_real_to_cplx(const double* src, double2* dst, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        dst[i] = make_double2(src[i], 0.0);
}

// Real parts of the non-redundant block, scaled, rows of pitch Kp (the pad
// columns are zero) or, when blocked, 4-column blocks [z][x/4][y][x%4];
// max |imag| into *maximg.
__global__ void k_extract_spectrum(const double2* a, float* out, int Px, int Py, int Pz, int Kp, int blocked,
                                   double scale, unsigned long long* maximg) {
    int hx = Px / 2 + 1, hy = Py / 2 + 1, hz = Pz / 2 + 1;
    long n = (long)Kp * hy * hz;
    double mi = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        int x, y, z;
        if (blocked) {
            const long q = i >> 2;
            y = (int)(q % hy);
            const long zb = q / hy;
            x = (int)(zb % (Kp >> 2)) * 4 + (int)(i & 3);
            z = (int)(zb / (Kp >> 2));
        } else {
            x = (int)(i % Kp); y = (int)((i / Kp) % hy); z = (int)(i / ((long)Kp * hy));
        }
        if (x >= hx) { out[i] = 0.f; continue; }
        double2 v = a[((long)z * Py + y) * Px + x];
        out[i] = (float)(v.x * scale);
        mi = fmax(mi, fabs(v.y));
    }
    atomicMax(maximg, (unsigned long long)__double_as_longlong(mi));
}

// ================================================================== float passes
__global__ void __launch_bounds__(kPassThreads) k_pass_a(PassArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* X1 = reinterpret_cast<float2*>(smem_raw);        // [Nz][HxP]
    float2* Z2 = X1 + a.Nz * a.HxP;                           // [Pz][W]
    if (a.active && !*a.active) return;
    const int y = blockIdx.x, c = blockIdx.y;
    const int M = a.M;
    const float* __restrict__ m =
        a.m_ind ? (a.m_sel ? *a.m_ind_w : *a.m_ind) + (long)c * a.ncell : a.m[c];
    // 1. load, scale (copypadmul2.cl:13-20) and pack pairs of reals
    for (int e = threadIdx.x; e < a.Nz * M; e += blockDim.x) {
        int z = e / M, n = e % M;
        float2 v = make_float2(0.f, 0.f);
#pragma unroll
        for (int h = 0; h < 2; h++) {
            int x = 2 * n + h;
            if (x < a.Nx) {
                int i = (z * a.Ny + y) * a.Nx + x;
                float fac = a.Ms == nullptr ? a.Ms_mul : __fmul_rn(a.Ms_mul, __ldg(a.Ms + i));
                float bsat = (float)(kMu0 * (double)fac);
                float w = a.vol == nullptr ? 1.0f : __fmul_rn(1.0f, __ldg(a.vol + i));
                float val = __fmul_rn(__fmul_rn(bsat, w), __ldg(m + i));
                if (h == 0) v.x = val; else v.y = val;
            }
        }
        X1[z * a.HxP + n] = v;
    }
    __syncthreads();
    // 2. complex FFT of length M on every row
    {
        int cap = fft_lines_per_batch(a.fx, a.Nz);
        for (int t0 = 0; t0 < a.Nz; t0 += cap) {
            int nt = a.Nz - t0 < cap ? a.Nz - t0 : cap;
            smem_fft<float>(X1 + t0 * a.HxP, nt, a.HxP, 1, a.fx, -1, false);
        }
    }
    // 3. unpack to the R2C half spectrum X[0..M]
    const int half = M / 2;
    for (int e = threadIdx.x; e < a.Nz * (half + 1); e += blockDim.x) {
        int z = e / (half + 1), k = e % (half + 1);
        float2* row = X1 + z * a.HxP;
        int k2 = M - k;
        float2 A = row[k], Bc = row[k2 == M ? 0 : k2];
        Bc.y = -Bc.y;  // conj(Z[M-k])
        float2 E = make_float2(0.5f * (A.x + Bc.x), 0.5f * (A.y + Bc.y));
        float2 D = make_float2(0.5f * (A.x - Bc.x), 0.5f * (A.y - Bc.y));
        float2 O = make_float2(D.y, -D.x);  // -i * D
        float2 W = a.twr[k];
        float2 WO = make_float2(W.x * O.x - W.y * O.y, W.x * O.y + W.y * O.x);
        float2 Xk = make_float2(E.x + WO.x, E.y + WO.y);
        float2 Xm = make_float2(E.x - WO.x, -(E.y - WO.y));  // conj(E - W^k O)
        row[k] = Xk;
        row[k2] = Xm;
    }
    __syncthreads();
    // 4. z transform per block of kx columns, written to spec
    float2* out = a.spec + (long)c * a.Pz * a.Ny * a.Lx + (long)y * a.Lx;
    const long kzs = (long)a.Ny * a.Lx;
    if (a.Pz == 1) {
        for (int k = threadIdx.x; k < a.Hx; k += blockDim.x) out[k] = X1[k];
        return;
    }
    const int W = kChunkW;
    for (int kx0 = 0; kx0 < a.Hx; kx0 += W) {
        for (int e = threadIdx.x; e < a.Pz * W; e += blockDim.x) {
            int z = e / W, w = e % W;
            float2 v = make_float2(0.f, 0.f);
            if (z < a.Nz && kx0 + w < a.Hx) v = X1[z * a.HxP + kx0 + w];
            Z2[e] = v;
        }
        __syncthreads();
        smem_fft<float>(Z2, W, 1, W, a.fz, -1, true);
        for (int e = threadIdx.x; e < a.Pz * W; e += blockDim.x) {
            int kz = e / W, w = e % W;
            if (kx0 + w < a.Hx) out[kz * kzs + kx0 + w] = Z2[e];
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kPassBThreads) k_pass_b(PassArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (a.active && !*a.active) return;
    float2* S = reinterpret_cast<float2*>(smem_raw);  // [Py][3*WB]
    const int WB = a.WB, W3 = 3 * WB;
    const int kx0 = blockIdx.x * WB, kz = blockIdx.y;
    const long cs = (long)a.Pz * a.Ny * a.Lx;  // component stride
    const float2* in = a.spec + (long)kz * a.Ny * a.Lx + kx0;
    for (int e = threadIdx.x; e < a.Py * W3; e += blockDim.x) {
        int yy = e / W3, r = e % W3, c = r / WB, w = r % WB;
        float2 v = make_float2(0.f, 0.f);
        if (yy < a.Ny && kx0 + w < a.Hx) v = in[c * cs + (long)yy * a.Lx + w];
        S[e] = v;
    }
    __syncthreads();
    smem_fft<float>(S, W3, 1, W3, a.fy, -1, true);
    // kernel multiply (kernmulrsymm3d.cl:41-90): mirror ky, kz into the stored block
    const int hy = a.Py / 2 + 1, hx = a.Hx;
    int kzm = kz;
    float sz = 1.f;
    if (kz > a.Pz / 2) { kzm = a.Pz - kz; sz = -1.f; }
    for (int e = threadIdx.x; e < a.Py * WB; e += blockDim.x) {
        int ky = e / WB, w = e % WB;
        int kx = kx0 + w;
        if (kx >= hx) continue;
        int kym = ky;
        float sy = 1.f;
        if (ky > a.Py / 2) { kym = a.Py - ky; sy = -1.f; }
        long I = ((long)kzm * hy + kym) * a.Kp + kx;
        float Kxx = __ldg(a.K[0] + I), Kyy = __ldg(a.K[1] + I), Kzz = __ldg(a.K[2] + I);
        float Kxy = __ldg(a.K[5] + I) * sy;
        float Kyz = 0.f, Kxz = 0.f;
        if (a.K[3] != nullptr) {
            Kyz = __ldg(a.K[3] + I) * (sy * sz);
            Kxz = __ldg(a.K[4] + I) * sz;
        }
        float2* row = S + ky * W3;
        float2 mx = row[w], my = row[WB + w], mz = row[2 * WB + w];
        row[w] = make_float2(mx.x * Kxx + my.x * Kxy + mz.x * Kxz, mx.y * Kxx + my.y * Kxy + mz.y * Kxz);
        row[WB + w] = make_float2(mx.x * Kxy + my.x * Kyy + mz.x * Kyz, mx.y * Kxy + my.y * Kyy + mz.y * Kyz);
        row[2 * WB + w] = make_float2(mx.x * Kxz + my.x * Kyz + mz.x * Kzz, mx.y * Kxz + my.y * Kyz + mz.y * Kzz);
    }
    __syncthreads();
    smem_fft<float>(S, W3, 1, W3, a.fy, +1, true);
    float2* outp = a.spec + (long)kz * a.Ny * a.Lx + kx0;
    for (int e = threadIdx.x; e < a.Ny * W3; e += blockDim.x) {
        int yy = e / W3, r = e % W3, c = r / WB, w = r % WB;
        if (kx0 + w < a.Hx) outp[c * cs + (long)yy * a.Lx + w] = S[e];
    }
}

__global__ void __launch_bounds__(kPassThreads) k_pass_c(PassArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* X1 = reinterpret_cast<float2*>(smem_raw);  // [Nz][HxP]
    float2* Z2 = X1 + a.Nz * a.HxP;                    // [Pz][W]
    if (a.active && !*a.active) return;
    const int y = blockIdx.x, c = blockIdx.y;
    const int M = a.M;
    const float2* in = a.spec + (long)c * a.Pz * a.Ny * a.Lx + (long)y * a.Lx;
    const long kzs = (long)a.Ny * a.Lx;
    // 1. inverse z transform per block of columns, keep z < Nz
    if (a.Pz == 1) {
        for (int k = threadIdx.x; k < a.Hx; k += blockDim.x) X1[k] = in[k];
    } else {
        const int W = kChunkW;
        for (int kx0 = 0; kx0 < a.Hx; kx0 += W) {
            for (int e = threadIdx.x; e < a.Pz * W; e += blockDim.x) {
                int kz = e / W, w = e % W;
                Z2[e] = (kx0 + w < a.Hx) ? in[kz * kzs + kx0 + w] : make_float2(0.f, 0.f);
            }
            __syncthreads();
            smem_fft<float>(Z2, W, 1, W, a.fz, +1, true);
            for (int e = threadIdx.x; e < a.Nz * W; e += blockDim.x) {
                int z = e / W, w = e % W;
                if (kx0 + w < a.Hx) X1[z * a.HxP + kx0 + w] = Z2[e];
            }
            __syncthreads();
        }
    }
    __syncthreads();
    // 2. pack the half spectrum into a length-M complex sequence (C2R)
    const int half = M / 2;
    for (int e = threadIdx.x; e < a.Nz * (half + 1); e += blockDim.x) {
        int z = e / (half + 1), k = e % (half + 1);
        float2* row = X1 + z * a.HxP;
        int k2 = M - k;
        float2 Xk = row[k], Xm = row[k2];
        if (k == 0) { Xk.y = 0.f; Xm.y = 0.f; }
        // Z[k] = (X[k] + conj X[M-k]) + i conj(W^k) (X[k] - conj X[M-k])
        float2 W = a.twr[k];
        float2 Wc = make_float2(W.x, -W.y);
        float2 S1 = make_float2(Xk.x + Xm.x, Xk.y - Xm.y);
        float2 D1 = make_float2(Xk.x - Xm.x, Xk.y + Xm.y);
        float2 T1 = make_float2(Wc.x * D1.x - Wc.y * D1.y, Wc.x * D1.y + Wc.y * D1.x);
        float2 Zk = make_float2(S1.x - T1.y, S1.y + T1.x);
        // Z[M-k] = (X[M-k] + conj X[k]) + i conj(W^(M-k)) (X[M-k] - conj X[k]),  conj(W^(M-k)) = -W^k
        float2 S2 = make_float2(Xm.x + Xk.x, Xm.y - Xk.y);
        float2 D2 = make_float2(Xm.x - Xk.x, Xm.y + Xk.y);
        float2 T2 = make_float2(-(W.x * D2.x - W.y * D2.y), -(W.x * D2.y + W.y * D2.x));
        float2 Zm = make_float2(S2.x - T2.y, S2.y + T2.x);
        if (k == 0) {
            row[0] = Zk;
        } else {
            row[k] = Zk;
            row[k2] = Zm;
        }
    }
    __syncthreads();
    // 3. inverse complex FFT of every row
    {
        int cap = fft_lines_per_batch(a.fx, a.Nz);
        for (int t0 = 0; t0 < a.Nz; t0 += cap) {
            int nt = a.Nz - t0 < cap ? a.Nz - t0 : cap;
            smem_fft<float>(X1 + t0 * a.HxP, nt, a.HxP, 1, a.fx, +1, false);
        }
    }
    // 4. unpack even/odd samples and crop (copyunpad.cl), overwrite B
    float* __restrict__ B = a.B[c];
    for (int e = threadIdx.x; e < a.Nz * a.Nx; e += blockDim.x) {
        int z = e / a.Nx, x = e % a.Nx;
        float2 v = X1[z * a.HxP + (x >> 1)];
        B[(z * a.Ny + y) * a.Nx + x] = (x & 1) ? v.y : v.x;
    }
}

// ================================================================== plan
static size_t pass_ac_smem(const umag_demag* d) {
    return sizeof(float2) * ((size_t)d->N[2] * d->HxP + (d->P[2] > 1 ? (size_t)d->P[2] * kChunkW : 0));
}
static size_t pass_b_smem(const umag_demag* d) { return sizeof(float2) * (size_t)d->P[1] * 3 * d->WB; }

// Tensor map for pass C's slab loads (PassArgs::slab_map): the blocked
// spectrum as floats (8 = four complex columns, y, kx/4, kz, component), a
// box of one (y, component) slab; only where the register passes use the
// slab shape and the slab fits the x/z scratch it borrows.  Without it pass C
// keeps its plain loads.
static void slab_setup(umag_demag* d) {
    const FastPasses& f = d->fast;
    if (!d->use_fast || !f.blocked || !f.slab_ok || d->Lx % 4 != 0) return;
    const int KB = d->Lx / 4, Ny = d->N[1], Pz = d->P[2];
    const size_t bytes = sizeof(float2) * 4 * (size_t)KB * Pz;
    if (bytes + 128 > f.ac_scratch || KB > 256 || Pz > 256) return;  // + the alignment slack
    EncodeTiledFn fn = encode_tiled();
    if (!fn || reinterpret_cast<uintptr_t>(d->spec) % 16 != 0) return;
    const cuuint64_t row = sizeof(float2) * 4;  // 32 bytes: four complex columns
    const cuuint64_t dims[5] = {8, (cuuint64_t)Ny, (cuuint64_t)KB, (cuuint64_t)Pz, 3};
    const cuuint64_t strides[4] = {row, row * Ny, row * Ny * KB, row * Ny * KB * Pz};
    const cuuint32_t box[5] = {8, 1, (cuuint32_t)KB, (cuuint32_t)Pz, 1};
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    CUtensorMap map;
    if (fn(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, d->spec, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
        CUDA_SUCCESS)
        return;
    CUtensorMap* dev = nullptr;
    if (cudaMalloc(&dev, sizeof(CUtensorMap)) != cudaSuccess) return;
    if (cudaMemcpyAsync(dev, &map, sizeof(map), cudaMemcpyHostToDevice, ctx().stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx().stream) != cudaSuccess) {
        cudaFree(dev);
        return;
    }
    d->slab_map = dev;
}

static int plan_common(umag_demag* d) {
    for (int i = 0; i < 3; i++) UMAG_REQUIRE(d->N[i] > 0, "mesh size must be positive");
    for (int i = 0; i < 3; i++) UMAG_REQUIRE(d->pbc[i] >= 0, "PBC repetitions must be non-negative");
    // mag/demagkernel.go:404-420: no padding along a periodic axis
    d->P[0] = d->pbc[0] ? d->N[0] : 2 * d->N[0];
    d->P[1] = d->pbc[1] ? d->N[1] : 2 * d->N[1];
    d->P[2] = d->pbc[2] ? d->N[2] : (d->N[2] > 5 ? 2 * d->N[2] : 2 * d->N[2] - 1);
    if (d->P[0] % 2 != 0)
        return set_error(UMAG_E_UNSUPPORTED, "periodic x needs an even Nx (the x transform packs pairs of reals)");
    d->M = d->P[0] / 2;
    d->Hx = d->M + 1;
    d->HxP = d->M + 1;
    d->Lx = (d->Hx + 3) / 4 * 4;
    d->is2d = d->N[2] == 1;
    // pass B column block: 3*WB*Py elements must fit the register capacity
    int wb = 8;
    FftLine<float> probe{};
    probe.L = d->P[1];
    probe.nst = fft_factor(d->P[1], probe.R);
    int capy = fft_line_cap(probe);
    while (wb > 1 && 3 * wb * d->P[1] > kPassBThreads * capy) wb /= 2;
    if (3 * wb * d->P[1] > kPassBThreads * capy)
        return set_error(UMAG_E_UNSUPPORTED, "padded Ny = %d too large for pass B", d->P[1]);
    d->WB = wb;
    if (pass_ac_smem(d) > 227 * 1024)
        return set_error(UMAG_E_UNSUPPORTED, "Nz*(Nx+1) too large for the x/z passes (%zu bytes smem)",
                         pass_ac_smem(d));
    if (pass_b_smem(d) > 227 * 1024) return set_error(UMAG_E_UNSUPPORTED, "pass B shared memory too large");
    float2* tw;
    UMAG_TRY(make_line<float>(d->M, d->fx, &tw)); d->tw_dev.push_back(tw);
    UMAG_TRY(make_line<float>(d->P[1], d->fy, &tw)); d->tw_dev.push_back(tw);
    UMAG_TRY(make_line<float>(d->P[2], d->fz, &tw)); d->tw_dev.push_back(tw);
    if (!fft_line_fits(d->fx, kPassThreads))
        return set_error(UMAG_E_UNSUPPORTED, "Nx = %d too large for the x pass", d->N[0]);
    if (d->P[2] > 1 && (long)kChunkW * d->P[2] > (long)kPassThreads * fft_line_cap(d->fz))
        return set_error(UMAG_E_UNSUPPORTED, "Nz = %d too large for the z transform", d->N[2]);
    auto twr = twiddles<float2>(d->P[0], d->M > 1 ? d->M : 2);  // exp(-2 pi i k / Px), k < Px/2
    UMAG_CUDA(cudaMalloc(&d->twr, sizeof(float2) * twr.size()));
    UMAG_CUDA(cudaMemcpyAsync(d->twr, twr.data(), sizeof(float2) * twr.size(), cudaMemcpyHostToDevice, ctx().stream));
    UMAG_CUDA(cudaStreamSynchronize(ctx().stream));
    size_t spec_elems = (size_t)3 * d->P[2] * d->N[1] * d->Lx;
    UMAG_CUDA(cudaMalloc(&d->spec, sizeof(float2) * spec_elems));
    UMAG_CUDA(cudaMemsetAsync(d->spec, 0, sizeof(float2) * spec_elems, ctx().stream));
    d->Kp = (d->Hx + 3) / 4 * 4;
    size_t kn = (size_t)d->Kp * (d->P[1] / 2 + 1) * (d->P[2] / 2 + 1);
    d->Kn = kn;
    for (int c = 0; c < 6; c++) {
        d->K[c] = nullptr;
        if (d->is2d && (c == 3 || c == 4)) continue;  // yz, xz vanish in 2D (newellDemagKernel.go:1314-1317)
        UMAG_CUDA(cudaMalloc(&d->K[c], sizeof(float) * kn));
    }
    // the opt-in limit is per kernel and process-wide: set it to the maximum
    // so plans of different sizes can coexist
    const int maxsm = 227 * 1024;
    UMAG_CUDA(cudaFuncSetAttribute(k_pass_a, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm));
    UMAG_CUDA(cudaFuncSetAttribute(k_pass_c, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm));
    UMAG_CUDA(cudaFuncSetAttribute(k_pass_b, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm));
    UMAG_CUDA(cudaFuncSetAttribute(k_fft_axis<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm));
    UMAG_TRY(demag_fast_setup());
    // the compile-time passes assume a zero-padded half along x and y
    const bool periodic = d->pbc[0] || d->pbc[1] || d->pbc[2];
    d->use_fast = !periodic && getenv("UMAG_GENERIC_FFT") == nullptr &&
                  demag_fast_select(d->M, d->P[1], d->P[2], d->fast);
    if (d->use_fast) UMAG_TRY(demag_fast_grid(d->fast, d->M, d->P[2]));
    slab_setup(d);
    return UMAG_OK;
}

// FP64 real-space kernel -> float32 spectrum (opencl/conv_demag.go:155-201)
static int kernel_to_spectrum(umag_demag* d, double* const Kr[6], cudaStream_t st) {
    const int Px = d->P[0], Py = d->P[1], Pz = d->P[2];
    long n = (long)Px * Py * Pz;
    double2* buf = nullptr;
    UMAG_CUDA(cudaMalloc(&buf, sizeof(double2) * n));
    FftLine<double> fl[3];
    double2* tws[3] = {nullptr, nullptr, nullptr};
    int st_ok = UMAG_OK;
    for (int ax = 0; ax < 3 && st_ok == UMAG_OK; ax++) {
        st_ok = make_line<double>(d->P[ax], fl[ax], &tws[ax]);
        if (st_ok == UMAG_OK && !fft_line_fits(fl[ax], 256))
            st_ok = set_error(UMAG_E_UNSUPPORTED, "kernel FFT line %d too long", d->P[ax]);
    }
    unsigned long long* dmax = nullptr;
    if (st_ok == UMAG_OK) st_ok = cudaMalloc(&dmax, sizeof(unsigned long long)) == cudaSuccess ? UMAG_OK : UMAG_E_CUDA;
    const int threads = 256;
    for (int c = 0; c < 6 && st_ok == UMAG_OK; c++) {
        if (d->K[c] == nullptr) continue;
        k_real_to_cplx<<<grid_for(n, threads), threads, 0, st>>>(Kr[c], buf, n);
        for (int ax = 0; ax < 3; ax++) {
            int L = d->P[ax];
            if (L == 1) continue;
            int G = ax == 0 ? 1 : 4;
            while (ax == 0 && (G * 2) * L * 16 <= 64 * 1024 && G < 8) G *= 2;
            size_t sm = sizeof(double2) * (size_t)G * L;
            if (sm > 200 * 1024) { st_ok = set_error(UMAG_E_UNSUPPORTED, "kernel FFT line %d too long", L); break; }
            long blocks;
            if (ax == 0) blocks = ((long)Py * Pz + G - 1) / G;
            else blocks = (long)((Px + G - 1) / G) * (ax == 1 ? Pz : Py);
            k_fft_axis<double><<<(unsigned)blocks, threads, sm, st>>>(buf, fl[ax], Px, Py, Pz, ax, G, -1);
        }
        cudaMemsetAsync(dmax, 0, sizeof(unsigned long long), st);
        long kn = (long)d->Kn;
        k_extract_spectrum<<<grid_for(kn, threads), threads, 0, st>>>(buf, d->K[c], Px, Py, Pz, d->Kp,
                                                                       d->use_fast && d->fast.blocked ? 1 : 0,
                                                                       1.0 / (double)n, dmax);
        unsigned long long hm = 0;
        cudaMemcpyAsync(&hm, dmax, sizeof(hm), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) { st_ok = set_error(UMAG_E_CUDA, "kernel FFT failed"); break; }
        double mi;
        memcpy(&mi, &hm, sizeof(mi));
        mi *= sqrt(1.0 / (double)n);
        if (mi > 1e-6) st_ok = set_error(UMAG_E_ARG, "FFT kernel imaginary part %g (opencl/conv_common.go:43-53)", mi);
    }
    cudaFree(buf);
    cudaFree(dmax);
    for (int ax = 0; ax < 3; ax++) cudaFree(tws[ax]);
    UMAG_LAUNCH_CHECK();
    return st_ok;
}

// Newell tensor in FP64 on the device (mag/newellDemagKernel.go:1108-1324)
static int build_newell(const umag_demag* d, const double cell[3], int arad, int zero_self, double* Kr[6],
                        cudaStream_t st) {
    NewellArgs a{};
    for (int i = 0; i < 3; i++) {
        a.P[i] = d->P[i];
        a.ext[i] = d->P[i] / 2 + 1;  // octant [0, P/2]
        // kernelRanges (mag/demagkernel.go:339-352)
        if (d->pbc[i] == 0) { a.r1[i] = -(d->P[i] - 1) / 2; a.r2[i] = (d->P[i] - 1) / 2; }
        else { a.r1[i] = -(d->P[i] * d->pbc[i] - 1); a.r2[i] = d->P[i] * d->pbc[i] - 1; }
    }
    if (d->P[2] == 1 && d->pbc[2] == 0) a.r2[2] = 0;
    double dx = cell[0], dy = cell[1], dz = cell[2];
    newell::reduce_cell(dx, dy, dz);
    a.dx = dx; a.dy = dy; a.dz = dz;
    a.scale = -1.0 / (4.0 * M_PI * dx * dy * dz);
    double r = (double)arad * pow(dx * dy * dz, 1.0 / 3.0);
    a.arad2 = r * r;
    a.use_asym = r >= 0.0;
    a.exx = newell::make_expansion(0, dx, dy, dz);
    a.exy = newell::make_expansion(1, dx, dy, dz);
    a.exz = newell::make_expansion(1, dx, dz, dy);
    a.eyy = newell::make_expansion(0, dy, dx, dz);
    a.eyz = newell::make_expansion(1, dy, dz, dx);
    a.ezz = newell::make_expansion(0, dz, dy, dx);
    long n = (long)d->P[0] * d->P[1] * d->P[2];
    for (int c = 0; c < 6; c++) UMAG_CUDA(cudaMemsetAsync(Kr[c], 0, sizeof(double) * n, st));
    long oct = (long)a.ext[0] * a.ext[1] * a.ext[2];
    k_newell_octant<<<grid_for(oct, 128, 32), 128, 0, st>>>(Kr[0], Kr[1], Kr[2], Kr[3], Kr[4], Kr[5], a);
    UMAG_LAUNCH_CHECK();
    k_newell_mirror<<<grid_for(n, 256), 256, 0, st>>>(Kr[0], Kr[1], Kr[2], Kr[3], Kr[4], Kr[5], d->P[0], d->P[1],
                                                       d->P[2]);
    UMAG_LAUNCH_CHECK();
    // self terms at the origin (:1300-1312)
    double self[6] = {-newell::self_nx(dx, dy, dz), -newell::self_nx(dy, dz, dx), -newell::self_nx(dz, dx, dy),
                      0.0, 0.0, 0.0};
    if (zero_self) for (int c = 0; c < 3; c++) self[c] += 1.0 / 3.0;
    for (int c = 0; c < 6; c++) UMAG_CUDA(cudaMemcpyAsync(Kr[c], &self[c], sizeof(double), cudaMemcpyHostToDevice, st));
    if (d->P[2] == 1) {
        UMAG_CUDA(cudaMemsetAsync(Kr[3], 0, sizeof(double) * n, st));
        UMAG_CUDA(cudaMemsetAsync(Kr[4], 0, sizeof(double) * n, st));
    }
    UMAG_CUDA(cudaStreamSynchronize(st));
    return UMAG_OK;
}

int demag_new_newell(int Nx, int Ny, int Nz, const int pbc[3], double cx, double cy, double cz, int arad,
                     int zero_self, umag_demag** out) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(out != nullptr, "out is NULL");
    UMAG_REQUIRE(cx > 0 && cy > 0 && cz > 0, "cell size must be positive");
    umag_demag* d = new umag_demag();
    d->N[0] = Nx; d->N[1] = Ny; d->N[2] = Nz;
    d->cell[0] = cx; d->cell[1] = cy; d->cell[2] = cz;
    d->arad = arad;
    d->zero_self = zero_self;
    for (int i = 0; i < 3; i++) d->pbc[i] = pbc ? pbc[i] : 0;
    int s = plan_common(d);
    if (s != UMAG_OK) { demag_free(d); return s; }
    cudaStream_t st = ctx().stream;
    long n = (long)d->P[0] * d->P[1] * d->P[2];
    double* Kr[6] = {};
    for (int c = 0; c < 6 && s == UMAG_OK; c++)
        if (cudaMalloc(&Kr[c], sizeof(double) * n) != cudaSuccess) s = set_error(UMAG_E_NOMEM, "kernel buffers");
    if (s == UMAG_OK) s = build_newell(d, d->cell, arad, zero_self, Kr, st);
    if (s == UMAG_OK) s = kernel_to_spectrum(d, Kr, st);
    for (int c = 0; c < 6; c++) cudaFree(Kr[c]);
    if (s != UMAG_OK) { demag_free(d); return s; }
    *out = d;
    return UMAG_OK;
}

// mag/demagkernel.go:113 CalcDemagKernel (engine/demag.go:124-133 demagConv):
// the brute-force kernel built on the GPU, FFT'd in FP64 like the Newell one
int demag_new_brute(int Nx, int Ny, int Nz, const int pbc[3], double cx, double cy, double cz, double accuracy,
                    umag_demag** out) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(out != nullptr, "out is NULL");
    UMAG_REQUIRE(cx > 0 && cy > 0 && cz > 0, "cell size must be positive");
    UMAG_REQUIRE(accuracy > 0, "demag accuracy must be positive");
    umag_demag* d = new umag_demag();
    d->N[0] = Nx; d->N[1] = Ny; d->N[2] = Nz;
    d->cell[0] = cx; d->cell[1] = cy; d->cell[2] = cz;
    d->kind = 1;
    d->accuracy = accuracy;
    for (int i = 0; i < 3; i++) d->pbc[i] = pbc ? pbc[i] : 0;
    int s = plan_common(d);
    if (s != UMAG_OK) { demag_free(d); return s; }
    cudaStream_t st = ctx().stream;
    long n = (long)d->P[0] * d->P[1] * d->P[2];
    double* Kr[6] = {};
    for (int c = 0; c < 6 && s == UMAG_OK; c++)
        if (cudaMalloc(&Kr[c], sizeof(double) * n) != cudaSuccess) s = set_error(UMAG_E_NOMEM, "kernel buffers");
    if (s == UMAG_OK) s = build_brute(d, accuracy, Kr, st);
    if (s == UMAG_OK) s = kernel_to_spectrum(d, Kr, st);
    for (int c = 0; c < 6; c++) cudaFree(Kr[c]);
    if (s != UMAG_OK) { demag_free(d); return s; }
    *out = d;
    return UMAG_OK;
}
int demag_new_from_kernel(int Nx, int Ny, int Nz, const double* const kern[6], umag_demag** out) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(out != nullptr && kern != nullptr, "NULL argument");
    umag_demag* d = new umag_demag();
    d->N[0] = Nx; d->N[1] = Ny; d->N[2] = Nz;
    d->kind = 2;
    int s = plan_common(d);
    if (s != UMAG_OK) { demag_free(d); return s; }
    long n = (long)d->P[0] * d->P[1] * d->P[2];
    double* Kr[6] = {};
    for (int c = 0; c < 6 && s == UMAG_OK; c++) {
        if (cudaMalloc(&Kr[c], sizeof(double) * n) != cudaSuccess) { s = set_error(UMAG_E_NOMEM, "kernel"); break; }
        const cudaError_t e = kern[c] ? cudaMemcpyAsync(Kr[c], kern[c], sizeof(double) * n, cudaMemcpyHostToDevice,
                                                        ctx().stream)
                                      : cudaMemsetAsync(Kr[c], 0, sizeof(double) * n, ctx().stream);
        if (e != cudaSuccess) s = set_error(UMAG_E_CUDA, "kernel upload: %s", cudaGetErrorString(e));
    }
    if (s == UMAG_OK) s = kernel_to_spectrum(d, Kr, ctx().stream);
    for (int c = 0; c < 6; c++) cudaFree(Kr[c]);
    if (s != UMAG_OK) { demag_free(d); return s; }
    *out = d;
    return UMAG_OK;
}

int demag_get_kernel(umag_demag* d, double* const host[6]) {
    UMAG_REQUIRE(d != nullptr, "NULL plan");
    long n = (long)d->P[0] * d->P[1] * d->P[2];
    double* Kr[6] = {};
    int s = UMAG_OK;
    for (int c = 0; c < 6 && s == UMAG_OK; c++)
        if (cudaMalloc(&Kr[c], sizeof(double) * n) != cudaSuccess) s = set_error(UMAG_E_NOMEM, "kernel buffers");
    if (s == UMAG_OK) {
        if (d->kind == 0) s = build_newell(d, d->cell, d->arad, d->zero_self, Kr, ctx().stream);
        else if (d->kind == 1) s = build_brute(d, d->accuracy, Kr, ctx().stream);
        else s = set_error(UMAG_E_UNSUPPORTED, "the plan was built from a caller-supplied kernel, which it does not keep");
    }
    for (int c = 0; c < 6 && s == UMAG_OK; c++)
        if (host[c] && cudaMemcpyAsync(host[c], Kr[c], sizeof(double) * n, cudaMemcpyDeviceToHost, ctx().stream) !=
                           cudaSuccess)
            s = set_error(UMAG_E_CUDA, "copy kernel");
    if (cudaStreamSynchronize(ctx().stream) != cudaSuccess && s == UMAG_OK) s = set_error(UMAG_E_CUDA, "copy kernel");
    for (int c = 0; c < 6; c++) cudaFree(Kr[c]);
    return s;
}

int demag_get_spectrum(umag_demag* d, float* const host[6]) {
    UMAG_REQUIRE(d != nullptr, "NULL plan");
    UMAG_CUDA(cudaStreamSynchronize(ctx().stream));
    const size_t hy = d->P[1] / 2 + 1, rows = d->Kn / d->Kp;  // rows = hy * hz
    const bool blocked = d->use_fast && d->fast.blocked;
    std::vector<float> tmp(blocked ? d->Kn : 0);
    for (int c = 0; c < 6; c++) {
        if (!host[c]) continue;
        if (!d->K[c]) {
            memset(host[c], 0, sizeof(float) * d->Hx * rows);
        } else if (!blocked) {
            // reference layout: rows of Px/2+1 floats (the device rows are padded to Kp)
            UMAG_CUDA(cudaMemcpy2DAsync(host[c], sizeof(float) * d->Hx, d->K[c], sizeof(float) * d->Kp,
                                        sizeof(float) * d->Hx, rows, cudaMemcpyDeviceToHost, ctx().stream));
            UMAG_CUDA(cudaStreamSynchronize(ctx().stream));
        } else {
            UMAG_CUDA(cudaMemcpyAsync(tmp.data(), d->K[c], sizeof(float) * d->Kn, cudaMemcpyDeviceToHost, ctx().stream));
            UMAG_CUDA(cudaStreamSynchronize(ctx().stream));
            const size_t nb = d->Kp / 4;
            for (size_t r = 0; r < rows; r++) {  // r = z * hy + y
                const size_t z = r / hy, y = r % hy;
                for (int x = 0; x < d->Hx; x++)
                    host[c][r * d->Hx + x] = tmp[((z * nb + x / 4) * hy + y) * 4 + x % 4];
            }
        }
    }
    return UMAG_OK;
}

void fill_pass_args(const umag_demag* d, PassArgs& a) {
    a.Nx = d->N[0]; a.Ny = d->N[1]; a.Nz = d->N[2];
    a.Px = d->P[0]; a.Py = d->P[1]; a.Pz = d->P[2];
    a.M = d->M; a.Hx = d->Hx; a.HxP = d->HxP; a.Lx = d->Lx; a.WB = d->WB;
    a.fx = d->fx; a.fy = d->fy; a.fz = d->fz;
    a.twr = d->twr;
    a.spec = d->spec;
    for (int c = 0; c < 6; c++) a.K[c] = d->K[c];
    a.Kp = d->Kp;
    a.blocked = d->use_fast && d->fast.blocked ? 1 : 0;
    a.Kblocked = a.blocked;
    a.slab_map = d->slab_map;
}

int demag_launch(const umag_demag* d, const PassArgs& a, cudaStream_t st) {
    if (d->use_fast) {
        const FastPasses& f = d->fast;
        f.a<<<dim3(d->N[1], 3), f.nt_ac, f.smem_ac, st>>>(a);
        UMAG_LAUNCH_CHECK();
        if (f.use_narrow) f.b_n<<<dim3(f.gbx_n, f.gby), f.nt_b_n, f.smem_b_n, st>>>(a);
        else f.b<<<dim3(f.gbx, f.gby), f.nt_b, f.smem_b, st>>>(a);
        UMAG_LAUNCH_CHECK();
        f.c<<<dim3(d->N[1], 3), f.nt_ac, f.smem_ac, st>>>(a);
        UMAG_LAUNCH_CHECK();
        return UMAG_OK;
    }
    size_t sac = pass_ac_smem(d), sb = pass_b_smem(d);
    k_pass_a<<<dim3(d->N[1], 3), kPassThreads, sac, st>>>(a);
    UMAG_LAUNCH_CHECK();
    k_pass_b<<<dim3((d->Hx + d->WB - 1) / d->WB, d->P[2]), kPassBThreads, sb, st>>>(a);
    UMAG_LAUNCH_CHECK();
    k_pass_c<<<dim3(d->N[1], 3), kPassThreads, sac, st>>>(a);
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

// the three passes for nb same-size instances at once (batched kernels; the
// per-instance pointers are shifted by the strides in PassArgs)
int demag_launch_batch(const umag_demag* d, const PassArgs& a, int nb, cudaStream_t st) {
    UMAG_REQUIRE(d->use_fast && d->fast.ab && d->fast.bb && d->fast.cb, "batched demag needs a compile-time FFT plan");
    UMAG_REQUIRE(nb >= 1 && 3L * nb <= 65535 && (long)d->fast.gby * nb <= 65535, "too many instances in one batch");
    const FastPasses& f = d->fast;
    // per-instance spectra: the slab map covers the plan's own spectrum only
    PassArgs ab = a;
    ab.slab_map = nullptr;
    f.ab<<<dim3(d->N[1], 3 * nb), f.nt_ac, f.smem_ac, st>>>(ab);
    UMAG_LAUNCH_CHECK();
    f.bb<<<dim3(f.gbx, f.gby * nb), f.nt_b, f.smem_b, st>>>(ab);
    UMAG_LAUNCH_CHECK();
    f.cb<<<dim3(d->N[1], 3 * nb), f.nt_ac, f.smem_ac, st>>>(ab);
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

// one pass of demag_launch (0: A, 1: B, 2: C)
static int demag_launch_pass(const umag_demag* d, const PassArgs& a, cudaStream_t st, int pass) {
    if (d->use_fast) {
        const FastPasses& f = d->fast;
        if (pass == 0) f.a<<<dim3(d->N[1], 3), f.nt_ac, f.smem_ac, st>>>(a);
        else if (pass == 1 && f.use_narrow) f.b_n<<<dim3(f.gbx_n, f.gby), f.nt_b_n, f.smem_b_n, st>>>(a);
        else if (pass == 1) f.b<<<dim3(f.gbx, f.gby), f.nt_b, f.smem_b, st>>>(a);
        else f.c<<<dim3(d->N[1], 3), f.nt_ac, f.smem_ac, st>>>(a);
    } else {
        size_t sac = pass_ac_smem(d), sb = pass_b_smem(d);
        if (pass == 0) k_pass_a<<<dim3(d->N[1], 3), kPassThreads, sac, st>>>(a);
        else if (pass == 1) k_pass_b<<<dim3((d->Hx + d->WB - 1) / d->WB, d->P[2]), kPassBThreads, sb, st>>>(a);
        else k_pass_c<<<dim3(d->N[1], 3), kPassThreads, sac, st>>>(a);
    }
    UMAG_LAUNCH_CHECK();
    return UMAG_OK;
}

int demag_exec(umag_demag* d, float* Bx, float* By, float* Bz, const float* mx, const float* my, const float* mz,
               const float* vol, const float* Ms, float Ms_mul, int pass) {
    UMAG_REQUIRE(d != nullptr, "NULL plan");
    UMAG_REQUIRE(Bx && By && Bz && mx && my && mz, "NULL field or magnetisation pointer");
    UMAG_REQUIRE(pass >= -1 && pass <= 2, "pass must be -1 (all), 0, 1 or 2");
    PassArgs a{};
    fill_pass_args(d, a);
    a.m[0] = mx; a.m[1] = my; a.m[2] = mz;
    a.B[0] = Bx; a.B[1] = By; a.B[2] = Bz;
    a.vol = vol; a.Ms = Ms; a.Ms_mul = Ms_mul;
    if (pass >= 0) return demag_launch_pass(d, a, ctx().stream, pass);
    UMAG_TRY(demag_launch(d, a, ctx().stream));
    // Exec completes before it returns, as the reference's does; a bulk copy
    // that timed out (a field left unwritten) is an error here, not a silent
    // wrong result.  Skipped while the stream is being captured.
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    UMAG_CUDA(cudaStreamIsCapturing(ctx().stream, &cs));
    if (cs == cudaStreamCaptureStatusNone) {
        unsigned n = 0;
        UMAG_TRY(demag_slab_timeouts(&n, ctx().stream));
        if (n != 0) return set_error(UMAG_E_TIMEOUT, "demag pass C: %u spectrum-slab copies timed out", n);
    }
    return UMAG_OK;
}

void demag_free(umag_demag* d) {
    if (!d) return;
    for (auto p : d->tw_dev) cudaFree(p);
    cudaFree(d->twr);
    cudaFree(d->spec);
    cudaFree(d->slab_map);
    for (int c = 0; c < 6; c++) cudaFree(d->K[c]);
    delete d;
}

}  // namespace umag
