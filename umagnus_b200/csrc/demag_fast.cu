// demag_fast.cu -- the demag passes with compile-time FFT plans.
//
// Same three passes and data layout as demag.cu (see its header comment),
// instantiated for the mesh sizes the benchmarks and common simulations use:
// every FFT index computation is a constant, register arrays are unrolled,
// twiddles are staged in shared memory.  demag_fast_select() returns the
// instantiation for a plan, or nothing (the generic kernels then run).
#include <mutex>

#include "demag.cuh"
#include "fft_pair.cuh"
#include "fft_reg.cuh"
#include "fft_static.cuh"
#include "tile.cuh"

namespace umag {

// pass C slab loads that gave up waiting (bounded mbarrier poll); the plain
// device-op API reads it after each demag_exec (engine launches report the
// timeout through the controller status instead, PassArgs::fault)
__device__ unsigned g_slab_timeouts = 0;

int demag_slab_timeouts(unsigned* out, cudaStream_t st) {
    UMAG_CUDA(cudaMemcpyFromSymbolAsync(out, g_slab_timeouts, sizeof(unsigned), 0, cudaMemcpyDeviceToHost, st));
    UMAG_CUDA(cudaStreamSynchronize(st));
    return UMAG_OK;
}
int demag_set_slab_timeouts(unsigned v) {
    UMAG_CUDA(cudaMemcpyToSymbol(g_slab_timeouts, &v, sizeof(unsigned)));
    UMAG_CUDA(cudaDeviceSynchronize());
    return UMAG_OK;
}

// record a pass that gave up waiting for a bulk copy: the counter, and the
// instance's controller status (7, as the torque kernel's tile wait) when
// the launch belongs to a simulation
__device__ __forceinline__ void pass_timeout(const PassArgs& a, int ib) {
    atomicAdd(&g_slab_timeouts, 1u);
    if (a.fault) atomicCAS(reinterpret_cast<int*>(reinterpret_cast<char*>(a.fault) + (long)ib * a.ctl_stride), 0, 7);
}


static constexpr double kMu0f = 4 * 3.1415926535897932384626433 * 1e-7;  // clh/constants.clh:5

constexpr int nz_of_pz(int PZ) { return PZ == 1 ? 1 : (PZ % 2 == 0 ? PZ / 2 : (PZ + 1) / 2); }
constexpr int kNT = 256;       // passes A, C
constexpr int kNTB = 512;      // pass B
constexpr int kElemCap = 24;   // complex elements per thread per FFT batch

template <int M, int PZ> struct AcShape {
    static constexpr int NZ = nz_of_pz(PZ);
    static constexpr int XP = M + 1;                                  // row pitch (holds X[0..M])
    static constexpr int ZB = sp_divisor_le(NZ, (kElemCap * kNT) / M);  // rows per x-FFT batch
    static constexpr int CW = PZ == 1 ? 1 : sp_divisor_le(M, (kElemCap * kNT) / PZ < 64 ? (kElemCap * kNT) / PZ : 64);
    static constexpr size_t smem = sizeof(float2) * ((size_t)M + PZ + (M / 2 + 1) + (size_t)NZ * XP +
                                                     (PZ > 1 ? (size_t)PZ * CW : 0));
};

// copypadmul2.cl:13-20: MU0*Ms (FP64 product rounded to float32) * vol * m
__device__ __forceinline__ float scaled_m(const PassArgs& a, const float* __restrict__ m, int i, float msmul) {
    float fac = a.Ms == nullptr ? msmul : __fmul_rn(msmul, __ldg(a.Ms + i));
    float bsat = (float)(kMu0f * (double)fac);
    float w = a.vol == nullptr ? 1.0f : __fmul_rn(1.0f, __ldg(a.vol + i));
    return __fmul_rn(__fmul_rn(bsat, w), __ldg(m + i));
}

// Per-instance views of PassArgs for batched launches (an ensemble of
// same-size instances, instance ib): spectrum scratch, field output, the
// instance's controller fields (m slots, active flag) and its Ms.  With
// ib = 0 (single-instance kernels) every offset folds away.
__device__ __forceinline__ float2* inst_spec(const PassArgs& a, int ib) { return a.spec + (long)ib * a.spec_stride; }
__device__ __forceinline__ float* inst_B(const PassArgs& a, int ib, int c) { return a.B[c] + (long)ib * a.b_stride; }
__device__ __forceinline__ bool inst_inactive(const PassArgs& a, int ib) {
    if (!a.active) return false;
    return !*reinterpret_cast<const int*>(reinterpret_cast<const char*>(a.active) + (long)ib * a.ctl_stride);
}
__device__ __forceinline__ const float* inst_m(const PassArgs& a, int ib, int c) {
    if (!a.m_ind) return a.m[c];
    const char* slot = reinterpret_cast<const char*>(a.m_sel ? a.m_ind_w : a.m_ind) + (long)ib * a.ctl_stride;
    return *reinterpret_cast<float* const*>(slot) + (long)c * a.ncell;
}
__device__ __forceinline__ float inst_msmul(const PassArgs& a, int ib) { return a.ms_mul_b ? a.ms_mul_b[ib] : a.Ms_mul; }

template <int M, int PZ>
__device__ __forceinline__ void k_fast_a_body(const PassArgs& a, const int bx, const int by, const int ib) {
    using S = AcShape<M, PZ>;
    constexpr int NZ = S::NZ, XP = S::XP, CW = S::CW, H = M / 2;
    extern __shared__ __align__(16) float2 sm[];
    float2* twx = sm;
    float2* twz = twx + M;
    float2* twr = twz + PZ;
    float2* X1 = twr + (H + 1);
    float2* Z2 = X1 + NZ * XP;
    if (inst_inactive(a, ib)) return;
    const int tid = threadIdx.x;
    for (int i = tid; i < M; i += kNT) twx[i] = a.fx.tw[i];
    if (PZ > 1)
        for (int i = tid; i < PZ; i += kNT) twz[i] = a.fz.tw[i];
    for (int i = tid; i <= H; i += kNT) twr[i] = a.twr[i];
    const int y = bx, c = by, Ny = a.Ny;
    const float* __restrict__ m = inst_m(a, ib, c);
    const float msm = inst_msmul(a, ib);
    // 1. scaled m, pairs of reals packed into complex (x = 2n, 2n+1), Nx = M
    for (int e = tid; e < NZ * M; e += kNT) {
        const int z = e / M, n = e % M;
        float2 v = make_float2(0.f, 0.f);  // x >= Nx is zero padding
        if (n < H) {
            const int i = (z * Ny + y) * M + 2 * n;
            v = make_float2(scaled_m(a, m, i, msm), scaled_m(a, m, i + 1, msm));
        }
        X1[z * XP + n] = v;
    }
    __syncthreads();
    // 2. length-M complex FFT of every row
#pragma unroll 1
    for (int rb = 0; rb < NZ; rb += S::ZB) sfft<float2, M, S::ZB, kNT, XP, 1, false, -1>(X1 + rb * XP, twx);
    // 3. R2C unpack: X[k] = E + W^k O, X[M-k] = conj(E - W^k O)
    for (int e = tid; e < NZ * (H + 1); e += kNT) {
        const int z = e / (H + 1), k = e % (H + 1);
        float2* row = X1 + z * XP;
        const int k2 = M - k;
        float2 A = row[k], B = row[k == 0 ? 0 : k2];
        float2 E = make_float2(0.5f * (A.x + B.x), 0.5f * (A.y - B.y));
        float2 D = make_float2(0.5f * (A.x - B.x), 0.5f * (A.y + B.y));
        float2 O = make_float2(D.y, -D.x);
        float2 W = twr[k];
        float2 WO = make_float2(W.x * O.x - W.y * O.y, W.x * O.y + W.y * O.x);
        row[k] = make_float2(E.x + WO.x, E.y + WO.y);
        row[k2] = make_float2(E.x - WO.x, WO.y - E.y);
    }
    __syncthreads();
    float2* out = inst_spec(a, ib) + (long)c * PZ * Ny * a.Lx + (long)y * a.Lx;
    const long kzs = (long)Ny * a.Lx;
    if constexpr (PZ == 1) {
        for (int k = tid; k <= M; k += kNT) out[k] = X1[k];
    } else {
        // 4. forward z FFT per block of CW columns, then the Nyquist column kx = M
#pragma unroll 1
        for (int kx0 = 0; kx0 < M; kx0 += CW) {
            for (int e = tid; e < PZ * CW; e += kNT) {
                const int z = e / CW, w = e % CW;
                Z2[e] = z < NZ ? X1[z * XP + kx0 + w] : make_float2(0.f, 0.f);
            }
            __syncthreads();
            sfft<float2, PZ, CW, kNT, 1, CW, true, -1>(Z2, twz);
            for (int e = tid; e < PZ * CW; e += kNT) {
                const int kz = e / CW, w = e % CW;
                out[kz * kzs + kx0 + w] = Z2[e];
            }
            __syncthreads();
        }
        for (int z = tid; z < PZ; z += kNT) Z2[z] = z < NZ ? X1[z * XP + M] : make_float2(0.f, 0.f);
        __syncthreads();
        sfft<float2, PZ, 1, kNT, 1, 1, true, -1>(Z2, twz);
        for (int kz = tid; kz < PZ; kz += kNT) out[kz * kzs + M] = Z2[kz];
    }
}
template <int M, int PZ>
__global__ void __launch_bounds__(kNT) k_fast_a(PassArgs a) { k_fast_a_body<M, PZ>(a, blockIdx.x, blockIdx.y, 0); }
// batched: blockIdx.y = index + per * instance (the inst_* views above)
template <int M, int PZ>
__global__ void __launch_bounds__(kNT) k_fast_a_bat(PassArgs a) {
    const int per = 3, b = blockIdx.y / per;
    k_fast_a_body<M, PZ>(a, blockIdx.x, blockIdx.y - b * per, b);
}

template <int M, int PZ>
__device__ __forceinline__ void k_fast_c_body(const PassArgs& a, const int bx, const int by, const int ib) {
    using S = AcShape<M, PZ>;
    constexpr int NZ = S::NZ, XP = S::XP, CW = S::CW, H = M / 2;
    extern __shared__ __align__(16) float2 sm[];
    float2* twx = sm;
    float2* twz = twx + M;
    float2* twr = twz + PZ;
    float2* X1 = twr + (H + 1);
    float2* Z2 = X1 + NZ * XP;
    if (inst_inactive(a, ib)) return;
    const int tid = threadIdx.x;
    for (int i = tid; i < M; i += kNT) twx[i] = a.fx.tw[i];
    if (PZ > 1)
        for (int i = tid; i < PZ; i += kNT) twz[i] = a.fz.tw[i];
    for (int i = tid; i <= H; i += kNT) twr[i] = a.twr[i];
    const int y = bx, c = by, Ny = a.Ny;
    const float2* in = inst_spec(a, ib) + (long)c * PZ * Ny * a.Lx + (long)y * a.Lx;
    const long kzs = (long)Ny * a.Lx;
    // 1. inverse z FFT per block of columns, keep z < NZ
    if constexpr (PZ == 1) {
        for (int k = tid; k <= M; k += kNT) X1[k] = in[k];
    } else {
#pragma unroll 1
        for (int kx0 = 0; kx0 < M; kx0 += CW) {
            for (int e = tid; e < PZ * CW; e += kNT) {
                const int kz = e / CW, w = e % CW;
                Z2[e] = in[kz * kzs + kx0 + w];
            }
            __syncthreads();
            sfft<float2, PZ, CW, kNT, 1, CW, true, +1>(Z2, twz);
            for (int e = tid; e < NZ * CW; e += kNT) {
                const int z = e / CW, w = e % CW;
                X1[z * XP + kx0 + w] = Z2[e];
            }
            __syncthreads();
        }
        for (int kz = tid; kz < PZ; kz += kNT) Z2[kz] = in[kz * kzs + M];
        __syncthreads();
        sfft<float2, PZ, 1, kNT, 1, 1, true, +1>(Z2, twz);
        for (int z = tid; z < NZ; z += kNT) X1[z * XP + M] = Z2[z];
    }
    __syncthreads();
    // 2. C2R pack: Z[k] = (X[k] + conj X[M-k]) + i conj(W^k) (X[k] - conj X[M-k])
    for (int e = tid; e < NZ * (H + 1); e += kNT) {
        const int z = e / (H + 1), k = e % (H + 1);
        float2* row = X1 + z * XP;
        const int k2 = M - k;
        float2 Xk = row[k], Xm = row[k2];
        if (k == 0) { Xk.y = 0.f; Xm.y = 0.f; }
        float2 W = twr[k];
        float2 S1 = make_float2(Xk.x + Xm.x, Xk.y - Xm.y);
        float2 D1 = make_float2(Xk.x - Xm.x, Xk.y + Xm.y);
        float2 T1 = make_float2(W.x * D1.x + W.y * D1.y, W.x * D1.y - W.y * D1.x);  // conj(W) * D1
        float2 Zk = make_float2(S1.x - T1.y, S1.y + T1.x);
        if (k == 0) {
            row[0] = Zk;
        } else {
            float2 S2 = make_float2(Xm.x + Xk.x, Xm.y - Xk.y);
            float2 D2 = make_float2(Xm.x - Xk.x, Xm.y + Xk.y);
            float2 T2 = make_float2(-(W.x * D2.x - W.y * D2.y), -(W.x * D2.y + W.y * D2.x));  // -W * D2
            row[k] = Zk;
            row[k2] = make_float2(S2.x - T2.y, S2.y + T2.x);
        }
    }
    __syncthreads();
    // 3. inverse length-M FFT of every row
#pragma unroll 1
    for (int rb = 0; rb < NZ; rb += S::ZB) sfft<float2, M, S::ZB, kNT, XP, 1, false, +1>(X1 + rb * XP, twx);
    // 4. unpack even/odd samples, crop and overwrite B (copyunpad.cl)
    float* __restrict__ B = inst_B(a, ib, c);
    for (int e = tid; e < NZ * H; e += kNT) {
        const int z = e / H, n = e % H;
        float2 v = X1[z * XP + n];
        *reinterpret_cast<float2*>(B + (z * Ny + y) * M + 2 * n) = v;
    }
}
template <int M, int PZ>
__global__ void __launch_bounds__(kNT) k_fast_c(PassArgs a) { k_fast_c_body<M, PZ>(a, blockIdx.x, blockIdx.y, 0); }
// batched: blockIdx.y = index + per * instance (the inst_* views above)
template <int M, int PZ>
__global__ void __launch_bounds__(kNT) k_fast_c_bat(PassArgs a) {
    const int per = 3, b = blockIdx.y / per;
    k_fast_c_body<M, PZ>(a, blockIdx.x, blockIdx.y - b * per, b);
}

template <int PY> struct BShape {
    static constexpr int WB0 = (kElemCap * kNTB) / (3 * PY);
    static constexpr int WB = WB0 >= 32 ? 32 : WB0 >= 16 ? 16 : WB0 >= 8 ? 8 : WB0 >= 4 ? 4 : WB0 >= 2 ? 2 : 1;
    static constexpr size_t smem = sizeof(float2) * ((size_t)PY + (size_t)PY * 3 * WB);
};

template <int PY>
__device__ __forceinline__ void k_fast_b_body(const PassArgs& a, const int bx, const int by, const int ib) {
    constexpr int WB = BShape<PY>::WB, W3 = 3 * WB, NY = PY / 2, HY = PY / 2 + 1;
    extern __shared__ __align__(16) float2 sm[];
    float2* twy = sm;
    float2* S = twy + PY;  // [PY][3*WB]
    if (inst_inactive(a, ib)) return;
    const int tid = threadIdx.x;
    for (int i = tid; i < PY; i += kNTB) twy[i] = a.fy.tw[i];
    const int kx0 = bx * WB, kz = by;
    const int hx = a.Hx, Pz = a.Pz;
    const long cs = (long)Pz * NY * a.Lx;
    const float2* in = inst_spec(a, ib) + (long)kz * NY * a.Lx + kx0;
    for (int e = tid; e < PY * W3; e += kNTB) {
        const int yy = e / W3, r = e % W3, c = r / WB, w = r % WB;
        float2 v = make_float2(0.f, 0.f);
        if (yy < NY && kx0 + w < hx) v = in[c * cs + (long)yy * a.Lx + w];
        S[e] = v;
    }
    __syncthreads();
    sfft<float2, PY, W3, kNTB, 1, W3, true, -1>(S, twy);
    // kernel multiply with the mirror symmetry of kernmulrsymm3d.cl:62-82
    int kzm = kz;
    float sz = 1.f;
    if (kz > Pz / 2) { kzm = Pz - kz; sz = -1.f; }
    const bool k3d = a.K[3] != nullptr;
    for (int e = tid; e < PY * WB; e += kNTB) {
        const int ky = e / WB, w = e % WB;
        const int kx = kx0 + w;
        if (kx >= hx) continue;
        int kym = ky;
        float sy = 1.f;
        if (ky > NY) { kym = PY - ky; sy = -1.f; }
        const long I = ((long)kzm * HY + kym) * a.Kp + kx;
        const float Kxx = __ldg(a.K[0] + I), Kyy = __ldg(a.K[1] + I), Kzz = __ldg(a.K[2] + I);
        const float Kxy = __ldg(a.K[5] + I) * sy;
        float Kyz = 0.f, Kxz = 0.f;
        if (k3d) {
            Kyz = __ldg(a.K[3] + I) * (sy * sz);
            Kxz = __ldg(a.K[4] + I) * sz;
        }
        float2* row = S + ky * W3;
        const float2 mx = row[w], my = row[WB + w], mz = row[2 * WB + w];
        row[w] = make_float2(mx.x * Kxx + my.x * Kxy + mz.x * Kxz, mx.y * Kxx + my.y * Kxy + mz.y * Kxz);
        row[WB + w] = make_float2(mx.x * Kxy + my.x * Kyy + mz.x * Kyz, mx.y * Kxy + my.y * Kyy + mz.y * Kyz);
        row[2 * WB + w] = make_float2(mx.x * Kxz + my.x * Kyz + mz.x * Kzz, mx.y * Kxz + my.y * Kyz + mz.y * Kzz);
    }
    __syncthreads();
    sfft<float2, PY, W3, kNTB, 1, W3, true, +1>(S, twy);
    float2* outp = inst_spec(a, ib) + (long)kz * NY * a.Lx + kx0;
    for (int e = tid; e < NY * W3; e += kNTB) {
        const int yy = e / W3, r = e % W3, c = r / WB, w = r % WB;
        if (kx0 + w < hx) outp[c * cs + (long)yy * a.Lx + w] = S[e];
    }
}
template <int PY>
__global__ void __launch_bounds__(kNTB) k_fast_b(PassArgs a) { k_fast_b_body<PY>(a, blockIdx.x, blockIdx.y, 0); }
// batched: blockIdx.y = index + per * instance (the inst_* views above)
template <int PY>
__global__ void __launch_bounds__(kNTB) k_fast_b_bat(PassArgs a) {
    const int per = a.Pz, b = blockIdx.y / per;
    k_fast_b_body<PY>(a, blockIdx.x, blockIdx.y - b * per, b);
}

// cp.async (global -> shared, asynchronous) helpers
__device__ __forceinline__ void cpa16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src));
}
__device__ __forceinline__ void cpa8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src));
}
__device__ __forceinline__ void cpa4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src));
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cpa_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

// Offset of spectrum column kx within one (component, kz, y = 0) plane, and
// the stride between rows y: blocked layout [kx/4][y][kx%4] or rows [y][kx].
__device__ __forceinline__ long spec_col(const PassArgs& a, int kx) {
    return a.blocked ? (long)(kx >> 2) * (a.Ny * 4) + (kx & 3) : (long)kx;
}
__device__ __forceinline__ long spec_rowstride(const PassArgs& a) { return a.blocked ? 4 : a.Lx; }
// Index of kernel element (kz, ky, kx), kz/ky in the stored non-redundant block
__device__ __forceinline__ long kern_idx(const PassArgs& a, int kz, int ky, int kx, int hy) {
    return a.Kblocked ? (((long)kz * (a.Kp >> 2) + (kx >> 2)) * hy + ky) * 4 + (kx & 3)
                      : ((long)kz * hy + ky) * a.Kp + kx;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Shared memory of a pass-B CTA (k_reg_b): the staged twiddle tables (TWN
// slots, an even count so what follows stays 16-byte aligned), two exchange
// buffers of WB padded lines, the kernel block [6][WB/KW][HY][KW] (KW = 4
// columns per 16-byte piece, or WB when narrower).
template <int PY, int WB> struct RegBShape {
    static constexpr int KW = WB >= 4 ? 4 : WB;
    static constexpr int TWN = (RgTw<PY>::size + 1) & ~1;
    static constexpr size_t smem = sizeof(float2) * ((size_t)TWN + (size_t)2 * WB * rg_line<PY>()) +
                                   sizeof(float) * (size_t)6 * (PY / 2 + 1) * WB;
    // three CTAs per SM (80 registers) up to Py = 512; longer lines hold more
    // live state per thread and keep two
    static constexpr int minb = PY <= 512 && 3 * (smem + 1024) <= 227 * 1024 ? 3 : 2;
};

// Pass B with the register-blocked FFT (power-of-two Py): thread (t, w) holds
// rows t + T*m (m < 8) of column kx0 + w for all three components.  Rows
// y >= Ny are zero padding (m >= 4): the loads are skipped and the first
// radix-8 butterfly folds them (dft8_zhalf); only rows y < Ny are computed by
// the inverse and stored.  With the blocked layouts a warp's loads and stores
// of one component are one contiguous run (WB = 4: 8 rows x 4 columns = 256
// bytes).  The components exchange one at a time through two buffers
// (rg_fft_fwd_seq), which with the kernel block fits three CTAs per SM; the
// kernel block arrives by bulk copies (6 contiguous runs per 4 columns,
// issued by one thread, completing on an mbarrier while the forward
// transform runs), or by 16-byte cp.async pieces where the block is not
// whole 4-column runs (narrow CTAs, the packed Nyquist column).
template <int PY, int WB>
__device__ __forceinline__ void k_reg_b_body(const PassArgs& a, const int bx, const int by, const int ib) {
    constexpr int T = PY / 8, NT = T * WB, NY = PY / 2, HY = PY / 2 + 1;
    constexpr int LP = rg_line<PY>();
    constexpr int KW = RegBShape<PY, WB>::KW;
    extern __shared__ __align__(16) float2 sm[];
    float2* tw = sm;                                 // staged twiddles (RgTw<PY>)
    float2* ex = tw + RegBShape<PY, WB>::TWN;        // [2][WB][LP] exchange lines
    float* Ks = reinterpret_cast<float*>(ex + 2 * WB * LP);  // [6][WB/KW][HY][KW] kernel block
    __shared__ __align__(8) uint64_t kbar;
    if (inst_inactive(a, ib)) return;
    const int tid = threadIdx.x;
    const int w = tid % WB, t = (tid / WB) & (T - 1);  // t < T: the mask tells the compiler
    const int hx = a.Hx, Pz = a.Pz;
    // The last column block holds only the Nyquist column kx = Hx - 1.  When
    // Pz is a multiple of WB its CTAs are packed: CTA by < Pz/WB handles that
    // column for the WB planes kz = by*WB + w (the others exit), so the grid
    // carries Pz/WB such CTAs instead of Pz mostly idle ones.
    const bool nyq = bx * WB == hx - 1 && WB > 1 && Pz % WB == 0 && Pz >= WB;
    if (nyq && by * WB >= Pz) return;
    rg_tw_fill<PY>(tw, a.fy.tw, tid, NT);
    const int kx0 = bx * WB;
    const int kx = nyq ? hx - 1 : kx0 + w, kz = nyq ? by * WB + w : by;
    auto kz_mirror = [&](int z) { return z > Pz / 2 ? Pz - z : z; };
    const int kzm = kz_mirror(kz);
    const float sz = kz > Pz / 2 ? -1.f : 1.f;
    const bool k3d = a.K[3] != nullptr;
    const int ncomp = k3d ? 6 : 4;
    auto kcomp = [&](int cc) { return k3d ? cc : (cc == 3 ? 5 : cc); };  // 2D stores xx yy zz xy
    // the kernel block: whole 4-column runs of the blocked kernel layout by
    // bulk copies, else 16- or 4-byte asynchronous copies
    bool bulk = false;
    if constexpr (WB % 4 == 0) bulk = !nyq && a.Kblocked && kx0 + WB <= a.Kp;
    if (bulk) {
        if (tid == 0) {
            mbar_init(&kbar, 1);
            mbar_expect_tx(&kbar, (uint32_t)(sizeof(float) * ncomp * HY * WB));
            for (int cc = 0; cc < ncomp; cc++)
                for (int b4 = 0; b4 < WB / 4; b4++)
                    bulk_g2s(Ks + kcomp(cc) * HY * WB + b4 * HY * 4, a.K[kcomp(cc)] + kern_idx(a, kzm, 0, kx0 + 4 * b4, HY),
                             (uint32_t)(sizeof(float) * HY * 4), &kbar);
        }
    } else {
        bool wide = false;
        if constexpr (WB % 4 == 0) {
            // 16-byte pieces of 4 columns (plan layouts: pitch padded to 4
            // floats, pad columns zero)
            wide = !nyq && a.Kp % 4 == 0 && kx0 + WB <= a.Kp;
            if (wide) {
                constexpr int CH = WB / 4;
                for (int e = tid; e < ncomp * HY * CH; e += NT) {
                    const int cc = e / (HY * CH), r = e % (HY * CH), ky = r / CH, ch = r % CH;
                    cpa16(Ks + kcomp(cc) * HY * WB + ch * HY * 4 + ky * 4, a.K[kcomp(cc)] + kern_idx(a, kzm, ky, kx0 + 4 * ch, HY));
                }
            }
        }
        if (!wide) {
            for (int e = tid; e < ncomp * HY * WB; e += NT) {
                const int cc = e / (HY * WB), r = e % (HY * WB), ky = r / WB, ww = r % WB;
                float* dst = Ks + kcomp(cc) * HY * WB + (ww / KW) * HY * KW + ky * KW + ww % KW;
                const int kxw = nyq ? hx - 1 : kx0 + ww, kzw = nyq ? kz_mirror(by * WB + ww) : kzm;
                if (kxw < hx) cpa4(dst, a.K[kcomp(cc)] + kern_idx(a, kzw, ky, kxw, HY));
                else *dst = 0.f;
            }
        }
        cpa_commit();
    }
    if (!k3d)  // 2D: no yz / xz components; zeros keep the multiply branch-free
        for (int e = tid; e < 2 * HY * WB; e += NT) Ks[3 * HY * WB + e] = 0.f;
    const bool col = kx < hx;
    const long cs = (long)Pz * NY * a.Lx, rs = spec_rowstride(a);
    const float2* in = inst_spec(a, ib) + (long)kz * NY * a.Lx + spec_col(a, kx);
    float2 v[3][8];
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int m = 0; m < 8; m++) {
            const int y = t + T * m;
            v[c][m] = (m < 4 && col) ? in[c * cs + y * rs] : make_float2(0.f, 0.f);
        }
    __syncthreads();  // twiddles, barrier initialised
    float2* exl = ex + w * LP;
    const int exs = WB * LP;
    rg_fft_fwd_seq<PY, 3, true>(v, t, exl, exs, tw);
    if (bulk) {
        for (int it = 0; !mbar_try_wait(&kbar, 0); it++) {
            if (it == kTileWaitLimit && tid == 0) pass_timeout(a, ib);
            if (it >= 2 * kTileWaitLimit) return;
        }
    } else {
        cpa_wait_all();
    }
    __syncthreads();
    // kernel multiply (kernmulrsymm3d.cl:41-90), mirrored into the stored block
    const float* kcol = Ks + (w / KW) * HY * KW + w % KW;
#pragma unroll
    for (int m = 0; m < 8; m++) {
        const int ky = t + T * m;
        int kym = ky;
        float sy = 1.f;
        if (ky > NY) { kym = PY - ky; sy = -1.f; }
        const float* kr = kcol + kym * KW;
        const float Kxx = kr[0], Kyy = kr[HY * WB], Kzz = kr[2 * HY * WB];
        const float Kxy = kr[5 * HY * WB] * sy;
        const float Kyz = kr[3 * HY * WB] * (sy * sz);
        const float Kxz = kr[4 * HY * WB] * sz;
        const float2 mx = v[0][m], my = v[1][m], mz = v[2][m];
        // conjugated products: the inverse is conj(FFT(conj(.))); explicit
        // multiply-adds (fft.cuh: the same bits in every instantiation)
        auto dot = [](float a, float ka, float b, float kb, float c, float kc) {
            return fma_rn(c, kc, fma_rn(b, kb, mul_rn(a, ka)));
        };
        v[0][m] = make_float2(dot(mx.x, Kxx, my.x, Kxy, mz.x, Kxz), -dot(mx.y, Kxx, my.y, Kxy, mz.y, Kxz));
        v[1][m] = make_float2(dot(mx.x, Kxy, my.x, Kyy, mz.x, Kyz), -dot(mx.y, Kxy, my.y, Kyy, mz.y, Kyz));
        v[2][m] = make_float2(dot(mx.x, Kxz, my.x, Kyz, mz.x, Kzz), -dot(mx.y, Kxz, my.y, Kyz, mz.y, Kzz));
    }
    // (the barrier before the multiply separates the forward transform's last
    // reads of the exchange buffers from the inverse's first writes)
    rg_fft_fwd_seq<PY, 3, false>(v, t, exl, exs, tw);
    if (col) {
        float2* out = inst_spec(a, ib) + (long)kz * NY * a.Lx + spec_col(a, kx);
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int m = 0; m < 4; m++) {
                const int y = t + T * m;
                out[c * cs + y * rs] = make_float2(v[c][m].x, -v[c][m].y);
            }
    }
}
template <int PY, int WB>
__global__ void __launch_bounds__((PY / 8) * WB, RegBShape<PY, WB>::minb) k_reg_b(PassArgs a) {
    k_reg_b_body<PY, WB>(a, blockIdx.x, blockIdx.y, 0);
}
// batched: blockIdx.y = index + per * instance (the inst_* views above)
template <int PY, int WB>
__global__ void __launch_bounds__((PY / 8) * WB, RegBShape<PY, WB>::minb) k_reg_b_bat(PassArgs a) {
    const int per = a.Pz, b = blockIdx.y / per;
    k_reg_b_body<PY, WB>(a, blockIdx.x, blockIdx.y - b * per, b);
}

// ---- passes A and C with the register-blocked FFT (3D, power-of-two sizes)
// x transform: TX = M/8 threads per row (one row per warp or less), rows z
// of one (y, component) slab; z transform: TZ = PZ/8 threads per column.
// Shared memory: staged x and z twiddle tables (RgTw; even slot counts keep
// the later regions 16-byte aligned), the R2C twiddles twr (M), the rows Xs
// [NZ][XP] and the exchange lines (x: one line of LX slots per row, padded
// rg_pad<4> after the first stage and rg_pad<4, 2> after the later ones).
template <int M, int PZ> struct RegAC {
    static constexpr int NZ = nz_of_pz(PZ), TX = M / 8, TZ = PZ / 8, NT = NZ * TX, CPR = NT / TZ;
    static constexpr int XP = ((M + 1 + 11) / 16) * 16 + 4;  // Xs row pitch, = 4 (mod 16) against bank conflicts
    static constexpr int LX = rg_line<M, 4, 2>(), LZ = rg_line<PZ, 3>();
    static constexpr int TWX = (RgTw<M>::size + 1) & ~1, TWZ = (RgTw<PZ>::size + 1) & ~1;
    static constexpr int EXN = NZ * LX > CPR * LZ ? NZ * LX : CPR * LZ;
    static constexpr size_t smem = sizeof(float2) * ((size_t)TWX + TWZ + M + (size_t)NZ * XP + EXN);
    static constexpr bool ok = rg_ok(M) && rg_ok(PZ) && TX <= 32 && PZ % 2 == 0 && NT % TZ == 0 && NT <= 1024;
};

template <int M, int PZ>
__device__ __forceinline__ void k_reg_a_body(const PassArgs& a, const int bx, const int by, const int ib) {
    using S = RegAC<M, PZ>;
    constexpr int NZ = S::NZ, TX = S::TX, TZ = S::TZ, NT = S::NT, CPR = S::CPR, XP = S::XP;
    extern __shared__ __align__(16) float2 sm[];
    float2* twx = sm;             // staged x twiddles (RgTw<M>)
    float2* twz = twx + S::TWX;   // staged z twiddles (RgTw<PZ>)
    float2* twr = twz + S::TWZ;   // M: exp(-2 pi i k / Px)
    float2* Xs = twr + M;         // [NZ][XP]
    float2* ex = Xs + NZ * XP; // exchange lines
    if (inst_inactive(a, ib)) return;
    const int tid = threadIdx.x;
    const int y = bx, c = by, Ny = a.Ny;
    const float* __restrict__ mp = inst_m(a, ib, c);
    const float msm = inst_msmul(a, ib);
    // x phase: row z, lane t holds packed z[n] = x[2n] + i x[2n+1], n = t + TX*j
    const int z = tid / TX, t = tid % TX;
    float2 v[1][8];
    const int rowi = (z * Ny + y) * M;
    if (a.Ms == nullptr && a.vol == nullptr) {
        // uniform Ms, no geometry: MU0*Ms once, and the pair (x, x+1) in one
        // 8-byte load (scaled_m's rounding: (bsat * 1) * m = bsat * m)
        const float bsat = (float)(kMu0f * (double)msm);
#pragma unroll
        for (int j = 0; j < 8; j++) {
            if (j < 4) {
                const float2 p = __ldg(reinterpret_cast<const float2*>(mp + rowi + 2 * (t + TX * j)));
                v[0][j] = make_float2(__fmul_rn(bsat, p.x), __fmul_rn(bsat, p.y));
            } else {
                v[0][j] = make_float2(0.f, 0.f);
            }
        }
    } else {
#pragma unroll
        for (int j = 0; j < 8; j++) {
            if (j < 4) {  // n < M/2 carries data, the rest is zero padding
                const int i = rowi + 2 * (t + TX * j);
                v[0][j] = make_float2(scaled_m(a, mp, i, msm), scaled_m(a, mp, i + 1, msm));
            } else {
                v[0][j] = make_float2(0.f, 0.f);
            }
        }
    }
    // the twiddle tables while the loads of m are in flight
    for (int i = tid; i < M; i += NT) twr[i] = a.twr[i];
    rg_tw_fill<M>(twx, a.fx.tw, tid, NT);
    if constexpr (PZ != 16 && PZ != 32) rg_tw_fill<PZ>(twz, a.fz.tw, tid, NT);  // (the pair z phase has none)
    __syncthreads();
    rg_fft_fwd<M, 1, true, 4, rg_radix(M, 0) == 8, 2>(v, t, ex + z * S::LX, 0, twx);  // n >= M/2 is zero padding
    // R2C unpack: partner element Z[M-k] lives in lane (TX - t) % TX, element 7-j
    // (or (8-j) & 7 for t = 0); exchanged with warp shuffles.
    const int lane = threadIdx.x & 31;
    const int plane = (lane & ~(TX - 1)) | ((TX - t) & (TX - 1));
    float2 Bv[8];
#pragma unroll
    for (int s = 0; s < 8; s++) {
        float2 r;
        r.x = __shfl_sync(0xffffffffu, v[0][s].x, plane);
        r.y = __shfl_sync(0xffffffffu, v[0][s].y, plane);
        if (t != 0) Bv[7 - s] = r;
        else Bv[(8 - s) & 7] = r;
    }
    float2* xrow = Xs + z * XP;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const int k = t + TX * j;
        const float2 A = v[0][j], B = Bv[j];
        float2 E = make_float2(0.5f * (A.x + B.x), 0.5f * (A.y - B.y));
        float2 D = make_float2(0.5f * (A.x - B.x), 0.5f * (A.y + B.y));
        float2 O = make_float2(D.y, -D.x);
        float2 W = twr[k];
        float2 WO = make_float2(W.x * O.x - W.y * O.y, W.x * O.y + W.y * O.x);
        xrow[k] = make_float2(E.x + WO.x, E.y + WO.y);
        if (k == 0) xrow[M] = make_float2(A.x - A.y, 0.f);  // Nyquist: Re Z0 - Im Z0
    }
    __syncthreads();
    float2* out = inst_spec(a, ib) + (long)c * PZ * Ny * a.Lx + (long)y * spec_rowstride(a);
    const long kzs = (long)Ny * a.Lx;
    if constexpr (PZ == 16 || PZ == 32) {
        // z phase on lane pairs, decimation in frequency: with x[n] = 0 for
        // n >= PZ/2, X[2r + t] = DFT_{PZ/2}( x[n] W_PZ^{n t} )[r], so lane t
        // of a pair produces the kz of parity t from the same PZ/2 inputs --
        // no exchange and no twiddle table.  The DC and Nyquist columns are
        // real in z and share one transform P of (x0 + i xM), split by
        // Hermitian symmetry (X0 = (P[k] + conj P[-k]) / 2, XM = (P[k] -
        // conj P[-k]) / 2i); P[-k] has the parity of k, so it is in the lane.
        constexpr int E2 = PZ / 2, CP2 = NT / 2;
        static_assert(E2 == NZ && M % CP2 == 0, "pair z phase");
        static_assert(NT % 32 == 0, "whole warps of lane pairs");
        // pair partners are lanes l and l ^ 16: a half-warp reads and writes 16
        // consecutive columns of one row
        const int t2 = (tid >> 4) & 1, cl2 = ((tid >> 5) << 4) | (tid & 15);
        const long kM = spec_col(a, M);
        // With one column per pair, the (y, component) slab of the blocked
        // spectrum is assembled in the x/z scratch ([kz][kx/4][kx%4], 128-byte
        // aligned; Xs is read into registers first) and written by one bulk
        // tensor store (the slab map pass C loads with), not by 8-byte
        // stores from every thread.
        constexpr bool kSlabShape = M / CP2 == 1;
        const bool slab = kSlabShape && a.slab_map != nullptr && ib == 0 && (smem_u32(Xs) & 15u) == 0;
        const int KB = a.Lx >> 2;
        float2* const sl = Xs + ((128u - (smem_u32(Xs) & 127u)) & 127u) / sizeof(float2);
#pragma unroll
        for (int r0 = 0; r0 < M / CP2; r0++) {
            const int kx = r0 * CP2 + cl2;
            const bool pk = kx == 0;
            float2 u[E2];
#pragma unroll
            for (int n = 0; n < E2; n++) {
                float2 q = Xs[n * XP + kx];
                if (pk) q.y = Xs[n * XP + M].x;
                u[n] = q;
            }
            if (slab) __syncthreads();  // every Xs read is done before the slab overwrites it
            if (t2) tw_ramp<PZ, 1, 0, E2>(u);
            reg_dft<E2>(u);  // u[r] = X[2r + t2]
            if (pk) {
#pragma unroll
                for (int r = 0; r < E2; r++) {
                    const float2 P = u[r], Q = t2 ? u[E2 - 1 - r] : u[(E2 - r) & (E2 - 1)];
                    const int kz = 2 * r + t2;
                    const float2 X0 = make_float2(0.5f * (P.x + Q.x), 0.5f * (P.y - Q.y));
                    const float2 XM = make_float2(0.5f * (P.y + Q.y), -0.5f * (P.x - Q.x));
                    if (slab) {
                        sl[kz * KB * 4] = X0;
                        sl[(kz * KB + (M >> 2)) * 4 + (M & 3)] = XM;
                    } else {
                        out[(long)kz * kzs] = X0;
                        out[(long)kz * kzs + kM] = XM;
                    }
                }
            } else if (slab) {
#pragma unroll
                for (int r = 0; r < E2; r++) sl[((2 * r + t2) * KB + (kx >> 2)) * 4 + (kx & 3)] = u[r];
            } else {
                const long ko = spec_col(a, kx);
#pragma unroll
                for (int r = 0; r < E2; r++) out[(long)(2 * r + t2) * kzs + ko] = u[r];
            }
        }
        if (slab) {
            // the block's padding columns M+1 .. 4 KB - 1 (read by no pass) as zeros
            const int padc = 4 * KB - (M + 1);
            for (int e = tid; e < PZ * padc; e += NT) {
                const int kz = e / padc, kx = M + 1 + e % padc;
                sl[(kz * KB + (kx >> 2)) * 4 + (kx & 3)] = make_float2(0.f, 0.f);
            }
            fence_proxy_async();
            __syncthreads();
            if (tid == 0) {
                tma_store_5d(a.slab_map, sl, 0, y, 0, 0, c);
                bulk_commit();
                bulk_wait_read0();
            }
        }
    } else {
        // z phase: column kx, TZ lanes, rows z = tz + TZ*j (zero padding for j >= 4).
        // The DC and Nyquist columns are real in z, so they share one complex
        // transform (x0 + i xM), split afterwards by Hermitian symmetry:
        // X0[k] = (P[k] + conj P[-k]) / 2, XM[k] = (P[k] - conj P[-k]) / 2i.
        // The M - 1 other columns then fill exactly M / CPR = 2 rounds.
        static_assert(M == 2 * CPR, "z rounds: M columns over CPR column groups");
        const int tz = tid % TZ, cl = tid / TZ;
        float2* exz = ex + cl * S::LZ;
    #pragma unroll
        for (int r = 0; r < 2; r++) {
            const int kx = r * CPR + cl;
            const bool pk = kx == 0;
            float2 u[1][8];
    #pragma unroll
            for (int j = 0; j < 8; j++) {
                float2 q = make_float2(0.f, 0.f);
                if (j < 4) {
                    q = Xs[(tz + TZ * j) * XP + kx];
                    if (pk) q.y = Xs[(tz + TZ * j) * XP + M].x;
                }
                u[0][j] = q;
            }
            rg_fft_fwd<PZ, 1, true>(u, tz, exz, 0, twz);
            if (r == 0 && tid < 32) {  // the warp holding column group 0
                const int pl = (lane & ~(TZ - 1)) | ((TZ - tz) & (TZ - 1));
                float2 pr[8];
    #pragma unroll
                for (int s = 0; s < 8; s++) {
                    float2 q;
                    q.x = __shfl_sync(0xffffffffu, u[0][s].x, pl);
                    q.y = __shfl_sync(0xffffffffu, u[0][s].y, pl);
                    if (tz != 0) pr[7 - s] = q;
                    else pr[(8 - s) & 7] = q;
                }
                if (pk) {
    #pragma unroll
                    for (int j = 0; j < 8; j++) {
                        const float2 P = u[0][j], Q = pr[j];
                        out[(tz + TZ * j) * kzs] = make_float2(0.5f * (P.x + Q.x), 0.5f * (P.y - Q.y));
                        out[(tz + TZ * j) * kzs + spec_col(a, M)] = make_float2(0.5f * (P.y + Q.y), -0.5f * (P.x - Q.x));
                    }
                    continue;
                }
            }
            const long ko = spec_col(a, kx);
    #pragma unroll
            for (int j = 0; j < 8; j++) out[(tz + TZ * j) * kzs + ko] = u[0][j];
        }
    }
}
template <int M, int PZ>
__global__ void __launch_bounds__(RegAC<M, PZ>::NT) k_reg_a(PassArgs a) { k_reg_a_body<M, PZ>(a, blockIdx.x, blockIdx.y, 0); }
// batched: blockIdx.y = index + per * instance (the inst_* views above)
template <int M, int PZ>
__global__ void __launch_bounds__(RegAC<M, PZ>::NT) k_reg_a_bat(PassArgs a) {
    const int per = 3, b = blockIdx.y / per;
    k_reg_a_body<M, PZ>(a, blockIdx.x, blockIdx.y - b * per, b);
}

template <int M, int PZ>
__device__ __forceinline__ void k_reg_c_body(const PassArgs& a, const int bx, const int by, const int ib) {
    using S = RegAC<M, PZ>;
    constexpr int NZ = S::NZ, TX = S::TX, TZ = S::TZ, NT = S::NT, CPR = S::CPR, XP = S::XP;
    extern __shared__ __align__(16) float2 sm[];
    float2* twx = sm;
    float2* twz = twx + S::TWX;
    float2* twr = twz + S::TWZ;
    float2* Xs = twr + M;
    float2* ex = Xs + NZ * XP;
    if (inst_inactive(a, ib)) return;
    const int tid = threadIdx.x;
    // the (y, component) slab of the spectrum by one bulk tensor copy into
    // the x/z scratch (Xs and the exchange lines, idle until the z phase has
    // its inputs in registers): [kz][kx/4][kx%4] complex
    constexpr bool kSlabShape = (PZ == 16 || PZ == 32) && M / (NT / 2) == 1;
    __shared__ __align__(8) uint64_t slab_bar;
    // (Xs is 16-byte aligned, so the 128-byte rounding below moves it by a
    // whole number of float2)
    const bool slab = kSlabShape && a.slab_map != nullptr && ib == 0 && (smem_u32(Xs) & 15u) == 0;
    const int y = bx, c = by, Ny = a.Ny;
    const int KB = a.Lx >> 2;  // four-column blocks per kz row of the slab
    // the copy's destination on a 128-byte boundary (the dynamic region
    // need not start on one; the plan leaves 128 bytes of slack)
    float2* const sl = Xs + ((128u - (smem_u32(Xs) & 127u)) & 127u) / sizeof(float2);
    // the copy is issued first (its initialisation is fenced for the async
    // proxy), so that it is in flight while the twiddle tables are filled;
    // the barrier below makes the initialisation visible to the other threads
    if (slab && tid == 0) {
        mbar_init(&slab_bar, 1);
        mbar_expect_tx(&slab_bar, (uint32_t)(sizeof(float2) * 4 * KB * PZ));
        tma_load_5d(sl, a.slab_map, 0, y, 0, 0, c, &slab_bar);
    }
    for (int i = tid; i < M; i += NT) twr[i] = a.twr[i];
    rg_tw_fill<M>(twx, a.fx.tw, tid, NT);
    if constexpr (PZ != 16 && PZ != 32) rg_tw_fill<PZ>(twz, a.fz.tw, tid, NT);  // (the pair z phase has none)
    __syncthreads();
    if (slab) {
        for (int it = 0; !mbar_try_wait(&slab_bar, 0); it++) {
            if (it == kTileWaitLimit && tid == 0) pass_timeout(a, ib);
            if (it >= 2 * kTileWaitLimit) return;
        }
    }
    const float2* in = inst_spec(a, ib) + (long)c * PZ * Ny * a.Lx + (long)y * spec_rowstride(a);
    const long kzs = (long)Ny * a.Lx;
    if constexpr (PZ == 16 || PZ == 32) {
        // z phase on lane pairs, inverse by the conjugate trick, decimation in
        // time: partner t transforms the samples kz = 2j + t (u = conj G),
        // partner 1 scales by W_PZ^k, and the kept outputs z < PZ/2 are
        // X[z] = A[z] + W^z B[z]; partner 0 forms z < PZ/4 and 1 the rest,
        // exchanging one value per output by shuffle.  The DC and Nyquist
        // columns invert to real sequences and share one transform of
        // G0 + i GM (real part -> column 0, imaginary -> column M).
        constexpr int E2 = PZ / 2, H2 = E2 / 2, CP2 = NT / 2;
        static_assert(E2 == NZ && M % CP2 == 0, "pair z phase");
        // pair partners are lanes l and l ^ 16: a half-warp reads and writes 16
        // consecutive columns of one row (conflict-free in shared memory)
        static_assert(NT % 32 == 0, "whole warps of lane pairs");
        const int t2 = (tid >> 4) & 1, cl2 = ((tid >> 5) << 4) | (tid & 15);
        const long kM = spec_col(a, M);
#pragma unroll
        for (int r0 = 0; r0 < M / CP2; r0++) {
            const int kx = r0 * CP2 + cl2;
            const bool pk = kx == 0;
            const long ko = spec_col(a, kx);
            float2 u[E2];
#pragma unroll
            for (int j = 0; j < E2; j++) {
                const int kz = 2 * j + t2;
                float2 q, g;
                if (slab) {
                    q = sl[(kz * KB + (kx >> 2)) * 4 + (kx & 3)];
                    g = sl[(kz * KB + (M >> 2)) * 4 + (M & 3)];
                } else {
                    q = in[(long)kz * kzs + ko];
                    g = pk ? in[(long)kz * kzs + kM] : make_float2(0.f, 0.f);
                }
                if (pk) q = make_float2(q.x - g.y, q.y + g.x);
                u[j] = make_float2(q.x, -q.y);
            }
            if (slab) __syncthreads();  // every input is in registers before Xs is written
            reg_dft<E2>(u);
            if (t2) tw_ramp<PZ, 1, 0, E2>(u);
#pragma unroll
            for (int i = 0; i < H2; i++) {
                const float2 snd = t2 ? u[i] : u[H2 + i];
                float2 rcv;
                rcv.x = __shfl_xor_sync(0xffffffffu, snd.x, 16);
                rcv.y = __shfl_xor_sync(0xffffffffu, snd.y, 16);
                const float2 own = t2 ? u[H2 + i] : u[i];
                const float2 X = make_float2(own.x + rcv.x, own.y + rcv.y);
                const int z = i + H2 * t2;
                if (pk) {
                    Xs[z * XP] = make_float2(X.x, 0.f);
                    Xs[z * XP + M] = make_float2(-X.y, 0.f);
                } else {
                    Xs[z * XP + kx] = make_float2(X.x, -X.y);
                }
            }
        }
    } else {
        // z phase: inverse transform (conjugate trick) of every column, keep z < NZ.
        // The DC and Nyquist columns invert to real sequences, so they share one
        // transform of G0 + i GM (real part -> column 0, imaginary -> column M);
        // the other columns fill exactly two rounds, whose loads are all issued
        // before the first transform.
        static_assert(M == 2 * CPR, "z rounds: M columns over CPR column groups");
        const int tz = tid % TZ, cl = tid / TZ;
        float2* exz = ex + cl * S::LZ;
        float2 u[2][1][8];
    #pragma unroll
        for (int r = 0; r < 2; r++) {
            const long ko = spec_col(a, r * CPR + cl), kM = spec_col(a, M);
    #pragma unroll
            for (int j = 0; j < 8; j++) {
                float2 q = in[(tz + TZ * j) * kzs + ko];
                if (r == 0 && cl == 0) {
                    const float2 g = in[(tz + TZ * j) * kzs + kM];
                    q = make_float2(q.x - g.y, q.y + g.x);
                }
                u[r][0][j] = make_float2(q.x, -q.y);
            }
        }
    #pragma unroll
        for (int r = 0; r < 2; r++) {
            const int kx = r * CPR + cl;
            rg_fft_fwd<PZ, 1, true>(u[r], tz, exz, 0, twz);
            if (r == 0 && cl == 0) {
    #pragma unroll
                for (int j = 0; j < 4; j++) {
                    Xs[(tz + TZ * j) * XP] = make_float2(u[r][0][j].x, 0.f);
                    Xs[(tz + TZ * j) * XP + M] = make_float2(-u[r][0][j].y, 0.f);
                }
            } else {
    #pragma unroll
                for (int j = 0; j < 4; j++) Xs[(tz + TZ * j) * XP + kx] = make_float2(u[r][0][j].x, -u[r][0][j].y);
            }
        }
    }
    __syncthreads();
    // x phase: C2R pack Z[k] = (X[k] + conj X[M-k]) + i conj(W^k)(X[k] - conj X[M-k]),
    // inverse transform by the conjugate trick, even/odd samples to B
    const int z = tid / TX, t = tid % TX;
    const float2* xrow = Xs + z * XP;
    float2 v[1][8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const int k = t + TX * j;
        float2 Xk = xrow[k], Xm = xrow[M - k];
        if (k == 0) { Xk.y = 0.f; Xm.y = 0.f; }
        const float2 W = twr[k];
        const float2 S1 = make_float2(Xk.x + Xm.x, Xk.y - Xm.y);
        const float2 D1 = make_float2(Xk.x - Xm.x, Xk.y + Xm.y);
        const float2 T1 = make_float2(W.x * D1.x + W.y * D1.y, W.x * D1.y - W.y * D1.x);
        v[0][j] = make_float2(S1.x - T1.y, -(S1.y + T1.x));  // conj(Z[k])
    }
    rg_fft_fwd<M, 1, true, 4, false, 2>(v, t, ex + z * S::LX, 0, twx);
    float* __restrict__ B = inst_B(a, ib, c);
    const int rowo = (z * Ny + y) * M;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int n = t + TX * j;
        *reinterpret_cast<float2*>(B + rowo + 2 * n) = make_float2(v[0][j].x, -v[0][j].y);
    }
}
// three 512-thread CTAs per SM (40 registers): measured faster for pass C on
// the 256x256x16 multilayer (28.8 -> 27.0 us); pass A keeps two (it spills)
template <int M, int PZ>
__global__ void __launch_bounds__(RegAC<M, PZ>::NT, (RegAC<M, PZ>::NT <= 512 ? 3 : 1))
    k_reg_c(PassArgs a) { k_reg_c_body<M, PZ>(a, blockIdx.x, blockIdx.y, 0); }
// batched: blockIdx.y = index + per * instance (the inst_* views above)
template <int M, int PZ>
__global__ void __launch_bounds__(RegAC<M, PZ>::NT) k_reg_c_bat(PassArgs a) {
    const int per = 3, b = blockIdx.y / per;
    k_reg_c_body<M, PZ>(a, blockIdx.x, blockIdx.y - b * per, b);
}

template <int PY> struct RegB {
    static constexpr int T = PY / 8;
    static constexpr int WB = T >= 256 ? 1 : 256 / T > 16 ? 16 : 256 / T;
    static constexpr int NT = T * WB;
    static constexpr size_t smem = RegBShape<PY, WB>::smem;
};

// one warp per CTA (or one column): for small meshes, where the default
// shape leaves most SMs idle
template <int PY> struct RegBNarrow {
    static constexpr int T = PY / 8;
    static constexpr int WB = T >= 32 ? 1 : 32 / T;
    static constexpr int NT = T * WB;
    static constexpr size_t smem = RegBShape<PY, WB>::smem;
};

// ------------------------------------------------------------------ dispatch
template <int M, int PZ> static void fill_ac(FastPasses& f) {
    if constexpr (RegAC<M, PZ>::ok && PZ >= 8) {
        f.a = k_reg_a<M, PZ>;
        f.c = k_reg_c<M, PZ>;
        f.ab = k_reg_a_bat<M, PZ>;
        f.cb = k_reg_c_bat<M, PZ>;
        f.smem_ac = RegAC<M, PZ>::smem;
        f.ac_scratch = sizeof(float2) * ((size_t)RegAC<M, PZ>::NZ * RegAC<M, PZ>::XP + RegAC<M, PZ>::EXN);
        f.slab_ok = (PZ == 16 || PZ == 32) && M / (RegAC<M, PZ>::NT / 2) == 1;
        f.nt_ac = RegAC<M, PZ>::NT;
        f.ac_reg = true;
    } else {
        f.a = k_fast_a<M, PZ>;
        f.c = k_fast_c<M, PZ>;
        f.ab = k_fast_a_bat<M, PZ>;
        f.cb = k_fast_c_bat<M, PZ>;
        f.smem_ac = AcShape<M, PZ>::smem;
        f.nt_ac = kNT;
    }
}
template <int PY> static void fill_b(FastPasses& f) {
    if constexpr (rg_ok(PY) && PY >= 32) {
        f.b = k_reg_b<PY, RegB<PY>::WB>;
        f.bb = k_reg_b_bat<PY, RegB<PY>::WB>;
        f.smem_b = RegB<PY>::smem;
        f.wb = RegB<PY>::WB;
        f.nt_b = RegB<PY>::NT;
        f.b_reg = true;
        if constexpr (RegBNarrow<PY>::WB < RegB<PY>::WB) {
            f.b_n = k_reg_b<PY, RegBNarrow<PY>::WB>;
            f.smem_b_n = RegBNarrow<PY>::smem;
            f.wb_n = RegBNarrow<PY>::WB;
            f.nt_b_n = RegBNarrow<PY>::NT;
        }
    } else {
        f.b = k_fast_b<PY>;
        f.bb = k_fast_b_bat<PY>;
        f.smem_b = BShape<PY>::smem;
        f.wb = BShape<PY>::WB;
        f.nt_b = kNTB;
    }
}

bool demag_fast_select(int M, int Py, int Pz, FastPasses& f) {
    f = FastPasses{};
    bool ac = true;
#define AC(m, pz) else if (M == m && Pz == pz) fill_ac<m, pz>(f);
    if (false) {}
    AC(16, 1) AC(24, 1) AC(32, 1) AC(48, 1) AC(64, 1) AC(96, 1) AC(128, 1) AC(192, 1) AC(256, 1) AC(384, 1)
    AC(512, 1) AC(1024, 1)
    AC(64, 12) AC(64, 16) AC(64, 32) AC(64, 64)
    AC(128, 12) AC(128, 16) AC(128, 32) AC(128, 64)
    AC(256, 12) AC(256, 16) AC(256, 32) AC(256, 64)
    AC(512, 12) AC(512, 16) AC(512, 32) AC(512, 64)
    else ac = false;
#undef AC
    bool b = true;
#define BB(py) else if (Py == py) fill_b<py>(f);
    if (false) {}
    BB(32) BB(48) BB(64) BB(96) BB(128) BB(192) BB(256) BB(384) BB(512) BB(1024) BB(2048)
    else b = false;
#undef BB
    if (!(ac && b)) f = FastPasses{};
    // 4-column-block spectrum layout when all three passes are register kernels
    f.blocked = ac && b && f.ac_reg && f.b_reg;
    return ac && b;
}

int demag_fast_grid(FastPasses& f, int M, int Pz, int sm_count) {
    if (sm_count <= 0) sm_count = ctx().sm_count;
    f.gbx = (unsigned)((M + 1 + f.wb - 1) / f.wb);
    f.gby = (unsigned)Pz;
    // a default pass-B grid smaller than the SM count runs on a few SMs: such
    // plans use CTAs of one warp instead for a single mesh (batched launches
    // have CTAs enough and keep the default); the arithmetic per column is
    // the same, bit for bit, because the butterflies and the kernel multiply
    // spell out their rounding (fft.cuh)
    if (f.b_n) {
        f.gbx_n = (unsigned)((M + 1 + f.wb_n - 1) / f.wb_n);
        f.use_narrow = (long)f.gbx * f.gby < sm_count;
    }
    return UMAG_OK;
}

static int demag_fast_setup_device();

int demag_fast_setup() {
    // cudaFuncSetAttribute applies to the current device's context, so the
    // opt-in is made once per device, under a lock (host threads may race)
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    UMAG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(UMAG_E_ARG, "device %d out of range", dev);
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return UMAG_OK;
    UMAG_TRY(demag_fast_setup_device());
    done[dev] = true;
    return UMAG_OK;
}

static int demag_fast_setup_device() {
    // opt in to the full 227 KB and ask for the largest shared-memory carveout,
    // so several CTAs of these shared-memory-heavy kernels fit on one SM
    auto attrs = [](void (*k)(PassArgs)) -> int {
        cudaFuncAttributes fa;  // the opt-in covers static + dynamic shared memory
        UMAG_CUDA(cudaFuncGetAttributes(&fa, k));
        UMAG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       227 * 1024 - (int)fa.sharedSizeBytes));
        UMAG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       cudaSharedmemCarveoutMaxShared));
        return UMAG_OK;
    };
    FastPasses f;
    const int Ms[] = {16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512, 1024};
    for (int m : Ms)
        if (demag_fast_select(m, 2 * m > 2048 ? 2048 : 2 * m, 1, f)) {
            UMAG_TRY(attrs(f.a));
            UMAG_TRY(attrs(f.c));
            UMAG_TRY(attrs(f.ab));
            UMAG_TRY(attrs(f.cb));
        }
    const int m3[] = {64, 128, 256, 512}, pz3[] = {12, 16, 32, 64};
    for (int m : m3)
        for (int pz : pz3)
            if (demag_fast_select(m, 2 * m, pz, f)) {
                UMAG_TRY(attrs(f.a));
                UMAG_TRY(attrs(f.c));
                UMAG_TRY(attrs(f.ab));
                UMAG_TRY(attrs(f.cb));
            }
    // pass B instantiations
    {
        FastPasses g{};
#define SETB(py)                                     \
    fill_b<py>(g);                                   \
    UMAG_TRY(attrs(g.b));                            \
    UMAG_TRY(attrs(g.bb));                           \
    if (g.b_n) UMAG_TRY(attrs(g.b_n));
        SETB(32) SETB(48) SETB(64) SETB(96) SETB(128) SETB(192) SETB(256) SETB(384) SETB(512) SETB(1024) SETB(2048)
#undef SETB
    }
    return UMAG_OK;
}

}  // namespace umag
