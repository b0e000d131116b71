// engine.cu -- a whole simulation on the device: effective field, torque,
// RK45DP / RK23 / Heun / RK4 steppers and the step controller.
//
// Restates engine/effectivefield.go, engine/torque.go, engine/rk45dp.go,
// engine/rk23.go, engine/heun.go, engine/rk4.go, engine/stepcontroller.go
// and engine/run.go:150-188 (adaptDt).  The solver state (time, dt in FP64,
// counters, accept/reject decision) lives in device memory and is updated
// by a one-thread controller kernel, so a step never waits for the host and
// many steps are replayed from one CUDA graph.  Buffers are addressed
// through a device-side slot table: accepting a step swaps the state and
// working magnetisation slots and moves k7 into the k1 slot (FSAL,
// engine/stepcontroller.go:76-78) without copying.
#include <cmath>
#include <cstddef>
#include <cstring>
#include <thread>
#include <vector>

#include "cellmath.cuh"
#include "common.cuh"
#include "demag.cuh"
#include "engine.cuh"
#include "ops.cuh"
#include "tile.cuh"

namespace umag {

// ---------------------------------------------------------------- device state
constexpr double kBoltzmann = 1.380650424e-23;  // mag/constants.go:9 Kb

struct DevCtl {
    float* m;        // state magnetisation (3N, SoA)
    float* mw;       // working / stage magnetisation
    float* k[7];     // stage torques
    float* bd;       // demag field of this instance (batched ensembles)
    double t, dt, t0, alarm, stop;
    float h;         // float32(dt * GammaLL) of the step in progress
    int active;      // 0: the step in progress is skipped (stop time reached)
    unsigned int err2, dm2, rel;  // float bit patterns, atomicMax targets
    int nan_seen;
    int accepted;
    double last_err, peak_err, last_torque;
    long long nsteps, nundone, nevals;
    int status;
    double max_err, rel_err, min_dt, max_dt, fix_dt, headroom, min_slope, gamma;
    // thermal field: k2 = float32(2 kB / ((GammaLL V) dt)) of the step in
    // progress (engine/temperature.go:111); therm_gv = GammaLL V (0: no thermal field)
    double therm_gv;
    float k2;
};

// Uniform parameters evaluated once on the device with the operations the
// per-cell path uses (bit-identical), so the per-cell kernel does no
// divisions or square roots for them.
struct LocalConsts {
    float inv_ms;  // inv_msat of a uniform Ms (amul.clh:19-26)
    float gilb;    // -1/(1+alpha^2) of a uniform alpha (lltorque2.cl:18)
    float u[3];    // normalised uniform easy axis (uniaxialanisotropy2.cl:19)
    float f1k;     // 2*(K1/Ms) for uniform K1 and Ms
    float f2k;     // 4*(K2/Ms) for uniform K2 and Ms
    PairCoef pc;   // region (0,0) exchange / DMI coefficients
};

// Per-instance uniform parameters of a batched ensemble (one record per
// instance, device memory): the LocalConsts of that instance's material,
// alpha, the applied field and Ms.
struct InstParams {
    LocalConsts kc;
    float alpha_mul, Ms_mul;
    float bext[3];
    int dmi;  // this instance uses the exchange+DMI stencil (engine/exchange.go:49-66: Dind != 0)
};

struct LocalArgs {
    Mesh3 g;
    int N;
    DevCtl* ctl;
    int m_sel;           // 0: ctl->m, 1: ctl->mw
    int out_slot;        // torque -> ctl->k[out_slot]
    float* tau_direct;   // if set, torque goes here instead
    float* beff;         // optional B_eff output
    const float* bd;     // demag field or NULL
    const float* aLUT;
    const float* dLUT;
    const uint8_t* regions;
    float wx, wy, wz, cx, cy, cz;
    int dmi, openbc, anis, zeeman, precess;
    const float* frozen;  // FrozenSpins LUT (256) or NULL
    const float* nodemag; // NoDemagSpins LUT (256) or NULL: demag field zeroed there
    int cubic;            // cubic anisotropy on (cp)
    CubicParams cp;
    const float* dbLUT;   // bulk DMI LUT or NULL
    int thermal;          // thermal field on (off while relaxing)
    const float* temp;
    float temp_mul;
    unsigned long long seed;
    int ms_uniform, alpha_uniform, anis_uniform;
    DmiPairLut dl;
    LocalConsts kc;
    UniaxParams up;
    const float* bext[3];
    const float* alpha;
    float alpha_mul;
    const float* Ms;
    float Ms_mul;
    const InstParams* ip;  // batched: per-instance parameters (uniform maps only)
    const float* mbuf1;    // the second magnetisation buffer (selects the tile map)
};

__global__ void k_local_consts(LocalArgs a, LocalConsts* out) {
    LocalConsts c{};
    c.inv_ms = a.Ms_mul == 0.0f ? 0.0f : fd(1.0f, a.Ms_mul);
    c.gilb = fd(-1.0f, fa(1.0f, fm(a.alpha_mul, a.alpha_mul)));
    f3 u{a.up.ux_mul, a.up.uy_mul, a.up.uz_mul};
    float len = __fsqrt_rn(dot3(u, u));
    float il = (len != 0.0f) ? fd(1.0f, len) : 0.0f;
    c.u[0] = fm(il, u.x); c.u[1] = fm(il, u.y); c.u[2] = fm(il, u.z);
    c.f1k = fm(2.0f, fm(a.up.K1_mul, c.inv_ms));
    c.f2k = fm(4.0f, fm(a.up.K2_mul, c.inv_ms));
    const float A = a.aLUT[0];
    c.pc.wax = fm(a.wx, A);
    c.pc.way = fm(a.wy, A);
    c.pc.waz = fm(a.wz, A);
    const float D = a.dLUT ? a.dLUT[0] : 0.0f;
    c.pc.sx = fd(fm(2.0f, A), fm(a.cx, a.cx));
    c.pc.sy = fd(fm(2.0f, A), fm(a.cy, a.cy));
    c.pc.sz = fd(fm(2.0f, A), fm(a.cz, a.cz));
    c.pc.dcx = fd(D, a.cx);
    c.pc.dcy = fd(D, a.cy);
    const float t = fd(fm(0.5f, D), A);
    c.pc.qx = fm(a.cx, t);
    c.pc.qy = fm(a.cy, t);
    *out = c;
}

// DMI coefficients per region pair (see DmiPairLut)
__global__ void k_dmi_pairs(const float* __restrict__ aLUT, const float* __restrict__ dLUT, float cx, float cy,
                            float cz, float* sx, float* sy, float* sz, float* dcx, float* dcy, float* qx, float* qy,
                            int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float A = aLUT[i], D = dLUT[i];
        sx[i] = fd(fm(2.0f, A), fm(cx, cx));
        sy[i] = fd(fm(2.0f, A), fm(cy, cy));
        sz[i] = fd(fm(2.0f, A), fm(cz, cz));
        dcx[i] = fd(D, cx);
        dcy[i] = fd(D, cy);
        float t = fd(fm(0.5f, D), A);
        qx[i] = fm(cx, t);
        qy[i] = fm(cy, t);
    }
}

__device__ __forceinline__ f3 lltorque_g(f3 m, f3 H, float alpha, float gilb) {
    f3 mxH = cross3(m, H);
    f3 mmxH = cross3(m, mxH);
    return f3{fm(gilb, fa(mxH.x, fm(alpha, mmxH.x))), fm(gilb, fa(mxH.y, fm(alpha, mmxH.y))),
              fm(gilb, fa(mxH.z, fm(alpha, mmxH.z)))};
}

// engine/effectivefield.go:14-24 + engine/torque.go:135-144 for one cell:
// B = demag; B += exchange(+DMI)/Ms; B += anisotropy; B += B_ext; torque.
// UREG: every cell is in region 0 (no region map), so the region-pair
// coefficients are scalars and no region is loaded.  TILE (with UREG, not
// BAT, non-periodic mesh): the CTA's magnetisation tile with its halo comes
// into shared memory by one TMA load (tile.cuh) and the stencils read it.
// UNI (with UREG, not BAT): a uniform material with only the common terms --
// uniform Ms, alpha and anisotropy, precession on, no OpenBC, and no
// NoDemagSpins, bulk DMI, cubic anisotropy, thermal field, FreezeSpins or
// B_eff output --
// so that those tests and branches leave the instruction stream; the
// arithmetic is the same operations in the same order.
template <bool UREG, bool BAT, bool TILE, bool UNI = false>
__global__ void __launch_bounds__(256) k_local_torque(const __grid_constant__ LocalArgs a,
                                                      const __grid_constant__ TileMaps tm) {
    static_assert(!TILE || (UREG && !BAT), "tiles: region-free, not batched");
    static_assert(!UNI || (UREG && !BAT), "uniform material: region-free, not batched");
    // BAT: blockIdx.z = iz + Nz * instance; the instance's controller,
    // demag field and uniform parameters replace the shared ones
    static_assert(!BAT || UREG, "batched ensembles have no region maps");
    int iz = blockIdx.z;
    DevCtl* ctl = a.ctl;
    const float* bd = a.bd;
    const LocalConsts* kcp = &a.kc;
    float alpha_mul = a.alpha_mul;
    const InstParams* ip = nullptr;
    if constexpr (BAT) {
        const int b = iz / a.g.Nz;
        iz -= b * a.g.Nz;
        ctl += b;
        bd = ctl->bd;
        ip = a.ip + b;
        kcp = &ip->kc;
        alpha_mul = ip->alpha_mul;
    }
    const LocalConsts& kc = *kcp;
    const bool dmi = BAT ? ip->dmi != 0 : a.dmi != 0;
    if (!ctl->active) return;
    int ix = blockIdx.x * blockDim.x + threadIdx.x;
    int iy = blockIdx.y * blockDim.y + threadIdx.y;
    const int N = a.N;
    const float* m = a.m_sel ? ctl->mw : ctl->m;
    const float *mx = m, *my = m + N, *mz = m + 2 * N;
    TileView tv{};
    if constexpr (TILE) {
        extern __shared__ __align__(128) float tile_raw[];
        __shared__ __align__(8) uint64_t bar;
        // the copy's destination on a 128-byte boundary whatever the offset of
        // the dynamic region (launched with 128 bytes of slack)
        float* const tile = tile_raw + ((128u - (smem_u32(tile_raw) & 127u)) & 127u) / sizeof(float);
        const bool three_d = a.g.Nz > 1;
        const uint32_t bytes = (uint32_t)tile_bytes(blockDim.x, blockDim.y, a.g.Nz);
        const bool leader = threadIdx.x == 0 && threadIdx.y == 0;
        if (leader) mbar_init(&bar, 1);
        __syncthreads();
        if (leader) {
            mbar_expect_tx(&bar, bytes);
            tma_load_4d(tile, &tm.map[m == a.mbuf1 ? 1 : 0], (int)(blockIdx.x * blockDim.x) - kTileHaloX,
                        (int)(blockIdx.y * blockDim.y) - 1, three_d ? iz - 1 : iz, 0, &bar);
        }
        // bounded wait: past the limit flag the failure, wait once more for
        // the copy in flight, and leave without writing
        for (int it = 0; !mbar_try_wait(&bar, 0); it++) {
            if (it == kTileWaitLimit && leader) atomicCAS(&ctl->status, 0, 7);
            if (it >= 2 * kTileWaitLimit) return;
        }
        tv = TileView{tile, tile_pitch(blockDim.x), tile_rows(blockDim.y), three_d ? 3 : 1, three_d ? 1 : 0};
    }
    if (ix >= a.g.Nx || iy >= a.g.Ny) return;
    int I = (iz * a.g.Ny + iy) * a.g.Nx + ix;
    f3 B{0.f, 0.f, 0.f};
    if (bd) B = f3{__ldg(bd + I), __ldg(bd + N + I), __ldg(bd + 2 * N + I)};
    // engine/demag.go:95-97: NoDemagSpins cells feel no demag field
    if (!BAT && !UNI && a.nodemag && __ldg(a.nodemag + (UREG ? 0 : __ldg(a.regions + I))) != 0.0f) B = f3{0.f, 0.f, 0.f};
    f3 m0;
    if constexpr (TILE) m0 = tv.at(threadIdx.x, threadIdx.y, 0, 0, 0);
    else m0 = ld3(mx, my, mz, I);
    if (!is0(m0)) {
        f3 e;
        if constexpr (TILE) {
            e = dmi ? dmi_sum_tile<UNI>(tv, threadIdx.x, threadIdx.y, kc.pc, a.openbc != 0, a.g.Nz > 1, m0)
                    : exchange_sum_tile(tv, threadIdx.x, threadIdx.y, kc.pc, a.g.Nz > 1, m0);
        } else if (!BAT && !UNI && a.dbLUT) {  // engine/exchange.go:60-61 AddDMIBulk
            e = dmibulk_sum(mx, my, mz, a.aLUT, a.dbLUT, a.regions, a.cx, a.cy, a.cz, a.g, a.openbc != 0, ix, iy,
                            iz, m0, UREG ? 0 : __ldg(a.regions + I));
        } else if constexpr (UREG) {
            e = dmi ? dmi_sum_u(mx, my, mz, kc.pc, a.g, a.openbc != 0, ix, iy, iz, m0)
                    : exchange_sum_u(mx, my, mz, kc.pc, a.g, ix, iy, iz, m0);
        } else {
            int r0 = __ldg(a.regions + I);
            e = a.dmi ? dmi_sum_lut(mx, my, mz, a.dl, a.regions, a.g, a.openbc != 0, ix, iy, iz, m0, r0)
                      : exchange_sum(mx, my, mz, a.aLUT, a.regions, a.wx, a.wy, a.wz, a.g, ix, iy, iz, m0, r0);
        }
        float inv = (BAT || UNI || a.ms_uniform) ? kc.inv_ms : inv_msat(a.Ms, a.Ms_mul, I);
        B.x = fa(B.x, fm(e.x, inv));
        B.y = fa(B.y, fm(e.y, inv));
        B.z = fa(B.z, fm(e.z, inv));
    }
    if (a.anis) {
        if (BAT || UNI || a.anis_uniform) {  // uniaxialanisotropy2.cl:27-34 with the uniform factors hoisted
            f3 u{kc.u[0], kc.u[1], kc.u[2]};
            float mu = dot3(m0, u);
            float f1 = fm(kc.f1k, mu);
            float f2 = fm(kc.f2k, fm(fm(mu, mu), mu));
            B.x = fa(B.x, fa(fm(f1, u.x), fm(f2, u.x)));
            B.y = fa(B.y, fa(fm(f1, u.y), fm(f2, u.y)));
            B.z = fa(B.z, fa(fm(f1, u.z), fm(f2, u.z)));
        } else {
            add_uniaxial(B, a.up, m0, I);
        }
    }
    if (!BAT && !UNI && a.cubic) add_cubic(B, a.cp, m0, I);  // engine/anisotropy.go:158
    if (a.zeeman) {
        if constexpr (BAT) {
            B.x = fa(B.x, ip->bext[0]);
            B.y = fa(B.y, ip->bext[1]);
            B.z = fa(B.z, ip->bext[2]);
        } else {
            const int r = UREG ? 0 : __ldg(a.regions + I);
            B.x = fa(B.x, __ldg(a.bext[0] + r));
            B.y = fa(B.y, __ldg(a.bext[1] + r));
            B.z = fa(B.z, __ldg(a.bext[2] + r));
        }
    }
    if (!BAT && !UNI && a.thermal) {  // engine/effectivefield.go:20-22 B_therm (temperature2.cl)
        const float sc = therm_scale(ctl->k2, amul(a.alpha, a.alpha_mul, I), amul(a.temp, a.temp_mul, I),
                                     inv_msat(a.Ms, a.Ms_mul, I));
        const f3 n = therm_normals(a.seed, ctl->nsteps, I);
        B.x = fa(B.x, fm(n.x, sc));
        B.y = fa(B.y, fm(n.y, sc));
        B.z = fa(B.z, fm(n.z, sc));
    }
    if (!UNI && a.beff) { a.beff[I] = B.x; a.beff[N + I] = B.y; a.beff[2 * N + I] = B.z; }
    f3 t;
    if (!UNI && !a.precess) t = llnoprecess(m0, B);
    else if (BAT || UNI || a.alpha_uniform) t = lltorque_g(m0, B, alpha_mul, kc.gilb);
    else t = lltorque(m0, B, amul(a.alpha, a.alpha_mul, I));
    // engine/torque.go:348-352 FreezeSpins (zeromask.cl)
    if (!BAT && !UNI && a.frozen && __ldg(a.frozen + (UREG ? 0 : __ldg(a.regions + I))) != 0.0f) t = f3{0.f, 0.f, 0.f};
    float* out = a.tau_direct ? a.tau_direct : ctl->k[a.out_slot];
    out[I] = t.x; out[N + I] = t.y; out[2 * N + I] = t.z;
}

// ---------------------------------------------------------------- stages
constexpr int kMaxTerms = 7;
struct StageArgs {
    DevCtl* ctl;
    int N;
    int nterm;
    int src_m;             // first term: 0 = ctl->m, 1 = ctl->mw (coefficient 1)
    int slot[kMaxTerms];   // k slots of terms 1..nterm-1
    float c[kMaxTerms];    // float32 constants multiplying h (terms 1..)
    int scale_h;           // 1: fac = c*h ; 0: fac = c
    int normalize;
    int only_if_accepted;  // RK4 final solution
    const float* vol;
};

// m_w = normalize(src + sum_j (c_j h) k_j) with Madd<n> rounding
// (opencl/madd.go, madd<n>.cl) then normalize2.cl.  NT = number of terms.
template <int NT, bool BAT>
__global__ void __launch_bounds__(256) k_stage(StageArgs a) {
    DevCtl* ctl = a.ctl + (BAT ? blockIdx.y : 0);  // BAT: one grid row per instance
    if (!ctl->active) return;
    if (a.only_if_accepted && !ctl->accepted) return;
    const float h = ctl->h;
    float fac[NT];
    const float* src[NT];
    fac[0] = 1.0f;
    src[0] = a.src_m ? ctl->mw : ctl->m;
#pragma unroll
    for (int j = 1; j < NT; j++) {
        fac[j] = a.scale_h ? fm(a.c[j], h) : a.c[j];
        src[j] = ctl->k[a.slot[j]];
    }
    float* dst = ctl->mw;
    const int N = a.N;
    // one component of one cell from its NT source values (Madd<NT> order)
    auto comb = [&](const float (&x)[NT]) {
        if constexpr (NT == 3) {
            return fa(fm(fac[0], x[0]), fa(fm(fac[1], x[1]), fm(fac[2], x[2])));
        } else {
            float acc = fm(fac[0], x[0]);
#pragma unroll
            for (int j = 1; j < NT; j++) acc = fa(acc, fm(fac[j], x[j]));
            return acc;
        }
    };
    auto finish = [&](float (&v)[3], float w) {
        if (a.normalize) {
            f3 r = normalize_vol(f3{v[0], v[1], v[2]}, w);
            v[0] = r.x; v[1] = r.y; v[2] = r.z;
        }
    };
    // Four cells per iteration with 16-byte loads and stores where every
    // array allows it (N a multiple of 4, 16-byte aligned bases): four times
    // the bytes in flight per thread; each cell's arithmetic is unchanged.
    bool vec = (N & 3) == 0 && (reinterpret_cast<uintptr_t>(dst) & 15) == 0 &&
               (!a.vol || (reinterpret_cast<uintptr_t>(a.vol) & 15) == 0);
#pragma unroll
    for (int j = 0; j < NT; j++) vec = vec && (reinterpret_cast<uintptr_t>(src[j]) & 15) == 0;
    if (vec) {
        const int N4 = N >> 2;
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < N4; q += gridDim.x * blockDim.x) {
            float v[4][3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                float4 x4[NT];
#pragma unroll
                for (int j = 0; j < NT; j++) x4[j] = reinterpret_cast<const float4*>(src[j] + (size_t)c * N)[q];
#pragma unroll
                for (int l = 0; l < 4; l++) {
                    float x[NT];
#pragma unroll
                    for (int j = 0; j < NT; j++) x[j] = l == 0 ? x4[j].x : l == 1 ? x4[j].y : l == 2 ? x4[j].z : x4[j].w;
                    v[l][c] = comb(x);
                }
            }
            const float4 w4 = a.vol ? reinterpret_cast<const float4*>(a.vol)[q] : make_float4(1.f, 1.f, 1.f, 1.f);
            finish(v[0], w4.x);
            finish(v[1], w4.y);
            finish(v[2], w4.z);
            finish(v[3], w4.w);
#pragma unroll
            for (int c = 0; c < 3; c++)
                reinterpret_cast<float4*>(dst + (size_t)c * N)[q] = make_float4(v[0][c], v[1][c], v[2][c], v[3][c]);
        }
        return;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        float v[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            float x[NT];
#pragma unroll
            for (int j = 0; j < NT; j++) x[j] = src[j][c * N + i];
            v[c] = comb(x);
        }
        finish(v, a.vol ? a.vol[i] : 1.0f);
        dst[i] = v[0]; dst[N + i] = v[1]; dst[2 * N + i] = v[2];
    }
}

// ---------------------------------------------------------------- error norms
struct ErrArgs {
    DevCtl* ctl;
    int N;
    int nterm;
    int slot[kMaxTerms];
    float e[kMaxTerms];
    int dm_slot;     // slot whose max norm is the torque of the new state (delM / k4 / dy)
    int heun;        // 1: error = |k[slot0] - k[slot1]| (MaxVecDiff)
};

// Fused: error combination (Madd rounding), max |Err|^2, max |delM|^2 and
// max |Err|/|delM| (VecNorm + Div + MaxAbs of stepcontroller.go:51-63);
// Err itself is never written to memory.
template <int NT, bool HEUN, bool BAT>
__global__ void __launch_bounds__(256) k_err_norms(ErrArgs a) {
    __shared__ float sh[32];
    DevCtl* ctl = a.ctl + (BAT ? blockIdx.y : 0);  // BAT: one grid row per instance
    if (!ctl->active) return;
    const float* k[NT];
    float e[NT];
#pragma unroll
    for (int j = 0; j < NT; j++) {
        k[j] = ctl->k[a.slot[j]];
        e[j] = a.e[j];
    }
    const float* dm = ctl->k[a.dm_slot];
    const int N = a.N;
    float me = 0.f, md = 0.f, mr = 0.f;
    int nan = 0;
    // one component of the error estimate of one cell (Madd<NT> order)
    auto comb = [&](const float (&x)[NT]) {
        if constexpr (HEUN) {
            return fs(x[0], x[1]);
        } else if constexpr (NT == 3) {
            return fa(fm(e[0], x[0]), fa(fm(e[1], x[1]), fm(e[2], x[2])));
        } else {
            float acc = fm(e[0], x[0]);
#pragma unroll
            for (int j = 1; j < NT; j++) acc = fa(acc, fm(e[j], x[j]));
            return acc;
        }
    };
    auto cell = [&](f3 E, f3 D) {
        float e2 = dot3(E, E), d2 = dot3(D, D);
        float en = __fsqrt_rn(e2), dn = __fsqrt_rn(d2);
        float r = dn == 0.0f ? 0.0f : fd(en, dn);
        nan |= (e2 != e2) | (d2 != d2);
        me = fmaxf(me, e2);
        md = fmaxf(md, d2);
        mr = fmaxf(mr, r);
    };
    // four cells per iteration with 16-byte loads where every array allows
    // it (the maxima do not depend on the order cells are visited in)
    bool vec = (N & 3) == 0 && (reinterpret_cast<uintptr_t>(dm) & 15) == 0;
#pragma unroll
    for (int j = 0; j < NT; j++) vec = vec && (reinterpret_cast<uintptr_t>(k[j]) & 15) == 0;
    if (vec) {
        const int N4 = N >> 2;
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < N4; q += gridDim.x * blockDim.x) {
            float E[4][3], D[4][3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                float4 x4[NT];
#pragma unroll
                for (int j = 0; j < NT; j++) x4[j] = reinterpret_cast<const float4*>(k[j] + (size_t)c * N)[q];
                const float4 d4 = reinterpret_cast<const float4*>(dm + (size_t)c * N)[q];
                D[0][c] = d4.x; D[1][c] = d4.y; D[2][c] = d4.z; D[3][c] = d4.w;
#pragma unroll
                for (int l = 0; l < 4; l++) {
                    float x[NT];
#pragma unroll
                    for (int j = 0; j < NT; j++) x[j] = l == 0 ? x4[j].x : l == 1 ? x4[j].y : l == 2 ? x4[j].z : x4[j].w;
                    E[l][c] = comb(x);
                }
            }
#pragma unroll
            for (int l = 0; l < 4; l++) cell(f3{E[l][0], E[l][1], E[l][2]}, f3{D[l][0], D[l][1], D[l][2]});
        }
    } else {
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
            float Ec[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                float x[NT];
#pragma unroll
                for (int j = 0; j < NT; j++) x[j] = k[j][c * N + i];
                Ec[c] = comb(x);
            }
            cell(f3{Ec[0], Ec[1], Ec[2]}, f3{dm[i], dm[N + i], dm[2 * N + i]});
        }
    }
    me = block_max<256>(me, sh);
    md = block_max<256>(md, sh);
    mr = block_max<256>(mr, sh);
    nan = __syncthreads_or(nan);
    if (threadIdx.x == 0) {
        atomic_max_nonneg(&ctl->err2, me);
        atomic_max_nonneg(&ctl->dm2, md);
        atomic_max_nonneg(&ctl->rel, mr);
        if (nan) atomicOr(&ctl->nan_seen, 1);
    }
}

// ---------------------------------------------------------------- controller
__device__ void adapt_dt(DevCtl* c, double corr) {
    if (c->fix_dt != 0) { c->dt = c->fix_dt; return; }
    if (isnan(corr)) corr = 1;
    if (corr == 0) { c->status = 1; return; }
    corr *= c->headroom;
    if (corr > 2) corr = 2;
    if (corr < 1. / 2.) corr = 1. / 2.;
    c->dt *= corr;
    if (c->min_dt != 0 && c->dt < c->min_dt) c->dt = c->min_dt;
    if (c->max_dt != 0 && c->dt > c->max_dt) c->dt = c->max_dt;
    // the float32 step h = dt*GammaLL, times the largest tableau coefficient
    // (|-355/33| < 16), must stay finite: zero torque (err = 0) doubles dt
    // every step, and an infinite h turns the stages into Inf*0 = NaN
    if (c->dt * c->gamma > 0x1p120) c->dt = 0x1p120 / c->gamma;
    if (c->dt == 0) { c->status = 2; return; }
    if (c->t < c->alarm && c->t + c->dt > c->alarm) c->dt = c->alarm - c->t;
    if (!(c->dt > 0)) c->status = 3;
}

// engine/rk45dp.go:16-50 (start of Step): fixed dt, h, t0, clear maxima;
// skip the step once the run's stop time is reached (engine/run.go:212-231).
__global__ void k_step_begin(DevCtl* c0, int nb) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;  // one thread per instance
    if (b >= nb) return;
    DevCtl* c = c0 + b;
    c->active = (c->t < c->stop) && c->status == 0;
    if (!c->active) return;
    if (c->fix_dt != 0) c->dt = c->fix_dt;
    c->h = (float)(c->dt * c->gamma);
    if (c->therm_gv != 0) c->k2 = (float)(2 * kBoltzmann / (c->therm_gv * c->dt));
    c->t0 = c->t;
    c->err2 = 0u; c->dm2 = 0u; c->rel = 0u;
    c->accepted = 0;
}

// kind 0: integralController (engine/stepcontroller.go:35-97), FSAL when fsal
// kind 1: simpleController (:13-32, RK4); kind 2: Heun (engine/heun.go:40-58)
// kind 3: Euler (engine/euler.go:16-35), always accepted
__global__ void k_controller(DevCtl* c0, int nb, int kind, int acc, int rej, int fsal_from, int fsal_to,
                             int nevals) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;  // one thread per instance
    if (b >= nb) return;
    DevCtl* c = c0 + b;
    if (!c->active) return;
    c->nevals += nevals;
    if (c->nan_seen) c->status = 4;
    if (kind == 3) {
        // setMaxTorque(dy0), then dt = FixDt, or float32(MaxErr / LastTorque)
        // treated as the largest allowed change of m; h is the float32 dt*GammaLL
        const double lt = sqrt((double)__uint_as_float(c->dm2));
        c->last_torque = lt;
        float hf;
        if (c->fix_dt != 0) {
            c->dt = c->fix_dt;
            hf = (float)(c->dt * c->gamma);
        } else {
            hf = (float)(c->max_err / lt);
            c->dt = (double)hf / c->gamma;
        }
        if (!(hf > 0.0f)) {  // euler.go:32 "Euler solver requires fixed time step > 0"
            c->status = 5;
            c->accepted = 0;
            return;
        }
        c->h = hf;
        const double err = (double)hf * lt;
        c->last_err = err;
        if (err > c->peak_err) c->peak_err = err;
        c->t = c->t0 + c->dt;
        c->nsteps++;
        c->accepted = 1;
        return;
    }
    double h = (double)c->h;
    double err = sqrt((double)__uint_as_float(c->err2)) * h;
    double maxdm = sqrt((double)__uint_as_float(c->dm2));
    bool ok = err < c->max_err || c->dt <= c->min_dt || c->fix_dt != 0;
    if (kind == 0) {
        if (ok) {
            int fail = 0;
            double rlerr = 0.0;
            if (!(maxdm < c->min_slope)) {
                rlerr = (double)__uint_as_float(c->rel);
                fail = 1;
            }
            if (fail == 0 || c->rel_err <= 0.0 || rlerr < c->rel_err || c->dt <= c->min_dt || c->fix_dt != 0) {
                c->last_err = err;
                if (err > c->peak_err) c->peak_err = err;
                c->last_torque = maxdm;
                c->nsteps++;
                c->t = c->t0 + c->dt;
                adapt_dt(c, fail == 0 ? pow(c->max_err / err, 1. / acc) : pow(c->rel_err / rlerr, 1. / acc));
                c->accepted = 1;
            } else {
                c->t = c->t0;
                c->nundone++;
                adapt_dt(c, pow(c->rel_err / rlerr, 1. / rej));
            }
        } else {
            c->t = c->t0;
            c->nundone++;
            adapt_dt(c, pow(c->max_err / err, 1. / rej));
        }
    } else if (kind == 1) {  // RK4: Time = t0 + dt was set before stage 4 (rk4.go:51)
        c->t = c->t0 + c->dt;
        if (ok) {
            c->nsteps++;
            adapt_dt(c, pow(c->max_err / err, 1. / acc));
            c->last_err = err;
            if (err > c->peak_err) c->peak_err = err;
            c->accepted = 1;
        } else {
            c->nundone++;
            adapt_dt(c, pow(c->max_err / err, 1. / rej));
            c->t = c->t0;
        }
    } else {  // Heun: time was advanced before the second evaluation
        if (ok) {
            c->t = c->t0 + c->dt;
            c->nsteps++;
            adapt_dt(c, pow(c->max_err / err, 1. / 2.));
            c->last_err = err;
            if (err > c->peak_err) c->peak_err = err;
            c->last_torque = maxdm;
            c->accepted = 1;
        } else {
            c->t = c->t0;
            c->nundone++;
            adapt_dt(c, pow(c->max_err / err, 1. / 3.));
        }
    }
    if (c->accepted && kind == 0 && fsal_from >= 0) {
        float* t = c->k[fsal_to];
        c->k[fsal_to] = c->k[fsal_from];
        c->k[fsal_from] = t;
    }
}

// accepted: the working magnetisation becomes the state (pointer swap);
// RK4 also records max |k4| here (setMaxTorque, engine/rk4.go:64)
__global__ void k_step_end(DevCtl* c0, int nb, int rk4) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;  // one thread per instance
    if (b >= nb) return;
    DevCtl* c = c0 + b;
    if (!c->active) return;
    if (c->accepted) {
        float* t = c->m;
        c->m = c->mw;
        c->mw = t;
        if (rk4) c->last_torque = sqrt((double)__uint_as_float(c->dm2));
    }
}

// ---------------------------------------------------------------- energies
// Per-term sums of dot(M_full, B_term) over the cells (engine/energy.go:51-69
// makeEdensAdder / dot, engine/anisotropy.go:164-216): M_full = Ms * m (* vol),
// the dot products in float32 as opencl.AddDotProduct/Dot form them, the sums
// accumulated in FP64 (compensated relative to the reference's float32
// reduction).  sums: [0] demag, [1] exchange (+DMI), [2] anisotropy from K1
// alone, [3] anisotropy from K2 alone, [4] Zeeman.
// the float32 dot products of cell I: [0] demag, [1] exchange (+DMI),
// [2] uniaxial anisotropy from K1 alone, [3] from K2 alone, [4] Zeeman,
// [5..7] cubic anisotropy from Kc1, Kc2, Kc3 alone, [8] thermal field
constexpr int kNE = 9;
__device__ __forceinline__ void energy_cell_terms(const LocalArgs& a, const float* __restrict__ vol, int I,
                                                  float t[kNE]) {
    const int N = a.N;
    const float* m = a.ctl->m;
    const float *mx = m, *my = m + N, *mz = m + 2 * N;
    const int ix = I % a.g.Nx, iy = (I / a.g.Nx) % a.g.Ny, iz = I / (a.g.Nx * a.g.Ny);
    const f3 m0 = ld3(mx, my, mz, I);
    const float ms = amul(a.Ms, a.Ms_mul, I);
    f3 Mf{fm(m0.x, ms), fm(m0.y, ms), fm(m0.z, ms)};
    if (vol) {
        const float w = __ldg(vol + I);
        Mf = f3{fm(Mf.x, w), fm(Mf.y, w), fm(Mf.z, w)};
    }
    for (int k = 0; k < kNE; k++) t[k] = 0.f;
    if (a.bd && !(a.nodemag && __ldg(a.nodemag + __ldg(a.regions + I)) != 0.0f))
        t[0] = dot3(Mf, f3{__ldg(a.bd + I), __ldg(a.bd + N + I), __ldg(a.bd + 2 * N + I)});
    if (!is0(m0)) {
        const int r0 = __ldg(a.regions + I);
        const f3 e = a.dbLUT ? dmibulk_sum(mx, my, mz, a.aLUT, a.dbLUT, a.regions, a.cx, a.cy, a.cz, a.g,
                                           a.openbc != 0, ix, iy, iz, m0, r0)
                   : a.dmi ? dmi_sum_lut(mx, my, mz, a.dl, a.regions, a.g, a.openbc != 0, ix, iy, iz, m0, r0)
                           : exchange_sum(mx, my, mz, a.aLUT, a.regions, a.wx, a.wy, a.wz, a.g, ix, iy, iz, m0, r0);
        const float inv = inv_msat(a.Ms, a.Ms_mul, I);
        t[1] = dot3(Mf, f3{fm(e.x, inv), fm(e.y, inv), fm(e.z, inv)});
    }
    if (a.anis) {
        UniaxParams p1 = a.up, p2 = a.up;
        p1.K2 = nullptr; p1.K2_mul = 0.f;
        p2.K1 = nullptr; p2.K1_mul = 0.f;
        f3 B1{0.f, 0.f, 0.f}, B2{0.f, 0.f, 0.f};
        add_uniaxial(B1, p1, m0, I);
        add_uniaxial(B2, p2, m0, I);
        t[2] = dot3(Mf, B1);
        t[3] = dot3(Mf, B2);
    }
    if (a.zeeman) {
        const int r = __ldg(a.regions + I);
        t[4] = dot3(Mf, f3{__ldg(a.bext[0] + r), __ldg(a.bext[1] + r), __ldg(a.bext[2] + r)});
    }
    if (a.thermal) {  // engine/temperature.go:21 Edens_therm: the field of the current step
        const float sc = therm_scale(a.ctl->k2, amul(a.alpha, a.alpha_mul, I), amul(a.temp, a.temp_mul, I),
                                     inv_msat(a.Ms, a.Ms_mul, I));
        const f3 n = therm_normals(a.seed, a.ctl->nsteps, I);
        t[8] = dot3(Mf, f3{fm(n.x, sc), fm(n.y, sc), fm(n.z, sc)});
    }
    if (a.cubic) {  // engine/anisotropy.go:191-206: each constant alone
        for (int k = 0; k < 3; k++) {
            CubicParams q = a.cp;
            if (k != 0) { q.K1 = nullptr; q.K1_mul = 0.f; }
            if (k != 1) { q.K2 = nullptr; q.K2_mul = 0.f; }
            if (k != 2) { q.K3 = nullptr; q.K3_mul = 0.f; }
            f3 Bc{0.f, 0.f, 0.f};
            add_cubic(Bc, q, m0, I);
            t[5 + k] = dot3(Mf, Bc);
        }
    }
}

__global__ void __launch_bounds__(256) k_energy_terms(LocalArgs a, const float* __restrict__ vol, double* sums) {
    __shared__ double sh[kNE][8];
    double acc[kNE] = {};
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < a.N; I += gridDim.x * blockDim.x) {
        float t[kNE];
        energy_cell_terms(a, vol, I, t);
        for (int k = 0; k < kNE; k++) acc[k] += (double)t[k];
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int t = 0; t < kNE; t++) {
        double v = acc[t];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[t][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < kNE) {
        double v = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += sh[threadIdx.x][w];
        atomicAdd(sums + threadIdx.x, v);
    }
}

// engine/demag.go:74-83: the demag convolution's volume with NoDemagSpins --
// a copy of the geometry (ones without one) zeroed where the region's value
// is non-zero (zeromask.cl), so those cells make no field
__global__ void k_nodemag_vol(const float* __restrict__ vol, const float* __restrict__ lut,
                              const uint8_t* __restrict__ regions, float* __restrict__ out, int N) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
        out[i] = __ldg(lut + __ldg(regions + i)) != 0.0f ? 0.0f : (vol ? __ldg(vol + i) : 1.0f);
}

// ---------------------------------------------------------------- host side
struct SimImpl {
    umag_sim_params p;
    umag_solver_params sp;
    int N;
    Mesh3 g;
    umag_demag* demag = nullptr;
    float* bufs = nullptr;        // 2 + 7 slots of 3N
    float* bd = nullptr;          // demag field 3N
    uint8_t* zero_regions = nullptr;
    float* dmi_pairs = nullptr;   // 7 x 32896 region-pair DMI coefficients
    float* demag_vol = nullptr;   // NoDemagSpins: geometry with the masked regions zeroed
    LocalConsts* kc_dev = nullptr;
    DevCtl* ctl = nullptr;        // device
    DevCtl* hctl = nullptr;       // pinned host mirror
    PassArgs pa{};
    LocalArgs la{};
    bool need_k1 = true;
    bool use_graph = true;
    int graph_steps = 16;
    cudaGraphExec_t gexec = nullptr;   // graph_steps steps
    cudaGraphExec_t gexec1 = nullptr;  // one step
    int launches_per_step = 0;
    double* esum = nullptr;            // energy term sums (kNE doubles)
    umag_tuning tune{{32, 8}, 256, 8, 4, 1};  // launch shapes (umag_sim_set_tuning)
    TileMaps tmaps{};                          // TMA maps of the two magnetisation buffers
    bool tile_ok = false;                      // the mesh and block shape allow tiles
    // batched ensemble class: nb same-size instances with uniform parameters
    int nb = 1;
    bool batched = false;
    InstParams* ip_dev = nullptr;
};

// stream the step/field launches go to: the library stream, or the stream of
// the ensemble class being captured
static thread_local cudaStream_t g_launch_stream = nullptr;
static cudaStream_t S() { return g_launch_stream ? g_launch_stream : ctx().stream; }
static unsigned ctl_grid(const SimImpl* s) { return (unsigned)((s->nb + 127) / 128); }

// one torque evaluation of ctl->(m | mw) into ctl->k[slot] (or a direct buffer)
static int launch_torque(SimImpl* s, int m_sel, int slot, float* tau_direct, float* beff, int* nl) {
    if (s->p.enable_demag) {
        PassArgs a = s->pa;
        a.m_sel = m_sel;
        if (s->batched) UMAG_TRY(demag_launch_batch(s->demag, a, s->nb, S()));
        else UMAG_TRY(demag_launch(s->demag, a, S()));
        if (nl) *nl += 3;
    }
    LocalArgs la = s->la;
    la.m_sel = m_sel;
    la.out_slot = slot;
    la.tau_direct = tau_direct;
    la.beff = beff;
    const int bx = s->tune.torque_block[0], by = s->tune.torque_block[1];
    dim3 blk(bx, by, 1), grd((s->g.Nx + bx - 1) / bx, (s->g.Ny + by - 1) / by, s->g.Nz * s->nb);
    // the uniform-material instantiation where every term it leaves out is off
    const bool uni = s->zero_regions && !la.nodemag && !la.dbLUT && !la.cubic && !la.thermal && !beff &&
                     !la.frozen && la.precess && la.alpha_uniform && la.ms_uniform && (!la.anis || la.anis_uniform) &&
                     !la.openbc;
    if (s->batched)
        k_local_torque<true, true, false><<<grd, blk, 0, S()>>>(la, s->tmaps);
    else if (s->zero_regions && s->tile_ok && s->tune.torque_tma && uni)
        k_local_torque<true, false, true, true><<<grd, blk, tile_bytes(bx, by, s->g.Nz) + 128, S()>>>(la, s->tmaps);
    else if (s->zero_regions && s->tile_ok && s->tune.torque_tma)
        k_local_torque<true, false, true><<<grd, blk, tile_bytes(bx, by, s->g.Nz) + 128, S()>>>(la, s->tmaps);
    else if (s->zero_regions)
        k_local_torque<true, false, false><<<grd, blk, 0, S()>>>(la, s->tmaps);
    else
        k_local_torque<false, false, false><<<grd, blk, 0, S()>>>(la, s->tmaps);
    UMAG_LAUNCH_CHECK();
    if (nl) *nl += 1;
    return UMAG_OK;
}

static int launch_stage(SimImpl* s, int src_m, std::initializer_list<int> slots, std::initializer_list<double> cs,
                        bool scale_h, bool normalize, bool only_if_accepted, int* nl) {
    StageArgs a{};
    a.ctl = s->ctl;
    a.N = s->N;
    a.src_m = src_m;
    a.nterm = 1 + (int)slots.size();
    int j = 1;
    for (int sl : slots) a.slot[j++] = sl;
    j = 1;
    for (double c : cs) a.c[j++] = (float)c;  // Go: untyped constant converted to float32
    a.scale_h = scale_h;
    a.normalize = normalize;
    a.only_if_accepted = only_if_accepted;
    a.vol = s->p.vol;
    const int th = s->tune.stage_threads;
    const dim3 g(s->batched ? (unsigned)((s->N + th - 1) / th) : (unsigned)grid_for(s->N, th, s->tune.stage_waves),
                 s->nb);
#define STAGE(n)                                                    \
    case n:                                                         \
        if (s->batched) k_stage<n, true><<<g, th, 0, S()>>>(a);     \
        else k_stage<n, false><<<g, th, 0, S()>>>(a);               \
        break;
    switch (a.nterm) {
        STAGE(2) STAGE(3) STAGE(4) STAGE(5) STAGE(6)
    default: return set_error(UMAG_E_ARG, "stage with %d terms", a.nterm);
    }
#undef STAGE
    UMAG_LAUNCH_CHECK();
    *nl += 1;
    return UMAG_OK;
}

static int launch_err(SimImpl* s, std::initializer_list<int> slots, std::initializer_list<double> es, int dm_slot,
                      bool heun, int* nl) {
    ErrArgs a{};
    a.ctl = s->ctl;
    a.N = s->N;
    a.nterm = (int)slots.size();
    int j = 0;
    for (int sl : slots) a.slot[j++] = sl;
    j = 0;
    for (double e : es) a.e[j++] = (float)e;
    a.dm_slot = dm_slot;
    a.heun = heun;
    const dim3 g(s->batched ? (unsigned)((s->N + 255) / 256) : (unsigned)grid_for(s->N, 256, s->tune.err_waves),
                 s->nb);
#define ERRN(n, hn)                                                       \
    do {                                                                  \
        if (s->batched) k_err_norms<n, hn, true><<<g, 256, 0, S()>>>(a);  \
        else k_err_norms<n, hn, false><<<g, 256, 0, S()>>>(a);            \
    } while (0)
    if (heun) ERRN(2, true);
    else if (a.nterm == 2) ERRN(2, false);
    else if (a.nterm == 4) ERRN(4, false);
    else if (a.nterm == 6) ERRN(6, false);
    else return set_error(UMAG_E_ARG, "error combination with %d terms", a.nterm);
#undef ERRN
    UMAG_LAUNCH_CHECK();
    *nl += 1;
    return UMAG_OK;
}

// Slots: k[0] = k1 (FSAL), k[1..6] = k2..k7 buffers.
static int launch_step(SimImpl* s, int* nl) {
    DevCtl* c = s->ctl;
    k_step_begin<<<ctl_grid(s), 128, 0, S()>>>(c, s->nb);
    UMAG_LAUNCH_CHECK();
    *nl += 1;
    switch (s->sp.solver) {
    case 5: {  // engine/rk45dp.go:52-97
        UMAG_TRY(launch_stage(s, 0, {0}, {1. / 5.}, true, true, false, nl));
        UMAG_TRY(launch_torque(s, 1, 1, nullptr, nullptr, nl));
        UMAG_TRY(launch_stage(s, 0, {0, 1}, {3. / 40., 9. / 40.}, true, true, false, nl));
        UMAG_TRY(launch_torque(s, 1, 2, nullptr, nullptr, nl));
        UMAG_TRY(launch_stage(s, 0, {0, 1, 2}, {44. / 45., -56. / 15., 32. / 9.}, true, true, false, nl));
        UMAG_TRY(launch_torque(s, 1, 3, nullptr, nullptr, nl));
        UMAG_TRY(launch_stage(s, 0, {0, 1, 2, 3}, {19372. / 6561., -25360. / 2187., 64448. / 6561., -212. / 729.},
                              true, true, false, nl));
        UMAG_TRY(launch_torque(s, 1, 4, nullptr, nullptr, nl));
        UMAG_TRY(launch_stage(s, 0, {0, 1, 2, 3, 4},
                              {9017. / 3168., -355. / 33., 46732. / 5247., 49. / 176., -5103. / 18656.}, true, true,
                              false, nl));
        UMAG_TRY(launch_torque(s, 1, 5, nullptr, nullptr, nl));
        UMAG_TRY(launch_stage(s, 0, {0, 2, 3, 4, 5},
                              {35. / 384., 500. / 1113., 125. / 192., -2187. / 6784., 11. / 84.}, true, true, false,
                              nl));
        UMAG_TRY(launch_torque(s, 1, 6, nullptr, nullptr, nl));
        // rk45dp.go:95 weight differences, as exact rationals rounded to float32
        UMAG_TRY(launch_err(s, {0, 2, 3, 4, 5, 6},
                            {71. / 57600., -71. / 16695., 71. / 1920., -17253. / 339200., 22. / 525., -1. / 40.}, 6,
                            false, nl));
        k_controller<<<ctl_grid(s), 128, 0, S()>>>(c, s->nb, 0, 5, 6, 6, 0, 6);
        break;
    }
    case 3: {  // engine/rk23.go:58-83
        UMAG_TRY(launch_stage(s, 0, {0}, {1. / 2.}, true, true, false, nl));
        UMAG_TRY(launch_torque(s, 1, 1, nullptr, nullptr, nl));
        UMAG_TRY(launch_stage(s, 0, {1}, {3. / 4.}, true, true, false, nl));
        UMAG_TRY(launch_torque(s, 1, 2, nullptr, nullptr, nl));
        UMAG_TRY(launch_stage(s, 0, {0, 1, 2}, {2. / 9., 1. / 3., 4. / 9.}, true, true, false, nl));
        UMAG_TRY(launch_torque(s, 1, 3, nullptr, nullptr, nl));
        UMAG_TRY(launch_err(s, {0, 1, 2, 3}, {5. / 72., -1. / 12., -1. / 9., 1. / 8.}, 3, false, nl));
        k_controller<<<ctl_grid(s), 128, 0, S()>>>(c, s->nb, 0, 3, 4, 3, 0, 3);
        break;
    }
    case 2: {  // engine/heun.go:15-59
        UMAG_TRY(launch_torque(s, 0, 0, nullptr, nullptr, nl));                      // dy0
        UMAG_TRY(launch_stage(s, 0, {0}, {1.0}, true, false, false, nl));            // y = y + dt*dy0
        UMAG_TRY(launch_torque(s, 1, 1, nullptr, nullptr, nl));                      // dy
        UMAG_TRY(launch_err(s, {0, 1}, {1.0, -1.0}, 1, true, nl));                   // |dy0 - dy|
        k_controller<<<ctl_grid(s), 128, 0, S()>>>(c, s->nb, 2, 2, 3, -1, -1, 2);
        UMAG_LAUNCH_CHECK();
        *nl += 1;
        // accepted: y = y + 0.5 dt dy - 0.5 dt dy0, normalised (heun.go:45-46)
        UMAG_TRY(launch_stage(s, 1, {1, 0}, {0.5, -0.5}, true, true, true, nl));
        k_step_end<<<ctl_grid(s), 128, 0, S()>>>(c, s->nb, 0);
        UMAG_LAUNCH_CHECK();
        *nl += 1;
        return UMAG_OK;
    }
    case 1: {  // engine/euler.go:11-36
        UMAG_TRY(launch_torque(s, 0, 0, nullptr, nullptr, nl));           // dy0
        UMAG_TRY(launch_err(s, {0, 0}, {1.0, -1.0}, 0, true, nl));        // max |dy0|
        k_controller<<<ctl_grid(s), 128, 0, S()>>>(c, s->nb, 3, 1, 1, -1, -1, 1);
        UMAG_LAUNCH_CHECK();
        *nl += 1;
        // y = y + dt*dy0 (Madd2), normalised (euler.go:33-34)
        UMAG_TRY(launch_stage(s, 0, {0}, {1.0}, true, true, true, nl));
        k_step_end<<<ctl_grid(s), 128, 0, S()>>>(c, s->nb, 0);
        UMAG_LAUNCH_CHECK();
        *nl += 1;
        return UMAG_OK;
    }
    case 4: {  // engine/rk4.go:11-69
        UMAG_TRY(launch_torque(s, 0, 0, nullptr, nullptr, nl));
        UMAG_TRY(launch_stage(s, 0, {0}, {1. / 2.}, true, true, false, nl));
        UMAG_TRY(launch_torque(s, 1, 1, nullptr, nullptr, nl));
        UMAG_TRY(launch_stage(s, 0, {1}, {1. / 2.}, true, true, false, nl));
        UMAG_TRY(launch_torque(s, 1, 2, nullptr, nullptr, nl));
        UMAG_TRY(launch_stage(s, 0, {2}, {1.}, true, true, false, nl));
        UMAG_TRY(launch_torque(s, 1, 3, nullptr, nullptr, nl));
        UMAG_TRY(launch_err(s, {0, 3}, {1., -1.}, 3, false, nl));
        k_controller<<<ctl_grid(s), 128, 0, S()>>>(c, s->nb, 1, 4, 5, -1, -1, 4);
        UMAG_LAUNCH_CHECK();
        *nl += 1;
        UMAG_TRY(launch_stage(s, 0, {0, 1, 2, 3}, {1. / 6., 1. / 3., 1. / 3., 1. / 6.}, true, true, true, nl));
        k_step_end<<<ctl_grid(s), 128, 0, S()>>>(c, s->nb, 1);
        UMAG_LAUNCH_CHECK();
        *nl += 1;
        return UMAG_OK;
    }
    default:
        return set_error(UMAG_E_ARG, "unknown solver %d", s->sp.solver);
    }
    UMAG_LAUNCH_CHECK();
    *nl += 1;
    k_step_end<<<ctl_grid(s), 128, 0, S()>>>(c, s->nb, 0);
    UMAG_LAUNCH_CHECK();
    *nl += 1;
    return UMAG_OK;
}

static int sync_ctl_to_host(SimImpl* s) {
    UMAG_CUDA(cudaMemcpyAsync(s->hctl, s->ctl, sizeof(DevCtl) * s->nb, cudaMemcpyDeviceToHost, S()));
    UMAG_CUDA(cudaStreamSynchronize(S()));
    return UMAG_OK;
}
static int push_ctl(SimImpl* s) {
    UMAG_CUDA(cudaMemcpyAsync(s->ctl, s->hctl, sizeof(DevCtl) * s->nb, cudaMemcpyHostToDevice, S()));
    UMAG_CUDA(cudaStreamSynchronize(S()));
    return UMAG_OK;
}

// FSAL k1 of the current state, before the first step of a run
// (engine/rk45dp.go:26-29; RunWhile frees the stepper, engine/run.go:207)
static int ensure_k1(SimImpl* s) {
    if (!s->need_k1) return UMAG_OK;
    if (s->sp.solver == 5 || s->sp.solver == 3) {
        UMAG_TRY(sync_ctl_to_host(s));
        for (int b = 0; b < s->nb; b++) s->hctl[b].active = 1;
        UMAG_TRY(push_ctl(s));
        UMAG_TRY(launch_torque(s, 0, 0, nullptr, nullptr, nullptr));
        UMAG_TRY(sync_ctl_to_host(s));
        for (int b = 0; b < s->nb; b++) s->hctl[b].nevals += 1;
        UMAG_TRY(push_ctl(s));
    }
    s->need_k1 = false;
    return UMAG_OK;
}

static void drop_graph(SimImpl* s) {
    if (s->gexec) cudaGraphExecDestroy(s->gexec);
    if (s->gexec1) cudaGraphExecDestroy(s->gexec1);
    s->gexec = nullptr;
    s->gexec1 = nullptr;
}

// capture `steps` steps into *out
static int capture_steps(SimImpl* s, int steps, cudaGraphExec_t* out) {
    cudaGraph_t graph;
    UMAG_CUDA(cudaStreamBeginCapture(S(), cudaStreamCaptureModeThreadLocal));
    int nl = 0;
    int st = UMAG_OK;
    for (int i = 0; i < steps && st == UMAG_OK; i++) st = launch_step(s, &nl);
    cudaError_t e = cudaStreamEndCapture(S(), &graph);
    if (st != UMAG_OK) return st;
    if (e != cudaSuccess) return set_error(UMAG_E_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(out, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return set_error(UMAG_E_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    return UMAG_OK;
}

// n steps with the stop time already in ctl: graphs of graph_steps steps,
// the remainder from a one-step graph
static int run_steps(SimImpl* s, long long n) {
    UMAG_TRY(ensure_k1(s));
    if (s->use_graph) {
        if (n >= s->graph_steps) {
            if (!s->gexec) UMAG_TRY(capture_steps(s, s->graph_steps, &s->gexec));
            for (; n >= s->graph_steps; n -= s->graph_steps) UMAG_CUDA(cudaGraphLaunch(s->gexec, S()));
        }
        if (n > 0) {
            if (!s->gexec1) UMAG_TRY(capture_steps(s, 1, &s->gexec1));
            for (; n > 0; n--) UMAG_CUDA(cudaGraphLaunch(s->gexec1, S()));
        }
        return UMAG_OK;
    }
    for (long long i = 0; i < n; i++) {
        int nl = 0;
        UMAG_TRY(launch_step(s, &nl));
    }
    return UMAG_OK;
}

// Tensor maps for the magnetisation tiles of the torque kernel (tile.cuh),
// when the mesh allows them: region-free, non-periodic, not batched, no bulk
// DMI, Nx a multiple of 4 (row strides and buffer offsets in 16-byte units),
// and a box of at most 256 elements per dimension.
static void tile_setup(SimImpl* s) {
    s->tile_ok = false;
    const int bx = s->tune.torque_block[0], by = s->tune.torque_block[1];
    if (s->batched || !s->zero_regions || s->g.pbc != 0 || s->la.dbLUT || s->g.Nx % 4 != 0) return;
    if (tile_pitch(bx) > 256 || tile_rows(by) > 256) return;
    EncodeTiledFn fn = encode_tiled();
    if (!fn) return;
    const cuuint64_t dims[4] = {(cuuint64_t)s->g.Nx, (cuuint64_t)s->g.Ny, (cuuint64_t)s->g.Nz, 3};
    const cuuint64_t strides[3] = {sizeof(float) * (cuuint64_t)s->g.Nx,
                                   sizeof(float) * (cuuint64_t)s->g.Nx * s->g.Ny, sizeof(float) * (cuuint64_t)s->N};
    const cuuint32_t box[4] = {(cuuint32_t)tile_pitch(bx), (cuuint32_t)tile_rows(by),
                               (cuuint32_t)(s->g.Nz > 1 ? 3 : 1), 3};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    for (int b = 0; b < 2; b++) {
        float* base = s->bufs + (size_t)b * 3 * s->N;
        if (reinterpret_cast<uintptr_t>(base) % 16 != 0) return;
        if (fn(&s->tmaps.map[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return;
    }
    s->tile_ok = true;
}

// The local-term arguments that follow from the material parameters in s->p
// (and the uniform factors evaluated from them); run at creation and again
// whenever a parameter is reassigned.
static int local_from_params(SimImpl* s) {
    const umag_sim_params* p = &s->p;
    LocalArgs& la = s->la;
    la.aLUT = p->aLUT;
    la.dLUT = p->dLUT;
    la.regions = s->p.regions;
    la.wx = (float)(2 / (p->cell[0] * p->cell[0]));
    la.wy = (float)(2 / (p->cell[1] * p->cell[1]));
    la.wz = (float)(2 / (p->cell[2] * p->cell[2]));
    la.cx = (float)p->cell[0]; la.cy = (float)p->cell[1]; la.cz = (float)p->cell[2];
    la.dmi = p->dLUT != nullptr;
    la.openbc = p->openbc;
    la.anis = (p->Ku1 != nullptr || p->Ku1_mul != 0.f || p->Ku2 != nullptr || p->Ku2_mul != 0.f);
    la.up = UniaxParams{p->Ms, p->Ku1, p->Ku2, p->anisU[0], p->anisU[1], p->anisU[2],
                        p->Ms_mul, p->Ku1_mul, p->Ku2_mul, p->anisU_mul[0], p->anisU_mul[1], p->anisU_mul[2]};
    la.zeeman = p->bextLUT[0] != nullptr;
    for (int i = 0; i < 3; i++) la.bext[i] = p->bextLUT[i];
    la.alpha = p->alpha;
    la.alpha_mul = p->alpha_mul;
    la.precess = p->precess;
    la.frozen = p->frozen_lut;
    la.nodemag = p->enable_demag ? p->nodemag_lut : nullptr;
    la.cubic = (p->Kc1 != nullptr || p->Kc1_mul != 0.f || p->Kc2 != nullptr || p->Kc2_mul != 0.f ||
                p->Kc3 != nullptr || p->Kc3_mul != 0.f);
    la.cp = CubicParams{p->Ms, p->Kc1, p->Kc2, p->Kc3, {p->anisC1[0], p->anisC1[1], p->anisC1[2]},
                        {p->anisC2[0], p->anisC2[1], p->anisC2[2]}, p->Ms_mul, p->Kc1_mul, p->Kc2_mul, p->Kc3_mul,
                        {p->anisC1_mul[0], p->anisC1_mul[1], p->anisC1_mul[2]},
                        {p->anisC2_mul[0], p->anisC2_mul[1], p->anisC2_mul[2]}};
    la.dbLUT = p->dbulkLUT;
    la.thermal = (p->temp != nullptr || p->temp_mul != 0.f);
    la.temp = p->temp;
    la.temp_mul = p->temp_mul;
    la.seed = p->therm_seed;
    la.Ms = p->Ms;
    la.Ms_mul = p->Ms_mul;
    la.ms_uniform = p->Ms == nullptr;
    la.alpha_uniform = p->alpha == nullptr;
    la.anis_uniform = p->Ms == nullptr && p->Ku1 == nullptr && p->Ku2 == nullptr && p->anisU[0] == nullptr &&
                      p->anisU[1] == nullptr && p->anisU[2] == nullptr;
    {  // uniform factors, evaluated on the device (bit-identical to the per-cell path)
        if (!s->kc_dev && cudaMalloc(&s->kc_dev, sizeof(LocalConsts)) != cudaSuccess)
            return set_error(UMAG_E_NOMEM, "consts");
        k_local_consts<<<1, 1, 0, S()>>>(la, s->kc_dev);
        if (cudaMemcpyAsync(&la.kc, s->kc_dev, sizeof(LocalConsts), cudaMemcpyDeviceToHost, S()) != cudaSuccess ||
            cudaStreamSynchronize(S()) != cudaSuccess)
            return set_error(UMAG_E_CUDA, "uniform constants");
    }
    if (s->demag) {
        s->pa.Ms = p->Ms;
        s->pa.Ms_mul = p->Ms_mul;
    }
    return UMAG_OK;
}

int sim_new(const umag_sim_params* p, const umag_solver_params* sp, umag_sim** out) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(p && sp && out, "NULL argument");
    UMAG_REQUIRE(p->N[0] > 0 && p->N[1] > 0 && p->N[2] > 0, "bad mesh size");
    UMAG_REQUIRE(p->aLUT != nullptr, "aLUT (exchange LUT) is required");
    UMAG_REQUIRE(sp->solver >= 1 && sp->solver <= 5,
                 "solver must be 1 (Euler), 2 (Heun), 3 (RK23), 4 (RK4) or 5 (RK45DP)");
    UMAG_REQUIRE(p->pbc[0] >= 0 && p->pbc[1] >= 0 && p->pbc[2] >= 0, "PBC repetitions must be non-negative");
    // engine/exchange.go:62-63
    UMAG_REQUIRE(!(p->dLUT && p->dbulkLUT), "Cannot have induced and interfacial DMI at the same time");
    SimImpl* s = new SimImpl();
    s->p = *p;
    s->sp = *sp;
    s->N = p->N[0] * p->N[1] * p->N[2];
    // data/mesh.go PBC_code: the stencils wrap along periodic axes
    s->g = Mesh3{p->N[0], p->N[1], p->N[2], (p->pbc[0] ? 1 : 0) | (p->pbc[1] ? 2 : 0) | (p->pbc[2] ? 4 : 0)};
    int st = UMAG_OK;
    size_t b3 = sizeof(float) * 3 * (size_t)s->N;
    auto fail = [&](int code) { sim_free(reinterpret_cast<umag_sim*>(s)); return code; };
    if (cudaMalloc(&s->bufs, b3 * 9) != cudaSuccess) return fail(set_error(UMAG_E_NOMEM, "state buffers"));
    if (cudaMemsetAsync(s->bufs, 0, b3 * 9, S()) != cudaSuccess) return fail(set_error(UMAG_E_CUDA, "state buffers"));
    if (!p->regions) {
        if (cudaMalloc(&s->zero_regions, s->N) != cudaSuccess) return fail(set_error(UMAG_E_NOMEM, "regions"));
        if (cudaMemsetAsync(s->zero_regions, 0, s->N, S()) != cudaSuccess) return fail(set_error(UMAG_E_CUDA, "regions"));
        s->p.regions = s->zero_regions;
    }
    if (p->enable_demag) {
        const int pbc[3] = {p->pbc[0], p->pbc[1], p->pbc[2]};
        if (p->demag_kernel == 1)
            st = demag_new_brute(p->N[0], p->N[1], p->N[2], pbc, p->cell[0], p->cell[1], p->cell[2],
                                 p->demag_accuracy > 0 ? p->demag_accuracy : 6.0, &s->demag);
        else
            st = demag_new_newell(p->N[0], p->N[1], p->N[2], pbc, p->cell[0], p->cell[1], p->cell[2],
                                  p->asymptotic_radius > 0 ? p->asymptotic_radius : 32, 0, &s->demag);
        if (st != UMAG_OK) return fail(st);
        if (cudaMalloc(&s->bd, b3) != cudaSuccess) return fail(set_error(UMAG_E_NOMEM, "demag field"));
    }
    if (cudaMalloc(&s->ctl, sizeof(DevCtl)) != cudaSuccess) return fail(set_error(UMAG_E_NOMEM, "ctl"));
    if (cudaMallocHost(&s->hctl, sizeof(DevCtl)) != cudaSuccess) return fail(set_error(UMAG_E_NOMEM, "ctl host"));
    DevCtl& c = *s->hctl;
    memset(&c, 0, sizeof(c));
    c.m = s->bufs;
    c.mw = s->bufs + 3 * (size_t)s->N;
    for (int i = 0; i < 7; i++) c.k[i] = s->bufs + (2 + i) * 3 * (size_t)s->N;
    c.dt = sp->dt;
    c.alarm = 0.0;
    c.stop = INFINITY;
    c.max_err = sp->max_err; c.rel_err = sp->rel_err; c.min_dt = sp->min_dt; c.max_dt = sp->max_dt;
    c.fix_dt = sp->fix_dt; c.headroom = sp->headroom; c.min_slope = sp->min_slope; c.gamma = sp->gamma_ll;
    c.active = 1;
    if (p->temp != nullptr || p->temp_mul != 0.f) {  // engine/temperature.go:111 (cellVolume: c0 c1 c2)
        c.therm_gv = sp->gamma_ll * (p->cell[0] * p->cell[1] * p->cell[2]);
        const double dt0 = sp->fix_dt != 0 ? sp->fix_dt : sp->dt;
        c.k2 = (float)(2 * kBoltzmann / (c.therm_gv * dt0));
    }
    st = push_ctl(s);
    if (st != UMAG_OK) return fail(st);
    // pass / local arguments
    if (s->demag) {
        fill_pass_args(s->demag, s->pa);
        s->pa.m_ind = &s->ctl->m;
        s->pa.m_ind_w = &s->ctl->mw;
        s->pa.active = &s->ctl->active;
        s->pa.fault = &s->ctl->status;
        s->pa.vol = p->vol;
        s->pa.Ms = p->Ms;
        s->pa.Ms_mul = p->Ms_mul;
        s->pa.ncell = s->N;
        for (int i = 0; i < 3; i++) s->pa.B[i] = s->bd + (size_t)i * s->N;
        if (p->nodemag_lut) {  // engine/demag.go:67-98 setMaskedDemagField
            if (cudaMalloc(&s->demag_vol, sizeof(float) * s->N) != cudaSuccess)
                return fail(set_error(UMAG_E_NOMEM, "NoDemagSpins volume"));
            k_nodemag_vol<<<grid_for(s->N, 256), 256, 0, S()>>>(p->vol, p->nodemag_lut, s->p.regions, s->demag_vol,
                                                                s->N);
            if (cudaStreamSynchronize(S()) != cudaSuccess) return fail(set_error(UMAG_E_CUDA, "NoDemagSpins volume"));
            s->pa.vol = s->demag_vol;
        }
    }
    LocalArgs& la = s->la;
    la.g = s->g;
    la.N = s->N;
    la.ctl = s->ctl;
    la.bd = s->bd;
    st = local_from_params(s);
    if (st != UMAG_OK) return fail(st);
    la.mbuf1 = s->bufs + 3 * (size_t)s->N;
    // default launch shapes for small meshes: enough CTAs to reach most SMs
    // (the autotuner may choose others; results do not depend on them)
    if ((long)((s->g.Nx + 31) / 32) * ((s->g.Ny + 7) / 8) * s->g.Nz < ctx().sm_count) s->tune.torque_block[1] = 2;
    if ((long)s->N < (long)ctx().sm_count * 256) s->tune.stage_threads = 64;
    tile_setup(s);
    if (la.dmi) {
        const int np = 256 * 257 / 2;
        if (cudaMalloc(&s->dmi_pairs, sizeof(float) * 7 * np) != cudaSuccess)
            return fail(set_error(UMAG_E_NOMEM, "DMI pair table"));
        float* t = s->dmi_pairs;
        la.dl = DmiPairLut{t, t + np, t + 2 * np, t + 3 * np, t + 4 * np, t + 5 * np, t + 6 * np};
        k_dmi_pairs<<<grid_for(np, 256), 256, 0, S()>>>(p->aLUT, p->dLUT, la.cx, la.cy, la.cz, t, t + np, t + 2 * np,
                                                        t + 3 * np, t + 4 * np, t + 5 * np, t + 6 * np, np);
        if (cudaStreamSynchronize(S()) != cudaSuccess) return fail(set_error(UMAG_E_CUDA, "DMI pair table"));
    }
    if (la.zeeman && (!p->bextLUT[1] || !p->bextLUT[2])) return fail(set_error(UMAG_E_ARG, "bextLUT needs 3 arrays"));
    int nl = 0;
    // count launches of one step (not enqueued: measured on a dry capture below)
    s->launches_per_step = 0;
    {
        cudaGraph_t graph;
        if (cudaStreamBeginCapture(S(), cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            st = launch_step(s, &nl);
            cudaStreamEndCapture(S(), &graph);
            cudaGraphDestroy(graph);
            if (st != UMAG_OK) return fail(st);
            s->launches_per_step = nl;
        }
    }
    *out = reinterpret_cast<umag_sim*>(s);
    return UMAG_OK;
}

int sim_free(umag_sim* h) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    if (!s) return UMAG_OK;
    cudaStreamSynchronize(S());
    drop_graph(s);
    if (s->demag) demag_free(s->demag);
    cudaFree(s->bufs);
    cudaFree(s->bd);
    cudaFree(s->zero_regions);
    cudaFree(s->dmi_pairs);
    cudaFree(s->demag_vol);
    cudaFree(s->kc_dev);
    cudaFree(s->esum);
    cudaFree(s->ctl);
    if (s->hctl) cudaFreeHost(s->hctl);
    delete s;
    return UMAG_OK;
}

// normalise = 0 restores a state read by sim_get_m exactly (normalising an
// already normalised float32 vector may change its last bit)
int sim_set_m(umag_sim* h, const float* mx, const float* my, const float* mz, int normalise) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s && mx && my && mz, "NULL argument");
    UMAG_TRY(sync_ctl_to_host(s));
    float* m = s->hctl->m;
    size_t b = sizeof(float) * s->N;
    UMAG_CUDA(cudaMemcpyAsync(m, mx, b, cudaMemcpyDeviceToDevice, S()));
    UMAG_CUDA(cudaMemcpyAsync(m + s->N, my, b, cudaMemcpyDeviceToDevice, S()));
    UMAG_CUDA(cudaMemcpyAsync(m + 2 * s->N, mz, b, cudaMemcpyDeviceToDevice, S()));
    // engine/magnetization.go:34 normalize() (normalize2.cl)
    if (normalise) UMAG_TRY(normalize(m, m + s->N, m + 2 * s->N, s->p.vol, s->N));
    else UMAG_CUDA(cudaStreamSynchronize(S()));
    s->need_k1 = true;
    return UMAG_OK;
}

int sim_m_ptrs(umag_sim* h, float** m3) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s && m3, "NULL argument");
    UMAG_TRY(sync_ctl_to_host(s));
    for (int c = 0; c < 3; c++) m3[c] = s->hctl->m + (size_t)c * s->N;
    return UMAG_OK;
}

int sim_get_m(umag_sim* h, float* mx, float* my, float* mz) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s && mx && my && mz, "NULL argument");
    float* m3[3];
    UMAG_TRY(sim_m_ptrs(h, m3));
    size_t b = sizeof(float) * s->N;
    float* dst[3] = {mx, my, mz};
    for (int c = 0; c < 3; c++) UMAG_CUDA(cudaMemcpyAsync(dst[c], m3[c], b, cudaMemcpyDefault, S()));
    UMAG_CUDA(cudaStreamSynchronize(S()));
    return UMAG_OK;
}

int sim_torque(umag_sim* h, float* tx, float* ty, float* tz, float* bx, float* by, float* bz) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s && tx && ty && tz, "NULL argument");
    UMAG_REQUIRE(ty == tx + s->N && tz == tx + 2 * s->N, "torque arrays must be one contiguous 3N buffer");
    if (bx) UMAG_REQUIRE(by == bx + s->N && bz == bx + 2 * s->N, "B_eff arrays must be one contiguous 3N buffer");
    UMAG_TRY(sync_ctl_to_host(s));
    s->hctl->active = 1;
    UMAG_TRY(push_ctl(s));
    UMAG_TRY(launch_torque(s, 0, 0, tx, bx, nullptr));
    UMAG_CUDA(cudaStreamSynchronize(S()));
    return UMAG_OK;
}

int sim_steps(umag_sim* h, int n) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s && n >= 0, "bad argument");
    UMAG_TRY(sync_ctl_to_host(s));
    s->hctl->stop = INFINITY;
    UMAG_TRY(push_ctl(s));
    return run_steps(s, n);
}

int sim_run(umag_sim* h, double seconds, int chunk, long long max_steps) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s && seconds >= 0, "bad argument");
    if (chunk <= 0) chunk = 64;
    UMAG_TRY(sync_ctl_to_host(s));
    double stop = s->hctl->t + seconds;
    s->hctl->stop = stop;
    s->hctl->alarm = stop;  // engine/run.go:190-195: adaptDt must not cross it
    UMAG_TRY(push_ctl(s));
    s->need_k1 = true;      // RunWhile frees the stepper (engine/run.go:207)
    long long done = 0;
    while (done < max_steps) {
        long long n = chunk;
        if (max_steps - done < n) n = max_steps - done;
        UMAG_TRY(run_steps(s, n));
        done += n;
        UMAG_TRY(sync_ctl_to_host(s));
        if (s->hctl->status != 0) return set_error(UMAG_E_SOLVER, "solver failure code %d at t=%g", s->hctl->status,
                                                   s->hctl->t);
        if (!(s->hctl->t < stop)) break;
    }
    return UMAG_OK;
}

// test hook: the device-side status word set as a kernel whose bounded wait
// gave up would set it (the host-side checks then see it)
int sim_plant_status(umag_sim* h, int code) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s, "NULL simulation");
    UMAG_CUDA(cudaStreamSynchronize(S()));
    UMAG_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(s->ctl) + offsetof(DevCtl, status), &code, sizeof(int),
                              cudaMemcpyHostToDevice, S()));
    UMAG_CUDA(cudaStreamSynchronize(S()));
    return UMAG_OK;
}

int sim_get_state(umag_sim* h, umag_solver_state* st) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s && st, "NULL argument");
    UMAG_TRY(sync_ctl_to_host(s));
    const DevCtl& c = *s->hctl;
    st->time = c.t; st->dt = c.dt; st->last_err = c.last_err; st->peak_err = c.peak_err;
    st->last_torque = c.last_torque; st->nsteps = c.nsteps; st->nundone = c.nundone; st->nevals = c.nevals;
    st->status = c.status;
    return UMAG_OK;
}

int sim_set_time(umag_sim* h, double t, double dt) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s, "NULL argument");
    UMAG_TRY(sync_ctl_to_host(s));
    s->hctl->t = t;
    if (dt > 0) s->hctl->dt = dt;
    return push_ctl(s);
}

int sim_average_m(umag_sim* h, double avg[3]) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s && avg, "NULL argument");
    float* m3[3];
    UMAG_TRY(sim_m_ptrs(h, m3));
    // engine/average.go:29-40: sum (or vol-weighted sum) over the magnet / cell count
    double ncell = (double)s->N;
    if (s->p.vol) UMAG_TRY(sum_dot(s->p.vol, nullptr, s->N, &ncell));
    for (int c = 0; c < 3; c++) {
        double v;
        UMAG_TRY(sum_dot(m3[c], s->p.vol, s->N, &v));
        avg[c] = v / ncell;
    }
    return UMAG_OK;
}

int sim_use_graph(umag_sim* h, int enable, int steps) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s, "NULL argument");
    s->use_graph = enable != 0;
    if (steps > 0 && steps != s->graph_steps) {
        s->graph_steps = steps;
        drop_graph(s);
    }
    return UMAG_OK;
}

int sim_torque_evals(umag_sim* h, int n) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s && n >= 0, "bad argument");
    UMAG_TRY(ensure_k1(s));
    UMAG_TRY(sync_ctl_to_host(s));
    s->hctl->active = 1;
    UMAG_TRY(push_ctl(s));
    for (int i = 0; i < n; i++) UMAG_TRY(launch_torque(s, 0, 0, nullptr, nullptr, nullptr));
    return UMAG_OK;
}

// engine/energy.go:27-35 GetTotalEnergy and its terms for the current m:
// E[0] total, E[1] demag (engine/demag.go:146), E[2] exchange incl. DMI
// (engine/exchange.go:79), E[3] anisotropy (engine/anisotropy.go:210),
// E[4] Zeeman (engine/zeeman.go:15).  Joules.
// engine/energy.go:36-42 SetTotalEdens: dst = 0, then each term's
// AddDotProduct(dst, prefactor, B_term, M_full) in float32, in the order the
// terms register (anisotropy -1/2 and -1/4, demag -1/2, exchange -1/2,
// Zeeman -1; engine/anisotropy.go:164-190, demag.go:31, exchange.go:34,
// zeeman.go:9)
__global__ void __launch_bounds__(256) k_energy_density(LocalArgs a, const float* __restrict__ vol, float* dst) {
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < a.N; I += gridDim.x * blockDim.x) {
        float t[kNE];
        energy_cell_terms(a, vol, I, t);
        float d = 0.0f;
        if (a.anis) {
            d = fa(d, fm(-0.5f, t[2]));
            d = fa(d, fm(-0.25f, t[3]));
        }
        if (a.cubic) {
            d = fa(d, fm(-0.25f, t[5]));
            d = fa(d, fm((float)(-1. / 6.), t[6]));
            d = fa(d, fm(-0.125f, t[7]));
        }
        if (a.bd) d = fa(d, fm(-0.5f, t[0]));
        d = fa(d, fm(-0.5f, t[1]));
        if (a.thermal) d = fa(d, fm(-1.0f, t[8]));
        if (a.zeeman) d = fa(d, fm(-1.0f, t[4]));
        dst[I] = d;
    }
}

int sim_energies(umag_sim* h, double E[5]) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s && E, "NULL argument");
    if (!s->esum) UMAG_CUDA(cudaMalloc(&s->esum, kNE * sizeof(double)));
    UMAG_TRY(sync_ctl_to_host(s));
    s->hctl->active = 1;
    UMAG_TRY(push_ctl(s));
    if (s->p.enable_demag) {
        PassArgs a = s->pa;
        a.m_sel = 0;
        UMAG_TRY(demag_launch(s->demag, a, S()));
    }
    UMAG_CUDA(cudaMemsetAsync(s->esum, 0, kNE * sizeof(double), S()));
    k_energy_terms<<<grid_for(s->N, 256, 4), 256, 0, S()>>>(s->la, s->p.vol, s->esum);
    UMAG_LAUNCH_CHECK();
    double t[kNE];
    UMAG_CUDA(cudaMemcpyAsync(t, s->esum, sizeof(t), cudaMemcpyDeviceToHost, S()));
    UMAG_CUDA(cudaStreamSynchronize(S()));
    const double V = s->p.cell[0] * s->p.cell[1] * s->p.cell[2];  // engine/energy.go:45-48 cellVolume
    const double Ed = -0.5 * V * t[0], Ee = -0.5 * V * t[1];
    // engine/anisotropy.go:164-206: uniaxial -1/2, -1/4; cubic -1/4, -1/6, -1/8
    const double Ea = V * (-0.5 * t[2] - 0.25 * t[3] - 0.25 * t[5] - t[6] / 6.0 - 0.125 * t[7]);
    const double Ez = -1.0 * V * t[4];
    const double Et = s->la.thermal ? -1.0 * V * t[8] : 0.0;  // engine/temperature.go:124-130
    E[1] = Ed; E[2] = Ee; E[3] = Ea; E[4] = Ez;
    // registration order of the terms (files anisotropy, demag, exchange, temperature, zeeman)
    E[0] = (((Ea + Ed) + Ee) + Et) + Ez;
    return UMAG_OK;
}

// per-cell total energy density (J/m^3) of the current m into dst (device, N floats)
int sim_energy_density(umag_sim* h, float* dst) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s && dst, "NULL argument");
    UMAG_REQUIRE(!s->batched, "energy density of a batched simulation");
    UMAG_TRY(sync_ctl_to_host(s));
    s->hctl->active = 1;
    UMAG_TRY(push_ctl(s));
    if (s->p.enable_demag) {
        PassArgs a = s->pa;
        a.m_sel = 0;
        UMAG_TRY(demag_launch(s->demag, a, S()));
    }
    k_energy_density<<<grid_for(s->N, 256), 256, 0, S()>>>(s->la, s->p.vol, dst);
    UMAG_LAUNCH_CHECK();
    UMAG_CUDA(cudaStreamSynchronize(S()));
    return UMAG_OK;
}

// switch the stepper / precession (engine/run.go:92-125 SetSolver); the
// stepper restarts (its FSAL torque is recomputed) and the step graphs are rebuilt
static void set_stepper(SimImpl* s, int solver, int precess) {
    if (s->sp.solver != solver || s->la.precess != precess) {
        s->sp.solver = solver;
        s->la.precess = precess;
        drop_graph(s);
    }
    s->need_k1 = true;
}

// engine/relax.go:134-141 relaxSteps: n accepted steps, then time is restored
static int relax_steps(SimImpl* s, int n) {
    UMAG_TRY(sync_ctl_to_host(s));
    const double t0 = s->hctl->t;
    const long long target = s->hctl->nsteps + n;
    s->hctl->stop = INFINITY;
    UMAG_TRY(push_ctl(s));
    s->need_k1 = true;  // runWhile frees the stepper (engine/run.go:207)
    for (int guard = 0; guard < 1000; guard++) {
        UMAG_TRY(sync_ctl_to_host(s));
        if (s->hctl->status != 0)
            return set_error(UMAG_E_SOLVER, "solver failure code %d during relax", s->hctl->status);
        if (s->hctl->nsteps >= target) break;
        UMAG_TRY(run_steps(s, target - s->hctl->nsteps));
    }
    UMAG_TRY(sync_ctl_to_host(s));
    s->hctl->t = t0;
    return push_ctl(s);
}

static int k1_max_norm(SimImpl* s, double* out) {
    UMAG_TRY(sync_ctl_to_host(s));
    const float* k = s->hctl->k[0];
    return max_vec_norm(k, k + s->N, k + 2 * (size_t)s->N, s->N, out);
}
static int k1_dot(SimImpl* s, float* out) {  // opencl.Dot(k1, k1), returned as float32
    UMAG_TRY(sync_ctl_to_host(s));
    double tot = 0;
    for (int c = 0; c < 3; c++) {
        const float* k = s->hctl->k[0] + (size_t)c * s->N;
        double v;
        UMAG_TRY(sum_dot(k, k, s->N, &v));
        tot += v;
    }
    *out = (float)tot;
    return UMAG_OK;
}

// engine/relax.go:23-112 Relax(): RK23 without precession, energy descent in
// chunks of 3 steps, then torque descent with MaxErr lowered by sqrt(2)
// down to 1e-9 (threshold <= 0), or steps while max |torque| > threshold.
int sim_relax(umag_sim* h, double threshold) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s, "NULL argument");
    UMAG_TRY(sync_ctl_to_host(s));
    const int prev_solver = s->sp.solver, prev_precess = s->la.precess;
    const double prev_err = s->hctl->max_err, prev_fix = s->hctl->fix_dt;
    const int prev_thermal = s->la.thermal;
    set_stepper(s, 3, 0);
    s->la.thermal = 0;  // engine/effectivefield.go:20: no B_therm while relaxing
    if (prev_thermal) drop_graph(s);  // the captured steps bake the flag in
    s->hctl->fix_dt = 0;
    UMAG_TRY(push_ctl(s));
    auto body = [&]() -> int {
        const int n = 3;  // evaluate the energy every 3 steps (relax.go:54)
        double E[5];
        UMAG_TRY(relax_steps(s, n));
        UMAG_TRY(sim_energies(h, E));
        double E0 = E[0];
        UMAG_TRY(relax_steps(s, n));
        UMAG_TRY(sim_energies(h, E));
        double E1 = E[0];
        for (int guard = 0; E1 < E0 && guard < 1000000; guard++) {
            UMAG_TRY(relax_steps(s, n));
            UMAG_TRY(sim_energies(h, E));
            E0 = E1;
            E1 = E[0];
        }
        if (threshold > 0) {
            for (;;) {
                double mt;
                UMAG_TRY(k1_max_norm(s, &mt));
                for (int guard = 0; mt > threshold && guard < 1000000; guard++) {
                    UMAG_TRY(relax_steps(s, n));
                    UMAG_TRY(k1_max_norm(s, &mt));
                }
                UMAG_TRY(sync_ctl_to_host(s));
                s->hctl->max_err /= std::sqrt(2.0);
                UMAG_TRY(push_ctl(s));
                if (s->hctl->max_err < 1e-9) break;
            }
        } else {
            float T0 = 0, T1;
            UMAG_TRY(k1_dot(s, &T1));
            for (;;) {
                UMAG_TRY(sync_ctl_to_host(s));
                if (!(s->hctl->max_err > 1e-9)) break;
                s->hctl->max_err /= std::sqrt(2.0);
                UMAG_TRY(push_ctl(s));
                UMAG_TRY(relax_steps(s, n));
                T0 = T1;
                UMAG_TRY(k1_dot(s, &T1));
                for (int guard = 0; T1 < T0 && guard < 1000000; guard++) {
                    UMAG_TRY(relax_steps(s, n));
                    T0 = T1;
                    UMAG_TRY(k1_dot(s, &T1));
                }
            }
        }
        return UMAG_OK;
    };
    const int st = body();
    // restore the caller's settings (relax.go:36-45)
    sync_ctl_to_host(s);
    s->hctl->max_err = prev_err;
    s->hctl->fix_dt = prev_fix;
    push_ctl(s);
    s->la.thermal = prev_thermal;
    drop_graph(s);
    set_stepper(s, prev_solver, prev_precess);
    return st;
}

// Reassigning solver settings between runs: SetSolver (engine/run.go:92-125,
// the stepper restarts), FixDt, MaxErr, RelErr, MinDt, MaxDt, Headroom,
// MinSlope, GammaLL.  The current time and dt are kept (assigning FixDt = 0
// resumes adaptive stepping from the last dt, as adaptDt does).
int sim_set_solver(umag_sim* h, const umag_solver_params* sp) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s && sp, "NULL argument");
    UMAG_REQUIRE(!s->batched, "solver settings of a batched simulation");
    UMAG_REQUIRE(sp->solver >= 1 && sp->solver <= 5,
                 "solver must be 1 (Euler), 2 (Heun), 3 (RK23), 4 (RK4) or 5 (RK45DP)");
    UMAG_TRY(sync_ctl_to_host(s));
    DevCtl& c = *s->hctl;
    c.max_err = sp->max_err; c.rel_err = sp->rel_err; c.min_dt = sp->min_dt; c.max_dt = sp->max_dt;
    c.fix_dt = sp->fix_dt; c.headroom = sp->headroom; c.min_slope = sp->min_slope;
    if (c.therm_gv != 0) c.therm_gv = sp->gamma_ll * (s->p.cell[0] * s->p.cell[1] * s->p.cell[2]);
    c.gamma = sp->gamma_ll;
    UMAG_TRY(push_ctl(s));
    const double dt_keep = s->sp.dt;
    const int prev = s->sp.solver;
    s->sp = *sp;
    s->sp.dt = dt_keep;
    s->sp.solver = prev;
    set_stepper(s, sp->solver, s->la.precess);  // new graphs only when the stepper changes
    return UMAG_OK;
}

// Launch shapes of the per-cell kernels: any valid shape gives the same
// results (per-cell arithmetic, max reductions), only the speed differs.
int sim_get_tuning(umag_sim* h, umag_tuning* t) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s && t, "NULL argument");
    *t = s->tune;
    return UMAG_OK;
}
int sim_set_tuning(umag_sim* h, const umag_tuning* t) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s && t, "NULL argument");
    const int bx = t->torque_block[0], by = t->torque_block[1];
    UMAG_REQUIRE(bx >= 32 && bx % 32 == 0 && by >= 1 && bx * by <= 256, "torque block %dx%d", bx, by);
    UMAG_REQUIRE(t->stage_threads == 64 || t->stage_threads == 128 || t->stage_threads == 256,
                 "stage threads %d", t->stage_threads);
    UMAG_REQUIRE(t->stage_waves >= 1 && t->stage_waves <= 64 && t->err_waves >= 1 && t->err_waves <= 64,
                 "waves must be 1..64");
    UMAG_REQUIRE(t->torque_tma == 0 || t->torque_tma == 1, "torque_tma must be 0 or 1");
    UMAG_CUDA(cudaStreamSynchronize(S()));
    s->tune = *t;
    if (!s->batched) tile_setup(s);  // the box follows the block shape
    drop_graph(s);  // the captured launches carry the old shapes
    return UMAG_OK;
}

// Reassigning a material parameter between runs (engine/parameter.go
// setRegion / SetValue): a per-cell device map (the caller keeps it alive
// while the simulation uses it) or NULL with a uniform value.
int sim_set_param(umag_sim* h, int which, const float* values, float mul) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s, "NULL argument");
    UMAG_REQUIRE(!s->batched, "parameters of a batched simulation");
    umag_sim_params& p = s->p;
    switch (which) {
    case UMAG_PARAM_MSAT: p.Ms = values; p.Ms_mul = mul; break;
    case UMAG_PARAM_ALPHA: p.alpha = values; p.alpha_mul = mul; break;
    case UMAG_PARAM_KU1: p.Ku1 = values; p.Ku1_mul = mul; break;
    case UMAG_PARAM_KU2: p.Ku2 = values; p.Ku2_mul = mul; break;
    case UMAG_PARAM_TEMP: p.temp = values; p.temp_mul = mul; break;
    case UMAG_PARAM_KC1: p.Kc1 = values; p.Kc1_mul = mul; break;
    case UMAG_PARAM_KC2: p.Kc2 = values; p.Kc2_mul = mul; break;
    case UMAG_PARAM_KC3: p.Kc3 = values; p.Kc3_mul = mul; break;
    default:
        if (which >= UMAG_PARAM_ANISU_X && which <= UMAG_PARAM_ANISU_X + 2) {
            p.anisU[which - UMAG_PARAM_ANISU_X] = values;
            p.anisU_mul[which - UMAG_PARAM_ANISU_X] = mul;
        } else if (which >= UMAG_PARAM_ANISC1_X && which <= UMAG_PARAM_ANISC1_X + 2) {
            p.anisC1[which - UMAG_PARAM_ANISC1_X] = values;
            p.anisC1_mul[which - UMAG_PARAM_ANISC1_X] = mul;
        } else if (which >= UMAG_PARAM_ANISC2_X && which <= UMAG_PARAM_ANISC2_X + 2) {
            p.anisC2[which - UMAG_PARAM_ANISC2_X] = values;
            p.anisC2_mul[which - UMAG_PARAM_ANISC2_X] = mul;
        } else {
            return set_error(UMAG_E_ARG, "unknown parameter %d", which);
        }
    }
    UMAG_CUDA(cudaStreamSynchronize(S()));
    drop_graph(s);  // the captured launches bake the old arguments in
    UMAG_TRY(local_from_params(s));
    if (which == UMAG_PARAM_TEMP) {  // engine/temperature.go:111: gamma V of the noise amplitude
        UMAG_TRY(sync_ctl_to_host(s));
        DevCtl& c = *s->hctl;
        c.therm_gv = s->la.thermal ? s->sp.gamma_ll * (p.cell[0] * p.cell[1] * p.cell[2]) : 0.0;
        if (c.therm_gv != 0) c.k2 = (float)(2 * kBoltzmann / (c.therm_gv * c.dt));
        UMAG_TRY(push_ctl(s));
    }
    s->need_k1 = true;  // the FSAL torque belongs to the old parameters
    return UMAG_OK;
}

// ================================================================ ensembles
// Many independent simulations advanced together (no reference counterpart:
// uMagNUS runs one simulation per process).  Instances with the same mesh
// form a class, run as one batched SimImpl: every field / stage / error
// kernel handles all instances of the class in one launch (grid extended by
// the instance index) and one controller thread per instance keeps its own
// time, dt and accept/reject decisions.  One CUDA graph steps every class,
// the classes on parallel branches.
//
// Scheduling: each class has its own stream and its own graph of
// graph_steps steps; the host keeps every unfinished class's stream fed with
// chunks of replays and polls each class on its own (an event after the
// chunk and its state copy), so a cheap class never waits for an expensive
// one.  When a chunk leaves at most 3/4 of a class's batch still running,
// the running instances are compacted to the front of the batch (their
// controller records, parameters and per-instance indices permuted; the
// state buffers stay where they are, the records point at them) and the
// class's graph is recaptured for the smaller batch, so finished instances
// stop costing launches.  Every instance's arithmetic is unchanged.
struct EnsClass {
    SimImpl* s = nullptr;
    // a general instance: one simulation made by sim_new from a full
    // umag_sim_params (region maps, per-cell maps, geometry, PBC, every
    // term), stepped by the single-simulation kernels on the class's stream
    bool general = false;
    std::vector<int> members;  // ensemble index of each batch slot
    float2* spec = nullptr;    // nb spectrum scratch copies
    float* params = nullptr;   // device: Ms[n_all], A00[n_all], D00[n_all]
    std::vector<float> hparams;  // host copy of params (permuted with the slots)
    int n_all = 0;             // instances of the class; the first s->nb slots are in the batch
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    cudaGraphExec_t gexec = nullptr;  // graph_steps steps of the current batch
    int gexec_nb = 0;                 // the batch size gexec was captured for
    bool busy = false, finished = false;
    long long replays = 0;
};
struct EnsImpl {
    std::vector<EnsClass> cls;
    std::vector<std::pair<int, int>> where;  // instance -> (class, slot in class)
    umag_solver_params sp;
    int graph_steps = 16;
};

static void ens_class_free(EnsClass& c) {
    if (c.gexec) cudaGraphExecDestroy(c.gexec);
    c.gexec = nullptr;
    if (c.s && c.general) {
        sim_free(reinterpret_cast<umag_sim*>(c.s));
        c.s = nullptr;
    }
    if (c.s) {
        SimImpl* s = c.s;
        drop_graph(s);
        if (s->demag) demag_free(s->demag);
        cudaFree(s->bufs);
        cudaFree(s->bd);
        cudaFree(s->zero_regions);
        cudaFree(s->kc_dev);
        cudaFree(s->ip_dev);
        cudaFree(s->ctl);
        if (s->hctl) cudaFreeHost(s->hctl);
        delete s;
        c.s = nullptr;
    }
    cudaFree(c.spec);
    cudaFree(c.params);
    if (c.st) cudaStreamDestroy(c.st);
    if (c.done) cudaEventDestroy(c.done);
    c.spec = nullptr;
    c.params = nullptr;
    c.st = nullptr;
    c.done = nullptr;
}

int ens_free(umag_ens* h) {
    EnsImpl* e = reinterpret_cast<EnsImpl*>(h);
    if (!e) return UMAG_OK;
    cudaDeviceSynchronize();
    for (auto& c : e->cls) ens_class_free(c);
    delete e;
    return UMAG_OK;
}

// one class: nb instances of mesh N, cell, with the listed parameters
static int ens_class_new(EnsClass& C, const umag_ens_instance* in, const std::vector<int>& members,
                         const umag_solver_params* sp, int demag) {
    const int nb = (int)members.size();
    const umag_ens_instance& r0 = in[members[0]];
    SimImpl* s = new SimImpl();
    C.s = s;
    C.members = members;
    C.n_all = nb;
    s->nb = nb;
    s->batched = true;
    s->sp = *sp;
    memset(&s->p, 0, sizeof(s->p));
    for (int i = 0; i < 3; i++) { s->p.N[i] = r0.N[i]; s->p.cell[i] = r0.cell[i]; }
    s->p.enable_demag = demag;
    s->p.precess = 1;
    s->N = r0.N[0] * r0.N[1] * r0.N[2];
    s->g = Mesh3{r0.N[0], r0.N[1], r0.N[2], 0};
    const size_t n3 = 3 * (size_t)s->N;
    UMAG_CUDA(cudaStreamCreateWithFlags(&C.st, cudaStreamNonBlocking));
    UMAG_CUDA(cudaEventCreateWithFlags(&C.done, cudaEventDisableTiming));
    UMAG_CUDA(cudaMalloc(&s->bufs, sizeof(float) * n3 * 9 * nb));
    UMAG_CUDA(cudaMemsetAsync(s->bufs, 0, sizeof(float) * n3 * 9 * nb, S()));
    UMAG_CUDA(cudaMalloc(&s->zero_regions, s->N));
    UMAG_CUDA(cudaMemsetAsync(s->zero_regions, 0, s->N, S()));
    s->p.regions = s->zero_regions;
    if (demag) {
        int pbc[3] = {0, 0, 0};
        UMAG_TRY(demag_new_newell(r0.N[0], r0.N[1], r0.N[2], pbc, r0.cell[0], r0.cell[1], r0.cell[2], 32, 0, &s->demag));
        UMAG_CUDA(cudaMalloc(&s->bd, sizeof(float) * n3 * nb));
        UMAG_CUDA(cudaMemsetAsync(s->bd, 0, sizeof(float) * n3 * nb, S()));
    }
    UMAG_CUDA(cudaMalloc(&s->ctl, sizeof(DevCtl) * nb));
    UMAG_CUDA(cudaMallocHost(&s->hctl, sizeof(DevCtl) * nb));
    memset(s->hctl, 0, sizeof(DevCtl) * nb);
    for (int b = 0; b < nb; b++) {
        DevCtl& c = s->hctl[b];
        float* base = s->bufs + (size_t)b * 9 * n3;
        c.m = base;
        c.mw = base + n3;
        for (int i = 0; i < 7; i++) c.k[i] = base + (2 + i) * n3;
        c.bd = s->bd ? s->bd + (size_t)b * n3 : nullptr;
        c.dt = sp->dt;
        c.stop = INFINITY;
        c.max_err = sp->max_err; c.rel_err = sp->rel_err; c.min_dt = sp->min_dt; c.max_dt = sp->max_dt;
        c.fix_dt = sp->fix_dt; c.headroom = sp->headroom; c.min_slope = sp->min_slope; c.gamma = sp->gamma_ll;
        c.active = 1;
    }
    UMAG_TRY(push_ctl(s));
    // per-instance uniform values: Ms, and the region-(0,0) LUT entries the
    // plain engine would use (engine/exchange.go:193-201 harmonic mean, float32)
    std::vector<float> hp(3 * nb);
    bool dmi = false, anis = false, zee = false;
    for (int b = 0; b < nb; b++) {
        const umag_ens_instance& r = in[members[b]];
        hp[b] = r.Ms;
        hp[nb + b] = 2.0f / (1.0f / r.Aex + 1.0f / r.Aex);
        const float D = r.Dind;
        hp[2 * nb + b] = D == 0.0f ? 0.0f : 2.0f / (1.0f / D + 1.0f / D);
        dmi |= D != 0.0f;
        anis |= r.Ku1 != 0.0f || r.Ku2 != 0.0f;
        zee |= r.B_ext[0] != 0.0f || r.B_ext[1] != 0.0f || r.B_ext[2] != 0.0f;
    }
    UMAG_CUDA(cudaMalloc(&C.params, sizeof(float) * 3 * nb));
    UMAG_CUDA(cudaMemcpyAsync(C.params, hp.data(), sizeof(float) * 3 * nb, cudaMemcpyHostToDevice, S()));
    C.hparams = hp;
    UMAG_CUDA(cudaStreamSynchronize(S()));
    UMAG_CUDA(cudaMalloc(&s->ip_dev, sizeof(InstParams) * nb));
    LocalArgs& la = s->la;
    la.g = s->g;
    la.N = s->N;
    la.ctl = s->ctl;
    la.bd = nullptr;
    la.regions = s->zero_regions;
    la.cx = (float)r0.cell[0]; la.cy = (float)r0.cell[1]; la.cz = (float)r0.cell[2];
    la.wx = (float)(2 / (r0.cell[0] * r0.cell[0]));
    la.wy = (float)(2 / (r0.cell[1] * r0.cell[1]));
    la.wz = (float)(2 / (r0.cell[2] * r0.cell[2]));
    la.dmi = dmi;
    la.openbc = 0;
    la.anis = anis;
    la.zeeman = zee;
    la.precess = 1;
    la.ms_uniform = 1; la.alpha_uniform = 1; la.anis_uniform = 1;
    la.ip = s->ip_dev;
    std::vector<InstParams> hip(nb);
    for (int b = 0; b < nb; b++) {  // uniform constants of each instance, bit-identical to the plain engine's
        const umag_ens_instance& r = in[members[b]];
        LocalArgs t = la;
        t.aLUT = C.params + nb + b;
        t.dLUT = C.params + 2 * nb + b;
        t.alpha_mul = r.alpha;
        t.Ms_mul = r.Ms;
        t.up = UniaxParams{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, r.Ms, r.Ku1, r.Ku2,
                           r.anisU[0], r.anisU[1], r.anisU[2]};
        k_local_consts<<<1, 1, 0, S()>>>(t, &s->ip_dev[b].kc);
        UMAG_LAUNCH_CHECK();
        hip[b].alpha_mul = r.alpha;
        hip[b].Ms_mul = r.Ms;
        hip[b].dmi = r.Dind != 0.0f;
        for (int c = 0; c < 3; c++) hip[b].bext[c] = r.B_ext[c];
    }
    UMAG_CUDA(cudaStreamSynchronize(S()));
    // fill the non-kc fields without touching kc
    for (int b = 0; b < nb; b++)
        UMAG_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(s->ip_dev + b) + offsetof(InstParams, alpha_mul),
                                  reinterpret_cast<char*>(&hip[b]) + offsetof(InstParams, alpha_mul),
                                  sizeof(InstParams) - offsetof(InstParams, alpha_mul), cudaMemcpyHostToDevice, S()));
    UMAG_CUDA(cudaStreamSynchronize(S()));
    if (demag) {
        fill_pass_args(s->demag, s->pa);
        const long spec_elems = 3L * s->demag->P[2] * s->demag->N[1] * s->demag->Lx;  // one plan's spectrum
        UMAG_CUDA(cudaMalloc(&C.spec, sizeof(float2) * spec_elems * nb));
        UMAG_CUDA(cudaMemsetAsync(C.spec, 0, sizeof(float2) * spec_elems * nb, S()));
        s->pa.spec = C.spec;
        s->pa.spec_stride = spec_elems;
        s->pa.m_ind = &s->ctl[0].m;
        s->pa.m_ind_w = &s->ctl[0].mw;
        s->pa.active = &s->ctl[0].active;
        s->pa.fault = &s->ctl[0].status;
        s->pa.ctl_stride = sizeof(DevCtl);
        s->pa.vol = nullptr;
        s->pa.Ms = nullptr;
        s->pa.Ms_mul = 0.0f;
        s->pa.ms_mul_b = C.params;
        s->pa.ncell = s->N;
        for (int c = 0; c < 3; c++) s->pa.B[c] = s->bd + (size_t)c * s->N;
        s->pa.b_stride = (long)n3;
    }
    return UMAG_OK;
}

// a class of one general instance: the simulation sim_new makes from the
// full parameter record, with its own stream and completion event
static int ens_class_new_general(EnsClass& C, int member, const umag_sim_params* p, const umag_solver_params* sp) {
    C.general = true;
    C.members = {member};
    C.n_all = 1;
    umag_sim* h = nullptr;
    UMAG_TRY(sim_new(p, sp, &h));
    C.s = reinterpret_cast<SimImpl*>(h);
    UMAG_CUDA(cudaStreamCreateWithFlags(&C.st, cudaStreamNonBlocking));
    UMAG_CUDA(cudaEventCreateWithFlags(&C.done, cudaEventDisableTiming));
    return UMAG_OK;
}

int ens_new(int n, const umag_ens_instance* in, const umag_solver_params* sp, int demag, umag_ens** out) {
    return ens_new_general(n, in, nullptr, sp, demag, out);
}

int ens_new_general(int n, const umag_ens_instance* in, const umag_sim_params* const* general,
                    const umag_solver_params* sp, int demag, umag_ens** out) {
    UMAG_TRY(ensure_init());
    UMAG_REQUIRE(n > 0 && sp && out, "bad argument");
    UMAG_REQUIRE(sp->solver >= 1 && sp->solver <= 5, "unknown solver");
    for (int i = 0; i < n; i++)
        UMAG_REQUIRE(in || (general && general[i]), "instance %d: no uniform record and no general parameters", i);
    EnsImpl* e = new EnsImpl();
    e->sp = *sp;
    e->where.resize(n);
    auto fail = [&](int code) { ens_free(reinterpret_cast<umag_ens*>(e)); return code; };
    // classes: same mesh and cell size; each general instance is a class of its own
    std::vector<std::vector<int>> groups;
    std::vector<int> gen_of;  // class -> general instance, or -1
    for (int i = 0; i < n; i++) {
        if (general && general[i]) {
            e->where[i] = {(int)groups.size(), 0};
            groups.push_back({i});
            gen_of.push_back(i);
            continue;
        }
        const umag_ens_instance& r = in[i];
        if (r.N[0] <= 0 || r.N[1] <= 0 || r.N[2] <= 0) return fail(set_error(UMAG_E_ARG, "instance %d: bad mesh", i));
        if (!(r.Ms > 0) || !(r.Aex > 0)) return fail(set_error(UMAG_E_ARG, "instance %d: Ms and Aex must be > 0", i));
        int g = -1;
        for (size_t k = 0; k < groups.size(); k++) {
            if (gen_of[k] >= 0) continue;
            const umag_ens_instance& q = in[groups[k][0]];
            if (q.N[0] == r.N[0] && q.N[1] == r.N[1] && q.N[2] == r.N[2] && q.cell[0] == r.cell[0] &&
                q.cell[1] == r.cell[1] && q.cell[2] == r.cell[2])
                g = (int)k;
        }
        if (g < 0) { groups.push_back({}); gen_of.push_back(-1); g = (int)groups.size() - 1; }
        e->where[i] = {g, (int)groups[g].size()};
        groups[g].push_back(i);
    }
    e->cls.resize(groups.size());
    for (size_t k = 0; k < groups.size(); k++) {
        const int st = gen_of[k] >= 0 ? ens_class_new_general(e->cls[k], gen_of[k], general[gen_of[k]], sp)
                                      : ens_class_new(e->cls[k], in, groups[k], sp, demag);
        if (st != UMAG_OK) return fail(st);
    }
    *out = reinterpret_cast<umag_ens*>(e);
    return UMAG_OK;
}

// every slot's controller record to the host (the batch may be smaller
// than the class after compaction; records past it do not change)
static int ens_sync_all(EnsClass& C) {
    SimImpl* s = C.s;
    UMAG_CUDA(cudaMemcpyAsync(s->hctl, s->ctl, sizeof(DevCtl) * C.n_all, cudaMemcpyDeviceToHost, S()));
    UMAG_CUDA(cudaStreamSynchronize(S()));
    return UMAG_OK;
}
static int ens_push_all(EnsClass& C) {
    SimImpl* s = C.s;
    UMAG_CUDA(cudaMemcpyAsync(s->ctl, s->hctl, sizeof(DevCtl) * C.n_all, cudaMemcpyHostToDevice, S()));
    UMAG_CUDA(cudaStreamSynchronize(S()));
    return UMAG_OK;
}

static SimImpl* ens_sim(EnsImpl* e, int i, int* b) {
    const auto& w = e->where[i];
    *b = w.second;
    return e->cls[w.first].s;
}

int ens_set_m(umag_ens* h, int i, const float* host_m) {
    EnsImpl* e = reinterpret_cast<EnsImpl*>(h);
    UMAG_REQUIRE(e && host_m && i >= 0 && i < (int)e->where.size(), "bad argument");
    int b;
    SimImpl* s = ens_sim(e, i, &b);
    UMAG_TRY(ens_sync_all(e->cls[e->where[i].first]));
    float* m = s->hctl[b].m;
    // on the library stream, so that the normalisation below sees the copy
    UMAG_CUDA(cudaMemcpyAsync(m, host_m, sizeof(float) * 3 * s->N, cudaMemcpyHostToDevice, S()));
    // engine/magnetization.go:34 (the geometry mask of a general instance; none in a batch)
    UMAG_TRY(normalize(m, m + s->N, m + 2 * (size_t)s->N, s->p.vol, s->N));
    UMAG_CUDA(cudaDeviceSynchronize());
    s->need_k1 = true;
    return UMAG_OK;
}

int ens_get_m(umag_ens* h, int i, float* host_m) {
    EnsImpl* e = reinterpret_cast<EnsImpl*>(h);
    UMAG_REQUIRE(e && host_m && i >= 0 && i < (int)e->where.size(), "bad argument");
    int b;
    SimImpl* s = ens_sim(e, i, &b);
    UMAG_TRY(ens_sync_all(e->cls[e->where[i].first]));
    UMAG_CUDA(cudaMemcpyAsync(host_m, s->hctl[b].m, sizeof(float) * 3 * s->N, cudaMemcpyDeviceToHost, S()));
    UMAG_CUDA(cudaStreamSynchronize(S()));
    return UMAG_OK;
}

int ens_get_state(umag_ens* h, int i, umag_solver_state* st) {
    EnsImpl* e = reinterpret_cast<EnsImpl*>(h);
    UMAG_REQUIRE(e && st && i >= 0 && i < (int)e->where.size(), "bad argument");
    int b;
    SimImpl* s = ens_sim(e, i, &b);
    UMAG_TRY(ens_sync_all(e->cls[e->where[i].first]));
    const DevCtl& c = s->hctl[b];
    st->time = c.t; st->dt = c.dt; st->last_err = c.last_err; st->peak_err = c.peak_err;
    st->last_torque = c.last_torque; st->nsteps = c.nsteps; st->nundone = c.nundone; st->nevals = c.nevals;
    st->status = c.status;
    return UMAG_OK;
}

// graph_steps steps of class C's current batch, captured on its stream
static int ens_capture(EnsImpl* e, EnsClass& C) {
    if (C.gexec && C.gexec_nb == C.s->nb) return UMAG_OK;  // still valid (shapes unchanged)
    if (C.gexec) { cudaGraphExecDestroy(C.gexec); C.gexec = nullptr; }
    g_launch_stream = C.st;
    const int st = capture_steps(C.s, e->graph_steps, &C.gexec);
    g_launch_stream = nullptr;
    C.gexec_nb = st == UMAG_OK ? C.s->nb : 0;
    return st;
}

// Compact the running instances of class C to the front of its batch (the
// host records are fresh: its stream is idle).  Slot k takes the instance of
// old slot order[k]: its controller record (which points at its own state
// buffers; the demag-field scratch pointer is the slot's), its parameters
// and its uniform constants.
static int ens_compact(EnsImpl* e, int ci) {
    EnsClass& C = e->cls[ci];
    if (C.general) return UMAG_OK;  // one instance: nothing to compact
    SimImpl* s = C.s;
    const int nb = s->nb;
    std::vector<int> order;
    for (int b = 0; b < nb; b++)
        if (s->hctl[b].t < s->hctl[b].stop && s->hctl[b].status == 0) order.push_back(b);
    const int na = (int)order.size();
    if (na == 0 || 4 * na > 3 * nb) return UMAG_OK;
    for (int b = 0; b < nb; b++)
        if (!(s->hctl[b].t < s->hctl[b].stop && s->hctl[b].status == 0)) order.push_back(b);
    std::vector<DevCtl> ctl(nb);
    std::vector<int> mem(nb);
    std::vector<float> hp = C.hparams;
    const size_t n3 = 3 * (size_t)s->N;
    InstParams* tmp = nullptr;
    UMAG_CUDA(cudaMalloc(&tmp, sizeof(InstParams) * nb));
    for (int k = 0; k < nb; k++) {
        const int o = order[k];
        ctl[k] = s->hctl[o];
        if (s->bd) ctl[k].bd = s->bd + (size_t)k * n3;
        mem[k] = C.members[o];
        for (int q = 0; q < 3; q++) hp[q * C.n_all + k] = C.hparams[q * C.n_all + o];
        UMAG_CUDA(cudaMemcpyAsync(tmp + k, s->ip_dev + o, sizeof(InstParams), cudaMemcpyDeviceToDevice, S()));
    }
    UMAG_CUDA(cudaMemcpyAsync(s->ip_dev, tmp, sizeof(InstParams) * nb, cudaMemcpyDeviceToDevice, S()));
    UMAG_CUDA(cudaStreamSynchronize(S()));
    cudaFree(tmp);
    for (int k = 0; k < nb; k++) {
        s->hctl[k] = ctl[k];
        C.members[k] = mem[k];
        e->where[mem[k]] = {ci, k};
    }
    C.hparams = hp;
    UMAG_CUDA(cudaMemcpyAsync(C.params, hp.data(), sizeof(float) * hp.size(), cudaMemcpyHostToDevice, S()));
    UMAG_TRY(ens_push_all(C));
    s->nb = na;
    return ens_capture(e, C);
}

// engine/run.go:190 Run(seconds) for every instance: each runs until its own
// time reaches start + seconds (its dt honours that alarm).  Classes advance
// independently, `chunk` graph replays at a time (at most max_replays each).
int ens_run(umag_ens* h, double seconds, int chunk, long long max_replays) {
    EnsImpl* e = reinterpret_cast<EnsImpl*>(h);
    UMAG_REQUIRE(e && seconds >= 0, "bad argument");
    if (chunk <= 0) chunk = 8;
    for (auto& C : e->cls) {
        SimImpl* s = C.s;
        UMAG_TRY(ens_sync_all(C));
        s->nb = C.n_all;  // every instance takes part again
        for (int b = 0; b < s->nb; b++) {
            s->hctl[b].stop = s->hctl[b].t + seconds;
            s->hctl[b].alarm = s->hctl[b].stop;
        }
        UMAG_TRY(ens_push_all(C));
        s->need_k1 = true;  // RunWhile frees the stepper (engine/run.go:207)
        UMAG_TRY(ensure_k1(s));
        UMAG_TRY(ens_capture(e, C));
        C.busy = false;
        C.finished = false;
        C.replays = 0;
    }
    UMAG_CUDA(cudaDeviceSynchronize());
    for (;;) {
        bool all_done = true, progressed = false;
        for (size_t ci = 0; ci < e->cls.size(); ci++) {
            EnsClass& C = e->cls[ci];
            SimImpl* s = C.s;
            if (C.finished) continue;
            all_done = false;
            if (C.busy) {
                const cudaError_t q = cudaEventQuery(C.done);
                if (q == cudaErrorNotReady) continue;
                if (q != cudaSuccess) return set_error(UMAG_E_CUDA, "ensemble class %zu: %s", ci, cudaGetErrorString(q));
                C.busy = false;
                progressed = true;
                int running = 0;
                for (int b = 0; b < s->nb; b++) {
                    const DevCtl& d = s->hctl[b];
                    if (d.status != 0)
                        return set_error(UMAG_E_SOLVER, "instance %d: solver failure code %d at t=%g", C.members[b],
                                         d.status, d.t);
                    running += d.t < d.stop;
                }
                if (running == 0 || C.replays >= max_replays) {
                    C.finished = true;
                    continue;
                }
                UMAG_TRY(ens_compact(e, (int)ci));
            }
            // the next chunk, then the batch's records back to the host
            for (int k = 0; k < chunk && C.replays < max_replays; k++, C.replays++)
                UMAG_CUDA(cudaGraphLaunch(C.gexec, C.st));
            UMAG_CUDA(cudaMemcpyAsync(s->hctl, s->ctl, sizeof(DevCtl) * s->nb, cudaMemcpyDeviceToHost, C.st));
            UMAG_CUDA(cudaEventRecord(C.done, C.st));
            C.busy = true;
            progressed = true;
        }
        if (all_done) break;
        if (!progressed) std::this_thread::yield();
    }
    UMAG_CUDA(cudaDeviceSynchronize());
    return UMAG_OK;
}

int ens_count(umag_ens* h, int* n_instances, int* n_classes) {
    EnsImpl* e = reinterpret_cast<EnsImpl*>(h);
    UMAG_REQUIRE(e, "NULL argument");
    if (n_instances) *n_instances = (int)e->where.size();
    if (n_classes) *n_classes = (int)e->cls.size();
    return UMAG_OK;
}

int ens_class_info(umag_ens* h, int cls, int N[3], int* n_instances) {
    EnsImpl* e = reinterpret_cast<EnsImpl*>(h);
    UMAG_REQUIRE(e && N && n_instances, "NULL argument");
    UMAG_REQUIRE(cls >= 0 && cls < (int)e->cls.size(), "class %d out of range", cls);
    const SimImpl* s = e->cls[cls].s;
    for (int i = 0; i < 3; i++) N[i] = s->p.N[i];
    *n_instances = e->cls[cls].n_all;
    return UMAG_OK;
}

int ens_class_general(umag_ens* h, int cls, int* general) {
    EnsImpl* e = reinterpret_cast<EnsImpl*>(h);
    UMAG_REQUIRE(e && general, "NULL argument");
    UMAG_REQUIRE(cls >= 0 && cls < (int)e->cls.size(), "class %d out of range", cls);
    *general = e->cls[cls].general ? 1 : 0;
    return UMAG_OK;
}

int ens_get_tuning(umag_ens* h, int cls, umag_tuning* t) {
    EnsImpl* e = reinterpret_cast<EnsImpl*>(h);
    UMAG_REQUIRE(e && t, "NULL argument");
    UMAG_REQUIRE(cls >= 0 && cls < (int)e->cls.size(), "class %d out of range", cls);
    *t = e->cls[cls].s->tune;
    return UMAG_OK;
}

// the class's launches take the new shapes at its next capture
int ens_set_tuning(umag_ens* h, int cls, const umag_tuning* t) {
    EnsImpl* e = reinterpret_cast<EnsImpl*>(h);
    UMAG_REQUIRE(e && t, "NULL argument");
    UMAG_REQUIRE(cls >= 0 && cls < (int)e->cls.size(), "class %d out of range", cls);
    EnsClass& C = e->cls[cls];
    UMAG_TRY(sim_set_tuning(reinterpret_cast<umag_sim*>(C.s), t));
    if (C.gexec) { cudaGraphExecDestroy(C.gexec); C.gexec = nullptr; }
    return UMAG_OK;
}

int sim_launches_per_step(umag_sim* h, int* n) {
    SimImpl* s = reinterpret_cast<SimImpl*>(h);
    UMAG_REQUIRE(s && n, "NULL argument");
    *n = s->launches_per_step;
    return UMAG_OK;
}

}  // namespace umag
