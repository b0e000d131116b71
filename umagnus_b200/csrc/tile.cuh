// tile.cuh -- magnetisation tiles with a one-cell halo, loaded by the Tensor
// Memory Accelerator (cp.async.bulk.tensor, no multicast) into shared memory
// for the field + torque kernel, and the exchange / interfacial-DMI stencils
// read from such a tile.
//
// A tile covers a CTA's BX x BY cells of one z plane.  The tensor map views
// one magnetisation buffer as a 4D array (x, y, z, component), x fastest;
// the box is (BX + 8) x (BY + 2) x (3 or 1 planes) x 3 components, started
// at x0 - 4 (x starts must be multiples of 4 floats = 16 bytes), y0 - 1 and
// z - 1.  Coordinates outside the mesh are filled with zeros.  A zero
// neighbour is what the reference's stencils see for a missing neighbour
// (dmi.cl: m1 = 0 outside the grid) and, for exchange and the z terms, it
// is replaced by m0 exactly as the clamped index (stencil.clh) gives m0: the
// arithmetic, hence the rounding, is the same as exchange_sum_u / dmi_sum_u.
// Periodic meshes keep the global loads (the box does not wrap).
#pragma once
#include <cuda.h>
#include <cstdint>

#include "cellmath.cuh"

namespace umag {

constexpr int kTileHaloX = 4;           // left halo rounded up to 16 bytes
constexpr int kTileWaitLimit = 1 << 16;  // mbarrier polls before the error flag

struct TileMaps {
    CUtensorMap map[2];  // one per magnetisation buffer (state / working)
};

__host__ __device__ constexpr int tile_pitch(int bx) { return bx + 2 * kTileHaloX; }
__host__ __device__ constexpr int tile_rows(int by) { return by + 2; }
__host__ __device__ inline size_t tile_bytes(int bx, int by, int nz) {
    return sizeof(float) * 3 * (size_t)(nz > 1 ? 3 : 1) * tile_rows(by) * tile_pitch(bx);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// One bounded wait step: the thread may be suspended until the phase
// completes or about kMbarSuspendNs nanoseconds pass (PTX suspendTimeHint),
// so waiting warps sleep instead of spinning through issue slots.
constexpr uint32_t kMbarSuspendNs = 1000;
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase), "r"(kMbarSuspendNs)
        : "memory");
    return ok != 0;
}
// 4D tiled load of the box at (x, y, z, c) into dst, completing on bar
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int y, int z, int c,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(c), "r"(smem_u32(bar))
        : "memory");
}

// 5D tiled load of the box at (c0..c4) into dst, completing on bar
__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            int c4, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
        "%6}], [%7];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
        : "memory");
}

// Bulk tensor store of a shared-memory box (the async proxy reads it): the
// writers' stores are made visible to that proxy by fence_proxy_async before
// the barrier that precedes the store; the issuing thread then commits the
// group and waits until the box has been read before the memory is reused or
// the CTA exits.  The global writes complete with the grid.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void tma_store_5d(const CUtensorMap* map, const void* src, int c0, int c1, int c2, int c3,
                                             int c4) {
    asm volatile(
        "cp.async.bulk.tensor.5d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];\n" ::"l"(
            reinterpret_cast<uint64_t>(map)),
        "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(src))
        : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }

// cuTensorMapEncodeTiled from the driver (looked up once; no libcuda link)
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
inline EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// Neighbour (dx, dy, dz) of the tile cell (tx, ty) on the centre plane zc
struct TileView {
    const float* t;
    int pitch, rows, planes, zc;
    __device__ __forceinline__ f3 at(int tx, int ty, int dx, int dy, int dz) const {
        const int i = ((zc + dz) * rows + ty + 1 + dy) * pitch + tx + kTileHaloX + dx;
        const int cs = planes * rows * pitch;
        return f3{t[i], t[cs + i], t[2 * cs + i]};
    }
};

// exchange_sum_u with the neighbours from a tile (same operations, same order)
__device__ __forceinline__ f3 exchange_sum_tile(const TileView& v, int tx, int ty, const PairCoef& P, bool three_d,
                                                f3 m0) {
    f3 b{0.f, 0.f, 0.f};
    const int nn = three_d ? 6 : 4;
#pragma unroll
    for (int k = 0; k < 6; k++) {
        if (k >= nn) break;
        const float s = k < 2 ? P.wax : (k < 4 ? P.way : P.waz);
        const int dx = k == 0 ? -1 : (k == 1 ? 1 : 0), dy = k == 2 ? -1 : (k == 3 ? 1 : 0);
        const int dz = k == 4 ? -1 : (k == 5 ? 1 : 0);
        f3 mn = v.at(tx, ty, dx, dy, dz);
        if (is0(mn)) mn = m0;
        b.x = fa(b.x, fm(s, fs(mn.x, m0.x)));
        b.y = fa(b.y, fm(s, fs(mn.y, m0.y)));
        b.z = fa(b.z, fm(s, fs(mn.z, m0.z)));
    }
    return b;
}

// dmi_sum_u with the neighbours from a tile (same operations, same order).
// CLOSED: the mesh is known not to use OpenBC, so every neighbour counts
// and a missing one is always extrapolated (computed and selected without
// a branch: the same values).
template <bool CLOSED = false>
__device__ __forceinline__ f3 dmi_sum_tile(const TileView& v, int tx, int ty, const PairCoef& P, bool openbc,
                                           bool three_d, f3 m0) {
    f3 h{0.f, 0.f, 0.f};
#pragma unroll
    for (int d = 0; d < 2; d++) {
#pragma unroll
        for (int side = -1; side <= 1; side += 2) {
            f3 mn = d == 0 ? v.at(tx, ty, side, 0, 0) : v.at(tx, ty, 0, side, 0);
            const bool missing = is0(mn);
            if (CLOSED || !missing || !openbc) {
                if (CLOSED) {
                    float q = d == 0 ? P.qx : P.qy;
                    if (side < 0) q = -q;
                    const f3 ext = d == 0 ? f3{fs(m0.x, fm(q, m0.z)), m0.y, fa(m0.z, fm(q, m0.x))}
                                          : f3{m0.x, fs(m0.y, fm(q, m0.z)), fa(m0.z, fm(q, m0.y))};
                    mn = missing ? ext : mn;
                } else if (missing) {
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
    if (three_d) {
#pragma unroll
        for (int side = -1; side <= 1; side += 2) {
            f3 mn = v.at(tx, ty, 0, 0, side);
            if (is0(mn)) mn = m0;
            h.x = fa(h.x, fm(P.sz, fs(mn.x, m0.x)));
            h.y = fa(h.y, fm(P.sz, fs(mn.y, m0.y)));
            h.z = fa(h.z, fm(P.sz, fs(mn.z, m0.z)));
        }
    }
    return h;
}

}  // namespace umag
