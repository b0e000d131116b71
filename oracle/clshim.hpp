// clshim.hpp -- lets the reference's OpenCL C hot-path kernels compile
// unchanged as C++17 for the CPU (TEST INFRASTRUCTURE ONLY).
//
// Used by build_ref.py, which includes the reference's own kernel sources
// (kernels_src/cl/*.cl, kernels_src/clh/*.clh) from the read-only reference
// tree and links them into oracle/_ref/libclref.so.  The resulting library
// runs the reference's kernel code on the host so the oracle's restatement
// can be checked against it; it is never part of the product.
//
// Semantics assumed for OpenCL built-ins (OpenCL 1.2 spec): dot/cross/
// length as written out below; normalize(v) = v * (1/sqrt(v.v)), zero for a
// zero vector.  Work-item functions read a thread-local NDRange position set
// by the driver loops in the generated wrappers.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <thread>
#include <vector>

#define __kernel
#define __global
#define __local
#define __constant const
#define __restrict
#define barrier(x)
#define CLK_LOCAL_MEM_FENCE 0

struct float3 { float x, y, z; };
struct double3 { double x, y, z; };
struct float2 { float x, y; };
struct double2 { double x, y; };
struct float4 { float x, y, z, w; };
struct double4 { double x, y, z, w; };

#define CLSHIM_VEC_OPS(V, S)                                                          \
    static inline V operator+(V a, V b) { return V{a.x + b.x, a.y + b.y, a.z + b.z}; } \
    static inline V operator-(V a, V b) { return V{a.x - b.x, a.y - b.y, a.z - b.z}; } \
    static inline V operator-(V a) { return V{-a.x, -a.y, -a.z}; }                     \
    static inline V operator*(S s, V a) { return V{s * a.x, s * a.y, s * a.z}; }       \
    static inline V operator*(V a, S s) { return V{a.x * s, a.y * s, a.z * s}; }       \
    static inline V& operator+=(V& a, V b) { a = a + b; return a; }                    \
    static inline V& operator-=(V& a, V b) { a = a - b; return a; }                    \
    static inline S dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }        \
    static inline V cross(V a, V b) {                                                  \
        return V{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; \
    }                                                                                  \
    static inline S length(V a) { return std::sqrt(dot(a, a)); }                       \
    static inline S distance(V a, V b) { return length(a - b); }                       \
    static inline V normalize(V a) {                                                   \
        S d = dot(a, a);                                                               \
        S inv = d > (S)0 ? (S)1 / std::sqrt(d) : (S)0;                                 \
        return V{a.x * inv, a.y * inv, a.z * inv};                                     \
    }
CLSHIM_VEC_OPS(float3, float)
CLSHIM_VEC_OPS(double3, double)
#undef CLSHIM_VEC_OPS

static inline int min(int a, int b) { return a < b ? a : b; }
static inline int max(int a, int b) { return a > b ? a : b; }
using std::fmax;
using std::sqrt;

// ---- NDRange emulation ---------------------------------------------------
struct clshim_item {
    size_t gid[3], gsize[3], lid[3], lsize[3], grp[3];
};
extern thread_local clshim_item clshim_cur;
static inline size_t get_global_id(int d) { return clshim_cur.gid[d]; }
static inline size_t get_global_size(int d) { return clshim_cur.gsize[d]; }
static inline size_t get_local_id(int d) { return clshim_cur.lid[d]; }
static inline size_t get_local_size(int d) { return clshim_cur.lsize[d]; }
static inline size_t get_group_id(int d) { return clshim_cur.grp[d]; }
static inline size_t get_num_groups(int d) { return clshim_cur.gsize[d] / clshim_cur.lsize[d]; }

// Host threads an NDRange is spread over (clref_set_threads); 1 = in order.
extern int clshim_nthreads;

// Runs body once per work-item of an NDRange with global size g and local
// size l (g a multiple of l in every dimension).  With clshim_nthreads > 1
// the linear work-item range is cut into one contiguous chunk per thread:
// valid for the wrapped kernels, which have no barriers and write only the
// elements of their own work-item.
template <class F>
static void clshim_ndrange(const size_t g[3], const size_t l[3], F body) {
    const size_t total = g[0] * g[1] * g[2];
    auto run = [&](size_t b, size_t e) {
        for (size_t i = b; i < e; i++) {
            const size_t p[3] = {i % g[0], (i / g[0]) % g[1], i / (g[0] * g[1])};
            for (int d = 0; d < 3; d++) {
                clshim_cur.gid[d] = p[d];
                clshim_cur.gsize[d] = g[d];
                clshim_cur.lsize[d] = l[d];
                clshim_cur.lid[d] = p[d] % l[d];
                clshim_cur.grp[d] = p[d] / l[d];
            }
            body();
        }
    };
    const int nt = clshim_nthreads;
    if (nt <= 1 || total < 8192) {
        run(0, total);
        return;
    }
    const size_t chunk = (total + nt - 1) / nt;
    std::vector<std::thread> th;
    for (int t = 1; t < nt; t++) {
        const size_t b = t * chunk, e = b + chunk < total ? b + chunk : total;
        if (b < e) th.emplace_back(run, b, e);
    }
    run(0, chunk < total ? chunk : total);
    for (auto& t : th) t.join();
}
