// ref_cl.h -- just enough OpenCL C, as host C++, to compile the reference's own kernels.
//
// TEST INFRASTRUCTURE ONLY.  ref_gen.py extracts named functions and kernels from the
// reference's .cl sources (UFF.cl, gridff_build.cl, GridFF.cl, Surface.cl) into
// oracle/_ref/gen/, rewriting only OpenCL syntax that C++ spells differently:
//   (float4)(a, b, c, d) and (float4){a, b}  ->  make_float4(a, b, c, d) / make_float4(a, b)
//   __local T name[N];                       ->  static T name[N];   (one work-group at a time)
// Their arithmetic is untouched.  This header supplies the vector types with the swizzles
// those kernels use (.xyz, .xy, .yz, .zw), component-wise operators, dot / cross / length,
// the float math built-ins, and an NDRange launcher whose work-items are fibers
// (ucontext), so barrier(CLK_LOCAL_MEM_FENCE) has its OpenCL meaning: every work-item of
// the group reaches it before any goes on.  A work-item that returns early leaves the
// group, as on a device.
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <vector>
#include <ucontext.h>

using std::cos;
using std::exp;
using std::fabs;
using std::floor;
using std::sin;
using std::sqrt;

#define __kernel
#define __global
#define __local
#define __constant const
#define __private
#define __read_only
#define __write_only
#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2
#define M_PI_F 3.14159265358979323846f

// ------------------------------------------------------------------ vector types
struct float2 { float x, y; };
struct float3;
// the identity swizzle v.xyz of a float3 (read only), converting to float3 where used
struct float3_xyz {
    float x, y, z;
    operator float3() const;
};
struct float3 {
    union {
        struct { float x, y, z; };
        struct { float2 xy; float z_; };
        struct { float x_; float2 yz; };
        float3_xyz xyz;
    };
};
inline float3_xyz::operator float3() const { float3 r; r.x = x; r.y = y; r.z = z; return r; }
struct float4 {
    union {
        struct { float x, y, z, w; };
        struct { float3 xyz; float w_; };
        struct { float2 xy; float2 zw; };
        struct { float x_; float2 yz; float w2_; };
    };
};
struct int2 { int x, y; };
struct int3 {
    union {
        struct { int x, y, z; };
        struct { int2 xy; int z_; };
    };
};
struct int4 {
    union {
        struct { int x, y, z, w; };
        struct { int3 xyz; int w_; };
        struct { int2 xy; int2 zw; };
    };
};

inline float2 make_float2(float a) { float2 r; r.x = r.y = a; return r; }
inline float2 make_float2(float a, float b) { float2 r; r.x = a; r.y = b; return r; }
inline float3 make_float3(float a) { float3 r; r.x = r.y = r.z = a; return r; }
inline float3 make_float3(float a, float b, float c) { float3 r; r.x = a; r.y = b; r.z = c; return r; }
inline float3 make_float3(float3 a) { return a; }
inline float4 make_float4(float a) { float4 r; r.x = r.y = r.z = r.w = a; return r; }
inline float4 make_float4(float a, float b, float c, float d) { float4 r; r.x = a; r.y = b; r.z = c; r.w = d; return r; }
inline float4 make_float4(float3 a, float d) { float4 r; r.x = a.x; r.y = a.y; r.z = a.z; r.w = d; return r; }
inline float4 make_float4(float4 a) { return a; }
inline int2 make_int2(int a, int b) { int2 r; r.x = a; r.y = b; return r; }
inline int3 make_int3(int a) { int3 r; r.x = r.y = r.z = a; return r; }
inline int3 make_int3(int a, int b, int c) { int3 r; r.x = a; r.y = b; r.z = c; return r; }
inline int4 make_int4(int a) { int4 r; r.x = r.y = r.z = r.w = a; return r; }
inline int4 make_int4(int a, int b, int c, int d) { int4 r; r.x = a; r.y = b; r.z = c; r.w = d; return r; }

// component-wise operators: vector (op) vector, vector (op) scalar, scalar (op) vector
#define CLV_OPS2(V, S)                                                                             \
    inline V operator+(V a, V b) { return make_##V(a.x + b.x, a.y + b.y); }                        \
    inline V operator-(V a, V b) { return make_##V(a.x - b.x, a.y - b.y); }                        \
    inline V operator*(V a, V b) { return make_##V(a.x * b.x, a.y * b.y); }                        \
    inline V operator/(V a, V b) { return make_##V(a.x / b.x, a.y / b.y); }                        \
    inline V operator*(V a, S s) { return make_##V(a.x * s, a.y * s); }                            \
    inline V operator*(S s, V a) { return make_##V(s * a.x, s * a.y); }                            \
    inline V operator/(V a, S s) { return make_##V(a.x / s, a.y / s); }                            \
    inline V operator-(V a) { return make_##V(-a.x, -a.y); }                                       \
    inline V& operator+=(V& a, V b) { a = a + b; return a; }                                       \
    inline V& operator-=(V& a, V b) { a = a - b; return a; }                                       \
    inline V& operator*=(V& a, V b) { a = a * b; return a; }                                       \
    inline V& operator*=(V& a, S s) { a = a * s; return a; }
#define CLV_OPS3(V, S)                                                                             \
    inline V operator+(V a, V b) { return make_##V(a.x + b.x, a.y + b.y, a.z + b.z); }             \
    inline V operator-(V a, V b) { return make_##V(a.x - b.x, a.y - b.y, a.z - b.z); }             \
    inline V operator*(V a, V b) { return make_##V(a.x * b.x, a.y * b.y, a.z * b.z); }             \
    inline V operator/(V a, V b) { return make_##V(a.x / b.x, a.y / b.y, a.z / b.z); }             \
    inline V operator*(V a, S s) { return make_##V(a.x * s, a.y * s, a.z * s); }                   \
    inline V operator*(S s, V a) { return make_##V(s * a.x, s * a.y, s * a.z); }                   \
    inline V operator/(V a, S s) { return make_##V(a.x / s, a.y / s, a.z / s); }                   \
    inline V operator-(V a) { return make_##V(-a.x, -a.y, -a.z); }                                 \
    inline V& operator+=(V& a, V b) { a = a + b; return a; }                                       \
    inline V& operator-=(V& a, V b) { a = a - b; return a; }                                       \
    inline V& operator*=(V& a, V b) { a = a * b; return a; }                                       \
    inline V& operator*=(V& a, S s) { a = a * s; return a; }
#define CLV_OPS4(V, S)                                                                             \
    inline V operator+(V a, V b) { return make_##V(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }  \
    inline V operator-(V a, V b) { return make_##V(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }  \
    inline V operator*(V a, V b) { return make_##V(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }  \
    inline V operator/(V a, V b) { return make_##V(a.x / b.x, a.y / b.y, a.z / b.z, a.w / b.w); }  \
    inline V operator*(V a, S s) { return make_##V(a.x * s, a.y * s, a.z * s, a.w * s); }          \
    inline V operator*(S s, V a) { return make_##V(s * a.x, s * a.y, s * a.z, s * a.w); }          \
    inline V operator/(V a, S s) { return make_##V(a.x / s, a.y / s, a.z / s, a.w / s); }          \
    inline V operator-(V a) { return make_##V(-a.x, -a.y, -a.z, -a.w); }                           \
    inline V& operator+=(V& a, V b) { a = a + b; return a; }                                       \
    inline V& operator-=(V& a, V b) { a = a - b; return a; }                                       \
    inline V& operator*=(V& a, V b) { a = a * b; return a; }                                       \
    inline V& operator*=(V& a, S s) { a = a * s; return a; }
CLV_OPS2(float2, float)
CLV_OPS3(float3, float)
CLV_OPS4(float4, float)
CLV_OPS2(int2, int)
CLV_OPS3(int3, int)
CLV_OPS4(int4, int)

inline float dot(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
inline float3 cross(float3 a, float3 b) { return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline float length(float3 a) { return std::sqrt(dot(a, a)); }
inline float length(float2 a) { return std::sqrt(dot(a, a)); }
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline float min(float a, float b) { return std::fmin(a, b); }
inline float max(float a, float b) { return std::fmax(a, b); }

// ------------------------------------------------------------------ NDRange launcher
namespace clref {

struct WorkItem {
    size_t gid[3], lid[3];
    ucontext_t ctx;
    bool done;
};

struct Launch {
    size_t gsize[3], lsize[3], group[3];
    WorkItem* cur;
    ucontext_t sched;
    std::function<void()> body;
};

inline Launch& L() {
    static thread_local Launch l;
    return l;
}

inline void trampoline() {
    L().body();
    L().cur->done = true;   // returning resumes uc_link, the scheduler
}

__attribute__((noinline)) inline void init_fiber(WorkItem& w, char* stack, size_t bytes, ucontext_t* link) {
    w.done = false;
    getcontext(&w.ctx);
    w.ctx.uc_stack.ss_sp = stack;
    w.ctx.uc_stack.ss_size = bytes;
    w.ctx.uc_link = link;
    makecontext(&w.ctx, trampoline, 0);
}

// Run body once per work-item of the NDRange global[3] in groups of local[3]; groups one after
// another, the work-items of a group as fibers switched at every barrier().
inline void launch(const size_t global[3], const size_t local[3], std::function<void()> body) {
    Launch& l = L();
    for (int d = 0; d < 3; d++) { l.gsize[d] = global[d]; l.lsize[d] = local[d]; }
    l.body = std::move(body);
    const size_t nl = local[0] * local[1] * local[2];
    const size_t stack_bytes = 256 * 1024;
    std::vector<WorkItem> wi(nl);
    std::vector<char> stacks(nl * stack_bytes);
    size_t ng[3];
    for (int d = 0; d < 3; d++) ng[d] = (global[d] + local[d] - 1) / local[d];
    for (size_t gz = 0; gz < ng[2]; gz++)
        for (size_t gy = 0; gy < ng[1]; gy++)
            for (size_t gx = 0; gx < ng[0]; gx++) {
                l.group[0] = gx; l.group[1] = gy; l.group[2] = gz;
                size_t k = 0;
                for (size_t lz = 0; lz < local[2]; lz++)
                    for (size_t ly = 0; ly < local[1]; ly++)
                        for (size_t lx = 0; lx < local[0]; lx++, k++) {
                            WorkItem& w = wi[k];
                            w.lid[0] = lx; w.lid[1] = ly; w.lid[2] = lz;
                            w.gid[0] = gx * local[0] + lx; w.gid[1] = gy * local[1] + ly; w.gid[2] = gz * local[2] + lz;
                            init_fiber(w, stacks.data() + k * stack_bytes, stack_bytes, &l.sched);
                        }
                // one pass = every live work-item runs to its next barrier or to its end
                bool live = true;
                while (live) {
                    live = false;
                    for (size_t i = 0; i < nl; i++) {
                        if (wi[i].done) continue;
                        l.cur = &wi[i];
                        swapcontext(&l.sched, &wi[i].ctx);
                        live = live || !wi[i].done;
                    }
                }
            }
}

}  // namespace clref

inline size_t get_global_id(int d) { return clref::L().cur->gid[d]; }
inline size_t get_local_id(int d) { return clref::L().cur->lid[d]; }
inline size_t get_group_id(int d) { return clref::L().group[d]; }
inline size_t get_global_size(int d) { return clref::L().gsize[d]; }
inline size_t get_local_size(int d) { return clref::L().lsize[d]; }
inline void barrier(int) { swapcontext(&clref::L().cur->ctx, &clref::L().sched); }
