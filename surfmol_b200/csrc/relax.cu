// relax.cu -- persistent multi-system UFF + GridFF FIRE kernel for sm_100a.
//
// One "team" (a warp, or a CTA of 64..512 threads) owns one system at a time and
// keeps its whole state in shared memory: positions, velocities, forces, per-atom
// parameters, and the bond-direction cache hneigh.  Teams pull system indices from a
// global counter, run up to max_steps FIRE steps without leaving the kernel, write the
// system back and pull the next one, so ragged and early-converging systems balance
// dynamically.  Per FIRE step a team runs:
//
//   A  bonds + hneigh per atom ............ opencl/UFF.cl:141-322 (evalBondsAndHNeigh_UFF)
//   B  angles / dihedrals / inversions ..... opencl/UFF.cl:326-795, assembled (801-880) in
//      one of three forms, all without atomics and in a fixed order (bitwise reproducible,
//      independent of co-resident systems):
//        rounds - host-packed rounds in which the atoms of each role are distinct, added
//                 straight into the force array between team syncs
//        gather - all terms at once into a piece buffer, then a per-atom CSR gather
//        owner  - each atom evaluates the terms it owns (angle apex, inversion centre, both
//                 central atoms of a dihedral), keeps its neighbours' pieces in registers and
//                 stores them by bond slot; each atom then gathers over its bond back-slots
//   C  intramolecular LJ + Coulomb ......... opencl/UFF.cl:57-95, 1595-1665 (1-2 exclusion)
//      with L lanes per atom splitting the partner loop, combined by shuffles
//   D  tricubic B-spline grid sample ....... opencl/UFF.cl:1384-1511, 1671-1711, four lanes
//      per atom, lane k fetching the voxels at z offset k of the 16 (x, y) columns, so the
//      four lanes of an atom read each 4-voxel column as one contiguous 64 B run
//   E  FIRE ................................ crates/apps/molengine/src/main.rs:237-277, with
//      the power / norm sums in FP64 and reduced inside the team
//
// Everything is FP32 except the FIRE sums, the FIRE state (dt, alpha) and the
// per-system energy, which are FP64.  Every loop is bounded; there are no spin waits.
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <cstdio>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>

#include "smr_internal.h"

namespace smr {

namespace {

constexpr float kCoulomb = 14.3996448915f;   // eV*A/e^2
constexpr unsigned FULL = 0xffffffffu;

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline size_t red_bytes(int T) { return T > 32 ? size_t(T / 32) * 4 * sizeof(double) : 0; }

// Shared memory of one team for systems of up to nmax atoms (and nfmax bonded force pieces in
// the gather form).
__host__ __device__ inline size_t team_bytes(int nmax, int nfmax, int T, int form) {
    size_t n = (size_t)nmax;
    return n * 16 * 5 + n * 64 + align16(n * 4) + align16(n * 8) + red_bytes(T) +
           (form == FORM_GATHER || form == FORM_GATHER_EXT ? (size_t)nfmax * 16 : 0) + (form == FORM_OWNER ? n * 64 : 0);
}

// Shared memory of one team: one base pointer and the capacity; every array's address is
// computed on use (keeping ten 64-bit pointers live would cost twenty registers).
struct Smem {
    char* base;
    int n;
    __device__ __forceinline__ float4* P() const { return (float4*)base; }                         // positions
    __device__ __forceinline__ float4* Lo() const { return (float4*)(base + (size_t)n * 16); }      // low parts of positions
    __device__ __forceinline__ float4* V() const { return (float4*)(base + (size_t)n * 32); }       // velocities
    __device__ __forceinline__ float4* F() const { return (float4*)(base + (size_t)n * 48); }       // forces, w = per-atom energy
    __device__ __forceinline__ float4* Q() const { return (float4*)(base + (size_t)n * 64); }       // R, sqrt(E), Q, H
    // hneigh (unit bond vector, 1/length) of bond slot s of atom i at H()[s * n + i]: slot-major,
    // so lanes handling consecutive atoms touch consecutive words
    __device__ __forceinline__ float4* H() const { return (float4*)(base + (size_t)n * 80); }
    __device__ __forceinline__ float4 hget(int h) const { return H()[(h & 3) * n + (h >> 2)]; }   // h = 4 * atom + slot
    __device__ __forceinline__ float* Eh() const { return (float*)(base + (size_t)n * 144); }        // bond + NB part of E_atom
    __device__ __forceinline__ short4* Ng() const { return (short4*)(base + (size_t)n * 144 + align16((size_t)n * 4)); }
    __device__ __forceinline__ double* red() const {
        return (double*)(base + (size_t)n * 144 + align16((size_t)n * 4) + align16((size_t)n * 8));
    }
    __device__ __forceinline__ float4* Pc(int T) const {   // gather form: bonded force pieces
        return (float4*)((char*)red() + red_bytes(T));
    }
    // owner form: piece of the terms owned by atom o on its neighbour in slot s, at Fs()[s * n + o]
    __device__ __forceinline__ float4* Fs(int T) const { return (float4*)((char*)red() + red_bytes(T)); }
};

__device__ __forceinline__ Smem carve(char* base, int nmax) { Smem s; s.base = base; s.n = nmax; return s; }

template <int T> __device__ __forceinline__ void team_sync() {
    if (T == 32) __syncwarp(); else __syncthreads();
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(FULL, v, o));
    return v;
}

// Sums of three doubles and the max of one float over the team; every rank gets the
// same values (butterfly within a warp, fixed-order sum over warps).
template <int T>
__device__ __forceinline__ void team_reduce4(double& a, double& b, double& c, float& m, double* red, int rank) {
    a = warp_sum(a); b = warp_sum(b); c = warp_sum(c); m = warp_max(m);
    if (T > 32) {
        const int w = rank >> 5;
        if ((rank & 31) == 0) { red[4 * w] = a; red[4 * w + 1] = b; red[4 * w + 2] = c; red[4 * w + 3] = (double)m; }
        __syncthreads();
        a = 0; b = 0; c = 0; m = 0.f;
#pragma unroll 1
        for (int k = 0; k < T / 32; k++) { a += red[4 * k]; b += red[4 * k + 1]; c += red[4 * k + 2]; m = fmaxf(m, (float)red[4 * k + 3]); }
        __syncthreads();
    }
}

template <int T>
__device__ __forceinline__ double team_sum(double v, double* red, int rank) {
    double b = 0, c = 0; float m = 0.f;
    team_reduce4<T>(v, b, c, m, red, rank);
    return v;
}

__device__ __forceinline__ int comp(short4 v, int s) { return s == 0 ? v.x : (s == 1 ? v.y : (s == 2 ? v.z : v.w)); }
__device__ __forceinline__ float comp(float4 v, int s) { return s == 0 ? v.x : (s == 1 ? v.y : (s == 2 ? v.z : v.w)); }

__device__ __forceinline__ void add4(float4& a, float x, float y, float z, float w) { a.x += x; a.y += y; a.z += z; a.w += w; }

template <class Rec> __device__ __forceinline__ Rec load_rec(const Rec* p) {
    const int4* q = reinterpret_cast<const int4*>(p);
    int4 u = __ldg(q), v = __ldg(q + 1);
    Rec r;
    *reinterpret_cast<int4*>(&r) = u;
    *(reinterpret_cast<int4*>(&r) + 1) = v;
    return r;
}

// ---- grid voxel loads
template <int GDT> __device__ __forceinline__ float4 load_voxel(const void* g, unsigned i);
// Grid voxels are read through the non-coherent path without allocating in L1: the stencil
// lines are used once per atom-step and would otherwise evict the topology records.
__device__ __forceinline__ float4 ldg_stream(const float4* p) {
    float4 v;
    asm("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
    return v;
}
__device__ __forceinline__ uint2 ldg_stream(const uint2* p) {
    uint2 v;
    asm("ld.global.nc.L1::no_allocate.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "l"(p));
    return v;
}
template <> __device__ __forceinline__ float4 load_voxel<GRID_F32>(const void* g, unsigned i) {
    return ldg_stream(reinterpret_cast<const float4*>(g) + i);
}
template <> __device__ __forceinline__ float4 load_voxel<GRID_F16>(const void* g, unsigned i) {
    uint2 u = ldg_stream(reinterpret_cast<const uint2*>(g) + i);
    float2 a = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
    float2 b = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
    return make_float4(a.x, a.y, b.x, b.y);
}
template <> __device__ __forceinline__ float4 load_voxel<GRID_BF16>(const void* g, unsigned i) {
    uint2 u = ldg_stream(reinterpret_cast<const uint2*>(g) + i);
    float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.x));
    float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.y));
    return make_float4(a.x, a.y, b.x, b.y);
}

// cubic B-spline value / derivative weights (opencl/UFF.cl:1410-1432)
__device__ __forceinline__ void bspline(float u, float b[4], float d[4]) {
    const float i6 = 1.0f / 6.0f, u2 = u * u, t = 1.0f - u;
    b[0] = i6 * t * t * t;
    b[1] = i6 * (3.0f * u2 * (u - 2.0f) + 4.0f);
    b[2] = i6 * (3.0f * u * (1.0f + u - u2) + 1.0f);
    b[3] = i6 * u2 * u;
    d[0] = -0.5f * t * t;
    d[1] = 0.5f * (3.0f * u2 - 4.0f * u);
    d[2] = 0.5f * (-3.0f * u2 + 2.0f * u + 1.0f);
    d[3] = 0.5f * u2;
}

__device__ __forceinline__ int imod(int i, int m) { int r = i % m; return r < 0 ? r + m : r; }

// One lane's share of an atom's tricubic stencil over a grid array of nzs z planes: the voxels at
// z offset kz of the 16 (x, y) columns of cell (ix, iy, iz), combined over the channels with the
// prefactors PL, summed with the x / y weights: sE = sum bx by c, sX = sum dx by c, sY = sum bx dy c.
// 32-bit voxel indices (the host keeps grids below 2^31 voxels): column offsets of the 4 x and 4 y
// stencil rows, wrapped periodically, then one add per voxel.  Brick copy (smr_internal.h):
// stencil row pair / quad b of column x lies in the 128-byte line of brick (x, y0 + b - b % DY,
// iz - 1), element (b % DY) * 4 + kz, so the 4 lanes of an atom read aligned 64 B (fp32) or
// 32 B (16-bit) pieces of it.
template <int GDT>
__device__ __forceinline__ void stencil_sums(const void* data, int brick, int nx, int ny, int nzs, int ix, int iy, int iz, int kz,
                                             float PLx, float PLy, float PLz, const float bx[4], const float dxw[4],
                                             const float by[4], const float dyw[4], float& sE, float& sX, float& sY) {
    constexpr int DY = GDT == GRID_F32 ? 2 : 4;
    const int x0 = imod(ix - 1, nx), y0 = imod(iy - 1, ny);
    const int ystr = brick ? (nzs - 3) * DY * 4 : nzs;
    const int nyz = ny * ystr;
    int yo[4];
#pragma unroll
    for (int b = 0; b < 4; b++) {
        const int yg = brick ? y0 + b - b % DY : y0 + b;
        yo[b] = (yg >= ny ? yg - ny : yg) * ystr + (brick ? (b % DY) * 4 : 0);
    }
    const int zoff = brick ? (iz - 1) * DY * 4 + kz : iz - 1 + kz;
#pragma unroll
    for (int ax = 0; ax < 4; ax++) {
        const int xg = x0 + ax;
        const unsigned xo = (unsigned)(xg >= nx ? xg - nx : xg) * (unsigned)nyz + (unsigned)zoff;
        float pE = 0.f, pY = 0.f;
#pragma unroll
        for (int b = 0; b < 4; b++) {
            const float4 v = load_voxel<GDT>(data, (unsigned)xo + (unsigned)yo[b]);
            const float cs = PLx * v.x + PLy * v.y + PLz * v.z;
            pE += by[b] * cs; pY += dyw[b] * cs;
        }
        sE += bx[ax] * pE; sX += dxw[ax] * pE; sY += bx[ax] * pY;
    }
}

// L2 prefetch of the brick lines of every atom's stencil (brick layout only): line l of an atom is
// x column l / (NL / 4), y brick (l % (NL / 4)) * DY; one prefetch per line, lines spread over the team.
// Cells are taken in FP32 (a line fetched for a cell the FP64 decision at a z bound moves is only
// an unused prefetch); cells outside [1, nz-2) fetch nothing.
template <int T, int GDT>
__device__ __forceinline__ void grid_prefetch_l2(const GridView& g, const Smem& S, int N, int rank) {
    constexpr int DY = GDT == GRID_F32 ? 2 : 4, NL = 16 / DY, VB = GDT == GRID_F32 ? 16 : 8;
    const int nzb = g.nz - 3;
    for (int t = rank; t < N * NL; t += T) {
        const int i = t / NL, l = t % NL;
        const float4 p = S.P()[i];
        const float ux = (p.x - g.p0[0]) * g.inv_step[0], uy = (p.y - g.p0[1]) * g.inv_step[1];
        const int iz = (int)((p.z - g.p0[2]) * g.inv_step[2]);
        if (iz < 1 || iz >= g.nz - 2) continue;
        int ix = (int)ux, iy = (int)uy;
        if (ux < 0) ix--;
        if (uy < 0) iy--;
        const int xg = imod(ix - 1 + l / (NL / 4), g.nx);
        const int yb = imod(iy - 1 + (l % (NL / 4)) * DY, g.ny);
        const size_t e = (((size_t)xg * g.ny + yb) * nzb + (iz - 1)) * (size_t)(DY * 4);
        const char* ptr = reinterpret_cast<const char*>(g.data) + e * VB;
        asm volatile("prefetch.global.L2 [%0];" :: "l"(ptr));
    }
}


// Cutoff decision for a pair whose FP32 r^2 lies within 1e-4 of rc^2: the squared distance from
// the exact coordinate differences in FP64, as the CPU evaluators compute it.  Not inlined: the
// rare path keeps its registers out of the partner loop.
__device__ __noinline__ bool beyond_cutoff_fp64(float4 pi, float4 li, float4 pj, float4 lj, float rc2) {
    const double dx = ((double)pj.x - (double)pi.x) + ((double)lj.x - (double)li.x);
    const double dy = ((double)pj.y - (double)pi.y) + ((double)lj.y - (double)li.y);
    const double dz = ((double)pj.z - (double)pi.z) + ((double)lj.z - (double)li.z);
    return dx * dx + dy * dy + dz * dz > (double)rc2;
}

// z cell of a position near the grid's lower or upper bound: (z - p0) / step in FP64 from the
// compensated position.  Not inlined: the rare path keeps its registers out of the stencil loop.
__device__ __noinline__ int grid_cell_z_fp64(float pz, float lz, const GridView& g) {
    return (int)((((double)pz + (double)lz) - g.p0z) / g.stepz);
}

// Folded surface, one lane's share of an atom: the z-decay terms iz = lane, lane + 4, ... of
// SurfaceFolded::eval_atom_scratch (crates/libs/surfff/src/lib.rs:277-320) with the atom's
// prefactors of NonBondedFF::make_plqs (crates/libs/molff/src/nonbonded.rs:98-108: e = exp(-alpha R),
// L = e sqrt(req1), P = e L).  Returns E and dE/du, dE/dv, dE/dz.  Not inlined: its registers stay
// out of the kernels' other phases.
__device__ __noinline__ float4 folded_part(const FoldedView f, float4 p, float4 lo, float4 q, int lane) {
    const float e = expf(-f.alpha * q.x);
    const float L = e * sqrtf(q.y), P = e * L, Q = q.z;
    const float z = p.z + lo.z;
    // fractional coordinates to ~1e-7 of a cell: the whole cells n are taken off inside the first
    // fma, so the products are rounded only once they are small, and the inverse's rounding
    // remainder and the positions' low words enter as corrections (one product rounding at |u| ~ 4
    // would already cost 2.4e-7, or 1.5e-6 rad of phase)
    const float nu = floorf(f.inv[0] * p.x + f.inv[2] * p.y), nv = floorf(f.inv[1] * p.x + f.inv[3] * p.y);
    float u = fmaf(f.inv[0], p.x, -nu), v = fmaf(f.inv[1], p.x, -nv);
    u = fmaf(f.inv[2], p.y, u); v = fmaf(f.inv[3], p.y, v);
    u = fmaf(f.inv_lo[0], p.x, fmaf(f.inv_lo[2], p.y, u)); v = fmaf(f.inv_lo[1], p.x, fmaf(f.inv_lo[3], p.y, v));
    u = fmaf(f.inv[0], lo.x, fmaf(f.inv[2], lo.y, u)); v = fmaf(f.inv[1], lo.x, fmaf(f.inv[3], lo.y, v));
    u -= floorf(u); v -= floorf(v);
    const float* kx = f.k;
    const float* ky = kx + f.nx;
    const float* kz = ky + f.ny;
    const float* z0 = kz + f.nz;
    const float tau = 6.28318530717958647692f;
    float E = 0.f, du = 0.f, dv = 0.f, dz = 0.f;
    for (int iz = lane; iz < f.nz; iz += 4) {
        const float bz = expf(-__ldg(kz + iz) * (z - __ldg(z0 + iz))), dbz = -__ldg(kz + iz) * bz;
        for (int iy = 0; iy < f.ny; iy++) {
            float sy, cy;
            sincospif(2.0f * __ldg(ky + iy) * v, &sy, &cy);
            const float dby = -tau * __ldg(ky + iy) * sy;
            for (int ix = 0; ix < f.nx; ix++) {
                float sx, cx;
                sincospif(2.0f * __ldg(kx + ix) * u, &sx, &cx);
                const float dbx = -tau * __ldg(kx + ix) * sx;
                const float4 c4 = __ldg(f.coef + ix + f.nx * (iy + f.ny * iz));
                const float c = c4.x * Q + c4.y * P + c4.z * L;
                E += c * cx * cy * bz;
                du += c * dbx * cy * bz;
                dv += c * cx * dby * bz;
                dz += c * cx * cy * dbz;
            }
        }
    }
    return make_float4(E, du, dv, dz);
}

// One LJ + damped-Coulomb pair (getLJQH, opencl/UFF.cl:82-95) at separation (dx, dy, dz) added to
// the force / energy of atom i.  qi.z carries the Coulomb constant (kCoulomb * Q_i, scaled once
// per atom by the caller).  Skipped pairs are evaluated at r^2 = 1 with zero well depth and
// charge product, so they add exactly 0.  fr = E0 u6 / r^2 (12 - 12 u6) - Ec / (r^2 + Rdamp^2).
__device__ __forceinline__ void ljq_pair(float dx, float dy, float dz, bool skip, float4 qi, float4 qj, float R2damp,
                                         float& fx, float& fy, float& fz, float& E) {
    float r2 = dx * dx + dy * dy + dz * dz;
    r2 = skip ? 1.0f : r2;
    const float R0 = qi.x + qj.x;
    const float E0 = skip ? 0.0f : qi.y * qj.y, Q = skip ? 0.0f : qi.z * qj.z;
    const float rs = rsqrtf(r2 + R2damp);            // 1/sqrt(r^2 + Rdamp^2)
    const float Ec = Q * rs;
    const float ir2 = 1.0f / r2;
    const float u2 = R0 * R0 * ir2, u6 = u2 * u2 * u2, vdW = u6 * E0;
    E += fmaf(u6 - 2.0f, vdW, Ec);
    const float fr = fmaf(vdW * ir2, fmaf(u6, -12.0f, 12.0f), -Ec * (rs * rs));
    fx = fmaf(dx, fr, fx); fy = fmaf(dy, fr, fy); fz = fmaf(dz, fr, fz);
}

// 1-3 exclusion (getNonBond_GridFF_Bspline_ex2, UFF.cl:1722-1930, with the lists of
// make_second_neighs, molff/src/nonbonded.rs:112-137): the partners of atom i excluded beyond its
// own bonds are its neighbours' neighbours.  They are read from the team's neighbour table in
// shared memory; entries may repeat or name i itself, which is excluded anyway.
struct Excl13 { short4 a, b, c, d; };

__device__ __forceinline__ short4 ng_or_none(const Smem& S, int g) {
    return g >= 0 ? S.Ng()[g] : make_short4(-1, -1, -1, -1);
}
__device__ __forceinline__ Excl13 excl13_of(const Smem& S, short4 ng) {
    return Excl13{ng_or_none(S, ng.x), ng_or_none(S, ng.y), ng_or_none(S, ng.z), ng_or_none(S, ng.w)};
}
__device__ __forceinline__ bool in4(int j, short4 v) { return (j == v.x) | (j == v.y) | (j == v.z) | (j == v.w); }
__device__ __forceinline__ bool is13(int j, const Excl13& e) { return in4(j, e.a) | in4(j, e.b) | in4(j, e.c) | in4(j, e.d); }
// the neighbours of atom g as bits of a 64-bit mask (systems of <= 64 atoms)
__device__ __forceinline__ unsigned long long ng_bits(const Smem& S, int g) {
    if (g < 0) return 0ull;
    const short4 n = S.Ng()[g];
    unsigned long long m = 0ull;
    if (n.x >= 0) m |= 1ull << (n.x & 63);
    if (n.y >= 0) m |= 1ull << (n.y & 63);
    if (n.z >= 0) m |= 1ull << (n.z & 63);
    if (n.w >= 0) m |= 1ull << (n.w & 63);
    return m;
}

// One pair of the team's atoms i, j (compensated positions); excluded pairs and, under a cutoff,
// pairs beyond it weigh 0.
template <bool CUT>
__device__ __forceinline__ void nb_pair(const KernelArgs& a, float4 pi, float4 li, float4 qi, float4 pj, float4 lj, float4 qj,
                                        bool excluded, float& fx, float& fy, float& fz, float& E) {
    const float dx = (pj.x - pi.x) + (lj.x - li.x), dy = (pj.y - pi.y) + (lj.y - li.y), dz = (pj.z - pi.z) + (lj.z - li.z);
    bool out = false;
    if (CUT) {
        const float r2 = dx * dx + dy * dy + dz * dz;
        out = r2 > a.rc2;
        // at the cutoff: decide in FP64, so FP32 rounding never moves a pair across it
        if (fabsf(r2 - a.rc2) < 1e-4f * a.rc2) out = beyond_cutoff_fp64(pi, li, pj, lj, a.rc2);
    }
    ljq_pair(dx, dy, dz, excluded || out, qi, qj, a.R2damp, fx, fy, fz, E);
}

// Four pairs of atom i (partners j[k], exclusion flags ex[k]) added in the order k = 0..3, as four
// nb_pair calls add them.  The FP64 cutoff decision is taken for the four behind one branch that
// is almost never taken: with a branch per pair the compiler keeps each pair's arithmetic in its
// own block and the pairs no longer overlap (measured: the per-pair form costs ~10 % of the step).
template <bool CUT>
__device__ __forceinline__ void nb_quad(const KernelArgs& a, const Smem& S, float4 pi, float4 li, float4 qi, const int j[4],
                                        const bool ex[4], float& fx, float& fy, float& fz, float& E) {
    float4 pj[4], lj[4], qj[4];
    float dx[4], dy[4], dz[4];
    bool out[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        pj[k] = S.P()[j[k]]; lj[k] = S.Lo()[j[k]]; qj[k] = S.Q()[j[k]];
        dx[k] = (pj[k].x - pi.x) + (lj[k].x - li.x);
        dy[k] = (pj[k].y - pi.y) + (lj[k].y - li.y);
        dz[k] = (pj[k].z - pi.z) + (lj[k].z - li.z);
        out[k] = false;
    }
    if (CUT) {
        float r2[4];
        bool band = false;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            r2[k] = dx[k] * dx[k] + dy[k] * dy[k] + dz[k] * dz[k];
            out[k] = r2[k] > a.rc2;
            band |= fabsf(r2[k] - a.rc2) < 1e-4f * a.rc2;
        }
        // at the cutoff: decide in FP64, so FP32 rounding never moves a pair across it
        if (band) {
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (fabsf(r2[k] - a.rc2) < 1e-4f * a.rc2) out[k] = beyond_cutoff_fp64(pi, li, pj[k], lj[k], a.rc2);
        }
    }
#pragma unroll
    for (int k = 0; k < 4; k++) ljq_pair(dx[k], dy[k], dz[k], ex[k] || out[k], qi, qj[k], a.R2damp, fx, fy, fz, E);
}

// ------------------------------------------------------------------ periodic systems
__device__ __forceinline__ int cell_f(int c, int k) { const int v = (c >> (4 * k)) & 15; return v >= 8 ? v - 16 : v; }

// Lattice shift of cell code c (4-bit offsets x | y << 4 | z << 8) for the lattice rows lat[0..2].
__device__ __forceinline__ float3 cell_shift(const float4* lat, int c) {
    const float4 A = __ldg(lat), B = __ldg(lat + 1), C = __ldg(lat + 2);
    const float ox = (float)cell_f(c, 0), oy = (float)cell_f(c, 1), oz = (float)cell_f(c, 2);
    return make_float3(ox * A.x + oy * B.x + oz * C.x, ox * A.y + oy * B.y + oz * C.y, ox * A.z + oy * B.z + oz * C.z);
}

// (pj + lj) - (pi + li) + s for a bond whose partner sits in another cell: the two coordinates
// differ by about a lattice vector, so the roundings of pj - pi and of adding s are recovered
// (TwoSum) and added back; the bond vector keeps the accuracy of an in-cell bond.
__device__ __forceinline__ float shifted_diff(float pj, float pi, float lj, float li, float s) {
    const float t = pj - pi, tb = t - pj, e1 = (pj - (t - tb)) + (-pi - tb);
    const float u = t + s, ub = u - t, e2 = (t - (u - ub)) + (s - ub);
    return u + ((e1 + e2) + (lj - li));
}

// Phase A for one atom of a system with periodic bonds: bond vectors (hneigh) and bond forces, a
// slot whose partner sits in another cell shifted by its lattice vector (UFF.cl:229-236).  Writes
// the atom's hneigh, force and bond energy; returns the bond energy.  Not inlined.
__device__ __forceinline__ float bonds_atom_pbc(Smem S, const float4* bk_, const float4* bl_, const short4* ngc_, const float4* lat, int i) {
    const float4 pi = S.P()[i], li = S.Lo()[i];
    const short4 ng = S.Ng()[i], gc = __ldg(ngc_ + i);
    const float4 bk = __ldg(bk_ + i), bl = __ldg(bl_ + i);
    float fx = 0.f, fy = 0.f, fz = 0.f, E = 0.f;
    for (int s = 0; s < 4; s++) {
        const int g = comp(ng, s);
        if (g < 0) { S.H()[s * S.n + i] = make_float4(0.f, 0.f, 0.f, 1e6f); continue; }
        const float4 pj = S.P()[g], lj = S.Lo()[g];
        const int cc = comp(gc, s);
        float dx, dy, dz;
        if (cc) {
            const float3 sh = cell_shift(lat, cc);
            dx = shifted_diff(pj.x, pi.x, lj.x, li.x, sh.x);
            dy = shifted_diff(pj.y, pi.y, lj.y, li.y, sh.y);
            dz = shifted_diff(pj.z, pi.z, lj.z, li.z, sh.z);
        } else {
            dx = (pj.x - pi.x) + (lj.x - li.x); dy = (pj.y - pi.y) + (lj.y - li.y); dz = (pj.z - pi.z) + (lj.z - li.z);
        }
        const float l2 = fmaxf(dx * dx + dy * dy + dz * dz, 1e-16f);
        const float l = sqrtf(l2), il = 1.0f / l;
        const float hx = dx * il, hy = dy * il, hz = dz * il;
        S.H()[s * S.n + i] = make_float4(hx, hy, hz, il);
        const float k = comp(bk, s), dl = l - comp(bl, s), fr = 2.0f * k * dl;
        fx += hx * fr; fy += hy * fr; fz += hz * fr;
        E += k * dl * dl;
    }
    S.F()[i] = make_float4(fx, fy, fz, E);
    S.Eh()[i] = E;
    return E;
}

// Position constraint of one atom (the constr / constrK springs of updateAtomsMMFFf4,
// opencl/UFF.cl:974-982): (target - position) * max(k, 0) when the atom has one.
__device__ __forceinline__ float3 constraint_force(const float4* cons, size_t g, float4 p, float4 lo) {
    const float4 c = __ldg(cons + 2 * g);
    if (!(c.w > 0.f)) return make_float3(0.f, 0.f, 0.f);
    const float4 k = __ldg(cons + 2 * g + 1);
    return make_float3(((c.x - p.x) - lo.x) * fmaxf(k.x, 0.f), ((c.y - p.y) - lo.y) * fmaxf(k.y, 0.f),
                       ((c.z - p.z) - lo.z) * fmaxf(k.z, 0.f));
}

// Pseudo-random vector of the Langevin drive of updateAtomsMMFFf4 (opencl/UFF.cl:982-991) for
// atom ia of its system: per component a byte of the 64-bit product (ia + c + (int)(m seed)) *
// 2654435761 >> 16, scaled to [0, 1), then sin((r + seed) * 124.4565).  The sum and product
// are rounded to FP32 as the kernel forms them; the sine is taken in FP64 and rounded, since
// the fast single-precision sine loses accuracy at these arguments (up to ~1e5 rad).
__device__ __noinline__ float3 langevin_noise(int ia, float seed) {
    const int c[3] = {136, 778, 4578};
    const float m[3] = {1000.f, 1013.f, 998.f};
    float out[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const long long x = (long long)(ia + c[k] + __float2int_rz(__fmul_rn(m[k], seed)));
        const float r = __fmul_rn((float)((x * 2654435761LL) >> 16 & 0xFF), 0.00390625f);
        const float arg = __fmul_rn(__fadd_rn(r, seed), 124.4565f);
        out[k] = (float)sin((double)arg);
    }
    return make_float3(out[0], out[1], out[2]);
}

constexpr double KB_EV = 8.617333262145e-5;        // eV/K, opencl/UFF.cl:52

// f += -gamma v + noise(ia, seed) amp, in the kernel's order (damping first)
__device__ __forceinline__ void add_langevin(float4& f, float4 v, int ia, float seed, float amp, float gamma) {
    const float3 r = langevin_noise(ia, seed);
    f.x = __fmaf_rn(r.x, amp, __fmaf_rn(v.x, -gamma, f.x));
    f.y = __fmaf_rn(r.y, amp, __fmaf_rn(v.y, -gamma, f.y));
    f.z = __fmaf_rn(r.z, amp, __fmaf_rn(v.z, -gamma, f.z));
}

// v + f dt with explicit roundings, so that both FIRE passes form the same velocity
__device__ __forceinline__ float4 kick(float4 v, float4 f, float dt) {
    return make_float4(__fmaf_rn(f.x, dt, v.x), __fmaf_rn(f.y, dt, v.y), __fmaf_rn(f.z, dt, v.z), v.w);
}

// beyond_cutoff_fp64 for a partner image shifted by s
__device__ __noinline__ bool beyond_cutoff_fp64_shift(float4 pi, float4 li, float4 pj, float4 lj, float sx, float sy, float sz, float rc2) {
    const double dx = ((double)pj.x - (double)pi.x) + ((double)lj.x - (double)li.x) + (double)sx;
    const double dy = ((double)pj.y - (double)pi.y) + ((double)lj.y - (double)li.y) + (double)sy;
    const double dz = ((double)pj.z - (double)pi.z) + ((double)lj.z - (double)li.z) + (double)sz;
    return dx * dx + dy * dy + dz * dz > (double)rc2;
}

// NB sum of atom i over the partners j = c, c + L, ... < N in every image of the system's
// (2 nx + 1)(2 ny + 1)(2 nz + 1) block (getNonBond_GridFF_Bspline with PBC, opencl/UFF.cl:1592-1650):
// an atom never meets its own images, a bonded pair is excluded only in the image of its bond
// (neighbour index and cell code both match).  Returns (F, E) of atom i.  Not inlined: the
// kernels' other phases keep their registers.
__device__ __forceinline__ float4 nb_atom_images(Smem S, float rc2, float R2damp, const float4* lat, int N, int i, int c,
                                              int L, short4 ng, short4 gc) {
    const float4 A = __ldg(lat), B = __ldg(lat + 1), C = __ldg(lat + 2);
    const int nx = (int)A.w, ny = (int)B.w, nz = (int)C.w;
    const bool cut = rc2 < 1e37f;
    const float4 pi = S.P()[i], li = S.Lo()[i];
    float4 qi = S.Q()[i];
    qi.z *= kCoulomb;                                 // ljq_pair takes kCoulomb * Q_i
    float fx = 0.f, fy = 0.f, fz = 0.f, E = 0.f;
    for (int j = c; j < N; j += L) {
        if (j == i) continue;
        const float4 pj = S.P()[j], lj = S.Lo()[j], qj = S.Q()[j];
        const float dx0 = (pj.x - pi.x) + (lj.x - li.x), dy0 = (pj.y - pi.y) + (lj.y - li.y), dz0 = (pj.z - pi.z) + (lj.z - li.z);
        for (int iz = -nz; iz <= nz; iz++)
            for (int iy = -ny; iy <= ny; iy++)
                for (int ix = -nx; ix <= nx; ix++) {
                    const int code = (ix & 15) | ((iy & 15) << 4) | ((iz & 15) << 8);
                    const bool bonded = (j == ng.x && code == gc.x) || (j == ng.y && code == gc.y) ||
                                        (j == ng.z && code == gc.z) || (j == ng.w && code == gc.w);
                    const float fxi = (float)ix, fyi = (float)iy, fzi = (float)iz;
                    const float sx = fxi * A.x + fyi * B.x + fzi * C.x, sy = fxi * A.y + fyi * B.y + fzi * C.y,
                                sz = fxi * A.z + fyi * B.z + fzi * C.z;
                    const float dx = dx0 + sx, dy = dy0 + sy, dz = dz0 + sz;
                    bool out = false;
                    if (cut) {
                        const float r2 = dx * dx + dy * dy + dz * dz;
                        out = r2 > rc2;
                        if (fabsf(r2 - rc2) < 1e-4f * rc2) out = beyond_cutoff_fp64_shift(pi, li, pj, lj, sx, sy, sz, rc2);
                    }
                    ljq_pair(dx, dy, dz, bonded || out, qi, qj, R2damp, fx, fy, fz, E);
                }
    }
    return make_float4(fx, fy, fz, E);
}

// lanes per atom for the NB partner loop: minimise passes x (partners per lane + the shuffle
// reduction, ~4 pair-equivalents per halving).  On B200 this picks 2 lanes for 40 atoms in a
// warp (measured 3 % faster than 4, 7 % faster than 1 or 8).
__device__ __forceinline__ int nb_lanes(int N, int T) {
    int best = 1; long long bc = 1LL << 60;
    int lg = 0;
    for (int L = 1; L <= 32; L <<= 1, lg++) {
        int G = T / L;
        if (G < 1) break;
        long long cost = (long long)((N + G - 1) / G) * ((N + L - 1) / L + 4 * lg);
        if (cost < bc) { bc = cost; best = L; }
    }
    return best;
}


// ------------------------------------------------------------------ bonded terms (opencl/UFF.cl:326-795)
// Each returns the force on every atom of the term and the term energy.
__device__ __forceinline__ float angle_term(const Smem& S, short4 sl, float4 p, float3& fpi, float3& fpj, float3& fpk) {
    const float4 qij = S.hget(sl.x), qkj = S.hget(sl.y);
    const float hx = qij.x + qkj.x, hy = qij.y + qkj.y, hz = qij.z + qkj.z;
    float c = 0.5f * (hx * hx + hy * hy + hz * hz - 2.0f);
    c = fminf(fmaxf(c, -1.0f), 1.0f);
    const float s = sqrtf(fmaxf(0.0f, 1.0f - c * c) + 1e-14f);
    const float is = (s > 1e-12f) ? 1.0f / s : 0.0f;
    const float c2x = c * c - s * s, c2y = c * s + s * c;
    const float c3x = c2x * c - c2y * s, c3y = c2x * s + c2y * c;
    // p = K*(c0, c1, c2, c3); the energy omits the c1 term, the force keeps it
    const float E = p.x + p.z * c2x + p.w * c3x;
    const float fm = p.y + p.z * c2y * is * 2.0f + p.w * c3y * is * 3.0f;
    const float fi = fm * qij.w, fk = fm * qkj.w, fic = fi * c, fkc = fk * c;
    fpi = make_float3(fic * qij.x - fi * qkj.x, fic * qij.y - fi * qkj.y, fic * qij.z - fi * qkj.z);
    fpk = make_float3(-fk * qij.x + fkc * qkj.x, -fk * qij.y + fkc * qkj.y, -fk * qij.z + fkc * qkj.z);
    fpj = make_float3((fk - fic) * qij.x + (fi - fkc) * qkj.x, (fk - fic) * qij.y + (fi - fkc) * qkj.y,
                      (fk - fic) * qij.z + (fi - fkc) * qkj.z);
    return E;
}

__device__ __forceinline__ float dihedral_term(const Smem& S, short4 sl, float4 p, float3& f1, float3& f2, float3& f3, float3& f4) {
    const float4 q12 = S.hget(sl.x), q32 = S.hget(sl.y), q43 = S.hget(sl.z);
    const float3 n123 = make_float3(q12.y * q32.z - q12.z * q32.y, q12.z * q32.x - q12.x * q32.z, q12.x * q32.y - q12.y * q32.x);
    const float3 n234 = make_float3(q43.y * q32.z - q43.z * q32.y, q43.z * q32.x - q43.x * q32.z, q43.x * q32.y - q43.y * q32.x);
    const float a2 = n123.x * n123.x + n123.y * n123.y + n123.z * n123.z;
    const float b2 = n234.x * n234.x + n234.y * n234.y + n234.z * n234.z;
    f1 = f2 = f3 = f4 = make_float3(0.f, 0.f, 0.f);
    if (a2 < 1e-30f || b2 < 1e-30f) return 0.f;
    const float il2a = 1.0f / a2, il2b = 1.0f / b2, inv = sqrtf(il2a * il2b);
    const float cx = (n123.x * n234.x + n123.y * n234.y + n123.z * n234.z) * inv;
    const float cy = -(n123.x * q43.x + n123.y * q43.y + n123.z * q43.z) * inv;
    float nx = cx, ny = cy;
    const int nn = (int)p.z;
    for (int k = 1; k < nn; k++) { const float t = nx * cx - ny * cy; ny = nx * cy + ny * cx; nx = t; }
    const float E = p.x * (1.0f + p.y * nx);
    const float f = -p.x * p.y * p.z * ny;
    const float s1 = -f * il2a * q12.w, s4 = f * il2b * q43.w;
    f1 = make_float3(n123.x * s1, n123.y * s1, n123.z * s1);
    f4 = make_float3(n234.x * s4, n234.y * s4, n234.z * s4);
    const float c123 = (q32.x * q12.x + q32.y * q12.y + q32.z * q12.z) * (q32.w / q12.w);
    const float c432 = (q32.x * q43.x + q32.y * q43.y + q32.z * q43.z) * (q32.w / q43.w);
    f3 = make_float3(-c123 * f1.x + (-c432 - 1.0f) * f4.x, -c123 * f1.y + (-c432 - 1.0f) * f4.y, -c123 * f1.z + (-c432 - 1.0f) * f4.z);
    f2 = make_float3((c123 - 1.0f) * f1.x + c432 * f4.x, (c123 - 1.0f) * f1.y + c432 * f4.y, (c123 - 1.0f) * f1.z + c432 * f4.z);
    return E;
}

__device__ __forceinline__ float inversion_term(const Smem& S, short4 sl, float4 p, float3& f1, float3& f2, float3& f3, float3& f4) {
    const float4 q21 = S.hget(sl.x), q31 = S.hget(sl.y), q41 = S.hget(sl.z);
    float3 n = make_float3(q21.y * q31.z - q21.z * q31.y, q21.z * q31.x - q21.x * q31.z, q21.x * q31.y - q21.y * q31.x);
    const float nn = n.x * n.x + n.y * n.y + n.z * n.z;
    float il = 0.0f;
    if (nn > 1e-16f) { il = rsqrtf(nn); n.x *= il; n.y *= il; n.z *= il; }
    else n = make_float3(0.f, 0.f, 0.f);
    float sw = -(n.x * q41.x + n.y * q41.y + n.z * q41.z);
    sw = fminf(fmaxf(sw, -1.0f), 1.0f);
    const float cw = sqrtf(1.0f - sw * sw);
    // p = (K, c0, c1, c2)
    const float E = p.x * (p.y + p.z * cw + p.w * (2.0f * cw * cw - 1.0f));
    const float dEdw = -p.x * (p.z * sw + 2.0f * p.w * (2.0f * sw * cw));
    const float ft = (cw > 1e-7f) ? dEdw / cw : 0.0f;
    const float fq41 = ft * q41.w, fi123 = ft * il;
    const float3 tq = make_float3(sw * fi123 * n.x + fi123 * q41.x, sw * fi123 * n.y + fi123 * q41.y, sw * fi123 * n.z + fi123 * q41.z);
    f4 = make_float3(fq41 * n.x + sw * fq41 * q41.x, fq41 * n.y + sw * fq41 * q41.y, fq41 * n.z + sw * fq41 * q41.z);
    f2 = make_float3((q31.y * tq.z - q31.z * tq.y) * q21.w, (q31.z * tq.x - q31.x * tq.z) * q21.w, (q31.x * tq.y - q31.y * tq.x) * q21.w);
    f3 = make_float3((tq.y * q21.z - tq.z * q21.y) * q31.w, (tq.z * q21.x - tq.x * q21.z) * q31.w, (tq.x * q21.y - tq.y * q21.x) * q31.w);
    f1 = make_float3(-(f2.x + f3.x + f4.x), -(f2.y + f3.y + f4.y), -(f2.z + f3.z + f4.z));
    return E;
}

__device__ __forceinline__ void addf(float4& a, const float3& f, float e) { a.x += f.x; a.y += f.y; a.z += f.z; a.w += e; }

// owner form: add a piece to the accumulator of bond slot s (a select chain, no local memory)
__device__ __forceinline__ void slot_add(float4& s0, float4& s1, float4& s2, float4& s3, int s, const float3& f, float e) {
    if (s == 0) addf(s0, f, e);
    else if (s == 1) addf(s1, f, e);
    else if (s == 2) addf(s2, f, e);
    else addf(s3, f, e);
}

// Energy accumulators of the evaluation-only launch (bond, angle, dihedral, inversion, NB, grid).
template <bool EVAL> struct EAcc { __device__ void add(int, double) {} };
template <> struct EAcc<true> {
    double e[6] = {0, 0, 0, 0, 0, 0};
    __device__ void add(int k, double v) { e[k] += v; }
};

// ------------------------------------------------------------------ force evaluation
template <int T, int GDT, bool EVAL, int FORM>
__device__ void eval_forces(const KernelArgs& a, const Smem& S, const TopoDev* __restrict__ tpp, int N, int rank, EAcc<EVAL>& acc,
                            const float4* lat, bool use_list = false, size_t ga0 = 0) {
#define TP(f) __ldg(&tpp->f)
    // periodic systems (lat: the slot's lattice rows) run in FORM_GATHER_EXT, the gather form plus
    // bonds to a partner's image in another cell (neighCell, UFF.cl:229-236) and NB image sums
    constexpr bool PBC = FORM == FORM_GATHER_EXT;
    constexpr int BF = PBC ? FORM_GATHER : FORM;
    const bool pbc_bonds = PBC && lat != nullptr && TP(pbc_bonds) != 0;
    // Grid lines into L2 ahead of phase D: positions do not change within a step, so the brick
    // lines of every atom's stencil are requested now and arrive while phases A-C run
    if (a.grid_prefetch && a.grid.brick && a.has_grid && !a.fold.on) grid_prefetch_l2<T, GDT>(a.grid, S, N, rank);
    // A: bonds and hneigh, one atom per rank (opencl/UFF.cl:141-322)
    if (pbc_bonds) {
        for (int i = rank; i < N; i += T) {
            const float E = bonds_atom_pbc(S, a.bk + TP(atom_off), a.bl + TP(atom_off), a.neighc + TP(atom_off), lat, i);
            acc.add(0, 0.5 * (double)E);
        }
    } else {
        for (int i = rank; i < N; i += T) {
            const float4 pi = S.P()[i], li = S.Lo()[i];
            const short4 ng = S.Ng()[i];
            const float4 bk = __ldg(a.bk + TP(atom_off) + i), bl = __ldg(a.bl + TP(atom_off) + i);
            float fx = 0.f, fy = 0.f, fz = 0.f, E = 0.f;
    #pragma unroll
            for (int s = 0; s < 4; s++) {
                const int g = comp(ng, s);
                if (g < 0) { S.H()[s * S.n + i] = make_float4(0.f, 0.f, 0.f, 1e6f); continue; }
                const float4 pj = S.P()[g], lj = S.Lo()[g];
                // difference of the compensated positions: its error is relative to the bond length,
                // not to the absolute coordinate (float positions alone would put ~1e-6 A of rounding
                // into every stiff bond and make the force field rough at the 1e-4 eV/A level)
                const float dx = (pj.x - pi.x) + (lj.x - li.x), dy = (pj.y - pi.y) + (lj.y - li.y), dz = (pj.z - pi.z) + (lj.z - li.z);
                const float l2 = fmaxf(dx * dx + dy * dy + dz * dz, 1e-16f);
                const float l = sqrtf(l2), il = 1.0f / l;
                const float hx = dx * il, hy = dy * il, hz = dz * il;
                S.H()[s * S.n + i] = make_float4(hx, hy, hz, il);
                const float k = comp(bk, s), dl = l - comp(bl, s), fr = 2.0f * k * dl;
                fx += hx * fr; fy += hy * fr; fz += hz * fr;
                E += k * dl * dl;
            }
            S.F()[i] = make_float4(fx, fy, fz, E);
            S.Eh()[i] = E;
            acc.add(0, 0.5 * (double)E);
        }
    }
    team_sync<T>();

    if (BF == FORM_ROUNDS) {
        // B (rounds): in one round the atoms of each role are distinct, so each role's pieces
        // are added with plain read-modify-writes separated by team syncs
        for (int r = 0; r < TP(ang_rounds); r++) {
            const AngRec rec = load_rec(a.angs + TP(ang_off) + (size_t)r * T + rank);
            const bool ok = rec.at.x >= 0;
            float3 f1, f2, f3;
            float E = 0.f;
            if (ok) { E = angle_term(S, rec.sl, rec.p, f1, f2, f3); acc.add(1, (double)E); }
            const float e3 = E / 3.0f;
            if (ok) addf(S.F()[rec.at.x], f1, e3);
            team_sync<T>();
            if (ok) addf(S.F()[rec.at.y], f2, e3);
            team_sync<T>();
            if (ok) addf(S.F()[rec.at.z], f3, e3);
            team_sync<T>();
        }
        for (int r = 0; r < TP(dih_rounds); r++) {
            const DihRec rec = load_rec(a.dihs + TP(dih_off) + (size_t)r * T + rank);
            const bool ok = rec.at.x >= 0;
            float3 f1, f2, f3, f4;
            float E = 0.f;
            if (ok) { E = dihedral_term(S, rec.sl, rec.p, f1, f2, f3, f4); acc.add(2, (double)E); }
            const float e4 = 0.25f * E;
            if (ok) addf(S.F()[rec.at.x], f1, e4);
            team_sync<T>();
            if (ok) addf(S.F()[rec.at.y], f2, e4);
            team_sync<T>();
            if (ok) addf(S.F()[rec.at.z], f3, e4);
            team_sync<T>();
            if (ok) addf(S.F()[rec.at.w], f4, e4);
            team_sync<T>();
        }
        for (int r = 0; r < TP(inv_rounds); r++) {
            const InvRec rec = load_rec(a.invs + TP(inv_off) + (size_t)r * T + rank);
            const bool ok = rec.at.x >= 0;
            float3 f1, f2, f3, f4;
            float E = 0.f;
            if (ok) { E = inversion_term(S, rec.sl, rec.p, f1, f2, f3, f4); acc.add(3, (double)E); }
            const float e4 = 0.25f * E;
            if (ok) addf(S.F()[rec.at.x], f1, e4);
            team_sync<T>();
            if (ok) addf(S.F()[rec.at.y], f2, e4);
            team_sync<T>();
            if (ok) addf(S.F()[rec.at.z], f3, e4);
            team_sync<T>();
            if (ok) addf(S.F()[rec.at.w], f4, e4);
            team_sync<T>();
        }
    } else if (BF == FORM_OWNER) {
        // B (owner): lane o evaluates the terms atom o owns and keeps every piece in registers: its
        // own, and those of its neighbours by bond slot (angles: apex j, pieces on i and k;
        // inversions: centre i, pieces on j, k, l; a dihedral i-j-k-l once at j, keeping the
        // pieces of j and i, and once at k, keeping those of k and l).  Records of one kind are
        // read row by row, a warp's lanes reading consecutive records.
        const int abase = TP(atom_off);
        for (int o0 = 0; o0 < N; o0 += T) {
            const int o = o0 + rank;
            const int meta = o < N ? __ldg(a.own_meta + abase + o) : 0;
            float4 fo = make_float4(0.f, 0.f, 0.f, 0.f), s0 = fo, s1 = fo, s2 = fo, s3 = fo;
            {
                const int cnt = meta & 255, m = __reduce_max_sync(FULL, cnt);
                const int off = TP(own_a_off) + o;
                for (int r = 0; r < m; r++) {
                    if (r < cnt) {
                        const short4 g = __ldg(a.own_geo + off + r * N);
                        const float4 p = __ldg(a.own_par + off + r * N);
                        float3 f1, f2, f3;
                        const float E = angle_term(S, g, p, f1, f2, f3);
                        acc.add(1, (double)E);
                        const float e3 = E / 3.0f;
                        addf(fo, f2, e3);
                        slot_add(s0, s1, s2, s3, g.x & 3, f1, e3);
                        slot_add(s0, s1, s2, s3, g.y & 3, f3, e3);
                    }
                }
            }
            {
                const int cnt = (meta >> 8) & 255, m = __reduce_max_sync(FULL, cnt);
                const int off = TP(own_i_off) + o;
                for (int r = 0; r < m; r++) {
                    if (r < cnt) {
                        const short4 g = __ldg(a.own_geo + off + r * N);
                        const float4 p = __ldg(a.own_par + off + r * N);
                        float3 f1, f2, f3, f4;
                        const float E = inversion_term(S, g, p, f1, f2, f3, f4);
                        acc.add(3, (double)E);
                        const float e4 = 0.25f * E;
                        addf(fo, f1, e4);
                        slot_add(s0, s1, s2, s3, g.x & 3, f2, e4);
                        slot_add(s0, s1, s2, s3, g.y & 3, f3, e4);
                        slot_add(s0, s1, s2, s3, g.z & 3, f4, e4);
                    }
                }
            }
            {
                const int cnt = (meta >> 16) & 255, m = __reduce_max_sync(FULL, cnt);
                const int off = TP(own_d_off) + o;
                for (int r = 0; r < m; r++) {
                    if (r < cnt) {
                        const short4 g = __ldg(a.own_geo + off + r * N);
                        const float4 p = __ldg(a.own_par + off + r * N);
                        float3 f1, f2, f3, f4;
                        const float E = dihedral_term(S, g, p, f1, f2, f3, f4);
                        acc.add(2, 0.5 * (double)E);
                        const float e4 = 0.25f * E;
                        const bool at_k = g.w != 0;          // this record is the k half
                        addf(fo, at_k ? f3 : f2, e4);
                        slot_add(s0, s1, s2, s3, at_k ? (g.z & 3) : (g.x & 3), at_k ? f4 : f1, e4);
                    }
                }
            }
            if (o < N) {
                add4(S.F()[o], fo.x, fo.y, fo.z, fo.w);
                float4* Fs = S.Fs(T);
                Fs[o] = s0; Fs[S.n + o] = s1; Fs[2 * S.n + o] = s2; Fs[3 * S.n + o] = s3;
            }
        }
        team_sync<T>();
        // assembly: atom i adds the piece each neighbour g holds for it, in slot order
        for (int i = rank; i < N; i += T) {
            const short4 ng = S.Ng()[i];
            const int meta = __ldg(a.own_meta + abase + i);
            float4 f = S.F()[i];
#pragma unroll
            for (int s = 0; s < 4; s++) {
                const int g = comp(ng, s);
                if (g >= 0) {
                    const int b = (meta >> (24 + 2 * s)) & 3;
                    const float4 v = S.Fs(T)[b * S.n + g];
                    f.x += v.x; f.y += v.y; f.z += v.z; f.w += v.w;
                }
            }
            S.F()[i] = f;
        }
        team_sync<T>();
    } else {
        // B (gather): all terms at once, each writing its pieces to its own slots (the reference's
        // fint array, opencl/UFF.cl:801-880), then every atom sums its pieces in a fixed order
        const int na = TP(nang), nd = TP(ndih), ni = TP(ninv);
        for (int t = rank; t < na + nd + ni; t += T) {
            float3 f1, f2, f3, f4;
            if (t < na) {
                const AngRec rec = load_rec(a.angs + TP(fang_off) + t);
                const float E = angle_term(S, rec.sl, rec.p, f1, f2, f3);
                acc.add(1, (double)E);
                const float e3 = E / 3.0f;
                float4* P = S.Pc(T) + 3 * t;
                P[0] = make_float4(f1.x, f1.y, f1.z, e3); P[1] = make_float4(f2.x, f2.y, f2.z, e3); P[2] = make_float4(f3.x, f3.y, f3.z, e3);
            } else if (t < na + nd) {
                const int u = t - na;
                const DihRec rec = load_rec(a.dihs + TP(fdih_off) + u);
                const float E = dihedral_term(S, rec.sl, rec.p, f1, f2, f3, f4);
                acc.add(2, (double)E);
                const float e4 = 0.25f * E;
                float4* P = S.Pc(T) + 3 * na + 4 * u;
                P[0] = make_float4(f1.x, f1.y, f1.z, e4); P[1] = make_float4(f2.x, f2.y, f2.z, e4);
                P[2] = make_float4(f3.x, f3.y, f3.z, e4); P[3] = make_float4(f4.x, f4.y, f4.z, e4);
            } else {
                const int u = t - na - nd;
                const InvRec rec = load_rec(a.invs + TP(finv_off) + u);
                const float E = inversion_term(S, rec.sl, rec.p, f1, f2, f3, f4);
                acc.add(3, (double)E);
                const float e4 = 0.25f * E;
                float4* P = S.Pc(T) + 3 * na + 4 * nd + 4 * u;
                P[0] = make_float4(f1.x, f1.y, f1.z, e4); P[1] = make_float4(f2.x, f2.y, f2.z, e4);
                P[2] = make_float4(f3.x, f3.y, f3.z, e4); P[3] = make_float4(f4.x, f4.y, f4.z, e4);
            }
        }
        team_sync<T>();
        const int c = rank & 3;
        for (int i0 = 0; i0 < N; i0 += T / 4) {
            const int i = i0 + (rank >> 2);
            float4 s4 = make_float4(0.f, 0.f, 0.f, 0.f);
            if (i < N) {
                const int2 se = __ldg(a.a2f + TP(atom_off) + i);
                for (int k = c; k < se.y; k += 4) {
                    const float4 v = S.Pc(T)[__ldg(a.a2f_idx + TP(a2f_off) + se.x + k)];
                    s4.x += v.x; s4.y += v.y; s4.z += v.z; s4.w += v.w;
                }
            }
            for (int o = 1; o < 4; o <<= 1) {
                s4.x += __shfl_xor_sync(FULL, s4.x, o); s4.y += __shfl_xor_sync(FULL, s4.y, o);
                s4.z += __shfl_xor_sync(FULL, s4.z, o); s4.w += __shfl_xor_sync(FULL, s4.w, o);
            }
            if (c == 0 && i < N) add4(S.F()[i], s4.x, s4.y, s4.z, s4.w);
        }
        team_sync<T>();
    }

    // C: intramolecular LJ + damped Coulomb over all pairs except bonded (1-2) neighbours
    // (opencl/UFF.cl:57-95, 1595-1665), or except 1-2 and 1-3 pairs with excl13 (UFF.cl:1722-1930).  Excluded pairs are evaluated at r2 = 1 and masked out,
    // so the partner loop has no branch and independent pairs overlap.
    {
        // with a neighbour list the partner count, not N, sets the lanes per atom
        const int Neff = use_list ? min(N, 160) : N;
        const int L = a.nb_lanes > 0 ? min(a.nb_lanes, min(T, 32)) : nb_lanes(Neff, T), G = T / L;
        const int c = rank & (L - 1);
        const bool small = N <= 64;
        // PBC images: uniform per system
        const bool images = PBC && lat != nullptr && __ldg(&lat[0].w) + __ldg(&lat[1].w) + __ldg(&lat[2].w) > 0.f;
        // the partner loop with the cutoff logic compiled in or out (uniform per launch)
        auto nb_atoms = [&](auto cut_tag) {
        constexpr bool CUT = decltype(cut_tag)::value;
        for (int i0 = 0; i0 < N; i0 += G) {
            // the last, partial pass spreads its atoms over all the team's lanes (uniform per team)
            int Lp = L;
            if (N - i0 < G) while (Lp < 32 && Lp * 2 * (N - i0) <= T) Lp <<= 1;
            const int i = i0 + rank / Lp, cp = rank & (Lp - 1);
            float fx = 0.f, fy = 0.f, fz = 0.f, E = 0.f;
            if (i < N) {
                const float4 pi = S.P()[i], li = S.Lo()[i];
                float4 qi = S.Q()[i];
                qi.z *= kCoulomb;                     // ljq_pair takes kCoulomb * Q_i
                const int cnt = use_list ? a.nbl_cnt[ga0 + i] : -1;
                if (cnt >= 0) {
                    // partners within rc + skin; exclusions were removed at the build.  Lane cp takes
                    // runs of 4 entries, one 8-byte load each (rows start on 512-byte boundaries);
                    // entries outside a run's count weigh 0 and index the atom itself, so a stale
                    // slot of the row is never dereferenced.  Inner partners (front of the row)
                    // stay inside the cutoff until the next rebuild: no cutoff test.  Shell partners
                    // (back of the row) take the full test.
                    const ushort4* row4 = reinterpret_cast<const ushort4*>(a.nbl + (ga0 + i) * (size_t)a.nbl_cap);
                    const int nin = cnt & 0xffff, nsh = cnt >> 16;
                    auto run4 = [&](int e, int lo, int hi, auto cut_run) {
                        const ushort4 v = row4[e >> 2];
                        const bool ok0 = e >= lo && e < hi, ok1 = e + 1 >= lo && e + 1 < hi;
                        const bool ok2 = e + 2 >= lo && e + 2 < hi, ok3 = e + 3 >= lo && e + 3 < hi;
                        const int jq[4] = {ok0 ? (int)v.x : i, ok1 ? (int)v.y : i, ok2 ? (int)v.z : i, ok3 ? (int)v.w : i};
                        const bool xq[4] = {!ok0, !ok1, !ok2, !ok3};
                        constexpr bool C = decltype(cut_run)::value;
                        if (T == 32) {
                            // warp teams (72 registers): pair by pair, the grouped form spills
#pragma unroll
                            for (int k = 0; k < 4; k++)
                                nb_pair<C>(a, pi, li, qi, S.P()[jq[k]], S.Lo()[jq[k]], S.Q()[jq[k]], xq[k], fx, fy, fz, E);
                        } else {
                            nb_quad<C>(a, S, pi, li, qi, jq, xq, fx, fy, fz, E);
                        }
                    };
#pragma unroll 2
                    for (int e = cp * 4; e < nin; e += Lp * 4) run4(e, 0, nin, std::integral_constant<bool, false>{});
                    const int s0 = (a.nbl_cap - nsh) & ~3;
                    for (int e = s0 + cp * 4; e < a.nbl_cap; e += Lp * 4) run4(e, a.nbl_cap - nsh, a.nbl_cap, std::integral_constant<bool, CUT>{});
                } else {
                    const short4 ng = S.Ng()[i];
                    unsigned long long ex = 1ull << (i & 63);
                    if (ng.x >= 0) ex |= 1ull << (ng.x & 63);
                    if (ng.y >= 0) ex |= 1ull << (ng.y & 63);
                    if (ng.z >= 0) ex |= 1ull << (ng.z & 63);
                    if (ng.w >= 0) ex |= 1ull << (ng.w & 63);
                    // 1-3 exclusion is compiled into the extended form only (the host runs every
                    // system in that form while it is on), so the other forms keep their registers
                    if (FORM == FORM_GATHER_EXT && a.excl13) {
                        if (small) {
                            ex |= ng_bits(S, ng.x) | ng_bits(S, ng.y) | ng_bits(S, ng.z) | ng_bits(S, ng.w);
                            for (int j = cp; j < N; j += Lp)
                                nb_pair<CUT>(a, pi, li, qi, S.P()[j], S.Lo()[j], S.Q()[j], (bool)((ex >> j) & 1ull), fx, fy, fz, E);
                        } else {
                            const Excl13 e13 = excl13_of(S, ng);
#pragma unroll 2
                            for (int j = cp; j < N; j += Lp) {
                                const bool excl = (j == i) | in4(j, ng) | is13(j, e13);
                                nb_pair<CUT>(a, pi, li, qi, S.P()[j], S.Lo()[j], S.Q()[j], excl, fx, fy, fz, E);
                            }
                        }
                    } else {
                        if (T == 32) {
                            // warp teams (72 registers): pair by pair, the grouped form spills
#pragma unroll 4
                            for (int j = cp; j < N; j += Lp) {
                                const bool excl = small ? (bool)((ex >> j) & 1ull) : (j == i || j == ng.x || j == ng.y || j == ng.z || j == ng.w);
                                nb_pair<CUT>(a, pi, li, qi, S.P()[j], S.Lo()[j], S.Q()[j], excl, fx, fy, fz, E);
                            }
                        } else
                        // partners j = cp, cp + Lp, ... in groups of four; slots past N take the atom
                        // itself, excluded (they add exactly 0)
                        for (int j0 = cp; j0 < N; j0 += 4 * Lp) {
                            int jq[4];
                            bool xq[4];
#pragma unroll
                            for (int k = 0; k < 4; k++) {
                                const int j = j0 + k * Lp;
                                const bool in = j < N;
                                jq[k] = in ? j : i;
                                xq[k] = !in || (small ? (bool)((ex >> j) & 1ull) : (j == i || j == ng.x || j == ng.y || j == ng.z || j == ng.w));
                            }
                            nb_quad<CUT>(a, S, pi, li, qi, jq, xq, fx, fy, fz, E);
                        }
                    }
                }
            }
            for (int o = 1; o < Lp; o <<= 1) {
                fx += __shfl_xor_sync(FULL, fx, o); fy += __shfl_xor_sync(FULL, fy, o);
                fz += __shfl_xor_sync(FULL, fz, o); E += __shfl_xor_sync(FULL, E, o);
            }
            if (cp == 0 && i < N) {
                add4(S.F()[i], fx, fy, fz, E);
                S.Eh()[i] += E;
                acc.add(4, 0.5 * (double)E);
            }
        }
        };
        if (images) {
            // periodic system: the same lanes-per-atom split over the image sums
            for (int i0 = 0; i0 < N; i0 += G) {
                const int i = i0 + rank / L;
                float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
                if (i < N) r = nb_atom_images(S, a.rc2, a.R2damp, lat, N, i, c, L, S.Ng()[i], __ldg(a.neighc + TP(atom_off) + i));
                for (int o = 1; o < L; o <<= 1) {
                    r.x += __shfl_xor_sync(FULL, r.x, o); r.y += __shfl_xor_sync(FULL, r.y, o);
                    r.z += __shfl_xor_sync(FULL, r.z, o); r.w += __shfl_xor_sync(FULL, r.w, o);
                }
                if (c == 0 && i < N) {
                    add4(S.F()[i], r.x, r.y, r.z, r.w);
                    S.Eh()[i] += r.w;
                    acc.add(4, 0.5 * (double)r.w);
                }
            }
        }
        else if (a.rc2 < 1e37f) nb_atoms(std::integral_constant<bool, true>{});
        else nb_atoms(std::integral_constant<bool, false>{});
    }
    team_sync<T>();

    // D': folded surface instead of the grid, 4 lanes per atom splitting the z-decay terms
    if (a.fold.on) {
        const FoldedView& f = a.fold;
        const int lane = rank & 3;
        for (int i0 = 0; i0 < N; i0 += T / 4) {
            const int i = i0 + (rank >> 2);
            float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
            if (i < N) r = folded_part(f, S.P()[i], S.Lo()[i], S.Q()[i], lane);
            for (int o = 1; o < 4; o <<= 1) {
                r.x += __shfl_xor_sync(FULL, r.x, o); r.y += __shfl_xor_sync(FULL, r.y, o);
                r.z += __shfl_xor_sync(FULL, r.z, o); r.w += __shfl_xor_sync(FULL, r.w, o);
            }
            if (lane == 0 && i < N) {
                float fx = -(r.y * f.inv[0] + r.z * f.inv[1]), fy = -(r.y * f.inv[2] + r.z * f.inv[3]), fz = -r.w;
                const float f2 = fx * fx + fy * fy + fz * fz;
                if (f2 > f.fmax * f.fmax) { const float sc = f.fmax / sqrtf(f2); fx *= sc; fy *= sc; fz *= sc; }   // eval_all_clamped
                add4(S.F()[i], fx, fy, fz, r.x);
                acc.add(5, (double)r.x);
            }
        }
    }
    // D: substrate grid, 4 lanes per atom; lane kz reads the voxels at z offset kz of the 16 (x, y)
    // columns of the stencil, so the 4 lanes of an atom read each column as one 64 B run
    else if (a.has_grid) {
        const GridView& g = a.grid;
        const int kz = rank & 3;
        for (int i0 = 0; i0 < N; i0 += T / 4) {
            const int i = i0 + (rank >> 2);
            float e = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
            if (i < N) {
                const float4 p = S.P()[i], lp = S.Lo()[i];
                const float ux = ((p.x - g.p0[0]) + lp.x) * g.inv_step[0];
                const float uy = ((p.y - g.p0[1]) + lp.y) * g.inv_step[1];
                const float uz = ((p.z - g.p0[2]) + lp.z) * g.inv_step[2];
                int ix = (int)ux, iy = (int)uy;
                int iz = (int)uz;
                if (ux < 0) ix--;
                if (uy < 0) iy--;
                // the substrate force vanishes outside planes [1, nz-2) (UFF.cl): near those two
                // bounds the cell is decided in FP64, as the CPU evaluators decide it
                if (fabsf(uz - 1.0f) < 1e-3f || fabsf(uz - (float)(g.nz - 2)) < 1e-3f) iz = grid_cell_z_fp64(p.z, lp.z, g);
                if (iz >= 1 && iz < g.nz - 2) {
                    const float tx = ux - ix, ty = uy - iy, tz = uz - iz;
                    float bx[4], dxw[4], by[4], dyw[4], bz[4], dzw[4];
                    bspline(tx, bx, dxw); bspline(ty, by, dyw); bspline(tz, bz, dzw);
                    // atom prefactors (opencl/UFF.cl:1681-1687) times the stored channel scales
                    const float4 q = S.Q()[i];
                    const float ej = expf(a.alpha_morse * q.x);
                    float PLx = ej * ej * q.y, PLy = ej * q.y, PLz = q.z;
                    float sE = 0.f, sX = 0.f, sY = 0.f;
                    if (GDT != GRID_F32 && iz - 1 < g.zsplit) {
                        // a 16-bit grid's FP32 near-surface planes (the cell is uniform over the atom's lanes)
                        PLx *= g.lo_scale[0]; PLy *= g.lo_scale[1]; PLz *= g.lo_scale[2];
                        stencil_sums<GRID_F32>(g.lo, g.brick, g.nx, g.ny, g.lo_nz, ix, iy, iz, kz, PLx, PLy, PLz, bx, dxw, by, dyw, sE, sX, sY);
                    } else {
                        // stored-value scales: per z plane (this lane reads one plane) or per channel
                        const float4 zs = g.zscale ? __ldg(g.zscale + (iz - 1 + kz)) : make_float4(g.scale[0], g.scale[1], g.scale[2], 1.f);
                        PLx *= zs.x; PLy *= zs.y; PLz *= zs.z;
                        stencil_sums<GDT>(g.data, g.brick, g.nx, g.ny, g.nz, ix, iy, iz, kz, PLx, PLy, PLz, bx, dxw, by, dyw, sE, sX, sY);
                    }
                    const float bzk = comp(make_float4(bz[0], bz[1], bz[2], bz[3]), kz);
                    const float dzk = comp(make_float4(dzw[0], dzw[1], dzw[2], dzw[3]), kz);
                    e = bzk * sE; gx = bzk * sX; gy = bzk * sY; gz = dzk * sE;
                }
            }
            e += __shfl_xor_sync(FULL, e, 1); gx += __shfl_xor_sync(FULL, gx, 1);
            gy += __shfl_xor_sync(FULL, gy, 1); gz += __shfl_xor_sync(FULL, gz, 1);
            e += __shfl_xor_sync(FULL, e, 2); gx += __shfl_xor_sync(FULL, gx, 2);
            gy += __shfl_xor_sync(FULL, gy, 2); gz += __shfl_xor_sync(FULL, gz, 2);
            if (kz == 0 && i < N) {
                add4(S.F()[i], -gx * g.inv_step[0], -gy * g.inv_step[1], -gz * g.inv_step[2], e);
                acc.add(5, (double)e);
            }
        }
    }
    team_sync<T>();
}
#undef TP

// ------------------------------------------------------------------ NB neighbour lists
// Rows of partners within rc + skin, one warp per atom: lane c tests partner j0 + c and ballots
// place the accepted ones.  A row holds two runs: from its front, in ascending order, the inner
// partners, those closer than rc - skin - 0.01 A, which stay inside the cutoff until the next
// rebuild (each atom moves at most skin / 2 before one), so their pairs need no cutoff test; from
// its back, in ascending order towards the front, the shell partners.  The count packs
// inner | shell << 16; rows longer than nbl_cap mark the atom -2 (all pairs).  Also records each
// atom's position at the build.
template <int T>
__device__ void build_nblist(const KernelArgs& a, const Smem& S, int N, size_t ga0, int rank) {
    const int lane = rank & 31, warp = rank >> 5;
    const float rl = sqrtf(a.rc2) + a.nbl_skin, rl2 = rl * rl;
    const float ri = sqrtf(a.rc2) - a.nbl_skin - 0.01f, ri2 = ri > 0.f ? ri * ri : -1.f;
    const int cap = a.nbl_cap;
    for (int i = warp; i < N; i += T / 32) {
        const float4 pi = S.P()[i], li = S.Lo()[i];
        const short4 ng = S.Ng()[i];
        unsigned short* row = a.nbl + (ga0 + i) * (size_t)cap;
        int nin = 0, nsh = 0;
        for (int j0 = 0; j0 < N; j0 += 32) {
            const int j = j0 + lane;
            bool inc = false, inner = false;
            if (j < N && j != i && j != ng.x && j != ng.y && j != ng.z && j != ng.w) {
                const float4 pj = S.P()[j], lj = S.Lo()[j];
                const float dx = (pj.x - pi.x) + (lj.x - li.x), dy = (pj.y - pi.y) + (lj.y - li.y), dz = (pj.z - pi.z) + (lj.z - li.z);
                const float d2 = dx * dx + dy * dy + dz * dz;
                inc = d2 < rl2;
                inner = d2 < ri2;
            }
            const unsigned below = (1u << lane) - 1u;
            const unsigned mi = __ballot_sync(FULL, inner), ms = __ballot_sync(FULL, inc && !inner);
            const int qi = nin + __popc(mi & below), qs = nsh + __popc(ms & below);
            if (inner && qi < cap) row[qi] = (unsigned short)j;
            else if (inc && !inner && qs < cap) row[cap - 1 - qs] = (unsigned short)j;
            nin += __popc(mi);
            nsh += __popc(ms);
        }
        if (lane == 0) {
            a.nbl_cnt[ga0 + i] = nin + nsh <= cap ? (nin | nsh << 16) : -2;
            a.nbl_ref[ga0 + i] = make_float4(pi.x + li.x, pi.y + li.y, pi.z + li.z, 0.f);
        }
    }
    team_sync<T>();
}

// true when some atom moved more than skin / 2 since the last build (same answer on every rank)
template <int T>
__device__ bool nblist_stale(const KernelArgs& a, const Smem& S, int N, size_t ga0, int rank) {
    float m = 0.f;
    for (int i = rank; i < N; i += T) {
        const float4 p = S.P()[i], l = S.Lo()[i], r = a.nbl_ref[ga0 + i];
        const float dx = (p.x - r.x) + l.x, dy = (p.y - r.y) + l.y, dz = (p.z - r.z) + l.z;
        m = fmaxf(m, dx * dx + dy * dy + dz * dz);
    }
    m = warp_max(m);
    if (T > 32) {
        double* red = S.red();
        if ((rank & 31) == 0) red[rank >> 5] = (double)m;
        __syncthreads();
        m = 0.f;
        for (int k = 0; k < T / 32; k++) m = fmaxf(m, (float)red[k]);
        __syncthreads();
    }
    const float h = 0.5f * a.nbl_skin;
    return m > h * h;
}

// ------------------------------------------------------------------ one system
template <int T, int GDT, bool EVAL, int FORM>
__device__ void run_system(const KernelArgs& a, const Smem& S, int w, int rank) {
    const int slot = a.work[w];
    const SlotState st = a.slots[slot];
    // a slot with dt < 0 has not started FIRE yet: zero velocities, dt0, alpha0
    const bool fresh = !EVAL && st.dt < 0.0;
    int steps = fresh ? 0 : st.steps;
    int nsteps = 0;
    if (!EVAL) {
        nsteps = min(st.target, a.phase_limit) - steps;
        if (a.step_budget > 0) nsteps = min(nsteps, a.step_budget - steps);
        if (st.status != 0 || nsteps <= 0) return;          // nothing to do in this launch
    }
    const TopoDev* tpp = a.topos + st.topo;
    const int tp_atom_off = __ldg(&tpp->atom_off);
    const int N = st.natoms;
    for (int i = rank; i < N; i += T) {
        S.P()[i] = a.pos[st.atom_off + i];
        S.Lo()[i] = a.plo[st.atom_off + i];     // zeroed whenever positions are set
        S.V()[i] = (EVAL || fresh) ? make_float4(0.f, 0.f, 0.f, 0.f) : a.vel[st.atom_off + i];
        const float4 q = __ldg(a.req + tp_atom_off + i);
        S.Q()[i] = q;
        S.Ng()[i] = a.neigh[tp_atom_off + i];
    }
    team_sync<T>();

    EAcc<EVAL> acc;
    const float4* lat = (st.flags & SLOT_PBC) ? a.lat + 3 * (size_t)slot : nullptr;
    if (EVAL) {
        eval_forces<T, GDT, EVAL, FORM>(a, S, tpp, N, rank, acc, lat);
        for (int i = rank; i < N; i += T) a.force[st.atom_off + i] = S.F()[i];
        if constexpr (EVAL) {
            double tot = 0, e[6];
            for (int k = 0; k < 6; k++) { e[k] = team_sum<T>(acc.e[k], S.red(), rank); tot += e[k]; }
            if (rank == 0) {
                double* out = a.ecomp + (size_t)w * 8;
                out[0] = tot;
                for (int k = 0; k < 6; k++) out[1 + k] = e[k];
                out[7] = 0.0;
            }
        }
        team_sync<T>();
        return;
    }

    // neighbour list: rebuilt on the first step after positions were set (fresh FIRE state) and
    // whenever an atom has moved more than skin / 2; both depend only on this system's trajectory
    const bool use_list = a.nbl != nullptr && N >= a.nbl_min && a.rc2 < 1e37f && FORM != FORM_GATHER_EXT;
    const size_t ga0 = (size_t)st.atom_off;
    bool need_build = use_list && fresh;
    double dt = fresh ? a.fire.dt0 : st.dt, alpha = fresh ? a.fire.alpha0 : st.alpha;
    int npos = fresh ? 0 : st.npos, status = st.status;
    float fmax = st.fmax;
    const float flim = (float)a.fire.flimit, flim2 = flim * flim;
    // constraint springs (extended form only): added after the force limit, they drive FIRE but
    // are not stored with the forces, as updateAtomsMMFFf4 stores the force before them
    const bool cons_on = FORM == FORM_GATHER_EXT && (st.flags & SLOT_CONS) != 0;
    // Langevin drive (extended form only, UFF.cl:982-991): -gamma v + noise(seed) sqrt(2 kB T gamma / dt)
    // on the force FIRE uses, v the velocity before the step; the seed advances by td.z per step
    // of the system, so chunked and unchunked runs draw the same numbers
    const bool therm_on = FORM == FORM_GATHER_EXT && (st.flags & SLOT_THERM) != 0;
    const float4 td = therm_on ? __ldg(a.tdrive + slot) : make_float4(0.f, 0.f, 0.f, 0.f);
    int ran = 0;
    for (int it = 0; it < nsteps; it++) {
        if (use_list) {
            if (need_build || nblist_stale<T>(a, S, N, ga0, rank)) build_nblist<T>(a, S, N, ga0, rank);
            need_build = false;
        }
        eval_forces<T, GDT, EVAL, FORM>(a, S, tpp, N, rank, acc, lat, use_list, ga0);
        ran = 1;
        const double dt_old = dt;
        const float dtf = (float)dt_old;
        double vf = 0.0, vv = 0.0, ff = 0.0;
        float f2m = 0.f;
        const float seed = therm_on ? __fmaf_rn(td.z, (float)steps, td.w) : 0.f;
        const float amp = therm_on ? (float)sqrt(2.0 * KB_EV * (double)td.x * (double)td.y / dt_old) : 0.f;
        for (int i = rank; i < N; i += T) {
            float4 f = S.F()[i];
            float f2 = f.x * f.x + f.y * f.y + f.z * f.z;
            if (flim > 0.f && f2 > flim2) {
                const float s = flim / sqrtf(f2);
                f.x *= s; f.y *= s; f.z *= s;
                S.F()[i] = f;
                f2 = f.x * f.x + f.y * f.y + f.z * f.z;
            }
            if (cons_on) {
                const float3 fc = constraint_force(a.cons, ga0 + i, S.P()[i], S.Lo()[i]);
                f.x += fc.x; f.y += fc.y; f.z += fc.z;
                f2 = f.x * f.x + f.y * f.y + f.z * f.z;
            }
            float4 v = S.V()[i];
            if (therm_on) {
                add_langevin(f, v, i, seed, amp, td.y);
                f2 = f.x * f.x + f.y * f.y + f.z * f.z;
                v = kick(v, f, dtf);          // the second pass rebuilds this velocity from the stored one
            } else {
                v.x += f.x * dtf; v.y += f.y * dtf; v.z += f.z * dtf;
                S.V()[i] = v;
            }
            f2m = fmaxf(f2m, f2);
            ff += (double)f2;
            vf += (double)(v.x * f.x + v.y * f.y + v.z * f.z);
            vv += (double)(v.x * v.x + v.y * v.y + v.z * v.z);
        }
        team_reduce4<T>(vf, vv, ff, f2m, S.red(), rank);
        const bool mix = vf > 0.0 && ff > 1e-30 && vv > 1e-30;
        float cv = 0.f, cf = 0.f;
        if (mix) {
            cv = (float)(1.0 - alpha);
            cf = (float)(alpha * sqrt(vv) / sqrt(ff));
            npos++;
            if (npos > a.fire.n_min) { dt = fmin(dt * a.fire.f_inc, a.fire.dt_max); alpha *= a.fire.f_alpha; }
        } else {
            npos = 0; dt *= a.fire.f_dec; alpha = a.fire.alpha0;
        }
        for (int i = rank; i < N; i += T) {
            float4 v = S.V()[i];
            if (mix || therm_on) {
                float4 f = S.F()[i];
                if (cons_on) {
                    const float3 fc = constraint_force(a.cons, ga0 + i, S.P()[i], S.Lo()[i]);
                    f.x += fc.x; f.y += fc.y; f.z += fc.z;
                }
                if (therm_on) {
                    add_langevin(f, v, i, seed, amp, td.y);
                    v = kick(v, f, dtf);
                }
                if (mix) { v.x = v.x * cv + f.x * cf; v.y = v.y * cv + f.y * cf; v.z = v.z * cv + f.z * cf; }
                else v = make_float4(0.f, 0.f, 0.f, 0.f);
            } else {
                v = make_float4(0.f, 0.f, 0.f, 0.f);
            }
            S.V()[i] = v;
            // x += v dt with the rounding error of every move carried in Lo (Fast2Sum): late FIRE
            // moves are ~1e-6 A, the size of one float ulp at 20 A, and would otherwise be lost
            float4 p = S.P()[i], lo = S.Lo()[i];
            float y, t;
            y = v.x * dtf + lo.x; t = p.x + y; lo.x = y - (t - p.x); p.x = t;
            y = v.y * dtf + lo.y; t = p.y + y; lo.y = y - (t - p.y); p.y = t;
            y = v.z * dtf + lo.z; t = p.z + y; lo.z = y - (t - p.z); p.z = t;
            S.P()[i] = p;
            S.Lo()[i] = lo;
        }
        steps++;
        fmax = sqrtf(f2m);
        team_sync<T>();
        if (!isfinite(ff) || !isfinite(vv)) { status = 3; break; }
        if ((double)fmax < a.fire.fconv) { status = 1; break; }
        if (a.step_budget > 0 && steps >= a.step_budget) { status = 2; break; }
    }
    double energy = st.energy;
    if (ran) {
        double e = 0.0;
        for (int i = rank; i < N; i += T) e += (double)S.F()[i].w - 0.5 * (double)S.Eh()[i];
        energy = team_sum<T>(e, S.red(), rank);
    }
    for (int i = rank; i < N; i += T) {
        a.pos[st.atom_off + i] = S.P()[i];
        a.plo[st.atom_off + i] = S.Lo()[i];
        a.vel[st.atom_off + i] = S.V()[i];
        if (ran) a.force[st.atom_off + i] = S.F()[i];
    }
    if (rank == 0) {
        SlotState& o = a.slots[slot];
        o.dt = dt; o.alpha = alpha; o.npos = npos; o.steps = steps; o.status = status;
        o.energy = energy; o.fmax = fmax;
    }
    team_sync<T>();
}

// GS (global state): the team's state lives in a slot of the global scratch instead of shared
// memory, for systems too large for it (team syncs order global memory within the block just as
// shared memory).  A compile-time choice: with the base pointer chosen at run time the compiler
// could no longer use shared-memory instructions for the state.
template <int T, int GDT, bool EVAL, int FORM, bool GS>
// warp teams: 4 per block; a 40-atom system's shared memory allows 7 blocks per SM in the rounds
// and gather forms and 6 in the owner form (slot pieces), which leaves it 85 registers
__global__ void __launch_bounds__(T == 32 ? 128 : T, relax_min_blocks(T, FORM))
relax_kernel(const KernelArgs a) {
    extern __shared__ __align__(16) char smem[];
    const int team = (T == 32) ? (threadIdx.x >> 5) : 0;
    const int rank = (T == 32) ? (threadIdx.x & 31) : threadIdx.x;
    const size_t tb = team_bytes(a.nmax, a.nfmax, T, FORM);
    char* tbase = GS ? a.gscratch + ((size_t)blockIdx.x * (T == 32 ? 4 : 1) + team) * tb : smem + (size_t)team * tb;
    const Smem S = carve(tbase, a.nmax);
    __shared__ int s_w;
    for (;;) {
        int w;
        if (T == 32) {
            if (rank == 0) w = atomicAdd(a.counter, 1);
            w = __shfl_sync(FULL, w, 0);
        } else {
            if (rank == 0) s_w = atomicAdd(a.counter, 1);
            __syncthreads();
            w = s_w;
            __syncthreads();
        }
        if (w >= a.nwork) break;
        run_system<T, GDT, EVAL, FORM>(a, S, w, rank);
    }
}

template <int T, int GDT, bool EVAL, int FORM, bool GS>
int launch_t(const KernelArgs& a, cudaStream_t s, int num_sms) {
    const int tpb = (T == 32) ? 4 : 1;           // teams per block
    const int block = T * tpb;
    const size_t state = (size_t)tpb * team_bytes(a.nmax, a.nfmax, T, FORM);
    const size_t smem = GS ? 0 : state;           // global-state launches use no dynamic shared memory
    auto kern = relax_kernel<T, GDT, EVAL, FORM, GS>;
    // blocks per SM of this instance, per (device, dynamic shared memory); handles driven from
    // several host threads (one per GPU, say) share the cache under its lock
    static std::mutex occ_mu;
    static std::map<std::pair<int, size_t>, int> occ_cache;
    int dev = 0;
    { cudaError_t e = cudaGetDevice(&dev); if (e != cudaSuccess) return (int)e; }
    int occ = -1;
    {
        std::lock_guard<std::mutex> lk(occ_mu);
        auto it = occ_cache.find({dev, smem});
        if (it != occ_cache.end()) occ = it->second;
    }
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
    }
    if (T > 32 && !GS) {
        // block teams: the preferred split of the SM's L1 between shared memory and cache
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, a.smem_carveout);
        if (e != cudaSuccess) return (int)e;
    }
    if (occ < 0) {
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, block, smem);
        if (e != cudaSuccess) return (int)e;
        std::lock_guard<std::mutex> lk(occ_mu);
        occ_cache[{dev, smem}] = occ;
    }
    if (occ < 1) return (int)cudaErrorInvalidConfiguration;
    int blocks_needed = (a.nwork + tpb - 1) / tpb;
    int grid = min(blocks_needed, occ * num_sms);
    if (GS) grid = min(grid, (int)(a.gscratch_bytes / state));   // one scratch slot per block
    if (grid < 1) grid = 1;
    kern<<<grid, block, smem, s>>>(a);
    return (int)cudaGetLastError();
}

template <int GDT, bool EVAL, int FORM>
int launch_team(const KernelArgs& a, int team, cudaStream_t s, int num_sms) {
    if (a.gscratch) {
        // global-state launches exist for the gather form with 128-512 threads (the host sends
        // every system too large for shared memory there)
        if constexpr (FORM == FORM_GATHER || FORM == FORM_GATHER_EXT) {
            switch (team) {
                case 128: return launch_t<128, GDT, EVAL, FORM, true>(a, s, num_sms);
                case 256: return launch_t<256, GDT, EVAL, FORM, true>(a, s, num_sms);
                case 512: return launch_t<512, GDT, EVAL, FORM, true>(a, s, num_sms);
            }
        }
        return (int)cudaErrorInvalidValue;
    }
    switch (team) {
        case 32: return launch_t<32, GDT, EVAL, FORM, false>(a, s, num_sms);
        case 64: return launch_t<64, GDT, EVAL, FORM, false>(a, s, num_sms);
        case 128: return launch_t<128, GDT, EVAL, FORM, false>(a, s, num_sms);
        case 256: return launch_t<256, GDT, EVAL, FORM, false>(a, s, num_sms);
        case 512: return launch_t<512, GDT, EVAL, FORM, false>(a, s, num_sms);
    }
    return (int)cudaErrorInvalidValue;
}

template <bool EVAL, int FORM>
int launch_dtype(const KernelArgs& a, int team, cudaStream_t s, int num_sms) {
    const int gdt = a.has_grid && !a.fold.on ? a.grid.dtype : GRID_F32;
    if (gdt == GRID_F16) return launch_team<GRID_F16, EVAL, FORM>(a, team, s, num_sms);
    if (gdt == GRID_BF16) return launch_team<GRID_BF16, EVAL, FORM>(a, team, s, num_sms);
    return launch_team<GRID_F32, EVAL, FORM>(a, team, s, num_sms);
}

}  // namespace

size_t team_smem_bytes(int nmax, int nfmax, int team, int form) {
    return team_bytes(nmax, nfmax, team, form) * (team == 32 ? 4 : 1);
}

namespace {
// copy n segments of float4: dst[dst_off[s] + i] = src[src_off[s] + i], i < len[s]; one block per segment
__global__ void copy_segments_kernel(const int* __restrict__ src_off, const int* __restrict__ len, const int* __restrict__ dst_off,
                                     const float4* __restrict__ src, float4* __restrict__ dst) {
    const int s = blockIdx.x;
    const int n = len[s], a = src_off[s], b = dst_off[s];
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[b + i] = src[a + i];
}
}  // namespace

int launch_copy_segments(const int* d_src_off, const int* d_len, const int* d_dst_off, int n, const float4* src, float4* dst,
                         cudaStream_t s) {
    if (n <= 0) return 0;
    copy_segments_kernel<<<n, 128, 0, s>>>(d_src_off, d_len, d_dst_off, src, dst);
    return (int)cudaGetLastError();
}

int launch_relax(const KernelArgs& a, int team, int form, int eval_only, cudaStream_t s, int num_sms, long long* launches) {
    if (a.nwork <= 0) return 0;
    int r;
    if (eval_only) r = form == FORM_GATHER ? launch_dtype<true, FORM_GATHER>(a, team, s, num_sms)
                     : form == FORM_OWNER ? launch_dtype<true, FORM_OWNER>(a, team, s, num_sms)
                     : form == FORM_GATHER_EXT ? launch_dtype<true, FORM_GATHER_EXT>(a, team, s, num_sms)
                                          : launch_dtype<true, FORM_ROUNDS>(a, team, s, num_sms);
    else r = form == FORM_GATHER ? launch_dtype<false, FORM_GATHER>(a, team, s, num_sms)
           : form == FORM_OWNER ? launch_dtype<false, FORM_OWNER>(a, team, s, num_sms)
           : form == FORM_GATHER_EXT ? launch_dtype<false, FORM_GATHER_EXT>(a, team, s, num_sms)
                                : launch_dtype<false, FORM_ROUNDS>(a, team, s, num_sms);
    if (launches && r == 0) (*launches)++;
    return r;
}

}  // namespace smr
