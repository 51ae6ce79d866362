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
//   B  angle / dihedral / inversion rounds  opencl/UFF.cl:326-795 with the assembly of
//      801-880 replaced by shared-memory adds: the host packs terms into rounds in which
//      the atoms of each role are distinct, so the adds need no atomics and run in a
//      fixed order (bitwise reproducible, independent of co-resident systems)
//   C  intramolecular LJ + Coulomb ......... opencl/UFF.cl:57-95, 1595-1665 (1-2 exclusion)
//      with L lanes per atom splitting the partner loop, combined by shuffles
//   D  tricubic B-spline grid sample ....... opencl/UFF.cl:1384-1511, 1671-1711, four lanes
//      per atom, each fetching one x-slice (16 voxels) through the read-only path
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
#include <tuple>

#include "smr_internal.h"

namespace smr {

namespace {

constexpr float kCoulomb = 14.3996448915f;   // eV*A/e^2
constexpr unsigned FULL = 0xffffffffu;

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline size_t red_bytes(int T) { return T > 32 ? size_t(T / 32) * 4 * sizeof(double) : 0; }

// Shared memory of one team for systems of up to nmax atoms.
__host__ __device__ inline size_t team_bytes(int nmax, int T) {
    size_t n = (size_t)nmax;
    return n * 16 * 5 + n * 64 + align16(n * 4) + align16(n * 8) + red_bytes(T);
}

struct Smem {
    float4* P;   // positions (w unused)
    float4* V;   // velocities
    float4* F;   // forces, w = per-atom energy (reference fapos.w convention)
    float4* Q;   // R, sqrt(E), Q, H
    float4* PL;  // grid prefactors (Pauli, London, Q, 0) times the grid channel scales
    float4* H;   // hneigh: 4 per atom, (unit bond vector, 1/length)
    float* Eh;   // bond + NB part of the per-atom energy (counted twice in fapos.w)
    short4* Ng;  // neighbour slots
    double* red; // team reduction scratch (T > 32)
};

__device__ inline Smem carve(char* base, int nmax, int T) {
    Smem s;
    size_t n = (size_t)nmax;
    s.P = (float4*)base; base += n * 16;
    s.V = (float4*)base; base += n * 16;
    s.F = (float4*)base; base += n * 16;
    s.Q = (float4*)base; base += n * 16;
    s.PL = (float4*)base; base += n * 16;
    s.H = (float4*)base; base += n * 64;
    s.Eh = (float*)base; base += align16(n * 4);
    s.Ng = (short4*)base; base += align16(n * 8);
    s.red = (double*)base;
    return s;
}

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
template <int GDT> __device__ __forceinline__ float4 load_voxel(const void* g, size_t i);
template <> __device__ __forceinline__ float4 load_voxel<GRID_F32>(const void* g, size_t i) {
    return __ldg(reinterpret_cast<const float4*>(g) + i);
}
template <> __device__ __forceinline__ float4 load_voxel<GRID_F16>(const void* g, size_t i) {
    uint2 u = __ldg(reinterpret_cast<const uint2*>(g) + i);
    float2 a = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
    float2 b = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
    return make_float4(a.x, a.y, b.x, b.y);
}
template <> __device__ __forceinline__ float4 load_voxel<GRID_BF16>(const void* g, size_t i) {
    uint2 u = __ldg(reinterpret_cast<const uint2*>(g) + i);
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

// lanes per atom for the NB partner loop: minimise passes x partners per lane
__device__ __forceinline__ int nb_lanes(int N, int T) {
    int best = 1; long long bc = 1LL << 60;
    for (int L = 1; L <= 32; L <<= 1) {
        int G = T / L;
        long long cost = (long long)((N + G - 1) / G) * ((N + L - 1) / L);
        if (cost < bc) { bc = cost; best = L; }
    }
    return best;
}

// ------------------------------------------------------------------ force evaluation
template <int T, int GDT, bool EVAL>
__device__ void eval_forces(const KernelArgs& a, const Smem& S, const TopoDev& tp, int N, int rank, double* eacc) {
    // A: bonds and hneigh, one atom per rank
    for (int i = rank; i < N; i += T) {
        const float4 pi = S.P[i];
        const short4 ng = S.Ng[i];
        const float4 bk = __ldg(a.bk + tp.atom_off + i), bl = __ldg(a.bl + tp.atom_off + i);
        float fx = 0.f, fy = 0.f, fz = 0.f, E = 0.f;
#pragma unroll
        for (int s = 0; s < 4; s++) {
            const int g = comp(ng, s);
            if (g < 0) { S.H[4 * i + s] = make_float4(0.f, 0.f, 0.f, 1e6f); continue; }
            const float4 pj = S.P[g];
            const float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
            const float l2 = fmaxf(dx * dx + dy * dy + dz * dz, 1e-16f);
            const float l = sqrtf(l2), il = 1.0f / l;
            const float hx = dx * il, hy = dy * il, hz = dz * il;
            S.H[4 * i + s] = make_float4(hx, hy, hz, il);
            const float k = comp(bk, s), dl = l - comp(bl, s), fr = 2.0f * k * dl;
            fx += hx * fr; fy += hy * fr; fz += hz * fr;
            E += k * dl * dl;
        }
        S.F[i] = make_float4(fx, fy, fz, E);
        S.Eh[i] = E;
        if (EVAL) eacc[0] += 0.5 * (double)E;
    }
    team_sync<T>();

    // B1: angles (Fourier form via complex powers)
    for (int r = 0; r < tp.ang_rounds; r++) {
        const AngRec rec = load_rec(a.angs + tp.ang_off + (size_t)r * T + rank);
        const bool ok = rec.at.x >= 0;
        float3 fpi = {0, 0, 0}, fpj = {0, 0, 0}, fpk = {0, 0, 0};
        float E = 0.f;
        if (ok) {
            const float4 qij = S.H[rec.sl.x], qkj = S.H[rec.sl.y];
            const float hx = qij.x + qkj.x, hy = qij.y + qkj.y, hz = qij.z + qkj.z;
            float c = 0.5f * (hx * hx + hy * hy + hz * hz - 2.0f);
            c = fminf(fmaxf(c, -1.0f), 1.0f);
            const float s = sqrtf(fmaxf(0.0f, 1.0f - c * c) + 1e-14f);
            const float is = (s > 1e-12f) ? 1.0f / s : 0.0f;
            const float c2x = c * c - s * s, c2y = c * s + s * c;
            const float c3x = c2x * c - c2y * s, c3y = c2x * s + c2y * c;
            const float4 p = rec.p;   // K*(c0, c1, c2, c3)
            E = p.x + p.z * c2x + p.w * c3x;
            const float fm = p.y + p.z * c2y * is * 2.0f + p.w * c3y * is * 3.0f;
            const float fi = fm * qij.w, fk = fm * qkj.w, fic = fi * c, fkc = fk * c;
            fpi = make_float3(fic * qij.x - fi * qkj.x, fic * qij.y - fi * qkj.y, fic * qij.z - fi * qkj.z);
            fpk = make_float3(-fk * qij.x + fkc * qkj.x, -fk * qij.y + fkc * qkj.y, -fk * qij.z + fkc * qkj.z);
            fpj = make_float3((fk - fic) * qij.x + (fi - fkc) * qkj.x, (fk - fic) * qij.y + (fi - fkc) * qkj.y,
                              (fk - fic) * qij.z + (fi - fkc) * qkj.z);
            if (EVAL) eacc[1] += (double)E;
        }
        const float e3 = E / 3.0f;
        if (ok) add4(S.F[rec.at.x], fpi.x, fpi.y, fpi.z, e3);
        team_sync<T>();
        if (ok) add4(S.F[rec.at.y], fpj.x, fpj.y, fpj.z, e3);
        team_sync<T>();
        if (ok) add4(S.F[rec.at.z], fpk.x, fpk.y, fpk.z, e3);
        team_sync<T>();
    }

    // B2: dihedrals
    for (int r = 0; r < tp.dih_rounds; r++) {
        const DihRec rec = load_rec(a.dihs + tp.dih_off + (size_t)r * T + rank);
        const bool ok = rec.at.x >= 0;
        float3 f1 = {0, 0, 0}, f2 = {0, 0, 0}, f3 = {0, 0, 0}, f4 = {0, 0, 0};
        float E = 0.f;
        if (ok) {
            const float4 q12 = S.H[rec.sl.x], q32 = S.H[rec.sl.y], q43 = S.H[rec.sl.z];
            const float3 n123 = make_float3(q12.y * q32.z - q12.z * q32.y, q12.z * q32.x - q12.x * q32.z, q12.x * q32.y - q12.y * q32.x);
            const float3 n234 = make_float3(q43.y * q32.z - q43.z * q32.y, q43.z * q32.x - q43.x * q32.z, q43.x * q32.y - q43.y * q32.x);
            const float a2 = n123.x * n123.x + n123.y * n123.y + n123.z * n123.z;
            const float b2 = n234.x * n234.x + n234.y * n234.y + n234.z * n234.z;
            if (!(a2 < 1e-30f || b2 < 1e-30f)) {
                const float il2a = 1.0f / a2, il2b = 1.0f / b2, inv = sqrtf(il2a * il2b);
                const float cx = (n123.x * n234.x + n123.y * n234.y + n123.z * n234.z) * inv;
                const float cy = -(n123.x * q43.x + n123.y * q43.y + n123.z * q43.z) * inv;
                float nx = cx, ny = cy;
                const int nn = (int)rec.p.z;
                for (int k = 1; k < nn; k++) { const float t = nx * cx - ny * cy; ny = nx * cy + ny * cx; nx = t; }
                E = rec.p.x * (1.0f + rec.p.y * nx);
                const float f = -rec.p.x * rec.p.y * rec.p.z * ny;
                const float s1 = -f * il2a * q12.w, s4 = f * il2b * q43.w;
                f1 = make_float3(n123.x * s1, n123.y * s1, n123.z * s1);
                f4 = make_float3(n234.x * s4, n234.y * s4, n234.z * s4);
                const float c123 = (q32.x * q12.x + q32.y * q12.y + q32.z * q12.z) * (q32.w / q12.w);
                const float c432 = (q32.x * q43.x + q32.y * q43.y + q32.z * q43.z) * (q32.w / q43.w);
                f3 = make_float3(-c123 * f1.x + (-c432 - 1.0f) * f4.x, -c123 * f1.y + (-c432 - 1.0f) * f4.y, -c123 * f1.z + (-c432 - 1.0f) * f4.z);
                f2 = make_float3((c123 - 1.0f) * f1.x + c432 * f4.x, (c123 - 1.0f) * f1.y + c432 * f4.y, (c123 - 1.0f) * f1.z + c432 * f4.z);
            }
            if (EVAL) eacc[2] += (double)E;
        }
        const float e4 = 0.25f * E;
        if (ok) add4(S.F[rec.at.x], f1.x, f1.y, f1.z, e4);
        team_sync<T>();
        if (ok) add4(S.F[rec.at.y], f2.x, f2.y, f2.z, e4);
        team_sync<T>();
        if (ok) add4(S.F[rec.at.z], f3.x, f3.y, f3.z, e4);
        team_sync<T>();
        if (ok) add4(S.F[rec.at.w], f4.x, f4.y, f4.z, e4);
        team_sync<T>();
    }

    // B3: inversions
    for (int r = 0; r < tp.inv_rounds; r++) {
        const InvRec rec = load_rec(a.invs + tp.inv_off + (size_t)r * T + rank);
        const bool ok = rec.at.x >= 0;
        float3 f1 = {0, 0, 0}, f2 = {0, 0, 0}, f3 = {0, 0, 0}, f4 = {0, 0, 0};
        float E = 0.f;
        if (ok) {
            const float4 q21 = S.H[rec.sl.x], q31 = S.H[rec.sl.y], q41 = S.H[rec.sl.z];
            float3 n = make_float3(q21.y * q31.z - q21.z * q31.y, q21.z * q31.x - q21.x * q31.z, q21.x * q31.y - q21.y * q31.x);
            const float nn = n.x * n.x + n.y * n.y + n.z * n.z;
            float il = 0.0f;
            if (nn > 1e-16f) { il = rsqrtf(nn); n.x *= il; n.y *= il; n.z *= il; }
            else n = make_float3(0.f, 0.f, 0.f);
            float sw = -(n.x * q41.x + n.y * q41.y + n.z * q41.z);
            sw = fminf(fmaxf(sw, -1.0f), 1.0f);
            const float cw = sqrtf(1.0f - sw * sw);
            const float4 p = rec.p;   // K, c0, c1, c2
            E = p.x * (p.y + p.z * cw + p.w * (2.0f * cw * cw - 1.0f));
            const float dEdw = -p.x * (p.z * sw + 2.0f * p.w * (2.0f * sw * cw));
            const float ft = (cw > 1e-7f) ? dEdw / cw : 0.0f;
            const float fq41 = ft * q41.w, fi123 = ft * il;
            const float3 tq = make_float3(sw * fi123 * n.x + fi123 * q41.x, sw * fi123 * n.y + fi123 * q41.y, sw * fi123 * n.z + fi123 * q41.z);
            f4 = make_float3(fq41 * n.x + sw * fq41 * q41.x, fq41 * n.y + sw * fq41 * q41.y, fq41 * n.z + sw * fq41 * q41.z);
            f2 = make_float3((q31.y * tq.z - q31.z * tq.y) * q21.w, (q31.z * tq.x - q31.x * tq.z) * q21.w, (q31.x * tq.y - q31.y * tq.x) * q21.w);
            f3 = make_float3((tq.y * q21.z - tq.z * q21.y) * q31.w, (tq.z * q21.x - tq.x * q21.z) * q31.w, (tq.x * q21.y - tq.y * q21.x) * q31.w);
            f1 = make_float3(-(f2.x + f3.x + f4.x), -(f2.y + f3.y + f4.y), -(f2.z + f3.z + f4.z));
            if (EVAL) eacc[3] += (double)E;
        }
        const float e4 = 0.25f * E;
        if (ok) add4(S.F[rec.at.x], f1.x, f1.y, f1.z, e4);
        team_sync<T>();
        if (ok) add4(S.F[rec.at.y], f2.x, f2.y, f2.z, e4);
        team_sync<T>();
        if (ok) add4(S.F[rec.at.z], f3.x, f3.y, f3.z, e4);
        team_sync<T>();
        if (ok) add4(S.F[rec.at.w], f4.x, f4.y, f4.z, e4);
        team_sync<T>();
    }

    // C: intramolecular LJ + damped Coulomb, all pairs except bonded (1-2) neighbours
    {
        const int L = nb_lanes(N, T), G = T / L;
        const int c = rank & (L - 1);
        for (int i0 = 0; i0 < N; i0 += G) {
            const int i = i0 + rank / L;
            float fx = 0.f, fy = 0.f, fz = 0.f, E = 0.f;
            if (i < N) {
                const float4 pi = S.P[i], qi = S.Q[i];
                const short4 ng = S.Ng[i];
                for (int j = c; j < N; j += L) {
                    if (j == i || j == ng.x || j == ng.y || j == ng.z || j == ng.w) continue;
                    const float4 pj = S.P[j];
                    const float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
                    const float r2 = dx * dx + dy * dy + dz * dz;
                    if (r2 > a.rc2) continue;
                    const float4 qj = S.Q[j];
                    const float R0 = qi.x + qj.x, E0 = qi.y * qj.y, Q = qi.z * qj.z;
                    const float rs = rsqrtf(r2 + a.R2damp);          // 1/sqrt(r^2 + Rdamp^2)
                    const float Ec = kCoulomb * Q * rs;
                    const float ir2 = 1.0f / r2;
                    const float u2 = R0 * R0 * ir2, u6 = u2 * u2 * u2, vdW = u6 * E0;
                    E += (u6 - 2.0f) * vdW + Ec;
                    const float fr = -12.0f * (u6 - 1.0f) * vdW * ir2 - Ec * (rs * rs);
                    fx += dx * fr; fy += dy * fr; fz += dz * fr;
                }
            }
            for (int o = 1; o < L; o <<= 1) {
                fx += __shfl_xor_sync(FULL, fx, o); fy += __shfl_xor_sync(FULL, fy, o);
                fz += __shfl_xor_sync(FULL, fz, o); E += __shfl_xor_sync(FULL, E, o);
            }
            if (c == 0 && i < N) {
                add4(S.F[i], fx, fy, fz, E);
                S.Eh[i] += E;
                if (EVAL) eacc[4] += 0.5 * (double)E;
            }
        }
    }
    team_sync<T>();

    // D: substrate grid, 4 lanes per atom (one x-slice of the 4x4x4 stencil each)
    if (a.has_grid) {
        const GridView& g = a.grid;
        const int xa = rank & 3;
        for (int i0 = 0; i0 < N; i0 += T / 4) {
            const int i = i0 + (rank >> 2);
            float e = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
            if (i < N) {
                const float4 p = S.P[i];
                const float ux = (p.x - g.p0[0]) * g.inv_step[0];
                const float uy = (p.y - g.p0[1]) * g.inv_step[1];
                const float uz = (p.z - g.p0[2]) * g.inv_step[2];
                int ix = (int)ux, iy = (int)uy;
                const int iz = (int)uz;
                if (ux < 0) ix--;
                if (uy < 0) iy--;
                if (iz >= 1 && iz < g.nz - 2) {
                    const float tx = ux - ix, ty = uy - iy, tz = uz - iz;
                    float bx[4], dxw[4], by[4], dyw[4], bz[4], dzw[4];
                    bspline(tx, bx, dxw); bspline(ty, by, dyw); bspline(tz, bz, dzw);
                    const float4 PL = S.PL[i];
                    const int xg = imod(ix - 1 + xa, g.nx);
                    const int y0 = imod(iy - 1, g.ny);
                    float sE = 0.f, sDy = 0.f, sDz = 0.f;
#pragma unroll
                    for (int b = 0; b < 4; b++) {
                        int yg = y0 + b;
                        if (yg >= g.ny) yg -= g.ny;
                        const size_t base = (size_t)(iz - 1) + (size_t)g.nz * ((size_t)yg + (size_t)g.ny * (size_t)xg);
                        float pz = 0.f, dz = 0.f;
#pragma unroll
                        for (int k = 0; k < 4; k++) {
                            const float4 v = load_voxel<GDT>(g.data, base + k);
                            const float cs = PL.x * v.x + PL.y * v.y + PL.z * v.z + PL.w * v.w;
                            pz += bz[k] * cs; dz += dzw[k] * cs;
                        }
                        sE += by[b] * pz; sDy += dyw[b] * pz; sDz += by[b] * dz;
                    }
                    const float bxa = comp(make_float4(bx[0], bx[1], bx[2], bx[3]), xa);
                    const float dxa = comp(make_float4(dxw[0], dxw[1], dxw[2], dxw[3]), xa);
                    e = bxa * sE; gx = dxa * sE; gy = bxa * sDy; gz = bxa * sDz;
                }
            }
            e += __shfl_xor_sync(FULL, e, 1); gx += __shfl_xor_sync(FULL, gx, 1);
            gy += __shfl_xor_sync(FULL, gy, 1); gz += __shfl_xor_sync(FULL, gz, 1);
            e += __shfl_xor_sync(FULL, e, 2); gx += __shfl_xor_sync(FULL, gx, 2);
            gy += __shfl_xor_sync(FULL, gy, 2); gz += __shfl_xor_sync(FULL, gz, 2);
            if (xa == 0 && i < N) {
                add4(S.F[i], -gx * g.inv_step[0], -gy * g.inv_step[1], -gz * g.inv_step[2], e);
                if (EVAL) eacc[5] += (double)e;
            }
        }
    }
    team_sync<T>();
}

// ------------------------------------------------------------------ one system
template <int T, int GDT, bool EVAL>
__device__ void run_system(const KernelArgs& a, const Smem& S, int w, int rank) {
    const int slot = a.work[w];
    const SlotState st = a.slots[slot];
    const TopoDev tp = a.topos[st.topo];
    const int N = st.natoms;
    // a slot with dt < 0 has not started FIRE yet: zero velocities, dt0, alpha0
    const bool fresh = !EVAL && st.dt < 0.0;
    for (int i = rank; i < N; i += T) {
        S.P[i] = a.pos[st.atom_off + i];
        S.V[i] = (EVAL || fresh) ? make_float4(0.f, 0.f, 0.f, 0.f) : a.vel[st.atom_off + i];
        const float4 q = __ldg(a.req + tp.atom_off + i);
        S.Q[i] = q;
        S.Ng[i] = a.neigh[tp.atom_off + i];
        const float ej = expf(a.alpha_morse * q.x);
        S.PL[i] = make_float4(ej * ej * q.y * a.grid.scale[0], ej * q.y * a.grid.scale[1], q.z * a.grid.scale[2], 0.f);
    }
    team_sync<T>();

    double eacc[6] = {0, 0, 0, 0, 0, 0};
    if (EVAL) {
        eval_forces<T, GDT, true>(a, S, tp, N, rank, eacc);
        for (int i = rank; i < N; i += T) a.force[st.atom_off + i] = S.F[i];
        double tot = 0;
        for (int k = 0; k < 6; k++) { eacc[k] = team_sum<T>(eacc[k], S.red, rank); tot += eacc[k]; }
        if (rank == 0) {
            double* out = a.ecomp + (size_t)w * 8;
            out[0] = tot;
            for (int k = 0; k < 6; k++) out[1 + k] = eacc[k];
            out[7] = 0.0;
        }
        team_sync<T>();
        return;
    }

    double dt = fresh ? a.fire.dt0 : st.dt, alpha = fresh ? a.fire.alpha0 : st.alpha;
    int npos = fresh ? 0 : st.npos, steps = fresh ? 0 : st.steps, status = st.status;
    float fmax = st.fmax;
    int nsteps = a.max_steps;
    if (a.step_budget > 0) nsteps = min(nsteps, a.step_budget - steps);
    if (status != 0) nsteps = 0;
    const float flim = (float)a.fire.flimit, flim2 = flim * flim;
    int ran = 0;
    for (int it = 0; it < nsteps; it++) {
        eval_forces<T, GDT, false>(a, S, tp, N, rank, eacc);
        ran = 1;
        const double dt_old = dt;
        const float dtf = (float)dt_old;
        double vf = 0.0, vv = 0.0, ff = 0.0;
        float f2m = 0.f;
        for (int i = rank; i < N; i += T) {
            float4 f = S.F[i];
            float f2 = f.x * f.x + f.y * f.y + f.z * f.z;
            if (flim > 0.f && f2 > flim2) {
                const float s = flim / sqrtf(f2);
                f.x *= s; f.y *= s; f.z *= s;
                S.F[i] = f;
                f2 = f.x * f.x + f.y * f.y + f.z * f.z;
            }
            f2m = fmaxf(f2m, f2);
            ff += (double)f2;
            float4 v = S.V[i];
            v.x += f.x * dtf; v.y += f.y * dtf; v.z += f.z * dtf;
            S.V[i] = v;
            vf += (double)(v.x * f.x + v.y * f.y + v.z * f.z);
            vv += (double)(v.x * v.x + v.y * v.y + v.z * v.z);
        }
        team_reduce4<T>(vf, vv, ff, f2m, S.red, rank);
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
            float4 v = S.V[i];
            if (mix) {
                const float4 f = S.F[i];
                v.x = v.x * cv + f.x * cf; v.y = v.y * cv + f.y * cf; v.z = v.z * cv + f.z * cf;
            } else {
                v = make_float4(0.f, 0.f, 0.f, 0.f);
            }
            S.V[i] = v;
            float4 p = S.P[i];
            p.x += v.x * dtf; p.y += v.y * dtf; p.z += v.z * dtf;
            S.P[i] = p;
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
        for (int i = rank; i < N; i += T) e += (double)S.F[i].w - 0.5 * (double)S.Eh[i];
        energy = team_sum<T>(e, S.red, rank);
    }
    for (int i = rank; i < N; i += T) {
        a.pos[st.atom_off + i] = S.P[i];
        a.vel[st.atom_off + i] = S.V[i];
        if (ran) a.force[st.atom_off + i] = S.F[i];
    }
    if (rank == 0) {
        SlotState& o = a.slots[slot];
        o.dt = dt; o.alpha = alpha; o.npos = npos; o.steps = steps; o.status = status;
        o.energy = energy; o.fmax = fmax;
    }
    team_sync<T>();
}

template <int T, int GDT, bool EVAL>
__global__ void __launch_bounds__(T == 32 ? 128 : T)
relax_kernel(const KernelArgs a) {
    extern __shared__ __align__(16) char smem[];
    const int team = (T == 32) ? (threadIdx.x >> 5) : 0;
    const int rank = (T == 32) ? (threadIdx.x & 31) : threadIdx.x;
    const Smem S = carve(smem + (size_t)team * team_bytes(a.nmax, T), a.nmax, T);
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
        run_system<T, GDT, EVAL>(a, S, w, rank);
    }
}

template <int T, int GDT, bool EVAL>
int launch_t(const KernelArgs& a, cudaStream_t s, int num_sms) {
    const int tpb = (T == 32) ? 4 : 1;           // teams per block
    const int block = T * tpb;
    const size_t smem = (size_t)tpb * team_bytes(a.nmax, T);
    auto kern = relax_kernel<T, GDT, EVAL>;
    static std::map<size_t, int> occ_cache;
    int occ;
    auto it = occ_cache.find(smem);
    if (it == occ_cache.end()) {
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return (int)e;
        }
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, block, smem);
        if (e != cudaSuccess) return (int)e;
        occ_cache[smem] = occ;
    } else {
        occ = it->second;
        if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }
    if (occ < 1) return (int)cudaErrorInvalidConfiguration;
    int blocks_needed = (a.nwork + tpb - 1) / tpb;
    int grid = min(blocks_needed, occ * num_sms);
    if (grid < 1) grid = 1;
    kern<<<grid, block, smem, s>>>(a);
    return (int)cudaGetLastError();
}

template <int GDT, bool EVAL>
int launch_gdt(const KernelArgs& a, int team, cudaStream_t s, int num_sms) {
    switch (team) {
        case 32: return launch_t<32, GDT, EVAL>(a, s, num_sms);
        case 64: return launch_t<64, GDT, EVAL>(a, s, num_sms);
        case 128: return launch_t<128, GDT, EVAL>(a, s, num_sms);
        case 256: return launch_t<256, GDT, EVAL>(a, s, num_sms);
        case 512: return launch_t<512, GDT, EVAL>(a, s, num_sms);
    }
    return (int)cudaErrorInvalidValue;
}

}  // namespace

size_t team_smem_bytes(int nmax) { return team_bytes(nmax, 512); }

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

int launch_relax(const KernelArgs& a, int team, int eval_only, cudaStream_t s, int num_sms, long long* launches) {
    if (a.nwork <= 0) return 0;
    int r;
    const int gdt = a.has_grid ? a.grid.dtype : GRID_F32;
    if (eval_only) {
        r = gdt == GRID_F16 ? launch_gdt<GRID_F16, true>(a, team, s, num_sms)
          : gdt == GRID_BF16 ? launch_gdt<GRID_BF16, true>(a, team, s, num_sms)
          : launch_gdt<GRID_F32, true>(a, team, s, num_sms);
    } else {
        r = gdt == GRID_F16 ? launch_gdt<GRID_F16, false>(a, team, s, num_sms)
          : gdt == GRID_BF16 ? launch_gdt<GRID_BF16, false>(a, team, s, num_sms)
          : launch_gdt<GRID_F32, false>(a, team, s, num_sms);
    }
    if (launches && r == 0) (*launches)++;
    return r;
}

}  // namespace smr
