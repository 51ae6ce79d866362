// Multi-replica rigid-atom relaxation (RAFF / RRsp3, "Current" massfull XPBD ports).
//
// The reference runs one step as three launches over all replicas, every intermediate in global
// memory (opencl/RRsp3.cl:1774-2048: compute_collision_multi, compute_ports_current_multi,
// apply_corrections_multi).  Here one persistent launch runs every step of a call: a team of
// threads (a warp for up to 32 atoms, else a block) owns a replica, keeps its positions,
// quaternions, momenta and per-step corrections in shared memory, and separates the passes of a
// step with team syncs; topology arrays (shared by all replicas) are read through L1.  Global
// memory is touched once per replica and call.  FP32 as the reference; no spin waits.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/surfmol_raff.h"

namespace {

struct RaffTopo {
    int natoms, nnode;
    const float* radius;          // natoms
    const int4* neighs;           // natoms
    const int4* excl1;            // natoms
    const int4* excl2;            // natoms
    const int* fixmask;           // natoms
    const float4* port_local;     // nnode * 4
    const float* kport;           // nnode * 4
    const int4* bk;               // natoms
};

struct RaffState {                // replica-major, as the reference's buffers
    float4* pos;                  // nsys * natoms (w: inverse mass)
    float4* quat;                 // nsys * natoms
    float4* dmom;                 // nsys * natoms
    float4* dqmom;                // nsys * natoms
    float4* coll;                 // nsys * natoms   (last step)
    float4* dnode;                // nsys * nnode    (last step)
    float4* drot;                 // nsys * nnode    (last step)
    float4* dneigh;               // nsys * nnode * 4 (last step)
};

struct RaffArgs {
    RaffTopo t;
    RaffState s;
    int nsys, nsteps, collide;
    float dt, relaxation, beta, rot_mass_scale;
};

__device__ __forceinline__ float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 div3(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }

// rotate v by the unit quaternion q = (x, y, z, w): v + 2w (u x v) + 2 u x (u x v), u = q.xyz
__device__ __forceinline__ float3 qrot(float4 q, float3 v) {
    const float3 u = make_float3(q.x, q.y, q.z);
    const float3 t = cross3(u, v) * 2.0f;
    return v + t * q.w + cross3(u, t);
}
// Hamilton product a b
__device__ __forceinline__ float4 qmul(float4 a, float4 b) {
    return make_float4(a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
                       a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z);
}
__device__ __forceinline__ float4 qnormalize(float4 q) {
    const float n2 = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
    if (n2 < 1e-16f) return make_float4(0.f, 0.f, 0.f, 1.f);
    const float s = rsqrtf(n2);
    return make_float4(q.x * s, q.y * s, q.z * s, q.w * s);
}
// rotation by angle about axis (normalised here), identity for a vanishing axis or angle
__device__ __forceinline__ float4 qaxis_angle(float3 axis, float angle) {
    const float a = sqrtf(dot3(axis, axis));
    if (a < 1e-8f || fabsf(angle) < 1e-8f) return make_float4(0.f, 0.f, 0.f, 1.f);
    const float3 n = div3(axis, a);
    float s, c;
    sincosf(angle * 0.5f, &s, &c);
    return make_float4(n.x * s, n.y * s, n.z * s, c);
}

template <int T> __device__ __forceinline__ void team_sync() {
    if (T == 32) __syncwarp(); else __syncthreads();
}

// Shared memory of one team: pos, quat, dmom, dqmom, coll (natoms each), dnode, drot (nnode each),
// dneigh (4 nnode), all float4.
__host__ __device__ inline size_t team_bytes(int n, int nn) { return ((size_t)5 * n + (size_t)6 * nn) * 16; }

// Sphere collision correction of atom i (compute_collision_multi, RRsp3.cl:1776-1832): Jacobi
// half-split of the overlap with every non-excluded atom, weighted by inverse mass.
__device__ float3 collision(const RaffTopo& t, const float4* P, int i) {
    const int n = t.natoms;
    const float4 pi4 = P[i];
    const float invMi = pi4.w, ri = __ldg(t.radius + i);
    float3 sum = make_float3(0.f, 0.f, 0.f);
    if (!(invMi > 1e-12f) || !(ri > 0.f)) return sum;
    const int4 e1 = __ldg(t.excl1 + i), e2 = __ldg(t.excl2 + i);
    const float3 p = f3(pi4);
    for (int j = 0; j < n; j++) {
        if (j == i) continue;
        if (j == e1.x || j == e1.y || j == e1.z || j == e1.w || j == e2.x || j == e2.y || j == e2.z || j == e2.w) continue;
        const float4 pj4 = P[j];
        const float invMj = pj4.w, rj = __ldg(t.radius + j);
        if (!(invMj > 1e-12f) || !(rj > 0.f)) continue;
        const float3 d = p - f3(pj4);
        const float d2 = dot3(d, d), rsum = ri + rj;
        if (d2 < rsum * rsum && d2 > 1e-16f) {
            const float dist = sqrtf(d2);
            const float3 nv = div3(d, dist);
            float dl = (rsum - dist) / (invMi + invMj + 1e-12f);
            dl *= 0.5f;
            sum = sum + nv * (dl * invMi);
        }
    }
    return sum;
}

// One port of the team (compute_ports_current_multi, RRsp3.cl:1837-1934): task t is slot t & 3 of
// node t >> 2, an XPBD impulse pulling the neighbour onto the port tip xi + R(qi) r_local.  The
// neighbour's recoil goes to the port's slot; the node's translation and rotation parts are
// returned for the 4-lane sum over its slots.
__device__ void port_task(const RaffArgs& a, const float4* P, const float4* Q, float4* dneigh, int t, float3& sdp, float3& sdt) {
    const RaffTopo& tp = a.t;
    const int i = t >> 2, k = t & 3;
    sdp = make_float3(0.f, 0.f, 0.f); sdt = make_float3(0.f, 0.f, 0.f);
    float4* out = dneigh + t;
    *out = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 pi4 = P[i];
    const float invMi = pi4.w;
    if (!(invMi > 1e-12f)) return;
    const int4 ng = __ldg(tp.neighs + i);
    const int j = k == 0 ? ng.x : (k == 1 ? ng.y : (k == 2 ? ng.z : ng.w));
    if (j < 0 || j >= tp.natoms) return;
    const float K = __ldg(tp.kport + t);
    if (!(K > 0.f)) return;
    const float4 pj4 = P[j];
    const float invMj = pj4.w;
    if (!(invMj > 1e-12f)) return;
    const float mi = 1.0f / invMi;
    const float invI = a.rot_mass_scale / (0.4f * mi + 1e-12f);
    const float dt2 = a.dt * a.dt + 1e-16f;
    const float3 r_arm = qrot(Q[i], f3(__ldg(tp.port_local + t)));
    const float3 diff = f3(pj4) - (f3(pi4) + r_arm);
    const float dist2 = dot3(diff, diff);
    if (dist2 < 1e-16f) return;
    const float dist = sqrtf(dist2);
    const float3 nv = div3(diff, dist);
    const float3 rxn = cross3(r_arm, nv);
    const float w_ang = dot3(rxn, rxn) * invI;
    const float alpha = 1.0f / (K * dt2);
    const bool jnode = j < tp.nnode;
    float w_total = invMi + invMj + w_ang + alpha + 1e-12f;
    if (jnode) w_total += w_ang;                       // as the reference: the node's own angular term again
    float imp = dist / w_total;
    if (jnode) imp *= 0.5f;                            // node-node ports act from both ends
    const float3 Pv = nv * imp;
    sdp = Pv * invMi;
    sdt = cross3(r_arm, Pv) * invI;
    const float3 rec = Pv * (-invMj);
    *out = make_float4(rec.x, rec.y, rec.z, 0.f);
}

// All ports of the team: 4 nnode tasks over the team's lanes (the 4 slots of a node on 4
// consecutive lanes of one warp), node sums by two shuffle steps.
template <int T>
__device__ void ports_all(const RaffArgs& a, const float4* P, const float4* Q, float4* dnode, float4* drot, float4* dneigh, int rank) {
    const int ntask = 4 * min(a.t.nnode, a.t.natoms);
    for (int t0 = 0; t0 < ntask; t0 += T) {            // uniform trip count: every lane reaches the shuffles
        const int t = t0 + rank;
        float3 sdp = make_float3(0.f, 0.f, 0.f), sdt = make_float3(0.f, 0.f, 0.f);
        if (t < ntask) port_task(a, P, Q, dneigh, t, sdp, sdt);
        for (int o = 1; o < 4; o <<= 1) {
            sdp.x += __shfl_xor_sync(0xffffffffu, sdp.x, o); sdp.y += __shfl_xor_sync(0xffffffffu, sdp.y, o);
            sdp.z += __shfl_xor_sync(0xffffffffu, sdp.z, o); sdt.x += __shfl_xor_sync(0xffffffffu, sdt.x, o);
            sdt.y += __shfl_xor_sync(0xffffffffu, sdt.y, o); sdt.z += __shfl_xor_sync(0xffffffffu, sdt.z, o);
        }
        if (t < ntask && (t & 3) == 0) {
            dnode[t >> 2] = make_float4(sdp.x, sdp.y, sdp.z, 0.f);
            drot[t >> 2] = make_float4(sdt.x, sdt.y, sdt.z, 0.f);
        }
    }
}

// Correction of atom i (apply_corrections_multi, RRsp3.cl:1939-2046, massless_rot = 0): collision
// plus port translation (own as a node, recoils gathered over its back-slots), fixed axes, Jacobi
// relaxation with heavy-ball momentum; a node also turns by its relaxed rotation vector.
__device__ void correct(const RaffArgs& a, float4* P, float4* Q, float4* M, float4* MQ, const float4* C, const float4* dnode,
                        const float4* drot, const float4* dneigh, int i) {
    const RaffTopo& t = a.t;
    const float4 p = P[i];
    if (!(p.w > 1e-12f)) return;
    const bool isnode = i < t.nnode;
    const float3 dx_coll = a.collide ? f3(C[i]) : make_float3(0.f, 0.f, 0.f);
    float3 dx_port = make_float3(0.f, 0.f, 0.f);
    if (isnode) dx_port = dx_port + f3(dnode[i]);
    const int4 bk = __ldg(t.bk + i);
    if (bk.x >= 0) dx_port = dx_port + f3(dneigh[bk.x]);
    if (bk.y >= 0) dx_port = dx_port + f3(dneigh[bk.y]);
    if (bk.z >= 0) dx_port = dx_port + f3(dneigh[bk.z]);
    if (bk.w >= 0) dx_port = dx_port + f3(dneigh[bk.w]);
    float3 dx = dx_coll + dx_port;
    const int msk = t.fixmask ? __ldg(t.fixmask + i) : 0;
    if (msk & 1) dx.x = 0.f;
    if (msk & 2) dx.y = 0.f;
    if (msk & 4) dx.z = 0.f;
    float3 move = dx * a.relaxation;
    if (a.beta != 0.f) move = move + f3(M[i]) * a.beta;
    if (msk & 8) {                                     // onto the plane z = 0
        if (fabsf(p.z) > 1e-6f) move.z -= p.z; else move.z = 0.f;
    }
    P[i] = make_float4(p.x + move.x, p.y + move.y, p.z + move.z, p.w);
    M[i] = make_float4(move.x, move.y, move.z, 0.f);
    if (!isnode || (msk & 7)) return;
    const float3 dth = f3(drot[i]) * a.relaxation;
    const float angle = sqrtf(dot3(dth, dth));
    const float4 q_old = Q[i];
    float4 q = q_old;
    if (angle > 1e-8f) q = qnormalize(qmul(qaxis_angle(div3(dth, angle), angle), q_old));
    if (a.beta != 0.f) {
        const float4 m = MQ[i];
        q = make_float4(q.x + m.x * a.beta, q.y + m.y * a.beta, q.z + m.z * a.beta, q.w + m.w * a.beta);
    }
    q = qnormalize(q);
    if (q.x * q_old.x + q.y * q_old.y + q.z * q_old.z + q.w * q_old.w < 0.f) q = make_float4(-q.x, -q.y, -q.z, -q.w);
    Q[i] = q;
    MQ[i] = make_float4(q.x - q_old.x, q.y - q_old.y, q.z - q_old.z, q.w - q_old.w);
}

// One team per replica, replicas strided over all teams of the launch (equal work per replica).
template <int T>
__global__ void __launch_bounds__(T == 32 ? 128 : T) raff_kernel(const RaffArgs a) {
    extern __shared__ __align__(16) char smem[];
    constexpr int TPB = T == 32 ? 4 : 1;
    const int team = T == 32 ? (int)(threadIdx.x >> 5) : 0;
    const int rank = T == 32 ? (int)(threadIdx.x & 31) : (int)threadIdx.x;
    const int n = a.t.natoms, nn = a.t.nnode;
    float4* P = (float4*)(smem + (size_t)team * team_bytes(n, nn));
    float4* Q = P + n;
    float4* M = Q + n;
    float4* MQ = M + n;
    float4* C = MQ + n;
    float4* DN = C + n;
    float4* DR = DN + nn;
    float4* DG = DR + nn;
    const int nteams = gridDim.x * TPB;
    for (int r = blockIdx.x * TPB + team; r < a.nsys; r += nteams) {
        const size_t ga = (size_t)r * n, gn = (size_t)r * nn;
        for (int i = rank; i < n; i += T) {
            P[i] = a.s.pos[ga + i]; Q[i] = a.s.quat[ga + i];
            M[i] = a.s.dmom[ga + i]; MQ[i] = a.s.dqmom[ga + i];
            C[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        team_sync<T>();
        for (int it = 0; it < a.nsteps; it++) {
            if (a.collide)
                for (int i = rank; i < n; i += T) { const float3 c = collision(a.t, P, i); C[i] = make_float4(c.x, c.y, c.z, 0.f); }
            ports_all<T>(a, P, Q, DN, DR, DG, rank);
            team_sync<T>();
            for (int i = rank; i < n; i += T) correct(a, P, Q, M, MQ, C, DN, DR, DG, i);
            team_sync<T>();
        }
        for (int i = rank; i < n; i += T) {
            a.s.pos[ga + i] = P[i]; a.s.quat[ga + i] = Q[i];
            a.s.dmom[ga + i] = M[i]; a.s.dqmom[ga + i] = MQ[i];
            if (a.nsteps > 0) a.s.coll[ga + i] = C[i];
        }
        if (a.nsteps > 0)
            for (int i = rank; i < nn; i += T) {
                a.s.dnode[gn + i] = DN[i]; a.s.drot[gn + i] = DR[i];
                for (int k = 0; k < 4; k++) a.s.dneigh[4 * (gn + i) + k] = DG[4 * i + k];
            }
        team_sync<T>();
    }
}

template <int T>
cudaError_t launch_t(const RaffArgs& a, cudaStream_t s, int num_sms) {
    constexpr int TPB = T == 32 ? 4 : 1;
    const size_t smem = (size_t)TPB * team_bytes(a.t.natoms, a.t.nnode);
    auto kern = raff_kernel<T>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    int occ = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, T * TPB, smem);
    if (e != cudaSuccess) return e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    const int blocks = std::max(1, std::min((a.nsys + TPB - 1) / TPB, occ * num_sms));
    kern<<<blocks, T * TPB, smem, s>>>(a);
    return cudaGetLastError();
}

// team size: a warp for up to 32 atoms, else the next power of two up to 1024 threads
cudaError_t launch_raff(const RaffArgs& a, cudaStream_t s, int num_sms) {
    const int n = a.t.natoms;
    if (n <= 32) return launch_t<32>(a, s, num_sms);
    if (n <= 64) return launch_t<64>(a, s, num_sms);
    if (n <= 128) return launch_t<128>(a, s, num_sms);
    if (n <= 256) return launch_t<256>(a, s, num_sms);
    if (n <= 512) return launch_t<512>(a, s, num_sms);
    return launch_t<1024>(a, s, num_sms);
}

}  // namespace

// ================================================================== handle and C ABI
struct smr_raff {
    int device = 0, natoms = 0, nsys = 0, nnode = 0, num_sms = 0;
    bool collide = false, have_topo = false, have_ports = false, have_state = false;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.f;
    std::string err;
    // shared topology
    float* radius = nullptr; int4* neighs = nullptr; int4* excl1 = nullptr; int4* excl2 = nullptr;
    int* fixmask = nullptr; int4* bk = nullptr; float4* port_local = nullptr; float* kport = nullptr;
    // per-replica state and last-step corrections
    float4 *pos = nullptr, *quat = nullptr, *dmom = nullptr, *dqmom = nullptr, *coll = nullptr;
    float4 *dnode = nullptr, *drot = nullptr, *dneigh = nullptr;
};

namespace {

int fail(smr_raff* r, int code, const char* fmt, ...) {
    char buf[400];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    r->err = buf;
    return code;
}

#define RCU(r, x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) return fail(r, SMR_RAFF_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_)); } while (0)

template <class Tp>
int upload(smr_raff* r, Tp* dst, const void* src, size_t bytes) {
    RCU(r, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, r->stream));
    RCU(r, cudaStreamSynchronize(r->stream));
    return SMR_RAFF_OK;
}

// node-port buffers sized for nnode nodes per replica (reallocated when nnode changes)
int alloc_nodes(smr_raff* r, int nnode) {
    cudaFree(r->port_local); cudaFree(r->kport); cudaFree(r->dnode); cudaFree(r->drot); cudaFree(r->dneigh);
    r->port_local = nullptr; r->kport = nullptr; r->dnode = r->drot = r->dneigh = nullptr;
    const size_t nn = (size_t)std::max(nnode, 1), ns = (size_t)r->nsys;
    RCU(r, cudaMalloc(&r->port_local, nn * 4 * 16));
    RCU(r, cudaMalloc(&r->kport, nn * 4 * 4));
    RCU(r, cudaMalloc(&r->dnode, ns * nn * 16));
    RCU(r, cudaMalloc(&r->drot, ns * nn * 16));
    RCU(r, cudaMalloc(&r->dneigh, ns * nn * 4 * 16));
    RCU(r, cudaMemsetAsync(r->dnode, 0, ns * nn * 16, r->stream));
    RCU(r, cudaMemsetAsync(r->drot, 0, ns * nn * 16, r->stream));
    RCU(r, cudaMemsetAsync(r->dneigh, 0, ns * nn * 4 * 16, r->stream));
    RCU(r, cudaStreamSynchronize(r->stream));
    r->nnode = nnode;
    return SMR_RAFF_OK;
}

// rows of one replica (isys >= 0) or of all, float4 -> w floats per row (3 or 4)
int download_rows(smr_raff* r, const float4* src, int rows, int isys, int w, float* out) {
    const size_t first = isys < 0 ? 0 : (size_t)isys * rows, cnt = isys < 0 ? (size_t)r->nsys * rows : (size_t)rows;
    std::vector<float4> h(cnt);
    if (cnt) {
        RCU(r, cudaMemcpyAsync(h.data(), src + first, cnt * 16, cudaMemcpyDeviceToHost, r->stream));
        RCU(r, cudaStreamSynchronize(r->stream));
    }
    for (size_t i = 0; i < cnt; i++) {
        out[w * i] = h[i].x; out[w * i + 1] = h[i].y; out[w * i + 2] = h[i].z;
        if (w == 4) out[w * i + 3] = h[i].w;
    }
    return SMR_RAFF_OK;
}

}  // namespace

extern "C" {

int smr_raff_create(const smr_raff_config* cfg, smr_raff** out) {
    if (!cfg || !out || cfg->natoms < 1 || cfg->natoms > 1024 || cfg->nsys < 1) return SMR_RAFF_ERR_ARG;
    smr_raff* r = new (std::nothrow) smr_raff();
    if (!r) return SMR_RAFF_ERR_ARG;
    r->device = cfg->device; r->natoms = cfg->natoms; r->nsys = cfg->nsys;
    auto bail = [&](int code) { smr_raff_destroy(r); return code; };
    if (cudaSetDevice(r->device) != cudaSuccess) return bail(SMR_RAFF_ERR_CUDA);
    cudaDeviceGetAttribute(&r->num_sms, cudaDevAttrMultiProcessorCount, r->device);
    if (cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(SMR_RAFF_ERR_CUDA);
    if (cudaEventCreate(&r->ev0) != cudaSuccess || cudaEventCreate(&r->ev1) != cudaSuccess) return bail(SMR_RAFF_ERR_CUDA);
    const size_t n = (size_t)r->natoms, ns = (size_t)r->nsys * n;
    if (cudaMalloc(&r->radius, n * 4) || cudaMalloc(&r->neighs, n * 16) || cudaMalloc(&r->excl1, n * 16) ||
        cudaMalloc(&r->excl2, n * 16) || cudaMalloc(&r->fixmask, n * 4) || cudaMalloc(&r->bk, n * 16) ||
        cudaMalloc(&r->pos, ns * 16) || cudaMalloc(&r->quat, ns * 16) || cudaMalloc(&r->dmom, ns * 16) ||
        cudaMalloc(&r->dqmom, ns * 16) || cudaMalloc(&r->coll, ns * 16))
        return bail(SMR_RAFF_ERR_CUDA);
    // the reference's initial state: no collisions, nothing fixed, no back-slots, zero momenta
    if (cudaMemsetAsync(r->radius, 0, n * 4, r->stream) || cudaMemsetAsync(r->fixmask, 0, n * 4, r->stream) ||
        cudaMemsetAsync(r->neighs, 0xff, n * 16, r->stream) || cudaMemsetAsync(r->excl1, 0xff, n * 16, r->stream) ||
        cudaMemsetAsync(r->excl2, 0xff, n * 16, r->stream) || cudaMemsetAsync(r->bk, 0xff, n * 16, r->stream) ||
        cudaMemsetAsync(r->pos, 0, ns * 16, r->stream) || cudaMemsetAsync(r->quat, 0, ns * 16, r->stream) ||
        cudaMemsetAsync(r->dmom, 0, ns * 16, r->stream) || cudaMemsetAsync(r->dqmom, 0, ns * 16, r->stream) ||
        cudaMemsetAsync(r->coll, 0, ns * 16, r->stream) || cudaStreamSynchronize(r->stream))
        return bail(SMR_RAFF_ERR_CUDA);
    if (alloc_nodes(r, 0) != SMR_RAFF_OK) return bail(SMR_RAFF_ERR_CUDA);
    *out = r;
    return SMR_RAFF_OK;
}

int smr_raff_destroy(smr_raff* r) {
    if (!r) return SMR_RAFF_ERR_ARG;
    if (r->stream) cudaStreamSynchronize(r->stream);
    for (void* p : {(void*)r->radius, (void*)r->neighs, (void*)r->excl1, (void*)r->excl2, (void*)r->fixmask, (void*)r->bk,
                    (void*)r->port_local, (void*)r->kport, (void*)r->pos, (void*)r->quat, (void*)r->dmom, (void*)r->dqmom,
                    (void*)r->coll, (void*)r->dnode, (void*)r->drot, (void*)r->dneigh})
        if (p) cudaFree(p);
    if (r->ev0) cudaEventDestroy(r->ev0);
    if (r->ev1) cudaEventDestroy(r->ev1);
    if (r->stream) cudaStreamDestroy(r->stream);
    delete r;
    return SMR_RAFF_OK;
}

const char* smr_raff_last_error(const smr_raff* r) { return r ? r->err.c_str() : "null handle"; }

int smr_raff_upload_radius(smr_raff* r, const float* radius) {
    if (!r || !radius) return SMR_RAFF_ERR_ARG;
    bool any = false;
    for (int i = 0; i < r->natoms; i++) {
        if (!std::isfinite(radius[i]) || radius[i] < 0.f) return fail(r, SMR_RAFF_ERR_ARG, "radius[%d] = %g must be finite and >= 0", i, radius[i]);
        any = any || radius[i] > 0.f;
    }
    r->collide = any;
    if (!any) {                                   // the reference zeroes the collision corrections
        RCU(r, cudaMemsetAsync(r->coll, 0, (size_t)r->nsys * r->natoms * 16, r->stream));
    }
    return upload(r, r->radius, radius, (size_t)r->natoms * 4);
}

int smr_raff_upload_neighs_and_exclusions(smr_raff* r, const int* neighs, const int* excl1, const int* excl2) {
    if (!r || !neighs || !excl1 || !excl2) return SMR_RAFF_ERR_ARG;
    for (int i = 0; i < 4 * r->natoms; i++)
        if (neighs[i] >= r->natoms || excl1[i] >= r->natoms || excl2[i] >= r->natoms)
            return fail(r, SMR_RAFF_ERR_ARG, "neighbour / exclusion entry %d outside [0, %d)", i, r->natoms);
    int e = upload(r, r->neighs, neighs, (size_t)r->natoms * 16);
    if (!e) e = upload(r, r->excl1, excl1, (size_t)r->natoms * 16);
    if (!e) e = upload(r, r->excl2, excl2, (size_t)r->natoms * 16);
    if (!e) r->have_topo = true;
    return e;
}

int smr_raff_upload_fixmask(smr_raff* r, const int* fixmask) {
    if (!r || !fixmask) return SMR_RAFF_ERR_ARG;
    return upload(r, r->fixmask, fixmask, (size_t)r->natoms * 4);
}

int smr_raff_upload_cluster_ports(smr_raff* r, const float* port_local, const float* k, int nnode) {
    if (!r || !port_local || !k) return SMR_RAFF_ERR_ARG;
    if (nnode < 0 || nnode > r->natoms) return fail(r, SMR_RAFF_ERR_ARG, "nnode=%d outside [0, %d]", nnode, r->natoms);
    if (nnode != r->nnode) { int e = alloc_nodes(r, nnode); if (e) return e; }
    int e = nnode ? upload(r, r->port_local, port_local, (size_t)nnode * 4 * 16) : 0;
    if (!e && nnode) e = upload(r, r->kport, k, (size_t)nnode * 4 * 4);
    if (!e) r->have_ports = true;
    return e;
}

int smr_raff_upload_bk_slots(smr_raff* r, const int* bk_slots) {
    if (!r || !bk_slots) return SMR_RAFF_ERR_ARG;
    for (int i = 0; i < 4 * r->natoms; i++)
        if (bk_slots[i] >= 4 * r->nnode) return fail(r, SMR_RAFF_ERR_ARG, "back-slot %d = %d beyond the %d node ports", i, bk_slots[i], 4 * r->nnode);
    return upload(r, r->bk, bk_slots, (size_t)r->natoms * 16);
}

int smr_raff_upload_state(smr_raff* r, const float* pos3, const float* inv_mass, const float* quat) {
    if (!r || !pos3 || !inv_mass) return SMR_RAFF_ERR_ARG;
    const size_t n = (size_t)r->natoms, ns = (size_t)r->nsys * n;
    std::vector<float4> p(ns), q(ns);
    for (size_t k = 0; k < ns; k++) {
        const float w = inv_mass[k % n];
        p[k] = make_float4(pos3[3 * k], pos3[3 * k + 1], pos3[3 * k + 2], w);
        if (w <= 1e-12f) p[k].x = p[k].y = p[k].z = NAN;      // padding atoms, as the reference stores them
        q[k] = quat ? make_float4(quat[4 * k], quat[4 * k + 1], quat[4 * k + 2], quat[4 * k + 3]) : make_float4(0.f, 0.f, 0.f, 1.f);
    }
    int e = upload(r, r->pos, p.data(), ns * 16);
    if (!e) e = upload(r, r->quat, q.data(), ns * 16);
    if (e) return e;
    RCU(r, cudaMemsetAsync(r->dmom, 0, ns * 16, r->stream));
    RCU(r, cudaMemsetAsync(r->dqmom, 0, ns * 16, r->stream));
    RCU(r, cudaStreamSynchronize(r->stream));
    r->have_state = true;
    return SMR_RAFF_OK;
}

int smr_raff_step(smr_raff* r, int nsteps, const smr_raff_step_config* cfg) {
    if (!r || !cfg || nsteps < 0) return SMR_RAFF_ERR_ARG;
    if (!r->have_ports) return fail(r, SMR_RAFF_ERR_STATE, "call smr_raff_upload_cluster_ports first (the reference's kernels are not built before it)");
    if (!r->have_state) return fail(r, SMR_RAFF_ERR_STATE, "no state uploaded");
    if (!(cfg->dt > 0.f) || !std::isfinite(cfg->relaxation) || !std::isfinite(cfg->momentum_beta) || !std::isfinite(cfg->rot_mass_scale))
        return fail(r, SMR_RAFF_ERR_ARG, "step config: dt must be > 0 and the factors finite");
    RaffArgs a{};
    a.t = RaffTopo{r->natoms, r->nnode, r->radius, r->neighs, r->excl1, r->excl2, r->fixmask, r->port_local, r->kport, r->bk};
    a.s = RaffState{r->pos, r->quat, r->dmom, r->dqmom, r->coll, r->dnode, r->drot, r->dneigh};
    a.nsys = r->nsys; a.nsteps = nsteps; a.collide = r->collide ? 1 : 0;
    a.dt = cfg->dt; a.relaxation = cfg->relaxation; a.beta = cfg->momentum_beta; a.rot_mass_scale = cfg->rot_mass_scale;
    if (team_bytes(r->natoms, r->nnode) > 227 * 1024) return fail(r, SMR_RAFF_ERR_ARG, "replica of %d atoms does not fit in shared memory", r->natoms);
    RCU(r, cudaEventRecord(r->ev0, r->stream));
    RCU(r, launch_raff(a, r->stream, r->num_sms));
    RCU(r, cudaEventRecord(r->ev1, r->stream));
    RCU(r, cudaStreamSynchronize(r->stream));
    RCU(r, cudaEventElapsedTime(&r->last_ms, r->ev0, r->ev1));
    return SMR_RAFF_OK;
}

int smr_raff_last_ms(const smr_raff* r, float* ms) {
    if (!r || !ms) return SMR_RAFF_ERR_ARG;
    *ms = r->last_ms;
    return SMR_RAFF_OK;
}

int smr_raff_download_pos(smr_raff* r, int isys, float* pos3) {
    if (!r || !pos3 || isys < -1 || isys >= r->nsys) return SMR_RAFF_ERR_ARG;
    return download_rows(r, r->pos, r->natoms, isys, 3, pos3);
}
int smr_raff_download_quat(smr_raff* r, int isys, float* quat4) {
    if (!r || !quat4 || isys < -1 || isys >= r->nsys) return SMR_RAFF_ERR_ARG;
    return download_rows(r, r->quat, r->natoms, isys, 4, quat4);
}
int smr_raff_download_dpos_coll(smr_raff* r, int isys, float* d3) {
    if (!r || !d3 || isys < -1 || isys >= r->nsys) return SMR_RAFF_ERR_ARG;
    return download_rows(r, r->coll, r->natoms, isys, 3, d3);
}
int smr_raff_download_dpos_node(smr_raff* r, int isys, float* d3) {
    if (!r || !d3 || isys < -1 || isys >= r->nsys) return SMR_RAFF_ERR_ARG;
    return download_rows(r, r->dnode, r->nnode, isys, 3, d3);
}

// ------------------------------------------------------------------ host preparation (pack.rs)
int smr_raff_node_order(int natoms, int nbonds, const int* bonds, int* perm) {
    if (natoms < 0 || nbonds < 0 || (nbonds && !bonds) || !perm) return SMR_RAFF_ERR_ARG;
    std::vector<int> deg(natoms, 0);
    for (int b = 0; b < nbonds; b++) {
        const int i = bonds[2 * b], j = bonds[2 * b + 1];
        if (i < 0 || j < 0 || i >= natoms || j >= natoms) return SMR_RAFF_ERR_ARG;
        if (i == j) continue;
        deg[i]++; deg[j]++;
    }
    int k = 0;
    for (int i = 0; i < natoms; i++) if (deg[i] > 1) perm[k++] = i;
    const int nnode = k;
    for (int i = 0; i < natoms; i++) if (deg[i] <= 1) perm[k++] = i;
    return nnode;
}

int smr_raff_build_neighs(int natoms, int nbonds, const int* bonds, int* neighs) {
    if (natoms < 0 || nbonds < 0 || (nbonds && !bonds) || !neighs) return SMR_RAFF_ERR_ARG;
    std::vector<int> deg(natoms, 0);
    for (int i = 0; i < 4 * natoms; i++) neighs[i] = -1;
    for (int b = 0; b < nbonds; b++) {
        const int i = bonds[2 * b], j = bonds[2 * b + 1];
        if (i < 0 || j < 0 || i >= natoms || j >= natoms) return SMR_RAFF_ERR_ARG;
        if (deg[i] >= 4 || deg[j] >= 4) return SMR_RAFF_ERR_ARG;   // more than 4 bonds on an atom
        neighs[4 * i + deg[i]++] = j;
        neighs[4 * j + deg[j]++] = i;
    }
    return SMR_RAFF_OK;
}

int smr_raff_exclusions(int natoms, const int* neighs, int* excl1, int* excl2) {
    if (natoms < 0 || !neighs || !excl1 || !excl2) return SMR_RAFF_ERR_ARG;
    for (int i = 0; i < natoms; i++) {
        int n1[4], c1 = 0, s2[4], c2 = 0;
        for (int k = 0; k < 4; k++) { excl1[4 * i + k] = -1; excl2[4 * i + k] = -1; }
        for (int k = 0; k < 4; k++) if (neighs[4 * i + k] >= 0) n1[c1++] = neighs[4 * i + k];
        for (int k = 0; k < c1; k++) excl1[4 * i + k] = n1[k];
        // second neighbours: neighbours of neighbours, not i, not a first neighbour, each once, at most 4
        for (int a = 0; a < c1 && c2 < 4; a++)
            for (int k = 0; k < 4 && c2 < 4; k++) {
                const int t = neighs[4 * n1[a] + k];
                if (t < 0 || t == i) continue;
                bool seen = false;
                for (int b = 0; b < c1; b++) seen = seen || n1[b] == t;
                for (int b = 0; b < c2; b++) seen = seen || s2[b] == t;
                if (!seen) s2[c2++] = t;
            }
        for (int k = 0; k < c2; k++) excl2[4 * i + k] = s2[k];
    }
    return SMR_RAFF_OK;
}

int smr_raff_bk_slots(int natoms, int nnode, const int* neighs, int* bk_slots) {
    if (natoms < 0 || nnode < 0 || nnode > natoms || !neighs || !bk_slots) return SMR_RAFF_ERR_ARG;
    std::vector<int> cnt(natoms, 0);
    for (int i = 0; i < 4 * natoms; i++) bk_slots[i] = -1;
    for (int il = 0; il < nnode; il++)
        for (int k = 0; k < 4; k++) {
            const int ja = neighs[4 * il + k];
            if (ja < 0) continue;
            if (ja >= natoms || cnt[ja] >= 4) return SMR_RAFF_ERR_ARG;    // more than 4 back-slots
            bk_slots[4 * ja + cnt[ja]++] = 4 * il + k;
        }
    return SMR_RAFF_OK;
}

int smr_raff_ports(int natoms, const float* pos3, const int* neighs, float k_stiff, float* port_local, float* k) {
    if (natoms < 0 || !pos3 || !neighs || !port_local || !k) return SMR_RAFF_ERR_ARG;
    for (int i = 0; i < natoms; i++)
        for (int s = 0; s < 4; s++) {
            const int j = neighs[4 * i + s];
            float* pl = port_local + 4 * (4 * i + s);
            pl[0] = pl[1] = pl[2] = pl[3] = 0.f;
            k[4 * i + s] = 0.f;
            if (j < 0) continue;
            if (j >= natoms) return SMR_RAFF_ERR_ARG;
            for (int d = 0; d < 3; d++) pl[d] = pos3[3 * j + d] - pos3[3 * i + d];
            k[4 * i + s] = k_stiff;
        }
    return SMR_RAFF_OK;
}

float smr_raff_element_mass(int Z) {
    // standard atomic weights of the elements the reference tabulates
    switch (Z) {
        case 1: return 1.008f;   case 3: return 6.94f;    case 4: return 9.012f;   case 5: return 10.81f;
        case 6: return 12.011f;  case 7: return 14.007f;  case 8: return 15.999f;  case 9: return 18.998f;
        case 10: return 20.180f; case 11: return 22.990f; case 12: return 24.305f; case 13: return 26.982f;
        case 14: return 28.085f; case 15: return 30.974f; case 16: return 32.06f;  case 17: return 35.45f;
        case 18: return 39.948f; case 19: return 39.098f; case 20: return 40.078f; case 26: return 55.845f;
        case 29: return 63.546f; case 30: return 65.38f;  case 35: return 79.904f; case 53: return 126.904f;
        default: return 12.0f;
    }
}

}  // extern "C"
