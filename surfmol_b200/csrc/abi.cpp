// abi.cpp -- the C ABI of include/surfmol_relax.h: handle, device arenas, slot
// allocator, launches and transfers.  Host-side only; kernels live in relax.cu / grid.cu.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/surfmol_relax.h"
#include "smr_internal.h"

using namespace smr;

namespace smr {
int launch_copy_segments(const int* d_src_off, const int* d_len, const int* d_dst_off, int n, const float4* src, float4* dst, cudaStream_t s);
}

namespace {

template <class T>
struct DArr {   // growable device array with a host mirror of the uploaded prefix
    T* d = nullptr;
    size_t cap = 0;
    ~DArr() { if (d) cudaFree(d); }
    // grow to at least n elements keeping the first `keep`; the copy is ordered after earlier
    // uploads on stream s and completes before the old buffer is freed
    cudaError_t reserve(size_t n, size_t keep, cudaStream_t s) {
        if (n <= cap) return cudaSuccess;
        size_t nc = std::max(n, cap * 2 + 1024);
        T* nd = nullptr;
        cudaError_t e = cudaMalloc(&nd, nc * sizeof(T));
        if (e != cudaSuccess) return e;
        if (d && keep) {
            e = cudaMemcpyAsync(nd, d, keep * sizeof(T), cudaMemcpyDeviceToDevice, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) { cudaFree(nd); return e; }
        }
        if (d) cudaFree(d);
        d = nd; cap = nc;
        return cudaSuccess;
    }
};

int default_team(int n) {
    if (n <= 64) return 32;
    if (n <= 160) return 64;
    if (n <= 448) return 128;
    if (n <= 1024) return 256;
    return 512;
}

}  // namespace

struct smr_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    int num_sms = 0;
    size_t smem_optin = 0;
    std::string err;

    int max_systems = 0;
    long long max_atoms = 0;

    // per-atom system state and per-slot state
    float4 *pos = nullptr, *plo = nullptr, *vel = nullptr, *force = nullptr, *stage = nullptr;
    SlotState* slots = nullptr;
    int* work = nullptr;
    int* counter = nullptr;
    double* ecomp = nullptr;
    int* xfer = nullptr;            // 3 * max_systems ints for gather / scatter descriptors
    std::vector<SlotState> hs;      // host mirror of slots
    std::vector<uint32_t> skey;     // per slot: Morton code of the system's lateral centre in the grid cell
    std::vector<int> free_slots;
    std::map<long long, long long> free_atoms;   // offset -> length
    float4* pinned = nullptr;       // staging for uploads / downloads (max_atoms float4)

    // topologies
    std::vector<HostTopo> topos;
    std::vector<char> topo_alive;       // 0 after smr_remove_topology (records dropped at compaction)
    std::vector<size_t> own_len;        // owner-form records of each topology
    size_t dead_atoms = 0;              // arena atoms of removed topologies not yet compacted
    std::vector<TopoDev> htd;
    DArr<TopoDev> dtd;
    std::vector<float4> hreq, hbk, hbl;
    std::vector<short4> hneigh, hneighc;              // neighbour slots, their cell codes
    std::vector<AngRec> hang; std::vector<DihRec> hdih; std::vector<InvRec> hinv;
    DArr<float4> dreq, dbk, dbl; DArr<short4> dneigh, dneighc;
    // per slot: lattice vectors with the images each side in w (3 float4), for slots with pbc set
    std::vector<float4> hlat;
    DArr<float4> dlat;
    DArr<float4> dcons;                 // per state atom 2 float4: constraint target (+ on) and stiffness
    DArr<float4> dtdrive;               // per slot: Langevin drive (T, gamma, seed increment per step, seed)
    DArr<AngRec> dang; DArr<DihRec> ddih; DArr<InvRec> dinv;
    std::vector<int2> ha2f; std::vector<int> hidx;      // gather form: per atom (start, count), piece indices
    DArr<int2> da2f; DArr<int> didx;
    std::vector<short4> hown_geo; std::vector<float4> hown_par; std::vector<int> hown_meta;   // owner form
    DArr<short4> down_geo; DArr<float4> down_par; DArr<int> down_meta;
    size_t up_atoms = 0, up_ang = 0, up_dih = 0, up_inv = 0, up_topo = 0, up_idx = 0, up_own = 0;   // uploaded prefixes
    std::map<int, int> team_override;   // max_atoms -> threads
    // schedule: stage k runs FIRE steps [stage_start[k], stage_start[k+1]) in stage_form[k] with
    // stage_team[k] threads per system (0: the form's default for the system's size)
    std::vector<int> stage_start{0};
    std::vector<int> stage_team{0};
    std::vector<int> stage_form{FORM_ROUNDS};
    int eval_form = FORM_ROUNDS;        // form and team (0: by size) of smr_eval_forces
    int eval_team = 0;
    int nb_lanes = 0;                   // tuning: lanes per atom of the NB loop (0: by size)
    // watchdog: the longest a call waits for its device work; a call that gives up returns
    // SMR_ERR_TIMEOUT with the work still running and marks the handle pending, and the next call
    // first waits for it (again bounded) and refreshes the host copy of the slot table
    double watchdog_s = 3600.0;
    bool pending = false;
    // NB neighbour lists for systems of at least nbl_min atoms under a cutoff (0: off)
    int nbl_min = 128, nbl_cap = 256, nbl_skin_ma = 1000;
    DArr<unsigned short> nbl; DArr<int> nbl_cnt; DArr<float4> nbl_ref;
    bool nbl_ready = false;

    // grid
    void* grid = nullptr;
    int grid_dtype = GRID_F32;
    int gdim[3] = {0, 0, 0};
    double gp0[3] = {0, 0, 0}, gstep[3] = {1, 1, 1};
    float gscale[4] = {1, 1, 1, 1};
    std::vector<float> gzscale;         // 16-bit grids: nz x 4 per-plane channel scales (empty: gscale)
    DArr<float4> dzscale;
    bool has_grid = false;
    // brick copy of the grid for the stencil reads (build_grid_bricks): rebuilt lazily before a
    // launch whenever the grid changed; brick_mode -1 = on for grids larger than L2, 0 off, 1 on
    unsigned long long grid_version = 0, brick_version = ~0ull;
    void* bricks = nullptr;
    size_t bricks_cap = 0;
    int brick_mode = -1;
    bool use_bricks = false;
    // 16-bit grid with FP32 near-surface planes (smr_convert_grid_split): the planes
    // [0, grid_zsplit + 3) of the FP32 grid it came from (z-fastest), their channel scales, and
    // their brick copy (built with the grid's); grid_zsplit = 0: none
    float4* grid_lo = nullptr;
    int grid_zsplit = 0;
    float glo_scale[4] = {1, 1, 1, 1};
    void* bricks_lo = nullptr;
    size_t bricks_lo_cap = 0;
    int grid_prefetch = 0;
    int smem_carveout = -1;             // block teams' preferred shared-memory carveout (%), -1 driver default
    int occ_tiers = 0;                  // split launch segments by the occupancy a system's size allows
    // folded surface: while set it is the substrate in place of the grid
    bool fold_on = false;
    int fold_n[3] = {0, 0, 0};
    float fold_inv[4] = {0, 0, 0, 0}, fold_inv_lo[4] = {0, 0, 0, 0};
    float fold_alpha = 2.f, fold_fmax = 100.f;
    DArr<float> dfold_k;                // kx, ky, kz, z0
    DArr<float4> dfold_coef;            // (cq, cp, cl, 0) per basis function

    smr_nb_params nb{1.0f, 1.5f, 0.0f, 0};

    DArr<char> gscr;                    // team state of systems too large for shared memory
    // graph replay of the batched launch sequence: when a call repeats the previous call's launch
    // plan (same systems, stages, segments and arguments) the plan is captured once and replayed
    bool graph_on = false;
    std::vector<long long> g_sig;          // plan of the captured graph
    cudaGraphExec_t g_exec = nullptr;
    long long g_launches = 0, g_replays = 0;
    int* work_pinned = nullptr;          // per-stage work lists (pinned: captured copies read them)
    size_t work_pinned_cap = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // the launch segments of one schedule stage (disjoint sets of systems, one team size each) run
    // concurrently on side streams, so one class's tail overlaps the next class's work
    static constexpr int kSide = 4;
    cudaStream_t side[kSide] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[kSide] = {};
    double last_ms = 0.0;
    long long last_launches = 0;
};

namespace {

int fail(smr_handle* h, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (h) h->err = buf;
    return code;
}

#define CU(h, x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) return fail(h, SMR_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_)); } while (0)

int team_for(const smr_handle* h, int n) {
    for (auto& kv : h->team_override) if (n <= kv.first) return kv.second;
    return default_team(n);
}

// a topology's records in every kernel form, prepared off the handle (thread-safe)
struct PreparedTopo { int team = 32; PackedTerms P; FlatTerms F; OwnerTerms O; bool own_ok = false; };

void prepare_topology(const HostTopo& T, int team, PreparedTopo& p) {
    p.team = team;
    pack_rounds(T, team, p.P);
    flat_terms(T, p.F);
    p.own_ok = owner_terms(T, p.O);
}

// run f(i) for i in [0, n) on the host cores
template <class F>
void parallel_for(int n, F f) {
    const int nt = std::max(1, std::min<int>(n, (int)std::thread::hardware_concurrency()));
    if (nt <= 1 || n < 4) { for (int i = 0; i < n; i++) f(i); return; }
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; t++)
        pool.emplace_back([&]() { for (int i = next++; i < n; i = next++) f(i); });
    for (auto& th : pool) th.join();
}

void commit_topology(smr_handle* h, const HostTopo& T, const PreparedTopo& pt);

// append a topology's device records (packed for its team) to the arenas
void append_topology(smr_handle* h, const HostTopo& T) {
    PreparedTopo p;
    prepare_topology(T, team_for(h, T.n), p);
    commit_topology(h, T, p);
}

void commit_topology(smr_handle* h, const HostTopo& T, const PreparedTopo& pt) {
    TopoDev td{};
    td.natoms = T.n;
    td.atom_off = (int)h->hreq.size();
    td.team = pt.team;
    td.pbc_bonds = 0;
    for (int c : T.neighc) if (c) td.pbc_bonds = 1;
    for (int a = 0; a < T.n; a++) {
        const double* r = &T.req[4 * a];
        h->hreq.push_back(make_float4((float)r[0], (float)r[1], (float)r[2], (float)r[3]));
        h->hneigh.push_back(make_short4((short)T.neighs[4 * a], (short)T.neighs[4 * a + 1], (short)T.neighs[4 * a + 2], (short)T.neighs[4 * a + 3]));
        if (T.neighc.empty()) h->hneighc.push_back(make_short4(0, 0, 0, 0));
        else h->hneighc.push_back(make_short4((short)T.neighc[4 * a], (short)T.neighc[4 * a + 1], (short)T.neighc[4 * a + 2], (short)T.neighc[4 * a + 3]));
        const double* kl = &T.bond_kl[8 * a];
        h->hbk.push_back(make_float4((float)kl[0], (float)kl[2], (float)kl[4], (float)kl[6]));
        h->hbl.push_back(make_float4((float)kl[1], (float)kl[3], (float)kl[5], (float)kl[7]));
    }
    const PackedTerms& P = pt.P;
    td.ang_off = (int)h->hang.size(); td.ang_rounds = P.ang_rounds; h->hang.insert(h->hang.end(), P.ang.begin(), P.ang.end());
    td.dih_off = (int)h->hdih.size(); td.dih_rounds = P.dih_rounds; h->hdih.insert(h->hdih.end(), P.dih.begin(), P.dih.end());
    td.inv_off = (int)h->hinv.size(); td.inv_rounds = P.inv_rounds; h->hinv.insert(h->hinv.end(), P.inv.begin(), P.inv.end());
    const FlatTerms& F = pt.F;
    td.nang = (int)F.ang.size(); td.ndih = (int)F.dih.size(); td.ninv = (int)F.inv.size(); td.npieces = F.npieces;
    td.fang_off = (int)h->hang.size(); h->hang.insert(h->hang.end(), F.ang.begin(), F.ang.end());
    td.fdih_off = (int)h->hdih.size(); h->hdih.insert(h->hdih.end(), F.dih.begin(), F.dih.end());
    td.finv_off = (int)h->hinv.size(); h->hinv.insert(h->hinv.end(), F.inv.begin(), F.inv.end());
    td.a2f_off = (int)h->hidx.size();
    h->ha2f.insert(h->ha2f.end(), F.a2f.begin(), F.a2f.end());
    h->hidx.insert(h->hidx.end(), F.idx.begin(), F.idx.end());
    const OwnerTerms& O = pt.O;
    td.own_ok = pt.own_ok ? 1 : 0;
    if (td.own_ok) {
        td.own_a_off = (int)h->hown_geo.size();
        td.own_i_off = td.own_a_off + O.rows_a * T.n;
        td.own_d_off = td.own_i_off + O.rows_i * T.n;
        h->hown_geo.insert(h->hown_geo.end(), O.geo.begin(), O.geo.end());
        h->hown_par.insert(h->hown_par.end(), O.par.begin(), O.par.end());
        h->hown_meta.insert(h->hown_meta.end(), O.meta.begin(), O.meta.end());
    } else {
        h->hown_meta.insert(h->hown_meta.end(), T.n, 0);
    }
    h->htd.push_back(td);
    h->own_len.push_back(pt.own_ok ? pt.O.geo.size() : 0);
}

// the arena record of a removed topology (kept so that topology ids stay stable)
void commit_dead(smr_handle* h) {
    TopoDev td{};
    td.atom_off = (int)h->hreq.size();
    td.team = 32;
    h->htd.push_back(td);
    h->own_len.push_back(0);
}

template <class T>
cudaError_t sync_arr(DArr<T>& d, const std::vector<T>& hv, size_t& up, cudaStream_t s) {
    if (hv.size() == up) return cudaSuccess;
    cudaError_t e = d.reserve(hv.size(), up, s);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(d.d + up, hv.data() + up, (hv.size() - up) * sizeof(T), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) up = hv.size();
    return e;
}

int upload_all(smr_handle* h) {
    cudaStream_t s = h->stream;
    size_t ua = h->up_atoms;
    size_t t;
    t = ua; CU(h, sync_arr(h->dreq, h->hreq, t, s));
    t = ua; CU(h, sync_arr(h->dneigh, h->hneigh, t, s));
    t = ua; CU(h, sync_arr(h->dneighc, h->hneighc, t, s));
    t = ua; CU(h, sync_arr(h->dbk, h->hbk, t, s));
    t = ua; CU(h, sync_arr(h->dbl, h->hbl, t, s));
    t = ua; CU(h, sync_arr(h->da2f, h->ha2f, t, s));
    t = ua; CU(h, sync_arr(h->down_meta, h->hown_meta, t, s));
    h->up_atoms = h->hreq.size();
    t = h->up_own; CU(h, sync_arr(h->down_geo, h->hown_geo, t, s));
    t = h->up_own; CU(h, sync_arr(h->down_par, h->hown_par, t, s));
    h->up_own = h->hown_geo.size();
    CU(h, sync_arr(h->didx, h->hidx, h->up_idx, s));
    CU(h, sync_arr(h->dang, h->hang, h->up_ang, s));
    CU(h, sync_arr(h->ddih, h->hdih, h->up_dih, s));
    CU(h, sync_arr(h->dinv, h->hinv, h->up_inv, s));
    CU(h, sync_arr(h->dtd, h->htd, h->up_topo, s));
    return 0;
}

// repack every topology for the current team mapping (after smr_set_team_size)
int repack_all(smr_handle* h) {
    h->htd.clear(); h->hreq.clear(); h->hneigh.clear(); h->hneighc.clear(); h->hbk.clear(); h->hbl.clear();
    h->hang.clear(); h->hdih.clear(); h->hinv.clear(); h->ha2f.clear(); h->hidx.clear();
    h->hown_geo.clear(); h->hown_par.clear(); h->hown_meta.clear();
    h->up_atoms = h->up_ang = h->up_dih = h->up_inv = h->up_topo = h->up_idx = h->up_own = 0;
    h->own_len.clear();
    h->dead_atoms = 0;
    std::vector<PreparedTopo> prep(h->topos.size());
    parallel_for((int)prep.size(), [&](int i) {
        if (h->topo_alive[i]) prepare_topology(h->topos[i], team_for(h, h->topos[i].n), prep[i]);
    });
    for (size_t i = 0; i < prep.size(); i++) {
        if (h->topo_alive[i]) commit_topology(h, h->topos[i], prep[i]);
        else commit_dead(h);
    }
    return upload_all(h);
}

// Drop the records of removed topologies from every arena: each live topology's ranges are
// copied in id order into fresh host mirrors, its offsets updated, and everything re-uploaded.
int compact_topologies(smr_handle* h) {
    smr_handle& o = *h;
    std::vector<float4> req, bk, bl; std::vector<short4> neigh, neighc; std::vector<int2> a2f; std::vector<int> meta, idx;
    std::vector<AngRec> ang; std::vector<DihRec> dih; std::vector<InvRec> inv;
    std::vector<short4> geo; std::vector<float4> par;
    auto cp = [](auto& dst, const auto& src, size_t off, size_t n) { dst.insert(dst.end(), src.begin() + off, src.begin() + off + n); };
    for (size_t id = 0; id < o.htd.size(); id++) {
        TopoDev& td = o.htd[id];
        if (!o.topo_alive[id]) { td = TopoDev{}; td.atom_off = (int)req.size(); td.team = 32; o.own_len[id] = 0; continue; }
        const size_t n = td.natoms, a0 = td.atom_off;
        td.atom_off = (int)req.size();
        cp(req, o.hreq, a0, n); cp(neigh, o.hneigh, a0, n); cp(neighc, o.hneighc, a0, n); cp(bk, o.hbk, a0, n); cp(bl, o.hbl, a0, n);
        cp(a2f, o.ha2f, a0, n); cp(meta, o.hown_meta, a0, n);
        const size_t T = td.team;
        size_t x;
        x = td.ang_off; td.ang_off = (int)ang.size(); cp(ang, o.hang, x, td.ang_rounds * T);
        x = td.fang_off; td.fang_off = (int)ang.size(); cp(ang, o.hang, x, td.nang);
        x = td.dih_off; td.dih_off = (int)dih.size(); cp(dih, o.hdih, x, td.dih_rounds * T);
        x = td.fdih_off; td.fdih_off = (int)dih.size(); cp(dih, o.hdih, x, td.ndih);
        x = td.inv_off; td.inv_off = (int)inv.size(); cp(inv, o.hinv, x, td.inv_rounds * T);
        x = td.finv_off; td.finv_off = (int)inv.size(); cp(inv, o.hinv, x, td.ninv);
        x = td.a2f_off; td.a2f_off = (int)idx.size(); cp(idx, o.hidx, x, td.npieces);
        if (td.own_ok) {
            const int shift = (int)geo.size() - td.own_a_off;
            cp(geo, o.hown_geo, td.own_a_off, o.own_len[id]); cp(par, o.hown_par, td.own_a_off, o.own_len[id]);
            td.own_a_off += shift; td.own_i_off += shift; td.own_d_off += shift;
        }
    }
    o.hreq.swap(req); o.hneigh.swap(neigh); o.hneighc.swap(neighc); o.hbk.swap(bk); o.hbl.swap(bl); o.ha2f.swap(a2f); o.hown_meta.swap(meta);
    o.hang.swap(ang); o.hdih.swap(dih); o.hinv.swap(inv); o.hidx.swap(idx); o.hown_geo.swap(geo); o.hown_par.swap(par);
    o.up_atoms = o.up_ang = o.up_dih = o.up_inv = o.up_topo = o.up_idx = o.up_own = 0;
    o.dead_atoms = 0;
    return upload_all(h);
}

long long alloc_atoms(smr_handle* h, long long n) {
    for (auto it = h->free_atoms.begin(); it != h->free_atoms.end(); ++it) {
        if (it->second >= n) {
            long long off = it->first, len = it->second;
            h->free_atoms.erase(it);
            if (len > n) h->free_atoms[off + n] = len - n;
            return off;
        }
    }
    return -1;
}

void free_atoms(smr_handle* h, long long off, long long n) {
    auto it = h->free_atoms.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != h->free_atoms.end() && it->first + it->second == nx->first) { it->second += nx->second; h->free_atoms.erase(nx); }
    if (it != h->free_atoms.begin()) {
        auto pv = std::prev(it);
        if (pv->first + pv->second == it->first) { pv->second += it->second; h->free_atoms.erase(it); }
    }
}

bool valid_slot(const smr_handle* h, int s) { return s >= 0 && s < h->max_systems && h->hs[s].active; }

int wait_stream(smr_handle* h, double timeout_s) {
    cudaEvent_t e;
    CU(h, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cudaEventRecord(e, h->stream);
    auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t q = cudaEventQuery(e);
        if (q == cudaSuccess) break;
        if (q != cudaErrorNotReady) { cudaEventDestroy(e); return fail(h, SMR_ERR_CUDA, "stream: %s", cudaGetErrorString(q)); }
        double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (dt > timeout_s) {
            cudaEventDestroy(e);
            h->pending = true;
            return fail(h, SMR_ERR_TIMEOUT, "device work not finished after %.3f s (the handle waits for it on the next call)", timeout_s);
        }
        std::this_thread::sleep_for(std::chrono::microseconds(dt < 0.01 ? 5 : 200));
    }
    cudaEventDestroy(e);
    return 0;
}

int download_slots(smr_handle* h) {
    CU(h, cudaMemcpyAsync(h->hs.data(), h->slots, h->hs.size() * sizeof(SlotState), cudaMemcpyDeviceToHost, h->stream));
    return wait_stream(h, h->watchdog_s);
}

// after a watchdog timeout: wait for the abandoned work (bounded), then refresh the slot table
int settle(smr_handle* h) {
    if (!h->pending) return 0;
    int r = wait_stream(h, h->watchdog_s);
    if (r) return r;
    h->pending = false;
    return download_slots(h);
}
#define SETTLE(h) do { int r_ = settle(h); if (r_) return r_; } while (0)

int upload_slots(smr_handle* h, const std::vector<int>& ids) {
    if (ids.size() > 32) {   // many slots: one copy of the whole table
        CU(h, cudaMemcpyAsync(h->slots, h->hs.data(), h->hs.size() * sizeof(SlotState), cudaMemcpyHostToDevice, h->stream));
        return wait_stream(h, h->watchdog_s);   // hs is pageable host memory: finish before it can change
    }
    for (int s : ids) CU(h, cudaMemcpyAsync(h->slots + s, &h->hs[s], sizeof(SlotState), cudaMemcpyHostToDevice, h->stream));
    return wait_stream(h, h->watchdog_s);
}

// The brick copy of the grid, (re)built when the grid changed since the last build; the grid of
// base_args is then the copy.  Off for the folded surface, for grids up to 128 MiB in auto mode
// (those stay in L2 and the 8x larger copy would not), and where the copy cannot be indexed.
int ensure_bricks(smr_handle* h) {
    h->use_bricks = false;
    if (!h->has_grid || h->fold_on || h->brick_mode == 0) return 0;
    const int nx = h->gdim[0], ny = h->gdim[1], nz = h->gdim[2];
    const size_t plain = (size_t)nx * ny * nz * (h->grid_dtype == SMR_GRID_F32 ? 16 : 8);
    if (h->brick_mode < 0 && plain <= (128u << 20)) return 0;
    const size_t bytes = grid_brick_bytes(nx, ny, nz);
    if (!bytes) return 0;
    if (h->bricks && h->brick_version == h->grid_version) { h->use_bricks = true; return 0; }
    if (bytes > h->bricks_cap) {
        if (h->bricks) { CU(h, cudaStreamSynchronize(h->stream)); cudaFree(h->bricks); h->bricks = nullptr; h->bricks_cap = 0; }
        cudaError_t e = cudaMalloc(&h->bricks, bytes);
        if (e != cudaSuccess) { h->bricks = nullptr; return fail(h, SMR_ERR_CAPACITY, "grid bricks (%zu bytes): %s", bytes, cudaGetErrorString(e)); }
        h->bricks_cap = bytes;
    }
    { const int e = build_grid_bricks(h->grid, h->grid_dtype, nx, ny, nz, h->bricks, h->stream);
      if (e) return fail(h, SMR_ERR_CUDA, "grid bricks: %s", cudaGetErrorString((cudaError_t)e)); }
    if (h->grid_zsplit > 0) {
        // the FP32 near-surface planes in the same layout
        const int nzl = h->grid_zsplit + 3;
        const size_t lb = grid_brick_bytes(nx, ny, nzl);
        if (!lb) return fail(h, SMR_ERR_CAPACITY, "grid bricks of the FP32 planes cannot be indexed");
        if (lb > h->bricks_lo_cap) {
            if (h->bricks_lo) { CU(h, cudaStreamSynchronize(h->stream)); cudaFree(h->bricks_lo); h->bricks_lo = nullptr; h->bricks_lo_cap = 0; }
            cudaError_t e = cudaMalloc(&h->bricks_lo, lb);
            if (e != cudaSuccess) { h->bricks_lo = nullptr; return fail(h, SMR_ERR_CAPACITY, "grid bricks of the FP32 planes (%zu bytes): %s", lb, cudaGetErrorString(e)); }
            h->bricks_lo_cap = lb;
        }
        const int e = build_grid_bricks(h->grid_lo, SMR_GRID_F32, nx, ny, nzl, h->bricks_lo, h->stream);
        if (e) return fail(h, SMR_ERR_CUDA, "grid bricks of the FP32 planes: %s", cudaGetErrorString((cudaError_t)e));
    }
    h->brick_version = h->grid_version;
    h->use_bricks = true;
    return 0;
}

KernelArgs base_args(smr_handle* h) {
    KernelArgs a{};
    a.counter = h->counter;
    a.slots = h->slots;
    a.topos = h->dtd.d;
    a.req = h->dreq.d; a.neigh = h->dneigh.d; a.bk = h->dbk.d; a.bl = h->dbl.d;
    a.neighc = h->dneighc.d; a.lat = h->dlat.d; a.cons = h->dcons.d; a.tdrive = h->dtdrive.d;
    a.angs = h->dang.d; a.dihs = h->ddih.d; a.invs = h->dinv.d;
    a.a2f = h->da2f.d; a.a2f_idx = h->didx.d;
    a.own_geo = h->down_geo.d; a.own_par = h->down_par.d; a.own_meta = h->down_meta.d;
    a.nb_lanes = h->nb_lanes;
    if (h->nbl_ready) {
        a.nbl = h->nbl.d; a.nbl_cnt = h->nbl_cnt.d; a.nbl_ref = h->nbl_ref.d;
        a.nbl_cap = h->nbl_cap; a.nbl_min = h->nbl_min; a.nbl_skin = 1e-3f * (float)h->nbl_skin_ma;
    }
    a.pos = h->pos; a.plo = h->plo; a.vel = h->vel; a.force = h->force;
    a.has_grid = h->has_grid ? 1 : 0;
    a.grid.data = h->use_bricks ? h->bricks : h->grid;
    a.grid.brick = h->use_bricks ? 1 : 0;
    a.grid.dtype = h->grid_dtype;
    a.grid.nx = h->gdim[0]; a.grid.ny = h->gdim[1]; a.grid.nz = h->gdim[2];
    for (int k = 0; k < 3; k++) { a.grid.p0[k] = (float)h->gp0[k]; a.grid.inv_step[k] = (float)(1.0 / h->gstep[k]); }
    for (int k = 0; k < 4; k++) a.grid.scale[k] = h->has_grid ? h->gscale[k] : 1.f;
    a.grid.zscale = (h->has_grid && !h->gzscale.empty()) ? h->dzscale.d : nullptr;
    a.grid.p0z = h->gp0[2]; a.grid.stepz = h->gstep[2];
    if (h->has_grid && h->grid_zsplit > 0) {
        a.grid.lo = h->use_bricks ? h->bricks_lo : (const void*)h->grid_lo;
        a.grid.zsplit = h->grid_zsplit; a.grid.lo_nz = h->grid_zsplit + 3;
        for (int k = 0; k < 4; k++) a.grid.lo_scale[k] = h->glo_scale[k];
    }
    if (h->fold_on) {
        a.fold.on = 1;
        a.fold.nx = h->fold_n[0]; a.fold.ny = h->fold_n[1]; a.fold.nz = h->fold_n[2];
        for (int k = 0; k < 4; k++) { a.fold.inv[k] = h->fold_inv[k]; a.fold.inv_lo[k] = h->fold_inv_lo[k]; }
        a.fold.alpha = h->fold_alpha; a.fold.fmax = h->fold_fmax;
        a.fold.k = h->dfold_k.d; a.fold.coef = h->dfold_coef.d;
    }
    a.R2damp = h->nb.rdamp * h->nb.rdamp;
    a.alpha_morse = h->nb.alpha_morse;
    a.rc2 = h->nb.rcut > 0 ? h->nb.rcut * h->nb.rcut : 3.0e38f;
    a.excl13 = h->nb.excl13 ? 1 : 0;
    a.grid_prefetch = h->grid_prefetch;
    a.smem_carveout = h->smem_carveout;
    return a;
}

// group slots by launch configuration; returns (team, form, begin, end, nmax, nfmax) segments
struct Seg { int team, form, begin, end, nmax, nfmax; bool gstate; };   // gstate: team state in global memory

int latency_team_for(int requested, int n) {
    if (requested) return requested;
    return n <= 64 ? 128 : (n <= 200 ? 256 : 512);
}

// Launch segments for a list of slots.  The form of every system is decided from the system
// alone (the requested form when the topology supports it and its own shared memory fits, else
// the rounds form with its topology's team; periodic or constrained systems, and all systems
// under 1-3 exclusion, always the extended gather form), never from what it is batched with; segments group
// equal (form, team) and are split wherever the segment's largest system would no longer fit.
std::vector<Seg> group_by(smr_handle* h, std::vector<int>& ids, int form, int req_team = 0) {
    struct Key { int form, team, n, nf, tier; };
    auto key_of = [&](int s) {
        const SlotState& st = h->hs[s];
        const TopoDev& td = h->htd[st.topo];
        const int n = st.natoms, nf = td.npieces;
        if (st.flags || h->nb.excl13) {
            // periodic or constrained systems, and every system while 1-3 exclusion is on: the
            // extended gather form, whatever the stage's form
            const int t = req_team ? req_team : td.team;
            if (team_smem_bytes(n, nf, t, FORM_GATHER_EXT) <= h->smem_optin) return Key{FORM_GATHER_EXT, t, n, nf};
            return Key{FORM_GATHER_EXT, std::max(td.team, n > 1024 ? 512 : 256), n, nf};
        }
        if (form == FORM_GATHER) {
            const int t = latency_team_for(req_team, n);
            if (team_smem_bytes(n, nf, t, FORM_GATHER) <= h->smem_optin) return Key{FORM_GATHER, t, n, nf};
        } else if (form == FORM_OWNER && td.own_ok) {
            const int t = req_team ? req_team : td.team;
            if (team_smem_bytes(n, nf, t, FORM_OWNER) <= h->smem_optin) return Key{FORM_OWNER, t, n, nf};
        }
        if (team_smem_bytes(n, nf, td.team, FORM_ROUNDS) <= h->smem_optin) return Key{FORM_ROUNDS, td.team, n, nf};
        // too large for shared memory in any form: the gather form (no per-team packing) with its
        // team state in global memory
        return Key{FORM_GATHER, std::max(td.team, n > 1024 ? 512 : 256), n, nf};
    };
    std::vector<Key> keys(h->max_systems);
    // occupancy tier: the blocks per SM a system's own shared memory allows under the register
    // budget; systems of different tiers run in different segments, so a segment of small systems
    // keeps its occupancy instead of taking the shared memory of the largest system of its team
    for (int s : ids) {
        Key k = key_of(s);
        k.tier = h->occ_tiers ? relax_blocks_per_sm(team_smem_bytes(k.n, k.nf, k.team, k.form), k.team, k.form) : 0;
        keys[s] = k;
    }
    std::stable_sort(ids.begin(), ids.end(), [&](int a, int b) {
        const Key &x = keys[a], &y = keys[b];
        if (x.form != y.form) return x.form < y.form;
        if (x.team != y.team) return x.team < y.team;
        if (x.tier != y.tier) return x.tier > y.tier;
        // systems that run at the same time then cover a small patch of the grid (L2 reuse)
        if (h->skey[a] != h->skey[b]) return h->skey[a] < h->skey[b];
        return x.n < y.n;
    });
    std::vector<Seg> segs;
    for (int i = 0; i < (int)ids.size(); i++) {
        const Key& k = keys[ids[i]];
        if (!segs.empty()) {
            Seg& g = segs.back();
            if (g.form == k.form && g.team == k.team && keys[ids[g.begin]].tier == k.tier &&
                (g.gstate || team_smem_bytes(std::max(g.nmax, k.n), std::max(g.nfmax, k.nf), k.team, k.form) <= h->smem_optin)) {
                g.end = i + 1; g.nmax = std::max(g.nmax, k.n); g.nfmax = std::max(g.nfmax, k.nf);
                continue;
            }
        }
        // a system whose state does not fit in shared memory starts a global-state segment
        const bool gs = team_smem_bytes(k.n, k.nf, k.team, k.form) > h->smem_optin;
        segs.push_back({k.team, k.form, i, i + 1, k.n, k.nf, gs});
    }
    return segs;
}


// Global-memory team state for the segments that do not fit in shared memory: each such segment
// gets its own region (segments of one stage run concurrently) of two blocks' state per SM.
// Returns the bytes needed; off[j] / len[j] are segment j's region (len 0: shared memory).
size_t plan_gscratch(const smr_handle* h, const std::vector<Seg>& segs, std::vector<size_t>& off, std::vector<size_t>& len) {
    size_t tot = 0;
    off.assign(segs.size(), 0);
    len.assign(segs.size(), 0);
    for (size_t j = 0; j < segs.size(); j++) {
        if (!segs[j].gstate) continue;
        const size_t b = (team_smem_bytes(segs[j].nmax, segs[j].nfmax, segs[j].team, segs[j].form) + 255) & ~size_t(255);
        off[j] = tot;
        len[j] = b * 2 * (size_t)h->num_sms;
        tot += len[j];
    }
    return tot;
}

int reserve_gscratch(smr_handle* h, size_t bytes) {
    cudaError_t e = h->gscr.reserve(bytes, 0, h->stream);
    if (e != cudaSuccess) return fail(h, SMR_ERR_CAPACITY, "global team state of %zu B: %s", bytes, cudaGetErrorString(e));
    return 0;
}

// a batch of slots must be distinct, active and fit the staging buffers
int check_batch(smr_handle* h, int nsys, const int* ids) {
    if (nsys > h->max_systems) return fail(h, SMR_ERR_CAPACITY, "%d slots requested, capacity %d", nsys, h->max_systems);
    std::vector<char> seen(h->max_systems, 0);
    for (int i = 0; i < nsys; i++) {
        int s = ids[i];
        if (!valid_slot(h, s)) return fail(h, SMR_ERR_ARG, "slot %d not active", s);
        if (seen[s]) return fail(h, SMR_ERR_ARG, "slot %d listed twice", s);
        seen[s] = 1;
    }
    return 0;
}

// excl13 (1-3 exclusion) is defined for systems without PBC images only
int check_excl13(smr_handle* h, const int* ids, int n) {
    if (!h->nb.excl13 || h->hlat.empty()) return 0;
    for (int i = 0; i < n; i++) {
        const int s = ids[i];
        if (!(h->hs[s].flags & SLOT_PBC)) continue;
        const float4* L = &h->hlat[3 * (size_t)s];
        if (L[0].w + L[1].w + L[2].w > 0.f)
            return fail(h, SMR_ERR_ARG, "slot %d has PBC images: 1-3 exclusion (excl13) is defined for systems without images", s);
    }
    return 0;
}

}  // namespace

// ====================================================================== API
extern "C" {

const char* smr_version(void) { return "surfmol_b200 0.1 (sm_100a)"; }

const char* smr_last_error(const smr_handle* h) { return h ? h->err.c_str() : "null handle"; }

int smr_create(const smr_config* cfg, smr_handle** out) {
    if (!cfg || !out) return SMR_ERR_ARG;
    *out = nullptr;
    if (cfg->max_systems <= 0 || cfg->max_atoms <= 0 || cfg->max_atoms > (1LL << 31) - 1) return SMR_ERR_ARG;
    smr_handle* h = new (std::nothrow) smr_handle();
    if (!h) return SMR_ERR_CAPACITY;
    h->device = cfg->device;
    h->max_systems = cfg->max_systems;
    h->max_atoms = cfg->max_atoms;
    auto bail = [&](int code) { smr_destroy(h); return code; };
    if (cudaSetDevice(h->device) != cudaSuccess) return bail(SMR_ERR_CUDA);
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, h->device); h->num_sms = v;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device); h->smem_optin = (size_t)v;
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(SMR_ERR_CUDA);
    size_t na = (size_t)cfg->max_atoms, ns = (size_t)cfg->max_systems;
    if (cudaMalloc(&h->pos, na * 16) || cudaMalloc(&h->plo, na * 16) || cudaMalloc(&h->vel, na * 16) || cudaMalloc(&h->force, na * 16) ||
        cudaMalloc(&h->stage, na * 16) || cudaMalloc(&h->slots, ns * sizeof(SlotState)) ||
        cudaMalloc(&h->work, ns * 4) || cudaMalloc(&h->counter, 64) || cudaMalloc(&h->ecomp, ns * 8 * 8) ||
        cudaMalloc(&h->xfer, ns * 3 * 4) || cudaMallocHost(&h->pinned, na * 16))
        return bail(SMR_ERR_CUDA);
    // zeroed on the handle's stream (a legacy-stream memset is not ordered with it)
    if (cudaMemsetAsync(h->slots, 0, ns * sizeof(SlotState), h->stream) || cudaMemsetAsync(h->vel, 0, na * 16, h->stream) ||
        cudaMemsetAsync(h->plo, 0, na * 16, h->stream) || cudaStreamSynchronize(h->stream))
        return bail(SMR_ERR_CUDA);
    h->hs.assign(ns, SlotState{});
    h->skey.assign(ns, 0u);
    h->hlat.assign(3 * (size_t)ns, make_float4(0.f, 0.f, 0.f, 0.f));
    for (int s = (int)ns - 1; s >= 0; s--) h->free_slots.push_back(s);
    h->free_atoms[0] = (long long)na;
    cudaEventCreate(&h->ev0);
    cudaEventCreate(&h->ev1);
    if (cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess) return bail(SMR_ERR_CUDA);
    for (int k = 0; k < smr_handle::kSide; k++)
        if (cudaStreamCreateWithFlags(&h->side[k], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->ev_join[k], cudaEventDisableTiming) != cudaSuccess)
            return bail(SMR_ERR_CUDA);
    *out = h;
    return SMR_OK;
}

int smr_destroy(smr_handle* h) {
    if (!h) return SMR_ERR_ARG;
    if (h->stream) cudaStreamSynchronize(h->stream);
    cudaFree(h->pos); cudaFree(h->plo); cudaFree(h->vel); cudaFree(h->force); cudaFree(h->stage); cudaFree(h->slots);
    cudaFree(h->work); cudaFree(h->counter); cudaFree(h->ecomp); cudaFree(h->xfer);
    if (h->pinned) cudaFreeHost(h->pinned);
    if (h->grid) cudaFree(h->grid);
    if (h->bricks) cudaFree(h->bricks);
    if (h->grid_lo) cudaFree(h->grid_lo);
    if (h->bricks_lo) cudaFree(h->bricks_lo);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->g_exec) cudaGraphExecDestroy(h->g_exec);
    if (h->work_pinned) cudaFreeHost(h->work_pinned);
    for (int k = 0; k < smr_handle::kSide; k++) {
        if (h->side[k]) cudaStreamDestroy(h->side[k]);
        if (h->ev_join[k]) cudaEventDestroy(h->ev_join[k]);
    }
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return SMR_OK;
}

int smr_set_nb_params(smr_handle* h, const smr_nb_params* p) {
    if (!h || !p) return SMR_ERR_ARG;
    if (!(p->rdamp >= 0.f) || !(p->alpha_morse > 0.f)) return fail(h, SMR_ERR_ARG, "rdamp must be >= 0 and alpha_morse > 0");
    if (p->excl13 != 0 && p->excl13 != 1) return fail(h, SMR_ERR_ARG, "excl13 must be 0 or 1");
    h->nb = *p;
    return SMR_OK;
}

int smr_set_tuning(smr_handle* h, int key, int value) {
    if (!h) return SMR_ERR_ARG;
    if (key == SMR_TUNE_NB_LANES) {
        if (value != 0 && value != 1 && value != 2 && value != 4 && value != 8 && value != 16 && value != 32)
            return fail(h, SMR_ERR_ARG, "NB lanes per atom must be 0, 1, 2, 4, 8, 16 or 32");
        h->nb_lanes = value;
        return SMR_OK;
    }
    if (key == SMR_TUNE_WATCHDOG_MS) {
        if (value < 1) return fail(h, SMR_ERR_ARG, "watchdog must be at least 1 ms");
        h->watchdog_s = 1e-3 * value;
        return SMR_OK;
    }
    if (key == SMR_TUNE_NBLIST_MIN) {
        if (value < 0) return fail(h, SMR_ERR_ARG, "neighbour-list size threshold must be >= 0");
        h->nbl_min = value;
        return SMR_OK;
    }
    if (key == SMR_TUNE_NBLIST_SKIN_MA) {
        if (value < 50 || value > 5000) return fail(h, SMR_ERR_ARG, "neighbour-list skin must be 50..5000 mA");
        h->nbl_skin_ma = value;
        return SMR_OK;
    }
    if (key == SMR_TUNE_SMEM_CARVEOUT) {
        if (value < -1 || value > 100) return fail(h, SMR_ERR_ARG, "shared-memory carveout must be -1 or 0..100");
        h->smem_carveout = value;
        return SMR_OK;
    }
    if (key == SMR_TUNE_OCC_TIERS) {
        if (value != 0 && value != 1) return fail(h, SMR_ERR_ARG, "occupancy tiers must be 0 or 1");
        h->occ_tiers = value;
        return SMR_OK;
    }
    if (key == SMR_TUNE_GRID_PREFETCH) {
        if (value != 0 && value != 1) return fail(h, SMR_ERR_ARG, "grid prefetch must be 0 or 1");
        h->grid_prefetch = value;
        return SMR_OK;
    }
    if (key == SMR_TUNE_GRID_BRICKS) {
        if (value < -1 || value > 1) return fail(h, SMR_ERR_ARG, "grid bricks must be -1 (auto), 0 or 1");
        h->brick_mode = value;
        return SMR_OK;
    }
    if (key == SMR_TUNE_NBLIST_CAP) {
        if (value < 32 || value > 4096 || value % 4) return fail(h, SMR_ERR_ARG, "neighbour-list capacity must be a multiple of 4 in 32..4096");
        if (h->nbl_ready && value != h->nbl_cap) {           // rows change shape: drop the lists
            h->nbl_ready = false;
        }
        h->nbl_cap = value;
        return SMR_OK;
    }
    return fail(h, SMR_ERR_ARG, "unknown tuning key %d", key);
}

int smr_get_tuning(smr_handle* h, int key, int* value) {
    if (!h || !value) return SMR_ERR_ARG;
    if (key == SMR_TUNE_NB_LANES) { *value = h->nb_lanes; return SMR_OK; }
    if (key == SMR_TUNE_NBLIST_MIN) { *value = h->nbl_min; return SMR_OK; }
    if (key == SMR_TUNE_WATCHDOG_MS) { *value = (int)std::min(2.0e9, h->watchdog_s * 1e3); return SMR_OK; }
    if (key == SMR_TUNE_NBLIST_SKIN_MA) { *value = h->nbl_skin_ma; return SMR_OK; }
    if (key == SMR_TUNE_NBLIST_CAP) { *value = h->nbl_cap; return SMR_OK; }
    if (key == SMR_TUNE_GRID_BRICKS) { *value = h->brick_mode; return SMR_OK; }
    if (key == SMR_TUNE_GRID_BRICKS_ACTIVE) { *value = h->use_bricks ? 1 : 0; return SMR_OK; }
    if (key == SMR_TUNE_GRID_PREFETCH) { *value = h->grid_prefetch; return SMR_OK; }
    if (key == SMR_TUNE_SMEM_CARVEOUT) { *value = h->smem_carveout; return SMR_OK; }
    if (key == SMR_TUNE_OCC_TIERS) { *value = h->occ_tiers; return SMR_OK; }
    return fail(h, SMR_ERR_ARG, "unknown tuning key %d", key);
}

int smr_set_team_size(smr_handle* h, int max_atoms, int threads) {
    if (!h) return SMR_ERR_ARG;
    SETTLE(h);
    if (threads != 0 && threads != 32 && threads != 64 && threads != 128 && threads != 256 && threads != 512)
        return fail(h, SMR_ERR_ARG, "team size must be 32, 64, 128, 256 or 512");
    if (threads == 0) h->team_override.erase(max_atoms);
    else h->team_override[max_atoms] = threads;
    return repack_all(h);
}

static size_t voxel_bytes(int dtype) { return dtype == SMR_GRID_F32 ? 16 : 8; }

// forget the FP32 near-surface planes of a split grid (the grid is being replaced or re-encoded)
static void drop_split(smr_handle* h) {
    if (h->grid_lo) { cudaStreamSynchronize(h->stream); cudaFree(h->grid_lo); h->grid_lo = nullptr; }
    h->grid_zsplit = 0;
}

// install per-plane scales (nz x 4 host floats; null: none) on the device
static int set_plane_scales(smr_handle* h, const float* ps, int nz) {
    if (!ps) { h->gzscale.clear(); return SMR_OK; }
    h->gzscale.assign(ps, ps + 4 * (size_t)nz);
    cudaError_t e = h->dzscale.reserve((size_t)nz, 0, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->dzscale.d, h->gzscale.data(), (size_t)nz * 16, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return fail(h, SMR_ERR_CUDA, "plane scales: %s", cudaGetErrorString(e));
    for (int c = 0; c < 4; c++) {                          // per-channel summary: the largest plane scale
        float m = 0.f;
        for (int z = 0; z < nz; z++) m = std::max(m, h->gzscale[4 * (size_t)z + c]);
        h->gscale[c] = m;
    }
    return SMR_OK;
}

int smr_set_surface_folded(smr_handle* h, const smr_folded_surface* f) {
    if (!h) return SMR_ERR_ARG;
    SETTLE(h);
    if (!f) { h->fold_on = false; return SMR_OK; }
    if (f->nx < 1 || f->ny < 1 || f->nz < 1 || f->nx > 64 || f->ny > 64 || f->nz > 64)
        return fail(h, SMR_ERR_ARG, "folded surface: nx, ny, nz must be 1..64 (got %d, %d, %d)", f->nx, f->ny, f->nz);
    if (!f->kx || !f->ky || !f->kz || !f->z0 || !f->cq || !f->cp || !f->cl) return fail(h, SMR_ERR_ARG, "folded surface: null array");
    const double det = f->ax * f->by - f->bx * f->ay;
    if (!(std::fabs(det) > 1e-12)) return fail(h, SMR_ERR_ARG, "folded surface: degenerate 2D lattice");
    if (!(f->fmax > 0) || !std::isfinite(f->alpha)) return fail(h, SMR_ERR_ARG, "folded surface: fmax must be positive, alpha finite");
    const int nx = f->nx, ny = f->ny, nz = f->nz, nb = nx * ny * nz;
    std::vector<float> k;
    for (int i = 0; i < nx; i++) k.push_back((float)f->kx[i]);
    for (int i = 0; i < ny; i++) k.push_back((float)f->ky[i]);
    for (int i = 0; i < nz; i++) k.push_back((float)f->kz[i]);
    for (int i = 0; i < nz; i++) k.push_back((float)f->z0[i]);
    std::vector<float4> c(nb);
    for (int i = 0; i < nb; i++) c[i] = make_float4((float)f->cq[i], (float)f->cp[i], (float)f->cl[i], 0.f);
    cudaError_t e = h->dfold_k.reserve(k.size(), 0, h->stream);
    if (e == cudaSuccess) e = h->dfold_coef.reserve((size_t)nb, 0, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->dfold_k.d, k.data(), k.size() * 4, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->dfold_coef.d, c.data(), (size_t)nb * 16, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);      // the host vectors are freed on return
    if (e != cudaSuccess) { h->fold_on = false; return fail(h, SMR_ERR_CUDA, "folded surface upload: %s", cudaGetErrorString(e)); }
    h->fold_n[0] = nx; h->fold_n[1] = ny; h->fold_n[2] = nz;
    const double idet = 1.0 / det;
    const double inv[4] = {f->by * idet, -f->bx * idet, -f->ay * idet, f->ax * idet};
    for (int k = 0; k < 4; k++) { h->fold_inv[k] = (float)inv[k]; h->fold_inv_lo[k] = (float)(inv[k] - (double)h->fold_inv[k]); }
    h->fold_alpha = (float)f->alpha; h->fold_fmax = (float)f->fmax;
    h->fold_on = true;
    return SMR_OK;
}

int smr_set_grid_planes(smr_handle* h, const void* coef, int dtype, const float* plane_scale, int nx, int ny, int nz,
                        const double p0[3], const double step[3]) {
    if (!h || !plane_scale) return SMR_ERR_ARG;
    if (dtype != SMR_GRID_F16 && dtype != SMR_GRID_BF16) return fail(h, SMR_ERR_ARG, "per-plane scales are for 16-bit grids");
    int r = smr_set_grid(h, coef, dtype, nullptr, nx, ny, nz, p0, step);
    if (r) return r;
    return set_plane_scales(h, plane_scale, nz);
}

int smr_get_grid_planes(smr_handle* h, float* plane_scale) {
    if (!h || !plane_scale) return SMR_ERR_ARG;
    if (!h->has_grid) return fail(h, SMR_ERR_STATE, "no grid set");
    const int nz = h->gdim[2];
    for (int z = 0; z < nz; z++)
        for (int c = 0; c < 4; c++)
            plane_scale[4 * (size_t)z + c] = h->gzscale.empty() ? h->gscale[c] : h->gzscale[4 * (size_t)z + c];
    return SMR_OK;
}

int smr_set_grid(smr_handle* h, const void* coef, int dtype, const float scale[4], int nx, int ny, int nz,
                 const double p0[3], const double step[3]) {
    if (!h || !coef || !p0 || !step) return SMR_ERR_ARG;
    SETTLE(h);
    if (dtype < 0 || dtype > 2) return fail(h, SMR_ERR_ARG, "unknown grid dtype %d", dtype);
    if (nx < 4 || ny < 4 || nz < 4) return fail(h, SMR_ERR_ARG, "grid must be at least 4x4x4 (got %dx%dx%d)", nx, ny, nz);
    if ((double)nx * ny * nz >= 2147483648.0) return fail(h, SMR_ERR_ARG, "grid of %dx%dx%d has 2^31 voxels or more", nx, ny, nz);
    if (!(step[0] > 0 && step[1] > 0 && step[2] > 0)) return fail(h, SMR_ERR_ARG, "grid steps must be positive");
    size_t nv = (size_t)nx * ny * nz, bytes = nv * voxel_bytes(dtype);
    void* d = nullptr;
    CU(h, cudaMalloc(&d, bytes));
    cudaError_t e = cudaMemcpyAsync(d, coef, bytes, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) { cudaFree(d); return fail(h, SMR_ERR_CUDA, "grid upload: %s", cudaGetErrorString(e)); }
    drop_split(h);
    if (h->grid) cudaFree(h->grid);
    h->grid = d; h->grid_version++; h->grid_dtype = dtype; h->has_grid = true;
    h->gdim[0] = nx; h->gdim[1] = ny; h->gdim[2] = nz;
    for (int k = 0; k < 3; k++) { h->gp0[k] = p0[k]; h->gstep[k] = step[k]; }
    for (int k = 0; k < 4; k++) h->gscale[k] = scale ? scale[k] : 1.f;
    h->gzscale.clear();
    return SMR_OK;
}

int smr_set_grid_device(smr_handle* h, const void* dev_coef, int dtype, const float scale[4], int nx, int ny, int nz,
                        const double p0[3], const double step[3]) {
    if (!h || !dev_coef || !p0 || !step) return SMR_ERR_ARG;
    SETTLE(h);
    if (dtype < 0 || dtype > 2) return fail(h, SMR_ERR_ARG, "unknown grid dtype %d", dtype);
    if (nx < 4 || ny < 4 || nz < 4) return fail(h, SMR_ERR_ARG, "grid must be at least 4x4x4 (got %dx%dx%d)", nx, ny, nz);
    if ((double)nx * ny * nz >= 2147483648.0) return fail(h, SMR_ERR_ARG, "grid of %dx%dx%d has 2^31 voxels or more", nx, ny, nz);
    if (!(step[0] > 0 && step[1] > 0 && step[2] > 0)) return fail(h, SMR_ERR_ARG, "grid steps must be positive");
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, dev_coef) != cudaSuccess || attr.type != cudaMemoryTypeDevice) {
        cudaGetLastError();
        return fail(h, SMR_ERR_ARG, "coefficients are not in device memory");
    }
    const size_t bytes = (size_t)nx * ny * nz * voxel_bytes(dtype);
    void* d = nullptr;
    CU(h, cudaMalloc(&d, bytes));
    cudaError_t e = cudaMemcpyAsync(d, dev_coef, bytes, cudaMemcpyDeviceToDevice, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) { cudaFree(d); return fail(h, SMR_ERR_CUDA, "grid copy: %s", cudaGetErrorString(e)); }
    drop_split(h);
    if (h->grid) cudaFree(h->grid);
    h->grid = d; h->grid_version++; h->grid_dtype = dtype; h->has_grid = true;
    h->gdim[0] = nx; h->gdim[1] = ny; h->gdim[2] = nz;
    for (int k = 0; k < 3; k++) { h->gp0[k] = p0[k]; h->gstep[k] = step[k]; }
    for (int k = 0; k < 4; k++) h->gscale[k] = scale ? scale[k] : 1.f;
    h->gzscale.clear();
    return SMR_OK;
}

int smr_get_grid(smr_handle* h, void* coef_out, int* dtype, float scale[4], int dims[3], double p0[3], double step[3]) {
    if (!h) return SMR_ERR_ARG;
    SETTLE(h);
    if (!h->has_grid) return fail(h, SMR_ERR_STATE, "no grid set");
    if (dtype) *dtype = h->grid_dtype;
    if (scale) for (int k = 0; k < 4; k++) scale[k] = h->gscale[k];
    if (dims) for (int k = 0; k < 3; k++) dims[k] = h->gdim[k];
    if (p0) for (int k = 0; k < 3; k++) p0[k] = h->gp0[k];
    if (step) for (int k = 0; k < 3; k++) step[k] = h->gstep[k];
    if (coef_out) {
        size_t bytes = (size_t)h->gdim[0] * h->gdim[1] * h->gdim[2] * voxel_bytes(h->grid_dtype);
        CU(h, cudaMemcpyAsync(coef_out, h->grid, bytes, cudaMemcpyDeviceToHost, h->stream));
        CU(h, cudaStreamSynchronize(h->stream));
    }
    return SMR_OK;
}

int smr_convert_grid(smr_handle* h, int dtype) {
    if (!h) return SMR_ERR_ARG;
    SETTLE(h);
    if (!h->has_grid) return fail(h, SMR_ERR_STATE, "no grid set");
    if (dtype == h->grid_dtype) return SMR_OK;
    size_t nv = (size_t)h->gdim[0] * h->gdim[1] * h->gdim[2];
    float4* f32 = nullptr;
    if (h->grid_dtype == SMR_GRID_F32) f32 = (float4*)h->grid;
    else {
        CU(h, cudaMalloc(&f32, nv * 16));
        // the decode table: the per-plane scales, or the channel scales on every plane
        const int nz = h->gdim[2];
        std::vector<float> tab(4 * (size_t)nz);
        smr_get_grid_planes(h, tab.data());
        int r = set_plane_scales(h, tab.data(), nz);
        if (r) { cudaFree(f32); return r; }
        if (decode_grid_16(h->grid, f32, nv, nz, h->grid_dtype, h->dzscale.d, h->stream)) { cudaFree(f32); return fail(h, SMR_ERR_CUDA, "grid decode failed"); }
    }
    void* out = nullptr;
    std::vector<float> ps;
    if (dtype == SMR_GRID_F32) out = f32;
    else {
        cudaError_t e = cudaMalloc(&out, nv * 8);
        if (e != cudaSuccess) { if ((void*)f32 != h->grid) cudaFree(f32); return fail(h, SMR_ERR_CUDA, "grid alloc: %s", cudaGetErrorString(e)); }
        ps.resize(4 * (size_t)h->gdim[2]);
        if (encode_grid_16(f32, out, nv, h->gdim[2], dtype, ps.data(), h->stream)) { cudaFree(out); return fail(h, SMR_ERR_CUDA, "grid encode failed"); }
        if ((void*)f32 != h->grid) cudaFree(f32);
        // an FP32 source's values are its stored values times its channel scales
        else for (size_t z = 0; z < (size_t)h->gdim[2]; z++) for (int c = 0; c < 4; c++) ps[4 * z + c] *= h->gscale[c];
    }
    CU(h, cudaStreamSynchronize(h->stream));
    drop_split(h);
    if (out != h->grid) cudaFree(h->grid);
    h->grid = out; h->grid_version++; h->grid_dtype = dtype;
    if (dtype == SMR_GRID_F32) { for (int k = 0; k < 4; k++) h->gscale[k] = 1.f; h->gzscale.clear(); }
    else { int r = set_plane_scales(h, ps.data(), h->gdim[2]); if (r) return r; }
    return SMR_OK;
}

int smr_convert_grid_split(smr_handle* h, int dtype, int zsplit) {
    if (!h) return SMR_ERR_ARG;
    SETTLE(h);
    if (!h->has_grid) return fail(h, SMR_ERR_STATE, "no grid set");
    if (h->grid_dtype != SMR_GRID_F32) return fail(h, SMR_ERR_STATE, "a split grid is made from an FP32 grid (current dtype %d)", h->grid_dtype);
    if (dtype != SMR_GRID_F16 && dtype != SMR_GRID_BF16) return fail(h, SMR_ERR_ARG, "split grids store F16 or BF16 above the split");
    const int nx = h->gdim[0], ny = h->gdim[1], nz = h->gdim[2];
    if (zsplit < 1 || zsplit > nz - 3) return fail(h, SMR_ERR_ARG, "zsplit must be 1..%d (got %d)", nz - 3, zsplit);
    const int nzl = zsplit + 3;
    float4* lo = nullptr;
    CU(h, cudaMalloc(&lo, (size_t)nx * ny * nzl * 16));
    if (extract_low_planes((const float4*)h->grid, (size_t)nx * ny, nz, nzl, lo, h->stream) ||
        cudaStreamSynchronize(h->stream) != cudaSuccess) {
        cudaFree(lo);
        return fail(h, SMR_ERR_CUDA, "copy of the FP32 planes failed");
    }
    float sc[4];
    for (int k = 0; k < 4; k++) sc[k] = h->gscale[k];
    const int r = smr_convert_grid(h, dtype);
    if (r) { cudaFree(lo); return r; }
    h->grid_lo = lo; h->grid_zsplit = zsplit;
    for (int k = 0; k < 4; k++) h->glo_scale[k] = sc[k];
    h->grid_version++;                                    // rebuild the brick copies
    return SMR_OK;
}

int smr_get_grid_split(smr_handle* h, int* zsplit, float* lo_out) {
    if (!h || !zsplit) return SMR_ERR_ARG;
    SETTLE(h);
    *zsplit = h->has_grid ? h->grid_zsplit : 0;
    if (lo_out && *zsplit > 0) {
        const size_t n = (size_t)h->gdim[0] * h->gdim[1] * (h->grid_zsplit + 3);
        std::vector<float4> tmp(n);
        CU(h, cudaMemcpyAsync(tmp.data(), h->grid_lo, n * 16, cudaMemcpyDeviceToHost, h->stream));
        CU(h, cudaStreamSynchronize(h->stream));
        for (size_t i = 0; i < n; i++) {
            lo_out[4 * i] = tmp[i].x * h->glo_scale[0]; lo_out[4 * i + 1] = tmp[i].y * h->glo_scale[1];
            lo_out[4 * i + 2] = tmp[i].z * h->glo_scale[2]; lo_out[4 * i + 3] = tmp[i].w * h->glo_scale[3];
        }
    }
    return SMR_OK;
}

int smr_build_grid(smr_handle* h, int nions, const double* ions, const double* ion_re, double Lx, double Ly,
                   int nx, int ny, int nz, const double p0[3], const double step[3], const smr_grid_build_params* p) {
    if (!h || !ions || !ion_re || !p0 || !step || !p || nions <= 0) return SMR_ERR_ARG;
    SETTLE(h);
    if (nx < 4 || ny < 4 || nz < 4) return fail(h, SMR_ERR_ARG, "grid must be at least 4x4x4");
    if ((double)nx * ny * nz >= 2147483648.0) return fail(h, SMR_ERR_ARG, "grid of %dx%dx%d has 2^31 voxels or more", nx, ny, nz);
    if (!(Lx > 0 && Ly > 0)) return fail(h, SMR_ERR_ARG, "cell must be positive");
    if (p->dtype < 0 || p->dtype > 2) return fail(h, SMR_ERR_ARG, "unknown grid dtype");
    double *dions = nullptr, *dre = nullptr;
    float4* out = nullptr;
    size_t nv = (size_t)nx * ny * nz;
    CU(h, cudaMalloc(&dions, (size_t)nions * 32));
    cudaError_t e = cudaMalloc(&dre, (size_t)nions * 32);
    if (e == cudaSuccess) e = cudaMalloc(&out, nv * 16);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dions, ions, (size_t)nions * 32, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        std::vector<double> re4(4 * (size_t)nions, 0.0);
        for (int i = 0; i < nions; i++) { re4[4 * i] = ion_re[2 * i]; re4[4 * i + 1] = ion_re[2 * i + 1]; }
        e = cudaMemcpyAsync(dre, re4.data(), re4.size() * 8, cudaMemcpyHostToDevice, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);   // re4 is freed on return
    }
    if (e != cudaSuccess) { cudaFree(dions); cudaFree(dre); cudaFree(out); return fail(h, SMR_ERR_CUDA, "grid build alloc: %s", cudaGetErrorString(e)); }
    GridBuildArgs A{};
    A.nions = nions; A.ions = dions; A.ion_re = dre; A.Lx = Lx; A.Ly = Ly; A.nx = nx; A.ny = ny; A.nz = nz;
    for (int k = 0; k < 3; k++) { A.p0[k] = p0[k]; A.step[k] = step[k]; }
    A.alpha = p->alpha_morse; A.npbc = p->npbc; A.ewald_tol = p->ewald_tol; A.morse_rcut = p->morse_rcut;
    char msg[400] = {0};
    int r = build_grid_device(A, out, h->stream, msg, sizeof(msg));
    cudaFree(dions); cudaFree(dre);
    if (r) { cudaFree(out); return fail(h, SMR_ERR_ARG, "grid build: %s", msg); }
    drop_split(h);
    if (h->grid) cudaFree(h->grid);
    h->grid = out; h->grid_version++; h->grid_dtype = SMR_GRID_F32; h->has_grid = true;
    h->gdim[0] = nx; h->gdim[1] = ny; h->gdim[2] = nz;
    for (int k = 0; k < 3; k++) { h->gp0[k] = p0[k]; h->gstep[k] = step[k]; }
    for (int k = 0; k < 4; k++) h->gscale[k] = 1.f;
    h->gzscale.clear();                                   // a previous 16-bit grid's plane scales
    if (p->dtype != SMR_GRID_F32) return smr_convert_grid(h, p->dtype);
    return SMR_OK;
}

// the sharded grid build's per-rank part: ions to the device, arguments, the raw evaluation
int smr_grid_raw_slab(smr_handle* h, int nions, const double* ions, const double* ion_re, double Lx, double Ly,
                      int nx, int ny, int nz, const double p0[3], const double step[3], const smr_grid_build_params* p,
                      int x0, int nxs, double* raw) {
    if (!h || !ions || !ion_re || !p0 || !step || !p || !raw || nions <= 0) return SMR_ERR_ARG;
    SETTLE(h);
    if (nx < 4 || ny < 4 || nz < 4) return fail(h, SMR_ERR_ARG, "grid must be at least 4x4x4");
    if ((double)nx * ny * nz >= 2147483648.0) return fail(h, SMR_ERR_ARG, "grid of %dx%dx%d has 2^31 voxels or more", nx, ny, nz);
    if (x0 < 0 || nxs < 1) return fail(h, SMR_ERR_ARG, "slab x0=%d, width %d", x0, nxs);
    if (!(Lx > 0 && Ly > 0)) return fail(h, SMR_ERR_ARG, "cell must be positive");
    double *dions = nullptr, *dre = nullptr;
    CU(h, cudaMalloc(&dions, (size_t)nions * 32));
    cudaError_t e = cudaMalloc(&dre, (size_t)nions * 32);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dions, ions, (size_t)nions * 32, cudaMemcpyHostToDevice, h->stream);
    std::vector<double> re4(4 * (size_t)nions, 0.0);
    for (int i = 0; i < nions; i++) { re4[4 * i] = ion_re[2 * i]; re4[4 * i + 1] = ion_re[2 * i + 1]; }
    if (e == cudaSuccess) e = cudaMemcpyAsync(dre, re4.data(), re4.size() * 8, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) { cudaFree(dions); cudaFree(dre); return fail(h, SMR_ERR_CUDA, "grid slab: %s", cudaGetErrorString(e)); }
    GridBuildArgs A{};
    A.nions = nions; A.ions = dions; A.ion_re = dre; A.Lx = Lx; A.Ly = Ly; A.nx = nx; A.ny = ny; A.nz = nz;
    for (int k = 0; k < 3; k++) { A.p0[k] = p0[k]; A.step[k] = step[k]; }
    A.alpha = p->alpha_morse; A.npbc = p->npbc; A.ewald_tol = p->ewald_tol; A.morse_rcut = p->morse_rcut;
    char msg[400] = {0};
    const int r = grid_raw_slab_device(A, x0, nxs, raw, h->stream, msg, sizeof(msg));
    cudaFree(dions); cudaFree(dre);
    if (r) return fail(h, SMR_ERR_ARG, "grid slab: %s", msg);
    return SMR_OK;
}

int smr_grid_from_raw(smr_handle* h, const double* raw, int nx, int ny, int nz, const double p0[3], const double step[3], int dtype) {
    if (!h || !raw || !p0 || !step) return SMR_ERR_ARG;
    SETTLE(h);
    if (nx < 4 || ny < 4 || nz < 4) return fail(h, SMR_ERR_ARG, "grid must be at least 4x4x4");
    if ((double)nx * ny * nz >= 2147483648.0) return fail(h, SMR_ERR_ARG, "grid of %dx%dx%d has 2^31 voxels or more", nx, ny, nz);
    if (dtype < 0 || dtype > 2) return fail(h, SMR_ERR_ARG, "unknown grid dtype");
    float4* out = nullptr;
    CU(h, cudaMalloc(&out, (size_t)nx * ny * nz * 16));
    char msg[400] = {0};
    if (grid_from_raw_device(raw, nx, ny, nz, out, h->stream, msg, sizeof(msg))) { cudaFree(out); return fail(h, SMR_ERR_CUDA, "grid fit: %s", msg); }
    drop_split(h);
    if (h->grid) cudaFree(h->grid);
    h->grid = out; h->grid_version++; h->grid_dtype = SMR_GRID_F32; h->has_grid = true;
    h->gdim[0] = nx; h->gdim[1] = ny; h->gdim[2] = nz;
    for (int k = 0; k < 3; k++) { h->gp0[k] = p0[k]; h->gstep[k] = step[k]; }
    for (int k = 0; k < 4; k++) h->gscale[k] = 1.f;
    h->gzscale.clear();
    if (dtype != SMR_GRID_F32) return smr_convert_grid(h, dtype);
    return SMR_OK;
}

int smr_add_molecule(smr_handle* h, int natoms, const int* Z, const double* pos, const double* charges,
                     double bond_cut, int* topo_id) {
    if (!h || !Z || !pos || !topo_id) return SMR_ERR_ARG;
    SETTLE(h);
    HostTopo T;
    char msg[300] = {0};
    if (build_molecule_topology(natoms, Z, pos, charges, bond_cut > 0 ? bond_cut : 1.8, T, msg, sizeof(msg)))
        return fail(h, SMR_ERR_ARG, "molecule: %s", msg);
    h->topos.push_back(std::move(T));
    h->topo_alive.push_back(1);
    append_topology(h, h->topos.back());
    int r = upload_all(h);
    if (r) return r;
    *topo_id = (int)h->topos.size() - 1;
    return SMR_OK;
}

int smr_add_molecule_pbc(smr_handle* h, int natoms, const int* Z, const double* pos, const double* charges,
                         double bond_cut, const double lvec[9], const int npbc[3], int* topo_id) {
    if (!h || !Z || !pos || !lvec || !topo_id) return SMR_ERR_ARG;
    SETTLE(h);
    if (npbc) for (int k = 0; k < 3; k++)
        if (npbc[k] < 0 || npbc[k] > 7) return fail(h, SMR_ERR_ARG, "npbc[%d]=%d outside [0, 7]", k, npbc[k]);
    HostTopo T;
    char msg[300] = {0};
    if (build_molecule_topology_pbc(natoms, Z, pos, charges, bond_cut > 0 ? bond_cut : 1.8, lvec, T, msg, sizeof(msg)))
        return fail(h, SMR_ERR_ARG, "periodic molecule: %s", msg);
    if (npbc) for (int k = 0; k < 3; k++) T.npbc[k] = npbc[k];
    h->topos.push_back(std::move(T));
    h->topo_alive.push_back(1);
    append_topology(h, h->topos.back());
    int r = upload_all(h);
    if (r) return r;
    *topo_id = (int)h->topos.size() - 1;
    return SMR_OK;
}

// write the lattice rows of the given slots to the device (the per-slot table is allocated on first use)
static int upload_lat(smr_handle* h, const std::vector<int>& ids) {
    if (ids.empty()) return SMR_OK;
    CU(h, h->dlat.reserve(h->hlat.size(), 0, h->stream));
    for (int s : ids) CU(h, cudaMemcpyAsync(h->dlat.d + 3 * (size_t)s, &h->hlat[3 * (size_t)s], 48, cudaMemcpyHostToDevice, h->stream));
    return wait_stream(h, h->watchdog_s);
}

// a slot's lattice and images: the rows of hlat and the slot flag (no flag without images or periodic bonds)
static void set_slot_lattice(smr_handle* h, int s, const double* lvec, const int* npbc) {
    const HostTopo& T = h->topos[h->hs[s].topo];
    bool on = !T.neighc.empty();
    for (int k = 0; k < 3; k++) {
        h->hlat[3 * (size_t)s + k] = make_float4((float)lvec[3 * k], (float)lvec[3 * k + 1], (float)lvec[3 * k + 2], (float)npbc[k]);
        on = on || npbc[k] > 0;
    }
    h->hs[s].flags = on ? (h->hs[s].flags | SLOT_PBC) : (h->hs[s].flags & ~SLOT_PBC);
}

int smr_set_pbc(smr_handle* h, int nsys, const int* slot_ids, const double* lvec, const int* npbc) {
    if (!h || nsys < 0 || (nsys && (!slot_ids || !lvec || !npbc))) return SMR_ERR_ARG;
    SETTLE(h);
    for (int i = 0; i < nsys; i++) {
        if (!valid_slot(h, slot_ids[i])) return fail(h, SMR_ERR_ARG, "slot %d not active", slot_ids[i]);
        for (int k = 0; k < 3; k++)
            if (npbc[3 * i + k] < 0 || npbc[3 * i + k] > 7) return fail(h, SMR_ERR_ARG, "system %d: npbc[%d]=%d outside [0, 7]", i, k, npbc[3 * i + k]);
        const HostTopo& T = h->topos[h->hs[slot_ids[i]].topo];
        for (int k = 0; k < 3; k++) {
            const bool crosses = [&] { for (size_t c = 0; c < T.neighc.size(); c++) if (cell_field(T.neighc[c], k)) return true; return false; }();
            const double* v = lvec + 9 * (size_t)i + 3 * k;
            if (crosses && v[0] == 0 && v[1] == 0 && v[2] == 0)
                return fail(h, SMR_ERR_ARG, "system %d: bonds cross lattice axis %d but its vector is zero", i, k);
        }
    }
    std::vector<int> ids(slot_ids, slot_ids + nsys);
    for (int i = 0; i < nsys; i++) set_slot_lattice(h, slot_ids[i], lvec + 9 * (size_t)i, npbc + 3 * (size_t)i);
    int r = upload_lat(h, ids);
    if (r) return r;
    return upload_slots(h, ids);
}

int smr_set_constraints(smr_handle* h, int slot, int n, const int* atoms, const double* target, const double* k) {
    if (!h || n < 0 || (n && (!atoms || !target || !k))) return SMR_ERR_ARG;
    SETTLE(h);
    if (!valid_slot(h, slot)) return fail(h, SMR_ERR_ARG, "slot %d not active", slot);
    SlotState& st = h->hs[slot];
    std::vector<float4> c(2 * (size_t)st.natoms, make_float4(0.f, 0.f, 0.f, 0.f));
    for (int i = 0; i < n; i++) {
        const int a = atoms[i];
        if (a < 0 || a >= st.natoms) return fail(h, SMR_ERR_ARG, "constraint %d: atom %d outside [0, %d)", i, a, st.natoms);
        for (int d = 0; d < 3; d++)
            if (!std::isfinite(target[3 * i + d]) || !std::isfinite(k[3 * i + d])) return fail(h, SMR_ERR_ARG, "constraint %d: non-finite value", i);
        c[2 * a] = make_float4((float)target[3 * i], (float)target[3 * i + 1], (float)target[3 * i + 2], 1.f);
        c[2 * a + 1] = make_float4((float)k[3 * i], (float)k[3 * i + 1], (float)k[3 * i + 2], 0.f);
    }
    if (n) {
        if (!h->dcons.d) {
            CU(h, h->dcons.reserve(2 * (size_t)h->max_atoms, 0, h->stream));
            CU(h, cudaMemsetAsync(h->dcons.d, 0, 2 * (size_t)h->max_atoms * 16, h->stream));
        }
        CU(h, cudaMemcpyAsync(h->dcons.d + 2 * (size_t)st.atom_off, c.data(), c.size() * 16, cudaMemcpyHostToDevice, h->stream));
        st.flags |= SLOT_CONS;
    } else {
        st.flags &= ~SLOT_CONS;
    }
    return upload_slots(h, {slot});                    // waits, so c may go
}

int smr_set_thermal_drive(smr_handle* h, int nsys, const int* slot_ids, const double* tdrive) {
    if (!h || nsys < 0 || (nsys && (!slot_ids || !tdrive))) return SMR_ERR_ARG;
    SETTLE(h);
    for (int i = 0; i < nsys; i++) {
        if (!valid_slot(h, slot_ids[i])) return fail(h, SMR_ERR_ARG, "slot %d not active", slot_ids[i]);
        const double* t = tdrive + 4 * (size_t)i;
        for (int k = 0; k < 4; k++)
            if (!std::isfinite(t[k])) return fail(h, SMR_ERR_ARG, "system %d: non-finite drive value", i);
        if (t[0] < 0.0) return fail(h, SMR_ERR_ARG, "system %d: temperature %g below 0", i, t[0]);
    }
    if (nsys == 0) return SMR_OK;
    if (!h->dtdrive.d) {
        CU(h, h->dtdrive.reserve(h->hs.size(), 0, h->stream));
        CU(h, cudaMemsetAsync(h->dtdrive.d, 0, h->hs.size() * 16, h->stream));
    }
    std::vector<float4> td(nsys);
    std::vector<int> ids(slot_ids, slot_ids + nsys);
    for (int i = 0; i < nsys; i++) {
        const double* t = tdrive + 4 * (size_t)i;
        td[i] = make_float4((float)t[0], (float)t[1], (float)t[2], (float)t[3]);
        SlotState& st = h->hs[slot_ids[i]];
        // the drive acts while gamma > 0, as in updateAtomsMMFFf4
        st.flags = td[i].y > 0.f ? (st.flags | SLOT_THERM) : (st.flags & ~SLOT_THERM);
        CU(h, cudaMemcpyAsync(h->dtdrive.d + slot_ids[i], &td[i], 16, cudaMemcpyHostToDevice, h->stream));
    }
    return upload_slots(h, ids);                      // waits, so td may go
}

int smr_get_pbc(smr_handle* h, int slot, double lvec[9], int npbc[3]) {
    if (!h || !lvec || !npbc) return SMR_ERR_ARG;
    SETTLE(h);
    if (!valid_slot(h, slot)) return fail(h, SMR_ERR_ARG, "slot %d not active", slot);
    for (int k = 0; k < 3; k++) {
        const float4 v = h->hlat[3 * (size_t)slot + k];
        const bool on = (h->hs[slot].flags & SLOT_PBC) != 0;
        lvec[3 * k] = on ? v.x : 0.0; lvec[3 * k + 1] = on ? v.y : 0.0; lvec[3 * k + 2] = on ? v.z : 0.0;
        npbc[k] = on ? (int)v.w : 0;
    }
    return SMR_OK;
}

int smr_add_molecules(smr_handle* h, int nmol, const int* natoms, const int* Z, const double* pos, const double* charges,
                      double bond_cut, int* topo_ids) {
    if (!h || nmol < 0 || (nmol && (!natoms || !Z || !pos || !topo_ids))) return SMR_ERR_ARG;
    SETTLE(h);
    std::vector<long long> off(nmol + 1, 0);
    for (int i = 0; i < nmol; i++) {
        if (natoms[i] <= 0) return fail(h, SMR_ERR_ARG, "molecule %d has %d atoms", i, natoms[i]);
        off[i + 1] = off[i] + natoms[i];
    }
    std::vector<HostTopo> T(nmol);
    std::vector<PreparedTopo> prep(nmol);
    std::vector<std::string> err(nmol);
    const double cut = bond_cut > 0 ? bond_cut : 1.8;
    parallel_for(nmol, [&](int i) {
        char msg[300] = {0};
        if (build_molecule_topology(natoms[i], Z + off[i], pos + 3 * off[i], charges ? charges + off[i] : nullptr, cut, T[i],
                                    msg, sizeof(msg))) { err[i] = msg[0] ? msg : "invalid molecule"; return; }
        prepare_topology(T[i], team_for(h, T[i].n), prep[i]);
    });
    for (int i = 0; i < nmol; i++) if (!err[i].empty()) return fail(h, SMR_ERR_ARG, "molecule %d: %s", i, err[i].c_str());
    for (int i = 0; i < nmol; i++) {
        h->topos.push_back(std::move(T[i]));
        h->topo_alive.push_back(1);
        commit_topology(h, h->topos.back(), prep[i]);
        topo_ids[i] = (int)h->topos.size() - 1;
    }
    return upload_all(h);
}

int smr_add_listed_molecule(smr_handle* h, int natoms, const int* Z, const int* type_ids, const double* charges,
                            int nbonds, const int* bonds, int nang, const int* angs, int ndih, const int* dihs,
                            int ninv, const int* invs, int* topo_id) {
    if (!h || !Z || !topo_id || (nbonds && !bonds) || (nang && !angs) || (ndih && !dihs) || (ninv && !invs)) return SMR_ERR_ARG;
    SETTLE(h);
    HostTopo T;
    char msg[300] = {0};
    if (build_listed_topology(natoms, Z, type_ids, charges, nbonds, bonds, nang, angs, ndih, dihs, ninv, invs, T, msg, sizeof(msg)))
        return fail(h, SMR_ERR_ARG, "topology: %s", msg);
    h->topos.push_back(std::move(T));
    h->topo_alive.push_back(1);
    append_topology(h, h->topos.back());
    int r = upload_all(h);
    if (r) return r;
    *topo_id = (int)h->topos.size() - 1;
    return SMR_OK;
}

int smr_add_topology(smr_handle* h, const smr_topology_desc* d, int* topo_id) {
    if (!h || !d || !topo_id || !d->req || !d->neighs || !d->bond_kl) return SMR_ERR_ARG;
    SETTLE(h);
    if ((d->nang && (!d->angs || !d->angp)) || (d->ndih && (!d->dihs || !d->dihp)) || (d->ninv && (!d->invs || !d->invp)))
        return fail(h, SMR_ERR_ARG, "term arrays missing");
    HostTopo T;
    char msg[300] = {0};
    if (build_desc_topology(d->natoms, d->req, d->neighs, d->bond_kl, d->nang, d->angs, d->angp, d->ndih, d->dihs, d->dihp,
                            d->ninv, d->invs, d->invp, T, msg, sizeof(msg)))
        return fail(h, SMR_ERR_ARG, "topology: %s", msg);
    h->topos.push_back(std::move(T));
    h->topo_alive.push_back(1);
    append_topology(h, h->topos.back());
    int r = upload_all(h);
    if (r) return r;
    *topo_id = (int)h->topos.size() - 1;
    return SMR_OK;
}

int smr_topology_counts(smr_handle* h, int id, int c[6]) {
    if (!h || !c || id < 0 || id >= (int)h->topos.size()) return SMR_ERR_ARG;
    const HostTopo& T = h->topos[id];
    const TopoDev& td = h->htd[id];
    c[0] = T.n; c[1] = (int)T.bonds.size() / 2; c[2] = (int)T.angs.size() / 3; c[3] = (int)T.dihs.size() / 4;
    c[4] = (int)T.invs.size() / 4; c[5] = td.ang_rounds + td.dih_rounds + td.inv_rounds;
    return SMR_OK;
}

int smr_topology_cells(smr_handle* h, int topo_id, int* cells) {
    if (!h || !cells) return SMR_ERR_ARG;
    if (topo_id < 0 || topo_id >= (int)h->topos.size() || !h->topo_alive[topo_id]) return fail(h, SMR_ERR_ARG, "unknown topology %d", topo_id);
    const HostTopo& T = h->topos[topo_id];
    for (int k = 0; k < 4 * T.n; k++) cells[k] = T.neighc.empty() ? 0 : T.neighc[k];
    return SMR_OK;
}

int smr_topology_export(smr_handle* h, int id, int* neighs, int* neighBs, int* bonds, double* bparams,
                        int* angs, int* ang_ngs, double* angp, int* dihs, int* dih_ngs, double* dihp,
                        int* invs, int* inv_ngs, double* invp, double* req, int* type_id) {
    if (!h || id < 0 || id >= (int)h->topos.size()) return SMR_ERR_ARG;
    const HostTopo& T = h->topos[id];
    auto cp = [](auto* dst, const auto& v) { if (dst) std::copy(v.begin(), v.end(), dst); };
    cp(neighs, T.neighs); cp(neighBs, T.neighBs); cp(bonds, T.bonds); cp(bparams, T.bparams);
    cp(angs, T.angs); cp(ang_ngs, T.ang_ngs); cp(angp, T.angp);
    cp(dihs, T.dihs); cp(dih_ngs, T.dih_ngs); cp(dihp, T.dihp);
    cp(invs, T.invs); cp(inv_ngs, T.inv_ngs); cp(invp, T.invp);
    cp(req, T.req); cp(type_id, T.type_id);
    return SMR_OK;
}

const char* smr_type_name(int id) { return type_name(id); }

// Launch order key of a system: Morton code (10 + 10 bits) of its lateral centre within the
// periodic grid cell, so a launch's work list walks the substrate patch by patch.
static uint32_t locality_key(const smr_handle* h, const float* pos, int n) {
    if (!h->has_grid || n <= 0) return 0u;
    double cx = 0, cy = 0;
    for (int a = 0; a < n; a++) { cx += pos[3 * a]; cy += pos[3 * a + 1]; }
    cx /= n; cy /= n;
    const double Lx = h->gdim[0] * h->gstep[0], Ly = h->gdim[1] * h->gstep[1];
    double fx = (cx - h->gp0[0]) / Lx, fy = (cy - h->gp0[1]) / Ly;
    fx -= std::floor(fx); fy -= std::floor(fy);
    const uint32_t qx = std::min<uint32_t>(1023u, (uint32_t)(fx * 1024.0)), qy = std::min<uint32_t>(1023u, (uint32_t)(fy * 1024.0));
    uint32_t k = 0;
    for (int b = 0; b < 10; b++) k |= ((qx >> b) & 1u) << (2 * b) | ((qy >> b) & 1u) << (2 * b + 1);
    return k;
}

int smr_add_systems(smr_handle* h, int nsys, const int* topo_ids, const float* pos, int* slot_ids) {
    if (!h || nsys < 0 || (nsys && (!topo_ids || !pos || !slot_ids))) return SMR_ERR_ARG;
    SETTLE(h);
    if ((int)h->free_slots.size() < nsys) return fail(h, SMR_ERR_CAPACITY, "only %zu free slots for %d systems", h->free_slots.size(), nsys);
    long long need = 0;
    for (int i = 0; i < nsys; i++) {
        if (topo_ids[i] < 0 || topo_ids[i] >= (int)h->topos.size() || !h->topo_alive[topo_ids[i]])
            return fail(h, SMR_ERR_ARG, "system %d: unknown topology %d", i, topo_ids[i]);
        need += h->topos[topo_ids[i]].n;
    }
    std::vector<int> ids(nsys), src(nsys), len(nsys), dst(nsys), lat_ids;
    long long p = 0;
    for (int i = 0; i < nsys; i++) {
        int n = h->topos[topo_ids[i]].n;
        long long off = alloc_atoms(h, n);
        if (off < 0) {
            for (int k = 0; k < i; k++) { free_atoms(h, h->hs[ids[k]].atom_off, h->hs[ids[k]].natoms); h->hs[ids[k]].active = 0; h->free_slots.push_back(ids[k]); }
            return fail(h, SMR_ERR_CAPACITY, "atom capacity exhausted (%lld atoms requested)", need);
        }
        int s = h->free_slots.back();
        h->free_slots.pop_back();
        SlotState& st = h->hs[s];
        st = SlotState{};
        st.topo = topo_ids[i]; st.atom_off = (int)off; st.natoms = n; st.active = 1; st.dt = -1.0;
        const HostTopo& T = h->topos[topo_ids[i]];
        if (!T.neighc.empty() || T.npbc[0] || T.npbc[1] || T.npbc[2]) { set_slot_lattice(h, s, T.lattice, T.npbc); lat_ids.push_back(s); }
        ids[i] = s; src[i] = (int)p; len[i] = n; dst[i] = (int)off;
        h->skey[s] = locality_key(h, pos + 3 * p, n);
        for (int a = 0; a < n; a++) h->pinned[p + a] = make_float4(pos[3 * (p + a)], pos[3 * (p + a) + 1], pos[3 * (p + a) + 2], 0.f);
        p += n;
    }
    if (nsys == 0) return SMR_OK;
    cudaStream_t s = h->stream;
    CU(h, cudaMemcpyAsync(h->stage, h->pinned, p * 16, cudaMemcpyHostToDevice, s));
    std::vector<int> desc(3 * nsys);
    std::copy(src.begin(), src.end(), desc.begin()); std::copy(len.begin(), len.end(), desc.begin() + nsys); std::copy(dst.begin(), dst.end(), desc.begin() + 2 * nsys);
    CU(h, cudaMemcpyAsync(h->xfer, desc.data(), desc.size() * 4, cudaMemcpyHostToDevice, s));
    if (launch_copy_segments(h->xfer, h->xfer + nsys, h->xfer + 2 * nsys, nsys, h->stage, h->pos, s)) return fail(h, SMR_ERR_CUDA, "scatter launch failed");
    CU(h, cudaMemsetAsync(h->stage, 0, (size_t)p * 16, s));
    if (launch_copy_segments(h->xfer, h->xfer + nsys, h->xfer + 2 * nsys, nsys, h->stage, h->plo, s)) return fail(h, SMR_ERR_CUDA, "scatter launch failed");
    int r = upload_lat(h, lat_ids);
    if (r) return r;
    r = upload_slots(h, ids);
    if (r) return r;
    r = wait_stream(h, h->watchdog_s);
    if (r) return r;
    std::copy(ids.begin(), ids.end(), slot_ids);
    return SMR_OK;
}

int smr_remove_systems(smr_handle* h, int nsys, const int* slot_ids) {
    if (!h || nsys < 0 || (nsys && !slot_ids)) return SMR_ERR_ARG;
    SETTLE(h);
    for (int i = 0; i < nsys; i++) if (!valid_slot(h, slot_ids[i])) return fail(h, SMR_ERR_ARG, "slot %d not active", slot_ids[i]);
    std::vector<int> ids(slot_ids, slot_ids + nsys);
    for (int s : ids) {
        free_atoms(h, h->hs[s].atom_off, h->hs[s].natoms);
        h->hs[s] = SlotState{};
        h->free_slots.push_back(s);
    }
    return upload_slots(h, ids);
}

int smr_set_positions(smr_handle* h, int nsys, const int* slot_ids, const float* pos) {
    if (!h || nsys < 0 || (nsys && (!slot_ids || !pos))) return SMR_ERR_ARG;
    SETTLE(h);
    { int r = check_batch(h, nsys, slot_ids); if (r) return r; }
    std::vector<int> src(nsys), len(nsys), dst(nsys);
    long long p = 0;
    for (int i = 0; i < nsys; i++) {
        if (!valid_slot(h, slot_ids[i])) return fail(h, SMR_ERR_ARG, "slot %d not active", slot_ids[i]);
        const SlotState& st = h->hs[slot_ids[i]];
        src[i] = (int)p; len[i] = st.natoms; dst[i] = st.atom_off;
        h->skey[slot_ids[i]] = locality_key(h, pos + 3 * p, st.natoms);
        for (int a = 0; a < st.natoms; a++) h->pinned[p + a] = make_float4(pos[3 * (p + a)], pos[3 * (p + a) + 1], pos[3 * (p + a) + 2], 0.f);
        p += st.natoms;
    }
    if (!nsys) return SMR_OK;
    std::vector<int> desc(3 * nsys);
    std::copy(src.begin(), src.end(), desc.begin()); std::copy(len.begin(), len.end(), desc.begin() + nsys); std::copy(dst.begin(), dst.end(), desc.begin() + 2 * nsys);
    CU(h, cudaMemcpyAsync(h->stage, h->pinned, p * 16, cudaMemcpyHostToDevice, h->stream));
    CU(h, cudaMemcpyAsync(h->xfer, desc.data(), desc.size() * 4, cudaMemcpyHostToDevice, h->stream));
    if (launch_copy_segments(h->xfer, h->xfer + nsys, h->xfer + 2 * nsys, nsys, h->stage, h->pos, h->stream)) return fail(h, SMR_ERR_CUDA, "scatter launch failed");
    // new positions carry no accumulated low part
    CU(h, cudaMemsetAsync(h->stage, 0, (size_t)p * 16, h->stream));
    if (launch_copy_segments(h->xfer, h->xfer + nsys, h->xfer + 2 * nsys, nsys, h->stage, h->plo, h->stream)) return fail(h, SMR_ERR_CUDA, "scatter launch failed");
    return wait_stream(h, h->watchdog_s);
}

int smr_active_slots(smr_handle* h, int* n, int* ids) {
    if (!h || !n) return SMR_ERR_ARG;
    int c = 0;
    for (int s = 0; s < h->max_systems; s++) if (h->hs[s].active) { if (ids) ids[c] = s; c++; }
    *n = c;
    return SMR_OK;
}

int smr_reset_fire(smr_handle* h, int nsys, const int* slot_ids) {
    if (!h || nsys < 0 || (nsys && !slot_ids)) return SMR_ERR_ARG;
    SETTLE(h);
    std::vector<int> ids;
    for (int i = 0; i < nsys; i++) {
        int s = slot_ids[i];
        if (!valid_slot(h, s)) return fail(h, SMR_ERR_ARG, "slot %d not active", s);
        SlotState& st = h->hs[s];
        st.status = 0; st.steps = 0; st.npos = 0; st.dt = -1.0; st.alpha = 0; st.energy = 0; st.fmax = 0;
        ids.push_back(s);
    }
    return upload_slots(h, ids);
}

int smr_eval_forces(smr_handle* h, int nsys, const int* slot_ids, float* forces, double* energy) {
    if (!h || nsys < 0 || (nsys && !slot_ids)) return SMR_ERR_ARG;
    SETTLE(h);
    { int r = check_batch(h, nsys, slot_ids); if (r) return r; }
    { int r = check_excl13(h, slot_ids, nsys); if (r) return r; }
    if (nsys == 0) return SMR_OK;
    std::vector<int> sorted(slot_ids, slot_ids + nsys);
    auto segs = group_by(h, sorted, h->eval_form, h->eval_team);
    std::vector<size_t> goff, glen;
    { int r = reserve_gscratch(h, plan_gscratch(h, segs, goff, glen)); if (r) return r; }
    std::vector<int> pos_in_input(h->max_systems);
    for (int i = 0; i < nsys; i++) pos_in_input[slot_ids[i]] = i;
    cudaStream_t s = h->stream;
    CU(h, cudaMemcpyAsync(h->work, sorted.data(), nsys * 4, cudaMemcpyHostToDevice, s));
    { int r = ensure_bricks(h); if (r) return r; }
    KernelArgs a = base_args(h);
    h->last_launches = 0;
    cudaEventRecord(h->ev0, s);
    for (size_t j = 0; j < segs.size(); j++) {
        const Seg& g = segs[j];
        a.work = h->work + g.begin; a.nwork = g.end - g.begin; a.nmax = g.nmax; a.nfmax = g.nfmax;
        a.gscratch = glen[j] ? h->gscr.d + goff[j] : nullptr; a.gscratch_bytes = glen[j];
        a.ecomp = h->ecomp + (size_t)g.begin * 8;
        CU(h, cudaMemsetAsync(h->counter, 0, 4, s));
        int r = launch_relax(a, g.team, g.form, 1, s, h->num_sms, &h->last_launches);
        if (r) return fail(h, SMR_ERR_CUDA, "eval launch: %s", cudaGetErrorString((cudaError_t)r));
    }
    cudaEventRecord(h->ev1, s);
    int r = wait_stream(h, h->watchdog_s);
    if (r) return r;
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->last_ms = ms;
    if (energy) {
        std::vector<double> e((size_t)nsys * 8);
        CU(h, cudaMemcpyAsync(e.data(), h->ecomp, e.size() * 8, cudaMemcpyDeviceToHost, h->stream));
        CU(h, cudaStreamSynchronize(h->stream));
        for (int i = 0; i < nsys; i++) std::copy(&e[(size_t)i * 8], &e[(size_t)i * 8 + 8], energy + (size_t)pos_in_input[sorted[i]] * 8);
    }
    if (forces) {
        r = smr_download(h, nsys, slot_ids, nullptr, forces, nullptr, nullptr, nullptr);
        if (r) return r;
    }
    return SMR_OK;
}

static bool team_ok(int t) { return t == 0 || t == 32 || t == 64 || t == 128 || t == 256 || t == 512; }
static bool form_ok(int f) { return f == FORM_ROUNDS || f == FORM_GATHER || f == FORM_OWNER; }

int smr_set_stages(smr_handle* h, int nstages, const int* starts, const int* forms, const int* teams, int eval_form) {
    if (!h || nstages < 1 || nstages > 16 || !starts || !forms || !teams) return SMR_ERR_ARG;
    if (starts[0] != 0) return fail(h, SMR_ERR_ARG, "the first stage must start at step 0");
    for (int k = 1; k < nstages; k++) if (starts[k] <= starts[k - 1]) return fail(h, SMR_ERR_ARG, "stage starts must increase");
    for (int k = 0; k < nstages; k++) {
        if (!team_ok(teams[k])) return fail(h, SMR_ERR_ARG, "stage team must be 0, 32, 64, 128, 256 or 512");
        if (!form_ok(forms[k])) return fail(h, SMR_ERR_ARG, "stage form must be 0 (rounds), 1 (gather) or 2 (owner)");
    }
    if (!form_ok(eval_form)) return fail(h, SMR_ERR_ARG, "eval form must be 0 (rounds), 1 (gather) or 2 (owner)");
    h->stage_start.assign(starts, starts + nstages);
    h->stage_form.assign(forms, forms + nstages);
    h->stage_team.assign(teams, teams + nstages);
    h->eval_form = eval_form;
    h->eval_team = 0;
    return SMR_OK;
}

int smr_get_stages(smr_handle* h, int* nstages, int* starts, int* forms, int* teams) {
    if (!h || !nstages) return SMR_ERR_ARG;
    const int n = (int)h->stage_start.size();
    if (starts && forms && teams) {
        if (*nstages < n) return fail(h, SMR_ERR_CAPACITY, "schedule has %d stages", n);
        std::copy(h->stage_start.begin(), h->stage_start.end(), starts);
        std::copy(h->stage_form.begin(), h->stage_form.end(), forms);
        std::copy(h->stage_team.begin(), h->stage_team.end(), teams);
    }
    *nstages = n;
    return SMR_OK;
}

int smr_set_schedule(smr_handle* h, int switch_step, int latency_team, int eval_form) {
    if (!h) return SMR_ERR_ARG;
    if (!team_ok(latency_team)) return fail(h, SMR_ERR_ARG, "latency team must be 0, 32, 64, 128, 256 or 512");
    int r;
    if (switch_step <= 0) { int st = 0, fm = FORM_ROUNDS, tm = 0; r = smr_set_stages(h, 1, &st, &fm, &tm, eval_form); }
    else {
        int st[2] = {0, switch_step}, fm[2] = {FORM_ROUNDS, FORM_GATHER}, tm[2] = {0, latency_team};
        r = smr_set_stages(h, 2, st, fm, tm, eval_form);
    }
    if (r == SMR_OK) h->eval_team = latency_team;
    return r;
}

int smr_get_schedule(smr_handle* h, int* switch_step, int* latency_team, int* eval_form) {
    if (!h) return SMR_ERR_ARG;
    if (switch_step) *switch_step = h->stage_start.size() > 1 ? h->stage_start[1] : 0;
    if (latency_team) *latency_team = h->stage_team.size() > 1 ? h->stage_team[1] : h->eval_team;
    if (eval_form) *eval_form = h->eval_form;
    return SMR_OK;
}

// every field a launch reads from its arguments, for comparing launch plans
static void sig_args(std::vector<long long>& v, const KernelArgs& a) {
    auto P = [&](const void* p) { v.push_back((long long)(uintptr_t)p); };
    auto F = [&](float x) { int b; std::memcpy(&b, &x, 4); v.push_back(b); };
    auto D = [&](double x) { long long b; std::memcpy(&b, &x, 8); v.push_back(b); };
    P(a.work); v.push_back(a.nwork); P(a.counter); P(a.slots); P(a.topos); P(a.req); P(a.neigh); P(a.bk); P(a.bl);
    P(a.angs); P(a.dihs); P(a.invs); P(a.pos); P(a.plo); P(a.vel); P(a.force);
    P(a.grid.data); v.push_back(a.grid.dtype); v.push_back(a.grid.nx); v.push_back(a.grid.ny); v.push_back(a.grid.nz);
    for (int k = 0; k < 3; k++) { F(a.grid.p0[k]); F(a.grid.inv_step[k]); }
    for (int k = 0; k < 4; k++) F(a.grid.scale[k]);
    P(a.grid.zscale); D(a.grid.p0z); D(a.grid.stepz); v.push_back(a.grid.brick);
    P(a.grid.lo); v.push_back(a.grid.zsplit); v.push_back(a.grid.lo_nz);
    for (int k = 0; k < 4; k++) F(a.grid.lo_scale[k]);
    v.push_back(a.has_grid); F(a.R2damp); F(a.alpha_morse); F(a.rc2);
    D(a.fire.dt0); D(a.fire.dt_max); D(a.fire.alpha0); D(a.fire.f_inc); D(a.fire.f_dec); D(a.fire.f_alpha);
    D(a.fire.fconv); D(a.fire.flimit); v.push_back(a.fire.n_min);
    v.push_back(a.phase_limit); v.push_back(a.step_budget); P(a.ecomp); v.push_back(a.nmax); v.push_back(a.nfmax);
    P(a.a2f); P(a.a2f_idx); P(a.own_geo); P(a.own_par); P(a.own_meta); v.push_back(a.nb_lanes);
    P(a.gscratch); v.push_back((long long)a.gscratch_bytes);
    P(a.neighc); P(a.lat); P(a.cons); P(a.tdrive);
    P(a.nbl); P(a.nbl_cnt); P(a.nbl_ref); v.push_back(a.nbl_cap); v.push_back(a.nbl_min); F(a.nbl_skin);
    v.push_back(a.fold.on); v.push_back(a.fold.nx); v.push_back(a.fold.ny); v.push_back(a.fold.nz);
    for (int k = 0; k < 4; k++) { F(a.fold.inv[k]); F(a.fold.inv_lo[k]); }
    F(a.fold.alpha); F(a.fold.fmax); P(a.fold.k); P(a.fold.coef);
}

int smr_set_graph(smr_handle* h, int on) {
    if (!h) return SMR_ERR_ARG;
    h->graph_on = on != 0;
    if (!h->graph_on && h->g_exec) { cudaGraphExecDestroy(h->g_exec); h->g_exec = nullptr; h->g_sig.clear(); }
    return SMR_OK;
}

int smr_graph_stats(smr_handle* h, long long* replays) {
    if (!h || !replays) return SMR_ERR_ARG;
    *replays = h->g_replays;
    return SMR_OK;
}

int smr_run_fire(smr_handle* h, int max_steps, int step_budget, const smr_fire_params* p, int mode, int* nfinished) {
    if (!h || !p || max_steps < 0) return SMR_ERR_ARG;
    SETTLE(h);
    if (mode != SMR_MODE_BATCHED && mode != SMR_MODE_PLAIN) return fail(h, SMR_ERR_ARG, "unknown mode %d", mode);
    if (!(p->dt0 > 0 && p->dt_max > 0 && p->f_dec > 0 && p->f_inc > 0)) return fail(h, SMR_ERR_ARG, "invalid FIRE parameters");
    {
        std::vector<int> run;
        for (int s = 0; s < h->max_systems; s++) if (h->hs[s].active && h->hs[s].status == SMR_ST_RUNNING) run.push_back(s);
        int r = check_excl13(h, run.data(), (int)run.size());
        if (r) return r;
    }
    // every running slot may advance to min(steps + max_steps, step_budget) in this call
    std::vector<int> ids;
    std::vector<int> start(h->max_systems, 0);
    for (int s = 0; s < h->max_systems; s++) {
        SlotState& st = h->hs[s];
        if (!st.active || st.status != SMR_ST_RUNNING) continue;
        const int cur = st.dt < 0 ? 0 : st.steps;
        long long tgt = (long long)cur + max_steps;
        if (step_budget > 0) tgt = std::min<long long>(tgt, step_budget);
        st.target = (int)std::min<long long>(tgt, 0x7fffffff);
        start[s] = cur;
        ids.push_back(s);
    }
    int r = upload_slots(h, ids);
    if (r) return r;
    // neighbour lists: allocated (max_atoms rows, all marked for rebuild) the first time a running
    // system is large enough under a cutoff
    if (!h->nbl_ready && h->nbl_min > 0 && h->nb.rcut > 0) {
        bool any = false;
        for (int sl : ids) any = any || h->hs[sl].natoms >= h->nbl_min;
        if (any) {
            const size_t na = (size_t)h->max_atoms;
            cudaError_t e = h->nbl.reserve(na * h->nbl_cap, 0, h->stream);
            if (e == cudaSuccess) e = h->nbl_cnt.reserve(na, 0, h->stream);
            if (e == cudaSuccess) e = h->nbl_ref.reserve(na, 0, h->stream);
            if (e == cudaSuccess) e = cudaMemsetAsync(h->nbl_cnt.d, 0xff, na * sizeof(int), h->stream);
            if (e == cudaSuccess) e = cudaMemsetAsync(h->nbl_ref.d, 0, na * sizeof(float4), h->stream);
            if (e != cudaSuccess) return fail(h, SMR_ERR_CAPACITY, "neighbour lists (%zu atoms x %d): %s", na, h->nbl_cap, cudaGetErrorString(e));
            h->nbl_ready = true;
        }
    }
    h->last_launches = 0;
    cudaStream_t s = h->stream;
    { int r = ensure_bricks(h); if (r) return r; }
    KernelArgs a = base_args(h);
    a.fire = FireDev{p->dt0, p->dt_max, p->alpha0, p->f_inc, p->f_dec, p->f_alpha, p->fconv, p->flimit, p->n_min};
    a.step_budget = step_budget;
    const int nst = (int)h->stage_start.size();
    auto stage_end = [&](int k) { return k + 1 < nst ? h->stage_start[k + 1] : 0x7fffffff; };
    // per stage: segments of the running systems in that stage's form and team
    std::vector<std::vector<int>> sids(nst, ids);
    std::vector<std::vector<Seg>> ssegs(nst);
    for (int k = 0; k < nst; k++) ssegs[k] = group_by(h, sids[k], h->stage_form[k], h->stage_team[k]);
    std::vector<std::vector<size_t>> goff(nst), glen(nst);
    size_t gneed = 0;
    for (int k = 0; k < nst; k++) gneed = std::max(gneed, plan_gscratch(h, ssegs[k], goff[k], glen[k]));
    r = reserve_gscratch(h, gneed);
    if (r) return r;
    cudaEventRecord(h->ev0, s);
    auto set_args = [&](const Seg& g, const int* work_base, int limit, int nwork_override, int* counter, size_t goffset, size_t gbytes) {
        a.work = work_base + g.begin; a.nwork = nwork_override > 0 ? nwork_override : g.end - g.begin;
        a.nmax = g.nmax; a.nfmax = g.nfmax; a.phase_limit = limit; a.counter = counter;
        a.gscratch = gbytes ? h->gscr.d + goffset : nullptr; a.gscratch_bytes = gbytes;
    };
    auto launch = [&](const Seg& g, const int* work_base, int limit, int nwork_override, cudaStream_t ls, int* counter,
                      size_t goffset, size_t gbytes) -> int {
        set_args(g, work_base, limit, nwork_override, counter, goffset, gbytes);
        CU(h, cudaMemsetAsync(counter, 0, 4, ls));
        int e = launch_relax(a, g.team, g.form, 0, ls, h->num_sms, &h->last_launches);
        if (e) return fail(h, SMR_ERR_CUDA, "relax launch: %s", cudaGetErrorString((cudaError_t)e));
        return 0;
    };
    if (mode == SMR_MODE_BATCHED) {
        // work lists of all stages in pinned memory (copied on the stream; a captured graph reads them)
        const size_t need = (size_t)nst * h->max_systems;
        if (need > h->work_pinned_cap) {
            if (h->work_pinned) cudaFreeHost(h->work_pinned);
            h->work_pinned = nullptr; h->work_pinned_cap = 0;
            CU(h, cudaMallocHost(&h->work_pinned, need * sizeof(int)));
            h->work_pinned_cap = need;
        }
        for (int k = 0; k < nst; k++) std::copy(sids[k].begin(), sids[k].end(), h->work_pinned + (size_t)k * h->max_systems);
        // stages run in order (every stage's launches redistribute the systems still running over
        // the GPU); the segments of one stage hold disjoint systems and run concurrently
        auto issue = [&]() -> int {
            for (int k = 0; k < nst; k++) {
                if (sids[k].empty()) continue;
                CU(h, cudaMemcpyAsync(h->work, h->work_pinned + (size_t)k * h->max_systems, sids[k].size() * 4, cudaMemcpyHostToDevice, s));
                const int m = (int)ssegs[k].size();
                const int nside = std::min(m, smr_handle::kSide);
                if (m > 1) {
                    CU(h, cudaEventRecord(h->ev_fork, s));
                    for (int j = 0; j < nside; j++) CU(h, cudaStreamWaitEvent(h->side[j], h->ev_fork, 0));
                }
                for (int j = 0; j < m; j++) {
                    cudaStream_t ls = m == 1 ? s : h->side[j % nside];
                    int* ctr = m == 1 ? h->counter : h->counter + (j % nside);
                    r = launch(ssegs[k][j], h->work, stage_end(k), 0, ls, ctr, goff[k][j], glen[k][j]);
                    if (r) return r;
                }
                if (m > 1)
                    for (int j = 0; j < nside; j++) {
                        CU(h, cudaEventRecord(h->ev_join[j], h->side[j]));
                        CU(h, cudaStreamWaitEvent(s, h->ev_join[j], 0));
                    }
            }
            return 0;
        };
        if (!h->graph_on) {
            r = issue();
            if (r) return r;
        } else {
            // the launch plan of this call (work lists, segments, every kernel argument), without issuing
            std::vector<long long> sig;
            long long nlaunch = 0;
            for (int k = 0; k < nst; k++) {
                if (sids[k].empty()) continue;
                sig.push_back(-1 - k);
                sig.insert(sig.end(), sids[k].begin(), sids[k].end());
                const int m = (int)ssegs[k].size();
                const int nside = std::min(m, smr_handle::kSide);
                for (int j = 0; j < m; j++) {
                    set_args(ssegs[k][j], h->work, stage_end(k), 0, m == 1 ? h->counter : h->counter + (j % nside), goff[k][j], glen[k][j]);
                    sig.push_back(ssegs[k][j].team); sig.push_back(ssegs[k][j].form); sig.push_back(m == 1 ? -1 : j % nside);
                    sig_args(sig, a);
                    nlaunch++;
                }
            }
            if (h->g_exec && sig == h->g_sig) {
                h->g_replays++;                                    // the same plan: replay it
            } else {
                cudaGraph_t graph = nullptr;
                const long long before = h->last_launches;
                CU(h, cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
                r = issue();
                cudaError_t ce = cudaStreamEndCapture(s, &graph);
                h->last_launches = before;
                if (r) { if (graph) cudaGraphDestroy(graph); return r; }
                if (ce != cudaSuccess) return fail(h, SMR_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
                cudaGraphExec_t ex = nullptr;
                cudaError_t ie = cudaGraphInstantiate(&ex, graph, 0);
                cudaGraphDestroy(graph);
                if (ie != cudaSuccess) return fail(h, SMR_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ie));
                if (h->g_exec) cudaGraphExecDestroy(h->g_exec);
                h->g_exec = ex;
                h->g_sig.swap(sig);
            }
            CU(h, cudaGraphLaunch(h->g_exec, s));
            h->last_launches += nlaunch;
        }
    } else {
        // plain form: one launch per system per FIRE step, status read back after each step
        CU(h, cudaMemcpyAsync(h->work, ids.data(), ids.size() * 4, cudaMemcpyHostToDevice, s));
        for (int kk = 0; kk < (int)ids.size(); kk++) {
            const int slot = ids[kk];
            const SlotState& st = h->hs[slot];
            std::vector<Seg> per_stage(nst);
            std::vector<size_t> pglen(nst, 0);
            for (int k = 0; k < nst; k++) {
                std::vector<int> one{slot};
                per_stage[k] = group_by(h, one, h->stage_form[k], h->stage_team[k])[0];
                per_stage[k].begin = kk; per_stage[k].end = kk + 1;
                std::vector<size_t> o1, l1;
                std::vector<Seg> g1{per_stage[k]};
                pglen[k] = plan_gscratch(h, g1, o1, l1);
                r = reserve_gscratch(h, pglen[k]);
                if (r) return r;
            }
            for (int steps = start[slot]; steps < st.target; steps++) {
                int k = 0;
                while (k + 1 < nst && steps >= h->stage_start[k + 1]) k++;
                r = launch(per_stage[k], h->work, steps + 1, 1, s, h->counter, 0, pglen[k]);
                if (r) return r;
                int stt = 0;
                CU(h, cudaMemcpyAsync(&stt, &h->slots[slot].status, 4, cudaMemcpyDeviceToHost, s));
                CU(h, cudaStreamSynchronize(s));
                if (stt != SMR_ST_RUNNING) break;
            }
        }
    }
    cudaEventRecord(h->ev1, s);
    r = wait_stream(h, h->watchdog_s);
    if (r) return r;
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->last_ms = ms;
    r = download_slots(h);
    if (r) return r;
    if (nfinished) {
        int c = 0;
        for (int s2 = 0; s2 < h->max_systems; s2++) if (h->hs[s2].active && h->hs[s2].status != SMR_ST_RUNNING) c++;
        *nfinished = c;
    }
    return SMR_OK;
}

int smr_download(smr_handle* h, int nsys, const int* slot_ids, float* pos, float* forces, double* energy, int* steps, int* status) {
    if (!h || nsys < 0 || (nsys && !slot_ids)) return SMR_ERR_ARG;
    SETTLE(h);
    { int r = check_batch(h, nsys, slot_ids); if (r) return r; }
    for (int i = 0; i < nsys; i++) if (!valid_slot(h, slot_ids[i])) return fail(h, SMR_ERR_ARG, "slot %d not active", slot_ids[i]);
    if (!nsys) return SMR_OK;
    int r = download_slots(h);
    if (r) return r;
    std::vector<int> src(nsys), len(nsys), dst(nsys);
    long long p = 0;
    for (int i = 0; i < nsys; i++) {
        const SlotState& st = h->hs[slot_ids[i]];
        src[i] = st.atom_off; len[i] = st.natoms; dst[i] = (int)p;
        p += st.natoms;
        if (energy) { energy[(size_t)i * SMR_E_NCOMP] = st.energy; for (int c = 1; c < SMR_E_NCOMP; c++) energy[(size_t)i * SMR_E_NCOMP + c] = 0.0; }
        if (steps) steps[i] = st.steps;
        if (status) status[i] = st.status;
    }
    std::vector<int> desc(3 * nsys);
    std::copy(src.begin(), src.end(), desc.begin()); std::copy(len.begin(), len.end(), desc.begin() + nsys); std::copy(dst.begin(), dst.end(), desc.begin() + 2 * nsys);
    cudaStream_t s = h->stream;
    CU(h, cudaMemcpyAsync(h->xfer, desc.data(), desc.size() * 4, cudaMemcpyHostToDevice, s));
    for (int which = 0; which < 2; which++) {
        float* out = which == 0 ? pos : forces;
        if (!out) continue;
        if (launch_copy_segments(h->xfer, h->xfer + nsys, h->xfer + 2 * nsys, nsys, which == 0 ? h->pos : h->force, h->stage, s))
            return fail(h, SMR_ERR_CUDA, "gather launch failed");
        CU(h, cudaMemcpyAsync(h->pinned, h->stage, p * 16, cudaMemcpyDeviceToHost, s));
        r = wait_stream(h, h->watchdog_s);
        if (r) return r;
        if (which == 0) for (long long a = 0; a < p; a++) { out[3 * a] = h->pinned[a].x; out[3 * a + 1] = h->pinned[a].y; out[3 * a + 2] = h->pinned[a].z; }
        else std::memcpy(out, h->pinned, p * 16);
    }
    return SMR_OK;
}

int smr_download_pos64(smr_handle* h, int nsys, const int* slot_ids, double* pos) {
    if (!h || nsys < 0 || (nsys && (!slot_ids || !pos))) return SMR_ERR_ARG;
    SETTLE(h);
    { int r = check_batch(h, nsys, slot_ids); if (r) return r; }
    for (int i = 0; i < nsys; i++) if (!valid_slot(h, slot_ids[i])) return fail(h, SMR_ERR_ARG, "slot %d not active", slot_ids[i]);
    if (!nsys) return SMR_OK;
    std::vector<int> desc(3 * nsys);
    long long p = 0;
    for (int i = 0; i < nsys; i++) {
        const SlotState& st = h->hs[slot_ids[i]];
        desc[i] = st.atom_off; desc[nsys + i] = st.natoms; desc[2 * nsys + i] = (int)p;
        p += st.natoms;
    }
    cudaStream_t s = h->stream;
    CU(h, cudaMemcpyAsync(h->xfer, desc.data(), desc.size() * 4, cudaMemcpyHostToDevice, s));
    std::vector<float4> hi((size_t)p);
    for (int which = 0; which < 2; which++) {
        if (launch_copy_segments(h->xfer, h->xfer + nsys, h->xfer + 2 * nsys, nsys, which == 0 ? h->pos : h->plo, h->stage, s))
            return fail(h, SMR_ERR_CUDA, "gather launch failed");
        CU(h, cudaMemcpyAsync(h->pinned, h->stage, p * 16, cudaMemcpyDeviceToHost, s));
        int r = wait_stream(h, h->watchdog_s);
        if (r) return r;
        if (which == 0) std::memcpy(hi.data(), h->pinned, p * 16);
    }
    for (long long a = 0; a < p; a++) {
        pos[3 * a] = (double)hi[a].x + (double)h->pinned[a].x;
        pos[3 * a + 1] = (double)hi[a].y + (double)h->pinned[a].y;
        pos[3 * a + 2] = (double)hi[a].z + (double)h->pinned[a].z;
    }
    return SMR_OK;
}

struct smr_topo { HostTopo T; PreparedTopo prep; bool prepared = false; };

int smr_topo_prepare(smr_topo* t, int team) {
    if (!t) return SMR_ERR_ARG;
    if (team == 0) team = default_team(t->T.n);
    if (team != 32 && team != 64 && team != 128 && team != 256 && team != 512) return SMR_ERR_ARG;
    prepare_topology(t->T, team, t->prep);
    t->prepared = true;
    return SMR_OK;
}

int smr_add_topos(smr_handle* h, int n, const smr_topo* const* topos, int* topo_ids) {
    if (!h || n < 0 || (n && (!topos || !topo_ids))) return SMR_ERR_ARG;
    SETTLE(h);
    for (int i = 0; i < n; i++) if (!topos[i]) return fail(h, SMR_ERR_ARG, "topology %d is null", i);
    for (int i = 0; i < n; i++) {
        const smr_topo* t = topos[i];
        h->topos.push_back(t->T);
        h->topo_alive.push_back(1);
        const int team = team_for(h, t->T.n);
        if (t->prepared && t->prep.team == team) commit_topology(h, h->topos.back(), t->prep);
        else append_topology(h, h->topos.back());
        topo_ids[i] = (int)h->topos.size() - 1;
    }
    return upload_all(h);
}

static int remove_one_topology(smr_handle* h, int id) {
    if (id < 0 || id >= (int)h->topos.size() || !h->topo_alive[id]) return fail(h, SMR_ERR_ARG, "topology %d not live", id);
    for (int s = 0; s < h->max_systems; s++)
        if (h->hs[s].active && h->hs[s].topo == id) return fail(h, SMR_ERR_STATE, "topology %d is used by slot %d", id, s);
    h->topo_alive[id] = 0;
    h->dead_atoms += h->topos[id].n;
    h->topos[id] = HostTopo{};
    return SMR_OK;
}

static int maybe_compact(smr_handle* h) {
    const size_t live = h->hreq.size() - h->dead_atoms;
    if (h->dead_atoms > 4096 && h->dead_atoms > live) return compact_topologies(h);
    return SMR_OK;
}

int smr_remove_topologies(smr_handle* h, int n, const int* ids) {
    if (!h || n < 0 || (n && !ids)) return SMR_ERR_ARG;
    SETTLE(h);
    for (int i = 0; i < n; i++) { int r = remove_one_topology(h, ids[i]); if (r) return r; }
    return maybe_compact(h);
}

int smr_remove_topology(smr_handle* h, int id) {
    if (!h) return SMR_ERR_ARG;
    SETTLE(h);
    int r = remove_one_topology(h, id);
    if (r) return r;
    return maybe_compact(h);
}

int smr_topo_build(int natoms, const int* Z, const double* pos, const double* charges, double bond_cut, smr_topo** out,
                   char* err, int errlen) {
    if (!Z || !pos || !out) return SMR_ERR_ARG;
    *out = nullptr;
    smr_topo* t = new (std::nothrow) smr_topo();
    if (!t) return SMR_ERR_CAPACITY;
    char msg[300] = {0};
    if (build_molecule_topology(natoms, Z, pos, charges, bond_cut > 0 ? bond_cut : 1.8, t->T, msg, sizeof(msg))) {
        if (err && errlen > 0) std::snprintf(err, errlen, "%s", msg);
        delete t;
        return SMR_ERR_ARG;
    }
    *out = t;
    return SMR_OK;
}

int smr_topo_build_listed(int natoms, const int* Z, const int* type_ids, const double* charges, int nbonds, const int* bonds,
                          int nang, const int* angs, int ndih, const int* dihs, int ninv, const int* invs, smr_topo** out,
                          char* err, int errlen) {
    if (!Z || !out || (nbonds && !bonds) || (nang && !angs) || (ndih && !dihs) || (ninv && !invs)) return SMR_ERR_ARG;
    *out = nullptr;
    smr_topo* t = new (std::nothrow) smr_topo();
    if (!t) return SMR_ERR_CAPACITY;
    char msg[300] = {0};
    if (build_listed_topology(natoms, Z, type_ids, charges, nbonds, bonds, nang, angs, ndih, dihs, ninv, invs, t->T, msg, sizeof(msg))) {
        if (err && errlen > 0) std::snprintf(err, errlen, "%s", msg);
        delete t;
        return SMR_ERR_ARG;
    }
    *out = t;
    return SMR_OK;
}

int smr_type_id(const char* name) { return name ? type_id_of(name) : -1; }

void smr_topo_free(smr_topo* t) { delete t; }

int smr_topo_counts(const smr_topo* t, int c[5]) {
    if (!t || !c) return SMR_ERR_ARG;
    c[0] = t->T.n; c[1] = (int)t->T.bonds.size() / 2; c[2] = (int)t->T.angs.size() / 3;
    c[3] = (int)t->T.dihs.size() / 4; c[4] = (int)t->T.invs.size() / 4;
    return SMR_OK;
}

int smr_topo_export(const smr_topo* t, int* neighs, int* neighBs, int* bonds, double* bparams,
                    int* angs, int* ang_ngs, double* angp, int* dihs, int* dih_ngs, double* dihp,
                    int* invs, int* inv_ngs, double* invp, double* req, int* type_id) {
    if (!t) return SMR_ERR_ARG;
    const HostTopo& T = t->T;
    auto cp = [](auto* dst, const auto& v) { if (dst) std::copy(v.begin(), v.end(), dst); };
    cp(neighs, T.neighs); cp(neighBs, T.neighBs); cp(bonds, T.bonds); cp(bparams, T.bparams);
    cp(angs, T.angs); cp(ang_ngs, T.ang_ngs); cp(angp, T.angp);
    cp(dihs, T.dihs); cp(dih_ngs, T.dih_ngs); cp(dihp, T.dihp);
    cp(invs, T.invs); cp(inv_ngs, T.inv_ngs); cp(invp, T.invp);
    cp(req, T.req); cp(type_id, T.type_id);
    return SMR_OK;
}

int smr_topo_rounds(const smr_topo* t, int team, int rounds[3], short* ang_at, short* dih_at, short* inv_at) {
    if (!t || !rounds || team <= 0) return SMR_ERR_ARG;
    PackedTerms P;
    pack_rounds(t->T, team, P);
    rounds[0] = P.ang_rounds; rounds[1] = P.dih_rounds; rounds[2] = P.inv_rounds;
    auto put = [](short* dst, const auto& recs) {
        if (!dst) return;
        for (size_t i = 0; i < recs.size(); i++) {
            dst[4 * i] = recs[i].at.x; dst[4 * i + 1] = recs[i].at.y; dst[4 * i + 2] = recs[i].at.z; dst[4 * i + 3] = recs[i].at.w;
        }
    };
    put(ang_at, P.ang); put(dih_at, P.dih); put(inv_at, P.inv);
    return SMR_OK;
}

int smr_add_topo(smr_handle* h, const smr_topo* t, int* topo_id) {
    if (!h || !t || !topo_id) return SMR_ERR_ARG;
    SETTLE(h);
    h->topos.push_back(t->T);
    h->topo_alive.push_back(1);
    const int team = team_for(h, t->T.n);
    if (t->prepared && t->prep.team == team) commit_topology(h, h->topos.back(), t->prep);   // packed off the handle
    else append_topology(h, h->topos.back());
    int r = upload_all(h);
    if (r) return r;
    *topo_id = (int)h->topos.size() - 1;
    return SMR_OK;
}

int smr_last_timing(smr_handle* h, double* ms, long long* launches) {
    if (!h) return SMR_ERR_ARG;
    if (ms) *ms = h->last_ms;
    if (launches) *launches = h->last_launches;
    return SMR_OK;
}

}  // extern "C"
