// smr_internal.h -- layouts shared by the host runtime (abi.cpp, topology.cpp) and
// the CUDA kernels (relax.cu, grid.cu).  Device memory is laid out as:
//
//   per atom of a topology (arena, indexed by TopoDev::atom_off + local atom):
//     float4 req   (R_vdW, sqrt(E_vdW), Q, H)
//     short4 neigh (up to 4 bonded neighbours, -1 padded; local indices)
//     float4 bk, bl (bond k and l0 of each neighbour slot)
//   per term, in "rounds" of T records (T = team size of the topology's class):
//     AngRec / DihRec / InvRec, 32 B each; within one round the atoms in each
//     role are pairwise distinct, so a team adds the round's force pieces to its
//     shared-memory force array without atomics and in a fixed order.
//   per atom of a system (state arena, indexed by SlotState::atom_off + local atom):
//     float4 pos, plo (low parts of the positions), vel, force (force.w = per-atom energy)
//   per system: SlotState (FIRE state, status, energy)
//   grid: z-fastest i = iz + nz*(iy + ny*ix), float4 or 4 x 16-bit per voxel.
#pragma once
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

namespace smr {

struct __align__(16) AngRec { short4 at; short4 sl; float4 p; };   // at (i,j,k,-) sl (ji,jk,-,-) p (K*c0..K*c3)
struct __align__(16) DihRec { short4 at; short4 sl; float4 p; };   // at (i,j,k,l) sl (ji,jk,kl,-) p (V, d, n, -)
struct __align__(16) InvRec { short4 at; short4 sl; float4 p; };   // at (i,j,k,l) sl (ij,ik,il,-) p (K, c0, c1, c2)

static_assert(sizeof(AngRec) == 32 && sizeof(DihRec) == 32 && sizeof(InvRec) == 32, "record size");

struct TopoDev {
    int natoms;
    int atom_off;                 // into req / neigh / bk / bl / a2f
    int ang_off, ang_rounds;      // into the AngRec arena; ang_rounds * team records
    int dih_off, dih_rounds;
    int inv_off, inv_rounds;
    int team;                     // team size the rounds were packed for
    // gather form: unpadded term records (canonical orientation), piece buffer and per-atom
    // lists of piece indices (angles 3 pieces, dihedrals and inversions 4; the pieces of term
    // kind k start at 0, 3*nang, 3*nang + 4*ndih)
    int fang_off, fdih_off, finv_off;
    int nang, ndih, ninv;
    int npieces;
    int a2f_off;                  // into the piece-index arena; per atom (start, count) at atom_off
    // owner form: every term is evaluated by an atom whose neighbour slots cover the term's
    // other atoms (angles by the apex, inversions by the centre, each dihedral twice: by j for
    // (i, j) and by k for (k, l)).  Records of one kind are stored by row: row r of owner o at
    // off + r * natoms + o, so a warp's lanes read consecutive records.
    int own_a_off, own_i_off, own_d_off;   // into the owner record arenas (geo + par)
    int own_ok;                   // 0: the topology cannot run the owner form (rounds instead)
    int pbc_bonds;                // 1: some bonds reach a neighbour's image in another cell (cell codes in neighc)
    int pad[2];
};
static_assert(sizeof(TopoDev) == 96, "TopoDev size");

struct SlotState {
    int topo;                     // topology id
    int atom_off;                 // into pos / vel / force
    int natoms;
    int status;                   // SMR_ST_*
    int steps;                    // FIRE steps done
    int npos;                     // FIRE consecutive uphill-free steps
    int active;                   // slot in use
    int target;                   // absolute step count this smr_run_fire call may reach
    double dt, alpha;             // FIRE adaptive state
    double energy;                // total physical energy at the last force evaluation
    float fmax;                   // max |F| at the last force evaluation
    int flags;                    // SLOT_PBC: lattice in KernelArgs::lat; SLOT_CONS: position constraints in KernelArgs::cons;
                                  // SLOT_THERM: Langevin drive in KernelArgs::tdrive
};

enum GridDtype { GRID_F32 = 0, GRID_F16 = 1, GRID_BF16 = 2 };

struct GridView {
    const void* data;
    int dtype;
    int nx, ny, nz;
    float p0[3];
    float inv_step[3];
    float scale[4];               // per-channel scale of the stored values (when zscale is null)
    const float4* zscale;         // 16-bit grids: per z plane and channel scale (null: scale[])
    int brick;                    // 1: data is the brick copy (build_grid_bricks), not the z-fastest grid
    double p0z, stepz;            // z origin and step in FP64 (cell decisions at the grid's z bounds)
    // 16-bit grids with FP32 near-surface planes (smr_convert_grid_split): a cell whose stencil
    // starts below plane zsplit (iz - 1 < zsplit) reads the FP32 copy lo of the planes
    // [0, lo_nz = zsplit + 3) instead, in the same layout as data (bricks or z-fastest), with
    // the channel scales lo_scale; zsplit = 0: no copy
    const void* lo;
    int zsplit, lo_nz;
    float lo_scale[4];
};

// folded-surface substrate (SurfaceFolded, crates/libs/surfff/src/lib.rs:126-351)
struct FoldedView {
    int on;
    int nx, ny, nz;
    float inv[4];                 // inv_ax, inv_bx, inv_ay, inv_by (rounded to float)
    float inv_lo[4];              // their rounding remainders: inverse = inv + inv_lo
    float alpha, fmax;            // make_plqs exponent, per-atom force clamp
    const float* k;               // kx[nx], ky[ny], kz[nz], z0[nz]
    const float4* coef;           // per basis function (cq, cp, cl, 0), index ix + nx (iy + ny iz)
};

struct FireDev {
    double dt0, dt_max, alpha0, f_inc, f_dec, f_alpha, fconv, flimit;
    int n_min;
};

struct KernelArgs {
    const int* work; int nwork; int* counter;
    SlotState* slots;
    const TopoDev* topos;
    const float4* req; const short4* neigh; const float4* bk; const float4* bl;
    // periodic molecules: per atom the cell code of each bond slot's partner image (4-bit
    // two's-complement lattice offsets x | y << 4 | z << 8; 0 = same cell), and per slot the
    // lattice: lat[3 s + k] = (vector k, number of images each side along it)
    const short4* neighc; const float4* lat;
    // position constraints: per state atom g, cons[2 g] = (target x, y, z, on), cons[2 g + 1] = (kx, ky, kz, 0)
    const float4* cons;
    // Langevin drive per slot: (T [K], gamma, seed increment per FIRE step, seed)
    const float4* tdrive;
    const AngRec* angs; const DihRec* dihs; const InvRec* invs;
    float4* pos; float4* plo; float4* vel; float4* force;
    GridView grid; int has_grid;
    FoldedView fold;              // fold.on: the substrate is the folded surface, not the grid
    float R2damp, alpha_morse, rc2;
    int excl13;                   // 1: 1-3 pairs excluded too (getNonBond_GridFF_Bspline_ex2)
    int grid_prefetch;            // 1: L2 prefetch of the brick lines at the start of each evaluation
    int smem_carveout;            // block teams: preferred shared-memory carveout in percent (-1: driver default)
    FireDev fire;
    int phase_limit;              // this launch runs a system until SlotState::steps reaches min(target, phase_limit)
    int step_budget;              // a system reaching this many steps gets SMR_ST_MAXSTEPS (<=0: none)
    double* ecomp;                // eval mode: per work item x 8 energy components
    int nmax;                     // max atoms of a system in this launch (shared-memory sizing)
    int nfmax;                    // gather form: max pieces of a system in this launch
    const int2* a2f;              // gather form: per atom (first piece-index entry, count)
    const int* a2f_idx;           // gather form: piece indices
    const short4* own_geo;        // owner form: hneigh indices (+ dihedral half in .w)
    const float4* own_par;        // owner form: term parameters
    const int* own_meta;          // owner form, per atom: n_ang | n_inv << 8 | n_dih << 16 | back slots << 24
    int nb_lanes;                 // lanes per atom in the NB partner loop (0: chosen from N and the team)
    // systems too large for shared memory: each team's state lives in this global buffer instead
    // (team k of the launch at k * team bytes); null for shared-memory launches
    char* gscratch;
    size_t gscratch_bytes;
    // NB neighbour lists (systems of at least nbl_min atoms under a cutoff, FIRE steps only): row of
    // state atom g at nbl + g * nbl_cap holds the partners within rc + skin in ascending order,
    // nbl_cnt[g] their number (-1: rebuild, -2: overflow, use all pairs), nbl_ref[g] the
    // position at the last build
    unsigned short* nbl;
    int* nbl_cnt;
    float4* nbl_ref;
    int nbl_cap, nbl_min;
    float nbl_skin;
};

// ---- host topology (topology.cpp)
struct HostTopo {
    int n = 0;
    std::vector<int> neighs, neighBs;                 // 4n
    std::vector<int> bonds; std::vector<double> bparams;
    std::vector<int> angs, ang_ngs; std::vector<double> angp;   // 3, 2, 5 per angle
    std::vector<int> dihs, dih_ngs; std::vector<double> dihp;   // 4, 3, 3
    std::vector<int> dih_kj;                          // slot of j in k's neighbour list (reversed dihedral)
    std::vector<int> invs, inv_ngs; std::vector<double> invp;   // 4, 3, 4
    std::vector<double> req;                          // 4n
    std::vector<double> bond_kl;                      // 8n: (k, l0) per neighbour slot
    std::vector<int> type_id;                         // n
    // periodic molecules: per neighbour slot the cell code of the partner's image (4n, empty for
    // molecules without periodic bonds), the lattice the molecule was built in and its images
    std::vector<int> neighc;
    double lattice[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    int npbc[3] = {0, 0, 0};
};

// cell code of a lattice offset (each component in [-8, 7]) and its components
inline int cell_code(int ox, int oy, int oz) { return (ox & 15) | ((oy & 15) << 4) | ((oz & 15) << 8); }
inline int cell_field(int c, int k) { int v = (c >> (4 * k)) & 15; return v >= 8 ? v - 16 : v; }

struct PackedTerms {
    std::vector<AngRec> ang; std::vector<DihRec> dih; std::vector<InvRec> inv;
    int ang_rounds = 0, dih_rounds = 0, inv_rounds = 0;
};

struct OwnerTerms {                // owner form of one topology
    std::vector<short4> geo;       // angle rows, then inversion rows, then dihedral rows
    std::vector<float4> par;
    std::vector<int> meta;         // per atom
    int rows_a = 0, rows_i = 0, rows_d = 0;
    bool ok = false;
};

struct FlatTerms {                 // gather form of one topology
    std::vector<AngRec> ang; std::vector<DihRec> dih; std::vector<InvRec> inv;
    std::vector<int2> a2f;         // per atom (start into idx, count)
    std::vector<int> idx;          // piece indices grouped by atom, in term order
    int npieces = 0;
};

// topology.cpp
int build_molecule_topology(int n, const int* Z, const double* pos, const double* q, double bond_cut, HostTopo& T,
                            char* err, int errlen);
int build_desc_topology(int natoms, const double* req, const int* neighs, const double* bond_kl,
                        int nang, const int* angs, const double* angp, int ndih, const int* dihs, const double* dihp,
                        int ninv, const int* invs, const double* invp, HostTopo& T, char* err, int errlen);
void pack_rounds(const HostTopo& T, int team, PackedTerms& out);
void flat_terms(const HostTopo& T, FlatTerms& out);
bool owner_terms(const HostTopo& T, OwnerTerms& out);
const char* type_name(int id);
int type_id_of(const char* name);
int build_molecule_topology_pbc(int n, const int* Z, const double* pos, const double* q, double bond_cut,
                                const double lvec[9], HostTopo& T, char* err, int errlen);
int build_listed_topology(int n, const int* Z, const int* type_ids, const double* q, int nb, const int* bonds, int na,
                          const int* angs, int nd, const int* dihs, int ni, const int* invs, HostTopo& T, char* err, int errlen);

// relax.cu
// FORM_GATHER_EXT: the gather form with the code of the rarer per-system features compiled in
// (periodic systems: bond shifts, NB image sums; position constraints); the host sends every
// system that uses one there, so the other forms carry none of it
enum SlotFlags { SLOT_PBC = 1, SLOT_CONS = 2, SLOT_THERM = 4 };
enum KernelForm { FORM_ROUNDS = 0, FORM_GATHER = 1, FORM_OWNER = 2, FORM_GATHER_EXT = 3 };
int launch_relax(const KernelArgs& a, int team, int form, int eval_only, cudaStream_t s, int num_sms, long long* launches);
size_t team_smem_bytes(int nmax, int nfmax, int team, int form);
// Minimum blocks per SM the relax kernel's __launch_bounds__ asks for: warp teams run 4 to a
// 128-thread block at 72 registers (80 in the owner form), 7 (6) blocks; 64- and 128-thread teams
// get the occupancy their shared memory allows for typical sizes (6 blocks up to 160 atoms, 3 up
// to 448), i.e. at most 168 registers, which the NB loop's grouped pairs would otherwise exceed
// (~187).  Lower caps for more resident teams were measured: 128 or 96 registers made the ragged
// workload 11-25 % slower, the extra teams thrashing L1 on their global reads.
constexpr int relax_min_blocks(int T, int form) {
    return T == 32 ? (form == FORM_OWNER ? 6 : 7) : T == 64 ? 6 : T == 128 ? 3 : 1;
}
// Blocks of one launch segment that fit on an SM by shared memory (228 KB per SM, 1 KB reserved
// per block), capped at 16 (the occupancy tiers of group_by).
inline int relax_blocks_per_sm(size_t smem_per_block, int T, int form) {
    const int by_smem = (int)(233472 / (smem_per_block + 1024));
    (void)T; (void)form;
    return by_smem < 16 ? by_smem : 16;
}

// grid.cu
struct GridBuildArgs {
    int nions; const double* ions; const double* ion_re;   // device pointers, 4 doubles per ion
    double Lx, Ly; int nx, ny, nz; double p0[3], step[3];
    double alpha; int npbc; double ewald_tol; double morse_rcut;
};
int build_grid_device(const GridBuildArgs& a, float4* out_f32, cudaStream_t s, char* err, int errlen);
// sharded build: raw FP64 (Pauli, London, Coulomb) triples of the x-planes [x0, x0 + xs), voxel-major
// z-fastest, into raw (device); then the fit and pack of a whole grid from such triples
int grid_raw_slab_device(const GridBuildArgs& a, int x0, int xs, double* raw, cudaStream_t s, char* err, int errlen);
int grid_from_raw_device(const double* raw, int nx, int ny, int nz, float4* out_f32, cudaStream_t s, char* err, int errlen);
// 16-bit storage with one power-of-two scale per z plane and channel: plane_scale_out gets nz x 4
// floats (host); decode takes them as a device table
int encode_grid_16(const float4* src, void* dst, size_t nvox, int nz, int dtype, float* plane_scale_out, cudaStream_t s);
int decode_grid_16(const void* src, float4* dst, size_t nvox, int nz, int dtype, const float4* d_plane_scale, cudaStream_t s);
// dst (nxy columns of nzl planes, z-fastest) = the planes [0, nzl) of src (nxy columns of nz planes)
int extract_low_planes(const float4* src, size_t nxy, int nz, int nzl, float4* dst, cudaStream_t s);
// Brick copy of a z-fastest grid for the relax kernel's stencil reads.  Brick (ix, iy, jz),
// jz in [0, nz - 3), is one 128-byte line holding the voxels (iy + dy mod ny, jz + k), k < 4,
// dy < grid_brick_rows(dtype) (2 rows of 16-byte float4 voxels, 4 rows of 8-byte 16-bit ones),
// stored dy-major.  0 elements when the grid is too small or the copy would need 2^32 voxels.
inline int grid_brick_rows(int dtype) { return dtype == GRID_F32 ? 2 : 4; }
size_t grid_brick_bytes(int nx, int ny, int nz);
int build_grid_bricks(const void* grid, int dtype, int nx, int ny, int nz, void* bricks, cudaStream_t s);

}  // namespace smr
