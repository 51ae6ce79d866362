/* surfmol_relax.h -- C ABI of the B200 multi-system UFF + GridFF FIRE relaxation library.
 *
 * One handle = one CUDA device + one stream; not thread-safe (callers serialise).
 * The library owns device memory; the caller owns every host array.  Every
 * function returns an int status (SMR_OK = 0, negative on error) and never
 * aborts; smr_last_error() gives the message of the last failure.
 *
 * Reference interfaces each entry point replaces (paths inside ProkopHapala/SurfMol):
 *   handle lifecycle ........ crates/libs/oclff/src/rrsp3.rs:742 (RRsp3Multi::new), :1085 (finish),
 *                             crates/libs/molff/src/ffi_uff.rs:42,82 (uff_new / uff_free)
 *   grid .................... crates/libs/oclff/src/surfff.rs:187-221 (GridFFBuildOcl / GridFFEvalOcl),
 *                             opencl/gridff_build.cl:350-463, opencl/Surface.cl:716-906 (builders),
 *                             opencl/UFF.cl:1524-1545 (BsplinePLQ, grid_ns, grid_invStep, grid_p0 arguments)
 *   molecules / topology .... crates/libs/molff/src/ffi_uff.rs:42-80 (uff_new: elements + positions ->
 *                             topology, UFF typing and parameters), crates/libs/molff/src/uff.rs:699-887
 *   systems ................. crates/libs/oclff/src/rrsp3.rs:936 (upload_state_multi)
 *   relaxation .............. crates/apps/molengine/src/main.rs:237-277 (relax_fire),
 *                             crates/libs/molff/src/ffi_uff.rs:133 (uff_relax),
 *                             crates/libs/oclff/src/rrsp3.rs:1028 (step_cluster_multi)
 *   evaluation .............. crates/libs/molff/src/ffi_uff.rs:96 (uff_eval),
 *                             crates/libs/surfmol/src/mol_world.rs:60-86 (eval_forces)
 *   read-back ............... crates/libs/oclff/src/rrsp3.rs:976,991 (download_pos_multi / _replica),
 *                             crates/libs/molff/src/ffi_uff.rs:109 (uff_get_pos)
 */
#ifndef SURFMOL_RELAX_H
#define SURFMOL_RELAX_H

#ifdef __cplusplus
extern "C" {
#endif

#define SMR_OK               0
#define SMR_ERR_ARG         -1   /* invalid argument (null pointer, bad size, bad id) */
#define SMR_ERR_CUDA        -2   /* CUDA runtime error */
#define SMR_ERR_CAPACITY    -3   /* slot / atom capacity or per-system size limit exceeded */
#define SMR_ERR_STATE       -4   /* call out of order (e.g. relax before a grid is set) */
#define SMR_ERR_UNSUPPORTED -5   /* option not implemented */
#define SMR_ERR_TIMEOUT     -6   /* device work did not finish within the watchdog limit */

/* per-system status word written by relaxation */
#define SMR_ST_RUNNING    0      /* steps remain, not converged */
#define SMR_ST_CONVERGED  1      /* max|F| < fconv */
#define SMR_ST_MAXSTEPS   2      /* step budget of the system used up */
#define SMR_ST_NONFINITE  3      /* a force or position became NaN/Inf; the system stopped */

#define SMR_GRID_F32   0         /* float4 coefficients */
#define SMR_GRID_F16   1         /* 4 x binary16, value = stored * scale[channel] */
#define SMR_GRID_BF16  2         /* 4 x bfloat16, value = stored * scale[channel] */

#define SMR_MODE_BATCHED 0       /* persistent kernel, all active systems, dynamic system scheduling */
#define SMR_MODE_PLAIN   1       /* one launch per system per FIRE step, status read back each step */

/* energy components returned per system (physical totals: each bond and NB pair once) */
#define SMR_E_TOTAL 0
#define SMR_E_BOND  1
#define SMR_E_ANGLE 2
#define SMR_E_DIH   3
#define SMR_E_INV   4
#define SMR_E_NB    5
#define SMR_E_GRID  6
#define SMR_E_NCOMP 8

typedef struct smr_handle smr_handle;

typedef struct {
    int       device;        /* CUDA device ordinal */
    int       max_systems;   /* slot capacity */
    long long max_atoms;     /* atom capacity summed over all slots */
    int       reserved[6];
} smr_config;

/* FIRE parameters: FireState (crates/libs/molff/src/raff.rs:1040-1062) + relax_fire's
 * dt0/dt_max/fconv (crates/apps/molengine/src/main.rs:237).  flimit <= 0: no force clamp. */
typedef struct {
    double dt0, dt_max, alpha0, f_inc, f_dec, f_alpha;
    int    n_min;
    double fconv;
    double flimit;
} smr_fire_params;

/* Non-bonded / grid-coupling parameters: GFFParams.x (rdamp), GFFParams.y (Morse alpha)
 * of opencl/UFF.cl:1534-1545; rcut <= 0 keeps every intramolecular pair.
 * excl13 = 0: bonded (1-2) pairs excluded, getNonBond_GridFF_Bspline (UFF.cl:1524-1718);
 * excl13 = 1: 1-2 and 1-3 pairs excluded, getNonBond_GridFF_Bspline_ex2 (UFF.cl:1722-1930)
 * with the exclusion lists of NonBondedFF::make_second_neighs (molff/src/nonbonded.rs:112-137).
 * A system with PBC images runs only with excl13 = 0 (the reference has no image-aware 1-3
 * list builder); smr_run_fire / smr_eval_forces refuse the combination with SMR_ERR_ARG. */
typedef struct {
    float rdamp;
    float alpha_morse;
    float rcut;
    int   excl13;
} smr_nb_params;

/* Grid build: Morse (Pauli, London) image sums + Ewald-2D Coulomb, exact B-spline fit. */
typedef struct {
    double alpha_morse;      /* Morse exponent of the substrate channels */
    int    npbc;             /* lateral images each side for the Morse sums (make_MorseFF nPBC) */
    double ewald_tol;        /* relative truncation of the reciprocal sum, e.g. 1e-12 */
    int    dtype;            /* SMR_GRID_* storage of the result */
    double morse_rcut;       /* <= 0: full image sum; > 0: skip ions farther than this (A) */
    int    reserved[4];
} smr_grid_build_params;

/* Explicit topology (callers doing their own typing); local atom indices. */
typedef struct {
    int           natoms;
    const double* req;       /* natoms x 4: R_vdW, sqrt(E_vdW), Q, H */
    const int*    neighs;    /* natoms x 4, -1 padded */
    const double* bond_kl;   /* natoms x 4 x 2: (k, l0) of the bond in each neighbour slot */
    int nang;  const int* angs;  const double* angp;   /* nang x 3 (i, j centre, k); nang x 5 (K, c0..c3) */
    int ndih;  const int* dihs;  const double* dihp;   /* ndih x 4; ndih x 3 (V, d, n) */
    int ninv;  const int* invs;  const double* invp;   /* ninv x 4 (centre first); ninv x 4 (K, c0, c1, c2) */
} smr_topology_desc;

int         smr_create(const smr_config* cfg, smr_handle** out);
int         smr_destroy(smr_handle* h);
const char* smr_last_error(const smr_handle* h);
const char* smr_version(void);

int smr_set_nb_params(smr_handle* h, const smr_nb_params* p);

/* Substrate grid: coef is a HOST array of nx*ny*nz*4 values (float for F32, uint16 for F16/BF16)
 * in z-fastest order i = iz + nz*(iy + ny*ix), channels (Pauli, London, Coulomb, H).
 * scale multiplies each stored channel (use 1 for F32). */
int smr_set_grid(smr_handle* h, const void* coef, int dtype, const float scale[4],
                 int nx, int ny, int nz, const double p0[3], const double step[3]);
int smr_get_grid(smr_handle* h, void* coef_out, int* dtype, float scale[4], int dims[3], double p0[3], double step[3]);
/* smr_set_grid from DEVICE memory (the "device pointer" form of the boundary's set_grid): the
 * coefficients are copied device to device on the handle's stream (the caller may free or reuse
 * its buffer on return).  Refused if dev_coef is not device memory. */
int smr_set_grid_device(smr_handle* h, const void* dev_coef, int dtype, const float scale[4],
                        int nx, int ny, int nz, const double p0[3], const double step[3]);
/* 16-bit grids with one scale per z plane and channel (value = stored * plane_scale[4*iz + c]);
 * smr_convert_grid to F16 / BF16 produces such grids (power-of-two scales fitted per plane: the
 * channels grow by orders of magnitude towards the surface, one scale per channel would waste
 * most of fp16's precision on the far planes).  smr_get_grid's scale[] then holds each channel's
 * largest plane scale; smr_get_grid_planes returns the nz x 4 table (the channel scales on every
 * plane for grids without one).  No counterpart in the reference (its grids are float32). */
int smr_set_grid_planes(smr_handle* h, const void* coef, int dtype, const float* plane_scale, int nx, int ny, int nz,
                        const double p0[3], const double step[3]);
int smr_get_grid_planes(smr_handle* h, float* plane_scale);
/* Folded-surface substrate, the reference's SurfaceFolded (crates/libs/surfff/src/lib.rs:126-351)
 * as MolWorld::eval_forces applies it (crates/libs/surfmol/src/mol_world.rs:80-83).  While set it
 * replaces the grid for every system: each atom gets
 *   E = sum_b (cq[b] Q + cp[b] P + cl[b] L) cos(2 pi kx[ix] u) cos(2 pi ky[iy] v) exp(-kz[iz] (z - z0[iz]))
 * over the basis b = ix + nx (iy + ny iz), (u, v) its fractional coordinates in the lattice
 * a = (ax, ay), b = (bx, by), and the atom's P = e L, L = e sqrt(req1), e = exp(-alpha R)
 * (NonBondedFF::make_plqs, req1 = sqrt(E_vdW) as the reference stores it); the force is clamped
 * to fmax per atom (eval_all_clamped; the reference passes 100 eV/A).  One coefficient set for all
 * atoms (the reference evaluates type 0 only).  Arrays are copied; evaluation is FP32.
 * smr_set_surface_folded(h, NULL) returns to the grid.  1 <= nx, ny, nz <= 64. */
typedef struct {
    double ax, bx, ay, by;
    int nx, ny, nz;
    const double *kx, *ky, *kz, *z0;      /* nx, ny, nz, nz */
    const double *cq, *cp, *cl;           /* nx * ny * nz each */
    double alpha;                         /* make_plqs exponent (the reference uses 2.0) */
    double fmax;                          /* per-atom force clamp */
} smr_folded_surface;
int smr_set_surface_folded(smr_handle* h, const smr_folded_surface* f);
/* Build on the device from ions (x, y, z, q) and their Morse (R, sqrt(E)); the slab is periodic
 * in an orthogonal Lx x Ly cell and lies entirely below p0[2]. */
int smr_build_grid(smr_handle* h, int nions, const double* ions, const double* ion_re, double Lx, double Ly,
                   int nx, int ny, int nz, const double p0[3], const double step[3],
                   const smr_grid_build_params* p);
/* Allocation-free grid build.  No counterpart in the reference.  For callers that cannot call
 * cudaMalloc (a host that owns all device memory through its own pool and forbids allocation
 * after start-up): builds the same float32 grid as smr_build_grid, without a handle, into
 * coef_out (a DEVICE buffer of nx*ny*nz*4 floats the caller owns), on the caller's stream
 * (void* cudaStream_t; 0 = default stream), asynchronously: order later uses of coef_out, and
 * other static builds, after that stream's work.  ions / ion_re are host arrays as for
 * smr_build_grid; pinned ones must stay unchanged until the stream's work is done (pageable ones
 * are copied before the call returns).  Scratch is one 8 MiB static device array per GPU (held
 * until exit): three FP64 channels (24 B per voxel) plus the Ewald tables must fit, i.e. at most
 * ~340,000 voxels (less for large cells or many ions), 4 <= nx, ny, nz <= 512.  Larger requests
 * fail with SMR_ERR_CAPACITY and a message in err.  The first call on a device looks up the
 * array's device address (make it before any stream capture); calls whose GPU work overlaps
 * share the array and race.  Returns SMR_OK or a negative SMR_ERR_* code; never allocates
 * device memory. */
typedef struct {
    double alpha_morse;
    int    npbc;
    double ewald_tol;
    int    dtype;              /* must be SMR_GRID_F32 */
    double morse_rcut;
} smr_grid_build_params_static;
int smr_build_grid_static(int nions, const double* ions, const double* ion_re, double Lx, double Ly,
                          int nx, int ny, int nz, const double p0[3], const double step[3],
                          const smr_grid_build_params_static* p, float* coef_out, void* stream,
                          char* err, int errlen);

/* Sharded grid build over several GPUs (each builds an x-slab, an all-gather replicates the raw
 * values, each fits the whole grid; the build of smr_build_grid split at its one exchange point):
 * smr_grid_raw_slab writes the raw, unfitted FP64 values (Pauli, London, Coulomb triples,
 * voxel-major, z-fastest) of the x-planes [x0, x0 + nxs) into raw, a DEVICE buffer of
 * 3 nxs ny nz doubles the caller owns (planes beyond nx are computed and may be discarded, so
 * equal slabs of ceil(nx / ranks) planes concatenate in rank order under an all-gather);
 * smr_grid_from_raw fits and installs the whole grid from the gathered raw values (3 nx ny nz
 * doubles on the device), as smr_build_grid would have built it.  No counterpart in the
 * reference (its grid build is single-device). */
int smr_grid_raw_slab(smr_handle* h, int nions, const double* ions, const double* ion_re, double Lx, double Ly,
                      int nx, int ny, int nz, const double p0[3], const double step[3], const smr_grid_build_params* p,
                      int x0, int nxs, double* raw);
int smr_grid_from_raw(smr_handle* h, const double* raw, int nx, int ny, int nz, const double p0[3], const double step[3], int dtype);
/* Re-encode the current grid to another storage dtype with per-channel scales (max|c| mapping). */
int smr_convert_grid(smr_handle* h, int dtype);
/* Split storage: the current FP32 grid becomes a 16-bit grid (dtype SMR_GRID_F16 or _BF16, per-plane
 * scales as smr_convert_grid makes them) plus an FP32 copy of its planes [0, zsplit + 3).  An atom
 * whose stencil starts below plane zsplit (cell iz - 1 < zsplit) is interpolated from the FP32
 * copy, every other atom from the 16-bit grid.  Near the surface the channels are large and nearly
 * cancel at a relaxed position, so 16-bit mantissas there cost ~4e-3 eV/A of force error (fp16);
 * above it they cost far less than 1e-4 eV/A.  1 <= zsplit <= nz - 3.  smr_get_grid returns the
 * 16-bit grid; any later set, build or conversion of the grid drops the FP32 copy.
 * smr_get_grid_split: zsplit (0: no split) and, when lo_out is non-null, the FP32 planes
 * (nx * ny * (zsplit + 3) * 4 floats, z-fastest, channel scales applied).  No counterpart in the
 * reference (its grids are float32). */
int smr_convert_grid_split(smr_handle* h, int dtype, int zsplit);
int smr_get_grid_split(smr_handle* h, int* zsplit, float* lo_out);

/* Molecule -> bonds by cutoff, UFF typing, terms and parameters (host, native), upload. */
int smr_add_molecule(smr_handle* h, int natoms, const int* Z, const double* pos, const double* charges,
                     double bond_cut, int* topo_id);
/* Batch form of smr_add_molecule: nmol molecules with natoms[i] atoms each, their Z / pos (x 3) /
 * charges (may be null) concatenated; typing and term packing run on all host cores, the device
 * upload happens once.  topo_ids: nmol ids out.  On error nothing is added. */
int smr_add_molecules(smr_handle* h, int nmol, const int* natoms, const int* Z, const double* pos, const double* charges,
                      double bond_cut, int* topo_ids);
int smr_add_topology(smr_handle* h, const smr_topology_desc* d, int* topo_id);
/* Periodic molecules and PBC images: the bond shifts (neighCell / pbc_shifts) of
 * evalBondsAndHNeigh_UFF (opencl/UFF.cl:141-236) and the NB image sums of
 * getNonBond_GridFF_Bspline (UFF.cl:1592-1650), with the lattice per system as lvecs[iS].
 * smr_add_molecule_pbc: bonds by cutoff to every image within one cell along each nonzero lattice
 * vector (lvec = a, b, c, 9 values; a zero vector is a non-periodic axis), each bond slot recording
 * its partner's cell.  Refused (SMR_ERR_ARG) when the cell is too small for index-based terms: an
 * atom bonding to its own image, a pair bonding in two images, or a 3-bond path closing through
 * the images.  npbc (may be null: one image each side along the periodic axes, 0 along the others)
 * is the default of the systems made from it: the NB sum runs over the (2 npbc + 1) images per axis,
 * excluding a bonded pair only in its bond's image and an atom's own images always.
 * smr_set_pbc: per slot lattice (nsys x 9) and images (nsys x 3, each 0..7); images on any
 * topology (an isolated molecule then meets its periodic copies); all-zero npbc on a molecule
 * without periodic bonds turns PBC off for the slot.  Systems with images use the all-pairs NB
 * loop (no neighbour lists).  smr_get_pbc reads a slot's setting back.  smr_topology_cells: the
 * cell code of each neighbour slot (natoms x 4): 4-bit two's-complement offsets x | y << 4 | z << 8. */
int smr_add_molecule_pbc(smr_handle* h, int natoms, const int* Z, const double* pos, const double* charges,
                         double bond_cut, const double lvec[9], const int npbc[3], int* topo_id);
int smr_set_pbc(smr_handle* h, int nsys, const int* slot_ids, const double* lvec, const int* npbc);
int smr_get_pbc(smr_handle* h, int slot, double lvec[9], int npbc[3]);
int smr_topology_cells(smr_handle* h, int topo_id, int* cells);
/* Position constraints: the constr / constrK springs of updateAtomsMMFFf4 (opencl/UFF.cl:974-982).
 * For n listed atoms (indices within the system) a target (x, y, z) and per-axis stiffness
 * (kx, ky, kz in eV/A^2; negative counts as 0): the force (target - position) * k is added after
 * the force limit and drives FIRE (its power, norms and the max|F| convergence test), but is not
 * part of the returned forces or energies, as the reference stores the force before it.  A call
 * replaces the system's constraints; n = 0 removes them.  Constrained systems run in the
 * extended gather form. */
int smr_set_constraints(smr_handle* h, int slot, int n, const int* atoms, const double* target, const double* k);
/* Langevin drive: the TDrives input of updateAtomsMMFFf4 (opencl/UFF.cl:982-991), per system
 * tdrive[4 i ..] = (T [K], gamma, seed increment per FIRE step, seed).  While gamma > 0 the force
 * FIRE uses gains -gamma v + noise sqrt(2 kB T gamma / dt), with v the velocity before the step,
 * dt the system's current FIRE step and noise the kernel's hashed vector of the atom index and
 * seed.  The reference's host changes the seed between launches.  Here the seed of FIRE step s
 * (counted from the last reset) is fma(increment, s, seed): an increment of 0 keeps the kernel's
 * fixed pattern, so chunked and unchunked runs stay identical either way.  Like the constraint
 * springs, the drive acts on FIRE (power, norms, the max|F| test) but not on the returned forces.
 * gamma <= 0 turns the drive off.  Driven systems run in the extended gather form. */
int smr_set_thermal_drive(smr_handle* h, int nsys, const int* slot_ids, const double* tdrive);
/* counts[6] = natoms, nbonds, nang, ndih, ninv, type-rounds (schedule length) */
int smr_topology_counts(smr_handle* h, int topo_id, int counts[6]);
/* Any output pointer may be null.  Layouts as the arrays of smr_topology_desc plus
 * neighBs (natoms x 4 bond index), bonds (nbonds x 2), bparams (nbonds x 2), type ids (natoms). */
int smr_topology_export(smr_handle* h, int topo_id, int* neighs, int* neighBs, int* bonds, double* bparams,
                        int* angs, int* ang_ngs, double* angp, int* dihs, int* dih_ngs, double* dihp,
                        int* invs, int* inv_ngs, double* invp, double* req, int* type_id);
const char* smr_type_name(int type_id);

/* Host-only molecule preparation (no device needed): the same pipeline smr_add_molecule
 * runs, exposed so callers can inspect or cache topologies.  smr_topo_rounds packs the
 * bonded terms into device rounds for a team size: rounds[3] = (angle, dihedral,
 * inversion) round counts; the atom arrays (rounds x team x 4 shorts, -1 = empty) may be
 * null to query the counts first. */
typedef struct smr_topo smr_topo;
int  smr_topo_build(int natoms, const int* Z, const double* pos, const double* charges, double bond_cut, smr_topo** out,
                    char* err, int errlen);
void smr_topo_free(smr_topo* t);
int  smr_topo_counts(const smr_topo* t, int counts[5]);
int  smr_topo_export(const smr_topo* t, int* neighs, int* neighBs, int* bonds, double* bparams,
                     int* angs, int* ang_ngs, double* angp, int* dihs, int* dih_ngs, double* dihp,
                     int* invs, int* inv_ngs, double* invp, double* req, int* type_id);
int  smr_topo_rounds(const smr_topo* t, int team, int rounds[3], short* ang_at, short* dih_at, short* inv_at);
int  smr_add_topo(smr_handle* h, const smr_topo* t, int* topo_id);
/* Topologies whose bonds and angle / dihedral / inversion lists come from a file (the reference's
 * TopologyData JSON, crates/libs/moltopo/src/export.rs:12-74, or UFFTOPO binary,
 * crates/apps/buildff/src/main.rs:10-28): the lists are used as they are, as Uff::from_topology
 * does (crates/libs/molff/src/uff.rs:238-240); atoms are typed from Z and the bond graph, or take
 * the given type ids (smr_type_id maps a UFF type name such as "C_R" to its id, -1 if unknown);
 * parameters follow the same UFF rules as smr_add_molecule.  bonds: nbonds x 2, angs: nang x 3
 * (centre in the middle), dihs: ndih x 4, invs: ninv x 4 (centre first); charges may be null. */
int  smr_topo_build_listed(int natoms, const int* Z, const int* type_ids, const double* charges, int nbonds, const int* bonds,
                           int nang, const int* angs, int ndih, const int* dihs, int ninv, const int* invs, smr_topo** out,
                           char* err, int errlen);
int  smr_add_listed_molecule(smr_handle* h, int natoms, const int* Z, const int* type_ids, const double* charges,
                             int nbonds, const int* bonds, int nang, const int* angs, int ndih, const int* dihs,
                             int ninv, const int* invs, int* topo_id);
int  smr_type_id(const char* name);
/* Pack a host topology's term records for a team size (0: the default for its size) without a
 * handle; thread-safe, so request topologies can be packed while the GPU works.  smr_add_topo then
 * uploads them as they are when the handle's team for that size matches.  No counterpart in the
 * reference. */
int  smr_topo_prepare(smr_topo* t, int team);
/* Release a topology no active slot uses; its id stays reserved.  The device records of removed
 * topologies are dropped by an automatic compaction once they outnumber the live ones (long-running
 * servers admit and retire molecules without growing the arenas).  No counterpart in the reference. */
int  smr_remove_topology(smr_handle* h, int topo_id);
/* Batch forms (one device upload / one compaction check per batch): attach n host topologies
 * (ids out), release n topologies.  No counterpart in the reference. */
int  smr_add_topos(smr_handle* h, int n, const smr_topo* const* topos, int* topo_ids);
int  smr_remove_topologies(smr_handle* h, int n, const int* topo_ids);

/* Systems: one slot per system; positions are float32 x,y,z concatenated over the systems. */
int smr_add_systems(smr_handle* h, int nsys, const int* topo_ids, const float* pos, int* slot_ids);
int smr_remove_systems(smr_handle* h, int nsys, const int* slot_ids);
int smr_set_positions(smr_handle* h, int nsys, const int* slot_ids, const float* pos);
int smr_active_slots(smr_handle* h, int* nslots, int* slot_ids /* may be null */);

/* One force evaluation of the given slots at their current positions.
 * forces: sum(natoms) x 4 (fx, fy, fz, E_atom) with E_atom in the reference's per-atom
 * convention (opencl/UFF.cl fapos.w: bond energy and NB pair energy on both atoms);
 * energy: nsys x SMR_E_NCOMP doubles (physical totals).  Either output may be null. */
int smr_eval_forces(smr_handle* h, int nsys, const int* slot_ids, float* forces, double* energy);

/* Relax every active, not yet finished slot for at most max_steps further FIRE steps.
 * A system's FIRE state (velocities, dt, alpha, n_pos, steps done) persists across calls,
 * so repeated calls continue the same trajectory.  step_budget caps the total steps of
 * each system (0 = no cap beyond max_steps).  nfinished (may be null) receives the
 * number of slots whose status is no longer SMR_ST_RUNNING. */
int smr_run_fire(smr_handle* h, int max_steps, int step_budget, const smr_fire_params* p, int mode, int* nfinished);
/* Restart FIRE (zero velocity, dt0, alpha0, n_pos 0, steps 0, status running) on slots. */
int smr_reset_fire(smr_handle* h, int nsys, const int* slot_ids);

/* Read back results; any output may be null.  pos: sum(natoms) x 3 float; forces: x 4;
 * energy: nsys x SMR_E_NCOMP (only SMR_E_TOTAL is maintained by relaxation: the energy at
 * the last force evaluation); steps: FIRE steps done; status: SMR_ST_*. */
int smr_download(smr_handle* h, int nsys, const int* slot_ids, float* pos, float* forces, double* energy,
                 int* steps, int* status);
/* Positions at full precision: the kernels carry each coordinate as a float plus the float
 * rounding error of its FIRE moves; this returns their sum as sum(natoms) x 3 doubles.  No
 * counterpart in the reference (its state is float only). */
int smr_download_pos64(smr_handle* h, int nsys, const int* slot_ids, double* pos);

/* Device time (ms, CUDA events on the handle's stream) of the last smr_run_fire /
 * smr_eval_forces call, and the number of kernel launches it made. */
int smr_last_timing(smr_handle* h, double* ms, long long* launches);

/* Force-evaluation forms of the kernels (results agree to rounding; each is deterministic):
 *  SMR_FORM_ROUNDS  bonded terms in host-packed conflict-free rounds added straight into the
 *                   shared-memory force array (one team size per topology): best throughput
 *                   when many small systems share the GPU
 *  SMR_FORM_GATHER  all bonded terms at once into a piece buffer, then a per-atom gather
 *                   (opencl/UFF.cl:801-880): most parallel per system, best latency
 *  SMR_FORM_OWNER   every term evaluated by the atom that owns it (angle apex, inversion centre,
 *                   both central atoms of a dihedral) with its neighbours' pieces kept in
 *                   registers and gathered over the bond back-slots: no team syncs between terms */
#define SMR_FORM_ROUNDS 0
#define SMR_FORM_GATHER 1
#define SMR_FORM_OWNER 2

/* Schedule of smr_run_fire (batched and plain alike): nstages (1..16) stages; stage k covers
 * FIRE steps [starts[k], starts[k+1]) of each system (the last one is open), starts[0] == 0 and
 * strictly increasing, and runs forms[k] with teams[k] threads per system (0: the form's default
 * for the system's size; else 32, 64, 128, 256 or 512).  A system whose topology or shared memory
 * does not allow the requested form runs the rounds form instead.  Which form a system runs
 * depends only on the system and its own step count, so results do not depend on what else runs.
 * In batched mode each stage is a separate launch over the systems still running (which also
 * spreads them evenly over the SMs again).  eval_form is the form of smr_eval_forces (team by
 * size).  Default: one stage, SMR_FORM_ROUNDS.  No counterpart in the reference (one OpenCL
 * kernel form). */
int smr_set_stages(smr_handle* h, int nstages, const int* starts, const int* forms, const int* teams, int eval_form);
/* *nstages: capacity of the arrays in, stage count out (arrays may be null to query the count). */
int smr_get_stages(smr_handle* h, int* nstages, int* starts, int* forms, int* teams);
/* Two-stage shortcut: rounds form until switch_step FIRE steps, then the gather form with
 * latency_team threads (0: by size); switch_step <= 0 keeps the rounds form throughout.
 * smr_eval_forces then runs eval_form with latency_team threads. */
int smr_set_schedule(smr_handle* h, int switch_step, int latency_team, int eval_form);
int smr_get_schedule(smr_handle* h, int* switch_step, int* latency_team, int* eval_form);

/* Team configuration of the persistent kernel: threads per system team for systems of
 * up to n atoms (0 = library default / autotuned). */
int smr_set_team_size(smr_handle* h, int max_atoms, int threads);

/* Tuning knobs (no counterpart in the reference; set by the autotuner or by hand):
 *   SMR_TUNE_NB_LANES  lanes per atom splitting the intramolecular NB partner loop
 *                      (1, 2, 4, 8, 16, 32; 0 = chosen from the system size and team) */
#define SMR_TUNE_NB_LANES 1
/*   SMR_TUNE_NBLIST_MIN     systems of at least this many atoms use NB neighbour lists during FIRE
 *                           when a cutoff is set (default 128; 0 = never): partners within
 *                           rc + skin, rebuilt when an atom has moved more than skin / 2
 *   SMR_TUNE_NBLIST_SKIN_MA skin in milli-Angstrom (default 1000)
 *   SMR_TUNE_NBLIST_CAP     partners per atom a list row holds (default 256, a multiple of 4; an
 *                           atom with more uses the all-pairs loop) */
#define SMR_TUNE_NBLIST_MIN 2
#define SMR_TUNE_NBLIST_SKIN_MA 3
#define SMR_TUNE_NBLIST_CAP 4
/*   SMR_TUNE_WATCHDOG_MS    the longest a call waits for its device work (default 3600000).  A call
 *                           that gives up returns SMR_ERR_TIMEOUT with the work still running; the
 *                           next call on the handle first waits for it (bounded by the same limit)
 *                           and refreshes its copy of the per-system state, so no result is lost */
#define SMR_TUNE_WATCHDOG_MS 5
/*   SMR_TUNE_GRID_BRICKS    grid layout the relax kernel reads: -1 (default) the brick copy for
 *                           grids larger than 128 MiB, 0 the z-fastest grid itself, 1 the brick
 *                           copy always.  The copy holds each 128-byte piece of the interpolation
 *                           stencil in one aligned line (8x the grid's memory); results are the
 *                           same bit for bit either way */
#define SMR_TUNE_GRID_BRICKS 6
/*   SMR_TUNE_GRID_BRICKS_ACTIVE (smr_get_tuning only) 1 if the last launch read the brick copy */
#define SMR_TUNE_GRID_BRICKS_ACTIVE 7
/*   SMR_TUNE_GRID_PREFETCH  1: with the brick copy, each force evaluation starts by requesting its
 *                           atoms' stencil lines into L2; 0 (default): no prefetch (on the ragged
 *                           workload it measured 12 % slower) */
#define SMR_TUNE_GRID_PREFETCH 8
/*   SMR_TUNE_SMEM_CARVEOUT  preferred share of the SM's L1 given to shared memory for block teams,
 *                           in percent (-1, default: the driver's choice)
 *   SMR_TUNE_OCC_TIERS      1: launch segments of one form and team are split by the blocks per
 *                           SM each system's shared memory allows, so small systems keep their
 *                           occupancy; 0 (default): one segment per form and team (the split
 *                           measured slower on the ragged workload) */
#define SMR_TUNE_SMEM_CARVEOUT 9
#define SMR_TUNE_OCC_TIERS 10
int smr_set_tuning(smr_handle* h, int key, int value);
int smr_get_tuning(smr_handle* h, int key, int* value);

/* CUDA-graph replay of smr_run_fire's batched launch sequence (work-list copies, counter resets,
 * one persistent launch per stage segment, the side-stream fork / join).  With it on, a call whose
 * launch plan (systems, stages, segments, every kernel argument) equals the previous captured one
 * replays that graph in a single launch; a new plan is captured, instantiated and launched.  Off
 * by default.  smr_graph_stats: replays so far.  No counterpart in the reference. */
int smr_set_graph(smr_handle* h, int on);
int smr_graph_stats(smr_handle* h, long long* replays);

#ifdef __cplusplus
}
#endif
#endif /* SURFMOL_RELAX_H */
