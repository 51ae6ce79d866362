/* surfmol_raff.h — C ABI of the multi-replica rigid-atom (RAFF / RRsp3) relaxation.
 *
 * Drop-in for the reference's RRsp3Multi harness (crates/libs/oclff/src/rrsp3.rs:699-1088) and
 * its kernels compute_collision_multi, compute_ports_current_multi and apply_corrections_multi
 * (opencl/RRsp3.cl:1774-2048): many replicas of one molecule whose heavy atoms ("nodes") are
 * rigid bodies (position + orientation quaternion) joined to their neighbours through ports
 * (XPBD position constraints, massfull "Current" variant), relaxed by Jacobi position updates
 * with optional heavy-ball momentum and sphere collisions.  The host-side preparation of
 * crates/libs/oclff/src/pack.rs (nodes-first ordering, neighbours, 1st / 2nd exclusions,
 * back-slots, ports, masses) is exported too.
 *
 * Arrays use the reference's layouts: per replica and atom float4 / (x, y, z) rows, replica-major;
 * topology arrays are shared by all replicas; indices are local to a replica.  Every call returns
 * SMR_RAFF_OK (0) or a negative code with a message in smr_raff_last_error.  All calls synchronise
 * before returning; host arrays stay owned by the caller.
 */
#ifndef SURFMOL_RAFF_H
#define SURFMOL_RAFF_H

#ifdef __cplusplus
extern "C" {
#endif

#define SMR_RAFF_OK 0
#define SMR_RAFF_ERR_ARG -1
#define SMR_RAFF_ERR_CUDA -2
#define SMR_RAFF_ERR_STATE -3

typedef struct smr_raff smr_raff;

typedef struct {
    int device;
    int natoms;          /* atoms per replica (padding atoms included: inverse mass 0) */
    int nsys;            /* replicas */
    int reserved[5];
} smr_raff_config;

/* StepConfig (rrsp3.rs:54-73), the fields the multi-replica step reads. */
typedef struct {
    float dt;            /* XPBD time step (alpha = 1 / (K dt^2)); reference default 0.1 */
    float k_coll;        /* accepted for the reference's signature; its collision kernel ignores it */
    float relaxation;    /* Jacobi relaxation factor (0.5) */
    float momentum_beta; /* heavy-ball momentum on positions and quaternions (0: off) */
    float rot_mass_scale;/* scales the inverse moment of inertia 1 / (0.4 m) (1.0) */
    int reserved[3];
} smr_raff_step_config;

/* RRsp3Multi::new (rrsp3.rs:740-837): state buffers for nsys replicas of natoms atoms. */
int smr_raff_create(const smr_raff_config* cfg, smr_raff** out);
int smr_raff_destroy(smr_raff* r);
const char* smr_raff_last_error(const smr_raff* r);

/* upload_radius (rrsp3.rs:848-858): sphere radii (>= 0); collisions run when any is > 0. */
int smr_raff_upload_radius(smr_raff* r, const float* radius);
/* upload_neighs_and_exclusions (rrsp3.rs:860-867): natoms x 4 each, -1 padded. */
int smr_raff_upload_neighs_and_exclusions(smr_raff* r, const int* neighs, const int* excl1, const int* excl2);
/* upload_fixmask (rrsp3.rs:869-872): bits 1 / 2 / 4 freeze x / y / z (and the rotation of a
 * node), bit 8 projects z onto the plane z = 0. */
int smr_raff_upload_fixmask(smr_raff* r, const int* fixmask);
/* upload_cluster_ports_multi (rrsp3.rs:884-918): port_local natoms x 4 float4 (arm in the
 * node's body frame, w unused), k natoms x 4 stiffness; the first nnode atoms are the nodes. */
int smr_raff_upload_cluster_ports(smr_raff* r, const float* port_local, const float* k, int nnode);
/* upload_bk_slots_multi (rrsp3.rs:920-923): natoms x 4 port indices (node * 4 + slot) whose
 * recoil an atom gathers, -1 padded. */
int smr_raff_upload_bk_slots(smr_raff* r, const int* bk_slots);
/* upload_state_multi (rrsp3.rs:926-955): positions nsys x natoms x 3, inverse masses natoms
 * (shared; an atom with inverse mass <= 1e-12 is padding and gets NaN coordinates, as the
 * reference stores it), quaternions nsys x natoms x 4 (x, y, z, w) or null for identity.
 * Momenta are reset to zero. */
int smr_raff_upload_state(smr_raff* r, const float* pos3, const float* inv_mass, const float* quat);

/* step_cluster_multi (rrsp3.rs:986-1005) run nsteps times: per step the collision, port and
 * correction passes of every replica.  All nsteps run inside one launch, each replica's state in
 * on-chip shared memory; results are those of nsteps calls of the reference's step. */
int smr_raff_step(smr_raff* r, int nsteps, const smr_raff_step_config* cfg);
/* device time of the last smr_raff_step (CUDA events on the handle's stream), ms */
int smr_raff_last_ms(const smr_raff* r, float* ms);

/* download_pos_multi / download_pos_replica / download_quat_replica /
 * download_dpos_coll_replica / download_dpos_node_replica (rrsp3.rs:958-1082).
 * isys = -1: all replicas (nsys x ...), else one replica.  The correction downloads return the
 * last step's values (dpos_node: nnode rows). */
int smr_raff_download_pos(smr_raff* r, int isys, float* pos3);
int smr_raff_download_quat(smr_raff* r, int isys, float* quat4);
int smr_raff_download_dpos_coll(smr_raff* r, int isys, float* d3);
int smr_raff_download_dpos_node(smr_raff* r, int isys, float* d3);

/* Host preparation (crates/libs/oclff/src/pack.rs), no GPU needed.
 * smr_raff_node_order (pack_molecules, pack.rs:54-116, one molecule): nodes (bond degree > 1)
 *   first, then caps, each in input order: perm[k] = input index of packed atom k; returns nnode.
 * smr_raff_build_neighs (build_neighs_from_bonds, pack.rs:155-172): neighs natoms x 4.
 * smr_raff_exclusions (make_exclusions_1st_2nd, pack.rs:176-212).
 * smr_raff_bk_slots (make_bk_slots_clustered, pack.rs:218-246, one group of natoms atoms).
 * smr_raff_ports (make_ports_from_neighs, pack.rs:293-313): port_local natoms x 4 x 4, k natoms x 4.
 * smr_raff_element_mass (element_mass, pack.rs:132-142): standard atomic weight of element Z
 *   (12.0 for elements outside the reference's table). */
int smr_raff_node_order(int natoms, int nbonds, const int* bonds, int* perm);
int smr_raff_build_neighs(int natoms, int nbonds, const int* bonds, int* neighs);
int smr_raff_exclusions(int natoms, const int* neighs, int* excl1, int* excl2);
int smr_raff_bk_slots(int natoms, int nnode, const int* neighs, int* bk_slots);
int smr_raff_ports(int natoms, const float* pos3, const int* neighs, float k_stiff, float* port_local, float* k);
float smr_raff_element_mass(int Z);

#ifdef __cplusplus
}
#endif
#endif
