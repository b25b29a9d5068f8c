/*
 * nbc_oracle.h -- FP64 CPU restatement of the reference's clump step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * B200 engine: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline may load it.  The engine never calls it.
 *
 * It restates, function by function, the single-GPU FP64 solver of
 * qubajin/nbody-clump (DEMClumpMain::RunSimulationClump,
 * src/dem_simulation_clump.cu:110-225) in plain C: the same pair list layout
 * (pitched rows of BranchLmtLen, front entries j>i, back entries j<i), the
 * same history ping-pong including its stale-entry behaviour, the same
 * summation orders where the reference has a sequential one, and the same
 * expression grouping in every contact law.  Parity is pinned against the
 * reference itself: the .ref.npz files under tests/golden hold the outputs of the unmodified
 * reference build (oracle/Makefile.ref) run on a B200.
 *
 * Additions that the reference has only on its sphere path are restated with
 * clump kinematics: the closed cylinder wall (src/dem_force_cylind_wall.cu:
 * 3-237) and the hierarchical grid (src/dem_hgrid_contlist.cu:57-248), the
 * latter race-free (the reference's cross-level appends race with its
 * same-level ones).  With nbo_desc.sphere_mode it restates the sphere-only
 * drivers themselves (class DEMmain: src/dem_integrate.cu,
 * src/dem_integrate_withglue.cu, src/dem_force_particle.cu:3-182,
 * src/dem_force_cube_wall.cu, src/dem_force_penetrator.cu:8-187 and the
 * drivers' history exchange, src/dem_simulation_{cylind,cube,split}.cu),
 * pinned to the reference's own runs of those drivers.
 */
#ifndef NBC_ORACLE_H
#define NBC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    /* world.par (src/dem_parameters.h:7-79) */
    int N, K, BL;
    int start_step, end_step, output_interval;
    double dt, E, nu, mu, e_rest, beta, cohesion, gravity, thresh;
    double world_origin[3], world_size[3], box_lo[3], box_hi[3];
    int is_wall, is_intruder;
    /* subspheres (ph columns) */
    const int* clump_id;
    const double* pos;     /* [N][3] */
    const double* local;   /* [N][3] */
    const double* mass;    /* [N] */
    const double* radius;  /* [N] */
    /* clumps (ch columns) */
    const double* cpos;    /* [K][3] */
    const double* cvel;    /* [K][3] */
    const double* cquat;   /* [K][4] x,y,z,w */
    const double* cangvel; /* [K][3] */
    const double* cprop;   /* [K][4] Ixx,Iyy,Izz,M */
    /* cube wall (Rocks/CubeWall.bt) */
    int has_cube;
    double cube_half[3], cube_centre[3], cube_vel[3], cube_quat[4], cube_angvel[3];
    /* closed cylinder wall (Rocks/CylindWall.bt), clump kinematics */
    int has_cyl;
    double cyl_radius, cyl_half_height, cyl_axis[3], cyl_centre[3], cyl_vel[3], cyl_angvel[3];
    /* intruder (Rocks/Penetrator.bt) */
    int intr_shape;   /* 0 cylinder, 1 sphere */
    int intr_motion;  /* 0 constant velocity, 1 gravity */
    int intr_wait;    /* gravity_after_contact */
    double intr_radius, intr_half_height, intr_axis[3], intr_prop[4];
    double intr_pos[3], intr_vel[3], intr_quat[4], intr_angvel[3];
    /* hierarchical grid: levels > 1 enables it; level[i] per subsphere */
    int levels;
    const int* level;          /* [N] 0 = coarsest */
    const double* level_cell;  /* [levels] cell size per level */
    /* the reference's sphere-only drivers (class DEMmain): bits 1 sphere
     * kinematics (first half-kick and attitude without the intruder, the
     * sphere laws' lever arms, penetrator cohesion), 2 the sphere cube wall
     * (no history, no rolling or twisting moment), 4 pair histories reset at
     * every rebuild; body_kind (or NULL) the split driver's Type per sphere.
     * One-sphere clumps with LocalPos = 0, sphere k = clump k. */
    int sphere_mode;
    const int* body_kind;
} nbo_desc;

typedef struct nbo_scene nbo_scene;

nbo_scene* nbo_create(const nbo_desc* d);
void nbo_destroy(nbo_scene* s);
void nbo_set_threads(int n);
/* Advance nsteps steps; returns 0, or a nonzero error (1 list overflow,
 * 2 non-finite wall input/output). */
int nbo_step(nbo_scene* s, int nsteps);

int nbo_num_pairs(const nbo_scene* s);
int nbo_step_count(const nbo_scene* s);
int nbo_rebuild_count(const nbo_scene* s);
/* subsphere state in current (cell-sorted) order */
void nbo_get_sub(const nbo_scene* s, int* part_fix, int* clump_id, double* pos, double* radius);
/* clump state [K] */
void nbo_get_clumps(const nbo_scene* s, double* pos, double* vel, double* quat, double* angvel,
                    double* force, double* torque);
/* per-subsphere pair force/torque sums (after the last step) and totals */
void nbo_get_sub_forces(const nbo_scene* s, double* fc, double* tc, double* fw, double* tw,
                        double* fi, double* ti);
/* pair list: Lpa/Lpb [P], Anei rows [N][BL], Ng/Ni [N] */
void nbo_get_pairs(const nbo_scene* s, int* lpa, int* lpb);
void nbo_get_rows(const nbo_scene* s, int* anei, int* ng, int* ni);
/* per-slot caches of the last step: force on i (CacheFc), normal force on i
 * (CacheFcn), contact point, and the histories written (Dv, Dt, Dr) [P][3] */
void nbo_get_pair_caches(const nbo_scene* s, double* cfc, double* cfcn, double* cpt,
                         double* dv, double* dt, double* dr);
/* force-chain rows of the reference's OutCnt output: Fcn and Cpt [N][BL][3] */
void nbo_get_chain(const nbo_scene* s, double* fcn_rows, double* cpt_rows);
/* intruder: pos, vel, last total force on particles, last total torque,
 * last recorded reaction, contact state */
void nbo_get_intruder(const nbo_scene* s, double* pos, double* vel, double* totf, double* tott,
                      double* reaction, int* state);
/* intruder per-subsphere diagnostics Fcn, Fct, Tcn, Tct [N][3] */
void nbo_get_intruder_diag(const nbo_scene* s, double* fcn, double* fct, double* tcn, double* tct);

#ifdef __cplusplus
}
#endif
#endif
