/*
 * nbc.h -- C ABI of the B200 DEM engine (libnbc.so).
 *
 * Drop-in boundary for the NBodyClump hot path: the reference exposes one
 * entry point, DEMClumpMain::RunSimulationClump() (src/dem_clump.h:36-96,
 * called from src/main.cpp:7-8), which reads world.par, the ph/ch .bt initial
 * conditions and Rocks/ files from the working directory, advances the clump
 * step loop (src/dem_simulation_clump.cu:110-259) and writes the binary
 * snapshot files.  nbc_open/nbc_run replace that call; the scene-level calls
 * below replace the reference's internal class interfaces for callers that
 * hold their scenes in memory (tests, batching, serving).
 *
 * Conventions: plain pointers and sizes only; every call returns nbc_status
 * (the reference calls exit() on every error, src/include/helper_cuda.h:
 * 985-1010); arrays are host memory unless named *_dev; vectors are
 * interleaved xyz (quaternions xyzw) in double precision.  The engine owns
 * all device memory.  Calls on one engine are not reentrant; separate
 * engines are independent.
 */
#ifndef NBC_H
#define NBC_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int nbc_status;
#define NBC_OK 0
#define NBC_ERR_ARG (-1)          /* invalid argument or inconsistent scene */
#define NBC_ERR_CUDA (-2)         /* a CUDA call failed (message in nbc_last_error) */
#define NBC_ERR_IO (-3)           /* missing or malformed input file (src/dem_subsphere_io.cu:40-141) */
#define NBC_ERR_NONFINITE (-4)    /* non-finite subsphere force (src/dem_force_cube_wall_clump.cu:295-331) */
#define NBC_ERR_NO_DEVICE (-5)    /* no CUDA device: the engine has no CPU fallback */
#define NBC_ERR_MEMORY (-6)       /* device allocation failed or over the engine's budget */
#define NBC_ERR_STATE (-7)        /* call not valid in the engine's state */

#define NBC_PREC_F64 0            /* every quantity in FP64, like the reference */
#define NBC_PREC_MIXED 1          /* contact law in FP32 (overlap and positions FP64) */

#define NBC_WALL_NONE 0
#define NBC_WALL_CUBE 1           /* Rocks/CubeWall.bt, src/dem_cube_wall_io.cu:21-53 */
#define NBC_WALL_CYLINDER 2       /* Rocks/CylindWall.bt, src/dem_cylind_wall_io.cu:20-55 */

#define NBC_INTR_NONE (-1)
#define NBC_INTR_CYLINDER 0       /* PenetratorShape, src/dem_parameters.h:93 */
#define NBC_INTR_SPHERE 1

#define NBC_MOTION_CONSTANT_VELOCITY 0   /* src/dem_penetrator_io.cu:100-115 */
#define NBC_MOTION_GRAVITY 1
#define NBC_MOTION_GRAVITY_AFTER_CONTACT 2

/* nbc_scene_desc.sphere_mode: the behaviour of the reference's sphere-only
 * drivers (class DEMmain, src/dem.h:31-99) where it differs from the clump
 * path.  0 = the clump path.  The bits need one-sphere clumps whose member
 * sits at the clump centre (LocalPos = 0). */
#define NBC_SPHERE_KINEMATICS 1   /* first half-kick and attitude without the
                                     intruder's force and torque (src/dem_integrate.cu:
                                     20-21,72); cohesion in the penetrator law
                                     (src/dem_force_penetrator.cu:119-123) */
#define NBC_SPHERE_CUBE_WALL 2    /* the sphere cube wall: tangential force
                                     without history, no rolling or twisting
                                     moment (src/dem_force_cube_wall.cu:70-141) */
#define NBC_SPHERE_RESET_HISTORY 4 /* pair spring histories restart from zero at
                                     every rebuild: the driver exchanges the history
                                     pointers once more after the list build has
                                     carried them and cleared the other buffer
                                     (src/dem_simulation_cylind.cu:141 after
                                     src/dem_grid.cu:687-749) */

/* DEMmain drivers for nbc_open_sphere */
#define NBC_DRIVER_CYLINDER 0     /* DEMmain::RunSimulation, src/dem_simulation_cylind.cu:3-211 */
#define NBC_DRIVER_CUBE 1         /* DEMmain::RunSimulation2, src/dem_simulation_cube.cu:3-226 */
#define NBC_DRIVER_SPLIT 2        /* DEMmain::RunSimulation_Split, src/dem_simulation_split.cu:3-211 */
#define NBC_DRIVER_HGRID 3        /* DEMmain::RunSimulation_HGrid, src/dem_simulation_hgrid.cu:3-201 */

/* One scene: the contents of world.par, ph/ch .bt and Rocks/ files.
 * Replaces Parameters/GlobalFlg (src/dem_parameters.h:7-79) plus the arrays
 * loaded by DEMSubSphereIo::LoadPhase (src/dem_subsphere_io.cu:151-193) and
 * DEMClumpSphereIo::LoadPhase (src/dem_clumpsphere_io.cu:24-62). */
typedef struct {
    int n_sub, n_clump, branch_len;          /* NumberBody, ClumpNum, BranchLmtLen */
    int start_step, end_step, output_interval;
    double dt, ymod, prat, frcoe, normres, beta, cohesion, gravity, thresh;
    double world_origin[3], world_size[3], box_lo[3], box_hi[3];
    int is_wall_force;                       /* isWallForce */
    /* subspheres (ph columns 3-11) */
    const int* clump_id;                     /* [n_sub], 0 .. n_clump-1 */
    const double* pos;                       /* [n_sub][3] */
    const double* local;                     /* [n_sub][3] body-frame offset */
    const double* mass;                      /* [n_sub] */
    const double* radius;                    /* [n_sub] */
    /* clumps (ch columns 2-18) */
    const double* clump_pos;                 /* [n_clump][3] */
    const double* clump_vel;                 /* [n_clump][3] */
    const double* clump_quat;                /* [n_clump][4] x y z w */
    const double* clump_angvel;              /* [n_clump][3] */
    const double* clump_prop;                /* [n_clump][4] Ixx Iyy Izz M */
    /* wall */
    int wall;                                /* NBC_WALL_* */
    double cube_half[3], cube_centre[3], cube_vel[3], cube_angvel[3];
    double cyl_radius, cyl_half_height, cyl_axis[3], cyl_centre[3], cyl_vel[3], cyl_angvel[3];
    /* intruder (penetrator) */
    int intruder;                            /* NBC_INTR_* */
    int intr_motion;                         /* NBC_MOTION_* */
    double intr_radius, intr_half_height, intr_axis[3], intr_prop[4];
    double intr_pos[3], intr_vel[3], intr_angvel[3];
    /* hierarchical grid: levels > 1 enables it */
    int levels;
    const int* level;                        /* [n_sub], 0 = coarsest */
    const double* level_cell;                /* [levels] cell size per level */
    int sphere_mode;                         /* NBC_SPHERE_* bits, 0 = the clump path */
    /* split driver (NBC_DRIVER_SPLIT) body kinds per clump, or NULL: 0 free,
     * 1 moved at the prescribed velocity (-0.2 y, -0.2 x, 0), 2 fixed
     * (src/dem_integrate_withglue.cu:3-60) */
    const int* body_kind;
} nbc_scene_desc;

typedef struct {
    int precision;      /* NBC_PREC_* */
    int lanes;          /* reserved, ignored: each subsphere's contact sum runs in the clump pass */
    int use_graph;      /* 1: one CUDA graph per step with a conditional rebuild node */
    int device;         /* CUDA device ordinal */
    double pair_slack;  /* pair capacity = slack * pairs of the first list; 0 = 1.6 and at least
                           the reference's own n_sub * BranchLmtLen/2 as far as 30% of free memory allows */
    int search_lanes;   /* lanes per subsphere in the neighbour search: 8, 16 or 32 (0 = 8) */
    int clump_batch;    /* members each lane of the clump pass loads at a time: 1, 2 or 4 (0 = 1) */
    int pair_blocks;    /* blocks per SM of the pair kernel's grid: 2 .. 16 (0 = 12) */
} nbc_options;

typedef struct nbc_engine nbc_engine;

/* last error message of the calling thread */
const char* nbc_last_error(void);
void nbc_default_options(nbc_options* opt);

/* --- drop-in entry point: DEMClumpMain::RunSimulationClump ------------- */
/* Read world.par, IniConFile, ch.00000000.bt and Rocks/ from workdir
 * (src/dem_simulation_clump.cu:3-72). */
nbc_status nbc_open(const char* workdir, const nbc_options* opt, nbc_engine** out);
/* Run StartStep..EndStep with the reference's outputs into workdir
 * (OutPart, OutClump, OutForce, OutCnt; src/dem_simulation_clump.cu:74-259). */
nbc_status nbc_run(nbc_engine* e);

/* --- drop-in entry points: the sphere-only drivers of class DEMmain ------
 * (src/dem.h:31-99; RunSimulation, RunSimulation2, RunSimulation_Split and
 * RunSimulation_HGrid, selected by NBC_DRIVER_*).  Reads world.par, the
 * 21-column ph file named by IniConFile (src/dem_io.cu:155-202), the
 * driver's wall (Rocks/CylindWall.bt, or Rocks/CubeWall.bt for
 * NBC_DRIVER_CUBE), Rocks/Penetrator.bt and, for NBC_DRIVER_HGRID, grid.bt
 * (src/dem_io.cu:204-248).  Each sphere becomes a one-sphere clump and the
 * scene runs with the driver's NBC_SPHERE_* behaviour; nbc_run then writes
 * the drivers' outputs (OutPart/ph.N.bin in the sphere layout, with an
 * intruder OutPart/intruder.N.bin and OutForce/fc.N.bin, and OutCnt for the
 * cube driver with an intruder). */
nbc_status nbc_open_sphere(const char* workdir, int driver, const nbc_options* opt, nbc_engine** out);

/* --- scene-level calls ---------------------------------------------------- */
nbc_status nbc_create(const nbc_scene_desc* const* scenes, int n_scenes, const nbc_options* opt,
                      nbc_engine** out);
nbc_status nbc_destroy(nbc_engine* e);
/* advance every scene by nsteps steps (the loop body of
 * src/dem_simulation_clump.cu:110-225) */
nbc_status nbc_step(nbc_engine* e, int nsteps);
/* like nbc_step, and the last step also records per-contact export data
 * (normal force and contact point per pair, force split per subsphere) */
nbc_status nbc_step_export(nbc_engine* e, int nsteps);
/* wait for the device; applies the pending second half-kick so the state
 * read back is the state after the last completed step */
nbc_status nbc_sync(nbc_engine* e);

nbc_status nbc_num_scenes(const nbc_engine* e, int* n);
/* steps, rebuilds, pairs in the current list, error bits */
nbc_status nbc_scene_stats(nbc_engine* e, int scene, int* steps, int* rebuilds, int* npairs, int* err);
/* over all scenes: the near pairs of the current list (those that can touch
 * before the next rebuild; the contact pass visits only them) and how many
 * of them touched at the last contact pass; no reference counterpart */
nbc_status nbc_contact_counts(nbc_engine* e, long long* near_pairs, long long* touching_pairs);
/* subspheres in the engine's current (cell-sorted) order; part_fix is the
 * original ph row (ParticleID of src/dem_clump.cu:170-171) */
nbc_status nbc_get_subspheres(nbc_engine* e, int scene, int* part_fix, int* clump_id, double* pos,
                              double* radius);
/* body-frame offset and mass of every subsphere, current order */
nbc_status nbc_get_subsphere_body(nbc_engine* e, int scene, double* local, double* mass);
nbc_status nbc_get_clumps(nbc_engine* e, int scene, double* pos, double* vel, double* quat,
                          double* angvel, double* force, double* torque);
/* force and torque on every subsphere from the last step (pairs + walls +
 * intruder, the reference's totF/totT, src/dem_clump.cu:89-101), current order */
nbc_status nbc_get_sub_forces(nbc_engine* e, int scene, double* force, double* torque);
/* after nbc_step_export: pair / wall / intruder parts [6][n_sub][3] */
nbc_status nbc_get_force_parts(nbc_engine* e, int scene, double* parts);
/* the half pair list in the reference's order (Lpa/Lpb, src/dem_grid.cu:
 * 561-601), subsphere indices in the current order; *npairs in/out */
nbc_status nbc_get_pairs(nbc_engine* e, int scene, int* npairs, int* lpa, int* lpb);
/* rows in the reference's pitched layout (Anei: front entries from slot 0,
 * back entries from slot bl-1 downwards, -1 elsewhere), [n_sub][bl] */
nbc_status nbc_get_rows(nbc_engine* e, int scene, int bl, int* anei, int* ng, int* ni);
/* after nbc_step_export: force-chain rows of the reference's OutCnt output
 * (CalFcnChain_cuk, src/dem_force_particle.cu:238-268): normal force and
 * contact point per row slot, [n_sub][bl][3] each */
nbc_status nbc_get_chain(nbc_engine* e, int scene, int bl, double* fcn, double* cpt);
/* after nbc_step_export: the normal force on the owner of every pair of the
 * half list, in list order (the reference's CacheFcn, src/dem_force_clump.cu:
 * 114-116; zero where the pair does not touch), [npairs][3]; *npairs in/out
 * as for nbc_get_pairs */
nbc_status nbc_get_pair_forces(nbc_engine* e, int scene, int* npairs, double* fcn);
/* intruder position, velocity, last reaction force/torque, contact state */
nbc_status nbc_get_intruder(nbc_engine* e, int scene, double* pos, double* vel, double* reaction,
                            double* torque, int* state);
/* after nbc_step_export: per-subsphere intruder diagnostics Fcn, Fct, Tcn,
 * Tct [4][n_sub][3] (src/dem_force_penetrator_clump.cu:127-177) */
nbc_status nbc_get_intruder_diag(nbc_engine* e, int scene, double* diag);
/* reaction force/torque recorded at each of the last `count` completed
 * steps (CacheFc/CacheTc of src/dem_integrate_penetrator.cu:108-109), [count][6] */
nbc_status nbc_get_intruder_history(nbc_engine* e, int scene, int count, double* out);
/* CUDA-event timing on the engine's streams (also inside graph launches, as
 * event nodes): enable = 1 times the contact kernel, 2 also every phase of
 * the step (nbc_timing_phases), 0 switches timing off; enabling resets the
 * totals.  read returns the summed contact-kernel time in ms, the number of
 * timed steps, the number of engine kernels launched and the number of
 * rebuilds since enabling */
nbc_status nbc_timing_enable(nbc_engine* e, int enable);
nbc_status nbc_timing_read(nbc_engine* e, double* contact_ms, int* contact_launches, long long* kernel_launches,
                           int* rebuilds);
/* (timing level 2) mean CUDA-event time per timed step, in ms, of its
 * phases: [0] k_clump, [1] the rebuild node (its condition evaluated, the
 * rebuild when taken), [2] k_boundary, [3] k_contact, [4] the whole step from
 * its first kernel to its last (k_boundary runs beside k_contact); no
 * reference counterpart */
nbc_status nbc_timing_phases(nbc_engine* e, double* phase_ms);
/* the launch shapes an engine uses (see nbc_options) and whether its
 * untimed steps run as a device-side loop in one graph launch (1) or one
 * step per graph launch (0, e.g. when use_graph is 0); no reference
 * counterpart */
nbc_status nbc_launch_info(nbc_engine* e, int* step_loop, int* search_lanes, int* clump_batch, int* pair_blocks);
/* device memory in use and wall time of the last nbc_step in ms */
nbc_status nbc_engine_info(nbc_engine* e, double* device_bytes, double* last_step_ms);
/* Exact checkpoint, replacing the reference's restart from StartStep
 * (src/world.par:28, the step loop of src/dem_simulation_clump.cu:110),
 * which restarts from ph/ch snapshots and loses the spring histories.  write
 * waits for the device, applies the pending half-kick (as nbc_sync) and
 * saves the whole state the next step needs: scene bookkeeping, every
 * subsphere in its current sort order with its wall and intruder spring
 * histories, every clump, each scene's current pair list with its spring
 * histories, touch flags and near rows, and the intruder force record.
 * read loads such a file into an engine created (nbc_create / nbc_open)
 * from the same scenes with the same precision, before its first step or
 * after; stepping on then gives bitwise the results of the run that was
 * saved.  Writing before the first step is NBC_ERR_STATE; a file of other
 * scenes or precision is NBC_ERR_ARG; a missing file NBC_ERR_IO. */
nbc_status nbc_checkpoint_write(nbc_engine* e, const char* path);
nbc_status nbc_checkpoint_read(nbc_engine* e, const char* path);
/* No reference counterpart (the reference runs one scene until EndStep).
 * Scene `scene` takes `nsteps` steps counted from the engine's creation and
 * then stands still while the engine's other scenes go on: its state, forces
 * and intruder record are exactly those of the scene run alone for nsteps
 * steps, and it costs no contact or boundary work afterwards.  0 removes the
 * limit.  Call between steps; nsteps below the steps already started is an
 * NBC_ERR_ARG. */
nbc_status nbc_set_scene_steps(nbc_engine* e, int scene, int nsteps);

/* --- batches of independent scenes ---------------------------------------
 * No reference counterpart (the reference runs one scene per process).  A
 * batch is one engine over all its scenes, concatenated: every kernel of a
 * step covers every scene in one launch, and a rebuild covers only the
 * scenes whose own rebuild test fired (each scene keeps its own rebuild
 * schedule and its own region of the pair buffers), so each scene's results
 * are bitwise those of the scene run alone.  nbc_create with several scenes
 * makes the same engine; the batch calls exist for callers that think in
 * batches. */
typedef struct nbc_batch nbc_batch;
nbc_status nbc_batch_create(const nbc_scene_desc* const* scenes, int n_scenes, const nbc_options* opt,
                            nbc_batch** out);
nbc_status nbc_batch_step(nbc_batch* b, int nsteps);
/* the batch's engine, for the getters above: scene i of the batch is scene i
 * of this engine; owned by the batch (do not pass it to nbc_destroy), valid
 * until nbc_batch_destroy */
nbc_status nbc_batch_engine(nbc_batch* b, nbc_engine** e);
nbc_status nbc_batch_destroy(nbc_batch* b);

/* --- request server (continuous batching) ---------------------------------
 * No reference counterpart.  A request is a scene (copied at submission) and
 * a step count.  nbc_server_advance advances every running request by up to
 * `chunk` steps (at most 1024) and admits queued requests in arrival order
 * while the head fits the device-memory budget (estimated before creation,
 * actual after) and fewer than max_active run.  The requests admitted in one
 * call share one engine (a cohort: one launch per kernel and step for all of
 * them, each standing still at its own step count, nbc_set_scene_steps);
 * cohorts run concurrently on their own streams, and a cohort's memory is
 * returned when its last request finishes.  A request's result is
 * the intruder reaction force and torque every sample_every steps and at its
 * last step ([n_samples][6], the reference's fc record,
 * src/dem_integrate_penetrator.cu:108-109) and the intruder's final position;
 * it equals the result of the same scene run alone.  state: 0 queued,
 * 1 running, 2 done, 3 failed (a request whose engine fails is retired with
 * its error and the others go on; asking for its curve returns the error). */
typedef struct nbc_server nbc_server;
nbc_status nbc_server_create(const nbc_options* opt, double budget_bytes, int max_active, nbc_server** out);
nbc_status nbc_server_submit(nbc_server* s, const nbc_scene_desc* scene, int nsteps, int sample_every, int* id);
nbc_status nbc_server_advance(nbc_server* s, int chunk, int* n_running, int* n_queued, int* n_finished);
nbc_status nbc_server_result(nbc_server* s, int id, int* state, int* steps_done, int* n_samples, double* curve,
                             double* intr_pos);
nbc_status nbc_server_release(nbc_server* s, int id);
nbc_status nbc_server_memory(nbc_server* s, double* used_bytes, double* budget_bytes);
nbc_status nbc_server_destroy(nbc_server* s);
/* requests per cohort at most (default 1: an engine per request); the
 * requests admitted in one call are grouped by step count, within 2x */
nbc_status nbc_server_set_cohort(nbc_server* s, int max_requests);

/* Autotuner (no reference counterpart): times trial_steps steps (after a
 * short warm-up) of engines made from these scenes with candidate launch
 * shapes -- lanes per subsphere of the neighbour search, members per lane
 * of the clump pass, blocks per SM of the pair kernel -- by coordinate
 * descent from the defaults, a candidate replacing the incumbent only when
 * it is at least 3% faster, and writes the fastest into opt (other fields
 * untouched).  The shapes change no result: every candidate computes the
 * same lists and forces bit for bit.  The choice is cached in the process
 * by scene shape (scenes, subspheres, clumps, grid levels, precision) and
 * trial length; best_ms_per_step (may be NULL) receives its time. */
nbc_status nbc_autotune(const nbc_scene_desc* const* scenes, int n_scenes, nbc_options* opt, int trial_steps,
                        double* best_ms_per_step);

/* Hierarchical-grid levels for a radius distribution (replaces the grid.bt
 * level table the reference's sphere path reads, src/dem_io.cu:204-248):
 * writes level[n] (0 = coarsest) and level_cell[<=max_levels], returns the
 * number of levels (1 = the reference's single-level grid is best). */
#define NBC_MAX_LEVELS 6
int nbc_choose_levels(const double* radius, int n, int max_levels, int* level, double* level_cell);

/* Mass properties of clump templates (replaces the Monte Carlo integration of
 * the reference's template builder, make_clump_template_lambda.m:172-209, for
 * many clumps at once): for clump k, members clump_start[k] ..
 * clump_start[k+1]-1 with centres[3 m] (clump frame) and radii[m], the union
 * of the spheres (overlap counted once) integrated over its bounding box
 * with `samples` points of a deterministic low-discrepancy sequence.
 * out[10 k ..]: volume, centroid xyz, and the second central moments per
 * unit volume xx yy zz xy xz yz (inertia = density * volume * (trace * I -
 * moments)).  Host arrays; runs on `device` and returns when done. */
nbc_status nbc_union_mass(const double* centres, const double* radii, const int* clump_start, int nclumps,
                          int samples, double* out, int device);

/* --- allocation-free cell sort ------------------------------------------
 * No counterpart in the reference (its sort allocates CUB scratch with
 * cudaMalloc on first use, src/dem_grid.cu:278-305).  For callers that
 * cannot call cudaMalloc -- device memory owned by another framework's pool,
 * or a run whose memory budget is fixed at start-up: the cell hash of a
 * list rebuild plus a stable radix sort by cell (the order of the engine's
 * sort), with the caller's
 * buffers and one scratch array compiled into the library (NBC_NOALLOC_MAX_N
 * elements, about 2.2 MB per GPU that loads the library, kept until exit).
 *   pos_dev   device array [n][3] of positions (caller-owned)
 *   grid      the padded grid: origin, cell size, dims, the box whose
 *             outside goes to the last cell (as the engine's hash)
 *   perm_dev  device out [n]: index of the subsphere at each sorted slot
 *   key_dev   device out [n]: its cell, ascending
 *   stream    cudaStream_t to launch on (NULL: the default stream); the
 *             call returns after launching, the caller synchronises.
 * n above NBC_NOALLOC_MAX_N returns NBC_ERR_ARG.  A call made outside a
 * stream capture looks up the scratch array's device address (again on
 * every such call, so a device reset is followed); a captured call reuses
 * the address the last uncaptured call on that device found, so make the
 * first call on a device before any stream capture (a captured first call
 * returns NBC_ERR_STATE).  Calls share the scratch array: calls that overlap
 * on the GPU race and must be serialised by the caller. */
#define NBC_NOALLOC_MAX_N 262144
typedef struct {
    double origin[3];
    double cell;
    int dims[3];
    double box_lo[3], box_hi[3];
} nbc_grid_desc;
nbc_status nbc_cell_sort_noalloc(const double* pos_dev, int n, const nbc_grid_desc* grid, int* perm_dev,
                                 int* key_dev, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* NBC_H */
