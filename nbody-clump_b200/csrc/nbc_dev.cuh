// nbc_dev.cuh -- device-side data layout of the B200 DEM engine.
//
// A *batch* holds S independent scenes concatenated: scene s owns the
// subsphere range [sub_off, sub_off+nsub) and the clump range
// [clump_off, clump_off+nclump).  Subspheres are stored in cell-sorted
// order within their scene (the reference keeps its particle arrays in the
// order of its last cell sort, src/dem_simulation_clump.cu:128-164); a
// rebuild only permutes within a scene, so scenes stay contiguous.
//
// Every kernel receives one pointer to a device-resident `Dev` table that
// holds all buffer pointers, so buffers can be re-allocated without
// re-capturing the CUDA graph.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace nbc {

constexpr int MAX_LEVELS = 6;   // NBC_MAX_LEVELS of the C ABI
constexpr int WALL_NONE = 0, WALL_CUBE = 1, WALL_CYL = 2;
// boundary slots of a subsphere: cube faces UpX, LowX, UpY, LowY, UpZ, LowZ
// (src/dem_force_cube_wall_clump.cu:228-292), or cylinder regions bottom cap,
// top cap, side (src/dem_force_cylind_wall.cu:178-233), then the intruder.
constexpr int NB_WALL_MAX = 6;
constexpr int SLOT_INTR = 6;
constexpr int NB_SLOTS = 7;

// error bits of SceneDyn::err
constexpr int ERR_LIST_OVERFLOW = 1;   // pair capacity exceeded (host grows and retries)
constexpr int ERR_NONFINITE = 2;       // non-finite wall input/output (src/dem_force_cube_wall_clump.cu:191-203)
constexpr int ERR_BAD_CLUMP = 4;       // clump id out of range
constexpr int ERR_ROW_OVERFLOW = 8;    // a row exceeded BranchLmtLen/2 (reference semantics, export only)

// ScenePar::sphere: the reference's sphere-only drivers where they differ
// from the clump path (bits 1, 2, 4 are NBC_SPHERE_* of the C ABI)
constexpr int SPH_KIN = 1;      // first half-kick and attitude without the intruder; penetrator cohesion
constexpr int SPH_CUBE = 2;     // cube wall without history and without rolling or twisting moment
constexpr int SPH_RESET = 4;    // pair histories restart from zero at every rebuild
constexpr int SPH_KINDS = 8;    // body kinds of the split driver (Dev::kind)

struct ScenePar {
    // integration and contact law (world.par, src/dem_parameters.h:49-66)
    double dt, E, nu, mu, damping, gravity, beta, cohesion, thresh;
    double kn_fac;  // 2E / (3 (1 - nu^2))                 src/dem_force_clump.cu:68
    double ks_fac;  // 2E / (1 + nu) / (2 - nu)            src/dem_force_clump.cu:71
    // grid (src/dem_subsphere_io.cu:195-230)
    double origin[3], cell[3], icell[3], box_lo[3], box_hi[3];
    int gdim[3];
    int cellnum;    // cells of this scene incl. the out-of-box bucket
    int cell_off;   // first global cell id of this scene
    int levels;     // 1 = single level grid
    double lcell[MAX_LEVELS];
    int ldim[MAX_LEVELS][3];
    int loff[MAX_LEVELS];
    // ranges
    int sub_off, nsub, clump_off, nclump;
    int bl;                // BranchLmtLen of the reference (row capacity of the export)
    // walls
    int wall;       // WALL_*
    double w_half[3], w_c[3], w_v[3], w_w[3];   // cube: half sizes, centre, velocity, angular velocity
    double cyl_R, cyl_H, cyl_axis[3];           // cylinder: radius, half height, axis (centre in w_c)
    // intruder
    int has_intr, intr_shape, intr_motion, intr_wait;  // shape 0 cylinder 1 sphere; motion 0 kinematic 1 gravity
    double intr_R, intr_H, intr_axis[3], intr_mass, intr_w[3];
    int sphere;     // SPH_* bits, 0 = the clump path
};

struct SceneDyn {
    double intr_p[3], intr_v[3];
    double totF[3], totT[3];       // sum over subspheres of the intruder force / torque (src/dem_force_penetrator.cu:237-248)
    double reaction[3], reaction_t[3];
    int intr_state;                // ContactState (src/dem_parameters.h:82-91)
    int rebuild;                   // set by the pose pass when a subsphere moved > Thresh
    int err;
    int step;                      // completed steps
    int nrebuild;
    int npairs;                    // pairs in the current list
    int pair_off;                  // first pair slot of this scene's region of the pair buffers
    int pcap;                      // pair slots of that region (set by the host, grown on overflow)
    int nnear;                     // near pairs of the current list (see k_near)
    int nbound;                    // boundary candidates of the current list (see k_bflag)
    int stop;                      // steps the scene takes before it stands still (0: no limit)
    int frozen;                    // the scene took no step at the last k_clump (its stop was reached)
    long long ifix[6];             // fixed-point sums of intruder force (2^-40 N) and torque (2^-44 N m)
};

// Pair list of a batch: scene s owns the pair slots [pair_off, pair_off +
// pcap) of every per-pair buffer, so a scene's rebuild rewrites its own region
// only.  Row offsets are absolute slots, one row array per scene with its end
// entry: subsphere i of scene s starts at row[i + s], ends at row[i + s + 1].
struct PairList {
    int* row;     // [N+S] front (owner) row offsets
    int* brow;    // [N+S] back row offsets
    int* nbr;     // [cap] front partner, bit 31 set for pairs inside one clump
    int* own;     // [cap] owner of each pair (the reference's Lpa)
    int* bnbr;    // [cap] back partner (the owner), bit 31 set inside one clump
    int* bpair;   // [cap] pair index of each back entry (the reference's Aref)
};

// entries of Dev::plan
constexpr int PL_NS = 0;     // rebuilt scenes
constexpr int PL_T = 1;      // their subspheres
constexpr int PL_TC = 2;     // their cell-table entries
constexpr int PL_T1 = 3;     // PL_T + 1 (scan length of the counts)
constexpr int PL_TK = 4;     // their clumps
constexpr int PL_CS = 5;     // work counter of k_search (subspheres claimed)
constexpr int PL_CC = 6;     // work counter of k_compact
constexpr int PL_TC1 = 7;    // PL_TC + 1 (scan length of the cell counts)
constexpr int PL_SIZE = 8;

struct Dev {
    int S, N, K;
    int cap;          // pair capacity of each list buffer
    int cells;        // total global cells (sum over scenes)
    int has_stops;    // some scene has a step limit (nbc_set_scene_steps): the kernels check for frozen scenes
    ScenePar* par;
    SceneDyn* dyn;
    int* sid;         // [N] scene of each subsphere
    int* csid;        // [K] scene of each clump
    // subspheres, sorted order.  Each persistent array has an alternate
    // buffer (suffix 2): a rebuild gathers the rebuilt scenes into the
    // alternates and writes them back once the new list is complete, so
    // nothing changes if it stops early.
    double4* posr;    double4* posr2;    // x y z r
    double4* lom;     double4* lom2;     // local offset (body frame) xyz, mass
    double4* cum;     double4* cum2;     // displacement since the last rebuild
    int* clump_id;    int* clump_id2;
    int* part_fix;    int* part_fix2;    // original index (ParticleID)
    int* level;       int* level2;       // hgrid level (0 = coarsest)
    int* key;         int* key2;         // global cell key at the last rebuild (sorted)
    void* kin;        void* kin2;        // double4 [N]: world arm, mass (the velocities are the
                                         // clump's; see Body in kernels.cuh)
    void* bhist;      void* bhist2;      // Real4 [NB_SLOTS][N][3] boundary histories (Dv, Dt, Dr adjacent)
    uint16_t* bbits;  uint16_t* bbits2;  // [N] boundary slots in contact at the last step
    void* fsum;       // Real4 [2][N]: force and torque on each subsphere (pairs + walls + intruder),
                      // written on request only (getters, export): the clump pass sums the slots itself
    void* fbnd;       // Real4 [2][N]: wall + intruder force and torque, valid where bbits != 0
    void* fint;       // Real4 [2][N]: intruder force and torque alone, valid where the intruder bit of
                      // bbits is set, in SPH_KIN scenes (null when there are none)
    // clumps
    double4* cpos;    // xyz
    double4* cvel;
    double4* cw;
    double4* cq;      // x y z w
    double4* cprop;   // Ixx Iyy Izz M
    int* mem_cl;      // [N] clump of each member slot (fixed: members stay in their clump's range)
    double4* cinv;    // 1/Ixx 1/Iyy 1/Izz 1/M (correctly rounded divisions, computed once)
    int* kind;        // [K] body kind of the split driver (0 free, 1 prescribed velocity, 2 fixed),
                      // read in SPH_KINDS scenes only (null when there are none)
    double4* cF;      // force on clump from the last force pass
    double4* cT;
    int* mem_start;   // [K+1]
    int* mem_idx;     // [N] member subspheres of each clump, ascending
    int* post_pending;// device flag: a force pass has run whose half-kick is pending
    // broad phase scratch
    int* kA; int* vA; int* kB; int* vB;   // radix sort ping-pong
    int* perm;        // [N] old index of new slot i (part_idx_pre)
    int* inv;         // [N] new slot of old index
    int* cstart;                          // [cells+1] first sorted slot of each cell
    int* scr;                             // [N][2][SCR_CAP] front / back scratch rows of the fused search
    int* cnt_f; int* cnt_b;               // [N+1] counts, scanned in place
    int* sfc;                             // [N] same-level front count (hierarchical grid)
    int* xcnt;                            // [N] cross-level entries placed so far (hierarchical grid)
    int* scan_tmp;                        // block sums
    unsigned long long* scan_st;          // single-launch scan: tile states (zero between scans)
    int* scan_ctl;                        // single-launch scan: ticket and finished-block counters
    int* scan_fail;                       // a single-launch scan gave up a wait (the step halted)
    int* any_rebuild;                     // device flag: some scene rebuilds this step
    // rebuild plan (k_plan): the scenes rebuilt at this step in ascending
    // order and prefix sums over them; every rebuild kernel runs over the
    // concatenation of the rebuilt scenes only
    int* plan;        // [PL_SIZE] counts, see PL_*
    int* ccnt;        // [cells + S + 1] subspheres per cell of the rebuilt scenes (the sort's counts; zero at rest)
    int* ccur;        // [cells + S + 1] fill cursors of the sort's scatter (zero at rest)
    int* pscene;      // [S] rebuilt scenes
    int* psub;        // [S+1] prefix of their subsphere counts
    int* pcell;       // [S+1] prefix of their cell-table entries (cellnum + 1)
    int* pclump;      // [S+1] prefix of their clump counts
    int* ppair;       // [S+1] prefix of the pairs of their new lists
    int* need;        // [S] pairs of the new list of each rebuilt scene, -1 for the others
    int* halt;                            // device flag: pair capacity exceeded, kernels stand still
    // pair lists: the current one and the one a rebuild builds (written
    // back into the current one), histories ping-pong between steps
    PairList L[2];
    int* lcur;        // index of the current list (0)
    void* H[2];       // per pair: Real4 (Dv.xyz, Dr.x), Real4 (Dt.xyz, Dr.y) adjacent, [2*cap] Real4, then Real Dr.z [cap]
    uint8_t* touch[2];// [cap] pair in contact at the step that wrote H
    // contact slots, one per near row entry (see k_near), written by every
    // contact pass (zero for a pair that does not touch) and summed by the
    // next clump pass in row order: front entries hold the force and torque
    // on the row's subsphere as owner, back entries as partner
    void* nfs;        // Real4 [cap][2]: force and torque (adjacent) per near front entry
    void* nbs;        // Real4 [cap][2]: force and torque (adjacent) per near back entry
    int* nbpos;       // [cap] the near back entry of each near pair
    // near rows (the entries that can touch before the next rebuild)
    // (kept in each scene's pair region like the list: rows [N+S] with
    // absolute slots, one row array per scene with its end entry)
    int2* nrb;        // [N+S] near row offsets (front, back), one record per subsphere
    int4* nfr;        // [cap] near front entries: pair slot, partner, owner, near back entry
    int* nbq;         // [cap] near back entries: pair slot
    int* nprefix;     // [S+1] prefix over the scenes of their near pairs (the contact pass's work items)
    int* bidx;        // [N] boundary candidates of scene s at [sub_off, sub_off + nbound) (see k_bflag)
    int* bprefix;     // [S+1] prefix over the scenes of their boundary candidates (k_boundary's work items)
    uint8_t* nearf;   // [cap] pair can touch before the next rebuild
    int* hgen;        // history generation: read H[hgen&1], write H[(hgen+1)&1]
    int* gstep;       // steps started by k_clump (counts steps across graph launches)
    int* kc_done;     // blocks of k_clump finished (last-block detection)
    int* lstep;       // steps started by k_clump, counted by its last block (per-scene stops)
    int* loop_left;   // steps left in a graph launch with a device-side step loop
    // export (per pair), written by the export variant of the contact kernel
    void* xfcn;       // Real4 [cap] normal force on the owner (CacheFcn)
    void* xcpt;       // double4 [cap] contact point (CacheCpt)
    void* xparts;     // Real4 [6][N]: pair F, T, wall F, T, intruder F, T
    void* xintr;      // Real4 [4][N]: intruder Fcn, Fct, Tcn, Tct
    // intruder force history ring (per scene), reaction force and torque
    double* ring;     // [S][ring_len][6]
    int ring_len;
};

}  // namespace nbc
