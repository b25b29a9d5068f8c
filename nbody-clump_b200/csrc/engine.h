// engine.h -- host interface of the B200 DEM engine (implementation in
// engine.cu, C ABI in capi.cpp).
#pragma once
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/nbc.h"

namespace nbc {

struct NonFinite : std::runtime_error {
    using std::runtime_error::runtime_error;
};
// a call that is not valid in the engine's state (NBC_ERR_STATE)
struct StateError : std::logic_error {
    using std::logic_error::logic_error;
};

// One batch of scenes resident on one GPU.
class EngineBase {
   public:
    virtual ~EngineBase() {}
    virtual void step(int n, bool export_last) = 0;
    virtual int enqueue(int n) = 0;   // launch up to n steps without waiting
    virtual int wait_steps() = 0;     // wait for them; the number done
    virtual void sync() = 0;
    virtual int num_scenes() const = 0;
    virtual void stats(int s, int* steps, int* rebuilds, int* npairs, int* err) = 0;
    virtual void contact_counts(long long* nnear, long long* ntouch) = 0;
    virtual void get_subspheres(int s, int* fix, int* cid, double* pos, double* rad) = 0;
    virtual void get_body(int s, double* local, double* mass) = 0;
    virtual void get_clump_prop(int s, double* prop) = 0;
    virtual void get_clumps(int s, double* pos, double* vel, double* quat, double* w, double* f, double* t) = 0;
    virtual void get_sub_forces(int s, double* f, double* t) = 0;
    virtual void get_force_parts(int s, double* parts) = 0;
    virtual void get_intruder_diag(int s, double* diag) = 0;
    virtual void get_pairs(int s, int* np, int* lpa, int* lpb) = 0;
    virtual void get_rows(int s, int bl, int* anei, int* ng, int* ni) = 0;
    virtual void get_chain(int s, int bl, double* fcn, double* cpt) = 0;
    virtual void get_pair_forces(int s, int* np, double* fcn) = 0;
    virtual void get_intruder(int s, double* pos, double* vel, double* reac, double* tq, int* state) = 0;
    virtual void get_intruder_history(int s, int count, double* out) = 0;
    virtual void info(double* bytes, double* ms) = 0;
    // launch shapes in use; step_loop: 1 if untimed steps run in a device-side
    // loop (captured and instantiated), 0 if one step per graph launch
    virtual void launch_info(int* step_loop, int* search_lanes, int* clump_batch, int* pair_blocks) = 0;
    virtual void set_stop(int s, int nsteps) = 0;
    virtual void timing_enable(int level) = 0;
    virtual void timing_read(double* contact_ms, int* contact_launches, long long* kernel_launches, int* rebuilds) = 0;
    virtual void timing_phases(double* phase_ms) = 0;
    // exact checkpoint of the state after the last completed step (see
    // EngineT::checkpoint_save); load into an engine made from the same
    // scenes and options
    virtual std::vector<char> checkpoint_save() = 0;
    virtual void checkpoint_load(const char* data, size_t bytes) = 0;
};

EngineBase* make_engine(const std::vector<const nbc_scene_desc*>& scenes, const nbc_options& opt);

}  // namespace nbc
