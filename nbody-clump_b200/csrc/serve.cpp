// serve.cpp -- batches of independent scenes and a request server, on top of
// the engine.
//
// The reference runs one scene per process (DEMClumpMain::RunSimulationClump,
// src/dem_simulation_clump.cu:110-259).  Here many scenes share one GPU:
//   nbc_batch_*   a fixed set of scenes in one engine: every kernel of a step
//                 covers all of them in one launch, a rebuild covers the
//                 scenes whose own rebuild test fired, and each scene's
//                 results are bitwise those of the scene run alone.
//   nbc_server_*  continuous batching: requests (a scene and a step count)
//                 are queued, admitted in arrival order while the device-
//                 memory budget and the slot limit allow, advanced together in
//                 chunks (each request has its own engine and stream, the
//                 host enqueues a chunk on every stream before waiting for
//                 any), and retired when their steps are done, which frees
//                 their memory for the next admissions.  The result of a
//                 request is the intruder's reaction force and torque sampled
//                 every `sample_every` steps (the reference's fc output,
//                 src/dem_integrate_penetrator.cu:108-109) and its final
//                 position.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "handle.h"

using nbc::fail;
using nbc::guard;

// ---------------------------------------------------------------------------
// batch
// ---------------------------------------------------------------------------

struct nbc_batch {
    std::unique_ptr<nbc_engine> eng;
};

extern "C" {

nbc_status nbc_batch_create(const nbc_scene_desc* const* scenes, int n, const nbc_options* opt, nbc_batch** out) {
    if (!scenes || n <= 0 || !out) return fail(NBC_ERR_ARG, "nbc_batch_create: no scenes");
    for (int s = 0; s < n; s++)
        if (!scenes[s]) return fail(NBC_ERR_ARG, "nbc_batch_create: null scene");
    *out = nullptr;
    nbc_options o;
    if (opt) o = *opt; else nbc_default_options(&o);
    std::unique_ptr<nbc_batch> b(new nbc_batch());
    nbc_status st = guard([&] {
        std::unique_ptr<nbc_engine> h(new nbc_engine());
        h->opt = o;
        std::vector<const nbc_scene_desc*> v(scenes, scenes + n);
        h->eng.reset(nbc::make_engine(v, o));
        b->eng = std::move(h);
    });
    if (st == NBC_OK) *out = b.release();
    return st;
}

nbc_status nbc_batch_step(nbc_batch* b, int nsteps) {
    if (!b || nsteps < 0) return fail(NBC_ERR_ARG, "nbc_batch_step: bad arguments");
    return guard([&] { b->eng->eng->step(nsteps, false); });
}

nbc_status nbc_batch_engine(nbc_batch* b, nbc_engine** e) {
    if (!b || !e) return fail(NBC_ERR_ARG, "nbc_batch_engine: bad arguments");
    *e = b->eng.get();
    return NBC_OK;
}

nbc_status nbc_batch_destroy(nbc_batch* b) {
    delete b;
    return NBC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// server
// ---------------------------------------------------------------------------

namespace {

// a scene descriptor with its own copies of every array
struct SceneCopy {
    nbc_scene_desc d{};
    std::vector<int> cid, level;
    std::vector<double> pos, local, mass, radius, cpos, cvel, cquat, cw, cprop, lcell;
    explicit SceneCopy(const nbc_scene_desc& s) : d(s) {
        const size_t n = (size_t)s.n_sub, k = (size_t)s.n_clump;
        auto cp = [](const auto* p, size_t m, auto& v) {
            if (p) v.assign(p, p + m);
            return p ? v.data() : nullptr;
        };
        d.clump_id = cp(s.clump_id, n, cid);
        d.pos = cp(s.pos, 3 * n, pos);
        d.local = cp(s.local, 3 * n, local);
        d.mass = cp(s.mass, n, mass);
        d.radius = cp(s.radius, n, radius);
        d.clump_pos = cp(s.clump_pos, 3 * k, cpos);
        d.clump_vel = cp(s.clump_vel, 3 * k, cvel);
        d.clump_quat = cp(s.clump_quat, 4 * k, cquat);
        d.clump_angvel = cp(s.clump_angvel, 3 * k, cw);
        d.clump_prop = cp(s.clump_prop, 4 * k, cprop);
        d.level = s.levels > 1 ? cp(s.level, n, level) : nullptr;
        d.level_cell = s.levels > 1 ? cp(s.level_cell, (size_t)s.levels, lcell) : nullptr;
    }
};

struct Request {
    int id = 0, state = 0;  // 0 queued, 1 active, 2 done, 3 failed
    int nsteps = 0, sample_every = 1, done = 0;
    double est_bytes = 0, bytes = 0;
    std::unique_ptr<SceneCopy> scene;
    std::unique_ptr<nbc_engine> eng;
    std::vector<double> curve;  // [samples][6]: reaction force, reaction torque
    double intr_pos[3] = {0, 0, 0};
    std::string error;
};

// device bytes a scene is expected to take before it is created: per
// subsphere state and grid, and pair buffers of about 12 pairs per subsphere
double estimate_bytes(const nbc_scene_desc& s, const nbc_options& o) {
    const double r = o.precision == NBC_PREC_F64 ? 8.0 : 4.0;
    const double per_sub = 1100.0 + 3 * 2 * 4 * r * 7;       // state, alternates, boundary histories
    const double per_pair = 2 * (16 + 2 * 4 * r + r + 1) + 5 * 4 * r + 32 + 9;
    const double cells = 2.0 * (double)s.n_sub * 4.0;          // grid table, a few ints per subsphere
    return (double)s.n_sub * per_sub + 12.0 * (double)s.n_sub * per_pair * 1.6 + cells;
}

}  // namespace

struct nbc_server {
    nbc_options opt;
    double budget = 0, used = 0;
    int max_active = 1, next_id = 1;
    std::map<int, std::unique_ptr<Request>> req;
    std::deque<int> queue;     // ids waiting for admission, in arrival order
    std::vector<int> active;   // ids being advanced
};

extern "C" {

nbc_status nbc_server_create(const nbc_options* opt, double budget_bytes, int max_active, nbc_server** out) {
    if (!out || max_active < 1 || !(budget_bytes > 0)) return fail(NBC_ERR_ARG, "nbc_server_create: bad arguments");
    std::unique_ptr<nbc_server> s(new nbc_server());
    if (opt) s->opt = *opt; else nbc_default_options(&s->opt);
    if (!(s->opt.pair_slack >= 1.0)) s->opt.pair_slack = 1.6;  // pair buffers sized by the first list
    s->budget = budget_bytes;
    s->max_active = max_active;
    *out = s.release();
    return NBC_OK;
}

nbc_status nbc_server_submit(nbc_server* s, const nbc_scene_desc* scene, int nsteps, int sample_every, int* id) {
    if (!s || !scene || nsteps < 1 || sample_every < 1 || !id) return fail(NBC_ERR_ARG, "nbc_server_submit: bad arguments");
    return guard([&] {
        std::unique_ptr<Request> r(new Request());
        r->id = s->next_id++;
        r->nsteps = nsteps;
        r->sample_every = sample_every;
        r->scene.reset(new SceneCopy(*scene));
        r->est_bytes = estimate_bytes(*scene, s->opt);
        *id = r->id;
        s->queue.push_back(r->id);
        s->req[r->id] = std::move(r);
    });
}

// Admit queued requests (in arrival order, while the head fits the budget
// and a slot is free), advance every active request by up to chunk steps
// (concurrently), record their samples and retire the finished ones.
nbc_status nbc_server_advance(nbc_server* s, int chunk, int* n_active, int* n_queued, int* n_done) {
    if (!s || chunk < 1) return fail(NBC_ERR_ARG, "nbc_server_advance: bad arguments");
    chunk = std::min(chunk, 1024);  // the engine's intruder ring keeps the last 1024 steps at least
    nbc_status st = guard([&] {
        // one chunk of every running request is put on its stream first, so
        // the GPU works while new requests are admitted and created
        const std::vector<int> running = s->active;
        std::vector<int> launched(running.size(), 0), want(running.size(), 0), did(running.size(), 0);
        // a request whose engine fails (non-finite force, device memory) is
        // retired with its error; the others go on
        auto retire_failed = [&](Request& r, const std::exception& e) {
            r.state = 3;
            r.error = e.what();
            s->used -= r.bytes;
            r.eng.reset();
            r.scene.reset();
        };
        for (size_t k = 0; k < running.size(); k++) {
            Request& r = *s->req[running[k]];
            want[k] = std::min(chunk, r.nsteps - r.done);
            try {
                launched[k] = r.eng->eng->enqueue(want[k]);
            } catch (const std::exception& e) {
                retire_failed(r, e);
            }
        }
        // admission: arrival order, while the head fits and a slot is free
        while (!s->queue.empty() && (int)s->active.size() < s->max_active) {
            Request& r = *s->req[s->queue.front()];
            if (!s->active.empty() && s->used + r.est_bytes > s->budget) break;
            s->queue.pop_front();
            std::unique_ptr<nbc_engine> h(new nbc_engine());
            h->opt = s->opt;
            std::vector<const nbc_scene_desc*> v(1, &r.scene->d);
            try {
                h->eng.reset(nbc::make_engine(v, s->opt));
            } catch (const std::exception& e) {
                r.state = 3;
                r.error = e.what();
                r.scene.reset();
                continue;
            }
            double b = 0, ms = 0;
            h->eng->info(&b, &ms);
            // whole bytes, so that the sum over running requests stays exact
            r.bytes = std::ceil(std::max(b, r.est_bytes));
            s->used += r.bytes;
            r.eng = std::move(h);
            r.state = 1;
            s->active.push_back(r.id);
        }
        // the rest of each running request's chunk (a capacity overflow can
        // stop a chunk early), waited for in turn
        for (size_t k = 0; k < running.size(); k++) {
            Request& r = *s->req[running[k]];
            if (r.state != 1) continue;
            try {
                if (launched[k] > 0) did[k] = r.eng->eng->wait_steps();
                while (did[k] < want[k]) {
                    r.eng->eng->enqueue(want[k] - did[k]);
                    did[k] += r.eng->eng->wait_steps();
                }
            } catch (const std::exception& e) {
                retire_failed(r, e);
            }
        }
        std::vector<int> still;
        for (size_t k = 0; k < running.size(); k++) {
            Request& r = *s->req[running[k]];
            if (r.state != 1) continue;
            // samples at the steps of this chunk that are multiples of sample_every
            const int first = r.done + 1, last = r.done + did[k];
            if (did[k] > 0) {
                r.eng->eng->sync();  // the last step's reaction is recorded by its closing half-kick
                std::vector<double> hist((size_t)did[k] * 6);
                r.eng->eng->get_intruder_history(0, did[k], hist.data());
                for (int st = first; st <= last; st++)
                    if (st % r.sample_every == 0 || st == r.nsteps)
                        r.curve.insert(r.curve.end(), &hist[(size_t)(st - first) * 6], &hist[(size_t)(st - first) * 6 + 6]);
            }
            r.done = last;
            if (r.done >= r.nsteps) {
                r.eng->eng->sync();
                double v[3], reac[3], tq[3];
                int state = 0;
                r.eng->eng->get_intruder(0, r.intr_pos, v, reac, tq, &state);
                s->used -= r.bytes;
                r.eng.reset();
                r.scene.reset();
                r.state = 2;
            } else {
                still.push_back(r.id);
            }
        }
        // the requests admitted in this round run from the next one
        for (size_t k = running.size(); k < s->active.size(); k++) still.push_back(s->active[k]);
        s->active = still;
    });
    if (n_active) *n_active = (int)s->active.size();
    if (n_queued) *n_queued = (int)s->queue.size();
    if (n_done) {
        int c = 0;
        for (auto& kv : s->req) c += kv.second->state >= 2;
        *n_done = c;
    }
    return st;
}

nbc_status nbc_server_result(nbc_server* s, int id, int* state, int* steps_done, int* n_samples, double* curve,
                             double* intr_pos) {
    if (!s) return fail(NBC_ERR_ARG, "nbc_server_result: null server");
    auto it = s->req.find(id);
    if (it == s->req.end()) return fail(NBC_ERR_ARG, "nbc_server_result: unknown request " + std::to_string(id));
    const Request& r = *it->second;
    if (state) *state = r.state;
    if (steps_done) *steps_done = r.done;
    if (n_samples) *n_samples = (int)(r.curve.size() / 6);
    if (curve && r.state == 2) std::copy(r.curve.begin(), r.curve.end(), curve);
    if (intr_pos && r.state == 2) std::copy(r.intr_pos, r.intr_pos + 3, intr_pos);
    // a failed request reports its state; asking for its result returns its error
    if (r.state == 3 && (curve || intr_pos)) return fail(NBC_ERR_STATE, "request " + std::to_string(id) + ": " + r.error);
    return NBC_OK;
}

nbc_status nbc_server_release(nbc_server* s, int id) {
    if (!s) return fail(NBC_ERR_ARG, "nbc_server_release: null server");
    auto it = s->req.find(id);
    if (it == s->req.end() || it->second->state < 2) return fail(NBC_ERR_STATE, "nbc_server_release: request not finished");
    s->req.erase(it);
    return NBC_OK;
}

nbc_status nbc_server_memory(nbc_server* s, double* used_bytes, double* budget_bytes) {
    if (!s) return fail(NBC_ERR_ARG, "nbc_server_memory: null server");
    if (used_bytes) *used_bytes = s->used;
    if (budget_bytes) *budget_bytes = s->budget;
    return NBC_OK;
}

nbc_status nbc_server_destroy(nbc_server* s) {
    delete s;
    return NBC_OK;
}

}  // extern "C"
