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
    std::vector<int> cid, level, kind;
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
        d.body_kind = cp(s.body_kind, k, kind);
    }
};

struct Request {
    int id = 0, state = 0;  // 0 queued, 1 running, 2 done, 3 failed
    int nsteps = 0, sample_every = 1, done = 0;
    double est_bytes = 0;
    std::unique_ptr<SceneCopy> scene;   // until its cohort is created
    int cohort = -1, slot = 0;          // its cohort and its scene there
    std::vector<double> curve;  // [samples][6]: reaction force, reaction torque
    double intr_pos[3] = {0, 0, 0};
    std::string error;
};

// The requests admitted in one round share one engine: one launch per kernel
// and step covers all of them, and each request's scene stands still once its
// own step count is reached (nbc_set_scene_steps) while the others go on.
// The engine and its memory are released when its last request finishes.
struct Cohort {
    std::unique_ptr<nbc_engine> eng;
    std::vector<int> ids;   // the request of each scene
    int started = 0;        // steps the engine has taken
    int longest = 0;        // the largest step count of its requests
    int open = 0;           // requests still running
    double bytes = 0;
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
    int max_active = 1, next_id = 1, next_cohort = 1;
    int cohort_max = 1;              // requests per cohort at most
    std::map<int, std::unique_ptr<Request>> req;
    std::deque<int> queue;           // ids waiting for admission, in arrival order
    std::map<int, Cohort> cohorts;   // running cohorts
    int running = 0;                 // requests admitted and not finished
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

// Advance every running cohort by up to chunk steps (all cohorts' chunks
// are enqueued before any is waited for), admit queued requests (arrival
// order, while the head fits the budget and a slot is free) into one new
// cohort created while the others run, record the new samples of every
// running request and retire the finished ones.
nbc_status nbc_server_advance(nbc_server* s, int chunk, int* n_active, int* n_queued, int* n_done) {
    if (!s || chunk < 1) return fail(NBC_ERR_ARG, "nbc_server_advance: bad arguments");
    chunk = std::min(chunk, 1024);  // the engine's intruder ring keeps the last 1024 steps at least
    nbc_status st = guard([&] {
        // a cohort whose engine fails (non-finite force, device memory) is
        // retired with its error on every request still running in it; the
        // other cohorts go on
        auto fail_cohort = [&](Cohort& c, const std::exception& e) {
            for (int id : c.ids) {
                auto f = s->req.find(id);   // finished requests may have been released
                if (f == s->req.end() || f->second->state != 1) continue;
                Request& r = *f->second;
                r.state = 3;
                r.error = e.what();
                s->running--;
            }
            c.open = 0;
        };
        std::vector<int> old;
        std::map<int, int> want, launched;
        for (auto& kv : s->cohorts) {
            Cohort& c = kv.second;
            old.push_back(kv.first);
            want[kv.first] = std::min(chunk, c.longest - c.started);
            try {
                launched[kv.first] = c.eng->eng->enqueue(want[kv.first]);
            } catch (const std::exception& e) {
                fail_cohort(c, e);
            }
        }
        // admission into one new cohort, created while the others run
        std::vector<int> adm;
        double add = 0;
        while (!s->queue.empty() && s->running + (int)adm.size() < s->max_active) {
            Request& r = *s->req[s->queue.front()];
            if ((s->running > 0 || !adm.empty()) && s->used + add + r.est_bytes > s->budget) break;
            s->queue.pop_front();
            adm.push_back(r.id);
            add += r.est_bytes;
        }
        // the admitted requests, in order of their step counts, form cohorts
        // of at most cohort_max requests whose step counts are within 2x
        std::stable_sort(adm.begin(), adm.end(), [&](int a, int b) { return s->req[a]->nsteps < s->req[b]->nsteps; });
        std::vector<std::vector<int>> groups;
        for (int id : adm) {
            if (groups.empty() || (int)groups.back().size() >= s->cohort_max ||
                s->req[id]->nsteps > 2 * s->req[groups.back().front()]->nsteps)
                groups.emplace_back();
            groups.back().push_back(id);
        }
        for (std::vector<int>& adm : groups) {
            double add = 0;
            for (int id : adm) add += s->req[id]->est_bytes;
            Cohort c;
            std::vector<const nbc_scene_desc*> v;
            for (int id : adm) v.push_back(&s->req[id]->scene->d);
            try {
                c.eng.reset(new nbc_engine());
                c.eng->opt = s->opt;
                c.eng->eng.reset(nbc::make_engine(v, s->opt));
                for (size_t k = 0; k < adm.size(); k++) {
                    Request& r = *s->req[adm[k]];
                    c.eng->eng->set_stop((int)k, r.nsteps);
                    c.longest = std::max(c.longest, r.nsteps);
                }
                double b = 0, ms = 0;
                c.eng->eng->info(&b, &ms);
                // whole bytes, so that the sum over running cohorts stays exact
                c.bytes = std::ceil(std::max(b, add));
                for (size_t k = 0; k < adm.size(); k++) {
                    Request& r = *s->req[adm[k]];
                    r.state = 1;
                    r.cohort = s->next_cohort;
                    r.slot = (int)k;
                    r.scene.reset();
                }
                c.ids = adm;
                c.open = (int)adm.size();
                s->used += c.bytes;
                s->running += (int)adm.size();
                s->cohorts[s->next_cohort++] = std::move(c);
            } catch (const std::exception& e) {
                for (int id : adm) {
                    Request& r = *s->req[id];
                    r.state = 3;
                    r.error = e.what();
                    r.scene.reset();
                }
            }
        }
        // the rest of each old cohort's chunk (a capacity overflow can stop a
        // chunk early), then the new samples of its requests
        for (int cid : old) {
            Cohort& c = s->cohorts[cid];
            if (c.open == 0) continue;
            try {
                int did = launched[cid] > 0 ? c.eng->eng->wait_steps() : 0;
                while (did < want[cid]) {
                    c.eng->eng->enqueue(want[cid] - did);
                    did += c.eng->eng->wait_steps();
                }
                c.started += did;
                if (did == 0) continue;
                c.eng->eng->sync();  // the last step's reaction is recorded by its closing half-kick
                for (int id : c.ids) {
                    auto f = s->req.find(id);   // finished requests may have been released
                    if (f == s->req.end() || f->second->state != 1) continue;
                    Request& r = *f->second;
                    const int now = std::min(c.started, r.nsteps), n = now - r.done;
                    if (n > 0) {
                        // samples at the new steps that are multiples of sample_every
                        std::vector<double> hist((size_t)n * 6);
                        c.eng->eng->get_intruder_history(r.slot, n, hist.data());
                        for (int k = r.done + 1; k <= now; k++)
                            if (k % r.sample_every == 0 || k == r.nsteps)
                                r.curve.insert(r.curve.end(), &hist[(size_t)(k - r.done - 1) * 6],
                                               &hist[(size_t)(k - r.done - 1) * 6 + 6]);
                        r.done = now;
                    }
                    if (r.done >= r.nsteps) {
                        double v[3], reac[3], tq[3];
                        int state = 0;
                        c.eng->eng->get_intruder(r.slot, r.intr_pos, v, reac, tq, &state);
                        r.state = 2;
                        c.open--;
                        s->running--;
                    }
                }
            } catch (const std::exception& e) {
                fail_cohort(c, e);
            }
        }
        // cohorts without running requests release their engine and memory
        for (auto it = s->cohorts.begin(); it != s->cohorts.end();) {
            if (it->second.open == 0) {
                s->used -= it->second.bytes;
                it = s->cohorts.erase(it);
            } else {
                ++it;
            }
        }
    });
    if (n_active) *n_active = s->running;
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

nbc_status nbc_server_set_cohort(nbc_server* s, int max_requests) {
    if (!s || max_requests < 1) return fail(NBC_ERR_ARG, "nbc_server_set_cohort: bad arguments");
    s->cohort_max = max_requests;
    return NBC_OK;
}

nbc_status nbc_server_destroy(nbc_server* s) {
    delete s;
    return NBC_OK;
}

}  // extern "C"
