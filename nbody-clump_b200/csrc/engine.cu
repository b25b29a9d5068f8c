// engine.cu -- host side of the B200 DEM engine and its C ABI (include/nbc.h).
//
// The Engine owns every device buffer of a batch of scenes, launches the
// kernels of kernels.cuh, captures one step as a CUDA graph whose rebuild
// branch is a conditional node, and converts device data to the reference's
// host layouts on request.  It replaces the host orchestration of
// DEMClumpMain::RunSimulationClump (src/dem_simulation_clump.cu:3-259), which
// synchronises with the device about 30 times per step.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdint>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/nbc.h"
#include "kernels.cuh"
#include "engine.h"

namespace nbc {

thread_local std::string g_last_error;

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
// an argument the caller can fix; the C ABI reports it as NBC_ERR_ARG
struct ArgError : std::invalid_argument {
    using std::invalid_argument::invalid_argument;
};

#define CK(call)                                                                             \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            throw CudaError(std::string(#call) + ": " + cudaGetErrorString(e_) + " at " +   \
                            __FILE__ + ":" + std::to_string(__LINE__));                      \
    } while (0)


static inline int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

// ---------------------------------------------------------------------------
// device memory helper
// ---------------------------------------------------------------------------
// Stream-ordered allocations from the device's default memory pool, kept in
// the pool when freed: creating and destroying engines while others run (a
// request server) neither synchronises the device (as cudaMalloc / cudaFree
// do) nor returns memory to the driver between requests.
struct DevMem {
    std::vector<void*> ptrs;
    double bytes = 0;
    cudaStream_t stream = nullptr;
    template <typename T>
    T* alloc(size_t n) {
        void* p = nullptr;
        size_t b = std::max<size_t>(n, 1) * sizeof(T);
        cudaError_t e = cudaMallocAsync(&p, b, stream);
        if (e != cudaSuccess) throw CudaError(std::string("cudaMalloc ") + std::to_string(b) + ": " + cudaGetErrorString(e));
        CK(cudaMemsetAsync(p, 0, b, stream));
        CK(cudaStreamSynchronize(stream));  // usable from any stream from here on
        ptrs.push_back(p);
        bytes += (double)b;
        return (T*)p;
    }
    void release(void* p, size_t b) {
        for (auto& q : ptrs)
            if (q == p) { cudaFreeAsync(p, stream); q = nullptr; bytes -= (double)b; }
    }
    void free_all() {
        for (void* p : ptrs)
            if (p) cudaFreeAsync(p, stream);
        ptrs.clear();
        if (stream) cudaStreamSynchronize(stream);
    }
    static void keep_pool(int device) {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t thr = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
    }
};

// Lays buffers out back to back (256-byte aligned) in one slab.  A layout
// function runs twice: with base 0 to size the slab, then with the slab's base.
struct Carver {
    uintptr_t base = 0;
    size_t off = 0;
    template <typename T>
    T* take(size_t n) {
        off = (off + 255) & ~(size_t)255;
        T* p = (T*)(base + off);
        off += std::max<size_t>(n, 1) * sizeof(T);
        return p;
    }
};

// Pinned host words for the engines' asynchronous flag reads, carved from
// pinned blocks shared by all engines of the process (pinned allocation is
// slow): a 16-word slot per engine, returned to a free list.
struct PinnedSlots {
    std::mutex mu;
    std::vector<int*> free_slots;
    int* get() {
        std::lock_guard<std::mutex> lk(mu);
        if (free_slots.empty()) {
            int* blk = nullptr;
            CK(cudaMallocHost(&blk, 4096 * sizeof(int)));
            for (int k = 0; k < 4096; k += 16) free_slots.push_back(blk + k);
        }
        int* p = free_slots.back();
        free_slots.pop_back();
        return p;
    }
    void put(int* p) {
        std::lock_guard<std::mutex> lk(mu);
        free_slots.push_back(p);
    }
};
static PinnedSlots g_pinned;

// A scene's arrays are checked before anything reaches the device: missing
// arrays, non-finite values, non-positive radii, masses and inertias, clump
// ids and grid levels out of range are argument errors (the reference reads
// its inputs unchecked, src/dem_subsphere_io.cu:151-193).
static void validate_scene(const nbc_scene_desc& D, int s) {
    const std::string at = "scene " + std::to_string(s) + ": ";
    if (D.n_sub <= 0 || D.n_clump <= 0 || !D.pos || !D.radius || !D.clump_id || !D.local || !D.mass ||
        !D.clump_pos || !D.clump_vel || !D.clump_quat || !D.clump_angvel || !D.clump_prop)
        throw ArgError(at + "empty or missing arrays");
    if (!(std::isfinite(D.dt) && D.dt > 0)) throw ArgError(at + "time step not positive");
    if (!(std::isfinite(D.thresh) && D.thresh >= 0)) throw ArgError(at + "Thresh negative or not finite");
    if (D.levels > 1 && (!D.level || !D.level_cell)) throw ArgError(at + "grid levels without level arrays");
    auto fin = [](const double* p, int n) {
        for (int k = 0; k < n; k++)
            if (!std::isfinite(p[k])) return false;
        return true;
    };
    for (int i = 0; i < D.n_sub; i++) {
        if (!fin(D.pos + 3 * i, 3) || !fin(D.local + 3 * i, 3))
            throw ArgError(at + "non-finite position at row " + std::to_string(i));
        if (!(std::isfinite(D.radius[i]) && D.radius[i] > 0) || !(std::isfinite(D.mass[i]) && D.mass[i] > 0))
            throw ArgError(at + "radius or mass not positive at row " + std::to_string(i));
        if (D.clump_id[i] < 0 || D.clump_id[i] >= D.n_clump)
            throw ArgError(at + "clump id out of range at row " + std::to_string(i));
        if (D.levels > 1 && (D.level[i] < 0 || D.level[i] >= D.levels))
            throw ArgError(at + "grid level out of range at row " + std::to_string(i));
    }
    for (int k = 0; k < D.n_clump; k++) {
        const double* q = D.clump_quat + 4 * k;
        const double* pr = D.clump_prop + 4 * k;
        if (!fin(D.clump_pos + 3 * k, 3) || !fin(D.clump_vel + 3 * k, 3) || !fin(D.clump_angvel + 3 * k, 3) ||
            !fin(q, 4) || q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3] == 0)
            throw ArgError(at + "non-finite or zero clump state at clump " + std::to_string(k));
        for (int c = 0; c < 4; c++)
            if (!(std::isfinite(pr[c]) && pr[c] > 0))
                throw ArgError(at + "clump inertia or mass not positive at clump " + std::to_string(k));
    }
    for (int l = 0; D.levels > 1 && l < D.levels; l++)
        if (!(std::isfinite(D.level_cell[l]) && D.level_cell[l] > 0))
            throw ArgError(at + "grid cell size not positive on level " + std::to_string(l));
}

template <typename R>
class EngineT final : public EngineBase {
   public:
    EngineT(const std::vector<const nbc_scene_desc*>& sc, const nbc_options& opt) : opt_(opt) { setup(sc); }
    ~EngineT() override {
        for (int t = 0; t < 3; t++) {
            if (gexec_[t]) cudaGraphExecDestroy(gexec_[t]);
            if (graph_[t]) cudaGraphDestroy(graph_[t]);
        }
        if (gexec_loop_) cudaGraphExecDestroy(gexec_loop_);
        if (graph_loop_) cudaGraphDestroy(graph_loop_);
        for (cudaEvent_t e : ev_) cudaEventDestroy(e);
        for (auto& row : gev_)
            for (cudaEvent_t e : row) if (e) cudaEventDestroy(e);
        if (ev_fork_) cudaEventDestroy(ev_fork_);
        if (ev_join_) cudaEventDestroy(ev_join_);
        mem_.free_all();
        if (stream2_) cudaStreamDestroy(stream2_);
        if (stream_) cudaStreamDestroy(stream_);
        if (hflag_) g_pinned.put(hflag_);
    }

    void step(int n, bool exp) override {
        auto t0 = std::chrono::steady_clock::now();
        int left = n;
        while (left > 0) {
            if (exp && left == 1) {
                clear_post_done();
                run_step_eager(true);
                left -= 1;
                continue;
            }
            enqueue(exp ? left - 1 : left);
            left -= wait_steps();
        }
        CK(cudaStreamSynchronize(stream_));
        check_errors();
        last_ms_ = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }

    // Asynchronous stepping: enqueue puts up to n steps on the engine's
    // stream and returns without waiting for them (an engine's first step,
    // and every step without a graph, runs eagerly before it returns);
    // wait_steps waits, finishes a step that a pair-capacity overflow stopped
    // and returns the number of steps done.  A step after an overflow is not
    // done: the caller enqueues the rest again.
    int enqueue(int n) override {
        clear_post_done();
        pend_ = 0;
        pend_eager_ = 0;
        while (n > 0 && (!opt_.use_graph || steps_done_ < 1)) {
            run_step_eager(false);
            pend_eager_++;
            n--;
        }
        if (n <= 0) return pend_eager_;
        if (timing_ == 0 && !loop_tried_) capture_loop();
        pend_before_ = read_gstep();
        if (timing_ == 0 && gexec_loop_) {
            launch_loop(n);
        } else {
            if (!gexec_[timing_]) capture(timing_);
            for (int i = 0; i < n; i++) launch_graph();
        }
        pend_ = n;
        return pend_eager_ + n;
    }
    int wait_steps() override {
        int done = pend_eager_;
        if (pend_ > 0) {
            CK(cudaStreamSynchronize(stream_));
            const int started = read_gstep() - pend_before_;
            launches_ += (1LL + CONTACT_LAUNCHES) * started + (timing_ == 0 && gexec_loop_ ? 1 : 0);
            if (read_int(h_.halt)) {
                check_scan();
                // the last step started stopped at its rebuild: finish it on the host path
                steps_done_ += started - 1;
                recover_halt();
            } else {
                steps_done_ += started;
            }
            done += started;
        }
        pend_ = pend_eager_ = 0;
        CK(cudaStreamSynchronize(stream_));
        check_errors();
        return done;
    }
    void clear_post_done() {
        if (post_done_) {
            // a sync applied the pending half-kick: the next pass must not repeat it
            CK(cudaMemsetAsync(h_.post_pending, 0, sizeof(int), stream_));
            post_done_ = false;
        }
    }

    void sync() override {
        // apply the pending second half-kick so the state is that of the last step
        int pending = 0;
        CK(cudaStreamSynchronize(stream_));
        copy_(&pending, h_.post_pending, sizeof(int), cudaMemcpyDeviceToHost);
        if (pending && !post_done_) {
            launch_clump(0);
            post_done_ = true;
        }
        CK(cudaStreamSynchronize(stream_));
        refresh_dev();
    }

    // ---- getters ----------------------------------------------------------
    int num_scenes() const override { return S_; }
    void stats(int s, int* steps, int* rebuilds, int* npairs, int* err) override {
        SceneDyn y = read_dyn(s);
        if (steps) *steps = y.step + start_step_[s];
        if (rebuilds) *rebuilds = y.nrebuild;
        if (npairs) *npairs = y.npairs;
        if (err) *err = y.err;
    }
    // near pairs of the current list (the pairs the contact pass visits) and
    // those of them that touched at the last contact pass, over all scenes
    void contact_counts(long long* nnear, long long* ntouch) override {
        refresh_dev();
        const int hg = read_int(h_.hgen);
        std::vector<SceneDyn> y = read_dyn_all();
        std::vector<uint8_t> t(h_.cap);
        copy_(t.data(), h_.touch[(hg + 1) & 1], (size_t)h_.cap, cudaMemcpyDeviceToHost);
        long long n = 0, c = 0;
        for (int s = 0; s < S_; s++) {
            std::vector<int4> rec(y[s].nnear);
            if (y[s].nnear)
                copy_(rec.data(), h_.nfr + y[s].pair_off, (size_t)y[s].nnear * sizeof(int4), cudaMemcpyDeviceToHost);
            for (const int4& e : rec) c += t[e.x] != 0;
            n += y[s].nnear;
        }
        if (nnear) *nnear = n;
        if (ntouch) *ntouch = c;
    }
    void get_subspheres(int s, int* fix, int* cid, double* pos, double* rad) override {
        refresh_dev();
        const ScenePar& P = hpar_[s];
        int n = P.nsub, o = P.sub_off;
        if (fix) {
            copy_(fix, h_.part_fix + o, n * sizeof(int), cudaMemcpyDeviceToHost);
        }
        if (cid) {
            copy_(cid, h_.clump_id + o, n * sizeof(int), cudaMemcpyDeviceToHost);
            for (int i = 0; i < n; i++) cid[i] -= P.clump_off;
        }
        if (pos || rad) {
            std::vector<double4> tmp(n);
            copy_(tmp.data(), h_.posr + o, n * sizeof(double4), cudaMemcpyDeviceToHost);
            for (int i = 0; i < n; i++) {
                if (pos) { pos[3 * i] = tmp[i].x; pos[3 * i + 1] = tmp[i].y; pos[3 * i + 2] = tmp[i].z; }
                if (rad) rad[i] = tmp[i].w;
            }
        }
    }
    void get_body(int s, double* local, double* mass) override {
        refresh_dev();
        const ScenePar& P = hpar_[s];
        std::vector<double4> tmp(P.nsub);
        copy_(tmp.data(), h_.lom + P.sub_off, P.nsub * sizeof(double4), cudaMemcpyDeviceToHost);
        for (int i = 0; i < P.nsub; i++) {
            if (local) { local[3 * i] = tmp[i].x; local[3 * i + 1] = tmp[i].y; local[3 * i + 2] = tmp[i].z; }
            if (mass) mass[i] = tmp[i].w;
        }
    }
    void get_clump_prop(int s, double* prop) override {
        const ScenePar& P = hpar_[s];
        std::vector<double4> tmp(P.nclump);
        copy_(tmp.data(), h_.cprop + P.clump_off, P.nclump * sizeof(double4), cudaMemcpyDeviceToHost);
        for (int i = 0; i < P.nclump; i++) {
            prop[4 * i] = tmp[i].x; prop[4 * i + 1] = tmp[i].y; prop[4 * i + 2] = tmp[i].z; prop[4 * i + 3] = tmp[i].w;
        }
    }
    void get_clumps(int s, double* pos, double* vel, double* quat, double* w, double* f, double* t) override {
        refresh_dev();
        const ScenePar& P = hpar_[s];
        int n = P.nclump, o = P.clump_off;
        std::vector<double4> tmp(n);
        auto pull3 = [&](double4* src, double* dst) {
            if (!dst) return;
            copy_(tmp.data(), src + o, n * sizeof(double4), cudaMemcpyDeviceToHost);
            for (int i = 0; i < n; i++) { dst[3 * i] = tmp[i].x; dst[3 * i + 1] = tmp[i].y; dst[3 * i + 2] = tmp[i].z; }
        };
        pull3(h_.cpos, pos);
        pull3(h_.cvel, vel);
        pull3(h_.cw, w);
        pull3(h_.cF, f);
        pull3(h_.cT, t);
        if (quat) {
            copy_(tmp.data(), h_.cq + o, n * sizeof(double4), cudaMemcpyDeviceToHost);
            for (int i = 0; i < n; i++) {
                quat[4 * i] = tmp[i].x; quat[4 * i + 1] = tmp[i].y; quat[4 * i + 2] = tmp[i].z; quat[4 * i + 3] = tmp[i].w;
            }
        }
    }
    void get_sub_forces(int s, double* f, double* t) override {
        refresh_dev();
        launch_sum(false);
        const ScenePar& P = hpar_[s];
        pull_r4(h_.fsum, P.sub_off, P.nsub, f);
        pull_r4((char*)h_.fsum + (size_t)N_ * sizeof(R4<R>), P.sub_off, P.nsub, t);
    }
    void get_force_parts(int s, double* parts) override {
        refresh_dev();
        const ScenePar& P = hpar_[s];
        for (int c = 0; c < 6; c++)
            pull_r4((char*)h_.xparts + (size_t)c * N_ * sizeof(R4<R>), P.sub_off, P.nsub, parts + (size_t)c * P.nsub * 3);
    }
    void get_intruder_diag(int s, double* diag) override {
        refresh_dev();
        const ScenePar& P = hpar_[s];
        for (int c = 0; c < 4; c++)
            pull_r4((char*)h_.xintr + (size_t)c * N_ * sizeof(R4<R>), P.sub_off, P.nsub, diag + (size_t)c * P.nsub * 3);
    }
    void get_pairs(int s, int* np, int* lpa, int* lpb) override {
        refresh_dev();
        SceneDyn y = read_dyn(s);
        const ScenePar& P = hpar_[s];
        int cap_in = *np;
        *np = y.npairs;
        if (!lpa && !lpb) return;
        if (cap_in < y.npairs) throw ArgError("pair buffer too small");
        int lc = read_int(h_.lcur);
        const PairList& Lc = h_.L[lc & 1];
        std::vector<int> own(y.npairs), nbr(y.npairs);
        copy_(own.data(), Lc.own + y.pair_off, y.npairs * sizeof(int), cudaMemcpyDeviceToHost);
        copy_(nbr.data(), Lc.nbr + y.pair_off, y.npairs * sizeof(int), cudaMemcpyDeviceToHost);
        for (int p = 0; p < y.npairs; p++) {
            if (lpa) lpa[p] = own[p] - P.sub_off;
            if (lpb) lpb[p] = (nbr[p] & IDX_MASK) - P.sub_off;
        }
    }
    // the reference's pitched rows (Anei, src/dem_grid.cu:466-552)
    void get_rows(int s, int bl, int* anei, int* ng, int* ni) override {
        RowData rd = pull_rows(s);
        const ScenePar& P = hpar_[s];
        const int n = P.nsub;
        if (anei) std::fill(anei, anei + (size_t)n * bl, -1);
        for (int i = 0; i < n; i++) {
            int nf = rd.row[i + 1] - rd.row[i], nb = rd.brow[i + 1] - rd.brow[i];
            if (ng) ng[i] = nf;
            if (ni) ni[i] = nb;
            if (!anei) continue;
            if (nf > bl / 2 || nb > bl / 2) throw ArgError("row longer than bl/2");
            for (int g = 0; g < nf; g++) anei[(size_t)i * bl + g] = (rd.nbr[rd.row[i] - rd.row[0] + g] & IDX_MASK) - P.sub_off;
            for (int c = 0; c < nb; c++)
                anei[(size_t)i * bl + bl - 1 - c] = (rd.bnbr[rd.brow[i] - rd.brow[0] + c] & IDX_MASK) - P.sub_off;
        }
    }
    // CalFcnChain_cuk (src/dem_force_particle.cu:238-268) on the export data
    void get_chain(int s, int bl, double* fcn, double* cpt) override {
        RowData rd = pull_rows(s);
        const ScenePar& P = hpar_[s];
        const int n = P.nsub;
        SceneDyn y = read_dyn(s);
        std::vector<R4<R>> xf(y.npairs);
        std::vector<double4> xc(y.npairs);
        copy_(xf.data(), (R4<R>*)h_.xfcn + y.pair_off, y.npairs * sizeof(R4<R>), cudaMemcpyDeviceToHost);
        copy_(xc.data(), (double4*)h_.xcpt + y.pair_off, y.npairs * sizeof(double4), cudaMemcpyDeviceToHost);
        std::fill(fcn, fcn + (size_t)n * bl * 3, 0.0);
        std::fill(cpt, cpt + (size_t)n * bl * 3, 0.0);
        const int p0 = rd.row[0];
        for (int i = 0; i < n; i++) {
            for (int g = 0; g < rd.row[i + 1] - rd.row[i]; g++) {
                int p = rd.row[i] - p0 + g;
                double* F = fcn + ((size_t)i * bl + g) * 3;
                double* C = cpt + ((size_t)i * bl + g) * 3;
                if (rd.nbr[p] < 0) continue;
                F[0] = xf[p].x; F[1] = xf[p].y; F[2] = xf[p].z;
                C[0] = xc[p].x; C[1] = xc[p].y; C[2] = xc[p].z;
            }
            for (int c = 0; c < rd.brow[i + 1] - rd.brow[i]; c++) {
                int k = rd.brow[i] - rd.brow[0] + c;
                if (rd.bnbr[k] < 0) continue;
                int p = rd.bpair[k] - y.pair_off;
                double* F = fcn + ((size_t)i * bl + bl - 1 - c) * 3;
                double* C = cpt + ((size_t)i * bl + bl - 1 - c) * 3;
                F[0] = -(double)xf[p].x; F[1] = -(double)xf[p].y; F[2] = -(double)xf[p].z;
                C[0] = xc[p].x; C[1] = xc[p].y; C[2] = xc[p].z;
            }
        }
    }
    // the normal force on the owner of every listed pair, list order (the
    // reference's CacheFcn, src/dem_force_clump.cu:114-116), from the export
    // step; zero for pairs that do not touch
    void get_pair_forces(int s, int* np, double* fcn) override {
        refresh_dev();
        SceneDyn y = read_dyn(s);
        const int cap_in = *np;
        *np = y.npairs;
        if (!fcn) return;
        if (cap_in < y.npairs) throw ArgError("pair buffer too small");
        std::vector<R4<R>> xf(y.npairs);
        copy_(xf.data(), (R4<R>*)h_.xfcn + y.pair_off, y.npairs * sizeof(R4<R>), cudaMemcpyDeviceToHost);
        for (int p = 0; p < y.npairs; p++) {
            fcn[3 * p] = xf[p].x; fcn[3 * p + 1] = xf[p].y; fcn[3 * p + 2] = xf[p].z;
        }
    }
    void get_intruder(int s, double* pos, double* vel, double* reac, double* tq, int* state) override {
        SceneDyn y = read_dyn(s);
        for (int c = 0; c < 3; c++) {
            if (pos) pos[c] = y.intr_p[c];
            if (vel) vel[c] = y.intr_v[c];
            if (reac) reac[c] = y.reaction[c];
            if (tq) tq[c] = y.reaction_t[c];
        }
        if (state) *state = y.intr_state;
    }
    void get_intruder_history(int s, int count, double* out) override {
        SceneDyn y = read_dyn(s);
        if (count > ring_len_) throw ArgError("history longer than the ring");
        std::vector<double> ring((size_t)ring_len_ * 6);
        copy_(ring.data(), h_.ring + (size_t)s * ring_len_ * 6, ring.size() * sizeof(double),
                      cudaMemcpyDeviceToHost);
        for (int c = 0; c < count; c++) {
            int st = y.step - count + c;
            if (st < 0) { for (int q = 0; q < 6; q++) out[c * 6 + q] = 0; continue; }
            int slot = st % ring_len_;
            for (int q = 0; q < 6; q++) out[c * 6 + q] = ring[(size_t)slot * 6 + q];
        }
    }
    void timing_enable(int level) override {
        CK(cudaStreamSynchronize(stream_));
        timing_ = level <= 0 ? 0 : (level == 1 ? 1 : 2);
        for (double& v : t_phase_ms_) v = 0;
        t_contact_n_ = 0;
        launches_ = 0;
        rebuilds_at_enable_ = total_rebuilds();
        ev_used_ = 0;
    }
    void timing_read(double* ms, int* nc, long long* nk, int* nr) override {
        CK(cudaStreamSynchronize(stream_));
        harvest_events();
        if (ms) *ms = t_phase_ms_[PH_CONTACT];
        if (nc) *nc = t_contact_n_;
        if (nk) *nk = launches_ + (long long)(total_rebuilds() - rebuilds_at_enable_) * rebuild_launches();
        if (nr) *nr = total_rebuilds() - rebuilds_at_enable_;
    }
    void timing_phases(double* ms) override {
        CK(cudaStreamSynchronize(stream_));
        harvest_events();
        for (int k = 0; k < NPH; k++) ms[k] = t_contact_n_ ? t_phase_ms_[k] / t_contact_n_ : 0.0;
    }
    // scene s stands still after nsteps steps counted from the engine's creation
    void set_stop(int s, int nsteps) override {
        if (s < 0 || s >= S_) throw ArgError("scene index out of range");
        if (nsteps < 0) throw ArgError("scene step count is negative");
        const int started = read_int(h_.lstep);
        if (nsteps != 0 && nsteps < started)
            throw ArgError("scene " + std::to_string(s) + " has started " + std::to_string(started) + " steps already");
        SceneDyn y = read_dyn(s);
        y.stop = nsteps;
        copy_(h_.dyn + s, &y, sizeof(SceneDyn), cudaMemcpyHostToDevice);
        if (nsteps && !h_.has_stops) {
            refresh_dev();
            h_.has_stops = 1;
            push_dev();
        }
    }
    // ---- exact checkpoint -------------------------------------------------
    // The state a step leaves for the next one, after nbc_sync (the pending
    // half-kick applied): every scene's bookkeeping (SceneDyn: steps, intruder
    // state, pair region, step limit), the history generation and step
    // counters, every subsphere in the current sort order (position and
    // radius, body offset and mass, displacement since the last rebuild,
    // clump, original index, grid level, cell key, contact kinematics, wall
    // and intruder spring histories and their contact bits, boundary
    // candidates), every clump's state and member list, and each scene's
    // pair region: the current half list with its back references, spring
    // histories and touch flags, the near rows and their contact slots, and
    // the intruder force ring.  Rebuild scratch is not saved: a rebuild
    // writes it before reading it.  Loading this into an engine made from
    // the same scenes and options and stepping on gives bitwise the run that
    // never stopped (the reference restarts from StartStep, src/world.par:28
    // and src/dem_simulation_clump.cu:110, with its spring histories lost).
    struct CkHeader {
        char magic[8];
        int version, S, N, K, cells, real_bytes, steps_done, hgen, gstep, lstep, ring_len;
        long long total_cap;
    };
    std::vector<char> checkpoint_save() override {
        if (steps_done_ < 1) throw StateError("checkpoint before the first step (there is no list yet)");
        sync();
        refresh_dev();
        CkHeader hd{};
        memcpy(hd.magic, "NBCCKPT", 8);
        hd.version = 1;
        hd.S = S_; hd.N = N_; hd.K = K_; hd.cells = h_.cells;
        hd.real_bytes = (int)sizeof(R);
        hd.steps_done = steps_done_;
        hd.hgen = read_int(h_.hgen);
        hd.gstep = read_int(h_.gstep);
        hd.lstep = read_int(h_.lstep);
        hd.ring_len = ring_len_;
        hd.total_cap = h_.cap;
        std::vector<char> out((const char*)&hd, (const char*)&hd + sizeof(hd));
        ck_blocks(out, nullptr, 0, hd);
        return out;
    }
    void checkpoint_load(const char* data, size_t bytes) override {
        if (bytes < sizeof(CkHeader)) throw ArgError("checkpoint too short");
        CkHeader hd;
        memcpy(&hd, data, sizeof(hd));
        if (memcmp(hd.magic, "NBCCKPT", 8) != 0 || hd.version != 1) throw ArgError("not an engine checkpoint");
        if (hd.S != S_ || hd.N != N_ || hd.K != K_ || hd.cells != h_.cells || hd.ring_len != ring_len_)
            throw ArgError("checkpoint of different scenes");
        if (hd.real_bytes != (int)sizeof(R)) throw ArgError("checkpoint of the other precision");
        if (bytes < sizeof(hd) + S_ * sizeof(SceneDyn)) throw ArgError("checkpoint too short");
        CK(cudaStreamSynchronize(stream_));
        // pair regions as saved (their sizes are in the saved SceneDyn)
        refresh_dev();
        mem_.release(pslab_, pslab_bytes_);
        alloc_pairs(std::max<long long>(hd.total_cap, 1));
        push_dev();
        std::vector<char> in(data, data + bytes);
        ck_blocks(in, &in, sizeof(hd), hd);
        steps_done_ = hd.steps_done;
        first_list_ = false;
        post_done_ = false;
        pend_ = pend_eager_ = 0;
        bool stops = false;
        for (const SceneDyn& v : read_dyn_all()) stops |= v.stop != 0;
        if (stops && !h_.has_stops) {
            h_.has_stops = 1;
            push_dev();
        }
        CK(cudaStreamSynchronize(stream_));
    }
    // Writes (src == nullptr: appends to out) or reads (from src at offset
    // off) the checkpoint's blocks in one fixed order.
    void ck_blocks(std::vector<char>& out, const std::vector<char>* src, size_t off, const CkHeader& hd) {
        const size_t N = N_;
        auto blk = [&](void* dev, size_t n) {
            if (!n) return;
            if (!src) {
                const size_t at = out.size();
                out.resize(at + n);
                copy_(out.data() + at, dev, n, cudaMemcpyDeviceToHost);
            } else {
                if (off + n > src->size()) throw ArgError("checkpoint truncated");
                copy_(dev, src->data() + off, n, cudaMemcpyHostToDevice);
                off += n;
            }
        };
        // scene bookkeeping first (its pair regions size the rest)
        blk(h_.dyn, S_ * sizeof(SceneDyn));
        std::vector<SceneDyn> y = read_dyn_all();
        // counters; the pending half-kick was applied by sync, so the next
        // step must not repeat it (post_pending saved as 0)
        int flags[4] = {hd.hgen, hd.gstep, hd.lstep, 0};
        if (!src) {
            const size_t at = out.size();
            out.resize(at + sizeof(flags));
            memcpy(out.data() + at, flags, sizeof(flags));
        } else {
            if (off + sizeof(flags) > src->size()) throw ArgError("checkpoint truncated");
            memcpy(flags, src->data() + off, sizeof(flags));
            off += sizeof(flags);
            copy_(h_.hgen, &flags[0], sizeof(int), cudaMemcpyHostToDevice);
            copy_(h_.gstep, &flags[1], sizeof(int), cudaMemcpyHostToDevice);
            copy_(h_.lstep, &flags[2], sizeof(int), cudaMemcpyHostToDevice);
            copy_(h_.post_pending, &flags[3], sizeof(int), cudaMemcpyHostToDevice);
            int zero = 0;
            copy_(h_.any_rebuild, &zero, sizeof(int), cudaMemcpyHostToDevice);
            copy_(h_.halt, &zero, sizeof(int), cudaMemcpyHostToDevice);
            copy_(h_.lcur, &zero, sizeof(int), cudaMemcpyHostToDevice);
            copy_(h_.kc_done, &zero, sizeof(int), cudaMemcpyHostToDevice);
        }
        // subspheres, current sort order
        blk(h_.posr, N * sizeof(double4));
        blk(h_.lom, N * sizeof(double4));
        blk(h_.cum, N * sizeof(double4));
        blk(h_.clump_id, N * sizeof(int));
        blk(h_.part_fix, N * sizeof(int));
        blk(h_.level, N * sizeof(int));
        blk(h_.key, N * sizeof(int));
        blk(h_.kin, N * sizeof(double4));
        blk(h_.bhist, (size_t)NB_SLOTS * 3 * N * sizeof(R4<R>));
        blk(h_.bbits, N * sizeof(uint16_t));
        blk(h_.fbnd, 2 * N * sizeof(R4<R>));
        if (h_.fint) blk(h_.fint, 2 * N * sizeof(R4<R>));
        blk(h_.bidx, N * sizeof(int));
        // clumps
        blk(h_.cpos, K_ * sizeof(double4));
        blk(h_.cvel, K_ * sizeof(double4));
        blk(h_.cw, K_ * sizeof(double4));
        blk(h_.cq, K_ * sizeof(double4));
        blk(h_.cprop, K_ * sizeof(double4));
        blk(h_.cinv, K_ * sizeof(double4));
        blk(h_.mem_cl, N * sizeof(int));
        blk(h_.cF, K_ * sizeof(double4));
        blk(h_.cT, K_ * sizeof(double4));
        blk(h_.mem_start, (K_ + 1) * sizeof(int));
        blk(h_.mem_idx, N * sizeof(int));
        // rows and work-item prefixes
        blk(h_.L[0].row, (N + S_) * sizeof(int));
        blk(h_.L[0].brow, (N + S_) * sizeof(int));
        blk(h_.nrb, (N + S_) * sizeof(int2));
        blk(h_.nprefix, (S_ + 1) * sizeof(int));
        blk(h_.bprefix, (S_ + 1) * sizeof(int));
        blk(h_.ring, (size_t)S_ * ring_len_ * 6 * sizeof(double));
        // each scene's pair region: the history generation the next contact
        // pass reads is (hgen + 1) & 1 (k_clump advances hgen first)
        const int g = (hd.hgen + 1) & 1;
        const size_t cap = h_.cap;
        for (int s = 0; s < S_; s++) {
            const size_t o = y[s].pair_off, np = y[s].npairs, nn = y[s].nnear;
            blk(h_.L[0].nbr + o, np * sizeof(int));
            blk(h_.L[0].own + o, np * sizeof(int));
            blk(h_.L[0].bnbr + o, np * sizeof(int));
            blk(h_.L[0].bpair + o, np * sizeof(int));
            R4<R>* H = (R4<R>*)h_.H[g];
            blk(H + 2 * o, 2 * np * sizeof(R4<R>));
            blk((R*)(H + 2 * cap) + o, np * sizeof(R));
            blk(h_.touch[g] + o, np);
            blk(h_.nearf + o, np);
            blk(h_.nbpos + o, np * sizeof(int));
            blk(h_.nfr + o, nn * sizeof(int4));
            blk(h_.nbq + o, nn * sizeof(int));
            R4<R>* fs = (R4<R>*)h_.nfs;
            R4<R>* bs = (R4<R>*)h_.nbs;
            blk(fs + 2 * o, 2 * nn * sizeof(R4<R>));
            blk(bs + 2 * o, 2 * nn * sizeof(R4<R>));
        }
        if (src && off != src->size()) throw ArgError("checkpoint has trailing bytes");
    }
    void launch_info(int* step_loop, int* search_lanes, int* clump_batch, int* pair_blocks) override {
        if (step_loop) {
            if (opt_.use_graph && !loop_tried_) capture_loop();
            *step_loop = gexec_loop_ ? 1 : 0;
        }
        if (search_lanes) *search_lanes = search_lanes_;
        if (clump_batch) *clump_batch = clump_batch_;
        if (pair_blocks) *pair_blocks = pair_bps_;
    }
    void info(double* bytes, double* ms) override {
        if (bytes) *bytes = mem_.bytes;
        if (ms) *ms = last_ms_;
    }

   private:
    nbc_options opt_;
    DevMem mem_;
    char* pslab_ = nullptr;  // the pair buffers' slab
    int4* relmap_ = nullptr; // [S] region moves of a re-layout
    size_t pslab_bytes_ = 0;
    cudaStream_t stream_ = nullptr;
    cudaStream_t stream2_ = nullptr;   // second branch of a step: k_boundary beside k_pairs
    cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr;
    Dev h_{};            // host copy of the device table
    Dev* d_ = nullptr;   // device table
    int S_ = 0, N_ = 0, K_ = 0;
    bool hgrid_ = false;
    bool sphere_any_ = false;   // some scene runs a sphere driver's behaviour (the clump pass's SPH build)
    bool sphere_kin_ = false;   // some scene runs the sphere drivers' kinematics (Dev::fint)
    bool has_kinds_ = false;    // some scene has split-driver body kinds (Dev::kind)
    bool first_list_ = true;
    int search_lanes_ = 8;
    int clump_batch_ = 1;    // members per lane per load batch of the clump pass
    int pair_bps_ = 12;      // blocks per SM of the pair kernel's grid
    int sm_count_ = 148;
    int ring_len_ = 1;
    std::vector<ScenePar> hpar_;
    std::vector<int> start_step_;
    int* hflag_ = nullptr;  // pinned
    int steps_done_ = 0;
    int pend_ = 0, pend_eager_ = 0, pend_before_ = 0;  // steps enqueued and not yet waited for
    bool post_done_ = false;
    double last_ms_ = 0;
    // step graphs by timing level: [0] plain, [1] event nodes around the
    // contact pass (k_pairs + k_sum), [2] event nodes at every mark
    cudaGraph_t graph_[3] = {nullptr, nullptr, nullptr};
    cudaGraphExec_t gexec_[3] = {nullptr, nullptr, nullptr};
    // the untimed graph with a device-side step loop (capture_loop)
    cudaGraph_t graph_loop_ = nullptr;
    cudaGraphExec_t gexec_loop_ = nullptr;
    cudaGraphNode_t loop_init_node_ = nullptr;
    bool loop_tried_ = false;
    std::string loop_error_;
    // kernel timing: one record of NMARK events per step, at the marks
    //   0 step start  1 after k_clump  2 after the rebuild node
    //   3/4 around k_boundary and 5 start of the contact pass (second branch)
    //   6 end of the contact pass (after k_sum)  7 step end
    static constexpr int NMARK = 8;
    static constexpr int PH_CLUMP = 0, PH_REBUILD = 1, PH_BOUNDARY = 2, PH_CONTACT = 3, PH_STEP = 4, NPH = 5;
    int timing_ = 0;
    double t_phase_ms_[NPH] = {0, 0, 0, 0, 0};
    int t_contact_n_ = 0;
    long long launches_ = 0;
    int rebuilds_at_enable_ = 0;
    std::vector<cudaEvent_t> ev_;   // records of NMARK events
    int ev_used_ = 0;               // records made and not yet harvested
    cudaEvent_t* rec_ = nullptr;    // the record being made by an eager step (null: none)
    int capture_timed_ = 0;
    cudaEvent_t gev_[3][NMARK] = {};
    cudaGraphNode_t gev_node_[3][NMARK] = {};

    int total_rebuilds() {
        std::vector<SceneDyn> y(S_);
        copy_(y.data(), h_.dyn, S_ * sizeof(SceneDyn), cudaMemcpyDeviceToHost);
        int n = 0;
        for (auto& v : y) n = std::max(n, v.nrebuild);
        return n;
    }
    // kernels one rebuild launches (launch_rebuild)
    // kernels of one rebuild in a graph (the eager path adds a k_check_cap):
    // plan, hash, the cell counts' scan, scatter, per-cell order and table,
    // reorder, search, scan, check, compact, (hgrid: xsort), backref, carry,
    // write-back, 2 near-row passes and their scan, the finishing pass
    int rebuild_launches() const { return 17 + (hgrid_ ? 1 : 0); }
    cudaEvent_t* next_record() {
        if ((size_t)(NMARK * (ev_used_ + 1)) > ev_.size()) {
            for (int k = 0; k < 64 * NMARK; k++) {
                cudaEvent_t e;
                CK(cudaEventCreate(&e));
                ev_.push_back(e);
            }
        }
        return &ev_[(size_t)NMARK * ev_used_++];
    }
    // marks recorded at timing level 1: only those around the contact pass
    static bool mark_on(int level, int k) { return level >= 2 || (level == 1 && (k == 5 || k == 6)); }
    void harvest_events() {
        for (int k = 0; k < ev_used_; k++) {
            const cudaEvent_t* e = &ev_[(size_t)NMARK * k];
            float ms[NPH] = {0, 0, 0, 0, 0};
            CK(cudaEventElapsedTime(&ms[PH_CONTACT], e[5], e[6]));
            if (timing_ >= 2) {
                CK(cudaEventElapsedTime(&ms[PH_CLUMP], e[0], e[1]));
                CK(cudaEventElapsedTime(&ms[PH_REBUILD], e[1], e[2]));
                CK(cudaEventElapsedTime(&ms[PH_BOUNDARY], e[3], e[4]));
                CK(cudaEventElapsedTime(&ms[PH_STEP], e[0], e[7]));
            }
            for (int p = 0; p < NPH; p++) t_phase_ms_[p] += ms[p];
            t_contact_n_++;
        }
        ev_used_ = 0;
    }
    // a timing mark on stream st: an event node while capturing a timed
    // graph, an event of the current record on an eager step
    void mark(int k, cudaStream_t st) {
        if (capturing_) {
            if (!mark_on(capture_timed_, k)) return;
            CK(cudaEventRecordWithFlags(gev_[capture_timed_][k], st, cudaEventRecordExternal));
            gev_node_[capture_timed_][k] = last_captured_node(st);
        } else if (rec_ && mark_on(timing_, k)) {
            CK(cudaEventRecord(rec_[k], st));
        }
    }

    struct RowData { std::vector<int> row, brow, nbr, bnbr, bpair; };

    // ---- setup --------------------------------------------------------------
    void setup(const std::vector<const nbc_scene_desc*>& sc) {
        for (size_t s = 0; s < sc.size(); s++) validate_scene(*sc[s], (int)s);
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw CudaError("no CUDA device");
        CK(cudaSetDevice(opt_.device));
        CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&stream2_, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming));
        hflag_ = g_pinned.get();
        mem_.stream = stream_;
        DevMem::keep_pool(opt_.device);
        search_lanes_ = opt_.search_lanes == 16 || opt_.search_lanes == 32 ? opt_.search_lanes : 8;
        clump_batch_ = opt_.clump_batch == 2 || opt_.clump_batch == 4 ? opt_.clump_batch : 1;
        // the clump pass's staged contact records (dynamic shared memory past the 48 KB default)
        CK(cudaFuncSetAttribute(k_clump<R, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)clump_dyn_smem<R, 1>()));
        CK(cudaFuncSetAttribute(k_clump<R, 2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)clump_dyn_smem<R, 2>()));
        CK(cudaFuncSetAttribute(k_clump<R, 4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)clump_dyn_smem<R, 4>()));
        CK(cudaFuncSetAttribute(k_clump<R, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)clump_dyn_smem<R, 1>()));
        CK(cudaFuncSetAttribute(k_clump<R, 2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)clump_dyn_smem<R, 2>()));
        CK(cudaFuncSetAttribute(k_clump<R, 4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)clump_dyn_smem<R, 4>()));
        pair_bps_ = opt_.pair_blocks >= 2 && opt_.pair_blocks <= 16 ? opt_.pair_blocks : 12;
        CK(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, opt_.device));
        S_ = (int)sc.size();
        hpar_.resize(S_);
        start_step_.resize(S_);
        std::vector<SceneDyn> hdyn(S_);
        int cells = 0;
        for (int s = 0; s < S_; s++) {
            const nbc_scene_desc& D = *sc[s];
            if (D.n_sub <= 0 || D.n_clump <= 0 || !D.pos || !D.radius || !D.clump_id)
                throw ArgError("scene " + std::to_string(s) + ": empty or missing arrays");
            ScenePar& P = hpar_[s];
            memset(&P, 0, sizeof(P));
            P.dt = D.dt; P.E = D.ymod; P.nu = D.prat; P.mu = D.frcoe; P.gravity = D.gravity;
            P.beta = D.beta; P.cohesion = D.cohesion; P.thresh = D.thresh;
            // LoadParameters (src/dem_subsphere_io.cu:143-145)
            const double lnCOR = std::log(D.normres), PI_REF = 3.14159265359;
            P.damping = 2.0 * std::sqrt(5.0 / 6.0) * lnCOR / std::sqrt(lnCOR * lnCOR + PI_REF * PI_REF);
            P.kn_fac = 2.0 * D.ymod / (3.0 * (1.0 - D.prat * D.prat));
            P.ks_fac = 2.0 * D.ymod / (1.0 + D.prat) / (2.0 - D.prat);
            P.bl = D.branch_len > 0 ? D.branch_len : 256;
            // SetMeshSize (src/dem_subsphere_io.cu:195-230)
            double rmax = 0;
            for (int i = 0; i < D.n_sub; i++) rmax = std::max(rmax, D.radius[i]);
            const double mesh = 3.0 * rmax;
            for (int a = 0; a < 3; a++) {
                P.cell[a] = mesh;
                P.icell[a] = 1.0 / mesh;
                P.origin[a] = D.world_origin[a] - mesh;
                double ws = D.world_size[a] + 2 * mesh;
                P.gdim[a] = (int)(unsigned)std::ceil(ws / mesh);
                P.box_lo[a] = D.box_lo[a];
                P.box_hi[a] = D.box_hi[a];
            }
            P.levels = D.levels > 1 ? D.levels : 1;
            if (P.levels > 1) hgrid_ = true;
            if (P.levels > MAX_LEVELS) throw ArgError("too many grid levels");
            if (P.levels == 1) {
                P.cellnum = P.gdim[0] * P.gdim[1] * P.gdim[2];
            } else {
                int off = 0;
                for (int l = 0; l < P.levels; l++) {
                    P.lcell[l] = D.level_cell[l];
                    for (int a = 0; a < 3; a++)
                        P.ldim[l][a] = (int)std::ceil((D.world_size[a] + 2 * mesh) / P.lcell[l]);
                    P.loff[l] = off;
                    off += P.ldim[l][0] * P.ldim[l][1] * P.ldim[l][2];
                }
                P.cellnum = off + 1;
            }
            P.cell_off = cells;
            cells += P.cellnum;
            P.sub_off = N_;
            P.nsub = D.n_sub;
            P.clump_off = K_;
            P.nclump = D.n_clump;
            N_ += D.n_sub;
            K_ += D.n_clump;
            // walls
            P.wall = D.is_wall_force ? D.wall : WALL_NONE;
            if (P.wall == WALL_CUBE) {
                for (int a = 0; a < 3; a++) {
                    P.w_half[a] = D.cube_half[a]; P.w_c[a] = D.cube_centre[a];
                    P.w_v[a] = D.cube_vel[a]; P.w_w[a] = D.cube_angvel[a];
                }
            } else if (P.wall == WALL_CYL) {
                P.cyl_R = D.cyl_radius; P.cyl_H = D.cyl_half_height;
                for (int a = 0; a < 3; a++) {
                    P.cyl_axis[a] = D.cyl_axis[a]; P.w_c[a] = D.cyl_centre[a];
                    P.w_v[a] = D.cyl_vel[a]; P.w_w[a] = D.cyl_angvel[a];
                }
            }
            SceneDyn& Y = hdyn[s];
            memset(&Y, 0, sizeof(Y));
            Y.rebuild = 1;  // the first step always builds the list (src/dem_simulation_clump.cu:124)
            P.has_intr = D.intruder == NBC_INTR_SPHERE || D.intruder == NBC_INTR_CYLINDER;
            if (P.has_intr) {
                P.intr_shape = D.intruder;
                P.intr_motion = D.intr_motion == NBC_MOTION_CONSTANT_VELOCITY ? 0 : 1;
                P.intr_wait = D.intr_motion == NBC_MOTION_GRAVITY_AFTER_CONTACT;
                P.intr_R = D.intr_radius;
                P.intr_H = D.intruder == NBC_INTR_SPHERE ? D.intr_radius : D.intr_half_height;
                for (int a = 0; a < 3; a++) {
                    P.intr_axis[a] = D.intr_axis[a];
                    P.intr_w[a] = D.intr_angvel[a];
                    Y.intr_p[a] = D.intr_pos[a];
                    Y.intr_v[a] = D.intr_vel[a];
                }
                P.intr_mass = D.intr_prop[3];
            }
            // the reference's sphere-only drivers (class DEMmain)
            if (D.sphere_mode & ~(NBC_SPHERE_KINEMATICS | NBC_SPHERE_CUBE_WALL | NBC_SPHERE_RESET_HISTORY))
                throw ArgError("scene " + std::to_string(s) + ": unknown sphere_mode bits");
            P.sphere = D.sphere_mode | (D.body_kind ? SPH_KINDS : 0);
            if (P.sphere) {
                // one-sphere clumps with the member at the centre: the clump
                // kinematics are then the sphere kinematics
                if (D.n_sub != D.n_clump)
                    throw ArgError("scene " + std::to_string(s) + ": sphere drivers need one subsphere per clump");
                std::vector<char> seen(D.n_clump, 0);
                for (int i = 0; i < D.n_sub; i++) {
                    const int c = D.clump_id[i];
                    if (c < 0 || c >= D.n_clump || seen[c] || D.local[3 * i] != 0.0 || D.local[3 * i + 1] != 0.0 ||
                        D.local[3 * i + 2] != 0.0)
                        throw ArgError("scene " + std::to_string(s) +
                                       ": sphere drivers need one subsphere per clump at its centre (LocalPos = 0)");
                    seen[c] = 1;
                }
            }
            if (P.sphere) sphere_any_ = true;
            if (P.sphere & SPH_KIN) sphere_kin_ = true;
            if (P.sphere & SPH_KINDS) {
                for (int k = 0; k < D.n_clump; k++)
                    if (D.body_kind[k] < 0 || D.body_kind[k] > 2)
                        throw ArgError("scene " + std::to_string(s) + ": body kind out of range at clump " +
                                       std::to_string(k));
                has_kinds_ = true;
                // bodies of kind 1 move without triggering a rebuild: every
                // listed pair stays in the contact pass (near margin unbounded)
                P.thresh = 1e100;
            }
            start_step_[s] = D.start_step;
            ring_len_ = std::max(ring_len_, std::max(1, D.output_interval));
        }
        ring_len_ = std::max(ring_len_, 1024);
        // list entries keep two flag bits above the subsphere index
        if ((long long)N_ >= (1LL << 30)) throw ArgError("more than 2^30 subspheres in one engine");
        h_.S = S_; h_.N = N_; h_.K = K_;
        h_.cells = cells;

        // host arrays in the input order
        std::vector<double4> posr(N_), lom(N_);
        std::vector<int> cid(N_), fix(N_), lev(N_, 0), sid(N_), csid(K_), mstart(K_ + 1, 0), midx(N_);
        std::vector<double4> cpos(K_), cvel(K_), cw(K_), cq(K_), cprop(K_);
        std::vector<int> kind(has_kinds_ ? K_ : 0, 0);
        for (int s = 0; s < S_; s++) {
            const nbc_scene_desc& D = *sc[s];
            const ScenePar& P = hpar_[s];
            for (int i = 0; i < D.n_sub; i++) {
                int g = P.sub_off + i;
                if (D.clump_id[i] < 0 || D.clump_id[i] >= D.n_clump)
                    throw ArgError("scene " + std::to_string(s) + ": clump id out of range at row " + std::to_string(i));
                posr[g] = make_double4(D.pos[3 * i], D.pos[3 * i + 1], D.pos[3 * i + 2], D.radius[i]);
                lom[g] = make_double4(D.local[3 * i], D.local[3 * i + 1], D.local[3 * i + 2], D.mass[i]);
                cid[g] = P.clump_off + D.clump_id[i];
                fix[g] = i;
                sid[g] = s;
                if (P.levels > 1) {
                    if (D.level[i] < 0 || D.level[i] >= P.levels)
                        throw ArgError("scene " + std::to_string(s) + ": grid level out of range at row " + std::to_string(i));
                    lev[g] = D.level[i];
                }
                mstart[cid[g] + 1]++;
            }
            for (int k = 0; k < D.n_clump; k++) {
                int g = P.clump_off + k;
                csid[g] = s;
                cpos[g] = make_double4(D.clump_pos[3 * k], D.clump_pos[3 * k + 1], D.clump_pos[3 * k + 2], 0);
                cvel[g] = make_double4(D.clump_vel[3 * k], D.clump_vel[3 * k + 1], D.clump_vel[3 * k + 2], 0);
                cw[g] = make_double4(D.clump_angvel[3 * k], D.clump_angvel[3 * k + 1], D.clump_angvel[3 * k + 2], 0);
                cq[g] = make_double4(D.clump_quat[4 * k], D.clump_quat[4 * k + 1], D.clump_quat[4 * k + 2], D.clump_quat[4 * k + 3]);
                cprop[g] = make_double4(D.clump_prop[4 * k], D.clump_prop[4 * k + 1], D.clump_prop[4 * k + 2], D.clump_prop[4 * k + 3]);
                // bits 0-1: Type; bits 2-3: the kind the split driver's first
                // half-kick sees, the body's original index (0, 1, 2, or 3 for
                // any larger index; see k_clump)
                if (has_kinds_ && D.body_kind) kind[g] = D.body_kind[k] | (std::min(k, 3) << 2);
            }
        }
        for (int k = 0; k < K_; k++) mstart[k + 1] += mstart[k];
        {
            std::vector<int> cur(mstart.begin(), mstart.end() - 1);
            for (int i = 0; i < N_; i++) midx[cur[cid[i]]++] = i;
        }

        // device allocation: the per-subsphere and per-clump buffers in one
        // slab, the pair buffers (which grow) in another
        const size_t N = N_;
        auto layout = [&](Carver& m) {
            h_.par = m.take<ScenePar>(S_);
            h_.dyn = m.take<SceneDyn>(S_);
            h_.sid = m.take<int>(N);
            h_.csid = m.take<int>(K_);
            h_.posr = m.take<double4>(N); h_.posr2 = m.take<double4>(N);
            h_.lom = m.take<double4>(N); h_.lom2 = m.take<double4>(N);
            h_.cum = m.take<double4>(N); h_.cum2 = m.take<double4>(N);
            h_.clump_id = m.take<int>(N); h_.clump_id2 = m.take<int>(N);
            h_.part_fix = m.take<int>(N); h_.part_fix2 = m.take<int>(N);
            h_.level = m.take<int>(N); h_.level2 = m.take<int>(N);
            h_.key = m.take<int>(N); h_.key2 = m.take<int>(N);
            // contact kinematics: world lever arm and mass, one FP64 double4 per
            // subsphere (the velocities are read from the clump's records)
            h_.kin = m.take<char>(N * sizeof(double4));
            h_.kin2 = m.take<char>(N * sizeof(double4));
            h_.bhist = m.take<R4<R>>((size_t)NB_SLOTS * 3 * N); h_.bhist2 = m.take<R4<R>>((size_t)NB_SLOTS * 3 * N);
            h_.bbits = m.take<uint16_t>(N); h_.bbits2 = m.take<uint16_t>(N);
            h_.fsum = m.take<R4<R>>(2 * N);
            h_.fbnd = m.take<R4<R>>(2 * N);
            h_.fint = sphere_kin_ ? m.take<R4<R>>(2 * N) : nullptr;
            h_.kind = has_kinds_ ? m.take<int>(K_) : nullptr;
            h_.cpos = m.take<double4>(K_); h_.cvel = m.take<double4>(K_); h_.cw = m.take<double4>(K_);
            h_.cq = m.take<double4>(K_); h_.cprop = m.take<double4>(K_);
            h_.cinv = m.take<double4>(K_);
            h_.mem_cl = m.take<int>(N);
            h_.cF = m.take<double4>(K_); h_.cT = m.take<double4>(K_);
            h_.mem_start = m.take<int>(K_ + 1);
            h_.mem_idx = m.take<int>(N);
            int* flags = m.take<int>(16);
            h_.post_pending = flags + 0;
            h_.any_rebuild = flags + 1;
            h_.halt = flags + 2;
            h_.lcur = flags + 3;
            h_.hgen = flags + 4;
            h_.gstep = flags + 5;
            h_.kc_done = flags + 6;
            h_.lstep = flags + 7;
            h_.loop_left = flags + 8;
            h_.scan_fail = flags + 9;
            h_.kA = m.take<int>(N); h_.vA = m.take<int>(N); h_.kB = m.take<int>(N); h_.vB = m.take<int>(N);
            h_.ccnt = m.take<int>((size_t)cells + S_ + 1);
            h_.ccur = m.take<int>((size_t)cells + S_ + 1);
            h_.perm = m.take<int>(N);
            h_.inv = m.take<int>(N);
            h_.cstart = m.take<int>(cells + 1);
            h_.scr = m.take<int>((size_t)N * 2 * SCR_CAP);
            h_.cnt_f = m.take<int>(N + 1);
            h_.nrb = m.take<int2>(N + S_);
            h_.nprefix = m.take<int>(S_ + 1);
            h_.bidx = m.take<int>(N);
            h_.bprefix = m.take<int>(S_ + 1);
            h_.cnt_b = m.take<int>(N + 1);
            h_.sfc = m.take<int>(N);
            h_.xcnt = m.take<int>(N + 1);
            const long long scan_tiles = std::max(cdiv(N + 1, SC_TILE), cdiv((long long)cells + S_ + 1, SC_TILE));
            h_.scan_tmp = m.take<int>(scan_tiles + 1);
            h_.scan_st = m.take<unsigned long long>(3 * scan_tiles + 3);
            h_.scan_ctl = m.take<int>(2);
            for (int l = 0; l < 2; l++) {
                h_.L[l].row = m.take<int>(N + S_);
                h_.L[l].brow = m.take<int>(N + S_);
            }
            h_.plan = m.take<int>(PL_SIZE);
            h_.pscene = m.take<int>(S_);
            h_.psub = m.take<int>(S_ + 1);
            h_.pcell = m.take<int>(S_ + 1);
            h_.pclump = m.take<int>(S_ + 1);
            h_.ppair = m.take<int>(S_ + 1);
            h_.need = m.take<int>(S_);
            relmap_ = m.take<int4>(S_);
            h_.xparts = m.take<R4<R>>(6 * N);
            h_.xintr = m.take<R4<R>>(4 * N);
            h_.ring_len = ring_len_;
            h_.ring = m.take<double>((size_t)S_ * ring_len_ * 6);
            d_ = m.take<Dev>(1);
        };
        Carver sz;
        layout(sz);
        Carver m{(uintptr_t)mem_.alloc<char>(sz.off)};
        layout(m);
        // the pair regions are sized at the first list (nothing is stored in them before)
        alloc_pairs(1);

        copy_(h_.par, hpar_.data(), S_ * sizeof(ScenePar), cudaMemcpyHostToDevice);
        copy_(h_.dyn, hdyn.data(), S_ * sizeof(SceneDyn), cudaMemcpyHostToDevice);
        copy_(h_.sid, sid.data(), N * sizeof(int), cudaMemcpyHostToDevice);
        copy_(h_.csid, csid.data(), K_ * sizeof(int), cudaMemcpyHostToDevice);
        copy_(h_.posr, posr.data(), N * sizeof(double4), cudaMemcpyHostToDevice);
        copy_(h_.lom, lom.data(), N * sizeof(double4), cudaMemcpyHostToDevice);
        copy_(h_.clump_id, cid.data(), N * sizeof(int), cudaMemcpyHostToDevice);
        copy_(h_.part_fix, fix.data(), N * sizeof(int), cudaMemcpyHostToDevice);
        copy_(h_.level, lev.data(), N * sizeof(int), cudaMemcpyHostToDevice);
        copy_(h_.cpos, cpos.data(), K_ * sizeof(double4), cudaMemcpyHostToDevice);
        copy_(h_.cvel, cvel.data(), K_ * sizeof(double4), cudaMemcpyHostToDevice);
        copy_(h_.cw, cw.data(), K_ * sizeof(double4), cudaMemcpyHostToDevice);
        copy_(h_.cq, cq.data(), K_ * sizeof(double4), cudaMemcpyHostToDevice);
        copy_(h_.cprop, cprop.data(), K_ * sizeof(double4), cudaMemcpyHostToDevice);
        if (h_.kind) copy_(h_.kind, kind.data(), K_ * sizeof(int), cudaMemcpyHostToDevice);
        {
            // the clump pass's reciprocals: IEEE divisions, bitwise those it formed each step
            std::vector<double4> cinv(K_);
            for (int k = 0; k < K_; k++)
                cinv[k] = make_double4(1.0 / cprop[k].x, 1.0 / cprop[k].y, 1.0 / cprop[k].z, 1.0 / cprop[k].w);
            copy_(h_.cinv, cinv.data(), K_ * sizeof(double4), cudaMemcpyHostToDevice);
            std::vector<int> mcl(N);
            for (int k = 0; k < K_; k++)
                for (int m = mstart[k]; m < mstart[k + 1]; m++) mcl[m] = k;
            copy_(h_.mem_cl, mcl.data(), N * sizeof(int), cudaMemcpyHostToDevice);
        }
        copy_(h_.mem_start, mstart.data(), (K_ + 1) * sizeof(int), cudaMemcpyHostToDevice);
        copy_(h_.mem_idx, midx.data(), N * sizeof(int), cudaMemcpyHostToDevice);
        // the first list is empty: rows of zeros (the slab is zeroed)
        int one = 1;
        copy_(h_.any_rebuild, &one, sizeof(int), cudaMemcpyHostToDevice);
        push_dev();
    }

    void alloc_pairs(long long cap) {
        if (cap > 2000000000LL) throw CudaError("pair capacity above 2^31");
        h_.cap = (int)cap;
        auto layout = [&](Carver& m) {
            for (int l = 0; l < 2; l++) {
                h_.L[l].nbr = m.take<int>(cap);
                h_.L[l].own = m.take<int>(cap);
                h_.L[l].bnbr = m.take<int>(cap);
                h_.L[l].bpair = m.take<int>(cap);
                h_.H[l] = m.take<char>(hist_bytes(cap));
                h_.touch[l] = m.take<uint8_t>(cap);
            }
            h_.nfs = m.take<R4<R>>(2 * cap);
            h_.nbs = m.take<R4<R>>(2 * cap);
            h_.nbpos = m.take<int>(cap);
            h_.nfr = m.take<int4>(cap);
            h_.nbq = m.take<int>(cap);
            h_.nearf = m.take<uint8_t>(cap);
            h_.xfcn = m.take<R4<R>>(cap);
            h_.xcpt = m.take<double4>(cap);
        };
        Carver sz;
        layout(sz);
        pslab_bytes_ = sz.off;
        pslab_ = mem_.alloc<char>(pslab_bytes_);
        Carver m{(uintptr_t)pslab_};
        layout(m);
    }
    static size_t hist_bytes(long long cap) { return (size_t)cap * (2 * sizeof(R4<R>) + sizeof(R)); }

    double slack() const { return opt_.pair_slack >= 1.0 ? opt_.pair_slack : 1.6; }
    // Bytes of the pair buffers per pair slot.
    static double bytes_per_pair() {
        return 2.0 * (4 * sizeof(int) + (double)hist_bytes(1) + 1) + 5 * sizeof(R4<R>) + sizeof(double4) +
               2 * sizeof(int) + sizeof(int4) + 1;
    }
    // Region capacities for the first lists: slack x each scene's pairs; with
    // the default slack at least the reference's own list capacity, n_sub x
    // BranchLmtLen/2, as far as 30% of the free device memory allows (growing
    // later costs a host round trip and a re-layout).
    std::vector<long long> first_capacities(const std::vector<long long>& need) {
        std::vector<long long> cap(S_);
        for (int s = 0; s < S_; s++) cap[s] = std::max<long long>(16, (long long)std::ceil(need[s] * slack()));
        if (opt_.pair_slack >= 1.0) return cap;
        double want = 0, have = 0;
        for (int s = 0; s < S_; s++) {
            have += (double)cap[s];
            want += std::max(0.0, (double)hpar_[s].nsub * (hpar_[s].bl / 2) - (double)cap[s]);
        }
        size_t fr = 0, tot = 0;
        CK(cudaMemGetInfo(&fr, &tot));
        const double budget = 0.3 * (double)fr / bytes_per_pair() - have;
        if (budget <= 0 || want <= 0) return cap;
        const double f = std::min(1.0, budget / want);
        for (int s = 0; s < S_; s++) {
            const double extra = std::max(0.0, (double)hpar_[s].nsub * (hpar_[s].bl / 2) - (double)cap[s]);
            cap[s] += (long long)(f * extra);
        }
        return cap;
    }
    // the regions after an overflow: every scene whose new list does not fit
    // gets slack x its pairs (at least 1,024 more slots)
    std::vector<long long> grown_capacities(const std::vector<int>& need, const std::vector<SceneDyn>& y) {
        std::vector<long long> cap(S_);
        for (int s = 0; s < S_; s++) {
            cap[s] = y[s].pcap;
            if (need[s] > y[s].pcap)
                cap[s] = std::max<long long>((long long)std::ceil(need[s] * slack()), (long long)y[s].pcap + 1024);
        }
        return cap;
    }
    std::vector<SceneDyn> read_dyn_all() {
        std::vector<SceneDyn> y(S_);
        copy_(y.data(), h_.dyn, S_ * sizeof(SceneDyn), cudaMemcpyDeviceToHost);
        return y;
    }
    // New pair regions of the given capacities: the pair buffers are
    // re-allocated and every scene's current list, the history generation
    // the next contact pass reads, touch and near flags move to its new
    // region (rows shifted).  The build list and the other generation need
    // nothing: a rebuild writes them before reading.
    void layout_pairs(const std::vector<long long>& pcap) {
        refresh_dev();
        std::vector<SceneDyn> y = read_dyn_all();
        std::vector<int4> map(S_);
        long long total = 0;
        int moved = 0;
        for (int s = 0; s < S_; s++) {
            map[s].x = y[s].pair_off;
            map[s].y = (int)total;
            map[s].z = y[s].npairs;
            map[s].w = moved;
            moved += y[s].npairs;
            y[s].pair_off = (int)total;
            y[s].pcap = (int)pcap[s];
            total += pcap[s];
            if (total > 2000000000LL) throw CudaError("pair capacity above 2^31");
        }
        const int hg = read_int(h_.hgen);
        Dev old = h_;
        char* old_slab = pslab_;
        const size_t old_bytes = pslab_bytes_;
        alloc_pairs(std::max<long long>(total, 1));
        copy_(h_.dyn, y.data(), S_ * sizeof(SceneDyn), cudaMemcpyHostToDevice);
        copy_(relmap_, map.data(), S_ * sizeof(int4), cudaMemcpyHostToDevice);
        push_dev();
        const int B = 256;
        if (moved > 0)
            k_relayout<R><<<std::min(148 * 8, cdiv(moved, B)), B, 0, stream_>>>(
                d_, old.L[0], old.H[hg & 1], old.touch[hg & 1], old.nearf, old.nfr, old.nbq, old.nbpos, old.cap,
                relmap_, moved);
        k_shift_rows<<<std::min(148 * 8, cdiv((long long)N_ + S_, B)), B, 0, stream_>>>(d_, relmap_);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(stream_));
        mem_.release(old_slab, old_bytes);
    }

    // Every copy goes through the engine's own stream.  cudaMemcpy would run
    // on the legacy default stream, which is not ordered with the engine's
    // non-blocking streams: a device-to-device copy (and the DMA of a pageable
    // host-to-device copy) may still be in flight when cudaMemcpy returns, so
    // a later kernel, or a stream-ordered free of the source, would race it.
    // Copies that touch host memory wait for the stream before returning.
    void copy_(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
        if (!bytes) return;
        CK(cudaMemcpyAsync(dst, src, bytes, kind, stream_));
        if (kind != cudaMemcpyDeviceToDevice) CK(cudaStreamSynchronize(stream_));
    }
    void push_dev() {
        CK(cudaStreamSynchronize(stream_));
        copy_(d_, &h_, sizeof(Dev), cudaMemcpyHostToDevice);
    }
    // the host copy of the pointer table, as the device has it
    void refresh_dev() {
        CK(cudaStreamSynchronize(stream_));
        copy_(&h_, d_, sizeof(Dev), cudaMemcpyDeviceToHost);
    }
    int read_int(const int* p) {
        CK(cudaStreamSynchronize(stream_));
        int v = 0;
        copy_(&v, p, sizeof(int), cudaMemcpyDeviceToHost);
        return v;
    }
    int read_gstep() { return read_int(h_.gstep); }
    SceneDyn read_dyn(int s) {
        CK(cudaStreamSynchronize(stream_));
        SceneDyn y;
        copy_(&y, h_.dyn + s, sizeof(SceneDyn), cudaMemcpyDeviceToHost);
        return y;
    }
    void pull_r4(const void* base, int off, int n, double* dst) {
        if (!dst) return;
        std::vector<R4<R>> tmp(n);
        copy_(tmp.data(), (const R4<R>*)base + off, n * sizeof(R4<R>), cudaMemcpyDeviceToHost);
        for (int i = 0; i < n; i++) { dst[3 * i] = tmp[i].x; dst[3 * i + 1] = tmp[i].y; dst[3 * i + 2] = tmp[i].z; }
    }
    RowData pull_rows(int s) {
        refresh_dev();
        const ScenePar& P = hpar_[s];
        int lc = read_int(h_.lcur);
        const PairList& Lc = h_.L[lc & 1];
        RowData rd;
        rd.row.resize(P.nsub + 1);
        rd.brow.resize(P.nsub + 1);
        copy_(rd.row.data(), Lc.row + P.sub_off + s, (P.nsub + 1) * sizeof(int), cudaMemcpyDeviceToHost);
        copy_(rd.brow.data(), Lc.brow + P.sub_off + s, (P.nsub + 1) * sizeof(int), cudaMemcpyDeviceToHost);
        int nf = rd.row[P.nsub] - rd.row[0], nb = rd.brow[P.nsub] - rd.brow[0];
        rd.nbr.resize(nf);
        rd.bnbr.resize(nb);
        rd.bpair.resize(nb);
        copy_(rd.nbr.data(), Lc.nbr + rd.row[0], nf * sizeof(int), cudaMemcpyDeviceToHost);
        copy_(rd.bnbr.data(), Lc.bnbr + rd.brow[0], nb * sizeof(int), cudaMemcpyDeviceToHost);
        copy_(rd.bpair.data(), Lc.bpair + rd.brow[0], nb * sizeof(int), cudaMemcpyDeviceToHost);
        return rd;
    }

    void check_scan() {
        if (read_int(h_.scan_fail)) throw CudaError("a list-rebuild scan gave up waiting on a tile (step halted)");
    }
    void check_errors() {
        check_scan();
        std::vector<SceneDyn> y(S_);
        copy_(y.data(), h_.dyn, S_ * sizeof(SceneDyn), cudaMemcpyDeviceToHost);
        for (int s = 0; s < S_; s++)
            if (y[s].err & ERR_NONFINITE) throw NonFinite("scene " + std::to_string(s) + ": non-finite force");
    }

    // ---- launches -------------------------------------------------------------
    void launch_clump(int do_pre, cudaGraphConditionalHandle cond = 0, int use_cond = 0,
                      cudaGraphConditionalHandle loop = 0, int use_loop = 0) {
        const int g = cdiv(K_ + S_, CL_THREADS);
        if (sphere_any_) {
            if (clump_batch_ == 1)
                k_clump<R, 1, true><<<g, CL_THREADS, clump_dyn_smem<R, 1>(), stream_>>>(d_, do_pre, cond, use_cond, loop, use_loop);
            else if (clump_batch_ == 4)
                k_clump<R, 4, true><<<g, CL_THREADS, clump_dyn_smem<R, 4>(), stream_>>>(d_, do_pre, cond, use_cond, loop, use_loop);
            else
                k_clump<R, 2, true><<<g, CL_THREADS, clump_dyn_smem<R, 2>(), stream_>>>(d_, do_pre, cond, use_cond, loop, use_loop);
        } else if (clump_batch_ == 1)
            k_clump<R, 1, false><<<g, CL_THREADS, clump_dyn_smem<R, 1>(), stream_>>>(d_, do_pre, cond, use_cond, loop, use_loop);
        else if (clump_batch_ == 4)
            k_clump<R, 4, false><<<g, CL_THREADS, clump_dyn_smem<R, 4>(), stream_>>>(d_, do_pre, cond, use_cond, loop, use_loop);
        else
            k_clump<R, 2, false><<<g, CL_THREADS, clump_dyn_smem<R, 2>(), stream_>>>(d_, do_pre, cond, use_cond, loop, use_loop);
        CK(cudaGetLastError());
        if (!capturing_) launches_ += 1;
    }
    bool capturing_ = false;
    // the contact pass: k_pairs, with k_boundary beside it on the second
    // stream (fork and join by events, which become graph edges when
    // captured), then k_sum
    void launch_contact(bool exp) {
        if (exp) {
            CK(cudaMemsetAsync(h_.xfcn, 0, (size_t)h_.cap * sizeof(R4<R>), stream_));
            CK(cudaMemsetAsync(h_.xcpt, 0, (size_t)h_.cap * sizeof(double4), stream_));
            // wall and intruder parts: k_boundary writes its candidates only
            CK(cudaMemsetAsync((R4<R>*)h_.xparts + 2 * (size_t)N_, 0, 4 * (size_t)N_ * sizeof(R4<R>), stream_));
            CK(cudaMemsetAsync(h_.xintr, 0, 4 * (size_t)N_ * sizeof(R4<R>), stream_));
        }
        CK(cudaEventRecord(ev_fork_, stream_));
        CK(cudaStreamWaitEvent(stream2_, ev_fork_, 0));
        // the start of the contact pass is marked on the side branch (same
        // dependencies), so only its end mark sits on the critical path
        mark(5, stream2_);
        mark(3, stream2_);
        // grid-stride over the boundary candidates (a device count)
        const int bg = std::min(sm_count_ * 8, cdiv(N_, BD_THREADS));
        if (sphere_any_) {
            if (exp) k_boundary<R, true, true><<<bg, BD_THREADS, 0, stream2_>>>(d_);
            else k_boundary<R, false, true><<<bg, BD_THREADS, 0, stream2_>>>(d_);
        } else if (exp) k_boundary<R, true, false><<<bg, BD_THREADS, 0, stream2_>>>(d_);
        else k_boundary<R, false, false><<<bg, BD_THREADS, 0, stream2_>>>(d_);
        mark(4, stream2_);
        CK(cudaEventRecord(ev_join_, stream2_));
        // grid-stride over the near pairs (a device count), so a fixed grid
        // stays valid as the list grows; a small scene gets a small grid so
        // that other scenes' kernels run beside it
        const int pg = std::min(sm_count_ * pair_bps_, cdiv(3LL * N_, PR_THREADS));
        if (exp) k_pairs<R, true><<<pg, PR_THREADS, 0, stream_>>>(d_);
        else k_pairs<R, false><<<pg, PR_THREADS, 0, stream_>>>(d_);
        CK(cudaStreamWaitEvent(stream_, ev_join_, 0));
        CK(cudaGetLastError());
        mark(6, stream_);
        if (!capturing_) launches_ += CONTACT_LAUNCHES;
        // the export step also records the per-subsphere pair part
        if (exp) launch_sum(true);
    }
    // per-subsphere totals of the last contact pass into fsum (the clump
    // pass sums the same slots itself; this runs for getters and exports)
    void launch_sum(bool exp) {
        if (exp) k_sum<R, true><<<cdiv(N_, CT_THREADS), CT_THREADS, 0, stream_>>>(d_);
        else k_sum<R, false><<<cdiv(N_, CT_THREADS), CT_THREADS, 0, stream_>>>(d_);
        CK(cudaGetLastError());
    }
    // exclusive scans of a0 (and a1, a2, of the same length) over [0, n), or
    // over [0, *dn) when dn is given (n then bounds it), in one launch
    void scan(int* a0, int* a1, int* a2, int n, const int* dn = nullptr) {
        // a grid of at most a few blocks per SM takes the tiles; a grid sized
        // for the largest length would start tens of thousands of blocks that
        // find nothing to do when few scenes are rebuilt
        const int nb = std::min(std::max(1, cdiv(n, SC_TILE)) * (a2 ? 3 : (a1 ? 2 : 1)), sm_count_ * 4);
        k_scan1<<<nb, SC_THREADS, 0, stream_>>>(a0, a1, a2, n, dn, h_.scan_st, h_.scan_ctl, h_.halt, h_.scan_fail);
    }
    // The rebuild block of src/dem_simulation_clump.cu:124-176, over the
    // scenes whose rebuild flag is set: every kernel but the near rows walks
    // the rebuilt scenes only (grid-stride over counts the plan puts on the
    // device), so a batch pays for the scenes it rebuilds.
    void launch_rebuild(bool eager) {
        const int B = 128;
        const int gN = std::min(cdiv(N_, B), 148 * 16);         // grid-stride grids
        const int sl = search_lanes_;
        const int gS = std::min(cdiv(N_, SEARCH_THREADS / sl), 148 * 16);
        const int* pl = h_.plan;
        k_plan<<<1, SC_THREADS, 0, stream_>>>(d_);
        k_hash<<<gN, B, 0, stream_>>>(d_);
        // counting sort by cell: the counts' scan, the scatter, each cell's
        // range in subsphere order with the permutation and the cell table
        scan(h_.ccnt, nullptr, nullptr, h_.cells + S_ + 1, pl + PL_TC1);
        k_cscatter<<<gN, B, 0, stream_>>>(d_);
        k_cellfix<<<std::min(cdiv(h_.cells + S_, 256), 148 * 16), 256, 0, stream_>>>(d_);
        k_reorder<R><<<gN, B, 0, stream_>>>(d_);
        if (sl == 16) k_search<16><<<gS, SEARCH_THREADS, 0, stream_>>>(d_);
        else if (sl == 32) k_search<32><<<gS, SEARCH_THREADS, 0, stream_>>>(d_);
        else k_search<8><<<gS, SEARCH_THREADS, 0, stream_>>>(d_);
        scan(h_.cnt_f, h_.cnt_b, nullptr, N_ + 1, pl + PL_T1);
        CK(cudaGetLastError());
        if (eager) {
            // size the regions to the first lists, or grow the ones that overflow
            k_check_cap<<<1, 256, 0, stream_>>>(d_, 0);
            CK(cudaStreamSynchronize(stream_));
            check_scan();
            std::vector<int> need(S_);
            copy_(need.data(), h_.need, S_ * sizeof(int), cudaMemcpyDeviceToHost);
            std::vector<SceneDyn> y = read_dyn_all();
            if (first_list_) {
                std::vector<long long> nd(S_);
                for (int s = 0; s < S_; s++) nd[s] = need[s] >= 0 ? need[s] : y[s].npairs;
                layout_pairs(first_capacities(nd));
                first_list_ = false;
            } else {
                bool grow = false;
                for (int s = 0; s < S_; s++) grow |= need[s] > y[s].pcap;
                if (grow) layout_pairs(grown_capacities(need, y));
            }
        }
        k_check_cap<<<1, 256, 0, stream_>>>(d_, 1);
        if (sl == 16) k_compact<16><<<gS, SEARCH_THREADS, 0, stream_>>>(d_);
        else if (sl == 32) k_compact<32><<<gS, SEARCH_THREADS, 0, stream_>>>(d_);
        else k_compact<8><<<gS, SEARCH_THREADS, 0, stream_>>>(d_);
        if (hgrid_) k_xsort<<<gN, B, 0, stream_>>>(d_);
        k_backref<<<gN, B, 0, stream_>>>(d_);
        const int gP = std::min(148 * 8, cdiv(8LL * N_, 256));
        k_carry<R><<<gP, 256, 0, stream_>>>(d_);
        k_writeback<R><<<gP, 256, 0, stream_>>>(d_);
        // near rows and boundary candidates of the rebuilt scenes (counts and
        // flags, their scans, rows and list with the rebuild's bookkeeping),
        // then the work-item prefixes over the scenes
        const int gNr = std::min(cdiv(N_, SEARCH_THREADS / 4), 148 * 16);
        k_near<false, 4><<<gNr, SEARCH_THREADS, 0, stream_>>>(d_);
        scan(h_.cnt_f, h_.cnt_b, h_.xcnt, N_ + 1, pl + PL_T1);
        k_near<true, 4><<<gNr, SEARCH_THREADS, 0, stream_>>>(d_);
        k_near_finish<<<std::min(cdiv(N_, SC_THREADS), 148 * 8), SC_THREADS, 0, stream_>>>(d_);
        CK(cudaGetLastError());
    }

    void run_step_eager(bool exp) {
        rec_ = timing_ ? next_record() : nullptr;
        mark(0, stream_);
        launch_clump(1);
        mark(1, stream_);
        CK(cudaMemcpyAsync(hflag_, h_.any_rebuild, sizeof(int), cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        if (hflag_[0]) launch_rebuild(true);
        mark(2, stream_);
        launch_contact(exp);
        mark(7, stream_);
        rec_ = nullptr;
        steps_done_ += 1;
    }

    // one step as a graph: k_clump, a conditional node holding the rebuild,
    // then k_boundary and k_contact on two branches; the timed variants have
    // event nodes at the timing marks
    void capture(int timed) {
        if (timed && !gev_[timed][0])
            for (int k = 0; k < NMARK; k++) CK(cudaEventCreate(&gev_[timed][k]));
        capturing_ = true;
        capture_timed_ = timed;
        cudaGraph_t& graph = graph_[timed];
        CK(cudaGraphCreate(&graph, 0));
        cudaGraphConditionalHandle hnd;
        CK(cudaGraphConditionalHandleCreate(&hnd, graph, 0, cudaGraphCondAssignDefault));
        CK(cudaStreamBeginCaptureToGraph(stream_, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        mark(0, stream_);
        launch_clump(1, hnd, 1);
        mark(1, stream_);
        cudaStreamCaptureStatus st;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        CK(cudaStreamGetCaptureInfo(stream_, &st, nullptr, nullptr, &deps, &ndeps));
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.conditional.handle = hnd;
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        cudaGraphNode_t cnode;
        CK(cudaGraphAddNode(&cnode, graph, deps, ndeps, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        CK(cudaStreamUpdateCaptureDependencies(stream_, &cnode, 1, cudaStreamSetCaptureDependencies));
        mark(2, stream_);
        launch_contact(false);
        mark(7, stream_);
        cudaGraph_t g2 = nullptr;
        CK(cudaStreamEndCapture(stream_, &g2));
        // the rebuild branch
        capture_timed_ = 0;
        CK(cudaStreamBeginCaptureToGraph(stream_, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        launch_rebuild(false);
        cudaGraph_t b2 = nullptr;
        CK(cudaStreamEndCapture(stream_, &b2));
        capturing_ = false;
        for (int k = 0; k < NMARK; k++)
            if (mark_on(timed, k) && !gev_node_[timed][k]) throw CudaError("event nodes missing from the step graph");
        CK(cudaGraphInstantiate(&gexec_[timed], graph, 0));
    }
    cudaGraphNode_t last_captured_node(cudaStream_t st) {
        cudaStreamCaptureStatus cs;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        CK(cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &deps, &nd));
        if (nd != 1) throw CudaError("unexpected capture dependencies");
        return deps[0];
    }
    void launch_graph() {
        if (timing_) {
            cudaEvent_t* r = next_record();
            for (int k = 0; k < NMARK; k++)
                if (mark_on(timing_, k))
                    CK(cudaGraphExecEventRecordNodeSetEvent(gexec_[timing_], gev_node_[timing_][k], r[k]));
        }
        CK(cudaGraphLaunch(gexec_[timing_], stream_));
    }

    // Many steps in one graph launch: a while node whose body is one step
    // (k_clump, the rebuild under an if node, the contact pass).  The step
    // count goes to the kernel node ahead of the loop; the last block of each
    // step's k_clump counts it down and ends the loop at zero, or at once
    // when a rebuild has run out of pair capacity (the host then finishes
    // that step, as after a per-step graph).  Step graphs with timing event
    // nodes stay one step per launch (an event node in a loop body would be
    // overwritten by every iteration).  If the loop graph cannot be built the
    // engine keeps launching one step per graph.
    void capture_loop() {
        loop_tried_ = true;
        capturing_ = true;
        capture_timed_ = 0;
        try {
            CK(cudaGraphCreate(&graph_loop_, 0));
            cudaGraphConditionalHandle hw;
            CK(cudaGraphConditionalHandleCreate(&hw, graph_loop_, 1, cudaGraphCondAssignDefault));
            CK(cudaStreamBeginCaptureToGraph(stream_, graph_loop_, nullptr, nullptr, 0,
                                             cudaStreamCaptureModeThreadLocal));
            k_loop_init<<<1, 1, 0, stream_>>>(h_.loop_left, 1);
            CK(cudaGetLastError());
            loop_init_node_ = last_captured_node(stream_);
            cudaGraph_t body = add_conditional(graph_loop_, hw, cudaGraphCondTypeWhile);
            cudaGraph_t g2 = nullptr;
            CK(cudaStreamEndCapture(stream_, &g2));
            cudaGraphConditionalHandle hif;
            CK(cudaGraphConditionalHandleCreate(&hif, body, 0, cudaGraphCondAssignDefault));
            CK(cudaStreamBeginCaptureToGraph(stream_, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
            launch_clump(1, hif, 1, hw, 1);
            cudaGraph_t rbody = add_conditional(body, hif, cudaGraphCondTypeIf);
            launch_contact(false);
            CK(cudaStreamEndCapture(stream_, &g2));
            CK(cudaStreamBeginCaptureToGraph(stream_, rbody, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
            launch_rebuild(false);
            CK(cudaStreamEndCapture(stream_, &g2));
            CK(cudaGraphInstantiate(&gexec_loop_, graph_loop_, 0));
        } catch (const CudaError& e) {
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            if (cudaStreamIsCapturing(stream_, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(stream_, &g);
            }
            (void)cudaGetLastError();
            if (gexec_loop_) cudaGraphExecDestroy(gexec_loop_);
            if (graph_loop_) cudaGraphDestroy(graph_loop_);
            gexec_loop_ = nullptr;
            graph_loop_ = nullptr;
            loop_error_ = e.what();
        }
        capturing_ = false;
    }
    // a conditional node after the capture's current dependencies; returns its body
    cudaGraph_t add_conditional(cudaGraph_t graph, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type) {
        cudaStreamCaptureStatus st;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        CK(cudaStreamGetCaptureInfo(stream_, &st, nullptr, nullptr, &deps, &ndeps));
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.conditional.handle = h;
        cp.conditional.type = type;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        CK(cudaGraphAddNode(&node, graph, deps, ndeps, &cp));
        CK(cudaStreamUpdateCaptureDependencies(stream_, &node, 1, cudaStreamSetCaptureDependencies));
        return cp.conditional.phGraph_out[0];
    }
    void launch_loop(int n) {
        int* left = h_.loop_left;
        void* args[] = {&left, &n};
        cudaKernelNodeParams kp = {};
        kp.func = (void*)k_loop_init;
        kp.gridDim = dim3(1);
        kp.blockDim = dim3(1);
        kp.kernelParams = args;
        CK(cudaGraphExecKernelNodeSetParams(gexec_loop_, loop_init_node_, &kp));
        CK(cudaGraphLaunch(gexec_loop_, stream_));
    }

    // a graph launch stopped at a rebuild whose pairs did not fit: grow and
    // finish that step's rebuild and contact pass on the host path
    void recover_halt() {
        refresh_dev();
        std::vector<int> need(S_);
        copy_(need.data(), h_.need, S_ * sizeof(int), cudaMemcpyDeviceToHost);
        std::vector<SceneDyn> y = read_dyn_all();
        layout_pairs(grown_capacities(need, y));
        int zero = 0;
        copy_(h_.halt, &zero, sizeof(int), cudaMemcpyHostToDevice);
        y = read_dyn_all();
        for (auto& v : y) v.err &= ~ERR_LIST_OVERFLOW;
        copy_(h_.dyn, y.data(), S_ * sizeof(SceneDyn), cudaMemcpyHostToDevice);
        launch_rebuild(true);
        launch_contact(false);
        CK(cudaStreamSynchronize(stream_));
        steps_done_ += 1;
    }
};

EngineBase* make_engine(const std::vector<const nbc_scene_desc*>& sc, const nbc_options& opt) {
    if (opt.precision == NBC_PREC_F64) return new EngineT<double>(sc, opt);
    return new EngineT<float>(sc, opt);
}

}  // namespace nbc
