// kernels.cuh -- sm_100a kernels of the B200 DEM engine.
//
// Step structure (one CUDA graph per step, see engine.cu):
//   k_clump      per clump: member force/torque sum and second half-kick of
//                the previous step, first half-kick, drift, attitude and the
//                pose of every member subsphere (+ rebuild test); one extra
//                thread per scene advances the intruder.
//   [rebuild]    only when some scene's subsphere moved more than Thresh
//                since that scene's last rebuild: hash with cell counts,
//                counting sort by cell (each cell's range in subsphere
//                order: the reference's stable sort), reorder and cell
//                table, count/scan/fill of the half pair list in the
//                reference's traversal order, back references, history
//                carry, near rows, clump member lists.
//   k_pairs      per near pair: overlap test, the law once for both
//                subspheres of a touching pair, the new spring history, the
//                force and torque on each side into its near-row slot
//   k_boundary   per boundary candidate: walls and intruder (beside k_pairs)
//   (the next step's k_clump sums each member's slots and boundary force)
#pragma once
#include "nbc_dev.cuh"
#include "nbc_math.cuh"

namespace nbc {

constexpr double FIX_F = 1099511627776.0;    // 2^40: fixed-point scale of intruder force sums
constexpr double FIX_T = 17592186044416.0;   // 2^44: fixed-point scale of intruder torque sums
constexpr int IDX_MASK = 0x7fffffff;
constexpr int INTRA = (int)0x80000000u;

// The contact slots of one subsphere (its near front entries, then its near
// back entries, in row order; SumContForce_clump, src/dem_force_clump.cu:
// 165-191, sums a subsphere's front entries, then its back entries).
template <typename R>
__device__ __forceinline__ void slot_sum(const R4<R>* __restrict__ fs, const R4<R>* __restrict__ bs, size_t cap,
                                         int rs, int re, int bs0, int be, V3<R>& F, V3<R>& T) {
    F = v3<R>(0, 0, 0);
    T = F;
    // not unrolled: a subsphere has a few near entries at most, and unrolled
    // copies cost the clump pass registers (and warps per SM)
#pragma unroll 1
    for (int e = rs; e < re; e++) {
        F = F + xyz<R>(fs[2 * (size_t)e]);
        T = T + xyz<R>(fs[2 * (size_t)e + 1]);
    }
#pragma unroll 1
    for (int e = bs0; e < be; e++) {
        F = F + xyz<R>(bs[2 * (size_t)e]);
        T = T + xyz<R>(bs[2 * (size_t)e + 1]);
    }
}

// ===========================================================================
// clump pass
// ===========================================================================

// 16-byte asynchronous copy global -> shared (no register holds the data in
// flight, so one thread can have many outstanding), and the wait for all of
// the calling thread's copies.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}
// a contact record staged for the clump pass: force and torque (two Real4)
template <typename R> struct SlotRec {
    R4<R> f, t;
};
template <typename R>
__device__ __forceinline__ void stage_rec(SlotRec<R>* dst, const R4<R>* f, const R4<R>* t) {
    for (int k = 0; k < (int)sizeof(R4<R>) / 16; k++) {
        cp_async16((char*)&dst->f + 16 * k, (const char*)f + 16 * k);
        cp_async16((char*)&dst->t + 16 * k, (const char*)t + 16 * k);
    }
}

// Integrate_Before_clump_cuk / Attitude_clump_cuk / Integrate_After_clump_cuk
// (src/dem_integrate_clumpsphere.cu:3-141), UpdatePos_cuk (src/dem_clump.cu:
// 113-138), ComputeTorqueFromWorldPos_Kernel + reduce_by_key
// (src/dem_clumpsphere.cu:86-151), IntegratePene_Before_cuk and
// Integrate_After_cuk (src/dem_integrate_penetrator.cu:3-113).
//
// One clump per lane, 32 clumps per warp.  The member work is spread over
// the warp instead: the members of the warp's clumps are one contiguous range
// of the member list, the lanes load all member indices of a chunk and then
// all member records (every load of the chunk in flight at once), each
// member's force and lever-arm torque go to shared memory, and each lane then
// sums its own clump's members in ascending order (the reduce_by_key order)
// and integrates its clump once.  The new poses are shared the same way and
// the lanes pose the members 32 at a time.  The lanes after the last clump
// hold one thread per scene for the intruder.
//
// A step (do_pre) also advances the spring-history generation so the next
// contact pass reads what the previous one wrote, and counts itself; the last
// block to finish sets the graph's rebuild condition (when given a handle)
// and counts the step in lstep.  A scene with a stop s takes the steps started
// at lstep = 0 .. s-1 and closes the last one at lstep = s; afterwards it
// stands still (frozen) while the other scenes go on, so its state is
// exactly that of the scene run alone for s steps.
__device__ __forceinline__ bool scene_pre(const SceneDyn& y, int do_pre, int L) {
    return do_pre && (y.stop == 0 || L < y.stop);
}
__device__ __forceinline__ bool scene_post(const SceneDyn& y, int post, int L) {
    return post && (y.stop == 0 || L <= y.stop);
}
constexpr int CL_THREADS = 128;
constexpr int CL_WARPS = CL_THREADS / 32;
// staged contact records per warp: cl_stage<J>() per member of a chunk on
// average; a lane whose members would overflow the warp's records sums from
// global memory directly (same order, same result).  Dynamic shared memory.
// Four records per member at J <= 2 (a shallower stage at J = 2 sends more
// lanes to the unstaged sums: 46.6 against 35.9 µs per cfg1 step); two at
// J = 4, whose 168 registers allow 3 blocks per SM that four records' 104 KB
// per block would cut to 2.
template <int J>
__host__ __device__ constexpr int cl_stage() {
    return J == 4 ? 2 : 4;
}
template <typename R, int J>
constexpr size_t clump_dyn_smem() {
    return (size_t)CL_WARPS * cl_stage<J>() * 32 * J * sizeof(SlotRec<R>);
}
// J: members each lane keeps in flight per batch of loads (a launch shape
// the autotuner picks; results do not depend on it); a warp stages 32 J
// members in shared memory at a time.  J <= 2 fits 128 registers (4 blocks,
// 16 warps per SM, of which J = 2's 60 KB of shared memory leaves 3) with a
// few bytes of spill; J = 4 keeps 3 blocks per SM.  J = 1 is the default
// (the fastest on the cfg1 and cfg3 states).
// One attitude step (Attitude_clump_cuk, src/dem_integrate_clumpsphere.cu:
// 45-90, the expressions of k_clump's own update): the split driver's bodies
// that turn without their first half-kick use it.
__device__ __forceinline__ double4 quat_step(double4 q, V3<double> w, V3<double> al, double Dt) {
    const V3<double> Wb = rot_w2b(q, w), Wdb = rot_w2b(q, al);
    double4 qd, qdd;
    qd.x = 0.50 * (Wb.x * q.w - Wb.y * q.z + Wb.z * q.y);
    qd.y = 0.50 * (Wb.x * q.z + Wb.y * q.w - Wb.z * q.x);
    qd.z = 0.50 * (-Wb.x * q.y + Wb.y * q.x + Wb.z * q.w);
    qd.w = 0.50 * (-Wb.x * q.x - Wb.y * q.y - Wb.z * q.z);
    qdd.x = (Wdb.x * q.w - Wdb.y * q.z + Wdb.z * q.y) * 0.50 + (Wb.x * qd.w - Wb.y * qd.z + Wb.z * qd.y) * 0.50;
    qdd.y = (Wdb.x * q.z + Wdb.y * q.w - Wdb.z * q.x) * 0.50 + (Wb.x * qd.z + Wb.y * qd.w - Wb.z * qd.x) * 0.50;
    qdd.z = (-Wdb.x * q.y + Wdb.y * q.x + Wdb.z * q.w) * 0.50 + (-Wb.x * qd.y + Wb.y * qd.x + Wb.z * qd.w) * 0.50;
    qdd.w = (-Wdb.x * q.x - Wdb.y * q.y - Wdb.z * q.z) * 0.50 + (-Wb.x * qd.x - Wb.y * qd.y - Wb.z * qd.z) * 0.50;
    const double h2 = 0.5 * Dt * Dt;
    double4 r;
    r.x = (q.x + Dt * qd.x) + h2 * qdd.x;
    r.y = (q.y + Dt * qd.y) + h2 * qdd.y;
    r.z = (q.z + Dt * qd.z) + h2 * qdd.z;
    r.w = (q.w + Dt * qd.w) + h2 * qdd.w;
    const double inv = 1.0 / sqrt(r.x * r.x + r.y * r.y + r.z * r.z + r.w * r.w);
    r.x *= inv; r.y *= inv; r.z *= inv; r.w *= inv;
    return r;
}

// SPH: the build for batches with a sphere-driver scene (ScenePar::sphere);
// the clump path's build carries none of that code.
template <typename R, int J, bool SPH>
__global__ void __launch_bounds__(CL_THREADS, J <= 2 ? 4 : 3) k_clump(const Dev* __restrict__ dp, int do_pre,
                                                      cudaGraphConditionalHandle cond, int use_cond,
                                                      cudaGraphConditionalHandle loop, int use_loop) {
    constexpr int CL_CHUNK = 32 * J;
    __shared__ double s_mf[CL_WARPS][6][CL_CHUNK];   // member force xyz, torque xyz
    __shared__ double s_cl[CL_WARPS][13][32];        // clump position, velocity, angular velocity, quaternion
    __shared__ int s_ms[CL_WARPS][33];               // member-list offsets of the warp's clumps
    __shared__ int s_sc[CL_WARPS][32];               // scene of each of the warp's clumps
    __shared__ int s_pre[CL_WARPS][32];              // the clump's scene takes this step
    extern __shared__ __align__(16) unsigned char cl_dsm[];   // staged contact records
    const Dev& d = *dp;
    if (*d.halt) {
        // a rebuild ran out of pair capacity: the host finishes that step, so
        // a device-side step loop ends here
        if (use_loop && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(loop, 0u);
        return;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int k0 = (blockIdx.x * CL_WARPS + warp) * 32;
    const int t = k0 + lane;
    const int post = *d.post_pending;
    const int L = *d.lstep;   // written only by the last block, after every block has read it
    if (do_pre && blockIdx.x == 0 && threadIdx.x == 0) {
        *d.hgen += 1;
        *d.gstep += 1;
    }
    // warp-uniform: this warp holds clumps of a scene that moves (a warp whose
    // clumps all belong to scenes standing still skips its work)
    const bool stops = d.has_stops;
    bool warp_live = k0 < d.K && !stops;
    if (k0 < d.K && stops) {
        const int nq = min(32, d.K - k0);
        const SceneDyn& yq = d.dyn[d.csid[lane < nq ? t : k0 + nq - 1]];
        warp_live = __any_sync(0xffffffffu, lane < nq && (scene_pre(yq, do_pre, L) || scene_post(yq, post, L)));
    }
    if (warp_live) {
        const int* __restrict__ mem_start = d.mem_start;
        const int* __restrict__ mem_idx = d.mem_idx;
        const double4* __restrict__ posr = d.posr;
        const int nk = min(32, d.K - k0);
        const bool isc = lane < nk;
        const int k = isc ? t : k0 + nk - 1;
        s_ms[warp][lane] = mem_start[k0 + min(lane, nk)];
        if (lane == 0) s_ms[warp][32] = mem_start[k0 + nk];
        const int sc = d.csid[k];
        double4 cp = d.cpos[k], cv = d.cvel[k], cw = d.cw[k], cq = d.cq[k], pr = d.cinv[k];
        const bool pre_k = stops ? scene_pre(d.dyn[sc], do_pre, L) : do_pre != 0;
        const bool post_k = stops ? scene_post(d.dyn[sc], post, L) : post != 0;
        s_sc[warp][lane] = sc;
        s_pre[warp][lane] = isc && pre_k;
        s_cl[warp][0][lane] = cp.x; s_cl[warp][1][lane] = cp.y; s_cl[warp][2][lane] = cp.z;
        __syncwarp();
        const int M0 = s_ms[warp][0], M1 = s_ms[warp][nk];
        const int mb = s_ms[warp][isc ? lane : nk - 1], me = s_ms[warp][isc ? lane + 1 : nk];
        // the warp-local clump of member slot m: mem_cl[m] - k0
        const int* __restrict__ mem_cl = d.mem_cl;
        const ScenePar& P = d.par[sc];
        const double Dt = P.dt;
        V3<double> F, T;
        if (post) {
            // ---- member sums, CL_CHUNK members of the warp's range at a time:
            // each member's contact slots (the contact pass of the last step),
            // its wall and intruder force, and its lever-arm torque
            const R4<R>* __restrict__ fsl = (const R4<R>*)d.nfs;
            const R4<R>* __restrict__ bsl = (const R4<R>*)d.nbs;
            const R4<R>* __restrict__ fbd = (const R4<R>*)d.fbnd;
            const int2* __restrict__ nrb = d.nrb;
            const uint16_t* __restrict__ bbits = d.bbits;
            const size_t N = (size_t)d.N, cap = (size_t)d.cap;
            SlotRec<R>* stage = (SlotRec<R>*)cl_dsm + (size_t)warp * cl_stage<J>() * CL_CHUNK;
            F = v3(0.0, 0.0, 0.0);
            T = F;
            for (int c0 = M0; c0 < M1; c0 += CL_CHUNK) {
                int idx[J], own[J];
#pragma unroll
                for (int j = 0; j < J; j++) {
                    const int m = c0 + 32 * j + lane;
                    idx[j] = m < M1 ? mem_idx[m] : -1;
                    own[j] = m < M1 ? mem_cl[m] - k0 : 0;
                }
                double4 ps[J];
                int r0[J], r1[J], q0[J], q1[J];
                uint16_t bb[J];
#pragma unroll
                for (int j = 0; j < J; j++) {
                    const int i = idx[j] < 0 ? 0 : idx[j];
                    const int ro = i + s_sc[warp][own[j]];
                    ps[j] = posr[i];
                    const int2 ra = nrb[ro], rb = nrb[ro + 1];
                    r0[j] = ra.x;
                    r1[j] = rb.x;
                    q0[j] = ra.y;
                    q1[j] = rb.y;
                    bb[j] = bbits[i];
                }
                // stage every contact record of the lane's members (front
                // slots, back slots, the boundary force) with asynchronous
                // copies: one wait for all of them instead of one per slot
                int nrec = 0;
#pragma unroll
                for (int j = 0; j < J; j++)
                    if (idx[j] >= 0) nrec += (r1[j] - r0[j]) + (q1[j] - q0[j]) + (bb[j] ? 1 : 0);
                int rbase = nrec;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, rbase, o);
                    if (lane >= o) rbase += y;
                }
                rbase -= nrec;
                const bool staged = rbase + nrec <= cl_stage<J>() * CL_CHUNK;
                SlotRec<R>* st = stage + rbase;
                if (staged) {
                    int o = 0;
#pragma unroll
                    for (int j = 0; j < J; j++) {
                        if (idx[j] < 0) continue;
                        for (int e = r0[j]; e < r1[j]; e++, o++) stage_rec<R>(st + o, fsl + 2 * (size_t)e, fsl + 2 * (size_t)e + 1);
                        for (int e = q0[j]; e < q1[j]; e++, o++) stage_rec<R>(st + o, bsl + 2 * (size_t)e, bsl + 2 * (size_t)e + 1);
                        if (bb[j]) { stage_rec<R>(st + o, fbd + idx[j], fbd + N + idx[j]); o++; }
                    }
                    cp_async_wait_all();
                }
                int o = 0;
#pragma unroll
                for (int j = 0; j < J; j++) {
                    if (idx[j] < 0) continue;
                    const int kk = own[j];
                    V3<R> fr, tr;
                    if (staged) {
                        // the order of slot_sum: front slots, back slots, then the boundary force
                        fr = v3<R>(0, 0, 0);
                        tr = fr;
                        const int ns = (r1[j] - r0[j]) + (q1[j] - q0[j]);
#pragma unroll 1
                        for (int e = 0; e < ns; e++, o++) {
                            fr = fr + xyz<R>(st[o].f);
                            tr = tr + xyz<R>(st[o].t);
                        }
                        if (bb[j]) {
                            fr = fr + xyz<R>(st[o].f);
                            tr = tr + xyz<R>(st[o].t);
                            o++;
                        }
                    } else {
                        slot_sum<R>(fsl, bsl, cap, r0[j], r1[j], q0[j], q1[j], fr, tr);
                        if (bb[j]) {
                            fr = fr + xyz<R>(fbd[idx[j]]);
                            tr = tr + xyz<R>(fbd[N + idx[j]]);
                        }
                    }
                    const V3<double> r = v3(ps[j].x - s_cl[warp][0][kk], ps[j].y - s_cl[warp][1][kk],
                                            ps[j].z - s_cl[warp][2][kk]);
                    const V3<double> f = v3((double)fr.x, (double)fr.y, (double)fr.z);
                    const int q = 32 * j + lane;
                    s_mf[warp][0][q] = f.x;
                    s_mf[warp][1][q] = f.y;
                    s_mf[warp][2][q] = f.z;
                    s_mf[warp][3][q] = (double)tr.x + (r.y * f.z - r.z * f.y);
                    s_mf[warp][4][q] = (double)tr.y + (r.z * f.x - r.x * f.z);
                    s_mf[warp][5][q] = (double)tr.z + (r.x * f.y - r.y * f.x);
                }
                __syncwarp();
                if (isc) {
                    const int lo = max(mb, c0), hi = min(me, c0 + CL_CHUNK);
                    for (int m = lo; m < hi; m++) {
                        const int q = m - c0;
                        const V3<double> f = v3(s_mf[warp][0][q], s_mf[warp][1][q], s_mf[warp][2][q]);
                        const V3<double> tc = v3(s_mf[warp][3][q], s_mf[warp][4][q], s_mf[warp][5][q]);
                        if (m == mb) { F = f; T = tc; }
                        else { F = F + f; T = T + tc; }
                    }
                }
                __syncwarp();
            }
            if (isc && post_k) {
                if (mb < me) {
                    if (!(isfinite(F.x) && isfinite(F.y) && isfinite(F.z) && isfinite(T.x) && isfinite(T.y) &&
                          isfinite(T.z)))
                        atomicOr(&d.dyn[sc].err, ERR_NONFINITE);
                    d.cF[k] = make_double4(F.x, F.y, F.z, 0.0);
                    d.cT[k] = make_double4(T.x, T.y, T.z, 0.0);
                } else {
                    F = xyzd(d.cF[k]);
                    T = xyzd(d.cT[k]);
                }
            }
            // split driver: only Type 0 takes the closing half-kick
            // (src/dem_integrate_withglue.cu:140)
            if (post_k && !(SPH && (P.sphere & SPH_KINDS) && (d.kind[k] & 3) != 0)) {
                V3<double> ac = pr.w * F;   // pr: the reciprocals 1/I, 1/M
                ac.z = ac.z + P.gravity;
                V3<double> al = v3(pr.x * T.x, pr.y * T.y, pr.z * T.z);
                cv.x += (0.5 * Dt) * ac.x; cv.y += (0.5 * Dt) * ac.y; cv.z += (0.5 * Dt) * ac.z;
                cw.x += (0.5 * Dt) * al.x; cw.y += (0.5 * Dt) * al.y; cw.z += (0.5 * Dt) * al.z;
            }
        } else {
            F = xyzd(d.cF[k]);
            T = xyzd(d.cT[k]);
        }
        if (do_pre) {
            const double4 cp_old = cp;
            if (SPH && (P.sphere & SPH_KIN) && mb < me) {
                // the sphere drivers' first half-kick and attitude leave the
                // intruder out (src/dem_integrate.cu:20-21,72); one member
                const int i0 = mem_idx[mb];
                if ((d.bbits[i0] >> SLOT_INTR) & 1) {
                    const R4<R>* __restrict__ fi = (const R4<R>*)d.fint;
                    const R4<R> a = fi[i0], b = fi[(size_t)d.N + i0];
                    F = F - v3((double)a.x, (double)a.y, (double)a.z);
                    T = T - v3((double)b.x, (double)b.y, (double)b.z);
                }
            }
            V3<double> ac = pr.w * F;   // pr: the reciprocals 1/I, 1/M
            ac.z = ac.z + P.gravity;
            V3<double> al = v3(pr.x * T.x, pr.y * T.y, pr.z * T.z);
            V3<double> v = xyzd(cv), w = xyzd(cw);
            V3<double> dist = Dt * v + (0.5 * Dt * Dt) * ac;
            cp.x += dist.x; cp.y += dist.y; cp.z += dist.z;
            v = v + (0.5 * Dt) * ac;
            w = w + (0.5 * Dt) * al;
            // attitude with the half-kicked angular velocity
            V3<double> Wb = rot_w2b(cq, w), Wdb = rot_w2b(cq, al);
            double4 q = cq, qd, qdd;
            qd.x = 0.50 * (Wb.x * q.w - Wb.y * q.z + Wb.z * q.y);
            qd.y = 0.50 * (Wb.x * q.z + Wb.y * q.w - Wb.z * q.x);
            qd.z = 0.50 * (-Wb.x * q.y + Wb.y * q.x + Wb.z * q.w);
            qd.w = 0.50 * (-Wb.x * q.x - Wb.y * q.y - Wb.z * q.z);
            qdd.x = (Wdb.x * q.w - Wdb.y * q.z + Wdb.z * q.y) * 0.50 + (Wb.x * qd.w - Wb.y * qd.z + Wb.z * qd.y) * 0.50;
            qdd.y = (Wdb.x * q.z + Wdb.y * q.w - Wdb.z * q.x) * 0.50 + (Wb.x * qd.z + Wb.y * qd.w - Wb.z * qd.x) * 0.50;
            qdd.z = (-Wdb.x * q.y + Wdb.y * q.x + Wdb.z * q.w) * 0.50 + (-Wb.x * qd.y + Wb.y * qd.x + Wb.z * qd.w) * 0.50;
            qdd.w = (-Wdb.x * q.x - Wdb.y * q.y - Wdb.z * q.z) * 0.50 + (-Wb.x * qd.x - Wb.y * qd.y - Wb.z * qd.z) * 0.50;
            const double h2 = 0.5 * Dt * Dt;
            q.x = (q.x + Dt * qd.x) + h2 * qdd.x;
            q.y = (q.y + Dt * qd.y) + h2 * qdd.y;
            q.z = (q.z + Dt * qd.z) + h2 * qdd.z;
            q.w = (q.w + Dt * qd.w) + h2 * qdd.w;
            const double inv = 1.0 / sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
            q.x *= inv; q.y *= inv; q.z *= inv; q.w *= inv;
            if (SPH && (P.sphere & SPH_KINDS)) {
                // split driver (src/dem_integrate_withglue.cu:3-110).  Its call
                // passes the original index where the first half-kick expects
                // Type (src/dem_simulation_split.cu:84-85 against
                // src/dem_integrate_withglue.cu:113-114), so the kick and the
                // move go by the body's original index (bits 2-3: 0 free, 1
                // driven at (-0.2 y, -0.2 x, 0), 2 or more still) and the
                // attitude by its Type (bits 0-1: turns only for Type 0)
                const int kd = d.kind[k], ka = kd & 3, kb = (kd >> 2) & 3;
                if (kb != 0) {
                    cp = cp_old;
                    w = xyzd(cw);
                    v = xyzd(cv);
                    if (kb == 1) {
                        v = v3(-0.2 * cp_old.y, -0.2 * cp_old.x, 0.0);
                        cp.x += Dt * v.x; cp.y += Dt * v.y; cp.z += Dt * v.z;
                    }
                    if (ka == 0) q = quat_step(cq, w, al, Dt);
                }
                if (ka != 0) q = cq;
            }
            if (!pre_k) {   // the scene stands still: keep the clump as it is
                cp = cp_old;
                v = xyzd(cv);
                w = xyzd(cw);
                q = cq;
            }
            if (isc && pre_k) {
                d.cpos[k] = cp;
                d.cvel[k] = make_double4(v.x, v.y, v.z, 0.0);
                d.cw[k] = make_double4(w.x, w.y, w.z, 0.0);
                d.cq[k] = q;
            }
            __syncwarp();   // the old positions in s_cl are no longer read
            s_cl[warp][0][lane] = cp.x; s_cl[warp][1][lane] = cp.y; s_cl[warp][2][lane] = cp.z;
            s_cl[warp][3][lane] = v.x; s_cl[warp][4][lane] = v.y; s_cl[warp][5][lane] = v.z;
            s_cl[warp][6][lane] = w.x; s_cl[warp][7][lane] = w.y; s_cl[warp][8][lane] = w.z;
            s_cl[warp][9][lane] = q.x; s_cl[warp][10][lane] = q.y; s_cl[warp][11][lane] = q.z;
            s_cl[warp][12][lane] = q.w;
            __syncwarp();
            // ---- poses of the members, 32 at a time
            double4* __restrict__ kv = (double4*)d.kin;   // per member: world arm, mass
            const double4* __restrict__ lom = d.lom;
            double4* __restrict__ cum = d.cum;
            double4* __restrict__ posw = d.posr;
            // J members per lane at a time: all indices, then all member
            // records, in flight together
            constexpr int JP = J;
            for (int c0 = M0; c0 < M1; c0 += 32 * JP) {
                int idx[JP], own[JP];
#pragma unroll
                for (int j = 0; j < JP; j++) {
                    const int m = c0 + 32 * j + lane;
                    idx[j] = m < M1 ? mem_idx[m] : -1;
                    own[j] = m < M1 ? mem_cl[m] - k0 : 0;
                }
                double4 lo[JP], old[JP], cu[JP];
#pragma unroll
                for (int j = 0; j < JP; j++) {
                    const int i = idx[j] < 0 ? 0 : idx[j];
                    lo[j] = lom[i];
                    old[j] = posw[i];
                    cu[j] = cum[i];
                }
#pragma unroll
                for (int j = 0; j < JP; j++) {
                    if (idx[j] < 0) continue;
                    const int i = idx[j];
                    const int kk = own[j];
                    if (!s_pre[warp][kk]) continue;
                    const double4 qk = make_double4(s_cl[warp][9][kk], s_cl[warp][10][kk], s_cl[warp][11][kk],
                                                    s_cl[warp][12][kk]);
                    const V3<double> arm = rot_b2w(qk, v3(lo[j].x, lo[j].y, lo[j].z));
                    const V3<double> p = v3(s_cl[warp][0][kk] + arm.x, s_cl[warp][1][kk] + arm.y,
                                            s_cl[warp][2][kk] + arm.z);
                    const double4 c = cu[j], o = old[j];
                    const V3<double> cn = v3((c.x + p.x) - o.x, (c.y + p.y) - o.y, (c.z + p.z) - o.z);
                    const V3<double> vk = v3(s_cl[warp][3][kk], s_cl[warp][4][kk], s_cl[warp][5][kk]);
                    const V3<double> wk = v3(s_cl[warp][6][kk], s_cl[warp][7][kk], s_cl[warp][8][kk]);
                    cum[i] = make_double4(cn.x, cn.y, cn.z, 0.0);
                    posw[i] = make_double4(p.x, p.y, p.z, o.w);
                    kv[i] = make_double4(arm.x, arm.y, arm.z, lo[j].w);
                    const int sk = s_sc[warp][kk];
                    double thr = d.par[sk].thresh;
                    if (SPH && (d.par[sk].sphere & SPH_KINDS))   // split driver: the free body of the first
                        thr = ((d.kind[k0 + kk] >> 2) & 3) == 0 ? 0.10 * o.w : INFINITY;   // half-kick at 0.1 r
                                                                  // (src/dem_integrate_withglue.cu:41)
                    if (len_floor(cn) > thr) {
                        SceneDyn& y = d.dyn[sk];
                        if (!*(volatile int*)&y.rebuild) atomicExch(&y.rebuild, 1);
                        if (!*(volatile int*)d.any_rebuild) atomicExch(d.any_rebuild, 1);
                    }
                }
            }
        }
        if (isc && post_k && !pre_k) {   // closing half-kick only (sync, or the scene's last step)
            d.cvel[k] = cv;
            d.cw[k] = cw;
        }
    }
    if (t >= d.K && t < d.K + d.S) {
        const int s = t - d.K;
        const ScenePar& P = d.par[s];
        SceneDyn& y = d.dyn[s];
        const double Dt = P.dt;
        const bool pre_s = scene_pre(y, do_pre, L), post_s = scene_post(y, post, L);
        if (post_s) {
            long long* fx = (long long*)&y.ifix[0];
            V3<double> tf = v3(fx[0] / FIX_F, fx[1] / FIX_F, fx[2] / FIX_F);
            V3<double> tt = v3(fx[3] / FIX_T, fx[4] / FIX_T, fx[5] / FIX_T);
            for (int c = 0; c < 6; c++) fx[c] = 0;
            y.totF[0] = tf.x; y.totF[1] = tf.y; y.totF[2] = tf.z;
            y.totT[0] = tt.x; y.totT[1] = tt.y; y.totT[2] = tt.z;
            if (P.has_intr) {
                if (P.intr_wait && y.intr_state == 1) y.intr_state = 2;
                V3<double> reac = v3(-tf.x, -tf.y, -tf.z);
                if (P.intr_motion == 1 && (!P.intr_wait || y.intr_state != 0)) {
                    V3<double> a = (1.0 / P.intr_mass) * reac;
                    a.z = a.z + P.gravity;
                    for (int c = 0; c < 3; c++) y.intr_v[c] += (0.5 * Dt) * (&a.x)[c];
                }
                y.reaction[0] = reac.x; y.reaction[1] = reac.y; y.reaction[2] = reac.z;
                y.reaction_t[0] = tt.x; y.reaction_t[1] = tt.y; y.reaction_t[2] = tt.z;
                double* ring = d.ring + ((size_t)s * d.ring_len + (y.step % d.ring_len)) * 6;
                ring[0] = reac.x; ring[1] = reac.y; ring[2] = reac.z;
                ring[3] = tt.x; ring[4] = tt.y; ring[5] = tt.z;
            }
            y.step += 1;
        }
        if (do_pre) y.frozen = !pre_s;
        if (pre_s && P.has_intr) {
            if (P.intr_motion == 1 && (!P.intr_wait || y.intr_state != 0)) {
                V3<double> a = (-1.0 / P.intr_mass) * v3(y.totF[0], y.totF[1], y.totF[2]);
                a.z = a.z + P.gravity;
                for (int c = 0; c < 3; c++) {
                    y.intr_p[c] = (y.intr_p[c] + Dt * y.intr_v[c]) + (0.5 * Dt * Dt) * (&a.x)[c];
                    y.intr_v[c] = y.intr_v[c] + (0.5 * Dt) * (&a.x)[c];
                }
            } else {
                for (int c = 0; c < 3; c++) y.intr_p[c] = y.intr_p[c] + Dt * y.intr_v[c];
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(d.kc_done, 1) == (int)gridDim.x - 1) {
            *d.kc_done = 0;
            if (do_pre) *d.lstep = L + 1;
            if (use_cond) cudaGraphSetConditional(cond, atomicAdd(d.any_rebuild, 0) ? 1u : 0u);
            if (use_loop) {
                const int left = *d.loop_left - 1;
                *d.loop_left = left;
                cudaGraphSetConditional(loop, left > 0 ? 1u : 0u);
            }
        }
    }
}

// The steps a graph launch with a device-side step loop takes (the first
// node of that graph; its argument is set before each launch).
static __global__ void k_loop_init(int* __restrict__ left, int n) { *left = n; }

// ===========================================================================
// broad phase
// ===========================================================================

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// A rebuild runs over the rebuilt scenes only.  k_plan lists them (ascending)
// with prefix sums of their subsphere, cell-table and clump counts; a rebuild
// kernel walks the concatenation of the rebuilt scenes with a grid-stride
// loop and finds the scene of an element by binary search in the prefix.
// Scenes that are not rebuilt keep their order, list region and histories
// untouched, so a rebuild costs in proportion to the scenes it rebuilds.
//
// plan_find: the k in [0, n) with pre[k] <= t < pre[k + 1] (empty scenes are
// passed over).
__device__ __forceinline__ int plan_find(const int* __restrict__ pre, int n, int t) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int m = (lo + hi + 1) >> 1;
        if (pre[m] <= t) lo = m;
        else hi = m - 1;
    }
    return lo;
}

// --- exclusive scan of ints (three passes) --------------------------------
// The length is n, or *dn when dn is given (a count computed on the device);
// the kernels walk the tiles with grid-stride loops, so a fixed grid serves
// any length.
constexpr int SC_THREADS = 256, SC_ITEMS = 4, SC_TILE = SC_THREADS * SC_ITEMS;

// Exclusive scan over a block of NT threads (every thread calls it); sh:
// NT/32 ints.
template <int NT = SC_THREADS>
__device__ __forceinline__ int block_excl_scan(int v, int* sh, int& total) {
    static_assert(NT % 32 == 0 && NT <= 1024, "whole warps, at most 32");
    constexpr int NW = NT / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < NW ? sh[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < NW) sh[lane] = w;
    }
    __syncthreads();
    const int warp_base = warp > 0 ? sh[warp - 1] : 0;
    total = sh[NW - 1];
    __syncthreads();
    return warp_base + x - v;
}

static __global__ void __launch_bounds__(SC_THREADS) k_scan_tiles(int* __restrict__ a, int n, int* __restrict__ sums,
                                                           const int* __restrict__ dn) {
    __shared__ int sh[SC_THREADS / 32];
    const int nn = dn ? *dn : n;
    const int tiles = (nn + SC_TILE - 1) / SC_TILE;
    for (int b = blockIdx.x; b < tiles; b += gridDim.x) {
        const int base = b * SC_TILE + threadIdx.x * SC_ITEMS;
        int v[SC_ITEMS], s = 0;
        for (int j = 0; j < SC_ITEMS; j++) { v[j] = base + j < nn ? a[base + j] : 0; s += v[j]; }
        int total;
        int ex = block_excl_scan(s, sh, total);
        for (int j = 0; j < SC_ITEMS; j++) {
            if (base + j < nn) a[base + j] = ex;
            ex += v[j];
        }
        if (threadIdx.x == 0) sums[b] = total;
    }
}

static __global__ void __launch_bounds__(SC_THREADS) k_scan_sums(int* __restrict__ sums, int nb, const int* __restrict__ dn) {
    __shared__ int sh[SC_THREADS / 32];
    if (dn) nb = (*dn + SC_TILE - 1) / SC_TILE;
    int carry = 0;
    for (int off = 0; off < nb; off += SC_THREADS) {
        int i = off + threadIdx.x;
        int v = i < nb ? sums[i] : 0;
        int total;
        int ex = block_excl_scan(v, sh, total);
        if (i < nb) sums[i] = carry + ex;
        carry += total;
    }
}

static __global__ void __launch_bounds__(SC_THREADS) k_scan_add(int* __restrict__ a, int n, const int* __restrict__ sums,
                                                         const int* __restrict__ dn) {
    const int nn = dn ? *dn : n;
    const int tiles = (nn + SC_TILE - 1) / SC_TILE;
    for (int b = blockIdx.x; b < tiles; b += gridDim.x) {
        const int base = b * SC_TILE + threadIdx.x * SC_ITEMS;
        const int add = sums[b];
        for (int j = 0; j < SC_ITEMS; j++)
            if (base + j < nn) a[base + j] += add;
    }
}

// --- exclusive scan of ints in one launch (decoupled look-back) ----------
// One to three arrays of the same length (n, or *dn) in one launch.  Blocks
// take tiles from a ticket counter until none is left: tickets [0, tiles)
// are the tiles of the first array, [tiles, 2 tiles) those of the second,
// and so on.  A tile
// publishes its aggregate, then looks back over its array's earlier tiles
// (32 at a time, one per lane of warp 0) and sums aggregates until it meets
// an inclusive prefix, and publishes its own inclusive prefix.  A block
// takes its next ticket only after finishing its tile, so a tile waits only
// on tiles held by blocks that are running: the wait always ends.  Each wait is still
// bounded (SCAN_SPIN_LIMIT polls); a block that gives up sets *fail and
// *halt, so every later kernel of the step returns at once and the host
// reports the failure instead of using the result.  The last block of the
// grid clears the tile states and the counters for the next scan.
// ctl: [0] ticket counter, [1] finished blocks.  st: one word per ticket,
// (state << 32) | value, state 1 = aggregate, 2 = inclusive prefix.
constexpr unsigned long long SCAN_AGG = 1ull << 32, SCAN_INC = 2ull << 32;
constexpr int SCAN_SPIN_LIMIT = 1 << 22;

static __global__ void __launch_bounds__(SC_THREADS) k_scan1(int* __restrict__ a0, int* __restrict__ a1,
                                                            int* __restrict__ a2, int n, const int* __restrict__ dn,
                                                            unsigned long long* __restrict__ st, int* __restrict__ ctl,
                                                            int* __restrict__ halt, int* __restrict__ fail) {
    __shared__ int sh[SC_THREADS / 32];
    __shared__ int s_ticket, s_excl, s_last;
    const int nn = dn ? *dn : n;
    const int tiles = (nn + SC_TILE - 1) / SC_TILE;
    const int narr = a2 ? 3 : (a1 ? 2 : 1);
    // a fixed grid takes tiles until none is left (the grid is set when the
    // launch is captured; the tile count is known only on the device)
    for (;;) {
        if (threadIdx.x == 0) s_ticket = atomicAdd(&ctl[0], 1);
        __syncthreads();
        const int tk = s_ticket;
        __syncthreads();
        if (tk >= narr * tiles) break;
        const int arr = tk / tiles;
        const int b = tk - arr * tiles;      // tile of its array
        int* __restrict__ a = arr == 0 ? a0 : (arr == 1 ? a1 : a2);
        unsigned long long* __restrict__ sa = st + (size_t)arr * tiles;
        const int base = b * SC_TILE + threadIdx.x * SC_ITEMS;
        int v[SC_ITEMS], sum = 0;
#pragma unroll
        for (int j = 0; j < SC_ITEMS; j++) { v[j] = base + j < nn ? a[base + j] : 0; sum += v[j]; }
        int total;
        int ex = block_excl_scan(sum, sh, total);
        if (threadIdx.x < 32) {
            const int lane = threadIdx.x;
            int excl = 0;
            if (b == 0) {
                if (lane == 0) atomicExch(&sa[0], SCAN_INC | (unsigned)total);
            } else {
                if (lane == 0) atomicExch(&sa[b], SCAN_AGG | (unsigned)total);
                bool ok = true;
                for (int j = b - 1;; j -= 32) {
                    const int t = j - lane;
                    unsigned long long w = SCAN_INC;   // before the first tile: an inclusive zero
                    if (t >= 0) {
                        int polls = 0;
                        while (((w = *(volatile unsigned long long*)&sa[t]) >> 32) == 0) {
                            if (++polls > SCAN_SPIN_LIMIT) { ok = false; w = SCAN_INC; break; }
                            __nanosleep(64);
                        }
                    }
                    const unsigned inc = __ballot_sync(0xffffffffu, (w >> 32) == 2);
                    const int upto = inc ? __ffs(inc) - 1 : 31;   // the nearest inclusive prefix ends the sum
                    int c = lane <= upto ? (int)(unsigned)w : 0;
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
                    excl += c;
                    if (inc) break;
                }
                if (!__all_sync(0xffffffffu, ok) && lane == 0) {
                    atomicExch(fail, 1);
                    atomicExch(halt, 1);
                }
                if (lane == 0) atomicExch(&sa[b], SCAN_INC | (unsigned)(excl + total));
            }
            if (lane == 0) s_excl = excl;
        }
        __syncthreads();
        ex += s_excl;
#pragma unroll
        for (int j = 0; j < SC_ITEMS; j++) {
            if (base + j < nn) a[base + j] = ex;
            ex += v[j];
        }
    }
    // every block has taken its ticket and is done with the tile states
    // once the finished count reaches the grid: the last one resets them
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(&ctl[1], 1) == (int)gridDim.x - 1;
    }
    __syncthreads();
    if (s_last) {
        for (int k = threadIdx.x; k < narr * tiles; k += SC_THREADS) st[k] = 0ull;
        if (threadIdx.x == 0) {
            ctl[0] = 0;
            ctl[1] = 0;
        }
    }
}

// --- LSD radix sort, 8-bit digits, stable (the reference sorts with CUB's
// stable DeviceRadixSort, src/dem_grid.cu:278-305); the allocation-free
// sort (noalloc.cu) uses it, the engine's rebuild sorts by counting --------
constexpr int RS_THREADS = 256, RS_ITEMS = 8, RS_TILE = RS_THREADS * RS_ITEMS;

// The plan of a rebuild (one block).  Rebuilt scenes are listed in ascending
// order; their cell keys (cell_off + local cell) ascend with the scene, so
// sorting the concatenation of their subspheres keeps every scene in its own
// range.
static __global__ void __launch_bounds__(SC_THREADS) k_plan(const Dev* __restrict__ dp) {
    __shared__ int sh[SC_THREADS / 32];
    const Dev& d = *dp;
    if (*d.halt) return;
    int ns = 0, nsub = 0, ncell = 0, nclump = 0;
    for (int b = 0; b < d.S; b += SC_THREADS) {
        const int s = b + threadIdx.x;
        const bool f = s < d.S && d.dyn[s].rebuild;
        int a1 = 0, a2 = 0, a3 = 0;
        if (f) {
            const ScenePar& P = d.par[s];
            a1 = P.nsub;
            a2 = P.cellnum + 1;
            a3 = P.nclump;
        }
        if (s < d.S) d.need[s] = -1;
        int t0, t1, t2, t3;
        const int e0 = block_excl_scan(f ? 1 : 0, sh, t0);
        const int e1 = block_excl_scan(a1, sh, t1);
        const int e2 = block_excl_scan(a2, sh, t2);
        const int e3 = block_excl_scan(a3, sh, t3);
        if (f) {
            d.pscene[ns + e0] = s;
            d.psub[ns + e0] = nsub + e1;
            d.pcell[ns + e0] = ncell + e2;
            d.pclump[ns + e0] = nclump + e3;
        }
        ns += t0;
        nsub += t1;
        ncell += t2;
        nclump += t3;
    }
    if (threadIdx.x == 0) {
        d.psub[ns] = nsub;
        d.pcell[ns] = ncell;
        d.pclump[ns] = nclump;
        d.plan[PL_NS] = ns;
        d.plan[PL_T] = nsub;
        d.plan[PL_TC] = ncell;
        d.plan[PL_T1] = nsub + 1;
        d.plan[PL_TK] = nclump;
        d.plan[PL_CS] = 0;
        d.plan[PL_CC] = 0;
        d.plan[PL_TC1] = ncell + 1;
    }
}

#define NBC_GRID_STRIDE(t, n) for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < (n); t += gridDim.x * blockDim.x)

// GetParticleCellIndex_cuk (src/dem_grid.cu:155-202); hierarchical variant
// GetParticleCellIndex_hGrid_cuk (src/dem_hgrid.cu:205-242) with the
// out-of-box bucket kept inside the scene's cell range.  Element t of the
// rebuilt concatenation: kA[t] = its cell's index u in the rebuilt scenes'
// cell table (pcell[k] + local cell), vA[t] = its subsphere; ccnt[u] counts
// the cell's subspheres.
//
// The stable sort by cell (the reference sorts with CUB's stable radix
// sort, src/dem_grid.cu:278-305) is a counting sort: the scan of ccnt gives
// each cell's first sorted slot, k_cscatter drops every element into its
// cell's range, and k_cellfix puts each cell's range back in ascending
// subsphere order -- the order a stable sort keeps -- and writes the
// permutation, its inverse, the sorted keys and the cell table.
static __global__ void k_hash(const Dev* __restrict__ dp) {
    const Dev& d = *dp;
    if (*d.halt) return;
    const int T = d.plan[PL_T], ns = d.plan[PL_NS];
    NBC_GRID_STRIDE(t, T) {
        const int k = plan_find(d.psub, ns, t);
        const ScenePar& P = d.par[d.pscene[k]];
        const int i = P.sub_off + (t - d.psub[k]);
        d.vA[t] = i;
        const double4 p = d.posr[i];
        int local;
        if (P.levels <= 1) {
            if (p.z >= P.box_hi[2] || p.y >= P.box_hi[1] || p.x >= P.box_hi[0] ||
                p.z < P.box_lo[2] || p.y < P.box_lo[1] || p.x < P.box_lo[0]) {
                local = P.cellnum - 1;
            } else {
                int cx = (int)floor((p.x - P.origin[0]) / P.cell[0]);
                int cy = (int)floor((p.y - P.origin[1]) / P.cell[1]);
                int cz = (int)floor((p.z - P.origin[2]) / P.cell[2]);
                cx = clampi(cx, 0, P.gdim[0] - 1);
                cy = clampi(cy, 0, P.gdim[1] - 1);
                cz = clampi(cz, 0, P.gdim[2] - 1);
                local = cz * P.gdim[1] * P.gdim[0] + cy * P.gdim[0] + cx;
                local = clampi(local, 0, P.cellnum - 1);
            }
        } else {
            if (p.z > P.box_hi[2] || p.y > P.box_hi[1] || p.x > P.box_hi[0] ||
                p.z < P.box_lo[2] || p.y < P.box_lo[1] || p.x < P.box_lo[0]) {
                local = P.cellnum - 1;
            } else {
                const int lv = d.level[i];
                const double c = P.lcell[lv];
                const int cx = clampi((int)floor((p.x - P.origin[0]) / c), 0, P.ldim[lv][0] - 1);
                const int cy = clampi((int)floor((p.y - P.origin[1]) / c), 0, P.ldim[lv][1] - 1);
                const int cz = clampi((int)floor((p.z - P.origin[2]) / c), 0, P.ldim[lv][2] - 1);
                local = P.loff[lv] + (cz * P.ldim[lv][1] * P.ldim[lv][0] + cy * P.ldim[lv][0] + cx);
            }
        }
        // the cell's index in the rebuilt scenes' cell table, and its count
        const int u = d.pcell[k] + local;
        d.kA[t] = u;
        atomicAdd(&d.ccnt[u], 1);
    }
}

// every element into its cell's range (in any order within the cell)
static __global__ void k_cscatter(const Dev* __restrict__ dp) {
    const Dev& d = *dp;
    if (*d.halt) return;
    const int T = d.plan[PL_T];
    NBC_GRID_STRIDE(t, T) {
        const int u = d.kA[t];
        d.vB[d.ccnt[u] + atomicAdd(&d.ccur[u], 1)] = d.vA[t];
    }
}

// Per cell of the rebuilt scenes: its range of the sorted order in
// ascending subsphere order (insertion sort; ranges longer than 32 -- the
// out-of-box bucket of a scene that has lost subspheres -- by Shell sort),
// then the permutation, its inverse and the sorted keys (key2) at the
// range's subsphere slots and the cell's start in the cell table (the entry
// after a scene's last cell is the next scene's first slot).  The cursors
// go back to zero for the next rebuild.
static __global__ void k_cellfix(const Dev* __restrict__ dp) {
    const Dev& d = *dp;
    if (*d.halt) return;
    const int TC = d.plan[PL_TC], ns = d.plan[PL_NS];
    int* __restrict__ v = d.vB;
    NBC_GRID_STRIDE(u, TC) {
        const int k = plan_find(d.pcell, ns, u);
        const ScenePar& P = d.par[d.pscene[k]];
        const int c = P.cell_off + (u - d.pcell[k]);
        const int a = d.ccnt[u], b = d.ccnt[u + 1];
        const int base = P.sub_off - d.psub[k];   // subsphere slot of sorted position t: base + t
        d.cstart[c] = base + a;
        d.ccur[u] = 0;
        if (b - a <= 32) {
            for (int x = a + 1; x < b; x++) {
                const int w = v[x];
                int y = x - 1;
                while (y >= a && v[y] > w) { v[y + 1] = v[y]; y--; }
                v[y + 1] = w;
            }
        } else {
            int gap = 1;
            while (gap < (b - a) / 3) gap = 3 * gap + 1;
            for (; gap > 0; gap /= 3)
                for (int x = a + gap; x < b; x++) {
                    const int w = v[x];
                    int y = x - gap;
                    while (y >= a && v[y] > w) { v[y + gap] = v[y]; y -= gap; }
                    v[y + gap] = w;
                }
        }
        for (int t = a; t < b; t++) {
            const int i = base + t, o = v[t];
            d.inv[o] = i;
            d.perm[i] = o;
            d.key2[i] = c;
        }
    }
}

// Tiles of RS_TILE keys, n keys (or *dn); the histogram of tile b, digit v
// sits at hist[v * tiles + b].  Grid-stride over the tiles.
static __global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const int* __restrict__ keys, int n, int shift,
                                                        int* __restrict__ hist, const int* __restrict__ dn) {
    __shared__ int h[256];
    const int tid = threadIdx.x;
    const int nn = dn ? *dn : n;
    const int tiles = (nn + RS_TILE - 1) / RS_TILE;
    for (int blk = blockIdx.x; blk < tiles; blk += gridDim.x) {
        h[tid] = 0;
        __syncthreads();
        for (int it = 0; it < RS_ITEMS; it++) {
            const int idx = blk * RS_TILE + it * RS_THREADS + tid;
            if (idx < nn) atomicAdd(&h[(keys[idx] >> shift) & 255], 1);
        }
        __syncthreads();
        hist[tid * tiles + blk] = h[tid];
        __syncthreads();
    }
}

static __global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(const int* __restrict__ kin, const int* __restrict__ vin,
                                                           int* __restrict__ kout, int* __restrict__ vout, int n,
                                                           int shift, const int* __restrict__ hist,
                                                           const int* __restrict__ dn) {
    __shared__ int base[256];
    __shared__ int wcnt[RS_THREADS / 32][257];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nn = dn ? *dn : n;
    const int tiles = (nn + RS_TILE - 1) / RS_TILE;
    for (int blk = blockIdx.x; blk < tiles; blk += gridDim.x) {
        base[tid] = hist[tid * tiles + blk];
        for (int it = 0; it < RS_ITEMS; it++) {
            for (int w = 0; w < RS_THREADS / 32; w++) wcnt[w][tid] = 0;
            __syncthreads();
            const int idx = blk * RS_TILE + it * RS_THREADS + tid;
            const bool valid = idx < nn;
            const int k = valid ? kin[idx] : 0;
            const int dig = valid ? ((k >> shift) & 255) : 256;
            const unsigned peers = __match_any_sync(0xffffffffu, dig);
            const int rank = __popc(peers & ((1u << lane) - 1u));
            if (valid && lane == __ffs(peers) - 1) wcnt[warp][dig] = __popc(peers);
            __syncthreads();
            if (valid) {
                int off = base[dig] + rank;
                for (int w = 0; w < warp; w++) off += wcnt[w][dig];
                kout[off] = k;
                vout[off] = vin[idx];
            }
            __syncthreads();
            int add = 0;
            for (int w = 0; w < RS_THREADS / 32; w++) add += wcnt[w][tid];
            base[tid] += add;
            __syncthreads();
        }
    }
}

// --- reorder and cell table ---------------------------------------------
// SortArray_*_cuk (src/dem_grid.cu:336-437) for every persistent per-subsphere
// array at once, into the alternate buffers (written back by k_writeback).
// The displacement accumulator restarts at zero (src/dem_simulation_clump.cu:172).
template <typename R>
__global__ void k_reorder(const Dev* __restrict__ dp) {
    const Dev& d = *dp;
    if (*d.halt) return;
    const int T = d.plan[PL_T], ns = d.plan[PL_NS];
    const size_t N = (size_t)d.N;
    {
        // the sort's cell counts back to zero for the next rebuild
        const int TC1 = d.plan[PL_TC1];
        NBC_GRID_STRIDE(u, TC1) d.ccnt[u] = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) { d.cnt_f[T] = 0; d.cnt_b[T] = 0; }
    NBC_GRID_STRIDE(t, T) {
        // the search's counters start at zero
        d.cnt_f[t] = 0;
        d.cnt_b[t] = 0;
        d.xcnt[t] = 0;
        const int k = plan_find(d.psub, ns, t);
        const int i = d.par[d.pscene[k]].sub_off + (t - d.psub[k]);
        const int o = d.perm[i];
        d.posr2[i] = d.posr[o];
        d.lom2[i] = d.lom[o];
        d.cum2[i] = make_double4(0, 0, 0, 0);
        d.clump_id2[i] = d.clump_id[o];
        d.part_fix2[i] = d.part_fix[o];
        d.level2[i] = d.level[o];
        d.bbits2[i] = d.bbits[o];
        ((double4*)d.kin2)[i] = ((const double4*)d.kin)[o];
        const R4<R>* b1 = (const R4<R>*)d.bhist;
        R4<R>* b2 = (R4<R>*)d.bhist2;
        const uint16_t bits = d.bbits[o];
        for (int sl = 0; sl < NB_SLOTS; sl++) {
            if (!(bits & (1u << sl))) continue;  // only live histories are ever read
            for (int c = 0; c < 3; c++) b2[((size_t)sl * N + i) * 3 + c] = b1[((size_t)sl * N + o) * 3 + c];
        }
    }
}

// --- neighbour search ----------------------------------------------------
// The candidate test and the order of CreateAnei_cuk (src/dem_grid.cu:466-552):
// cells in z, y, x order over -1..1, partners ascending within a cell,
// candidate if |xi - xj|^2 < (1.5 (ri + rj))^2 in FP64; j > i goes to the
// front (owner) row of i, j < i to its back row.
//
// Hierarchical grid (CreateAnei_hGrid_cuk, src/dem_hgrid_contlist.cu:57-161):
// a subsphere searches its own level and every coarser one (level 0 is the
// coarsest); a pair across levels is owned by the coarser subsphere: the
// finer one records a back entry, the coarser one a front entry, placed after
// its same-level front entries in ascending order of the finer partner.
//
// A group of SL lanes searches for one subsphere.  The three x-neighbour
// cells of one (z, y) stencil row hold one contiguous range of the sorted
// order, [cstart[first cell], cstart[last cell + 1]), so a subsphere on level
// t visits 9 (t + 1) ranges.  The lanes first resolve all ranges at once
// (each lane a contiguous chunk of rows), prefix-sum their lengths, and then
// walk the concatenation of the ranges SL candidates at a time: the
// concatenation is the discovery order, and hits are appended in it through
// ballot prefixes.  One pass both counts and stores the hits: into a
// fixed-size scratch row per subsphere (the fused search), or, for rows too
// long for the scratch, straight into the final list once its offsets are
// known (the fallback of k_compact).
constexpr int SEARCH_THREADS = 128;
constexpr int SCR_CAP = 32;                   // scratch entries per front row and per back row
constexpr int CROSS_TAG = 0x40000000;         // scratch only: back entry whose partner is coarser
constexpr int MAX_ROWS = 9 * MAX_LEVELS;

template <int SL>
struct SearchShared {
    int rs[SEARCH_THREADS / SL][MAX_ROWS];        // first sorted index of each stencil row
    int pre[SEARCH_THREADS / SL][MAX_ROWS + 1];   // exclusive prefix of the row lengths
};

// FILL = false: count the hits and store them in subsphere i's scratch rows,
// count cross-level entries into the coarser partner's cnt_f.  FILL = true:
// write the hits into the list rows at the scanned offsets and claim the
// cross-level slots of the coarser partners.  The counts of subsphere j sit
// at j + tb (its element of the rebuilt concatenation); a front row starts at
// slot cnt_f[j + tb] + poff, a back row at cnt_b[j + tb] + boff.
template <bool FILL, int SL>
__device__ __forceinline__ void group_search(const Dev& d, const ScenePar& P, const PairList& Nw, int i, int lane,
                                             int* __restrict__ rs, int* __restrict__ pre, int tb, int poff, int boff,
                                             int& nf_out, int& nb_out) {
    // buffer pointers in registers: the stores below could otherwise alias
    // the pointer table and force it to be re-read on every candidate
    const double4* __restrict__ posr = d.posr2;
    const int* __restrict__ cid = d.clump_id2;
    const int* __restrict__ cstart = d.cstart;
    int* __restrict__ cnt_f = d.cnt_f;
    int* __restrict__ xcnt = d.xcnt;
    const int* __restrict__ sfc = d.sfc;
    int* __restrict__ nbr = Nw.nbr;
    int* __restrict__ own = Nw.own;
    int* __restrict__ bnbr = Nw.bnbr;
    const unsigned gm = SL == 32 ? 0xffffffffu : (((1u << SL) - 1u) << ((threadIdx.x & 31) & ~(SL - 1)));
    const int gshift = (threadIdx.x & 31) & ~(SL - 1);
    __syncwarp(gm);  // the group's previous subsphere is done with rs / pre
    const double4 pi = posr[i];
    const int ci = cid[i];
    const int my = P.levels > 1 ? d.level2[i] : 0;
    const int nrows = 9 * (my + 1);
    // ---- ranges of the stencil rows: lane k resolves rows [k C, k C + C)
    {
        constexpr int MAXC = (MAX_ROWS + SL - 1) / SL;
        const int C = (nrows + SL - 1) / SL;
        const int r0 = min(lane * C, nrows), r1 = min(r0 + C, nrows);
        // the cells of the lane's rows first, then all their cstart loads at
        // once (the rows are independent), then the lengths
        int ca[MAXC], cb[MAXC];
        int lc = -1, gx = 0, gy = 0, gz = 0, base = 0, cx0 = 0, cy0 = 0, cz0 = 0;
#pragma unroll
        for (int k = 0; k < MAXC; k++) {
            const int r = r0 + k;
            ca[k] = -1;
            cb[k] = -1;
            if (r >= r1) continue;
            const int l = my - r / 9, rr = r % 9;
            if (l != lc) {
                lc = l;
                if (P.levels <= 1) {
                    gx = P.gdim[0]; gy = P.gdim[1]; gz = P.gdim[2];
                    base = P.cell_off;
                    cx0 = (int)floor((pi.x - P.origin[0]) * P.icell[0]);
                    cy0 = (int)floor((pi.y - P.origin[1]) * P.icell[1]);
                    cz0 = (int)floor((pi.z - P.origin[2]) * P.icell[2]);
                } else {
                    gx = P.ldim[l][0]; gy = P.ldim[l][1]; gz = P.ldim[l][2];
                    base = P.cell_off + P.loff[l];
                    const double c = P.lcell[l];
                    cx0 = (int)floor((pi.x - P.origin[0]) / c);
                    cy0 = (int)floor((pi.y - P.origin[1]) / c);
                    cz0 = (int)floor((pi.z - P.origin[2]) / c);
                }
            }
            const int z = cz0 + rr / 3 - 1, y = cy0 + rr % 3 - 1;
            const int xa = max(cx0 - 1, 0), xb = min(cx0 + 1, gx - 1);
            if (xa <= xb && z >= 0 && z < gz && y >= 0 && y < gy) {
                const int c0 = base + (z * gy + y) * gx;
                ca[k] = c0 + xa;
                cb[k] = c0 + xb + 1;
            }
        }
#pragma unroll
        for (int k = 0; k < MAXC; k++) {
            if (ca[k] >= 0) {
                ca[k] = cstart[ca[k]];
                cb[k] = cstart[cb[k]];
            }
        }
        int acc = 0;
#pragma unroll
        for (int k = 0; k < MAXC; k++) {
            const int r = r0 + k;
            if (r >= r1) continue;
            const int s = ca[k] >= 0 ? ca[k] : 0, n = ca[k] >= 0 ? cb[k] - ca[k] : 0;
            rs[r] = s;
            pre[r] = acc;
            acc += n;
        }
        int inc = acc;
#pragma unroll
        for (int o = 1; o < SL; o <<= 1) {
            const int v = __shfl_up_sync(gm, inc, o, SL);
            if (lane >= o) inc += v;
        }
        const int ex = inc - acc;
        for (int r = r0; r < r1; r++) pre[r] += ex;
        const int total = __shfl_sync(gm, inc, SL - 1, SL);
        if (lane == 0) pre[nrows] = total;
        __syncwarp(gm);
    }
    const int total = pre[nrows];
    // ---- candidates in discovery order, SL at a time; the next batch's
    // positions are loaded before the current batch is tested
    const unsigned lt = (1u << lane) - 1u;
    int nf = 0, nb = 0;
    const int rf = FILL ? cnt_f[i + tb] + poff : 0, rb = FILL ? d.cnt_b[i + tb] + boff : 0;
    int* __restrict__ scr_f = d.scr + (size_t)i * (2 * SCR_CAP);
    int* __restrict__ scr_b = scr_f + SCR_CAP;
    int r = 0;
    // the next candidate's position and clump are loaded a batch ahead
    int jn = -1, rn = 0, cn = 0;
    double4 pn = make_double4(0, 0, 0, 0);
    if (lane < total) {
        while (pre[r + 1] <= lane) r++;
        jn = rs[r] + (lane - pre[r]);
        rn = r;
        pn = posr[jn];
        cn = cid[jn];
    }
    for (int b0 = 0; b0 < total; b0 += SL) {
        const int j = jn, rj = rn, cj = cn;
        const double4 pj = pn;
        const int f = b0 + SL + lane;
        jn = -1;
        if (f < total) {
            while (pre[r + 1] <= f) r++;
            jn = rs[r] + (f - pre[r]);
            rn = r;
            pn = posr[jn];
            cn = cid[jn];
        }
        const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        const double d2 = dx * dx + dy * dy + dz * dz;
        const double lim = 1.50 * (pi.w + pj.w);
        const bool hit = j >= 0 && j != i && d2 < lim * lim;
        const bool same = rj < 9;
        const bool front = hit && same && i < j;
        const bool back = hit && !front;
        const bool cross = hit && !same;
        const unsigned fm = __ballot_sync(gm, front) >> gshift;
        const unsigned bm = __ballot_sync(gm, back) >> gshift;
        if (hit) {
            const int flag = cj == ci ? INTRA : 0;
            if (FILL) {
                if (front) {
                    const int q = rf + nf + __popc(fm & lt);
                    nbr[q] = j | flag;
                    own[q] = i;
                } else {
                    bnbr[rb + nb + __popc(bm & lt)] = j | flag;
                    if (cross) {
                        // the coarser partner owns the pair: claim a slot after
                        // its same-level front entries (sorted afterwards)
                        const int q = cnt_f[j + tb] + poff + sfc[j + tb] + atomicAdd(&xcnt[j + tb], 1);
                        nbr[q] = i | flag;
                        own[q] = j;
                    }
                }
            } else {
                if (front) {
                    const int q = nf + __popc(fm & lt);
                    if (q < SCR_CAP) scr_f[q] = j | flag;
                } else {
                    const int q = nb + __popc(bm & lt);
                    if (q < SCR_CAP) scr_b[q] = j | flag | (cross ? CROSS_TAG : 0);
                    if (cross) atomicAdd(&cnt_f[j + tb], 1);
                }
            }
        }
        nf += __popc(fm);
        nb += __popc(bm);
    }
    nf_out = nf;
    nb_out = nb;
}

// the subsphere of element t of the rebuilt concatenation and its scene
struct PlanItem {
    int k, s, i;
};
__device__ __forceinline__ PlanItem plan_item(const Dev& d, int ns, int t) {
    PlanItem r;
    r.k = plan_find(d.psub, ns, t);
    r.s = d.pscene[r.k];
    r.i = d.par[r.s].sub_off + (t - d.psub[r.k]);
    return r;
}

// The next chunk of a block's work: the search and the compaction cost
// differ a lot between subspheres (finer levels search more rows), so
// blocks claim chunks of one element per lane group from a counter instead
// of taking fixed strides; a block that drew cheap subspheres takes more.
__device__ __forceinline__ int claim_chunk(int* ctr, int n, int* sh) {
    if (threadIdx.x == 0) *sh = atomicAdd(ctr, n);
    __syncthreads();
    const int b = *sh;
    __syncthreads();
    return b;
}

// The fused search: counts (cnt_f[t] = same-level front entries + cross-level
// entries found by finer partners, cnt_b[t] = back entries) and the hits in
// scratch rows.  A group of SL lanes per subsphere, grid-stride.
template <int SL>
__global__ void __launch_bounds__(SEARCH_THREADS, 8) k_search(const Dev* __restrict__ dp) {
    __shared__ SearchShared<SL> sh;
    __shared__ int s_claim;
    const Dev& d = *dp;
    if (*d.halt) return;
    const int g = threadIdx.x / SL;
    const int lane = threadIdx.x % SL;
    const int T = d.plan[PL_T], ns = d.plan[PL_NS];
    for (;;) {
        const int c0 = claim_chunk(d.plan + PL_CS, SEARCH_THREADS / SL, &s_claim);
        if (c0 >= T) break;
        const int t = c0 + g;
        if (t >= T) continue;
        const PlanItem it = plan_item(d, ns, t);
        const ScenePar& P = d.par[it.s];
        int nf = 0, nb = 0;
        if (d.key2[it.i] != P.cell_off + P.cellnum - 1)  // out-of-box subspheres do not search
            group_search<false, SL>(d, P, d.L[1], it.i, lane, sh.rs[g], sh.pre[g], t - it.i, 0, 0, nf, nb);
        if (lane == 0) {
            atomicAdd(&d.cnt_f[t], nf);
            d.cnt_b[t] = nb;
            d.sfc[t] = nf;
            if (nf > P.bl / 2 || nb > P.bl / 2) atomicOr(&d.dyn[it.s].err, ERR_ROW_OVERFLOW);
        }
    }
}

// After the scans: the pairs of each rebuilt scene's new list (front and
// back entries are equally many: every pair is one owner entry and one
// partner entry) into need[s], their prefix over the rebuilt scenes into
// ppair; with stop set, a list longer than its scene's region stops the
// step (the host grows the regions and runs the rebuild again).  One block.
static __global__ void k_check_cap(const Dev* __restrict__ dp, int stop) {
    const Dev& d = *dp;
    if (*d.halt) return;
    const int ns = d.plan[PL_NS];
    for (int k = threadIdx.x; k < ns; k += blockDim.x) {
        const int s = d.pscene[k];
        const int a = d.psub[k], b = d.psub[k + 1];
        const int nf = d.cnt_f[b] - d.cnt_f[a], nb = d.cnt_b[b] - d.cnt_b[a];
        const int need = max(nf, nb);
        d.need[s] = need;
        d.ppair[k] = d.cnt_f[a];
        if (stop && need > d.dyn[s].pcap) {
            *d.halt = 1;
            atomicOr(&d.dyn[s].err, ERR_LIST_OVERFLOW);
        }
    }
    if (threadIdx.x == 0) d.ppair[ns] = d.cnt_f[d.psub[ns]];
}

// The new rows in the build list L[1], in the scene's region: copied from
// the scratch rows (and the cross-level slots of coarser partners claimed),
// or searched again for rows longer than the scratch.
template <int SL>
__global__ void __launch_bounds__(SEARCH_THREADS) k_compact(const Dev* __restrict__ dp) {
    __shared__ SearchShared<SL> sh;
    __shared__ int s_claim;
    const Dev& d = *dp;
    if (*d.halt) return;
    const int g = threadIdx.x / SL;
    const int lane = threadIdx.x % SL;
    const int T = d.plan[PL_T], ns = d.plan[PL_NS];
    const PairList& Nw = d.L[1];
    for (;;) {
        const int c0 = claim_chunk(d.plan + PL_CC, SEARCH_THREADS / SL, &s_claim);
        if (c0 >= T) break;
        const int t = c0 + g;
        if (t >= T) continue;
        const PlanItem it = plan_item(d, ns, t);
        const int i = it.i, s = it.s, tb = t - i;
        const ScenePar& P = d.par[s];
        const int t0 = d.psub[it.k];
        const int base = d.dyn[s].pair_off;
        const int poff = base - d.cnt_f[t0], boff = base - d.cnt_b[t0];
        const int rf = d.cnt_f[t] + poff, rb = d.cnt_b[t] + boff;
        if (lane == 0) {
            Nw.row[i + s] = rf;
            Nw.brow[i + s] = rb;
            if (i == P.sub_off + P.nsub - 1) {
                Nw.row[i + s + 1] = d.cnt_f[t + 1] + poff;
                Nw.brow[i + s + 1] = d.cnt_b[t + 1] + boff;
            }
        }
        if (d.key2[i] == P.cell_off + P.cellnum - 1) continue;
        const int nf = d.sfc[t], nb = d.cnt_b[t + 1] - d.cnt_b[t];
        if (nf <= SCR_CAP && nb <= SCR_CAP) {
            const int* scr_f = d.scr + (size_t)i * (2 * SCR_CAP);
            const int* scr_b = scr_f + SCR_CAP;
            for (int k = lane; k < nf; k += SL) { Nw.nbr[rf + k] = scr_f[k]; Nw.own[rf + k] = i; }
            for (int k = lane; k < nb; k += SL) {
                const int v = scr_b[k];
                Nw.bnbr[rb + k] = v & ~CROSS_TAG;
                if (v & CROSS_TAG) {
                    const int tj = (v & (IDX_MASK & ~CROSS_TAG)) + tb;
                    const int q = d.cnt_f[tj] + poff + d.sfc[tj] + atomicAdd(&d.xcnt[tj], 1);
                    Nw.nbr[q] = i | (v & INTRA);
                    Nw.own[q] = tj - tb;
                }
            }
        } else {
            int f2, b2;
            group_search<true, SL>(d, P, Nw, i, lane, sh.rs[g], sh.pre[g], tb, poff, boff, f2, b2);
        }
    }
}

// hierarchical grid: the cross-level entries of each owner row in ascending
// order of the finer partner (their slots were claimed with atomics)
static __global__ void k_xsort(const Dev* __restrict__ dp) {
    const Dev& d = *dp;
    if (*d.halt) return;
    const int T = d.plan[PL_T], ns = d.plan[PL_NS];
    const PairList& Nw = d.L[1];
    NBC_GRID_STRIDE(t, T) {
        const PlanItem it = plan_item(d, ns, t);
        const int b = Nw.row[it.i + it.s] + d.sfc[t], e = Nw.row[it.i + it.s + 1];
        for (int m = b + 1; m < e; m++) {
            const int v = Nw.nbr[m];
            int q = m - 1;
            while (q >= b && (Nw.nbr[q] & IDX_MASK) > (v & IDX_MASK)) { Nw.nbr[q + 1] = Nw.nbr[q]; q--; }
            Nw.nbr[q + 1] = v;
        }
    }
}

// The reverse map of CreateContList_cuk (src/dem_grid.cu:561-601): for each
// back entry of i (owner j), the slot of the pair (j, i) in j's front row.
// A front row is two ascending runs of partners: the same-level entries
// (the search visits the stencil's cells in ascending cell order, and the
// subspheres are sorted by cell), then the cross-level entries (k_xsort), so
// the slot is found by binary search in the run of i's level.
__device__ __forceinline__ int find_partner(const int* __restrict__ nbr, int lo, int hi, int key) {
    int len = hi - lo;
    while (len > 0) {
        const int h = len >> 1;
        if ((nbr[lo + h] & IDX_MASK) < key) { lo += h + 1; len -= h + 1; }
        else len = h;
    }
    return lo < hi && (nbr[lo] & IDX_MASK) == key ? lo : -1;
}

static __global__ void k_backref(const Dev* __restrict__ dp) {
    const Dev& d = *dp;
    if (*d.halt) return;
    const int T = d.plan[PL_T], ns = d.plan[PL_NS];
    const PairList& Nw = d.L[1];
    NBC_GRID_STRIDE(t, T) {
        const PlanItem it = plan_item(d, ns, t);
        const int s = it.s, i = it.i, tb = t - i;
        for (int k = Nw.brow[i + s]; k < Nw.brow[i + s + 1]; k++) {
            const int j = Nw.bnbr[k] & IDX_MASK;
            const int rs = Nw.row[j + s], re = Nw.row[j + s + 1], mid = rs + d.sfc[j + tb];
            const bool same = d.level2[i] == d.level2[j];
            int found = same ? find_partner(Nw.nbr, rs, mid, i) : find_partner(Nw.nbr, mid, re, i);
            if (found < 0)   // not where the order puts it: scan the row
                for (int q = rs; q < re; q++)
                    if ((Nw.nbr[q] & IDX_MASK) == i) { found = q; break; }
            Nw.bpair[k] = found;
        }
    }
}

// InheritContHistory_cuk (src/dem_grid.cu:603-647): each new pair copies the
// spring history of the same pair in the current list, negated when the
// owner changed; pairs absent from it start from zero.  The new history and
// touch flag go to the generation the next contact pass writes (free now) and
// are written back by k_writeback_pairs.
template <typename R>
__device__ __forceinline__ void carry_one(const Dev& d, int p, int s) {
    const int hg = *d.hgen;
    const PairList& O = d.L[0];
    const PairList& Nw = d.L[1];
    const size_t cap = (size_t)d.cap;
    const R4<R>* Hi = (const R4<R>*)d.H[hg & 1];
    R4<R>* Ho = (R4<R>*)d.H[(hg + 1) & 1];
    const uint8_t* ti = d.touch[hg & 1];
    uint8_t* to = d.touch[(hg + 1) & 1];
    const int jr = Nw.nbr[p];
    if (jr < 0) { to[p] = 0; d.nearf[p] = 0; return; }  // pair inside one clump
    const int i = Nw.own[p], j = jr;
    const ScenePar& P = d.par[s];
    // near flag of the new pair (see k_near): distance below ri + rj + 2 Thresh
    {
        const double4 pi = d.posr2[i], pj = d.posr2[j];
        const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        const double m = 2.0 * P.thresh * (1.0 + 1e-6) + 1e-12;
        const double lim = (pi.w + pj.w) + m;
        const bool nr = dx * dx + dy * dy + dz * dz < lim * lim;
        d.nearf[p] = nr;
        if (!nr) {
            to[p] = 0;  // cannot touch before the next rebuild: no live history
            return;
        }
    }
    int q = -1;
    R sign = R(1);
    if (P.sphere & SPH_RESET) {
        // DEMmain::RunSimulation and _Split exchange the history pointers
        // once more after the list build has carried the histories and
        // cleared the other buffer (src/dem_simulation_cylind.cu:141,
        // src/dem_grid.cu:687-749): after a rebuild every pair starts from zero
        q = -1;
    } else {
        const int io = d.perm[i], jo = d.perm[j];
        int oo, ot;
        if (P.levels > 1 && d.level2[i] != d.level2[j]) {
            const bool i_coarse = d.level2[i] < d.level2[j];
            oo = i_coarse ? io : jo;
            ot = i_coarse ? jo : io;
        } else {
            oo = io < jo ? io : jo;
            ot = io < jo ? jo : io;
        }
        sign = oo == io ? R(1) : R(-1);
        // the first entry of the old owner row with partner ot, four
        // entries loaded at a time
        const int rb = O.row[oo + s], re = O.row[oo + s + 1];
        for (int r = rb; r < re && q < 0; r += 4) {
            int v[4];
#pragma unroll
            for (int k = 0; k < 4; k++) v[k] = r + k < re ? (O.nbr[r + k] & IDX_MASK) : -1;
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (q < 0 && v[k] == ot) q = r + k;
        }
    }
    if (q >= 0 && ti[q]) {
        for (int h = 0; h < 2; h++) {
            R4<R> v = Hi[2 * (size_t)q + h];
            v.x *= sign; v.y *= sign; v.z *= sign; v.w *= sign;
            Ho[2 * (size_t)p + h] = v;
        }
        const R* h2i = (const R*)(Hi + 2 * cap);
        R* h2o = (R*)(Ho + 2 * cap);
        h2o[p] = sign * h2i[q];
        to[p] = 1;
    } else {
        to[p] = 0;
    }
}

// the pairs of the rebuilt scenes' new lists (element u of their
// concatenation is slot pair_off + u - ppair[k] of its scene's region)
template <typename R>
__global__ void k_carry(const Dev* __restrict__ dp) {
    const Dev& d = *dp;
    if (*d.halt) return;
    const int ns = d.plan[PL_NS];
    const int np = d.ppair[ns];
    NBC_GRID_STRIDE(u, np) {
        const int k = plan_find(d.ppair, ns, u);
        const int s = d.pscene[k];
        carry_one<R>(d, d.dyn[s].pair_off + (u - d.ppair[k]), s);
    }
}

// Commits a rebuild.  When every scene was rebuilt (always for a single
// scene) the gathered buffers, the build list and the carried history
// generation become the current ones by exchanging pointers in the table
// (one thread); k_near then clears the other touch generation for the pairs
// that are not near (it still holds the flags of the previous list).
// Otherwise the rebuilt scenes' gathered per-subsphere state, new rows, list
// entries, carried histories and touch flags are written back into the
// current buffers and the generation the next contact pass reads (both
// generations then agree on the region).
template <typename R>
__global__ void k_writeback(Dev* __restrict__ dp) {
    const Dev& d = *dp;
    if (*d.halt) return;
    const int ns = d.plan[PL_NS];
    if (ns == d.S) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            Dev& w = *dp;
#define NBC_SWAP(a, b) { auto tmp_ = w.a; w.a = w.b; w.b = tmp_; }
            NBC_SWAP(posr, posr2) NBC_SWAP(lom, lom2) NBC_SWAP(cum, cum2) NBC_SWAP(clump_id, clump_id2)
            NBC_SWAP(part_fix, part_fix2) NBC_SWAP(level, level2) NBC_SWAP(key, key2) NBC_SWAP(kin, kin2)
            NBC_SWAP(bhist, bhist2) NBC_SWAP(bbits, bbits2)
            NBC_SWAP(L[0], L[1]) NBC_SWAP(H[0], H[1]) NBC_SWAP(touch[0], touch[1])
#undef NBC_SWAP
        }
        return;
    }
    const int T = d.plan[PL_T];
    const size_t N = (size_t)d.N;
    const PairList& Lc = d.L[0];
    const PairList& Nw = d.L[1];
    NBC_GRID_STRIDE(t, T) {
        const PlanItem it = plan_item(d, ns, t);
        const int i = it.i, s = it.s;
        d.posr[i] = d.posr2[i];
        d.lom[i] = d.lom2[i];
        d.cum[i] = d.cum2[i];
        d.clump_id[i] = d.clump_id2[i];
        d.part_fix[i] = d.part_fix2[i];
        d.level[i] = d.level2[i];
        d.key[i] = d.key2[i];
        ((double4*)d.kin)[i] = ((const double4*)d.kin2)[i];
        const uint16_t bits = d.bbits2[i];
        d.bbits[i] = bits;
        const R4<R>* b2 = (const R4<R>*)d.bhist2;
        R4<R>* b1 = (R4<R>*)d.bhist;
        for (int sl = 0; sl < NB_SLOTS; sl++) {
            if (!(bits & (1u << sl))) continue;
            for (int c = 0; c < 3; c++) b1[((size_t)sl * N + i) * 3 + c] = b2[((size_t)sl * N + i) * 3 + c];
        }
        Lc.row[i + s] = Nw.row[i + s];
        Lc.brow[i + s] = Nw.brow[i + s];
        if (i == d.par[s].sub_off + d.par[s].nsub - 1) {
            Lc.row[i + s + 1] = Nw.row[i + s + 1];
            Lc.brow[i + s + 1] = Nw.brow[i + s + 1];
        }
    }
    const int np = d.ppair[ns];
    const int hg = *d.hgen;
    const size_t cap = (size_t)d.cap;
    R4<R>* Hc = (R4<R>*)d.H[hg & 1];
    const R4<R>* Hn = (const R4<R>*)d.H[(hg + 1) & 1];
    uint8_t* tc = d.touch[hg & 1];
    const uint8_t* tn = d.touch[(hg + 1) & 1];
    NBC_GRID_STRIDE(u, np) {
        const int k = plan_find(d.ppair, ns, u);
        const int p = d.dyn[d.pscene[k]].pair_off + (u - d.ppair[k]);
        Lc.nbr[p] = Nw.nbr[p];
        Lc.own[p] = Nw.own[p];
        Lc.bnbr[p] = Nw.bnbr[p];
        Lc.bpair[p] = Nw.bpair[p];
        const uint8_t f = tn[p];
        tc[p] = f;
        if (f) {
            Hc[2 * (size_t)p] = Hn[2 * (size_t)p];
            Hc[2 * (size_t)p + 1] = Hn[2 * (size_t)p + 1];
            ((R*)(Hc + 2 * cap))[p] = ((const R*)(Hn + 2 * cap))[p];
        }
    }
}

// Boundary candidates.  Walls do not move (their velocity enters only the
// contact law), and between two rebuilds of a scene every subsphere stays
// within Thresh of where it was at the rebuild, so a subsphere farther than
// 2 Thresh from every wall region at a rebuild cannot touch a wall before
// the next one.  At each rebuild the near-row count pass flags, per rebuilt
// subsphere (new order), whether it is within that margin of a wall --
// every subsphere of a scene with an intruder is a candidate, the intruder
// moves -- and clears the wall contact bits of the others (they are not in
// contact now); the fill pass lists the candidates in the scene's range of
// bidx, and k_boundary visits only them.
__device__ __forceinline__ bool bound_candidate(const Dev& d, const ScenePar& P, int i) {
    bool cand = P.has_intr;
    if (!cand && P.wall != WALL_NONE) {
        const double4 pp = d.posr[i];
        const double m = 2.0 * P.thresh * (1.0 + 1e-6) + 1e-12;
        const double r = pp.w + m;
        const double ex = pp.x - P.w_c[0], ey = pp.y - P.w_c[1], ez = pp.z - P.w_c[2];
        if (P.wall == WALL_CUBE) {
            cand = fabs(ex) + r >= P.w_half[0] * (1 - 1e-9) || fabs(ey) + r >= P.w_half[1] * (1 - 1e-9) ||
                   fabs(ez) + r >= P.w_half[2] * (1 - 1e-9);
        } else {
            const double ax = ex * P.cyl_axis[0] + ey * P.cyl_axis[1] + ez * P.cyl_axis[2];
            const double rr = ex * ex + ey * ey + ez * ez - ax * ax;
            const double in = P.cyl_R - r;
            cand = fabs(ax) + r >= P.cyl_H * (1 - 1e-9) || in <= 0 || rr >= in * in * (1 - 1e-9);
        }
    }
    return cand;
}

// Near rows.  Between two rebuilds of a scene every subsphere stays within
// Thresh of where it was at the rebuild (a larger displacement triggers the
// next one), so a pair whose distance at a rebuild is at least ri + rj +
// 2 Thresh cannot touch before the next one.  k_carry flags the near pairs
// of a rebuilt scene and clears the touch flag of the others (in both
// generations, after the write-back); the near rows list a rebuilt scene's
// near entries in its pair region (front: pair slot in row order, back: the
// pair slot of each near back entry) and the contact pass visits only them,
// with the same results as visiting the whole list.  FILL = false counts
// them into cnt_f / cnt_b of the rebuilt concatenation and flags the
// boundary candidates into xcnt; FILL = true writes the rows and the
// candidate list at the scanned offsets, and finishes the rebuild's
// bookkeeping: per-clump member lists of the rebuilt scenes in ascending
// subsphere order (the order thrust::sort_by_key gives reduce_by_key,
// src/dem_clumpsphere.cu:123-147), the scenes' pair and near counts.
template <bool FILL, int SL>
__global__ void __launch_bounds__(SEARCH_THREADS) k_near(const Dev* __restrict__ dp) {
    const Dev& d = *dp;
    if (*d.halt) return;
    const int T = d.plan[PL_T], ns = d.plan[PL_NS];
    const int lane = threadIdx.x % SL;
    const unsigned gm = SL == 32 ? 0xffffffffu : (((1u << SL) - 1u) << ((threadIdx.x & 31) & ~(SL - 1)));
    const int gshift = (threadIdx.x & 31) & ~(SL - 1);
    const unsigned lt = (1u << lane) - 1u;
    const PairList& Lc = d.L[0];
    const uint8_t* __restrict__ nearf = d.nearf;
    const int* __restrict__ bpair = Lc.bpair;
    // after the pointer exchange of k_writeback: the other touch generation
    // still holds the old list's flags
    uint8_t* __restrict__ tother = !FILL && ns == d.S ? d.touch[(*d.hgen + 1) & 1] : nullptr;
    if (!FILL && blockIdx.x == 0 && threadIdx.x == 0) { d.cnt_f[T] = 0; d.cnt_b[T] = 0; d.xcnt[T] = 0; }
    for (int t = blockIdx.x * (SEARCH_THREADS / SL) + threadIdx.x / SL; t < T;
         t += gridDim.x * (SEARCH_THREADS / SL)) {
        const PlanItem it = plan_item(d, ns, t);
        const int i = it.i, s = it.s;
        int nf = 0, nb = 0, rf = 0, rb = 0;
        if (FILL) {
            const int t0 = d.psub[it.k], base = d.dyn[s].pair_off;
            rf = base + d.cnt_f[t] - d.cnt_f[t0];
            rb = base + d.cnt_b[t] - d.cnt_b[t0];
            if (lane == 0) {
                d.nrb[i + s] = make_int2(rf, rb);
                if (i == d.par[s].sub_off + d.par[s].nsub - 1) {
                    d.nrb[i + s + 1] = make_int2(base + d.cnt_f[t + 1] - d.cnt_f[t0], base + d.cnt_b[t + 1] - d.cnt_b[t0]);
                }
            }
        }
        const int rs = Lc.row[i + s], re = Lc.row[i + s + 1];
        for (int k0 = rs; k0 < re; k0 += SL) {
            const int k = k0 + lane;
            const bool nr = k < re && nearf[k];
            if (tother && k < re && !nr) tother[k] = 0;
            const unsigned m = __ballot_sync(gm, nr) >> gshift;
            if (FILL && nr) d.nfr[rf + nf + __popc(m & lt)] = make_int4(k, Lc.nbr[k], i, -1);
            nf += __popc(m);
        }
        const int bs = Lc.brow[i + s], be = Lc.brow[i + s + 1];
        for (int k0 = bs; k0 < be; k0 += SL) {
            const int k = k0 + lane;
            int q = -1;
            if (k < be) q = bpair[k];
            const bool nr = q >= 0 && nearf[q];
            const unsigned m = __ballot_sync(gm, nr) >> gshift;
            if (FILL && nr) {
                const int e = rb + nb + __popc(m & lt);
                d.nbq[e] = q;
                d.nbpos[q] = e;
            }
            nb += __popc(m);
        }
        if (!FILL && lane == 0) {
            d.cnt_f[t] = nf;
            d.cnt_b[t] = nb;
            const bool cand = bound_candidate(d, d.par[s], i);
            if (!cand) d.bbits[i] = 0;
            d.xcnt[t] = cand ? 1 : 0;
        }
        if (FILL && lane == 0) {
            const ScenePar& P = d.par[s];
            const int t0 = d.psub[it.k];
            if (d.xcnt[t + 1] - d.xcnt[t]) d.bidx[P.sub_off + d.xcnt[t] - d.xcnt[t0]] = i;
            if (i == P.sub_off + P.nsub - 1) d.dyn[s].nbound = d.xcnt[t + 1] - d.xcnt[t0];
        }
    }
    if (FILL) {
        const int TK = d.plan[PL_TK];
        NBC_GRID_STRIDE(u, TK + ns + 1) {
            if (u < TK) {
                const int k = plan_find(d.pclump, ns, u);
                const int c = d.par[d.pscene[k]].clump_off + (u - d.pclump[k]);
                const int mb = d.mem_start[c], me = d.mem_start[c + 1];
                for (int m = mb; m < me; m++) d.mem_idx[m] = d.inv[d.mem_idx[m]];
                for (int m = mb + 1; m < me; m++) {
                    int v = d.mem_idx[m], q = m - 1;
                    while (q >= mb && d.mem_idx[q] > v) { d.mem_idx[q + 1] = d.mem_idx[q]; q--; }
                    d.mem_idx[q + 1] = v;
                }
            } else if (u < TK + ns) {
                const int k = u - TK;
                SceneDyn& y = d.dyn[d.pscene[k]];
                y.npairs = d.ppair[k + 1] - d.ppair[k];
                y.nnear = d.cnt_f[d.psub[k + 1]] - d.cnt_f[d.psub[k]];
                y.nrebuild++;
                y.rebuild = 0;
            } else {
                *d.any_rebuild = 0;
            }
        }
    }
}

// The last pass of a rebuild: the contact pass's work items (near pairs) and
// the boundary candidates of every scene as prefixes over the scenes (block
// 0), and each rebuilt subsphere's near front records completed with the
// near back entry of their pair (the near-row fill pass writes both rows at
// once, so a front record cannot take it there).
static __global__ void __launch_bounds__(SC_THREADS) k_near_finish(const Dev* __restrict__ dp) {
    __shared__ int sh[SC_THREADS / 32];
    const Dev& d = *dp;
    if (*d.halt) return;
    if (blockIdx.x == 0) {
        int run = 0, brun = 0;
        for (int b = 0; b < d.S; b += SC_THREADS) {
            const int s = b + threadIdx.x;
            int tot;
            const int ex = block_excl_scan(s < d.S ? d.dyn[s].nnear : 0, sh, tot);
            if (s < d.S) d.nprefix[s] = run + ex;
            run += tot;
            const int bx = block_excl_scan(s < d.S ? d.dyn[s].nbound : 0, sh, tot);
            if (s < d.S) d.bprefix[s] = brun + bx;
            brun += tot;
        }
        if (threadIdx.x == 0) {
            d.nprefix[d.S] = run;
            d.bprefix[d.S] = brun;
        }
    }
    const int T = d.plan[PL_T], ns = d.plan[PL_NS];
    NBC_GRID_STRIDE(t, T) {
        const PlanItem it = plan_item(d, ns, t);
        const int i = it.i, s = it.s;
        for (int e = d.nrb[i + s].x; e < d.nrb[i + s + 1].x; e++) d.nfr[e].w = d.nbpos[d.nfr[e].x];
    }
}

// Moves every scene's list to a new layout of the pair regions (the host
// grows them): entries, back references, the history generation the next
// contact pass reads, touch and near flags.  map[s] = (old first slot, new
// first slot, pairs, prefix of the pairs over the scenes); d holds the new
// buffers.
template <typename R>
__global__ void k_relayout(const Dev* __restrict__ dp, PairList ol, const void* __restrict__ oh,
                           const uint8_t* __restrict__ ot, const uint8_t* __restrict__ onear,
                           const int4* __restrict__ onfr, const int* __restrict__ onbq,
                           const int* __restrict__ onbpos, int ocap,
                           const int4* __restrict__ map, int total) {
    const Dev& d = *dp;
    const int hg = *d.hgen;
    const size_t cap = (size_t)d.cap, oc = (size_t)ocap;
    const R4<R>* Ho = (const R4<R>*)oh;
    R4<R>* Hn = (R4<R>*)d.H[hg & 1];
    const PairList& Lc = d.L[0];
    NBC_GRID_STRIDE(u, total) {
        int lo = 0, hi = d.S - 1;
        while (lo < hi) {
            const int m = (lo + hi + 1) >> 1;
            if (map[m].w <= u) lo = m;
            else hi = m - 1;
        }
        const int4 m = map[lo];
        const int po = m.x + (u - m.w), pn = m.y + (u - m.w);
        Lc.nbr[pn] = ol.nbr[po];
        Lc.own[pn] = ol.own[po];
        Lc.bnbr[pn] = ol.bnbr[po];
        const int bq = ol.bpair[po];
        Lc.bpair[pn] = bq >= 0 ? bq + (m.y - m.x) : bq;
        const uint8_t f = ot[po];
        d.touch[hg & 1][pn] = f;
        d.nearf[pn] = onear[po];
        const int4 fr = onfr[po];             // slots past the near count carry nothing
        d.nfr[pn] = make_int4(fr.x + (m.y - m.x), fr.y, fr.z, fr.w + (m.y - m.x));
        d.nbq[pn] = onbq[po] + (m.y - m.x);
        d.nbpos[pn] = onear[po] ? onbpos[po] + (m.y - m.x) : -1;
        if (f) {
            Hn[2 * (size_t)pn] = Ho[2 * (size_t)po];
            Hn[2 * (size_t)pn + 1] = Ho[2 * (size_t)po + 1];
            ((R*)(Hn + 2 * cap))[pn] = ((const R*)(Ho + 2 * oc))[po];
        }
    }
}

// the current rows and near rows follow their scene's region: every offset of scene s
// moves by its region's move (the subsphere threads take the row starts,
// one thread per scene the end entry)
static __global__ void k_shift_rows(const Dev* __restrict__ dp, const int4* __restrict__ map) {
    const Dev& d = *dp;
    const PairList& Lc = d.L[0];
    NBC_GRID_STRIDE(u, d.N + d.S) {
        int s, r;
        if (u < d.N) {
            s = d.sid[u];
            r = u + s;
        } else {
            s = u - d.N;
            r = d.par[s].sub_off + d.par[s].nsub + s;
        }
        const int delta = map[s].y - map[s].x;
        Lc.row[r] += delta;
        Lc.brow[r] += delta;
        d.nrb[r].x += delta;
        d.nrb[r].y += delta;
    }
}

// ===========================================================================
// contact kernel
// ===========================================================================

template <typename R> struct Law {
    double kn_fac, ks_fac, damping;   // stiffness and damping factors (the normal force is FP64)
    R beta, mu, dt;
};

template <typename R> struct LawOut {
    V3<R> Fn, Ft, Mr, Mt;  // normal and tangential force on the body, rolling and twisting moments
    V3<R> hs, ht, hr;      // new tangential, twisting and rolling histories
    R FnL;
};

// The Hertz-Mindlin law with rolling and twisting springs shared by the
// pair, wall and intruder kernels of the reference
// (src/dem_force_clump.cu:66-161, src/dem_force_cube_wall_clump.cu:62-166,
// src/dem_force_penetrator_clump.cu:76-173).  n points from the other body
// toward this body's contact side, Vtot is this body's contact-point velocity
// relative to the other's, Dth = dt (w_this - w_other) for walls and the
// intruder, dt (w_other_side...) as the pair caller passes it.
//
// The normal force Kn Dn n + Cn Vnor is evaluated in FP64 whatever R is: on a
// separating contact its elastic and damping terms nearly cancel (the net
// force of the contact can be a thousandth of either), so rounding them to
// FP32 would leave that contact's force with an error of 1e-4 of itself.  The
// tangential, rolling and twisting parts, the histories and everything after
// run in R.  With R = double every operation is the reference's, in its order.
template <typename R>
__device__ __forceinline__ void hm_law(const Law<R>& L, V3<double> nd, double Dn, V3<double> Vtot, V3<R> Dth,
                                       double Rij, double Mij, R cs_mult, V3<R> H, V3<R> Mr, V3<R> Mt,
                                       LawOut<R>& o) {
    const double sq = sqrt(Rij * Dn);
    const double Kn = L.kn_fac * sq;
    const double Cn = L.damping * sqrt(Kn * Mij);
    const R Ks = (R)(L.ks_fac * sq);
    const R Cs = cs_mult * (R)L.damping * sqrt(Ks * (R)Mij);
    const R br = L.beta * (R)Rij;
    const R Kr = R(0.25) * (R)Kn * br * br;
    const R Cr = R(0.25) * (R)Cn * br * br;
    const R Kt = R(0.50) * Ks * br * br;
    const R Ct = R(0.50) * Cs * br * br;
    const double ERR = dot(nd, Vtot);
    const V3<double> Vnor = ERR * nd;
    const V3<R> Vtan = cvt<R>(Vtot - Vnor);
    const V3<double> Fn = (Kn * Dn) * nd + Cn * Vnor;
    const V3<R> n = cvt<R>(nd);
    o.Fn = cvt<R>(Fn);
    o.FnL = (R)len_floor(Fn);
    V3<R> Ft = (-Ks) * (L.dt * Vtan) + Cs * Vtan + H;
    const R FtL = len_floor(Ft);
    if (FtL > o.FnL * L.mu) {
        Ft = (L.mu * o.FnL * (R(1) / FtL)) * Ft;
        o.hs = Ft;
    } else {
        o.hs = Ft - Cs * Vtan;
    }
    o.Ft = Ft;
    const R DthL = dot(Dth, n);
    const V3<R> DthT = DthL * n;
    const V3<R> DthR = Dth - DthT;
    V3<R> rm = Kr * DthR + Mr;
    const R rmL = len_floor(rm);
    const R rcap = R(0.525) * L.beta * (R)Rij * o.FnL;
    if (rmL > rcap) {
        rm = (rcap * (R(1) / rmL)) * rm;
        o.hr = rm;
    } else {
        o.hr = rm;
        rm = rm - (Cr * (R(1) / L.dt)) * DthR;
    }
    V3<R> tm = Kt * DthT + Mt;
    const R tmL = len_floor(tm);
    const R tcap = R(0.65) * L.mu * L.beta * (R)Rij * o.FnL;
    if (tmL > tcap) {
        tm = (tcap * (R(1) / tmL)) * tm;
        o.ht = tm;
    } else {
        o.ht = tm;
        tm = tm - (Ct * (R(1) / L.dt)) * DthT;
    }
    o.Mr = rm;
    o.Mt = tm;
}

// The contact kinematics of a subsphere in FP64 (its clump's velocity and
// angular velocity, its world arm and mass): a bed moving as a whole gives
// touching subspheres nearly equal contact-point velocities, so their
// difference is formed in FP64 before the law rounds anything.  The
// subsphere's own record is one double4 (world arm, mass) written by the
// pose pass; the velocities are read from its clump's records (the values the
// clump pass wrote with the same half-kick), so a clump's velocity is stored
// once rather than once per member.
template <typename R> struct Body {
    double4 p;              // position, radius
    V3<double> v, w, arm;   // clump velocity, clump angular velocity, world arm
    double m;
};

template <typename R>
__device__ __forceinline__ void load_kin(const Dev& d, int i, int c, Body<R>& b) {
    const double4 r = ((const double4*)d.kin)[i], v = d.cvel[c], w = d.cw[c];
    b.arm = v3(r.x, r.y, r.z);
    b.m = r.w;
    b.v = v3(v.x, v.y, v.z);
    b.w = v3(w.x, w.y, w.z);
}

// The pair law of ContactForce_clump_cuk (src/dem_force_clump.cu:3-163) with
// a in the role of particleI, evaluated once for both bodies of a touching
// pair: the force and torque on a and the torque on b.  Seen from b every
// input of the law is exactly negated (normal, relative velocity, rotation
// increment, negated history), so the law's outputs are negated too: the
// force on b is -fa and its torque uses b's own lever Ab = (rb^2 - ra^2 +
// d^2) / 2d.  Geometry, lever arms and the contact-point velocity are FP64.
// Returns false when the pair does not overlap.
template <typename R>
__device__ __forceinline__ bool pair_contact2(const Law<R>& L, R cohesion, const Body<R>& a, const Body<R>& b,
                                              V3<R> H, V3<R> Mr, V3<R> Mt, V3<R>& fa, V3<R>& ta, V3<R>& tb,
                                              LawOut<R>& o, double& Ap_out, V3<double>& n_out) {
    const double dx = b.p.x - a.p.x, dy = b.p.y - a.p.y, dz = b.p.z - a.p.z;
    const double DistS = dx * dx + dy * dy + dz * dz;
    const double DistL = sqrt(DistS);
    const double Dn = a.p.w + b.p.w - DistL;
    if (!(Dn > 0.0)) return false;
    const double DistR = 1.0 / DistL;
    const V3<double> nd = v3(DistR * dx, DistR * dy, DistR * dz);
    const double Ap = 0.50 * (a.p.w * a.p.w - b.p.w * b.p.w + DistS) * DistR;
    const double An = DistL - Ap;
    const double Ab = 0.50 * (b.p.w * b.p.w - a.p.w * a.p.w + DistS) * DistR;
    const double Rij = a.p.w * b.p.w / (a.p.w + b.p.w);
    const double Mij = a.m * b.m / (a.m + b.m);
    const V3<double> ARMa = a.arm + Ap * nd;
    const V3<double> ARMb = b.arm - An * nd;
    const V3<double> Vtot = (b.v - a.v) + (cross(b.w, ARMb) - cross(a.w, ARMa));
    const V3<R> Dth = L.dt * cvt<R>(a.w - b.w);
    hm_law<R>(L, nd, Dn, Vtot, Dth, Rij, Mij, R(1), H, Mr, Mt, o);
    const V3<R> n = cvt<R>(nd);
    const R br = L.beta * (R)Rij;
    fa = (-o.Fn - o.Ft) + (cohesion * br * br) * n;
    const V3<R> nxF = cross(n, o.Ft);
    ta = ((-(R)Ap) * nxF - o.Mr) - o.Mt;
    tb = ((-(R)Ab) * nxF + o.Mr) + o.Mt;
    Ap_out = Ap;
    n_out = nd;
    return true;
}

// a wall or intruder contact: normal n (toward the subsphere), lever Ap,
// overlap Dn, wall point RVo relative to the wall centre, wall velocity and
// angular velocity wv, ww (FP64 geometry and velocities, as for pairs)
template <typename R>
__device__ __forceinline__ void boundary_contact(const Law<R>& L, const Body<R>& a, V3<double> nd, double Ap,
                                                 double Dn, V3<double> RVo, V3<double> wv, V3<double> ww,
                                                 double Rij, double Mij, R cs_mult, V3<R> H, V3<R> Mr, V3<R> Mt,
                                                 V3<R>& f, V3<R>& t, LawOut<R>& o, V3<R>& arm_out) {
    const V3<double> Arm = (-a.arm) + Ap * nd;
    const V3<double> Vwall = cross(ww, RVo);
    const V3<double> Vtot = (a.v - wv) + (cross(Arm, a.w) - Vwall);
    const V3<R> Dth = L.dt * cvt<R>(a.w - ww);
    hm_law<R>(L, nd, Dn, Vtot, Dth, Rij, Mij, cs_mult, H, Mr, Mt, o);
    const V3<R> n = cvt<R>(nd);
    f = o.Fn + o.Ft;
    t = ((-(R)Ap) * cross(n, o.Ft) - o.Mr) - o.Mt;
    arm_out = cvt<R>(Arm);
}

// pair history layout: R4 (Dv.xyz, Dr.x) at [2q], R4 (Dt.xyz, Dr.y) at
// [2q + 1] (one 32-byte record in FP32), Dr.z as a scalar after the 2*cap R4s
template <typename R>
__device__ __forceinline__ void hist_read(const R4<R>* H, size_t cap, size_t q, V3<R>& hs, V3<R>& ht, V3<R>& hr) {
    R4<R> a = H[2 * q], b = H[2 * q + 1];
    const R c = ((const R*)(H + 2 * cap))[q];
    hs = v3<R>(a.x, a.y, a.z);
    ht = v3<R>(b.x, b.y, b.z);
    hr = v3<R>(a.w, b.w, c);
}
template <typename R>
__device__ __forceinline__ void hist_write(R4<R>* H, size_t cap, size_t q, V3<R> hs, V3<R> ht, V3<R> hr) {
    H[2 * q] = pack<R>(hs, hr.x);
    H[2 * q + 1] = pack<R>(ht, hr.y);
    ((R*)(H + 2 * cap))[q] = hr.z;
}

constexpr int CT_THREADS = 256;
constexpr int BD_THREADS = 128;

// Walls and intruder, one thread per boundary candidate: the face tests of
// CubeWallInteraction_clump_cuk (src/dem_force_cube_wall_clump.cu:185-298),
// the region tests of CylindWallInteraction_cuk (src/dem_force_cylind_wall.cu:
// 152-237) with clump kinematics, PrePenetrator / GetSphereIntruderContact /
// ForcePene_clump_cuk (src/dem_contact_penetrator.cu:8-84,
// src/dem_sphere_intruder.cuh:20-51, src/dem_force_penetrator_clump.cu:4-182).
// Writes the summed boundary force/torque where some slot is in contact and
// the slot mask; the intruder totals go to fixed-point accumulators.  SPH:
// the build for batches with a sphere-driver scene (ScenePar::sphere); the
// clump path's build carries none of that code.
template <typename R, bool EXPORT, bool SPH>
__device__ __forceinline__ void boundary_one(const Dev& d, int i, int s);

template <typename R, bool EXPORT, bool SPH>
__global__ void __launch_bounds__(BD_THREADS) k_boundary(const Dev* __restrict__ dp) {
    const Dev& d = *dp;
    if (*d.halt) return;
    const int S = d.S;
    const int* __restrict__ bpre = d.bprefix;
    const int nb = bpre[S];
    for (int w = blockIdx.x * BD_THREADS + threadIdx.x; w < nb; w += gridDim.x * BD_THREADS) {
        // work item w: boundary candidate w - bprefix[s] of scene s
        const int s = S == 1 ? 0 : plan_find(bpre, S, w);
        const int i = d.bidx[d.par[s].sub_off + (w - bpre[s])];
        boundary_one<R, EXPORT, SPH>(d, i, s);
    }
}

template <typename R, bool EXPORT, bool SPH>
__device__ __forceinline__ void boundary_one(const Dev& d, int i, int s) {
    const double4 pp = d.posr[i];   // issued before the scene's flag is known
    const uint16_t bb_old = d.bbits[i];
    if (d.has_stops && d.dyn[s].frozen) return;   // a scene past its stop stands still
    const ScenePar& P = d.par[s];
    const size_t N = (size_t)d.N;
    const double r = pp.w;
    const int nwall = P.wall == WALL_CUBE ? 6 : (P.wall == WALL_CYL ? 3 : 0);
    {
        // conservative early-out: clearly inside every wall and outside the
        // intruder's bounding sphere (margins of 1e-9 relative cover rounding)
        const double ex = pp.x - P.w_c[0], ey = pp.y - P.w_c[1], ez = pp.z - P.w_c[2];
        bool near = false;
        if (P.wall == WALL_CUBE) {
            near = fabs(ex) + r >= P.w_half[0] * (1 - 1e-9) || fabs(ey) + r >= P.w_half[1] * (1 - 1e-9) ||
                   fabs(ez) + r >= P.w_half[2] * (1 - 1e-9);
        } else if (P.wall == WALL_CYL) {
            const double ax = ex * P.cyl_axis[0] + ey * P.cyl_axis[1] + ez * P.cyl_axis[2];
            const double rr = ex * ex + ey * ey + ez * ez - ax * ax;
            const double in = P.cyl_R - r;
            near = fabs(ax) + r >= P.cyl_H * (1 - 1e-9) || in <= 0 || rr >= in * in * (1 - 1e-9);
        }
        if (!near && P.has_intr) {
            const SceneDyn& y = d.dyn[s];
            const double qx = pp.x - y.intr_p[0], qy = pp.y - y.intr_p[1], qz = pp.z - y.intr_p[2];
            const double reach = (P.intr_shape == 1 ? P.intr_R : sqrt(P.intr_R * P.intr_R + P.intr_H * P.intr_H) +
                                  0.80 * P.cell[0] * 1.7320508075688772) + r;
            near = qx * qx + qy * qy + qz * qz <= reach * reach * (1 + 1e-9);
        }
        if (!near) {
            if (bb_old) d.bbits[i] = 0;
            if (EXPORT) {
                R4<R>* xp = (R4<R>*)d.xparts;
                R4<R>* xi = (R4<R>*)d.xintr;
                const R4<R> z = pack<R>(v3<R>(0, 0, 0), R(0));
                for (int c = 2; c < 6; c++) xp[(size_t)c * N + i] = z;
                for (int c = 0; c < 4; c++) xi[(size_t)c * N + i] = z;
            }
            return;
        }
    }
    uint16_t bb_new = 0;
    R4<R>* BH = (R4<R>*)d.bhist;
    V3<R> wF = v3<R>(0, 0, 0), wT = wF, iF = wF, iT = wF;
    Body<R> me;
    bool have_kin = false;
    Law<R> L;
    L.kn_fac = P.kn_fac; L.ks_fac = P.ks_fac; L.damping = P.damping;
    L.beta = (R)P.beta; L.mu = (R)P.mu; L.dt = (R)P.dt;
    const V3<double> RV = v3(pp.x - P.w_c[0], pp.y - P.w_c[1], pp.z - P.w_c[2]);
    // cylinder geometry shared by its three regions
    double ERRc = 0, nrmc = 0;
    V3<double> RVbc = v3(0.0, 0.0, 0.0), RVtc = RVbc, axv = RVbc;
    if (P.wall == WALL_CYL) {
        axv = v3(P.cyl_axis[0], P.cyl_axis[1], P.cyl_axis[2]);
        ERRc = dot(RV, axv);
        RVbc = RV - ERRc * axv;
        RVtc = ERRc * axv;
        nrmc = len_floor(RVbc);
    }
    for (int slot = 0; slot < NB_SLOTS; slot++) {
        const bool is_wall = slot < nwall;
        const bool is_intr = slot == SLOT_INTR && P.has_intr;
        if (!is_wall && !is_intr) continue;
        double Apd = 0, Dnd = 0;
        V3<double> nd = v3(0.0, 0.0, 0.0), RVo = nd;
        bool on = false;
        double Rij = r, Mij = 0.0;
        R csm = R(2);
        V3<double> wv = v3(P.w_v[0], P.w_v[1], P.w_v[2]);
        V3<double> ww = v3(P.w_w[0], P.w_w[1], P.w_w[2]);
        if (is_wall && P.wall == WALL_CUBE) {
            const int ax = slot >> 1;
            const bool up = (slot & 1) == 0;
            const double e = (ax == 0 ? RV.x : (ax == 1 ? RV.y : RV.z)), h = P.w_half[ax];
            on = up ? (e > 0 && e + r - h > 0) : (e < 0 && e - r + h < 0);
            if (on) {
                const double o = (h / fabs(e)) * e;
                RVo = RV;
                if (ax == 0) RVo.x = o; else if (ax == 1) RVo.y = o; else RVo.z = o;
                const double sgn = up ? -1.0 : 1.0;
                if (ax == 0) nd.x = sgn; else if (ax == 1) nd.y = sgn; else nd.z = sgn;
                Apd = dot(RV - RVo, nd);
                Dnd = r - Apd;
                on = Dnd > 0.0;
            }
        } else if (is_wall) {
            const double d_cap = fabs(ERRc) - P.cyl_H + r;
            const double d_side = nrmc - P.cyl_R + r;
            if (slot == 0) on = d_cap >= 1e-14 && ERRc < 0;
            else if (slot == 1) on = d_cap >= 1e-14 && ERRc > 0;
            else on = d_side >= 1e-14;
            if (on) {
                RVo = slot < 2 ? (P.cyl_H / fabs(ERRc)) * RVtc + RVbc : (P.cyl_R / nrmc) * RVbc + RVtc;
                const V3<double> RVn = RV - RVo;
                Dnd = r - len_floor(RVn);
                on = Dnd > 0.0;
                if (on) {
                    const double DistL = sqrt(RVn.x * RVn.x + RVn.y * RVn.y + RVn.z * RVn.z);
                    nd = (1.0 / DistL) * RVn;
                    Apd = DistL;
                }
            }
        } else {
            const SceneDyn& y = d.dyn[s];
            const V3<double> RI = v3(pp.x - y.intr_p[0], pp.y - y.intr_p[1], pp.z - y.intr_p[2]);
            wv = v3(y.intr_v[0], y.intr_v[1], y.intr_v[2]);
            ww = v3(P.intr_w[0], P.intr_w[1], P.intr_w[2]);
            csm = R(1);
            if (P.intr_shape == 1) {
                const double cd = len_floor(RI);
                if (cd > 1.0e-15) nd = (1.0 / cd) * RI;
                else {
                    V3<double> fb = v3(P.intr_axis[0], P.intr_axis[1], P.intr_axis[2]);
                    double t2 = sqrt(dot(fb, fb));
                    nd = t2 > 1e-20 ? (1.0 / t2) * fb : v3(0.0, 0.0, 0.0);
                    if (len_floor(nd) < 1.0e-15) nd = v3(0.0, 0.0, 1.0);
                }
                RVo = P.intr_R * nd;
                const double gap = cd - P.intr_R;
                Dnd = r - gap;
                Apd = gap;
                on = Dnd > 0.0;
                Rij = r * P.intr_R / (r + P.intr_R);
            } else {
                const double LatDx = P.cell[0];
                const V3<double> pv = v3(P.intr_axis[0], P.intr_axis[1], P.intr_axis[2]);
                const double ERR = dot(RI, pv);
                if (fabs(ERR) < (P.intr_H + 0.80 * LatDx)) {
                    const V3<double> RVb = RI - ERR * pv;
                    const double nrm = len_floor(RVb);
                    if (nrm < (P.intr_R + 0.80 * LatDx)) {
                        const V3<double> RVt = ERR * pv;
                        if (fabs(ERR) < P.intr_H) RVo = ((1.0 / nrm) * P.intr_R) * RVb + RVt;
                        else if (nrm < P.intr_R) RVo = ((1.0 / fabs(ERR)) * P.intr_H) * RVt + RVb;
                        else RVo = ((1.0 / nrm) * P.intr_R) * RVb + ((1.0 / fabs(ERR)) * P.intr_H) * RVt;
                        const V3<double> RVn = RI - RVo;
                        const double DistL = sqrt(RVn.x * RVn.x + RVn.y * RVn.y + RVn.z * RVn.z);
                        Dnd = r - DistL;
                        on = Dnd > 0.0;
                        if (on) { nd = (1.0 / DistL) * RVn; Apd = DistL; }
                    }
                }
            }
            if (on && P.intr_wait) atomicCAS(&d.dyn[s].intr_state, 0, 1);
        }
        if (!on) continue;
        if (!have_kin) {
            me.p = pp;
            load_kin<R>(d, i, d.clump_id[i], me);
            have_kin = true;
        }
        if (is_intr) Mij = P.intr_motion == 1 ? me.m * P.intr_mass / (me.m + P.intr_mass) : me.m;
        else Mij = me.m;
        V3<R> hs = v3<R>(0, 0, 0), ht = hs, hr = hs;
        const size_t hb = (size_t)slot * 3 * N;
        // the sphere driver's cube wall keeps no history
        const bool memless = SPH && is_wall && P.wall == WALL_CUBE && (P.sphere & SPH_CUBE);
        if (!memless && (bb_old & (1u << slot))) {
            R4<R> a = BH[hb + 3 * i], b = BH[hb + 3 * i + 1], c = BH[hb + 3 * i + 2];
            hs = xyz<R>(a); ht = xyz<R>(b); hr = xyz<R>(c);
        }
        V3<R> f, t, arm;
        LawOut<R> o;
        boundary_contact<R>(L, me, nd, Apd, Dnd, RVo, wv, ww, Rij, Mij, csm, hs, hr, ht,
                            f, t, o, arm);
        if (SPH && memless) {
            // tangential torque only: the moments and the history writes
            // are commented out there (src/dem_force_cube_wall.cu:86-87,137-141)
            t = (-(R)Apd) * cross(cvt<R>(nd), o.Ft);
        } else {
            BH[hb + 3 * i] = pack<R>(o.hs, R(0));
            BH[hb + 3 * i + 1] = pack<R>(o.ht, R(0));
            BH[hb + 3 * i + 2] = pack<R>(o.hr, R(0));
        }
        if (SPH && is_intr && (P.sphere & SPH_KIN)) {
            // the sphere driver's penetrator law adds cohesion
            // (src/dem_force_penetrator.cu:119-123)
            const double cf = ((-P.cohesion) * (P.beta * Rij)) * (P.beta * Rij);
            f = f + cvt<R>(cf * nd);
        }
        bb_new |= (uint16_t)(1u << slot);
        if (is_intr) {
            iF = iF + f;
            iT = iT + t;
            // torque on the intruder about its centre (src/dem_force_penetrator_clump.cu:125,170)
            const V3<R> pt = (-cross(cvt<R>(RVo), f) + o.Mr) + o.Mt;
            long long* fx = (long long*)&d.dyn[s].ifix[0];
            atomicAdd((unsigned long long*)&fx[0], (unsigned long long)llrint((double)f.x * FIX_F));
            atomicAdd((unsigned long long*)&fx[1], (unsigned long long)llrint((double)f.y * FIX_F));
            atomicAdd((unsigned long long*)&fx[2], (unsigned long long)llrint((double)f.z * FIX_F));
            atomicAdd((unsigned long long*)&fx[3], (unsigned long long)llrint((double)pt.x * FIX_T));
            atomicAdd((unsigned long long*)&fx[4], (unsigned long long)llrint((double)pt.y * FIX_T));
            atomicAdd((unsigned long long*)&fx[5], (unsigned long long)llrint((double)pt.z * FIX_T));
            if (EXPORT) {
                R4<R>* xi = (R4<R>*)d.xintr;
                xi[i] = pack<R>(o.Fn, R(0));
                xi[N + i] = pack<R>(o.Ft, R(0));
                xi[2 * N + i] = pack<R>(cross(o.Fn, arm), R(0));
                xi[3 * N + i] = pack<R>((cross(o.Ft, arm) - o.Mr) - o.Mt, R(0));
            }
        } else {
            wF = wF + f;
            wT = wT + t;
        }
    }
    d.bbits[i] = bb_new;
    if (bb_new) {
        R4<R>* fb = (R4<R>*)d.fbnd;
        fb[i] = pack<R>(wF + iF, R(0));
        fb[N + i] = pack<R>(wT + iT, R(0));
        if (SPH && (P.sphere & SPH_KIN) && (bb_new & (1u << SLOT_INTR))) {
            R4<R>* fi = (R4<R>*)d.fint;
            fi[i] = pack<R>(iF, R(0));
            fi[N + i] = pack<R>(iT, R(0));
        }
    }
    if (EXPORT) {
        R4<R>* xp = (R4<R>*)d.xparts;
        xp[2 * N + i] = pack<R>(wF, R(0));
        xp[3 * N + i] = pack<R>(wT, R(0));
        xp[4 * N + i] = pack<R>(iF, R(0));
        xp[5 * N + i] = pack<R>(iT, R(0));
        if (!(bb_new & (1u << SLOT_INTR))) {
            R4<R>* xi = (R4<R>*)d.xintr;
            const R4<R> z = pack<R>(v3<R>(0, 0, 0), R(0));
            xi[i] = z; xi[N + i] = z; xi[2 * N + i] = z; xi[3 * N + i] = z;
        }
    }
}

// Overlap of a listed pair: the reference's test ri + rj - |d| > 0 in FP64
// (src/dem_force_clump.cu:46-50), with the square root taken only when |d|^2
// is within 1e-12 of (ri + rj)^2, so the decision is the reference's exactly.
__device__ __forceinline__ bool overlaps(double4 a, double4 b) {
    const double dx = b.x - a.x, dy = b.y - a.y, dz = b.z - a.z;
    const double d2 = dx * dx + dy * dy + dz * dz;
    const double s = a.w + b.w, s2 = s * s;
    if (d2 > s2 * (1.0 + 1e-12)) return false;
    if (d2 < s2 * (1.0 - 1e-12)) return true;
    return a.w + b.w - sqrt(d2) > 0.0;
}

// The law of one touching near pair (front entry ef of scene s, pair slot p,
// owner i of clump ci, partner jr of clump cj, near back entry eb; a.p and b.p
// loaded): kinematics and spring history in, new history, touch flag and the
// four contact slots out (and the export record).
template <typename R, bool EXPORT>
__device__ __forceinline__ void pair_law(const Dev& d, int s, int ef, int p, int i, int jr, int ci, int cj, int eb,
                                         Body<R>& a, Body<R>& b) {
    const int hg = *d.hgen;
    const size_t cap = (size_t)d.cap;
    load_kin<R>(d, i, ci, a);
    load_kin<R>(d, jr, cj, b);
    V3<R> hs = v3<R>(0, 0, 0), ht = hs, hr = hs;
    if (d.touch[hg & 1][p]) hist_read<R>((const R4<R>*)d.H[hg & 1], cap, p, hs, ht, hr);
    const ScenePar& P = d.par[s];
    Law<R> L;
    L.kn_fac = P.kn_fac; L.ks_fac = P.ks_fac; L.damping = P.damping;
    L.beta = (R)P.beta; L.mu = (R)P.mu; L.dt = (R)P.dt;
    V3<R> fa, ta, tb;
    LawOut<R> o;
    double Ap;
    V3<double> nd;
    pair_contact2<R>(L, (R)P.cohesion, a, b, hs, hr, ht, fa, ta, tb, o, Ap, nd);
    hist_write<R>((R4<R>*)d.H[(hg + 1) & 1], cap, p, o.hs, o.ht, o.hr);
    d.touch[(hg + 1) & 1][p] = 1;
    R4<R>* fs = (R4<R>*)d.nfs;
    R4<R>* bs = (R4<R>*)d.nbs;
    fs[2 * (size_t)ef] = pack<R>(fa, R(0));
    fs[2 * (size_t)ef + 1] = pack<R>(ta, R(0));
    bs[2 * (size_t)eb] = pack<R>(-fa, R(0));
    bs[2 * (size_t)eb + 1] = pack<R>(tb, R(0));
    if (EXPORT) {
        R4<R>* xf = (R4<R>*)d.xfcn;
        double4* xc = (double4*)d.xcpt;
        xf[p] = pack<R>(-o.Fn, R(0));
        xc[p] = make_double4(a.p.x + Ap * nd.x, a.p.y + Ap * nd.y, a.p.z + Ap * nd.z, 0.0);
    }
}

// Pairs, one thread per near front entry (grid-stride, so a captured launch
// covers a list that has grown since): the overlap test, and for touching
// pairs the law once (ContactForce_clump_cuk, src/dem_force_clump.cu:3-163,
// for both particles of the pair) and the owner's new spring history.  The
// force and torque on the owner go to the entry's front slot, those on the
// partner to the pair's near back slot (zero when the pair does not touch),
// so the clump pass sums every subsphere's contacts from two contiguous slot
// ranges in row order.  Block 0 marks this step's closing half-kick as
// pending.
constexpr int PR_THREADS = 256;

// resident blocks of k_pairs per SM: the FP64 contact kinematics of two
// bodies need up to 128 registers a thread without spilling
#ifndef NBC_PAIR_MINB
#define NBC_PAIR_MINB 2
#endif
constexpr int CONTACT_LAUNCHES = 2;   // k_pairs and k_boundary
template <typename R, bool EXPORT>
__global__ void __launch_bounds__(PR_THREADS, NBC_PAIR_MINB) k_pairs(const Dev* __restrict__ dp) {
    const Dev& d = *dp;
    if (*d.halt) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) *d.post_pending = 1;
    const int hg = *d.hgen;
    const int S = d.S;
    const int* __restrict__ npre = d.nprefix;
    const int np = npre[S];
    const int4* __restrict__ nfr = d.nfr;
    const double4* __restrict__ posr = d.posr;
    const int* __restrict__ cid = d.clump_id;
    uint8_t* __restrict__ to = d.touch[(hg + 1) & 1];
    R4<R>* __restrict__ fs = (R4<R>*)d.nfs;
    R4<R>* __restrict__ bs = (R4<R>*)d.nbs;
    const R4<R> zero = pack<R>(v3<R>(0, 0, 0), R(0));
    // work item w: near front entry w - nprefix[s] of scene s; its record
    // (pair slot, partner, owner, near back entry) is loaded one item ahead
    auto fetch = [&](int w, int4& rec, int& s, int& ef) {
        if (w >= np) return false;
        s = S == 1 ? 0 : plan_find(npre, S, w);
        const SceneDyn& ys = d.dyn[s];
        if (d.has_stops && ys.frozen) return false;
        ef = ys.pair_off + (w - npre[s]);
        rec = nfr[ef];
        return true;
    };
    const int stride = gridDim.x * blockDim.x;
    int4 recn = make_int4(0, 0, 0, 0);
    int sn = 0, efn = 0;
    bool liven = fetch(blockIdx.x * blockDim.x + threadIdx.x, recn, sn, efn);
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < np; w += stride) {
        const int4 rec = recn;
        const int s = sn, ef = efn;
        const bool live = liven;
        liven = fetch(w + stride, recn, sn, efn);
        if (!live) continue;
        const int p = rec.x, jr = rec.y, i = rec.z, eb = rec.w;
        Body<R> a, b;
        bool on = jr >= 0;   // pairs inside one clump have no force (src/dem_force_clump.cu:18-19)
        int ci = 0, cj = 0;
        if (on) {
            a.p = posr[i];
            b.p = posr[jr];
            ci = cid[i];      // with the positions, for the kinematics of a touching pair
            cj = cid[jr];
            on = overlaps(a.p, b.p);
        }
        if (!on) {
            to[p] = 0;
            fs[2 * (size_t)ef] = zero;
            fs[2 * (size_t)ef + 1] = zero;
            bs[2 * (size_t)eb] = zero;
            bs[2 * (size_t)eb + 1] = zero;
            continue;
        }
        pair_law<R, EXPORT>(d, s, ef, p, i, jr, ci, cj, eb, a, b);
    }
}

// The contact force and torque on subsphere i: its contact slots, then the
// wall and intruder force where a boundary slot is in contact -- the sum the
// clump pass forms, so the per-subsphere totals read back are bitwise the
// ones it integrates.
template <typename R>
__device__ __forceinline__ void contact_sum(const Dev& d, int i, int s, V3<R>& F, V3<R>& T, V3<R>* pairF = nullptr,
                                            V3<R>* pairT = nullptr) {
    const size_t N = (size_t)d.N;
    const int2 ra = d.nrb[i + s], rb = d.nrb[i + s + 1];
    slot_sum<R>((const R4<R>*)d.nfs, (const R4<R>*)d.nbs, (size_t)d.cap, ra.x, rb.x, ra.y, rb.y, F, T);
    if (pairF) { *pairF = F; *pairT = T; }
    if (d.bbits[i]) {
        const R4<R>* fb = (const R4<R>*)d.fbnd;
        F = F + xyz<R>(fb[i]);
        T = T + xyz<R>(fb[N + i]);
    }
}

// Per subsphere, on request (the force getters and the export step): the
// totals of contact_sum into fsum, the pair part into the export record.
template <typename R, bool EXPORT>
__global__ void __launch_bounds__(CT_THREADS) k_sum(const Dev* __restrict__ dp) {
    const Dev& d = *dp;
    if (*d.halt) return;
    const int i = blockIdx.x * CT_THREADS + threadIdx.x;
    if (i >= d.N) return;
    const size_t N = (size_t)d.N;
    const int s = d.S == 1 ? 0 : d.sid[i];
    if (d.has_stops && d.dyn[s].frozen) return;
    V3<R> F, T, pF, pT;
    contact_sum<R>(d, i, s, F, T, &pF, &pT);
    if (EXPORT) {
        R4<R>* xp = (R4<R>*)d.xparts;
        xp[i] = pack<R>(pF, R(0));
        xp[N + i] = pack<R>(pT, R(0));
    }
    R4<R>* fo = (R4<R>*)d.fsum;
    fo[i] = pack<R>(F, R(0));
    fo[N + i] = pack<R>(T, R(0));
}

}  // namespace nbc
