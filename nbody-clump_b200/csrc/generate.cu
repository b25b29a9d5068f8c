// generate.cu -- mass properties of clump templates (scene generation).
//
// The reference's template builder (make_clump_template_lambda.m:172-209)
// estimates the union volume, centre of mass and inertia tensor of a clump's
// overlapping spheres by deterministic Monte Carlo integration over the
// clump's bounding box, counting overlap once.  nbc_union_mass does that for
// many clumps at once: one block per clump, the points of a Kronecker
// low-discrepancy sequence (the three-dimensional R sequence: coordinates
// frac(0.5 + n a_d), a_d = 1/g^d with g the positive root of g^4 = g + 1, so
// that 1, a_1, a_2, a_3 are rationally independent), so the result is the
// same on every run and converges faster than random points.  The host turns the
// moments into mass, centre of mass and inertia (scenegen.py) and rotates
// the template into its principal frame.
#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/nbc.h"
#include "handle.h"

namespace {

constexpr int UM_THREADS = 256;
constexpr int UM_MAX_MEMBERS = 64;   // members of one clump staged in shared memory

// Sums over one block in a fixed tree order (deterministic).
__device__ __forceinline__ double block_sum(double v, double* sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double t = 0;
    if (warp == 0) {
        t = lane < UM_THREADS / 32 ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    }
    __syncthreads();
    return t;   // valid in thread 0
}

// out[k][10]: volume, centroid (3), second central moments per unit volume
// xx, yy, zz, xy, xz, yz (the centroid and moments relative to the clump's
// own frame).
__global__ void __launch_bounds__(UM_THREADS) k_union_mass(const double* __restrict__ cen,
                                                           const double* __restrict__ rad,
                                                           const int* __restrict__ start, int K, int samples,
                                                           double* __restrict__ out) {
    __shared__ double4 s_m[UM_MAX_MEMBERS];
    __shared__ double s_box[6];
    __shared__ double sh[UM_THREADS / 32];
    const double g = 1.22074408460575947536;   // g^4 = g + 1
    const double a1 = 1.0 / g, a2 = 1.0 / (g * g), a3 = 1.0 / (g * g * g);
    for (int k = blockIdx.x; k < K; k += gridDim.x) {
        const int m0 = start[k], nm = start[k + 1] - start[k];
        for (int j = threadIdx.x; j < nm && j < UM_MAX_MEMBERS; j += UM_THREADS)
            s_m[j] = make_double4(cen[3 * (m0 + j)], cen[3 * (m0 + j) + 1], cen[3 * (m0 + j) + 2], rad[m0 + j]);
        if (threadIdx.x == 0) {
            double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
            for (int j = 0; j < nm; j++) {
                const double r = rad[m0 + j];
                for (int c = 0; c < 3; c++) {
                    lo[c] = fmin(lo[c], cen[3 * (m0 + j) + c] - r);
                    hi[c] = fmax(hi[c], cen[3 * (m0 + j) + c] + r);
                }
            }
            for (int c = 0; c < 3; c++) { s_box[c] = lo[c]; s_box[3 + c] = hi[c] - lo[c]; }
        }
        __syncthreads();
        const double bx = s_box[0], by = s_box[1], bz = s_box[2], ex = s_box[3], ey = s_box[4], ez = s_box[5];
        // moments about the box centre (small coordinates, little cancellation)
        const double ox = bx + 0.5 * ex, oy = by + 0.5 * ey, oz = bz + 0.5 * ez;
        double c0 = 0, sx = 0, sy = 0, sz = 0, sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
        for (int n = threadIdx.x; n < samples; n += UM_THREADS) {
            const double u = 0.5 + n * a1, v = 0.5 + n * a2, w = 0.5 + n * a3;
            const double x = bx + ex * (u - floor(u)), y = by + ey * (v - floor(v)), z = bz + ez * (w - floor(w));
            bool in = false;
            for (int j = 0; j < nm && !in; j++) {
                const double4 m = j < UM_MAX_MEMBERS ? s_m[j]
                                                     : make_double4(cen[3 * (m0 + j)], cen[3 * (m0 + j) + 1],
                                                                    cen[3 * (m0 + j) + 2], rad[m0 + j]);
                const double dx = x - m.x, dy = y - m.y, dz = z - m.z;
                in = dx * dx + dy * dy + dz * dz <= m.w * m.w;
            }
            if (in) {
                const double px = x - ox, py = y - oy, pz = z - oz;
                c0 += 1.0;
                sx += px; sy += py; sz += pz;
                sxx += px * px; syy += py * py; szz += pz * pz;
                sxy += px * py; sxz += px * pz; syz += py * pz;
            }
        }
        const double n_in = block_sum(c0, sh);
        const double tx = block_sum(sx, sh), ty = block_sum(sy, sh), tz = block_sum(sz, sh);
        const double txx = block_sum(sxx, sh), tyy = block_sum(syy, sh), tzz = block_sum(szz, sh);
        const double txy = block_sum(sxy, sh), txz = block_sum(sxz, sh), tyz = block_sum(syz, sh);
        if (threadIdx.x == 0) {
            double* o = out + 10 * (size_t)k;
            const double vol = ex * ey * ez * n_in / samples;
            const double inv = n_in > 0 ? 1.0 / n_in : 0.0;
            const double mx = tx * inv, my = ty * inv, mz = tz * inv;
            o[0] = vol;
            o[1] = ox + mx; o[2] = oy + my; o[3] = oz + mz;
            o[4] = txx * inv - mx * mx; o[5] = tyy * inv - my * my; o[6] = tzz * inv - mz * mz;
            o[7] = txy * inv - mx * my; o[8] = txz * inv - mx * mz; o[9] = tyz * inv - my * mz;
        }
        __syncthreads();
    }
}

template <typename T>
T* dev_copy(const T* h, size_t n) {
    T* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) throw std::runtime_error("cudaMalloc failed");
    if (n && cudaMemcpy(p, h, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(p);
        throw std::runtime_error("copy to the device failed");
    }
    return p;
}

}  // namespace

extern "C" nbc_status nbc_union_mass(const double* centres, const double* radii, const int* clump_start, int nclumps,
                                     int samples, double* out, int device) {
    return nbc::guard([&] {
        if (!centres || !radii || !clump_start || !out || nclumps < 0 || samples < 1)
            throw std::invalid_argument("nbc_union_mass: null pointer, negative clump count or no samples");
        if (nclumps == 0) return;
        const int nm = clump_start[nclumps];
        if (clump_start[0] != 0 || nm < 0) throw std::invalid_argument("nbc_union_mass: clump_start must start at 0");
        for (int k = 0; k < nclumps; k++)
            if (clump_start[k + 1] <= clump_start[k])
                throw std::invalid_argument("nbc_union_mass: every clump needs at least one member");
        for (int j = 0; j < nm; j++)
            if (!(radii[j] > 0)) throw std::invalid_argument("nbc_union_mass: radii must be positive");
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw std::runtime_error("no CUDA device");
        if (cudaSetDevice(device) != cudaSuccess) throw std::runtime_error("cudaSetDevice failed");
        double* dc = nullptr;
        double* dr = nullptr;
        int* ds = nullptr;
        double* dout = nullptr;
        std::string err;
        try {
            dc = dev_copy(centres, 3 * (size_t)nm);
            dr = dev_copy(radii, (size_t)nm);
            ds = dev_copy(clump_start, (size_t)nclumps + 1);
            if (cudaMalloc(&dout, 10 * (size_t)nclumps * sizeof(double)) != cudaSuccess)
                throw std::runtime_error("cudaMalloc failed");
            k_union_mass<<<std::min(nclumps, 148 * 64), UM_THREADS>>>(dc, dr, ds, nclumps, samples, dout);
            cudaError_t e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaDeviceSynchronize();
            if (e != cudaSuccess) throw std::runtime_error(std::string("k_union_mass: ") + cudaGetErrorString(e));
            if (cudaMemcpy(out, dout, 10 * (size_t)nclumps * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
                throw std::runtime_error("copy from the device failed");
        } catch (const std::exception& x) {
            err = x.what();
        }
        cudaFree(dc);
        cudaFree(dr);
        cudaFree(ds);
        cudaFree(dout);
        if (!err.empty()) throw std::runtime_error(err);
    });
}
