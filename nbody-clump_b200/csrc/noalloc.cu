// noalloc.cu -- a cell sort that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host program whose device memory
// is owned by another framework's pool, or code running where allocation is
// forbidden once a run has started (a memory budget fixed at start-up).
// nbc_cell_sort_noalloc gives them the engine's cell hash and a stable radix
// sort by cell (the order of the first half of a list rebuild) using only
// buffers the caller passes plus one scratch array compiled into this library.
//
// Scratch: `g_sort_scratch` below, NBC_NOALLOC_MAX_N elements of key/value
// ping-pong plus the radix histograms, about 2.2 MB, held on every GPU that
// loads the library until the process exits.  Every call on a device shares
// it and it keeps the previous call's contents (the histograms are rebuilt
// from zero by each pass, the ping-pong halves are fully overwritten), so
// calls whose work overlaps on the GPU -- on two streams, or from two host
// threads -- race on it and must be serialised by the caller.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/nbc.h"
#include "kernels.cuh"

namespace nbc {
extern thread_local std::string g_last_error;
}

namespace {

constexpr int MAX_N = NBC_NOALLOC_MAX_N;
constexpr int MAX_TILES = (MAX_N + nbc::RS_TILE - 1) / nbc::RS_TILE;
constexpr int HIST = 256 * MAX_TILES;
constexpr int SCAN_SUMS = (HIST + nbc::SC_TILE - 1) / nbc::SC_TILE + 1;
constexpr size_t SCRATCH_INTS = 2 * (size_t)MAX_N + HIST + SCAN_SUMS;

// the scratch array; host code must not pass its name to a kernel (in host
// code it is only a stand-in), it uses the device address looked up below
__device__ __align__(256) int g_sort_scratch[SCRATCH_INTS];

constexpr int MAX_DEVICES = 64;
int* g_scratch_addr[MAX_DEVICES] = {nullptr};
std::mutex g_scratch_mu;

nbc_status fail(nbc_status code, const std::string& m) {
    nbc::g_last_error = m;
    return code;
}

// GetParticleCellIndex_cuk (src/dem_grid.cu:155-202) on caller buffers
__global__ void k_hash_plain(const double* __restrict__ pos, int n, nbc_grid_desc g, int* __restrict__ keys,
                             int* __restrict__ vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    const int cellnum = g.dims[0] * g.dims[1] * g.dims[2];
    int local;
    if (z >= g.box_hi[2] || y >= g.box_hi[1] || x >= g.box_hi[0] || z < g.box_lo[2] || y < g.box_lo[1] ||
        x < g.box_lo[0]) {
        local = cellnum - 1;
    } else {
        int cx = nbc::clampi((int)floor((x - g.origin[0]) / g.cell), 0, g.dims[0] - 1);
        int cy = nbc::clampi((int)floor((y - g.origin[1]) / g.cell), 0, g.dims[1] - 1);
        int cz = nbc::clampi((int)floor((z - g.origin[2]) / g.cell), 0, g.dims[2] - 1);
        local = nbc::clampi(cz * g.dims[1] * g.dims[0] + cy * g.dims[0] + cx, 0, cellnum - 1);
    }
    keys[i] = local;
    vals[i] = i;
}

void scan_ints(int* a, int n, int* sums, cudaStream_t st) {
    const int nb = (n + nbc::SC_TILE - 1) / nbc::SC_TILE;
    nbc::k_scan_tiles<<<nb, nbc::SC_THREADS, 0, st>>>(a, n, sums, nullptr);
    nbc::k_scan_sums<<<1, nbc::SC_THREADS, 0, st>>>(sums, nb, nullptr);
    nbc::k_scan_add<<<nb, nbc::SC_THREADS, 0, st>>>(a, n, sums, nullptr);
}

}  // namespace

extern "C" nbc_status nbc_cell_sort_noalloc(const double* pos_dev, int n, const nbc_grid_desc* grid, int* perm_dev,
                                            int* key_dev, void* stream) {
    if (n < 0 || n > MAX_N)
        return fail(NBC_ERR_ARG, "nbc_cell_sort_noalloc: n = " + std::to_string(n) + " is outside 0.." +
                                     std::to_string(MAX_N) + " (the size of the library's scratch array)");
    if (!grid || (n > 0 && (!pos_dev || !perm_dev || !key_dev)))
        return fail(NBC_ERR_ARG, "nbc_cell_sort_noalloc: null argument");
    const long long cells = (long long)grid->dims[0] * grid->dims[1] * grid->dims[2];
    if (grid->dims[0] <= 0 || grid->dims[1] <= 0 || grid->dims[2] <= 0 || cells > (1LL << 30) || !(grid->cell > 0))
        return fail(NBC_ERR_ARG, "nbc_cell_sort_noalloc: bad grid");
    if (n == 0) return NBC_OK;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(NBC_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= MAX_DEVICES) return fail(NBC_ERR_ARG, "device ordinal too large");
    cudaStream_t st = (cudaStream_t)stream;
    int* scratch;
    {
        // The scratch array's device address, with the device current.  It
        // is looked up again on every call made outside a stream capture (a
        // device reset rebuilds the context and may move the array); a call
        // inside a capture uses the address the last uncaptured call on this
        // device found, so the first call on a device must come before any
        // capture.
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        e = cudaStreamIsCapturing(st, &cs);
        if (e != cudaSuccess)
            return fail(NBC_ERR_CUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e));
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        if (cs == cudaStreamCaptureStatusNone) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_sort_scratch);
            if (e != cudaSuccess)
                return fail(NBC_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_scratch_addr[dev] = (int*)p;
        } else if (!g_scratch_addr[dev]) {
            return fail(NBC_ERR_STATE, "nbc_cell_sort_noalloc: the first call on a device must not be captured");
        }
        scratch = g_scratch_addr[dev];
    }
    int* kB = scratch;
    int* vB = kB + MAX_N;
    int* hist = vB + MAX_N;
    int* sums = hist + HIST;
    int bits = 1;
    while ((1LL << bits) < cells) bits++;
    const int passes = (bits + 7) / 8;
    const int tiles = (n + nbc::RS_TILE - 1) / nbc::RS_TILE;
    // the caller's output buffers are one side of the ping-pong; with an odd
    // pass count the first pass starts from the scratch side so the last
    // pass lands in the caller's buffers
    int *ki, *vi, *ko, *vo;
    if (passes % 2 == 1) { ki = kB; vi = vB; ko = key_dev; vo = perm_dev; }
    else { ki = key_dev; vi = perm_dev; ko = kB; vo = vB; }
    k_hash_plain<<<(n + 127) / 128, 128, 0, st>>>(pos_dev, n, *grid, ki, vi);
    for (int p = 0; p < passes; p++) {
        nbc::k_rs_hist<<<tiles, nbc::RS_THREADS, 0, st>>>(ki, n, 8 * p, hist, nullptr);
        scan_ints(hist, 256 * tiles, sums, st);
        nbc::k_rs_scatter<<<tiles, nbc::RS_THREADS, 0, st>>>(ki, vi, ko, vo, n, 8 * p, hist, nullptr);
        int* t = ki; ki = ko; ko = t;
        t = vi; vi = vo; vo = t;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(NBC_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return NBC_OK;
}
