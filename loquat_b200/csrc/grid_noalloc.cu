/*
 * Neighbour search that allocates nothing.
 *
 * lq_grid_neighbor_search needs a grid object (lq_grid_create) whose
 * working arrays come from cudaMalloc.  Some callers cannot allocate device
 * memory on their own: a host code that hands this library a fixed slice of
 * a GPU whose memory its own pool has already reserved (cudaMalloc then
 * fails, or breaks the pool's budget), and a time-step loop that cannot
 * afford cudaMalloc's device-wide synchronisation in the middle of a step.
 * For them this file keeps the search's working arrays in one file-scope
 * device array of fixed size, so the call takes only the caller's inputs
 * and outputs.
 *
 * Limits: at most LQ_NOALLOC_MAX_PARTICLES particles and LQ_NOALLOC_MAX_CELLS
 * cells per call; larger problems are rejected with LQ_ERR_ARG.  The array
 * (17 MiB) is held on every device that loads this code, until the process
 * exits.  Every call on a device shares it and it keeps the previous call's
 * contents; the per-cell counters are cleared at the start of each call.
 * Calls that overlap on the GPU (two streams, or two host threads) race on
 * the array and produce wrong results: serialise them.
 *
 * Host code sees only a host-side stand-in for the array; its device
 * address is looked up with cudaGetSymbolAddress (with the device current)
 * on every call made outside stream capture, so a module reloaded after
 * cudaDeviceReset is found again, and cached per device for calls made
 * while the stream is being captured.  A call inside a capture before any
 * call outside one on that device is rejected with LQ_ERR_ARG: make one
 * call before capture begins.
 *
 * Particles outside the lattice all land in the last cell, whose in-cell
 * ordering is one thread's insertion sort: keep their number small (the
 * health word of the native driver counts them).
 */
#include <mutex>

#include "lq_internal.cuh"

namespace {

constexpr int kMaxParticles = LQ_NOALLOC_MAX_PARTICLES;
constexpr int kMaxCells = LQ_NOALLOC_MAX_CELLS;
constexpr size_t kTable = sizeof(int) * (size_t)(kMaxParticles > kMaxCells + 1 ? kMaxParticles : kMaxCells + 1);
constexpr size_t kScanBytes = (size_t)1 << 20;
constexpr size_t kScratchBytes = 4 * kTable + kScanBytes;   /* key | rank | count | start | scan */

static __device__ __align__(256) unsigned char g_search_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

/* Device address of the scratch array on the current device: asked of
 * the runtime outside stream capture, the cached answer inside one. */
int scratch_address(cudaStream_t stream, void** out)
{
    int dev = 0;
    LQ_TRY_CUDA(cudaGetDevice(&dev), "noalloc search: cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return lqb::set_error(LQ_ERR_ARG, "noalloc search: device %d out of range", dev);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess) {
        cudaGetLastError();
        cs = cudaStreamCaptureStatusActive;   /* cannot tell: treat as capturing, ask nothing */
    }
    std::lock_guard<std::mutex> lock(g_mu);
    if (cs == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_search_scratch);
        if (e != cudaSuccess) return lqb::cuda_status(e, "noalloc search: cudaGetSymbolAddress");
        g_addr[dev] = p;
    } else if (!g_addr[dev]) {
        return lqb::set_error(LQ_ERR_ARG,
                              "lq_grid_neighbor_search_noalloc: first call on device %d made during stream capture; "
                              "make one call before capture begins",
                              dev);
    }
    *out = g_addr[dev];
    return LQ_OK;
}

}  // namespace

extern "C" int lq_grid_neighbor_search_noalloc(const void* par_host, const void* par_device, const float* pospres,
                                               int* part_cel, int* part_idx, int* cell_beg, int* cell_end,
                                               void* stream)
{
    if (!par_host || !par_device)
        return lqb::set_error(LQ_ERR_ARG, "lq_grid_neighbor_search_noalloc: null Parameters");
    const Parameters* ph = static_cast<const Parameters*>(par_host);
    const int np = ph->np, ncell = ph->ncell;
    if (np < 0 || ncell < 1) return lqb::set_error(LQ_ERR_ARG, "lq_grid_neighbor_search_noalloc: bad sizes");
    if (np > kMaxParticles || ncell > kMaxCells)
        return lqb::set_error(LQ_ERR_ARG,
                              "lq_grid_neighbor_search_noalloc: np=%d ncell=%d exceed the fixed scratch limits "
                              "(np <= %d, ncell <= %d); use lq_grid_create + lq_grid_neighbor_search",
                              np, ncell, kMaxParticles, kMaxCells);
    if ((np > 0 && (!pospres || !part_cel || !part_idx)) || !cell_beg || !cell_end)
        return lqb::set_error(LQ_ERR_ARG, "lq_grid_neighbor_search_noalloc: null array");
    size_t scan = 0;
    LQ_TRY(lqb::scan_scratch_bytes(ncell, &scan));
    if (scan > kScanBytes)
        return lqb::set_error(LQ_ERR_ARG, "lq_grid_neighbor_search_noalloc: scan needs %zu bytes of scratch, %zu fixed",
                              scan, kScanBytes);
    void* base = nullptr;
    LQ_TRY(scratch_address(static_cast<cudaStream_t>(stream), &base));
    char* b = static_cast<char*>(base);
    lqb::GridBuffers g;
    g.np_cap = np;
    g.ncell_cap = ncell;
    g.key = reinterpret_cast<int*>(b);
    g.rank = reinterpret_cast<int*>(b + kTable);
    g.count = reinterpret_cast<int*>(b + 2 * kTable);   /* cleared inside grid_search */
    g.start = reinterpret_cast<int*>(b + 3 * kTable);
    g.scan_tmp = b + 4 * kTable;
    g.scan_bytes = kScanBytes;
    g.part_idx = part_idx;
    g.part_cel = part_cel;
    g.beg = cell_beg;
    g.end = cell_end;
    return lqb::grid_search(ph, static_cast<const Parameters*>(par_device), reinterpret_cast<const float4*>(pospres),
                            g, true, nullptr, static_cast<cudaStream_t>(stream));
}
