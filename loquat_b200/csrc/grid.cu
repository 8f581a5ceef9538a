/*
 * LOQUAT-B200 neighbour grid (replaces the closed LoquatGrid of the
 * reference, src/loquat_grid.h:28-66).
 *
 * A stable counting sort by cell key instead of a full radix sort: the key
 * range is the cell count, so one histogram + one scan place every particle.
 *   1. k_hash_count  key per particle, warp-aggregated atomic count per cell,
 *                    the atomic's return value is the particle's rank
 *   2. scan          exclusive sum of the counts -> cell start table
 *   3. k_scatter     slot = start[key] + rank
 *   4. k_cell_order  ranks from atomics are not ordered across warps, so each
 *                    cell's slot range is put back in ascending previous-slot
 *                    order (insertion sort; input order is nearly sorted
 *                    because particles move little between searches).  The
 *                    result equals a stable sort by key, bit for bit.
 *   5. k_bounds      per-cell begin/end (-1 when empty), only for callers of
 *                    the reference interface; the native driver reads the
 *                    start table directly.
 * HBM traffic per particle: 16 B position read, 8 B key+rank written and read
 * back, 8 B sorted outputs; plus 12 B per cell for count, start and bounds.
 */
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <unordered_map>
#include <utility>

#include <cub/device/device_scan.cuh>

#include "lq_internal.cuh"
#include "lq_device.cuh"
#include <loquat_grid.h>

namespace lqb {

namespace {

constexpr int kBlock = 256;

inline int blocks_for(long long n, int b = kBlock) { return (int)((n + b - 1) / b); }

__global__ void __launch_bounds__(kBlock) k_hash_count(const Parameters* __restrict__ P, int np, int npb,
                                                       const float4* __restrict__ pos, int* __restrict__ key,
                                                       int* __restrict__ rank, int* __restrict__ count,
                                                       int* __restrict__ health, const float4* __restrict__ idep,
                                                       Frames fr)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < np;
    int k = 0;
    if (active) {
        const float ih = __ldg(&P->i_h);
        const int nx = __ldg(&P->cell_num_x), ny = __ldg(&P->cell_num_y), nz = __ldg(&P->cell_num_z);
        const float4 p = __ldg(pos + i);
        int cy = cell_axis(p.y, ih, ny);
        if (fr.rows) {
            /* local cell, then the object's row block */
            const float s = floorf(0.5f * p.y * ih);
            const int local = (s >= 0.0f && s < 1.0e9f) ? (int)s : -1;
            cy = local < 0 ? -1 : frame_row(fr, __ldg(&idep[i].x), local);
        }
        const int cx = cell_axis(p.x, ih, nx), cz = cell_axis(p.z, ih, nz);
        if (cx < 0 || cy < 0 || cz < 0) {
            k = __ldg(&P->ncell_delete);
            if (health) atomicAdd(health + (i < npb ? HEALTH_BND_OUT : HEALTH_MAT_OUT), 1);
        } else {
            k = (i < npb ? 0 : __ldg(&P->ncell_one_layer)) + (cx * ny + cy) * nz + cz;
        }
    }
    const unsigned act = __ballot_sync(0xffffffffu, active);
    if (!active) return;
    const unsigned peers = __match_any_sync(act, k);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(count + k, __popc(peers));
    base = __shfl_sync(peers, base, leader);
    key[i] = k;
    rank[i] = base + __popc(peers & ((1u << lane) - 1u));
}

__global__ void __launch_bounds__(kBlock) k_fill_int(int* __restrict__ p, int n, int v)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

__global__ void k_add_int(int* __restrict__ p, int v) { *p += v; }

__global__ void __launch_bounds__(kBlock) k_scatter(int np, const int* __restrict__ key, const int* __restrict__ rank,
                                                    const int* __restrict__ start, int* __restrict__ part_idx,
                                                    int* __restrict__ part_cel)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const int k = key[i];
    const int d = __ldg(start + k) + rank[i];
    if (!lq_in_range(d, np)) return;
    part_idx[d] = i;
    part_cel[d] = k;
}

__global__ void __launch_bounds__(kBlock) k_cell_order(int ncell, const int* __restrict__ start,
                                                       int* __restrict__ part_idx)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    const int s = __ldg(start + c), e = __ldg(start + c + 1);
    /* most cells arrive in order (their particles came from one warp):
     * a read-only pass finds them and leaves them untouched */
    bool sorted = true;
    for (int a = s + 1; a < e && sorted; ++a) sorted = part_idx[a - 1] < part_idx[a];
    if (sorted) return;
    for (int a = s + 1; a < e; ++a) {
        const int v = part_idx[a];
        int b = a - 1;
        while (b >= s && part_idx[b] > v) {
            part_idx[b + 1] = part_idx[b];
            --b;
        }
        part_idx[b + 1] = v;
    }
}

__global__ void __launch_bounds__(kBlock) k_bounds(int ncell, const int* __restrict__ start, int* __restrict__ beg,
                                                   int* __restrict__ end)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    const int s = __ldg(start + c), e = __ldg(start + c + 1);
    beg[c] = e > s ? s : -1;
    end[c] = e > s ? e : -1;
}

__global__ void __launch_bounds__(kBlock) k_gather_f4(int n, const int* __restrict__ idx, const float4* __restrict__ in,
                                                      float4* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int j = __ldg(idx + i);
    if (lq_in_range(j, n)) out[i] = __ldg(in + j);
}

/* tensor2d as three float2 words: consecutive threads write consecutive words. */
__global__ void __launch_bounds__(kBlock) k_gather_t2(int n, const int* __restrict__ idx, const float2* __restrict__ in,
                                                      float2* __restrict__ out)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3LL * n) return;
    const int i = (int)(t / 3);
    const int w = (int)(t - 3LL * i);
    const int j = __ldg(idx + i);
    if (lq_in_range(j, n)) out[t] = __ldg(in + 3LL * j + w);
}

__global__ void __launch_bounds__(kBlock) k_gather_state(int n, const int* __restrict__ idx, State in, State out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int j = __ldg(idx + i);
    if (!lq_in_range(j, n)) return;
    out.pos[i] = __ldg(in.pos + j);
    out.vel[i] = __ldg(in.vel + j);
    out.idep[i] = __ldg(in.idep + j);
    store_t2(out.str, i, load_t2(in.str, j));
    store_t2(out.stn, i, load_t2(in.stn, j));
    if (in.xlo) {
        out.xlo[i] = in.xlo[j];
        out.vlo[i] = in.vlo[j];
    }
}

}  // namespace

int fill_int(int* p, int n, int v, cudaStream_t s)
{
    if (n <= 0) return LQ_OK;
    k_fill_int<<<blocks_for(n), kBlock, 0, s>>>(p, n, v);
    LQ_TRY_CUDA(cudaGetLastError(), "k_fill_int");
    return LQ_OK;
}

int add_int(int* p, int v, cudaStream_t s)
{
    k_add_int<<<1, 1, 0, s>>>(p, v);
    LQ_TRY_CUDA(cudaGetLastError(), "k_add_int");
    return LQ_OK;
}

int scan_scratch_bytes(int ncell, size_t* bytes)
{
    *bytes = 0;
    LQ_TRY_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, *bytes, (const int*)nullptr, (int*)nullptr, ncell + 1),
                "scan scratch query");
    return LQ_OK;
}

int grid_search(const Parameters* ph, const Parameters* pd, const float4* pos, GridBuffers& g, bool bounds,
                int* health, cudaStream_t s, const float4* idep, const Frames& fr)
{
    const int np = ph->np, npb = ph->npb, ncell = ph->ncell;
    if (np < 0 || npb < 0 || npb > np || ncell < 1)
        return set_error(LQ_ERR_ARG, "grid_search: bad sizes np=%d npb=%d ncell=%d", np, npb, ncell);
    if (np > g.np_cap || ncell > g.ncell_cap)
        return set_error(LQ_ERR_ARG, "grid_search: np=%d ncell=%d exceed grid capacity np=%d ncell=%d", np, ncell,
                         g.np_cap, g.ncell_cap);
    if (ph->ncell != 2 * ph->ncell_one_layer + 1 || ph->ncell_delete != ncell - 1)
        return set_error(LQ_ERR_ARG, "grid_search: Parameters cell counts are not initialised");
    LQ_TRY(fill_int(g.count, ncell + 1, 0, s));
    if (np > 0) {
        if (fr.rows && !idep) return set_error(LQ_ERR_ARG, "grid_search: frames need the idep array");
        k_hash_count<<<blocks_for(np), kBlock, 0, s>>>(pd, np, npb, pos, g.key, g.rank, g.count, health, idep, fr);
        LQ_TRY_CUDA(cudaGetLastError(), "k_hash_count");
    }
    size_t bytes = g.scan_bytes;
    LQ_TRY_CUDA(cub::DeviceScan::ExclusiveSum(g.scan_tmp, bytes, g.count, g.start, ncell + 1, s), "cell scan");
    if (np > 0) {
        k_scatter<<<blocks_for(np), kBlock, 0, s>>>(np, g.key, g.rank, g.start, g.part_idx, g.part_cel);
        LQ_TRY_CUDA(cudaGetLastError(), "k_scatter");
        k_cell_order<<<blocks_for(ncell), kBlock, 0, s>>>(ncell, g.start, g.part_idx);
        LQ_TRY_CUDA(cudaGetLastError(), "k_cell_order");
    }
    if (bounds) {
        k_bounds<<<blocks_for(ncell), kBlock, 0, s>>>(ncell, g.start, g.beg, g.end);
        LQ_TRY_CUDA(cudaGetLastError(), "k_bounds");
    }
    return LQ_OK;
}

int gather_float4(int n, const int* idx, const float4* in, float4* out, cudaStream_t s)
{
    if (n <= 0) return LQ_OK;
    k_gather_f4<<<blocks_for(n), kBlock, 0, s>>>(n, idx, in, out);
    LQ_TRY_CUDA(cudaGetLastError(), "k_gather_f4");
    return LQ_OK;
}

int gather_tensor2d(int n, const int* idx, const tensor2d* in, tensor2d* out, cudaStream_t s)
{
    if (n <= 0) return LQ_OK;
    k_gather_t2<<<blocks_for(3LL * n), kBlock, 0, s>>>(n, idx, reinterpret_cast<const float2*>(in),
                                                        reinterpret_cast<float2*>(out));
    LQ_TRY_CUDA(cudaGetLastError(), "k_gather_t2");
    return LQ_OK;
}

/* This translation unit's count of bounds violations (always 0 without
 * LQ_CHECKED). */
int bounds_count_grid(unsigned long long* v)
{
#ifdef LQ_CHECKED
    LQ_TRY_CUDA(cudaMemcpyFromSymbol(v, lq_bounds_count, sizeof(*v)), "bounds counter");
#else
    *v = 0;
#endif
    return LQ_OK;
}

/* --------------------------------------------- identities of the grids */
namespace {

struct IdentityRecord {
    int* ident = nullptr;
    int* tmp = nullptr;
    int np = 0;
    long long gen = 0;
};
std::mutex g_id_mu;
std::unordered_map<const int*, IdentityRecord> g_ids;
long long g_id_gen = 0;

__global__ void __launch_bounds__(kBlock) k_iota(int n, int* __restrict__ p)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = i;
}

__global__ void __launch_bounds__(kBlock) k_follow(int n, const int* __restrict__ part_idx,
                                                   const int* __restrict__ in, int* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int j = __ldg(part_idx + i);
    out[i] = lq_in_range(j, n) ? __ldg(in + j) : -1;
}

}  // namespace

int identity_reset(const int* key, int np)
{
    std::lock_guard<std::mutex> lock(g_id_mu);
    IdentityRecord& r = g_ids[key];
    if (r.np != np || !r.ident) {
        cudaFree(r.ident);
        cudaFree(r.tmp);
        r = IdentityRecord{};
        const size_t b = sizeof(int) * (size_t)(np > 0 ? np : 1);
        cudaError_t e = cudaMalloc((void**)&r.ident, b);
        if (e == cudaSuccess) e = cudaMalloc((void**)&r.tmp, b);
        if (e != cudaSuccess) {
            cudaFree(r.ident);
            cudaFree(r.tmp);
            g_ids.erase(key);
            return set_error(LQ_ERR_ALLOC, "grid identities: %s", cudaGetErrorString(e));
        }
        r.np = np;
    }
    r.gen = ++g_id_gen;
    if (np > 0) {
        k_iota<<<blocks_for(np), kBlock>>>(np, r.ident);
        LQ_TRY_CUDA(cudaGetLastError(), "k_iota");
    }
    return LQ_OK;
}

int identity_after_search(const int* key, const int* part_idx, int np, cudaStream_t s)
{
    std::lock_guard<std::mutex> lock(g_id_mu);
    auto it = g_ids.find(key);
    if (it == g_ids.end()) return LQ_OK;
    IdentityRecord& r = it->second;
    if (np != r.np) {
        /* a search over another particle count: identities restart */
        r.gen = ++g_id_gen;
        if (np > r.np || np <= 0) return LQ_OK;
    }
    if (np <= 0) return LQ_OK;
    k_follow<<<blocks_for(np), kBlock, 0, s>>>(np, part_idx, r.ident, r.tmp);
    LQ_TRY_CUDA(cudaGetLastError(), "k_follow");
    std::swap(r.ident, r.tmp);
    return LQ_OK;
}

void identity_release(const int* key)
{
    std::lock_guard<std::mutex> lock(g_id_mu);
    auto it = g_ids.find(key);
    if (it == g_ids.end()) return;
    cudaFree(it->second.ident);
    cudaFree(it->second.tmp);
    g_ids.erase(it);
}

bool identity_find(const int* key, GridIdentity* out)
{
    std::lock_guard<std::mutex> lock(g_id_mu);
    auto it = g_ids.find(key);
    if (it == g_ids.end() || !it->second.ident) return false;
    out->ident = it->second.ident;
    out->np = it->second.np;
    out->gen = it->second.gen;
    return true;
}

int gather_state(int n, const int* idx, const State& in, const State& out, cudaStream_t s)
{
    if (n <= 0) return LQ_OK;
    k_gather_state<<<blocks_for(n), kBlock, 0, s>>>(n, idx, in, out);
    LQ_TRY_CUDA(cudaGetLastError(), "k_gather_state");
    return LQ_OK;
}

}  // namespace lqb

/* ------------------------------------------------------------------ C ABI */

namespace {

struct LqGrid {
    lqb::GridBuffers g;
};

void free_grid_buffers(lqb::GridBuffers& g)
{
    if (g.beg) lqb::identity_release(g.beg);
    cudaFree(g.key);
    cudaFree(g.rank);
    cudaFree(g.count);
    cudaFree(g.start);
    cudaFree(g.part_idx);
    cudaFree(g.part_cel);
    cudaFree(g.beg);
    cudaFree(g.end);
    cudaFree(g.scan_tmp);
    g = lqb::GridBuffers();
}

int alloc_grid_buffers(lqb::GridBuffers& g, int np, int ncell)
{
    if (np < 0 || ncell < 1) return lqb::set_error(LQ_ERR_ARG, "grid: bad sizes np=%d ncell=%d", np, ncell);
    free_grid_buffers(g);
    size_t npb = sizeof(int) * (size_t)(np > 0 ? np : 1);
    size_t ncb = sizeof(int) * (size_t)(ncell + 1);
    LQ_TRY(lqb::scan_scratch_bytes(ncell, &g.scan_bytes));
    cudaError_t e = cudaSuccess;
    e = e ? e : cudaMalloc(&g.key, npb);
    e = e ? e : cudaMalloc(&g.rank, npb);
    e = e ? e : cudaMalloc(&g.part_idx, npb);
    e = e ? e : cudaMalloc(&g.part_cel, npb);
    e = e ? e : cudaMalloc(&g.count, ncb);
    e = e ? e : cudaMalloc(&g.start, ncb);
    e = e ? e : cudaMalloc(&g.beg, ncb);
    e = e ? e : cudaMalloc(&g.end, ncb);
    e = e ? e : cudaMalloc(&g.scan_tmp, g.scan_bytes > 0 ? g.scan_bytes : 16);
    if (e != cudaSuccess) {
        free_grid_buffers(g);
        return lqb::set_error(LQ_ERR_ALLOC, "grid: device allocation failed: %s", cudaGetErrorString(e));
    }
    g.np_cap = np;
    g.ncell_cap = ncell;
    return lqb::identity_reset(g.beg, np);
}

}  // namespace

extern "C" int lq_grid_create(int np, int ncell, void** grid)
{
    if (!grid) return lqb::set_error(LQ_ERR_ARG, "lq_grid_create: null output");
    *grid = nullptr;
    LqGrid* G = new LqGrid();
    int st = alloc_grid_buffers(G->g, np, ncell);
    if (st != LQ_OK) {
        delete G;
        return st;
    }
    *grid = G;
    return LQ_OK;
}

extern "C" int lq_grid_resize(void* grid, int np, int ncell)
{
    if (!grid) return lqb::set_error(LQ_ERR_ARG, "lq_grid_resize: null grid");
    return alloc_grid_buffers(static_cast<LqGrid*>(grid)->g, np, ncell);
}

extern "C" int lq_grid_destroy(void* grid)
{
    if (!grid) return LQ_OK;
    LqGrid* G = static_cast<LqGrid*>(grid);
    free_grid_buffers(G->g);
    delete G;
    return LQ_OK;
}

extern "C" int lq_grid_neighbor_search(void* grid, const void* par_host, const void* par_device,
                                       const float* pospres, const float* idep, void* stream)
{
    (void)idep;
    if (!grid || !par_host || !par_device || (!pospres && static_cast<const Parameters*>(par_host)->np > 0))
        return lqb::set_error(LQ_ERR_ARG, "lq_grid_neighbor_search: null argument");
    LqGrid* G = static_cast<LqGrid*>(grid);
    const Parameters* ph = static_cast<const Parameters*>(par_host);
    LQ_TRY(lqb::grid_search(ph, static_cast<const Parameters*>(par_device), reinterpret_cast<const float4*>(pospres),
                            G->g, true, nullptr, static_cast<cudaStream_t>(stream)));
    return lqb::identity_after_search(G->g.beg, G->g.part_idx, ph->np, static_cast<cudaStream_t>(stream));
}

extern "C" int lq_grid_arrays(void* grid, const int** part_cel, const int** part_idx, const int** cell_beg,
                              const int** cell_end, const int** cell_start)
{
    if (!grid) return lqb::set_error(LQ_ERR_ARG, "lq_grid_arrays: null grid");
    LqGrid* G = static_cast<LqGrid*>(grid);
    if (part_cel) *part_cel = G->g.part_cel;
    if (part_idx) *part_idx = G->g.part_idx;
    if (cell_beg) *cell_beg = G->g.beg;
    if (cell_end) *cell_end = G->g.end;
    if (cell_start) *cell_start = G->g.start;
    return LQ_OK;
}

extern "C" int lq_grid_sort_float4(void* grid, int np, float* data, float* cache, void* stream)
{
    if (!grid || (np > 0 && (!data || !cache))) return lqb::set_error(LQ_ERR_ARG, "lq_grid_sort_float4: null argument");
    LqGrid* G = static_cast<LqGrid*>(grid);
    if (np > G->g.np_cap) return lqb::set_error(LQ_ERR_ARG, "lq_grid_sort_float4: np exceeds grid capacity");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    LQ_TRY(lqb::gather_float4(np, G->g.part_idx, reinterpret_cast<const float4*>(data),
                              reinterpret_cast<float4*>(cache), s));
    LQ_TRY_CUDA(cudaMemcpyAsync(data, cache, sizeof(float4) * (size_t)np, cudaMemcpyDeviceToDevice, s), "copy back");
    return LQ_OK;
}

extern "C" int lq_grid_sort_tensor2d(void* grid, int np, float* data, float* cache, void* stream)
{
    if (!grid || (np > 0 && (!data || !cache)))
        return lqb::set_error(LQ_ERR_ARG, "lq_grid_sort_tensor2d: null argument");
    LqGrid* G = static_cast<LqGrid*>(grid);
    if (np > G->g.np_cap) return lqb::set_error(LQ_ERR_ARG, "lq_grid_sort_tensor2d: np exceeds grid capacity");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    LQ_TRY(lqb::gather_tensor2d(np, G->g.part_idx, reinterpret_cast<const tensor2d*>(data),
                                reinterpret_cast<tensor2d*>(cache), s));
    LQ_TRY_CUDA(cudaMemcpyAsync(data, cache, sizeof(tensor2d) * (size_t)np, cudaMemcpyDeviceToDevice, s),
                "copy back");
    return LQ_OK;
}

/* ------------------------------------------------- C++ drop-in LoquatGrid */
/* The eight private members keep the reference layout (src/loquat_grid.h:32-41).
 * buffer holds [count | start | scan scratch], each 256-byte aligned. */

namespace {

[[noreturn]] void die(const char* what)
{
    fprintf(stderr, "LoquatGrid::%s failed: %s\n", what, lq_last_error());
    exit(EXIT_FAILURE);
}

inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

LoquatGrid::LoquatGrid()
    : part_cel(nullptr), part_idx(nullptr), cell_beg(nullptr), cell_end(nullptr), part_cel_cache(nullptr),
      part_idx_cache(nullptr), buffer(nullptr), buffer_storage_bytes(0)
{
}

LoquatGrid::~LoquatGrid()
{
    if (cell_beg) lqb::identity_release(cell_beg);
    cudaFree(part_cel);
    cudaFree(part_idx);
    cudaFree(cell_beg);
    cudaFree(cell_end);
    cudaFree(part_cel_cache);
    cudaFree(part_idx_cache);
    cudaFree(buffer);
}

void LoquatGrid::GridConfig(Parameters* par_host)
{
    ResizeArrayLength(par_host->np, par_host->ncell);
    /* ParticleInteraction's working arrays too, at set-up as the reference
     * allocates its own, so the step loop allocates nothing */
    if (lq_interaction_reserve(par_host) != LQ_OK) die("GridConfig");
}

void LoquatGrid::ResizeArrayLength(int np_new, int ncell_new)
{
    if (np_new < 0 || ncell_new < 1) {
        lqb::set_error(LQ_ERR_ARG, "bad sizes np=%d ncell=%d", np_new, ncell_new);
        die("ResizeArrayLength");
    }
    if (cell_beg) lqb::identity_release(cell_beg);
    cudaFree(part_cel);
    cudaFree(part_idx);
    cudaFree(cell_beg);
    cudaFree(cell_end);
    cudaFree(part_cel_cache);
    cudaFree(part_idx_cache);
    cudaFree(buffer);
    size_t scan = 0;
    if (lqb::scan_scratch_bytes(ncell_new, &scan) != LQ_OK) die("ResizeArrayLength");
    const size_t npb = sizeof(int) * (size_t)(np_new > 0 ? np_new : 1);
    const size_t ncb = sizeof(int) * (size_t)ncell_new;
    const size_t tab = align256(sizeof(int) * (size_t)(ncell_new + 1));
    buffer_storage_bytes = 2 * tab + align256(scan > 0 ? scan : 16);
    cudaError_t e = cudaSuccess;
    e = e ? e : cudaMalloc(&part_cel, npb);
    e = e ? e : cudaMalloc(&part_idx, npb);
    e = e ? e : cudaMalloc(&cell_beg, ncb);
    e = e ? e : cudaMalloc(&cell_end, ncb);
    e = e ? e : cudaMalloc(&part_cel_cache, npb);
    e = e ? e : cudaMalloc(&part_idx_cache, npb);
    e = e ? e : cudaMalloc(&buffer, buffer_storage_bytes);
    if (e != cudaSuccess) {
        lqb::set_error(LQ_ERR_ALLOC, "%s", cudaGetErrorString(e));
        die("ResizeArrayLength");
    }
    /* particle identities through the searches (ParticleInteraction keeps
     * its neighbour lists across searches with them) */
    if (lqb::identity_reset(cell_beg, np_new) != LQ_OK) die("ResizeArrayLength");
}

void LoquatGrid::SortParticleByCellIndex(Parameters* par_host)
{
    (void)par_host; /* the sort runs inside NeighborSearch */
}

void LoquatGrid::NeighborSearch(Parameters* par_host, Parameters* par_device, float4* pospres, float4* idep)
{
    (void)idep;
    const int ncell = par_host->ncell;
    const size_t tab = align256(sizeof(int) * (size_t)(ncell + 1));
    lqb::GridBuffers g;
    g.np_cap = par_host->np;
    g.ncell_cap = ncell;
    g.key = part_cel_cache;
    g.rank = part_idx_cache;
    g.count = static_cast<int*>(buffer);
    g.start = reinterpret_cast<int*>(static_cast<char*>(buffer) + tab);
    g.scan_tmp = static_cast<char*>(buffer) + 2 * tab;
    g.scan_bytes = buffer_storage_bytes - 2 * tab;
    g.part_idx = part_idx;
    g.part_cel = part_cel;
    g.beg = cell_beg;
    g.end = cell_end;
    if (lqb::grid_search(par_host, par_device, pospres, g, true, nullptr, 0) != LQ_OK) die("NeighborSearch");
    if (lqb::identity_after_search(cell_beg, part_idx, par_host->np, 0) != LQ_OK) die("NeighborSearch");
}

void LoquatGrid::SortArrayFloat4(int np, float4* data, float4* data_cache)
{
    if (lqb::gather_float4(np, part_idx, data, data_cache, 0) != LQ_OK) die("SortArrayFloat4");
    cudaError_t e = cudaMemcpyAsync(data, data_cache, sizeof(float4) * (size_t)np, cudaMemcpyDeviceToDevice, 0);
    if (e != cudaSuccess) {
        lqb::cuda_status(e, "copy back");
        die("SortArrayFloat4");
    }
}

void LoquatGrid::SortArrayTensor2d(int np, tensor2d* data, tensor2d* data_cache)
{
    if (lqb::gather_tensor2d(np, part_idx, data, data_cache, 0) != LQ_OK) die("SortArrayTensor2d");
    cudaError_t e = cudaMemcpyAsync(data, data_cache, sizeof(tensor2d) * (size_t)np, cudaMemcpyDeviceToDevice, 0);
    if (e != cudaSuccess) {
        lqb::cuda_status(e, "copy back");
        die("SortArrayTensor2d");
    }
}
