/*
 * LOQUAT-B200 native time-step driver: the hot loop of
 * LoquatSph::RunSimulation (reference src/loquat.cu:322-409), re-planned
 * for one B200.
 *
 * The reference searches and re-sorts the particles before every stage
 * (twice per step) and every phase visits the 27 neighbouring cells again.
 * Here the particle order and neighbour lists are kept across steps,
 * Verlet-style: the lists hold every pair within 2h + skin, and they are
 * rebuilt (search, stable sort, gather, list build) only when the particles
 * could have moved far enough for a pair to cross the 2h cut-off unseen.
 * Every evaluation therefore sees exactly the pairs within 2h, as a fresh
 * search would; only the float summation order differs.
 *
 *   per step (state in S, order fixed between rebuilds)
 *     [rebuild if flagged: search S, gather S -> T, copy T -> S, record the
 *      positions, build material and boundary lists]
 *     Adami(S), interaction(S), predictor S -> S2          (S is the snapshot)
 *     Adami(S2), interaction(S2), corrector (S2, S) -> S   (raises the flag)
 *     (Adami writes the boundary stress into S and S2; the integrators
 *     update the material slots only; S2 is a stage buffer: the predictor
 *     writes what the neighbour kernels and the corrector read from it,
 *     not its strain or low words)
 *   every N steps: Shepard(S) -> T.str, copy back            (reference :400-409)
 *
 * The rebuild decision stays on the device: a one-thread kernel turns the
 * flag into the condition of an IF node of the step's CUDA graph.  Without
 * graphs (or if the driver cannot build the conditional node) the host
 * reads the flag before each step, which gives the same sequence of
 * rebuilds.  dt = cfl h / cs is constant, as in the reference.
 *
 * Two-level lists (a wide cut-off 2h + wide above 2h + skin): the rebuild
 * after a sort builds wide lists, and the lists the stages read are renewed
 * from them (filtered at the current positions, no search) whenever the
 * skin runs out; a sort happens only once a particle has moved
 * (wide - skin) / 2 from its position at the wide build.  A second IF node
 * holds the renewal.
 */
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <utility>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "lq_internal.cuh"

namespace {

using lqb::State;

constexpr float kDefaultSkinOverH = 0.05f;

struct LqSim {
    Parameters ph{};
    Parameters* pd = nullptr;
    int np = 0, npb = 0, npm = 0;
    long long step = 0;
    double time = 0.0;
    int flags = 0;
    float skin = 0.0f;                 /* list cut-off = 2h + skin */
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;       /* captures the rebuild body */
    State S{}, S2{}, T{};
    float4* xbuild = nullptr;          /* positions when the lists were built */
    float wide = 0.0f;                 /* two-level lists: wide cut-off 2h + wide (0: one level) */
    float4* xwide = nullptr;           /* positions when the wide lists were built */
    lqb::NeighborList wlm, wlb;        /* shell parts of the wide lists, material and boundary targets */
    int* inner_m = nullptr;            /* inner parts' counts (their entries open the stages' lists) */
    int* inner_b = nullptr;
    int* renewals = nullptr;           /* device counter of lists renewed from the wide ones */
    lqb::Rates R{};
    lqb::GridBuffers g;
    lqb::NeighborList nlm, nlb;        /* material targets, boundary targets */
    int* bact = nullptr;               /* boundary slots whose lists can hold entries, ascending */
    int* nbact = nullptr;              /* device count of bact */
    void* bsel_tmp = nullptr;          /* scratch of their selection */
    size_t bsel_bytes = 0;
    int* health = nullptr;
    int* rebuild = nullptr;            /* device flag: rebuild before the next step */
    int* rebuilds = nullptr;           /* device counter of rebuilds */
    int* host_flag = nullptr;          /* pinned mirror for the eager path */
    lqb::MaterialTable mt;             /* per-object materials (optional) */
    lqb::MaterialTable vw;             /* von Wolffersdorff rows (model 3) */
    float* rec = nullptr;              /* packed neighbour data, np x 13 floats */
    float* rho_f = nullptr;            /* density filter output (LQ_SIM_DENSITY_FILTER) */
    int pair_shape = 0;                /* launch shape of the pair kernel (lqb::kPairShapes) */
    lqb::TileOrder tile;               /* targets in tile order (tiled shapes; allocated on first use) */
    unsigned* vmax2 = nullptr;         /* max |v|^2, |a|^2 bits (LQ_SIM_DYNAMIC_DT) */
    double* dtime = nullptr;           /* device-side time (LQ_SIM_DYNAMIC_DT) */
    lqb::Frames fr;                    /* per-object grid rows (optional) */
    std::vector<float> mt_host, vw_host; /* host copies of the tables, for checkpoints */
    std::vector<int> fr_host;
    std::vector<void*> allocs;
    cudaGraphExec_t step_exec = nullptr;
    cudaGraphExec_t shep_exec = nullptr;
    bool conditional = false;
};

int dev_alloc(LqSim* S, void** p, size_t bytes)
{
    cudaError_t e = cudaMalloc(p, bytes > 0 ? bytes : 16);
    if (e != cudaSuccess)
        return lqb::set_error(LQ_ERR_ALLOC, "sim: cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    S->allocs.push_back(*p);
    return LQ_OK;
}

bool tiled(const LqSim* S) { return lqb::kPairShapes[S->pair_shape][2] != 0; }

/* Bits of the device flag: the lists must be renewed before the next step;
 * the wide lists no longer cover a renewal (a sort is due). */
constexpr int kFlagLists = 1, kFlagSort = 2, kFlagAll = 3;

bool two_level(const LqSim* S) { return S->wide > S->skin && S->wlm.list != nullptr; }

/* Wide lists and their build positions, on first use of two-level lists. */
int ensure_wide_lists(LqSim* S)
{
    if (S->wlm.list) return LQ_OK;
    LQ_TRY(dev_alloc(S, (void**)&S->xwide, (size_t)S->np * sizeof(float4)));
    S->wlm.stride = S->nlm.stride;
    LQ_TRY(dev_alloc(S, (void**)&S->wlm.list, sizeof(int) * (size_t)LQ_NBR_CAP * S->wlm.stride));
    LQ_TRY(dev_alloc(S, (void**)&S->wlm.count, sizeof(int) * (size_t)S->wlm.stride));
    S->wlb.stride = S->nlb.stride;
    LQ_TRY(dev_alloc(S, (void**)&S->wlb.list, sizeof(int) * (size_t)LQ_NBR_CAP * S->wlb.stride));
    LQ_TRY(dev_alloc(S, (void**)&S->wlb.count, sizeof(int) * (size_t)S->wlb.stride));
    LQ_TRY(dev_alloc(S, (void**)&S->inner_m, sizeof(int) * (size_t)S->wlm.stride));
    LQ_TRY(dev_alloc(S, (void**)&S->inner_b, sizeof(int) * (size_t)S->wlb.stride));
    return LQ_OK;
}

/* The pair kernel's target order for tiled launch shapes (null otherwise). */
const int* tile_order(const LqSim* S) { return tiled(S) ? S->tile.order : nullptr; }

/* Buffers of the tile order, on first use of a tiled shape. */
int ensure_tile_order(LqSim* S)
{
    if (!tiled(S) || S->tile.order) return LQ_OK;
    int nseg = 0;
    size_t bytes = 0;
    LQ_TRY(lqb::tile_order_scratch(&S->ph, &nseg, &bytes));
    LQ_TRY(dev_alloc(S, (void**)&S->tile.seg, sizeof(int) * 3 * (size_t)nseg));
    LQ_TRY(dev_alloc(S, &S->tile.scan_tmp, bytes));
    LQ_TRY(dev_alloc(S, (void**)&S->tile.order, sizeof(int) * (size_t)(S->npm > 0 ? S->npm : 1)));
    S->tile.nseg_cap = nseg;
    S->tile.scan_bytes = bytes;
    return LQ_OK;
}

int alloc_state(LqSim* S, State& st)
{
    const size_t n = (size_t)S->np;
    LQ_TRY(dev_alloc(S, (void**)&st.pos, n * sizeof(float4)));
    LQ_TRY(dev_alloc(S, (void**)&st.vel, n * sizeof(float4)));
    LQ_TRY(dev_alloc(S, (void**)&st.idep, n * sizeof(float4)));
    LQ_TRY(dev_alloc(S, (void**)&st.str, n * sizeof(tensor2d)));
    LQ_TRY(dev_alloc(S, (void**)&st.stn, n * sizeof(tensor2d)));
    if (S->flags & LQ_SIM_MIXED) {
        LQ_TRY(dev_alloc(S, (void**)&st.xlo, n * sizeof(float4)));
        LQ_TRY(dev_alloc(S, (void**)&st.vlo, n * sizeof(float4)));
    }
    return LQ_OK;
}

void release(LqSim* S)
{
    if (S->stream) cudaStreamSynchronize(S->stream);
    if (S->step_exec) cudaGraphExecDestroy(S->step_exec);
    if (S->shep_exec) cudaGraphExecDestroy(S->shep_exec);
    S->step_exec = S->shep_exec = nullptr;
    for (void* p : S->allocs) cudaFree(p);
    S->allocs.clear();
    if (S->host_flag) cudaFreeHost(S->host_flag);
    S->host_flag = nullptr;
    if (S->side) cudaStreamDestroy(S->side);
    if (S->stream) cudaStreamDestroy(S->stream);
    S->side = S->stream = nullptr;
}

/* ------------------------------------------------------------- kernels */

/* The gathered state back into S and the build positions; boundary slots
 * also into S2.  From then on only Adami changes a boundary slot, writing
 * its stress into both buffers, so the integrators leave boundary slots
 * alone. */
__global__ void k_copy_state(int n, int npb, State in, State out, State out2, float4* __restrict__ xbuild)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (i < npb) {
        out2.pos[i] = in.pos[i];
        out2.vel[i] = in.vel[i];
        out2.idep[i] = in.idep[i];
        const float2* a = reinterpret_cast<const float2*>(in.str) + 3 * (size_t)i;
        float2* b = reinterpret_cast<float2*>(out2.str) + 3 * (size_t)i;
        b[0] = a[0];
        b[1] = a[1];
        b[2] = a[2];
        a = reinterpret_cast<const float2*>(in.stn) + 3 * (size_t)i;
        b = reinterpret_cast<float2*>(out2.stn) + 3 * (size_t)i;
        b[0] = a[0];
        b[1] = a[1];
        b[2] = a[2];
        if (in.xlo) {
            out2.xlo[i] = in.xlo[i];
            out2.vlo[i] = in.vlo[i];
        }
    }
    const float4 x = in.pos[i];
    out.pos[i] = x;
    xbuild[i] = x;
    out.vel[i] = in.vel[i];
    out.idep[i] = in.idep[i];
    const float2* a = reinterpret_cast<const float2*>(in.str) + 3 * (size_t)i;
    float2* b = reinterpret_cast<float2*>(out.str) + 3 * (size_t)i;
    b[0] = a[0];
    b[1] = a[1];
    b[2] = a[2];
    a = reinterpret_cast<const float2*>(in.stn) + 3 * (size_t)i;
    b = reinterpret_cast<float2*>(out.stn) + 3 * (size_t)i;
    b[0] = a[0];
    b[1] = a[1];
    b[2] = a[2];
    if (in.xlo) {
        out.xlo[i] = in.xlo[i];
        out.vlo[i] = in.vlo[i];
    }
}

/* Low words of an uploaded float state: zero (mixed form). */
__global__ void k_widen(int n, State st)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    st.xlo[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    st.vlo[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

__global__ void k_copy_t2(int first, int n, const tensor2d* __restrict__ in, tensor2d* __restrict__ out)
{
    const int i = first + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= first + n) return;
    const float2* a = reinterpret_cast<const float2*>(in) + 3 * (size_t)i;
    float2* b = reinterpret_cast<float2*>(out) + 3 * (size_t)i;
    b[0] = a[0];
    b[1] = a[1];
    b[2] = a[2];
}

/* Turns the rebuild flag into the IF condition and clears it. */
__global__ void k_decide(cudaGraphConditionalHandle h, int* flag, int* count)
{
    const int f = *flag;
    cudaGraphSetConditional(h, (f & kFlagLists) ? 1u : 0u);
    if (f & kFlagLists) *count += 1;
    *flag = 0;
}

/* Two-level lists: a sort and wide build when the lists are due and the
 * wide ones no longer cover a renewal; a renewal whenever the lists are
 * due (after a sort too, which leaves only wide lists). */
__global__ void k_decide2(cudaGraphConditionalHandle h_sort, cudaGraphConditionalHandle h_renew, int* flag,
                          int* sorts, int* renewals)
{
    const int f = *flag;
    const bool due = (f & kFlagLists) != 0;
    const bool sort = due && (f & kFlagSort) != 0;
    cudaGraphSetConditional(h_sort, sort ? 1u : 0u);
    cudaGraphSetConditional(h_renew, due ? 1u : 0u);
    if (sort) *sorts += 1;
    else if (due) *renewals += 1;
    *flag = 0;
}

/* The positions the current lists were renewed at. */
__global__ void k_record_positions(int n, const float4* __restrict__ pos, float4* __restrict__ xbuild)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) xbuild[i] = pos[i];
}

inline int blocks(int n) { return (n + 255) / 256; }

/* Density filter result into the state (its low word zero in the mixed form). */
__global__ void k_set_density(int npb, int npm, const float* __restrict__ rho, float4* __restrict__ vel,
                              float4* __restrict__ vlo)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npm) return;
    const int i = npb + t;
    const float r = rho[i];
    vel[i].w = r;
    if (vlo) vlo[i].w = 0.0f;
}

/* Largest |v|^2 and |a|^2 over the material particles: non-negative floats
 * order like their bit patterns, so an unsigned atomicMax reduces them. */
__global__ void k_dt_max(int npb, int npm, const float4* __restrict__ vel, const float4* __restrict__ accad,
                         unsigned* __restrict__ m2)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    float v2 = 0.0f, a2 = 0.0f;
    if (t < npm) {
        const float4 v = vel[npb + t], a = accad[npb + t];
        v2 = v.x * v.x + v.y * v.y + v.z * v.z;
        a2 = a.x * a.x + a.y * a.y + a.z * a.z;
        if (!(v2 >= 0.0f)) v2 = 0.0f;   /* non-finite values are the health word's business */
        if (!(a2 >= 0.0f)) a2 = 0.0f;
    }
    for (int o = 16; o > 0; o >>= 1) {
        v2 = fmaxf(v2, __shfl_xor_sync(0xffffffffu, v2, o));
        a2 = fmaxf(a2, __shfl_xor_sync(0xffffffffu, a2, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(m2, __float_as_uint(v2));
        atomicMax(m2 + 1, __float_as_uint(a2));
    }
}

/* time += the step just taken; dt of the next step from the maxima;
 * maxima cleared for the next reduction. */
__global__ void k_dt_update(Parameters* P, unsigned* m2, double* time)
{
    const float v = sqrtf(__uint_as_float(m2[0])), a = sqrtf(__uint_as_float(m2[1]));
    *time += (double)P->dt;
    float dt = P->h / (P->cs + v);
    if (a > 0.0f) dt = fminf(dt, sqrtf(P->h / a));
    P->dt = P->cfl * dt;
    m2[0] = 0u;
    m2[1] = 0u;
}

/* ------------------------------------------------------------ sequences */

/* Material and boundary lists from the sorted state in S: the lists the
 * stages read, or with two-level lists the wide ones, whose pairs closer
 * than 2h + 2 skin - wide (less a rounding margin of h / 1000) open the
 * stages' lists and the rest form the shell lists that renewals filter.
 * Then the boundary targets Adami visits: the slots with an entry, or with
 * two-level lists an inner or shell entry (a renewal fills a row only from
 * these, so the set holds until the next build). */
int build_lists(LqSim* S, cudaStream_t s)
{
    const Parameters* ph = &S->ph;
    const Parameters* pd = S->pd;
    const lqb::Cells cells{S->g.start, nullptr, nullptr};
    if (!two_level(S)) {
        const float cut = 2.0f * ph->h + S->skin;
        LQ_TRY(lqb::launch_neighbor_list_range(ph, pd, S->npb, S->npm, 0, cut, S->S.pos, cells, S->nlm, S->health,
                                               s, S->S.idep, S->fr));
        LQ_TRY(lqb::launch_neighbor_list_range(ph, pd, 0, S->npb, 1, cut, S->S.pos, cells, S->nlb, S->health, s,
                                               S->S.idep, S->fr));
        return lqb::launch_boundary_targets(S->npb, S->nlb.count, nullptr, S->bact, S->nbact, S->bsel_tmp,
                                            S->bsel_bytes, s);
    }
    const float cut = 2.0f * ph->h + S->wide;
    const float inner = 2.0f * ph->h + 2.0f * S->skin - S->wide - 1.0e-3f * ph->h;
    const lqb::NeighborList im{S->nlm.list, S->inner_m, S->nlm.stride};
    const lqb::NeighborList ib{S->nlb.list, S->inner_b, S->nlb.stride};
    LQ_TRY(lqb::launch_neighbor_list_range(ph, pd, S->npb, S->npm, 0, cut, S->S.pos, cells, im, S->health, s,
                                           S->S.idep, S->fr, &S->wlm, inner));
    LQ_TRY(lqb::launch_neighbor_list_range(ph, pd, 0, S->npb, 1, cut, S->S.pos, cells, ib, S->health, s, S->S.idep,
                                           S->fr, &S->wlb, inner));
    return lqb::launch_boundary_targets(S->npb, S->inner_b, S->wlb.count, S->bact, S->nbact, S->bsel_tmp,
                                        S->bsel_bytes, s);
}

/* Two-level lists: the lists the stages read renewed from the wide ones at
 * the current positions, and those positions recorded. */
int enqueue_renewal(LqSim* S, cudaStream_t s)
{
    const Parameters* ph = &S->ph;
    const float cut = 2.0f * ph->h + S->skin;
    LQ_TRY(lqb::launch_list_refresh(ph, S->npb, S->npm, cut, S->S.pos, S->inner_m, S->wlm, S->nlm, S->health, s));
    LQ_TRY(lqb::launch_list_refresh(ph, 0, S->npb, cut, S->S.pos, S->inner_b, S->wlb, S->nlb, S->health, s));
    k_record_positions<<<blocks(S->np), 256, 0, s>>>(S->np, S->S.pos, S->xbuild);
    LQ_TRY_CUDA(cudaGetLastError(), "k_record_positions");
    return LQ_OK;
}

/* The pair sums of a stage in the current launch shape. */
int enqueue_interaction(LqSim* S, const State& st, cudaStream_t s)
{
    const lqb::Cells cells{S->g.start, nullptr, nullptr};
    return lqb::launch_interaction_list(&S->ph, S->pd, st, S->R, cells, S->nlm, s, S->fr, S->flags & LQ_SIM_MIXED,
                                        S->rec, S->pair_shape, false, tile_order(S));
}

/* The material slots' packed neighbour data after a filter changed S. */
int enqueue_material_pack(LqSim* S, cudaStream_t s)
{
    return lqb::launch_pack_neighbors(&S->ph, S->S, S->rec, S->npb, s, S->flags & LQ_SIM_MIXED);
}

/* Search, sort and list build; leaves the state in S with fresh lists. */
int enqueue_rebuild(LqSim* S, cudaStream_t s)
{
    const Parameters* ph = &S->ph;
    const Parameters* pd = S->pd;
    LQ_TRY(lqb::grid_search(ph, pd, S->S.pos, S->g, false, S->health, s, S->S.idep, S->fr));
    LQ_TRY(lqb::gather_state(S->np, S->g.part_idx, S->S, S->T, s));
    k_copy_state<<<blocks(S->np), 256, 0, s>>>(S->np, S->npb, S->T, S->S, S->S2,
                                               two_level(S) ? S->xwide : S->xbuild);
    LQ_TRY_CUDA(cudaGetLastError(), "k_copy_state");
    LQ_TRY(build_lists(S, s));
    /* every slot's packed neighbour data (the boundary slots keep theirs
     * until the next build) */
    LQ_TRY(lqb::launch_pack_neighbors(ph, S->S, S->rec, 0, s, S->flags & LQ_SIM_MIXED));
    return lqb::launch_tile_order(ph, S->g.start, S->pair_shape, S->tile, s);
}

/* Dynamic time step (LQ_SIM_DYNAMIC_DT): the next step's dt into the
 * device Parameters, the time advanced on the device. */
int enqueue_dynamic_dt(LqSim* S, cudaStream_t s)
{
    if (!(S->flags & LQ_SIM_DYNAMIC_DT)) return LQ_OK;
    if (S->npm > 0) {
        k_dt_max<<<blocks(S->npm), 256, 0, s>>>(S->npb, S->npm, S->S.vel, S->R.accad, S->vmax2);
        LQ_TRY_CUDA(cudaGetLastError(), "k_dt_max");
    }
    k_dt_update<<<1, 1, 0, s>>>(S->pd, S->vmax2, S->dtime);
    LQ_TRY_CUDA(cudaGetLastError(), "k_dt_update");
    return LQ_OK;
}

/* Density Shepard filter (LQ_SIM_DENSITY_FILTER) on the lists. */
int enqueue_density_filter(LqSim* S, cudaStream_t s)
{
    const lqb::Cells cells{S->g.start, nullptr, nullptr};
    LQ_TRY(lqb::launch_density_filter_list(&S->ph, S->pd, S->S, S->rho_f, S->nlm, cells, s, S->fr, S->rec,
                                           tile_order(S)));
    if (S->npm > 0) {
        k_set_density<<<blocks(S->npm), 256, 0, s>>>(S->npb, S->npm, S->rho_f, S->S.vel, S->S.vlo);
        LQ_TRY_CUDA(cudaGetLastError(), "k_set_density");
    }
    return enqueue_material_pack(S, s);
}

/* Adami for a stage.  The material slots' packed neighbour data are
 * current (the integrator that wrote the stage's state packed them, or the
 * list build, or the filters' pack after them); Adami reads them and
 * writes the boundary slots' packed stress itself (boundary positions and
 * velocities are packed at each list build and do not change in between),
 * so the pair kernel needs no pack. */
int enqueue_adami_pack(LqSim* S, const State& st, cudaStream_t s)
{
    /* both state buffers take the boundary stress, so their boundary slots
     * stay equal and the integrators never touch them */
    tensor2d* other = st.str == S->S.str ? S->S2.str : S->S.str;
    return lqb::launch_adami_packed(&S->ph, S->pd, st, S->nlb, S->rec, s, other, S->bact, S->nbact);
}


/* The two stages of a step on the current lists. */
int enqueue_stages(LqSim* S, cudaStream_t s)
{
    const Parameters* ph = &S->ph;
    const Parameters* pd = S->pd;
    /* predictor stage (reference src/loquat.cu:343-368) */
    LQ_TRY(enqueue_adami_pack(S, S->S, s));
    LQ_TRY(enqueue_interaction(S, S->S, s));
    LQ_TRY(lqb::launch_predict(ph, pd, S->S, S->S2, nullptr, S->R, s, S->mt, S->vw, S->rec, true));
    /* corrector stage (reference src/loquat.cu:371-396) */
    LQ_TRY(enqueue_adami_pack(S, S->S2, s));
    LQ_TRY(enqueue_interaction(S, S->S2, s));
    LQ_TRY(lqb::launch_correct_into(ph, pd, S->S2, S->S, S->S, S->R, S->health, S->xbuild, S->rebuild, S->skin, s,
                                    S->mt, S->vw, two_level(S) ? S->xwide : nullptr, S->wide, S->rec));
    return enqueue_dynamic_dt(S, s);
}

/* Shepard stress filter (reference src/loquat.cu:400-409) on the lists. */
int enqueue_shepard(LqSim* S, cudaStream_t s)
{
    const lqb::Cells cells{S->g.start, nullptr, nullptr};
    LQ_TRY(lqb::launch_shepard_list(&S->ph, S->pd, S->S, S->T.str, S->nlm, cells, s, S->fr, S->rec, tile_order(S)));
    if (S->npm > 0) {
        k_copy_t2<<<blocks(S->npm), 256, 0, s>>>(S->npb, S->npm, S->T.str, S->S.str);
        LQ_TRY_CUDA(cudaGetLastError(), "k_copy_t2");
    }
    return enqueue_material_pack(S, s);
}

/* An IF node on handle h after the capture's current dependencies, its body
 * captured from `body` on the side stream; the capture continues after it. */
int capture_if(LqSim* S, cudaGraphConditionalHandle h, int (*body)(LqSim*, cudaStream_t))
{
    cudaStream_t s = S->stream;
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    LQ_TRY_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &ndeps), "capture info");
    /* the parameter record's C union has no usable C++ default
     * constructor: zero raw storage and view it as the record */
    alignas(cudaGraphNodeParams) unsigned char cp_raw[sizeof(cudaGraphNodeParams)];
    memset(cp_raw, 0, sizeof(cp_raw));
    cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cp_raw);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    LQ_TRY_CUDA(cudaGraphAddNode(&cnode, cg, deps, ndeps, &cp), "conditional node");
    cudaGraph_t graph_body = cp.conditional.phGraph_out[0];
    LQ_TRY_CUDA(cudaStreamBeginCaptureToGraph(S->side, graph_body, nullptr, nullptr, 0,
                                              cudaStreamCaptureModeThreadLocal),
                "body capture");
    const int st = body(S, S->side);
    cudaGraph_t body_out = nullptr;
    const cudaError_t e = cudaStreamEndCapture(S->side, &body_out);
    LQ_TRY(st);
    LQ_TRY_CUDA(e, "body end capture");
    LQ_TRY_CUDA(cudaStreamUpdateCaptureDependencies(s, &cnode, 1, cudaStreamSetCaptureDependencies),
                "capture dependencies");
    return LQ_OK;
}

/* Step graph: decide -> IF(rebuild) [-> IF(renewal)] -> stages. */
int capture_step(LqSim* S)
{
    cudaStream_t s = S->stream;
    LQ_TRY_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
    int st = LQ_OK;
    cudaGraph_t graph = nullptr;
    do {
        cudaStreamCaptureStatus cs;
        cudaGraph_t cg = nullptr;
        cudaError_t e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, nullptr, nullptr);
        if (e != cudaSuccess) { st = lqb::cuda_status(e, "capture info"); break; }
        cudaGraphConditionalHandle h_sort, h_renew;
        e = cudaGraphConditionalHandleCreate(&h_sort, cg, 0, 0);
        if (e == cudaSuccess && two_level(S)) e = cudaGraphConditionalHandleCreate(&h_renew, cg, 0, 0);
        if (e != cudaSuccess) { st = lqb::cuda_status(e, "conditional handle"); break; }
        if (two_level(S))
            k_decide2<<<1, 1, 0, s>>>(h_sort, h_renew, S->rebuild, S->rebuilds, S->renewals);
        else
            k_decide<<<1, 1, 0, s>>>(h_sort, S->rebuild, S->rebuilds);
        e = cudaGetLastError();
        if (e != cudaSuccess) { st = lqb::cuda_status(e, "k_decide"); break; }
        st = capture_if(S, h_sort, enqueue_rebuild);
        if (st == LQ_OK && two_level(S)) st = capture_if(S, h_renew, enqueue_renewal);
        if (st != LQ_OK) break;
        st = enqueue_stages(S, s);
    } while (0);
    cudaError_t e = cudaStreamEndCapture(s, &graph);
    if (st != LQ_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    if (e != cudaSuccess) return lqb::cuda_status(e, "end capture");
    e = cudaGraphInstantiate(&S->step_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        S->step_exec = nullptr;
        return lqb::cuda_status(e, "graph instantiate");
    }
    return LQ_OK;
}

int capture_plain(LqSim* S, int (*fn)(LqSim*, cudaStream_t), cudaGraphExec_t* exec)
{
    cudaGraph_t graph = nullptr;
    LQ_TRY_CUDA(cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    int st = fn(S, S->stream);
    cudaError_t e = cudaStreamEndCapture(S->stream, &graph);
    if (st != LQ_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    if (e != cudaSuccess) return lqb::cuda_status(e, "end capture");
    e = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return lqb::cuda_status(e, "graph instantiate");
    return LQ_OK;
}

/* Reads the rebuild flag on the host and decides as k_decide / k_decide2
 * do: clears it and counts the sort or the renewal. */
int host_take_flag(LqSim* S, bool* sort, bool* renew)
{
    cudaStream_t s = S->stream;
    LQ_TRY_CUDA(cudaMemcpyAsync(S->host_flag, S->rebuild, sizeof(int), cudaMemcpyDeviceToHost, s), "flag read");
    LQ_TRY_CUDA(cudaStreamSynchronize(s), "flag read");
    const int f = *S->host_flag;
    const bool due = (f & kFlagLists) != 0;
    const bool two = two_level(S);
    *sort = due && (!two || (f & kFlagSort) != 0);
    *renew = two && due;
    if (f) LQ_TRY(lqb::fill_int(S->rebuild, 1, 0, s));
    if (*sort) LQ_TRY(lqb::add_int(S->rebuilds, 1, s));
    else if (*renew) LQ_TRY(lqb::add_int(S->renewals, 1, s));
    return LQ_OK;
}

/* One step without the step graph: the host reads the flag. */
int eager_step(LqSim* S)
{
    bool sort = false, renew = false;
    LQ_TRY(host_take_flag(S, &sort, &renew));
    if (sort) LQ_TRY(enqueue_rebuild(S, S->stream));
    if (renew) LQ_TRY(enqueue_renewal(S, S->stream));
    return enqueue_stages(S, S->stream);
}

int upload(LqSim* S, const float* pos, const float* vel, const float* idep, const float* str, const float* stn,
           State& dst)
{
    const size_t n = (size_t)S->np;
    cudaStream_t s = S->stream;
    LQ_TRY_CUDA(cudaMemcpyAsync(dst.pos, pos, n * sizeof(float4), cudaMemcpyHostToDevice, s), "upload pos");
    LQ_TRY_CUDA(cudaMemcpyAsync(dst.vel, vel, n * sizeof(float4), cudaMemcpyHostToDevice, s), "upload vel");
    LQ_TRY_CUDA(cudaMemcpyAsync(dst.idep, idep, n * sizeof(float4), cudaMemcpyHostToDevice, s), "upload idep");
    LQ_TRY_CUDA(cudaMemcpyAsync(dst.str, str, n * sizeof(tensor2d), cudaMemcpyHostToDevice, s), "upload str");
    LQ_TRY_CUDA(cudaMemcpyAsync(dst.stn, stn, n * sizeof(tensor2d), cudaMemcpyHostToDevice, s), "upload stn");
    return LQ_OK;
}

int set_flag(LqSim* S, int v) { return lqb::fill_int(S->rebuild, 1, v, S->stream); }

/* New positions, order or list settings: sort and build all lists first. */
int flag_full_rebuild(LqSim* S) { return set_flag(S, kFlagAll); }

int widen(LqSim* S)
{
    if (!S->S.xlo) return LQ_OK;
    k_widen<<<blocks(S->np), 256, 0, S->stream>>>(S->np, S->S);
    LQ_TRY_CUDA(cudaGetLastError(), "k_widen");
    return LQ_OK;
}

int build_graphs(LqSim* S)
{
    if (S->step_exec) cudaGraphExecDestroy(S->step_exec);
    if (S->shep_exec) cudaGraphExecDestroy(S->shep_exec);
    S->step_exec = S->shep_exec = nullptr;
    S->conditional = false;
    LQ_TRY(ensure_tile_order(S));
    if (!(S->flags & LQ_SIM_GRAPH)) return LQ_OK;
    /* model 3 steps need the von Wolffersdorff table; capture once it is set */
    if (S->ph.constitutive_model == 3 && S->vw.n == 0) return LQ_OK;
    if (capture_step(S) == LQ_OK) {
        S->conditional = true;
    } else {
        cudaGetLastError(); /* fall back to host-decided rebuilds */
        S->step_exec = nullptr;
    }
    LQ_TRY(capture_plain(S, enqueue_shepard, &S->shep_exec));
    return LQ_OK;
}

int create(LqSim* S, const Parameters* par, const float* pos, const float* vel, const float* idep, const float* str,
           const float* stn, int flags)
{
    S->ph = *par;
    S->np = par->np;
    S->npb = par->npb;
    S->npm = par->npm;
    S->flags = flags;
    S->pair_shape = lqb::default_pair_shape(S->npm);
    if (S->np <= 0 || S->npb < 0 || S->npm < 0 || S->npb + S->npm != S->np)
        return lqb::set_error(LQ_ERR_ARG, "lq_sim_create: inconsistent counts np=%d npb=%d npm=%d", S->np, S->npb,
                              S->npm);
    if (S->ph.ncell != 2 * S->ph.ncell_one_layer + 1 || S->ph.ncell_one_layer <= 0 || S->ph.h <= 0.0f)
        return lqb::set_error(LQ_ERR_ARG, "lq_sim_create: Parameters not initialised (call lq_initialize_parameters)");
    if (!(S->ph.cs > 0.0f) || !(S->ph.cfl > 0.0f))
        return lqb::set_error(LQ_ERR_ARG, "lq_sim_create: cs and cfl must be positive");
    if (S->ph.constitutive_model < 1 || S->ph.constitutive_model > 3)
        return lqb::set_error(LQ_ERR_ARG, "lq_sim_create: constitutive_model must be 1, 2 or 3");
    S->ph.dt = S->ph.cfl * S->ph.h / S->ph.cs; /* reference src/loquat.cu:333 */
    S->time = (double)S->ph.time;
    S->skin = kDefaultSkinOverH * S->ph.h;
    LQ_TRY_CUDA(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking), "stream create");
    LQ_TRY_CUDA(cudaStreamCreateWithFlags(&S->side, cudaStreamNonBlocking), "stream create");
    LQ_TRY_CUDA(cudaMallocHost((void**)&S->host_flag, sizeof(int)), "pinned flag");
    LQ_TRY(dev_alloc(S, (void**)&S->pd, sizeof(Parameters)));
    LQ_TRY(alloc_state(S, S->S));
    LQ_TRY(alloc_state(S, S->S2));
    LQ_TRY(alloc_state(S, S->T));
    const size_t n = (size_t)S->np;
    LQ_TRY(dev_alloc(S, (void**)&S->xbuild, n * sizeof(float4)));
    if (S->flags & LQ_SIM_DENSITY_FILTER) LQ_TRY(dev_alloc(S, (void**)&S->rho_f, n * sizeof(float)));
    if (S->flags & LQ_SIM_DYNAMIC_DT) {
        LQ_TRY(dev_alloc(S, (void**)&S->vmax2, 2 * sizeof(unsigned)));
        LQ_TRY(dev_alloc(S, (void**)&S->dtime, sizeof(double)));
    }
    LQ_TRY(dev_alloc(S, (void**)&S->rec, n * 13 * sizeof(float)));   /* cudaMalloc: 256-byte aligned */
    LQ_TRY(dev_alloc(S, (void**)&S->R.accad, n * sizeof(float4)));
    LQ_TRY(dev_alloc(S, (void**)&S->R.spin, n * sizeof(float4)));
    LQ_TRY(dev_alloc(S, (void**)&S->R.acestn, n * sizeof(tensor2d)));
    LQ_TRY(dev_alloc(S, (void**)&S->health, sizeof(int) * lqb::HEALTH_WORDS));
    LQ_TRY(dev_alloc(S, (void**)&S->rebuild, sizeof(int)));
    LQ_TRY(dev_alloc(S, (void**)&S->rebuilds, sizeof(int)));
    LQ_TRY(dev_alloc(S, (void**)&S->renewals, sizeof(int)));
    S->nlm.stride = ((S->npm > 0 ? S->npm : 1) + 31) / 32 * 32;
    LQ_TRY(dev_alloc(S, (void**)&S->nlm.list, sizeof(int) * (size_t)LQ_NBR_CAP * S->nlm.stride));
    LQ_TRY(dev_alloc(S, (void**)&S->nlm.count, sizeof(int) * (size_t)S->nlm.stride));
    S->nlb.stride = ((S->npb > 0 ? S->npb : 1) + 31) / 32 * 32;
    LQ_TRY(dev_alloc(S, (void**)&S->nlb.list, sizeof(int) * (size_t)LQ_NBR_CAP * S->nlb.stride));
    LQ_TRY(dev_alloc(S, (void**)&S->nlb.count, sizeof(int) * (size_t)S->nlb.stride));
    LQ_TRY(dev_alloc(S, (void**)&S->bact, sizeof(int) * (size_t)S->nlb.stride));
    LQ_TRY(dev_alloc(S, (void**)&S->nbact, sizeof(int)));
    S->bsel_bytes = lqb::boundary_targets_temp_bytes(S->npb);
    LQ_TRY(dev_alloc(S, &S->bsel_tmp, S->bsel_bytes));
    const int ncell = S->ph.ncell;
    lqb::GridBuffers& g = S->g;
    LQ_TRY(lqb::scan_scratch_bytes(ncell, &g.scan_bytes));
    LQ_TRY(dev_alloc(S, (void**)&g.key, n * sizeof(int)));
    LQ_TRY(dev_alloc(S, (void**)&g.rank, n * sizeof(int)));
    LQ_TRY(dev_alloc(S, (void**)&g.part_idx, n * sizeof(int)));
    LQ_TRY(dev_alloc(S, (void**)&g.part_cel, n * sizeof(int)));
    LQ_TRY(dev_alloc(S, (void**)&g.count, sizeof(int) * (size_t)(ncell + 1)));
    LQ_TRY(dev_alloc(S, (void**)&g.start, sizeof(int) * (size_t)(ncell + 1)));
    LQ_TRY(dev_alloc(S, &g.scan_tmp, g.scan_bytes));
    g.np_cap = S->np;
    g.ncell_cap = ncell;

    LQ_TRY_CUDA(cudaMemsetAsync(S->R.accad, 0, n * sizeof(float4), S->stream), "zero rates");
    LQ_TRY_CUDA(cudaMemsetAsync(S->R.spin, 0, n * sizeof(float4), S->stream), "zero rates");
    LQ_TRY_CUDA(cudaMemsetAsync(S->R.acestn, 0, n * sizeof(tensor2d), S->stream), "zero rates");
    LQ_TRY_CUDA(cudaMemsetAsync(S->health, 0, sizeof(int) * lqb::HEALTH_WORDS, S->stream), "zero health");
    LQ_TRY_CUDA(cudaMemsetAsync(S->rebuilds, 0, sizeof(int), S->stream), "zero counter");
    LQ_TRY_CUDA(cudaMemsetAsync(S->nbact, 0, sizeof(int), S->stream), "zero boundary targets");
    LQ_TRY_CUDA(cudaMemsetAsync(S->renewals, 0, sizeof(int), S->stream), "zero counter");
    LQ_TRY_CUDA(cudaMemcpyAsync(S->pd, &S->ph, sizeof(Parameters), cudaMemcpyHostToDevice, S->stream),
                "upload Parameters");
    LQ_TRY(upload(S, pos, vel, idep, str, stn, S->S));
    LQ_TRY(widen(S));
    if (S->flags & LQ_SIM_DYNAMIC_DT) {
        LQ_TRY_CUDA(cudaMemsetAsync(S->vmax2, 0, 2 * sizeof(unsigned), S->stream), "dt maxima");
        LQ_TRY_CUDA(cudaMemcpyAsync(S->dtime, &S->time, sizeof(double), cudaMemcpyHostToDevice, S->stream),
                    "device time");
    }
    /* the first step searches and sorts (reference src/loquat.cu:297-298) */
    LQ_TRY(flag_full_rebuild(S));
    LQ_TRY_CUDA(cudaStreamSynchronize(S->stream), "sim create");
    LQ_TRY(build_graphs(S));
    return LQ_OK;
}

}  // namespace

extern "C" int lq_sim_create(const void* par_host, const float* pospres, const float* velrhop, const float* idep,
                             const float* str, const float* stn, int flags, void** sim)
{
    if (!sim) return lqb::set_error(LQ_ERR_ARG, "lq_sim_create: null output");
    *sim = nullptr;
    if (!par_host || !pospres || !velrhop || !idep || !str || !stn)
        return lqb::set_error(LQ_ERR_ARG, "lq_sim_create: null argument");
    LqSim* S = new LqSim();
    int st = create(S, static_cast<const Parameters*>(par_host), pospres, velrhop, idep, str, stn, flags);
    if (st != LQ_OK) {
        release(S);
        delete S;
        return st;
    }
    *sim = S;
    return LQ_OK;
}

extern "C" int lq_sim_destroy(void* sim)
{
    if (!sim) return LQ_OK;
    LqSim* S = static_cast<LqSim*>(sim);
    release(S);
    delete S;
    return LQ_OK;
}

extern "C" int lq_sim_step(void* sim, int nsteps)
{
    if (!sim || nsteps < 0) return lqb::set_error(LQ_ERR_ARG, "lq_sim_step: bad argument");
    LqSim* S = static_cast<LqSim*>(sim);
    if (S->ph.constitutive_model == 3 && S->vw.n == 0)
        return lqb::set_error(LQ_ERR_ARG, "lq_sim_step: constitutive model 3 needs lq_sim_set_hypoplastic first");
    const int N = S->ph.stress_shepard_filter;
    nvtxRangePushA(S->step_exec ? "lq/steps (graph)" : "lq/steps (eager)");
    struct PopRange {
        ~PopRange() { nvtxRangePop(); }
    } pop_range;
    for (int k = 0; k < nsteps; ++k) {
        S->ph.time = (float)S->time;
        if (S->step_exec) {
            LQ_TRY_CUDA(cudaGraphLaunch(S->step_exec, S->stream), "step graph launch");
        } else {
            LQ_TRY(eager_step(S));
        }
        if (N != 0 && S->step % N == 0 && S->step != 0) {
            if (S->shep_exec) {
                LQ_TRY_CUDA(cudaGraphLaunch(S->shep_exec, S->stream), "Shepard graph launch");
            } else {
                LQ_TRY(enqueue_shepard(S, S->stream));
            }
        }
        const int Nd = S->ph.density_shepard_filter;
        if ((S->flags & LQ_SIM_DENSITY_FILTER) && Nd > 0 && S->step % Nd == 0 && S->step != 0)
            LQ_TRY(enqueue_density_filter(S, S->stream));
        S->time += (double)S->ph.dt;   /* the fixed step; the device keeps the time of dynamic steps */
        S->step++;
    }
    return LQ_OK;
}

extern "C" int lq_sim_synchronize(void* sim)
{
    if (!sim) return lqb::set_error(LQ_ERR_ARG, "lq_sim_synchronize: null sim");
    LQ_TRY_CUDA(cudaStreamSynchronize(static_cast<LqSim*>(sim)->stream), "sim synchronize");
    return LQ_OK;
}

extern "C" int lq_sim_stream(void* sim, void** stream)
{
    if (!sim || !stream) return lqb::set_error(LQ_ERR_ARG, "lq_sim_stream: null argument");
    *stream = static_cast<LqSim*>(sim)->stream;
    return LQ_OK;
}

extern "C" int lq_sim_upload(void* sim, const float* pospres, const float* velrhop, const float* idep,
                             const float* str, const float* stn)
{
    if (!sim || !pospres || !velrhop || !idep || !str || !stn)
        return lqb::set_error(LQ_ERR_ARG, "lq_sim_upload: null argument");
    LqSim* S = static_cast<LqSim*>(sim);
    LQ_TRY(upload(S, pospres, velrhop, idep, str, stn, S->S));
    LQ_TRY(widen(S));
    return flag_full_rebuild(S); /* new positions: search and rebuild the lists first */
}

extern "C" int lq_sim_download(void* sim, float* pospres, float* velrhop, float* idep, float* str, float* stn)
{
    if (!sim) return lqb::set_error(LQ_ERR_ARG, "lq_sim_download: null sim");
    LqSim* S = static_cast<LqSim*>(sim);
    const size_t n = (size_t)S->np;
    cudaStream_t s = S->stream;
    if (pospres) LQ_TRY_CUDA(cudaMemcpyAsync(pospres, S->S.pos, n * sizeof(float4), cudaMemcpyDeviceToHost, s), "dl");
    if (velrhop) LQ_TRY_CUDA(cudaMemcpyAsync(velrhop, S->S.vel, n * sizeof(float4), cudaMemcpyDeviceToHost, s), "dl");
    if (idep) LQ_TRY_CUDA(cudaMemcpyAsync(idep, S->S.idep, n * sizeof(float4), cudaMemcpyDeviceToHost, s), "dl");
    if (str) LQ_TRY_CUDA(cudaMemcpyAsync(str, S->S.str, n * sizeof(tensor2d), cudaMemcpyDeviceToHost, s), "dl");
    if (stn) LQ_TRY_CUDA(cudaMemcpyAsync(stn, S->S.stn, n * sizeof(tensor2d), cudaMemcpyDeviceToHost, s), "dl");
    LQ_TRY_CUDA(cudaStreamSynchronize(s), "download");
    return LQ_OK;
}

extern "C" int lq_sim_state(void* sim, float** pospres, float** velrhop, float** idep, float** str, float** stn)
{
    if (!sim) return lqb::set_error(LQ_ERR_ARG, "lq_sim_state: null sim");
    LqSim* S = static_cast<LqSim*>(sim);
    if (pospres) *pospres = (float*)S->S.pos;
    if (velrhop) *velrhop = (float*)S->S.vel;
    if (idep) *idep = (float*)S->S.idep;
    if (str) *str = (float*)S->S.str;
    if (stn) *stn = (float*)S->S.stn;
    return LQ_OK;
}

extern "C" int lq_sim_clock(void* sim, long long* step, double* time)
{
    if (!sim) return lqb::set_error(LQ_ERR_ARG, "lq_sim_clock: null sim");
    LqSim* S = static_cast<LqSim*>(sim);
    if (step) *step = S->step;
    if (time) {
        *time = S->time;
        if (S->flags & LQ_SIM_DYNAMIC_DT) {
            LQ_TRY_CUDA(cudaMemcpyAsync(time, S->dtime, sizeof(double), cudaMemcpyDeviceToHost, S->stream),
                        "device time");
            LQ_TRY_CUDA(cudaStreamSynchronize(S->stream), "device time");
        }
    }
    return LQ_OK;
}

extern "C" int lq_sim_health(void* sim, int* health4)
{
    if (!sim || !health4) return lqb::set_error(LQ_ERR_ARG, "lq_sim_health: null argument");
    LqSim* S = static_cast<LqSim*>(sim);
    LQ_TRY_CUDA(cudaMemcpyAsync(health4, S->health, sizeof(int) * lqb::HEALTH_WORDS, cudaMemcpyDeviceToHost,
                                S->stream),
                "health read");
    LQ_TRY_CUDA(cudaMemsetAsync(S->health, 0, sizeof(int) * lqb::HEALTH_WORDS, S->stream), "health reset");
    LQ_TRY_CUDA(cudaStreamSynchronize(S->stream), "health read");
    return LQ_OK;
}

extern "C" int lq_sim_rebuilds(void* sim, long long* count)
{
    if (!sim || !count) return lqb::set_error(LQ_ERR_ARG, "lq_sim_rebuilds: null argument");
    LqSim* S = static_cast<LqSim*>(sim);
    int c = 0;
    LQ_TRY_CUDA(cudaMemcpyAsync(&c, S->rebuilds, sizeof(int), cudaMemcpyDeviceToHost, S->stream), "rebuild count");
    LQ_TRY_CUDA(cudaStreamSynchronize(S->stream), "rebuild count");
    *count = c;
    return LQ_OK;
}

extern "C" int lq_sim_set_skin(void* sim, float skin_over_h)
{
    if (!sim || !(skin_over_h >= 0.0f) || skin_over_h > 2.0f)
        return lqb::set_error(LQ_ERR_ARG, "lq_sim_set_skin: skin/h must be in [0, 2]");
    LqSim* S = static_cast<LqSim*>(sim);
    LQ_TRY_CUDA(cudaStreamSynchronize(S->stream), "set skin");
    S->skin = skin_over_h * S->ph.h;
    LQ_TRY(flag_full_rebuild(S));
    LQ_TRY(build_graphs(S));
    return LQ_OK;
}

extern "C" int lq_sim_set_wide_skin(void* sim, float wide_over_h)
{
    if (!sim || !(wide_over_h >= 0.0f) || wide_over_h > 2.0f)
        return lqb::set_error(LQ_ERR_ARG, "lq_sim_set_wide_skin: wide/h must be in [0, 2]");
    LqSim* S = static_cast<LqSim*>(sim);
    LQ_TRY_CUDA(cudaStreamSynchronize(S->stream), "set wide skin");
    if (wide_over_h > 0.0f) LQ_TRY(ensure_wide_lists(S));
    S->wide = wide_over_h * S->ph.h;
    LQ_TRY(flag_full_rebuild(S));
    LQ_TRY(build_graphs(S));
    return LQ_OK;
}

extern "C" int lq_sim_renewals(void* sim, long long* count)
{
    if (!sim || !count) return lqb::set_error(LQ_ERR_ARG, "lq_sim_renewals: null argument");
    LqSim* S = static_cast<LqSim*>(sim);
    int c = 0;
    LQ_TRY_CUDA(cudaMemcpyAsync(&c, S->renewals, sizeof(int), cudaMemcpyDeviceToHost, S->stream), "renewal count");
    LQ_TRY_CUDA(cudaStreamSynchronize(S->stream), "renewal count");
    *count = c;
    return LQ_OK;
}

extern "C" int lq_sim_set_materials(void* sim, int n, const float* table)
{
    if (!sim || n < 0 || (n > 0 && !table)) return lqb::set_error(LQ_ERR_ARG, "lq_sim_set_materials: bad argument");
    LqSim* S = static_cast<LqSim*>(sim);
    LQ_TRY_CUDA(cudaStreamSynchronize(S->stream), "set materials");
    float* d = nullptr;
    if (n > 0) {
        LQ_TRY(dev_alloc(S, (void**)&d, sizeof(float) * 5 * (size_t)n));
        LQ_TRY_CUDA(cudaMemcpy(d, table, sizeof(float) * 5 * (size_t)n, cudaMemcpyHostToDevice), "material table");
    }
    S->mt.p = d;
    S->mt.n = n;
    S->mt_host.assign(table, table + 5 * (size_t)n);
    LQ_TRY(build_graphs(S));
    return LQ_OK;
}

extern "C" int lq_sim_set_hypoplastic(void* sim, int n, const float* table)
{
    if (!sim || n < 1 || !table) return lqb::set_error(LQ_ERR_ARG, "lq_sim_set_hypoplastic: bad argument");
    for (int k = 0; k < n; ++k) {
        const float* r = table + 10 * (size_t)k;
        const bool ok = r[0] > 0.0f && r[0] < 90.0f && r[1] > 0.0f && r[2] > 0.0f && r[2] < 1.0f && r[3] > 0.0f &&
                        r[3] < r[4] && r[4] < r[5] && r[6] >= 0.0f && r[7] >= 0.0f && r[8] > 0.0f && r[8] < 1.0f &&
                        r[9] >= 1.0f && r[9] <= 100000.0f;
        if (!ok)
            return lqb::set_error(LQ_ERR_ARG,
                                  "lq_sim_set_hypoplastic: row %d needs 0 < phic < 90, hs > 0, 0 < n < 1, "
                                  "0 < ed0 < ec0 < ei0, alpha, beta >= 0, 0 < tol < 1, 1 <= max_substeps <= 1e5",
                                  k);
    }
    LqSim* S = static_cast<LqSim*>(sim);
    LQ_TRY_CUDA(cudaStreamSynchronize(S->stream), "set hypoplastic");
    float* d = nullptr;
    LQ_TRY(dev_alloc(S, (void**)&d, sizeof(float) * 10 * (size_t)n));
    LQ_TRY_CUDA(cudaMemcpy(d, table, sizeof(float) * 10 * (size_t)n, cudaMemcpyHostToDevice), "hypoplastic table");
    S->vw.p = d;
    S->vw.n = n;
    S->vw_host.assign(table, table + 10 * (size_t)n);
    LQ_TRY(build_graphs(S));
    return LQ_OK;
}

extern "C" int lq_sim_set_frames(void* sim, int n, const int* rows)
{
    if (!sim || n < 0 || (n > 0 && !rows)) return lqb::set_error(LQ_ERR_ARG, "lq_sim_set_frames: bad argument");
    LqSim* S = static_cast<LqSim*>(sim);
    for (int k = 0; k < n; ++k) {
        if (rows[2 * k] < 0 || rows[2 * k + 1] < 0 || rows[2 * k] + rows[2 * k + 1] > S->ph.cell_num_y)
            return lqb::set_error(LQ_ERR_ARG, "lq_sim_set_frames: object %d rows [%d, +%d) outside cell_num_y=%d", k,
                                  rows[2 * k], rows[2 * k + 1], S->ph.cell_num_y);
    }
    LQ_TRY_CUDA(cudaStreamSynchronize(S->stream), "set frames");
    int* d = nullptr;
    if (n > 0) {
        LQ_TRY(dev_alloc(S, (void**)&d, sizeof(int) * 2 * (size_t)n));
        LQ_TRY_CUDA(cudaMemcpy(d, rows, sizeof(int) * 2 * (size_t)n, cudaMemcpyHostToDevice), "frame table");
    }
    S->fr.rows = d;
    S->fr.n = n;
    S->fr_host.assign(rows, rows + 2 * (size_t)n);
    LQ_TRY(flag_full_rebuild(S));
    LQ_TRY(build_graphs(S));
    return LQ_OK;
}

extern "C" int lq_sim_launches_per_step(void* sim, int* plain, int* with_shepard)
{
    if (!sim) return lqb::set_error(LQ_ERR_ARG, "lq_sim_launches_per_step: null sim");
    LqSim* S = static_cast<LqSim*>(sim);
    /* own kernels of a step without a rebuild: decide (graph only), Adami
     * (when npb > 0), interaction and integrator (which packs the material
     * slots' neighbour data) per stage; a Shepard pass adds the filter, its
     * copy and the material pack */
    const int stage = (S->npb > 0 ? 1 : 0) + 1 + 1;
    const int decide = S->conditional ? 1 : 0;
    const int dyn = (S->flags & LQ_SIM_DYNAMIC_DT) ? (S->npm > 0 ? 2 : 1) : 0;
    if (plain) *plain = decide + 2 * stage + dyn;
    if (with_shepard) *with_shepard = decide + 2 * stage + dyn + (S->npm > 0 ? 3 : 0);
    return LQ_OK;
}

/* ------------------------------------------------------------- autotuning */
extern "C" int lq_sim_pair_shape(void* sim, int* shape)
{
    if (!sim || !shape) return lqb::set_error(LQ_ERR_ARG, "lq_sim_pair_shape: null argument");
    *shape = static_cast<LqSim*>(sim)->pair_shape;
    return LQ_OK;
}

extern "C" int lq_sim_set_pair_shape(void* sim, int shape)
{
    if (!sim || shape < 0 || shape >= lqb::kPairShapeCount)
        return lqb::set_error(LQ_ERR_ARG, "lq_sim_set_pair_shape: shape must be in [0, %d)", lqb::kPairShapeCount);
    LqSim* S = static_cast<LqSim*>(sim);
    LQ_TRY_CUDA(cudaStreamSynchronize(S->stream), "set pair shape");
    S->pair_shape = shape;
    LQ_TRY(build_graphs(S));
    if (!tiled(S)) return LQ_OK;
    /* the lists are current unless a search is pending: order them now */
    LQ_TRY_CUDA(cudaMemcpyAsync(S->host_flag, S->rebuild, sizeof(int), cudaMemcpyDeviceToHost, S->stream),
                "flag read");
    LQ_TRY_CUDA(cudaStreamSynchronize(S->stream), "flag read");
    if (*S->host_flag == 0) LQ_TRY(lqb::launch_tile_order(&S->ph, S->g.start, S->pair_shape, S->tile, S->stream));
    LQ_TRY_CUDA(cudaStreamSynchronize(S->stream), "tile order");
    return LQ_OK;
}

namespace {

/* A device copy of everything a trial step changes, so that tuning leaves
 * the simulation where it was. */
struct Snapshot {
    std::vector<std::pair<void*, size_t>> items;   /* (live buffer, bytes) */
    std::vector<void*> copies;
    long long step = 0;
    double time = 0.0;
    float skin = 0.0f, wide = 0.0f;
    int shape = 0;
    ~Snapshot()
    {
        for (void* p : copies) cudaFree(p);
    }
    int take(LqSim* S)
    {
        const size_t n = (size_t)S->np;
        items = {{S->S.pos, n * sizeof(float4)},  {S->S.vel, n * sizeof(float4)},
                 {S->S.idep, n * sizeof(float4)}, {S->S.str, n * sizeof(tensor2d)},
                 {S->S.stn, n * sizeof(tensor2d)}, {S->health, sizeof(int) * lqb::HEALTH_WORDS},
                 {S->rebuilds, sizeof(int)},      {S->pd, sizeof(Parameters)},
                 {S->renewals, sizeof(int)}};
        if (S->S.xlo) {
            items.push_back({S->S.xlo, n * sizeof(float4)});
            items.push_back({S->S.vlo, n * sizeof(float4)});
        }
        if (S->dtime) items.push_back({S->dtime, sizeof(double)});
        for (auto& it : items) {
            void* c = nullptr;
            cudaError_t e = cudaMalloc(&c, it.second);
            if (e != cudaSuccess)
                return lqb::set_error(LQ_ERR_ALLOC, "autotune: no room for a state copy (%zu bytes): %s", it.second,
                                      cudaGetErrorString(e));
            copies.push_back(c);
            LQ_TRY_CUDA(cudaMemcpyAsync(c, it.first, it.second, cudaMemcpyDeviceToDevice, S->stream), "snapshot");
        }
        step = S->step;
        time = S->time;
        skin = S->skin;
        wide = S->wide;
        shape = S->pair_shape;
        return LQ_OK;
    }
    int restore(LqSim* S)
    {
        for (size_t k = 0; k < items.size(); ++k)
            LQ_TRY_CUDA(cudaMemcpyAsync(items[k].first, copies[k], items[k].second, cudaMemcpyDeviceToDevice,
                                        S->stream),
                        "restore");
        S->step = step;
        S->time = time;
        return flag_full_rebuild(S); /* lists are rebuilt before the next step */
    }
};

int cuda_ok(cudaError_t e, const char* what) { return e == cudaSuccess ? LQ_OK : lqb::cuda_status(e, what); }

/* ms per step of `steps` steps from a state flagged for a sort: the sort
 * and list build that start every run are inside the window, so settings
 * whose lists last long pay for one build in `steps` steps, not nothing. */
int time_steps(LqSim* S, int steps, float* ms)
{
    cudaEvent_t a, b;
    LQ_TRY_CUDA(cudaEventCreate(&a), "event");
    LQ_TRY_CUDA(cudaEventCreate(&b), "event");
    int st = LQ_OK;
    if (st == LQ_OK) st = cuda_ok(cudaEventRecord(a, S->stream), "event");
    if (st == LQ_OK) st = lq_sim_step(S, steps);
    if (st == LQ_OK) st = cuda_ok(cudaEventRecord(b, S->stream), "event");
    if (st == LQ_OK) st = cuda_ok(cudaEventSynchronize(b), "event");
    if (st == LQ_OK) st = cuda_ok(cudaEventElapsedTime(ms, a, b), "event");
    if (st == LQ_OK) *ms /= (float)steps;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return st;
}

}  // namespace

extern "C" int lq_sim_autotune(void* sim, int steps, int* shape_out, float* skin_over_h_out)
{
    if (!sim || steps < 1) return lqb::set_error(LQ_ERR_ARG, "lq_sim_autotune: bad argument");
    LqSim* S = static_cast<LqSim*>(sim);
    if (S->ph.constitutive_model == 3 && S->vw.n == 0)
        return lqb::set_error(LQ_ERR_ARG, "lq_sim_autotune: set the model-3 table first");
    Snapshot snap;
    LQ_TRY(snap.take(S));
    const float h = S->ph.h;
    int best_shape = S->pair_shape;
    float best_skin = S->skin, best_wide = S->wide, best_ms = 3.4e38f;
    float best_factor = S->skin / h;   /* skin / h as the caller would pass it to lq_sim_set_skin */
    float factor = best_factor;
    float shape_ms[lqb::kPairShapeCount];
    auto trial = [&](int shape, float skin, float wide, int nsteps = 0) -> int {
        LQ_TRY(snap.restore(S));
        S->pair_shape = shape;
        S->skin = skin;
        if (wide > skin) LQ_TRY(ensure_wide_lists(S));
        S->wide = wide;
        LQ_TRY(build_graphs(S));
        float ms = 0.0f;
        LQ_TRY(time_steps(S, nsteps > 0 ? nsteps : steps, &ms));
        shape_ms[shape] = ms;
        if (ms < best_ms) {
            best_ms = ms;
            best_shape = shape;
            best_skin = skin;
            best_wide = wide;
            best_factor = factor;
        }
        return LQ_OK;
    };
    /* launch shapes at the current lists, then one-level skins with the best
     * shape, then two-level lists over the best skin whose wide margin
     * (wide - skin <= 0.2 h) keeps a pair that the 3 x 3-column walk of the
     * wide build leaves out below the kernel factor (0.2)^3, as the
     * one-level skins do */
    int st = LQ_OK;
    for (int k = 0; k < lqb::kPairShapeCount && st == LQ_OK; ++k) st = trial(k, snap.skin, snap.wide);
    /* the shapes within 5 % of the fastest at the starting lists (at most
     * four): re-timed once the lists are chosen */
    std::vector<int> contenders;
    if (st == LQ_OK) {
        const float first_best = best_ms;
        for (int k = 0; k < lqb::kPairShapeCount; ++k)
            if (shape_ms[k] <= 1.05f * first_best) contenders.push_back(k);
        std::sort(contenders.begin(), contenders.end(), [&](int a, int b) { return shape_ms[a] < shape_ms[b]; });
        if (contenders.size() > 4) contenders.resize(4);
    }
    const float skins[] = {0.02f, 0.05f, 0.1f, 0.2f};
    const int shape = best_shape;
    for (float f : skins) {
        factor = f;
        if (st == LQ_OK && (f * h != snap.skin || snap.wide > snap.skin)) st = trial(shape, f * h, 0.0f);
    }
    /* two-level lists over the best one-level skin and over narrow skins,
     * whose lists hold fewer pairs beyond 2h while cheap renewals keep them
     * current */
    const float margins[] = {0.1f, 0.2f};
    const float best1 = best_factor;
    const float two_skins[] = {best1, 0.02f, 0.01f};
    for (int a = 0; a < 3 && st == LQ_OK; ++a) {
        const float f = two_skins[a];
        if (a > 0 && f >= best1) continue;       /* narrower than the best one-level skin only */
        factor = f;
        for (float m : margins)
            if (st == LQ_OK) st = trial(shape, f * h, (f + m) * h);
    }
    /* the contending shapes again at the chosen lists, each over twice the
     * steps, the fastest of this round kept: a 40-step trial at the
     * starting lists (mostly a list build) does not separate shapes a few
     * percent apart at the lists they will run with */
    if (st == LQ_OK && contenders.size() > 1) {
        const float skin = best_skin, wide = best_wide;
        factor = best_factor;
        best_ms = 3.4e38f;
        for (int k : contenders)
            if (st == LQ_OK) st = trial(k, skin, wide, 2 * steps);
    }
    /* back to the state before tuning, with the chosen configuration */
    int st2 = snap.restore(S);
    S->pair_shape = st == LQ_OK ? best_shape : snap.shape;
    S->skin = st == LQ_OK ? best_skin : snap.skin;
    S->wide = st == LQ_OK ? best_wide : snap.wide;
    if (st2 == LQ_OK) st2 = build_graphs(S);
    if (st2 == LQ_OK) st2 = cuda_ok(cudaStreamSynchronize(S->stream), "autotune");
    if (st != LQ_OK) return st;
    if (st2 != LQ_OK) return st2;
    if (shape_out) *shape_out = S->pair_shape;
    if (skin_over_h_out) *skin_over_h_out = best_factor;
    return LQ_OK;
}

extern "C" int lq_sim_wide_skin(void* sim, float* wide_over_h)
{
    if (!sim || !wide_over_h) return lqb::set_error(LQ_ERR_ARG, "lq_sim_wide_skin: null argument");
    LqSim* S = static_cast<LqSim*>(sim);
    *wide_over_h = two_level(S) ? S->wide / S->ph.h : 0.0f;
    return LQ_OK;
}

/* ------------------------------------------------------------ checkpoints */
/* Binary checkpoint, little-endian as written by this library:
 *   "LQB200CK" | u32 version | u32 flags | i64 step | f64 time | f32 skin |
 *   i32 np, npb, npm | Parameters (208 B) |
 *   pospres, velrhop, idep (np x 16 B) | str, stn (np x 24 B) |
 *   [mixed form: x and v+rho in FP64, np x 32 B each] |
 *   i32 n + n x 5 f32 materials | i32 n + n x 10 f32 model-3 rows | i32 n + n x 2 i32 frames |
 *   [f32 wide: the two-level lists' cut-off beyond 2h; files without it load with one-level lists] */
namespace {

constexpr char kCkMagic[8] = {'L', 'Q', 'B', '2', '0', '0', 'C', 'K'};
constexpr uint32_t kCkVersion = 1;

struct CkWriter {
    FILE* f;
    bool ok = true;
    void put(const void* p, size_t n)
    {
        if (ok && n) ok = fwrite(p, 1, n, f) == n;
    }
    template <class T> void val(const T& v) { put(&v, sizeof(T)); }
};

struct CkReader {
    const std::vector<char>& b;
    size_t at = 0;
    bool ok = true;
    const char* take(size_t n)
    {
        if (!ok || b.size() - at < n) {
            ok = false;
            return nullptr;
        }
        const char* p = b.data() + at;
        at += n;
        return p;
    }
    template <class T> T val()
    {
        T v{};
        if (const char* p = take(sizeof(T))) memcpy(&v, p, sizeof(T));
        return v;
    }
};

}  // namespace

extern "C" int lq_sim_save_checkpoint(void* sim, const char* path)
{
    if (!sim || !path) return lqb::set_error(LQ_ERR_ARG, "lq_sim_save_checkpoint: null argument");
    LqSim* S = static_cast<LqSim*>(sim);
    const size_t n = (size_t)S->np;
    std::vector<float> pos(4 * n), vel(4 * n), idep(4 * n), str(6 * n), stn(6 * n);
    std::vector<double> xd, vd;
    LQ_TRY(lq_sim_download(sim, pos.data(), vel.data(), idep.data(), str.data(), stn.data()));
    if (S->S.xlo) {
        /* the file keeps the mixed form's values in FP64: high + low words */
        std::vector<float> xl(4 * n), vl(4 * n);
        LQ_TRY_CUDA(cudaMemcpyAsync(xl.data(), S->S.xlo, n * sizeof(float4), cudaMemcpyDeviceToHost, S->stream),
                    "checkpoint x");
        LQ_TRY_CUDA(cudaMemcpyAsync(vl.data(), S->S.vlo, n * sizeof(float4), cudaMemcpyDeviceToHost, S->stream),
                    "checkpoint v");
        LQ_TRY_CUDA(cudaStreamSynchronize(S->stream), "checkpoint read");
        xd.resize(4 * n);
        vd.resize(4 * n);
        for (size_t k = 0; k < 4 * n; ++k) {
            xd[k] = (k % 4 == 3) ? 0.0 : (double)pos[k] + (double)xl[k];
            vd[k] = (double)vel[k] + (double)vl[k];
        }
    }
    Parameters par = S->ph;
    double time = S->time;
    if (S->flags & LQ_SIM_DYNAMIC_DT) {
        /* the next step's dt and the time live on the device */
        LQ_TRY_CUDA(cudaMemcpyAsync(&par.dt, &S->pd->dt, sizeof(float), cudaMemcpyDeviceToHost, S->stream),
                    "checkpoint dt");
        LQ_TRY_CUDA(cudaMemcpyAsync(&time, S->dtime, sizeof(double), cudaMemcpyDeviceToHost, S->stream),
                    "checkpoint time");
        LQ_TRY_CUDA(cudaStreamSynchronize(S->stream), "checkpoint dt");
    }
    FILE* f = fopen(path, "wb");
    if (!f) return lqb::set_error(LQ_ERR_IO, "cannot write checkpoint %s", path);
    CkWriter w{f};
    w.put(kCkMagic, sizeof(kCkMagic));
    w.val(kCkVersion);
    w.val((uint32_t)S->flags);
    w.val((int64_t)S->step);
    w.val(time);
    w.val(S->skin);
    w.val((int32_t)S->np);
    w.val((int32_t)S->npb);
    w.val((int32_t)S->npm);
    w.put(&par, sizeof(Parameters));
    for (auto* a : {&pos, &vel, &idep, &str, &stn}) w.put(a->data(), a->size() * sizeof(float));
    if (!xd.empty()) {
        w.put(xd.data(), xd.size() * sizeof(double));
        w.put(vd.data(), vd.size() * sizeof(double));
    }
    w.val((int32_t)S->mt.n);
    w.put(S->mt_host.data(), S->mt_host.size() * sizeof(float));
    w.val((int32_t)S->vw.n);
    w.put(S->vw_host.data(), S->vw_host.size() * sizeof(float));
    w.val((int32_t)S->fr.n);
    w.put(S->fr_host.data(), S->fr_host.size() * sizeof(int));
    w.val(two_level(S) ? S->wide : 0.0f);
    const bool ok = w.ok && fclose(f) == 0;
    if (!ok) return lqb::set_error(LQ_ERR_IO, "write error on checkpoint %s", path);
    /* the run that continues searches before its next step, as a run
     * restarted from this file does, so both take identical steps */
    return flag_full_rebuild(S);
}

extern "C" int lq_sim_load_checkpoint(const char* path, int flags, void** sim)
{
    if (!path || !sim) return lqb::set_error(LQ_ERR_ARG, "lq_sim_load_checkpoint: null argument");
    *sim = nullptr;
    std::vector<char> buf;
    {
        FILE* f = fopen(path, "rb");
        if (!f) return lqb::set_error(LQ_ERR_IO, "cannot open checkpoint %s", path);
        char chunk[1 << 16];
        size_t got;
        while ((got = fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + got);
        fclose(f);
    }
    CkReader r{buf};
    const char* magic = r.take(sizeof(kCkMagic));
    if (!magic || memcmp(magic, kCkMagic, sizeof(kCkMagic)) != 0)
        return lqb::set_error(LQ_ERR_IO, "%s is not a LOQUAT-B200 checkpoint", path);
    const uint32_t version = r.val<uint32_t>();
    if (r.ok && version != kCkVersion)
        return lqb::set_error(LQ_ERR_IO, "%s: checkpoint version %u, this library reads %u", path, version,
                              kCkVersion);
    const uint32_t saved_flags = r.val<uint32_t>();
    const long long step = r.val<int64_t>();
    const double time = r.val<double>();
    const float skin = r.val<float>();
    const int np = r.val<int32_t>(), npb = r.val<int32_t>(), npm = r.val<int32_t>();
    Parameters par;
    const char* pp = r.take(sizeof(Parameters));
    if (!r.ok || np <= 0 || npb < 0 || npm < 0 || npb + npm != np)
        return lqb::set_error(LQ_ERR_IO, "%s: truncated or inconsistent checkpoint header", path);
    memcpy(&par, pp, sizeof(par));
    if (par.np != np || par.npb != npb || par.npm != npm)
        return lqb::set_error(LQ_ERR_IO, "%s: particle counts disagree with its Parameters", path);
    if ((saved_flags & LQ_SIM_MIXED) != ((uint32_t)flags & LQ_SIM_MIXED))
        return lqb::set_error(LQ_ERR_ARG, "%s was written by the %s form; load it with the same LQ_SIM_MIXED flag",
                              path, (saved_flags & LQ_SIM_MIXED) ? "mixed-precision" : "plain FP32");
    const uint32_t ext = LQ_SIM_DENSITY_FILTER | LQ_SIM_DYNAMIC_DT;
    if ((saved_flags & ext) != ((uint32_t)flags & ext))
        return lqb::set_error(LQ_ERR_ARG, "%s: load it with the LQ_SIM_DENSITY_FILTER / LQ_SIM_DYNAMIC_DT flags it "
                              "was saved with (%u)", path, saved_flags & ext);
    const size_t n = (size_t)np;
    const float* arr[5];
    const size_t width[5] = {4, 4, 4, 6, 6};
    for (int k = 0; k < 5; ++k) arr[k] = reinterpret_cast<const float*>(r.take(width[k] * n * sizeof(float)));
    const char* xd = nullptr;
    const char* vd = nullptr;
    if (saved_flags & LQ_SIM_MIXED) {
        xd = r.take(n * sizeof(double4));
        vd = r.take(n * sizeof(double4));
    }
    std::vector<float> mt, vw;
    std::vector<int> fr;
    const int nmt = r.val<int32_t>();
    if (r.ok && nmt > 0)
        if (const char* p = r.take(5 * (size_t)nmt * sizeof(float)))
            mt.assign(reinterpret_cast<const float*>(p), reinterpret_cast<const float*>(p) + 5 * (size_t)nmt);
    const int nvw = r.val<int32_t>();
    if (r.ok && nvw > 0)
        if (const char* p = r.take(10 * (size_t)nvw * sizeof(float)))
            vw.assign(reinterpret_cast<const float*>(p), reinterpret_cast<const float*>(p) + 10 * (size_t)nvw);
    const int nfr = r.val<int32_t>();
    if (r.ok && nfr > 0)
        if (const char* p = r.take(2 * (size_t)nfr * sizeof(int)))
            fr.assign(reinterpret_cast<const int*>(p), reinterpret_cast<const int*>(p) + 2 * (size_t)nfr);
    const float wide = (r.ok && buf.size() - r.at == sizeof(float)) ? r.val<float>() : 0.0f;
    if (!r.ok || nmt < 0 || nvw < 0 || nfr < 0 || r.at != buf.size() || !(wide >= 0.0f))
        return lqb::set_error(LQ_ERR_IO, "%s: truncated or malformed checkpoint", path);

    /* aligned copies of the state arrays (the file offsets are not) */
    std::vector<float> a[5];
    for (int k = 0; k < 5; ++k) a[k].assign(arr[k], arr[k] + width[k] * n);
    void* out = nullptr;
    LQ_TRY(lq_sim_create(&par, a[0].data(), a[1].data(), a[2].data(), a[3].data(), a[4].data(), flags, &out));
    LqSim* S = static_cast<LqSim*>(out);
    auto fail = [&](int st) {
        lq_sim_destroy(out);
        return st;
    };
    if (xd) {
        /* low words: what the FP64 values leave beyond the float state */
        std::vector<double> hx(4 * n), hv(4 * n);
        memcpy(hx.data(), xd, n * sizeof(double4));
        memcpy(hv.data(), vd, n * sizeof(double4));
        std::vector<float> xl(4 * n), vl(4 * n);
        for (size_t k = 0; k < 4 * n; ++k) {
            xl[k] = (k % 4 == 3) ? 0.0f : (float)(hx[k] - (double)a[0][k]);
            vl[k] = (float)(hv[k] - (double)a[1][k]);
        }
        cudaError_t e = cudaMemcpyAsync(S->S.xlo, xl.data(), n * sizeof(float4), cudaMemcpyHostToDevice, S->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(S->S.vlo, vl.data(), n * sizeof(float4), cudaMemcpyHostToDevice, S->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(S->stream);
        if (e != cudaSuccess)
            return fail(lqb::set_error(LQ_ERR_CUDA, "checkpoint FP64 state: %s", cudaGetErrorString(e)));
    }
    S->step = step;
    S->time = time;
    S->ph.time = (float)time;
    if (flags & LQ_SIM_DYNAMIC_DT) {
        /* the saved next-step dt (create set the fixed one) and the time */
        cudaError_t e = cudaMemcpyAsync(&S->pd->dt, &par.dt, sizeof(float), cudaMemcpyHostToDevice, S->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(S->dtime, &S->time, sizeof(double), cudaMemcpyHostToDevice, S->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(S->stream);
        if (e != cudaSuccess)
            return fail(lqb::set_error(LQ_ERR_CUDA, "checkpoint dt: %s", cudaGetErrorString(e)));
    }
    int st = LQ_OK;
    if (st == LQ_OK && nmt > 0) st = lq_sim_set_materials(out, nmt, mt.data());
    if (st == LQ_OK && nvw > 0) st = lq_sim_set_hypoplastic(out, nvw, vw.data());
    if (st == LQ_OK && nfr > 0) st = lq_sim_set_frames(out, nfr, fr.data());
    if (st == LQ_OK && (skin != S->skin || wide > skin)) {
        S->skin = skin;            /* as saved, not through skin / h */
        if (wide > skin) st = ensure_wide_lists(S);
        S->wide = wide;
        if (st == LQ_OK) st = build_graphs(S);
    }
    if (st != LQ_OK) return fail(st);
    *sim = out;
    return LQ_OK;
}

extern "C" int lq_sim_neighbor_entries(void* sim, long long* material, long long* boundary)
{
    if (!sim || !material || !boundary) return lqb::set_error(LQ_ERR_ARG, "lq_sim_neighbor_entries: null argument");
    LqSim* S = static_cast<LqSim*>(sim);
    LQ_TRY_CUDA(cudaStreamSynchronize(S->stream), "neighbor entries");
    auto total = [](const int* d, int n, long long* out) -> int {
        std::vector<int> h((size_t)(n > 0 ? n : 0));
        if (n > 0) LQ_TRY_CUDA(cudaMemcpy(h.data(), d, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost), "counts");
        long long t = 0;
        for (int c : h) t += c < LQ_NBR_CAP ? c : LQ_NBR_CAP;
        *out = t;
        return LQ_OK;
    };
    LQ_TRY(total(S->nlm.count, S->npm, material));
    LQ_TRY(total(S->nlb.count, S->npb, boundary));
    return LQ_OK;
}

extern "C" int lq_sim_rebuild_launches(void* sim, int* launches)
{
    if (!sim || !launches) return lqb::set_error(LQ_ERR_ARG, "lq_sim_rebuild_launches: null argument");
    LqSim* S = static_cast<LqSim*>(sim);
    /* count reset, hash, scatter, cell order (the scan is a library
     * kernel), gather, copy, material list, boundary list (when npb > 0),
     * full pack of the neighbour data, tile segments and fill (tiled
     * shapes; their scan is a library kernel) */
    *launches = 4 + 1 + 1 + 1 + (S->npb > 0 ? 1 : 0) + 1 + (tiled(S) && S->npm > 0 ? 2 : 0);
    /* with two-level lists the lists the stages read are renewed from the
     * wide ones right after */
    int renewal = 0;
    LQ_TRY(lq_sim_renewal_launches(sim, &renewal));
    *launches += renewal;
    return LQ_OK;
}

extern "C" int lq_sim_renewal_launches(void* sim, int* launches)
{
    if (!sim || !launches) return lqb::set_error(LQ_ERR_ARG, "lq_sim_renewal_launches: null argument");
    LqSim* S = static_cast<LqSim*>(sim);
    /* material and boundary (when npb > 0) list renewal, positions record */
    *launches = two_level(S) ? (S->npm > 0 ? 1 : 0) + (S->npb > 0 ? 1 : 0) + 1 : 0;
    return LQ_OK;
}

/* ------------------------------------------------------------ profiling */

namespace {

/* Phases timed by lq_sim_profile: the reference's Timer phases
 * (reference include/types.h:158-173, src/loquat.cu:345-395) with the
 * search and the list build split out. */
enum { PH_SEARCH = 0, PH_GATHER, PH_ADAMI, PH_INTERACTION, PH_INTEGRATE, PH_SHEPARD, PH_LIST, PH_RENEW, PH_COUNT };
/* NVTX range names of the phases (host ranges around each phase's
 * launches; a tool such as ncu can select kernels by them with
 * --nvtx --nvtx-include "lq/interaction/") */
const char* const kPhaseNames[PH_COUNT] = {"lq/search", "lq/gather", "lq/adami", "lq/interaction",
                                           "lq/integrate", "lq/shepard", "lq/list", "lq/renew"};

struct PhaseTimer {
    std::vector<cudaEvent_t> ev;
    std::vector<int> phase;
    int used = 0;
    int mark(cudaStream_t s, int ph)
    {
        if (used + 2 > (int)ev.size()) return lqb::set_error(LQ_ERR_ARG, "profile: event pool exhausted");
        phase.push_back(ph);
        nvtxRangePushA(kPhaseNames[ph]);
        LQ_TRY_CUDA(cudaEventRecord(ev[used], s), "profile event");
        used += 1;
        return LQ_OK;
    }
    int close(cudaStream_t s)
    {
        nvtxRangePop();
        LQ_TRY_CUDA(cudaEventRecord(ev[used], s), "profile event");
        used += 1;
        return LQ_OK;
    }
};

int profiled_step(LqSim* S, PhaseTimer& T)
{
    const Parameters* ph = &S->ph;
    const Parameters* pd = S->pd;
    cudaStream_t s = S->stream;
    bool rebuild = false, renew = false;
    LQ_TRY(host_take_flag(S, &rebuild, &renew));
    if (rebuild) {
        LQ_TRY(T.mark(s, PH_SEARCH));
        LQ_TRY(lqb::grid_search(ph, pd, S->S.pos, S->g, false, S->health, s, S->S.idep, S->fr));
        LQ_TRY(T.close(s));
        LQ_TRY(T.mark(s, PH_GATHER));
        LQ_TRY(lqb::gather_state(S->np, S->g.part_idx, S->S, S->T, s));
        k_copy_state<<<blocks(S->np), 256, 0, s>>>(S->np, S->npb, S->T, S->S, S->S2,
                                                   two_level(S) ? S->xwide : S->xbuild);
        LQ_TRY_CUDA(cudaGetLastError(), "k_copy_state");
        LQ_TRY(T.close(s));
        LQ_TRY(T.mark(s, PH_LIST));
        LQ_TRY(build_lists(S, s));
        LQ_TRY(lqb::launch_pack_neighbors(ph, S->S, S->rec, 0, s, S->flags & LQ_SIM_MIXED));
        LQ_TRY(lqb::launch_tile_order(ph, S->g.start, S->pair_shape, S->tile, s));
        LQ_TRY(T.close(s));
    }
    if (renew) {
        LQ_TRY(T.mark(s, PH_RENEW));
        LQ_TRY(enqueue_renewal(S, s));
        LQ_TRY(T.close(s));
    }
    State* cur[2] = {&S->S, &S->S2};
    for (int stage = 0; stage < 2; ++stage) {
        LQ_TRY(T.mark(s, PH_ADAMI));
        LQ_TRY(enqueue_adami_pack(S, *cur[stage], s));
        LQ_TRY(T.close(s));
        LQ_TRY(T.mark(s, PH_INTERACTION));
        LQ_TRY(enqueue_interaction(S, *cur[stage], s));
        LQ_TRY(T.close(s));
        LQ_TRY(T.mark(s, PH_INTEGRATE));
        if (stage == 0)
            LQ_TRY(lqb::launch_predict(ph, pd, S->S, S->S2, nullptr, S->R, s, S->mt, S->vw, S->rec, true));
        else {
            LQ_TRY(lqb::launch_correct_into(ph, pd, S->S2, S->S, S->S, S->R, S->health, S->xbuild, S->rebuild,
                                            S->skin, s, S->mt, S->vw, two_level(S) ? S->xwide : nullptr,
                                            S->wide, S->rec));
            LQ_TRY(enqueue_dynamic_dt(S, s));
        }
        LQ_TRY(T.close(s));
    }
    return LQ_OK;
}

}  // namespace

extern "C" int lq_sim_profile(void* sim, int nsteps, double* phase_ms, int* phase_launches)
{
    if (!sim || nsteps < 0 || !phase_ms) return lqb::set_error(LQ_ERR_ARG, "lq_sim_profile: bad argument");
    LqSim* S = static_cast<LqSim*>(sim);
    PhaseTimer T;
    T.ev.resize((size_t)nsteps * 2 * (4 + 6 + 2) + 4);   /* rebuild and renewal, two stages, filters */
    for (auto& e : T.ev) LQ_TRY_CUDA(cudaEventCreate(&e), "profile event create");
    int st = LQ_OK;
    const int N = S->ph.stress_shepard_filter;
    for (int k = 0; k < nsteps && st == LQ_OK; ++k) {
        S->ph.time = (float)S->time;
        st = profiled_step(S, T);
        if (st == LQ_OK && N != 0 && S->step % N == 0 && S->step != 0) {
            st = T.mark(S->stream, PH_SHEPARD);
            if (st == LQ_OK) st = enqueue_shepard(S, S->stream);
            if (st == LQ_OK) st = T.close(S->stream);
        }
        const int Nd = S->ph.density_shepard_filter;
        if (st == LQ_OK && (S->flags & LQ_SIM_DENSITY_FILTER) && Nd > 0 && S->step % Nd == 0 && S->step != 0) {
            st = T.mark(S->stream, PH_SHEPARD);
            if (st == LQ_OK) st = enqueue_density_filter(S, S->stream);
            if (st == LQ_OK) st = T.close(S->stream);
        }
        S->time += (double)S->ph.dt;
        S->step++;
    }
    if (st == LQ_OK) {
        cudaError_t e = cudaStreamSynchronize(S->stream);
        if (e != cudaSuccess) st = lqb::cuda_status(e, "profile synchronize");
    }
    for (int p = 0; p < PH_COUNT; ++p) {
        phase_ms[p] = 0.0;
        if (phase_launches) phase_launches[p] = 0;
    }
    if (st == LQ_OK) {
        for (size_t k = 0; k < T.phase.size(); ++k) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, T.ev[2 * k], T.ev[2 * k + 1]);
            phase_ms[T.phase[k]] += ms;
            if (phase_launches) phase_launches[T.phase[k]] += 1;
        }
    }
    for (auto& e : T.ev) cudaEventDestroy(e);
    return st;
}
