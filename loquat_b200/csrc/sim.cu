/*
 * LOQUAT-B200 native time-step driver: the hot loop of
 * LoquatSph::RunSimulation (reference src/loquat.cu:322-409) with the same
 * stage order, re-planned for one B200:
 *
 *   reference (per step)                      here
 *   search + 5 gathers (+copy back each)      search + 1 fused 5-array gather
 *   Adami, interaction                        Adami, interaction
 *   5 snapshot copies + predictor             predictor A -> B (A is the snapshot)
 *   search + 10 gathers (+copy back each)     search + 1 fused 5-array gather B -> C
 *   Adami, interaction                        Adami, interaction
 *   corrector (snapshot re-sorted)            corrector in place on C, reading the
 *                                             snapshot A through the new permutation
 *   every N steps: search + 5 gathers +       every N steps: search + gather C -> A,
 *   Shepard + copy back                       Shepard A -> C
 *   per-step H2D Parameters + 8 host syncs    one CUDA graph launch per step, no sync
 *
 * Buffer roles are fixed (the state is in C at every step boundary), so a
 * step and a Shepard pass are each captured once as a CUDA graph and
 * replayed.  dt = cfl h / cs is constant, as in the reference.
 */
#include <cstring>
#include <vector>

#include "lq_internal.cuh"

namespace {

using lqb::State;

struct LqSim {
    Parameters ph{};
    Parameters* pd = nullptr;
    int np = 0, npb = 0, npm = 0;
    long long step = 0;
    double time = 0.0;
    int flags = 0;
    cudaStream_t stream = nullptr;
    State A{}, B{}, C{};
    lqb::Rates R{};
    lqb::GridBuffers g;
    int* health = nullptr;
    std::vector<void*> allocs;
    cudaGraphExec_t step_exec = nullptr;
    cudaGraphExec_t shep_exec = nullptr;
};

int dev_alloc(LqSim* S, void** p, size_t bytes)
{
    cudaError_t e = cudaMalloc(p, bytes > 0 ? bytes : 16);
    if (e != cudaSuccess) return lqb::set_error(LQ_ERR_ALLOC, "sim: cudaMalloc(%zu) failed: %s", bytes,
                                                cudaGetErrorString(e));
    S->allocs.push_back(*p);
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
    return LQ_OK;
}

void release(LqSim* S)
{
    if (S->step_exec) cudaGraphExecDestroy(S->step_exec);
    if (S->shep_exec) cudaGraphExecDestroy(S->shep_exec);
    if (S->stream) cudaStreamSynchronize(S->stream);
    for (void* p : S->allocs) cudaFree(p);
    S->allocs.clear();
    if (S->stream) cudaStreamDestroy(S->stream);
    S->stream = nullptr;
}

/* One time step; the state is in C before and after. */
int enqueue_step(LqSim* S)
{
    const Parameters* ph = &S->ph;
    const Parameters* pd = S->pd;
    cudaStream_t s = S->stream;
    const lqb::Cells cells{S->g.start, nullptr, nullptr};
    /* predictor stage (reference src/loquat.cu:343-368) */
    LQ_TRY(lqb::grid_search(ph, pd, S->C.pos, S->g, false, S->health, s));
    LQ_TRY(lqb::gather_state(S->np, S->g.part_idx, S->C, S->A, s));
    LQ_TRY(lqb::launch_adami(ph, pd, S->A, cells, s));
    LQ_TRY(lqb::launch_interaction(ph, pd, S->A, S->R, cells, s));
    LQ_TRY(lqb::launch_predict(ph, pd, S->A, S->B, nullptr, S->R, s));
    /* corrector stage (reference src/loquat.cu:371-396) */
    LQ_TRY(lqb::grid_search(ph, pd, S->B.pos, S->g, false, S->health, s));
    LQ_TRY(lqb::gather_state(S->np, S->g.part_idx, S->B, S->C, s));
    LQ_TRY(lqb::launch_adami(ph, pd, S->C, cells, s));
    LQ_TRY(lqb::launch_interaction(ph, pd, S->C, S->R, cells, s));
    LQ_TRY(lqb::launch_correct(ph, pd, S->C, S->A, S->g.part_idx, S->R, S->health, s));
    return LQ_OK;
}

/* Phases timed by lq_sim_profile, the reference's Timer phases
 * (reference include/types.h:158-173, src/loquat.cu:345-395) with the
 * search split from the gathers. */
enum { PH_SEARCH = 0, PH_GATHER, PH_ADAMI, PH_INTERACTION, PH_INTEGRATE, PH_SHEPARD, PH_COUNT };

struct PhaseTimer {
    std::vector<cudaEvent_t> ev;
    std::vector<int> phase;
    int used = 0;
    int mark(cudaStream_t s, int ph)
    {
        if (used + 2 > (int)ev.size()) return lqb::set_error(LQ_ERR_ARG, "profile: event pool exhausted");
        phase.push_back(ph);
        LQ_TRY_CUDA(cudaEventRecord(ev[used], s), "profile event");
        used += 1;
        return LQ_OK;
    }
    int close(cudaStream_t s)
    {
        LQ_TRY_CUDA(cudaEventRecord(ev[used], s), "profile event");
        used += 1;
        return LQ_OK;
    }
};

/* One eager time step with an event pair around every phase. */
int enqueue_step_timed(LqSim* S, PhaseTimer& T)
{
    const Parameters* ph = &S->ph;
    const Parameters* pd = S->pd;
    cudaStream_t s = S->stream;
    const lqb::Cells cells{S->g.start, nullptr, nullptr};
    State* in[2] = {&S->C, &S->B};
    State* out[2] = {&S->A, &S->C};
    for (int stage = 0; stage < 2; ++stage) {
        LQ_TRY(T.mark(s, PH_SEARCH));
        LQ_TRY(lqb::grid_search(ph, pd, in[stage]->pos, S->g, false, S->health, s));
        LQ_TRY(T.close(s));
        LQ_TRY(T.mark(s, PH_GATHER));
        LQ_TRY(lqb::gather_state(S->np, S->g.part_idx, *in[stage], *out[stage], s));
        LQ_TRY(T.close(s));
        LQ_TRY(T.mark(s, PH_ADAMI));
        LQ_TRY(lqb::launch_adami(ph, pd, *out[stage], cells, s));
        LQ_TRY(T.close(s));
        LQ_TRY(T.mark(s, PH_INTERACTION));
        LQ_TRY(lqb::launch_interaction(ph, pd, *out[stage], S->R, cells, s));
        LQ_TRY(T.close(s));
        LQ_TRY(T.mark(s, PH_INTEGRATE));
        if (stage == 0)
            LQ_TRY(lqb::launch_predict(ph, pd, S->A, S->B, nullptr, S->R, s));
        else
            LQ_TRY(lqb::launch_correct(ph, pd, S->C, S->A, S->g.part_idx, S->R, S->health, s));
        LQ_TRY(T.close(s));
    }
    return LQ_OK;
}

/* Shepard stress filter (reference src/loquat.cu:400-409). */
int enqueue_shepard(LqSim* S)
{
    const Parameters* ph = &S->ph;
    const Parameters* pd = S->pd;
    cudaStream_t s = S->stream;
    const lqb::Cells cells{S->g.start, nullptr, nullptr};
    LQ_TRY(lqb::grid_search(ph, pd, S->C.pos, S->g, false, S->health, s));
    LQ_TRY(lqb::gather_state(S->np, S->g.part_idx, S->C, S->A, s));
    LQ_TRY(lqb::launch_shepard(ph, pd, S->A, S->C.str, &S->C, cells, s));
    return LQ_OK;
}

int capture(LqSim* S, int (*fn)(LqSim*), cudaGraphExec_t* exec)
{
    cudaGraph_t graph = nullptr;
    LQ_TRY_CUDA(cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    int st = fn(S);
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

int create(LqSim* S, const Parameters* par, const float* pos, const float* vel, const float* idep, const float* str,
           const float* stn, int flags)
{
    S->ph = *par;
    S->np = par->np;
    S->npb = par->npb;
    S->npm = par->npm;
    S->flags = flags;
    if (S->np <= 0 || S->npb < 0 || S->npm < 0 || S->npb + S->npm != S->np)
        return lqb::set_error(LQ_ERR_ARG, "lq_sim_create: inconsistent counts np=%d npb=%d npm=%d", S->np, S->npb,
                              S->npm);
    if (S->ph.ncell != 2 * S->ph.ncell_one_layer + 1 || S->ph.ncell_one_layer <= 0 || S->ph.h <= 0.0f)
        return lqb::set_error(LQ_ERR_ARG, "lq_sim_create: Parameters not initialised (call lq_initialize_parameters)");
    if (!(S->ph.cs > 0.0f) || !(S->ph.cfl > 0.0f))
        return lqb::set_error(LQ_ERR_ARG, "lq_sim_create: cs and cfl must be positive");
    if (S->ph.constitutive_model != 1 && S->ph.constitutive_model != 2)
        return lqb::set_error(LQ_ERR_ARG, "lq_sim_create: constitutive_model must be 1 or 2");
    S->ph.dt = S->ph.cfl * S->ph.h / S->ph.cs; /* reference src/loquat.cu:333 */
    S->time = (double)S->ph.time;
    LQ_TRY_CUDA(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking), "stream create");
    LQ_TRY(dev_alloc(S, (void**)&S->pd, sizeof(Parameters)));
    LQ_TRY(alloc_state(S, S->A));
    LQ_TRY(alloc_state(S, S->B));
    LQ_TRY(alloc_state(S, S->C));
    const size_t n = (size_t)S->np;
    LQ_TRY(dev_alloc(S, (void**)&S->R.accad, n * sizeof(float4)));
    LQ_TRY(dev_alloc(S, (void**)&S->R.spin, n * sizeof(float4)));
    LQ_TRY(dev_alloc(S, (void**)&S->R.acestn, n * sizeof(tensor2d)));
    LQ_TRY(dev_alloc(S, (void**)&S->health, sizeof(int) * lqb::HEALTH_WORDS));
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
    LQ_TRY_CUDA(cudaMemcpyAsync(S->pd, &S->ph, sizeof(Parameters), cudaMemcpyHostToDevice, S->stream),
                "upload Parameters");
    /* initial search + primary sort (reference src/loquat.cu:297-298) */
    LQ_TRY(upload(S, pos, vel, idep, str, stn, S->A));
    LQ_TRY(lqb::grid_search(&S->ph, S->pd, S->A.pos, S->g, false, S->health, S->stream));
    LQ_TRY(lqb::gather_state(S->np, S->g.part_idx, S->A, S->C, S->stream));
    LQ_TRY_CUDA(cudaStreamSynchronize(S->stream), "sim create");
    if (S->flags & LQ_SIM_GRAPH) {
        LQ_TRY(capture(S, enqueue_step, &S->step_exec));
        LQ_TRY(capture(S, enqueue_shepard, &S->shep_exec));
    }
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
    const int N = S->ph.stress_shepard_filter;
    for (int k = 0; k < nsteps; ++k) {
        S->ph.time = (float)S->time;
        if (S->step_exec) {
            LQ_TRY_CUDA(cudaGraphLaunch(S->step_exec, S->stream), "step graph launch");
        } else {
            LQ_TRY(enqueue_step(S));
        }
        if (N != 0 && S->step % N == 0 && S->step != 0) {
            if (S->shep_exec) {
                LQ_TRY_CUDA(cudaGraphLaunch(S->shep_exec, S->stream), "Shepard graph launch");
            } else {
                LQ_TRY(enqueue_shepard(S));
            }
        }
        S->time += (double)S->ph.dt;
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
    return upload(S, pospres, velrhop, idep, str, stn, S->C);
}

extern "C" int lq_sim_download(void* sim, float* pospres, float* velrhop, float* idep, float* str, float* stn)
{
    if (!sim) return lqb::set_error(LQ_ERR_ARG, "lq_sim_download: null sim");
    LqSim* S = static_cast<LqSim*>(sim);
    const size_t n = (size_t)S->np;
    cudaStream_t s = S->stream;
    if (pospres) LQ_TRY_CUDA(cudaMemcpyAsync(pospres, S->C.pos, n * sizeof(float4), cudaMemcpyDeviceToHost, s), "dl");
    if (velrhop) LQ_TRY_CUDA(cudaMemcpyAsync(velrhop, S->C.vel, n * sizeof(float4), cudaMemcpyDeviceToHost, s), "dl");
    if (idep) LQ_TRY_CUDA(cudaMemcpyAsync(idep, S->C.idep, n * sizeof(float4), cudaMemcpyDeviceToHost, s), "dl");
    if (str) LQ_TRY_CUDA(cudaMemcpyAsync(str, S->C.str, n * sizeof(tensor2d), cudaMemcpyDeviceToHost, s), "dl");
    if (stn) LQ_TRY_CUDA(cudaMemcpyAsync(stn, S->C.stn, n * sizeof(tensor2d), cudaMemcpyDeviceToHost, s), "dl");
    LQ_TRY_CUDA(cudaStreamSynchronize(s), "download");
    return LQ_OK;
}

extern "C" int lq_sim_state(void* sim, float** pospres, float** velrhop, float** idep, float** str, float** stn)
{
    if (!sim) return lqb::set_error(LQ_ERR_ARG, "lq_sim_state: null sim");
    LqSim* S = static_cast<LqSim*>(sim);
    if (pospres) *pospres = (float*)S->C.pos;
    if (velrhop) *velrhop = (float*)S->C.vel;
    if (idep) *idep = (float*)S->C.idep;
    if (str) *str = (float*)S->C.str;
    if (stn) *stn = (float*)S->C.stn;
    return LQ_OK;
}

extern "C" int lq_sim_clock(void* sim, long long* step, double* time)
{
    if (!sim) return lqb::set_error(LQ_ERR_ARG, "lq_sim_clock: null sim");
    LqSim* S = static_cast<LqSim*>(sim);
    if (step) *step = S->step;
    if (time) *time = S->time;
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

extern "C" int lq_sim_launches_per_step(void* sim, int* plain, int* with_shepard)
{
    if (!sim) return lqb::set_error(LQ_ERR_ARG, "lq_sim_launches_per_step: null sim");
    LqSim* S = static_cast<LqSim*>(sim);
    /* own kernels per stage: hash, scatter, cell order, gather, Adami (if
     * npb), interaction, predictor/corrector; the cell scan is a library
     * kernel and is not counted */
    const int per_search = 3;
    const int stage = per_search + 1 + (S->npb > 0 ? 1 : 0) + 1 + 1;
    if (plain) *plain = 2 * stage;
    if (with_shepard) *with_shepard = 2 * stage + per_search + 1 + 1;
    return LQ_OK;
}

extern "C" int lq_sim_profile(void* sim, int nsteps, double* phase_ms, int* phase_launches)
{
    if (!sim || nsteps < 0 || !phase_ms) return lqb::set_error(LQ_ERR_ARG, "lq_sim_profile: bad argument");
    LqSim* S = static_cast<LqSim*>(sim);
    PhaseTimer T;
    const int per_step = 2 * 5 * 2 + 2;
    T.ev.resize((size_t)nsteps * per_step + 4);
    for (auto& e : T.ev) LQ_TRY_CUDA(cudaEventCreate(&e), "profile event create");
    int st = LQ_OK;
    const int N = S->ph.stress_shepard_filter;
    for (int k = 0; k < nsteps && st == LQ_OK; ++k) {
        S->ph.time = (float)S->time;
        st = enqueue_step_timed(S, T);
        if (st == LQ_OK && N != 0 && S->step % N == 0 && S->step != 0) {
            st = T.mark(S->stream, PH_SHEPARD);
            if (st == LQ_OK) st = enqueue_shepard(S);
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
