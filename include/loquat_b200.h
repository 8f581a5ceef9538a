/*
 * LOQUAT-B200 C ABI.
 *
 * Plain C entry points over the sm_100a kernels of the per-step SPH path.
 * Every function returns an int status (LQ_OK = 0); lq_last_error() gives the
 * message of the last failure on the calling thread.  No function exits the
 * process.  The C++ drop-in surface (loquat_grid.h, particle_interaction.h,
 * predictor_corrector.h, adami_boundary.h, field_smoothing.h) is a thin layer
 * over these calls that keeps the reference's print-and-exit behaviour.
 *
 * Conventions
 *   par            pointer to a 208-byte Parameters record (types.h); "host"
 *                  means host memory, "device" means device memory.
 *   float4 arrays  float[np][4]  (pospres, velrhop, idep, accad, spin)
 *   tensor2d arrays float[np][6] (str, stn, acestn), order xx yy zz xy xz yz
 *   stream         a cudaStream_t; NULL is the legacy default stream, which
 *                  is what the reference uses for every launch.
 *   Device arrays are caller-owned unless stated otherwise.
 */
#ifndef LOQUAT_B200_C_ABI_H
#define LOQUAT_B200_C_ABI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LQ_OK            0
#define LQ_ERR_ARG       1   /* bad argument (null pointer, size, layout)     */
#define LQ_ERR_CUDA      2   /* CUDA runtime error                            */
#define LQ_ERR_ALLOC     3   /* device or host allocation failed              */
#define LQ_ERR_IO        4   /* file missing, malformed or truncated          */
#define LQ_ERR_STATE     5   /* simulation health check failed                */
#define LQ_ERR_NOTFOUND  6   /* required XML key absent                       */

#define LQ_ABI_VERSION   1

/* ---- library ------------------------------------------------------------ */
int         lq_abi_version(void);
size_t      lq_parameters_size(void);            /* == sizeof(Parameters) = 208 */
const char* lq_last_error(void);
const char* lq_status_string(int status);

/* Derived constants: h, 1/h, eta, m, cell counts, layer size, Wendland C2
 * constants, W(0), W(dr).  Replaces LoquatSph::InitializeParameters
 * (reference src/loquat.cu:111-139), same float arithmetic. */
int lq_initialize_parameters(void* par_host);

/* dt = cfl * h / cs (reference src/loquat.cu:325-333; dynamic dt is not
 * implemented there either). Writes par_host->dt. */
int lq_update_time_step(void* par_host);

/* ---- neighbour grid (replaces LoquatGrid, reference src/loquat_grid.h:28-66) */
/* Allocates the grid arrays for np particles and ncell cells
 * (GridConfig, ResizeArrayLength). */
int lq_grid_create(int np, int ncell, void** grid);
int lq_grid_resize(void* grid, int np, int ncell);
int lq_grid_destroy(void* grid);
/* Hash, stable sort and cell bounds (LoquatGrid::NeighborSearch,
 * reference src/loquat_grid.h:60).  pospres/idep: device float4[np].  The
 * stable order within a cell is restored by one thread per cell, in one
 * read-only pass when the cell arrives in order (as it does when particles
 * move little between searches) and by insertion otherwise: particles
 * outside the lattice share one cell, so keep their number small. */
int lq_grid_neighbor_search(void* grid, const void* par_host, const void* par_device,
                            const float* pospres, const float* idep, void* stream);
/* Device pointers owned by the grid.  cell_start has ncell + 1 entries:
 * the particles of cell c are the sorted slots [cell_start[c], cell_start[c+1]). */
int lq_grid_arrays(void* grid, const int** part_cel, const int** part_idx,
                   const int** cell_beg, const int** cell_end, const int** cell_start);
/* data[i] <- data[part_idx[i]] through cache (LoquatGrid::SortArrayFloat4 /
 * SortArrayTensor2d, reference src/loquat_grid.h:62-64). */
int lq_grid_sort_float4(void* grid, int np, float* data, float* cache, void* stream);
int lq_grid_sort_tensor2d(void* grid, int np, float* data, float* cache, void* stream);

/* Neighbour search that allocates nothing; this entry point has no
 * counterpart in the reference.  It is for callers that cannot allocate
 * device memory themselves (a host code whose memory pool already holds
 * the GPU's memory, a step loop that cannot take cudaMalloc's device-wide
 * synchronisation).  Same result as lq_grid_neighbor_search, but the
 * caller passes the outputs (part_cel, part_idx: int[np]; cell_beg,
 * cell_end: int[ncell]) and the working arrays live in one fixed 17 MiB
 * device array inside the library, held on every device that loads it
 * until exit.  Limits: np <= LQ_NOALLOC_MAX_PARTICLES, ncell <=
 * LQ_NOALLOC_MAX_CELLS, else LQ_ERR_ARG.  All calls on a device share that
 * array: calls that overlap on the GPU race.  Each call made outside
 * stream capture looks up the array's device address (with that device
 * current, so a module reloaded after cudaDeviceReset is found again);
 * calls during a capture reuse the last address, so make one call on the
 * device before any capture begins (a first call inside a capture returns
 * LQ_ERR_ARG).  Particles outside the lattice share one cell, ordered by
 * a single thread: keep their number small. */
#define LQ_NOALLOC_MAX_PARTICLES 1048576
#define LQ_NOALLOC_MAX_CELLS     1048575
int lq_grid_neighbor_search_noalloc(const void* par_host, const void* par_device, const float* pospres,
                                    int* part_cel, int* part_idx, int* cell_beg, int* cell_end, void* stream);

/* ---- per-stage operators ------------------------------------------------ */
/* Sizes the working arrays of lq_particle_interaction on the current device
 * (cell starts, target order, neighbour lists, packed neighbour data) for
 * the particle and cell counts of par_host.  No counterpart in the
 * reference, whose ParticleInteraction is closed; it plays the part of the
 * reference's set-up allocation (src/loquat.cu:142-165) for this
 * operator: the drop-in LoquatGrid::GridConfig calls it, and a C caller
 * makes it once before its step loop, after which a call with the same or
 * smaller counts allocates nothing (a larger one grows the arrays,
 * synchronising the device first). */
int lq_interaction_reserve(const void* par_host);

/* How often lq_particle_interaction on the current device built its
 * neighbour lists afresh and how often it carried them over from an
 * earlier call.  No counterpart in the reference.  Lists are carried when
 * the cell_beg passed belongs to a grid of this library (lq_grid_* or the
 * drop-in LoquatGrid), whose searches track each particle's identity,
 * the caller has re-sorted its arrays after each search (as the reference
 * does), and no particle has moved half a skin of 0.05 h since the build;
 * the grid's searches and the interaction must run on one stream. */
int lq_interaction_stats(long long* rebuilds, long long* reuses);

/* reference src/particle_interaction.h:27-40 */
int lq_particle_interaction(const void* par_host, const void* par_device,
                            const float* pospres, const float* velrhop, const float* idep,
                            const float* str, const float* stn,
                            float* accad, float* spin, float* acestn,
                            const int* cell_beg, const int* cell_end, void* stream);

/* reference src/adami_boundary.h:27-34 */
int lq_adami_boundary(const void* par_host, const void* par_device,
                      const float* pospres, const float* velrhop, float* str,
                      const int* cell_beg, const int* cell_end, void* stream);

/* reference src/field_smoothing.h:27-35 */
int lq_stress_regularization(const void* par_host, const void* par_device,
                             const float* pospres, const float* velrhop, float* str,
                             float* tensor2d_cache,
                             const int* cell_beg, const int* cell_end, void* stream);

/* reference src/predictor_corrector.h:30-48 */
int lq_predictor(const void* par_host, const void* par_device,
                 float* pospres, float* velrhop, float* idep, float* str, float* stn,
                 float* pospres_ini, float* velrhop_ini, float* idep_ini,
                 float* str_ini, float* stn_ini,
                 const float* accad, const float* spin, const float* acestn, void* stream);

/* reference src/predictor_corrector.h:51-67 */
int lq_corrector(const void* par_host, const void* par_device,
                 float* pospres, float* velrhop, float* idep, float* str, float* stn,
                 const float* pospres_ini, const float* velrhop_ini, const float* idep_ini,
                 const float* str_ini, const float* stn_ini,
                 const float* accad, const float* spin, const float* acestn, void* stream);

/* ---- whole-step driver (the hot loop of LoquatSph::RunSimulation,
 *      reference src/loquat.cu:322-409) ------------------------------------ */
#define LQ_SIM_GRAPH   1   /* replay each step as one captured CUDA graph      */
#define LQ_SIM_MIXED   2   /* mixed precision: FP64 position, velocity and
                              density accumulation and FP64 stress updates in
                              the integrator, compensated sums in the
                              interaction; the neighbour kernels read FP32 */
/* Features the reference reads from its parameter file but never applies
 * (density-shepard-filter, src/loquat_io.cu:180; dynamic-time-step,
 * src/loquat.cu:325-333).  Off unless asked for here, so a case behaves as
 * in the reference whatever its file says. */
#define LQ_SIM_DENSITY_FILTER 4  /* every density_shepard_filter steps (> 0),
                                    after the stress filter: rho_i =
                                    sum m W / sum (m/rho_j) W over the material
                                    layer, self included */
#define LQ_SIM_DYNAMIC_DT     8  /* after each step, dt = cfl min(h / (cs +
                                    v_max), sqrt(h / a_max)) over the material
                                    particles (never above cfl h / cs); the
                                    time then lives on the device and
                                    lq_sim_clock synchronises to read it */

/* Creates a simulation from host arrays (np = par->np particles, boundary
 * first).  par must have been through lq_initialize_parameters.  The state
 * is uploaded, sorted once (reference src/loquat.cu:297-298) and kept on
 * the device. */
int lq_sim_create(const void* par_host,
                  const float* pospres, const float* velrhop, const float* idep,
                  const float* str, const float* stn, int flags, void** sim);
int lq_sim_destroy(void* sim);
/* Advances nsteps time steps, queued on the simulation's stream. */
int lq_sim_step(void* sim, int nsteps);
int lq_sim_synchronize(void* sim);
int lq_sim_stream(void* sim, void** stream);
/* Host <-> device copies of the whole state, in the current sorted order. */
int lq_sim_upload(void* sim, const float* pospres, const float* velrhop, const float* idep,
                  const float* str, const float* stn);
int lq_sim_download(void* sim, float* pospres, float* velrhop, float* idep,
                    float* str, float* stn);
/* Device pointers of the current state (valid until the next lq_sim_step). */
int lq_sim_state(void* sim, float** pospres, float** velrhop, float** idep,
                 float** str, float** stn);
/* Step counter and simulated time. */
int lq_sim_clock(void* sim, long long* step, double* time);
/* Health word, counted since the last read: [0] non-finite material values,
 * [1] material and [2] boundary particles found outside the cell lattice by
 * a search, [3] particles with more than 192 neighbours within 2h + skin.
 * Reading it synchronises the stream and clears it. */
int lq_sim_health(void* sim, int* health4);
/* Neighbour lists are kept across steps and rebuilt (search, sort, list
 * build) only when a particle's displacement since the last build plus a
 * bound on its next step's motion reaches half the skin; the lists hold
 * every pair within 2h + skin.  Default skin 0.05 h; setting it forces a
 * rebuild before the next step.  lq_sim_rebuilds counts rebuilds so far. */
int lq_sim_set_skin(void* sim, float skin_over_h);
int lq_sim_rebuilds(void* sim, long long* count);
/* Two-level lists: with wide_over_h above the skin, a rebuild builds wider
 * lists (every pair within 2h + wide) and the lists the stages read are
 * renewed from them at the current positions, without a search, whenever
 * the skin runs out; the search and sort wait until a particle has moved
 * (wide - skin) / 2 from its position at the wide build.  0 (the default)
 * or a value not above the skin gives one-level lists.  Forces a rebuild
 * before the next step; the first call allocates the wide lists.
 * lq_sim_wide_skin reads the setting in effect (0 for one level),
 * lq_sim_renewals counts renewals without a search so far.  No reference
 * counterpart. */
int lq_sim_set_wide_skin(void* sim, float wide_over_h);
int lq_sim_wide_skin(void* sim, float* wide_over_h);
int lq_sim_renewals(void* sim, long long* count);
/* Per-object materials, for many independent scenarios in one simulation
 * (each scenario's particles placed farther than 2h from the others):
 * a material particle uses row (int)idep.x of the n x 5 host table (the
 * five model parameters of Parameters.model_par_1..5; the constitutive
 * model itself stays global).  Rows out of range are clamped.  n = 0
 * returns to the global parameters.  No reference counterpart: the
 * reference runs one scenario per process. */
int lq_sim_set_materials(void* sim, int n, const float* table);
/* Constitutive model 3 (von Wolffersdorff hypoplasticity with a limit-state
 * surface, integrated in FP64 with adaptive explicit sub-steps; no reference
 * counterpart).  table is n x 10 floats per object id (row (int)idep.x,
 * clamped): phi_c in degrees, h_s in Pa, n, e_d0, e_c0, e_i0, alpha, beta,
 * the relative sub-step tolerance and the maximum number of sub-steps.  The
 * void ratio of each particle lives in idep.z.  Required before the first
 * step when Parameters.constitutive_model is 3; rows are checked
 * (0 < phi_c < 90, 0 < e_d0 < e_c0 < e_i0, ...). */
int lq_sim_set_hypoplastic(void* sim, int n, const float* table);
/* Per-object grid frames, for the same use: each object keeps local
 * coordinates and owns a block of grid rows in y.  rows is n x 2 ints,
 * (first row, number of rows) for object ids 0..n-1; a particle's local y
 * cell c maps to grid row first + c, and c outside [0, rows) counts as
 * outside the lattice.  Blocks of objects that must not interact need at
 * least one empty row between them.  Forces a search before the next step.
 * No reference counterpart. */
int lq_sim_set_frames(void* sim, int n, const int* rows);
/* Own kernel launches of a step without a rebuild (plain) and of a step
 * with the Shepard pass; a rebuild adds lq_sim_rebuild_launches more (the
 * renewal that follows it with two-level lists included) and a renewal
 * without a search lq_sim_renewal_launches. */
int lq_sim_launches_per_step(void* sim, int* plain, int* with_shepard);
int lq_sim_rebuild_launches(void* sim, int* launches);
int lq_sim_renewal_launches(void* sim, int* launches);
/* Launch shape of the pair kernel.  0-4: one thread per target in slot
 * order, threads per block x resident blocks per SM (which caps its
 * registers): 0 = 128 x 6, 1 = 64 x 12, 2 = 256 x 3, 3 = 128 x 5,
 * 4 = 128 x 7.  7-10: one thread per target in tile order (the targets of a
 * block form a compact box of cells, so its neighbours stay in L1; the
 * order is rebuilt after every search): 7 = 768 x 1, 8 = 384 x 2,
 * 9 = 640 x 1, 10 = 320 x 2.  All of these give bit-identical results.
 * 5, 6: warp-cooperative, 8 or 32 lanes share a target's list and combine
 * their sums with shuffle reductions (for small cases); the summation
 * order differs, so results agree to rounding.  A new simulation starts
 * with shape 9 when its material particles fill four waves of 640-thread
 * blocks on every SM, else with shape 0.  No reference counterpart. */
int lq_sim_set_pair_shape(void* sim, int shape);
int lq_sim_pair_shape(void* sim, int* shape);
/* Autotuner: times `steps` steps for each pair kernel shape at the current
 * lists, then for one-level skins of 0.02, 0.05, 0.1 and 0.2 h with the
 * fastest shape, then two-level lists with wide margins of 0.1 and 0.2 h
 * over the fastest skin and over skins of 0.02 and 0.01 h narrower than
 * it; then it times again, over 2 x `steps` at the fastest lists, every
 * shape that came within 5 % of the fastest in the first round (at most
 * four), and keeps the fastest of that round (the wide setting is
 * read with lq_sim_wide_skin).  Every trial starts from a device copy of
 * the state taken at the call and its window opens with the search and
 * list build that start every run, so settings whose lists last long pay
 * for one build per window.  The state, step, time and health word are put
 * back afterwards, so tuning does not advance the simulation (it rebuilds
 * its lists before the next step).  Allocates the state copy for the
 * duration of the call. */
int lq_sim_autotune(void* sim, int steps, int* shape, float* skin_over_h);
/* Bounds violations counted so far in this process by a library built with
 * -D LQ_CHECKED (loquat_b200/liblqb200_checked.so): its list and grid
 * kernels check every index they gather or scatter through and skip and
 * count a bad one instead of accessing memory.  -1 from the product
 * library, which has no checks.  Synchronises the device. */
int lq_debug_bounds_violations(long long* count);
/* Checkpoints of a simulation: the state (with the FP64 copies of the
 * mixed form), step, time, skin and the per-object tables, in a binary file
 * of this library's own format.  Saving forces a neighbour search before the
 * simulation's next step, so a simulation loaded from the file with the same
 * precision form and the run that continues take bit-identical steps.
 * lq_sim_load_checkpoint creates the simulation (flags as for
 * lq_sim_create; every flag but LQ_SIM_GRAPH must match the saved run's).  The reference
 * restarts from its output XML and particle file instead, which round to
 * float text and drop the void ratio. */
int lq_sim_save_checkpoint(void* sim, const char* path);
int lq_sim_load_checkpoint(const char* path, int flags, void** sim);
/* Entries in the current neighbour lists of material and of boundary
 * particles (pairs within 2h + skin at the last build), for work
 * accounting; synchronises the simulation's stream. */
int lq_sim_neighbor_entries(void* sim, long long* material, long long* boundary);
/* Advances nsteps steps launching kernels one by one with CUDA events
 * around each phase, then synchronises and returns the summed device time
 * per phase in phase_ms[8]: search, gather, Adami, interaction pairs,
 * integrate, Shepard, neighbour-list build, renewal of two-level lists
 * (the phases of the reference's Timer, include/types.h:158-173, timed on
 * the device instead of with std::clock, with the search and the list
 * build and renewal split out).  phase_launches[8] (may be NULL) receives
 * how many times each phase ran. */
int lq_sim_profile(void* sim, int nsteps, double* phase_ms, int* phase_launches);

/* ---- XML / .dat formats (reference src/loquat_io.cu:69-370) ------------ */
int lq_io_load_parameters(const char* xml_path, void* par_host);
int lq_io_save_parameters(const char* xml_path, const void* par_host);
/* Constitutive model 3 in the parameter file (extension keys with no
 * reference counterpart): vw-phi-c, vw-hs, vw-n, vw-ed0, vw-ec0, vw-ei0,
 * vw-alpha, vw-beta, vw-tolerance (float), vw-max-substeps (int) and
 * vw-initial-void-ratio (float, for soil particles whose idep.z is 0; the
 * 22-column particle file does not carry idep.z).  vw_row receives the
 * 10-float row of lq_sim_set_hypoplastic. */
int lq_io_load_hypoplastic(const char* xml_path, float* vw_row, float* e0);
int lq_io_save_parameters_vw(const char* xml_path, const void* par_host, const float* vw_row, float e0);
int lq_io_load_particles(const char* dat_path, int np,
                         float* pospres, float* velrhop, float* idep, float* str, float* stn);
int lq_io_save_particles(const char* dat_path, int np,
                         const float* pospres, const float* velrhop, const float* idep,
                         const float* str, const float* stn);
/* ParaView output (reference src/loquat_io.cu:372-548): one ASCII .vtu
 * file per object id, <dir>/<id>_<output_number>.vtu. */
int lq_io_save_vtu(const char* dir, int output_number, int np,
                   const float* pospres, const float* velrhop, const float* idep,
                   const float* str, const float* stn);

#ifdef __cplusplus
}
#endif

#endif /* LOQUAT_B200_C_ABI_H */
