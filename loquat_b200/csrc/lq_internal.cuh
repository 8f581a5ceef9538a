/*
 * LOQUAT-B200 internal declarations shared by the translation units of the
 * library: array bundles, launch wrappers and error reporting.
 */
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include <types.h>
#include <loquat_b200.h>

namespace lqb {

/* ---------------------------------------------------------------- errors */
int set_error(int status, const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what);

#define LQ_TRY_CUDA(expr, what)                                    \
    do {                                                           \
        cudaError_t lq_e_ = (expr);                                \
        if (lq_e_ != cudaSuccess) return ::lqb::cuda_status(lq_e_, what); \
    } while (0)

#define LQ_TRY(expr)                                               \
    do {                                                           \
        int lq_s_ = (expr);                                        \
        if (lq_s_ != LQ_OK) return lq_s_;                          \
    } while (0)

/* --------------------------------------------------------------- arrays */
/* The five sorted state arrays (reference src/loquat.h:61-66). */
struct State {
    float4* pos;     /* x, y, z, pressure                 */
    float4* vel;     /* vx, vy, vz, density               */
    float4* idep;    /* object id, plastic strain, -, -   */
    tensor2d* str;   /* Cauchy stress, tension positive   */
    tensor2d* stn;   /* total strain                      */
    /* mixed-precision form only: the low words of the position (x, y, z, 0)
     * and of the velocity and density (vx, vy, vz, density).  With the
     * float high words above (the reference's pospres / velrhop, which the
     * neighbour kernels read) they carry the FP64 values the integrator
     * accumulates in, hi + lo to about 48 bits, in half the bytes of FP64
     * copies. */
    float4* xlo = nullptr;
    float4* vlo = nullptr;
};

/* Per-stage rates written by the interaction pass (reference src/loquat.h:74-77). */
struct Rates {
    float4* accad;     /* dv/dt, drho/dt   */
    float4* spin;      /* W_yx, W_zx, W_zy */
    tensor2d* acestn;  /* strain rate      */
};

/* Cell lookup.  With `start` (ncell + 1 entries) the particles of cell c are
 * [start[c], start[c+1]).  Otherwise `beg`/`end` hold the reference's
 * per-cell bounds with -1 for an empty cell. */
struct Cells {
    const int* start;
    const int* beg;
    const int* end;
};

/* Per-object constitutive parameters: when p is set, a material particle
 * uses row (int)idep.x (clamped to [0, n)) of the n x 5 table p in place of
 * model_par_1..5.  Lets one simulation hold many independent scenarios
 * with their own materials. */
struct MaterialTable {
    const float* p = nullptr;
    int n = 0;
};

/* Per-object cell frames: when rows is set, a particle with object id k
 * ((int)idep.x, clamped to [0, n)) lies in its own block of grid rows: its
 * local y cell c (0 <= c < rows[2k+1], else outside the lattice) maps to
 * grid row rows[2k] + c.  Positions stay local to each object, so many
 * independent scenarios share one grid without losing float precision. */
struct Frames {
    const int* rows = nullptr;
    int n = 0;
};

/* Health counters written by the kernels (see lq_sim_health). */
enum { HEALTH_NONFINITE = 0, HEALTH_MAT_OUT = 1, HEALTH_BND_OUT = 2, HEALTH_NBR_OVERFLOW = 3, HEALTH_WORDS = 4 };

/* ----------------------------------------------------------------- grid */
struct GridBuffers {
    int np_cap = 0, ncell_cap = 0;
    int* key = nullptr;       /* unsorted cell key              np */
    int* rank = nullptr;      /* rank inside the cell           np */
    int* count = nullptr;     /* particles per cell             ncell + 1 */
    int* start = nullptr;     /* exclusive scan of count        ncell + 1 */
    int* part_idx = nullptr;  /* sorted slot -> previous slot   np */
    int* part_cel = nullptr;  /* sorted key                     np */
    int* beg = nullptr;       /* optional per-cell bounds       ncell */
    int* end = nullptr;
    void* scan_tmp = nullptr;
    size_t scan_bytes = 0;
};

/* Sizes the scan scratch for n_cells + 1 entries. */
int scan_scratch_bytes(int ncell, size_t* bytes);
/* Bounds violations counted by the grid and the neighbour kernels of a
 * bounds-checked build (-D LQ_CHECKED); 0 otherwise. */
int bounds_count_grid(unsigned long long* v);
int bounds_count_sph(unsigned long long* v);

/* Hash, count, scan, scatter and in-cell ordering: a stable sort of the
 * particles by cell key.  Writes key, rank, count, start, part_idx,
 * part_cel, and beg/end when `bounds` is set.  `health` may be null. */
int grid_search(const Parameters* par_host, const Parameters* par_dev, const float4* pos, GridBuffers& g,
                bool bounds, int* health, cudaStream_t s, const float4* idep = nullptr,
                const Frames& fr = Frames());

/* Particle identities of the drop-in grids (lq_grid_* and LoquatGrid),
 * keyed by the grid's cell_beg array: ident[slot] is the slot the particle
 * now there had when the grid was sized (its order before the first
 * search), updated by every search through the grid's part_idx.  A caller
 * that re-sorts its arrays after each search, as the reference does,
 * keeps its particles and these identities in step, which lets the
 * drop-in interaction carry neighbour lists across searches.  `gen`
 * changes when the grid is resized. */
struct GridIdentity {
    const int* ident = nullptr;
    int np = 0;
    long long gen = 0;
};
int identity_reset(const int* key, int np);
int identity_after_search(const int* key, const int* part_idx, int np, cudaStream_t s);
void identity_release(const int* key);
bool identity_find(const int* key, GridIdentity* out);

int gather_float4(int n, const int* idx, const float4* in, float4* out, cudaStream_t s);
int gather_tensor2d(int n, const int* idx, const tensor2d* in, tensor2d* out, cudaStream_t s);
/* Gathers all five state arrays in one pass: out[i] = in[idx[i]]. */
int gather_state(int n, const int* idx, const State& in, const State& out, cudaStream_t s);

/* ------------------------------------------------------ neighbour lists */
/* Neighbours stored per material particle; a particle with more walks its
 * 27 cells directly instead. */
#define LQ_NBR_CAP 192

struct NeighborList {
    int* list = nullptr;    /* int[LQ_NBR_CAP * stride], entry k of particle t at k * stride + t */
    int* count = nullptr;   /* int[stride] */
    int stride = 0;         /* >= npm, multiple of 32 */
};

/* ------------------------------------------------------------ operators */
int launch_neighbor_list(const Parameters* par_host, const Parameters* par_dev, const float4* pos, const Cells& c,
                         const NeighborList& nl, cudaStream_t s);
/* `rec` (np x 13 floats, 16-byte aligned; required) holds the neighbour
 * data packed into dense arrays (position and density, velocity and
 * sigma/rho^2: 52 bytes per particle, 48 in the compensated form, whose
 * velocity is packed into two words) that the pair kernel gathers; with
 * `pack` they are packed from the state first, in the form of
 * `compensated`.  With `rows` (thread-per-target shapes, `pack` set)
 * target t reads list row rows[t] (-1: walk the stencil), whose entries
 * index records packed in another slot order: slot i's record goes to
 * map[i], target t's own at npb + rows[t]. */
int launch_interaction_list(const Parameters* par_host, const Parameters* par_dev, const State& st, const Rates& r,
                            const Cells& c, const NeighborList& nl, cudaStream_t s, const Frames& fr = Frames(),
                            bool compensated = false, float* rec = nullptr, int shape = 0, bool pack = true,
                            const int* order = nullptr, const int* rows = nullptr, const int* map = nullptr);
/* The packed neighbour arrays of slots [first, np) from the state;
 * packed_velocity selects the compensated pair kernel's record. */
int launch_pack_neighbors(const Parameters* par_host, const State& st, float* rec, int first, cudaStream_t s,
                          bool packed_velocity, const int* map = nullptr);
/* Adami over the boundary lists reading the packed arrays (material slots
 * packed), writing the boundary stress into the state, into str2 when set
 * and into the stress words of the packed arrays (the boundary slots'
 * other words, from the last full pack, stay).  With act / nact (device;
 * from launch_boundary_targets; act holds at least npb ints) only the
 * slots act[0 .. *nact) are visited. */
int launch_adami_packed(const Parameters* par_host, const Parameters* par_dev, const State& st,
                        const NeighborList& nl, float* rec, cudaStream_t s, tensor2d* str2 = nullptr,
                        const int* act = nullptr, const int* nact = nullptr);
/* The boundary slots t < npb with count[t] > 0 or count2[t] > 0 (count2
 * may be null), ascending, into act[0 .. *nact) on the device; temp holds
 * boundary_targets_temp_bytes(npb) bytes of scratch. */
size_t boundary_targets_temp_bytes(int npb);
int launch_boundary_targets(int npb, const int* count, const int* count2, int* act, int* nact, void* temp,
                            size_t temp_bytes, cudaStream_t s);
/* Launch shapes of the packed pair kernel: {threads per block, resident
 * blocks per SM, tile order}, or {128, -G, 0} for the warp-cooperative form
 * with G lanes per target.  Shapes with the tile order take their targets
 * from TileOrder::order (launch_tile_order, after each search). */
constexpr int kPairShapeCount = 11;
constexpr int kDefaultTiledShape = 9;   /* 640 x 1, tile order */
extern const int kPairShapes[kPairShapeCount][3];
/* Launch shape of a new simulation with npm material particles. */
int default_pair_shape(int npm);
/* Targets of the pair kernel in tile order, and the scratch that builds it:
 * order holds npm target indices; seg holds 3 x nseg_cap ints (segment
 * begin, length, offset). */
struct TileOrder {
    int* order = nullptr;
    int* seg = nullptr;
    int nseg_cap = 0;
    void* scan_tmp = nullptr;
    size_t scan_bytes = 0;
};
/* Segments (for the smallest tile height) and scan scratch bytes; the
 * segment scratch is 3 x nseg ints. */
int tile_order_scratch(const Parameters* par_host, int* nseg, size_t* scan_bytes);
/* The tile order for launch shape `shape` from the grid's cell starts
 * (nothing for shapes without it). */
int launch_tile_order(const Parameters* par_host, const int* start, int shape, const TileOrder& to, cudaStream_t s);
int launch_adami(const Parameters* par_host, const Parameters* par_dev, const State& st, const Cells& c,
                 cudaStream_t s);
/* Shepard filter of material stress into out_str[npb, np).  When `full` is
 * set the kernel also copies every other array (and the boundary stress)
 * from `st` to `out`, producing a complete new state. */
int launch_shepard(const Parameters* par_host, const Parameters* par_dev, const State& st, tensor2d* out_str,
                   const State* full, const Cells& c, cudaStream_t s);
/* Predictor: out <- in advanced by dt/2 on material slots; boundary slots
 * are left alone (the native driver's Adami writes both of its state
 * buffers), except that with a snapshot `snap` (may be all-null), which
 * receives a copy of `in`, a separate `out` takes their stress.  With `rec` (the packed neighbour arrays) each
 * material slot's entry is written from its new values, in the record of
 * the form (the mixed form's packed velocity when the state has low
 * words); the same holds for the corrector below.  With `stage` (no
 * snapshot, out distinct from in) out is a stage buffer read only by the
 * neighbour kernels and launch_correct_into: its strain, its low words and
 * its hypoplastic plastic strain are not written. */
int launch_predict(const Parameters* par_host, const Parameters* par_dev, const State& in, const State& out,
                   const State* snap, const Rates& r, cudaStream_t s, const MaterialTable& mt = MaterialTable(),
                   const MaterialTable& vw = MaterialTable(), float* rec = nullptr, bool stage = false);
/* Corrector in place on `cur`; ini values read at ini_idx[i] (identity when
 * ini_idx is null).  Non-finite results are counted in health. */
int launch_correct(const Parameters* par_host, const Parameters* par_dev, const State& cur, const State& ini,
                   const int* ini_idx, const Rates& r, int* health, cudaStream_t s);

/* Corrector from snapshot `ini` and current `cur` into `out`, material
 * slots only (boundary slots must already be the same in all three);
 * material particles raise bit 1 of *rebuild when neighbour
 * lists built at xbuild with this skin may not hold through the next step,
 * and (with xwide) bit 2 when a particle has moved (wide - skin) / 2 or
 * more from xwide, where lists with cut-off 2h + wide were built: lists
 * renewed from those now could miss a pair. */
int launch_correct_into(const Parameters* par_host, const Parameters* par_dev, const State& cur, const State& ini,
                        const State& out, const Rates& r, int* health, const float4* xbuild, int* rebuild,
                        float skin, cudaStream_t s, const MaterialTable& mt = MaterialTable(),
                        const MaterialTable& vw = MaterialTable(), const float4* xwide = nullptr,
                        float wide = 0.0f, float* rec = nullptr);

/* List-driven Shepard filter (material targets and neighbours) reading
 * the neighbours from the packed records `rec` (required; the material
 * slots' records must hold the state st), targets in the tile order
 * `order` when set; a target whose list overflowed walks its 27 cells in
 * `c` over the state instead. */
int launch_shepard_list(const Parameters* par_host, const Parameters* par_dev, const State& st, tensor2d* out_str,
                        const NeighborList& nl, const Cells& c, cudaStream_t s, const Frames& fr, float* rec,
                        const int* order = nullptr);
/* Density Shepard filter of material slots into rho_out[npb, np) over the
 * material lists, from the packed records likewise (overflowed lists walk
 * their 27 cells in `c`). */
int launch_density_filter_list(const Parameters* par_host, const Parameters* par_dev, const State& st,
                               float* rho_out, const NeighborList& nl, const Cells& c, cudaStream_t s,
                               const Frames& fr, float* rec, const int* order = nullptr);
/* Neighbour lists of targets [first, first + n) from grid layers
 * layer_lo..1 with cut-off radius `cut` (2h plus skin); list overflows are
 * counted in health[HEALTH_NBR_OVERFLOW].  With `shell`, pairs at distance
 * `inner` or more go to the shell list instead (wide build of two-level
 * lists; nl.count then receives the inner counts).  With `gate` the
 * kernel does nothing unless *gate is non-zero (a decision taken on the
 * device). */
int launch_neighbor_list_range(const Parameters* par_host, const Parameters* par_dev, int first, int n, int layer_lo,
                               float cut, const float4* pos, const Cells& c, const NeighborList& nl, int* health,
                               cudaStream_t s, const float4* idep = nullptr, const Frames& fr = Frames(),
                               const NeighborList* shell = nullptr, float inner = 0.0f, const int* gate = nullptr);
/* Two-level lists of targets [first, first + n): rows [0, inner_count[t])
 * of nl, written by the wide build, kept, and the entries of the shell list
 * now within `cut` appended (positions pos). */
int launch_list_refresh(const Parameters* par_host, int first, int n, float cut, const float4* pos,
                        const int* inner_count, const NeighborList& shell, const NeighborList& nl, int* health,
                        cudaStream_t s);
/* Fills n ints with v; adds v to one int. */
int fill_int(int* p, int n, int v, cudaStream_t s);
int add_int(int* p, int v, cudaStream_t s);

/* Host-side copy of Parameters derivation (reference src/loquat.cu:111-139). */
void initialize_parameters(Parameters* p);

}  // namespace lqb
