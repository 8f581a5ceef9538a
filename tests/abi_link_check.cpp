// Link check of the drop-in surface: a caller written against the
// reference's headers (loquat_grid.h, particle_interaction.h,
// predictor_corrector.h, adami_boundary.h, field_smoothing.h, types.h) and
// the C ABI header must compile against include/ and link against
// liblqb200.so with every symbol resolved.  It only takes addresses; it
// makes no CUDA call.
#include <cstdio>
#include <types.h>
#include <loquat_grid.h>
#include <particle_interaction.h>
#include <predictor_corrector.h>
#include <adami_boundary.h>
#include <field_smoothing.h>
#include <loquat_b200.h>

static_assert(sizeof(Parameters) == 208, "Parameters layout");
static_assert(sizeof(tensor2d) == 24, "tensor2d layout");
static_assert(sizeof(LoquatGrid) == 6 * sizeof(int*) + sizeof(void*) + sizeof(size_t), "LoquatGrid layout");

int main()
{
    void (LoquatGrid::*m1)(Parameters*) = &LoquatGrid::GridConfig;
    void (LoquatGrid::*m2)(int, int) = &LoquatGrid::ResizeArrayLength;
    void (LoquatGrid::*m3)(Parameters*, Parameters*, float4*, float4*) = &LoquatGrid::NeighborSearch;
    void (LoquatGrid::*m4)(int, float4*, float4*) = &LoquatGrid::SortArrayFloat4;
    void (LoquatGrid::*m5)(int, tensor2d*, tensor2d*) = &LoquatGrid::SortArrayTensor2d;
    const void* fns[] = {
        (const void*)&ParticleInteraction, (const void*)&Predictor, (const void*)&Corrector,
        (const void*)&AdamiBoundary, (const void*)&StressRegularization,
        (const void*)&lq_abi_version, (const void*)&lq_parameters_size, (const void*)&lq_last_error,
        (const void*)&lq_status_string, (const void*)&lq_initialize_parameters, (const void*)&lq_update_time_step,
        (const void*)&lq_grid_create, (const void*)&lq_grid_resize, (const void*)&lq_grid_destroy,
        (const void*)&lq_grid_neighbor_search, (const void*)&lq_grid_arrays, (const void*)&lq_grid_sort_float4,
        (const void*)&lq_grid_sort_tensor2d, (const void*)&lq_grid_neighbor_search_noalloc, (const void*)&lq_particle_interaction, (const void*)&lq_adami_boundary,
        (const void*)&lq_stress_regularization, (const void*)&lq_predictor, (const void*)&lq_corrector,
        (const void*)&lq_sim_create, (const void*)&lq_sim_destroy, (const void*)&lq_sim_step,
        (const void*)&lq_sim_synchronize, (const void*)&lq_sim_stream, (const void*)&lq_sim_upload,
        (const void*)&lq_sim_download, (const void*)&lq_sim_state, (const void*)&lq_sim_clock,
        (const void*)&lq_sim_health, (const void*)&lq_sim_launches_per_step, (const void*)&lq_sim_profile,
        (const void*)&lq_sim_set_skin, (const void*)&lq_sim_set_materials, (const void*)&lq_sim_set_hypoplastic, (const void*)&lq_sim_set_frames, (const void*)&lq_sim_rebuilds, (const void*)&lq_sim_rebuild_launches, (const void*)&lq_sim_set_wide_skin, (const void*)&lq_sim_wide_skin, (const void*)&lq_sim_renewals, (const void*)&lq_sim_renewal_launches, (const void*)&lq_sim_neighbor_entries, (const void*)&lq_debug_bounds_violations, (const void*)&lq_sim_set_pair_shape, (const void*)&lq_sim_pair_shape, (const void*)&lq_sim_autotune, (const void*)&lq_sim_save_checkpoint, (const void*)&lq_sim_load_checkpoint,
        (const void*)&lq_io_load_parameters,
        (const void*)&lq_io_save_parameters, (const void*)&lq_io_load_hypoplastic, (const void*)&lq_io_save_parameters_vw, (const void*)&lq_io_load_particles, (const void*)&lq_io_save_particles,
        (const void*)&lq_io_save_vtu,
    };
    int n = 0;
    for (const void* f : fns) n += f != nullptr;
    LoquatGrid* g = new LoquatGrid();   // constructor and destructor make no CUDA call with null members
    delete g;
    (void)m1; (void)m2; (void)m3; (void)m4; (void)m5;
    printf("%d %zu\n", n, lq_parameters_size());
    return n == (int)(sizeof(fns) / sizeof(fns[0])) ? 0 : 1;
}
