// The reference's hot loop (src/loquat.cu:285-409), written against the
// drop-in headers exactly as the reference's LoquatSph::RunSimulation calls
// them: LoquatGrid, AdamiBoundary, ParticleInteraction, Predictor,
// Corrector, StressRegularization, with the reference's array set and
// SortArraysPrimary / SortArraysAll (src/loquat.cu:190-213).
//
//   dropin_driver <project> <nsteps> <out.dat>
// reads <project>.xml and <project>.dat, runs nsteps, writes the state.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include <types.h>
#include <loquat_grid.h>
#include <particle_interaction.h>
#include <predictor_corrector.h>
#include <adami_boundary.h>
#include <field_smoothing.h>
#include <loquat_b200.h>

#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { fprintf(stderr, "%s: %s\n", #x, cudaGetErrorString(e_)); return 2; } } while (0)
#define LQ(x) do { int s_ = (x); if (s_ != 0) { fprintf(stderr, "%s: %s\n", #x, lq_last_error()); return 3; } } while (0)

int main(int argc, char** argv)
{
    if (argc < 4) { fprintf(stderr, "usage: %s <project> <nsteps> <out.dat>\n", argv[0]); return 1; }
    const std::string project = argv[1];
    const int nsteps = atoi(argv[2]);
    Parameters* par_host = new Parameters;
    LQ(lq_io_load_parameters((project + ".xml").c_str(), par_host));
    LQ(lq_initialize_parameters(par_host));
    const int np = par_host->np;
    std::vector<float> h_pos(4 * np), h_vel(4 * np), h_idep(4 * np), h_str(6 * np), h_stn(6 * np);
    LQ(lq_io_load_particles((project + ".dat").c_str(), np, h_pos.data(), h_vel.data(), h_idep.data(), h_str.data(), h_stn.data()));

    Parameters* par_device;
    float4 *pospres, *velrhop, *idep, *pospres_ini, *velrhop_ini, *idep_ini, *accad, *spin, *float4_cache;
    tensor2d *str, *stn, *str_ini, *stn_ini, *acestn, *tensor2d_cache;
    CK(cudaMalloc(&par_device, sizeof(Parameters)));
    float4** f4[] = {&pospres, &velrhop, &idep, &pospres_ini, &velrhop_ini, &idep_ini, &accad, &spin, &float4_cache};
    for (float4** p : f4) CK(cudaMalloc(p, np * sizeof(float4)));
    tensor2d** t2[] = {&str, &stn, &str_ini, &stn_ini, &acestn, &tensor2d_cache};
    for (tensor2d** p : t2) CK(cudaMalloc(p, np * sizeof(tensor2d)));
    CK(cudaMemcpy(pospres, h_pos.data(), np * sizeof(float4), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(velrhop, h_vel.data(), np * sizeof(float4), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(idep, h_idep.data(), np * sizeof(float4), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(str, h_str.data(), np * sizeof(tensor2d), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(stn, h_stn.data(), np * sizeof(tensor2d), cudaMemcpyHostToDevice));

    LoquatGrid* grid = new LoquatGrid();
    grid->GridConfig(par_host);
    auto sort_primary = [&]() {
        grid->SortArrayFloat4(np, pospres, float4_cache);
        grid->SortArrayFloat4(np, velrhop, float4_cache);
        grid->SortArrayFloat4(np, idep, float4_cache);
        grid->SortArrayTensor2d(np, str, tensor2d_cache);
        grid->SortArrayTensor2d(np, stn, tensor2d_cache);
    };
    auto sort_all = [&]() {
        sort_primary();
        grid->SortArrayFloat4(np, pospres_ini, float4_cache);
        grid->SortArrayFloat4(np, velrhop_ini, float4_cache);
        grid->SortArrayFloat4(np, idep_ini, float4_cache);
        grid->SortArrayTensor2d(np, str_ini, tensor2d_cache);
        grid->SortArrayTensor2d(np, stn_ini, tensor2d_cache);
    };
    CK(cudaMemcpy(par_device, par_host, sizeof(Parameters), cudaMemcpyHostToDevice));
    grid->NeighborSearch(par_host, par_device, pospres, idep);
    sort_primary();

    double time = (double)par_host->time;
    for (int step = 0; step < nsteps; ++step) {
        par_host->dt = par_host->cfl * par_host->h / par_host->cs;
        par_host->time = (float)time;
        CK(cudaMemcpy(par_device, par_host, sizeof(Parameters), cudaMemcpyHostToDevice));
        grid->NeighborSearch(par_host, par_device, pospres, idep);
        sort_primary();
        cudaDeviceSynchronize();
        AdamiBoundary(par_host, par_device, pospres, velrhop, str, grid->GetCellBeg(), grid->GetCellEnd());
        ParticleInteraction(par_host, par_device, pospres, velrhop, idep, str, stn, accad, spin, acestn,
                            grid->GetCellBeg(), grid->GetCellEnd());
        Predictor(par_host, par_device, pospres, velrhop, idep, str, stn, pospres_ini, velrhop_ini, idep_ini,
                  str_ini, stn_ini, accad, spin, acestn);
        cudaDeviceSynchronize();
        grid->NeighborSearch(par_host, par_device, pospres, idep);
        sort_all();
        AdamiBoundary(par_host, par_device, pospres, velrhop, str, grid->GetCellBeg(), grid->GetCellEnd());
        ParticleInteraction(par_host, par_device, pospres, velrhop, idep, str, stn, accad, spin, acestn,
                            grid->GetCellBeg(), grid->GetCellEnd());
        Corrector(par_host, par_device, pospres, velrhop, idep, str, stn, pospres_ini, velrhop_ini, idep_ini,
                  str_ini, stn_ini, accad, spin, acestn);
        cudaDeviceSynchronize();
        if (par_host->stress_shepard_filter != 0 && step % par_host->stress_shepard_filter == 0 && step != 0) {
            grid->NeighborSearch(par_host, par_device, pospres, idep);
            sort_primary();
            StressRegularization(par_host, par_device, pospres, velrhop, str, tensor2d_cache, grid->GetCellBeg(),
                                 grid->GetCellEnd());
        }
        time += (double)par_host->dt;
    }
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpy(h_pos.data(), pospres, np * sizeof(float4), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(h_vel.data(), velrhop, np * sizeof(float4), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(h_idep.data(), idep, np * sizeof(float4), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(h_str.data(), str, np * sizeof(tensor2d), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(h_stn.data(), stn, np * sizeof(tensor2d), cudaMemcpyDeviceToHost));
    LQ(lq_io_save_particles(argv[3], np, h_pos.data(), h_vel.data(), h_idep.data(), h_str.data(), h_stn.data()));
    delete grid;
    for (float4** p : f4) cudaFree(*p);
    for (tensor2d** p : t2) cudaFree(*p);
    cudaFree(par_device);
    printf("ok %d\n", np);
    return 0;
}
