/*
 * loquat: command-line driver over the LOQUAT-B200 library, the counterpart
 * of the reference's executable (reference src/main.cpp, src/loquat.cu:216-476).
 *
 *   loquat <project> [gpu] [--mixed] [--no-graph] [--density-filter] [--dynamic-dt]
 *
 * --density-filter and --dynamic-dt switch on features the reference reads
 * from its parameter file but never applies (LQ_SIM_DENSITY_FILTER,
 * LQ_SIM_DYNAMIC_DT).  With --dynamic-dt the steps have no fixed length, so
 * the loop steps one at a time and reads the simulated time back from the
 * device, saving once the time since the last output exceeds
 * output-frequency.
 *
 * Reads <project>.xml and <project>.dat, writes output_<n>.xml and <n>.dat
 * (output-format 1) or <id>_<n>.vtu files (output-format 2) into the folder
 * <project>/ every output-frequency of simulated time, and prints the
 * reference's progress lines and a summary.  Output n = 0 is the initial
 * state.  The time loop runs as chunks of graph-replayed steps between
 * outputs; the step count and output times follow the reference's loop
 * (time += dt; output when the time since the last output exceeds
 * output-frequency).
 */
#include <sys/stat.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <types.h>
#include <loquat_b200.h>

namespace {

void fail(const char* what)
{
    fprintf(stderr, "Error! %s: %s\n", what, lq_last_error());
    exit(EXIT_FAILURE);
}

#define LQ_CALL(x) do { if ((x) != LQ_OK) fail(#x); } while (0)

struct Host {
    std::vector<float> pos, vel, idep, str, stn;
    void resize(int n)
    {
        pos.resize(4 * (size_t)n);
        vel.resize(4 * (size_t)n);
        idep.resize(4 * (size_t)n);
        str.resize(6 * (size_t)n);
        stn.resize(6 * (size_t)n);
    }
};

/* vw: the model-3 row when constitutive-model is 3 (its keys are written
 * with the parameters), else null */
void save(const std::string& dir, Parameters& par, Host& h, const float* vw, float e0)
{
    const std::string xml = dir + "/output_" + std::to_string(par.output_number) + ".xml";
    if (vw)
        LQ_CALL(lq_io_save_parameters_vw(xml.c_str(), &par, vw, e0));
    else
        LQ_CALL(lq_io_save_parameters(xml.c_str(), &par));
    if (par.output_format == 2) {
        LQ_CALL(lq_io_save_vtu(dir.c_str(), par.output_number, par.np, h.pos.data(), h.vel.data(), h.idep.data(),
                               h.str.data(), h.stn.data()));
    } else {
        const std::string dat = dir + "/" + std::to_string(par.output_number) + ".dat";
        LQ_CALL(lq_io_save_particles(dat.c_str(), par.np, h.pos.data(), h.vel.data(), h.idep.data(), h.str.data(),
                                     h.stn.data()));
    }
}

}  // namespace

int main(int argc, char** argv)
{
    printf("**********************************\n** LOQUAT-B200 (sm_100a)         **\n"
           "**********************************\n\n");
    std::string project;
    int device = 0;
    int flags = LQ_SIM_GRAPH;
    for (int a = 1; a < argc; ++a) {
        if (!strcmp(argv[a], "--mixed")) flags |= LQ_SIM_MIXED;
        else if (!strcmp(argv[a], "--no-graph")) flags &= ~LQ_SIM_GRAPH;
        else if (!strcmp(argv[a], "--density-filter")) flags |= LQ_SIM_DENSITY_FILTER;
        else if (!strcmp(argv[a], "--dynamic-dt")) flags |= LQ_SIM_DYNAMIC_DT;
        else if (project.empty()) project = argv[a];
        else device = atoi(argv[a]);
    }
    if (project.empty()) {
        printf("Error! Please give the project name!\n");
        return EXIT_FAILURE;
    }
    int ngpu = 0;
    cudaGetDeviceCount(&ngpu);
    printf("Number of GPUs on this computer: %d\n", ngpu);
    for (int i = 0; i < ngpu; ++i) {
        cudaDeviceProp p;
        cudaGetDeviceProperties(&p, i);
        printf("  (%d) %s %zu MB (%d.%d)\n", i, p.name, p.totalGlobalMem / 1048576, p.major, p.minor);
    }
    if (device < 0 || device >= ngpu) {
        printf("Error! GPU %d does not exist\n", device);
        return EXIT_FAILURE;
    }
    cudaSetDevice(device);
    printf("\nSimulation running on GPU %d\n", device);

    Parameters par;
    LQ_CALL(lq_io_load_parameters((project + ".xml").c_str(), &par));
    LQ_CALL(lq_initialize_parameters(&par));
    printf("ncellx = %d, ncelly = %d, ncellz = %d, ncell = %d\n\n", par.cell_num_x, par.cell_num_y, par.cell_num_z,
           par.ncell);
    Host h;
    h.resize(par.np);
    LQ_CALL(lq_io_load_particles((project + ".dat").c_str(), par.np, h.pos.data(), h.vel.data(), h.idep.data(),
                                 h.str.data(), h.stn.data()));
    /* constitutive model 3: material row and initial void ratio from the
     * parameter file's extension keys; the particle file has no void ratio */
    float vw_row[10] = {0};
    float e0 = 0.0f;
    const bool vw = par.constitutive_model == 3;
    if (vw) {
        LQ_CALL(lq_io_load_hypoplastic((project + ".xml").c_str(), vw_row, &e0));
        for (int i = par.npb; i < par.np; ++i)
            if (h.idep[4 * (size_t)i + 2] == 0.0f) h.idep[4 * (size_t)i + 2] = e0;
    }
    const std::string dir = project;
    mkdir(dir.c_str(), 0755);

    void* sim = nullptr;
    LQ_CALL(lq_sim_create(&par, h.pos.data(), h.vel.data(), h.idep.data(), h.str.data(), h.stn.data(), flags, &sim));
    if (vw) LQ_CALL(lq_sim_set_hypoplastic(sim, 1, vw_row));
    LQ_CALL(lq_update_time_step(&par));
    save(dir, par, h, vw ? vw_row : nullptr, e0);

    const double dt = par.dt;
    double time = par.time;
    double output_time = 0.0;
    long long step = 0, step_interval = 0;
    const auto t_start = std::chrono::steady_clock::now();
    auto t_interval = t_start;
    double saving = 0.0;
    const bool dynamic = (flags & LQ_SIM_DYNAMIC_DT) != 0;
    double last_output = time;
    while (dynamic && time < (double)par.time_max) {
        LQ_CALL(lq_sim_step(sim, 1));
        ++step;
        long long st = 0;
        LQ_CALL(lq_sim_clock(sim, &st, &time));
        if (time - last_output > (double)par.output_frequency || time >= (double)par.time_max) {
            const auto now = std::chrono::steady_clock::now();
            const double interval = std::chrono::duration<double>(now - t_interval).count();
            const double fps = (double)(step - step_interval) / interval;
            par.time = (float)time;
            par.output_number++;
            LQ_CALL(lq_sim_download(sim, h.pos.data(), h.vel.data(), h.idep.data(), h.str.data(), h.stn.data()));
            const auto s0 = std::chrono::steady_clock::now();
            save(dir, par, h, vw ? vw_row : nullptr, e0);
            saving += std::chrono::duration<double>(std::chrono::steady_clock::now() - s0).count();
            printf("----------Save-----------\nTime = %0.5f | Step = %lld | FPS = %0.5f\n", par.time, step - 1, fps);
            printf("Save file: %s/output_%d.xml\n\n", dir.c_str(), par.output_number);
            last_output = time;
            step_interval = step;
            t_interval = std::chrono::steady_clock::now();
        }
    }
    while (!dynamic && time < (double)par.time_max) {
        /* steps until the reference's loop would save (output_time > freq is
         * checked after a step and before time advances) or stop */
        long long k = 0;
        double t = time, ot = output_time;
        bool save_now = false;
        while (t < (double)par.time_max) {
            ++k;
            if (ot > (double)par.output_frequency) {
                save_now = true;
                break;
            }
            t += dt;
            ot += dt;
        }
        LQ_CALL(lq_sim_step(sim, (int)k));
        step += k;
        if (save_now) {
            time = t;
            LQ_CALL(lq_sim_synchronize(sim));
            const auto now = std::chrono::steady_clock::now();
            const double interval = std::chrono::duration<double>(now - t_interval).count();
            const double fps = (double)(step - step_interval) / interval;
            par.time = (float)time;
            par.output_number++;
            LQ_CALL(lq_sim_download(sim, h.pos.data(), h.vel.data(), h.idep.data(), h.str.data(), h.stn.data()));
            const auto s0 = std::chrono::steady_clock::now();
            save(dir, par, h, vw ? vw_row : nullptr, e0);
            saving += std::chrono::duration<double>(std::chrono::steady_clock::now() - s0).count();
            printf("----------Save-----------\nTime = %0.5f | Step = %lld | FPS = %0.5f\n", par.time, step - 1, fps);
            printf("Number of particles: %d | Number of cells: %d\n", par.np, par.ncell);
            printf("Save file: %s/output_%d.xml\n\n", dir.c_str(), par.output_number);
            output_time = 0.0 + dt;
            time += dt;
            step_interval = step;
            t_interval = std::chrono::steady_clock::now();
        } else {
            time = t;
            output_time = ot;
        }
    }
    LQ_CALL(lq_sim_synchronize(sim));
    const double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    int health[4];
    LQ_CALL(lq_sim_health(sim, health));
    long long rebuilds = 0;
    LQ_CALL(lq_sim_rebuilds(sim, &rebuilds));
    printf("Simulation finished ...\n\n----------SUMMARY----------\n");
    printf("1. Total wall time = %.3f s\n", total);
    printf("2. Saving = %.3f s\n", saving);
    printf("3. Total steps = %lld\n", step);
    printf("4. Average time step = %g\n", step ? time / (double)step : 0.0);
    printf("5. Average FPS = %.3f\n", step / (total - saving));
    printf("6. Particle-steps/s = %.4g (material particles)\n", (double)par.npm * step / (total - saving));
    printf("7. Neighbour-list rebuilds = %lld\n", rebuilds);
    printf("8. Health: non-finite %d, escaped %d/%d, list overflow %d\n", health[0], health[1], health[2], health[3]);
    lq_sim_destroy(sim);
    return health[0] == 0 ? EXIT_SUCCESS : 2;
}
