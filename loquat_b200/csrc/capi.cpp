/*
 * LOQUAT-B200 C ABI: library information, error reporting and the
 * parameter derivation of LoquatSph::InitializeParameters.
 */
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <string>

#include <cuda_runtime.h>
#include "lq_internal.cuh"

namespace lqb {

namespace {
thread_local std::string g_last_error;
}

int set_error(int status, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return status;
}

int cuda_status(cudaError_t e, const char* what)
{
    return set_error(LQ_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

/* Derived constants with the reference's float arithmetic
 * (reference src/loquat.cu:111-139): the same inputs give the same bits. */
void initialize_parameters(Parameters* p)
{
    p->h = p->dr * p->hdr;
    p->i_h = 1.0f / p->h;
    p->eta = 0.01f * p->h * p->h;
    p->m = p->dr * p->dr * p->dr * p->rho0;
    p->cell_num_x = static_cast<int>(0.5f * p->i_h * p->domain_size_x) + 1;
    p->cell_num_y = static_cast<int>(0.5f * p->i_h * p->domain_size_y) + 1;
    p->cell_num_z = static_cast<int>(0.5f * p->i_h * p->domain_size_z) + 1;
    p->ncell_one_layer = p->cell_num_x * p->cell_num_y * p->cell_num_z;
    p->ncell = 2 * p->ncell_one_layer + 1;
    p->ncell_delete = p->ncell - 1;
    /* Wendland C2 on support 2h: W = C (2-q)^4 (q + 1/2), grad W = C' (2-q)^3 x_ij */
    p->kernel_normalization_par = 42.0f / 256.0f / (powf(p->h, 3) * PI);
    p->kernel_gradient_normalization_par = -5.0f * 42.0f / 256.0f / (powf(p->h, 5) * PI);
    if (p->artificial_pressure == 1) {
        p->kernel_zero = p->kernel_normalization_par * 2.0f * 2.0f * 2.0f * 2.0f * 0.5f;
        const float q = p->dr * p->i_h;
        p->kernel_dr = p->kernel_normalization_par * (2.0f - q) * (2.0f - q) * (2.0f - q) * (2.0f - q) * (q + 0.5f);
    }
}

}  // namespace lqb

extern "C" int lq_abi_version(void) { return LQ_ABI_VERSION; }

extern "C" size_t lq_parameters_size(void) { return sizeof(Parameters); }

extern "C" const char* lq_last_error(void) { return lqb::g_last_error.c_str(); }

extern "C" const char* lq_status_string(int status)
{
    switch (status) {
    case LQ_OK: return "ok";
    case LQ_ERR_ARG: return "invalid argument";
    case LQ_ERR_CUDA: return "CUDA error";
    case LQ_ERR_ALLOC: return "allocation failed";
    case LQ_ERR_IO: return "I/O error";
    case LQ_ERR_STATE: return "simulation health check failed";
    case LQ_ERR_NOTFOUND: return "required key not found";
    default: return "unknown status";
    }
}

extern "C" int lq_initialize_parameters(void* par_host)
{
    if (!par_host) return lqb::set_error(LQ_ERR_ARG, "lq_initialize_parameters: null Parameters");
    Parameters* p = static_cast<Parameters*>(par_host);
    if (!(p->dr > 0.0f) || !(p->hdr > 0.0f))
        return lqb::set_error(LQ_ERR_ARG, "lq_initialize_parameters: particle-size and h-over-dr must be positive");
    if (!(p->domain_size_x > 0.0f) || !(p->domain_size_y > 0.0f) || !(p->domain_size_z > 0.0f))
        return lqb::set_error(LQ_ERR_ARG, "lq_initialize_parameters: domain sizes must be positive");
    lqb::initialize_parameters(p);
    const double cells = (double)p->cell_num_x * p->cell_num_y * p->cell_num_z;
    if (cells * 2.0 + 1.0 > 2147483647.0)
        return lqb::set_error(LQ_ERR_ARG, "lq_initialize_parameters: %.0f cells per layer overflow int keys", cells);
    return LQ_OK;
}

extern "C" int lq_update_time_step(void* par_host)
{
    if (!par_host) return lqb::set_error(LQ_ERR_ARG, "lq_update_time_step: null Parameters");
    Parameters* p = static_cast<Parameters*>(par_host);
    p->dt = p->cfl * p->h / p->cs;
    return LQ_OK;
}
