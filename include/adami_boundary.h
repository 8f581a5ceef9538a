/*
 * LOQUAT-B200 drop-in for the reference's Adami dummy-particle boundary
 * (reference: src/adami_boundary.h:27-34, src/adami_boundary.cu:27-143).
 *
 * For each boundary slot i in [0, npb) the stress is extrapolated from the
 * material particles of the 27 neighbouring cells (material layer only):
 *   sigma_kk = (S_kk - rho0 g_k P_k) / w,   sigma_kl = S_kl / w   (k != l)
 * with S = sum sigma_j W V_j, P = sum (x_i - x_j) W V_j, w = sum W V_j.
 * Slots with w == 0 keep their stress.
 */
#pragma once
#ifndef LOQUAT_B200_ADAMI_BOUNDARY_H
#define LOQUAT_B200_ADAMI_BOUNDARY_H

#include <cuda_runtime.h>
#include <types.h>
#include "loquat_grid.h"

void AdamiBoundary(
        Parameters* par_host,
        Parameters* par_device,
        float4* pospres,
        float4* velrhop,
        tensor2d* str,
        const int* cell_beg,
        const int* cell_end);

#endif
