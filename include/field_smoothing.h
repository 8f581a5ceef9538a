/*
 * LOQUAT-B200 drop-in for the reference's Shepard stress filter
 * (reference: src/field_smoothing.h:27-35, src/field_smoothing.cu:27-144).
 *
 * For each material slot i: sigma_i <- sum sigma_j W V_j / sum W V_j over the
 * material particles of the 27 neighbouring cells, self included.  The
 * result is staged in tensor2d_cache[npb, np) and then copied into str.
 */
#pragma once
#ifndef LOQUAT_B200_FIELD_SMOOTHING_H
#define LOQUAT_B200_FIELD_SMOOTHING_H

#include <stdio.h>
#include <cuda_runtime.h>
#include <types.h>

void StressRegularization(
        Parameters* par_host,
        Parameters* par_device,
        float4* pospres,
        float4* velrhop,
        tensor2d* str,
        tensor2d* tensor2d_cache,
        const int* cell_beg,
        const int* cell_end);

#endif
