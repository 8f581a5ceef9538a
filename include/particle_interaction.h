/*
 * LOQUAT-B200 drop-in for the reference's particle-interaction pass
 * (reference: src/particle_interaction.h:27-40; implementation closed there).
 *
 * For every material slot i in [npb, np) it writes
 *   accad[i]  = (dv/dt, drho/dt)     momentum + gravity, continuity
 *   spin[i]   = (W_yx, W_zx, W_zy, 0) spin tensor, W = (L - L^T) / 2
 *   acestn[i] = sym(L)                strain rate
 * with L_ab = sum_j V_j (v_j - v_i)_a dW_ij/dx_b over both grid layers.
 * Boundary slots [0, npb) of the outputs are left untouched.
 * The formulation is written out in the oracle and the design notes.
 */
#pragma once
#ifndef LOQUAT_B200_PARTICLE_INTERACTION_H
#define LOQUAT_B200_PARTICLE_INTERACTION_H

#include <iostream>
#include <cuda_runtime.h>
#include <types.h>

void ParticleInteraction(
        Parameters* par_host,
        Parameters* par_device,
        float4* pospres,
        float4* velrhop,
        float4* idep,
        tensor2d* str,
        tensor2d* stn,
        float4* accad,
        float4* spin,
        tensor2d* acestn,
        const int* cell_beg,
        const int* cell_end);

#endif
