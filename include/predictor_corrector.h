/*
 * LOQUAT-B200 drop-in for the reference's predictor-corrector integrator
 * (reference: src/predictor_corrector.h:30-67, src/predictor_corrector.cu:221-336).
 *
 * Predictor: snapshots the five state arrays into the *_ini arrays and
 * advances material slots [npb, np) by dt/2.  Corrector: advances the
 * material slots by dt from the (re-sorted) snapshot.  The stress update is
 * Drucker-Prager (constitutive_model 1) or the four-parameter hypoplastic
 * model (constitutive_model 2), both with the Jaumann rate.
 */
#pragma once
#ifndef LOQUAT_B200_PREDICTOR_CORRECTOR_H
#define LOQUAT_B200_PREDICTOR_CORRECTOR_H

#include <stdio.h>
#include <cuda_runtime.h>
#include <types.h>

void Predictor(
        Parameters* par_host,
        Parameters* par_device,
        float4* pospres,
        float4* velrhop,
        float4* idep,
        tensor2d* str,
        tensor2d* stn,
        float4* pospres_ini,
        float4* velrhop_ini,
        float4* idep_ini,
        tensor2d* str_ini,
        tensor2d* stn_ini,
        float4* accad,
        float4* spin,
        tensor2d* acestn);

void Corrector(
        Parameters* par_host,
        Parameters* par_device,
        float4* pospres,
        float4* velrhop,
        float4* idep,
        tensor2d* str,
        tensor2d* stn,
        float4* pospres_ini,
        float4* velrhop_ini,
        float4* idep_ini,
        tensor2d* str_ini,
        tensor2d* stn_ini,
        float4* accad,
        float4* spin,
        tensor2d* acestn);

#endif
