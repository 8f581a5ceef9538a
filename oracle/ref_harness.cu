/*
 * TEST INFRASTRUCTURE ONLY: C entry points around the reference's own open
 * CUDA kernels, so tests can feed them the same device arrays as the product
 * and read back their outputs.  Built by `make ref` into _ref/ together with
 * the reference sources src/predictor_corrector.cu, src/adami_boundary.cu and
 * src/field_smoothing.cu, compiled unchanged.  Each wrapper forwards to the
 * reference function of the same role and synchronises, because the
 * reference launches on the legacy default stream and expects its caller to
 * synchronise after every phase (reference src/loquat.cu:343-396).
 */
#include <cuda_runtime.h>
#include <types.h>
#include "predictor_corrector.h"
#include "adami_boundary.h"
#include "field_smoothing.h"

extern "C" {

int ref_predictor(void* ph, void* pd, void* pos, void* vel, void* idep, void* str, void* stn,
                  void* pos0, void* vel0, void* idep0, void* str0, void* stn0,
                  void* accad, void* spin, void* acestn)
{
    Predictor((Parameters*)ph, (Parameters*)pd, (float4*)pos, (float4*)vel, (float4*)idep,
              (tensor2d*)str, (tensor2d*)stn, (float4*)pos0, (float4*)vel0, (float4*)idep0,
              (tensor2d*)str0, (tensor2d*)stn0, (float4*)accad, (float4*)spin, (tensor2d*)acestn);
    return (int)cudaDeviceSynchronize();
}

int ref_corrector(void* ph, void* pd, void* pos, void* vel, void* idep, void* str, void* stn,
                  void* pos0, void* vel0, void* idep0, void* str0, void* stn0,
                  void* accad, void* spin, void* acestn)
{
    Corrector((Parameters*)ph, (Parameters*)pd, (float4*)pos, (float4*)vel, (float4*)idep,
              (tensor2d*)str, (tensor2d*)stn, (float4*)pos0, (float4*)vel0, (float4*)idep0,
              (tensor2d*)str0, (tensor2d*)stn0, (float4*)accad, (float4*)spin, (tensor2d*)acestn);
    return (int)cudaDeviceSynchronize();
}

int ref_adami(void* ph, void* pd, void* pos, void* vel, void* str, const int* beg, const int* end)
{
    AdamiBoundary((Parameters*)ph, (Parameters*)pd, (float4*)pos, (float4*)vel, (tensor2d*)str, beg, end);
    return (int)cudaDeviceSynchronize();
}

int ref_shepard(void* ph, void* pd, void* pos, void* vel, void* str, void* cache, const int* beg, const int* end)
{
    StressRegularization((Parameters*)ph, (Parameters*)pd, (float4*)pos, (float4*)vel, (tensor2d*)str,
                         (tensor2d*)cache, beg, end);
    return (int)cudaDeviceSynchronize();
}

}
