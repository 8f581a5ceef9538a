/* The mixed form's packed neighbour velocity, shared by the device kernels
 * that write and read it (sph.cu: store_packed, pair_terms) and by host
 * code that checks it.  No CUDA types: the header compiles with a plain
 * C++ compiler too.
 *
 * A velocity (vx, vy, vz) goes into two 32-bit words as one shared
 * exponent and three signed 18-bit mantissas.  The quantum is
 * q = 2^(E - 17) for the least E with max |v_k| < 2^E, E raised once more
 * if a component rounds to 2^17 q, and never below -109 (q stays a normal
 * float); each component becomes m_k q with m_k = v_k / q rounded to
 * nearest even, so its error is at most q / 2, 2^-18 of the largest
 * component's binade (a 16-bit float would leave 2^-11 of each
 * component's own).  The pair sums use the neighbour's velocity through
 * differences v_i - v_j of nearly equal velocities, which is why a shared
 * scale with long mantissas serves them better than three short floats.
 *
 * Layout, with offset-binary mantissas u_k = m_k + 2^17 in [0, 2^18):
 *   w0 = ux in bits 0-17, bits 0-13 of uz in bits 18-31;
 *   w1 = bits 14-17 of uz in bits 0-3, uy in bits 4-21, bit 22 zero, q's
 *        FP32 exponent field in bits 23-30 (so w1 & 0x7F800000 read as a
 *        float is q), bit 31 zero.
 * The decode ORs each u_k into the bits of 2^23 (giving the float
 * 2^23 + u_k) and takes one FMA, (2^23 + u_k) q - (2^23 + 2^17) q = m_k q,
 * exact: ten instructions and no integer-to-float conversion.  A
 * non-finite velocity packs to q = inf and decodes to NaN. */
#pragma once

#include <cmath>
#include <cstring>

#if defined(__CUDACC__)
#define LQ_PACK_HD __host__ __device__ __forceinline__
#else
#define LQ_PACK_HD inline
#endif

namespace lqb {

LQ_PACK_HD unsigned pack_bits(float f)
{
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    unsigned u;
    std::memcpy(&u, &f, sizeof u);
    return u;
#endif
}

LQ_PACK_HD float pack_float(unsigned u)
{
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f;
    std::memcpy(&f, &u, sizeof f);
    return f;
#endif
}

/* (w0, w1) of the layout above. */
LQ_PACK_HD void pack_velocity_words(float vx, float vy, float vz, unsigned& w0, unsigned& w1)
{
    const float m = fmaxf(fabsf(vx), fmaxf(fabsf(vy), fabsf(vz)));
    if (!(fabsf(vx) <= 3.0e38f && fabsf(vy) <= 3.0e38f && fabsf(vz) <= 3.0e38f)) {   /* inf or NaN */
        w0 = 0u;
        w1 = 0x7F800000u;
        return;
    }
    int e;
    frexpf(m, &e);                  /* m < 2^e (e = 0 for m = 0) */
    if (e < -109) e = -109;
    float mx = rintf(ldexpf(vx, 17 - e)), my = rintf(ldexpf(vy, 17 - e)), mz = rintf(ldexpf(vz, 17 - e));
    if (fmaxf(mx, fmaxf(my, mz)) > 131071.0f) {     /* a component rounded to 2^17 q */
        ++e;
        mx = rintf(ldexpf(vx, 17 - e));
        my = rintf(ldexpf(vy, 17 - e));
        mz = rintf(ldexpf(vz, 17 - e));
    }
    const unsigned ux = (unsigned)((int)mx + 131072), uy = (unsigned)((int)my + 131072),
                   uz = (unsigned)((int)mz + 131072);
    w0 = ux | (uz << 18);
    w1 = (uz >> 14) | (uy << 4) | ((unsigned)(e - 17 + 127) << 23);
}

/* The velocity (vx, vy, vz) that (w0, w1) hold. */
LQ_PACK_HD void unpack_velocity_words(unsigned w0, unsigned w1, float& vx, float& vy, float& vz)
{
    const float q = pack_float(w1 & 0x7F800000u);
    const float c = -8519680.0f * q;                       /* -(2^23 + 2^17) q */
    const unsigned uz = ((w0 >> 18) | (w1 << 14)) & 0x3FFFFu;
    vx = fmaf(pack_float((w0 & 0x3FFFFu) | 0x4B000000u), q, c);
    vy = fmaf(pack_float(((w1 >> 4) & 0x3FFFFu) | 0x4B000000u), q, c);
    vz = fmaf(pack_float(uz | 0x4B000000u), q, c);
}

}  // namespace lqb
