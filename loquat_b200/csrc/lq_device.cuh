/*
 * LOQUAT-B200 device helpers: cell arithmetic, neighbour-range lookup and
 * the constitutive updates.  Everything here is inlined into the kernels.
 */
#pragma once

#include <cuda_runtime.h>
#include <types.h>
#include "lq_internal.cuh"

namespace lqb {

/* 8-byte accesses of a 24-byte tensor2d (the widest aligned access). */
__device__ __forceinline__ tensor2d load_t2(const tensor2d* p, int i)
{
    const float2* q = reinterpret_cast<const float2*>(p) + 3 * (size_t)i;
    float2 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
    return make_tensor2d(a.x, a.y, b.x, b.y, c.x, c.y);
}

__device__ __forceinline__ tensor2d load_t2_rw(const tensor2d* p, int i)
{
    const float2* q = reinterpret_cast<const float2*>(p) + 3 * (size_t)i;
    float2 a = q[0], b = q[1], c = q[2];
    return make_tensor2d(a.x, a.y, b.x, b.y, c.x, c.y);
}

__device__ __forceinline__ void store_t2(tensor2d* p, int i, const tensor2d& t)
{
    float2* q = reinterpret_cast<float2*>(p) + 3 * (size_t)i;
    q[0] = make_float2(t.xx, t.yy);
    q[1] = make_float2(t.zz, t.xy);
    q[2] = make_float2(t.xz, t.yz);
}

/* Cell coordinate along one axis: floor((0.5 x) / h) from the raw
 * coordinate (reference src/adami_boundary.cu:80-82).  Returns -1 outside
 * [0, n) and for NaN. */
__device__ __forceinline__ int cell_axis(float x, float i_h, int n)
{
    float s = floorf(0.5f * x * i_h);
    return (s >= 0.0f && s < (float)n) ? (int)s : -1;
}

/* Coordinate used as the centre of a 27-cell stencil.  Values far outside
 * the lattice (and NaN) are clamped to -2 or 2^30 so that neighbour offsets
 * cannot overflow; such stencils touch no cell. */
__device__ __forceinline__ int stencil_axis(float x, float i_h)
{
    const float s = floorf(0.5f * x * i_h);
    return (int)fminf(fmaxf(s, -2.0f), 1073741824.0f);
}

/* Grid row of a particle's local y cell under per-object frames: returns
 * -1 when the local cell is outside its object's rows. */
__device__ __forceinline__ int frame_row(const Frames& fr, float id, int cy_local)
{
    int k = (int)id;
    k = k < 0 ? 0 : (k >= fr.n ? fr.n - 1 : k);
    const int base = __ldg(fr.rows + 2 * k), rows = __ldg(fr.rows + 2 * k + 1);
    return (cy_local >= 0 && cy_local < rows) ? base + cy_local : -1;
}

/* Stencil centre row under frames (clamped like stencil_axis). */
__device__ __forceinline__ int frame_stencil_row(const Frames& fr, float id, int cy_local)
{
    int k = (int)id;
    k = k < 0 ? 0 : (k >= fr.n ? fr.n - 1 : k);
    const int base = __ldg(fr.rows + 2 * k), rows = __ldg(fr.rows + 2 * k + 1);
    /* a stencil centred outside the object's rows touches none of them */
    if (cy_local < -1 || cy_local > rows) return -2;
    return base + cy_local;
}

/* The particles of the three cells (X, Y, zlo..zhi) of one layer are one
 * contiguous slot range because keys are z-fastest and the sort is by key.
 * Returns false when the range is empty. */
__device__ __forceinline__ bool zrun_range(const Cells& c, int base, int zlo, int zhi, int& s, int& e)
{
    if (c.start) {
        s = __ldg(c.start + base + zlo);
        e = __ldg(c.start + base + zhi + 1);
        return e > s;
    }
    s = -1;
    for (int z = zlo; z <= zhi; ++z) {
        int b = __ldg(c.beg + base + z);
        if (b != -1) {
            if (s < 0) s = b;
            e = __ldg(c.end + base + z);
        }
    }
    return s >= 0;
}

/* Jaumann co-rotational term with spin (W_yx, W_zx, W_zy)
 * (reference src/predictor_corrector.cu:40-45). */
__device__ __forceinline__ tensor2d jaumann(const float4& w, const tensor2d& s)
{
    tensor2d r;
    r.xx = -2.0f * (w.x * s.xy + w.y * s.xz);
    r.yy = 2.0f * (w.x * s.xy - w.z * s.yz);
    r.zz = 2.0f * (w.y * s.xz + w.z * s.yz);
    r.xy = w.x * (s.xx - s.yy) - w.z * s.xz - w.y * s.yz;
    r.xz = w.y * (s.xx - s.zz) + w.z * s.xy - w.x * s.yz;
    r.yz = w.z * (s.yy - s.zz) + w.x * s.xz + w.y * s.xy;
    return r;
}

struct Material {
    int model;
    float p1, p2, p3, p4, p5;
};

__device__ __forceinline__ Material load_material(const Parameters* P)
{
    Material m;
    m.model = __ldg(&P->constitutive_model);
    m.p1 = __ldg(&P->model_par_1);
    m.p2 = __ldg(&P->model_par_2);
    m.p3 = __ldg(&P->model_par_3);
    m.p4 = __ldg(&P->model_par_4);
    m.p5 = __ldg(&P->model_par_5);
    return m;
}

/* The material of a particle with object id `id` (see MaterialTable). */
__device__ __forceinline__ Material particle_material(const Material& base, const MaterialTable& mt, float id)
{
    if (!mt.p) return base;
    int k = (int)id;
    k = k < 0 ? 0 : (k >= mt.n ? mt.n - 1 : k);
    const float* r = mt.p + 5 * k;
    Material m = base;
    m.p1 = __ldg(r + 0);
    m.p2 = __ldg(r + 1);
    m.p3 = __ldg(r + 2);
    m.p4 = __ldg(r + 3);
    m.p5 = __ldg(r + 4);
    return m;
}

/* Drucker-Prager: elastic trial with Jaumann rate, tension cut-off, radial
 * return to the cone (reference src/predictor_corrector.cu:30-105).
 * K = p1, G = p2, k_phi = p3, k_psi = p4, k_c = p5. */
__device__ __forceinline__ void dp_update(const Material& M, float dtp, const float4& w, const tensor2d& d,
                                          float& p, float& ep, tensor2d& s)
{
    const float K = M.p1, G = M.p2, kphi = M.p3, kpsi = M.p4, kc = M.p5;
    tensor2d r = jaumann(w, s);
    r = r + d * (2.0f * G);
    float ace = (K - 2.0f / 3.0f * G) * (d.xx + d.yy + d.zz);
    r.xx += ace;
    r.yy += ace;
    r.zz += ace;
    s = s + r * dtp;

    float sm = (s.xx + s.yy + s.zz) / 3.0f;
    s.xx -= sm;
    s.yy -= sm;
    s.zz -= sm;

    float tenf = (kphi == 0.0f) ? 0.0f : kc / kphi;
    float over = sm - tenf;                      /* tension cut-off */
    if (over >= 0.0f) {
        float dl = over / K;
        sm = tenf;
        ep += dl * (1.0f / 3.0f) * sqrtf(2.0f);
    }
    float tau = sqrtf(0.5f * J2(s));
    float f = tau + kphi * sm - kc;              /* shear yield function */
    if (f > 0.0f) {
        float dl = f / (G + K * kphi * kpsi);
        sm -= K * kpsi * dl;
        float ratio = tau < 1e-10f ? 1.0f : (kc - kphi * sm) / tau;
        s.xx *= ratio;
        s.yy *= ratio;
        s.zz *= ratio;
        s.xy *= ratio;
        s.xz *= ratio;
        s.yz *= ratio;
        ep += dl * sqrtf(1.0f / 3.0f + 2.0f / 9.0f * kpsi * kpsi);
    }
    s.xx += sm;
    s.yy += sm;
    s.zz += sm;
    p = -sm;
}

/* Four-parameter hypoplastic rate (c1..c4 = p1..p4, cohesion = p5) with the
 * Jaumann term, cohesion shift and tension cap
 * (reference src/predictor_corrector.cu:111-165).  The near-zero-stress
 * reset leaves T_xz as it is, as the reference does. */
__device__ __forceinline__ void hypo_update(const Material& M, float dtp, const tensor2d& d, const float4& w,
                                            tensor2d& s)
{
    const float c1 = M.p1, c2 = M.p2, c3 = M.p3, c4 = M.p4, coh = M.p5;
    tensor2d jau = jaumann(w, s);
    tensor2d T = s;
    if (coh > 0.0f) {
        T.xx -= coh;
        T.yy -= coh;
        T.zz -= coh;
    }
    float t1 = T.xx + T.yy + T.zz;
    if (fabsf(t1) < 4.0f) {
        t1 = -4.0f;
        T.xx = -1.0f;
        T.yy = -1.0f;
        T.zz = -2.0f;
        T.xy = 0.0f;
        T.yz = 0.0f;
    }
    tensor2d Ts = T;
    Ts.xx -= t1 / 3.0f;
    Ts.yy -= t1 / 3.0f;
    Ts.zz -= t1 / 3.0f;
    float d1 = d.xx + d.yy + d.zz;
    float td = J2(T, d);
    float nd = sqrtf(J2(d));
    tensor2d rate = jau + d * (c1 * t1) + T * (c2 * d1 + c3 * td / t1) + (T + Ts) * (c4 * nd);
    s = s + rate * dtp;
    float pres = (s.xx + s.yy + s.zz) / 3.0f;
    if (pres > coh) {
        s.xx -= (pres - coh);
        s.yy -= (pres - coh);
        s.zz -= (pres - coh);
    }
}

/* ---------------------------------------------- FP64 stress updates */
/* The same updates in double precision, for the mixed-precision form: the
 * return map's plastic multiplier and the hypoplastic rate are formed and
 * applied in FP64, and only the stored result is rounded to float. */
struct T6d {
    double xx, yy, zz, xy, xz, yz;
};

__device__ __forceinline__ T6d widen6(const tensor2d& t) { return T6d{t.xx, t.yy, t.zz, t.xy, t.xz, t.yz}; }

__device__ __forceinline__ tensor2d narrow6(const T6d& t)
{
    return make_tensor2d((float)t.xx, (float)t.yy, (float)t.zz, (float)t.xy, (float)t.xz, (float)t.yz);
}

__device__ __forceinline__ double contract6(const T6d& a, const T6d& b)
{
    return a.xx * b.xx + a.yy * b.yy + a.zz * b.zz + 2.0 * (a.xy * b.xy + a.xz * b.xz + a.yz * b.yz);
}

__device__ __forceinline__ T6d jaumann_d(const float4& w4, const T6d& s)
{
    const double wx = w4.x, wy = w4.y, wz = w4.z;
    T6d r;
    r.xx = -2.0 * (wx * s.xy + wy * s.xz);
    r.yy = 2.0 * (wx * s.xy - wz * s.yz);
    r.zz = 2.0 * (wy * s.xz + wz * s.yz);
    r.xy = wx * (s.xx - s.yy) - wz * s.xz - wy * s.yz;
    r.xz = wy * (s.xx - s.zz) + wz * s.xy - wx * s.yz;
    r.yz = wz * (s.yy - s.zz) + wx * s.xz + wy * s.xy;
    return r;
}

__device__ __forceinline__ void dp_update_d(const Material& M, double dtp, const float4& w, const T6d& d, double& p,
                                            double& ep, T6d& s)
{
    const double K = M.p1, G = M.p2, kphi = M.p3, kpsi = M.p4, kc = M.p5;
    T6d r = jaumann_d(w, s);
    const double ace = (K - 2.0 / 3.0 * G) * (d.xx + d.yy + d.zz);
    r.xx += 2.0 * G * d.xx + ace;
    r.yy += 2.0 * G * d.yy + ace;
    r.zz += 2.0 * G * d.zz + ace;
    r.xy += 2.0 * G * d.xy;
    r.xz += 2.0 * G * d.xz;
    r.yz += 2.0 * G * d.yz;
    s.xx += r.xx * dtp; s.yy += r.yy * dtp; s.zz += r.zz * dtp;
    s.xy += r.xy * dtp; s.xz += r.xz * dtp; s.yz += r.yz * dtp;
    double sm = (s.xx + s.yy + s.zz) / 3.0;
    s.xx -= sm; s.yy -= sm; s.zz -= sm;
    const double tenf = (M.p3 == 0.0f) ? 0.0 : kc / kphi;
    const double over = sm - tenf;
    if (over >= 0.0) {
        ep += over / K * (1.0 / 3.0) * sqrt(2.0);
        sm = tenf;
    }
    const double tau = sqrt(0.5 * contract6(s, s));
    const double f = tau + kphi * sm - kc;
    if (f > 0.0) {
        const double dl = f / (G + K * kphi * kpsi);
        sm -= K * kpsi * dl;
        const double ratio = tau < (double)1e-10f ? 1.0 : (kc - kphi * sm) / tau;
        s.xx *= ratio; s.yy *= ratio; s.zz *= ratio;
        s.xy *= ratio; s.xz *= ratio; s.yz *= ratio;
        ep += dl * sqrt(1.0 / 3.0 + 2.0 / 9.0 * kpsi * kpsi);
    }
    s.xx += sm; s.yy += sm; s.zz += sm;
    p = -sm;
}

__device__ __forceinline__ void hypo_update_d(const Material& M, double dtp, const T6d& d, const float4& w, T6d& s)
{
    const double c1 = M.p1, c2 = M.p2, c3 = M.p3, c4 = M.p4, coh = M.p5;
    const T6d jau = jaumann_d(w, s);
    T6d T = s;
    if (M.p5 > 0.0f) {
        T.xx -= coh; T.yy -= coh; T.zz -= coh;
    }
    double t1 = T.xx + T.yy + T.zz;
    if (fabs(t1) < 4.0) {
        t1 = -4.0;
        T.xx = -1.0; T.yy = -1.0; T.zz = -2.0;
        T.xy = 0.0; T.yz = 0.0;   /* T.xz kept, as the reference does */
    }
    const double d1 = d.xx + d.yy + d.zz;
    const double td = contract6(T, d);
    const double nd = sqrt(contract6(d, d));
    const double a = c2 * d1 + c3 * td / t1, b = c4 * nd, c = c1 * t1;
    const double third = t1 / 3.0;
    s.xx += (jau.xx + d.xx * c + T.xx * a + (2.0 * T.xx - third) * b) * dtp;
    s.yy += (jau.yy + d.yy * c + T.yy * a + (2.0 * T.yy - third) * b) * dtp;
    s.zz += (jau.zz + d.zz * c + T.zz * a + (2.0 * T.zz - third) * b) * dtp;
    s.xy += (jau.xy + d.xy * c + T.xy * a + 2.0 * T.xy * b) * dtp;
    s.xz += (jau.xz + d.xz * c + T.xz * a + 2.0 * T.xz * b) * dtp;
    s.yz += (jau.yz + d.yz * c + T.yz * a + 2.0 * T.yz * b) * dtp;
    const double pres = (s.xx + s.yy + s.zz) / 3.0;
    if (pres > coh) {
        s.xx -= pres - coh; s.yy -= pres - coh; s.zz -= pres - coh;
    }
}

}  // namespace lqb
