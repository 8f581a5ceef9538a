/*
 * LOQUAT-B200 device helpers: cell arithmetic, neighbour-range lookup and
 * the constitutive updates.  Everything here is inlined into the kernels.
 */
#pragma once

#include <cstdio>

#include <cuda_runtime.h>
#include <types.h>
#include "lq_internal.cuh"
#include "lq_pack.h"

namespace lqb {

/* Bounds-checked builds (-D LQ_CHECKED): the list and grid kernels check
 * every index they gather or scatter through before the access; a
 * violation is counted in this translation unit's counter and the access is
 * skipped.  This stands in for a device memory checker.  In the product
 * build the check is a constant true and compiles away. */
#ifdef LQ_CHECKED
static __device__ unsigned long long lq_bounds_count;
__device__ __forceinline__ bool lq_in_range_at(long long j, long long n, int line)
{
    if (j >= 0 && j < n) return true;
    /* the first few violations name their source line */
    if (atomicAdd(&lq_bounds_count, 1ull) < 4ull)
        printf("LQ_CHECKED: bounds violation at line %d: index %lld, limit %lld\n", line, j, n);
    return false;
}
#define lq_in_range(j, n) lq_in_range_at((long long)(j), (long long)(n), __LINE__)
#else
__device__ __forceinline__ constexpr bool lq_in_range(long long, long long) { return true; }
#endif

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

/* A double from float high and low words, and back: hi is the value
 * rounded to float, lo the float rounding of what hi leaves out. */
__device__ __forceinline__ double4 join4(const float4& hi, const float4& lo)
{
    return make_double4((double)hi.x + (double)lo.x, (double)hi.y + (double)lo.y, (double)hi.z + (double)lo.z,
                        (double)hi.w + (double)lo.w);
}

__device__ __forceinline__ void split4(const double4& d, float4& hi, float4& lo)
{
    hi = make_float4((float)d.x, (float)d.y, (float)d.z, (float)d.w);
    lo = make_float4((float)(d.x - (double)hi.x), (float)(d.y - (double)hi.y), (float)(d.z - (double)hi.z),
                     (float)(d.w - (double)hi.w));
}

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

/* ------------------------------------ von Wolffersdorff (model 3) */
/* Hypoplasticity with a predefined limit-state surface (von Wolffersdorff
 * 1996), tension positive, integrated in FP64 by explicit sub-steps (Euler /
 * Heun pair with the relative stress difference kept below tol); not in the
 * reference.  Row: phic (deg), hs, n, ed0, ec0, ei0, alpha, beta, tol,
 * max sub-steps.  Equations:
 *   Tdot = fb fe / (That:That) [F^2 D + a^2 That (That:D) + fd a F (That + That*) |D|] + Jaumann
 *   with That = T/trT, a = sqrt3 (3 - sin phic) / (2 sqrt2 sin phic),
 *   F from tan psi = sqrt3 |That*| and cos3theta, e_x = e_x0 exp(-(-trT/hs)^n),
 *   fe = (ec/e)^beta, fd = ((e-ed)/(ec-ed))^alpha, edot = (1+e) tr D.
 * Stresses with tr T > -3 Pa are replaced by -1 Pa isotropic before the
 * rate is formed; where tan psi exceeds sqrt2 (F undefined: a tensile
 * principal direction) the deviator of That is scaled back to
 * tan psi = sqrt2 (1 - 1e-3) at the same mean stress. */
struct VWConst {
    double a, a2, fbk, lnhs, ihs, n, ed0, ec0, lnec0, ei0, alpha, beta, tol;
    int maxsub;
};

/* Row constants; the powers of constants are formed once here:
 * fbk = (hs / n) (ei0 / ec0)^beta / (3 + a^2 - a sqrt3 ((ei0 - ed0) / (ec0 - ed0))^alpha). */
__device__ __forceinline__ VWConst vw_const(const MaterialTable& mt, float id)
{
    int k = (int)id;
    k = k < 0 ? 0 : (k >= mt.n ? mt.n - 1 : k);
    const float* r = mt.p + 10 * k;
    VWConst c;
    const double phic = (double)__ldg(r) * 3.14159265358979323846 / 180.0;
    const double sphi = sin(phic);
    const double hs = __ldg(r + 1);
    c.a = sqrt(3.0) * (3.0 - sphi) / (2.0 * sqrt(2.0) * sphi);
    c.a2 = c.a * c.a;
    c.n = __ldg(r + 2);
    c.ed0 = __ldg(r + 3);
    c.ec0 = __ldg(r + 4);
    c.ei0 = __ldg(r + 5);
    c.alpha = __ldg(r + 6);
    c.beta = __ldg(r + 7);
    c.tol = __ldg(r + 8);
    c.maxsub = (int)__ldg(r + 9);
    c.lnhs = log(hs);
    c.ihs = 1.0 / hs;
    c.lnec0 = log(c.ec0);
    const double den = 3.0 + c.a2 - c.a * sqrt(3.0) * pow((c.ei0 - c.ed0) / (c.ec0 - c.ed0), c.alpha);
    c.fbk = (hs / c.n) * pow(c.ei0 / c.ec0, c.beta) / den;
    return c;
}

__device__ __forceinline__ double trace_cube6(const T6d& A)
{
    return A.xx * A.xx * A.xx + A.yy * A.yy * A.yy + A.zz * A.zz * A.zz +
           3.0 * (A.xy * A.xy * (A.xx + A.yy) + A.xz * A.xz * (A.xx + A.zz) + A.yz * A.yz * (A.yy + A.zz)) +
           6.0 * A.xy * A.xz * A.yz;
}

/* The rate with the state-dependent powers through shared logarithms:
 * pr = -trT/hs, pr^n = exp(n ln pr), pr^(1-n) = pr / pr^n, ex = exp(-pr^n),
 * fe = exp(beta (ln ec0 - pr^n - ln e)), fd = exp(alpha ln((e - ed) / (ec - ed))).
 * The stretching d stays in float (it is read as float) and the deviator
 * That* is formed from That where needed, to spare registers. */
__device__ __forceinline__ void vw_rate_d(const VWConst& c, const T6d& Tin, double e, const tensor2d& d,
                                          const float4& w, T6d& R, double& edot)
{
    T6d Th = Tin;
    double trT = Th.xx + Th.yy + Th.zz;
    if (!(trT < -3.0)) {
        Th = T6d{-1.0, -1.0, -1.0, 0.0, 0.0, 0.0};
        trT = -3.0;
    }
    const double it = 1.0 / trT;
    Th = T6d{Th.xx * it, Th.yy * it, Th.zz * it, Th.xy * it, Th.xz * it, Th.yz * it};
    const double third = 1.0 / 3.0;
    /* That* = That - I/3: the off-diagonal parts are That's */
    double sxx = Th.xx - third, syy = Th.yy - third, szz = Th.zz - third;
    double TsTs = sxx * sxx + syy * syy + szz * szz + 2.0 * (Th.xy * Th.xy + Th.xz * Th.xz + Th.yz * Th.yz);
    double tpsi = sqrt(3.0 * TsTs);
    const double lim = sqrt(2.0) * (1.0 - 1e-3);
    if (tpsi > lim) {
        const double f = lim / tpsi;
        sxx *= f; syy *= f; szz *= f;
        Th = T6d{sxx + third, syy + third, szz + third, Th.xy * f, Th.xz * f, Th.yz * f};
        TsTs *= f * f;
        tpsi = lim;
    }
    const double ThTh = contract6(Th, Th);
    double c3t = 1.0;
    if (TsTs > 1e-30) {
        const T6d Ts{sxx, syy, szz, Th.xy, Th.xz, Th.yz};
        c3t = -sqrt(6.0) * trace_cube6(Ts) / (TsTs * sqrt(TsTs));
    }
    c3t = fmax(-1.0, fmin(1.0, c3t));
    const double F = sqrt(fmax(tpsi * tpsi / 8.0 + (2.0 - tpsi * tpsi) / (2.0 + sqrt(2.0) * tpsi * c3t), 0.0)) -
                     tpsi / (2.0 * sqrt(2.0));
    const double lnpr = log(-trT) - c.lnhs;
    const double prn = exp(c.n * lnpr);
    const double ex = exp(-prn);
    const double ei = c.ei0 * ex, ec = c.ec0 * ex, ed = c.ed0 * ex;
    const double fe = exp(c.beta * (c.lnec0 - prn - log(e)));
    const double q = (e - ed) / (ec - ed);
    const double fd = q > 0.0 ? exp(c.alpha * log(q)) : (c.alpha == 0.0 ? 1.0 : 0.0);
    const double fb = c.fbk * (1.0 + 1.0 / ei) * (-trT * c.ihs) / prn;
    const double dxx = d.xx, dyy = d.yy, dzz = d.zz, dxy = d.xy, dxz = d.xz, dyz = d.yz;
    const double ThD = Th.xx * dxx + Th.yy * dyy + Th.zz * dzz + 2.0 * (Th.xy * dxy + Th.xz * dxz + Th.yz * dyz);
    const double nD = sqrt(dxx * dxx + dyy * dyy + dzz * dzz + 2.0 * (dxy * dxy + dxz * dxz + dyz * dyz));
    const double k0 = fb * fe / ThTh;
    const double F2 = F * F, nf = fd * c.a * F * nD;
    const T6d J = jaumann_d(w, Tin);
    R.xx = k0 * (F2 * dxx + c.a2 * Th.xx * ThD + nf * (Th.xx + sxx)) + J.xx;
    R.yy = k0 * (F2 * dyy + c.a2 * Th.yy * ThD + nf * (Th.yy + syy)) + J.yy;
    R.zz = k0 * (F2 * dzz + c.a2 * Th.zz * ThD + nf * (Th.zz + szz)) + J.zz;
    R.xy = k0 * (F2 * dxy + c.a2 * Th.xy * ThD + nf * (2.0 * Th.xy)) + J.xy;
    R.xz = k0 * (F2 * dxz + c.a2 * Th.xz * ThD + nf * (2.0 * Th.xz)) + J.xz;
    R.yz = k0 * (F2 * dyz + c.a2 * Th.yz * ThD + nf * (2.0 * Th.yz)) + J.yz;
    edot = (1.0 + e) * (dxx + dyy + dzz);
}

/* Adaptive explicit integration over dt; returns the number of sub-steps.
 * The loop has one rate evaluation site (inlined once): each pass evaluates
 * either the first rate k1 of a trial at (s, e) or the second, k2, at the
 * Euler point s + h k1.  The Heun result is s + h/2 (k1 + k2) and its
 * difference from the Euler point, h/2 (k2 - k1), is the error estimate; a
 * rejected trial keeps its k1. */
__device__ __forceinline__ int vw_update_d(const VWConst& c, double dt, const tensor2d& d, const float4& w, T6d& s,
                                           double& e)
{
    double t = 0.0, h = dt;
    int steps = 0;
    T6d k1{}, x = s;
    double ke1 = 0.0, xe = e;
    bool have_k1 = false;
    while (t < dt) {
        T6d r;
        double re;
        vw_rate_d(c, x, xe, d, w, r, re);
        if (!have_k1) {
            k1 = r;
            ke1 = re;
            have_k1 = true;
        } else {
            const double hh = 0.5 * h;
            const T6d s2{s.xx + hh * (k1.xx + r.xx), s.yy + hh * (k1.yy + r.yy), s.zz + hh * (k1.zz + r.zz),
                         s.xy + hh * (k1.xy + r.xy), s.xz + hh * (k1.xz + r.xz), s.yz + hh * (k1.yz + r.yz)};
            const T6d df{hh * (r.xx - k1.xx), hh * (r.yy - k1.yy), hh * (r.zz - k1.zz),
                         hh * (r.xy - k1.xy), hh * (r.xz - k1.xz), hh * (r.yz - k1.yz)};
            const double err = sqrt(contract6(df, df) / fmax(contract6(s2, s2), 1e-30));
            ++steps;
            const bool last = steps >= c.maxsub - 1 || h <= dt * 1e-6;
            if (err <= c.tol || last) {
                s = s2;
                e += hh * (ke1 + re);
                t += h;
                const double g = err > 0.0 ? 0.9 * sqrt(c.tol / err) : 2.0;
                h *= fmin(2.0, fmax(0.2, g));
                have_k1 = false;
                x = s;
                xe = e;
                continue;
            }
            h *= fmax(0.2, 0.9 * sqrt(c.tol / err));
        }
        /* trial from (s, e) with the first rate k1 */
        h = fmin(h, dt - t);
        if (steps >= c.maxsub - 1) h = dt - t;
        x = T6d{s.xx + h * k1.xx, s.yy + h * k1.yy, s.zz + h * k1.zz, s.xy + h * k1.xy, s.xz + h * k1.xz,
                s.yz + h * k1.yz};
        xe = e + h * ke1;
    }
    return steps;
}

/* Packed neighbour data for the list pair kernel: dense arrays over all
 * slots, with s = sigma / rho^2,
 *   nb.xr[j] = (x, y, z, rho), nb.sa[j] = (sxx, syy, szz, sxy),
 *   nb.sb[j] = (sxz, syz, v0, v1),
 * where the plain form keeps (v0, v1) = (vx, vy) and vz in nb.vz[j]
 * (52 bytes per particle, four gathers per pair) and the mixed form packs
 * the whole velocity into v0, v1 (pack_velocity: 48 bytes, three 16-byte
 * gathers per pair).  The pair kernel is bound by the L1 data pipe: a
 * warp's gathered neighbours sit close together in memory and the pipe's
 * work follows the load instructions and the sectors each gathers, so the
 * record holds only the 13 values a pair needs (no pressure word of
 * pospres, no 24-byte stress records read as three 8-byte loads).
 * 1 / rho is formed as the state-array pair body forms it. */
struct NbrArrays {
    float4* xr;
    float4* sa;
    float4* sb;
    float* vz;
};

/* The mixed form's gathered velocity in two words (lq_pack.h: a shared
 * exponent and three 18-bit mantissas). */
__device__ __forceinline__ float2 pack_velocity(float vx, float vy, float vz)
{
    unsigned w0, w1;
    pack_velocity_words(vx, vy, vz, w0, w1);
    return make_float2(__uint_as_float(w0), __uint_as_float(w1));
}

__device__ __forceinline__ float3 unpack_velocity(float v0, float v1)
{
    float3 v;
    unpack_velocity_words(__float_as_uint(v0), __float_as_uint(v1), v.x, v.y, v.z);
    return v;
}

/* One slot's entry of the packed arrays from its velocity, density and
 * stress (the pack kernel and the integrators write it alike; the
 * list-driven Adami rewrites only the stress words, store_packed_stress). */
template <bool kPk>
__device__ __forceinline__ void store_packed(const NbrArrays& nb, int i, const float4& v, const tensor2d& str)
{
    const float rinv = __fdividef(1.0f, v.w);
    const float r2 = rinv * rinv;
    nb.sa[i] = make_float4(str.xx * r2, str.yy * r2, str.zz * r2, str.xy * r2);
    if (kPk) {
        const float2 w = pack_velocity(v.x, v.y, v.z);
        nb.sb[i] = make_float4(str.xz * r2, str.yz * r2, w.x, w.y);
    } else {
        nb.sb[i] = make_float4(str.xz * r2, str.yz * r2, v.x, v.y);
        nb.vz[i] = v.z;
    }
}

/* The stress words of a slot's packed entry (sigma / rho^2, as
 * store_packed writes them); its position, density and velocity words are
 * left as they are. */
__device__ __forceinline__ void store_packed_stress(const NbrArrays& nb, int i, float rho, const tensor2d& str)
{
    const float rinv = __fdividef(1.0f, rho);
    const float r2 = rinv * rinv;
    nb.sa[i] = make_float4(str.xx * r2, str.yy * r2, str.zz * r2, str.xy * r2);
    *reinterpret_cast<float2*>(nb.sb + i) = make_float2(str.xz * r2, str.yz * r2);
}

/* The packed arrays inside `rec` (np x 13 floats, 16-byte aligned). */
inline NbrArrays nbr_arrays(float* rec, int np)
{
    const size_t n = (size_t)np;
    return NbrArrays{reinterpret_cast<float4*>(rec), reinterpret_cast<float4*>(rec) + n,
                     reinterpret_cast<float4*>(rec) + 2 * n, rec + 12 * n};
}

}  // namespace lqb
