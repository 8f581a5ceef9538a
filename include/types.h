/*
 * LOQUAT-B200: plain-old-data types shared by the host and every kernel.
 *
 * Drop-in contract: `tensor2d` and `Parameters` are layout-identical to the
 * reference's `include/types.h:36-38` and `include/types.h:89-155`, so a caller
 * compiled against the reference headers passes the same bytes.  Field names,
 * order and types are fixed by that ABI; everything else here is this
 * project's own code.
 *
 *   tensor2d   : 6 x float = 24 bytes, symmetric second-order tensor stored
 *                (xx, yy, zz, xy, xz, yz).  Arrays of it have a 24-byte stride,
 *                so the widest aligned vector access is 8 bytes.
 *   Parameters : 52 four-byte fields = 208 bytes, no padding.
 */
#pragma once
#ifndef LOQUAT_B200_TYPES_H
#define LOQUAT_B200_TYPES_H

#ifndef PI
#define PI (3.14159265358979323846f)
#endif

#include <ctime>
#include <cuda_runtime.h>

typedef struct {
    float xx, yy, zz, xy, xz, yz;
} tensor2d;

static __inline__ __host__ __device__ tensor2d make_tensor2d(float v)
{
    tensor2d t;
    t.xx = v; t.yy = v; t.zz = v; t.xy = v; t.xz = v; t.yz = v;
    return t;
}

static __inline__ __host__ __device__ tensor2d make_tensor2d(float a, float b, float c,
                                                             float d, float e, float f)
{
    tensor2d t;
    t.xx = a; t.yy = b; t.zz = c; t.xy = d; t.xz = e; t.yz = f;
    return t;
}

static __inline__ __host__ __device__ tensor2d operator+(const tensor2d& a, const tensor2d& b)
{
    return make_tensor2d(a.xx + b.xx, a.yy + b.yy, a.zz + b.zz, a.xy + b.xy, a.xz + b.xz, a.yz + b.yz);
}

static __inline__ __host__ __device__ tensor2d operator-(const tensor2d& a, const tensor2d& b)
{
    return make_tensor2d(a.xx - b.xx, a.yy - b.yy, a.zz - b.zz, a.xy - b.xy, a.xz - b.xz, a.yz - b.yz);
}

static __inline__ __host__ __device__ tensor2d operator*(const tensor2d& a, const float& s)
{
    return make_tensor2d(a.xx * s, a.yy * s, a.zz * s, a.xy * s, a.xz * s, a.yz * s);
}

static __inline__ __host__ __device__ tensor2d operator/(const tensor2d& a, const float& s)
{
    return make_tensor2d(a.xx / s, a.yy / s, a.zz / s, a.xy / s, a.xz / s, a.yz / s);
}

static __inline__ __host__ __device__ float trace(const tensor2d& a)
{
    return a.xx + a.yy + a.zz;
}

/* Full contraction a:a of a symmetric tensor (off-diagonals counted twice).
 * The reference (include/types.h:77-80) writes the factor 2 as a double
 * literal, so the diagonal part is summed in float and the off-diagonal
 * part is accumulated in double before the result is rounded to float.
 * That evaluation order is kept because the Drucker-Prager yield test and
 * the hypoplastic norm depend on it. */
static __inline__ __host__ __device__ float J2(const tensor2d& a)
{
    float diag = a.xx * a.xx + a.yy * a.yy + a.zz * a.zz;
    double s = (double)diag;
    s += 2.0 * a.xy * a.xy;
    s += 2.0 * a.xz * a.xz;
    s += 2.0 * a.yz * a.yz;
    return (float)s;
}

/* Full contraction a:b, same evaluation order as J2(a). */
static __inline__ __host__ __device__ float J2(const tensor2d& a, const tensor2d& b)
{
    float diag = a.xx * b.xx + a.yy * b.yy + a.zz * b.zz;
    double s = (double)diag;
    s += 2.0 * a.xy * b.xy;
    s += 2.0 * a.xz * b.xz;
    s += 2.0 * a.yz * b.yz;
    return (float)s;
}

typedef struct {
    int np;                 /* total particles                                  */
    int npb;                /* boundary (Adami dummy) particles, stored first   */
    int npm;                /* material particles, stored after the boundary    */
    int np_delete;          /* deleted particles (kept for layout)              */

    float domain_size_x;
    float domain_size_y;
    float domain_size_z;

    float domain_min_x;
    float domain_min_y;
    float domain_min_z;

    int cell_num_x;         /* cells per axis, cell edge = 2h                   */
    int cell_num_y;
    int cell_num_z;
    int ncell;              /* 2 * ncell_one_layer + 1                          */
    int ncell_one_layer;    /* cells of one layer (boundary or material)        */
    int ncell_delete;       /* key of particles outside the domain = ncell - 1  */

    float h;                /* smoothing length                                 */
    float i_h;              /* 1 / h                                            */
    float eta;              /* 0.01 h^2, viscosity singularity guard            */
    float dr;               /* particle spacing                                 */
    float hdr;              /* h / dr                                           */

    float m;                /* particle mass = dr^3 rho0                        */
    float cs;               /* speed of sound                                   */
    float cfl;              /* CFL number                                       */
    float rho0;             /* reference density                                */

    int constitutive_model; /* 1 Drucker-Prager, 2 hypoplastic                  */
    float model_par_1;
    float model_par_2;
    float model_par_3;
    float model_par_4;
    float model_par_5;

    int density_shepard_filter;
    int stress_shepard_filter;
    int dynamic_time_step;
    int integration_method;
    int viscosity_type;
    float artificial_viscosity_alpha;

    int artificial_pressure;
    float artificial_pressure_coefficient;

    float acc_x;
    float acc_y;
    float acc_z;

    float time_max;
    float time;
    float dt;
    float output_frequency;
    int output_number;

    float kernel_normalization_par;           /* Wendland C2: 42 / (256 pi h^3)   */
    float kernel_gradient_normalization_par;  /* -5 * 42 / (256 pi h^5)           */

    float kernel_zero;      /* W(0)                                             */
    float kernel_dr;        /* W(dr)                                            */

    int output_format;      /* 1 .dat, 2 .vtu                                   */
} Parameters;

typedef struct {
    double total;
    double neighbor_search;
    double adami_boundary;
    double interaction;
    double integration;
    double saving;

    std::clock_t clock_initial;
    std::clock_t clock_neighbor_search;
    std::clock_t clock_adami_boundary;
    std::clock_t clock_interaction;
    std::clock_t clock_integration;
    std::clock_t clock_saving;
    std::clock_t clock_interval;
} Timer;

#endif /* LOQUAT_B200_TYPES_H */
