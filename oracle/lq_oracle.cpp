/*
 * LOQUAT per-step SPH path: CPU FP64 oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this file.  It is used by tests/, by __graft_entry__.smoke() as the
 * checker, and by bench.py's CPU-baseline leg (--impl reference).
 *
 * It restates, in double precision with OpenMP, the reference's algorithm
 * for one time step (reference src/loquat.cu:322-409):
 *   neighbour grid   contract of src/loquat_grid.h:58-64 as pinned by its
 *                    consumers (src/adami_boundary.cu:80-103)   -> or_grid_*
 *   Adami boundary   src/adami_boundary.cu:27-123               -> adami()
 *   interaction      src/particle_interaction.h:27-40 (closed)  -> interaction()
 *   predictor        src/predictor_corrector.cu:169-218         -> predictor()
 *   corrector        src/predictor_corrector.cu:256-307         -> corrector()
 *   Drucker-Prager   src/predictor_corrector.cu:30-105          -> dp_update()
 *   hypoplastic      src/predictor_corrector.cu:111-165         -> hypo_update()
 *   Shepard filter   src/field_smoothing.cu:65-121              -> shepard()
 *   constants        src/loquat.cu:111-139                      -> or_initialize_parameters()
 *
 * Parity status.  Predictor, corrector, both constitutive models, Adami and
 * Shepard follow open reference code and are pinned against that code's own
 * outputs (golden vectors made by compiling the reference's kernels, see
 * tests/golden/).  The grid contract is pinned by its open consumers.  The
 * particle-interaction pass is closed in the reference (its static library
 * is not distributed), so its formulation below is written from the
 * published weakly-compressible SPH equations for elastoplastic soil:
 * parity of the interaction against the reference is UNPINNED.
 *
 * Array layouts match the product: float4-like arrays are double[n][4],
 * tensor arrays double[n][6] in the order xx yy zz xy xz yz.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

namespace {

/* Mirror of the 208-byte Parameters record (reference include/types.h:89-155). */
struct OrParams {
    int np, npb, npm, np_delete;
    float domain_size_x, domain_size_y, domain_size_z;
    float domain_min_x, domain_min_y, domain_min_z;
    int cell_num_x, cell_num_y, cell_num_z, ncell, ncell_one_layer, ncell_delete;
    float h, i_h, eta, dr, hdr;
    float m, cs, cfl, rho0;
    int constitutive_model;
    float model_par_1, model_par_2, model_par_3, model_par_4, model_par_5;
    int density_shepard_filter, stress_shepard_filter, dynamic_time_step, integration_method, viscosity_type;
    float artificial_viscosity_alpha;
    int artificial_pressure;
    float artificial_pressure_coefficient;
    float acc_x, acc_y, acc_z;
    float time_max, time, dt, output_frequency;
    int output_number;
    float kernel_normalization_par, kernel_gradient_normalization_par;
    float kernel_zero, kernel_dr;
    int output_format;
};
static_assert(sizeof(OrParams) == 208, "Parameters mirror must be 208 bytes");

const float kPiF = 3.14159265358979323846f;

/* ------------------------------------------------------------------ cells */

/* Cell coordinate along one axis, float arithmetic exactly as the device
 * computes it: floorf((0.5f * x) * i_h) (reference src/adami_boundary.cu:80-82).
 * Returns -1 outside [0, n) and for NaN. */
inline int cell_axis_f(float x, float i_h, int n)
{
    float s = std::floor(0.5f * x * i_h);
    if (!(s >= 0.0f) || !(s < (float)n)) return -1;
    return (int)s;
}

inline int cell_axis_d(double x, double i_h, int n)
{
    double s = std::floor(0.5 * x * i_h);
    if (!(s >= 0.0) || !(s < (double)n)) return -1;
    return (int)s;
}

/* Unclamped cell coordinate used to centre a 27-cell stencil. */
inline int stencil_axis_f(float x, float i_h) { return (int)std::floor(0.5f * x * i_h); }
inline int stencil_axis_d(double x, double i_h) { return (int)std::floor(0.5 * x * i_h); }

struct Grid {
    std::vector<int> key, part_idx, part_cel, start, beg, end;
};

/* Stable counting sort by cell key.  Key = layer offset + linear cell id with
 * z fastest (reference src/adami_boundary.cu:99-100); layer 0 holds slots
 * [0, npb), layer 1 holds [npb, np); out-of-lattice particles get
 * ncell_delete (reference src/loquat.cu:123-124). */
void build_grid(const OrParams& P, int np, int npb, const double* pos, bool float_cells, Grid& g)
{
    const int nx = P.cell_num_x, ny = P.cell_num_y, nz = P.cell_num_z;
    const int L = P.ncell_one_layer, ncell = P.ncell;
    g.key.assign(np, 0);
    for (int i = 0; i < np; ++i) {
        int cx, cy, cz;
        if (float_cells) {
            cx = cell_axis_f((float)pos[4 * i + 0], P.i_h, nx);
            cy = cell_axis_f((float)pos[4 * i + 1], P.i_h, ny);
            cz = cell_axis_f((float)pos[4 * i + 2], P.i_h, nz);
        } else {
            cx = cell_axis_d(pos[4 * i + 0], (double)P.i_h, nx);
            cy = cell_axis_d(pos[4 * i + 1], (double)P.i_h, ny);
            cz = cell_axis_d(pos[4 * i + 2], (double)P.i_h, nz);
        }
        int k;
        if (cx < 0 || cy < 0 || cz < 0) k = P.ncell_delete;
        else k = (i < npb ? 0 : L) + (cx * ny + cy) * nz + cz;
        g.key[i] = k;
    }
    g.start.assign(ncell + 1, 0);
    for (int i = 0; i < np; ++i) g.start[g.key[i] + 1]++;
    for (int c = 0; c < ncell; ++c) g.start[c + 1] += g.start[c];
    std::vector<int> fill(g.start.begin(), g.start.end() - 1);
    g.part_idx.assign(np, 0);
    g.part_cel.assign(np, 0);
    for (int i = 0; i < np; ++i) {           /* ascending i: stable */
        int s = fill[g.key[i]]++;
        g.part_idx[s] = i;
        g.part_cel[s] = g.key[i];
    }
    g.beg.assign(ncell, -1);
    g.end.assign(ncell, -1);
    for (int c = 0; c < ncell; ++c) {
        if (g.start[c + 1] > g.start[c]) {
            g.beg[c] = g.start[c];
            g.end[c] = g.start[c + 1];
        }
    }
}

void gather(int np, int width, const int* idx, std::vector<double>& a, std::vector<double>& tmp)
{
    tmp.resize((size_t)np * width);
    for (int i = 0; i < np; ++i)
        for (int k = 0; k < width; ++k) tmp[(size_t)i * width + k] = a[(size_t)idx[i] * width + k];
    a.swap(tmp);
}

/* Visits every candidate j of the 27 cells around (cx, cy, cz) in one layer. */
template <class F>
inline void for_stencil(const OrParams& P, int cx, int cy, int cz, int layer_off,
                        const int* beg, const int* end, F&& f)
{
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                int X = cx + dx, Y = cy + dy, Z = cz + dz;
                if (X < 0 || X > P.cell_num_x - 1 || Y < 0 || Y > P.cell_num_y - 1 || Z < 0 ||
                    Z > P.cell_num_z - 1)
                    continue;
                int c = (X * P.cell_num_y + Y) * P.cell_num_z + Z + layer_off;
                int b = beg[c];
                if (b == -1) continue;
                for (int j = b; j < end[c]; ++j) f(j);
            }
}

inline void stencil_centre(const OrParams& P, const double* xi, bool float_cells, int& cx, int& cy, int& cz)
{
    if (float_cells) {
        cx = stencil_axis_f((float)xi[0], P.i_h);
        cy = stencil_axis_f((float)xi[1], P.i_h);
        cz = stencil_axis_f((float)xi[2], P.i_h);
    } else {
        cx = stencil_axis_d(xi[0], (double)P.i_h);
        cy = stencil_axis_d(xi[1], (double)P.i_h);
        cz = stencil_axis_d(xi[2], (double)P.i_h);
    }
}

inline double wendland(const OrParams& P, double q)
{
    double t = 2.0 - q;
    return (double)P.kernel_normalization_par * t * t * t * t * (q + 0.5);
}

/* ------------------------------------------------------------ Adami (a6) */
/* reference src/adami_boundary.cu:65-123 */
void adami(const OrParams& P, int np, int npb, const double* pos, const double* vel, double* str,
           const int* beg, const int* end, bool float_cells)
{
    (void)np;
    const double ih = P.i_h, m = P.m, rho0 = P.rho0;
    const double g[3] = {P.acc_x, P.acc_y, P.acc_z};
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < npb; ++i) {
        const double* xi = pos + 4 * (size_t)i;
        double S[6] = {0, 0, 0, 0, 0, 0}, Pk[3] = {0, 0, 0}, w = 0;
        int cx, cy, cz;
        stencil_centre(P, xi, float_cells, cx, cy, cz);
        for_stencil(P, cx, cy, cz, P.ncell_one_layer, beg, end, [&](int j) {
            const double* xj = pos + 4 * (size_t)j;
            double d[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
            double q = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) * ih;
            if (q < 2.0) {
                double kv = wendland(P, q) * (m / vel[4 * (size_t)j + 3]);
                for (int k = 0; k < 6; ++k) S[k] += str[6 * (size_t)j + k] * kv;
                for (int k = 0; k < 3; ++k) Pk[k] += d[k] * kv;
                w += kv;
            }
        });
        if (w > 0.0) {
            double* si = str + 6 * (size_t)i;
            for (int k = 0; k < 3; ++k) si[k] = (S[k] - rho0 * g[k] * Pk[k]) / w;
            for (int k = 3; k < 6; ++k) si[k] = S[k] / w;
        }
    }
}

/* ------------------------------------------------------ interaction (a5) */
/* Formulation (weakly compressible SPH for elastoplastic soil, Wendland C2,
 * stress tension-positive); reference interface src/particle_interaction.h:27-40.
 * For material slot i over both layers' 27 cells, j != i, q = |x_ij|/h < 2:
 *   g      = C' (2 - q)^3 x_ij                           (grad_i W_ij)
 *   drho  += m (v_i - v_j) . g
 *   a     += m (sig_i/rho_i^2 + sig_j/rho_j^2) g
 *   a     -= m Pi_ij g,  Pi_ij = -alpha cs mu / rhobar,
 *            mu = h v_ij.x_ij / (r^2 + eta) when v_ij.x_ij < 0   (viscosity_type 1)
 *   a     += m (R_i + R_j) f^4 g (diagonal), R_i,aa = -eps sig_i,aa/rho_i^2 if sig_i,aa > 0,
 *            f = W(q)/W(dr)                                (artificial_pressure 1)
 *   L_ab  += (m/rho_j) (v_j - v_i)_a g_b
 * accad = (a + gravity, drho); acestn = sym L; spin = (W_yx, W_zx, W_zy, 0),
 * W = (L - L^T)/2, the convention the Jaumann code needs
 * (reference src/predictor_corrector.cu:40-45). */
/* Precision experiment (test infrastructure): rounding applied to a
 * neighbour's velocity and sigma/rho^2 as the interaction gathers them,
 * as a GPU form that packed those gathers into 16-bit floats would see
 * them; the target's own values stay exact.  Bit 0: velocity to FP16,
 * bit 1: sigma/rho^2 to FP16, bit 2: velocity to BF16, bit 3: sigma/rho^2
 * to BF16 (round to nearest even); bits 4 and 5: the packed velocity forms
 * of gather_velocity.  0 (the default) rounds nothing. */
int g_gather_rounding = 0;

/* x rounded to nearest even with `bits` significant bits, numbers below
 * 2^emin keeping the quantum of 2^emin (the subnormals of a format whose
 * least normal exponent is emin).  On a float input it equals the FP16
 * (bits 11, emin -14) and BF16 (bits 8, emin -126) conversions for every
 * value below the FP16 maximum, without their software calls on the host. */
inline double round_significand(double x, int bits, int emin)
{
    if (x == 0.0 || !std::isfinite(x)) return x;
    int e;
    std::frexp(x, &e);
    if (e - 1 < emin) e = emin + 1;
    const double q = std::ldexp(1.0, e - bits);
    return std::nearbyint(x / q) * q;
}

inline double gather_round(double x, int f16_bit, int bf16_bit)
{
    if (g_gather_rounding & f16_bit) return round_significand((double)(float)x, 11, -14);
    if (g_gather_rounding & bf16_bit) return round_significand((double)(float)x, 8, -126);
    return x;
}

/* A neighbour's gathered velocity under the rounding experiment: bits 0
 * and 2 as above; bit 4, each component as a 21-bit float (FP32's sign and
 * exponent, 13 significant bits); bit 5, one shared exponent and three
 * signed 18-bit mantissas: the quantum is 2^(E - 17) for the least E with
 * max |v_k| < 2^E, doubled once if a rounded mantissa leaves
 * [-2^17, 2^17 - 1]. */
inline void gather_velocity(const double* vj, double out[3])
{
    for (int k = 0; k < 3; ++k) out[k] = gather_round(vj[k], 1, 4);
    if (g_gather_rounding & 16)
        for (int k = 0; k < 3; ++k) out[k] = round_significand((double)(float)out[k], 13, -126);
    if (g_gather_rounding & 32) {
        double f[3], m = 0.0;
        for (int k = 0; k < 3; ++k) {
            f[k] = (double)(float)out[k];
            m = std::max(m, std::fabs(f[k]));
        }
        if (m == 0.0 || !std::isfinite(m)) return;
        int e;
        std::frexp(m, &e);          /* m < 2^e */
        for (int pass = 0; pass < 2; ++pass) {
            const double q = std::ldexp(1.0, e - 17);
            bool fits = true;
            double r[3];
            for (int k = 0; k < 3; ++k) {
                r[k] = std::nearbyint(f[k] / q);
                fits = fits && r[k] >= -131072.0 && r[k] <= 131071.0;
            }
            if (fits || pass == 1) {
                for (int k = 0; k < 3; ++k) out[k] = r[k] * q;
                return;
            }
            ++e;
        }
    }
}

void interaction(const OrParams& P, int np, int npb, const double* pos, const double* vel, const double* str,
                 double* accad, double* spin, double* acestn, const int* beg, const int* end, bool float_cells)
{
    const double ih = P.i_h, m = P.m, h = P.h, eta = P.eta, cs = P.cs;
    const double Cg = P.kernel_gradient_normalization_par;
    const double alpha = P.artificial_viscosity_alpha;
    const bool visc = P.viscosity_type == 1;
    const bool artp = P.artificial_pressure == 1;
    const double eps = P.artificial_pressure_coefficient;
    const double wdr = P.kernel_dr;
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = npb; i < np; ++i) {
        const double* xi = pos + 4 * (size_t)i;
        const double* vi = vel + 4 * (size_t)i;
        const double* si = str + 6 * (size_t)i;
        const double rhoi = vi[3];
        const double ri2 = 1.0 / (rhoi * rhoi);
        double Ri[3] = {0, 0, 0};
        if (artp)
            for (int k = 0; k < 3; ++k) Ri[k] = si[k] > 0.0 ? -eps * si[k] * ri2 : 0.0;
        double drho = 0, a[3] = {0, 0, 0}, Lg[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        int cx, cy, cz;
        stencil_centre(P, xi, float_cells, cx, cy, cz);
        auto body = [&](int j) {
            if (j == i) return;
            const double* xj = pos + 4 * (size_t)j;
            double d[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
            double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            double q = std::sqrt(r2) * ih;
            if (!(q < 2.0)) return;
            const double* vj = vel + 4 * (size_t)j;
            const double* sj = str + 6 * (size_t)j;
            double t = 2.0 - q;
            double fac = Cg * t * t * t;
            double g[3] = {fac * d[0], fac * d[1], fac * d[2]};
            double vg[3];
            gather_velocity(vj, vg);
            double vij[3] = {vi[0] - vg[0], vi[1] - vg[1], vi[2] - vg[2]};
            drho += vij[0] * g[0] + vij[1] * g[1] + vij[2] * g[2];
            double rhoj = vj[3];
            double rj2 = 1.0 / (rhoj * rhoj);
            /* symmetric stress term; full 3x3 from the 6 components */
            double T[6];
            for (int k = 0; k < 6; ++k) T[k] = si[k] * ri2 + gather_round(sj[k] * rj2, 2, 8);
            a[0] += m * (T[0] * g[0] + T[3] * g[1] + T[4] * g[2]);
            a[1] += m * (T[3] * g[0] + T[1] * g[1] + T[5] * g[2]);
            a[2] += m * (T[4] * g[0] + T[5] * g[1] + T[2] * g[2]);
            if (visc) {
                double vr = vij[0] * d[0] + vij[1] * d[1] + vij[2] * d[2];
                if (vr < 0.0) {
                    double mu = h * vr / (r2 + eta);
                    double Pi = -alpha * cs * mu / (0.5 * (rhoi + rhoj));
                    for (int k = 0; k < 3; ++k) a[k] -= m * Pi * g[k];
                }
            }
            if (artp) {
                double f = wendland(P, q) / wdr;
                double f4 = f * f * f * f;
                for (int k = 0; k < 3; ++k) {
                    double Rj = sj[k] > 0.0 ? -eps * sj[k] * rj2 : 0.0;
                    a[k] += m * (Ri[k] + Rj) * f4 * g[k];
                }
            }
            double Vj = m / rhoj;
            for (int aa = 0; aa < 3; ++aa)
                for (int bb = 0; bb < 3; ++bb) Lg[3 * aa + bb] -= Vj * vij[aa] * g[bb];
        };
        for_stencil(P, cx, cy, cz, 0, beg, end, body);
        for_stencil(P, cx, cy, cz, P.ncell_one_layer, beg, end, body);
        double* ac = accad + 4 * (size_t)i;
        ac[0] = a[0] + P.acc_x;
        ac[1] = a[1] + P.acc_y;
        ac[2] = a[2] + P.acc_z;
        ac[3] = m * drho;
        double* e = acestn + 6 * (size_t)i;
        e[0] = Lg[0];
        e[1] = Lg[4];
        e[2] = Lg[8];
        e[3] = 0.5 * (Lg[1] + Lg[3]);
        e[4] = 0.5 * (Lg[2] + Lg[6]);
        e[5] = 0.5 * (Lg[5] + Lg[7]);
        double* w = spin + 4 * (size_t)i;
        w[0] = 0.5 * (Lg[3] - Lg[1]);   /* W_yx */
        w[1] = 0.5 * (Lg[6] - Lg[2]);   /* W_zx */
        w[2] = 0.5 * (Lg[7] - Lg[5]);   /* W_zy */
        w[3] = 0.0;
    }
}

/* -------------------------------------------------------- Shepard (a12) */
/* reference src/field_smoothing.cu:65-121: material layer only, self
 * included, no guard on a zero weight sum. */
void shepard(const OrParams& P, int np, int npb, const double* pos, const double* vel, const double* str,
             double* out, const int* beg, const int* end, bool float_cells)
{
    const double ih = P.i_h, m = P.m;
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = npb; i < np; ++i) {
        const double* xi = pos + 4 * (size_t)i;
        double S[6] = {0, 0, 0, 0, 0, 0}, w = 0;
        int cx, cy, cz;
        stencil_centre(P, xi, float_cells, cx, cy, cz);
        for_stencil(P, cx, cy, cz, P.ncell_one_layer, beg, end, [&](int j) {
            const double* xj = pos + 4 * (size_t)j;
            double d[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
            double q = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) * ih;
            if (q < 2.0) {
                double kv = wendland(P, q) * (m / vel[4 * (size_t)j + 3]);
                for (int k = 0; k < 6; ++k) S[k] += str[6 * (size_t)j + k] * kv;
                w += kv;
            }
        });
        for (int k = 0; k < 6; ++k) out[6 * (size_t)i + k] = S[k] / w;
    }
}

/* Density Shepard filter (not applied by the reference, whose parameter
 * density-shepard-filter is read but unused, src/loquat_io.cu:180): for a
 * material particle, rho~_i = sum_j m W_ij / sum_j (m / rho_j) W_ij over the
 * material layer, self included -- the stress filter's neighbour set and
 * weights applied to the density. */
void shepard_density(const OrParams& P, int np, int npb, const double* pos, const double* vel, double* rho_out,
                     const int* beg, const int* end, bool float_cells)
{
    const double ih = P.i_h, m = P.m;
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = npb; i < np; ++i) {
        const double* xi = pos + 4 * (size_t)i;
        double num = 0, w = 0;
        int cx, cy, cz;
        stencil_centre(P, xi, float_cells, cx, cy, cz);
        for_stencil(P, cx, cy, cz, P.ncell_one_layer, beg, end, [&](int j) {
            const double* xj = pos + 4 * (size_t)j;
            double d[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
            double q = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) * ih;
            if (q < 2.0) {
                const double wk = wendland(P, q);
                num += m * wk;
                w += wk * (m / vel[4 * (size_t)j + 3]);
            }
        });
        rho_out[i] = num / w;
    }
}

/* Dynamic time step (the reference reads dynamic-time-step but always uses
 * cfl h / cs, src/loquat.cu:325-333): from the material particles' largest
 * speed and acceleration at the end of a step,
 *   dt = cfl min(h / (cs + v_max), sqrt(h / a_max)),
 * never above the fixed cfl h / cs. */
double dynamic_dt(const OrParams& P, int np, int npb, const double* vel, const double* accad)
{
    double v2 = 0, a2 = 0;
    for (int i = npb; i < np; ++i) {
        const double* v = vel + 4 * (size_t)i;
        const double* a = accad + 4 * (size_t)i;
        v2 = std::fmax(v2, v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        a2 = std::fmax(a2, a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    }
    const double h = P.h, cs = P.cs;
    double dt = h / (cs + std::sqrt(v2));
    if (a2 > 0) dt = std::fmin(dt, std::sqrt(h / std::sqrt(a2)));
    return (double)P.cfl * dt;
}

/* ------------------------------------------- constitutive models (a9, a10) */
inline double contract(const double* a, const double* b)
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + 2.0 * (a[3] * b[3] + a[4] * b[4] + a[5] * b[5]);
}

/* Jaumann co-rotational term for spin (W_yx, W_zx, W_zy)
 * (reference src/predictor_corrector.cu:40-45). */
inline void jaumann(const double* w, const double* s, double* j)
{
    j[0] = -2.0 * (w[0] * s[3] + w[1] * s[4]);
    j[1] = 2.0 * (w[0] * s[3] - w[2] * s[5]);
    j[2] = 2.0 * (w[1] * s[4] + w[2] * s[5]);
    j[3] = w[0] * (s[0] - s[1]) - w[2] * s[4] - w[1] * s[5];
    j[4] = w[1] * (s[0] - s[2]) + w[2] * s[3] - w[0] * s[5];
    j[5] = w[2] * (s[1] - s[2]) + w[0] * s[4] + w[1] * s[3];
}

/* Drucker-Prager with tension cut-off and radial return
 * (reference src/predictor_corrector.cu:30-105). */
void dp_update(const OrParams& P, double dtp, const double* w, const double* d, double& p, double& ep, double* s)
{
    const double K = P.model_par_1, G = P.model_par_2, kphi = P.model_par_3, kpsi = P.model_par_4,
                 kc = P.model_par_5;
    double r[6];
    jaumann(w, s, r);
    for (int k = 0; k < 6; ++k) r[k] += d[k] * (2.0 * G);
    double ace = (K - 2.0 / 3.0 * G) * (d[0] + d[1] + d[2]);
    for (int k = 0; k < 3; ++k) r[k] += ace;
    for (int k = 0; k < 6; ++k) s[k] += r[k] * dtp;
    double sm = (s[0] + s[1] + s[2]) / 3.0;
    for (int k = 0; k < 3; ++k) s[k] -= sm;
    double tenf = (P.model_par_3 == 0.0f) ? 0.0 : kc / kphi;
    double dpTi = sm - tenf;
    if (dpTi >= 0.0) {
        ep += dpTi / K * (1.0 / 3.0) * std::sqrt(2.0);
        sm = tenf;
    }
    double tau = std::sqrt(0.5 * contract(s, s));
    double dpFi = tau + kphi * sm - kc;
    if (dpFi > 0.0) {
        double dl = dpFi / (G + K * kphi * kpsi);
        sm -= K * kpsi * dl;
        double ratio = tau < (double)1e-10f ? 1.0 : (kc - kphi * sm) / tau;
        for (int k = 0; k < 6; ++k) s[k] *= ratio;
        ep += dl * std::sqrt(1.0 / 3.0 + 2.0 / 9.0 * kpsi * kpsi);
    }
    for (int k = 0; k < 3; ++k) s[k] += sm;
    p = -sm;
}

/* Four-parameter hypoplastic rate with Jaumann term, cohesion shift and
 * tension cap (reference src/predictor_corrector.cu:111-165).  The
 * near-zero-stress reset does not clear T_xz: the reference assigns xy twice
 * (src/predictor_corrector.cu:140-141), and that is kept. */
void hypo_update(const OrParams& P, double dtp, const double* d, const double* w, double* s)
{
    const double c1 = P.model_par_1, c2 = P.model_par_2, c3 = P.model_par_3, c4 = P.model_par_4,
                 coh = P.model_par_5;
    double jau[6];
    jaumann(w, s, jau);
    double T[6];
    for (int k = 0; k < 6; ++k) T[k] = s[k];
    if (P.model_par_5 > 0.0f)
        for (int k = 0; k < 3; ++k) T[k] -= coh;
    double t1 = T[0] + T[1] + T[2];
    if (std::fabs(t1) < 4.0) {
        t1 = -4.0;
        T[0] = -1.0;
        T[1] = -1.0;
        T[2] = -2.0;
        T[3] = 0.0; /* xy */
        T[5] = 0.0; /* yz; xz keeps its value */
    }
    double Ts[6];
    for (int k = 0; k < 6; ++k) Ts[k] = T[k];
    for (int k = 0; k < 3; ++k) Ts[k] -= t1 / 3.0;
    double d1 = d[0] + d[1] + d[2];
    double t1d1 = contract(T, d);
    double nd = std::sqrt(contract(d, d));
    for (int k = 0; k < 6; ++k) {
        double rate = jau[k] + d[k] * (c1 * t1) + T[k] * (c2 * d1 + c3 * t1d1 / t1) + (T[k] + Ts[k]) * (c4 * nd);
        s[k] += rate * dtp;
    }
    double pres = (s[0] + s[1] + s[2]) / 3.0;
    if (pres > coh)
        for (int k = 0; k < 3; ++k) s[k] -= (pres - coh);
}

/* -------------------------------------- von Wolffersdorff (model 3) */
/* Not in the reference (its hypoplastic model is the four-parameter one
 * above): the hypoplastic relation with a predefined limit-state surface of
 * von Wolffersdorff (1996, Mech. Cohes.-Frict. Mater. 1:251-271), written
 * from the published equations, tension positive (T < 0 in compression):
 *   Tdot = fb fe / (That:That) [F^2 D + a^2 That (That:D) + fd a F (That + That*) |D|] + Jaumann
 *   That = T / tr T, That* = That - I/3, |D| = sqrt(D:D)
 *   a = sqrt3 (3 - sin phic) / (2 sqrt2 sin phic)
 *   F = sqrt(tan^2 psi / 8 + (2 - tan^2 psi) / (2 + sqrt2 tan psi cos3theta)) - tan psi / (2 sqrt2)
 *   tan psi = sqrt3 |That*|, cos3theta = -sqrt6 tr(That*^3) / (That*:That*)^{3/2}
 *   e_x = e_x0 exp(-(-tr T / hs)^n) for x = i, c, d
 *   fe = (ec / e)^beta, fd = ((e - ed) / (ec - ed))^alpha
 *   fb = (hs / n) (ei0 / ec0)^beta (1 + ei) / ei (-tr T / hs)^(1 - n)
 *        / (3 + a^2 - a sqrt3 ((ei0 - ed0) / (ec0 - ed0))^alpha)
 *   edot = (1 + e) tr D
 * A stress with tr T > -3 Pa (free surface, tension) is reset to -1 Pa
 * isotropic before the rate is formed, as the four-parameter model resets
 * near-zero stress; a stress with tan psi beyond sqrt2 (where F is not
 * defined: a tensile principal direction) has its deviator scaled back to
 * tan psi = sqrt2 (1 - 1e-3) at the same mean stress.  The step is integrated by explicit sub-steps (Euler /
 * Heun pair) whose relative stress difference is kept below `tol`.
 * Table row: phic (deg), hs (Pa), n, ed0, ec0, ei0, alpha, beta, tol,
 * max sub-steps. */
struct VW {
    double sphi, a, hs, n, ed0, ec0, ei0, alpha, beta, tol, fbden;
    int maxsub;
};

VW vw_constants(const float* row)
{
    VW c;
    const double phic = row[0] * 3.14159265358979323846 / 180.0;
    c.sphi = std::sin(phic);
    c.a = std::sqrt(3.0) * (3.0 - c.sphi) / (2.0 * std::sqrt(2.0) * c.sphi);
    c.hs = row[1];
    c.n = row[2];
    c.ed0 = row[3];
    c.ec0 = row[4];
    c.ei0 = row[5];
    c.alpha = row[6];
    c.beta = row[7];
    c.tol = row[8];
    c.maxsub = (int)row[9];
    c.fbden = 3.0 + c.a * c.a - c.a * std::sqrt(3.0) * std::pow((c.ei0 - c.ed0) / (c.ec0 - c.ed0), c.alpha);
    return c;
}

/* tr(A^3) of a symmetric tensor (xx yy zz xy xz yz) */
inline double trace_cube(const double* A)
{
    const double xx = A[0], yy = A[1], zz = A[2], xy = A[3], xz = A[4], yz = A[5];
    return xx * xx * xx + yy * yy * yy + zz * zz * zz + 3.0 * (xy * xy * (xx + yy) + xz * xz * (xx + zz) +
                                                                yz * yz * (yy + zz)) + 6.0 * xy * xz * yz;
}

void vw_rate(const VW& c, const double* T_in, double e, const double* d, const double* w, double* Tdot, double* edot)
{
    double T[6];
    for (int k = 0; k < 6; ++k) T[k] = T_in[k];
    double trT = T[0] + T[1] + T[2];
    if (!(trT < -3.0)) {
        for (int k = 0; k < 3; ++k) T[k] = -1.0;
        for (int k = 3; k < 6; ++k) T[k] = 0.0;
        trT = -3.0;
    }
    double Th[6], Ts[6];
    for (int k = 0; k < 6; ++k) Th[k] = T[k] / trT;
    for (int k = 0; k < 6; ++k) Ts[k] = Th[k];
    for (int k = 0; k < 3; ++k) Ts[k] -= 1.0 / 3.0;
    double TsTs = contract(Ts, Ts);
    double tpsi = std::sqrt(3.0 * TsTs);
    /* F is undefined from tan psi = sqrt2 on (states with tension): the
     * deviator is scaled back inside, keeping the mean stress */
    const double lim = std::sqrt(2.0) * (1.0 - 1e-3);
    if (tpsi > lim) {
        const double f = lim / tpsi;
        for (int k = 0; k < 6; ++k) Ts[k] *= f;
        for (int k = 0; k < 6; ++k) Th[k] = Ts[k];
        for (int k = 0; k < 3; ++k) Th[k] += 1.0 / 3.0;
        TsTs *= f * f;
        tpsi = lim;
    }
    const double ThTh = contract(Th, Th);
    double c3t = 1.0;
    if (TsTs > 1e-30) c3t = -std::sqrt(6.0) * trace_cube(Ts) / std::pow(TsTs, 1.5);
    c3t = std::fmax(-1.0, std::fmin(1.0, c3t));
    const double F =
        std::sqrt(std::fmax(tpsi * tpsi / 8.0 + (2.0 - tpsi * tpsi) / (2.0 + std::sqrt(2.0) * tpsi * c3t), 0.0)) -
        tpsi / (2.0 * std::sqrt(2.0));
    const double pr = -trT / c.hs;
    const double ex = std::exp(-std::pow(pr, c.n));
    const double ei = c.ei0 * ex, ec = c.ec0 * ex, ed = c.ed0 * ex;
    const double fe = std::pow(ec / e, c.beta);
    const double fd = std::pow(std::fmax((e - ed) / (ec - ed), 0.0), c.alpha);
    const double fb = (c.hs / c.n) * std::pow(c.ei0 / c.ec0, c.beta) * (1.0 + ei) / ei * std::pow(pr, 1.0 - c.n) /
                      c.fbden;
    const double ThD = contract(Th, d);
    const double nD = std::sqrt(contract(d, d));
    const double k0 = fb * fe / ThTh;
    double jau[6];
    jaumann(w, T_in, jau);
    for (int k = 0; k < 6; ++k)
        Tdot[k] = k0 * (F * F * d[k] + c.a * c.a * Th[k] * ThD + fd * c.a * F * (Th[k] + Ts[k]) * nD) + jau[k];
    *edot = (1.0 + e) * (d[0] + d[1] + d[2]);
}

/* Adaptive explicit integration of the model over dt; returns sub-steps. */
int vw_update(const VW& c, double dt, const double* d, const double* w, double* s, double& e)
{
    double t = 0.0, h = dt;
    int steps = 0;
    while (t < dt) {
        h = std::fmin(h, dt - t);
        if (steps >= c.maxsub - 1) h = dt - t;
        double k1[6], k2[6], s1[6], s2[6], ke1, ke2;
        vw_rate(c, s, e, d, w, k1, &ke1);
        for (int k = 0; k < 6; ++k) s1[k] = s[k] + h * k1[k];
        const double e1 = e + h * ke1;
        vw_rate(c, s1, e1, d, w, k2, &ke2);
        double num = 0.0, den = 0.0;
        for (int k = 0; k < 6; ++k) {
            s2[k] = s[k] + 0.5 * h * (k1[k] + k2[k]);
            const double df = 0.5 * h * (k2[k] - k1[k]);   /* Heun minus Euler */
            num += df * df * (k < 3 ? 1.0 : 2.0);
            den += s2[k] * s2[k] * (k < 3 ? 1.0 : 2.0);
        }
        const double err = std::sqrt(num / std::fmax(den, 1e-30));
        ++steps;
        /* the last allowed sub-step is accepted whatever its error, so the
         * whole interval is always integrated */
        const bool last = steps >= c.maxsub - 1 || h <= dt * 1e-6;
        if (err <= c.tol || last) {
            for (int k = 0; k < 6; ++k) s[k] = s2[k];
            e += 0.5 * h * (ke1 + ke2);
            t += h;
            const double g = err > 0.0 ? 0.9 * std::sqrt(c.tol / err) : 2.0;
            h *= std::fmin(2.0, std::fmax(0.2, g));
        } else {
            h *= std::fmax(0.2, 0.9 * std::sqrt(c.tol / err));
        }
    }
    return steps;
}

/* ---------------------------------------------- predictor / corrector */
struct StateView {
    double *pos, *vel, *idep, *str, *stn;
};

/* Per-object material rows for model 3 (10 floats each). */
struct VWTable {
    const float* rows = nullptr;
    int n = 0;
};

inline VW vw_for(const VWTable& t, double id)
{
    int k = (int)id;
    k = k < 0 ? 0 : (k >= t.n ? t.n - 1 : k);
    return vw_constants(t.rows + 10 * k);
}

/* reference src/predictor_corrector.cu:169-218 (material slots only; the
 * snapshot of all slots is taken by the caller) */
void predictor(const OrParams& P, int np, int npb, StateView S, const double* accad, const double* spin,
               const double* acestn, const VWTable& vwt = VWTable())
{
    const double hdt = 0.5 * (double)P.dt;
#pragma omp parallel for schedule(static)
    for (int i = npb; i < np; ++i) {
        double* x = S.pos + 4 * (size_t)i;
        double* v = S.vel + 4 * (size_t)i;
        const double* a = accad + 4 * (size_t)i;
        for (int k = 0; k < 4; ++k) v[k] += hdt * a[k];
        for (int k = 0; k < 3; ++k) x[k] += hdt * v[k];
        double* e = S.stn + 6 * (size_t)i;
        const double* de = acestn + 6 * (size_t)i;
        for (int k = 0; k < 6; ++k) e[k] += de[k] * hdt;
        double p = x[3];
        double ep = S.idep[4 * (size_t)i + 1];
        double* s = S.str + 6 * (size_t)i;
        const double* w = spin + 4 * (size_t)i;
        if (P.constitutive_model == 1) {
            dp_update(P, hdt, w, de, p, ep, s);
        } else if (P.constitutive_model == 3) {
            double ev = S.idep[4 * (size_t)i + 2];
            vw_update(vw_for(vwt, S.idep[4 * (size_t)i]), hdt, de, w, s, ev);
            S.idep[4 * (size_t)i + 2] = ev;
            ep = std::sqrt(2.0 / 3.0 * contract(e, e));
        } else {
            hypo_update(P, hdt, de, w, s);
            ep = std::sqrt(2.0 / 3.0 * contract(e, e));
        }
        x[3] = p;
        S.idep[4 * (size_t)i + 1] = ep;
    }
}

/* reference src/predictor_corrector.cu:256-307 */
void corrector(const OrParams& P, int np, int npb, StateView S, StateView I, const double* accad,
               const double* spin, const double* acestn, const VWTable& vwt = VWTable())
{
    const double dt = (double)P.dt;
#pragma omp parallel for schedule(static)
    for (int i = npb; i < np; ++i) {
        double* x = S.pos + 4 * (size_t)i;
        double* v = S.vel + 4 * (size_t)i;
        const double* x0 = I.pos + 4 * (size_t)i;
        const double* v0 = I.vel + 4 * (size_t)i;
        const double* a = accad + 4 * (size_t)i;
        for (int k = 0; k < 4; ++k) v[k] = v0[k] + dt * a[k];
        for (int k = 0; k < 3; ++k) x[k] = 0.5 * (v[k] + v0[k]) * dt + x0[k];
        double* e = S.stn + 6 * (size_t)i;
        const double* e0 = I.stn + 6 * (size_t)i;
        const double* de = acestn + 6 * (size_t)i;
        for (int k = 0; k < 6; ++k) e[k] = e0[k] + de[k] * dt;
        double p = x[3];
        double ep = I.idep[4 * (size_t)i + 1];
        double s[6];
        for (int k = 0; k < 6; ++k) s[k] = I.str[6 * (size_t)i + k];
        const double* w = spin + 4 * (size_t)i;
        if (P.constitutive_model == 1) {
            dp_update(P, dt, w, de, p, ep, s);
        } else if (P.constitutive_model == 3) {
            double ev = I.idep[4 * (size_t)i + 2];
            vw_update(vw_for(vwt, I.idep[4 * (size_t)i]), dt, de, w, s, ev);
            S.idep[4 * (size_t)i + 2] = ev;
            ep = std::sqrt(2.0 / 3.0 * contract(e, e));
        } else {
            hypo_update(P, dt, de, w, s);
            ep = std::sqrt(2.0 / 3.0 * contract(e, e));
        }
        x[3] = p;
        for (int k = 0; k < 6; ++k) S.str[6 * (size_t)i + k] = s[k];
        S.idep[4 * (size_t)i + 1] = ep;
    }
}

/* ------------------------------------------------------------ full step */
struct OrSim {
    OrParams P;
    int np, npb;
    long long step;
    double time;
    std::vector<double> pos, vel, idep, str, stn;
    std::vector<double> pos0, vel0, idep0, str0, stn0;
    std::vector<double> accad, spin, acestn, tmp;
    std::vector<float> vw_rows;
    VWTable vwt;
    Grid g;
    bool density_filter = false;   /* extensions, off as in the reference */
    bool dynamic = false;
    double dt_next = 0.0;

    StateView cur() { return {pos.data(), vel.data(), idep.data(), str.data(), stn.data()}; }
    StateView ini() { return {pos0.data(), vel0.data(), idep0.data(), str0.data(), stn0.data()}; }

    void search() { build_grid(P, np, npb, pos.data(), false, g); }
    void sort_primary()   /* reference src/loquat.cu:190-197 */
    {
        const int* ix = g.part_idx.data();
        gather(np, 4, ix, pos, tmp);
        gather(np, 4, ix, vel, tmp);
        gather(np, 4, ix, idep, tmp);
        gather(np, 6, ix, str, tmp);
        gather(np, 6, ix, stn, tmp);
    }
    void sort_all()       /* reference src/loquat.cu:200-213 */
    {
        sort_primary();
        const int* ix = g.part_idx.data();
        gather(np, 4, ix, pos0, tmp);
        gather(np, 4, ix, vel0, tmp);
        gather(np, 4, ix, idep0, tmp);
        gather(np, 6, ix, str0, tmp);
        gather(np, 6, ix, stn0, tmp);
    }
    void adami_stage()
    {
        adami(P, np, npb, pos.data(), vel.data(), str.data(), g.beg.data(), g.end.data(), false);
    }
    void interaction_stage()
    {
        interaction(P, np, npb, pos.data(), vel.data(), str.data(), accad.data(), spin.data(), acestn.data(),
                    g.beg.data(), g.end.data(), false);
    }
    /* One time step (reference src/loquat.cu:322-409). */
    void one_step()
    {
        P.dt = P.cfl * P.h / P.cs;
        if (dynamic && dt_next > 0.0) P.dt = (float)dt_next;
        P.time = (float)time;
        search();
        sort_primary();
        adami_stage();
        interaction_stage();
        pos0 = pos; vel0 = vel; idep0 = idep; str0 = str; stn0 = stn;
        predictor(P, np, npb, cur(), accad.data(), spin.data(), acestn.data(), vwt);
        search();
        sort_all();
        adami_stage();
        interaction_stage();
        corrector(P, np, npb, cur(), ini(), accad.data(), spin.data(), acestn.data(), vwt);
        const int N = P.stress_shepard_filter;
        if (N != 0 && step % N == 0 && step != 0) {
            search();
            sort_primary();
            std::vector<double> out(str);
            shepard(P, np, npb, pos.data(), vel.data(), str.data(), out.data(), g.beg.data(), g.end.data(), false);
            for (size_t k = (size_t)npb * 6; k < out.size(); ++k) str[k] = out[k];
        }
        const int Nd = P.density_shepard_filter;
        if (density_filter && Nd > 0 && step % Nd == 0 && step != 0) {
            search();
            sort_primary();
            std::vector<double> rho(np);
            shepard_density(P, np, npb, pos.data(), vel.data(), rho.data(), g.beg.data(), g.end.data(), false);
            for (int i = npb; i < np; ++i) vel[4 * (size_t)i + 3] = rho[i];
        }
        time += (double)P.dt;
        step++;
        if (dynamic) dt_next = dynamic_dt(P, np, npb, vel.data(), accad.data());
    }
};

} // namespace

extern "C" {

int or_parameters_size(void) { return (int)sizeof(OrParams); }

void or_set_gather_rounding(int mode) { g_gather_rounding = mode; }

int or_set_threads(int n)
{
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
}

/* reference src/loquat.cu:111-139, float arithmetic as there */
int or_initialize_parameters(void* pv)
{
    OrParams* p = (OrParams*)pv;
    p->h = p->dr * p->hdr;
    p->i_h = 1.0f / p->h;
    p->eta = 0.01f * p->h * p->h;
    p->m = p->dr * p->dr * p->dr * p->rho0;
    p->cell_num_x = (int)(0.5f * p->i_h * p->domain_size_x) + 1;
    p->cell_num_y = (int)(0.5f * p->i_h * p->domain_size_y) + 1;
    p->cell_num_z = (int)(0.5f * p->i_h * p->domain_size_z) + 1;
    p->ncell_one_layer = p->cell_num_x * p->cell_num_y * p->cell_num_z;
    p->ncell = 2 * p->ncell_one_layer + 1;
    p->ncell_delete = p->ncell - 1;
    p->kernel_normalization_par = 42.0f / 256.0f / (powf(p->h, 3) * kPiF);
    p->kernel_gradient_normalization_par = -5.0f * 42.0f / 256.0f / (powf(p->h, 5) * kPiF);
    if (p->artificial_pressure == 1) {
        p->kernel_zero = p->kernel_normalization_par * 2.0f * 2.0f * 2.0f * 2.0f * 0.5f;
        float q = p->dr * p->i_h;
        p->kernel_dr = p->kernel_normalization_par * (2.0f - q) * (2.0f - q) * (2.0f - q) * (2.0f - q) * (q + 0.5f);
    }
    return 0;
}

/* Neighbour grid in float cell arithmetic: the bit-exact reference for the
 * device grid.  pos: float[np][4]. Outputs: part_cel/part_idx int[np],
 * cell_beg/cell_end int[ncell], cell_start int[ncell + 1]. */
int or_grid_float(const void* pv, int np, int npb, const float* pos, int* part_cel, int* part_idx, int* cell_beg,
                  int* cell_end, int* cell_start)
{
    const OrParams& P = *(const OrParams*)pv;
    std::vector<double> pd((size_t)np * 4);
    for (size_t k = 0; k < pd.size(); ++k) pd[k] = pos[k];
    Grid g;
    build_grid(P, np, npb, pd.data(), true, g);
    std::memcpy(part_cel, g.part_cel.data(), sizeof(int) * np);
    std::memcpy(part_idx, g.part_idx.data(), sizeof(int) * np);
    std::memcpy(cell_beg, g.beg.data(), sizeof(int) * P.ncell);
    std::memcpy(cell_end, g.end.data(), sizeof(int) * P.ncell);
    std::memcpy(cell_start, g.start.data(), sizeof(int) * (P.ncell + 1));
    return 0;
}

/* Per-operator entry points on sorted inputs.  Positions are float values
 * carried in double, and stencils are centred with the device's float cell
 * arithmetic so both sides visit the same cells. */
int or_interaction(const void* pv, int np, int npb, const double* pos, const double* vel, const double* str,
                   double* accad, double* spin, double* acestn, const int* beg, const int* end)
{
    interaction(*(const OrParams*)pv, np, npb, pos, vel, str, accad, spin, acestn, beg, end, true);
    return 0;
}

int or_adami(const void* pv, int np, int npb, const double* pos, const double* vel, double* str, const int* beg,
             const int* end)
{
    adami(*(const OrParams*)pv, np, npb, pos, vel, str, beg, end, true);
    return 0;
}

int or_shepard(const void* pv, int np, int npb, const double* pos, const double* vel, const double* str,
               double* out, const int* beg, const int* end)
{
    shepard(*(const OrParams*)pv, np, npb, pos, vel, str, out, beg, end, true);
    return 0;
}

/* Predictor on material slots (no snapshot). */
int or_predictor(const void* pv, int np, int npb, double* pos, double* vel, double* idep, double* str, double* stn,
                 const double* accad, const double* spin, const double* acestn)
{
    predictor(*(const OrParams*)pv, np, npb, {pos, vel, idep, str, stn}, accad, spin, acestn);
    return 0;
}

int or_corrector(const void* pv, int np, int npb, double* pos, double* vel, double* idep, double* str, double* stn,
                 const double* pos0, const double* vel0, const double* idep0, const double* str0,
                 const double* stn0, const double* accad, const double* spin, const double* acestn)
{
    StateView I{(double*)pos0, (double*)vel0, (double*)idep0, (double*)str0, (double*)stn0};
    corrector(*(const OrParams*)pv, np, npb, {pos, vel, idep, str, stn}, I, accad, spin, acestn);
    return 0;
}

/* Single-particle constitutive updates (for analytic unit tests). */
int or_dp_update(const void* pv, double dtp, const double* spin3, const double* d6, double* p, double* ep,
                 double* s6)
{
    dp_update(*(const OrParams*)pv, dtp, spin3, d6, *p, *ep, s6);
    return 0;
}

int or_hypo_update(const void* pv, double dtp, const double* d6, const double* spin3, double* s6)
{
    hypo_update(*(const OrParams*)pv, dtp, d6, spin3, s6);
    return 0;
}

/* Whole-simulation oracle.  Arrays double[np][4] / [np][6]. */
void* or_sim_create(const void* pv, const double* pos, const double* vel, const double* idep, const double* str,
                    const double* stn, long long step0, double time0)
{
    OrSim* s = new OrSim();
    s->P = *(const OrParams*)pv;
    s->np = s->P.np;
    s->npb = s->P.npb;
    s->step = step0;
    s->time = time0;
    size_t n = (size_t)s->np;
    s->pos.assign(pos, pos + 4 * n);
    s->vel.assign(vel, vel + 4 * n);
    s->idep.assign(idep, idep + 4 * n);
    s->str.assign(str, str + 6 * n);
    s->stn.assign(stn, stn + 6 * n);
    s->accad.assign(4 * n, 0.0);
    s->spin.assign(4 * n, 0.0);
    s->acestn.assign(6 * n, 0.0);
    /* initial search + primary sort (reference src/loquat.cu:297-298) */
    s->search();
    s->sort_primary();
    return s;
}

/* Model-3 material rows (n x 10 floats, by object id). */
int or_sim_set_vw(void* sv, int n, const float* rows)
{
    OrSim* s = (OrSim*)sv;
    s->vw_rows.assign(rows, rows + 10 * (size_t)n);
    s->vwt.rows = s->vw_rows.data();
    s->vwt.n = n;
    return 0;
}

/* One model-3 update of a single material point (unit tests). */
int or_vw_update(const float* row, double dt, const double* d6, const double* spin3, double* s6, double* e)
{
    return vw_update(vw_constants(row), dt, d6, spin3, s6, *e);
}

int or_vw_rate(const float* row, const double* s6, double e, const double* d6, const double* spin3, double* rate6,
               double* erate)
{
    vw_rate(vw_constants(row), s6, e, d6, spin3, rate6, erate);
    return 0;
}

/* Extensions with no reference behaviour: the density Shepard filter every
 * density_shepard_filter steps, and the dynamic time step. */
int or_sim_set_extensions(void* sv, int density_filter, int dynamic_dt)
{
    OrSim* s = (OrSim*)sv;
    s->density_filter = density_filter != 0;
    s->dynamic = dynamic_dt != 0;
    return 0;
}

double or_sim_time(void* sv) { return ((OrSim*)sv)->time; }

int or_sim_step(void* sv, int n)
{
    OrSim* s = (OrSim*)sv;
    if (s->P.constitutive_model == 3 && s->vwt.n == 0) return -1; /* model 3 needs or_sim_set_vw */
    for (int k = 0; k < n; ++k) s->one_step();
    return 0;
}

int or_sim_get(void* sv, double* pos, double* vel, double* idep, double* str, double* stn)
{
    OrSim* s = (OrSim*)sv;
    std::memcpy(pos, s->pos.data(), sizeof(double) * s->pos.size());
    std::memcpy(vel, s->vel.data(), sizeof(double) * s->vel.size());
    std::memcpy(idep, s->idep.data(), sizeof(double) * s->idep.size());
    std::memcpy(str, s->str.data(), sizeof(double) * s->str.size());
    std::memcpy(stn, s->stn.data(), sizeof(double) * s->stn.size());
    return 0;
}

long long or_sim_steps_done(void* sv) { return ((OrSim*)sv)->step; }

void or_sim_destroy(void* sv) { delete (OrSim*)sv; }

} // extern "C"
