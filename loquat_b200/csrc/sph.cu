/*
 * LOQUAT-B200 neighbour-loop kernels: particle interaction, Adami boundary
 * and Shepard stress filter, with their C ABI entry points and the C++
 * drop-in functions of the reference interface.
 *
 * Layout: the state is cell-sorted AoS as the reference stores it
 * (float4 position/velocity, 24-byte tensor2d).  Because cell keys are
 * z-fastest, the particles of three z-adjacent cells of one (x, y) column
 * are one contiguous slot range, so a 27-cell stencil is 9 contiguous runs
 * per layer; neighbouring threads (consecutive sorted particles) walk the
 * same runs and their loads hit L1.
 */
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <utility>
#include <vector>

#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "lq_internal.cuh"
#include "lq_tile.h"
#include "lq_device.cuh"
#include <adami_boundary.h>
#include <field_smoothing.h>
#include <particle_interaction.h>

namespace lqb {

namespace {

constexpr int kBlock = 128;

inline int blocks_for(long long n, int b) { return (int)((n + b - 1) / b); }

/* -------------------------------------------------------- interaction */
/* Formulation (weakly compressible SPH, Wendland C2, tension-positive
 * stress); the reference's implementation of this pass is closed
 * (src/particle_interaction.h:27-40):
 *   g      = C' (2 - q)^3 x_ij                    grad_i W_ij, q = r/h < 2
 *   drho  += m v_ij . g
 *   a     += m (sig_i/rho_i^2 + sig_j/rho_j^2) g  - m Pi_ij g  [+ m (R_i+R_j) f^4 g]
 *   L     -= (m/rho_j) v_ij (x) g
 * over both layers, j != i.  Pi_ij is Monaghan's viscosity with
 * mu = h v_ij.x_ij / (r^2 + eta) for approaching pairs; R is the diagonal
 * artificial stress -eps sig_aa / rho^2 of tensile components, f = W/W(dr).
 *
 * Neighbours are visited through lists: k_neighbor_list walks the union
 * of a warp's lanes' 27-cell stencils in lockstep (one broadcast load per
 * candidate, one distance test per lane) and writes each lane's hits to a
 * global list in coalesced rows; the pair kernels then evaluate each
 * particle's pairs from its list with every lane busy.  The native driver
 * keeps the lists across steps (Verlet lists with a skin); the drop-in
 * ParticleInteraction builds them at each call in the caller's grid.  A
 * particle whose list overflowed walks its stencil directly (walk_stencil),
 * in the same order. */

struct PairConst {
    float ih, h, eta, m, Cg, Cw, avc, eps, wdr, cut2;
    bool visc, artp;
};

__device__ __forceinline__ PairConst load_pair_const(const Parameters* __restrict__ P)
{
    PairConst K;
    K.ih = __ldg(&P->i_h);
    K.h = __ldg(&P->h);
    K.eta = __ldg(&P->eta);
    K.m = __ldg(&P->m);
    K.Cg = __ldg(&P->kernel_gradient_normalization_par);
    K.Cw = __ldg(&P->kernel_normalization_par);
    K.visc = __ldg(&P->viscosity_type) == 1;
    /* alpha * cs; zero without viscosity, so the packed pair body can
     * evaluate the term unconditionally (it then adds exact zeros) */
    K.avc = K.visc ? __ldg(&P->artificial_viscosity_alpha) * __ldg(&P->cs) : 0.0f;
    K.artp = __ldg(&P->artificial_pressure) == 1;
    K.eps = __ldg(&P->artificial_pressure_coefficient);
    K.wdr = __ldg(&P->kernel_dr);
    K.cut2 = 4.0f * K.h * K.h * 1.0001f; /* candidate test; the pair body applies q < 2 exactly */
    return K;
}

/* The particle whose rates are being summed, and its running sums. */
struct Target {
    float4 x, v;
    float Sxx, Syy, Szz, Sxy, Sxz, Syz; /* sigma_i / rho_i^2 */
    float Rx, Ry, Rz;                   /* artificial stress of i */
    float drho, ax, ay, az;
    float cdrho, cax, cay, caz;         /* compensation terms (mixed form) */
    float l00, l01, l02, l10, l11, l12, l20, l21, l22;
};

/* Compensated (Kahan) accumulation: sum + y with the lost low-order part
 * carried in c. */
__device__ __forceinline__ void kahan_add(float& sum, float& c, float y)
{
    const float yy = y - c;
    const float t = sum + yy;
    c = (t - sum) - yy;
    sum = t;
}

__device__ __forceinline__ void load_target(const PairConst& K, const State& st, int i, bool active, Target& T)
{
    T.x = make_float4(0.f, 0.f, 0.f, 0.f);
    T.v = make_float4(0.f, 0.f, 0.f, 1.f);
    tensor2d si = make_tensor2d(0.0f);
    if (active) {
        T.x = __ldg(st.pos + i);
        T.v = __ldg(st.vel + i);
        si = load_t2(st.str, i);
    }
    const float ri2 = 1.0f / (T.v.w * T.v.w);
    T.Sxx = si.xx * ri2; T.Syy = si.yy * ri2; T.Szz = si.zz * ri2;
    T.Sxy = si.xy * ri2; T.Sxz = si.xz * ri2; T.Syz = si.yz * ri2;
    T.Rx = T.Ry = T.Rz = 0.f;
    if (K.artp) {
        T.Rx = si.xx > 0.f ? -K.eps * T.Sxx : 0.f;
        T.Ry = si.yy > 0.f ? -K.eps * T.Syy : 0.f;
        T.Rz = si.zz > 0.f ? -K.eps * T.Szz : 0.f;
    }
    T.drho = T.ax = T.ay = T.az = 0.f;
    T.cdrho = T.cax = T.cay = T.caz = 0.f;
    T.l00 = T.l01 = T.l02 = T.l10 = T.l11 = T.l12 = T.l20 = T.l21 = T.l22 = 0.f;
}

__device__ __forceinline__ float sqrt_approx(float x)
{
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

/* One pair, without branches: a pair at q >= 2 gets a zero kernel gradient
 * and adds zero to every sum.  kKahan compensates the density and
 * momentum sums. */
template <bool kKahan = false>
__device__ __forceinline__ void pair_body(const PairConst& K, const State& st, Target& T, int j)
{
    const float4 xj = __ldg(st.pos + j);
    const float4 vj = __ldg(st.vel + j);
    const tensor2d sj = load_t2(st.str, j);
    const float dx = T.x.x - xj.x, dy = T.x.y - xj.y, dz = T.x.z - xj.z;
    const float r2 = dx * dx + dy * dy + dz * dz;
    const float q = sqrt_approx(r2) * K.ih;
    const float t = fmaxf(2.0f - q, 0.0f);
    const float fac = K.Cg * t * t * t;
    const float gx = fac * dx, gy = fac * dy, gz = fac * dz;
    const float vx = T.v.x - vj.x, vy = T.v.y - vj.y, vz = T.v.z - vj.z;
    if (kKahan)
        kahan_add(T.drho, T.cdrho, vx * gx + vy * gy + vz * gz);
    else
        T.drho += vx * gx + vy * gy + vz * gz;
    const float rinv = __fdividef(1.0f, vj.w);
    const float rj2 = rinv * rinv;
    const float Txx = T.Sxx + sj.xx * rj2, Tyy = T.Syy + sj.yy * rj2, Tzz = T.Szz + sj.zz * rj2;
    const float Txy = T.Sxy + sj.xy * rj2, Txz = T.Sxz + sj.xz * rj2, Tyz = T.Syz + sj.yz * rj2;
    float px = Txx * gx + Txy * gy + Txz * gz;
    float py = Txy * gx + Tyy * gy + Tyz * gz;
    float pz = Txz * gx + Tyz * gy + Tzz * gz;
    if (K.visc) {
        /* Pi = -alpha cs h vr / ((r^2 + eta) rhobar) for vr < 0 */
        const float vr = fminf(vx * dx + vy * dy + vz * dz, 0.0f);
        const float pi = __fdividef(-K.avc * K.h * vr, (r2 + K.eta) * (0.5f * (T.v.w + vj.w)));
        px -= pi * gx;
        py -= pi * gy;
        pz -= pi * gz;
    }
    if (K.artp) {
        const float wk = K.Cw * t * t * t * t * (q + 0.5f);
        const float f = __fdividef(wk, K.wdr);
        const float f4 = (f * f) * (f * f);
        const float Rjx = sj.xx > 0.f ? -K.eps * sj.xx * rj2 : 0.f;
        const float Rjy = sj.yy > 0.f ? -K.eps * sj.yy * rj2 : 0.f;
        const float Rjz = sj.zz > 0.f ? -K.eps * sj.zz * rj2 : 0.f;
        px += (T.Rx + Rjx) * f4 * gx;
        py += (T.Ry + Rjy) * f4 * gy;
        pz += (T.Rz + Rjz) * f4 * gz;
    }
    if (kKahan) {
        kahan_add(T.ax, T.cax, px);
        kahan_add(T.ay, T.cay, py);
        kahan_add(T.az, T.caz, pz);
    } else {
        T.ax += px;
        T.ay += py;
        T.az += pz;
    }
    const float Vj = K.m * rinv;
    const float wx = Vj * vx, wy = Vj * vy, wz = Vj * vz;
    T.l00 -= wx * gx; T.l01 -= wx * gy; T.l02 -= wx * gz;
    T.l10 -= wy * gx; T.l11 -= wy * gy; T.l12 -= wy * gz;
    T.l20 -= wz * gx; T.l21 -= wz * gy; T.l22 -= wz * gz;
}

/* One pair from the packed arrays, its density-rate and momentum terms
 * added to (drho, ax, ay, az) and its velocity-gradient terms to T.  The
 * viscosity term is always evaluated (K.avc is zero without viscosity), so
 * a run of pairs has no branch between them; kArtp adds the artificial
 * stress.  A pair of a particle with itself (the filler of a list's last
 * group of four) adds exact zeros: r = 0 makes the kernel gradient zero. */
template <bool kArtp, bool kPk>
__device__ __forceinline__ void pair_terms(const PairConst& K, const NbrArrays& nb, Target& T, int j, float& drho,
                                           float& ax, float& ay, float& az)
{
    const float4 xr = __ldg(nb.xr + j);
    const float4 sa = __ldg(nb.sa + j);
    const float4 sb = __ldg(nb.sb + j);
    const float3 vj = kPk ? unpack_velocity(sb.z, sb.w) : make_float3(sb.z, sb.w, __ldg(nb.vz + j));
    const float a[8] = {xr.x, xr.y, xr.z, 0.0f, vj.x, vj.y, vj.z, xr.w};
    const float b[6] = {sa.x, sa.y, sa.z, sa.w, sb.x, sb.y};
    const float dx = T.x.x - a[0], dy = T.x.y - a[1], dz = T.x.z - a[2];
    const float r2 = dx * dx + dy * dy + dz * dz;
    const float q = sqrt_approx(r2) * K.ih;
    const float t = fmaxf(2.0f - q, 0.0f);
    const float fac = K.Cg * t * t * t;
    const float gx = fac * dx, gy = fac * dy, gz = fac * dz;
    const float vx = T.v.x - a[4], vy = T.v.y - a[5], vz = T.v.z - a[6];
    drho += vx * gx + vy * gy + vz * gz;
    const float Txx = T.Sxx + b[0], Tyy = T.Syy + b[1], Tzz = T.Szz + b[2];
    const float Txy = T.Sxy + b[3], Txz = T.Sxz + b[4], Tyz = T.Syz + b[5];
    float px = Txx * gx + Txy * gy + Txz * gz;
    float py = Txy * gx + Tyy * gy + Tyz * gz;
    float pz = Txz * gx + Tyz * gy + Tzz * gz;
    {
        /* Pi = -alpha cs h vr / ((r^2 + eta) rhobar) for vr < 0 */
        const float vr = fminf(vx * dx + vy * dy + vz * dz, 0.0f);
        const float pi = __fdividef(-K.avc * K.h * vr, (r2 + K.eta) * (0.5f * (T.v.w + a[7])));
        px -= pi * gx;
        py -= pi * gy;
        pz -= pi * gz;
    }
    if (kArtp) {
        const float wk = K.Cw * t * t * t * t * (q + 0.5f);
        const float f = __fdividef(wk, K.wdr);
        const float f4 = (f * f) * (f * f);
        const float Rjx = b[0] > 0.f ? -K.eps * b[0] : 0.f;
        const float Rjy = b[1] > 0.f ? -K.eps * b[1] : 0.f;
        const float Rjz = b[2] > 0.f ? -K.eps * b[2] : 0.f;
        px += (T.Rx + Rjx) * f4 * gx;
        py += (T.Ry + Rjy) * f4 * gy;
        pz += (T.Rz + Rjz) * f4 * gz;
    }
    ax += px;
    ay += py;
    az += pz;
    const float Vj = K.m * __fdividef(1.0f, a[7]);
    const float wx = Vj * vx, wy = Vj * vy, wz = Vj * vz;
    T.l00 -= wx * gx; T.l01 -= wx * gy; T.l02 -= wx * gz;
    T.l10 -= wy * gx; T.l11 -= wy * gy; T.l12 -= wy * gz;
    T.l20 -= wz * gx; T.l21 -= wz * gy; T.l22 -= wz * gz;
}

/* One pair into T's sums.  kKahan selects the mixed form: the density
 * and momentum sums compensated pair by pair, and the neighbour's velocity
 * gathered in the packed record. */
template <bool kKahan = false>
__device__ __forceinline__ void pair_body_rec(const PairConst& K, const NbrArrays& nb, Target& T, int j)
{
    if (kKahan) {
        float d = 0.f, x = 0.f, y = 0.f, z = 0.f;
        if (K.artp)
            pair_terms<true, true>(K, nb, T, j, d, x, y, z);
        else
            pair_terms<false, true>(K, nb, T, j, d, x, y, z);
        kahan_add(T.drho, T.cdrho, d);
        kahan_add(T.ax, T.cax, x);
        kahan_add(T.ay, T.cay, y);
        kahan_add(T.az, T.caz, z);
    } else if (K.artp) {
        pair_terms<true, false>(K, nb, T, j, T.drho, T.ax, T.ay, T.az);
    } else {
        pair_terms<false, false>(K, nb, T, j, T.drho, T.ax, T.ay, T.az);
    }
}

__device__ __forceinline__ void store_rates(const Parameters* __restrict__ P, const PairConst& K, const Rates& rt,
                                            int i, const Target& T)
{
    rt.accad[i] = make_float4(K.m * T.ax + __ldg(&P->acc_x), K.m * T.ay + __ldg(&P->acc_y),
                              K.m * T.az + __ldg(&P->acc_z), K.m * T.drho);
    rt.spin[i] = make_float4(0.5f * (T.l10 - T.l01), 0.5f * (T.l20 - T.l02), 0.5f * (T.l21 - T.l12), 0.0f);
    store_t2(rt.acestn, i,
             make_tensor2d(T.l00, T.l11, T.l22, 0.5f * (T.l01 + T.l10), 0.5f * (T.l02 + T.l20),
                           0.5f * (T.l12 + T.l21)));
}

/* The 27-cell walk of one particle (both layers), calling f(j) for every
 * candidate that passes the distance test, in the order shared by every
 * neighbour visit of this file: layer, then column (dy outer, dx inner),
 * then slot. */
template <class F>
__device__ __forceinline__ void walk_stencil(const Parameters* __restrict__ P, const PairConst& K, const State& st,
                                             const Cells& cells, int i, const float4& xi, F&& f,
                                             const Frames& fr = Frames())
{
    const int nx = __ldg(&P->cell_num_x), ny = __ldg(&P->cell_num_y), nz = __ldg(&P->cell_num_z);
    const int L = __ldg(&P->ncell_one_layer);
    const int cx = stencil_axis(xi.x, K.ih), cz = stencil_axis(xi.z, K.ih);
    int cy = stencil_axis(xi.y, K.ih);
    if (fr.rows) cy = frame_stencil_row(fr, __ldg(&st.idep[i].x), cy);
    const int zlo = max(cz - 1, 0), zhi = min(cz + 1, nz - 1);
    if (zlo > zhi) return;
    for (int layer = 0; layer < 2; ++layer) {
        const int off = layer ? L : 0;
        for (int col = 0; col < 9; ++col) {
            const int X = cx + (col % 3) - 1, Y = cy + (col / 3) - 1;
            if (X < 0 || X >= nx || Y < 0 || Y >= ny) continue;
            int s, e;
            if (!zrun_range(cells, off + (X * ny + Y) * nz, zlo, zhi, s, e)) continue;
            for (int j = s; j < e; ++j) {
                const float4 xj = __ldg(st.pos + j);
                const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
                if (dx * dx + dy * dy + dz * dz < K.cut2 && j != i) f(j);
            }
        }
    }
}

#ifndef LQ_PAIR_MIN_BLOCKS
#define LQ_PAIR_MIN_BLOCKS 6   /* 128-thread blocks per SM: 80 registers */
#endif

constexpr int kListWarps = kBlock / 32;
constexpr int kStage = 32;
constexpr int kUnroll = 8;

/* Neighbour lists: list[k * stride + t] is the k-th neighbour slot of target
 * slot first + t, count[t] their number (entries past LQ_NBR_CAP are not
 * stored).  Candidates come from grid layers layer_lo..1 (0: both layers,
 * 1: material only) and are kept when r^2 < cut2, the cut-off (2h) plus any
 * skin.  Lanes are grouped by grid column; each group
 * walks the union of its lanes' stencils, so the loop and every candidate
 * load are warp-uniform and each lane only runs its distance test.  A lane's
 * own slot passes the test too: its pair adds exactly zero.  Along z the
 * walk covers every cell the lane's cut-off sphere reaches (two cells down
 * or up when the particle lies within the skin of a cell face), so a list
 * holds all its particle's pairs within the cut-off in those columns,
 * whatever the group; across columns it covers the 3 x 3 around the
 * particle's own, which holds every pair within 2h.  A pair within
 * 2h + skin that lies two columns apart is left out: it is more than 2h
 * apart when the list is built, so until the next build its distance stays
 * above 2h - skin (q > 2 - skin/h), where the kernel factor (2 - q)^3 stays
 * below (skin/h)^3.  Hits are staged per lane in shared memory and flushed
 * in rows.
 *
 * With `shell` (the wide build of two-level lists) the hits are split: those
 * with r^2 < inner2 go to `list` (count_out[t] of them) and the rest to
 * shell (shell_count[t]), each list in hit order; each part stores at most
 * LQ_NBR_CAP entries. */
template <bool kSplit>
__global__ void __launch_bounds__(kBlock) k_neighbor_list(const Parameters* __restrict__ P, int first, int ntarget,
                                                          int layer_lo, float cut2, const float4* __restrict__ pos,
                                                          Cells cells, int* __restrict__ list,
                                                          int* __restrict__ count_out, int stride,
                                                          int* __restrict__ health, const float4* __restrict__ idep,
                                                          Frames fr, int* __restrict__ shell,
                                                          int* __restrict__ shell_count, float inner2,
                                                          const int* __restrict__ gate)
{
    if (gate && *gate == 0) return;     /* the whole grid leaves: no collective is split */
    __shared__ int stage[kListWarps][kStage][32];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = first + t;
    const bool active = t < ntarget;
    const PairConst K = load_pair_const(P);
    const int nx = __ldg(&P->cell_num_x), ny = __ldg(&P->cell_num_y), nz = __ldg(&P->cell_num_z);
    const int L = __ldg(&P->ncell_one_layer);
    const int np_all = __ldg(&P->np);
    const float4 xi = active ? __ldg(pos + i) : make_float4(0.f, 0.f, 0.f, 0.f);
    int* my_stage = &stage[w][0][lane];

    /* staged hits carry bit 31 when they go to the shell part */
    int staged = 0, ni = 0, ns = 0;
    auto flush = [&]() {
        const int maxc = (int)__reduce_max_sync(FULL, (unsigned)staged);
        for (int k = 0; k < maxc; ++k)
            if (k < staged) {
                const int e = my_stage[32 * k];
                if (kSplit && e < 0) {
                    if (ns < LQ_NBR_CAP) shell[(size_t)ns * stride + t] = e & 0x7fffffff;
                    ++ns;
                } else {
                    if (ni < LQ_NBR_CAP) list[(size_t)ni * stride + t] = e;
                    ++ni;
                }
            }
        staged = 0;
        __syncwarp();
    };
    auto test = [&](bool mine, const float4& xj, int j) {
        const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        const float r2 = dx * dx + dy * dy + dz * dz;
        if (mine && r2 < cut2) {
            my_stage[32 * staged] = (kSplit && !(r2 < inner2)) ? (int)((unsigned)j | 0x80000000u) : j;
            ++staged;
        }
    };

    /* the z cells the particle's cut-off sphere reaches (a run walks the
     * group's union of them), so a lane's list never depends on which
     * other lanes share its group */
    const float cut = sqrtf(cut2);
    int cx = 0, cy = 0, czl = 0, czh = 0;
    if (active) {
        cx = stencil_axis(xi.x, K.ih);
        cy = stencil_axis(xi.y, K.ih);
        czl = stencil_axis(xi.z - cut, K.ih);
        czh = stencil_axis(xi.z + cut, K.ih);
        if (fr.rows) cy = frame_stencil_row(fr, __ldg(&idep[i].x), cy);
    }
    unsigned todo = __ballot_sync(FULL, active);
    while (todo) {
        const int leader = __ffs(todo) - 1;
        const int gx = __shfl_sync(FULL, cx, leader), gy = __shfl_sync(FULL, cy, leader);
        const bool mine = active && cx == gx && cy == gy;
        todo &= ~__ballot_sync(FULL, mine);
        const int zmin = __reduce_min_sync(FULL, mine ? czl : INT_MAX);
        const int zmax = __reduce_max_sync(FULL, mine ? czh : INT_MIN);
        const int zlo = max(zmin, 0), zhi = min(zmax, nz - 1);
        if (zlo > zhi) continue;
        for (int layer = layer_lo; layer < 2; ++layer) {
            const int off = layer ? L : 0;
            for (int col = 0; col < 9; ++col) {
                const int X = gx + (col % 3) - 1, Y = gy + (col / 3) - 1;
                if (X < 0 || X >= nx || Y < 0 || Y >= ny) continue;
                int s, e;
                if (!zrun_range(cells, off + (X * ny + Y) * nz, zlo, zhi, s, e)) continue;
                if (!lq_in_range(s, np_all) || !lq_in_range(e - 1, np_all)) continue;
                int j = s;
                for (; j + kUnroll <= e; j += kUnroll) {
                    if (__any_sync(FULL, staged > kStage - kUnroll)) flush();
                    float4 xj[kUnroll];
#pragma unroll
                    for (int u = 0; u < kUnroll; ++u) xj[u] = __ldg(pos + j + u);
#pragma unroll
                    for (int u = 0; u < kUnroll; ++u) test(mine, xj[u], j + u);
                }
                if (__any_sync(FULL, staged > kStage - kUnroll)) flush();
                for (; j < e; ++j) test(mine, __ldg(pos + j), j);
            }
        }
    }
    flush();
    if (active) {
        count_out[t] = ni;
        if (kSplit) shell_count[t] = ns;
        if ((ni > LQ_NBR_CAP || ns > LQ_NBR_CAP) && health) atomicAdd(health + HEALTH_NBR_OVERFLOW, 1);
    }
}

/* Slot i's packed record, at i or (with map) at map[i], the index lists
 * of another slot order gather it at (slots with none are skipped). */
template <bool kPk>
__global__ void __launch_bounds__(kBlock) k_pack_neighbors(int first, int np, State st, NbrArrays nb,
                                                           const int* __restrict__ map)
{
    const int i = first + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    int o = i;
    if (map) {
        o = __ldg(map + i);
        if ((unsigned)o >= (unsigned)np) return;
    }
    const float4 x = __ldg(st.pos + i);
    const float4 v = __ldg(st.vel + i);
    nb.xr[o] = make_float4(x.x, x.y, x.z, v.w);
    store_packed<kPk>(nb, o, v, load_t2(st.str, i));
}

/* A list entry: each 128-byte row of a list is read once per launch, so it
 * bypasses L1 (no allocation) and leaves L1 to the neighbour data that the
 * targets of a block share. */
__device__ __forceinline__ int ld_list(const int* p)
{
    int v;
    asm("ld.global.nc.L1::no_allocate.b32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

/* Two-level lists: the lists the stages read (cut-off 2h + skin) renewed
 * at the current positions without a search.  The wide build (cut-off
 * 2h + wide) wrote each target's pairs closer than inner = 2h + 2 skin -
 * wide into rows [0, ni) of the stages' list and the rest into its shell
 * list.  While no particle has moved (wide - skin) / 2 from its position at
 * that build (the corrector's check), a pair's distance has changed by less
 * than wide - skin, so every inner pair is still within 2h + skin and every
 * pair now within 2h + skin was within 2h + wide: the renewal keeps rows
 * [0, ni) as they are and appends, in their order, the shell entries now
 * within the cut-off.  Entries are fetched a group ahead so the position
 * gathers overlap.  Overflows keep LQ_NBR_CAP valid rows and a count above
 * it (the pair kernel then walks that target's stencil): a truncated shell
 * list fills the rows after the inner part with its stored entries. */
__global__ void __launch_bounds__(kBlock) k_list_refresh(int first, int ntarget, int np, float cut2,
                                                         const float4* __restrict__ pos,
                                                         const int* __restrict__ inner_count,
                                                         const int* __restrict__ shell,
                                                         const int* __restrict__ shell_count, int* __restrict__ list,
                                                         int* __restrict__ count, int stride,
                                                         int* __restrict__ health)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntarget) return;
    const int ni = __ldg(inner_count + t), ns = __ldg(shell_count + t);
    const int* p = shell + t;
    if (ni > LQ_NBR_CAP) {
        count[t] = ni;          /* rows [0, LQ_NBR_CAP) hold inner entries */
        return;
    }
    if (ns > LQ_NBR_CAP) {
        for (int k = 0; ni + k < LQ_NBR_CAP; ++k) list[(size_t)(ni + k) * stride + t] = ld_list(p + (size_t)k * stride);
        count[t] = ni + ns;
        return;
    }
    const int i = first + t;
    const float4 xi = __ldg(pos + i);
    /* groups of kG entries; the last group is filled up with the target's
     * own slot (a valid address; never kept) */
    constexpr int kG = 8;
    int nxt[kG];
#pragma unroll
    for (int u = 0; u < kG; ++u) nxt[u] = u < ns ? ld_list(p + (size_t)u * stride) : i;
    int n = ni;
    for (int k = 0; k < ns; k += kG) {
        int j[kG];
        float4 xj[kG];
#pragma unroll
        for (int u = 0; u < kG; ++u) {
            j[u] = nxt[u];
            nxt[u] = k + kG + u < ns ? ld_list(p + (size_t)(k + kG + u) * stride) : i;
        }
#pragma unroll
        for (int u = 0; u < kG; ++u) xj[u] = lq_in_range(j[u], np) ? __ldg(pos + j[u]) : xi;
#pragma unroll
        for (int u = 0; u < kG; ++u) {
            const float dx = xi.x - xj[u].x, dy = xi.y - xj[u].y, dz = xi.z - xj[u].z;
            if (k + u < ns && lq_in_range(j[u], np) && dx * dx + dy * dy + dz * dz < cut2) {
                if (n < LQ_NBR_CAP) list[(size_t)n * stride + t] = j[u];
                ++n;
            }
        }
    }
    count[t] = n;
    if (n > LQ_NBR_CAP && health) atomicAdd(health + HEALTH_NBR_OVERFLOW, 1);
}

/* The sums over one target's list (entry k at p[k * stride]), four
 * entries per group, the next group's entries fetched ahead so the
 * dependent neighbour loads do not wait on the list stream.  The last
 * group is filled up with the target itself (exact zeros), so a group has
 * no branch.  The compensated (mixed) form adds each group's plain sum of
 * four pairs to the compensated sums and reads the packed velocity. */
template <bool kKahan, bool kArtp>
__device__ __forceinline__ void list_sums(const PairConst& K, const NbrArrays& nb, Target& T, const int* p, int n,
                                          int stride, int i, int np)
{
    const size_t step4 = 4 * (size_t)stride;
    int nxt[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) nxt[u] = u < n ? ld_list(p + u * stride) : i;
    for (int k = 0; k < n; k += 4) {
        p += step4;
        int cur[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            cur[u] = nxt[u];
            nxt[u] = k + 4 + u < n ? ld_list(p + u * stride) : i;
        }
        if (kKahan) {
            float d = 0.f, x = 0.f, y = 0.f, z = 0.f;
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (lq_in_range(cur[u], np)) pair_terms<kArtp, true>(K, nb, T, cur[u], d, x, y, z);
            kahan_add(T.drho, T.cdrho, d);
            kahan_add(T.ax, T.cax, x);
            kahan_add(T.ay, T.cay, y);
            kahan_add(T.az, T.caz, z);
        } else {
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (lq_in_range(cur[u], np))
                    pair_terms<kArtp, false>(K, nb, T, cur[u], T.drho, T.ax, T.ay, T.az);
        }
    }
}

/* Pair sums over the lists from the packed neighbour arrays; a particle
 * whose list overflowed walks its stencil over the state arrays instead.
 * kThreads x kMinBlocks is the launch shape: the block size and
 * the resident blocks per SM the register allocation is capped for; the
 * shapes of kPairShapes are compiled and one is chosen per simulation
 * (lq_sim_autotune times them). */
template <bool kKahan, int kThreads, int kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_interaction_rec(
    const Parameters* __restrict__ P, int np, int npb, State st, Rates rt, Cells cells, const int* __restrict__ list,
    const int* __restrict__ count, int stride, Frames fr, NbrArrays nb, const int* __restrict__ order,
    const int* __restrict__ rows)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= np - npb) return;
    /* thread g takes target order[g] (tile order) or target g (slot order) */
    const int t = order ? __ldg(order + g) : g;
    if (!lq_in_range(t, np - npb)) return;
    const int i = npb + t;
    const PairConst K = load_pair_const(P);
    Target T;
    load_target(K, st, i, true, T);
    /* with rows: target t's list is row rows[t] (-1: none), whose entries
     * index records packed in that other slot order, the target's own at
     * npb + row (the filler of the last group) */
    int row = t, self = i;
    if (rows) {
        row = __ldg(rows + t);
        self = npb + row;
    }
    const int n = row >= 0 ? __ldg(count + row) : LQ_NBR_CAP + 1;
    if (n <= LQ_NBR_CAP) {
        if (K.artp)
            list_sums<kKahan, true>(K, nb, T, list + row, n, stride, self, np);
        else
            list_sums<kKahan, false>(K, nb, T, list + row, n, stride, self, np);
    } else {
        walk_stencil(P, K, st, cells, i, T.x, [&](int j) { pair_body<kKahan>(K, st, T, j); }, fr);
    }
    store_rates(P, K, rt, i, T);
}

/* ------------------------------------------------- tile order of targets */
/* The pair kernel's targets in tile order (lq_tile.h has the index
 * arithmetic): tiles of 3 x 3 columns by tz cells, each tile column one run
 * of consecutive slots.  A block of the pair kernel then holds a compact
 * box of targets whose neighbourhood fits in L1, instead of a thin z-run of
 * one column whose neighbours the next block on the SM does not share. */
__global__ void __launch_bounds__(kBlock) k_tile_segments(const int* __restrict__ start, TileGrid tg, int npb,
                                                          int np, int* __restrict__ seg_beg,
                                                          int* __restrict__ seg_len)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= tg.nseg) return;
    int b, len;
    tile_segment(tg, start, npb, np, s, &b, &len);
    seg_beg[s] = b;
    seg_len[s] = len;
}

/* One warp per segment writes its targets (slot - npb) at the segment's
 * offset. */
__global__ void __launch_bounds__(kBlock) k_tile_fill(int nseg, int npb, int npm, const int* __restrict__ seg_beg,
                                                      const int* __restrict__ seg_len,
                                                      const int* __restrict__ seg_off, int* __restrict__ order)
{
    const int w = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (w >= nseg) return;
    const int b = __ldg(seg_beg + w), n = __ldg(seg_len + w), o = __ldg(seg_off + w);
    for (int k = lane; k < n; k += 32)
        if (o + k < npm) order[o + k] = b + k - npb;
}

/* Warp-cooperative form: a group of G lanes (G = 8 or 32) shares one
 * target, lane g taking list entries g, g + G, ...; the group's partial sums
 * are combined with shuffle reductions.  With few targets (a small case) a
 * thread per target leaves most of the GPU idle and each thread's chain of
 * dependent gathers long; groups give G times the parallelism.  In the
 * compensated form each lane keeps its Kahan pair and the reduction adds
 * sum - compensation. */
template <int G>
__device__ __forceinline__ float group_sum(float v)
{
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, G);
    return v;
}

template <bool kKahan, int G>
__global__ void __launch_bounds__(128) k_interaction_group(const Parameters* __restrict__ P, int np, int npb,
                                                           State st, Rates rt, Cells cells,
                                                           const int* __restrict__ list,
                                                           const int* __restrict__ count, int stride, Frames fr,
                                                           NbrArrays nb)
{
    const int gid = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    const int g = threadIdx.x % G;
    const int t = gid;
    const int i = npb + t;
    const bool active = i < np;      /* whole groups leave together: no early return before the shuffles */
    const PairConst K = load_pair_const(P);
    Target T;
    load_target(K, st, active ? i : npb, active, T);
    const int n = active ? __ldg(count + t) : 0;
    if (n <= LQ_NBR_CAP) {
        for (int k = g; k < n; k += G) {
            const int j = __ldg(list + (size_t)k * stride + t);
            if (lq_in_range(j, np)) pair_body_rec<kKahan>(K, nb, T, j);
        }
    } else if (g == 0) {
        walk_stencil(P, K, st, cells, i, T.x, [&](int j) { pair_body<kKahan>(K, st, T, j); }, fr);
    }
    if (kKahan) {
        T.drho -= T.cdrho;
        T.ax -= T.cax;
        T.ay -= T.cay;
        T.az -= T.caz;
    }
    T.drho = group_sum<G>(T.drho);
    T.ax = group_sum<G>(T.ax);
    T.ay = group_sum<G>(T.ay);
    T.az = group_sum<G>(T.az);
    T.l00 = group_sum<G>(T.l00); T.l01 = group_sum<G>(T.l01); T.l02 = group_sum<G>(T.l02);
    T.l10 = group_sum<G>(T.l10); T.l11 = group_sum<G>(T.l11); T.l12 = group_sum<G>(T.l12);
    T.l20 = group_sum<G>(T.l20); T.l21 = group_sum<G>(T.l21); T.l22 = group_sum<G>(T.l22);
    if (active && g == 0) store_rates(P, K, rt, i, T);
}

/* ------------------------------------------------------------- Adami */
/* Per-cell visiting order and the float expressions follow the reference
 * kernel (src/adami_boundary.cu:27-123) so both produce the same sums. */
__device__ __forceinline__ bool cell_range(const Cells& c, int cell, int& s, int& e)
{
    if (c.start) {
        s = __ldg(c.start + cell);
        e = __ldg(c.start + cell + 1);
        return e > s;
    }
    s = __ldg(c.beg + cell);
    if (s == -1) return false;
    e = __ldg(c.end + cell);
    return true;
}

__global__ void __launch_bounds__(kBlock) k_adami(const Parameters* __restrict__ P, int npb, State st, Cells cells)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npb) return;
    const float ih = __ldg(&P->i_h), m = __ldg(&P->m), Cw = __ldg(&P->kernel_normalization_par);
    const int nx = __ldg(&P->cell_num_x), ny = __ldg(&P->cell_num_y), nz = __ldg(&P->cell_num_z);
    const int L = __ldg(&P->ncell_one_layer);
    const float4 xi = __ldg(st.pos + i);
    tensor2d S = make_tensor2d(0.0f);
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    const int cx = stencil_axis(xi.x, ih), cy = stencil_axis(xi.y, ih), cz = stencil_axis(xi.z, ih);
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const int X = cx + dx, Y = cy + dy, Z = cz + dz;
                if (X < 0 || X > nx - 1 || Y < 0 || Y > ny - 1 || Z < 0 || Z > nz - 1) continue;
                int s, e;
                if (!cell_range(cells, X * ny * nz + Y * nz + Z + L, s, e)) continue;
                for (int j = s; j < e; ++j) {
                    const float4 xj = __ldg(st.pos + j);
                    const float3 d = make_float3(xi.x - xj.x, xi.y - xj.y, xi.z - xj.z);
                    const float q = norm3df(d.x, d.y, d.z) * ih;
                    if (q < 2.0f) {
                        const float ker = Cw * (2.0f - q) * (2.0f - q) * (2.0f - q) * (2.0f - q) * (q + 0.5f);
                        const float vol = m / __ldg(&st.vel[j].w);
                        const tensor2d sj = load_t2(st.str, j);
                        S.xx += sj.xx * ker * vol;
                        S.yy += sj.yy * ker * vol;
                        S.zz += sj.zz * ker * vol;
                        S.xy += sj.xy * ker * vol;
                        S.xz += sj.xz * ker * vol;
                        S.yz += sj.yz * ker * vol;
                        acc.x += d.x * ker * vol;
                        acc.y += d.y * ker * vol;
                        acc.z += d.z * ker * vol;
                        acc.w += ker * vol;
                    }
                }
            }
    if (acc.w > 0.0f) {
        const float rho0 = __ldg(&P->rho0);
        tensor2d out;
        out.xx = (S.xx - rho0 * __ldg(&P->acc_x) * acc.x) / acc.w;
        out.yy = (S.yy - rho0 * __ldg(&P->acc_y) * acc.y) / acc.w;
        out.zz = (S.zz - rho0 * __ldg(&P->acc_z) * acc.z) / acc.w;
        out.xy = S.xy / acc.w;
        out.xz = S.xz / acc.w;
        out.yz = S.yz / acc.w;
        store_t2(st.str, i, out);
    }
}

/* ------------------------------------------------------------ Shepard */
/* Reference kernel src/field_smoothing.cu:65-121: material layer, self
 * included, no guard on a zero weight sum. */
__global__ void __launch_bounds__(kBlock) k_shepard(const Parameters* __restrict__ P, int np, int npb, State st,
                                                    tensor2d* __restrict__ out_str, State full, bool copy_full,
                                                    Cells cells)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np) return;
    if (t < npb) {
        if (copy_full) {
            full.pos[t] = __ldg(st.pos + t);
            full.vel[t] = __ldg(st.vel + t);
            full.idep[t] = __ldg(st.idep + t);
            store_t2(full.str, t, load_t2(st.str, t));
            store_t2(full.stn, t, load_t2(st.stn, t));
        }
        return;
    }
    const int i = t;
    const float ih = __ldg(&P->i_h), m = __ldg(&P->m), Cw = __ldg(&P->kernel_normalization_par);
    const int nx = __ldg(&P->cell_num_x), ny = __ldg(&P->cell_num_y), nz = __ldg(&P->cell_num_z);
    const int L = __ldg(&P->ncell_one_layer);
    const float4 xi = __ldg(st.pos + i);
    tensor2d S = make_tensor2d(0.0f);
    float w = 0.0f;
    const int cx = stencil_axis(xi.x, ih), cy = stencil_axis(xi.y, ih), cz = stencil_axis(xi.z, ih);
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const int X = cx + dx, Y = cy + dy, Z = cz + dz;
                if (X < 0 || X > nx - 1 || Y < 0 || Y > ny - 1 || Z < 0 || Z > nz - 1) continue;
                int s, e;
                if (!cell_range(cells, X * ny * nz + Y * nz + Z + L, s, e)) continue;
                for (int j = s; j < e; ++j) {
                    const float4 xj = __ldg(st.pos + j);
                    const float3 d = make_float3(xi.x - xj.x, xi.y - xj.y, xi.z - xj.z);
                    const float q = norm3df(d.x, d.y, d.z) * ih;
                    if (q < 2.0f) {
                        const float ker = Cw * (2.0f - q) * (2.0f - q) * (2.0f - q) * (2.0f - q) * (q + 0.5f);
                        const float vol = m / __ldg(&st.vel[j].w);
                        const tensor2d sj = load_t2(st.str, j);
                        S.xx += sj.xx * ker * vol;
                        S.yy += sj.yy * ker * vol;
                        S.zz += sj.zz * ker * vol;
                        S.xy += sj.xy * ker * vol;
                        S.xz += sj.xz * ker * vol;
                        S.yz += sj.yz * ker * vol;
                        w += ker * vol;
                    }
                }
            }
    S.xx /= w;
    S.yy /= w;
    S.zz /= w;
    S.xy /= w;
    S.xz /= w;
    S.yz /= w;
    store_t2(out_str, i, S);
    if (copy_full) {
        full.pos[i] = xi;
        full.vel[i] = __ldg(st.vel + i);
        full.idep[i] = __ldg(st.idep + i);
        store_t2(full.stn, i, load_t2(st.stn, i));
    }
}

/* ------------------------------------------------- list-driven Adami */
/* The Adami extrapolation of k_adami, summed over a boundary particle's
 * list of material neighbours (built with a skin; pairs at q >= 2 add
 * exact zeros, as the cell walk skips them), reading the neighbours from
 * the packed arrays (sigma_j V_j W = s_j rho_j m W with s = sigma / rho^2),
 * and writing the
 * boundary particle's new stress into the state (and into str2, the native
 * driver's other state buffer, whose boundary slots so always equal the
 * state's) and, scaled, into the packed arrays, which then need no pack of
 * the boundary slots before the pair kernel.  Targets without neighbours
 * keep all of them as they were.  With `act`, thread t takes the boundary
 * slot act[t] for t < *nact (the slots whose lists can hold entries, in
 * slot order, from launch_boundary_targets): most boundary particles of a
 * wall have no material neighbour, and without the compaction a warp ran
 * as long as its longest list over lanes that had none.  Each target's
 * sums run in list order in one thread either way, so the results do not
 * depend on the compaction. */
/* threads per block of the list-driven Adami: 128 measured against 64 and
 * 256 (256: -4 % on the 256-scenario ensemble, +10 % on the cylinder; 64:
 * +1 % and equal) */
#ifndef LQ_ADAMI_BLOCK
#define LQ_ADAMI_BLOCK 128
#endif
/* Entries per group of the list-driven Adami, chosen per launch: groups of
 * four where the targets fit in about one wave of the GPU (each thread's
 * chain of dependent gathers is then the time: the cylinder's 0.34 M
 * boundary particles, ~19 entries per active one), pairs from
 * kAdamiPairTargets boundary particles on (48 registers against 62: more
 * warps and fewer filler entries where enough targets keep the memory
 * system busy; on the 256-scenario ensemble's 16.2 M, 1.17 against 1.28 ms
 * per step, groups of eight 1.24).  The sums do not depend on the group
 * size.  The bounds-checked build sets the threshold to 0, so its tests
 * take the pairs path. */
#ifndef LQ_ADAMI_PAIR_TARGETS
#define LQ_ADAMI_PAIR_TARGETS (4 << 20)
#endif
constexpr int kAdamiPairTargets = LQ_ADAMI_PAIR_TARGETS;
template <int kG>
__global__ void __launch_bounds__(LQ_ADAMI_BLOCK) k_adami_packed(const Parameters* __restrict__ P, int npb, State st,
                                                         const int* __restrict__ list,
                                                         const int* __restrict__ count, int stride, NbrArrays nb,
                                                         tensor2d* __restrict__ str2, const int* __restrict__ act,
                                                         const int* __restrict__ nact)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npb) return;
    if (act) {
        /* act holds npb slots, so both loads are issued together */
        const int na = __ldg(nact), a = __ldg(act + i);
        if (i >= na) return;
        i = a;
    }
    const int n = min(__ldg(count + i), LQ_NBR_CAP);
    if (n == 0) return;
    const int np_all = __ldg(&P->np);
    const float ih = __ldg(&P->i_h), m = __ldg(&P->m), Cw = __ldg(&P->kernel_normalization_par);
    const float4 xi = __ldg(st.pos + i);
    tensor2d S = make_tensor2d(0.0f);
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    /* groups of kG entries, the next group's entries fetched ahead and
     * every gather of a group issued together; a pair at q >= 2 (and the
     * filler of the last group, the target's own record) gets the kernel
     * factor 0 and adds exact zeros, so the loop has no branch and its sums
     * do not depend on kG */
    const int* p = list + i;
    int nxt[kG];
#pragma unroll
    for (int u = 0; u < kG; ++u) nxt[u] = u < n ? __ldg(p + (size_t)u * stride) : i;
    for (int k = 0; k < n; k += kG) {
        int j[kG];
#pragma unroll
        for (int u = 0; u < kG; ++u) {
            j[u] = lq_in_range(nxt[u], np_all) ? nxt[u] : i;
            nxt[u] = k + kG + u < n ? __ldg(p + (size_t)(k + kG + u) * stride) : i;
        }
        float4 xr[kG], sa[kG];
        float2 sb[kG];
#pragma unroll
        for (int u = 0; u < kG; ++u) {
            xr[u] = __ldg(nb.xr + j[u]);
            sa[u] = __ldg(nb.sa + j[u]);
            sb[u] = __ldg(reinterpret_cast<const float2*>(nb.sb + j[u]));
        }
#pragma unroll
        for (int u = 0; u < kG; ++u) {
            const float3 d = make_float3(xi.x - xr[u].x, xi.y - xr[u].y, xi.z - xr[u].z);
            /* the approximate square root and quotient of the pair kernel */
            const float q = sqrt_approx(d.x * d.x + d.y * d.y + d.z * d.z) * ih;
            const float t = k + u < n ? fmaxf(2.0f - q, 0.0f) : 0.0f;
            const float ker = Cw * t * t * t * t * (q + 0.5f);
            const float kv = ker * __fdividef(m, xr[u].w);
            const float cs = m * xr[u].w * ker;
            S.xx += sa[u].x * cs;
            S.yy += sa[u].y * cs;
            S.zz += sa[u].z * cs;
            S.xy += sa[u].w * cs;
            S.xz += sb[u].x * cs;
            S.yz += sb[u].y * cs;
            acc.x += d.x * kv;
            acc.y += d.y * kv;
            acc.z += d.z * kv;
            acc.w += kv;
        }
    }
    if (acc.w > 0.0f) {
        const float rho0 = __ldg(&P->rho0);
        const float inv = 1.0f / acc.w;
        tensor2d out;
        out.xx = (S.xx - rho0 * __ldg(&P->acc_x) * acc.x) * inv;
        out.yy = (S.yy - rho0 * __ldg(&P->acc_y) * acc.y) * inv;
        out.zz = (S.zz - rho0 * __ldg(&P->acc_z) * acc.z) * inv;
        out.xy = S.xy * inv;
        out.xz = S.xz * inv;
        out.yz = S.yz * inv;
        store_t2(st.str, i, out);
        if (str2) store_t2(str2, i, out);
        /* a boundary particle's velocity and density stay as the list
         * build packed them; only its stress words change */
        store_packed_stress(nb, i, __ldg(&st.vel[i].w), out);
    }
}

/* ------------------------------------------ list-driven Shepard filters */
/* The walk of the native driver's two filters over a material target's
 * list, from the packed records (written from the state the filter reads:
 * the corrector packs every material slot, and each filter packs again
 * after changing the state): branch-free groups of four, the next group's
 * entries fetched ahead.  add(W, xr, sa, sb) gets the kernel value of each
 * entry, 0 for boundary neighbours (the filters use the material layer
 * only), for pairs at q >= 2 and for the filler of the last group (the
 * target's own slot); the list holds the target itself at q = 0.  kStress
 * also gathers the sigma / rho^2 words. */
template <bool kStress, class F>
__device__ __forceinline__ void filter_groups(const NbrArrays& nb, const int* p, int n, int stride, int i, int npb,
                                              int np, const float4& xi, float ih, float Cw, F&& add)
{
    int nxt[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) nxt[u] = u < n ? ld_list(p + (size_t)u * stride) : i;
    for (int k = 0; k < n; k += 4) {
        int j[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            j[u] = lq_in_range(nxt[u], np) ? nxt[u] : i;
            nxt[u] = k + 4 + u < n ? ld_list(p + (size_t)(k + 4 + u) * stride) : i;
        }
        float4 xr[4], sa[4];
        float2 sb[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            xr[u] = __ldg(nb.xr + j[u]);
            if (kStress) {
                sa[u] = __ldg(nb.sa + j[u]);
                sb[u] = __ldg(reinterpret_cast<const float2*>(nb.sb + j[u]));
            } else {
                sa[u] = make_float4(0.f, 0.f, 0.f, 0.f);
                sb[u] = make_float2(0.f, 0.f);
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float dx = xi.x - xr[u].x, dy = xi.y - xr[u].y, dz = xi.z - xr[u].z;
            const float q = sqrt_approx(dx * dx + dy * dy + dz * dz) * ih;
            const float t = (k + u < n && j[u] >= npb) ? fmaxf(2.0f - q, 0.0f) : 0.0f;
            add(Cw * t * t * t * t * (q + 0.5f), xr[u], sa[u], sb[u]);
        }
    }
}

/* The Shepard stress filter of k_shepard over a material particle's list:
 * sum sigma_j V_j W / sum V_j W over the material neighbours, with
 * sigma_j V_j W = s_j rho_j m W from the packed records (s = sigma /
 * rho^2, as Adami reads them).  Targets in the pair kernel's tile order
 * when `order` is set.  A particle whose list overflowed walks its 27
 * cells over the state instead.  Writes the filtered stress of material
 * slots to out_str. */
__global__ void __launch_bounds__(kBlock) k_shepard_list(const Parameters* __restrict__ P, int np, int npb, State st,
                                                         tensor2d* __restrict__ out_str,
                                                         const int* __restrict__ list,
                                                         const int* __restrict__ count, int stride, Cells cells,
                                                         Frames fr, NbrArrays nb, const int* __restrict__ order)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= np - npb) return;
    const int t = order ? __ldg(order + g) : g;
    if (!lq_in_range(t, np - npb)) return;
    const int i = npb + t;
    const int n = __ldg(count + t);
    const float ih = __ldg(&P->i_h), m = __ldg(&P->m), Cw = __ldg(&P->kernel_normalization_par);
    const float4 xi = __ldg(st.pos + i);
    tensor2d S = make_tensor2d(0.0f);
    float w = 0.0f;
    if (n <= LQ_NBR_CAP) {
        filter_groups<true>(nb, list + t, n, stride, i, npb, np, xi, ih, Cw,
                            [&](float ker, const float4& xr, const float4& sa, const float2& sb) {
                                const float cs = m * xr.w * ker;
                                S.xx += sa.x * cs;
                                S.yy += sa.y * cs;
                                S.zz += sa.z * cs;
                                S.xy += sa.w * cs;
                                S.xz += sb.x * cs;
                                S.yz += sb.y * cs;
                                w += ker * __fdividef(m, xr.w);
                            });
    } else {
        /* overflowed list (counted in the health word): the particle itself
         * and its 27-cell walk in the grid the lists were built from, as
         * the pair kernel does */
        auto add = [&](int j) {
            if (j < npb || !lq_in_range(j, np)) return;
            const float4 xj = __ldg(st.pos + j);
            const float3 d = make_float3(xi.x - xj.x, xi.y - xj.y, xi.z - xj.z);
            const float q = norm3df(d.x, d.y, d.z) * ih;
            if (q < 2.0f) {
                const float ker = Cw * (2.0f - q) * (2.0f - q) * (2.0f - q) * (2.0f - q) * (q + 0.5f);
                const float vol = m / __ldg(&st.vel[j].w);
                const tensor2d sj = load_t2(st.str, j);
                S.xx += sj.xx * ker * vol;
                S.yy += sj.yy * ker * vol;
                S.zz += sj.zz * ker * vol;
                S.xy += sj.xy * ker * vol;
                S.xz += sj.xz * ker * vol;
                S.yz += sj.yz * ker * vol;
                w += ker * vol;
            }
        };
        add(i);
        walk_stencil(P, load_pair_const(P), st, cells, i, xi, add, fr);
    }
    const float inv = 1.0f / w;
    S.xx *= inv;
    S.yy *= inv;
    S.zz *= inv;
    S.xy *= inv;
    S.xz *= inv;
    S.yz *= inv;
    store_t2(out_str, i, S);
}

/* Density Shepard filter over a material particle's list (boundary
 * neighbours skipped; the list holds the particle itself, at q = 0):
 * rho~_i = sum m W / sum (m / rho_j) W, from the packed records' positions
 * and densities; targets in tile order when `order` is set. */
__global__ void __launch_bounds__(kBlock) k_density_filter_list(const Parameters* __restrict__ P, int np, int npb,
                                                                State st, float* __restrict__ rho_out,
                                                                const int* __restrict__ list,
                                                                const int* __restrict__ count, int stride,
                                                                Cells cells, Frames fr, NbrArrays nb,
                                                                const int* __restrict__ order)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= np - npb) return;
    const int t = order ? __ldg(order + g) : g;
    if (!lq_in_range(t, np - npb)) return;
    const int i = npb + t;
    const int n = __ldg(count + t);
    const float ih = __ldg(&P->i_h), m = __ldg(&P->m), Cw = __ldg(&P->kernel_normalization_par);
    const float4 xi = __ldg(st.pos + i);
    float num = 0.0f, den = 0.0f;
    if (n <= LQ_NBR_CAP) {
        filter_groups<false>(nb, list + t, n, stride, i, npb, np, xi, ih, Cw,
                             [&](float ker, const float4& xr, const float4&, const float2&) {
                                 num += m * ker;
                                 den += ker * __fdividef(m, xr.w);
                             });
    } else {
        /* overflowed list: the particle itself and its 27-cell walk */
        auto add = [&](int j) {
            if (j < npb || !lq_in_range(j, np)) return;
            const float4 xj = __ldg(st.pos + j);
            const float3 d = make_float3(xi.x - xj.x, xi.y - xj.y, xi.z - xj.z);
            const float q = norm3df(d.x, d.y, d.z) * ih;
            if (q < 2.0f) {
                const float ker = Cw * (2.0f - q) * (2.0f - q) * (2.0f - q) * (2.0f - q) * (q + 0.5f);
                num += m * ker;
                den += ker * (m / __ldg(&st.vel[j].w));
            }
        };
        add(i);
        walk_stencil(P, load_pair_const(P), st, cells, i, xi, add, fr);
    }
    rho_out[i] = num / den;
}

}  // namespace

int launch_density_filter_list(const Parameters* ph, const Parameters* pd, const State& st, float* rho_out,
                               const NeighborList& nl, const Cells& c, cudaStream_t s, const Frames& fr,
                               float* rec, const int* order)
{
    if (ph->npm <= 0) return LQ_OK;
    if (!rec) return set_error(LQ_ERR_ARG, "density filter: the packed neighbour records are required");
    k_density_filter_list<<<blocks_for(ph->npm, kBlock), kBlock, 0, s>>>(pd, ph->np, ph->npb, st, rho_out, nl.list,
                                                                        nl.count, nl.stride, c, fr,
                                                                        nbr_arrays(rec, ph->np), order);
    LQ_TRY_CUDA(cudaGetLastError(), "k_density_filter_list");
    return LQ_OK;
}

/* Launch shapes of the pair kernel: threads per block x resident blocks
 * per SM (the register cap); a negative second entry -G marks the
 * warp-cooperative form with G lanes per target.  Shape 0 is the default. */
const int kPairShapes[kPairShapeCount][3] = {{kBlock, LQ_PAIR_MIN_BLOCKS, 0},
                                             {64, 12, 0},
                                             {256, 3, 0},
                                             {128, 5, 0},
                                             {128, 7, 0},
                                             {128, -8, 0},
                                             {128, -32, 0},
                                             {768, 1, 1},
                                             {384, 2, 1},
                                             {640, 1, 1},
                                             {320, 2, 1}};

/* The native driver's launch shape before any tuning: the tiled 640 x 1
 * shape once the targets fill at least four waves of 640-thread blocks on
 * every SM, the 128-thread shape 0 below that (a small case would leave
 * SMs idle with large blocks). */
int default_pair_shape(int npm)
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                  cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return (long long)npm >= 4LL * sms * kPairShapes[kDefaultTiledShape][0] ? kDefaultTiledShape : 0;
}

/* Tile height (cells) for a block of `threads` targets: a 3 x 3-column
 * tile of that height holds about one block at (2 h / dr)^3 particles per
 * cell. */
static int tile_height(const Parameters* ph, int threads)
{
    const double ppc = std::pow(2.0 * (double)ph->hdr, 3.0);
    const int tz = (int)std::lround((double)threads / (9.0 * (ppc > 1.0 ? ppc : 1.0)));
    return tz < 1 ? 1 : tz;
}

static TileGrid tile_grid_of(const Parameters* ph, int tz)
{
    return tile_grid(ph->cell_num_x, ph->cell_num_y, ph->cell_num_z, ph->ncell_one_layer, tz);
}

int tile_order_scratch(const Parameters* ph, int* nseg, size_t* scan_bytes)
{
    *nseg = tile_grid_of(ph, 1).nseg;   /* the most segments any tile height needs */
    *scan_bytes = 0;
    LQ_TRY_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, *scan_bytes, (const int*)nullptr, (int*)nullptr, *nseg),
                "tile scan scratch query");
    return LQ_OK;
}


int launch_tile_order(const Parameters* ph, const int* start, int shape, const TileOrder& to, cudaStream_t s)
{
    if (shape < 0 || shape >= kPairShapeCount || kPairShapes[shape][2] != 1 || ph->npm <= 0) return LQ_OK;
    if (!to.order || !to.seg) return set_error(LQ_ERR_ARG, "tile order: buffers not allocated");
    const TileGrid tg = tile_grid_of(ph, tile_height(ph, kPairShapes[shape][0]));
    const int nseg = tg.nseg;
    if (nseg > to.nseg_cap) return set_error(LQ_ERR_ARG, "tile order: %d segments > capacity %d", nseg, to.nseg_cap);
    int* beg = to.seg;
    int* len = to.seg + to.nseg_cap;
    int* off = to.seg + 2 * (size_t)to.nseg_cap;
    k_tile_segments<<<blocks_for(nseg, kBlock), kBlock, 0, s>>>(start, tg, ph->npb, ph->np, beg, len);
    LQ_TRY_CUDA(cudaGetLastError(), "k_tile_segments");
    size_t bytes = to.scan_bytes;
    LQ_TRY_CUDA(cub::DeviceScan::ExclusiveSum(to.scan_tmp, bytes, len, off, nseg, s), "tile scan");
    k_tile_fill<<<blocks_for(nseg, kBlock / 32), kBlock, 0, s>>>(nseg, ph->npb, ph->npm, beg, len, off, to.order);
    LQ_TRY_CUDA(cudaGetLastError(), "k_tile_fill");
    return LQ_OK;
}

/* This translation unit's count of bounds violations (always 0 without
 * LQ_CHECKED). */
int bounds_count_sph(unsigned long long* v)
{
#ifdef LQ_CHECKED
    LQ_TRY_CUDA(cudaMemcpyFromSymbol(v, lq_bounds_count, sizeof(*v)), "bounds counter");
#else
    *v = 0;
#endif
    return LQ_OK;
}


int launch_neighbor_list(const Parameters* ph, const Parameters* pd, const float4* pos, const Cells& c,
                         const NeighborList& nl, cudaStream_t s)
{
    return launch_neighbor_list_range(ph, pd, ph->npb, ph->npm, 0, 2.0f * ph->h * 1.00005f, pos, c, nl, nullptr, s);
}

int launch_list_refresh(const Parameters* ph, int first, int n, float cut, const float4* pos,
                        const int* inner_count, const NeighborList& shell, const NeighborList& nl, int* health,
                        cudaStream_t s)
{
    if (n <= 0) return LQ_OK;
    if (nl.stride < n || shell.stride != nl.stride)
        return set_error(LQ_ERR_ARG, "list renewal: strides %d / %d, targets %d", nl.stride, shell.stride, n);
    k_list_refresh<<<blocks_for(n, kBlock), kBlock, 0, s>>>(first, n, ph->np, cut * cut, pos, inner_count, shell.list,
                                                           shell.count, nl.list, nl.count, nl.stride, health);
    LQ_TRY_CUDA(cudaGetLastError(), "k_list_refresh");
    return LQ_OK;
}

int launch_neighbor_list_range(const Parameters* ph, const Parameters* pd, int first, int n, int layer_lo, float cut,
                               const float4* pos, const Cells& c, const NeighborList& nl, int* health,
                               cudaStream_t s, const float4* idep, const Frames& fr, const NeighborList* shell,
                               float inner, const int* gate)
{
    if (fr.rows && !idep) return set_error(LQ_ERR_ARG, "neighbour list: frames need the idep array");
    if (n <= 0) return LQ_OK;
    if (nl.stride < n) return set_error(LQ_ERR_ARG, "neighbour list stride %d < targets %d", nl.stride, n);
    if (shell && shell->stride != nl.stride)
        return set_error(LQ_ERR_ARG, "neighbour list: shell stride %d differs from %d", shell->stride, nl.stride);
    const float inner2 = inner > 0.0f ? inner * inner : 0.0f;
    if (shell)
        k_neighbor_list<true><<<blocks_for(n, kBlock), kBlock, 0, s>>>(pd, first, n, layer_lo, cut * cut, pos, c,
                                                                      nl.list, nl.count, nl.stride, health, idep, fr,
                                                                      shell->list, shell->count, inner2, gate);
    else
        k_neighbor_list<false><<<blocks_for(n, kBlock), kBlock, 0, s>>>(pd, first, n, layer_lo, cut * cut, pos, c,
                                                                       nl.list, nl.count, nl.stride, health, idep,
                                                                       fr, nullptr, nullptr, 0.0f, gate);
    LQ_TRY_CUDA(cudaGetLastError(), "k_neighbor_list");
    return LQ_OK;
}

int launch_pack_neighbors(const Parameters* ph, const State& st, float* rec, int first, cudaStream_t s,
                          bool packed_velocity, const int* map)
{
    const int n = ph->np - first;
    if (n <= 0) return LQ_OK;
    const NbrArrays nb = nbr_arrays(rec, ph->np);
    if (packed_velocity)
        k_pack_neighbors<true><<<blocks_for(n, kBlock), kBlock, 0, s>>>(first, ph->np, st, nb, map);
    else
        k_pack_neighbors<false><<<blocks_for(n, kBlock), kBlock, 0, s>>>(first, ph->np, st, nb, map);
    LQ_TRY_CUDA(cudaGetLastError(), "k_pack_neighbors");
    return LQ_OK;
}

int launch_adami_packed(const Parameters* ph, const Parameters* pd, const State& st, const NeighborList& nl,
                        float* rec, cudaStream_t s, tensor2d* str2, const int* act, const int* nact)
{
    if (ph->npb <= 0) return LQ_OK;
    if (!act != !nact) return set_error(LQ_ERR_ARG, "Adami: compacted targets need both act and nact");
    if (nl.stride < ph->npb) return set_error(LQ_ERR_ARG, "Adami: list stride %d < %d targets", nl.stride, ph->npb);
    const NbrArrays nb = nbr_arrays(rec, ph->np);
    const int grid = blocks_for(ph->npb, LQ_ADAMI_BLOCK);
    if (ph->npb >= kAdamiPairTargets)
        k_adami_packed<2><<<grid, LQ_ADAMI_BLOCK, 0, s>>>(pd, ph->npb, st, nl.list, nl.count, nl.stride, nb, str2, act,
                                                          nact);
    else
        k_adami_packed<4><<<grid, LQ_ADAMI_BLOCK, 0, s>>>(pd, ph->npb, st, nl.list, nl.count, nl.stride, nb, str2, act,
                                                          nact);
    LQ_TRY_CUDA(cudaGetLastError(), "k_adami_packed");
    return LQ_OK;
}

namespace {
/* A boundary list row that holds, or can gain by renewal, an entry. */
struct HasEntries {
    const int* a;
    const int* b;
    __device__ bool operator()(int i) const { return __ldg(a + i) > 0 || (b && __ldg(b + i) > 0); }
};
}   // namespace

size_t boundary_targets_temp_bytes(int npb)
{
    size_t bytes = 0;
    if (npb <= 0) return 0;
    cub::DeviceSelect::If(nullptr, bytes, thrust::counting_iterator<int>(0), (int*)nullptr, (int*)nullptr, npb,
                          HasEntries{nullptr, nullptr});
    return bytes;
}

int launch_boundary_targets(int npb, const int* count, const int* count2, int* act, int* nact, void* temp,
                            size_t temp_bytes, cudaStream_t s)
{
    if (npb <= 0) return LQ_OK;
    if (!count || !act || !nact || !temp)
        return set_error(LQ_ERR_ARG, "boundary targets: missing count, output or scratch");
    size_t bytes = temp_bytes;
    LQ_TRY_CUDA(cub::DeviceSelect::If(temp, bytes, thrust::counting_iterator<int>(0), act, nact, npb,
                                      HasEntries{count, count2}, s),
                "boundary targets (select)");
    return LQ_OK;
}

int launch_shepard_list(const Parameters* ph, const Parameters* pd, const State& st, tensor2d* out_str,
                        const NeighborList& nl, const Cells& c, cudaStream_t s, const Frames& fr, float* rec,
                        const int* order)
{
    if (ph->npm <= 0) return LQ_OK;
    if (!rec) return set_error(LQ_ERR_ARG, "Shepard filter: the packed neighbour records are required");
    k_shepard_list<<<blocks_for(ph->npm, kBlock), kBlock, 0, s>>>(pd, ph->np, ph->npb, st, out_str, nl.list,
                                                                 nl.count, nl.stride, c, fr, nbr_arrays(rec, ph->np),
                                                                 order);
    LQ_TRY_CUDA(cudaGetLastError(), "k_shepard_list");
    return LQ_OK;
}

int launch_interaction_list(const Parameters* ph, const Parameters* pd, const State& st, const Rates& r,
                            const Cells& c, const NeighborList& nl, cudaStream_t s, const Frames& fr,
                            bool compensated, float* rec, int shape, bool pack, const int* order,
                            const int* rows, const int* map)
{
    if (ph->npm <= 0) return LQ_OK;
    if (rec) {
        if (reinterpret_cast<uintptr_t>(rec) % 16 != 0)
            return set_error(LQ_ERR_ARG, "interaction: packed neighbour arrays must be 16-byte aligned");
        const NbrArrays nb = nbr_arrays(rec, ph->np);
        if (rows && (!map || !pack || shape == 5 || shape == 6))
            return set_error(LQ_ERR_ARG, "interaction: list rows need a record map, a pack and a thread-per-target "
                             "shape");
        if (pack) LQ_TRY(launch_pack_neighbors(ph, st, rec, 0, s, compensated, rows ? map : nullptr));
        if (shape >= 0 && shape < kPairShapeCount && kPairShapes[shape][2] == 1 && !order)
            return set_error(LQ_ERR_ARG, "interaction: launch shape %d needs the tile order", shape);
        if (shape < 0 || shape >= kPairShapeCount || kPairShapes[shape][2] != 1) order = nullptr;
#define LQ_PAIR_LAUNCH(T, B)                                                                                \
    (compensated ? k_interaction_rec<true, T, B><<<blocks_for(ph->npm, T), T, 0, s>>>(                      \
                       pd, ph->np, ph->npb, st, r, c, nl.list, nl.count, nl.stride, fr, nb, order, rows)       \
                 : k_interaction_rec<false, T, B><<<blocks_for(ph->npm, T), T, 0, s>>>(                     \
                       pd, ph->np, ph->npb, st, r, c, nl.list, nl.count, nl.stride, fr, nb, order, rows))
        switch (shape) {
            case 7: LQ_PAIR_LAUNCH(768, 1); break;
            case 8: LQ_PAIR_LAUNCH(384, 2); break;
            case 9: LQ_PAIR_LAUNCH(640, 1); break;
            case 10: LQ_PAIR_LAUNCH(320, 2); break;
            case 1: LQ_PAIR_LAUNCH(64, 12); break;
            case 2: LQ_PAIR_LAUNCH(256, 3); break;
            case 3: LQ_PAIR_LAUNCH(128, 5); break;
            case 4: LQ_PAIR_LAUNCH(128, 7); break;
            case 5:
            case 6: {
                const int G = shape == 5 ? 8 : 32;
                const int nthreads = ph->npm * G;
                const int grid = (nthreads + 127) / 128;
                if (G == 8) {
                    if (compensated)
                        k_interaction_group<true, 8><<<grid, 128, 0, s>>>(pd, ph->np, ph->npb, st, r, c, nl.list,
                                                                          nl.count, nl.stride, fr, nb);
                    else
                        k_interaction_group<false, 8><<<grid, 128, 0, s>>>(pd, ph->np, ph->npb, st, r, c, nl.list,
                                                                           nl.count, nl.stride, fr, nb);
                } else {
                    if (compensated)
                        k_interaction_group<true, 32><<<grid, 128, 0, s>>>(pd, ph->np, ph->npb, st, r, c, nl.list,
                                                                           nl.count, nl.stride, fr, nb);
                    else
                        k_interaction_group<false, 32><<<grid, 128, 0, s>>>(pd, ph->np, ph->npb, st, r, c, nl.list,
                                                                            nl.count, nl.stride, fr, nb);
                }
                break;
            }
            default: LQ_PAIR_LAUNCH(kBlock, LQ_PAIR_MIN_BLOCKS); break;
        }
#undef LQ_PAIR_LAUNCH
        LQ_TRY_CUDA(cudaGetLastError(), "k_interaction_rec");
        return LQ_OK;
    }
    return set_error(LQ_ERR_ARG, "interaction: the packed neighbour arrays are required");
}

int launch_adami(const Parameters* ph, const Parameters* pd, const State& st, const Cells& c, cudaStream_t s)
{
    if (ph->npb <= 0) return LQ_OK;
    k_adami<<<blocks_for(ph->npb, kBlock), kBlock, 0, s>>>(pd, ph->npb, st, c);
    LQ_TRY_CUDA(cudaGetLastError(), "k_adami");
    return LQ_OK;
}

int launch_shepard(const Parameters* ph, const Parameters* pd, const State& st, tensor2d* out_str, const State* full,
                   const Cells& c, cudaStream_t s)
{
    if (ph->npm <= 0) return LQ_OK;
    State f = full ? *full : State{nullptr, nullptr, nullptr, nullptr, nullptr};
    /* threads cover [0, np): boundary slots only copy (with `full`) */
    k_shepard<<<blocks_for(ph->np, kBlock), kBlock, 0, s>>>(pd, ph->np, ph->npb, st, out_str, f, full != nullptr, c);
    LQ_TRY_CUDA(cudaGetLastError(), "k_shepard");
    return LQ_OK;
}

}  // namespace lqb

/* ------------------------------------------------------------------ C ABI */

namespace {

bool bad_par(const void* ph, const void* pd) { return ph == nullptr || pd == nullptr; }

lqb::State state_of(const float* pos, const float* vel, const float* idep, const float* str, const float* stn)
{
    return lqb::State{(float4*)pos, (float4*)vel, (float4*)idep, (tensor2d*)str, (tensor2d*)stn};
}

}  // namespace

namespace {

/* Launch shape of the drop-in interaction's pair kernel (lqb::kPairShapes). */
constexpr int kDropInShape = 9;
/* Skin of the drop-in interaction's lists (of h) when the caller's grid
 * tracks particle identities: the lists then hold every pair within
 * 2h + skin and are carried across calls until some particle has moved
 * half the skin. */
constexpr float kDropInSkinOverH = 0.05f;

/* Working arrays of the drop-in interaction, one set per device: the cell
 * starts derived from the caller's cell_beg / cell_end, the pair kernel's
 * tile order with its scratch, the neighbour lists
 * and the packed neighbour data.  lq_interaction_reserve sizes them from a
 * Parameters record (the drop-in LoquatGrid's GridConfig calls it, where
 * the reference allocates its arrays); a call that needs more than was
 * reserved grows them itself, synchronising the device before the old
 * arrays are freed.  Calls that overlap on the GPU share the arrays and
 * must not. */
struct DropInWorkspace {
    int np = 0, ncell = 0, nseg = 0, npm = 0;
    int* start = nullptr;           /* ncell + 1 cell starts */
    int* counts = nullptr;          /* ncell + 1 particles per cell */
    void* scan_tmp = nullptr;       /* cell-start scan */
    size_t scan_bytes = 0;
    lqb::TileOrder to;              /* tile order and its segment scratch */
    lqb::NeighborList nl;           /* material targets' lists */
    float* rec = nullptr;           /* packed neighbour data, 13 floats per particle */
    /* lists carried across calls (caller grids that track identities) */
    float4* xbuild = nullptr;       /* np: positions at the build, by identity */
    int* build_of = nullptr;        /* np: identity -> slot at the build */
    int* rows = nullptr;            /* npm: target -> its list's row (the target's slot at the build) */
    int* pidx = nullptr;            /* np: slot -> its particle's slot at the build (its record's index) */
    int* moved = nullptr;           /* device flag: a particle moved half the skin since the build */
    int* tally = nullptr;           /* device counts of [0] builds and [1] reuses of carried lists */
    const int* key = nullptr;       /* the grid (its cell_beg) the carried lists belong to */
    long long gen = -1;
    int np_built = 0, npb_built = 0;
    bool built = false;
    long long rebuilds = 0, reuses = 0;   /* counts of earlier workspaces (tally holds this one's) */
    std::vector<void*> allocs;
};
std::mutex g_ws_mutex;
std::vector<DropInWorkspace> g_ws;

void free_workspace(DropInWorkspace& w)
{
    for (void* p : w.allocs) cudaFree(p);
    w = DropInWorkspace{};
}

int ws_alloc(DropInWorkspace& w, void** p, size_t bytes)
{
    cudaError_t e = cudaMalloc(p, bytes > 0 ? bytes : 16);
    if (e != cudaSuccess)
        return lqb::set_error(LQ_ERR_ALLOC, "interaction workspace: cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    w.allocs.push_back(*p);
    return LQ_OK;
}

/* Sizes every array for the Parameters' particle and cell counts. */
int size_workspace(DropInWorkspace& w, const Parameters* ph)
{
    const int np = ph->np > 1 ? ph->np : 1, ncell = ph->ncell, npm = ph->npm > 1 ? ph->npm : 1;
    int nseg = 0;
    size_t seg_scan = 0, cell_scan = 0;
    LQ_TRY(lqb::tile_order_scratch(ph, &nseg, &seg_scan));
    LQ_TRY(lqb::scan_scratch_bytes(ncell, &cell_scan));
    if (np <= w.np && ncell <= w.ncell && nseg <= w.nseg && npm <= w.npm && w.rec) return LQ_OK;
    if (!w.allocs.empty()) LQ_TRY_CUDA(cudaDeviceSynchronize(), "interaction workspace");
    long long rebuilds = w.rebuilds, reuses = w.reuses;
    if (w.tally) {
        int t[2] = {0, 0};
        LQ_TRY_CUDA(cudaMemcpy(t, w.tally, sizeof(t), cudaMemcpyDeviceToHost), "interaction workspace");
        rebuilds += t[0];
        reuses += t[1];
    }
    free_workspace(w);
    DropInWorkspace n;
    n.rebuilds = rebuilds;
    n.reuses = reuses;
    int st = LQ_OK;
    auto A = [&](void** p, size_t bytes) {
        if (st == LQ_OK) st = ws_alloc(n, p, bytes);
    };
    A((void**)&n.start, sizeof(int) * ((size_t)ncell + 1));
    A((void**)&n.counts, sizeof(int) * ((size_t)ncell + 1));
    A(&n.scan_tmp, cell_scan);
    n.scan_bytes = cell_scan;
    A((void**)&n.to.seg, sizeof(int) * 3 * (size_t)nseg);
    A(&n.to.scan_tmp, seg_scan);
    n.to.nseg_cap = nseg;
    n.to.scan_bytes = seg_scan;
    A((void**)&n.rec, sizeof(float) * 13 * (size_t)np);
    n.nl.stride = (npm + 31) / 32 * 32;
    A((void**)&n.nl.list, sizeof(int) * (size_t)LQ_NBR_CAP * n.nl.stride);
    A((void**)&n.nl.count, sizeof(int) * (size_t)n.nl.stride);
    A((void**)&n.to.order, sizeof(int) * (size_t)npm);
    A((void**)&n.xbuild, sizeof(float4) * (size_t)np);
    A((void**)&n.build_of, sizeof(int) * (size_t)np);
    A((void**)&n.rows, sizeof(int) * (size_t)npm);
    A((void**)&n.pidx, sizeof(int) * (size_t)np);
    A((void**)&n.moved, sizeof(int));
    A((void**)&n.tally, 2 * sizeof(int));
    if (st == LQ_OK) {
        const cudaError_t e = cudaMemset(n.tally, 0, 2 * sizeof(int));
        if (e != cudaSuccess) st = lqb::set_error(LQ_ERR_CUDA, "interaction workspace: %s", cudaGetErrorString(e));
    }
    if (st != LQ_OK) {
        free_workspace(n);
        return st;
    }
    n.np = np;
    n.ncell = ncell;
    n.nseg = nseg;
    n.npm = npm;
    w = std::move(n);
    return LQ_OK;
}

int dropin_workspace(const Parameters* ph, DropInWorkspace** out)
{
    int dev = 0;
    LQ_TRY_CUDA(cudaGetDevice(&dev), "interaction workspace");
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    if ((int)g_ws.size() <= dev) g_ws.resize((size_t)dev + 1);
    DropInWorkspace& w = g_ws[(size_t)dev];
    LQ_TRY(size_workspace(w, ph));
    *out = &w;
    return LQ_OK;
}

/* Carrying lists across calls.  The caller's grid gives each slot's
 * particle identity (lqb::identity_*).  A build keeps its lists as they are
 * (rows and entries are slots at the build) and records, by identity, each
 * particle's build slot and position.  Every call packs each particle's
 * neighbour record at its build slot, so the pair kernel gathers through
 * the stored entries as they are, each target reading the row of its build
 * slot; a later call whose particles have all moved less than half the
 * skin only maps slots to build slots (k_record_index).  The records stay
 * in the cell order of the build. */
__global__ void __launch_bounds__(256) k_moved_half_skin(int np, const float4* __restrict__ pos,
                                                         const int* __restrict__ ident,
                                                         const float4* __restrict__ xbuild, float half_skin2,
                                                         int* __restrict__ moved)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= np) return;
    const int id = __ldg(ident + c);
    bool far = true;
    if ((unsigned)id < (unsigned)np) {
        const float4 x = __ldg(pos + c), b = __ldg(xbuild + id);
        const float dx = x.x - b.x, dy = x.y - b.y, dz = x.z - b.z;
        far = !(dx * dx + dy * dy + dz * dz < half_skin2);
    }
    if (far) *moved = 1;
}

/* The call's decision, counted: a build when a particle moved (or nothing
 * was carried), else a reuse. */
__global__ void k_tally_decision(const int* __restrict__ moved, int* __restrict__ tally)
{
    tally[*moved ? 0 : 1] += 1;
}

/* Each slot's record index, the build slot of its particle (-1 when its
 * particle has none), and each material target's list row (its record
 * index less npb; -1: no carried list, the pair kernel walks its
 * stencil). */
__global__ void __launch_bounds__(256) k_record_index(int np, int npb, const int* __restrict__ ident,
                                                      const int* __restrict__ build_of, int* __restrict__ pidx,
                                                      int* __restrict__ rows)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= np) return;
    const int id = __ldg(ident + c);
    const int b = (unsigned)id < (unsigned)np ? __ldg(build_of + id) : -1;
    const int o = (unsigned)b < (unsigned)np ? b : -1;
    pidx[c] = o;
    if (c >= npb) rows[c - npb] = o >= npb ? o - npb : -1;
}

/* A build recorded for carrying (skipped unless *moved): each particle's
 * build slot and position, by identity. */
__global__ void __launch_bounds__(256) k_store_build(int np, const int* __restrict__ ident,
                                                     const float4* __restrict__ pos, float4* __restrict__ xbuild,
                                                     int* __restrict__ build_of, const int* __restrict__ moved)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= np || !*moved) return;
    const int id = __ldg(ident + c);
    if ((unsigned)id < (unsigned)np) {
        xbuild[id] = __ldg(pos + c);
        build_of[id] = c;
    }
}

/* Particles per cell from the reference's per-cell bounds (-1: empty). */
__global__ void __launch_bounds__(256) k_cell_counts(int ncell, const int* __restrict__ beg,
                                                     const int* __restrict__ end, int* __restrict__ counts)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > ncell) return;
    int n = 0;
    if (c < ncell) {
        const int b = __ldg(beg + c);
        n = b == -1 ? 0 : __ldg(end + c) - b;
    }
    counts[c] = n;
}

}  // namespace

extern "C" int lq_interaction_stats(long long* rebuilds, long long* reuses)
{
    if (!rebuilds || !reuses) return lqb::set_error(LQ_ERR_ARG, "lq_interaction_stats: null argument");
    int dev = 0;
    LQ_TRY_CUDA(cudaGetDevice(&dev), "interaction stats");
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    *rebuilds = 0;
    *reuses = 0;
    if (dev < (int)g_ws.size()) {
        const DropInWorkspace& w = g_ws[(size_t)dev];
        int t[2] = {0, 0};
        if (w.tally) {
            /* the decisions are counted on the device by the calls' streams */
            LQ_TRY_CUDA(cudaDeviceSynchronize(), "interaction stats");
            LQ_TRY_CUDA(cudaMemcpy(t, w.tally, sizeof(t), cudaMemcpyDeviceToHost), "interaction stats");
        }
        *rebuilds = w.rebuilds + t[0];
        *reuses = w.reuses + t[1];
    }
    return LQ_OK;
}

extern "C" int lq_interaction_reserve(const void* par_host)
{
    if (!par_host) return lqb::set_error(LQ_ERR_ARG, "lq_interaction_reserve: null Parameters");
    const Parameters* ph = static_cast<const Parameters*>(par_host);
    if (ph->np < 0 || ph->npm < 0 || ph->ncell < 1)
        return lqb::set_error(LQ_ERR_ARG, "lq_interaction_reserve: bad sizes np=%d npm=%d ncell=%d", ph->np, ph->npm,
                              ph->ncell);
    DropInWorkspace* w = nullptr;
    return dropin_workspace(ph, &w);
}

/* The reference's ParticleInteraction (src/particle_interaction.h:27-40).
 * The caller's grid (cell_beg / cell_end: every particle sorted into its
 * cell, cells in key order) gives the cell starts; the material targets
 * are ordered into compact tiles, their neighbours within 2h are found by
 * the 27-cell walk in the reference's visiting order into lists, and the
 * pair kernel sums over the lists from the packed neighbour data, in plain
 * FP32 as the reference computes. */
extern "C" int lq_particle_interaction(const void* par_host, const void* par_device, const float* pospres,
                                       const float* velrhop, const float* idep, const float* str, const float* stn,
                                       float* accad, float* spin, float* acestn, const int* cell_beg,
                                       const int* cell_end, void* stream)
{
    if (bad_par(par_host, par_device)) return lqb::set_error(LQ_ERR_ARG, "lq_particle_interaction: null Parameters");
    const Parameters* ph = static_cast<const Parameters*>(par_host);
    if (ph->npm > 0 && (!pospres || !velrhop || !str || !accad || !spin || !acestn || !cell_beg || !cell_end))
        return lqb::set_error(LQ_ERR_ARG, "lq_particle_interaction: null array");
    if (ph->npm <= 0) return LQ_OK;
    lqb::Rates r{(float4*)accad, (float4*)spin, (tensor2d*)acestn};
    const Parameters* pd = static_cast<const Parameters*>(par_device);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const lqb::State st = state_of(pospres, velrhop, idep, str, stn);
    DropInWorkspace* w = nullptr;
    LQ_TRY(dropin_workspace(ph, &w));
    const int ncell = ph->ncell;
    k_cell_counts<<<(ncell + 256) / 256, 256, 0, s>>>(ncell, cell_beg, cell_end, w->counts);
    LQ_TRY_CUDA(cudaGetLastError(), "k_cell_counts");
    size_t bytes = w->scan_bytes;
    LQ_TRY_CUDA(cub::DeviceScan::ExclusiveSum(w->scan_tmp, bytes, w->counts, w->start, ncell + 1, s),
                "cell start scan");
    const lqb::Cells c{w->start, nullptr, nullptr};
    const int np = ph->np, npb = ph->npb, npm = ph->npm;
    const int nb256 = (np + 255) / 256;
    lqb::GridIdentity gi;
    if (lqb::identity_find(cell_beg, &gi) && gi.np == np) {
        /* the caller's grid tracks its particles: carry the lists while
         * every particle stays within half the skin of its build position.
         * The device decides (no host synchronisation): both paths are
         * enqueued and the one not taken returns at once. */
        const float skin = kDropInSkinOverH * ph->h;
        const bool carried =
            w->built && w->key == cell_beg && w->gen == gi.gen && w->np_built == np && w->npb_built == npb;
        if (carried) {
            LQ_TRY_CUDA(cudaMemsetAsync(w->moved, 0, sizeof(int), s), "moved flag");
            k_moved_half_skin<<<nb256, 256, 0, s>>>(np, st.pos, gi.ident, w->xbuild, 0.25f * skin * skin, w->moved);
            LQ_TRY_CUDA(cudaGetLastError(), "k_moved_half_skin");
        } else {
            LQ_TRY(lqb::fill_int(w->moved, 1, 1, s));
        }
        k_tally_decision<<<1, 1, 0, s>>>(w->moved, w->tally);
        LQ_TRY_CUDA(cudaGetLastError(), "k_tally_decision");
        /* a build (skipped unless moved): fresh lists in the current
         * slots, kept with each particle's build slot and position */
        LQ_TRY(lqb::launch_neighbor_list_range(ph, pd, npb, npm, 0, 2.0f * ph->h + skin, st.pos, c, w->nl, nullptr,
                                               s, nullptr, lqb::Frames(), nullptr, 0.0f, w->moved));
        k_store_build<<<nb256, 256, 0, s>>>(np, gi.ident, st.pos, w->xbuild, w->build_of, w->moved);
        LQ_TRY_CUDA(cudaGetLastError(), "k_store_build");
        w->built = true;
        w->key = cell_beg;
        w->gen = gi.gen;
        w->np_built = np;
        w->npb_built = npb;
        /* either way the pair kernel reads the lists of the last build,
         * each target at the row of its build slot, with the records
         * packed at the build slots: a reuse maps only slots */
        k_record_index<<<nb256, 256, 0, s>>>(np, npb, gi.ident, w->build_of, w->pidx, w->rows);
        LQ_TRY_CUDA(cudaGetLastError(), "k_record_index");
        LQ_TRY(lqb::launch_tile_order(ph, w->start, kDropInShape, w->to, s));
        return lqb::launch_interaction_list(ph, pd, st, r, c, w->nl, s, lqb::Frames(), false, w->rec, kDropInShape,
                                            true, w->to.order, w->rows, w->pidx);
    }
    /* a grid of the caller's own: lists built in its slots at every call,
     * with the pair body's own cut-off test (q < 2 with the candidate
     * slack of the cell walk) */
    const float cut = 2.0f * ph->h * sqrtf(1.0001f);
    LQ_TRY(lqb::launch_neighbor_list_range(ph, pd, npb, npm, 0, cut, st.pos, c, w->nl, nullptr, s));
    w->built = false;
    LQ_TRY(lqb::launch_tile_order(ph, w->start, kDropInShape, w->to, s));
    return lqb::launch_interaction_list(ph, pd, st, r, c, w->nl, s, lqb::Frames(), false, w->rec, kDropInShape, true,
                                        w->to.order);
}

extern "C" int lq_adami_boundary(const void* par_host, const void* par_device, const float* pospres,
                                 const float* velrhop, float* str, const int* cell_beg, const int* cell_end,
                                 void* stream)
{
    if (bad_par(par_host, par_device)) return lqb::set_error(LQ_ERR_ARG, "lq_adami_boundary: null Parameters");
    const Parameters* ph = static_cast<const Parameters*>(par_host);
    if (ph->npb > 0 && (!pospres || !velrhop || !str || !cell_beg || !cell_end))
        return lqb::set_error(LQ_ERR_ARG, "lq_adami_boundary: null array");
    lqb::Cells c{nullptr, cell_beg, cell_end};
    return lqb::launch_adami(ph, static_cast<const Parameters*>(par_device),
                             state_of(pospres, velrhop, nullptr, str, nullptr), c, static_cast<cudaStream_t>(stream));
}

extern "C" int lq_stress_regularization(const void* par_host, const void* par_device, const float* pospres,
                                        const float* velrhop, float* str, float* tensor2d_cache, const int* cell_beg,
                                        const int* cell_end, void* stream)
{
    if (bad_par(par_host, par_device))
        return lqb::set_error(LQ_ERR_ARG, "lq_stress_regularization: null Parameters");
    const Parameters* ph = static_cast<const Parameters*>(par_host);
    if (ph->npm <= 0) return LQ_OK;
    if (!pospres || !velrhop || !str || !tensor2d_cache || !cell_beg || !cell_end)
        return lqb::set_error(LQ_ERR_ARG, "lq_stress_regularization: null array");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    lqb::Cells c{nullptr, cell_beg, cell_end};
    LQ_TRY(lqb::launch_shepard(ph, static_cast<const Parameters*>(par_device),
                               state_of(pospres, velrhop, nullptr, str, nullptr), (tensor2d*)tensor2d_cache, nullptr,
                               c, s));
    /* copy the filtered material stress back (reference src/field_smoothing.cu:144) */
    LQ_TRY_CUDA(cudaMemcpyAsync((tensor2d*)str + ph->npb, (tensor2d*)tensor2d_cache + ph->npb,
                                sizeof(tensor2d) * (size_t)ph->npm, cudaMemcpyDeviceToDevice, s),
                "Shepard copy back");
    return LQ_OK;
}

/* ------------------------------------------- C++ drop-in functions */

namespace {

void check_or_die(int st, const char* what)
{
    if (st != LQ_OK) {
        fprintf(stderr, "%s failed: %s\n", what, lq_last_error());
        exit(EXIT_FAILURE);
    }
}

}  // namespace

void ParticleInteraction(Parameters* par_host, Parameters* par_device, float4* pospres, float4* velrhop,
                         float4* idep, tensor2d* str, tensor2d* stn, float4* accad, float4* spin, tensor2d* acestn,
                         const int* cell_beg, const int* cell_end)
{
    check_or_die(lq_particle_interaction(par_host, par_device, (const float*)pospres, (const float*)velrhop,
                                         (const float*)idep, (const float*)str, (const float*)stn, (float*)accad,
                                         (float*)spin, (float*)acestn, cell_beg, cell_end, nullptr),
                 "ParticleInteraction");
}

void AdamiBoundary(Parameters* par_host, Parameters* par_device, float4* pospres, float4* velrhop, tensor2d* str,
                   const int* cell_beg, const int* cell_end)
{
    check_or_die(lq_adami_boundary(par_host, par_device, (const float*)pospres, (const float*)velrhop, (float*)str,
                                   cell_beg, cell_end, nullptr),
                 "AdamiBoundary");
}

void StressRegularization(Parameters* par_host, Parameters* par_device, float4* pospres, float4* velrhop,
                          tensor2d* str, tensor2d* tensor2d_cache, const int* cell_beg, const int* cell_end)
{
    check_or_die(lq_stress_regularization(par_host, par_device, (const float*)pospres, (const float*)velrhop,
                                          (float*)str, (float*)tensor2d_cache, cell_beg, cell_end, nullptr),
                 "StressRegularization");
}

extern "C" int lq_debug_bounds_violations(long long* count)
{
    if (!count) return lqb::set_error(LQ_ERR_ARG, "lq_debug_bounds_violations: null argument");
#ifdef LQ_CHECKED
    LQ_TRY_CUDA(cudaDeviceSynchronize(), "bounds counter");
    unsigned long long a = 0, b = 0;
    LQ_TRY(lqb::bounds_count_sph(&a));
    LQ_TRY(lqb::bounds_count_grid(&b));
    *count = (long long)(a + b);
#else
    *count = -1;
#endif
    return LQ_OK;
}
