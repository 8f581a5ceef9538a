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
#include <cstdio>
#include <cstdlib>

#include "lq_internal.cuh"
#include "lq_device.cuh"
#include <adami_boundary.h>
#include <field_smoothing.h>
#include <particle_interaction.h>

namespace lqb {

namespace {

constexpr int kInteractionBlock = 128;
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
 * Work layout.  One thread per material particle, 32 consecutive sorted
 * particles per warp.  A warp's particles mostly share one grid column
 * (X, Y); lanes are grouped by column and each group walks the union of its
 * lanes' stencils in lockstep: the candidate loop is warp-uniform, every
 * candidate position is one broadcast load, and each lane only runs the
 * cheap distance test.  Hits are appended to a per-lane list in shared
 * memory; when any lane's list is full (and at the end) the warp flushes,
 * each lane evaluating its own pairs, so the ~80-flop pair body runs with
 * most lanes busy instead of once per candidate at ~15% lane use.  A lane
 * meets its neighbours in the same order as a per-thread 27-cell walk, so
 * the sums are bit-identical to that.
 * Per pair: 3 loads (pos 16 B, vel 16 B, stress 24 B), about 80 flops. */
constexpr int kIntWarps = kInteractionBlock / 32;
constexpr int kHitCap = 64;

__global__ void __launch_bounds__(kInteractionBlock) k_interaction(const Parameters* __restrict__ P, int np, int npb,
                                                                   State st, Rates rt, Cells cells)
{
    __shared__ int hits[kIntWarps][kHitCap][32];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int i = npb + blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < np;

    const float ih = __ldg(&P->i_h), h = __ldg(&P->h), eta = __ldg(&P->eta), m = __ldg(&P->m);
    const float Cg = __ldg(&P->kernel_gradient_normalization_par);
    const float Cw = __ldg(&P->kernel_normalization_par);
    const bool visc = __ldg(&P->viscosity_type) == 1;
    const float avc = __ldg(&P->artificial_viscosity_alpha) * __ldg(&P->cs); /* alpha * cs */
    const bool artp = __ldg(&P->artificial_pressure) == 1;
    const float eps = __ldg(&P->artificial_pressure_coefficient);
    const float wdr = __ldg(&P->kernel_dr);
    const int nx = __ldg(&P->cell_num_x), ny = __ldg(&P->cell_num_y), nz = __ldg(&P->cell_num_z);
    const int L = __ldg(&P->ncell_one_layer);
    const float cut2 = 4.0f * h * h * 1.0001f; /* prefilter; exact test is q < 2 */

    float4 xi = make_float4(0.f, 0.f, 0.f, 0.f), vi = make_float4(0.f, 0.f, 0.f, 1.f);
    tensor2d si = make_tensor2d(0.0f);
    if (active) {
        xi = __ldg(st.pos + i);
        vi = __ldg(st.vel + i);
        si = load_t2(st.str, i);
    }
    const float rhoi = vi.w;
    const float ri2 = 1.0f / (rhoi * rhoi);
    const float Sxx = si.xx * ri2, Syy = si.yy * ri2, Szz = si.zz * ri2;
    const float Sxy = si.xy * ri2, Sxz = si.xz * ri2, Syz = si.yz * ri2;
    float Rix = 0.f, Riy = 0.f, Riz = 0.f;
    if (artp) {
        Rix = si.xx > 0.f ? -eps * Sxx : 0.f;
        Riy = si.yy > 0.f ? -eps * Syy : 0.f;
        Riz = si.zz > 0.f ? -eps * Szz : 0.f;
    }

    float drho = 0.f, ax = 0.f, ay = 0.f, az = 0.f;
    float l00 = 0.f, l01 = 0.f, l02 = 0.f, l10 = 0.f, l11 = 0.f, l12 = 0.f, l20 = 0.f, l21 = 0.f, l22 = 0.f;

    auto pair = [&](int j) {
        const float4 xj = __ldg(st.pos + j);
        const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        const float r2 = dx * dx + dy * dy + dz * dz;
        const float q = sqrtf(r2) * ih;
        if (!(q < 2.0f)) return;
        const float4 vj = __ldg(st.vel + j);
        const tensor2d sj = load_t2(st.str, j);
        const float t = 2.0f - q;
        const float fac = Cg * t * t * t;
        const float gx = fac * dx, gy = fac * dy, gz = fac * dz;
        const float vx = vi.x - vj.x, vy = vi.y - vj.y, vz = vi.z - vj.z;
        drho += vx * gx + vy * gy + vz * gz;
        const float rinv = __frcp_rn(vj.w);
        const float rj2 = rinv * rinv;
        const float Txx = Sxx + sj.xx * rj2, Tyy = Syy + sj.yy * rj2, Tzz = Szz + sj.zz * rj2;
        const float Txy = Sxy + sj.xy * rj2, Txz = Sxz + sj.xz * rj2, Tyz = Syz + sj.yz * rj2;
        ax += Txx * gx + Txy * gy + Txz * gz;
        ay += Txy * gx + Tyy * gy + Tyz * gz;
        az += Txz * gx + Tyz * gy + Tzz * gz;
        if (visc) {
            const float vr = vx * dx + vy * dy + vz * dz;
            if (vr < 0.f) {
                const float mu = h * vr / (r2 + eta);
                const float pi = -avc * mu / (0.5f * (rhoi + vj.w));
                ax -= pi * gx;
                ay -= pi * gy;
                az -= pi * gz;
            }
        }
        if (artp) {
            const float wk = Cw * t * t * t * t * (q + 0.5f);
            const float f = wk / wdr;
            const float f4 = (f * f) * (f * f);
            const float Rjx = sj.xx > 0.f ? -eps * sj.xx * rj2 : 0.f;
            const float Rjy = sj.yy > 0.f ? -eps * sj.yy * rj2 : 0.f;
            const float Rjz = sj.zz > 0.f ? -eps * sj.zz * rj2 : 0.f;
            ax += (Rix + Rjx) * f4 * gx;
            ay += (Riy + Rjy) * f4 * gy;
            az += (Riz + Rjz) * f4 * gz;
        }
        const float Vj = m * rinv;
        const float wx = Vj * vx, wy = Vj * vy, wz = Vj * vz;
        l00 -= wx * gx; l01 -= wx * gy; l02 -= wx * gz;
        l10 -= wy * gx; l11 -= wy * gy; l12 -= wy * gz;
        l20 -= wz * gx; l21 -= wz * gy; l22 -= wz * gz;
    };

    int count = 0;
    auto flush = [&]() {
        const int maxc = (int)__reduce_max_sync(FULL, (unsigned)count);
        for (int k = 0; k < maxc; ++k)
            if (k < count) pair(hits[w][k][lane]);
        count = 0;
        __syncwarp();
    };

    int cx = 0, cy = 0, cz = 0;
    if (active) {
        cx = stencil_axis(xi.x, ih);
        cy = stencil_axis(xi.y, ih);
        cz = stencil_axis(xi.z, ih);
    }
    unsigned todo = __ballot_sync(FULL, active);
    while (todo) {
        const int leader = __ffs(todo) - 1;
        const int gx = __shfl_sync(FULL, cx, leader), gy = __shfl_sync(FULL, cy, leader);
        const bool mine = active && cx == gx && cy == gy;
        todo &= ~__ballot_sync(FULL, mine);
        const int zmin = __reduce_min_sync(FULL, mine ? cz : INT_MAX);
        const int zmax = __reduce_max_sync(FULL, mine ? cz : INT_MIN);
        const int zlo = max(zmin - 1, 0), zhi = min(zmax + 1, nz - 1);
        if (zlo > zhi) continue;
        for (int layer = 0; layer < 2; ++layer) {
            const int off = layer ? L : 0;
            for (int col = 0; col < 9; ++col) {
                const int X = gx + (col % 3) - 1, Y = gy + (col / 3) - 1;
                if (X < 0 || X >= nx || Y < 0 || Y >= ny) continue;
                int s, e;
                if (!zrun_range(cells, off + (X * ny + Y) * nz, zlo, zhi, s, e)) continue;
                for (int j = s; j < e; ++j) {
                    const float4 xj = __ldg(st.pos + j);
                    if (mine) {
                        const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
                        const float r2 = dx * dx + dy * dy + dz * dz;
                        if (r2 < cut2 && j != i) {
                            hits[w][count][lane] = j;
                            ++count;
                        }
                    }
                    if (__any_sync(FULL, count == kHitCap)) flush();
                }
            }
        }
    }
    flush();
    if (!active) return;
    rt.accad[i] = make_float4(m * ax + __ldg(&P->acc_x), m * ay + __ldg(&P->acc_y), m * az + __ldg(&P->acc_z),
                              m * drho);
    rt.spin[i] = make_float4(0.5f * (l10 - l01), 0.5f * (l20 - l02), 0.5f * (l21 - l12), 0.0f);
    store_t2(rt.acestn, i,
             make_tensor2d(l00, l11, l22, 0.5f * (l01 + l10), 0.5f * (l02 + l20), 0.5f * (l12 + l21)));
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

}  // namespace

int launch_interaction(const Parameters* ph, const Parameters* pd, const State& st, const Rates& r, const Cells& c,
                       cudaStream_t s)
{
    if (ph->npm <= 0) return LQ_OK;
    k_interaction<<<blocks_for(ph->npm, kInteractionBlock), kInteractionBlock, 0, s>>>(pd, ph->np, ph->npb, st, r,
                                                                                      c);
    LQ_TRY_CUDA(cudaGetLastError(), "k_interaction");
    return LQ_OK;
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

extern "C" int lq_particle_interaction(const void* par_host, const void* par_device, const float* pospres,
                                       const float* velrhop, const float* idep, const float* str, const float* stn,
                                       float* accad, float* spin, float* acestn, const int* cell_beg,
                                       const int* cell_end, void* stream)
{
    if (bad_par(par_host, par_device)) return lqb::set_error(LQ_ERR_ARG, "lq_particle_interaction: null Parameters");
    const Parameters* ph = static_cast<const Parameters*>(par_host);
    if (ph->npm > 0 && (!pospres || !velrhop || !str || !accad || !spin || !acestn || !cell_beg || !cell_end))
        return lqb::set_error(LQ_ERR_ARG, "lq_particle_interaction: null array");
    lqb::Cells c{nullptr, cell_beg, cell_end};
    lqb::Rates r{(float4*)accad, (float4*)spin, (tensor2d*)acestn};
    return lqb::launch_interaction(ph, static_cast<const Parameters*>(par_device),
                                   state_of(pospres, velrhop, idep, str, stn), r, c,
                                   static_cast<cudaStream_t>(stream));
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
