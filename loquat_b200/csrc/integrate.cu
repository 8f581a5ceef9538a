/*
 * LOQUAT-B200 predictor-corrector integrator with the Drucker-Prager and
 * hypoplastic stress updates (reference src/predictor_corrector.cu:169-336),
 * its C ABI entry points and the C++ drop-in functions.
 *
 * The reference issues five device-to-device snapshot copies and then the
 * predictor kernel; here the snapshot is written by the same kernel that
 * reads the state, so the state is read once.  The native driver skips the
 * snapshot entirely: the predictor writes into a second buffer and the
 * corrector reads the untouched first buffer through the new sort
 * permutation.
 */
#include <cstdio>
#include <cstdlib>

#include "lq_internal.cuh"
#include "lq_device.cuh"
#include <predictor_corrector.h>

namespace lqb {

namespace {

constexpr int kBlock = 128;
/* resident blocks per SM asked of the model-3 instantiations: 4 caps them at
 * 128 registers (a few spilled bytes), measured faster than 1 (168 registers)
 * and 6 (80) on the 2.85 M-particle slope */
#ifndef LQ_VW_MIN_BLOCKS
#define LQ_VW_MIN_BLOCKS 4
#endif
/* resident blocks per SM asked of the other instantiations: 6 caps them at
 * 80 registers (the mixed form's FP64 return map spills ~130 B), 24 warps
 * per SM instead of 16 for the uncapped 117-120; on the 256-scenario
 * ensemble the mixed integrators took 2.19 ms per step against 2.25 (5),
 * 2.22 (7), 2.36 (8) and 2.49 uncapped; the plain ones (78 registers) are
 * unaffected */
#ifndef LQ_INT_MIN_BLOCKS
#define LQ_INT_MIN_BLOCKS 6
#endif

inline int blocks_for(long long n, int b) { return (int)((n + b - 1) / b); }

/* FP64 position (pressure p in the float word's w) and velocity into the
 * float high words x, v and, with `lo`, the low words of `out` at slot i. */
__device__ __forceinline__ void split_words(const State& out, int i, const double4& xd, const double4& vd, float p,
                                            float4& x, float4& v, bool lo = true)
{
    float4 xl, vl;
    split4(make_double4(xd.x, xd.y, xd.z, 0.0), x, xl);
    split4(vd, v, vl);
    x.w = p;
    if (lo) {
        out.xlo[i] = xl;
        out.vlo[i] = vl;
    }
}

/* The same, storing the high words too. */
__device__ __forceinline__ void store_split(const State& out, int i, const double4& xd, const double4& vd, float p,
                                            bool lo = true)
{
    float4 x, v;
    split_words(out, i, xd, vd, p, x, v, lo);
    out.pos[i] = x;
    out.vel[i] = v;
}

/* A material slot's entry of the pair kernel's packed neighbour arrays from
 * the position, velocity and stress just stored (what k_pack_neighbors
 * would write from them), when nb is set: the native driver's integrators
 * pack the slots they update, so a stage needs no pack of its own.  kPk
 * (the mixed form) packs the velocity into two words. */
template <bool kPk>
__device__ __forceinline__ void pack_slot(const NbrArrays& nb, int i, const float4& x, const float4& v,
                                          const tensor2d& s)
{
    if (!nb.xr) return;
    nb.xr[i] = make_float4(x.x, x.y, x.z, v.w);
    store_packed<kPk>(nb, i, v, s);
}

/* Half step of the material slots (reference src/predictor_corrector.cu:169-218):
 * v += dt/2 a; rho += dt/2 drho; x += dt/2 v_new; eps += dt/2 deps;
 * stress and plastic strain from the model at dt/2.  With `stage` the
 * output is a stage buffer that only the neighbour kernels and the
 * corrector read: the position and velocity high words (with the
 * pressure), the object word and the stress; the corrector restarts the
 * strain, the plastic strain and the FP64 kinematics from its snapshot, so
 * the strain (neither read nor written), the low words and, for the
 * hypoplastic model, the plastic strain are left out. */
template <bool kMixed, bool kVW>
__global__ void __launch_bounds__(kBlock, kVW ? LQ_VW_MIN_BLOCKS : LQ_INT_MIN_BLOCKS) k_predict(const Parameters* __restrict__ P, int np, int npb, State in,
                                                    State out, State snap, bool do_snap, Rates rt, MaterialTable mt,
                                                    MaterialTable vw, NbrArrays nb, bool stage)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    /* boundary slots change only by Adami, which writes both state buffers
     * of the native driver; without a snapshot there is nothing to do */
    if (i < npb && !do_snap) return;
    const float4 x0 = in.pos[i];
    const float4 v0 = in.vel[i];
    const float4 id = in.idep[i];
    const tensor2d s0 = load_t2_rw(in.str, i);
    const tensor2d e0 = stage ? make_tensor2d(0.0f) : load_t2_rw(in.stn, i);
    if (do_snap) {
        snap.pos[i] = x0;
        snap.vel[i] = v0;
        snap.idep[i] = id;
        store_t2(snap.str, i, s0);
        store_t2(snap.stn, i, e0);
    }
    if (i < npb) {
        /* a boundary slot of another output buffer takes the stress (the
         * Adami extrapolation); the rest never changes */
        if (out.pos != in.pos) store_t2(out.str, i, s0);
        return;
    }
    const float dt = __ldg(&P->dt);
    const Material M = particle_material(load_material(P), mt, id.x);
    const float4 a = __ldg(rt.accad + i);
    const float4 w = __ldg(rt.spin + i);
    const tensor2d de = load_t2(rt.acestn, i);

    if (kMixed) {
        /* FP64 accumulation of velocity, density and position; FP64 stress update */
        const double hdt = 0.5 * (double)dt;
        double4 vd = join4(v0, in.vlo[i]), xd = join4(x0, in.xlo[i]);
        vd.x += hdt * a.x; vd.y += hdt * a.y; vd.z += hdt * a.z; vd.w += hdt * a.w;
        xd.x += hdt * vd.x; xd.y += hdt * vd.y; xd.z += hdt * vd.z;
        T6d e = widen6(e0), dd = widen6(de);
        e.xx += dd.xx * hdt; e.yy += dd.yy * hdt; e.zz += dd.zz * hdt;
        e.xy += dd.xy * hdt; e.xz += dd.xz * hdt; e.yz += dd.yz * hdt;
        double p = x0.w, ep = id.y, ev = id.z;
        T6d sd = widen6(s0);
        if (kVW) {
            /* the kinematics are stored before the sub-stepping, whose FP64
             * registers then need not share the SM with them */
            store_split(out, i, xd, vd, x0.w, !stage);
            if (!stage) store_t2(out.stn, i, narrow6(e));
            const float epf = stage ? id.y : (float)sqrt(2.0 / 3.0 * contract6(e, e));
            vw_update_d(vw_const(vw, id.x), hdt, de, w, sd, ev);
            out.idep[i] = make_float4(id.x, epf, (float)ev, id.w);
            const tensor2d sn = narrow6(sd);
            store_t2(out.str, i, sn);
            pack_slot<kMixed>(nb, i, out.pos[i], out.vel[i], sn);   /* kinematics stored above */
            return;
        }
        if (M.model == 1) {
            dp_update_d(M, hdt, w, dd, p, ep, sd);
        } else {
            hypo_update_d(M, hdt, dd, w, sd);
            if (!stage) ep = sqrt(2.0 / 3.0 * contract6(e, e));
        }
        float4 xh, vh;
        split_words(out, i, xd, vd, (float)p, xh, vh, !stage);
        out.pos[i] = xh;
        out.vel[i] = vh;
        out.idep[i] = make_float4(id.x, (float)ep, (float)ev, id.w);
        const tensor2d sn = narrow6(sd);
        store_t2(out.str, i, sn);
        if (!stage) store_t2(out.stn, i, narrow6(e));
        pack_slot<kMixed>(nb, i, xh, vh, sn);
        return;
    }
    float4 v = v0;
    v.x += 0.5f * dt * a.x;
    v.y += 0.5f * dt * a.y;
    v.z += 0.5f * dt * a.z;
    v.w += 0.5f * dt * a.w;
    float4 x = x0;
    x.x += 0.5f * dt * v.x;
    x.y += 0.5f * dt * v.y;
    x.z += 0.5f * dt * v.z;
    const tensor2d e = e0 + de * (0.5f * dt);

    float p = x0.w;
    float ep = id.y, ev = id.z;
    tensor2d s = s0;
    if (kVW) {
        /* the adaptive sub-stepping runs in FP64 in both forms; the
         * kinematics are stored first */
        out.pos[i] = x;
        out.vel[i] = v;
        if (!stage) store_t2(out.stn, i, e);
        const float epf = stage ? id.y : sqrtf(2.0f / 3.0f * J2(e));
        T6d sd = widen6(s0);
        double evd = ev;
        vw_update_d(vw_const(vw, id.x), 0.5 * (double)dt, de, w, sd, evd);
        out.idep[i] = make_float4(id.x, epf, (float)evd, id.w);
        const tensor2d sn = narrow6(sd);
        store_t2(out.str, i, sn);
        pack_slot<kMixed>(nb, i, out.pos[i], out.vel[i], sn);   /* kinematics stored above */
        return;
    }
    if (M.model == 1) {
        dp_update(M, 0.5f * dt, w, de, p, ep, s);
    } else {
        hypo_update(M, 0.5f * dt, de, w, s);
        if (!stage) ep = sqrtf(2.0f / 3.0f * J2(e));
    }
    x.w = p;
    out.pos[i] = x;
    out.vel[i] = v;
    out.idep[i] = make_float4(id.x, ep, ev, id.w);
    store_t2(out.str, i, s);
    if (!stage) store_t2(out.stn, i, e);
    pack_slot<kMixed>(nb, i, x, v, s);
}

/* Full step from the snapshot (reference src/predictor_corrector.cu:256-307):
 * v = v0 + dt a; x = x0 + dt/2 (v + v0); eps = eps0 + dt deps; the model
 * restarts from the snapshot stress and plastic strain; the pressure passed
 * in is the current one.  Reads the current state `cur` and the snapshot
 * `ini` (at ini_idx[i], or i), writes `out` (which may be `cur` or `ini`).
 * When out differs from cur, boundary slots are copied from cur (their
 * stress is the latest Adami extrapolation).  With `verlet`, each material
 * particle also checks whether neighbour lists built at positions xbuild
 * stay valid through the next step: it raises *rebuild when twice its
 * displacement plus a bound on its next step's motion reaches the skin. */
struct VerletCheck {
    const float4* xbuild;
    int* rebuild;
    float half_skin;
    float dt_bound;   /* the largest step the next one can take */
    const float4* xwide;   /* two-level lists: positions at the wide build */
    float half_margin;     /* (wide - skin) / 2 */
};

/* The list checks of one material particle at its new position x. */
__device__ __forceinline__ void verlet_check(const VerletCheck& vc, int i, const float4& x, const float4& v,
                                             const float4& a)
{
    const float4 xb = __ldg(vc.xbuild + i);
    const float dx = x.x - xb.x, dy = x.y - xb.y, dz = x.z - xb.z;
    const float moved = sqrtf(dx * dx + dy * dy + dz * dz);
    const float speed = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    const float accel = sqrtf(a.x * a.x + a.y * a.y + a.z * a.z);
    /* next step: the predictor half step and the corrector full step
     * move a particle by at most dt |v| + dt^2 |a| each; 2x covers both */
    const float dtb = vc.dt_bound;
    const float ahead = 2.0f * dtb * (speed + dtb * accel);
    if (!(moved + ahead < vc.half_skin)) atomicOr(vc.rebuild, 1);
    if (vc.xwide) {
        /* lists renewed at x from the wide ones hold every pair within
         * 2h + skin while no particle is (wide - skin) / 2 from xwide */
        const float4 xw = __ldg(vc.xwide + i);
        const float ex = x.x - xw.x, ey = x.y - xw.y, ez = x.z - xw.z;
        if (!(sqrtf(ex * ex + ey * ey + ez * ez) < vc.half_margin)) atomicOr(vc.rebuild, 2);
    }
}

template <bool kMixed, bool kVW>
__global__ void __launch_bounds__(kBlock, kVW ? LQ_VW_MIN_BLOCKS : LQ_INT_MIN_BLOCKS) k_correct(const Parameters* __restrict__ P, int np, int npb, State cur,
                                                    State ini, const int* __restrict__ ini_idx, State out, Rates rt,
                                                    int* __restrict__ health, VerletCheck verlet, int first,
                                                    MaterialTable mt, MaterialTable vw, NbrArrays nb)
{
    const int i = first + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    if (i < npb) return;    /* boundary slots: Adami writes both buffers */
    const int k = ini_idx ? __ldg(ini_idx + i) : i;
    const float dt = __ldg(&P->dt);
    const float4 a = __ldg(rt.accad + i);
    const float4 w = __ldg(rt.spin + i);
    const tensor2d de = load_t2(rt.acestn, i);
    const float4 x0 = ini.pos[k];
    const float4 v0 = ini.vel[k];
    const float4 id0 = ini.idep[k];
    const float ep0 = id0.y;
    const tensor2d s0 = load_t2_rw(ini.str, k);
    const tensor2d e0 = load_t2_rw(ini.stn, k);
    const float4 xc = cur.pos[i];
    const float4 id = cur.idep[i];
    const Material M = particle_material(load_material(P), mt, id.x);

    if (kVW) {
        /* model 3: the kinematics, the health of the kinematics and the
         * Verlet check come before the FP64 sub-stepping, so that its
         * registers need not share the SM with them */
        float4 v, x;
        tensor2d e;
        float ep;
        if (kMixed) {
            const double ddt = dt;
            const double4 v0d = join4(v0, ini.vlo[k]), x0d = join4(x0, ini.xlo[k]);
            double4 vd, xd;
            vd.x = v0d.x + ddt * a.x; vd.y = v0d.y + ddt * a.y; vd.z = v0d.z + ddt * a.z; vd.w = v0d.w + ddt * a.w;
            xd.x = 0.5 * (vd.x + v0d.x) * ddt + x0d.x;
            xd.y = 0.5 * (vd.y + v0d.y) * ddt + x0d.y;
            xd.z = 0.5 * (vd.z + v0d.z) * ddt + x0d.z;
            xd.w = 0.0;
            T6d ed = widen6(e0);
            const T6d dd = widen6(de);
            ed.xx += dd.xx * ddt; ed.yy += dd.yy * ddt; ed.zz += dd.zz * ddt;
            ed.xy += dd.xy * ddt; ed.xz += dd.xz * ddt; ed.yz += dd.yz * ddt;
            split_words(out, i, xd, vd, xc.w, x, v);
            e = narrow6(ed);
            ep = (float)sqrt(2.0 / 3.0 * contract6(ed, ed));
        } else {
            v.x = v0.x + dt * a.x;
            v.y = v0.y + dt * a.y;
            v.z = v0.z + dt * a.z;
            v.w = v0.w + dt * a.w;
            x.x = 0.5f * (v.x + v0.x) * dt + x0.x;
            x.y = 0.5f * (v.y + v0.y) * dt + x0.y;
            x.z = 0.5f * (v.z + v0.z) * dt + x0.z;
            x.w = xc.w;
            e = e0 + de * dt;
            ep = sqrtf(2.0f / 3.0f * J2(e));
        }
        out.pos[i] = x;
        out.vel[i] = v;
        store_t2(out.stn, i, e);
        const bool bad = !(isfinite(x.x) && isfinite(x.y) && isfinite(x.z) && isfinite(v.x) && isfinite(v.y) &&
                           isfinite(v.z) && isfinite(v.w));
        if (verlet.xbuild) verlet_check(verlet, i, x, v, a);
        T6d sd = widen6(s0);
        double evd = id0.z;
        vw_update_d(vw_const(vw, id.x), (double)dt, de, w, sd, evd);
        const tensor2d s = narrow6(sd);
        out.idep[i] = make_float4(id.x, ep, (float)evd, id.w);
        store_t2(out.str, i, s);
        pack_slot<kMixed>(nb, i, out.pos[i], out.vel[i], s);   /* kinematics stored above */
        if (health && (bad || !(isfinite(s.xx) && isfinite(s.yy) && isfinite(s.zz) && isfinite(s.xy) &&
                                isfinite(s.xz) && isfinite(s.yz))))
            atomicAdd(health + HEALTH_NONFINITE, 1);
        return;
    }
    float4 v, x;
    tensor2d s, e;
    float ep, ev = id.z;
    if (kMixed) {
        const double ddt = dt;
        const double4 v0d = join4(v0, ini.vlo[k]), x0d = join4(x0, ini.xlo[k]);
        double4 vd, xd;
        vd.x = v0d.x + ddt * a.x; vd.y = v0d.y + ddt * a.y; vd.z = v0d.z + ddt * a.z; vd.w = v0d.w + ddt * a.w;
        xd.x = 0.5 * (vd.x + v0d.x) * ddt + x0d.x;
        xd.y = 0.5 * (vd.y + v0d.y) * ddt + x0d.y;
        xd.z = 0.5 * (vd.z + v0d.z) * ddt + x0d.z;
        xd.w = 0.0;
        T6d ed = widen6(e0), dd = widen6(de);
        ed.xx += dd.xx * ddt; ed.yy += dd.yy * ddt; ed.zz += dd.zz * ddt;
        ed.xy += dd.xy * ddt; ed.xz += dd.xz * ddt; ed.yz += dd.yz * ddt;
        double pd = xc.w, epd = ep0;
        T6d sd = widen6(s0);
        if (M.model == 1) {
            dp_update_d(M, ddt, w, dd, pd, epd, sd);
        } else {
            hypo_update_d(M, ddt, dd, w, sd);
            epd = sqrt(2.0 / 3.0 * contract6(ed, ed));
        }
        split_words(out, i, xd, vd, (float)pd, x, v);
        s = narrow6(sd);
        e = narrow6(ed);
        ep = (float)epd;
    } else {
        v.x = v0.x + dt * a.x;
        v.y = v0.y + dt * a.y;
        v.z = v0.z + dt * a.z;
        v.w = v0.w + dt * a.w;
        x.x = 0.5f * (v.x + v0.x) * dt + x0.x;
        x.y = 0.5f * (v.y + v0.y) * dt + x0.y;
        x.z = 0.5f * (v.z + v0.z) * dt + x0.z;
        e = e0 + de * dt;
        float p = xc.w;
        ep = ep0;
        s = s0;
        if (M.model == 1) {
            dp_update(M, dt, w, de, p, ep, s);
        } else {
            hypo_update(M, dt, de, w, s);
            ep = sqrtf(2.0f / 3.0f * J2(e));
        }
        x.w = p;
    }
    out.pos[i] = x;
    out.vel[i] = v;
    out.idep[i] = make_float4(id.x, ep, ev, id.w);
    store_t2(out.str, i, s);
    store_t2(out.stn, i, e);
    pack_slot<kMixed>(nb, i, x, v, s);
    if (health) {
        const bool ok = isfinite(x.x) && isfinite(x.y) && isfinite(x.z) && isfinite(v.x) && isfinite(v.y) &&
                        isfinite(v.z) && isfinite(v.w) && isfinite(s.xx) && isfinite(s.yy) && isfinite(s.zz) &&
                        isfinite(s.xy) && isfinite(s.xz) && isfinite(s.yz);
        if (!ok) atomicAdd(health + HEALTH_NONFINITE, 1);
    }
    if (verlet.xbuild) verlet_check(verlet, i, x, v, a);
}

}  // namespace

int launch_predict(const Parameters* ph, const Parameters* pd, const State& in, const State& out, const State* snap,
                   const Rates& r, cudaStream_t s, const MaterialTable& mt, const MaterialTable& vw, float* rec,
                   bool stage)
{
    if (ph->np <= 0) return LQ_OK;
    if (ph->constitutive_model == 3 && (!vw.p || vw.n <= 0))
        return set_error(LQ_ERR_ARG, "predictor: constitutive model 3 needs a von Wolffersdorff table");
    const bool do_snap = snap && snap->pos;
    if (stage && (do_snap || out.pos == in.pos))
        return set_error(LQ_ERR_ARG, "predictor: a stage buffer needs its own output and no snapshot");
    State sn = do_snap ? *snap : State{nullptr, nullptr, nullptr, nullptr, nullptr};
    /* model 3 gets its own instantiation: its FP64 sub-stepping needs far
     * more registers than the other models' kernels */
    const bool vwm = ph->constitutive_model == 3;
    const int nb = blocks_for(ph->np, kBlock);
    const NbrArrays pk = rec ? nbr_arrays(rec, ph->np) : NbrArrays{nullptr, nullptr, nullptr, nullptr};
    if (in.xlo && out.xlo) {
        if (vwm) k_predict<true, true><<<nb, kBlock, 0, s>>>(pd, ph->np, ph->npb, in, out, sn, do_snap, r, mt, vw, pk,
                                                              stage);
        else k_predict<true, false><<<nb, kBlock, 0, s>>>(pd, ph->np, ph->npb, in, out, sn, do_snap, r, mt, vw, pk,
                                                              stage);
    } else {
        if (vwm) k_predict<false, true><<<nb, kBlock, 0, s>>>(pd, ph->np, ph->npb, in, out, sn, do_snap, r, mt, vw, pk,
                                                              stage);
        else k_predict<false, false><<<nb, kBlock, 0, s>>>(pd, ph->np, ph->npb, in, out, sn, do_snap, r, mt, vw, pk,
                                                              stage);
    }
    LQ_TRY_CUDA(cudaGetLastError(), "k_predict");
    return LQ_OK;
}

int launch_correct(const Parameters* ph, const Parameters* pd, const State& cur, const State& ini,
                   const int* ini_idx, const Rates& r, int* health, cudaStream_t s)
{
    if (ph->npm <= 0) return LQ_OK;
    if (ph->constitutive_model == 3)
        return set_error(LQ_ERR_ARG, "corrector: constitutive model 3 needs a von Wolffersdorff table");
    k_correct<false, false><<<blocks_for(ph->npm, kBlock), kBlock, 0, s>>>(pd, ph->np, ph->npb, cur, ini, ini_idx, cur, r, health,
                                                             VerletCheck{nullptr, nullptr, 0.0f, 0.0f, nullptr, 0.0f}, ph->npb,
                                                             MaterialTable(), MaterialTable(),
                                                             NbrArrays{nullptr, nullptr, nullptr, nullptr});
    LQ_TRY_CUDA(cudaGetLastError(), "k_correct");
    return LQ_OK;
}

int launch_correct_into(const Parameters* ph, const Parameters* pd, const State& cur, const State& ini,
                        const State& out, const Rates& r, int* health, const float4* xbuild, int* rebuild,
                        float skin, cudaStream_t s, const MaterialTable& mt, const MaterialTable& vw,
                        const float4* xwide, float wide, float* rec)
{
    if (ph->np <= 0) return LQ_OK;
    if (ph->constitutive_model == 3 && (!vw.p || vw.n <= 0))
        return set_error(LQ_ERR_ARG, "corrector: constitutive model 3 needs a von Wolffersdorff table");
    /* a dynamic step never exceeds the fixed one, cfl h / cs (ph->dt) */
    if (xwide && !(wide > skin)) return set_error(LQ_ERR_ARG, "corrector: the wide cut-off must exceed the skin");
    const VerletCheck vc{xbuild, rebuild, 0.5f * skin, ph->dt, xwide, 0.5f * (wide - skin)};
    const bool vwm = ph->constitutive_model == 3;
    if (ph->npm <= 0) return LQ_OK;
    /* material slots only: boundary slots are written by Adami into both
     * buffers */
    const int nb = blocks_for(ph->npm, kBlock), f = ph->npb;
    const NbrArrays pk = rec ? nbr_arrays(rec, ph->np) : NbrArrays{nullptr, nullptr, nullptr, nullptr};
    if (cur.xlo && ini.xlo && out.xlo) {
        if (vwm) k_correct<true, true><<<nb, kBlock, 0, s>>>(pd, ph->np, ph->npb, cur, ini, nullptr, out, r, health, vc, f, mt, vw, pk);
        else k_correct<true, false><<<nb, kBlock, 0, s>>>(pd, ph->np, ph->npb, cur, ini, nullptr, out, r, health, vc, f, mt, vw, pk);
    } else {
        if (vwm) k_correct<false, true><<<nb, kBlock, 0, s>>>(pd, ph->np, ph->npb, cur, ini, nullptr, out, r, health, vc, f, mt, vw, pk);
        else k_correct<false, false><<<nb, kBlock, 0, s>>>(pd, ph->np, ph->npb, cur, ini, nullptr, out, r, health, vc, f, mt, vw, pk);
    }
    LQ_TRY_CUDA(cudaGetLastError(), "k_correct");
    return LQ_OK;
}

}  // namespace lqb

/* ------------------------------------------------------------------ C ABI */

extern "C" int lq_predictor(const void* par_host, const void* par_device, float* pospres, float* velrhop,
                            float* idep, float* str, float* stn, float* pospres_ini, float* velrhop_ini,
                            float* idep_ini, float* str_ini, float* stn_ini, const float* accad, const float* spin,
                            const float* acestn, void* stream)
{
    if (!par_host || !par_device) return lqb::set_error(LQ_ERR_ARG, "lq_predictor: null Parameters");
    const Parameters* ph = static_cast<const Parameters*>(par_host);
    if (ph->npm == 0) return LQ_OK; /* reference returns before the snapshot too */
    if (!pospres || !velrhop || !idep || !str || !stn || !pospres_ini || !velrhop_ini || !idep_ini || !str_ini ||
        !stn_ini || !accad || !spin || !acestn)
        return lqb::set_error(LQ_ERR_ARG, "lq_predictor: null array");
    lqb::State st{(float4*)pospres, (float4*)velrhop, (float4*)idep, (tensor2d*)str, (tensor2d*)stn};
    lqb::State sn{(float4*)pospres_ini, (float4*)velrhop_ini, (float4*)idep_ini, (tensor2d*)str_ini,
                  (tensor2d*)stn_ini};
    lqb::Rates r{(float4*)accad, (float4*)spin, (tensor2d*)acestn};
    return lqb::launch_predict(ph, static_cast<const Parameters*>(par_device), st, st, &sn, r,
                               static_cast<cudaStream_t>(stream));
}

extern "C" int lq_corrector(const void* par_host, const void* par_device, float* pospres, float* velrhop,
                            float* idep, float* str, float* stn, const float* pospres_ini, const float* velrhop_ini,
                            const float* idep_ini, const float* str_ini, const float* stn_ini, const float* accad,
                            const float* spin, const float* acestn, void* stream)
{
    if (!par_host || !par_device) return lqb::set_error(LQ_ERR_ARG, "lq_corrector: null Parameters");
    const Parameters* ph = static_cast<const Parameters*>(par_host);
    if (ph->npm == 0) return LQ_OK;
    if (!pospres || !velrhop || !idep || !str || !stn || !pospres_ini || !velrhop_ini || !idep_ini || !str_ini ||
        !stn_ini || !accad || !spin || !acestn)
        return lqb::set_error(LQ_ERR_ARG, "lq_corrector: null array");
    lqb::State st{(float4*)pospres, (float4*)velrhop, (float4*)idep, (tensor2d*)str, (tensor2d*)stn};
    lqb::State in{(float4*)pospres_ini, (float4*)velrhop_ini, (float4*)idep_ini, (tensor2d*)str_ini,
                  (tensor2d*)stn_ini};
    lqb::Rates r{(float4*)accad, (float4*)spin, (tensor2d*)acestn};
    return lqb::launch_correct(ph, static_cast<const Parameters*>(par_device), st, in, nullptr, r, nullptr,
                               static_cast<cudaStream_t>(stream));
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

void Predictor(Parameters* par_host, Parameters* par_device, float4* pospres, float4* velrhop, float4* idep,
               tensor2d* str, tensor2d* stn, float4* pospres_ini, float4* velrhop_ini, float4* idep_ini,
               tensor2d* str_ini, tensor2d* stn_ini, float4* accad, float4* spin, tensor2d* acestn)
{
    check_or_die(lq_predictor(par_host, par_device, (float*)pospres, (float*)velrhop, (float*)idep, (float*)str,
                              (float*)stn, (float*)pospres_ini, (float*)velrhop_ini, (float*)idep_ini,
                              (float*)str_ini, (float*)stn_ini, (const float*)accad, (const float*)spin,
                              (const float*)acestn, nullptr),
                 "Predictor");
}

void Corrector(Parameters* par_host, Parameters* par_device, float4* pospres, float4* velrhop, float4* idep,
               tensor2d* str, tensor2d* stn, float4* pospres_ini, float4* velrhop_ini, float4* idep_ini,
               tensor2d* str_ini, tensor2d* stn_ini, float4* accad, float4* spin, tensor2d* acestn)
{
    check_or_die(lq_corrector(par_host, par_device, (float*)pospres, (float*)velrhop, (float*)idep, (float*)str,
                              (float*)stn, (const float*)pospres_ini, (const float*)velrhop_ini,
                              (const float*)idep_ini, (const float*)str_ini, (const float*)stn_ini,
                              (const float*)accad, (const float*)spin, (const float*)acestn, nullptr),
                 "Corrector");
}
