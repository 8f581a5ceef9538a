// Host check of the mixed form's packed neighbour velocity
// (loquat_b200/csrc/lq_pack.h), the code the GPU's pack and pair kernels
// run.  Over random and edge-case velocities it asserts that the decode
// equals an independent statement of the rounding rule in doubles (a
// shared quantum q = 2^(E - 17) for the least E with max |v_k| < 2^E,
// raised once if a mantissa leaves [-2^17, 2^17 - 1]; each component
// rounded to nearest even on a multiple of q), that every error is at
// most q / 2, that w1's reserved bits stay zero, and that a non-finite
// velocity decodes to NaN.  Prints "OK <cases>" on success.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <random>

#include "lq_pack.h"

static int g_fail = 0;

static void expect(bool ok, const char* what, float x, float y, float z)
{
    if (!ok && g_fail++ < 10) std::printf("FAIL %s at (%.9g, %.9g, %.9g)\n", what, x, y, z);
}

static void rule(float vx, float vy, float vz, double out[3], double& q)
{
    const double f[3] = {vx, vy, vz};
    const double m = std::fmax(std::fabs(f[0]), std::fmax(std::fabs(f[1]), std::fabs(f[2])));
    int e = 0;
    if (m > 0.0) std::frexp(m, &e);
    if (e < -109) e = -109;
    for (int pass = 0; pass < 2; ++pass) {
        q = std::ldexp(1.0, e - 17);
        bool fits = true;
        for (int k = 0; k < 3; ++k) {
            out[k] = std::nearbyint(f[k] / q);
            fits = fits && out[k] >= -131072.0 && out[k] <= 131071.0;
        }
        if (fits) break;
        ++e;
    }
    for (int k = 0; k < 3; ++k) out[k] *= q;
}

static void check(float vx, float vy, float vz)
{
    unsigned w0, w1;
    lqb::pack_velocity_words(vx, vy, vz, w0, w1);
    float d[3];
    lqb::unpack_velocity_words(w0, w1, d[0], d[1], d[2]);
    double want[3], q;
    rule(vx, vy, vz, want, q);
    const float v[3] = {vx, vy, vz};
    for (int k = 0; k < 3; ++k) {
        expect((double)d[k] == want[k], "decode differs from the rounding rule", vx, vy, vz);
        expect(std::fabs((double)d[k] - (double)v[k]) <= 0.5 * q, "error above q / 2", vx, vy, vz);
    }
    expect((w1 & 0x80400000u) == 0u, "reserved bits of w1 set", vx, vy, vz);
}

int main()
{
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<double> uni(-1.0, 1.0);
    std::uniform_int_distribution<int> expo(-40, 12);
    long cases = 0;
    // random velocities over many magnitudes, with components of unequal size
    for (int n = 0; n < 2000000; ++n) {
        const int e0 = expo(rng);
        const float s0 = (float)std::ldexp(1.0, e0);
        const float s1 = (n % 3 == 0) ? (float)std::ldexp(1.0, e0 - (n % 29)) : s0;
        check((float)(uni(rng) * s0), (float)(uni(rng) * s1), (float)(uni(rng) * s0));
        ++cases;
    }
    // values on and around binade edges, where a mantissa can round to 2^17
    for (int e = -30; e <= 10; ++e) {
        const float b = (float)std::ldexp(1.0, e);
        const float edge[] = {b, std::nextafter(b, 0.0f), std::nextafter(b, 2.0f * b), 0.5f * b, -b,
                              -std::nextafter(b, 0.0f), (float)(b * (1.0 - std::ldexp(1.0, -19)))};
        for (float a : edge)
            for (float c : edge) {
                check(a, c, 0.0f);
                check(0.0f, a, -c);
                check(c, -a, a);
                cases += 3;
            }
    }
    // zeros, tiny values, a ties-to-even case
    check(0.0f, 0.0f, 0.0f);
    check(-0.0f, 1e-38f, -1e-38f);
    check(1e-35f, 0.0f, 0.0f);
    check(1.0f, (float)std::ldexp(3.0, -18), (float)std::ldexp(-5.0, -18));
    cases += 4;
    // non-finite input decodes to NaN
    const float bad[] = {INFINITY, -INFINITY, NAN};
    for (float b : bad) {
        unsigned w0, w1;
        lqb::pack_velocity_words(1.0f, b, 0.5f, w0, w1);
        float d[3];
        lqb::unpack_velocity_words(w0, w1, d[0], d[1], d[2]);
        expect(std::isnan(d[0]) && std::isnan(d[1]) && std::isnan(d[2]), "non-finite not NaN", 1.0f, b, 0.5f);
        ++cases;
    }
    if (g_fail) {
        std::printf("%d failures\n", g_fail);
        return 1;
    }
    std::printf("OK %ld\n", cases);
    return 0;
}
