// Host check of the pair kernel's tile order (loquat_b200/csrc/lq_tile.h,
// the index arithmetic that k_tile_segments runs on the device): for
// random cell-start tables over many lattice shapes and tile heights, the
// segments must partition the material slots [npb, np) into a permutation
// of the targets, and every segment inside the material layer must hold
// the slots of one column's tz cells.  Built and run by
// tests/test_tile_order.py; prints "OK <cases>" or the first failure.
#include <cstdio>
#include <random>
#include <vector>

#include "lq_tile.h"

namespace {

int fail(const char* what, int nx, int ny, int nz, int tz, int npb)
{
    std::printf("FAIL %s: lattice %d x %d x %d, tz %d, npb %d\n", what, nx, ny, nz, tz, npb);
    return 1;
}

int check(std::mt19937& rng, int nx, int ny, int nz, int tz, int npb_shift)
{
    const int L = nx * ny * nz, ncell = 2 * L + 1;
    std::uniform_int_distribution<int> cnt(0, 4);
    std::vector<int> count(ncell), start(ncell + 1, 0);
    for (int c = 0; c < ncell; ++c) count[c] = (c % 5 == 3) ? 0 : cnt(rng);  // some empty cells
    for (int c = 0; c < ncell; ++c) start[c + 1] = start[c] + count[c];
    const int np = start[ncell];
    int npb = start[L] + npb_shift;
    if (npb < 0) npb = 0;
    if (npb > np) npb = np;
    std::vector<int> cell_of(np);
    for (int c = 0; c < ncell; ++c)
        for (int j = start[c]; j < start[c + 1]; ++j) cell_of[j] = c;

    const lqb::TileGrid g = lqb::tile_grid(nx, ny, nz, L, tz);
    std::vector<int> beg(g.nseg), len(g.nseg), off(g.nseg + 1, 0);
    for (int s = 0; s < g.nseg; ++s) {
        lqb::tile_segment(g, start.data(), npb, np, s, &beg[s], &len[s]);
        if (len[s] < 0) return fail("negative length", nx, ny, nz, tz, npb);
        if (len[s] > 0 && (beg[s] < npb || beg[s] + len[s] > np)) return fail("segment outside [npb, np)", nx, ny, nz, tz, npb);
        off[s + 1] = off[s] + len[s];
        if (s < g.nseg - 2 && len[s] > 0) {
            // one column, z within [z0, z0 + tz), all in the material layer
            const int c0 = cell_of[beg[s]] - L;
            const int col = c0 / nz, z0 = (c0 % nz) / tz * tz;
            for (int j = beg[s]; j < beg[s] + len[s]; ++j) {
                const int c = cell_of[j] - L;
                if (c < 0 || c >= L) return fail("slot outside the material layer", nx, ny, nz, tz, npb);
                if (c / nz != col || c % nz < z0 || c % nz >= z0 + tz) return fail("segment spans columns or tiles", nx, ny, nz, tz, npb);
            }
        }
    }
    const int npm = np - npb;
    if (off[g.nseg] != npm) return fail("segments do not add up to the material count", nx, ny, nz, tz, npb);
    std::vector<int> order(npm, -1), seen(npm, 0);
    for (int s = 0; s < g.nseg; ++s)
        for (int k = 0; k < len[s]; ++k) order[off[s] + k] = beg[s] + k - npb;   // as k_tile_fill writes it
    for (int v : order) {
        if (v < 0 || v >= npm) return fail("target out of range", nx, ny, nz, tz, npb);
        if (seen[v]++) return fail("target twice", nx, ny, nz, tz, npb);
    }
    return 0;
}

}  // namespace

int main()
{
    std::mt19937 rng(12345);
    const int lattices[][3] = {{1, 1, 1}, {2, 5, 3}, {7, 4, 11}, {3, 3, 6}, {10, 1, 2}, {4, 8, 1}, {9, 9, 17}};
    const int heights[] = {1, 2, 3, 6, 7, 20};
    const int shifts[] = {0, -3, 5};   // sound state; material slots below the layer; npb inside it
    int cases = 0;
    for (const auto& d : lattices)
        for (int tz : heights)
            for (int sh : shifts)
                for (int rep = 0; rep < 3; ++rep) {
                    if (check(rng, d[0], d[1], d[2], tz, sh)) return 1;
                    ++cases;
                }
    std::printf("OK %d\n", cases);
    return 0;
}
