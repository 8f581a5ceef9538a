/* Index arithmetic of the pair kernel's tile order, shared by the device
 * kernel that builds the order (sph.cu: k_tile_segments) and by host code
 * that checks it.  No CUDA types: the header compiles with a plain C++
 * compiler too.
 *
 * The material layer's lattice (cells L .. 2L-1 of the grid, key
 * L + (cx * ny + cy) * nz + cz, z fastest) is cut into tiles of 3 x 3
 * columns by tz cells, numbered with the z index fastest; within a tile
 * the nine columns come in order c = 0..8 (cx + c % 3, cy + c / 3), each
 * column's tz cells being one run of consecutive slots.  Segment
 * s < nseg - 2 is column s % 9 of tile s / 9; segment nseg - 2 holds the
 * material slots below the material layer (none in a sound state) and
 * segment nseg - 1 the out-of-lattice cell (key 2L) up to np.  Every
 * segment is clamped to [npb, np), so the segments partition the material
 * slots [npb, np) whenever start is a non-decreasing cell-start table with
 * start[2L] <= np. */
#pragma once

#if defined(__CUDACC__)
#define LQ_TILE_HD __host__ __device__ __forceinline__
#else
#define LQ_TILE_HD inline
#endif

namespace lqb {

struct TileGrid {
    int nx, ny, nz;   /* cells per axis */
    int L;            /* cells per layer */
    int tz;           /* tile height in cells */
    int nty, ntz;     /* tiles along y and z */
    int nseg;         /* segments: 9 per tile + 2 */
};

LQ_TILE_HD TileGrid tile_grid(int nx, int ny, int nz, int L, int tz)
{
    TileGrid g;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.L = L;
    g.tz = tz;
    g.nty = (ny + 2) / 3;
    g.ntz = (nz + tz - 1) / tz;
    g.nseg = ((nx + 2) / 3) * g.nty * g.ntz * 9 + 2;
    return g;
}

/* Slot range [*b, *b + *len) of segment s, for material slots [npb, np). */
LQ_TILE_HD void tile_segment(const TileGrid& g, const int* start, int npb, int np, int s, int* b_out, int* len_out)
{
    int b = npb, e = npb;
    if (s < g.nseg - 2) {
        const int c = s % 9, tile = s / 9;
        const int kz = tile % g.ntz, rest = tile / g.ntz;
        const int X = 3 * (rest / g.nty) + c % 3, Y = 3 * (rest % g.nty) + c / 3, z0 = kz * g.tz;
        if (X < g.nx && Y < g.ny && z0 < g.nz) {
            const int key0 = g.L + (X * g.ny + Y) * g.nz + z0;
            const int ncz = g.nz - z0 < g.tz ? g.nz - z0 : g.tz;
            b = start[key0];
            e = start[key0 + ncz];
        }
    } else if (s == g.nseg - 2) {
        e = start[g.L];
    } else {
        b = start[2 * g.L];
        e = np;
    }
    b = b > npb ? b : npb;
    e = e < np ? e : np;
    *b_out = b;
    *len_out = e > b ? e - b : 0;
}

}  // namespace lqb
