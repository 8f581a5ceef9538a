/*
 * LOQUAT-B200 drop-in for the reference's neighbour grid
 * (reference: src/loquat_grid.h:28-66; implementation closed there).
 *
 * The private member list is part of the ABI: a caller compiled against the
 * reference header allocates a LoquatGrid of exactly these eight members, so
 * no member may be added.  This build uses them as follows:
 *   part_cel        sorted cell key of every particle            int[np]
 *   part_idx        sorted slot -> previous slot (the permutation) int[np]
 *   cell_beg        first sorted slot of each cell, -1 if empty   int[ncell]
 *   cell_end        one past the last slot, -1 if empty           int[ncell]
 *   part_cel_cache  unsorted cell key                              int[np]
 *   part_idx_cache  rank of a particle inside its cell             int[np]
 *   buffer          cell start table (ncell + 1 ints) + scan scratch
 *   buffer_storage_bytes  size of buffer
 *
 * Cell key (pinned by the reference's consumers, adami_boundary.cu:80-100):
 *   c_a = floor(0.5 * x_a * (1/h)) per axis from the raw coordinate,
 *   key = layer * ncell_one_layer + (cx * cell_num_y + cy) * cell_num_z + cz,
 *   layer = 0 for slots [0, npb) (boundary) and 1 for [npb, np) (material),
 *   key = ncell_delete for any particle outside the cell lattice.
 * The sort is stable: inside a cell, particles keep their previous order.
 * All work is queued on the legacy default stream, like the reference.
 */
#pragma once
#ifndef LOQUAT_B200_LOQUAT_GRID_H
#define LOQUAT_B200_LOQUAT_GRID_H

#include <cuda_runtime.h>
#include <types.h>

class LoquatGrid
{
    private:

        int* part_cel;
        int* part_idx;
        int* cell_beg;
        int* cell_end;

        int* part_cel_cache;
        int* part_idx_cache;
        void* buffer;

        size_t buffer_storage_bytes;

        void SortParticleByCellIndex(Parameters* par_host);

    public:

        LoquatGrid();

        ~LoquatGrid();

        const int* GetPartCel() const { return part_cel; }
        const int* GetPartIdx() const { return part_idx; }
        const int* GetCellBeg() const { return cell_beg; }
        const int* GetCellEnd() const { return cell_end; }

        void GridConfig(Parameters* par_host);

        void ResizeArrayLength(int np_new, int ncell_new);

        void NeighborSearch(Parameters* par_host, Parameters* par_device, float4* pospres, float4* idep);

        void SortArrayFloat4(int np, float4* data, float4* data_cache);

        void SortArrayTensor2d(int np, tensor2d* data, tensor2d* data_cache);
};

#endif
