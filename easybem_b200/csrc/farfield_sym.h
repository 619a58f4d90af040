// Symmetric far field of the fused FP32 SL+DL apply (farfield_sym.cu): every
// unordered quadrature-point pair is evaluated once and feeds both triangle
// orders.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "farfield.cuh"

namespace eb {

constexpr int kSymRule = 7;  // the engine's quadrature rule size (index 4)
// source cells per upper work item: 0 takes the build's default (8 cells,
// 256 source triangles)
constexpr int kSymCellsPerItem = 0;
// the same in a batch: coarser items keep the merged work list short (many
// meshes share each launch, and the list is rebuilt whenever the solver's
// systems change)
constexpr int kSymBatchCellsPerItem = 32;
// largest slot allocation the symmetric engine takes (one FP64 value per
// output, 128-triangle tile and row): 2^35 bytes (32 GiB), an SL+DL mesh of
// 524,288 triangles
constexpr size_t kSymMaxSlotBytes = (size_t)1 << 35;

// Source cells per upper work item for a requested count (0: the build's default).
int far_sym_cells_per_item(int cells_per_item);
// Work list of the symmetric plan for nitems = ne target rows (one item per
// triangle) and ncells cells; returns the largest number of partial slots of
// a row (sym_row_slots gives each row's).
int far_sym_items(int nitems, int ncells, int cells_per_item, std::vector<WorkItem>& items);
// Variants with a symmetric kernel: SL+DL (nsl = nd = 1) and SL only with 1,
// 3 or 4 right-hand sides, in FP32 and FP64.
bool far_sym_variant(bool fp32, int nsl, int nd);
// Dynamic shared memory of one CTA (staged tile + transposed-sum buffer).
size_t far_sym_smem_bytes(bool fp32, int nsl, int nd);
// Resident CTAs per SM.
int far_sym_occupancy(bool fp32, int nsl, int nd);
cudaError_t far_sym_launch(bool fp32, int nsl, int nd, const FarMeshDesc* dm, const WorkItem* di, int n, int* dc,
                           int grid, cudaStream_t st);

}  // namespace eb
