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
// largest mesh the symmetric engine takes: its partial slots (one FP64 pair
// per 128-triangle tile and row) stay at or below 2^35 bytes (32 GiB)
constexpr int kSymMaxTriangles = 524288;

// Work list of the symmetric plan for nitems = ne target rows (one item per
// triangle) and ncells cells; returns the number of partial slots per row.
int far_sym_items(int nitems, int ncells, int cells_per_item, std::vector<WorkItem>& items);
// Dynamic shared memory of one CTA (staged tile + transposed-sum buffer) of
// the FP32 (fp32) or FP64 kernel.
size_t far_sym_smem_bytes(bool fp32);
// Resident CTAs per SM.
int far_sym_occupancy(bool fp32);
cudaError_t far_sym_launch(bool fp32, const FarMeshDesc* dm, const WorkItem* di, int n, int* dc, int grid,
                           cudaStream_t st);

}  // namespace eb
