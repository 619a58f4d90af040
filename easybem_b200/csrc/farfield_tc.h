// Tensor-core far field of the fused FP32 SL+DL apply (farfield_tc.cu).
#pragma once

#include <cuda_runtime.h>

#include "farfield.cuh"

namespace eb {

constexpr int kTcChunk = 112;  // source points per MMA (half a cell: 16 triangles x 7 points)
constexpr int kTcRule = 7;     // triangle-rule points the kernel is built for (quadrature index 4)

// Bytes of the per-mesh source operands: one 14,336-byte block (224 rows x
// 64 bytes) per cell for the distance GEMM, the same for the DL GEMM, and one
// float charge per padded source point.
inline size_t far_tc_operand_bytes(int ncells) { return (size_t)ncells * kCell * kTcRule * 64; }
inline size_t far_tc_charge_bytes(int ncells) { return (size_t)ncells * kCell * kTcRule * 4; }

// Pipe work per far quadrature pair of the kernel as built: MUFU reciprocal
// square roots, FMA-pipe lane operations, tensor-core flops.
void far_tc_costs(double* mufu_per_pair, double* fma_ops_per_pair, double* tensor_flops_per_pair);

// Once per mesh: the distance-GEMM source operand from the FP32 positions.
cudaError_t far_tc_prep_static(int ne, int ncells, const float4* pos32, float4* bd2, cudaStream_t st);
// Per apply, after the record preparation of the fused FP32 variant: the
// DL-GEMM source operand and the SL charges.
cudaError_t far_tc_prep_dl(int ne, int ncells, const float4* rec, const float4* splane32, float4* be, float* charges,
                           cudaStream_t st);
// Per-entry arguments of the batched DL-operand preparation.
struct TcPrepArgs {
  int ne, ncells;
  const float4* rec;       // records of the fused FP32 variant
  const float4* splane32;  // n_j and the cell-relative plane offset
  float4* be;              // DL-GEMM source operand out
  float* charges;          // SL charges out
  const int* active;       // optional: skip while *active == 0
};
// Blocks [off[e], off[e+1]) of 256 threads prepare entry e.
cudaError_t far_tc_prep_dl_batch(const TcPrepArgs* d_args, const int* d_off, int n, int nblocks, cudaStream_t st);
// Thread blocks of 256 points far_tc_prep_dl_batch needs for a mesh.
inline int far_tc_prep_blocks(int ncells) { return (ncells * kCell * kTcRule + 255) / 256; }

// The persistent kernel (grid = SM count); *d_error becomes 1 if a bounded
// wait ran out.
cudaError_t far_tc_launch(const FarMeshDesc* d_meshes, const WorkItem* d_items, int nitems, int* d_counter,
                          int* d_error, int grid, cudaStream_t st);

}  // namespace eb
