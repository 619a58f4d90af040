// Far-field kernels: the regular triangle-pair Gauss quadrature treated as an
// N-body sum over quadrature points.
//
// The reference evaluates one triangle pair per thread from host-packed
// geometry (src/BEM3dLaplaceGPU.cu:445-488 SL, :775-827 DL, launched from
// :1292 and :1533). Here each thread owns the quadrature points of one target
// triangle (item), a CTA owns kTT targets, and source quadrature points are
// staged through shared memory in tiles and broadcast to all threads:
//
//   SL:  acc_a += c_b / |x_a - y_b|,          c_b = w_b J_j t_j
//   DL:  acc_a += (x_a - y_b).p_b / |x_a-y_b|^3, p_b = w_b J_j u_h(y_b) n_j
//
// with the target weights w_a J_i / (4 pi) applied when the item is folded.
// Pairs of triangles sharing a vertex are skipped (the FP64 Sauter-Schwab
// near field supplies them). Each work item covers one target tile and one
// contiguous range of source cells; results of different items go to
// separate partial slots, summed in a fixed order by the finalize kernel, so
// the result is bitwise reproducible regardless of scheduling.
//
// FP32 variant: coordinates are stored relative to the centre of the source
// cell (kCell triangles) and of the target triangle, the per-cell offset is
// formed in FP64, so |x - y| keeps full FP32 relative accuracy for close
// pairs; per-cell partial sums are folded into a two-sum (float-float)
// accumulator per target item.
#pragma once

#include <cuda_runtime.h>

#include "common.h"
#include "mesh_host.h"

namespace eb {

#ifndef EB_TT
#define EB_TT 128
#endif
constexpr int kTT = EB_TT;  // target items (threads) per CTA
constexpr int kWarpItems = 32;  // target items per warp: the CUDA-core kernel's separation test is per warp
constexpr int kTS = 64;   // source triangles per shared-memory tile (Q <= 7)
constexpr int kMaxRecSlots = 3;  // record slots of the widest variant
constexpr int kMaxOutputs = 5;   // SL charges + DL of the widest variant
// Shared memory of a staged source tile: 16 bytes per FP32 record slot,
// 32 per FP64 slot.
__host__ __device__ constexpr size_t far_smem_bytes(int src_tile, int Q, int nrec, bool fp32)
{
  return (size_t)src_tile * Q * nrec * (fp32 ? 16 : 32);
}
constexpr int kPrepBlock = 256;     // threads per block of the record preparation (one source point each)
constexpr int kFinalizeBlock = 128; // threads per block of the finalize
constexpr int kFinalizeLanes = 4;   // threads per output row (partial sums and CSR entries split over them)
constexpr int kFinalizeRows = kFinalizeBlock / kFinalizeLanes;  // output rows per finalize block

// FP64 record slot (two 16-byte halves).
struct __align__(16) dq {
  double x, y, z, w;
};

// Source-point record layout (FP32: float4 slots, FP64: dq slots):
//   slot0 = (-2 y, |y|^2), y the quadrature point relative to its cell centre;
//   slot1.. = the strengths [s_0 .. s_{nd-1} (DL columns), c_0, c_1, ...], four
//   per slot, where
//   c_r = w_b J_j t_r[j] are the SL charges and s = w_b J_j u_h(y_b) the DL
//   strength. Far cells use |x - y|^2 = |x|^2 + |y|^2 - 2 x.y directly from
//   slot0; near cells recover y = -(1/2)(-2y) exactly.
__host__ __device__ constexpr int rec_slots(int nsl, int nd) { return 1 + (nsl + nd + 3) / 4; }

// Slot and component of SL charge r after nd DL strengths (DL strength c is
// slot 1 + c / 4, component c % 4).
__host__ __device__ constexpr int charge_slot(int r, int nd) { return 1 + (r + nd) / 4; }
__host__ __device__ constexpr int charge_comp(int r, int nd) { return (r + nd) % 4; }

// A source cell is "far" from a group of target items (a warp's 32 in the
// CUDA-core kernel, a 128-item tile in the tensor-core kernel) when the
// distance of their bounding-sphere centres exceeds kFarRatio times the sum
// of the radii (which bound every vertex): no shared vertex is possible (any
// ratio above 1), and |x|^2 + |y|^2 - 2 x.y loses at most ((k+1)/(k-1))^2
// ulps to cancellation for the closest pairs (k = kFarRatio; 19 at 1.6).
// Measured at the L6 icosphere with 128-item groups: 1.6 leaves 9 % of the
// (target, source triangle) pairs in the other cells (20 % at 2.5) with the
// same mixed-precision error (9e-8); per warp it leaves 4 %.
#ifndef EB_FAR_RATIO
#define EB_FAR_RATIO 1.6
#endif
constexpr double kFarRatio = EB_FAR_RATIO;

// Per-mesh view used by the far-field kernels (device pointers).
struct FarMeshDesc {
  const float4* tgt32;  // [nitems*K]: (x_a - centroid) in FP32, weight w_a
  const dq* tgt64;      // [nitems*K]: (x_a - centroid) in FP64, weight w_a
  const float4* tgtw32; // [nitems*K]: w_a * (phi_0, phi_1, phi_2)(x_a), P1 test weights (FP32)
  const dq* tgtw64;     // [nitems*K]: the same in FP64
  const dq* tcent;      // [nitems]: centroid of the item's triangle (FP64)
  const dq* tnrm;       // [nitems]: unit normal of the item's triangle (FP64)
  const dq* snrm;       // [ne]: unit normal n_j and plane offset P0_j . n_j of sorted sources
  const float4* splane32;  // [ne]: n_j and (P0_j - c_cell) . n_j in FP32 (far cells)
  const dq* splane64;      // [ne]: the same in FP64
  const int4* tvid;     // [nitems]: vertex ids of the item's triangle (-1 if padding)
  const void* rec;      // [ne*Q*nrec] source records (float4 or dq), sorted order
  const int4* svid;     // [ne]: vertex ids of sorted source triangles
  const dq* ccent;      // [ncells]: cell centre and bounding radius (FP64)
  const dq* ttile;      // [ntiles]: target-tile centre and bounding radius (FP64)
  const dq* twarp;      // [nitems / kWarpItems, rounded up]: the same per warp of target items
  double* partial;      // [nout][nsplit][nitems]
  const int* active;    // optional: skip this mesh's work while *active == 0
  // tensor-core kernel only: source operands per cell (UMMA layout) and charges
  const float4* tc_bd2;
  const float4* tc_be;
  const float* tc_charge;
  int nitems, ne, Q, nsplit, src_tile;
};

struct WorkItem {
  int mesh, tgt0, cell0, cell1, split;
};

// Per-mesh arguments of the record-preparation and finalize kernels (device
// pointers); a batch passes an array of them.
struct ApplyArgs {
  // source records
  const void* pos;       // static positions (float4 or dq)
  const double* wj;      // w_b J_j per source point
  const int4* svid;      // sorted source triangle vertex ids
  const int* perm;       // sorted -> original triangle index
  const double* bary;    // triangle-rule points (eta1, eta2)
  const double* t;       // SL densities, nsl columns of stride tstride
  int tstride;
  const double* u;       // DL densities (vertex values), nd columns of stride ustride
  int ustride;
  void* rec;             // records out
  int ne, Q;
  // finalize
  int nchunk, nsplit, nitems;
  const int* iperm;
  const dq* trin;        // per sorted triangle: unit normal, J
  const double* partial;
  const int* sl_rowptr;
  const int* sl_col;
  const double* sl_val;
  const int* dl_rowptr;
  const int* dl_col;
  const double* dl_val;
  double* v;             // SL outputs, nsl columns of stride vstride
  int vstride;
  double* q;             // DL outputs, nd columns of stride qstride
  int qstride;
  const int* active;     // optional: skip this mesh while *active == 0
  // symmetric far field: source cells per upper work item (0: every row has
  // nsplit slots); row s of tile T = s / kTT then has T + 1 + (its tile's upper
  // items) slots, and the rest are never written nor read
  int sym_cells = 0;
};

// Partial slots a row of the symmetric plan holds (sorted row s, ne rows,
// cells_per_item cells per upper item): one per earlier tile, the diagonal,
// one per upper item of its own tile.
__host__ __device__ inline int sym_row_slots(int s, int ne, int cells_per_item)
{
  const int t = s / kTT;
  const int ncells = (ne + kCell - 1) / kCell;
  const int c0 = (t + 1) * (kTT / kCell);
  return t + 1 + (c0 < ncells ? (ncells - c0 + cells_per_item - 1) / cells_per_item : 0);
}

}  // namespace eb
