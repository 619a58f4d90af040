// Host-side preparation of one surface mesh for the device apply.
//
// Replaces the reference's host topology (src/meshTopology.cpp:22-261, an
// O(ne * nedges) edge search) and its per-matvec host pair enumeration
// (src/BEM3dLaplaceGPU.cu:1224-1260) with one O(ne log ne) pass at mesh
// creation: triangles are reordered along a Morton curve of their centroids,
// grouped in cells of kCell consecutive triangles (the far-field source
// granularity), and the near pairs (triangles sharing at least one vertex)
// are listed once in CSR form for the Sauter-Schwab correction.
#pragma once

#include <cstdint>
#include <vector>

#include "quadrature.h"

namespace eb {

constexpr int kCell = 32;  // source triangles per cell (shared origin for FP32 coordinates)

struct HostMesh {
  int nv = 0, ne = 0, order = 4, Q = 0;
  Quadrature quad;
  std::vector<double> nodes;  // [nv][3]
  std::vector<int> elems;     // [ne][3], 0-based

  // Morton order: perm[s] = original index of sorted triangle s; iperm inverse.
  std::vector<int> perm, iperm;
  int ncells = 0;
  std::vector<double> cell_center;  // [ncells][3]

  // Target items: a triangle's Q points split into chunks of at most K points.
  int K = 0;        // target points per item (compile-time kernel width)
  int nchunk = 0;   // items per triangle
  int nitems = 0;   // ne * nchunk

  // Near pairs (including coincident), CSR by original test triangle.
  std::vector<int> sl_rowptr, sl_col;  // col = original trial triangle
  std::vector<int> pair_i;             // original test triangle of each pair
  std::vector<int8_t> pair_kind;
  // DL near CSR over vertex columns; entry e = 3*pair + k feeds slot dl_slot_of[e].
  std::vector<int> dl_rowptr, dl_col;
  std::vector<int> dl_contrib_ptr, dl_contrib;  // slot -> entries, ascending

  long long far_quad_pairs = 0;  // regular quadrature-point pairs per apply
  bool topology_on_device = false;  // near-pair lists built by device_topology
  // (target item, source triangle) pairs in source cells well separated from
  // the item's warp of target items, and in the others (where a far-field kernel
  // masks vertex-sharing pairs and forms differences directly); set with the
  // static tables
  long long far_cell_tri_pairs = 0, near_cell_tri_pairs = 0;
};

// Validates and prepares (Morton order, cells, target items and, when
// topology is set, the near-pair CSR through host_topology); returns EB_OK or
// an error status with a message.
int prepare_host_mesh(int nv, const double* nodes, int ne, const int* elems1, int order, HostMesh* m,
                      bool topology = true);

// The near-pair CSR (sl_*, pair_*, dl_*) and far_quad_pairs of a prepared
// mesh, on the host. device_topology (topology.cu) builds the same arrays on
// the GPU for large meshes.
void host_topology(HostMesh* m);

// The same arrays built on the current GPU (topology.cu); *done is false when
// a row has too many candidates and the caller must use host_topology.
int device_topology(HostMesh* m, bool* done);
// Meshes with at least this many triangles use device_topology.
int device_topology_min();

// Target items per triangle and points per item for Q quadrature points.
void target_split(int Q, int* K, int* nchunk);

}  // namespace eb
