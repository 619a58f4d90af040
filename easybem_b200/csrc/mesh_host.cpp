#include "mesh_host.h"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <string>

#include "common.h"
#include "pairs.h"

namespace eb {

void target_split(int Q, int* K, int* nchunk)
{
  // Q <= 7 fits one item per triangle; larger rules are split into chunks of
  // at most 8 points (the last chunk padded with zero-weight points).
  if (Q <= 7) { *K = Q; *nchunk = 1; return; }
  *K = 8;
  *nchunk = (Q + 7) / 8;
}

static uint64_t spread21(uint64_t x)
{
  x &= 0x1fffff;
  x = (x | x << 32) & 0x1f00000000ffffULL;
  x = (x | x << 16) & 0x1f0000ff0000ffULL;
  x = (x | x << 8) & 0x100f00f00f00f00fULL;
  x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
  x = (x | x << 2) & 0x1249249249249249ULL;
  return x;
}

int prepare_host_mesh(int nv, const double* nodes, int ne, const int* elems1, int order, HostMesh* m,
                      bool topology)
{
  if (nv < 3 || ne < 1 || !nodes || !elems1)
    return set_error(EB_ERR_INVALID, "mesh needs >= 3 vertices, >= 1 triangle and non-null arrays");
  if (!make_quadrature(order, &m->quad))
    return set_error(EB_ERR_INVALID, "quadrature order must be in 0.." + std::to_string(kMaxOrder));
  m->nv = nv;
  m->ne = ne;
  m->order = order;
  m->Q = m->quad.nt;
  m->nodes.assign(nodes, nodes + 3 * (size_t)nv);
  m->elems.resize(3 * (size_t)ne);
  for (int i = 0; i < ne; i++) {
    for (int k = 0; k < 3; k++) {
      const int v = elems1[3 * i + k];
      if (v < 1 || v > nv)
        return set_error(EB_ERR_MESH, "triangle " + std::to_string(i) + " has vertex index " +
                                          std::to_string(v) + " outside 1.." + std::to_string(nv));
      m->elems[3 * i + k] = v - 1;
    }
    const int* f = &m->elems[3 * i];
    if (f[0] == f[1] || f[1] == f[2] || f[0] == f[2])
      return set_error(EB_ERR_MESH, "triangle " + std::to_string(i) + " repeats a vertex");
    const d3 a = mk3(nodes[3 * f[0]], nodes[3 * f[0] + 1], nodes[3 * f[0] + 2]);
    const d3 b = mk3(nodes[3 * f[1]], nodes[3 * f[1] + 1], nodes[3 * f[1] + 2]);
    const d3 c = mk3(nodes[3 * f[2]], nodes[3 * f[2] + 1], nodes[3 * f[2] + 2]);
    const d3 n = cross3(b - a, c - a);
    const double area2 = std::sqrt(dot3(n, n));
    const double scale = dot3(b - a, b - a) + dot3(c - a, c - a);
    if (!(area2 > 1e-14 * scale) || !std::isfinite(area2))
      return set_error(EB_ERR_MESH, "triangle " + std::to_string(i) + " is degenerate (zero area)");
  }

  // Morton order of centroids.
  std::vector<double> cent(3 * (size_t)ne);
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int i = 0; i < ne; i++)
    for (int d = 0; d < 3; d++) {
      const int* f = &m->elems[3 * i];
      const double c = (nodes[3 * f[0] + d] + nodes[3 * f[1] + d] + nodes[3 * f[2] + d]) / 3.0;
      cent[3 * i + d] = c;
      lo[d] = std::min(lo[d], c);
      hi[d] = std::max(hi[d], c);
    }
  double ext = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1e-300});
  std::vector<std::pair<uint64_t, int>> keys(ne);
  for (int i = 0; i < ne; i++) {
    uint64_t k = 0;
    for (int d = 0; d < 3; d++) {
      double s = (cent[3 * i + d] - lo[d]) / ext;
      uint64_t q = (uint64_t)std::min(2097151.0, std::max(0.0, s * 2097151.0));
      k |= spread21(q) << d;
    }
    keys[i] = {k, i};
  }
  std::sort(keys.begin(), keys.end());
  m->perm.resize(ne);
  m->iperm.resize(ne);
  for (int s = 0; s < ne; s++) {
    m->perm[s] = keys[s].second;
    m->iperm[keys[s].second] = s;
  }
  m->ncells = (ne + kCell - 1) / kCell;
  m->cell_center.assign(3 * (size_t)m->ncells, 0.0);
  for (int c = 0; c < m->ncells; c++) {
    const int s0 = c * kCell, s1 = std::min(ne, s0 + kCell);
    for (int d = 0; d < 3; d++) {
      double acc = 0.0;
      for (int s = s0; s < s1; s++) acc += cent[3 * m->perm[s] + d];
      m->cell_center[3 * c + d] = acc / (s1 - s0);
    }
  }
  target_split(m->Q, &m->K, &m->nchunk);
  m->nitems = ne * m->nchunk;
  if (topology) host_topology(m);
  return EB_OK;
}

void host_topology(HostMesh* m)
{
  const int nv = m->nv, ne = m->ne;
  // Vertex -> triangles.
  std::vector<int> vptr(nv + 1, 0), vtri(3 * (size_t)ne);
  for (int i = 0; i < 3 * ne; i++) vptr[m->elems[i] + 1]++;
  for (int v = 0; v < nv; v++) vptr[v + 1] += vptr[v];
  {
    std::vector<int> fill(vptr.begin(), vptr.end() - 1);
    for (int i = 0; i < ne; i++)
      for (int k = 0; k < 3; k++) vtri[fill[m->elems[3 * i + k]]++] = i;
  }

  // Near pairs per test triangle (sorted by trial index), DL slots per row.
  m->sl_rowptr.assign(ne + 1, 0);
  m->sl_col.clear();
  m->pair_i.clear();
  m->pair_kind.clear();
  m->dl_rowptr.assign(ne + 1, 0);
  m->dl_col.clear();
  std::vector<int> cand;
  std::vector<std::pair<int, int>> dl_entries;  // (column, entry id)
  long long near_incl_repeat = 0;
  std::vector<int> contrib_ptr(1, 0), contrib;
  for (int i = 0; i < ne; i++) {
    cand.clear();
    for (int k = 0; k < 3; k++) {
      const int v = m->elems[3 * i + k];
      for (int p = vptr[v]; p < vptr[v + 1]; p++) cand.push_back(vtri[p]);
    }
    std::sort(cand.begin(), cand.end());
    cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
    near_incl_repeat += (long long)cand.size();
    dl_entries.clear();
    for (int j : cand) {
      const PairGeom g = classify_pair(&m->elems[3 * i], &m->elems[3 * j], i == j);
      if (g.kind == kPairRepeat) continue;  // a repeated triangle contributes nothing
      const int p = (int)m->sl_col.size();
      m->sl_col.push_back(j);
      m->pair_i.push_back(i);
      m->pair_kind.push_back((int8_t)g.kind);
      if (g.kind == kPairVertex || g.kind == kPairEdge) {
        int slots[3];
        dl_trial_slots(g, slots);
        for (int k = 0; k < 3; k++) dl_entries.push_back({m->elems[3 * j + slots[k]], 3 * p + k});
      }
    }
    m->sl_rowptr[i + 1] = (int)m->sl_col.size();
    std::sort(dl_entries.begin(), dl_entries.end());
    for (size_t e = 0; e < dl_entries.size(); e++) {
      if (e == 0 || dl_entries[e].first != dl_entries[e - 1].first) {
        if (e > 0) contrib_ptr.push_back((int)contrib.size());
        m->dl_col.push_back(dl_entries[e].first);
      }
      contrib.push_back(dl_entries[e].second);
    }
    if (!dl_entries.empty()) contrib_ptr.push_back((int)contrib.size());
    m->dl_rowptr[i + 1] = (int)m->dl_col.size();
  }
  m->dl_contrib_ptr.swap(contrib_ptr);
  m->dl_contrib.swap(contrib);
  m->far_quad_pairs = ((long long)ne * ne - near_incl_repeat) * (long long)m->Q * m->Q;
}

}  // namespace eb
