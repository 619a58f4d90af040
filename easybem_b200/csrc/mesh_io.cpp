// Surface mesh ingestion on the host: the two file formats the reference's
// drivers read and its uniform 1->4 refinement (python/examples/
// surface3dMesh.py:51-83 load3dSurface, :86-146 load3dSurfaceFromNetgen,
// :149-221 refineMesh), as C-ABI entry points so that callers without
// Python can build the meshes the reference's drivers use.
//
// All three fill caller-owned arrays. Called with null arrays they only
// report the sizes (a file is read twice; refinement counts the edges).
// Elements are 1-based vertex triples, as everywhere in this ABI.
#include <algorithm>
#include <cctype>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

#include "../../include/easybem_gpu.h"
#include "common.h"

namespace {

using eb::set_error;

struct SurfaceFile {
  std::vector<double> nodes;  // [n][3]
  std::vector<int> elems;     // [m][3], 1-based
  std::vector<int> labels;    // [m]
};

int copy_out(const SurfaceFile& f, int* nnodes, double* nodes, int* nelems, int* elems, int* labels)
{
  const int n = (int)(f.nodes.size() / 3), m = (int)f.labels.size();
  if (nnodes) *nnodes = n;
  if (nelems) *nelems = m;
  if (nodes) std::memcpy(nodes, f.nodes.data(), sizeof(double) * f.nodes.size());
  if (elems) std::memcpy(elems, f.elems.data(), sizeof(int) * f.elems.size());
  if (labels) std::memcpy(labels, f.labels.data(), sizeof(int) * f.labels.size());
  return EB_OK;
}

bool next_nonempty(std::istream& in, std::string& line)
{
  while (std::getline(in, line)) {
    for (char c : line)
      if (!std::isspace((unsigned char)c)) return true;
  }
  return false;
}

std::string lower_trim(const std::string& s)
{
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) a++;
  while (b > a && std::isspace((unsigned char)s[b - 1])) b--;
  std::string r = s.substr(a, b - a);
  for (char& c : r) c = (char)std::tolower((unsigned char)c);
  return r;
}

// load3dSurface: dim, vertices per element, n, n coordinate lines, m, m
// vertex triples, m again, m lines "index label".
int read_txt(const char* path, SurfaceFile& f)
{
  std::ifstream in(path);
  if (!in) return set_error(EB_ERR_INVALID, std::string("cannot open ") + path);
  std::string ln;
  auto bad = [&](const char* what) { return set_error(EB_ERR_INVALID, std::string(path) + ": " + what); };
  int dim = 0, npe = 0, n = 0, m = 0, m2 = 0;
  if (!next_nonempty(in, ln) || !(std::istringstream(ln) >> dim)) return bad("missing dimension");
  if (!next_nonempty(in, ln) || !(std::istringstream(ln) >> npe)) return bad("missing vertices per element");
  if (dim != 3 || npe != 3) return bad("expected a 3-D triangular surface");
  if (!next_nonempty(in, ln) || !(std::istringstream(ln) >> n) || n < 0) return bad("missing vertex count");
  f.nodes.resize((size_t)3 * n);
  for (int i = 0; i < n; i++) {
    std::istringstream s;
    if (!next_nonempty(in, ln)) return bad("too few vertices");
    s.str(ln);
    if (!(s >> f.nodes[3 * i] >> f.nodes[3 * i + 1] >> f.nodes[3 * i + 2])) return bad("bad vertex line");
  }
  if (!next_nonempty(in, ln) || !(std::istringstream(ln) >> m) || m < 0) return bad("missing triangle count");
  f.elems.resize((size_t)3 * m);
  for (int i = 0; i < m; i++) {
    std::istringstream s;
    if (!next_nonempty(in, ln)) return bad("too few triangles");
    s.str(ln);
    if (!(s >> f.elems[3 * i] >> f.elems[3 * i + 1] >> f.elems[3 * i + 2])) return bad("bad triangle line");
  }
  if (!next_nonempty(in, ln) || !(std::istringstream(ln) >> m2)) return bad("missing label count");
  if (m2 != m) return bad("triangle count mismatch");
  f.labels.resize(m);
  for (int i = 0; i < m; i++) {
    std::istringstream s;
    int idx = 0;
    if (!next_nonempty(in, ln)) return bad("too few label lines");
    s.str(ln);
    if (!(s >> idx >> f.labels[i])) return bad("bad label line");
  }
  return EB_OK;
}

// load3dSurfaceFromNetgen: the "points" section (count, then x y z per
// line) and the "surfaceelementsgi" section (count, then
// "surfnr bcnr domin domout np p1 p2 p3 ..." per line, 1-based points).
int read_vol(const char* path, SurfaceFile& f)
{
  std::ifstream in(path);
  if (!in) return set_error(EB_ERR_INVALID, std::string("cannot open ") + path);
  std::vector<std::string> lines;
  std::string ln;
  while (std::getline(in, ln)) lines.push_back(ln);
  auto bad = [&](const std::string& what) { return set_error(EB_ERR_INVALID, std::string(path) + ": " + what); };
  auto find = [&](const char* name) {
    for (size_t i = 0; i < lines.size(); i++)
      if (lower_trim(lines[i]) == name) return (long)i;
    return -1L;
  };
  long i = find("points");
  if (i < 0 || i + 1 >= (long)lines.size()) return bad("section points not found");
  int n = 0;
  if (!(std::istringstream(lines[i + 1]) >> n) || n < 0 || i + 2 + n > (long)lines.size()) return bad("bad point count");
  f.nodes.resize((size_t)3 * n);
  for (int k = 0; k < n; k++) {
    std::istringstream s(lines[i + 2 + k]);
    if (!(s >> f.nodes[3 * k] >> f.nodes[3 * k + 1] >> f.nodes[3 * k + 2])) return bad("bad point line");
  }
  i = find("surfaceelementsgi");
  if (i < 0 || i + 1 >= (long)lines.size()) return bad("section surfaceelementsgi not found");
  int m = 0;
  if (!(std::istringstream(lines[i + 1]) >> m) || m < 0 || i + 2 + m > (long)lines.size())
    return bad("bad surface element count");
  f.elems.resize((size_t)3 * m);
  f.labels.resize(m);
  for (int k = 0; k < m; k++) {
    std::istringstream s(lines[i + 2 + k]);
    int surfnr = 0, bc = 0, din = 0, dout = 0, np = 0;
    if (!(s >> surfnr >> bc >> din >> dout >> np) || np < 3) return bad("bad surface element line");
    if (!(s >> f.elems[3 * k] >> f.elems[3 * k + 1] >> f.elems[3 * k + 2])) return bad("bad surface element line");
    f.labels[k] = surfnr;
  }
  return EB_OK;
}

}  // namespace

extern "C" {

int eb_read_surface_txt(const char* path, int* nnodes, double* nodes, int* nelems, int* elems, int* labels)
{
  if (!path) return set_error(EB_ERR_INVALID, "null path");
  SurfaceFile f;
  EB_CHECK(read_txt(path, f));
  return copy_out(f, nnodes, nodes, nelems, elems, labels);
}

int eb_read_netgen_vol(const char* path, int* nnodes, double* nodes, int* nelems, int* elems, int* labels)
{
  if (!path) return set_error(EB_ERR_INVALID, "null path");
  SurfaceFile f;
  EB_CHECK(read_vol(path, f));
  return copy_out(f, nnodes, nodes, nelems, elems, labels);
}

int eb_mesh_refine(int nnodes, const double* nodes, int nelems, const int* elems, const int* labels,
                   int* nnodes_out, double* nodes_out, int* nelems_out, int* elems_out, int* labels_out)
{
  if (nnodes < 0 || nelems < 0 || (nelems > 0 && !elems) || (nnodes > 0 && !nodes))
    return set_error(EB_ERR_INVALID, "bad mesh arguments");
  if ((long long)nelems * 4 > 0x7fffffffLL) return set_error(EB_ERR_INVALID, "refined mesh too large");
  for (long long k = 0; k < 3LL * nelems; k++)
    if (elems[k] < 1 || elems[k] > nnodes) return set_error(EB_ERR_MESH, "vertex index out of range");
  // undirected edges (sorted endpoints) of every triangle, in the order
  // (v0,v1), (v1,v2), (v2,v0) for all triangles; midpoints numbered after the
  // vertices in lexicographic order of the unique edges
  const long long m = nelems;
  std::vector<std::pair<int, int>> e(3 * m);
  for (long long k = 0; k < m; k++)
    for (int j = 0; j < 3; j++) {
      const int a = elems[3 * k + j] - 1, b = elems[3 * k + (j + 1) % 3] - 1;
      e[j * m + k] = {std::min(a, b), std::max(a, b)};
    }
  std::vector<std::pair<int, int>> u(e);
  std::sort(u.begin(), u.end());
  u.erase(std::unique(u.begin(), u.end()), u.end());
  const long long n2 = (long long)nnodes + (long long)u.size();
  if (n2 > 0x7fffffffLL) return set_error(EB_ERR_INVALID, "refined mesh too large");
  if (nnodes_out) *nnodes_out = (int)n2;
  if (nelems_out) *nelems_out = (int)(4 * m);
  if (nodes_out) {
    std::memcpy(nodes_out, nodes, sizeof(double) * 3 * (size_t)nnodes);
    for (size_t k = 0; k < u.size(); k++)
      for (int c = 0; c < 3; c++)
        nodes_out[3 * (nnodes + k) + c] = 0.5 * (nodes[3 * u[k].first + c] + nodes[3 * u[k].second + c]);
  }
  if (elems_out) {
    auto mid = [&](long long idx) {
      return nnodes + (int)(std::lower_bound(u.begin(), u.end(), e[idx]) - u.begin());
    };
    // children of triangle k at k, m + k, 2m + k, 3m + k (the reference's vstack order)
    for (long long k = 0; k < m; k++) {
      const int i0 = elems[3 * k] - 1, i1 = elems[3 * k + 1] - 1, i2 = elems[3 * k + 2] - 1;
      const int m01 = mid(k), m12 = mid(m + k), m20 = mid(2 * m + k);
      const int tri[4][3] = {{i0, m01, m20}, {m01, i1, m12}, {m20, m12, i2}, {m01, m12, m20}};
      for (int c = 0; c < 4; c++)
        for (int j = 0; j < 3; j++) elems_out[3 * (c * m + k) + j] = tri[c][j] + 1;
    }
  }
  if (labels_out && labels)
    for (long long k = 0; k < m; k++)
      for (int c = 0; c < 4; c++) labels_out[c * m + k] = labels[k];
  return EB_OK;
}

}  // extern "C"
