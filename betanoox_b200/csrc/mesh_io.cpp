// mesh_io.cpp -- BETA's mesh files (host only).
//
// BasicMesh::ReadMesh (BasicMesh.cpp:79-190) and ReadMeshBinary (:192-268)
// read a mesh as:
//   numNodes numElements numDims
//   [processCommands  setCoordinateReadOption xyz|xy|yz|x ...  endCommands]
//   numNodes lines:    nodeNum coordinates (x; x y; y z; or x y z, by the read option)
//   numElements lines: elementNum nnpe node_1 ... node_nnpe
// with node numbers counted from 0 or from 1 (nodeOffset = 1 when the first
// node is numbered 1, BasicElement.cpp:208-226), elements stored under their
// own number.  The binary file holds the same fields as 32-bit ints and
// doubles, every node with x y z (Node::readBinary, node.cpp:113-122).
// Here a mesh is returned as the arrays beta_gpu_mesh_upload takes: xyz
// (nnode x ndim, the read option's coordinates in x, y, z order), and the
// connectivity as 0-based node indices in BETA's local order, elements in
// ascending element number.  Every element must have the same nnpe.
#include "../../include/beta_gpu.h"

#include <algorithm>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

namespace {

struct Mesh {
  int ndim = 0, nnode = 0, nelem = 0, nnpe = 0;
  std::vector<double> xyz;
  std::vector<int> conn;
};

// read option: which of x, y, z a node line carries
enum { kX = 1, kXY = 2, kYZ = 3, kXYZ = 4 };

int finish(std::vector<std::pair<int, std::vector<int>>>& el, const std::vector<int>& nodenum, Mesh& M) {
  // node numbers index the node list after the offset (BasicElement::read)
  const int off = (!nodenum.empty() && nodenum[0] == 1) ? 1 : 0;
  std::stable_sort(el.begin(), el.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
  M.nelem = (int)el.size();
  M.nnpe = el.empty() ? 0 : (int)el[0].second.size();
  M.conn.resize((size_t)M.nelem * M.nnpe);
  for (int e = 0; e < M.nelem; ++e) {
    if ((int)el[e].second.size() != M.nnpe) return BETA_GPU_ERR_UNSUPPORTED;  // mixed element sizes
    if (e > 0 && el[e].first == el[e - 1].first) return BETA_GPU_ERR_ARG;  // duplicate element number
    for (int a = 0; a < M.nnpe; ++a) {
      const int idx = el[e].second[a] - off;
      if (idx < 0 || idx >= M.nnode) return BETA_GPU_ERR_ARG;
      M.conn[(size_t)e * M.nnpe + a] = idx;
    }
  }
  return BETA_GPU_OK;
}

int read_text(const char* path, Mesh& M) {
  std::ifstream is(path);
  if (!is) return BETA_GPU_ERR_ARG;
  int nnode, nelem, ndim;
  if (!(is >> nnode >> nelem >> ndim) || nnode < 0 || nelem < 0) return BETA_GPU_ERR_ARG;
  if (ndim < -3 || ndim > 3 || ndim == 0) return BETA_GPU_ERR_ARG;  // |numDims| in 1..3
  ndim = ndim < 0 ? -ndim : ndim;
  int opt = ndim == 1 ? kX : (ndim == 2 ? kXY : kXYZ);
  // optional command block (BasicMesh.cpp:98-113)
  std::streampos at = is.tellg();
  std::string tok;
  if (is >> tok && tok == "processCommands") {
    while (is >> tok && tok != "endCommands") {
      if (tok == "setCoordinateReadOption" && (is >> tok)) {
        if (tok == "xyz") opt = kXYZ;
        else if (tok == "xy") opt = kXY;
        else if (tok == "yz") opt = kYZ;
        else if (tok == "x") opt = kX;
      }
    }
    if (tok != "endCommands") return BETA_GPU_ERR_ARG;
  } else {
    is.clear();
    is.seekg(at);
  }
  M.ndim = ndim;
  M.nnode = nnode;
  M.xyz.assign((size_t)nnode * ndim, 0.0);
  std::vector<int> nodenum(nnode);
  for (int i = 0; i < nnode; ++i) {
    double x = 0, y = 0, z = 0;
    if (!(is >> nodenum[i])) return BETA_GPU_ERR_ARG;
    bool ok = true;
    switch (opt) {
      case kX: ok = (bool)(is >> x); break;
      case kXY: ok = (bool)(is >> x >> y); break;
      case kYZ: ok = (bool)(is >> y >> z); break;
      default: ok = (bool)(is >> x >> y >> z); break;
    }
    if (!ok) return BETA_GPU_ERR_ARG;
    const double c[3] = {x, y, z};
    for (int d = 0; d < ndim; ++d) M.xyz[(size_t)i * ndim + d] = c[d];
  }
  std::vector<std::pair<int, std::vector<int>>> el(nelem);
  for (int e = 0; e < nelem; ++e) {
    int num, nnpe;
    if (!(is >> num >> nnpe) || nnpe < 1 || nnpe > 64) return BETA_GPU_ERR_ARG;
    el[e].first = num;
    el[e].second.resize(nnpe);
    for (int a = 0; a < nnpe; ++a)
      if (!(is >> el[e].second[a])) return BETA_GPU_ERR_ARG;
  }
  return finish(el, nodenum, M);
}

int read_binary(const char* path, Mesh& M) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return BETA_GPU_ERR_ARG;
  auto rd = [&](void* p, size_t sz, size_t n) { return std::fread(p, sz, n, f) == n; };
  int nnode, nelem, ndim;
  int rc = BETA_GPU_ERR_ARG;
  std::vector<int> nodenum;
  std::vector<std::pair<int, std::vector<int>>> el;
  if (rd(&nnode, sizeof(int), 1) && rd(&nelem, sizeof(int), 1) && rd(&ndim, sizeof(int), 1) && nnode >= 0 &&
      nelem >= 0 && ndim != 0 && ndim >= -3 && ndim <= 3) {
    ndim = ndim < 0 ? -ndim : ndim;
    M.ndim = ndim;
    M.nnode = nnode;
    M.xyz.assign((size_t)nnode * ndim, 0.0);
    nodenum.resize(nnode);
    bool ok = true;
    for (int i = 0; i < nnode && ok; ++i) {
      double c[3];
      ok = rd(&nodenum[i], sizeof(int), 1) && rd(c, sizeof(double), 3);
      for (int d = 0; d < ndim && ok; ++d) M.xyz[(size_t)i * ndim + d] = c[d];
    }
    el.resize(nelem);
    for (int e = 0; e < nelem && ok; ++e) {
      int nnpe = 0;
      ok = rd(&el[e].first, sizeof(int), 1) && rd(&nnpe, sizeof(int), 1) && nnpe >= 1 && nnpe <= 64;
      if (ok) {
        el[e].second.resize(nnpe);
        ok = rd(el[e].second.data(), sizeof(int), nnpe);
      }
    }
    if (ok) rc = finish(el, nodenum, M);
  }
  std::fclose(f);
  return rc;
}

}  // namespace

extern "C" {

BETA_GPU_API int beta_gpu_read_mesh(const char* path, int binary, int* ndim, int* nnode, int* nelem, int* nnpe,
                                    double* xyz, int* conn) {
  if (!path || !ndim || !nnode || !nelem || !nnpe) return BETA_GPU_ERR_ARG;
  Mesh M;
  const int rc = binary ? read_binary(path, M) : read_text(path, M);
  if (rc != BETA_GPU_OK) return rc;
  *ndim = M.ndim;
  *nnode = M.nnode;
  *nelem = M.nelem;
  *nnpe = M.nnpe;
  if (xyz) std::copy(M.xyz.begin(), M.xyz.end(), xyz);
  if (conn) std::copy(M.conn.begin(), M.conn.end(), conn);
  return BETA_GPU_OK;
}

BETA_GPU_API int beta_gpu_write_mesh(const char* path, int binary, int ndim, int nnode, const double* xyz, int nelem,
                                     int nnpe, const int* conn, int first_number) {
  if (!path || ndim < 1 || ndim > 3 || nnode < 0 || nelem < 0 || nnpe < 1 || (nnode && !xyz) ||
      (nelem && !conn) || (first_number != 0 && first_number != 1))
    return BETA_GPU_ERR_ARG;
  if (binary) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return BETA_GPU_ERR_ARG;
    bool ok = std::fwrite(&nnode, sizeof(int), 1, f) == 1 && std::fwrite(&nelem, sizeof(int), 1, f) == 1 &&
              std::fwrite(&ndim, sizeof(int), 1, f) == 1;
    for (int i = 0; i < nnode && ok; ++i) {
      const int num = i + first_number;
      double c[3] = {0, 0, 0};
      for (int d = 0; d < ndim; ++d) c[d] = xyz[(size_t)i * ndim + d];
      ok = std::fwrite(&num, sizeof(int), 1, f) == 1 && std::fwrite(c, sizeof(double), 3, f) == 3;
    }
    for (int e = 0; e < nelem && ok; ++e) {
      const int num = e + first_number;
      ok = std::fwrite(&num, sizeof(int), 1, f) == 1 && std::fwrite(&nnpe, sizeof(int), 1, f) == 1;
      for (int a = 0; a < nnpe && ok; ++a) {
        const int nd = conn[(size_t)e * nnpe + a] + first_number;
        ok = std::fwrite(&nd, sizeof(int), 1, f) == 1;
      }
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? BETA_GPU_OK : BETA_GPU_ERR_ARG;
  }
  std::ofstream os(path);
  if (!os) return BETA_GPU_ERR_ARG;
  os.precision(17);
  os << nnode << " " << nelem << " " << ndim << '\n';
  for (int i = 0; i < nnode; ++i) {
    os << i + first_number;
    for (int d = 0; d < ndim; ++d) os << " " << xyz[(size_t)i * ndim + d];
    os << '\n';
  }
  for (int e = 0; e < nelem; ++e) {
    os << e + first_number << " " << nnpe;
    for (int a = 0; a < nnpe; ++a) os << " " << conn[(size_t)e * nnpe + a] + first_number;
    os << '\n';
  }
  return os ? BETA_GPU_OK : BETA_GPU_ERR_ARG;
}

}  // extern "C"
