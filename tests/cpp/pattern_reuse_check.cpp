// Host structure build: a pattern rebuilt into the memory of an earlier one
// (HostPattern::keep_scratch, as a solver context does) must equal a fresh
// build of the same mesh in every field.  Meshes of different sizes and
// kinds are built one after another into one reused pattern: hex8 grids
// with 3 and 1 dofs per node, natural and shuffled node numberings, and a
// quad4 plate with an unused node and a degenerate element (a repeated
// node).  Each mesh is also built single-threaded, which must give the same
// result, and a hash of every field is printed, so that a build compiled with
// BETA_PATTERN_MARK_BUDGET=0 (the bandwidth-sized marker form on every mesh)
// can be compared with the default one.  Every mesh is built a second time
// with column runs allowed (run_request 3, fresh and into a second reused
// pattern), which must keep every field but the column layout and place
// every block where its run says.  Exit code 0 when every build matches.
#include "../../betanoox_b200/csrc/pattern.hpp"

#include <algorithm>
#include <cstdio>
#include <random>
#include <string>
#include <vector>

using betagpu::HostPattern;

template <class A>
static bool same(const A& a, const A& b) {
  return a.size() == b.size() && std::equal(a.begin(), a.end(), b.begin());
}

static bool equal(const HostPattern& P, const HostPattern& Q) {
  return same(P.nrp, Q.nrp) && same(P.ncol, Q.ncol) && same(P.ndiag, Q.ndiag) && P.nblk == Q.nblk &&
         P.ncolor == Q.ncolor && same(P.color_ptr, Q.color_ptr) && same(P.elem_by_color, Q.elem_by_color) &&
         same(P.slot, Q.slot) && P.nslice == Q.nslice && same(P.bsoff, Q.bsoff) && same(P.bcol, Q.bcol) &&
         P.nchunk == Q.nchunk && P.nsslice == Q.nsslice && same(P.ssoff, Q.ssoff) && same(P.scol, Q.scol) &&
         same(P.soff, Q.soff) && same(P.srowlen, Q.srowlen) && same(P.sdiag, Q.sdiag) &&
         P.nnz_full == Q.nnz_full && P.nnz_lower == Q.nnz_lower && P.run == Q.run && same(P.vpos, Q.vpos) &&
         P.compact == Q.compact && same(P.cptr, Q.cptr) && same(P.ccol, Q.ccol);
}

// A build with runs allowed (R) against the one-column-per-block build E of
// the same mesh: the same graph, colouring, slot map and scalar layout; and,
// when runs were chosen, every block (I, q) at a distinct virtual position of
// its row whose run column + offset is its column, the diagonal remapped,
// every run inside the node range.  Prints the run length chosen.
static bool runs_valid(const HostPattern& P, const HostPattern& E, const char* name) {
  bool ok = same(P.nrp, E.nrp) && same(P.ncol, E.ncol) && same(P.slot, E.slot) && same(P.color_ptr, E.color_ptr) &&
            same(P.elem_by_color, E.elem_by_color) && same(P.ssoff, E.ssoff) && same(P.scol, E.scol) &&
            same(P.soff, E.soff) && same(P.sdiag, E.sdiag) && P.nnz_lower == E.nnz_lower && P.nslice == E.nslice;
  if (P.run == 1) {
    ok = ok && equal(P, E);
  } else {
    const int R = P.run;
    ok = ok && (long long)P.vpos.size() == P.nblk && P.nchunk == P.bsoff[P.nslice] &&
         (long long)P.bcol.size() * R == P.nchunk * 32;
    for (int s = 0; ok && s <= P.nslice; ++s) ok = P.bsoff[s] % R == 0;
    for (size_t k = 0; ok && k < P.bcol.size(); ++k) ok = P.bcol[k] >= 0 && P.bcol[k] <= P.nnode - R;
    std::vector<char> seen;
    for (int I = 0; ok && I < P.nnode; ++I) {
      const int s = I / 32, lane = I % 32, w = P.bsoff[s + 1] - P.bsoff[s];
      seen.assign(w, 0);
      for (int q = P.nrp[I]; ok && q < P.nrp[I + 1]; ++q) {
        const int v = P.vpos[q];
        ok = v < w && !seen[v] && P.bcol[((size_t)P.bsoff[s] / R + v / R) * 32 + lane] + v % R == P.ncol[q];
        if (ok) seen[v] = 1;
      }
      ok = ok && P.ndiag[I] == P.vpos[P.nrp[I] + E.ndiag[I]];
    }
    // the compact form gives every lane of every slice the same run columns
    if (ok && P.compact) {
      ok = (int)P.cptr.size() == P.nslice;
      for (int s = 0; ok && s < P.nslice; ++s) {
        const int w = (P.bsoff[s + 1] - P.bsoff[s]) / R;
        for (int k = 0; ok && k < w; ++k)
          for (int lane = 0; ok && lane < 32; ++lane) {
            const int c = P.cptr[s];
            const int j0 = c < 0 ? 32 * s + lane + P.ccol[(size_t)~c + k] : P.ccol[(size_t)c + (size_t)k * 32 + lane];
            ok = j0 == P.bcol[((size_t)P.bsoff[s] / R + k) * 32 + lane];
          }
      }
    }
  }
  std::printf("runs %-55s run=%d compact=%d %s\n", name, P.run, P.compact ? 1 : 0, ok ? "valid" : "INVALID");
  return ok;
}

static unsigned long long hash_of(const HostPattern& P) {
  unsigned long long h = 1469598103934665603ull;
  auto mix = [&](long long v) { h ^= (unsigned long long)v; h *= 1099511628211ull; };
  auto all = [&](const auto& a) { mix((long long)a.size()); for (size_t i = 0; i < a.size(); ++i) mix(a[i]); };
  all(P.nrp); all(P.ncol); all(P.ndiag); all(P.color_ptr); all(P.elem_by_color); all(P.slot); all(P.bsoff);
  all(P.bcol); all(P.ssoff); all(P.scol); all(P.soff); all(P.srowlen); all(P.sdiag); all(P.unused); all(P.vpos);
  all(P.cptr); all(P.ccol);
  mix(P.run);
  mix(P.compact);
  mix(P.nblk); mix(P.ncolor); mix(P.nchunk); mix(P.nnz_full); mix(P.nnz_lower);
  return h;
}

struct Mesh {
  std::string name;
  int nnode = 0, nelem = 0, nnpe = 0, nd = 0;
  std::vector<int> conn;
  std::vector<unsigned char> rest;
};

static Mesh hex8(int n, int nd, bool shuffled, unsigned seed) {
  Mesh M;
  const int m = n + 1;
  M.name = "hex8 n=" + std::to_string(n) + " nd=" + std::to_string(nd) + (shuffled ? " shuffled" : "");
  M.nnode = m * m * m;
  M.nelem = n * n * n;
  M.nnpe = 8;
  M.nd = nd;
  std::vector<int> p(M.nnode);
  for (int i = 0; i < M.nnode; ++i) p[i] = i;
  if (shuffled) {
    std::mt19937 rng(seed);
    std::shuffle(p.begin(), p.end(), rng);
  }
  auto nid = [&](int a, int b, int c) { return p[a + m * (b + m * c)]; };
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        const int c[8] = {nid(i, j, k),     nid(i, j + 1, k),     nid(i, j + 1, k + 1),     nid(i, j, k + 1),
                          nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i + 1, j + 1, k + 1), nid(i + 1, j, k + 1)};
        M.conn.insert(M.conn.end(), c, c + 8);
      }
  M.rest.assign((size_t)M.nnode * nd, 0);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i) M.rest[(size_t)nd * nid(i, j, 0)] = 1;  // first component on z = 0
  return M;
}

static Mesh quad4_with_extras(int nx, int ny) {
  Mesh M;
  const int m = nx + 1;
  M.name = "quad4 " + std::to_string(nx) + "x" + std::to_string(ny) + " + unused node + degenerate element";
  M.nnode = m * (ny + 1) + 1;  // the last node belongs to no element
  M.nelem = nx * ny + 1;
  M.nnpe = 4;
  M.nd = 2;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const int c[4] = {i + m * j, i + 1 + m * j, i + 1 + m * (j + 1), i + m * (j + 1)};
      M.conn.insert(M.conn.end(), c, c + 4);
    }
  const int d[4] = {0, 1, 1, m};  // a repeated node
  M.conn.insert(M.conn.end(), d, d + 4);
  M.rest.assign((size_t)M.nnode * 2, 0);
  for (int j = 0; j <= ny; ++j) M.rest[2 * (m * j)] = M.rest[2 * (m * j) + 1] = 1;
  return M;
}

// The node graph and slot map against their definition, built here the
// plain way (per node: its elements' nodes, sorted and deduplicated): row I
// holds exactly the nodes that share an element with I (I alone for a node
// in no element), ascending; ndiag is I's position in its row (one column per
// block); and slot[e][a][b] is the position of conn[e][b] in row conn[e][a].
static bool graph_semantics(const HostPattern& P, const Mesh& M) {
  std::vector<std::vector<int>> elems(M.nnode);
  for (int e = 0; e < M.nelem; ++e)
    for (int a = 0; a < M.nnpe; ++a) elems[M.conn[(size_t)e * M.nnpe + a]].push_back(e);
  std::vector<int> row;
  for (int I = 0; I < M.nnode; ++I) {
    row.clear();
    for (int e : elems[I])
      row.insert(row.end(), M.conn.begin() + (size_t)e * M.nnpe, M.conn.begin() + (size_t)(e + 1) * M.nnpe);
    if (row.empty()) row.push_back(I);
    std::sort(row.begin(), row.end());
    row.erase(std::unique(row.begin(), row.end()), row.end());
    if ((int)row.size() != P.nrp[I + 1] - P.nrp[I] || !std::equal(row.begin(), row.end(), P.ncol.begin() + P.nrp[I]))
      return false;
    if (P.run == 1 && P.ncol[P.nrp[I] + P.ndiag[I]] != I) return false;
  }
  const int np = M.nnpe * M.nnpe;
  for (int e = 0; e < M.nelem; ++e)
    for (int a = 0; a < M.nnpe; ++a)
      for (int b = 0; b < M.nnpe; ++b) {
        const int I = M.conn[(size_t)e * M.nnpe + a], J = M.conn[(size_t)e * M.nnpe + b];
        const int q = P.slot[(size_t)e * np + a * M.nnpe + b];
        if (q >= P.nrp[I + 1] - P.nrp[I] || P.ncol[P.nrp[I] + q] != J) return false;
      }
  return true;
}

int main() {
  std::vector<Mesh> meshes = {hex8(6, 3, false, 0),  hex8(24, 3, false, 0), hex8(24, 1, true, 3),
                              quad4_with_extras(150, 90), hex8(40, 3, true, 5), hex8(5, 1, false, 0),
                              hex8(24, 3, false, 0),  hex8(70, 1, false, 0)};
  HostPattern reused, reused_runs;
  reused.keep_scratch = true;
  reused_runs.keep_scratch = true;
  reused_runs.run_request = 3;
  int bad = 0;
  for (const Mesh& M : meshes) {
    std::vector<int> fd(M.nnode);
    for (int i = 0; i < M.nnode; ++i) fd[i] = M.nd * i;
    HostPattern fresh;
    const std::string e1 = betagpu::build_pattern(M.nnode, M.nelem, M.nnpe, M.nd, M.conn.data(), fd.data(),
                                                  M.rest.data(), fresh, true);
    const std::string e2 = betagpu::build_pattern(M.nnode, M.nelem, M.nnpe, M.nd, M.conn.data(), fd.data(),
                                                  M.rest.data(), reused, true);
    // the same build on one thread (as the batch engine runs it) must agree:
    // nothing may depend on the thread count or on the concurrent colouring
    HostPattern serial;
    betagpu::pattern_serial_on_this_thread(true);
    const std::string e3 = betagpu::build_pattern(M.nnode, M.nelem, M.nnpe, M.nd, M.conn.data(), fd.data(),
                                                  M.rest.data(), serial, true);
    betagpu::pattern_serial_on_this_thread(false);
#if defined(BETA_PATTERN_MARK_BUDGET) && BETA_PATTERN_MARK_BUDGET == 0
    const bool marks_kept = reused.s_mark.empty();  // nothing node-sized is held
#else
    const bool marks_kept = !reused.s_mark.empty();
#endif
    const bool ok = e1.empty() && e2.empty() && e3.empty() && equal(fresh, reused) && equal(fresh, serial) &&
                    same(fresh.unused, reused.unused) && same(fresh.unused, serial.unused) &&
                    fresh.s_mark.empty() && marks_kept;
    std::printf("%-60s %s\n", M.name.c_str(), ok ? "equal" : "DIFFERENT");
    const bool gok = ok && graph_semantics(fresh, M);
    std::printf("graph %-54s %s\n", M.name.c_str(), gok ? "as defined" : "NOT AS DEFINED");
    bad += gok || !ok ? 0 : 1;
    std::printf("hash %-55s %016llx\n", M.name.c_str(), hash_of(fresh));
    bad += ok ? 0 : 1;
    // the column-run layout, fresh and rebuilt into reused memory
    HostPattern runs;
    runs.run_request = 3;
    const std::string e4 = betagpu::build_pattern(M.nnode, M.nelem, M.nnpe, M.nd, M.conn.data(), fd.data(),
                                                  M.rest.data(), runs, true);
    const std::string e5 = betagpu::build_pattern(M.nnode, M.nelem, M.nnpe, M.nd, M.conn.data(), fd.data(),
                                                  M.rest.data(), reused_runs, true);
    const bool rok = e4.empty() && e5.empty() && runs_valid(runs, fresh, M.name.c_str()) && equal(runs, reused_runs);
    std::printf("hash runs %-50s %016llx\n", M.name.c_str(), hash_of(runs));
    bad += rok ? 0 : 1;
  }
  // invalid input is refused with its message, on any thread count
  {
    Mesh M = hex8(30, 3, false, 0);
    std::vector<int> fd(M.nnode);
    for (int i = 0; i < M.nnode; ++i) fd[i] = M.nd * i;
    HostPattern Q;
    std::vector<int> bad_conn = M.conn;
    bad_conn[bad_conn.size() - 3] = M.nnode;  // one node index past the end, near the end of the list
    const std::string e1 = betagpu::build_pattern(M.nnode, M.nelem, M.nnpe, M.nd, bad_conn.data(), fd.data(),
                                                  M.rest.data(), Q, false);
    std::vector<int> bad_fd = fd;
    bad_fd[M.nnode / 2] += 1;
    const std::string e2 = betagpu::build_pattern(M.nnode, M.nelem, M.nnpe, M.nd, M.conn.data(), bad_fd.data(),
                                                  M.rest.data(), Q, false);
    const bool ok = e1 == "build_pattern: connectivity out of range" &&
                    e2 == "build_pattern: first_dof must be the uniform node-major numbering ndpn*node";
    std::printf("%-60s %s\n", "invalid connectivity and numbering", ok ? "refused" : "NOT REFUSED");
    bad += ok ? 0 : 1;
  }
  return bad ? 1 : 0;
}
