// pattern.cpp -- host-side integer structure (see pattern.hpp).
#include "pattern.hpp"

#include <algorithm>
#include <cstring>
#include <functional>
#include <thread>

namespace betagpu {

static thread_local bool t_serial = false;

void pattern_serial_on_this_thread(bool on) { t_serial = on; }

// Number of contiguous chunks parallel_chunks splits n items into.
// Bytes the node-sized marker arrays of the node-graph passes may take in all
// (a test build sets 0 to run the bandwidth-sized form on every mesh, and
// BETA_PATTERN_SPAN_CAP=0 as well to sort and deduplicate every row).
#ifndef BETA_PATTERN_MARK_BUDGET
#define BETA_PATTERN_MARK_BUDGET (512LL << 20)
#endif

static int chunk_count(long long n) {
  unsigned hw = std::thread::hardware_concurrency();
  int t = (int)std::min<unsigned>(hw ? hw : 1, 64);
  return (t_serial || n < 20000 || t <= 1) ? 1 : t;
}

// body(chunk, lo, hi) over t contiguous ranges of [0, n), one thread each.
static void parallel_chunks_n(int t, long long n, const std::function<void(int, long long, long long)>& body) {
  if (t <= 1) { body(0, 0, n); return; }
  std::vector<std::thread> th;
  for (int k = 0; k < t; ++k) th.emplace_back(body, k, n * k / t, n * (k + 1) / t);
  for (auto& x : th) x.join();
}

// body(chunk, lo, hi) over chunk_count(n) contiguous ranges, one thread each.
static void parallel_chunks(long long n, const std::function<void(int, long long, long long)>& body) {
  parallel_chunks_n(chunk_count(n), n, body);
}

static void parallel_for(long long n, const std::function<void(long long, long long)>& body) {
  parallel_chunks(n, [&](int, long long lo, long long hi) { body(lo, hi); });
}

// Empties every output of P but keeps the memory of its vectors.
static void reset_keep(HostPattern& P) {
  P.nnode = P.nelem = P.nnpe = P.ndpn = P.ndof = 0;
  for (auto* v : {&P.nrp, &P.ndiag, &P.color_ptr, &P.elem_by_color, &P.bsoff, &P.soff, &P.srowlen, &P.unused})
    v->clear();
  P.scol.clear();
  P.ncol.clear();
  P.bcol.clear();
  P.vpos.clear();
  P.run = 1;
  P.compact = false;
  P.cptr.clear();
  P.ccol.clear();
  P.slot.clear();
  P.ssoff.clear();
  P.sdiag.clear();
  P.nblk = P.nchunk = P.nnz_full = P.nnz_lower = 0;
  P.ncolor = P.nslice = P.nsslice = 0;
}

static void release_scratch(HostPattern& P) {
  if (P.keep_scratch) return;
  std::vector<int>().swap(P.s_icnt);
  std::vector<int>().swap(P.s_inc);
  std::vector<int>().swap(P.s_ccnt);
  std::vector<int>().swap(P.s_color);
  std::vector<int>().swap(P.s_ufree);
  std::vector<uint64_t>().swap(P.s_used);
  std::vector<std::vector<int>>().swap(P.s_mark);
  std::vector<FillVec<int>>().swap(P.s_rows);
}

// Column storage of the node-block layout for a caller that accepts runs
// (P.run_request = R > 1): one column index per run of up to R consecutive
// node columns when that makes the FP32 matrix (values + columns) at least
// 5 % smaller than one index per block, else one per block.  The rows are
// in ncol; ndiag holds graph positions on entry and virtual ones on exit.
// A row's runs are formed greedily over its ascending columns: a run starts
// at the first column not yet covered (moved back to nnode - R at the end of
// the node range, so its R gathers stay in bounds) and covers every column
// below its start + R.  The runs of a row ascend, so the SpMV visits the
// non-zero blocks in the same column order as the one-index layout and
// adds exact zeros between them.
static void build_columns(HostPattern& P) {
  const int nnode = P.nnode, R = P.run_request, bb = P.ndpn * P.ndpn;
  P.run = 1;
  P.vpos.clear();
  auto runs_of = [&](long long i, auto&& emit) {
    const int q0 = P.nrp[i], len = P.nrp[i + 1] - q0;
    const int* c = P.ncol.data() + q0;
    int m = 0;
    for (int k = 0; k < len; ++m) {
      const int s0 = std::min(c[k], nnode - R);
      emit(m, s0);
      for (; k < len && c[k] < s0 + R; ++k) P.vpos[q0 + k] = (uint16_t)(R * m + (c[k] - s0));
    }
    return m;
  };
  std::vector<int> wr(P.nslice, 0);
  if (nnode >= R) {
    parallel_for(P.nslice, [&](long long lo, long long hi) {
      for (long long s = lo; s < hi; ++s) {
        int w = 0;
        for (long long i = s * 32; i < std::min<long long>(nnode, s * 32 + 32); ++i) {
          const int q0 = P.nrp[i], len = P.nrp[i + 1] - q0;
          const int* c = P.ncol.data() + q0;
          int m = 0;
          for (int k = 0; k < len; ++m) {
            const int s0 = std::min(c[k], nnode - R);
            while (k < len && c[k] < s0 + R) ++k;
          }
          w = std::max(w, m);
        }
        wr[s] = w;
      }
    });
  }
  long long nrc = 0;
  int wmax = 0;
  for (int w : wr) {
    nrc += w;
    wmax = std::max(wmax, w);
  }
  const double run_bytes = (double)nrc * 32 * (4.0 + 4.0 * R * bb);
  const double ell_bytes = (double)P.nchunk * 32 * (4.0 + 4.0 * bb);
  const bool use_runs = nnode >= R && (long long)R * wmax <= 65535 && R * nrc * 32LL * bb <= 2000000000LL &&
                        run_bytes <= 0.95 * ell_bytes;
  if (!use_runs) {
    P.bcol.resize((size_t)P.nchunk * 32);
    parallel_for(P.nslice, [&](long long lo, long long hi) {
      for (long long s = lo; s < hi; ++s) {
        const int w = P.bsoff[s + 1] - P.bsoff[s];
        for (int l = 0; l < 32; ++l) {
          const long long i = s * 32 + l;
          int* bc = P.bcol.data() + (size_t)P.bsoff[s] * 32 + l;
          int k = 0;
          if (i < nnode)
            for (int q = P.nrp[i]; q < P.nrp[i + 1]; ++q, ++k) bc[(size_t)k * 32] = P.ncol[q];
          for (; k < w; ++k) bc[(size_t)k * 32] = i < nnode ? (int)i : 0;
        }
      }
    });
    return;
  }
  P.run = R;
  P.compact = false;
  P.cptr.clear();
  P.ccol.clear();
  for (int s = 0; s < P.nslice; ++s) P.bsoff[s + 1] = P.bsoff[s] + R * wr[s];
  P.nchunk = P.bsoff[P.nslice];
  P.bcol.resize((size_t)nrc * 32);
  P.vpos.resize((size_t)P.nblk);
  parallel_for(P.nslice, [&](long long lo, long long hi) {
    for (long long s = lo; s < hi; ++s) {
      const long long r0 = P.bsoff[s] / R;
      const int w = wr[s];
      for (int l = 0; l < 32; ++l) {
        const long long i = s * 32 + l;
        int* bc = P.bcol.data() + (size_t)r0 * 32 + l;
        int m = 0;
        if (i < nnode) {
          m = runs_of(i, [&](int k, int s0) { bc[(size_t)k * 32] = s0; });
          P.ndiag[i] = P.vpos[P.nrp[i] + P.ndiag[i]];
        }
        const int pad = i < nnode ? std::min((int)i, nnode - R) : 0;
        for (; m < w; ++m) bc[(size_t)m * 32] = pad;
      }
    }
  });
  if (!P.compact_request) return;
  // the compact form: slices whose every run sits at one offset from the row
  std::vector<char> uni(P.nslice, 0);
  parallel_for(P.nslice, [&](long long lo, long long hi) {
    for (long long s = lo; s < hi; ++s) {
      if ((s + 1) * 32 > nnode) continue;  // a partial last slice keeps its columns
      const int* c = P.bcol.data() + (size_t)(P.bsoff[s] / R) * 32;
      bool u = true;
      for (int k = 0; k < wr[s] && u; ++k) {
        const int off = c[(size_t)k * 32] - (int)(s * 32);
        for (int l = 1; l < 32; ++l)
          if (c[(size_t)k * 32 + l] - (int)(s * 32 + l) != off) {
            u = false;
            break;
          }
      }
      uni[s] = u ? 1 : 0;
    }
  });
  long long full = 0, small = 0;
  for (int s = 0; s < P.nslice; ++s) (uni[s] ? small : full) += wr[s];
  const double before = (double)nrc * 32 * 4, after = (double)(full * 32 + small + P.nslice) * 4;
  const double values = (double)P.nchunk * 32 * 4.0 * bb;
  if (before - after < 0.02 * (values + before) || full * 32 + small > 2000000000LL) return;
  P.cptr.resize(P.nslice);
  long long at = 0;
  for (int s = 0; s < P.nslice; ++s) {
    P.cptr[s] = uni[s] ? ~(int)at : (int)at;
    at += uni[s] ? wr[s] : 32LL * wr[s];
  }
  P.ccol.resize((size_t)at);
  parallel_for(P.nslice, [&](long long lo, long long hi) {
    for (long long s = lo; s < hi; ++s) {
      const int* c = P.bcol.data() + (size_t)(P.bsoff[s] / R) * 32;
      if (P.cptr[s] < 0) {
        int* d = P.ccol.data() + ~P.cptr[s];
        for (int k = 0; k < wr[s]; ++k) d[k] = c[(size_t)k * 32] - (int)(s * 32);
      } else {
        std::copy(c, c + (size_t)wr[s] * 32, P.ccol.begin() + P.cptr[s]);
      }
    }
  });
  P.compact = true;
}

std::string build_pattern(int nnode, int nelem, int nnpe, int ndpn, const int* conn,
                          const int* first_dof, const unsigned char* rest, HostPattern& P, bool with_scalar) {
  if (nnode <= 0 || nelem <= 0 || nnpe <= 0 || nnpe > 8 || ndpn < 1 || ndpn > 3)
    return "build_pattern: bad sizes";
  {
    bool bad_dof = false, bad_conn = false;  // each set only to true, by any thread
    parallel_for(nnode, [&](long long lo, long long hi) {
      bool bad = false;
      for (long long i = lo; i < hi; ++i) bad |= first_dof[i] != ndpn * (int)i;
      if (bad) __atomic_store_n(&bad_dof, true, __ATOMIC_RELAXED);
    });
    parallel_for((long long)nelem * nnpe, [&](long long lo, long long hi) {
      bool bad = false;
      for (long long k = lo; k < hi; ++k) bad |= conn[k] < 0 || conn[k] >= nnode;
      if (bad) __atomic_store_n(&bad_conn, true, __ATOMIC_RELAXED);
    });
    if (bad_dof) return "build_pattern: first_dof must be the uniform node-major numbering ndpn*node";
    if (bad_conn) return "build_pattern: connectivity out of range";
  }
  reset_keep(P);
  P.nnode = nnode; P.nelem = nelem; P.nnpe = nnpe; P.ndpn = ndpn; P.ndof = nnode * ndpn;

  // ---- greedy element colouring (one 64-bit colour mask per node) ----
  // Serial (each element's colour depends on the ones before it) and
  // independent of the node graph, so it runs on its own thread while the
  // graph passes below use the others.  It writes only its own outputs.
  std::string colour_err;
  auto colour = [&]() {
    std::vector<uint64_t>& used = P.s_used;
    used.assign(nnode, 0);
    std::vector<int>& color = P.s_color;
    color.resize(nelem);
    int maxc = 0;
    for (int e = 0; e < nelem; ++e) {
      const int* ce = conn + (long long)e * nnpe;
      uint64_t m = 0;
      for (int a = 0; a < nnpe; ++a) m |= used[ce[a]];
      if (m == ~0ULL) {
        colour_err = "build_pattern: more than 64 element colours";
        return;
      }
      int c = __builtin_ctzll(~m);
      color[e] = c;
      maxc = std::max(maxc, c + 1);
      for (int a = 0; a < nnpe; ++a) used[ce[a]] |= (1ULL << c);
    }
    P.ncolor = maxc;
    P.color_ptr.assign(maxc + 1, 0);
    for (int e = 0; e < nelem; ++e) P.color_ptr[color[e] + 1]++;
    for (int c = 0; c < maxc; ++c) P.color_ptr[c + 1] += P.color_ptr[c];
    P.elem_by_color.resize(nelem);
    std::vector<int> fill(P.color_ptr.begin(), P.color_ptr.end() - 1);
    for (int e = 0; e < nelem; ++e) P.elem_by_color[fill[color[e]]++] = e;
  };
  struct Joiner {  // the colouring thread is joined on every way out
    std::thread t;
    ~Joiner() {
      if (t.joinable()) t.join();
    }
  } colouring;
  if (chunk_count(nelem) > 1)
    colouring.t = std::thread(colour);
  else
    colour();

  // ---- node -> element incidence -------------------------------------
  // A counting sort by node with one count array per element chunk (no
  // atomics): chunk t counts its entries per node, the counts become
  // per-chunk offsets within each node's list, and chunk t fills its part in
  // element order, so every node's elements come out ascending.  The
  // chunks are at most the mean entries per node, so the count arrays never
  // outgrow the incidence list itself.
  std::vector<int>& icnt = P.s_icnt;
  icnt.assign(nnode + 1, 0);
  const int nec = (int)std::max(1LL, std::min<long long>(chunk_count(nelem), (long long)nelem * nnpe / nnode));
  std::vector<int>& ccnt = P.s_ccnt;
  ccnt.resize((size_t)nec * nnode);
  parallel_chunks_n(nec, nelem, [&](int t, long long e0, long long e1) {
    int* c = ccnt.data() + (size_t)t * nnode;
    std::fill(c, c + nnode, 0);
    for (long long k = e0 * nnpe; k < e1 * nnpe; ++k) ++c[conn[k]];
  });
  parallel_for(nnode, [&](long long lo, long long hi) {
    for (long long i = lo; i < hi; ++i) {
      int s = 0;
      for (int t = 0; t < nec; ++t) {
        int& c = ccnt[(size_t)t * nnode + i];
        const int v = c;
        c = s;
        s += v;
      }
      icnt[i + 1] = s;
    }
  });
  for (int i = 0; i < nnode; ++i) icnt[i + 1] += icnt[i];
  std::vector<int>& inc = P.s_inc;
  inc.resize(icnt[nnode]);
  parallel_chunks_n(nec, nelem, [&](int t, long long e0, long long e1) {
    int* c = ccnt.data() + (size_t)t * nnode;
    for (long long k = e0 * nnpe; k < e1 * nnpe; ++k) {
      const int i = conn[k];
      inc[icnt[i] + c[i]++] = (int)(k / nnpe);
    }
  });

  P.unused.clear();
  for (int i = 0; i < nnode; ++i)
    if (icnt[i] == icnt[i + 1]) P.unused.push_back(i);

  // free dofs per node, for the reference's lower-triangle count below
  std::vector<int>& ufree = P.s_ufree;
  ufree.resize(nnode);
  parallel_for(nnode, [&](long long lo, long long hi) {
    for (long long I = lo; I < hi; ++I) {
      int f = 0;
      for (int j = 0; j < ndpn; ++j) f += rest[ndpn * I + j] ? 0 : 1;
      ufree[I] = f;
    }
  });

  // ---- node graph: one pass over the rows, then their columns placed ----
  // Neighbours of node i are deduplicated with a marker array (mark[J - lo]
  // == i + 1 once J is taken), so only the distinct ones are sorted.  Each
  // chunk of rows has its own marker and position arrays: node-sized ones
  // (kept between builds of a solver context) while all of them fit in
  // kMarkBudget bytes; beyond that each chunk marks within the span of node
  // ids its rows reach, which follows the numbering's bandwidth, and a chunk
  // whose span is still wider than kSpanCap sorts and deduplicates each row
  // instead.
  struct Span { int lo = 0, hi = -1; };
  const int nck = chunk_count(nnode);
  constexpr long long kMarkBudget = BETA_PATTERN_MARK_BUDGET;
  const bool node_sized = 2LL * nck * nnode * (long long)sizeof(int) <= kMarkBudget;
#ifdef BETA_PATTERN_SPAN_CAP
  const long long kSpanCap = BETA_PATTERN_SPAN_CAP;  // a test build: 0 sorts every row
#else
  const long long kSpanCap = 4LL * ((nnode + nck - 1) / nck) + 65536;
#endif
  if (node_sized) {
    P.s_mark.resize(2 * nck);  // per chunk: the marker, and the positions of the current row
  } else {
    std::vector<std::vector<int>>().swap(P.s_mark);
  }
  auto collect = [&](int i, std::vector<int>& buf, int* mark, int lo, int stamp) {
    buf.clear();
    for (int k = icnt[i]; k < icnt[i + 1]; ++k) {
      const int* ce = conn + (long long)inc[k] * nnpe;
      if (mark) {
        for (int a = 0; a < nnpe; ++a) {
          const int J = ce[a];
          if (mark[J - lo] != stamp) {
            mark[J - lo] = stamp;
            buf.push_back(J);
          }
        }
      } else {
        buf.insert(buf.end(), ce, ce + nnpe);
      }
    }
    if (buf.empty()) buf.push_back(i);  // a node in no element keeps its diagonal
    if (buf.size() <= 64) {  // the usual row (27 nodes for hex8): insertion sort, about 6 % off the build
      int* v = buf.data();
      const int len = (int)buf.size();
      for (int k = 1; k < len; ++k) {
        const int t = v[k];
        int j = k - 1;
        while (j >= 0 && v[j] > t) {
          v[j + 1] = v[j];
          --j;
        }
        v[j + 1] = t;
      }
    } else {
      std::sort(buf.begin(), buf.end());
    }
    if (!mark) buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
  };

  // The row pass collects each node row i (sorted) once, keeps it in its
  // chunk's buffer P.s_rows[ck] (rows lo..hi back to back) and writes from it:
  //   * the row length into nrp[i + 1], and ndiag;
  //   * the element -> node-pair block map: with pos[J] = J's position in
  //     row i, each incident element (e, a) with conn[e][a] == i gets
  //     slot[e][a][b] = pos[conn[e][b]] (every node of the element is in the
  //     row); each (e, a) belongs to one row, so the writes do not overlap;
  //   * the reference's lower-triangle count of its dof rows: a free row
  //     r = I*ndpn + i holds the free dofs c <= r of its node row (all free
  //     dofs of the neighbours J < I -- those before the diagonal -- and the
  //     free dofs j <= i of I itself); a restrained row holds its diagonal.
  // After the prefix over nrp the place pass copies each chunk's rows into
  // ncol (one contiguous range per chunk; both passes split the rows into
  // the same chunks) and, with one column per block, each row into its lane
  // of the node-block sliced ELL, padded to the slice width with the row's
  // own node.
  P.nrp.assign(nnode + 1, 0);
  P.ndiag.resize(nnode);
  const int npair = nnpe * nnpe;
  P.slot.resize((size_t)nelem * npair);
  if ((int)P.s_rows.size() < nck) P.s_rows.resize(nck);
  std::vector<long long> lower(nck, 0);
  parallel_chunks(nnode, [&](int ck, long long lo, long long hi) {
    std::vector<int> buf, local, local_pos;
    FillVec<int>& rows = P.s_rows[ck];
    rows.clear();
    int *mark = nullptr, *pos = nullptr;
    Span sp{0, nnode - 1};
    if (node_sized) {
      P.s_mark[ck].assign(nnode, 0);
      std::vector<int>& pv = P.s_mark[nck + ck];
      if ((long long)pv.size() < nnode) pv.resize(nnode);
      mark = P.s_mark[ck].data();
      pos = pv.data();
    } else {
      sp = Span{(int)lo, (int)hi - 1};
      for (long long i = lo; i < hi; ++i)
        for (int k = icnt[i]; k < icnt[i + 1]; ++k) {
          const int* ce = conn + (long long)inc[k] * nnpe;
          for (int a = 0; a < nnpe; ++a) {
            sp.lo = std::min(sp.lo, ce[a]);
            sp.hi = std::max(sp.hi, ce[a]);
          }
        }
      if ((long long)sp.hi - sp.lo + 1 <= kSpanCap) {
        local.assign((size_t)(sp.hi - sp.lo + 1), 0);
        local_pos.resize((size_t)(sp.hi - sp.lo + 1));
        mark = local.data();
        pos = local_pos.data();
      }
    }
    long long acc = 0;
    for (long long i = lo; i < hi; ++i) {
      collect((int)i, buf, mark, sp.lo, (int)i + 1);
      const int len = (int)buf.size();
      rows.insert(rows.end(), buf.begin(), buf.end());
      P.nrp[i + 1] = len;
      const int d = (int)(std::lower_bound(buf.begin(), buf.end(), (int)i) - buf.begin());
      P.ndiag[i] = d;
      if (pos)
        for (int k = 0; k < len; ++k) pos[buf[k] - sp.lo] = k;
      for (int k = icnt[i]; k < icnt[i + 1]; ++k) {
        const long long e = inc[k];
        const int* ce = conn + e * nnpe;
        for (int a = 0; a < nnpe; ++a) {
          if (ce[a] != (int)i) continue;
          uint16_t* sl = P.slot.data() + e * npair + a * nnpe;
          for (int b = 0; b < nnpe; ++b)  // J's position in the sorted row
            sl[b] = (uint16_t)(pos ? pos[ce[b] - sp.lo]
                                   : std::lower_bound(buf.begin(), buf.end(), ce[b]) - buf.begin());
        }
      }
      if (icnt[i] == icnt[i + 1]) {  // a node in no element: its rows hold the diagonal alone
        acc += ndpn;
        continue;
      }
      long long below = 0;
      for (int k = 0; k < d; ++k) below += ufree[buf[k]];
      int own = 0;
      for (int j = 0; j < ndpn; ++j) {
        if (rest[i * ndpn + j]) {
          acc += 1;
        } else {
          ++own;
          acc += below + own;
        }
      }
    }
    lower[ck] = acc;
  });
  for (int i = 0; i < nnode; ++i) {
    if (P.nrp[i + 1] > 65535) return "build_pattern: a node with more than 65535 neighbours";
    if ((long long)P.nrp[i] + P.nrp[i + 1] > 2000000000LL) return "build_pattern: node graph too large";
    P.nrp[i + 1] += P.nrp[i];
  }
  P.nblk = P.nrp[nnode];

  // ---- node-block sliced ELL: slice widths from the row lengths -------
  P.nslice = (nnode + 31) / 32;
  P.bsoff.assign(P.nslice + 1, 0);
  for (int s = 0; s < P.nslice; ++s) {
    int w = 0;
    for (int i = s * 32; i < std::min(nnode, s * 32 + 32); ++i) w = std::max(w, P.nrp[i + 1] - P.nrp[i]);
    P.bsoff[s + 1] = P.bsoff[s] + w;
  }
  P.nchunk = P.bsoff[P.nslice];
  if (P.nchunk * 32LL * ndpn * ndpn > 2000000000LL) return "build_pattern: block layout exceeds 2^31 entries";

  // ---- place pass --------------------------------------------------------
  P.ncol.resize(P.nblk);
  // with runs requested the columns are laid out after this pass (build_columns)
  const bool ell_now = P.run_request <= 1;
  if (ell_now) P.bcol.resize((size_t)P.nchunk * 32);
  parallel_chunks(nnode, [&](int ck, long long lo, long long hi) {
    const int* row = P.s_rows[ck].data();
    std::copy(row, row + (P.nrp[hi] - P.nrp[lo]), P.ncol.begin() + P.nrp[lo]);
    if (!ell_now) return;
    for (long long i = lo; i < hi; ++i) {
      const int len = P.nrp[i + 1] - P.nrp[i];
      const int* r = row + (P.nrp[i] - P.nrp[lo]);
      const long long s = i / 32;
      const int w = P.bsoff[s + 1] - P.bsoff[s];
      int* bc = P.bcol.data() + (size_t)P.bsoff[s] * 32 + (i % 32);
      for (int k = 0; k < len; ++k) bc[(size_t)k * 32] = r[k];
      for (int k = len; k < w; ++k) bc[(size_t)k * 32] = (int)i;
    }
  });
  // the row buffers (nblk ints in all) stay for the next build of a solver
  // context only within the marker budget
  if (!P.keep_scratch || (long long)P.nblk * (long long)sizeof(int) > kMarkBudget)
    std::vector<FillVec<int>>().swap(P.s_rows);
  // lanes past the last node in the last slice
  if (ell_now) {
    for (int i = nnode; i < P.nslice * 32; ++i) {
      const int s = i / 32, w = P.bsoff[s + 1] - P.bsoff[s];
      for (int k = 0; k < w; ++k) P.bcol[(size_t)(P.bsoff[s] + k) * 32 + (i % 32)] = 0;
    }
  } else {
    build_columns(P);
  }
  P.nnz_lower = 0;
  for (long long v : lower) P.nnz_lower += v;

  if (colouring.t.joinable()) colouring.t.join();
  if (!colour_err.empty()) return colour_err;
  if (!with_scalar) {
    release_scratch(P);
    return "";
  }
  std::string msg = build_scalar(P, rest);
  release_scratch(P);
  return msg;
}

static bool node_unused(const HostPattern& P, int I) {
  return !P.unused.empty() && std::binary_search(P.unused.begin(), P.unused.end(), I);
}

std::string build_scalar(HostPattern& P, const unsigned char* rest) {
  const int nnode = P.nnode, ndpn = P.ndpn;
  const int ndof = P.ndof;
  std::vector<int> ufree(nnode, 0);
  for (int i = 0; i < nnode; ++i)
    for (int j = 0; j < ndpn; ++j) ufree[i] += rest[ndpn * i + j] ? 0 : 1;
  P.soff.resize(P.nblk);
  std::vector<int> nodelen(nnode);
  parallel_for(nnode, [&](long long lo, long long hi) {
    for (long long i = lo; i < hi; ++i) {
      int acc = 0;
      for (int k = P.nrp[i]; k < P.nrp[i + 1]; ++k) { P.soff[k] = acc; acc += ufree[P.ncol[k]]; }
      nodelen[i] = acc;
    }
  });
  P.srowlen.resize(ndof);
  P.nsslice = (ndof + 31) / 32;
  P.ssoff.assign(P.nsslice + 1, 0);
  // row lengths, per-slice widths (in ssoff[s+1]) and the nonzero count, by
  // slices on all threads; then the prefix over slices
  std::vector<long long> part(chunk_count(P.nsslice), 0);
  parallel_chunks(P.nsslice, [&](int ck, long long lo, long long hi) {
    long long acc = 0;
    for (long long s = lo; s < hi; ++s) {
      int w = 0;
      for (int r = (int)s * 32; r < std::min(ndof, (int)s * 32 + 32); ++r) {
        const int len = (rest[r] || node_unused(P, r / ndpn)) ? 1 : nodelen[r / ndpn];
        P.srowlen[r] = len;
        acc += len;
        w = std::max(w, len);
      }
      P.ssoff[s + 1] = (long long)w * 32;
    }
    part[ck] = acc;
  });
  P.nnz_full = 0;
  for (long long v : part) P.nnz_full += v;
  for (int s = 0; s < P.nsslice; ++s) P.ssoff[s + 1] += P.ssoff[s];
  if (P.ssoff[P.nsslice] > 2000000000LL) return "build_pattern: scalar layout exceeds 2^31 entries";
  P.scol.resize(P.ssoff[P.nsslice]);  // every lane is written below, padding included
  P.sdiag.assign(ndof, 0);
  parallel_for(P.nsslice, [&](long long lo, long long hi) {
    for (long long s = lo; s < hi; ++s) {
      int w = (int)((P.ssoff[s + 1] - P.ssoff[s]) / 32);
      for (int lane = 0; lane < 32; ++lane) {
        int r = (int)s * 32 + lane;
        long long base = P.ssoff[s] + lane;
        int k = 0;
        if (r < ndof) {
          if (rest[r] || node_unused(P, r / ndpn)) {
            P.scol[base] = r;
            P.sdiag[r] = base;
            k = 1;
          } else {
            int I = r / ndpn;
            for (int q = P.nrp[I]; q < P.nrp[I + 1]; ++q) {
              int J = P.ncol[q];
              for (int j = 0; j < ndpn; ++j) {
                int c = J * ndpn + j;
                if (rest[c]) continue;
                if (c == r) P.sdiag[r] = base + (long long)k * 32;
                P.scol[base + (long long)k * 32] = c;
                ++k;
              }
            }
          }
        }
        for (; k < w; ++k) P.scol[base + (long long)k * 32] = r < ndof ? r : 0;
      }
    }
  });
  return "";
}

void export_lower_pattern(const HostPattern& P, const unsigned char* rest, long long* row_ptr,
                          int* col) {
  long long p = 0;
  const int nd = P.ndpn;
  for (int r = 0; r < P.ndof; ++r) {
    row_ptr[r] = p;
    if (rest[r] || node_unused(P, r / nd)) { col[p++] = r; continue; }
    int I = r / nd;
    long long start = p;
    for (int k = P.nrp[I]; k < P.nrp[I + 1]; ++k) {
      int J = P.ncol[k];
      for (int j = 0; j < nd; ++j) {
        int c = J * nd + j;
        if (!rest[c] && c <= r) col[p++] = c;
      }
    }
    if (p == start) col[p++] = r;
  }
  row_ptr[P.ndof] = p;
}

void export_lower_values_scalar(const HostPattern& P, const unsigned char* rest, const double* sval,
                                double* out) {
  long long p = 0;
  const int nd = P.ndpn;
  for (int r = 0; r < P.ndof; ++r) {
    long long base = P.ssoff[r / 32] + (r % 32);
    if (rest[r] || node_unused(P, r / nd)) { out[p++] = sval[P.sdiag[r]]; continue; }
    int I = r / nd;
    int k = 0;
    for (int q = P.nrp[I]; q < P.nrp[I + 1]; ++q) {
      int J = P.ncol[q];
      for (int j = 0; j < nd; ++j) {
        int c = J * nd + j;
        if (rest[c]) continue;
        if (c <= r) out[p++] = sval[base + (long long)k * 32];
        ++k;
      }
    }
  }
}

void export_lower_values_block(const HostPattern& P, const unsigned char* rest, const float* bval,
                               double* out) {
  long long p = 0;
  const int nd = P.ndpn, bb = nd * nd;
  for (int r = 0; r < P.ndof; ++r) {
    int I = r / nd, i = r % nd;
    long long chunk0 = P.bsoff[I / 32];
    int lane = I % 32;
    if (rest[r] || node_unused(P, I)) {
      long long ch = chunk0 + P.ndiag[I];
      out[p++] = bval[ch * 32 * bb + (long long)(i * nd + i) * 32 + lane];
      continue;
    }
    for (int q = P.nrp[I]; q < P.nrp[I + 1]; ++q) {
      int J = P.ncol[q];
      long long ch = chunk0 + (P.run > 1 ? (int)P.vpos[q] : q - P.nrp[I]);
      for (int j = 0; j < nd; ++j) {
        int c = J * nd + j;
        if (rest[c] || c > r) continue;
        out[p++] = bval[ch * 32 * bb + (long long)(i * nd + j) * 32 + lane];
      }
    }
  }
}

}  // namespace betagpu
