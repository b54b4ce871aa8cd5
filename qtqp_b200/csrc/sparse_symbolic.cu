// Symbolic analysis of the supernodal Cholesky factorisation used for sparse
// QPs whose Gram matrix G = P + A^T D A is neither dense nor narrow-banded
// (host code only; no CUDA call).
//
// Reference counterpart: the sparse direct backends behind the plugin
// interface (src/qtqp/solvers_sparse.py:96-121, SuperLU through
// scipy.sparse.linalg.factorized; src/qtqp/solvers_gpu.py:27-116, cuDSS),
// which order and factorise the regularised KKT matrix.  This build factorises
// the Gram matrix of the same system (the dense backend's reduction,
// src/qtqp/solvers_dense.py:99-116), so the symbolic stage works on G's
// pattern: the union of P's pattern and a clique per row of A.
//
// Stages:
//  1. a minimum-degree ordering of G's pattern on the quotient graph
//     (variables and elements, element absorption, supervariables of
//     indistinguishable variables, and the approximate external degree bound
//     d_i <= |A_i| + |L_p \ i| + sum_{e in E_i \ p} |L_e \ L_p| of Amestoy,
//     Davis and Duff, "An approximate minimum degree ordering algorithm",
//     SIAM J. Matrix Anal. Appl. 17(4), 1996);
//  2. the elimination tree (Liu's algorithm with path compression) and a
//     postorder of it, composed with the ordering, so that every subtree is
//     a contiguous range of columns;
//  3. column counts from the row subtrees, fundamental supernodes, relaxed
//     amalgamation (a child merged into its parent when the explicit zeros it
//     adds stay small) and a split of supernodes wider than kSnMaxWidth;
//  4. the row structure of each supernode (its columns, the pattern of its
//     columns below them, the structures of its children);
//  5. the left-looking update lists (for each supernode, the descendants with
//     rows in its column range, the first such row and how many);
//  6. the schedule of the grid: whole subtrees mapped to blocks (largest
//     first onto the least loaded block), and the supernodes above them by
//     level;
//  7. the map of G's lower entries (in the final ordering) to positions in
//     the supernodes' column-major value blocks.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "common.cuh"

namespace qtqp {

namespace {

using Adj = std::vector<std::vector<int>>;

// ----------------------------------------------------------------------------
// Stage 1: approximate minimum degree on the quotient graph.
// ----------------------------------------------------------------------------
class MinDegree {
 public:
  explicit MinDegree(const Adj& adj)
      : n_(int(adj.size())), av_(adj), ae_(n_), le_(n_), nv_(n_, 1), kind_(n_, 0), deg_(n_),
        head_(n_ + 1, -1), nxt_(n_, -1), prv_(n_, -1), chain_next_(n_, -1), chain_last_(n_),
        mark_(n_, 0), wst_(n_, 0), w_(n_, 0), bucket_of_(n_, -1) {
    for (int i = 0; i < n_; ++i) chain_last_[i] = i;
  }

  std::vector<int> order() {
    std::vector<int> out;
    out.reserve(n_);
    for (int i = 0; i < n_; ++i) {
      deg_[i] = int(av_[i].size());
      insert(i);
    }
    int remaining = n_, mindeg = 0;
    std::vector<int> lp;
    while (int(out.size()) < n_) {
      while (mindeg <= n_ && head_[mindeg] < 0) ++mindeg;
      if (mindeg > n_) break;  // cannot happen: every live variable is in a bucket
      const int p = head_[mindeg];
      remove(p);
      // L_p = (A_p u union_{e in E_p} L_e) \ {p}, principal variables only.
      const int stamp = ++stamp_;
      mark_[p] = stamp;
      lp.clear();
      for (int v : av_[p])
        if (live(v) && mark_[v] != stamp) {
          mark_[v] = stamp;
          lp.push_back(v);
        }
      for (int e : ae_[p]) {
        if (kind_[e] != 1) continue;
        for (int v : le_[e])
          if (live(v) && mark_[v] != stamp) {
            mark_[v] = stamp;
            lp.push_back(v);
          }
        kind_[e] = 2;  // absorbed into p
        std::vector<int>().swap(le_[e]);
      }
      // p and the variables merged into it are eliminated together.
      for (int v = p; v >= 0; v = chain_next_[v]) out.push_back(v);
      remaining -= nv_[p];
      kind_[p] = 1;
      le_[p] = lp;
      std::vector<int>().swap(av_[p]);
      std::vector<int>().swap(ae_[p]);
      int deg_lp = 0;
      for (int i : lp) {
        remove(i);
        deg_lp += nv_[i];
      }
      // w(e) = |L_e \ L_p| (weighted) for the elements next to L_p.
      const int wtag = ++wtag_;
      for (int i : lp)
        for (int e : ae_[i]) {
          if (kind_[e] != 1 || e == p) continue;
          if (wst_[e] != wtag) {
            wst_[e] = wtag;
            w_[e] = element_weight(e);
          }
          w_[e] -= nv_[i];
        }
      // New lists and degree bounds of the variables of L_p.
      for (int i : lp) {
        std::vector<int>& E = ae_[i];
        size_t k = 0;
        long ext = 0;
        for (int e : E) {
          if (kind_[e] != 1 || e == p) continue;
          if (wst_[e] == wtag && w_[e] <= 0) {  // L_e inside L_p: absorb e into p
            kind_[e] = 2;
            std::vector<int>().swap(le_[e]);
            continue;
          }
          E[k++] = e;
          ext += (wst_[e] == wtag) ? w_[e] : element_weight(e);
        }
        E.resize(k);
        E.push_back(p);
        std::vector<int>& V = av_[i];
        k = 0;
        for (int v : V) {
          if (!live(v) || v == i || mark_[v] == stamp) continue;  // covered by p
          V[k++] = v;
          ext += nv_[v];
        }
        V.resize(k);
        ext += deg_lp - nv_[i];
        long d = std::min<long>(long(deg_[i]) + deg_lp - nv_[i], ext);
        d = std::min<long>(d, remaining - nv_[i]);
        deg_[i] = int(std::max<long>(d, 0));
      }
      merge_indistinguishable(lp);
      for (int i : lp)
        if (nv_[i] > 0) {
          insert(i);
          mindeg = std::min(mindeg, deg_[i]);
        }
    }
    return out;
  }

 private:
  bool live(int v) const { return kind_[v] == 0 && nv_[v] > 0; }

  int element_weight(int e) {
    std::vector<int>& L = le_[e];
    size_t k = 0;
    int wsum = 0;
    for (int v : L)
      if (live(v)) {
        L[k++] = v;
        wsum += nv_[v];
      }
    L.resize(k);
    return wsum;
  }

  // Variables of L_p with equal variable and element lists are merged into
  // one supervariable (found by a hash of the lists, confirmed by comparing
  // the sorted lists).
  void merge_indistinguishable(const std::vector<int>& lp) {
    if (lp.size() < 2) return;
    std::vector<std::pair<unsigned long long, int>> h;
    h.reserve(lp.size());
    for (int i : lp) {
      unsigned long long s = 0;
      for (int v : av_[i]) s += unsigned(v) * 2654435761ull;
      for (int e : ae_[i]) s += unsigned(e) * 40503ull + 1;
      h.push_back({s, i});
    }
    std::sort(h.begin(), h.end());
    for (size_t a = 0; a < h.size();) {
      size_t b = a + 1;
      while (b < h.size() && h[b].first == h[a].first) ++b;
      if (b - a > 1) {
        for (size_t x = a; x < b; ++x) {
          std::sort(av_[h[x].second].begin(), av_[h[x].second].end());
          std::sort(ae_[h[x].second].begin(), ae_[h[x].second].end());
        }
        for (size_t x = a; x < b; ++x) {
          const int i = h[x].second;
          if (nv_[i] == 0) continue;
          for (size_t y = x + 1; y < b; ++y) {
            const int j = h[y].second;
            if (nv_[j] == 0 || av_[i] != av_[j] || ae_[i] != ae_[j]) continue;
            nv_[i] += nv_[j];
            deg_[i] = std::max(0, deg_[i] - nv_[j]);
            nv_[j] = 0;
            chain_next_[chain_last_[i]] = j;
            chain_last_[i] = chain_last_[j];
            std::vector<int>().swap(av_[j]);
            std::vector<int>().swap(ae_[j]);
          }
        }
      }
      a = b;
    }
  }

  void insert(int i) {
    const int d = std::min(deg_[i], n_);
    prv_[i] = -1;
    nxt_[i] = head_[d];
    if (head_[d] >= 0) prv_[head_[d]] = i;
    head_[d] = i;
    bucket_of_[i] = d;
  }
  void remove(int i) {
    const int d = bucket_of_[i];
    if (d < 0) return;
    if (prv_[i] >= 0) {
      nxt_[prv_[i]] = nxt_[i];
    } else {
      head_[d] = nxt_[i];
    }
    if (nxt_[i] >= 0) prv_[nxt_[i]] = prv_[i];
    bucket_of_[i] = -1;
  }
  int n_;
  Adj av_, ae_, le_;
  std::vector<int> nv_;
  std::vector<char> kind_;  // 0 variable, 1 element, 2 absorbed element
  std::vector<int> deg_, head_, nxt_, prv_, chain_next_, chain_last_;
  std::vector<int> mark_, wst_, w_;
  std::vector<int> bucket_of_;
  int stamp_ = 0, wtag_ = 0;
};

// ----------------------------------------------------------------------------
// Stages 2-7.
// ----------------------------------------------------------------------------
struct Plan {
  int n = 0, nsuper = 0, blocks = 0;
  std::vector<int32_t> perm;  // new -> old
  std::vector<int32_t> first, rows, colsn;
  std::vector<int64_t> rowptr, valptr;
  std::vector<int32_t> upd_ptr, upd_src, upd_off, upd_cnt;
  std::vector<int32_t> cta_ptr, cta_range, top_ptr, top_list, top_slab;
  std::vector<int32_t> gcol, grow;
  std::vector<int64_t> gpos;
  int max_rows = 0, max_width = 0, tree_levels = 0;
  int64_t nnz_l = 0;
  double flops = 0.0;
};

// G's pattern (no diagonal), one sorted list per column.
static int gram_pattern(int n, int m, const int32_t* ap, const int32_t* ai, const int32_t* pp,
                        const int32_t* pi, Adj& adj) {
  std::vector<int> rcnt(m + 1, 0);
  for (int j = 0; j < n; ++j) {
    if (ap[j + 1] < ap[j]) return fail(QTQP_ERR_BAD_ARG, "qtqp_sparse_analyze: bad A colptr");
    for (int q = ap[j]; q < ap[j + 1]; ++q) {
      if (ai[q] < 0 || ai[q] >= m)
        return fail(QTQP_ERR_BAD_ARG, "qtqp_sparse_analyze: A row index out of range");
      ++rcnt[ai[q] + 1];
    }
  }
  for (int r = 0; r < m; ++r) rcnt[r + 1] += rcnt[r];
  std::vector<int> rcol(rcnt[m]), fill(rcnt.begin(), rcnt.end() - 1);
  for (int j = 0; j < n; ++j)
    for (int q = ap[j]; q < ap[j + 1]; ++q) rcol[fill[ai[q]]++] = j;
  adj.assign(n, {});
  std::vector<int> mark(n, -1);
  for (int j = 0; j < n; ++j) {
    mark[j] = j;
    for (int q = ap[j]; q < ap[j + 1]; ++q) {
      const int r = ai[q];
      for (int t = rcnt[r]; t < rcnt[r + 1]; ++t) {
        const int k = rcol[t];
        if (mark[k] != j) {
          mark[k] = j;
          adj[j].push_back(k);
        }
      }
    }
    if (pp != nullptr) {
      if (pp[j + 1] < pp[j]) return fail(QTQP_ERR_BAD_ARG, "qtqp_sparse_analyze: bad P colptr");
      for (int q = pp[j]; q < pp[j + 1]; ++q) {
        const int i = pi[q];
        if (i < 0 || i >= n)
          return fail(QTQP_ERR_BAD_ARG, "qtqp_sparse_analyze: P row index out of range");
        if (mark[i] != j) {
          mark[i] = j;
          adj[j].push_back(i);
        }
      }
    }
    std::sort(adj[j].begin(), adj[j].end());
  }
  // P's pattern is symmetric for a symmetric P; make the union symmetric
  // regardless, so that the adjacency is a graph.
  if (pp != nullptr) {
    std::vector<std::vector<int>> extra(n);
    for (int j = 0; j < n; ++j)
      for (int i : adj[j])
        if (!std::binary_search(adj[i].begin(), adj[i].end(), j)) extra[i].push_back(j);
    for (int i = 0; i < n; ++i)
      if (!extra[i].empty()) {
        adj[i].insert(adj[i].end(), extra[i].begin(), extra[i].end());
        std::sort(adj[i].begin(), adj[i].end());
        adj[i].erase(std::unique(adj[i].begin(), adj[i].end()), adj[i].end());
      }
  }
  return QTQP_OK;
}

// The pattern relabelled by pinv (old -> new), sorted.
static Adj relabel(const Adj& adj, const std::vector<int>& perm, const std::vector<int>& pinv) {
  const int n = int(adj.size());
  Adj out(n);
  for (int k = 0; k < n; ++k) {
    const std::vector<int>& src = adj[perm[k]];
    out[k].reserve(src.size());
    for (int v : src) out[k].push_back(pinv[v]);
    std::sort(out[k].begin(), out[k].end());
  }
  return out;
}

// Elimination tree of the symmetric pattern (Liu, with path compression).
static std::vector<int> etree(const Adj& adj) {
  const int n = int(adj.size());
  std::vector<int> parent(n, -1), anc(n, -1);
  for (int k = 0; k < n; ++k)
    for (int i : adj[k]) {
      if (i >= k) break;
      int r = i;
      while (anc[r] != -1 && anc[r] != k) {
        const int t = anc[r];
        anc[r] = k;
        r = t;
      }
      if (anc[r] == -1) {
        anc[r] = k;
        parent[r] = k;
      }
    }
  return parent;
}

// Postorder of a forest (children in increasing order, roots in increasing order).
static std::vector<int> postorder(const std::vector<int>& parent) {
  const int n = int(parent.size());
  std::vector<int> head(n, -1), next(n, -1);
  for (int j = n - 1; j >= 0; --j)
    if (parent[j] >= 0) {
      next[j] = head[parent[j]];
      head[parent[j]] = j;
    }
  std::vector<int> post;
  post.reserve(n);
  std::vector<int> stack;
  for (int r = 0; r < n; ++r) {
    if (parent[r] >= 0) continue;
    stack.push_back(r);
    while (!stack.empty()) {
      const int j = stack.back();
      if (head[j] >= 0) {  // descend into the next unvisited child
        const int c = head[j];
        head[j] = next[c];
        stack.push_back(c);
      } else {
        stack.pop_back();
        post.push_back(j);
      }
    }
  }
  return post;
}

static int build_plan(int n, int m, const int32_t* ap, const int32_t* ai, const int32_t* pp,
                      const int32_t* pi, int ordering, int blocks, Plan& P) {
  Adj adj;
  int rc = gram_pattern(n, m, ap, ai, pp, pi, adj);
  if (rc) return rc;
  std::vector<int> order(n);
  if (ordering == 1) {
    order = MinDegree(adj).order();
    if (int(order.size()) != n) return fail(QTQP_ERR_BAD_ARG, "qtqp_sparse_analyze: ordering failed");
  } else {
    std::iota(order.begin(), order.end(), 0);
  }
  std::vector<int> pinv(n);
  for (int k = 0; k < n; ++k) pinv[order[k]] = k;
  Adj a1 = relabel(adj, order, pinv);
  // Postorder of the elimination tree, composed with the ordering.
  const std::vector<int> post = postorder(etree(a1));
  std::vector<int> perm(n);
  for (int k = 0; k < n; ++k) perm[k] = order[post[k]];
  for (int k = 0; k < n; ++k) pinv[perm[k]] = k;
  const Adj g = relabel(adj, perm, pinv);
  const std::vector<int> parent = etree(g);
  // Column counts of L (row subtrees).
  std::vector<int> cc(n, 0), mark(n, -1), nchild(n, 0);
  for (int k = 0; k < n; ++k) {
    mark[k] = k;
    for (int i : g[k]) {
      if (i >= k) break;
      for (int j = i; mark[j] != k; j = parent[j]) {
        ++cc[j];
        mark[j] = k;
      }
    }
    ++cc[k];
    if (parent[k] >= 0) ++nchild[parent[k]];
  }
  // Fundamental supernodes.
  struct Sn {
    int f, w, nr, parent;
    int64_t nz;  // true nonzeros of L in its columns
  };
  std::vector<Sn> fund;
  std::vector<int> fsn(n);
  for (int j = 0; j < n; ++j) {
    const bool join = j > 0 && parent[j - 1] == j && cc[j - 1] == cc[j] + 1 && nchild[j] == 1;
    if (!join) fund.push_back({j, 0, cc[j], -1, 0});
    Sn& s = fund.back();
    ++s.w;
    s.nz += cc[j];
    fsn[j] = int(fund.size()) - 1;
  }
  for (size_t s = 0; s < fund.size(); ++s) {
    const int last = fund[s].f + fund[s].w - 1;
    fund[s].parent = parent[last] >= 0 ? fsn[parent[last]] : -1;
  }
  // Relaxed amalgamation: in postorder, the record just before a supernode
  // is its last child when its parent is that supernode; merge it when the
  // explicit zeros stay small (thresholds by the merged width).
  std::vector<int> rep(fund.size());
  std::iota(rep.begin(), rep.end(), 0);
  auto find = [&](int x) {
    while (rep[x] != x) x = rep[x] = rep[rep[x]];
    return x;
  };
  std::vector<int> keep;  // indices of merged records, in order
  for (int s = 0; s < int(fund.size()); ++s) {
    Sn cur = fund[s];
    while (!keep.empty()) {
      const int c = keep.back();
      const Sn& ch = fund[c];
      if (ch.parent < 0 || find(ch.parent) != s || ch.f + ch.w != cur.f) break;
      const int W = ch.w + cur.w, NR = ch.w + cur.nr;
      if (W > kSnMaxWidth) break;
      const double stored = double(W) * NR - 0.5 * double(W) * (W - 1);
      const double zeros = stored - double(ch.nz + cur.nz);
      const double zf = zeros / stored;
      const bool ok = W <= 4 || (W <= 16 && zf < 0.8) || (W <= 48 && zf < 0.1) || zf < 0.05;
      if (!ok) break;
      cur.f = ch.f;
      cur.w = W;
      cur.nr = NR;
      cur.nz = ch.nz + cur.nz;
      rep[c] = s;
      keep.pop_back();
    }
    fund[s] = cur;
    keep.push_back(s);
  }
  // Final supernodes (splitting the ones wider than kSnMaxWidth).
  std::vector<int> fin_first;
  for (int s : keep) {
    const Sn& r = fund[s];
    for (int c = 0; c < r.w; c += kSnMaxWidth) fin_first.push_back(r.f + c);
  }
  fin_first.push_back(n);
  const int S = int(fin_first.size()) - 1;
  P.n = n;
  P.nsuper = S;
  P.blocks = blocks;
  P.perm.assign(perm.begin(), perm.end());
  P.first.assign(fin_first.begin(), fin_first.end());
  P.colsn.assign(n, 0);
  for (int s = 0; s < S; ++s)
    for (int j = fin_first[s]; j < fin_first[s + 1]; ++j) P.colsn[j] = s;
  std::vector<int> sparent(S, -1);
  for (int s = 0; s < S; ++s) {
    const int last = fin_first[s + 1] - 1;
    sparent[s] = parent[last] >= 0 ? P.colsn[parent[last]] : -1;
  }
  std::vector<std::vector<int>> kids(S);
  for (int s = 0; s < S; ++s)
    if (sparent[s] >= 0) kids[sparent[s]].push_back(s);
  // Row structures.
  P.rowptr.assign(S + 1, 0);
  P.valptr.assign(S + 1, 0);
  std::vector<std::vector<int>> R(S);
  std::fill(mark.begin(), mark.end(), -1);
  for (int s = 0; s < S; ++s) {
    const int f = fin_first[s], l = fin_first[s + 1];
    std::vector<int>& rs = R[s];
    for (int j = f; j < l; ++j) {
      rs.push_back(j);
      mark[j] = s;
    }
    for (int j = f; j < l; ++j)
      for (int i : g[j])
        if (i >= l && mark[i] != s) {
          mark[i] = s;
          rs.push_back(i);
        }
    for (int c : kids[s])
      for (int r : R[c])
        if (r >= f && mark[r] != s) {
          mark[r] = s;
          rs.push_back(r);
        }
    std::sort(rs.begin() + (l - f), rs.end());
    P.rowptr[s + 1] = P.rowptr[s] + int64_t(rs.size());
    P.valptr[s + 1] = P.valptr[s] + int64_t(rs.size()) * (l - f);
    P.max_rows = std::max(P.max_rows, int(rs.size()));
    P.max_width = std::max(P.max_width, l - f);
  }
  P.rows.reserve(P.rowptr[S]);
  for (int s = 0; s < S; ++s) P.rows.insert(P.rows.end(), R[s].begin(), R[s].end());
  // Left-looking update lists: for each descendant d, the runs of its rows
  // (beyond its own columns) that fall into one supernode's column range.
  {
    std::vector<int32_t> cnt(S + 1, 0);
    for (int d = 0; d < S; ++d) {
      const int w = fin_first[d + 1] - fin_first[d];
      const int nr = int(P.rowptr[d + 1] - P.rowptr[d]);
      const int32_t* rd = P.rows.data() + P.rowptr[d];
      for (int r = w; r < nr;) {
        const int t = P.colsn[rd[r]];
        int e = r + 1;
        while (e < nr && P.colsn[rd[e]] == t) ++e;
        ++cnt[t + 1];
        r = e;
      }
    }
    for (int s = 0; s < S; ++s) cnt[s + 1] += cnt[s];
    P.upd_ptr.assign(cnt.begin(), cnt.end());
    const int U = cnt[S];
    P.upd_src.assign(U, 0);
    P.upd_off.assign(U, 0);
    P.upd_cnt.assign(U, 0);
    std::vector<int32_t> fillp(cnt.begin(), cnt.end() - 1);
    for (int d = 0; d < S; ++d) {
      const int w = fin_first[d + 1] - fin_first[d];
      const int nr = int(P.rowptr[d + 1] - P.rowptr[d]);
      const int32_t* rd = P.rows.data() + P.rowptr[d];
      for (int r = w; r < nr;) {
        const int t = P.colsn[rd[r]];
        int e = r + 1;
        while (e < nr && P.colsn[rd[e]] == t) ++e;
        const int u = fillp[t]++;
        P.upd_src[u] = d;
        P.upd_off[u] = r;
        P.upd_cnt[u] = e - r;
        r = e;
      }
    }
  }
  // Work per supernode (multiply-adds): its updates, the Cholesky of its
  // diagonal block and the triangular solve of the rows below.
  std::vector<double> work(S, 0.0), sub(S, 0.0);
  std::vector<int> size(S, 1), level(S, 0);
  for (int s = 0; s < S; ++s) {
    const double w = fin_first[s + 1] - fin_first[s];
    const double nr = double(P.rowptr[s + 1] - P.rowptr[s]);
    double wk = w * w * w / 6.0 + (nr - w) * w * w / 2.0;
    for (int u = P.upd_ptr[s]; u < P.upd_ptr[s + 1]; ++u) {
      const int d = P.upd_src[u];
      const double wd = fin_first[d + 1] - fin_first[d];
      const double rem = double(P.rowptr[d + 1] - P.rowptr[d]) - P.upd_off[u];
      wk += rem * P.upd_cnt[u] * wd;
    }
    // A supernode also costs a fixed latency (its barriers and dependent loads,
    // tens of microseconds on one block), worth about 2e5 multiply-adds of
    // a block's throughput; without it, blocks given many small supernodes
    // finish their subtrees last.
    work[s] = wk + 2e5;
    P.flops += 2.0 * wk;
    P.nnz_l += int64_t(nr * w - w * (w - 1) / 2);
  }
  for (int s = 0; s < S; ++s) {
    sub[s] += work[s];
    if (sparent[s] >= 0) {
      sub[sparent[s]] += sub[s];
      size[sparent[s]] += size[s];
      level[sparent[s]] = std::max(level[sparent[s]], level[s] + 1);
    }
    P.tree_levels = std::max(P.tree_levels, level[s] + 1);
  }
  // Schedule: subtrees of at most total / (4 blocks) work go whole to one
  // block (a subtree is the contiguous range [s - size + 1, s]); the
  // supernodes above them run level by level over the grid.
  double total = 0.0;
  for (int s = 0; s < S; ++s)
    if (sparent[s] < 0) total += sub[s];
  const double chunk = total / (4.0 * blocks);
  std::vector<char> top(S, 0);
  std::vector<int> roots;
  for (int s = S - 1; s >= 0; --s) {
    const bool above = sparent[s] < 0 || top[sparent[s]];
    if (!above) continue;
    if (sub[s] > chunk && !kids[s].empty()) {
      top[s] = 1;
    } else {
      roots.push_back(s);
    }
  }
  std::sort(roots.begin(), roots.end(), [&](int a, int b) { return sub[a] > sub[b]; });
  std::vector<double> load(blocks, 0.0);
  std::vector<std::vector<int>> mine(blocks);
  for (int r : roots) {
    const int b = int(std::min_element(load.begin(), load.end()) - load.begin());
    load[b] += sub[r];
    mine[b].push_back(r);
  }
  P.cta_ptr.assign(blocks + 1, 0);
  for (int b = 0; b < blocks; ++b) {
    std::sort(mine[b].begin(), mine[b].end());
    for (int r : mine[b]) {
      P.cta_range.push_back(r - size[r] + 1);
      P.cta_range.push_back(r);
    }
    P.cta_ptr[b + 1] = int32_t(P.cta_range.size() / 2);
  }
  std::vector<int> tlev(S, -1);
  int ntl = 0;
  for (int s = 0; s < S; ++s) {
    if (!top[s]) continue;
    int lv = 0;
    for (int c : kids[s])
      if (top[c]) lv = std::max(lv, tlev[c] + 1);
    tlev[s] = lv;
    ntl = std::max(ntl, lv + 1);
  }
  P.top_ptr.assign(ntl + 1, 0);
  for (int s = 0; s < S; ++s)
    if (top[s]) ++P.top_ptr[tlev[s] + 1];
  for (int l = 0; l < ntl; ++l) P.top_ptr[l + 1] += P.top_ptr[l];
  P.top_list.assign(P.top_ptr[ntl], 0);
  {
    std::vector<int32_t> fl(P.top_ptr.begin(), P.top_ptr.end() - 1);
    for (int s = 0; s < S; ++s)
      if (top[s]) P.top_list[fl[tlev[s]]++] = s;
  }
  // Row slabs of the top supernodes (work items of the grid), prefix counts.
  P.top_slab.assign(P.top_list.size() + 1, 0);
  for (size_t q = 0; q < P.top_list.size(); ++q) {
    const int s = P.top_list[q];
    const int nr = int(P.rowptr[s + 1] - P.rowptr[s]);
    P.top_slab[q + 1] = P.top_slab[q] + (nr + kSnSlabRows - 1) / kSnSlabRows;
  }
  // G's lower entries (diagonal first in each column) and their positions.
  for (int j = 0; j < n; ++j) {
    const int s = P.colsn[j];
    const int f = fin_first[s];
    const int64_t nr = P.rowptr[s + 1] - P.rowptr[s];
    const int32_t* rs = P.rows.data() + P.rowptr[s];
    const int64_t base = P.valptr[s] + int64_t(j - f) * nr;
    P.gcol.push_back(j);
    P.grow.push_back(j);
    P.gpos.push_back(base + (j - f));
    for (int i : g[j]) {
      if (i <= j) continue;
      const int32_t* hit = std::lower_bound(rs, rs + nr, i);
      if (hit == rs + nr || *hit != i)
        return fail(QTQP_ERR_BAD_ARG, "qtqp_sparse_analyze: internal error (structure)");
      P.gcol.push_back(j);
      P.grow.push_back(i);
      P.gpos.push_back(base + (hit - rs));
    }
  }
  return QTQP_OK;
}

}  // namespace
}  // namespace qtqp

using namespace qtqp;

extern "C" int qtqp_sparse_analyze(int32_t n, int32_t m, const int32_t* h_a_colptr,
                                   const int32_t* h_a_rowind, const int32_t* h_p_colptr,
                                   const int32_t* h_p_rowind, int32_t ordering, int32_t blocks,
                                   void** h_plan, qtqp_sparse_desc* h_desc) {
  if (h_plan == nullptr || h_desc == nullptr)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_sparse_analyze: null output");
  *h_plan = nullptr;
  if (n < 1 || m < 0 || h_a_colptr == nullptr || (h_a_colptr[n] > 0 && h_a_rowind == nullptr) ||
      (h_p_colptr != nullptr && h_p_colptr[n] > 0 && h_p_rowind == nullptr))
    return fail(QTQP_ERR_BAD_ARG, "qtqp_sparse_analyze: bad sizes or pointers");
  if (ordering != 0 && ordering != 1)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_sparse_analyze: ordering must be 0 (natural) or 1 "
                                  "(minimum degree)");
  if (blocks < 1 || blocks > kGridMaxBlocks)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_sparse_analyze: blocks out of range");
  Plan* P = new Plan();
  int rc;
  try {
    rc = build_plan(n, m, h_a_colptr, h_a_rowind, h_p_colptr, h_p_rowind, ordering, blocks, *P);
  } catch (const std::bad_alloc&) {
    rc = fail(QTQP_ERR_BAD_ARG, "qtqp_sparse_analyze: out of host memory");
  }
  if (rc) {
    delete P;
    return rc;
  }
  qtqp_sparse_desc& d = *h_desc;
  std::memset(&d, 0, sizeof(d));
  d.n = n;
  d.nsuper = P->nsuper;
  d.blocks = blocks;
  d.top_levels = int32_t(P->top_ptr.size()) - 1;
  d.max_rows = P->max_rows;
  d.max_width = P->max_width;
  d.tree_levels = P->tree_levels;
  d.nvals = P->valptr.back();
  d.ngram = int64_t(P->gcol.size());
  d.nrows = int64_t(P->rows.size());
  d.nupd = int64_t(P->upd_src.size());
  d.nranges = int64_t(P->cta_range.size() / 2);
  d.ntop = int64_t(P->top_list.size());
  d.nnz_l = P->nnz_l;
  d.top_row_slabs = P->top_slab.back();
  d.flops = P->flops;
  int64_t o = 0;
  auto put = [&](int64_t& off, size_t count) {
    off = o;
    o += int64_t((count + 3) & ~size_t(3));  // 16-byte aligned sections
  };
  put(d.o_first, P->first.size());
  put(d.o_colsn, P->colsn.size());
  put(d.o_rows, P->rows.size());
  put(d.o_upd_ptr, P->upd_ptr.size());
  put(d.o_upd_src, P->upd_src.size());
  put(d.o_upd_off, P->upd_off.size());
  put(d.o_upd_cnt, P->upd_cnt.size());
  put(d.o_cta_ptr, P->cta_ptr.size());
  put(d.o_cta_range, P->cta_range.size());
  put(d.o_top_ptr, P->top_ptr.size());
  put(d.o_top_list, P->top_list.size());
  put(d.o_top_slab, P->top_slab.size());
  put(d.o_gcol, P->gcol.size());
  put(d.o_grow, P->grow.size());
  d.n32 = o;
  o = 0;
  auto put64 = [&](int64_t& off, size_t count) {
    off = o;
    o += int64_t((count + 1) & ~size_t(1));
  };
  put64(d.o_rowptr, P->rowptr.size());
  put64(d.o_valptr, P->valptr.size());
  put64(d.o_gpos, P->gpos.size());
  d.n64 = o;
  *h_plan = P;
  return QTQP_OK;
}

extern "C" int qtqp_sparse_export(const void* h_plan, const qtqp_sparse_desc* h_desc,
                                  int32_t* h_perm, int32_t* h_pool32, int64_t* h_pool64) {
  if (h_plan == nullptr || h_desc == nullptr || h_perm == nullptr || h_pool32 == nullptr ||
      h_pool64 == nullptr)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_sparse_export: null argument");
  const Plan& P = *static_cast<const Plan*>(h_plan);
  const qtqp_sparse_desc& d = *h_desc;
  if (d.n != P.n || d.nsuper != P.nsuper)
    return fail(QTQP_ERR_BAD_ARG, "qtqp_sparse_export: descriptor of another plan");
  std::memcpy(h_perm, P.perm.data(), sizeof(int32_t) * P.perm.size());
  std::memset(h_pool32, 0, sizeof(int32_t) * d.n32);
  std::memset(h_pool64, 0, sizeof(int64_t) * d.n64);
  auto cp = [&](int64_t off, const std::vector<int32_t>& v) {
    if (!v.empty()) std::memcpy(h_pool32 + off, v.data(), sizeof(int32_t) * v.size());
  };
  auto cp64 = [&](int64_t off, const std::vector<int64_t>& v) {
    if (!v.empty()) std::memcpy(h_pool64 + off, v.data(), sizeof(int64_t) * v.size());
  };
  cp(d.o_first, P.first);
  cp(d.o_colsn, P.colsn);
  cp(d.o_rows, P.rows);
  cp(d.o_upd_ptr, P.upd_ptr);
  cp(d.o_upd_src, P.upd_src);
  cp(d.o_upd_off, P.upd_off);
  cp(d.o_upd_cnt, P.upd_cnt);
  cp(d.o_cta_ptr, P.cta_ptr);
  cp(d.o_cta_range, P.cta_range);
  cp(d.o_top_ptr, P.top_ptr);
  cp(d.o_top_list, P.top_list);
  cp(d.o_top_slab, P.top_slab);
  cp(d.o_gcol, P.gcol);
  cp(d.o_grow, P.grow);
  cp64(d.o_rowptr, P.rowptr);
  cp64(d.o_valptr, P.valptr);
  cp64(d.o_gpos, P.gpos);
  return QTQP_OK;
}

extern "C" void qtqp_sparse_free(void* h_plan) { delete static_cast<Plan*>(h_plan); }
