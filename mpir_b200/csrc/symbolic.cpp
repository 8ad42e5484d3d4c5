// Host symbolic analysis; see symbolic.hpp.
#include "symbolic.hpp"

#include <algorithm>
#include <limits>
#include <map>
#include <numeric>

namespace mpir {
namespace {

// ---------------------------------------------------------------------------
// Graph of the symmetric pattern (no diagonal), node ids int32.
struct Graph {
  int32_t              n = 0;
  std::vector<int64_t> xadj;
  std::vector<int32_t> adj;
  int32_t              deg(int32_t v) const {
    return static_cast<int32_t>(xadj[v + 1] - xadj[v]);
  }
};

Graph build_graph(int64_t n, const int64_t *Ap, const int64_t *Ai) {
  Graph g;
  g.n = static_cast<int32_t>(n);
  g.xadj.assign(n + 1, 0);
  for (int64_t j = 0; j < n; j++)
    for (int64_t p = Ap[j]; p < Ap[j + 1]; p++) {
      const int64_t i = Ai[p];
      if (i == j) continue;
      g.xadj[i + 1]++;
      g.xadj[j + 1]++;
    }
  for (int64_t v = 0; v < n; v++) g.xadj[v + 1] += g.xadj[v];
  g.adj.resize(g.xadj[n]);
  std::vector<int64_t> fill(g.xadj.begin(), g.xadj.end() - 1);
  for (int64_t j = 0; j < n; j++)
    for (int64_t p = Ap[j]; p < Ap[j + 1]; p++) {
      const int64_t i = Ai[p];
      if (i == j) continue;
      g.adj[fill[i]++] = static_cast<int32_t>(j);
      g.adj[fill[j]++] = static_cast<int32_t>(i);
    }
  return g;
}

// ---------------------------------------------------------------------------
// Recursive nested dissection by breadth-first level sets (George & Liu):
// from a pseudo-peripheral node, the level that splits the set in half is a
// vertex separator; nodes of that level with no neighbour in the next level
// do not separate anything and join the first part.  Each part is ordered
// before the separator.  Sets of at most kLeaf nodes keep their order.
class NestedDissection {
 public:
  explicit NestedDissection(const Graph &g)
      : g_(g), tag_(g.n, 0), level_(g.n, -1) {}

  void order(std::vector<int32_t> nodes, std::vector<int32_t> &out) {
    out_ = &out;
    split(nodes);
  }

 private:
#ifndef MPIR_ND_LEAF
#define MPIR_ND_LEAF 64
#endif
  static constexpr size_t kLeaf = MPIR_ND_LEAF;
  const Graph            &g_;
  std::vector<int32_t>    tag_, level_;
  int32_t                 cur_ = 0;
  std::vector<int32_t>   *out_ = nullptr;

  // BFS over nodes carrying tag t.  Fills `order` with visit order and
  // level_; returns the number of levels.
  int bfs(int32_t root, int32_t t, std::vector<int32_t> &order,
          std::vector<int32_t> &count) {
    order.clear();
    count.clear();
    order.push_back(root);
    level_[root] = 0;
    size_t head  = 0;
    while (head < order.size()) {
      const int32_t v = order[head++];
      const int32_t l = level_[v];
      if (static_cast<int32_t>(count.size()) <= l) count.push_back(0);
      count[l]++;
      for (int64_t p = g_.xadj[v]; p < g_.xadj[v + 1]; p++) {
        const int32_t u = g_.adj[p];
        if (tag_[u] == t && level_[u] < 0) {
          level_[u] = l + 1;
          order.push_back(u);
        }
      }
    }
    return static_cast<int>(count.size());
  }

  void reset_levels(const std::vector<int32_t> &nodes) {
    for (int32_t v : nodes) level_[v] = -1;
  }

  void split(std::vector<int32_t> &S) {
    if (S.empty()) return;
    const int32_t t = ++cur_;
    for (int32_t v : S) tag_[v] = t;
    if (S.size() <= kLeaf) {
      out_->insert(out_->end(), S.begin(), S.end());
      return;
    }
    // Connected components.
    std::vector<int32_t>              order, count;
    std::vector<std::vector<int32_t>> comps;
    reset_levels(S);
    for (int32_t v : S) {
      if (level_[v] >= 0) continue;
      bfs(v, t, order, count);
      comps.push_back(order);
    }
    if (comps.size() > 1) {
      for (auto &c : comps) split(c);
      return;
    }
    // Pseudo-peripheral root.
    int32_t root = S[0];
    int     ecc  = -1;
    for (int it = 0; it < 6; it++) {
      reset_levels(S);
      const int nl = bfs(root, t, order, count);
      if (nl - 1 <= ecc) break;
      ecc          = nl - 1;
      int32_t best = -1;
      for (size_t q = order.size(); q-- > 0;) {
        const int32_t v = order[q];
        if (level_[v] != nl - 1) break;
        if (best < 0 || g_.deg(v) < g_.deg(best)) best = v;
      }
      root = best;
    }
    reset_levels(S);
    const int nl = bfs(root, t, order, count);
    if (nl < 3) {  // no level separates: keep as one block
      out_->insert(out_->end(), S.begin(), S.end());
      return;
    }
    const int64_t half = static_cast<int64_t>(S.size()) / 2;
    int           m    = 1;
    int64_t       cum  = 0;
    for (int l = 0; l < nl; l++) {
      if (cum + count[l] > half) {
        m = l;
        break;
      }
      cum += count[l];
    }
    m = std::clamp(m, 1, nl - 2);
    std::vector<int32_t> A, B, sep;
    for (int32_t v : order) {
      const int l = level_[v];
      if (l < m) {
        A.push_back(v);
      } else if (l > m) {
        B.push_back(v);
      } else {
        bool separates = false;
        for (int64_t p = g_.xadj[v]; p < g_.xadj[v + 1] && !separates; p++) {
          const int32_t u = g_.adj[p];
          separates       = tag_[u] == t && level_[u] == m + 1;
        }
        (separates ? sep : A).push_back(v);
      }
    }
    reset_levels(S);
    for (int32_t v : sep) tag_[v] = 0;
    split(A);
    split(B);
    out_->insert(out_->end(), sep.begin(), sep.end());
  }
};

// ---------------------------------------------------------------------------
// Permuted upper CSC: entry p of the caller (row i, col j) lands at
// (min(q_i, q_j), max(q_i, q_j)) with q = iperm; rows ascending per column.
void permute_upper(int64_t n, const int64_t *Ap, const int64_t *Ai,
                   const std::vector<int64_t> &iperm, std::vector<int64_t> &Cp,
                   std::vector<int64_t> &Ci, std::vector<int64_t> &Csrc) {
  const int64_t        nnz = Ap[n];
  std::vector<int64_t> r(nnz), c(nnz);
  for (int64_t j = 0; j < n; j++)
    for (int64_t p = Ap[j]; p < Ap[j + 1]; p++) {
      const int64_t a = iperm[Ai[p]], b = iperm[j];
      r[p]                  = std::min(a, b);
      c[p]                  = std::max(a, b);
    }
  // Bucket by row, then stably by column: rows end up ascending.
  std::vector<int64_t> rp(n + 1, 0), byrow(nnz);
  for (int64_t p = 0; p < nnz; p++) rp[r[p] + 1]++;
  for (int64_t i = 0; i < n; i++) rp[i + 1] += rp[i];
  for (int64_t p = 0; p < nnz; p++) byrow[rp[r[p]]++] = p;
  Cp.assign(n + 1, 0);
  for (int64_t p = 0; p < nnz; p++) Cp[c[p] + 1]++;
  for (int64_t j = 0; j < n; j++) Cp[j + 1] += Cp[j];
  std::vector<int64_t> fill(Cp.begin(), Cp.end() - 1);
  Ci.resize(nnz);
  Csrc.resize(nnz);
  for (int64_t q = 0; q < nnz; q++) {
    const int64_t p = byrow[q];
    const int64_t d = fill[c[p]]++;
    Ci[d]           = r[p];
    Csrc[d]         = p;
  }
}

// Transpose of an upper CSC: for each i the columns j > i holding (i, j).
void upper_rows(int64_t n, const std::vector<int64_t> &Cp,
                const std::vector<int64_t> &Ci, std::vector<int64_t> &Rp,
                std::vector<int64_t> &Rj) {
  Rp.assign(n + 1, 0);
  for (int64_t j = 0; j < n; j++)
    for (int64_t p = Cp[j]; p < Cp[j + 1]; p++)
      if (Ci[p] < j) Rp[Ci[p] + 1]++;
  for (int64_t i = 0; i < n; i++) Rp[i + 1] += Rp[i];
  Rj.resize(Rp[n]);
  std::vector<int64_t> fill(Rp.begin(), Rp.end() - 1);
  for (int64_t j = 0; j < n; j++)
    for (int64_t p = Cp[j]; p < Cp[j + 1]; p++)
      if (Ci[p] < j) Rj[fill[Ci[p]]++] = j;
}

// Elimination tree by Liu's algorithm with path compression over the
// ancestor links: parent[i] = min{ j > i : L(j, i) != 0 }.
void liu_etree(int64_t n, const int64_t *Cp, const int64_t *Ci,
               std::vector<int64_t> &parent) {
  parent.assign(n, -1);
  std::vector<int64_t> anc(n, -1);
  for (int64_t j = 0; j < n; j++)
    for (int64_t p = Cp[j]; p < Cp[j + 1]; p++)
      for (int64_t i = Ci[p]; i != -1 && i < j;) {
        const int64_t next = anc[i];
        anc[i]             = j;
        if (next == -1) parent[i] = j;
        i = next;
      }
}

// Post-order of a forest (children visited in increasing order).
void postorder(int64_t n, const std::vector<int64_t> &parent,
               std::vector<int64_t> &post) {
  std::vector<int64_t> head(n, -1), next(n, -1), stack;
  for (int64_t j = n; j-- > 0;) {
    if (parent[j] < 0) continue;
    next[j]         = head[parent[j]];
    head[parent[j]] = j;
  }
  post.clear();
  post.reserve(n);
  for (int64_t r = 0; r < n; r++) {
    if (parent[r] >= 0) continue;
    stack.push_back(r);
    while (!stack.empty()) {
      const int64_t v = stack.back();
      const int64_t c = head[v];
      if (c < 0) {
        stack.pop_back();
        post.push_back(v);
      } else {
        head[v] = next[c];
        stack.push_back(c);
      }
    }
  }
}

// Column counts of L (diagonal included) from the row subtrees, after
// Gilbert, Ng & Peyton (1994): each row subtree's leaves and the least
// common ancestors of consecutive leaves give +1/-1 marks that sum up the
// tree to the counts.  Rows of the lower triangle come from Rp/Rj.
void column_counts(int64_t n, const std::vector<int64_t> &parent,
                   const std::vector<int64_t> &post,
                   const std::vector<int64_t> &Rp,
                   const std::vector<int64_t> &Rj,
                   std::vector<int64_t>       &cc) {
  std::vector<int64_t> first(n, -1), maxfirst(n, -1), prevleaf(n, -1),
      anc(n);
  cc.assign(n, 0);
  for (int64_t k = 0; k < n; k++) {
    int64_t j = post[k];
    cc[j]     = first[j] == -1 ? 1 : 0;
    for (; j != -1 && first[j] == -1; j = parent[j]) first[j] = k;
  }
  std::iota(anc.begin(), anc.end(), 0);
  for (int64_t k = 0; k < n; k++) {
    const int64_t j = post[k];
    if (parent[j] != -1) cc[parent[j]]--;
    for (int64_t p = Rp[j]; p < Rp[j + 1]; p++) {
      const int64_t i = Rj[p];  // i > j with A(j, i) != 0
      if (first[j] <= maxfirst[i]) continue;
      maxfirst[i]         = first[j];
      const int64_t jprev = prevleaf[i];
      prevleaf[i]         = j;
      cc[j]++;
      if (jprev == -1) continue;
      int64_t q = jprev;
      while (q != anc[q]) q = anc[q];
      for (int64_t s = jprev; s != q;) {
        const int64_t up = anc[s];
        anc[s]           = q;
        s                = up;
      }
      cc[q]--;
    }
    if (parent[j] != -1) anc[j] = parent[j];
  }
  for (int64_t j = 0; j < n; j++)
    if (parent[j] != -1) cc[parent[j]] += cc[j];
}

// First-fit arena with coalescing, used to plan offsets ahead of time.
class ArenaPlan {
 public:
  int64_t alloc(int64_t size) {
    size = (size + 63) / 64 * 64;
    for (auto it = free_.begin(); it != free_.end(); ++it)
      if (it->second >= size) {
        const int64_t off = it->first, rest = it->second - size;
        free_.erase(it);
        if (rest > 0) free_[off + size] = rest;
        return off;
      }
    const int64_t off = top_;
    top_ += size;
    peak_ = std::max(peak_, top_);
    return off;
  }
  void release(int64_t off, int64_t size) {
    size = (size + 63) / 64 * 64;
    auto it = free_.emplace(off, size).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
        it = pv;
      }
    }
    if (it->first + it->second == top_) {
      top_ = it->first;
      free_.erase(it);
    }
  }
  int64_t peak() const { return peak_; }

 private:
  std::map<int64_t, int64_t> free_;
  int64_t                    top_ = 0, peak_ = 0;
};

// Everything derived from supernode ranges and row structures.
void finish_schedule(Symbolic &S) {
  const int64_t n = S.n, ns = S.ns;
  S.col2sup.assign(n, 0);
  for (int64_t J = 0; J < ns; J++)
    for (int64_t j = S.sfirst[J]; j < S.sfirst[J + 1]; j++) S.col2sup[j] = J;
  S.sparent.assign(ns, -1);
  for (int64_t J = 0; J < ns; J++) {
    const int64_t last = S.sfirst[J + 1] - 1;
    const int64_t p    = S.etree[last];
    S.sparent[J]       = p < 0 ? -1 : S.col2sup[p];
  }
  // Panels.
  S.slofs.assign(ns + 1, 0);
  S.zofs.assign(ns + 1, 0);
  S.max_h = S.max_w = 0;
  for (int64_t J = 0; J < ns; J++) {
    S.slofs[J + 1] = S.slofs[J] + S.h(J) * S.w(J);
    S.zofs[J + 1]  = S.zofs[J] + S.h(J);
    S.max_h        = std::max(S.max_h, S.h(J));
    S.max_w        = std::max(S.max_w, S.w(J));
  }
  S.panel_elems = S.slofs[ns];
  S.z_elems     = S.zofs[ns];
  // Children and levels.
  S.child_ptr.assign(ns + 1, 0);
  for (int64_t J = 0; J < ns; J++)
    if (S.sparent[J] >= 0) S.child_ptr[S.sparent[J] + 1]++;
  for (int64_t J = 0; J < ns; J++) S.child_ptr[J + 1] += S.child_ptr[J];
  S.child_list.resize(S.child_ptr[ns]);
  {
    std::vector<int64_t> fill(S.child_ptr.begin(), S.child_ptr.end() - 1);
    for (int64_t J = 0; J < ns; J++)
      if (S.sparent[J] >= 0)
        S.child_list[fill[S.sparent[J]]++] = static_cast<int32_t>(J);
  }
  S.slevel.assign(ns, 0);
  for (int64_t J = 0; J < ns; J++)
    if (S.sparent[J] >= 0)
      S.slevel[S.sparent[J]] = std::max(S.slevel[S.sparent[J]], S.slevel[J] + 1);
  S.nlevels = 0;
  for (int64_t J = 0; J < ns; J++) S.nlevels = std::max(S.nlevels, S.slevel[J] + 1);
  S.level_ptr.assign(S.nlevels + 1, 0);
  for (int64_t J = 0; J < ns; J++) S.level_ptr[S.slevel[J] + 1]++;
  for (int32_t t = 0; t < S.nlevels; t++) S.level_ptr[t + 1] += S.level_ptr[t];
  S.level_sup.resize(ns);
  {
    std::vector<int64_t> fill(S.level_ptr.begin(), S.level_ptr.end() - 1);
    for (int64_t J = 0; J < ns; J++)
      S.level_sup[fill[S.slevel[J]]++] = static_cast<int32_t>(J);
  }
  // Relative row maps into the parent's index set.
  S.srel.assign(S.srows.size(), -1);
  {
    std::vector<int32_t> pos(n, -1);
    for (int64_t P = 0; P < ns; P++) {
      const int64_t b = S.srowptr[P], e = S.srowptr[P + 1];
      for (int64_t q = b; q < e; q++) pos[S.srows[q]] = static_cast<int32_t>(q - b);
      for (int64_t c = S.child_ptr[P]; c < S.child_ptr[P + 1]; c++) {
        const int64_t C = S.child_list[c];
        for (int64_t q = S.srowptr[C] + S.w(C); q < S.srowptr[C + 1]; q++)
          S.srel[q] = pos[S.srows[q]];
      }
    }
  }
  // Update-matrix arena: U_J is written when level(J) runs and read when
  // level(parent) runs.
  S.uofs.assign(ns, -1);
  {
    ArenaPlan plan;
    for (int32_t t = 0; t < S.nlevels; t++) {
      for (int64_t q = S.level_ptr[t]; q < S.level_ptr[t + 1]; q++) {
        const int64_t J = S.level_sup[q], r = S.h(J) - S.w(J);
        if (r > 0) S.uofs[J] = plan.alloc(r * r);
      }
      for (int64_t q = S.level_ptr[t]; q < S.level_ptr[t + 1]; q++) {
        const int64_t P = S.level_sup[q];
        for (int64_t c = S.child_ptr[P]; c < S.child_ptr[P + 1]; c++) {
          const int64_t C = S.child_list[c], r = S.h(C) - S.w(C);
          if (r > 0) plan.release(S.uofs[C], r * r);
        }
      }
    }
    S.uarena_elems = plan.peak();
  }
}

// Supernodes from the etree and counts: column j joins j-1's supernode when
// j is j-1's parent and L(:, j-1) = {j} + L(:, j).
void find_supernodes(Symbolic &S) {
  const int64_t n = S.n;
  S.sfirst.clear();
  for (int64_t j = 0; j < n; j++) {
    const bool join = j > 0 && S.etree[j - 1] == j && S.Lnz[j - 1] == S.Lnz[j] + 1;
    if (!join) S.sfirst.push_back(j);
  }
  S.sfirst.push_back(n);
  S.ns = static_cast<int64_t>(S.sfirst.size()) - 1;
}

// Relaxed amalgamation.  A supernode whose columns end right before its
// parent's first column may be merged into the parent; the merged panel
// keeps the parent's row set R_P, so each merged child column gains
// (h_P - |R_child|) explicit zeros.  Merges are accepted when the merged
// width is tiny or the zero fraction of the merged lower-trapezoidal panel
// stays small (thresholds in the style of the usual relaxed-supernode
// heuristics).  Only counts are needed: |R_J| = Lnz of J's last column.
void relax_supernodes(Symbolic &S) {
  const int64_t        ns = S.ns;
  std::vector<int64_t> col2sup(S.n);
  for (int64_t J = 0; J < ns; J++)
    for (int64_t j = S.sfirst[J]; j < S.sfirst[J + 1]; j++) col2sup[j] = J;
  std::vector<int64_t> first(S.sfirst.begin(), S.sfirst.end() - 1);
  std::vector<double>  zeros(ns, 0.0);
  std::vector<char>    dead(ns, 0);
  for (int64_t J = 0; J < ns; J++) {
    const int64_t last = S.sfirst[J + 1] - 1;
    if (S.etree[last] < 0) continue;
    const int64_t P = col2sup[S.etree[last]];
    if (S.sfirst[P] != last + 1) continue;  // not the adjacent child
    const double wj = static_cast<double>(last + 1 - first[J]);
    const double rj = static_cast<double>(S.Lnz[last]);
    const double wp = static_cast<double>(S.sfirst[P + 1] - S.sfirst[P]);
    const double rp = static_cast<double>(S.Lnz[S.sfirst[P + 1] - 1]);
    const double w  = wj + wp, h = w + rp;
    const double z  = zeros[J] + zeros[P] + wj * (wp + rp - rj);
    const double tot  = w * h - w * (w - 1) / 2;
    const double frac = z / tot;
    const bool   ok   = w <= 4 || (w <= 16 && frac < 0.8) ||
                    (w <= 48 && frac < 0.1) || frac < 0.05;
    if (!ok) continue;
    first[P] = first[J];
    zeros[P] = z;
    dead[J]  = 1;
  }
  std::vector<int64_t> sf;
  for (int64_t J = 0; J < ns; J++)
    if (!dead[J]) sf.push_back(first[J]);
  sf.push_back(S.n);
  S.sfirst = std::move(sf);
  S.ns     = static_cast<int64_t>(S.sfirst.size()) - 1;
}

}  // namespace

int64_t etree_counts(int64_t n, const int64_t *Ap, const int64_t *Ai,
                     int64_t *etree, int64_t *Lnz) {
  for (int64_t j = 0; j < n; j++) {
    if (Ap[j] == Ap[j + 1]) return kBadInput;
    for (int64_t p = Ap[j]; p < Ap[j + 1]; p++)
      if (Ai[p] > j || Ai[p] < 0) return kBadInput;
  }
  std::vector<int64_t> Cp(Ap, Ap + n + 1), Ci(Ai, Ai + Ap[n]);
  std::vector<int64_t> parent, post, Rp, Rj, cc;
  liu_etree(n, Cp.data(), Ci.data(), parent);
  postorder(n, parent, post);
  upper_rows(n, Cp, Ci, Rp, Rj);
  column_counts(n, parent, post, Rp, Rj, cc);
  int64_t total = 0;
  for (int64_t j = 0; j < n; j++) {
    etree[j] = parent[j];
    Lnz[j]   = cc[j] - 1;
    if (total > std::numeric_limits<int64_t>::max() - Lnz[j]) return kOverflow;
    total += Lnz[j];
  }
  return total;
}

int analyze(int64_t n, const int64_t *Ap, const int64_t *Ai,
            const int8_t *diag_sign, Ordering ord, Symbolic &S,
            std::string &err) {
  S   = Symbolic{};
  S.n = n;
  if (n < 0) {
    err = "negative dimension";
    return kBadArgument;
  }
  if (n > std::numeric_limits<int32_t>::max() - 1) {
    err = "dimension exceeds int32 row indices";
    return kBadArgument;
  }
  // Input checks in the order QDLDL_etree makes them (qdldl.hpp:58-78).
  for (int64_t j = 0; j < n; j++)
    if (Ap[j] == Ap[j + 1]) {
      err = "empty column " + std::to_string(j);
      return kBadInput;
    }
  for (int64_t j = 0; j < n; j++)
    for (int64_t p = Ap[j]; p < Ap[j + 1]; p++)
      if (Ai[p] > j || Ai[p] < 0) {
        err = "entry below the diagonal in column " + std::to_string(j);
        return kBadInput;
      }
  S.nnz = n > 0 ? Ap[n] : 0;

  // Ordering.
  S.perm.resize(n);
  std::iota(S.perm.begin(), S.perm.end(), 0);
  if (ord == Ordering::Auto && n > 0) {
    Graph g = build_graph(n, Ap, Ai);
    std::vector<int32_t> first, second, out;
    for (int64_t i = 0; i < n; i++)
      ((diag_sign == nullptr || diag_sign[i] > 0) ? first : second)
          .push_back(static_cast<int32_t>(i));
    // Only the first block's internal edges steer its dissection.
    if (!second.empty()) {
      std::vector<char> in1(n, 0);
      for (int32_t v : first) in1[v] = 1;
      Graph h;
      h.n = g.n;
      h.xadj.assign(n + 1, 0);
      for (int64_t v = 0; v < n; v++) {
        int64_t cnt = 0;
        if (in1[v])
          for (int64_t p = g.xadj[v]; p < g.xadj[v + 1]; p++) cnt += in1[g.adj[p]];
        h.xadj[v + 1] = h.xadj[v] + cnt;
      }
      h.adj.resize(h.xadj[n]);
      for (int64_t v = 0, q = 0; v < n; v++)
        if (in1[v])
          for (int64_t p = g.xadj[v]; p < g.xadj[v + 1]; p++)
            if (in1[g.adj[p]]) h.adj[q++] = g.adj[p];
      g = std::move(h);
    }
    NestedDissection nd(g);
    nd.order(first, out);
    out.insert(out.end(), second.begin(), second.end());
    for (int64_t k = 0; k < n; k++) S.perm[k] = out[k];
  }
  S.iperm.resize(n);
  for (int64_t k = 0; k < n; k++) S.iperm[S.perm[k]] = k;

  permute_upper(n, Ap, Ai, S.iperm, S.Cp, S.Ci, S.Csrc);
  std::vector<int64_t> parent, post;
  liu_etree(n, S.Cp.data(), S.Ci.data(), parent);
  if (ord == Ordering::Auto && n > 0) {
    // Post-order the elimination tree: same fill, contiguous subtrees.
    postorder(n, parent, post);
    std::vector<int64_t> p2(n);
    for (int64_t k = 0; k < n; k++) p2[k] = S.perm[post[k]];
    S.perm = std::move(p2);
    for (int64_t k = 0; k < n; k++) S.iperm[S.perm[k]] = k;
    permute_upper(n, Ap, Ai, S.iperm, S.Cp, S.Ci, S.Csrc);
    liu_etree(n, S.Cp.data(), S.Ci.data(), parent);
  }
  postorder(n, parent, post);
  std::vector<int64_t> Rp, Rj, cc;
  upper_rows(n, S.Cp, S.Ci, Rp, Rj);
  column_counts(n, parent, post, Rp, Rj, cc);
  S.etree = parent;
  S.Lnz.resize(n);
  S.nnzL = 0;
  for (int64_t j = 0; j < n; j++) {
    S.Lnz[j] = cc[j] - 1;
    if (S.nnzL > std::numeric_limits<int64_t>::max() - S.Lnz[j]) {
      err = "nnz(L) overflows";
      return kOverflow;
    }
    S.nnzL += S.Lnz[j];
  }

  find_supernodes(S);
  relax_supernodes(S);
  const int64_t ns = S.ns;
  // Row structures: R_J = rows beyond J from A's lower columns in J and from
  // the children's R sets.  Children precede parents in column order.  This
  // is the exact structure of J's last column; the other columns of a
  // relaxed supernode are padded to it with explicit zeros.
  std::vector<int64_t> col2sup(n);
  for (int64_t J = 0; J < ns; J++)
    for (int64_t j = S.sfirst[J]; j < S.sfirst[J + 1]; j++) col2sup[j] = J;
  std::vector<std::vector<int32_t>> R(ns);
  std::vector<int64_t>              mark(n, -1);
  std::vector<std::vector<int32_t>> kids(ns);
  for (int64_t J = 0; J < ns; J++) {
    const int64_t last = S.sfirst[J + 1] - 1;
    if (parent[last] >= 0) kids[col2sup[parent[last]]].push_back(static_cast<int32_t>(J));
  }
  for (int64_t J = 0; J < ns; J++) {
    const int64_t f = S.sfirst[J], l = S.sfirst[J + 1];
    auto         &out = R[J];
    for (int64_t j = f; j < l; j++)
      for (int64_t p = Rp[j]; p < Rp[j + 1]; p++) {
        const int64_t r = Rj[p];
        if (r >= l && mark[r] != J) {
          mark[r] = J;
          out.push_back(static_cast<int32_t>(r));
        }
      }
    for (int32_t C : kids[J]) {
      for (int32_t r : R[C])
        if (r >= l && mark[r] != J) {
          mark[r] = J;
          out.push_back(r);
        }
      std::vector<int32_t>().swap(R[C]);  // children are done with
      R[C].clear();
    }
    std::sort(out.begin(), out.end());
    if (S.Lnz[l - 1] != static_cast<int64_t>(out.size())) {
      err = "internal: supernode structure disagrees with column counts";
      return kBadArgument;
    }
    // Stash the finished row set in srows now (children's R are freed).
    if (J == 0) S.srowptr.assign(1, 0);
    for (int64_t j = f; j < l; j++) S.srows.push_back(static_cast<int32_t>(j));
    S.srows.insert(S.srows.end(), out.begin(), out.end());
    S.srowptr.push_back(static_cast<int64_t>(S.srows.size()));
  }
  if (ns == 0) S.srowptr.assign(1, 0);
  finish_schedule(S);

  // Scatter map of the caller's entries into the panels, and scaling info.
  S.amap.resize(S.nnz);
  S.arow.resize(S.nnz);
  S.acol.resize(S.nnz);
  S.diag_pos.assign(n, -1);
  for (int64_t j0 = 0; j0 < n; j0++)
    for (int64_t p = Ap[j0]; p < Ap[j0 + 1]; p++) {
      const int64_t i0 = Ai[p];
      S.arow[p]        = static_cast<int32_t>(i0);
      S.acol[p]        = static_cast<int32_t>(j0);
      if (i0 == j0) S.diag_pos[j0] = p;
      const int64_t a = S.iperm[i0], b = S.iperm[j0];
      const int64_t i = std::min(a, b), j = std::max(a, b);
      const int64_t J = S.col2sup[i];
      const int64_t f = S.sfirst[J], l = S.sfirst[J + 1], w = l - f;
      int64_t       lr;
      if (j < l) {
        lr = j - f;
      } else {
        const int32_t *rb = S.srows.data() + S.srowptr[J] + w;
        const int32_t *re = S.srows.data() + S.srowptr[J + 1];
        const int32_t *it = std::lower_bound(rb, re, static_cast<int32_t>(j));
        lr                = w + (it - rb);
      }
      S.amap[p] = S.slofs[J] + (i - f) * S.h(J) + lr;
    }
  // Full symmetric CSR of P K P^T.
  S.Kp.assign(n + 1, 0);
  for (int64_t j0 = 0; j0 < n; j0++)
    for (int64_t p = Ap[j0]; p < Ap[j0 + 1]; p++) {
      S.Kp[S.iperm[Ai[p]] + 1]++;
      if (Ai[p] != j0) S.Kp[S.iperm[j0] + 1]++;
    }
  for (int64_t i = 0; i < n; i++) S.Kp[i + 1] += S.Kp[i];
  S.Kj.resize(S.Kp[n]);
  S.Ksrc.resize(S.Kp[n]);
  {
    // Fill column by column in permuted order so each row's columns ascend.
    std::vector<int64_t> fill(S.Kp.begin(), S.Kp.end() - 1);
    for (int64_t c = 0; c < n; c++) {
      // entries of permuted column c: (r, c) for r <= c from Ci and (r, c)
      // for r > c from the transpose; visit both in ascending row order.
      for (int64_t q = S.Cp[c]; q < S.Cp[c + 1]; q++) {
        const int64_t r   = S.Ci[q];
        const int64_t dst = fill[r]++;
        S.Kj[dst]         = static_cast<int32_t>(c);
        S.Ksrc[dst]       = S.Csrc[q];
      }
    }
    // Lower part: row r gets column c < r from the permuted upper column r.
    // The pass above put (r, c) with r <= c; now add (c', r') transposes.
    // Rows are filled in increasing column order because the pass above
    // visits columns in increasing order and the transposes below are added
    // afterwards; sort each row to restore ascending columns.
    for (int64_t c = 0; c < n; c++)
      for (int64_t q = S.Cp[c]; q < S.Cp[c + 1]; q++) {
        const int64_t r = S.Ci[q];
        if (r == c) continue;
        const int64_t dst = fill[c]++;
        S.Kj[dst]         = static_cast<int32_t>(r);
        S.Ksrc[dst]       = S.Csrc[q];
      }
    std::vector<std::pair<int32_t, int64_t>> tmp;
    for (int64_t i = 0; i < n; i++) {
      const int64_t b = S.Kp[i], e = S.Kp[i + 1];
      tmp.resize(e - b);
      for (int64_t q = b; q < e; q++) tmp[q - b] = {S.Kj[q], S.Ksrc[q]};
      std::sort(tmp.begin(), tmp.end());
      for (int64_t q = b; q < e; q++) {
        S.Kj[q]   = tmp[q - b].first;
        S.Ksrc[q] = tmp[q - b].second;
      }
    }
  }
  return kOk;
}

int analyze_from_L(int64_t n, const int64_t *Lp, const int64_t *Li,
                   Symbolic &S, std::string &err) {
  S   = Symbolic{};
  S.n = n;
  S.perm.resize(n);
  std::iota(S.perm.begin(), S.perm.end(), 0);
  S.iperm = S.perm;
  S.etree.assign(n, -1);
  S.Lnz.resize(n);
  for (int64_t j = 0; j < n; j++) {
    S.Lnz[j] = Lp[j + 1] - Lp[j];
    if (S.Lnz[j] < 0) {
      err = "column pointers decrease";
      return kBadArgument;
    }
    if (S.Lnz[j] > 0) S.etree[j] = Li[Lp[j]];
    for (int64_t p = Lp[j]; p < Lp[j + 1]; p++)
      if (Li[p] <= j || Li[p] >= n || (p > Lp[j] && Li[p] <= Li[p - 1])) {
        err = "L column " + std::to_string(j) + " is not strictly lower with ascending rows";
        return kBadArgument;
      }
  }
  S.nnzL = n > 0 ? Lp[n] : 0;
  find_supernodes(S);
  S.srowptr.assign(1, 0);
  for (int64_t J = 0; J < S.ns; J++) {
    const int64_t f = S.sfirst[J], l = S.sfirst[J + 1];
    for (int64_t j = f; j < l; j++) S.srows.push_back(static_cast<int32_t>(j));
    const int64_t last = l - 1;
    for (int64_t p = Lp[last]; p < Lp[last + 1]; p++)
      S.srows.push_back(static_cast<int32_t>(Li[p]));
    S.srowptr.push_back(static_cast<int64_t>(S.srows.size()));
    // Every column of J must be {j+1..l-1} + R_J.
    for (int64_t j = f; j < l; j++) {
      int64_t q = Lp[j];
      for (int64_t r = j + 1; r < l; r++, q++)
        if (q >= Lp[j + 1] || Li[q] != r) {
          err = "L pattern is not a factor pattern at column " + std::to_string(j);
          return kBadArgument;
        }
      for (int64_t p = Lp[last]; p < Lp[last + 1]; p++, q++)
        if (q >= Lp[j + 1] || Li[q] != Li[p]) {
          err = "L pattern is not a factor pattern at column " + std::to_string(j);
          return kBadArgument;
        }
    }
  }
  // Supernode parents must follow the pattern's elimination tree.
  finish_schedule(S);
  for (int64_t J = 0; J < S.ns; J++) {
    const int64_t P = S.sparent[J];
    if (P < 0) continue;
    for (int64_t q = S.srowptr[J] + S.w(J); q < S.srowptr[J + 1]; q++)
      if (S.srel[q] < 0) {
        err = "L pattern is not closed under its elimination tree";
        return kBadArgument;
      }
  }
  return kOk;
}

}  // namespace mpir
