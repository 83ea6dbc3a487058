// Host symbolic analysis. See symbolic.hpp for the reference mapping.
#include "symbolic.hpp"

#include <algorithm>
#include <cstdint>
#include <iterator>
#include <stdexcept>

namespace symla_host {

CscPattern symmetricPatternNoDiag(int n, const int* colptr, const int* rowind) {
  // ordering.hpp:44-75: collect (r,c) and (c,r) for every stored off-diagonal
  // entry, sort and dedupe per column. Done with a counting pass instead of
  // per-column vectors; the resulting arrays are identical.
  CscPattern out;
  out.n = n;
  std::vector<int> cnt(static_cast<size_t>(n) + 1, 0);
  for (int c = 0; c < n; ++c) {
    for (int p = colptr[c]; p < colptr[c + 1]; ++p) {
      const int r = rowind[p];
      if (r < 0 || r >= n) throw std::invalid_argument("symla: row index out of range");
      if (r == c) continue;
      ++cnt[c + 1];
      ++cnt[r + 1];
    }
  }
  for (int c = 0; c < n; ++c) cnt[c + 1] += cnt[c];
  std::vector<int> tmp(cnt[n]);
  std::vector<int> pos(cnt.begin(), cnt.end() - 1);
  for (int c = 0; c < n; ++c) {
    for (int p = colptr[c]; p < colptr[c + 1]; ++p) {
      const int r = rowind[p];
      if (r == c) continue;
      tmp[pos[c]++] = r;
      tmp[pos[r]++] = c;
    }
  }
  out.colPtr.assign(static_cast<size_t>(n) + 1, 0);
  out.rowIdx.clear();
  out.rowIdx.reserve(tmp.size());
  for (int c = 0; c < n; ++c) {
    auto b = tmp.begin() + cnt[c];
    auto e = tmp.begin() + cnt[c + 1];
    std::sort(b, e);
    auto u = std::unique(b, e);
    out.rowIdx.insert(out.rowIdx.end(), b, u);
    out.colPtr[c + 1] = static_cast<int>(out.rowIdx.size());
  }
  return out;
}

CscPattern permutedSymmetricPattern(const CscPattern& sym, const std::vector<int>& newIndexOf) {
  const int n = sym.n;
  CscPattern out;
  out.n = n;
  out.colPtr.assign(static_cast<size_t>(n) + 1, 0);
  for (int c = 0; c < n; ++c) out.colPtr[newIndexOf[c] + 1] = sym.colPtr[c + 1] - sym.colPtr[c];
  for (int c = 0; c < n; ++c) out.colPtr[c + 1] += out.colPtr[c];
  out.rowIdx.resize(sym.rowIdx.size());
  for (int c = 0; c < n; ++c) {
    const int nc = newIndexOf[c];
    int w = out.colPtr[nc];
    for (int p = sym.colPtr[c]; p < sym.colPtr[c + 1]; ++p) out.rowIdx[w++] = newIndexOf[sym.rowIdx[p]];
    std::sort(out.rowIdx.begin() + out.colPtr[nc], out.rowIdx.begin() + out.colPtr[nc + 1]);
  }
  return out;
}

std::vector<int> computeOrdering(const CscPattern& sym, OrderingType type) {
  const int n = sym.n;
  if (type == OrderingType::Natural) {
    std::vector<int> perm(n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    return perm;
  }
  if (type == OrderingType::AMD) return amdOrder(sym);
  if (type == OrderingType::Metis || type == OrderingType::MetisIperm) {
    if (n == 0) return {};
    return metisOrder(sym, type == OrderingType::MetisIperm);
  }
  throw std::invalid_argument("symla::computeOrdering: unknown OrderingType");
}

std::vector<int> eliminationTreeParent(const CscPattern& P) {
  // elimination_tree.hpp:78-96 -- Liu's algorithm with path compression.
  const int n = P.n;
  std::vector<int> parent(n, -1), ancestor(n, -1);
  for (int j = 0; j < n; ++j) {
    for (int idx = P.colPtr[j]; idx < P.colPtr[j + 1]; ++idx) {
      const int i = P.rowIdx[idx];
      if (i >= j) continue;
      int r = i;
      while (ancestor[r] != -1 && ancestor[r] != j) {
        const int t = ancestor[r];
        ancestor[r] = j;
        r = t;
      }
      if (ancestor[r] == -1) {
        ancestor[r] = j;
        parent[r] = j;
      }
    }
  }
  return parent;
}

EliminationTree columnStructure(const CscPattern& P, std::vector<Supernode>* fundamental,
                                std::vector<Supernode>* groups) {
  // Struct(L*j) = (Struct(A*j) ∩ {i>j}) ∪ children's structures minus the
  // child itself (elimination_tree.hpp:98-131), formed by merging sorted
  // lists: the column's own entries below
  // the diagonal (sorted in P) and each child's structure without the child
  // (sorted, all >= j). A column's structure lives only until its parent has
  // consumed it; what the callers need of it is kept on the way:
  //  - fundamental: the supernodes of symbolic.hpp:229-247 (column j
  //    continues the previous one's iff parent[j-1] == j and colCount[j-1]
  //    == colCount[j] + 1), each with its first column's structure;
  //  - groups: for given contiguous column groups, the sorted union of their
  //    columns' structures (symbolic.hpp:385-396) as each group's rowPattern.
  const int n = P.n;
  EliminationTree tree;
  tree.n = n;
  tree.parent = eliminationTreeParent(P);
  tree.colCount.assign(n, 0);
  std::vector<int> headChild(n, -1), nextSib(n, -1);
  for (int j = n - 1; j >= 0; --j) {
    const int p = tree.parent[j];
    if (p != -1) {
      nextSib[j] = headChild[p];
      headChild[p] = j;
    }
  }
  if (fundamental) fundamental->clear();
  std::vector<std::vector<int>> pats(n);
  std::vector<int> cur, tmp;
  std::vector<int> mark(n, -1), gwork;
  size_t g = 0;  // current group
  for (int j = 0; j < n; ++j) {
    cur.assign(1, j);
    {
      const int* b = P.rowIdx.data() + P.colPtr[j];
      const int* e = P.rowIdx.data() + P.colPtr[j + 1];
      cur.insert(cur.end(), std::upper_bound(b, e, j), e);
    }
    for (int c = headChild[j]; c != -1; c = nextSib[c]) {
      const auto& cp = pats[c];
      tmp.clear();
      std::set_union(cur.begin(), cur.end(), cp.begin() + 1, cp.end(), std::back_inserter(tmp));
      cur.swap(tmp);
      std::vector<int>().swap(pats[c]);
    }
    tree.colCount[j] = static_cast<int>(cur.size());
    if (fundamental) {
      const bool continues = j > 0 && tree.parent[j - 1] == j && tree.colCount[j - 1] == tree.colCount[j] + 1;
      if (continues) {
        ++fundamental->back().ncols;
      } else {
        Supernode sn;
        sn.firstCol = j;
        sn.ncols = 1;
        sn.rowPattern = cur;
        fundamental->push_back(std::move(sn));
      }
    }
    if (groups && g < groups->size()) {
      Supernode& G = (*groups)[g];
      for (int i : cur)
        if (mark[i] != static_cast<int>(g)) {
          mark[i] = static_cast<int>(g);
          gwork.push_back(i);
        }
      if (j == G.firstCol + G.ncols - 1) {
        std::sort(gwork.begin(), gwork.end());
        G.rowPattern = gwork;
        gwork.clear();
        ++g;
      }
    }
    if (tree.parent[j] != -1) pats[j].swap(cur);
  }
  return tree;
}

std::vector<int> postorder(const std::vector<int>& parent) {
  const int n = static_cast<int>(parent.size());
  // children lists in increasing index order; roots in increasing order.
  std::vector<int> head(n, -1), next(n, -1);
  std::vector<int> roots;
  for (int j = n - 1; j >= 0; --j) {
    const int p = parent[j];
    if (p != -1) {
      next[j] = head[p];
      head[p] = j;
    }
  }
  for (int j = 0; j < n; ++j)
    if (parent[j] == -1) roots.push_back(j);
  std::vector<int> order;
  order.reserve(n);
  // Iterative DFS reproducing the recursive visit(node): visit children in
  // order, then emit node.
  std::vector<int> stack;
  std::vector<int> cursor(n, -2);  // -2: not started
  for (int r : roots) {
    stack.push_back(r);
    while (!stack.empty()) {
      const int v = stack.back();
      if (cursor[v] == -2) cursor[v] = head[v];
      const int c = cursor[v];
      if (c != -1) {
        cursor[v] = next[c];
        stack.push_back(c);
      } else {
        order.push_back(v);
        stack.pop_back();
      }
    }
  }
  return order;
}

namespace {

std::int64_t storageNnzOf(int ncols, size_t m) {
  const std::int64_t k = ncols;
  const std::int64_t mm = static_cast<std::int64_t>(m);
  return k * mm - k * (k - 1) / 2;
}

}  // namespace

SymbolicFactor analyze(int n, const int* colptr, const int* rowind, OrderingType ordering,
                       const SymbolicFactorOptions& options) {
  SymbolicFactor sf;
  if (n < 0) throw std::invalid_argument("symla::analyze: negative size");
  if (n == 0) {
    sf.etree.n = 0;
    return sf;
  }
  const CscPattern sym = symmetricPatternNoDiag(n, colptr, rowind);

  // Step 1-2 (symbolic.hpp:206-208)
  std::vector<int> perm0 = computeOrdering(sym, ordering);
  if (static_cast<int>(perm0.size()) != n) throw std::runtime_error("symla::analyze: ordering has wrong size");
  std::vector<int> newIndexOf(n);
  for (int k = 0; k < n; ++k) newIndexOf[perm0[k]] = k;
  CscPattern A0 = permutedSymmetricPattern(sym, newIndexOf);

  // Step 3 (symbolic.hpp:212-216)
  std::vector<int> postNodes = postorder(eliminationTreeParent(A0));
  std::vector<int> finalPerm(n);
  for (int k = 0; k < n; ++k) finalPerm[k] = perm0[postNodes[k]];
  for (int k = 0; k < n; ++k) newIndexOf[finalPerm[k]] = k;
  CscPattern A1 = permutedSymmetricPattern(sym, newIndexOf);

  // Step 4-5 (symbolic.hpp:222-247)
  std::vector<Supernode> funda;
  EliminationTree tree = columnStructure(A1, &funda, nullptr);
  const int numFunda = static_cast<int>(funda.size());

  // Step 6a (symbolic.hpp:253-267)
  std::vector<int> colToFunda(n, -1);
  for (int i = 0; i < numFunda; ++i)
    for (int c = funda[i].firstCol; c < funda[i].firstCol + funda[i].ncols; ++c) colToFunda[c] = i;
  std::vector<int> parentFunda(numFunda, -1);
  std::vector<std::vector<int>> childrenFunda(numFunda);
  for (int i = 0; i < numFunda; ++i) {
    const int lastCol = funda[i].firstCol + funda[i].ncols - 1;
    const int p = tree.parent[lastCol];
    if (p != -1) {
      const int pf = colToFunda[p];
      parentFunda[i] = pf;
      childrenFunda[pf].push_back(i);
    }
  }

  // Step 6b (symbolic.hpp:275-329): union-find relaxed amalgamation.
  std::vector<int> dsu(numFunda);
  for (int i = 0; i < numFunda; ++i) dsu[i] = i;
  auto find = [&](int x) {
    while (dsu[x] != x) {
      dsu[x] = dsu[dsu[x]];
      x = dsu[x];
    }
    return x;
  };
  struct Agg {
    int ncols = 0;
    std::vector<int> rowPattern;
    std::vector<int> segments;
  };
  std::vector<Agg> agg(numFunda);
  for (int i = 0; i < numFunda; ++i) {
    agg[i].ncols = funda[i].ncols;
    agg[i].rowPattern = funda[i].rowPattern;
    agg[i].segments = {i};
  }
  std::vector<int> mergedPattern;
  for (int i = 0; i < numFunda; ++i) {
    for (int c : childrenFunda[i]) {
      const int cr = find(c);
      if (cr == i) continue;
      const int mergedNcols = agg[i].ncols + agg[cr].ncols;
      if (mergedNcols > options.max_relax_size) continue;
      mergedPattern.clear();
      mergedPattern.reserve(agg[i].rowPattern.size() + agg[cr].rowPattern.size());
      std::set_union(agg[i].rowPattern.begin(), agg[i].rowPattern.end(), agg[cr].rowPattern.begin(),
                     agg[cr].rowPattern.end(), std::back_inserter(mergedPattern));
      const std::int64_t mergedStorage = storageNnzOf(mergedNcols, mergedPattern.size());
      const std::int64_t origStorage = storageNnzOf(agg[i].ncols, agg[i].rowPattern.size()) +
                                       storageNnzOf(agg[cr].ncols, agg[cr].rowPattern.size());
      const double extraFrac = static_cast<double>(mergedStorage - origStorage) / static_cast<double>(mergedStorage);
      if (extraFrac > options.max_relax_fill_fraction) continue;
      dsu[cr] = i;
      agg[i].ncols = mergedNcols;
      agg[i].rowPattern.swap(mergedPattern);
      agg[i].segments.insert(agg[i].segments.end() - 1, agg[cr].segments.begin(), agg[cr].segments.end());
      std::vector<int>().swap(agg[cr].rowPattern);
    }
  }

  // Step 6c (symbolic.hpp:335-349)
  std::vector<int> finalRoots;
  for (int i = 0; i < numFunda; ++i)
    if (find(i) == i) finalRoots.push_back(i);
  const int numFinal = static_cast<int>(finalRoots.size());
  std::vector<int> compactOf(numFunda, -1);
  for (int k = 0; k < numFinal; ++k) compactOf[finalRoots[k]] = k;
  std::vector<int> finalParentCompact(numFinal);
  for (int k = 0; k < numFinal; ++k) {
    const int r = finalRoots[k];
    const int pf = parentFunda[r];
    finalParentCompact[k] = (pf == -1) ? -1 : compactOf[find(pf)];
  }
  std::vector<int> groupPostorder = postorder(finalParentCompact);

  // Step 6d (symbolic.hpp:353-366)
  std::vector<Supernode> finalSupernodes;
  finalSupernodes.reserve(numFinal);
  std::vector<int> newOrder;
  newOrder.reserve(n);
  for (int gk : groupPostorder) {
    const int r = finalRoots[gk];
    Supernode sn;
    sn.firstCol = static_cast<int>(newOrder.size());
    sn.ncols = agg[r].ncols;
    for (int fi : agg[r].segments)
      for (int c = funda[fi].firstCol; c < funda[fi].firstCol + funda[fi].ncols; ++c) newOrder.push_back(c);
    finalSupernodes.push_back(std::move(sn));
  }
  std::vector<Agg>().swap(agg);
  std::vector<Supernode>().swap(funda);

  // Step 6e (symbolic.hpp:372-381)
  std::vector<int> combinedPerm(n);
  for (int k = 0; k < n; ++k) combinedPerm[k] = finalPerm[newOrder[k]];
  for (int k = 0; k < n; ++k) newIndexOf[combinedPerm[k]] = k;
  CscPattern A2 = permutedSymmetricPattern(sym, newIndexOf);
  // and Step 6f (symbolic.hpp:385-396): each final supernode's pattern is the
  // union of its member columns' patterns
  sf.etree = columnStructure(A2, &sf.fundamentalSupernodes, &finalSupernodes);
  sf.perm = combinedPerm;
  sf.supernodes = std::move(finalSupernodes);
  return sf;
}

}  // namespace symla_host
