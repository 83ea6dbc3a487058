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
  if (type == OrderingType::Metis) {
    if (n == 0) return {};
    return metisOrder(sym);
  }
  throw std::invalid_argument("symla::computeOrdering: unknown OrderingType");
}

EliminationTree buildEliminationTree(const CscPattern& P, std::vector<std::vector<int>>* rowPatterns) {
  const int n = P.n;
  EliminationTree tree;
  tree.n = n;
  tree.parent.assign(n, -1);
  tree.colCount.assign(n, 0);
  if (n == 0) {
    if (rowPatterns) rowPatterns->clear();
    return tree;
  }
  // elimination_tree.hpp:78-96 -- Liu's algorithm with path compression.
  std::vector<int> ancestor(n, -1);
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
        tree.parent[r] = j;
      }
    }
  }
  // elimination_tree.hpp:98-131 -- Struct(L*j) = (Struct(A*j) ∩ {i>j}) ∪
  // children's patterns minus the child itself. Computed with a marker array
  // and one sort per column (the set is unique, so the result is identical
  // to the reference's repeated set_union).
  std::vector<int> headChild(n, -1), nextSib(n, -1);
  for (int j = n - 1; j >= 0; --j) {
    const int p = tree.parent[j];
    if (p != -1) {
      nextSib[j] = headChild[p];
      headChild[p] = j;
    }
  }
  std::vector<std::vector<int>> pats(n);
  std::vector<int> mark(n, -1);
  std::vector<int> work;
  for (int j = 0; j < n; ++j) {
    work.clear();
    work.push_back(j);
    mark[j] = j;
    for (int idx = P.colPtr[j]; idx < P.colPtr[j + 1]; ++idx) {
      const int i = P.rowIdx[idx];
      if (i > j && mark[i] != j) {
        mark[i] = j;
        work.push_back(i);
      }
    }
    for (int c = headChild[j]; c != -1; c = nextSib[c]) {
      const auto& cp = pats[c];
      for (size_t t = 1; t < cp.size(); ++t) {
        const int i = cp[t];
        if (mark[i] != j) {
          mark[i] = j;
          work.push_back(i);
        }
      }
      if (!rowPatterns) std::vector<int>().swap(pats[c]);
    }
    std::sort(work.begin(), work.end());
    tree.colCount[j] = static_cast<int>(work.size());
    pats[j] = work;
  }
  if (rowPatterns) *rowPatterns = std::move(pats);
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

std::vector<Supernode> computeFundamentalSupernodes(const EliminationTree& t,
                                                    const std::vector<std::vector<int>>& patterns) {
  // symbolic.hpp:229-247
  std::vector<Supernode> out;
  const int nn = t.n;
  int j = 0;
  while (j < nn) {
    const int start = j;
    while (j + 1 < nn && t.parent[j] == j + 1 && t.colCount[j] == t.colCount[j + 1] + 1) ++j;
    Supernode sn;
    sn.firstCol = start;
    sn.ncols = j - start + 1;
    sn.rowPattern = patterns[start];
    out.push_back(std::move(sn));
    ++j;
  }
  return out;
}

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
  EliminationTree tree0 = buildEliminationTree(A0, nullptr);
  std::vector<int> postNodes = postorder(tree0.parent);
  std::vector<int> finalPerm(n);
  for (int k = 0; k < n; ++k) finalPerm[k] = perm0[postNodes[k]];
  for (int k = 0; k < n; ++k) newIndexOf[finalPerm[k]] = k;
  CscPattern A1 = permutedSymmetricPattern(sym, newIndexOf);

  // Step 4 (symbolic.hpp:222-226)
  std::vector<std::vector<int>> rowPatterns;
  EliminationTree tree = buildEliminationTree(A1, &rowPatterns);

  // Step 5
  std::vector<Supernode> funda = computeFundamentalSupernodes(tree, rowPatterns);
  std::vector<std::vector<int>>().swap(rowPatterns);
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
  std::vector<std::vector<int>> rowPatterns2;
  EliminationTree tree2 = buildEliminationTree(A2, &rowPatterns2);
  sf.perm = combinedPerm;
  sf.etree = tree2;
  sf.fundamentalSupernodes = computeFundamentalSupernodes(tree2, rowPatterns2);

  // Step 6f (symbolic.hpp:385-396): union of member columns' patterns.
  std::vector<int> mark(n, -1);
  std::vector<int> work;
  for (size_t s = 0; s < finalSupernodes.size(); ++s) {
    auto& sn = finalSupernodes[s];
    work.clear();
    for (int c = sn.firstCol; c < sn.firstCol + sn.ncols; ++c) {
      for (int i : rowPatterns2[c]) {
        if (mark[i] != static_cast<int>(s)) {
          mark[i] = static_cast<int>(s);
          work.push_back(i);
        }
      }
    }
    std::sort(work.begin(), work.end());
    sn.rowPattern = work;
  }
  sf.supernodes = std::move(finalSupernodes);
  return sf;
}

}  // namespace symla_host
