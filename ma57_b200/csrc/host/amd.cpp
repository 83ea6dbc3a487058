// Approximate minimum degree ordering on the quotient graph, written from the
// published algorithm (P. R. Amestoy, T. A. Davis, I. S. Duff, "An approximate
// minimum degree ordering algorithm", SIAM J. Matrix Anal. Appl. 17(4):886-905,
// 1996): element absorption, aggressive absorption, the approximate external
// degree bound of eq. (4), and supervariable detection by hashing.
//
// The reference calls SuiteSparse's amd_order (ordering.hpp:99-114); that
// library is not available here, so this is the project's own implementation
// of the same published method. Ties are broken by the most recently inserted
// variable of the minimum-degree bucket. The permutation it produces is the
// one both the GPU path and the CPU oracle consume.
#include "symbolic.hpp"

#include <algorithm>
#include <cstdint>
#include <stdexcept>

namespace symla_host {

std::vector<int> amdOrder(const CscPattern& sym) {
  const int n = sym.n;
  std::vector<int> order;
  order.reserve(n);
  if (n == 0) return order;

  // Per node state. A node is a variable until it is eliminated, when it
  // becomes an element (its id is reused).
  std::vector<std::vector<int>> Evar(n);  // elements adjacent to variable i
  std::vector<std::vector<int>> Avar(n);  // variables adjacent to variable i
  std::vector<std::vector<int>> Lel(n);   // variables of element e
  std::vector<int> nv(n, 1);              // supervariable weight (0: merged away)
  std::vector<char> isElem(n, 0);
  std::vector<char> absorbed(n, 0);       // element absorbed into another
  std::vector<int64_t> elemSize(n, 0);    // weighted |Le|
  std::vector<int> degree(n, 0);
  std::vector<std::vector<int>> members(n);  // variables merged into principal i

  for (int i = 0; i < n; ++i) {
    Avar[i].assign(sym.rowIdx.begin() + sym.colPtr[i], sym.rowIdx.begin() + sym.colPtr[i + 1]);
    degree[i] = static_cast<int>(Avar[i].size());
  }

  // Degree buckets (doubly linked lists).
  std::vector<int> head(static_cast<size_t>(n) + 1, -1), nxt(n, -1), prv(n, -1);
  auto bucketInsert = [&](int i) {
    int d = std::min(std::max(degree[i], 0), n);
    nxt[i] = head[d];
    prv[i] = -1;
    if (head[d] != -1) prv[head[d]] = i;
    head[d] = i;
  };
  auto bucketRemove = [&](int i) {
    int d = std::min(std::max(degree[i], 0), n);
    if (prv[i] != -1)
      nxt[prv[i]] = nxt[i];
    else
      head[d] = nxt[i];
    if (nxt[i] != -1) prv[nxt[i]] = prv[i];
    nxt[i] = prv[i] = -1;
  };
  for (int i = n - 1; i >= 0; --i) bucketInsert(i);

  std::vector<int64_t> w(n, 0);  // |Le \ Lme| scratch, offset by wflg
  int64_t wflg = 1;
  std::vector<int> inLme(n, -1);  // stamp: inLme[i] == me while building Lme
  std::vector<int> Lme;
  std::vector<int64_t> hashv(n, 0);
  int nel = 0;
  int mindeg = 0;

  while (nel < n) {
    while (mindeg <= n && head[mindeg] == -1) ++mindeg;
    if (mindeg > n) throw std::runtime_error("symla AMD: degree bucket underflow");
    const int me = head[mindeg];
    bucketRemove(me);

    // --- Form the new element Lme = (union of Le, e in E_me) ∪ A_me \ {me}.
    Lme.clear();
    inLme[me] = me;
    int64_t lmeSize = 0;
    for (int e : Evar[me]) {
      if (absorbed[e]) continue;
      for (int i : Lel[e]) {
        if (nv[i] == 0 || isElem[i] || inLme[i] == me) continue;
        inLme[i] = me;
        Lme.push_back(i);
        lmeSize += nv[i];
      }
      absorbed[e] = 1;  // e ⊆ Lme: absorbed into me
      std::vector<int>().swap(Lel[e]);
    }
    for (int i : Avar[me]) {
      if (nv[i] == 0 || isElem[i] || inLme[i] == me) continue;
      inLme[i] = me;
      Lme.push_back(i);
      lmeSize += nv[i];
    }
    std::vector<int>().swap(Evar[me]);
    std::vector<int>().swap(Avar[me]);
    isElem[me] = 1;
    nel += nv[me];
    order.push_back(me);

    // --- Remove Lme's variables from their buckets.
    for (int i : Lme) bucketRemove(i);

    // --- |Le \ Lme| for every element adjacent to a variable of Lme.
    if (wflg > (int64_t(1) << 60)) {
      std::fill(w.begin(), w.end(), 0);
      wflg = 1;
    }
    const int64_t wf = wflg;
    for (int i : Lme) {
      for (int e : Evar[i]) {
        if (absorbed[e] || e == me) continue;
        if (w[e] < wf) w[e] = elemSize[e] + wf;
        w[e] -= nv[i];
      }
    }

    // --- Degree update, list pruning, aggressive absorption.
    for (int i : Lme) {
      // Prune elements: drop absorbed ones and those now inside Lme.
      int64_t deg = 0;
      auto& Ei = Evar[i];
      size_t wr = 0;
      for (size_t t = 0; t < Ei.size(); ++t) {
        const int e = Ei[t];
        if (absorbed[e] || e == me) continue;
        const int64_t ext = w[e] - wf;
        if (ext <= 0) {
          absorbed[e] = 1;  // aggressive absorption: Le ⊆ Lme
          std::vector<int>().swap(Lel[e]);
          continue;
        }
        deg += ext;
        Ei[wr++] = e;
      }
      Ei.resize(wr);
      Ei.push_back(me);
      // Prune variables: drop eliminated, merged-away, and those covered by me.
      auto& Ai = Avar[i];
      wr = 0;
      for (size_t t = 0; t < Ai.size(); ++t) {
        const int j = Ai[t];
        if (isElem[j] || nv[j] == 0 || inLme[j] == me || j == i) continue;
        deg += nv[j];
        Ai[wr++] = j;
      }
      Ai.resize(wr);
      const int64_t others = lmeSize - nv[i];
      int64_t d = deg + others;
      d = std::min<int64_t>(d, static_cast<int64_t>(degree[i]) + others);
      d = std::min<int64_t>(d, static_cast<int64_t>(n - nel) - nv[i]);
      degree[i] = static_cast<int>(std::max<int64_t>(d, 0));
    }
    wflg = wf + static_cast<int64_t>(n) + 2;
    for (int i : Lme) {
      // w entries touched this step are < wflg from now on
      (void)i;
    }

    // --- Supervariable detection among Lme by hashing (E_i, A_i).
    for (int i : Lme) {
      int64_t h = 0;
      for (int e : Evar[i]) h += e;
      for (int j : Avar[i]) h += j;
      hashv[i] = h;
    }
    // Group candidates by hash: sort Lme copy by hash.
    std::vector<int> cand(Lme.begin(), Lme.end());
    std::sort(cand.begin(), cand.end(), [&](int a, int b) {
      if (hashv[a] != hashv[b]) return hashv[a] < hashv[b];
      return a < b;
    });
    for (size_t s = 0; s < cand.size();) {
      size_t t = s;
      while (t < cand.size() && hashv[cand[t]] == hashv[cand[s]]) ++t;
      for (size_t a = s; a < t; ++a) {
        const int i = cand[a];
        if (nv[i] == 0) continue;
        std::vector<int> Ei(Evar[i]), Ai(Avar[i]);
        std::sort(Ei.begin(), Ei.end());
        std::sort(Ai.begin(), Ai.end());
        for (size_t b = a + 1; b < t; ++b) {
          const int j = cand[b];
          if (nv[j] == 0) continue;
          if (Evar[j].size() != Ei.size() || Avar[j].size() != Ai.size()) continue;
          std::vector<int> Ej(Evar[j]), Aj(Avar[j]);
          std::sort(Ej.begin(), Ej.end());
          std::sort(Aj.begin(), Aj.end());
          if (Ej != Ei || Aj != Ai) continue;
          // j is indistinguishable from i: merge.
          nv[i] += nv[j];
          degree[i] -= nv[j];
          nv[j] = 0;
          members[i].push_back(j);
          for (int mm : members[j]) members[i].push_back(mm);
          std::vector<int>().swap(members[j]);
          std::vector<int>().swap(Evar[j]);
          std::vector<int>().swap(Avar[j]);
        }
      }
      s = t;
    }

    // --- New element size and re-insertion of surviving variables.
    int64_t newSize = 0;
    size_t wr = 0;
    for (int i : Lme) {
      if (nv[i] == 0) continue;
      newSize += nv[i];
      Lme[wr++] = i;
      if (degree[i] < 0) degree[i] = 0;
      bucketInsert(i);
      mindeg = std::min(mindeg, std::min(degree[i], n));
    }
    Lme.resize(wr);
    Lel[me] = Lme;
    elemSize[me] = newSize;
  }

  // Expand supervariables: each eliminated principal variable is followed by
  // the variables merged into it.
  std::vector<int> perm;
  perm.reserve(n);
  for (int p : order) {
    perm.push_back(p);
    for (int mm : members[p]) perm.push_back(mm);
  }
  if (static_cast<int>(perm.size()) != n) throw std::runtime_error("symla AMD: incomplete ordering");
  return perm;
}

}  // namespace symla_host
