// Approximate minimum degree ordering, without aggressive absorption.
//
// The reference orders with the vendored AMDBAR routine (f2c'd Fortran,
// external/src/amdbar.c:8, called from src/taucs_ccs_order.c:87-256), the
// "variation 2" of the MC47/AMD family described in P. Amestoy, T. Davis and
// I. Duff, "An approximate minimum degree ordering algorithm", SIAM J. Matrix
// Anal. Appl. 17(4), 1996: quotient-graph elimination with approximate
// external degrees, element absorption, mass elimination and supervariable
// detection by hashing, followed by a postorder numbering of non-principal
// variables.  This file restates that published algorithm in C++ (per-node
// lists instead of one workspace array with garbage collection; separate
// hash-bucket heads instead of sharing the degree-list heads).  Every step
// that decides the ORDER is kept identical -- list construction order from
// the CCS traversal (src/taucs_ccs_order.c:190-209), degree lists with head
// insertion, the scan order that builds each new element, the in-place list
// pruning and rotation that puts the new element first, the 1-based hash
// sums modulo max(1,n-1), bucket scanning order, reinsertion order and the
// final numbering -- because the permutation must match the reference's bit
// for bit.  Memory layout and workspace compaction do not influence the
// result and are not reproduced.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "internal.h"

namespace tb {

int amd_order(int n, const int* colptr, const int* rowind, int* perm, int* invperm) {
  if (n <= 0) return 0;
  constexpr int NONE = -1;
  std::vector<std::vector<int>> lst(n);
  // adjacency lists in the order the reference fills its workspace
  {
    std::vector<int> cnt(n, 0);
    for (int j = 0; j < n; j++)
      for (int ip = colptr[j]; ip < colptr[j + 1]; ip++) {
        const int i = rowind[ip];
        if (i != j) { cnt[i]++; cnt[j]++; }
      }
    for (int i = 0; i < n; i++) lst[i].reserve(cnt[i]);
    for (int j = 0; j < n; j++)
      for (int ip = colptr[j]; ip < colptr[j + 1]; ip++) {
        const int i = rowind[ip];
        if (i != j) { lst[i].push_back(j); lst[j].push_back(i); }
      }
  }
  std::vector<int> elen(n, 0), nv(n, 1), degree(n), next(n, NONE), last(n, NONE), link(n, NONE);
  std::vector<int64_t> w(n, 1);
  std::vector<int> head(n + 1, NONE);                       // degree lists, degrees 1..n
  const int hmod = std::max(1, n - 1);
  std::vector<int> bucket(hmod + 1, NONE);                  // hash buckets 1..hmod
  int64_t wflg = 2;
  int mindeg = 1, nel = 0, dmax = 0;

  for (int i = 0; i < n; i++) degree[i] = (int) lst[i].size();
  for (int i = 0; i < n; i++) {
    const int deg = degree[i];
    if (deg > 0) {
      const int inext = head[deg];
      if (inext != NONE) last[inext] = i;
      next[i] = inext;
      head[deg] = i;
    } else {
      nel++;
      elen[i] = -nel;
      w[i] = 0;
    }
  }

  std::vector<int> lme;
  lme.reserve(1024);
  while (nel < n) {
    // pivot: head of the lowest nonempty degree list
    int deg = mindeg, me = NONE;
    for (; deg <= n; deg++) {
      me = head[deg];
      if (me != NONE) break;
    }
    mindeg = deg;
    {
      const int inext = next[me];
      if (inext != NONE) last[inext] = NONE;
      head[deg] = inext;
    }
    const int elenme = elen[me];
    elen[me] = -(nel + 1);
    int nvpiv = nv[me];
    nel += nvpiv;
    nv[me] = -nvpiv;
    int degme = 0;

    // the new element: variables of me's elements, then me's own variables
    lme.clear();
    auto take = [&](int i) {
      const int nvi = nv[i];
      if (nvi <= 0) return;
      degme += nvi;
      nv[i] = -nvi;
      lme.push_back(i);
      const int ilast = last[i], inext = next[i];
      if (inext != NONE) last[inext] = ilast;
      if (ilast != NONE) next[ilast] = inext;
      else head[degree[i]] = inext;
    };
    {
      std::vector<int>& lm = lst[me];
      for (int k = 0; k < elenme; k++) {
        const int e = lm[k];
        for (int i : lst[e]) take(i);
        link[e] = me;       // element e absorbed into me
        w[e] = 0;
        std::vector<int>().swap(lst[e]);
      }
      for (size_t p = (size_t) elenme; p < lm.size(); p++) take(lm[p]);
    }
    degree[me] = degme;

    // |Le \ Lme| for every element e adjacent to a variable of Lme
    for (int i : lme) {
      const int eln = elen[i];
      if (eln > 0) {
        const int nvi = -nv[i];
        const int64_t wnvi = wflg - nvi;
        for (int p = 0; p < eln; p++) {
          const int e = lst[i][p];
          int64_t we = w[e];
          if (we >= wflg) we -= nvi;
          else if (we != 0) we = degree[e] + wnvi;
          w[e] = we;
        }
      }
    }

    // degree bounds, list pruning, mass elimination, hashing
    for (int i : lme) {
      std::vector<int>& li = lst[i];
      const int eln_old = elen[i];
      int pn = 0;
      int64_t hash = 0;
      int64_t dg = 0;
      for (int p = 0; p < eln_old; p++) {
        const int e = li[p];
        const int64_t we = w[e];
        if (we != 0) {
          dg += we - wflg;
          li[pn++] = e;
          hash += e + 1;
        }
      }
      elen[i] = pn + 1;
      const int p3 = pn;
      for (size_t p = (size_t) eln_old; p < li.size(); p++) {
        const int j = li[p];
        const int nvj = nv[j];
        if (nvj > 0) {
          dg += nvj;
          li[pn++] = j;
          hash += j + 1;
        }
      }
      if (elen[i] == 1 && p3 == pn) {
        // mass elimination: i is adjacent only to me
        link[i] = me;
        const int nvi = -nv[i];
        degme -= nvi;
        nvpiv += nvi;
        nel += nvi;
        nv[i] = 0;
        elen[i] = 0;
        std::vector<int>().swap(li);
      } else {
        degree[i] = (int) std::min<int64_t>(degree[i], dg);
        // me goes first; the old first element and first variable rotate
        li[pn] = li[p3];
        li[p3] = li[0];
        li[0] = me;
        li.resize(pn + 1);
        const int h = (int) (hash % hmod) + 1;
        next[i] = bucket[h];
        bucket[h] = i;
        last[i] = h;
      }
    }
    degree[me] = degme;
    dmax = std::max(dmax, degme);
    wflg += dmax;

    // supervariable detection within each hash bucket
    for (int i0 : lme) {
      if (nv[i0] >= 0) continue;
      const int h = last[i0];
      int i = bucket[h];
      if (i == NONE) continue;
      bucket[h] = NONE;
      while (i != NONE) {
        if (next[i] == NONE) break;
        const std::vector<int>& li = lst[i];
        const size_t ln = li.size();
        const int eln = elen[i];
        for (size_t p = 1; p < ln; p++) w[li[p]] = wflg;
        int jlast = i, j = next[i];
        while (j != NONE) {
          const std::vector<int>& lj = lst[j];
          bool same = lj.size() == ln && elen[j] == eln;
          for (size_t p = 1; same && p < ln; p++) same = (w[lj[p]] == wflg);
          if (same) {
            link[j] = i;
            nv[i] += nv[j];
            nv[j] = 0;
            elen[j] = 0;
            std::vector<int>().swap(lst[j]);
            j = next[j];
            next[jlast] = j;
          } else {
            jlast = j;
            j = next[j];
          }
        }
        wflg++;
        i = next[i];
      }
    }

    // reinsert the principal variables of Lme into the degree lists
    const int nleft = n - nel;
    size_t p = 0;
    for (size_t q = 0; q < lme.size(); q++) {
      const int i = lme[q];
      const int nvi = -nv[i];
      if (nvi > 0) {
        nv[i] = nvi;
        const int d = std::max(1, std::min(degree[i] + degme - nvi, nleft - nvi));
        const int inext = head[d];
        if (inext != NONE) last[inext] = i;
        next[i] = inext;
        last[i] = NONE;
        head[d] = i;
        mindeg = std::min(mindeg, d);
        degree[i] = d;
        lme[p++] = i;
      }
    }
    nv[me] = nvpiv + degme;
    lst[me].assign(lme.begin(), lme.begin() + p);
    if (p == 0) w[me] = 0;
  }

  // number non-principal variables just before their representative element
  for (int i = 0; i < n; i++) {
    if (elen[i] != 0) continue;
    int j = link[i];
    while (elen[j] >= 0) j = link[j];
    const int e = j;
    int k = -elen[e];
    j = i;
    while (elen[j] >= 0) {
      const int jn = link[j];
      link[j] = e;
      if (elen[j] == 0) elen[j] = k++;
      j = jn;
    }
    elen[e] = -k;
  }
  for (int i = 0; i < n; i++) {
    const int k = elen[i] < 0 ? -elen[i] : elen[i];
    perm[k - 1] = i;
  }
  for (int k = 0; k < n; k++) invperm[perm[k]] = k;
  return 0;
}

}  // namespace tb
