// Host symbolic phase.  It must reproduce the reference's supernodal
// structure bit for bit -- the same supernode slots, the same row order inside
// each sn_struct, the same child lists -- because that structure is part of
// the drop-in contract (the factor handle exposes it and the numeric phase is
// defined on it).  The traversal orders below therefore follow the
// reference's recursions exactly; they are written as explicit-stack loops so
// that etrees that are paths of length n do not exhaust the C stack.
//
//   etree ............................. src/taucs_sn_llt.c:3243-3340
//   etree child lists (ascending) ..... src/taucs_sn_llt.c:3771-3776
//   depth guard (BFS from the root) ... src/taucs_sn_llt.c:3781-3834
//   fundamental supernodes ............ src/taucs_sn_llt.c:1377-1517
//   relaxed amalgamation .............. src/taucs_sn_llt.c:1527-1786
//     thresholds ...................... src/taucs_sn_llt.c:1715-1725
//     started from slot n_sn-1 only ... src/taucs_sn_llt.c:3925-3935
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "internal.h"

namespace tb {

int etree(int n, const int* colptr, const int* rowind, int* parent) {
  // rows of the strict lower triangle (for row i: columns j < i)
  std::vector<int> rp(n + 1, 0), ci, anc(n);
  for (int j = 0; j < n; j++)
    for (int ip = colptr[j]; ip < colptr[j + 1]; ip++)
      if (rowind[ip] > j) rp[rowind[ip] + 1]++;
  for (int i = 0; i < n; i++) rp[i + 1] += rp[i];
  ci.resize(std::max(rp[n], 1));
  std::vector<int> fill(rp.begin(), rp.end() - 1);
  for (int j = 0; j < n; j++)
    for (int ip = colptr[j]; ip < colptr[j + 1]; ip++)
      if (rowind[ip] > j) ci[fill[rowind[ip]]++] = j;
  // ancestor walk with path compression; the etree of a pattern is unique
  for (int i = 0; i < n; i++) {
    parent[i] = n;
    anc[i] = n;
    for (int kp = rp[i]; kp < rp[i + 1]; kp++) {
      int k = ci[kp];
      while (k != n && k < i) {
        int up = anc[k];
        anc[k] = i;
        if (up == n) { parent[k] = i; break; }
        k = up;
      }
    }
  }
  return 0;
}

namespace {

struct Znz { double zeros, nonzeros; };

struct SymCtx {
  int n;
  const int* colptr;
  const int* rowind;
  std::vector<int> efirst, enext;   // etree child lists
  std::vector<int> col2sn, map, tmp;
  Symbolic* S;
};

// Body of the reference's recursive_symbolic_elimination after its children
// have been visited (src/taucs_sn_llt.c:1416-1516).
bool fundamental_visit(SymCtx& c, int j) {
  Symbolic& S = *c.S;
  bool chain = true;
  if (j == c.n) chain = false;
  else if (c.efirst[j] == -1) chain = false;
  else if (c.enext[c.efirst[j]] != -1) chain = false;
  else {
    int ch = c.efirst[j];
    for (int ip = c.colptr[j]; ip < c.colptr[j + 1]; ip++)
      chain = chain && (c.map[c.rowind[ip]] == ch);
  }
  if (chain) {
    int csn = c.col2sn[c.efirst[j]];
    c.col2sn[j] = csn;
    std::vector<int>& st = S.sn_struct[csn];
    int ip = S.sn_size[csn];
    while (ip < S.sn_up_size[csn] && st[ip] != j) ip++;
    if (ip >= S.sn_up_size[csn]) return false;  // structure not nested: corrupt input
    st[ip] = st[S.sn_size[csn]];
    st[S.sn_size[csn]] = j;
    for (ip = S.sn_size[csn]; ip < S.sn_up_size[csn]; ip++) c.map[st[ip]] = j;
    S.sn_size[csn]++;
    return true;
  }
  int nnz = 0;
  if (j < c.n) {
    c.tmp[nnz++] = j;
    c.map[j] = j;
    for (int ch = c.efirst[j]; ch != -1; ch = c.enext[ch]) {
      int csn = c.col2sn[ch];
      const std::vector<int>& st = S.sn_struct[csn];
      for (int ip = S.sn_size[csn]; ip < S.sn_up_size[csn]; ip++) {
        int i = st[ip];
        if (i > j && c.map[i] != j) { c.map[i] = j; c.tmp[nnz++] = i; }
      }
    }
    for (int ip = c.colptr[j]; ip < c.colptr[j + 1]; ip++) {
      int i = c.rowind[ip];
      if (c.map[i] != j) { c.map[i] = j; c.tmp[nnz++] = i; }
    }
  }
  // first etree child's supernode heads the list; later ones are prepended
  for (int ch = c.efirst[j]; ch != -1; ch = c.enext[ch]) {
    int csn = c.col2sn[ch];
    if (ch == c.efirst[j]) S.first_child[S.n_sn] = csn;
    else { S.next_child[csn] = S.first_child[S.n_sn]; S.first_child[S.n_sn] = csn; }
  }
  if (j < c.n) {
    c.col2sn[j] = S.n_sn;
    S.sn_size[S.n_sn] = 1;
    S.sn_up_size[S.n_sn] = nnz;
    S.sn_struct[S.n_sn].assign(c.tmp.begin(), c.tmp.begin() + nnz);
    S.n_sn++;
  }
  return true;
}

// Body of recursive_amalgamate_supernodes after its children returned
// (src/taucs_sn_llt.c:1589-1785); czsum is the sum of the children's results.
Znz amalgamate_visit(SymCtx& c, int sn, Znz czsum, std::vector<double>& zcount) {
  Symbolic& S = *c.S;
  std::vector<int>& ssz = S.sn_size;
  std::vector<int>& sup = S.sn_up_size;
  Znz me;
  me.zeros = 0.0;
  // int arithmetic, as in the reference
  me.nonzeros = (double) (((sup[sn] - ssz[sn]) * ssz[sn]) + (ssz[sn] * (ssz[sn] + 1)) / 2);
  if (S.first_child[sn] == -1) return me;

  Znz merged = me;
  merged.nonzeros += czsum.nonzeros;
  merged.zeros += czsum.zeros;

  int nnz = 0;
  for (int cs = S.first_child[sn]; cs != -1; cs = S.next_child[cs])
    for (int ip = 0; ip < ssz[cs]; ip++) { int i = S.sn_struct[cs][ip]; c.map[i] = sn; c.tmp[nnz++] = i; }
  for (int ip = 0; ip < ssz[sn]; ip++) { int i = S.sn_struct[sn][ip]; c.map[i] = sn; c.tmp[nnz++] = i; }
  const int new_s = nnz;
  for (int cs = S.first_child[sn]; cs != -1; cs = S.next_child[cs])
    for (int ip = ssz[cs]; ip < sup[cs]; ip++) {
      int i = S.sn_struct[cs][ip];
      if (c.map[i] != sn) { c.map[i] = sn; c.tmp[nnz++] = i; }
    }
  for (int ip = ssz[sn]; ip < sup[sn]; ip++) {
    int i = S.sn_struct[sn][ip];
    if (c.map[i] != sn) { c.map[i] = sn; c.tmp[nnz++] = i; }
  }
  const int new_f = nnz;

  // zeros introduced per row by merging (exact integer-valued doubles)
  for (int ip = 0; ip < new_s; ip++) zcount[c.tmp[ip]] = (double) (ip + 1);
  for (int ip = new_s; ip < new_f; ip++) zcount[c.tmp[ip]] = (double) new_s;
  for (int cs = S.first_child[sn]; cs != -1; cs = S.next_child[cs]) {
    for (int ip = 0; ip < ssz[cs]; ip++) zcount[S.sn_struct[cs][ip]] -= (double) (ip + 1);
    for (int ip = ssz[cs]; ip < sup[cs]; ip++) zcount[S.sn_struct[cs][ip]] -= (double) ssz[cs];
  }
  for (int ip = 0; ip < ssz[sn]; ip++) zcount[S.sn_struct[sn][ip]] -= (double) (ip + 1);
  for (int ip = ssz[sn]; ip < sup[sn]; ip++) zcount[S.sn_struct[sn][ip]] -= (double) ssz[sn];
  for (int ip = 0; ip < new_f; ip++) merged.zeros += zcount[c.tmp[ip]];

  const bool merge = (new_s < 16)
      || ((ssz[sn] < 50) && (merged.zeros < 0.5 * merged.nonzeros))
      || ((ssz[sn] < 250) && (merged.zeros < 0.25 * merged.nonzeros))
      || ((ssz[sn] < 500) && (merged.zeros < 0.10 * merged.nonzeros))
      || (merged.zeros < 0.05 * merged.nonzeros);
  if (!merge) return me;

  ssz[sn] = new_s;
  sup[sn] = new_f;
  S.sn_struct[sn].assign(c.tmp.begin(), c.tmp.begin() + new_f);

  int nch = 0;
  for (int cs = S.first_child[sn]; cs != -1; cs = S.next_child[cs]) {
    for (int ip = 0; ip < ssz[cs]; ip++) c.col2sn[S.sn_struct[cs][ip]] = sn;
    for (int g = S.first_child[cs]; g != -1; g = S.next_child[g]) c.tmp[nch++] = g;
  }
  for (int cs = S.first_child[sn]; cs != -1; cs = S.next_child[cs]) {
    std::vector<int>().swap(S.sn_struct[cs]);
    ssz[cs] = 0;
    sup[cs] = 0;
  }
  S.first_child[sn] = -1;
  for (int k = 0; k < nch; k++) {
    S.next_child[c.tmp[k]] = S.first_child[sn];
    S.first_child[sn] = c.tmp[k];
  }
  return merged;
}

}  // namespace

int symbolic_analyze(int n, const int* colptr, const int* rowind, int max_depth, Symbolic* out) {
  Symbolic& S = *out;
  S = Symbolic();
  S.n = n;
  SymCtx c;
  c.n = n; c.colptr = colptr; c.rowind = rowind; c.S = &S;
  try {
    std::vector<int> parent(n + 1);
    etree(n, colptr, rowind, parent.data());
    c.efirst.assign(n + 1, -1);
    c.enext.assign(n + 1, -1);
    for (int j = n - 1; j >= 0; j--) { c.enext[j] = c.efirst[parent[j]]; c.efirst[parent[j]] = j; }

    // depth: number of BFS generations below the virtual root
    {
      std::vector<int> cur(1, n), nxt;
      int depth = -1;
      while (!cur.empty()) {
        nxt.clear();
        for (int v : cur)
          for (int ch = c.efirst[v]; ch != -1; ch = c.enext[ch]) nxt.push_back(ch);
        cur.swap(nxt);
        depth++;
      }
      tprintf("\t\tElimination tree depth is %d\n", depth);
      if (max_depth && depth > max_depth) {
        tprintf("taucs_ccs_symbolic_elimination: etree depth %d, maximum allowed is %d\n", depth, max_depth);
        return TAUCS_ERROR_MAXDEPTH;
      }
    }

    S.sn_size.assign(n + 1, 0);
    S.sn_up_size.assign(n + 1, 0);
    S.first_child.assign(n + 1, -1);
    S.next_child.assign(n + 1, -1);
    S.sn_struct.assign(n + 1, std::vector<int>());
    c.col2sn.assign(n + 1, -1);
    c.map.assign(n + 1, -1);
    c.tmp.assign(n + 1, 0);

    // postorder walk of the etree from the virtual root, children in list order
    {
      std::vector<int> stack, it(c.efirst);
      stack.reserve(1024);
      stack.push_back(n);
      while (!stack.empty()) {
        int j = stack.back();
        int ch = it[j];
        if (ch != -1) { it[j] = c.enext[ch]; stack.push_back(ch); continue; }
        stack.pop_back();
        if (!fundamental_visit(c, j)) return TAUCS_ERROR;
      }
    }

    // relaxed amalgamation from the last created supernode
    std::fill(c.map.begin(), c.map.end(), -1);
    if (S.n_sn > 0) {
      std::vector<double> zcount(n + 1, 0.0);
      std::vector<Znz> res(S.n_sn + 1, Znz{0.0, 0.0});
      std::vector<Znz> acc(S.n_sn + 1, Znz{0.0, 0.0});
      std::vector<int> stack, it(S.n_sn + 1, -2);
      const int root = S.n_sn - 1;
      stack.push_back(root);
      while (!stack.empty()) {
        int sn = stack.back();
        if (it[sn] == -2) it[sn] = S.first_child[sn];
        int ch = it[sn];
        if (ch != -1) { it[sn] = S.next_child[ch]; stack.push_back(ch); continue; }
        stack.pop_back();
        res[sn] = amalgamate_visit(c, sn, acc[sn], zcount);
        if (!stack.empty()) {
          int p = stack.back();
          acc[p].nonzeros += res[sn].nonzeros;
          acc[p].zeros += res[sn].zeros;
        }
      }
    }
    S.sn_size.resize(std::max(S.n_sn, 0));
    S.sn_up_size.resize(std::max(S.n_sn, 0));
    S.first_child.resize(S.n_sn + 1);
    S.next_child.resize(S.n_sn + 1);
    S.sn_struct.resize(S.n_sn);
  } catch (const std::bad_alloc&) {
    return TAUCS_ERROR_NOMEM;
  }
  return TAUCS_SUCCESS;
}

}  // namespace tb
