// Multiple minimum external degree ordering (host), bit-identical with the
// reference's "genmmd" ordering.
//
// The algorithm is J. W. H. Liu's multiple minimum-degree method ("Modification
// of the minimum-degree algorithm by multiple elimination", ACM TOMS 11(2),
// 1985): minimum degree on the quotient graph of the elimination graph, with
// indistinguishable nodes merged into supernodes, external degrees, and every
// node of degree <= mindeg + delta eliminated before the degrees are updated.
// The reference vendors SPARSPAK's implementation (external/src/genmmd.c,
// genmmd_ :56, mmdint_ :235, mmdelm_ :310, mmdupd_ :575, mmdnum_ :945) and
// drives it from taucs_ccs_genmmd (src/taucs_ccs_order.c:262-442) with
// delta = 1 and maxint = 2^31 - 1.  The permutation depends on the order in
// which the quotient graph's lists are written and read (ties between nodes
// of equal degree are broken by list order), so the storage discipline is
// the published one: every node's adjacency lives in its own segment of one
// array, an eliminated node's segment is reused for the element it becomes,
// a negative entry -e continues the list in the segment of element e, and a
// zero ends it.  Nodes are numbered 1..n inside this file (0 ends a list).
#include <climits>
#include <vector>

#include "internal.h"

namespace tb {

namespace {

struct MmdState {
  int n = 0;
  int delta = 1;
  int maxint = INT_MAX;
  std::vector<int> xadj;     // segment of node v: [xadj[v], xadj[v + 1])
  std::vector<int> adj;      // node ids, -e links, 0 terminators
  std::vector<int> head;     // head[d]: first node of external degree d - 1
  std::vector<int> fwd;      // degree-list successor; < 0 once eliminated (-number) or merged (-target)
  std::vector<int> bwd;      // degree-list predecessor, -d at a list head, 0 = needs update, -maxint = inactive
  std::vector<int> qsize;    // nodes represented by a supernode (0: merged away)
  std::vector<int> link;     // temporary singly linked lists
  std::vector<int> mark;     // marker values compared with the running tag
  int tag = 1;

  // Calls visit(v) for every positive entry of the list that starts in the
  // segment of `start`, following -e links; stops at a zero or at the end
  // of a segment, or when visit returns false.
  template <typename Visit>
  void walk(int start, Visit visit) const {
    int seg = start;
    for (;;) {
      int next = 0;
      for (int i = xadj[seg]; i < xadj[seg + 1]; i++) {
        const int v = adj[i];
        if (v < 0) { next = -v; break; }
        if (v == 0) return;
        if (!visit(v)) return;
      }
      if (next == 0) return;
      seg = next;
    }
  }

  void reset_marks() {
    tag = 1;
    for (int i = 1; i <= n; i++)
      if (mark[i] < maxint) mark[i] = 0;
  }

  // Degree lists indexed by degree, every node in the list of its initial
  // degree (its number of neighbours + 1), pushed at the head in node order.
  void init() {
    for (int v = 1; v <= n; v++) {
      head[v] = 0;
      qsize[v] = 1;
      mark[v] = 0;
      link[v] = 0;
    }
    for (int v = 1; v <= n; v++) {
      const int d = xadj[v + 1] - xadj[v] + 1;
      const int first = head[d];
      fwd[v] = first;
      head[d] = v;
      if (first > 0) bwd[first] = v;
      bwd[v] = -d;
    }
  }

  void unlink_from_degree_list(int v) {
    const int prev = bwd[v];
    if (prev == 0 || prev == -maxint) return;
    const int next = fwd[v];
    if (next > 0) bwd[next] = prev;
    if (prev > 0) fwd[prev] = next;
    if (prev < 0) head[-prev] = next;
  }

  void push_degree_list(int v, int d) {
    const int first = head[d];
    fwd[v] = first;
    bwd[v] = -d;
    if (first > 0) bwd[first] = v;
    head[d] = v;
  }

  // Eliminates node p: its reachable set (uneliminated neighbours, and the
  // uneliminated members of the elements adjacent to it) is written into
  // p's segment, continuing into the absorbed elements' segments; then every
  // reachable node drops the neighbours now covered by element p, and either
  // is merged into p (nothing else left) or gets p as a neighbour and is
  // flagged for a degree update.
  void eliminate(int p) {
    mark[p] = tag;
    int elements = 0;                       // absorbed elements, linked through `link`
    int wpos = xadj[p], wend = xadj[p + 1] - 1;
    for (int i = xadj[p]; i <= wend; i++) {
      const int v = adj[i];
      if (v == 0) break;
      if (mark[v] >= tag) continue;
      mark[v] = tag;
      if (fwd[v] < 0) {
        link[v] = elements;
        elements = v;
      } else {
        adj[wpos++] = v;
      }
    }
    for (int e = elements; e > 0; e = link[e]) {
      adj[wend] = -e;                       // the list being written continues in e's segment
      walk(e, [&](int v) {
          if (mark[v] >= tag || fwd[v] < 0) return true;
          mark[v] = tag;
          while (wpos >= wend) {            // segment full: continue in the next linked one
            const int nxt = -adj[wend];
            wpos = xadj[nxt];
            wend = xadj[nxt + 1] - 1;
          }
          adj[wpos++] = v;
          return true;
        });
    }
    if (wpos <= wend) adj[wpos] = 0;

    walk(p, [&](int r) {
      unlink_from_degree_list(r);
      const int beg = xadj[r], end = xadj[r + 1] - 1;
      int keep = beg;
      for (int j = beg; j <= end; j++) {
        const int v = adj[j];
        if (v == 0) break;
        if (mark[v] >= tag) continue;
        adj[keep++] = v;
      }
      const int left = keep - beg;
      if (left <= 0) {
        qsize[p] += qsize[r];
        qsize[r] = 0;
        mark[r] = maxint;
        fwd[r] = -p;
        bwd[r] = -maxint;
      } else {
        fwd[r] = left + 1;
        bwd[r] = 0;
        adj[keep++] = p;
        if (keep <= end) adj[keep] = 0;
      }
      return true;
    });
  }

  // External degree of every node flagged by the eliminations of one
  // multiple-elimination step (the new elements are linked from `elems`).
  // Nodes with exactly two list entries (the element and one more) are
  // handled first: another such node of the same two elements is merged
  // into them, a node adjacent to more is marked as outmatched.
  void update(int elems, int* mdeg) {
    const int mdeg0 = *mdeg + delta;
    for (int e = elems; e > 0; e = link[e]) {
      int mtag = tag + mdeg0;
      if (mtag >= maxint) {
        reset_marks();
        mtag = tag + mdeg0;
      }
      int q2 = 0, qx = 0, deg0 = 0;
      walk(e, [&](int v) {
        if (qsize[v] == 0) return true;
        deg0 += qsize[v];
        mark[v] = mtag;
        if (bwd[v] != 0) return true;
        if (fwd[v] == 2) {
          link[v] = q2;
          q2 = v;
        } else {
          link[v] = qx;
          qx = v;
        }
        return true;
      });
      for (int v = q2; v > 0; v = link[v]) {
        if (bwd[v] != 0) continue;
        tag++;
        int deg = deg0;
        int other = adj[xadj[v]];
        if (other == e) other = adj[xadj[v] + 1];
        if (fwd[other] >= 0) {
          deg += qsize[other];
        } else {
          walk(other, [&](int u) {
            if (u == v || qsize[u] == 0) return true;
            if (mark[u] < tag) {
              mark[u] = tag;
              deg += qsize[u];
              return true;
            }
            if (bwd[u] != 0) return true;
            if (fwd[u] == 2) {            // indistinguishable from v: merge into v
              qsize[v] += qsize[u];
              qsize[u] = 0;
              mark[u] = maxint;
              fwd[u] = -v;
              bwd[u] = -maxint;
            } else {                      // outmatched by v
              bwd[u] = -maxint;
            }
            return true;
          });
        }
        deg = deg - qsize[v] + 1;
        push_degree_list(v, deg);
        if (deg < *mdeg) *mdeg = deg;
      }
      for (int v = qx; v > 0; v = link[v]) {
        if (bwd[v] != 0) continue;
        tag++;
        int deg = deg0;
        for (int i = xadj[v]; i < xadj[v + 1]; i++) {
          const int u = adj[i];
          if (u == 0) break;
          if (mark[u] >= tag) continue;
          mark[u] = tag;
          if (fwd[u] >= 0) {
            deg += qsize[u];
            continue;
          }
          walk(u, [&](int w) {
            if (mark[w] < tag) {
              mark[w] = tag;
              deg += qsize[w];
            }
            return true;
          });
        }
        deg = deg - qsize[v] + 1;
        push_degree_list(v, deg);
        if (deg < *mdeg) *mdeg = deg;
      }
      tag = mtag;
    }
  }

  // Final numbering: every merged node follows the node it was merged into
  // (through chains of merges), in the order of its first appearance.
  void number(std::vector<int>& perm) {
    for (int v = 1; v <= n; v++) perm[v] = qsize[v] <= 0 ? fwd[v] : -fwd[v];
    for (int v = 1; v <= n; v++) {
      if (perm[v] > 0) continue;
      int root = v;
      while (perm[root] <= 0) root = -perm[root];
      const int num = perm[root] + 1;
      fwd[v] = -num;
      perm[root] = num;
      for (int f = v;;) {                  // path compression
        const int nf = -perm[f];
        if (nf <= 0) break;
        perm[f] = -root;
        f = nf;
      }
    }
    for (int v = 1; v <= n; v++) {
      const int num = -fwd[v];
      fwd[v] = num;
      perm[num] = v;
    }
  }

  void run(std::vector<int>& perm) {
    init();
    int num = 1;
    // isolated nodes first
    for (int v = head[1]; v > 0;) {
      const int nxt = fwd[v];
      mark[v] = maxint;
      fwd[v] = -num;
      num++;
      v = nxt;
    }
    if (num <= n) {
      tag = 1;
      head[1] = 0;
      int mdeg = 2;
      bool done = false;
      while (!done) {
        while (head[mdeg] <= 0) mdeg++;
        const int limit = mdeg + delta;
        int elems = 0;
        for (;;) {
          const int p = head[mdeg];
          if (p <= 0) {
            if (++mdeg > limit) break;
            continue;
          }
          const int nxt = fwd[p];
          head[mdeg] = nxt;
          if (nxt > 0) bwd[nxt] = -mdeg;
          fwd[p] = -num;
          if (num + qsize[p] > n) { done = true; break; }
          if (++tag >= maxint) reset_marks();
          eliminate(p);
          num += qsize[p];
          link[p] = elems;
          elems = p;
        }
        if (done || num > n) break;
        update(elems, &mdeg);
      }
    }
    number(perm);
  }
};

}  // namespace

int mmd_order(int n, const int* colptr, const int* rowind, int* perm, int* invperm) {
  if (n <= 0) return 0;
  MmdState S;
  S.n = n;
  // adjacency lists without the diagonal, each entry written to both ends in
  // the order of a column-by-column scan (src/taucs_ccs_order.c:344-385)
  std::vector<int> len(n + 2, 0);
  for (int j = 0; j < n; j++)
    for (int p = colptr[j]; p < colptr[j + 1]; p++) {
      const int i = rowind[p];
      if (i < 0 || i >= n) return -1;
      if (i != j) { len[i + 1]++; len[j + 1]++; }
    }
  S.xadj.assign(n + 2, 0);
  for (int v = 1; v <= n; v++) S.xadj[v + 1] = S.xadj[v] + len[v];
  S.adj.assign((size_t) S.xadj[n + 1] + 1, 0);
  std::vector<int> fill(S.xadj.begin(), S.xadj.end());
  for (int j = 0; j < n; j++)
    for (int p = colptr[j]; p < colptr[j + 1]; p++) {
      const int i = rowind[p];
      if (i != j) {
        S.adj[fill[i + 1]++] = j + 1;
        S.adj[fill[j + 1]++] = i + 1;
      }
    }
  S.head.assign(n + 2, 0);
  S.fwd.assign(n + 2, 0);
  S.bwd.assign(n + 2, 0);
  S.qsize.assign(n + 2, 0);
  S.link.assign(n + 2, 0);
  S.mark.assign(n + 2, 0);
  std::vector<int> p1(n + 2, 0);
  S.run(p1);
  for (int k = 0; k < n; k++) perm[k] = p1[k + 1] - 1;
  for (int k = 0; k < n; k++) invperm[perm[k]] = k;
  return 0;
}

}  // namespace tb
