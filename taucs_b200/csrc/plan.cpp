// Execution plan for the device numeric phase, built once per symbolic
// factor.  It turns the reference-layout supernodal structure into:
//
//  * fronts in DEVICE ORDER: grouped by height in the supernodal tree
//    (leaves = level 0), so that one launch covers every front of a level;
//    the reference instead recurses depth-first (src/taucs_sn_llt.c:1829-1977);
//  * a per-front LOCAL ROW ORDER that is ascending in the global index.  The
//    supernode's columns precede its update rows in that order (update rows
//    are proper etree ancestors of every column of the supernode), the column
//    order is a topological order of the etree restricted to the supernode, so
//    the dense factor of the front has the same entries as the reference's
//    factor (sn_struct order, src/taucs_sn_llt.c:1603-1649) -- and the
//    child->parent index maps become monotone, so extend-add never needs the
//    reference's transpose swap (src/taucs_sn_llt.c:1218-1222);
//  * offsets into one L arena (panel f x s, ld f, per front) and one update
//    arena whose offsets are assigned by a first-fit planner over the
//    lifetime [level(front), level(parent)] of each update matrix -- the
//    device replacement for the reference's calloc/free front stack
//    (src/taucs_sn_llt.c:1013-1078, :1797-1827);
//  * the assembly lists of A's entries per front column and the tile lists of
//    the front-build kernel.
#include <algorithm>
#include <cstdio>
#include <map>
#include <set>
#include <numeric>

#include "internal.h"
#include "kernels.h"

namespace tb {

namespace {

// best-fit allocator over [0, inf) offsets (in doubles), 256-byte granules:
// free blocks indexed by offset (for coalescing) and by (length, offset)
// (for the smallest block that fits, O(log n) per call)
struct ArenaPlanner {
  std::map<int64_t, int64_t> free_;              // offset -> length
  std::set<std::pair<int64_t, int64_t>> by_len_;  // (length, offset)
  int64_t top = 0;
  static int64_t round(int64_t n) { return (n + 31) & ~int64_t(31); }
  void add(int64_t off, int64_t len) {
    free_[off] = len;
    by_len_.emplace(len, off);
  }
  void drop(std::map<int64_t, int64_t>::iterator it) {
    by_len_.erase({it->second, it->first});
    free_.erase(it);
  }
  int64_t alloc(int64_t n) {
    n = round(n);
    auto b = by_len_.lower_bound({n, INT64_MIN});
    if (b != by_len_.end()) {
      const int64_t off = b->second, len = b->first;
      drop(free_.find(off));
      if (len > n) add(off + n, len - n);
      return off;
    }
    // extend the top (merge with a free block that ends at top)
    if (!free_.empty()) {
      auto last = std::prev(free_.end());
      if (last->first + last->second == top) {
        const int64_t off = last->first;
        drop(last);
        top = off + n;
        return off;
      }
    }
    const int64_t off = top;
    top += n;
    return off;
  }
  void release(int64_t off, int64_t n) {
    n = round(n);
    // coalesce with the neighbours, then insert once
    auto nx = free_.lower_bound(off);
    if (nx != free_.end() && off + n == nx->first) {
      n += nx->second;
      drop(nx);
    }
    auto pv = free_.lower_bound(off);
    if (pv != free_.begin()) {
      --pv;
      if (pv->first + pv->second == off) {
        off = pv->first;
        n += pv->second;
        drop(pv);
      }
    }
    add(off, n);
  }
};

}  // namespace

int build_plan(const Symbolic& S, int n, const int* colptr, const int* rowind, Plan* out) {
  Plan& P = *out;
  P = Plan();
  P.n = n;
  P.nnz = colptr[n];
  const int root = S.n_sn;

  // live supernodes reachable from the virtual root, tree parent, height
  std::vector<int> parent_sn(S.n_sn + 1, -1), height(S.n_sn + 1, 0), post;
  post.reserve(S.n_sn);
  {
    std::vector<int> stack, it(S.first_child.begin(), S.first_child.end());
    stack.push_back(root);
    while (!stack.empty()) {
      int v = stack.back();
      int c = it[v];
      if (c != -1) {
        it[v] = S.next_child[c];
        parent_sn[c] = v;
        stack.push_back(c);
        continue;
      }
      stack.pop_back();
      if (v != root) {
        post.push_back(v);
        int p = parent_sn[v];
        if (p != root) height[p] = std::max(height[p], height[v] + 1);
      }
    }
  }
  const int nf = (int) post.size();
  P.n_fronts = nf;
  int H = 0;
  for (int v : post) H = std::max(H, height[v] + 1);
  P.n_levels = H;

  // device order: by level, then by postorder position
  std::vector<int> order(post);
  {
    std::vector<int> pos(S.n_sn + 1, 0);
    for (int i = 0; i < nf; i++) pos[post[i]] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
      if (height[a] != height[b]) return height[a] < height[b];
      return pos[a] < pos[b];
    });
  }
  std::vector<int> dev_of(S.n_sn + 1, -1);
  for (int i = 0; i < nf; i++) dev_of[order[i]] = i;

  P.fronts.resize(nf);
  // rows (sorted) and sizes
  std::vector<int> col_front(n, -1), col_local(n, -1);
  int64_t rows_total = 0;
  for (int i = 0; i < nf; i++) rows_total += S.sn_up_size[order[i]];
  P.rows.resize(rows_total);
  int64_t roff = 0;
  for (int i = 0; i < nf; i++) {
    int sn = order[i];
    FrontDesc& F = P.fronts[i];
    F.sn = sn;
    F.s = S.sn_size[sn];
    F.f = S.sn_up_size[sn];
    F.level = height[sn];
    F.parent = parent_sn[sn] == root ? -1 : dev_of[parent_sn[sn]];
    F.rows_off = (int) roff;
    const std::vector<int>& st = S.sn_struct[sn];
    int* r = P.rows.data() + roff;
    std::copy(st.begin(), st.begin() + F.f, r);
    std::sort(r, r + F.f);
    // the supernode's columns must be the F.s smallest rows
    {
      std::vector<int> cols(st.begin(), st.begin() + F.s);
      std::sort(cols.begin(), cols.end());
      if (!std::equal(cols.begin(), cols.end(), r)) {
        set_error("plan: supernode columns are not the leading rows of its structure");
        return TAUCS_ERROR;
      }
    }
    for (int c = 0; c < F.s; c++) { col_front[r[c]] = i; col_local[r[c]] = c; }
    roff += F.f;
    P.max_front = std::max(P.max_front, F.f);
    P.max_s = std::max(P.max_s, F.s);
  }

  // children lists in the reference's child order (extend-add summation order)
  P.children.reserve(nf);
  for (int i = 0; i < nf; i++) {
    FrontDesc& F = P.fronts[i];
    F.child_begin = (int) P.children.size();
    for (int c = S.first_child[F.sn]; c != -1; c = S.next_child[c])
      if (dev_of[c] >= 0) P.children.push_back(dev_of[c]);
    F.child_end = (int) P.children.size();
  }

  // L arena: level-contiguous panels
  int64_t loff = 0;
  for (int i = 0; i < nf; i++) {
    FrontDesc& F = P.fronts[i];
    F.l_off = loff;
    loff += ArenaPlanner::round((int64_t) F.f * F.s);
  }
  P.l_len = std::max<int64_t>(loff, 32);

  // child -> parent maps (parent-local index of each update row)
  int64_t moff = 0;
  for (int i = 0; i < nf; i++) moff += P.fronts[i].f - P.fronts[i].s;
  P.maps.assign(std::max<int64_t>(moff, 1), 0);
  moff = 0;
  for (int i = 0; i < nf; i++) {
    FrontDesc& F = P.fronts[i];
    F.map_off = (int) moff;
    const int m = F.f - F.s;
    if (m > 0) {
      if (F.parent < 0) {
        set_error("plan: a root supernode has update rows");
        return TAUCS_ERROR;
      }
      const FrontDesc& Pf = P.fronts[F.parent];
      const int* pr = P.rows.data() + Pf.rows_off;
      const int* cr = P.rows.data() + F.rows_off + F.s;
      for (int k = 0; k < m; k++) {
        const int* it = std::lower_bound(pr, pr + Pf.f, cr[k]);
        if (it == pr + Pf.f || *it != cr[k]) {
          set_error("plan: update row missing from the parent's structure");
          return TAUCS_ERROR;
        }
        P.maps[moff + k] = (int) (it - pr);
      }
    }
    moff += m;
  }

  // small fronts with only small fronts below them (children come before
  // parents in device order): one persistent launch factors all of them
  // before the level launches (numeric.cu)
  std::vector<char> pure(nf, 0);
  for (int i = 0; i < nf; i++) {
    const FrontDesc& F = P.fronts[i];
    bool ok = F.f <= SMALL_F_MAX;
    for (int ci = F.child_begin; ok && ci < F.child_end; ci++) ok = pure[P.children[ci]];
    pure[i] = ok;
  }

  // update arena.  The persistent launch runs the small fronts of all levels
  // in no fixed order among unrelated subtrees, so their update matrices get
  // slots of their own, live from the start: released at its end when the
  // consumer is in the persistent set too, else at the consumer's level.
  // The other fronts' update matrices live over [level(front), level(parent)].
  {
    ArenaPlanner ap;
    std::vector<std::vector<int>> free_at(H + 1);
    std::vector<int> free_now;
    for (int i = 0; i < nf; i++) {
      FrontDesc& F = P.fronts[i];
      const int64_t m = F.f - F.s;
      if (!pure[i]) continue;
      F.u_off = -1;
      if (m <= 0) continue;
      F.u_off = ap.alloc(m * m);
      if (pure[F.parent]) free_now.push_back(i);
      else free_at[P.fronts[F.parent].level].push_back(i);
    }
    for (int i : free_now) {
      const int64_t m = P.fronts[i].f - P.fronts[i].s;
      ap.release(P.fronts[i].u_off, m * m);
    }
    int fi = 0;
    for (int h = 0; h < H; h++) {
      int fe = fi;
      while (fe < nf && P.fronts[fe].level == h) fe++;
      for (int i = fi; i < fe; i++) {
        FrontDesc& F = P.fronts[i];
        if (pure[i]) continue;
        const int64_t m = F.f - F.s;
        if (m > 0) {
          F.u_off = ap.alloc(m * m);
          free_at[P.fronts[F.parent].level].push_back(i);
        } else {
          F.u_off = -1;
        }
      }
      for (int i : free_at[h]) {
        const int64_t m = P.fronts[i].f - P.fronts[i].s;
        ap.release(P.fronts[i].u_off, m * m);
      }
      fi = fe;
    }
    P.u_len = std::max<int64_t>(ap.top, 32);
  }

  // solve vectors: per front f entries per right-hand side
  P.v_len = rows_total;
  for (int i = 0; i < nf; i++) P.fronts[i].v_off = P.fronts[i].rows_off;

  // assembly: A's entries per front column, sorted by local row
  {
    std::vector<int> cnt(nf > 0 ? (size_t) rows_total + nf : 1, 0);
    // acol_ptr layout: per front s+1 entries
    int64_t aoff = 0;
    for (int i = 0; i < nf; i++) { P.fronts[i].acol_off = (int) aoff; aoff += P.fronts[i].s + 1; }
    P.acol_ptr.assign(aoff > 0 ? aoff : 1, 0);
    std::vector<int> colcount(n, 0);
    for (int j = 0; j < n; j++) colcount[j] = colptr[j + 1] - colptr[j];
    for (int i = 0; i < nf; i++) {
      FrontDesc& F = P.fronts[i];
      int* ap = P.acol_ptr.data() + F.acol_off;
      const int* r = P.rows.data() + F.rows_off;
      ap[0] = 0;
      for (int c = 0; c < F.s; c++) ap[c + 1] = ap[c] + colcount[r[c]];
    }
    // global prefix per front
    int64_t eoff = 0;
    std::vector<int64_t> fbase(nf);
    for (int i = 0; i < nf; i++) {
      fbase[i] = eoff;
      eoff += P.acol_ptr[P.fronts[i].acol_off + P.fronts[i].s];
    }
    if (eoff != P.nnz) {
      set_error("plan: some columns of A are not covered by the supernodal structure");
      return TAUCS_ERROR;
    }
    P.a_rows.assign(std::max<int64_t>(eoff, 1), 0);
    P.a_idx.assign(std::max<int64_t>(eoff, 1), 0);
    for (int i = 0; i < nf; i++) {
      FrontDesc& F = P.fronts[i];
      int* ap = P.acol_ptr.data() + F.acol_off;
      for (int c = 0; c <= F.s; c++) ap[c] += (int) fbase[i];
    }
    std::vector<std::pair<int, int>> tmp;
    for (int j = 0; j < n; j++) {
      const int fi = col_front[j];
      if (fi < 0) { set_error("plan: column without a supernode"); return TAUCS_ERROR; }
      const FrontDesc& F = P.fronts[fi];
      const int* r = P.rows.data() + F.rows_off;
      tmp.clear();
      for (int ip = colptr[j]; ip < colptr[j + 1]; ip++) {
        const int* it = std::lower_bound(r, r + F.f, rowind[ip]);
        if (it == r + F.f || *it != rowind[ip]) {
          set_error("plan: entry of A outside the structure of L");
          return TAUCS_ERROR;
        }
        tmp.emplace_back((int) (it - r), ip);
      }
      std::stable_sort(tmp.begin(), tmp.end(),
                       [](const std::pair<int, int>& a, const std::pair<int, int>& b) { return a.first < b.first; });
      int dst = P.acol_ptr[F.acol_off + col_local[j]];
      for (auto& e : tmp) { P.a_rows[dst] = e.first; P.a_idx[dst] = e.second; dst++; }
    }
  }

  // inverses of the diagonal blocks and solve flags for the big fronts
  {
    int64_t doff = 0;
    int boff = 0;
    for (int i = 0; i < nf; i++) {
      FrontDesc& F = P.fronts[i];
      if (F.f > SMALL_F_MAX) {
        const int nbs = (F.s + PANEL_NB - 1) / PANEL_NB;
        F.dinv_off = doff;
        doff += (int64_t) nbs * PANEL_NB * PANEL_NB;
        F.blk_off = boff;
        boff += nbs;
      } else {
        F.dinv_off = -1;
        F.blk_off = -1;
      }
    }
    P.dinv_len = std::max<int64_t>(doff, 32);
    P.n_blk = std::max(boff, 1);
    int64_t poff = 0;
    for (int i = 0; i < nf; i++) {
      FrontDesc& F = P.fronts[i];
      const int m = F.f - F.s;
      if (F.f > SMALL_F_MAX && m > 0) {
        F.nchunk = (m + SOLVE_RCH - 1) / SOLVE_RCH;
        F.part_off = poff;
        poff += (int64_t) F.nchunk * F.s * SOLVE_NRHS;
      } else {
        F.nchunk = 0;
        F.part_off = -1;
      }
    }
    // the walks' tagged values follow, 8-byte aligned: per 64-row block
    // the chain's 64 x 8 results, then the helpers' 64 x 8 partial sums, as
    // (tag, value) pairs of 8 bytes (two FP32 elements each)
    poff = (poff + 1) & ~int64_t(1);
    P.fpart_off = poff;
    poff += (int64_t) P.n_blk * 2 * PANEL_NB * SOLVE_NRHS * 2;
    P.part_len = std::max<int64_t>(poff, 32);
    // split copies of the big fronts' panels for the FP32 tensor-core
    // products; the levels run one after another, so each level starts the
    // arena afresh.  One tile of slack at the end: the bulk copies of a
    // 128-row tile may read past the last row group of the last front.
    int64_t soff = 0, smax = 0;
    for (int i = 0; i < nf; i++) {
      FrontDesc& F = P.fronts[i];
      if (i > 0 && P.fronts[i - 1].level != F.level) soff = 0;
      if (F.f > SMALL_F_MAX) {
        F.sp_off = soff;
        soff += 2 * sp_part_bytes(F, 0) / 4;   // format 0 is the larger one
        smax = std::max(smax, soff);
      } else {
        F.sp_off = -1;
      }
    }
    P.sp_len = smax + 16 * 32 * 4;
  }

  // levels, front classes, build tiles
  P.levels.resize(H);
  {
    int fi = 0;
    for (int h = 0; h < H; h++) {
      LevelPlan& LP = P.levels[h];
      LP.front_begin = fi;
      while (fi < nf && P.fronts[fi].level == h) fi++;
      LP.front_end = fi;
      std::vector<int2_> fwd_upd;   // forward blocks of update rows, after the diagonal ones
      for (int i = LP.front_begin; i < LP.front_end; i++) {
        const FrontDesc& F = P.fronts[i];
        if (F.f <= SMALL_F_MAX) {
          LP.small_fronts.push_back(i);
        } else {
          LP.big_fronts.push_back(i);
          LP.max_s_big = std::max(LP.max_s_big, F.s);
          LP.max_m_big = std::max(LP.max_m_big, F.f - F.s);
          // panel region: rows [0,f), columns [0,s); U region: m x m
          for (int c0 = 0; c0 < F.s; c0 += BUILD_TC)
            for (int r0 = (c0 / BUILD_TR) * BUILD_TR; r0 < F.f; r0 += BUILD_TR)
              LP.build_tiles.push_back(Tile{i, r0, c0, 0});
          const int m = F.f - F.s;
          for (int c0 = 0; c0 < m; c0 += BUILD_TC)
            for (int r0 = (c0 / BUILD_TR) * BUILD_TR; r0 < m; r0 += BUILD_TR)
              LP.build_tiles.push_back(Tile{i, r0, -1 - c0, 0});
          const int nrb = (F.f + PANEL_NB - 1) / PANEL_NB, nbs = (F.s + PANEL_NB - 1) / PANEL_NB;
          for (int r = 0; r < nbs; r++) LP.solve_fwd_blocks.push_back(int2_{i, r});
          for (int r = nbs; r < nrb; r++) fwd_upd.push_back(int2_{i, r});
          for (int k = nbs - 1; k >= 0; k--) LP.solve_bwd_blocks.push_back(int2_{i, k});
          const int nch = (m + SOLVE_RCH - 1) / SOLVE_RCH;
          for (int k = 0; k < nbs; k++)
            for (int c = 0; c < nch; c++) LP.solve_l21_tasks.push_back(int2_{i, (k << 16) | c});
        }
      }
      LP.n_fwd_diag = (int) LP.solve_fwd_blocks.size();
      LP.solve_fwd_blocks.insert(LP.solve_fwd_blocks.end(), fwd_upd.begin(), fwd_upd.end());
      // the fused small-front kernel is launched per size class
      std::stable_sort(LP.small_fronts.begin(), LP.small_fronts.end(),
                       [&](int a, int b) { return P.fronts[a].f < P.fronts[b].f; });
      while (LP.small_warp < (int) LP.small_fronts.size() &&
             P.fronts[LP.small_fronts[LP.small_warp]].f <= SOLVE_WARP_F)
        LP.small_warp++;
    }
  }

  // the persistent set: the fronts whose subtree has only fronts of order
  // <= SMALL_WARP_F, then the others, each part in device (level) order
  {
    std::vector<int> task(nf, -1), smax(nf, 0);
    for (int i = 0; i < nf; i++) {
      const FrontDesc& F = P.fronts[i];
      smax[i] = F.f;
      for (int ci = F.child_begin; ci < F.child_end; ci++) smax[i] = std::max(smax[i], smax[P.children[ci]]);
    }
    for (int part = 0; part < 2; part++) {
      for (int i = 0; i < nf; i++) {
        const FrontDesc& F = P.fronts[i];
        if (!pure[i] || (smax[i] <= SMALL_WARP_F) != (part == 0)) continue;
        task[i] = (int) P.pers_fronts.size();
        P.pers_fronts.push_back(i);
        P.pers_pending.push_back(F.child_end - F.child_begin);
        if (part == 1) P.pers_fmax = std::max(P.pers_fmax, F.f);
      }
      if (part == 0) P.pers_nwarp = (int) P.pers_fronts.size();
    }
    P.pers_parent.assign(P.pers_fronts.size(), -1);
    for (size_t t = 0; t < P.pers_fronts.size(); t++) {
      const int par = P.fronts[P.pers_fronts[t]].parent;
      if (par >= 0) P.pers_parent[t] = task[par];
    }
    for (LevelPlan& LP : P.levels) {
      for (int i : LP.small_fronts)
        if (task[i] < 0) LP.small_numeric.push_back(i);
      while (LP.small_numeric_warp < (int) LP.small_numeric.size() &&
             P.fronts[LP.small_numeric[LP.small_numeric_warp]].f <= SOLVE_WARP_F)
        LP.small_numeric_warp++;
    }
  }

  // statistics: the reference's relaxed flop count (src/taucs_sn_llt.c:3957-3965)
  double flops = 0.0, ea = 0.0, sb = 0.0;
  for (int i = 0; i < nf; i++) {
    const FrontDesc& F = P.fronts[i];
    for (int k = 0, c = F.f; k < F.s; k++, c--) flops += 1.0 + (double) c * (double) c;
    const double m = F.f - F.s;
    ea += 8.0 * m * (m + 1) / 2 + 16.0 * m * (m + 1) / 2 + 4.0 * m;
    sb += 2.0 * 8.0 * ((double) F.s * (F.s + 1) / 2 + m * F.s) + 2.0 * 4.0 * F.f + 2.0 * 2.0 * 8.0 * F.f;
  }
  ea += 12.0 * (double) P.nnz;
  sb += 16.0 * (double) n;
  P.flops = flops;
  P.ea_bytes = ea;
  P.solve_bytes = sb;
  return TAUCS_SUCCESS;
}

}  // namespace tb
