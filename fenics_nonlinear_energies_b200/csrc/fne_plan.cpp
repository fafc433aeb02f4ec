// Host-side construction of the row-gather plan.
//
// The reference scatters the element Hessian stack with
//   contrib = elem_hess[hess_e, hess_i, hess_j]; np.add.at(owned_vals, hess_positions, contrib)
// (src/core/petsc/reordered_element_base.py:1754-1756), where hess_positions
// come from a searchsorted of (row, col) keys into the owned COO pattern
// (:1464-1534).  Here the same map is regrouped by OUTPUT ROW: every owned
// row lists the (element, local node) incidences of its node and, per
// incidence, where each element column lands inside the row.  A kernel thread
// then produces one row by summing those contributions in a fixed order, so
// no atomics are needed and the result is bit-reproducible.  As in the
// reference, a missing (row, col) key is an error (FNE_ELAYOUT).
#include <algorithm>
#include <unordered_map>

#include "fne_internal.h"

namespace fne {

int build_row_plan(const fne_desc* d, RowPlan& P) {
  const int npe = d->npe, bs = d->block_size, nde = npe * bs;
  const int64_t E = d->n_elem, lo = d->lo, hi = d->hi, nf = d->n_free;
  if (npe < 1 || bs < 1 || bs > 3 || kOffShift + kOffBits * npe > 32)
    return set_error(FNE_EINVAL, "row plan: unsupported npe/block_size");
  if (lo < 0 || hi < lo || hi > nf) return set_error(FNE_EINVAL, "row plan: bad owned range");
  if (hi - lo >= (int64_t)INT32_MAX || d->nnz >= (int64_t)INT32_MAX || E >= (int64_t)INT32_MAX)
    return set_error(FNE_EBOUNDS, "row plan: sizes beyond 32-bit indexing");
  const int64_t* t2f = d->total_to_free_reord;

  // ---- element node codes -------------------------------------------------
  std::vector<int32_t> code(E * npe);
  std::vector<char> local(E, 0);
  for (int64_t e = 0; e < E; ++e) {
    for (int a = 0; a < npe; ++a) {
      const int64_t* ed = d->elems + e * nde + a * bs;
      const int64_t base = ed[0];
      if (base < 0 || base >= d->n_total || base % bs != 0)
        return set_error(FNE_EBOUNDS, "row plan: element DOF out of range / not node-blocked");
      int nfree = 0;
      for (int c = 0; c < bs; ++c) {
        if (ed[c] != base + c)
          return set_error(FNE_EINVAL, "row plan: element DOFs are not node-blocked");
        if (t2f[base + c] >= 0) ++nfree;
      }
      if (nfree == bs) {
        const int64_t r0 = t2f[base];
        for (int c = 1; c < bs; ++c)
          if (t2f[base + c] != r0 + c)
            return set_error(FNE_EINVAL, "row plan: node components not consecutive after reordering");
        if (r0 >= (int64_t)INT32_MAX) return set_error(FNE_EBOUNDS, "row plan: id beyond int32");
        code[e * npe + a] = (int32_t)r0;
        if (r0 >= lo && r0 < hi) local[e] = 1;
      } else if (nfree == 0) {
        if (base + 1 >= (int64_t)INT32_MAX) return set_error(FNE_EBOUNDS, "row plan: id beyond int32");
        code[e * npe + a] = (int32_t)(-1 - base);
      } else {
        return set_error(FNE_EINVAL,
                         "row plan: node with partially fixed components (use the Mohr-Coulomb path)");
      }
    }
  }

  // ---- local elements (overlap: any owned DOF), weights ---------------------
  std::vector<int32_t> lidx(E, -1);
  P.local_elems.clear();
  P.elem_code.clear();
  P.elem_weight.clear();
  P.dir_only.clear();
  P.dir_only_code.clear();
  for (int64_t e = 0; e < E; ++e) {
    bool any_free = false;
    for (int a = 0; a < npe; ++a) any_free |= code[e * npe + a] >= 0;
    if (!any_free) {
      P.dir_only.push_back(e);
      for (int a = 0; a < npe; ++a) P.dir_only_code.push_back(code[e * npe + a]);
    }
    if (!local[e]) continue;
    double w = d->energy_weights ? d->energy_weights[e] : 1.0;
    if (w != 0.0 && w != 1.0) return set_error(FNE_EINVAL, "row plan: energy weights must be 0 or 1");
    lidx[e] = (int32_t)P.local_elems.size();
    P.local_elems.push_back(e);
    for (int a = 0; a < npe; ++a) P.elem_code.push_back(code[e * npe + a]);
    P.elem_weight.push_back(w != 0.0 ? 1 : 0);
  }

  // ---- output rows (row-grouped owned COO pattern) --------------------------
  const int64_t n_owned = hi - lo;
  std::vector<int64_t> rev(n_owned, -1);  // reordered - lo -> total DOF
  for (int64_t t = 0; t < d->n_total; ++t)
    if (t2f[t] >= lo && t2f[t] < hi) rev[t2f[t] - lo] = t;
  for (int64_t i = 0; i < n_owned; ++i)
    if (rev[i] < 0) return set_error(FNE_EINVAL, "row plan: owned DOF without total DOF");

  std::vector<int64_t> row_id;
  std::vector<int64_t> rptr;
  std::vector<char> seen(n_owned, 0);
  for (int64_t j = 0; j < d->nnz; ++j) {
    const int64_t r = d->owned_rows[j];
    if (r < lo || r >= hi) return set_error(FNE_EBOUNDS, "row plan: owned row outside [lo, hi)");
    if (d->owned_cols[j] < 0 || d->owned_cols[j] >= nf)
      return set_error(FNE_EBOUNDS, "row plan: column out of range");
    if (j == 0 || d->owned_rows[j - 1] != r) {
      if (seen[r - lo]) return set_error(FNE_ELAYOUT, "row plan: COO pattern is not row-grouped");
      seen[r - lo] = 1;
      row_id.push_back(r);
      rptr.push_back(j);
    }
  }
  // owned DOFs absent from the pattern: gradient-only rows of length 0
  for (int64_t i = 0; i < n_owned; ++i)
    if (!seen[i]) {
      row_id.push_back(lo + i);
      rptr.push_back(d->nnz);
    }
  rptr.push_back(d->nnz);
  const int32_t n_rows = (int32_t)row_id.size();
  P.n_rows = n_rows;
  P.row_ptr.assign(rptr.begin(), rptr.end());
  P.row_node.resize(n_rows);
  P.row_comp.resize(n_rows);
  P.row_gpos.resize(n_rows);

  // row-nodes in order of first appearance; the first row of each node is the
  // one whose column layout defines the offsets (all rows must agree)
  std::unordered_map<int64_t, int32_t> node_idx;
  std::vector<int32_t> node_first_row;
  std::vector<int64_t> node_of;
  int32_t max_len = 0;
  for (int32_t k = 0; k < n_rows; ++k) {
    const int64_t t = rev[row_id[k] - lo];
    const int64_t node = t / bs;
    auto it = node_idx.find(node);
    int32_t ni;
    if (it == node_idx.end()) {
      ni = (int32_t)node_of.size();
      node_idx.emplace(node, ni);
      node_of.push_back(node);
      node_first_row.push_back(k);
    } else {
      ni = it->second;
    }
    P.row_node[k] = ni;
    P.row_comp[k] = (uint8_t)(t % bs);
    P.row_gpos[k] = (int32_t)(row_id[k] - lo);
    max_len = std::max<int32_t>(max_len, P.row_ptr[k + 1] - P.row_ptr[k]);
  }
  P.max_row_len = max_len;
  if (max_len >= (int32_t)kNoCol)
    return set_error(FNE_EBOUNDS, "row plan: a row has more than 126 entries");
  const int32_t n_nodes = (int32_t)node_of.size();
  P.n_nodes = n_nodes;

  // rows of each node (to validate identical column layouts)
  std::vector<std::vector<int32_t>> node_rows(n_nodes);
  for (int32_t k = 0; k < n_rows; ++k) node_rows[P.row_node[k]].push_back(k);

  // ---- incidences ----------------------------------------------------------
  std::vector<int32_t> cnt(n_nodes + 1, 0);
  struct Inc {
    int32_t node, le;
    uint32_t info;
  };
  std::vector<Inc> incs;
  incs.reserve(P.local_elems.size() * npe);
  std::vector<std::pair<int64_t, int32_t>> rowcols;  // (col, offset) of one row
  for (size_t le = 0; le < P.local_elems.size(); ++le) {
    const int64_t e = P.local_elems[le];
    bool flagged = false;
    for (int a = 0; a < npe; ++a) {
      const int32_t ca = code[e * npe + a];
      if (ca < lo || ca >= hi) continue;  // not an owned row-node
      const int64_t node = rev[ca - lo] / bs;
      auto it = node_idx.find(node);
      if (it == node_idx.end()) return set_error(FNE_ELAYOUT, "row plan: owned node has no row");
      const int32_t ni = it->second;
      uint32_t info = (uint32_t)a;
      if (!flagged && P.elem_weight[le]) {
        info |= kEnergyFlag;
        flagged = true;
      }
      // column offsets, validated on every row of the node
      for (int b = 0; b < npe; ++b) {
        const int32_t cb = code[e * npe + b];
        uint32_t off = kNoCol;
        if (cb >= 0) {
          bool first = true;
          for (int32_t k : node_rows[ni]) {
            const int64_t s = P.row_ptr[k], len = P.row_ptr[k + 1] - s;
            int64_t pos = -1;
            for (int64_t q = 0; q < len; ++q)
              if (d->owned_cols[s + q] == cb) {
                pos = q;
                break;
              }
            if (pos < 0)
              return set_error(FNE_ELAYOUT, "Scatter lookup found mismatched owned COO entries");
            for (int c = 1; c < bs; ++c)
              if (pos + c >= len || d->owned_cols[s + pos + c] != cb + c)
                return set_error(FNE_ELAYOUT, "row plan: node block columns not consecutive");
            if (first) {
              off = (uint32_t)pos;
              first = false;
            } else if ((uint32_t)pos != off) {
              return set_error(FNE_ELAYOUT, "row plan: rows of one node differ in column layout");
            }
          }
        }
        info |= (off & 127u) << (kOffShift + kOffBits * b);
      }
      incs.push_back({ni, (int32_t)le, info});
      cnt[ni + 1]++;
    }
  }
  for (int32_t i = 0; i < n_nodes; ++i) cnt[i + 1] += cnt[i];
  P.inc_ptr = cnt;
  P.inc_elem.resize(incs.size());
  P.inc_info.resize(incs.size());
  std::vector<int32_t> fill(cnt.begin(), cnt.end() - 1);
  for (const Inc& x : incs) {  // stable: element order within a node
    const int32_t p = fill[x.node]++;
    P.inc_elem[p] = x.le;
    P.inc_info[p] = x.info;
  }
  return FNE_OK;
}

}  // namespace fne

namespace fne {

bool build_inc_plan(RowPlan& P, int threads, IncPlan& Q) {
  const int32_t n_local = (int32_t)P.local_elems.size();
  const int npe = n_local ? (int)(P.elem_code.size() / n_local) : 3;
  if (npe != 3) return false;
  const int32_t n_rows = P.n_rows;
  // locality: sort elements by the first row (output order) that needs them
  std::vector<int32_t> first(n_local, INT32_MAX);
  for (int32_t k = 0; k < n_rows; ++k) {
    const int32_t nd = P.row_node[k];
    for (int32_t i = P.inc_ptr[nd]; i < P.inc_ptr[nd + 1]; ++i)
      first[P.inc_elem[i]] = std::min(first[P.inc_elem[i]], k);
  }
  std::vector<int32_t> order(n_local);
  for (int32_t i = 0; i < n_local; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return first[a] < first[b]; });
  std::vector<int32_t> newidx(n_local);
  for (int32_t i = 0; i < n_local; ++i) newidx[order[i]] = i;
  {
    std::vector<int64_t> le(n_local);
    std::vector<int32_t> code(P.elem_code.size());
    std::vector<uint8_t> w(n_local);
    for (int32_t i = 0; i < n_local; ++i) {
      le[i] = P.local_elems[order[i]];
      w[i] = P.elem_weight[order[i]];
      for (int a = 0; a < npe; ++a) code[(size_t)i * npe + a] = P.elem_code[(size_t)order[i] * npe + a];
    }
    P.local_elems.swap(le);
    P.elem_code.swap(code);
    P.elem_weight.swap(w);
    for (auto& e : P.inc_elem) e = newidx[e];
  }
  // CTAs: greedy runs of whole rows with at most `threads` incidences
  Q.cta_row.assign(1, 0);
  Q.cta_inc.assign(1, 0);
  Q.inc_elem.clear();
  Q.inc_word.clear();
  Q.inc_rowl.clear();
  Q.max_rank = 0;
  Q.max_rows = 0;
  Q.max_len = 0;
  int32_t cnt = 0, rows_in = 0, row0 = 0;
  for (int32_t k = 0; k < n_rows; ++k) {
    const int32_t nd = P.row_node[k];
    const int32_t m = P.inc_ptr[nd + 1] - P.inc_ptr[nd];
    if (m > threads || m > 16) return false;
    if (cnt + m > threads || rows_in == 65535) {
      Q.cta_row.push_back(k);
      Q.cta_inc.push_back((int32_t)Q.inc_elem.size());
      Q.max_rows = std::max(Q.max_rows, rows_in);
      Q.max_len = std::max(Q.max_len, P.row_ptr[k] - P.row_ptr[row0]);
      cnt = 0;
      rows_in = 0;
      row0 = k;
    }
    for (int32_t j = 0; j < m; ++j) {
      const int32_t i = P.inc_ptr[nd] + j;
      const uint32_t info = P.inc_info[i];
      uint32_t w = (info & 3u) | ((info & kEnergyFlag) ? 4u : 0u) | ((uint32_t)j << 3);
      w |= ((info >> kOffShift) & ((1u << (3 * kOffBits)) - 1u)) << 7;
      Q.inc_elem.push_back(P.inc_elem[i]);
      Q.inc_word.push_back(w);
      Q.inc_rowl.push_back((uint16_t)rows_in);
    }
    Q.max_rank = std::max(Q.max_rank, m - 1);
    cnt += m;
    ++rows_in;
  }
  Q.cta_row.push_back(n_rows);
  Q.cta_inc.push_back((int32_t)Q.inc_elem.size());
  Q.max_rows = std::max(Q.max_rows, rows_in);
  Q.max_len = std::max(Q.max_len, P.row_ptr[n_rows] - P.row_ptr[row0]);
  Q.n_cta = (int32_t)Q.cta_row.size() - 1;
  return true;
}

}  // namespace fne

namespace fne {

static int32_t next_pow2(int64_t x) {
  int64_t p = 1;
  while (p < x) p <<= 1;
  return (int32_t)p;
}

bool build_sweep_plan(RowPlan& P, int nb, int n_seg, int max_win_entries, int max_win_rows, SweepPlan& Q) {
  const int32_t n_local = (int32_t)P.local_elems.size();
  const int npe = n_local ? (int)(P.elem_code.size() / n_local) : 3;
  if (npe != 3 || nb > 512 || n_local == 0) return false;
  const int32_t n_rows = P.n_rows;
  // first / last row of every element
  std::vector<int32_t> first(n_local, INT32_MAX), last(n_local, -1);
  for (int32_t k = 0; k < n_rows; ++k) {
    const int32_t nd = P.row_node[k];
    for (int32_t i = P.inc_ptr[nd]; i < P.inc_ptr[nd + 1]; ++i) {
      first[P.inc_elem[i]] = std::min(first[P.inc_elem[i]], k);
      last[P.inc_elem[i]] = std::max(last[P.inc_elem[i]], k);
    }
  }
  std::vector<int32_t> order(n_local);
  for (int32_t i = 0; i < n_local; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return first[a] < first[b]; });
  std::vector<int32_t> newidx(n_local);
  for (int32_t i = 0; i < n_local; ++i) newidx[order[i]] = i;
  {
    std::vector<int64_t> le(n_local);
    std::vector<int32_t> code(P.elem_code.size());
    std::vector<uint8_t> w(n_local);
    std::vector<int32_t> f2(n_local), l2(n_local);
    for (int32_t i = 0; i < n_local; ++i) {
      le[i] = P.local_elems[order[i]];
      w[i] = P.elem_weight[order[i]];
      f2[i] = first[order[i]];
      l2[i] = last[order[i]];
      for (int a = 0; a < npe; ++a) code[(size_t)i * npe + a] = P.elem_code[(size_t)order[i] * npe + a];
    }
    P.local_elems.swap(le);
    P.elem_code.swap(code);
    P.elem_weight.swap(w);
    first.swap(f2);
    last.swap(l2);
    for (auto& e : P.inc_elem) e = newidx[e];
  }
  // incidences of every row sorted by (new) element index
  std::vector<int32_t> rinc_ptr(n_rows + 1, 0);
  for (int32_t k = 0; k < n_rows; ++k) rinc_ptr[k + 1] = rinc_ptr[k] + (P.inc_ptr[P.row_node[k] + 1] - P.inc_ptr[P.row_node[k]]);
  std::vector<std::pair<int32_t, uint32_t>> rinc(rinc_ptr[n_rows]);  // (element, info)
  for (int32_t k = 0; k < n_rows; ++k) {
    const int32_t nd = P.row_node[k];
    int32_t q = rinc_ptr[k];
    for (int32_t i = P.inc_ptr[nd]; i < P.inc_ptr[nd + 1]; ++i) rinc[q++] = {P.inc_elem[i], P.inc_info[i]};
    std::sort(rinc.begin() + rinc_ptr[k], rinc.begin() + rinc_ptr[k + 1]);
  }
  // segments: balance the elements each CTA evaluates (own + pre)
  n_seg = std::max(1, std::min(n_seg, n_rows));
  Q.nb = nb;
  Q.seg_row.assign(1, 0);
  {
    // cumulative own-element count by first row
    std::vector<int64_t> cum(n_rows + 1, 0);
    for (int32_t i = 0; i < n_local; ++i)
      if (first[i] < n_rows) cum[first[i] + 1]++;
    for (int32_t k = 0; k < n_rows; ++k) cum[k + 1] += cum[k];
    for (int s = 1; s < n_seg; ++s) {
      const int64_t target = (int64_t)n_local * s / n_seg;
      int32_t r = (int32_t)(std::lower_bound(cum.begin(), cum.end(), target) - cum.begin());
      r = std::max(r, Q.seg_row.back() + 1);
      if (r >= n_rows) break;
      Q.seg_row.push_back(r);
    }
    Q.seg_row.push_back(n_rows);
  }
  Q.n_seg = (int32_t)Q.seg_row.size() - 1;
  Q.seg_elem.assign(3 * (size_t)Q.n_seg, 0);
  Q.seg_batch.assign(1, 0);
  Q.batch_done.clear();
  Q.ent_ptr.assign(1, 0);
  Q.inc_base.clear();
  Q.ent_row.clear();
  Q.ent_pos.clear();
  Q.ent_meta.clear();
  Q.inc_word.clear();
  int64_t need_entries = 1, need_rows = 1;
  std::vector<std::vector<std::pair<int32_t, int32_t>>> per_batch;  // (row, rinc index) lists
  for (int32_t s = 0; s < Q.n_seg; ++s) {
    const int32_t R0 = Q.seg_row[s], R1 = Q.seg_row[s + 1];
    const int32_t o_lo = (int32_t)(std::lower_bound(first.begin(), first.end(), R0) - first.begin());
    const int32_t o_hi = (int32_t)(std::lower_bound(first.begin(), first.end(), R1) - first.begin());
    // pre elements: smallest element index touching a row of the segment
    int32_t p_lo = o_lo;
    for (int32_t k = R0; k < R1; ++k)
      if (rinc_ptr[k + 1] > rinc_ptr[k]) p_lo = std::min(p_lo, rinc[rinc_ptr[k]].first);
    Q.seg_elem[3 * s] = p_lo;
    Q.seg_elem[3 * s + 1] = o_lo;
    Q.seg_elem[3 * s + 2] = o_hi;
    const int32_t nbat = (o_hi - p_lo + nb - 1) / nb;
    per_batch.assign(nbat, {});
    for (int32_t k = R0; k < R1; ++k)
      for (int32_t q = rinc_ptr[k]; q < rinc_ptr[k + 1]; ++q) {
        const int32_t e = rinc[q].first;
        if (e < p_lo || e >= o_hi) return false;  // cannot happen for a consistent plan
        per_batch[(e - p_lo) / nb].push_back({k, q});
      }
    int32_t done = R0, maxrow = R0 - 1;
    for (int32_t b = 0; b < nbat; ++b) {
      const int32_t e0 = p_lo + b * nb;
      auto& lst = per_batch[b];  // already grouped by row (rows ascending, incidences ascending)
      Q.inc_base.push_back((int32_t)Q.inc_word.size());
      const int32_t base = (int32_t)Q.inc_word.size();
      for (size_t x = 0; x < lst.size();) {
        const int32_t row = lst[x].first;
        size_t y = x;
        const int32_t start = (int32_t)Q.inc_word.size() - base;
        while (y < lst.size() && lst[y].first == row) {
          const int32_t e = rinc[lst[y].second].first;
          const uint32_t info = rinc[lst[y].second].second;
          uint32_t w = (uint32_t)(e - e0) | ((info & 3u) << 9);
          w |= ((info >> kOffShift) & ((1u << (3 * kOffBits)) - 1u)) << 11;
          Q.inc_word.push_back(w);
          ++y;
        }
        const int32_t cnt = (int32_t)(y - x);
        if (start >= 65536 || cnt > 255) return false;
        Q.ent_row.push_back(row);
        Q.ent_pos.push_back(P.row_ptr[row]);
        Q.ent_meta.push_back((uint32_t)start | ((uint32_t)cnt << 16));
        maxrow = std::max(maxrow, row);
        x = y;
      }
      Q.ent_ptr.push_back((int32_t)Q.ent_row.size());
      // live window after this batch: positions [row_ptr[done], row_ptr[maxrow + 1])
      if (maxrow >= done) {
        need_entries = std::max<int64_t>(need_entries, (int64_t)P.row_ptr[maxrow + 1] - P.row_ptr[done]);
        need_rows = std::max<int64_t>(need_rows, (int64_t)maxrow + 1 - done);
      }
      const int32_t nxt = (b + 1 < nbat) ? first[e0 + nb] : R1;
      done = std::max(done, std::min(std::max(nxt, R0), R1));
      Q.batch_done.push_back(done);
    }
    Q.seg_batch.push_back((int32_t)Q.batch_done.size());
  }
  Q.gpos_identity = true;
  for (int32_t k = 0; k < n_rows; ++k)
    if (P.row_gpos[k] != k) {
      Q.gpos_identity = false;
      break;
    }
  Q.win_entries = next_pow2(need_entries);
  Q.win_rows = next_pow2(need_rows);
  return Q.win_entries <= max_win_entries && Q.win_rows <= max_win_rows;
}

}  // namespace fne

namespace fne {

int build_block_plan(int64_t n_local, int npn, int bs, const int64_t* elem_dofs, const fne_desc* d, BlockPlan& P) {
  const int64_t lo = d->lo, hi = d->hi, nf = d->n_free, nnz = d->nnz, nt = d->n_total;
  const int64_t* t2f = d->total_to_free_reord;
  if (bs < 1 || bs > 3 || npn < 1 || (int64_t)npn * npn * n_local >= (int64_t)INT32_MAX ||
      (int64_t)npn * n_local >= (int64_t)INT32_MAX || nnz >= (int64_t)INT32_MAX)
    return set_error(FNE_EBOUNDS, "block plan: sizes beyond the packed format");
  // reordered free id -> total DOF
  std::vector<int64_t> orig(nf, -1);
  for (int64_t t = 0; t < nt; ++t)
    if (t2f[t] >= 0) orig[t2f[t]] = t;
  const int64_t n_nodes = (nt + bs - 1) / bs;
  // row nodes in the order of their first COO row
  std::vector<int32_t> rn_of(n_nodes, -1);
  std::vector<int64_t> rn_node;
  P.rn_row.clear();
  P.rn_gpos.clear();
  std::vector<int32_t> row_end;  // per (rn, c): end position of the row
  for (int64_t j = 0; j < nnz; ++j) {
    if (j > 0 && d->owned_rows[j] == d->owned_rows[j - 1]) continue;
    const int64_t r = d->owned_rows[j];
    if (r < lo || r >= hi) return set_error(FNE_ELAYOUT, "block plan: owned row outside [lo, hi)");
    const int64_t t = orig[r];
    const int64_t node = t / bs;
    const int c = (int)(t % bs);
    if (rn_of[node] < 0) {
      rn_of[node] = (int32_t)rn_node.size();
      rn_node.push_back(node);
      for (int k = 0; k < bs; ++k) {
        P.rn_row.push_back(-1);
        P.rn_gpos.push_back(-1);
        row_end.push_back(-1);
      }
    }
    const int32_t k = rn_of[node];
    if (P.rn_row[k * bs + c] >= 0) return set_error(FNE_ELAYOUT, "block plan: COO pattern is not row-grouped");
    P.rn_row[k * bs + c] = (int32_t)j;
    P.rn_gpos[k * bs + c] = (int32_t)(r - lo);
  }
  const int32_t n_rn = (int32_t)rn_node.size();
  for (int32_t k = 0; k < n_rn; ++k)
    for (int c = 0; c < bs; ++c) {
      const int32_t s0 = P.rn_row[k * bs + c];
      if (s0 < 0) continue;
      int64_t e = s0;
      while (e < nnz && d->owned_rows[e] == d->owned_rows[s0]) ++e;
      row_end[k * bs + c] = (int32_t)e;
    }
  // owned free rows without COO entries would be missed
  for (int64_t r = lo; r < hi; ++r) {
    const int64_t node = orig[r] / bs;
    if (rn_of[node] < 0 || P.rn_row[rn_of[node] * bs + (int)(orig[r] % bs)] < 0)
      return set_error(FNE_ELAYOUT, "block plan: owned row without COO entries");
  }
  P.n_rnodes = n_rn;
  // column-node blocks of every row node: consecutive columns of one node
  // form a block; all rows of the node must agree on the blocks
  std::vector<int32_t> rn_blk(n_rn + 1, 0);
  std::vector<int64_t> blk_node;
  std::vector<uint32_t> blk_word;
  for (int32_t k = 0; k < n_rn; ++k) {
    rn_blk[k] = (int32_t)blk_node.size();
    bool first_row = true;
    size_t b_first = blk_node.size();
    for (int c = 0; c < bs; ++c) {
      const int32_t s0 = P.rn_row[k * bs + c];
      if (s0 < 0) continue;
      const int32_t s1 = row_end[k * bs + c];
      size_t bi = b_first;
      int64_t j = s0;
      while (j < s1) {
        const int64_t node = orig[d->owned_cols[j]] / bs;
        const int64_t off = j - s0;
        uint32_t mask = 0;
        int prev = -1;
        while (j < s1 && orig[d->owned_cols[j]] / bs == node) {
          const int comp = (int)(orig[d->owned_cols[j]] % bs);
          if (comp <= prev) return set_error(FNE_ELAYOUT, "block plan: node columns not in component order");
          prev = comp;
          mask |= 1u << comp;
          ++j;
        }
        if (off > 0xFFFF) return set_error(FNE_EBOUNDS, "block plan: row longer than 65535 entries");
        const uint32_t w = (uint32_t)off | (mask << 16);
        if (first_row) {
          blk_node.push_back(node);
          blk_word.push_back(w);
        } else {
          if (bi >= blk_node.size() || blk_node[bi] != node || blk_word[bi] != w)
            return set_error(FNE_ELAYOUT, "block plan: rows of one node differ in their columns");
          ++bi;
        }
      }
      if (!first_row && bi != blk_node.size())
        return set_error(FNE_ELAYOUT, "block plan: rows of one node differ in their columns");
      first_row = false;
    }
  }
  rn_blk[n_rn] = (int32_t)blk_node.size();
  // (row node, column node) -> block: per row node, blocks sorted by node
  std::vector<int32_t> sorted_blk(blk_node.size());
  for (int32_t k = 0; k < n_rn; ++k) {
    for (int32_t b = rn_blk[k]; b < rn_blk[k + 1]; ++b) sorted_blk[b] = b;
    std::sort(sorted_blk.begin() + rn_blk[k], sorted_blk.begin() + rn_blk[k + 1],
              [&](int32_t x, int32_t y) { return blk_node[x] < blk_node[y]; });
  }
  auto find_blk = [&](int32_t k, int64_t node) -> int32_t {
    int32_t a = rn_blk[k], b = rn_blk[k + 1];
    while (a < b) {
      const int32_t m = (a + b) >> 1;
      if (blk_node[sorted_blk[m]] < node) a = m + 1; else b = m;
    }
    return (a < rn_blk[k + 1] && blk_node[sorted_blk[a]] == node) ? sorted_blk[a] : -1;
  };
  auto has_free = [&](int64_t node) {
    for (int c = 0; c < bs; ++c) {
      const int64_t t = node * bs + c;
      if (t < nt && t2f[t] >= 0) return true;
    }
    return false;
  };
  // contributions (count, fill) in element order; gradient incidences
  const int nde = npn * bs;
  std::vector<int32_t> cnt(blk_node.size() + 1, 0), fill;
  std::vector<int32_t> icnt(n_rn + 1, 0), ifill;
  std::vector<int32_t> con, inc;
  P.elem_rn.assign((size_t)n_local * npn, -1);
  for (int pass = 0; pass < 2; ++pass) {
    if (pass == 1) {
      for (size_t b = 0; b < blk_node.size(); ++b) cnt[b + 1] += cnt[b];
      for (int32_t k = 0; k < n_rn; ++k) icnt[k + 1] += icnt[k];
      con.assign(cnt[blk_node.size()], 0);
      inc.assign(icnt[n_rn], 0);
      fill.assign(cnt.begin(), cnt.end() - 1);
      ifill.assign(icnt.begin(), icnt.end() - 1);
    }
    for (int64_t el = 0; el < n_local; ++el) {
      const int64_t* ed = elem_dofs + el * nde;
      for (int a = 0; a < npn; ++a) {
        const int64_t na = ed[a * bs] / bs;
        if (na < 0 || na >= n_nodes) return set_error(FNE_EBOUNDS, "block plan: element DOF out of range");
        const int32_t k = rn_of[na];
        P.elem_rn[(size_t)el * npn + a] = k;
        if (k < 0) continue;
        if (pass == 0) icnt[k + 1]++; else inc[ifill[k]++] = (int32_t)(el * npn + a);
        for (int b = 0; b < npn; ++b) {
          const int64_t nb = ed[b * bs] / bs;
          if (!has_free(nb)) continue;
          const int32_t blk = find_blk(k, nb);
          if (blk < 0) return set_error(FNE_ELAYOUT, "Scatter lookup found mismatched owned COO entries");
          if (pass == 0) cnt[blk + 1]++; else con[fill[blk]++] = (int32_t)((el * npn + a) * npn + b);
        }
      }
    }
  }
  P.blk.resize(blk_node.size());
  for (size_t b = 0; b < blk_node.size(); ++b) {
    const int32_t c = cnt[b + 1] - cnt[b];
    if (c >= (1 << 13)) return set_error(FNE_EBOUNDS, "block plan: more than 8191 contributions to one block");
    P.blk[b] = blk_word[b] | ((uint32_t)c << 19);
  }
  P.rn_blk = std::move(rn_blk);
  P.rn_con.assign(n_rn + 1, 0);
  for (int32_t k = 0; k < n_rn; ++k) P.rn_con[k + 1] = cnt[P.rn_blk[k + 1]];
  P.rn_con[0] = 0;
  P.con = std::move(con);
  P.rn_inc = std::move(icnt);
  P.inc = std::move(inc);
  return FNE_OK;
}

}  // namespace fne

namespace fne {

int build_direct_plan(const BlockPlan& bp, int64_t n_local, int npn, int bs, DirectPlan& D) {
  const int nn = npn * npn;
  if (nn > 0x7FFF || bs > 3) return set_error(FNE_EBOUNDS, "direct plan: element too large");
  D.code.assign((size_t)n_local * nn, 0xFFFF);
  std::vector<int32_t> n_sh(n_local, 0);
  // pass 1: direct codes and shared counts
  for (int32_t k = 0; k < bp.n_rnodes; ++k) {
    int32_t c0 = bp.rn_con[k];
    for (int32_t b = bp.rn_blk[k]; b < bp.rn_blk[k + 1]; ++b) {
      const uint32_t w = bp.blk[b];
      const int32_t cnt = (int32_t)(w >> 19);
      const uint32_t off = w & 0xFFFFu, dm = (w >> 16) & 7u;
      for (int32_t j = c0; j < c0 + cnt; ++j) {
        const int32_t code = bp.con[j];
        const int32_t el = code / nn, a = (code % nn) / npn, bb = code % npn;
        if (cnt == 1) {
          if (off > 0xFFF) return set_error(FNE_EBOUNDS, "direct plan: row longer than 4095 entries");
          D.code[(size_t)el * nn + a * npn + bb] = (uint16_t)(off | (dm << 12));
        } else {
          n_sh[el]++;
        }
      }
      c0 += cnt;
    }
  }
  D.sbase.assign(n_local, 0);
  int64_t tot = 0;
  for (int64_t e = 0; e < n_local; ++e) {
    D.sbase[e] = (int32_t)tot;
    tot += n_sh[e];
    if (n_sh[e] > 0x7FFE) return set_error(FNE_EBOUNDS, "direct plan: too many shared blocks in one element");
  }
  if (tot >= (int64_t)INT32_MAX / 16) return set_error(FNE_EBOUNDS, "direct plan: shared buffer beyond 32-bit indexing");
  D.n_slots = tot;
  // pass 2: shared slots and the fix-up plan over the shared blocks
  std::fill(n_sh.begin(), n_sh.end(), 0);
  BlockPlan& F = D.fix;
  F = BlockPlan();
  F.rn_blk.push_back(0);
  F.rn_con.push_back(0);
  for (int32_t k = 0; k < bp.n_rnodes; ++k) {
    int32_t c0 = bp.rn_con[k];
    bool any = false;
    for (int32_t b = bp.rn_blk[k]; b < bp.rn_blk[k + 1]; ++b) {
      const uint32_t w = bp.blk[b];
      const int32_t cnt = (int32_t)(w >> 19);
      if (cnt >= 2) {
        any = true;
        F.blk.push_back(w);
        for (int32_t j = c0; j < c0 + cnt; ++j) {
          const int32_t code = bp.con[j];
          const int32_t el = code / nn, a = (code % nn) / npn, bb = code % npn;
          const int32_t slot = n_sh[el]++;
          D.code[(size_t)el * nn + a * npn + bb] = (uint16_t)(0x8000u | (uint32_t)slot);
          F.con.push_back(D.sbase[el] + slot);
        }
      }
      c0 += cnt;
    }
    if (any) {
      for (int c = 0; c < bs; ++c) F.rn_row.push_back(bp.rn_row[(size_t)k * bs + c]);
      F.rn_blk.push_back((int32_t)F.blk.size());
      F.rn_con.push_back((int32_t)F.con.size());
    }
  }
  F.n_rnodes = (int32_t)F.rn_blk.size() - 1;
  // fix-up order of the slots (used when the buffer is laid out that way)
  D.sidx.assign((size_t)tot, -1);
  for (size_t j = 0; j < F.con.size(); ++j) D.sidx[(size_t)F.con[j]] = (int32_t)j;
  // flat fix-up (bs = 2): one descriptor per shared block; its contributions
  // are the buffer slots fix.con[start .. start + count)
  if (bs == 2) {
    D.fdesc.clear();
    for (int32_t k = 0; k < F.n_rnodes; ++k) {
      int32_t c0 = F.rn_con[k];
      for (int32_t b = F.rn_blk[k]; b < F.rn_blk[k + 1]; ++b) {
        const uint32_t w = F.blk[b];
        const int32_t cnt = (int32_t)(w >> 19);
        const int32_t off = (int32_t)(w & 0xFFFFu);
        const int32_t r0 = F.rn_row[(size_t)k * 2], r1 = F.rn_row[(size_t)k * 2 + 1];
        D.fdesc.push_back(r0 >= 0 ? r0 + off : -1);
        D.fdesc.push_back(r1 >= 0 ? r1 + off : -1);
        D.fdesc.push_back(c0);
        D.fdesc.push_back(cnt | (int32_t)(((w >> 16) & 7u) << 16));
        c0 += cnt;
      }
    }
  }
  return FNE_OK;
}

}  // namespace fne

// ---------------------------------------------------------------------------
// Row-cluster plan (see ClusterPlan in fne_internal.h).
// ---------------------------------------------------------------------------
namespace fne {

bool build_cluster_plan(const RowPlan& P, int64_t lo, int64_t hi, int max_rows, int max_jobs, int max_incs,
                        int max_win, bool gpos_identity, ClusterPlan& Q) {
  const int32_t n_local = (int32_t)P.local_elems.size();
  const int32_t n_rows = P.n_rows;
  if (n_local == 0 || n_rows == 0 || P.elem_code.size() != (size_t)n_local * 3) return false;
  if (max_rows < 1 || max_jobs < 8 || max_jobs > (1 << kClJobBits) || max_incs < 8) return false;
  if ((int64_t)n_rows != hi - lo || P.n_nodes != n_rows) return false;  // scalar rows: one per owned node
  std::vector<int32_t> row_of((size_t)(hi - lo), -1);
  for (int32_t k = 0; k < n_rows; ++k) {
    row_of[P.row_gpos[k]] = k;
    if (P.row_ptr[k + 1] - P.row_ptr[k] > 14) return false;  // 4-bit column offsets
  }
  auto inc_begin = [&](int32_t k) { return P.inc_ptr[P.row_node[k]]; };
  auto inc_end = [&](int32_t k) { return P.inc_ptr[P.row_node[k] + 1]; };
  auto row_len = [&](int32_t k) { return P.row_ptr[k + 1] - P.row_ptr[k]; };
  for (int32_t k = 0; k < n_rows; ++k)
    if (inc_end(k) - inc_begin(k) + 3 > std::min(max_jobs, max_incs) || row_len(k) > max_win) return false;
  // jobs a row adds to cluster c (its elements not yet in c)
  std::vector<int32_t> estamp(n_local, -1);
  auto new_jobs = [&](int32_t k, int32_t c, bool commit) {
    int32_t n = 0;
    for (int32_t i = inc_begin(k); i < inc_end(k); ++i) {
      const int32_t le = P.inc_elem[i];
      if (estamp[le] != c) {
        ++n;
        if (commit) estamp[le] = c;
      }
    }
    return n;
  };

  // ---- graph-grown clusters: BFS from the lowest unassigned row ------------
  std::vector<int32_t> cl_of(n_rows, -1), queue;
  std::vector<std::vector<int32_t>> clusters;
  queue.reserve(n_rows);
  int32_t seed = 0;
  while (true) {
    while (seed < n_rows && cl_of[seed] >= 0) ++seed;
    if (seed >= n_rows) break;
    const int32_t c = (int32_t)clusters.size();
    clusters.emplace_back();
    std::vector<int32_t>& rows = clusters.back();
    int64_t njobs = new_jobs(seed, c, true);
    int64_t nincs = inc_end(seed) - inc_begin(seed);
    int64_t nwin = row_len(seed);
    cl_of[seed] = c;
    rows.push_back(seed);
    queue.clear();
    queue.push_back(seed);
    bool full = false;
    for (size_t qh = 0; qh < queue.size() && !full; ++qh) {
      const int32_t k = queue[qh];
      for (int32_t i = inc_begin(k); i < inc_end(k) && !full; ++i) {
        const int32_t le = P.inc_elem[i];
        for (int b = 0; b < 3; ++b) {
          const int32_t cb = P.elem_code[(size_t)le * 3 + b];
          if (cb < lo || cb >= hi) continue;
          const int32_t kb = row_of[cb - lo];
          if (kb < 0 || cl_of[kb] >= 0) continue;
          const int32_t ni = inc_end(kb) - inc_begin(kb);
          // + 3: padding to a multiple of 4
          if ((int)rows.size() >= max_rows || njobs + new_jobs(kb, c, false) + 3 > max_jobs ||
              nincs + ni + 3 > max_incs || nwin + row_len(kb) > max_win) {
            full = true;
            break;
          }
          cl_of[kb] = c;
          rows.push_back(kb);
          njobs += new_jobs(kb, c, true);
          nincs += ni;
          nwin += row_len(kb);
          queue.push_back(kb);
        }
      }
    }
  }
  const int32_t n_cl = (int32_t)clusters.size();

  // ---- per cluster: jobs (energy-counting first), rows, incidences ---------
  Q = ClusterPlan{};
  Q.n_cl = n_cl;
  Q.table.reserve((size_t)n_cl * 8);
  std::vector<int32_t> stamp(n_local, -1), slot(n_local, -1);
  std::vector<std::pair<int32_t, int32_t>> jobs;  // (energy ? 0 : 1, local element)
  for (int32_t c = 0; c < n_cl; ++c) {
    std::vector<int32_t>& rows = clusters[c];
    std::sort(rows.begin(), rows.end());
    jobs.clear();
    for (int32_t k : rows)
      for (int32_t i = inc_begin(k); i < inc_end(k); ++i) {
        const int32_t le = P.inc_elem[i];
        if (stamp[le] != c) {
          stamp[le] = c;
          slot[le] = (int32_t)jobs.size();
          jobs.emplace_back(1, le);
        }
      }
    // the element energy is counted where the element's energy row (its
    // first owned node, energy weight 1) lies
    for (int32_t k : rows)
      for (int32_t i = inc_begin(k); i < inc_end(k); ++i)
        if (P.inc_info[i] & kEnergyFlag) jobs[slot[P.inc_elem[i]]].first = 0;
    std::sort(jobs.begin(), jobs.end());
    const int32_t j0 = (int32_t)Q.job_elem.size();
    int32_t je = j0;
    for (const auto& jb : jobs) {
      slot[jb.second] = (int32_t)Q.job_elem.size() - j0;
      Q.job_elem.push_back(jb.second);
      if (jb.first == 0) je = (int32_t)Q.job_elem.size();
    }
    while (Q.job_elem.size() % 4) Q.job_elem.push_back(-1);
    const int32_t j1 = (int32_t)Q.job_elem.size();
    const int32_t r0 = (int32_t)(Q.rows.size() / 4), i0 = (int32_t)Q.incs.size();
    const int32_t u0 = (int32_t)(Q.runs.size() / 4);
    int32_t wo = 0;
    for (int32_t k : rows) {
      const int32_t n_inc = inc_end(k) - inc_begin(k), len = row_len(k);
      if (n_inc > 0x7fff) return false;
      Q.rows.insert(Q.rows.end(), {gpos_identity ? k : P.row_gpos[k], wo, len | (n_inc << 16),
                                   (int32_t)Q.incs.size() - i0});
      // runs of rows whose COO ranges are adjacent
      const size_t nu = Q.runs.size() / 4;
      if (len > 0) {
        if ((int32_t)nu > u0 && Q.runs[4 * (nu - 1) + 1] + Q.runs[4 * (nu - 1) + 2] == P.row_ptr[k])
          Q.runs[4 * (nu - 1) + 2] += len;
        else
          Q.runs.insert(Q.runs.end(), {wo, P.row_ptr[k], len, 0});
      }
      wo += len;
      for (int32_t i = inc_begin(k); i < inc_end(k); ++i) {
        const uint32_t info = P.inc_info[i];
        uint32_t w = (uint32_t)slot[P.inc_elem[i]] | ((info & 3u) << kClJobBits);
        for (int b = 0; b < 3; ++b) {
          uint32_t off = (info >> (kOffShift + kOffBits * b)) & 127u;
          if (off == kNoCol) off = kClNoCol;
          w |= off << (kClJobBits + 2 + 4 * b);
        }
        Q.incs.push_back(w);
      }
    }
    while (Q.incs.size() % 4) Q.incs.push_back(0u);
    const int32_t r1 = (int32_t)(Q.rows.size() / 4), i1 = (int32_t)Q.incs.size();
    Q.table.insert(Q.table.end(), {j0, je, j1, r0, r1, i0, i1, u0});
    Q.max_win = std::max(Q.max_win, wo);
    Q.max_runs = std::max(Q.max_runs, (int32_t)(Q.runs.size() / 4) - u0);
    Q.max_jobs = std::max(Q.max_jobs, j1 - j0);
    Q.max_rows = std::max(Q.max_rows, r1 - r0);
    Q.max_incs = std::max(Q.max_incs, i1 - i0);
    if (Q.max_jobs > max_jobs || Q.max_incs > max_incs) return false;
    if (Q.job_elem.size() >= (size_t)INT32_MAX / 8 || Q.incs.size() >= (size_t)INT32_MAX / 8) return false;
  }
  const int32_t nj = (int32_t)Q.job_elem.size(), nr = (int32_t)(Q.rows.size() / 4);
  const int32_t ni = (int32_t)Q.incs.size(), nu = (int32_t)(Q.runs.size() / 4);
  Q.table.insert(Q.table.end(), {nj, nj, nj, nr, nr, ni, ni, nu});
  return true;
}

}  // namespace fne
