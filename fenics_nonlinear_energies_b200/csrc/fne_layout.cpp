// Host-side DOF layout: permutation, PETSc ownership split, owned COO pattern
// and element owners.  Same results as the reference's build_global_layout
// (src/core/petsc/reordered_element_base.py:380-506) for the global-adjacency
// branch, with select_permutation modes 'none' and 'block_xyz' (:159-200) and
// the PETSc block split of src/core/petsc/dof_partition.py:27-55, 502-521.
#include "fne_internal.h"

#include <algorithm>
#include <cstring>
#include <numeric>

namespace fne {

void ownership_range(int64_t n, int rank, int size, int bs, int64_t* lo, int64_t* hi) {
  if (bs > 1) {
    int64_t l, h;
    ownership_range(n / bs, rank, size, 1, &l, &h);
    *lo = l * bs;
    *hi = h * bs;
    return;
  }
  int64_t q = n / size, r = n % size;
  if (rank < r) {
    *lo = rank * (q + 1);
    *hi = *lo + q + 1;
  } else {
    *lo = rank * q + r;
    *hi = *lo + q;
  }
}

int64_t rank_of_dof(int64_t dof, int64_t n, int size, int bs) {
  if (bs > 1) return rank_of_dof(dof / bs, n / bs, size, 1);
  int64_t q = n / size, r = n % size;
  int64_t boundary = r * (q + 1);
  if (dof < boundary) return dof / (q + 1);
  return r + (dof - boundary) / q;
}

// Free-DOF adjacency in original free numbering, CSR with ascending columns:
// the union of all (free, free) DOF pairs of each element.
void element_adjacency(int64_t n_total, int64_t n_free, const int64_t* freedofs, int64_t n_elem,
                       int ndof_e, const int64_t* elems, std::vector<int64_t>& indptr,
                       std::vector<int64_t>& indices) {
  std::vector<int64_t> t2f(n_total, -1);
  for (int64_t i = 0; i < n_free; ++i) t2f[freedofs[i]] = i;
  // free dof -> incident elements
  std::vector<int64_t> cnt(n_free + 1, 0);
  for (int64_t e = 0; e < n_elem; ++e)
    for (int k = 0; k < ndof_e; ++k) {
      int64_t f = t2f[elems[e * ndof_e + k]];
      if (f >= 0) cnt[f + 1]++;
    }
  for (int64_t i = 0; i < n_free; ++i) cnt[i + 1] += cnt[i];
  std::vector<int64_t> inc(cnt[n_free]);
  std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
  for (int64_t e = 0; e < n_elem; ++e)
    for (int k = 0; k < ndof_e; ++k) {
      int64_t f = t2f[elems[e * ndof_e + k]];
      if (f >= 0) inc[fill[f]++] = e;
    }
  indptr.assign(n_free + 1, 0);
  indices.clear();
  std::vector<int64_t> cols;
  for (int64_t r = 0; r < n_free; ++r) {
    cols.clear();
    for (int64_t j = cnt[r]; j < cnt[r + 1]; ++j) {
      int64_t e = inc[j];
      for (int k = 0; k < ndof_e; ++k) {
        int64_t c = t2f[elems[e * ndof_e + k]];
        if (c >= 0) cols.push_back(c);
      }
    }
    std::sort(cols.begin(), cols.end());
    cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
    indices.insert(indices.end(), cols.begin(), cols.end());
    indptr[r + 1] = (int64_t)indices.size();
  }
}

}  // namespace fne

using namespace fne;

namespace fne {

int layout_check_desc(const fne_layout_desc* d) {
  const int bs = d->block_size;
  if (bs < 1 || d->n_free < 0 || d->n_total < d->n_free || d->ndof_e < 1 || d->n_elem < 0 ||
      d->comm_size < 1 || d->comm_rank < 0 || d->comm_rank >= d->comm_size)
    return set_error(FNE_EINVAL, "fne_layout_build: invalid sizes");
  if (d->n_free % bs != 0)
    return set_error(FNE_EINVAL, "fne_layout_build: n_free not divisible by block_size");
  for (int64_t i = 0; i < d->n_free; ++i) {
    if (d->freedofs[i] < 0 || d->freedofs[i] >= d->n_total)
      return set_error(FNE_EBOUNDS, "fne_layout_build: freedof out of range");
    if (i && d->freedofs[i] <= d->freedofs[i - 1])
      return set_error(FNE_EINVAL, "fne_layout_build: freedofs must be strictly ascending");
  }
  for (int64_t i = 0; i < d->n_elem * (int64_t)d->ndof_e; ++i)
    if (d->elems[i] < 0 || d->elems[i] >= d->n_total)
      return set_error(FNE_EBOUNDS, "fne_layout_build: element DOF out of range");
  return FNE_OK;
}

}  // namespace fne

extern "C" int fne_layout_build(const fne_layout_desc* d, fne_layout** out) {
  if (!d || !out) return set_error(FNE_EINVAL, "fne_layout_build: null argument");
  *out = nullptr;
  const int bs = d->block_size;
  if (const int rc = layout_check_desc(d); rc != FNE_OK) return rc;

  auto* L = new (std::nothrow) fne_layout();
  if (!L) return set_error(FNE_ENOMEM, "fne_layout_build: out of host memory");
  const int64_t nf = d->n_free;
  L->n_total = d->n_total;
  L->n_free = nf;
  L->n_elem = d->n_elem;

  // --- permutation (select_permutation :183-200) ---
  L->perm.resize(nf);
  if (d->perm_override) {
    std::vector<char> seen(nf, 0);
    for (int64_t i = 0; i < nf; ++i) {
      int64_t p = d->perm_override[i];
      if (p < 0 || p >= nf || seen[p]) {
        delete L;
        return set_error(FNE_EINVAL,
                         "Permutation override must contain each free DOF exactly once");
      }
      seen[p] = 1;
      L->perm[i] = p;
    }
  } else if (d->reorder == FNE_REORDER_NONE) {
    std::iota(L->perm.begin(), L->perm.end(), 0);
  } else if (d->reorder == FNE_REORDER_BLOCK_XYZ) {
    // perm_block_xyz (:159-170): node of every block_size-th free DOF, stable
    // lexicographic sort on (x, y, z), expanded back to DOFs.
    if (!d->coords || d->dim < 1) {
      delete L;
      return set_error(FNE_EINVAL, "block_xyz needs node coordinates");
    }
    const int64_t nb = nf / bs;
    std::vector<int64_t> node(nb), bp(nb);
    for (int64_t i = 0; i < nb; ++i) {
      node[i] = d->freedofs[i * bs] / bs;
      if (node[i] >= d->n_nodes) {
        delete L;
        return set_error(FNE_EBOUNDS, "block_xyz: node id beyond coords");
      }
    }
    std::iota(bp.begin(), bp.end(), 0);
    const double* X = d->coords;
    const int dim = d->dim;
    std::stable_sort(bp.begin(), bp.end(), [&](int64_t a, int64_t b) {
      const double* xa = X + node[a] * dim;
      const double* xb = X + node[b] * dim;
      for (int k = 0; k < dim; ++k) {
        if (xa[k] < xb[k]) return true;
        if (xb[k] < xa[k]) return false;
      }
      return false;
    });
    for (int64_t i = 0; i < nb; ++i)
      for (int c = 0; c < bs; ++c) L->perm[i * bs + c] = bp[i] * bs + c;
  } else {
    delete L;
    return set_error(FNE_EINVAL, "Unsupported element reorder mode");
  }
  L->iperm.resize(nf);
  for (int64_t i = 0; i < nf; ++i) L->iperm[L->perm[i]] = i;

  ownership_range(nf, d->comm_rank, d->comm_size, bs, &L->lo, &L->hi);

  L->t2f.assign(d->n_total, -1);
  for (int64_t i = 0; i < nf; ++i) L->t2f[d->freedofs[i]] = L->iperm[i];

  // --- adjacency (CSR storage order, as adjacency.tocsr().nonzero()) ---
  std::vector<int64_t> indptr, indices;
  if (d->adj_indptr && d->adj_indices) {
    indptr.assign(d->adj_indptr, d->adj_indptr + nf + 1);
    indices.assign(d->adj_indices, d->adj_indices + indptr[nf]);
    for (int64_t c : indices)
      if (c < 0 || c >= nf) {
        delete L;
        return set_error(FNE_EBOUNDS, "adjacency column out of range");
      }
  } else {
    element_adjacency(d->n_total, nf, d->freedofs, d->n_elem, d->ndof_e, d->elems, indptr,
                      indices);
  }
  const int64_t nnz = indptr[nf];
  L->coo_rows.resize(nnz);
  L->coo_cols.resize(nnz);
  for (int64_t r = 0; r < nf; ++r)
    for (int64_t j = indptr[r]; j < indptr[r + 1]; ++j) {
      L->coo_rows[j] = L->iperm[r];
      L->coo_cols[j] = L->iperm[indices[j]];
    }
  for (int64_t j = 0; j < nnz; ++j)
    if (L->coo_rows[j] >= L->lo && L->coo_rows[j] < L->hi) {
      L->owned_rows.push_back(L->coo_rows[j]);
      L->owned_cols.push_back(L->coo_cols[j]);
    }

  // --- element owners (:439-450): rank of the element's smallest reordered DOF ---
  L->elem_owner.assign(d->n_elem, -1);
  for (int64_t e = 0; e < d->n_elem; ++e) {
    int64_t mn = nf;
    for (int k = 0; k < d->ndof_e; ++k) {
      int64_t r = L->t2f[d->elems[e * d->ndof_e + k]];
      if (r >= 0 && r < mn) mn = r;
    }
    if (mn < nf) L->elem_owner[e] = rank_of_dof(mn, nf, d->comm_size, bs);
  }
  *out = L;
  return FNE_OK;
}

extern "C" int fne_layout_sizes(const fne_layout* L, int64_t* n_free, int64_t* lo, int64_t* hi,
                                int64_t* nnz_total, int64_t* nnz_owned, int64_t* n_elem) {
  if (!L) return set_error(FNE_EINVAL, "fne_layout_sizes: null layout");
  if (n_free) *n_free = L->n_free;
  if (lo) *lo = L->lo;
  if (hi) *hi = L->hi;
  if (nnz_total) *nnz_total = L->on_device ? L->dev.nnz_total : (int64_t)L->coo_rows.size();
  if (nnz_owned) *nnz_owned = L->on_device ? L->dev.nnz_owned : (int64_t)L->owned_rows.size();
  if (n_elem) *n_elem = L->n_elem;
  return FNE_OK;
}

extern "C" int fne_layout_copy(const fne_layout* L, int64_t* perm, int64_t* iperm, int64_t* t2f,
                               int64_t* coo_rows, int64_t* coo_cols, int64_t* owned_rows,
                               int64_t* owned_cols, int64_t* elem_owner) {
  if (!L) return set_error(FNE_EINVAL, "fne_layout_copy: null layout");
  if (L->on_device) return layout_device_copy(L, perm, iperm, t2f, coo_rows, coo_cols, owned_rows, owned_cols,
                                              elem_owner);
  auto cp = [](int64_t* dst, const std::vector<int64_t>& v) {
    if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(int64_t));
  };
  cp(perm, L->perm);
  cp(iperm, L->iperm);
  cp(t2f, L->t2f);
  cp(coo_rows, L->coo_rows);
  cp(coo_cols, L->coo_cols);
  cp(owned_rows, L->owned_rows);
  cp(owned_cols, L->owned_cols);
  cp(elem_owner, L->elem_owner);
  return FNE_OK;
}

extern "C" void fne_layout_free(fne_layout* L) {
  if (L && L->on_device) layout_device_release(L);
  delete L;
}
