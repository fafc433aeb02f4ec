// Device DOF layout: the arrays of fne_layout_build (fne_layout.cpp) built on
// the GPU, bit for bit the same.  Replaces the reference's
// build_global_layout (src/core/petsc/reordered_element_base.py:380-506) and
// select_permutation (:159-200) for large meshes, where the host build is
// seconds and the reference's minutes.
//
//  * block_xyz permutation: a stable lexicographic sort of the free blocks'
//    nodes on (x, y, z) = three stable radix sorts (z, then y, then x) of
//    order-preserving 64-bit images of the coordinates;
//  * adjacency (no adjacency given): every (row, col) free-DOF pair of every
//    element as the key row * n_free + col (original free numbering),
//    radix-sorted and made unique: rows ascending, columns ascending within a
//    row, as scipy's CSR of the element graph;
//  * COO = iperm[row], iperm[col]; owned = the entries whose row is in
//    [lo, hi), order kept (stable selection); element owner = rank of the
//    element's smallest reordered free DOF.
// Sorting and selection use CUB (CUDA toolkit headers).  The arguments are
// checked on the host exactly as fne_layout_build checks them.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>

#include <algorithm>
#include <cstdint>
#include <new>
#include <string>
#include <vector>

#include "fne_internal.h"

namespace fne {
namespace {

constexpr int kT = 256;

int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + kT - 1) / kT, 148 * 64)); }

#define FNE_GRID_STRIDE(i, n) \
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

__global__ void k_fill(int64_t* a, int64_t n, int64_t v) {
  FNE_GRID_STRIDE(i, n) a[i] = v;
}

__global__ void k_iota(int64_t* a, int64_t n) {
  FNE_GRID_STRIDE(i, n) a[i] = i;
}

// out[idx[i]] = i (inverse permutation, total -> free position)
__global__ void k_scatter_pos(const int64_t* __restrict__ idx, int64_t n, int64_t* __restrict__ out) {
  FNE_GRID_STRIDE(i, n) out[idx[i]] = i;
}

// out[idx[i]] = val[i]
__global__ void k_scatter_val(const int64_t* __restrict__ idx, const int64_t* __restrict__ val, int64_t n,
                              int64_t* __restrict__ out) {
  FNE_GRID_STRIDE(i, n) out[idx[i]] = val[i];
}

__global__ void k_block_nodes(const int64_t* __restrict__ freedofs, int64_t nb, int bs, int64_t n_nodes,
                              int64_t* __restrict__ node, int* err) {
  FNE_GRID_STRIDE(i, nb) {
    const int64_t v = freedofs[i * bs] / bs;
    node[i] = v < n_nodes ? v : 0;
    if (v >= n_nodes) atomicOr(err, 1);
  }
}

// Order-preserving unsigned image of a double (-0.0 and +0.0 map together,
// as they compare equal).
__device__ __forceinline__ uint64_t ordered_bits(double v) {
  if (v == 0.0) v = 0.0;
  const uint64_t u = (uint64_t)__double_as_longlong(v);
  return (u >> 63) ? ~u : (u | (1ull << 63));
}

__global__ void k_coord_keys(const double* __restrict__ X, int dim, int k, const int64_t* __restrict__ node,
                             const int64_t* __restrict__ order, int64_t nb, uint64_t* __restrict__ key) {
  FNE_GRID_STRIDE(i, nb) key[i] = ordered_bits(X[node[order[i]] * dim + k]);
}

__global__ void k_expand_perm(const int64_t* __restrict__ bp, int64_t nb, int bs, int64_t* __restrict__ perm) {
  FNE_GRID_STRIDE(i, nb) {
    for (int c = 0; c < bs; ++c) perm[i * bs + c] = bp[i] * bs + c;
  }
}

// One key per (element, local DOF a, local DOF b); pairs with a Dirichlet
// DOF get the sentinel n_free^2, which sorts last.
__global__ void k_pairs(const int64_t* __restrict__ elems, int64_t n_elem, int k,
                        const int64_t* __restrict__ t2f_orig, int64_t nf, uint64_t* __restrict__ keys) {
  const int64_t kk = (int64_t)k * k;
  FNE_GRID_STRIDE(idx, n_elem * kk) {
    const int64_t e = idx / kk;
    const int a = (int)((idx / k) % k), b = (int)(idx % k);
    const int64_t fa = t2f_orig[elems[e * k + a]], fb = t2f_orig[elems[e * k + b]];
    keys[idx] = (fa >= 0 && fb >= 0) ? (uint64_t)(fa * nf + fb) : (uint64_t)nf * (uint64_t)nf;
  }
}

__global__ void k_coo_from_keys(const uint64_t* __restrict__ keys, int64_t nnz, int64_t nf,
                                const int64_t* __restrict__ iperm, int64_t* __restrict__ rows,
                                int64_t* __restrict__ cols) {
  FNE_GRID_STRIDE(j, nnz) {
    const int64_t key = (int64_t)keys[j];
    rows[j] = iperm[key / nf];
    cols[j] = iperm[key % nf];
  }
}

// Given adjacency (CSR, storage order): thread per row.
__global__ void k_coo_from_csr(const int64_t* __restrict__ indptr, const int64_t* __restrict__ indices, int64_t nf,
                               const int64_t* __restrict__ iperm, int64_t* __restrict__ rows,
                               int64_t* __restrict__ cols, int* err) {
  FNE_GRID_STRIDE(r, nf) {
    const int64_t ir = iperm[r];
    for (int64_t j = indptr[r]; j < indptr[r + 1]; ++j) {
      const int64_t c = indices[j];
      const bool ok = c >= 0 && c < nf;
      if (!ok) atomicOr(err, 2);
      rows[j] = ir;
      cols[j] = ok ? iperm[c] : -1;
    }
  }
}

__global__ void k_owned_flags(const int64_t* __restrict__ rows, int64_t nnz, int64_t lo, int64_t hi,
                              char* __restrict__ flags) {
  FNE_GRID_STRIDE(j, nnz) flags[j] = rows[j] >= lo && rows[j] < hi;
}

__device__ int64_t rank_of_dof_dev(int64_t dof, int64_t n, int size, int bs) {
  if (bs > 1) {
    dof /= bs;
    n /= bs;
  }
  const int64_t q = n / size, r = n % size;
  const int64_t boundary = r * (q + 1);
  if (dof < boundary) return dof / (q + 1);
  return r + (dof - boundary) / q;
}

__global__ void k_elem_owner(const int64_t* __restrict__ elems, int64_t n_elem, int k,
                             const int64_t* __restrict__ t2f, int64_t nf, int size, int bs,
                             int64_t* __restrict__ owner) {
  FNE_GRID_STRIDE(e, n_elem) {
    int64_t mn = nf;
    for (int a = 0; a < k; ++a) {
      const int64_t r = t2f[elems[e * k + a]];
      if (r >= 0 && r < mn) mn = r;
    }
    owner[e] = mn < nf ? rank_of_dof_dev(mn, nf, size, bs) : -1;
  }
}

// Device buffers of one build; freed on every exit path.
struct Scratch {
  std::vector<void*> ptrs;
  ~Scratch() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <typename T>
  T* alloc(int64_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, (size_t)std::max<int64_t>(1, n) * sizeof(T)) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
  template <typename T>
  T* upload(const T* h, int64_t n) {
    T* d = alloc<T>(n);
    if (d && n > 0 && cudaMemcpy(d, h, (size_t)n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
    return d;
  }
  // hands a buffer over to the layout (no longer freed here)
  void keep(void* p) { ptrs.erase(std::remove(ptrs.begin(), ptrs.end(), p), ptrs.end()); }
};

int bit_width(uint64_t v) {
  int b = 0;
  while (v) {
    ++b;
    v >>= 1;
  }
  return std::max(b, 1);
}

int cuda_fail(const char* what) {
  const cudaError_t e = cudaGetLastError();
  return set_error(e == cudaErrorMemoryAllocation ? FNE_ENOMEM : FNE_ECUDA,
                   std::string("fne_layout_build_device: ") + what + ": " + cudaGetErrorString(e));
}

}  // namespace

int layout_device_copy(const fne_layout* L, int64_t* perm, int64_t* iperm, int64_t* t2f, int64_t* coo_rows,
                       int64_t* coo_cols, int64_t* owned_rows, int64_t* owned_cols, int64_t* elem_owner) {
  struct Item {
    int64_t* dst;
    const int64_t* src;
    int64_t n;
  } items[] = {{perm, L->dev.perm, L->n_free},
               {iperm, L->dev.iperm, L->n_free},
               {t2f, L->dev.t2f, L->n_total},
               {coo_rows, L->dev.coo_rows, L->dev.nnz_total},
               {coo_cols, L->dev.coo_cols, L->dev.nnz_total},
               {owned_rows, L->dev.owned_rows, L->dev.nnz_owned},
               {owned_cols, L->dev.owned_cols, L->dev.nnz_owned},
               {elem_owner, L->dev.elem_owner, L->n_elem}};
  for (const Item& it : items)
    if (it.dst && it.n > 0 &&
        cudaMemcpy(it.dst, it.src, (size_t)it.n * sizeof(int64_t), cudaMemcpyDeviceToHost) != cudaSuccess)
      return set_error(FNE_ECUDA, std::string("fne_layout_copy: ") + cudaGetErrorString(cudaGetLastError()));
  return FNE_OK;
}

void layout_device_release(fne_layout* L) {
  auto& d = L->dev;
  if (!d.owned_is_coo) {
    cudaFree(d.owned_rows);
    cudaFree(d.owned_cols);
  }
  for (int64_t* p : {d.perm, d.iperm, d.t2f, d.coo_rows, d.coo_cols, d.elem_owner}) cudaFree(p);
  d = {};
}

}  // namespace fne

using namespace fne;

extern "C" int fne_layout_build_device(const fne_layout_desc* d, fne_layout** out) {
  if (!d || !out) return set_error(FNE_EINVAL, "fne_layout_build_device: null argument");
  *out = nullptr;
  if (const int rc = layout_check_desc(d); rc != FNE_OK) return rc;
  const int bs = d->block_size;
  const int64_t nf = d->n_free, nt = d->n_total, ne = d->n_elem;
  const int k = d->ndof_e;
  const bool given_adj = d->adj_indptr && d->adj_indices;
  if (!given_adj && nf > 0 && (uint64_t)nf > (uint64_t)3037000499ll)  // nf^2 must fit in 63 bits
    return set_error(FNE_EINVAL, "fne_layout_build_device: too many free DOFs for 64-bit pair keys");
  int64_t perm_override_bad = -1;
  if (d->perm_override) {
    std::vector<char> seen(nf, 0);
    for (int64_t i = 0; i < nf && perm_override_bad < 0; ++i) {
      const int64_t p = d->perm_override[i];
      if (p < 0 || p >= nf || seen[p]) perm_override_bad = i;
      else seen[p] = 1;
    }
    if (perm_override_bad >= 0)
      return set_error(FNE_EINVAL, "Permutation override must contain each free DOF exactly once");
  } else if (d->reorder == FNE_REORDER_BLOCK_XYZ) {
    if (!d->coords || d->dim < 1) return set_error(FNE_EINVAL, "block_xyz needs node coordinates");
  } else if (d->reorder != FNE_REORDER_NONE) {
    return set_error(FNE_EINVAL, "Unsupported element reorder mode");
  }
  std::vector<int64_t> h_indptr;
  if (given_adj) {
    h_indptr.assign(d->adj_indptr, d->adj_indptr + nf + 1);
    for (int64_t r = 0; r < nf; ++r)
      if (h_indptr[r + 1] < h_indptr[r]) return set_error(FNE_EINVAL, "adjacency indptr must be non-decreasing");
  }

  Scratch S;
  int* err = S.alloc<int>(1);
  const int64_t* freedofs = S.upload(d->freedofs, nf);
  const int64_t* elems = S.upload(d->elems, ne * k);
  int64_t* perm = S.alloc<int64_t>(nf);
  int64_t* iperm = S.alloc<int64_t>(nf);
  int64_t* t2f = S.alloc<int64_t>(nt);
  int64_t* t2f_orig = S.alloc<int64_t>(nt);
  int64_t* owner = S.alloc<int64_t>(ne);
  if (!err || !freedofs || !elems || !perm || !iperm || !t2f || !t2f_orig || !owner)
    return cuda_fail("allocation / upload");
  cudaMemset(err, 0, sizeof(int));

  // --- permutation ---
  if (d->perm_override) {
    if (nf > 0 && cudaMemcpy(perm, d->perm_override, (size_t)nf * sizeof(int64_t), cudaMemcpyHostToDevice) !=
                      cudaSuccess)
      return cuda_fail("upload");
  } else if (d->reorder == FNE_REORDER_NONE) {
    k_iota<<<grid_for(nf), kT>>>(perm, nf);
  } else {
    const int64_t nb = nf / bs;
    const double* X = S.upload(d->coords, d->n_nodes * (int64_t)d->dim);
    int64_t* node = S.alloc<int64_t>(nb);
    int64_t* ord[2] = {S.alloc<int64_t>(nb), S.alloc<int64_t>(nb)};
    uint64_t* key[2] = {S.alloc<uint64_t>(nb), S.alloc<uint64_t>(nb)};
    if (!X || !node || !ord[0] || !ord[1] || !key[0] || !key[1]) return cuda_fail("allocation / upload");
    k_block_nodes<<<grid_for(nb), kT>>>(freedofs, nb, bs, d->n_nodes, node, err);
    k_iota<<<grid_for(nb), kT>>>(ord[0], nb);
    cub::DoubleBuffer<uint64_t> kb(key[0], key[1]);
    cub::DoubleBuffer<int64_t> vb(ord[0], ord[1]);
    size_t tmp_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, kb, vb, nb);
    void* tmp = S.alloc<char>((int64_t)tmp_bytes);
    if (!tmp) return cuda_fail("allocation");
    for (int c = d->dim - 1; c >= 0; --c) {  // least significant coordinate first; radix sort is stable
      k_coord_keys<<<grid_for(nb), kT>>>(X, d->dim, c, node, vb.Current(), nb, kb.Current());
      size_t bytes = tmp_bytes;
      if (cub::DeviceRadixSort::SortPairs(tmp, bytes, kb, vb, nb) != cudaSuccess) return cuda_fail("coordinate sort");
    }
    k_expand_perm<<<grid_for(nb), kT>>>(vb.Current(), nb, bs, perm);
  }
  k_scatter_pos<<<grid_for(nf), kT>>>(perm, nf, iperm);
  k_fill<<<grid_for(nt), kT>>>(t2f, nt, -1);
  k_scatter_val<<<grid_for(nf), kT>>>(freedofs, iperm, nf, t2f);
  k_fill<<<grid_for(nt), kT>>>(t2f_orig, nt, -1);
  k_scatter_pos<<<grid_for(nf), kT>>>(freedofs, nf, t2f_orig);
  if (cudaGetLastError() != cudaSuccess) return cuda_fail("permutation kernels");

  // --- adjacency -> COO in CSR order ---
  int64_t nnz = 0;
  int64_t *coo_rows = nullptr, *coo_cols = nullptr;
  if (given_adj) {
    nnz = h_indptr[nf];
    const int64_t* indptr = S.upload(h_indptr.data(), nf + 1);
    const int64_t* indices = S.upload(d->adj_indices, nnz);
    coo_rows = S.alloc<int64_t>(nnz);
    coo_cols = S.alloc<int64_t>(nnz);
    if (!indptr || !indices || !coo_rows || !coo_cols) return cuda_fail("allocation / upload");
    cudaMemset(coo_rows, 0, (size_t)std::max<int64_t>(1, nnz) * sizeof(int64_t));  // entries before indptr[0]
    cudaMemset(coo_cols, 0, (size_t)std::max<int64_t>(1, nnz) * sizeof(int64_t));
    k_coo_from_csr<<<grid_for(nf), kT>>>(indptr, indices, nf, iperm, coo_rows, coo_cols, err);
  } else {
    const int64_t np = ne * (int64_t)k * k;
    uint64_t* keys[2] = {S.alloc<uint64_t>(np), S.alloc<uint64_t>(np)};
    int64_t* n_sel = S.alloc<int64_t>(1);
    if (!keys[0] || !keys[1] || !n_sel) return cuda_fail("allocation of the element pair keys");
    cudaMemset(n_sel, 0, sizeof(int64_t));
    k_pairs<<<grid_for(np), kT>>>(elems, ne, k, t2f_orig, nf, keys[0]);
    const uint64_t sentinel = (uint64_t)nf * (uint64_t)nf;
    const int end_bit = bit_width(sentinel);
    cub::DoubleBuffer<uint64_t> kb(keys[0], keys[1]);
    size_t sort_bytes = 0, uniq_bytes = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, sort_bytes, kb, np, 0, end_bit);
    cub::DeviceSelect::Unique(nullptr, uniq_bytes, keys[0], keys[1], n_sel, np);
    const size_t tmp_bytes = std::max(sort_bytes, uniq_bytes);
    void* tmp = S.alloc<char>((int64_t)tmp_bytes);
    if (!tmp) return cuda_fail("allocation of the sort scratch");
    size_t bytes = tmp_bytes;
    if (cub::DeviceRadixSort::SortKeys(tmp, bytes, kb, np, 0, end_bit) != cudaSuccess) return cuda_fail("pair sort");
    bytes = tmp_bytes;
    if (cub::DeviceSelect::Unique(tmp, bytes, kb.Current(), kb.Alternate(), n_sel, np) != cudaSuccess)
      return cuda_fail("unique");
    int64_t n_unique = 0;
    uint64_t last = 0;
    if (cudaMemcpy(&n_unique, n_sel, sizeof(int64_t), cudaMemcpyDeviceToHost) != cudaSuccess)
      return cuda_fail("count read");
    if (n_unique > 0 && cudaMemcpy(&last, kb.Alternate() + (n_unique - 1), sizeof(uint64_t),
                                   cudaMemcpyDeviceToHost) != cudaSuccess)
      return cuda_fail("count read");
    nnz = n_unique - ((n_unique > 0 && last == sentinel) ? 1 : 0);
    coo_rows = S.alloc<int64_t>(nnz);
    coo_cols = S.alloc<int64_t>(nnz);
    if (!coo_rows || !coo_cols) return cuda_fail("allocation of the COO arrays");
    k_coo_from_keys<<<grid_for(nnz), kT>>>(kb.Alternate(), nnz, nf, iperm, coo_rows, coo_cols);
  }
  if (cudaGetLastError() != cudaSuccess) return cuda_fail("COO kernels");

  // --- ownership, owned COO, element owners ---
  int64_t lo = 0, hi = 0;
  ownership_range(nf, d->comm_rank, d->comm_size, bs, &lo, &hi);
  int64_t *owned_rows = coo_rows, *owned_cols = coo_cols, nnz_owned = nnz;
  if (d->comm_size > 1) {
    char* flags = S.alloc<char>(nnz);
    int64_t* n_sel = S.alloc<int64_t>(1);
    owned_rows = S.alloc<int64_t>(nnz);
    owned_cols = S.alloc<int64_t>(nnz);
    if (!flags || !n_sel || !owned_rows || !owned_cols) return cuda_fail("allocation of the owned arrays");
    cudaMemset(n_sel, 0, sizeof(int64_t));
    k_owned_flags<<<grid_for(nnz), kT>>>(coo_rows, nnz, lo, hi, flags);
    size_t tmp_bytes = 0;
    cub::DeviceSelect::Flagged(nullptr, tmp_bytes, coo_rows, flags, owned_rows, n_sel, nnz);
    void* tmp = S.alloc<char>((int64_t)tmp_bytes);
    if (!tmp) return cuda_fail("allocation");
    size_t bytes = tmp_bytes;
    if (cub::DeviceSelect::Flagged(tmp, bytes, coo_rows, flags, owned_rows, n_sel, nnz) != cudaSuccess)
      return cuda_fail("owned selection");
    bytes = tmp_bytes;
    if (cub::DeviceSelect::Flagged(tmp, bytes, coo_cols, flags, owned_cols, n_sel, nnz) != cudaSuccess)
      return cuda_fail("owned selection");
    if (cudaMemcpy(&nnz_owned, n_sel, sizeof(int64_t), cudaMemcpyDeviceToHost) != cudaSuccess)
      return cuda_fail("count read");
  }
  k_elem_owner<<<grid_for(ne), kT>>>(elems, ne, k, t2f, nf, d->comm_size, bs, owner);
  int h_err = 0;
  if (cudaMemcpy(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return cuda_fail("kernels");
  if (h_err & 1) return set_error(FNE_EBOUNDS, "block_xyz: node id beyond coords");
  if (h_err & 2) return set_error(FNE_EBOUNDS, "adjacency column out of range");

  auto* L = new (std::nothrow) fne_layout();
  if (!L) return set_error(FNE_ENOMEM, "fne_layout_build_device: out of host memory");
  L->n_total = nt;
  L->n_free = nf;
  L->n_elem = ne;
  L->lo = lo;
  L->hi = hi;
  L->on_device = true;
  L->dev.nnz_total = nnz;
  L->dev.nnz_owned = nnz_owned;
  L->dev.perm = perm;
  L->dev.iperm = iperm;
  L->dev.t2f = t2f;
  L->dev.coo_rows = coo_rows;
  L->dev.coo_cols = coo_cols;
  L->dev.owned_rows = owned_rows;
  L->dev.owned_cols = owned_cols;
  L->dev.owned_is_coo = owned_rows == coo_rows;
  L->dev.elem_owner = owner;
  for (void* p : {(void*)perm, (void*)iperm, (void*)t2f, (void*)coo_rows, (void*)coo_cols, (void*)owned_rows,
                  (void*)owned_cols, (void*)owner})
    S.keep(p);
  *out = L;
  return FNE_OK;
}
