// Internal declarations shared by the host-side C++ files of libfne_asm.so.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/fne_asm.h"

// Result of fne_layout_build (host vectors) or fne_layout_build_device (the
// same arrays in device memory; the host vectors stay empty).
struct fne_layout {
  int64_t n_total = 0, n_free = 0, lo = 0, hi = 0, n_elem = 0;
  std::vector<int64_t> perm, iperm, t2f, coo_rows, coo_cols, owned_rows, owned_cols, elem_owner;
  bool on_device = false;
  struct {
    int64_t nnz_total = 0, nnz_owned = 0;
    int64_t *perm = nullptr, *iperm = nullptr, *t2f = nullptr, *coo_rows = nullptr, *coo_cols = nullptr,
            *owned_rows = nullptr, *owned_cols = nullptr, *elem_owner = nullptr;
    bool owned_is_coo = false;  // one rank: the owned arrays alias the COO arrays
  } dev;
};

namespace fne {

// Device layout arrays: D2H copy into caller buffers / release.
int layout_device_copy(const fne_layout* L, int64_t* perm, int64_t* iperm, int64_t* t2f, int64_t* coo_rows,
                       int64_t* coo_cols, int64_t* owned_rows, int64_t* owned_cols, int64_t* elem_owner);
void layout_device_release(fne_layout* L);
// Host-side argument checks shared by the host and device layout builds.
int layout_check_desc(const fne_layout_desc* d);

// Thread-local last-error message (fne_last_error()).
int set_error(int code, const std::string& msg);

void ownership_range(int64_t n, int rank, int size, int bs, int64_t* lo, int64_t* hi);
int64_t rank_of_dof(int64_t dof, int64_t n, int size, int bs);
void element_adjacency(int64_t n_total, int64_t n_free, const int64_t* freedofs, int64_t n_elem,
                       int ndof_e, const int64_t* elems, std::vector<int64_t>& indptr,
                       std::vector<int64_t>& indices);

// Sentinel column offset: the element node has no free DOF (Dirichlet column).
constexpr uint32_t kNoCol = 127u;
// Incidence word: bits 0-2 local node a, bit 3 energy flag, then 7-bit column
// offsets (DOF units, relative to the row start) of element nodes 0..npe-1.
constexpr int kOffShift = 4;
constexpr int kOffBits = 7;
constexpr uint32_t kEnergyFlag = 8u;

// Row-gather plan: the reference's element -> COO scatter map
// (_build_scatter_data) regrouped by output row.  Row k of the owned COO
// pattern owns positions [row_ptr[k], row_ptr[k+1]); its values are the sum,
// over the incidences of the row's node, of the element Hessian row.
struct RowPlan {
  int32_t n_rows = 0;                // owned rows (every owned DOF once)
  int32_t n_nodes = 0;               // owned row-nodes
  std::vector<int32_t> row_ptr;      // [n_rows+1] output positions
  std::vector<int32_t> row_node;     // [n_rows] index into inc_ptr
  std::vector<uint8_t> row_comp;     // [n_rows] component of the row's DOF
  std::vector<int32_t> row_gpos;     // [n_rows] reordered id - lo (gradient slot)
  std::vector<int32_t> inc_ptr;      // [n_nodes+1]
  std::vector<int32_t> inc_elem;     // [n_inc] local element index
  std::vector<uint32_t> inc_info;    // [n_inc] packed (a, flag, offsets)
  std::vector<int64_t> local_elems;  // local element -> global element id
  std::vector<int32_t> elem_code;    // [n_local * npe] node gather code
  std::vector<uint8_t> elem_weight;  // [n_local] 0/1 energy weight
  std::vector<int64_t> dir_only;     // elements without any free DOF
  std::vector<int32_t> dir_only_code;
  int32_t max_row_len = 0;
};

// Builds the plan for node-uniform problems (every node has all or none of
// its block_size DOFs free).  Returns FNE_OK or an error (set_error called).
int build_row_plan(const fne_desc* d, RowPlan& P);

// Incidence-parallel plan (scalar P1 triangles): one thread per
// (row, element) incidence.  CTA c owns rows [cta_row[c], cta_row[c+1]) and
// their incidences [cta_inc[c], cta_inc[c+1]) (at most `threads` of them).
// inc_word: bits 0-1 local node a, bit 2 energy flag, bits 3-6 rank of the
// incidence within its row, then 7-bit column offsets of element nodes 0..2
// (127 = Dirichlet column).  inc_rowl: row index within the CTA.
struct IncPlan {
  int32_t n_cta = 0;
  int32_t max_rank = 0;       // largest rank (incidences per row - 1)
  int32_t max_rows = 0;       // most rows of one CTA
  int32_t max_len = 0;        // largest output slice of one CTA
  std::vector<int32_t> cta_row, cta_inc;
  std::vector<int32_t> inc_elem;
  std::vector<uint32_t> inc_word;
  std::vector<uint16_t> inc_rowl;
};

// Sorts P's local elements by the first row that needs them (locality),
// permuting the element arrays and P.inc_elem, and builds Q.  Returns false
// when the mesh does not fit the packed format.
bool build_inc_plan(RowPlan& P, int threads, IncPlan& Q);

// Banded-sweep plan (scalar P1 triangles).  Elements are sorted by the
// first output row f(e) that needs them.  CTA s sweeps the row segment
// [seg_row[s], seg_row[s+1]): it evaluates the elements [seg_elem[3s],
// seg_elem[3s+2]) in batches of `nb` (the first ones, below seg_elem[3s+1],
// only feed rows of the segment; the energy is counted for
// [seg_elem[3s+1], seg_elem[3s+2])).  After batch b every row below
// batch_done[b] is final and is streamed out of the shared-memory ring
// window.  Batch b's row entries ent_ptr[b]..: ent_row = row, ent_meta = first
// incidence (relative to inc_base[b], bits 0-15) | count << 16; incidence
// word: bits 0-8 batch-local element (nb <= 512), 9-10 local node a, then
// 7-bit column offsets of element nodes 0..2 from bit 11 (127 = Dirichlet).
struct SweepPlan {
  int32_t nb = 0;                       // elements per batch (= threads)
  int32_t n_seg = 0;
  int32_t win_entries = 0;              // ring window size (power of two)
  int32_t win_rows = 0;                 // ring window for gradient rows (power of two)
  std::vector<int32_t> seg_row;         // [n_seg+1]
  std::vector<int32_t> seg_elem;        // [3*n_seg] (pre start, own start, own end)
  std::vector<int32_t> seg_batch;       // [n_seg+1]
  std::vector<int32_t> batch_done;      // [n_batch]
  std::vector<int32_t> ent_ptr;         // [n_batch+1]
  std::vector<int32_t> inc_base;        // [n_batch]
  std::vector<int32_t> ent_row;         // [n_ent]
  std::vector<int32_t> ent_pos;         // [n_ent] COO position of the row's first entry
  std::vector<uint32_t> ent_meta;       // [n_ent]
  bool gpos_identity = false;           // gradient slot of row k is k
  std::vector<uint32_t> inc_word;       // [n_inc_sweep]
};

// Sorts P's local elements by first row (permuting element arrays and
// P.inc_elem) and builds Q with n_seg segments.  Returns false when the mesh
// does not fit (window larger than max_win_entries, rows longer than 126...).
bool build_sweep_plan(RowPlan& P, int nb, int n_seg, int max_win_entries, int max_win_rows, SweepPlan& Q);

// Row-cluster plan (scalar P1 triangles).  The owned rows are split into
// compact clusters (graph-grown over the element graph); CTA c evaluates
// every element that touches cluster c's rows (the cluster's "jobs"; an
// element on a cluster border is a job of each neighbouring cluster) into
// shared memory, then one thread per row sums, in a fixed order, the
// contributions its incidence list names into the row's slots of a
// shared-memory window, which is streamed out run by run: deterministic, no
// atomics, every COO value and gradient entry written to HBM once.
//   cluster table, 8 ints per cluster: {first job, end of the
//     energy-counting jobs, end of the jobs (padded to a multiple of 4),
//     first row, end of the rows, first incidence, end of the incidences
//     (padded to a multiple of 4), first run}; the first job and first
//     incidence are multiples of 4; the run range ends where the next
//     cluster's begins (run_end of the last cluster = number of runs);
//   job j: the local element job_elem[j] (-1 = padding job);
//   row i: {gradient slot, window offset, row length | incidences << 16,
//     first incidence relative to the cluster's first};
//   run: {window offset, first COO position, values, 0} -- consecutive rows
//     whose COO ranges are adjacent;
//   incidence word: bits 0-10 the job's index inside the cluster, bits 11-12
//     the row's node a in that element, bits 13-24 the 4-bit column offsets
//     (inside the row) of element nodes 0..2 (15 = no column).
struct ClusterPlan {
  int32_t n_cl = 0;
  int32_t max_jobs = 0;              // most jobs of one cluster (padded)
  int32_t max_rows = 0;              // most rows of one cluster
  int32_t max_incs = 0;              // most incidences of one cluster (padded)
  int32_t max_win = 0;               // most COO values of one cluster
  int32_t max_runs = 0;              // most runs of one cluster
  std::vector<int32_t> table;        // [(n_cl + 1) * 8]; the extra entry closes the run ranges
  std::vector<int32_t> job_elem;     // [n_jobs]
  std::vector<int32_t> rows;         // [n_rows_total * 4]
  std::vector<int32_t> runs;         // [n_runs * 4]
  std::vector<uint32_t> incs;        // [n_incs_total]
};
constexpr int kClJobBits = 11;
constexpr uint32_t kClNoCol = 15u;

// Builds Q from P (P is not modified); a cluster stops growing at max_rows
// rows, max_jobs jobs or max_incs incidences (both counted padded) or
// max_win COO values.  Returns false when the mesh does not fit the packed
// format (a row longer than 14 entries, a row alone beyond a budget).
bool build_cluster_plan(const RowPlan& P, int64_t lo, int64_t hi, int max_rows, int max_jobs, int max_incs,
                        int max_win, bool gpos_identity, ClusterPlan& Q);

// Node-block gather plan: the element matrices (stored per element as node
// pairs a <= b of bs x bs blocks) are summed per output block (row node A,
// column node B) -- the bs x bs values of rows (A, c) at columns (B, d).
// Row node k owns blocks [rn_blk[k], rn_blk[k+1]) in the order of their
// columns inside its rows, and contributions [rn_con[k], rn_con[k+1]).
// blk word: bits 0-15 column offset of node B's first free column inside the
// rows of A, bits 16-18 mask of B's free components, bits 19-31 number of
// contributions.  con: el * npn^2 + a * npn + b (local element el, local
// nodes a of A and b of B), element order within a block.  rn_row / rn_gpos:
// COO start position / gradient slot of row (A, c), -1 when that DOF is not
// an owned free row.  inc: el * npn + a per (row node, element) incidence.
struct BlockPlan {
  int32_t n_rnodes = 0;
  std::vector<int32_t> rn_blk, rn_con, rn_row, rn_gpos, rn_inc;
  std::vector<uint32_t> blk;
  std::vector<int32_t> con, inc;
  std::vector<int32_t> elem_rn;  // [n_local * npn] row node of each element node, -1 if none
};

// Direct-write plan for kernels that hold whole element matrices: for every
// element and directed node pair (a -> b) a 16-bit code: 0xFFFF = no output
// (row or column node without an owned free DOF); bit 15 set = the output
// block (node(a), node(b)) has several contributing elements, bits 0-14 =
// this element's slot among its shared blocks (its values go to the shared
// buffer at position sbase[e] + slot, or sidx[sbase[e] + slot] when the
// buffer is in fix-up order, bs * bs values row-major (c, d));
// else bits 0-11 = column offset of node(b) inside the rows of node(a), bits
// 12-14 = mask of node(b)'s free components (the element writes the block
// straight into the COO rows).  fix: node-block plan over the shared blocks
// only, whose contribution codes are element slots (sbase[e] + slot, element
// order per block).
struct DirectPlan {
  std::vector<uint16_t> code;   // [n_local * npn * npn]
  std::vector<int32_t> sbase;   // [n_local]
  int64_t n_slots = 0;
  BlockPlan fix;
  // flat fix-up (bs = 2): per shared block 4 ints: COO position of its first
  // column in row (A, 0) and in row (A, 1) (-1 if absent), its first entry
  // in fix.con (= its first buffer position in fix-up order), and
  // count | component mask << 16
  std::vector<int32_t> fdesc;
  // buffer position of every element slot for a buffer laid out in fix-up
  // order (sidx[fix.con[j]] = j): the contributions of one shared block then
  // sit at consecutive positions, in element order
  std::vector<int32_t> sidx;
};
int build_direct_plan(const BlockPlan& bp, int64_t n_local, int npn, int bs, DirectPlan& D);

// elem_dofs: [n_local * npn * bs] total DOFs (dof = bs * node + component) of
// the local elements in kernel order.  Returns FNE_OK, or FNE_ELAYOUT /
// FNE_EBOUNDS (set_error called) when the COO pattern is not node-blocked or
// exceeds the packed format.
int build_block_plan(int64_t n_local, int npn, int bs, const int64_t* elem_dofs, const fne_desc* d, BlockPlan& P);

// Mohr-Coulomb (plane strain, Pk triangles) handle, csrc/fne_mc.cu.
struct McHandle;
int mc_create(const fne_desc* d, McHandle** out);
int mc_eval(McHandle* h, const double* u, int flags, double* energy, double* grad, void* hess, void* stream);
int mc_set_dirichlet(McHandle* h, const double* dirichlet);
void mc_info(const McHandle* h, fne_info* info);
int mc_check_status(McHandle* h);
int mc_poll_status(McHandle* h);
int mc_set_wait_limit(McHandle* h, long long polls);
int mc_hvp_prepare(McHandle* h, const double* u, void* stream);
int mc_hvp(McHandle* h, const double* x, double* y, void* stream);
int mc_hvp_diagonal(McHandle* h, double* diag, void* stream);
void mc_destroy(McHandle* h);

// 3-D Mohr-Coulomb (P1 / P2 tetrahedra) handle, csrc/fne_mc3d.cu.
struct Mc3dHandle;
int mc3d_create(const fne_desc* d, Mc3dHandle** out);
int mc3d_eval(Mc3dHandle* h, const double* u, int flags, double* energy, double* grad, void* hess, void* stream);
int mc3d_set_dirichlet(Mc3dHandle* h, const double* dirichlet);
void mc3d_info(const Mc3dHandle* h, fne_info* info);
void mc3d_destroy(Mc3dHandle* h);

// Gather code of one element node: >= 0 reordered id of component 0 (free
// node); < 0: -1 - total DOF of component 0 (Dirichlet node).
}  // namespace fne
