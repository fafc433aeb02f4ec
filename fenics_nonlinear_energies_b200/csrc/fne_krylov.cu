// Jacobi-preconditioned conjugate gradients on the owned COO Hessian, kept on
// the device for the Newton driver's linear solve (the reference hands the
// assembled matrix to PETSc: core/petsc/scalar_problem_driver.py:154-226 and
// hyperelasticity/jax_petsc/solver.py:257-330 call ksp.setOperators,
// ksp.setTolerances(rtol, max_it), ksp.solve and ksp.getIterationNumber).
//
// One CG iteration is two kernels and no host round trip:
//   k_cg_spmv   p = z + beta p_old (lazily, row by row), Ap = A p and the
//               block partials of p.Ap; the last block to finish reduces the
//               partials in a fixed order and sets alpha = rz / p.Ap, or stops
//               the solve at non-positive curvature;
//   k_cg_update x += alpha p, r -= alpha Ap, z = D^-1 r and the partials of
//               r.z and r.r; the last block sets beta, rz and the convergence
//               flag ||r||^2 <= rtol^2 ||b||^2.
// Scalars live in a device CgState; kernels of an iteration after the stop
// return at once, so a CUDA graph of `chunk` iterations can run past the stop
// unchanged and the host reads the state once per graph launch.  p_old and
// p_new alternate between two buffers by the parity of the iteration count
// held in the state.  Reductions use a fixed launch shape and a fixed order:
// the result of a solve is reproducible bit for bit.
//
// The stopping rules are those of the scalar CG restated in oracle/krylov.py:
// stop at the first iterate with ||r|| <= rtol ||b||, at p.Ap <= 0 (the last
// iterate, or b itself when it happens at the first iteration), or after
// max_it iterations; a zero right-hand side returns x = 0 after 0 iterations.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <new>
#include <string>
#include <vector>

#include "fne_internal.h"

namespace fne {
namespace {

constexpr int kCgThreads = 256;

// Row batches per warp iteration of the SpMV for G lanes per row.
constexpr int spmv_unroll(int G) { return G <= 8 ? 4 : 2; }

struct CgState {
  double rz, alpha, beta, tol2;
  int32_t active, stage, neg_first, its, it, maxit;
  int32_t reason;     // 0 converged, 1 non-positive curvature, 2 iteration limit, 3 zero right-hand side
  uint32_t count[3];  // last-block counters of init, spmv, update
};

struct CgVecs {
  const int32_t* crow;
  const int32_t* col;
  const void* vals;
  const double* dinv;
  double* x;
  double* r;
  double* z;
  double* Ap;
  double* p0;
  double* p1;
  double* partial;  // [2 * grid]
  CgState* st;
  int32_t n;
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block sum of up to two values (fixed order); the result is valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double (&sm)[NV][kCgThreads / 32]) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    v[j] = warp_sum(v[j]);
    if (lane == 0) sm[j][w] = v[j];
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      double t = lane < kCgThreads / 32 ? sm[j][lane] : 0.0;
#pragma unroll
      for (int o = 4; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      v[j] = t;
    }
  }
}

// Writes this block's partials; returns true in every thread of the last
// block to finish, whose v[] then holds the grid totals (valid in thread 0).
template <int NV>
__device__ bool last_block_total(double (&v)[NV], double* partial, uint32_t* counter) {
  __shared__ double sm[NV][kCgThreads / 32];
  __shared__ bool last;
  block_sum<NV>(v, sm);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) partial[j * gridDim.x + blockIdx.x] = v[j];
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double t[NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    t[j] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += kCgThreads) t[j] += __ldcg(partial + j * gridDim.x + b);
  }
  __syncthreads();
  block_sum<NV>(t, sm);
#pragma unroll
  for (int j = 0; j < NV; ++j) v[j] = t[j];
  if (threadIdx.x == 0) *counter = 0u;
  return true;
}

__global__ void __launch_bounds__(kCgThreads) k_cg_init(CgVecs a, const double* __restrict__ b, double rtol,
                                                        int maxit) {
  double v[2] = {0.0, 0.0};
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
    const double bi = b[i];
    const double zi = a.dinv[i] * bi;
    a.r[i] = bi;
    a.z[i] = zi;
    a.x[i] = 0.0;
    a.p0[i] = 0.0;
    a.p1[i] = 0.0;
    v[0] += bi * zi;
    v[1] += bi * bi;
  }
  if (last_block_total<2>(v, a.partial, &a.st->count[0]) && threadIdx.x == 0) {
    CgState* s = a.st;
    s->rz = v[0];
    s->tol2 = (rtol * rtol) * v[1];
    s->alpha = 0.0;
    s->beta = 0.0;
    s->active = !(v[1] == 0.0);
    s->reason = s->active ? 2 : 3;
    s->stage = 0;
    s->neg_first = 0;
    s->its = 0;
    s->it = 0;
    s->maxit = maxit;
  }
}

// G lanes per row, U row batches per warp iteration (their index, column and
// gather loads are in flight together); VT the stored value type (FP32 values
// are widened on load).
template <int G, typename VT, int U>
__global__ void __launch_bounds__(kCgThreads) k_cg_spmv(CgVecs a) {
  CgState* s = a.st;
  if (!s->active || s->it >= s->maxit) return;
  const double beta = s->beta;
  const bool odd = ((s->it + 1) & 1) != 0;  // this iteration's index is it + 1
  double* __restrict__ pn = odd ? a.p1 : a.p0;
  const double* __restrict__ po = odd ? a.p0 : a.p1;
  const double* __restrict__ z = a.z;
  const VT* __restrict__ vals = static_cast<const VT*>(a.vals);
  // Rows are taken RPW * U at a time by each warp; the loop bound is the
  // same for all lanes of a warp, so the shuffles below see the full warp.
  constexpr int RPW = 32 / G;
  const int lane = threadIdx.x & 31, sub = lane % G, rsub = lane / G;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int n_warps = gridDim.x * (kCgThreads / 32);
  double v[1] = {0.0};
  for (int base = warp * RPW * U; base < a.n; base += n_warps * RPW * U) {
    int k0[U], k1[U];
    double zr[U], pr[U], sum[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int row = base + u * RPW + rsub;
      const bool valid = row < a.n;
      k0[u] = valid ? __ldg(a.crow + row) : 0;
      k1[u] = valid ? __ldg(a.crow + row + 1) : 0;
      zr[u] = valid && sub == 0 ? z[row] : 0.0;
      pr[u] = valid && sub == 0 ? po[row] : 0.0;
    }
    int c[U];
    double w[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = k0[u] + sub;
      const bool ok = k < k1[u];
      c[u] = ok ? __ldg(a.col + k) : -1;
      w[u] = ok ? (double)vals[k] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) sum[u] = c[u] >= 0 ? w[u] * (z[c[u]] + beta * po[c[u]]) : 0.0;
#pragma unroll
    for (int u = 0; u < U; ++u)
      for (int k = k0[u] + sub + G; k < k1[u]; k += G) {
        const int cc = __ldg(a.col + k);
        sum[u] += (double)vals[k] * (z[cc] + beta * po[cc]);
      }
#pragma unroll
    for (int u = 0; u < U; ++u) {
#pragma unroll
      for (int o = G / 2; o > 0; o >>= 1) sum[u] += __shfl_xor_sync(0xffffffffu, sum[u], o, G);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int row = base + u * RPW + rsub;
      if (row < a.n && sub == 0) {
        const double p = zr[u] + beta * pr[u];
        pn[row] = p;
        a.Ap[row] = sum[u];
        v[0] += p * sum[u];
      }
    }
  }
  if (last_block_total<1>(v, a.partial, &s->count[1]) && threadIdx.x == 0) {
    const double pAp = v[0];
    s->it += 1;
    s->its += 1;
    const bool curv = pAp > 0.0;
    if (s->it == 1) s->neg_first = !curv;
    if (curv) {
      s->alpha = s->rz / pAp;
      s->stage = 1;
    } else {
      s->alpha = 0.0;
      s->active = 0;
      s->stage = 0;
      s->reason = 1;
    }
  }
}

__device__ __forceinline__ void cg_update_one(double alpha, double& x, double p, double& r, double ap, double d,
                                              double& z, double (&v)[2]) {
  x += alpha * p;
  r -= alpha * ap;
  z = d * r;
  v[0] += r * z;
  v[1] += r * r;
}

// Vectors are padded to a multiple of 32 entries, so every vector starts on a
// 256-byte boundary and is read and written as double2 (two pairs in flight
// per thread); an odd last entry is done by thread 0.
__global__ void __launch_bounds__(kCgThreads) k_cg_update(CgVecs a) {
  CgState* s = a.st;
  if (s->stage != 1) return;
  const double alpha = s->alpha;
  const double2* __restrict__ p = reinterpret_cast<const double2*>((s->it & 1) ? a.p1 : a.p0);
  double2* __restrict__ x = reinterpret_cast<double2*>(a.x);
  double2* __restrict__ r = reinterpret_cast<double2*>(a.r);
  double2* __restrict__ z = reinterpret_cast<double2*>(a.z);
  const double2* __restrict__ ap = reinterpret_cast<const double2*>(a.Ap);
  const double2* __restrict__ dv = reinterpret_cast<const double2*>(a.dinv);
  double v[2] = {0.0, 0.0};
  const int n2 = a.n >> 1;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (int i = tid; i < n2; i += 2 * stride) {
    const int j = i + stride;
    const bool two = j < n2;
    double2 xa = x[i], pa = p[i], ra = r[i], aa = ap[i], da = dv[i], za;
    double2 xb, pb, rb, ab, db, zb;
    if (two) {
      xb = x[j];
      pb = p[j];
      rb = r[j];
      ab = ap[j];
      db = dv[j];
    }
    cg_update_one(alpha, xa.x, pa.x, ra.x, aa.x, da.x, za.x, v);
    cg_update_one(alpha, xa.y, pa.y, ra.y, aa.y, da.y, za.y, v);
    x[i] = xa;
    r[i] = ra;
    z[i] = za;
    if (two) {
      cg_update_one(alpha, xb.x, pb.x, rb.x, ab.x, db.x, zb.x, v);
      cg_update_one(alpha, xb.y, pb.y, rb.y, ab.y, db.y, zb.y, v);
      x[j] = xb;
      r[j] = rb;
      z[j] = zb;
    }
  }
  if ((a.n & 1) && tid == 0) {
    const int i = a.n - 1;
    const double* pp = reinterpret_cast<const double*>(p);
    cg_update_one(alpha, a.x[i], pp[i], a.r[i], a.Ap[i], a.dinv[i], a.z[i], v);
  }
  if (last_block_total<2>(v, a.partial, &s->count[2]) && threadIdx.x == 0) {
    s->beta = v[0] / s->rz;
    s->rz = v[0];
    s->active = !(v[1] <= s->tol2);
    if (!s->active) s->reason = 0;
    s->stage = 0;
  }
}

// CSR values in row order from the COO values, and the Jacobi scaling
// 1 / |a_ii| (1 where the diagonal is missing, zero or not a number).
template <typename VT>
__global__ void k_cg_values(int64_t nnz, int32_t n, const int32_t* __restrict__ order,
                            const int32_t* __restrict__ diag, const VT* __restrict__ coo, VT* __restrict__ vals,
                            double* __restrict__ dinv) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += stride) vals[k] = coo[order[k]];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int32_t d = diag[i];
    const double v = d >= 0 ? fabs((double)coo[d]) : 1.0;
    dinv[i] = 1.0 / (v > 0.0 ? v : 1.0);
  }
}

int cg_status(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(FNE_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return FNE_OK;
}

}  // namespace
}  // namespace fne

struct fne_cg {
  int32_t n = 0;
  int64_t nv = 0;  // vector stride: n rounded up to a multiple of 32
  int64_t nnz = 0;
  int group = 8;
  int vals_fp32 = 0;
  int chunk = 16;
  int grid_spmv = 1, grid_vec = 1;
  int32_t* crow = nullptr;
  int32_t* col = nullptr;
  int32_t* order = nullptr;
  int32_t* diag = nullptr;
  void* vals = nullptr;
  double* dinv = nullptr;
  double* work = nullptr;  // x, r, z, Ap, p0, p1
  double* partial = nullptr;
  fne::CgState* st = nullptr;
  fne::CgState* st_host = nullptr;
  cudaStream_t cap = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool have_matrix = false;
};

namespace {

using fne::set_error;

fne::CgVecs vecs_of(const fne_cg* c) {
  fne::CgVecs a;
  a.crow = c->crow;
  a.col = c->col;
  a.vals = c->vals;
  a.dinv = c->dinv;
  a.x = c->work;
  a.r = c->work + 1 * (size_t)c->nv;
  a.z = c->work + 2 * (size_t)c->nv;
  a.Ap = c->work + 3 * (size_t)c->nv;
  a.p0 = c->work + 4 * (size_t)c->nv;
  a.p1 = c->work + 5 * (size_t)c->nv;
  a.partial = c->partial;
  a.st = c->st;
  a.n = c->n;
  return a;
}

void launch_spmv(const fne_cg* c, cudaStream_t s) {
  const fne::CgVecs a = vecs_of(c);
  const dim3 g(c->grid_spmv), b(fne::kCgThreads);
#define FNE_CG_SPMV(G)                                                                        \
  if (c->group == G) {                                                                        \
    if (c->vals_fp32)                                                                         \
      fne::k_cg_spmv<G, float, fne::spmv_unroll(G)><<<g, b, 0, s>>>(a);                       \
    else                                                                                      \
      fne::k_cg_spmv<G, double, fne::spmv_unroll(G)><<<g, b, 0, s>>>(a);                      \
    return;                                                                                   \
  }
  FNE_CG_SPMV(4)
  FNE_CG_SPMV(8)
  FNE_CG_SPMV(16)
  FNE_CG_SPMV(32)
#undef FNE_CG_SPMV
}

int resident_spmv(int group, int fp32) {
  int r = 1;
#define FNE_CG_OCC(G)                                                                                   \
  if (group == G) {                                                                                     \
    if (fp32)                                                                                           \
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, fne::k_cg_spmv<G, float, fne::spmv_unroll(G)>,  \
                                                    fne::kCgThreads, 0);                                \
    else                                                                                                \
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, fne::k_cg_spmv<G, double, fne::spmv_unroll(G)>, \
                                                    fne::kCgThreads, 0);                                \
    return r;                                                                                           \
  }
  FNE_CG_OCC(4)
  FNE_CG_OCC(8)
  FNE_CG_OCC(16)
  FNE_CG_OCC(32)
#undef FNE_CG_OCC
  return r;
}

void cg_free(fne_cg* c) {
  if (!c) return;
  if (c->exec) cudaGraphExecDestroy(c->exec);
  if (c->cap) cudaStreamDestroy(c->cap);
  cudaFree(c->crow);
  cudaFree(c->col);
  cudaFree(c->order);
  cudaFree(c->diag);
  cudaFree(c->vals);
  cudaFree(c->dinv);
  cudaFree(c->work);
  cudaFree(c->partial);
  cudaFree(c->st);
  if (c->st_host) cudaFreeHost(c->st_host);
  delete c;
}

int build_graph(fne_cg* c) {
  cudaGraph_t graph = nullptr;
  if (cudaStreamBeginCapture(c->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return fne::cg_status("fne_cg_solve: begin capture");
  const fne::CgVecs a = vecs_of(c);
  for (int j = 0; j < c->chunk; ++j) {
    launch_spmv(c, c->cap);
    fne::k_cg_update<<<c->grid_vec, fne::kCgThreads, 0, c->cap>>>(a);
  }
  cudaError_t e = cudaStreamEndCapture(c->cap, &graph);
  if (e != cudaSuccess) return set_error(FNE_ECUDA, std::string("fne_cg_solve: capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&c->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    c->exec = nullptr;
    return set_error(FNE_ECUDA, std::string("fne_cg_solve: instantiate: ") + cudaGetErrorString(e));
  }
  return FNE_OK;
}

}  // namespace

extern "C" int fne_cg_create(int32_t n, int64_t nnz, const int64_t* rows, const int64_t* cols, int32_t vals_fp32,
                             int32_t chunk, fne_cg** out) {
  if (!out || n < 0 || nnz < 0 || (nnz > 0 && (!rows || !cols)) || nnz > INT32_MAX || chunk < 1 || chunk > 4096)
    return set_error(FNE_EINVAL, "fne_cg_create: bad arguments");
  *out = nullptr;
  std::vector<int32_t> crow((size_t)n + 1, 0), col((size_t)nnz), order((size_t)nnz), diag((size_t)n, -1);
  for (int64_t k = 0; k < nnz; ++k) {
    if (rows[k] < 0 || rows[k] >= n || cols[k] < 0 || cols[k] >= n)
      return set_error(FNE_EBOUNDS, "fne_cg_create: COO entry " + std::to_string(k) + " outside the n x n block");
    ++crow[(size_t)rows[k] + 1];
  }
  for (int32_t i = 0; i < n; ++i) crow[i + 1] += crow[i];
  std::vector<int32_t> fill(crow.begin(), crow.end() - 1);
  for (int64_t k = 0; k < nnz; ++k) {  // stable: COO order within a row
    const int32_t pos = fill[(size_t)rows[k]]++;
    order[pos] = (int32_t)k;
    col[pos] = (int32_t)cols[k];
    if (rows[k] == cols[k]) diag[(size_t)rows[k]] = (int32_t)k;
  }
  fne_cg* c = new (std::nothrow) fne_cg();
  if (!c) return set_error(FNE_EINVAL, "fne_cg_create: out of host memory");
  c->n = n;
  c->nv = ((int64_t)n + 31) / 32 * 32;
  c->nnz = nnz;
  c->vals_fp32 = vals_fp32 ? 1 : 0;
  c->chunk = chunk;
  const double avg = n > 0 ? (double)nnz / n : 0.0;
  c->group = avg <= 6.0 ? 4 : avg <= 12.0 ? 8 : avg <= 24.0 ? 16 : 32;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // One full wave: SMs x resident blocks of each kernel (grid-stride loops).
  const int per_sm_spmv = std::max(1, resident_spmv(c->group, c->vals_fp32));
  int per_sm_vec = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_vec, fne::k_cg_update, fne::kCgThreads, 0);
  per_sm_vec = std::max(1, per_sm_vec);
  const int64_t want_spmv = ((int64_t)n * c->group + fne::kCgThreads - 1) / fne::kCgThreads;
  const int64_t want_vec = ((int64_t)n + fne::kCgThreads - 1) / fne::kCgThreads;
  c->grid_spmv = (int)std::max<int64_t>(1, std::min<int64_t>(want_spmv, (int64_t)sms * per_sm_spmv));
  c->grid_vec = (int)std::max<int64_t>(1, std::min<int64_t>(want_vec, (int64_t)sms * per_sm_vec));
  const size_t vsz = c->vals_fp32 ? sizeof(float) : sizeof(double);
  const int gmax = std::max(c->grid_spmv, c->grid_vec);
  bool ok = cudaMalloc(&c->crow, crow.size() * sizeof(int32_t)) == cudaSuccess &&
            cudaMalloc(&c->col, std::max<size_t>(1, col.size()) * sizeof(int32_t)) == cudaSuccess &&
            cudaMalloc(&c->order, std::max<size_t>(1, order.size()) * sizeof(int32_t)) == cudaSuccess &&
            cudaMalloc(&c->diag, std::max<size_t>(1, diag.size()) * sizeof(int32_t)) == cudaSuccess &&
            cudaMalloc(&c->vals, std::max<size_t>(1, (size_t)nnz) * vsz) == cudaSuccess &&
            cudaMalloc(&c->dinv, std::max<size_t>(32, (size_t)c->nv) * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&c->work, std::max<size_t>(32, 6 * (size_t)c->nv) * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&c->partial, 2 * (size_t)gmax * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&c->st, sizeof(fne::CgState)) == cudaSuccess &&
            cudaHostAlloc(&c->st_host, sizeof(fne::CgState), cudaHostAllocDefault) == cudaSuccess &&
            cudaStreamCreateWithFlags(&c->cap, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && cudaMemcpy(c->crow, crow.data(), crow.size() * sizeof(int32_t), cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && (nnz == 0 || (cudaMemcpy(c->col, col.data(), col.size() * sizeof(int32_t), cudaMemcpyHostToDevice) ==
                               cudaSuccess &&
                           cudaMemcpy(c->order, order.data(), order.size() * sizeof(int32_t),
                                      cudaMemcpyHostToDevice) == cudaSuccess));
  ok = ok && (n == 0 || cudaMemcpy(c->diag, diag.data(), diag.size() * sizeof(int32_t), cudaMemcpyHostToDevice) ==
                            cudaSuccess);
  ok = ok && cudaMemset(c->st, 0, sizeof(fne::CgState)) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    cg_free(c);
    return set_error(FNE_ECUDA, "fne_cg_create: device allocation or copy failed");
  }
  *out = c;
  return FNE_OK;
}

extern "C" int fne_cg_set_matrix(fne_cg* c, const void* coo_vals, void* stream) {
  if (!c || (c->nnz > 0 && !coo_vals)) return set_error(FNE_EINVAL, "fne_cg_set_matrix: bad arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t work = std::max<int64_t>(c->nnz, c->n);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, 148 * 16));
  if (c->vals_fp32)
    fne::k_cg_values<float><<<grid, 256, 0, s>>>(c->nnz, c->n, c->order, c->diag, static_cast<const float*>(coo_vals),
                                                 static_cast<float*>(c->vals), c->dinv);
  else
    fne::k_cg_values<double><<<grid, 256, 0, s>>>(c->nnz, c->n, c->order, c->diag,
                                                  static_cast<const double*>(coo_vals), static_cast<double*>(c->vals),
                                                  c->dinv);
  const int rc = fne::cg_status("fne_cg_set_matrix");
  if (rc == FNE_OK) c->have_matrix = true;
  return rc;
}

extern "C" int fne_cg_solve(fne_cg* c, const double* b, double* x, double rtol, int32_t maxit, int32_t* its,
                            int32_t* reason, void* stream) {
  if (!c || (c->n > 0 && (!b || !x)) || maxit < 0 || !(rtol >= 0.0))
    return set_error(FNE_EINVAL, "fne_cg_solve: bad arguments");
  if (!c->have_matrix) return set_error(FNE_EINVAL, "fne_cg_solve: fne_cg_set_matrix was not called");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!c->exec) {
    const int rc = build_graph(c);
    if (rc != FNE_OK) return rc;
  }
  const fne::CgVecs a = vecs_of(c);
  fne::k_cg_init<<<c->grid_vec, fne::kCgThreads, 0, s>>>(a, b, rtol, maxit);
  int rc = fne::cg_status("fne_cg_solve: init");
  if (rc != FNE_OK) return rc;
  fne::CgState* h = c->st_host;
  for (;;) {
    if (cudaMemcpyAsync(h, c->st, sizeof(fne::CgState), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return fne::cg_status("fne_cg_solve: state read");
    if (!h->active || h->it >= h->maxit) break;
    if (cudaGraphLaunch(c->exec, s) != cudaSuccess) return fne::cg_status("fne_cg_solve: graph launch");
  }
  const double* src = h->neg_first ? b : a.x;
  if (c->n > 0 && cudaMemcpyAsync(x, src, (size_t)c->n * sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return fne::cg_status("fne_cg_solve: result copy");
  if (its) *its = h->neg_first ? 1 : h->its;
  if (reason) *reason = h->reason;
  return FNE_OK;
}

extern "C" int fne_cg_destroy(fne_cg* c) {
  cg_free(c);
  return FNE_OK;
}
