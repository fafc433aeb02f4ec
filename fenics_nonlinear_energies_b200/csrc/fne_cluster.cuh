// Row-cluster kernel for P1 triangles (p-Laplace, Ginzburg-Landau): a fused
// energy / gradient / Hessian pass selected with kernel_variant 8 (the banded
// sweep stays the default: on the 1024^2 grid this kernel measured 149 us per
// FP64 pass against the sweep's 134 us, bound by its ~800 instructions per
// element).  Included by fne_asm.cu
// after the element physics (tri_full, tri_energy_r) and the FP64 energy
// reduction.
//
// A persistent CTA (one per SM, 512 threads) walks its share of the row
// clusters (ClusterPlan, fne_internal.h) through a two-deep software
// pipeline of shared-memory staging buffers:
//   - one thread issues TMA bulk copies (cp.async.bulk, completion counted on
//     mbarriers; no tensor map, no multicast, this GPU's memory only) of a
//     cluster's contiguous ranges: the jobs' gather codes (one barrier), then
//     their geometry, the row and run records and the incidence words (a
//     second barrier), two clusters ahead of the one being computed;
//   - once cluster i+1's codes are in, every thread starts asynchronous
//     8-byte copies (cp.async) of the nodal values its jobs need, so that
//     gather runs while cluster i is computed;
//   - cluster i: every job evaluated once, barrier-free (its gradient
//     replaces its nodal values, the upper triangle of its Hessian its
//     geometry); then one thread per row sums the row's incidence list, in
//     its fixed order, into the row's slots of a shared-memory window (no
//     atomics, bit-reproducible) and writes the gradient entry; the window is
//     streamed out run by run (consecutive rows with adjacent COO ranges),
//     coalesced.
// Each output value is written to HBM once; each element is read once per
// cluster it touches (about 1.1x on the 1024^2 grid).  Every wait on an
// mbarrier is bounded: a CTA that gives up sets the status word, waits once
// more (bounded) for the copies it issued, contributes a NaN energy partial
// and stops writing.
//
// Job records are structure-of-arrays over the job index j (array stride
// n_jobs): int32 code[3][n_jobs] (reordered free index, or -1 - total DOF
// for a Dirichlet node) and Real geo[7][n_jobs] = vol, dvx0..2, dvy0..2 --
// 68 B per job in FP64, 40 B in FP32; row records int4 {gradient slot,
// window offset, length | incidences << 16, first incidence}; run records
// and incidence words as in ClusterPlan.  A cluster's job and incidence
// ranges start at multiples of 4 and are padded to them, so every bulk copy
// starts on a 16-byte boundary and moves a multiple of 16 bytes.

constexpr int kClThreads = 512;
constexpr long long kClWaitLimit = 1LL << 22;

struct ClusterArgs {
  const int4* __restrict__ table;    // [n_cl + 1][2] cluster table (ClusterPlan)
  const int* __restrict__ codes;     // [3][n_jobs]
  const void* __restrict__ reals;    // [7][n_jobs] geometry (Real)
  const int4* __restrict__ rows;     // row records
  const int4* __restrict__ runs;     // run records
  const unsigned* __restrict__ incs; // incidence words
  int* err;                          // status word (1 = a copy wait gave up)
  long long wait_limit;              // polls of each mbarrier wait
  int n_jobs;                        // array stride of the job records
  int cap_j, cap_r, cap_u, cap_i;    // staging capacities (jobs and incidences multiples of 4)
  int cap_w;                         // window slots
};

// Shared-memory layout: two staging buffers of {int code[3][cap_j],
// Real geo[7][cap_j], double v[3][cap_j], int4 rows[cap_r], int4
// runs[cap_u], uint32 incs[cap_i]}, then Real win[cap_w] (16-byte aligned
// when cap_j and cap_i are multiples of 4).
template <typename Real>
struct ClLayout {
  int cj, cr, cu, ci, cw;
  __host__ __device__ size_t geo_off() const { return (size_t)cj * 12; }
  __host__ __device__ size_t v_off() const { return geo_off() + (size_t)cj * 7 * sizeof(Real); }
  __host__ __device__ size_t rows_off() const { return v_off() + (size_t)cj * 24; }
  __host__ __device__ size_t runs_off() const { return rows_off() + (size_t)cr * 16; }
  __host__ __device__ size_t inc_off() const { return runs_off() + (size_t)cu * 16; }
  __host__ __device__ size_t buf_bytes() const { return inc_off() + (size_t)ci * 4; }
  __host__ __device__ size_t win_off() const { return 2 * buf_bytes(); }
  __host__ __device__ size_t bytes() const { return win_off() + (size_t)cw * sizeof(Real); }
};

namespace clk {

__device__ __forceinline__ uint32_t saddr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void bar_init(uint32_t bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void bar_expect(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// 1-D bulk copy global -> this CTA's shared memory (no tensor map, no multicast)
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
// bounded wait for the phase of the given parity; false when it gave up
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity, long long limit) {
  for (long long it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
// order this thread's generic-proxy shared-memory accesses before later
// async-proxy (bulk copy) writes to the same bytes
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// 8-byte asynchronous global -> shared copy (cp.async, L1-allocating)
__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

}  // namespace clk

// One cluster's ranges from the cluster table.
struct ClRange {
  int j0, n_energy, nj, r0, nr, i0, ni, u0, nu;
};
__device__ __forceinline__ ClRange cl_range(const int4* __restrict__ table, int c) {
  const int4 t0 = __ldg(table + 2 * c), t1 = __ldg(table + 2 * c + 1), t2 = __ldg(table + 2 * c + 3);
  return ClRange{t0.x, t0.y - t0.x, t0.z - t0.x, t0.w, t1.x - t0.w, t1.y, t1.z - t1.y, t1.w, t2.w - t1.w};
}

// Issued by one thread: the bulk copies of cluster c into staging buffer sb.
template <typename Real>
__device__ __forceinline__ void cl_issue(const ClusterArgs& C, const ClLayout<Real>& L, unsigned char* sb, int c,
                                         uint32_t bar_codes, uint32_t bar_rest) {
  const ClRange R = cl_range(C.table, c);
  const uint32_t ib = (uint32_t)R.nj * 4u, rb = (uint32_t)R.nj * (uint32_t)sizeof(Real);
  const Real* reals = static_cast<const Real*>(C.reals);
  clk::bar_expect(bar_codes, 3u * ib);
  if (R.nj > 0)
    for (int k = 0; k < 3; ++k)
      clk::bulk_g2s(clk::saddr(sb + (size_t)k * L.cj * 4), C.codes + (size_t)k * C.n_jobs + R.j0, ib, bar_codes);
  clk::bar_expect(bar_rest, 7u * rb + (uint32_t)(R.nr + R.nu) * 16u + (uint32_t)R.ni * 4u);
  if (R.nj > 0)
    for (int k = 0; k < 7; ++k)
      clk::bulk_g2s(clk::saddr(sb + L.geo_off() + (size_t)k * L.cj * sizeof(Real)), reals + (size_t)k * C.n_jobs + R.j0,
                    rb, bar_rest);
  if (R.nr > 0) clk::bulk_g2s(clk::saddr(sb + L.rows_off()), C.rows + R.r0, (uint32_t)R.nr * 16u, bar_rest);
  if (R.nu > 0) clk::bulk_g2s(clk::saddr(sb + L.runs_off()), C.runs + R.u0, (uint32_t)R.nu * 16u, bar_rest);
  if (R.ni > 0) clk::bulk_g2s(clk::saddr(sb + L.inc_off()), C.incs + R.i0, (uint32_t)R.ni * 4u, bar_rest);
}

// Every thread: asynchronous copies of the nodal values of buffer sb's jobs.
template <typename Real>
__device__ __forceinline__ void cl_gather(const RowArgs& A, const ClLayout<Real>& L, unsigned char* sb, int nj) {
  const int* code = reinterpret_cast<const int*>(sb);
  const uint32_t v = clk::saddr(sb + L.v_off());
  for (int jl = threadIdx.x; jl < nj; jl += kClThreads)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int cd = code[k * L.cj + jl];
      const double* src = cd >= 0 ? A.u + cd : A.dir + (-1 - cd);
      clk::cp_async8(v + (uint32_t)((k * L.cj + jl) * 8), src);
    }
  clk::cp_async_commit();
}

template <typename Real, int FAM, int WANT, typename HOut>
__global__ void __launch_bounds__(kClThreads, 1) k_cluster_tri(RowArgs A, ClusterArgs C, Phys P,
                                                              double* __restrict__ grad, HOut* __restrict__ hess,
                                                              EnergyOut eo, int n_cl) {
  const ClLayout<Real> L{C.cap_j, C.cap_r, C.cap_u, C.cap_i, C.cap_w};
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Real* win = reinterpret_cast<Real*>(smem_raw + L.win_off());
  __shared__ __align__(8) unsigned long long s_bar[4];  // {codes, rest} per staging buffer
  __shared__ int s_ok, s_last;
  __shared__ double s_ws[32];
  const int tid = threadIdx.x;
  const int G = gridDim.x;
  const int n_mine = n_cl > (int)blockIdx.x ? (n_cl - 1 - (int)blockIdx.x) / G + 1 : 0;
  auto cluster = [&](int i) { return (int)blockIdx.x + i * G; };
  auto buf = [&](int i) { return smem_raw + (size_t)(i & 1) * L.buf_bytes(); };
  auto bar = [&](int i, int k) { return clk::saddr(&s_bar[2 * (i & 1) + k]); };
  auto parity = [&](int i) { return (uint32_t)((i >> 1) & 1); };

  if (tid == 0) {
    for (int k = 0; k < 4; ++k) clk::bar_init(clk::saddr(&s_bar[k]));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int i = 0; i < 2 && i < n_mine; ++i) cl_issue<Real>(C, L, buf(i), cluster(i), bar(i, 0), bar(i, 1));
    s_ok = n_mine == 0 || clk::bar_wait(bar(0, 0), 0, C.wait_limit);
  }
  __syncthreads();
  bool ok = s_ok != 0;
  if (ok && n_mine > 0) cl_gather<Real>(A, L, buf(0), cl_range(C.table, cluster(0)).nj);
  double eacc = 0.0;
  int i = 0;
  for (; ok && i < n_mine; ++i) {
    unsigned char* sb = buf(i);
    const ClRange R = cl_range(C.table, cluster(i));
    int* s_code = reinterpret_cast<int*>(sb);
    Real* s_geo = reinterpret_cast<Real*>(sb + L.geo_off());
    double* s_v = reinterpret_cast<double*>(sb + L.v_off());
    const int4* s_rows = reinterpret_cast<const int4*>(sb + L.rows_off());
    const int4* s_runs = reinterpret_cast<const int4*>(sb + L.runs_off());
    const unsigned* s_inc = reinterpret_cast<const unsigned*>(sb + L.inc_off());
    (void)s_code;
    // this cluster's geometry / rows / incidences, and its gathered values
    if (tid == 0) s_ok = clk::bar_wait(bar(i, 1), parity(i), C.wait_limit);
    clk::cp_async_wait_all();
    __syncthreads();
    if (!s_ok) {
      ok = false;
      break;
    }
    // evaluate every job once
    const int cj = L.cj;
    for (int jl = tid; jl < R.nj; jl += kClThreads) {
      TriElem<Real> t;
      t.vol = s_geo[jl];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        t.dvx[k] = s_geo[(1 + k) * cj + jl];
        t.dvy[k] = s_geo[(4 + k) * cj + jl];
      }
      const Real v[3] = {(Real)s_v[jl], (Real)s_v[cj + jl], (Real)s_v[2 * cj + jl]};
      Real g[3], H[6];
      tri_full<Real, FAM>(P, v, t, g, H);
      if ((WANT & W_E) && jl < R.n_energy) eacc += tri_energy_r<Real, FAM>(P, v, t);
#pragma unroll
      for (int k = 0; k < 3; ++k) s_v[k * cj + jl] = (double)g[k];
#pragma unroll
      for (int k = 0; k < 6; ++k) s_geo[(1 + k) * cj + jl] = H[k];
    }
    if ((WANT & W_E) && A.rhs)  // load term -f.u of the cluster's rows
      for (int r = tid; r < R.nr; r += kClThreads) {
        const int gp = s_rows[r].x;
        eacc -= A.rhs[gp] * A.u[A.lo + gp];
      }
    // the next cluster's nodal values start arriving while this one finishes
    if (i + 1 < n_mine) {
      if (tid == 0) s_ok = clk::bar_wait(bar(i + 1, 0), parity(i + 1), C.wait_limit);
      __syncthreads();
      if (!s_ok) {
        ok = false;
        break;
      }
      cl_gather<Real>(A, L, buf(i + 1), cl_range(C.table, cluster(i + 1)).nj);
    } else {
      __syncthreads();
    }
    // one thread per row: the row's incidences, in order, into its window
    // slots; the gradient entry straight out
    for (int r = tid; r < R.nr; r += kClThreads) {
      const int4 Rw = s_rows[r];
      const int len = Rw.z & 0xffff, n_inc = Rw.z >> 16;
      Real* rw = win + Rw.y;
      if (WANT & W_H)
        for (int q = 0; q < len; ++q) rw[q] = Real(0);
      double gacc = 0.0;
      const unsigned* inc = s_inc + Rw.w;
      for (int k = 0; k < n_inc; ++k) {
        const unsigned w = inc[k];
        const int jl = (int)(w & ((1u << kClJobBits) - 1u));
        const int a = (int)((w >> kClJobBits) & 3u);
        if (WANT & W_G) gacc += s_v[a * cj + jl];
        if (WANT & W_H) {
#pragma unroll
          for (int b = 0; b < 3; ++b) {
            const unsigned off = (w >> (kClJobBits + 2 + 4 * b)) & 15u;
            if (off != kClNoCol) rw[off] += s_geo[(1 + sym_index(a, b)) * cj + jl];
          }
        }
      }
      if (WANT & W_G) grad[Rw.x] = gacc - (A.rhs ? A.rhs[Rw.x] : 0.0);
    }
    __syncthreads();
    // the window out, run by run (coalesced)
    if (WANT & W_H) {
      const int n_win = R.nr > 0 ? s_rows[R.nr - 1].y + (s_rows[R.nr - 1].z & 0xffff) : 0;
      int run = 0;
      for (int q = tid; q < n_win; q += kClThreads) {
        while (run + 1 < R.nu && s_runs[run + 1].x <= q) ++run;  // runs ascend; q grows per thread
        const int4 U = s_runs[run];
        hess[U.y + (q - U.x)] = (HOut)win[q];
      }
    }
    // staging buffer free again: cluster i + 2 goes into it
    clk::fence_proxy_async();
    __syncthreads();
    if (tid == 0 && i + 2 < n_mine) cl_issue<Real>(C, L, sb, cluster(i + 2), bar(i + 2, 0), bar(i + 2, 1));
  }
  if (!ok) {
    clk::cp_async_wait_all();
    if (tid == 0) {
      // let the copies this CTA issued land before its shared memory is released
      for (int k = i; k < i + 2 && k < n_mine; ++k) {
        clk::bar_wait(bar(k, 0), parity(k), kClWaitLimit);
        clk::bar_wait(bar(k, 1), parity(k), kClWaitLimit);
      }
      atomicExch(C.err, 1);
    }
    eacc = tid == 0 ? __longlong_as_double(0x7ff8000000000000LL) : 0.0;
  }
  __syncthreads();
  if (WANT & W_E) energy_finalize(eacc, eo);
}
