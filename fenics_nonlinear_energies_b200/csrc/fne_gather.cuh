// Node-block gather: sums stored element matrices / gradients into the owned
// COO values and the owned gradient (the reference's np.add.at scatter,
// src/core/petsc/reordered_element_base.py:1754-1756, regrouped by output).
//
// One warp per row node A; lane j of a round handles output block j of A
// (column node B): it adds the bs x bs block of every contributing element in
// element order and writes the block's rows -- consecutive lanes hold
// consecutive column blocks of the same rows, so the stores are coalesced.
// The gradient rows of A are summed over A's (element, local node)
// incidences with a fixed-order butterfly.  No atomics; bit-reproducible.
#pragma once

#include <cuda_runtime.h>

namespace fne {

struct NodeGatherArgs {
  int n_rnodes;
  const int* __restrict__ rn_blk;   // [n + 1]
  const int* __restrict__ rn_con;   // [n + 1]
  const int* __restrict__ rn_row;   // [n * bs]
  const int* __restrict__ rn_gpos;  // [n * bs]
  const int* __restrict__ rn_inc;   // [n + 1]
  const unsigned* __restrict__ blk;
  const int* __restrict__ con;
  const int* __restrict__ inc;
  const double* __restrict__ rhs;   // [n_owned] or null
};

// Element matrices: kbuf[el * NPAIR * BS * BS + pair(a, b) * BS * BS + c * BS + d]
// = K[(a, c), (b, d)] for a <= b (pair in row-major upper-triangle order);
// element gradients: gbuf[(el * NPN + a) * BS + c].  SLOTS: the contribution
// codes are slots of a buffer of oriented blocks (kbuf[slot * BS * BS + c * BS
// + d]), as written by the direct-write epilogue for shared blocks.
template <typename Real, typename HOut, int BS, int NPN, bool WANT_H, bool WANT_G, bool SLOTS = false>
__global__ void __launch_bounds__(256) k_node_gather(NodeGatherArgs G, const Real* __restrict__ kbuf,
                                                     const Real* __restrict__ gbuf, HOut* __restrict__ out,
                                                     double* __restrict__ grad) {
  constexpr int NPAIR = NPN * (NPN + 1) / 2, KS = NPAIR * BS * BS, NN = NPN * NPN;
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  for (int A = gw; A < G.n_rnodes; A += nw) {
    if (WANT_H) {
      int rowp[BS];
#pragma unroll
      for (int c = 0; c < BS; ++c) rowp[c] = __ldg(G.rn_row + A * BS + c);
      const int b0 = __ldg(G.rn_blk + A), b1 = __ldg(G.rn_blk + A + 1);
      int cbase = __ldg(G.rn_con + A);
      for (int base = b0; base < b1; base += 32) {
        const int b = base + lane;
        const unsigned w = b < b1 ? __ldg(G.blk + b) : 0u;
        const int cnt = (int)(w >> 19);
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int t = __shfl_up_sync(full, incl, o);
          if (lane >= o) incl += t;
        }
        const int start = cbase + incl - cnt;
        cbase += __shfl_sync(full, incl, 31);
        if (b < b1) {
          Real acc[BS][BS];
#pragma unroll
          for (int c = 0; c < BS; ++c)
#pragma unroll
            for (int d = 0; d < BS; ++d) acc[c][d] = Real(0);
          // U contributions per round: their code and value loads are independent
          constexpr int U = BS * BS * (int)sizeof(Real) <= 16 ? 4 : 2;
          int j = 0;
          for (; j + U <= cnt; j += U) {
            int code[U];
#pragma unroll
            for (int x = 0; x < U; ++x) code[x] = __ldg(G.con + start + j + x);
            Real v[U][BS * BS];
            bool tr[U];
#pragma unroll
            for (int x = 0; x < U; ++x) {
              const Real* s;
              if (SLOTS) {
                tr[x] = false;
                s = kbuf + (long long)code[x] * BS * BS;
              } else {
                const int el = code[x] / NN;
                const int r = code[x] - el * NN;
                const int a = r / NPN, bb = r - a * NPN;
                tr[x] = a > bb;
                const int lo = tr[x] ? bb : a, hi = tr[x] ? a : bb;
                s = kbuf + (long long)el * KS + (lo * NPN - lo * (lo - 1) / 2 + (hi - lo)) * BS * BS;
              }
#pragma unroll
              for (int i = 0; i < BS * BS; ++i) v[x][i] = s[i];
            }
#pragma unroll
            for (int x = 0; x < U; ++x)
#pragma unroll
              for (int c = 0; c < BS; ++c)
#pragma unroll
                for (int d = 0; d < BS; ++d) acc[c][d] += tr[x] ? v[x][d * BS + c] : v[x][c * BS + d];
          }
          for (; j < cnt; ++j) {
            const int code = __ldg(G.con + start + j);
            bool tr = false;
            const Real* s;
            if (SLOTS) {
              s = kbuf + (long long)code * BS * BS;
            } else {
              const int el = code / NN;
              const int r = code - el * NN;
              const int a = r / NPN, bb = r - a * NPN;
              tr = a > bb;
              const int lo = tr ? bb : a, hi = tr ? a : bb;
              s = kbuf + (long long)el * KS + (lo * NPN - lo * (lo - 1) / 2 + (hi - lo)) * BS * BS;
            }
            Real v[BS * BS];
#pragma unroll
            for (int i = 0; i < BS * BS; ++i) v[i] = s[i];
#pragma unroll
            for (int c = 0; c < BS; ++c)
#pragma unroll
              for (int d = 0; d < BS; ++d) acc[c][d] += tr ? v[d * BS + c] : v[c * BS + d];
          }
          const int off = (int)(w & 0xFFFFu);
          const unsigned dm = (w >> 16) & 7u;
#pragma unroll
          for (int c = 0; c < BS; ++c) {
            if (rowp[c] < 0) continue;
            int k = 0;
#pragma unroll
            for (int d = 0; d < BS; ++d)
              if ((dm >> d) & 1u) out[rowp[c] + off + k++] = (HOut)acc[c][d];
          }
        }
      }
    }
    if (WANT_G) {
      const int i0 = __ldg(G.rn_inc + A), i1 = __ldg(G.rn_inc + A + 1);
      Real gs[BS];
#pragma unroll
      for (int c = 0; c < BS; ++c) gs[c] = Real(0);
      for (int i = i0 + lane; i < i1; i += 32) {
        const int code = __ldg(G.inc + i);
#pragma unroll
        for (int c = 0; c < BS; ++c) gs[c] += gbuf[(long long)code * BS + c];
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int c = 0; c < BS; ++c) gs[c] += __shfl_xor_sync(full, gs[c], o);
      if (lane < BS) {
        Real v = gs[0];
#pragma unroll
        for (int c = 1; c < BS; ++c)
          if (lane == c) v = gs[c];
        const int gp = __ldg(G.rn_gpos + A * BS + lane);
        if (gp >= 0) grad[gp] = (double)v - (G.rhs ? G.rhs[gp] : 0.0);
      }
    }
  }
}

// Shared-block fix-up for bs = 2 (direct-write epilogue): one thread per
// shared output block sums its contributions (slots of 4 values, element
// order) and writes the block's two rows.  slots == nullptr: the buffer is in
// fix-up order and the block's contributions are the consecutive slots
// desc.z .. desc.z + count - 1 (streamed); else they are the buffer slots
// slots[desc.z .. desc.z + count) (gathered).  SB: the buffer's value type
// (float: tensor-core path; double: FP64 DMMA path).
template <typename HOut, typename SB>
__global__ void __launch_bounds__(256) k_fixup2(int n_blk, const int4* __restrict__ desc,
                                                const int* __restrict__ slots, const SB* __restrict__ sbuf,
                                                HOut* __restrict__ out) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < n_blk; b += gridDim.x * blockDim.x) {
    const int4 ds = __ldg(desc + b);
    const int cnt = ds.w & 0xFFFF;
    const unsigned dm = (unsigned)(ds.w >> 16) & 3u;
    SB a00 = 0, a01 = 0, a10 = 0, a11 = 0;
    if (slots == nullptr) {
      if constexpr (sizeof(SB) == 4) {
        const float4* sb = reinterpret_cast<const float4*>(sbuf) + ds.z;
#pragma unroll 4
        for (int j = 0; j < cnt; ++j) {
          const float4 v = __ldg(sb + j);
          a00 += v.x; a01 += v.y; a10 += v.z; a11 += v.w;
        }
      } else {
        const double2* sb = reinterpret_cast<const double2*>(sbuf) + 2LL * ds.z;
#pragma unroll 2
        for (int j = 0; j < cnt; ++j) {
          const double2 u0 = __ldg(sb + 2 * j), w0 = __ldg(sb + 2 * j + 1);
          a00 += u0.x; a01 += u0.y; a10 += w0.x; a11 += w0.y;
        }
      }
    } else {
      // slot indices several at a time, so several buffer loads are in
      // flight; the sums keep element order
      const int* sl = slots + ds.z;
      int j = 0;
      if constexpr (sizeof(SB) == 4) {
        const float4* sb = reinterpret_cast<const float4*>(sbuf);
        for (; j + 4 <= cnt; j += 4) {
          const float4 v0 = __ldg(sb + __ldg(sl + j)), v1 = __ldg(sb + __ldg(sl + j + 1));
          const float4 v2 = __ldg(sb + __ldg(sl + j + 2)), v3 = __ldg(sb + __ldg(sl + j + 3));
          a00 += v0.x; a01 += v0.y; a10 += v0.z; a11 += v0.w;
          a00 += v1.x; a01 += v1.y; a10 += v1.z; a11 += v1.w;
          a00 += v2.x; a01 += v2.y; a10 += v2.z; a11 += v2.w;
          a00 += v3.x; a01 += v3.y; a10 += v3.z; a11 += v3.w;
        }
        for (; j < cnt; ++j) {
          const float4 v = __ldg(sb + __ldg(sl + j));
          a00 += v.x; a01 += v.y; a10 += v.z; a11 += v.w;
        }
      } else {
        const double2* sb = reinterpret_cast<const double2*>(sbuf);
        for (; j + 2 <= cnt; j += 2) {
          const long long p0 = 2LL * __ldg(sl + j), p1 = 2LL * __ldg(sl + j + 1);
          const double2 u0 = __ldg(sb + p0), w0 = __ldg(sb + p0 + 1);
          const double2 u1 = __ldg(sb + p1), w1 = __ldg(sb + p1 + 1);
          a00 += u0.x; a01 += u0.y; a10 += w0.x; a11 += w0.y;
          a00 += u1.x; a01 += u1.y; a10 += w1.x; a11 += w1.y;
        }
        for (; j < cnt; ++j) {
          const long long p0 = 2LL * __ldg(sl + j);
          const double2 u0 = __ldg(sb + p0), w0 = __ldg(sb + p0 + 1);
          a00 += u0.x; a01 += u0.y; a10 += w0.x; a11 += w0.y;
        }
      }
    }
    const SB r0[2] = {a00, a01}, r1[2] = {a10, a11};
    int k = 0;
#pragma unroll
    for (int d = 0; d < 2; ++d)
      if ((dm >> d) & 1u) {
        if (ds.x >= 0) out[ds.x + k] = (HOut)r0[d];
        if (ds.y >= 0) out[ds.y + k] = (HOut)r1[d];
        ++k;
      }
  }
}

// Gradient rows, one thread per row node: the node's element entries summed
// in element order, minus the load vector.
template <typename Real, int BS>
__global__ void __launch_bounds__(256) k_rowgrad(int n_rnodes, const int* __restrict__ rn_inc,
                                                 const int* __restrict__ inc, const int* __restrict__ rn_gpos,
                                                 const Real* __restrict__ gbuf, const double* __restrict__ rhs,
                                                 double* __restrict__ grad) {
  for (int A = blockIdx.x * blockDim.x + threadIdx.x; A < n_rnodes; A += gridDim.x * blockDim.x) {
    Real gs[BS];
#pragma unroll
    for (int c = 0; c < BS; ++c) gs[c] = Real(0);
    const int i1 = __ldg(rn_inc + A + 1);
    for (int i = __ldg(rn_inc + A); i < i1; ++i) {
      const long long code = __ldg(inc + i);
#pragma unroll
      for (int c = 0; c < BS; ++c) gs[c] += gbuf[code * BS + c];
    }
#pragma unroll
    for (int c = 0; c < BS; ++c) {
      const int gp = __ldg(rn_gpos + A * BS + c);
      if (gp >= 0) grad[gp] = (double)gs[c] - (rhs ? rhs[gp] : 0.0);
    }
  }
}

}  // namespace fne
