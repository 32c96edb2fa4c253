// SELL-C-sigma matrix view, the per-row product and the block reduction shared
// by the single-system Krylov kernels (k_krylov.cu) and the multi-system
// persistent kernels (k_batch.cu).
#pragma once
#include <cuda_runtime.h>

#include "pbgpu_internal.cuh"

namespace pbgpu {

constexpr int kBlock = 256;
// resident blocks per SM the direct SpMV kernels are compiled for
// (registers <= 65536 / (256 * blocks)): 5 (48 registers, 40 warps per SM:
// the SpMV is latency-bound and gains more from resident warps than from
// unrolling), 4 (64 registers) for kernels with three or more fused reductions
constexpr int kSpmvMinBlocks = 5;
constexpr int kSpmvMinBlocksWide = 4;
// the G = 4 row product (one group per iteration, no unrolling) fits in 40
// registers: 6 blocks, 48 warps per SM, to keep more gathers in flight.
// G = 8 names the same G = 4 layout walked two groups per iteration (all
// index and value loads of both groups issued before the first gather): half
// the dependent load round trips per 8-wide row.  Bounded to 5 blocks it
// compiles to 48 registers: measured on a 14.5 M DoF system, 0.494 ms per
// SpMV against 0.526 at 4 blocks (60 registers, fewer warps) and 0.552 at 6
// (40 registers: the compiler then issues the second group's loads after the
// first group's gathers, as the one-group loop does)
template <int G>
__host__ __device__ constexpr int spmv_min_blocks() {
  return G == 4 ? 6 : G == 8 ? 5 : kSpmvMinBlocks;
}

template <typename T>
struct SellT {
  const int64_t* slice_ptr;
  const int32_t* slice_w;
  const int32_t* scol;
  const T* sval;
  int64_t n_pad;
  int C;
  int G;  // columns per row stored contiguously: 1, 2 or 4
};

template <typename T>
struct V2 {};
template <>
struct V2<double> {
  using t = double2;
};
template <>
struct V2<float> {
  using t = float2;
};

// The last W mod 4 columns of a G = 4 row (G = 2: W mod 2), stored one per
// lane after the groups (a warp's loads of one tail column are contiguous):
// all index and value loads first, then the gathers, in column order.
template <typename T, int G>
__device__ __forceinline__ void sell_tail(const SellT<T>& A, int lane, const T* __restrict__ x, int W, int64_t sb,
                                          T& acc) {
  constexpr int kMaxTail = G - 1;
  const int Wg = W & ~(G - 1);
  const int nt = W - Wg;
  if (nt == 0) return;
  const int64_t tb = sb + (int64_t)Wg * A.C + lane;
  int32_t tc[kMaxTail];
  T tv[kMaxTail];
#pragma unroll
  for (int j = 0; j < kMaxTail; ++j)
    if (j < nt) {
      tc[j] = __ldcs(A.scol + tb + (int64_t)j * A.C);
      tv[j] = __ldcs(A.sval + tb + (int64_t)j * A.C);
    }
#pragma unroll
  for (int j = 0; j < kMaxTail; ++j)
    if (j < nt) acc += tv[j] * x[tc[j]];
}

// y_p = sum_j A(p, j) x_j for SELL row p, element j at sell_elem(): columns
// in groups of G (one vector load per group, a warp's loads of one group
// contiguous), then the tail columns of a slice whose width the assembly did
// not pad to a multiple of G.
// (W and sb: width and first element of the row's slice, lane: the row's
// position in it)
template <typename T, int G>
__device__ __forceinline__ T sell_row(const SellT<T>& A, int lane, const T* __restrict__ x, int W, int64_t sb) {
  T acc = 0;
  if constexpr (G == 1) {
    const int64_t base = sb + lane;
    const int64_t stride = A.C;
#pragma unroll 4
    for (int j = 0; j < W; ++j) {
      const int64_t k = base + j * stride;
      acc += __ldcs(A.sval + k) * x[__ldcs(A.scol + k)];
    }
    return acc;
  } else if constexpr (G == 2) {
    const int64_t base = sb + 2 * lane;
    const int64_t stride = 2 * (int64_t)A.C;
#pragma unroll 2
    for (int g = 0; g < (W >> 1); ++g) {
      const int64_t k = base + g * stride;
      const int2 c = __ldcs(reinterpret_cast<const int2*>(A.scol + k));
      const typename V2<T>::t v = __ldcs(reinterpret_cast<const typename V2<T>::t*>(A.sval + k));
      acc += v.x * x[c.x];
      acc += v.y * x[c.y];
    }
    sell_tail<T, 2>(A, lane, x, W, sb, acc);
  } else if constexpr (G == 8) {
    // the G = 4 layout, two groups per iteration
    const int64_t base = sb + 4 * lane;
    const int64_t stride = 4 * (int64_t)A.C;
    const int ng = W >> 2;
    int g = 0;
#pragma unroll 1
    for (; g + 1 < ng; g += 2) {
      const int64_t k0 = base + g * stride, k1 = k0 + stride;
      const int4 c0 = __ldcs(reinterpret_cast<const int4*>(A.scol + k0));
      const int4 c1 = __ldcs(reinterpret_cast<const int4*>(A.scol + k1));
      if constexpr (sizeof(T) == 8) {
        const double2 v00 = __ldcs(reinterpret_cast<const double2*>(A.sval + k0));
        const double2 v01 = __ldcs(reinterpret_cast<const double2*>(A.sval + k0 + 2));
        const double2 v10 = __ldcs(reinterpret_cast<const double2*>(A.sval + k1));
        const double2 v11 = __ldcs(reinterpret_cast<const double2*>(A.sval + k1 + 2));
        const T x0 = x[c0.x], x1 = x[c0.y], x2 = x[c0.z], x3 = x[c0.w];
        const T x4 = x[c1.x], x5 = x[c1.y], x6 = x[c1.z], x7 = x[c1.w];
        acc += v00.x * x0;
        acc += v00.y * x1;
        acc += v01.x * x2;
        acc += v01.y * x3;
        acc += v10.x * x4;
        acc += v10.y * x5;
        acc += v11.x * x6;
        acc += v11.y * x7;
      } else {
        const float4 v0 = __ldcs(reinterpret_cast<const float4*>(A.sval + k0));
        const float4 v1 = __ldcs(reinterpret_cast<const float4*>(A.sval + k1));
        const T x0 = x[c0.x], x1 = x[c0.y], x2 = x[c0.z], x3 = x[c0.w];
        const T x4 = x[c1.x], x5 = x[c1.y], x6 = x[c1.z], x7 = x[c1.w];
        acc += v0.x * x0;
        acc += v0.y * x1;
        acc += v0.z * x2;
        acc += v0.w * x3;
        acc += v1.x * x4;
        acc += v1.y * x5;
        acc += v1.z * x6;
        acc += v1.w * x7;
      }
    }
    if (g < ng) {
      const int64_t k = base + g * stride;
      const int4 c = __ldcs(reinterpret_cast<const int4*>(A.scol + k));
      if constexpr (sizeof(T) == 8) {
        const double2 v0 = __ldcs(reinterpret_cast<const double2*>(A.sval + k));
        const double2 v1 = __ldcs(reinterpret_cast<const double2*>(A.sval + k + 2));
        acc += v0.x * x[c.x];
        acc += v0.y * x[c.y];
        acc += v1.x * x[c.z];
        acc += v1.y * x[c.w];
      } else {
        const float4 v = __ldcs(reinterpret_cast<const float4*>(A.sval + k));
        acc += v.x * x[c.x];
        acc += v.y * x[c.y];
        acc += v.z * x[c.z];
        acc += v.w * x[c.w];
      }
    }
    sell_tail<T, 4>(A, lane, x, W, sb, acc);
  } else {
    const int64_t base = sb + 4 * lane;
    const int64_t stride = 4 * (int64_t)A.C;
#pragma unroll 1
    for (int g = 0; g < (W >> 2); ++g) {
      const int64_t k = base + g * stride;
      const int4 c = __ldcs(reinterpret_cast<const int4*>(A.scol + k));
      if constexpr (sizeof(T) == 8) {
        const double2 v0 = __ldcs(reinterpret_cast<const double2*>(A.sval + k));
        const double2 v1 = __ldcs(reinterpret_cast<const double2*>(A.sval + k + 2));
        acc += v0.x * x[c.x];
        acc += v0.y * x[c.y];
        acc += v1.x * x[c.z];
        acc += v1.y * x[c.w];
      } else {
        const float4 v = __ldcs(reinterpret_cast<const float4*>(A.sval + k));
        acc += v.x * x[c.x];
        acc += v.y * x[c.y];
        acc += v.z * x[c.z];
        acc += v.w * x[c.w];
      }
    }
    sell_tail<T, 4>(A, lane, x, W, sb, acc);
  }
  return acc;
}

template <typename T, int G>
__device__ __forceinline__ T sell_row(const SellT<T>& A, int64_t p, const T* __restrict__ x) {
  const int64_t s = A.C == 32 ? (p >> 5) : p / A.C;  // the default slice height needs no division
  return sell_row<T, G>(A, (int)(p - s * A.C), x, A.slice_w[s], A.slice_ptr[s]);
}

// fn(i, (A x)_i) for the rows of this thread (grid-stride loop).  (Loading
// the next row's slice metadata ahead of the current row measured slower for
// G = 4: it costs registers the gathers need.)
template <typename T, int G, typename Fn>
__device__ __forceinline__ void spmv_direct_rows(const SellT<T>& A, const T* __restrict__ x, Fn&& fn) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < A.n_pad; i += (int64_t)gridDim.x * blockDim.x)
    fn(i, sell_row<T, G>(A, i, x));
}

// Block-wide sum of K values; result valid in thread 0.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K]) {
  __shared__ double sh[K][kBlock / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double a = v[k];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if (lane == 0) sh[k][wid] = a;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double a = lane < kBlock / 32 ? sh[k][lane] : 0.0;
      for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
      v[k] = a;
    }
  }
  __syncthreads();
}

}  // namespace pbgpu
