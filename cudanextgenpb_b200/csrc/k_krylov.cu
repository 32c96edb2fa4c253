// Krylov solve of the assembled SELL-C-sigma system: replaces LIS / MUMPS
// (lis_compute_electric_potential, src/pb_class.cpp:2244-2329;
// mumps_compute_electric_potential, :2200-2239).
//
// Design (B200, HBM-bound):
//  * SpMV: one thread per row, SELL slices of C rows; each row's columns are
//    stored in groups of G (1, 2 or 4) lane-interleaved, so a warp's loads of
//    one group are contiguous (G = 4: one 16-byte column load and two 16-byte
//    value loads per 4 nonzeros).  Rows are sorted by length inside windows of
//    sigma rows, which keeps padding near zero on these irregular meshes.
//    Matrix streams are loaded with the evict-first hint (__ldcs) so the
//    gathered vector stays resident in the 126 MB L2.
//  * For the C = 32, G = 1 layout the SpMV instead stages each warp's slices
//    through shared memory with bulk async copies (cp.async.bulk, mbarrier
//    completion, double-buffered), so the matrix stream never stalls a warp
//    and only the vector gathers remain on the critical path.
//  * Every dot product is fused into the kernel that produces its operands;
//    block partials are reduced by the last block to finish (ticket counter), in
//    fixed block order, so results are deterministic and the Krylov scalars
//    (alpha, beta, omega, convergence flag) never leave the device.
//  * Kernels return immediately once the device flag `done` is set, so the host
//    launches iterations in chunks (captured as a CUDA graph) and polls the flag
//    once per chunk.
//  * Mixed precision: FP32 matrix and vectors (FP32 SpMV accumulation) in the
//    inner solve; the outer residual b - A x, the refinement update and the
//    final residual are FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <type_traits>

#include "pbgpu_internal.cuh"
#include "sell.cuh"
#include "tma.cuh"

namespace pbgpu {

// ---------------------------------------------------------------------------
// SpMV with the matrix staged through shared memory by bulk async copies
// (G = 1, C = 32 layout).  Each warp owns a sequence of slices (grid stride);
// a slice is copied in chunks of up to NC columns (values and column ids,
// contiguous in the G = 1 layout), one chunk ahead of the one being multiplied,
// into two per-warp buffers completed through mbarriers.  The matrix stream is
// then fully asynchronous and each lane's x gathers (column ids read from
// shared memory) are all independent.  Copies carry an L2 evict-first hint so
// the gathered vector stays resident in L2.
constexpr int kTmaWarps = kBlock / 32;

template <typename T, int NC>
__host__ __device__ constexpr size_t tma_buf_bytes() {
  return (size_t)NC * 32 * (sizeof(T) + sizeof(int32_t));
}
template <typename T, int NC>
__host__ __device__ constexpr size_t tma_smem_bytes() {
  return (size_t)kTmaWarps * 2 * tma_buf_bytes<T, NC>() + (size_t)kTmaWarps * 2 * sizeof(uint64_t);
}

// Calls fn(row, y) for every row of every slice of this warp; false when a
// bounded wait (limit wait_ns) gave up (the warp's outstanding copies are then
// waited for, with the default limit, before it returns).
template <typename T, int NC, typename Fn>
__device__ __forceinline__ bool spmv_tma_rows(const SellT<T>& A, const T* __restrict__ x, Fn&& fn,
                                              uint64_t wait_ns) {
  extern __shared__ __align__(128) unsigned char tma_smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t nwarps = (int64_t)gridDim.x * kTmaWarps;
  const int64_t n_slices = A.n_pad / 32;
  unsigned char* base = tma_smem + (size_t)wib * 2 * tma_buf_bytes<T, NC>();
  // buffer b: values at base + b * buf, column ids right after them
  auto vbuf = [&](int b) { return reinterpret_cast<T*>(base + b * tma_buf_bytes<T, NC>()); };
  auto cbuf = [&](int b) {
    return reinterpret_cast<int32_t*>(base + b * tma_buf_bytes<T, NC>() + (size_t)NC * 32 * sizeof(T));
  };
  uint64_t* bars = reinterpret_cast<uint64_t*>(tma_smem + (size_t)kTmaWarps * 2 * tma_buf_bytes<T, NC>()) + 2 * wib;
  if (lane == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_fence_init();
  }
  __syncwarp();
  const uint64_t pol = l2_evict_first_policy();
  // copy columns [jj, jj + 16) of the slice at element offset ptr (width ww) into buffer b
  auto issue = [&](int64_t ptr, int jj, int ww, int b) {
    if (lane == 0) {
      const int nc = min(NC, ww - jj);
      const int64_t off = ptr + (int64_t)jj * 32;
      const uint32_t bv = (uint32_t)(nc * 32 * sizeof(T)), bc = (uint32_t)(nc * 32 * sizeof(int32_t));
      mbar_arrive_expect_tx(&bars[b], nc > 0 ? bv + bc : 0u);
      if (nc > 0) {
        bulk_g2s(vbuf(b), A.sval + off, bv, &bars[b], pol);
        bulk_g2s(cbuf(b), A.scol + off, bc, &bars[b], pol);
      }
    }
  };
  // current slice (s, W, P) and the warp's next slice (sn, Wn, Pn): the next
  // slice's width and offset are loaded one slice ahead, so issuing its copy
  // never waits on a global load
  int64_t s = (int64_t)blockIdx.x * kTmaWarps + wib;
  if (s >= n_slices) return true;
  int W = A.slice_w[s];
  int64_t P = A.slice_ptr[s];
  int64_t sn = s + nwarps;
  int Wn = sn < n_slices ? A.slice_w[sn] : 0;
  int64_t Pn = sn < n_slices ? A.slice_ptr[sn] : 0;
  int j0 = 0;
  uint32_t phases = 0;  // bit b: parity of buffer b's next completion
  int b = 0;
  issue(P, 0, W, 0);
  T acc = 0;
  while (true) {
    const bool more_cols = j0 + NC < W;
    const bool next = more_cols || sn < n_slices;
    if (more_cols)
      issue(P, j0 + NC, W, b ^ 1);
    else if (next)
      issue(Pn, 0, Wn, b ^ 1);
    // every lane observes the phase itself (acquiring the copied bytes); the
    // vote keeps the warp together should any lane reach the limit
    if (!__all_sync(0xffffffffu, mbar_wait_bounded(&bars[b], (phases >> b) & 1u, wait_ns))) {
      // give up: let this warp's copies land before the block can exit
      mbar_wait_bounded(&bars[b], (phases >> b) & 1u);
      if (next) mbar_wait_bounded(&bars[b ^ 1], (phases >> (b ^ 1)) & 1u);
      return false;
    }
    phases ^= 1u << b;
    const int nc = min(NC, W - j0);
    const T* vs = vbuf(b);
    const int32_t* cs = cbuf(b);
    // all gathers of the chunk are issued before the first use
    T xv[NC];
#pragma unroll
    for (int j = 0; j < NC; ++j) xv[j] = j < nc ? x[cs[j * 32 + lane]] : (T)0;
#pragma unroll
    for (int j = 0; j < NC; ++j)
      if (j < nc) acc += vs[j * 32 + lane] * xv[j];
    __syncwarp();
    b ^= 1;
    if (more_cols) {
      j0 += NC;
      continue;
    }
    fn(s * 32 + lane, acc);
    acc = 0;
    if (!next) break;
    s = sn;
    W = Wn;
    P = Pn;
    j0 = 0;
    sn = s + nwarps;
    Wn = sn < n_slices ? A.slice_w[sn] : 0;
    Pn = sn < n_slices ? A.slice_ptr[sn] : 0;
  }
  return true;
}

// Write this block's partials; returns true in the last block to finish, whose
// thread 0 then holds the grid-wide sums in v (summed in block order).
template <int K>
__device__ __forceinline__ bool grid_sum(double (&v)[K], double* partials, unsigned* ticket) {
  block_sum<K>(v);
  __shared__ bool last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) partials[blockIdx.x * K + k] = v[k];
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; ++k) acc[k] = 0.0;
  // each thread sums a strided subset in order, then a fixed tree
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] += __ldcg(partials + b * K + k);
  block_sum<K>(acc);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = acc[k];
    *ticket = 0;
  }
  return true;
}

__device__ __forceinline__ bool finite(double v) { return isfinite(v); }

// Stopping rule (LIS -conv_cond): 0 / 1: ||r||_2 <= tol ||b||_2 (x0 = 0);
// 2: ||r||_1 <= tol_w ||b||_1 + tol.
struct ConvRule {
  int mode;
  double tol, tol_w;
};

__device__ __forceinline__ void set_conv(KrylovScalars* ks, const ConvRule& cr, double bb, double b1) {
  ks->conv = cr.mode;
  ks->bb = bb;
  ks->rr_ref = bb;
  ks->b1 = b1;
  ks->tol2 = cr.tol * cr.tol * bb;
  ks->tol1 = cr.tol_w * b1 + cr.tol;
}

// convergence on rr = ||r||_2^2 and r1 = ||r||_1
__device__ __forceinline__ bool conv_met(const KrylovScalars* ks, double rr, double r1) {
  return ks->conv == 2 ? r1 <= ks->tol1 : rr <= ks->tol2;
}

// ---------------------------------------------------------------------------
// CG (Jacobi preconditioner), templated on the storage precision.
template <typename T>
__global__ void k_cg_init(int64_t n, const T* __restrict__ b, const T* __restrict__ dinv, T* __restrict__ x,
                          T* __restrict__ r, T* __restrict__ p, KrylovScalars* ks, double* partials, ConvRule cr) {
  double v[3] = {0.0, 0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T bi = b[i];
    const T zi = dinv ? dinv[i] * bi : (T)0;
    x[i] = 0;
    r[i] = bi;
    p[i] = zi;
    v[0] += (double)bi * (double)zi;
    v[1] += (double)bi * (double)bi;
    v[2] += fabs((double)bi);
  }
  if (grid_sum<3>(v, partials, &ks->ticket[0]) && threadIdx.x == 0) {
    ks->rz = v[0];
    set_conv(ks, cr, v[1], v[2]);
    ks->iter = 0;
    ks->status = PBGPU_OK;
    ks->done = (v[1] == 0.0);
    if (!finite(v[0]) || !finite(v[1])) {
      ks->status = PBGPU_BREAKDOWN;
      ks->done = 1;
    }
  }
}

template <typename T, int G>
__global__ void __launch_bounds__(kBlock, spmv_min_blocks<G>()) k_cg_spmv(SellT<T> A, const T* __restrict__ p, T* __restrict__ q, KrylovScalars* ks, double* partials) {
  if (ks->done) return;
  double v[1] = {0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < A.n_pad; i += (int64_t)gridDim.x * blockDim.x) {
    const T y = sell_row<T, G>(A, i, p);
    q[i] = y;
    v[0] += (double)p[i] * (double)y;
  }
  if (grid_sum<1>(v, partials, &ks->ticket[1]) && threadIdx.x == 0) {
    ks->pq = v[0];
    ks->alpha = ks->rz / v[0];
    if (!(v[0] > 0.0) || !finite(ks->alpha)) {
      ks->status = PBGPU_BREAKDOWN;
      ks->done = 1;
    }
  }
}

template <typename T>
__global__ void k_cg_update(int64_t n, T* __restrict__ x, T* __restrict__ r, const T* __restrict__ p,
                            const T* __restrict__ q, const T* __restrict__ dinv, KrylovScalars* ks, double* partials,
                            int ru_ok) {
  if (ks->done) return;
  const T alpha = (T)ks->alpha;
  double v[3] = {0.0, 0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    const T ri = r[i] - alpha * q[i];
    r[i] = ri;
    if (dinv) v[0] += (double)ri * (double)(dinv[i] * ri);
    v[1] += (double)ri * (double)ri;
    v[2] += fabs((double)ri);
  }
  if (grid_sum<3>(v, partials, &ks->ticket[2]) && threadIdx.x == 0) {
    ks->iter += 1;
    ks->fold = 0;  // the last p-update has folded the previous correction
    ks->rr = v[1];
    ks->r1 = v[2];
    if (!finite(v[0]) || !finite(v[1])) {
      ks->status = PBGPU_BREAKDOWN;
      ks->done = 1;
    } else if (ks->reliable && ru_ok && (conv_met(ks, v[1], v[2]) || v[1] <= ks->delta2 * ks->rr_ref)) {
      ks->ru = 1;  // the FP64 residual (k_ru_residual) decides and supplies beta
    } else if (!ks->reliable && conv_met(ks, v[1], v[2])) {
      ks->done = 1;  // (with reliable updates only the FP64 residual ends the solve)
    } else if (ks->iter >= ks->max_iter) {
      ks->status = PBGPU_NOT_CONVERGED;
      ks->done = 1;
    } else if (dinv) {  // block Jacobi: beta comes from k_bj_apply
      ks->beta = v[0] / ks->rz;
      ks->rz = v[0];
    }
  }
}

// ---------------------------------------------------------------------------
// Reliable updates of the FP32 CG (mixed precision): once its recursive
// residual has fallen by delta since the last FP64 residual (or meets the
// target), b - A (x + d) is computed in FP64 with the FP32 correction d, CG
// continues from it keeping its search direction, and the p-update of the
// same iteration folds d into x (x += d, d = 0).  The residual kernel runs on
// every kRuPeriod-th iteration of a captured chunk and on its last one (it
// returns at once unless an update is due); the updates in between may not
// ask for one, so an update (and the FP64 check that ends the solve) comes at
// most kRuPeriod - 1 iterations after its trigger, and the solve launches
// about 3 + 1/kRuPeriod kernels per iteration.
constexpr int kRuPeriod = 4;

// Iteration k of a chunk of check_every runs the residual kernel: every
// kRuPeriod-th, and the chunk's last one, so every chunk can end the solve.
static inline bool ru_iteration(int k, int check_every) {
  return k % kRuPeriod == kRuPeriod - 1 || k == check_every - 1;
}

// y_p = sum_j A(p, j) (x_j + d_j) in the order of sell_row, x_j + d_j formed
// first (the value x_j takes once d is folded in)
__device__ __forceinline__ double sell_row_sum(const SellT<double>& A, int64_t p, const double* __restrict__ x,
                                               const float* __restrict__ d) {
  const int64_t s = p / A.C;
  const int lane = (int)(p - s * A.C);
  const int W = A.slice_w[s];
  const int64_t sb = A.slice_ptr[s];
  double acc = 0.0;
  for (int j = 0; j < W; ++j) {
    const int64_t k = sell_elem(sb, W, A.C, A.G, lane, j);
    const int32_t c = __ldcs(A.scol + k);
    acc += __ldcs(A.sval + k) * (x[c] + (double)d[c]);
  }
  return acc;
}

__global__ void __launch_bounds__(kBlock, kSpmvMinBlocksWide)
    k_ru_residual(SellT<double> A, int64_t n, const double* __restrict__ b, const double* __restrict__ x,
                  const float* __restrict__ d, float* __restrict__ r32, const float* __restrict__ dinv32,
                  KrylovScalars* ks, double* partials) {
  if (ks->done || !ks->ru) return;
  double a[3] = {0.0, 0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < A.n_pad; i += (int64_t)gridDim.x * blockDim.x) {
    const double ri = i < n ? b[i] - sell_row_sum(A, i, x, d) : 0.0;
    const float rf = (float)ri;
    r32[i] = rf;
    a[0] += ri * ri;
    a[1] += (double)rf * (double)(dinv32[i] * rf);
    a[2] += fabs(ri);
  }
  if (grid_sum<3>(a, partials, &ks->ticket[7]) && threadIdx.x == 0) {
    ks->rr = a[0];
    ks->r1 = a[2];
    ks->ru = 0;
    ks->fold = 1;
    if (!finite(a[0]) || !finite(a[1])) {
      ks->status = PBGPU_BREAKDOWN;
      ks->done = 1;
    } else if (conv_met(ks, a[0], a[2])) {
      ks->done = 1;
    } else if (ks->iter >= ks->max_iter) {
      ks->status = PBGPU_NOT_CONVERGED;
      ks->done = 1;
    } else {
      ks->beta = a[1] / ks->rz;
      ks->rz = a[1];
      ks->rr_ref = a[0];
    }
  }
}

// p = Dinv r + beta p (FP32, Jacobi), and x += d, d = 0 after an FP64 residual
__global__ void k_cg_pupdate_fold(int64_t n, float* __restrict__ p, const float* __restrict__ r,
                                  const float* __restrict__ dinv, double* __restrict__ x, float* __restrict__ d,
                                  const KrylovScalars* ks) {
  if (ks->done) return;
  const float beta = (float)ks->beta;
  const bool fold = ks->fold != 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    p[i] = dinv[i] * r[i] + beta * p[i];
    if (fold) {
      x[i] += (double)d[i];
      d[i] = 0.f;
    }
  }
}

// p = z + beta p with z = Dinv r (Jacobi) or z given (block Jacobi)
template <typename T>
__global__ void k_cg_pupdate(int64_t n, T* __restrict__ p, const T* __restrict__ r, const T* __restrict__ dinv,
                             const T* __restrict__ z, const KrylovScalars* ks) {
  if (ks->done) return;
  const T beta = (T)ks->beta;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = (z ? z[i] : dinv[i] * r[i]) + beta * p[i];
}

// ---------------------------------------------------------------------------
// Block-Jacobi preconditioner: M = blockdiag(A_kk) over blocks of kBjBlock
// consecutive nodes in node (Morton) order, i.e. small spatially compact node
// groups (2 x 2 x 2 nodes in uniform regions).  The inverse blocks are built
// once per assembled system in FP64 and stored symmetrised in FP32 (a fixed
// SPD operator either way, so CG's theory holds); the apply runs in the
// vectors' precision.  Vectors live in SELL order, the blocks in node order:
// iperm maps one to the other.
constexpr int kBjBlock = 8;

// one thread per block: gather A_kk from the SELL rows, invert (Gauss-Jordan,
// SPD so no pivoting), write the symmetrised inverse row-major
template <typename T, int BS>
__global__ void k_bj_setup(SellT<double> A, int64_t n, const int32_t* __restrict__ perm,
                           const int32_t* __restrict__ iperm, float* __restrict__ binv, int* __restrict__ bad) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t n_blk = (n + BS - 1) / BS;
  if (k >= n_blk) return;
  double D[BS][BS], I[BS][BS];
#pragma unroll
  for (int a = 0; a < BS; ++a)
#pragma unroll
    for (int b = 0; b < BS; ++b) {
      D[a][b] = 0.0;
      I[a][b] = a == b ? 1.0 : 0.0;
    }
  const int64_t k0 = k * BS;
#pragma unroll
  for (int li = 0; li < BS; ++li) {
    const int64_t i = k0 + li;
    if (i >= n) {
      D[li][li] = 1.0;
      continue;
    }
    const int64_t p = iperm[i];
    const int64_t s = p / A.C;
    const int lane = (int)(p - s * A.C);
    const int W = A.slice_w[s];
    for (int j = 0; j < W; ++j) {
      const int64_t idx = sell_elem(A.slice_ptr[s], W, A.C, A.G, lane, j);
      const int64_t node = perm[A.scol[idx]];
      const int64_t d = node - k0;
#pragma unroll
      for (int b = 0; b < BS; ++b)
        if (d == b) D[li][b] += A.sval[idx];
    }
  }
  bool ok = true;
#pragma unroll
  for (int c = 0; c < BS; ++c) {
    const double piv = D[c][c];
    ok = ok && piv > 0.0 && isfinite(piv);
    const double ip = 1.0 / piv;
#pragma unroll
    for (int b = 0; b < BS; ++b) {
      D[c][b] *= ip;
      I[c][b] *= ip;
    }
#pragma unroll
    for (int a = 0; a < BS; ++a) {
      if (a == c) continue;
      const double f = D[a][c];
#pragma unroll
      for (int b = 0; b < BS; ++b) {
        D[a][b] -= f * D[c][b];
        I[a][b] -= f * I[c][b];
      }
    }
  }
  if (!ok) atomicExch(bad, 1);
  float* out = binv + k * BS * BS;
#pragma unroll
  for (int a = 0; a < BS; ++a)
#pragma unroll
    for (int b = 0; b < BS; ++b) out[a * BS + b] = (float)(0.5 * (I[a][b] + I[b][a]));
}

// z = M^-1 r; with DOT also (r, z) and beta = (r, z)_new / (r, z)_old
template <typename T, int BS, bool DOT>
__global__ void k_bj_apply(int64_t n, const int32_t* __restrict__ iperm, const float* __restrict__ binv,
                           const T* __restrict__ r, T* __restrict__ z, KrylovScalars* ks, double* partials) {
  if (ks->done) return;
  double v[1] = {0.0};
  const int64_t n_rows = (n + BS - 1) / BS * BS;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_rows;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k0 = i - i % BS;
    const float* row = binv + i * BS;
    T acc = 0;
#pragma unroll
    for (int j = 0; j < BS; ++j)
      if (k0 + j < n) acc += (T)row[j] * r[iperm[k0 + j]];
    if (i < n) {
      const int32_t pi = iperm[i];
      z[pi] = acc;
      if (DOT) v[0] += (double)r[pi] * (double)acc;
    }
  }
  if constexpr (DOT) {
    if (grid_sum<1>(v, partials, &ks->ticket[6]) && threadIdx.x == 0) {
      // the first apply (iteration 0) starts the recurrence with beta = 0
      ks->beta = ks->iter == 0 ? 0.0 : v[0] / ks->rz;
      ks->rz = v[0];
      if (!finite(v[0]) || (ks->iter > 0 && !finite(ks->beta))) {
        ks->status = PBGPU_BREAKDOWN;
        ks->done = 1;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// BiCGStab (right Jacobi preconditioning), templated on the storage precision.
template <typename T>
__global__ void k_bicg_init(int64_t n, const T* __restrict__ b, T* __restrict__ x, T* __restrict__ r,
                            T* __restrict__ rh, T* __restrict__ p, T* __restrict__ v, KrylovScalars* ks,
                            double* partials, ConvRule cr) {
  double s[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T bi = b[i];
    x[i] = 0;
    r[i] = bi;
    rh[i] = bi;
    p[i] = 0;
    v[i] = 0;
    s[0] += (double)bi * (double)bi;
    s[1] += fabs((double)bi);
  }
  if (grid_sum<2>(s, partials, &ks->ticket[0]) && threadIdx.x == 0) {
    set_conv(ks, cr, s[0], s[1]);
    ks->rho = 1.0;
    ks->alpha = 1.0;
    ks->omega = 1.0;
    ks->rv = s[0];              // rho_new = (rh, r)
    ks->beta = s[0];            // (rho_new / rho) * (alpha / omega)
    ks->iter = 0;
    ks->s_conv = 0;
    ks->status = PBGPU_OK;
    ks->done = (s[0] == 0.0);
    if (!finite(s[0])) {
      ks->status = PBGPU_BREAKDOWN;
      ks->done = 1;
    }
  }
}

// p = r + beta (p - omega v);  ph = Dinv p
template <typename T>
__global__ void k_bicg_p(int64_t n, T* __restrict__ p, T* __restrict__ ph, const T* __restrict__ r,
                         const T* __restrict__ v, const T* __restrict__ dinv, const KrylovScalars* ks) {
  if (ks->done) return;
  const T beta = (T)ks->beta, omega = (T)ks->omega;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T pi = r[i] + beta * (p[i] - omega * v[i]);
    p[i] = pi;
    if (dinv) ph[i] = dinv[i] * pi;
  }
}

// v = A ph;  alpha = rho_new / (rh, v)
template <typename T, int G>
__global__ void __launch_bounds__(kBlock, spmv_min_blocks<G>()) k_bicg_v(SellT<T> A, const T* __restrict__ ph, T* __restrict__ v, const T* __restrict__ rh,
                         KrylovScalars* ks, double* partials) {
  if (ks->done) return;
  double s[1] = {0.0};
  spmv_direct_rows<T, G>(A, ph, [&](int64_t i, T y) {
    v[i] = y;
    s[0] += (double)rh[i] * (double)y;
  });
  if (grid_sum<1>(s, partials, &ks->ticket[1]) && threadIdx.x == 0) {
    ks->alpha = ks->rv / s[0];
    if (s[0] == 0.0 || !finite(ks->alpha)) {
      ks->status = PBGPU_BREAKDOWN;
      ks->done = 1;
    }
  }
}

// s = r - alpha v;  sh = Dinv s;  (s, s)
template <typename T>
__global__ void k_bicg_s(int64_t n, const T* __restrict__ r, const T* __restrict__ v, T* __restrict__ s,
                         T* __restrict__ sh, const T* __restrict__ dinv, KrylovScalars* ks, double* partials) {
  if (ks->done) return;
  const T alpha = (T)ks->alpha;
  double a[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T si = r[i] - alpha * v[i];
    s[i] = si;
    if (dinv) sh[i] = dinv[i] * si;
    a[0] += (double)si * (double)si;
    a[1] += fabs((double)si);
  }
  if (grid_sum<2>(a, partials, &ks->ticket[2]) && threadIdx.x == 0) {
    ks->ss = a[0];
    ks->r1 = a[1];
    ks->s_conv = conv_met(ks, a[0], a[1]);
  }
}

// t = A sh;  omega = (t, s) / (t, t)
template <typename T, int G>
__global__ void __launch_bounds__(kBlock, kSpmvMinBlocksWide) k_bicg_t(SellT<T> A, const T* __restrict__ sh, T* __restrict__ t, const T* __restrict__ s,
                         KrylovScalars* ks, double* partials) {
  if (ks->done || ks->s_conv) return;
  double a[2] = {0.0, 0.0};
  spmv_direct_rows<T, G>(A, sh, [&](int64_t i, T y) {
    t[i] = y;
    a[0] += (double)y * (double)s[i];
    a[1] += (double)y * (double)y;
  });
  if (grid_sum<2>(a, partials, &ks->ticket[3]) && threadIdx.x == 0) {
    ks->ts = a[0];
    ks->tt = a[1];
    ks->omega = a[1] > 0.0 ? a[0] / a[1] : 0.0;
  }
}

// x += alpha ph + omega sh;  r = s - omega t;  (r, r), (rh, r)
template <typename T>
__global__ void k_bicg_x(int64_t n, T* __restrict__ x, T* __restrict__ r, const T* __restrict__ ph,
                         const T* __restrict__ sh, const T* __restrict__ s, const T* __restrict__ t,
                         const T* __restrict__ rh, KrylovScalars* ks, double* partials) {
  if (ks->done) return;
  const T alpha = (T)ks->alpha;
  if (ks->s_conv) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      x[i] += alpha * ph[i];
    double z[1] = {0.0};
    if (grid_sum<1>(z, partials, &ks->ticket[4]) && threadIdx.x == 0) {
      ks->iter += 1;
      ks->rr = ks->ss;
      ks->done = 1;
    }
    return;
  }
  const T omega = (T)ks->omega;
  double a[3] = {0.0, 0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] += alpha * ph[i] + omega * sh[i];
    const T ri = s[i] - omega * t[i];
    r[i] = ri;
    a[0] += (double)ri * (double)ri;
    a[1] += (double)rh[i] * (double)ri;
    a[2] += fabs((double)ri);
  }
  if (grid_sum<3>(a, partials, &ks->ticket[4]) && threadIdx.x == 0) {
    ks->iter += 1;
    ks->rr = a[0];
    ks->r1 = a[2];
    const double rho_new = a[1];
    if (!finite(a[0]) || !finite(a[1])) {
      ks->status = PBGPU_BREAKDOWN;
      ks->done = 1;
    } else if (conv_met(ks, a[0], a[2])) {
      ks->done = 1;
    } else if (ks->iter >= ks->max_iter) {
      ks->status = PBGPU_NOT_CONVERGED;
      ks->done = 1;
    } else if (rho_new == 0.0 || ks->omega == 0.0) {
      ks->status = PBGPU_BREAKDOWN;
      ks->done = 1;
    } else {
      ks->beta = (rho_new / ks->rv) * (ks->alpha / ks->omega);
      ks->rho = ks->rv;
      ks->rv = rho_new;
    }
  }
}

// ---------------------------------------------------------------------------
// FP64 residual r = b - A x, its norm, and an fp32 copy (mixed precision).
template <int G>
__global__ void __launch_bounds__(kBlock, kSpmvMinBlocksWide) k_residual(SellT<double> A, int64_t n, const double* __restrict__ b, const double* __restrict__ x,
                           double* __restrict__ r, float* __restrict__ r32, KrylovScalars* ks, double* partials) {
  double a[4] = {0.0, 0.0, 0.0, 0.0};
  spmv_direct_rows<double, G>(A, x, [&](int64_t i, double y) {
    const double ri = i < n ? b[i] - y : 0.0;
    if (r) r[i] = ri;
    if (r32) r32[i] = (float)ri;
    a[0] += ri * ri;
    a[1] += i < n ? b[i] * b[i] : 0.0;
    a[2] += fabs(ri);
    a[3] += i < n ? fabs(b[i]) : 0.0;
  });
  if (grid_sum<4>(a, partials, &ks->ticket[5]) && threadIdx.x == 0) {
    ks->rr = a[0];
    ks->bb = a[1];
    ks->r1 = a[2];
    ks->b1 = a[3];
  }
}

// ---------------------------------------------------------------------------
// The SpMV kernels again with the matrix staged by bulk async copies (C = 32,
// G = 1).  A bounded wait that gives up ends the solve with PBGPU_TIMEOUT.
// resident blocks per SM of the staged kernels: their FP64 shared memory
// (2 buffers x NC columns x 8 warps) allows 4 blocks at NC = 8, 3 at 12, 2 at 16
__host__ __device__ constexpr int tma_min_blocks(int nc) { return nc <= 8 ? 4 : nc <= 12 ? 3 : 2; }

__device__ __forceinline__ void tma_timeout(KrylovScalars* ks) {
  if ((threadIdx.x & 31) == 0) {
    atomicExch(&ks->status, (int)PBGPU_TIMEOUT);
    atomicExch(&ks->done, 1);
  }
}
// Block-uniform early exit: a staged kernel that timed out sets `done` while
// other blocks of the same launch may still be starting, so one thread reads
// the flags for the whole block (the warps must stay complete for the votes).
__device__ __forceinline__ bool block_skip(const KrylovScalars* ks, bool with_s_conv) {
  __shared__ int skip;
  if (threadIdx.x == 0) {
    const volatile int* f = reinterpret_cast<const volatile int*>(&ks->done);
    skip = *f != 0 || (with_s_conv && *reinterpret_cast<const volatile int*>(&ks->s_conv) != 0);
  }
  __syncthreads();
  return skip != 0;
}
__device__ __forceinline__ bool timed_out(const KrylovScalars* ks) {
  return *reinterpret_cast<const volatile int*>(&ks->status) == PBGPU_TIMEOUT;
}

template <typename T, int NC>
__global__ void __launch_bounds__(kBlock, tma_min_blocks(NC))
    k_cg_spmv_tma(SellT<T> A, const T* __restrict__ p, T* __restrict__ q, KrylovScalars* ks, double* partials) {
  if (block_skip(ks, false)) return;
  double v[1] = {0.0};
  if (!spmv_tma_rows<T, NC>(A, p, [&](int64_t i, T y) {
        q[i] = y;
        v[0] += (double)p[i] * (double)y;
      }, ks->wait_ns))
    tma_timeout(ks);
  if (grid_sum<1>(v, partials, &ks->ticket[1]) && threadIdx.x == 0 && !timed_out(ks)) {
    ks->pq = v[0];
    ks->alpha = ks->rz / v[0];
    if (!(v[0] > 0.0) || !finite(ks->alpha)) {
      ks->status = PBGPU_BREAKDOWN;
      ks->done = 1;
    }
  }
}

template <typename T, int NC>
__global__ void __launch_bounds__(kBlock, tma_min_blocks(NC))
    k_bicg_v_tma(SellT<T> A, const T* __restrict__ ph, T* __restrict__ v, const T* __restrict__ rh,
                 KrylovScalars* ks, double* partials) {
  if (block_skip(ks, false)) return;
  double s[1] = {0.0};
  if (!spmv_tma_rows<T, NC>(A, ph, [&](int64_t i, T y) {
        v[i] = y;
        s[0] += (double)rh[i] * (double)y;
      }, ks->wait_ns))
    tma_timeout(ks);
  if (grid_sum<1>(s, partials, &ks->ticket[1]) && threadIdx.x == 0 && !timed_out(ks)) {
    ks->alpha = ks->rv / s[0];
    if (s[0] == 0.0 || !finite(ks->alpha)) {
      ks->status = PBGPU_BREAKDOWN;
      ks->done = 1;
    }
  }
}

template <typename T, int NC>
__global__ void __launch_bounds__(kBlock, tma_min_blocks(NC))
    k_bicg_t_tma(SellT<T> A, const T* __restrict__ sh, T* __restrict__ t, const T* __restrict__ s,
                 KrylovScalars* ks, double* partials) {
  if (block_skip(ks, true)) return;
  double a[2] = {0.0, 0.0};
  if (!spmv_tma_rows<T, NC>(A, sh, [&](int64_t i, T y) {
        t[i] = y;
        a[0] += (double)y * (double)s[i];
        a[1] += (double)y * (double)y;
      }, ks->wait_ns))
    tma_timeout(ks);
  if (grid_sum<2>(a, partials, &ks->ticket[3]) && threadIdx.x == 0 && !timed_out(ks)) {
    ks->ts = a[0];
    ks->tt = a[1];
    ks->omega = a[1] > 0.0 ? a[0] / a[1] : 0.0;
  }
}

template <int NC>
__global__ void __launch_bounds__(kBlock, tma_min_blocks(NC))
    k_residual_tma(SellT<double> A, int64_t n, const double* __restrict__ b, const double* __restrict__ x,
                   double* __restrict__ r, float* __restrict__ r32, KrylovScalars* ks, double* partials) {
  double a[4] = {0.0, 0.0, 0.0, 0.0};
  if (!spmv_tma_rows<double, NC>(A, x, [&](int64_t i, double y) {
        const double ri = i < n ? b[i] - y : 0.0;
        if (r) r[i] = ri;
        if (r32) r32[i] = (float)ri;
        a[0] += ri * ri;
        a[1] += i < n ? b[i] * b[i] : 0.0;
        a[2] += fabs(ri);
        a[3] += i < n ? fabs(b[i]) : 0.0;
      }, ks->wait_ns))
    tma_timeout(ks);
  if (grid_sum<4>(a, partials, &ks->ticket[5]) && threadIdx.x == 0) {
    ks->rr = a[0];
    ks->bb = a[1];
    ks->r1 = a[2];
    ks->b1 = a[3];
  }
}

// ---------------------------------------------------------------------------
// CGS (conjugate gradient squared, right preconditioning M), templated on the
// storage precision; LIS's default solver in the reference's options
// (src/pb_class.cpp:970).  Per iteration, with rho = (rh, r):
//   u = r + beta q;  p = u + beta (q + beta p);  ph = M^-1 p;  v = A ph
//   alpha = rho / (rh, v);  q = u - alpha v;  uh = M^-1 (u + q)
//   x += alpha uh;  r -= alpha A uh;  beta = rho_new / rho
// The last SpMV is fused with the x / r updates and the three reductions.
// Buffers: u in `s`, uh in `sh`, and u + q in `v` once v is consumed.

template <typename T>
__global__ void k_cgs_init(int64_t n, const T* __restrict__ b, T* __restrict__ x, T* __restrict__ r,
                           T* __restrict__ rh, T* __restrict__ p, T* __restrict__ q, KrylovScalars* ks,
                           double* partials, ConvRule cr) {
  double s[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T bi = b[i];
    x[i] = 0;
    r[i] = bi;
    rh[i] = bi;
    p[i] = 0;
    q[i] = 0;
    s[0] += (double)bi * (double)bi;
    s[1] += fabs((double)bi);
  }
  if (grid_sum<2>(s, partials, &ks->ticket[0]) && threadIdx.x == 0) {
    set_conv(ks, cr, s[0], s[1]);
    ks->rv = s[0];  // rho = (rh, r)
    ks->beta = 0.0;
    ks->iter = 0;
    ks->status = PBGPU_OK;
    ks->done = (s[0] == 0.0);
    if (!finite(s[0])) {
      ks->status = PBGPU_BREAKDOWN;
      ks->done = 1;
    }
  }
}

// u = r + beta q;  p = u + beta (q + beta p);  ph = Dinv p (Jacobi)
template <typename T>
__global__ void k_cgs_p(int64_t n, const T* __restrict__ r, const T* __restrict__ q, T* __restrict__ u,
                        T* __restrict__ p, T* __restrict__ ph, const T* __restrict__ dinv, const KrylovScalars* ks) {
  if (ks->done) return;
  const T beta = (T)ks->beta;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T qi = q[i];
    const T ui = r[i] + beta * qi;
    const T pi = ui + beta * (qi + beta * p[i]);
    u[i] = ui;
    p[i] = pi;
    if (dinv) ph[i] = dinv[i] * pi;
  }
}

// q = u - alpha v;  w = u + q;  uh = Dinv w (Jacobi), else w is left in v for
// the block-Jacobi apply
template <typename T>
__global__ void k_cgs_q(int64_t n, const T* __restrict__ u, T* __restrict__ v, T* __restrict__ q,
                        T* __restrict__ uh, const T* __restrict__ dinv, const KrylovScalars* ks) {
  if (ks->done) return;
  const T alpha = (T)ks->alpha;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T ui = u[i];
    const T qi = ui - alpha * v[i];
    q[i] = qi;
    if (dinv)
      uh[i] = dinv[i] * (ui + qi);
    else
      v[i] = ui + qi;
  }
}

// The rows of y = A x for this kernel: staged (NC > 0) or direct.
template <typename T, int G, int NC, typename Fn>
__device__ __forceinline__ bool spmv_rows(const SellT<T>& A, const T* __restrict__ x, Fn&& fn, uint64_t wait_ns) {
  if constexpr (NC > 0) {
    return spmv_tma_rows<T, NC>(A, x, fn, wait_ns);
  } else {
    spmv_direct_rows<T, G>(A, x, fn);
    return true;
  }
}

// v = A ph;  alpha = rho / (rh, v)
template <typename T, int G, int NC>
__global__ void __launch_bounds__(kBlock, NC > 0 ? tma_min_blocks(NC) : spmv_min_blocks<G>())
    k_cgs_v(SellT<T> A, const T* __restrict__ ph, T* __restrict__ v, const T* __restrict__ rh, KrylovScalars* ks,
            double* partials) {
  if (block_skip(ks, false)) return;
  double a[1] = {0.0};
  if (!spmv_rows<T, G, NC>(A, ph, [&](int64_t i, T y) {
        v[i] = y;
        a[0] += (double)rh[i] * (double)y;
      }, ks->wait_ns))
    tma_timeout(ks);
  if (grid_sum<1>(a, partials, &ks->ticket[1]) && threadIdx.x == 0 && !timed_out(ks)) {
    ks->alpha = ks->rv / a[0];
    if (a[0] == 0.0 || !finite(ks->alpha)) {
      ks->status = PBGPU_BREAKDOWN;
      ks->done = 1;
    }
  }
}

// r -= alpha A uh;  x += alpha uh;  (r, r), (rh, r), ||r||_1; convergence; beta
template <typename T, int G, int NC>
__global__ void __launch_bounds__(kBlock, NC > 0 ? tma_min_blocks(NC) : kSpmvMinBlocksWide)
    k_cgs_r(SellT<T> A, const T* __restrict__ uh, T* __restrict__ x, T* __restrict__ r, const T* __restrict__ rh,
            KrylovScalars* ks, double* partials) {
  if (block_skip(ks, false)) return;
  const T alpha = (T)ks->alpha;
  double a[3] = {0.0, 0.0, 0.0};
  if (!spmv_rows<T, G, NC>(A, uh, [&](int64_t i, T y) {
        x[i] += alpha * uh[i];
        const T ri = r[i] - alpha * y;
        r[i] = ri;
        a[0] += (double)ri * (double)ri;
        a[1] += (double)rh[i] * (double)ri;
        a[2] += fabs((double)ri);
      }, ks->wait_ns))
    tma_timeout(ks);
  if (grid_sum<3>(a, partials, &ks->ticket[3]) && threadIdx.x == 0 && !timed_out(ks)) {
    ks->iter += 1;
    ks->rr = a[0];
    ks->r1 = a[2];
    if (!finite(a[0]) || !finite(a[1])) {
      ks->status = PBGPU_BREAKDOWN;
      ks->done = 1;
    } else if (conv_met(ks, a[0], a[2])) {
      ks->done = 1;
    } else if (ks->iter >= ks->max_iter) {
      ks->status = PBGPU_NOT_CONVERGED;
      ks->done = 1;
    } else if (a[1] == 0.0) {
      ks->status = PBGPU_BREAKDOWN;
      ks->done = 1;
    } else {
      ks->beta = a[1] / ks->rv;
      ks->rv = a[1];
    }
  }
}

__global__ void k_axpy_f32(int64_t n, double* __restrict__ x, const float* __restrict__ d) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] += (double)d[i];
}

__global__ void k_to_f32(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

template <typename T>
__global__ void k_fill(int64_t n, T* __restrict__ a, T v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    a[i] = v;
}

__global__ void k_gather_phi(int64_t n, const int32_t* __restrict__ iperm, const double* __restrict__ x,
                             double* __restrict__ phi) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) phi[i] = x[iperm[i]];
}

// ---------------------------------------------------------------------------
// Host drivers.

static int grid_blocks(const Context* c, int64_t n) {
  const int64_t cap = (int64_t)c->sm_count * 8;
  int64_t g = (n + kBlock - 1) / kBlock;
  if (g > cap) g = cap;
  return (int)(g < 1 ? 1 : g);
}

// Blocks of a grid-stride kernel that fill the GPU in exactly one wave: its
// resident blocks per SM (kBlock threads, no dynamic shared memory) times the
// SMs, or fewer when the rows need fewer.  The SpMV kernels hold 5 or 6
// blocks per SM; a grid of 8 per SM would leave a second wave of blocks
// running on a partly occupied GPU after the first finished (every block of a
// grid-stride loop has the same number of rows).
static int wave_grid(const Context* c, const void* kernel, int64_t rows) {
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kBlock, 0) != cudaSuccess || occ <= 0) {
    cudaGetLastError();
    return grid_blocks(c, rows);
  }
  const int64_t need = (rows + kBlock - 1) / kBlock;
  const int64_t g = std::min<int64_t>(need, (int64_t)c->sm_count * occ);
  return (int)(g < 1 ? 1 : g);
}

// Chunk width (columns per bulk copy) of the staged SpMV for this context:
// 0 when the staged path does not apply (layouts other than C = 32, G = 1) or
// is switched off with PBGPU_SPMV=direct; PBGPU_SPMV_COLS=8|12|16 overrides
// the context's choice.
static int staged_cols(const Context* c, int C, int G) {
  if (C != 32 || G != 1) return 0;
  const char* env = std::getenv("PBGPU_SPMV");
  if (env && std::strcmp(env, "direct") == 0) return 0;
  int nc = c->spmv_cols;
  if (const char* e2 = std::getenv("PBGPU_SPMV_COLS")) nc = std::atoi(e2);
  return (nc == 8 || nc == 12 || nc == 16) ? nc : 16;
}

// The G = 4 layout is walked two column groups per iteration (sell_row<T, 8>:
// the same sums in the same order, with half the dependent load round trips;
// measured 2-4 % faster than one group per iteration on 3.3 M and 14.5 M DoF
// systems).  PBGPU_SPMV_PAIRS=0 selects the one-group kernel.
static bool spmv_pairs() {
  const char* e = std::getenv("PBGPU_SPMV_PAIRS");
  return !(e && e[0] == '0');
}

// Grid of the staged SpMV kernels for storage type T and chunk width NC:
// resident blocks per SM at their dynamic shared memory; 0 if they cannot run.
template <typename T, int NC>
static int tma_grid(Context* c) {
  const int smem = (int)tma_smem_bytes<T, NC>();
  int occ = 0;
  auto setup = [&](const void* f) -> cudaError_t {
    cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    int o = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, f, kBlock, smem);
    occ = occ == 0 ? o : std::min(occ, o);
    return e;
  };
  cudaError_t e = setup((const void*)k_cg_spmv_tma<T, NC>);
  if (e == cudaSuccess) e = setup((const void*)k_bicg_v_tma<T, NC>);
  if (e == cudaSuccess) e = setup((const void*)k_bicg_t_tma<T, NC>);
  if (e == cudaSuccess) e = setup((const void*)k_cgs_v<T, 1, NC>);
  if (e == cudaSuccess) e = setup((const void*)k_cgs_r<T, 1, NC>);
  if (e == cudaSuccess && sizeof(T) == sizeof(double)) e = setup((const void*)k_residual_tma<NC>);
  if (e != cudaSuccess || occ <= 0) {
    cudaGetLastError();
    return 0;  // the direct kernels serve the layout as well
  }
  return c->sm_count * std::min(occ, 8);
}

template <typename T>
struct KrylovVecs {
  T *x, *r, *p, *q, *rh, *v, *s, *t, *ph, *sh;
  const T *b, *dinv;  // dinv: 1 / diag (Jacobi), ones (no preconditioner), null (block Jacobi)
  SellT<T> A;
  T* z = nullptr;                   // block Jacobi: preconditioned residual (CG)
  // reliable updates (T = float): the FP64 system and solution
  const SellT<double>* A64 = nullptr;
  const double* b64 = nullptr;
  double* x64 = nullptr;
  int64_t n_rows = 0;
  const float* bj = nullptr;        // block Jacobi: inverse blocks, node order
  const int32_t* iperm = nullptr;   // node -> SELL position
  int64_t n_nodes = 0;
};

// Run one Krylov solve on (A, b) with stopping rule cr; x0 = 0.  GW is the
// SELL column-group width of A; NC > 0 selects the staged SpMV with chunks of
// NC columns (GW = 1).
template <typename T, int GW, int NC>
static int krylov_g(Context* c, int method, const KrylovVecs<T>& K, ConvRule cr, int max_iter, int check_every,
                    int* iters, int* status) {
  const int64_t n = K.A.n_pad;
  const int G = grid_blocks(c, n);
  // one-wave grids of the kernels that multiply by the matrix
  const int Gs = wave_grid(c, method == PBGPU_CG    ? (const void*)k_cg_spmv<T, GW>
                              : method == PBGPU_CGS ? (const void*)k_cgs_v<T, GW, 0>
                                                    : (const void*)k_bicg_v<T, GW>, n);
  const int Gw = wave_grid(c, method == PBGPU_CGS ? (const void*)k_cgs_r<T, GW, 0> : (const void*)k_bicg_t<T, GW>, n);
  KrylovScalars* ks = c->ks.get();
  double* part = c->partials.get();
  PBGPU_CUDA(c, cudaMemsetAsync(ks, 0, sizeof(KrylovScalars), c->stream));
  int mi = max_iter;
  PBGPU_CUDA(c, cudaMemcpyAsync(&ks->max_iter, &mi, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  unsigned long long wns = (unsigned long long)(c->wait_s * 1e9);
  PBGPU_CUDA(c, cudaMemcpyAsync(&ks->wait_ns, &wns, sizeof(wns), cudaMemcpyHostToDevice, c->stream));
  if (K.x64 && method == PBGPU_CG) {
    static const int on = 1;
    static const double delta2 = 0.01;  // an FP64 residual every 10x reduction of the FP32 one
    PBGPU_CUDA(c, cudaMemcpyAsync(&ks->reliable, &on, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    PBGPU_CUDA(c, cudaMemcpyAsync(&ks->delta2, &delta2, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  }
  const bool bj = K.dinv == nullptr;
  const int Gb = grid_blocks(c, (K.n_nodes + kBjBlock - 1) / kBjBlock * kBjBlock);
  // z = M^-1 r (with (r, z) and beta when `dot`)
  auto bj_apply = [&](const T* in, T* out, bool dot) {
    if (dot)
      k_bj_apply<T, kBjBlock, true><<<Gb, kBlock, 0, c->stream>>>(K.n_nodes, K.iperm, K.bj, in, out, ks, part);
    else
      k_bj_apply<T, kBjBlock, false><<<Gb, kBlock, 0, c->stream>>>(K.n_nodes, K.iperm, K.bj, in, out, ks, part);
  };
  if (method == PBGPU_CG) {
    k_cg_init<T><<<G, kBlock, 0, c->stream>>>(n, K.b, K.dinv, K.x, K.r, K.p, ks, part, cr);
    c->launches += 1;
    if (bj) {  // p = z = M^-1 b
      bj_apply(K.r, K.z, true);
      k_cg_pupdate<T><<<G, kBlock, 0, c->stream>>>(n, K.p, K.r, K.dinv, K.z, ks);
      c->launches += 2;
    }
  } else if (method == PBGPU_CGS) {
    k_cgs_init<T><<<G, kBlock, 0, c->stream>>>(n, K.b, K.x, K.r, K.rh, K.p, K.q, ks, part, cr);
    c->launches += 1;
  } else {
    k_bicg_init<T><<<G, kBlock, 0, c->stream>>>(n, K.b, K.x, K.r, K.rh, K.p, K.v, ks, part, cr);
    c->launches += 1;
  }
  PBGPU_CUDA(c, cudaGetLastError());
  // With profiling on, events recorded around every SpMV launch become event
  // nodes of the graph; the elapsed times of the launches that did work are
  // summed after each chunk.
  const int tg = NC > 0 ? tma_grid<T, (NC > 0 ? NC : 16)>(c) : 0;
  const size_t smem = tma_smem_bytes<T, (NC > 0 ? NC : 16)>();
  const int spmv_per_it = method == PBGPU_CG ? 1 : 2;
  std::vector<cudaEvent_t> ev;
  if (c->profiling) {
    ev.resize(2 * spmv_per_it * check_every);
    for (cudaEvent_t& e : ev) PBGPU_CUDA(c, cudaEventCreate(&e));
  }
  // cudaEventRecordExternal makes the record a node of the captured graph
  // (a plain record inside a capture only orders streams)
  auto mark = [&](int k, int which, int end) {
    if (c->profiling)
      cudaEventRecordWithFlags(ev[2 * (k * spmv_per_it + which) + end], c->stream, cudaEventRecordExternal);
  };
  // the chunk of iterations is captured once and replayed
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  PBGPU_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int kernels_per_chunk = 0;
  for (int k = 0; k < check_every; ++k) {
    kernels_per_chunk += (method == PBGPU_CG ? 3 : method == PBGPU_CGS ? 4 : 5) + (bj ? (method == PBGPU_CG ? 1 : 2) : 0) +
                         (K.x64 && method == PBGPU_CG && ru_iteration(k, check_every) ? 1 : 0);
    if (method == PBGPU_CG) {
      mark(k, 0, 0);
      if (tg)
        k_cg_spmv_tma<T, (NC > 0 ? NC : 16)><<<tg, kBlock, smem, c->stream>>>(K.A, K.p, K.q, ks, part);
      else
        k_cg_spmv<T, GW><<<Gs, kBlock, 0, c->stream>>>(K.A, K.p, K.q, ks, part);
      mark(k, 0, 1);
      const bool ru_here = K.x64 && ru_iteration(k, check_every);
      k_cg_update<T><<<G, kBlock, 0, c->stream>>>(n, K.x, K.r, K.p, K.q, K.dinv, ks, part, ru_here ? 1 : 0);
      bool folded = false;
      if constexpr (std::is_same<T, float>::value) {
        if (K.x64) {
          // the FP64 residual b - A (x + d) when an update is due, then the
          // p-update that also folds d into x
          if (ru_here)
            k_ru_residual<<<wave_grid(c, (const void*)k_ru_residual, K.A64->n_pad), kBlock, 0, c->stream>>>(
                *K.A64, K.n_rows, K.b64, K.x64, K.x, K.r, K.dinv, ks, part);
          k_cg_pupdate_fold<<<G, kBlock, 0, c->stream>>>(n, K.p, K.r, K.dinv, K.x64, K.x, ks);
          folded = true;
        }
      }
      if (!folded) {
        if (bj) bj_apply(K.r, K.z, true);
        k_cg_pupdate<T><<<G, kBlock, 0, c->stream>>>(n, K.p, K.r, K.dinv, K.z, ks);
      }
    } else if (method == PBGPU_CGS) {
      k_cgs_p<T><<<G, kBlock, 0, c->stream>>>(n, K.r, K.q, K.s, K.p, K.ph, K.dinv, ks);
      if (bj) bj_apply(K.p, K.ph, false);
      mark(k, 0, 0);
      if (tg)
        k_cgs_v<T, 1, (NC > 0 ? NC : 16)><<<tg, kBlock, smem, c->stream>>>(K.A, K.ph, K.v, K.rh, ks, part);
      else
        k_cgs_v<T, GW, 0><<<Gs, kBlock, 0, c->stream>>>(K.A, K.ph, K.v, K.rh, ks, part);
      mark(k, 0, 1);
      k_cgs_q<T><<<G, kBlock, 0, c->stream>>>(n, K.s, K.v, K.q, K.sh, K.dinv, ks);
      if (bj) bj_apply(K.v, K.sh, false);
      mark(k, 1, 0);
      if (tg)
        k_cgs_r<T, 1, (NC > 0 ? NC : 16)><<<tg, kBlock, smem, c->stream>>>(K.A, K.sh, K.x, K.r, K.rh, ks, part);
      else
        k_cgs_r<T, GW, 0><<<Gw, kBlock, 0, c->stream>>>(K.A, K.sh, K.x, K.r, K.rh, ks, part);
      mark(k, 1, 1);
    } else {
      k_bicg_p<T><<<G, kBlock, 0, c->stream>>>(n, K.p, K.ph, K.r, K.v, K.dinv, ks);
      if (bj) bj_apply(K.p, K.ph, false);
      mark(k, 0, 0);
      if (tg)
        k_bicg_v_tma<T, (NC > 0 ? NC : 16)><<<tg, kBlock, smem, c->stream>>>(K.A, K.ph, K.v, K.rh, ks, part);
      else
        k_bicg_v<T, GW><<<Gs, kBlock, 0, c->stream>>>(K.A, K.ph, K.v, K.rh, ks, part);
      mark(k, 0, 1);
      k_bicg_s<T><<<G, kBlock, 0, c->stream>>>(n, K.r, K.v, K.s, K.sh, K.dinv, ks, part);
      if (bj) bj_apply(K.s, K.sh, false);
      mark(k, 1, 0);
      if (tg)
        k_bicg_t_tma<T, (NC > 0 ? NC : 16)><<<tg, kBlock, smem, c->stream>>>(K.A, K.sh, K.t, K.s, ks, part);
      else
        k_bicg_t<T, GW><<<Gw, kBlock, 0, c->stream>>>(K.A, K.sh, K.t, K.s, ks, part);
      mark(k, 1, 1);
      k_bicg_x<T><<<G, kBlock, 0, c->stream>>>(n, K.x, K.r, K.ph, K.sh, K.s, K.t, K.rh, ks, part);
    }
  }
  cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
  if (ce != cudaSuccess) {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    return cuda_fail(c, ce, "cudaStreamEndCapture");
  }
  ce = cudaGraphInstantiate(&exec, graph, 0);
  if (ce != cudaSuccess) {
    cudaGraphDestroy(graph);
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    return cuda_fail(c, ce, "cudaGraphInstantiate");
  }
  int rc = PBGPU_OK;
  const int max_chunks = max_iter / check_every + 2;
  int prev_iter = 0;
  // Chunk j leaves its scalars in the pinned slot ks_host[j % 2] and marks
  // them with event evc[j % 2].  The next chunk is launched before the host
  // waits for the current one, so the stream does not idle while the host
  // reads a chunk's scalars and launches the graph again; a chunk launched
  // after the solve ended does nothing (every kernel returns at once once
  // ks->done is set, and none of them changes the scalars then).  With
  // profiling on, each chunk is waited for before the next is launched: the
  // chunks share the SpMV timing events.
  const bool ahead = !c->profiling;
  auto launch_chunk = [&](int j) -> cudaError_t {
    cudaError_t e = cudaGraphLaunch(exec, c->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(c->ks_host + (j & 1), ks, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaEventRecord(c->evc[j & 1], c->stream);
    return e;
  };
  int launched = 0;
  const KrylovScalars* h = c->ks_host;
  ce = launch_chunk(0);
  if (ce == cudaSuccess) launched = 1;
  for (int chunk = 0; ce == cudaSuccess && chunk < max_chunks; ++chunk) {
    if (ahead && launched < max_chunks) {
      ce = launch_chunk(launched);
      if (ce != cudaSuccess) break;
      ++launched;
    }
    ce = cudaEventSynchronize(c->evc[chunk & 1]);
    if (ce != cudaSuccess) break;
    h = c->ks_host + (chunk & 1);
    const int now = h->iter;
    if (c->profiling) {
      // iteration k of this chunk did its SpMV(s) when it is below the count
      // of completed iterations; the t-SpMV of a BiCGStab iteration that
      // stopped on ||s|| did not run
      for (int k = 0; k < check_every && prev_iter + k < now; ++k)
        for (int w = 0; w < spmv_per_it; ++w) {
          if (w == 1 && prev_iter + k == now - 1 && h->s_conv) continue;
          float ms = 0.f;
          if (cudaEventElapsedTime(&ms, ev[2 * (k * spmv_per_it + w)], ev[2 * (k * spmv_per_it + w) + 1]) ==
              cudaSuccess) {
            c->spmv_ms += ms;
            c->spmv_launches += 1;
          } else {
            cudaGetLastError();  // measurement only
          }
        }
    }
    prev_iter = now;
    if (h->done) break;
    if (!ahead && launched < max_chunks) {
      ce = launch_chunk(launched);
      if (ce != cudaSuccess) break;
      ++launched;
    }
  }
  // the chunk launched past the last one waited for (its kernels return at once)
  const cudaError_t e_drain = cudaStreamSynchronize(c->stream);
  if (ce == cudaSuccess) ce = e_drain;
  if (ce != cudaSuccess) rc = cuda_fail(c, ce, "krylov chunk");
  c->launches += (int64_t)kernels_per_chunk * launched;
  if (h != c->ks_host) std::memcpy(c->ks_host, h, sizeof(KrylovScalars));
  const cudaError_t e_exec = cudaGraphExecDestroy(exec);
  const cudaError_t e_graph = cudaGraphDestroy(graph);
  cudaError_t e_ev = cudaSuccess;
  for (cudaEvent_t e : ev) {
    const cudaError_t d = cudaEventDestroy(e);
    if (d != cudaSuccess) e_ev = d;
  }
  if (rc != PBGPU_OK) return rc;
  if (e_exec != cudaSuccess) return cuda_fail(c, e_exec, "cudaGraphExecDestroy");
  if (e_graph != cudaSuccess) return cuda_fail(c, e_graph, "cudaGraphDestroy");
  if (e_ev != cudaSuccess) return cuda_fail(c, e_ev, "cudaEventDestroy");
  *iters = c->ks_host->iter;
  c->krylov_iters += c->ks_host->iter;
  c->spmv_bytes = (double)c->nnz * (sizeof(T) + 4) + 2.0 * (double)c->n * sizeof(T);
  *status = c->ks_host->done ? c->ks_host->status : PBGPU_NOT_CONVERGED;
  return PBGPU_OK;
}

template <typename T>
static int krylov(Context* c, int method, const KrylovVecs<T>& K, ConvRule cr, int max_iter, int check_every,
                  int* iters, int* status) {
  switch (staged_cols(c, K.A.C, K.A.G)) {
    case 8: return krylov_g<T, 1, 8>(c, method, K, cr, max_iter, check_every, iters, status);
    case 12: return krylov_g<T, 1, 12>(c, method, K, cr, max_iter, check_every, iters, status);
    case 16: return krylov_g<T, 1, 16>(c, method, K, cr, max_iter, check_every, iters, status);
    default: break;
  }
  switch (K.A.G) {
    case 1: return krylov_g<T, 1, 0>(c, method, K, cr, max_iter, check_every, iters, status);
    case 2: return krylov_g<T, 2, 0>(c, method, K, cr, max_iter, check_every, iters, status);
    default:
      if (spmv_pairs())  // the G = 4 layout walked two groups per iteration
        return krylov_g<T, 8, 0>(c, method, K, cr, max_iter, check_every, iters, status);
      return krylov_g<T, 4, 0>(c, method, K, cr, max_iter, check_every, iters, status);
  }
}

// r = b - A x (fp64); optional fp64 / fp32 copies of r; norms into ks
static void launch_residual(Context* c, const SellT<double>& A, int64_t n, double* r, float* r32) {
  const int g = wave_grid(c, A.G == 1 ? (const void*)k_residual<1> : A.G == 2 ? (const void*)k_residual<2>
                                                                      : (const void*)k_residual<4>, A.n_pad);
  auto staged = [&](auto nc_tag) -> bool {
    constexpr int NC = decltype(nc_tag)::value;
    const int tg = tma_grid<double, NC>(c);
    if (!tg) return false;
    k_residual_tma<NC><<<tg, kBlock, tma_smem_bytes<double, NC>(), c->stream>>>(A, n, c->b.get(), c->x.get(), r,
                                                                              r32, c->ks.get(), c->partials.get());
    return true;
  };
  switch (staged_cols(c, A.C, A.G)) {
    case 8: if (staged(std::integral_constant<int, 8>{})) return; break;
    case 12: if (staged(std::integral_constant<int, 12>{})) return; break;
    case 16: if (staged(std::integral_constant<int, 16>{})) return; break;
    default: break;
  }
  switch (A.G) {
    case 1: k_residual<1><<<g, kBlock, 0, c->stream>>>(A, n, c->b.get(), c->x.get(), r, r32, c->ks.get(), c->partials.get()); break;
    case 2: k_residual<2><<<g, kBlock, 0, c->stream>>>(A, n, c->b.get(), c->x.get(), r, r32, c->ks.get(), c->partials.get()); break;
    default: k_residual<4><<<g, kBlock, 0, c->stream>>>(A, n, c->b.get(), c->x.get(), r, r32, c->ks.get(), c->partials.get()); break;
  }
}

static cudaError_t alloc_vectors(Context* c, int64_t n_pad, bool mixed) {
  cudaError_t e;
  DBuf<double>* v64[] = {&c->x, &c->r, &c->p, &c->q, &c->rh, &c->v, &c->s, &c->t, &c->ph, &c->sh};
  for (DBuf<double>* b : v64)
    if ((e = b->alloc(n_pad)) != cudaSuccess) return e;
  if (mixed) {
    DBuf<float>* v32[] = {&c->x32, &c->r32, &c->p32, &c->q32, &c->b32, &c->dinv32};
    for (DBuf<float>* b : v32)
      if ((e = b->alloc(n_pad)) != cudaSuccess) return e;
    if ((e = c->sval32.alloc(c->sell_len)) != cudaSuccess) return e;
  }
  if ((e = c->partials.alloc((size_t)c->sm_count * 8 * 4)) != cudaSuccess) return e;
  return c->ks.alloc(1);
}

// Builds the block-Jacobi inverse blocks of the current system (once per
// assembly); PBGPU_BREAKDOWN when a diagonal block is not positive definite.
static int build_block_jacobi(Context* c, const SellT<double>& A) {
  if (c->bj_ready) return PBGPU_OK;
  const int64_t n_blk = (c->n + kBjBlock - 1) / kBjBlock;
  PBGPU_CUDA(c, c->bjinv.alloc((size_t)n_blk * kBjBlock * kBjBlock));
  int* bad = reinterpret_cast<int*>(&c->ks_host->status);  // scratch flag in pinned memory
  Scratch<int> dbad(c, kScKrBad);
  PBGPU_CUDA(c, dbad.alloc(1));
  PBGPU_CUDA(c, cudaMemsetAsync(dbad.get(), 0, sizeof(int), c->stream));
  k_bj_setup<double, kBjBlock><<<grid_for(n_blk, 128), 128, 0, c->stream>>>(A, c->n, c->perm.get(), c->iperm.get(),
                                                                            c->bjinv.get(), dbad.get());
  PBGPU_LAUNCHED(c);
  PBGPU_CUDA(c, cudaMemcpyAsync(bad, dbad.get(), sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  if (*bad) return c->fail(PBGPU_BREAKDOWN, "solve: a block-Jacobi diagonal block is not positive definite");
  c->bj_ready = true;
  return PBGPU_OK;
}

int run_solve(Context* c, const pbgpu_solver_opts* o, pbgpu_solve_stats* st) {
  if (!c->have_system) return c->fail(PBGPU_ERR_STATE, "solve: assemble has not run");
  pbgpu_solver_opts opt;
  if (o)
    opt = *o;
  else
    pbgpu_default_solver_opts(&opt);
  if (opt.method != PBGPU_CG && opt.method != PBGPU_BICGSTAB && opt.method != PBGPU_CGS)
    return c->fail(PBGPU_ERR_ARG, "solve: unknown method");
  if (opt.conv_cond < 0 || opt.conv_cond > 2 || !(opt.tol_w >= 0))
    return c->fail(PBGPU_ERR_ARG, "solve: conv_cond must be 0, 1 or 2 and tol_w non-negative");
  const ConvRule rule{opt.conv_cond, opt.tol, opt.tol_w};
  if (opt.precond != PBGPU_PRECOND_NONE && opt.precond != PBGPU_PRECOND_JACOBI &&
      opt.precond != PBGPU_PRECOND_BLOCK_JACOBI)
    return c->fail(PBGPU_ERR_ARG, "solve: unknown preconditioner");
  if (!(opt.tol > 0) || opt.max_iter <= 0) return c->fail(PBGPU_ERR_ARG, "solve: tol and max_iter must be positive");
  if (opt.check_every <= 0) opt.check_every = 16;
  const bool mixed = opt.precision == PBGPU_MIXED;
  const int64_t n = c->n, n_pad = c->n_slices * c->C;
  PBGPU_CUDA(c, alloc_vectors(c, n_pad, mixed));
  // the scalars start from zero (tickets included) before any kernel of this
  // solve reads them: the mixed path's first residual runs before the first
  // Krylov run clears them itself
  PBGPU_CUDA(c, cudaMemsetAsync(c->ks.get(), 0, sizeof(KrylovScalars), c->stream));
  {
    const unsigned long long wns = (unsigned long long)(c->wait_s * 1e9);
    PBGPU_CUDA(c, cudaMemcpyAsync(&c->ks.get()->wait_ns, &wns, sizeof(wns), cudaMemcpyHostToDevice, c->stream));
  }
  PBGPU_CUDA(c, cudaEventRecord(c->ev0, c->stream));
  int iters = 0, status = PBGPU_OK, outer = 0;
  SellT<double> A64{c->slice_ptr.get(), c->slice_w.get(), c->scol.get(), c->sval.get(), n_pad, c->C, c->G};
  const bool bj = opt.precond == PBGPU_PRECOND_BLOCK_JACOBI;
  if (bj) {
    const int rc = build_block_jacobi(c, A64);
    if (rc != PBGPU_OK) return rc;
  }
  const double* diag64 = c->dinv.get();
  if (opt.precond == PBGPU_PRECOND_NONE) {
    PBGPU_CUDA(c, c->ones.alloc(n_pad));
    k_fill<double><<<grid_blocks(c, n_pad), kBlock, 0, c->stream>>>(n_pad, c->ones.get(), 1.0);
    PBGPU_LAUNCHED(c);
    diag64 = c->ones.get();
  } else if (bj) {
    diag64 = nullptr;
  }
  if (!mixed) {
    KrylovVecs<double> K{c->x.get(), c->r.get(), c->p.get(), c->q.get(), c->rh.get(), c->v.get(), c->s.get(),
                         c->t.get(), c->ph.get(), c->sh.get(), c->b.get(), diag64, A64};
    if (bj) {
      PBGPU_CUDA(c, c->z.alloc(n_pad));
      PBGPU_CUDA(c, cudaMemsetAsync(c->z.get(), 0, n_pad * sizeof(double), c->stream));
      K.z = c->z.get();
      K.bj = c->bjinv.get();
      K.iperm = c->iperm.get();
      K.n_nodes = n;
    }
    int rc = krylov<double>(c, opt.method, K, rule, opt.max_iter, opt.check_every, &iters, &status);
    if (rc != PBGPU_OK) return rc;
    if (status == PBGPU_TIMEOUT) return c->fail(PBGPU_TIMEOUT, "solve: SpMV copy wait timed out");
  } else {
    // FP32 copies of the matrix values and of 1/diag
    const int G = grid_blocks(c, c->sell_len);
    k_to_f32<<<G, kBlock, 0, c->stream>>>(c->sell_len, c->sval.get(), c->sval32.get());
    k_to_f32<<<grid_blocks(c, n_pad), kBlock, 0, c->stream>>>(n_pad, c->dinv.get(), c->dinv32.get());
    c->launches += 1;
    PBGPU_LAUNCHED(c);
    SellT<float> A32{c->slice_ptr.get(), c->slice_w.get(), c->scol.get(), c->sval32.get(), n_pad, c->C, c->G};
    PBGPU_CUDA(c, cudaMemsetAsync(c->x.get(), 0, n_pad * sizeof(double), c->stream));
    const int max_outer = opt.max_outer > 0 ? opt.max_outer : 50;
    const double inner = opt.inner_tol > 0 ? opt.inner_tol : 1e-5;
    // the fp32 inner solve keeps its own x (the correction d), r, p, q
    const float* diag32 = c->dinv32.get();
    if (opt.precond == PBGPU_PRECOND_NONE) {
      PBGPU_CUDA(c, c->ones32.alloc(n_pad));
      k_fill<float><<<grid_blocks(c, n_pad), kBlock, 0, c->stream>>>(n_pad, c->ones32.get(), 1.0f);
      PBGPU_LAUNCHED(c);
      diag32 = c->ones32.get();
    } else if (bj) {
      diag32 = nullptr;
    }
    KrylovVecs<float> K{c->x32.get(), c->r32.get(), c->p32.get(), c->q32.get(), nullptr, nullptr, nullptr,
                        nullptr, nullptr, nullptr, c->b32.get(), diag32, A32};
    if (bj) {
      PBGPU_CUDA(c, c->z32.alloc(n_pad));
      PBGPU_CUDA(c, cudaMemsetAsync(c->z32.get(), 0, n_pad * sizeof(float), c->stream));
      K.z = c->z32.get();
      K.bj = c->bjinv.get();
      K.iperm = c->iperm.get();
      K.n_nodes = n;
    }
    Scratch<float> rh32(c, kScKrRh32), v32(c, kScKrV32), s32(c, kScKrS32), t32(c, kScKrT32),
        ph32(c, kScKrPh32), sh32(c, kScKrSh32);
    if (opt.method != PBGPU_CG) {
      PBGPU_CUDA(c, rh32.alloc(n_pad));
      PBGPU_CUDA(c, v32.alloc(n_pad));
      PBGPU_CUDA(c, s32.alloc(n_pad));
      PBGPU_CUDA(c, t32.alloc(n_pad));
      PBGPU_CUDA(c, ph32.alloc(n_pad));
      PBGPU_CUDA(c, sh32.alloc(n_pad));
      K.rh = rh32.get();
      K.v = v32.get();
      K.s = s32.get();
      K.t = t32.get();
      K.ph = ph32.get();
      K.sh = sh32.get();
    }
    status = PBGPU_NOT_CONVERGED;
    const bool reliable = opt.method == PBGPU_CG && !bj;
    if (reliable) {
      // FP32 CG with reliable FP64 residual updates: one Krylov run
      k_to_f32<<<grid_blocks(c, n_pad), kBlock, 0, c->stream>>>(n_pad, c->b.get(), c->b32.get());
      PBGPU_LAUNCHED(c);
      K.A64 = &A64;
      K.b64 = c->b.get();
      K.x64 = c->x.get();
      K.n_rows = n;
      int it = 0, ist = 0;
      int rc = krylov<float>(c, opt.method, K, rule, opt.max_iter, opt.check_every, &it, &ist);
      if (rc != PBGPU_OK) return rc;
      if (ist == PBGPU_TIMEOUT) return c->fail(PBGPU_TIMEOUT, "solve: SpMV copy wait timed out");
      // a correction not yet folded in (the run stopped in the FP32 recursion)
      k_axpy_f32<<<grid_blocks(c, n_pad), kBlock, 0, c->stream>>>(n_pad, c->x.get(), c->x32.get());
      PBGPU_LAUNCHED(c);
      iters = it;
      outer = 1;
      status = ist;
    }
    for (outer = 1; !reliable && outer <= max_outer; ++outer) {
      // r = b - A x in fp64, handed to the inner solve in fp32
      launch_residual(c, A64, n, nullptr, c->b32.get());
      PBGPU_LAUNCHED(c);
      PBGPU_CUDA(c, cudaMemcpyAsync(c->ks_host, c->ks.get(), sizeof(KrylovScalars), cudaMemcpyDeviceToHost, c->stream));
      PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
      if (c->ks_host->status == PBGPU_TIMEOUT) return c->fail(PBGPU_TIMEOUT, "solve: SpMV copy wait timed out");
      const double rr = c->ks_host->rr, bb = c->ks_host->bb;
      if (!std::isfinite(rr)) {
        status = PBGPU_BREAKDOWN;
        break;
      }
      const bool met = rule.mode == 2 ? c->ks_host->r1 <= rule.tol_w * c->ks_host->b1 + rule.tol
                                      : rr <= opt.tol * opt.tol * bb;
      if (met) {
        status = PBGPU_OK;
        break;
      }
      // inner tolerance: reduce the residual by `inner`, never below what fp32 can resolve;
      // an inner solve that stagnates in fp32 (CGS, BiCGStab) is cut off and its
      // correction used all the same, the fp64 residual decides
      int it = 0, ist = 0;
      const int left = std::min(opt.max_iter - iters, std::max(256, opt.max_iter / 8));
      if (left <= 0) break;
      int rc = krylov<float>(c, opt.method, K, ConvRule{0, inner, 1.0}, left, opt.check_every, &it, &ist);
      if (rc != PBGPU_OK) return rc;
      if (ist == PBGPU_TIMEOUT) return c->fail(PBGPU_TIMEOUT, "solve: SpMV copy wait timed out");
      iters += it;
      if (ist == PBGPU_BREAKDOWN && it == 0) {
        status = PBGPU_BREAKDOWN;
        break;
      }
      k_axpy_f32<<<grid_blocks(c, n_pad), kBlock, 0, c->stream>>>(n_pad, c->x.get(), c->x32.get());
      PBGPU_LAUNCHED(c);
    }
  }
  PBGPU_CUDA(c, cudaEventRecord(c->ev1, c->stream));
  // true residual in fp64
  launch_residual(c, A64, n, nullptr, nullptr);
  PBGPU_LAUNCHED(c);
  PBGPU_CUDA(c, cudaMemcpyAsync(c->ks_host, c->ks.get(), sizeof(KrylovScalars), cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, c->phi.alloc(n));
  k_gather_phi<<<grid_for(n, 256), 256, 0, c->stream>>>(n, c->iperm.get(), c->x.get(), c->phi.get());
  PBGPU_LAUNCHED(c);
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  float ms = 0;
  PBGPU_CUDA(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  if (c->ks_host->status == PBGPU_TIMEOUT) return c->fail(PBGPU_TIMEOUT, "solve: SpMV copy wait timed out");
  const double rel = c->ks_host->bb > 0 ? std::sqrt(c->ks_host->rr / c->ks_host->bb) : 0.0;
  if (st) {
    st->status = status;
    st->iterations = iters;
    st->outer = outer;
    st->rel_residual = rel;
    st->device_ms = ms;
  }
  c->have_phi = true;
  if (status == PBGPU_NOT_CONVERGED) return c->fail(status, "solve: iteration limit reached");
  if (status == PBGPU_BREAKDOWN) return c->fail(status, "solve: Krylov breakdown or non-finite value");
  return PBGPU_OK;
}

}  // namespace pbgpu
