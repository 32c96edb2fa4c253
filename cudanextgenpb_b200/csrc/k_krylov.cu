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

#include <cmath>

#include "pbgpu_internal.cuh"

namespace pbgpu {

constexpr int kBlock = 256;
// resident blocks per SM the SpMV kernels are compiled for (registers <= 65536 / (256 * 5))
constexpr int kSpmvMinBlocks = 5;

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

// y_p = sum_j A(p, j) x_j for SELL row p.  Element j of row p sits at
// slice_ptr[s] + (j / G) G C + lane G + j % G, so for every G a warp's loads
// of one column group are contiguous.
template <typename T, int G>
__device__ __forceinline__ T sell_row(const SellT<T>& A, int64_t p, const T* __restrict__ x) {
  const int64_t s = p / A.C;
  const int lane = (int)(p - s * A.C);
  const int W = A.slice_w[s];
  T acc = 0;
  if constexpr (G == 1) {
    const int64_t base = A.slice_ptr[s] + lane;
    const int64_t stride = A.C;
#pragma unroll 4
    for (int j = 0; j < W; ++j) {
      const int64_t k = base + j * stride;
      acc += __ldcs(A.sval + k) * x[__ldcs(A.scol + k)];
    }
  } else if constexpr (G == 2) {
    const int64_t base = A.slice_ptr[s] + 2 * lane;
    const int64_t stride = 2 * (int64_t)A.C;
#pragma unroll 2
    for (int g = 0; g < (W >> 1); ++g) {
      const int64_t k = base + g * stride;
      const int2 c = __ldcs(reinterpret_cast<const int2*>(A.scol + k));
      const typename V2<T>::t v = __ldcs(reinterpret_cast<const typename V2<T>::t*>(A.sval + k));
      acc += v.x * x[c.x];
      acc += v.y * x[c.y];
    }
  } else {
    const int64_t base = A.slice_ptr[s] + 4 * lane;
    const int64_t stride = 4 * (int64_t)A.C;
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
  }
  return acc;
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

// ---------------------------------------------------------------------------
// CG (Jacobi preconditioner), templated on the storage precision.
template <typename T>
__global__ void k_cg_init(int64_t n, const T* __restrict__ b, const T* __restrict__ dinv, T* __restrict__ x,
                          T* __restrict__ r, T* __restrict__ p, KrylovScalars* ks, double* partials, double tol) {
  double v[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T bi = b[i];
    const T zi = dinv[i] * bi;
    x[i] = 0;
    r[i] = bi;
    p[i] = zi;
    v[0] += (double)bi * (double)zi;
    v[1] += (double)bi * (double)bi;
  }
  if (grid_sum<2>(v, partials, &ks->ticket[0]) && threadIdx.x == 0) {
    ks->rz = v[0];
    ks->bb = v[1];
    ks->tol2 = tol * tol * v[1];
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
__global__ void __launch_bounds__(kBlock, kSpmvMinBlocks) k_cg_spmv(SellT<T> A, const T* __restrict__ p, T* __restrict__ q, KrylovScalars* ks, double* partials) {
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
                            const T* __restrict__ q, const T* __restrict__ dinv, KrylovScalars* ks, double* partials) {
  if (ks->done) return;
  const T alpha = (T)ks->alpha;
  double v[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    const T ri = r[i] - alpha * q[i];
    r[i] = ri;
    v[0] += (double)ri * (double)(dinv[i] * ri);
    v[1] += (double)ri * (double)ri;
  }
  if (grid_sum<2>(v, partials, &ks->ticket[2]) && threadIdx.x == 0) {
    ks->iter += 1;
    ks->rr = v[1];
    if (!finite(v[0]) || !finite(v[1])) {
      ks->status = PBGPU_BREAKDOWN;
      ks->done = 1;
    } else if (v[1] <= ks->tol2) {
      ks->done = 1;
    } else if (ks->iter >= ks->max_iter) {
      ks->status = PBGPU_NOT_CONVERGED;
      ks->done = 1;
    } else {
      ks->beta = v[0] / ks->rz;
      ks->rz = v[0];
    }
  }
}

template <typename T>
__global__ void k_cg_pupdate(int64_t n, T* __restrict__ p, const T* __restrict__ r, const T* __restrict__ dinv,
                             const KrylovScalars* ks) {
  if (ks->done) return;
  const T beta = (T)ks->beta;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = dinv[i] * r[i] + beta * p[i];
}

// ---------------------------------------------------------------------------
// BiCGStab (right Jacobi preconditioning), templated on the storage precision.
template <typename T>
__global__ void k_bicg_init(int64_t n, const T* __restrict__ b, T* __restrict__ x, T* __restrict__ r,
                            T* __restrict__ rh, T* __restrict__ p, T* __restrict__ v, KrylovScalars* ks,
                            double* partials, double tol) {
  double s[1] = {0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T bi = b[i];
    x[i] = 0;
    r[i] = bi;
    rh[i] = bi;
    p[i] = 0;
    v[i] = 0;
    s[0] += (double)bi * (double)bi;
  }
  if (grid_sum<1>(s, partials, &ks->ticket[0]) && threadIdx.x == 0) {
    ks->bb = s[0];
    ks->tol2 = tol * tol * s[0];
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
    ph[i] = dinv[i] * pi;
  }
}

// v = A ph;  alpha = rho_new / (rh, v)
template <typename T, int G>
__global__ void __launch_bounds__(kBlock, kSpmvMinBlocks) k_bicg_v(SellT<T> A, const T* __restrict__ ph, T* __restrict__ v, const T* __restrict__ rh,
                         KrylovScalars* ks, double* partials) {
  if (ks->done) return;
  double s[1] = {0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < A.n_pad; i += (int64_t)gridDim.x * blockDim.x) {
    const T y = sell_row<T, G>(A, i, ph);
    v[i] = y;
    s[0] += (double)rh[i] * (double)y;
  }
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
  double a[1] = {0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T si = r[i] - alpha * v[i];
    s[i] = si;
    sh[i] = dinv[i] * si;
    a[0] += (double)si * (double)si;
  }
  if (grid_sum<1>(a, partials, &ks->ticket[2]) && threadIdx.x == 0) {
    ks->ss = a[0];
    ks->s_conv = a[0] <= ks->tol2;
  }
}

// t = A sh;  omega = (t, s) / (t, t)
template <typename T, int G>
__global__ void __launch_bounds__(kBlock, kSpmvMinBlocks) k_bicg_t(SellT<T> A, const T* __restrict__ sh, T* __restrict__ t, const T* __restrict__ s,
                         KrylovScalars* ks, double* partials) {
  if (ks->done || ks->s_conv) return;
  double a[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < A.n_pad; i += (int64_t)gridDim.x * blockDim.x) {
    const T y = sell_row<T, G>(A, i, sh);
    t[i] = y;
    a[0] += (double)y * (double)s[i];
    a[1] += (double)y * (double)y;
  }
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
  double a[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] += alpha * ph[i] + omega * sh[i];
    const T ri = s[i] - omega * t[i];
    r[i] = ri;
    a[0] += (double)ri * (double)ri;
    a[1] += (double)rh[i] * (double)ri;
  }
  if (grid_sum<2>(a, partials, &ks->ticket[4]) && threadIdx.x == 0) {
    ks->iter += 1;
    ks->rr = a[0];
    const double rho_new = a[1];
    if (!finite(a[0]) || !finite(a[1])) {
      ks->status = PBGPU_BREAKDOWN;
      ks->done = 1;
    } else if (a[0] <= ks->tol2) {
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
__global__ void __launch_bounds__(kBlock, kSpmvMinBlocks) k_residual(SellT<double> A, int64_t n, const double* __restrict__ b, const double* __restrict__ x,
                           double* __restrict__ r, float* __restrict__ r32, KrylovScalars* ks, double* partials) {
  double a[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < A.n_pad; i += (int64_t)gridDim.x * blockDim.x) {
    const double ri = i < n ? b[i] - sell_row<double, G>(A, i, x) : 0.0;
    if (r) r[i] = ri;
    if (r32) r32[i] = (float)ri;
    a[0] += ri * ri;
    a[1] += i < n ? b[i] * b[i] : 0.0;
  }
  if (grid_sum<2>(a, partials, &ks->ticket[5]) && threadIdx.x == 0) {
    ks->rr = a[0];
    ks->bb = a[1];
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

template <typename T>
struct KrylovVecs {
  T *x, *r, *p, *q, *rh, *v, *s, *t, *ph, *sh;
  const T *b, *dinv;
  SellT<T> A;
};

// Run one Krylov solve on (A, b) to relative tolerance tol; x0 = 0.  GW is the
// SELL column-group width of A.
template <typename T, int GW>
static int krylov_g(Context* c, int method, const KrylovVecs<T>& K, double tol, int max_iter, int check_every,
                    int* iters, int* status) {
  const int64_t n = K.A.n_pad;
  const int G = grid_blocks(c, n);
  KrylovScalars* ks = c->ks.get();
  double* part = c->partials.get();
  PBGPU_CUDA(c, cudaMemsetAsync(ks, 0, sizeof(KrylovScalars), c->stream));
  int mi = max_iter;
  PBGPU_CUDA(c, cudaMemcpyAsync(&ks->max_iter, &mi, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  if (method == PBGPU_CG)
    k_cg_init<T><<<G, kBlock, 0, c->stream>>>(n, K.b, K.dinv, K.x, K.r, K.p, ks, part, tol);
  else
    k_bicg_init<T><<<G, kBlock, 0, c->stream>>>(n, K.b, K.x, K.r, K.rh, K.p, K.v, ks, part, tol);
  PBGPU_CUDA(c, cudaGetLastError());
  c->launches += 1;
  // With profiling on, events recorded around every SpMV launch become event
  // nodes of the graph; the elapsed times of the launches that did work are
  // summed after each chunk.
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
  for (int k = 0; k < check_every; ++k) {
    if (method == PBGPU_CG) {
      mark(k, 0, 0);
      k_cg_spmv<T, GW><<<G, kBlock, 0, c->stream>>>(K.A, K.p, K.q, ks, part);
      mark(k, 0, 1);
      k_cg_update<T><<<G, kBlock, 0, c->stream>>>(n, K.x, K.r, K.p, K.q, K.dinv, ks, part);
      k_cg_pupdate<T><<<G, kBlock, 0, c->stream>>>(n, K.p, K.r, K.dinv, ks);
    } else {
      k_bicg_p<T><<<G, kBlock, 0, c->stream>>>(n, K.p, K.ph, K.r, K.v, K.dinv, ks);
      mark(k, 0, 0);
      k_bicg_v<T, GW><<<G, kBlock, 0, c->stream>>>(K.A, K.ph, K.v, K.rh, ks, part);
      mark(k, 0, 1);
      k_bicg_s<T><<<G, kBlock, 0, c->stream>>>(n, K.r, K.v, K.s, K.sh, K.dinv, ks, part);
      mark(k, 1, 0);
      k_bicg_t<T, GW><<<G, kBlock, 0, c->stream>>>(K.A, K.sh, K.t, K.s, ks, part);
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
  const int kernels_per_chunk = (method == PBGPU_CG ? 3 : 5) * check_every;
  int rc = PBGPU_OK;
  const int max_chunks = max_iter / check_every + 2;
  int prev_iter = 0;
  for (int chunk = 0; chunk < max_chunks; ++chunk) {
    ce = cudaGraphLaunch(exec, c->stream);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(c->ks_host, ks, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, c->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(c->stream);
    if (ce != cudaSuccess) {
      rc = cuda_fail(c, ce, "krylov chunk");
      break;
    }
    c->launches += kernels_per_chunk;
    const int now = c->ks_host->iter;
    if (c->profiling) {
      // iteration k of this chunk did its SpMV(s) when it is below the count
      // of completed iterations; the t-SpMV of a BiCGStab iteration that
      // stopped on ||s|| did not run
      for (int k = 0; k < check_every && prev_iter + k < now; ++k)
        for (int w = 0; w < spmv_per_it; ++w) {
          if (w == 1 && prev_iter + k == now - 1 && c->ks_host->s_conv) continue;
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
    if (c->ks_host->done) break;
  }
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
static int krylov(Context* c, int method, const KrylovVecs<T>& K, double tol, int max_iter, int check_every,
                  int* iters, int* status) {
  switch (K.A.G) {
    case 1: return krylov_g<T, 1>(c, method, K, tol, max_iter, check_every, iters, status);
    case 2: return krylov_g<T, 2>(c, method, K, tol, max_iter, check_every, iters, status);
    default: return krylov_g<T, 4>(c, method, K, tol, max_iter, check_every, iters, status);
  }
}

// r = b - A x (fp64); optional fp64 / fp32 copies of r; norms into ks
static void launch_residual(Context* c, const SellT<double>& A, int64_t n, double* r, float* r32) {
  const int g = grid_blocks(c, A.n_pad);
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

int run_solve(Context* c, const pbgpu_solver_opts* o, pbgpu_solve_stats* st) {
  if (!c->have_system) return c->fail(PBGPU_ERR_STATE, "solve: assemble has not run");
  pbgpu_solver_opts opt;
  if (o)
    opt = *o;
  else
    pbgpu_default_solver_opts(&opt);
  if (opt.method != PBGPU_CG && opt.method != PBGPU_BICGSTAB) return c->fail(PBGPU_ERR_ARG, "solve: unknown method");
  if (!(opt.tol > 0) || opt.max_iter <= 0) return c->fail(PBGPU_ERR_ARG, "solve: tol and max_iter must be positive");
  if (opt.check_every <= 0) opt.check_every = 16;
  const bool mixed = opt.precision == PBGPU_MIXED;
  const int64_t n = c->n, n_pad = c->n_slices * c->C;
  PBGPU_CUDA(c, alloc_vectors(c, n_pad, mixed));
  PBGPU_CUDA(c, cudaEventRecord(c->ev0, c->stream));
  int iters = 0, status = PBGPU_OK, outer = 0;
  SellT<double> A64{c->slice_ptr.get(), c->slice_w.get(), c->scol.get(), c->sval.get(), n_pad, c->C, c->G};
  if (!mixed) {
    KrylovVecs<double> K{c->x.get(), c->r.get(), c->p.get(), c->q.get(), c->rh.get(), c->v.get(), c->s.get(),
                         c->t.get(), c->ph.get(), c->sh.get(), c->b.get(), c->dinv.get(), A64};
    int rc = krylov<double>(c, opt.method, K, opt.tol, opt.max_iter, opt.check_every, &iters, &status);
    if (rc != PBGPU_OK) return rc;
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
    KrylovVecs<float> K{c->x32.get(), c->r32.get(), c->p32.get(), c->q32.get(), nullptr, nullptr, nullptr,
                        nullptr, nullptr, nullptr, c->b32.get(), c->dinv32.get(), A32};
    DBuf<float> rh32, v32, s32, t32, ph32, sh32;
    if (opt.method == PBGPU_BICGSTAB) {
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
    for (outer = 1; outer <= max_outer; ++outer) {
      // r = b - A x in fp64, handed to the inner solve in fp32
      launch_residual(c, A64, n, nullptr, c->b32.get());
      PBGPU_LAUNCHED(c);
      PBGPU_CUDA(c, cudaMemcpyAsync(c->ks_host, c->ks.get(), sizeof(KrylovScalars), cudaMemcpyDeviceToHost, c->stream));
      PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
      const double rr = c->ks_host->rr, bb = c->ks_host->bb;
      if (!std::isfinite(rr)) {
        status = PBGPU_BREAKDOWN;
        break;
      }
      if (rr <= opt.tol * opt.tol * bb) {
        status = PBGPU_OK;
        break;
      }
      // inner tolerance: reduce the residual by `inner`, never below what fp32 can resolve
      int it = 0, ist = 0;
      const int left = opt.max_iter - iters;
      if (left <= 0) break;
      int rc = krylov<float>(c, opt.method, K, inner, left, opt.check_every, &it, &ist);
      if (rc != PBGPU_OK) return rc;
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
