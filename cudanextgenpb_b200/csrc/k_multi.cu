// Many right-hand sides on one assembled system: the same molecule with k
// charge vectors (e.g. titration states flipping charges on a few sites).  No
// counterpart in the reference, which solves one charge set per run
// (lis_compute_electric_potential, src/pb_class.cpp:2244-2329).
//
// The matrix does not depend on the charges, so it is assembled once; each
// charge vector gets its density map and right-hand side (run_rhs), and the k
// systems A x_j = b_j are solved by k independent Jacobi-CG recurrences that
// share every SpMV: the vectors are stored row-major with the k columns of a
// row contiguous (padded to a multiple of 32), a warp walks rows with its
// lanes over the columns, and each matrix row is read once for all columns
// while the gathered x rows are contiguous 256-byte segments.  Per-column
// scalars live on the device; per-column reductions are deterministic (fixed
// block order); columns that converged stop updating.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "pbgpu_internal.cuh"
#include "sell.cuh"

namespace pbgpu {

constexpr int kMrWarps = kBlock / 32;

struct MrScalars {
  double* rz;      // kp
  double* alpha;
  double* beta;
  double* tol2;
  double* rr;
  double* bb;
  int* done;       // kp
  int* iters;      // kp
  int* status;     // kp
  int* all_done;   // 1
  unsigned* ticket;  // 4
};

// Per-column block sums of the KT values each lane holds (columns lane +
// 32 t); after the call thread c < kp of the block holds column c's block
// sum of value set m in out[m].
template <int KT, int M>
__device__ __forceinline__ void mr_block_sum(double (&v)[M][KT], double (&out)[M]) {
  constexpr int KP = 32 * KT;
  __shared__ double sh[M][kMrWarps][KP];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int m = 0; m < M; ++m)
#pragma unroll
    for (int t = 0; t < KT; ++t) sh[m][w][lane + 32 * t] = v[m][t];
  __syncthreads();
#pragma unroll
  for (int m = 0; m < M; ++m) {
    double a = 0.0;
    if (threadIdx.x < KP)
      for (int ww = 0; ww < kMrWarps; ++ww) a += sh[m][ww][threadIdx.x];
    out[m] = a;
  }
  __syncthreads();
}

// Block partials -> grid sums per column in the last block (fixed order).
// Returns true in the last block; thread c < kp then holds column c's sums.
template <int KT, int M>
__device__ __forceinline__ bool mr_grid_sum(double (&v)[M][KT], double* partials, unsigned* ticket,
                                            double (&out)[M]) {
  constexpr int KP = 32 * KT;
  mr_block_sum<KT, M>(v, out);
  if (threadIdx.x < KP)
#pragma unroll
    for (int m = 0; m < M; ++m) partials[((size_t)blockIdx.x * M + m) * KP + threadIdx.x] = out[m];
  __threadfence();
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return false;
  __threadfence();
  if (threadIdx.x < KP)
#pragma unroll
    for (int m = 0; m < M; ++m) {
      double a = 0.0;
      for (unsigned b = 0; b < gridDim.x; ++b) a += __ldcg(partials + ((size_t)b * M + m) * KP + threadIdx.x);
      out[m] = a;
    }
  if (threadIdx.x == 0) *ticket = 0;
  return true;
}

// the entries of SELL row p (G = 4 layout with tail), fn(col, val) in order
template <typename Fn>
__device__ __forceinline__ void mr_row(const SellT<double>& A, int64_t p, Fn&& fn) {
  const int lane = threadIdx.x & 31;
  const int64_t s = p / A.C;
  const int W = A.slice_w[s];
  const int64_t sb = A.slice_ptr[s];
  const int rl = (int)(p - s * A.C);
  for (int e0 = 0; e0 < W; e0 += 32) {
    int32_t col = 0;
    double val = 0.0;
    if (e0 + lane < W) {
      const int64_t k = sell_elem(sb, W, A.C, A.G, rl, e0 + lane);
      col = __ldcs(A.scol + k);
      val = __ldcs(A.sval + k);
    }
    const int ne = min(32, W - e0);
    for (int e = 0; e < ne; ++e) fn(__shfl_sync(0xffffffffu, col, e), __shfl_sync(0xffffffffu, val, e));
  }
}

template <int KT>
__global__ void __launch_bounds__(kBlock) k_mr_init(int64_t n_pad, const double* __restrict__ B,
                                                    const double* __restrict__ dinv, double* __restrict__ X,
                                                    double* __restrict__ R, double* __restrict__ P, MrScalars S,
                                                    double* partials, double tol) {
  constexpr int KP = 32 * KT;
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  double v[2][KT] = {};
  for (int64_t i = w0; i < n_pad; i += nw) {
    const double d = dinv[i];
#pragma unroll
    for (int t = 0; t < KT; ++t) {
      const int64_t e = i * KP + lane + 32 * t;
      const double b = B[e];
      X[e] = 0.0;
      R[e] = b;
      P[e] = d * b;
      v[0][t] += b * d * b;
      v[1][t] += b * b;
    }
  }
  double out[2];
  if (mr_grid_sum<KT, 2>(v, partials, &S.ticket[0], out) && threadIdx.x < KP) {
    const int c = threadIdx.x;
    S.rz[c] = out[0];
    S.bb[c] = out[1];
    S.tol2[c] = tol * tol * out[1];
    S.iters[c] = 0;
    S.status[c] = PBGPU_OK;
    S.done[c] = out[1] == 0.0;
    if (c == 0) *S.all_done = 0;
  }
}

// Q = A P; per column p.q and alpha
template <int KT>
__global__ void __launch_bounds__(kBlock) k_mr_spmm(SellT<double> A, const double* P, double* __restrict__ Q,
                                                    MrScalars S, double* partials) {
  constexpr int KP = 32 * KT;
  if (*S.all_done) return;
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  double v[1][KT] = {};
  for (int64_t i = w0; i < A.n_pad; i += nw) {
    double acc[KT] = {};
    mr_row(A, i, [&](int32_t c, double a) {
#pragma unroll
      for (int t = 0; t < KT; ++t) acc[t] += a * P[(int64_t)c * KP + lane + 32 * t];
    });
#pragma unroll
    for (int t = 0; t < KT; ++t) {
      const int64_t e = i * KP + lane + 32 * t;
      Q[e] = acc[t];
      v[0][t] += P[e] * acc[t];
    }
  }
  double out[1];
  if (mr_grid_sum<KT, 1>(v, partials, &S.ticket[1], out) && threadIdx.x < KP) {
    const int c = threadIdx.x;
    if (!S.done[c]) {
      const double a = S.rz[c] / out[0];
      if (!(out[0] > 0.0) || !isfinite(a)) {
        S.status[c] = PBGPU_BREAKDOWN;
        S.done[c] = 1;
        S.alpha[c] = 0.0;
      } else {
        S.alpha[c] = a;
      }
    } else {
      S.alpha[c] = 0.0;
    }
  }
}

// x += alpha p; r -= alpha q; per column (r, z), (r, r); convergence; beta
template <int KT>
__global__ void __launch_bounds__(kBlock) k_mr_update(int64_t n_pad, double* __restrict__ X, double* __restrict__ R,
                                                      const double* __restrict__ P, const double* __restrict__ Q,
                                                      const double* __restrict__ dinv, MrScalars S, double* partials,
                                                      int max_iter) {
  constexpr int KP = 32 * KT;
  if (*S.all_done) return;
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  double al[KT];
#pragma unroll
  for (int t = 0; t < KT; ++t) al[t] = S.alpha[lane + 32 * t];  // 0 for finished columns
  double v[2][KT] = {};
  for (int64_t i = w0; i < n_pad; i += nw) {
    const double d = dinv[i];
#pragma unroll
    for (int t = 0; t < KT; ++t) {
      const int64_t e = i * KP + lane + 32 * t;
      X[e] += al[t] * P[e];
      const double r = R[e] - al[t] * Q[e];
      R[e] = r;
      v[0][t] += r * d * r;
      v[1][t] += r * r;
    }
  }
  double out[2];
  __shared__ int any_open;
  if (threadIdx.x == 0) any_open = 0;
  if (mr_grid_sum<KT, 2>(v, partials, &S.ticket[2], out)) {
    if (threadIdx.x < KP) {
      const int c = threadIdx.x;
      if (!S.done[c]) {
        S.iters[c] += 1;
        S.rr[c] = out[1];
        if (!isfinite(out[0]) || !isfinite(out[1])) {
          S.status[c] = PBGPU_BREAKDOWN;
          S.done[c] = 1;
        } else if (out[1] <= S.tol2[c]) {
          S.done[c] = 1;
        } else if (S.iters[c] >= max_iter) {
          S.status[c] = PBGPU_NOT_CONVERGED;
          S.done[c] = 1;
        } else {
          S.beta[c] = out[0] / S.rz[c];
          S.rz[c] = out[0];
        }
      }
      if (!S.done[c]) atomicOr(&any_open, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) *S.all_done = any_open ? 0 : 1;
  }
}

// p = z + beta p for the open columns
template <int KT>
__global__ void __launch_bounds__(kBlock) k_mr_pupdate(int64_t n_pad, double* __restrict__ P,
                                                       const double* __restrict__ R, const double* __restrict__ dinv,
                                                       MrScalars S) {
  constexpr int KP = 32 * KT;
  if (*S.all_done) return;
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  double be[KT];
  bool open[KT];
#pragma unroll
  for (int t = 0; t < KT; ++t) {
    open[t] = !S.done[lane + 32 * t];
    be[t] = S.beta[lane + 32 * t];
  }
  for (int64_t i = w0; i < n_pad; i += nw) {
    const double d = dinv[i];
#pragma unroll
    for (int t = 0; t < KT; ++t) {
      const int64_t e = i * KP + lane + 32 * t;
      if (open[t]) P[e] = d * R[e] + be[t] * P[e];
    }
  }
}

__global__ void k_mr_put(int64_t n_pad, int kp, int j, const double* __restrict__ b, double* __restrict__ B) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n_pad) B[i * kp + j] = b[i];
}

__global__ void k_mr_get(int64_t n_pad, int kp, int j, const double* __restrict__ X, double* __restrict__ x) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n_pad) x[i] = X[i * kp + j];
}

__global__ void k_mr_set_charges(int64_t na, const double* __restrict__ q, double4* __restrict__ atoms) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < na) atoms[i].w = q[i];
}

__global__ void k_mr_gather_phi(int64_t n, const int32_t* __restrict__ iperm, const double* __restrict__ x,
                                double* __restrict__ phi) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) phi[i] = x[iperm[i]];
}

template <int KT>
static int mr_solve(Context* c, int k, const pbgpu_solver_opts& o, double* X, double* R, double* P, double* Q,
                    const double* B, MrScalars S, double* part, std::vector<int>& iters, std::vector<int>& status,
                    std::vector<double>& rel, float* ms) {
  constexpr int KP = 32 * KT;
  const int64_t n_pad = c->n_slices * c->C;
  const int G = (int)std::min<int64_t>((n_pad + kMrWarps - 1) / kMrWarps, (int64_t)c->sm_count * 8);
  const SellT<double> A{c->slice_ptr.get(), c->slice_w.get(), c->scol.get(), c->sval.get(), n_pad, c->C, c->G};
  PBGPU_CUDA(c, cudaMemsetAsync(S.ticket, 0, 4 * sizeof(unsigned), c->stream));
  PBGPU_CUDA(c, cudaEventRecord(c->ev0, c->stream));
  k_mr_init<KT><<<G, kBlock, 0, c->stream>>>(n_pad, B, c->dinv.get(), X, R, P, S, part, o.tol);
  PBGPU_LAUNCHED(c);
  // padded columns (zero right-hand sides) are done from the start
  const int chunk = o.check_every > 0 ? o.check_every : 16;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  PBGPU_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  for (int it = 0; it < chunk; ++it) {
    k_mr_spmm<KT><<<G, kBlock, 0, c->stream>>>(A, P, Q, S, part);
    k_mr_update<KT><<<G, kBlock, 0, c->stream>>>(n_pad, X, R, P, Q, c->dinv.get(), S, part, o.max_iter);
    k_mr_pupdate<KT><<<G, kBlock, 0, c->stream>>>(n_pad, P, R, c->dinv.get(), S);
  }
  cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
  if (e != cudaSuccess) return cuda_fail(c, e, "multi-rhs capture");
  e = cudaGraphInstantiate(&exec, graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    return cuda_fail(c, e, "multi-rhs graph");
  }
  int all = 0;
  int rc = PBGPU_OK;
  for (int64_t done = 0; done <= (int64_t)o.max_iter + chunk && !all; done += chunk) {
    e = cudaGraphLaunch(exec, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&all, S.all_done, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
      rc = cuda_fail(c, e, "multi-rhs chunk");
      break;
    }
    c->launches += 3 * chunk;
  }
  cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  if (rc != PBGPU_OK) return rc;
  PBGPU_CUDA(c, cudaEventRecord(c->ev1, c->stream));
  std::vector<int> hi(KP), hs(KP), hd(KP);
  std::vector<double> hrr(KP), hbb(KP);
  PBGPU_CUDA(c, cudaMemcpyAsync(hi.data(), S.iters, KP * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaMemcpyAsync(hs.data(), S.status, KP * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaMemcpyAsync(hd.data(), S.done, KP * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaMemcpyAsync(hrr.data(), S.rr, KP * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaMemcpyAsync(hbb.data(), S.bb, KP * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  PBGPU_CUDA(c, cudaEventElapsedTime(ms, c->ev0, c->ev1));
  for (int j = 0; j < k; ++j) {
    iters[j] = hi[j];
    status[j] = hd[j] ? hs[j] : PBGPU_NOT_CONVERGED;
    rel[j] = hbb[j] > 0 ? std::sqrt(hrr[j] / hbb[j]) : 0.0;
  }
  return PBGPU_OK;
}

int run_solve_charges(Context* c, int k, const double* charges, const pbgpu_solver_opts* opts, int fast,
                      pbgpu_energy_out* energies, pbgpu_solve_stats* stats) {
  if (!c->have_system) return c->fail(PBGPU_ERR_STATE, "solve_charges: assemble has not run");
  if (k <= 0 || k > 64 || !charges) return c->fail(PBGPU_ERR_ARG, "solve_charges: 1 <= k <= 64 charge vectors");
  pbgpu_solver_opts o;
  if (opts)
    o = *opts;
  else
    pbgpu_default_solver_opts(&o);
  if (o.method != PBGPU_CG || o.precond != PBGPU_PRECOND_JACOBI || o.precision != PBGPU_FP64 || o.conv_cond == 2)
    return c->fail(PBGPU_ERR_ARG, "solve_charges: FP64 Jacobi CG with a relative 2-norm tolerance");
  if (!(o.tol > 0) || o.max_iter <= 0) return c->fail(PBGPU_ERR_ARG, "solve_charges: tol and max_iter must be positive");
  const int KT = k <= 32 ? 1 : 2;
  const int kp = 32 * KT;
  const int64_t n_pad = c->n_slices * c->C, na = c->na;
  const size_t vec = (size_t)n_pad * kp;
  PBGPU_CUDA(c, c->mr_b.alloc(vec));
  PBGPU_CUDA(c, c->mr_x.alloc(vec));
  PBGPU_CUDA(c, c->mr_r.alloc(vec));
  PBGPU_CUDA(c, c->mr_p.alloc(vec));
  PBGPU_CUDA(c, c->mr_q.alloc(vec));
  PBGPU_CUDA(c, c->mr_scal.alloc(6 * kp));
  PBGPU_CUDA(c, c->mr_int.alloc(3 * kp + 1 + 4));
  PBGPU_CUDA(c, c->mr_part.alloc((size_t)c->sm_count * 8 * 2 * kp));
  PBGPU_CUDA(c, c->mr_q_dev.alloc(na > 0 ? na : 1));
  PBGPU_CUDA(c, cudaMemsetAsync(c->mr_b.get(), 0, vec * sizeof(double), c->stream));
  // the context's own charges, restored at the end
  std::vector<double4> atoms(na > 0 ? na : 1);
  if (na > 0)
    PBGPU_CUDA(c, cudaMemcpyAsync(atoms.data(), c->atoms.get(), na * sizeof(double4), cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  std::vector<double> q0(na);
  for (int64_t i = 0; i < na; ++i) q0[i] = atoms[i].w;
  auto set_charges = [&](const double* q) -> int {
    if (na == 0) return PBGPU_OK;
    PBGPU_CUDA(c, cudaMemcpyAsync(c->mr_q_dev.get(), q, na * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    k_mr_set_charges<<<grid_for(na, 256), 256, 0, c->stream>>>(na, c->mr_q_dev.get(), c->atoms.get());
    PBGPU_LAUNCHED(c);
    PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    return PBGPU_OK;
  };
  int st;
  for (int j = 0; j < k; ++j) {
    if ((st = set_charges(charges + (size_t)j * na)) != PBGPU_OK) return st;
    if ((st = run_density(c)) != PBGPU_OK) return st;
    if ((st = run_rhs(c)) != PBGPU_OK) return st;
    k_mr_put<<<grid_for(n_pad, 256), 256, 0, c->stream>>>(n_pad, kp, j, c->b.get(), c->mr_b.get());
    PBGPU_LAUNCHED(c);
  }
  double* sc = c->mr_scal.get();
  int* si = c->mr_int.get();
  MrScalars S{sc, sc + kp, sc + 2 * kp, sc + 3 * kp, sc + 4 * kp, sc + 5 * kp,
              si, si + kp, si + 2 * kp, si + 3 * kp, reinterpret_cast<unsigned*>(si + 3 * kp + 1)};
  std::vector<int> iters(k), status(k);
  std::vector<double> rel(k);
  float ms = 0.f;
  st = KT == 1 ? mr_solve<1>(c, k, o, c->mr_x.get(), c->mr_r.get(), c->mr_p.get(), c->mr_q.get(), c->mr_b.get(), S,
                             c->mr_part.get(), iters, status, rel, &ms)
               : mr_solve<2>(c, k, o, c->mr_x.get(), c->mr_r.get(), c->mr_p.get(), c->mr_q.get(), c->mr_b.get(), S,
                             c->mr_part.get(), iters, status, rel, &ms);
  if (st != PBGPU_OK) return st;
  c->krylov_iters += *std::max_element(iters.begin(), iters.end());
  // per column: potential, energies with that column's charges
  PBGPU_CUDA(c, c->x.alloc(n_pad));
  PBGPU_CUDA(c, c->phi.alloc(c->n));
  for (int j = 0; j < k; ++j) {
    k_mr_get<<<grid_for(n_pad, 256), 256, 0, c->stream>>>(n_pad, kp, j, c->mr_x.get(), c->x.get());
    PBGPU_LAUNCHED(c);
    k_mr_gather_phi<<<grid_for(c->n, 256), 256, 0, c->stream>>>(c->n, c->iperm.get(), c->x.get(), c->phi.get());
    PBGPU_LAUNCHED(c);
    c->have_phi = true;
    if (energies) {
      if ((st = set_charges(charges + (size_t)j * na)) != PBGPU_OK) return st;
      if ((st = run_energy(c, fast, &energies[j])) != PBGPU_OK) return st;
    }
    if (stats) {
      stats[j].status = status[j];
      stats[j].iterations = iters[j];
      stats[j].outer = 0;
      stats[j].rel_residual = rel[j];
      stats[j].device_ms = ms;
    }
  }
  // the context's own charges, density map and right-hand side again; the
  // potential left in the context is the last column's
  if ((st = set_charges(q0.data())) != PBGPU_OK) return st;
  if ((st = run_density(c)) != PBGPU_OK) return st;
  if ((st = run_rhs(c)) != PBGPU_OK) return st;
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  for (int j = 0; j < k; ++j)
    if (status[j] == PBGPU_NOT_CONVERGED) return c->fail(status[j], "solve_charges: iteration limit reached");
  for (int j = 0; j < k; ++j)
    if (status[j] == PBGPU_BREAKDOWN) return c->fail(status[j], "solve_charges: breakdown");
  return PBGPU_OK;
}

}  // namespace pbgpu
