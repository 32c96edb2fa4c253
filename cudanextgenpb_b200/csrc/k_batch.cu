// Multi-system Krylov solve: many assembled systems (one per context) advanced
// together by ONE persistent cooperative kernel per chunk of steps.  This is
// the batching layer over lis_compute_electric_potential
// (src/pb_class.cpp:2244-2329): the reference solves one system per process;
// here independent molecules share the GPU in one launch.
//
// Design:
//  * Every member keeps its own SELL matrix and vectors; the kernel walks a
//    table of member descriptors.  Rows are grouped in row-blocks of 256 rows.
//  * Every member owns a group of the resident CTAs, sized in proportion to
//    its row-blocks (at least one); a CTA works for one member only and owns
//    the same rows in every phase.  Members never wait for one another: the
//    barriers between phases are per member, over its group alone, and a
//    member that has converged lets its CTAs return.
//  * Reductions are per member and deterministic: each row-block writes its
//    partial sums, and the last CTA of the group to reach the barrier sums
//    them with one warp in a fixed order and updates the member's scalars
//    before it releases the others.
//  * Each member runs Jacobi-preconditioned CG on A d = r in the inner type
//    TI (float: FP32 matrix and vectors; double: plain FP64) with the
//    solution accumulated in FP64.  In FP32 the CG uses reliable updates:
//    whenever its recursive residual has fallen by 10x since the last FP64
//    residual, x += d, the residual b - A x is recomputed in FP64 and the CG
//    continues from it keeping its search direction, so the iteration count
//    stays that of FP64 CG.  The FP64 residual also makes the final
//    convergence test.  Members move through these phases independently:
//    one step of the kernel does one CG iteration for members in the inner
//    phase and the residual / start / update work for the others.
//  * A step has three row phases, each closed by the member's barrier
//    (bounded spin: a barrier that times out sets an error flag and every
//    CTA returns at its next barrier).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "pbgpu_internal.cuh"
#include "sell.cuh"
#include "tma.cuh"

namespace pbgpu {

constexpr int kRowBlock = kBlock;  // rows per row-block
constexpr int kBatchMinBlocks = 4;

// Phases of a member: Outer (first FP64 residual), Start (CG start on it),
// Inner (CG iterations in TI), Apply (inner target met: x += xi, then FP64
// residual), Reliable (mixed precision: the TI residual fell by delta since
// the last FP64 residual: x += xi, FP64 residual), Resume (continue CG from
// the fresh FP64 residual keeping the search direction), Done.
enum { kPhOuter = 0, kPhStart = 1, kPhInner = 2, kPhApply = 3, kPhDone = 4, kPhReliable = 5, kPhResume = 6 };

template <typename TI>
struct BMember {
  SellT<double> A;       // FP64 system (SELL order)
  const double* b;
  double* x;             // solution
  SellT<TI> Ai;          // inner matrix (FP32 copy or the FP64 values)
  const TI* dinv;        // 1 / diag in TI
  TI* bi;                // inner right-hand side = outer residual
  TI* xi;                // inner solution = correction
  TI* r;
  TI* p;
  TI* q;
  int64_t rb0;           // first global row-block
  int nrb;               // row-blocks of this member
};

struct BState {
  double bb, rr64, tol2;      // ||b||^2, ||b - A x||^2, tol^2 ||b||^2
  double rz, alpha, beta, rri, tol2i;
  double inner_tol;
  double rr_ref;              // ||b - A x||^2 at the last FP64 residual
  double delta2;              // reliable update when the TI residual^2 < delta2 * rr_ref (0: off)
  int phase, iters, inner_it, outer, status, max_iter, inner_cap, plain;
};

// Barrier of one member's CTA group (count of arrivals, generation).
struct MemBar {
  unsigned count;
  unsigned gen;
};

// A CTA's assignment: the member slot it works for, its index in the
// member's group and the group's size.
struct CtaGroup {
  int slot, k, size, pad;
};

// Barrier over the `size` CTAs of one member's group.  The last CTA to arrive
// runs `last` (the member's reduction and scalar update) before it releases
// the others.  The wait is bounded (wait_ns of wall time, 2 s unless the
// batch's wait limit says otherwise), after which the shared error flag is
// set; every caller then returns false.  A zero limit gives up at once without
// polling (tests drive the timeout path with it).
template <class F>
__device__ __forceinline__ bool member_barrier(MemBar* b, int size, int* err, uint64_t wait_ns, F&& last) {
  __shared__ int is_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = &b->gen;
    const unsigned gen = *vgen;
    __threadfence();
    is_last = atomicAdd(&b->count, 1u) == (unsigned)size - 1u;
    if (!is_last && wait_ns == 0) {
      atomicExch(err, 1);
    } else if (!is_last) {
      const uint64_t t0 = global_ns();
      uint32_t it = 0;
      while (*vgen == gen) {
        if ((++it & 255u) == 0 && global_ns() - t0 > wait_ns) {
          atomicExch(err, 1);
          break;
        }
        if (*reinterpret_cast<volatile int*>(err)) break;
      }
    }
    __threadfence();
  }
  __syncthreads();
  if (is_last) {
    last();
    __syncthreads();
    if (threadIdx.x == 0) {
      b->count = 0;
      __threadfence();
      atomicAdd(&b->gen, 1u);
    }
  }
  __syncthreads();
  return *reinterpret_cast<volatile int*>(err) == 0;
}

// Member scalars and row-block partials, which other CTAs of the running
// kernel write, are read through L2 only (ld.global.cg).  The gathered vector
// entries are plain loads (L1-cached): they are read only after a member
// barrier whose acquire fence (fence.sc.gpu) orders them after the writers'
// release, never through the read-only path.  Every row is owned by the same
// thread in every phase, so a thread's own rows need no care.
template <typename T>
__device__ __forceinline__ T ldcg(const T* p) {
  return __ldcg(p);
}

template <typename T>
__device__ __forceinline__ T ld_plain(const T* p) {
  return *p;
}

// y_i = sum_j A(i, j) x_j of a G = 4 SELL row (sell_elem layout).
template <typename T>
__device__ __forceinline__ T batch_row(const SellT<T>& A, int64_t p, const T* x) {
  const int64_t s = p / A.C;
  const int lane = (int)(p - s * A.C);
  const int W = A.slice_w[s];
  const int64_t sb = A.slice_ptr[s];
  const int64_t base = sb + 4 * lane;
  const int64_t stride = 4 * (int64_t)A.C;
  T acc = 0;
#pragma unroll 2
  for (int g = 0; g < (W >> 2); ++g) {
    const int64_t k = base + g * stride;
    const int4 c = __ldcs(reinterpret_cast<const int4*>(A.scol + k));
    if constexpr (sizeof(T) == 8) {
      const double2 v0 = __ldcs(reinterpret_cast<const double2*>(A.sval + k));
      const double2 v1 = __ldcs(reinterpret_cast<const double2*>(A.sval + k + 2));
      acc += v0.x * ld_plain(x + c.x);
      acc += v0.y * ld_plain(x + c.y);
      acc += v1.x * ld_plain(x + c.z);
      acc += v1.y * ld_plain(x + c.w);
    } else {
      const float4 v = __ldcs(reinterpret_cast<const float4*>(A.sval + k));
      acc += v.x * ld_plain(x + c.x);
      acc += v.y * ld_plain(x + c.y);
      acc += v.z * ld_plain(x + c.z);
      acc += v.w * ld_plain(x + c.w);
    }
  }
  const int Wg = W & ~3;
  const int64_t tb = sb + (int64_t)Wg * A.C + lane;
  for (int j = Wg; j < W; ++j) {
    const int64_t k = tb + (int64_t)(j - Wg) * A.C;
    acc += __ldcs(A.sval + k) * ld_plain(x + __ldcs(A.scol + k));
  }
  return acc;
}

// Sum of this member's row-block partials (K per row-block) by one warp, in a
// fixed order; valid in all lanes.
template <int K>
__device__ __forceinline__ void member_sum(const double* part, int64_t rb0, int nrb, double (&out)[K]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < K; ++k) out[k] = 0.0;
  for (int j = lane; j < nrb; j += 32)
#pragma unroll
    for (int k = 0; k < K; ++k) out[k] += ldcg(part + (rb0 + j) * 2 + k);
#pragma unroll
  for (int k = 0; k < K; ++k)
    for (int o = 16; o > 0; o >>= 1) out[k] += __shfl_xor_sync(0xffffffffu, out[k], o);
}

// Member decisions after the first phase (warp 0 of the group's last CTA):
// the FP64 residual norm of an outer step, or alpha of a CG iteration.
template <typename TI>
__device__ __forceinline__ void member_after_spmv(BState& S, const BMember<TI>& M, const double* part) {
  const int lane = threadIdx.x & 31;
  const int ph = ldcg(&S.phase);
  if (ph == kPhDone || ph == kPhStart || ph == kPhResume) return;
  double a[2];
  member_sum<2>(part, M.rb0, M.nrb, a);
  if (lane != 0) return;
  if (ph == kPhOuter || ph == kPhApply || ph == kPhReliable) {
    if (S.outer == 0) {
      S.bb = a[1];
      S.tol2 = S.tol2 * a[1];  // tol^2 was stored; scale by ||b||^2
    }
    S.rr64 = a[0];
    S.outer += 1;
    if (!isfinite(a[0])) {
      S.status = PBGPU_BREAKDOWN;
      S.phase = kPhDone;
    } else if (a[0] <= S.tol2) {
      S.phase = kPhDone;
    } else if (S.iters >= S.max_iter) {
      S.status = PBGPU_NOT_CONVERGED;
      S.phase = kPhDone;
    } else {
      // the TI recursion aims at the final target; with reliable updates
      // (mixed precision) its residual is refreshed from FP64 on the way
      S.rr_ref = a[0];
      S.tol2i = S.tol2;
      S.phase = ph == kPhOuter ? kPhStart : kPhResume;
      S.inner_it = 0;
    }
  } else {  // inner
    const double alpha = S.rz / a[0];
    if (!(a[0] > 0.0) || !isfinite(alpha)) {
      S.status = PBGPU_BREAKDOWN;
      S.phase = kPhDone;
    } else {
      S.alpha = alpha;
    }
  }
}

// Member decisions after the second phase: rz of a (re)start, or beta and the
// stopping tests of a CG iteration.
template <typename TI>
__device__ __forceinline__ void member_after_update(BState& S, const BMember<TI>& M, const double* part) {
  const int lane = threadIdx.x & 31;
  const int ph = ldcg(&S.phase);
  if (ph != kPhStart && ph != kPhResume && ph != kPhInner) return;
  double a[2];
  member_sum<2>(part, M.rb0, M.nrb, a);
  if (lane != 0) return;
  if (ph == kPhStart) {
    S.rz = a[0];
    S.phase = kPhInner;
  } else if (ph == kPhResume) {
    // CG continues from the fresh residual: p = z + beta p in the third phase
    S.beta = a[0] / S.rz;
    S.rz = a[0];
    S.phase = isfinite(S.beta) ? kPhInner : kPhDone;
    if (S.phase == kPhDone) S.status = PBGPU_BREAKDOWN;
  } else {
    S.iters += 1;
    S.inner_it += 1;
    S.rri = a[1];
    if (!isfinite(a[0]) || !isfinite(a[1])) {
      S.status = PBGPU_BREAKDOWN;
      S.phase = kPhDone;
    } else if (a[1] <= S.tol2i || S.inner_it >= S.inner_cap || S.iters >= S.max_iter) {
      S.phase = kPhApply;
    } else if (a[1] <= S.delta2 * S.rr_ref) {
      S.phase = kPhReliable;
    } else {
      S.beta = a[0] / S.rz;
      S.rz = a[0];
    }
  }
}

template <typename TI>
__global__ void __launch_bounds__(kBlock, kBatchMinBlocks)
    k_batch_cg(const BMember<TI>* __restrict__ mem, const CtaGroup* __restrict__ groups, BState* st, double* part,
               MemBar* bars, int* err, int steps, unsigned long long wait_ns) {
  const CtaGroup G = groups[blockIdx.x];
  const BMember<TI>& M = mem[G.slot];
  BState& S = st[G.slot];
  MemBar* mb = bars + G.slot;
  const int warp = threadIdx.x >> 5;
  __shared__ int ph_s;
  auto read_phase = [&]() {
    __syncthreads();
    if (threadIdx.x == 0) ph_s = ldcg(&S.phase);
    __syncthreads();
    return ph_s;
  };
  for (int step = 0; step < steps; ++step) {
    // ---- phase 1: outer residual (outer / apply / reliable) or q = A p (inner)
    int ph = read_phase();
    if (ph == kPhDone) return;
    for (int rb = G.k; rb < M.nrb; rb += G.size) {
      const int64_t i = (int64_t)rb * kRowBlock + threadIdx.x;
      double v[2] = {0.0, 0.0};
      if ((ph == kPhOuter || ph == kPhApply || ph == kPhReliable) && i < M.A.n_pad) {
        const double ri = M.b[i] - batch_row<double>(M.A, i, M.x);
        M.bi[i] = (TI)ri;
        v[0] = ri * ri;
        v[1] = M.b[i] * M.b[i];
      } else if (ph == kPhInner && i < M.A.n_pad) {
        const TI y = batch_row<TI>(M.Ai, i, M.p);
        M.q[i] = y;
        v[0] = (double)M.p[i] * (double)y;
      }
      block_sum<2>(v);
      if (threadIdx.x == 0) {
        part[(M.rb0 + rb) * 2] = v[0];
        part[(M.rb0 + rb) * 2 + 1] = v[1];
      }
    }
    if (!member_barrier(mb, G.size, err, wait_ns, [&] {
          if (warp == 0) member_after_spmv<TI>(S, M, part);
        }))
      return;
    // ---- phase 2: inner start (xi = 0, r = bi, p = z) or inner update
    ph = read_phase();
    if (ph == kPhDone) return;
    for (int rb = G.k; rb < M.nrb; rb += G.size) {
      const int64_t i = (int64_t)rb * kRowBlock + threadIdx.x;
      double v[2] = {0.0, 0.0};
      if ((ph == kPhStart || ph == kPhResume) && i < M.A.n_pad) {
        const TI ri = M.bi[i];
        const TI zi = M.dinv[i] * ri;
        M.xi[i] = 0;
        M.r[i] = ri;
        if (ph == kPhStart) M.p[i] = zi;
        v[0] = (double)ri * (double)zi;
      } else if (ph == kPhInner && i < M.A.n_pad) {
        const TI alpha = (TI)ldcg(&S.alpha);
        M.xi[i] += alpha * M.p[i];
        const TI ri = M.r[i] - alpha * M.q[i];
        M.r[i] = ri;
        v[0] = (double)ri * (double)(M.dinv[i] * ri);
        v[1] = (double)ri * (double)ri;
      }
      block_sum<2>(v);
      if (threadIdx.x == 0) {
        part[(M.rb0 + rb) * 2] = v[0];
        part[(M.rb0 + rb) * 2 + 1] = v[1];
      }
    }
    if (!member_barrier(mb, G.size, err, wait_ns, [&] {
          if (warp == 0) member_after_update<TI>(S, M, part);
        }))
      return;
    // ---- phase 3: p = z + beta p (inner) or x += xi (apply / reliable)
    ph = read_phase();
    if (ph == kPhDone) return;
    if (ph == kPhInner || ph == kPhApply || ph == kPhReliable) {
      const TI beta = ph == kPhInner ? (TI)ldcg(&S.beta) : (TI)0;
      for (int rb = G.k; rb < M.nrb; rb += G.size) {
        const int64_t i = (int64_t)rb * kRowBlock + threadIdx.x;
        if (i >= M.A.n_pad) continue;
        if (ph == kPhInner)
          M.p[i] = M.dinv[i] * M.r[i] + beta * M.p[i];
        else
          M.x[i] += (double)M.xi[i];
      }
    }
    if (!member_barrier(mb, G.size, err, wait_ns, [] {})) return;
  }
}

template <typename TI>
__global__ void k_batch_gather(const BMember<TI>* __restrict__ mem, int s, int64_t n,
                               const int32_t* __restrict__ iperm, double* __restrict__ phi) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) phi[i] = mem[s].x[iperm[i]];
}

__global__ void k_batch_to_f32(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

}  // namespace pbgpu

using namespace pbgpu;

// A batch keeps one descriptor and one state per slot; slots without a member
// are "done" and own no row-blocks.  A session (begin .. step ..) fixes the
// solver options; members added during a session start at the next step.
struct pbgpu_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int sm_count = 148;
  int blocks_per_sm = 0;  // 0: as many as fit
  double wait_s = 2.0;    // limit of each member barrier wait (pbgpu_batch_set_wait_limit)
  std::string err;
  std::vector<pbgpu_ctx*> slots;
  std::vector<char> pending;  // member needs its vectors and state set up
  bool session = false;
  bool mixed = false;
  pbgpu_solver_opts opts{};
  bool dirty = true;          // row-block table out of date
  int64_t n_rb = 0;
  DBuf<BMember<double>> m64;
  DBuf<BMember<float>> m32;
  std::vector<BMember<double>> h64;
  std::vector<BMember<float>> h32;
  DBuf<CtaGroup> groups;
  std::vector<CtaGroup> h_groups;
  DBuf<double> part;
  DBuf<BState> st;
  DBuf<MemBar> bars;          // one per slot
  DBuf<int> errf;             // barrier timeout flag
  bool bars_reset = true;     // clear the member barriers before the next launch
  BState* st_host = nullptr;
  size_t st_cap = 0;
  int* err_host = nullptr;          // pinned copy of the timeout flag
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool in_flight = false;           // a launch whose states are not yet read
  bool kernel_in_flight = false;
  int flight_members = 0;
  int64_t launches = 0;
  float last_ms = 0.f;
  int fail(int code, const std::string& m) {
    err = m;
    return code;
  }
};

namespace {

int bfail(pbgpu_batch* b, cudaError_t e, const char* what) {
  cudaGetLastError();
  return b->fail(PBGPU_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define BATCH_CUDA(b, expr)                                                   \
  do {                                                                        \
    cudaError_t _e = (expr);                                                  \
    if (_e != cudaSuccess) return bfail((b), _e, #expr);                      \
  } while (0)

// Per-slot device arrays sized for every slot index.
int ensure_capacity(pbgpu_batch* B) {
  const size_t n = std::max<size_t>(B->slots.size(), 1);
  if (B->st_cap >= n) return PBGPU_OK;
  const size_t cap = std::max<size_t>(n, 2 * B->st_cap);
  BState* h = nullptr;
  BATCH_CUDA(B, cudaMallocHost(&h, cap * sizeof(BState)));
  for (size_t k = 0; k < cap; ++k) {
    h[k] = BState{};
    h[k].phase = kPhDone;
  }
  if (B->st_host) {
    std::memcpy(h, B->st_host, B->st_cap * sizeof(BState));
    cudaFreeHost(B->st_host);
  }
  B->st_host = h;
  // device copies: grow and carry the live states over
  DBuf<BState> nst;
  BATCH_CUDA(B, nst.alloc(cap));
  BATCH_CUDA(B, cudaMemcpyAsync(nst.get(), h, cap * sizeof(BState), cudaMemcpyHostToDevice, B->stream));
  if (B->st.get() && B->st_cap)
    BATCH_CUDA(B, cudaMemcpyAsync(nst.get(), B->st.get(), B->st_cap * sizeof(BState), cudaMemcpyDeviceToDevice,
                                  B->stream));
  BATCH_CUDA(B, cudaStreamSynchronize(B->stream));
  B->st.swap(nst);
  B->h64.resize(cap);
  B->h32.resize(cap);
  BATCH_CUDA(B, B->m64.alloc(cap));
  BATCH_CUDA(B, B->m32.alloc(cap));
  B->st_cap = cap;
  return PBGPU_OK;
}

// Vectors, FP32 copies and descriptor of a new member; its state starts at
// the first outer step with x = 0.
template <typename TI>
int prepare_member(pbgpu_batch* B, int slot) {
  Context* c = &B->slots[slot]->c;
  AcctScope acct(&c->dev_bytes);
  StreamScope sscope(c->stream);  // pool allocations on the member's own stream
  BATCH_CUDA(B, cudaStreamSynchronize(c->stream));  // the member's assembly is complete
  if (c->G != 4 || c->C != 32) return B->fail(PBGPU_ERR_ARG, "batch: members must be assembled with chunk 32, group 4");
  const int64_t n_pad = c->n_slices * c->C;
  const bool mixed = std::is_same<TI, float>::value;
  cudaError_t e = cudaSuccess;
  DBuf<double>* v64[] = {&c->x, &c->r, &c->p, &c->q, &c->rh, &c->s};
  for (DBuf<double>* d : v64)
    if (e == cudaSuccess) e = d->alloc(n_pad);
  if (mixed) {
    DBuf<float>* v32[] = {&c->x32, &c->r32, &c->p32, &c->q32, &c->b32, &c->dinv32};
    for (DBuf<float>* d : v32)
      if (e == cudaSuccess) e = d->alloc(n_pad);
    if (e == cudaSuccess) e = c->sval32.alloc(c->sell_len);
  }
  if (e != cudaSuccess) return bfail(B, e, "batch: member vectors");
  BATCH_CUDA(B, cudaStreamSynchronize(c->stream));  // the allocations are ordered on that stream
  BATCH_CUDA(B, cudaMemsetAsync(c->x.get(), 0, n_pad * sizeof(double), B->stream));
  if (mixed) {
    const int g = (int)std::min<int64_t>((c->sell_len + kBlock - 1) / kBlock, (int64_t)B->sm_count * 8);
    k_batch_to_f32<<<g, kBlock, 0, B->stream>>>(c->sell_len, c->sval.get(), c->sval32.get());
    k_batch_to_f32<<<g, kBlock, 0, B->stream>>>(n_pad, c->dinv.get(), c->dinv32.get());
    B->launches += 2;
    BATCH_CUDA(B, cudaGetLastError());
  }
  BMember<TI> M{};
  M.A = SellT<double>{c->slice_ptr.get(), c->slice_w.get(), c->scol.get(), c->sval.get(), n_pad, c->C, c->G};
  M.b = c->b.get();
  M.x = c->x.get();
  if constexpr (std::is_same<TI, float>::value) {
    M.Ai = SellT<float>{c->slice_ptr.get(), c->slice_w.get(), c->scol.get(), c->sval32.get(), n_pad, c->C, c->G};
    M.dinv = c->dinv32.get();
    M.bi = c->b32.get();
    M.xi = c->x32.get();
    M.r = c->r32.get();
    M.p = c->p32.get();
    M.q = c->q32.get();
    B->h32[slot] = M;
  } else {
    M.Ai = M.A;
    M.dinv = c->dinv.get();
    M.bi = c->rh.get();
    M.xi = c->s.get();
    M.r = c->r.get();
    M.p = c->p.get();
    M.q = c->q.get();
    B->h64[slot] = M;
  }
  const pbgpu_solver_opts& o = B->opts;
  BState S{};
  S.tol2 = o.tol * o.tol;  // scaled by ||b||^2 at the first outer step
  S.inner_tol = o.inner_tol > 0 ? o.inner_tol : 1e-5;
  S.phase = kPhOuter;
  S.status = PBGPU_OK;
  S.max_iter = o.max_iter;
  S.inner_cap = o.max_iter;
  S.plain = mixed ? 0 : 1;
  S.delta2 = mixed ? 0.01 : 0.0;  // reliable update every 10x residual reduction in FP32
  B->st_host[slot] = S;
  BATCH_CUDA(B, cudaMemcpyAsync(B->st.get() + slot, &B->st_host[slot], sizeof(BState), cudaMemcpyHostToDevice,
                                B->stream));
  B->pending[slot] = 0;
  B->dirty = true;
  return PBGPU_OK;
}

// Descriptors of the current members and their row-block ranges.
template <typename TI>
int upload_tables(pbgpu_batch* B) {
  std::vector<BMember<TI>>& hm = *[&]() {
    if constexpr (std::is_same<TI, float>::value)
      return &B->h32;
    else
      return &B->h64;
  }();
  std::vector<int32_t> rbs;
  for (size_t k = 0; k < B->slots.size(); ++k) {
    if (!B->slots[k]) {
      hm[k] = BMember<TI>{};
      continue;
    }
    hm[k].rb0 = (int64_t)rbs.size();
    hm[k].nrb = (int)((hm[k].A.n_pad + kRowBlock - 1) / kRowBlock);
    for (int j = 0; j < hm[k].nrb; ++j) rbs.push_back((int32_t)k);
  }
  B->n_rb = (int64_t)rbs.size();
  BMember<TI>* dm;
  if constexpr (std::is_same<TI, float>::value)
    dm = B->m32.get();
  else
    dm = B->m64.get();
  BATCH_CUDA(B, cudaMemcpyAsync(dm, hm.data(), B->slots.size() * sizeof(BMember<TI>), cudaMemcpyHostToDevice,
                                B->stream));
  BATCH_CUDA(B, B->part.alloc(2 * std::max<int64_t>(B->n_rb, 1)));
  B->dirty = false;
  return PBGPU_OK;
}

// Launches one persistent kernel of up to `steps` steps over the current
// members and queues the copy of their states to the host; returns without
// waiting (batch_wait completes it).
template <typename TI>
int batch_launch(pbgpu_batch* B, int steps) {
  int rc;
  if ((rc = ensure_capacity(B)) != PBGPU_OK) return rc;
  for (size_t k = 0; k < B->slots.size(); ++k)
    if (B->slots[k] && B->pending[k] && (rc = prepare_member<TI>(B, (int)k)) != PBGPU_OK) return rc;
  if (B->dirty && (rc = upload_tables<TI>(B)) != PBGPU_OK) return rc;
  const int nm = (int)B->slots.size();
  B->flight_members = nm;
  if (!B->ev0) {
    BATCH_CUDA(B, cudaEventCreate(&B->ev0));
    BATCH_CUDA(B, cudaEventCreate(&B->ev1));
    BATCH_CUDA(B, cudaMallocHost(&B->err_host, sizeof(int)));
  }
  *B->err_host = 0;
  B->kernel_in_flight = false;
  // members that take part: set up and not finished
  const std::vector<BMember<TI>>& hm = *[&]() {
    if constexpr (std::is_same<TI, float>::value)
      return &B->h32;
    else
      return &B->h64;
  }();
  std::vector<int> act;
  for (int k = 0; k < nm; ++k)
    if (B->slots[k] && !B->pending[k] && B->st_host[k].phase != kPhDone && hm[k].nrb > 0) act.push_back(k);
  if (!act.empty() && steps > 0) {
    int occ = 0;
    BATCH_CUDA(B, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_batch_cg<TI>, kBlock, 0));
    if (occ <= 0) return B->fail(PBGPU_ERR_CUDA, "batch: kernel cannot be resident");
    if (B->blocks_per_sm > 0) occ = std::min(occ, B->blocks_per_sm);
    const int64_t cap = (int64_t)occ * B->sm_count;
    if ((int64_t)act.size() > cap)
      return B->fail(PBGPU_ERR_CAPACITY, "batch: more unfinished members than resident CTAs (" + std::to_string(cap) + ")");
    // CTA groups: one CTA each, then one more at a time to the member with
    // the most row-blocks per CTA, up to the resident CTAs or one CTA per
    // row-block
    std::vector<int> g(act.size(), 1);
    int64_t left = cap - (int64_t)act.size();
    while (left > 0) {
      int best = -1;
      double bw = 0.0;
      for (size_t j = 0; j < act.size(); ++j) {
        const int nrb = hm[act[j]].nrb;
        if (g[j] >= nrb) continue;
        const double w = (double)nrb / g[j];
        if (w > bw) {
          bw = w;
          best = (int)j;
        }
      }
      if (best < 0) break;
      ++g[best];
      --left;
    }
    B->h_groups.clear();
    for (size_t j = 0; j < act.size(); ++j)
      for (int k = 0; k < g[j]; ++k) B->h_groups.push_back(CtaGroup{act[j], k, g[j], 0});
    const int grid = (int)B->h_groups.size();
    BATCH_CUDA(B, B->groups.alloc(grid));
    BATCH_CUDA(B, cudaMemcpyAsync(B->groups.get(), B->h_groups.data(), grid * sizeof(CtaGroup),
                                  cudaMemcpyHostToDevice, B->stream));
    if (B->bars.n < B->st_cap || !B->bars.get()) {
      BATCH_CUDA(B, B->bars.alloc(B->st_cap));
      B->bars_reset = true;
    }
    if (B->bars_reset) {
      BATCH_CUDA(B, cudaMemsetAsync(B->bars.get(), 0, B->bars.n * sizeof(MemBar), B->stream));
      B->bars_reset = false;
    }
    BATCH_CUDA(B, B->errf.alloc(1));
    BATCH_CUDA(B, cudaMemsetAsync(B->errf.get(), 0, sizeof(int), B->stream));
    const BMember<TI>* a_mem;
    if constexpr (std::is_same<TI, float>::value)
      a_mem = B->m32.get();
    else
      a_mem = B->m64.get();
    const CtaGroup* a_groups = B->groups.get();
    BState* a_st = B->st.get();
    double* a_part = B->part.get();
    MemBar* a_bars = B->bars.get();
    int* a_err = B->errf.get();
    int a_steps = steps;
    unsigned long long a_wait = (unsigned long long)(B->wait_s * 1e9);
    void* args[] = {&a_mem, &a_groups, &a_st, &a_part, &a_bars, &a_err, &a_steps, &a_wait};
    BATCH_CUDA(B, cudaEventRecord(B->ev0, B->stream));
    BATCH_CUDA(B, cudaLaunchCooperativeKernel((const void*)k_batch_cg<TI>, dim3(grid), dim3(kBlock), args, 0,
                                              B->stream));
    B->launches += 1;
    BATCH_CUDA(B, cudaEventRecord(B->ev1, B->stream));
    BATCH_CUDA(B, cudaMemcpyAsync(B->err_host, B->errf.get(), sizeof(int), cudaMemcpyDeviceToHost, B->stream));
    B->kernel_in_flight = true;
  }
  BATCH_CUDA(B, cudaMemcpyAsync(B->st_host, B->st.get(), nm * sizeof(BState), cudaMemcpyDeviceToHost, B->stream));
  B->in_flight = true;
  return PBGPU_OK;
}

int batch_wait(pbgpu_batch* B, int* n_active) {
  if (B->in_flight) {
    B->in_flight = false;
    BATCH_CUDA(B, cudaStreamSynchronize(B->stream));
    if (B->kernel_in_flight) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, B->ev0, B->ev1) == cudaSuccess) B->last_ms += ms;
      B->kernel_in_flight = false;
      if (*B->err_host) {
        B->bars_reset = true;
        return B->fail(PBGPU_TIMEOUT, "batch: member barrier wait timed out");
      }
    }
  }
  int active = 0;
  for (int k = 0; k < B->flight_members && (size_t)k < B->slots.size(); ++k)
    active += B->slots[k] && !B->pending[k] && B->st_host[k].phase != kPhDone;
  for (size_t k = 0; k < B->slots.size(); ++k) active += B->slots[k] && B->pending[k];
  if (n_active) *n_active = active;
  return PBGPU_OK;
}

// Potential of a finished member into its context (node order) and its stats.
template <typename TI>
int finish_member(pbgpu_batch* B, int slot, pbgpu_solve_stats* stats) {
  Context* c = &B->slots[slot]->c;
  AcctScope acct(&c->dev_bytes);
  StreamScope sscope(c->stream);  // pool allocations on the member's own stream
  const BState& S = B->st_host[slot];
  BATCH_CUDA(B, c->phi.alloc(c->n));
  BATCH_CUDA(B, cudaStreamSynchronize(c->stream));
  const BMember<TI>* dm;
  if constexpr (std::is_same<TI, float>::value)
    dm = B->m32.get();
  else
    dm = B->m64.get();
  k_batch_gather<TI><<<(int)((c->n + 255) / 256), 256, 0, B->stream>>>(dm, slot, c->n, c->iperm.get(), c->phi.get());
  B->launches += 1;
  BATCH_CUDA(B, cudaGetLastError());
  BATCH_CUDA(B, cudaStreamSynchronize(B->stream));
  c->have_phi = true;
  c->krylov_iters += S.iters;
  if (stats) {
    stats->status = S.phase == kPhDone ? S.status : PBGPU_NOT_CONVERGED;
    stats->iterations = S.iters;
    stats->outer = S.outer;
    stats->rel_residual = S.bb > 0 ? std::sqrt(S.rr64 / S.bb) : 0.0;
    stats->device_ms = B->last_ms;
  }
  return PBGPU_OK;
}

int check_opts(pbgpu_batch* b, const pbgpu_solver_opts& o) {
  if (o.method != PBGPU_CG) return b->fail(PBGPU_ERR_ARG, "batch: members are solved with CG");
  if (o.precond != PBGPU_PRECOND_JACOBI) return b->fail(PBGPU_ERR_ARG, "batch: members use the Jacobi preconditioner");
  if (o.conv_cond == 2) return b->fail(PBGPU_ERR_ARG, "batch: conv_cond 0 or 1 (relative 2-norm)");
  if (!(o.tol > 0) || o.max_iter <= 0) return b->fail(PBGPU_ERR_ARG, "batch: tol and max_iter must be positive");
  return PBGPU_OK;
}

}  // namespace

namespace pbgpu {
int64_t batch_launch_count(const pbgpu_batch* b) { return b ? b->launches : 0; }
}  // namespace pbgpu

extern "C" {

int pbgpu_batch_create(pbgpu_batch** out, int device, void* cuda_stream) {
  if (!out) return PBGPU_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return PBGPU_ERR_CUDA;
  }
  if (device < 0 || device >= ndev) return PBGPU_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return PBGPU_ERR_CUDA;
  int coop = 0;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
  if (!coop) return PBGPU_ERR_CUDA;
  pbgpu_batch* b = new (std::nothrow) pbgpu_batch();
  if (!b) return PBGPU_ERR_OOM;
  b->device = device;
  cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (cuda_stream) {
    b->stream = static_cast<cudaStream_t>(cuda_stream);
  } else {
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete b;
      return PBGPU_ERR_CUDA;
    }
    b->own_stream = true;
  }
  *out = b;
  return PBGPU_OK;
}

void pbgpu_batch_destroy(pbgpu_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->st_host) cudaFreeHost(b->st_host);
  if (b->err_host) cudaFreeHost(b->err_host);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  cudaStream_t s = b->stream;
  const bool own = b->own_stream;
  delete b;
  if (own && s) cudaStreamDestroy(s);
}

const char* pbgpu_batch_last_error(const pbgpu_batch* b) { return b ? b->err.c_str() : "null batch"; }

int pbgpu_batch_add(pbgpu_batch* b, pbgpu_ctx* ctx, int* slot) {
  if (!b || !ctx) return PBGPU_ERR_ARG;
  if (ctx->c.device != b->device) return b->fail(PBGPU_ERR_ARG, "batch_add: context is on another device");
  if (!ctx->c.have_system) return b->fail(PBGPU_ERR_STATE, "batch_add: the context has no assembled system");
  for (pbgpu_ctx* m : b->slots)
    if (m == ctx) return b->fail(PBGPU_ERR_ARG, "batch_add: context is already a member");
  int k = -1;
  for (size_t j = 0; j < b->slots.size(); ++j)
    if (!b->slots[j]) {
      k = (int)j;
      break;
    }
  if (k < 0) {
    k = (int)b->slots.size();
    b->slots.push_back(nullptr);
    b->pending.push_back(0);
  }
  b->slots[k] = ctx;
  b->pending[k] = 1;
  b->dirty = true;
  if (slot) *slot = k;
  return PBGPU_OK;
}

int pbgpu_batch_remove(pbgpu_batch* b, int slot) {
  if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot]) return PBGPU_ERR_ARG;
  if (b->in_flight) return b->fail(PBGPU_ERR_STATE, "batch_remove: a launch is in flight (pbgpu_batch_wait)");
  b->slots[slot] = nullptr;
  b->pending[slot] = 0;
  if (b->st_host && (size_t)slot < b->st_cap) {
    b->st_host[slot].phase = kPhDone;
    if (cudaSetDevice(b->device) != cudaSuccess) return PBGPU_ERR_CUDA;
    const cudaError_t e = cudaMemcpyAsync(b->st.get() + slot, &b->st_host[slot], sizeof(BState),
                                          cudaMemcpyHostToDevice, b->stream);
    if (e != cudaSuccess) return bfail(b, e, "batch_remove");
    if ((size_t)slot + 1 == b->slots.size()) cudaStreamSynchronize(b->stream);
  }
  b->dirty = true;
  return PBGPU_OK;
}

int pbgpu_batch_size(const pbgpu_batch* b) {
  if (!b) return -1;
  int n = 0;
  for (pbgpu_ctx* m : b->slots) n += m != nullptr;
  return n;
}

int pbgpu_batch_set_blocks_per_sm(pbgpu_batch* b, int blocks) {
  if (!b || blocks < 0) return PBGPU_ERR_ARG;
  b->blocks_per_sm = blocks;
  return PBGPU_OK;
}

int pbgpu_batch_set_wait_limit(pbgpu_batch* b, double seconds) {
  if (!b || !(seconds >= 0.0) || seconds > 60.0) return PBGPU_ERR_ARG;
  b->wait_s = seconds;
  return PBGPU_OK;
}

int pbgpu_batch_begin(pbgpu_batch* b, const pbgpu_solver_opts* opts) {
  if (!b) return PBGPU_ERR_ARG;
  pbgpu_solver_opts o;
  if (opts)
    o = *opts;
  else
    pbgpu_default_solver_opts(&o);
  const int rc = check_opts(b, o);
  if (rc != PBGPU_OK) return rc;
  if (b->in_flight) return b->fail(PBGPU_ERR_STATE, "batch_begin: a launch is in flight (pbgpu_batch_wait)");
  b->opts = o;
  b->mixed = o.precision == PBGPU_MIXED;
  b->session = true;
  b->last_ms = 0.f;
  for (size_t k = 0; k < b->slots.size(); ++k) b->pending[k] = b->slots[k] != nullptr;
  b->dirty = true;
  return PBGPU_OK;
}

int pbgpu_batch_launch(pbgpu_batch* b, int steps) {
  if (!b || steps < 0) return PBGPU_ERR_ARG;
  if (!b->session) return b->fail(PBGPU_ERR_STATE, "batch_launch: no session (pbgpu_batch_begin)");
  if (b->in_flight) return b->fail(PBGPU_ERR_STATE, "batch_launch: the previous launch was not waited for");
  if (cudaSetDevice(b->device) != cudaSuccess) return PBGPU_ERR_CUDA;
  cudaGetLastError();
  return b->mixed ? batch_launch<float>(b, steps) : batch_launch<double>(b, steps);
}

int pbgpu_batch_wait(pbgpu_batch* b, int* n_active) {
  if (!b) return PBGPU_ERR_ARG;
  if (cudaSetDevice(b->device) != cudaSuccess) return PBGPU_ERR_CUDA;
  return batch_wait(b, n_active);
}

int pbgpu_batch_step(pbgpu_batch* b, int steps, int* n_active) {
  const int rc = pbgpu_batch_launch(b, steps);
  if (rc != PBGPU_OK) return rc;
  return pbgpu_batch_wait(b, n_active);
}

int pbgpu_batch_member(pbgpu_batch* b, int slot, int* done, pbgpu_solve_stats* stats) {
  if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot]) return PBGPU_ERR_ARG;
  if (b->in_flight) return b->fail(PBGPU_ERR_STATE, "batch_member: a launch is in flight (pbgpu_batch_wait)");
  if (!b->session || b->pending[slot] || !b->st_host || (size_t)slot >= b->st_cap) {
    if (done) *done = 0;
    return PBGPU_OK;
  }
  const bool fin = b->st_host[slot].phase == kPhDone;
  if (done) *done = fin;
  if (!fin) return PBGPU_OK;
  if (cudaSetDevice(b->device) != cudaSuccess) return PBGPU_ERR_CUDA;
  return b->mixed ? finish_member<float>(b, slot, stats) : finish_member<double>(b, slot, stats);
}

int pbgpu_batch_solve(pbgpu_batch* b, const pbgpu_solver_opts* opts, pbgpu_solve_stats* stats) {
  int rc = pbgpu_batch_begin(b, opts);
  if (rc != PBGPU_OK) return rc;
  const pbgpu_solver_opts& o = b->opts;
  const int chunk = o.check_every > 0 ? std::max(o.check_every, 16) : 64;
  const int max_outer = o.max_outer > 0 ? o.max_outer : 50;
  const int64_t max_steps = (int64_t)o.max_iter + 4LL * (max_outer + 2);
  int active = 1;
  for (int64_t done = 0; done < max_steps && active > 0; done += chunk)
    if ((rc = pbgpu_batch_step(b, chunk, &active)) != PBGPU_OK) return rc;
  int worst = PBGPU_OK;
  for (size_t k = 0; k < b->slots.size(); ++k) {
    if (!b->slots[k]) continue;
    pbgpu_solve_stats t{};
    int fin = 0;
    if (b->st_host[k].phase != kPhDone) {
      // iteration budget used up: report the member as not converged
      b->st_host[k].phase = kPhDone;
      b->st_host[k].status = PBGPU_NOT_CONVERGED;
    }
    if ((rc = pbgpu_batch_member(b, (int)k, &fin, &t)) != PBGPU_OK) return rc;
    if (stats) stats[k] = t;
    if (t.status != PBGPU_OK && worst == PBGPU_OK) worst = t.status;
  }
  b->session = false;
  if (worst == PBGPU_NOT_CONVERGED) return b->fail(worst, "batch: a member reached the iteration limit");
  if (worst == PBGPU_BREAKDOWN) return b->fail(worst, "batch: a member broke down");
  return PBGPU_OK;
}

}  // extern "C"
