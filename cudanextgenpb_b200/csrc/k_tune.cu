// SELL layout autotuner: no counterpart in the reference (LIS stores CSR).
// The SpMV is the dominant kernel of every solve, and which layout feeds it
// best (slice height C, sorting window sigma, column-group width G, and for
// C = 32, G = 1 the chunk width of the shared-memory-staged kernel) depends on
// the matrix.  pbgpu_autotune assembles the context's system in each candidate
// layout, times the CG SpMV of a few Jacobi-CG iterations with CUDA events,
// keeps the fastest layout assembled, and remembers it per matrix size class
// (log2 of the row count) for later pbgpu_assemble calls made with NULL
// options in this process.
#include <cuda_runtime.h>

#include <cmath>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "pbgpu_internal.cuh"

namespace pbgpu {

struct Tuned {
  pbgpu_sell_opts sell;
  int cols;
};

static std::mutex g_tune_mu;
static std::map<int, Tuned> g_tuned;  // size class -> layout

static int size_class(int64_t n) {
  int k = 0;
  while ((int64_t(1) << (k + 1)) <= n) ++k;
  return k;
}

bool tuned_layout(int64_t n, pbgpu_sell_opts* sell, int* cols) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tuned.find(size_class(n));
  if (it == g_tuned.end()) return false;
  *sell = it->second.sell;
  *cols = it->second.cols;
  return true;
}

}  // namespace pbgpu

using namespace pbgpu;

extern "C" {

int pbgpu_autotune(pbgpu_ctx* h, int iterations, pbgpu_sell_opts* best, int* best_cols, double* best_spmv_ms) {
  if (!h) return PBGPU_ERR_ARG;
  Context* c = &h->c;
  if (!c->have_markers || !c->have_density) return c->fail(PBGPU_ERR_STATE, "autotune: density map required");
  if (iterations <= 0) iterations = 24;
  AcctScope acct(&c->dev_bytes);
  StreamScope sscope(c->stream);
  if (cudaSetDevice(c->device) != cudaSuccess) return c->fail(PBGPU_ERR_CUDA, "autotune: cudaSetDevice");
  struct Cand {
    pbgpu_sell_opts s;
    int cols;
  };
  const std::vector<Cand> cands = {
      {{32, 2048, 4}, 0},  {{32, 2048, 2}, 0},  {{32, 2048, 1}, 16}, {{32, 2048, 1}, 12},
      {{32, 256, 4}, 0},   {{32, 16384, 4}, 0}, {{64, 2048, 4}, 0},
  };
  // timing solves: CG, Jacobi, a fixed number of iterations
  pbgpu_solver_opts o;
  pbgpu_default_solver_opts(&o);
  o.method = PBGPU_CG;
  o.precond = PBGPU_PRECOND_JACOBI;
  o.precision = PBGPU_FP64;
  o.tol = 1e-300;
  o.max_iter = iterations;
  o.check_every = iterations;
  const bool prof = c->profiling;
  const int64_t l0 = c->launches, s0 = c->spmv_launches, k0 = c->krylov_iters;
  const double m0 = c->spmv_ms;
  const int cols0 = c->spmv_cols;
  double best_t = 1e300;
  int bi = -1;
  int rc = PBGPU_OK;
  for (size_t i = 0; i < cands.size(); ++i) {
    if ((rc = run_assemble(c, &cands[i].s)) != PBGPU_OK) break;
    c->spmv_cols = cands[i].cols ? cands[i].cols : cols0;
    c->profiling = true;
    c->spmv_ms = 0.0;
    c->spmv_launches = 0;
    pbgpu_solve_stats st{};
    rc = run_solve(c, &o, &st);
    if (rc == PBGPU_NOT_CONVERGED) rc = PBGPU_OK;  // the iteration cap is the point
    if (rc != PBGPU_OK) break;
    const double t = c->spmv_launches ? c->spmv_ms / (double)c->spmv_launches : 1e300;
    if (t < best_t) {
      best_t = t;
      bi = (int)i;
    }
  }
  c->profiling = prof;
  c->launches = l0;
  c->spmv_launches = s0;
  c->spmv_ms = m0;
  c->krylov_iters = k0;
  c->err.clear();
  if (rc != PBGPU_OK || bi < 0) {
    c->spmv_cols = cols0;
    return rc != PBGPU_OK ? rc : c->fail(PBGPU_ERR_STATE, "autotune: no candidate could be timed");
  }
  const Cand& b = cands[bi];
  c->spmv_cols = b.cols ? b.cols : cols0;
  if ((rc = run_assemble(c, &b.s)) != PBGPU_OK) return rc;
  c->have_phi = false;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[size_class(c->n)] = Tuned{b.s, c->spmv_cols};
  }
  if (best) *best = b.s;
  if (best_cols) *best_cols = b.cols;
  if (best_spmv_ms) *best_spmv_ms = best_t;
  return PBGPU_OK;
}

}  // extern "C"
