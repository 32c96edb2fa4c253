// assemple_system_matrix on the device (src/pb_class.cpp:2053-2159): the
// box-method operator of bimpp's bim3a_laplacian_frac + bim3a_reaction_frac
// (or bim3a_reaction with a Stern layer) + bim3a_rhs + bim3a_dirichlet_bc,
// written straight into a SELL-C-sigma matrix.
//
// Each matrix row is gathered by one thread from the node's incidence list
// (octant, corner), so no atomics touch the values.  Per incidence the thread
// rebuilds the octant's local coefficients it needs (the corner's 3 edge
// conductances, the lumped reaction, V/8 * rho) and spreads them over the
// independent nodes behind each local corner (a hanging corner over its parents
// with weight 1/num_parents: A = P^T K P).  Pass 1 counts each row's distinct
// columns, the SELL layout is derived from those lengths (rows sorted by length
// inside windows of sigma rows, slices of C rows as wide as their longest
// row), pass 2 writes values and columns in SELL numbering.  Dirichlet
// nodes become identity rows and are eliminated from the other rows into the
// right-hand side, which keeps the matrix symmetric.
#include <algorithm>
#include <cstdlib>
#include <cub/cub.cuh>

#include "pbgpu_internal.cuh"

namespace pbgpu {

struct AsmView {
  const int64_t* inc_ptr;
  const uint32_t* inc;
  const int4* oct;
  const int32_t* oct_nodes;
  const int4* hang_par;
  const int8_t* hang_np;
  const double* eps;
  const double* react;
  const double* react_cell;
  const double* rho;
  const double* frac;
  const int32_t* border_pos;
  const uint8_t* dirichlet;
  const double* gval;
  int64_t n;
  int stern;
  double lo[3], len[3];
};

__device__ __forceinline__ double corner_val(const double* __restrict__ v, int32_t nd, const AsmView& A) {
  if (nd < A.n) return v[nd];
  const int64_t h = nd - A.n;
  const int4 p = A.hang_par[h];
  const int np = A.hang_np[h];
  double t = 0.0;
  t += v[p.x] / np;
  t += v[p.y] / np;
  if (np == 4) {
    t += v[p.z] / np;
    t += v[p.w] / np;
  }
  return t;
}

// Independent nodes behind node id nd, with weights.
__device__ __forceinline__ int expand(int32_t nd, const AsmView& A, int32_t g[4], double w[4]) {
  if (nd < A.n) {
    g[0] = nd;
    w[0] = 1.0;
    return 1;
  }
  const int64_t h = nd - A.n;
  const int4 p = A.hang_par[h];
  const int np = A.hang_np[h];
  g[0] = p.x;
  g[1] = p.y;
  g[2] = p.z;
  g[3] = p.w;
  const double wi = 1.0 / np;
  for (int j = 0; j < 4; ++j) w[j] = wi;
  return np;
}

// Threads per block of the row kernels; the shared-memory slot arrays below
// are laid out for exactly this many threads (slot k of thread t at
// [k * kAsmBlock + t], so the lanes of a warp hit distinct banks whichever
// slots they are at).
constexpr int kAsmBlock = 128;
// The first pass writes each row's distinct columns, sorted, into a 128-byte
// line of kColLine entries, of which the first kShRow may be used; rows of a
// 2:1 balanced octree hold at most ~25.  A row with more is gathered into the
// local-memory accumulator (kMaxRow slots) instead.
// PBGPU_ASM_SLOTS=4 lowers both limits to 4, which sends most rows down that
// path (for tests of it).
constexpr int kColLine = 32;
constexpr int kHashSlots = 64;  // per-thread hash set of the first pass (at most kColLine used)
constexpr uint8_t kWideRow = 0xff;
constexpr int kShRow = 28;
constexpr int kShFew = 4;

static bool asm_few_slots() {
  const char* e = std::getenv("PBGPU_ASM_SLOTS");
  return e && std::atoi(e) == kShFew;
}

// Sorted (column, value) accumulator of one thread in local memory, used only
// for rows that overflow the shared-memory one.
struct RowAcc {
  int32_t col[kMaxRow];
  double val[kMaxRow];
  int m = 0;
  bool overflow = false;
  __device__ __forceinline__ int32_t c_at(int j) const { return col[j]; }
  __device__ __forceinline__ double v_at(int j) const { return val[j]; }
  __device__ __forceinline__ void add(int32_t c, double v) {
    int j = m - 1;
    while (j >= 0 && col[j] > c) --j;
    if (j >= 0 && col[j] == c) {
      val[j] += v;
      return;
    }
    if (m == kMaxRow) {
      overflow = true;
      return;
    }
    for (int k = m - 1; k > j; --k) {
      col[k + 1] = col[k];
      val[k + 1] = val[k];
    }
    col[j + 1] = c;
    val[j + 1] = v;
    ++m;
  }
};

// The same accumulator in shared memory (the right-hand-side-only gather).
template <int K>
struct ShAcc {
  int32_t* col;  // this thread's slot 0; slot k at col[k * kAsmBlock]
  double* val;
  int m = 0;
  bool overflow = false;
  __device__ __forceinline__ int32_t c_at(int j) const { return col[j * kAsmBlock]; }
  __device__ __forceinline__ double v_at(int j) const { return val[j * kAsmBlock]; }
  __device__ __forceinline__ void add(int32_t c, double v) {
    if (overflow) return;
    int j = m - 1;
    while (j >= 0 && col[j * kAsmBlock] > c) --j;
    if (j >= 0 && col[j * kAsmBlock] == c) {
      val[j * kAsmBlock] += v;
      return;
    }
    if (m == K) {
      overflow = true;
      return;
    }
    for (int k = m - 1; k > j; --k) {
      col[(k + 1) * kAsmBlock] = col[k * kAsmBlock];
      val[(k + 1) * kAsmBlock] = val[k * kAsmBlock];
    }
    col[(j + 1) * kAsmBlock] = c;
    val[(j + 1) * kAsmBlock] = v;
    ++m;
  }
};

// Local box-method coefficients of every octant, computed once per octant
// with the expressions (and accumulation order) of the local matrix: the 12
// edge conductances wha(eps_i1, eps_i2, f) * area_h, the 8 diagonal entries
// (sum of the corner's 3 conductances in edge order, then the lumped reaction
// kappa_c * V/8 * w_c, w_c the product of the corner's half-edge shares), and
// the 8 right-hand-side terms V/8 * rho_c.
__global__ void k_octant_local(AsmView A, int64_t n_oct, double* __restrict__ cond, double* __restrict__ kd,
                               double* __restrict__ fr) {
  const int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (o >= n_oct) return;
  const int4 q = A.oct[o];
  const int32_t s = 1 << (kRootLog - q.w);
  const int32_t qc[3] = {q.x, q.y, q.z};
  double h[3];
  for (int d = 0; d < 3; ++d) h[d] = coord(A.lo[d], A.len[d], qc[d] + s) - coord(A.lo[d], A.len[d], qc[d]);
  const double area_h[3] = {h[1] * h[2] / h[0] * 0.25, h[0] * h[2] / h[1] * 0.25, h[0] * h[1] / h[2] * 0.25};
  const double v8 = h[0] * h[1] * h[2] * 0.125;
  const int32_t bp = A.border_pos[o];
  const int4 na = reinterpret_cast<const int4*>(A.oct_nodes)[2 * o];
  const int4 nb = reinterpret_cast<const int4*>(A.oct_nodes)[2 * o + 1];
  const int32_t nd[8] = {na.x, na.y, na.z, na.w, nb.x, nb.y, nb.z, nb.w};
  double ec[8], w[8], k[8];
  for (int c = 0; c < 8; ++c) {
    ec[c] = corner_val(A.eps, nd[c], A);
    w[c] = 1.0;
    k[c] = 0.0;
  }
  double* co = cond + 12 * o;
  for (int e = 0; e < 12; ++e) {
    const int i1 = d_edge_nodes[2 * e], i2 = d_edge_nodes[2 * e + 1];
    const double f = bp >= 0 ? A.frac[12 * (int64_t)bp + e] : 0.5;
    const double c = wha(ec[i1], ec[i2], f) * area_h[d_edge_axis[e]];
    co[e] = c;
    k[i1] += c;
    k[i2] += c;
    w[i1] *= fmin(1.0, 2.0 * f);
    w[i2] *= fmin(1.0, 2.0 * (1.0 - f));
  }
  for (int c = 0; c < 8; ++c) {
    if (A.stern)
      k[c] += A.react_cell[o] * v8;
    else
      k[c] += corner_val(A.react, nd[c], A) * v8 * w[c];
    kd[8 * o + c] = k[c];
    fr[8 * o + c] = v8 * corner_val(A.rho, nd[c], A);
  }
}

struct LocalView {
  const double* cond;
  const double* kd;
  const double* fr;
};

// The 3 edges at corner a in ascending edge id, with their axes.
__device__ __forceinline__ void corner_edges(int a, int ed[3], int ax[3]) {
  for (int d = 0; d < 3; ++d) {
    ed[d] = edge_of(a, d);
    ax[d] = d;
  }
  for (int u = 0; u < 3; ++u)
    for (int v = u + 1; v < 3; ++v)
      if (ed[v] < ed[u]) {
        int tmp = ed[u];
        ed[u] = ed[v];
        ed[v] = tmp;
        tmp = ax[u];
        ax[u] = ax[v];
        ax[v] = tmp;
      }
}

// Gather row i of A and its right-hand side entry (before Dirichlet handling)
// from the octants' local coefficients: A = P^T K P over the node's incidences.
template <class Acc>
__device__ void gather_row(int64_t i, const AsmView& A, const LocalView& L, Acc& R, double& rhs) {
  rhs = 0.0;
  for (int64_t e = A.inc_ptr[i]; e < A.inc_ptr[i + 1]; ++e) {
    const uint32_t t = A.inc[e];
    const int64_t o = t >> 3;
    const int a = (int)(t & 7);
    const int32_t nda = A.oct_nodes[t];
    const double wa = nda < A.n ? 1.0 : 1.0 / A.hang_np[nda - A.n];
    const double kaa = L.kd[t];
    int ed[3], ax[3];
    corner_edges(a, ed, ax);
    int32_t g[4];
    double w[4];
    int ng = expand(nda, A, g, w);
    for (int j = 0; j < ng; ++j) R.add(g[j], wa * kaa * w[j]);
    for (int u = 0; u < 3; ++u) {
      const int32_t ndb = A.oct_nodes[8 * o + (a ^ (1 << ax[u]))];
      const double kab = 0.0 - L.cond[12 * o + ed[u]];
      ng = expand(ndb, A, g, w);
      for (int j = 0; j < ng; ++j) R.add(g[j], wa * kab * w[j]);
    }
    rhs += wa * L.fr[t];
  }
}

// Sorted set of column ids held by one thread (pass 1 needs no values), in
// local memory (kMaxRow slots, the overflow path) or in shared memory with the
// slot layout of ShAcc.
struct ColSet {
  int32_t col[kMaxRow];
  int m = 0;
  bool overflow = false;
  __device__ __forceinline__ int32_t c_at(int j) const { return col[j]; }
  __device__ __forceinline__ void add(int32_t c) {
    int j = m - 1;
    while (j >= 0 && col[j] > c) --j;
    if (j >= 0 && col[j] == c) return;
    if (m == kMaxRow) {
      overflow = true;
      return;
    }
    for (int k = m - 1; k > j; --k) col[k + 1] = col[k];
    col[j + 1] = c;
    ++m;
  }
};

// Set of column ids of one thread in shared memory: open addressing over
// kHashSlots slots (empty = -1), at most `limit` (< kHashSlots) ids, so a
// probe always ends at the id or at an empty slot.  One add is a hash and
// usually one probe, whatever the row's length.
struct HashSet {
  int32_t* tab;  // this thread's slot 0; slot k at tab[k * kAsmBlock]
  int limit;
  int m = 0;
  bool overflow = false;
  __device__ __forceinline__ void clear() {
#pragma unroll 8
    for (int k = 0; k < kHashSlots; ++k) tab[k * kAsmBlock] = -1;
  }
  __device__ __forceinline__ void add(int32_t c) {
    if (overflow) return;
    uint32_t h = ((uint32_t)c * 2654435761u) >> (32 - 6);
    for (;;) {
      const int32_t v = tab[h * kAsmBlock];
      if (v == c) return;
      if (v < 0) {
        if (m == limit) {
          overflow = true;
          return;
        }
        tab[h * kAsmBlock] = c;
        ++m;
        return;
      }
      h = (h + 1) & (kHashSlots - 1);
    }
  }
  // moves the ids to slots 0 .. m-1 in ascending order (in place: the write
  // position never passes the slot being read)
  __device__ __forceinline__ void compact_sorted() {
    int w = 0;
    for (int k = 0; k < kHashSlots; ++k) {
      const int32_t v = tab[k * kAsmBlock];
      if (v < 0) continue;
      int j = w - 1;
      while (j >= 0 && tab[j * kAsmBlock] > v) {
        tab[(j + 1) * kAsmBlock] = tab[j * kAsmBlock];
        --j;
      }
      tab[(j + 1) * kAsmBlock] = v;
      ++w;
    }
  }
};
static_assert(kHashSlots == 64 && kShRow <= kColLine && kColLine < kHashSlots,
              "the hash takes the top 6 bits; a probe needs a free slot; a row fits its line");

template <class Set>
__device__ __forceinline__ void add_expanded(int32_t nd, const AsmView& A, Set& S) {
  if (nd < A.n) {
    S.add(nd);
    return;
  }
  const int64_t h = nd - A.n;
  const int4 p = A.hang_par[h];
  S.add(p.x);
  S.add(p.y);
  if (A.hang_np[h] == 4) {
    S.add(p.z);
    S.add(p.w);
  }
}

// Distinct columns of row i before Dirichlet elimination.
template <class Set>
__device__ __forceinline__ void row_columns(int64_t i, const AsmView& A, Set& S) {
  for (int64_t e = A.inc_ptr[i]; e < A.inc_ptr[i + 1]; ++e) {
    const uint32_t t = A.inc[e];
    const int64_t o = t >> 3;
    const int a = (int)(t & 7);
    add_expanded(A.oct_nodes[t], A, S);
    for (int d = 0; d < 3; ++d) add_expanded(A.oct_nodes[8 * o + (a ^ (1 << d))], A, S);
  }
}

template <class Set>
__device__ __forceinline__ int32_t live_columns(const Set& S, const AsmView& A) {
  int32_t m = 0;
  for (int j = 0; j < S.m; ++j) m += A.dirichlet[S.c_at(j)] ? 0 : 1;
  return m;
}

// Pass 1 (topology only): each row's distinct columns before Dirichlet
// elimination, sorted, into its line of `cols` (kColLine entries from
// i * kColLine), their number into ucnt, and the number of stored columns
// (Dirichlet columns removed) into rowlen.  A row with more than `limit`
// distinct columns gets ucnt = kWideRow and is counted by the local-memory
// set.  Thread k takes row order[k]: rows sorted by incidence count, so the
// lanes of a warp walk incidence lists of one length.
__global__ void __launch_bounds__(kAsmBlock) k_row_cols(AsmView A, const int32_t* __restrict__ order, int limit,
                                                        int32_t* __restrict__ rowlen, int32_t* __restrict__ cols,
                                                        uint8_t* __restrict__ ucnt, int* __restrict__ overflow) {
  __shared__ int32_t s_tab[kHashSlots * kAsmBlock];
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= A.n) return;
  const int64_t i = order[k];
  if (A.dirichlet[i]) {
    rowlen[i] = 1;
    ucnt[i] = 0;
    return;
  }
  HashSet S{s_tab + threadIdx.x, limit};
  S.clear();
  row_columns(i, A, S);
  if (!S.overflow) {
    S.compact_sorted();
    int32_t* line = cols + i * kColLine;
    int32_t live = 0;
    for (int j = 0; j < S.m; ++j) {
      const int32_t c = S.tab[j * kAsmBlock];
      line[j] = c;
      live += A.dirichlet[c] ? 0 : 1;
    }
    rowlen[i] = live;
    ucnt[i] = (uint8_t)S.m;
    return;
  }
  ColSet W;
  row_columns(i, A, W);
  if (W.overflow) atomicExch(overflow, 1);
  rowlen[i] = live_columns(W, A);
  ucnt[i] = kWideRow;
}

// Rows ordered by incidence count (keys of the ordering sort).
__global__ void k_inc_count_keys(const int64_t* __restrict__ inc_ptr, int64_t n, uint8_t* __restrict__ key,
                                 int32_t* __restrict__ id) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t c = inc_ptr[i + 1] - inc_ptr[i];
  key[i] = (uint8_t)(c < 255 ? c : 255);
  id[i] = (int32_t)i;
}

// Accumulator over a row's known sorted columns (the line pass 1 wrote),
// staged in shared memory with the values: an add finds its column by binary
// search and adds into the column's value slot.  The value slots start at
// -0.0, so the first add leaves exactly its own value, and every column sums
// its contributions in arrival order: the same values as the insertion
// accumulators.
struct LineAcc {
  int32_t* col;  // this thread's slot 0; slot k at col[k * kAsmBlock]
  double* val;
  int m;
  bool overflow = false;
  __device__ __forceinline__ int32_t c_at(int j) const { return col[j * kAsmBlock]; }
  __device__ __forceinline__ double v_at(int j) const { return val[j * kAsmBlock]; }
  // the line is 128-byte aligned: four columns per 16-byte load
  __device__ __forceinline__ void load(const int32_t* __restrict__ line) {
    const int4* l4 = reinterpret_cast<const int4*>(line);
    for (int j = 0; j < m; j += 4) {
      const int4 q = __ldg(l4 + (j >> 2));
      col[j * kAsmBlock] = q.x;
      if (j + 1 < m) col[(j + 1) * kAsmBlock] = q.y;
      if (j + 2 < m) col[(j + 2) * kAsmBlock] = q.z;
      if (j + 3 < m) col[(j + 3) * kAsmBlock] = q.w;
    }
    for (int j = 0; j < m; ++j) val[j * kAsmBlock] = -0.0;
  }
  __device__ __forceinline__ void add(int32_t c, double v) {
    int lo = 0, hi = m;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (col[mid * kAsmBlock] < c)
        lo = mid + 1;
      else
        hi = mid;
    }
    if (lo < m && col[lo * kAsmBlock] == c)
      val[lo * kAsmBlock] += v;
    else
      overflow = true;  // not in the line: cannot happen for lines of pass 1
  }
};

struct SellOut {
  const int64_t* slice_ptr;
  const int32_t* slice_w;
  const int32_t* iperm;
  const int32_t* perm;
  int32_t* scol;
  double* sval;
  double* b;
  double* dinv;
  int C;
  int G;  // columns per row stored contiguously (1, 2 or 4)
};

// Element j of SELL row p (slice width W).
__device__ __forceinline__ int64_t sell_index(const SellOut& S, int64_t p, int W, int j) {
  const int64_t sl = p / S.C;
  return sell_elem(S.slice_ptr[sl], W, S.C, S.G, (int)(p - sl * S.C), j);
}

// Row i (SELL position p, slice width W) from its accumulated entries:
// Dirichlet columns go to the right-hand side, the others are stored in
// ascending node order.  Returns the number of elements written.
template <bool RHS_ONLY, class Acc>
__device__ __forceinline__ int emit_row(const Acc& R, double rhs, int64_t p, int64_t i, int W, const AsmView& A,
                                        const SellOut& S) {
  int j = 0;
  double diag = 1.0;
  for (int u = 0; u < R.m; ++u) {
    const int32_t cn = R.c_at(u);
    const double v = R.v_at(u);
    if (A.dirichlet[cn]) {
      rhs -= v * A.gval[cn];
      continue;
    }
    if (RHS_ONLY) continue;
    if (cn == i) diag = v;
    const int64_t k = sell_index(S, p, W, j++);
    S.scol[k] = S.iperm[cn];
    S.sval[k] = v;
  }
  S.b[p] = rhs;
  if (!RHS_ONLY) S.dinv[p] = 1.0 / diag;
  return j;
}

// Pass 2: values, columns (SELL numbering), right-hand side, 1/diagonal.
// One thread per SELL position p < n (row perm[p]), so the 32 lanes of a warp
// fill one slice and every store of element j is one contiguous warp store.
__global__ void __launch_bounds__(kAsmBlock) k_row_fill(AsmView A, LocalView L, SellOut S,
                                                        const int32_t* __restrict__ cols,
                                                        const uint8_t* __restrict__ ucnt) {
  __shared__ int32_t s_col[kShRow * kAsmBlock];
  __shared__ double s_val[kShRow * kAsmBlock];
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= A.n) return;
  const int64_t i = S.perm[p];
  const int W = S.slice_w[p / S.C];
  int j = 0;
  if (A.dirichlet[i]) {
    S.b[p] = A.gval[i];
    const int64_t k = sell_index(S, p, W, j++);
    S.scol[k] = (int32_t)p;
    S.sval[k] = 1.0;
    S.dinv[p] = 1.0;
  } else {
    const uint8_t m = ucnt[i];
    bool done = false;
    double rhs;
    if (m != kWideRow) {
      LineAcc R{s_col + threadIdx.x, s_val + threadIdx.x, m};
      R.load(cols + i * kColLine);
      gather_row(i, A, L, R, rhs);
      if (!R.overflow) {
        j = emit_row<false>(R, rhs, p, i, W, A, S);
        done = true;
      }
    }
    if (!done) {
      RowAcc Q;
      gather_row(i, A, L, Q, rhs);
      j = emit_row<false>(Q, rhs, p, i, W, A, S);
    }
  }
  for (; j < W; ++j) {
    const int64_t k = sell_index(S, p, W, j);
    S.scol[k] = (int32_t)p;
    S.sval[k] = 0.0;
  }
}

// The right-hand side alone (new charges on an assembled system): the
// values are gathered again into a shared-memory insertion accumulator, for
// the Dirichlet columns' elimination.
template <int K>
__global__ void __launch_bounds__(kAsmBlock) k_row_rhs(AsmView A, LocalView L, SellOut S) {
  __shared__ int32_t s_col[K * kAsmBlock];
  __shared__ double s_val[K * kAsmBlock];
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= A.n) return;
  const int64_t i = S.perm[p];
  const int W = S.slice_w[p / S.C];
  if (A.dirichlet[i]) {
    S.b[p] = A.gval[i];
    return;
  }
  ShAcc<K> R{s_col + threadIdx.x, s_val + threadIdx.x};
  double rhs;
  gather_row(i, A, L, R, rhs);
  if (!R.overflow) {
    emit_row<true>(R, rhs, p, i, W, A, S);
  } else {
    RowAcc Q;
    gather_row(i, A, L, Q, rhs);
    emit_row<true>(Q, rhs, p, i, W, A, S);
  }
}

// a[1] = stored elements (the slice offsets' end), a[2] = overflow flag; a[0]
// holds nnz already
__global__ void k_asm_totals(const int64_t* __restrict__ slice_end, const int* __restrict__ ovf,
                             unsigned long long* __restrict__ a) {
  a[1] = (unsigned long long)*slice_end;
  a[2] = (unsigned long long)*ovf;
}

// Padding rows past n in the last slice.
__global__ void k_pad_rows(SellOut S, int64_t n, int64_t n_pad) {
  const int64_t p = n + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= n_pad) return;
  const int W = S.slice_w[p / S.C];
  for (int j = 0; j < W; ++j) {
    const int64_t k = sell_index(S, p, W, j);
    S.scol[k] = (int32_t)p;
    S.sval[k] = 0.0;
  }
  S.b[p] = 0.0;
  S.dinv[p] = 0.0;
}

// Dirichlet flags and values (src/pb_class.cpp:2113-2149, 3531-3571).
__global__ void k_dirichlet(const int4* __restrict__ node_xyz, int64_t n, int bc, double3 lo, double3 len,
                            const double4* __restrict__ atoms, int64_t na, double eps_in, double eps_out, double kappa,
                            uint8_t* __restrict__ dir, double* __restrict__ gval) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int4 p = node_xyz[i];
  const bool onb = bc != 0 && (p.w & 1);
  dir[i] = onb;
  double g = 0.0;
  if (onb) {
    const double x = coord(lo.x, len.x, p.x), y = coord(lo.y, len.y, p.y), z = coord(lo.z, len.z, p.z);
    if (bc == 2) {
      for (int64_t a = 0; a < na; ++a) {
        const double4 A = atoms[a];
        const double d = norm3d(A.x - x, A.y - y, A.z - z);
        g += A.w * exp(-kappa * d) / (d * eps_out);
      }
    } else if (bc == 3) {
      const double rs = 2.0;
      const double pout = eps_out * (1.0 + kappa * rs), pin = eps_in * rs;
      const double d = norm3d(x, y, z);
      g = d <= rs ? 1.0 / (pout * rs) + (rs - d) / (pin * d) : exp(kappa * (rs - d)) / (d * pout);
    }
  }
  gval[i] = g;
}

// Sort key for SELL-C-sigma: window, then longer rows first, then node id
// (radix sort is stable, so equal keys keep node order).
__global__ void k_sigma_keys(const int32_t* __restrict__ rowlen, int64_t n, int sigma, uint64_t* __restrict__ key,
                             int32_t* __restrict__ id) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t L = (uint32_t)min(rowlen[i], 0xffff);
  key[i] = ((uint64_t)(i / sigma) << 16) | (uint64_t)(0xffff - L);
  id[i] = (int32_t)i;
}

__global__ void k_sum_rowlen(const int32_t* __restrict__ rowlen, int64_t n, unsigned long long* __restrict__ total) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  unsigned long long v = i < n ? (unsigned long long)rowlen[i] : 0ull;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(total, v);
}

__global__ void k_identity(int32_t* __restrict__ perm, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) perm[i] = (int32_t)i;
}

__global__ void k_iperm(const int32_t* __restrict__ perm, int64_t n, int32_t* __restrict__ iperm) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p < n) iperm[perm[p]] = (int32_t)p;
}

__global__ void k_slice_width(const int32_t* __restrict__ perm, const int32_t* __restrict__ rowlen, int64_t n,
                              int64_t n_slices, int C, int G, bool pad, int32_t* __restrict__ w,
                              int64_t* __restrict__ elems) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n_slices) return;
  int mx = 1;
  for (int l = 0; l < C; ++l) {
    const int64_t p = s * C + l;
    if (p < n) mx = max(mx, rowlen[perm[p]]);
  }
  if (pad) mx = (mx + G - 1) / G * G;  // padded to whole groups: no tail columns
  w[s] = mx;
  elems[s] = (int64_t)mx * C;
}

// Slice widths padded to a multiple of the group (PBGPU_SELL_PAD=1), or the
// last W mod G columns of a slice stored one per lane with no padding.
static bool sell_pad() {
  const char* e = std::getenv("PBGPU_SELL_PAD");
  return e && e[0] == '1';
}

// The assembly's view of a context (dirichlet / gval must be current).
static AsmView asm_view(Context* c) {
  AsmView A;
  A.inc_ptr = c->inc_ptr.get();
  A.inc = c->inc.get();
  A.oct = c->oct.get();
  A.oct_nodes = c->oct_nodes.get();
  A.hang_par = c->hang_par.get();
  A.hang_np = c->hang_np.get();
  A.eps = c->eps.get();
  A.react = c->react.get();
  A.react_cell = c->model.stern_layer_surf == 1 ? c->react_cell.get() : nullptr;
  A.rho = c->rho.get();
  A.frac = c->frac.get();
  A.border_pos = c->border_pos.get();
  A.dirichlet = c->dirichlet.get();
  A.gval = c->gval.get();
  A.n = c->n;
  A.stern = c->model.stern_layer_surf == 1;
  for (int d = 0; d < 3; ++d) {
    A.lo[d] = c->lo[d];
    A.len[d] = c->len[d];
  }
  return A;
}

int run_assemble(Context* c, const pbgpu_sell_opts* o) {
  if (!c->have_markers) return c->fail(PBGPU_ERR_STATE, "assemble: create_markers has not run");
  if (!c->have_density) return c->fail(PBGPU_ERR_STATE, "assemble: create_density_map has not run");
  int C = (o && o->chunk > 0) ? o->chunk : 32;
  int sigma = (o && o->sigma > 0) ? o->sigma : 2048;
  int G = (o && o->group > 0) ? o->group : 4;
  if (C % 32 != 0 || C > 1024) return c->fail(PBGPU_ERR_ARG, "SELL chunk must be a multiple of 32, at most 1024");
  if (sigma % C != 0 && sigma != 1) return c->fail(PBGPU_ERR_ARG, "SELL sigma must be 1 or a multiple of the chunk");
  if (G != 1 && G != 2 && G != 4) return c->fail(PBGPU_ERR_ARG, "SELL group must be 1, 2 or 4");
  c->C = C;
  c->sigma = sigma;
  c->G = G;
  c->have_system = false;  // a failed re-assembly leaves no stale system behind
  c->have_phi = false;
  const int64_t n = c->n;
  const double3 lo = make_double3(c->lo[0], c->lo[1], c->lo[2]);
  const double3 len = make_double3(c->len[0], c->len[1], c->len[2]);
  PBGPU_CUDA(c, c->dirichlet.alloc(n));
  PBGPU_CUDA(c, c->gval.alloc(n));
  k_dirichlet<<<grid_for(n, 128), 128, 0, c->stream>>>(c->node_xyz.get(), n, c->model.bc_type, lo, len,
                                                        c->atoms.get(), c->na, c->eps_in, c->eps_out, c->kappa,
                                                        c->dirichlet.get(), c->gval.get());
  PBGPU_LAUNCHED(c);

  const AsmView A = asm_view(c);
  PBGPU_CUDA(c, c->rowlen.alloc(n));
  Scratch<int> ovf(c, kScAsmOvf);
  PBGPU_CUDA(c, ovf.alloc(1));
  PBGPU_CUDA(c, cudaMemsetAsync(ovf.get(), 0, sizeof(int), c->stream));
  // pass 1 walks the rows in order of incidence count (a one-byte radix sort)
  Scratch<uint8_t> okey(c, kScAsmOrdKey), okey2(c, kScAsmOrdKey2);
  Scratch<int32_t> oid(c, kScAsmOrdId), ord(c, kScAsmOrd);
  PBGPU_CUDA(c, okey.alloc(n));
  PBGPU_CUDA(c, okey2.alloc(n));
  PBGPU_CUDA(c, oid.alloc(n));
  PBGPU_CUDA(c, ord.alloc(n));
  k_inc_count_keys<<<grid_for(n, 256), 256, 0, c->stream>>>(c->inc_ptr.get(), n, okey.get(), oid.get());
  PBGPU_LAUNCHED(c);
  {
    size_t ob = 0;
    PBGPU_CUDA(c, cub::DeviceRadixSort::SortPairs(nullptr, ob, okey.get(), okey2.get(), oid.get(), ord.get(), (int)n,
                                                  0, 8, c->stream));
    PBGPU_CUDA(c, ensure_tmp(c, ob));
    PBGPU_CUDA(c, cub::DeviceRadixSort::SortPairs(c->tmp.get(), ob, okey.get(), okey2.get(), oid.get(), ord.get(),
                                                  (int)n, 0, 8, c->stream));
    c->launches += cub_radix_launches(n, 8);
  }
  Scratch<int32_t> ucols(c, kScAsmCols);
  Scratch<uint8_t> ucnt(c, kScAsmUcnt);
  PBGPU_CUDA(c, ucols.alloc(n * kColLine));
  PBGPU_CUDA(c, ucnt.alloc(n));
  // a row longer than kMaxRow keeps kMaxRow in rowlen and raises the flag,
  // which is read with the matrix size below, before any row is filled
  k_row_cols<<<grid_for(n, kAsmBlock), kAsmBlock, 0, c->stream>>>(A, ord.get(), asm_few_slots() ? kShFew : kShRow,
                                                                  c->rowlen.get(), ucols.get(), ucnt.get(), ovf.get());
  PBGPU_LAUNCHED(c);

  // SELL-C-sigma permutation
  const int64_t n_slices = (n + C - 1) / C, n_pad = n_slices * C;
  PBGPU_CUDA(c, c->perm.alloc(n_pad));
  PBGPU_CUDA(c, c->iperm.alloc(n_pad));
  if (sigma > 1) {
    Scratch<uint64_t> k0(c, kScAsmK0), k1(c, kScAsmK1);
    Scratch<int32_t> id0(c, kScAsmId0);
    PBGPU_CUDA(c, k0.alloc(n));
    PBGPU_CUDA(c, k1.alloc(n));
    PBGPU_CUDA(c, id0.alloc(n));
    k_sigma_keys<<<grid_for(n, 256), 256, 0, c->stream>>>(c->rowlen.get(), n, sigma, k0.get(), id0.get());
    PBGPU_LAUNCHED(c);
    size_t bytes = 0;
    PBGPU_CUDA(c, cub::DeviceRadixSort::SortPairs(nullptr, bytes, k0.get(), k1.get(), id0.get(), c->perm.get(), (int)n,
                                                  0, 64, c->stream));
    PBGPU_CUDA(c, ensure_tmp(c, bytes));
    PBGPU_CUDA(c, cub::DeviceRadixSort::SortPairs(c->tmp.get(), bytes, k0.get(), k1.get(), id0.get(), c->perm.get(),
                                                  (int)n, 0, 64, c->stream));
    c->launches += cub_radix_launches(n, 64);
  } else {
    k_identity<<<grid_for(n, 256), 256, 0, c->stream>>>(c->perm.get(), n);
    PBGPU_LAUNCHED(c);
  }
  k_iperm<<<grid_for(n, 256), 256, 0, c->stream>>>(c->perm.get(), n, c->iperm.get());
  PBGPU_LAUNCHED(c);
  PBGPU_CUDA(c, c->slice_w.alloc(n_slices));
  PBGPU_CUDA(c, c->slice_ptr.alloc(n_slices + 1));
  Scratch<int64_t> elems(c, kScAsmElems);
  PBGPU_CUDA(c, elems.alloc(n_slices + 1));
  PBGPU_CUDA(c, cudaMemsetAsync(elems.get(), 0, (n_slices + 1) * sizeof(int64_t), c->stream));
  k_slice_width<<<grid_for(n_slices, 128), 128, 0, c->stream>>>(c->perm.get(), c->rowlen.get(), n, n_slices, C, G,
                                                                 sell_pad(), c->slice_w.get(), elems.get());
  PBGPU_LAUNCHED(c);
  size_t bytes = 0;
  PBGPU_CUDA(c, cub::DeviceScan::ExclusiveSum(nullptr, bytes, elems.get(), c->slice_ptr.get(), n_slices + 1, c->stream));
  PBGPU_CUDA(c, ensure_tmp(c, bytes));
  PBGPU_CUDA(c, cub::DeviceScan::ExclusiveSum(c->tmp.get(), bytes, elems.get(), c->slice_ptr.get(), n_slices + 1,
                                              c->stream));
  c->launches += kCubScanLaunches;
  // nnz = sum of row lengths; the stored length, nnz and the overflow flag
  // come back in one read (the only host wait of the assembly)
  Scratch<unsigned long long> nnz_d(c, kScAsmNnz);
  PBGPU_CUDA(c, nnz_d.alloc(4));
  PBGPU_CUDA(c, cudaMemsetAsync(nnz_d.get(), 0, sizeof(unsigned long long), c->stream));
  k_sum_rowlen<<<grid_for(n, 256), 256, 0, c->stream>>>(c->rowlen.get(), n, nnz_d.get());
  PBGPU_LAUNCHED(c);
  k_asm_totals<<<1, 1, 0, c->stream>>>(c->slice_ptr.get() + n_slices, ovf.get(), nnz_d.get());
  PBGPU_LAUNCHED(c);
  unsigned long long tot[3] = {0, 0, 0};
  PBGPU_CUDA(c, readback(c, tot, nnz_d.get(), sizeof(tot)));
  const int64_t nnz = (int64_t)tot[0], total = (int64_t)tot[1];
  if (tot[2]) return c->fail(PBGPU_ERR_CAPACITY, "assemble: a matrix row has more than kMaxRow columns");
  c->n_slices = n_slices;
  c->sell_len = total;
  c->nnz = nnz;
  PBGPU_CUDA(c, c->scol.alloc(total));
  PBGPU_CUDA(c, c->sval.alloc(total));
  PBGPU_CUDA(c, c->b.alloc(n_pad));
  PBGPU_CUDA(c, c->dinv.alloc(n_pad));
  SellOut S{c->slice_ptr.get(), c->slice_w.get(), c->iperm.get(), c->perm.get(), c->scol.get(), c->sval.get(),
            c->b.get(), c->dinv.get(), C, G};
  // local coefficients of every octant, once
  Scratch<double> ocond(c, kScAsmCond), okd(c, kScAsmKd), ofr(c, kScAsmFr);
  PBGPU_CUDA(c, ocond.alloc(12 * c->n_oct));
  PBGPU_CUDA(c, okd.alloc(8 * c->n_oct));
  PBGPU_CUDA(c, ofr.alloc(8 * c->n_oct));
  k_octant_local<<<grid_for(c->n_oct, 128), 128, 0, c->stream>>>(A, c->n_oct, ocond.get(), okd.get(), ofr.get());
  PBGPU_LAUNCHED(c);
  const LocalView L{ocond.get(), okd.get(), ofr.get()};
  k_row_fill<<<grid_for(n, kAsmBlock), kAsmBlock, 0, c->stream>>>(A, L, S, ucols.get(), ucnt.get());
  PBGPU_LAUNCHED(c);
  ucols.release();  // 128 B per row, needed by the fill alone (freed in stream order)
  if (n_pad > n) {
    k_pad_rows<<<grid_for(n_pad - n, 128), 128, 0, c->stream>>>(S, n, n_pad);
    PBGPU_LAUNCHED(c);
  }
  c->have_system = true;
  c->bj_ready = false;
  c->have_phi = false;
  return PBGPU_OK;
}

// Right-hand side of the assembled system for the context's current atoms and
// density map (the matrix does not depend on the charges): Dirichlet values,
// the octants' V/8 rho terms and the eliminated Dirichlet columns, summed as
// in the full assembly.
int run_rhs(Context* c) {
  if (!c->have_system) return c->fail(PBGPU_ERR_STATE, "rhs: assemble has not run");
  if (!c->have_density) return c->fail(PBGPU_ERR_STATE, "rhs: create_density_map has not run");
  const int64_t n = c->n;
  const double3 lo = make_double3(c->lo[0], c->lo[1], c->lo[2]);
  const double3 len = make_double3(c->len[0], c->len[1], c->len[2]);
  k_dirichlet<<<grid_for(n, 128), 128, 0, c->stream>>>(c->node_xyz.get(), n, c->model.bc_type, lo, len,
                                                        c->atoms.get(), c->na, c->eps_in, c->eps_out, c->kappa,
                                                        c->dirichlet.get(), c->gval.get());
  PBGPU_LAUNCHED(c);
  const AsmView A = asm_view(c);
  SellOut S{c->slice_ptr.get(), c->slice_w.get(), c->iperm.get(), c->perm.get(), c->scol.get(), c->sval.get(),
            c->b.get(), c->dinv.get(), c->C, c->G};
  Scratch<double> ocond(c, kScAsmCond), okd(c, kScAsmKd), ofr(c, kScAsmFr);
  PBGPU_CUDA(c, ocond.alloc(12 * c->n_oct));
  PBGPU_CUDA(c, okd.alloc(8 * c->n_oct));
  PBGPU_CUDA(c, ofr.alloc(8 * c->n_oct));
  k_octant_local<<<grid_for(c->n_oct, 128), 128, 0, c->stream>>>(A, c->n_oct, ocond.get(), okd.get(), ofr.get());
  PBGPU_LAUNCHED(c);
  const LocalView L{ocond.get(), okd.get(), ofr.get()};
  if (asm_few_slots())
    k_row_rhs<kShFew><<<grid_for(n, kAsmBlock), kAsmBlock, 0, c->stream>>>(A, L, S);
  else
    k_row_rhs<kShRow><<<grid_for(n, kAsmBlock), kAsmBlock, 0, c->stream>>>(A, L, S);
  PBGPU_LAUNCHED(c);
  return PBGPU_OK;
}

// CSR (node order, ascending columns) of the assembled system, for parity checks.
int export_system(Context* c, int64_t* nnz_out, int64_t* row_ptr, int32_t* col, double* val, double* rhs) {
  if (!c->have_system) return c->fail(PBGPU_ERR_STATE, "get_system: assemble has not run");
  if (nnz_out) *nnz_out = c->nnz;
  if (!row_ptr && !col && !val && !rhs) return PBGPU_OK;
  const int64_t n = c->n, n_pad = c->n_slices * c->C;
  std::vector<int64_t> sp(c->n_slices + 1);
  std::vector<int32_t> sw(c->n_slices), perm(n_pad), iperm(n_pad), rl(n), sc(c->sell_len);
  std::vector<double> sv(c->sell_len), bb(n_pad);
  PBGPU_CUDA(c, cudaMemcpyAsync(sp.data(), c->slice_ptr.get(), sp.size() * 8, cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaMemcpyAsync(sw.data(), c->slice_w.get(), sw.size() * 4, cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaMemcpyAsync(perm.data(), c->perm.get(), n * 4, cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaMemcpyAsync(iperm.data(), c->iperm.get(), n * 4, cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaMemcpyAsync(rl.data(), c->rowlen.get(), n * 4, cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaMemcpyAsync(sc.data(), c->scol.get(), sc.size() * 4, cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaMemcpyAsync(sv.data(), c->sval.get(), sv.size() * 8, cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaMemcpyAsync(bb.data(), c->b.get(), n_pad * 8, cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  const int C = c->C;
  int64_t w = 0;
  if (row_ptr) row_ptr[0] = 0;
  std::vector<std::pair<int32_t, double>> row;
  for (int64_t i = 0; i < n; ++i) {
    const int64_t p = iperm[i];
    const int64_t s = p / C;
    const int lane = (int)(p % C);
    row.clear();
    for (int j = 0; j < rl[i]; ++j) {
      const int64_t k = sell_elem(sp[s], sw[s], C, c->G, lane, j);
      row.push_back({perm[sc[k]], sv[k]});
    }
    std::sort(row.begin(), row.end());
    for (auto& e : row) {
      if (col) col[w] = e.first;
      if (val) val[w] = e.second;
      ++w;
    }
    if (row_ptr) row_ptr[i + 1] = w;
    if (rhs) rhs[i] = bb[p];
  }
  return PBGPU_OK;
}

}  // namespace pbgpu
