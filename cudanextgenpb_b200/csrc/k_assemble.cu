// assemple_system_matrix on the device (src/pb_class.cpp:2053-2159): the
// box-method operator of bimpp's bim3a_laplacian_frac + bim3a_reaction_frac
// (or bim3a_reaction with a Stern layer) + bim3a_rhs + bim3a_dirichlet_bc,
// written straight into a SELL-C-sigma matrix.
//
// Each matrix row is gathered by one thread from the node's incidence list
// (octant, corner), so no atomics touch the values.  The octants' local
// coefficients (12 edge conductances, 8 lumped diagonal terms, 8 V/8 * rho
// terms) are computed once per octant; per incidence the thread spreads the
// corner's terms over the independent nodes behind each local corner (a
// hanging corner over its parents with weight 1/num_parents: A = P^T K P),
// accumulating them in a per-thread hash map in shared memory.  Pass 1 runs
// in node order, so the rows of a warp share octants, and writes each row's
// distinct columns and values, sorted, into a line of its own; the SELL
// layout is derived from the row lengths (rows sorted by length inside
// windows of sigma rows, slices of C rows as wide as their longest row), and
// pass 2 copies the lines in SELL order, so every store is a warp-wide one.
// Dirichlet nodes become identity rows and are eliminated from the other rows
// into the right-hand side, which keeps the matrix symmetric.
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

// v / np for a hanging node's parent count: 2 and 4 (the counts a 2:1 tree
// has) are powers of two, so the product with 1/2 or 1/4 is the quotient
// exactly, without the cost of a double division.
__device__ __forceinline__ double div_np(double v, int np) {
  return np == 2 ? v * 0.5 : np == 4 ? v * 0.25 : v / np;
}

__device__ __forceinline__ double corner_val(const double* __restrict__ v, int32_t nd, const AsmView& A) {
  if (nd < A.n) return v[nd];
  const int64_t h = nd - A.n;
  const int4 p = A.hang_par[h];
  const int np = A.hang_np[h];
  double t = 0.0;
  t += div_np(v[p.x], np);
  t += div_np(v[p.y], np);
  if (np == 4) {
    t += div_np(v[p.z], np);
    t += div_np(v[p.w], np);
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
  const double wi = div_np(1.0, np);
  for (int j = 0; j < 4; ++j) w[j] = wi;
  return np;
}

// Threads per block of the row kernels; the shared-memory slot arrays below
// are laid out for exactly this many threads (slot k of thread t at
// [k * kAsmBlock + t], so the lanes of a warp hit distinct banks whichever
// slots they are at).
constexpr int kAsmBlock = 128;
// The gather pass writes each row's distinct columns, sorted, with their
// values into lines of kLine entries; rows of a 2:1 balanced octree hold at
// most ~25.  A row with more is gathered into the local-memory accumulator
// (kMaxRow slots) instead, in both passes.  PBGPU_ASM_SLOTS=4 lowers the limit
// to 4, which sends most rows down that path (for tests of it).
constexpr int kLine = 28;
constexpr int kHash = 32;  // hash slots per thread: more than kLine, so a probe always ends
constexpr int kGatherNB = 4;  // incidences whose loads a gather issues together (measured: 2: 12.3 ms, 4: 11.6 ms)
constexpr uint8_t kWideRow = 0xff;
constexpr int kShFew = 4;
static_assert(kLine < kHash && (kHash & (kHash - 1)) == 0, "a probe needs a free slot");

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

// Local box-method coefficients of every octant, computed once per octant
// with the expressions (and accumulation order) of the local matrix: the 12
// edge conductances wha(eps_i1, eps_i2, f) * area_h, the 8 diagonal entries
// (sum of the corner's 3 conductances in edge order, then the lumped reaction
// kappa_c * V/8 * w_c, w_c the product of the corner's half-edge shares), and
// the 8 right-hand-side terms V/8 * rho_c.
// 8 blocks of 128 per SM (64 registers): measured faster than the 108-register
// build at 4, its spills notwithstanding.
__global__ void __launch_bounds__(128, 8) k_octant_local(AsmView A, int64_t n_oct, double* __restrict__ cond,
                                                         double* __restrict__ kd, double* __restrict__ fr) {
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

// The 3 edges at corner a in ascending edge id, with their axes: the z edge
// (8-11) is always the last, the x and y edges (0-7) in either order.
__device__ __forceinline__ void corner_edges(int a, int ed[3], int ax[3]) {
  const int e0 = edge_of(a, 0), e1 = edge_of(a, 1);
  const bool sw = e1 < e0;
  ed[0] = sw ? e1 : e0;
  ax[0] = sw ? 1 : 0;
  ed[1] = sw ? e0 : e1;
  ax[1] = sw ? 0 : 1;
  ed[2] = edge_of(a, 2);
  ax[2] = 2;
}

// One incidence's loads: the corner's node and its 3 edge neighbours, the
// corner's diagonal term, the 3 edge conductances (negated) and V/8 rho.
struct IncLoads {
  int32_t nd[4];
  double k[4];
  double fr;
};

// t = 8 * octant + corner fits 32 bits (the incidence build checks 8 n_oct <
// 2^32), so the corner entries of t's octant are t with its low 3 bits
// replaced; the 12 conductances per octant need 64-bit offsets.
__device__ __forceinline__ void load_inc(uint32_t t, const AsmView& A, const LocalView& L, IncLoads& d) {
  const int a = (int)(t & 7);
  const uint32_t t0 = t & ~7u;
  const int64_t c0 = (int64_t)(t >> 3) * 12;
  int ed[3], ax[3];
  corner_edges(a, ed, ax);
  d.nd[0] = A.oct_nodes[t];
  d.k[0] = L.kd[t];
  d.fr = L.fr[t];
#pragma unroll
  for (int u = 0; u < 3; ++u) {
    d.nd[1 + u] = A.oct_nodes[t0 | (uint32_t)(a ^ (1 << ax[u]))];
    d.k[1 + u] = 0.0 - L.cond[c0 + ed[u]];
  }
}

template <class Acc>
__device__ __forceinline__ void apply_inc(const IncLoads& d, const AsmView& A, Acc& R, double& rhs) {
  const double wa = d.nd[0] < A.n ? 1.0 : div_np(1.0, A.hang_np[d.nd[0] - A.n]);
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    int32_t g[4];
    double w[4];
    const int ng = expand(d.nd[r], A, g, w);
    for (int j = 0; j < ng; ++j) R.add(g[j], wa * d.k[r] * w[j]);
  }
  rhs += wa * d.fr;
}

// Gather row i of A and its right-hand side entry (before Dirichlet handling)
// from the octants' local coefficients: A = P^T K P over the node's
// incidences, in incidence order (for each, the corner's own term, then its 3
// edges in ascending edge id, each spread over the independent nodes behind
// the node it reaches).  The loads of NB incidences are issued before any of
// them is accumulated.
template <int NB, class Acc>
__device__ void gather_row(int64_t i, const AsmView& A, const LocalView& L, Acc& R, double& rhs) {
  rhs = 0.0;
  const int64_t e0 = A.inc_ptr[i], e1 = A.inc_ptr[i + 1];
  for (int64_t e = e0; e < e1; e += NB) {
    IncLoads d[NB];
#pragma unroll
    for (int q = 0; q < NB; ++q) load_inc(A.inc[e + q < e1 ? e + q : e], A, L, d[q]);
#pragma unroll
    for (int q = 0; q < NB; ++q)
      if (e + q < e1) apply_inc(d[q], A, R, rhs);
  }
}

// (column, value) map of one thread in shared memory: open addressing over
// kHash slots (empty key = -1), at most `limit` (<= kLine) columns.  An add is
// a hash and usually one probe; a column's first add stores its value and
// later ones add to it, so each column sums its contributions in arrival
// order, exactly as the insertion accumulator does.
struct HashMap {
  int32_t* key;  // this thread's slot 0; slot k at key[k * kAsmBlock]
  double* val;
  int limit;
  int m = 0;
  bool overflow = false;
  __device__ __forceinline__ void clear() {
#pragma unroll 8
    for (int k = 0; k < kHash; ++k) key[k * kAsmBlock] = -1;
  }
  __device__ __forceinline__ void add(int32_t c, double v) {
    if (overflow) return;
    uint32_t h = ((uint32_t)c * 2654435761u) >> 27;  // top 5 bits: kHash = 32
    for (;;) {
      const int32_t k = key[h * kAsmBlock];
      if (k == c) {
        val[h * kAsmBlock] += v;
        return;
      }
      if (k < 0) {
        if (m == limit) {
          overflow = true;
          return;
        }
        key[h * kAsmBlock] = c;
        val[h * kAsmBlock] = v;
        ++m;
        return;
      }
      h = (h + 1) & (kHash - 1);
    }
  }
  // moves the entries to slots 0 .. m-1 in ascending column order (in place:
  // the write position never passes the slot being read)
  __device__ __forceinline__ void compact_sorted() {
    int w = 0;
    for (int s = 0; s < kHash; ++s) {
      const int32_t k = key[s * kAsmBlock];
      if (k < 0) continue;
      const double v = val[s * kAsmBlock];
      int j = w - 1;
      while (j >= 0 && key[j * kAsmBlock] > k) {
        key[(j + 1) * kAsmBlock] = key[j * kAsmBlock];
        val[(j + 1) * kAsmBlock] = val[j * kAsmBlock];
        --j;
      }
      key[(j + 1) * kAsmBlock] = k;
      val[(j + 1) * kAsmBlock] = v;
      ++w;
    }
  }
};
static_assert(kHash == 32, "HashMap::add takes the top 5 bits of the product");

// Pass 1: one thread per row in node order (neighbouring rows share octants,
// so their gathers meet in L1).  Each row's distinct columns, sorted, and
// their values (before Dirichlet elimination) go to its lines of `cols` and
// `vals` (kLine entries from i * kLine), their number to ucnt, the sum of its
// V/8 rho terms to rhs_part, and, unless rowlen is null (right-hand side
// only), the number of stored columns (Dirichlet columns removed) to rowlen.
// A row with more than `limit` columns gets ucnt = kWideRow and is gathered
// again by the second pass.
template <int NB>
__global__ void __launch_bounds__(kAsmBlock) k_row_gather(AsmView A, LocalView L, int limit,
                                                          int32_t* __restrict__ rowlen, int32_t* __restrict__ cols,
                                                          double* __restrict__ vals, double* __restrict__ rhs_part,
                                                          uint8_t* __restrict__ ucnt, int* __restrict__ overflow) {
  __shared__ int32_t s_key[kHash * kAsmBlock];
  __shared__ double s_val[kHash * kAsmBlock];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  if (A.dirichlet[i]) {
    if (rowlen) rowlen[i] = 1;
    ucnt[i] = 0;
    return;
  }
  HashMap R{s_key + threadIdx.x, s_val + threadIdx.x, limit};
  R.clear();
  double rhs;
  gather_row<NB>(i, A, L, R, rhs);
  int32_t live = 0;
  if (!R.overflow) {
    R.compact_sorted();
    int32_t* cl = cols + i * kLine;
    double* vl = vals + i * kLine;
    for (int j = 0; j < R.m; ++j) {
      const int32_t c = R.key[j * kAsmBlock];
      cl[j] = c;
      vl[j] = R.val[j * kAsmBlock];
      live += A.dirichlet[c] ? 0 : 1;
    }
    ucnt[i] = (uint8_t)R.m;
    rhs_part[i] = rhs;
  } else {
    RowAcc Q;
    gather_row<1>(i, A, L, Q, rhs);
    if (Q.overflow) atomicExch(overflow, 1);
    for (int j = 0; j < Q.m; ++j) live += A.dirichlet[Q.col[j]] ? 0 : 1;
    ucnt[i] = kWideRow;
  }
  if (rowlen) rowlen[i] = live;
}

// A row's lines as an accumulator view for emit_row.
struct LineView {
  const int32_t* col;
  const double* val;
  int m;
  __device__ __forceinline__ int32_t c_at(int j) const { return __ldg(col + j); }
  __device__ __forceinline__ double v_at(int j) const { return __ldg(val + j); }
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

// Pass 2: values, columns (SELL numbering), right-hand side, 1/diagonal, from
// the lines of pass 1.  One thread per SELL position p < n (row perm[p]), so
// the 32 lanes of a warp fill one slice and every store of element j is one
// contiguous warp store.  RHS_ONLY: the right-hand side alone (new charges on
// an assembled system).
template <bool RHS_ONLY>
__global__ void __launch_bounds__(kAsmBlock) k_row_emit(AsmView A, LocalView L, SellOut S,
                                                        const int32_t* __restrict__ cols,
                                                        const double* __restrict__ vals,
                                                        const double* __restrict__ rhs_part,
                                                        const uint8_t* __restrict__ ucnt) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= A.n) return;
  const int64_t i = S.perm[p];
  const int W = S.slice_w[p / S.C];
  int j = 0;
  if (A.dirichlet[i]) {
    S.b[p] = A.gval[i];
    if (RHS_ONLY) return;
    const int64_t k = sell_index(S, p, W, j++);
    S.scol[k] = (int32_t)p;
    S.sval[k] = 1.0;
    S.dinv[p] = 1.0;
  } else {
    const uint8_t m = ucnt[i];
    if (m != kWideRow) {
      const LineView R{cols + i * kLine, vals + i * kLine, m};
      j = emit_row<RHS_ONLY>(R, rhs_part[i], p, i, W, A, S);
    } else {
      RowAcc Q;
      double rhs;
      gather_row<1>(i, A, L, Q, rhs);
      j = emit_row<RHS_ONLY>(Q, rhs, p, i, W, A, S);
    }
    if (RHS_ONLY) return;
  }
  for (; j < W; ++j) {
    const int64_t k = sell_index(S, p, W, j);
    S.scol[k] = (int32_t)p;
    S.sval[k] = 0.0;
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
  // local coefficients of every octant, once
  Scratch<double> ocond(c, kScAsmCond), okd(c, kScAsmKd), ofr(c, kScAsmFr);
  PBGPU_CUDA(c, ocond.alloc(12 * c->n_oct));
  PBGPU_CUDA(c, okd.alloc(8 * c->n_oct));
  PBGPU_CUDA(c, ofr.alloc(8 * c->n_oct));
  k_octant_local<<<grid_for(c->n_oct, 128), 128, 0, c->stream>>>(A, c->n_oct, ocond.get(), okd.get(), ofr.get());
  PBGPU_LAUNCHED(c);
  const LocalView L{ocond.get(), okd.get(), ofr.get()};
  // pass 1: every row's columns and values into its lines (336 B per row,
  // freed after pass 2).  A row longer than kMaxRow raises the flag, which
  // is read with the matrix size below, before any row is written.
  Scratch<int32_t> lcols(c, kScAsmCols);
  Scratch<double> lvals(c, kScAsmVals), rpart(c, kScAsmRhs);
  Scratch<uint8_t> ucnt(c, kScAsmUcnt);
  PBGPU_CUDA(c, lcols.alloc(n * kLine));
  PBGPU_CUDA(c, lvals.alloc(n * kLine));
  PBGPU_CUDA(c, rpart.alloc(n));
  PBGPU_CUDA(c, ucnt.alloc(n));
  k_row_gather<kGatherNB><<<grid_for(n, kAsmBlock), kAsmBlock, 0, c->stream>>>(
      A, L, asm_few_slots() ? kShFew : kLine, c->rowlen.get(), lcols.get(), lvals.get(), rpart.get(), ucnt.get(),
      ovf.get());
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
  k_row_emit<false><<<grid_for(n, kAsmBlock), kAsmBlock, 0, c->stream>>>(A, L, S, lcols.get(), lvals.get(),
                                                                          rpart.get(), ucnt.get());
  PBGPU_LAUNCHED(c);
  lcols.release();  // freed in stream order, after pass 2
  lvals.release();
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
  Scratch<int32_t> lcols(c, kScAsmCols);
  Scratch<double> lvals(c, kScAsmVals), rpart(c, kScAsmRhs);
  Scratch<uint8_t> ucnt(c, kScAsmUcnt);
  Scratch<int> ovf(c, kScAsmOvf);
  PBGPU_CUDA(c, lcols.alloc(n * kLine));
  PBGPU_CUDA(c, lvals.alloc(n * kLine));
  PBGPU_CUDA(c, rpart.alloc(n));
  PBGPU_CUDA(c, ucnt.alloc(n));
  PBGPU_CUDA(c, ovf.alloc(1));
  k_row_gather<kGatherNB><<<grid_for(n, kAsmBlock), kAsmBlock, 0, c->stream>>>(
      A, L, asm_few_slots() ? kShFew : kLine, nullptr, lcols.get(), lvals.get(), rpart.get(), ucnt.get(), ovf.get());
  PBGPU_LAUNCHED(c);
  k_row_emit<true><<<grid_for(n, kAsmBlock), kAsmBlock, 0, c->stream>>>(A, L, S, lcols.get(), lvals.get(),
                                                                         rpart.get(), ucnt.get());
  PBGPU_LAUNCHED(c);
  lcols.release();
  lvals.release();
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
