// create_density_map on the device (src/pb_class.cpp:1944-2050, atom search
// :3633-3729) and the node -> (octant, corner) incidence lists that the patch
// volumes, the right-hand side and the matrix rows are gathered from.
//
// Every node-wise sum here is a gather in a fixed order (incidences sorted by
// octant, then corner; charge contributions sorted by atom, corner, parent), so
// results are deterministic and, compiled without FMA contraction, equal bit for
// bit to the sequential CPU restatement.
#include <cstdlib>
#include <cub/cub.cuh>

#include "pbgpu_internal.cuh"

namespace pbgpu {


__global__ void k_oct_keys(const int4* __restrict__ oct, int64_t n_oct, uint64_t* __restrict__ key) {
  const int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (o >= n_oct) return;
  const int4 q = oct[o];
  key[o] = morton3(q.x, q.y, q.z);
}

void launch_oct_keys(const int4* oct, int64_t n_oct, uint64_t* key, cudaStream_t s) {
  k_oct_keys<<<grid_for(n_oct, 256), 256, 0, s>>>(oct, n_oct, key);
}

__global__ void k_inc_count(const int32_t* __restrict__ oct_nodes, int64_t n8, int64_t n,
                            const int4* __restrict__ hang_par, const int8_t* __restrict__ hang_np,
                            int32_t* __restrict__ cnt) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n8) return;
  const int32_t nd = oct_nodes[t];
  if (nd < n) {
    atomicAdd(cnt + nd, 1);
    return;
  }
  const int64_t h = nd - n;
  const int4 p = hang_par[h];
  const int np = hang_np[h];
  atomicAdd(cnt + p.x, 1);
  atomicAdd(cnt + p.y, 1);
  if (np == 4) {
    atomicAdd(cnt + p.z, 1);
    atomicAdd(cnt + p.w, 1);
  }
}

__global__ void k_inc_fill(const int32_t* __restrict__ oct_nodes, int64_t n8, int64_t n,
                           const int4* __restrict__ hang_par, const int8_t* __restrict__ hang_np,
                           const int64_t* __restrict__ ptr, int32_t* __restrict__ cursor, uint32_t* __restrict__ inc) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n8) return;
  const int32_t nd = oct_nodes[t];
  if (nd < n) {
    inc[ptr[nd] + atomicAdd(cursor + nd, 1)] = (uint32_t)t;
    return;
  }
  const int64_t h = nd - n;
  const int4 p = hang_par[h];
  const int np = hang_np[h];
  inc[ptr[p.x] + atomicAdd(cursor + p.x, 1)] = (uint32_t)t;
  inc[ptr[p.y] + atomicAdd(cursor + p.y, 1)] = (uint32_t)t;
  if (np == 4) {
    inc[ptr[p.z] + atomicAdd(cursor + p.z, 1)] = (uint32_t)t;
    inc[ptr[p.w] + atomicAdd(cursor + p.w, 1)] = (uint32_t)t;
  }
}

// Sort each node's incidence list ascending.  The lists hold 8 entries for
// most nodes and a few dozen at most (parents of hanging nodes), so each
// thread sorts its list in shared memory (slot k of thread t at
// [k * kIncBlock + t], conflict-free across a warp) and writes it back once; a
// longer list is sorted in place in global memory (PBGPU_ASM_SLOTS=4 sets 4
// slots, which sends most lists down that path, for tests of it).
constexpr int kIncBlock = 128;
constexpr int kIncSh = 48;
constexpr int kIncFew = 4;

template <int K>
__global__ void __launch_bounds__(kIncBlock) k_inc_sort(const int64_t* __restrict__ ptr, uint32_t* __restrict__ inc,
                                                        int64_t n) {
  __shared__ uint32_t s_inc[K * kIncBlock];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t b = ptr[i], e = ptr[i + 1];
  if (e - b > K) {
    for (int64_t k = b + 1; k < e; ++k) {
      const uint32_t v = inc[k];
      int64_t j = k - 1;
      while (j >= b && inc[j] > v) {
        inc[j + 1] = inc[j];
        --j;
      }
      inc[j + 1] = v;
    }
    return;
  }
  uint32_t* my = s_inc + threadIdx.x;
  const int m = (int)(e - b);
  for (int k = 0; k < m; ++k) {
    const uint32_t v = inc[b + k];
    int j = k - 1;
    while (j >= 0 && my[j * kIncBlock] > v) {
      my[(j + 1) * kIncBlock] = my[j * kIncBlock];
      --j;
    }
    my[(j + 1) * kIncBlock] = v;
  }
  for (int k = 0; k < m; ++k) inc[b + k] = my[k * kIncBlock];
}

int build_incidence(Context* c) {
  if (c->have_incidence) return PBGPU_OK;
  const int64_t n = c->n, n8 = 8 * c->n_oct;
  if (n8 >= (int64_t(1) << 32)) return c->fail(PBGPU_ERR_CAPACITY, "too many octants for 32-bit incidence entries");
  Scratch<int32_t> cnt(c, kScDenCnt);
  PBGPU_CUDA(c, cnt.alloc(n + 1));
  PBGPU_CUDA(c, cudaMemsetAsync(cnt.get(), 0, (n + 1) * sizeof(int32_t), c->stream));
  k_inc_count<<<grid_for(n8, 256), 256, 0, c->stream>>>(c->oct_nodes.get(), n8, n, c->hang_par.get(),
                                                         c->hang_np.get(), cnt.get());
  PBGPU_LAUNCHED(c);
  PBGPU_CUDA(c, c->inc_ptr.alloc(n + 1));
  size_t bytes = 0;
  PBGPU_CUDA(c, cub::DeviceScan::ExclusiveSum(nullptr, bytes, cnt.get(), c->inc_ptr.get(), n + 1, c->stream));
  PBGPU_CUDA(c, ensure_tmp(c, bytes));
  PBGPU_CUDA(c, cub::DeviceScan::ExclusiveSum(c->tmp.get(), bytes, cnt.get(), c->inc_ptr.get(), n + 1, c->stream));
  c->launches += kCubScanLaunches;
  int64_t total = 0;
  PBGPU_CUDA(c, readback(c, &total, c->inc_ptr.get() + n, sizeof(int64_t)));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  PBGPU_CUDA(c, c->inc.alloc(total > 0 ? total : 1));
  PBGPU_CUDA(c, cudaMemsetAsync(cnt.get(), 0, (n + 1) * sizeof(int32_t), c->stream));
  k_inc_fill<<<grid_for(n8, 256), 256, 0, c->stream>>>(c->oct_nodes.get(), n8, n, c->hang_par.get(), c->hang_np.get(),
                                                        c->inc_ptr.get(), cnt.get(), c->inc.get());
  PBGPU_LAUNCHED(c);
  const char* few = std::getenv("PBGPU_ASM_SLOTS");
  if (few && std::atoi(few) == kIncFew)
    k_inc_sort<kIncFew><<<grid_for(n, kIncBlock), kIncBlock, 0, c->stream>>>(c->inc_ptr.get(), c->inc.get(), n);
  else
    k_inc_sort<kIncSh><<<grid_for(n, kIncBlock), kIncBlock, 0, c->stream>>>(c->inc_ptr.get(), c->inc.get(), n);
  PBGPU_LAUNCHED(c);
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  c->have_incidence = true;
  return PBGPU_OK;
}

struct Geo {
  double lo[3], len[3];
};

// Eighth of the octant volume, h = coord(upper) - coord(lower) per axis.
__device__ __forceinline__ double oct_v8(const int4 q, const Geo& g, double h[3]) {
  const int32_t s = 1 << (kRootLog - q.w);
  h[0] = coord(g.lo[0], g.len[0], q.x + s) - coord(g.lo[0], g.len[0], q.x);
  h[1] = coord(g.lo[1], g.len[1], q.y + s) - coord(g.lo[1], g.len[1], q.y);
  h[2] = coord(g.lo[2], g.len[2], q.z + s) - coord(g.lo[2], g.len[2], q.z);
  return h[0] * h[1] * h[2] * 0.125;
}

// vol_patch = sum over incident corners of V/8 (bim3a_rhs of ones); a hanging
// corner hands V/8/num_parents to each parent.
__global__ void k_vol_patch(int64_t n, const int64_t* __restrict__ ptr, const uint32_t* __restrict__ inc,
                            const int4* __restrict__ oct, const int32_t* __restrict__ oct_nodes,
                            const int8_t* __restrict__ hang_np, Geo g, double* __restrict__ vol_patch) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double acc = 0.0;
  for (int64_t e = ptr[i]; e < ptr[i + 1]; ++e) {
    const uint32_t t = inc[e];
    double h[3];
    const double v8 = oct_v8(oct[t >> 3], g, h);
    const int32_t nd = oct_nodes[t];
    if (nd < n)
      acc += v8;
    else
      acc += v8 / hang_np[nd - n];
  }
  vol_patch[i] = acc;
}

// Octant containing an atom: l - tol < p <= r - tol on every axis
// (controlla_coordinate, src/pb_class.cpp:3633-3676).
__global__ void k_locate_atoms(const double4* __restrict__ atoms, int64_t na, const uint64_t* __restrict__ oct_key,
                               const int4* __restrict__ oct, int64_t n_oct, Geo g, double tol,
                               int32_t* __restrict__ atom_oct) {
  const int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (a >= na) return;
  const double4 P = atoms[a];
  const double p[3] = {P.x, P.y, P.z};
  int32_t gi[3];
  for (int d = 0; d < 3; ++d) {
    double t = (p[d] + tol - g.lo[d]) / g.len[d] * (double)kRoot;
    if (!(t > -2.0)) t = -2.0;
    if (t > kRoot + 2.0) t = kRoot + 2.0;
    gi[d] = (int32_t)floor(t);
  }
  int32_t found = -1;
  for (int dz = -1; dz <= 1 && found < 0; ++dz)
    for (int dy = -1; dy <= 1 && found < 0; ++dy)
      for (int dx = -1; dx <= 1 && found < 0; ++dx) {
        const int32_t x = gi[0] + dx, y = gi[1] + dy, z = gi[2] + dz;
        if (x < 0 || y < 0 || z < 0 || x >= kRoot || y >= kRoot || z >= kRoot) continue;
        const uint64_t key = morton3(x, y, z);
        // upper_bound - 1
        int64_t lo = 0, hi = n_oct;
        while (lo < hi) {
          const int64_t mid = (lo + hi) >> 1;
          if (oct_key[mid] <= key)
            lo = mid + 1;
          else
            hi = mid;
        }
        const int64_t o = lo - 1;
        if (o < 0) continue;
        const int4 q = oct[o];
        const int32_t s = 1 << (kRootLog - q.w);
        const int32_t qc[3] = {q.x, q.y, q.z};
        bool in = true;
        for (int d = 0; d < 3 && in; ++d) {
          const double l = coord(g.lo[d], g.len[d], qc[d]), r = coord(g.lo[d], g.len[d], qc[d] + s);
          in = (p[d] > l - tol) && (p[d] <= r - tol);
        }
        if (in) found = (int32_t)o;
      }
  atom_oct[a] = found;
}

// Trilinear weight of corner c at point p in octant q (src/pb_class.cpp:2018-2021).
__device__ __forceinline__ double tri_weight(const int4 q, int c, const double p[3], const Geo& g, double volume) {
  const int32_t s = 1 << (kRootLog - q.w);
  const int o = 7 - c;
  const double X = coord(g.lo[0], g.len[0], q.x + (o & 1) * s);
  const double Y = coord(g.lo[1], g.len[1], q.y + ((o >> 1) & 1) * s);
  const double Z = coord(g.lo[2], g.len[2], q.z + ((o >> 2) & 1) * s);
  return fabs((p[0] - X) * (p[1] - Y) * (p[2] - Z)) / volume;
}

__device__ __forceinline__ double oct_volume(const int4 q, const Geo& g) {
  double h[3];
  oct_v8(q, g, h);
  return h[0] * h[1] * h[2];
}

// One slot per (atom, corner, parent): key = node << 32 | atom << 5 | corner << 2 | parent.
__global__ void k_charge_contrib(const double4* __restrict__ atoms, int64_t na, const int32_t* __restrict__ atom_oct,
                                 const int4* __restrict__ oct, const int32_t* __restrict__ oct_nodes, int64_t n,
                                 const int4* __restrict__ hang_par, const int8_t* __restrict__ hang_np,
                                 const double* __restrict__ vol_patch, Geo g, uint64_t* __restrict__ key,
                                 double* __restrict__ val) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= 8 * na) return;
  const int64_t a = t >> 3;
  const int c = (int)(t & 7);
  uint64_t* K = key + 4 * t;
  double* V = val + 4 * t;
  for (int j = 0; j < 4; ++j) {
    K[j] = kEmptyKey;
    V[j] = 0.0;
  }
  const int32_t o = atom_oct[a];
  if (o < 0) return;
  const double4 P = atoms[a];
  const double p[3] = {P.x, P.y, P.z};
  const int4 q = oct[o];
  const double w = tri_weight(q, c, p, g, oct_volume(q, g));
  const int32_t nd = oct_nodes[8 * (int64_t)o + c];
  const uint64_t low = ((uint64_t)a << 5) | ((uint64_t)c << 2);
  if (nd < n) {
    K[0] = ((uint64_t)nd << 32) | low;
    V[0] = P.w * 4.0 * kPi * w / vol_patch[nd];
    return;
  }
  const int64_t h = nd - n;
  const int4 pp = hang_par[h];
  const int np = hang_np[h];
  const int32_t par[4] = {pp.x, pp.y, pp.z, pp.w};
  for (int j = 0; j < np; ++j) {
    const double denom = np * vol_patch[par[j]];
    K[j] = ((uint64_t)par[j] << 32) | low | (uint64_t)j;
    V[j] = P.w * 4.0 * kPi * w / denom;
  }
}

// Sequential sum of each node's sorted contributions.
__global__ void k_segment_sum(const uint64_t* __restrict__ key, const double* __restrict__ val, int64_t m,
                              double* __restrict__ rho) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= m) return;
  const uint64_t k = key[t];
  if (k == kEmptyKey) return;
  const uint32_t node = (uint32_t)(k >> 32);
  if (t > 0 && (uint32_t)(key[t - 1] >> 32) == node) return;
  double acc = 0.0;
  for (int64_t u = t; u < m && key[u] != kEmptyKey && (uint32_t)(key[u] >> 32) == node; ++u) acc += val[u];
  rho[node] = acc;
}

int run_density(Context* c) {
  int st = build_incidence(c);
  if (st != PBGPU_OK) return st;
  const int64_t n = c->n, na = c->na;
  Geo g;
  for (int d = 0; d < 3; ++d) {
    g.lo[d] = c->lo[d];
    g.len[d] = c->len[d];
  }
  PBGPU_CUDA(c, c->vol_patch.alloc(n));
  PBGPU_CUDA(c, c->rho.alloc(n));
  k_vol_patch<<<grid_for(n, 256), 256, 0, c->stream>>>(n, c->inc_ptr.get(), c->inc.get(), c->oct.get(),
                                                        c->oct_nodes.get(), c->hang_np.get(), g, c->vol_patch.get());
  PBGPU_LAUNCHED(c);
  PBGPU_CUDA(c, cudaMemsetAsync(c->rho.get(), 0, n * sizeof(double), c->stream));
  PBGPU_CUDA(c, c->atom_oct.alloc(na > 0 ? na : 1));
  if (na > 0) {
    k_locate_atoms<<<grid_for(na, 128), 128, 0, c->stream>>>(c->atoms.get(), na, c->oct_key.get(), c->oct.get(),
                                                              c->n_oct, g, c->tol, c->atom_oct.get());
    PBGPU_LAUNCHED(c);
    const int64_t m = 32 * na;
    Scratch<uint64_t> k0(c, kScDenK0), k1(c, kScDenK1);
    Scratch<double> v0(c, kScDenV0), v1(c, kScDenV1);
    PBGPU_CUDA(c, k0.alloc(m));
    PBGPU_CUDA(c, k1.alloc(m));
    PBGPU_CUDA(c, v0.alloc(m));
    PBGPU_CUDA(c, v1.alloc(m));
    k_charge_contrib<<<grid_for(8 * na, 128), 128, 0, c->stream>>>(
        c->atoms.get(), na, c->atom_oct.get(), c->oct.get(), c->oct_nodes.get(), n, c->hang_par.get(),
        c->hang_np.get(), c->vol_patch.get(), g, k0.get(), v0.get());
    PBGPU_LAUNCHED(c);
    size_t bytes = 0;
    PBGPU_CUDA(c, cub::DeviceRadixSort::SortPairs(nullptr, bytes, k0.get(), k1.get(), v0.get(), v1.get(), (int)m, 0,
                                                  64, c->stream));
    PBGPU_CUDA(c, ensure_tmp(c, bytes));
    PBGPU_CUDA(c, cub::DeviceRadixSort::SortPairs(c->tmp.get(), bytes, k0.get(), k1.get(), v0.get(), v1.get(), (int)m,
                                                  0, 64, c->stream));
    c->launches += cub_radix_launches(m, 64);
    k_segment_sum<<<grid_for(m, 256), 256, 0, c->stream>>>(k1.get(), v1.get(), m, c->rho.get());
    PBGPU_LAUNCHED(c);
    PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  c->have_density = true;
  return PBGPU_OK;
}

}  // namespace pbgpu
