// Mesh construction on the GPU: the surface refinement of the octree
// (refine_surface, src/pb_class.cpp:1468-1745), the node numbering with
// hanging nodes that p8est_nodes / tmesh_3d provide, and the ray crossing
// tables of the three axes (NanoShaper's ray cache, src/raytracer.cpp:379-467;
// here the analytic van der Waals union of spheres).  Starts from the initial
// octree of init_tmesh* (given by the host, or built here: a uniform octree
// refined inside a box) and leaves the context as pbgpu_set_mesh +
// pbgpu_set_rays would, with no host round trip of the mesh.
//
// Every step restates the host build (host/octree.cpp, host/surface.cpp,
// host/pb_class.cpp) with the same expressions, so the GPU and host meshes are
// identical: leaves stay in Morton order; the hanging-corner kernel finds
// neighbor cells in a hash table of the leaves (Morton key and level -> leaf
// index), the other lookups are binary searches on the sorted Morton keys;
// refinement splits marked leaves in place and
// restores 2:1 balance by ripple iterations from the split parents (refine)
// or the merged parents (coarsen); rays are cast through the spheres of one
// 2D bin per ray, the intervals sorted by (lo, hi) and merged.  Compiled
// without FMA contraction, so positions and normals are bit-identical.
#include <cub/cub.cuh>
#include <math_constants.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pbgpu_internal.cuh"

namespace pbgpu {

constexpr int kQMaxLevel = 18;  // P8EST_QMAXLEVEL

__device__ __forceinline__ int32_t qsize(int level) { return 1 << (kRootLog - level); }

__device__ __forceinline__ bool inside_root(int32_t x, int32_t y, int32_t z) {
  return x >= 0 && y >= 0 && z >= 0 && x < kRoot && y < kRoot && z < kRoot;
}

__device__ __forceinline__ int child_id(const int4 q) {
  const int s = kRootLog - q.w;
  return ((q.x >> s) & 1) | (((q.y >> s) & 1) << 1) | (((q.z >> s) & 1) << 2);
}

// last leaf whose key is <= the point's key (the leaf containing the point)
__device__ __forceinline__ int64_t find_leaf(const uint64_t* __restrict__ keys, int64_t n, int32_t x, int32_t y,
                                             int32_t z) {
  const uint64_t k = morton3((uint32_t)x, (uint32_t)y, (uint32_t)z);
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (keys[mid] <= k)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo - 1;
}

struct Tree {
  int4* leaves;
  uint64_t* keys;
  int64_t n;
  const uint64_t* hk;  // open-addressing table of (Morton key << 5 | level) of every leaf, or null
  const int32_t* hv;   // the leaf's index in each used slot of hk
  int cap_log;         // the table's capacity is 2^cap_log
};

__device__ __forceinline__ uint64_t leaf_hash_key(int32_t x, int32_t y, int32_t z, int level) {
  return (morton3((uint32_t)x, (uint32_t)y, (uint32_t)z) << 5) | (uint64_t)level;
}

// inserts every leaf and its index into the table (capacity at least twice
// the leaves; keys are distinct, one per leaf)
__global__ void k_leaf_hash(const int4* __restrict__ leaves, int64_t n, uint64_t* __restrict__ hk,
                            int32_t* __restrict__ hv, int cap_log) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int4 q = leaves[i];
  const uint64_t key = leaf_hash_key(q.x, q.y, q.z, q.w);
  const uint64_t mask = (1ull << cap_log) - 1;
  uint64_t s = hash_slot(key, cap_log);
  for (uint64_t probe = 0; probe <= mask; ++probe) {
    const unsigned long long prev =
        atomicCAS(reinterpret_cast<unsigned long long*>(hk + s), (unsigned long long)kEmptyKey, (unsigned long long)key);
    if (prev == kEmptyKey) {
      hv[s] = (int32_t)i;
      return;
    }
    s = (s + 1) & mask;
  }
}

// index of the leaf of `level` with lower corner (x, y, z), or -1
__device__ __forceinline__ int64_t leaf_index(const Tree& t, int32_t x, int32_t y, int32_t z, int level) {
  const uint64_t key = leaf_hash_key(x, y, z, level);
  const uint64_t mask = (1ull << t.cap_log) - 1;
  uint64_t s = hash_slot(key, t.cap_log);
  for (uint64_t probe = 0; probe <= mask; ++probe) {
    const uint64_t k = t.hk[s];
    if (k == key) return t.hv[s];
    if (k == kEmptyKey) return -1;
    s = (s + 1) & mask;
  }
  return -1;
}

__device__ __forceinline__ bool leaf_in_hash(const Tree& t, int32_t x, int32_t y, int32_t z, int level) {
  return leaf_index(t, x, y, z, level) >= 0;
}

// index of the leaf that contains the point (x, y, z) when that leaf's level
// is at most lmax, else -1 (the containing leaf is finer): one probe per
// level, from lmax down, as exactly one leaf contains the point
__device__ __forceinline__ int64_t containing_leaf_upto(const Tree& t, int32_t x, int32_t y, int32_t z, int lmax) {
  if (t.hk) {
    for (int l = lmax; l >= 0; --l) {
      const int32_t m = ~(qsize(l) - 1);
      const int64_t j = leaf_index(t, x & m, y & m, z & m, l);
      if (j >= 0) return j;
    }
    return -1;
  }
  const int64_t j = find_leaf(t.keys, t.n, x, y, z);
  return t.leaves[j].w <= lmax ? j : -1;
}

// is the cell of `level` with lower corner (x, y, z) (aligned to that level) a
// leaf: a table probe when the tree has its table, else a binary search
__device__ __forceinline__ bool is_leaf_at(const Tree& t, int32_t x, int32_t y, int32_t z, int level) {
  if (!inside_root(x, y, z)) return false;
  if (t.hk) return leaf_in_hash(t, x, y, z, level);
  return t.leaves[find_leaf(t.keys, t.n, x, y, z)].w == level;
}

__global__ void k_tree_keys(int4* __restrict__ leaves, int64_t n, uint64_t* __restrict__ keys) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) keys[i] = morton3(leaves[i].x, leaves[i].y, leaves[i].z);
}

// Are the 6 cells of `level` with lower corners (x[j], y[j], z[j]) leaves?  With
// the tree's table, the first probes of all 6 are loaded before any is
// resolved (a cell outside the root is not a leaf).
__device__ __forceinline__ void leaves_at6(const Tree& t, const int32_t (&x)[6], const int32_t (&y)[6],
                                           const int32_t (&z)[6], int level, bool (&out)[6]) {
  if (!t.hk) {
#pragma unroll
    for (int j = 0; j < 6; ++j) out[j] = is_leaf_at(t, x[j], y[j], z[j], level);
    return;
  }
  const uint64_t mask = (1ull << t.cap_log) - 1;
  uint64_t key[6], slot[6], first[6];
  bool in[6];
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    in[j] = inside_root(x[j], y[j], z[j]);
    key[j] = leaf_hash_key(x[j], y[j], z[j], level);
    slot[j] = hash_slot(key[j], t.cap_log);
  }
#pragma unroll
  for (int j = 0; j < 6; ++j) first[j] = in[j] ? t.hk[slot[j]] : kEmptyKey;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    bool found = false;
    if (in[j]) {
      uint64_t k = first[j], s = slot[j];
      for (uint64_t probe = 0; probe <= mask; ++probe) {
        if (k == key[j]) {
          found = true;
          break;
        }
        if (k == kEmptyKey) break;
        s = (s + 1) & mask;
        k = t.hk[s];
      }
    }
    out[j] = found;
  }
}

// Hanging corners (host Octree::hanging_masks): corner c of leaf q (child k of
// parent P) lies at a parent-edge midpoint when c ^ k has one bit set, at a
// parent-face centre when it has two; it hangs when a level-(L-1) cell
// sharing that edge (face) with P is a leaf.  Those cells lie on k's side of
// P on every axis: the 3 across P's faces and the 3 across its edges next to
// k.  A midpoint of P's edge along axis a hangs when the face cell across
// either other axis, or the edge cell across both, is a leaf; a face centre
// with normal axis a hangs when the face cell across a is.
__global__ void k_hanging(Tree t, uint8_t* __restrict__ mask) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= t.n) return;
  const int4 q = t.leaves[i];
  if (q.w == 0) {
    mask[i] = 0;
    return;
  }
  const int L = q.w;
  const int32_t PS = 1 << (kRootLog - L + 1);
  const int32_t P[3] = {q.x & ~(PS - 1), q.y & ~(PS - 1), q.z & ~(PS - 1)};
  const int k = child_id(q);
  int32_t off[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) off[a] = ((k >> a) & 1) ? PS : -PS;
  // cells 0-2: across the face normal to axis a; 3-5: across the edge along axis a
  int32_t cx[6], cy[6], cz[6];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    cx[a] = P[0] + (a == 0 ? off[0] : 0);
    cy[a] = P[1] + (a == 1 ? off[1] : 0);
    cz[a] = P[2] + (a == 2 ? off[2] : 0);
    cx[3 + a] = P[0] + (a == 0 ? 0 : off[0]);
    cy[3 + a] = P[1] + (a == 1 ? 0 : off[1]);
    cz[3 + a] = P[2] + (a == 2 ? 0 : off[2]);
  }
  bool leaf[6];
  leaves_at6(t, cx, cy, cz, L - 1, leaf);
  unsigned bits = 0;  // bit j: cell j is a leaf
#pragma unroll
  for (int j = 0; j < 6; ++j) bits |= leaf[j] ? 1u << j : 0u;
  uint8_t m8 = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int m = c ^ k;
    const int pc = __popc(m);
    unsigned need = 0;  // the cells that make corner c hang
    if (pc == 1) {
      const int a = __ffs(m) - 1;
      need = (1u << ((a + 1) % 3)) | (1u << ((a + 2) % 3)) | (1u << (3 + a));
    } else if (pc == 2) {
      need = 1u << (__ffs(~m & 7) - 1);
    }
    if (bits & need) m8 |= (uint8_t)(1u << c);
  }
  mask[i] = m8;
}

// ---------------------------------------------------------------------------
// Ray casting through the union of spheres (host SphereUnion::cast).

struct SphereBins {
  double o0, o1, cell;
  int n0, n1;
  const int32_t* start;  // n0 * n1 + 1
  const int32_t* items;
};

struct Spheres {
  const double4* s;  // x, y, z, r
  int64_t n;
  SphereBins bins[3];
};

struct RayDom {
  double lo[3], len[3];
};

__device__ __forceinline__ void transverse(int axis, int& t0, int& t1) {
  t0 = axis == 0 ? 1 : 0;
  t1 = axis == 2 ? 1 : 2;
}

__device__ __forceinline__ double comp(const double4& v, int a) { return a == 0 ? v.x : a == 1 ? v.y : v.z; }

// bin of the ray, -1 when the ray misses every bin
__device__ __forceinline__ int64_t ray_bin(const SphereBins& B, double u, double v) {
  const double f0 = (u - B.o0) / B.cell, f1 = (v - B.o1) / B.cell;
  if (f0 < 0 || f1 < 0) return -1;
  const int p = (int)f0, q = (int)f1;
  if (p >= B.n0 || q >= B.n1) return -1;
  return (int64_t)p * B.n1 + q;
}

// pass 1: intersecting spheres per ray
__global__ void k_cast_count(const uint64_t* __restrict__ keys, int64_t nk, int axis, Spheres S, RayDom D,
                             int64_t* __restrict__ cnt) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= nk) return;
  int t0, t1;
  transverse(axis, t0, t1);
  const uint64_t key = keys[r];
  const double u = coord(D.lo[t0], D.len[t0], (int32_t)(key >> 20));
  const double v = coord(D.lo[t1], D.len[t1], (int32_t)(key & 0xfffff));
  const SphereBins& B = S.bins[axis];
  int64_t m = 0;
  const int64_t bin = S.n ? ray_bin(B, u, v) : -1;
  if (bin >= 0)
    for (int32_t k = B.start[bin]; k < B.start[bin + 1]; ++k) {
      const double4 c = S.s[B.items[k]];
      const double d0 = u - comp(c, t0), d1 = v - comp(c, t1);
      const double s2 = c.w * c.w - (d0 * d0 + d1 * d1);
      m += s2 > 0;
    }
  cnt[r + 1] = m;
  if (r == 0) cnt[0] = 0;
}

struct Interval {
  double lo, hi;
  int32_t slo, shi;
};

// pass 2: the intervals of each ray at its offset
__global__ void k_cast_fill(const uint64_t* __restrict__ keys, int64_t nk, int axis, Spheres S, RayDom D,
                            const int64_t* __restrict__ off, Interval* __restrict__ iv) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= nk) return;
  int t0, t1;
  transverse(axis, t0, t1);
  const uint64_t key = keys[r];
  const double u = coord(D.lo[t0], D.len[t0], (int32_t)(key >> 20));
  const double v = coord(D.lo[t1], D.len[t1], (int32_t)(key & 0xfffff));
  const SphereBins& B = S.bins[axis];
  int64_t w = off[r];
  const int64_t bin = S.n ? ray_bin(B, u, v) : -1;
  if (bin < 0) return;
  for (int32_t k = B.start[bin]; k < B.start[bin + 1]; ++k) {
    const int32_t i = B.items[k];
    const double4 c = S.s[i];
    const double d0 = u - comp(c, t0), d1 = v - comp(c, t1);
    const double s2 = c.w * c.w - (d0 * d0 + d1 * d1);
    if (!(s2 > 0)) continue;
    const double sq = sqrt(s2);
    const double ca = comp(c, axis);
    iv[w++] = Interval{ca - sq, ca + sq, i, i};
  }
}

// pass 3: sort each ray's intervals by (lo, hi), keeping the fill order of
// equal ones, merge overlapping ones and write the crossings (position,
// sphere) at twice the ray's offset.  One warp per ray: the intervals are
// sorted in registers by a bitonic network on the key (lo, hi, fill index),
// which gives the order of a stable insertion sort, then lane 0 merges them.
// A ray of more than 128 intervals is sorted by lane 0 alone.

__device__ __forceinline__ bool iv_less(double alo, double ahi, int aid, double blo, double bhi, int bid) {
  return alo < blo || (alo == blo && (ahi < bhi || (ahi == bhi && aid < bid)));
}

template <int E>
__device__ __forceinline__ void iv_cmp_swap(double (&lo)[E], double (&hi)[E], int (&id)[E], int e, int f, bool up) {
  // positions e < f in this lane; ascending (up) keeps the smaller at e
  const bool fl = iv_less(lo[f], hi[f], id[f], lo[e], hi[e], id[e]);
  if (fl == up) {
    const double tl = lo[e], th = hi[e];
    const int ti = id[e];
    lo[e] = lo[f];
    hi[e] = hi[f];
    id[e] = id[f];
    lo[f] = tl;
    hi[f] = th;
    id[f] = ti;
  }
}

// bitonic sort of 32 * E keys, element g = lane * E + e
template <int E>
__device__ __forceinline__ void warp_bitonic_iv(double (&lo)[E], double (&hi)[E], int (&id)[E], int lane) {
  constexpr unsigned kFull = 0xffffffffu;
  for (int k = 2; k <= 32 * E; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j >= E) {
        const int lj = j / E;
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int g = lane * E + e;
          const double olo = __shfl_xor_sync(kFull, lo[e], lj);
          const double ohi = __shfl_xor_sync(kFull, hi[e], lj);
          const int oid = __shfl_xor_sync(kFull, id[e], lj);
          const bool up = (g & k) == 0, lower = (g & j) == 0;
          const bool other_less = iv_less(olo, ohi, oid, lo[e], hi[e], id[e]);
          if (lower == up ? other_less : !other_less) {
            lo[e] = olo;
            hi[e] = ohi;
            id[e] = oid;
          }
        }
      } else if (j == 1) {
#pragma unroll
        for (int e = 0; e < E; e += 2) iv_cmp_swap<E>(lo, hi, id, e, e + 1, ((lane * E + e) & k) == 0);
      } else if (E >= 4 && j == 2) {
#pragma unroll
        for (int e = 0; e < E; ++e)
          if ((e & 2) == 0) iv_cmp_swap<E>(lo, hi, id, e, e + 2, ((lane * E + e) & k) == 0);
      }
    }
  }
}

template <int E>
__device__ __forceinline__ void warp_sort_ray(Interval* a, int m, int lane) {
  double lo[E], hi[E];
  int id[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int g = lane * E + e;
    if (g < m) {
      lo[e] = a[g].lo;
      hi[e] = a[g].hi;
      id[e] = g;
    } else {
      lo[e] = CUDART_INF;
      hi[e] = CUDART_INF;
      id[e] = 0x7fffffff;
    }
  }
  warp_bitonic_iv<E>(lo, hi, id, lane);
  Interval v[E];
#pragma unroll
  for (int e = 0; e < E; ++e)
    if (lane * E + e < m) v[e] = a[id[e]];
  __syncwarp();
#pragma unroll
  for (int e = 0; e < E; ++e)
    if (lane * E + e < m) a[lane * E + e] = v[e];
  __syncwarp();
}

__global__ void k_cast_merge(int64_t nk, const int64_t* __restrict__ off, Interval* __restrict__ iv,
                             double* __restrict__ xs, int32_t* __restrict__ xsph, int64_t* __restrict__ ncr) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= nk) return;  // whole warps: blockDim is a multiple of 32
  Interval* a = iv + off[r];
  const int m = (int)(off[r + 1] - off[r]);
  if (m > 128) {
    if (lane == 0) {
      for (int i = 1; i < m; ++i) {
        const Interval e = a[i];
        int j = i - 1;
        while (j >= 0 && (a[j].lo > e.lo || (a[j].lo == e.lo && a[j].hi > e.hi))) {
          a[j + 1] = a[j];
          --j;
        }
        a[j + 1] = e;
      }
    }
    __syncwarp();
  } else if (m > 64) {
    warp_sort_ray<4>(a, m, lane);
  } else if (m > 32) {
    warp_sort_ray<2>(a, m, lane);
  } else if (m > 1) {
    warp_sort_ray<1>(a, m, lane);
  }
  if (lane != 0) return;
  int64_t w = 2 * off[r];
  int64_t nc = 0;
  if (m > 0) {
    Interval cur = a[0];
    for (int k = 1; k < m; ++k) {
      if (a[k].lo <= cur.hi) {
        if (a[k].hi > cur.hi) {
          cur.hi = a[k].hi;
          cur.shi = a[k].shi;
        }
      } else {
        xs[w] = cur.lo;
        xsph[w++] = cur.slo;
        xs[w] = cur.hi;
        xsph[w++] = cur.shi;
        nc += 2;
        cur = a[k];
      }
    }
    xs[w] = cur.lo;
    xsph[w++] = cur.slo;
    xs[w] = cur.hi;
    xsph[w++] = cur.shi;
    nc += 2;
  }
  ncr[r + 1] = nc;
  if (r == 0) ncr[0] = 0;
}

// pass 4: compact crossings (and their outward normals) by ray
__global__ void k_cast_emit(const uint64_t* __restrict__ keys, int64_t nk, int axis, Spheres S, RayDom D,
                            const int64_t* __restrict__ off, const double* __restrict__ xs,
                            const int32_t* __restrict__ xsph, const int64_t* __restrict__ coff,
                            double* __restrict__ inters, double* __restrict__ normals) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= nk) return;
  int t0, t1;
  transverse(axis, t0, t1);
  const uint64_t key = keys[r];
  const double u = coord(D.lo[t0], D.len[t0], (int32_t)(key >> 20));
  const double v = coord(D.lo[t1], D.len[t1], (int32_t)(key & 0xfffff));
  const int64_t src = 2 * off[r], dst = coff[r], m = coff[r + 1] - coff[r];
  for (int64_t j = 0; j < m; ++j) {
    const double x = xs[src + j];
    inters[dst + j] = x;
    if (normals) {
      const double4 c = S.s[xsph[src + j]];
      double pnt[3];
      pnt[axis] = x;
      pnt[t0] = u;
      pnt[t1] = v;
      normals[3 * (dst + j) + 0] = (pnt[0] - c.x) / c.w;
      normals[3 * (dst + j) + 1] = (pnt[1] - c.y) / c.w;
      normals[3 * (dst + j) + 2] = (pnt[2] - c.z) / c.w;
    }
  }
}

// ---------------------------------------------------------------------------
// Surface classification of the corners (host corner_inside_z) and the
// refinement / coarsening marks of refine_surface.

__global__ void k_zcol_count(Tree t, const uint8_t* __restrict__ hm, int64_t* __restrict__ cnt) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= t.n) return;
  int m = 0;
  for (int col = 0; col < 4; ++col) m += !((hm[i] >> col & 1) && (hm[i] >> (col + 4) & 1));
  cnt[i + 1] = m;
  if (i == 0) cnt[0] = 0;
}

__global__ void k_zcol_fill(Tree t, const uint8_t* __restrict__ hm, const int64_t* __restrict__ off,
                            uint64_t* __restrict__ keys) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= t.n) return;
  const int4 q = t.leaves[i];
  const int32_t s = qsize(q.w);
  int64_t w = off[i];
  for (int col = 0; col < 4; ++col) {
    if ((hm[i] >> col & 1) && (hm[i] >> (col + 4) & 1)) continue;
    keys[w++] = ray_key(q.x + (col & 1) * s, q.y + ((col >> 1) & 1) * s);
  }
}

__device__ __forceinline__ int64_t find_key(const uint64_t* __restrict__ keys, int64_t n, uint64_t k) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (keys[mid] < k)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo < n && keys[lo] == k) ? lo : -1;
}

// mode 0: refine marks (level < maxlevel, corners on both sides); mode 1:
// coarsen marks (level > minlevel, all corners on one side)
__global__ void k_surface_marks(Tree t, const uint8_t* __restrict__ hm, const uint64_t* __restrict__ rkeys,
                                int64_t nr, const int64_t* __restrict__ coff, const double* __restrict__ inters,
                                RayDom D, int mode, int minlevel, int maxlevel, uint8_t* __restrict__ marks) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= t.n) return;
  const int4 q = t.leaves[i];
  marks[i] = 0;
  if (mode == 0 ? q.w >= maxlevel : q.w <= minlevel) return;
  const int32_t s = qsize(q.w);
  const double z0 = coord(D.lo[2], D.len[2], q.z), z1 = coord(D.lo[2], D.len[2], q.z + s);
  double mn = 2.0, mxv = 0.0;
  for (int col = 0; col < 4; ++col) {
    const bool h0 = hm[i] >> col & 1, h1 = hm[i] >> (col + 4) & 1;
    if (h0 && h1) continue;
    const int64_t r = find_key(rkeys, nr, ray_key(q.x + (col & 1) * s, q.y + ((col >> 1) & 1) * s));
    const double* I = r >= 0 ? inters + coff[r] : nullptr;
    const int m = r >= 0 ? (int)(coff[r + 1] - coff[r]) : 0;
    for (int h = 0; h < 2; ++h) {
      if (h ? h1 : h0) continue;
      const double z = h ? z1 : z0;
      int k = 0;
      while (k < m && z >= I[k]) ++k;
      const double v = (double)(k & 1);
      mxv = fmax(mxv, v);
      mn = fmin(mn, v);
    }
  }
  if (mode == 0)
    marks[i] = (mxv > 0.5 && mn < 0.5) && q.w < kQMaxLevel;
  else
    marks[i] = mn > 0.5 || mxv < 0.5;
}

// ---------------------------------------------------------------------------
// The initial octree of init_tmesh* (src/pb_class.cpp:1290-1391): a uniform
// octree, then box refinement (host Octree::uniform and refine_in_box).

// leaf i of the uniform octree at `level`, in Morton order
__global__ void k_uniform(int level, int64_t n, int4* __restrict__ leaves) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t x = 0, y = 0, z = 0;
  for (int b = 0; b < level; ++b) {
    x |= (uint32_t)((i >> (3 * b)) & 1) << b;
    y |= (uint32_t)((i >> (3 * b + 1)) & 1) << b;
    z |= (uint32_t)((i >> (3 * b + 2)) & 1) << b;
  }
  const int32_t s = qsize(level);
  leaves[i] = make_int4((int32_t)x * s, (int32_t)y * s, (int32_t)z * s, level);
}

// refine marks of one box-refinement pass: leaves below `level` with a
// non-hanging corner inside the closed box [bl, br]
__global__ void k_box_marks(Tree t, const uint8_t* __restrict__ hm, RayDom D, double3 bl, double3 br, int level,
                            uint8_t* __restrict__ marks) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= t.n) return;
  const int4 q = t.leaves[i];
  uint8_t m = 0;
  if (q.w < level) {
    const int32_t s = qsize(q.w);
    for (int c = 0; c < 8 && !m; ++c) {
      if (hm[i] >> c & 1) continue;
      const double x = coord(D.lo[0], D.len[0], q.x + (c & 1) * s);
      const double y = coord(D.lo[1], D.len[1], q.y + ((c >> 1) & 1) * s);
      const double z = coord(D.lo[2], D.len[2], q.z + ((c >> 2) & 1) * s);
      m = x >= bl.x && x <= br.x && y >= bl.y && y <= br.y && z >= bl.z && z <= br.z;
    }
  }
  marks[i] = m;
}

// ---------------------------------------------------------------------------
// Split / merge / balance.

__global__ void k_split_count(const uint8_t* __restrict__ marks, int64_t n, int64_t* __restrict__ cnt) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  cnt[i + 1] = marks[i] ? 8 : 1;
  if (i == 0) cnt[0] = 0;
}

__global__ void k_split_fill(const int4* __restrict__ in, const uint8_t* __restrict__ marks, int64_t n,
                             const int64_t* __restrict__ off, int4* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int4 q = in[i];
  const int64_t w = off[i];
  if (!marks[i]) {
    out[w] = q;
    return;
  }
  const int32_t h = qsize(q.w) >> 1;
  for (int c = 0; c < 8; ++c)
    out[w + c] = make_int4(q.x + (c & 1) * h, q.y + ((c >> 1) & 1) * h, q.z + ((c >> 2) & 1) * h, q.w + 1);
}

// The balance kernels give each seed a group of kBalLanes lanes, which split
// the seed's neighbour lookups (each a binary search over the leaf keys)
// between them: on a small tree the grid is a fraction of one wave, and the
// kernel takes as long as one thread's chain of dependent lookups.
constexpr int kBalLanes = 8;

// a leaf X is too coarse when a level-(l+1) cell touching it from outside is
// itself refined (host touches_too_fine).  The cells to look at: per axis,
// offset -h (the side below), 0 or h (alongside, two half cells) or S (the
// side above), every combination but the 8 inside X, 56 in all; lane r of the
// group looks at combinations r, r + kBalLanes, ...
__device__ bool touches_too_fine_part(const Tree& t, const int4 X, int r) {
  const int32_t h = qsize(X.w) >> 1;
  for (int u = r; u < 64; u += kBalLanes) {
    // offset (a - 1) h for a = 0 .. 3: -h, 0, h, S
    const int a0 = u & 3, a1 = (u >> 2) & 3, a2 = (u >> 4) & 3;
    if ((a0 == 1 || a0 == 2) && (a1 == 1 || a1 == 2) && (a2 == 1 || a2 == 2)) continue;
    const int32_t sx = X.x + (a0 - 1) * h, sy = X.y + (a1 - 1) * h, sz = X.z + (a2 - 1) * h;
    if (!inside_root(sx, sy, sz)) continue;
    if (containing_leaf_upto(t, sx, sy, sz, X.w + 1) < 0) return true;
  }
  return false;
}

__device__ __forceinline__ void mark_once(uint8_t* marks, int64_t j) {
  // byte flags set with a word-wide OR (other threads mark the neighbouring bytes)
  unsigned* word = reinterpret_cast<unsigned*>(marks + (j & ~int64_t(3)));
  atomicOr(word, 1u << (8 * (j & 3)));
}

__global__ void k_balance_coarse(Tree t, const int4* __restrict__ seeds, int64_t ns, uint8_t* __restrict__ marks) {
  const int64_t gt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t s = gt / kBalLanes;
  const int r = (int)(gt % kBalLanes);
  if (s >= ns) return;
  const int4 P = seeds[s];
  const int32_t sz = qsize(P.w);
  for (int u = r; u < 27; u += kBalLanes) {
    if (u == 13) continue;  // the seed itself
    const int dx = u % 3 - 1, dy = (u / 3) % 3 - 1, dz = u / 9 - 1;
    const int32_t nx = P.x + dx * sz, ny = P.y + dy * sz, nz = P.z + dz * sz;
    if (!inside_root(nx, ny, nz)) continue;
    const int64_t j = containing_leaf_upto(t, nx, ny, nz, P.w - 1);
    if (j >= 0) mark_once(marks, j);
  }
}

// every lane of the grid reaches the group vote: the block size is a multiple
// of 32 and kBalLanes divides 32, so groups never straddle warps
__global__ void k_balance_fine(Tree t, const int4* __restrict__ seeds, int64_t ns, uint8_t* __restrict__ marks) {
  const int64_t gt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t s = gt / kBalLanes;
  const int r = (int)(gt % kBalLanes);
  bool active = s < ns;
  int64_t j = -1;
  int4 X = make_int4(0, 0, 0, 0);
  if (active) {
    X = seeds[s];
    if (t.hk) {
      j = leaf_index(t, X.x, X.y, X.z, X.w);
      active = j >= 0;  // else no longer a leaf
    } else {
      j = find_leaf(t.keys, t.n, X.x, X.y, X.z);
      const int4 L = t.leaves[j];
      active = L.w == X.w && L.x == X.x && L.y == X.y && L.z == X.z;
    }
  }
  const bool hit = active && touches_too_fine_part(t, X, r);
  const unsigned group = ((1u << kBalLanes) - 1u) << ((threadIdx.x & 31) & ~(kBalLanes - 1));
  const unsigned any = __ballot_sync(0xffffffffu, hit) & group;
  if (any && r == 0) mark_once(marks, j);
}

__global__ void k_parent_of(int4* __restrict__ q, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) q[i].w -= 1;  // a family's first child shares its parent's lower corner
}

__global__ void k_children(const int4* __restrict__ parents, int64_t np, int4* __restrict__ kids) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= np) return;
  const int4 P = parents[p];
  const int32_t h = qsize(P.w) >> 1;
  for (int c = 0; c < 8; ++c)
    kids[8 * p + c] = make_int4(P.x + (c & 1) * h, P.y + ((c >> 1) & 1) * h, P.z + ((c >> 2) & 1) * h, P.w + 1);
}

// families of 8 marked siblings (host Octree::coarsen): start flags
__global__ void k_family_start(Tree t, const uint8_t* __restrict__ marks, uint8_t* __restrict__ fam) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= t.n) return;
  const int4 q = t.leaves[i];
  bool f = q.w > 0 && child_id(q) == 0 && i + 7 < t.n;
  if (f) {
    const int32_t h = qsize(q.w);
    for (int c = 0; c < 8 && f; ++c) {
      const int4 o = t.leaves[i + c];
      f = marks[i + c] && o.w == q.w && o.x == q.x + (c & 1) * h && o.y == q.y + ((c >> 1) & 1) * h &&
          o.z == q.z + ((c >> 2) & 1) * h;
    }
  }
  fam[i] = f;
}

// output count per leaf: 1 for a family start (its parent) or a leaf outside
// every family, 0 for the other 7 family members
__global__ void k_merge_count(const uint8_t* __restrict__ fam, int64_t n, int64_t* __restrict__ cnt) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  bool covered = false;
  for (int d = 1; d <= 7 && !covered; ++d) covered = i - d >= 0 && fam[i - d];
  cnt[i + 1] = (fam[i] || !covered) ? 1 : 0;
  if (i == 0) cnt[0] = 0;
}

__global__ void k_merge_fill(const int4* __restrict__ in, const uint8_t* __restrict__ fam, int64_t n,
                             const int64_t* __restrict__ off, int4* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n || off[i + 1] == off[i]) return;
  const int4 q = in[i];
  out[off[i]] = fam[i] ? make_int4(q.x, q.y, q.z, q.w - 1) : q;
}

// ---------------------------------------------------------------------------
// Nodes (host Octree::build_nodes).

__global__ void k_indep_count(Tree t, const uint8_t* __restrict__ hm, int64_t* __restrict__ cnt) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= t.n) return;
  const int4 q = t.leaves[i];
  const int32_t s = qsize(q.w);
  int c0 = 0;
  for (int c = 0; c < 8; ++c) {
    if (hm[i] >> c & 1) continue;
    const int32_t p[3] = {q.x + (c & 1) * s, q.y + ((c >> 1) & 1) * s, q.z + ((c >> 2) & 1) * s};
    bool own = true;
    for (int a = 0; a < 3; ++a)
      if (((c >> a) & 1) && p[a] != kRoot) own = false;
    c0 += own;
  }
  cnt[i + 1] = c0;
  if (i == 0) cnt[0] = 0;
}

__global__ void k_indep_fill(Tree t, const uint8_t* __restrict__ hm, const int64_t* __restrict__ off,
                             uint64_t* __restrict__ codes) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= t.n) return;
  const int4 q = t.leaves[i];
  const int32_t s = qsize(q.w);
  int64_t w = off[i];
  for (int c = 0; c < 8; ++c) {
    if (hm[i] >> c & 1) continue;
    const int32_t p[3] = {q.x + (c & 1) * s, q.y + ((c >> 1) & 1) * s, q.z + ((c >> 2) & 1) * s};
    bool own = true;
    for (int a = 0; a < 3; ++a)
      if (((c >> a) & 1) && p[a] != kRoot) own = false;
    if (own) codes[w++] = morton3(p[0], p[1], p[2]);
  }
}

__global__ void k_hang_count(Tree t, const uint8_t* __restrict__ hm, int64_t* __restrict__ cnt) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= t.n) return;
  cnt[i + 1] = __popc(hm[i]);
  if (i == 0) cnt[0] = 0;
}

__global__ void k_hang_fill(Tree t, const uint8_t* __restrict__ hm, const int64_t* __restrict__ off,
                            uint64_t* __restrict__ codes) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= t.n) return;
  const int4 q = t.leaves[i];
  const int32_t s = qsize(q.w);
  int64_t w = off[i];
  for (int c = 0; c < 8; ++c)
    if (hm[i] >> c & 1) codes[w++] = morton3(q.x + (c & 1) * s, q.y + ((c >> 1) & 1) * s, q.z + ((c >> 2) & 1) * s);
}

__device__ __forceinline__ void decode_morton(uint64_t k, int32_t out[3]) {
  uint32_t v[3] = {0, 0, 0};
  for (int b = 0; b < 21; ++b)
    for (int a = 0; a < 3; ++a) v[a] |= (uint32_t)((k >> (3 * b + a)) & 1) << b;
  out[0] = (int32_t)v[0];
  out[1] = (int32_t)v[1];
  out[2] = (int32_t)v[2];
}

// node coordinates with the boundary flag of pbgpu_set_mesh
__global__ void k_node_xyz(const uint64_t* __restrict__ codes, int64_t n, int4* __restrict__ xyz) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= n) return;
  int32_t p[3];
  decode_morton(codes[j], p);
  int flag = 0;
  for (int a = 0; a < 3; ++a)
    if (p[a] == 0 || p[a] == kRoot) flag = 1;
  xyz[j] = make_int4(p[0], p[1], p[2], flag);
}

// Index of each of K keys in the n sorted, distinct codes, or -1: K branch-free
// binary searches in lockstep, so the K loads of every halving step are in
// flight together.  The answer stays in [base, base + len): a step keeps the
// upper part when its first code is <= the key, else the lower one.
template <int K>
__device__ __forceinline__ void code_index_k(const uint64_t* __restrict__ codes, int64_t n, const uint64_t (&key)[K],
                                             int64_t (&idx)[K]) {
  if (n <= 0) {
#pragma unroll
    for (int c = 0; c < K; ++c) idx[c] = -1;
    return;
  }
  int64_t base[K];
#pragma unroll
  for (int c = 0; c < K; ++c) base[c] = 0;
  for (int64_t len = n; len > 1;) {
    const int64_t half = len >> 1;
#pragma unroll
    for (int c = 0; c < K; ++c) base[c] = codes[base[c] + half] <= key[c] ? base[c] + half : base[c];
    len -= half;
  }
#pragma unroll
  for (int c = 0; c < K; ++c) idx[c] = codes[base[c]] == key[c] ? base[c] : -1;
}

// corner node ids; for hanging corners also the parents (every leaf that
// touches a hanging node writes the same values)
__global__ void k_corner_nodes(Tree t, const uint8_t* __restrict__ hm, const uint64_t* __restrict__ codes,
                               int64_t n_indep, const uint64_t* __restrict__ hcodes, int64_t n_hang,
                               int32_t* __restrict__ oct_nodes, int4* __restrict__ hang_par,
                               int8_t* __restrict__ hang_np, int* __restrict__ bad) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= t.n) return;
  const int4 q = t.leaves[i];
  const int32_t s = qsize(q.w);
  const int k = q.w > 0 ? child_id(q) : 0;
  const unsigned hang = hm[i];
  uint64_t key[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) key[c] = morton3(q.x + (c & 1) * s, q.y + ((c >> 1) & 1) * s, q.z + ((c >> 2) & 1) * s);
  int64_t ji[8], jh[8];
  code_index_k<8>(codes, n_indep, key, ji);
  if (hang) {
    code_index_k<8>(hcodes, n_hang, key, jh);
  } else {
#pragma unroll
    for (int c = 0; c < 8; ++c) jh[c] = -1;
  }
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    if (!(hang >> c & 1)) {
      if (ji[c] < 0) *bad = 1;
      oct_nodes[8 * i + c] = (int32_t)ji[c];
      continue;
    }
    const int64_t h = jh[c];
    if (h < 0) *bad = 1;
    oct_nodes[8 * i + c] = (int32_t)(n_indep + h);
    const int32_t PS = 1 << (kRootLog - q.w + 1);
    const int32_t P[3] = {q.x & ~(PS - 1), q.y & ~(PS - 1), q.z & ~(PS - 1)};
    const int m = c ^ k;
    // the parent's corners on the hanging node's edge (2) or face (4), in
    // corner order: those that agree with the hanging point on every axis
    // where it sits on the parent's boundary
    uint64_t pkey[4];
    int np = 0;
    for (int pc = 0; pc < 8; ++pc) {
      bool on = true;
      for (int a = 0; a < 3; ++a) {
        if ((m >> a) & 1) continue;
        const int want = (((k >> a) & 1) + ((c >> a) & 1)) / 2;
        if (((pc >> a) & 1) != want) on = false;
      }
      if (!on || np == 4) continue;
      pkey[np++] = morton3(P[0] + (pc & 1) * PS, P[1] + ((pc >> 1) & 1) * PS, P[2] + ((pc >> 2) & 1) * PS);
    }
    if (np == 0) {  // not a hanging point of this leaf's parent
      *bad = 1;
      continue;
    }
    for (int u = np; u < 4; ++u) pkey[u] = pkey[0];
    int64_t pj[4];
    code_index_k<4>(codes, n_indep, pkey, pj);
    int32_t par[4];
    for (int u = 0; u < np; ++u) {
      if (pj[u] < 0) *bad = 1;
      par[u] = (int32_t)pj[u];
    }
    // ascending; padded with the first parent as pbgpu_set_mesh stores them
    for (int a = 1; a < np; ++a)
      for (int b = a; b > 0 && par[b - 1] > par[b]; --b) {
        const int32_t tmp = par[b];
        par[b] = par[b - 1];
        par[b - 1] = tmp;
      }
    if (h >= 0) {
      hang_np[h] = (int8_t)np;
      hang_par[h] = make_int4(par[0], np > 1 ? par[1] : par[0], np > 2 ? par[2] : par[0], np > 3 ? par[3] : par[0]);
    }
  }
}

// transverse ray keys of every node point (independent and hanging) for one axis
__global__ void k_node_ray_keys(const int4* __restrict__ xyz, int64_t n, const uint64_t* __restrict__ hcodes,
                                int64_t nh, int axis, uint64_t* __restrict__ keys) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= n + nh) return;
  int32_t p[3];
  if (j < n) {
    const int4 v = xyz[j];
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
  } else {
    decode_morton(hcodes[j - n], p);
  }
  const int t0 = axis == 0 ? 1 : 0, t1 = axis == 2 ? 1 : 2;
  keys[j] = ray_key(p[t0], p[t1]);
}

__global__ void k_has_cross(const int64_t* __restrict__ coff, int64_t nk, uint8_t* __restrict__ flag) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r < nk) flag[r] = coff[r + 1] > coff[r];
}

// keys and crossing offsets of the rays that have crossings (rays without
// any add nothing to the offsets, so coff at a kept ray is its offset)
__global__ void k_gather_keys(const int64_t* __restrict__ sel, int64_t ns, const uint64_t* __restrict__ keys,
                              const int64_t* __restrict__ coff, int64_t nk, uint64_t* __restrict__ out_keys,
                              int64_t* __restrict__ ptr) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j > ns) return;
  if (j == ns) {
    ptr[ns] = coff[nk];
    return;
  }
  out_keys[j] = keys[sel[j]];
  ptr[j] = coff[sel[j]];
}

}  // namespace pbgpu

// ===========================================================================
// Host driver.

namespace pbgpu {
namespace {

struct BinsHost {
  double o0 = 0, o1 = 0;
  int n0 = 1, n1 = 1;
  std::vector<int32_t> start, items;
};

// 2D bins of the spheres over each axis' transverse plane, with the
// expressions of the host SphereUnion::build (cell = twice the largest radius)
void build_bins(const std::vector<double4>& sp, double& cell, BinsHost B[3]) {
  double rmax = 0;
  for (const double4& s : sp) rmax = std::max(rmax, s.w);
  cell = rmax > 0 ? 2.0 * rmax : 1.0;
  const int64_t n = (int64_t)sp.size();
  auto cmp = [](const double4& v, int a) { return a == 0 ? v.x : a == 1 ? v.y : v.z; };
  for (int axis = 0; axis < 3; ++axis) {
    const int t0 = axis == 0 ? 1 : 0, t1 = axis == 2 ? 1 : 2;
    BinsHost& b = B[axis];
    if (n == 0) {
      b.n0 = b.n1 = 1;
      b.start.assign(2, 0);
      b.items.clear();
      continue;
    }
    double mn0 = 1e300, mx0 = -1e300, mn1 = 1e300, mx1 = -1e300;
    for (const double4& s : sp) {
      mn0 = std::min(mn0, cmp(s, t0) - s.w);
      mx0 = std::max(mx0, cmp(s, t0) + s.w);
      mn1 = std::min(mn1, cmp(s, t1) - s.w);
      mx1 = std::max(mx1, cmp(s, t1) + s.w);
    }
    b.o0 = mn0;
    b.o1 = mn1;
    b.n0 = std::max(1, int((mx0 - mn0) / cell) + 1);
    b.n1 = std::max(1, int((mx1 - mn1) / cell) + 1);
    std::vector<int32_t> cnt(size_t(b.n0) * b.n1 + 1, 0);
    auto range = [&](const double4& s, int& a0, int& a1, int& c0, int& c1) {
      a0 = std::max(0, int((cmp(s, t0) - s.w - b.o0) / cell));
      a1 = std::min(b.n0 - 1, int((cmp(s, t0) + s.w - b.o0) / cell));
      c0 = std::max(0, int((cmp(s, t1) - s.w - b.o1) / cell));
      c1 = std::min(b.n1 - 1, int((cmp(s, t1) + s.w - b.o1) / cell));
    };
    for (const double4& s : sp) {
      int a0, a1, c0, c1;
      range(s, a0, a1, c0, c1);
      for (int p = a0; p <= a1; ++p)
        for (int q = c0; q <= c1; ++q) cnt[size_t(p) * b.n1 + q + 1]++;
    }
    for (size_t k = 1; k < cnt.size(); ++k) cnt[k] += cnt[k - 1];
    b.start = cnt;
    b.items.assign(cnt.back(), 0);
    std::vector<int32_t> fill(cnt.begin(), cnt.end() - 1);
    for (int64_t i = 0; i < n; ++i) {
      int a0, a1, c0, c1;
      range(sp[i], a0, a1, c0, c1);
      for (int p = a0; p <= a1; ++p)
        for (int q = c0; q <= c1; ++q) b.items[fill[size_t(p) * b.n1 + q]++] = int32_t(i);
    }
  }
}

struct Builder {
  Context* c;
  Spheres S{};
  RayDom D{};
  DBuf<double4> sph;
  DBuf<int32_t> bstart[3], bitems[3];
  // the tree (double-buffered)
  DBuf<int4> leaves, leaves2;
  DBuf<uint64_t> keys;
  int64_t n = 0;
  DBuf<uint8_t> marks, hm, fam;
  DBuf<int64_t> cnt, off;
  DBuf<int> bad;

  // table of the current leaves for exact-cell lookups (k_hanging), rebuilt
  // on first use after the tree changes
  DBuf<uint64_t> lhash;
  DBuf<int32_t> lhval;
  int lhash_log = 0;
  bool lhash_ok = false;

  Tree tree() { return Tree{leaves.get(), keys.get(), n, nullptr, nullptr, 0}; }

  int hashed_tree(Tree* t) {
    if (!lhash_ok) {
      int lg = 4;
      while ((int64_t(1) << lg) < 2 * n) ++lg;
      PBGPU_CUDA(c, lhash.alloc(size_t(1) << lg));
      PBGPU_CUDA(c, lhval.alloc(size_t(1) << lg));
      PBGPU_CUDA(c, cudaMemsetAsync(lhash.get(), 0xff, (size_t(1) << lg) * sizeof(uint64_t), st()));
      k_leaf_hash<<<grid_for(n, 256), 256, 0, st()>>>(leaves.get(), n, lhash.get(), lhval.get(), lg);
      PBGPU_LAUNCHED(c);
      lhash_log = lg;
      lhash_ok = true;
    }
    *t = Tree{leaves.get(), keys.get(), n, lhash.get(), lhval.get(), lhash_log};
    return PBGPU_OK;
  }
  cudaStream_t st() const { return c->stream; }

  int fail_cuda(cudaError_t e, const char* what) { return cuda_fail(c, e, what); }

  // inclusive scan of cnt[0 .. m] (cnt[0] = 0) into off; returns off[m]
  int scan(int64_t m, int64_t* total) {
    size_t bytes = 0;
    PBGPU_CUDA(c, cub::DeviceScan::InclusiveSum(nullptr, bytes, cnt.get(), off.get(), m + 1, st()));
    PBGPU_CUDA(c, ensure_tmp(c, bytes));
    PBGPU_CUDA(c, cub::DeviceScan::InclusiveSum(c->tmp.get(), bytes, cnt.get(), off.get(), m + 1, st()));
    c->launches += kCubScanLaunches;
    PBGPU_CUDA(c, readback(c, total, off.get() + m, sizeof(int64_t)));
    PBGPU_CUDA(c, cudaStreamSynchronize(st()));
    return PBGPU_OK;
  }

  int ensure_counts(int64_t m) {
    PBGPU_CUDA(c, cnt.alloc(m + 1));
    PBGPU_CUDA(c, off.alloc(m + 1));
    return PBGPU_OK;
  }

  int rekey() {
    lhash_ok = false;
    PBGPU_CUDA(c, keys.alloc(n > 0 ? n : 1));
    k_tree_keys<<<grid_for(n, 256), 256, 0, st()>>>(leaves.get(), n, keys.get());
    PBGPU_LAUNCHED(c);
    return PBGPU_OK;
  }

  // sort + unique of m keys in `k` (reordered in place) that use the low
  // `bits` bits (40 for ray keys, 60 for Morton codes of node points); *nu unique
  int sort_unique(DBuf<uint64_t>& k, int64_t m, int64_t* nu, int bits) {
    DBuf<uint64_t> k2;
    DBuf<int64_t> nsel;
    PBGPU_CUDA(c, k2.alloc(m > 0 ? m : 1));
    PBGPU_CUDA(c, nsel.alloc(1));
    if (m == 0) {
      *nu = 0;
      return PBGPU_OK;
    }
    size_t bytes = 0;
    PBGPU_CUDA(c, cub::DeviceRadixSort::SortKeys(nullptr, bytes, k.get(), k2.get(), (int)m, 0, bits, st()));
    PBGPU_CUDA(c, ensure_tmp(c, bytes));
    PBGPU_CUDA(c, cub::DeviceRadixSort::SortKeys(c->tmp.get(), bytes, k.get(), k2.get(), (int)m, 0, bits, st()));
    c->launches += cub_radix_launches(m, bits);
    bytes = 0;
    PBGPU_CUDA(c, cub::DeviceSelect::Unique(nullptr, bytes, k2.get(), k.get(), nsel.get(), (int)m, st()));
    PBGPU_CUDA(c, ensure_tmp(c, bytes));
    PBGPU_CUDA(c, cub::DeviceSelect::Unique(c->tmp.get(), bytes, k2.get(), k.get(), nsel.get(), (int)m, st()));
    c->launches += kCubSelectLaunches;
    PBGPU_CUDA(c, readback(c, nu, nsel.get(), sizeof(int64_t)));
    PBGPU_CUDA(c, cudaStreamSynchronize(st()));
    return PBGPU_OK;
  }

  // casts the nk sorted rays `rk` of one axis: crossing offsets coff (nk + 1),
  // positions and (optionally) normals, compact in ray order
  int cast(const uint64_t* rk, int64_t nk, int axis, DBuf<int64_t>& coff, DBuf<double>& inters,
           DBuf<double>* normals) {
    PBGPU_CUDA(c, coff.alloc(nk + 1));
    if (nk == 0) {
      PBGPU_CUDA(c, cudaMemsetAsync(coff.get(), 0, sizeof(int64_t), st()));
      return PBGPU_OK;
    }
    int rc;
    if ((rc = ensure_counts(nk)) != PBGPU_OK) return rc;
    k_cast_count<<<grid_for(nk, 128), 128, 0, st()>>>(rk, nk, axis, S, D, cnt.get());
    PBGPU_LAUNCHED(c);
    int64_t ni = 0;
    if ((rc = scan(nk, &ni)) != PBGPU_OK) return rc;
    DBuf<Interval> iv;
    DBuf<double> xs;
    DBuf<int32_t> xsph;
    DBuf<int64_t> ioff, ncr;
    PBGPU_CUDA(c, iv.alloc(ni > 0 ? ni : 1));
    PBGPU_CUDA(c, xs.alloc(2 * ni > 0 ? 2 * ni : 1));
    PBGPU_CUDA(c, xsph.alloc(2 * ni > 0 ? 2 * ni : 1));
    PBGPU_CUDA(c, ioff.alloc(nk + 1));
    PBGPU_CUDA(c, ncr.alloc(nk + 1));
    PBGPU_CUDA(c, cudaMemcpyAsync(ioff.get(), off.get(), (nk + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice, st()));
    k_cast_fill<<<grid_for(nk, 128), 128, 0, st()>>>(rk, nk, axis, S, D, ioff.get(), iv.get());
    PBGPU_LAUNCHED(c);
    k_cast_merge<<<grid_for(32 * nk, 128), 128, 0, st()>>>(nk, ioff.get(), iv.get(), xs.get(), xsph.get(), ncr.get());
    PBGPU_LAUNCHED(c);
    PBGPU_CUDA(c, cudaMemcpyAsync(cnt.get(), ncr.get(), (nk + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice, st()));
    int64_t nc = 0;
    if ((rc = scan(nk, &nc)) != PBGPU_OK) return rc;
    PBGPU_CUDA(c, cudaMemcpyAsync(coff.get(), off.get(), (nk + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice, st()));
    PBGPU_CUDA(c, inters.alloc(nc > 0 ? nc : 1));
    if (normals) PBGPU_CUDA(c, normals->alloc(3 * nc > 0 ? 3 * nc : 1));
    k_cast_emit<<<grid_for(nk, 128), 128, 0, st()>>>(rk, nk, axis, S, D, ioff.get(), xs.get(), xsph.get(),
                                                     coff.get(), inters.get(), normals ? normals->get() : nullptr);
    PBGPU_LAUNCHED(c);
    return PBGPU_OK;
  }

  int hanging() {
    PBGPU_CUDA(c, hm.alloc(n > 0 ? n : 1));
    Tree t;
    const int rc = hashed_tree(&t);
    if (rc != PBGPU_OK) return rc;
    k_hanging<<<grid_for(n, 128), 128, 0, st()>>>(t, hm.get());
    PBGPU_LAUNCHED(c);
    return PBGPU_OK;
  }

  // refine (mode 0) or coarsen (mode 1) marks from the z-ray classification
  int surface_marks(int mode, int minlevel, int maxlevel) {
    int rc;
    if ((rc = hanging()) != PBGPU_OK) return rc;
    if ((rc = ensure_counts(n)) != PBGPU_OK) return rc;
    k_zcol_count<<<grid_for(n, 256), 256, 0, st()>>>(tree(), hm.get(), cnt.get());
    PBGPU_LAUNCHED(c);
    int64_t nzk = 0;
    if ((rc = scan(n, &nzk)) != PBGPU_OK) return rc;
    DBuf<uint64_t> zk;
    PBGPU_CUDA(c, zk.alloc(nzk > 0 ? nzk : 1));
    k_zcol_fill<<<grid_for(n, 256), 256, 0, st()>>>(tree(), hm.get(), off.get(), zk.get());
    PBGPU_LAUNCHED(c);
    int64_t nu = 0;
    if ((rc = sort_unique(zk, nzk, &nu, kRayKeyBits)) != PBGPU_OK) return rc;
    DBuf<int64_t> coff;
    DBuf<double> inters;
    if ((rc = cast(zk.get(), nu, 2, coff, inters, nullptr)) != PBGPU_OK) return rc;
    PBGPU_CUDA(c, marks.alloc((n + 3) & ~int64_t(3)));
    k_surface_marks<<<grid_for(n, 128), 128, 0, st()>>>(tree(), hm.get(), zk.get(), nu, coff.get(), inters.get(), D,
                                                        mode, minlevel, maxlevel, marks.get());
    PBGPU_LAUNCHED(c);
    return PBGPU_OK;
  }

  // split the marked leaves; `parents` receives the split leaves (in order)
  int split(DBuf<int4>& parents, int64_t* np) {
    int rc;
    if ((rc = ensure_counts(n)) != PBGPU_OK) return rc;
    k_split_count<<<grid_for(n, 256), 256, 0, st()>>>(marks.get(), n, cnt.get());
    PBGPU_LAUNCHED(c);
    int64_t nn = 0;
    if ((rc = scan(n, &nn)) != PBGPU_OK) return rc;
    if (nn == n) {  // nothing marked: the tree stays as it is
      *np = 0;
      return PBGPU_OK;
    }
    DBuf<int64_t> nsel;
    PBGPU_CUDA(c, nsel.alloc(1));
    PBGPU_CUDA(c, parents.alloc(n > 0 ? n : 1));
    size_t bytes = 0;
    PBGPU_CUDA(c, cub::DeviceSelect::Flagged(nullptr, bytes, leaves.get(), marks.get(), parents.get(), nsel.get(),
                                             (int)n, st()));
    PBGPU_CUDA(c, ensure_tmp(c, bytes));
    PBGPU_CUDA(c, cub::DeviceSelect::Flagged(c->tmp.get(), bytes, leaves.get(), marks.get(), parents.get(),
                                             nsel.get(), (int)n, st()));
    c->launches += kCubSelectLaunches;
    // every split leaf becomes 8 and every other one stays: nn = n + 7 np,
    // so the parents' count needs no read of its own; the fill and whatever
    // reads the new leaves next are ordered on the stream
    *np = (nn - n) / 7;
    PBGPU_CUDA(c, leaves2.alloc(nn > 0 ? nn : 1));
    k_split_fill<<<grid_for(n, 256), 256, 0, st()>>>(leaves.get(), marks.get(), n, off.get(), leaves2.get());
    PBGPU_LAUNCHED(c);
    leaves.swap(leaves2);
    n = nn;
    return rekey();
  }

  // ripple balance from coarse seeds (cells that gained children) and fine
  // seeds (leaves that must not touch anything two levels finer)
  int balance(DBuf<int4>& coarse, int64_t nc, DBuf<int4>& fine, int64_t nf, bool fine_children) {
    int rc;
    for (int guard = 0; (nc > 0 || nf > 0) && guard < 64; ++guard) {
      PBGPU_CUDA(c, marks.alloc((n + 3) & ~int64_t(3)));
      PBGPU_CUDA(c, cudaMemsetAsync(marks.get(), 0, (n + 3) & ~int64_t(3), st()));
      // binary searches here: the table would be rebuilt after every pass of
      // the ripple, which measured slower than the searches it saves
      const Tree ht = tree();
      if (nc > 0) {
        k_balance_coarse<<<grid_for(nc * kBalLanes, 128), 128, 0, st()>>>(ht, coarse.get(), nc, marks.get());
        PBGPU_LAUNCHED(c);
      }
      if (nf > 0) {
        k_balance_fine<<<grid_for(nf * kBalLanes, 128), 128, 0, st()>>>(ht, fine.get(), nf, marks.get());
        PBGPU_LAUNCHED(c);
      }
      // the split's scan total is the only read of the pass: no split, no
      // change, the ripple has settled
      int64_t np = 0;
      if ((rc = split(coarse, &np)) != PBGPU_OK) return rc;
      if (np == 0) return PBGPU_OK;
      nc = np;
      nf = 0;
      if (fine_children) {
        PBGPU_CUDA(c, fine.alloc(8 * np > 0 ? 8 * np : 1));
        k_children<<<grid_for(np, 256), 256, 0, st()>>>(coarse.get(), np, fine.get());
        PBGPU_LAUNCHED(c);
        nf = 8 * np;
      }
    }
    if (nc > 0 || nf > 0) return c->fail(PBGPU_ERR_STATE, "build_mesh: 2:1 balance did not settle");
    return PBGPU_OK;
  }

  // uniform octree at `level`
  int uniform(int level) {
    if (level < 0 || level > 8) return c->fail(PBGPU_ERR_ARG, "build_mesh: uniform level must be 0..8");
    n = int64_t(1) << (3 * level);
    PBGPU_CUDA(c, leaves.alloc(n));
    k_uniform<<<grid_for(n, 256), 256, 0, st()>>>(level, n, leaves.get());
    PBGPU_LAUNCHED(c);
    return rekey();
  }

  // refine_in_box: up to `level` passes, each splitting the leaves below
  // `level` with a non-hanging corner in the box and restoring 2:1 balance; a
  // pass that marks nothing ends it (every later pass would mark nothing too)
  int box_refine(const double bl[3], const double br[3], int level) {
    int rc;
    for (int it = 0; it < level; ++it) {
      if ((rc = hanging()) != PBGPU_OK) return rc;
      PBGPU_CUDA(c, marks.alloc((n + 3) & ~int64_t(3)));
      k_box_marks<<<grid_for(n, 128), 128, 0, st()>>>(tree(), hm.get(), D, make_double3(bl[0], bl[1], bl[2]),
                                                      make_double3(br[0], br[1], br[2]), level, marks.get());
      PBGPU_LAUNCHED(c);
      DBuf<int4> parents, none;
      int64_t np = 0;
      if ((rc = split(parents, &np)) != PBGPU_OK) return rc;
      if (np == 0) break;
      if ((rc = balance(parents, np, none, 0, false)) != PBGPU_OK) return rc;
    }
    return PBGPU_OK;
  }

  int refine_step(int maxlevel) {
    int rc;
    if ((rc = surface_marks(0, 0, maxlevel)) != PBGPU_OK) return rc;
    DBuf<int4> parents, none;
    int64_t np = 0;
    if ((rc = split(parents, &np)) != PBGPU_OK) return rc;
    return balance(parents, np, none, 0, false);
  }

  int coarsen_step(int minlevel) {
    int rc;
    if ((rc = surface_marks(1, minlevel, 0)) != PBGPU_OK) return rc;
    PBGPU_CUDA(c, fam.alloc(n > 0 ? n : 1));
    k_family_start<<<grid_for(n, 256), 256, 0, st()>>>(tree(), marks.get(), fam.get());
    PBGPU_LAUNCHED(c);
    if ((rc = ensure_counts(n)) != PBGPU_OK) return rc;
    k_merge_count<<<grid_for(n, 256), 256, 0, st()>>>(fam.get(), n, cnt.get());
    PBGPU_LAUNCHED(c);
    int64_t nn = 0;
    if ((rc = scan(n, &nn)) != PBGPU_OK) return rc;
    // merged parents: the family's first child with the level decremented
    DBuf<int4> merged, none;
    DBuf<int64_t> nsel;
    PBGPU_CUDA(c, nsel.alloc(1));
    PBGPU_CUDA(c, merged.alloc(n > 0 ? n : 1));
    size_t bytes = 0;
    PBGPU_CUDA(c, cub::DeviceSelect::Flagged(nullptr, bytes, leaves.get(), fam.get(), merged.get(), nsel.get(),
                                             (int)n, st()));
    PBGPU_CUDA(c, ensure_tmp(c, bytes));
    PBGPU_CUDA(c, cub::DeviceSelect::Flagged(c->tmp.get(), bytes, leaves.get(), fam.get(), merged.get(), nsel.get(),
                                             (int)n, st()));
    c->launches += kCubSelectLaunches;
    // every family of 8 becomes its parent: nn = n - 7 nm
    const int64_t nm = (n - nn) / 7;
    PBGPU_CUDA(c, leaves2.alloc(nn > 0 ? nn : 1));
    k_merge_fill<<<grid_for(n, 256), 256, 0, st()>>>(leaves.get(), fam.get(), n, off.get(), leaves2.get());
    PBGPU_LAUNCHED(c);
    if (nm > 0) {
      k_parent_of<<<grid_for(nm, 256), 256, 0, st()>>>(merged.get(), nm);
      PBGPU_LAUNCHED(c);
    }
    leaves.swap(leaves2);
    n = nn;
    if ((rc = rekey()) != PBGPU_OK) return rc;
    return balance(none, 0, merged, nm, true);
  }
};

}  // namespace
}  // namespace pbgpu

using namespace pbgpu;

extern "C" int pbgpu_build_mesh(pbgpu_ctx* h, const pbgpu_mesh_build* in) {
  if (!h) return PBGPU_ERR_ARG;
  Context* c = &h->c;
  if (!in || in->n_oct < 0 || (in->n_oct > 0 && (!in->oct_xyz || !in->oct_level)) || in->n_spheres < 0 ||
      (in->n_spheres > 0 && !in->spheres))
    return c->fail(PBGPU_ERR_ARG, "build_mesh: bad initial octree or null arrays");
  if (in->n_oct == 0 && (in->init_level < 0 || in->init_level > 8 || in->box_level < 0 || in->box_level > kQMaxLevel))
    return c->fail(PBGPU_ERR_ARG, "build_mesh: init_level must be 0..8 and box_level 0..18");
  for (int a = 0; a < 3; ++a)
    if (!(in->hi[a] > in->lo[a])) return c->fail(PBGPU_ERR_ARG, "build_mesh: empty domain box");
  AcctScope acct(&c->dev_bytes);
  StreamScope sscope(c->stream, &c->blk_cache);
  if (cudaSetDevice(c->device) != cudaSuccess) return c->fail(PBGPU_ERR_CUDA, "build_mesh: cudaSetDevice");
  cudaGetLastError();
  c->have_mesh = c->have_markers = c->have_incidence = c->have_density = c->have_system = c->have_phi = false;
  for (int a = 0; a < 3; ++a) c->have_rays[a] = false;

  Builder B;
  B.c = c;
  for (int a = 0; a < 3; ++a) {
    B.D.lo[a] = in->lo[a];
    B.D.len[a] = in->hi[a] - in->lo[a];
  }
  // spheres and their bins
  std::vector<double4> sp;
  for (int64_t i = 0; i < in->n_spheres; ++i) {
    const double* v = in->spheres + 4 * i;
    if (!(v[3] > 0)) continue;
    sp.push_back(make_double4(v[0], v[1], v[2], v[3]));
  }
  BinsHost bins[3];
  double cell = 1.0;
  build_bins(sp, cell, bins);
  PBGPU_CUDA(c, B.sph.alloc(sp.size() > 0 ? sp.size() : 1));
  if (!sp.empty())
    PBGPU_CUDA(c, cudaMemcpyAsync(B.sph.get(), sp.data(), sp.size() * sizeof(double4), cudaMemcpyHostToDevice, c->stream));
  B.S.s = B.sph.get();
  B.S.n = (int64_t)sp.size();
  for (int a = 0; a < 3; ++a) {
    PBGPU_CUDA(c, B.bstart[a].alloc(bins[a].start.size()));
    PBGPU_CUDA(c, B.bitems[a].alloc(bins[a].items.size() > 0 ? bins[a].items.size() : 1));
    PBGPU_CUDA(c, cudaMemcpyAsync(B.bstart[a].get(), bins[a].start.data(), bins[a].start.size() * sizeof(int32_t),
                                  cudaMemcpyHostToDevice, c->stream));
    if (!bins[a].items.empty())
      PBGPU_CUDA(c, cudaMemcpyAsync(B.bitems[a].get(), bins[a].items.data(), bins[a].items.size() * sizeof(int32_t),
                                    cudaMemcpyHostToDevice, c->stream));
    B.S.bins[a] = SphereBins{bins[a].o0, bins[a].o1, cell, bins[a].n0, bins[a].n1, B.bstart[a].get(), B.bitems[a].get()};
  }
  // the initial octree: the caller's, or built here (init_tmesh*)
  int rc;
  if (in->n_oct > 0) {
    B.n = in->n_oct;
    std::vector<int4> q(B.n);
    for (int64_t i = 0; i < B.n; ++i)
      q[i] = make_int4(in->oct_xyz[3 * i], in->oct_xyz[3 * i + 1], in->oct_xyz[3 * i + 2], in->oct_level[i]);
    PBGPU_CUDA(c, B.leaves.alloc(B.n));
    PBGPU_CUDA(c, cudaMemcpyAsync(B.leaves.get(), q.data(), B.n * sizeof(int4), cudaMemcpyHostToDevice, c->stream));
    PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    if ((rc = B.rekey()) != PBGPU_OK) return rc;
  } else {
    if ((rc = B.uniform(in->init_level)) != PBGPU_OK) return rc;
    if (in->box_level > 0 && (rc = B.box_refine(in->box_lo, in->box_hi, in->box_level)) != PBGPU_OK) return rc;
  }
  // refine_surface: refinement / coarsening cycles
  if (in->refine) {
    const int cycles = std::max(in->maxlevel - in->unilevel, in->unilevel - in->minlevel);
    for (int kk = 0; kk < cycles; ++kk) {
      if ((rc = B.refine_step(in->maxlevel)) != PBGPU_OK) return rc;
      if ((rc = B.coarsen_step(in->minlevel)) != PBGPU_OK) return rc;
    }
  }
  // nodes
  if ((rc = B.hanging()) != PBGPU_OK) return rc;
  const int64_t no = B.n;
  if ((rc = B.ensure_counts(no)) != PBGPU_OK) return rc;
  k_indep_count<<<grid_for(no, 256), 256, 0, c->stream>>>(B.tree(), B.hm.get(), B.cnt.get());
  PBGPU_LAUNCHED(c);
  int64_t ni = 0;
  if ((rc = B.scan(no, &ni)) != PBGPU_OK) return rc;
  DBuf<uint64_t> codes, codes2, hcodes;
  PBGPU_CUDA(c, codes.alloc(ni > 0 ? ni : 1));
  PBGPU_CUDA(c, codes2.alloc(ni > 0 ? ni : 1));
  k_indep_fill<<<grid_for(no, 256), 256, 0, c->stream>>>(B.tree(), B.hm.get(), B.off.get(), codes.get());
  PBGPU_LAUNCHED(c);
  {
    size_t bytes = 0;
    PBGPU_CUDA(c, cub::DeviceRadixSort::SortKeys(nullptr, bytes, codes.get(), codes2.get(), (int)ni, 0, kMortonBits,
                                                 c->stream));
    PBGPU_CUDA(c, ensure_tmp(c, bytes));
    PBGPU_CUDA(c, cub::DeviceRadixSort::SortKeys(c->tmp.get(), bytes, codes.get(), codes2.get(), (int)ni, 0,
                                                 kMortonBits, c->stream));
    c->launches += cub_radix_launches(ni, kMortonBits);
    codes.swap(codes2);
  }
  if ((rc = B.ensure_counts(no)) != PBGPU_OK) return rc;
  k_hang_count<<<grid_for(no, 256), 256, 0, c->stream>>>(B.tree(), B.hm.get(), B.cnt.get());
  PBGPU_LAUNCHED(c);
  int64_t nhc = 0;
  if ((rc = B.scan(no, &nhc)) != PBGPU_OK) return rc;
  PBGPU_CUDA(c, hcodes.alloc(nhc > 0 ? nhc : 1));
  k_hang_fill<<<grid_for(no, 256), 256, 0, c->stream>>>(B.tree(), B.hm.get(), B.off.get(), hcodes.get());
  PBGPU_LAUNCHED(c);
  int64_t nh = 0;
  if ((rc = B.sort_unique(hcodes, nhc, &nh, kMortonBits)) != PBGPU_OK) return rc;
  if (ni + nh >= (int64_t(1) << 31)) return c->fail(PBGPU_ERR_CAPACITY, "build_mesh: too many nodes");
  PBGPU_CUDA(c, B.bad.alloc(1));
  PBGPU_CUDA(c, cudaMemsetAsync(B.bad.get(), 0, sizeof(int), c->stream));
  // the context's mesh
  PBGPU_CUDA(c, c->node_xyz.alloc(ni > 0 ? ni : 1));
  k_node_xyz<<<grid_for(ni, 256), 256, 0, c->stream>>>(codes.get(), ni, c->node_xyz.get());
  PBGPU_LAUNCHED(c);
  PBGPU_CUDA(c, c->oct_nodes.alloc(8 * no));
  PBGPU_CUDA(c, c->hang_par.alloc(nh > 0 ? nh : 1));
  PBGPU_CUDA(c, c->hang_np.alloc(nh > 0 ? nh : 1));
  k_corner_nodes<<<grid_for(no, 128), 128, 0, c->stream>>>(B.tree(), B.hm.get(), codes.get(), ni, hcodes.get(), nh,
                                                            c->oct_nodes.get(), c->hang_par.get(), c->hang_np.get(),
                                                            B.bad.get());
  PBGPU_LAUNCHED(c);
  int bad = 0;
  PBGPU_CUDA(c, readback(c, &bad, B.bad.get(), sizeof(int)));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  if (bad) return c->fail(PBGPU_ERR_STATE, "build_mesh: a corner or hanging parent is not an independent node");
  PBGPU_CUDA(c, c->oct.alloc(no));
  PBGPU_CUDA(c, cudaMemcpyAsync(c->oct.get(), B.leaves.get(), no * sizeof(int4), cudaMemcpyDeviceToDevice, c->stream));
  PBGPU_CUDA(c, c->oct_key.alloc(no));
  PBGPU_CUDA(c, cudaMemcpyAsync(c->oct_key.get(), B.keys.get(), no * sizeof(uint64_t), cudaMemcpyDeviceToDevice,
                                c->stream));
  c->n_oct = no;
  c->n = ni;
  c->nh = nh;
  for (int a = 0; a < 3; ++a) {
    c->lo[a] = in->lo[a];
    c->len[a] = in->hi[a] - in->lo[a];
  }
  c->tol = in->locate_tol;
  // ray tables of the three axes over every node point
  for (int axis = 0; axis < 3; ++axis) {
    DBuf<uint64_t> rk;
    PBGPU_CUDA(c, rk.alloc(ni + nh > 0 ? ni + nh : 1));
    k_node_ray_keys<<<grid_for(ni + nh, 256), 256, 0, c->stream>>>(c->node_xyz.get(), ni, hcodes.get(), nh, axis,
                                                                    rk.get());
    PBGPU_LAUNCHED(c);
    int64_t nk = 0;
    if ((rc = B.sort_unique(rk, ni + nh, &nk, kRayKeyBits)) != PBGPU_OK) return rc;
    Rays& R = c->rays[axis];
    DBuf<int64_t> coff;
    if ((rc = B.cast(rk.get(), nk, axis, coff, R.inters, &R.normals)) != PBGPU_OK) return rc;
    // keep the rays that have crossings
    DBuf<uint8_t> flag;
    DBuf<int64_t> sel, nsel;
    PBGPU_CUDA(c, flag.alloc(nk > 0 ? nk : 1));
    PBGPU_CUDA(c, sel.alloc(nk > 0 ? nk : 1));
    PBGPU_CUDA(c, nsel.alloc(1));
    int64_t ns = 0;
    if (nk > 0) {
      k_has_cross<<<grid_for(nk, 256), 256, 0, c->stream>>>(coff.get(), nk, flag.get());
      PBGPU_LAUNCHED(c);
      cub::CountingInputIterator<int64_t> idx(0);
      size_t bytes = 0;
      PBGPU_CUDA(c, cub::DeviceSelect::Flagged(nullptr, bytes, idx, flag.get(), sel.get(), nsel.get(), (int)nk,
                                               c->stream));
      PBGPU_CUDA(c, ensure_tmp(c, bytes));
      PBGPU_CUDA(c, cub::DeviceSelect::Flagged(c->tmp.get(), bytes, idx, flag.get(), sel.get(), nsel.get(), (int)nk,
                                               c->stream));
      c->launches += kCubSelectLaunches;
      PBGPU_CUDA(c, readback(c, &ns, nsel.get(), sizeof(int64_t)));
      PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    PBGPU_CUDA(c, R.keys.alloc(ns > 0 ? ns : 1));
    PBGPU_CUDA(c, R.ptr.alloc(ns + 1));
    if (ns > 0) {
      k_gather_keys<<<grid_for(ns + 1, 256), 256, 0, c->stream>>>(sel.get(), ns, rk.get(), coff.get(), nk, R.keys.get(),
                                                              R.ptr.get());
      PBGPU_LAUNCHED(c);
    } else {
      PBGPU_CUDA(c, cudaMemsetAsync(R.ptr.get(), 0, sizeof(int64_t), c->stream));
    }
    int64_t nc = 0;
    if (nk > 0) PBGPU_CUDA(c, readback(c, &nc, coff.get() + nk, sizeof(int64_t)));
    PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    R.n = ns;
    R.nc = nc;
    if ((rc = build_ray_hash_from(c, axis, R.keys.get())) != PBGPU_OK) return rc;
    c->have_rays[axis] = true;
  }
  c->have_mesh = true;
  return PBGPU_OK;
}

extern "C" int pbgpu_get_mesh_counts(pbgpu_ctx* h, int64_t* n_oct, int64_t* n_nodes, int64_t* n_hang,
                                     int64_t* n_rays) {
  if (!h) return PBGPU_ERR_ARG;
  const Context& c = h->c;
  if (!c.have_mesh) return PBGPU_ERR_STATE;
  if (n_oct) *n_oct = c.n_oct;
  if (n_nodes) *n_nodes = c.n;
  if (n_hang) *n_hang = c.nh;
  if (n_rays)
    for (int a = 0; a < 3; ++a) n_rays[a] = c.rays[a].n;
  return PBGPU_OK;
}

// The context's mesh copied back to host arrays (any may be NULL), sized by
// pbgpu_get_mesh_counts; box receives lo[3] and the extent hi - lo [3] the
// node coordinates are computed from.
extern "C" int pbgpu_get_mesh(pbgpu_ctx* h, int32_t* oct_xyz, int8_t* oct_level, int32_t* oct_nodes,
                              int32_t* node_xyz, int8_t* hang_np, int32_t* hang_par, double* box) {
  if (!h) return PBGPU_ERR_ARG;
  Context* c = &h->c;
  if (!c->have_mesh) return c->fail(PBGPU_ERR_STATE, "get_mesh: no mesh");
  if (cudaSetDevice(c->device) != cudaSuccess) return c->fail(PBGPU_ERR_CUDA, "get_mesh: cudaSetDevice");
  std::vector<int4> v;
  if (oct_xyz || oct_level) {
    v.resize(c->n_oct);
    PBGPU_CUDA(c, cudaMemcpyAsync(v.data(), c->oct.get(), c->n_oct * sizeof(int4), cudaMemcpyDeviceToHost, c->stream));
    PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int64_t i = 0; i < c->n_oct; ++i) {
      if (oct_xyz) {
        oct_xyz[3 * i] = v[i].x;
        oct_xyz[3 * i + 1] = v[i].y;
        oct_xyz[3 * i + 2] = v[i].z;
      }
      if (oct_level) oct_level[i] = (int8_t)v[i].w;
    }
  }
  if (oct_nodes)
    PBGPU_CUDA(c, cudaMemcpyAsync(oct_nodes, c->oct_nodes.get(), 8 * c->n_oct * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                  c->stream));
  std::vector<int8_t> np;
  if ((hang_np || hang_par) && c->nh) {
    np.resize(c->nh);
    PBGPU_CUDA(c, cudaMemcpyAsync(np.data(), c->hang_np.get(), c->nh, cudaMemcpyDeviceToHost, c->stream));
  }
  if (hang_par && c->nh)
    PBGPU_CUDA(c, cudaMemcpyAsync(hang_par, c->hang_par.get(), c->nh * sizeof(int4), cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  if (hang_np && c->nh) std::memcpy(hang_np, np.data(), c->nh);
  if (hang_par)  // the device pads unused parent slots; the host layout marks them -1
    for (int64_t i = 0; i < c->nh; ++i)
      for (int j = np[i]; j < 4; ++j) hang_par[4 * i + j] = -1;
  if (node_xyz) {
    v.resize(c->n);
    PBGPU_CUDA(c, cudaMemcpyAsync(v.data(), c->node_xyz.get(), c->n * sizeof(int4), cudaMemcpyDeviceToHost, c->stream));
    PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int64_t i = 0; i < c->n; ++i) {
      node_xyz[3 * i] = v[i].x;
      node_xyz[3 * i + 1] = v[i].y;
      node_xyz[3 * i + 2] = v[i].z;
    }
  }
  if (box)
    for (int a = 0; a < 3; ++a) {
      box[a] = c->lo[a];
      box[3 + a] = c->len[a];
    }
  return PBGPU_OK;
}
