// create_markers and cube_fraction_intersection on the device
// (src/pb_class.cpp:1793-1941, 2422-2532, is_in_ns_surf :769-805,
// is_in_ns_surf_stern :1752-1790).
//
// Surface rays live in one open-addressing hash table per axis (key = the two
// transverse integer coordinates), so a node finds its ray in O(1) probes
// instead of the reference's std::map lookups.  Node classification is one
// thread per node, octant markers one thread per octant, and the 12 edge
// fractions of a border octant one thread per (octant, edge).
#include <cub/cub.cuh>

#include "pbgpu_internal.cuh"

namespace pbgpu {

__global__ void k_hash_insert(const uint64_t* __restrict__ keys, int64_t n, uint64_t* hk, int32_t* hv, int64_t cap,
                              int cap_log, int* overflow) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t key = keys[i];
  uint64_t s = hash_slot(key, cap_log);
  for (int64_t probe = 0; probe < cap; ++probe) {
    const unsigned long long prev =
        atomicCAS(reinterpret_cast<unsigned long long*>(hk + s), (unsigned long long)kEmptyKey, (unsigned long long)key);
    if (prev == kEmptyKey || prev == key) {
      hv[s] = (int32_t)i;
      return;
    }
    s = (s + 1) & (uint64_t)(cap - 1);
  }
  atomicExch(overflow, 1);
}

// Hash build needs the key array on the device; the caller passes it.
int build_ray_hash_from(Context* c, int axis, const uint64_t* d_keys) {
  Rays& R = c->rays[axis];
  if (R.n == 0) {
    R.cap = 0;
    R.cap_log = 0;
    return PBGPU_OK;
  }
  int lg = 4;
  while ((int64_t(1) << lg) < 2 * R.n) ++lg;
  R.cap_log = lg;
  R.cap = int64_t(1) << lg;
  PBGPU_CUDA(c, R.hkeys.alloc(R.cap));
  PBGPU_CUDA(c, R.hval.alloc(R.cap));
  PBGPU_CUDA(c, cudaMemsetAsync(R.hkeys.get(), 0xff, R.cap * sizeof(uint64_t), c->stream));
  Scratch<int> ovf(c, kScMkOvf);
  PBGPU_CUDA(c, ovf.alloc(1));
  PBGPU_CUDA(c, cudaMemsetAsync(ovf.get(), 0, sizeof(int), c->stream));
  k_hash_insert<<<grid_for(R.n, 256), 256, 0, c->stream>>>(d_keys, R.n, R.hkeys.get(), R.hval.get(), R.cap, R.cap_log,
                                                           ovf.get());
  PBGPU_LAUNCHED(c);
  int h_ovf = 0;
  PBGPU_CUDA(c, readback(c, &h_ovf, ovf.get(), sizeof(int)));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  if (h_ovf) return c->fail(PBGPU_ERR_CAPACITY, "ray hash table overflow");
  return PBGPU_OK;
}

// is_in_ns_surf along z: odd number of crossings at or below z -> inside.
// Stern variant (is_in_ns_surf_stern): thresholds shifted by -stern*sign with a
// strict comparison.
__global__ void k_classify_nodes(const int4* __restrict__ node_xyz, int64_t n, RayView rz, double lo2, double len2,
                                 double eps_in, double eps_out, double react_out, int stern, double stern_w,
                                 uint8_t* __restrict__ inside, double* __restrict__ eps, double* __restrict__ react) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int4 p = node_xyz[i];
  const double z = coord(lo2, len2, p.z);
  const int32_t r = ray_find(rz.hk, rz.hv, rz.cap, rz.cap_log, ray_key(p.x, p.y));
  int in = 0, in_stern = 0;
  if (r >= 0) {
    const int64_t b = rz.ptr[r], e = rz.ptr[r + 1];
    int64_t k = b;
    while (k < e && z >= rz.inters[k]) ++k;
    in = (int)((k - b) & 1);
    if (stern) {
      int64_t j = b;
      double sign = 1.0;
      if (!(z < rz.inters[b] - stern_w)) {
        while (j < e && z > (rz.inters[j] - stern_w * sign)) {
          ++j;
          sign = -sign;
        }
      }
      in_stern = (int)((j - b) & 1);
    }
  }
  inside[i] = (uint8_t)(in | (in_stern << 1));
  eps[i] = in ? eps_in : eps_out;
  react[i] = in ? 0.0 : react_out;
}

// Octant marker (src/pb_class.cpp:1910-1916): 2 out (no inside corner),
// 1 border (some but not all non-hanging corners inside), 0 in.
__global__ void k_octant_markers(const int32_t* __restrict__ oct_nodes, int64_t n_oct, int64_t n,
                                 const uint8_t* __restrict__ inside, int stern, double react_out,
                                 uint8_t* __restrict__ marker, uint8_t* __restrict__ is_border,
                                 double* __restrict__ react_cell) {
  const int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (o >= n_oct) return;
  const int4 a = reinterpret_cast<const int4*>(oct_nodes)[2 * o];
  const int4 b = reinterpret_cast<const int4*>(oct_nodes)[2 * o + 1];
  const int32_t nd[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
  int num_int = 0, num_hang = 0, num_stern = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    if (nd[c] >= n) {
      ++num_hang;
      continue;
    }
    const uint8_t f = inside[nd[c]];
    num_int += f & 1;
    num_stern += (f & 1) + ((f >> 1) & 1);
  }
  uint8_t m = 0;
  if (num_int == 0)
    m = 2;
  else if (num_int < 8 - num_hang)
    m = 1;
  marker[o] = m;
  is_border[o] = (m == 1);
  if (stern) react_cell[o] = num_stern != 0 ? 0.0 : react_out;
}

__global__ void k_border_pos(const int32_t* __restrict__ border, int64_t nb, int32_t* __restrict__ border_pos) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b < nb) border_pos[border[b]] = (int32_t)b;
}

// cube_fraction_intersection: the position, relative to the edge's first
// corner, of the last crossing of the ray through that corner that lies on
// the edge; 0.5 when none.
__global__ void k_fractions(const int4* __restrict__ oct, const int32_t* __restrict__ border, int64_t nb, RayView rx,
                            RayView ry, RayView rzv, double3 lo, double3 len, double* __restrict__ frac) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= 12 * nb) return;
  const int64_t bi = t / 12;
  const int e = (int)(t % 12);
  const int4 q = oct[border[bi]];
  const int32_t s = 1 << (kRootLog - q.w);
  const int axis = d_edge_axis[e], i1 = d_edge_nodes[2 * e], i2 = d_edge_nodes[2 * e + 1];
  const int32_t p1[3] = {q.x + (i1 & 1) * s, q.y + ((i1 >> 1) & 1) * s, q.z + ((i1 >> 2) & 1) * s};
  const int32_t p2a = (axis == 0 ? q.x + (i2 & 1) * s : axis == 1 ? q.y + ((i2 >> 1) & 1) * s : q.z + ((i2 >> 2) & 1) * s);
  const double loa = axis == 0 ? lo.x : axis == 1 ? lo.y : lo.z;
  const double lena = axis == 0 ? len.x : axis == 1 ? len.y : len.z;
  const double x1 = coord(loa, lena, p1[axis]), x2 = coord(loa, lena, p2a);
  const RayView& R = axis == 0 ? rx : axis == 1 ? ry : rzv;
  const int t0 = axis == 0 ? 1 : 0, t1 = axis == 2 ? 1 : 2;
  double f = 0.5;
  const int32_t r = ray_find(R.hk, R.hv, R.cap, R.cap_log, ray_key(p1[t0], p1[t1]));
  if (r >= 0) {
    for (int64_t k = R.ptr[r]; k < R.ptr[r + 1]; ++k) {
      const double I = R.inters[k];
      if (I >= x1 && I <= x2) f = (I - x1) / (x2 - x1);
    }
  }
  frac[t] = f;
}

int run_markers(Context* c) {
  const int64_t n = c->n, no = c->n_oct;
  PBGPU_CUDA(c, c->inside.alloc(n));
  PBGPU_CUDA(c, c->eps.alloc(n));
  PBGPU_CUDA(c, c->react.alloc(n));
  PBGPU_CUDA(c, c->marker.alloc(no));
  PBGPU_CUDA(c, c->border_pos.alloc(no));
  const int stern = c->model.stern_layer_surf == 1;
  if (stern) PBGPU_CUDA(c, c->react_cell.alloc(no));
  const double react_out = c->eps_out * c->k2;
  k_classify_nodes<<<grid_for(n, 256), 256, 0, c->stream>>>(
      c->node_xyz.get(), n, ray_view(c->rays[2]), c->lo[2], c->len[2], c->eps_in, c->eps_out, react_out, stern,
      c->model.stern_layer, c->inside.get(), c->eps.get(), c->react.get());
  PBGPU_LAUNCHED(c);
  Scratch<uint8_t> flags(c, kScMkFlags);
  PBGPU_CUDA(c, flags.alloc(no));
  k_octant_markers<<<grid_for(no, 256), 256, 0, c->stream>>>(c->oct_nodes.get(), no, n, c->inside.get(), stern,
                                                              react_out, c->marker.get(), flags.get(),
                                                              stern ? c->react_cell.get() : nullptr);
  PBGPU_LAUNCHED(c);
  // border list in ascending octant order
  Scratch<int32_t> sel(c, kScMkSel);
  Scratch<int64_t> nsel(c, kScMkNsel);
  PBGPU_CUDA(c, sel.alloc(no));
  PBGPU_CUDA(c, nsel.alloc(1));
  cub::CountingInputIterator<int32_t> idx(0);
  size_t bytes = 0;
  PBGPU_CUDA(c, cub::DeviceSelect::Flagged(nullptr, bytes, idx, flags.get(), sel.get(), nsel.get(), no, c->stream));
  PBGPU_CUDA(c, ensure_tmp(c, bytes));
  PBGPU_CUDA(c, cub::DeviceSelect::Flagged(c->tmp.get(), bytes, idx, flags.get(), sel.get(), nsel.get(), no, c->stream));
  c->launches += kCubSelectLaunches;
  int64_t nb = 0;
  PBGPU_CUDA(c, readback(c, &nb, nsel.get(), sizeof(int64_t)));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  c->nb = nb;
  PBGPU_CUDA(c, c->border.alloc(nb > 0 ? nb : 1));
  if (nb) PBGPU_CUDA(c, cudaMemcpyAsync(c->border.get(), sel.get(), nb * sizeof(int32_t), cudaMemcpyDeviceToDevice, c->stream));
  PBGPU_CUDA(c, cudaMemsetAsync(c->border_pos.get(), 0xff, no * sizeof(int32_t), c->stream));
  if (nb) {
    k_border_pos<<<grid_for(nb, 256), 256, 0, c->stream>>>(c->border.get(), nb, c->border_pos.get());
    PBGPU_LAUNCHED(c);
  }
  PBGPU_CUDA(c, c->frac.alloc(nb > 0 ? 12 * nb : 12));
  if (nb) {
    const double3 lo = make_double3(c->lo[0], c->lo[1], c->lo[2]);
    const double3 len = make_double3(c->len[0], c->len[1], c->len[2]);
    k_fractions<<<grid_for(12 * nb, 256), 256, 0, c->stream>>>(c->oct.get(), c->border.get(), nb, ray_view(c->rays[0]),
                                                                ray_view(c->rays[1]), ray_view(c->rays[2]), lo, len,
                                                                c->frac.get());
    PBGPU_LAUNCHED(c);
  }
  // flags/sel are freed at scope exit: make sure the stream is done with them
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  c->have_markers = true;
  return PBGPU_OK;
}

}  // namespace pbgpu
