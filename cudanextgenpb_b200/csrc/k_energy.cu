// Post-processing on the device: potential at the atoms
// (write_potential_on_atoms_fast, src/pb_class.cpp:2333-2417) and the
// electrostatic energy (energy / energy_fast, :2791-3338).
//
// The reference walks every border octant and, for each epsilon-jump edge
// (flux term) and each marching-cubes triangle vertex (ionic term), sums over
// all charged atoms.  Every such surface point lies on a ray crossing, and a
// crossing is shared by the octants around its edge, so the same point enters
// the pair sum up to ~10 times with different coefficients.  Here:
//  (1) one thread per border octant evaluates the reference's per-element
//      coefficients (flux F, and coef * N with coef = phi0 * area / (12 pi) for
//      a triangle vertex) and adds them into an accumulator of the crossing
//      they sit on (elements whose edge has no crossing keep their own point).
//      The accumulators are 128-bit fixed point (2^-64 resolution) updated by
//      integer atomics: integer addition is associative, so each crossing's
//      sum is exact and the same whatever order the octants add in, and the
//      energies are bit-for-bit reproducible; the elements without a crossing
//      are put in (octant, element) order before they become points;
//  (2) the used crossings are compacted into a point list (V, F, D);
//  (3) one FP64 pair kernel over points x charged atoms, atoms staged in shared
//      memory tiles, evaluates sum_a q_a / r (flux) and sum_a q_a (V - x_a).D / r^3
//      (ionic) together, with 1/r from a Newton-Raphson reciprocal square root.
// The point of a crossing is the crossing itself (transverse coordinates of the
// ray, position along it); the reference recomputes it per edge as
// x1 + frac * h, which agrees to the last bit or two.
#include <cub/cub.cuh>

#include "mc_tables.h"
#include "pbgpu_internal.cuh"

namespace pbgpu {

__device__ __constant__ int8_t d_tri[256][16];

struct EnergyView {
  const int4* oct;
  const int32_t* oct_nodes;
  const int4* hang_par;
  const int8_t* hang_np;
  const int32_t* border;
  const double* eps;
  const double* phi;
  RayView rays[3];
  int64_t slot_base[3];   // first accumulator slot of each axis' crossings
  unsigned long long* acc;  // per crossing: F, Dx, Dy, Dz, each 128-bit fixed point (low, high words)
  uint8_t* used;
  int32_t* slot_ray;      // ray of each used crossing
  double4* extra_p;       // elements on edges without a crossing
  double4* extra_d;
  unsigned long long* extra_key;  // (border octant << 8) | element number in the octant
  unsigned long long* n_extra;
  int64_t extra_cap;
  int64_t n, nb;
  double lo[3], len[3];
  double eps_out;
  int ionic, fast;
  double h0[3];  // energy_fast: spacing of the first border octant
};

__device__ __forceinline__ double cval(const double* __restrict__ v, int32_t nd, const EnergyView& E) {
  if (nd < E.n) return v[nd];
  const int64_t h = nd - E.n;
  const int4 p = E.hang_par[h];
  const int np = E.hang_np[h];
  double t = 0.0;
  t += v[p.x] / np;
  t += v[p.y] / np;
  if (np == 4) {
    t += v[p.z] / np;
    t += v[p.w] / np;
  }
  return t;
}

struct CellCtx {
  int4 q;
  int32_t s;
  double h[3], area_h[3];
  double te[8], tp[8];
  double N[3];
};

__device__ __forceinline__ void cell_load(const EnergyView& E, int64_t b, CellCtx& C) {
  const int64_t o = E.border[b];
  C.q = E.oct[o];
  C.s = 1 << (kRootLog - C.q.w);
  const int32_t qc[3] = {C.q.x, C.q.y, C.q.z};
  for (int d = 0; d < 3; ++d)
    C.h[d] = E.fast ? E.h0[d] : coord(E.lo[d], E.len[d], qc[d] + C.s) - coord(E.lo[d], E.len[d], qc[d]);
  C.area_h[0] = C.h[1] * C.h[2] / C.h[0] * 0.25;
  C.area_h[1] = C.h[0] * C.h[2] / C.h[1] * 0.25;
  C.area_h[2] = C.h[0] * C.h[1] / C.h[2] * 0.25;
  for (int c = 0; c < 8; ++c) {
    const int32_t nd = E.oct_nodes[8 * o + c];
    C.te[c] = cval(E.eps, nd, E);
    C.tp[c] = cval(E.phi, nd, E);
  }
  C.N[0] = C.N[1] = C.N[2] = 0.0;
}

__device__ __forceinline__ int32_t corner_i(const CellCtx& C, int c, int a) {
  const int32_t base = a == 0 ? C.q.x : a == 1 ? C.q.y : C.q.z;
  return base + ((c >> a) & 1) * C.s;
}

// normal_intersection (src/pb_class.cpp:2535-2568): updates C.N when a crossing
// lies on the edge and returns the fraction (0.5 when none); *slot is the
// global accumulator slot of that crossing or -1.
__device__ __forceinline__ double normal_intersection(const EnergyView& E, CellCtx& C, int e, int64_t* slot,
                                                      int32_t* ray) {
  const int axis = d_edge_axis[e], i1 = d_edge_nodes[2 * e], i2 = d_edge_nodes[2 * e + 1];
  const double x1 = coord(E.lo[axis], E.len[axis], corner_i(C, i1, axis));
  const double x2 = coord(E.lo[axis], E.len[axis], corner_i(C, i2, axis));
  const int t0 = axis == 0 ? 1 : 0, t1 = axis == 2 ? 1 : 2;
  const RayView& R = E.rays[axis];
  double f = 0.5;
  *slot = -1;
  const int32_t r = ray_find(R.hk, R.hv, R.cap, R.cap_log, ray_key(corner_i(C, i1, t0), corner_i(C, i1, t1)));
  *ray = r;
  if (r >= 0)
    for (int64_t k = R.ptr[r]; k < R.ptr[r + 1]; ++k) {
      const double I = R.inters[k];
      if (I >= x1 && I <= x2) {
        C.N[0] = R.normals[3 * k];
        C.N[1] = R.normals[3 * k + 1];
        C.N[2] = R.normals[3 * k + 2];
        f = (I - x1) / (x2 - x1);
        *slot = E.slot_base[axis] + k;
      }
    }
  return f;
}

__device__ __forceinline__ void edge_point(const EnergyView& E, const CellCtx& C, int e, double f, double V[3]) {
  const int axis = d_edge_axis[e], i1 = d_edge_nodes[2 * e];
  for (int a = 0; a < 3; ++a) V[a] = coord(E.lo[a], E.len[a], corner_i(C, i1, a));
  V[axis] += f * C.h[axis];
}

__device__ __forceinline__ int cube_index(const CellCtx& C, double eps_out) {
  const int mc[8] = {0, 1, 3, 2, 4, 5, 7, 6};
  int k = 0;
  for (int v = 0; v < 8; ++v)
    if (C.te[mc[v]] < (eps_out - 1e-10)) k |= 1 << v;
  return k;
}

// a[0] (low word) and a[1] (high word, signed) += v as 128-bit fixed point
// with 64 fraction bits: v = hi + lo 2^-64 with 0 <= lo < 2^64 is exact for
// |v| < 2^63 down to 2^-64 (smaller parts drop, 5e-20 absolute); the carry of
// the low word goes into the high one, so the total is exact in any order.
__device__ __forceinline__ void add_fixed128(unsigned long long* a, double v) {
  const double fl = floor(v);
  const unsigned long long lo = (unsigned long long)((v - fl) * 0x1p64);
  const unsigned long long hi = (unsigned long long)(long long)fl;
  const unsigned long long old = atomicAdd(a, lo);
  atomicAdd(a + 1, hi + (old + lo < old ? 1ull : 0ull));
}

__device__ __forceinline__ double fixed128_value(const unsigned long long* a) {
  return (double)(long long)a[1] + (double)a[0] * 0x1p-64;
}

__device__ __forceinline__ void add_point(const EnergyView& E, int64_t b, int& local, int64_t slot, int32_t ray,
                                          const double V[3], double F, double Dx, double Dy, double Dz) {
  const int elem = local++;
  if (slot >= 0) {
    unsigned long long* a = E.acc + 8 * slot;
    if (F != 0.0) add_fixed128(a, F);
    if (Dx != 0.0) add_fixed128(a + 2, Dx);
    if (Dy != 0.0) add_fixed128(a + 4, Dy);
    if (Dz != 0.0) add_fixed128(a + 6, Dz);
    E.used[slot] = 1;
    E.slot_ray[slot] = ray;
    return;
  }
  const unsigned long long i = atomicAdd(E.n_extra, 1ull);
  if ((int64_t)i < E.extra_cap) {
    E.extra_p[i] = make_double4(V[0], V[1], V[2], F);
    E.extra_d[i] = make_double4(Dx, Dy, Dz, 0.0);
    E.extra_key[i] = ((unsigned long long)b << 8) | (unsigned long long)elem;
  }
}

// (1) per border octant: the reference's element coefficients, accumulated on
// the crossings they sit on.
__global__ void k_energy_accumulate(EnergyView E) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b >= E.nb) return;
  CellCtx C;
  cell_load(E, b, C);
  int local = 0;  // element number in this octant (at most 12 + 15)
  for (int e = 0; e < 12; ++e) {
    const int i1 = d_edge_nodes[2 * e], i2 = d_edge_nodes[2 * e + 1];
    double dir;
    if (C.te[i1] < C.te[i2])
      dir = 1;
    else if (C.te[i1] > C.te[i2])
      dir = -1;
    else
      continue;
    int64_t slot;
    int32_t ray;
    const double f = normal_intersection(E, C, e, &slot, &ray);
    double V[3];
    edge_point(E, C, e, f, V);
    const double F = -(C.tp[i2] - C.tp[i1]) * wha(C.te[i1], C.te[i2], f) * dir * C.area_h[d_edge_axis[e]];
    add_point(E, b, local, slot, ray, V, F, 0.0, 0.0, 0.0);
  }
  if (!E.ionic) return;
  const int k = cube_index(C, E.eps_out);
  if (k == 0 || k == 255) return;
  const double inv_4pi = 1.0 / (4.0 * kPi);
  for (int t = 0; t < 5 && d_tri[k][3 * t] >= 0; ++t) {
    double VT[3][3], NT[3][3], ps[3];
    int64_t sl[3];
    int32_t ry[3];
    for (int j = 0; j < 3; ++j) {
      const int e = d_tri[k][3 * t + j];
      const int i1 = d_edge_nodes[2 * e], i2 = d_edge_nodes[2 * e + 1];
      const double f = normal_intersection(E, C, e, &sl[j], &ry[j]);
      edge_point(E, C, e, f, VT[j]);
      NT[j][0] = C.N[0];
      NT[j][1] = C.N[1];
      NT[j][2] = C.N[2];
      ps[j] = C.tp[i1] + f * C.te[i2] * (C.tp[i2] - C.tp[i1]) / (C.te[i2] * f + C.te[i1] * (1 - f));
    }
    double ab[3], ac[3];
    for (int a = 0; a < 3; ++a) {
      ab[a] = VT[0][a] - VT[1][a];
      ac[a] = VT[0][a] - VT[2][a];
    }
    const double area =
        0.5 * norm3d(ab[1] * ac[2] - ab[2] * ac[1], ab[0] * ac[2] - ab[2] * ac[0], ab[1] * ac[0] - ab[0] * ac[1]);
    for (int j = 0; j < 3; ++j) {
      const double coef = ps[j] * inv_4pi * area / 3.0;
      add_point(E, b, local, sl[j], ry[j], VT[j], 0.0, coef * NT[j][0], coef * NT[j][1], coef * NT[j][2]);
    }
  }
}

// (2) used crossing -> point (transverse coordinates of its ray, position along it)
__global__ void k_energy_points(const int32_t* __restrict__ used_slots, int64_t m, EnergyView E,
                                double4* __restrict__ P, double4* __restrict__ D) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int64_t slot = used_slots[i];
  const int axis = slot >= E.slot_base[2] ? 2 : (slot >= E.slot_base[1] ? 1 : 0);
  const int64_t k = slot - E.slot_base[axis];
  const RayView& R = E.rays[axis];
  const int32_t r = E.slot_ray[slot];
  const uint64_t key = R.keys[r];
  const int t0 = axis == 0 ? 1 : 0, t1 = axis == 2 ? 1 : 2;
  double V[3];
  V[axis] = R.inters[k];
  V[t0] = coord(E.lo[t0], E.len[t0], (int32_t)(key >> 20));
  V[t1] = coord(E.lo[t1], E.len[t1], (int32_t)(key & 0xfffff));
  const unsigned long long* a = E.acc + 8 * slot;
  P[i] = make_double4(V[0], V[1], V[2], fixed128_value(a));
  D[i] = make_double4(fixed128_value(a + 2), fixed128_value(a + 4), fixed128_value(a + 6), 0.0);
}

__global__ void k_iota_u64(unsigned long long* __restrict__ a, int64_t m) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < m) a[i] = (unsigned long long)i;
}

// the elements without a crossing in (octant, element) order
__global__ void k_gather_extras(const unsigned long long* __restrict__ order, int64_t m, const double4* __restrict__ xp,
                                const double4* __restrict__ xd, double4* __restrict__ P, double4* __restrict__ D) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int64_t j = (int64_t)order[i];
  P[i] = xp[j];
  D[i] = xd[j];
}

constexpr int kTile = 256;

// (3) sum over points of F sum_a q_a / r  and  sum_a q_a (V - x_a).D / r^3
template <bool IONIC>
__global__ void __launch_bounds__(kTile) k_energy_pairs(const double4* __restrict__ P, const double4* __restrict__ D,
                                                        int64_t np, const double4* __restrict__ atoms, int64_t m,
                                                        double* __restrict__ partials) {
  __shared__ double4 tile[kTile];
  double acc1 = 0.0, acc2 = 0.0, accF = 0.0;
  for (int64_t base = blockIdx.x * (int64_t)kTile; base < np; base += (int64_t)gridDim.x * kTile) {
    const int64_t e = base + threadIdx.x;
    const bool live = e < np;
    const double4 V = live ? P[e] : make_double4(0, 0, 0, 0);
    const double4 Dv = (IONIC && live) ? D[e] : make_double4(0, 0, 0, 0);
    double s1 = 0.0, s2 = 0.0;
    for (int64_t a0 = 0; a0 < m; a0 += kTile) {
      __syncthreads();
      if (a0 + threadIdx.x < m) tile[threadIdx.x] = atoms[a0 + threadIdx.x];
      __syncthreads();
      const int lim = (int)min((int64_t)kTile, m - a0);
#pragma unroll 4
      for (int j = 0; j < lim; ++j) {
        const double4 A = tile[j];
        const double dx = V.x - A.x, dy = V.y - A.y, dz = V.z - A.z;
        const double y = rsqrt_nr1(dx * dx + dy * dy + dz * dz);
        s1 += A.w * y;
        if (IONIC) s2 += A.w * (dx * Dv.x + dy * Dv.y + dz * Dv.z) * (y * y * y);
      }
    }
    if (live) {
      acc1 += V.w * s1;
      acc2 += s2;
      accF += V.w;
    }
  }
  typedef cub::BlockReduce<double, kTile> BR;
  __shared__ typename BR::TempStorage tmp;
  const double t1 = BR(tmp).Sum(acc1);
  __syncthreads();
  const double t2 = BR(tmp).Sum(acc2);
  __syncthreads();
  const double t3 = BR(tmp).Sum(accF);
  if (threadIdx.x == 0) {
    partials[3 * blockIdx.x] = t1;
    partials[3 * blockIdx.x + 1] = t2;
    partials[3 * blockIdx.x + 2] = t3;
  }
}

// sum_{i<j} q_i q_j / r_ij
__global__ void __launch_bounds__(kTile) k_coulomb(const double4* __restrict__ atoms, int64_t m,
                                                   double* __restrict__ partials) {
  __shared__ double4 tile[kTile];
  double acc = 0.0;
  for (int64_t base = blockIdx.x * (int64_t)kTile; base < m; base += (int64_t)gridDim.x * kTile) {
    const int64_t i = base + threadIdx.x;
    const double4 P = i < m ? atoms[i] : make_double4(0, 0, 0, 0);
    double s = 0.0;
    for (int64_t a0 = base; a0 < m; a0 += kTile) {  // j >= base covers every j > i
      __syncthreads();
      if (a0 + threadIdx.x < m) tile[threadIdx.x] = atoms[a0 + threadIdx.x];
      __syncthreads();
      const int lim = (int)min((int64_t)kTile, m - a0);
      for (int j = 0; j < lim; ++j) {
        if (a0 + j <= i) continue;
        const double4 A = tile[j];
        const double dx = P.x - A.x, dy = P.y - A.y, dz = P.z - A.z;
        s += A.w * rsqrt_nr(dx * dx + dy * dy + dz * dz);
      }
    }
    if (i < m) acc += P.w * s;
  }
  typedef cub::BlockReduce<double, kTile> BR;
  __shared__ typename BR::TempStorage tmp;
  const double tot = BR(tmp).Sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = tot;
}

// write_potential_on_atoms_fast: trilinear interpolation in the atom's octant.
__global__ void k_phi_atoms(const double4* __restrict__ atoms, int64_t na, const int32_t* __restrict__ atom_oct,
                            EnergyView E, double* __restrict__ out) {
  const int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (a >= na) return;
  const int32_t o = atom_oct[a];
  if (o < 0) {
    out[a] = __longlong_as_double(0x7ff8000000000000LL);
    return;
  }
  const double4 P = atoms[a];
  const int4 q = E.oct[o];
  const int32_t s = 1 << (kRootLog - q.w);
  const int32_t qc[3] = {q.x, q.y, q.z};
  double lo_c[3], hi_c[3];
  for (int d = 0; d < 3; ++d) {
    lo_c[d] = coord(E.lo[d], E.len[d], qc[d]);
    hi_c[d] = coord(E.lo[d], E.len[d], qc[d] + s);
  }
  const double volume = (hi_c[0] - lo_c[0]) * (hi_c[1] - lo_c[1]) * (hi_c[2] - lo_c[2]);
  double phi = 0.0;
  for (int c = 0; c < 8; ++c) {
    const int oc = 7 - c;
    const double X = (oc & 1) ? hi_c[0] : lo_c[0], Y = ((oc >> 1) & 1) ? hi_c[1] : lo_c[1],
                 Z = ((oc >> 2) & 1) ? hi_c[2] : lo_c[2];
    const double w = fabs((P.x - X) * (P.y - Y) * (P.z - Z)) / volume;
    phi += cval(E.phi, E.oct_nodes[8 * (int64_t)o + c], E) * w;
  }
  out[a] = phi;
}

// The table goes to constant memory of the context's device on every call
// (4 KiB), so contexts on different devices each get their copy.
static int ensure_tri(Context* c) {
  signed char tri[256][16];
  pbmc::expand_tri_table(tri);
  PBGPU_CUDA(c, cudaMemcpyToSymbolAsync(d_tri, tri, sizeof(tri), 0, cudaMemcpyHostToDevice, c->stream));
  return PBGPU_OK;
}

static EnergyView energy_view(Context* c, int fast) {
  EnergyView E{};
  E.oct = c->oct.get();
  E.oct_nodes = c->oct_nodes.get();
  E.hang_par = c->hang_par.get();
  E.hang_np = c->hang_np.get();
  E.border = c->border.get();
  E.eps = c->eps.get();
  E.phi = c->phi.get();
  int64_t base = 0;
  for (int a = 0; a < 3; ++a) {
    E.rays[a] = ray_view(c->rays[a]);
    E.lo[a] = c->lo[a];
    E.len[a] = c->len[a];
    E.h0[a] = 0.0;
    E.slot_base[a] = base;
    base += c->rays[a].nc;
  }
  E.n = c->n;
  E.nb = c->nb;
  E.eps_out = c->eps_out;
  E.fast = fast;
  E.ionic = c->model.calc_energy == 2 && c->kappa > 1.e-5;
  return E;
}

int run_phi_atoms(Context* c, double* out) {
  if (!c->have_phi) return c->fail(PBGPU_ERR_STATE, "phi_on_atoms: solve has not run");
  if (!c->have_density) return c->fail(PBGPU_ERR_STATE, "phi_on_atoms: create_density_map has not run");
  if (c->na == 0) return PBGPU_OK;
  Scratch<double> d(c, kScEnPhi);
  PBGPU_CUDA(c, d.alloc(c->na));
  EnergyView E = energy_view(c, 0);
  k_phi_atoms<<<grid_for(c->na, 128), 128, 0, c->stream>>>(c->atoms.get(), c->na, c->atom_oct.get(), E, d.get());
  PBGPU_LAUNCHED(c);
  PBGPU_CUDA(c, cudaMemcpyAsync(out, d.get(), c->na * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  return PBGPU_OK;
}

static int sum_partials(Context* c, const double* d, int nblk, int stride, double* out) {
  std::vector<double> h((size_t)nblk * stride);
  PBGPU_CUDA(c, readback(c, h.data(), d, h.size() * sizeof(double)));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  for (int k = 0; k < stride; ++k) {
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += h[(size_t)b * stride + k];
    out[k] = s;
  }
  return PBGPU_OK;
}

// The surface points of every border octant's elements, merged per crossing
// (steps (1) and (2) above): P[i] = (V, F) and, with `ionic`, D[i] = sum of
// coef * N of the triangle vertices on that crossing.  `fast` takes the
// spacing of the first border octant for every octant, as energy_fast and
// pot_field_fast do.  The lists live in the context's scratch slots.
int surface_points(Context* c, int fast, bool ionic, SurfacePoints* out) {
  out->P = nullptr;
  out->D = nullptr;
  out->n = 0;
  int st = ensure_tri(c);
  if (st != PBGPU_OK) return st;
  EnergyView E = energy_view(c, fast);
  E.ionic = ionic;
  const int64_t nb = c->nb;
  if (nb == 0) return PBGPU_OK;
  if (fast) {
    int32_t b0 = 0;
    int4 q;
    PBGPU_CUDA(c, readback(c, &b0, c->border.get(), sizeof(int32_t)));
    PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    PBGPU_CUDA(c, readback(c, &q, c->oct.get() + b0, sizeof(int4)));
    PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    const int32_t s = 1 << (kRootLog - q.w);
    const int32_t qc[3] = {q.x, q.y, q.z};
    for (int a = 0; a < 3; ++a) {
      const double l = c->lo[a] + c->len[a] * (double(qc[a]) * 0x1p-19);
      const double r = c->lo[a] + c->len[a] * (double(qc[a] + s) * 0x1p-19);
      E.h0[a] = r - l;
    }
  }
  const int64_t nslots = c->rays[0].nc + c->rays[1].nc + c->rays[2].nc;
  const int64_t ns = nslots > 0 ? nslots : 1;
  Scratch<unsigned long long> acc(c, kScEnAcc);
  Scratch<uint8_t> used(c, kScEnUsed);
  Scratch<int32_t> slot_ray(c, kScEnSlotRay), sel(c, kScEnSel);
  Scratch<int64_t> nsel(c, kScEnNsel);
  Scratch<unsigned long long> n_extra(c, kScEnNextra);
  // elements whose edge carries no crossing (an epsilon jump seen through a
  // hanging corner) keep their own point; their list starts at nb entries and
  // is grown and the pass repeated if it overflows
  int64_t extra_cap = nb + 1024;
  Scratch<double4> xp(c, kScEnXp), xd(c, kScEnXd);
  Scratch<unsigned long long> xk(c, kScEnXk), xk2(c, kScEnXk2), xi(c, kScEnXi), xi2(c, kScEnXi2);
  PBGPU_CUDA(c, acc.alloc(8 * ns));
  PBGPU_CUDA(c, used.alloc(ns));
  PBGPU_CUDA(c, slot_ray.alloc(ns));
  PBGPU_CUDA(c, sel.alloc(ns));
  PBGPU_CUDA(c, nsel.alloc(1));
  PBGPU_CUDA(c, n_extra.alloc(1));
  E.acc = acc.get();
  E.used = used.get();
  E.slot_ray = slot_ray.get();
  E.n_extra = n_extra.get();
  unsigned long long nx = 0;
  for (int attempt = 0; attempt < 2; ++attempt) {
    PBGPU_CUDA(c, xp.alloc(extra_cap));
    PBGPU_CUDA(c, xd.alloc(extra_cap));
    PBGPU_CUDA(c, xk.alloc(extra_cap));
    PBGPU_CUDA(c, cudaMemsetAsync(acc.get(), 0, 8 * ns * sizeof(unsigned long long), c->stream));
    PBGPU_CUDA(c, cudaMemsetAsync(used.get(), 0, ns, c->stream));
    PBGPU_CUDA(c, cudaMemsetAsync(n_extra.get(), 0, sizeof(unsigned long long), c->stream));
    E.extra_p = xp.get();
    E.extra_d = xd.get();
    E.extra_key = xk.get();
    E.extra_cap = extra_cap;
    k_energy_accumulate<<<grid_for(nb, 128), 128, 0, c->stream>>>(E);
    PBGPU_LAUNCHED(c);
    PBGPU_CUDA(c, readback(c, &nx, n_extra.get(), sizeof(nx)));
    PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    if ((int64_t)nx <= extra_cap) break;
    extra_cap = (int64_t)nx;
  }
  if ((int64_t)nx > extra_cap) return c->fail(PBGPU_ERR_CAPACITY, "energy: surface element list overflow");
  cub::CountingInputIterator<int32_t> idx(0);
  size_t bytes = 0;
  PBGPU_CUDA(c, cub::DeviceSelect::Flagged(nullptr, bytes, idx, used.get(), sel.get(), nsel.get(), ns, c->stream));
  PBGPU_CUDA(c, ensure_tmp(c, bytes));
  PBGPU_CUDA(c, cub::DeviceSelect::Flagged(c->tmp.get(), bytes, idx, used.get(), sel.get(), nsel.get(), ns, c->stream));
  c->launches += kCubSelectLaunches;
  int64_t np = 0;
  PBGPU_CUDA(c, readback(c, &np, nsel.get(), sizeof(int64_t)));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  const int64_t npts = np + (int64_t)nx;
  Scratch<double4> P(c, kScEnP), D(c, kScEnD);
  PBGPU_CUDA(c, P.alloc(npts > 0 ? npts : 1));
  PBGPU_CUDA(c, D.alloc(npts > 0 ? npts : 1));
  if (np) {
    k_energy_points<<<grid_for(np, 256), 256, 0, c->stream>>>(sel.get(), np, E, P.get(), D.get());
    PBGPU_LAUNCHED(c);
  }
  if (nx) {
    // the order the atomics handed out is arbitrary: sort by (octant, element)
    const int m = (int)nx;
    PBGPU_CUDA(c, xk2.alloc(m));
    PBGPU_CUDA(c, xi.alloc(m));
    PBGPU_CUDA(c, xi2.alloc(m));
    k_iota_u64<<<grid_for(m, 256), 256, 0, c->stream>>>(xi.get(), m);
    PBGPU_LAUNCHED(c);
    size_t bytes = 0;
    PBGPU_CUDA(c, cub::DeviceRadixSort::SortPairs(nullptr, bytes, xk.get(), xk2.get(), xi.get(), xi2.get(), m, 0, 64,
                                                  c->stream));
    PBGPU_CUDA(c, ensure_tmp(c, bytes));
    PBGPU_CUDA(c, cub::DeviceRadixSort::SortPairs(c->tmp.get(), bytes, xk.get(), xk2.get(), xi.get(), xi2.get(), m, 0,
                                                  64, c->stream));
    c->launches += cub_radix_launches(m, 64);
    k_gather_extras<<<grid_for(m, 256), 256, 0, c->stream>>>(xi2.get(), m, xp.get(), xd.get(), P.get() + np,
                                                             D.get() + np);
    PBGPU_LAUNCHED(c);
  }
  out->P = P.get();
  out->D = D.get();
  out->n = npts;
  return PBGPU_OK;
}

int run_energy(Context* c, int fast, pbgpu_energy_out* out) {
  if (!c->have_phi) return c->fail(PBGPU_ERR_STATE, "energy: solve has not run");
  if (!c->have_markers) return c->fail(PBGPU_ERR_STATE, "energy: create_markers has not run");
  int st;
  const int64_t nb = c->nb;
  const double inv_4pi = 1.0 / (4.0 * kPi);
  const double constant_pol = (1.0 / c->eps_out - 1.0 / c->eps_in) * inv_4pi;
  const double constant_react = (1.0 / c->eps_out) * inv_4pi;
  const bool ionic = c->model.calc_energy == 2 && c->kappa > 1.e-5;
  const bool polar = c->model.calc_energy == 1 || (c->model.calc_energy == 2 && c->kappa < 1.e-5);
  // charged atoms (|q| > 1e-5, src/pb_class.cpp:2829-2834)
  std::vector<double4> ha(c->na);
  if (c->na) {
    PBGPU_CUDA(c, cudaMemcpyAsync(ha.data(), c->atoms.get(), c->na * sizeof(double4), cudaMemcpyDeviceToHost, c->stream));
    PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  std::vector<double4> qa;
  double net = 0.0;
  for (const double4& a : ha) {
    net += a.w;
    if (std::fabs(a.w) > 1.e-5) qa.push_back(a);
  }
  const int64_t m = (int64_t)qa.size();
  Scratch<double4> dq(c, kScEnQ);
  PBGPU_CUDA(c, dq.alloc(m > 0 ? m : 1));
  if (m) PBGPU_CUDA(c, cudaMemcpyAsync(dq.get(), qa.data(), m * sizeof(double4), cudaMemcpyHostToDevice, c->stream));
  const int nblk = c->sm_count * 4;
  PBGPU_CUDA(c, c->energy_part.alloc(3 * nblk));
  double first_int = 0.0, second_int = 0.0, charge_pol = 0.0, coul = 0.0;
  if ((polar || ionic) && nb > 0) {
    SurfacePoints sp;
    if ((st = surface_points(c, fast, ionic, &sp)) != PBGPU_OK) return st;
    const int64_t npts = sp.n;
    c->energy_points = npts;
    c->energy_pairs += npts * m;
    if (npts) {
      double s[3] = {0, 0, 0};
      if (ionic)
        k_energy_pairs<true><<<nblk, kTile, 0, c->stream>>>(sp.P, sp.D, npts, dq.get(), m, c->energy_part.get());
      else
        k_energy_pairs<false><<<nblk, kTile, 0, c->stream>>>(sp.P, sp.D, npts, dq.get(), m, c->energy_part.get());
      PBGPU_LAUNCHED(c);
      if ((st = sum_partials(c, c->energy_part.get(), nblk, 3, s)) != PBGPU_OK) return st;
      first_int = s[0];
      second_int = s[1];
      charge_pol = s[2];
    }
  }
  if (c->model.calc_coulombic == 1 && m > 1) {
    k_coulomb<<<nblk, kTile, 0, c->stream>>>(dq.get(), m, c->energy_part.get());
    PBGPU_LAUNCHED(c);
    if ((st = sum_partials(c, c->energy_part.get(), nblk, 1, &coul)) != PBGPU_OK) return st;
    coul *= 1.0 / c->eps_in;
  }
  pbgpu_energy_out e{};
  e.energy_pol = (polar || ionic) ? 0.5 * constant_pol * first_int : 0.0;
  e.energy_react = ionic ? 0.5 * (second_int - first_int * constant_react) : 0.0;
  e.energy_coul = coul;
  e.charge_flux = charge_pol / (4.0 * kPi);
  e.net_charge = net;
  e.sum = e.energy_pol + e.energy_react + e.energy_coul;
  *out = e;
  return PBGPU_OK;
}

}  // namespace pbgpu
