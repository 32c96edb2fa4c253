// Post-processing on the device: potential at the atoms
// (write_potential_on_atoms_fast, src/pb_class.cpp:2333-2417) and the
// electrostatic energy (energy / energy_fast, :2791-3338).
//
// The energy is split in two phases.  (1) One thread per border octant builds
// the octant's surface elements exactly as the reference walks them: one flux
// element (point V on each epsilon-jump edge, flux F) per jump edge, and three
// vertex elements (point V, outward normal N, coefficient phi0 * area / (12 pi))
// per marching-cubes triangle.  Counts go through a scan so the elements are
// packed in border order.  (2) The pair sums over elements x charged atoms run
// as FP64 N-body kernels with the atoms staged in shared memory tiles; block
// partials are summed in fixed order, so the energy is deterministic.
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
// lies on the edge, returns the fraction (0.5 when none).
__device__ __forceinline__ double normal_intersection(const EnergyView& E, CellCtx& C, int e) {
  const int axis = d_edge_axis[e], i1 = d_edge_nodes[2 * e], i2 = d_edge_nodes[2 * e + 1];
  const double x1 = coord(E.lo[axis], E.len[axis], corner_i(C, i1, axis));
  const double x2 = coord(E.lo[axis], E.len[axis], corner_i(C, i2, axis));
  const int t0 = axis == 0 ? 1 : 0, t1 = axis == 2 ? 1 : 2;
  const RayView& R = E.rays[axis];
  double f = 0.5;
  const int32_t r = ray_find(R.hk, R.hv, R.cap, R.cap_log, ray_key(corner_i(C, i1, t0), corner_i(C, i1, t1)));
  if (r >= 0)
    for (int64_t k = R.ptr[r]; k < R.ptr[r + 1]; ++k) {
      const double I = R.inters[k];
      if (I >= x1 && I <= x2) {
        C.N[0] = R.normals[3 * k];
        C.N[1] = R.normals[3 * k + 1];
        C.N[2] = R.normals[3 * k + 2];
        f = (I - x1) / (x2 - x1);
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

// counts of flux elements and triangle-vertex elements per border octant
__global__ void k_energy_count(EnergyView E, int32_t* __restrict__ nflux, int32_t* __restrict__ ntri) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b >= E.nb) return;
  CellCtx C;
  cell_load(E, b, C);
  int nf = 0;
  for (int e = 0; e < 12; ++e) nf += C.te[d_edge_nodes[2 * e]] != C.te[d_edge_nodes[2 * e + 1]];
  int nt = 0;
  if (E.ionic) {
    const int k = cube_index(C, E.eps_out);
    if (k != 0 && k != 255)
      while (nt < 5 && d_tri[k][3 * nt] >= 0) ++nt;
  }
  nflux[b] = nf;
  ntri[b] = 3 * nt;
}

__global__ void k_energy_fill(EnergyView E, const int64_t* __restrict__ off_flux, const int64_t* __restrict__ off_tri,
                              double4* __restrict__ flux, double4* __restrict__ triv, double4* __restrict__ trin) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b >= E.nb) return;
  CellCtx C;
  cell_load(E, b, C);
  int64_t wf = off_flux[b];
  for (int e = 0; e < 12; ++e) {
    const int i1 = d_edge_nodes[2 * e], i2 = d_edge_nodes[2 * e + 1];
    double dir;
    if (C.te[i1] < C.te[i2])
      dir = 1;
    else if (C.te[i1] > C.te[i2])
      dir = -1;
    else
      continue;
    const double f = normal_intersection(E, C, e);
    double V[3];
    edge_point(E, C, e, f, V);
    const double F = -(C.tp[i2] - C.tp[i1]) * wha(C.te[i1], C.te[i2], f) * dir * C.area_h[d_edge_axis[e]];
    flux[wf++] = make_double4(V[0], V[1], V[2], F);
  }
  if (!E.ionic) return;
  const int k = cube_index(C, E.eps_out);
  if (k == 0 || k == 255) return;
  int64_t wt = off_tri[b];
  const double inv_4pi = 1.0 / (4.0 * kPi);
  for (int t = 0; t < 5 && d_tri[k][3 * t] >= 0; ++t) {
    double VT[3][3], NT[3][3], ps[3];
    for (int j = 0; j < 3; ++j) {
      const int e = d_tri[k][3 * t + j];
      const int i1 = d_edge_nodes[2 * e], i2 = d_edge_nodes[2 * e + 1];
      const double f = normal_intersection(E, C, e);
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
      triv[wt] = make_double4(VT[j][0], VT[j][1], VT[j][2], ps[j] * inv_4pi * area / 3.0);
      trin[wt] = make_double4(NT[j][0], NT[j][1], NT[j][2], 0.0);
      ++wt;
    }
  }
}

constexpr int kTile = 256;

// sum over elements e of coef_e * sum_a q_a / |x_a - V_e|
__global__ void __launch_bounds__(kTile) k_nbody_flux(const double4* __restrict__ el, int64_t ne,
                                                      const double4* __restrict__ atoms, int64_t m,
                                                      double* __restrict__ partials) {
  __shared__ double4 tile[kTile];
  double acc = 0.0;
  for (int64_t base = blockIdx.x * (int64_t)kTile; base < ne; base += (int64_t)gridDim.x * kTile) {
    const int64_t e = base + threadIdx.x;
    const double4 E = e < ne ? el[e] : make_double4(0, 0, 0, 0);
    double s = 0.0;
    for (int64_t a0 = 0; a0 < m; a0 += kTile) {
      __syncthreads();
      if (a0 + threadIdx.x < m) tile[threadIdx.x] = atoms[a0 + threadIdx.x];
      __syncthreads();
      const int lim = (int)min((int64_t)kTile, m - a0);
#pragma unroll 4
      for (int j = 0; j < lim; ++j) {
        const double4 A = tile[j];
        const double dx = A.x - E.x, dy = A.y - E.y, dz = A.z - E.z;
        s += A.w * rsqrt(dx * dx + dy * dy + dz * dz);
      }
    }
    if (e < ne) acc += E.w * s;  // idle lanes sit at the origin and may hit an atom there
  }
  typedef cub::BlockReduce<double, kTile> BR;
  __shared__ typename BR::TempStorage tmp;
  const double tot = BR(tmp).Sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = tot;
}

// sum over vertex elements of coef_e * sum_a q_a (V_e - x_a).N_e / |V_e - x_a|^3
__global__ void __launch_bounds__(kTile) k_nbody_tri(const double4* __restrict__ ev, const double4* __restrict__ en,
                                                     int64_t ne, const double4* __restrict__ atoms, int64_t m,
                                                     double* __restrict__ partials) {
  __shared__ double4 tile[kTile];
  double acc = 0.0;
  for (int64_t base = blockIdx.x * (int64_t)kTile; base < ne; base += (int64_t)gridDim.x * kTile) {
    const int64_t e = base + threadIdx.x;
    const double4 V = e < ne ? ev[e] : make_double4(0, 0, 0, 0);
    const double4 N = e < ne ? en[e] : make_double4(0, 0, 0, 0);
    double s = 0.0;
    for (int64_t a0 = 0; a0 < m; a0 += kTile) {
      __syncthreads();
      if (a0 + threadIdx.x < m) tile[threadIdx.x] = atoms[a0 + threadIdx.x];
      __syncthreads();
      const int lim = (int)min((int64_t)kTile, m - a0);
#pragma unroll 4
      for (int j = 0; j < lim; ++j) {
        const double4 A = tile[j];
        const double dx = V.x - A.x, dy = V.y - A.y, dz = V.z - A.z;
        const double ri = rsqrt(dx * dx + dy * dy + dz * dz);
        s += A.w * (dx * N.x + dy * N.y + dz * N.z) * (ri * ri * ri);
      }
    }
    if (e < ne) acc += V.w * s;
  }
  typedef cub::BlockReduce<double, kTile> BR;
  __shared__ typename BR::TempStorage tmp;
  const double tot = BR(tmp).Sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = tot;
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
        s += A.w * rsqrt(dx * dx + dy * dy + dz * dz);
      }
    }
    if (i < m) acc += P.w * s;
  }
  typedef cub::BlockReduce<double, kTile> BR;
  __shared__ typename BR::TempStorage tmp;
  const double tot = BR(tmp).Sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = tot;
}

__global__ void k_flux_total(const double4* __restrict__ flux, int64_t ne, double* __restrict__ partials) {
  double acc = 0.0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne; e += (int64_t)gridDim.x * blockDim.x)
    acc += flux[e].w;
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
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  return PBGPU_OK;
}

static EnergyView energy_view(Context* c, int fast) {
  EnergyView E;
  E.oct = c->oct.get();
  E.oct_nodes = c->oct_nodes.get();
  E.hang_par = c->hang_par.get();
  E.hang_np = c->hang_np.get();
  E.border = c->border.get();
  E.eps = c->eps.get();
  E.phi = c->phi.get();
  for (int a = 0; a < 3; ++a) {
    E.rays[a] = ray_view(c->rays[a]);
    E.lo[a] = c->lo[a];
    E.len[a] = c->len[a];
    E.h0[a] = 0.0;
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
  DBuf<double> d;
  PBGPU_CUDA(c, d.alloc(c->na));
  EnergyView E = energy_view(c, 0);
  k_phi_atoms<<<grid_for(c->na, 128), 128, 0, c->stream>>>(c->atoms.get(), c->na, c->atom_oct.get(), E, d.get());
  PBGPU_LAUNCHED(c);
  PBGPU_CUDA(c, cudaMemcpyAsync(out, d.get(), c->na * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  return PBGPU_OK;
}

static int sum_partials(Context* c, const double* d, int nblk, double* out) {
  std::vector<double> h(nblk);
  PBGPU_CUDA(c, cudaMemcpyAsync(h.data(), d, nblk * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  double s = 0.0;
  for (double v : h) s += v;
  *out = s;
  return PBGPU_OK;
}

int run_energy(Context* c, int fast, pbgpu_energy_out* out) {
  if (!c->have_phi) return c->fail(PBGPU_ERR_STATE, "energy: solve has not run");
  if (!c->have_markers) return c->fail(PBGPU_ERR_STATE, "energy: create_markers has not run");
  int st = ensure_tri(c);
  if (st != PBGPU_OK) return st;
  EnergyView E = energy_view(c, fast);
  const int64_t nb = c->nb;
  if (fast && nb > 0) {
    int32_t b0 = 0;
    int4 q;
    PBGPU_CUDA(c, cudaMemcpy(&b0, c->border.get(), sizeof(int32_t), cudaMemcpyDeviceToHost));
    PBGPU_CUDA(c, cudaMemcpy(&q, c->oct.get() + b0, sizeof(int4), cudaMemcpyDeviceToHost));
    const int32_t s = 1 << (kRootLog - q.w);
    const int32_t qc[3] = {q.x, q.y, q.z};
    for (int a = 0; a < 3; ++a) {
      const double l = c->lo[a] + c->len[a] * (double(qc[a]) * 0x1p-19);
      const double r = c->lo[a] + c->len[a] * (double(qc[a] + s) * 0x1p-19);
      E.h0[a] = r - l;
    }
  }
  const double inv_4pi = 1.0 / (4.0 * kPi);
  const double constant_pol = (1.0 / c->eps_out - 1.0 / c->eps_in) * inv_4pi;
  const double constant_react = (1.0 / c->eps_out) * inv_4pi;
  const bool ionic = E.ionic;
  const bool polar = c->model.calc_energy == 1 || (c->model.calc_energy == 2 && c->kappa < 1.e-5);
  // charged atoms
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
  DBuf<double4> dq;
  PBGPU_CUDA(c, dq.alloc(m > 0 ? m : 1));
  if (m) PBGPU_CUDA(c, cudaMemcpyAsync(dq.get(), qa.data(), m * sizeof(double4), cudaMemcpyHostToDevice, c->stream));
  const int nblk = c->sm_count * 4;
  PBGPU_CUDA(c, c->energy_part.alloc(4 * nblk));
  double first_int = 0.0, second_int = 0.0, charge_pol = 0.0, coul = 0.0;
  if ((polar || ionic) && nb > 0) {
    DBuf<int32_t> nf, nt;
    DBuf<int64_t> of, ot;
    PBGPU_CUDA(c, nf.alloc(nb + 1));
    PBGPU_CUDA(c, nt.alloc(nb + 1));
    PBGPU_CUDA(c, of.alloc(nb + 1));
    PBGPU_CUDA(c, ot.alloc(nb + 1));
    PBGPU_CUDA(c, cudaMemsetAsync(nf.get() + nb, 0, sizeof(int32_t), c->stream));
    PBGPU_CUDA(c, cudaMemsetAsync(nt.get() + nb, 0, sizeof(int32_t), c->stream));
    k_energy_count<<<grid_for(nb, 128), 128, 0, c->stream>>>(E, nf.get(), nt.get());
    PBGPU_LAUNCHED(c);
    size_t bytes = 0;
    PBGPU_CUDA(c, cub::DeviceScan::ExclusiveSum(nullptr, bytes, nf.get(), of.get(), nb + 1, c->stream));
    PBGPU_CUDA(c, ensure_tmp(c, bytes));
    PBGPU_CUDA(c, cub::DeviceScan::ExclusiveSum(c->tmp.get(), bytes, nf.get(), of.get(), nb + 1, c->stream));
    PBGPU_CUDA(c, cub::DeviceScan::ExclusiveSum(c->tmp.get(), bytes, nt.get(), ot.get(), nb + 1, c->stream));
    c->launches += 2 * kCubScanLaunches;
    int64_t nflux = 0, ntri = 0;
    PBGPU_CUDA(c, cudaMemcpyAsync(&nflux, of.get() + nb, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
    PBGPU_CUDA(c, cudaMemcpyAsync(&ntri, ot.get() + nb, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
    PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
    DBuf<double4> fl, tv, tn;
    PBGPU_CUDA(c, fl.alloc(nflux > 0 ? nflux : 1));
    PBGPU_CUDA(c, tv.alloc(ntri > 0 ? ntri : 1));
    PBGPU_CUDA(c, tn.alloc(ntri > 0 ? ntri : 1));
    k_energy_fill<<<grid_for(nb, 128), 128, 0, c->stream>>>(E, of.get(), ot.get(), fl.get(), tv.get(), tn.get());
    PBGPU_LAUNCHED(c);
    double* P = c->energy_part.get();
    if (nflux) {
      k_flux_total<<<nblk, kTile, 0, c->stream>>>(fl.get(), nflux, P);
      PBGPU_LAUNCHED(c);
      if ((st = sum_partials(c, P, nblk, &charge_pol)) != PBGPU_OK) return st;
      if (m) {
        k_nbody_flux<<<nblk, kTile, 0, c->stream>>>(fl.get(), nflux, dq.get(), m, P);
        PBGPU_LAUNCHED(c);
        if ((st = sum_partials(c, P, nblk, &first_int)) != PBGPU_OK) return st;
      }
    }
    if (ionic && ntri && m) {
      k_nbody_tri<<<nblk, kTile, 0, c->stream>>>(tv.get(), tn.get(), ntri, dq.get(), m, P);
      PBGPU_LAUNCHED(c);
      if ((st = sum_partials(c, P, nblk, &second_int)) != PBGPU_OK) return st;
    }
  }
  if (c->model.calc_coulombic == 1 && m > 1) {
    k_coulomb<<<nblk, kTile, 0, c->stream>>>(dq.get(), m, c->energy_part.get());
    PBGPU_LAUNCHED(c);
    if ((st = sum_partials(c, c->energy_part.get(), nblk, &coul)) != PBGPU_OK) return st;
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
