// Potential and field at the atoms, split into Coulomb, polarisation and
// ionic parts: pot_field (src/pb_class.cpp:4390-5060) and pot_field_fast
// (:3732-4388).
//
// The reference walks every border octant and, for each flux element and each
// marching-cubes triangle vertex, loops over all atoms adding into per-atom
// arrays.  Here the elements are first merged per crossing into the surface
// points that the energy path builds (surface_points: P = (V, F) and
// D = sum of coef * N, coef = phi0 * area / (12 pi)), and the sums are turned
// around: one thread per atom walks the points, staged through shared memory
// in tiles, so every per-atom sum has one writer and a fixed order.  The
// point list is cut into chunks along the grid's y dimension so that a few
// thousand atoms still fill the GPU; a second kernel adds the chunk partials
// in chunk order and applies the reference's constants, including its final
// phi_i -= phi_p / constant_pol * constant_react (:4285-4288).
//
// Per atom a at x_a, with d = x_a - V, r = |d| and dot = -(d . D):
//   phi_p  = constant_pol * sum F / r
//   E_p    = constant_pol * sum F d / r^3
//   phi_i' = sum dot / r^3
//   E_i'   = sum D / r^3 + 3 d dot / r^5
// which are the reference's element sums, regrouped by crossing (linear in F
// and in coef * N).  The Coulomb part runs over all atom pairs j != i:
//   phi_c = sum q_j / r / eps_in,   E_c = sum q_j (x_i - x_j) / r^3 / eps_in.
// Every atom counts, charged or not, as in the reference's loops.
//
// The surface kernel is bound by the FP64 pipe; 1/r takes one Newton step
// from the FP32 estimate (relative error ~1e-13 per term), the Coulomb kernel
// two.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "pbgpu_internal.cuh"

namespace pbgpu {

constexpr int kPfTile = 128;
constexpr int kPfMaxChunks = 1024;
constexpr int kPfRaw = 8;   // per-atom surface sums
constexpr int kPfCoul = 4;  // per-atom Coulomb sums

// part[(chunk * 8 + k) * na + a]: the chunk's raw surface sums of atom a;
// fpart[chunk]: the chunk's sum of F (written by the first atom tile).
template <bool IONIC, bool FIELD>
__global__ void __launch_bounds__(kPfTile) k_pf_surface(const double4* __restrict__ P, const double4* __restrict__ D,
                                                        int64_t np, int64_t chunk_len,
                                                        const double4* __restrict__ atoms, int64_t na,
                                                        double* __restrict__ part, double* __restrict__ fpart) {
  __shared__ double4 sP[kPfTile];
  __shared__ double4 sD[IONIC ? kPfTile : 1];
  const int64_t a = blockIdx.x * (int64_t)kPfTile + threadIdx.x;
  const bool live = a < na;
  const double4 A = live ? atoms[a] : make_double4(0, 0, 0, 0);
  const int64_t p0 = blockIdx.y * chunk_len;
  const int64_t p1 = min(np, p0 + chunk_len);
  double sp = 0.0, sfx = 0.0, sfy = 0.0, sfz = 0.0;
  double si = 0.0, six = 0.0, siy = 0.0, siz = 0.0;
  double fsum = 0.0;
  for (int64_t base = p0; base < p1; base += kPfTile) {
    __syncthreads();
    const int64_t i = base + threadIdx.x;
    if (i < p1) {
      const double4 v = P[i];
      sP[threadIdx.x] = v;
      fsum += v.w;
      if (IONIC) sD[threadIdx.x] = D[i];
    }
    __syncthreads();
    const int lim = (int)min((int64_t)kPfTile, p1 - base);
#pragma unroll 2
    for (int j = 0; j < lim; ++j) {
      const double4 V = sP[j];
      const double dx = A.x - V.x, dy = A.y - V.y, dz = A.z - V.z;
      const double y = rsqrt_nr1(dx * dx + dy * dy + dz * dz);
      sp += V.w * y;
      double y3 = 0.0;
      if (FIELD || IONIC) y3 = y * y * y;
      if (FIELD) {
        const double fy3 = V.w * y3;
        sfx += dx * fy3;
        sfy += dy * fy3;
        sfz += dz * fy3;
      }
      if (IONIC) {
        const double4 Dv = sD[j];
        const double dot = -(dx * Dv.x + dy * Dv.y + dz * Dv.z);
        si += dot * y3;
        if (FIELD) {
          const double t = 3.0 * dot * (y3 * y * y);
          six += Dv.x * y3 + dx * t;
          siy += Dv.y * y3 + dy * t;
          siz += Dv.z * y3 + dz * t;
        }
      }
    }
  }
  if (live) {
    double* o = part + (int64_t)blockIdx.y * kPfRaw * na + a;
    o[0 * na] = sp;
    o[1 * na] = sfx;
    o[2 * na] = sfy;
    o[3 * na] = sfz;
    o[4 * na] = si;
    o[5 * na] = six;
    o[6 * na] = siy;
    o[7 * na] = siz;
  }
  if (blockIdx.x == 0) {
    typedef cub::BlockReduce<double, kPfTile> BR;
    __shared__ typename BR::TempStorage tmp;
    const double t = BR(tmp).Sum(fsum);
    if (threadIdx.x == 0) fpart[blockIdx.y] = t;
  }
}

// cpart[(chunk * 4 + k) * na + i]: sum over the chunk's atoms j != i of
// q_j / r and q_j (x_i - x_j) / r^3.
__global__ void __launch_bounds__(kPfTile) k_pf_coulomb(const double4* __restrict__ atoms, int64_t na,
                                                        int64_t chunk_len, double* __restrict__ cpart) {
  __shared__ double4 sA[kPfTile];
  const int64_t i = blockIdx.x * (int64_t)kPfTile + threadIdx.x;
  const bool live = i < na;
  const double4 X = live ? atoms[i] : make_double4(0, 0, 0, 0);
  const int64_t j0 = blockIdx.y * chunk_len;
  const int64_t j1 = min(na, j0 + chunk_len);
  double s = 0.0, ex = 0.0, ey = 0.0, ez = 0.0;
  for (int64_t base = j0; base < j1; base += kPfTile) {
    __syncthreads();
    if (base + threadIdx.x < j1) sA[threadIdx.x] = atoms[base + threadIdx.x];
    __syncthreads();
    const int lim = (int)min((int64_t)kPfTile, j1 - base);
    for (int k = 0; k < lim; ++k) {
      if (base + k == i) continue;
      const double4 B = sA[k];
      const double dx = X.x - B.x, dy = X.y - B.y, dz = X.z - B.z;
      const double y = rsqrt_nr(dx * dx + dy * dy + dz * dz);
      const double qy = B.w * y;
      const double qy3 = qy * y * y;
      s += qy;
      ex += dx * qy3;
      ey += dy * qy3;
      ez += dz * qy3;
    }
  }
  if (live) {
    double* o = cpart + (int64_t)blockIdx.y * kPfCoul * na + i;
    o[0 * na] = s;
    o[1 * na] = ex;
    o[2 * na] = ey;
    o[3 * na] = ez;
  }
}

struct PfConsts {
  double den_in, constant_pol, constant_react;
  int columns;
  int surface;
};

// Chunk partials -> the 12 columns of pot_field.dat, plus per-atom energy
// terms et[3 a + {0,1,2}] = q_a * (raw phi_p, raw phi_i, phi_c).
__global__ void k_pf_finish(const double* __restrict__ part, int nchunks, const double* __restrict__ cpart,
                            int ncchunks, const double4* __restrict__ atoms, int64_t na, PfConsts K,
                            double* __restrict__ out, double* __restrict__ et) {
  const int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (a >= na) return;
  double raw[kPfRaw] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (K.surface)
    for (int c = 0; c < nchunks; ++c)
      for (int k = 0; k < kPfRaw; ++k) raw[k] += part[((int64_t)c * kPfRaw + k) * na + a];
  double cl[kPfCoul] = {0, 0, 0, 0};
  for (int c = 0; c < ncchunks; ++c)
    for (int k = 0; k < kPfCoul; ++k) cl[k] += cpart[((int64_t)c * kPfCoul + k) * na + a];
  double v[PBGPU_PF_COLUMNS];
  v[PBGPU_PF_PHI_C] = cl[0] * K.den_in;
  v[PBGPU_PF_EX_C] = cl[1] * K.den_in;
  v[PBGPU_PF_EY_C] = cl[2] * K.den_in;
  v[PBGPU_PF_EZ_C] = cl[3] * K.den_in;
  v[PBGPU_PF_PHI_P] = raw[0] * K.constant_pol;
  v[PBGPU_PF_EX_P] = raw[1] * K.constant_pol;
  v[PBGPU_PF_EY_P] = raw[2] * K.constant_pol;
  v[PBGPU_PF_EZ_P] = raw[3] * K.constant_pol;
  v[PBGPU_PF_PHI_I] = raw[4] - v[PBGPU_PF_PHI_P] / K.constant_pol * K.constant_react;
  v[PBGPU_PF_EX_I] = raw[5] - v[PBGPU_PF_EX_P] / K.constant_pol * K.constant_react;
  v[PBGPU_PF_EY_I] = raw[6] - v[PBGPU_PF_EY_P] / K.constant_pol * K.constant_react;
  v[PBGPU_PF_EZ_I] = raw[7] - v[PBGPU_PF_EZ_P] / K.constant_pol * K.constant_react;
  for (int k = 0; k < PBGPU_PF_COLUMNS; ++k) out[a * PBGPU_PF_COLUMNS + k] = ((K.columns >> k) & 1) ? v[k] : 0.0;
  const double q = atoms[a].w;
  et[3 * a + 0] = q * raw[0];
  et[3 * a + 1] = q * raw[4];
  et[3 * a + 2] = q * v[PBGPU_PF_PHI_C];
}

static void chunking(int64_t na, int64_t nitems, int sm_count, int* nchunks, int64_t* chunk_len) {
  const int64_t tiles = (na + kPfTile - 1) / kPfTile;
  const int64_t target = (int64_t)sm_count * 8;
  int64_t ch = (target + tiles - 1) / tiles;
  const int64_t item_tiles = std::max<int64_t>(1, (nitems + kPfTile - 1) / kPfTile);
  ch = std::max<int64_t>(1, std::min<int64_t>({ch, item_tiles, kPfMaxChunks}));
  int64_t len = (nitems + ch - 1) / ch;
  len = std::max<int64_t>(kPfTile, (len + kPfTile - 1) / kPfTile * kPfTile);
  *chunk_len = len;
  *nchunks = (int)std::max<int64_t>(1, (nitems + len - 1) / len);
}

int run_pot_field(Context* c, int fast, int pt, int ft, double* per_atom, pbgpu_pot_field_out* out) {
  if (!out) return c->fail(PBGPU_ERR_ARG, "pot_field: out is NULL");
  if (pt < 0 || pt > 2 || ft < 0 || ft > 2)
    return c->fail(PBGPU_ERR_ARG, "pot_field: calc_potential_terms and calc_field_terms take 0, 1 or 2");
  if (!c->have_phi) return c->fail(PBGPU_ERR_STATE, "pot_field: solve has not run");
  if (!c->have_markers) return c->fail(PBGPU_ERR_STATE, "pot_field: create_markers has not run");
  // the reference's branches (src/pb_class.cpp:3840, 3884, 3937, 4035, 4125):
  // a1/a2 flux only, b1/b2/b3 flux + triangles (salt)
  const bool salt = c->kappa > 1.e-5;
  const bool a1 = (ft == 1 || (ft == 2 && !salt)) && pt < 2;
  const bool a2 = !a1 && (pt == 1 || (pt == 2 && !salt)) && ft == 0;
  const bool b1 = ft == 2 && salt;
  const bool b2 = !b1 && pt == 2 && salt && ft == 0;
  const bool b3 = !b1 && !b2 && pt == 2 && salt && ft == 1;
  const bool surface = a1 || a2 || b1 || b2 || b3;
  const bool ionic = b1 || b2 || b3;
  const bool field = a1 || b1 || b3;
  // the columns of pot_field.dat under the same options (:4281-4375)
  const int kC = (1 << PBGPU_PF_PHI_C) | (7 << PBGPU_PF_EX_C);
  const int kP = 1 << PBGPU_PF_PHI_P, kEP = 7 << PBGPU_PF_EX_P;
  const int kI = 1 << PBGPU_PF_PHI_I, kEI = 7 << PBGPU_PF_EX_I;
  int columns = 0;
  if (b1)
    columns = kC | kP | kEP | kI | kEI;
  else if (b2)
    columns = kC | kP | kI;
  else if (b3)
    columns = kC | kP | kEP | kI;
  else if (a2)
    columns = kC | kP;
  else if (a1)
    columns = kC | kP | kEP;

  const int64_t na = c->na;
  const double inv_4pi = 1.0 / (4.0 * kPi);
  PfConsts K;
  K.den_in = 1.0 / c->eps_in;
  K.constant_pol = (1.0 / c->eps_out - 1.0 / c->eps_in) * inv_4pi;
  K.constant_react = (1.0 / c->eps_out) * inv_4pi;
  K.columns = columns;
  K.surface = 0;
  *out = pbgpu_pot_field_out{};
  out->columns = columns;
  if (na == 0) return PBGPU_OK;

  int st;
  SurfacePoints sp{nullptr, nullptr, 0};
  if (surface && c->nb > 0)
    if ((st = surface_points(c, fast, ionic, &sp)) != PBGPU_OK) return st;
  const bool run_surface = surface && sp.n > 0;
  K.surface = run_surface ? 1 : 0;

  int nch = 0, ncc = 0;
  int64_t len = 0, clen = 0;
  if (run_surface) chunking(na, sp.n, c->sm_count, &nch, &len);
  chunking(na, na, c->sm_count, &ncc, &clen);
  const int64_t n_part = run_surface ? (int64_t)nch * kPfRaw * na : 0;
  const int64_t n_cpart = (int64_t)ncc * kPfCoul * na;
  Scratch<double> part(c, kScPfPart), res(c, kScPfOut);
  PBGPU_CUDA(c, part.alloc(n_part + n_cpart + kPfMaxChunks));
  PBGPU_CUDA(c, res.alloc(na * (PBGPU_PF_COLUMNS + 3)));
  double* d_part = part.get();
  double* d_cpart = d_part + n_part;
  double* d_fpart = d_cpart + n_cpart;
  double* d_out = res.get();
  double* d_et = d_out + na * PBGPU_PF_COLUMNS;
  const unsigned tiles = (unsigned)((na + kPfTile - 1) / kPfTile);
  if (run_surface) {
    const dim3 grid(tiles, (unsigned)nch);
    if (ionic && field)
      k_pf_surface<true, true><<<grid, kPfTile, 0, c->stream>>>(sp.P, sp.D, sp.n, len, c->atoms.get(), na, d_part,
                                                                d_fpart);
    else if (ionic)
      k_pf_surface<true, false><<<grid, kPfTile, 0, c->stream>>>(sp.P, sp.D, sp.n, len, c->atoms.get(), na, d_part,
                                                                 d_fpart);
    else if (field)
      k_pf_surface<false, true><<<grid, kPfTile, 0, c->stream>>>(sp.P, sp.D, sp.n, len, c->atoms.get(), na, d_part,
                                                                 d_fpart);
    else
      k_pf_surface<false, false><<<grid, kPfTile, 0, c->stream>>>(sp.P, sp.D, sp.n, len, c->atoms.get(), na,
                                                                  d_part, d_fpart);
    PBGPU_LAUNCHED(c);
    c->energy_points = sp.n;
    c->energy_pairs += sp.n * na;
  }
  k_pf_coulomb<<<dim3(tiles, (unsigned)ncc), kPfTile, 0, c->stream>>>(c->atoms.get(), na, clen, d_cpart);
  PBGPU_LAUNCHED(c);
  k_pf_finish<<<grid_for(na, 128), 128, 0, c->stream>>>(d_part, nch, d_cpart, ncc, c->atoms.get(), na, K, d_out,
                                                        d_et);
  PBGPU_LAUNCHED(c);
  std::vector<double> et((size_t)na * 3);
  std::vector<double> fp(run_surface ? nch : 0);
  if (per_atom)
    PBGPU_CUDA(c, cudaMemcpyAsync(per_atom, d_out, na * PBGPU_PF_COLUMNS * sizeof(double), cudaMemcpyDeviceToHost,
                                  c->stream));
  PBGPU_CUDA(c, cudaMemcpyAsync(et.data(), d_et, et.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (run_surface)
    PBGPU_CUDA(c, cudaMemcpyAsync(fp.data(), d_fpart, nch * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  PBGPU_CUDA(c, cudaStreamSynchronize(c->stream));
  double first_int = 0.0, second_int = 0.0, coul2 = 0.0, charge_pol = 0.0;
  for (int64_t a = 0; a < na; ++a) {
    first_int += et[3 * a];
    second_int += et[3 * a + 1];
    coul2 += et[3 * a + 2];
  }
  for (double f : fp) charge_pol += f;
  out->energy_pol = surface ? 0.5 * K.constant_pol * first_int : 0.0;
  out->energy_react = ionic ? 0.5 * (second_int - first_int * K.constant_react) : 0.0;
  out->energy_coul = 0.5 * coul2;
  out->charge_flux = charge_pol / (4.0 * kPi);
  return PBGPU_OK;
}

}  // namespace pbgpu
