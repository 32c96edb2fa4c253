// Linear octree with 2:1 full balance and p8est-style node tables.
// See octree.h for the conventions and the reference call sites.
#include "octree.h"

#include <omp.h>

#include <algorithm>
#include <cstring>
#include <parallel/algorithm>
#include <stdexcept>

namespace pbh {

static inline uint64_t spread3(uint64_t v) {
  v &= 0x1fffffULL;
  v = (v | v << 32) & 0x1f00000000ffffULL;
  v = (v | v << 16) & 0x1f0000ff0000ffULL;
  v = (v | v << 8) & 0x100f00f00f00f00fULL;
  v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
  v = (v | v << 2) & 0x1249249249249249ULL;
  return v;
}

uint64_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}

static inline bool inside_root(int32_t x, int32_t y, int32_t z) {
  return x >= 0 && y >= 0 && z >= 0 && x < kRootLen && y < kRootLen && z < kRootLen;
}

static inline int child_id(const Octant& q) {
  const int s = kMaxLevel - q.level;
  return ((q.x >> s) & 1) | (((q.y >> s) & 1) << 1) | (((q.z >> s) & 1) << 2);
}

void Octree::rebuild_keys() {
  const int64_t n = size();
  keys.resize(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) keys[i] = morton3(leaves[i].x, leaves[i].y, leaves[i].z);
}

void Octree::uniform(int level) {
  if (level < 0 || level > kQMaxLevel) throw std::runtime_error("uniform: bad level");
  const int64_t n = int64_t(1) << (3 * level);
  leaves.resize(n);
  const int32_t s = 1 << (kMaxLevel - level);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    uint32_t x = 0, y = 0, z = 0;
    for (int b = 0; b < level; ++b) {
      x |= uint32_t((i >> (3 * b)) & 1) << b;
      y |= uint32_t((i >> (3 * b + 1)) & 1) << b;
      z |= uint32_t((i >> (3 * b + 2)) & 1) << b;
    }
    leaves[i] = Octant{int32_t(x) * s, int32_t(y) * s, int32_t(z) * s, level};
  }
  rebuild_keys();
}

int64_t Octree::find_leaf(int32_t x, int32_t y, int32_t z) const {
  const uint64_t k = morton3(uint32_t(x), uint32_t(y), uint32_t(z));
  auto it = std::upper_bound(keys.begin(), keys.end(), k);
  return int64_t(it - keys.begin()) - 1;
}

bool Octree::is_leaf_at(int32_t x, int32_t y, int32_t z, int level) const {
  if (!inside_root(x, y, z)) return false;
  const int64_t j = find_leaf(x, y, z);
  return leaves[j].level == level;
}

std::vector<Octant> Octree::split_marked(const std::vector<uint8_t>& marks) {
  const int64_t n = size();
  std::vector<int64_t> off(n + 1);
  off[0] = 0;
  for (int64_t i = 0; i < n; ++i) off[i + 1] = off[i] + (marks[i] ? 8 : 1);
  std::vector<Octant> out(off[n]);
  std::vector<Octant> parents;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const Octant q = leaves[i];
    if (marks[i]) {
      const int32_t h = q.size() >> 1;
      for (int c = 0; c < 8; ++c)
        out[off[i] + c] = Octant{q.x + (c & 1) * h, q.y + ((c >> 1) & 1) * h,
                                 q.z + ((c >> 2) & 1) * h, q.level + 1};
    } else {
      out[off[i]] = q;
    }
  }
  for (int64_t i = 0; i < n; ++i)
    if (marks[i]) parents.push_back(leaves[i]);
  leaves.swap(out);
  rebuild_keys();
  return parents;
}

// A leaf X of level l is too coarse for its surroundings when one of the
// level-(l+1) cells touching it from outside is itself refined.
static bool touches_too_fine(const Octree& t, const Octant& X) {
  const int32_t S = X.size(), h = S >> 1;
  int32_t opts[3][2];
  int nopt[3];
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        if (!dx && !dy && !dz) continue;
        const int d[3] = {dx, dy, dz};
        const int32_t base[3] = {X.x, X.y, X.z};
        for (int a = 0; a < 3; ++a) {
          if (d[a] < 0) {
            opts[a][0] = base[a] - h;
            nopt[a] = 1;
          } else if (d[a] > 0) {
            opts[a][0] = base[a] + S;
            nopt[a] = 1;
          } else {
            opts[a][0] = base[a];
            opts[a][1] = base[a] + h;
            nopt[a] = 2;
          }
        }
        for (int i = 0; i < nopt[0]; ++i)
          for (int j = 0; j < nopt[1]; ++j)
            for (int k = 0; k < nopt[2]; ++k) {
              const int32_t sx = opts[0][i], sy = opts[1][j], sz = opts[2][k];
              if (!inside_root(sx, sy, sz)) continue;
              const int64_t f = t.find_leaf(sx, sy, sz);
              if (t.leaves[f].level > X.level + 1) return true;
            }
      }
  return false;
}

// Ripple balance.  coarse_seeds: cells that just gained children; their 26
// same-level neighbours must not lie inside a coarser leaf.  fine_seeds: leaves
// that must not touch anything more than one level finer.
static void balance_loop(Octree& t, std::vector<Octant> coarse_seeds, std::vector<Octant> fine_seeds,
                         bool fine_check_children) {
  while (!coarse_seeds.empty() || !fine_seeds.empty()) {
    std::vector<uint8_t> marks(t.size(), 0);
    int64_t nmark = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : nmark)
    for (int64_t s = 0; s < (int64_t)coarse_seeds.size(); ++s) {
      const Octant P = coarse_seeds[s];
      const int32_t sz = P.size();
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            if (!dx && !dy && !dz) continue;
            const int32_t nx = P.x + dx * sz, ny = P.y + dy * sz, nz = P.z + dz * sz;
            if (!inside_root(nx, ny, nz)) continue;
            const int64_t j = t.find_leaf(nx, ny, nz);
            if (t.leaves[j].level < P.level) {
              if (!__atomic_exchange_n(&marks[j], uint8_t(1), __ATOMIC_RELAXED)) ++nmark;
            }
          }
    }
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : nmark)
    for (int64_t s = 0; s < (int64_t)fine_seeds.size(); ++s) {
      const Octant X = fine_seeds[s];
      const int64_t j = t.find_leaf(X.x, X.y, X.z);
      const Octant& L = t.leaves[j];
      if (L.level != X.level || L.x != X.x || L.y != X.y || L.z != X.z) continue;  // no longer a leaf
      if (touches_too_fine(t, X)) {
        if (!__atomic_exchange_n(&marks[j], uint8_t(1), __ATOMIC_RELAXED)) ++nmark;
      }
    }
    if (nmark == 0) break;
    std::vector<Octant> parents = t.split_marked(marks);
    coarse_seeds = parents;
    fine_seeds.clear();
    if (fine_check_children) {
      fine_seeds.reserve(parents.size() * 8);
      for (const Octant& P : parents) {
        const int32_t h = P.size() >> 1;
        for (int c = 0; c < 8; ++c)
          fine_seeds.push_back(Octant{P.x + (c & 1) * h, P.y + ((c >> 1) & 1) * h,
                                      P.z + ((c >> 2) & 1) * h, P.level + 1});
      }
    }
  }
}

void Octree::balance_from(std::vector<Octant> parents) {
  balance_loop(*this, std::move(parents), {}, false);
}

void Octree::refine(const std::vector<uint8_t>& marks) {
  if ((int64_t)marks.size() != size()) throw std::runtime_error("refine: marks size");
  std::vector<uint8_t> m(marks);
  for (int64_t i = 0; i < size(); ++i)
    if (leaves[i].level >= kQMaxLevel) m[i] = 0;
  balance_from(split_marked(m));
}

void Octree::coarsen(const std::vector<uint8_t>& marks) {
  if ((int64_t)marks.size() != size()) throw std::runtime_error("coarsen: marks size");
  const int64_t n = size();
  std::vector<Octant> out;
  out.reserve(n);
  std::vector<Octant> merged;
  int64_t i = 0;
  while (i < n) {
    const Octant q = leaves[i];
    if (q.level > 0 && child_id(q) == 0 && i + 7 < n) {
      const int32_t h = q.size();
      bool fam = true;
      for (int c = 0; c < 8 && fam; ++c) {
        const Octant& o = leaves[i + c];
        fam = marks[i + c] && o.level == q.level && o.x == q.x + (c & 1) * h &&
              o.y == q.y + ((c >> 1) & 1) * h && o.z == q.z + ((c >> 2) & 1) * h;
      }
      if (fam) {
        const Octant P{q.x, q.y, q.z, q.level - 1};
        out.push_back(P);
        merged.push_back(P);
        i += 8;
        continue;
      }
    }
    out.push_back(q);
    ++i;
  }
  leaves.swap(out);
  rebuild_keys();
  balance_loop(*this, {}, std::move(merged), true);
}

// Hanging corners.  For leaf q (level L, child id k of parent P) corner c lies
// at a parent-edge midpoint when c^k has one bit set, at a parent-face centre
// when it has two.  It hangs when a level-(L-1) cell sharing that edge (resp.
// face) with P is a leaf.
std::vector<uint8_t> Octree::hanging_masks() const {
  const int64_t n = size();
  std::vector<uint8_t> mask(n, 0);
#pragma omp parallel
  {
    // memo of the 27 neighbour-is-leaf flags for the last parent seen
    Octant lastP{-1, -1, -1, -1};
    int8_t nb[27];
#pragma omp for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      const Octant q = leaves[i];
      if (q.level == 0) continue;
      const int L = q.level;
      const int32_t PS = 1 << (kMaxLevel - L + 1);
      const Octant P{q.x & ~(PS - 1), q.y & ~(PS - 1), q.z & ~(PS - 1), L - 1};
      if (P.x != lastP.x || P.y != lastP.y || P.z != lastP.z || P.level != lastP.level) {
        lastP = P;
        for (int t = 0; t < 27; ++t) nb[t] = -1;
      }
      auto nbr = [&](int dx, int dy, int dz) -> bool {
        const int t = (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1);
        if (nb[t] < 0) nb[t] = is_leaf_at(P.x + dx * PS, P.y + dy * PS, P.z + dz * PS, L - 1) ? 1 : 0;
        return nb[t] == 1;
      };
      const int k = child_id(q);
      uint8_t m8 = 0;
      for (int c = 0; c < 8; ++c) {
        const int m = c ^ k;
        const int pc = __builtin_popcount(m);
        if (pc == 0 || pc == 3) continue;
        // side of P on each axis where the corner sits on P's boundary plane
        int side[3];
        for (int a = 0; a < 3; ++a) side[a] = (((k >> a) & 1) + ((c >> a) & 1)) == 0 ? -1 : 1;
        bool hang = false;
        if (pc == 1) {
          const int a = __builtin_ctz(m);  // edge axis
          const int b = (a + 1) % 3, cc = (a + 2) % 3;
          int d1[3] = {0, 0, 0}, d2[3] = {0, 0, 0}, d3[3] = {0, 0, 0};
          d1[b] = side[b];
          d2[cc] = side[cc];
          d3[b] = side[b];
          d3[cc] = side[cc];
          hang = nbr(d1[0], d1[1], d1[2]) || nbr(d2[0], d2[1], d2[2]) || nbr(d3[0], d3[1], d3[2]);
        } else {
          const int nrm = __builtin_ctz(~m & 7);  // face normal axis
          int d[3] = {0, 0, 0};
          d[nrm] = side[nrm];
          hang = nbr(d[0], d[1], d[2]);
        }
        if (hang) m8 |= uint8_t(1u << c);
      }
      mask[i] = m8;
    }
  }
  return mask;
}

static inline void corner_xyz(const Octant& q, int c, int32_t out[3]) {
  const int32_t s = q.size();
  out[0] = q.x + (c & 1) * s;
  out[1] = q.y + ((c >> 1) & 1) * s;
  out[2] = q.z + ((c >> 2) & 1) * s;
}

static inline void decode_morton(uint64_t k, int32_t out[3]) {
  uint32_t v[3] = {0, 0, 0};
  for (int b = 0; b < 21; ++b)
    for (int a = 0; a < 3; ++a) v[a] |= uint32_t((k >> (3 * b + a)) & 1) << b;
  out[0] = int32_t(v[0]);
  out[1] = int32_t(v[1]);
  out[2] = int32_t(v[2]);
}

NodeTable Octree::build_nodes() const {
  const int64_t n = size();
  const std::vector<uint8_t> mask = hanging_masks();
  NodeTable T;

  // Independent nodes: each is emitted once, by the leaf that contains it under
  // the half-open rule (the point clamped into the root on upper faces).
  std::vector<int64_t> cnt(n + 1, 0);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    int c0 = 0;
    for (int c = 0; c < 8; ++c) {
      if (mask[i] >> c & 1) continue;
      int32_t p[3];
      corner_xyz(leaves[i], c, p);
      bool own = true;
      for (int a = 0; a < 3; ++a)
        if (((c >> a) & 1) && p[a] != kRootLen) own = false;
      c0 += own;
    }
    cnt[i + 1] = c0;
  }
  for (int64_t i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
  std::vector<uint64_t> codes(cnt[n]);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    int64_t w = cnt[i];
    for (int c = 0; c < 8; ++c) {
      if (mask[i] >> c & 1) continue;
      int32_t p[3];
      corner_xyz(leaves[i], c, p);
      bool own = true;
      for (int a = 0; a < 3; ++a)
        if (((c >> a) & 1) && p[a] != kRootLen) own = false;
      if (own) codes[w++] = morton3(p[0], p[1], p[2]);
    }
  }
  __gnu_parallel::sort(codes.begin(), codes.end());
  if (std::adjacent_find(codes.begin(), codes.end()) != codes.end())
    throw std::runtime_error("build_nodes: an independent node was emitted twice");
  T.n_indep = (int64_t)codes.size();
  T.indep_xyz.resize(3 * T.n_indep);
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < T.n_indep; ++j) decode_morton(codes[j], &T.indep_xyz[3 * j]);

  // Hanging nodes.
  std::vector<uint64_t> hcodes;
  for (int64_t i = 0; i < n; ++i) {
    if (!mask[i]) continue;
    for (int c = 0; c < 8; ++c)
      if (mask[i] >> c & 1) {
        int32_t p[3];
        corner_xyz(leaves[i], c, p);
        hcodes.push_back(morton3(p[0], p[1], p[2]));
      }
  }
  std::sort(hcodes.begin(), hcodes.end());
  hcodes.erase(std::unique(hcodes.begin(), hcodes.end()), hcodes.end());
  T.n_hang = (int64_t)hcodes.size();
  T.hang_xyz.resize(3 * T.n_hang);
  T.hang_np.assign(T.n_hang, 0);
  T.hang_par.assign(4 * T.n_hang, -1);

  auto indep_index = [&](const int32_t p[3]) -> int64_t {
    const uint64_t k = morton3(p[0], p[1], p[2]);
    auto it = std::lower_bound(codes.begin(), codes.end(), k);
    if (it == codes.end() || *it != k) return -1;
    return int64_t(it - codes.begin());
  };

  T.oct_nodes.resize(8 * n);
  std::vector<uint8_t> hang_done(T.n_hang, 0);
  bool bad_parent = false;
#pragma omp parallel for schedule(static) reduction(|| : bad_parent)
  for (int64_t i = 0; i < n; ++i) {
    const Octant q = leaves[i];
    const int k = (q.level > 0) ? child_id(q) : 0;
    for (int c = 0; c < 8; ++c) {
      int32_t p[3];
      corner_xyz(q, c, p);
      if (!(mask[i] >> c & 1)) {
        const int64_t j = indep_index(p);
        if (j < 0) bad_parent = true;
        T.oct_nodes[8 * i + c] = int32_t(j);
        continue;
      }
      const uint64_t hk = morton3(p[0], p[1], p[2]);
      const int64_t h = int64_t(std::lower_bound(hcodes.begin(), hcodes.end(), hk) - hcodes.begin());
      T.oct_nodes[8 * i + c] = int32_t(T.n_indep + h);
      if (__atomic_exchange_n(&hang_done[h], uint8_t(1), __ATOMIC_RELAXED)) continue;
      // parents: corners of the parent's edge (1 differing bit) or face (2 bits)
      const int32_t PS = 1 << (kMaxLevel - q.level + 1);
      const int32_t P[3] = {q.x & ~(PS - 1), q.y & ~(PS - 1), q.z & ~(PS - 1)};
      const int m = c ^ k;
      int32_t par[4];
      int np = 0;
      for (int pc = 0; pc < 8; ++pc) {
        // parent corner pc lies on the edge/face containing the point when it
        // agrees with the point on every axis where the point is on P's boundary
        bool on = true;
        for (int a = 0; a < 3; ++a) {
          if ((m >> a) & 1) continue;  // point at mid-plane on this axis
          const int want = (((k >> a) & 1) + ((c >> a) & 1)) / 2;  // 0 lower, 1 upper
          if (((pc >> a) & 1) != want) on = false;
        }
        if (!on) continue;
        const int32_t pp[3] = {P[0] + (pc & 1) * PS, P[1] + ((pc >> 1) & 1) * PS,
                               P[2] + ((pc >> 2) & 1) * PS};
        const int64_t j = indep_index(pp);
        if (j < 0) bad_parent = true;
        par[np++] = int32_t(j);
      }
      std::sort(par, par + np);
      T.hang_np[h] = int8_t(np);
      for (int t = 0; t < np; ++t) T.hang_par[4 * h + t] = par[t];
      T.hang_xyz[3 * h + 0] = p[0];
      T.hang_xyz[3 * h + 1] = p[1];
      T.hang_xyz[3 * h + 2] = p[2];
    }
  }
  if (bad_parent) throw std::runtime_error("build_nodes: a corner or hanging parent is not an independent node");
  return T;
}

bool Octree::check_complete() const {
  // volumes add up and Morton order is strict
  long double vol = 0;
  for (int64_t i = 0; i < size(); ++i) {
    const long double s = leaves[i].size();
    vol += s * s * s;
    if (i && keys[i] <= keys[i - 1]) return false;
  }
  const long double r = kRootLen;
  return vol == r * r * r;
}

bool Octree::check_balanced() const {
  for (int64_t i = 0; i < size(); ++i) {
    const Octant q = leaves[i];
    const int32_t s = q.size();
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          if (!dx && !dy && !dz) continue;
          const int32_t nx = q.x + dx * s, ny = q.y + dy * s, nz = q.z + dz * s;
          if (!inside_root(nx, ny, nz)) continue;
          if (leaves[find_leaf(nx, ny, nz)].level < q.level - 1) return false;
        }
  }
  return true;
}

}  // namespace pbh
