// Analytic ray caster over a union of spheres and the host ray cache.
#include "surface.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <parallel/algorithm>
#include <stdexcept>

#include "octree.h"

namespace pbh {

void Domain::set(const double l[3], const double h[3]) {
  for (int a = 0; a < 3; ++a) {
    lo[a] = l[a];
    hi[a] = h[a];
    len[a] = h[a] - l[a];
  }
}

double Domain::coord(int axis, int32_t i) const {
  const double t = double(i) * 0x1p-19;  // exact
  const double p = len[axis] * t;
  return lo[axis] + p;
}

static inline void transverse(int axis, int& t0, int& t1) {
  t0 = axis == 0 ? 1 : 0;
  t1 = axis == 2 ? 1 : 2;
}

void SphereUnion::build(const std::vector<Atom>& atoms, double inflate) {
  cx_.clear();
  cy_.clear();
  cz_.clear();
  r_.clear();
  double rmax = 0;
  for (const Atom& a : atoms) {
    const double r = a.radius + inflate;
    if (!(r > 0)) continue;
    cx_.push_back(a.pos[0]);
    cy_.push_back(a.pos[1]);
    cz_.push_back(a.pos[2]);
    r_.push_back(r);
    rmax = std::max(rmax, r);
  }
  cell_ = rmax > 0 ? 2.0 * rmax : 1.0;
  const int64_t n = n_spheres();
  const std::vector<double>* c[3] = {&cx_, &cy_, &cz_};
  for (int axis = 0; axis < 3; ++axis) {
    int t0, t1;
    transverse(axis, t0, t1);
    Bins& B = bins_[axis];
    if (n == 0) {
      B.n0 = B.n1 = 1;
      B.start.assign(2, 0);
      B.items.clear();
      continue;
    }
    double mn0 = 1e300, mx0 = -1e300, mn1 = 1e300, mx1 = -1e300;
    for (int64_t i = 0; i < n; ++i) {
      mn0 = std::min(mn0, (*c[t0])[i] - r_[i]);
      mx0 = std::max(mx0, (*c[t0])[i] + r_[i]);
      mn1 = std::min(mn1, (*c[t1])[i] - r_[i]);
      mx1 = std::max(mx1, (*c[t1])[i] + r_[i]);
    }
    B.o0 = mn0;
    B.o1 = mn1;
    B.n0 = std::max(1, int((mx0 - mn0) / cell_) + 1);
    B.n1 = std::max(1, int((mx1 - mn1) / cell_) + 1);
    std::vector<int32_t> cnt(size_t(B.n0) * B.n1 + 1, 0);
    auto range = [&](int64_t i, int& a0, int& a1, int& b0, int& b1) {
      a0 = std::max(0, int(((*c[t0])[i] - r_[i] - B.o0) / cell_));
      a1 = std::min(B.n0 - 1, int(((*c[t0])[i] + r_[i] - B.o0) / cell_));
      b0 = std::max(0, int(((*c[t1])[i] - r_[i] - B.o1) / cell_));
      b1 = std::min(B.n1 - 1, int(((*c[t1])[i] + r_[i] - B.o1) / cell_));
    };
    for (int64_t i = 0; i < n; ++i) {
      int a0, a1, b0, b1;
      range(i, a0, a1, b0, b1);
      for (int p = a0; p <= a1; ++p)
        for (int q = b0; q <= b1; ++q) cnt[size_t(p) * B.n1 + q + 1]++;
    }
    for (size_t k = 1; k < cnt.size(); ++k) cnt[k] += cnt[k - 1];
    B.start = cnt;
    B.items.assign(cnt.back(), 0);
    std::vector<int32_t> fill(cnt.begin(), cnt.end() - 1);
    for (int64_t i = 0; i < n; ++i) {
      int a0, a1, b0, b1;
      range(i, a0, a1, b0, b1);
      for (int p = a0; p <= a1; ++p)
        for (int q = b0; q <= b1; ++q) B.items[fill[size_t(p) * B.n1 + q]++] = int32_t(i);
    }
  }
}

void SphereUnion::cast(int axis, double u, double v, std::vector<double>& inters,
                       std::vector<double>& normals) const {
  inters.clear();
  normals.clear();
  if (n_spheres() == 0) return;
  int t0, t1;
  transverse(axis, t0, t1);
  const Bins& B = bins_[axis];
  const double f0 = (u - B.o0) / cell_, f1 = (v - B.o1) / cell_;
  if (f0 < 0 || f1 < 0) return;
  const int p = int(f0), q = int(f1);
  if (p >= B.n0 || q >= B.n1) return;
  const size_t bin = size_t(p) * B.n1 + q;
  const std::vector<double>* c[3] = {&cx_, &cy_, &cz_};
  struct Iv {
    double lo, hi;
    int32_t slo, shi;
  };
  Iv buf[64];
  std::vector<Iv> big;
  Iv* iv = buf;
  int niv = 0;
  for (int32_t k = B.start[bin]; k < B.start[bin + 1]; ++k) {
    const int32_t i = B.items[k];
    const double d0 = u - (*c[t0])[i], d1 = v - (*c[t1])[i];
    const double s2 = r_[i] * r_[i] - (d0 * d0 + d1 * d1);
    if (!(s2 > 0)) continue;
    const double s = std::sqrt(s2);
    const double ca = (*c[axis])[i];
    const Iv e{ca - s, ca + s, i, i};
    if (iv == buf && niv == 64) {
      big.assign(buf, buf + 64);
      iv = nullptr;
    }
    if (iv == buf)
      buf[niv++] = e;
    else {
      big.push_back(e);
      ++niv;
    }
  }
  if (!niv) return;
  Iv* a = (iv == buf) ? buf : big.data();
  std::sort(a, a + niv, [](const Iv& x, const Iv& y) { return x.lo < y.lo || (x.lo == y.lo && x.hi < y.hi); });
  auto emit = [&](double x, int32_t s) {
    double pnt[3];
    pnt[axis] = x;
    pnt[t0] = u;
    pnt[t1] = v;
    inters.push_back(x);
    normals.push_back((pnt[0] - cx_[s]) / r_[s]);
    normals.push_back((pnt[1] - cy_[s]) / r_[s]);
    normals.push_back((pnt[2] - cz_[s]) / r_[s]);
  };
  Iv cur = a[0];
  for (int k = 1; k < niv; ++k) {
    if (a[k].lo <= cur.hi) {
      if (a[k].hi > cur.hi) {
        cur.hi = a[k].hi;
        cur.shi = a[k].shi;
      }
    } else {
      emit(cur.lo, cur.slo);
      emit(cur.hi, cur.shi);
      cur = a[k];
    }
  }
  emit(cur.lo, cur.slo);
  emit(cur.hi, cur.shi);
}

static inline uint64_t mix(uint64_t k) { return k * 0x9E3779B97F4A7C15ull; }

void RayCache::clear() {
  for (int a = 0; a < 3; ++a) {
    tab_[a] = Table();
    inters_[a].clear();
    normals_[a].clear();
  }
}

int64_t RayCache::find(int axis, uint64_t key) const {
  const Table& T = tab_[axis];
  if (T.size == 0) return -1;
  uint64_t s = (mix(key) >> 20) & T.mask;
  while (true) {
    const uint64_t k = T.key[s];
    if (k == key) return (int64_t)s;
    if (k == ~0ull) return -1;
    s = (s + 1) & T.mask;
  }
}

void RayCache::insert(int axis, uint64_t key, int64_t off, int32_t n) {
  Table& T = tab_[axis];
  uint64_t s = (mix(key) >> 20) & T.mask;
  while (T.key[s] != ~0ull && T.key[s] != key) s = (s + 1) & T.mask;
  if (T.key[s] == ~0ull) ++T.size;
  T.key[s] = key;
  T.off[s] = off;
  T.n[s] = n;
}

void RayCache::grow(int axis, int64_t need) {
  Table& T = tab_[axis];
  if (2 * need <= (int64_t)T.key.size()) return;
  uint64_t cap = 1024;
  while ((int64_t)cap < 2 * need) cap <<= 1;
  Table old = std::move(T);
  T = Table();
  T.key.assign(cap, ~0ull);
  T.off.assign(cap, 0);
  T.n.assign(cap, 0);
  T.mask = cap - 1;
  for (size_t s = 0; s < old.key.size(); ++s)
    if (old.key[s] != ~0ull) insert(axis, old.key[s], old.off[s], old.n[s]);
}

const double* RayCache::crossings(int axis, uint64_t key, int32_t* n) const {
  const int64_t s = find(axis, key);
  if (s < 0) {
    *n = 0;
    return nullptr;
  }
  *n = tab_[axis].n[s];
  return inters_[axis].data() + tab_[axis].off[s];
}

void RayCache::ensure(int axis, std::vector<uint64_t> keys) {
  if (!surf || !dom) throw std::runtime_error("RayCache: surface/domain not set");
  __gnu_parallel::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  std::vector<uint64_t> miss;
  miss.reserve(keys.size());
  for (uint64_t k : keys)
    if (find(axis, k) < 0) miss.push_back(k);
  if (miss.empty()) return;
  int t0, t1;
  transverse(axis, t0, t1);
  const int64_t m = (int64_t)miss.size();
  std::vector<std::vector<double>> I(m), N(m);
#pragma omp parallel for schedule(dynamic, 512)
  for (int64_t j = 0; j < m; ++j) {
    const int32_t ia = int32_t(miss[j] >> 20), ib = int32_t(miss[j] & 0xfffff);
    surf->cast(axis, dom->coord(t0, ia), dom->coord(t1, ib), I[j], N[j]);
  }
  grow(axis, tab_[axis].size + m);
  for (int64_t j = 0; j < m; ++j) {
    insert(axis, miss[j], (int64_t)inters_[axis].size(), (int32_t)I[j].size());
    inters_[axis].insert(inters_[axis].end(), I[j].begin(), I[j].end());
    normals_[axis].insert(normals_[axis].end(), N[j].begin(), N[j].end());
  }
}

int RayCache::parity(int axis, uint64_t key, double x) const {
  int32_t n = 0;
  const double* I = crossings(axis, key, &n);
  if (!I) throw std::runtime_error("RayCache::parity: ray not cast");
  int i = 0;
  while (i < n && x >= I[i]) ++i;
  return i & 1;
}

RayTable RayCache::table(int axis, const std::vector<uint64_t>& keys_in) const {
  std::vector<uint64_t> keys(keys_in);
  __gnu_parallel::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  RayTable T;
  for (uint64_t k : keys) {
    const int64_t s = find(axis, k);
    if (s < 0) throw std::runtime_error("RayCache::table: ray not cast");
    const int32_t n = tab_[axis].n[s];
    if (n == 0) continue;
    T.keys.push_back(k);
    const int64_t o = tab_[axis].off[s];
    T.inters.insert(T.inters.end(), inters_[axis].begin() + o, inters_[axis].begin() + o + n);
    T.normals.insert(T.normals.end(), normals_[axis].begin() + 3 * o, normals_[axis].begin() + 3 * (o + n));
    T.ptr.push_back((int64_t)T.inters.size());
  }
  return T;
}

}  // namespace pbh
