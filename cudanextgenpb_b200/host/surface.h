// Surface input for the PB path: the molecular surface seen through axis-aligned
// rays, in the form NanoShaper hands to the reference (crossings_t: sorted
// intersections along the ray plus an outward unit normal at each,
// src/raytracer.cpp:379-467, include/raytracer.h:37-85).
//
// NanoShaper is not available to this build, so the surface is produced here by
// an exact analytic ray caster over a union of spheres:
//   * probe = 0: van der Waals surface (equal to the SES of a single sphere),
//   * probe > 0: solvent-accessible surface (radii inflated by the probe).
// A ray is identified by the integer octree coordinates (a, b) of its two
// transverse axes in ascending axis order (axis 0: (y, z); axis 1: (x, z);
// axis 2: (x, y)), the same pairing the reference uses for its ray keys
// (src/pb_class.cpp:1856-1880).
#pragma once
#include <array>
#include <cstdint>
#include <unordered_map>
#include <vector>

namespace pbh {

struct Atom {
  double pos[3];
  double charge;
  double radius;
};

// Affine map from integer octree coordinates to physical coordinates, one
// rounding in the product and one in the sum (no fused multiply-add).  Every
// component of this build evaluates node coordinates with exactly this formula
// so that the ray keys, the in/out parity tests and the edge fractions agree bit
// for bit.
struct Domain {
  double lo[3], hi[3], len[3];
  void set(const double l[3], const double h[3]);
  double coord(int axis, int32_t i) const;
};

class SphereUnion {
 public:
  void build(const std::vector<Atom>& atoms, double inflate);
  // Cast the axis-aligned ray at transverse physical coordinates (u, v).
  void cast(int axis, double u, double v, std::vector<double>& inters, std::vector<double>& normals) const;
  int64_t n_spheres() const { return (int64_t)cx_.size(); }

 private:
  std::vector<double> cx_, cy_, cz_, r_;
  double cell_ = 1.0;
  // per axis: 2D bins over the transverse plane
  struct Bins {
    double o0 = 0, o1 = 0;
    int n0 = 1, n1 = 1;
    std::vector<int32_t> start, items;
  } bins_[3];
};

// All rays of one axis with at least one crossing, sorted by key.
struct RayTable {
  std::vector<uint64_t> keys;
  std::vector<int64_t> ptr{0};
  std::vector<double> inters;
  std::vector<double> normals;
  int64_t n() const { return (int64_t)keys.size(); }
};

inline uint64_t ray_key(int32_t a, int32_t b) { return (uint64_t(uint32_t(a)) << 20) | uint64_t(uint32_t(b)); }

// Host cache of cast rays.  ensure() casts every missing ray (in parallel);
// lookups afterwards are read-only and thread-safe.  Rays are kept in a flat
// open-addressing table (linear probing, load <= 1/2).
class RayCache {
 public:
  const SphereUnion* surf = nullptr;
  const Domain* dom = nullptr;
  void ensure(int axis, std::vector<uint64_t> keys);
  // Parity of the crossings at or below x (the reference's is_in_ns_surf,
  // src/pb_class.cpp:769-805): 1 inside, 0 outside.
  int parity(int axis, uint64_t key, double x) const;
  // Crossings of a cast ray (nullptr when the ray has not been cast).
  const double* crossings(int axis, uint64_t key, int32_t* n) const;
  bool parity_known(int axis, uint64_t key) const { return find(axis, key) >= 0; }
  RayTable table(int axis, const std::vector<uint64_t>& keys) const;
  void clear();

 private:
  struct Table {
    std::vector<uint64_t> key;  // ~0 = empty
    std::vector<int64_t> off;
    std::vector<int32_t> n;
    uint64_t mask = 0;
    int64_t size = 0;
  } tab_[3];
  std::vector<double> inters_[3], normals_[3];
  int64_t find(int axis, uint64_t key) const;
  void insert(int axis, uint64_t key, int64_t off, int32_t n);
  void grow(int axis, int64_t need);
};

}  // namespace pbh
