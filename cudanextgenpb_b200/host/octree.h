// Linear octree over one tree (the unit cube mapped onto the domain box), with
// 2:1 balance across faces, edges and corners and p8est-style node tables:
// independent nodes and hanging nodes (edge-hanging with 2 parents, face-hanging
// with 4 parents).
//
// This is the mesh the reference obtains from bimpp's tmesh_3d over p4est 2.8.6
// (refine/coarsen with P8EST_CONNECT_FULL balance).  Conventions kept from p4est:
//  * integer coordinates in units of 2^-19 of the root (P8EST_MAXLEVEL = 19),
//  * Morton order of octants with x in the lowest bit (child id = x | y<<1 | z<<2),
//  * corner c of an octant sits at lower + ((c>>0)&1, (c>>1)&1, (c>>2)&1) * size,
//  * independent nodes numbered in Morton order of their coordinates (the order
//    in which p8est_nodes_new sorts its indep_nodes).
// Reference call sites: src/pb_class.cpp:1290-1391 (init refinement) and
// :1468-1745 (surface refine/coarsen), quadrant accessors is_hanging / gt /
// num_parents / gparent used throughout src/pb_class.cpp.
#pragma once
#include <array>
#include <cstdint>
#include <functional>
#include <vector>

namespace pbh {

constexpr int kMaxLevel = 19;                 // P8EST_MAXLEVEL
constexpr int kQMaxLevel = 18;                // P8EST_QMAXLEVEL
constexpr int32_t kRootLen = 1 << kMaxLevel;  // P8EST_ROOT_LEN

struct Octant {
  int32_t x, y, z;
  int32_t level;
  int32_t size() const { return 1 << (kMaxLevel - level); }
};

uint64_t morton3(uint32_t x, uint32_t y, uint32_t z);

// Nodes of a balanced octree.  oct_nodes[8*q + c] < n_indep names an
// independent node; otherwise n_indep + h names hanging node h.
struct NodeTable {
  int64_t n_indep = 0;
  std::vector<int32_t> indep_xyz;   // 3 * n_indep, integer coordinates
  int64_t n_hang = 0;
  std::vector<int32_t> hang_xyz;    // 3 * n_hang
  std::vector<int8_t> hang_np;      // 2 (edge) or 4 (face)
  std::vector<int32_t> hang_par;    // 4 * n_hang, ascending, -1 padded
  std::vector<int32_t> oct_nodes;   // 8 * n_oct
};

class Octree {
 public:
  std::vector<Octant> leaves;   // Morton order
  std::vector<uint64_t> keys;   // Morton key of each leaf's lower corner

  void uniform(int level);
  int64_t size() const { return (int64_t)leaves.size(); }

  // Leaf whose half-open box contains the integer point (0 <= p < kRootLen).
  int64_t find_leaf(int32_t x, int32_t y, int32_t z) const;

  // Split every marked leaf once, then restore 2:1 balance.
  void refine(const std::vector<uint8_t>& marks);
  // Merge every complete family of 8 sibling leaves that are all marked, then
  // restore 2:1 balance (balance only ever refines).
  void coarsen(const std::vector<uint8_t>& marks);

  // Per-leaf 8-bit mask of hanging corners (bit c set: corner c hangs).
  std::vector<uint8_t> hanging_masks() const;

  NodeTable build_nodes() const;

  // Checks used by the tests: complete cover, 2:1 balance.
  bool check_complete() const;
  bool check_balanced() const;

  // Refine the marked leaves once, without balancing; returns the refined
  // leaves (now parents of 8 children each).
  std::vector<Octant> split_marked(const std::vector<uint8_t>& marks);
  bool is_leaf_at(int32_t x, int32_t y, int32_t z, int level) const;

 private:
  void rebuild_keys();
  void balance_from(std::vector<Octant> parents);
};

}  // namespace pbh
