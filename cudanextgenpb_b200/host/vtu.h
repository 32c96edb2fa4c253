// VTU output of a node field on the octree: the reference's VTKWriter
// (src/vtk_class.cpp:20-429) as called by the driver for map_type = vtu
// (src/poisson_boltzmann.cpp:319-351).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace pbh {

// The mesh a field lives on: the arrays of pbgpu_mesh plus the box the
// integer coordinates map into (a corner at integer i sits at
// lo + extent * (i * 2^-19)).
struct VtuMesh {
  int64_t n_oct = 0;
  const int32_t* oct_xyz = nullptr;
  const int8_t* oct_level = nullptr;
  const int32_t* oct_nodes = nullptr;
  int64_t n_nodes = 0;
  const int32_t* node_xyz = nullptr;
  int64_t n_hang = 0;
  const int8_t* hang_np = nullptr;
  const int32_t* hang_par = nullptr;
  double lo[3] = {0, 0, 0}, extent[3] = {0, 0, 0};
};

// Writes <basename>_0000.vtu: an UnstructuredGrid of voxels (VTK type 11),
// one per octant, with the field as point data, every array appended raw
// with a 4-byte length in front (the reference's layout).  Points are the
// independent nodes in id order, then one point per octant corner that is a
// hanging node, carrying the mean of the node's parents.  Fails (returns
// false, message in *err) when the file cannot be written or an array
// exceeds the 4-byte length field.
bool write_vtu(const std::string& basename, const std::string& fieldname, const VtuMesh& m, const double* values,
               std::string* err);

// Writes total_<basename>.pvtu for each (field, base) pair, naming the
// pieces <basename>_0000.vtu .. of n_pieces ranks.
bool write_pvtu(const std::vector<std::string>& fieldnames, const std::vector<std::string>& basenames, int n_pieces,
                std::string* err);

}  // namespace pbh
