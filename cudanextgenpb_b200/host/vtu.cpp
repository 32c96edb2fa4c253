// VTU writer; see vtu.h.  The XML layout, the array names ("Array" for the
// points, "connectivity", "offsets", "types"), the 4-byte length before each
// appended array and the hanging-corner points follow the reference's
// VTKWriter (src/vtk_class.cpp:98-160 point set, :318-429 file layout) so
// that its readers and viewers load these files unchanged.
#include "vtu.h"

#include <climits>
#include <cstdio>
#include <cstring>

namespace pbh {

namespace {

constexpr double kUnit = 1.0 / 524288.0;  // 2^-19: integer coordinate -> fraction of the box

double coord(const VtuMesh& m, int a, int64_t i) { return m.lo[a] + m.extent[a] * (double(i) * kUnit); }

struct Block {
  const void* data;
  int64_t bytes;
};

bool put(FILE* f, const void* p, size_t n) { return std::fwrite(p, 1, n, f) == n; }

bool put_block(FILE* f, const Block& b) {
  const int32_t len = (int32_t)b.bytes;
  return put(f, &len, 4) && (b.bytes == 0 || put(f, b.data, (size_t)b.bytes));
}

}  // namespace

bool write_vtu(const std::string& basename, const std::string& fieldname, const VtuMesh& m, const double* values,
               std::string* err) {
  const std::string base = basename.empty() ? "default" : basename;
  const std::string field = fieldname.empty() ? "field" : fieldname;
  char path[4096];
  std::snprintf(path, sizeof(path), "%s_%4.4d.vtu", base.c_str(), 0);
  // points: independent nodes, then one per hanging corner occurrence
  const int64_t n = m.n_nodes;
  int64_t extra = 0;
  for (int64_t i = 0; i < 8 * m.n_oct; ++i) extra += m.oct_nodes[i] >= n;
  const int64_t npts = n + extra;
  std::vector<double> pts((size_t)(3 * npts));
  std::vector<double> val((size_t)npts);
  std::vector<int32_t> conn((size_t)(8 * m.n_oct));
  for (int64_t i = 0; i < n; ++i) {
    for (int a = 0; a < 3; ++a) pts[3 * i + a] = coord(m, a, m.node_xyz[3 * i + a]);
    val[i] = values[i];
  }
  int64_t next = n;
  for (int64_t o = 0; o < m.n_oct; ++o) {
    const int32_t s = 1 << (19 - m.oct_level[o]);
    for (int c = 0; c < 8; ++c) {
      const int32_t nd = m.oct_nodes[8 * o + c];
      if (nd < n) {
        conn[8 * o + c] = nd;
        continue;
      }
      const int64_t h = nd - n;
      for (int a = 0; a < 3; ++a) pts[3 * next + a] = coord(m, a, m.oct_xyz[3 * o + a] + ((c >> a) & 1) * s);
      const int np = m.hang_np[h];
      double sum = 0.0;
      for (int j = 0; j < np; ++j) sum += values[m.hang_par[4 * h + j]];
      val[next] = sum / np;
      conn[8 * o + c] = (int32_t)next;
      ++next;
    }
  }
  if (npts > INT_MAX) {
    if (err) *err = "write_vtu: more points than 32-bit connectivity can index";
    return false;
  }
  std::vector<int32_t> offsets((size_t)m.n_oct), types((size_t)m.n_oct, 11);
  for (int64_t i = 0; i < m.n_oct; ++i) offsets[i] = (int32_t)(8 * (i + 1));
  const Block blocks[5] = {{pts.data(), (int64_t)(pts.size() * sizeof(double))},
                           {conn.data(), (int64_t)(conn.size() * sizeof(int32_t))},
                           {offsets.data(), (int64_t)(offsets.size() * sizeof(int32_t))},
                           {types.data(), (int64_t)(types.size() * sizeof(int32_t))},
                           {val.data(), (int64_t)(val.size() * sizeof(double))}};
  int64_t off[5];
  int64_t acc = 0;
  for (int k = 0; k < 5; ++k) {
    if (blocks[k].bytes > INT32_MAX) {
      if (err) *err = "write_vtu: an array exceeds the 4-byte length of the appended-data layout";
      return false;
    }
    off[k] = acc;
    acc += 4 + blocks[k].bytes;
  }
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    if (err) *err = std::string("write_vtu: cannot open ") + path;
    return false;
  }
  std::string x;
  x += "<?xml version=\"1.0\"?>\n";
  x += "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
  x += "<UnstructuredGrid>\n";
  x += "<Piece NumberOfPoints=\"" + std::to_string(npts) + "\" NumberOfCells=\"" + std::to_string(m.n_oct) + "\">\n";
  x += "<Points>\n";
  x += "<DataArray type=\"Float64\" Name=\"Array\" NumberOfComponents=\"3\" format=\"appended\" offset=\"" +
       std::to_string(off[0]) + "\">\n</DataArray>\n";
  x += "</Points>\n<Cells>\n";
  x += "<DataArray type=\"Int32\" Name=\"connectivity\" format=\"appended\" offset=\"" + std::to_string(off[1]) +
       "\">\n</DataArray>\n";
  x += "<DataArray type=\"Int32\" Name=\"offsets\" format=\"appended\" offset=\"" + std::to_string(off[2]) +
       "\">\n</DataArray>\n";
  x += "<DataArray type=\"Int32\" Name=\"types\" format=\"appended\" offset=\"" + std::to_string(off[3]) +
       "\">\n</DataArray>\n";
  x += "</Cells>\n<PointData>\n";
  x += "<DataArray type=\"Float64\" Name=\"" + field + "\" NumberOfComponents=\"1\" format=\"appended\" offset=\"" +
       std::to_string(off[4]) + "\">\n</DataArray>\n";
  x += "</PointData>\n</Piece>\n</UnstructuredGrid>\n <AppendedData encoding=\"raw\">\n_";
  bool ok = put(f, x.data(), x.size());
  for (int k = 0; k < 5 && ok; ++k) ok = put_block(f, blocks[k]);
  const char* tail = " </AppendedData>\n</VTKFile>\n";
  ok = ok && put(f, tail, std::strlen(tail));
  ok = (std::fclose(f) == 0) && ok;
  if (!ok && err) *err = std::string("write_vtu: write failed on ") + path;
  return ok;
}

bool write_pvtu(const std::vector<std::string>& fieldnames, const std::vector<std::string>& basenames, int n_pieces,
                std::string* err) {
  if (fieldnames.size() != basenames.size()) {
    if (err) *err = "write_pvtu: one field name per base name";
    return false;
  }
  for (size_t i = 0; i < basenames.size(); ++i) {
    const std::string path = "total_" + basenames[i] + ".pvtu";
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) {
      if (err) *err = "write_pvtu: cannot open " + path;
      return false;
    }
    std::fprintf(f, "<?xml version=\"1.0\"?>\n");
    std::fprintf(f, "<VTKFile type=\"PUnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n");
    std::fprintf(f, "  <PUnstructuredGrid>\n");
    std::fprintf(f, "    <PPoints>\n");
    std::fprintf(f, "      <PDataArray type=\"Float64\" NumberOfComponents=\"3\" Name=\"Array\"/>\n");
    std::fprintf(f, "    </PPoints>\n");
    std::fprintf(f, "    <PCells>\n");
    std::fprintf(f, "      <PDataArray type=\"Int32\" Name=\"connectivity\"/>\n");
    std::fprintf(f, "      <PDataArray type=\"Int32\" Name=\"offsets\"/>\n");
    std::fprintf(f, "      <PDataArray type=\"Int32\" Name=\"types\"/>\n");
    std::fprintf(f, "    </PCells>\n");
    std::fprintf(f, "    <PPointData>\n");
    std::fprintf(f, "      <PDataArray type=\"Float64\" Name=\"%s\"/>\n", fieldnames[i].c_str());
    std::fprintf(f, "    </PPointData>\n");
    for (int r = 0; r < n_pieces; ++r)
      std::fprintf(f, "    <Piece Source=\"%s_%4.4d.vtu\"/>\n", basenames[i].c_str(), r);
    std::fprintf(f, "  </PUnstructuredGrid>\n");
    std::fprintf(f, "</VTKFile>\n");
    if (std::fclose(f) != 0) {
      if (err) *err = "write_pvtu: write failed on " + path;
      return false;
    }
  }
  return true;
}

}  // namespace pbh
