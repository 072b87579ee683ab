// VTK output of the lattice fields, in the files the reference's writer
// (src/solver/io/vtk_writer/) produces: one XML StructuredGrid `.vts` per
// block with Float64 cell data (structured_grid_writer.cpp), a
// vtkMultiBlockDataSet `.vtm` index per timestep and a Collection `.pvd`
// series (parallel_vtk_index.cpp), named as AmrVtkWriter names them
// (amr_vtk_writer.cpp).  Host code: octlb_gpu_write_vtk takes the fields from
// the device through octlb_gpu_get_fields.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iterator>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/octlb_gpu.h"

namespace {

// Base64 (RFC 4648 alphabet, '=' padding) of n bytes.
std::string base64(const unsigned char* p, size_t n) {
  static const char kAlphabet[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
  std::string s;
  s.reserve((n + 2) / 3 * 4);
  for (size_t i = 0; i < n; i += 3) {
    const uint32_t rem = static_cast<uint32_t>(n - i);
    const uint32_t w = (static_cast<uint32_t>(p[i]) << 16) | (rem > 1 ? static_cast<uint32_t>(p[i + 1]) << 8 : 0u) |
                       (rem > 2 ? static_cast<uint32_t>(p[i + 2]) : 0u);
    s += kAlphabet[(w >> 18) & 63];
    s += kAlphabet[(w >> 12) & 63];
    s += rem > 1 ? kAlphabet[(w >> 6) & 63] : '=';
    s += rem > 2 ? kAlphabet[w & 63] : '=';
  }
  return s;
}

// Payload of a binary DataArray (header_type UInt32): base64 of the byte
// count as a little-endian uint32 followed by the little-endian Float64 values.
void put_float64(std::ostream& out, const double* v, size_t count) {
  const uint32_t bytes = static_cast<uint32_t>(count * sizeof(double));
  std::vector<unsigned char> raw(sizeof(bytes) + count * sizeof(double));
  std::memcpy(raw.data(), &bytes, sizeof(bytes));
  if (count) std::memcpy(raw.data() + sizeof(bytes), v, count * sizeof(double));
  out << base64(raw.data(), raw.size());
}

std::string step_tag(int step) {
  char b[16];
  std::snprintf(b, sizeof(b), "%05d", step);
  return b;
}

// Point coordinate i of n along [lo, hi] (the reference's vertex placement).
double along(double lo, double hi, int i, int n) { return lo + (hi - lo) * static_cast<double>(i) / n; }

}  // namespace

extern "C" int octlb_vtk_write_block(const char* path, int nx, int ny, int nz, const double bounds[6], int nfields,
                                     const char* const* names, const int* comps, const double* const* data) {
  if (!path || !bounds || nx <= 0 || ny <= 0 || nz <= 0 || nfields < 0 || (nfields > 0 && (!names || !comps || !data)))
    return OCTLB_EINVAL;
  for (int f = 0; f < nfields; ++f)
    if (!names[f] || !data[f] || comps[f] < 1 || comps[f] > 3) return OCTLB_EINVAL;
  const long long cells = static_cast<long long>(nx) * ny * nz;
  const long long points = static_cast<long long>(nx + 1) * (ny + 1) * (nz + 1);
  std::ofstream out(path, std::ios::trunc);
  if (!out) return OCTLB_EINVAL;
  out << "<?xml version=\"1.0\"?>\n"
      << "<VTKFile type=\"StructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\" header_type=\"UInt32\">\n"
      << "  <StructuredGrid WholeExtent=\"0 " << nx << " 0 " << ny << " 0 " << nz << "\">\n"
      << "    <Piece Extent=\"0 " << nx << " 0 " << ny << " 0 " << nz << "\" NumberOfPoints=\"" << points
      << "\" NumberOfCells=\"" << cells << "\">\n"
      << "      <PointData>\n"
      << "      </PointData>\n"
      << "      <CellData>\n";
  for (int f = 0; f < nfields; ++f) {
    out << "        <DataArray type=\"Float64\" Name=\"" << names[f] << "\" NumberOfComponents=\"" << comps[f]
        << "\" format=\"binary\" encoding=\"base64\">\n          ";
    put_float64(out, data[f], static_cast<size_t>(cells * comps[f]));
    out << "\n        </DataArray>\n";
  }
  std::vector<double> xyz(static_cast<size_t>(points) * 3);
  size_t k3 = 0;
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i) {
        xyz[k3++] = along(bounds[0], bounds[3], i, nx);
        xyz[k3++] = along(bounds[1], bounds[4], j, ny);
        xyz[k3++] = along(bounds[2], bounds[5], k, nz);
      }
  out << "      </CellData>\n"
      << "      <Points>\n"
      << "        <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"binary\" encoding=\"base64\">\n"
      << "          ";
  put_float64(out, xyz.data(), xyz.size());
  out << "\n        </DataArray>\n"
      << "      </Points>\n"
      << "    </Piece>\n"
      << "  </StructuredGrid>\n"
      << "</VTKFile>\n";
  return out.good() ? OCTLB_OK : OCTLB_EINVAL;
}

extern "C" int octlb_vtk_write_index(const char* output_dir, const char* base_name, int step, int n_files,
                                     const char* const* vts_relative_paths) {
  if (!output_dir || !base_name || n_files < 0 || (n_files > 0 && !vts_relative_paths)) return OCTLB_EINVAL;
  const std::string dir(output_dir), base(base_name), tag = step_tag(step);
  std::error_code ec;
  std::filesystem::create_directories(dir, ec);
  {
    std::ofstream vtm(dir + "/" + base + "_T" + tag + ".vtm", std::ios::trunc);
    if (!vtm) return OCTLB_EINVAL;
    vtm << "<?xml version=\"1.0\"?>\n"
        << "<VTKFile type=\"vtkMultiBlockDataSet\" version=\"1.0\" byte_order=\"LittleEndian\">\n"
        << "<vtkMultiBlockDataSet>\n";
    for (int i = 0; i < n_files; ++i) {
      if (!vts_relative_paths[i]) return OCTLB_EINVAL;
      vtm << "<Block index=\"" << i << "\">\n"
          << "<DataSet index=\"0\" file=\"" << vts_relative_paths[i] << "\"/>\n"
          << "</Block>\n";
    }
    vtm << "</vtkMultiBlockDataSet>\n"
        << "</VTKFile>\n";
    if (!vtm.good()) return OCTLB_EINVAL;
  }
  // The series: header and empty collection on first use, then each
  // timestep's entry goes in before the closing tags.
  const std::string pvd = dir + "/" + base + ".pvd";
  const std::string tail = "</Collection>\n</VTKFile>\n";
  std::string text;
  {
    std::ifstream in(pvd, std::ios::binary);
    if (in) text.assign(std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>());
  }
  if (text.empty())
    text = "<?xml version=\"1.0\"?>\n<VTKFile type=\"Collection\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
           "<Collection>\n" + tail;
  if (text.size() < tail.size() || text.compare(text.size() - tail.size(), tail.size(), tail) != 0)
    return OCTLB_EINVAL;  // not a series this writer made
  text.resize(text.size() - tail.size());
  std::ostringstream entry;
  entry << "<DataSet timestep=\"" << step << "\" group=\"\" part=\"0\" file=\"" << base << "_T" << tag
        << ".vtm\"/>\n";
  text += entry.str() + tail;
  std::ofstream out(pvd, std::ios::binary | std::ios::trunc);
  if (!out) return OCTLB_EINVAL;
  out << text;
  return out.good() ? OCTLB_OK : OCTLB_EINVAL;
}
