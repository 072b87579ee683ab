// The reference's VTK writer (src/solver/io/vtk_writer/) as a program, built
// into oracle/_ref/ref_vtk.  TEST INFRASTRUCTURE ONLY: it writes the files the
// GPU library's writer is compared with byte for byte.  It runs in its own
// process: the library's C++ runtime then meets no other one.
//
//   ref_vtk block <out.vts> <in.bin>
//       WriteStructuredGridVts (structured_grid_writer.cpp).  in.bin, little
//       endian: int32 nx, ny, nz, nfields; float64 bounds[6] (x_min y_min
//       z_min x_max y_max z_max); per field int32 name length, the name,
//       int32 components, then float64 values in the file's cell order
//       (i fastest, then j, then k).
//   ref_vtk index <dir> <base> <step> <vts path>...
//       AmrVtkWriter::WriteVtmAndPvd on one rank (amr_vtk_writer.cpp): the
//       .vtm of the step listing the paths (relative to dir), and its entry
//       appended to dir/base.pvd.
//   ref_vtk decode <payload file>
//       vtk_binary::DecodeFloat64Array of a base64 payload, one value per
//       line (%.17g).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <span>
#include <stdexcept>
#include <string>
#include <vector>

#include "src/solver/io/vtk_writer/parallel_vtk_index.h"
#include "src/solver/io/vtk_writer/structured_grid_writer.h"
#include "src/solver/io/vtk_writer/vtk_binary_codec.h"

using namespace octlb;

namespace {

template <typename T>
T take(const std::string& buf, size_t& pos) {
  T v{};
  if (pos + sizeof(T) > buf.size()) throw std::runtime_error("short input");
  std::memcpy(&v, buf.data() + pos, sizeof(T));
  pos += sizeof(T);
  return v;
}

int block(const char* out, const char* in) {
  std::ifstream f(in, std::ios::binary);
  const std::string buf((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  size_t pos = 0;
  const int nx = take<int32_t>(buf, pos), ny = take<int32_t>(buf, pos), nz = take<int32_t>(buf, pos);
  const int nfields = take<int32_t>(buf, pos);
  double b[6];
  for (double& x : b) x = take<double>(buf, pos);
  VtkBlockMeta meta;
  meta.nx = nx;
  meta.ny = ny;
  meta.nz = nz;
  meta.bounds = BoundingBox{b[0], b[1], b[2], b[3], b[4], b[5]};
  std::vector<std::string> names(static_cast<size_t>(nfields));
  std::vector<std::vector<double>> values(static_cast<size_t>(nfields));
  std::vector<VtkCellFieldView> views;
  const long long cells = static_cast<long long>(nx) * ny * nz;
  for (int k = 0; k < nfields; ++k) {
    const int len = take<int32_t>(buf, pos);
    names[k].assign(buf.data() + pos, static_cast<size_t>(len));
    pos += static_cast<size_t>(len);
    const int c = take<int32_t>(buf, pos);
    values[k].resize(static_cast<size_t>(cells * c));
    for (double& x : values[k]) x = take<double>(buf, pos);
  }
  for (int k = 0; k < nfields; ++k) {
    const std::vector<double>* v = &values[k];
    const int c = static_cast<int>(v->size() / static_cast<size_t>(cells));
    views.push_back({names[k], c, [v, c, nx, ny](int i, int j, int kk, double* o) {
                       const long long cell = (static_cast<long long>(kk) * ny + j) * nx + i;
                       for (int q = 0; q < c; ++q) o[q] = (*v)[static_cast<size_t>(cell * c + q)];
                     }});
  }
  WriteStructuredGridVts(out, meta, std::span<const VtkCellFieldView>(views.data(), views.size()));
  return 0;
}

int write_index(int argc, char** argv) {
  const std::string dir = argv[2], base = argv[3];
  const int step = std::atoi(argv[4]);
  std::vector<std::string> rel(argv + 5, argv + argc);
  char tag[16];
  std::snprintf(tag, sizeof(tag), "%05d", step);
  WriteVtmIndex(MPI_COMM_WORLD, step, dir, base, rel);
  AppendPvdTimestep(step, dir + "/" + base + ".pvd", base + "_T" + tag + ".vtm");
  return 0;
}

int decode(const char* in) {
  std::ifstream f(in, std::ios::binary);
  const std::string payload((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  for (double v : vtk_binary::DecodeFloat64Array(payload)) std::printf("%.17g\n", v);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  try {
    const std::string cmd = argc > 1 ? argv[1] : "";
    if (cmd == "block" && argc == 4) return block(argv[2], argv[3]);
    if (cmd == "index" && argc >= 5) return write_index(argc, argv);
    if (cmd == "decode" && argc == 3) return decode(argv[2]);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ref_vtk: %s\n", e.what());
    return 1;
  }
  std::fprintf(stderr, "usage: ref_vtk block <out.vts> <in.bin> | index <dir> <base> <step> <vts>... | decode <file>\n");
  return 2;
}
