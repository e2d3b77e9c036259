// Result files of a SIMPLE run in the reference's export formats
// (src/io/ResultExporter.cpp:36-110 with CSVWriter.cpp and VTKWriter.cpp):
// residuals.csv always; fields.csv and solution.vtk only when every velocity
// and pressure value is finite (the reference skips them otherwise).  2D:
// CSVWriter::writeFields (:16-80) and VTKWriter::writeSolution (:29-171,
// single-block grid); 3D: CSVWriter::writeFields3D (:82-103) and
// VTKWriter::writeCellFields (:186-272) with pressure, velocity magnitude and
// velocity.  Every real is printed in the reference's one export format,
// scientific with 17 significant digits in the "C" locale
// (DeterministicOstream.hpp), i.e. printf's "%.17e"; cell centroids and grid
// vertices are the uniform grid's (i + 1/2) h and i h, h = length / cells.
// Host code only: cfdb_simple_write_results downloads the session's device
// fields first.
#include <cuda_runtime.h>
#include <sys/stat.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "cfdb.h"
#include "cfdb_internal.cuh"

namespace {

// One buffered output file; the writer appends with printf-style calls.
struct Out {
  FILE* f = nullptr;
  explicit Out(const std::string& path) { f = std::fopen(path.c_str(), "w"); }
  ~Out() {
    if (f) std::fclose(f);
  }
  bool ok() const { return f != nullptr; }
  void real(double v) { std::fprintf(f, "%.17e", v); }
  void text(const char* s) { std::fputs(s, f); }
  void integer(long long v) { std::fprintf(f, "%lld", v); }
  void ch(char c) { std::fputc(c, f); }
  bool close() {
    const bool good = std::ferror(f) == 0;
    const bool closed = std::fclose(f) == 0;
    f = nullptr;
    return good && closed;
  }
};

// Creates dir and its parents (create_directories).
bool make_dirs(const std::string& dir) {
  if (dir.empty()) return false;
  std::string cur;
  for (size_t i = 0; i <= dir.size(); ++i) {
    if (i == dir.size() || dir[i] == '/') {
      cur = dir.substr(0, i);
      if (!cur.empty() && mkdir(cur.c_str(), 0777) != 0 && errno != EEXIST) return false;
    }
  }
  struct stat st;
  return stat(dir.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}

double magnitude(double x, double y, double z, bool three) {
  // dot(v, v) of the reference's Vector3 (Vector3.hpp:78-82): the z term
  // only when it is non-zero
  const double in_plane = (x * x) + (y * y);
  const double normal = three ? z * z : 0.0;
  return std::sqrt(normal == 0.0 ? in_plane : in_plane + normal);
}

}  // namespace

extern "C" {

cfdb_status cfdb_write_results(const cfdb_simple_case* cs, const double* u, const double* v,
                               const double* w, const double* p, const double* history,
                               int64_t rows, double global_imbalance, const char* dir,
                               int* fields_written) {
  if (!cs || !u || !v || !p || !dir || rows < 0 || (rows > 0 && !history)) return CFDB_ERR_INVALID_ARGUMENT;
  const int dim = cs->grid.dim;
  if (dim != 2 && dim != 3) return CFDB_ERR_INVALID_ARGUMENT;
  if (dim == 3 && !w) return CFDB_ERR_INVALID_ARGUMENT;
  const int64_t nx = cs->grid.n[0], ny = cs->grid.n[1], nz = dim == 3 ? cs->grid.n[2] : 1;
  if (nx < 1 || ny < 1 || nz < 1) return CFDB_ERR_INVALID_ARGUMENT;
  const double hx = cs->grid.len[0] / (double)nx, hy = cs->grid.len[1] / (double)ny;
  const double hz = dim == 3 ? cs->grid.len[2] / (double)nz : 0.0;
  const int64_t n = nx * ny * nz;
  const std::string d(dir);
  if (!make_dirs(d)) return CFDB_ERR_INVALID_ARGUMENT;
  if (fields_written) *fields_written = 0;

  // residuals.csv (CSVWriter::writeResiduals, :105-142): one row per outer
  // iteration, the final global imbalance repeated on every row
  {
    Out o(d + "/residuals.csv");
    if (!o.ok()) return CFDB_ERR_INVALID_ARGUMENT;
    o.text(dim == 3 ? "iteration,u_residual,v_residual,w_residual,p_residual,continuity_residual,"
                      "global_mass_imbalance\n"
                    : "iteration,u_residual,v_residual,p_residual,continuity_residual,"
                      "global_mass_imbalance\n");
    for (int64_t k = 0; k < rows; ++k) {
      const double* h = history + 5 * k;  // {u, v, w, p, continuity}
      o.integer(k + 1);
      for (int c : {0, 1, 2, 3, 4}) {
        if (c == 2 && dim == 2) continue;
        o.ch(',');
        o.real(h[c]);
      }
      o.ch(',');
      o.real(global_imbalance);
      o.ch('\n');
    }
    if (!o.close()) return CFDB_ERR_INVALID_ARGUMENT;
  }

  for (int64_t c = 0; c < n; ++c)
    if (!std::isfinite(u[c]) || !std::isfinite(v[c]) || !std::isfinite(p[c]) ||
        (dim == 3 && !std::isfinite(w[c])))
      return CFDB_OK;  // no field files for a non-finite result

  // cell centres and nodes as AxisSpacing computes them (uniform: (i + 0.5)
  // delta and i delta; from node coordinates: 0.5 (n_i + n_i+1) and n_i)
  const double* const* nd = cs->nodes;
  auto cx = [&](int64_t i) { return nd[0] ? 0.5 * (nd[0][i] + nd[0][i + 1]) : ((double)i + 0.5) * hx; };
  auto cy = [&](int64_t j) { return nd[1] ? 0.5 * (nd[1][j] + nd[1][j + 1]) : ((double)j + 0.5) * hy; };
  auto cz = [&](int64_t k) {
    return (dim == 3 && nd[2]) ? 0.5 * (nd[2][k] + nd[2][k + 1]) : ((double)k + 0.5) * hz;
  };
  auto nxp = [&](int64_t i) { return nd[0] ? nd[0][i] : (double)i * hx; };
  auto nyp = [&](int64_t j) { return nd[1] ? nd[1][j] : (double)j * hy; };
  auto nzp = [&](int64_t k) { return (dim == 3 && nd[2]) ? nd[2][k] : (double)k * hz; };

  // fields.csv
  {
    Out o(d + "/fields.csv");
    if (!o.ok()) return CFDB_ERR_INVALID_ARGUMENT;
    o.text(dim == 3 ? "cell_id,x,y,z,velocity_x,velocity_y,velocity_z,velocity_magnitude,pressure\n"
                    : "cell_id,x,y,velocity_x,velocity_y,velocity_magnitude,pressure\n");
    for (int64_t c = 0; c < n; ++c) {
      const int64_t i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
      o.integer(c);
      o.ch(',');
      o.real(cx(i));
      o.ch(',');
      o.real(cy(j));
      if (dim == 3) {
        o.ch(',');
        o.real(cz(k));
      }
      o.ch(',');
      o.real(u[c]);
      o.ch(',');
      o.real(v[c]);
      if (dim == 3) {
        o.ch(',');
        o.real(w[c]);
      }
      o.ch(',');
      o.real(magnitude(u[c], v[c], dim == 3 ? w[c] : 0.0, dim == 3));
      o.ch(',');
      o.real(p[c]);
      o.ch('\n');
    }
    if (!o.close()) return CFDB_ERR_INVALID_ARGUMENT;
  }

  // solution.vtk
  {
    Out o(d + "/solution.vtk");
    if (!o.ok()) return CFDB_ERR_INVALID_ARGUMENT;
    o.text("# vtk DataFile Version 3.0\n");
    o.text(dim == 3 ? "CFDApp cell fields\n" : "CFDApp solution\n");
    o.text("ASCII\nDATASET UNSTRUCTURED_GRID\n");
    const int64_t px = nx + 1, py = ny + 1, pz = dim == 3 ? nz + 1 : 1;
    o.text("POINTS ");
    o.integer(px * py * pz);
    o.text(" double\n");
    for (int64_t k = 0; k < pz; ++k)
      for (int64_t j = 0; j < py; ++j)
        for (int64_t i = 0; i < px; ++i) {
          o.real(nxp(i));
          o.ch(' ');
          o.real(nyp(j));
          if (dim == 3) {
            o.ch(' ');
            o.real(nzp(k));
            o.ch('\n');
          } else {
            o.text(" 0\n");
          }
        }
    auto pt = [&](int64_t i, int64_t j, int64_t k) { return ((k * py) + j) * px + i; };
    const int per = dim == 3 ? 8 : 4;
    o.text("CELLS ");
    o.integer(n);
    o.ch(' ');
    o.integer(n * (per + 1));
    o.ch('\n');
    for (int64_t k = 0; k < nz; ++k)
      for (int64_t j = 0; j < ny; ++j)
        for (int64_t i = 0; i < nx; ++i) {
          const int64_t q[8] = {pt(i, j, k),         pt(i + 1, j, k),     pt(i + 1, j + 1, k),
                                pt(i, j + 1, k),     pt(i, j, k + 1),     pt(i + 1, j, k + 1),
                                pt(i + 1, j + 1, k + 1), pt(i, j + 1, k + 1)};
          o.integer(per);
          for (int t = 0; t < per; ++t) {
            o.ch(' ');
            o.integer(q[t]);
          }
          o.ch('\n');
        }
    o.text("CELL_TYPES ");
    o.integer(n);
    o.ch('\n');
    for (int64_t c = 0; c < n; ++c) o.text(dim == 3 ? "12\n" : "9\n");
    o.text("CELL_DATA ");
    o.integer(n);
    o.ch('\n');
    auto mag = [&](int64_t c) { return magnitude(u[c], v[c], dim == 3 ? w[c] : 0.0, dim == 3); };
    o.text("SCALARS pressure double 1\nLOOKUP_TABLE default\n");
    for (int64_t c = 0; c < n; ++c) {
      o.real(p[c]);
      o.ch('\n');
    }
    if (dim == 3) {
      // writeCellFields: scalar fields in the order given, then vectors
      o.text("SCALARS velocity_magnitude double 1\nLOOKUP_TABLE default\n");
      for (int64_t c = 0; c < n; ++c) {
        o.real(mag(c));
        o.ch('\n');
      }
      o.text("VECTORS velocity double\n");
      for (int64_t c = 0; c < n; ++c) {
        o.real(u[c]);
        o.ch(' ');
        o.real(v[c]);
        o.ch(' ');
        o.real(w[c]);
        o.ch('\n');
      }
    } else {
      // writeSolution: pressure, velocity, velocity magnitude
      o.text("VECTORS velocity double\n");
      for (int64_t c = 0; c < n; ++c) {
        o.real(u[c]);
        o.ch(' ');
        o.real(v[c]);
        o.text(" 0\n");
      }
      o.text("SCALARS velocity_magnitude double 1\nLOOKUP_TABLE default\n");
      for (int64_t c = 0; c < n; ++c) {
        o.real(mag(c));
        o.ch('\n');
      }
    }
    if (!o.close()) return CFDB_ERR_INVALID_ARGUMENT;
  }
  if (fields_written) *fields_written = 1;
  return CFDB_OK;
}

}  // extern "C"
