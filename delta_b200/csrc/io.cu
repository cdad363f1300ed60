// io.cu -- the reference's on-disk formats: the legacy VTK snapshot of the triangulated
// particles (writeGeometryToVTK, delta/core/io/write.cpp:226-306) and the .mbfcp scene
// reader (readmbfcp, delta/core/io/read.cpp:345-546).  Host code; the device entry point
// copies the meshes back first.
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "internal.h"

namespace delta {
namespace {

delta_status write_vtk(const std::string &path, int32_t step, int32_t n_bodies, const int64_t *tri_offset,
                       const double *x, const double *y, const double *z) {
  // file name as write.cpp:231-237: path + "geometry_" + step + ".vtk"
  const std::string filename = path + "geometry_" + std::to_string((unsigned)step) + ".vtk";
  FILE *fp = std::fopen(filename.c_str(), "w+");
  if (!fp) return set_error(DELTA_ERR_INVALID, "delta_write_vtk: cannot open " + filename + ": " + std::strerror(errno));
  const int64_t faces = tri_offset[n_bodies] - tri_offset[0];
  const int64_t vertices = 3 * faces;
  std::fprintf(fp,
               "# vtk DataFile Version 2.0\n"
               "Output vtk file\n"
               "ASCII\n\n"
               "DATASET UNSTRUCTURED_GRID\n"
               "POINTS %lld double\n",
               (long long)vertices);
  for (int64_t v = 3 * tri_offset[0]; v < 3 * tri_offset[n_bodies]; ++v)
    std::fprintf(fp, "%.5f %.5f %.5f\n", x[v], y[v], z[v]);
  std::fprintf(fp, "\nCELLS %lld %lld\n", (long long)faces, (long long)(4 * faces));
  for (int64_t f = 0; f < faces; ++f)
    std::fprintf(fp, "3 %lld %lld %lld\n", (long long)(3 * f), (long long)(3 * f + 1), (long long)(3 * f + 2));
  std::fprintf(fp, "\nCELL_TYPES %lld\n", (long long)faces);
  for (int64_t f = 0; f < faces; ++f) std::fputs("5\n", fp);
  const bool ok = std::ferror(fp) == 0;
  std::fclose(fp);
  return ok ? DELTA_OK : set_error(DELTA_ERR_INVALID, "delta_write_vtk: write failed: " + filename);
}

// writeGeometryToVTKVTK (delta/core/io/write.cpp:10-70) without the VTK library: the same
// unstructured grid of particle centres, written as ASCII VTK XML.  The reference inserts
// the centres into a vtkPoints (float by default, so Float32), the linear velocity as the
// "direction" vectors and then calls SetScalars twice, radius and then epsilon; the second
// call replaces the first attribute, so the file holds "direction" and "epsilon" (Float64)
// and no cells.  The reference's writer encodes the arrays in binary; the arrays and their
// values are the same.
delta_status write_vtu(const std::string &path, int32_t step, int64_t n, const double *centre,
                       const double *velocity, const double *eps) {
  const std::string filename = path + "geometry_" + std::to_string(step) + ".vtu";
  FILE *fp = std::fopen(filename.c_str(), "w");
  if (!fp) return set_error(DELTA_ERR_INVALID, "delta_write_vtu: cannot open " + filename + ": " + std::strerror(errno));
  std::fprintf(fp,
               "<?xml version=\"1.0\"?>\n"
               "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
               "  <UnstructuredGrid>\n"
               "    <Piece NumberOfPoints=\"%lld\" NumberOfCells=\"0\">\n"
               "      <PointData Scalars=\"epsilon\" Vectors=\"direction\">\n"
               "        <DataArray type=\"Float64\" Name=\"direction\" NumberOfComponents=\"3\" format=\"ascii\">\n",
               (long long)n);
  for (int64_t i = 0; i < n; ++i)
    std::fprintf(fp, "%.17g %.17g %.17g\n", velocity[i], velocity[n + i], velocity[2 * n + i]);
  std::fputs("        </DataArray>\n"
             "        <DataArray type=\"Float64\" Name=\"epsilon\" format=\"ascii\">\n", fp);
  for (int64_t i = 0; i < n; ++i) std::fprintf(fp, "%.17g\n", eps[i]);
  std::fputs("        </DataArray>\n"
             "      </PointData>\n"
             "      <CellData>\n"
             "      </CellData>\n"
             "      <Points>\n"
             "        <DataArray type=\"Float32\" Name=\"Points\" NumberOfComponents=\"3\" format=\"ascii\">\n", fp);
  for (int64_t i = 0; i < n; ++i)
    std::fprintf(fp, "%.9g %.9g %.9g\n", (double)(float)centre[i], (double)(float)centre[n + i],
                 (double)(float)centre[2 * n + i]);
  std::fputs("        </DataArray>\n"
             "      </Points>\n"
             "      <Cells>\n"
             "        <DataArray type=\"Int64\" Name=\"connectivity\" format=\"ascii\">\n"
             "        </DataArray>\n"
             "        <DataArray type=\"Int64\" Name=\"offsets\" format=\"ascii\">\n"
             "        </DataArray>\n"
             "        <DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n"
             "        </DataArray>\n"
             "      </Cells>\n"
             "    </Piece>\n"
             "  </UnstructuredGrid>\n"
             "</VTKFile>\n", fp);
  const bool ok = std::ferror(fp) == 0;
  std::fclose(fp);
  return ok ? DELTA_OK : set_error(DELTA_ERR_INVALID, "delta_write_vtu: write failed: " + filename);
}

// std::stoi / std::stof / std::stod on a substring as read.cpp does; false on a parse error
template <class F>
bool parse_at(const std::string &line, size_t pos, size_t len, F conv) {
  if (pos > line.size()) return false;
  try {
    conv(line.substr(pos, len));
  } catch (...) {
    return false;
  }
  return true;
}

}  // namespace
}  // namespace delta

using namespace delta;

extern "C" {

delta_status delta_write_vtk_host(const char *path, int32_t step, int32_t n_bodies, const int64_t *tri_offset,
                                  const double *x, const double *y, const double *z) {
  if (!path || n_bodies < 0 || !tri_offset || (tri_offset[n_bodies] > tri_offset[0] && (!x || !y || !z)))
    return set_error(DELTA_ERR_INVALID, "delta_write_vtk_host: bad argument");
  return write_vtk(path, step, n_bodies, tri_offset, x, y, z);
}

delta_status delta_write_vtu_host(const char *path, int32_t step, int64_t n, const double *centre,
                                  const double *velocity, const double *eps) {
  if (!path || n < 0 || (n > 0 && (!centre || !velocity || !eps)))
    return set_error(DELTA_ERR_INVALID, "delta_write_vtu_host: bad argument");
  return write_vtu(path, step, n, centre, velocity, eps);
}

delta_status delta_write_vtk(delta_ctx *ctx, const char *path, int32_t step, const delta_meshes *meshes) {
  if (!ctx || !path || !meshes || meshes->n_bodies < 0 || !meshes->tri_offset)
    return set_error(DELTA_ERR_INVALID, "delta_write_vtk: bad argument");
  const int32_t nb = meshes->n_bodies;
  std::vector<int64_t> off(nb + 1);
  cudaError_t e = cudaMemcpyAsync(off.data(), meshes->tri_offset, sizeof(int64_t) * (nb + 1), cudaMemcpyDeviceToHost,
                                  ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_error(e, "delta_write_vtk: offsets");
  const int64_t nv = 3 * (off[nb] - off[0]);
  std::vector<double> x(nv), y(nv), z(nv);
  if (nv > 0) {
    const size_t bytes = sizeof(double) * nv;
    const int64_t v0 = 3 * off[0];
    e = cudaMemcpyAsync(x.data(), meshes->x + v0, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(y.data(), meshes->y + v0, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(z.data(), meshes->z + v0, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_error(e, "delta_write_vtk: vertices");
  }
  // host arrays start at vertex 3*off[0]: rebase the offsets
  const int64_t base = off[0];
  for (auto &o : off) o -= base;
  return write_vtk(path, step, nb, off.data(), x.data(), y.data(), z.data());
}

delta_status delta_read_mbfcp(const char *filename, delta_mbfcp *out, int64_t capacity, int64_t *n_out) {
  if (!filename || !out || !n_out || capacity < 0 ||
      (capacity > 0 && (!out->id || !out->centre || !out->radius)))
    return set_error(DELTA_ERR_INVALID, "delta_read_mbfcp: bad argument");
  *n_out = 0;
  std::ifstream file(filename);
  if (!file.is_open()) return set_error(DELTA_ERR_INVALID, std::string("delta_read_mbfcp: cannot open ") + filename);
  int64_t n = 0;
  bool bad = false;
  out->bodies = 0;
  out->has_materials = 0;
  for (std::string line; std::getline(file, line);) {
    if (line.empty()) continue;
    // materials block, read.cpp:374-437 (fields at the reference's fixed offsets)
    if (line.find("SURFACE_MATERIALS:") != std::string::npos) {
      // the 19 lines after the header: surf1, surf2, model, friction, cohesion, spring,
      // dashpot, -, bulk count, label, model, young, poisson, density, -, -, gravity x,y,z
      std::string l[19];
      for (int k = 0; k < 19 && std::getline(file, l[k]); ++k) {
      }
      bad |= !parse_at(l[3], 10, std::string::npos, [&](const std::string &s) { out->friction = std::stof(s); });
      bad |= !parse_at(l[5], 8, std::string::npos, [&](const std::string &s) { out->spring = std::stof(s); });
      bad |= !parse_at(l[6], 8, std::string::npos, [&](const std::string &s) { out->dashpot = std::stof(s); });
      bad |= !parse_at(l[13], 9, std::string::npos, [&](const std::string &s) { out->density = std::stof(s); });
      for (int k = 0; k < 3; ++k)
        bad |= !parse_at(l[16 + k], 10, std::string::npos,
                         [&](const std::string &s) { out->gravity[k] = std::stof(s); });
      out->has_materials = 1;
      line = l[18];
    }
    // read.cpp:440-443
    if (line.find("BODIES:") != std::string::npos)
      bad |= !parse_at(line, 8, std::string::npos, [&](const std::string &s) { out->bodies = std::stoi(s); });
    // a body, read.cpp:476-540: only SPHERES shapes give particles
    if (line.find("ID:") != std::string::npos && line.find("SURFID:") != 0) {
      int id = 0;
      bad |= !parse_at(line, 3, std::string::npos, [&](const std::string &s) { id = std::stoi(s); });
      // label, kinematics, bulk material, shapes, then the line checked for SPHERES
      for (int k = 0; k < 5 && std::getline(file, line); ++k) {
      }
      if (line.find("SPHERES:") != std::string::npos) {
        double c[3] = {0, 0, 0}, rad = 0;
        std::getline(file, line);
        for (int k = 0; k < 3; ++k)
          bad |= !parse_at(line, 8 + 6 * k, 4, [&](const std::string &s) { c[k] = std::stod(s); });
        std::getline(file, line);
        bad |= !parse_at(line, 8, 4, [&](const std::string &s) { rad = std::stod(s); });
        if (n < capacity) {
          out->id[n] = id;
          for (int k = 0; k < 3; ++k) out->centre[3 * n + k] = c[k];
          out->radius[n] = rad;
        }
        ++n;
      }
    }
  }
  *n_out = n;
  if (bad) return set_error(DELTA_ERR_INVALID, std::string("delta_read_mbfcp: malformed field in ") + filename);
  if (n > capacity) return set_error(DELTA_ERR_CAPACITY, "delta_read_mbfcp: more spheres than capacity");
  return DELTA_OK;
}

}  // extern "C"
