// af_io.cpp -- state files and VTU output (host code; the reference's output_results,
// Atmospheric_Flow.cc:886-918, and a restart format the reference does not have).
//
// State file (little-endian, version 1):
//   char magic[8] = "AFSTATE1"; int32 version, nx, nz, degree, periodic_x, gravity;
//   float64 radial_a, time; int64 step; float64 vertices[(nz+1)(nx+1)2];
//   float64 rho[n], u[2n], p[n]      (n = nx nz (degree+1)^2, deal.II DoF layout)
// VTU: the reference's DataOut::build_patches(mapping, degree, curved_inner_cells) output in
// 2D: every cell subdivided into degree x degree quadrilaterals on equispaced reference
// points, fields interpolated there from the Gauss-Lobatto nodes, points mapped with the
// cell's bilinear geometry; point data "rho", "u" (3 components, z = 0 as VTK vectors) and
// "p"; ASCII float64.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/af_gpu.h"
#include "af_tables.cuh"

namespace af {
void set_last_error(const char* msg);
}

namespace {

int ioerr(int code, const std::string& msg) {
  af::set_last_error(msg.c_str());
  return code;
}

const char kMagic[8] = {'A', 'F', 'S', 'T', 'A', 'T', 'E', '1'};

bool valid_mesh(const af_mesh_desc* m, int degree) {
  return m && m->vertices && m->nx > 0 && m->nz > 0 && degree >= 1 && degree <= 6;
}

// value of Lagrange basis j (Gauss-Lobatto nodes nd) at s
double lagrange(const std::vector<long double>& nd, int j, double s) {
  return (double)af::host::lag(nd, j, (long double)s);
}

}  // namespace

extern "C" {

int af_io_write_state(const char* path, const af_mesh_desc* mesh, int degree, double time, long long step,
                      const double* rho, const double* u, const double* p) {
  if (!path || !valid_mesh(mesh, degree) || !rho || !u || !p) return ioerr(AF_BAD_ARG, "af_io_write_state: bad argument");
  FILE* f = std::fopen(path, "wb");
  if (!f) return ioerr(AF_BAD_ARG, std::string("af_io_write_state: cannot open ") + path);
  const long n = (long)mesh->nx * mesh->nz * (degree + 1) * (degree + 1);
  const long nv = (long)(mesh->nx + 1) * (mesh->nz + 1) * 2;
  const int32_t hdr[6] = {1, mesh->nx, mesh->nz, degree, mesh->periodic_x, mesh->gravity};
  const double ra = mesh->radial_a;
  const int64_t st = step;
  bool ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(hdr, sizeof(hdr), 1, f) == 1 &&
            std::fwrite(&ra, 8, 1, f) == 1 && std::fwrite(&time, 8, 1, f) == 1 && std::fwrite(&st, 8, 1, f) == 1 &&
            std::fwrite(mesh->vertices, 8, nv, f) == (size_t)nv && std::fwrite(rho, 8, n, f) == (size_t)n &&
            std::fwrite(u, 8, 2 * n, f) == (size_t)(2 * n) && std::fwrite(p, 8, n, f) == (size_t)n;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? AF_OK : ioerr(AF_BAD_ARG, std::string("af_io_write_state: write failed: ") + path);
}

int af_io_read_state_header(const char* path, af_state_header* h) {
  if (!path || !h) return ioerr(AF_BAD_ARG, "af_io_read_state_header: bad argument");
  FILE* f = std::fopen(path, "rb");
  if (!f) return ioerr(AF_BAD_ARG, std::string("af_io_read_state_header: cannot open ") + path);
  char mg[8];
  int32_t hdr[6];
  double ra = 0, t = 0;
  int64_t st = 0;
  const bool ok = std::fread(mg, 1, 8, f) == 8 && std::memcmp(mg, kMagic, 8) == 0 &&
                  std::fread(hdr, sizeof(hdr), 1, f) == 1 && hdr[0] == 1 && std::fread(&ra, 8, 1, f) == 1 &&
                  std::fread(&t, 8, 1, f) == 1 && std::fread(&st, 8, 1, f) == 1;
  std::fclose(f);
  if (!ok) return ioerr(AF_BAD_ARG, std::string("af_io_read_state_header: not a version-1 state file: ") + path);
  h->nx = hdr[1];
  h->nz = hdr[2];
  h->degree = hdr[3];
  h->periodic_x = hdr[4];
  h->gravity = hdr[5];
  h->radial_a = ra;
  h->time = t;
  h->step = st;
  return AF_OK;
}

int af_io_read_state(const char* path, double* vertices, double* rho, double* u, double* p) {
  af_state_header h{};
  int r = af_io_read_state_header(path, &h);
  if (r != AF_OK) return r;
  if (!vertices || !rho || !u || !p) return ioerr(AF_BAD_ARG, "af_io_read_state: null buffer");
  FILE* f = std::fopen(path, "rb");
  if (!f) return ioerr(AF_BAD_ARG, std::string("af_io_read_state: cannot open ") + path);
  const long n = (long)h.nx * h.nz * (h.degree + 1) * (h.degree + 1);
  const long nv = (long)(h.nx + 1) * (h.nz + 1) * 2;
  bool ok = std::fseek(f, 8 + 6 * 4 + 3 * 8, SEEK_SET) == 0 && std::fread(vertices, 8, nv, f) == (size_t)nv &&
            std::fread(rho, 8, n, f) == (size_t)n && std::fread(u, 8, 2 * n, f) == (size_t)(2 * n) &&
            std::fread(p, 8, n, f) == (size_t)n;
  std::fclose(f);
  return ok ? AF_OK : ioerr(AF_BAD_ARG, std::string("af_io_read_state: truncated file: ") + path);
}

int af_io_write_vtu(const char* path, const af_mesh_desc* mesh, int degree, const double* rho, const double* u,
                    const double* p) {
  if (!path || !valid_mesh(mesh, degree) || !rho || !u || !p) return ioerr(AF_BAD_ARG, "af_io_write_vtu: bad argument");
  const int P = degree, P1 = P + 1, ND = P1 * P1;
  const int nx = mesh->nx, nz = mesh->nz, ncell = nx * nz;
  const std::vector<long double> nd = af::host::gll(P);
  std::vector<double> L(P1 * P1);  // L[i][j] = l_j(i / P), equispaced patch points
  for (int i = 0; i < P1; ++i)
    for (int j = 0; j < P1; ++j) L[i * P1 + j] = lagrange(nd, j, (double)i / P);
  FILE* f = std::fopen(path, "w");
  if (!f) return ioerr(AF_BAD_ARG, std::string("af_io_write_vtu: cannot open ") + path);
  const long npts = (long)ncell * ND, ncells_vtk = (long)ncell * P * P;
  std::fprintf(f, "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n");
  std::fprintf(f, "<UnstructuredGrid>\n<Piece NumberOfPoints=\"%ld\" NumberOfCells=\"%ld\">\n", npts, ncells_vtk);
  std::vector<double> t(ND), v(ND);
  auto interp = [&](const double* src) {  // nodal -> equispaced patch values of one cell field
    for (int iz = 0; iz < P1; ++iz)
      for (int ix = 0; ix < P1; ++ix) {
        double s = 0.0;
        for (int jx = 0; jx < P1; ++jx) s += L[ix * P1 + jx] * src[iz * P1 + jx];
        t[iz * P1 + ix] = s;
      }
    for (int iz = 0; iz < P1; ++iz)
      for (int ix = 0; ix < P1; ++ix) {
        double s = 0.0;
        for (int jz = 0; jz < P1; ++jz) s += L[iz * P1 + jz] * t[jz * P1 + ix];
        v[iz * P1 + ix] = s;
      }
  };
  // points
  std::fprintf(f, "<Points>\n<DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n");
  const double* X = mesh->vertices;
  const int W = nx + 1;
  for (int c = 0; c < ncell; ++c) {
    const int i = c % nx, j = c / nx;
    const double* v0 = X + 2 * (j * W + i);
    const double* v1 = X + 2 * (j * W + i + 1);
    const double* v2 = X + 2 * ((j + 1) * W + i);
    const double* v3 = X + 2 * ((j + 1) * W + i + 1);
    for (int iz = 0; iz < P1; ++iz)
      for (int ix = 0; ix < P1; ++ix) {
        const double a = (double)ix / P, b = (double)iz / P;
        const double x = (1 - a) * (1 - b) * v0[0] + a * (1 - b) * v1[0] + (1 - a) * b * v2[0] + a * b * v3[0];
        const double z = (1 - a) * (1 - b) * v0[1] + a * (1 - b) * v1[1] + (1 - a) * b * v2[1] + a * b * v3[1];
        std::fprintf(f, "%.17g %.17g 0\n", x, z);
      }
  }
  std::fprintf(f, "</DataArray>\n</Points>\n<Cells>\n<DataArray type=\"Int64\" Name=\"connectivity\" format=\"ascii\">\n");
  for (long c = 0; c < ncell; ++c)
    for (int iz = 0; iz < P; ++iz)
      for (int ix = 0; ix < P; ++ix) {
        const long b = c * ND + iz * P1 + ix;
        std::fprintf(f, "%ld %ld %ld %ld\n", b, b + 1, b + P1 + 1, b + P1);
      }
  std::fprintf(f, "</DataArray>\n<DataArray type=\"Int64\" Name=\"offsets\" format=\"ascii\">\n");
  for (long k = 1; k <= ncells_vtk; ++k) std::fprintf(f, "%ld\n", 4 * k);
  std::fprintf(f, "</DataArray>\n<DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n");
  for (long k = 0; k < ncells_vtk; ++k) std::fprintf(f, "9\n");  // VTK_QUAD
  std::fprintf(f, "</DataArray>\n</Cells>\n<PointData Scalars=\"rho\" Vectors=\"u\">\n");
  std::fprintf(f, "<DataArray type=\"Float64\" Name=\"rho\" format=\"ascii\">\n");
  for (int c = 0; c < ncell; ++c) {
    interp(rho + (size_t)c * ND);
    for (int k = 0; k < ND; ++k) std::fprintf(f, "%.17g\n", v[k]);
  }
  std::fprintf(f, "</DataArray>\n<DataArray type=\"Float64\" Name=\"u\" NumberOfComponents=\"3\" format=\"ascii\">\n");
  std::vector<double> ux(ND);
  for (int c = 0; c < ncell; ++c) {
    interp(u + (size_t)c * 2 * ND);
    ux = v;
    interp(u + (size_t)c * 2 * ND + ND);
    for (int k = 0; k < ND; ++k) std::fprintf(f, "%.17g %.17g 0\n", ux[k], v[k]);
  }
  std::fprintf(f, "</DataArray>\n<DataArray type=\"Float64\" Name=\"p\" format=\"ascii\">\n");
  for (int c = 0; c < ncell; ++c) {
    interp(p + (size_t)c * ND);
    for (int k = 0; k < ND; ++k) std::fprintf(f, "%.17g\n", v[k]);
  }
  std::fprintf(f, "</DataArray>\n</PointData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n");
  const bool ok = std::ferror(f) == 0;
  return (std::fclose(f) == 0 && ok) ? AF_OK : ioerr(AF_BAD_ARG, std::string("af_io_write_vtu: write failed: ") + path);
}

}  // extern "C"
