// The on-disk formats either side of a solve: restart files and VTU output.
//
// Restart files follow write_restart / read_restart
// (src/FiniteElement/include/iceicle/fe_function/restart.hpp:20-108): plain
// text, the mesh node coordinates ("x y " per node), one newline, then u in
// layout order, every value followed by a space, 16 significant digits.
//
// VTU files follow PVDWriter (src/io/include/iceicle/pvd_writer.hpp): an ASCII
// UnstructuredGrid in the discontinuous layout, every element its own VTK cell
// with its own copies of the points. The cell type follows the larger of the
// geometry order and the basis order (1: VTK_QUAD, 2: VTK_BIQUADRATIC_QUAD,
// 3 and above: VTK_QUADRATIC_QUAD), the points are the cell's reference nodes
// mapped through the element's geometry, and every field is the basis
// expansion evaluated at those nodes. Residual files carry the full residual
// and its domain and trace parts; the MDG file carries the interface
// conservation residual of the selected nodes as an isoparametric nodal field.
//
// The state comes from the device in one copy; evaluation at the VTK nodes and
// the formatting run on the host, which is where the file is written.
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <string>
#include <vector>

#include "icx_internal.h"

namespace {

icx_status io_fail(icx_ctx* c, icx_status st, const std::string& msg) {
  if (c) c->err = msg;
  return st;
}

// appends v formatted as printf's %.<prec>g (what an ostream with
// setprecision(prec) and the default float format prints)
void put(std::string& out, double v, int prec) {
  char buf[64];
  int n = std::snprintf(buf, sizeof(buf), "%.*g", prec, v);
  out.append(buf, (size_t)n);
}

bool write_file(const std::filesystem::path& path, const std::string& text) {
  FILE* f = std::fopen(path.string().c_str(), "wb");
  if (!f) return false;
  bool ok = std::fwrite(text.data(), 1, text.size(), f) == text.size();
  ok = (std::fclose(f) == 0) && ok;
  return ok;
}

bool make_dir(const std::filesystem::path& d) {
  std::error_code ec;
  std::filesystem::create_directories(d, ec);
  return !ec;
}

// reference nodes of the VTK cell used for a given order (pvd_writer.hpp:98-140,
// get_vtk_element :175-243)
struct VtkCell {
  std::vector<double> xi;  // [n][2]
  int id;
};

VtkCell vtk_cell(int order) {
  if (order <= 1) return {{-1, -1, 1, -1, 1, 1, -1, 1}, 9};
  if (order == 2) return {{-1, -1, 1, -1, 1, 1, -1, 1, 0, -1, 1, 0, 0, 1, -1, 0, 0, 0}, 28};
  return {{-1, -1, 1, -1, 1, 1, -1, 1, 0, -1, 1, 0, 0, 1, -1, 0}, 23};
}

// tensor-product values of order pn of a basis family at xi, basis index i0 * (pn+1) + i1
void tp_values(int kind, int pn, const double xi[2], double* phi) {
  double a[16], b[16];
  icx::basis_values(kind, pn, xi[0], a);
  icx::basis_values(kind, pn, xi[1], b);
  for (int i = 0; i <= pn; ++i)
    for (int j = 0; j <= pn; ++j) phi[i * (pn + 1) + j] = a[i] * b[j];
}

void xml_open(std::string& o, const char* name, const std::vector<std::pair<std::string, std::string>>& attrs) {
  o += '<';
  o += name;
  for (const auto& a : attrs) o += " " + a.first + "=\"" + a.second + "\"";
  o += ">\n";
}
void xml_close(std::string& o, const char* name) {
  o += "</";
  o += name;
  o += ">\n";
}

// the grid part of a discontinuous-layout VTU (write_dg_unstructured_grid,
// pvd_writer.hpp:988-1088) up to and including the opening PointData tag
void grid(std::string& o, const icx_ctx* c, const VtkCell& cell, int prec) {
  const int E = c->n_elem;
  const int nv = (int)cell.xi.size() / 2;
  o += "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n";
  xml_open(o, "UnstructuredGrid", {});
  xml_open(o, "Piece", {{"NumberOfPoints", std::to_string((size_t)E * nv)}, {"NumberOfCells", std::to_string(E)}});
  xml_open(o, "Points", {});
  xml_open(o, "DataArray", {{"type", "Float64"}, {"Name", "Points"}, {"NumberOfComponents", "3"}, {"format", "ascii"}});
  for (int e = 0; e < E; ++e)
    for (int k = 0; k < nv; ++k) {
      double x[2];
      icx::element_point(c, e, &cell.xi[2 * k], x);
      put(o, x[0], prec);
      o += ' ';
      put(o, x[1], prec);
      o += " 0 \n";
    }
  xml_close(o, "DataArray");
  xml_close(o, "Points");
  xml_open(o, "Cells", {});
  xml_open(o, "DataArray", {{"type", "Int64"}, {"Name", "connectivity"}, {"format", "ascii"}});
  size_t g = 0;
  for (int e = 0; e < E; ++e) {
    for (int k = 0; k < nv; ++k) o += std::to_string(g++) + " ";
    o += '\n';
  }
  xml_close(o, "DataArray");
  xml_open(o, "DataArray", {{"type", "Int64"}, {"Name", "offsets"}, {"format", "ascii"}});
  for (int e = 0; e < E; ++e) o += std::to_string((size_t)(e + 1) * nv) + " ";
  o += '\n';
  xml_close(o, "DataArray");
  xml_open(o, "DataArray", {{"type", "Int64"}, {"Name", "types"}, {"format", "ascii"}});
  for (int e = 0; e < E; ++e) o += std::to_string(cell.id) + " ";
  o += '\n';
  xml_close(o, "DataArray");
  xml_close(o, "Cells");
  xml_open(o, "PointData", {});
}

void footer(std::string& o) {
  xml_close(o, "PointData");
  xml_close(o, "Piece");
  xml_close(o, "UnstructuredGrid");
  o += "</VTKFile>\n";
}

// one Float64 DataArray: the point values pv[point][nf], component f
void field(std::string& o, const std::string& name, const std::vector<double>& pv, int nf, int f, int E, int nv,
           int prec) {
  xml_open(o, "DataArray", {{"type", "Float64"}, {"Name", name}, {"format", "ascii"}});
  size_t k = 0;
  for (int e = 0; e < E; ++e) {
    for (int j = 0; j < nv; ++j, ++k) {
      o += ' ';
      put(o, pv[k * nf + f], prec);
    }
    o += '\n';
  }
  xml_close(o, "DataArray");
}

// values at the VTK nodes of the element expansion v[e][nbasis][neq] of order pn
std::vector<double> at_nodes(const std::vector<double>& v, int E, int kind, int pn, int neq, const VtkCell& cell) {
  const int nb = (pn + 1) * (pn + 1), nv = (int)cell.xi.size() / 2;
  std::vector<double> phi((size_t)nv * nb);
  for (int k = 0; k < nv; ++k) tp_values(kind, pn, &cell.xi[2 * k], &phi[(size_t)k * nb]);
  std::vector<double> out((size_t)E * nv * neq, 0.0);
  for (int e = 0; e < E; ++e)
    for (int k = 0; k < nv; ++k)
      for (int q = 0; q < neq; ++q) {
        double s = 0.0;
        for (int i = 0; i < nb; ++i) s += v[((size_t)e * nb + i) * neq + q] * phi[(size_t)k * nb + i];
        out[((size_t)e * nv + k) * neq + q] = s;
      }
  return out;
}

std::vector<std::string> names_or(const char* const* names, int n, std::vector<std::string> dflt) {
  if (!names) return dflt;
  std::vector<std::string> r;
  for (int i = 0; i < n; ++i) r.push_back(names[i] ? names[i] : "");
  return r;
}

std::vector<std::string> default_fields(const icx_ctx* c) {
  if (c->phys.pde == ICX_PDE_BURGERS) return {"u"};
  return {"rho", "rhou", "rhov", "rhoe"};
}
std::vector<std::string> default_residuals(const icx_ctx* c) {
  if (c->phys.pde == ICX_PDE_BURGERS) return {"residual"};
  return {"density_conservation", "momentum_u_conservation", "momentum_v_conservation", "energy_conservation"};
}

icx_status check_ctx(icx_ctx* c) {
  if (!c || !c->ready) return io_fail(c, ICX_ERR_INVALID, "context not set up");
  if (!c->parts.empty()) return io_fail(c, ICX_ERR_UNSUPPORTED, "restart and VTU files describe one mesh, not a batch");
  return ICX_OK;
}

size_t n_unknowns(const icx_ctx* c) { return (size_t)c->dm.E * c->dm.nb * c->dm.neq; }

}  // namespace

extern "C" {

icx_status icx_write_restart(icx_ctx* c, const double* d_u, int k, int rank, const char* dir) {
  icx_status st = check_ctx(c);
  if (st != ICX_OK) return st;
  if (!d_u) return io_fail(c, ICX_ERR_INVALID, "null state");
  cudaSetDevice(c->device);
  std::vector<double> u(n_unknowns(c));
  if (cudaMemcpy(u.data(), d_u, sizeof(double) * u.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
    return io_fail(c, ICX_ERR_CUDA, "copy of u to the host failed");
  std::filesystem::path d = dir ? std::filesystem::path(dir) : std::filesystem::current_path() / "RESTART";
  if (!make_dir(d)) return io_fail(c, ICX_ERR_INVALID, "cannot create " + d.string());
  std::string o;
  o.reserve((c->coord.size() + u.size()) * 24 + 16);
  for (double x : c->coord) {
    put(o, x, 16);
    o += ' ';
  }
  o += '\n';
  for (double v : u) {
    put(o, v, 16);
    o += ' ';
  }
  std::filesystem::path f = d / ("restart" + std::to_string(k) + "_" + std::to_string(rank));
  if (!write_file(f, o)) return io_fail(c, ICX_ERR_INVALID, "cannot write " + f.string());
  return ICX_OK;
}

icx_status icx_read_restart(icx_ctx* c, double* d_u, const char* name, int rank, const char* dir) {
  icx_status st = check_ctx(c);
  if (st != ICX_OK) return st;
  if (!d_u || !name) return io_fail(c, ICX_ERR_INVALID, "null state or file name");
  std::filesystem::path d = dir ? std::filesystem::path(dir) : std::filesystem::current_path() / "RESTART";
  std::filesystem::path f = d / (std::string(name) + "_" + std::to_string(rank));
  FILE* fp = std::fopen(f.string().c_str(), "rb");
  if (!fp) return io_fail(c, ICX_ERR_INVALID, "cannot open " + f.string());
  std::string text;
  char buf[1 << 16];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof(buf), fp)) > 0) text.append(buf, n);
  std::fclose(fp);
  const size_t nc = c->coord.size(), nu = n_unknowns(c);
  std::vector<double> vals;
  vals.reserve(nc + nu);
  const char* p = text.c_str();
  while (vals.size() < nc + nu) {
    char* end = nullptr;
    errno = 0;
    double v = std::strtod(p, &end);
    if (end == p) break;
    vals.push_back(v);
    p = end;
  }
  if (vals.size() < nc + nu)
    return io_fail(c, ICX_ERR_INVALID,
                   f.string() + ": " + std::to_string(vals.size()) + " numbers, expected " + std::to_string(nc + nu));
  if ((st = icx_mesh_set_coords(c, vals.data())) != ICX_OK) return st;
  cudaSetDevice(c->device);
  if (cudaMemcpy(d_u, vals.data() + nc, sizeof(double) * nu, cudaMemcpyHostToDevice) != cudaSuccess)
    return io_fail(c, ICX_ERR_CUDA, "copy of u to the device failed");
  return ICX_OK;
}

icx_status icx_write_vtu(icx_ctx* c, const double* d_u, int kind, int itime, const char* dir,
                         const char* collection, const char* const* names, int precision) {
  icx_status st = check_ctx(c);
  if (st != ICX_OK) return st;
  if (!d_u || (kind != ICX_VTU_SOLUTION && kind != ICX_VTU_RESIDUAL) || precision < 1 || precision > 17)
    return io_fail(c, ICX_ERR_INVALID, "bad VTU arguments");
  cudaSetDevice(c->device);
  const int E = c->dm.E, neq = c->dm.neq, P = c->p;
  const size_t N = n_unknowns(c);
  // fields as element expansions [e][nb][neq], one block of N per field set
  std::vector<double> v(kind == ICX_VTU_SOLUTION ? N : 3 * N);
  cudaError_t e = cudaSuccess;
  if (kind == ICX_VTU_SOLUTION) {
    e = cudaMemcpy(v.data(), d_u, sizeof(double) * N, cudaMemcpyDeviceToHost);
  } else {
    double* d_r = nullptr;
    e = cudaMalloc((void**)&d_r, sizeof(double) * 2 * N);
    if (e != cudaSuccess) return io_fail(c, ICX_ERR_NOMEM, "residual buffers");
    e = icx::launch_residual(c->dm, c->phys, d_u, d_r, 0);
    if (e == cudaSuccess) e = icx::launch_residual_domain(c->dm, c->phys, d_u, d_r + N, 0);
    if (e == cudaSuccess) e = cudaMemcpy(v.data(), d_r, sizeof(double) * 2 * N, cudaMemcpyDeviceToHost);
    cudaFree(d_r);
    // trace part = full residual - domain part
    for (size_t i = 0; i < N; ++i) v[2 * N + i] = v[i] - v[N + i];
  }
  if (e != cudaSuccess) return io_fail(c, ICX_ERR_CUDA, std::string("VTU fields: ") + cudaGetErrorString(e));
  const VtkCell cell = vtk_cell(std::max(c->geo_order, P));
  const int nv = (int)cell.xi.size() / 2;
  std::string o;
  grid(o, c, cell, precision);
  if (kind == ICX_VTU_SOLUTION) {
    auto nm = names_or(names, neq, default_fields(c));
    auto pv = at_nodes(v, E, c->basis, P, neq, cell);
    for (int q = 0; q < neq; ++q) field(o, nm[q], pv, neq, q, E, nv, precision);
  } else {
    auto nm = names_or(names, neq, default_residuals(c));
    const char* prefix[3] = {"", "domain_", "trace_"};
    for (int part = 0; part < 3; ++part) {
      std::vector<double> vp(v.begin() + part * N, v.begin() + (part + 1) * N);
      auto pv = at_nodes(vp, E, c->basis, P, neq, cell);
      for (int q = 0; q < neq; ++q) field(o, prefix[part] + nm[q], pv, neq, q, E, nv, precision);
    }
  }
  footer(o);
  std::filesystem::path d = dir ? std::filesystem::path(dir) : std::filesystem::current_path() / "iceicle_data";
  if (!make_dir(d)) return io_fail(c, ICX_ERR_INVALID, "cannot create " + d.string());
  const char* coll = collection ? collection : (kind == ICX_VTU_SOLUTION ? "data" : "residuals");
  std::filesystem::path f = d / (std::string(coll) + std::to_string(itime) + ".vtu");
  if (!write_file(f, o)) return io_fail(c, ICX_ERR_INVALID, "cannot write " + f.string());
  return ICX_OK;
}

icx_status icx_write_vtu_mdg(icx_ctx* c, const double* d_ic, int itime, const char* dir, const char* collection,
                             const char* const* names, int precision) {
  icx_status st = check_ctx(c);
  if (st != ICX_OK) return st;
  if (!d_ic || precision < 1 || precision > 17) return io_fail(c, ICX_ERR_INVALID, "bad VTU arguments");
  int nsel = 0, ngeo = 0;
  if (icx_mdg_info(c, &nsel, &ngeo) != ICX_OK || nsel <= 0)
    return io_fail(c, ICX_ERR_INVALID, "no MDG node selection (icx_mdg_select)");
  std::vector<int> sel(nsel);
  if ((st = icx_mdg_selected_nodes(c, sel.data())) != ICX_OK) return st;
  const int neq = c->dm.neq, G = c->geo_order, E = c->n_elem, ng = (G + 1) * (G + 1);
  std::vector<double> ic((size_t)nsel * neq);
  cudaSetDevice(c->device);
  if (cudaMemcpy(ic.data(), d_ic, sizeof(double) * ic.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
    return io_fail(c, ICX_ERR_CUDA, "copy of the interface residual failed");
  // nodal field: selected nodes carry their residual, all others zero
  const size_t n_nodes = c->coord.size() / 2;
  std::vector<double> nodal(n_nodes * neq, 0.0);
  for (int i = 0; i < nsel; ++i)
    for (int q = 0; q < neq; ++q) nodal[(size_t)sel[i] * neq + q] = ic[(size_t)i * neq + q];
  // isoparametric expansion per element: coefficients are the element's nodes
  std::vector<double> v((size_t)E * ng * neq);
  for (int e = 0; e < E; ++e)
    for (int n = 0; n < ng; ++n)
      for (int q = 0; q < neq; ++q)
        v[((size_t)e * ng + n) * neq + q] = nodal[(size_t)c->el_nodes[(size_t)e * ng + n] * neq + q];
  const VtkCell cell = vtk_cell(G);
  const int nv = (int)cell.xi.size() / 2;
  std::string o;
  grid(o, c, cell, precision);
  auto nm = names_or(names, neq, default_fields(c));
  auto pv = at_nodes(v, E, ICX_BASIS_LAGRANGE, G, neq, cell);
  for (int q = 0; q < neq; ++q) field(o, nm[q], pv, neq, q, E, nv, precision);
  footer(o);
  std::filesystem::path d = dir ? std::filesystem::path(dir) : std::filesystem::current_path() / "iceicle_data";
  if (!make_dir(d)) return io_fail(c, ICX_ERR_INVALID, "cannot create " + d.string());
  std::filesystem::path f =
      d / (std::string(collection ? collection : "mdg_residuals") + std::to_string(itime) + ".vtu");
  if (!write_file(f, o)) return io_fail(c, ICX_ERR_INVALID, "cannot write " + f.string());
  return ICX_OK;
}

}  // extern "C"
