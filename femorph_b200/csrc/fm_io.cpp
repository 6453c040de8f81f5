// .dat keyword reader and legacy-VTK writer with the reference's formats.
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "fm_internal.hpp"

using namespace fm;

namespace {

std::string upper(std::string s) {
  for (auto& c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}

// boost::trim + boost::split(is_any_of(" ,"), token_compress_on) as used by
// femModel::ReadFromFEMTextFile (femModel.cpp:3790-3794).
void tokenize(const std::string& line, std::vector<std::string>& tok) {
  tok.clear();
  size_t b = 0, e = line.size();
  while (b < e && std::isspace((unsigned char)line[b])) ++b;
  while (e > b && std::isspace((unsigned char)line[e - 1])) --e;
  std::string cur;
  size_t i = b;
  while (i < e) {
    char c = line[i];
    if (c == ' ' || c == ',') {
      tok.push_back(cur);
      cur.clear();
      while (i < e && (line[i] == ' ' || line[i] == ',')) ++i;
    } else {
      cur.push_back(c);
      ++i;
    }
  }
  tok.push_back(cur);
}

double tokd(const std::vector<std::string>& t, size_t i) { return i < t.size() ? atof(t[i].c_str()) : 0.0; }
int toki(const std::vector<std::string>& t, size_t i) { return i < t.size() ? atoi(t[i].c_str()) : 0; }

}  // namespace

extern "C" int fm_problem_read_dat(const char* path, int32_t solver, int32_t precision, fm_problem** out) {
  if (!path || !out) return fail(FM_ERR_INVALID, "null argument");
  *out = nullptr;
  std::ifstream in(path);
  if (!in) return fail(FM_ERR_IO, std::string("cannot open ") + path);
  std::vector<double> coords, vel_vals, dir_vals, pres_vals;
  std::vector<int32_t> conn, vel_node, vel_dir, dir_node, pres_node;
  int etype = 0;
  fm_params prm;
  memset(&prm, 0, sizeof(prm));
  prm.solver = solver;
  prm.precision = precision;
  bool have_dual = false;
  std::string glob = "NONE";
  std::string line;
  std::vector<std::string> t;
  int64_t lineno = 0;
  while (std::getline(in, line)) {
    ++lineno;
    tokenize(line, t);
    const std::string k = upper(t[0]);
    if (k == "NODE") {
      coords.push_back(tokd(t, 2));
      coords.push_back(tokd(t, 3));
      coords.push_back(tokd(t, 4));
    } else if (k == "ELEMENT") {
      const std::string et = upper(t.size() > 1 ? t[1] : "");
      int npe = et == "TET4" ? 4 : (et == "HEXA8" ? 8 : 0);
      if (!npe) return fail(FM_ERR_INVALID, "line " + std::to_string(lineno) + ": element type " + et +
                                                " is not handled by the explicit flow solvers");
      if (etype && etype != npe) return fail(FM_ERR_INVALID, "mixed element types are not supported");
      etype = npe;
      for (int a = 0; a < npe; ++a) conn.push_back(toki(t, 4 + a) - 1);
    } else if (k == "NODEDIRBC") {
      dir_node.push_back(toki(t, 1) - 1);
      dir_vals.push_back(tokd(t, 2));
      // one value: the reference stores a 1-entry row and setDirichletBC then
      // reads past it; missing components are taken as 0 here.
      dir_vals.push_back(t.size() > 3 ? tokd(t, 3) : 0.0);
      dir_vals.push_back(t.size() > 3 ? tokd(t, 4) : 0.0);
    } else if (k == "NODEVEL") {
      vel_node.push_back(toki(t, 1) - 1);
      for (int c = 0; c < 4; ++c) vel_vals.push_back(tokd(t, 2 + c));
      vel_dir.push_back(t.size() > 6 ? (int32_t)atof(t[6].c_str()) : 6);
    } else if (k == "NODEPRES") {
      pres_node.push_back(toki(t, 1) - 1);
      pres_vals.push_back(tokd(t, 2));
    } else if (k == "NODEDOF") {
      if (t.size() > 2) glob = upper(t[2]);
    } else if (k == "TIMESTEP") {
      prm.time_step = tokd(t, 1);
      prm.total_steps = toki(t, 2);
      prm.save_every = toki(t, 3);
    } else if (k == "DUALSTEP") {
      prm.dual_step = tokd(t, 1);
      prm.tot_dual_steps = toki(t, 2);
      have_dual = true;
    } else if (k == "VMSPROPS") {
      for (int c = 0; c < 5; ++c) prm.props[c] = tokd(t, 1 + c);
    } else if (k == "EXOPTS") {
      for (int c = 0; c < 6; ++c) prm.ex_opts[c] = toki(t, 1 + c) != 0;
    } else if (k == "EXITCOND") {
      prm.exit_condition = tokd(t, 1);
    } else if (k == "SOLVER") {
      const std::string v = upper(t.size() > 1 ? t[1] : "");
      prm.solver = v == "SUPG" ? FM_SOLVER_SUPG : FM_SOLVER_VMS;
    } else if (k == "PRECISION") {
      const std::string v = upper(t.size() > 1 ? t[1] : "");
      prm.precision = v == "MIXED" ? FM_MIXED : FM_FP64;
    }
  }
  if (glob == "NONE") prm.glob_fixed = FM_FIX_NONE;
  else if (glob == "X") prm.glob_fixed = FM_FIX_X;
  else if (glob == "Y") prm.glob_fixed = FM_FIX_Y;
  else if (glob == "Z") prm.glob_fixed = FM_FIX_Z;
  else if (glob == "XY") prm.glob_fixed = FM_FIX_X | FM_FIX_Y;
  else if (glob == "YZ") prm.glob_fixed = FM_FIX_Y | FM_FIX_Z;
  else if (glob == "XZ") prm.glob_fixed = FM_FIX_X | FM_FIX_Z;
  else return fail(FM_ERR_INVALID, "ERROR: Invalid GLOBAL FIXED DOFs String.");
  if (!have_dual) {
    prm.dual_step = prm.time_step;  // uninitialised in the reference; dt is the documented default
    prm.tot_dual_steps = 0;
  }
  fm_mesh m;
  m.elem_type = etype;
  m.n_nodes = (int64_t)coords.size() / 3;
  m.n_elems = etype ? (int64_t)conn.size() / etype : 0;
  m.coords = coords.data();
  m.conn = conn.data();
  fm_bc bc;
  bc.n_vel_rows = (int64_t)vel_node.size();
  bc.vel_node = vel_node.data();
  bc.vel_vals = vel_vals.data();
  bc.vel_dir = vel_dir.data();
  bc.n_dir = (int64_t)dir_node.size();
  bc.dir_node = dir_node.data();
  bc.dir_vals = dir_vals.data();
  bc.n_pres = (int64_t)pres_node.size();
  bc.pres_node = pres_node.data();
  bc.pres_vals = pres_vals.data();
  return fm_problem_create(&m, &bc, &prm, nullptr, out);
}

// femModel::ExportToVTKLegacy (femModel.cpp:1294-1530) for the explicit
// solvers' result lists: VMS writes velocity + pressure (node) and res_v,
// res_p, subgrid_u, subgrid_p (element); SUPG velocity (node) and pressure,
// lambda, regime (element).  res_v/res_p are the reference's diagnostic
// centroid averages of a partially assembled residual (they depend on the
// element loop order and carry no state); they are written as zeros.
extern "C" int fm_problem_write_vtk(fm_problem* p, const char* path) {
  if (!p || !path) return fail(FM_ERR_INVALID, "null argument");
  const int64_t N = p->N, E = p->E;
  const bool vms = p->params.solver == FM_SOLVER_VMS;
  std::vector<double> u(N * 3), pres(vms ? N : E), e3(vms ? E * 3 : E * 2);
  if (p->batch) {
    int r = fm_problem_get_state(p, u.data(), pres.data(), e3.data(), nullptr);
    if (r) return r;
  } else {
    return fail(FM_ERR_INVALID, "problem is not in a batch");
  }
  FILE* f = fopen(path, "w");
  if (!f) return fail(FM_ERR_IO, std::string("cannot open ") + path);
  fprintf(f, "# vtk DataFile Version 2.0\nModel Exported from feMorph\nASCII\nDATASET UNSTRUCTURED_GRID\n");
  fprintf(f, "POINTS %d float\n", (int)N);
  for (int64_t i = 0; i < N; ++i) fprintf(f, "%e %e %e\n", p->coords[i * 3], p->coords[i * 3 + 1], p->coords[i * 3 + 2]);
  const int npe = p->etype;
  fprintf(f, "CELLS %d %d\n", (int)E, (int)(E * (npe + 1)));
  for (int64_t e = 0; e < E; ++e) {
    fprintf(f, "%d ", npe);
    for (int a = 0; a < npe; ++a) fprintf(f, "%d ", p->conn[e * npe + a]);
    fprintf(f, "\n");
  }
  fprintf(f, "CELL_TYPES %d\n", (int)E);
  for (int64_t e = 0; e < E; ++e) fprintf(f, "%d\n", npe == 4 ? 10 : 12);
  fprintf(f, "POINT_DATA %d\n", (int)N);
  fprintf(f, "VECTORS DXYZ double\n");
  for (int64_t i = 0; i < N; ++i) fprintf(f, "%e %e %e\n", 0.0, 0.0, 0.0);
  fprintf(f, "VECTORS velocity double\n");
  for (int64_t i = 0; i < N; ++i) fprintf(f, "%e %e %e \n", u[i * 3], u[i * 3 + 1], u[i * 3 + 2]);
  if (vms) {
    fprintf(f, "SCALARS pressure double 1\nLOOKUP_TABLE default\n");
    for (int64_t i = 0; i < N; ++i) fprintf(f, "%e \n", pres[i]);
  }
  std::vector<double> dirbc(N, 0.0);
  for (int32_t n : p->vel_node) dirbc[n] = 2.0;
  for (int32_t n : p->pres_node) dirbc[n] = 3.0;
  for (int32_t n : p->dir_node) dirbc[n] = 1.0;
  fprintf(f, "SCALARS dirBC double 1\nLOOKUP_TABLE default\n");
  for (int64_t i = 0; i < N; ++i) fprintf(f, "%e\n", dirbc[i]);
  fprintf(f, "SCALARS neuBC double\nLOOKUP_TABLE default\n");
  for (int64_t i = 0; i < N; ++i) fprintf(f, "%e\n", 0.0);
  fprintf(f, "CELL_DATA %d\n", (int)E);
  fprintf(f, "VECTORS normal double\n");
  for (int64_t e = 0; e < E; ++e) fprintf(f, "%e %e %e\n", 0.0, 0.0, 0.0);
  fprintf(f, "SCALARS source double 1\nLOOKUP_TABLE default\n");
  for (int64_t e = 0; e < E; ++e) fprintf(f, "%e\n", 0.0);
  if (vms) {
    fprintf(f, "VECTORS res_v double\n");
    for (int64_t e = 0; e < E; ++e) fprintf(f, "%e %e %e \n", 0.0, 0.0, 0.0);
    fprintf(f, "SCALARS res_p double 1\nLOOKUP_TABLE default\n");
    for (int64_t e = 0; e < E; ++e) fprintf(f, "%e \n", 0.0);
    fprintf(f, "VECTORS subgrid_u double\n");
    for (int64_t e = 0; e < E; ++e) fprintf(f, "%e %e %e \n", e3[e * 3], e3[e * 3 + 1], e3[e * 3 + 2]);
    fprintf(f, "SCALARS subgrid_p double 1\nLOOKUP_TABLE default\n");
    for (int64_t e = 0; e < E; ++e) fprintf(f, "%e \n", 0.0);
  } else {
    fprintf(f, "SCALARS pressure double 1\nLOOKUP_TABLE default\n");
    for (int64_t e = 0; e < E; ++e) fprintf(f, "%e \n", pres[e]);
    fprintf(f, "SCALARS lambda double 1\nLOOKUP_TABLE default\n");
    for (int64_t e = 0; e < E; ++e) fprintf(f, "%e \n", e3[e * 2]);
    fprintf(f, "SCALARS regime double 1\nLOOKUP_TABLE default\n");
    for (int64_t e = 0; e < E; ++e) fprintf(f, "%e \n", e3[e * 2 + 1]);
  }
  fclose(f);
  return FM_OK;
}
