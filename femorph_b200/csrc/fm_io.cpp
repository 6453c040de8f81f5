// .dat keyword reader and legacy-VTK writer with the reference's formats.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cctype>
#include <cerrno>
#include <charconv>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "fm_internal.hpp"

using namespace fm;

namespace {

// A token of a line: [b, e).  The file buffer is NUL-terminated, and every
// token is followed by a separator, a line end or the terminator, so strtod
// and strtol stop at the token's end as atof / atoi on the token would.
struct Tok {
  const char* b = nullptr;
  const char* e = nullptr;
};

// boost::trim + boost::split(is_any_of(" ,"), token_compress_on) on one line
// (femModel::ReadFromFEMTextFile, femModel.cpp:3790-3794); returns the
// number of tokens (at least 1; tokens beyond maxtok are counted, not kept).
int split_line(const char* b, const char* e, Tok* tok, int maxtok) {
  while (b < e && std::isspace((unsigned char)*b)) ++b;
  while (e > b && std::isspace((unsigned char)e[-1])) --e;
  int n = 0;
  const char* cur = b;
  const char* i = b;
  while (i < e) {
    if (*i == ' ' || *i == ',') {
      if (n < maxtok) tok[n] = {cur, i};
      ++n;
      while (i < e && (*i == ' ' || *i == ',')) ++i;
      cur = i;
    } else {
      ++i;
    }
  }
  if (n < maxtok) tok[n] = {cur, e};
  return n + 1;
}

bool tok_is(const Tok& t, const char* kw) {  // case-insensitive equality
  const size_t n = strlen(kw);
  if ((size_t)(t.e - t.b) != n) return false;
  for (size_t i = 0; i < n; ++i)
    if (std::toupper((unsigned char)t.b[i]) != kw[i]) return false;
  return true;
}
std::string tok_upper(const Tok& t) {
  std::string s(t.b, t.e);
  for (auto& c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}
// A token's number as strtod / strtol read it from the token's start.  A
// token that is exactly a finite decimal number in std::from_chars's grammar
// (no '+', no hex) takes that path, whose result is the same correctly
// rounded value; a token of at most nine digits after an optional '-' is
// summed directly; every other token goes through strtod / strtol.
double tok_dbl(const Tok& t) {
  double v = 0.0;
  const auto r = std::from_chars(t.b, t.e, v);
  if (r.ec == std::errc() && r.ptr == t.e && std::isfinite(v)) return v;
  return strtod(t.b, nullptr);
}
int tok_int(const Tok& t) {
  const char* q = t.b + (t.b < t.e && *t.b == '-');
  const ptrdiff_t nd = t.e - q;
  if (nd >= 1 && nd <= 9) {
    int v = 0;
    for (; q < t.e && *q >= '0' && *q <= '9'; ++q) v = v * 10 + (*q - '0');
    if (q == t.e) return *t.b == '-' ? -v : v;
  }
  return (int)strtol(t.b, nullptr, 10);
}
double tdbl(const Tok* t, int n, int i) { return i < n ? tok_dbl(t[i]) : 0.0; }
int tint(const Tok* t, int n, int i) { return i < n ? tok_int(t[i]) : 0; }

// The whole file in a NUL-terminated host buffer, read in pieces by the host
// threads (pread; the buffer is not zero-filled first).
int read_file(const char* path, hvec<char>& buf) {
  const int fd = open(path, O_RDONLY);
  if (fd < 0) return fail(FM_ERR_IO, std::string("cannot open ") + path);
  struct stat st;
  if (fstat(fd, &st) != 0) {
    close(fd);
    return fail(FM_ERR_IO, std::string("cannot read ") + path);
  }
  const int64_t size = std::max<int64_t>(0, (int64_t)st.st_size);
  buf.resize((size_t)size + 1);
  std::atomic<bool> ok{true};
  parallel_blocks(size, [&](int64_t b, int64_t e, int) {
    while (b < e) {
      const ssize_t r = pread(fd, buf.data() + b, (size_t)(e - b), (off_t)b);
      if (r < 0 && errno == EINTR) continue;
      if (r <= 0) {
        ok = false;
        return;
      }
      b += r;
    }
  }, 1 << 22);
  close(fd);
  buf[(size_t)size] = '\0';
  if (!ok) return fail(FM_ERR_IO, std::string("cannot read ") + path);
  return FM_OK;
}

// Everything one block of lines contributes, in line order.
struct DatBlock {
  std::vector<double> coords, vel_vals, dir_vals, pres_vals;
  std::vector<int32_t> conn, vel_node, vel_dir, dir_node, pres_node;
  // Poisson keywords (femModel.cpp:3909-3925, 3999-4011, 4185-4200)
  std::vector<double> diff, src_val, neu_val;
  std::vector<int32_t> src_el, neu_cnt, neu_nodes;
  int etype = 0;
  int64_t etype_line = -1;              // first ELEMENT line of a handled type (block-local)
  int64_t change_line = -1;             // first ELEMENT line whose type differs from etype
  int64_t bad_line = -1;                // first ELEMENT line of an unhandled type
  std::string bad_type;
  std::vector<std::pair<int64_t, std::vector<std::string>>> scalars;  // (local line, upper-cased tokens)
  int64_t lines = 0;
};

void parse_block(const char* b, const char* e, DatBlock& B) {
  constexpr int MT = 16;
  Tok t[MT];
  const char* line = b;
  while (line < e) {
    const char* le = (const char*)memchr(line, '\n', (size_t)(e - line));
    if (!le) le = e;
    const int n = split_line(line, le, t, MT);
    const int nt = n < MT ? n : MT;
    const int64_t ln = B.lines++;
    if (tok_is(t[0], "NODE")) {
      B.coords.push_back(tdbl(t, nt, 2));
      B.coords.push_back(tdbl(t, nt, 3));
      B.coords.push_back(tdbl(t, nt, 4));
    } else if (tok_is(t[0], "ELEMENT")) {
      const int npe = (nt > 1 && tok_is(t[1], "TET4")) ? 4 : ((nt > 1 && tok_is(t[1], "HEXA8")) ? 8 : 0);
      if (!npe) {
        if (B.bad_line < 0) {
          B.bad_line = ln;
          B.bad_type = nt > 1 ? tok_upper(t[1]) : std::string();
        }
      } else {
        if (!B.etype) {
          B.etype = npe;
          B.etype_line = ln;
        } else if (B.etype != npe && B.change_line < 0) {
          B.change_line = ln;
        }
        for (int a = 0; a < npe; ++a) B.conn.push_back(tint(t, nt, 4 + a) - 1);
      }
    } else if (tok_is(t[0], "NODEDIRBC")) {
      B.dir_node.push_back(tint(t, nt, 1) - 1);
      B.dir_vals.push_back(tdbl(t, nt, 2));
      // one value: the reference stores a 1-entry row and setDirichletBC then
      // reads past it; missing components are taken as 0 here.
      B.dir_vals.push_back(n > 3 ? tdbl(t, nt, 3) : 0.0);
      B.dir_vals.push_back(n > 3 ? tdbl(t, nt, 4) : 0.0);
    } else if (tok_is(t[0], "NODEVEL")) {
      B.vel_node.push_back(tint(t, nt, 1) - 1);
      for (int c = 0; c < 4; ++c) B.vel_vals.push_back(tdbl(t, nt, 2 + c));
      B.vel_dir.push_back(n > 6 ? (int32_t)tdbl(t, nt, 6) : 6);
    } else if (tok_is(t[0], "NODEPRES")) {
      B.pres_node.push_back(tint(t, nt, 1) - 1);
      B.pres_vals.push_back(tdbl(t, nt, 2));
    } else if (tok_is(t[0], "ELDIFF")) {
      // rows are kept in file order whatever their element number, as the
      // reference's reader does (femModel.cpp:3909-3925)
      for (int c = 0; c < 3; ++c) B.diff.push_back(tdbl(t, nt, 2 + c));
    } else if (tok_is(t[0], "ELSOURCE")) {
      B.src_el.push_back(tint(t, nt, 1) - 1);
      B.src_val.push_back(tdbl(t, nt, 2));
    } else if (tok_is(t[0], "FACENEUMANN")) {
      // element, face nodes..., value (femModel.cpp:4185-4200)
      const int k = std::max(0, std::min(n, MT) - 3);
      for (int i = 0; i < k; ++i) B.neu_nodes.push_back(tint(t, nt, 2 + i) - 1);
      B.neu_cnt.push_back(k);
      B.neu_val.push_back(n <= MT ? tdbl(t, nt, n - 1) : 0.0);
    } else if (tok_is(t[0], "NODEDOF") || tok_is(t[0], "TIMESTEP") || tok_is(t[0], "DUALSTEP") ||
               tok_is(t[0], "VMSPROPS") || tok_is(t[0], "EXOPTS") || tok_is(t[0], "EXITCOND") ||
               tok_is(t[0], "SOLVER") || tok_is(t[0], "PRECISION") || tok_is(t[0], "PROBLEM")) {
      std::vector<std::string> v;
      for (int i = 0; i < nt; ++i) v.emplace_back(t[i].b, t[i].e);
      v[0] = tok_upper(t[0]);
      B.scalars.emplace_back(ln, std::move(v));
    }
    line = le + 1;
  }
}

// One array of every block, in block order, into dst: sized once, the blocks
// copied on their own threads and released.
template <class T, class Get>
void join_blocks(std::vector<DatBlock>& blk, Get get, hvec<T>& dst) {
  std::vector<size_t> off(blk.size() + 1, 0);
  for (size_t k = 0; k < blk.size(); ++k) off[k + 1] = off[k] + get(blk[k]).size();
  dst.resize(off.back());
  std::vector<std::thread> th;
  for (size_t k = 0; k < blk.size(); ++k)
    th.emplace_back([&, k] {
      std::vector<T>& v = get(blk[k]);
      std::copy(v.begin(), v.end(), dst.begin() + (std::ptrdiff_t)off[k]);
      std::vector<T>().swap(v);
    });
  for (auto& x : th) x.join();
}

}  // namespace

// Reads the whole file, cuts it at line ends into one block per host thread,
// parses the blocks in parallel and joins them in file order (keyword rows
// keep their order; for the single-valued keywords the last line wins, as in
// the reference's sequential reader).
extern "C" int fm_problem_read_dat(const char* path, int32_t solver, int32_t precision, fm_problem** out) {
  NvtxRange nvtx_range("fm_problem_read_dat");
  if (!path || !out) return fail(FM_ERR_INVALID, "null argument");
  *out = nullptr;
  hvec<char> buf;
  if (int r = read_file(path, buf)) return r;
  const char* base = buf.data();
  const int64_t len = (int64_t)buf.size() - 1;
  const int64_t hw = std::max<int64_t>(1, std::min<int64_t>(32, std::thread::hardware_concurrency()));
  const int64_t nb = std::min<int64_t>(hw, std::max<int64_t>(1, len / (1 << 20)));
  std::vector<int64_t> cut(nb + 1, 0);
  cut[nb] = len;
  for (int64_t k = 1; k < nb; ++k) {
    int64_t c = std::max(cut[k - 1], len * k / nb);
    while (c < len && base[c - 1] != '\n') ++c;  // start of a line
    cut[k] = c;
  }
  std::vector<DatBlock> blk(nb);
  {
    std::vector<std::thread> th;
    for (int64_t k = 0; k < nb; ++k)
      th.emplace_back([&, k] { parse_block(base + cut[k], base + cut[k + 1], blk[k]); });
    for (auto& x : th) x.join();
  }
  std::vector<double> vel_vals, dir_vals, pres_vals;
  std::vector<int32_t> vel_node, vel_dir, dir_node, pres_node;
  int etype = 0;
  fm_params prm;
  memset(&prm, 0, sizeof(prm));
  prm.solver = solver;
  prm.precision = precision;
  bool have_dual = false;
  std::string glob = "NONE";
  int64_t line0 = 0;
  auto cat = [](auto& dst, const auto& src) { dst.insert(dst.end(), src.begin(), src.end()); };
  for (int64_t k = 0; k < nb; ++k) {
    DatBlock& B = blk[k];
    // the first element-type problem in file order, as the sequential reader meets it
    const int64_t INF = INT64_MAX;
    int64_t at_mix = B.change_line >= 0 ? B.change_line : INF;
    if (B.etype && etype && B.etype != etype) at_mix = std::min(at_mix, B.etype_line);
    const int64_t at_bad = B.bad_line >= 0 ? B.bad_line : INF;
    if (at_bad < at_mix)
      return fail(FM_ERR_INVALID, "line " + std::to_string(line0 + at_bad + 1) + ": element type " + B.bad_type +
                                      " is not handled by the explicit flow solvers");
    if (at_mix < INF) return fail(FM_ERR_INVALID, "mixed element types are not supported");
    if (B.etype) etype = B.etype;
    cat(vel_node, B.vel_node); cat(vel_vals, B.vel_vals); cat(vel_dir, B.vel_dir);
    cat(dir_node, B.dir_node); cat(dir_vals, B.dir_vals);
    cat(pres_node, B.pres_node); cat(pres_vals, B.pres_vals);
    for (auto& sc : B.scalars) {
      const std::vector<std::string>& t = sc.second;
      const int n = (int)t.size();
      auto d = [&](int i) { return i < n ? atof(t[i].c_str()) : 0.0; };
      auto in = [&](int i) { return i < n ? atoi(t[i].c_str()) : 0; };
      const std::string& kw = t[0];
      if (kw == "NODEDOF") {
        if (n > 2) {
          glob = t[2];
          for (auto& c : glob) c = (char)std::toupper((unsigned char)c);
        }
      } else if (kw == "TIMESTEP") {
        prm.time_step = d(1);
        prm.total_steps = in(2);
        prm.save_every = in(3);
      } else if (kw == "DUALSTEP") {
        prm.dual_step = d(1);
        prm.tot_dual_steps = in(2);
        have_dual = true;
      } else if (kw == "VMSPROPS") {
        for (int c = 0; c < 5; ++c) prm.props[c] = d(1 + c);
      } else if (kw == "EXOPTS") {
        for (int c = 0; c < 6; ++c) prm.ex_opts[c] = in(1 + c) != 0;
      } else if (kw == "EXITCOND") {
        prm.exit_condition = d(1);
      } else if (kw == "SOLVER") {
        std::string v = n > 1 ? t[1] : "";
        for (auto& c : v) c = (char)std::toupper((unsigned char)c);
        prm.solver = v == "SUPG" ? FM_SOLVER_SUPG : FM_SOLVER_VMS;
      } else if (kw == "PRECISION") {
        std::string v = n > 1 ? t[1] : "";
        for (auto& c : v) c = (char)std::toupper((unsigned char)c);
        prm.precision = v == "MIXED" ? FM_MIXED : FM_FP64;
      }
    }
    line0 += B.lines;
  }
  hvec<double> coords;
  hvec<int32_t> conn;
  join_blocks(blk, [](DatBlock& B) -> std::vector<double>& { return B.coords; }, coords);
  join_blocks(blk, [](DatBlock& B) -> std::vector<int32_t>& { return B.conn; }, conn);
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
namespace {

// printf("%e") of a double, byte for byte: std::to_chars in scientific form
// with six digits gives the same correctly rounded digits and layout for
// finite values; the others go through snprintf.
inline char* put_e(char* b, double v) {
  if (std::isfinite(v)) return std::to_chars(b, b + 32, v, std::chars_format::scientific, 6).ptr;
  return b + snprintf(b, 32, "%e", v);
}
inline char* put_d(char* b, int v) { return std::to_chars(b, b + 16, v).ptr; }
// "%e<end>" and "%e %e %e<end>" rows (end: "\n" or " \n"); returns the length.
inline int put_e1(char* b, double v, const char* end) {
  char* q = put_e(b, v);
  while (*end) *q++ = *end++;
  return (int)(q - b);
}
inline int put_e3(char* b, const double* v, const char* end) {
  char* q = put_e(b, v[0]);
  *q++ = ' ';
  q = put_e(q, v[1]);
  *q++ = ' ';
  q = put_e(q, v[2]);
  while (*end) *q++ = *end++;
  return (int)(q - b);
}

// n copies of one row (a section of constant values), written in large
// pieces.
void write_const_rows(FILE* f, int64_t n, const std::string& row) {
  const int64_t per = std::max<int64_t>(1, (1 << 20) / (int64_t)std::max<size_t>(1, row.size()));
  std::string chunk;
  chunk.reserve((size_t)std::min(n, per) * row.size());
  for (int64_t k = 0; k < std::min(n, per); ++k) chunk += row;
  for (int64_t done = 0; done < n; done += per) {
    const int64_t m = std::min(per, n - done);
    fwrite(chunk.data(), 1, (size_t)m * row.size(), f);
  }
}
// The row printf writes for this format and these values.
template <class... A>
std::string row_of(const char* fmt, A... a) {
  char b[256];
  const int k = snprintf(b, sizeof(b), fmt, a...);
  return std::string(b, (size_t)k);
}

// The state the writers export: the device state of a problem in a batch;
// a problem not yet stepped outside a batch exports the initial state given
// at fm_problem_create (zeros without one; Dirichlet values are applied at
// placement) with zero element fields.
int writer_state(fm_problem* p, std::vector<double>& u, std::vector<double>& pres, std::vector<double>& e3) {
  const int64_t N = p->N, E = p->E;
  const bool vms = p->params.solver == FM_SOLVER_VMS;
  u.assign((size_t)N * 3, 0.0);
  pres.assign((size_t)(vms ? N : E), 0.0);
  e3.assign((size_t)(vms ? E * 3 : E * 2), 0.0);
  if (p->batch) return fm_problem_get_state(p, u.data(), pres.data(), e3.data(), nullptr);
  if (p->steps_done > 0) return fail(FM_ERR_INVALID, "the problem left its batch after stepping: its state is gone");
  if (!p->init.empty())
    for (int64_t i = 0; i < N; ++i) {
      for (int k = 0; k < 3; ++k) u[i * 3 + k] = p->init[i * 4 + k];
      if (vms) pres[i] = p->init[i * 4 + 3];
    }
  return FM_OK;
}

// Writes rows 0..n-1, row i formatted by fmt(i, buf) (returns its length,
// < 256), formatting blocks of rows on host threads and writing the blocks
// in order: the bytes are those of the sequential fprintf loop.
template <class F>
void write_rows(FILE* f, int64_t n, F fmt) {
  const int64_t hw = std::max<int64_t>(1, std::min<int64_t>(32, std::thread::hardware_concurrency()));
  const int64_t nb = std::min<int64_t>(hw * 4, std::max<int64_t>(1, n / 65536));
  std::vector<std::string> out(nb);
  auto work = [&](int64_t k) {
    std::string& o = out[k];
    char buf[256];
    for (int64_t i = n * k / nb; i < n * (k + 1) / nb; ++i) o.append(buf, (size_t)fmt(i, buf));
  };
  if (nb == 1) {
    work(0);
  } else {
    std::vector<std::thread> th;
    const int64_t nt = std::min<int64_t>(hw, nb);
    for (int64_t w = 0; w < nt; ++w)
      th.emplace_back([&, w] {
        for (int64_t k = w; k < nb; k += nt) work(k);
      });
    for (auto& x : th) x.join();
  }
  for (auto& o : out) fwrite(o.data(), 1, o.size(), f);
}

}  // namespace

// femModel::ExportToVTKLegacy (femModel.cpp:1294-1530) for the explicit
// solvers' result lists: VMS writes velocity + pressure (node) and res_v,
// res_p, subgrid_u, subgrid_p (element); SUPG velocity (node) and pressure,
// lambda, regime (element).  res_v/res_p are the reference's diagnostic
// centroid averages of a partially assembled residual (they depend on the
// element loop order and carry no state); they are written as zeros.  The
// rows are formatted on the host threads (write_rows).
extern "C" int fm_problem_write_vtk(fm_problem* p, const char* path) {
  NvtxRange nvtx_range("fm_problem_write_vtk");
  if (!p || !path) return fail(FM_ERR_INVALID, "null argument");
  const int64_t N = p->N, E = p->E;
  const bool vms = p->params.solver == FM_SOLVER_VMS;
  std::vector<double> u, pres, e3;
  if (int r = writer_state(p, u, pres, e3)) return r;
  FILE* f = fopen(path, "w");
  if (!f) return fail(FM_ERR_IO, std::string("cannot open ") + path);
  const double* X = p->coords.data();
  const int npe = p->etype;
  const int32_t* cn = p->conn.data();
  fprintf(f, "# vtk DataFile Version 2.0\nModel Exported from feMorph\nASCII\nDATASET UNSTRUCTURED_GRID\n");
  fprintf(f, "POINTS %d float\n", (int)N);
  write_rows(f, N, [&](int64_t i, char* b) { return put_e3(b, X + i * 3, "\n"); });
  fprintf(f, "CELLS %d %d\n", (int)E, (int)(E * (npe + 1)));
  write_rows(f, E, [&](int64_t e, char* b) {
    char* q = put_d(b, npe);
    *q++ = ' ';
    for (int a = 0; a < npe; ++a) {
      q = put_d(q, cn[e * npe + a]);
      *q++ = ' ';
    }
    *q++ = '\n';
    return (int)(q - b);
  });
  fprintf(f, "CELL_TYPES %d\n", (int)E);
  const int ctype = npe == 4 ? 10 : 12;
  write_const_rows(f, E, row_of("%d\n", ctype));
  fprintf(f, "POINT_DATA %d\n", (int)N);
  fprintf(f, "VECTORS DXYZ double\n");
  write_const_rows(f, N, row_of("%e %e %e\n", 0.0, 0.0, 0.0));
  fprintf(f, "VECTORS velocity double\n");
  write_rows(f, N, [&](int64_t i, char* b) { return put_e3(b, u.data() + i * 3, " \n"); });
  if (vms) {
    fprintf(f, "SCALARS pressure double 1\nLOOKUP_TABLE default\n");
    write_rows(f, N, [&](int64_t i, char* b) { return put_e1(b, pres[i], " \n"); });
  }
  std::vector<double> dirbc(N, 0.0);
  for (int32_t n : p->vel_node) dirbc[n] = 2.0;
  for (int32_t n : p->pres_node) dirbc[n] = 3.0;
  for (int32_t n : p->dir_node) dirbc[n] = 1.0;
  fprintf(f, "SCALARS dirBC double 1\nLOOKUP_TABLE default\n");
  write_rows(f, N, [&](int64_t i, char* b) { return put_e1(b, dirbc[i], "\n"); });
  fprintf(f, "SCALARS neuBC double\nLOOKUP_TABLE default\n");
  write_const_rows(f, N, row_of("%e\n", 0.0));
  fprintf(f, "CELL_DATA %d\n", (int)E);
  fprintf(f, "VECTORS normal double\n");
  write_const_rows(f, E, row_of("%e %e %e\n", 0.0, 0.0, 0.0));
  fprintf(f, "SCALARS source double 1\nLOOKUP_TABLE default\n");
  write_const_rows(f, E, row_of("%e\n", 0.0));
  if (vms) {
    fprintf(f, "VECTORS res_v double\n");
    write_const_rows(f, E, row_of("%e %e %e \n", 0.0, 0.0, 0.0));
    fprintf(f, "SCALARS res_p double 1\nLOOKUP_TABLE default\n");
    write_const_rows(f, E, row_of("%e \n", 0.0));
    fprintf(f, "VECTORS subgrid_u double\n");
    write_rows(f, E, [&](int64_t e, char* b) { return put_e3(b, e3.data() + e * 3, " \n"); });
    fprintf(f, "SCALARS subgrid_p double 1\nLOOKUP_TABLE default\n");
    write_const_rows(f, E, row_of("%e \n", 0.0));
  } else {
    fprintf(f, "SCALARS pressure double 1\nLOOKUP_TABLE default\n");
    write_rows(f, E, [&](int64_t e, char* b) { return put_e1(b, pres[e], " \n"); });
    fprintf(f, "SCALARS lambda double 1\nLOOKUP_TABLE default\n");
    write_rows(f, E, [&](int64_t e, char* b) { return put_e1(b, e3[e * 2], " \n"); });
    fprintf(f, "SCALARS regime double 1\nLOOKUP_TABLE default\n");
    write_rows(f, E, [&](int64_t e, char* b) { return put_e1(b, e3[e * 2 + 1], " \n"); });
  }
  const bool ok = ferror(f) == 0;
  fclose(f);
  return ok ? FM_OK : fail(FM_ERR_IO, std::string("cannot write ") + path);
}

namespace {

// Big-endian copies for legacy binary VTK, converted on host threads.
template <class T>
void put_be(FILE* f, const T* v, int64_t n) {
  hvec<T> o((size_t)n);
  const int64_t hw = std::max<int64_t>(1, std::min<int64_t>(32, std::thread::hardware_concurrency()));
  const int64_t nt = std::min<int64_t>(hw, std::max<int64_t>(1, n / 65536));
  std::vector<std::thread> th;
  for (int64_t w = 0; w < nt; ++w)
    th.emplace_back([&, w] {
      for (int64_t i = n * w / nt; i < n * (w + 1) / nt; ++i) {
        unsigned char b[sizeof(T)];
        memcpy(b, &v[i], sizeof(T));
        std::reverse(b, b + sizeof(T));
        memcpy(&o[i], b, sizeof(T));
      }
    });
  for (auto& x : th) x.join();
  fwrite(o.data(), sizeof(T), (size_t)n, f);
}

// `bytes` zero bytes (the big-endian form of a section of zeros).
void put_zeros(FILE* f, int64_t bytes) {
  static const char z[1 << 16] = {};
  while (bytes > 0) {
    const size_t m = (size_t)std::min<int64_t>(bytes, (int64_t)sizeof(z));
    fwrite(z, 1, m, f);
    bytes -= (int64_t)m;
  }
}

}  // namespace

// The layout of fm_problem_write_vtk in legacy BINARY form (big-endian
// float32 points, int32 cells and types, float64 data): the same sections
// and names, an order of magnitude smaller and faster to write than the
// ASCII %e text at the benchmark sizes.  No counterpart in the reference,
// which writes ASCII only.
extern "C" int fm_problem_write_vtk_binary(fm_problem* p, const char* path) {
  NvtxRange nvtx_range("fm_problem_write_vtk_binary");
  if (!p || !path) return fail(FM_ERR_INVALID, "null argument");
  const int64_t N = p->N, E = p->E;
  const bool vms = p->params.solver == FM_SOLVER_VMS;
  std::vector<double> u, pres, e3;
  if (int r = writer_state(p, u, pres, e3)) return r;
  FILE* f = fopen(path, "wb");
  if (!f) return fail(FM_ERR_IO, std::string("cannot open ") + path);
  const int npe = p->etype;
  fprintf(f, "# vtk DataFile Version 2.0\nModel Exported from feMorph\nBINARY\nDATASET UNSTRUCTURED_GRID\n");
  fprintf(f, "POINTS %d float\n", (int)N);
  {
    std::vector<float> x((size_t)N * 3);
    for (int64_t i = 0; i < N * 3; ++i) x[i] = (float)p->coords[i];
    put_be(f, x.data(), N * 3);
  }
  fprintf(f, "\nCELLS %d %d\n", (int)E, (int)(E * (npe + 1)));
  {
    hvec<int32_t> c((size_t)E * (npe + 1));
    parallel_blocks(E, [&](int64_t eb, int64_t ee, int) {
      for (int64_t e = eb; e < ee; ++e) {
        c[e * (npe + 1)] = npe;
        for (int a = 0; a < npe; ++a) c[e * (npe + 1) + 1 + a] = p->conn[e * npe + a];
      }
    }, 1 << 16);
    put_be(f, c.data(), (int64_t)c.size());
  }
  fprintf(f, "\nCELL_TYPES %d\n", (int)E);
  {
    std::vector<int32_t> t((size_t)E, npe == 4 ? 10 : 12);
    put_be(f, t.data(), E);
  }
  // v == nullptr: a section of zeros
  auto vec = [&](const char* name, const double* v, int64_t n) {
    fprintf(f, "\nVECTORS %s double\n", name);
    if (v) put_be(f, v, n * 3);
    else put_zeros(f, n * 3 * (int64_t)sizeof(double));
  };
  auto sca = [&](const char* name, const double* v, int64_t n) {
    fprintf(f, "\nSCALARS %s double 1\nLOOKUP_TABLE default\n", name);
    if (v) put_be(f, v, n);
    else put_zeros(f, n * (int64_t)sizeof(double));
  };
  fprintf(f, "\nPOINT_DATA %d", (int)N);
  vec("DXYZ", nullptr, N);
  vec("velocity", u.data(), N);
  if (vms) sca("pressure", pres.data(), N);
  std::vector<double> dirbc(N, 0.0);
  for (int32_t n : p->vel_node) dirbc[n] = 2.0;
  for (int32_t n : p->pres_node) dirbc[n] = 3.0;
  for (int32_t n : p->dir_node) dirbc[n] = 1.0;
  sca("dirBC", dirbc.data(), N);
  sca("neuBC", nullptr, N);
  fprintf(f, "\nCELL_DATA %d", (int)E);
  vec("normal", nullptr, E);
  sca("source", nullptr, E);
  if (vms) {
    vec("res_v", nullptr, E);
    sca("res_p", nullptr, E);
    vec("subgrid_u", e3.data(), E);
    sca("subgrid_p", nullptr, E);
  } else {
    std::vector<double> lam(E), reg(E);
    for (int64_t e = 0; e < E; ++e) {
      lam[e] = e3[e * 2];
      reg[e] = e3[e * 2 + 1];
    }
    sca("pressure", pres.data(), E);
    sca("lambda", lam.data(), E);
    sca("regime", reg.data(), E);
  }
  fprintf(f, "\n");
  const bool ok = ferror(f) == 0;
  fclose(f);
  return ok ? FM_OK : fail(FM_ERR_IO, std::string("cannot write ") + path);
}

// VTK XML UnstructuredGrid (.vtu) with the arrays raw-appended
// (little-endian, UInt64 block sizes): the sections of the legacy writers,
// FP64 points and data, int32 connectivity, read by ParaView and VTK without
// any text parsing.  No counterpart in the reference (ASCII legacy VTK only).
extern "C" int fm_problem_write_vtu(fm_problem* p, const char* path) {
  NvtxRange nvtx_range("fm_problem_write_vtu");
  static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "the VTU writer emits little-endian data");
  if (!p || !path) return fail(FM_ERR_INVALID, "null argument");
  const int64_t N = p->N, E = p->E;
  const int npe = p->etype;
  const bool vms = p->params.solver == FM_SOLVER_VMS;
  std::vector<double> u, pres, e3;
  if (int r = writer_state(p, u, pres, e3)) return r;
  std::vector<double> dirbc(N, 0.0), lam, reg;
  for (int32_t n : p->vel_node) dirbc[n] = 2.0;
  for (int32_t n : p->pres_node) dirbc[n] = 3.0;
  for (int32_t n : p->dir_node) dirbc[n] = 1.0;
  if (!vms) {
    lam.resize(E);
    reg.resize(E);
    for (int64_t e = 0; e < E; ++e) {
      lam[e] = e3[e * 2];
      reg[e] = e3[e * 2 + 1];
    }
  }
  std::vector<int32_t> offs(E);
  for (int64_t e = 0; e < E; ++e) offs[e] = (int32_t)((e + 1) * npe);
  std::vector<uint8_t> types(E, npe == 4 ? 10 : 12);
  struct Block {
    std::string xml;  // DataArray attributes, without the offset
    const void* data;
    uint64_t bytes;
  };
  auto arr = [](const char* type, const char* name, int comps, const void* d, uint64_t bytes) {
    std::string a = std::string("type=\"") + type + "\"";
    if (name) a += std::string(" Name=\"") + name + "\"";
    if (comps > 1) a += " NumberOfComponents=\"" + std::to_string(comps) + "\"";
    return Block{a, d, bytes};
  };
  std::vector<Block> pd, cd, pts, cells;
  const uint64_t n8 = (uint64_t)N * 8, e8 = (uint64_t)E * 8;
  pd.push_back(arr("Float64", "DXYZ", 3, nullptr, n8 * 3));
  pd.push_back(arr("Float64", "velocity", 3, u.data(), n8 * 3));
  if (vms) pd.push_back(arr("Float64", "pressure", 1, pres.data(), n8));
  pd.push_back(arr("Float64", "dirBC", 1, dirbc.data(), n8));
  pd.push_back(arr("Float64", "neuBC", 1, nullptr, n8));
  cd.push_back(arr("Float64", "normal", 3, nullptr, e8 * 3));
  cd.push_back(arr("Float64", "source", 1, nullptr, e8));
  if (vms) {
    cd.push_back(arr("Float64", "res_v", 3, nullptr, e8 * 3));
    cd.push_back(arr("Float64", "res_p", 1, nullptr, e8));
    cd.push_back(arr("Float64", "subgrid_u", 3, e3.data(), e8 * 3));
    cd.push_back(arr("Float64", "subgrid_p", 1, nullptr, e8));
  } else {
    cd.push_back(arr("Float64", "pressure", 1, pres.data(), e8));
    cd.push_back(arr("Float64", "lambda", 1, lam.data(), e8));
    cd.push_back(arr("Float64", "regime", 1, reg.data(), e8));
  }
  pts.push_back(arr("Float64", nullptr, 3, p->coords.data(), n8 * 3));
  cells.push_back(arr("Int32", "connectivity", 1, p->conn.data(), (uint64_t)E * npe * 4));
  cells.push_back(arr("Int32", "offsets", 1, offs.data(), (uint64_t)E * 4));
  cells.push_back(arr("UInt8", "types", 1, types.data(), (uint64_t)E));
  FILE* f = fopen(path, "wb");
  if (!f) return fail(FM_ERR_IO, std::string("cannot open ") + path);
  uint64_t off = 0;
  std::vector<const Block*> order;
  auto section = [&](const char* tag, std::vector<Block>& bs) {
    fprintf(f, "      <%s>\n", tag);
    for (const Block& b : bs) {
      fprintf(f, "        <DataArray %s format=\"appended\" offset=\"%llu\"/>\n", b.xml.c_str(),
              (unsigned long long)off);
      off += 8 + b.bytes;
      order.push_back(&b);
    }
    fprintf(f, "      </%s>\n", tag);
  };
  fprintf(f, "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" "
             "byte_order=\"LittleEndian\" header_type=\"UInt64\">\n  <UnstructuredGrid>\n"
             "    <Piece NumberOfPoints=\"%lld\" NumberOfCells=\"%lld\">\n",
          (long long)N, (long long)E);
  section("PointData", pd);
  section("CellData", cd);
  section("Points", pts);
  section("Cells", cells);
  fprintf(f, "    </Piece>\n  </UnstructuredGrid>\n  <AppendedData encoding=\"raw\">\n   _");
  for (const Block* b : order) {
    fwrite(&b->bytes, 8, 1, f);
    if (b->data) fwrite(b->data, 1, b->bytes, f);
    else put_zeros(f, (int64_t)b->bytes);  // a section of zeros
  }
  fprintf(f, "\n  </AppendedData>\n</VTKFile>\n");
  const bool ok = ferror(f) == 0;
  fclose(f);
  return ok ? FM_OK : fail(FM_ERR_IO, std::string("cannot write ") + path);
}

// The Poisson model of a .dat file (the keywords femPoissonSolver::solve
// reads: PROBLEM, NODE, ELEMENT, ELDIFF, ELSOURCE, FACENEUMANN, NODEDIRBC),
// read like fm_problem_read_dat (blocks parsed on the host threads, joined
// in file order), then assembled and uploaded by fm_poisson_create.
extern "C" int fm_poisson_read_dat(const char* path, int32_t device, fm_poisson** out) {
  NvtxRange nvtx_range("fm_poisson_read_dat");
  if (!path || !out) return fail(FM_ERR_INVALID, "null argument");
  *out = nullptr;
  hvec<char> buf;
  if (int r = read_file(path, buf)) return r;
  const char* base = buf.data();
  const int64_t len = (int64_t)buf.size() - 1;
  const int64_t hw = std::max<int64_t>(1, std::min<int64_t>(32, std::thread::hardware_concurrency()));
  const int64_t nb = std::min<int64_t>(hw, std::max<int64_t>(1, len / (1 << 20)));
  std::vector<int64_t> cut(nb + 1, 0);
  cut[nb] = len;
  for (int64_t k = 1; k < nb; ++k) {
    int64_t c = std::max(cut[k - 1], len * k / nb);
    while (c < len && base[c - 1] != '\n') ++c;
    cut[k] = c;
  }
  std::vector<DatBlock> blk(nb);
  {
    std::vector<std::thread> th;
    for (int64_t k = 0; k < nb; ++k)
      th.emplace_back([&, k] { parse_block(base + cut[k], base + cut[k + 1], blk[k]); });
    for (auto& x : th) x.join();
  }
  std::vector<double> src_val, neu_val, dir_val;
  std::vector<int32_t> src_el, neu_off(1, 0), neu_nodes, dir_node;
  int etype = 0, problem = FM_POISSON_CLASSIC;
  auto cat = [](auto& dst, const auto& src) { dst.insert(dst.end(), src.begin(), src.end()); };
  for (int64_t k = 0; k < nb; ++k) {
    const DatBlock& B = blk[k];
    if (B.bad_line >= 0) return fail(FM_ERR_INVALID, "element type " + B.bad_type + " is not handled");
    if (B.change_line >= 0 || (B.etype && etype && B.etype != etype))
      return fail(FM_ERR_INVALID, "mixed element types are not supported");
    if (B.etype) etype = B.etype;
    cat(src_el, B.src_el);
    cat(src_val, B.src_val);
    cat(neu_val, B.neu_val);
    cat(neu_nodes, B.neu_nodes);
    for (int32_t c : B.neu_cnt) neu_off.push_back(neu_off.back() + c);
    cat(dir_node, B.dir_node);
    for (size_t i = 0; i < B.dir_node.size(); ++i) dir_val.push_back(B.dir_vals[3 * i]);
    for (const auto& sc : B.scalars)
      if (sc.second[0] == "PROBLEM") {
        std::string v = sc.second.size() > 1 ? sc.second[1] : "";
        for (auto& c : v) c = (char)std::toupper((unsigned char)c);
        if (v == "POISSON") problem = FM_POISSON_CLASSIC;
        else if (v == "PPE") problem = FM_POISSON_PPE;
        else if (v == "DISTANCE") problem = FM_POISSON_DISTANCE;
        else return fail(FM_ERR_INVALID, "PROBLEM " + v + " is not a Poisson problem");
      }
  }
  hvec<double> coords, diff;
  hvec<int32_t> conn;
  join_blocks(blk, [](DatBlock& B) -> std::vector<double>& { return B.coords; }, coords);
  join_blocks(blk, [](DatBlock& B) -> std::vector<int32_t>& { return B.conn; }, conn);
  join_blocks(blk, [](DatBlock& B) -> std::vector<double>& { return B.diff; }, diff);
  const int64_t E = etype ? (int64_t)conn.size() / etype : 0;
  if ((int64_t)diff.size() < 3 * E) return fail(FM_ERR_INVALID, "fewer ELDIFF rows than elements");
  fm_poisson_desc d;
  d.elem_type = etype;
  d.problem = problem;
  d.n_nodes = (int64_t)coords.size() / 3;
  d.n_elems = E;
  d.coords = coords.data();
  d.conn = conn.data();
  d.diffusivity = diff.data();
  d.n_sources = (int64_t)src_el.size();
  d.source_elem = src_el.data();
  d.source_value = src_val.data();
  d.n_neumann = (int64_t)neu_val.size();
  d.neumann_off = neu_off.data();
  d.neumann_nodes = neu_nodes.data();
  d.neumann_value = neu_val.data();
  d.n_dirichlet = (int64_t)dir_node.size();
  d.dir_node = dir_node.data();
  d.dir_value = dir_val.data();
  return fm_poisson_create(&d, device, out);
}

// femModel::ExportToVTKLegacy (femModel.cpp:1294-1530) for the Poisson
// solver's result list (femSolver.cpp:613-648): POINTS, the connectivity the
// solver used (after FixedElementConnectivities), DXYZ, "PoissonResult",
// dirBC, neuBC; CELL_DATA normal (zeros: the Poisson driver builds no face
// list), diffusivity, source and, for PROBLEM DISTANCE, "cellDistance".
extern "C" int fm_poisson_write_vtk(fm_poisson* s, const char* path) {
  NvtxRange nvtx_range("fm_poisson_write_vtk");
  if (!s || !path) return fail(FM_ERR_INVALID, "null argument");
  const PoissonHostView* v = poisson_host_view(s);
  const int64_t N = v->N, E = v->E;
  const int npe = v->npe;
  std::vector<double> x(N), dist(v->problem == FM_POISSON_DISTANCE ? E : 0);
  int r = fm_poisson_get_solution(s, x.data(), dist.empty() ? nullptr : dist.data());
  if (r) return r;
  FILE* f = fopen(path, "w");
  if (!f) return fail(FM_ERR_IO, std::string("cannot open ") + path);
  const double* X = v->coords;
  const int32_t* cn = v->conn;
  fprintf(f, "# vtk DataFile Version 2.0\nModel Exported from feMorph\nASCII\nDATASET UNSTRUCTURED_GRID\n");
  fprintf(f, "POINTS %d float\n", (int)N);
  write_rows(f, N, [&](int64_t i, char* b) { return snprintf(b, 256, "%e %e %e\n", X[i * 3], X[i * 3 + 1], X[i * 3 + 2]); });
  fprintf(f, "CELLS %d %d\n", (int)E, (int)(E * (npe + 1)));
  write_rows(f, E, [&](int64_t e, char* b) {
    int k = snprintf(b, 256, "%d ", npe);
    for (int a = 0; a < npe; ++a) k += snprintf(b + k, 256 - k, "%d ", cn[e * npe + a]);
    k += snprintf(b + k, 256 - k, "\n");
    return k;
  });
  fprintf(f, "CELL_TYPES %d\n", (int)E);
  const int ctype = npe == 4 ? 10 : 12;
  write_rows(f, E, [&](int64_t, char* b) { return snprintf(b, 256, "%d\n", ctype); });
  fprintf(f, "POINT_DATA %d\n", (int)N);
  fprintf(f, "VECTORS DXYZ double\n");
  write_rows(f, N, [&](int64_t, char* b) { return snprintf(b, 256, "%e %e %e\n", 0.0, 0.0, 0.0); });
  fprintf(f, "SCALARS PoissonResult double 1\nLOOKUP_TABLE default\n");
  write_rows(f, N, [&](int64_t i, char* b) { return snprintf(b, 256, "%e \n", x[i]); });
  fprintf(f, "SCALARS dirBC double 1\nLOOKUP_TABLE default\n");
  write_rows(f, N, [&](int64_t i, char* b) { return snprintf(b, 256, "%e\n", v->dir[i]); });
  fprintf(f, "SCALARS neuBC double\nLOOKUP_TABLE default\n");
  write_rows(f, N, [&](int64_t i, char* b) { return snprintf(b, 256, "%e\n", v->neu[i]); });
  fprintf(f, "CELL_DATA %d\n", (int)E);
  fprintf(f, "VECTORS normal double\n");
  write_rows(f, E, [&](int64_t, char* b) { return snprintf(b, 256, "%e %e %e\n", 0.0, 0.0, 0.0); });
  fprintf(f, "VECTORS diffusivity double\n");
  write_rows(f, E, [&](int64_t e, char* b) {
    return snprintf(b, 256, "%e %e %e\n", v->diff[e * 3], v->diff[e * 3 + 1], v->diff[e * 3 + 2]);
  });
  fprintf(f, "SCALARS source double 1\nLOOKUP_TABLE default\n");
  write_rows(f, E, [&](int64_t e, char* b) { return snprintf(b, 256, "%e\n", v->src[e]); });
  if (!dist.empty()) {
    fprintf(f, "SCALARS cellDistance double 1\nLOOKUP_TABLE default\n");
    write_rows(f, E, [&](int64_t e, char* b) { return snprintf(b, 256, "%e \n", dist[e]); });
  }
  const bool ok = ferror(f) == 0;
  fclose(f);
  return ok ? FM_OK : fail(FM_ERR_IO, std::string("cannot write ") + path);
}
