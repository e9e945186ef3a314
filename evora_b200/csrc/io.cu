// io.cu -- the reference's file formats for the hydro state (host code):
// dump files, unit files, in-run snapshots and the post-processor's cuts and
// slices.  The text is produced with the edit descriptors of fortran_fmt.h;
// the arithmetic that feeds it (pressure, temperature, the state vector) is
// the reference's FP64 arithmetic in its operation order.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/evora_gpu.h"
#include "../../include/evora_io.h"
#include "chemistry.cuh"
#include "common.h"
#include "cosmology.cuh"
#include "fortran_fmt.h"

namespace evora {
namespace {

namespace ft = fortran;

// ---------------------------------------------------------------- files --
bool write_file(const std::string& path, const std::string& text, bool append) {
  std::FILE* f = std::fopen(path.c_str(), append ? "ab" : "wb");
  if (!f) return false;
  const bool ok = std::fwrite(text.data(), 1, text.size(), f) == text.size();
  return (std::fclose(f) == 0) && ok;
}

bool write_bytes(const std::string& path, const void* data, size_t bytes) {
  std::FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const bool ok = bytes == 0 || std::fwrite(data, 1, bytes, f) == bytes;
  return (std::fclose(f) == 0) && ok;
}

// One Fortran unformatted sequential record: length, payload, length.
bool put_record(std::FILE* f, const void* data, uint64_t bytes) {
  const int32_t m = (int32_t)bytes;
  return std::fwrite(&m, 4, 1, f) == 1 && (bytes == 0 || std::fwrite(data, 1, bytes, f) == bytes) &&
         std::fwrite(&m, 4, 1, f) == 1;
}

// Reads one record of exactly `bytes` bytes; false on a marker mismatch.
bool get_record(std::FILE* f, void* data, uint64_t bytes) {
  int32_t a = 0, b = 0;
  if (std::fread(&a, 4, 1, f) != 1 || (uint64_t)(uint32_t)a != bytes) return false;
  if (bytes && std::fread(data, 1, bytes, f) != bytes) return false;
  return std::fread(&b, 4, 1, f) == 1 && b == a;
}

constexpr uint64_t kMaxRecord = 2147483639ull;   // 2^31 - 9: one gfortran record

std::string dir_join(const char* dir, const std::string& name) {
  std::string d = dir ? dir : "";
  if (!d.empty() && d.back() != '/') d += '/';
  return d + name;
}

// A Fortran E/F/D input field: "0.1E+01", "0.1D+01", "-0.1+100" (an
// exponent of three digits without the letter).
double parse_real(std::string s) {
  size_t b = s.find_first_not_of(' ');
  if (b == std::string::npos) return 0.0;
  s = s.substr(b);
  while (!s.empty() && s.back() == ' ') s.pop_back();
  for (auto& c : s)
    if (c == 'd' || c == 'D') c = 'E';
  if (s.find_first_of("eE") == std::string::npos) {
    const size_t k = s.find_last_of("+-");
    if (k != std::string::npos && k > 0) s.insert(k, "E");
  }
  return std::strtod(s.c_str(), nullptr);
}

// ------------------------------------------------------------ arithmetic --
// The gas constants of module global that pressure() reads.
struct HostGas {
  double g1, g1inv, de_thresh1;
  bool de;
};

// pressure(q, press), comp.f90:45-85, FP64 in the reference's order; with
// dualenergy, q(5) or q(6) is resynchronised in place.
double host_pressure(double* q, const HostGas& c, unsigned* err) {
  const double m2 = (q[1] * q[1]) + (q[2] * q[2]) + (q[3] * q[3]);
  const double kin = 0.5 * m2 / q[0];
  double press;
  if (c.de) {
    const double ratio = kin / q[4];
    if (ratio > c.de_thresh1) {
      press = q[5] * std::pow(q[0], c.g1);
      q[4] = kin + press * c.g1inv;
    } else {
      press = c.g1 * (q[4] - kin);
      q[5] = press / std::pow(q[0], c.g1);
    }
  } else {
    press = c.g1 * (q[4] - kin);
  }
  if (press <= 0.0) *err |= EVORA_ERR_PRESSURE;
  return press;
}

// press2temp without chemistry, comp.f90:87-102.
double press2temp(double press, double rho, double temp0) { return press / rho * temp0; }

// press2temp of a cell q(nq): with chemistry T = p / sum(n) temp0, n =
// q(7:12) summed in element order, else p / rho temp0 (comp.f90:87-102).
double cell_temp(double press, const double* q, bool chemistry, double temp0) {
  if (!chemistry) return press2temp(press, q[0], temp0);
  const double ns = q[6] + q[7] + q[8] + q[9] + q[10] + q[11];
  return press / ns * temp0;
}

// compparameter's side effect on the domain bounds (parameter.f90:164-265):
// a 1D run resets ymin, ymax, zmin, zmax to [0, dx], a 2D run zmin, zmax.
struct Geometry {
  evora_derived d;
  double xmin, xmax, ymin, ymax, zmin, zmax;
};

int geometry(const evora_params* p, Geometry* G) {
  int rc = evora_compparameter(p, &G->d);
  if (rc) return rc;
  G->xmin = p->xmin; G->xmax = p->xmax;
  G->ymin = p->ymin; G->ymax = p->ymax;
  G->zmin = p->zmin; G->zmax = p->zmax;
  if (G->d.onedimension) {
    G->ymin = 0.0; G->ymax = G->d.dx;
    G->zmin = 0.0; G->zmax = G->d.dx;
  }
  if (G->d.twodimension) {
    G->zmin = 0.0; G->zmax = G->d.dx;
  }
  return 0;
}

HostGas host_gas(const evora_params* p, const Geometry& G) {
  return {G.d.g1, G.d.g1inv, G.d.de_thresh1, p->dualenergy != 0};
}

// coordinates(ix, iy, iz, x, y, z), comp.f90:150-162.
double coord(double x0, int i, double dx) { return x0 + (double)(i - 1) * dx; }

std::string line_E(const double* v, int n, int w, int d) {
  std::string s;
  for (int i = 0; i < n; ++i) s += ft::E(v[i], w, d);
  s += '\n';
  return s;
}

// ------------------------------------------------------------- snapshot --
// Cell access for the snapshot writer: either a whole q(nq, nx, ny, nz)
// (nq = 12 with chemistry) or the z = z1 plane plus the y = y1 plane of
// q(6, ...) (the cells on both live in the z plane, so every cell has
// exactly one copy).
struct CellView {
  double* q = nullptr;     // whole grid, or nullptr
  double* zp = nullptr;    // z plane: 6 * (ix + nx * iy)
  double* yp = nullptr;    // y plane: 6 * (ix + nx * iz)
  int nx = 0, ny = 0, z1 = 0, y1 = 0;
  int nq = EVORA_NQ;       // values per cell of the whole grid
  double* at(int ix, int iy, int iz) const {   // 1-based
    if (q) return q + (size_t)nq * ((ix - 1) + (size_t)nx * ((iy - 1) + (size_t)ny * (iz - 1)));
    if (iz == z1) return zp + (size_t)EVORA_NQ * ((ix - 1) + (size_t)nx * (iy - 1));
    return yp + (size_t)EVORA_NQ * ((ix - 1) + (size_t)nx * (iz - 1));
  }
};

// snapshot.f90:218-314 (cuts and slices) for one rank holding all z planes.
int snapshot_text(const evora_params* p, const Geometry& G, const CellView& v, const evora_units* u, int k3,
                  int what, const char* dir) {
  const HostGas c = host_gas(p, G);
  const int nx = p->nx, ny = p->ny, nz = p->nz;
  const int x1 = std::max(nx / 2, 1), y1 = std::max(ny / 2, 1), z1 = std::max(nz / 2, 1);
  (void)x1;
  const std::string name = ft::I0(k3, 3);
  unsigned err = 0;
  const bool chem = p->chemistry != 0;
  auto row = [&](int ix, int iy, int iz, double* press, double* temp) {
    double* q = v.at(ix, iy, iz);
    *press = host_pressure(q, c, &err);
    *temp = cell_temp(*press, q, chem, u->temp0);
    return q;
  };
  if (what & EVORA_SNAP_CUT) {
    std::string text;
    for (int ix = 1; ix <= nx && !err; ++ix) {   // x-cut
      double press, temp;
      double* q = row(ix, y1, z1, &press, &temp);
      const double r[5] = {coord(G.d.x0, ix, G.d.dx), q[0], temp, q[1] / q[0] * u->velocity0, press * u->press0};
      text += line_E(r, 5, 16, 6);
    }
    if (err) return (int)err;
    if (!write_file(dir_join(dir, name + ".x"), text, false)) return EVORA_ERR_IO;
    if (!G.d.onedimension) {                     // x0-cut
      text.clear();
      for (int ix = 1; ix <= nx && !err; ++ix) {
        double press, temp;
        double* q = row(ix, 1, z1, &press, &temp);
        const double r[5] = {coord(G.d.x0, ix, G.d.dx), q[0], temp, q[1] / q[0] * u->velocity0,
                             press * u->press0};
        text += line_E(r, 5, 16, 6);
      }
      if (err) return (int)err;
      if (!write_file(dir_join(dir, name + ".x0"), text, false)) return EVORA_ERR_IO;
    }
  }
  if (what & EVORA_SNAP_SLICE) {
    std::string text;
    for (int ix = 1; ix <= nx && !err; ++ix) {   // xy-slice
      for (int iy = 1; iy <= ny && !err; ++iy) {
        double press, temp;
        double* q = row(ix, iy, z1, &press, &temp);
        const double r[5] = {coord(G.d.x0, ix, G.d.dx), coord(G.d.y0, iy, G.d.dy), q[0], temp, press * u->press0};
        text += line_E(r, 5, 16, 6);
      }
      text += '\n';                              // write (20,*): an empty record
    }
    if (err) return (int)err;
    if (!write_file(dir_join(dir, name + ".xy"), text, false)) return EVORA_ERR_IO;
    text.clear();
    for (int iz = 1; iz <= nz && !err; ++iz) {   // xz-slice (opened for append)
      for (int ix = 1; ix <= nx && !err; ++ix) {
        double press, temp;
        double* q = row(ix, y1, iz, &press, &temp);
        const double r[5] = {coord(G.d.x0, ix, G.d.dx), coord(G.d.z0, iz, G.d.dz), q[0], temp, press * u->press0};
        text += line_E(r, 5, 16, 6);
      }
      text += '\n';
    }
    if (err) return (int)err;
    if (!write_file(dir_join(dir, name + ".xz"), text, true)) return EVORA_ERR_IO;
  }
  return 0;
}

// The TIME entry of writebovhead (write.f90:89-93): the redshift with
// supercomoving, else t.
double bov_time(const evora_params* p, const evora_units* u) { return p->supercomoving ? u->redshift : u->t; }

// writebovhead (write.f90:66-104); t is the TIME entry.
bool bov_head(const evora_params* p, const Geometry& G, double t, const std::string& name, const char* var,
              const char* dir) {
  std::string file2 = name + "." + var + ".bovdata";
  file2.resize(127, ' ');                        // character(len=127)
  const std::string varname = std::strcmp(var, "dens") == 0 ? "Density" : "Temperature";
  std::string s;
  s += "TIME: " + ft::E(t, 10, 2) + "\n";
  s += "DATA_FILE: " + ft::A(file2, 20) + "\n";
  s += "DATA_SIZE: " + ft::I(p->nx, 5) + ft::I(p->ny, 5) + ft::I(p->nz, 5) + "\n";
  s += "DATA_FORMAT: FLOAT\n";
  s += "VARIABLE:" + ft::A(varname, 20) + "\n";
  s += "DATA_ENDIAN: LITTLE\n";
  s += "CENTERING: ZONAL\n";
  s += "BRICK_ORIGIN: " + ft::E(G.xmin, 12, 2) + ft::E(G.ymin, 12, 2) + ft::E(G.zmin, 12, 2) + "\n";
  s += "BRICK_SIZE: " + ft::E(G.xmax - G.xmin, 12, 2) + ft::E(G.ymax - G.ymin, 12, 2) +
       ft::E(G.zmax - G.zmin, 12, 2) + "\n";
  return write_file(dir_join(dir, name + "." + var + ".bov"), s, false);
}

// The brick files: direct-access records of nx*ny FP32 values, one per z
// plane (snapshot.f90:317-341); written whole.
int bov_data(const evora_params* p, const std::string& name, const float* dens, const float* temp,
             const char* dir) {
  const size_t n = (size_t)p->nx * p->ny * p->nz;
  if (!write_bytes(dir_join(dir, name + ".dens.bovdata"), dens, n * 4)) return EVORA_ERR_IO;
  if (!write_bytes(dir_join(dir, name + ".temp.bovdata"), temp, n * 4)) return EVORA_ERR_IO;
  return 0;
}

// ------------------------------------------------------------------ post --
// The chemistry the post-processor's state vector needs (post.f90:58-62):
// chiH, chiHe, and compbackground + compcoef from the dump's unit file.
struct PostChem {
  bool on = false, cooling = false;
  int background = 0;
  double chiH = 0.0, chiHe = 0.0;
  evora::ChemCoef k{};
};

PostChem post_chem(const evora_params* p, const evora_units* u) {
  PostChem pc;
  if (!p->chemistry) return pc;
  pc.on = true;
  pc.cooling = p->cooling != 0;
  pc.background = p->background;
  pc.chiH = p->rhoh / evora::kMH;
  pc.chiHe = p->rhohe / evora::kMHe;
  const double uv = evora::compbackground(p->background, p->bg, p->j0, u->redshift, u->cosmo, 0.0);
  evora::compcoef(evora::ChemUnits{u->chem0, u->photo0, u->cool0, u->heat0}, uv, pc.k);
  return pc;
}

// compstate(q, state), comp.f90:201-239: the hydro build's 12 values; with
// chemistry (nstate = 26) also the species per density q(7:12)/rho, the
// number densities q(7:12) number0 and, with cooling, Lambda and Gamma of
// cool at the cell's T after cieabundance has put the cell's species in
// equilibrium in q itself, as the reference's call does (its state(25:26)
// are unset without cooling; here 0).
void compstate(double* q, const HostGas& c, double fb, const evora_units* u, const PostChem& pc, double* state,
               unsigned* err) {
  const double press = host_pressure(q, c, err);
  const double temp = cell_temp(press, q, pc.on, u->temp0);
  state[0] = q[0] / fb;
  for (int i = 1; i < 6; ++i) state[i] = q[i];
  state[6] = state[0] * u->density0;
  for (int i = 0; i < 3; ++i) state[7 + i] = q[1 + i] / state[0] * u->velocity0;
  state[10] = press * u->press0;
  state[11] = temp;
  if (!pc.on) return;
  for (int i = 6; i < 12; ++i) {
    state[i + 6] = q[i] / state[0];
    state[i + 12] = q[i] * u->number0;
  }
  state[24] = state[25] = 0.0;
  if (pc.cooling) {
    const double nH = pc.chiH * q[0], nHe = pc.chiHe * q[0];
    double chemrate[evora::kNchem], coolrate[evora::kNcool];
    evora::comprates<true>(temp, pc.k, pc.background, 1, chemrate, coolrate);
    evora::cieabundance(nH, nHe, q + 6, chemrate, pc.background, pc.k.uv, *err);
    evora::cool(q + 6, coolrate, pc.background, state[24], state[25]);
  }
}

constexpr int kNstate = 12, kNstateChem = 26;

const char* const kStateNames[] = {"rho",     "rho u",   "rho v",   "rho w",    "E",      "S",     "rho_phys",
                                   "u",       "v",       "w",       "p",        "T",      "xi_HI", "xi_HII",
                                   "xi_HeI",  "xi_HeII", "xi_HeIII", "xi_e",    "n_HI",   "n_HII", "n_HeI",
                                   "n_HeII",  "n_HeIII", "n_e",     "lambda",   "gamma"};

// writecut (write.f90:106-132)
bool writecut(const std::vector<double>& a, int n, int nvar, const char* outdir, const char* infile,
              const char* name) {
  std::string s = "#" + ft::A("x", 15);
  for (const char* h : kStateNames) s += ft::A(h, 16);
  s += '\n';
  for (int i = 0; i < n; ++i) s += line_E(&a[(size_t)nvar * i], nvar, 16, 6);
  return write_file(dir_join(outdir, std::string(infile) + "." + name + ".cut"), s, false);
}

// writeslice (write.f90:134-164)
bool writeslice(const std::vector<double>& a, int n1, int n2, int nvar, const char* outdir, const char* infile,
                const char* name) {
  std::string s = "#" + ft::A("x", 15) + ft::A("y", 16);
  for (const char* h : kStateNames) s += ft::A(h, 16);
  s += '\n';
  for (int i1 = 0; i1 < n1; ++i1) {
    for (int i2 = 0; i2 < n2; ++i2) s += line_E(&a[(size_t)nvar * (i1 + (size_t)n1 * i2)], nvar, 16, 6);
    s += "  \n";                                 // write (25,*) " "
  }
  return write_file(dir_join(outdir, std::string(infile) + "." + name + ".slice"), s, false);
}

}  // namespace
}  // namespace evora

using namespace evora;

extern "C" {

int evora_write_dump(const char* path, const double* q, int32_t nn, int32_t nx, int32_t ny, int32_t nz, int32_t lz,
                     int32_t mz) {
  if (!path || !q || nn < 1 || nx < 1 || ny < 1 || nz < 1 || lz < 1 || mz < lz || mz > nz) return EVORA_ERR_ARG;
  evora::dropin_resident_read(q);
  const uint64_t bytes = 8ull * nn * nx * ny * (uint64_t)(mz - lz + 1);
  if (bytes > kMaxRecord) return EVORA_ERR_ARG;
  std::FILE* f = std::fopen(path, "wb");
  if (!f) return EVORA_ERR_IO;
  const int32_t head[6] = {nn, nx, ny, nz, lz, mz};
  bool ok = put_record(f, head, sizeof head) && put_record(f, q, bytes);
  ok = (std::fclose(f) == 0) && ok;
  return ok ? 0 : EVORA_ERR_IO;
}

int evora_read_dump_header(const char* path, int32_t header[6]) {
  if (!path || !header) return EVORA_ERR_ARG;
  std::FILE* f = std::fopen(path, "rb");
  if (!f) return EVORA_ERR_IO;
  const bool ok = get_record(f, header, 24);
  std::fclose(f);
  return ok ? 0 : EVORA_ERR_IO;
}

int evora_read_dump(const char* path, int32_t header[6], double* q, int64_t capacity) {
  if (!path || !header || !q) return EVORA_ERR_ARG;
  std::FILE* f = std::fopen(path, "rb");
  if (!f) return EVORA_ERR_IO;
  int rc = 0;
  if (!get_record(f, header, 24)) {
    rc = EVORA_ERR_IO;
  } else {
    const int64_t nv = (int64_t)header[0] * header[1] * header[2] * (int64_t)(header[5] - header[4] + 1);
    if (header[0] < 1 || header[1] < 1 || header[2] < 1 || header[5] < header[4] || nv > capacity) rc = EVORA_ERR_ARG;
    else if (!get_record(f, q, 8ull * (uint64_t)nv)) rc = EVORA_ERR_IO;
  }
  std::fclose(f);
  return rc;
}

}  // extern "C"

namespace {

// compunits (units.f90:46-72) from the bases h, d0, t0, l0, m0 at expansion
// factor cosmo; module global's pi and the default-real literals are single
// precision (global.f90:98), x**2.0 is x*x (as gcc folds pow(x, 2.0)).
void units_at(const double b[5], double g, double fb, double t, double cosmo, double redshift, evora_units* u) {
  const double pi = (double)3.1415927f;
  const double d0 = b[1], t0 = b[2], l0 = b[3], m0 = b[4];
  const double g1 = g - 1.0;
  std::memset(u, 0, sizeof *u);
  u->t = t;
  u->cosmo = cosmo;
  u->redshift = redshift;
  u->density0 = d0 / std::pow(cosmo, 3.0);
  u->length0 = l0 * cosmo;
  u->time0 = t0 * (cosmo * cosmo);
  u->velocity0 = l0 / cosmo / t0;
  u->temp0 = (l0 * l0) / (cosmo * cosmo) / (t0 * t0) * m0 / kKb;
  u->press0 = d0 * l0 * l0 / (t0 * t0) / std::pow(cosmo, 5.0);
  u->number0 = d0 / std::pow(cosmo, 3.0) / m0;
  u->chem0 = d0 * t0 / cosmo / m0;
  u->photo0 = t0 * (cosmo * cosmo);
  u->cool0 = g1 * std::pow(t0, 3.0) * cosmo * d0 / (l0 * l0) / (m0 * m0);
  u->heat0 = g1 * std::pow(t0, 3.0) * std::pow(cosmo, 4.0) / (l0 * l0) / m0;
  u->kappa0 = std::pow(cosmo, 5.0) * std::pow(t0, 3.0) / d0 / std::pow(l0, 4.0) * 0.5 * kappa_coef();
  const double mfp_coef = (double)0.023f * kMegapc * 1e-16 * 1e-3;
  u->meanfreepath0 = (cosmo * cosmo) * m0 / l0 / d0 * 0.5 * (double)4.2f * mfp_coef;
  u->jeans0 = std::sqrt(pi * g * fb);
  u->jeansfloor0 = 0.0;
}

}  // namespace

extern "C" {

void evora_units_noncomoving(double t, double g, double fb, evora_units* u) {
  // supercomoving false: h = d0 = t0 = l0 = 1, m0 = kb, cosmo = 1
  const double b[5] = {1.0, 1.0, 1.0, 1.0, kKb};
  units_at(b, g, fb, t, 1.0, 0.0, u);
}

int evora_compunits(const evora_params* p, const evora_time* s, evora_units* u) {
  if (!p || !u) return EVORA_ERR_ARG;
  evora_derived d;
  int rc = evora_compparameter(p, &d);
  if (rc) return rc;
  double b[5];
  unit_bases(p, b);
  double t = p->tstart, cosmo = 1.0, redshift = 0.0;
  if (s) {
    t = s->t;
    cosmo = s->cosmo;
    redshift = s->redshift;
  } else if (p->supercomoving) {
    cosmo = 1.0 / (1.0 + p->zstart);   // cosmostart (cosmology.f90:32-33)
    redshift = p->zstart;
  }
  units_at(b, d.g, p->fb, t, cosmo, redshift, u);
  if (p->jeansfloor) {   // units.f90:66-71
    const double r = d.dx / u->jeans0 / p->c_jeans;
    u->jeansfloor0 = r * r;
  }
  return 0;
}

int evora_write_units(const char* path, const evora_units* u) {
  if (!path || !u) return EVORA_ERR_ARG;
  const char* const label[18] = {"t =             ", "cosmo =         ", "redshift =      ", "length0 =       ",
                                 "time0 =         ", "density0 =      ", "velocity0 =     ", "temp0 =         ",
                                 "press0 =        ", "number0 =       ", "chem0 =         ", "photo0 =        ",
                                 "cool0 =         ", "heat0 =         ", "jeans0 =        ", "jeansfloor0 =   ",
                                 "kappa0 =        ", "meanfreepath0 = "};
  const double* v = &u->t;
  std::string s;
  for (int i = 0; i < 18; ++i) s += std::string(label[i]) + ft::E(v[i], 16, 8) + "\n";
  return write_file(path, s, false) ? 0 : EVORA_ERR_IO;
}

int evora_read_units(const char* path, evora_units* u) {
  if (!path || !u) return EVORA_ERR_ARG;
  std::FILE* f = std::fopen(path, "rb");
  if (!f) return EVORA_ERR_IO;
  double* v = &u->t;
  char line[256];
  int i = 0;
  for (; i < 18 && std::fgets(line, sizeof line, f); ++i) {
    std::string s = line;
    while (!s.empty() && (s.back() == '\n' || s.back() == '\r')) s.pop_back();
    v[i] = s.size() > 16 ? parse_real(s.substr(16, 16)) : 0.0;   // '(A16,E16.8)'
  }
  std::fclose(f);
  return i == 18 ? 0 : EVORA_ERR_IO;
}

int evora_snapshot(const evora_params* p, double* q, const evora_units* u, int32_t k3, int32_t what,
                   const char* dir) {
  if (!p || !q || !u || k3 < 0) return EVORA_ERR_ARG;
  evora::dropin_resident_write(q);
  Geometry G;
  int rc = geometry(p, &G);
  if (rc) return rc;
  CellView v;
  v.q = q;
  v.nx = p->nx;
  v.ny = p->ny;
  v.nq = p->chemistry ? EVORA_NQ_CHEM : EVORA_NQ;
  rc = snapshot_text(p, G, v, u, k3, what, dir);
  if (rc || !(what & EVORA_SNAP_BOV)) return rc;
  const std::string name = ft::I0(k3, 3);
  if (!bov_head(p, G, bov_time(p, u), name, "dens", dir) || !bov_head(p, G, bov_time(p, u), name, "temp", dir))
    return EVORA_ERR_IO;
  const HostGas c = host_gas(p, G);
  const size_t n = (size_t)p->nx * p->ny * p->nz;
  std::vector<float> dens(n), temp(n);
  unsigned err = 0;
  for (size_t i = 0; i < n && !err; ++i) {
    double* cell = q + (size_t)v.nq * i;
    dens[i] = (float)cell[0];
    const double press = host_pressure(cell, c, &err);
    temp[i] = (float)cell_temp(press, cell, p->chemistry != 0, u->temp0);
  }
  if (err) return (int)err;
  return bov_data(p, name, dens.data(), temp.data(), dir);
}

int evora_grid_snapshot(evora_grid* g, const evora_units* u, int32_t k3, int32_t what, const char* dir) {
  if (!g || !u || k3 < 0) return EVORA_ERR_ARG;
  const evora_params* p = grid_params(g);
  if (p->chemistry) {
    // the temperatures read the species: the whole q(12) through the host
    // writer; with dualenergy its resynchronised cells go back to the grid
    std::vector<double> q((size_t)EVORA_NQ_CHEM * p->nx * p->ny * p->nz);
    int rc = evora_grid_get_q(g, q.data());
    if (!rc) rc = evora_snapshot(p, q.data(), u, k3, what, dir);
    if (!rc && p->dualenergy) rc = evora_grid_set_q(g, q.data());
    return rc;
  }
  Geometry G;
  int rc = geometry(p, &G);
  if (rc) return rc;
  const int nx = p->nx, ny = p->ny, nz = p->nz;
  const int y1 = std::max(ny / 2, 1), z1 = std::max(nz / 2, 1);
  if (what & (EVORA_SNAP_CUT | EVORA_SNAP_SLICE)) {
    std::vector<double> zp((size_t)EVORA_NQ * nx * ny), yp((size_t)EVORA_NQ * nx * nz);
    if ((rc = evora_grid_get_plane(g, 3, z1, zp.data()))) return rc;
    if ((rc = evora_grid_get_plane(g, 2, y1, yp.data()))) return rc;
    CellView v;
    v.zp = zp.data();
    v.yp = yp.data();
    v.nx = nx;
    v.ny = ny;
    v.z1 = z1;
    v.y1 = y1;
    rc = snapshot_text(p, G, v, u, k3, what, dir);
    if (rc) return rc;
    if (p->dualenergy) {
      // the y plane's copy of its z = z1 row is stale: take it from the z plane
      for (int ix = 1; ix <= nx; ++ix)
        std::memcpy(v.yp + (size_t)EVORA_NQ * ((ix - 1) + (size_t)nx * (z1 - 1)), v.at(ix, y1, z1),
                    sizeof(double) * EVORA_NQ);
      if ((rc = evora_grid_set_plane(g, 2, y1, yp.data()))) return rc;
      if ((rc = evora_grid_set_plane(g, 3, z1, zp.data()))) return rc;
    }
  }
  if (!(what & EVORA_SNAP_BOV)) return 0;
  const std::string name = ft::I0(k3, 3);
  if (!bov_head(p, G, bov_time(p, u), name, "dens", dir) || !bov_head(p, G, bov_time(p, u), name, "temp", dir))
    return EVORA_ERR_IO;
  const size_t n = (size_t)nx * ny * nz;
  std::vector<float> dens(n), temp(n);
  if ((rc = grid_bov(g, u->temp0, dens.data(), temp.data()))) return rc;
  return bov_data(p, name, dens.data(), temp.data(), dir);
}

int evora_cuts_and_slices(const evora_params* p, double fb, const evora_units* u, const char* datadir,
                          const char* infile, const char* outdir) {
  if (!p || !u || !infile) return EVORA_ERR_ARG;
  Geometry G;
  int rc = geometry(p, &G);
  if (rc) return rc;
  const HostGas c = host_gas(p, G);
  const PostChem pc = post_chem(p, u);
  const int nq = pc.on ? EVORA_NQ_CHEM : EVORA_NQ;
  const int nx = p->nx, ny = p->ny, nz = p->nz;
  const double xmid = std::max(nx / 2, 1), ymid = std::max(ny / 2, 1), zmid = std::max(nz / 2, 1);
  const bool one = G.d.onedimension, two = G.d.twodimension;
  const bool cut_x = true, cut_y = !one, slice_xy = !one, cut_xy = !one && nx == ny;
  const bool cut_z = !one && !two, slice_xz = cut_z, slice_yz = cut_z, cut_xyz = cut_z && nx == ny && ny == nz;
  const int nstate = pc.on ? kNstateChem : kNstate;
  const int nv = nstate + 1, ns = nstate + 2;
  std::vector<double> cx, cy, cz, cxy, cxyz, sxy, sxz, syz;
  // coordinates (post.f90:124-170): k - 0.5 in default real, sqrt(2.0) and
  // sqrt(3.0) of default reals
  auto hc = [](int k) { return (double)((float)k - 0.5f); };
  if (cut_x) {
    cx.assign((size_t)nv * nx, 0.0);
    for (int k = 1; k <= nx; ++k) cx[(size_t)nv * (k - 1)] = G.xmin + hc(k) * G.d.dx;
  }
  if (cut_y) {
    cy.assign((size_t)nv * ny, 0.0);
    for (int k = 1; k <= ny; ++k) cy[(size_t)nv * (k - 1)] = G.ymin + hc(k) * G.d.dy;
  }
  if (cut_z) {
    cz.assign((size_t)nv * nz, 0.0);
    for (int k = 1; k <= nz; ++k) cz[(size_t)nv * (k - 1)] = G.zmin + hc(k) * G.d.dz;
  }
  if (cut_xy) {
    cxy.assign((size_t)nv * nx, 0.0);
    for (int k = 1; k <= nx; ++k) cxy[(size_t)nv * (k - 1)] = (double)std::sqrt(2.0f) * (G.xmin + hc(k) * G.d.dx);
  }
  if (cut_xyz) {
    cxyz.assign((size_t)nv * nx, 0.0);
    for (int k = 1; k <= nx; ++k) cxyz[(size_t)nv * (k - 1)] = (double)std::sqrt(3.0f) * (G.xmin + hc(k) * G.d.dx);
  }
  auto slice_init = [&](std::vector<double>& a, int n1, int n2, double m1, double d1, double m2, double d2) {
    a.assign((size_t)ns * n1 * n2, 0.0);
    for (int i2 = 1; i2 <= n2; ++i2)
      for (int i1 = 1; i1 <= n1; ++i1) {
        double* e = &a[(size_t)ns * ((i1 - 1) + (size_t)n1 * (i2 - 1))];
        e[0] = m1 + hc(i1) * d1;
        e[1] = m2 + hc(i2) * d2;
      }
  };
  if (slice_xy) slice_init(sxy, nx, ny, G.xmin, G.d.dx, G.ymin, G.d.dy);
  if (slice_xz) slice_init(sxz, nx, nz, G.xmin, G.d.dx, G.zmin, G.d.dz);
  if (slice_yz) slice_init(syz, ny, nz, G.ymin, G.d.dy, G.zmin, G.d.dz);

  // gather (post.f90:177-219): the ranks' files until one ends at nz
  unsigned err = 0;
  int mz = 0;
  std::vector<double> q;
  for (int j = 0; mz != nz; ++j) {
    if (j > 99999) return EVORA_ERR_IO;
    const std::string path = dir_join(datadir, std::string(infile) + "." + ft::I0(j, 3));
    int32_t h[6];
    if ((rc = evora_read_dump_header(path.c_str(), h))) return rc;
    if (h[0] != nq || h[1] != nx || h[2] != ny || h[3] != nz || h[4] < 1 || h[5] < h[4] || h[5] > nz)
      return EVORA_ERR_ARG;
    q.resize((size_t)nq * nx * ny * (h[5] - h[4] + 1));
    if ((rc = evora_read_dump(path.c_str(), h, q.data(), (int64_t)q.size()))) return rc;
    const int lz = h[4];
    mz = h[5];
    for (int iz = lz; iz <= mz; ++iz)
      for (int iy = 1; iy <= ny; ++iy)
        for (int ix = 1; ix <= nx; ++ix) {
          double* cell = &q[(size_t)nq * ((ix - 1) + (size_t)nx * ((iy - 1) + (size_t)ny * (iz - lz)))];
          auto st = [&](std::vector<double>& a, size_t idx, int off) {
            compstate(cell, c, fb, u, pc, &a[idx + off], &err);
          };
          if (cut_x && iy == ymid && iz == zmid) st(cx, (size_t)nv * (ix - 1), 1);
          if (cut_y && ix == xmid && iz == zmid) st(cy, (size_t)nv * (iy - 1), 1);
          if (cut_z && ix == xmid && iy == ymid) st(cz, (size_t)nv * (iz - 1), 1);
          if (cut_xy && iz == zmid && ix == iy) st(cxy, (size_t)nv * (ix - 1), 1);
          if (cut_xyz && ix == iy && ix == iz) st(cxyz, (size_t)nv * (ix - 1), 1);
          if (slice_xy && iz == zmid) st(sxy, (size_t)ns * ((ix - 1) + (size_t)nx * (iy - 1)), 2);
          if (slice_xz && iy == ymid) st(sxz, (size_t)ns * ((ix - 1) + (size_t)nx * (iz - 1)), 2);
          if (slice_yz && ix == xmid) st(syz, (size_t)ns * ((iy - 1) + (size_t)ny * (iz - 1)), 2);
          if (err) return (int)err;
        }
  }
  // write (post.f90:224-231); the .xyz file receives the diagonal cut's data
  bool ok = true;
  if (cut_x) ok = ok && writecut(cx, nx, nv, outdir, infile, "x");
  if (cut_y) ok = ok && writecut(cy, ny, nv, outdir, infile, "y");
  if (cut_z) ok = ok && writecut(cz, nz, nv, outdir, infile, "z");
  if (cut_xy) ok = ok && writecut(cxy, nx, nv, outdir, infile, "xy");
  if (cut_xyz) ok = ok && writecut(cxy, nx, nv, outdir, infile, "xyz");
  if (slice_xy) ok = ok && writeslice(sxy, nx, ny, ns, outdir, infile, "xy");
  if (slice_xz) ok = ok && writeslice(sxz, nx, nz, ns, outdir, infile, "xz");
  if (slice_yz) ok = ok && writeslice(syz, ny, nz, ns, outdir, infile, "yz");
  return ok ? 0 : EVORA_ERR_IO;
}

}  // extern "C"
