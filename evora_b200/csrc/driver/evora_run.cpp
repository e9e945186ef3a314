// evora_run -- the hydro run of the reference's driver (main.f90) on top of
// the C ABI: reads the parameter file, builds the initial condition, runs the
// time loop with the state resident on the GPU and writes the reference's
// output files.
//
//   evora_run <parameterfile> [--ic shocktube|kevinhelmholtz|dump:FILE]
//             [--fp32] [--strict] [--entropy] [--workdir DIR]
//             [--print-params]
//
// Input: namelist group para (parameter.f90:26-105) and, for the shocktube,
// ic_para (ic/shocktube.f90:39-47).  The reference compiles one ic/<name>.f90
// into the binary (object/Makefile:57-58); here --ic chooses at run time.
// --ic dump:FILE reads the initial state from a dump in writedata's format
// (write.f90:47-65; nn = 6, or 12 with the species of a chemistry run, the
// whole grid in one file), the way ic/grafic.f90 reads an external initial
// condition: the cosmological box's Zel'dovich IC (ic/cosmo.f90) is built
// outside the driver and run through it.
// Self-gravity (gravity = .true.), the temperature / Jeans pressure floors,
// thermal conduction (conduction = .true. with simplekappa = .true.) and,
// with comoving coordinates (supercomoving = .true.), the expansion factor's
// integration, the comoving units and the expansion terms run on the device
// with each hydro step as in main.f90:119-185.  With chemistry (the CIE
// build: nq = 12, species n(H, H+, He, He+, He++, e-) in q(7:12)) the IC's
// species come from initchem (main.f90:94), every step runs chem(q) and,
// with cooldt, the cooling time step, and dumps and snapshots carry q(12);
// the non-equilibrium build (noncie), which grids do not run, is refused.
// With supercomoving, data/<k4>.000 and data/<k4>.units are written when a
// step lands on dump_redshift(k4) (main.f90:197-202), and the cadence
// variable is tsnap = a * nsnap.
//
// Output, under the working directory, as the reference writes it:
//   data/parameter           writeparameter (parameter.f90:267-337)
//   data/in.000, data/out.000, data/{in,out}.units
//                            writedump (write.f90:26-65, units.f90:76-113)
//   data/evo                 evolution (snapshot.f90:159-193)
//   data/log, stdout         screen (snapshot.f90:132-155)
//   snap/<k3>.{x,x0,xy,xz,dens.bov,...}
//                            snapshot (snapshot.f90:196-360) when cut, slice
//                            or bov is set
// The output cadence is main.f90:184-195: tsnap = (t - tstart) / (tend -
// tstart) * nsnap; each counter k1 (screen), k2 (evolution), k3 (snapshot)
// fires at most once per step and then advances by one.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <sys/stat.h>
#include <unistd.h>

#include "../../../include/evora_gpu.h"
#include "../../../include/evora_io.h"
#include "params_file.h"

using namespace evora;
using namespace evora::driver;
namespace ft = evora::fortran;

namespace {

// ic/shocktube.f90:49-100 with coordinates() of comp.f90:150-162
void ic_shocktube(const evora_params& p, const evora_derived& d, const std::map<std::string, std::string>& ic,
                  std::vector<double>* q) {
  auto get = [&](const char* k, double def) {
    auto it = ic.find(k);
    return it == ic.end() ? def : to_real(it->second);
  };
  const double dl = get("dl", 1.0), ul = get("ul", 0.0), pl = get("pl", 1.0);
  const double dr = get("dr", 0.125), ur = get("ur", 0.0), pr = get("pr", 0.1);
  const double xd = get("x_diss", 0.5);
  const int dir = (int)get("dir", 1);
  q->assign((size_t)EVORA_NQ * p.nx * p.ny * p.nz, 0.0);
  for (int iz = 1; iz <= p.nz; ++iz)
    for (int iy = 1; iy <= p.ny; ++iy)
      for (int ix = 1; ix <= p.nx; ++ix) {
        const double x = d.x0 + (double)(ix - 1) * d.dx;
        const double y = d.y0 + (double)(iy - 1) * d.dy;
        const double z = d.z0 + (double)(iz - 1) * d.dz;
        const bool left = (dir == 1 && x < xd) || (dir == 2 && y < xd) || (dir == 3 && z < xd);
        const double rho = left ? dl : dr, u = left ? ul : ur, pp = left ? pl : pr;
        double* c = q->data() + (size_t)EVORA_NQ * ((ix - 1) + (size_t)p.nx * ((iy - 1) + (size_t)p.ny * (iz - 1)));
        c[0] = rho;
        c[1] = dir == 1 ? rho * u : 0.0;
        c[2] = dir == 2 ? rho * u : 0.0;
        c[3] = dir == 3 ? rho * u : 0.0;
        c[4] = 0.5 * rho * (u * u) + pp / d.g1;
        c[5] = pp / std::pow(rho, d.g1);
      }
}

// ic/kevinhelmholtz.f90:40-69; pi and the literals 0.1 and 0.05 are default
// (single precision) reals there (global.f90:98).
void ic_kh(const evora_params& p, const evora_derived& d, std::vector<double>* q) {
  const double pi = (double)3.1415927f;
  q->assign((size_t)EVORA_NQ * p.nx * p.ny * p.nz, 0.0);
  for (int iz = 1; iz <= p.nz; ++iz)
    for (int iy = 1; iy <= p.ny; ++iy)
      for (int ix = 1; ix <= p.nx; ++ix) {
        const double x = d.x0 + (double)(ix - 1) * d.dx;
        const double y = d.y0 + (double)(iy - 1) * d.dy;
        const double r = std::fabs(y - 0.5);
        const double rho = r <= 0.25 ? 2.0 : 1.0, u = r <= 0.25 ? 0.5 : -0.5;
        const double v = (double)0.1f * std::sin(4 * pi * x) *
                         (std::exp(-((y - 0.25) * (y - 0.25)) / (double)0.05f) +
                          std::exp(-((y - 0.75) * (y - 0.75)) / (double)0.05f));
        const double pp = 2.5;
        double* c = q->data() + (size_t)EVORA_NQ * ((ix - 1) + (size_t)p.nx * ((iy - 1) + (size_t)p.ny * (iz - 1)));
        c[0] = rho;
        c[1] = rho * u;
        c[2] = rho * v;
        c[3] = 0;
        c[4] = .5 * rho * ((u * u) + (v * v)) + pp / (d.g - 1);
        c[5] = pp / std::pow(rho, d.g - 1);
      }
}

bool append(const std::string& path, const std::string& text) {
  std::FILE* f = std::fopen(path.c_str(), "ab");
  if (!f) return false;
  const bool ok = std::fwrite(text.data(), 1, text.size(), f) == text.size();
  return (std::fclose(f) == 0) && ok;
}

bool write_new(const std::string& path, const std::string& text) {
  std::FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const bool ok = std::fwrite(text.data(), 1, text.size(), f) == text.size();
  return (std::fclose(f) == 0) && ok;
}

int fail(const char* what, int rc) {
  std::fprintf(stderr, "ERROR %s (status %d) %s\n", what, rc, evora_last_error());
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr,
                 "usage: %s <parameterfile> [--ic shocktube|kevinhelmholtz|dump:FILE] [--fp32] [--strict] [--entropy] "
                 "[--workdir DIR] [--print-params]\n",
                 argv[0]);
    return 2;
  }
  std::string icname = "shocktube", workdir;
  int precision = EVORA_FP64, flags = 0;
  bool print_only = false;
  for (int i = 2; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--ic" && i + 1 < argc) icname = argv[++i];
    else if (a == "--fp32") precision = EVORA_FP32;
    else if (a == "--strict") flags |= EVORA_STRICT;
    else if (a == "--entropy") flags |= EVORA_CARRY_ENTROPY;
    else if (a == "--workdir" && i + 1 < argc) workdir = argv[++i];
    else if (a == "--print-params") print_only = true;
    else {
      std::fprintf(stderr, "unknown option %s\n", a.c_str());
      return 2;
    }
  }
  // readparameter (parameter.f90:26-105)
  std::string text;
  if (!read_text(argv[1], &text)) {
    std::printf(" ERROR file not found: %s\n", argv[1]);   // parameter.f90:91-93
    return 1;
  }
  if (!workdir.empty() && chdir(workdir.c_str()) != 0) {
    std::fprintf(stderr, "ERROR cannot enter %s\n", workdir.c_str());
    return 1;
  }
  std::map<std::string, std::string> para, icp;
  if (!read_group(text, "para", &para)) {
    std::fprintf(stderr, "ERROR no namelist group para in %s\n", argv[1]);
    return 1;
  }
  read_group(text, "ic_para", &icp);
  RunParams run = defaults();
  std::string unknown;
  apply_namelist(para, &run, &unknown);
  if (!unknown.empty()) {
    std::fprintf(stderr, "ERROR unknown entries in namelist para: %s\n", unknown.c_str());
    return 1;
  }
  evora_params p = hydro_params(run);
  const int nsnap = (int)run["nsnap"];
  const double fb = run["fb"];
  const bool cut = run.flag("cut"), slice = run.flag("slice"), bov = run.flag("bov");
  evora_derived d;
  int rc = evora_compparameter(&p, &d);
  if (print_only) {
    std::fputs(parameter_text(run).c_str(), stdout);
    std::printf("status =        %16d\n", rc);
    return rc ? 1 : 0;
  }
  const std::string off = unsupported(run);
  if (!off.empty()) {
    std::fprintf(stderr, "ERROR not on the hydro path: %s\n", off.c_str());
    return 1;
  }
  if (rc) return fail("invalid parameters", rc);
  mkdir("data", 0755);
  if (cut || slice || bov) mkdir("snap", 0755);
  if (!write_new("data/parameter", parameter_text(run))) {
    std::printf(" ERROR file not found: data/parameter\n");
    return 1;
  }
  std::remove("data/evo");
  std::remove("data/log");

  // ic(q) and the first dump (main.f90:80-97)
  std::vector<double> q;
  const bool chem = p.chemistry != 0;
  const int nq = chem ? EVORA_NQ_CHEM : EVORA_NQ;
  bool have_species = false;   // the IC carries q(7:12)
  if (icname == "shocktube") ic_shocktube(p, d, icp, &q);
  else if (icname == "kevinhelmholtz") ic_kh(p, d, &q);
  else if (icname.rfind("dump:", 0) == 0) {
    const std::string path = icname.substr(5);
    int32_t h[6];
    if ((rc = evora_read_dump_header(path.c_str(), h))) return fail("IC dump", rc);
    if (!((h[0] == EVORA_NQ || (chem && h[0] == EVORA_NQ_CHEM)) && h[1] == p.nx && h[2] == p.ny && h[3] == p.nz &&
          h[4] == 1 && h[5] == p.nz)) {
      std::fprintf(stderr, "ERROR IC dump %s: nn,nx,ny,nz,lz,mz = %d,%d,%d,%d,%d,%d do not fit the run\n",
                   path.c_str(), h[0], h[1], h[2], h[3], h[4], h[5]);
      return 1;
    }
    std::vector<double> qd((size_t)h[0] * p.nx * p.ny * p.nz);
    if ((rc = evora_read_dump(path.c_str(), h, qd.data(), (int64_t)qd.size()))) return fail("IC dump", rc);
    have_species = h[0] == EVORA_NQ_CHEM;
    q.swap(qd);
  } else {
    std::fprintf(stderr, "unknown IC %s\n", icname.c_str());
    return 2;
  }
  (void)fb;
  if (chem && !have_species) {
    // q(12): the IC's q(1:6), then initchem (main.f90:93-94) sets the
    // equilibrium species through the drop-in layer
    const size_t n = (size_t)p.nx * p.ny * p.nz;
    std::vector<double> q12((size_t)EVORA_NQ_CHEM * n, 0.0);
    for (size_t i = 0; i < n; ++i)
      for (int f = 0; f < EVORA_NQ; ++f) q12[(size_t)EVORA_NQ_CHEM * i + f] = q[(size_t)EVORA_NQ * i + f];
    if ((rc = evora_set_params(&p))) return fail("set_params", rc);
    if ((rc = evora_initchem(q12.data()))) return fail("initchem", rc);
    q.swap(q12);
  }
  evora_units u;   // compunits at the start (main.f90:58-62)
  if ((rc = evora_compunits(&p, nullptr, &u))) return fail("compunits", rc);
  const bool comoving = p.supercomoving != 0;
  auto dump = [&](const char* name) {
    const std::string base = std::string("data/") + name;
    int r = evora_write_dump((base + ".000").c_str(), q.data(), nq, p.nx, p.ny, p.nz, 1, p.nz);
    if (!r) r = evora_write_units((base + ".units").c_str(), &u);
    return r;
  };
  if ((rc = dump("in"))) return fail("writedump in", rc);

  evora_grid* g = nullptr;
  if ((rc = evora_grid_create(&p, precision, flags, &g))) return fail("grid_create", rc);
  if ((rc = evora_grid_set_q(g, q.data()))) return fail("grid_set_q", rc);

  int k1 = 0, k2 = 0, k3 = 0;
  int64_t k = 0;
  double t = p.tstart, dt = 0.0, tsnap = 0.0;
  int32_t go = 1;
  auto evolution = [&]() {   // snapshot.f90:159-193
    double tot[6];
    int r = evora_grid_totals(g, tot);
    if (r) return r;
    std::string s;
    if (k2 == 0)
      s += "#" + ft::A("t", 15) + ft::A("dt", 16) + ft::A("a", 16) + ft::A("z", 16) + ft::A("totalmass", 16) +
           ft::A("totalenergy", 16) + ft::A("totalentropy", 16) + "\n";
    const double row[7] = {t, dt, u.cosmo, u.redshift, tot[0] * d.volume, tot[4] * d.volume, tot[5] * d.volume};
    for (double x : row) s += ft::E(x, 16, 6);
    s += "\n";
    k2 = k2 + 1;
    return append("data/evo", s) ? 0 : EVORA_ERR_IO;
  };
  auto screen = [&]() {      // snapshot.f90:132-155
    std::string s;
    if (comoving) {
      s = ft::I(k1, 4) + ft::I(k, 6) + ft::E(t, 12, 4) + ft::E(dt, 12, 4) + ft::F(u.cosmo, 12, 4) +
          ft::F(u.redshift, 12, 2) + "\n";
    } else {
      const double tpro = tsnap / nsnap * 100;
      s = ft::I(k1, 4) + ft::I(k, 6) + ft::E(t, 12, 4) + ft::E(dt, 12, 4) + std::string(11, ' ') +
          ft::F(tpro, 12, 1) + "%\n";
    }
    std::fputs(s.c_str(), stdout);
    std::fflush(stdout);
    append("data/log", s);
    k1 = k1 + 1;
  };
  auto snapshot = [&]() {
    u.t = t;
    const int what = (cut ? EVORA_SNAP_CUT : 0) | (slice ? EVORA_SNAP_SLICE : 0) | (bov ? EVORA_SNAP_BOV : 0);
    int r = evora_grid_snapshot(g, &u, k3, what, "snap");
    k3 = k3 + 1;
    return r;
  };

  if ((rc = evolution())) return fail("evolution", rc);           // main.f90:100
  if ((cut || slice || bov) && (rc = snapshot())) return fail("snapshot", rc);
  if (run.flag("iconly")) {                                        // main.f90:106
    evora_grid_destroy(g);
    return 0;
  }
  while (go) {                                                     // main.f90:109-203
    rc = evora_grid_step(g, 1, 1);
    if (rc) {
      // the reference stops where the failing routine detects the error
      // (cleanstop), without a final dump
      std::fprintf(stderr, "ERROR hydro step failed (status %d) after t = %.17g\n", rc, t);
      evora_grid_destroy(g);
      return 1;
    }
    if ((rc = evora_grid_time(g, &t, &dt, &go, &k))) return fail("grid_time", rc);
    int32_t dumpk = 0;
    if (comoving) {
      // compunits after compcosmo (main.f90:132-133); tsnap = cosmo * nsnap
      evora_time s;
      if ((rc = evora_grid_cosmo(g, &s, &dumpk))) return fail("grid_cosmo", rc);
      if ((rc = evora_compunits(&p, &s, &u))) return fail("compunits", rc);
      tsnap = s.cosmo * nsnap;
    } else {
      u.t = t;
      tsnap = (t - p.tstart) / (p.tend - p.tstart) * nsnap;
    }
    if (tsnap >= (double)k1) screen();
    if (tsnap >= (double)k2 && (rc = evolution())) return fail("evolution", rc);
    if ((cut || slice || bov) && tsnap >= (double)k3 && (rc = snapshot())) return fail("snapshot", rc);
    if (dumpk) {   // main.f90:197-202: writedump(q, k4 as I0.3)
      if ((rc = evora_grid_get_q(g, q.data()))) return fail("grid_get_q", rc);
      if ((rc = dump(ft::I0(dumpk, 3).c_str()))) return fail("writedump", rc);
    }
  }
  if ((rc = evora_grid_get_q(g, q.data()))) return fail("grid_get_q", rc);
  u.t = t;
  if ((rc = dump("out"))) return fail("writedump out", rc);        // main.f90:206
  evora_grid_destroy(g);
  std::puts(" ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~");   // endscreen
  std::puts(" done!");
  std::puts(" ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~");
  return 0;
}
