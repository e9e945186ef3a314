// evora_post -- the post-processor's "cs" mode (post.f90:26-78, 85-246) for
// the dumps a run wrote:
//
//   evora_post cs <snapshot> [--workdir DIR]
//
// rereads data/parameter (rereadparameter, parameter.f90:339-411), runs
// compparameter, reads data/<snapshot>.units (readunits, units.f90:115-159)
// and writes out/<snapshot>.{x,y,z,xy,xyz}.cut and .{xy,xz,yz}.slice from
// data/<snapshot>.000, .001, ...  The other modes of the reference's post
// (bov, phase, ps) are not part of the hydro path's formats.
#include <cstdio>
#include <string>

#include <sys/stat.h>
#include <unistd.h>

#include "../../../include/evora_gpu.h"
#include "../../../include/evora_io.h"
#include "params_file.h"

using namespace evora::driver;

int main(int argc, char** argv) {
  if (argc < 3) {   // post.f90:33-38
    std::puts(" ERROR to few arguments");
    std::puts(" USAGE bin/post <mode> <snapshot> <option>");
    return 1;
  }
  const std::string mode = argv[1], infile = argv[2];
  for (int i = 3; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--workdir" && i + 1 < argc) {
      if (chdir(argv[++i]) != 0) {
        std::fprintf(stderr, "ERROR cannot enter %s\n", argv[i]);
        return 1;
      }
    }
  }
  if (mode != "cs") {
    std::puts(" wrong mode");
    std::puts(" choose cs");
    return 1;
  }
  std::string text;
  if (!read_text("data/parameter", &text)) {
    std::puts(" ERROR file not found: data/parameter");
    return 1;
  }
  RunParams run;
  if (!reread(text, &run)) {
    std::puts(" ERROR data/parameter is incomplete");
    return 1;
  }
  const evora_params p = hydro_params(run);
  evora_derived d;
  int rc = evora_compparameter(&p, &d);
  if (rc) {
    std::fprintf(stderr, "ERROR invalid parameters (status %d)\n", rc);
    return 1;
  }
  evora_units u;
  const std::string units = "data/" + infile + ".units";
  if (evora_read_units(units.c_str(), &u)) {
    std::printf(" ERROR file not found: %s\n", units.c_str());
    return 1;
  }
  std::puts(" cuts and slices");
  mkdir("out", 0755);
  rc = evora_cuts_and_slices(&p, run["fb"], &u, "data", infile.c_str(), "out");
  if (rc) {
    std::fprintf(stderr, "ERROR cuts and slices failed (status %d)\n", rc);
    return 1;
  }
  return 0;
}
