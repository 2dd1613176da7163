// sourceshape.cpp -- laph_sourceshape, the replacement of LapH_EigSys's
// sourceshape program (src/sourceshape.cpp): for one configuration and
// timeslice, read the eigensystem <in_path>/eigenvectors.%04d.%03d
// (read_evectors_bin_ts, modules/read_write.cpp:40-68), form the source shape
// psi(r) on the device (source_shape_complete, modules/sourceshape_funcs.cpp:30-81),
// average it over equal radii (avg_radii, :100-135), print "r psi" and write
// sourceshape_nev<nev>.<config>.<t> and its .bin twin into the working
// directory (write_sourceshape_ascii/_bin, modules/read_write.cpp:205-234).
//
// Same positional arguments as the reference (configuration, timeslice, nev),
// which stops with garbage arguments where this one prints its usage.
// --weighted reads <in_path>/eigenvalues.%04d.%03d and weights eigenvector n
// by sqrt|ev_n| first (weight_eigenvectors, commented out in the reference's
// main but part of its library, sourceshape_funcs.cpp:85-96).
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/laph_gpu.h"

namespace {

int die(int st, const char* what) {
  std::fprintf(stderr, "laph_sourceshape: %s: %s (%s)\n", what, laph_strerror(st), laph_last_error());
  return 1;
}

void usage() {
  std::fprintf(stderr, "usage: laph_sourceshape [--parameters FILE] [--weighted] CONFIG TIMESLICE NEV\n");
}

}  // namespace

int main(int argc, char** argv) {
  std::string params = "parameters.txt";
  int weighted = 0;
  std::vector<std::string> pos;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--parameters" && i + 1 < argc) params = argv[++i];
    else if (a == "--weighted") weighted = 1;
    else if (!a.empty() && a[0] == '-' && !(a.size() > 1 && a[1] >= '0' && a[1] <= '9')) {
      usage();
      return 2;
    } else {
      pos.push_back(a);
    }
  }
  if (pos.size() != 3) {
    std::printf("No parameters entered. Arguments are: configuration timeslice dim(V)\n");
    usage();
    return 2;
  }
  const int config = std::atoi(pos[0].c_str()), t = std::atoi(pos[1].c_str()), nev = std::atoi(pos[2].c_str());
  std::printf("Entered parameters: config: %d ts: %d nev: %d\n", config, t, nev);
  laph_config P;
  int st = laph_parse_parameters(params.c_str(), &P);
  if (st != LAPH_OK) return die(st, "parameters");
  const int L = P.LX;
  if (nev < 1 || L < 2 || (L & 1) || t < 0) {
    std::fprintf(stderr, "laph_sourceshape: need nev >= 1, an even LX and a timeslice >= 0\n");
    return 2;
  }
  const int dim = 3 * L * L * L;
  const char* dir = P.in_path[0] ? P.in_path : ".";
  std::vector<double> V((size_t)2 * dim * nev);
  st = laph_read_eigsys_bin(dir, "eigenvectors", config, t, dim, nev, V.data());
  if (st != LAPH_OK) return die(st, "read eigenvectors");
  std::vector<double> ev;
  if (weighted) {
    ev.resize(nev);
    st = laph_read_eigenvalues_bin(dir, "eigenvalues", config, t, nev, ev.data());
    if (st != LAPH_OK) return die(st, "read eigenvalues");
  }
  const int H = L / 2, n = H * H * H;
  std::vector<double> psi(n), r(n), avg(n);
  std::printf("calculating, please wait...\n");
  const int device = std::getenv("LAPH_DEVICE") ? std::atoi(std::getenv("LAPH_DEVICE")) : 0;
  st = laph_sourceshape(V.data(), L, nev, weighted ? ev.data() : nullptr, 0, psi.data(), device);
  if (st != LAPH_OK) return die(st, "sourceshape");
  int navg = 0;
  st = laph_sourceshape_avg(L, psi.data(), r.data(), avg.data(), &navg);
  if (st != LAPH_OK) return die(st, "average");
  std::printf("avg complete\nLength of average vector:%d\n", navg);
  for (int i = 0; i < navg; ++i) std::printf("%.12g %.12g\n", r[i], avg[i]);
  st = laph_write_sourceshape(nullptr, config, t, nev, navg, r.data(), avg.data());
  if (st != LAPH_OK) return die(st, "write");
  return 0;
}
