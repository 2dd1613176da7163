// ref_dump.cpp -- test infrastructure: a driver around the reference's own
// parameter parser (IO::set_values, modules/par_io.cpp:8-131) and lookup
// tables (Nav::init / get_up / get_dn, modules/navigation.cpp:27-88), the two
// parts of the path that compile from the reference's sources without Eigen,
// PETSc, SLEPc or c-lime.  Built into oracle/_ref/ref_dump by `make ref` from
// the sources where they lie; the tests compare laph_parse_parameters and the
// oracle's site indexing with what it prints.
//
//   ref_dump params FILE   one JSON object: the IO getters after set_values
//                          ("threw": true if set_values threw)
//   ref_dump nav FILE      {"L": L, "up": [[x, y, z] per site], "dn": [...]}
//                          after set_values(FILE) and Nav::init()
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>

#include "navigation.h"
#include "par_io.h"

namespace {

void json_str(const char* key, const std::string& v, bool comma) {
  std::printf("\"%s\": \"", key);
  for (char c : v) {
    if (c == '"' || c == '\\') std::printf("\\%c", c);
    else if ((unsigned char)c < 0x20) std::printf("\\u%04x", (unsigned char)c);
    else std::putchar(c);
  }
  std::printf("\"%s", comma ? ", " : "");
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3 || (std::strcmp(argv[1], "params") != 0 && std::strcmp(argv[1], "nav") != 0)) {
    std::fprintf(stderr, "usage: ref_dump params|nav FILE\n");
    return 2;
  }
  // set_values loops until eof(), which a stream that failed to open never reaches
  FILE* probe = std::fopen(argv[2], "r");
  if (!probe) {
    std::fprintf(stderr, "ref_dump: cannot open %s\n", argv[2]);
    return 2;
  }
  std::fclose(probe);
  IO* io = IO::getInstance();
  try {
    io->set_values(argv[2]);
  } catch (const std::exception& e) {
    std::printf("{\"threw\": true, \"what\": \"%s\"}\n", e.what());
    return 0;
  }
  if (std::strcmp(argv[1], "params") == 0) {
    std::printf("{\"threw\": false, ");
    const char* ints[] = {"LT", "LX", "NEV", "iter", "DEG", "OMP_THRDS", "V3", "MAT_ENTRIES", "V_TS", "V4_LIME"};
    for (const char* k : ints) std::printf("\"%s\": %d, ", k, io->get_int(k));
    const char* floats[] = {"alpha_1", "alpha_1_i", "alpha_1_f", "alpha_2", "alpha_2_i", "alpha_2_f",
                            "lambda_l", "lambda_c"};
    for (const char* k : floats) {
      const double v = io->get_float(k);
      // non-finite values in the spellings Python's json module reads
      if (std::isnan(v)) std::printf("\"%s\": NaN, ", k);
      else if (std::isinf(v)) std::printf("\"%s\": %sInfinity, ", k, v < 0 ? "-" : "");
      else std::printf("\"%s\": %.17g, ", k, v);
    }
    json_str("conf", io->get_path("conf"), true);
    json_str("res", io->get_path("res"), true);
    json_str("in_path", io->get_path("in_path"), true);
    json_str("phase_path", io->get_path("phase_path"), true);
    json_str("ev1", io->get_path("ev1"), true);
    json_str("ev2", io->get_path("ev2"), false);
    std::printf("}\n");
    return 0;
  }
  const int L = io->get_int("LX"), V3 = io->get_int("V3");
  if (L < 1 || V3 != L * L * L) {
    std::fprintf(stderr, "ref_dump: LX must be set\n");
    return 2;
  }
  Nav* nav = Nav::getInstance();
  nav->init();
  std::printf("{\"L\": %d, \"up\": [", L);
  for (int i = 0; i < V3; ++i)
    std::printf("%s[%d, %d, %d]", i ? ", " : "", nav->get_up(i, 0), nav->get_up(i, 1), nav->get_up(i, 2));
  std::printf("], \"dn\": [");
  for (int i = 0; i < V3; ++i)
    std::printf("%s[%d, %d, %d]", i ? ", " : "", nav->get_dn(i, 0), nav->get_dn(i, 1), nav->get_dn(i, 2));
  std::printf("]}\n");
  return 0;
}
