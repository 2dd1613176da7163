// solver_stub.cu -- placeholder for the batched block solver entry points.
#include <cstring>
#include "common.cuh"
using namespace laph;
extern "C" {
void laph_solve_opts_default(laph_solve_opts* o) { std::memset(o, 0, sizeof *o); }
int laph_solver_create(laph_solver**, const laph_problem*, int, const laph_solve_opts*, int) { set_error("not built"); return LAPH_EINVAL; }
int laph_solver_destroy(laph_solver*) { return LAPH_OK; }
int laph_solver_set_links(laph_solver*, int, const double*, int, int) { return LAPH_EINVAL; }
int laph_solver_run(laph_solver*, laph_result*) { return LAPH_EINVAL; }
int laph_solver_get(laph_solver*, int, double*, double*, double*, int) { return LAPH_EINVAL; }
int laph_solver_timings(laph_solver*, double*) { return LAPH_EINVAL; }
int laph_solver_counters(laph_solver*, long long*) { return LAPH_EINVAL; }
}
