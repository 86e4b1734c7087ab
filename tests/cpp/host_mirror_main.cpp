// Drives the C++ host mirror (include/tarang_b200.hpp) the way the reference's
// Ifluid_main loop drives its classes: basis, FluidVF, IC, RK4 steps, energy,
// divergence and E(k).  Prints one JSON line; tests/test_cpp_host.py compares it
// with the same run through the Python binding.
#include <cstdio>
#include <vector>
#include <cmath>

#include "tarang_b200.hpp"

int main(int argc, char** argv) {
  using namespace tarang_b200;
  const int N = argc > 1 ? atoi(argv[1]) : 32;
  const int steps = argc > 2 ? atoi(argv[2]) : 5;
  ts_config c;
  ts_config_default(&c);
  c.N[0] = c.N[1] = c.N[2] = N;
  c.nu = 0.01;
  c.dt = 1e-3;
  try {
    FFF_PENCIL basis(c);
    FluidVF U(basis);
    std::vector<double> Eic(basis.no_shells());
    for (size_t s = 1; s < Eic.size(); ++s) Eic[s] = std::pow((double)s, 4) * std::exp(-2.0 * std::pow(s / 4.0, 2));
    U.Init_cond_energy_spectrum(Eic, 0, 0.5);
    const double e0 = U.Compute_total_energy();
    Time_advance_incompress::RK4(U, steps);
    const double e1 = U.Compute_total_energy();
    const double div = U.Compute_divergence_field();
    std::vector<double> Ek = basis.Compute_shell_spectrum(U.cvf(), 3);
    printf("{\"e0\": %.17g, \"e1\": %.17g, \"div\": %.17g, \"Ek\": [", e0, e1, div);
    for (size_t i = 0; i < Ek.size(); ++i) printf("%s%.17g", i ? ", " : "", Ek[i]);
    printf("]}\n");
  } catch (const ts_error& e) {
    fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
