// Drives the C++ host mirror (include/tarang_b200.hpp) the way the reference's
// main loops drive their classes: basis, fields, IC, RK4 steps, diagnostics.
// Usage: host_mirror <mode> [N] [steps], mode one of
//   fff       FFF_PENCIL + FluidVF: energy, divergence, E(k), Pi(R)
//   fff_tuned the same after Universal::Autotune
//   rbc       SFF_PENCIL + FluidVF + FluidSF: energies and Nusselt number
//   rbc_sss   SSS_PENCIL + FluidVF + FluidSF (FP64): a roll set from the host, RK4(U, T),
//             energies and Nusselt number
//   ensemble  two RBC members of different sizes advanced together: Nusselt numbers
//   adjoint   FFF rotational FP64: cotangent of the start state of an nsteps window
//   mhd       FFF incompressible MHD: energies of U and B, max |div B|
// Prints one JSON line; tests/test_cpp_host.py compares it with the same run
// through the Python binding.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "tarang_b200.hpp"

using namespace tarang_b200;

static void print_list(const char* key, const std::vector<double>& v, bool last) {
  printf("\"%s\": [", key);
  for (size_t i = 0; i < v.size(); ++i) printf("%s%.17g", i ? ", " : "", v[i]);
  printf("]%s", last ? "" : ", ");
}

static std::vector<double> k4_gauss(int nsh, double k0) {
  std::vector<double> E(nsh);
  for (int s = 1; s < nsh; ++s) E[s] = std::pow((double)s, 4) * std::exp(-2.0 * std::pow(s / k0, 2));
  return E;
}

static int run_fff(int N, int steps, bool tuned) {
  ts_config c;
  ts_config_default(&c);
  c.N[0] = c.N[1] = c.N[2] = N;
  c.nu = 0.01;
  c.dt = 1e-3;
  FFF_PENCIL basis(c);
  FluidVF U(basis);
  U.Init_cond_energy_spectrum(k4_gauss(basis.no_shells(), 4.0), 0, 0.5);
  // the tuned kernels must give the rule's results to rounding: the default
  // tuning here; `fff_tuned` runs the autotuner first
  if (tuned) basis.Autotune(1);
  const double e0 = U.Compute_total_energy();
  Time_advance_incompress::RK4(U, steps);
  const double e1 = U.Compute_total_energy();
  const double div = U.Compute_divergence_field();
  std::vector<double> Ek = basis.Compute_shell_spectrum(U.cvf(), 3);
  std::vector<double> Pi = EnergyTr::Compute_flux(U, {2.0, 4.0, 8.0});
  printf("{\"e0\": %.17g, \"e1\": %.17g, \"div\": %.17g, ", e0, e1, div);
  print_list("Ek", Ek, false);
  print_list("Pi", Pi, true);
  printf("}\n");
  return 0;
}

static int run_rbc(int N, int steps) {
  const double Ra = 1e5, Pr = 1.0;
  ts_config c;
  ts_config_default(&c);
  c.N[0] = c.N[1] = c.N[2] = N;
  c.kfactor[0] = M_PI;
  c.kfactor[1] = c.kfactor[2] = 2 * M_PI;
  c.precision = TS_F32;
  c.Ra = Ra;
  c.Pr = Pr;
  c.nu = std::sqrt(Pr / Ra);
  c.kappa = 1 / std::sqrt(Pr * Ra);
  c.dt = 1e-3;
  SFF_PENCIL basis(c);
  FluidVF U(basis);
  FluidSF T(basis);
  T.Init_cond_perturbation(0.01, 4.0, 3);
  Time_advance_incompress::RK4(U, T, steps);
  const double eu = U.Compute_total_energy();
  const double et = T.Compute_total_energy();
  const double nu = Correlation::Get_Nusselt_no(U, T);
  printf("{\"eu\": %.17g, \"eT\": %.17g, \"Nu\": %.17g}\n", eu, et, nu);
  return 0;
}

// RBC on the SSS basis: real coefficients in the padded layout (N + 2 reals per z line),
// u_x = 0.1 and theta = 0.05 on mode (1, 1, 1), u_y balancing the divergence, and a
// second theta mode (2, 1, 0), copied in from the host
static int run_rbc_sss(int N, int steps) {
  const double Ra = 1e5, Pr = 1.0;
  ts_config c;
  ts_config_default(&c);
  c.N[0] = c.N[1] = c.N[2] = N;
  c.kfactor[0] = M_PI;
  c.kfactor[1] = c.kfactor[2] = M_PI / std::sqrt(2.0);
  c.precision = TS_F64;
  c.Ra = Ra;
  c.Pr = Pr;
  c.nu = std::sqrt(Pr / Ra);
  c.kappa = 1 / std::sqrt(Pr * Ra);
  c.dt = 1e-3;
  SSS_PENCIL basis(c);
  FluidVF U(basis);
  FluidSF T(basis);
  const size_t line = N + 2, nreal = (size_t)N * N * line;
  std::vector<double> u(3 * nreal, 0.0), t(nreal, 0.0);
  auto at = [&](int lx, int ly, int lz) { return ((size_t)lx * N + ly) * line + lz; };
  u[at(1, 1, 1)] = 0.1;
  u[nreal + at(1, 1, 1)] = -0.1 * c.kfactor[0] / c.kfactor[1];
  t[at(1, 1, 1)] = 0.05;
  t[at(2, 1, 0)] = 0.02;
  if (cudaMemcpy(U.cvf(), u.data(), u.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(T.csf(), t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    fprintf(stderr, "cudaMemcpy failed\n");
    return 1;
  }
  Time_advance_incompress::RK4(U, T, steps);
  const double eu = U.Compute_total_energy();
  const double et = T.Compute_total_energy();
  const double nu = Correlation::Get_Nusselt_no(U, T);
  printf("{\"eu\": %.17g, \"eT\": %.17g, \"Nu\": %.17g}\n", eu, et, nu);
  return 0;
}

static int run_ensemble(int N, int steps) {
  ts_config c;
  ts_config_default(&c);
  c.basis = TS_BASIS_SFF;
  c.kfactor[0] = M_PI;
  c.kfactor[1] = c.kfactor[2] = 2 * M_PI;
  c.precision = TS_F32;
  c.dt = 1e-4;
  c.force_type = TS_FORCE_RBC;
  std::vector<ts_member> members(2);
  const int sizes[2] = {N, N + N / 2};
  const double ra[2] = {1e5, 1e6};
  for (int m = 0; m < 2; ++m) {
    for (int i = 0; i < 3; ++i) members[m].N[i] = sizes[m];
    members[m].Ra = ra[m];
    members[m].Pr = 1.0;
  }
  Ensemble ens(c, members);
  ens.Init_temperature(0.01, 4.0, 7);
  ens.Run(steps);
  printf("{");
  print_list("Nu", ens.Nusselt(), true);
  printf("}\n");
  return 0;
}

static int run_mhd(int N, int steps) {
  ts_config c;
  ts_config_default(&c);
  c.N[0] = c.N[1] = c.N[2] = N;
  c.nu = 0.01;
  c.kappa = 0.02;  // eta
  c.dt = 1e-3;
  c.dealias_mode = TS_DEALIAS_TWO_THIRDS;
  FFF_PENCIL basis(c);
  FluidVF U(basis), W(basis);
  U.Init_cond_energy_spectrum(k4_gauss(basis.no_shells(), 4.0), 0, 0.5);
  W.Init_cond_energy_spectrum(k4_gauss(basis.no_shells(), 3.0), 1, 0.3);
  Time_advance_incompress::RK4(U, W, steps);
  printf("{\"eu\": %.17g, \"eb\": %.17g, \"divb\": %.17g}\n", U.Compute_total_energy(), W.Compute_total_energy(),
         W.Compute_divergence_field());
  return 0;
}

static int run_adjoint(int N, int steps) {
  ts_config c;
  ts_config_default(&c);
  c.N[0] = c.N[1] = c.N[2] = N;
  c.nlin_form = TS_NLIN_ROTATIONAL;
  c.dealias_mode = TS_DEALIAS_TWO_THIRDS;
  c.nu = 0.01;
  c.dt = 1e-3;
  FFF_PENCIL basis(c);
  FluidVF U(basis);
  FluidVF Lam(basis);
  U.Init_cond_energy_spectrum(k4_gauss(basis.no_shells(), 4.0), 0, 0.5);
  // cotangent of the final state: the state itself (the gradient of an energy-like loss)
  if (cudaMemcpy(Lam.cvf(), U.cvf(), U.bytes(), cudaMemcpyDeviceToDevice) != cudaSuccess)
    throw ts_error(TS_ERR_CUDA, "cudaMemcpy");
  Adjoint adj(basis, steps);
  adj.Window(U.cvf(), steps, Lam.cvf());
  check(ts_plan_status(basis.plan()), "ts_plan_status");
  const double el = basis.Get_total_energy(Lam.cvf(), 3);
  std::vector<double> Ek = basis.Compute_shell_spectrum(Lam.cvf(), 3);
  printf("{\"elam\": %.17g, ", el);
  print_list("Ek", Ek, true);
  printf("}\n");
  return 0;
}

int main(int argc, char** argv) {
  const char* mode = argc > 1 ? argv[1] : "fff";
  const int N = argc > 2 ? atoi(argv[2]) : 32;
  const int steps = argc > 3 ? atoi(argv[3]) : 5;
  try {
    if (!strcmp(mode, "fff")) return run_fff(N, steps, false);
    if (!strcmp(mode, "fff_tuned")) return run_fff(N, steps, true);
    if (!strcmp(mode, "rbc")) return run_rbc(N, steps);
    if (!strcmp(mode, "rbc_sss")) return run_rbc_sss(N, steps);
    if (!strcmp(mode, "ensemble")) return run_ensemble(N, steps);
    if (!strcmp(mode, "adjoint")) return run_adjoint(N, steps);
    if (!strcmp(mode, "mhd")) return run_mhd(N, steps);
    fprintf(stderr, "unknown mode %s\n", mode);
    return 2;
  } catch (const ts_error& e) {
    fprintf(stderr, "%s\n", e.what());
    return 1;
  }
}
