// C++ host mirror of the reference's hot-path interface over the C ABI.
//
// Same class and method names as anandogc/tarang (paths inside trunk/lib):
//   FluidVF                         fluid/fluid_base/FluidVF.h:73-180
//   FFF_PENCIL / SFF_PENCIL         basis/FFF/pencil/FFF_pencil.h:51, basis/SFF/pencil/SFF_pencil.h:52
//   SSF_PENCIL / SSS_PENCIL         basis/SSF/pencil/SSF_pencil.h, basis/SSS/pencil/SSS_pencil.h
//   Nlin_incompress::Compute_nlin   fluid/incompressible/nlin/Nlin.h:79
//   Time_advance_incompress::RK4    fluid/incompressible/time_advance/Time_advance.h:69-187
//   FluidSF                         fluid/fluid_base/FluidSF.h:42
//   Correlation::Get_Nusselt_no     fluid/fluid_base/Correlation.cc:144
//   EnergyTr::Compute_flux          fluid/incompressible/energytr/compute_flux.cc:51
// Ensemble and Adjoint have no reference counterpart.
// Differences from the reference, by design: fields live in device memory
// (one contiguous block per vector field, the reference's (Nx,Ny,Nz/2+1)
// layout per component), errors throw ts_error instead of exit(1), and the
// parity string that the reference passes through a global is an argument.
#pragma once
#include <cuda_runtime.h>

#include <complex>
#include <stdexcept>
#include <string>
#include <vector>

#include "tarang_b200.h"

namespace tarang_b200 {

struct ts_error : std::runtime_error {
  int status;
  ts_error(int s, const std::string& where)
      : std::runtime_error(where + ": status " + std::to_string(s) + " " + ts_last_error()), status(s) {}
};

inline void check(int s, const char* where) {
  if (s != TS_OK) throw ts_error(s, where);
}

// Owns a ts_plan: the basis object of the reference (FFF_PENCIL / SFF_PENCIL
// constructor + fftk.Init, FFF_pencil.cc:31-135).
class Universal {
 public:
  explicit Universal(const ts_config& c) : cfg_(c) {
    check(ts_plan_create(&cfg_, &plan_), "ts_plan_create");
    long long e = 0;
    int b = 0;
    check(ts_plan_sizes(plan_, &e, &b), "ts_plan_sizes");
    elems_ = e;
    bytes_ = b;
    check(ts_plan_num_shells(plan_, &nshells_), "ts_plan_num_shells");
  }
  ~Universal() {
    if (plan_) ts_plan_destroy(plan_);
  }
  Universal(const Universal&) = delete;
  Universal& operator=(const Universal&) = delete;

  ts_plan* plan() const { return plan_; }
  const ts_config& config() const { return cfg_; }
  long long elems_per_component() const { return elems_; }
  int bytes_per_complex() const { return bytes_; }
  int no_shells() const { return nshells_; }

  // Forward_transform / Inverse_transform (FFF_pencil_tr.cc:43-66): device pointers
  void Forward_transform(const void* Ar, void* A, const char* parity = "FFF", int ncomp = 1) {
    check(ts_fft_forward(plan_, parity, Ar, A, ncomp), "Forward_transform");
  }
  void Inverse_transform(const void* A, void* Ar, const char* parity = "FFF", int ncomp = 1) {
    check(ts_fft_inverse(plan_, parity, A, Ar, ncomp), "Inverse_transform");
  }
  // Compute_shell_spectrum (universal_energy.cc:279-366), summed over ncomp components
  std::vector<double> Compute_shell_spectrum(const void* A, int ncomp = 3) {
    std::vector<double> Ek(nshells_);
    check(ts_shell_spectrum(plan_, A, ncomp, Ek.data(), nshells_), "Compute_shell_spectrum");
    return Ek;
  }
  double Get_total_energy(const void* A, int ncomp = 1) {
    double e = 0;
    check(ts_energy(plan_, A, ncomp, &e), "Get_total_energy");
    return e;
  }
  // launch tuning: the fastest kernel candidate per pass class on this GPU
  // (ts_plan_autotune); returns the JSON timing report
  std::string Autotune(int reps = 3) {
    std::string rep(1 << 16, '\0');
    check(ts_plan_autotune(plan_, reps, &rep[0], rep.size()), "Autotune");
    rep.resize(rep.find('\0'));
    return rep;
  }
  ts_tuning Get_tuning() const {
    ts_tuning t;
    check(ts_plan_get_tuning(plan_, &t), "Get_tuning");
    return t;
  }
  void Set_tuning(const ts_tuning& t) { check(ts_plan_set_tuning(plan_, &t), "Set_tuning"); }

 private:
  ts_config cfg_;
  ts_plan* plan_ = nullptr;
  long long elems_ = 0;
  int bytes_ = 0;
  int nshells_ = 0;
};

class FFF_PENCIL : public Universal {
 public:
  explicit FFF_PENCIL(ts_config c) : Universal((c.basis = TS_BASIS_FFF, c)) {}
};

class SFF_PENCIL : public Universal {
 public:
  explicit SFF_PENCIL(ts_config c) : Universal((c.basis = TS_BASIS_SFF, c)) {}
};

// basis/SSF/pencil (sin/cos along x and y): transforms and the fluid RK4
class SSF_PENCIL : public Universal {
 public:
  explicit SSF_PENCIL(ts_config c) : Universal((c.basis = TS_BASIS_SSF, c)) {}
};

// basis/SSS/pencil (sin/cos along every axis, real coefficients): transforms and the fluid RK4
class SSS_PENCIL : public Universal {
 public:
  explicit SSS_PENCIL(ts_config c) : Universal((c.basis = TS_BASIS_SSS, c)) {}
};

// Velocity field: cvf (V1, V2, V3) and nlin (nlin1..3), each a contiguous
// device block of 3 components.
class FluidSF;

class FluidVF {
 public:
  explicit FluidVF(Universal& basis) : basis_(basis) {
    bytes_ = 3ull * basis.elems_per_component() * basis.bytes_per_complex();
    if (cudaMalloc(&cvf_, bytes_) != cudaSuccess || cudaMalloc(&nlin_, bytes_) != cudaSuccess)
      throw ts_error(TS_ERR_NOMEM, "FluidVF");
    cudaMemset(cvf_, 0, bytes_);
    cudaMemset(nlin_, 0, bytes_);
  }
  ~FluidVF() {
    cudaFree(cvf_);
    cudaFree(nlin_);
  }
  FluidVF(const FluidVF&) = delete;
  FluidVF& operator=(const FluidVF&) = delete;

  void* cvf() { return cvf_; }
  void* nlin() { return nlin_; }
  size_t bytes() const { return bytes_; }
  Universal& basis() { return basis_; }

  // Init_cond_energy_helicity_spectrum construction (init_cond_energy.cc:67-120)
  void Init_cond_energy_spectrum(const std::vector<double>& Eic, uint64_t seed, double energy) {
    check(ts_init_energy_spectrum(basis_.plan(), Eic.data(), (int)Eic.size(), seed, energy, cvf_),
          "Init_cond_energy_spectrum");
  }
  double Compute_total_energy() { return basis_.Get_total_energy(cvf_, 3); }
  double Compute_divergence_field() {
    double d = 0;
    check(ts_max_div(basis_.plan(), cvf_, &d), "Compute_divergence_field");
    return d;
  }
  void Copy_to_host(void* host) { cudaMemcpy(host, cvf_, bytes_, cudaMemcpyDeviceToHost); }
  void Copy_from_host(const void* host) { cudaMemcpy(cvf_, host, bytes_, cudaMemcpyHostToDevice); }
  // the slaved field of a PRZERO / PRINFTY run (FluidVF.cc:228-272); defined after FluidSF
  inline void Zero_Prandtl_number_compute_temperature(FluidSF& T);
  inline void Infinite_Prandtl_number_compute_velocity(FluidSF& T);

 private:
  Universal& basis_;
  void* cvf_ = nullptr;
  void* nlin_ = nullptr;
  size_t bytes_ = 0;
};

struct Nlin_incompress {
  // dealias U.cvf in place, U.nlin = F[(u.grad)u] (compute_nlin.cc:58-109)
  static void Compute_nlin(FluidVF& U) { check(ts_nlin(U.basis().plan(), U.cvf(), U.nlin()), "Compute_nlin"); }
};

// Scalar field (the RBC temperature): csf F, one device component.
class FluidSF {
 public:
  explicit FluidSF(Universal& basis) : basis_(basis) {
    bytes_ = basis.elems_per_component() * basis.bytes_per_complex();
    if (cudaMalloc(&csf_, bytes_) != cudaSuccess) throw ts_error(TS_ERR_NOMEM, "FluidSF");
    cudaMemset(csf_, 0, bytes_);
  }
  ~FluidSF() { cudaFree(csf_); }
  FluidSF(const FluidSF&) = delete;
  FluidSF& operator=(const FluidSF&) = delete;

  void* csf() { return csf_; }
  size_t bytes() const { return bytes_; }
  Universal& basis() { return basis_; }
  // amplitude amp, uniform random phases on the modes with |K|/kfactor <= kmax
  void Init_cond_perturbation(double amp, double kmax, uint64_t seed) {
    check(ts_init_temperature_perturbation(basis_.plan(), amp, kmax, seed, csf_), "Init_cond_perturbation");
  }
  double Compute_total_energy() { return basis_.Get_total_energy(csf_, 1); }
  void Copy_to_host(void* host) { cudaMemcpy(host, csf_, bytes_, cudaMemcpyDeviceToHost); }

 private:
  Universal& basis_;
  void* csf_ = nullptr;
  size_t bytes_ = 0;
};

// T = U.V1 / K^2 (the plan's Pr_option must be PRZERO)
inline void FluidVF::Zero_Prandtl_number_compute_temperature(FluidSF& T) {
  check(ts_rbc_slave(basis_.plan(), cvf_, T.csf()), "Zero_Prandtl_number_compute_temperature");
}
// U = vs P(T x) / K^2 (the plan's Pr_option must be PRINFTY)
inline void FluidVF::Infinite_Prandtl_number_compute_velocity(FluidSF& T) {
  check(ts_rbc_slave(basis_.plan(), cvf_, T.csf()), "Infinite_Prandtl_number_compute_velocity");
}

struct Time_advance_incompress {
  // RK4(U,P,F) + strong reality condition when the plan enables it (RK.cc:91-170, Time_advance.cc:59-60)
  static void RK4(FluidVF& U, int nsteps = 1) { check(ts_rk4_step(U.basis().plan(), U.cvf(), nsteps), "RK4"); }
  // RK4(U,W,P,F) for incompressible MHD (RK_VF_MHD.cc:126), W = B, FFF, no force;
  // eta = the basis config's kappa
  static void RK4(FluidVF& U, FluidVF& W, int nsteps = 1) {
    check(ts_rk4_step_mhd(U.basis().plan(), U.cvf(), W.cvf(), nsteps), "RK4");
  }
  // RK4(U,T,P,F) (RK_SF.cc:97): RBC on the SFF basis (the plan's Pr_option / Uscaling), or a
  // passive scalar (kind SCALAR_INCOMPRESS, no force) on the FFF basis
  static void RK4(FluidVF& U, FluidSF& T, int nsteps = 1) {
    ts_plan* p = U.basis().plan();
    if (U.basis().config().basis != TS_BASIS_FFF) check(ts_rk4_step_rbc(p, U.cvf(), T.csf(), nsteps), "RK4");
    else check(ts_rk4_step_scalar(p, U.cvf(), T.csf(), nsteps), "RK4");
  }
};

struct Correlation {
  // Get_Nusselt_no (Correlation.cc:144-176): nu0 + nuc <U1, T> with the factors of the plan's
  // scaling (PRLARGE / ULARGE: 1 + 2 sqrt(Ra Pr) <U1, T>)
  static double Get_Nusselt_no(FluidVF& U, FluidSF& T) {
    double nu = 0;
    check(ts_nusselt(U.basis().plan(), U.cvf(), T.csf(), &nu), "Get_Nusselt_no");
    return nu;
  }
};

struct EnergyTr {
  // Compute_flux(U) (compute_flux.cc:51): Pi(R_i) for every sphere radius
  static std::vector<double> Compute_flux(FluidVF& U, const std::vector<double>& radii) {
    std::vector<double> Pi(radii.size());
    check(ts_flux(U.basis().plan(), U.cvf(), radii.data(), (int)radii.size(), Pi.data()), "Compute_flux");
    return Pi;
  }
};

// Many RBC runs of uneven sizes advanced together (no reference counterpart:
// the reference runs one field per MPI job).
class Ensemble {
 public:
  Ensemble(const ts_config& base, const std::vector<ts_member>& members) {
    check(ts_ensemble_create(&base, members.data(), (int)members.size(), &ens_), "ts_ensemble_create");
    n_ = members.size();
  }
  ~Ensemble() {
    if (ens_) ts_ensemble_destroy(ens_);
  }
  Ensemble(const Ensemble&) = delete;
  Ensemble& operator=(const Ensemble&) = delete;
  void Init_temperature(double amp, double kmax, uint64_t seed) {
    check(ts_ensemble_init_temperature(ens_, amp, kmax, seed), "Init_temperature");
  }
  void Run(int nsteps) { check(ts_ensemble_run(ens_, nsteps), "ts_ensemble_run"); }
  std::string Autotune(int reps = 3) {
    std::string rep(1 << 18, '\0');
    check(ts_ensemble_autotune(ens_, reps, &rep[0], rep.size()), "Ensemble::Autotune");
    rep.resize(rep.find('\0'));
    return rep;
  }
  std::vector<double> Nusselt() {
    std::vector<double> nu(n_);
    check(ts_ensemble_nusselt(ens_, nu.data()), "ts_ensemble_nusselt");
    return nu;
  }

 private:
  ts_ensemble* ens_ = nullptr;
  size_t n_ = 0;
};

// Discrete adjoint of the FFF rotational IF-RK4 step (no reference counterpart).
// Window(u_start, n, lam): lam enters as the cotangent of the state n steps after
// u_start and leaves as the cotangent of u_start; the work buffer is owned here.
class Adjoint {
 public:
  explicit Adjoint(Universal& basis, int window) : basis_(basis), window_(window) {
    check(ts_adjoint_work_bytes(basis.plan(), window, &bytes_), "ts_adjoint_work_bytes");
    if (cudaMalloc(&work_, bytes_) != cudaSuccess) throw ts_error(TS_ERR_NOMEM, "Adjoint");
  }
  ~Adjoint() { cudaFree(work_); }
  Adjoint(const Adjoint&) = delete;
  Adjoint& operator=(const Adjoint&) = delete;
  void Window(const void* u_start, int nsteps, void* lam) {
    if (nsteps > window_) throw ts_error(TS_ERR_ARG, "Adjoint::Window: nsteps above the window");
    check(ts_adjoint_window(basis_.plan(), u_start, nsteps, lam, work_, bytes_), "ts_adjoint_window");
  }

 private:
  Universal& basis_;
  int window_;
  size_t bytes_ = 0;
  void* work_ = nullptr;
};

}  // namespace tarang_b200
