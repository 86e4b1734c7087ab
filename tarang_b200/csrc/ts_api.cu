// C ABI of the B200 pseudo-spectral IF-RK4 path (declared in include/tarang_b200.h).
//
// The plan replaces the reference's FFF_PENCIL basis object + FFTK plan
// (basis/FFF/pencil/FFF_pencil.cc:31-277) and the static work arrays of
// Time_advance_incompress::RK4 (RK.cc:95-96: Vcopy, tot_Vrhs).  The caller's
// u_hat is the state (the reference's U.cvf); the plan owns the stage field,
// the RK accumulator, six product / transform work fields and twiddle tables.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>
#include <stdio.h>
#include <mutex>
#include <vector>
#include <string>
#include "tarang_b200.h"
#include "ts_launch.h"

namespace ts {
long long g_launches = 0;
bool size_supported(int n) { return n == 16 || n == 32 || n == 64 || n == 128 || n == 256 || n == 512 || n == 1024; }
}  // namespace ts

using namespace ts;

static thread_local std::string g_last_error;

#define CK(x)                                                   \
  do {                                                          \
    cudaError_t e_ = (x);                                       \
    if (e_ != cudaSuccess) {                                    \
      g_last_error = std::string(#x) + ": " + cudaGetErrorString(e_); \
      return (int)(e_ == cudaErrorMemoryAllocation ? TS_ERR_NOMEM : TS_ERR_CUDA); \
    }                                                           \
  } while (0)

#define CKS(x)                          \
  do {                                  \
    int s_ = (x);                       \
    if (s_ != TS_OK) return s_;         \
  } while (0)

struct ts_plan {
  ts_config cfg;
  Geo g;
  int prec;           // 0 f64, 1 f32
  size_t cb;          // bytes per complex
  cudaStream_t st = nullptr;
  void* Ucur = nullptr;
  void* tot = nullptr;
  void* P = nullptr;  // nP components of transform / product work fields
  int nP = 0;
  int nS = 0;         // components of the stage field Ucur and the accumulator tot
  void* twx = nullptr;
  void* twy = nullptr;
  void* twz = nullptr;
  void* fcube = nullptr;
  int fkm = 0;
  double* esup = nullptr;
  double* hsup = nullptr;
  double* mis_d = nullptr;
  int nsup = 0;
  std::vector<double> mis;  // modes_in_shell (host)
  int nshells = 0;
  double* dscr = nullptr;   // diagnostics scratch
  size_t dscr_n = 0;
  void* stage_u = nullptr;  // staging for host pointers (3 components)
  void* stage_t = nullptr;  // staging for host pointers (1 component)
  void* stage_b = nullptr;  // staging for host pointers (3 components, the MHD field B)
  int* err_d = nullptr;     // device error word (bounded waits that gave up)
  int* err_h = nullptr;     // pinned copy, refreshed after every step call
  double rbc_cu = 1, rbc_cT = 1;    // RBC buoyancy coefficients U.F1 = cu T, T.F = cT U.V1
  double rbc_nu0 = 1, rbc_nuc = 0;  // Nusselt number nu0 + nuc <U.V1, T>
  int rbc_slave = 0;                // 1: PRZERO (T slaved to U), 2: PRINFTY (U slaved to T)
  double rbc_vs = 0;                // PRINFTY: factor of the slaved velocity
  double* eax[3] = {nullptr, nullptr, nullptr};  // per-axis exp(-nu dt K_i^2 / 2)
  float2* eaxf[3] = {nullptr, nullptr, nullptr}; // the same as FP32 (hi, lo) pairs
  double* eaxT[3] = {nullptr, nullptr, nullptr}; // per-axis exp(-kappa dt K_i^2 / 2) (SFF scalar)
  void* twq = nullptr;      // SFF, SSF: exp(-2 pi i j / (4 Nx)), j < 4 Nx
  void* twqy = nullptr;     // SSF, SSS: exp(-2 pi i j / (4 Ny)), j < 4 Ny
  void* twqz = nullptr;     // SSS: exp(-2 pi i j / (4 Nz)), j < 4 Nz
  // per-kernel-class CUDA event timing (ts_profile_*)
  bool prof = false;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  struct ProfRec {
    int cls;
    double bytes;  // algorithmic bytes of the bracketed launches (< 0: the class's static model)
    cudaEvent_t b, e;
  };
  std::vector<ProfRec> ev_rec;
  double prof_ms[TS_KCLASS_COUNT] = {0};
  long long prof_n[TS_KCLASS_COUNT] = {0};
  double prof_bytes[TS_KCLASS_COUNT] = {0};  // summed per-launch algorithmic bytes
  long long prof_nb[TS_KCLASS_COUNT] = {0};  // launches whose bytes were recorded
};

// ---------------------------------------------------------------------------
// profiling: events around each launch of a kernel class
// ---------------------------------------------------------------------------
static cudaEvent_t prof_event(ts_plan* p) {
  if (p->ev_used == p->ev_pool.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    p->ev_pool.push_back(e);
  }
  return p->ev_pool[p->ev_used++];
}

static void prof_collect(ts_plan* p) {
  if (p->ev_rec.empty()) return;
  cudaStreamSynchronize(p->st);
  for (auto& r : p->ev_rec) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, r.b, r.e) == cudaSuccess) {
      p->prof_ms[r.cls] += ms;
      p->prof_n[r.cls] += 1;
      if (r.bytes >= 0) {
        p->prof_bytes[r.cls] += r.bytes;
        p->prof_nb[r.cls] += 1;
      }
    }
  }
  p->ev_rec.clear();
  p->ev_used = 0;
}

// bytes: the algorithmic bytes of the launches the scope brackets (every field
// element they must read or write, once); < 0 leaves the class's static model
struct ProfScope {
  ts_plan* p;
  int cls;
  double bytes;
  cudaEvent_t b = nullptr;
  ProfScope(ts_plan* p_, int c, double by = -1.0) : p(p_), cls(c), bytes(by) {
    if (p->prof) {
      if (p->ev_used + 2 > 8192) prof_collect(p);
      b = prof_event(p);
      if (b) cudaEventRecord(b, p->st);
    }
  }
  ~ProfScope() {
    if (p->prof && b) {
      cudaEvent_t e = prof_event(p);
      if (e) {
        cudaEventRecord(e, p->st);
        p->ev_rec.push_back({cls, bytes, b, e});
      }
    }
  }
};

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
// Scaling-dependent RBC coefficients (non-Chebyshev bases): diss_coefficients nu, kappa
// (Iscalar_main.cc:52-92), buoyancy U.Force1 += cu T, T.Force += cT U.V1
// (compute_force_RBC.cc:104-150) and the Nusselt number nu0 + nuc <U.V1, T>
// (Correlation::Get_Nusselt_no, Correlation.cc:144-176).  PRZERO / PRINFTY slave one
// field to the other (Single_time_step_RBC, Tadvance_functions.cc:380-395): T = U.V1 / K^2
// (no T force, kappa = 0), or U = vs P(T x) / K^2 (no U force) with the velocity factor
// vs of FluidVF.cc:259-271.
static int rbc_coefficients(int pr_option, int uscaling, double Ra, double Pr, double* nu, double* kappa, double* cu,
                            double* cT, double* nu0, double* nuc, double* vs = nullptr) {
  if (uscaling != TS_U_LARGE && uscaling != TS_U_SMALL) return TS_ERR_ARG;
  const bool small = uscaling == TS_U_SMALL;
  if (vs) *vs = 0;
  if (pr_option == TS_PR_LARGE) {
    *nu = small ? Pr : sqrt(Pr / Ra);
    *kappa = small ? 1.0 : 1.0 / sqrt(Pr * Ra);
    *cu = small ? Ra * Pr : 1.0;
    *cT = 1.0;
    *nu0 = 1.0;
    *nuc = small ? 2.0 : 2.0 * sqrt(Ra * Pr);
    return TS_OK;
  }
  if (pr_option == TS_PR_SMALL) {
    *nu = small ? 1.0 : sqrt(Pr / Ra);
    *kappa = small ? 1.0 / Pr : 1.0 / sqrt(Pr * Ra);
    *cu = small ? Ra : Pr;
    *cT = 1.0 / Pr;
    *nu0 = 1.0;
    *nuc = small ? 2.0 * Pr * Pr : 2.0 * Pr * sqrt(Ra * Pr);
    return TS_OK;
  }
  if (pr_option == TS_PR_ZERO) {
    // the buoyancy of the PRSMALL branch; Nu reports 2 <U.V1, T> (Nu = 1 at Pr = 0)
    *nu = 1.0;
    *kappa = 0.0;
    *cu = small ? Ra : Pr;
    *cT = 0.0;
    *nu0 = 0.0;
    *nuc = 2.0;
    return TS_OK;
  }
  if (pr_option == TS_PR_INFTY) {
    *nu = small ? Pr : 1.0 / sqrt(Ra);
    *kappa = small ? 1.0 : 1.0 / sqrt(Ra);
    *cu = 0.0;
    *cT = 1.0;
    *nu0 = 1.0;
    *nuc = small ? 2.0 : 2.0 * sqrt(Ra);
    if (vs) *vs = small ? Ra : sqrt(Ra);
    return TS_OK;
  }
  return TS_ERR_ARG;
}

// the status of the plan's health word as last copied to the host (err_h)
static int health_status(ts_plan* p) {
  if (*p->err_h & HEALTH_TIMEOUT) {
    g_last_error = "a bounded device wait gave up (a bulk copy never arrived)";
    return TS_ERR_TIMEOUT;
  }
  if (*p->err_h & HEALTH_NONFINITE) {
    g_last_error = "a step wrote a NaN or Inf into the state";
    return TS_ERR_NAN;
  }
  return TS_OK;
}
static bool is_device_ptr(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

template <typename T>
static int upload_twiddles(int L, void** dst) {
  // exp(-2 pi i m / L), evaluated in double and rounded once to T
  std::vector<T> h(2 * L);
  for (int m = 0; m < L; ++m) {
    const double a = -2.0 * M_PI * (double)m / (double)L;
    h[2 * m] = (T)cos(a);
    h[2 * m + 1] = (T)sin(a);
  }
  CK(cudaMalloc(dst, sizeof(T) * 2 * L));
  CK(cudaMemcpy(*dst, h.data(), sizeof(T) * 2 * L, cudaMemcpyHostToDevice));
  return TS_OK;
}

static void compute_modes_in_shell(ts_plan* p) {
  // Compute_modes_in_shell_array (universal_basic.cc:104-143): full box count
  const int Nx = p->g.Nx, Ny = p->g.Ny, Nz = p->g.Nz;
  const double* kf = p->g.kf;
  // Min_radius_outside of the basis (FFF_pencil_inline.h:497-504, SFF_pencil_inline.h:423-430,
  // SSF_pencil_inline.h:444-451, SSS_pencil_inline.h:469-476)
  int kmax;
  if (p->g.basis == 0)
    kmax = (int)ceil(sqrt(pow((Nx / 2) * kf[0], 2) + pow((Ny / 2) * kf[1], 2) + pow((Nz / 2) * kf[2], 2)));
  else if (p->g.basis == 2)
    kmax = (int)ceil(sqrt(pow((Nx - 1) * kf[0], 2) + pow((Ny - 1) * kf[1], 2) + pow((Nz / 2) * kf[2], 2)));
  else if (p->g.basis == 3)
    kmax = (int)ceil(sqrt(pow((Nx - 1) * kf[0], 2) + pow((Ny - 1) * kf[1], 2) + pow((Nz - 1) * kf[2], 2)));
  else
    kmax = (int)ceil(sqrt(pow((Nx - 1) * kf[0], 2) + pow((Ny / 2) * kf[1], 2) + pow((Nz / 2) * kf[2], 2)));
  p->nshells = kmax + 1;
  const int kxm = Nx / 2, kym = Ny / 2, kzm = Nz / 2;
  int top = kmax + 2;
  {
    const double m = sqrt(pow(kxm * kf[0], 2) + pow(kym * kf[1], 2) + pow(kzm * kf[2], 2));
    if ((int)ceil(m) + 2 > top) top = (int)ceil(m) + 2;
  }
  p->mis.assign(top, 0.0);
  for (int kx = -kxm + 1; kx <= kxm; ++kx)
    for (int ky = -kym + 1; ky <= kym; ++ky)
      for (int kz = -kzm + 1; kz <= kzm; ++kz) {
        const double K = sqrt(pow(kx * kf[0], 2) + pow(ky * kf[1], 2) + pow(kz * kf[2], 2));
        p->mis[(int)ceil(K)] += 1;
      }
}

static int ensure_scratch(ts_plan* p, size_t n) {
  if (p->dscr_n >= n) return TS_OK;
  if (p->dscr) cudaFree(p->dscr);
  p->dscr = nullptr;
  p->dscr_n = 0;
  CK(cudaMalloc(&p->dscr, n * sizeof(double)));
  p->dscr_n = n;
  return TS_OK;
}

static int ensure_stage(void** buf, size_t bytes) {
  if (*buf) return TS_OK;
  CK(cudaMalloc(buf, bytes));
  return TS_OK;
}

// Integrating-factor tables: E(1/2)(K) = exp(-nu dt K^2 / 2) factorises over the
// axes, exp(-nu dt/2 Kx^2) exp(-nu dt/2 Ky^2) exp(-nu dt/2 Kz^2) (FP64)
// tabf (optional): the same factors as FP32 pairs hi = fl32(x), lo = fl32(x - hi)
static int upload_if_tables(ts_plan* p, double nu, double dt, double** tab, float2** tabf = nullptr) {
  const Geo& g = p->g;
  // SSS: real z coefficients kz = lz < Nz
  const int n[3] = {g.Nx, g.Ny, g.basis == TS_BASIS_SSS ? g.Nz : g.Hz};
  for (int ax = 0; ax < 3; ++ax) {
    std::vector<double> h(n[ax]);
    for (int l = 0; l < n[ax]; ++l) {
      int k;
      if (ax == 0) k = g.basis == 0 ? (l <= g.Nx / 2 ? l : l - g.Nx) : l;
      else if (ax == 1) k = g.basis >= TS_BASIS_SSF ? l : (l <= g.Ny / 2 ? l : l - g.Ny);
      else k = l;
      const double K = k * g.kf[ax];
      h[l] = exp(-nu * 0.5 * dt * (K * K));
    }
    if (!tab[ax]) CK(cudaMalloc(&tab[ax], n[ax] * sizeof(double)));
    CK(cudaMemcpy(tab[ax], h.data(), n[ax] * sizeof(double), cudaMemcpyHostToDevice));
    if (tabf) {
      std::vector<float2> hf(n[ax]);
      for (int l = 0; l < n[ax]; ++l) {
        hf[l].x = (float)h[l];
        hf[l].y = (float)(h[l] - (double)hf[l].x);
      }
      if (!tabf[ax]) CK(cudaMalloc(&tabf[ax], n[ax] * sizeof(float2)));
      CK(cudaMemcpy(tabf[ax], hf.data(), n[ax] * sizeof(float2), cudaMemcpyHostToDevice));
    }
  }
  return TS_OK;
}

// dispatch a Launch<T>::fn call on the plan's precision
#define LAUNCH(p, fn, ...) \
  ((p)->prec == 1 ? Launch<float>::fn(__VA_ARGS__) : Launch<double>::fn(__VA_ARGS__))

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

void ts_config_default(ts_config* c) {
  memset(c, 0, sizeof(*c));
  c->basis = TS_BASIS_FFF;
  c->N[0] = c->N[1] = c->N[2] = 64;
  c->kfactor[0] = c->kfactor[1] = c->kfactor[2] = 1.0;
  c->precision = TS_F64;
  c->nlin_form = TS_NLIN_CONSERVATIVE;
  c->dealias_mode = TS_DEALIAS_REFERENCE_CORNER;
  c->reality_fix = 1;
  c->nu = 0.01;
  c->kappa = 0.01;
  c->dt = 1e-3;
  c->force_type = TS_FORCE_NONE;
  c->Ra = 1e5;
  c->Pr = 1.0;
}

long long ts_kernel_launch_count(void) { return g_launches; }
const char* ts_last_error(void) { return g_last_error.c_str(); }

int ts_plan_destroy(ts_plan* p) {
  if (!p) return TS_ERR_ARG;
  void* bufs[] = {p->Ucur, p->tot, p->P, p->twx, p->twy, p->twz, p->fcube, p->esup, p->hsup, p->mis_d, p->dscr,
                  p->stage_u, p->stage_t, p->stage_b, p->twqy, p->twqz};
  for (void* b : bufs)
    if (b) cudaFree(b);
  for (cudaEvent_t e : p->ev_pool) cudaEventDestroy(e);
  for (int i = 0; i < 3; ++i) {
    if (p->eax[i]) cudaFree(p->eax[i]);
    if (p->eaxf[i]) cudaFree(p->eaxf[i]);
    if (p->eaxT[i]) cudaFree(p->eaxT[i]);
  }
  if (p->twq) cudaFree(p->twq);
  if (p->err_d) cudaFree(p->err_d);
  if (p->err_h) cudaFreeHost(p->err_h);
  delete p;
  return TS_OK;
}

int ts_plan_create(const ts_config* cfg, ts_plan** out) {
  if (!cfg || !out) return TS_ERR_ARG;
  *out = nullptr;
  for (int i = 0; i < 3; ++i) {
    // 48 and 96 (factor 3) are supported for the SFF path
    const bool mixed = (cfg->N[i] == 48 || cfg->N[i] == 96) && cfg->basis != TS_BASIS_FFF;
    // SFF takes Ny = 1: a two-dimensional run in the x-z plane (program.two_dimension)
    const bool flat = i == 1 && cfg->N[1] == 1 && cfg->basis == TS_BASIS_SFF;
    if (!size_supported(cfg->N[i]) && !mixed && !flat) {
      g_last_error = "N must be a power of two in [16, 1024] (48 and 96 also for SFF; Ny = 1 on SFF)";
      return TS_ERR_ARG;
    }
  }
  if (cfg->basis != TS_BASIS_FFF && cfg->basis != TS_BASIS_SFF && cfg->basis != TS_BASIS_SSF &&
      cfg->basis != TS_BASIS_SSS)
    return TS_ERR_ARG;
  if (cfg->precision != TS_F64 && cfg->precision != TS_F32) return TS_ERR_ARG;
  if (cfg->dealias_mode < 0 || cfg->dealias_mode > 2) return TS_ERR_ARG;
  if (cfg->nlin_form != TS_NLIN_CONSERVATIVE && cfg->nlin_form != TS_NLIN_ROTATIONAL) return TS_ERR_ARG;
  if (cfg->basis != TS_BASIS_FFF && cfg->nlin_form == TS_NLIN_ROTATIONAL) return TS_ERR_UNSUPPORTED;
  if ((cfg->basis == TS_BASIS_SSF || cfg->basis == TS_BASIS_SSS) && (cfg->N[0] > 512 || cfg->N[1] > 512)) {
    g_last_error = "SSF and SSS support Nx, Ny <= 512";
    return TS_ERR_UNSUPPORTED;
  }
  if (cfg->basis == TS_BASIS_SSS && (cfg->N[2] % 3 == 0)) {
    g_last_error = "SSS needs a power-of-two Nz";
    return TS_ERR_UNSUPPORTED;
  }
  // the RBC coefficients of the plan's scaling (any basis: ts_rk4_step_rbc and ts_nusselt use them)
  double rbc_nu = 0, rbc_kappa = 0, rbc_cu = 1, rbc_cT = 1, rbc_nu0 = 1, rbc_nuc = 0, rbc_vs = 0;
  {
    const int rc0 = rbc_coefficients(cfg->Pr_option, cfg->Uscaling, cfg->Ra, cfg->Pr, &rbc_nu, &rbc_kappa, &rbc_cu,
                                     &rbc_cT, &rbc_nu0, &rbc_nuc, &rbc_vs);
    if (rc0 != TS_OK) return rc0;
  }
  ts_plan* p = new ts_plan();
  p->cfg = *cfg;
  p->rbc_cu = rbc_cu;
  p->rbc_cT = rbc_cT;
  p->rbc_nu0 = rbc_nu0;
  p->rbc_nuc = rbc_nuc;
  p->rbc_slave = cfg->Pr_option == TS_PR_ZERO ? 1 : (cfg->Pr_option == TS_PR_INFTY ? 2 : 0);
  p->rbc_vs = rbc_vs;
  p->cfg.energy_supply = nullptr;
  p->cfg.helicity_supply = nullptr;
  Geo& g = p->g;
  g.Nx = cfg->N[0];
  g.Ny = cfg->N[1];
  g.Nz = cfg->N[2];
  g.Hz = g.Nz / 2 + 1;
  g.S = (long long)g.Nx * g.Ny * g.Hz;
  for (int i = 0; i < 3; ++i) g.kf[i] = cfg->kfactor[i];
  g.basis = cfg->basis;
  g.dealias = cfg->dealias_mode;
  p->prec = cfg->precision == TS_F32 ? 1 : 0;
  p->cb = p->prec ? 8 : 16;
  int rc = TS_OK;
#define CKP(x)                     \
  do {                             \
    rc = (x);                      \
    if (rc != TS_OK) {             \
      ts_plan_destroy(p);          \
      return rc;                   \
    }                              \
  } while (0)
  auto alloc = [&](void** b, size_t bytes) -> int {
    CK(cudaMalloc(b, bytes));
    return TS_OK;
  };
  // SFF (Boussinesq): stage / accumulator fields carry T as a fourth component,
  // and the z pass makes nine products
  const int ncs = cfg->basis == TS_BASIS_SFF ? 4 : 3,
            nps = cfg->basis == TS_BASIS_SFF ? 9 : (cfg->basis == TS_BASIS_SSS ? 12 : 6);
  if (cfg->basis == TS_BASIS_SFF && g.Nx > 512) {
    g_last_error = "SFF supports Nx <= 512";
    ts_plan_destroy(p);
    return TS_ERR_UNSUPPORTED;
  }
  CKP(alloc(&p->Ucur, ncs * g.S * p->cb));
  CKP(alloc(&p->tot, ncs * g.S * p->cb));
  CKP(alloc(&p->P, nps * g.S * p->cb));
  p->nP = nps;
  p->nS = ncs;
  if (p->prec) {
    CKP(upload_twiddles<float>(g.Nx, &p->twx));
    CKP(upload_twiddles<float>(g.Ny, &p->twy));
    CKP(upload_twiddles<float>(g.Nz, &p->twz));
  } else {
    CKP(upload_twiddles<double>(g.Nx, &p->twx));
    CKP(upload_twiddles<double>(g.Ny, &p->twy));
    CKP(upload_twiddles<double>(g.Nz, &p->twz));
  }
  compute_modes_in_shell(p);
  CKP(alloc((void**)&p->mis_d, p->mis.size() * sizeof(double)));
  if (cudaMemcpy(p->mis_d, p->mis.data(), p->mis.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    ts_plan_destroy(p);
    return TS_ERR_CUDA;
  }
  if (cfg->force_type == TS_FORCE_CARATI_ENERGY_SUPPLY) {
    if (cfg->basis != TS_BASIS_FFF || !cfg->energy_supply || cfg->n_supply <= 0 ||
        cfg->force_outer_radius <= cfg->force_inner_radius) {
      ts_plan_destroy(p);
      return TS_ERR_ARG;
    }
    double kfmin = fmin(g.kf[0], fmin(g.kf[1], g.kf[2]));
    p->fkm = (int)ceil(cfg->force_outer_radius / kfmin);
    if (p->fkm >= g.Nx / 2 || p->fkm >= g.Ny / 2 || p->fkm > g.Nz / 2) {
      g_last_error = "forcing band must lie inside the box";
      ts_plan_destroy(p);
      return TS_ERR_ARG;
    }
    p->nsup = cfg->n_supply;
    const int n = 2 * p->fkm + 1;
    CKP(alloc(&p->fcube, 3ull * n * n * (p->fkm + 1) * p->cb));
    CKP(alloc((void**)&p->esup, p->nsup * sizeof(double)));
    if (cudaMemcpy(p->esup, cfg->energy_supply, p->nsup * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
      ts_plan_destroy(p);
      return TS_ERR_CUDA;
    }
    if (cfg->helicity_supply) {
      CKP(alloc((void**)&p->hsup, p->nsup * sizeof(double)));
      if (cudaMemcpy(p->hsup, cfg->helicity_supply, p->nsup * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
        ts_plan_destroy(p);
        return TS_ERR_CUDA;
      }
    }
  } else if (cfg->force_type != TS_FORCE_NONE && cfg->force_type != TS_FORCE_RBC) {
    ts_plan_destroy(p);
    return TS_ERR_ARG;
  }
  CKP(ensure_scratch(p, 4096));
  CKP(alloc((void**)&p->err_d, sizeof(int)));
  if (cudaMemset(p->err_d, 0, sizeof(int)) != cudaSuccess || cudaMallocHost(&p->err_h, sizeof(int)) != cudaSuccess) {
    ts_plan_destroy(p);
    return TS_ERR_CUDA;
  }
  *p->err_h = 0;
  CKP(upload_if_tables(p, cfg->nu, cfg->dt, p->eax, p->eaxf));
  // the scalar's factors: the SFF Boussinesq step and the FFF passive-scalar step
  CKP(upload_if_tables(p, cfg->kappa, cfg->dt, p->eaxT));
  if (cfg->basis == TS_BASIS_SSS) {
    // sin/cos along z: the 4 Nz quarter-step table
    if (p->prec) CKP(upload_twiddles<float>(4 * g.Nz, &p->twqz));
    else CKP(upload_twiddles<double>(4 * g.Nz, &p->twqz));
  }
  if (cfg->basis == TS_BASIS_SSF || cfg->basis == TS_BASIS_SSS) {
    // sin/cos along y: the 4 Ny quarter-step table
    if (p->prec) CKP(upload_twiddles<float>(4 * g.Ny, &p->twqy));
    else CKP(upload_twiddles<double>(4 * g.Ny, &p->twqy));
  }
  if (cfg->basis != TS_BASIS_FFF) {
    if (p->prec) CKP(upload_twiddles<float>(4 * g.Nx, &p->twq));
    else CKP(upload_twiddles<double>(4 * g.Nx, &p->twq));
  }
#undef CKP
  *out = p;
  return TS_OK;
}

int ts_plan_set_stream(ts_plan* p, void* stream) {
  if (!p) return TS_ERR_ARG;
  p->st = (cudaStream_t)stream;
  return TS_OK;
}

int ts_plan_sizes(const ts_plan* p, long long* elems, int* bytes) {
  if (!p) return TS_ERR_ARG;
  if (elems) *elems = p->g.S;
  if (bytes) *bytes = (int)p->cb;
  return TS_OK;
}

int ts_plan_num_shells(const ts_plan* p, int* n) {
  if (!p || !n) return TS_ERR_ARG;
  *n = p->nshells;
  return TS_OK;
}

int ts_alloc_field(const ts_plan* p, int ncomp, void** field) {
  if (!p || !field || ncomp < 1) return TS_ERR_ARG;
  *field = nullptr;
  const size_t bytes = (size_t)ncomp * (size_t)p->g.S * p->cb;
  void* f = nullptr;
  CK(cudaMalloc(&f, bytes));
  cudaError_t e = cudaMemset(f, 0, bytes);
  if (e != cudaSuccess) {
    cudaFree(f);
    g_last_error = std::string("ts_alloc_field: ") + cudaGetErrorString(e);
    return TS_ERR_CUDA;
  }
  *field = f;
  return TS_OK;
}

int ts_free_field(void* field) {
  if (field) CK(cudaFree(field));
  return TS_OK;
}

int ts_plan_status(ts_plan* p) {
  if (!p) return TS_ERR_ARG;
  CK(cudaStreamSynchronize(p->st));
  CK(cudaMemcpy(p->err_h, p->err_d, sizeof(int), cudaMemcpyDeviceToHost));
  return health_status(p);
}

int ts_plan_clear_status(ts_plan* p) {
  if (!p) return TS_ERR_ARG;
  CK(cudaStreamSynchronize(p->st));
  CK(cudaMemset(p->err_d, 0, sizeof(int)));
  *p->err_h = 0;
  return TS_OK;
}

int ts_plan_expire_wait(ts_plan* p, int polls) {
  if (!p || polls < 1 || polls > (1 << 22)) return TS_ERR_ARG;
  CK(LAUNCH(p, expire_wait, p->err_d, polls, p->st));
  CK(cudaMemcpyAsync(p->err_h, p->err_d, sizeof(int), cudaMemcpyDeviceToHost, p->st));
  return TS_OK;
}

int ts_plan_set_dt(ts_plan* p, double dt) {
  if (!p || !(dt > 0)) return TS_ERR_ARG;
  if (dt == p->cfg.dt) return TS_OK;
  CK(cudaStreamSynchronize(p->st));
  p->cfg.dt = dt;
  CKS(upload_if_tables(p, p->cfg.nu, dt, p->eax, p->eaxf));
  CKS(upload_if_tables(p, p->cfg.kappa, dt, p->eaxT));
  return TS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// right-hand side pipeline (FFF)
// ---------------------------------------------------------------------------
// Algorithmic bytes of each pass of one FFF right-hand side: every element the pass
// must read or write, once, with the dealias skipping counted as it runs.  Two
// thirds (kept): the x inverse reads the nxk x nyk x nzk modes that can be nonzero
// and writes all Nx rows of the nyk x nzk kept columns; the y inverse reads their
// nyk rows and writes all Ny rows of the nzk kept z planes; the z pass reads those
// planes and writes full lines.  Other modes: the x inverse does not read the
// corner box's zeros.  fwd_x: the products plus the state fields of the mode and
// stage (stage 1 reads U0 and writes Ucur, tot; stages 2-3 also read tot; stage 4
// reads U0, tot and writes Uout).
static double fff_pass_bytes(const ts_plan* p, int cls, int nin, int nout, int kept, int mode = MODE_STEP,
                             int stage = 1) {
  const Geo& g = p->g;
  auto kept_count = [](int N, bool half) {
    int n = 0;
    for (int l = 0; l < (half ? N / 2 + 1 : N); ++l) {
      const int k = half ? l : (l <= N / 2 ? l : l - N);
      n += 3 * (k < 0 ? -k : k) <= N;
    }
    return (double)n;
  };
  const double S = (double)g.S, Nx = g.Nx, Ny = g.Ny, cb = (double)p->cb;
  const double nxk = kept_count(g.Nx, false), nyk = kept_count(g.Ny, false), nzk = kept_count(g.Nz, true);
  double nz_read = S;  // modes of a component the x inverse reads
  if (!kept && g.dealias == TS_DEALIAS_REFERENCE_CORNER) {
    const double bx = (double)((2 * g.Nx / 3 - 1) - (g.Nx / 3 + 1) + 1), by = (double)((2 * g.Ny / 3 - 1) - (g.Ny / 3 + 1) + 1);
    const double bz = (double)(g.Nz / 2 - (g.Nz / 3 + 1) + 1);
    nz_read = S - (bx > 0 ? bx : 0) * (by > 0 ? by : 0) * (bz > 0 ? bz : 0);
  }
  double e = 0;
  switch (cls) {
    case TS_KCLASS_INV_X: e = kept ? 3 * nxk * nyk * nzk + nin * Nx * nyk * nzk : 3 * nz_read + nin * S; break;
    case TS_KCLASS_Y_INV: e = kept ? nin * (Nx * nyk * nzk + Nx * Ny * nzk) : 2.0 * nin * S; break;
    case TS_KCLASS_Z: e = kept ? nin * Nx * Ny * nzk + nout * S : (nin + nout) * S; break;
    case TS_KCLASS_Y_FWD: e = 2.0 * nout * S; break;
    case TS_KCLASS_FWD_X: {
      double st = 3;  // MODE_FLUX reads the field, MODE_NLIN writes N
      if (mode == MODE_STEP) st = (stage == 1 || stage == 4) ? 9 : 12;
      if (mode == MODE_ADJ) st = stage == 1 ? 6 : (stage == 4 ? 9 : 12);
      e = (nout + st) * S;
      break;
    }
    default: break;
  }
  return e * cb;
}

static int rhs_fff(ts_plan* p, const void* Uin, int mode, const StageArgs& a_in) {
  const Geo& g = p->g;
  StageArgs a = a_in;
  a.err = p->err_d;
  a.ex = p->eax[0];
  a.ey = p->eax[1];
  a.ez = p->eax[2];
  a.exf = p->eaxf[0];
  a.eyf = p->eaxf[1];
  a.ezf = p->eaxf[2];
  const int rot = p->cfg.nlin_form == TS_NLIN_ROTATIONAL;
  const int nin = rot ? 6 : 3, nout = rot ? 3 : 6;
  // two-thirds dealiasing: after the x inverse only the columns with 3|ky| <= Ny and
  // 3 kz <= Nz can be nonzero, so the inverse x pass writes only those, the y
  // inverse transforms only kz <= Nz/3 and reads only the 3|ky| <= Ny rows, and the
  // z pass reads only kz <= Nz/3 (the skipped memory is never read)
  const int kept = g.dealias == TS_DEALIAS_TWO_THIRDS;
  auto by = [&](int cls) { return p->prof ? fff_pass_bytes(p, cls, nin, nout, kept, mode, a.stage) : -1.0; };
  {
    ProfScope ps(p, TS_KCLASS_INV_X, by(TS_KCLASS_INV_X));
    CK(LAUNCH(p, inv_x, g, rot, Uin, p->P, p->twx, nullptr, 0.0, p->st, kept));
  }
  {
    ProfScope ps(p, TS_KCLASS_Y_INV, by(TS_KCLASS_Y_INV));
    CK(LAUNCH(p, strided, g, 1, +1, p->P, nin, p->twy, p->st, 0, 0, kept ? g.Nz / 3 + 1 : 0, kept));
  }
  {
    ProfScope ps(p, TS_KCLASS_Z, by(TS_KCLASS_Z));
    CK(LAUNCH(p, z_fused, g, rot, p->P, p->twz, p->err_d, p->st, 1, 0, kept ? g.Nz / 3 : -1));
  }
  { ProfScope ps(p, TS_KCLASS_Y_FWD, by(TS_KCLASS_Y_FWD)); CK(LAUNCH(p, strided, g, 1, -1, p->P, nout, p->twy, p->st)); }
  { ProfScope ps(p, TS_KCLASS_FWD_X, by(TS_KCLASS_FWD_X)); CK(LAUNCH(p, fwd_x, g, rot, mode, p->P, a, p->twx, p->st)); }
  return TS_OK;
}

// One IF-RK4 step from U0; stage 4 writes the new state to Uout (nullptr: in
// place) and the reality fix is applied there.  keep != nullptr: the stage
// fields U1, U2, U3 are written to keep (9 components) instead of the plan's
// single stage field; stages_only: stop after stage 3.
static int step_fff(ts_plan* p, void* U0, void* Uout = nullptr, void* keep = nullptr, bool stages_only = false) {
  const Geo& g = p->g;
  const long long cs = 3 * g.S * (long long)p->cb;
  StageArgs a;
  memset(&a, 0, sizeof(a));
  a.U0 = U0;
  a.Uout = Uout ? Uout : U0;
  a.Ucur = p->Ucur;
  a.tot = p->tot;
  a.nu = p->cfg.nu;
  a.dt = p->cfg.dt;
  a.reality = p->cfg.reality_fix;
  a.fcube = p->cfg.force_type == TS_FORCE_CARATI_ENERGY_SUPPLY ? p->fcube : nullptr;
  a.fkm = p->fkm;
  for (int stage = 1; stage <= (stages_only ? 3 : 4); ++stage) {
    const void* Uin = stage == 1 ? U0 : (keep ? (const void*)((const char*)keep + (stage - 2) * cs) : p->Ucur);
    if (keep && stage <= 3) a.Ucur = (char*)keep + (stage - 1) * cs;
    if (a.fcube) {
      ProfScope ps(p, TS_KCLASS_OTHER);
      CK(LAUNCH(p, carati, g, Uin, p->fcube, p->fkm, p->cfg.force_inner_radius, p->cfg.force_outer_radius, p->esup,
                p->hsup, p->mis_d, p->nsup, p->st));
    }
    a.stage = stage;
    CKS(rhs_fff(p, Uin, MODE_STEP, a));
  }
  if (p->cfg.reality_fix && !stages_only) {
    ProfScope ps(p, TS_KCLASS_OTHER);
    CK(LAUNCH(p, reality, g, a.Uout, 3, p->st));
  }
  return TS_OK;
}

// ---------------------------------------------------------------------------
// discrete adjoint of step_fff (rotational form, unforced)
// ---------------------------------------------------------------------------
static int adjoint_supported(ts_plan* p) {
  if (p->cfg.basis != TS_BASIS_FFF || p->cfg.nlin_form != TS_NLIN_ROTATIONAL ||
      p->cfg.force_type != TS_FORCE_NONE) {
    g_last_error = "the adjoint step is implemented for FFF, rotational form, unforced plans";
    return TS_ERR_UNSUPPORTED;
  }
  if (p->nP < 9) {
    // the adjoint right-hand side transforms nine fields (u, w, and the projected cotangent)
    CK(cudaStreamSynchronize(p->st));
    CK(cudaFree(p->P));
    p->P = nullptr;
    p->nP = 0;
    CK(cudaMalloc(&p->P, 9 * p->g.S * p->cb));
    p->nP = 9;
  }
  return TS_OK;
}

// lam <- (d step / d U0)^T lam, with U0 the state at the start of the step and
// `stages` its stage fields U1, U2, U3 (from step_fff with keep)
static int adjoint_step_fff(ts_plan* p, const void* U0, const void* stages, void* lam) {
  const Geo& g = p->g;
  const long long cs = 3 * g.S * (long long)p->cb;
  const int kept = g.dealias == TS_DEALIAS_TWO_THIRDS;
  if (p->cfg.reality_fix) {
    ProfScope ps(p, TS_KCLASS_OTHER);
    CK(LAUNCH(p, reality_adj, g, lam, 3, p->st));
  }
  StageArgs a;
  memset(&a, 0, sizeof(a));
  a.U0 = lam;
  a.Uout = lam;
  a.Ucur = p->Ucur;
  a.tot = p->tot;
  a.nu = p->cfg.nu;
  a.dt = p->cfg.dt;
  a.err = p->err_d;
  a.ex = p->eax[0];
  a.ey = p->eax[1];
  a.ez = p->eax[2];
  for (int stage = 4; stage >= 1; --stage) {
    // the stage's linearisation point: its input U_{stage-1} (dealiased on load)
    const void* Uin = stage == 1 ? U0 : (const void*)((const char*)stages + (stage - 2) * cs);
    const void* cot = stage == 4 ? (const void*)lam : (const void*)p->Ucur;
    const double lsc = stage == 4 ? p->cfg.dt / 6.0 : 1.0;
    a.stage = stage;
    if (kept) {
      // u, w (fields 0-5) on the kept columns only, as in rhs_fff; the cotangent fields 6-8 are full
      {
        ProfScope ps(p, TS_KCLASS_INV_X);
        CK(LAUNCH(p, inv_x, g, 1, Uin, p->P, p->twx, nullptr, 0.0, p->st, 1));
        CK(LAUNCH(p, inv_x, g, 4, Uin, p->P, p->twx, cot, lsc, p->st));
      }
      {
        ProfScope ps(p, TS_KCLASS_Y_INV);
        CK(LAUNCH(p, strided, g, 1, +1, p->P, 6, p->twy, p->st, 0, 0, g.Nz / 3 + 1, 1));
        CK(LAUNCH(p, strided, g, 1, +1, (char*)p->P + 6 * g.S * (long long)p->cb, 3, p->twy, p->st));
      }
    } else {
      { ProfScope ps(p, TS_KCLASS_INV_X); CK(LAUNCH(p, inv_x, g, 3, Uin, p->P, p->twx, cot, lsc, p->st)); }
      { ProfScope ps(p, TS_KCLASS_Y_INV); CK(LAUNCH(p, strided, g, 1, +1, p->P, 9, p->twy, p->st)); }
    }
    { ProfScope ps(p, TS_KCLASS_Z); CK(LAUNCH(p, z_fused, g, 3, p->P, p->twz, p->err_d, p->st, 1, 0, kept ? g.Nz / 3 : -1)); }
    { ProfScope ps(p, TS_KCLASS_Y_FWD); CK(LAUNCH(p, strided, g, 1, -1, p->P, 6, p->twy, p->st)); }
    { ProfScope ps(p, TS_KCLASS_FWD_X); CK(LAUNCH(p, fwd_x, g, 3, MODE_ADJ, p->P, a, p->twx, p->st)); }
  }
  return TS_OK;
}

// one IF-RK4 step of the Boussinesq system on the SFF basis (RK_SF.cc:97-221)
static int step_rbc(ts_plan* p, void* U0, void* T0) {
  const Geo& g = p->g;
  SffArgs a;
  memset(&a, 0, sizeof(a));
  a.cu = p->rbc_cu;
  a.cT = p->rbc_cT;
  a.slave = p->rbc_slave;
  a.vs = p->rbc_vs;
  a.health = p->err_d;
  a.U0 = U0;
  a.T0 = T0;
  a.Ucur = p->Ucur;
  a.tot = p->tot;
  a.dt = p->cfg.dt;
  a.reality = p->cfg.reality_fix;
  for (int i = 0; i < 3; ++i) {
    a.eu[i] = p->eax[i];
    a.et[i] = p->eaxT[i];
  }
  const long long cb = (long long)p->cb;
  for (int stage = 1; stage <= 4; ++stage) {
    const void* Uin = stage == 1 ? U0 : p->Ucur;
    const void* Tin = stage == 1 ? T0 : (const void*)((const char*)p->Ucur + 3 * g.S * cb);
    a.stage = stage;
    a.U1in = Uin;
    a.Tin = Tin;
    { ProfScope ps(p, TS_KCLASS_INV_X); CK(LAUNCH(p, sff_inv_x, g, Uin, Tin, p->P, p->twq, p->st)); }
    { ProfScope ps(p, TS_KCLASS_Y_INV); CK(LAUNCH(p, strided, g, 1, +1, p->P, 4, p->twy, p->st)); }
    { ProfScope ps(p, TS_KCLASS_Z); CK(LAUNCH(p, z_fused, g, 2, p->P, p->twz, p->err_d, p->st)); }
    { ProfScope ps(p, TS_KCLASS_Y_FWD); CK(LAUNCH(p, strided, g, 1, -1, p->P, 9, p->twy, p->st)); }
    { ProfScope ps(p, TS_KCLASS_FWD_X); CK(LAUNCH(p, sff_fwd_x, g, p->P, a, p->twq, p->st)); }
  }
  if (p->cfg.reality_fix) {
    ProfScope ps(p, TS_KCLASS_OTHER);
    CK(LAUNCH(p, reality, g, U0, 3, p->st));
    CK(LAUNCH(p, reality, g, T0, 1, p->st));
  }
  return TS_OK;
}

// ---------------------------------------------------------------------------
// FFF passive scalar (program.kind SCALAR_INCOMPRESS): RK4(U,T,P,F) with no force
// ---------------------------------------------------------------------------
static int ensure_work(ts_plan* p, int nstage, int nprod);

static int scalar_supported(ts_plan* p) {
  if (p->cfg.basis != TS_BASIS_FFF || p->cfg.force_type != TS_FORCE_NONE ||
      p->cfg.nlin_form != TS_NLIN_CONSERVATIVE) {
    g_last_error = "the passive-scalar step is implemented for FFF, conservative form, unforced plans";
    return TS_ERR_UNSUPPORTED;
  }
  // stage and accumulator fields carry T as a fourth component; the z pass makes nine products
  return ensure_work(p, 4, 9);
}

// one IF-RK4 step of U and the passive scalar T on the FFF basis (RK_SF.cc:97-221 with
// Compute_force_TO_rhs_scalar, Tadvance_functions.cc:464-474, and Compute_nlin_scalar,
// compute_nlin_SF.cc:75-112): dealiased u, T to real space, the nine products u_i u_j and
// u_i T (z pass form 2), forward transforms, then N, NT, the projection and the stage update
static int step_scalar_fff(ts_plan* p, void* U0, void* T0) {
  const Geo& g = p->g;
  SffArgs a;
  memset(&a, 0, sizeof(a));
  a.health = p->err_d;
  a.U0 = U0;
  a.T0 = T0;
  a.Ucur = p->Ucur;
  a.tot = p->tot;
  a.dt = p->cfg.dt;
  a.reality = p->cfg.reality_fix;
  for (int i = 0; i < 3; ++i) {
    a.eu[i] = p->eax[i];
    a.et[i] = p->eaxT[i];
  }
  const long long cb = (long long)p->cb;
  const int kept = g.dealias == TS_DEALIAS_TWO_THIRDS;
  void* P3 = (char*)p->P + 3 * g.S * cb;
  for (int stage = 1; stage <= 4; ++stage) {
    const void* Uin = stage == 1 ? U0 : p->Ucur;
    const void* Tin = stage == 1 ? T0 : (const void*)((const char*)p->Ucur + 3 * g.S * cb);
    a.stage = stage;
    a.U1in = Uin;
    a.Tin = Tin;
    {
      ProfScope ps(p, TS_KCLASS_INV_X);
      CK(LAUNCH(p, inv_x, g, 0, Uin, p->P, p->twx, nullptr, 0.0, p->st, kept));
      CK(LAUNCH(p, dealias_copy, g, Tin, P3, 1, p->st));
      CK(LAUNCH(p, strided, g, 0, +1, P3, 1, p->twx, p->st));
    }
    { ProfScope ps(p, TS_KCLASS_Y_INV); CK(LAUNCH(p, strided, g, 1, +1, p->P, 4, p->twy, p->st, 0, 0, kept ? g.Nz / 3 + 1 : 0, kept)); }
    { ProfScope ps(p, TS_KCLASS_Z); CK(LAUNCH(p, z_fused, g, 2, p->P, p->twz, p->err_d, p->st, 1, 0, kept ? g.Nz / 3 : -1)); }
    { ProfScope ps(p, TS_KCLASS_Y_FWD); CK(LAUNCH(p, strided, g, 1, -1, p->P, 9, p->twy, p->st)); }
    {
      ProfScope ps(p, TS_KCLASS_FWD_X);
      CK(LAUNCH(p, strided, g, 0, -1, p->P, 9, p->twx, p->st));
      CK(LAUNCH(p, scalar_epi, g, p->P, a, p->st));
    }
  }
  if (p->cfg.reality_fix) {
    ProfScope ps(p, TS_KCLASS_OTHER);
    CK(LAUNCH(p, reality, g, U0, 3, p->st));
    CK(LAUNCH(p, reality, g, T0, 1, p->st));
  }
  return TS_OK;
}

// ---------------------------------------------------------------------------
// FFF incompressible MHD: RK4(U, W, P, F) with W = B, no force
// ---------------------------------------------------------------------------
static int ensure_work(ts_plan* p, int nstage, int nprod) {
  if (p->nS >= nstage && p->nP >= nprod) return TS_OK;
  CK(cudaStreamSynchronize(p->st));
  if (p->nS < nstage) {
    CK(cudaFree(p->Ucur));
    CK(cudaFree(p->tot));
    p->Ucur = p->tot = nullptr;
    p->nS = 0;
    CK(cudaMalloc(&p->Ucur, nstage * p->g.S * p->cb));
    CK(cudaMalloc(&p->tot, nstage * p->g.S * p->cb));
    p->nS = nstage;
  }
  if (p->nP < nprod) {
    CK(cudaFree(p->P));
    p->P = nullptr;
    p->nP = 0;
    CK(cudaMalloc(&p->P, nprod * p->g.S * p->cb));
    p->nP = nprod;
  }
  return TS_OK;
}

static int mhd_supported(ts_plan* p) {
  if (p->cfg.basis != TS_BASIS_FFF || p->cfg.force_type != TS_FORCE_NONE) {
    g_last_error = "the MHD step is implemented for FFF, unforced plans";
    return TS_ERR_UNSUPPORTED;
  }
  // stage and accumulator fields carry U and B (6 components); nine Elsasser products
  return ensure_work(p, 6, 9);
}

// one IF-RK4 step of U (nu) and B (eta = the plan's kappa) (RK_VF_MHD.cc:126-186,
// Compute_force_TO_rhs Tadvance_functions.cc:506-517, Compute_nlin(U, W)
// compute_nlin_VF_MHD.cc:40-95): dealiased u, b to real space, the nine Elsasser
// products Zp_i Zm_j (z pass form 5), forward transforms, then the MHD epilogue
static int step_mhd_fff(ts_plan* p, void* U0, void* B0) {
  const Geo& g = p->g;
  SffArgs a;
  memset(&a, 0, sizeof(a));
  a.health = p->err_d;
  a.U0 = U0;
  a.T0 = B0;
  a.Ucur = p->Ucur;
  a.tot = p->tot;
  a.dt = p->cfg.dt;
  a.reality = p->cfg.reality_fix;
  for (int i = 0; i < 3; ++i) {
    a.eu[i] = p->eax[i];
    a.et[i] = p->eaxT[i];
  }
  const long long cs = 3 * g.S * (long long)p->cb;
  const int kept = g.dealias == TS_DEALIAS_TWO_THIRDS;
  void* P3 = (char*)p->P + cs;
  for (int stage = 1; stage <= 4; ++stage) {
    const void* Uin = stage == 1 ? U0 : p->Ucur;
    const void* Bin = stage == 1 ? B0 : (const void*)((const char*)p->Ucur + cs);
    a.stage = stage;
    {
      ProfScope ps(p, TS_KCLASS_INV_X);
      CK(LAUNCH(p, inv_x, g, 0, Uin, p->P, p->twx, nullptr, 0.0, p->st, kept));
      CK(LAUNCH(p, inv_x, g, 0, Bin, P3, p->twx, nullptr, 0.0, p->st, kept));
    }
    { ProfScope ps(p, TS_KCLASS_Y_INV); CK(LAUNCH(p, strided, g, 1, +1, p->P, 6, p->twy, p->st, 0, 0, kept ? g.Nz / 3 + 1 : 0, kept)); }
    { ProfScope ps(p, TS_KCLASS_Z); CK(LAUNCH(p, z_fused, g, 5, p->P, p->twz, p->err_d, p->st, 1, 0, kept ? g.Nz / 3 : -1)); }
    { ProfScope ps(p, TS_KCLASS_Y_FWD); CK(LAUNCH(p, strided, g, 1, -1, p->P, 9, p->twy, p->st)); }
    {
      ProfScope ps(p, TS_KCLASS_FWD_X);
      CK(LAUNCH(p, strided, g, 0, -1, p->P, 9, p->twx, p->st));
      CK(LAUNCH(p, mhd_epi, g, p->P, a, p->st));
    }
  }
  if (p->cfg.reality_fix) {
    ProfScope ps(p, TS_KCLASS_OTHER);
    CK(LAUNCH(p, reality, g, U0, 3, p->st));
    CK(LAUNCH(p, reality, g, B0, 3, p->st));
  }
  return TS_OK;
}

// SSF plans offer the transforms only
static int ssf_transforms_only() {
  g_last_error = "SSF and SSS plans offer the transforms and ts_rk4_step only";
  return TS_ERR_UNSUPPORTED;
}

// the geometry that makes the x-axis sin/cos kernel transform along y: every
// x-plane of every component is one "component" of Ny rows x Hz columns
static Geo y_as_x(const Geo& g) {
  Geo h = g;
  h.Nx = g.Ny;
  h.Ny = 1;
  h.S = (long long)g.Ny * g.Hz;
  h.dealias = 0;
  return h;
}

// ---------------------------------------------------------------------------
// SSF fluid step (sin/cos along x and y; sincostr_switch "SCF"), conservative form,
// unforced: RK4(U,P,F) (RK.cc:91-170) with standalone transforms; with a temperature
// T the Boussinesq step RK4(U,T,P,F) (RK_SF.cc:97-221, PRLARGE / ULARGE buoyancy).
// With nf = 3 (fluid) or 4 (U, T) fields and np = 6 or 9 products, P holds [0, np):
// the nf spectra after the x and y inverses, which the fused z pass turns into the
// np product spectra in place.
// ---------------------------------------------------------------------------
static int ssf_step_supported(ts_plan* p, bool rbc) {
  const int basis = p->cfg.basis;
  if ((basis != TS_BASIS_SSF && basis != TS_BASIS_SSS) || p->cfg.nlin_form != TS_NLIN_CONSERVATIVE ||
      p->cfg.force_type != TS_FORCE_NONE) {
    g_last_error = rbc ? "the SSF / SSS Boussinesq step is the conservative, unforced one"
                       : "the SSF / SSS step is the conservative, unforced fluid step";
    return TS_ERR_UNSUPPORTED;
  }
  const int nf = rbc ? 4 : 3, np = rbc ? 9 : 6;
  return ensure_work(p, nf, np);
}

// the RBC epilogue's arguments (U, T in place; stage fields U then T in Ucur, tot)
static SffArgs ssf_rbc_args(ts_plan* p, void* U0, void* T0) {
  SffArgs a;
  memset(&a, 0, sizeof(a));
  a.cu = p->rbc_cu;
  a.cT = p->rbc_cT;
  a.health = p->err_d;
  a.U0 = U0;
  a.T0 = T0;
  a.Ucur = p->Ucur;
  a.tot = p->tot;
  a.dt = p->cfg.dt;
  for (int i = 0; i < 3; ++i) {
    a.eu[i] = p->eax[i];
    a.et[i] = p->eaxT[i];
  }
  return a;
}

static int step_ssf(ts_plan* p, void* U0, void* T0 = nullptr) {
  const Geo& g = p->g;
  const Geo gy = y_as_x(g);
  const long long cs = g.S * (long long)p->cb;  // bytes of one component
  const int nf = T0 ? 4 : 3, np = T0 ? 9 : 6;
  char* P = (char*)p->P;
  StageArgs a;
  memset(&a, 0, sizeof(a));
  a.U0 = U0;
  a.Uout = U0;
  a.Ucur = p->Ucur;
  a.tot = p->tot;
  a.dt = p->cfg.dt;
  a.err = p->err_d;
  a.ex = p->eax[0];
  a.ey = p->eax[1];
  a.ez = p->eax[2];
  SffArgs b = ssf_rbc_args(p, U0, T0);
  // x, y sine (1) / cosine (0) letters of Vx = SCF, Vy = CSF, Vz = CCF, T = SCF and of the
  // products u1u1, u2u2, u3u3 (Vi2 = CCF), u1u2 (VxVy = SSF), u2u3 (VyVz = CSF),
  // u3u1 (VxVz = SCF), u1T (CCF), u2T (SSF), u3T (SCF)
  const int vx[4] = {1, 0, 0, 1}, vy[4] = {0, 1, 0, 0};
  const int qx[9] = {0, 0, 0, 1, 0, 1, 0, 1, 1}, qy[9] = {0, 0, 0, 1, 1, 0, 0, 1, 0};
  const double sy = 1.0 / (2.0 * g.Ny), sx = 1.0 / (2.0 * g.Nx * (double)g.Nz);
  // the same letters as bit masks (bit c = field c), one batched launch per pass
  int mx_in = 0, my_in = 0, mx_out = 0, my_out = 0;
  for (int c = 0; c < nf; ++c) mx_in |= vx[c] << c, my_in |= vy[c] << c;
  for (int f = 0; f < np; ++f) mx_out |= qx[f] << f, my_out |= qy[f] << f;
  for (int stage = 1; stage <= 4; ++stage) {
    const void* Uin = stage == 1 ? U0 : p->Ucur;
    const void* Tin = stage == 1 ? (const void*)T0 : (const void*)((const char*)p->Ucur + 3 * cs);
    a.stage = b.stage = stage;
    b.U1in = Uin;
    b.Tin = Tin;
    {
      ProfScope ps(p, TS_KCLASS_INV_X);
      if (T0 && stage > 1) {
        CK(LAUNCH(p, dealias_copy, g, Uin, P, 4, p->st));  // U and T are adjacent in Ucur
      } else {
        CK(LAUNCH(p, dealias_copy, g, Uin, P, 3, p->st));
        if (T0) CK(LAUNCH(p, dealias_copy, g, Tin, P + 3 * cs, 1, p->st));
      }
      CK(LAUNCH(p, sff_x, g, +1, P, 1, mx_in, 1.0, p->twq, p->st, nf, g.S));
    }
    {
      ProfScope ps(p, TS_KCLASS_Y_INV);
      CK(LAUNCH(p, sff_x, gy, +1, P, g.Nx, my_in, 1.0, p->twqy, p->st, nf, g.S));
    }
    {
      // z is a Fourier axis as on FFF: the fused z pass (inverse, the products of form 0
      // or 2 in real space, forward; unnormalised) reads the nf spectra and writes the
      // np product spectra in place
      ProfScope ps(p, TS_KCLASS_Z);
      CK(LAUNCH(p, z_fused, g, T0 ? 2 : 0, P, p->twz, p->err_d, p->st));
    }
    {
      ProfScope ps(p, TS_KCLASS_Y_FWD);
      CK(LAUNCH(p, sff_x, gy, -1, P, g.Nx, my_out, sy, p->twqy, p->st, np, g.S));
    }
    {
      ProfScope ps(p, TS_KCLASS_FWD_X);
      CK(LAUNCH(p, sff_x, g, -1, P, 1, mx_out, sx, p->twq, p->st, np, g.S));
      if (T0) CK(LAUNCH(p, ssf_rbc_epi, g, P, b, p->st));
      else CK(LAUNCH(p, ssf_epi, g, P, a, p->st));
    }
  }
  return TS_OK;
}

// ---------------------------------------------------------------------------
// SSS fluid step (sin/cos along every axis; sincostr_switch "SCC"), conservative,
// unforced, on real coefficients; with T the Boussinesq step as on SSF.  P holds
// [0, np): the nf coefficient lines after the x and y inverses, which the fused SSS
// z pass turns into the np product coefficients in place.
// ---------------------------------------------------------------------------
static int step_sss(ts_plan* p, void* U0, void* T0 = nullptr) {
  const Geo& g = p->g;
  const Geo gy = y_as_x(g);
  const long long cs = g.S * (long long)p->cb;
  const int nf = T0 ? 4 : 3, np = T0 ? 9 : 6;
  char* P = (char*)p->P;
  StageArgs a;
  memset(&a, 0, sizeof(a));
  a.U0 = U0;
  a.Uout = U0;
  a.Ucur = p->Ucur;
  a.tot = p->tot;
  a.dt = p->cfg.dt;
  a.err = p->err_d;
  a.ex = p->eax[0];
  a.ey = p->eax[1];
  a.ez = p->eax[2];
  SffArgs b = ssf_rbc_args(p, U0, T0);
  // sine (1) / cosine (0) letters: Vx = SCC, Vy = CSC, Vz = CCS, T = SCC; products u1u1,
  // u2u2, u3u3 (CCC), u1u2 (SSC), u2u3 (CSS), u3u1 (SCS), u1T (CCC), u2T (SSC), u3T (SCS)
  const int vx[4] = {1, 0, 0, 1}, vy[4] = {0, 1, 0, 0}, vz[4] = {0, 0, 1, 0};
  const int qx[9] = {0, 0, 0, 1, 0, 1, 0, 1, 1}, qy[9] = {0, 0, 0, 1, 1, 0, 0, 1, 0};
  const int qz[9] = {0, 0, 0, 0, 1, 1, 0, 0, 1};
  // the same letters as bit masks (bit c = field c), one batched launch per pass
  int mx_in = 0, my_in = 0, mx_out = 0, my_out = 0;
  for (int c = 0; c < nf; ++c) mx_in |= vx[c] << c, my_in |= vy[c] << c;
  for (int f = 0; f < np; ++f) mx_out |= qx[f] << f, my_out |= qy[f] << f;
  for (int stage = 1; stage <= 4; ++stage) {
    const void* Uin = stage == 1 ? U0 : p->Ucur;
    const void* Tin = stage == 1 ? (const void*)T0 : (const void*)((const char*)p->Ucur + 3 * cs);
    a.stage = b.stage = stage;
    b.U1in = Uin;
    b.Tin = Tin;
    {
      ProfScope ps(p, TS_KCLASS_INV_X);
      if (T0 && stage > 1) {
        CK(LAUNCH(p, sss_dealias_copy, g, Uin, P, 4, p->st));  // U and T are adjacent in Ucur
      } else {
        CK(LAUNCH(p, sss_dealias_copy, g, Uin, P, 3, p->st));
        if (T0) CK(LAUNCH(p, sss_dealias_copy, g, Tin, P + 3 * cs, 1, p->st));
      }
      CK(LAUNCH(p, sff_x, g, +1, P, 1, mx_in, 1.0, p->twq, p->st, nf, g.S));
    }
    {
      ProfScope ps(p, TS_KCLASS_Y_INV);
      CK(LAUNCH(p, sff_x, gy, +1, P, g.Nx, my_in, 1.0, p->twqy, p->st, nf, g.S));
    }
    {
      // the fused z pass: sin/cos inverse of the nf lines, the products, sin/cos forward
      ProfScope ps(p, TS_KCLASS_Z);
      int zin = 0, zout = 0;
      for (int c = 0; c < nf; ++c) zin |= vz[c] << c;
      for (int f = 0; f < np; ++f) zout |= qz[f] << f;
      CK(LAUNCH(p, sss_z_fused, g, T0 ? 2 : 0, P, p->twz, p->twqz, zin, zout, p->st));
    }
    {
      ProfScope ps(p, TS_KCLASS_Y_FWD);
      CK(LAUNCH(p, sff_x, gy, -1, P, g.Nx, my_out, 1.0 / (2.0 * g.Ny), p->twqy, p->st, np, g.S));
    }
    {
      ProfScope ps(p, TS_KCLASS_FWD_X);
      CK(LAUNCH(p, sff_x, g, -1, P, 1, mx_out, 1.0 / (2.0 * g.Nx), p->twq, p->st, np, g.S));
      if (T0) CK(LAUNCH(p, sss_rbc_epi, g, P, b, p->st));
      else CK(LAUNCH(p, sss_epi, g, P, a, p->st));
    }
  }
  return TS_OK;
}

// run fn(device_ptr) on a field that may live on the host
template <typename Fn>
static int with_device(ts_plan* p, void** stage, const void* ptr, size_t bytes, bool copy_back, Fn&& fn) {
  if (is_device_ptr(ptr)) return fn(const_cast<void*>(ptr));
  CKS(ensure_stage(stage, bytes));
  CK(cudaMemcpyAsync(*stage, ptr, bytes, cudaMemcpyHostToDevice, p->st));
  CKS(fn(*stage));
  if (copy_back) CK(cudaMemcpyAsync(const_cast<void*>(ptr), *stage, bytes, cudaMemcpyDeviceToHost, p->st));
  CK(cudaStreamSynchronize(p->st));
  return TS_OK;
}

extern "C" {

int ts_rk4_step(ts_plan* p, void* u_hat, int nsteps) {
  if (!p || !u_hat || nsteps < 0) return TS_ERR_ARG;
  if (p->cfg.basis == TS_BASIS_SSF || p->cfg.basis == TS_BASIS_SSS) {
    const bool sss = p->cfg.basis == TS_BASIS_SSS;
    CKS(ssf_step_supported(p, false));
    // the health word of earlier calls (copied back without a sync)
    if (*p->err_h) return health_status(p);
    int rc = with_device(p, &p->stage_u, u_hat, 3 * p->g.S * p->cb, true, [&](void* U) -> int {
      for (int s = 0; s < nsteps; ++s) CKS(sss ? step_sss(p, U) : step_ssf(p, U));
      return (int)TS_OK;
    });
    if (rc == TS_OK) CK(cudaMemcpyAsync(p->err_h, p->err_d, sizeof(int), cudaMemcpyDeviceToHost, p->st));
    return rc;
  }
  if (p->cfg.basis != TS_BASIS_FFF) return TS_ERR_UNSUPPORTED;
  // a bounded device wait that gave up in an earlier call (read without a sync)
  // the health word of earlier calls (copied back without a sync)
  if (*p->err_h) return health_status(p);
  int rc = with_device(p, &p->stage_u, u_hat, 3 * p->g.S * p->cb, true, [&](void* U) -> int {
    for (int s = 0; s < nsteps; ++s) CKS(step_fff(p, U));
    return (int)TS_OK;
  });
  if (rc == TS_OK) CK(cudaMemcpyAsync(p->err_h, p->err_d, sizeof(int), cudaMemcpyDeviceToHost, p->st));
  return rc;
}

static bool aligned16(const void* q) { return ((uintptr_t)q & 15) == 0; }

int ts_rk4_step_keep(ts_plan* p, const void* u_hat, void* u_next, void* stages) {
  if (!p || !u_hat || !u_next || !stages) return TS_ERR_ARG;
  if (p->cfg.basis != TS_BASIS_FFF) return TS_ERR_UNSUPPORTED;
  if (!is_device_ptr(u_hat) || !is_device_ptr(u_next) || !is_device_ptr(stages) || !aligned16(u_hat) ||
      !aligned16(u_next) || !aligned16(stages)) {
    g_last_error = "ts_rk4_step_keep: 16-byte aligned device pointers required";
    return TS_ERR_ARG;
  }
  // the health word of earlier calls (copied back without a sync)
  if (*p->err_h) return health_status(p);
  CKS(step_fff(p, const_cast<void*>(u_hat), u_next, stages));
  CK(cudaMemcpyAsync(p->err_h, p->err_d, sizeof(int), cudaMemcpyDeviceToHost, p->st));
  return TS_OK;
}

int ts_adjoint_step(ts_plan* p, const void* u_hat, const void* stages, void* lam_hat) {
  if (!p || !u_hat || !stages || !lam_hat) return TS_ERR_ARG;
  CKS(adjoint_supported(p));
  if (!is_device_ptr(u_hat) || !is_device_ptr(stages) || !is_device_ptr(lam_hat) || !aligned16(lam_hat)) {
    g_last_error = "ts_adjoint_step: device pointers required (lam_hat 16-byte aligned)";
    return TS_ERR_ARG;
  }
  // the health word of earlier calls (copied back without a sync)
  if (*p->err_h) return health_status(p);
  CKS(adjoint_step_fff(p, u_hat, stages, lam_hat));
  CK(cudaMemcpyAsync(p->err_h, p->err_d, sizeof(int), cudaMemcpyDeviceToHost, p->st));
  return TS_OK;
}

int ts_adjoint_work_bytes(const ts_plan* p, int nsteps, size_t* bytes) {
  if (!p || nsteps < 1 || !bytes) return TS_ERR_ARG;
  *bytes = (size_t)nsteps * 12 * (size_t)p->g.S * p->cb;
  return TS_OK;
}

int ts_adjoint_window(ts_plan* p, const void* u_start, int nsteps, void* lam_hat, void* work, size_t work_bytes) {
  if (!p || !u_start || !lam_hat || !work || nsteps < 1) return TS_ERR_ARG;
  CKS(adjoint_supported(p));
  size_t need = 0;
  CKS(ts_adjoint_work_bytes(p, nsteps, &need));
  if (work_bytes < need) {
    g_last_error = "ts_adjoint_window: work buffer smaller than ts_adjoint_work_bytes";
    return TS_ERR_ARG;
  }
  if (!is_device_ptr(u_start) || !is_device_ptr(lam_hat) || !is_device_ptr(work) || !aligned16(u_start) ||
      !aligned16(lam_hat) || !aligned16(work)) {
    g_last_error = "ts_adjoint_window: 16-byte aligned device pointers required";
    return TS_ERR_ARG;
  }
  // the health word of earlier calls (copied back without a sync)
  if (*p->err_h) return health_status(p);
  // work slot n = [U_n (3 components), U1, U2, U3 of step n (9)]; U_0 is u_start itself
  const size_t cs = 3 * (size_t)p->g.S * p->cb, slot = 4 * cs;
  char* w = (char*)work;
  auto state = [&](int n) -> void* { return n == 0 ? const_cast<void*>(u_start) : (void*)(w + n * slot); };
  for (int n = 0; n < nsteps; ++n) {
    const bool last = n == nsteps - 1;
    CKS(step_fff(p, state(n), last ? nullptr : state(n + 1), w + n * slot + cs, last));
  }
  for (int n = nsteps - 1; n >= 0; --n) CKS(adjoint_step_fff(p, state(n), w + n * slot + cs, lam_hat));
  CK(cudaMemcpyAsync(p->err_h, p->err_d, sizeof(int), cudaMemcpyDeviceToHost, p->st));
  return TS_OK;
}

int ts_rk4_step_rbc(ts_plan* p, void* u_hat, void* T_hat, int nsteps) {
  if (!p || !u_hat || !T_hat || nsteps < 0) return TS_ERR_ARG;
  if (p->cfg.basis == TS_BASIS_SSF || p->cfg.basis == TS_BASIS_SSS) {
    const bool sss = p->cfg.basis == TS_BASIS_SSS;
    if (p->rbc_slave) {
      g_last_error = "Pr_option PRZERO / PRINFTY step on SFF plans only";
      return TS_ERR_UNSUPPORTED;
    }
    CKS(ssf_step_supported(p, true));
    // the health word of earlier calls (copied back without a sync)
    if (*p->err_h) return health_status(p);
    const size_t bu = 3 * p->g.S * p->cb, bt = p->g.S * p->cb;
    int rc = with_device(p, &p->stage_u, u_hat, bu, true, [&](void* U) -> int {
      return with_device(p, &p->stage_t, T_hat, bt, true, [&](void* T) -> int {
        for (int s = 0; s < nsteps; ++s) CKS(sss ? step_sss(p, U, T) : step_ssf(p, U, T));
        return (int)TS_OK;
      });
    });
    if (rc == TS_OK) CK(cudaMemcpyAsync(p->err_h, p->err_d, sizeof(int), cudaMemcpyDeviceToHost, p->st));
    return rc;
  }
  if (p->cfg.basis != TS_BASIS_SFF) return TS_ERR_UNSUPPORTED;
  // the health word of earlier calls (copied back without a sync)
  if (*p->err_h) return health_status(p);
  const size_t bu = 3 * p->g.S * p->cb, bt = p->g.S * p->cb;
  int rc = with_device(p, &p->stage_u, u_hat, bu, true, [&](void* U) -> int {
    return with_device(p, &p->stage_t, T_hat, bt, true, [&](void* T) -> int {
      for (int s = 0; s < nsteps; ++s) CKS(step_rbc(p, U, T));
      return (int)TS_OK;
    });
  });
  if (rc == TS_OK) CK(cudaMemcpyAsync(p->err_h, p->err_d, sizeof(int), cudaMemcpyDeviceToHost, p->st));
  return rc;
}

int ts_rk4_step_scalar(ts_plan* p, void* u_hat, void* T_hat, int nsteps) {
  if (!p || !u_hat || !T_hat || nsteps < 0) return TS_ERR_ARG;
  CKS(scalar_supported(p));
  // the health word of earlier calls (copied back without a sync)
  if (*p->err_h) return health_status(p);
  const size_t bu = 3 * p->g.S * p->cb, bt = p->g.S * p->cb;
  int rc = with_device(p, &p->stage_u, u_hat, bu, true, [&](void* U) -> int {
    return with_device(p, &p->stage_t, T_hat, bt, true, [&](void* T) -> int {
      for (int s = 0; s < nsteps; ++s) CKS(step_scalar_fff(p, U, T));
      return (int)TS_OK;
    });
  });
  if (rc == TS_OK) CK(cudaMemcpyAsync(p->err_h, p->err_d, sizeof(int), cudaMemcpyDeviceToHost, p->st));
  return rc;
}

int ts_rk4_step_mhd(ts_plan* p, void* u_hat, void* b_hat, int nsteps) {
  if (!p || !u_hat || !b_hat || nsteps < 0) return TS_ERR_ARG;
  CKS(mhd_supported(p));
  // the health word of earlier calls (copied back without a sync)
  if (*p->err_h) return health_status(p);
  const size_t bu = 3 * p->g.S * p->cb;
  int rc = with_device(p, &p->stage_u, u_hat, bu, true, [&](void* U) -> int {
    return with_device(p, &p->stage_b, b_hat, bu, true, [&](void* B) -> int {
      for (int s = 0; s < nsteps; ++s) CKS(step_mhd_fff(p, U, B));
      return (int)TS_OK;
    });
  });
  if (rc == TS_OK) CK(cudaMemcpyAsync(p->err_h, p->err_d, sizeof(int), cudaMemcpyDeviceToHost, p->st));
  return rc;
}

int ts_init_temperature_perturbation(ts_plan* p, double amp, double kmax, uint64_t seed, void* T_hat) {
  if (!p || !T_hat || !(amp >= 0) || !(kmax >= 0)) return TS_ERR_ARG;
  if (p->cfg.basis != TS_BASIS_SFF) return TS_ERR_UNSUPPORTED;
  return with_device(p, &p->stage_t, T_hat, p->g.S * p->cb, true, [&](void* T) -> int {
    unsigned long long z = seed + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    CK(LAUNCH(p, init_temp, p->g, T, amp, kmax, z ^ (z >> 31), p->st));
    CK(LAUNCH(p, reality, p->g, T, 1, p->st));
    CK(cudaStreamSynchronize(p->st));
    return (int)TS_OK;
  });
}

int ts_nlin(ts_plan* p, void* u_hat, void* nlin_hat) {
  if (p && (p->cfg.basis == TS_BASIS_SSF || p->cfg.basis == TS_BASIS_SSS)) return ssf_transforms_only();
  if (!p || !u_hat || !nlin_hat) return TS_ERR_ARG;
  if (p->cfg.basis != TS_BASIS_FFF) return TS_ERR_UNSUPPORTED;
  const size_t bytes = 3 * p->g.S * p->cb;
  return with_device(p, &p->stage_u, u_hat, bytes, true, [&](void* U) -> int {
    // the reference dealiases U in place before the transforms (compute_nlin.cc:61-62)
    if (p->g.dealias) CK(LAUNCH(p, dealias_copy, p->g, U, U, 3, p->st));
    if (is_device_ptr(nlin_hat)) {
      StageArgs a;
      memset(&a, 0, sizeof(a));
      a.nout = nlin_hat;
      return rhs_fff(p, U, MODE_NLIN, a);
    }
    StageArgs a;
    memset(&a, 0, sizeof(a));
    a.nout = p->Ucur;
    CKS(rhs_fff(p, U, MODE_NLIN, a));
    CK(cudaMemcpyAsync(nlin_hat, p->Ucur, bytes, cudaMemcpyDeviceToHost, p->st));
    CK(cudaStreamSynchronize(p->st));
    return (int)TS_OK;
  });
}

int ts_energy(ts_plan* p, const void* a_hat, int ncomp, double* energy) {
  if (!p || !a_hat || !energy || ncomp < 1 || ncomp > 3) return TS_ERR_ARG;
  return with_device(p, &p->stage_u, a_hat, (size_t)ncomp * p->g.S * p->cb, false, [&](void* A) -> int {
    CK(cudaMemsetAsync(p->dscr, 0, sizeof(double), p->st));
    CK(LAUNCH(p, energy, p->g, A, A, ncomp, p->dscr, p->st));
    CK(cudaMemcpyAsync(energy, p->dscr, sizeof(double), cudaMemcpyDeviceToHost, p->st));
    CK(cudaStreamSynchronize(p->st));
    return (int)TS_OK;
  });
}

int ts_max_div(ts_plan* p, const void* u_hat, double* max_div) {
  if (!p || !u_hat || !max_div) return TS_ERR_ARG;
  return with_device(p, &p->stage_u, u_hat, 3 * p->g.S * p->cb, false, [&](void* U) -> int {
    CK(cudaMemsetAsync(p->dscr, 0, sizeof(double), p->st));
    CK(LAUNCH(p, maxdiv, p->g, U, (unsigned long long*)p->dscr, p->st));
    CK(cudaMemcpyAsync(max_div, p->dscr, sizeof(double), cudaMemcpyDeviceToHost, p->st));
    CK(cudaStreamSynchronize(p->st));
    return (int)TS_OK;
  });
}

int ts_shell_spectrum(ts_plan* p, const void* a_hat, int ncomp, double* Ek, int n_shells) {
  if (!p || !a_hat || !Ek || ncomp < 1 || ncomp > 3 || n_shells < 1) return TS_ERR_ARG;
  const int nsh = p->nshells;
  return with_device(p, &p->stage_u, a_hat, (size_t)ncomp * p->g.S * p->cb, false, [&](void* A) -> int {
    CKS(ensure_scratch(p, 2ull * nsh * (1 + shell_blocks(p->g, SHELL_MAX_BLOCKS))));
    CK(LAUNCH(p, shell, p->g, A, ncomp, nsh, p->dscr, p->st));
    std::vector<double> h(2 * nsh);
    CK(cudaMemcpyAsync(h.data(), p->dscr, 2 * nsh * sizeof(double), cudaMemcpyDeviceToHost, p->st));
    CK(cudaStreamSynchronize(p->st));
    // Stepanov normalisation (universal_energy.cc:350-362), 3D: 4 pi / (count kf1 kf2 kf3)
    const double kfp = p->g.kf[0] * p->g.kf[1] * p->g.kf[2];
    for (int i = 0; i < n_shells; ++i) {
      if (i >= nsh) { Ek[i] = 0; continue; }
      const double cnt = h[nsh + i];
      Ek[i] = cnt <= 0 ? 0.0 : h[i] * (4 * M_PI) / (cnt * kfp);
    }
    return (int)TS_OK;
  });
}

int ts_shell_sums(ts_plan* p, const void* a_hat, const void* b_hat, int ncomp, double* sums, double* counts,
                  int n_shells) {
  if (!p || !a_hat || ncomp < 1 || ncomp > 3 || n_shells < 1 || (!sums && !counts)) return TS_ERR_ARG;
  if (!is_device_ptr(a_hat) || (b_hat && !is_device_ptr(b_hat))) {
    g_last_error = "ts_shell_sums: device pointers required";
    return TS_ERR_ARG;
  }
  const int nsh = p->nshells;
  CKS(ensure_scratch(p, 2ull * nsh * (1 + shell_blocks(p->g, SHELL_MAX_BLOCKS))));
  CK(LAUNCH(p, shell, p->g, a_hat, ncomp, nsh, p->dscr, p->st, b_hat));
  std::vector<double> h(2 * nsh);
  CK(cudaMemcpyAsync(h.data(), p->dscr, 2 * nsh * sizeof(double), cudaMemcpyDeviceToHost, p->st));
  CK(cudaStreamSynchronize(p->st));
  for (int i = 0; i < n_shells; ++i) {
    if (sums) sums[i] = i < nsh ? h[i] : 0.0;
    if (counts) counts[i] = i < nsh ? h[nsh + i] : 0.0;
  }
  return TS_OK;
}

int ts_force_field(ts_plan* p, const void* u_hat, void* f_hat) {
  if (p && (p->cfg.basis == TS_BASIS_SSF || p->cfg.basis == TS_BASIS_SSS)) return ssf_transforms_only();
  if (!p || !u_hat || !f_hat) return TS_ERR_ARG;
  if (p->cfg.force_type != TS_FORCE_CARATI_ENERGY_SUPPLY) {
    g_last_error = "ts_force_field: the plan has no Carati forcing";
    return TS_ERR_UNSUPPORTED;
  }
  if (!is_device_ptr(u_hat) || !is_device_ptr(f_hat)) return TS_ERR_ARG;
  const Geo& g = p->g;
  CK(LAUNCH(p, carati, g, u_hat, p->fcube, p->fkm, p->cfg.force_inner_radius, p->cfg.force_outer_radius, p->esup,
            p->hsup, p->mis_d, p->nsup, p->st));
  CK(cudaMemsetAsync(f_hat, 0, 3 * g.S * p->cb, p->st));
  CK(LAUNCH(p, force_scatter, g, p->fcube, f_hat, p->fkm, p->st));
  CK(cudaStreamSynchronize(p->st));
  return TS_OK;
}

// the reference's per-sphere flux on the SSF and SFF bases: per radius the giver inputs
// (D U and D U inside the sphere), the x sin/cos inverse, the y inverse (sin/cos on SSF,
// FFT on SFF), the FFF z pass with the nine products u_j G_i, the y and x forward passes
// with the products' sine letters, and the sum outside the sphere (the step's passes,
// with the giver's product set)
static int flux_ssf(ts_plan* p, const void* U, const double* radii, int n_radii, double* Pi) {
  const Geo& g = p->g;
  const Geo gy = y_as_x(g);
  const bool sff = g.basis == TS_BASIS_SFF;
  const long long nb = 1 + 148 * 16;
  CKS(ensure_work(p, p->nS, 9));
  CKS(ensure_scratch(p, (size_t)n_radii * nb));
  // x, y sine letters of u (SSF: Vx = SCF, Vy = CSF, Vz = CCF; SFF: Vx = SFF, Vy = Vz = CFF,
  // no y letters), the giver has the same; the product u_j G_i (field 3 j + i) is a sine
  // series along an axis when exactly one factor is
  const int vx[3] = {1, 0, 0}, vy[3] = {0, sff ? 0 : 1, 0};
  int mx_in = 0, my_in = 0, mx_out = 0, my_out = 0;
  for (int c = 0; c < 3; ++c) {
    mx_in |= (vx[c] << c) | (vx[c] << (3 + c));
    my_in |= (vy[c] << c) | (vy[c] << (3 + c));
  }
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) {
      mx_out |= (vx[j] ^ vx[i]) << (3 * j + i);
      my_out |= (vy[j] ^ vy[i]) << (3 * j + i);
    }
  // forward normalisation: 1 / (2 Ny) on the SSF y sin/cos pass, and the rest
  // (1 / (2 Nx Nz), on SFF 1 / (2 Nx Ny Nz)) on the x pass
  const double sy = 1.0 / (2.0 * g.Ny), sx = 1.0 / (2.0 * g.Nx * (double)g.Nz * (sff ? g.Ny : 1));
  for (int r = 0; r < n_radii; ++r) {
    CK(LAUNCH(p, ssf_giver, g, U, p->P, radii[r], p->st));
    CK(LAUNCH(p, sff_x, g, +1, p->P, 1, mx_in, 1.0, p->twq, p->st, 6, g.S));
    if (sff) CK(LAUNCH(p, strided, g, 1, +1, p->P, 6, p->twy, p->st));
    else CK(LAUNCH(p, sff_x, gy, +1, p->P, g.Nx, my_in, 1.0, p->twqy, p->st, 6, g.S));
    CK(LAUNCH(p, z_fused, g, 6, p->P, p->twz, p->err_d, p->st));
    if (sff) CK(LAUNCH(p, strided, g, 1, -1, p->P, 9, p->twy, p->st));
    else CK(LAUNCH(p, sff_x, gy, -1, p->P, g.Nx, my_out, sy, p->twqy, p->st, 9, g.S));
    CK(LAUNCH(p, sff_x, g, -1, p->P, 1, mx_out, sx, p->twq, p->st, 9, g.S));
    CK(LAUNCH(p, ssf_flux_outside, g, p->P, U, radii[r], mx_out, my_out, p->dscr + r * nb, p->st));
  }
  std::vector<double> h(n_radii);
  for (int r = 0; r < n_radii; ++r)
    CK(cudaMemcpyAsync(&h[r], p->dscr + r * nb, sizeof(double), cudaMemcpyDeviceToHost, p->st));
  CK(cudaStreamSynchronize(p->st));
  for (int r = 0; r < n_radii; ++r) Pi[r] = -h[r];
  return TS_OK;
}

// the reference's per-sphere flux on the SSS basis (real coefficients; sincostr_switch
// "SCC": Vx = SCC, Vy = CSC, Vz = CCS, the giver the same): per radius the giver inputs,
// the x and y sin/cos inverses, the fused SSS z pass with the nine products u_j G_i
// (sin/cos inverse, products, sin/cos forward), the y and x forward passes with the
// products' sine letters, and the sum outside the sphere
static int flux_sss(ts_plan* p, const void* U, const double* radii, int n_radii, double* Pi) {
  const Geo& g = p->g;
  const Geo gy = y_as_x(g);
  const long long nb = 1 + 148 * 16;
  CKS(ensure_work(p, p->nS, 9));
  CKS(ensure_scratch(p, (size_t)n_radii * nb));
  const int vx[3] = {1, 0, 0}, vy[3] = {0, 1, 0}, vz[3] = {0, 0, 1};
  int mx_in = 0, my_in = 0, mz_in = 0, mx_out = 0, my_out = 0, mz_out = 0;
  for (int c = 0; c < 3; ++c) {
    mx_in |= (vx[c] << c) | (vx[c] << (3 + c));
    my_in |= (vy[c] << c) | (vy[c] << (3 + c));
    mz_in |= (vz[c] << c) | (vz[c] << (3 + c));
  }
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) {
      mx_out |= (vx[j] ^ vx[i]) << (3 * j + i);
      my_out |= (vy[j] ^ vy[i]) << (3 * j + i);
      mz_out |= (vz[j] ^ vz[i]) << (3 * j + i);
    }
  for (int r = 0; r < n_radii; ++r) {
    CK(LAUNCH(p, sss_giver, g, U, p->P, radii[r], p->st));
    CK(LAUNCH(p, sff_x, g, +1, p->P, 1, mx_in, 1.0, p->twq, p->st, 6, g.S));
    CK(LAUNCH(p, sff_x, gy, +1, p->P, g.Nx, my_in, 1.0, p->twqy, p->st, 6, g.S));
    CK(LAUNCH(p, sss_z_fused, g, 6, p->P, p->twz, p->twqz, mz_in, mz_out, p->st));
    CK(LAUNCH(p, sff_x, gy, -1, p->P, g.Nx, my_out, 1.0 / (2.0 * g.Ny), p->twqy, p->st, 9, g.S));
    CK(LAUNCH(p, sff_x, g, -1, p->P, 1, mx_out, 1.0 / (2.0 * g.Nx), p->twq, p->st, 9, g.S));
    CK(LAUNCH(p, sss_flux_outside, g, p->P, U, radii[r], mx_out, my_out, mz_out, p->dscr + r * nb, p->st));
  }
  std::vector<double> h(n_radii);
  for (int r = 0; r < n_radii; ++r)
    CK(cudaMemcpyAsync(&h[r], p->dscr + r * nb, sizeof(double), cudaMemcpyDeviceToHost, p->st));
  CK(cudaStreamSynchronize(p->st));
  for (int r = 0; r < n_radii; ++r) Pi[r] = -h[r];
  return TS_OK;
}

int ts_flux(ts_plan* p, const void* u_hat, const double* radii, int n_radii, double* Pi) {
  if (!p || !u_hat || !radii || !Pi || n_radii < 1) return TS_ERR_ARG;
  if (n_radii >= FLUX_MAX_BINS) {
    g_last_error = "ts_flux: at most " + std::to_string(FLUX_MAX_BINS - 1) + " radii";
    return TS_ERR_ARG;
  }
  // the reference's default radii need not ascend on small grids
  // (Global_process_advanced_vars.cc:133-154); the one-pass form bins ascending radii
  bool ascending = true;
  for (int i = 0; i < n_radii; ++i) {
    if (radii[i] != radii[i]) return TS_ERR_ARG;
    if (i > 0 && radii[i] < radii[i - 1]) ascending = false;
  }
  const Geo& g = p->g;
  if (p->cfg.basis == TS_BASIS_SSF || p->cfg.basis == TS_BASIS_SFF)
    return with_device(p, &p->stage_u, u_hat, 3 * g.S * p->cb, false,
                       [&](void* U) -> int { return flux_ssf(p, U, radii, n_radii, Pi); });
  if (p->cfg.basis == TS_BASIS_SSS)
    return with_device(p, &p->stage_u, u_hat, 3 * g.S * p->cb, false,
                       [&](void* U) -> int { return flux_sss(p, U, radii, n_radii, Pi); });
  const long long nb = 1 + 148 * 16;  // a result plus the per-block partials of one reduction
  return with_device(p, &p->stage_u, u_hat, 3 * g.S * p->cb, false, [&](void* U) -> int {
    std::vector<double> h(n_radii + 1);
    if (g.dealias == TS_DEALIAS_TWO_THIRDS && ascending) {
      // one pass: with two-thirds dealiasing the products of kept modes alias only onto
      // modes the dealiased field does not hold, so <u_<, (u.grad)u> = -<u_>, (u.grad)u_<>
      // and Pi(R) = sum_{|K| <= R} 2 mult Re(N . conj(D U)) from one nonlinear term
      CKS(ensure_scratch(p, (size_t)(n_radii + 1) * nb + n_radii));
      double* bins = p->dscr;
      double* rad = p->dscr + (n_radii + 1) * nb;
      CK(cudaMemcpyAsync(rad, radii, n_radii * sizeof(double), cudaMemcpyHostToDevice, p->st));
      StageArgs a;
      memset(&a, 0, sizeof(a));
      a.Ud = U;
      a.bins = bins;
      a.radii = rad;
      a.nradii = n_radii;
      CKS(rhs_fff(p, U, MODE_FLUX, a));
      CK(cudaMemcpyAsync(h.data(), bins, (n_radii + 1) * sizeof(double), cudaMemcpyDeviceToHost, p->st));
      CK(cudaStreamSynchronize(p->st));
      double acc = 0;
      for (int i = 0; i < n_radii; ++i) {
        acc += h[i];
        Pi[i] = acc;
      }
      return (int)TS_OK;
    }
    // the reference's per-sphere form (EnergyTr::Compute_flux, compute_flux.cc:51-65), which
    // under the corner-box (or no) dealiasing differs from the one-pass form by the aliased
    // part of the products: per radius R, the giver G = D U inside |K| <= R (Fill_in_sphere),
    // the giver nonlinear term N_i = sum_j D_j F[u_j G_i] (Compute_nlin(U, Giver)) and
    // Pi(R) = -sum_{|K| > R} 2 mult Re(N . conj(D U))
    CKS(ensure_work(p, p->nS, 9));
    CKS(ensure_scratch(p, (size_t)n_radii * nb));
    for (int i = 0; i < n_radii; ++i) {
      CK(LAUNCH(p, inv_x, g, 5, U, p->P, p->twx, nullptr, 0.0, p->st, 0, radii[i]));
      CK(LAUNCH(p, strided, g, 1, +1, p->P, 6, p->twy, p->st));
      CK(LAUNCH(p, z_fused, g, 6, p->P, p->twz, p->err_d, p->st));
      CK(LAUNCH(p, strided, g, 1, -1, p->P, 9, p->twy, p->st));
      CK(LAUNCH(p, strided, g, 0, -1, p->P, 9, p->twx, p->st));
      CK(LAUNCH(p, flux_outside, g, p->P, U, radii[i], p->dscr + i * nb, p->st));
    }
    for (int i = 0; i < n_radii; ++i)
      CK(cudaMemcpyAsync(&h[i], p->dscr + i * nb, sizeof(double), cudaMemcpyDeviceToHost, p->st));
    CK(cudaStreamSynchronize(p->st));
    for (int i = 0; i < n_radii; ++i) Pi[i] = -h[i];
    return (int)TS_OK;
  });
}

int ts_dealias_field(ts_plan* p, void* a_hat, int ncomp) {
  if (!p || !a_hat || ncomp < 1 || ncomp > 3) return TS_ERR_ARG;
  if (!p->g.dealias) return TS_OK;
  return with_device(p, &p->stage_u, a_hat, (size_t)ncomp * p->g.S * p->cb, true, [&](void* A) -> int {
    // SSS: real coefficients, each element read and written by the same thread
    if (p->cfg.basis == TS_BASIS_SSS) CK(LAUNCH(p, sss_dealias_copy, p->g, A, A, ncomp, p->st));
    else CK(LAUNCH(p, dealias_copy, p->g, A, A, ncomp, p->st));
    CK(cudaStreamSynchronize(p->st));
    return (int)TS_OK;
  });
}

int ts_nusselt(ts_plan* p, const void* u_hat, const void* T_hat, double* Nu) {
  if (!p || !u_hat || !T_hat || !Nu) return TS_ERR_ARG;
  if (p->cfg.basis == TS_BASIS_FFF) return TS_ERR_UNSUPPORTED;
  if (!is_device_ptr(u_hat) || !is_device_ptr(T_hat)) return TS_ERR_ARG;
  CK(cudaMemsetAsync(p->dscr, 0, sizeof(double), p->st));
  CK(LAUNCH(p, energy, p->g, u_hat, T_hat, 1, p->dscr, p->st));
  double e = 0;
  CK(cudaMemcpyAsync(&e, p->dscr, sizeof(double), cudaMemcpyDeviceToHost, p->st));
  CK(cudaStreamSynchronize(p->st));
  *Nu = p->rbc_nu0 + p->rbc_nuc * e;
  return TS_OK;
}

int ts_rbc_slave(ts_plan* p, void* u_hat, void* T_hat) {
  if (!p || !u_hat || !T_hat || !p->rbc_slave) return TS_ERR_ARG;
  if (p->cfg.basis != TS_BASIS_SFF) return TS_ERR_UNSUPPORTED;
  const size_t bu = 3 * p->g.S * p->cb, bt = p->g.S * p->cb;
  return with_device(p, &p->stage_u, u_hat, bu, true, [&](void* U) -> int {
    return with_device(p, &p->stage_t, T_hat, bt, true, [&](void* T) -> int {
      CK(LAUNCH(p, rbc_slave, p->g, U, T, p->rbc_slave, p->rbc_vs, p->st));
      CK(cudaStreamSynchronize(p->st));
      return (int)TS_OK;
    });
  });
}

int ts_init_energy_spectrum(ts_plan* p, const double* E_ic, int n, uint64_t seed, double target_energy,
                            void* u_hat) {
  if (p && (p->cfg.basis == TS_BASIS_SSF || p->cfg.basis == TS_BASIS_SSS)) return ssf_transforms_only();
  if (!p || !E_ic || n < 1 || !u_hat) return TS_ERR_ARG;
  if (p->cfg.basis != TS_BASIS_FFF) return TS_ERR_UNSUPPORTED;
  return with_device(p, &p->stage_u, u_hat, 3 * p->g.S * p->cb, true, [&](void* U) -> int {
    const int nsh = (int)p->mis.size();
    CKS(ensure_scratch(p, 2 * nsh + 1));
    std::vector<double> e(nsh, 0.0);
    for (int i = 0; i < n && i < nsh; ++i) e[i] = E_ic[i];
    double* Ed = p->dscr + 1;
    CK(cudaMemcpyAsync(Ed, e.data(), nsh * sizeof(double), cudaMemcpyHostToDevice, p->st));
    // key = splitmix64(seed), as the oracle's uniform01
    unsigned long long z = seed + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    const unsigned long long key = z ^ (z >> 31);
    CK(LAUNCH(p, init_ic, p->g, U, Ed, p->mis_d, nsh, key, p->st));
    CK(LAUNCH(p, reality, p->g, U, 3, p->st));
    if (target_energy > 0) {
      CK(cudaMemsetAsync(p->dscr, 0, sizeof(double), p->st));
      CK(LAUNCH(p, energy, p->g, U, U, 3, p->dscr, p->st));
      double en = 0;
      CK(cudaMemcpyAsync(&en, p->dscr, sizeof(double), cudaMemcpyDeviceToHost, p->st));
      CK(cudaStreamSynchronize(p->st));
      if (!(en > 0)) return (int)TS_ERR_ARG;
      CK(LAUNCH(p, scale, U, 3 * p->g.S, sqrt(target_energy / en), p->st));
    }
    CK(cudaStreamSynchronize(p->st));
    return (int)TS_OK;
  });
}

// parity string -> x basis: FFF plans take "FFF"; SFF plans take "SFF" (sine
// along x) or "CFF" (cosine), the first letter of the reference's
// sincostr_switch entries (global/Global.cc:137-145).  Returns -1 if invalid.
// x parity: 0 Fourier (FFF), 1 sine, 2 cosine; *yp: the y parity of an SSF plan
// (1 sine, 2 cosine; 0 Fourier otherwise)
static int x_parity(const ts_plan* p, const char* parity, int* yp = nullptr, int* zp = nullptr) {
  if (yp) *yp = 0;
  if (zp) *zp = 0;
  if (p->cfg.basis == TS_BASIS_FFF) return strcmp(parity, "FFF") == 0 ? 0 : -1;
  if (p->cfg.basis == TS_BASIS_SSS) {
    if (strlen(parity) != 3) return -1;
    int l[3];
    for (int i = 0; i < 3; ++i) {
      l[i] = parity[i] == 'S' ? 1 : (parity[i] == 'C' ? 2 : -1);
      if (l[i] < 0) return -1;
    }
    if (yp) *yp = l[1];
    if (zp) *zp = l[2];
    return l[0];
  }
  if (p->cfg.basis == TS_BASIS_SSF) {
    if (strlen(parity) != 3 || parity[2] != 'F') return -1;
    const int x = parity[0] == 'S' ? 1 : (parity[0] == 'C' ? 2 : -1);
    const int y = parity[1] == 'S' ? 1 : (parity[1] == 'C' ? 2 : -1);
    if (x < 0 || y < 0) return -1;
    if (yp) *yp = y;
    return x;
  }
  if (strcmp(parity, "SFF") == 0) return 1;
  if (strcmp(parity, "CFF") == 0) return 2;
  return -1;
}


int ts_fft_forward(ts_plan* p, const char* parity, const void* real_in, void* spec_out, int ncomp) {
  if (!p || !parity || !real_in || !spec_out || ncomp < 1 || ncomp > 3) return TS_ERR_ARG;
  int yp = 0, zp = 0;
  const int xp = x_parity(p, parity, &yp, &zp);
  if (xp < 0) {
    g_last_error = "parity must be \"FFF\" (FFF plan), \"SFF\" / \"CFF\" (SFF plan), [SC][SC]F (SSF plan) or "
                   "[SC][SC][SC] (SSS plan)";
    return TS_ERR_ARG;
  }
  if (!is_device_ptr(real_in) || !is_device_ptr(spec_out)) return TS_ERR_ARG;
  const Geo& g = p->g;
  if (zp) {
    // SSS: sin/cos / (2 Nz) along z on the real lines, then y and x on the coefficient
    // pairs viewed as complex (each pass acts on both reals of a pair)
    const long long cs = g.S * (long long)p->cb, nl = (long long)ncomp * g.Nx * g.Ny;
    char* P = (char*)p->P;
    CK(LAUNCH(p, sss_zperm_fwd, real_in, P, nl, g.Nz, zp == 1, p->st));
    CK(LAUNCH(p, z_single, g, -1, P, P + 3 * cs, ncomp, p->twz, p->st));
    CK(LAUNCH(p, sss_zpost_fwd, P + 3 * cs, spec_out, nl, g.Nz, zp == 1, 1.0 / (2.0 * g.Nz), p->twqz, p->st));
    CK(LAUNCH(p, sff_x, y_as_x(g), -1, spec_out, ncomp * g.Nx, yp == 1, 1.0 / (2.0 * g.Ny), p->twqy, p->st));
    CK(LAUNCH(p, sff_x, g, -1, spec_out, ncomp, xp == 1, 1.0 / (2.0 * g.Nx), p->twq, p->st));
    return TS_OK;
  }
  if (yp) {
    // SSF (SSF_pencil_tr.cc:43-51): z Fourier, then sin/cos / (2 Ny) along y, sin/cos
    // / (2 Nx) along x with the z normalisation
    CK(LAUNCH(p, z_single, g, -1, real_in, spec_out, ncomp, p->twz, p->st));
    CK(LAUNCH(p, sff_x, y_as_x(g), -1, spec_out, ncomp * g.Nx, yp == 1, 1.0 / (2.0 * g.Ny), p->twqy, p->st));
    CK(LAUNCH(p, sff_x, g, -1, spec_out, ncomp, xp == 1, 1.0 / (2.0 * g.Nx * (double)g.Nz), p->twq, p->st));
    return TS_OK;
  }
  CK(LAUNCH(p, z_single, g, -1, real_in, spec_out, ncomp, p->twz, p->st));
  CK(LAUNCH(p, strided, g, 1, -1, spec_out, ncomp, p->twy, p->st));
  if (xp == 0) {
    CK(LAUNCH(p, strided, g, 0, -1, spec_out, ncomp, p->twx, p->st));
    CK(LAUNCH(p, scale, spec_out, ncomp * g.S, 1.0 / ((double)g.Nx * g.Ny * g.Nz), p->st));
  } else {
    // sin/cos analysis / (2 Nx) along x (SFF_pencil_tr.cc:43-55), Fourier / (Ny Nz) along y, z
    CK(LAUNCH(p, sff_x, g, -1, spec_out, ncomp, xp == 1, 1.0 / (2.0 * g.Nx * (double)g.Ny * g.Nz), p->twq, p->st));
  }
  return TS_OK;
}

int ts_fft_inverse(ts_plan* p, const char* parity, const void* spec_in, void* real_out, int ncomp) {
  if (!p || !parity || !spec_in || !real_out || ncomp < 1 || ncomp > 3) return TS_ERR_ARG;
  int yp = 0, zp = 0;
  const int xp = x_parity(p, parity, &yp, &zp);
  if (xp < 0) {
    g_last_error = "parity must be \"FFF\" (FFF plan), \"SFF\" / \"CFF\" (SFF plan), [SC][SC]F (SSF plan) or "
                   "[SC][SC][SC] (SSS plan)";
    return TS_ERR_ARG;
  }
  if (!is_device_ptr(spec_in) || !is_device_ptr(real_out)) return TS_ERR_ARG;
  const Geo& g = p->g;
  // the reference copies the input to X_transform first (FFF_pencil_tr.cc:59)
  CK(cudaMemcpyAsync(p->P, spec_in, ncomp * g.S * p->cb, cudaMemcpyDeviceToDevice, p->st));
  if (zp) {
    const long long cs = g.S * (long long)p->cb, nl = (long long)ncomp * g.Nx * g.Ny;
    char* P = (char*)p->P;
    CK(LAUNCH(p, sff_x, g, +1, P, ncomp, xp == 1, 1.0, p->twq, p->st));
    CK(LAUNCH(p, sff_x, y_as_x(g), +1, P, ncomp * g.Nx, yp == 1, 1.0, p->twqy, p->st));
    CK(LAUNCH(p, sss_zpre_inv, P, P + 3 * cs, nl, g.Nz, zp == 1, p->twqz, p->st));
    CK(LAUNCH(p, z_single, g, +1, P + 3 * cs, P + 6 * cs, ncomp, p->twz, p->st));
    CK(LAUNCH(p, sss_zperm_inv, P + 6 * cs, real_out, nl, g.Nz, zp == 1, p->st));
    return TS_OK;
  }
  if (yp) {
    CK(LAUNCH(p, sff_x, g, +1, p->P, ncomp, xp == 1, 1.0, p->twq, p->st));
    CK(LAUNCH(p, sff_x, y_as_x(g), +1, p->P, ncomp * g.Nx, yp == 1, 1.0, p->twqy, p->st));
    CK(LAUNCH(p, z_single, g, +1, p->P, real_out, ncomp, p->twz, p->st));
    return TS_OK;
  }
  if (xp == 0) CK(LAUNCH(p, strided, g, 0, +1, p->P, ncomp, p->twx, p->st));
  else CK(LAUNCH(p, sff_x, g, +1, p->P, ncomp, xp == 1, 1.0, p->twq, p->st));
  CK(LAUNCH(p, strided, g, 1, +1, p->P, ncomp, p->twy, p->st));
  CK(LAUNCH(p, z_single, g, +1, p->P, real_out, ncomp, p->twz, p->st));
  return TS_OK;
}

}  // extern "C"

extern "C" {

int ts_profile_enable(ts_plan* p, int enable) {
  if (!p) return TS_ERR_ARG;
  prof_collect(p);
  p->prof = enable != 0;
  return TS_OK;
}

int ts_profile_reset(ts_plan* p) {
  if (!p) return TS_ERR_ARG;
  prof_collect(p);
  for (int i = 0; i < TS_KCLASS_COUNT; ++i) {
    p->prof_ms[i] = 0;
    p->prof_n[i] = 0;
    p->prof_bytes[i] = 0;
    p->prof_nb[i] = 0;
  }
  return TS_OK;
}

int ts_profile_read(ts_plan* p, int kclass, double* total_ms, long long* launches, double* bytes_per_launch) {
  if (!p || kclass < 0 || kclass >= TS_KCLASS_COUNT) return TS_ERR_ARG;
  prof_collect(p);
  if (total_ms) *total_ms = p->prof_ms[kclass];
  if (launches) *launches = p->prof_n[kclass];
  if (bytes_per_launch && p->prof_nb[kclass] > 0 && p->prof_nb[kclass] == p->prof_n[kclass]) {
    // every launch recorded its own algorithmic bytes (the FFF step and the adjoint)
    *bytes_per_launch = p->prof_bytes[kclass] / (double)p->prof_nb[kclass];
  } else if (bytes_per_launch) {
    // static model: every field a launch must read or write, once
    const double f = (double)p->g.S * (double)p->cb;
    const int rot = p->cfg.nlin_form == TS_NLIN_ROTATIONAL;
    double b = 0;
    if (p->cfg.basis == TS_BASIS_SFF) {
      // u1, u2, u3, T in; nine products out; the epilogue's state traffic averages 16 fields over a step
      const double sff[TS_KCLASS_COUNT] = {8 * f, 8 * f, 13 * f, 18 * f, 25 * f, 0};
      *bytes_per_launch = kclass < TS_KCLASS_COUNT ? sff[kclass] : 0;
      return TS_OK;
    }
    switch (kclass) {
      case TS_KCLASS_INV_X: b = (3 + (rot ? 6 : 3)) * f; break;          // read U, write W
      case TS_KCLASS_Y_INV: b = 2.0 * (rot ? 6 : 3) * f; break;          // in place
      case TS_KCLASS_Z: b = (rot ? 6 + 3 : 3 + 6) * f; break;            // read W, write P
      case TS_KCLASS_Y_FWD: b = 2.0 * (rot ? 3 : 6) * f; break;
      case TS_KCLASS_FWD_X: b = ((rot ? 3 : 6) + 13.5) * f; break;       // P + stage-averaged state traffic
      default: b = 0; break;
    }
    *bytes_per_launch = b;
  }
  return TS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Ensemble of independent RBC runs (uneven sizes).  Members of the same grid
// form a group whose fields sit in contiguous arrays (member stride = its
// field count x S), so every kernel of a group step covers all of its members
// in one launch (member = blockIdx.y, or folded into the field / line count);
// each member keeps its own integrating-factor tables (its Ra sets nu, kappa).
// One ensemble step = one CUDA graph launch whose parallel branches are the
// groups' step sequences (fork on the origin stream, one stream per group).
// Every member also has its own plan, used for diagnostics and for stepping a
// member on its own; its state is a view into the group arrays.
// ---------------------------------------------------------------------------
struct ens_group {
  std::vector<int> idx;  // member indices
  ts_plan* gp = nullptr; // the first member's plan: geometry, twiddles, error word
  void* U = nullptr;     // B x 3S
  void* T = nullptr;     // B x S
  void* Ucur = nullptr;  // B x 4S
  void* tot = nullptr;   // B x 4S
  void* P = nullptr;     // B x 9S
  double* eu = nullptr;  // B x (Nx + Ny + Hz): exp(-nu dt K_i^2 / 2) per axis, per member
  double* et = nullptr;  // same with kappa
  cudaStream_t st = nullptr;
  cudaEvent_t done = nullptr;
  int* health = nullptr;  // B health words (a slice of the ensemble's array), member j at j
};

struct ts_ensemble {
  std::vector<ts_plan*> plans;
  std::vector<void*> U, T;  // member views into the group arrays
  std::vector<ens_group> groups;
  int* health = nullptr;    // one health word per member, in group order (ens_group::health)
  cudaEvent_t fork = nullptr;
  cudaStream_t origin = nullptr;
  bool own_origin = false;
  cudaGraph_t graph = nullptr;      // one ensemble step
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graphK = nullptr;     // kEnsSteps ensemble steps, each group a chain of its own
  cudaGraphExec_t execK = nullptr;
  // graph schedule of the size groups: parallel branches between one fork and one join,
  // or (serial) one chain, group after group, each with the GPU to itself
  bool serial = false;
};
// ensemble steps per launch of the multi-step graph: the size groups advance this many
// steps between one fork and one join, so a group does not wait for the slowest one
// after every step
constexpr int kEnsSteps = 8;

// one IF-RK4 step of every member of a group (step_rbc with member strides)
static int step_rbc_group(ens_group& G) {
  ts_plan* p = G.gp;
  const Geo& g = p->g;
  const int B = (int)G.idx.size();
  const long long S = g.S, cb = (long long)p->cb;
  const long long TL = (long long)g.Nx + g.Ny + g.Hz;
  SffArgs a;
  memset(&a, 0, sizeof(a));
  a.cu = G.gp->rbc_cu;
  a.cT = G.gp->rbc_cT;
  a.U0 = G.U;
  a.T0 = G.T;
  a.Ucur = G.Ucur;
  a.tot = G.tot;
  a.dt = p->cfg.dt;
  a.reality = p->cfg.reality_fix;
  const long long aoff[3] = {0, g.Nx, (long long)g.Nx + g.Ny};
  for (int i = 0; i < 3; ++i) {
    a.eu[i] = G.eu + aoff[i];
    a.et[i] = G.et + aoff[i];
  }
  a.mtab = TL;
  a.health = G.health;
  a.msU0 = 3 * S;
  a.msT0 = S;
  a.msUcur = 4 * S;
  a.msTot = 4 * S;
  a.msP = 9 * S;
  for (int stage = 1; stage <= 4; ++stage) {
    const void* Uin = stage == 1 ? G.U : G.Ucur;
    const void* Tin = stage == 1 ? G.T : (const void*)((const char*)G.Ucur + 3 * S * cb);
    const long long msUin = stage == 1 ? 3 * S : 4 * S, msTin = stage == 1 ? S : 4 * S;
    a.stage = stage;
    a.U1in = Uin;
    a.Tin = Tin;
    a.msU1in = msUin;
    a.msTin = msTin;
    CK(LAUNCH(p, sff_inv_x, g, Uin, Tin, G.P, p->twq, G.st, B, msUin, msTin, 9 * S));
    CK(LAUNCH(p, strided, g, 1, +1, G.P, 4 * B, p->twy, G.st, 4, 9 * S));
    CK(LAUNCH(p, z_fused, g, 2, G.P, p->twz, p->err_d, G.st, B, 9 * S));
    CK(LAUNCH(p, strided, g, 1, -1, G.P, 9 * B, p->twy, G.st));
    CK(LAUNCH(p, sff_fwd_x, g, G.P, a, p->twq, G.st, B));
  }
  if (p->cfg.reality_fix) {
    CK(LAUNCH(p, reality, g, G.U, 3 * B, G.st));
    CK(LAUNCH(p, reality, g, G.T, B, G.st));
  }
  return TS_OK;
}

extern "C" {

int ts_ensemble_destroy(ts_ensemble* e) {
  if (!e) return TS_ERR_ARG;
  if (e->exec) cudaGraphExecDestroy(e->exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  if (e->execK) cudaGraphExecDestroy(e->execK);
  if (e->graphK) cudaGraphDestroy(e->graphK);
  for (ens_group& G : e->groups) {
    void* bufs[] = {G.U, G.T, G.Ucur, G.tot, G.P, G.eu, G.et};
    for (void* b : bufs)
      if (b) cudaFree(b);
    if (G.st) cudaStreamDestroy(G.st);
    if (G.done) cudaEventDestroy(G.done);
  }
  for (ts_plan* p : e->plans)
    if (p) ts_plan_destroy(p);
  if (e->health) cudaFree(e->health);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->own_origin && e->origin) cudaStreamDestroy(e->origin);
  delete e;
  return TS_OK;
}

int ts_ensemble_create(const ts_config* base, const ts_member* members, int count, ts_ensemble** out) {
  if (!base || !members || count < 1 || !out) return TS_ERR_ARG;
  *out = nullptr;
  ts_ensemble* e = new ts_ensemble();
  auto fail = [&](int rc) {
    ts_ensemble_destroy(e);
    return rc;
  };
  if (cudaStreamCreateWithFlags(&e->origin, cudaStreamNonBlocking) != cudaSuccess) return fail(TS_ERR_CUDA);
  e->own_origin = true;
  if (cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess) return fail(TS_ERR_CUDA);
  e->plans.assign(count, nullptr);
  e->U.assign(count, nullptr);
  e->T.assign(count, nullptr);
  std::vector<int> gof(count, -1);
  for (int m = 0; m < count; ++m) {
    ts_config c = *base;
    c.basis = TS_BASIS_SFF;
    c.force_type = TS_FORCE_RBC;
    for (int i = 0; i < 3; ++i) c.N[i] = members[m].N[i];
    c.Ra = members[m].Ra;
    c.Pr = members[m].Pr;
    if (!(c.Ra > 0) || !(c.Pr > 0)) return fail(TS_ERR_ARG);
    if (c.Pr_option == TS_PR_ZERO || c.Pr_option == TS_PR_INFTY) {
      g_last_error = "ensembles step PRLARGE / PRSMALL members (no slaved field)";
      return fail(TS_ERR_UNSUPPORTED);
    }
    // nu, kappa of the scaling (Iscalar_main.cc:52-92; ULARGE: sqrt(Pr/Ra), 1/sqrt(Pr Ra))
    double cu, cT, nu0, nuc;
    const int rs = rbc_coefficients(c.Pr_option, c.Uscaling, c.Ra, c.Pr, &c.nu, &c.kappa, &cu, &cT, &nu0, &nuc);
    if (rs != TS_OK) return fail(rs);
    int rc = ts_plan_create(&c, &e->plans[m]);
    if (rc != TS_OK) return fail(rc);
    for (size_t k = 0; k < e->groups.size() && gof[m] < 0; ++k) {
      const Geo& h = e->groups[k].gp->g;
      if (h.Nx == c.N[0] && h.Ny == c.N[1] && h.Nz == c.N[2]) gof[m] = (int)k;
    }
    if (gof[m] < 0) {
      e->groups.emplace_back();
      e->groups.back().gp = e->plans[m];
      gof[m] = (int)e->groups.size() - 1;
    }
    e->groups[gof[m]].idx.push_back(m);
  }
  // one launch covers a group's members with the group's buoyancy coefficients: they must
  // agree (they do for PRLARGE / ULARGE, cu = cT = 1; other scalings carry Ra or Pr)
  for (ens_group& G : e->groups)
    for (int m : G.idx)
      if (e->plans[m]->rbc_cu != G.gp->rbc_cu || e->plans[m]->rbc_cT != G.gp->rbc_cT) {
        g_last_error = "ensemble members of one grid size need equal buoyancy coefficients (PRLARGE / ULARGE)";
        return fail(TS_ERR_UNSUPPORTED);
      }
  if (cudaMalloc(&e->health, count * sizeof(int)) != cudaSuccess) return fail(TS_ERR_NOMEM);
  if (cudaMemset(e->health, 0, count * sizeof(int)) != cudaSuccess) return fail(TS_ERR_CUDA);
  size_t hoff = 0;
  for (ens_group& G : e->groups) {
    G.health = e->health + hoff;
    hoff += G.idx.size();
  }
  for (ens_group& G : e->groups) {
    const Geo& g = G.gp->g;
    const size_t B = G.idx.size(), S = (size_t)g.S, cb = G.gp->cb;
    const size_t TL = (size_t)g.Nx + g.Ny + g.Hz;
    if (cudaMalloc(&G.U, B * 3 * S * cb) != cudaSuccess || cudaMalloc(&G.T, B * S * cb) != cudaSuccess ||
        cudaMalloc(&G.Ucur, B * 4 * S * cb) != cudaSuccess || cudaMalloc(&G.tot, B * 4 * S * cb) != cudaSuccess ||
        cudaMalloc(&G.P, B * 9 * S * cb) != cudaSuccess || cudaMalloc(&G.eu, B * TL * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&G.et, B * TL * sizeof(double)) != cudaSuccess)
      return fail(TS_ERR_NOMEM);
    if (cudaMemset(G.U, 0, B * 3 * S * cb) != cudaSuccess || cudaMemset(G.T, 0, B * S * cb) != cudaSuccess)
      return fail(TS_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&G.st, cudaStreamNonBlocking) != cudaSuccess) return fail(TS_ERR_CUDA);
    if (cudaEventCreateWithFlags(&G.done, cudaEventDisableTiming) != cudaSuccess) return fail(TS_ERR_CUDA);
    const size_t n[3] = {(size_t)g.Nx, (size_t)g.Ny, (size_t)g.Hz}, off[3] = {0, (size_t)g.Nx, (size_t)g.Nx + g.Ny};
    for (size_t j = 0; j < B; ++j) {
      ts_plan* p = e->plans[G.idx[j]];
      p->st = G.st;
      e->U[G.idx[j]] = (char*)G.U + j * 3 * S * cb;
      e->T[G.idx[j]] = (char*)G.T + j * S * cb;
      for (int i = 0; i < 3; ++i) {
        if (cudaMemcpy(G.eu + j * TL + off[i], p->eax[i], n[i] * sizeof(double), cudaMemcpyDeviceToDevice) !=
                cudaSuccess ||
            cudaMemcpy(G.et + j * TL + off[i], p->eaxT[i], n[i] * sizeof(double), cudaMemcpyDeviceToDevice) !=
                cudaSuccess)
          return fail(TS_ERR_CUDA);
      }
    }
  }
  *out = e;
  return TS_OK;
}

int ts_ensemble_member(ts_ensemble* e, int m, ts_plan** plan, void** u_hat, void** T_hat) {
  if (!e || m < 0 || m >= (int)e->plans.size()) return TS_ERR_ARG;
  if (plan) *plan = e->plans[m];
  if (u_hat) *u_hat = e->U[m];
  if (T_hat) *T_hat = e->T[m];
  return TS_OK;
}

int ts_ensemble_init_temperature(ts_ensemble* e, double amp, double kmax, uint64_t seed) {
  if (!e) return TS_ERR_ARG;
  CK(cudaStreamSynchronize(e->origin));
  for (size_t m = 0; m < e->plans.size(); ++m) {
    CK(cudaMemset(e->U[m], 0, 3 * e->plans[m]->g.S * e->plans[m]->cb));
    CKS(ts_init_temperature_perturbation(e->plans[m], amp, kmax, seed + m, e->T[m]));
  }
  return TS_OK;
}

// captures `steps` ensemble steps into one graph: a fork on the origin stream, each
// size group's steps as one chain on its own stream, a join
static int ens_capture(ts_ensemble* e, int steps, cudaGraph_t* graph_out, cudaGraphExec_t* exec_out) {
  for (ts_plan* p : e->plans) p->prof = false;
  CK(cudaDeviceSynchronize());
  CK(cudaStreamBeginCapture(e->origin, cudaStreamCaptureModeRelaxed));
  int rc = TS_OK;
  cudaEventRecord(e->fork, e->origin);
  for (size_t k = 0; k < e->groups.size() && rc == TS_OK; ++k) {
    ens_group& G = e->groups[k];
    // parallel: every group starts at the fork; serial: after the previous group
    cudaStreamWaitEvent(G.st, (e->serial && k > 0) ? e->groups[k - 1].done : e->fork, 0);
    for (int s = 0; s < steps && rc == TS_OK; ++s) rc = step_rbc_group(G);
    cudaEventRecord(G.done, G.st);
    if (!e->serial || k + 1 == e->groups.size()) cudaStreamWaitEvent(e->origin, G.done, 0);
  }
  cudaGraph_t graph = nullptr;
  cudaError_t ce = cudaStreamEndCapture(e->origin, &graph);
  if (rc != TS_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  CK(ce);
  *graph_out = graph;
  CK(cudaGraphInstantiate(exec_out, graph, 0));
  return TS_OK;
}

int ts_ensemble_run(ts_ensemble* e, int nsteps) {
  if (!e || nsteps < 0) return TS_ERR_ARG;
  if (nsteps >= kEnsSteps && !e->execK) CKS(ens_capture(e, kEnsSteps, &e->graphK, &e->execK));
  if (nsteps % kEnsSteps && !e->exec) CKS(ens_capture(e, 1, &e->graph, &e->exec));
  for (int s = 0; s < nsteps / kEnsSteps; ++s) CK(cudaGraphLaunch(e->execK, e->origin));
  for (int s = 0; s < nsteps % kEnsSteps; ++s) CK(cudaGraphLaunch(e->exec, e->origin));
  return TS_OK;
}

int ts_ensemble_synchronize(ts_ensemble* e) {
  if (!e) return TS_ERR_ARG;
  CK(cudaStreamSynchronize(e->origin));
  return TS_OK;
}

int ts_ensemble_health(ts_ensemble* e, int* status, int clear) {
  if (!e || !status) return TS_ERR_ARG;
  CK(cudaStreamSynchronize(e->origin));
  std::vector<int> h(e->plans.size(), 0);
  CK(cudaMemcpy(h.data(), e->health, h.size() * sizeof(int), cudaMemcpyDeviceToHost));
  size_t off = 0;
  for (ens_group& G : e->groups) {
    // a bounded wait that gave up in a group's launch counts against all its members
    int ge = 0;
    CK(cudaMemcpy(&ge, G.gp->err_d, sizeof(int), cudaMemcpyDeviceToHost));
    for (size_t j = 0; j < G.idx.size(); ++j) {
      const int w = h[off + j] | ge;
      status[G.idx[j]] = (w & HEALTH_TIMEOUT) ? TS_ERR_TIMEOUT : ((w & HEALTH_NONFINITE) ? TS_ERR_NAN : TS_OK);
    }
    off += G.idx.size();
    if (clear) {
      CK(cudaMemset(G.gp->err_d, 0, sizeof(int)));
      *G.gp->err_h = 0;
    }
  }
  if (clear) CK(cudaMemset(e->health, 0, e->plans.size() * sizeof(int)));
  return TS_OK;
}

int ts_ensemble_nusselt(ts_ensemble* e, double* Nu) {
  if (!e || !Nu) return TS_ERR_ARG;
  CK(cudaStreamSynchronize(e->origin));
  for (size_t m = 0; m < e->plans.size(); ++m) CKS(ts_nusselt(e->plans[m], e->U[m], e->T[m], &Nu[m]));
  return TS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// launch tuning: coordinate descent over the five pass classes of a step
// ---------------------------------------------------------------------------
namespace {

const char* const kTuneName[TUNE_NCLASS] = {"x_inv", "y_inv", "z", "y_fwd", "x_fwd"};

int plan_form(const ts_plan* p) { return p->cfg.basis == TS_BASIS_SFF ? 2 : p->cfg.nlin_form; }

bool tune_valid(const ts_plan* p, const Geo& g, int cls, int v) {
  return p->prec == 1 ? Launch<float>::tune_valid(g, plan_form(p), cls, v)
                      : Launch<double>::tune_valid(g, plan_form(p), cls, v);
}
bool tune_blocks(const ts_plan* p, const Geo& g, int cls) {
  return p->prec == 1 ? Launch<float>::tune_blocks(g, plan_form(p), cls)
                      : Launch<double>::tune_blocks(g, plan_form(p), cls);
}

// best over `reps` trials of the time of n calls of fn on stream st, per call
template <typename Fn> int time_calls(cudaStream_t st, int n, int reps, Fn&& fn, double* ms) {
  cudaEvent_t a = nullptr, b = nullptr;
  CK(cudaEventCreate(&a));
  if (cudaEventCreate(&b) != cudaSuccess) {
    cudaEventDestroy(a);
    return TS_ERR_CUDA;
  }
  int rc = fn();  // warm-up (first launches of a new kernel candidate)
  double best = 1e300;
  for (int r = 0; r < reps && rc == TS_OK; ++r) {
    cudaEventRecord(a, st);
    for (int i = 0; i < n && rc == TS_OK; ++i) rc = fn();
    cudaEventRecord(b, st);
    float t = 0;
    if (rc == TS_OK && (cudaEventSynchronize(b) != cudaSuccess || cudaEventElapsedTime(&t, a, b) != cudaSuccess))
      rc = TS_ERR_CUDA;
    if (rc == TS_OK && t / n < best) best = t / n;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms = best;
  return rc;
}

void json_num(std::string& js, double x) {
  char buf[64];
  snprintf(buf, sizeof(buf), "%.6g", x);
  js += buf;
}

// Tunes g (the geometry a plan's or a group's launches read) class by class;
// measure(&ms) times the objective with the current g.  Appends a JSON object.
template <typename Measure> int descend(const ts_plan* p, Geo& g, Measure&& measure, std::string& js) {
  double best = 0;
  CKS(measure(&best));
  js += "{\"start_ms\": ";
  json_num(js, best);
  for (int cls = 0; cls < TUNE_NCLASS; ++cls) {
    js += ", \"";
    js += kTuneName[cls];
    js += "\": {\"tried\": [";
    bool first = true;
    auto log = [&](int v, int b, double t) {
      char buf[96];
      snprintf(buf, sizeof(buf), "%s[%d, %d, %.6g]", first ? "" : ", ", v, b, t);
      js += buf;
      first = false;
    };
    if (cls > 0) CKS(measure(&best));  // re-time the incumbent: clocks drift between classes
    log(g.tv[cls], g.tb[cls], best);
    const int v0 = g.tv[cls];
    int bv = v0;
    for (int v = 0; v < TUNE_NCAND; ++v) {
      if (v == v0 || !tune_valid(p, g, cls, v)) continue;
      g.tv[cls] = (signed char)v;
      const signed char keep_b = g.tb[cls];
      if (!tune_blocks(p, g, cls)) g.tb[cls] = 0;
      double t = 0;
      const int rc = measure(&t);
      g.tb[cls] = keep_b;
      if (rc != TS_OK) {
        g.tv[cls] = (signed char)bv;
        return rc;
      }
      log(v, tune_blocks(p, g, cls) ? g.tb[cls] : 0, t);
      if (t < 0.99 * best) {
        best = t;
        bv = v;
      }
    }
    g.tv[cls] = (signed char)bv;
    if (!tune_blocks(p, g, cls)) {
      g.tb[cls] = 0;
    } else {
      const int b0 = g.tb[cls];
      int bb = b0;
      for (int b = 0; b <= 4; ++b) {
        if (b == b0) continue;
        g.tb[cls] = (signed char)b;
        double t = 0;
        const int rc = measure(&t);
        if (rc != TS_OK) {
          g.tb[cls] = (signed char)bb;
          return rc;
        }
        log(bv, b, t);
        if (t < 0.99 * best) {
          best = t;
          bb = b;
        }
      }
      g.tb[cls] = (signed char)bb;
    }
    char buf[96];
    snprintf(buf, sizeof(buf), "], \"variant\": %d, \"blocks_per_sm\": %d}", g.tv[cls], g.tb[cls]);
    js += buf;
  }
  // confirm against the rule: time both settings twice, interleaved, and keep the
  // rule unless the picks are at least 1 % faster on the best of the two trials
  {
    const Geo tuned = g;
    Geo rule = g;
    for (int c = 0; c < TUNE_NCLASS; ++c) rule.tv[c] = rule.tb[c] = 0;
    double bt = 1e300, br = 1e300;
    for (int r = 0; r < 2; ++r) {
      double t = 0;
      g = tuned;
      CKS(measure(&t));
      if (t < bt) bt = t;
      g = rule;
      CKS(measure(&t));
      if (t < br) br = t;
    }
    g = bt < 0.99 * br ? tuned : rule;
    best = bt < 0.99 * br ? bt : br;
    js += ", \"confirm\": {\"tuned_ms\": ";
    json_num(js, bt);
    js += ", \"rule_ms\": ";
    json_num(js, br);
    js += bt < 0.99 * br ? ", \"kept\": \"tuned\"}" : ", \"kept\": \"rule\"}";
    char buf[160];
    snprintf(buf, sizeof(buf), ", \"final\": {\"variant\": [%d, %d, %d, %d, %d], \"blocks_per_sm\": [%d, %d, %d, %d, %d]}",
             g.tv[0], g.tv[1], g.tv[2], g.tv[3], g.tv[4], g.tb[0], g.tb[1], g.tb[2], g.tb[3], g.tb[4]);
    js += buf;
  }
  js += ", \"end_ms\": ";
  json_num(js, best);
  js += "}";
  return TS_OK;
}

void copy_report(const std::string& js, char* report, size_t len) {
  if (!report || len == 0) return;
  const size_t n = js.size() < len - 1 ? js.size() : len - 1;
  memcpy(report, js.data(), n);
  report[n] = 0;
}

void ens_invalidate(ts_ensemble* e) {
  if (e->exec) cudaGraphExecDestroy(e->exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  if (e->execK) cudaGraphExecDestroy(e->execK);
  if (e->graphK) cudaGraphDestroy(e->graphK);
  e->exec = nullptr;
  e->graph = nullptr;
  e->execK = nullptr;
  e->graphK = nullptr;
}

}  // namespace

extern "C" {

int ts_tuning_candidates(const ts_plan* p, int cls, int* mask, int* blocks) {
  if (!p || cls < 0 || cls >= TUNE_NCLASS || !mask) return TS_ERR_ARG;
  int m = 0;
  for (int v = 0; v < TUNE_NCAND; ++v)
    if (tune_valid(p, p->g, cls, v)) m |= 1 << v;
  *mask = m;
  if (blocks) *blocks = tune_blocks(p, p->g, cls) ? 1 : 0;
  return TS_OK;
}

int ts_plan_get_tuning(const ts_plan* p, ts_tuning* t) {
  if (!p || !t) return TS_ERR_ARG;
  for (int c = 0; c < TUNE_NCLASS; ++c) {
    t->variant[c] = p->g.tv[c];
    t->blocks_per_sm[c] = p->g.tb[c];
  }
  return TS_OK;
}

int ts_plan_set_tuning(ts_plan* p, const ts_tuning* t) {
  if (!p || !t) return TS_ERR_ARG;
  Geo g = p->g;
  for (int c = 0; c < TUNE_NCLASS; ++c) {
    g.tv[c] = (signed char)t->variant[c];
    if (t->variant[c] < 0 || t->variant[c] >= TUNE_NCAND || !tune_valid(p, g, c, t->variant[c])) {
      g_last_error = std::string("ts_plan_set_tuning: candidate ") + std::to_string(t->variant[c]) + " of class " +
                     kTuneName[c] + " does not exist for this plan";
      return TS_ERR_ARG;
    }
  }
  for (int c = 0; c < TUNE_NCLASS; ++c) {
    const int b = t->blocks_per_sm[c];
    if (b < 0 || b > 8 || (b > 0 && !tune_blocks(p, g, c))) {
      g_last_error = std::string("ts_plan_set_tuning: blocks_per_sm ") + std::to_string(b) + " not accepted for " +
                     kTuneName[c];
      return TS_ERR_ARG;
    }
    g.tb[c] = (signed char)b;
  }
  CK(cudaStreamSynchronize(p->st));  // launches already queued keep the old tuning
  p->g = g;
  return TS_OK;
}

int ts_plan_autotune(ts_plan* p, int reps, char* report, size_t report_len) {
  if (p && (p->cfg.basis == TS_BASIS_SSF || p->cfg.basis == TS_BASIS_SSS)) return ssf_transforms_only();
  if (!p || reps < 1) return TS_ERR_ARG;
  const bool sff = p->cfg.basis == TS_BASIS_SFF;
  const size_t bu = 3 * (size_t)p->g.S * p->cb, bt = (size_t)p->g.S * p->cb;
  void *U = nullptr, *T = nullptr;
  CK(cudaStreamSynchronize(p->st));
  if (cudaMalloc(&U, bu) != cudaSuccess || (sff && cudaMalloc(&T, bt) != cudaSuccess)) {
    if (U) cudaFree(U);
    cudaGetLastError();
    return TS_ERR_NOMEM;
  }
  const bool prof = p->prof;
  p->prof = false;
  int rc = TS_OK;
  auto fail = [&](int r) {
    p->prof = prof;
    cudaStreamSynchronize(p->st);
    cudaFree(U);
    cudaFree(T);
    return r;
  };
  // scratch state: the benchmark's k^4 exp(-2 (k/4)^2) spectrum (FFF) or a
  // temperature perturbation from rest (SFF)
  if (sff) {
    if (cudaMemsetAsync(U, 0, bu, p->st) != cudaSuccess) return fail(TS_ERR_CUDA);
    if ((rc = ts_init_temperature_perturbation(p, 1e-3, 4.0, 3, T)) != TS_OK) return fail(rc);
  } else {
    std::vector<double> E(p->nshells > 1 ? p->nshells : 2, 0.0);
    for (size_t k = 1; k < E.size(); ++k) E[k] = pow((double)k, 4) * exp(-2.0 * pow(k / 4.0, 2));
    if ((rc = ts_init_energy_spectrum(p, E.data(), (int)E.size(), 1, 0.5, U)) != TS_OK) return fail(rc);
  }
  auto step = [&]() -> int { return sff ? step_rbc(p, U, T) : step_fff(p, U); };
  double t1 = 0;
  if ((rc = time_calls(p->st, 1, 1, step, &t1)) != TS_OK) return fail(rc);
  int n = t1 > 0 ? (int)ceil(3.0 / t1) : 64;
  n = n < 1 ? 1 : (n > 64 ? 64 : n);
  auto measure = [&](double* ms) { return time_calls(p->st, n, reps, step, ms); };
  std::string js;
  rc = descend(p, p->g, measure, js);
  if (rc == TS_OK) copy_report(js, report, report_len);
  return fail(rc);
}

int ts_ensemble_get_tuning(ts_ensemble* e, int m, ts_tuning* t) {
  if (!e || m < 0 || m >= (int)e->plans.size()) return TS_ERR_ARG;
  for (const ens_group& G : e->groups)
    for (int i : G.idx)
      if (i == m) return ts_plan_get_tuning(G.gp, t);
  return TS_ERR_ARG;
}

int ts_ensemble_set_tuning(ts_ensemble* e, int m, const ts_tuning* t) {
  if (!e || m < 0 || m >= (int)e->plans.size()) return TS_ERR_ARG;
  for (ens_group& G : e->groups)
    for (int i : G.idx)
      if (i == m) {
        CK(cudaStreamSynchronize(e->origin));
        CKS(ts_plan_set_tuning(G.gp, t));
        ens_invalidate(e);
        return TS_OK;
      }
  return TS_ERR_ARG;
}

int ts_ensemble_autotune(ts_ensemble* e, int reps, char* report, size_t report_len) {
  if (!e || reps < 1) return TS_ERR_ARG;
  CK(cudaStreamSynchronize(e->origin));
  // save the members' states; tuning steps run on the group arrays
  std::vector<void*> saved;
  size_t total = 0;
  for (const ens_group& G : e->groups) total += 4 * (size_t)G.idx.size() * G.gp->g.S * G.gp->cb;
  void* save = nullptr;
  if (cudaMalloc(&save, total) != cudaSuccess) {
    cudaGetLastError();
    return TS_ERR_NOMEM;
  }
  size_t off = 0;
  for (const ens_group& G : e->groups) {
    const size_t B = G.idx.size(), S = (size_t)G.gp->g.S, cb = G.gp->cb;
    if (cudaMemcpy((char*)save + off, G.U, B * 3 * S * cb, cudaMemcpyDeviceToDevice) != cudaSuccess ||
        cudaMemcpy((char*)save + off + B * 3 * S * cb, G.T, B * S * cb, cudaMemcpyDeviceToDevice) != cudaSuccess) {
      cudaFree(save);
      return TS_ERR_CUDA;
    }
    off += 4 * B * S * cb;
  }
  auto restore = [&]() -> int {
    cudaStreamSynchronize(e->origin);
    size_t o = 0;
    int r = TS_OK;
    for (const ens_group& G : e->groups) {
      const size_t B = G.idx.size(), S = (size_t)G.gp->g.S, cb = G.gp->cb;
      if (cudaMemcpy(G.U, (char*)save + o, B * 3 * S * cb, cudaMemcpyDeviceToDevice) != cudaSuccess ||
          cudaMemcpy(G.T, (char*)save + o + B * 3 * S * cb, B * S * cb, cudaMemcpyDeviceToDevice) != cudaSuccess)
        r = TS_ERR_CUDA;
      o += 4 * B * S * cb;
    }
    cudaFree(save);
    return r;
  };
  auto step = [&]() -> int { return ts_ensemble_run(e, 1); };
  double t1 = 0;
  int rc = time_calls(e->origin, 1, 1, step, &t1);
  int n = t1 > 0 ? (int)ceil(30.0 / t1) : 16;
  n = n < 1 ? 1 : (n > 16 ? 16 : n);
  auto measure = [&](double* ms) {
    ens_invalidate(e);  // the next run re-captures the graph with the current tuning
    return time_calls(e->origin, n, reps, step, ms);
  };
  std::string js = "{\"groups\": [";
  for (size_t k = 0; k < e->groups.size() && rc == TS_OK; ++k) {
    ens_group& G = e->groups[k];
    char buf[128];
    snprintf(buf, sizeof(buf), "%s{\"N\": [%d, %d, %d], \"members\": %d, \"tuning\": ", k ? ", " : "", G.gp->g.Nx,
             G.gp->g.Ny, G.gp->g.Nz, (int)G.idx.size());
    js += buf;
    rc = descend(G.gp, G.gp->g, measure, js);
    js += "}";
  }
  js += "]";
  // the graph schedule: time kEnsSteps ensemble steps per launch both ways, keep the faster
  if (rc == TS_OK) {
    auto stepK = [&]() -> int { return ts_ensemble_run(e, kEnsSteps); };
    double ms[2] = {0, 0};
    for (int sc = 0; sc < 2 && rc == TS_OK; ++sc) {
      e->serial = sc == 1;
      ens_invalidate(e);
      rc = time_calls(e->origin, 2, reps, stepK, &ms[sc]);
    }
    e->serial = rc == TS_OK && ms[1] < ms[0];
    char buf[160];
    snprintf(buf, sizeof(buf), ", \"schedule\": \"%s\", \"parallel_ms\": %.4f, \"serial_ms\": %.4f",
             e->serial ? "serial" : "parallel", ms[0] / kEnsSteps, ms[1] / kEnsSteps);
    js += buf;
  }
  js += "}";
  ens_invalidate(e);
  const int rr = restore();
  if (rc == TS_OK) rc = rr;
  if (rc == TS_OK) copy_report(js, report, report_len);
  return rc;
}

}  // extern "C"
