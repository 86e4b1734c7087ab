// Host-side launchers of the templated kernels, instantiated per precision in
// ts_kern_f32.cu / ts_kern_f64.cu (compiled in parallel).
#pragma once
#include <cuda_runtime.h>
#include "ts_fff.cuh"
#include "ts_sff.cuh"

namespace ts {

extern long long g_launches;  // kernels launched by this library
constexpr unsigned SHELL_MAX_BLOCKS = 4 * 148;  // blocks of the plan's shell-sum kernel
// blocks of k_shell for a geometry and a cap (the sums' rounding depends on it, so a
// geometry and cap always give the same blocks)
inline unsigned shell_blocks(const Geo& g, unsigned cap) {
  const long long lines = (long long)g.Nx * g.Ny;
  const long long b = (lines + SHELL_WARPS - 1) / SHELL_WARPS;
  return (unsigned)(b < (long long)cap ? b : (long long)cap);
}

template <typename T> struct Launch {
  // strided-axis FFT on nf fields in place: axis 0 = x (L = Nx), 1 = y (L = Ny);
  // dir -1 forward, +1 inverse; outputs scaled by `scale`
  // per > 0: the nf fields are nf / per members of per fields each, members mstride complex apart
  // inner_eff > 0: transform only the first inner_eff columns (y axis: kz < inner_eff);
  // zero_hi: rows with 3|k| > L are zero and not read (two-thirds dealiased input)
  static cudaError_t strided(const Geo& g, int axis, int dir, void* data, int nf, const void* tw, cudaStream_t st,
                             int per = 0, long long mstride = 0, int inner_eff = 0, int zero_hi = 0);
  // form 0 conservative (3 fields out), 1 rotational (6), 3 adjoint of the rotational form (9: also
  // lsc c^-1 P lam from the cotangent lam)
  // kept != 0 (forms 0, 1 with two-thirds dealiasing): write only the columns with 3|ky| <= Ny, 3 kz <= Nz
  // form 5: u and the giver u inside |K| <= rad (6 fields) for the per-sphere energy flux
  static cudaError_t inv_x(const Geo& g, int form, const void* U, void* W, const void* tw, const void* lam,
                           double lsc, cudaStream_t st, int kept = 0, double rad = 0.0);
  // form 0 conservative, 1 rotational, 2 Boussinesq (u, T), 3 adjoint of the rotational form,
  // 5 MHD (Elsasser products), 6 flux giver (u_i g_j)
  // nmem members, member fields msP complex apart
  // zkeep >= 0: input rows kz > zkeep are zero and not read
  static cudaError_t z_fused(const Geo& g, int form, void* P, const void* tw, int* err, cudaStream_t st,
                             int nmem = 1, long long msP = 0, int zkeep = -1);
  static cudaError_t z_single(const Geo& g, int dir, const void* in, void* out, int ncomp, const void* tw, cudaStream_t st);
  // SSS: the fused z pass on real coefficients (form 0 / 2 products; zin / zout sine masks)
  static cudaError_t sss_z_fused(const Geo& g, int form, void* P, const void* tw, const void* tq, int zin, int zout,
                                 cudaStream_t st);
  // a.U0 / a.Ud / a.tot must be 16-byte aligned (TMA)
  // form 0 / 1 / 3 as inv_x; mode MODE_STEP, MODE_FLUX, MODE_NLIN (forms 0, 1) or MODE_ADJ (form 3)
  static cudaError_t fwd_x(const Geo& g, int form, int mode, const void* P, const StageArgs& a, const void* tw,
                           cudaStream_t st);
  // SFF x passes (sin/cos along x): inverse of u1,u2,u3,T into P[0..3]; forward of the nine
  // Boussinesq products + force, projection and the IF-RK4 stage update
  // nmem members: member strides (complex elements) of U, Tf, W; SffArgs carries its own
  static cudaError_t sff_inv_x(const Geo& g, const void* U, const void* Tf, void* W, const void* tq, cudaStream_t st,
                               int nmem = 1, long long msU = 0, long long msT = 0, long long msW = 0);
  static cudaError_t sff_fwd_x(const Geo& g, const void* P, const SffArgs& a, const void* tq, cudaStream_t st,
                               int nmem = 1);
  // standalone sin/cos x transform of ncomp components in place (dir -1 forward with scale scl, +1 inverse);
  // nbatch > 1 repeats it on the fields at A + b * bstride (complex elements), field b with parity bit b of sine
  static cudaError_t sff_x(const Geo& g, int dir, void* A, int ncomp, int sine, double scl, const void* tq,
                           cudaStream_t st, int nbatch = 1, long long bstride = 0);
  // FFF passive scalar: elementwise epilogue of the nine x-transformed products in P
  static cudaError_t scalar_epi(const Geo& g, const void* P, const SffArgs& a, cudaStream_t st);
  // SSS z sin/cos helpers on nlines lines of N reals (padded to N + 2)
  static cudaError_t sss_zperm_fwd(const void* u, void* v, long long nlines, int N, int sine, cudaStream_t st);
  static cudaError_t sss_zpost_fwd(const void* Z, void* c, long long nlines, int N, int sine, double scl,
                                   const void* tq, cudaStream_t st);
  static cudaError_t sss_zpre_inv(const void* c, void* Vout, long long nlines, int N, int sine, const void* tq,
                                  cudaStream_t st);
  static cudaError_t sss_zperm_inv(const void* v, void* u, long long nlines, int N, int sine, cudaStream_t st);
  // SSS fluid step: dealiased copy of real coefficients, and the epilogue
  static cudaError_t sss_dealias_copy(const Geo& g, const void* A, void* B, int ncomp, cudaStream_t st);
  static cudaError_t sss_epi(const Geo& g, const void* P, const StageArgs& a, cudaStream_t st);
  // SSF fluid step: elementwise epilogue of the six forward-transformed products in P
  static cudaError_t ssf_epi(const Geo& g, const void* P, const StageArgs& a, cudaStream_t st);
  // SSF / SSS Boussinesq step: epilogues of the nine forward-transformed products in P
  static cudaError_t ssf_rbc_epi(const Geo& g, const void* P, const SffArgs& a, cudaStream_t st);
  static cudaError_t sss_rbc_epi(const Geo& g, const void* P, const SffArgs& a, cudaStream_t st);
  // FFF MHD: elementwise epilogue of the nine x-transformed Elsasser products in P
  static cudaError_t mhd_epi(const Geo& g, const void* P, const SffArgs& a, cudaStream_t st);
  static cudaError_t reality(const Geo& g, void* A, int ncomp, cudaStream_t st);
  static cudaError_t rbc_slave(const Geo& g, void* U, void* Tf, int slave, double vs, cudaStream_t st);
  static cudaError_t reality_adj(const Geo& g, void* A, int ncomp, cudaStream_t st);
  static cudaError_t carati(const Geo& g, const void* U, void* fc, int km, double rin, double rout, const double* es,
                            const double* hs, const double* mis, int nsup, cudaStream_t st);
  static cudaError_t energy(const Geo& g, const void* A, const void* B, int ncomp, double* out, cudaStream_t st);
  static cudaError_t maxdiv(const Geo& g, const void* U, unsigned long long* out, cudaStream_t st);
  // shell sums of the shells s = ceil|K| < nbins into bins[0, nbins) and the counts into bins[nbins, 2 nbins);
  // B != nullptr: cross spectrum Re(A . conj(B)).  bins must hold 2 nbins (1 + shell_blocks(g, cap))
  // doubles (the per-block partials follow the result); the sums are reproducible bit for bit
  static cudaError_t shell(const Geo& g, const void* A, int ncomp, int nbins, double* bins, cudaStream_t st,
                           const void* B = nullptr, unsigned cap = SHELL_MAX_BLOCKS);
  // per-sphere energy flux: out[0] = sum over |K| > R of 2 mult Re(N . conj(D U)), N from the
  // nine x-forward-transformed giver products in P; out must hold 1 + 148 * 16 doubles
  static cudaError_t ssf_giver(const Geo& g, const void* U, void* P, double R, cudaStream_t st);
  static cudaError_t ssf_flux_outside(const Geo& g, const void* P, const void* U, double R, int qx, int qy,
                                      double* out, cudaStream_t st);
  static cudaError_t flux_outside(const Geo& g, const void* P, const void* U, double R, double* out,
                                  cudaStream_t st);
  // the same on SSS (real coefficients, sine letters along x, y and z)
  static cudaError_t sss_giver(const Geo& g, const void* U, void* P, double R, cudaStream_t st);
  static cudaError_t sss_flux_outside(const Geo& g, const void* P, const void* U, double R, int qx, int qy, int qz,
                                      double* out, cudaStream_t st);
  static cudaError_t force_scatter(const Geo& g, const void* fc, void* F, int km, cudaStream_t st);
  static cudaError_t init_ic(const Geo& g, void* U, const double* Eic, const double* mis, int nsh,
                             unsigned long long key, cudaStream_t st);
  static cudaError_t scale(void* A, long long n, double s, cudaStream_t st);
  static cudaError_t init_temp(const Geo& g, void* A, double amp, double kmax, unsigned long long key, cudaStream_t st);
  static cudaError_t dealias_copy(const Geo& g, const void* A, void* B, int ncomp, cudaStream_t st);
  // one block whose bounded wait gives up after `polls` polls (test of the timeout path)
  static cudaError_t expire_wait(int* err, int polls, cudaStream_t st);
  // launch tuning (Geo::tv, Geo::tb): whether kernel candidate v (0 = the rule) of pass class
  // cls exists for this geometry and product form (form as z_fused; the basis selects the
  // SFF x kernels), and whether the class takes a blocks-per-SM count (persistent launches)
  static bool tune_valid(const Geo& g, int form, int cls, int v);
  static bool tune_blocks(const Geo& g, int form, int cls);
};

bool size_supported(int n);

}  // namespace ts
