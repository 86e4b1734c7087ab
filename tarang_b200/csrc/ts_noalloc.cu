// Allocation-free shell spectrum: ts_shell_spectrum_noalloc (include/tarang_b200.h).
//
// For callers that cannot allocate device memory at the point where they need
// E(k): a time-stepping driver that has already reserved almost all of the
// GPU's memory for its fields (a 1024^3 FP64 run keeps about 130 GB resident),
// or a loop that must not stall its stream, since cudaMalloc / cudaFree may
// synchronize the device.  The shell accumulators live in a file-scope
// __device__ array instead of plan scratch: this entry point calls no
// cudaMalloc, cudaFree or other allocating routine and needs no plan.
//
// The array holds, for up to TS_NOALLOC_MAX_SHELLS shells, the result (sum and
// mode count per shell) and the per-block partial sums of the shell kernel's
// kNoallocBlocks blocks: 2 x 4096 x (1 + 32) doubles, 2.06 MiB, on every GPU that
// loads the library, until the process exits.  Every call on a device shares it
// and it keeps the previous call's contents; each call overwrites every entry it
// reads before reading it (the partials of every block, then the result), so
// calls that overlap on the GPU (different streams, or different host threads)
// race and must be ordered by the caller.  The sums are added in a fixed order,
// so two calls on the same field give the same bits.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <mutex>
#include "tarang_b200.h"
#include "ts_launch.h"
#include "ts_misc.cuh"

namespace {

// blocks of the shell kernel on this path (its partial sums live in the static array)
constexpr unsigned kNoallocBlocks = 32;
static __device__ __align__(256) double g_noalloc_bins[2 * TS_NOALLOC_MAX_SHELLS * (1 + kNoallocBlocks)];

constexpr int kMaxDevices = 64;
double* g_bins_addr[kMaxDevices] = {nullptr};
std::mutex g_bins_mu;
// errors are reported as a status code plus one line on stderr (the reference
// reports errors on cout / cerr, e.g. FFF_pencil.cc:84-87)
void set_err(const char* what, cudaError_t e) {
  fprintf(stderr, "ts_shell_spectrum_noalloc: %s%s%s\n", what, e == cudaSuccess ? "" : ": ",
          e == cudaSuccess ? "" : cudaGetErrorString(e));
}

// Device address of g_noalloc_bins for the current device.  In host code the
// symbol is a host-side stand-in, so the address is looked up once per device,
// with that device current, on the first call made on it.
int bins_for_current_device(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { set_err("cudaGetDevice", e); return TS_ERR_CUDA; }
  if (dev < 0 || dev >= kMaxDevices) { set_err("device index out of range", cudaSuccess); return TS_ERR_ARG; }
  std::lock_guard<std::mutex> lk(g_bins_mu);
  if (!g_bins_addr[dev]) {
    double* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_noalloc_bins);
    if (e != cudaSuccess || !p) { set_err("cudaGetSymbolAddress(g_noalloc_bins)", e); return TS_ERR_CUDA; }
    g_bins_addr[dev] = p;
  }
  *out = g_bins_addr[dev];
  return TS_OK;
}

bool on_device(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Stepanov normalisation of the accumulated bins (universal_energy.cc:350-362, 3D)
__global__ void k_shell_finish(const double* __restrict__ bins, int nsh, double kfp, double* Ek, int n_shells) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_shells; i += gridDim.x * blockDim.x) {
    double v = 0.0;
    if (i < nsh) {
      const double cnt = bins[nsh + i];
      v = cnt <= 0 ? 0.0 : bins[i] * (4.0 * 3.14159265358979323846) / (cnt * kfp);
    }
    Ek[i] = v;
  }
}

template <typename T>
int run(const ts::Geo& g, const void* a, int ncomp, int kmax, double* bins, double* Ek, int n_shells, double kfp,
        cudaStream_t st) {
  const int nsh = kmax + 1;
  // the shell kernel writes every block's partial bins, then the fixed-order sum
  // writes bins[0, 2 nsh): nothing is read before this call has written it
  cudaError_t e = ts::Launch<T>::shell(g, a, ncomp, nsh, bins, st, nullptr, kNoallocBlocks);
  if (e != cudaSuccess) { set_err("shell kernel launch", e); return TS_ERR_CUDA; }
  k_shell_finish<<<(n_shells + 255) / 256, 256, 0, st>>>(bins, nsh, kfp, Ek, n_shells);
  ++ts::g_launches;
  e = cudaGetLastError();
  if (e != cudaSuccess) { set_err("kernel launch", e); return TS_ERR_CUDA; }
  return TS_OK;
}

}  // namespace

extern "C" int ts_shell_spectrum_noalloc(int basis, int precision, const int N[3], const double kfactor[3],
                                         const void* a_hat, int ncomp, double* Ek, int n_shells, void* stream) {
  if (!N || !kfactor || !a_hat || !Ek || ncomp < 1 || ncomp > 3 || n_shells < 1) return TS_ERR_ARG;
  if ((basis != TS_BASIS_FFF && basis != TS_BASIS_SFF) || (precision != TS_F64 && precision != TS_F32))
    return TS_ERR_ARG;
  for (int i = 0; i < 3; ++i)
    if (!ts::size_supported(N[i]) || !(kfactor[i] > 0)) return TS_ERR_ARG;
  if (!on_device(a_hat) || !on_device(Ek)) {
    set_err("a_hat and Ek must be device pointers", cudaSuccess);
    return TS_ERR_ARG;
  }
  ts::Geo g;
  g.Nx = N[0]; g.Ny = N[1]; g.Nz = N[2];
  g.Hz = g.Nz / 2 + 1;
  g.S = (long long)g.Nx * g.Ny * g.Hz;
  for (int i = 0; i < 3; ++i) g.kf[i] = kfactor[i];
  g.basis = basis;
  g.dealias = 0;
  // Min_radius_outside (FFF_pencil_inline.h:497-504, SFF_pencil_inline.h:423-430)
  const double ex = (basis == TS_BASIS_FFF ? (g.Nx / 2) : (g.Nx - 1)) * g.kf[0];
  const int kmax = (int)ceil(sqrt(ex * ex + pow((g.Ny / 2) * g.kf[1], 2) + pow((g.Nz / 2) * g.kf[2], 2)));
  if (kmax + 1 > TS_NOALLOC_MAX_SHELLS) {
    fprintf(stderr, "ts_shell_spectrum_noalloc: %d shells exceed the static limit TS_NOALLOC_MAX_SHELLS = %d\n",
            kmax + 1, TS_NOALLOC_MAX_SHELLS);
    return TS_ERR_ARG;
  }
  double* bins = nullptr;
  int rc = bins_for_current_device(&bins);
  if (rc != TS_OK) return rc;
  const double kfp = g.kf[0] * g.kf[1] * g.kf[2];
  cudaStream_t st = (cudaStream_t)stream;
  return precision == TS_F32 ? run<float>(g, a_hat, ncomp, kmax, bins, Ek, n_shells, kfp, st)
                             : run<double>(g, a_hat, ncomp, kmax, bins, Ek, n_shells, kfp, st);
}
