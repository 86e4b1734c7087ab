// Launcher definitions, included once per precision by ts_kern_f32.cu and
// ts_kern_f64.cu with TS_REAL defined to float / double.
#include <type_traits>
#include "ts_launch.h"
#include "ts_misc.cuh"

namespace ts {

namespace {

typedef TS_REAL T;
typedef C<T> V;

// elements per thread of the register FFTs; columns per block (rows of 128 B)
constexpr int E_REG = std::is_same<T, float>::value ? 16 : 8;
// at L = 1024 the 16-element register FFT would spill under the 512-thread cap
constexpr int e_reg(int L) { return (L >= 1024 ? 8 : E_REG) < L ? (L >= 1024 ? 8 : E_REG) : L; }
// forward-x kernel: 4 elements per thread (3 accumulators each); on B200 at 256^3
// the 512-thread blocks beat the 8-element, 256-thread form by 6 % in FP32 (3.03
// vs 3.09 ms per step) and 2.5 % in FP64 (6.78 vs 6.96 ms)
constexpr int E_ACC = 4;
constexpr int E_ACC_ALT = 8;
constexpr int CWMAX = std::is_same<T, float>::value ? 16 : 8;
constexpr int emin(int a, int b) { return a < b ? a : b; }
constexpr int cw_for(int L, int E) {
  return emin(CWMAX, (512 * E / L) > 0 ? (512 * E / L) : 1);
}
// 8-byte units per complex (TMA boxes are expressed in 8-byte words)
constexpr int UNITS = (int)sizeof(V) / 8;
// column tile width of the TMA x-pass kernels: 64-byte rows, and at least two
// 8-byte units so every tile start is 16-byte aligned
// (the epilogue kernel's 8 tiles + padded exchange tile must fit in 220 KB)
constexpr int xcw_fit(int L, int cw) {
  return (cw > (std::is_same<T, float>::value ? 2 : 1) &&
          (size_t)9 * L * cw * sizeof(V) + (size_t)L * sizeof(V) > 220 * 1024)
             ? xcw_fit(L, cw / 2) : cw;
}
constexpr int xcw(int L) { return xcw_fit(L, std::is_same<T, float>::value ? 8 : 4); }

template <typename Fn> bool dispatch_L(int L, Fn&& fn) {
  switch (L) {
    case 16: fn(std::integral_constant<int, 16>{}); return true;
    case 32: fn(std::integral_constant<int, 32>{}); return true;
    case 64: fn(std::integral_constant<int, 64>{}); return true;
    case 128: fn(std::integral_constant<int, 128>{}); return true;
    case 256: fn(std::integral_constant<int, 256>{}); return true;
    case 512: fn(std::integral_constant<int, 512>{}); return true;
    case 1024: fn(std::integral_constant<int, 1024>{}); return true;
  }
  return false;
}

// SFF launchers also take the non-power-of-two sizes 48 and 96: their FFT
// lengths 3 * 2^k run with 12 elements per thread (radices 4, 2, 3)
template <typename Fn> bool dispatch_L_sff(int L, Fn&& fn) {
  if (dispatch_L(L, fn)) return true;
  {
    switch (L) {
      case 48: fn(std::integral_constant<int, 48>{}); return true;
      case 96: fn(std::integral_constant<int, 96>{}); return true;
    }
  }
  return false;
}
// elements per thread for a length that may carry a factor 3
// (6 where the power-of-two choice is 4 or less: the FP64 SFF forward x kernel
// holds four accumulators per element and spilled at 12)
constexpr int e_mixed(int L, int e_pow2) { return L % 3 == 0 ? (e_pow2 >= 8 ? 12 : 6) : (e_pow2 < L ? e_pow2 : L); }

template <typename K> cudaError_t smem_attr(K kernel, size_t bytes) {
  if (bytes > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) cudaGetLastError();  // do not leave the error for a later launch to report
    return e;
  }
  return cudaSuccess;
}

inline unsigned grid1d(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (unsigned)b;
}

// lines per block of the z kernels: about 96 KB of shared memory (two blocks per SM)
inline int z_lines(int nbuf, int H) {
  const long long per = 2LL * nbuf * H * (long long)sizeof(V);
  long long nl = (96 * 1024) / per;
  if (nl < 1) nl = 1;
  if (nl > 16) nl = 16;
  return (int)nl;
}

}  // namespace

// strided passes at L = 1024 in FP32: 16 elements per thread and 8-column tiles
// (64-byte rows) with the exchange in the consumed staging tile; on B200 this
// moved the x pass from 1.2 to 2.35 TB/s and the y pass from 2.0 to 2.9 TB/s
// against 4-column tiles
constexpr bool wide1024(int L) { return std::is_same<T, float>::value && L == 1024; }
constexpr int str_e(int L) { return wide1024(L) ? 16 : e_mixed(L, e_reg(L)); }
constexpr int str_cw(int L) { return wide1024(L) ? 8 : cw_for(L, str_e(L)); }
constexpr int str_nt(int L) { return wide1024(L) ? 2 : 3; }

// ---------------------------------------------------------------------------
// Launch-tuning candidates.  Candidate 0 of every pass class is the fixed rule;
// the others change the radix schedule (elements per thread E: the Stockham
// passes use radix min(E, remaining)), the column-tile width CW or the number of
// staging tiles NT.  A candidate that does not fit (threads per block, shared
// memory) or repeats an earlier one is invalid and launches as the rule.
// ---------------------------------------------------------------------------
constexpr int NCAND = TUNE_NCAND;
struct Tile { int E, CW, NT; };
constexpr bool tile_eq(Tile a, Tile b) { return a.E == b.E && a.CW == b.CW && a.NT == b.NT; }
constexpr bool tile_fits(int L, Tile c, int tiles) {
  return c.E > 0 && c.CW > 0 && L % c.E == 0 && c.CW * (L / c.E) <= 1024 && c.CW * (L / c.E) >= 32 &&
         (size_t)tiles * L * c.CW * sizeof(V) <= 227 * 1024;
}

// strided passes (y inverse / y forward)
constexpr Tile str_cand(int L, int v) {
  return v == 0 ? Tile{str_e(L), str_cw(L), str_nt(L)}
       : v == 1 ? (L % 3 != 0 && str_e(L) > 4 ? Tile{str_e(L) / 2, str_cw(L), str_nt(L)} : Tile{0, 0, 0})
       : v == 2 ? (str_cw(L) > 1 ? Tile{str_e(L), str_cw(L) / 2, str_nt(L)} : Tile{0, 0, 0})
       : v == 3 ? Tile{str_e(L), str_cw(L), 5 - str_nt(L)}
       : v == 4 ? Tile{str_e(L), str_cw(L), 4}
       : v == 5 ? (wide1024(L) ? Tile{32, 8, 1} : Tile{0, 0, 0})
       : v == 6 ? (wide1024(L) ? Tile{32, 16, 1} : Tile{0, 0, 0})
                : Tile{0, 0, 0};
}
constexpr bool str_valid(int L, int v) {
  return v == 0 || (v == 6 && wide1024(L) && tile_fits(L, str_cand(L, 6), 1)) || (v < NCAND && tile_fits(L, str_cand(L, v), str_tiles(str_cand(L, v).NT)) &&
                    !tile_eq(str_cand(L, v), str_cand(L, 0)) && (v < 2 || !tile_eq(str_cand(L, v), str_cand(L, 1))) &&
                    (v < 3 || !tile_eq(str_cand(L, v), str_cand(L, 2))) &&
                    (v < 4 || !tile_eq(str_cand(L, v), str_cand(L, 3))) &&
                    (v < 5 || !tile_eq(str_cand(L, v), str_cand(L, 4))));
}

template <int L, int VV, typename Fn> void with_str_tile(Fn&& fn) {
  if constexpr (str_valid(L, VV)) fn(std::integral_constant<int, VV>{});
  else fn(std::integral_constant<int, 0>{});
}

template <> cudaError_t Launch<T>::strided(const Geo& g, int axis, int dir, void* data, int nf, const void* tw,
                                           cudaStream_t st, int per, long long mstride, int inner_eff,
                                           int zero_hi) {
  if (per <= 0) per = nf;
  cudaError_t err = cudaErrorInvalidValue;
  const int L = axis == 0 ? g.Nx : g.Ny;
  if (L == 1) return cudaSuccess;  // a one-point transform is the identity (two-dimensional runs)
  // the y passes follow the tuning of their class; x passes keep the rule
  const int cls = axis == 1 ? (dir > 0 ? TUNE_Y_INV : TUNE_Y_FWD) : -1;
  const int v = cls >= 0 ? g.tv[cls] : 0, bps = cls >= 0 ? g.tb[cls] : 0;
  dispatch_L_sff(L, [&](auto Lc) {
    constexpr int LL = decltype(Lc)::value;
    auto run = [&](auto vc) {
      constexpr Tile c = str_cand(LL, decltype(vc)::value);
      constexpr int E = c.E, CW = c.CW, NT = c.NT;
      const int inner = inner_eff > 0 ? inner_eff : (axis == 0 ? g.Ny * g.Hz : g.Hz);
      const long long rstride = axis == 0 ? (long long)g.Ny * g.Hz : g.Hz;
      const long long ostride = axis == 0 ? 0 : (long long)g.Ny * g.Hz;
      const int nouter = axis == 0 ? 1 : g.Nx;
      const long long nwork = (long long)nf * ((inner + CW - 1) / CW) * nouter;
      const size_t sm = (size_t)str_tiles(NT) * LL * CW * sizeof(V);
      // persistent grid: as many blocks as fit on the 148 SMs at once (or the tuned count)
      const int cap = (CW * (LL / E)) <= 256 ? 2 : 1;
      const int fit = (int)((227 * 1024) / sm);
      const int per_sm = bps > 0 ? bps : (fit < cap ? fit : cap);
      long long blocks = 148LL * (per_sm > 0 ? per_sm : 1);
      if (blocks > nwork) blocks = nwork;
      auto launch = [&](auto k) {
        if ((err = smem_attr(k, sm)) != cudaSuccess) return;
        k<<<(unsigned)blocks, CW * (LL / E), sm, st>>>((V*)data, nf, g.S, inner, rstride, ostride, nouter,
                                                      (const V*)tw, per, mstride, zero_hi);
        ++g_launches;
        err = cudaGetLastError();
      };
      if (dir < 0) launch(k_strided_fft<T, LL, E, CW, -1, NT>);
      else launch(k_strided_fft<T, LL, E, CW, 1, NT>);
    };
    // the y passes of 1024 points in FP32: the one-tile, 32-element form on 16-column
    // tiles (tile 6) is the rule (on B200 at 1024^3: y inverse 9.9 ms against 10.4 for the
    // two-tile, 16-element form on 8 columns; y forward 7.5 against 7.6 for 32 elements on
    // 8 columns and 8.9 for the 16-element form); for the y forward pass candidate 5 is
    // then the 16-element form
    int vv = (wide1024(LL) && axis == 1) ? (v == 0 ? 6 : ((dir < 0 && v == 5) ? 0 : v)) : v;
    // the x forward pass of 1024 points in FP32 (the split form's FFT): 16-column tiles,
    // 128-byte row segments, 32 elements per thread, one staging tile (tile 6, not a tuning
    // candidate).  An x row is Ny*Hz complex long (4.2 MB at 1024^3), so every row of a
    // tile is a separate memory page; twice the bytes per row visit took the forward x
    // FFT + epilogue from 20.4 to 17.0 ms per right-hand side at 1024^3 on B200
    if (wide1024(LL) && axis == 0 && dir < 0) vv = 6;
    switch (vv) {
      case 6: with_str_tile<LL, 6>(run); break;
      case 1: with_str_tile<LL, 1>(run); break;
      case 2: with_str_tile<LL, 2>(run); break;
      case 3: with_str_tile<LL, 3>(run); break;
      case 4: with_str_tile<LL, 4>(run); break;
      case 5: with_str_tile<LL, 5>(run); break;
      default: run(std::integral_constant<int, 0>{});
    }
  });
  return err;
}

// inverse x pass (FFF forms 0, 1): 8 elements per thread in FP32 (U held in
// registers across the output fields; 16 at L = 1024 with per-field loads)
constexpr int ix_e(int L) { return wide1024(L) ? 16 : (std::is_same<T, float>::value ? (8 < L ? 8 : L) : e_reg(L)); }
constexpr int ix_cw(int L) { return wide1024(L) ? 8 : cw_for(L, ix_e(L)); }
constexpr int ix_e_alt(int L) {
  return std::is_same<T, float>::value ? (ix_e(L) == 8 ? (16 <= L ? 16 : 0) : 8) : (ix_e(L) > 4 ? ix_e(L) / 2 : 0);
}
// candidate 3 (FP32): the persistent prefetching kernel k_inv_x_pf, 8 elements per thread
// (the three components of U held in registers), staging + exchange tiles (NT = 4 tiles);
// candidate 4 (FP32, 1024-point lines): 32 elements per thread over 8-column tiles
// (256-thread blocks, two per SM; radix 32 x 32, one exchange per field);
// candidate 5 (FP32, 1024-point lines, two-thirds dealiasing): k_inv_x_st, the tile's
// kept U rows staged in shared memory in one cp.async group (the rule elsewhere)
constexpr Tile ix_cand(int L, int v) {
  return v == 0 ? Tile{ix_e(L), ix_cw(L), 1}
       : v == 1 ? (ix_e_alt(L) > 0 ? Tile{ix_e_alt(L), cw_for(L, ix_e_alt(L)), 1} : Tile{0, 0, 0})
       : v == 2 ? (ix_cw(L) > 1 ? Tile{ix_e(L), ix_cw(L) / 2, 1} : Tile{0, 0, 0})
       : v == 3 ? (std::is_same<T, float>::value ? Tile{8, cw_for(L, 8), 4} : Tile{0, 0, 0})
       : v == 4 ? (wide1024(L) ? Tile{32, 8, 1} : Tile{0, 0, 0})
       : v == 5 ? (wide1024(L) ? Tile{16, 8, 2} : Tile{0, 0, 0})
                : Tile{0, 0, 0};
}
constexpr bool ix_valid(int L, int v) {
  return v == 0 || (v < NCAND && tile_fits(L, ix_cand(L, v), ix_cand(L, v).NT == 4 ? 4 : 1) &&
                    !tile_eq(ix_cand(L, v), ix_cand(L, 0)) && (v < 2 || !tile_eq(ix_cand(L, v), ix_cand(L, 1))) &&
                    (v < 3 || !tile_eq(ix_cand(L, v), ix_cand(L, 2))) &&
                    (v < 4 || !tile_eq(ix_cand(L, v), ix_cand(L, 3))) &&
                    (v < 5 || !tile_eq(ix_cand(L, v), ix_cand(L, 4))));
}

template <> cudaError_t Launch<T>::inv_x(const Geo& g, int form, const void* U, void* W, const void* tw,
                                         const void* lam, double lsc, cudaStream_t st, int kept, double rad) {
  cudaError_t err_ = cudaErrorInvalidValue;
  // forms 0 and 1 follow the tuning; the adjoint forms keep the rule
  const int v = form <= 1 ? g.tv[TUNE_X_INV] : 0;
  dispatch_L(g.Nx, [&](auto Lc) {
    constexpr int LL = decltype(Lc)::value;
    // 1024 points in FP32 under two-thirds dealiasing: the staged kernel k_inv_x_st is the
    // rule (on B200 7.0 against 10.1 ms per launch at 1024^3) and candidate 5 is then the
    // direct-load kernel
    const int vv = (ix_valid(LL, 5) && kept && form <= 1) ? (v == 0 ? 5 : (v == 5 ? 0 : v)) : v;
    if constexpr (ix_valid(LL, 5)) {
      if (vv == 5 && kept) {
        // the kept U rows of a tile staged in shared memory (one load latency per tile)
        constexpr Tile c = ix_cand(LL, 5);
        constexpr int E = c.E, CW = c.CW;
        const size_t sm = ((size_t)LL + 3 * ix_kept_rows<LL>()) * CW * sizeof(V);
        const int nzk = g.Nz / 3 + 1;
        const unsigned blocks = (unsigned)((2 * (g.Ny / 3) + 1) * ((nzk + CW - 1) / CW));
        auto run = [&](auto kern) {
          if ((err_ = smem_attr(kern, sm)) != cudaSuccess) return;
          kern<<<blocks, CW * (LL / E), sm, st>>>((const V*)U, (V*)W, g, (const V*)tw);
          ++g_launches;
          err_ = cudaGetLastError();
        };
        if (form == 0) { run(k_inv_x_st<T, LL, E, CW, 0>); return; }
        if (form == 1) { run(k_inv_x_st<T, LL, E, CW, 1>); return; }
      }
    }
    if constexpr (ix_valid(LL, 3)) {
      if (vv == 3) {
        // persistent, prefetching form: one block per SM
        constexpr Tile c = ix_cand(LL, 3);
        constexpr int E = c.E, CW = c.CW;
        const size_t sm = 4ull * LL * CW * sizeof(V);
        const int nzk = g.Nz / 3 + 1;
        const long long ntiles = kept ? (long long)(2 * (g.Ny / 3) + 1) * ((nzk + CW - 1) / CW)
                                      : (long long)((g.Ny * g.Hz + CW - 1) / CW);
        const unsigned blocks = (unsigned)(ntiles < 148 ? ntiles : 148);
        auto run = [&](auto kern) {
          if ((err_ = smem_attr(kern, sm)) != cudaSuccess) return;
          kern<<<blocks, CW * (LL / E), sm, st>>>((const V*)U, (V*)W, g, (const V*)tw, kept);
          ++g_launches;
          err_ = cudaGetLastError();
        };
        if (form == 0) run(k_inv_x_pf<T, LL, E, CW, 0>);
        else if (form == 1) run(k_inv_x_pf<T, LL, E, CW, 1>);
        return;
      }
    }
    // the direct-load kernel measured faster than the TMA-staged k_inv_x on B200
    // (0.19 vs 0.28 ms at 256^3 FP32, rotational); k_inv_x stays available
    auto tile = [&](auto vc) {
      constexpr Tile c = ix_cand(LL, decltype(vc)::value);
      constexpr int E = c.E, CW = c.CW;
      const int inner = g.Ny * g.Hz;
      const size_t sm = (size_t)LL * CW * sizeof(V);
      const int nzk = g.Nz / 3 + 1;
      const unsigned blocks = kept ? (unsigned)((2 * (g.Ny / 3) + 1) * ((nzk + CW - 1) / CW))
                                   : (unsigned)((inner + CW - 1) / CW);
      auto run = [&](auto kern) {
        if ((err_ = smem_attr(kern, sm)) != cudaSuccess) return;
        kern<<<blocks, CW * (LL / E), sm, st>>>((const V*)U, (V*)W, g, (const V*)tw, (const V*)lam, (T)lsc, kept,
                                                 rad);
        ++g_launches;
        err_ = cudaGetLastError();
      };
      if (form == 0) run(k_inv_x_ld<T, LL, E, CW, 0>);
      else if (form == 1) run(k_inv_x_ld<T, LL, E, CW, 1>);
      else if constexpr (decltype(vc)::value == 0) {
        if (form == 3) run(k_inv_x_ld<T, LL, E, CW, 3>);
        else if (form == 4) run(k_inv_x_ld<T, LL, E, CW, 4>);
        else if (form == 5) run(k_inv_x_ld<T, LL, E, CW, 5>);
      }
    };
    if (vv == 1 && ix_valid(LL, 1)) {
      if constexpr (ix_valid(LL, 1)) tile(std::integral_constant<int, 1>{});
    } else if (vv == 2 && ix_valid(LL, 2)) {
      if constexpr (ix_valid(LL, 2)) tile(std::integral_constant<int, 2>{});
    } else if (vv == 4 && ix_valid(LL, 4)) {
      if constexpr (ix_valid(LL, 4)) tile(std::integral_constant<int, 4>{});
    } else {
      tile(std::integral_constant<int, 0>{});
    }
  });
  return err_;
}

// shared-memory slot variant of the z pass: E elements per thread, nl lines per
// block within about 106 KB of shared memory
template <int NZ, int FORM, int E>
static cudaError_t z_slots(const Geo& g, void* P, const void* tw, cudaStream_t st, int nmem, long long msP,
                           int zkeep) {
  constexpr int M = NZ / 2;
  constexpr int TPL = M / E;
  constexpr int NIN = z_nin(FORM), NOUT = z_nout(FORM);
  constexpr int NSL = NIN > NOUT ? NIN : NOUT;
  const long long nlines = (long long)g.Nx * g.Ny;
  int nl = 256 / TPL;
  while (nl > 1 && (size_t)NSL * nl * zslot<M>() * sizeof(V) > 106 * 1024) nl /= 2;
  const size_t sm = (size_t)NSL * nl * zslot<M>() * sizeof(V);
  cudaError_t err;
  auto k = k_z_fused<T, NZ, E, FORM>;
  if ((err = smem_attr(k, sm)) != cudaSuccess) return err;
  k<<<dim3((unsigned)((nlines + nl - 1) / nl), nmem), nl * TPL, sm, st>>>((V*)P, g, (const V*)tw, nl, msP, zkeep);
  ++g_launches;
  return cudaGetLastError();
}

// z candidates (forms 0, 1, 2): 1 = the slot kernel with 8 elements per thread
// (12 with a factor 3), 2 = the slot kernel with 4 (power-of-two lines), 3 = the
// FP32 register kernel with 4 elements per thread (lines of up to 256 points),
// 4 = on 1024-point lines in FP32, the register kernel that loads each component just
// before its transform (the rule there issues every load up front)
template <int NZ, int FORM> constexpr bool z_rule_slots() {
  constexpr int M = NZ / 2;
  return !(std::is_same<T, float>::value && M <= 512) &&
         !(!std::is_same<T, float>::value && FORM <= 2 && M % 3 != 0 && M / ztma_e<T>() <= 32);
}
template <int NZ, int FORM> constexpr bool z_valid(int v) {
  constexpr int M = NZ / 2;
  return v == 0 || (FORM <= 2 && ((v == 1 && !z_rule_slots<NZ, FORM>()) ||
                                  (v == 2 && M % 3 != 0 && M >= 8 && M / 4 <= 256) ||
                                  (v == 3 && std::is_same<T, float>::value && M % 3 != 0 && M >= 8 && M / 4 <= 64) ||
                                  (v == 4 && std::is_same<T, float>::value && M == 512)));
}

template <int NZ, int FORM>
static cudaError_t z_fused_impl(const Geo& g, void* P, const void* tw, int* zerr, cudaStream_t st, int nmem,
                                long long msP, int zkeep, int v) {
  constexpr int M = NZ / 2;
  if (zkeep < 0) zkeep = M;
  constexpr int NIN = z_nin(FORM);
  const long long nlines = (long long)g.Nx * g.Ny;
  cudaError_t err;
  if constexpr (z_valid<NZ, FORM>(1)) {
    if (v == 1) return z_slots<NZ, FORM, e_mixed(M, 8)>(g, P, tw, st, nmem, msP, zkeep);
  }
  if constexpr (z_valid<NZ, FORM>(2)) {
    if (v == 2) return z_slots<NZ, FORM, 4>(g, P, tw, st, nmem, msP, zkeep);
  }
  if constexpr (z_valid<NZ, FORM>(4)) {
    // 1024-point z lines in FP32: the register kernel with every component's loads issued
    // up front is the rule (on B200 13.0 against 15.8 ms per launch at 1024^3); candidate 4
    // loads each component just before its transform
    constexpr int NT = zreg_threads<FORM>(), LPB = NT / (M / 8);
    const dim3 grid((unsigned)((nlines + LPB - 1) / LPB), nmem);
    if (v == 4) k_z_reg<T, NZ, FORM, 0, false><<<grid, NT, 0, st>>>((V*)P, g, (const V*)tw, msP, zkeep);
    else if (v == 0) k_z_reg<T, NZ, FORM, 0, true><<<grid, NT, 0, st>>>((V*)P, g, (const V*)tw, msP, zkeep);
    if (v == 4 || v == 0) {
      ++g_launches;
      return cudaGetLastError();
    }
  }
  if constexpr (z_valid<NZ, FORM>(3)) {
    if (v == 3) {
      constexpr int NT = zreg_threads<FORM>(), LPB = NT / (M / 4);
      k_z_reg<T, NZ, FORM, 4><<<dim3((unsigned)((nlines + LPB - 1) / LPB), nmem), NT, 0, st>>>((V*)P, g, (const V*)tw,
                                                                                              msP, zkeep);
      ++g_launches;
      return cudaGetLastError();
    }
  }
  if constexpr (FORM <= 2 && M % 3 != 0 && M / ztma_e<T>() <= 32 && !std::is_same<T, float>::value) {
    // FP64: bulk-copy variant (whole groups, 16-byte aligned group starts)
    constexpr int LPB = ztma_lpb<T, NZ>();
    const size_t sm = 2ull * NIN * LPB * (M + 1) * sizeof(V) + (size_t)LPB * zslot<M>() * sizeof(V) + 128;
    if (nlines % LPB == 0 && (LPB * (M + 1) * sizeof(V)) % 16 == 0 && sm <= 220 * 1024) {
      const long long ngroups = nlines / LPB;
      auto k = k_z_tma<T, NZ, FORM>;
      if ((err = smem_attr(k, sm)) != cudaSuccess) return err;
      k<<<dim3((unsigned)(ngroups < 148 ? ngroups : 148), nmem), 256, sm, st>>>((V*)P, g, (const V*)tw, zerr, msP,
                                                                                 zkeep);
      ++g_launches;
      return cudaGetLastError();
    }
  }
  if constexpr (FORM == 3 && !std::is_same<T, float>::value && M % 3 != 0 && M / 4 <= 32) {
    // FP64 adjoint: register-resident with 4 elements per thread
    constexpr int NT = zreg_threads<3>(), LPB = NT / (M / 4);
    k_z_reg_adj<T, NZ><<<(unsigned)((nlines + LPB - 1) / LPB), NT, 0, st>>>((V*)P, g, (const V*)tw, zkeep);
    ++g_launches;
    return cudaGetLastError();
  }
  if constexpr (M <= 512 && (M % 3 != 0 || FORM != 3) && std::is_same<T, float>::value) {
    // FP32: register-resident variant, lines of M/E lanes (E = 8, or 12 with a factor 3;
    // up to two warps per line)
    constexpr int NT = zreg_threads<FORM>(), LPB = NT / (M / ((M % 3 == 0) ? 12 : 8));
    if constexpr (FORM == 3)
      k_z_reg_adj<T, NZ><<<(unsigned)((nlines + LPB - 1) / LPB), NT, 0, st>>>((V*)P, g, (const V*)tw, zkeep);
    else
      k_z_reg<T, NZ, FORM><<<dim3((unsigned)((nlines + LPB - 1) / LPB), nmem), NT, 0, st>>>((V*)P, g, (const V*)tw,
                                                                                           msP, zkeep);
    ++g_launches;
    return cudaGetLastError();
  }
  // shared-memory slot variant (large lines, and line lengths with a factor 3)
  return z_slots<NZ, FORM, e_mixed(M, 8)>(g, P, tw, st, nmem, msP, zkeep);
}

template <> cudaError_t Launch<T>::z_fused(const Geo& g, int form, void* P, const void* tw, int* zerr,
                                           cudaStream_t st, int nmem, long long msP, int zkeep) {
  cudaError_t err = cudaErrorInvalidValue;
  if (form == 3 && nmem != 1) return err;  // the adjoint z pass has no member batching
  dispatch_L_sff(g.Nz, [&](auto Lc) {
    constexpr int NZ = decltype(Lc)::value;
    const int v = g.tv[TUNE_Z];
    if (form == 0) err = z_fused_impl<NZ, 0>(g, P, tw, zerr, st, nmem, msP, zkeep, v);
    else if (form == 1) err = z_fused_impl<NZ, 1>(g, P, tw, zerr, st, nmem, msP, zkeep, v);
    else if (form == 2) err = z_fused_impl<NZ, 2>(g, P, tw, zerr, st, nmem, msP, zkeep, v);
    else if (form == 5) err = z_fused_impl<NZ, 5>(g, P, tw, zerr, st, nmem, msP, zkeep, 0);
    else if (form == 6) err = z_fused_impl<NZ, 6>(g, P, tw, zerr, st, nmem, msP, zkeep, 0);
    else if constexpr (NZ % 3 != 0) err = z_fused_impl<NZ, 3>(g, P, tw, zerr, st, 1, 0, zkeep, 0);
  });
  return err;
}

// SSS fused z pass (form 0 or 2): the slot layout of the FFF slot kernel with NIN
// input slots and one work slot per line, lines per block within about 106 KB of
// shared memory
template <int NZ, int FORM>
static cudaError_t sss_z_slots(const Geo& g, void* P, const void* tw, const void* tq, int zin, int zout,
                               cudaStream_t st) {
  constexpr int M = NZ / 2;
  // 4 elements per thread: twice the threads per z line of the 8-element form, and half
  // the shared memory per block, so more warps per SM for this latency-bound pass
  constexpr int E = (M % 3 != 0 && M >= 8) ? 4 : e_mixed(M, 8);
  constexpr int TPL = M / E;
  constexpr int NSL = z_nin(FORM) + 1;
  const long long nlines = (long long)g.Nx * g.Ny;
  int nl = 256 / TPL;
  while (nl > 1 && (size_t)NSL * nl * zslot<M>() * sizeof(V) > 106 * 1024) nl /= 2;
  const size_t sm = (size_t)NSL * nl * zslot<M>() * sizeof(V);
  cudaError_t err;
  auto k = k_sss_z_fused<T, NZ, E, FORM>;
  if ((err = smem_attr(k, sm)) != cudaSuccess) return err;
  k<<<(unsigned)((nlines + nl - 1) / nl), nl * TPL, sm, st>>>((V*)P, g, (const V*)tw, (const V*)tq, nl, zin, zout,
                                                              (T)(1.0 / (2.0 * NZ)));
  ++g_launches;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::sss_z_fused(const Geo& g, int form, void* P, const void* tw, const void* tq, int zin,
                                               int zout, cudaStream_t st) {
  cudaError_t err = cudaErrorInvalidValue;
  if (form != 0 && form != 2 && form != 6) return err;
  dispatch_L(g.Nz, [&](auto Lc) {
    constexpr int NZ = decltype(Lc)::value;
    err = form == 0 ? sss_z_slots<NZ, 0>(g, P, tw, tq, zin, zout, st)
        : form == 2 ? sss_z_slots<NZ, 2>(g, P, tw, tq, zin, zout, st)
                    : sss_z_slots<NZ, 6>(g, P, tw, tq, zin, zout, st);
  });
  return err;
}

template <> cudaError_t Launch<T>::z_single(const Geo& g, int dir, const void* in, void* out, int ncomp,
                                            const void* tw, cudaStream_t st) {
  cudaError_t err = cudaErrorInvalidValue;
  dispatch_L(g.Nz, [&](auto Lc) {
    constexpr int NZ = decltype(Lc)::value;
    constexpr int M = NZ / 2, H = M + 1;
    constexpr int E = emin(E_REG, M);
    const int nl = z_lines(1, H);
    const size_t sm = 2ull * nl * H * sizeof(V);
    const long long nlines = (long long)g.Nx * g.Ny;
    dim3 grid((unsigned)((nlines + nl - 1) / nl), ncomp);
    if (dir < 0) {
      auto k = k_z_single<T, NZ, E, -1>;
      if ((err = smem_attr(k, sm)) != cudaSuccess) return;
      k<<<grid, 256, sm, st>>>((const V*)in, (V*)out, g, (const V*)tw, nl, ncomp);
    } else {
      auto k = k_z_single<T, NZ, E, 1>;
      if ((err = smem_attr(k, sm)) != cudaSuccess) return;
      k<<<grid, 256, sm, st>>>((const V*)in, (V*)out, g, (const V*)tw, nl, ncomp);
    }
    ++g_launches;
    err = cudaGetLastError();
  });
  return err;
}

template <int FORM, int MODE, int LL, int E, int CW>
static cudaError_t fwd_x_fused(const Geo& g, const void* P, const StageArgs& a, const void* tw, cudaStream_t st);

// forward x candidates (MODE_STEP): 1 = the split form (strided x FFT, then the
// elementwise epilogue) where the rule is the fused TMA kernel; 2 = the fused
// kernel with half-width column tiles (32-byte rows in FP32; where the rule
// splits, the fused kernel at the rule's tile width); 3 = the fused kernel with
// 8 elements per thread (half the threads)
constexpr bool fx_rule_fused(int L) { return xcw(L) * sizeof(V) >= 64; }
constexpr int fx_cw2(int L) { return fx_rule_fused(L) ? xcw(L) / 2 : xcw(L); }
constexpr bool fx_valid(int L, int v) {
  return v == 0 || (v == 1 && fx_rule_fused(L)) || (v == 2 && fx_cw2(L) * sizeof(V) >= 16 && fx_cw2(L) * (L / emin(E_ACC, L)) >= 32) ||
         (v == 3 && fx_rule_fused(L) && emin(E_ACC_ALT, L) != emin(E_ACC, L));
}


template <int FORM, int MODE, int LL>
static cudaError_t fwd_x_impl(const Geo& g, const void* P, const StageArgs& a, const void* tw, cudaStream_t st) {
  constexpr int CW = xcw(LL);
  const int v = MODE == MODE_STEP ? g.tv[TUNE_X_FWD] : 0;
  if constexpr (fx_valid(LL, 2)) {
    if (v == 2) return fwd_x_fused<FORM, MODE, LL, emin(E_ACC, LL), fx_cw2(LL)>(g, P, a, tw, st);
  }
  if constexpr (fx_valid(LL, 3)) {
    if (v == 3) return fwd_x_fused<FORM, MODE, LL, emin(E_ACC_ALT, LL), CW>(g, P, a, tw, st);
  }
  const bool split = CW * sizeof(V) < 64 || v == 1;
  if (split) {
    // tiles narrower than 64-byte rows: forward x FFT in place, then the elementwise epilogue
    constexpr int NF = FORM == 1 ? 3 : 6;
    cudaError_t err = Launch<T>::strided(g, 0, -1, const_cast<void*>(P), NF, tw, st);
    if (err != cudaSuccess) return err;
    const unsigned blocks = grid1d(g.S, 256);
    k_spec_epi<T, FORM, MODE><<<blocks, 256, 0, st>>>((const V*)P, g, a);
    ++g_launches;
    if (MODE == MODE_FLUX) {
      k_bins_finish<<<1, 64, 0, st>>>(a.bins + (a.nradii + 1), (int)blocks, a.nradii + 1, a.bins);
      ++g_launches;
    }
    return cudaGetLastError();
  }
  if constexpr (CW * sizeof(V) >= 64) return fwd_x_fused<FORM, MODE, LL, emin(E_ACC, LL), CW>(g, P, a, tw, st);
  return cudaErrorInvalidValue;
}

template <int FORM, int MODE, int LL, int E, int CW>
static cudaError_t fwd_x_fused(const Geo& g, const void* P, const StageArgs& a, const void* tw, cudaStream_t st) {
  const int inner = g.Ny * g.Hz;
  const int ntiles = (inner + CW - 1) / CW;
  size_t sm = (size_t)(MODE == MODE_NLIN ? 2 : 8) * LL * CW * sizeof(V) + (size_t)LL * (CW + 1) * sizeof(V) + 128;
  const int bps = MODE == MODE_STEP ? g.tb[TUNE_X_FWD] : 0;
  const int per_sm = bps > 0 ? bps : ((int)((220 * 1024) / sm) >= 2 ? 2 : 1);
  const int blocks = ntiles < 148 * per_sm ? ntiles : 148 * per_sm;
  const int br = LL < 256 ? LL : 256;
  CUtensorMap mP, mA, mB;
  cudaError_t err = make_field_map(&mP, P, inner, 6LL * g.Nx, UNITS, CW, br);
  if (err != cudaSuccess) return err;
  const void* A = MODE == MODE_FLUX ? a.Ud : ((MODE == MODE_STEP || MODE == MODE_ADJ) ? a.U0 : P);
  const void* B = (MODE == MODE_STEP || MODE == MODE_ADJ) ? a.tot : P;
  if ((err = make_field_map(&mA, A, inner, 3LL * g.Nx, UNITS, CW, br)) != cudaSuccess) return err;
  if ((err = make_field_map(&mB, B, inner, 3LL * g.Nx, UNITS, CW, br)) != cudaSuccess) return err;
  auto k = k_fwd_x<T, LL, E, CW, FORM, MODE>;
  if ((err = smem_attr(k, sm)) != cudaSuccess) return err;
  k<<<blocks, CW * (LL / E), sm, st>>>(mP, mA, mB, g, a, (const V*)tw);
  ++g_launches;
  if (MODE == MODE_FLUX) {
    k_bins_finish<<<1, 64, 0, st>>>(a.bins + (a.nradii + 1), blocks, a.nradii + 1, a.bins);
    ++g_launches;
  }
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::fwd_x(const Geo& g, int form, int mode, const void* P, const StageArgs& a,
                                         const void* tw, cudaStream_t st) {
  cudaError_t err = cudaErrorInvalidValue;
  dispatch_L(g.Nx, [&](auto Lc) {
    constexpr int LL = decltype(Lc)::value;
    if (form == 3) {
      if (mode == MODE_ADJ) err = fwd_x_impl<3, MODE_ADJ, LL>(g, P, a, tw, st);
    } else if (form == 1) {
      if (mode == MODE_STEP) err = fwd_x_impl<1, MODE_STEP, LL>(g, P, a, tw, st);
      else if (mode == MODE_FLUX) err = fwd_x_impl<1, MODE_FLUX, LL>(g, P, a, tw, st);
      else err = fwd_x_impl<1, MODE_NLIN, LL>(g, P, a, tw, st);
    } else {
      if (mode == MODE_STEP) err = fwd_x_impl<0, MODE_STEP, LL>(g, P, a, tw, st);
      else if (mode == MODE_FLUX) err = fwd_x_impl<0, MODE_FLUX, LL>(g, P, a, tw, st);
      else err = fwd_x_impl<0, MODE_NLIN, LL>(g, P, a, tw, st);
    }
  });
  return err;
}

// SFF x candidates. Inverse: 1 = 4 elements per thread (power-of-two lengths),
// 2 = half-width column tiles. Forward: 1 = the other split choice (fused
// epilogue from 64 points on, split below), 2 = half-width column tiles.
constexpr int sx_e(int N, int dir) { return e_mixed(N, dir > 0 ? 8 : (std::is_same<T, float>::value ? 8 : 4)); }
constexpr Tile sx_cand(int N, int dir, int v) {
  return v == 0 ? Tile{sx_e(N, dir), cw_for(N, sx_e(N, dir)), 1}
       : v == 1 ? (dir > 0 ? (N % 3 != 0 && sx_e(N, dir) > 4 ? Tile{4, cw_for(N, 4), 1} : Tile{0, 0, 0})
                           : Tile{sx_e(N, dir), cw_for(N, sx_e(N, dir)), 2})
       : v == 2 ? (cw_for(N, sx_e(N, dir)) > 1 ? Tile{sx_e(N, dir), cw_for(N, sx_e(N, dir)) / 2, 1} : Tile{0, 0, 0})
                : Tile{0, 0, 0};
}
constexpr bool sx_valid(int N, int dir, int v) {
  return v == 0 || (N <= 512 && v < 3 && tile_fits(N, sx_cand(N, dir, v), 3) &&
                    !tile_eq(sx_cand(N, dir, v), sx_cand(N, dir, 0)));
}

template <> cudaError_t Launch<T>::sff_inv_x(const Geo& g, const void* U, const void* Tf, void* W, const void* tq,
                                             cudaStream_t st, int nmem, long long msU, long long msT, long long msW) {
  cudaError_t err = cudaErrorInvalidValue;
  const int v = g.tv[TUNE_X_INV];
  dispatch_L_sff(g.Nx, [&](auto Lc) {
    constexpr int NN = decltype(Lc)::value;
    if constexpr (NN <= 512) {
      // one NN-point FFT per column and field, 8 elements per thread
      auto run = [&](auto vc) {
        constexpr Tile c = sx_cand(NN, 1, decltype(vc)::value);
        constexpr int E = c.E, CW = c.CW;
        const int inner = g.Ny * g.Hz;
        const size_t sm = 3ull * NN * CW * sizeof(V);  // exchange + 2 staging tiles
        auto k = k_sff_inv_x<T, NN, E, CW>;
        if ((err = smem_attr(k, sm)) != cudaSuccess) return;
        k<<<dim3((inner + CW - 1) / CW, nmem), CW * (NN / E), sm, st>>>((const V*)U, (const V*)Tf, (V*)W, g,
                                                                     (const V*)tq, msU, msT, msW);
        ++g_launches;
        err = cudaGetLastError();
      };
      if (v == 1 && sx_valid(NN, 1, 1)) {
        if constexpr (sx_valid(NN, 1, 1)) run(std::integral_constant<int, 1>{});
      } else if (v == 2 && sx_valid(NN, 1, 2)) {
        if constexpr (sx_valid(NN, 1, 2)) run(std::integral_constant<int, 2>{});
      } else {
        run(std::integral_constant<int, 0>{});
      }
    }
  });
  return err;
}

template <> cudaError_t Launch<T>::sff_fwd_x(const Geo& g, const void* P, const SffArgs& a, const void* tq,
                                             cudaStream_t st, int nmem) {
  cudaError_t err = cudaErrorInvalidValue;
  const int v = g.tv[TUNE_X_FWD];
  dispatch_L_sff(g.Nx, [&](auto Lc) {
    constexpr int NN = decltype(Lc)::value;
    if constexpr (NN <= 512) {
      // one NN-point FFT per column and product; four accumulators per element:
      // 8 (FP32) / 4 (FP64) elements per thread
      auto run = [&](auto vc) {
        constexpr Tile c = sx_cand(NN, -1, decltype(vc)::value);
        constexpr int E = c.E, CW = c.CW;
        const int inner = g.Ny * g.Hz;
        const size_t sm = 3ull * NN * CW * sizeof(V);
        // from 64 points on, the x kernel writes the assembled vectors and a coalesced
        // elementwise kernel does the epilogue (its ten state reads stalled the fused form)
        constexpr bool SPLIT = (NN >= 64) != (c.NT == 2);
        auto k = k_sff_fwd_x<T, NN, E, CW, SPLIT>;
        if ((err = smem_attr(k, sm)) != cudaSuccess) return;
        k<<<dim3((inner + CW - 1) / CW, nmem), CW * (NN / E), sm, st>>>((V*)P, g, a, (const V*)tq);
        ++g_launches;
        if ((err = cudaGetLastError()) != cudaSuccess || !SPLIT) return;
        k_sff_epi<T><<<dim3(grid1d(g.S, 256), nmem), 256, 0, st>>>((const V*)P, g, a);
        ++g_launches;
        err = cudaGetLastError();
      };
      if (v == 1 && sx_valid(NN, -1, 1)) {
        if constexpr (sx_valid(NN, -1, 1)) run(std::integral_constant<int, 1>{});
      } else if (v == 2 && sx_valid(NN, -1, 2)) {
        if constexpr (sx_valid(NN, -1, 2)) run(std::integral_constant<int, 2>{});
      } else {
        run(std::integral_constant<int, 0>{});
      }
    }
  });
  return err;
}

template <> cudaError_t Launch<T>::sff_x(const Geo& g, int dir, void* A, int ncomp, int sine, double scl,
                                         const void* tq, cudaStream_t st, int nbatch, long long bstride) {
  cudaError_t err = cudaErrorInvalidValue;
  dispatch_L_sff(g.Nx, [&](auto Lc) {
    constexpr int NN = decltype(Lc)::value;
    if constexpr (NN <= 512) {
      constexpr int E = e_mixed(NN, 8);
      constexpr int CW = cw_for(NN, E);
      const int inner = g.Ny * g.Hz;
      const size_t sm = (size_t)NN * CW * sizeof(V);
      const dim3 grid((unsigned)(((long long)ncomp * inner + CW - 1) / CW), 1, nbatch);
      auto run = [&](auto k) {
        if ((err = smem_attr(k, sm)) != cudaSuccess) return;
        k<<<grid, CW * (NN / E), sm, st>>>((V*)A, g, (const V*)tq, sine, scl, bstride, ncomp);
        ++g_launches;
        err = cudaGetLastError();
      };
      if (dir < 0) run(k_sff_x<T, NN, E, CW, -1>);
      else run(k_sff_x<T, NN, E, CW, 1>);
    }
  });
  return err;
}

template <> cudaError_t Launch<T>::reality(const Geo& g, void* A, int ncomp, cudaStream_t st) {
  const long long n = (long long)g.Nx * g.Ny * ncomp;
  k_reality<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>((V*)A, ncomp, g);
  ++g_launches;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::rbc_slave(const Geo& g, void* U, void* Tf, int slave, double vs, cudaStream_t st) {
  k_rbc_slave<T><<<grid1d(g.S, 256), 256, 0, st>>>((V*)U, (V*)Tf, g, slave, vs);
  ++g_launches;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::reality_adj(const Geo& g, void* A, int ncomp, cudaStream_t st) {
  const long long n = (long long)g.Nx * g.Ny * ncomp;
  k_reality_adj<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>((V*)A, ncomp, g);
  ++g_launches;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::carati(const Geo& g, const void* U, void* fc, int km, double rin, double rout,
                                          const double* es, const double* hs, const double* mis, int nsup,
                                          cudaStream_t st) {
  k_carati<T><<<1, 256, 0, st>>>((const V*)U, (V*)fc, g, km, rin, rout, es, hs, mis, nsup);
  ++g_launches;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::energy(const Geo& g, const void* A, const void* B, int ncomp, double* out,
                                          cudaStream_t st) {
  // out[0] = the sum; out[1 .. blocks] hold the per-block partial sums (blocks <= 148 * 16)
  const unsigned blocks = grid1d(g.S, 256);
  k_energy<T><<<blocks, 256, 0, st>>>((const V*)A, (const V*)B, ncomp, g, out);
  k_sum_partials<<<1, 256, 0, st>>>(out, (int)blocks);
  g_launches += 2;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::maxdiv(const Geo& g, const void* U, unsigned long long* out, cudaStream_t st) {
  k_maxdiv<T><<<grid1d(g.S, 256), 256, 0, st>>>((const V*)U, g, out);
  ++g_launches;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::shell(const Geo& g, const void* A, int ncomp, int nbins, double* bins,
                                         cudaStream_t st, const void* B, unsigned cap) {
  const size_t sm = (size_t)(SHELL_WARPS + 1) * nbins * sizeof(double);
  if (sm > 220 * 1024) return cudaErrorInvalidValue;
  cudaError_t err = smem_attr(k_shell<T>, sm);
  if (err != cudaSuccess) return err;
  const unsigned blocks = shell_blocks(g, cap);
  k_shell<T><<<blocks, 32 * SHELL_WARPS, sm, st>>>((const V*)A, (const V*)B, ncomp, g, nbins, bins + 2 * nbins);
  k_bins_finish<<<(2 * nbins + 255) / 256, 256, 0, st>>>(bins + 2 * nbins, (int)blocks, 2 * nbins, bins);
  g_launches += 2;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::expire_wait(int* err, int polls, cudaStream_t st) {
  k_expire_wait<<<1, 32, 0, st>>>(err, polls);
  ++g_launches;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::flux_outside(const Geo& g, const void* P, const void* U, double R, double* out,
                                                cudaStream_t st) {
  const unsigned blocks = grid1d(g.S, 256);
  k_flux_outside<T><<<blocks, 256, 0, st>>>((const V*)P, (const V*)U, g, R, out);
  k_sum_partials<<<1, 256, 0, st>>>(out, (int)blocks);
  g_launches += 2;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::ssf_giver(const Geo& g, const void* U, void* P, double R, cudaStream_t st) {
  k_ssf_giver<T><<<grid1d(g.S, 256), 256, 0, st>>>((const V*)U, (V*)P, g, R);
  ++g_launches;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::ssf_flux_outside(const Geo& g, const void* P, const void* U, double R, int qx,
                                                    int qy, double* out, cudaStream_t st) {
  const unsigned blocks = grid1d(g.S, 256);
  k_ssf_flux_outside<T><<<blocks, 256, 0, st>>>((const V*)P, (const V*)U, g, R, qx, qy, out);
  k_sum_partials<<<1, 256, 0, st>>>(out, (int)blocks);
  g_launches += 2;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::sss_giver(const Geo& g, const void* U, void* P, double R, cudaStream_t st) {
  k_sss_giver<T><<<grid1d(2 * g.S, 256), 256, 0, st>>>((const T*)U, (T*)P, g, R);
  ++g_launches;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::sss_flux_outside(const Geo& g, const void* P, const void* U, double R, int qx,
                                                    int qy, int qz, double* out, cudaStream_t st) {
  const unsigned blocks = grid1d(2 * g.S, 256);
  k_sss_flux_outside<T><<<blocks, 256, 0, st>>>((const T*)P, (const T*)U, g, R, qx, qy, qz, out);
  k_sum_partials<<<1, 256, 0, st>>>(out, (int)blocks);
  g_launches += 2;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::force_scatter(const Geo& g, const void* fc, void* F, int km, cudaStream_t st) {
  const long long n = 3LL * (2 * km + 1) * (2 * km + 1) * (km + 1);
  k_force_scatter<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>((const V*)fc, (V*)F, g, km);
  ++g_launches;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::init_ic(const Geo& g, void* U, const double* Eic, const double* mis, int nsh,
                                           unsigned long long key, cudaStream_t st) {
  k_init_ic<T><<<grid1d(g.S, 256), 256, 0, st>>>((V*)U, g, Eic, mis, nsh, key);
  ++g_launches;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::init_temp(const Geo& g, void* A, double amp, double kmax, unsigned long long key,
                                             cudaStream_t st) {
  k_init_temp<T><<<grid1d(g.S, 256), 256, 0, st>>>((V*)A, g, amp, kmax, key);
  ++g_launches;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::scale(void* A, long long n, double s, cudaStream_t st) {
  k_scale<T><<<grid1d(n, 256), 256, 0, st>>>((V*)A, n, s);
  ++g_launches;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::scalar_epi(const Geo& g, const void* P, const SffArgs& a, cudaStream_t st) {
  k_scalar_epi<T><<<grid1d(g.S, 256), 256, 0, st>>>((const V*)P, g, a);
  ++g_launches;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::sss_zperm_fwd(const void* u, void* v, long long nlines, int N, int sine,
                                                cudaStream_t st) {
  k_sss_zperm_fwd<T><<<grid1d(nlines * (N + 2), 256), 256, 0, st>>>((const T*)u, (T*)v, nlines, N, sine);
  ++g_launches;
  return cudaGetLastError();
}
template <> cudaError_t Launch<T>::sss_zpost_fwd(const void* Z, void* c, long long nlines, int N, int sine, double scl,
                                                const void* tq, cudaStream_t st) {
  k_sss_zpost_fwd<T><<<grid1d(nlines * (N + 2), 256), 256, 0, st>>>((const V*)Z, (T*)c, nlines, N, sine, scl,
                                                                     (const V*)tq);
  ++g_launches;
  return cudaGetLastError();
}
template <> cudaError_t Launch<T>::sss_zpre_inv(const void* c, void* Vout, long long nlines, int N, int sine,
                                               const void* tq, cudaStream_t st) {
  k_sss_zpre_inv<T><<<grid1d(nlines * (N / 2 + 1), 256), 256, 0, st>>>((const T*)c, (V*)Vout, nlines, N, sine,
                                                                        (const V*)tq);
  ++g_launches;
  return cudaGetLastError();
}
template <> cudaError_t Launch<T>::sss_zperm_inv(const void* v, void* u, long long nlines, int N, int sine,
                                                cudaStream_t st) {
  k_sss_zperm_inv<T><<<grid1d(nlines * (N + 2), 256), 256, 0, st>>>((const T*)v, (T*)u, nlines, N, sine);
  ++g_launches;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::sss_dealias_copy(const Geo& g, const void* A, void* B, int ncomp,
                                                   cudaStream_t st) {
  k_sss_dealias_copy<T><<<dim3(grid1d(g.S, 256), ncomp), 256, 0, st>>>((const T*)A, (T*)B, ncomp, g);
  ++g_launches;
  return cudaGetLastError();
}
template <> cudaError_t Launch<T>::sss_epi(const Geo& g, const void* P, const StageArgs& a, cudaStream_t st) {
  k_sss_epi<T><<<grid1d(2 * g.S, 256), 256, 0, st>>>((const T*)P, g, a);
  ++g_launches;
  return cudaGetLastError();
}


template <> cudaError_t Launch<T>::ssf_epi(const Geo& g, const void* P, const StageArgs& a, cudaStream_t st) {
  k_ssf_epi<T><<<grid1d(g.S, 256), 256, 0, st>>>((const V*)P, g, a);
  ++g_launches;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::ssf_rbc_epi(const Geo& g, const void* P, const SffArgs& a, cudaStream_t st) {
  k_ssf_rbc_epi<T><<<grid1d(g.S, 256), 256, 0, st>>>((const V*)P, g, a);
  ++g_launches;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::sss_rbc_epi(const Geo& g, const void* P, const SffArgs& a, cudaStream_t st) {
  k_sss_rbc_epi<T><<<grid1d(2 * g.S, 256), 256, 0, st>>>((const T*)P, g, a);
  ++g_launches;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::mhd_epi(const Geo& g, const void* P, const SffArgs& a, cudaStream_t st) {
  k_mhd_epi<T><<<grid1d(g.S, 256), 256, 0, st>>>((const V*)P, g, a);
  ++g_launches;
  return cudaGetLastError();
}

template <> cudaError_t Launch<T>::dealias_copy(const Geo& g, const void* A, void* B, int ncomp, cudaStream_t st) {
  k_dealias_copy<T><<<dim3(grid1d(g.S, 256), ncomp), 256, 0, st>>>((const V*)A, (V*)B, ncomp, g);
  ++g_launches;
  return cudaGetLastError();
}

template <> bool Launch<T>::tune_valid(const Geo& g, int form, int cls, int v) {
  if (v == 0) return true;
  if (v < 0 || v >= NCAND) return false;
  const bool sff = g.basis == 1;
  bool ok = false;
  switch (cls) {
    case TUNE_Y_INV:
    case TUNE_Y_FWD:
      dispatch_L_sff(g.Ny, [&](auto Lc) { ok = str_valid(decltype(Lc)::value, v); });
      break;
    case TUNE_X_INV:
      if (sff) dispatch_L_sff(g.Nx, [&](auto Lc) { ok = sx_valid(decltype(Lc)::value, 1, v); });
      else if (form <= 1) dispatch_L(g.Nx, [&](auto Lc) { ok = ix_valid(decltype(Lc)::value, v); });
      break;
    case TUNE_X_FWD:
      if (sff) dispatch_L_sff(g.Nx, [&](auto Lc) { ok = sx_valid(decltype(Lc)::value, -1, v); });
      else if (form <= 1) dispatch_L(g.Nx, [&](auto Lc) { ok = fx_valid(decltype(Lc)::value, v); });
      break;
    case TUNE_Z:
      dispatch_L_sff(g.Nz, [&](auto Lc) {
        constexpr int NZ = decltype(Lc)::value;
        ok = form == 0 ? z_valid<NZ, 0>(v) : form == 1 ? z_valid<NZ, 1>(v) : form == 2 ? z_valid<NZ, 2>(v) : false;
      });
      break;
    default:
      break;
  }
  return ok;
}

template <> bool Launch<T>::tune_blocks(const Geo& g, int form, int cls) {
  if (cls == TUNE_Y_INV || cls == TUNE_Y_FWD) return true;
  bool ok = false;
  if (cls == TUNE_X_FWD && g.basis == 0 && form <= 1)
    dispatch_L(g.Nx, [&](auto Lc) {
      constexpr int LL = decltype(Lc)::value;
      const int v = g.tv[TUNE_X_FWD];
      ok = (v == 0 && fx_rule_fused(LL)) || (v >= 2 && fx_valid(LL, v));
    });
  return ok;
}

}  // namespace ts
