// FFF (triply periodic Fourier) kernels of the IF-RK4 right-hand side.
//
// Spectral layout (identical to the reference's Blitz arrays, FFF_pencil.cc:209-233):
// one component = complex (Nx, Ny, Hz = Nz/2+1), C order, kx and ky in FFT order;
// a vector field is three components stored back to back.
//
// One right-hand-side evaluation is five launches:
//   inv_x  : dealias on load (+ vorticity for the rotational form), inverse FFT along x
//   y      : inverse FFT along y (in place)
//   z      : C2R along z -> real-space products -> R2C along z (one kernel, smem resident)
//   y      : forward FFT along y (in place)
//   fwd_x  : forward FFT along x + N_i assembly + force + Leray projection
//            + the IF-RK4 stage update (or a flux reduction / plain N output)
#pragma once
#include "ts_common.cuh"
#include "ts_tma.cuh"

namespace ts {

// pass classes of the launch tuning: inverse x, inverse y, z, forward y, forward x
enum { TUNE_X_INV = 0, TUNE_Y_INV = 1, TUNE_Z = 2, TUNE_Y_FWD = 3, TUNE_X_FWD = 4, TUNE_NCLASS = 5, TUNE_NCAND = 6 };

struct Geo {
  int Nx, Ny, Nz, Hz;
  long long S;          // complex elements per component
  double kf[3];         // kfactor (reference kfactor[1..3])
  int basis;            // 0 FFF, 1 SFF
  int dealias;          // 0 none, 1 reference corner, 2 two thirds
  // launch tuning per pass class: kernel candidate (0 = the fixed rule) and
  // blocks per SM of the persistent launches (0 = the rule)
  signed char tv[TUNE_NCLASS] = {0, 0, 0, 0, 0};
  signed char tb[TUNE_NCLASS] = {0, 0, 0, 0, 0};
};

// warps per block of the shell-sum kernel k_shell (each warp walks whole z lines)
constexpr int SHELL_WARPS = 4;

// ---------------------------------------------------------------------------
// plain strided-axis FFT (x or y axis) over nf fields, in place
// element (o, row, col) at o*ostride + row*rstride + col, col < inner.
// Persistent and double-buffered: block b walks the work items
// w = b, b + G, ... (w -> field, column tile, outer index); while item w is
// transformed (registers + exchange tile) the tile of its next item streams
// into the other staging tile with cp.async.
// Shared memory: 2 staging tiles + 1 exchange tile of L x CW complex (NT = 3),
// or 2 staging tiles with the consumed one doubling as the exchange tile
// (NT = 2: wider column tiles fit, e.g. 8 columns at L = 1024 in FP32), or
// 3 staging tiles with the consumed one as the exchange tile (NT = 4: the tiles of
// the next two items stream in while one is transformed), or one tile that is also
// the exchange tile (NT = 1: no prefetch inside a block; the blocks sharing an SM
// overlap one another's loads).
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int str_tiles(int nt) { return nt == 4 ? 3 : nt; }
template <typename T, int L, int E, int CW, int DIR, int NT = 3>
__global__ void __launch_bounds__(CW * (L / E), (CW * (L / E)) <= 256 ? 2 : 1)
    k_strided_fft(C<T>* __restrict__ data, int nf, long long fstride, int inner, long long rstride,
                  long long ostride, int nouter, const C<T>* __restrict__ tw, int per, long long mstride,
                  int zero_hi) {
  typedef C<T> V;
  static_assert(NT >= 1 && NT <= 4, "one to three staging tiles");
  constexpr int NBUF = NT == 4 ? 3 : (NT == 1 ? 1 : 2);  // staging tiles: items in flight = NBUF - 1 ahead
  constexpr bool XC = NT != 3;           // exchange in the consumed staging tile
  extern __shared__ __align__(16) unsigned char smraw[];
  V* stage = reinterpret_cast<V*>(smraw);
  const int c = threadIdx.x % CW, t = threadIdx.x / CW;
  const int ntx = (inner + CW - 1) / CW;
  const long long nwork = (long long)nf * ntx * nouter;
  // work item -> (pointer of its column, column valid); field f is field f % per
  // of member f / per (members mstride apart; per = nf for one member)
  auto locate = [&](long long w, bool& ok) -> V* {
    const int f = (int)(w % nf);
    const long long r = w / nf;
    const int tx = (int)(r % ntx);
    const long long o = r / ntx;
    const int col = tx * CW + c;
    ok = col < inner;
    return data + (f / per) * mstride + (f % per) * fstride + o * ostride + (ok ? col : 0);
  };
  auto issue = [&](long long w, int buf) {
    if (w < nwork) {
      bool ok;
      const V* d = locate(w, ok);
      if (ok) {
        V* st = stage + buf * L * CW + c;
#pragma unroll
        for (int s = 0; s < E; ++s) {
          const int r = load_row<L, E>(t, s);
          if (!(zero_hi && 3 * (r < L - r ? r : L - r) > L)) cp_async(st + r * CW, d + r * rstride);
        }
      }
    }
    cp_async_commit();
  };
  // the first NBUF - 1 items; every issue commits one cp.async group (empty past the end)
  issue(blockIdx.x, 0);
  if (NBUF == 3) issue(blockIdx.x + gridDim.x, 1);
  int buf = 0;
  for (long long w = blockIdx.x; w < nwork; w += gridDim.x, buf = (buf + 1 == NBUF ? 0 : buf + 1)) {
    // item w + (NBUF-1) G into the tile item w - G used (every thread passed the
    // barrier after its last exchange read), then wait for item w's group
    issue(w + (NBUF - 1) * (long long)gridDim.x, buf == 0 ? NBUF - 1 : buf - 1);
    cp_async_wait<NBUF - 1>();
    bool ok;
    V* d = locate(w, ok);
    V v[E];
    const V* st = stage + buf * L * CW + c;
#pragma unroll
    for (int s = 0; s < E; ++s) {
      // zero_hi: rows with 3 |k| > L (two-thirds dealiased) are zero and were not loaded
      const int r = load_row<L, E>(t, s);
      v[s] = (ok && !(zero_hi && 3 * (r < L - r ? r : L - r) > L)) ? st[r * CW] : mk<V>(0, 0);
    }
    // each thread read back only what it staged itself; the barrier is for the
    // exchange writes into the consumed tile (NT = 2, 4)
    if (XC) __syncthreads();
    fft_regs<L, E, DIR, 0, false, false, best_swk(L, E, CW, (int)sizeof(V))>(
        v, t, XC ? stage + buf * L * CW : stage + 2 * L * CW, CW, c, tw, 1);
    if (ok) {
#pragma unroll
      for (int s = 0; s < E; ++s) d[final_row<L, E>(t, s) * rstride] = v[s];
    }
  }
}

// ---------------------------------------------------------------------------
// inverse x pass: W_i = IFFT_x(D(U_i)); rotational form also W_{3+i} = IFFT_x(D(omega_i)),
// omega = i K x D(U).  col = ly*Hz + lz; row = lx.
// Persistent over column tiles.  Thread 0 streams the three components of a
// tile into shared memory with TMA (2-D boxes of CW columns x <=256 rows,
// mbarrier completion), double buffered so tile k+1 loads while tile k is
// transformed.  Shared memory: 2 x 3 staging tiles + 1 exchange tile.
// ---------------------------------------------------------------------------
template <typename T, int L, int E, int CW, bool ROT>
__global__ void __launch_bounds__(CW * (L / E), 1)
    k_inv_x(const __grid_constant__ CUtensorMap mU, C<T>* __restrict__ W, Geo g, const C<T>* __restrict__ tw,
            int* err) {
  typedef C<T> V;
  constexpr int TILE = L * CW, BR = L < 256 ? L : 256, UNITS = (int)sizeof(V) / 8;
  extern __shared__ __align__(128) unsigned char smraw_[];
  // TMA destinations: 128-byte aligned (the launcher adds 128 bytes of slack)
  unsigned char* smraw = smraw_ + ((128 - (smem_u32(smraw_) & 127)) & 127);
  V* stage = reinterpret_cast<V*>(smraw);  // [2][3][TILE]
  V* xch = stage + 6 * TILE;
  __shared__ __align__(8) uint64_t bar[2];
  const int c = threadIdx.x % CW, t = threadIdx.x / CW;
  const int inner = g.Ny * g.Hz;
  const int ntiles = (inner + CW - 1) / CW;
  const long long rstride = inner;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto issue = [&](int tile, int slot) {
    if (tile >= ntiles) return;
    mbar_expect_tx(&bar[slot], 3u * TILE * (unsigned)sizeof(V));
    for (int comp = 0; comp < 3; ++comp)
      for (int r0 = 0; r0 < L; r0 += BR)
        tma_load_2d(stage + (slot * 3 + comp) * TILE + r0 * CW, &mU, tile * CW * UNITS, comp * g.Nx + r0, &bar[slot]);
  };
  if (threadIdx.x == 0) {
    issue(blockIdx.x, 0);
    issue(blockIdx.x + gridDim.x, 1);
  }
  const int nout = ROT ? 6 : 3;
  int k = 0;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++k) {
    // slots alternate, so slot k & 1 completes its phase (k >> 1) & 1
    const int slot = k & 1;
    const uint32_t phase = (uint32_t)(k >> 1) & 1u;
    const bool got = mbar_wait(&bar[slot], phase, err);
    if (__syncthreads_or(!got)) {
      // give every copy in flight (this tile's and the next tile's, issued into the
      // other slot) a second bounded chance to land before the block's shared memory
      // goes away, then leave
      if (threadIdx.x == 0) {
        mbar_wait(&bar[slot], phase, nullptr);
        if (tile + (int)gridDim.x < ntiles) mbar_wait(&bar[slot ^ 1], (uint32_t)((k + 1) >> 1) & 1u, nullptr);
      }
      return;
    }
    const int col = tile * CW + c;
    const bool ok = col < inner;
    const int ly = ok ? col / g.Hz : 0, lz = ok ? col % g.Hz : 0;
    const T Ky = (T)(kfft(ly, g.Ny) * g.kf[1]), Kz = (T)(lz * g.kf[2]);
    const V* st = stage + slot * 3 * TILE + c;
    for (int f = 0; f < nout; ++f) {
      V v[E];
#pragma unroll
      for (int s = 0; s < E; ++s) {
        const int lx = load_row<L, E>(t, s);
        V a = mk<V>(0, 0);
        if (ok && !dealias_zero(g.dealias, g.basis, lx, ly, lz, g.Nx, g.Ny, g.Nz)) {
          if (f < 3) {
            a = st[f * TILE + lx * CW];
          } else {
            // omega_i = i (K_{i+1} U_{i+2} - K_{i+2} U_{i+1})  (indices mod 3)
            const T Kx = (T)(kfft(lx, g.Nx) * g.kf[0]);
            const int i = f - 3, i1 = i == 2 ? 0 : i + 1, i2 = i == 0 ? 2 : i - 1;
            const T Ka = i1 == 0 ? Kx : (i1 == 1 ? Ky : Kz);
            const T Kb = i2 == 0 ? Kx : (i2 == 1 ? Ky : Kz);
            const V ub = st[i2 * TILE + lx * CW], ua = st[i1 * TILE + lx * CW];
            a = mul_i<1>(sub(scale(ub, Ka), scale(ua, Kb)));
          }
        }
        v[s] = a;
      }
      if (f == nout - 1) {
        // every thread has read this slot: refill it with the tile after next
        __syncthreads();
        if (threadIdx.x == 0) issue(tile + 2 * gridDim.x, slot);
      }
      fft_regs<L, E, 1, 0, false, false, best_swk(L, E, CW, (int)sizeof(V))>(v, t, xch, CW, c, tw, 1);
      if (ok) {
        V* d = W + f * g.S + col;
#pragma unroll
        for (int s = 0; s < E; ++s) d[final_row<L, E>(t, s) * rstride] = v[s];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// inverse x pass, direct-load variant (one column tile per block, loads straight
// into registers; two blocks of 256 threads per SM).  Same result as k_inv_x.
// FORM 0: W_0..2 = D U.  FORM 1: also W_3..5 = D omega.  FORM 3 (adjoint of the
// rotational right-hand side): also W_6..8 = lsc c^-1 P Lam, the Leray-projected
// cotangent divided by the C2R weight c (2 on the planes 0 < kz < Nz/2, else 1).
// ---------------------------------------------------------------------------
// FORM 4: the cotangent fields 6..8 of FORM 3 only (written at W + 6 S ...)
// FORM 5 (the giver of the per-sphere energy flux): W_0..2 = D U and W_3..5 = D U
// inside the sphere |K| <= rad (Fill_in_sphere, fill_space.cc:56-64), zero outside
__host__ __device__ constexpr int inv_x_nout(int form) { return form == 0 ? 3 : ((form == 1 || form == 5) ? 6 : 9); }
__host__ __device__ constexpr int inv_x_first(int form) { return form == 4 ? 6 : 0; }

template <typename T, int L, int E, int CW, int FORM>
__global__ void __launch_bounds__(CW * (L / E), (CW * (L / E)) <= 256 ? 2 : 1)
    k_inv_x_ld(const C<T>* __restrict__ U, C<T>* __restrict__ W, Geo g, const C<T>* __restrict__ tw,
               const C<T>* __restrict__ Lam, T lsc, int kept, double rad) {
  typedef C<T> V;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* sm = reinterpret_cast<V*>(smraw);
  const int c = threadIdx.x % CW, t = threadIdx.x / CW;
  const int inner = g.Ny * g.Hz;
  int col;
  bool ok;
  if (kept) {
    // two-thirds dealiasing: only the columns with 3|ky| <= Ny and 3 kz <= Nz can be
    // nonzero; block = (kept ly, tile of CW kept lz); the other columns are not
    // written, and the y and z passes treat them as zero without reading them
    const int qy = g.Ny / 3, nzk = g.Nz / 3 + 1, ntz = (nzk + CW - 1) / CW;
    const int iy = blockIdx.x / ntz, lzc = (blockIdx.x % ntz) * CW + c;
    const int ky = iy <= qy ? iy : iy - (2 * qy + 1);
    ok = lzc < nzk;
    col = ((ky + g.Ny) % g.Ny) * g.Hz + (ok ? lzc : 0);
  } else {
    col = blockIdx.x * CW + c;
    ok = col < inner;
  }
  const int ly = ok ? col / g.Hz : 0, lz = ok ? col % g.Hz : 0;
  const T Ky = (T)(kfft(ly, g.Ny) * g.kf[1]), Kz = (T)(lz * g.kf[2]);
  const long long rstride = inner;
  constexpr int nout = inv_x_nout(FORM);
  const T lw = (lz > 0 && 2 * lz < g.Nz) ? lsc * (T)0.5 : lsc;
  // FORM 5: |K| <= rad with |K| = sqrt((Kx^2 + Ky^2) + Kz^2) in FP64 (Kmagnitude)
  const double Kyd = kfft(ly, g.Ny) * g.kf[1], Kzd = lz * g.kf[2];
  auto in_sphere = [&](int lx) {
    const double Kxd = kfft(lx, g.Nx) * g.kf[0];
    return sqrt((Kxd * Kxd + Kyd * Kyd) + Kzd * Kzd) <= rad;
  };
  // FP32 with up to 8 elements per thread: the three (dealiased) components of U
  // are loaded once, up front, and every output field is built from registers
  // (FP64 would spill them)
  constexpr bool UPFRONT = E <= 8 && sizeof(T) == 4 && FORM != 4;
  V u[UPFRONT ? 3 : 1][UPFRONT ? E : 1];
  if constexpr (UPFRONT) {
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int lx = load_row<L, E>(t, s);
      const long long off = lx * rstride + col;
      const bool z = !ok || dealias_zero(g.dealias, g.basis, lx, ly, lz, g.Nx, g.Ny, g.Nz);
#pragma unroll
      for (int c = 0; c < 3; ++c) u[c][s] = z ? mk<V>(0, 0) : U[c * g.S + off];
    }
  }
  // unrolled (register path) so that the register-array indices below are compile-time constants
  constexpr int kUnroll = UPFRONT ? nout : 1;
#pragma unroll kUnroll
  for (int f = inv_x_first(FORM); f < nout; ++f) {
    V v[E];
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int lx = load_row<L, E>(t, s);
      const long long off = lx * rstride + col;
      V a = mk<V>(0, 0);
      if (UPFRONT && f < 6) {
        if (f < 3) {
          a = u[f][s];
        } else if (FORM == 5) {
          a = in_sphere(lx) ? u[f - 3][s] : mk<V>(0, 0);
        } else {
          const T Kx = (T)(kfft(lx, g.Nx) * g.kf[0]);
          const int i = f - 3, i1 = i == 2 ? 0 : i + 1, i2 = i == 0 ? 2 : i - 1;
          const T Ka = i1 == 0 ? Kx : (i1 == 1 ? Ky : Kz);
          const T Kb = i2 == 0 ? Kx : (i2 == 1 ? Ky : Kz);
          a = mul_i<1>(sub(scale(u[i2][s], Ka), scale(u[i1][s], Kb)));
        }
      } else if ((FORM == 3 || FORM == 4) && f >= 6) {
        if (ok) {
          // (P Lam)_i = Lam_i - K_i (K . Lam) / K^2, identity at K = 0
          const T Kx = (T)(kfft(lx, g.Nx) * g.kf[0]);
          const V l0 = Lam[off], l1 = Lam[g.S + off], l2 = Lam[2 * g.S + off];
          const T K2 = (Kx * Kx + Ky * Ky) + Kz * Kz;
          const V d = add(add(scale(l0, Kx), scale(l1, Ky)), scale(l2, Kz));
          const V q = K2 > (T)0 ? mk<V>(d.x / K2, d.y / K2) : mk<V>(0, 0);
          const int i = f - 6;
          const T Ki = i == 0 ? Kx : (i == 1 ? Ky : Kz);
          a = scale(sub(i == 0 ? l0 : (i == 1 ? l1 : l2), scale(q, Ki)), lw);
        }
      } else if (ok && !dealias_zero(g.dealias, g.basis, lx, ly, lz, g.Nx, g.Ny, g.Nz)) {
        if (f < 3) {
          a = U[f * g.S + off];
        } else if (FORM == 5) {
          a = in_sphere(lx) ? U[(f - 3) * g.S + off] : mk<V>(0, 0);
        } else {
          // omega_i = i (K_{i+1} U_{i+2} - K_{i+2} U_{i+1})  (indices mod 3)
          const T Kx = (T)(kfft(lx, g.Nx) * g.kf[0]);
          const int i = f - 3, i1 = i == 2 ? 0 : i + 1, i2 = i == 0 ? 2 : i - 1;
          const T Ka = i1 == 0 ? Kx : (i1 == 1 ? Ky : Kz);
          const T Kb = i2 == 0 ? Kx : (i2 == 1 ? Ky : Kz);
          const V ub = U[i2 * g.S + off], ua = U[i1 * g.S + off];
          a = mul_i<1>(sub(scale(ub, Ka), scale(ua, Kb)));
        }
      }
      v[s] = a;
    }
    fft_regs<L, E, 1, 0, false, false, best_swk(L, E, CW, (int)sizeof(V))>(v, t, sm, CW, c, tw, 1);
    if (ok) {
      V* d = W + f * g.S + col;
#pragma unroll
      for (int s = 0; s < E; ++s) d[final_row<L, E>(t, s) * rstride] = v[s];
    }
  }
}


// ---------------------------------------------------------------------------
// inverse x pass with the tile's U staged in shared memory (two-thirds dealiasing,
// FORM 0 / 1): one column tile per block (the kept-column mapping of k_inv_x_ld); every
// thread stages the kept rows (3 |kx| <= Nx) of the three components that it will read
// itself with cp.async, all in one group, so a tile pays one load latency instead of one
// per output field; the output fields are then built from shared memory (the vorticity
// from the staged components) and transformed through a separate exchange tile.
// Shared memory: 3 x LK x CW staged complex (LK = 2 (L/3) + 1 kept rows) + L x CW exchange.
// ---------------------------------------------------------------------------
template <int L> __host__ __device__ constexpr int ix_kept_rows() { return 2 * (L / 3) + 1; }
template <typename T, int L, int E, int CW, int FORM>
__global__ void __launch_bounds__(CW * (L / E), 1)
    k_inv_x_st(const C<T>* __restrict__ U, C<T>* __restrict__ W, Geo g, const C<T>* __restrict__ tw) {
  typedef C<T> V;
  static_assert(FORM == 0 || FORM == 1, "the fluid forms");
  constexpr int LK = ix_kept_rows<L>(), Q = L / 3;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* xch = reinterpret_cast<V*>(smraw);  // exchange tile, L x CW
  V* stg = xch + L * CW;                  // staged kept rows, 3 x LK x CW
  const int c = threadIdx.x % CW, t = threadIdx.x / CW;
  const int inner = g.Ny * g.Hz;
  const long long rstride = inner;
  const int qy = g.Ny / 3, nzk = g.Nz / 3 + 1, ntz = (nzk + CW - 1) / CW;
  const int iy = blockIdx.x / ntz, lzc = (blockIdx.x % ntz) * CW + c;
  const int ky = iy <= qy ? iy : iy - (2 * qy + 1);
  const bool ok = lzc < nzk;
  const int col = ((ky + g.Ny) % g.Ny) * g.Hz + (ok ? lzc : 0);
  const int lz = ok ? lzc : 0;
  const T Ky = (T)(ky * g.kf[1]), Kz = (T)(lz * g.kf[2]);
  // staged row of x row lx (kept rows only: lx <= Q or lx >= L - Q)
  auto krow = [](int lx) { return lx <= Q ? lx : lx - (L - 2 * Q - 1); };
  auto kept = [](int lx) { return lx <= Q || lx >= L - Q; };
  if (ok) {
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int lx = load_row<L, E>(t, s);
      if (kept(lx))
#pragma unroll
        for (int q = 0; q < 3; ++q) cp_async(stg + (q * LK + krow(lx)) * CW + c, U + q * g.S + lx * rstride + col);
    }
  }
  cp_async_commit();
  cp_async_wait<0>();  // each thread reads back only the rows it staged itself
  constexpr int nout = FORM == 0 ? 3 : 6;
#pragma unroll 1
  for (int f = 0; f < nout; ++f) {
    V v[E];
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int lx = load_row<L, E>(t, s);
      V a = mk<V>(0, 0);
      if (ok && kept(lx)) {
        const V* st = stg + krow(lx) * CW + c;
        if (f < 3) {
          a = st[f * LK * CW];
        } else {
          // omega_i = i (K_{i+1} U_{i+2} - K_{i+2} U_{i+1})  (indices mod 3)
          const T Kx = (T)(kfft(lx, g.Nx) * g.kf[0]);
          const int i = f - 3, i1 = i == 2 ? 0 : i + 1, i2 = i == 0 ? 2 : i - 1;
          const T Ka = i1 == 0 ? Kx : (i1 == 1 ? Ky : Kz);
          const T Kb = i2 == 0 ? Kx : (i2 == 1 ? Ky : Kz);
          a = mul_i<1>(sub(scale(st[i2 * LK * CW], Ka), scale(st[i1 * LK * CW], Kb)));
        }
      }
      v[s] = a;
    }
    fft_regs<L, E, 1, 0, false, false, best_swk(L, E, CW, (int)sizeof(V))>(v, t, xch, CW, c, tw, 1);
    if (ok) {
      V* d = W + f * g.S + col;
#pragma unroll
      for (int s = 0; s < E; ++s) d[final_row<L, E>(t, s) * rstride] = v[s];
    }
  }
}

// ---------------------------------------------------------------------------
// inverse x pass, persistent with a prefetch (FP32, FORM 0 / 1): each block walks the
// column tiles tile = blockIdx.x + k G; every thread stages the dealiased U rows it
// owns (rows load_row(t, s) of its column) with cp.async into its own slots of a
// staging tile, moves them to registers, issues the copies of its next tile into the
// same slots (only it reads them, so no barrier is needed) and then transforms the
// output fields of the current tile from registers while the next tile streams in.
// Same result as k_inv_x_ld.  Shared memory: the staging tile (3 L CW) + the
// exchange tile (L CW).
// ---------------------------------------------------------------------------
template <typename T, int L, int E, int CW, int FORM>
__global__ void __launch_bounds__(CW * (L / E), 1)
    k_inv_x_pf(const C<T>* __restrict__ U, C<T>* __restrict__ W, Geo g, const C<T>* __restrict__ tw, int kept) {
  typedef C<T> V;
  static_assert(FORM == 0 || FORM == 1, "the fluid forms");
  extern __shared__ __align__(16) unsigned char smraw[];
  V* xch = reinterpret_cast<V*>(smraw);  // exchange tile, L x CW
  V* stg = xch + L * CW;                  // staging tile, 3 x L x CW
  const int c = threadIdx.x % CW, t = threadIdx.x / CW;
  const int inner = g.Ny * g.Hz;
  const long long rstride = inner;
  const int qy = g.Ny / 3, nzk = g.Nz / 3 + 1, ntz = (nzk + CW - 1) / CW;
  const int ntiles = kept ? (2 * qy + 1) * ntz : (inner + CW - 1) / CW;
  // column of this thread in tile `tile` (the mapping of k_inv_x_ld's blocks)
  auto column = [&](int tile, bool& ok) -> int {
    if (kept) {
      const int iy = tile / ntz, lzc = (tile % ntz) * CW + c;
      const int ky = iy <= qy ? iy : iy - (2 * qy + 1);
      ok = lzc < nzk;
      return ((ky + g.Ny) % g.Ny) * g.Hz + (ok ? lzc : 0);
    }
    const int col = tile * CW + c;
    ok = col < inner;
    return ok ? col : 0;
  };
  auto issue = [&](int tile) {
    if (tile < ntiles) {
      bool ok;
      const int col = column(tile, ok);
      if (ok) {
        const int ly = col / g.Hz, lz = col % g.Hz;
#pragma unroll
        for (int s = 0; s < E; ++s) {
          const int lx = load_row<L, E>(t, s);
          if (!dealias_zero(g.dealias, g.basis, lx, ly, lz, g.Nx, g.Ny, g.Nz))
#pragma unroll
            for (int q = 0; q < 3; ++q) cp_async(stg + (q * L + lx) * CW + c, U + q * g.S + lx * rstride + col);
        }
      }
    }
    cp_async_commit();
  };
  constexpr int nout = FORM == 0 ? 3 : 6;
  issue(blockIdx.x);
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    cp_async_wait<0>();
    bool ok;
    const int col = column(tile, ok);
    const int ly = col / g.Hz, lz = col % g.Hz;
    const T Ky = (T)(kfft(ly, g.Ny) * g.kf[1]), Kz = (T)(lz * g.kf[2]);
    V u[3][E];
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int lx = load_row<L, E>(t, s);
      const bool z = !ok || dealias_zero(g.dealias, g.basis, lx, ly, lz, g.Nx, g.Ny, g.Nz);
#pragma unroll
      for (int q = 0; q < 3; ++q) u[q][s] = z ? mk<V>(0, 0) : stg[(q * L + lx) * CW + c];
    }
    // the slots are this thread's own: the next tile may stream into them now
    issue(tile + gridDim.x);
#pragma unroll
    for (int f = 0; f < nout; ++f) {
      V v[E];
#pragma unroll
      for (int s = 0; s < E; ++s) {
        if (f < 3) {
          v[s] = u[f][s];
        } else {
          // omega_i = i (K_{i+1} U_{i+2} - K_{i+2} U_{i+1})  (indices mod 3)
          const int lx = load_row<L, E>(t, s);
          const T Kx = (T)(kfft(lx, g.Nx) * g.kf[0]);
          const int i = f - 3, i1 = i == 2 ? 0 : i + 1, i2 = i == 0 ? 2 : i - 1;
          const T Ka = i1 == 0 ? Kx : (i1 == 1 ? Ky : Kz);
          const T Kb = i2 == 0 ? Kx : (i2 == 1 ? Ky : Kz);
          v[s] = mul_i<1>(sub(scale(u[i2][s], Ka), scale(u[i1][s], Kb)));
        }
      }
      fft_regs<L, E, 1, 0, false, false, best_swk(L, E, CW, (int)sizeof(V))>(v, t, xch, CW, c, tw, 1);
      if (ok) {
        V* d = W + f * g.S + col;
#pragma unroll
        for (int s = 0; s < E; ++s) d[final_row<L, E>(t, s) * rstride] = v[s];
      }
    }
  }
  cp_async_wait<0>();  // nothing in flight when the block leaves
}

// ---------------------------------------------------------------------------
// z pass: C2R of the NIN input lines, real-space products, R2C of the NOUT
// product lines.  Lines are contiguous (Hz = M+1 complex, M = Nz/2); a block
// handles `nl` consecutive (x,y) lines of every component, with TPL = M/E
// threads per line.  Each component's line is transformed in registers and
// exchanged through its own padded shared-memory slot (M + M/16 complex);
// after the inverse transforms slot c holds the real line of component c
// packed as M complex (re = even point, im = odd point), the products are
// formed in place per point, and each product line is transformed forward in
// its slot and post-processed straight to global memory.
// In place on P: outputs overwrite the first NOUT components at the same
// lines, after every input line has been read.
// FORM 0 (conservative): in u1,u2,u3 -> out u1u1,u2u2,u3u3,u1u2,u2u3,u3u1
// FORM 1 (rotational):   in u1..3,w1..3 -> out u x w
// ---------------------------------------------------------------------------
template <int M> __host__ __device__ constexpr int zslot() { return M + M / 16 + 1; }

// Real-space product forms of the z pass.
// FORM 0 (conservative):  in u1,u2,u3       -> u1u1,u2u2,u3u3,u1u2,u2u3,u3u1
// FORM 1 (rotational):    in u1..3,w1..3    -> u x w
// FORM 2 (Boussinesq):    in u1,u2,u3,T     -> the six u_i u_j, then u1T,u2T,u3T
//                         (compute_diag_offdiag.cc:47-136)
// FORM 3 (adjoint of the rotational form): in u, w, mu -> mu x u, then w x mu
// FORM 5 (MHD):           in u1..3, b1..3      -> Zp_i Zm_j (f = 3 i + j), Zp = u + b, Zm = u - b
//                         (compute_nlin_VF_MHD.cc:40-95, MHD.cc:75-84)
// FORM 6 (flux giver):    in u1..3, g1..3      -> u_i g_j (f = 3 i + j), for the giver nonlinear
//                         term N_i = sum_j D_j F[u_j g_i] (compute_nlin_ET_VF.cc:71-87)
__host__ __device__ constexpr int z_nin(int form) {
  return form == 0 ? 3 : (form == 1 ? 6 : (form == 2 ? 4 : ((form == 5 || form == 6) ? 6 : 9)));
}
__host__ __device__ constexpr int z_nout(int form) {
  return form == 0 ? 6 : (form == 1 ? 3 : (form == 2 ? 9 : ((form == 5 || form == 6) ? 9 : 6)));
}

// component f of a x b for real points packed two per complex (re, im independent)
template <typename V> __device__ __forceinline__ V cross_pk(int f, const V* a, const V* b) {
  const int i = f == 2 ? 0 : f + 1, j = f == 0 ? 2 : f - 1;
  return mk<V>(a[i].x * b[j].x - a[j].x * b[i].x, a[i].y * b[j].y - a[j].y * b[i].y);
}
// factor indices (a, b) of product output f for FORM 0 / 2
__host__ __device__ constexpr int z_pa(int f, int form = 0) {
  return (form == 5 || form == 6) ? f / 3 : (f < 3 ? f : (f < 6 ? f - 3 : f - 6));
}
__host__ __device__ constexpr int z_pb(int f, int form = 0) {
  return (form == 5 || form == 6) ? 3 + f % 3 : (f < 3 ? f : (f < 6 ? (f == 5 ? 0 : f - 2) : 3));
}
// FORM 5: the real lines of u and b (packed two points per complex) become the
// Elsasser lines Zp = u + b, Zm = u - b in place
template <int FORM, typename V> __device__ __forceinline__ void z_elsasser(V* in) {
  if constexpr (FORM == 5) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const V u = in[c], b = in[c + 3];
      in[c] = add(u, b);
      in[c + 3] = sub(u, b);
    }
  }
}

template <typename T, int NZ, int E, int FORM>
__global__ void __launch_bounds__(256) k_z_fused(C<T>* __restrict__ P, Geo g, const C<T>* __restrict__ tw, int nl,
                                                 long long msP, int zkeep) {
  typedef C<T> V;
  constexpr int M = NZ / 2, H = M + 1, TPL = M / E, LDS = zslot<M>();
  constexpr int NIN = z_nin(FORM), NOUT = z_nout(FORM);
  extern __shared__ __align__(16) unsigned char smraw[];
  V* sm = reinterpret_cast<V*>(smraw);
  const long long nlines = (long long)g.Nx * g.Ny;
  // member blockIdx.y (P + blockIdx.y * msP holds its fields)
  P += blockIdx.y * msP;
  const long long line0 = (long long)blockIdx.x * nl;
  const int nh = (int)((nlines - line0) < nl ? (nlines - line0) : nl);
  const int l = threadIdx.x / TPL, t = threadIdx.x % TPL;
  const bool live = l < nh;
  const long long lbase = (line0 + (live ? l : 0)) * H;
  auto slot = [&](int c, int ll) { return sm + (c * nl + ll) * LDS; };

  // A. inverse: Z[k] = (X + Y) + i conj(w^k)(X - Y), Y = conj(X[M-k]) (imag of X[0], X[M] dropped),
  //    then the length-M inverse FFT gives z[n] = u[2n] + i u[2n+1]
  for (int c = 0; c < NIN; ++c) {
    const V* X = P + c * g.S + lbase;
    V v[E];
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int k = load_row<M, E>(t, s);
      V a = mk<V>(0, 0), b = mk<V>(0, 0);
      const int zk = (FORM == 3 && c >= 6) ? M : zkeep;  // the adjoint's cotangent lines are full
      if (live && k <= zk) a = X[k];
      if (live && M - k <= zk) b = conjg(X[M - k]);
      if (k == 0) { a.y = 0; b.y = 0; }
      v[s] = add(add(a, b), mul_i<1>(mul(conjg(tw[k]), sub(a, b))));
    }
    V* sl = slot(c, l < nl ? l : 0);
    fft_regs<M, E, 1, 0, true>(v, t, sl, 1, 0, tw, 2);
#pragma unroll
    for (int s = 0; s < E; ++s) sl[prow<true>(final_row<M, E>(t, s))] = v[s];
  }
  __syncthreads();
  // B. products, in place per real point pair
  for (int e = threadIdx.x; e < nl * M; e += blockDim.x) {
    const int ll = e / M, m = prow<true>(e % M);
    V in[NIN];
#pragma unroll
    for (int c = 0; c < NIN; ++c) in[c] = slot(c, ll)[m];
    z_elsasser<FORM>(in);
    if constexpr (FORM == 3) {
#pragma unroll
      for (int f = 0; f < 3; ++f) {
        slot(f, ll)[m] = cross_pk(f, in + 6, in);
        slot(3 + f, ll)[m] = cross_pk(f, in + 3, in + 6);
      }
    } else if (FORM != 1) {
#pragma unroll
      for (int f = 0; f < NOUT; ++f)
        slot(f, ll)[m] = mk<V>(in[z_pa(f, FORM)].x * in[z_pb(f, FORM)].x, in[z_pa(f, FORM)].y * in[z_pb(f, FORM)].y);
    } else {
      slot(0, ll)[m] = mk<V>(in[1].x * in[5].x - in[2].x * in[4].x, in[1].y * in[5].y - in[2].y * in[4].y);
      slot(1, ll)[m] = mk<V>(in[2].x * in[3].x - in[0].x * in[5].x, in[2].y * in[3].y - in[0].y * in[5].y);
      slot(2, ll)[m] = mk<V>(in[0].x * in[4].x - in[1].x * in[3].x, in[0].y * in[4].y - in[1].y * in[3].y);
    }
  }
  __syncthreads();
  // C. forward: length-M FFT of z[n] = p[2n] + i p[2n+1], then
  //    X[k] = 1/2 (Z + Z') - i/2 w^k (Z - Z'), Z' = conj(Z[M-k]), Z[M] = Z[0]
  for (int c = 0; c < NOUT; ++c) {
    V* sl = slot(c, l < nl ? l : 0);
    V v[E];
#pragma unroll
    for (int s = 0; s < E; ++s) v[s] = sl[prow<true>(load_row<M, E>(t, s))];
    __syncthreads();
    fft_regs<M, E, -1, 0, true>(v, t, sl, 1, 0, tw, 2);
#pragma unroll
    for (int s = 0; s < E; ++s) sl[prow<true>(final_row<M, E>(t, s))] = v[s];
    __syncthreads();
    V* dst = P + c * g.S + line0 * H;
    for (int e = threadIdx.x; e < nh * H; e += blockDim.x) {
      const int ll = e / H, k = e % H;
      const V* z = slot(c, ll);
      const V Z = z[prow<true>(k == M ? 0 : k)];
      const V Zp = conjg(z[prow<true>(k == 0 ? 0 : M - k)]);
      const V s = scale(add(Z, Zp), (T)0.5);
      const V d = mul_i<-1>(mul(tw[k], scale(sub(Z, Zp), (T)0.5)));
      dst[e] = add(s, d);
    }
  }
}

// ---------------------------------------------------------------------------
// SSS z pass, fused: per z line of real coefficients (N + 2 reals, the padded real
// layout), the sin/cos inverse of the NIN inputs, the real products of FORM 0 / 2,
// and the sin/cos forward of the NOUT products, in place.  The sin/cos transforms are
// the x / y passes' algorithm along z: a quarter-step twiddle (tq = e^{-i pi m / 2N})
// on the half spectrum of the reordered line v (v_k = u_2k, v_{N-1-k} = +-u_{2k+1},
// minus for a sine series) and one real FFT of length N, the same real FFT and slot
// layout as k_z_fused.  The lines are never put back in natural order: the product of
// two reordered lines is the reordered product with the product's own sign pattern
// (sine x sine = cosine, sine x cosine = sine, and the sign flips multiply), so the
// forward transform takes it as it is.  zin / zout: bit c set = input / output c is a
// sine series along z; scl = 1 / (2N).
//   inverse: V_m = conj(w_m) (c_m - i c_{N-m}) (cosine, V_0 = c_0),
//            conj(w_m) (s_{N-m} - i s_m) (sine, V_0 = 0); real inverse FFT of V
//   forward: Z = real FFT of v; c_m = 2 scl Re(w_m Z_m) (cosine), -2 scl Im(w_m Z_m)
//            (sine), Z_m = conj(Z_{N-m}) above N/2; the two padding reals written 0
// ---------------------------------------------------------------------------
template <typename T, int NZ, int E, int FORM>
__global__ void __launch_bounds__(256) k_sss_z_fused(C<T>* __restrict__ P, Geo g, const C<T>* __restrict__ tw,
                                                     const C<T>* __restrict__ tq, int nl, int zin, int zout,
                                                     T scl) {
  typedef C<T> V;
  constexpr int N = NZ, M = NZ / 2, H = M + 1, TPL = M / E, LDS = zslot<M>();
  constexpr int NIN = z_nin(FORM), NOUT = z_nout(FORM);
  static_assert(FORM == 0 || FORM == 2 || FORM == 6,
                "SSS z pass: conservative products, with or without T, or the flux giver's products");
  extern __shared__ __align__(16) unsigned char smraw[];
  V* sm = reinterpret_cast<V*>(smraw);
  const long long nlines = (long long)g.Nx * g.Ny;
  const long long line0 = (long long)blockIdx.x * nl;
  const int nh = (int)((nlines - line0) < nl ? (nlines - line0) : nl);
  const int l = threadIdx.x / TPL, t = threadIdx.x % TPL;
  const bool live = l < nh;
  const long long lbase = (line0 + (live ? l : 0)) * H;
  auto slot = [&](int c, int ll) { return sm + (c * nl + ll) * LDS; };

  // A. inverse of each input line into its slot (real points packed two per complex)
  for (int c = 0; c < NIN; ++c) {
    const T* cl = reinterpret_cast<const T*>(P + c * g.S + lbase);  // reals 0 .. N-1 of the line
    const bool sine = (zin >> c) & 1;
    auto half = [&](int m) -> V {  // V_m, 0 <= m <= M
      if (m == 0) return mk<V>(sine ? (T)0 : cl[0], (T)0);
      const T a = sine ? cl[N - m] : cl[m], b = sine ? cl[m] : cl[N - m];
      return mul(conjg(tq[m]), mk<V>(a, -b));
    };
    V v[E];
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int k = load_row<M, E>(t, s);
      V a = mk<V>(0, 0), b = mk<V>(0, 0);
      if (live) {
        a = half(k);
        b = conjg(half(M - k));
      }
      if (k == 0) { a.y = 0; b.y = 0; }
      v[s] = add(add(a, b), mul_i<1>(mul(conjg(tw[k]), sub(a, b))));
    }
    V* sl = slot(c, l < nl ? l : 0);
    fft_regs<M, E, 1, 0, true>(v, t, sl, 1, 0, tw, 2);
#pragma unroll
    for (int s = 0; s < E; ++s) sl[prow<true>(final_row<M, E>(t, s))] = v[s];
  }
  __syncthreads();
  // B + C. per product: the product of two input lines formed as the forward FFT loads
  // it (the input slots stay intact), the FFT in the line's work slot, then the real
  // sin/cos coefficients.  NIN + 1 slots per line instead of max(NIN, NOUT) keep more
  // lines, and so more warps, per SM.
  const int lw = l < nl ? l : 0;
  for (int c = 0; c < NOUT; ++c) {
    V* sl = slot(NIN, lw);
    const V* sa = slot(z_pa(c, FORM), lw);
    const V* sb = slot(z_pb(c, FORM), lw);
    V v[E];
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int r = prow<true>(load_row<M, E>(t, s));
      v[s] = mk<V>(sa[r].x * sb[r].x, sa[r].y * sb[r].y);
    }
    __syncthreads();  // the previous product's coefficients have been read from the work slot
    fft_regs<M, E, -1, 0, true>(v, t, sl, 1, 0, tw, 2);
#pragma unroll
    for (int s = 0; s < E; ++s) sl[prow<true>(final_row<M, E>(t, s))] = v[s];
    __syncthreads();
    const bool sine = (zout >> c) & 1;
    V* dst = P + c * g.S + line0 * H;  // complex slot j holds reals 2j, 2j + 1
    for (int e = threadIdx.x; e < nh * H; e += blockDim.x) {
      const int ll = e / H, j = e % H;
      const V* z = slot(NIN, ll);
      T o[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int m = 2 * j + h;
        o[h] = (T)0;
        if (m < N) {
          const int k = m <= M ? m : N - m;
          const V Z = z[prow<true>(k == M ? 0 : k)];
          const V Zp = conjg(z[prow<true>(k == 0 ? 0 : M - k)]);
          V X = add(scale(add(Z, Zp), (T)0.5), mul_i<-1>(mul(tw[k], scale(sub(Z, Zp), (T)0.5))));
          if (m > M) X = conjg(X);
          const V w = mul(tq[m], X);
          o[h] = sine ? (T)-2 * scl * w.y : (T)2 * scl * w.x;
        }
      }
      dst[e] = mk<V>(o[0], o[1]);
    }
  }
}

// ---------------------------------------------------------------------------
// z pass, register-resident variant (M = Nz/2 <= 512): one line per group of
// TPL = M/8 consecutive lanes, 8 elements per thread.  The inverse transform
// (forward radix schedule) leaves every component's real line in registers in
// the order the forward transform with the reversed schedule expects, so the
// products are formed in registers and fed straight to the forward FFTs.  The
// real-transform pair terms X[M-k] come from the partner lane by a warp
// shuffle; shared memory holds only one exchange line per line group.
// ---------------------------------------------------------------------------
// threads per block of k_z_reg: up to six components live in registers, so it
// runs 64-thread blocks, six per SM, with a 170-register budget (FP32 only; FP64
// would spill and uses the other z kernels).  On B200 at 256^3 the 64-thread
// blocks streamed 2.88 TB/s against 2.71 for 128-thread blocks.
template <int FORM> __host__ __device__ constexpr int zreg_threads() { return 64; }

// C2R of one line held by TPL lanes (input rows k = t + s*TPL): the pair terms
// X[M-k] come from the partner lane by a warp shuffle (TPL <= 32) or straight
// from global memory (a line spread over several warps; the second read of the
// line hits L1), then the length-M inverse FFT (forward radix schedule) leaves
// the packed real line in registers
// Register layout of a line: with a first radix equal to E (powers of two), slot
// s of lane t holds row t + s*TPL on input (forward schedule) and on output
// (reversed schedule), and the pair terms X[M-k] sit in the partner lane of the
// same warp (TPL <= 32): warp shuffles.  Otherwise (a line over two warps, or a
// radix-3 schedule whose rows follow load_row / final_row) the inverse reads the
// pair terms from global memory (L1 hits) and the forward swaps them through the
// line's exchange buffer.
template <int M, int E, int TPL> __host__ __device__ constexpr bool zreg_shfl() {
  return radix_at(M, E, 0) == E && TPL <= 32;
}

// rows of a line into registers (and X[M] on lane t = 0 for the shuffle path);
// issued for every component of a line before any of them is transformed
// (rows above zkeep are zero and not read: two-thirds dealiasing along z)
template <typename T, int M, int E, int TPL>
__device__ __forceinline__ void zreg_load(const C<T>* X, bool live, int t, C<T> (&a)[E], C<T>& XM, int zkeep) {
  typedef C<T> V;
#pragma unroll
  for (int s = 0; s < E; ++s) {
    const int k = load_row<M, E>(t, s);
    a[s] = (live && k <= zkeep) ? X[k] : mk<V>(0, 0);
  }
  XM = (zreg_shfl<M, E, TPL>() && live && t == 0 && M <= zkeep) ? X[M] : mk<V>(0, 0);
}

// C2R of a loaded line (a, XM from zreg_load); the packed real line replaces a
template <typename T, int M, int E, int TPL>
__device__ __forceinline__ void zreg_inverse_loaded(const C<T>* X, bool live, int t, int partner,
                                                    const C<T>* __restrict__ tw, C<T>* xch, C<T> (&a)[E],
                                                    const C<T>& XM, int zkeep) {
  typedef C<T> V;
  V out[E];
#pragma unroll
  for (int s = 0; s < E; ++s) {
    // Z[k] = (X + Y) + i conj(w^k)(X - Y), Y = conj(X[M-k]); imag of X[0], X[M] dropped
    const int k = load_row<M, E>(t, s);
    V b;
    if constexpr (zreg_shfl<M, E, TPL>()) {
      b.x = __shfl_sync(0xffffffffu, a[E - 1 - s].x, partner);
      b.y = __shfl_sync(0xffffffffu, a[E - 1 - s].y, partner);
      if (t == 0) b = (s == 0) ? XM : a[(E - s) % E];
    } else {
      b = (live && M - k <= zkeep) ? X[M - k] : mk<V>(0, 0);
    }
    b = conjg(b);
    V x = a[s];
    if (k == 0) { x.y = 0; b.y = 0; }
    out[s] = add(add(x, b), mul_i<1>(mul(conjg(tw[k]), sub(x, b))));
  }
  fft_regs<M, E, 1, 0, true, false>(out, t, xch, 1, 0, tw, 2);
#pragma unroll
  for (int s = 0; s < E; ++s) a[s] = out[s];
}

template <typename T, int M, int E, int TPL>
__device__ __forceinline__ void zreg_inverse(const C<T>* X, bool live, int t, int partner,
                                             const C<T>* __restrict__ tw, C<T>* xch, C<T> (&out)[E]) {
  typedef C<T> V;
  V XM;
  zreg_load<T, M, E, TPL>(X, live, t, out, XM, M);
  zreg_inverse_loaded<T, M, E, TPL>(X, live, t, partner, tw, xch, out, XM, M);
}

// R2C of one packed real line in registers (reversed radix schedule, so the
// inverse's output order is its input order) and the store of its M+1 rows
template <typename T, int M, int E, int TPL>
__device__ __forceinline__ void zreg_forward_store(C<T> (&p)[E], C<T>* Xo, bool live, int t, int partner,
                                                   const C<T>* __restrict__ tw, C<T>* xch) {
  typedef C<T> V;
  constexpr bool SH = zreg_shfl<M, E, TPL>();
  fft_regs<M, E, -1, 0, true, true>(p, t, xch, 1, 0, tw, 2);
  // X[k] = 1/2 (Z + Z') - i/2 w^k (Z - Z'), Z' = conj(Z[M-k]), Z[M] = Z[0]
  if constexpr (!SH) {
#pragma unroll
    for (int s = 0; s < E; ++s) xch[prow<true>(final_row<M, E, true>(t, s))] = p[s];
    __syncthreads();
  }
#pragma unroll
  for (int s = 0; s < E; ++s) {
    const int k = final_row<M, E, true>(t, s);
    V zp;
    if constexpr (SH) {
      zp.x = __shfl_sync(0xffffffffu, p[E - 1 - s].x, partner);
      zp.y = __shfl_sync(0xffffffffu, p[E - 1 - s].y, partner);
      if (t == 0) zp = p[(E - s) % E];
    } else {
      zp = xch[prow<true>((M - k) % M)];
    }
    zp = conjg(zp);
    const V z = p[s];
    const V o = add(scale(add(z, zp), (T)0.5), mul_i<-1>(mul(tw[k], scale(sub(z, zp), (T)0.5))));
    if (live) Xo[k] = o;
    if (k == 0 && live) {
      // X[M] = Re Z[0] + Im Z[0] (Z[M] = Z[0])
      const V zc = conjg(z);
      Xo[M] = add(scale(add(z, zc), (T)0.5), mul_i<-1>(mul(tw[M], scale(sub(z, zc), (T)0.5))));
    }
  }
  if constexpr (!SH) __syncthreads();  // the exchange line is reused next
}

// blocks per SM the register z kernel is compiled for: 6 (170 registers), 3 for
// the 12-element radix-3 lines (which would spill at 170), 4 for 512-point lines
// (two warps per line, the pair terms through the exchange line; spilled at 170)
// (8 for the 4-element variant)
// (4 for the MHD and flux-giver forms, which hold six lines while they make nine products)
template <int NZ, int EZ = 0, int FORM = 0> __host__ __device__ constexpr int zreg_min_blocks() {
  return EZ == 4 ? 8 : ((NZ / 2) % 3 == 0 ? 3 : ((NZ >= 1024 || FORM == 5 || FORM == 6) ? 4 : 6));
}

// EZ = 0: 8 elements per thread, 12 for a line length with a factor 3 (radices
// 4, 2|4, 3); EZ = 4: 4 elements per thread (twice the lanes per line).
// BATCH: a line over two warps also issues every component's loads before the first
// transform (one load latency per line instead of one per component)
template <typename T, int NZ, int FORM, int EZ = 0, bool BATCH = false>
__global__ void __launch_bounds__(zreg_threads<FORM>(), zreg_min_blocks<NZ, EZ, FORM>())
    k_z_reg(C<T>* __restrict__ P, Geo g, const C<T>* __restrict__ tw, long long msP, int zkeep) {
  typedef C<T> V;
  constexpr int M = NZ / 2, H = M + 1, E = EZ ? EZ : ((M % 3 == 0) ? 12 : 8), TPL = M / E, LDX = zslot<M>();
  static_assert(TPL >= 1 && TPL <= 64, "a line spans at most two warps");
  constexpr int NIN = z_nin(FORM), NOUT = z_nout(FORM);
  static_assert(NIN <= 6, "the adjoint form runs in k_z_reg_adj");
  constexpr int LPB = zreg_threads<FORM>() / TPL;
  __shared__ __align__(16) V xch_all[LPB * LDX];
  P += blockIdx.y * msP;  // member blockIdx.y
  const int l = threadIdx.x / TPL, t = threadIdx.x % TPL;
  const int lane = threadIdx.x & 31;
  const int partner = (lane - t) + (TPL - t) % TPL;  // lane holding row M - k
  const long long nlines = (long long)g.Nx * g.Ny;
  const long long line = (long long)blockIdx.x * LPB + l;
  const bool live = line < nlines;
  V* xch = xch_all + l * LDX;

  V in[NIN][E];
  if constexpr (TPL <= 32 || BATCH) {
    // lines within a warp: every component's loads are issued before the first transform
    V XM[NIN];
#pragma unroll
    for (int c = 0; c < NIN; ++c)
      zreg_load<T, M, E, TPL>(P + c * g.S + (live ? line : 0) * H, live, t, in[c], XM[c], zkeep);
#pragma unroll
    for (int c = 0; c < NIN; ++c)
      zreg_inverse_loaded<T, M, E, TPL>(P + c * g.S + (live ? line : 0) * H, live, t, partner, tw, xch, in[c], XM[c],
                                        zkeep);
  } else {
#pragma unroll
    for (int c = 0; c < NIN; ++c) {
      V XM;
      zreg_load<T, M, E, TPL>(P + c * g.S + (live ? line : 0) * H, live, t, in[c], XM, zkeep);
      zreg_inverse_loaded<T, M, E, TPL>(P + c * g.S + (live ? line : 0) * H, live, t, partner, tw, xch, in[c], XM,
                                        zkeep);
    }
  }
  // real-space products; each complex register holds two real points
  if constexpr (FORM == 5) {
#pragma unroll
    for (int s = 0; s < E; ++s) {
      V col[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) col[c] = in[c][s];
      z_elsasser<FORM>(col);
#pragma unroll
      for (int c = 0; c < 6; ++c) in[c][s] = col[c];
    }
  }
  if (FORM == 1) {
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const V u1 = in[0][s], u2 = in[1][s], u3 = in[2][s], w1 = in[3][s], w2 = in[4][s], w3 = in[5][s];
      in[0][s] = mk<V>(u2.x * w3.x - u3.x * w2.x, u2.y * w3.y - u3.y * w2.y);
      in[1][s] = mk<V>(u3.x * w1.x - u1.x * w3.x, u3.y * w1.y - u1.y * w3.y);
      in[2][s] = mk<V>(u1.x * w2.x - u2.x * w1.x, u1.y * w2.y - u2.y * w1.y);
    }
  }
#pragma unroll
  for (int f = 0; f < NOUT; ++f) {
    V p[E];
#pragma unroll
    for (int s = 0; s < E; ++s) {
      if (FORM == 1) {
        p[s] = in[f][s];
      } else {
        const int a = z_pa(f, FORM), b = z_pb(f, FORM);
        p[s] = mk<V>(in[a][s].x * in[b][s].x, in[a][s].y * in[b][s].y);
      }
    }
    zreg_forward_store<T, M, E, TPL>(p, P + f * g.S + (live ? line : 0) * H, live, t, partner, tw, xch);
  }
}

// ---------------------------------------------------------------------------
// z pass of the adjoint right-hand side, register-resident (FP32 M <= 512, FP64 M <= 128).
// Inputs per line: u (components 0-2), w (3-5), mu (6-8); outputs mu x u into
// components 0-2 and w x mu into 3-5.  Staged so that at most six components
// are live: mu and u are inverted, mu x u is transformed and stored over u,
// then w is inverted into u's registers and w x mu is stored over w.
// ---------------------------------------------------------------------------
template <typename T, int NZ>
__global__ void __launch_bounds__(zreg_threads<3>(), sizeof(T) == 8 ? 3 : 6)
    k_z_reg_adj(C<T>* __restrict__ P, Geo g, const C<T>* __restrict__ tw, int zkeep) {
  typedef C<T> V;
  // 8 elements per thread in FP32, 4 in FP64 (six components live at once)
  constexpr int M = NZ / 2, H = M + 1, E = sizeof(T) == 8 ? 4 : 8, TPL = M / E, LDX = zslot<M>();
  static_assert(TPL >= 1 && TPL <= 64, "a line spans at most two warps");
  constexpr int LPB = zreg_threads<3>() / TPL;
  __shared__ __align__(16) V xch_all[LPB * LDX];
  const int l = threadIdx.x / TPL, t = threadIdx.x % TPL;
  const int lane = threadIdx.x & 31;
  const int partner = (lane - t) + (TPL - t) % TPL;
  const long long nlines = (long long)g.Nx * g.Ny;
  const long long line = (long long)blockIdx.x * LPB + l;
  const bool live = line < nlines;
  const long long lo = (live ? line : 0) * H;
  V* xch = xch_all + l * LDX;

  V mu[3][E], w[3][E];
#pragma unroll
  for (int c = 0; c < 3; ++c) zreg_inverse<T, M, E, TPL>(P + (6 + c) * g.S + lo, live, t, partner, tw, xch, mu[c]);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    V XM;
    zreg_load<T, M, E, TPL>(P + c * g.S + lo, live, t, w[c], XM, zkeep);
    zreg_inverse_loaded<T, M, E, TPL>(P + c * g.S + lo, live, t, partner, tw, xch, w[c], XM, zkeep);
  }
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    V p[E];
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const V a[3] = {mu[0][s], mu[1][s], mu[2][s]}, b[3] = {w[0][s], w[1][s], w[2][s]};
      p[s] = cross_pk(f, a, b);
    }
    zreg_forward_store<T, M, E, TPL>(p, P + f * g.S + lo, live, t, partner, tw, xch);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    V XM;
    zreg_load<T, M, E, TPL>(P + (3 + c) * g.S + lo, live, t, w[c], XM, zkeep);
    zreg_inverse_loaded<T, M, E, TPL>(P + (3 + c) * g.S + lo, live, t, partner, tw, xch, w[c], XM, zkeep);
  }
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    V p[E];
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const V a[3] = {w[0][s], w[1][s], w[2][s]}, b[3] = {mu[0][s], mu[1][s], mu[2][s]};
      p[s] = cross_pk(f, a, b);
    }
    zreg_forward_store<T, M, E, TPL>(p, P + (3 + f) * g.S + lo, live, t, partner, tw, xch);
  }
}

// ---------------------------------------------------------------------------
// z pass, bulk-copy variant: persistent over groups of LPB consecutive (x,y)
// lines.  A group's input lines are contiguous per component (LPB*H complex,
// 16-byte aligned), so thread 0 fetches each component with one 1-D
// cp.async.bulk into shared memory, double buffered across groups.  Each line
// is transformed by TPL = M/E lanes in registers (pair terms X[M-k] read from
// shared memory on the way in, exchanged by warp shuffles on the way out); the
// products are formed in registers and fed to the forward FFTs with the
// reversed radix schedule.  Shared memory: 2 x NIN x LPB x H input + LPB
// exchange lines.
// ---------------------------------------------------------------------------
template <typename T> __host__ __device__ constexpr int ztma_e() { return sizeof(T) == 4 ? 8 : 4; }
template <typename T, int NZ> __host__ __device__ constexpr int ztma_lpb() { return 256 / ((NZ / 2) / ztma_e<T>()); }

template <typename T, int NZ, int FORM>
__global__ void __launch_bounds__(256, 1) k_z_tma(C<T>* __restrict__ P, Geo g, const C<T>* __restrict__ tw,
                                                  int* err, long long msP, int zkeep) {
  typedef C<T> V;
  constexpr int M = NZ / 2, H = M + 1, E = ztma_e<T>(), TPL = M / E, LDX = zslot<M>();
  constexpr int LPB = ztma_lpb<T, NZ>();
  static_assert(TPL >= 1 && TPL <= 32, "line group must fit in a warp");
  constexpr int NIN = z_nin(FORM), NOUT = z_nout(FORM);
  constexpr int GRP = LPB * H;  // complex per component per group
  extern __shared__ __align__(128) unsigned char smraw_[];
  unsigned char* smraw = smraw_ + ((128 - (smem_u32(smraw_) & 127)) & 127);
  V* inb = reinterpret_cast<V*>(smraw);  // [2][NIN][GRP]
  V* xch_all = inb + 2 * NIN * GRP;      // [LPB][LDX]
  __shared__ __align__(8) uint64_t bar[2];
  const int l = threadIdx.x / TPL, t = threadIdx.x % TPL;
  const int lane = threadIdx.x & 31;
  const int partner = (lane - t) + (TPL - t) % TPL;  // lane holding row M - k
  const long long ngroups = (long long)g.Nx * g.Ny / LPB;
  V* xch = xch_all + l * LDX;
  P += blockIdx.y * msP;  // member blockIdx.y
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto issue = [&](long long grp, int slot) {
    if (grp >= ngroups) return;
    mbar_expect_tx(&bar[slot], (unsigned)(NIN * GRP * sizeof(V)));
    for (int c = 0; c < NIN; ++c)
      bulk_load(inb + (slot * NIN + c) * GRP, P + c * g.S + grp * GRP, (unsigned)(GRP * sizeof(V)), &bar[slot]);
  };
  if (threadIdx.x == 0) {
    issue(blockIdx.x, 0);
    issue(blockIdx.x + gridDim.x, 1);
  }
  int k = 0;
  for (long long grp = blockIdx.x; grp < ngroups; grp += gridDim.x, ++k) {
    // slots alternate, so slot k & 1 completes its phase (k >> 1) & 1
    const int slot = k & 1;
    const uint32_t phase = (uint32_t)(k >> 1) & 1u;
    const bool got = mbar_wait(&bar[slot], phase, err);
    if (__syncthreads_or(!got)) {
      // drain this group's copies and the next group's (other slot), each wait bounded
      if (threadIdx.x == 0) {
        mbar_wait(&bar[slot], phase, nullptr);
        if (grp + (long long)gridDim.x < ngroups) mbar_wait(&bar[slot ^ 1], (uint32_t)((k + 1) >> 1) & 1u, nullptr);
      }
      return;
    }
    V in[NIN][E];
#pragma unroll
    for (int c = 0; c < NIN; ++c) {
      const V* X = inb + (slot * NIN + c) * GRP + l * H;
#pragma unroll
      for (int s = 0; s < E; ++s) {
        // Z[k] = (X + Y) + i conj(w^k)(X - Y), Y = conj(X[M-k]); imag of X[0], X[M] dropped
        const int kk = t + s * TPL;
        V x = kk <= zkeep ? X[kk] : mk<V>(0, 0), b = M - kk <= zkeep ? conjg(X[M - kk]) : mk<V>(0, 0);
        if (kk == 0) { x.y = 0; b.y = 0; }
        in[c][s] = add(add(x, b), mul_i<1>(mul(conjg(tw[kk]), sub(x, b))));
      }
    }
    // every thread has read this slot: refill it with the group after next
    __syncthreads();
    if (threadIdx.x == 0) issue(grp + 2 * (long long)gridDim.x, slot);
#pragma unroll
    for (int c = 0; c < NIN; ++c) fft_regs<M, E, 1, 0, true, false>(in[c], t, xch, 1, 0, tw, 2);
    if (FORM == 1) {
#pragma unroll
      for (int s = 0; s < E; ++s) {
        const V u1 = in[0][s], u2 = in[1][s], u3 = in[2][s], w1 = in[3][s], w2 = in[4][s], w3 = in[5][s];
        in[0][s] = mk<V>(u2.x * w3.x - u3.x * w2.x, u2.y * w3.y - u3.y * w2.y);
        in[1][s] = mk<V>(u3.x * w1.x - u1.x * w3.x, u3.y * w1.y - u1.y * w3.y);
        in[2][s] = mk<V>(u1.x * w2.x - u2.x * w1.x, u1.y * w2.y - u2.y * w1.y);
      }
    }
    const long long line = grp * LPB + l;
#pragma unroll
    for (int f = 0; f < NOUT; ++f) {
      V p[E];
#pragma unroll
      for (int s = 0; s < E; ++s) {
        if (FORM == 1) {
          p[s] = in[f][s];
        } else {
          const int a = z_pa(f), b = z_pb(f);
          p[s] = mk<V>(in[a][s].x * in[b][s].x, in[a][s].y * in[b][s].y);
        }
      }
      fft_regs<M, E, -1, 0, true, true>(p, t, xch, 1, 0, tw, 2);
      // X[k] = 1/2 (Z + Z') - i/2 w^k (Z - Z'), Z' = conj(Z[M-k]), Z[M] = Z[0]; rows k = t + s*TPL
      V* Xo = P + f * g.S + line * H;
#pragma unroll
      for (int s = 0; s < E; ++s) {
        V zp;
        zp.x = __shfl_sync(0xffffffffu, p[E - 1 - s].x, partner);
        zp.y = __shfl_sync(0xffffffffu, p[E - 1 - s].y, partner);
        if (t == 0) zp = p[(E - s) % E];
        zp = conjg(zp);
        const int kk = t + s * TPL;
        const V z = p[s];
        Xo[kk] = add(scale(add(z, zp), (T)0.5), mul_i<-1>(mul(tw[kk], scale(sub(z, zp), (T)0.5))));
      }
      if (t == 0) {
        const V z = p[0], zp = conjg(p[0]);
        Xo[M] = add(scale(add(z, zp), (T)0.5), mul_i<-1>(mul(tw[M], scale(sub(z, zp), (T)0.5))));
      }
    }
  }
}

// ---------------------------------------------------------------------------
// forward x pass + spectral epilogue
// ---------------------------------------------------------------------------
struct StageArgs {
  void* U0;          // state (Vcopy); MODE_ADJ: the adjoint state Lam, overwritten at stage 1
  void* Uout;        // MODE_STEP: where stage 4 writes the new state (U0 for an in-place step)
  void* Ucur;        // stage field; MODE_ADJ: the next stage's cotangent lam
  void* tot;         // RK accumulator; MODE_ADJ: the adjoint accumulator
  void* nout;        // MODE_NLIN: output N (3 comps)
  const void* Ud;    // MODE_FLUX: field whose dealiased copy multiplies N
  double* bins;      // MODE_FLUX: nradii + 1 sums, then per-block partial sums, nradii + 1 per block
  const double* radii;
  int nradii;
  const void* fcube; // force cube (3 comps of (2km+1)^2 (km+1)), nullptr = no force
  int fkm;
  double nu, dt;
  int stage;         // 1..4
  int reality;       // zero the kz = Nz/2 plane at the end of stage 4
  int* err;          // set to 1 when a bounded wait gives up
  const double* ex;  // per-axis integrating factors exp(-nu dt K_i^2 / 2), FP64
  const double* ey;
  const double* ez;
  const float2* exf; // the same as FP32 (hi, lo) pairs (nullptr: split the FP64 product)
  const float2* eyf;
  const float2* ezf;
};

enum { MODE_STEP = 0, MODE_FLUX = 1, MODE_NLIN = 2, MODE_ADJ = 3 };
// MODE_FLUX: at most FLUX_MAX_BINS - 1 radii (each thread keeps one FP64 partial per sphere)
constexpr int FLUX_MAX_BINS = 64;

// Assembly of the stage's spectral vector from forward-transformed product f
// (p already scaled by 1/(Nx Ny Nz)):
//   FORM 0: N_i = sum_j i K_j F[u_i u_j]  (compute_diag_offdiag.cc:47-98)
//   FORM 1: N = -F[u x omega]
//   FORM 3: A_i + (i K x B)_i  (adjoint; B = products 0-2, A = products 3-5)
template <int FORM, typename V, typename S>
__device__ __forceinline__ void accum_product(int f, V p, S Kx, S Ky, S Kz, V& a0, V& a1, V& a2) {
  if (FORM == 0) {
    switch (f) {
      case 0: a0 = add(a0, ik(Kx, p)); break;
      case 1: a1 = add(a1, ik(Ky, p)); break;
      case 2: a2 = add(a2, ik(Kz, p)); break;
      case 3: a0 = add(a0, ik(Ky, p)); a1 = add(a1, ik(Kx, p)); break;
      case 4: a1 = add(a1, ik(Kz, p)); a2 = add(a2, ik(Ky, p)); break;
      default: a2 = add(a2, ik(Kx, p)); a0 = add(a0, ik(Kz, p)); break;
    }
  } else if (FORM == 3) {
    switch (f) {
      case 0: a1 = add(a1, ik(Kz, p)); a2 = sub(a2, ik(Ky, p)); break;
      case 1: a2 = add(a2, ik(Kx, p)); a0 = sub(a0, ik(Kz, p)); break;
      case 2: a0 = add(a0, ik(Ky, p)); a1 = sub(a1, ik(Kx, p)); break;
      case 3: a0 = add(a0, p); break;
      case 4: a1 = add(a1, p); break;
      default: a2 = add(a2, p); break;
    }
  } else {
    if (f == 0) a0 = scale(p, (S)-1);
    else if (f == 1) a1 = scale(p, (S)-1);
    else a2 = scale(p, (S)-1);
  }
}

// ey[ly] ez[lz] from the FP32 pair tables (once per column), for the FP32 step
template <typename T, int MODE>
__device__ __forceinline__ Fac<float> col_pair(const StageArgs& a, int ly, int lz) {
  if constexpr (std::is_same<T, float>::value && MODE == MODE_STEP) {
    if (a.exf) return pair_mul(a.eyf[ly], a.ezf[lz]);
  }
  return Fac<float>{1.0f, 0.0f};
}

// Per-mode epilogue of a right-hand side at spectral element (lx, ly, lz),
// linear offset `off` in a component.  N1..N3 = the assembled vector; the
// state the mode reads comes from st0[i * sstr] (U0 / Lam / the flux field)
// and st1[i * sstr] (tot / the adjoint accumulator), i = component; the
// fused x kernel passes its shared-memory state tiles, the elementwise
// epilogue kernel the global arrays.  exy = ey[ly] ez[lz] (MODE_STEP, MODE_ADJ); pexy = the
// same product from the FP32 pair tables (FP32 MODE_STEP with a.exf; see col_pair).
template <typename T, int MODE>
__device__ __forceinline__ void spec_epilogue(const Geo& g, const StageArgs& a, int lx, int ly, int lz,
                                              long long off, double exy, Fac<float> pexy, C<T> N1, C<T> N2,
                                              C<T> N3, const C<T>* st0, const C<T>* st1, long long sstr,
                                              double* sbins) {
  typedef C<T> V;
  const int kx = kfft(lx, g.Nx), ky = kfft(ly, g.Ny);
  const double Kxd = kx * g.kf[0], Kyd = ky * g.kf[1], Kzd = lz * g.kf[2];
  if (MODE == MODE_NLIN) {
    V* no = reinterpret_cast<V*>(a.nout);
    no[off] = N1; no[g.S + off] = N2; no[2 * g.S + off] = N3;
    return;
  }
  if (MODE == MODE_FLUX) {
    // contribution 2 mult Re(N . conj(D(U))) to the first sphere with |K| <= R
    if (dealias_zero(g.dealias, g.basis, lx, ly, lz, g.Nx, g.Ny, g.Nz)) return;
    const V u1 = st0[0], u2 = st0[sstr], u3 = st0[2 * sstr];
    double re = (double)N1.x * u1.x + (double)N1.y * u1.y + (double)N2.x * u2.x + (double)N2.y * u2.y +
                (double)N3.x * u3.x + (double)N3.y * u3.y;
    double mult = lz > 0 ? 1.0 : 0.5;
    if (kx == g.Nx / 2 || (ky == g.Ny / 2 && g.Ny > 1)) mult *= 2;
    const double Kmag = sqrt((Kxd * Kxd + Kyd * Kyd) + Kzd * Kzd);
    int b = 0;
    while (b < a.nradii && Kmag > a.radii[b]) ++b;
    sbins[b] += 2.0 * mult * re;  // the calling thread's own partials, in a fixed element order
    return;
  }
  if (MODE == MODE_ADJ) {
    const double eh = a.ex[lx] * exy;
    const double e1 = eh * eh;
    const T Eh = (T)eh, E1 = (T)e1;
    const bool dz = dealias_zero(g.dealias, g.basis, lx, ly, lz, g.Nx, g.Ny, g.Nz);
    const T cw = dz ? (T)0 : ((lz > 0 && 2 * lz < g.Nz) ? (T)2 : (T)1);
    V* Lm = reinterpret_cast<V*>(a.U0);
    V* lam = reinterpret_cast<V*>(a.Ucur);
    V* Ac = reinterpret_cast<V*>(a.tot);
    const V Wv[3] = {scale(N1, cw), scale(N2, cw), scale(N3, cw)};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const long long o = i * g.S + off;
      const V W = Wv[i];
      if (a.stage == 4) {
        const V Lv = st0[i * sstr];
        Ac[o] = add(scale(Lv, E1), scale(W, E1));
        lam[o] = add(scale(Lv, (T)(a.dt / 3 * eh)), scale(W, (T)(a.dt * eh)));
      } else if (a.stage == 1) {
        Lm[o] = add(st1[i * sstr], W);
      } else {
        const V Lv = st0[i * sstr], Acc = st1[i * sstr];
        Ac[o] = add(Acc, scale(W, Eh));
        lam[o] = a.stage == 3 ? add(scale(Lv, (T)(a.dt / 3 * eh)), scale(W, (T)(0.5 * a.dt)))
                              : add(scale(Lv, (T)(a.dt / 6 * e1)), scale(W, (T)(0.5 * a.dt * eh)));
      }
    }
    return;
  }
  // ---- MODE_STEP ----
  const T Kx = (T)Kxd, Ky = (T)Kyd, Kz = (T)Kzd;
  if (a.fcube) {
    const int km = a.fkm;
    if (abs(kx) <= km && abs(ky) <= km && lz <= km) {
      const V* fc = reinterpret_cast<const V*>(a.fcube);
      const int n = 2 * km + 1;
      const long long fo = ((long long)(kx + km) * n + (ky + km)) * (km + 1) + lz;
      const long long fs = (long long)n * n * (km + 1);
      N1 = sub(N1, fc[fo]); N2 = sub(N2, fc[fs + fo]); N3 = sub(N3, fc[2 * fs + fo]);  // Add_force
    }
  }
  // Leray projection: p = (i K . N)/K^2, p(0)=0; N <- -(N + i K p)
  const double K2 = (Kxd * Kxd + Kyd * Kyd) + Kzd * Kzd;
  const V div = add(add(ik(Kx, N1), ik(Ky, N2)), ik(Kz, N3));
  const V pr = (K2 > 0) ? mk<V>(div.x / (T)K2, div.y / (T)K2) : mk<V>(0, 0);
  const V Rv[3] = {scale(add(N1, ik(Kx, pr)), (T)-1), scale(add(N2, ik(Ky, pr)), (T)-1),
                   scale(add(N3, ik(Kz, pr)), (T)-1)};
  // integrating factors (FP64): E(1/2) = ex ey ez = exp(-nu dt K^2 / 2), E(1) = E(1/2)^2
  Fac<T> Feh, Fe1;
  if constexpr (std::is_same<T, float>::value) {
    if (a.exf) {
      // E(1/2) = ex ey ez and E(1) = E(1/2)^2 as FP32 pair products (about 46 bits; no
      // FP64 operation or conversion per mode)
      Feh = pair_mul(a.exf[lx], pexy);
      Fe1 = pair_mul(Feh, Feh);
    } else {
      const double eh = a.ex[lx] * exy;
      Feh = fac<T>(eh);
      Fe1 = fac<T>(eh * eh);
    }
  } else {
    const double eh = a.ex[lx] * exy;
    Feh = fac<T>(eh);
    Fe1 = fac<T>(eh * eh);
  }
  const Fac<T> Fc1 = fac<T>(a.dt), Fc2 = fac<T>(0.5 * a.dt), Fc3 = fac<T>((1.0 / 3) * a.dt),
               Fc6 = fac<T>((1.0 / 6) * a.dt);
  V* Uc = reinterpret_cast<V*>(a.Ucur);
  V* tot = reinterpret_cast<V*>(a.tot);
  const bool dz = dealias_zero(g.dealias, g.basis, lx, ly, lz, g.Nx, g.Ny, g.Nz);
  // IF-RK4 stage update (RK.cc:91-170 with Single_time_step / Compute_RK4_parts)
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const long long o = i * g.S + off;
    const V R = Rv[i];
    const V u0 = st0[i * sstr];
    if (a.stage == 1) {
      Uc[o] = rk_u1_c(dz ? mk<V>(0, 0) : u0, R, Feh, Fc2);
      tot[o] = rk_t1_c(R, Fe1, Fc6);
    } else {
      const V tt = st1[i * sstr];
      if (a.stage == 2) {
        Uc[o] = rk_u2_c(u0, R, Feh, Fc2);
        tot[o] = rk_tacc_c(tt, R, Feh, Fc3);
      } else if (a.stage == 3) {
        Uc[o] = rk_u3_c(u0, R, Feh, Fc1);
        tot[o] = rk_tacc_c(tt, R, Feh, Fc3);
      } else {
        const V un = rk_u4_c(u0, tt, R, Fe1, Fc6);
        reinterpret_cast<V*>(a.Uout)[o] = (a.reality && lz == g.Nz / 2) ? mk<V>(0, 0) : un;
        health_mark(nonfinite(un), a.err);
      }
    }
  }
}

// Persistent over column tiles.  Thread 0 streams the product fields of a tile
// through two TMA staging tiles (item = (tile, field); item i+2 is issued as
// soon as every thread has read item i), and the RK state the epilogue needs
// (U0 and tot, or the flux field) into six state tiles at tile start.
// Shared memory: 2 product tiles + 1 exchange tile + 6 state tiles (+ flux bins).
//
// FORM 3 / MODE_ADJ (discrete adjoint of the rotational stage; products
// B = F(mu x u) in fields 0-2 and A = F(w x mu) in 3-5):
//   W = D c (A + i K x B)  = the cotangent of the stage input, and with
//   L = Lam (state tiles 0-2), Acc = tot (tiles 3-5), lam = Ucur:
//   stage 4: Acc = E1 L + E1 W,  lam = dt/3 Eh L + dt Eh W
//   stage 3: Acc += Eh W,        lam = dt/3 Eh L + dt/2 W
//   stage 2: Acc += Eh W,        lam = dt/6 E1 L + dt/2 Eh W
//   stage 1: Lam = Acc + W
template <typename T, int L, int E, int CW, int FORM, int MODE>
__global__ void __launch_bounds__(CW * (L / E), 1)
    k_fwd_x(const __grid_constant__ CUtensorMap mP, const __grid_constant__ CUtensorMap mA,
            const __grid_constant__ CUtensorMap mB, Geo g, StageArgs a, const C<T>* __restrict__ tw) {
  typedef C<T> V;
  constexpr int NF = FORM == 1 ? 3 : 6;
  constexpr int TILE = L * CW, BR = L < 256 ? L : 256, UNITS = (int)sizeof(V) / 8;
  constexpr int NST = MODE == MODE_NLIN ? 0 : 6;
  extern __shared__ __align__(128) unsigned char smraw_[];
  // TMA destinations: 128-byte aligned (the launcher adds 128 bytes of slack)
  unsigned char* smraw = smraw_ + ((128 - (smem_u32(smraw_) & 127)) & 127);
  V* pst = reinterpret_cast<V*>(smraw);
  V* xch = pst + 2 * TILE;              // exchange tile, row pitch CW (L x (CW + 1) reserved)
  V* sst = xch + L * (CW + 1);
  // MODE_FLUX: per-thread FP64 partials of the spheres (thread-local, fixed element order;
  // summed over the block by block_sum and over blocks by k_bins_finish: reproducible)
  double tb[MODE == MODE_FLUX ? FLUX_MAX_BINS : 1];
  __shared__ __align__(8) uint64_t bar[3];  // product slots 0, 1; state
  const int c = threadIdx.x % CW, t = threadIdx.x / CW;
  const int inner = g.Ny * g.Hz;
  const int ntiles = (inner + CW - 1) / CW;
  const long long rstride = inner;
  const T inv = (T)(1.0 / ((double)g.Nx * g.Ny * g.Nz));
  // state tiles: [0,3) = U0 (or the flux field) from map mA, [3,6) = tot from map mB;
  // tiles [sfirst, nstate) are loaded
  const int nstate = MODE == MODE_FLUX ? 3
                     : (MODE == MODE_STEP ? (a.stage == 1 ? 3 : 6) : (MODE == MODE_ADJ ? (a.stage == 4 ? 3 : 6) : 0));
  const int sfirst = (MODE == MODE_ADJ && a.stage == 1) ? 3 : 0;

  if (MODE == MODE_FLUX)
    for (int i = 0; i <= a.nradii; ++i) tb[i] = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < 3; ++i) mbar_init(&bar[i], 1);
    fence_mbar_init();
  }
  __syncthreads();
  const long long nitems = (long long)NF * ((ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x);
  auto issue_item = [&](long long i) {
    if (i >= nitems) return;
    const int tile = blockIdx.x + (int)(i / NF) * gridDim.x, f = (int)(i % NF), slot = (int)(i & 1);
    mbar_expect_tx(&bar[slot], (unsigned)TILE * (unsigned)sizeof(V));
    for (int r0 = 0; r0 < L; r0 += BR)
      tma_load_2d(pst + slot * TILE + r0 * CW, &mP, tile * CW * UNITS, f * g.Nx + r0, &bar[slot]);
  };
  auto issue_state = [&](int tile) {
    if (nstate == 0) return;
    mbar_expect_tx(&bar[2], (unsigned)(nstate - sfirst) * TILE * (unsigned)sizeof(V));
    for (int comp = sfirst; comp < nstate; ++comp)
      for (int r0 = 0; r0 < L; r0 += BR)
        tma_load_2d(sst + comp * TILE + r0 * CW, comp < 3 ? &mA : &mB, tile * CW * UNITS, (comp % 3) * g.Nx + r0,
                    &bar[2]);
  };
  if (threadIdx.x == 0) {
    issue_item(0);
    issue_item(1);
  }
  // mbarrier phases of the two product slots and the state barrier (scalars:
  // a runtime-indexed array would live in local memory)
  uint32_t ph0 = 0, ph1 = 0, phs = 0;
  long long item = 0;
  // after a wait gave up: a second bounded wait on every copy still in flight (the
  // product items `item` and item + 1, and this tile's state tiles if pending), so no
  // bulk copy lands in the shared memory of a block that has left
  auto drain = [&](bool state_pending) {
    if (threadIdx.x != 0) return;
    for (long long i = item; i < item + 2 && i < nitems; ++i) mbar_wait(&bar[i & 1], (i & 1) ? ph1 : ph0, nullptr);
    if (state_pending) mbar_wait(&bar[2], phs, nullptr);
  };
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    if (threadIdx.x == 0) issue_state(tile);
    const int col = tile * CW + c;
    const bool ok = col < inner;
    const int ly = ok ? col / g.Hz : 0, lz = ok ? col % g.Hz : 0;
    const int ky = kfft(ly, g.Ny);
    const double Kyd = ky * g.kf[1], Kzd = lz * g.kf[2];
    const T Ky = (T)Kyd, Kz = (T)Kzd;

    V acc[3][E];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int s = 0; s < E; ++s) acc[i][s] = mk<V>(0, 0);

    for (int f = 0; f < NF; ++f, ++item) {
      const int slot = (int)(item & 1);
      const uint32_t phase = slot ? ph1 : ph0;
      const bool got = mbar_wait(&bar[slot], phase, a.err);
      if (__syncthreads_or(!got)) {
        drain(nstate > 0);
        return;
      }
      if (slot) ph1 ^= 1;
      else ph0 ^= 1;
      V v[E];
      const V* st = pst + slot * TILE + c;
#pragma unroll
      for (int s = 0; s < E; ++s) v[s] = ok ? st[load_row<L, E>(t, s) * CW] : mk<V>(0, 0);
      __syncthreads();
      if (threadIdx.x == 0) issue_item(item + 2);
      // exchange rows of pitch CW with the modelled best row swizzle (at 4
      // elements and 8 columns: bit 0 flipped by bit 2, since the first pass stores
      // rows 4 apart from neighbouring threads; 1.0x the minimum wavefronts against
      // 2.0x with the earlier padded pitch CW + 1)
      fft_regs<L, E, -1, 0, false, false, best_swk(L, E, CW, (int)sizeof(V))>(v, t, xch, CW, c, tw, 1);
#pragma unroll
      for (int s = 0; s < E; ++s) {
        const int lx = final_row<L, E>(t, s);
        const T Kx = (T)(kfft(lx, g.Nx) * g.kf[0]);
        const V p = scale(v[s], inv);
        accum_product<FORM>(f, p, Kx, Ky, Kz, acc[0][s], acc[1][s], acc[2][s]);
      }
    }
    if (nstate) {
      const bool got = mbar_wait(&bar[2], phs, a.err);
      if (__syncthreads_or(!got)) {
        drain(true);
        return;
      }
      phs ^= 1;
    }
    if (ok) {
      const double exy = (MODE == MODE_STEP || MODE == MODE_ADJ) ? a.ey[ly] * a.ez[lz] : 0.0;
      const Fac<float> pexy = col_pair<T, MODE>(a, ly, lz);
#pragma unroll
      for (int s = 0; s < E; ++s) {
        const int lx = final_row<L, E>(t, s);
        const long long off = lx * rstride + col;
        const int so = lx * CW + c;
        spec_epilogue<T, MODE>(g, a, lx, ly, lz, off, exy, pexy, acc[0][s], acc[1][s], acc[2][s], sst + so,
                               sst + 3 * TILE + so, TILE, tb);
      }
    }
    // the next tile's state load overwrites the state tiles
    __syncthreads();
  }
  if (MODE == MODE_FLUX) {
    for (int i = 0; i <= a.nradii; ++i) {
      const double v = block_sum(tb[i]);
      if (threadIdx.x == 0) a.bins[(long long)(blockIdx.x + 1) * (a.nradii + 1) + i] = v;
    }
  }
}

// ---------------------------------------------------------------------------
// Elementwise spectral epilogue, used where the fused x kernel's column tiles
// would have rows narrower than 64 bytes (FP32 and FP64 at Nx >= 512): the NF
// product fields have already been forward-transformed along x in place
// (k_strided_fft); one thread per spectral element, every array access
// coalesced.  Same arithmetic as k_fwd_x's epilogue (spec_epilogue).
// ---------------------------------------------------------------------------
template <typename T, int FORM, int MODE>
__global__ void __launch_bounds__(256) k_spec_epi(const C<T>* __restrict__ P, Geo g, StageArgs a) {
  typedef C<T> V;
  constexpr int NF = FORM == 1 ? 3 : 6;
  double tb[MODE == MODE_FLUX ? FLUX_MAX_BINS : 1];  // MODE_FLUX: per-thread sphere partials
  if (MODE == MODE_FLUX)
    for (int i = 0; i <= a.nradii; ++i) tb[i] = 0.0;
  const T inv = (T)(1.0 / ((double)g.Nx * g.Ny * g.Nz));
  const V* st0 = reinterpret_cast<const V*>(MODE == MODE_FLUX ? a.Ud : a.U0);
  const V* st1 = reinterpret_cast<const V*>(a.tot);
  // the state fields the epilogue reads at this stage (U0 / Lam / the flux field; tot)
  const bool ld0 = MODE != MODE_NLIN && !(MODE == MODE_ADJ && a.stage == 1);
  const bool ld1 = (MODE == MODE_STEP && a.stage > 1) || (MODE == MODE_ADJ && a.stage != 4);
  // two elements per thread and iteration (e and e + stride): every load of both is
  // issued before either is used, twice the loads in flight of one element at a time
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long e0 = (long long)blockIdx.x * blockDim.x + threadIdx.x; e0 < g.S; e0 += 2 * stride) {
    const bool has1 = e0 + stride < g.S;
    V pv[2][NF], s0[2][3], s1[2][3];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const long long e = e0 + j * stride;
      if (j == 0 || has1) {
#pragma unroll
        for (int f = 0; f < NF; ++f) pv[j][f] = P[f * g.S + e];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          s0[j][i] = ld0 ? st0[i * g.S + e] : mk<V>(0, 0);
          s1[j][i] = ld1 ? st1[i * g.S + e] : mk<V>(0, 0);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const long long e = e0 + j * stride;
      if (j == 1 && !has1) break;
      const int lz = (int)(e % g.Hz);
      const long long r = e / g.Hz;
      const int ly = (int)(r % g.Ny), lx = (int)(r / g.Ny);
      const T Kx = (T)(kfft(lx, g.Nx) * g.kf[0]), Ky = (T)(kfft(ly, g.Ny) * g.kf[1]), Kz = (T)(lz * g.kf[2]);
      V a0 = mk<V>(0, 0), a1 = mk<V>(0, 0), a2 = mk<V>(0, 0);
#pragma unroll
      for (int f = 0; f < NF; ++f) accum_product<FORM>(f, scale(pv[j][f], inv), Kx, Ky, Kz, a0, a1, a2);
      const double exy = (MODE == MODE_STEP || MODE == MODE_ADJ) ? a.ey[ly] * a.ez[lz] : 0.0;
      spec_epilogue<T, MODE>(g, a, lx, ly, lz, e, exy, col_pair<T, MODE>(a, ly, lz), a0, a1, a2, s0[j], s1[j], 1, tb);
    }
  }
  if (MODE == MODE_FLUX) {
    for (int i = 0; i <= a.nradii; ++i) {
      const double v = block_sum(tb[i]);
      if (threadIdx.x == 0) a.bins[(long long)(blockIdx.x + 1) * (a.nradii + 1) + i] = v;
    }
  }
}

}  // namespace ts

namespace ts {
// ---------------------------------------------------------------------------
// standalone z transforms for the Forward/Inverse_transform entry points:
// DIR=-1: real padded (Nx,Ny,Nz+2) -> spectral lines (Nx,Ny,Hz), unnormalised
// DIR=+1: spectral lines -> real padded, unnormalised; pads written as 0
// ---------------------------------------------------------------------------
template <typename T, int NZ, int E, int DIR>
__global__ void k_z_single(const C<T>* __restrict__ in, C<T>* __restrict__ out, Geo g, const C<T>* __restrict__ tw,
                           int nl, int ncomp) {
  typedef C<T> V;
  constexpr int M = NZ / 2, H = M + 1;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* bufA = reinterpret_cast<V*>(smraw);
  V* bufB = bufA + nl * H;
  const long long nlines = (long long)g.Nx * g.Ny;
  const long long line0 = (long long)blockIdx.x * nl;
  const int nh = (int)((nlines - line0) < nl ? (nlines - line0) : nl);
  const int comp = blockIdx.y;
  // real line stride = Nz+2 reals = H complex: both layouts have H complex per line
  const V* src = in + comp * g.S + line0 * H;
  V* dst = out + comp * g.S + line0 * H;
  for (int e = threadIdx.x; e < nh * H; e += blockDim.x) bufA[e] = src[e];
  __syncthreads();
  if (DIR > 0) {
    for (int e = threadIdx.x; e < nl * M; e += blockDim.x) {
      const int l = e / M, k = e % M;
      if (l >= nh) continue;
      const V* x = bufA + l * H;
      V X = x[k], Y = conjg(x[M - k]);
      if (k == 0) { X.y = 0; Y.y = 0; }
      bufB[l * H + k] = add(add(X, Y), mul_i<1>(mul(conjg(tw[k]), sub(X, Y))));
    }
    __syncthreads();
    V* r = fft_smem_lines<M, E, 1>(bufB, bufA, nl, H, tw, 2);
    for (int e = threadIdx.x; e < nh * H; e += blockDim.x) {
      const int l = e / H, k = e % H;
      dst[e] = k < M ? r[l * H + k] : mk<V>(0, 0);
    }
  } else {
    // padded real line: reals 0..NZ-1 = complex 0..M-1 of the line, pad = complex M
    V* r = fft_smem_lines<M, E, -1>(bufA, bufB, nl, H, tw, 2);
    V* o2 = (r == bufA) ? bufB : bufA;
    for (int e = threadIdx.x; e < nl * H; e += blockDim.x) {
      const int l = e / H, k = e % H;
      if (l >= nh) continue;
      const V* z = r + l * H;
      const V Z = z[k == M ? 0 : k];
      const V Zp = conjg(z[k == 0 ? 0 : M - k]);
      const V s = scale(add(Z, Zp), (T)0.5);
      const V d = mul_i<-1>(mul(tw[k], scale(sub(Z, Zp), (T)0.5)));
      o2[e] = add(s, d);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nh * H; e += blockDim.x) dst[e] = o2[e];
  }
}

template <typename T>
__global__ void k_scale_range(C<T>* A, long long n, double s) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    C<T> a = A[e];
    A[e] = mk<C<T>>((T)(a.x * s), (T)(a.y * s));
  }
}
}  // namespace ts
