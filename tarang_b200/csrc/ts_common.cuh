// Shared device building blocks for the B200 pseudo-spectral path:
// complex arithmetic, register-resident radix-2/4/8/16 DFTs, a Stockham FFT
// whose passes exchange through shared memory, and the spectral index maps of
// the FFF / SFF bases (Get_kx / Get_ky / Get_kz of
// basis/FFF/pencil/FFF_pencil_inline.h:63-111 and SFF_pencil_inline.h:63-109).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>

namespace ts {

template <typename T> struct cplx_of;
template <> struct cplx_of<float> { typedef float2 type; };
template <> struct cplx_of<double> { typedef double2 type; };
template <typename T> using C = typename cplx_of<T>::type;

template <typename V> __device__ __forceinline__ V mk(decltype(V::x) a, decltype(V::x) b) { V r; r.x = a; r.y = b; return r; }
template <typename V> __device__ __forceinline__ V add(V a, V b) { return mk<V>(a.x + b.x, a.y + b.y); }
template <typename V> __device__ __forceinline__ V sub(V a, V b) { return mk<V>(a.x - b.x, a.y - b.y); }
template <typename V> __device__ __forceinline__ V mul(V a, V b) { return mk<V>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <typename V> __device__ __forceinline__ V conjg(V a) { return mk<V>(a.x, -a.y); }
template <typename V, typename S> __device__ __forceinline__ V scale(V a, S s) { return mk<V>(a.x * s, a.y * s); }

// FP32 complex add / sub / real scale as one paired instruction (add / sub / mul
// .rn.f32x2, sm_100): each lane rounds exactly as the scalar operation, so the
// results are unchanged while the FFT butterflies (mostly adds) issue half the
// floating-point instructions
#define TS_F32X2(OP)                                                                           \
  asm("{\n\t.reg .b64 pa, pb, pr;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t" OP \
      ".rn.f32x2 pr, pa, pb;\n\tmov.b64 {%0, %1}, pr;\n\t}"                                  \
      : "=f"(r.x), "=f"(r.y)                                                                   \
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y))
template <> __device__ __forceinline__ float2 add<float2>(float2 a, float2 b) {
  float2 r;
  TS_F32X2("add");
  return r;
}
template <> __device__ __forceinline__ float2 sub<float2>(float2 a, float2 b) {
  float2 r;
  TS_F32X2("sub");
  return r;
}
template <> __device__ __forceinline__ float2 scale<float2, float>(float2 a, float s) {
  float2 r;
  const float2 b = make_float2(s, s);
  TS_F32X2("mul");
  return r;
}
#undef TS_F32X2
// multiply by +i (SIGN=+1) or -i (SIGN=-1)
template <int SIGN, typename V> __device__ __forceinline__ V mul_i(V a) {
  return SIGN > 0 ? mk<V>(-a.y, a.x) : mk<V>(a.y, -a.x);
}
// i * K * a for real K
template <typename V, typename S> __device__ __forceinline__ V ik(S K, V a) { return mk<V>(-K * a.y, K * a.x); }

// cos / sin of pi*k/16, k = 0..16 (exact mathematical constants)
__device__ __forceinline__ double c32(int k) {
  const double t[17] = {1.0, 0.98078528040323044913, 0.92387953251128675613, 0.83146961230254523708,
                        0.70710678118654752440, 0.55557023301960222474, 0.38268343236508977173,
                        0.19509032201612826785, 0.0, -0.19509032201612826785, -0.38268343236508977173,
                        -0.55557023301960222474, -0.70710678118654752440, -0.83146961230254523708,
                        -0.92387953251128675613, -0.98078528040323044913, -1.0};
  return t[k];
}
__device__ __forceinline__ double s32(int k) { return k <= 8 ? c32(8 - k) : c32(k - 8); }

// In-register DFT of size R (2, 3, 4, 8, 16, 32), natural order in and out.
// DIR = -1: forward (e^{-2 pi i jk/R}), +1: inverse (unnormalised).
template <int R, int DIR, typename V> struct DFT;
template <int DIR, typename V> struct DFT<1, DIR, V> {
  static __device__ __forceinline__ void run(V*) {}
};
template <int DIR, typename V> struct DFT<2, DIR, V> {
  static __device__ __forceinline__ void run(V* v) {
    V a = v[0];
    v[0] = add(a, v[1]);
    v[1] = sub(a, v[1]);
  }
};
template <int DIR, typename V> struct DFT<3, DIR, V> {
  // X1 = a - (b+c)/2 + DIR i (sqrt3/2)(b-c), X2 = a - (b+c)/2 - DIR i (sqrt3/2)(b-c)
  static __device__ __forceinline__ void run(V* v) {
    typedef decltype(V::x) S;
    const V a = v[0], s = add(v[1], v[2]), d = sub(v[1], v[2]);
    const V t = sub(a, scale(s, (S)0.5));
    const V u = scale(mul_i<DIR>(d), (S)0.86602540378443864676);
    v[0] = add(a, s);
    v[1] = add(t, u);
    v[2] = sub(t, u);
  }
};
template <int R, int DIR, typename V> struct DFT {
  // radix-2 decimation in time: X[k] = E[k] + w^k O[k], X[k+R/2] = E[k] - w^k O[k]
  static __device__ __forceinline__ void run(V* v) {
    typedef decltype(V::x) S;
    V e[R / 2], o[R / 2];
#pragma unroll
    for (int k = 0; k < R / 2; ++k) { e[k] = v[2 * k]; o[k] = v[2 * k + 1]; }
    DFT<R / 2, DIR, V>::run(e);
    DFT<R / 2, DIR, V>::run(o);
#pragma unroll
    for (int k = 0; k < R / 2; ++k) {
      V t;
      static_assert(R <= 32, "the twiddle table covers radices up to 32");
      const int q = k * (32 / R);  // angle pi*q/16 = 2 pi k / R
      if (k == 0) t = o[k];
      else if (4 * k == R) t = mul_i<DIR>(o[k]);
      else t = mul(o[k], mk<V>((S)c32(q), (S)(DIR * s32(q))));
      v[k] = add(e[k], t);
      v[k + R / 2] = sub(e[k], t);
    }
  }
};

// ---------------------------------------------------------------------------
// Stockham radix schedule for length L with at most E elements per thread.
// ---------------------------------------------------------------------------
// L = 2^a (or 3 * 2^a): the power-of-two part is split into passes of radix
// min(lowbit(E), remaining); a factor 3 is one final radix-3 pass.  Every radix
// divides E, so a thread always owns whole butterflies.
__host__ __device__ constexpr int lowbit(int x) { return x & (-x); }
__host__ __device__ constexpr int rad2(int L2, int E2, int p) {
  return p == 0 ? (L2 < E2 ? L2 : E2) : rad2(L2 / (L2 < E2 ? L2 : E2), E2, p - 1);
}
__host__ __device__ constexpr int np2(int L2, int E2) { return L2 <= 1 ? 0 : 1 + np2(L2 / (L2 < E2 ? L2 : E2), E2); }
__host__ __device__ constexpr int radix_at(int L, int E, int p) {
  return p < np2(lowbit(L), lowbit(E)) ? rad2(lowbit(L), lowbit(E), p) : L / lowbit(L);
}
__host__ __device__ constexpr int npasses(int L, int E) {
  return np2(lowbit(L), lowbit(E)) + (L != lowbit(L) ? 1 : 0);
}
__host__ __device__ constexpr int ns_at(int L, int E, int p) {
  // product of the radices before pass p
  return p == 0 ? 1 : radix_at(L, E, p - 1) * ns_at(L, E, p - 1);
}

// Radix schedule, optionally reversed (REV): running a transform with the
// reversed schedule makes its input order equal to the output order of the
// forward schedule and vice versa, so an inverse FFT (forward schedule) can feed
// a forward FFT (reversed schedule) straight from registers.
__host__ __device__ constexpr int radix_sched(int L, int E, int p, bool rev) {
  return rev ? radix_at(L, E, npasses(L, E) - 1 - p) : radix_at(L, E, p);
}
__host__ __device__ constexpr int ns_sched(int L, int E, int p, bool rev) {
  return p == 0 ? 1 : radix_sched(L, E, p - 1, rev) * ns_sched(L, E, p - 1, rev);
}

// Element held in register slot s after pass p: butterfly q = s / R, input/output r = s % R.
// Thread t of a line owns butterflies j = t*(E/R) + q.
// Input row  of slot (q,r) for pass p: j + r*(L/R).
// Output row of slot (q,r) for pass p: (j/Ns)*Ns*R + (j%Ns) + r*Ns.
template <int L, int E, int P, bool REV = false> struct Pass {
  static constexpr int R = radix_sched(L, E, P, REV);
  static constexpr int NS = ns_sched(L, E, P, REV);
  static_assert(E % R == 0 && L % E == 0, "every radix must divide the elements per thread");
  static constexpr int B = E / R;  // butterflies per thread
  static __device__ __forceinline__ int in_row(int t, int s) {
    const int j = t * B + s / R;
    return j + (s % R) * (L / R);
  }
  static __device__ __forceinline__ int out_row(int t, int s) {
    const int j = t * B + s / R;
    return (j / NS) * NS * R + (j % NS) + (s % R) * NS;
  }
};

// Modelled shared-memory wavefronts of the exchanges of one fft_regs<L, E> call on
// a tile of CW columns (row pitch CW, column = thread % CW, element of WB bytes),
// with the row swizzle xrow<false, k> (k = 0: none): for every store and load
// request of the first (up to) four warps, the largest number of threads whose
// element falls in one bank group of WB bytes (128-byte rows of 32 banks).
// Rows follow Pass::out_row (stores after pass p) and Pass::in_row (loads for p + 1).
__host__ __device__ constexpr int xch_wavefronts(int L, int E, int CW, int WB, int k) {
  const int units = 128 / WB;
  const int threads = CW * (L / E);
  const int nw = threads >= 128 ? 4 : (threads + 31) / 32;
  const int np = npasses(L, E);
  int R[16] = {}, NS[16] = {};
  for (int p = 0; p < np && p < 16; ++p) {
    R[p] = radix_at(L, E, p);
    NS[p] = p == 0 ? 1 : NS[p - 1] * R[p - 1];
  }
  int total = 0;
  for (int w = 0; w < nw; ++w)
    for (int p = 0; p + 1 < np; ++p)
      for (int s = 0; s < E; ++s)
        for (int side = 0; side < 2; ++side) {
          int cnt[32] = {};
          int worst = 0;
          const int pp = side == 0 ? p : p + 1;
          const int Rr = R[pp], B = E / Rr;
          for (int i = 0; i < 32; ++i) {
            const int tid = w * 32 + i;
            if (tid >= threads) break;
            const int t = tid / CW, c = tid % CW;
            const int j = t * B + s / Rr;
            int r = side == 0 ? (j / NS[pp]) * NS[pp] * Rr + (j % NS[pp]) + (s % Rr) * NS[pp]
                              : j + (s % Rr) * (L / Rr);
            if (k > 0) r ^= (r >> k) & 1;
            const int g = (r * CW + c) % units;
            if (++cnt[g] > worst) worst = cnt[g];
          }
          total += worst;
        }
  return total;
}
// the row swizzle with the fewest modelled wavefronts (0 unless it saves at least 5 %)
__host__ __device__ constexpr int best_swk(int L, int E, int CW, int WB) {
  const int base = xch_wavefronts(L, E, CW, WB, 0);
  int best = base, bk = 0;
  for (int k = 1; k <= 6 && (2 << k) <= L; ++k) {
    const int v = xch_wavefronts(L, E, CW, WB, k);
    if (v < best) {
      best = v;
      bk = k;
    }
  }
  return 20 * best <= 19 * base ? bk : 0;
}

// Row of register slot s at load time (first pass input) and after the last pass.
template <int L, int E, bool REV = false> __device__ __forceinline__ int load_row(int t, int s) {
  return Pass<L, E, 0, REV>::in_row(t, s);
}
template <int L, int E, bool REV = false> __device__ __forceinline__ int final_row(int t, int s) {
  return Pass<L, E, npasses(L, E) - 1, REV>::out_row(t, s);
}

// Butterflies of pass P on the registers (twiddle then DFT_R).  tw: table of
// Ltab entries exp(-2 pi i m / Ltab), Ltab = L * tws (tws = table stride).
template <int L, int E, int P, int DIR, bool REV = false, typename V>
__device__ __forceinline__ void pass_compute(V* v, int t, const V* __restrict__ tw, int tws) {
  typedef Pass<L, E, P, REV> PP;
  constexpr int R = PP::R, NS = PP::NS;
#pragma unroll
  for (int q = 0; q < PP::B; ++q) {
    V* b = v + q * R;
    if (NS > 1) {
      const int j = t * PP::B + q;
      const int k = j % NS;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        V w = tw[(r * k * (L / (NS * R))) * tws];
        if (DIR > 0) w.y = -w.y;
        b[r] = mul(b[r], w);
      }
    }
    DFT<R, DIR, V>::run(b);
  }
}

// padded shared-memory row index: one spare slot every 16 complex values keeps
// the threads of a line (consecutive rows E apart) on distinct banks
template <bool PAD> __device__ __forceinline__ int prow(int r) { return PAD ? r + (r >> 4) : r; }
// exchange row of logical row r: padded (PAD), or with bit 0 flipped by bit SWK
// (SWK > 0; a permutation of the rows) so that rows 2^SWK apart, which one
// radix pass stores from neighbouring threads, land on different bank pairs
template <bool PAD, int SWK> __device__ __forceinline__ int xrow(int r) {
  return SWK > 0 ? (r ^ ((r >> SWK) & 1)) : prow<PAD>(r);
}

// Full FFT of one line whose E-element slice per thread is in registers (loaded
// in load_row order); the line's L elements are exchanged through shared memory
// `sm` addressed as sm[row*rs + cs] (caller supplies the per-thread column
// offset cs and the row stride rs).  All threads of the block must call it.
// On return v[s] holds output row final_row(t, s).
template <int L, int E, int DIR, int P = 0, bool PAD = false, bool REV = false, int SWK = 0, typename V>
__device__ __forceinline__ void fft_regs(V* v, int t, V* sm, int rs, int cs, const V* __restrict__ tw, int tws) {
  pass_compute<L, E, P, DIR, REV>(v, t, tw, tws);
  if constexpr (P + 1 < npasses(L, E)) {
#pragma unroll
    for (int s = 0; s < E; ++s) sm[xrow<PAD, SWK>(Pass<L, E, P, REV>::out_row(t, s)) * rs + cs] = v[s];
    __syncthreads();
#pragma unroll
    for (int s = 0; s < E; ++s) v[s] = sm[xrow<PAD, SWK>(Pass<L, E, P + 1, REV>::in_row(t, s)) * rs + cs];
    __syncthreads();
    fft_regs<L, E, DIR, P + 1, PAD, REV, SWK>(v, t, sm, rs, cs, tw, tws);
  }
}

// ---------------------------------------------------------------------------
// Shared-memory line FFTs with all threads of the block cooperating
// (used by the contiguous-axis kernels, where lines are short and the real
// transform pre/post-processing needs element pairs k, M-k).
// Stockham ping-pong: reads src, writes dst, swaps; returns the buffer that
// holds the result.  Lines are at src + l*ld.
// ---------------------------------------------------------------------------
template <int L, int E, int DIR, int P = 0, typename V>
__device__ V* fft_smem_lines(V* src, V* dst, int nlines, int ld, const V* __restrict__ tw, int tws) {
  typedef Pass<L, E, P> PP;
  constexpr int R = PP::R, NS = PP::NS;
  const int nb = nlines * (L / R);
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    const int line = b / (L / R);
    const int j = b % (L / R);
    const int k = j % NS;
    V v[R];
    const V* s = src + line * ld;
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = s[j + r * (L / R)];
    if (NS > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        V w = tw[(r * k * (L / (NS * R))) * tws];
        if (DIR > 0) w.y = -w.y;
        v[r] = mul(v[r], w);
      }
    }
    DFT<R, DIR, V>::run(v);
    V* d = dst + line * ld;
    const int o = (j / NS) * NS * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) d[o + r * NS] = v[r];
  }
  __syncthreads();
  if constexpr (P + 1 < npasses(L, E)) return fft_smem_lines<L, E, DIR, P + 1>(dst, src, nlines, ld, tw, tws);
  else return dst;
}

// ---------------------------------------------------------------------------
// asynchronous global -> shared copies (cp.async): each thread stages the
// elements it will read itself, so a per-thread wait_group is enough.
// ---------------------------------------------------------------------------
template <typename V> __device__ __forceinline__ void cp_async(V* dst, const V* src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(V) == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
  else asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// ---------------------------------------------------------------------------
// Index maps
// ---------------------------------------------------------------------------
__device__ __forceinline__ int kfft(int l, int N) { return l <= N / 2 ? l : l - N; }

// Dealias predicates: true when the mode is ZEROED.
// mode 1 = reference corner box (FFF_pencil_basic.cc:87-90 / SFF_pencil_basic.cc:94-97),
// mode 2 = two-thirds cube.
// SSS (real coefficients, lzr = real z index < Nz): SSS_PENCIL::Dealias zeroes
// lx >= 2Nx/3+1, ly >= 2Ny/3+1, lzr >= Nz/3 (SSS_pencil_basic.cc:129-134); two-thirds
// zeroes 3 k > 2 N on any axis
__device__ __forceinline__ bool sss_dealias_zero(int mode, int lx, int ly, int lzr, int Nx, int Ny, int Nz) {
  if (mode == 1) return lx >= 2 * Nx / 3 + 1 && ly >= 2 * Ny / 3 + 1 && lzr >= Nz / 3;
  if (mode == 2) return 3 * lx > 2 * Nx || 3 * ly > 2 * Ny || 3 * lzr > 2 * Nz;
  return false;
}

__device__ __forceinline__ bool dealias_zero(int mode, int basis, int lx, int ly, int lz, int Nx, int Ny, int Nz) {
  if (mode == 1) {
    bool mx = basis == 0 ? (lx >= Nx / 3 + 1 && lx <= 2 * Nx / 3 - 1) : (lx >= 2 * Nx / 3 + 1);
    // SSF (sin/cos along y too): ly >= 2Ny/3 + 1 (SSF_pencil_basic.cc:103-106)
    bool my = basis == 2 ? (ly >= 2 * Ny / 3 + 1) : (ly >= Ny / 3 + 1 && ly <= 2 * Ny / 3 - 1);
    bool mz = lz >= Nz / 3 + 1 && lz <= Nz / 2;
    return mx && my && mz;
  }
  if (mode == 2) {
    int kx = basis == 0 ? kfft(lx, Nx) : lx;
    int ky = kfft(ly, Ny);
    bool bx = basis == 0 ? (3 * abs(kx) > Nx) : (3 * kx > 2 * Nx);
    bool by = basis == 2 ? (3 * ly > 2 * Ny) : (3 * abs(ky) > Ny);
    return bx || by || (3 * lz > Nz);
  }
  return false;
}

// ---------------------------------------------------------------------------
// FP64 reductions in a fixed order (butterfly within a warp, warps in index order),
// so that every sum built from them is reproducible bit for bit
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// every thread of the block must call it; thread 0 (warp 0) holds the sum
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[32];
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  v = (threadIdx.x < (blockDim.x + 31) / 32) ? red[threadIdx.x] : 0.0;
  if (w == 0) v = warp_sum(v);
  return v;
}

// out[i] = sum over b = 0..nblocks-1 of part[b * n + i], b in increasing order:
// the fixed-order final sum of per-block partial bins
static __global__ void k_bins_finish(const double* __restrict__ part, int nblocks, int n, double* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0;
    for (int b = 0; b < nblocks; ++b) s += part[(long long)b * n + i];
    out[i] = s;
  }
}

// ---------------------------------------------------------------------------
// health word of a plan (or of one ensemble member): bit HEALTH_TIMEOUT = a bounded
// wait gave up, bit HEALTH_NONFINITE = a step wrote a NaN or Inf into the state
// (the reference aborts on a NaN total energy, Ifluid_main.cc:127-129)
// ---------------------------------------------------------------------------
constexpr int HEALTH_TIMEOUT = 1, HEALTH_NONFINITE = 2;
__device__ __forceinline__ void health_mark(bool bad, int* hw) {
  if (bad && hw && !(*(volatile int*)hw & HEALTH_NONFINITE)) atomicOr(hw, HEALTH_NONFINITE);
}
template <typename V> __device__ __forceinline__ bool nonfinite(const V& v) { return !(isfinite(v.x) && isfinite(v.y)); }

// ---------------------------------------------------------------------------
// IF-RK4 stage arithmetic of one mode (RK.cc:91-170: Single_time_step,
// Compute_RK4_parts).  eh = E(1/2) = exp(-nu dt K^2 / 2), e1 = E(1) (from FP64 tables);
// c = the dt factor.  Each factor reaches the arithmetic as a Fac: in FP64 the value; in
// FP32 the pair hi = fl32(x), lo = fl32(x - hi), applied as a x = fma(a, hi, a lo), so
// the factor carries about 48 bits.  A factor rounded to FP32 (eh or e1 to 24 bits) would
// scale a mode by the same wrong amount every step, a bias that grows linearly with the
// step count.  The state update u0 E(1) + (tot + R dt/6) folds the small terms into one
// fma chain, fma(u0, e1.hi, fma(u0, e1.lo, tot + R dt/6)), so the decay u0 (E(1) - 1),
// often below half an FP32 ulp of u0, reaches the single final rounding instead of being
// rounded away (which would bias slowly decaying modes towards no decay).  No FP64
// operation and no FP64 <-> FP32 conversion runs per component.
// ---------------------------------------------------------------------------
template <typename S> struct Fac;
template <> struct Fac<double> { double v; };
template <> struct Fac<float> { float hi, lo; };
template <typename S> __device__ __forceinline__ Fac<S> fac(double x);
template <> __device__ __forceinline__ Fac<double> fac<double>(double x) { return {x}; }
template <> __device__ __forceinline__ Fac<float> fac<float>(double x) {
  const float h = (float)x;
  return {h, (float)(x - (double)h)};
}
__device__ __forceinline__ float fmulx(float a, Fac<float> f) { return fmaf(a, f.hi, a * f.lo); }
// product of two pairs (hi + lo): the rounded product of the high parts plus its exact
// rounding error (fma) and the cross terms; the sum hi + lo carries about 46 bits
__device__ __forceinline__ Fac<float> pair_mul(Fac<float> a, Fac<float> b) {
  const float h = a.hi * b.hi;
  return {h, fmaf(a.lo, b.hi, fmaf(a.hi, b.lo, fmaf(a.hi, b.hi, -h)))};
}
__device__ __forceinline__ Fac<float> pair_mul(float2 a, Fac<float> b) { return pair_mul(Fac<float>{a.x, a.y}, b); }
__device__ __forceinline__ Fac<float> pair_mul(float2 a, float2 b) { return pair_mul(Fac<float>{a.x, a.y}, Fac<float>{b.x, b.y}); }
// a x + b, the low part of x folded into b before the final fma
__device__ __forceinline__ float fmaddx(float a, Fac<float> f, float b) { return fmaf(a, f.hi, fmaf(a, f.lo, b)); }

// FP64: the plain expressions
__device__ __forceinline__ double rk_u1(double u0, double R, Fac<double> eh, Fac<double> c) {
  return (u0 + R * c.v) * eh.v;               // (u0 + R dt/2) E(1/2)
}
__device__ __forceinline__ double rk_t1(double R, Fac<double> e1, Fac<double> c) { return (R * e1.v) * c.v; }
__device__ __forceinline__ double rk_u2(double u0, double R, Fac<double> eh, Fac<double> c) {
  return u0 * eh.v + R * c.v;                 // u0 E(1/2) + R dt/2
}
__device__ __forceinline__ double rk_tacc(double tt, double R, Fac<double> eh, Fac<double> c) {
  return tt + (R * eh.v) * c.v;               // tot + (R E(1/2)) dt/3
}
__device__ __forceinline__ double rk_u3(double u0, double R, Fac<double> eh, Fac<double> c) {
  return (u0 * eh.v + R * c.v) * eh.v;        // (u0 E(1/2) + R dt) E(1/2)
}
__device__ __forceinline__ double rk_u4(double u0, double tt, double R, Fac<double> e1, Fac<double> c) {
  return u0 * e1.v + (tt + R * c.v);          // u0 E(1) + (tot + R dt/6)
}
// FP32: exact factors, small terms folded before the last rounding
__device__ __forceinline__ float rk_u1(float u0, float R, Fac<float> eh, Fac<float> c) {
  return fmulx(fmaf(R, c.hi, fmaf(R, c.lo, u0)), eh);
}
__device__ __forceinline__ float rk_t1(float R, Fac<float> e1, Fac<float> c) { return fmulx(fmulx(R, e1), c); }
__device__ __forceinline__ float rk_u2(float u0, float R, Fac<float> eh, Fac<float> c) {
  return fmaddx(u0, eh, fmulx(R, c));
}
__device__ __forceinline__ float rk_tacc(float tt, float R, Fac<float> eh, Fac<float> c) {
  return tt + fmulx(fmulx(R, eh), c);
}
__device__ __forceinline__ float rk_u3(float u0, float R, Fac<float> eh, Fac<float> c) {
  return fmulx(fmaddx(u0, eh, fmulx(R, c)), eh);
}
__device__ __forceinline__ float rk_u4(float u0, float tt, float R, Fac<float> e1, Fac<float> c) {
  return fmaddx(u0, e1, tt + fmulx(R, c));
}
#define TS_RK_CPLX(NAME, ...) \
  template <typename V, typename F> __device__ __forceinline__ V NAME##_c(__VA_ARGS__)
TS_RK_CPLX(rk_u1, V u0, V R, F eh, F c) { return mk<V>(rk_u1(u0.x, R.x, eh, c), rk_u1(u0.y, R.y, eh, c)); }
TS_RK_CPLX(rk_t1, V R, F e1, F c) { return mk<V>(rk_t1(R.x, e1, c), rk_t1(R.y, e1, c)); }
TS_RK_CPLX(rk_u2, V u0, V R, F eh, F c) { return mk<V>(rk_u2(u0.x, R.x, eh, c), rk_u2(u0.y, R.y, eh, c)); }
TS_RK_CPLX(rk_tacc, V tt, V R, F eh, F c) { return mk<V>(rk_tacc(tt.x, R.x, eh, c), rk_tacc(tt.y, R.y, eh, c)); }
TS_RK_CPLX(rk_u3, V u0, V R, F eh, F c) { return mk<V>(rk_u3(u0.x, R.x, eh, c), rk_u3(u0.y, R.y, eh, c)); }
TS_RK_CPLX(rk_u4, V u0, V tt, V R, F e1, F c) {
  return mk<V>(rk_u4(u0.x, tt.x, R.x, e1, c), rk_u4(u0.y, tt.y, R.y, e1, c));
}
#undef TS_RK_CPLX

}  // namespace ts
