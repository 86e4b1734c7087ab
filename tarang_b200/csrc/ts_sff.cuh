// SFF (sin/cos x Fourier x Fourier) kernels of the Boussinesq IF-RK4 step.
//
// Along x the fields are sine (S) or cosine (C) series on the staggered grid
// x_n = (n+1/2) Lx/Nx with modes m = 0..Nx-1 stored at lx = m
// (SFF_pencil_inline.h:63; sine m = 0 unused, the m = Nx sine term dropped):
//   C:  u_n = c_0 + 2 sum_m c_m cos(pi m (2n+1)/(2N)),  c_m = (1/N) sum_n u_n cos(...)
//   S:  u_n =       2 sum_m c_m sin(pi m (2n+1)/(2N)),  c_m = (1/N) sum_n u_n sin(...)
// Each x transform is one N-point complex FFT with O(N) pre/post-processing
// (the reordering method for the type-II/III cosine transform, applied to the
// complex data left by the y and z Fourier passes; the transforms are
// real-linear, so real and imaginary parts ride in one complex FFT):
//   forward:  v_k = u_{2k} (k < N/2), v_k = +-u_{2(N-1-k)+1} (k >= N/2, minus for S),
//             Z = FFT_N(v), w_m = e^{-i pi m/(2N)},
//             C: c_m = (1/2N) (w_m Z_m + conj(w_m) Z_{N-m}),
//             S: c_m = (i/2N) (w_m Z_m - conj(w_m) Z_{N-m})        (Z_N = Z_0)
//   inverse:  C: V_m = conj(w_m) (c_m - i c_{N-m}),  S: V_m = conj(w_m) (s_{N-m} - i s_m),
//             V_0 = c_0 (C) or 0 (S), c_N = 0; v = inverse FFT_N(V) (unscaled);
//             u_{2k} = v_k, u_{2k+1} = v_{N-1-k}, and u_n *= (-1)^n for S.
// Parities (global/Global.cc:137-145, sincostr "SFF"): u1 S, u2 C, u3 C, T S;
// products u1u1 u2u2 u3u3 C, u1u2 S, u2u3 C, u3u1 S, u1T C, u2T S, u3T S.
// x derivative of a C series is -Kx (result S), of an S series +Kx (result C)
// (SFF_pencil_tr.cc:77-106).
#pragma once
#include "ts_fff.cuh"

namespace ts {

struct SffArgs {
  const void* U0;   // velocity state (3 comps), updated at stage 4
  const void* T0;   // temperature state (1 comp), updated at stage 4
  void* Ucur;       // stage fields: 3 velocity comps then T
  void* tot;        // RK accumulators: 3 velocity comps then T
  const void* U1in; // stage input u1 and T (un-dealiased: the RBC force uses them)
  const void* Tin;
  const double* eu[3];  // exp(-nu dt K_i^2 / 2) per axis
  const double* et[3];  // exp(-kappa dt K_i^2 / 2) per axis
  double dt;
  int stage;
  int reality;
  // batched members (blockIdx.y = member): member strides of each array in
  // complex elements, and of the integrating-factor tables in doubles (0 for one run)
  long long msU0, msT0, msUcur, msTot, msU1in, msTin, msP;
  long long mtab;
  // buoyancy coefficients U.Force1 = cu T, T.Force = cT U.V1 (compute_force_RBC.cc:104-150)
  double cu, cT;
  // health words, one per member (the member index of the batch): a NaN or Inf written
  // into the state at stage 4 sets HEALTH_NONFINITE (nullptr: no check)
  int* health;
  // Pr_option PRZERO (slave = 1: T = U.V1 / K^2) or PRINFTY (slave = 2: U = vs P(T x) / K^2,
  // vs = sqrt(Ra) or Ra); 0: both fields advanced (SFF epilogue only)
  int slave;
  double vs;
};

// blocks per SM the SFF x kernels are compiled for: power-of-two lengths (8
// elements per thread) stay at or under 128 registers per thread (16+ warps per
// SM); the 12-element mixed-radix variants need the larger register budget
// (the FP64 6-element mixed-radix forward kernel: 3 blocks of 128 threads, a
// 170-register budget)
__host__ __device__ constexpr int sff_min_blocks(int threads, int e) {
  return e > 8 ? (threads <= 256 ? 2 : 1) : (e == 6 ? (threads <= 128 ? 3 : 1) : (threads <= 256 ? 512 / threads : 1));
}

// parity of product field f: true = sine
__host__ __device__ constexpr bool sff_prod_sine(int f) { return f == 3 || f == 5 || f == 7 || f == 8; }

// ---------------------------------------------------------------------------
// inverse x pass: W_f = inverse sin/cos transform of D(field_f), f = u1,u2,u3,T.
// tq: 4N entries exp(-2 pi i j/(4N)) (every fourth entry is the N-point FFT table).
// The four fields' columns stream through two cp.async staging tiles (field f+2
// is in flight while f is transformed); the pre-processing pairs rows m and
// N - m, so a barrier follows each tile's arrival.
// Shared memory: exchange tile + 2 staging tiles of N x CW complex.
// ---------------------------------------------------------------------------
template <typename T, int N, int E, int CW>
__global__ void __launch_bounds__(CW * (N / E), sff_min_blocks(CW * (N / E), E))
    k_sff_inv_x(const C<T>* __restrict__ U, const C<T>* __restrict__ Tf, C<T>* __restrict__ W, Geo g,
                const C<T>* __restrict__ tq, long long msU, long long msT, long long msW) {
  typedef C<T> V;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* xch = reinterpret_cast<V*>(smraw);
  V* stage = xch + N * CW;
  // member blockIdx.y of a batch (strides 0 for one run)
  U += blockIdx.y * msU;
  Tf += blockIdx.y * msT;
  W += blockIdx.y * msW;
  const int c = threadIdx.x % CW, t = threadIdx.x / CW;
  const int inner = g.Ny * g.Hz;
  const int col = blockIdx.x * CW + c;
  const bool ok = col < inner;
  const int ly = ok ? col / g.Hz : 0, lz = ok ? col % g.Hz : 0;
  const long long rstride = inner;
  auto issue = [&](int f, int buf) {
    if (f < 4 && ok) {
      const V* src = (f < 3 ? U + f * g.S : Tf) + col;
#pragma unroll
      for (int s = 0; s < E; ++s) {
        const int m = load_row<N, E>(t, s);
        cp_async(stage + (buf * N + m) * CW + c, src + m * rstride);
      }
    }
    cp_async_commit();
  };
  issue(0, 0);
  issue(1, 1);
  for (int f = 0; f < 4; ++f) {
    const bool sine = f == 0 || f == 3;
    const int buf = f & 1;
    cp_async_wait<1>();
    __syncthreads();  // every thread's rows of field f have arrived
    const V* st = stage + buf * N * CW + c;
    // coefficient q of the (dealiased) series; 0 outside 1..N-1
    auto coef = [&](int q) -> V {
      if (!ok || q <= 0 || q >= N || dealias_zero(g.dealias, 1, q, ly, lz, g.Nx, g.Ny, g.Nz)) return mk<V>(0, 0);
      return st[q * CW];
    };
    V v[E];
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int m = load_row<N, E>(t, s);
      V z;
      if (m == 0) {
        // cosine: V_0 = c_0; sine: V_0 = 0
        z = (!sine && ok && !dealias_zero(g.dealias, 1, 0, ly, lz, g.Nx, g.Ny, g.Nz)) ? st[0] : mk<V>(0, 0);
      } else {
        const V p = sine ? coef(N - m) : coef(m), q = sine ? coef(m) : coef(N - m);
        z = mul(conjg(tq[m]), sub(p, mul_i<1>(q)));
      }
      v[s] = z;
    }
    __syncthreads();  // every thread has read tile buf: field f + 2 may overwrite it
    issue(f + 2, buf);
    fft_regs<N, E, 1, 0, false, false, best_swk(N, E, CW, (int)sizeof(V))>(v, t, xch, CW, c, tq, 4);
    if (ok) {
      V* d = W + f * g.S + col;
#pragma unroll
      for (int s = 0; s < E; ++s) {
        const int k = final_row<N, E>(t, s);
        const int n = k < N / 2 ? 2 * k : 2 * (N - 1 - k) + 1;
        d[n * rstride] = (sine && (n & 1)) ? scale(v[s], (T)-1) : v[s];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Standalone sin/cos transform along x, in place on component blockIdx.y of A
// (spectral layout: rows lx, columns ly*Hz + lz): the x part of
// SFF_PENCIL::Forward_transform / Inverse_transform (SFF_pencil_tr.cc:43-68)
// for one parity (sine != 0: S, else C).
// DIR = -1: rows hold real-space x points (after the z and y transforms); the
//           coefficients c_m * (2N * scl) replace them (scl carries the y, z
//           normalisation as well).
// DIR = +1: rows hold coefficients; the unscaled synthesis replaces them.
// Every thread loads its rows before the first barrier inside the FFT and
// stores after the last one, so the in-place update needs no extra buffer.
// ---------------------------------------------------------------------------
// Planes: the nplanes planes of g.S elements (components, or the x-planes of a y pass)
// are one run of nplanes * Ny * Hz columns, so no column tile straddles idle columns
// at a plane's end.  Batches: blockIdx.z = b runs the pass on the planes at
// A + b * bstride, whose parity is bit b of smask (one batch: b = 0, smask = 0 or 1).
template <typename T, int N, int E, int CW, int DIR>
__global__ void __launch_bounds__(CW * (N / E), sff_min_blocks(CW * (N / E), E))
    k_sff_x(C<T>* __restrict__ A, Geo g, const C<T>* __restrict__ tq, int smask, double scl, long long bstride,
            int nplanes) {
  typedef C<T> V;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* xch = reinterpret_cast<V*>(smraw);
  const int c = threadIdx.x % CW, t = threadIdx.x / CW;
  const int inner = g.Ny * g.Hz;
  const int col = blockIdx.x * CW + c;  // plane col / inner, column col % inner
  const bool ok = col < nplanes * inner;
  const long long rstride = inner;
  const int sine = (smask >> blockIdx.z) & 1;
  const int pl = ok ? col / inner : 0, cc = ok ? col % inner : 0;
  V* a = A + (long long)pl * g.S + blockIdx.z * bstride + cc;
  V v[E];
  if (DIR < 0) {
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int k = load_row<N, E>(t, s);
      V x = ok ? a[(k < N / 2 ? 2 * k : 2 * (N - 1 - k) + 1) * rstride] : mk<V>(0, 0);
      if (sine && k >= N / 2) x = scale(x, (T)-1);
      v[s] = x;
    }
    fft_regs<N, E, -1, 0, false, false, best_swk(N, E, CW, (int)sizeof(V))>(v, t, xch, CW, c, tq, 4);
#pragma unroll
    for (int s = 0; s < E; ++s) xch[final_row<N, E>(t, s) * CW + c] = v[s];
    __syncthreads();
    V zr[E];
#pragma unroll
    for (int s = 0; s < E; ++s) zr[s] = xch[((N - final_row<N, E>(t, s)) % N) * CW + c];
    if (ok) {
#pragma unroll
      for (int s = 0; s < E; ++s) {
        const int m = final_row<N, E>(t, s);
        const V wz = mul(tq[m], v[s]), wzr = mul(conjg(tq[m]), zr[s]);
        a[m * rstride] = sine ? mul_i<1>(scale(sub(wz, wzr), (T)scl)) : scale(add(wz, wzr), (T)scl);
      }
    }
  } else {
    auto coef = [&](int q) -> V { return (ok && q > 0 && q < N) ? a[q * rstride] : mk<V>(0, 0); };
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int m = load_row<N, E>(t, s);
      V z;
      if (m == 0) {
        z = (!sine && ok) ? a[0] : mk<V>(0, 0);
      } else {
        const V p = sine ? coef(N - m) : coef(m), q = sine ? coef(m) : coef(N - m);
        z = mul(conjg(tq[m]), sub(p, mul_i<1>(q)));
      }
      v[s] = z;
    }
    fft_regs<N, E, 1, 0, false, false, best_swk(N, E, CW, (int)sizeof(V))>(v, t, xch, CW, c, tq, 4);
    if (ok) {
#pragma unroll
      for (int s = 0; s < E; ++s) {
        const int k = final_row<N, E>(t, s);
        const int n = k < N / 2 ? 2 * k : 2 * (N - 1 - k) + 1;
        a[n * rstride] = (sine && (n & 1)) ? scale(v[s], (T)-1) : v[s];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Boussinesq epilogue at spectral element (m, ly, lz) of batch member mb (offset
// `off` in a component): force U.F1 = cu T, T.F = cT U.V1 of the stage input, SFF
// projection, IF-RK4 stage update of U (nu) and T (kappa).  N1..N3, NT = the
// assembled nonlinear terms (before the force).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void sff_epilogue(const Geo& g, const SffArgs& a, long long mb, int m, int ly, int lz,
                                             long long off, C<T> N1, C<T> N2, C<T> N3, C<T> NT) {
  typedef C<T> V;
  const V* U0 = reinterpret_cast<const V*>(a.U0) + mb * a.msU0;
  const V* T0 = reinterpret_cast<const V*>(a.T0) + mb * a.msT0;
  V* Uc = reinterpret_cast<V*>(a.Ucur) + mb * a.msUcur;
  V* tot = reinterpret_cast<V*>(a.tot) + mb * a.msTot;
  const V* U1in = reinterpret_cast<const V*>(a.U1in) + mb * a.msU1in;
  const V* Tin = reinterpret_cast<const V*>(a.Tin) + mb * a.msTin;
  const long long tb = mb * a.mtab;
  const double Kxd = m * g.kf[0], Kyd = kfft(ly, g.Ny) * g.kf[1], Kzd = lz * g.kf[2];
  const T Kx = (T)Kxd, Ky = (T)Kyd, Kz = (T)Kzd;
  // force (compute_force_RBC.cc:104-150): U.F1 = cu T, T.F = cT U.V1 of the stage input
  // (cu = cT = 1 for PRLARGE / ULARGE); nlin -= F
  N1 = sub(N1, scale(Tin[off], (T)a.cu));
  NT = sub(NT, scale(U1in[off], (T)a.cT));
  // projection with SFF parities: div = +Kx N1 + i Ky N2 + i Kz N3; grad_x p = -Kx p
  const double K2 = (Kxd * Kxd + Kyd * Kyd) + Kzd * Kzd;
  const V div = add(add(scale(N1, Kx), ik(Ky, N2)), ik(Kz, N3));
  const V pr = (K2 > 0) ? mk<V>(div.x / (T)K2, div.y / (T)K2) : mk<V>(0, 0);
  N1 = add(N1, scale(pr, -Kx));
  N2 = add(N2, ik(Ky, pr));
  N3 = add(N3, ik(Kz, pr));
  const V Rv[4] = {scale(N1, (T)-1), scale(N2, (T)-1), scale(N3, (T)-1), scale(NT, (T)-1)};
  const double ehu = a.eu[0][tb + m] * a.eu[1][tb + ly] * a.eu[2][tb + lz];
  const double eht = a.et[0][tb + m] * a.et[1][tb + ly] * a.et[2][tb + lz];
  const Fac<T> Fhu = fac<T>(ehu), F1u = fac<T>(ehu * ehu), Fht = fac<T>(eht), F1t = fac<T>(eht * eht);
  const Fac<T> Fc1 = fac<T>(a.dt), Fc2 = fac<T>(0.5 * a.dt), Fc3 = fac<T>((1.0 / 3) * a.dt),
               Fc6 = fac<T>((1.0 / 6) * a.dt);
  const bool dz = dealias_zero(g.dealias, 1, m, ly, lz, g.Nx, g.Ny, g.Nz);
  // the stage update of field i; returns the value stored (the new stage field, or at
  // stage 4 the new state)
  auto advance = [&](int i) -> V {
    const Fac<T> Feh = i < 3 ? Fhu : Fht, Fe1 = i < 3 ? F1u : F1t;
    const long long o = i * g.S + off;
    const V R = Rv[i];
    const V u0 = i < 3 ? U0[o] : T0[off];
    V r;
    if (a.stage == 1) {
      Uc[o] = r = rk_u1_c(dz ? mk<V>(0, 0) : u0, R, Feh, Fc2);
      tot[o] = rk_t1_c(R, Fe1, Fc6);
    } else if (a.stage == 2) {
      Uc[o] = r = rk_u2_c(u0, R, Feh, Fc2);
      tot[o] = rk_tacc_c(tot[o], R, Feh, Fc3);
    } else if (a.stage == 3) {
      Uc[o] = r = rk_u3_c(u0, R, Feh, Fc1);
      tot[o] = rk_tacc_c(tot[o], R, Feh, Fc3);
    } else {
      r = rk_u4_c(u0, tot[o], R, Fe1, Fc6);
      if (a.reality && lz == g.Nz / 2) r = mk<V>(0, 0);
      if (i < 3) const_cast<V*>(U0)[o] = r;
      else const_cast<V*>(T0)[off] = r;
      health_mark(nonfinite(r), a.health ? a.health + mb : nullptr);
    }
    return r;
  };
  // a slaved field i: the stage field, or at stage 4 the state
  auto store = [&](int i, V v) {
    if (a.stage < 4) Uc[i * g.S + off] = v;
    else if (i < 3) const_cast<V*>(U0)[i * g.S + off] = v;
    else const_cast<V*>(T0)[off] = v;
  };
  if (a.slave == 1) {
    // PRZERO (Single_time_step_RBC, Tadvance_functions.cc:383-386): U advanced, then
    // T = U.V1 / K^2 with T(0) = 0 (Zero_Prandtl_number_compute_temperature, FluidVF.cc:228-232)
    const V v1 = advance(0);
    advance(1);
    advance(2);
    store(3, K2 > 0 ? mk<V>((T)((double)v1.x / K2), (T)((double)v1.y / K2)) : mk<V>(0, 0));
    return;
  }
  if (a.slave == 2) {
    // PRINFTY (:388-391): T advanced, then U from it (Infinite_Prandtl_number_compute_velocity,
    // FluidVF.cc:235-272): X = Kx T / K^2 (T has the Vx parity), V1 = (T - Kx X) / K^2,
    // V2 = i Ky X / K^2, V3 = i Kz X / K^2 (X has the divergence parity), times vs; 0 at K = 0
    const V t = advance(3);
    if (K2 > 0) {
      const double Xr = (Kxd * t.x) / K2, Xi = (Kxd * t.y) / K2;
      store(0, mk<V>((T)(a.vs * (((double)t.x - Kxd * Xr) / K2)), (T)(a.vs * (((double)t.y - Kxd * Xi) / K2))));
      store(1, mk<V>((T)(a.vs * ((-Kyd * Xi) / K2)), (T)(a.vs * ((Kyd * Xr) / K2))));
      store(2, mk<V>((T)(a.vs * ((-Kzd * Xi) / K2)), (T)(a.vs * ((Kzd * Xr) / K2))));
    } else {
      for (int i = 0; i < 3; ++i) store(i, mk<V>(0, 0));
    }
    return;
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) advance(i);
}

// The slaved field of a PRZERO / PRINFTY state (SFF): slave = 1: T = U.V1 / K^2;
// slave = 2: U = vs P(T x) / K^2 (the formulas of sff_epilogue, for initial conditions).
template <typename T>
__global__ void __launch_bounds__(256) k_rbc_slave(C<T>* __restrict__ U, C<T>* __restrict__ Tf, Geo g, int slave,
                                                   double vs) {
  typedef C<T> V;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < g.S; e += stride) {
    const int lz = (int)(e % g.Hz);
    const long long r = e / g.Hz;
    const int ly = (int)(r % g.Ny), m = (int)(r / g.Ny);
    const double Kxd = m * g.kf[0], Kyd = kfft(ly, g.Ny) * g.kf[1], Kzd = lz * g.kf[2];
    const double K2 = (Kxd * Kxd + Kyd * Kyd) + Kzd * Kzd;
    if (slave == 1) {
      const V v1 = U[e];
      Tf[e] = K2 > 0 ? mk<V>((T)((double)v1.x / K2), (T)((double)v1.y / K2)) : mk<V>(0, 0);
    } else {
      const V t = Tf[e];
      if (K2 > 0) {
        const double Xr = (Kxd * t.x) / K2, Xi = (Kxd * t.y) / K2;
        U[e] = mk<V>((T)(vs * (((double)t.x - Kxd * Xr) / K2)), (T)(vs * (((double)t.y - Kxd * Xi) / K2)));
        U[g.S + e] = mk<V>((T)(vs * ((-Kyd * Xi) / K2)), (T)(vs * ((Kyd * Xr) / K2)));
        U[2 * g.S + e] = mk<V>((T)(vs * ((-Kzd * Xi) / K2)), (T)(vs * ((Kzd * Xr) / K2)));
      } else {
        U[e] = U[g.S + e] = U[2 * g.S + e] = mk<V>(0, 0);
      }
    }
  }
}

// Elementwise Boussinesq epilogue (the split form of k_sff_fwd_x): N1..N3, NT
// in P components 0-3 of member blockIdx.y; one thread per element, every array
// access coalesced.
template <typename T>
__global__ void __launch_bounds__(256) k_sff_epi(const C<T>* __restrict__ P, Geo g, SffArgs a) {
  const long long mb = blockIdx.y;
  P += mb * a.msP;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < g.S; e += stride) {
    const int lz = (int)(e % g.Hz);
    const long long r = e / g.Hz;
    const int ly = (int)(r % g.Ny), m = (int)(r / g.Ny);
    sff_epilogue<T>(g, a, mb, m, ly, lz, e, P[e], P[g.S + e], P[2 * g.S + e], P[3 * g.S + e]);
  }
}

// ---------------------------------------------------------------------------
// forward x pass + Boussinesq epilogue (PRLARGE / ULARGE):
//   N1 = Dx(u1u1) + iKy F[u1u2] + iKz F[u3u1],  N2 = iKy F[u2u2] + Dx(u1u2) + iKz F[u2u3],
//   N3 = iKz F[u3u3] + iKy F[u2u3] + Dx(u3u1),  NT = Dx(u1T) + iKy F[u2T] + iKz F[u3T]
//   (compute_diag_offdiag.cc:47-136); force U.F1 = cu T, T.F = cT U.V1 (compute_force_RBC.cc:104-150);
//   N -= F; p = div(N)/K^2; N += grad p; R = -N, RT = -NT; IF-RK4 stage update of U (nu) and T (kappa)
//   (RK_SF.cc:97-221, Tadvance_functions.cc:57-90,226-237,372-395,589-611).
// ---------------------------------------------------------------------------
// The nine product columns stream through two cp.async staging tiles (field
// f+2 is in flight while f is transformed); each thread stages exactly the
// elements it reads back, in FFT input order, so the reordering is done by the
// copy and no barrier guards the staging tiles.
// Shared memory: exchange tile + 2 staging tiles of N x CW complex.
template <typename T, int N, int E, int CW, bool SPLIT>
__global__ void __launch_bounds__(CW * (N / E), sff_min_blocks(CW * (N / E), E))
    k_sff_fwd_x(C<T>* __restrict__ P, Geo g, SffArgs a, const C<T>* __restrict__ tq) {
  typedef C<T> V;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* xch = reinterpret_cast<V*>(smraw);
  V* stage = xch + N * CW;
  const int c = threadIdx.x % CW, t = threadIdx.x / CW;
  const int inner = g.Ny * g.Hz;
  const int col = blockIdx.x * CW + c;
  const bool ok = col < inner;
  const int ly = ok ? col / g.Hz : 0, lz = ok ? col % g.Hz : 0;
  const int ky = kfft(ly, g.Ny);
  const double Kyd = ky * g.kf[1], Kzd = lz * g.kf[2];
  const T Ky = (T)Kyd, Kz = (T)Kzd;
  const long long rstride = inner;
  const double scl = 1.0 / (2.0 * N * (double)g.Ny * g.Nz);
  const long long mb = blockIdx.y;  // member of a batch
  P += mb * a.msP;

  V acc[4][E];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int s = 0; s < E; ++s) acc[i][s] = mk<V>(0, 0);

  // field f's column into staging tile buf, row k of the tile = FFT input k
  // (even points, then odd points reversed)
  auto issue = [&](int f, int buf) {
    if (f < 9 && ok) {
      const V* src = P + f * g.S + col;
#pragma unroll
      for (int s = 0; s < E; ++s) {
        const int k = load_row<N, E>(t, s);
        cp_async(stage + (buf * N + k) * CW + c, src + (k < N / 2 ? 2 * k : 2 * (N - 1 - k) + 1) * rstride);
      }
    }
    cp_async_commit();
  };
  issue(0, 0);
  issue(1, 1);
  for (int f = 0; f < 9; ++f) {
    const bool sine = sff_prod_sine(f);
    const int buf = f & 1;
    cp_async_wait<1>();
    V v[E];
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int k = load_row<N, E>(t, s);
      V x = mk<V>(0, 0);
      if (ok) {
        x = stage[(buf * N + k) * CW + c];
        if (sine && k >= N / 2) x = scale(x, (T)-1);
      }
      v[s] = x;
    }
    issue(f + 2, buf);
    fft_regs<N, E, -1, 0, false, false, best_swk(N, E, CW, (int)sizeof(V))>(v, t, xch, CW, c, tq, 4);
    // pair terms Z_{N-m} through the exchange tile
#pragma unroll
    for (int s = 0; s < E; ++s) xch[final_row<N, E>(t, s) * CW + c] = v[s];
    __syncthreads();
    V zr[E];
#pragma unroll
    for (int s = 0; s < E; ++s) zr[s] = xch[((N - final_row<N, E>(t, s)) % N) * CW + c];
    __syncthreads();
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int m = final_row<N, E>(t, s);
      const V wz = mul(tq[m], v[s]), wzr = mul(conjg(tq[m]), zr[s]);
      const V cm = sine ? mul_i<1>(scale(sub(wz, wzr), (T)scl)) : scale(add(wz, wzr), (T)scl);
      const T Kx = (T)(m * g.kf[0]);
      switch (f) {
        case 0: acc[0][s] = add(acc[0][s], scale(cm, -Kx)); break;
        case 1: acc[1][s] = add(acc[1][s], ik(Ky, cm)); break;
        case 2: acc[2][s] = add(acc[2][s], ik(Kz, cm)); break;
        case 3: acc[0][s] = add(acc[0][s], ik(Ky, cm)); acc[1][s] = add(acc[1][s], scale(cm, Kx)); break;
        case 4: acc[1][s] = add(acc[1][s], ik(Kz, cm)); acc[2][s] = add(acc[2][s], ik(Ky, cm)); break;
        case 5: acc[0][s] = add(acc[0][s], ik(Kz, cm)); acc[2][s] = add(acc[2][s], scale(cm, Kx)); break;
        case 6: acc[3][s] = add(acc[3][s], scale(cm, -Kx)); break;
        case 7: acc[3][s] = add(acc[3][s], ik(Ky, cm)); break;
        default: acc[3][s] = add(acc[3][s], ik(Kz, cm)); break;
      }
    }
  }
  if (!ok) return;
#pragma unroll
  for (int s = 0; s < E; ++s) {
    const int m = final_row<N, E>(t, s);
    const long long off = m * rstride + col;
    if (SPLIT) {
      // the assembled vectors replace products 0-3 of this column (every read of them is done)
#pragma unroll
      for (int i = 0; i < 4; ++i) P[i * g.S + off] = acc[i][s];
    } else {
      sff_epilogue<T>(g, a, mb, m, ly, lz, off, acc[0][s], acc[1][s], acc[2][s], acc[3][s]);
    }
  }
}

// ---------------------------------------------------------------------------
// FFF passive scalar (program.kind SCALAR_INCOMPRESS), elementwise epilogue after the
// forward x FFT of the nine products of form 2 (u1u1, u2u2, u3u3, u1u2, u2u3,
// u3u1, u1T, u2T, u3T; unnormalised):
//   N_i = sum_j i K_j F[u_j u_i]  (compute_diag_offdiag.cc:47-98, conservative)
//   NT  = sum_j i K_j F[u_j T]    (compute_diag_offdiag.cc:116-136)
//   no force (Add_force with F = 0); p = (i K . N)/K^2, N <- N + i K p; R = -N,
//   RT = -NT; IF-RK4 stage update of U (nu) and T (kappa) as the Boussinesq
//   epilogue (RK_SF.cc:97-221).  One thread per element, every access coalesced.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_scalar_epi(const C<T>* __restrict__ P, Geo g, SffArgs a) {
  typedef C<T> V;
  const T inv = (T)(1.0 / ((double)g.Nx * g.Ny * g.Nz));
  const V* U0 = reinterpret_cast<const V*>(a.U0);
  const V* T0 = reinterpret_cast<const V*>(a.T0);
  V* Uc = reinterpret_cast<V*>(a.Ucur);
  V* tot = reinterpret_cast<V*>(a.tot);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < g.S; e += stride) {
    const int lz = (int)(e % g.Hz);
    const long long r = e / g.Hz;
    const int ly = (int)(r % g.Ny), lx = (int)(r / g.Ny);
    const double Kxd = kfft(lx, g.Nx) * g.kf[0], Kyd = kfft(ly, g.Ny) * g.kf[1], Kzd = lz * g.kf[2];
    const T Kx = (T)Kxd, Ky = (T)Kyd, Kz = (T)Kzd;
    V p[9];
#pragma unroll
    for (int f = 0; f < 9; ++f) p[f] = scale(P[f * g.S + e], inv);
    // x, then y, then z derivative terms, as the reference accumulates them
    V N1 = add(add(ik(Kx, p[0]), ik(Ky, p[3])), ik(Kz, p[5]));
    V N2 = add(add(ik(Kx, p[3]), ik(Ky, p[1])), ik(Kz, p[4]));
    V N3 = add(add(ik(Kx, p[5]), ik(Ky, p[4])), ik(Kz, p[2]));
    const V NT = add(add(ik(Kx, p[6]), ik(Ky, p[7])), ik(Kz, p[8]));
    const double K2 = (Kxd * Kxd + Kyd * Kyd) + Kzd * Kzd;
    const V div = add(add(ik(Kx, N1), ik(Ky, N2)), ik(Kz, N3));
    const V pr = (K2 > 0) ? mk<V>(div.x / (T)K2, div.y / (T)K2) : mk<V>(0, 0);
    N1 = add(N1, ik(Kx, pr));
    N2 = add(N2, ik(Ky, pr));
    N3 = add(N3, ik(Kz, pr));
    const V Rv[4] = {scale(N1, (T)-1), scale(N2, (T)-1), scale(N3, (T)-1), scale(NT, (T)-1)};
    const double ehu = a.eu[0][lx] * a.eu[1][ly] * a.eu[2][lz];
    const double eht = a.et[0][lx] * a.et[1][ly] * a.et[2][lz];
    const Fac<T> Fhu = fac<T>(ehu), F1u = fac<T>(ehu * ehu), Fht = fac<T>(eht), F1t = fac<T>(eht * eht);
    const Fac<T> Fc1 = fac<T>(a.dt), Fc2 = fac<T>(0.5 * a.dt), Fc3 = fac<T>((1.0 / 3) * a.dt),
                 Fc6 = fac<T>((1.0 / 6) * a.dt);
    const bool dz = dealias_zero(g.dealias, 0, lx, ly, lz, g.Nx, g.Ny, g.Nz);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const Fac<T> Feh = i < 3 ? Fhu : Fht, Fe1 = i < 3 ? F1u : F1t;
      const long long o = i * g.S + e;
      const V R = Rv[i];
      const V u0 = i < 3 ? U0[o] : T0[e];
      if (a.stage == 1) {
        Uc[o] = rk_u1_c(dz ? mk<V>(0, 0) : u0, R, Feh, Fc2);
        tot[o] = rk_t1_c(R, Fe1, Fc6);
      } else if (a.stage == 2) {
        Uc[o] = rk_u2_c(u0, R, Feh, Fc2);
        tot[o] = rk_tacc_c(tot[o], R, Feh, Fc3);
      } else if (a.stage == 3) {
        Uc[o] = rk_u3_c(u0, R, Feh, Fc1);
        tot[o] = rk_tacc_c(tot[o], R, Feh, Fc3);
      } else {
        V un = rk_u4_c(u0, tot[o], R, Fe1, Fc6);
        if (a.reality && lz == g.Nz / 2) un = mk<V>(0, 0);
        if (i < 3) const_cast<V*>(U0)[o] = un;
        else const_cast<V*>(T0)[e] = un;
        health_mark(nonfinite(un), a.health);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// FFF incompressible MHD (RK4(U, W, P, F) with W = B, no force), elementwise
// epilogue after the forward x FFT of the nine products P_ij = F[Zp_i Zm_j]
// (f = 3 i + j, unnormalised) of the z pass form 5:
//   Zp.nlin_i = sum_j D_j P_ij, Zm.nlin_i = sum_j D_j P_ji, accumulated as the
//   reference does (diagonal term, then the off-diagonal products in the order of
//   compute_diag_offdiag.cc:202-258); U.nlin = (Zp.nlin + Zm.nlin)/2,
//   B.nlin = (Zp.nlin - Zm.nlin)/2 (MHD.cc:150-161); pressure from U.nlin;
//   R_U = -(U.nlin + i K p), R_B = -B.nlin (Tadvance_functions.cc:259-267); IF-RK4
//   stage update of U (nu, tables eu) and B (eta, tables et), RK_VF_MHD.cc:126-186.
//   a.U0 = U (3 components), a.T0 = B (3), Ucur and tot carry 6 components.
//   Compiled for three blocks per SM (66 registers): with 123 it ran 20 % slower.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256, 3) k_mhd_epi(const C<T>* __restrict__ P, Geo g, SffArgs a) {
  typedef C<T> V;
  const T inv = (T)(1.0 / ((double)g.Nx * g.Ny * g.Nz));
  const V* U0 = reinterpret_cast<const V*>(a.U0);
  const V* B0 = reinterpret_cast<const V*>(a.T0);
  V* Uc = reinterpret_cast<V*>(a.Ucur);
  V* tot = reinterpret_cast<V*>(a.tot);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < g.S; e += stride) {
    const int lz = (int)(e % g.Hz);
    const long long r = e / g.Hz;
    const int ly = (int)(r % g.Ny), lx = (int)(r / g.Ny);
    const double Kxd = kfft(lx, g.Nx) * g.kf[0], Kyd = kfft(ly, g.Ny) * g.kf[1], Kzd = lz * g.kf[2];
    const T K[3] = {(T)Kxd, (T)Kyd, (T)Kzd};
    V q[9];
#pragma unroll
    for (int f = 0; f < 9; ++f) q[f] = scale(P[f * g.S + e], inv);
    // Zp.nlin (np) and Zm.nlin (nm)
    V np[3], nm[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) np[i] = nm[i] = ik(K[i], q[4 * i]);
    np[0] = add(np[0], ik(K[1], q[1])); nm[1] = add(nm[1], ik(K[0], q[1]));   // P01
    nm[0] = add(nm[0], ik(K[1], q[3])); np[1] = add(np[1], ik(K[0], q[3]));   // P10
    np[1] = add(np[1], ik(K[2], q[5])); nm[2] = add(nm[2], ik(K[1], q[5]));   // P12
    nm[1] = add(nm[1], ik(K[2], q[7])); np[2] = add(np[2], ik(K[1], q[7]));   // P21
    nm[0] = add(nm[0], ik(K[2], q[6])); np[2] = add(np[2], ik(K[0], q[6]));   // P20
    np[0] = add(np[0], ik(K[2], q[2])); nm[2] = add(nm[2], ik(K[0], q[2]));   // P02
    V NU[3], NB[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      NU[i] = scale(add(np[i], nm[i]), (T)0.5);
      NB[i] = scale(sub(np[i], nm[i]), (T)0.5);
    }
    const double K2 = (Kxd * Kxd + Kyd * Kyd) + Kzd * Kzd;
    const V div = add(add(ik(K[0], NU[0]), ik(K[1], NU[1])), ik(K[2], NU[2]));
    const V pr = (K2 > 0) ? mk<V>(div.x / (T)K2, div.y / (T)K2) : mk<V>(0, 0);
    V Rv[6];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      Rv[i] = scale(add(NU[i], ik(K[i], pr)), (T)-1);
      Rv[3 + i] = scale(NB[i], (T)-1);
    }
    const double ehu = a.eu[0][lx] * a.eu[1][ly] * a.eu[2][lz];
    const double ehb = a.et[0][lx] * a.et[1][ly] * a.et[2][lz];
    const Fac<T> Fhu = fac<T>(ehu), F1u = fac<T>(ehu * ehu), Fht = fac<T>(ehb), F1t = fac<T>(ehb * ehb);
    const Fac<T> Fc1 = fac<T>(a.dt), Fc2 = fac<T>(0.5 * a.dt), Fc3 = fac<T>((1.0 / 3) * a.dt),
                 Fc6 = fac<T>((1.0 / 6) * a.dt);
    const bool dz = dealias_zero(g.dealias, 0, lx, ly, lz, g.Nx, g.Ny, g.Nz);
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      const Fac<T> Feh = i < 3 ? Fhu : Fht, Fe1 = i < 3 ? F1u : F1t;
      const long long o = i * g.S + e;
      const V R = Rv[i];
      const V u0 = i < 3 ? U0[o] : B0[(i - 3) * g.S + e];
      if (a.stage == 1) {
        Uc[o] = rk_u1_c(dz ? mk<V>(0, 0) : u0, R, Feh, Fc2);
        tot[o] = rk_t1_c(R, Fe1, Fc6);
      } else if (a.stage == 2) {
        Uc[o] = rk_u2_c(u0, R, Feh, Fc2);
        tot[o] = rk_tacc_c(tot[o], R, Feh, Fc3);
      } else if (a.stage == 3) {
        Uc[o] = rk_u3_c(u0, R, Feh, Fc1);
        tot[o] = rk_tacc_c(tot[o], R, Feh, Fc3);
      } else {
        V un = rk_u4_c(u0, tot[o], R, Fe1, Fc6);
        if (a.reality && lz == g.Nz / 2) un = mk<V>(0, 0);
        if (i < 3) const_cast<V*>(U0)[o] = un;
        else const_cast<V*>(B0)[(i - 3) * g.S + e] = un;
        health_mark(nonfinite(un), a.health);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// SSF fluid step (sincostr_switch "SCF": Vx = SCF, Vy = CSF, Vz = CCF), elementwise
// epilogue after the forward transforms of the six products (normalised; parities
// Vi2 = CCF for u_i u_i, VxVy = SSF, VyVz = CSF, VxVz = SCF; Global.cc:184-191).
// Derivatives (SSF_pencil_tr.cc): x and y parity S -> +K, C -> -K; z -> i Kz.
//   N1 = Dx(u1u1) + Dy(u1u2) + Dz(u3u1), N2 = Dy(u2u2) + Dx(u1u2) + Dz(u2u3),
//   N3 = Dz(u3u3) + Dy(u2u3) + Dx(u3u1)  (compute_diag_offdiag.cc:47-98)
//   div = Dx^Vx N1 + Dy^Vy N2 + Dz N3, p = div/K^2, N += (Dx^div p, Dy^div p, Dz p), R = -N;
//   IF-RK4 stage update as the FFF step (RK.cc:91-170); no reality condition.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_ssf_epi(const C<T>* __restrict__ P, Geo g, StageArgs a) {
  typedef C<T> V;
  const V* U0 = reinterpret_cast<const V*>(a.U0);
  V* Uc = reinterpret_cast<V*>(a.Ucur);
  V* tot = reinterpret_cast<V*>(a.tot);
  V* Uo = reinterpret_cast<V*>(a.Uout);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < g.S; e += stride) {
    const int lz = (int)(e % g.Hz);
    const long long r = e / g.Hz;
    const int ly = (int)(r % g.Ny), lx = (int)(r / g.Ny);
    const double Kxd = lx * g.kf[0], Kyd = ly * g.kf[1], Kzd = lz * g.kf[2];
    const T Kx = (T)Kxd, Ky = (T)Kyd, Kz = (T)Kzd;
    V q[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) q[f] = P[f * g.S + e];
    // x / y derivative of a sine (+K) or cosine (-K) series
    auto dS = [](T K, V A) { return scale(A, K); };
    auto dC = [](T K, V A) { return scale(A, -K); };
    V N1 = add(add(dC(Kx, q[0]), dS(Ky, q[3])), ik(Kz, q[5]));
    V N2 = add(add(dC(Ky, q[1]), dS(Kx, q[3])), ik(Kz, q[4]));
    V N3 = add(add(ik(Kz, q[2]), dS(Ky, q[4])), dS(Kx, q[5]));
    const double K2 = (Kxd * Kxd + Kyd * Kyd) + Kzd * Kzd;
    const V div = add(add(dS(Kx, N1), dS(Ky, N2)), ik(Kz, N3));
    const V pr = (K2 > 0) ? mk<V>(div.x / (T)K2, div.y / (T)K2) : mk<V>(0, 0);
    N1 = add(N1, dC(Kx, pr));
    N2 = add(N2, dC(Ky, pr));
    N3 = add(N3, ik(Kz, pr));
    const V Rv[3] = {scale(N1, (T)-1), scale(N2, (T)-1), scale(N3, (T)-1)};
    const double eh = a.ex[lx] * a.ey[ly] * a.ez[lz];
    const Fac<T> Feh = fac<T>(eh), Fe1 = fac<T>(eh * eh);
    const Fac<T> Fc1 = fac<T>(a.dt), Fc2 = fac<T>(0.5 * a.dt), Fc3 = fac<T>((1.0 / 3) * a.dt),
                 Fc6 = fac<T>((1.0 / 6) * a.dt);
    const bool dz = dealias_zero(g.dealias, 2, lx, ly, lz, g.Nx, g.Ny, g.Nz);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const long long o = i * g.S + e;
      const V R = Rv[i];
      const V u0 = U0[o];
      if (a.stage == 1) {
        Uc[o] = rk_u1_c(dz ? mk<V>(0, 0) : u0, R, Feh, Fc2);
        tot[o] = rk_t1_c(R, Fe1, Fc6);
      } else if (a.stage == 2) {
        Uc[o] = rk_u2_c(u0, R, Feh, Fc2);
        tot[o] = rk_tacc_c(tot[o], R, Feh, Fc3);
      } else if (a.stage == 3) {
        Uc[o] = rk_u3_c(u0, R, Feh, Fc1);
        tot[o] = rk_tacc_c(tot[o], R, Feh, Fc3);
      } else {
        const V un = rk_u4_c(u0, tot[o], R, Fe1, Fc6);
        Uo[o] = un;
        health_mark(nonfinite(un), a.err);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// SSS fluid step (sincostr_switch "SCC": Vx = SCC, Vy = CSC, Vz = CCS), on real
// coefficients in the padded real layout (Nz + 2 reals per line, lzr < Nz used):
// dealiased copy, and the elementwise epilogue after the forward transforms of the
// six products (Vi2 = CCC, VxVy = SSC, VyVz = CSS, VxVz = SCS; Global.cc:221-228).
// Derivatives along every axis: parity S -> +K, C -> -K (SSS_pencil_tr.cc).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_sss_dealias_copy(const T* __restrict__ A, T* __restrict__ B, int ncomp,
                                                          Geo g) {
  // component blockIdx.y; one pair of reals (z indices 2 lz, 2 lz + 1) per element, 32-bit
  // index arithmetic (a component holds < 2^31 pairs)
  typedef C<T> V;
  const V* a = reinterpret_cast<const V*>(A);
  V* b = reinterpret_cast<V*>(B);
  const int n = (int)g.S;
  const long long off = (long long)blockIdx.y * g.S;
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
    const int lz = m % g.Hz, r = m / g.Hz;
    const int ly = r % g.Ny, lx = r / g.Ny;
    V x = a[off + m];
    if (2 * lz >= g.Nz || sss_dealias_zero(g.dealias, lx, ly, 2 * lz, g.Nx, g.Ny, g.Nz)) x.x = (T)0;
    if (2 * lz + 1 >= g.Nz || sss_dealias_zero(g.dealias, lx, ly, 2 * lz + 1, g.Nx, g.Ny, g.Nz)) x.y = (T)0;
    b[off + m] = x;
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_sss_epi(const T* __restrict__ P, Geo g, StageArgs a) {
  const long long per = 2 * g.S;
  const T* U0 = reinterpret_cast<const T*>(a.U0);
  T* Uc = reinterpret_cast<T*>(a.Ucur);
  T* tot = reinterpret_cast<T*>(a.tot);
  T* Uo = reinterpret_cast<T*>(a.Uout);
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < per; e += (long long)gridDim.x * blockDim.x) {
    const int lzr = (int)(e % (g.Nz + 2));
    if (lzr >= g.Nz) continue;  // padding
    const long long r = e / (g.Nz + 2);
    const int ly = (int)(r % g.Ny), lx = (int)(r / g.Ny);
    const double Kxd = lx * g.kf[0], Kyd = ly * g.kf[1], Kzd = lzr * g.kf[2];
    const T Kx = (T)Kxd, Ky = (T)Kyd, Kz = (T)Kzd;
    T q[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) q[f] = P[f * per + e];
    T N1 = (-Kx * q[0] + Ky * q[3]) + Kz * q[5];
    T N2 = (-Ky * q[1] + Kx * q[3]) + Kz * q[4];
    T N3 = (-Kz * q[2] + Ky * q[4]) + Kx * q[5];
    const double K2 = (Kxd * Kxd + Kyd * Kyd) + Kzd * Kzd;
    const T div = (Kx * N1 + Ky * N2) + Kz * N3;
    const T pr = K2 > 0 ? div / (T)K2 : (T)0;
    N1 += -Kx * pr;
    N2 += -Ky * pr;
    N3 += -Kz * pr;
    const T Rv[3] = {-N1, -N2, -N3};
    const double eh = a.ex[lx] * a.ey[ly] * a.ez[lzr];
    const Fac<T> Feh = fac<T>(eh), Fe1 = fac<T>(eh * eh);
    const Fac<T> Fc1 = fac<T>(a.dt), Fc2 = fac<T>(0.5 * a.dt), Fc3 = fac<T>((1.0 / 3) * a.dt),
                 Fc6 = fac<T>((1.0 / 6) * a.dt);
    const bool dz = sss_dealias_zero(g.dealias, lx, ly, lzr, g.Nx, g.Ny, g.Nz);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const long long o = i * per + e;
      const T R = Rv[i], u0 = U0[o];
      if (a.stage == 1) {
        Uc[o] = rk_u1(dz ? (T)0 : u0, R, Feh, Fc2);
        tot[o] = rk_t1(R, Fe1, Fc6);
      } else if (a.stage == 2) {
        Uc[o] = rk_u2(u0, R, Feh, Fc2);
        tot[o] = rk_tacc(tot[o], R, Feh, Fc3);
      } else if (a.stage == 3) {
        Uc[o] = rk_u3(u0, R, Feh, Fc1);
        tot[o] = rk_tacc(tot[o], R, Feh, Fc3);
      } else {
        const T un = rk_u4(u0, tot[o], R, Fe1, Fc6);
        Uo[o] = un;
        health_mark(!isfinite(un), a.err);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Boussinesq RBC (PRLARGE, ULARGE) on the SSF and SSS bases: the temperature takes
// the Vx parity and the products u_x T, u_y T, u_z T take Vi2, VxVy and VxVz
// (Global_process_basic_vars.cc:108, 114-116).  Epilogues after the forward
// transforms of the nine products (u1u1, u2u2, u3u3, u1u2, u2u3, u3u1, u1T, u2T,
// u3T; normalised):
//   N as the fluid step; NT = Dx(u1T) + Dy(u2T) + Dz(u3T) (compute_diag_offdiag.cc:116-136);
//   force (compute_force_RBC.cc:104-150): U.F1 = cu T, T.F = cT U.V1, both from the
//   un-dealiased stage input; N1 -= T, NT -= u1 (Add_force); pressure from N;
//   R = -N, RT = -NT; IF-RK4 stage update of U (nu, tables eu) and T (kappa,
//   tables et) as RK_SF.cc:97-221, in place at stage 4; no reality condition.
// SSF: x and y derivatives of a sine series +K, of a cosine series -K; z: i Kz.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_ssf_rbc_epi(const C<T>* __restrict__ P, Geo g, SffArgs a) {
  typedef C<T> V;
  V* U0 = const_cast<V*>(reinterpret_cast<const V*>(a.U0));
  V* T0 = const_cast<V*>(reinterpret_cast<const V*>(a.T0));
  const V* U1in = reinterpret_cast<const V*>(a.U1in);
  const V* Tin = reinterpret_cast<const V*>(a.Tin);
  V* Uc = reinterpret_cast<V*>(a.Ucur);
  V* tot = reinterpret_cast<V*>(a.tot);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < g.S; e += stride) {
    const int lz = (int)(e % g.Hz);
    const long long r = e / g.Hz;
    const int ly = (int)(r % g.Ny), lx = (int)(r / g.Ny);
    const double Kxd = lx * g.kf[0], Kyd = ly * g.kf[1], Kzd = lz * g.kf[2];
    const T Kx = (T)Kxd, Ky = (T)Kyd, Kz = (T)Kzd;
    V q[9];
#pragma unroll
    for (int f = 0; f < 9; ++f) q[f] = P[f * g.S + e];
    auto dS = [](T K, V A) { return scale(A, K); };
    auto dC = [](T K, V A) { return scale(A, -K); };
    V N1 = add(add(dC(Kx, q[0]), dS(Ky, q[3])), ik(Kz, q[5]));
    V N2 = add(add(dC(Ky, q[1]), dS(Kx, q[3])), ik(Kz, q[4]));
    V N3 = add(add(ik(Kz, q[2]), dS(Ky, q[4])), dS(Kx, q[5]));
    V NT = add(add(dC(Kx, q[6]), dS(Ky, q[7])), ik(Kz, q[8]));
    N1 = sub(N1, scale(Tin[e], (T)a.cu));
    NT = sub(NT, scale(U1in[e], (T)a.cT));
    const double K2 = (Kxd * Kxd + Kyd * Kyd) + Kzd * Kzd;
    const V div = add(add(dS(Kx, N1), dS(Ky, N2)), ik(Kz, N3));
    const V pr = (K2 > 0) ? mk<V>(div.x / (T)K2, div.y / (T)K2) : mk<V>(0, 0);
    N1 = add(N1, dC(Kx, pr));
    N2 = add(N2, dC(Ky, pr));
    N3 = add(N3, ik(Kz, pr));
    const V Rv[4] = {scale(N1, (T)-1), scale(N2, (T)-1), scale(N3, (T)-1), scale(NT, (T)-1)};
    const double ehu = a.eu[0][lx] * a.eu[1][ly] * a.eu[2][lz];
    const double eht = a.et[0][lx] * a.et[1][ly] * a.et[2][lz];
    const Fac<T> Fhu = fac<T>(ehu), F1u = fac<T>(ehu * ehu), Fht = fac<T>(eht), F1t = fac<T>(eht * eht);
    const Fac<T> Fc1 = fac<T>(a.dt), Fc2 = fac<T>(0.5 * a.dt), Fc3 = fac<T>((1.0 / 3) * a.dt),
                 Fc6 = fac<T>((1.0 / 6) * a.dt);
    const bool dz = dealias_zero(g.dealias, 2, lx, ly, lz, g.Nx, g.Ny, g.Nz);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const Fac<T> Feh = i < 3 ? Fhu : Fht, Fe1 = i < 3 ? F1u : F1t;
      const long long o = i * g.S + e;
      const V R = Rv[i];
      const V u0 = i < 3 ? U0[o] : T0[e];
      if (a.stage == 1) {
        Uc[o] = rk_u1_c(dz ? mk<V>(0, 0) : u0, R, Feh, Fc2);
        tot[o] = rk_t1_c(R, Fe1, Fc6);
      } else if (a.stage == 2) {
        Uc[o] = rk_u2_c(u0, R, Feh, Fc2);
        tot[o] = rk_tacc_c(tot[o], R, Feh, Fc3);
      } else if (a.stage == 3) {
        Uc[o] = rk_u3_c(u0, R, Feh, Fc1);
        tot[o] = rk_tacc_c(tot[o], R, Feh, Fc3);
      } else {
        const V un = rk_u4_c(u0, tot[o], R, Fe1, Fc6);
        if (i < 3) U0[o] = un;
        else T0[e] = un;
        health_mark(nonfinite(un), a.health);
      }
    }
  }
}

// SSS: real coefficients in the padded real layout; every axis sine +K, cosine -K.
// Parities: u1u1..u3u3 CCC, u1u2 SSC, u2u3 CSS, u3u1 SCS, u1T CCC, u2T SSC, u3T SCS.
template <typename T>
__global__ void __launch_bounds__(256) k_sss_rbc_epi(const T* __restrict__ P, Geo g, SffArgs a) {
  const long long per = 2 * g.S;
  T* U0 = const_cast<T*>(reinterpret_cast<const T*>(a.U0));
  T* T0 = const_cast<T*>(reinterpret_cast<const T*>(a.T0));
  const T* U1in = reinterpret_cast<const T*>(a.U1in);
  const T* Tin = reinterpret_cast<const T*>(a.Tin);
  T* Uc = reinterpret_cast<T*>(a.Ucur);
  T* tot = reinterpret_cast<T*>(a.tot);
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < per; e += (long long)gridDim.x * blockDim.x) {
    const int lzr = (int)(e % (g.Nz + 2));
    if (lzr >= g.Nz) continue;  // padding
    const long long r = e / (g.Nz + 2);
    const int ly = (int)(r % g.Ny), lx = (int)(r / g.Ny);
    const double Kxd = lx * g.kf[0], Kyd = ly * g.kf[1], Kzd = lzr * g.kf[2];
    const T Kx = (T)Kxd, Ky = (T)Kyd, Kz = (T)Kzd;
    T q[9];
#pragma unroll
    for (int f = 0; f < 9; ++f) q[f] = P[f * per + e];
    T N1 = (-Kx * q[0] + Ky * q[3]) + Kz * q[5];
    T N2 = (-Ky * q[1] + Kx * q[3]) + Kz * q[4];
    T N3 = (-Kz * q[2] + Ky * q[4]) + Kx * q[5];
    T NT = (-Kx * q[6] + Ky * q[7]) + Kz * q[8];
    N1 -= (T)a.cu * Tin[e];
    NT -= (T)a.cT * U1in[e];
    const double K2 = (Kxd * Kxd + Kyd * Kyd) + Kzd * Kzd;
    const T div = (Kx * N1 + Ky * N2) + Kz * N3;
    const T pr = K2 > 0 ? div / (T)K2 : (T)0;
    N1 += -Kx * pr;
    N2 += -Ky * pr;
    N3 += -Kz * pr;
    const T Rv[4] = {-N1, -N2, -N3, -NT};
    const double ehu = a.eu[0][lx] * a.eu[1][ly] * a.eu[2][lzr];
    const double eht = a.et[0][lx] * a.et[1][ly] * a.et[2][lzr];
    const Fac<T> Fhu = fac<T>(ehu), F1u = fac<T>(ehu * ehu), Fht = fac<T>(eht), F1t = fac<T>(eht * eht);
    const Fac<T> Fc1 = fac<T>(a.dt), Fc2 = fac<T>(0.5 * a.dt), Fc3 = fac<T>((1.0 / 3) * a.dt),
                 Fc6 = fac<T>((1.0 / 6) * a.dt);
    const bool dz = sss_dealias_zero(g.dealias, lx, ly, lzr, g.Nx, g.Ny, g.Nz);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const Fac<T> Feh = i < 3 ? Fhu : Fht, Fe1 = i < 3 ? F1u : F1t;
      const long long o = i * per + e;
      const T R = Rv[i], u0 = i < 3 ? U0[o] : T0[e];
      if (a.stage == 1) {
        Uc[o] = rk_u1(dz ? (T)0 : u0, R, Feh, Fc2);
        tot[o] = rk_t1(R, Fe1, Fc6);
      } else if (a.stage == 2) {
        Uc[o] = rk_u2(u0, R, Feh, Fc2);
        tot[o] = rk_tacc(tot[o], R, Feh, Fc3);
      } else if (a.stage == 3) {
        Uc[o] = rk_u3(u0, R, Feh, Fc1);
        tot[o] = rk_tacc(tot[o], R, Feh, Fc3);
      } else {
        const T un = rk_u4(u0, tot[o], R, Fe1, Fc6);
        if (i < 3) U0[o] = un;
        else T0[e] = un;
        health_mark(!isfinite(un), a.health);
      }
    }
  }
}

}  // namespace ts
