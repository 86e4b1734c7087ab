// SFF (sin/cos x Fourier x Fourier) kernels of the Boussinesq IF-RK4 step.
//
// Along x the fields are sine (S) or cosine (C) series on the staggered grid
// x_n = (n+1/2) Lx/Nx with modes m = 0..Nx-1 stored at lx = m
// (SFF_pencil_inline.h:63; sine m = 0 unused, the m = Nx sine term dropped):
//   C:  u_n = c_0 + 2 sum_m c_m cos(pi m (2n+1)/(2N)),  c_m = (1/N) sum_n u_n cos(...)
//   S:  u_n =       2 sum_m c_m sin(pi m (2n+1)/(2N)),  c_m = (1/N) sum_n u_n sin(...)
// Each x transform is a 2N-point complex FFT of the even (C) / odd (S)
// extension with quarter-step twiddles e^{-i pi k/(2N)} before or after, so it
// applies to the complex data left by the y and z Fourier passes directly.
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
};

// parity of product field f: true = sine
__host__ __device__ constexpr bool sff_prod_sine(int f) { return f == 3 || f == 5 || f == 7 || f == 8; }

// ---------------------------------------------------------------------------
// inverse x pass: W_f = inverse sin/cos transform of D(field_f), f = u1,u2,u3,T.
// tq: 4N entries exp(-2 pi i j/(4N)) (its even entries are the 2N-FFT table).
// ---------------------------------------------------------------------------
template <typename T, int N, int E, int CW>
__global__ void __launch_bounds__(CW * (2 * N / E), (CW * (2 * N / E)) <= 256 ? 2 : 1)
    k_sff_inv_x(const C<T>* __restrict__ U, const C<T>* __restrict__ Tf, C<T>* __restrict__ W, Geo g,
                const C<T>* __restrict__ tq) {
  typedef C<T> V;
  constexpr int L2 = 2 * N;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* xch = reinterpret_cast<V*>(smraw);
  const int c = threadIdx.x % CW, t = threadIdx.x / CW;
  const int inner = g.Ny * g.Hz;
  const int col = blockIdx.x * CW + c;
  const bool ok = col < inner;
  const int ly = ok ? col / g.Hz : 0, lz = ok ? col % g.Hz : 0;
  const long long rstride = inner;
  for (int f = 0; f < 4; ++f) {
    const V* src = (f < 3 ? U + f * g.S : Tf) + (ok ? col : 0);
    const bool sine = f == 0 || f == 3;
    V v[E];
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int k = load_row<L2, E>(t, s);
      const int m = k <= N ? k : L2 - k;
      V z = mk<V>(0, 0);
      if (ok && k != N && !(sine && m == 0) && !dealias_zero(g.dealias, 1, m, ly, lz, g.Nx, g.Ny, g.Nz)) {
        const V a = src[m * rstride];
        if (k == 0) z = a;                                   // cosine c_0
        else if (k < N) z = mul(conjg(tq[m]), a);            // e^{+i pi m/2N} c_m
        else z = mul(tq[m], a);                              // e^{-i pi m/2N} c_m
        if (sine) z = (k < N) ? mul_i<-1>(z) : mul_i<1>(z);  // -i / +i for the sine series
      }
      v[s] = z;
    }
    fft_regs<L2, E, 1>(v, t, xch, CW, c, tq, 2);
    if (ok) {
      V* d = W + f * g.S + col;
#pragma unroll
      for (int s = 0; s < E; ++s) {
        const int n = final_row<L2, E>(t, s);
        if (n < N) d[n * rstride] = v[s];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// forward x pass + Boussinesq epilogue (PRLARGE / ULARGE):
//   N1 = Dx(u1u1) + iKy F[u1u2] + iKz F[u3u1],  N2 = iKy F[u2u2] + Dx(u1u2) + iKz F[u2u3],
//   N3 = iKz F[u3u3] + iKy F[u2u3] + Dx(u3u1),  NT = Dx(u1T) + iKy F[u2T] + iKz F[u3T]
//   (compute_diag_offdiag.cc:47-136); force U.F1 = T, T.F = U.V1 (compute_force_RBC.cc:104-150);
//   N -= F; p = div(N)/K^2; N += grad p; R = -N, RT = -NT; IF-RK4 stage update of U (nu) and T (kappa)
//   (RK_SF.cc:97-221, Tadvance_functions.cc:57-90,226-237,372-395,589-611).
// ---------------------------------------------------------------------------
template <typename T, int N, int E, int CW>
__global__ void __launch_bounds__(CW * (2 * N / E), (CW * (2 * N / E)) <= 256 ? 2 : 1)
    k_sff_fwd_x(const C<T>* __restrict__ P, Geo g, SffArgs a, const C<T>* __restrict__ tq) {
  typedef C<T> V;
  constexpr int L2 = 2 * N;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* xch = reinterpret_cast<V*>(smraw);
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

  V acc[4][E];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int s = 0; s < E; ++s) acc[i][s] = mk<V>(0, 0);

  for (int f = 0; f < 9; ++f) {
    const bool sine = sff_prod_sine(f);
    const V* src = P + f * g.S + (ok ? col : 0);
    V v[E];
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int k = load_row<L2, E>(t, s);
      V x = mk<V>(0, 0);
      if (ok) {
        x = src[(k < N ? k : L2 - 1 - k) * rstride];  // even / odd extension
        if (sine && k >= N) x = scale(x, (T)-1);
      }
      v[s] = x;
    }
    fft_regs<L2, E, -1>(v, t, xch, CW, c, tq, 2);
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int m = final_row<L2, E>(t, s);
      if (m >= N) continue;
      V cm = scale(mul(tq[m], v[s]), (T)scl);
      if (sine) cm = (m == 0) ? mk<V>(0, 0) : mul_i<1>(cm);
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
  const V* U0 = reinterpret_cast<const V*>(a.U0);
  const V* T0 = reinterpret_cast<const V*>(a.T0);
  V* Uc = reinterpret_cast<V*>(a.Ucur);
  V* tot = reinterpret_cast<V*>(a.tot);
  const V* U1in = reinterpret_cast<const V*>(a.U1in);
  const V* Tin = reinterpret_cast<const V*>(a.Tin);
  const double eyz_u = a.eu[1][ly] * a.eu[2][lz], eyz_t = a.et[1][ly] * a.et[2][lz];
#pragma unroll
  for (int s = 0; s < E; ++s) {
    const int m = final_row<L2, E>(t, s);
    if (m >= N) continue;
    const long long off = m * rstride + col;
    const double Kxd = m * g.kf[0];
    const T Kx = (T)Kxd;
    // force (ULARGE): U.F1 = T, T.F = U.V1 of the stage input; nlin -= F
    V N1 = sub(acc[0][s], Tin[off]), N2 = acc[1][s], N3 = acc[2][s];
    const V NT = sub(acc[3][s], U1in[off]);
    // projection with SFF parities: div = +Kx N1 + i Ky N2 + i Kz N3; grad_x p = -Kx p
    const double K2 = (Kxd * Kxd + Kyd * Kyd) + Kzd * Kzd;
    const V div = add(add(scale(N1, Kx), ik(Ky, N2)), ik(Kz, N3));
    const V pr = (K2 > 0) ? mk<V>(div.x / (T)K2, div.y / (T)K2) : mk<V>(0, 0);
    N1 = add(N1, scale(pr, -Kx));
    N2 = add(N2, ik(Ky, pr));
    N3 = add(N3, ik(Kz, pr));
    const V Rv[4] = {scale(N1, (T)-1), scale(N2, (T)-1), scale(N3, (T)-1), scale(NT, (T)-1)};
    const double ehu = a.eu[0][m] * eyz_u, eht = a.et[0][m] * eyz_t;
    const bool dz = dealias_zero(g.dealias, 1, m, ly, lz, g.Nx, g.Ny, g.Nz);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const double eh = i < 3 ? ehu : eht;
      const T Eh = (T)eh, E1 = (T)(eh * eh);
      const long long o = i * g.S + off;
      const V R = Rv[i];
      const V u0 = i < 3 ? U0[o] : T0[off];
      if (a.stage == 1) {
        Uc[o] = scale(add(dz ? mk<V>(0, 0) : u0, scale(R, (T)(0.5 * a.dt))), Eh);
        tot[o] = scale(scale(R, E1), (T)((1.0 / 6) * a.dt));
      } else if (a.stage == 2) {
        Uc[o] = add(scale(u0, Eh), scale(R, (T)(0.5 * a.dt)));
        tot[o] = add(tot[o], scale(scale(R, Eh), (T)((1.0 / 3) * a.dt)));
      } else if (a.stage == 3) {
        Uc[o] = scale(add(scale(u0, Eh), scale(R, (T)a.dt)), Eh);
        tot[o] = add(tot[o], scale(scale(R, Eh), (T)((1.0 / 3) * a.dt)));
      } else {
        V un = add(scale(u0, E1), add(tot[o], scale(R, (T)((1.0 / 6) * a.dt))));
        if (a.reality && lz == g.Nz / 2) un = mk<V>(0, 0);
        if (i < 3) const_cast<V*>(U0)[o] = un;
        else const_cast<V*>(T0)[off] = un;
      }
    }
  }
}

}  // namespace ts
