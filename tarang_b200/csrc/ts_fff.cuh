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

namespace ts {

struct Geo {
  int Nx, Ny, Nz, Hz;
  long long S;          // complex elements per component
  double kf[3];         // kfactor (reference kfactor[1..3])
  int basis;            // 0 FFF, 1 SFF
  int dealias;          // 0 none, 1 reference corner, 2 two thirds
};

// ---------------------------------------------------------------------------
// plain strided-axis FFT (x or y axis) over nf fields, in place
// element (o, row, col) at o*ostride + row*rstride + col, col < inner
// ---------------------------------------------------------------------------
template <typename T, int L, int E, int CW, int DIR>
__global__ void __launch_bounds__(CW * (L / E), (CW * (L / E)) <= 256 ? 2 : 1) k_strided_fft(C<T>* __restrict__ data, int nf, long long fstride,
                                                               int inner, long long rstride, long long ostride,
                                                               const C<T>* __restrict__ tw) {
  typedef C<T> V;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* sm = reinterpret_cast<V*>(smraw);
  const int c = threadIdx.x % CW, t = threadIdx.x / CW;
  const int col = blockIdx.x * CW + c;
  const bool ok = col < inner;
  const long long base = (long long)blockIdx.y * ostride + (ok ? col : 0);
  for (int f = 0; f < nf; ++f) {
    V* d = data + f * fstride + base;
    V v[E];
#pragma unroll
    for (int s = 0; s < E; ++s) v[s] = ok ? d[load_row<L, E>(t, s) * rstride] : mk<V>(0, 0);
    fft_regs<L, E, DIR>(v, t, sm, CW, c, tw, 1);
    if (ok) {
#pragma unroll
      for (int s = 0; s < E; ++s) d[final_row<L, E>(t, s) * rstride] = v[s];
    }
  }
}

// ---------------------------------------------------------------------------
// inverse x pass: W_i = IFFT_x(D(U_i)); rotational form also W_{3+i} = IFFT_x(D(omega_i)),
// omega = i K x D(U).  col = ly*Hz + lz; row = lx.
// ---------------------------------------------------------------------------
template <typename T, int L, int E, int CW, bool ROT>
__global__ void __launch_bounds__(CW * (L / E), (CW * (L / E)) <= 256 ? 2 : 1) k_inv_x(const C<T>* __restrict__ U, C<T>* __restrict__ W, Geo g,
                                                         const C<T>* __restrict__ tw) {
  typedef C<T> V;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* sm = reinterpret_cast<V*>(smraw);
  const int c = threadIdx.x % CW, t = threadIdx.x / CW;
  const int inner = g.Ny * g.Hz;
  const int col = blockIdx.x * CW + c;
  const bool ok = col < inner;
  const int ly = ok ? col / g.Hz : 0, lz = ok ? col % g.Hz : 0;
  const T Ky = (T)(kfft(ly, g.Ny) * g.kf[1]), Kz = (T)(lz * g.kf[2]);
  const long long rstride = inner;
  const int nout = ROT ? 6 : 3;
  for (int f = 0; f < nout; ++f) {
    V v[E];
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int lx = load_row<L, E>(t, s);
      const long long off = lx * rstride + col;
      V a = mk<V>(0, 0);
      if (ok && !dealias_zero(g.dealias, g.basis, lx, ly, lz, g.Nx, g.Ny, g.Nz)) {
        if (f < 3) {
          a = U[f * g.S + off];
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
    fft_regs<L, E, 1>(v, t, sm, CW, c, tw, 1);
    if (ok) {
      V* d = W + f * g.S + col;
#pragma unroll
      for (int s = 0; s < E; ++s) d[final_row<L, E>(t, s) * rstride] = v[s];
    }
  }
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

template <typename T, int NZ, int E, int FORM>
__global__ void __launch_bounds__(256) k_z_fused(C<T>* __restrict__ P, Geo g, const C<T>* __restrict__ tw, int nl) {
  typedef C<T> V;
  constexpr int M = NZ / 2, H = M + 1, TPL = M / E, LDS = zslot<M>();
  constexpr int NIN = FORM == 0 ? 3 : 6, NOUT = FORM == 0 ? 6 : 3;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* sm = reinterpret_cast<V*>(smraw);
  const long long nlines = (long long)g.Nx * g.Ny;
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
      if (live) { a = X[k]; b = conjg(X[M - k]); }
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
    if (FORM == 0) {
      slot(0, ll)[m] = mk<V>(in[0].x * in[0].x, in[0].y * in[0].y);
      slot(1, ll)[m] = mk<V>(in[1].x * in[1].x, in[1].y * in[1].y);
      slot(2, ll)[m] = mk<V>(in[2].x * in[2].x, in[2].y * in[2].y);
      slot(3, ll)[m] = mk<V>(in[0].x * in[1].x, in[0].y * in[1].y);
      slot(4, ll)[m] = mk<V>(in[1].x * in[2].x, in[1].y * in[2].y);
      slot(5, ll)[m] = mk<V>(in[2].x * in[0].x, in[2].y * in[0].y);
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
// forward x pass + spectral epilogue
// ---------------------------------------------------------------------------
struct StageArgs {
  void* U0;          // state (Vcopy), updated in place at stage 4
  void* Ucur;        // stage field
  void* tot;         // RK accumulator
  void* nout;        // MODE_NLIN: output N (3 comps)
  const void* Ud;    // MODE_FLUX: field whose dealiased copy multiplies N
  double* bins;      // MODE_FLUX: per-sphere accumulators (global)
  const double* radii;
  int nradii;
  const void* fcube; // force cube (3 comps of (2km+1)^2 (km+1)), nullptr = no force
  int fkm;
  double nu, dt;
  int stage;         // 1..4
  int reality;       // zero the kz = Nz/2 plane at the end of stage 4
};

enum { MODE_STEP = 0, MODE_FLUX = 1, MODE_NLIN = 2 };

template <typename T, int L, int E, int CW, int FORM, int MODE>
__global__ void __launch_bounds__(CW * (L / E), (CW * (L / E)) <= 256 ? 2 : 1) k_fwd_x(const C<T>* __restrict__ P, Geo g, StageArgs a,
                                                         const C<T>* __restrict__ tw) {
  typedef C<T> V;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* sm = reinterpret_cast<V*>(smraw);
  double* sbins = reinterpret_cast<double*>(smraw + (size_t)L * CW * sizeof(V));
  const int c = threadIdx.x % CW, t = threadIdx.x / CW;
  const int inner = g.Ny * g.Hz;
  const int col = blockIdx.x * CW + c;
  const bool ok = col < inner;
  const int ly = ok ? col / g.Hz : 0, lz = ok ? col % g.Hz : 0;
  const int ky = kfft(ly, g.Ny);
  const double Kyd = ky * g.kf[1], Kzd = lz * g.kf[2];
  const T Ky = (T)Kyd, Kz = (T)Kzd;
  const long long rstride = inner;
  const T inv = (T)(1.0 / ((double)g.Nx * g.Ny * g.Nz));
  constexpr int NF = FORM == 0 ? 6 : 3;

  V acc[3][E];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int s = 0; s < E; ++s) acc[i][s] = mk<V>(0, 0);

  for (int f = 0; f < NF; ++f) {
    V v[E];
    const V* d = P + f * g.S + (ok ? col : 0);
#pragma unroll
    for (int s = 0; s < E; ++s) v[s] = ok ? d[load_row<L, E>(t, s) * rstride] : mk<V>(0, 0);
    fft_regs<L, E, -1>(v, t, sm, CW, c, tw, 1);
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int lx = final_row<L, E>(t, s);
      const T Kx = (T)(kfft(lx, g.Nx) * g.kf[0]);
      const V p = scale(v[s], inv);
      if (FORM == 0) {
        // N_i = sum_j i K_j F[u_i u_j]  (compute_diag_offdiag.cc:47-98)
        switch (f) {
          case 0: acc[0][s] = add(acc[0][s], ik(Kx, p)); break;
          case 1: acc[1][s] = add(acc[1][s], ik(Ky, p)); break;
          case 2: acc[2][s] = add(acc[2][s], ik(Kz, p)); break;
          case 3: acc[0][s] = add(acc[0][s], ik(Ky, p)); acc[1][s] = add(acc[1][s], ik(Kx, p)); break;
          case 4: acc[1][s] = add(acc[1][s], ik(Kz, p)); acc[2][s] = add(acc[2][s], ik(Ky, p)); break;
          default: acc[2][s] = add(acc[2][s], ik(Kx, p)); acc[0][s] = add(acc[0][s], ik(Kz, p)); break;
        }
      } else {
        // N = -F[u x omega]
        if (f == 0) acc[0][s] = scale(p, (T)-1);
        else if (f == 1) acc[1][s] = scale(p, (T)-1);
        else acc[2][s] = scale(p, (T)-1);
      }
    }
  }

  if (MODE == MODE_FLUX) {
    for (int i = threadIdx.x; i < a.nradii + 1; i += blockDim.x) sbins[i] = 0.0;
    __syncthreads();
  }

  if (ok) {
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int lx = final_row<L, E>(t, s);
      const long long off = lx * rstride + col;
      const int kx = kfft(lx, g.Nx);
      const double Kxd = kx * g.kf[0];
      V N1 = acc[0][s], N2 = acc[1][s], N3 = acc[2][s];
      if (MODE == MODE_NLIN) {
        V* no = reinterpret_cast<V*>(a.nout);
        no[off] = N1; no[g.S + off] = N2; no[2 * g.S + off] = N3;
        continue;
      }
      if (MODE == MODE_FLUX) {
        // contribution 2 mult Re(N . conj(D(U))) to the first sphere with |K| <= R
        const V* Ud = reinterpret_cast<const V*>(a.Ud);
        if (dealias_zero(g.dealias, g.basis, lx, ly, lz, g.Nx, g.Ny, g.Nz)) continue;
        const V u1 = Ud[off], u2 = Ud[g.S + off], u3 = Ud[2 * g.S + off];
        double re = (double)N1.x * u1.x + (double)N1.y * u1.y + (double)N2.x * u2.x + (double)N2.y * u2.y +
                    (double)N3.x * u3.x + (double)N3.y * u3.y;
        double mult = lz > 0 ? 1.0 : 0.5;
        if (kx == g.Nx / 2 || (ky == g.Ny / 2 && g.Ny > 1)) mult *= 2;
        const double Kmag = sqrt((Kxd * Kxd + Kyd * Kyd) + Kzd * Kzd);
        int b = 0;
        while (b < a.nradii && Kmag > a.radii[b]) ++b;
        atomicAdd(&sbins[b], 2.0 * mult * re);
        continue;
      }
      // ---- MODE_STEP ----
      const T Kx = (T)Kxd;
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
      V div = add(add(ik(Kx, N1), ik(Ky, N2)), ik(Kz, N3));
      const V p = (K2 > 0) ? mk<V>(div.x / (T)K2, div.y / (T)K2) : mk<V>(0, 0);
      V R1 = scale(add(N1, ik(Kx, p)), (T)-1);
      V R2 = scale(add(N2, ik(Ky, p)), (T)-1);
      V R3 = scale(add(N3, ik(Kz, p)), (T)-1);
      // IF-RK4 stage update (RK.cc:91-170 with Single_time_step / Compute_RK4_parts)
      const double eh = exp(-a.nu * 0.5 * a.dt * K2);
      const double e1 = exp(-a.nu * 1.0 * a.dt * K2);
      const T Eh = (T)eh, E1 = (T)e1;
      V* U0 = reinterpret_cast<V*>(a.U0);
      V* Uc = reinterpret_cast<V*>(a.Ucur);
      V* tot = reinterpret_cast<V*>(a.tot);
      const V Rv[3] = {R1, R2, R3};
      const T dt = (T)a.dt;
      const bool dz = dealias_zero(g.dealias, g.basis, lx, ly, lz, g.Nx, g.Ny, g.Nz);
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const long long o = i * g.S + off;
        const V R = Rv[i];
        if (a.stage == 1) {
          V u0 = dz ? mk<V>(0, 0) : U0[o];
          Uc[o] = scale(add(u0, scale(R, (T)(0.5 * a.dt))), Eh);
          tot[o] = scale(scale(R, E1), (T)((1.0 / 6) * a.dt));
        } else if (a.stage == 2) {
          Uc[o] = add(scale(U0[o], Eh), scale(R, (T)(0.5 * a.dt)));
          tot[o] = add(tot[o], scale(scale(R, Eh), (T)((1.0 / 3) * a.dt)));
        } else if (a.stage == 3) {
          Uc[o] = scale(add(scale(U0[o], Eh), scale(R, dt)), Eh);
          tot[o] = add(tot[o], scale(scale(R, Eh), (T)((1.0 / 3) * a.dt)));
        } else {
          V tt = add(tot[o], scale(R, (T)((1.0 / 6) * a.dt)));
          V un = add(scale(U0[o], E1), tt);
          if (a.reality && lz == g.Nz / 2) un = mk<V>(0, 0);
          U0[o] = un;
        }
      }
    }
  }
  if (MODE == MODE_FLUX) {
    __syncthreads();
    for (int i = threadIdx.x; i < a.nradii + 1; i += blockDim.x)
      if (sbins[i] != 0.0) atomicAdd(&a.bins[i], sbins[i]);
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
