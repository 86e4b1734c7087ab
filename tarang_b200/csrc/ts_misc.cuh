// Plane-sized and reduction kernels: strong reality condition, Carati force on
// the forcing band, total energy, max |div|, shell spectrum E(k), and the
// random-phase helical initial condition.
#pragma once
#include "ts_fff.cuh"

namespace ts {

// ---------------------------------------------------------------------------
// Satisfy_strong_reality_condition_in_Array (FFF_pencil_basic.cc:139-179,
// SFF_pencil_basic.cc:143-167) on ncomp consecutive components.
// Targets and sources of the kz=0 copy are disjoint, so the copy runs in place.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_reality(C<T>* A, int ncomp, Geo g) {
  typedef C<T> V;
  const long long plane = (long long)g.Nx * g.Ny;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= plane * ncomp) return;
  const int comp = (int)(e / plane);
  const int lx = (int)((e % plane) / g.Ny), ly = (int)(e % g.Ny);
  V* a = A + comp * g.S;
  const int ky = kfft(ly, g.Ny);
  const int iym = ((-ky) % g.Ny + g.Ny) % g.Ny;
  const long long Hz = g.Hz;
  if (g.basis == 0) {
    if (lx > g.Nx / 2 && ky != g.Ny / 2) {
      const int mkx = -kfft(lx, g.Nx);
      a[((long long)lx * g.Ny + ly) * Hz] = conjg(a[((long long)mkx * g.Ny + iym) * Hz]);
    } else if (lx == 0 && ky < 0) {
      a[(long long)ly * Hz] = conjg(a[(long long)iym * Hz]);
    }
  } else {
    if (ky < 0) a[((long long)lx * g.Ny + ly) * Hz] = conjg(a[((long long)lx * g.Ny + iym) * Hz]);
    else if (ky == 0) { V v = a[((long long)lx * g.Ny) * Hz]; v.y = -v.y; a[((long long)lx * g.Ny) * Hz] = v; }
  }
  a[((long long)lx * g.Ny + ly) * Hz + g.Nz / 2] = mk<V>(0, 0);
}

// Transpose of k_reality (FFF), in place: every kz = 0 entry that k_reality
// overwrites with conj(source) adds its conjugate to that source and becomes 0;
// the kz = Nz/2 plane is zeroed.  One thread per (source, copy) pair, so the
// pairs are disjoint and no entry is both read and written by two threads.
template <typename T>
__global__ void k_reality_adj(C<T>* A, int ncomp, Geo g) {
  typedef C<T> V;
  const long long plane = (long long)g.Nx * g.Ny;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= plane * ncomp) return;
  const int comp = (int)(e / plane);
  const int lx = (int)((e % plane) / g.Ny), ly = (int)(e % g.Ny);
  V* a = A + comp * g.S;
  const int ky = kfft(ly, g.Ny);
  const int iym = ((-ky) % g.Ny + g.Ny) % g.Ny;
  const long long Hz = g.Hz;
  long long cp = -1;  // the copy of this source entry, if any
  if (lx >= 1 && 2 * lx < g.Nx && ky != g.Ny / 2) cp = ((long long)(g.Nx - lx) * g.Ny + iym) * Hz;
  else if (lx == 0 && ky > 0 && 2 * ky < g.Ny) cp = (long long)iym * Hz;
  if (cp >= 0) {
    const long long so = ((long long)lx * g.Ny + ly) * Hz;
    a[so] = add(a[so], conjg(a[cp]));
    a[cp] = mk<V>(0, 0);
  }
  a[((long long)lx * g.Ny + ly) * Hz + g.Nz / 2] = mk<V>(0, 0);
}

// Scatter the force cube (3 components of (2km+1)^2 (km+1) modes, kx, ky = -km..km,
// kz = 0..km) into a full spectral field F (zeroed by the caller).
template <typename T>
__global__ void k_force_scatter(const C<T>* __restrict__ fc, C<T>* __restrict__ F, Geo g, int km) {
  const int n = 2 * km + 1;
  const long long ncube = (long long)n * n * (km + 1);
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 3 * ncube) return;
  const int c = (int)(e / ncube);
  const long long r = e % ncube;
  const int kx = (int)(r / (n * (km + 1))) - km, ky = (int)((r / (km + 1)) % n) - km, lz = (int)(r % (km + 1));
  const int lx = (kx + g.Nx) % g.Nx, ly = (ky + g.Ny) % g.Ny;
  F[c * g.S + ((long long)lx * g.Ny + ly) * g.Hz + lz] = fc[e];
}

// ---------------------------------------------------------------------------
// Carati constant-energy-supply force (non-global alpha/beta) on the cube
// |kx|,|ky|,kz <= km; compute_force_Carati.cc:158-205, force_alpha_beta.cc:56-85,
// then the strong reality condition on the force (compute_force_main.cc:67-73).
// One block.  fc: 3 comps of (2km+1)(2km+1)(km+1).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_carati(const C<T>* __restrict__ U, C<T>* fc, Geo g, int km, double r_in, double r_out,
                         const double* __restrict__ esup, const double* __restrict__ hsup,
                         const double* __restrict__ mis, int nsup) {
  typedef C<T> V;
  const int n = 2 * km + 1;
  const int ncube = n * n * (km + 1);
  for (int e = threadIdx.x; e < ncube; e += blockDim.x) {
    const int kx = e / (n * (km + 1)) - km;
    const int ky = (e / (km + 1)) % n - km;
    const int kz = e % (km + 1);
    V F[3] = {mk<V>(0, 0), mk<V>(0, 0), mk<V>(0, 0)};
    const double Kx = kx * g.kf[0], Ky = ky * g.kf[1], Kz = kz * g.kf[2];
    const double K = sqrt((Kx * Kx + Ky * Ky) + Kz * Kz);
    const bool inbox = abs(kx) <= g.Nx / 2 && abs(ky) <= g.Ny / 2 && kz <= g.Nz / 2 &&
                       !(kx == -g.Nx / 2) && !(ky == -g.Ny / 2);
    if (inbox && K > r_in && K <= r_out) {
      const int index = (int)ceil(K);
      const int lx = kx >= 0 ? kx : kx + g.Nx, ly = ky >= 0 ? ky : ky + g.Ny;
      const long long off = ((long long)lx * g.Ny + ly) * g.Hz + kz;
      double vr[3], vi[3];
      for (int i = 0; i < 3; ++i) { V u = U[i * g.S + off]; vr[i] = u.x; vi[i] = u.y; }
      const double me = (vr[0] * vr[0] + vi[0] * vi[0] + vr[1] * vr[1] + vi[1] * vi[1] + vr[2] * vr[2] + vi[2] * vi[2]) / 2;
      if (me > 1e-15 && index < nsup && mis[index] > 0) {
        const double ek = esup[index] / mis[index];
        const double hk = hsup ? hsup[index] / mis[index] : 0.0;
        // K . (Vr x Vi)
        const double cx = vr[1] * vi[2] - vr[2] * vi[1], cy = vr[2] * vi[0] - vr[0] * vi[2], cz = vr[0] * vi[1] - vr[1] * vi[0];
        const double mh = Kx * cx + Ky * cy + Kz * cz;
        const double denr = 2.0 * ((K * me) * (K * me) - mh * mh);
        double alpha = 0, beta = 0;
        if (fabs(denr) > 1e-15) {
          alpha = (K * K * ek * me - hk * mh) / denr;
          beta = (hk * me - ek * mh) / denr;
        } else {
          alpha = ek / (4 * me);
          beta = alpha / K;
        }
        // omega = i K x V
        const double Kv[3] = {Kx, Ky, Kz};
        for (int i = 0; i < 3; ++i) {
          const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
          // (K x V)_i = K_i1 V_i2 - K_i2 V_i1 ; omega = i (K x V)
          const double crr = Kv[i1] * vr[i2] - Kv[i2] * vr[i1];
          const double cri = Kv[i1] * vi[i2] - Kv[i2] * vi[i1];
          const double wr = -cri, wi = crr;
          F[i] = mk<V>((T)(alpha * vr[i] + beta * wr), (T)(alpha * vi[i] + beta * wi));
        }
      }
    }
    for (int i = 0; i < 3; ++i) fc[i * ncube + e] = F[i];
  }
  __syncthreads();
  // reality on the kz = 0 plane of the cube: F(kx<0,ky,0) = conj(F(-kx,-ky,0)) for ky != Ny/2,
  // F(0,ky<0,0) = conj(F(0,-ky,0)); kz = Nz/2 never lies in the cube unless km >= Nz/2.
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int kx = e / n - km, ky = e % n - km;
    bool tgt = (kx < 0 && ky != g.Ny / 2) || (kx == 0 && ky < 0);
    if (!tgt) continue;
    const int src = ((-kx + km) * n + (-ky + km)) * (km + 1);
    const int dst = ((kx + km) * n + (ky + km)) * (km + 1);
    for (int i = 0; i < 3; ++i) fc[i * ncube + dst] = conjg(fc[i * ncube + src]);
  }
  if (km >= g.Nz / 2) {
    __syncthreads();
    for (int e = threadIdx.x; e < n * n; e += blockDim.x)
      for (int i = 0; i < 3; ++i) fc[i * ncube + e * (km + 1) + g.Nz / 2] = mk<V>(0, 0);
  }
}

// ---------------------------------------------------------------------------
// Test of the bounded-wait path (ts_plan_expire_wait): one thread waits on an
// mbarrier that expects one arrival which never comes, with no bulk copy in flight,
// so mbar_wait gives up after `polls` polls, sets the timeout bit of *err and the
// kernel returns.
// ---------------------------------------------------------------------------
static __global__ void k_expire_wait(int* err, int polls) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
    mbar_wait(&bar, 0, err, polls);  // phase 0 never completes
  }
}

// ---------------------------------------------------------------------------
// reductions (FP64 accumulation; warp_sum / block_sum are in ts_common.cuh)
// ---------------------------------------------------------------------------

// plane weights of the total energy: FFF 1/2 on kz=0 (FFF_pencil_energy.cc:59-68);
// SFF 2, minus 1 on kz=0, minus 1 on m=0, plus 1/2 on (m=0,kz=0) (SFF_pencil_energy.cc:76-95);
// SSF and SSS: 4 sum, minus 2 on each of the lx = 0, ly = 0, lz = 0 planes, plus the
// lines where two meet, minus 1/2 at the origin (SSF_pencil_energy.cc:76-103,
// SSS_pencil_energy.cc:69-98), i.e. 4, 2, 1, 1/2 for none, one, two, three zero indices
__device__ __forceinline__ double energy_weight(int basis, int lx, int ly, int lz) {
  if (basis == 0) return lz == 0 ? 0.5 : 1.0;
  if (basis >= 2) {
    const int zeros = (lx == 0) + (ly == 0) + (lz == 0);
    return zeros == 0 ? 4.0 : zeros == 1 ? 2.0 : zeros == 2 ? 1.0 : 0.5;
  }
  double w = 2.0;
  if (lz == 0) w -= 1.0;
  if (lx == 0) w -= 1.0;
  if (lx == 0 && lz == 0) w += 0.5;
  return w;
}

// out[0] += sum_w Re(A.conj(B)) over ncomp components (A == B gives the energy).
// SSS: the coefficients are real, two per complex slot, z index 2 lz and 2 lz + 1
// (the padding reals at Nz, Nz + 1 are skipped).  SSF: at the origin the reference
// subtracts half the product of the real parts only (1/2 Re a Re b + Im a Im b).
template <typename T>
__global__ void k_energy(const C<T>* __restrict__ A, const C<T>* __restrict__ B, int ncomp, Geo g, double* out) {
  const long long n = g.S;
  double s = 0;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int lz = (int)(e % g.Hz);
    const int ly = (int)((e / g.Hz) % g.Ny);
    const int lx = (int)(e / ((long long)g.Ny * g.Hz));
    double dr = 0, di = 0;
    for (int i = 0; i < ncomp; ++i) {
      const C<T> a = A[i * n + e], b = B[i * n + e];
      dr += (double)a.x * b.x;
      di += (double)a.y * b.y;
    }
    if (g.basis == 3) {
      if (2 * lz < g.Nz) s += energy_weight(3, lx, ly, 2 * lz) * dr;
      if (2 * lz + 1 < g.Nz) s += energy_weight(3, lx, ly, 2 * lz + 1) * di;
    } else if (g.basis == 2 && lx == 0 && ly == 0 && lz == 0) {
      s += 0.5 * dr + di;
    } else {
      s += energy_weight(g.basis, lx, ly, lz) * (dr + di);
    }
  }
  s = block_sum(s);
  if (threadIdx.x == 0) out[1 + blockIdx.x] = s;  // partial sums, added in a fixed order by k_sum_partials
}

// out[0] = sum of the n partial sums out[1..n], in an order that does not depend
// on scheduling (one block), so energies and the normalised initial condition are
// reproducible bit for bit
static __global__ void k_sum_partials(double* out, int n) {
  double s = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += out[1 + i];
  s = block_sum(s);
  if (threadIdx.x == 0) out[0] = s;
}

// max over modes of |div U| (FFF: i K.U; SFF: Kx U1 (sine parity) + i Ky U2 + i Kz U3;
// SSF (Vx = SCF, Vy = CSF, Vz = CCF): Kx U1 + Ky U2 + i Kz U3; SSS (real, Vx = SCC,
// Vy = CSC, Vz = CCS): Kx U1 + Ky U2 + Kz U3 per real coefficient, z index 2 lz, 2 lz + 1)
template <typename T>
__global__ void k_maxdiv(const C<T>* __restrict__ U, Geo g, unsigned long long* out) {
  const long long n = g.S;
  double m = 0;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int lz = (int)(e % g.Hz);
    const int ly = (int)((e / g.Hz) % g.Ny);
    const int lx = (int)(e / ((long long)g.Ny * g.Hz));
    const double Kx = (g.basis == 0 ? kfft(lx, g.Nx) : lx) * g.kf[0];
    const double Ky = (g.basis >= 2 ? ly : kfft(ly, g.Ny)) * g.kf[1], Kz = lz * g.kf[2];
    const C<T> u1 = U[e], u2 = U[n + e], u3 = U[2 * n + e];
    double dr, di;
    if (g.basis == 0) {
      dr = -(Kx * u1.y + Ky * u2.y + Kz * u3.y);
      di = Kx * u1.x + Ky * u2.x + Kz * u3.x;
    } else if (g.basis == 1) {
      dr = Kx * u1.x - (Ky * u2.y + Kz * u3.y);
      di = Kx * u1.y + (Ky * u2.x + Kz * u3.x);
    } else if (g.basis == 2) {
      dr = Kx * u1.x + Ky * u2.x - Kz * u3.y;
      di = Kx * u1.y + Ky * u2.y + Kz * u3.x;
    } else {
      // two real coefficients per slot: z wavenumbers 2 lz and 2 lz + 1 (padding skipped)
      dr = (2 * lz < g.Nz) ? fabs(Kx * u1.x + Ky * u2.x + 2.0 * Kz * u3.x) : 0.0;
      di = (2 * lz + 1 < g.Nz) ? fabs(Kx * u1.y + Ky * u2.y + (2 * lz + 1) * g.kf[2] * u3.y) : 0.0;
      m = fmax(m, fmax(dr, di));
      continue;
    }
    m = fmax(m, sqrt(dr * dr + di * di));
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// multiplicity factor (FFF_pencil_inline.h:583-602, SFF_pencil_inline.h:492-515)
// SSF / SSS (SSF_pencil_inline.h:512-532, SSS_pencil_inline.h:537-556): 1/2 at the
// origin, 1 with two zero grid indices, 2 with one, 4 with none (indices lx, ly, lz)
__device__ __forceinline__ double multiplicity(int basis, int lx, int ly, int lz, int Nx, int Ny) {
  if (basis >= 2) {
    const int zeros = (lx == 0) + (ly == 0) + (lz == 0);
    return zeros == 0 ? 4.0 : zeros == 1 ? 2.0 : zeros == 2 ? 1.0 : 0.5;
  }
  const int ky = kfft(ly, Ny);
  double f;
  if (basis == 0) {
    f = lz > 0 ? 1.0 : 0.5;
    if (kfft(lx, Nx) == Nx / 2 || (ky == Ny / 2 && Ny > 1)) f *= 2;
  } else {
    if (lz > 0) f = lx > 0 ? 2.0 : 1.0;
    else f = lx > 0 ? 1.0 : 0.5;
    if (ky == Ny / 2 && Ny > 1) f *= 2;
  }
  return f;
}

// Shell spectrum accumulation (Compute_local_shell_spectrum universal_energy.cc:279-313), on
// every basis over the complex array shape: for every shell s = ceil|K| < nbins, sums[s] = sum mult |K|^2 sum_i Re(A_i conj(B_i)) (B = A:
// |A|^2) and counts[s] = sum 2 mult.  Reproducible bit for bit, without atomics on the sums:
// each warp walks whole z lines (|K| grows along a line, so the modes of one shell sit in
// adjacent lanes of a 32-mode chunk), adds a chunk by a segmented scan whose segment tails
// update the warp's own shared bins, and the block writes its partial bins (warps added in
// index order) to part[blockIdx.x][2 nbins] (sums, then counts) for k_bins_finish.  The
// counts are sums of small integers, exact in any order (shared atomics).
template <typename T>
__global__ void __launch_bounds__(32 * SHELL_WARPS)
    k_shell(const C<T>* __restrict__ A, const C<T>* __restrict__ B, int ncomp, Geo g, int nbins,
            double* __restrict__ part) {
  extern __shared__ double sb[];  // [SHELL_WARPS][nbins] sums, then [nbins] counts
  double* cnt = sb + SHELL_WARPS * nbins;
  for (int i = threadIdx.x; i < (SHELL_WARPS + 1) * nbins; i += blockDim.x) sb[i] = 0;
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* wb = sb + w * nbins;
  const long long n = g.S, nlines = (long long)g.Nx * g.Ny;
  if (!B) B = A;
  for (long long line = (long long)blockIdx.x * SHELL_WARPS + w; line < nlines;
       line += (long long)gridDim.x * SHELL_WARPS) {
    const int lx = (int)(line / g.Ny), ly = (int)(line % g.Ny);
    const double Kx = (g.basis == 0 ? kfft(lx, g.Nx) : lx) * g.kf[0];
    const double Ky = (g.basis >= 2 ? ly : kfft(ly, g.Ny)) * g.kf[1];
    // SSS: the complex view of the real coefficients, pair (2 lz, 2 lz + 1) as slot lz < Nz/2
    // with kz = lz (the padding slot lz = Nz/2 is not a mode)
    const int nz = g.basis == 3 ? g.Nz / 2 : g.Hz;
    for (int z0 = 0; z0 < g.Hz; z0 += 32) {
      const int lz = z0 + lane;
      int key = 0x7fffffff;
      double v = 0, c = 0;
      if (lz < nz) {
        const double Kz = lz * g.kf[2];
        const double Kmag = sqrt((Kx * Kx + Ky * Ky) + Kz * Kz);
        const int idx = (int)ceil(Kmag);
        if (idx < nbins) {
          const long long e = line * g.Hz + lz;
          const double f = multiplicity(g.basis, lx, ly, lz, g.Nx, g.Ny);
          double a2 = 0;
          for (int i = 0; i < ncomp; ++i) {
            const C<T> a = A[i * n + e], b = B[i * n + e];
            a2 += (double)a.x * b.x + (double)a.y * b.y;
          }
          key = idx;
          v = f * a2 * (Kmag * Kmag);
          c = 2 * f;
        }
      }
      // keys do not decrease along the chunk: inclusive scan within runs of equal keys
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const double vo = __shfl_up_sync(0xffffffffu, v, o), co = __shfl_up_sync(0xffffffffu, c, o);
        const int ko = __shfl_up_sync(0xffffffffu, key, o);
        if (lane >= o && ko == key) {
          v += vo;
          c += co;
        }
      }
      const int kn = __shfl_down_sync(0xffffffffu, key, 1);
      if (key != 0x7fffffff && (lane == 31 || kn != key)) {
        wb[key] += v;
        atomicAdd(&cnt[key], c);
      }
      __syncwarp();
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nbins; i += blockDim.x) {
    double t = 0;
    for (int k = 0; k < SHELL_WARPS; ++k) t += sb[k * nbins + i];
    part[(long long)blockIdx.x * 2 * nbins + i] = t;
    part[(long long)blockIdx.x * 2 * nbins + nbins + i] = cnt[i];
  }
}

// Energy flux out of one sphere, per-sphere form (EnergyTr::Compute_flux compute_flux.cc:51-65):
// P holds the nine x-forward-transformed giver products F[u_a g_b] (component 3 a + b,
// unnormalised), so N_i = sum_j i K_j F[u_j g_i] / (Nx Ny Nz) (compute_nlin_ET_VF.cc:71-87);
// out[1 + block] = sum over the modes with |K| > R of 2 mult Re(N . conj(D U))
// (Prod_out_sphere_nlinV prod_nlinV.cc:61-69, Local_shell_mult_single universal_ET.cc:51-70),
// D = the dealias mask; k_sum_partials adds the blocks in a fixed order.
template <typename T>
__global__ void k_flux_outside(const C<T>* __restrict__ P, const C<T>* __restrict__ U, Geo g, double R,
                               double* __restrict__ out) {
  const long long n = g.S;
  const double inv = 1.0 / ((double)g.Nx * g.Ny * g.Nz);
  double s = 0;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int lz = (int)(e % g.Hz);
    const int ly = (int)((e / g.Hz) % g.Ny);
    const int lx = (int)(e / ((long long)g.Ny * g.Hz));
    if (dealias_zero(g.dealias, 0, lx, ly, lz, g.Nx, g.Ny, g.Nz)) continue;
    const double K[3] = {kfft(lx, g.Nx) * g.kf[0], kfft(ly, g.Ny) * g.kf[1], lz * g.kf[2]};
    const double Kmag = sqrt((K[0] * K[0] + K[1] * K[1]) + K[2] * K[2]);
    if (!(Kmag > R)) continue;
    double re = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      double nr = 0, ni = 0;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const C<T> q = P[(3 * j + i) * n + e];
        nr -= K[j] * (double)q.y;
        ni += K[j] * (double)q.x;
      }
      const C<T> u = U[i * n + e];
      re += (nr * inv) * (double)u.x + (ni * inv) * (double)u.y;
    }
    s += 2.0 * multiplicity(0, lx, ly, lz, g.Nx, g.Ny) * re;
  }
  s = block_sum(s);
  if (threadIdx.x == 0) out[1 + blockIdx.x] = s;
}

// ---------------------------------------------------------------------------
// SSF and SFF per-sphere energy flux (EnergyTr::Compute_flux, compute_flux.cc:51-65):
// k_ssf_giver writes the inputs of the giver nonlinear term, D U into P[0, 3) and the
// giver D(U inside |K| <= R) (Fill_in_sphere, fill_space.cc:56-64) into P[3, 6), with
// Kx = lx kx (sin/cos along x), Ky = ly ky on SSF (sin/cos along y) and the FFT-order
// ky on SFF (Fourier along y), Kz = lz kz; after the transforms P[3 j + i] holds
// F[u_j G_i], normalised, with x / y sine letters qx, qy (bit f); k_ssf_flux_outside
// then forms N_i = sum_j D_j F[u_j G_i] (D on a sin/cos axis: +K on a sine series, -K
// on a cosine series; on a Fourier axis: i K) and sums 2 mult Re(N . conj(D U)) over
// |K| > R, per block (k_sum_partials adds the blocks).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double flux_ky(const Geo& g, int ly) {
  return (g.basis == 1 ? (double)kfft(ly, g.Ny) : (double)ly) * g.kf[1];
}

template <typename T>
__global__ void k_ssf_giver(const C<T>* __restrict__ U, C<T>* __restrict__ P, Geo g, double R) {
  const long long n = g.S;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int lz = (int)(e % g.Hz);
    const int ly = (int)((e / g.Hz) % g.Ny);
    const int lx = (int)(e / ((long long)g.Ny * g.Hz));
    const bool dz = dealias_zero(g.dealias, g.basis, lx, ly, lz, g.Nx, g.Ny, g.Nz);
    const double Kx = lx * g.kf[0], Ky = flux_ky(g, ly), Kz = lz * g.kf[2];
    const bool in = sqrt((Kx * Kx + Ky * Ky) + Kz * Kz) <= R;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const C<T> u = dz ? mk<C<T>>(0, 0) : U[i * n + e];
      P[i * n + e] = u;
      P[(3 + i) * n + e] = in ? u : mk<C<T>>(0, 0);
    }
  }
}

template <typename T>
__global__ void k_ssf_flux_outside(const C<T>* __restrict__ P, const C<T>* __restrict__ U, Geo g, double R,
                                   int qx, int qy, double* __restrict__ out) {
  const long long n = g.S;
  double s = 0;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int lz = (int)(e % g.Hz);
    const int ly = (int)((e / g.Hz) % g.Ny);
    const int lx = (int)(e / ((long long)g.Ny * g.Hz));
    if (dealias_zero(g.dealias, g.basis, lx, ly, lz, g.Nx, g.Ny, g.Nz)) continue;
    const double K[3] = {lx * g.kf[0], flux_ky(g, ly), lz * g.kf[2]};
    const double Kmag = sqrt((K[0] * K[0] + K[1] * K[1]) + K[2] * K[2]);
    if (!(Kmag > R)) continue;
    double re = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      double nr = 0, ni = 0;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int f = 3 * j + i;
        const C<T> q = P[f * n + e];
        if (j == 2 || (j == 1 && g.basis == 1)) {  // i K_j X on a Fourier axis
          nr -= K[j] * (double)q.y;
          ni += K[j] * (double)q.x;
        } else {
          const int sine = j == 0 ? (qx >> f & 1) : (qy >> f & 1);
          const double d = sine ? K[j] : -K[j];
          nr += d * (double)q.x;
          ni += d * (double)q.y;
        }
      }
      const C<T> u = U[i * n + e];
      re += nr * (double)u.x + ni * (double)u.y;
    }
    s += 2.0 * multiplicity(g.basis, lx, ly, lz, g.Nx, g.Ny) * re;
  }
  s = block_sum(s);
  if (threadIdx.x == 0) out[1 + blockIdx.x] = s;
}

// ---------------------------------------------------------------------------
// SSS per-sphere energy flux (compute_flux.cc:51-65 on the SSS basis, whose sphere fill
// and shell product, SSS_pencil_ET.cc:50-70 and 662-678, loop over the real
// coefficients with kz the real z index): k_sss_giver writes D U into P[0, 3) and the
// giver D(U on |K| <= R) into P[3, 6), in the padded real layout (Nx, Ny, Nz + 2) of
// each component; after the transforms P[3 j + i] holds the coefficients of F[u_j G_i]
// with sine letters qx, qy, qz (bit f); k_sss_flux_outside forms
// N_i = sum_j D_j F[u_j G_i] (+K_j on a sine series, -K_j on a cosine series) and sums
// 2 mult N_i D u_i over |K| > R, per block.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_sss_giver(const T* __restrict__ U, T* __restrict__ P, Geo g, double R) {
  const long long n = 2 * g.S;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int lzr = (int)(e % (g.Nz + 2));
    const long long r = e / (g.Nz + 2);
    const int ly = (int)(r % g.Ny), lx = (int)(r / g.Ny);
    const bool dz = lzr >= g.Nz || sss_dealias_zero(g.dealias, lx, ly, lzr, g.Nx, g.Ny, g.Nz);
    const double Kx = lx * g.kf[0], Ky = ly * g.kf[1], Kz = lzr * g.kf[2];
    const bool in = sqrt((Kx * Kx + Ky * Ky) + Kz * Kz) <= R;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const T u = dz ? (T)0 : U[i * n + e];
      P[i * n + e] = u;
      P[(3 + i) * n + e] = in ? u : (T)0;
    }
  }
}

template <typename T>
__global__ void k_sss_flux_outside(const T* __restrict__ P, const T* __restrict__ U, Geo g, double R, int qx,
                                   int qy, int qz, double* __restrict__ out) {
  const long long n = 2 * g.S;
  double s = 0;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int lzr = (int)(e % (g.Nz + 2));
    const long long r = e / (g.Nz + 2);
    const int ly = (int)(r % g.Ny), lx = (int)(r / g.Ny);
    if (lzr >= g.Nz || sss_dealias_zero(g.dealias, lx, ly, lzr, g.Nx, g.Ny, g.Nz)) continue;
    const double K[3] = {lx * g.kf[0], ly * g.kf[1], lzr * g.kf[2]};
    const double Kmag = sqrt((K[0] * K[0] + K[1] * K[1]) + K[2] * K[2]);
    if (!(Kmag > R)) continue;
    double re = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      double nr = 0;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int f = 3 * j + i;
        const int sine = ((j == 0 ? qx : (j == 1 ? qy : qz)) >> f) & 1;
        nr += (sine ? K[j] : -K[j]) * (double)P[f * n + e];
      }
      re += nr * (double)U[i * n + e];
    }
    s += 2.0 * multiplicity(3, lx, ly, lzr, g.Nx, g.Ny) * re;
  }
  s = block_sum(s);
  if (threadIdx.x == 0) out[1 + blockIdx.x] = s;
}

// ---------------------------------------------------------------------------
// random-phase helical initial condition (init_cond_energy.cc:67-120 construction;
// this project's counter-based splitmix64 phases, identical to the oracle)
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double uniform01(unsigned long long key, unsigned long long ctr) {
  return (double)(splitmix64(key ^ ctr) >> 11) * (1.0 / 9007199254740992.0);
}

template <typename T>
__global__ void k_init_ic(C<T>* U, Geo g, const double* __restrict__ Eic, const double* __restrict__ mis, int nsh,
                          unsigned long long key) {
  typedef C<T> V;
  const long long n = g.S;
  const double PI = 3.14159265358979323846;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int lz = (int)(e % g.Hz);
    const int ly = (int)((e / g.Hz) % g.Ny);
    const int lx = (int)(e / ((long long)g.Ny * g.Hz));
    const double Kx = kfft(lx, g.Nx) * g.kf[0], Ky = kfft(ly, g.Ny) * g.kf[1], Kz = lz * g.kf[2];
    const double Kmag = sqrt((Kx * Kx + Ky * Ky) + Kz * Kz);
    double r[3][2] = {{0, 0}, {0, 0}, {0, 0}};
    const int idx = (int)ceil(Kmag);
    if (Kmag > 1e-15 && idx < nsh && mis[idx] > 0) {
      const double ek = Eic[idx] / mis[idx];
      if (ek >= 1e-15) {
        const double a = sqrt(ek / 2.0);
        const double php = 2 * PI * uniform01(key, 2ull * (unsigned long long)e);
        const double phm = 2 * PI * uniform01(key, 2ull * (unsigned long long)e + 1);
        const double upr = a * cos(php), upi = a * sin(php), umr = a * cos(phm), umi = a * sin(phm);
        // U1 = i (u- - u+), U2 = u- + u+
        const double U1r = -(umi - upi), U1i = umr - upr, U2r = umr + upr, U2i = umi + upi;
        // polar angle of K with z (Get_polar_angle), azimuth from (Kx, Ky)
        const double kperp = sqrt(Kx * Kx + Ky * Ky);
        double th;
        if (fabs(kperp) > 1e-15) th = fabs(Kz) > 1e-15 ? atan(kperp / Kz) : PI / 2;
        else th = Kz >= 0 ? 0.0 : PI;
        if (th < 0) th += PI;
        double ph = 0;
        if (fabs(kperp) > 1e-15) {
          double c = Kx / kperp;
          c = c > 1 ? 1 : (c < -1 ? -1 : c);
          ph = acos(c);
          if (Ky < 0) ph = 2 * PI - ph;
        }
        const double st = sin(th), ct = cos(th), sp = sin(ph), cp = cos(ph);
        // vpll = -U2 sin th; vh1 = U1 sin ph + U2 cos th cos ph; vh2 = -U1 cos ph + U2 sin ph cos th
        r[2][0] = -U2r * st; r[2][1] = -U2i * st;
        r[0][0] = U1r * sp + U2r * ct * cp; r[0][1] = U1i * sp + U2i * ct * cp;
        r[1][0] = -U1r * cp + U2r * sp * ct; r[1][1] = -U1i * cp + U2i * sp * ct;
      }
    }
    for (int i = 0; i < 3; ++i) U[i * n + e] = mk<V>((T)r[i][0], (T)r[i][1]);
  }
}

// temperature perturbation for RBC: amplitude amp, uniform random phase
// 2 pi uniform01(key, e) on modes with grid radius |(m, ky, kz)| <= kmax, m >= 1
template <typename T>
__global__ void k_init_temp(C<T>* A, Geo g, double amp, double kmax, unsigned long long key) {
  const long long n = g.S;
  const double PI = 3.14159265358979323846;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int lz = (int)(e % g.Hz);
    const int ly = (int)((e / g.Hz) % g.Ny);
    const int lx = (int)(e / ((long long)g.Ny * g.Hz));
    const int ky = kfft(ly, g.Ny);
    const double r = sqrt((double)lx * lx + (double)ky * ky + (double)lz * lz);
    C<T> v = mk<C<T>>(0, 0);
    if (r <= kmax && lx >= 1) {
      const double ph = 2 * PI * uniform01(key, (unsigned long long)e);
      v = mk<C<T>>((T)(amp * cos(ph)), (T)(amp * sin(ph)));
    }
    A[e] = v;
  }
}

template <typename T>
__global__ void k_scale(C<T>* A, long long n, double s) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    C<T> a = A[e];
    A[e] = mk<C<T>>((T)(a.x * s), (T)(a.y * s));
  }
}

// dealiased copy (for flux): B = D(A) on ncomp components
template <typename T>
__global__ void k_dealias_copy(const C<T>* __restrict__ A, C<T>* B, int ncomp, Geo g) {
  // component blockIdx.y; 32-bit index arithmetic (a component holds < 2^31 modes)
  const int n = (int)g.S;
  const long long off = (long long)blockIdx.y * g.S;
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
    const int lz = m % g.Hz, r = m / g.Hz;
    const int ly = r % g.Ny, lx = r / g.Ny;
    B[off + m] = dealias_zero(g.dealias, g.basis, lx, ly, lz, g.Nx, g.Ny, g.Nz) ? mk<C<T>>(0, 0) : A[off + m];
  }
}

// ---------------------------------------------------------------------------
// SSS basis: sine/cosine transforms along z of real data (z lines contiguous, the
// padded real layout of N + 2 values per line).  Same algorithm as the x / y
// passes (one N-point FFT per line of the reordered sequence v), with the FFT
// done by the z real-to-complex / complex-to-real kernels and the reordering and
// the quarter-step twiddles e^{-i pi m / 2N} (tq, 4N entries) in these kernels.
// ---------------------------------------------------------------------------
// v_k = u_{2k} (k < N/2), +-u_{2(N-1-k)+1} (k >= N/2; minus for the sine series)
template <typename T>
__global__ void k_sss_zperm_fwd(const T* __restrict__ u, T* __restrict__ v, long long nlines, int N, int sine) {
  const long long n = nlines * (N + 2);
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / (N + 2);
    const int k = (int)(e % (N + 2));
    const T* ul = u + l * (N + 2);
    T x = 0;
    if (k < N / 2) x = ul[2 * k];
    else if (k < N) x = sine ? -ul[2 * (N - 1 - k) + 1] : ul[2 * (N - 1 - k) + 1];
    v[e] = x;
  }
}
// real coefficients from the half spectrum Z of v: c_m = 2 scl Re(w_m Z_m) (cosine),
// -2 scl Im(w_m Z_m) (sine), Z_m = conj(Z_{N-m}) above N/2
template <typename T>
__global__ void k_sss_zpost_fwd(const C<T>* __restrict__ Z, T* __restrict__ c, long long nlines, int N, int sine,
                                double scl, const C<T>* __restrict__ tq) {
  typedef C<T> V;
  const int H = N / 2 + 1;
  const long long n = nlines * (N + 2);
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / (N + 2);
    const int m = (int)(e % (N + 2));
    T out = 0;
    if (m < N) {
      const V* Zl = Z + l * H;
      const V zm = m <= N / 2 ? Zl[m] : conjg(Zl[N - m]);
      const V t = mul(tq[m], zm);
      out = sine ? (T)(-2.0 * scl) * t.y : (T)(2.0 * scl) * t.x;
    }
    c[e] = out;
  }
}
// half spectrum V of the inverse: V_m = conj(w_m) (c_m - i c_{N-m}) (cosine, V_0 = c_0),
// conj(w_m) (s_{N-m} - i s_m) (sine, V_0 = 0); c_N = s_N = 0
template <typename T>
__global__ void k_sss_zpre_inv(const T* __restrict__ c, C<T>* __restrict__ Vout, long long nlines, int N, int sine,
                               const C<T>* __restrict__ tq) {
  typedef C<T> V;
  const int H = N / 2 + 1;
  const long long n = nlines * H;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / H;
    const int m = (int)(e % H);
    const T* cl = c + l * (N + 2);
    V z;
    if (m == 0) {
      z = mk<V>(sine ? (T)0 : cl[0], 0);
    } else {
      const T a = sine ? cl[N - m] : cl[m], b = sine ? cl[m] : cl[N - m];
      z = mul(conjg(tq[m]), mk<V>(a, -b));
    }
    Vout[e] = z;
  }
}
// u_{2k} = v_k, u_{2k+1} = v_{N-1-k}; the sine series negates the odd points
template <typename T>
__global__ void k_sss_zperm_inv(const T* __restrict__ v, T* __restrict__ u, long long nlines, int N, int sine) {
  const long long n = nlines * (N + 2);
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / (N + 2);
    const int q = (int)(e % (N + 2));
    T x = 0;
    if (q < N) {
      const int h = q >> 1;  // (q - 1) / 2 for odd q, q / 2 for even q
      const int k = (q & 1) ? N - 1 - h : h;
      x = v[l * (N + 2) + k];
      if (sine && (q & 1)) x = -x;
    }
    u[e] = x;
  }
}

}  // namespace ts
