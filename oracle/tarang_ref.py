"""FP64 CPU oracle for the Tarang-2 pseudo-spectral IF-RK4 hot path.

TEST INFRASTRUCTURE ONLY.  This module is the checker for the CUDA product
path: only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it.  The product path
(``tarang_b200``) never calls it and fails loudly when its CUDA library is
missing.

What it restates (file:line are paths inside anandogc/tarang ``trunk/lib``):

* FFF basis index maps, wavenumbers, multiplicity   basis/FFF/pencil/FFF_pencil_inline.h:63-111,486-504,583-602
* FFF transforms (FFTK over FFTW, forward / N^3)    basis/FFF/pencil/FFF_pencil_tr.cc:43-66
* i k derivatives                                    basis/FFF/pencil/FFF_pencil_tr.cc:70-145
* dealias (corner box, intersection semantics)       basis/FFF/pencil/FFF_pencil_basic.cc:87-90,228-259
* strong reality condition                           basis/FFF/pencil/FFF_pencil_basic.cc:139-179
* conservative nonlinear term                        fluid/incompressible/nlin/compute_nlin.cc:58-109,
                                                     fluid/incompressible/nlin/compute_diag_offdiag.cc:47-112
* pressure / projection / rhs                        fluid/incompressible/Pressure.cc:56-72,
                                                     basis/basicfn/universal_basic.cc:202-225,343-363,
                                                     fluid/incompressible/time_advance/Tadvance_functions.cc:45-53,148-191
* IF-RK4 with the Single_time_step branch table      fluid/incompressible/time_advance/RK.cc:91-170,
                                                     Tadvance_functions.cc:298-324,566-570,
                                                     fluid/fluid_base/FluidVF.cc:308-389
* Carati constant energy supply (non-global alpha)   fluid/fluid_base/force/compute_force_Carati.cc:61-210,
                                                     force_alpha_beta.cc:56-85, compute_force_main.cc:43-80
* shell spectrum E(k) (Stepanov normalisation)       basis/basicfn/universal_energy.cc:279-366
* modes_in_shell                                     basis/basicfn/universal_basic.cc:104-143
* total energy                                       basis/FFF/pencil/FFF_pencil_energy.cc:59-68, fields/Cvf.cc:213-221
* energy flux Pi(R) per sphere                       fluid/incompressible/energytr/compute_flux.cc:51-65,
                                                     fill_space.cc:56-64, prod_nlinV.cc:61-69,
                                                     basis/basicfn/universal_ET.cc:51-70
* helical random-phase IC construction               fluid/fluid_base/io/input/init_cond_energy.cc:67-120,
                                                     fields/Cvf.cc:387-452, FFF_pencil_inline.h:228-247,819-845,
                                                     basis/basicfn/basicfn_inline.h:357-405
* SFF basis (sin/cos along x)                        basis/SFF/pencil/SFF_pencil_tr.cc:43-174,
                                                     SFF_pencil_basic.cc:94-97,143-167,
                                                     SFF_pencil_inline.h:63-109,412-430,492-515,
                                                     SFF_pencil_energy.cc:76-95, global/Global.cc:137-165
* Boussinesq RBC step (PRLARGE / ULARGE)             fluid/incompressible/time_advance/RK_SF.cc:97-221,
                                                     Tadvance_functions.cc:57-90,226-237,372-395,477-489,589-611,
                                                     fluid/incompressible/nlin/compute_nlin_SF.cc:75-142,
                                                     compute_diag_offdiag.cc:116-136,
                                                     fluid/fluid_base/force/compute_force_RBC.cc:104-150,
                                                     fluid/fluid_base/Correlation.cc:144-160
* discrete adjoint of the FFF rotational IF-RK4 step  (no reference counterpart: the exact transpose of
                                                     rk4_step, derived in the adjoint section below)

Parity status: the transform arithmetic of the reference lives in the
un-vendored FFTK library (no source, no version pin) and the reference ships
no golden vectors or tests, so parity at the FFTK boundary is UNPINNED.  The
FFF convention (forward divides by N^3, inverse unscaled) is inferred from the
reference's energy functions and Taylor-Green IC and checked here by
known-answer tests.  The SFF x-grid stagger (type-II/III sin/cos pair) is a
choice, pinned only by the energy / Parseval identities.

Random initial conditions use this project's counter-based splitmix64
generator (the reference seeds Blitz++ with ``my_id*time(0)``,
init_cond_energy.cc:75-76, which is not reproducible); the CUDA library
implements the same generator bit-for-bit.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np
import scipy.fft as sfft

MYEPS = 1e-15    # global/Global.cc:62
MYEPS2 = 1e-5    # global/Global.cc:63

DEALIAS_NONE = 0
DEALIAS_REFERENCE_CORNER = 1
DEALIAS_TWO_THIRDS = 2

WORKERS = int(os.environ.get("TS_ORACLE_WORKERS", os.cpu_count() or 1))


# ----------------------------------------------------------------------------
# counter-based RNG (this project's own; identical in csrc/ic.cu)
# ----------------------------------------------------------------------------
_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser (Steele, Lea & Flood 2014) on a uint64 array."""
    with np.errstate(over="ignore"):
        z = (x + np.uint64(0x9E3779B97F4A7C15)) & _M64
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M64
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M64
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, counter: np.ndarray) -> np.ndarray:
    """U[0,1) double from (seed, counter): splitmix64(splitmix64(seed) ^ counter) >> 11."""
    key = _splitmix64(np.array([seed], dtype=np.uint64))[0]
    h = _splitmix64(key ^ counter.astype(np.uint64))
    return (h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


# ----------------------------------------------------------------------------
# grid / basis
# ----------------------------------------------------------------------------
@dataclass
class Grid:
    """Spectral grid of one field: complex shape (Nx, Ny, Nz//2+1), C order.

    FFF: kx, ky in FFT order (``Get_kx`` FFF_pencil_inline.h:63, ``Get_ky`` :94),
    kz = 0..Nz/2 (:107).  SFF: kx = lx = 0..Nx-1 (SFF_pencil_inline.h:63).
    ``kfactor`` is (kf1, kf2, kf3), i.e. the reference's kfactor[1..3].
    """
    N: tuple
    kfactor: tuple = (1.0, 1.0, 1.0)
    basis: str = "FFF"
    kx: np.ndarray = field(init=False)
    ky: np.ndarray = field(init=False)
    kz: np.ndarray = field(init=False)

    def __post_init__(self):
        Nx, Ny, Nz = self.N
        lx = np.arange(Nx)
        if self.basis == "FFF":
            self.kx = np.where(lx <= Nx // 2, lx, lx - Nx)
        elif self.basis in ("SFF", "SSF", "SSS"):
            self.kx = lx.copy()
        else:
            raise ValueError(self.basis)
        ly = np.arange(Ny)
        # SSF: sin/cos along y as well, ky = ly (SSF_pencil_inline.h Get_ky)
        self.ky = ly.copy() if self.basis in ("SSF", "SSS") else np.where(ly <= Ny // 2, ly, ly - Ny)
        # SSS: sin/cos along z as well, real coefficients (Nx, Ny, Nz), kz = lz (SSS_pencil_inline.h)
        self.kz = np.arange(Nz) if self.basis == "SSS" else np.arange(Nz // 2 + 1)

    @property
    def shape(self):
        Nx, Ny, Nz = self.N
        return (Nx, Ny, Nz) if self.basis == "SSS" else (Nx, Ny, Nz // 2 + 1)

    @property
    def rshape(self):
        return tuple(self.N)

    def K(self):
        kf = self.kfactor
        Kx = (self.kx * kf[0]).astype(np.float64)[:, None, None]
        Ky = (self.ky * kf[1]).astype(np.float64)[None, :, None]
        Kz = (self.kz * kf[2]).astype(np.float64)[None, None, :]
        return Kx, Ky, Kz

    def Ksqr(self):
        Kx, Ky, Kz = self.K()
        # universal_basic.cc:202-225 accumulates Kx^2 + Ky^2 + Kz^2 in this order
        return (Kx ** 2 + Ky ** 2) + Kz ** 2

    def Kmag(self):
        return np.sqrt(self.Ksqr())

    def multiplicity(self):
        """Multiplicity_factor: FFF_pencil_inline.h:583-602, SFF_pencil_inline.h:492-515."""
        Nx, Ny, Nz = self.N
        kx = self.kx[:, None, None]
        ky = self.ky[None, :, None]
        kz = self.kz[None, None, :]
        if self.basis == "FFF":
            f = np.where(kz > 0, 1.0, 0.5)
            dbl = (kx == Nx // 2) | ((ky == Ny // 2) & (Ny > 1))
            return np.broadcast_to(np.where(dbl, 2 * f, f), self.shape).copy()
        if self.basis in ("SSF", "SSS"):
            # SSF_pencil_inline.h:512-532, SSS_pencil_inline.h:537-556: 1/2 at the origin, 1 with
            # two zero indices, 2 with one, 4 with none (grid indices kx = lx, ly, lz)
            zeros = (kx == 0).astype(int) + (ky == 0).astype(int) + (kz == 0).astype(int)
            f = np.choose(np.minimum(zeros, 3), [4.0, 2.0, 1.0, 0.5])
            return np.broadcast_to(f, self.shape).copy()
        m = kx
        f = np.where(kz > 0, np.where(m > 0, 2.0, 1.0), np.where(m > 0, 1.0, 0.5))
        dbl = (ky == Ny // 2) & (Ny > 1)
        return np.broadcast_to(np.where(dbl, 2 * f, f), self.shape).copy()

    def min_radius_outside(self):
        """Min_radius_outside: FFF_pencil_inline.h:497-504, SFF_pencil_inline.h:423-430,
        SSF_pencil_inline.h:444-451, SSS_pencil_inline.h:469-476."""
        Nx, Ny, Nz = self.N
        kf = self.kfactor
        if self.basis == "FFF":
            return int(math.ceil(math.sqrt((Nx // 2 * kf[0]) ** 2 + (Ny // 2 * kf[1]) ** 2 + (Nz // 2 * kf[2]) ** 2)))
        if self.basis == "SSF":
            return int(math.ceil(math.sqrt(((Nx - 1) * kf[0]) ** 2 + ((Ny - 1) * kf[1]) ** 2 + (Nz // 2 * kf[2]) ** 2)))
        if self.basis == "SSS":
            return int(math.ceil(math.sqrt(((Nx - 1) * kf[0]) ** 2 + ((Ny - 1) * kf[1]) ** 2 + ((Nz - 1) * kf[2]) ** 2)))
        return int(math.ceil(math.sqrt(((Nx - 1) * kf[0]) ** 2 + (Ny // 2 * kf[1]) ** 2 + (Nz // 2 * kf[2]) ** 2)))

    def n_shells(self):
        return self.min_radius_outside() + 1

    def modes_in_shell(self):
        """Compute_modes_in_shell_array: universal_basic.cc:104-143 (full box count)."""
        Nx, Ny, Nz = self.N
        kf = self.kfactor
        kxm, kym, kzm = Nx // 2, Ny // 2, Nz // 2
        kx = np.arange(-kxm + 1, kxm + 1) * kf[0]
        ky = np.arange(-kym + 1, kym + 1) * kf[1]
        kz = np.arange(-kzm + 1, kzm + 1) * kf[2]
        Kmag = np.sqrt(kx[:, None, None] ** 2 + ky[None, :, None] ** 2 + kz[None, None, :] ** 2)
        idx = np.ceil(Kmag).astype(np.int64).ravel()
        size = max(self.n_shells(), int(idx.max()) + 1)
        return np.bincount(idx, minlength=size).astype(np.float64)


# ----------------------------------------------------------------------------
# dealias and reality
# ----------------------------------------------------------------------------
def dealias_mask(g: Grid, mode: int) -> np.ndarray:
    """Boolean mask of modes ZEROED by the dealias step.

    REFERENCE_CORNER restates FFF_PENCIL::Dealias (FFF_pencil_basic.cc:87-90 ->
    Assign_sub_array :228-259): only the box where lx in [Nx/3+1, 2Nx/3-1] AND
    ly in [Ny/3+1, 2Ny/3-1] AND lz in [Nz/3+1, Nz/2] (array indices) is zeroed.
    SFF: lx in [2Nx/3+1, Nx-1] AND the same y/z ranges (SFF_pencil_basic.cc:94-97).
    TWO_THIRDS zeroes every mode with 3|k_i| > N_i on any axis (3 m > 2 Nx on the
    SFF sin/cos axis).
    """
    Nx, Ny, Nz = g.N
    lx = np.arange(Nx)[:, None, None]
    ly = np.arange(Ny)[None, :, None]
    lz = np.arange(Nz // 2 + 1)[None, None, :]
    if mode == DEALIAS_NONE:
        return np.zeros(g.shape, dtype=bool)
    if mode == DEALIAS_REFERENCE_CORNER and g.basis == "SSS":
        # SSS_PENCIL::Dealias (SSS_pencil_basic.cc:129-134): lx >= 2Nx/3+1, ly >= 2Ny/3+1, lz >= Nz/3
        lzr = np.arange(Nz)[None, None, :]
        return np.broadcast_to((lx >= 2 * Nx // 3 + 1) & (ly >= 2 * Ny // 3 + 1) & (lzr >= Nz // 3), g.shape).copy()
    if mode == DEALIAS_REFERENCE_CORNER:
        if g.basis == "FFF":
            mx = (lx >= Nx // 3 + 1) & (lx <= 2 * Nx // 3 - 1)
        else:
            mx = lx >= 2 * Nx // 3 + 1
        if g.basis == "SSF":
            # SSF_PENCIL::Dealias (SSF_pencil_basic.cc:103-106): lx >= 2Nx/3+1, ly >= 2Ny/3+1, lz >= Nz/3+1
            my = ly >= 2 * Ny // 3 + 1
        else:
            my = (ly >= Ny // 3 + 1) & (ly <= 2 * Ny // 3 - 1)
        mz = (lz >= Nz // 3 + 1) & (lz <= Nz // 2)
        return np.broadcast_to(mx & my & mz, g.shape).copy()
    if mode == DEALIAS_TWO_THIRDS:
        kx = g.kx[:, None, None]
        ky = g.ky[None, :, None]
        kz = g.kz[None, None, :]
        if g.basis == "FFF":
            bx = 3 * np.abs(kx) > Nx
        else:
            bx = 3 * kx > 2 * Nx
        by = (3 * ky > 2 * Ny) if g.basis in ("SSF", "SSS") else (3 * np.abs(ky) > Ny)
        bz = (3 * kz > 2 * Nz) if g.basis == "SSS" else (3 * kz > Nz)
        m = bx | by | bz
        return np.broadcast_to(m, g.shape).copy()
    raise ValueError(mode)


def dealias(g: Grid, A: np.ndarray, mode: int) -> np.ndarray:
    B = A.copy()
    B[..., dealias_mask(g, mode)] = 0
    return B


def reality_fix(g: Grid, A: np.ndarray) -> np.ndarray:
    """Satisfy_strong_reality_condition_in_Array on one complex array.

    FFF (FFF_pencil_basic.cc:139-179): for kx<0 and ky != Ny/2,
    A(kx,ky,0) = conj(A(-kx,-ky,0)); for kx=0, ky<0, A(0,ky,0) = conj(A(0,-ky,0));
    then the kz=Nz/2 plane is zeroed.
    SFF (SFF_pencil_basic.cc:143-167): for every m and ky<=0,
    A(m,ky,0) = conj(A(m,-ky,0)); kz=Nz/2 plane zeroed.
    """
    Nx, Ny, Nz = g.N
    B = A.copy()
    if g.basis in ("SSF", "SSS"):
        return B  # SSF_pencil_basic.cc:127-130 (and SSS): nothing to do
    plane = A[:, :, 0].copy()
    iy_minus = (-g.ky) % Ny  # Get_iy(-ky)
    if g.basis == "FFF":
        for lx in range(Nx // 2 + 1, Nx):
            mkx = -g.kx[lx]
            sel = g.ky != Ny // 2
            B[lx, sel, 0] = np.conj(plane[mkx, iy_minus[sel]])
        sel = g.ky < 0
        B[0, sel, 0] = np.conj(plane[0, iy_minus[sel]])
    else:
        sel = g.ky <= 0
        B[:, sel, 0] = np.conj(plane[:, iy_minus[sel]])
    B[:, :, Nz // 2] = 0
    return B


def reality_fix_vec(g: Grid, V: np.ndarray) -> np.ndarray:
    return np.stack([reality_fix(g, V[i]) for i in range(V.shape[0])])


# ----------------------------------------------------------------------------
# transforms
# ----------------------------------------------------------------------------
def _x_forward_sincos(g: Grid, B: np.ndarray, parity: str, axis: int = 0) -> np.ndarray:
    """Sine/cosine analysis along x (axis 0; y for the SSF basis, axis 1) with the FFTW
    RODFT10/REDFT10 scaling / (2 N).

    Sine: coefficient of 2 sin(m pi x/Lx) stored at lx=m for m=1..Nx-1 (lx=0 is 0,
    the m=Nx coefficient is dropped).  Cosine: c_0 + sum 2 c_m cos(m pi x/Lx), m=0..Nx-1.
    Staggered grid x_j = (j+1/2) Lx/Nx (type-II forward / type-III inverse).
    """
    N = g.N[axis]
    if parity == "S":
        Y = sfft.dst(B, type=2, axis=axis, workers=WORKERS) / (2.0 * N)
        Y = np.moveaxis(Y, axis, 0)
        out = np.zeros_like(Y)
        out[1:] = Y[:-1]
        return np.moveaxis(out, 0, axis)
    if parity == "C":
        return sfft.dct(B, type=2, axis=axis, workers=WORKERS) / (2.0 * N)
    raise ValueError(parity)


def _x_inverse_sincos(g: Grid, A: np.ndarray, parity: str, axis: int = 0) -> np.ndarray:
    if parity == "S":
        Am = np.moveaxis(A, axis, 0)
        Y = np.zeros_like(Am)
        Y[:-1] = Am[1:]
        return sfft.dst(np.moveaxis(Y, 0, axis), type=3, axis=axis, workers=WORKERS)
    if parity == "C":
        return sfft.dct(A, type=3, axis=axis, workers=WORKERS)
    raise ValueError(parity)


def forward(g: Grid, ur: np.ndarray, parity: str = "F") -> np.ndarray:
    """Real (Nx,Ny,Nz) -> spectral (Nx,Ny,Nz/2+1).  FFF: A = N^-3 sum u e^{-ik.x}."""
    if g.basis == "FFF":
        return sfft.rfftn(ur, norm="forward", workers=WORKERS)
    if g.basis == "SSF":
        # SSF_pencil_tr.cc:43-51: sin/cos along x and y by the parity's first two letters
        Bz = sfft.rfft(ur, axis=2, norm="forward", workers=WORKERS)
        return _x_forward_sincos(g, _x_forward_sincos(g, Bz, parity[1], axis=1), parity[0])
    if g.basis == "SSS":
        # SSS_pencil_tr.cc: sin/cos along every axis, real coefficients
        B = _x_forward_sincos(g, ur, parity[2], axis=2)
        return _x_forward_sincos(g, _x_forward_sincos(g, B, parity[1], axis=1), parity[0])
    Byz = sfft.rfftn(ur, axes=(1, 2), norm="forward", workers=WORKERS)
    return _x_forward_sincos(g, Byz, parity)


def inverse(g: Grid, A: np.ndarray, parity: str = "F") -> np.ndarray:
    """Spectral -> real, unnormalised (u = sum A e^{ik.x}); imag of kz=0 and kz=Nz/2 ignored."""
    if g.basis == "FFF":
        return sfft.irfftn(A, s=g.rshape, norm="forward", workers=WORKERS)
    Nx, Ny, Nz = g.N
    if g.basis == "SSF":
        Bxy = _x_inverse_sincos(g, _x_inverse_sincos(g, A, parity[0]), parity[1], axis=1)
        return sfft.irfft(Bxy, n=Nz, axis=2, norm="forward", workers=WORKERS)
    if g.basis == "SSS":
        Bxy = _x_inverse_sincos(g, _x_inverse_sincos(g, A, parity[0]), parity[1], axis=1)
        return _x_inverse_sincos(g, Bxy, parity[2], axis=2)
    Bx = _x_inverse_sincos(g, A, parity)
    return sfft.irfftn(Bx, s=(Ny, Nz), axes=(1, 2), norm="forward", workers=WORKERS)


# ----------------------------------------------------------------------------
# derivatives (FFF: i K ; SFF x: real factor by parity)
# ----------------------------------------------------------------------------
def xderiv(g: Grid, A: np.ndarray, parity: str = "F") -> np.ndarray:
    """FFF_pencil_tr.cc:70-79 (i Kx); SFF_pencil_tr.cc:77-90 and SSF_pencil_tr.cc:69-90
    (x parity S -> +Kx, C -> -Kx)."""
    Kx, _, _ = g.K()
    if g.basis == "FFF":
        return (1j * Kx) * A
    return (Kx if parity[0] == "S" else -Kx) * A


def yderiv(g: Grid, A: np.ndarray, parity: str = "F") -> np.ndarray:
    """i Ky; SSF (SSF_PENCIL::Yderiv): y parity S -> +Ky, C -> -Ky."""
    _, Ky, _ = g.K()
    if g.basis in ("SSF", "SSS"):
        return (Ky if parity[1] == "S" else -Ky) * A
    return (1j * Ky) * A


def zderiv(g: Grid, A: np.ndarray, parity: str = "F") -> np.ndarray:
    """i Kz; SSS (SSS_PENCIL::Zderiv, SSS_pencil_tr.cc:171-189): z parity S -> +Kz, C -> -Kz."""
    _, _, Kz = g.K()
    if g.basis == "SSS":
        return (Kz if parity[2] == "S" else -Kz) * A
    return (1j * Kz) * A


# SFF parity strings (global/Global.cc:137-145) -> first letter is the x parity
SFF_PARITY = {"Vx": "S", "Vy": "C", "Vz": "C", "div": "C", "Vi2": "C", "VxVy": "S", "VxVz": "S",
              "VyVz": "C", "F": "S", "FVx": "C", "FVy": "S", "FVz": "S"}


# SSF parity strings for sincostr_switch "SCF" (global/Global.cc:184-191): x, y, z letters
SSF_PARITY = {"Vx": "SCF", "Vy": "CSF", "Vz": "CCF", "div": "CCF", "Vi2": "CCF", "VxVy": "SSF", "VxVz": "SCF",
              "VyVz": "CSF"}


# SSS parity strings for sincostr_switch "SCC" (global/Global.cc:221-228)
SSS_PARITY = {"Vx": "SCC", "Vy": "CSC", "Vz": "CCS", "div": "CCC", "Vi2": "CCC", "VxVy": "SSC", "VxVz": "SCS",
              "VyVz": "CSS"}

# a scalar F (the temperature) takes the Vx parity on every basis and the products
# u_x F, u_y F, u_z F take Vi2, VxVy and VxVz (Global_process_basic_vars.cc:108, 114-116)
for _tab in (SSF_PARITY, SSS_PARITY):
    _tab.update(F=_tab["Vx"], FVx=_tab["Vi2"], FVy=_tab["VxVy"], FVz=_tab["VxVz"])


def _par(g: Grid, key: str) -> str:
    if g.basis == "SSS":
        return SSS_PARITY[key]
    if g.basis == "SSF":
        return SSF_PARITY[key]
    return "F" if g.basis == "FFF" else SFF_PARITY[key]


# ----------------------------------------------------------------------------
# nonlinear term
# ----------------------------------------------------------------------------
def velocity_real(g: Grid, V: np.ndarray) -> list:
    """CVF::Inverse_transform (fields/Cvf.cc:172-185) with the Vx/Vy/Vz parities."""
    return [inverse(g, V[0], _par(g, "Vx")), inverse(g, V[1], _par(g, "Vy")), inverse(g, V[2], _par(g, "Vz"))]


def nlin_conservative_from_real(g: Grid, ur: list, wr: list | None = None) -> np.ndarray:
    """N_i = sum_j D_j F[u_j w_i] in the reference's accumulation order.

    Compute_nlin_diag / Compute_nlin_offdiag (compute_diag_offdiag.cc:47-98) for
    w = u, and the giver form (compute_nlin_ET_VF.cc:71-87) for w given.
    """
    if wr is None:
        wr = ur
    p = lambda k: _par(g, k)
    n1 = xderiv(g, forward(g, ur[0] * wr[0], p("Vi2")), p("Vi2"))
    n2 = yderiv(g, forward(g, ur[1] * wr[1], p("Vi2")), p("Vi2"))
    n3 = zderiv(g, forward(g, ur[2] * wr[2], p("Vi2")), p("Vi2"))
    if wr is ur:
        X = forward(g, ur[0] * ur[1], p("VxVy"))
        n1 = n1 + yderiv(g, X, p("VxVy"))
        n2 = n2 + xderiv(g, X, p("VxVy"))
        X = forward(g, ur[1] * ur[2], p("VyVz"))
        n2 = n2 + zderiv(g, X, p("VyVz"))
        n3 = n3 + yderiv(g, X, p("VyVz"))
        X = forward(g, ur[2] * ur[0], p("VxVz"))
        n1 = n1 + zderiv(g, X, p("VxVz"))
        n3 = n3 + xderiv(g, X, p("VxVz"))
    else:
        # giver form: nlin_i = sum_j D_j F[u_j w_i]
        n1 = n1 + yderiv(g, forward(g, ur[1] * wr[0], p("VxVy")), p("VxVy")) \
            + zderiv(g, forward(g, ur[2] * wr[0], p("VxVz")), p("VxVz"))
        n2 = n2 + xderiv(g, forward(g, ur[0] * wr[1], p("VxVy")), p("VxVy")) \
            + zderiv(g, forward(g, ur[2] * wr[1], p("VyVz")), p("VyVz"))
        n3 = n3 + xderiv(g, forward(g, ur[0] * wr[2], p("VxVz")), p("VxVz")) \
            + yderiv(g, forward(g, ur[1] * wr[2], p("VyVz")), p("VyVz"))
    return np.stack([n1, n2, n3])


def nlin_conservative(g: Grid, V: np.ndarray) -> np.ndarray:
    """Compute_nlin on an already-dealiased field (compute_nlin.cc:58-109)."""
    return nlin_conservative_from_real(g, velocity_real(g, V))


def vorticity(g: Grid, V: np.ndarray) -> np.ndarray:
    """omega = i K x V (FFF; Compute_vorticity universal_basic.cc:49-66)."""
    Kx, Ky, Kz = g.K()
    return np.stack([1j * (Ky * V[2] - Kz * V[1]), 1j * (Kz * V[0] - Kx * V[2]), 1j * (Kx * V[1] - Ky * V[0])])


def nlin_rotational(g: Grid, V: np.ndarray) -> np.ndarray:
    """N = -F[u x omega] (FFF only): equals the conservative N up to a gradient and aliasing."""
    if g.basis != "FFF":
        raise ValueError("rotational form is implemented for FFF only")
    u = [inverse(g, V[i]) for i in range(3)]
    W = vorticity(g, V)
    w = [inverse(g, W[i]) for i in range(3)]
    c1 = u[1] * w[2] - u[2] * w[1]
    c2 = u[2] * w[0] - u[0] * w[2]
    c3 = u[0] * w[1] - u[1] * w[0]
    return -np.stack([forward(g, c1), forward(g, c2), forward(g, c3)])


# ----------------------------------------------------------------------------
# projection / rhs
# ----------------------------------------------------------------------------
def project_rhs(g: Grid, N: np.ndarray) -> np.ndarray:
    """Pressure::Compute_pressure + Compute_rhs: N <- -(N + D p), p = div(N)/K^2, p(0)=0.

    Pressure.cc:56-72, universal_basic.cc:202-225 (divide, A(0,0,0)=0),
    Compute_divergence universal_basic.cc:343-352, Add_pressure_gradient and
    Compute_rhs Tadvance_functions.cc:148-191.  SFF parities: div with Vx
    (S -> +Kx), gradient with div parity (C -> -Kx).
    """
    div = xderiv(g, N[0], _par(g, "Vx")) + yderiv(g, N[1], _par(g, "Vy")) + zderiv(g, N[2], _par(g, "Vz"))
    K2 = g.Ksqr()
    with np.errstate(divide="ignore", invalid="ignore"):
        p = div / K2
    p[0, 0, 0] = 0
    n1 = N[0] + xderiv(g, p, _par(g, "div"))
    n2 = N[1] + yderiv(g, p, _par(g, "div"))
    n3 = N[2] + zderiv(g, p, _par(g, "div"))
    return -np.stack([n1, n2, n3])


def max_abs_div(g: Grid, V: np.ndarray) -> float:
    """max |div V| as in Universal::Compute_divergence(field) universal_basic.cc:343-356."""
    div = xderiv(g, V[0], _par(g, "Vx")) + yderiv(g, V[1], _par(g, "Vy")) + zderiv(g, V[2], _par(g, "Vz"))
    return float(np.max(np.abs(div)))


# ----------------------------------------------------------------------------
# forcing: Carati constant energy supply, non-global alpha/beta
# ----------------------------------------------------------------------------
@dataclass
class CaratiForcing:
    inner_radius: float
    outer_radius: float
    energy_supply: np.ndarray      # per shell index (ceil |K|)
    helicity_supply: np.ndarray | None = None


def carati_force(g: Grid, V: np.ndarray, f: CaratiForcing, modes_in_shell: np.ndarray) -> np.ndarray:
    """F = alpha V + beta omega on the band inner < |K| <= outer.

    compute_force_Carati.cc:61-75 (no-forcing early exit), :158-205 (non-global
    alpha/beta per mode), force_alpha_beta.cc:56-85 (F = alpha u + beta omega),
    then compute_force_main.cc:67-73 (strong reality condition on F).
    Modal energy |V|^2/2 (FFF_pencil_inline.h:607-610), modal helicity
    K.(Re V x Im V) (:618-634), modal vorticity i K x V (:646-664).
    """
    F = np.zeros_like(V)
    es = np.asarray(f.energy_supply, dtype=np.float64)
    hs = np.zeros_like(es) if f.helicity_supply is None else np.asarray(f.helicity_supply, dtype=np.float64)
    if abs(es.sum()) + abs(hs.sum()) < MYEPS:
        return F
    Kmag = g.Kmag()
    band = (Kmag > f.inner_radius) & (Kmag <= f.outer_radius)
    # the reference loops kx in [-kx_max, kx_max] etc. (kx_max = ceil(outer/kf)); with
    # outer < N/2 every stored band mode is visited exactly once.
    Kx, Ky, Kz = g.K()
    Kx = np.broadcast_to(Kx, g.shape)
    Ky = np.broadcast_to(Ky, g.shape)
    Kz = np.broadcast_to(Kz, g.shape)
    W = vorticity(g, V)
    idxs = np.argwhere(band)
    for (lx, ly, lz) in idxs:
        K = Kmag[lx, ly, lz]
        index = int(math.ceil(K))
        v = V[:, lx, ly, lz]
        modal_energy = float(np.sum(np.abs(v) ** 2) / 2)
        if modal_energy > MYEPS:
            eps_k = es[index] / modes_in_shell[index]
            hel_k = hs[index] / modes_in_shell[index]
            vr, vi = v.real, v.imag
            Kv = np.array([Kx[lx, ly, lz], Ky[lx, ly, lz], Kz[lx, ly, lz]])
            modal_hel = float(np.dot(Kv, np.cross(vr, vi)))
            denr = 2.0 * ((K * modal_energy) ** 2 - modal_hel ** 2)
            epsh_by_k_epse = hel_k / (K * eps_k) if eps_k != 0 else np.inf
            if abs(denr) > MYEPS:
                alpha = (K ** 2 * eps_k * modal_energy - hel_k * modal_hel) / denr
                beta = (hel_k * modal_energy - eps_k * modal_hel) / denr
            elif abs(epsh_by_k_epse - 1) < MYEPS:
                alpha = eps_k / (4 * modal_energy)
                beta = alpha / K
            else:
                raise RuntimeError("max helicity supply case")
            F[:, lx, ly, lz] = alpha * v + beta * W[:, lx, ly, lz]
    return reality_fix_vec(g, F)


# ----------------------------------------------------------------------------
# IF-RK4
# ----------------------------------------------------------------------------
@dataclass
class FluidConfig:
    grid: Grid
    nu: float
    dt: float
    dealias_mode: int = DEALIAS_REFERENCE_CORNER
    nlin_form: str = "conservative"        # or "rotational"
    reality_fix: bool = True
    forcing: CaratiForcing | None = None


def exp_ksqr(g: Grid, A: np.ndarray, factor: float) -> np.ndarray:
    """Array_exp_ksqr: A * exp(factor K^2) (universal_basic.cc:235-252)."""
    return A * np.exp(factor * g.Ksqr())


def fluid_rhs(cfg: FluidConfig, U: np.ndarray, mis: np.ndarray) -> tuple:
    """Compute_force_TO_rhs (Tadvance_functions.cc:441-453).

    Returns (rhs, dealiased U): the reference dealiases U in place inside
    Compute_nlin (compute_nlin.cc:61-62), and the caller's Single_time_step
    then works on the dealiased U.
    """
    g = cfg.grid
    F = None
    if cfg.forcing is not None:
        F = carati_force(g, U, cfg.forcing, mis)       # forcing sees the un-dealiased U
    Ud = dealias(g, U, cfg.dealias_mode) if cfg.dealias_mode else U.copy()
    if cfg.nlin_form == "conservative":
        N = nlin_conservative(g, Ud)
    else:
        N = nlin_rotational(g, Ud)
    if F is not None:
        N = N - F                                       # Add_force :45-53
    return project_rhs(g, N), Ud


def rk4_step(cfg: FluidConfig, U0: np.ndarray, mis: np.ndarray | None = None) -> np.ndarray:
    """Time_advance_incompress::RK4(U,P,F), RK.cc:91-170, then the reality fix
    (Time_advance.cc:59-60).  E(a) = exp(-nu K^2 a dt); Single_time_step branch
    table Tadvance_functions.cc:298-324; Compute_RK4_parts :566-570."""
    g = cfg.grid
    if mis is None:
        mis = g.modes_in_shell()
    nu, dt = cfg.nu, cfg.dt
    E = lambda A, a: exp_ksqr(g, A, -nu * a * dt)
    Vcopy = U0.copy()
    # stage 1: Single_time_step(.5,.5,.5): a==b -> Add then Mult
    R, Ud = fluid_rhs(cfg, U0, mis)
    U = E(Ud + (0.5 * dt) * R, 0.5)
    tot = (dt / 6.0) * E(R, 1.0)
    # stage 2: Single_time_step(.5,0,.5): b==0 -> Mult then Add
    R, _ = fluid_rhs(cfg, U, mis)
    U = E(Vcopy, 0.5) + (0.5 * dt) * R
    tot = tot + (dt / 3.0) * E(R, 0.5)
    # stage 3: Single_time_step(1,.5,1): Mult(a-b), Add, Mult(b)
    R, _ = fluid_rhs(cfg, U, mis)
    U = E(E(Vcopy, 0.5) + dt * R, 0.5)
    tot = tot + (dt / 3.0) * E(R, 0.5)
    # stage 4: Compute_RK4_parts(0, 1/6): no exp factor
    R, _ = fluid_rhs(cfg, U, mis)
    tot = tot + (dt / 6.0) * R
    U = E(Vcopy, 1.0) + tot
    if cfg.reality_fix:
        U = reality_fix_vec(g, U)
    return U


# ----------------------------------------------------------------------------
# diagnostics
# ----------------------------------------------------------------------------
def _sincos3_sum(d: np.ndarray, d0: float) -> float:
    """SSF / SSS Get_local_energy plane sums (SSF_pencil_energy.cc:76-103,
    SSS_pencil_energy.cc:69-98): 4 sum d, minus 2 on each of the lx = 0, ly = 0 and
    lz = 0 planes, plus the lines where two of them meet, minus d0 / 2 at the origin
    (d0 = the product of the real parts there)."""
    e = 4 * d.sum()
    e += -2 * d[0].sum() + d[0, :, 0].sum()
    e += d[0, 0, :].sum() - 0.5 * d0
    e += -2 * d[:, 0, :].sum() + d[:, 0, 0].sum()
    e += -2 * d[:, :, 0].sum()
    return float(e)


def total_energy(g: Grid, V: np.ndarray) -> float:
    """CVF::Compute_total_energy: per component sum|A|^2 - 1/2 sum_{kz=0}|A|^2 (FFF);
    SFF weights 2 / 1 / 1/2 (SFF_pencil_energy.cc:76-95); SSF and SSS weights
    4 / 2 / 1 / 1/2 by the number of zero indices (_sincos3_sum)."""
    e = 0.0
    for A in V:
        a2 = np.abs(A) ** 2
        if g.basis == "FFF":
            e += a2.sum() - 0.5 * a2[:, :, 0].sum()
        elif g.basis in ("SSF", "SSS"):
            e += _sincos3_sum(a2, float(np.real(A[0, 0, 0])) ** 2)
        else:
            e += 2 * a2.sum() - a2[:, :, 0].sum() - a2[0].sum() + 0.5 * a2[0, :, 0].sum()
    return float(e)


def total_energy_scalar(g: Grid, A: np.ndarray) -> float:
    return total_energy(g, A[None])


def cross_energy(g: Grid, A: np.ndarray, B: np.ndarray) -> float:
    """Get_local_energy(A,B) = mydot with the same plane weights (FFF_pencil_energy.cc:81-89)."""
    d = (A * np.conj(B)).real
    if g.basis == "FFF":
        return float(d.sum() - 0.5 * d[:, :, 0].sum())
    if g.basis in ("SSF", "SSS"):
        return _sincos3_sum(d, float(np.real(A[0, 0, 0]) * np.real(B[0, 0, 0])))
    return float(2 * d.sum() - d[:, :, 0].sum() - d[0].sum() + 0.5 * d[0, :, 0].sum())


def sss_complex_view(g: Grid, V: np.ndarray) -> tuple:
    """The complex view the reference's shell loop takes of SSS real coefficients: the pair
    (2 lz, 2 lz + 1) of a z line is one complex slot lz < Nz/2 (the loop runs over the complex
    array shape, universal_energy.cc:276-306, with kz = Get_kz(lz) = lz); returns the
    complex array and the Grid of that view (kz = 0 .. Nz/2 - 1)."""
    Nx, Ny, Nz = g.N
    A = V[..., 0:Nz:2] + 1j * V[..., 1:Nz:2]
    gc = Grid(g.N, g.kfactor, "SSS")
    gc.kz = np.arange(Nz // 2)
    return A, gc


def shell_spectrum(g: Grid, V: np.ndarray, n: int = 0) -> np.ndarray:
    """Compute_shell_spectrum per component and summed (universal_energy.cc:279-366).

    Sk(ceil|K|) += mult |K|^n |A|^2 |K|^2; count += 2 mult; Sk *= 4 pi /(count kf1 kf2 kf3).
    SSS: over the complex view of the real coefficients (``sss_complex_view``).
    """
    if g.basis == "SSS":
        V, gc = sss_complex_view(g, V)
        kmax = g.min_radius_outside()
        g = gc
    else:
        kmax = g.min_radius_outside()
    Kmag = g.Kmag()
    idx = np.ceil(Kmag).astype(np.int64)
    mult = np.broadcast_to(g.multiplicity(), Kmag.shape) if g.basis != "SSS" else _sss_mult(g)
    ok = idx <= kmax
    nsh = kmax + 1
    count = np.bincount(idx[ok], weights=2 * mult[ok], minlength=nsh)
    kf = g.kfactor
    out = np.zeros(nsh)
    for A in V:
        w = mult * (Kmag ** n) * (np.abs(A) ** 2) * Kmag ** 2
        Sk = np.bincount(idx[ok], weights=w[ok], minlength=nsh)
        with np.errstate(divide="ignore", invalid="ignore"):
            Sk = np.where(count > 0, Sk * 4 * math.pi / (count * kf[0] * kf[1] * kf[2]), 0.0)
        out += Sk
    return out


def _sss_mult(g: Grid) -> np.ndarray:
    """SSS Multiplicity_factor on the complex view (kz = lz < Nz/2)."""
    kx = g.kx[:, None, None]
    ky = g.ky[None, :, None]
    kz = g.kz[None, None, :]
    zeros = (kx == 0).astype(int) + (ky == 0).astype(int) + (kz == 0).astype(int)
    return np.choose(np.minimum(zeros, 3), [4.0, 2.0, 1.0, 0.5]).astype(np.float64)


def shell_mult_single(g: Grid, A: np.ndarray, B: np.ndarray, inner: float, outer: float) -> float:
    """Local_shell_mult_single universal_ET.cc:51-70: sum 2 mult Re(A B*) on inner<|K|<=outer."""
    Kmag = g.Kmag()
    sel = (Kmag > inner) & (Kmag <= outer)
    return float(np.sum(2 * g.multiplicity()[sel] * (A[sel] * np.conj(B[sel])).real))


def flux_per_sphere(g: Grid, U: np.ndarray, radii, dealias_mode: int) -> np.ndarray:
    """EnergyTr::Compute_flux (compute_flux.cc:51-65): one giver nonlinear term per sphere.

    Giver = U inside |K| <= R (Fill_in_sphere fill_space.cc:56-64); U and the giver
    are dealiased; nlin_i = F[d_j(u_j giver_i)]; Pi(R) = -sum_{|K|>R} 2 mult Re(nlin.U*).
    """
    Ud = dealias(g, U, dealias_mode) if dealias_mode else U
    Kmag = g.Kmag()
    ur = velocity_real(g, Ud)
    out = []
    for R in radii:
        G = np.where(Kmag <= R, Ud, 0)
        G = dealias(g, G, dealias_mode) if dealias_mode else G
        wr = velocity_real(g, G)
        Nl = nlin_conservative_from_real(g, ur, wr)
        out.append(-sum(shell_mult_single(g, Nl[i], Ud[i], R, np.inf) for i in range(3)))
    return np.array(out)


def flux_one_pass(g: Grid, U: np.ndarray, radii, dealias_mode: int) -> np.ndarray:
    """Pi(R) = sum_{|K|<=R} 2 mult Re(N.U*), N = F[(u.grad)u] of the dealiased U.

    Equal to the per-sphere form for solenoidal, alias-free (TWO_THIRDS) fields:
    <u_<, (u.grad)u> = -<u_>, (u.grad)u_<>.
    """
    Ud = dealias(g, U, dealias_mode) if dealias_mode else U
    N = nlin_conservative(g, Ud)
    Kmag = g.Kmag()
    mult = g.multiplicity()
    d = 2 * mult * sum((N[i] * np.conj(Ud[i])).real for i in range(3))
    return np.array([float(d[Kmag <= R].sum()) for R in radii])


# ----------------------------------------------------------------------------
# initial condition
# ----------------------------------------------------------------------------
def _polar_angle(kperp, kpll):
    """Get_polar_angle basicfn_inline.h:357-377."""
    with np.errstate(divide="ignore", invalid="ignore"):
        t = np.where(np.abs(kperp) > MYEPS,
                     np.where(np.abs(kpll) > MYEPS, np.arctan(kperp / np.where(kpll == 0, 1, kpll)), np.pi / 2),
                     np.where(kpll >= 0, 0.0, np.pi))
    return np.where(t >= 0, t, t + np.pi)


def _azimuthal_angle(kh1, kh2):
    """Get_azimuthal_angle basicfn_inline.h:389-405."""
    kperp = np.sqrt(kh1 ** 2 + kh2 ** 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        ang = np.arccos(np.clip(kh1 / np.where(kperp == 0, 1, kperp), -1, 1))
    ang = np.where(kh2 >= 0, ang, 2 * np.pi - ang)
    return np.where(np.abs(kperp) > MYEPS, ang, 0.0)


def spectrum_k4_gauss(nsh: int, k0: float) -> np.ndarray:
    """E_IC(s) = s^4 exp(-2 (s/k0)^2) for shell s>=1 (E_IC(0) = 0)."""
    s = np.arange(nsh, dtype=np.float64)
    E = s ** 4 * np.exp(-2.0 * (s / k0) ** 2)
    E[0] = 0
    return E


def init_energy_spectrum(g: Grid, E_ic: np.ndarray, seed: int, target_energy: float | None = None,
                         H_ic: np.ndarray | None = None) -> np.ndarray:
    """Random-phase solenoidal field with per-shell energy E_ic (FFF).

    Construction of Init_cond_energy_helicity_spectrum_k_ne0 (init_cond_energy.cc:67-120):
    e_k = E_ic(ceil|K|)/modes_in_shell, a_+- = sqrt((e_k +- h_k/|K|)/2), random phases,
    helical -> Craya (FFF_pencil_inline.h:232-236) -> Cartesian (:238-247) with the
    anisotropy axis z (anisotropy_dirn 3: V = (vh1, vh2, vpll), Cvf.cc:416-424).
    The phases come from this project's generator: counter 2m (plus) and 2m+1 (minus)
    for linear mode index m = (lx*Ny + ly)*(Nz/2+1) + lz.  The mean mode is 0; the
    strong reality condition is applied, then the field is rescaled to
    ``target_energy`` (Tarang energy) when given.
    """
    if g.basis != "FFF":
        raise ValueError("FFF only")
    mis = g.modes_in_shell()
    Kx, Ky, Kz = [np.broadcast_to(a, g.shape) for a in g.K()]
    Kmag = g.Kmag()
    idx = np.ceil(Kmag).astype(np.int64)
    Eic = np.zeros(max(len(E_ic), idx.max() + 1))
    Eic[:len(E_ic)] = E_ic
    Hic = np.zeros_like(Eic)
    if H_ic is not None:
        Hic[:len(H_ic)] = H_ic
    with np.errstate(divide="ignore", invalid="ignore"):
        ek = np.where(mis[np.minimum(idx, len(mis) - 1)] > 0, Eic[idx] / mis[np.minimum(idx, len(mis) - 1)], 0.0)
        hk = np.where(mis[np.minimum(idx, len(mis) - 1)] > 0, Hic[idx] / mis[np.minimum(idx, len(mis) - 1)], 0.0)
    live = (Kmag > MYEPS) & (ek >= MYEPS)
    with np.errstate(divide="ignore", invalid="ignore"):
        ap = np.sqrt(np.maximum((ek + hk / np.where(Kmag > 0, Kmag, 1)) / 2, 0))
        am = np.sqrt(np.maximum((ek - hk / np.where(Kmag > 0, Kmag, 1)) / 2, 0))
    m = np.arange(int(np.prod(g.shape)), dtype=np.uint64).reshape(g.shape)
    php = 2 * np.pi * uniform01(seed, 2 * m)
    phm = 2 * np.pi * uniform01(seed, 2 * m + 1)
    up = ap * np.exp(1j * php)
    um = am * np.exp(1j * phm)
    U1 = 1j * (um - up)
    U2 = um + up
    theta = _polar_angle(np.sqrt(Kx ** 2 + Ky ** 2), Kz)
    phi = _azimuthal_angle(Kx, Ky)
    vpll = -U2 * np.sin(theta)
    vh1 = U1 * np.sin(phi) + U2 * np.cos(theta) * np.cos(phi)
    vh2 = -U1 * np.cos(phi) + U2 * np.sin(phi) * np.cos(theta)
    V = np.stack([vh1, vh2, vpll])
    V = np.where(live[None], V, 0)
    V = reality_fix_vec(g, V)
    if target_energy is not None:
        e = total_energy(g, V)
        V = V * math.sqrt(target_energy / e)
    return V


# ----------------------------------------------------------------------------
# Boussinesq RBC on SFF, SSF and SSS (Pr_option PRLARGE / PRSMALL, Uscaling ULARGE / USMALL)
# ----------------------------------------------------------------------------
def rbc_coefficients(pr_option: str, uscaling: str, Ra: float, Pr: float) -> dict:
    """The scaling-dependent coefficients of an RBC run (non-Chebyshev bases):

    * nu, kappa: diss_coefficients (src/solvers/iscalar/Iscalar_main.cc:52-92);
    * cu, cT: U.Force1 += cu T and T.Force += cT U.V1 (compute_force_RBC.cc:104-150);
    * nu0, nuc: Nu = nu0 + nuc <U.V1, T> (Correlation::Get_Nusselt_no, Correlation.cc:144-176);
    * vs: PRINFTY only, the factor of the slaved velocity (FluidVF.cc:259-271).

    PRZERO (T slaved to U: only U is advanced, kappa = 0, no T force) and PRINFTY (U slaved
    to T: only T is advanced, no U force) step through rbc_rk4_step_slaved."""
    if pr_option == "PRZERO":
        # PRZERO shares the PRSMALL branch of the buoyancy; Nu reports 2 <U.V1, T> (no 1 +)
        return dict(nu=1.0, kappa=0.0, cu=Ra if uscaling == "USMALL" else Pr, cT=0.0, nu0=0.0, nuc=2.0)
    if pr_option == "PRINFTY":
        if uscaling == "USMALL":
            return dict(nu=Pr, kappa=1.0, cu=0.0, cT=1.0, nu0=1.0, nuc=2.0, vs=Ra)
        return dict(nu=1.0 / math.sqrt(Ra), kappa=1.0 / math.sqrt(Ra), cu=0.0, cT=1.0, nu0=1.0,
                    nuc=2.0 * math.sqrt(Ra), vs=math.sqrt(Ra))
    if pr_option == "PRLARGE":
        if uscaling == "USMALL":
            return dict(nu=Pr, kappa=1.0, cu=Ra * Pr, cT=1.0, nu0=1.0, nuc=2.0)
        return dict(nu=math.sqrt(Pr / Ra), kappa=1.0 / math.sqrt(Pr * Ra), cu=1.0, cT=1.0, nu0=1.0,
                    nuc=2.0 * math.sqrt(Ra * Pr))
    if pr_option == "PRSMALL":
        if uscaling == "USMALL":
            return dict(nu=1.0, kappa=1.0 / Pr, cu=Ra, cT=1.0 / Pr, nu0=1.0, nuc=2.0 * Pr ** 2)
        return dict(nu=math.sqrt(Pr / Ra), kappa=1.0 / math.sqrt(Pr * Ra), cu=Pr, cT=1.0 / Pr, nu0=1.0,
                    nuc=2.0 * Pr * math.sqrt(Ra * Pr))
    raise ValueError(f"Pr_option {pr_option}")


def divide_ksqr(g: Grid, A: np.ndarray) -> np.ndarray:
    """Array_divide_ksqr (universal_basic.cc:202-225): A / K^2 with A(0,0,0) = 0."""
    K2 = g.Ksqr()
    with np.errstate(divide="ignore", invalid="ignore"):
        B = A / K2
    B[0, 0, 0] = 0.0
    return B


def rbc_slave_temperature(g: Grid, U: np.ndarray) -> np.ndarray:
    """Zero_Prandtl_number_compute_temperature (FluidVF.cc:228-232): T = U.V1 / K^2."""
    return divide_ksqr(g, U[0])


def rbc_slave_velocity(g: Grid, T: np.ndarray, vs: float) -> np.ndarray:
    """Infinite_Prandtl_number_compute_velocity (FluidVF.cc:235-272): X = Dx(T) / K^2 (T with
    the Vx parity), V2 = Dy(X) / K^2, V3 = Dz(X) / K^2, V1 = (Dx(X) + T) / K^2 (X with the
    divergence parity), all times vs (sqrt(Ra) for ULARGE, Ra for USMALL)."""
    p = lambda k: _par(g, k)
    X = divide_ksqr(g, xderiv(g, T, p("Vx")))
    V2 = divide_ksqr(g, yderiv(g, X, p("div")))
    V3 = divide_ksqr(g, zderiv(g, X, p("div")))
    V1 = divide_ksqr(g, xderiv(g, X, p("div")) + T)
    return vs * np.stack([V1, V2, V3])


@dataclass
class RBCConfig:
    grid: Grid
    Ra: float
    Pr: float
    dt: float
    dealias_mode: int = DEALIAS_REFERENCE_CORNER
    reality_fix: bool = True
    pr_option: str = "PRLARGE"
    uscaling: str = "ULARGE"

    @property
    def coeffs(self):
        return rbc_coefficients(self.pr_option, self.uscaling, self.Ra, self.Pr)

    @property
    def nu(self):
        return self.coeffs["nu"]

    @property
    def kappa(self):
        return self.coeffs["kappa"]


@dataclass
class ScalarConfig:
    """Incompressible flow with a passive scalar (program.kind SCALAR_INCOMPRESS), no force."""
    grid: Grid
    nu: float
    kappa: float
    dt: float
    dealias_mode: int = DEALIAS_REFERENCE_CORNER
    reality_fix: bool = True
    buoyancy = False


def rbc_rhs(cfg, U: np.ndarray, T: np.ndarray) -> tuple:
    """Compute_force_TO_rhs_RBC (Tadvance_functions.cc:477-489), PRLARGE / ULARGE, or
    Compute_force_TO_rhs_scalar (Tadvance_functions.cc:464-474) for a ScalarConfig.

    Force (compute_force_RBC.cc:104-150): U.F1 = T, T.F = U.V1 (both from the
    un-dealiased stage input); none for the passive scalar.  Nonlinear
    (compute_nlin_SF.cc:75-112): dealias U, T; T.nlin = sum_j D_j F[u_j T]
    (compute_diag_offdiag.cc:116-136 with FVx/FVy/FVz parities) and the velocity
    nlin; nlin -= F; pressure; rhs = -(nlin + grad p), T.rhs = -T.nlin.
    """
    g = cfg.grid
    buoyancy = getattr(cfg, "buoyancy", True)
    co = cfg.coeffs if buoyancy else None
    FU1 = co["cu"] * T if buoyancy else np.zeros_like(T)
    FT = co["cT"] * U[0] if buoyancy else np.zeros_like(T)
    Ud = dealias(g, U, cfg.dealias_mode)
    Td = dealias(g, T, cfg.dealias_mode)
    ur = velocity_real(g, Ud)
    Tr = inverse(g, Td, _par(g, "F"))
    p = lambda k: _par(g, k)
    Tn = xderiv(g, forward(g, ur[0] * Tr, p("FVx")), p("FVx"))
    Tn = Tn + yderiv(g, forward(g, ur[1] * Tr, p("FVy")), p("FVy"))
    Tn = Tn + zderiv(g, forward(g, ur[2] * Tr, p("FVz")), p("FVz"))
    N = nlin_conservative_from_real(g, ur)
    N[0] = N[0] - FU1
    Tn = Tn - FT
    return project_rhs(g, N), -Tn, Ud, Td


def rbc_rk4_step(cfg, U0: np.ndarray, T0: np.ndarray) -> tuple:
    """RK4(U,T,P,F) RK_SF.cc:97-221 with Single_time_step_scalar (U with nu, T with kappa);
    an RBCConfig (SFF, SSF or SSS, buoyancy) or a ScalarConfig (passive scalar)."""
    if getattr(cfg, "pr_option", "") in ("PRZERO", "PRINFTY"):
        return rbc_rk4_step_slaved(cfg, U0, T0)
    g = cfg.grid
    dt = cfg.dt
    EU = lambda A, a: exp_ksqr(g, A, -cfg.nu * a * dt)
    ET = lambda A, a: exp_ksqr(g, A, -cfg.kappa * a * dt)
    R, S, Ud, Td = rbc_rhs(cfg, U0, T0)
    U = EU(Ud + 0.5 * dt * R, 0.5)
    T = ET(Td + 0.5 * dt * S, 0.5)
    totU = (dt / 6) * EU(R, 1.0)
    totT = (dt / 6) * ET(S, 1.0)
    R, S, _, _ = rbc_rhs(cfg, U, T)
    U = EU(U0, 0.5) + 0.5 * dt * R
    T = ET(T0, 0.5) + 0.5 * dt * S
    totU = totU + (dt / 3) * EU(R, 0.5)
    totT = totT + (dt / 3) * ET(S, 0.5)
    R, S, _, _ = rbc_rhs(cfg, U, T)
    U = EU(EU(U0, 0.5) + dt * R, 0.5)
    T = ET(ET(T0, 0.5) + dt * S, 0.5)
    totU = totU + (dt / 3) * EU(R, 0.5)
    totT = totT + (dt / 3) * ET(S, 0.5)
    R, S, _, _ = rbc_rhs(cfg, U, T)
    totU = totU + (dt / 6) * R
    totT = totT + (dt / 6) * S
    U = EU(U0, 1.0) + totU
    T = ET(T0, 1.0) + totT
    if cfg.reality_fix:
        U = reality_fix_vec(g, U)
        T = reality_fix(g, T)
    return U, T


def rbc_rk4_step_slaved(cfg: RBCConfig, U0: np.ndarray, T0: np.ndarray) -> tuple:
    """RK4(U,T,P,F) (RK_SF.cc:97-221) under PRZERO or PRINFTY, where one field is slaved to
    the other (Single_time_step_RBC / Compute_RK4_parts_RBC, Tadvance_functions.cc:380-395,
    :598-609; final assembly RK_SF.cc:196-213).

    PRZERO: force U.F1 = cu T of the stage input, no T force (compute_force_RBC.cc:117-153);
    nlin of U only (compute_nlin_SF.cc:266-268); pressure and rhs of U; U advanced with nu
    and T = U.V1 / K^2 after every stage and after the final assembly.
    PRINFTY: force T.F = cT U.V1 of the stage input (before the nonlinear term); nlin:
    dealias T, U = slave(T) (so the products use the dealiased T and the velocity slaved to
    it), T.nlin = sum_j D_j F[u_j T] (compute_nlin_SF.cc:271-299); no pressure; T advanced
    with kappa and U = slave(T) after every stage and after the final assembly."""
    g = cfg.grid
    dt = cfg.dt
    co = cfg.coeffs
    p = lambda k: _par(g, k)
    if cfg.pr_option == "PRZERO":
        EU = lambda A, a: exp_ksqr(g, A, -co["nu"] * a * dt)

        def rhs(U, T):
            FU1 = co["cu"] * T
            Ud = dealias(g, U, cfg.dealias_mode)
            N = nlin_conservative_from_real(g, velocity_real(g, Ud))
            N[0] = N[0] - FU1
            return project_rhs(g, N), Ud

        R, Ud = rhs(U0, T0)
        U = EU(Ud + 0.5 * dt * R, 0.5)
        tot = (dt / 6) * EU(R, 1.0)
        R, _ = rhs(U, rbc_slave_temperature(g, U))
        U = EU(U0, 0.5) + 0.5 * dt * R
        tot = tot + (dt / 3) * EU(R, 0.5)
        R, _ = rhs(U, rbc_slave_temperature(g, U))
        U = EU(EU(U0, 0.5) + dt * R, 0.5)
        tot = tot + (dt / 3) * EU(R, 0.5)
        R, _ = rhs(U, rbc_slave_temperature(g, U))
        U = EU(U0, 1.0) + (tot + (dt / 6) * R)
        T = rbc_slave_temperature(g, U)
    elif cfg.pr_option == "PRINFTY":
        ET = lambda A, a: exp_ksqr(g, A, -co["kappa"] * a * dt)

        def rhs(U, T):
            FT = co["cT"] * U[0]
            Td = dealias(g, T, cfg.dealias_mode)
            ur = velocity_real(g, rbc_slave_velocity(g, Td, co["vs"]))
            Tr = inverse(g, Td, p("F"))
            Tn = xderiv(g, forward(g, ur[0] * Tr, p("FVx")), p("FVx"))
            Tn = Tn + yderiv(g, forward(g, ur[1] * Tr, p("FVy")), p("FVy"))
            Tn = Tn + zderiv(g, forward(g, ur[2] * Tr, p("FVz")), p("FVz"))
            return -(Tn - FT), Td

        S, Td = rhs(U0, T0)
        T = ET(Td + 0.5 * dt * S, 0.5)
        tot = (dt / 6) * ET(S, 1.0)
        S, _ = rhs(rbc_slave_velocity(g, T, co["vs"]), T)
        T = ET(T0, 0.5) + 0.5 * dt * S
        tot = tot + (dt / 3) * ET(S, 0.5)
        S, _ = rhs(rbc_slave_velocity(g, T, co["vs"]), T)
        T = ET(ET(T0, 0.5) + dt * S, 0.5)
        tot = tot + (dt / 3) * ET(S, 0.5)
        S, _ = rhs(rbc_slave_velocity(g, T, co["vs"]), T)
        T = ET(T0, 1.0) + (tot + (dt / 6) * S)
        U = rbc_slave_velocity(g, T, co["vs"])
    else:
        raise ValueError(cfg.pr_option)
    if cfg.reality_fix:
        U = reality_fix_vec(g, U)
        T = reality_fix(g, T)
    return U, T


# ----------------------------------------------------------------------------
# incompressible MHD (FFF): RK4(U, W, P, F) with W = B, no force
# ----------------------------------------------------------------------------
@dataclass
class MHDConfig:
    grid: Grid
    nu: float
    eta: float
    dt: float
    dealias_mode: int = DEALIAS_REFERENCE_CORNER
    reality_fix: bool = True


def mhd_nlin(g: Grid, U: np.ndarray, B: np.ndarray) -> tuple:
    """Nlin_incompress::Compute_nlin(U, W) (compute_nlin_VF_MHD.cc:40-95) on dealiased
    fields: Elsasser real fields Zp = u + b, Zm = u - b (MHD.cc:75-84); diagonal terms
    Zp.nlin_i = Zm.nlin_i = D_i F[Zp_i Zm_i] (compute_diag_offdiag.cc:139-164), then
    the six off-diagonal products in the reference's order (:202-258), so that
    Zp.nlin_i = sum_j D_j F[Zp_i Zm_j] and Zm.nlin_i = sum_j D_j F[Zp_j Zm_i];
    U.nlin = (Zp.nlin + Zm.nlin)/2, B.nlin = (Zp.nlin - Zm.nlin)/2 (MHD.cc:150-161)."""
    u = [inverse(g, U[i]) for i in range(3)]
    b = [inverse(g, B[i]) for i in range(3)]
    zp = [u[i] + b[i] for i in range(3)]
    zm = [u[i] - b[i] for i in range(3)]
    D = [lambda A: xderiv(g, A), lambda A: yderiv(g, A), lambda A: zderiv(g, A)]
    P = lambda i, j: forward(g, zp[i] * zm[j])
    npl = [D[i](P(i, i)) for i in range(3)]
    nmi = [a.copy() for a in npl]
    X = P(0, 1); npl[0] = npl[0] + D[1](X); nmi[1] = nmi[1] + D[0](X)
    X = P(1, 0); nmi[0] = nmi[0] + D[1](X); npl[1] = npl[1] + D[0](X)
    X = P(1, 2); npl[1] = npl[1] + D[2](X); nmi[2] = nmi[2] + D[1](X)
    X = P(2, 1); nmi[1] = nmi[1] + D[2](X); npl[2] = npl[2] + D[1](X)
    X = P(2, 0); nmi[0] = nmi[0] + D[2](X); npl[2] = npl[2] + D[0](X)
    X = P(0, 2); npl[0] = npl[0] + D[2](X); nmi[2] = nmi[2] + D[0](X)
    NU = np.stack([0.5 * (npl[i] + nmi[i]) for i in range(3)])
    NB = np.stack([0.5 * (npl[i] - nmi[i]) for i in range(3)])
    return NU, NB


def mhd_rhs(cfg: MHDConfig, U: np.ndarray, B: np.ndarray) -> tuple:
    """Compute_force_TO_rhs(U, W, P, F) (Tadvance_functions.cc:506-517) with no force:
    dealias U, B in place, nlin, pressure from U.nlin, U.rhs = -(U.nlin + D p),
    W.rhs = -W.nlin (Compute_rhs(U, W, P), :259-267)."""
    g = cfg.grid
    Ud = dealias(g, U, cfg.dealias_mode) if cfg.dealias_mode else U.copy()
    Bd = dealias(g, B, cfg.dealias_mode) if cfg.dealias_mode else B.copy()
    NU, NB = mhd_nlin(g, Ud, Bd)
    return project_rhs(g, NU), -NB, Ud, Bd


def mhd_rk4_step(cfg: MHDConfig, U0: np.ndarray, B0: np.ndarray) -> tuple:
    """RK4(U, W, P, F) (RK_VF_MHD.cc:126-186): the fluid RK4 stages for U (nu) and
    W = B (eta), then the strong reality condition on both (Time_advance.cc:126-129)."""
    g = cfg.grid
    dt = cfg.dt
    EU = lambda A, a: exp_ksqr(g, A, -cfg.nu * a * dt)
    EB = lambda A, a: exp_ksqr(g, A, -cfg.eta * a * dt)
    R, S, Ud, Bd = mhd_rhs(cfg, U0, B0)
    U = EU(Ud + 0.5 * dt * R, 0.5)
    B = EB(Bd + 0.5 * dt * S, 0.5)
    totU = (dt / 6) * EU(R, 1.0)
    totB = (dt / 6) * EB(S, 1.0)
    R, S, _, _ = mhd_rhs(cfg, U, B)
    U = EU(U0, 0.5) + 0.5 * dt * R
    B = EB(B0, 0.5) + 0.5 * dt * S
    totU = totU + (dt / 3) * EU(R, 0.5)
    totB = totB + (dt / 3) * EB(S, 0.5)
    R, S, _, _ = mhd_rhs(cfg, U, B)
    U = EU(EU(U0, 0.5) + dt * R, 0.5)
    B = EB(EB(B0, 0.5) + dt * S, 0.5)
    totU = totU + (dt / 3) * EU(R, 0.5)
    totB = totB + (dt / 3) * EB(S, 0.5)
    R, S, _, _ = mhd_rhs(cfg, U, B)
    totU = totU + (dt / 6) * R
    totB = totB + (dt / 6) * S
    U = EU(U0, 1.0) + totU
    B = EB(B0, 1.0) + totB
    if cfg.reality_fix:
        U = reality_fix_vec(g, U)
        B = reality_fix_vec(g, B)
    return U, B


def nusselt(cfg: RBCConfig, U: np.ndarray, T: np.ndarray) -> float:
    """Get_Nusselt_no (Correlation.cc:144-176): nu0 + nuc <U1, T> with the scaling's factors
    (PRLARGE / ULARGE: 1 + 2 sqrt(Ra Pr) <U1, T>)."""
    co = cfg.coeffs
    return co["nu0"] + co["nuc"] * cross_energy(cfg.grid, U[0], T)


def rbc_temperature_ic(g: Grid, amp: float, kmax_grid: float, seed: int) -> np.ndarray:
    """T perturbation: amplitude ``amp`` with uniform random phases on the modes whose grid
    wavenumber |(m, ky, kz)| <= kmax_grid, m >= 1 (sine parity), kz < Nz/2; then the
    strong reality condition.  Counter = linear mode index m."""
    mm = g.kx[:, None, None]
    ky = g.ky[None, :, None]
    kz = g.kz[None, None, :]
    r = np.sqrt(mm ** 2 + ky ** 2 + kz ** 2)
    sel = np.broadcast_to((r <= kmax_grid) & (mm >= 1), g.shape)
    cnt = np.arange(int(np.prod(g.shape)), dtype=np.uint64).reshape(g.shape)
    ph = 2 * np.pi * uniform01(seed, cnt)
    T = np.where(sel, amp * np.exp(1j * ph), 0)
    return reality_fix(g, T)


# ----------------------------------------------------------------------------
# discrete adjoint of the FFF IF-RK4 step (rotational form, unforced)
#
# The reference has no adjoint; this is the exact transpose of rk4_step above
# (the forward it differentiates follows RK.cc:91-170), derived here:
#
#   rhs(U) = g(D U),  g(V) = P F[u x w],  u = I V,  w = I (iK x V)
#
# in the real inner product <A, B> = Re sum A conj(B) over the stored
# half-spectrum arrays (which is also torch's convention for the gradient of a
# real loss with respect to a complex tensor).  With c = 1 on the kz = 0 and
# kz = Nz/2 planes and 2 elsewhere (the C2R weights), F^T = N^-3 I c^-1 and
# I^T = N^3 c F, so
#
#   g'(V)^T lam = c [ F(w x mu) + iK x F(mu x u) ],   mu = I(c^-1 P lam),
#
# and the IF-RK4 stage recurrences are transposed stage by stage
# (rk4_step_adjoint).  The strong reality condition is real-linear; its
# transpose folds the Hermitian-copied half of the kz = 0 plane back onto its
# source entries (reality_fix_adjoint).
# ----------------------------------------------------------------------------
def c2r_weights(g: Grid) -> np.ndarray:
    """c(kz): 1 on the kz = 0 and kz = Nz/2 planes, 2 on the planes in between."""
    Nz = g.N[2]
    c = np.full(g.shape, 2.0)
    c[:, :, 0] = 1.0
    c[:, :, Nz // 2] = 1.0
    return c


def leray(g: Grid, N: np.ndarray) -> np.ndarray:
    """P N = N - K (K.N)/K^2 (identity at K = 0); project_rhs(N) = -P N."""
    Kx, Ky, Kz = g.K()
    K2 = g.Ksqr()
    d = Kx * N[0] + Ky * N[1] + Kz * N[2]
    with np.errstate(divide="ignore", invalid="ignore"):
        q = np.where(K2 > 0, d / np.where(K2 > 0, K2, 1.0), 0.0)
    return np.stack([N[0] - Kx * q, N[1] - Ky * q, N[2] - Kz * q])


def _cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def rhs_rotational_adjoint(g: Grid, V: np.ndarray, lam: np.ndarray) -> np.ndarray:
    """g'(V)^T lam for g(V) = P F[u x w] (the rotational right-hand side of a dealiased V)."""
    c = c2r_weights(g)
    u = [inverse(g, V[i]) for i in range(3)]
    W = vorticity(g, V)
    w = [inverse(g, W[i]) for i in range(3)]
    Pl = leray(g, lam) / c
    mu = [inverse(g, Pl[i]) for i in range(3)]
    A = np.stack([forward(g, x) for x in _cross(w, mu)])
    B = np.stack([forward(g, x) for x in _cross(mu, u)])
    return c * (A + vorticity(g, B))


def reality_fix_adjoint(g: Grid, A: np.ndarray) -> np.ndarray:
    """Transpose of reality_fix (FFF): each kz = 0 entry that reality_fix overwrites with
    conj(source) adds its conjugate to the source and becomes 0; the kz = Nz/2 plane is 0."""
    if g.basis != "FFF":
        raise ValueError("FFF only")
    Nx, Ny, Nz = g.N
    B = A.copy()
    plane = A[:, :, 0].copy()
    iy_minus = (-g.ky) % Ny
    for lx in range(Nx // 2 + 1, Nx):
        src = -g.kx[lx]
        sel = g.ky != Ny // 2
        B[src, iy_minus[sel], 0] += np.conj(plane[lx, sel])
        B[lx, sel, 0] = 0
    sel = g.ky < 0
    B[0, iy_minus[sel], 0] += np.conj(plane[0, sel])
    B[0, sel, 0] = 0
    B[:, :, Nz // 2] = 0
    return B


def reality_fix_vec_adjoint(g: Grid, V: np.ndarray) -> np.ndarray:
    return np.stack([reality_fix_adjoint(g, V[i]) for i in range(V.shape[0])])


def rk4_stages(cfg: FluidConfig, U0: np.ndarray) -> list:
    """The stage inputs [U0, U1, U2, U3] of one rk4_step (each enters rhs dealiased)."""
    g = cfg.grid
    if cfg.nlin_form != "rotational" or cfg.forcing is not None or g.basis != "FFF":
        raise ValueError("adjoint: FFF, rotational form, unforced")
    mis = g.modes_in_shell()
    nu, dt = cfg.nu, cfg.dt
    E = lambda A, a: exp_ksqr(g, A, -nu * a * dt)
    R, Ud = fluid_rhs(cfg, U0, mis)
    U1 = E(Ud + (0.5 * dt) * R, 0.5)
    R, _ = fluid_rhs(cfg, U1, mis)
    U2 = E(U0, 0.5) + (0.5 * dt) * R
    R, _ = fluid_rhs(cfg, U2, mis)
    U3 = E(E(U0, 0.5) + dt * R, 0.5)
    return [U0, U1, U2, U3]


def rk4_step_adjoint(cfg: FluidConfig, U0: np.ndarray, Lam: np.ndarray) -> np.ndarray:
    """(d rk4_step / d U0)^T Lam: the stage recurrences of rk4_step transposed, last stage first.

    With W_s = D g'(D U_{s-1})^T lam_s (the cotangent of stage input U_{s-1}):
      L = RF^T Lam;  lam_4 = dt/6 L
      A  = E1 L + E1 W_4,  lam_3 = dt/3 Eh L + dt Eh W_4
      A += Eh W_3,         lam_2 = dt/3 Eh L + dt/2 W_3
      A += Eh W_2,         lam_1 = dt/6 E1 L + dt/2 Eh W_2
      result = A + W_1
    """
    g = cfg.grid
    dt = cfg.dt
    stages = rk4_stages(cfg, U0)
    D = lambda A: dealias(g, A, cfg.dealias_mode) if cfg.dealias_mode else A
    Eh = np.exp(-cfg.nu * 0.5 * dt * g.Ksqr())
    E1 = Eh * Eh
    gT = lambda s, lam: D(rhs_rotational_adjoint(g, D(stages[s]), lam))
    L = reality_fix_vec_adjoint(g, Lam) if cfg.reality_fix else Lam.copy()
    W = gT(3, (dt / 6) * L)
    A = E1 * L + E1 * W
    lam = (dt / 3) * Eh * L + dt * Eh * W
    W = gT(2, lam)
    A = A + Eh * W
    lam = (dt / 3) * Eh * L + (0.5 * dt) * W
    W = gT(1, lam)
    A = A + Eh * W
    lam = (dt / 6) * E1 * L + (0.5 * dt) * Eh * W
    W = gT(0, lam)
    return A + W


def energy_weights(g: Grid) -> np.ndarray:
    """Tarang FFF energy weights per stored mode: 1, and 1/2 on the kz = 0 plane."""
    w = np.ones(g.shape)
    w[:, :, 0] = 0.5
    return w


def adjoint_loss(g: Grid, U: np.ndarray, Ut: np.ndarray) -> tuple:
    """J = 1/2 ||U - Ut||^2 in the energy norm (total_energy of the difference) and dJ/dU."""
    w = energy_weights(g)
    d = U - Ut
    return float(np.sum(w * np.abs(d) ** 2)), 2.0 * w * d
