"""Seeded synthetic workloads for the RT step.

The reference's production inputs (density cubes, source catalogues) are not shipped, so every
workload here is generated from a seed with the shapes and value distributions of the named
configurations:

* gas: Gaussian random field g on N^3 with P(k) ~ k^-2 (periodic FFT), unit variance;
  1 + delta = exp(sigma_ln * g - sigma_ln^2 / 2) (mean 1), T = 1e4 K;
* sources at uniform-random cell centres with log-uniform or dN/dL ~ L^-2 luminosities
  (inverse CDF L = 1 / (1/Lmin - u (1/Lmin - 1/Lmax)));
* 5 frequency bins 14.48/16.7/20.03/25.78/39.23 eV with an alpha = 1.5 power-law spectrum;
* dt is imposed through cl_factor with tstep_factor = 1, as dt = tstep_factor dx / (cl_factor c)
  (rt_funcs.cc:9-12).

The same arrays feed the CUDA path and the CPU oracles (written in the reference's own input
formats: density as float32 N^3 in (i, j, k) order with k fastest, io_funcs.cc:33-62; the
catalogue as 5 doubles per source x, y, z [h^-1 cMpc], mass, Ndot, io_funcs.cc:190-206; the halo
count as one int64, io_funcs.cc:164-166).
"""
from __future__ import annotations

import dataclasses
import os
from typing import List, Optional

import numpy as np

# physical constants as the reference defines them (global_constants.h)
HH = 0.68
KPC_TO_CM = 3.086e21
MPC_TO_CM = 3.086e24
YR_TO_S = 3.154e7
CL = 2.998e10
H_EV = 4.135667e-15
NU_EV_5BIN = (14.48, 16.7, 20.03, 25.78, 39.23)


@dataclasses.dataclass
class BoxSpec:
    """One periodic box: grid, gas recipe, sources and time stepping."""

    name: str
    n: int
    box_hmpc: float          # comoving side in h^-1 cMpc
    z: float
    sigma_ln: float
    n_src: int
    lum_law: str             # "loguniform" or "powerlaw2"
    lum_min: float
    lum_max: float
    dt_myr: float
    steps: int
    clump_model: str = "const"   # "const" (C = 1) or "sqrt" (C = 1 + 3 (1+delta)^0.5)
    seed: int = 1234
    ray_per_cell_max: int = 22   # global_variables.cc:40; lowered in merge tests
    rkill_cmpc: float = 50.0     # remove rays beyond this comoving radius (0 = never)
    src_region: int = 0          # 0: sources anywhere; m > 0: sources in the centred m^3 cells

    # ---- derived quantities, computed with the reference's float arithmetic -------------
    def a_snap(self) -> np.float32:
        return np.float32(1.0 / (1.0 + self.z))

    def lx0_kpc(self) -> np.float32:
        # float const Lx0 = box*1e3/hh (user_inputs.h:92)
        return np.float32(self.box_hmpc * 1e3 / HH)

    def dx0(self) -> np.float32:
        # float dx0 = Lx0/Nx*kpc_to_cm (global_variables.cc:69)
        return np.float32(float(self.lx0_kpc() / np.float32(self.n)) * KPC_TO_CM)

    def dx(self) -> np.float32:
        # Lx = Lx0*a (gas_funcs.cc:595); dx[i] = Lx/Nx*kpc_to_cm (init_funcs.cc:23)
        lx = np.float32(self.lx0_kpc() * self.a_snap())
        return np.float32(float(lx / np.float32(self.n)) * KPC_TO_CM)

    def cl_factor(self) -> float:
        """cl_factor giving dt = dt_myr with tstep_factor = 1 (rt_funcs.cc:11)."""
        return float(np.float32(float(self.dx()) / (self.dt_myr * 1e6 * YR_TO_S * CL)))

    def rkill_cm(self) -> float:
        return self.rkill_cmpc * MPC_TO_CM if self.rkill_cmpc > 0 else 0.0


def _gaussian_field(n: int, rng: np.random.Generator) -> np.ndarray:
    white = rng.standard_normal((n, n, n))
    fk = np.fft.rfftn(white)
    kx = np.fft.fftfreq(n)
    kz = np.fft.rfftfreq(n)
    k2 = kx[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2
    k2[0, 0, 0] = 1.0
    fk /= np.sqrt(k2)          # P(k) ~ k^-2  <=>  amplitude ~ k^-1
    fk[0, 0, 0] = 0.0
    g = np.fft.irfftn(fk, s=(n, n, n), axes=(0, 1, 2))
    g /= g.std()
    return g


@dataclasses.dataclass
class BoxInputs:
    spec: BoxSpec
    delta1: np.ndarray        # float32 [N,N,N], 1 + delta (mean 1)
    src_pos: np.ndarray       # float64 [S,3] positions in h^-1 cMpc (cell centres)
    src_lum: np.ndarray       # float64 [S] photons/s
    clump: Optional[np.ndarray]  # float32 [N,N,N] or None for constant C = 1


def make_inputs(spec: BoxSpec) -> BoxInputs:
    rng = np.random.default_rng(spec.seed)
    g = _gaussian_field(spec.n, rng)
    delta1 = np.exp(spec.sigma_ln * g - 0.5 * spec.sigma_ln ** 2).astype(np.float32)
    if spec.src_region > 0:
        cells = rng.integers(0, spec.src_region, size=(spec.n_src, 3)) + (spec.n - spec.src_region) // 2
    else:
        cells = rng.integers(0, spec.n, size=(spec.n_src, 3))
    pos = (cells.astype(np.float64) + 0.5) * (spec.box_hmpc / spec.n)
    u = rng.random(spec.n_src)
    if spec.lum_law == "loguniform":
        lum = 10.0 ** (np.log10(spec.lum_min) + u * (np.log10(spec.lum_max) - np.log10(spec.lum_min)))
    elif spec.lum_law == "powerlaw2":
        lum = 1.0 / (1.0 / spec.lum_min - u * (1.0 / spec.lum_min - 1.0 / spec.lum_max))
    else:
        raise ValueError(spec.lum_law)
    clump = None
    if spec.clump_model == "sqrt":
        clump = (np.float32(1.0) + np.float32(3.0) * np.sqrt(delta1)).astype(np.float32)
    elif spec.clump_model != "const":
        raise ValueError(spec.clump_model)
    return BoxInputs(spec, delta1, pos, lum, clump)


def grid_sources(inp: BoxInputs):
    """Sources gridded per cell the way read_source_catalog does (io_funcs.cc:184-229): the
    luminosities of sources sharing a cell add up, and the list is in (i, j, k) order."""
    s = inp.spec
    lx0 = float(s.lx0_kpc())
    idx = np.floor(inp.src_pos / HH / lx0 * 1e3 * s.n).astype(np.int64) % s.n
    flat = (idx[:, 0] * s.n + idx[:, 1]) * s.n + idx[:, 2]
    grid = {}
    for c, l in zip(flat.tolist(), inp.src_lum.tolist()):
        grid[c] = grid.get(c, 0.0) + 1.0 * l      # fesc = 1
    cells = np.array(sorted(grid.keys()), dtype=np.int64)
    lums = np.array([grid[c] for c in cells.tolist()], dtype=np.float64)
    ijk = np.stack([cells // (s.n * s.n), (cells // s.n) % s.n, cells % s.n], axis=1).astype(np.int32)
    return ijk, lums


def write_reference_inputs(inp: BoxInputs, directory: str) -> None:
    """Write density / catalogue / halo count in the reference's own binary formats."""
    os.makedirs(directory, exist_ok=True)
    inp.delta1.astype(np.float32).tofile(os.path.join(directory, "density.bin"))
    cat = np.zeros((inp.src_pos.shape[0], 5), dtype=np.float64)
    cat[:, 0:3] = inp.src_pos
    cat[:, 4] = inp.src_lum
    cat.tofile(os.path.join(directory, "catalog.bin"))
    np.array([inp.src_pos.shape[0]], dtype=np.int64).tofile(os.path.join(directory, "numhalos.bin"))
    if inp.clump is not None:
        inp.clump.astype(np.float32).tofile(os.path.join(directory, "clump.bin"))


# ---- the named configurations -------------------------------------------------------------

def config_S(seed: int = 1234) -> BoxSpec:
    """64^3, 25 h^-1 cMpc at z=8, sigma_ln 0.5, 32 log-uniform [1e50,1e53] sources, 10 x 1 Myr."""
    return BoxSpec("S", 64, 25.0, 8.0, 0.5, 32, "loguniform", 1e50, 1e53, 1.0, 10, "const", seed)


def config_M(seed: int = 1234) -> BoxSpec:
    """128^3, 50 h^-1 cMpc at z=7, sigma_ln 0.7, 1024 L^-2 [1e50,1e54] sources, 20 x 0.5 Myr,
    clumping C = 1 + 3 (1+delta)^0.5."""
    return BoxSpec("M", 128, 50.0, 7.0, 0.7, 1024, "powerlaw2", 1e50, 1e54, 0.5, 20, "sqrt", seed)


def config_L(seed: int = 1234) -> BoxSpec:
    """256^3, 100 h^-1 cMpc at z=6.5, sigma_ln 0.8, 16384 L^-2 [1e50,1e54] sources, 50 x 0.25 Myr."""
    return BoxSpec("L", 256, 100.0, 6.5, 0.8, 16384, "powerlaw2", 1e50, 1e54, 0.25, 50, "const", seed)


def config_A(seed: int = 1234) -> BoxSpec:
    """Adjoint box: 128^3, 50 h^-1 cMpc at z=7, 256 log-uniform [1e51,1e53] sources, 1 x 1 Myr.
    Rays travel about one cell in the single step, so the sources are placed in the centred 32^3
    cells: the objective (Gamma_HI summed over the centred 16^3 cells) then sees ~30 sources
    instead of the ~1 a box-wide placement would give."""
    return BoxSpec("A", 128, 50.0, 7.0, 0.7, 256, "loguniform", 1e51, 1e53, 1.0, 1, "const", seed,
                   src_region=32)


def config_E(seed: int = 4321, nbox: int = 96) -> List[BoxSpec]:
    """Uneven ensemble: N in {32,64,96,128} at the shared comoving cell size, sigma_ln ~ U[0.3,0.9],
    source counts log-uniform in [8, 4096], L^-2 [1e50,1e54], 10 x 0.5 Myr at z=7."""
    rng = np.random.default_rng(seed)
    cell_hmpc = 25.0 / 64.0
    out = []
    for b in range(nbox):
        n = int(rng.choice([32, 64, 96, 128]))
        sig = float(rng.uniform(0.3, 0.9))
        nsrc = int(round(10.0 ** rng.uniform(np.log10(8.0), np.log10(4096.0))))
        out.append(BoxSpec(f"E{b:02d}", n, n * cell_hmpc, 7.0, sig, nsrc, "powerlaw2", 1e50, 1e54, 0.5, 10,
                           "const", seed * 1000 + b))
    return out


def config_tiny(n: int = 16, n_src: int = 6, steps: int = 6, seed: int = 7, name: str = "T16",
                clump_model: str = "const", ray_per_cell_max: int = 22, dt_myr: float = 1.0,
                z: float = 8.0, lum_min: float = 1e52, lum_max: float = 1e54, sigma_ln: float = 0.5,
                src_region: int = 0) -> BoxSpec:
    """Small boxes for parity tests (same cell size as S)."""
    return BoxSpec(name, n, 25.0 * n / 64.0, z, sigma_ln, n_src, "loguniform", lum_min, lum_max, dt_myr, steps,
                   clump_model, seed, ray_per_cell_max, src_region=src_region)


CONFIGS = {"S": config_S, "M": config_M, "L": config_L, "A": config_A}


# ---- synthetic sub-grid tables ------------------------------------------------------------
# The reference's sub-grid model reads RadHydro tables (27 runs: 3 photo-ionisation rates x 3
# reionisation redshifts x 3 overdensities, Nt = 5000 rows of time since ionisation, two mean free
# paths, HI fraction, temperature; subgrid.cc:20-47) and a linear -> non-linear overdensity table
# (500 cosmic times x 500 delta/sigma; subgrid.cc:49-95), neither of which is shipped. These are
# smooth closed-form stand-ins with the tables' shapes; the same arrays feed the device, the
# oracle and (written in the reference's file formats) the compiled reference.
SG_NT = 5000
SG_NDLIN = 500


def subgrid_radhydro():
    """Per run (q rate, m reionisation redshift, p density, the reference's loop order) the 4
    table columns after the time: mfp (frequency-averaged, 912 A), HI fraction, temperature."""
    t_yr = np.arange(SG_NT, dtype=np.float64) * 2.0e5           # 0 .. 1 Gyr since ionisation
    cols = np.zeros((3, 3, 3, 4, SG_NT))
    for q in range(3):
        for m in range(3):
            for p in range(3):
                g = 10.0 ** (q - 1)                              # Gamma / 3e-13
                d = 2.0 ** (p - 1)                               # 1 + delta ~ 0.5, 1, 2
                z = 1.0 + 0.1 * m
                relax = 1.0 + 4.0 * np.exp(-t_yr / 3.0e7)
                mfp0 = 8.0 * g ** (2.0 / 3.0) / d / z / relax
                mfp1 = 0.6 * mfp0
                fh1 = 2.0e-4 / g ** 0.7 * d ** 0.8 * z * (1.0 + 3.0 * np.exp(-t_yr / 1.0e7))
                temp = 1.2e4 * d ** 0.3 / z * (1.0 + 1.5 * np.exp(-t_yr / 5.0e7))
                cols[q, m, p] = np.stack([mfp0, mfp1, np.minimum(fh1, 0.9), temp])
    return {"time_yr": t_yr, "cols": cols}


def subgrid_delta_over_sigma(t0: float, t1: float):
    """The linear -> non-linear overdensity table: times from t0 to t1 [s], delta/sigma in
    [-4, 4], and a lognormal-like growth of the non-linear overdensity with time."""
    t = np.linspace(t0, t1, SG_NDLIN)
    ds = np.linspace(-4.0, 4.0, SG_NDLIN)
    grow = 0.2 + 0.5 * (t - t0) / (t1 - t0)
    dnl = np.exp(grow[:, None] * ds[None, :]) - 1.0
    return {"t": t, "ds": ds, "dnl": dnl}


def subgrid_arrays(t0: float, t1: float):
    """The tables as the reference holds them in memory after reading the files (the layout
    frt_set_subgrid takes): time_RH and fh1_RH as flat [Nt][3][3][3] floats written at the gamma
    index q + 1 (subgrid.cc:24-36), with one slot more for the last row's spill; times in s; the
    overdensity table as floats."""
    rh = subgrid_radhydro()
    n = SG_NT * 27 + 1
    time = np.zeros(n, np.float32)
    fh1 = np.zeros(n, np.float32)
    t_s = (rh["time_yr"].astype(np.float32).astype(np.float64) * YR_TO_S).astype(np.float32)
    for q in range(3):
        for m in range(3):
            for p in range(3):
                off = ((np.arange(SG_NT) * 3 + m) * 3 + p) * 3 + (q + 1)
                time[off] = t_s
                fh1[off] = rh["cols"][q, m, p, 2].astype(np.float32)
    ds = subgrid_delta_over_sigma(t0, t1)
    return {"time": time, "fh1": fh1, "t_dnl": ds["t"].astype(np.float32), "ds": ds["ds"].astype(np.float32),
            "dnl": ds["dnl"].astype(np.float32).ravel()}


def cosmic_time_lcdm(a: float, h: float = HH, omega_m: float = 0.305) -> float:
    """Age of a flat LambdaCDM universe at scale factor a [s] (closed form,
    t = 2 / (3 H0 sqrt(OL)) asinh(sqrt(OL / Om) a^1.5)); the cosmic times the sub-grid model
    reads (tinit and the RadHydro reionisation redshifts) for a synthetic run."""
    h0 = 100.0 * h * 1e5 / MPC_TO_CM
    ol = 1.0 - omega_m
    return float(2.0 / (3.0 * h0 * np.sqrt(ol)) * np.arcsinh(np.sqrt(ol / omega_m) * a ** 1.5))


def subgrid_inputs(z: float):
    """Tables and cosmic-time constants for frt_set_subgrid on a box starting at redshift z:
    {tinit, t(z=12), t(z=8), t(z=5.5), tre_dom = t(z=12, 8, 6)}, the overdensity table spanning
    z = 16 to 4.5."""
    ct = lambda zz: cosmic_time_lcdm(1.0 / (1.0 + zz))   # noqa: E731
    consts = [ct(z), ct(12.0), ct(8.0), ct(5.5), ct(12.0), ct(8.0), ct(6.0)]
    return subgrid_arrays(ct(16.0), ct(4.5)), np.asarray(consts, np.float32)
