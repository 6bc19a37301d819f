"""Case set-up for the single-phase RK3 step: grids, initial conditions and the benchmark configurations.

The face arrays follow generateGrid (src/genGridandIC.f90:14-265) operation by operation, so the library derives
the same centres, dx/dz, weights and Poisson operators as the reference's initialize
(src/initialization.f90:243-644).  Initial conditions are produced the way the reference receives them on a
restart (src/input_output.f90:1225-1341): every velocity array in its ghosted one-rank shape, with the ghosts
already filled by the boundary rules of apply_boundary_conditions (src/boundary_conditions.f90:186-260).

Namelist mapping (one rank): a periodic direction with N independent cells over a period L uses n = N+2 faces
and a namelist length L*(N+1)/N, because the last interior cell duplicates the first
(src/initialization.f90:329-345); a wall direction with N cells uses n = N+1 faces over L.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace
from typing import Dict, Optional, Tuple

import numpy as np

PI = 4.0 * math.atan(1.0)   # pi = 4d0*datan(1d0), src/global.f90:21


@dataclass
class Case:
    """One simulation case: the &DOMAIN/&PHYSICS/&NUMERICS/&BOUNDARY_CONDITIONS subset the step reads."""
    name: str
    nx: int                      # namelist face counts (one rank)
    ny: int
    nz: int
    Lx_i: float                  # namelist lengths
    Ly_i: float
    Lz_i: float
    grid_type: int = 1           # 1 uniform y, 2 symmetric tanh
    alpha_grid: float = 0.0
    y_bc_type: int = 1           # 0 periodic, 1 walls
    x_bc_type: int = 0           # 0 periodic, 1 inflow/outflow (the DCT-IV Poisson path only)
    z_bc_type: int = 0           # 0 periodic, 1 walls (with y walls: the 4-wall duct's Poisson path only)
    nu: float = 1e-3
    dt: float = 1e-3
    dPdx: float = 0.0
    dPdz: float = 0.0
    sgs_model: int = 0
    Cs_vreman: float = 0.17
    C_amd: float = 1.0 / 3.0
    flat_wall_model_flag: int = 0
    advection_scheme: int = 0    # 0 skew-symmetric, 1 divergence form, 2 skew + upwind-biased dissipation
    adv_order: int = 3           # advection_scheme = 2: dissipation order (3 or 5)
    adv_beta0: float = 0.05      # advection_scheme = 2: dissipation coefficient
    adv_wall_layers: int = -1
    wm_filter_mode: int = -1
    wm_filter_Tf_fac: float = 1.0
    flow_forcing_mode: int = 0
    Ub_target: float = 0.0
    ic: str = "tgv"              # tgv | poiseuille_uniform | reichardt_gauss | zero
    ic_amplitude: float = 1.0    # TGV amplitude / Poiseuille bulk velocity / Reichardt u_tau
    noise: float = 0.0           # noise amplitude (uniform half-width, or Gaussian sigma)
    seed: int = 0
    nsteps: int = 100
    meta: Dict[str, object] = field(default_factory=dict)

    # ---- derived sizes ----
    @property
    def nxg(self) -> int:
        return self.nx + 1

    @property
    def nyg(self) -> int:
        return self.ny + 1

    @property
    def nzg(self) -> int:
        return self.nz + 1

    @property
    def cells(self) -> Tuple[int, int, int]:
        """Independent cells (Nx, Ny, Nz): periodic directions drop the duplicated last cell."""
        nyc = self.ny - 2 if self.y_bc_type == 0 else self.ny - 1
        return (self.nx - 2, nyc, self.nz - 2)

    @property
    def n_cells(self) -> int:
        a, b, c = self.cells
        return a * b * c

    def shapes(self) -> Dict[str, Tuple[int, int, int]]:
        """Ghosted Fortran shapes of the reference's arrays (src/initialization.f90:204-219)."""
        nx, ny, nz, nxg, nyg, nzg = self.nx, self.ny, self.nz, self.nxg, self.nyg, self.nzg
        return {"U": (nx, nyg, nzg), "V": (nxg, ny, nzg), "W": (nxg, nyg, nz), "P": (nxg, nyg, nzg),
                "rhs_u": (nx - 2, nyg - 2, nzg - 2), "rhs_v": (nxg - 2, ny - 2, nzg - 2),
                "rhs_w": (nxg - 2, nyg - 2, nz - 2), "rhs_p": (nxg - 1, nyg - 2, nzg - 1),
                "tau_x": (nx, 2, nzg), "tau_z": (nxg, 2, nz)}

    def with_(self, **kw) -> "Case":
        return replace(self, **kw)


# ----------------------------------------------------------------------------------------------------------
# Grid: generateGrid (src/genGridandIC.f90:14-265), grid types 1 and 2, uniform x and z.
def faces(case: Case) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    nx, ny, nz = case.nx, case.ny, case.nz
    x = np.array([case.Lx_i * float(i - 1) / float(nx - 1) for i in range(1, nx + 1)], dtype=np.float64)
    z = np.array([case.Lz_i * float(k - 1) / float(nz - 1) for k in range(1, nz + 1)], dtype=np.float64)
    if case.grid_type == 1:
        y = np.array([case.Ly_i * float(j - 1) / float(ny - 1) for j in range(1, ny + 1)], dtype=np.float64)
    elif case.grid_type == 2:
        a = case.alpha_grid
        y = np.empty(ny, dtype=np.float64)
        for j in range(1, ny + 1):
            eta = float(j - 1) / float(ny - 1)
            y[j - 1] = case.Ly_i * 0.5 * (1.0 + math.tanh(a * (eta - 0.5)) / math.tanh(0.5 * a))
    else:
        raise ValueError(f"grid_type {case.grid_type} is outside the single-phase path (1 or 2)")
    return x, y, z


def centres(f: np.ndarray) -> np.ndarray:
    """Ghosted centres of a face array (src/initialization.f90:250-270): interior midpoints plus mirrored ghosts."""
    n = f.size
    m = 0.5 * (f[:-1] + f[1:])
    c = np.empty(n + 1)
    c[1:n] = m
    c[0] = m[0] - 2.0 * (m[0] - f[0])
    c[n] = m[-1] + 2.0 * (f[-1] - m[-1])
    return c


# ----------------------------------------------------------------------------------------------------------
# Ghost fill of the velocity arrays (apply_boundary_conditions with one rank, src/boundary_conditions.f90:186-260).
def fill_ghosts(case: Case, U: np.ndarray, V: np.ndarray, W: np.ndarray) -> None:
    """Apply the periodic x/z wraps, the y rule (periodic or no-slip mirror), then the x/z wraps again."""
    nx, ny, nz, nxg, nyg, nzg = case.nx, case.ny, case.nz, case.nxg, case.nyg, case.nzg

    def px(F, faces_):
        if faces_:
            F[0] = F[nx - 2]; F[nx - 1] = F[1]
        else:
            F[0] = F[nxg - 3]; F[nxg - 2] = F[1]; F[nxg - 1] = F[2]

    def pz(F, faces_):
        if faces_:
            F[:, :, 0] = F[:, :, nz - 2]; F[:, :, nz - 1] = F[:, :, 1]
        else:
            F[:, :, 0] = F[:, :, nzg - 3]; F[:, :, nzg - 2] = F[:, :, 1]; F[:, :, nzg - 1] = F[:, :, 2]

    def py(F, faces_):
        if case.y_bc_type == 0:
            if faces_:
                F[:, 0] = F[:, ny - 2]; F[:, ny - 1] = F[:, 1]
            else:
                F[:, 0] = F[:, nyg - 3]; F[:, nyg - 2] = F[:, 1]; F[:, nyg - 1] = F[:, 2]
        else:   # apply_Robin_bc_y with alpha = 0: faces -> 0, centres -> mirror
            if faces_:
                F[:, 0] = 0.0 * F[:, 1]; F[:, ny - 1] = 0.0 * F[:, ny - 2]
            else:
                F[:, 0] = -F[:, 1]; F[:, nyg - 1] = -F[:, nyg - 2]

    for _ in range(2):
        px(U, True); px(V, False); px(W, False)
        pz(U, False); pz(V, False); pz(W, True)
        if _ == 0:
            py(U, False); py(V, True); py(W, False)


def allocate_state(case: Case):
    s = case.shapes()
    U = np.zeros(s["U"], order="F"); V = np.zeros(s["V"], order="F")
    W = np.zeros(s["W"], order="F"); P = np.zeros(s["P"], order="F")
    return U, V, W, P


def _reichardt_plus(yp: float) -> float:
    """Reichardt mean profile of generateIC's ic_type 4 (src/genGridandIC.f90:541-552), C = 5.17, k = 0.41."""
    C_ch, k_ch = 5.17, 0.41
    return (1.0 / k_ch * math.log(1.0 + k_ch * yp) +
            (C_ch - (1.0 / k_ch) * math.log(k_ch)) * (1.0 - math.exp(-yp / 11.0) - yp / 11.0 * math.exp(-yp / 3.0)))


def reichardt_bulk(Re_tau: float) -> float:
    """Bulk U+ of the Reichardt profile: trapezoidal rule of src/genGridandIC.f90:466-481, divided by Re_tau."""
    n_int = 10000
    dyp = Re_tau / float(n_int)
    s = 0.0
    for ii in range(0, n_int + 1):
        yp = max(float(ii) * dyp, 1e-10)
        up = _reichardt_plus(yp)
        s = s + (0.5 * up if ii in (0, n_int) else up)
    return s * dyp / Re_tau


def initial_condition(case: Case):
    """Velocity (and pressure) arrays of the case's initial condition in the reference's ghosted shapes.

    tgv: U = A sin(kx x_f) cos(ky y_c) cos(kz z_c), V = -A (kx/ky) cos(kx x_c) sin(ky y_f) cos(kz z_c), W = 0,
         sampled at the staggered positions as generateIC's ic_type 6 (src/genGridandIC.f90:304-356), with
         every wavenumber 2*pi/(L_in - d) of the discrete period (the reference's ic_type 6 uses 2*pi/Ly in y,
         which is not periodic on the duplicated-cell grid); P = A^2 (cos 2x + cos 2y)(cos 2z + 2)/16 at centres
         (ignored by the step: the pressure is a pure per-stage projection).
    poiseuille_uniform: U = 1.5 Ub (1 - (y_c - 1)^2) plus i.i.d. uniform noise of half-width `noise` on every
         independent U, V, W value, numpy PCG64(seed), drawn U then V then W, each in Fortran order.
    reichardt_gauss: U = u_tau U+(y+) of the Reichardt profile (Re_tau = u_tau h / nu, h = Ly/2) plus Gaussian
         noise of standard deviation `noise` on every independent value, PCG64(seed), same order.
    """
    U, V, W, P = allocate_state(case)
    x, y, z = faces(case)
    nx, ny, nz, nxg, nyg, nzg = case.nx, case.ny, case.nz, case.nxg, case.nyg, case.nzg
    # 0-based numpy index a <-> Fortran index a+1
    xc = np.zeros(nxg); xc[1:nxg - 1] = 0.5 * (x[:-1] + x[1:])
    yc = np.zeros(nyg); yc[1:nyg - 1] = 0.5 * (y[:-1] + y[1:])
    zc = np.zeros(nzg); zc[1:nzg - 1] = 0.5 * (z[:-1] + z[1:])
    Nx, Ny, Nz = case.cells
    if case.ic == "tgv":
        A = case.ic_amplitude
        kx = 2.0 * PI / (case.Lx_i - (x[1] - x[0]))
        ky = 2.0 * PI / (case.Ly_i - (y[1] - y[0])) if case.y_bc_type == 0 else 2.0 * PI / case.Ly_i
        kz = 2.0 * PI / (case.Lz_i - (z[1] - z[0]))
        sx_f = np.sin(kx * x)
        for kk in range(1, nzg - 1):
            czc = math.cos(kz * zc[kk])
            for jj in range(1, nyg - 1):
                U[:, jj, kk] = A * sx_f * math.cos(ky * yc[jj]) * czc
        cx_c = np.cos(kx * xc[1:nxg - 1])
        for kk in range(1, nzg - 1):
            czc = math.cos(kz * zc[kk])
            for jj in range(1, ny - 1):
                V[1:nxg - 1, jj, kk] = -A * (kx / ky) * cx_c * math.sin(ky * y[jj]) * czc
        X, Y, Z = np.meshgrid(xc, yc, zc, indexing="ij")
        P[:] = A * A * (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0) / 16.0
    elif case.ic in ("poiseuille_uniform", "reichardt_gauss", "zero"):
        prof = np.zeros(nyg)
        for jj in range(1, nyg - 1):
            if case.ic == "poiseuille_uniform":
                Ub = case.ic_amplitude
                prof[jj] = 1.5 * Ub * (1.0 - (yc[jj] - 1.0) ** 2)
            elif case.ic == "reichardt_gauss":
                u_tau = case.ic_amplitude
                h = 0.5 * case.Ly_i
                Re_tau = u_tau * h / case.nu
                y_norm = 2.0 * yc[jj] / case.Ly_i - 1.0
                yp = (1.0 - y_norm) * Re_tau if y_norm >= 0.0 else (1.0 + y_norm) * Re_tau
                prof[jj] = _reichardt_plus(yp) * u_tau
        U[:, :, :] = prof[None, :, None]
        if case.noise > 0.0:
            rng = np.random.Generator(np.random.PCG64(case.seed))
            nyv = Ny if case.y_bc_type == 0 else Ny - 1   # interior V faces
            if case.ic == "reichardt_gauss":
                draw = lambda shp: rng.normal(0.0, case.noise, size=shp[::-1]).transpose(2, 1, 0)
            else:
                draw = lambda shp: rng.uniform(-case.noise, case.noise, size=shp[::-1]).transpose(2, 1, 0)
            U[1:1 + Nx, 1:1 + Ny, 1:1 + Nz] += draw((Nx, Ny, Nz))
            V[1:1 + Nx, 1:1 + nyv, 1:1 + Nz] += draw((Nx, nyv, Nz))
            W[1:1 + Nx, 1:1 + Ny, 1:1 + Nz] += draw((Nx, Ny, Nz))
    else:
        raise ValueError(f"unknown initial condition {case.ic!r}")
    fill_ghosts(case, U, V, W)
    return U, V, W, P


# ----------------------------------------------------------------------------------------------------------
# Configurations.  Periodic lengths follow the n = N+2, L_in = L(N+1)/N mapping.
def _periodic(N: int, L: float) -> Tuple[int, float]:
    return N + 2, L * (N + 1) / N


def tgv(N: int = 64, Re: float = 1600.0, dt: float = 1e-3, nsteps: int = 100, name: Optional[str] = None) -> Case:
    """Taylor-Green vortex in the triply periodic cube [0, 2pi]^3 on N^3 independent cells (DNS)."""
    n, L = _periodic(N, 2.0 * PI)
    return Case(name=name or f"tgv{N}", nx=n, ny=n, nz=n, Lx_i=L, Ly_i=L, Lz_i=L, grid_type=1, y_bc_type=0,
                nu=1.0 / Re, dt=dt, sgs_model=0, ic="tgv", ic_amplitude=1.0, nsteps=nsteps)


def channel(Nx: int, Ny: int, Nz: int, Lx: float, Lz: float, alpha: float, Re_tau: float, Ub: float, dt: float,
            seed: int, nsteps: int, name: str, noise_frac: float = 0.1) -> Case:
    """Constant-flux DNS channel, walls at y = 0 and 2, laminar Poiseuille IC plus uniform noise of
    noise_frac times the centreline velocity."""
    nx, Lxi = _periodic(Nx, Lx)
    nz, Lzi = _periodic(Nz, Lz)
    Uc = 1.5 * Ub
    return Case(name=name, nx=nx, ny=Ny + 1, nz=nz, Lx_i=Lxi, Ly_i=2.0, Lz_i=Lzi, grid_type=2, alpha_grid=alpha,
                y_bc_type=1, nu=1.0 / Re_tau, dt=dt, sgs_model=0, flow_forcing_mode=1, Ub_target=Ub,
                ic="poiseuille_uniform", ic_amplitude=Ub, noise=noise_frac * Uc, seed=seed, nsteps=nsteps)


def chan180(dt: float = 2e-3, nsteps: int = 200) -> Case:
    """Re_tau = 180 channel DNS, 4pi x 2 x 4pi/3 on 128 x 96 x 128 cells, tanh 2.0, constant flux."""
    return channel(128, 96, 128, 4.0 * PI, 4.0 * PI / 3.0, 2.0, 180.0, 15.6, dt, 180, nsteps, "chan180")


def chan550(dt: float = 4e-4, nsteps: int = 100) -> Case:
    """Re_tau = 550 channel DNS, 2pi x 2 x pi on 256 x 192 x 256 cells, tanh 2.0, constant flux (the throughput
    case)."""
    return channel(256, 192, 256, 2.0 * PI, PI, 2.0, 550.0, 18.3, dt, 550, nsteps, "chan550")


def les395(dt: float = 1e-3, nsteps: int = 500) -> Case:
    """Wall-modelled AMD LES at Re_tau = 395, 2pi x 2 x pi on 96 x 64 x 96 cells, tanh 1.5, dPdx = 1, Reichardt
    mean plus Gaussian noise (sigma = 5% of the profile's bulk velocity)."""
    nx, Lxi = _periodic(96, 2.0 * PI)
    nz, Lzi = _periodic(96, PI)
    Ub = reichardt_bulk(395.0)
    return Case(name="les395", nx=nx, ny=65, nz=nz, Lx_i=Lxi, Ly_i=2.0, Lz_i=Lzi, grid_type=2, alpha_grid=1.5,
                y_bc_type=1, nu=1.0 / 395.0, dt=dt, dPdx=1.0, sgs_model=2, flat_wall_model_flag=1,
                ic="reichardt_gauss", ic_amplitude=1.0, noise=0.05 * Ub, seed=395, nsteps=nsteps)


# The reference's three regression cases on 18 x 17 x 18 faces (tests/regression/*/input_parameters), with a
# seeded noise field standing in for the unseeded Random_number of ic_type 4.
def tgv_small() -> Case:
    L = 6.283185307179586
    return Case(name="tgv_small", nx=18, ny=17, nz=18, Lx_i=L, Ly_i=L, Lz_i=L, grid_type=1, y_bc_type=0, nu=0.01,
                dt=0.01, sgs_model=0, ic="tgv", ic_amplitude=1.0, nsteps=20)


def chan_small() -> Case:
    return Case(name="chan_small", nx=18, ny=17, nz=18, Lx_i=3.0, Ly_i=2.0, Lz_i=1.5, grid_type=1, y_bc_type=1,
                nu=0.005, dt=0.002, dPdx=1.0, sgs_model=0, ic="reichardt_gauss", ic_amplitude=1.0,
                noise=0.05 * 5.0, seed=17, nsteps=20)


def chan_les_amd_small() -> Case:
    return Case(name="chan_les_amd_small", nx=18, ny=17, nz=18, Lx_i=3.0, Ly_i=2.0, Lz_i=1.5, grid_type=2,
                alpha_grid=2.0, y_bc_type=1, nu=0.002531645569620253, dt=0.002, dPdx=1.0, sgs_model=2,
                Cs_vreman=0.17, flat_wall_model_flag=1, ic="reichardt_gauss", ic_amplitude=1.0, noise=0.05 * 5.0,
                seed=18, nsteps=20)


def chan_les_vreman_small() -> Case:
    """The wall-modelled LES regression grid with the Vreman closure (sgs_model = 1, Cs_vreman = 0.17) in place of
    AMD: the other eddy-viscosity branch of compute_vreman (src/sgs_model.f90:212-216)."""
    return chan_les_amd_small().with_(name="chan_les_vreman_small", sgs_model=1)


def inflow_outflow(nx: int = 18, ny: int = 17, nz: int = 18, grid_type: int = 2, name: Optional[str] = None) -> Case:
    """An inflow/outflow-x grid (x_bc_type = 1) with y walls and periodic z, 3 x 2 x 1.5: the pressure solve of the
    DCT-IV path (src/projection.f90:124-130,334-343) only; such a case does not step."""
    return Case(name=name or f"inflow_outflow{nx}", nx=nx, ny=ny, nz=nz, Lx_i=3.0, Ly_i=2.0, Lz_i=1.5,
                grid_type=grid_type, alpha_grid=2.0, y_bc_type=1, x_bc_type=1, nu=0.01, dt=0.002, ic="zero")


def duct(nx: int = 18, ny: int = 17, nz: int = 18, grid_type: int = 2, name: Optional[str] = None) -> Case:
    """A 4-wall duct (z_bc_type = 1 with y walls, periodic x), 3 x 2 x 1.5: the pressure solve of the z-eigenmode
    path (src/projection.f90:172-217) only; such a case does not step."""
    return Case(name=name or f"duct{nx}", nx=nx, ny=ny, nz=nz, Lx_i=3.0, Ly_i=2.0, Lz_i=1.5, grid_type=grid_type,
                alpha_grid=2.0, y_bc_type=1, z_bc_type=1, nu=0.01, dt=0.002, ic="zero")


def inflow_duct(nx: int = 18, ny: int = 17, nz: int = 18, grid_type: int = 2, name: Optional[str] = None) -> Case:
    """A 4-wall duct with inflow/outflow x (x_bc_type = 1, z_bc_type = 1, y walls), 3 x 2 x 1.5: the DCT-IV x transform
    with the z-eigenmode transform (the reference's CPU build; src/projection.f90:124-130,172-217,334-343); the
    pressure solve only."""
    return Case(name=name or f"inflow_duct{nx}", nx=nx, ny=ny, nz=nz, Lx_i=3.0, Ly_i=2.0, Lz_i=1.5, grid_type=grid_type,
                alpha_grid=2.0, y_bc_type=1, x_bc_type=1, z_bc_type=1, nu=0.01, dt=0.002, ic="zero")


def spanwise_wall(nx: int = 18, ny: int = 18, nz: int = 18, name: Optional[str] = None) -> Case:
    """Spanwise walls alone (z_bc_type = 1 with periodic x and y), 3 x 2 x 1.5: the pressure solve of the z-wall path
    (src/projection.f90:136-143,219-250) only; such a case does not step."""
    return Case(name=name or f"spanwise_wall{nx}", nx=nx, ny=ny, nz=nz, Lx_i=3.0, Ly_i=2.0, Lz_i=1.5, grid_type=1,
                y_bc_type=0, z_bc_type=1, nu=0.01, dt=0.002, ic="zero")


CONFIGS = {"tgv64": tgv, "chan180": chan180, "les395": les395, "chan550": chan550,
           "tgv_small": tgv_small, "chan_small": chan_small, "chan_les_amd_small": chan_les_amd_small,
           "chan_les_vreman_small": chan_les_vreman_small}


def get(name: str, **kw) -> Case:
    if name not in CONFIGS:
        raise KeyError(f"unknown configuration {name!r}; known: {sorted(CONFIGS)}")
    return CONFIGS[name](**kw)
