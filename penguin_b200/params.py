"""Runtime physics/grid parameters of one disk (or tube).

The reference fixes these at compile time in ``include/parameters.h``
(flags ``:4-13``, grid ``:43-97``, hydro ``:115-127``, boundaries ``:140-149``,
disk ``:155-171``, planet ``:177-188``, domain ``:194-207``).  Here they are a
runtime struct so that one library build serves every configuration and so
that an ensemble can carry different parameters per disk.  Field names keep
the reference's spelling; ``kill_width_out`` and the dust fields are the only
additions (the reference uses ``kill_width`` for both damping zones).

``PGParams`` is the ctypes mirror of ``pg_params`` in ``include/penguin_b200.h``.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math

PI = 3.1415926535897932384626434
TWOPI = 2.0 * PI
HPI = 0.5 * PI
NPAD = 3  # recon_flag 6 (PPM on 4th-order slopes) -> 3 ghost cells (include/parameters.h:49-53)


@dataclasses.dataclass
class Params:
    ndim: int = 2
    xres: int = 1024
    yres: int = 3072
    geomx: int = 1          # 0 cartesian, 1 cylindrical radius
    geomy: int = 3          # 0 cartesian, 3 azimuth
    gridx: int = 1          # 0 linear, 1 logarithmic
    gridy: int = 0
    xmin: float = 0.4
    xmax: float = 2.5
    ymin: float = 0.0
    ymax: float = TWOPI
    EOS_flag: int = 0       # 0 locally isothermal, 2 adiabatic
    internal_e_flag: int = 1
    gam: float = 1.0
    CFL: float = 0.3
    bound_lft: int = 0      # 0 analytic initial state, 1 zero gradient, 2 reflecting
    bound_rgh: int = 0
    init_flag: int = 2      # 2 = polar disk (analytic state for ghosts and damping)
    frame_omega: float = 1.0
    p_alpha: float = 1.0
    p_beta: float = 1.0
    ss_alpha: float = 1.0e-3
    sc_h: float = 0.05
    planet_radius: float = 1.0
    visc_flag: int = 1
    OrbAdv_flag: int = 1
    kill_flag: int = 1
    kill_width: float = 5.0
    kill_width_out: float = 2.4
    n_planet: int = 1
    planet_mass: float = 1.0e-3
    planet_ecc: float = 0.0
    rs_fac: float = 0.6
    ramp_time: float = 10.0 * TWOPI
    zmin: float = HPI - 4.0 * 0.05
    zmax: float = HPI
    dust_flag: int = 0
    Stokes: float = 0.01
    D_G_ratio: float = 0.01
    cool_flag: int = 0      # 0 off, 1 t_c = beta r^1.5, 2 t_c = beta / Sigma sqrt(p/Sigma) / h
    beta_cool: float = 0.001
    twobd_flag: int = 0     # 1: star and planet orbit their barycentre (two-body frame)
    # ndim 3: polar cells, geometry (0 cartesian, 5 polar angle), grid (0 linear,
    # 1 log, 2/3/4 non-uniform) and the polar boundaries at zmin / zmax
    # (0 analytic state, 1 zero gradient, 2 reflecting, 3 periodic)
    zres: int = 1
    geomz: int = 0
    gridz: int = 0
    bound_bom: int = 2
    bound_top: int = 2

    # ----------------------------------------------------------------- sizes
    @property
    def ypad(self) -> int:
        return NPAD if self.ndim > 1 else 0

    @property
    def zpad(self) -> int:
        return NPAD if self.ndim > 2 else 0

    @property
    def xarr(self) -> int:
        return self.xres + 2 * NPAD

    @property
    def yarr(self) -> int:
        return self.yres + 2 * self.ypad

    @property
    def zarr(self) -> int:
        return self.zres + 2 * self.zpad

    @property
    def cells(self) -> int:
        return self.xres * self.yres * (self.zres if self.ndim > 2 else 1)

    def replace(self, **kw) -> "Params":
        return dataclasses.replace(self, **kw)

    def validate(self) -> None:
        if self.ndim == 3:
            validate_3d(self)
            return
        if self.ndim not in (1, 2):
            raise ValueError("ndim must be 1, 2 or 3")
        if self.ndim == 1 and self.yres != 1:
            raise ValueError("ndim 1 needs yres == 1")
        if self.xres < 2 * NPAD or (self.ndim == 2 and self.yres < 2 * NPAD):
            raise ValueError("resolution below the 3-cell stencil half-width")
        if self.EOS_flag not in (0, 2):
            raise ValueError("EOS_flag must be 0 (isothermal) or 2 (adiabatic)")
        if self.geomx not in (0, 1) or self.geomy not in (0, 3):
            raise ValueError("supported geometries: geomx 0/1, geomy 0/3")
        if any(b not in (0, 1, 2) for b in (self.bound_lft, self.bound_rgh)):
            raise ValueError("radial boundaries must be 0, 1 or 2")
        if self.n_planet not in (0, 1):
            raise ValueError("n_planet must be 0 or 1")
        if self.cool_flag not in (0, 1, 2):
            raise ValueError("cool_flag must be 0, 1 or 2")
        if self.cool_flag and not self.beta_cool > 0.0:
            raise ValueError("cooling needs beta_cool > 0")
        if self.twobd_flag not in (0, 1):
            raise ValueError("twobd_flag must be 0 or 1")


class PGParams(ctypes.Structure):
    """ctypes mirror of ``pg_params`` (include/penguin_b200.h)."""

    _fields_ = [
        ("ndim", ctypes.c_int), ("xres", ctypes.c_int), ("yres", ctypes.c_int),
        ("geomx", ctypes.c_int), ("geomy", ctypes.c_int), ("gridx", ctypes.c_int), ("gridy", ctypes.c_int),
        ("xmin", ctypes.c_double), ("xmax", ctypes.c_double), ("ymin", ctypes.c_double), ("ymax", ctypes.c_double),
        ("eos_flag", ctypes.c_int), ("internal_e_flag", ctypes.c_int),
        ("gam", ctypes.c_double), ("cfl", ctypes.c_double),
        ("bound_lft", ctypes.c_int), ("bound_rgh", ctypes.c_int), ("init_flag", ctypes.c_int),
        ("frame_omega", ctypes.c_double),
        ("p_alpha", ctypes.c_double), ("p_beta", ctypes.c_double), ("ss_alpha", ctypes.c_double),
        ("sc_h", ctypes.c_double), ("planet_radius", ctypes.c_double),
        ("visc_flag", ctypes.c_int), ("orbadv_flag", ctypes.c_int), ("kill_flag", ctypes.c_int),
        ("kill_width", ctypes.c_double), ("kill_width_out", ctypes.c_double),
        ("n_planet", ctypes.c_int),
        ("planet_mass", ctypes.c_double), ("planet_ecc", ctypes.c_double),
        ("rs_fac", ctypes.c_double), ("ramp_time", ctypes.c_double),
        ("zmin", ctypes.c_double), ("zmax", ctypes.c_double),
        ("dust_flag", ctypes.c_int),
        ("stokes", ctypes.c_double), ("d_g_ratio", ctypes.c_double),
        ("cool_flag", ctypes.c_int), ("beta_cool", ctypes.c_double),
        ("twobd_flag", ctypes.c_int),
        ("zres", ctypes.c_int), ("geomz", ctypes.c_int), ("gridz", ctypes.c_int),
        ("bound_bom", ctypes.c_int), ("bound_top", ctypes.c_int),
    ]

    @classmethod
    def from_params(cls, p: Params) -> "PGParams":
        p.validate()
        return cls(
            p.ndim, p.xres, p.yres, p.geomx, p.geomy, p.gridx, p.gridy,
            p.xmin, p.xmax, p.ymin, p.ymax, p.EOS_flag, p.internal_e_flag, p.gam, p.CFL,
            p.bound_lft, p.bound_rgh, p.init_flag, p.frame_omega,
            p.p_alpha, p.p_beta, p.ss_alpha, p.sc_h, p.planet_radius,
            p.visc_flag, p.OrbAdv_flag, p.kill_flag, p.kill_width, p.kill_width_out,
            p.n_planet, p.planet_mass, p.planet_ecc, p.rs_fac, p.ramp_time, p.zmin, p.zmax,
            p.dust_flag, p.Stokes, p.D_G_ratio, p.cool_flag, p.beta_cool, p.twobd_flag,
            p.zres, p.geomz, p.gridz, p.bound_bom, p.bound_top,
        )


# --------------------------------------------------------------- workloads
def sod_tube(n: int = 1024) -> Params:
    """1D Sod shock tube: uniform cartesian cells on [0,1], gamma 1.4, total-energy
    form, PPM + HLLC, CFL 0.5, zero-gradient (outflow) ends."""
    return Params(
        ndim=1, xres=n, yres=1, geomx=0, geomy=0, gridx=0, gridy=0,
        xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0,
        EOS_flag=2, internal_e_flag=0, gam=1.4, CFL=0.5,
        bound_lft=1, bound_rgh=1, init_flag=1,
        visc_flag=0, OrbAdv_flag=0, kill_flag=0, n_planet=1, planet_mass=0.0,
    )


def planet_disk(nr: int = 1024, nphi: int = 3072, *, q: float = 1.0e-3, alpha: float = 1.0e-3,
                h: float = 0.05, rmin: float = 0.4, rmax: float = 2.5,
                kill_in: float = 0.5, kill_out: float = 2.2, ramp_orbits: float = 10.0) -> Params:
    """2D polar planet-disk: log-spaced radii, uniform azimuth, locally isothermal
    with flat h/r (p_beta 1), Sigma ~ r^-1 (p_alpha 1), alpha viscosity, one planet
    on a fixed circular orbit at r=1 with smoothing 0.6 H and a mass ramp, wave
    damping inside ``kill_in`` and outside ``kill_out``, orbital advection on.

    The damping widths are expressed like the reference's ``kill_width`` (units of
    H at the domain edge): inner = (kill_in - rmin) / H(rmin), outer = (rmax -
    kill_out) / H(rmax), with H = h r.
    """
    kw_in = (kill_in - rmin) / (h * rmin)
    kw_out = (rmax - kill_out) / (h * rmax)
    return Params(
        ndim=2, xres=nr, yres=nphi, xmin=rmin, xmax=rmax, sc_h=h, ss_alpha=alpha,
        planet_mass=q, rs_fac=0.6, ramp_time=ramp_orbits * TWOPI,
        kill_width=kw_in, kill_width_out=kw_out, zmin=HPI - 4.0 * h,
    )


def dust_disk(nr: int = 768, nphi: int = 2048, *, stokes: float = 0.01, q: float = 3.0e-4,
              alpha: float = 1.0e-4, d_g_ratio: float = 0.01) -> Params:
    """The planet-disk with one pressureless dust fluid (dust_flag): constant
    Stokes number, initial dust-to-gas ratio ``d_g_ratio``, dust velocity from the
    drift solution (init_CD, src/init/init.cu:351-454)."""
    return planet_disk(nr, nphi, q=q, alpha=alpha).replace(dust_flag=1, Stokes=stokes, D_G_ratio=d_g_ratio)


def adiabatic_disk(nr: int = 1024, nphi: int = 3072, *, cool_flag: int = 0, beta_cool: float = 0.001,
                   gam: float = 1.4, internal_e_flag: int = 1, **kw) -> Params:
    """The planet-disk with an ideal-gas equation of state (EOS_flag 2): p starts
    at cs^2 Sigma and then evolves with the internal-energy equation (or the total
    energy with ``internal_e_flag`` 0); optional Newtonian cooling of p/Sigma
    towards cs^2 (cool_flag 1: t_c = beta r^1.5; 2: t_c = beta / Sigma
    sqrt(p/Sigma) / h; src/solver/cool/cool.cu)."""
    return planet_disk(nr, nphi, **kw).replace(EOS_flag=2, gam=gam, internal_e_flag=internal_e_flag,
                                               cool_flag=cool_flag, beta_cool=beta_cool)


def adjoint_disk(nr: int = 256, nphi: int = 768, *, q: float = 5.0e-4, alpha: float = 1.0e-3,
                 h: float = 0.05) -> Params:
    """The disk of the gradient workload: log r in [0.5, 2], h/r 0.05, alpha 1e-3,
    q 5e-4, orbital advection, no wave damping (the adjoint covers kill_flag 0)."""
    return planet_disk(nr, nphi, q=q, alpha=alpha, h=h, rmin=0.5, rmax=2.0).replace(kill_flag=0)


def reference_disk(nr: int, nphi: int, **kw) -> Params:
    """Planet-disk variant that the reference can run as-is: it has a single
    ``kill_width`` for both damping zones (src/killwave/killwave.cu:30-34), so
    both widths are set to the outer one (2.4 H)."""
    p = planet_disk(nr, nphi, **kw)
    return p.replace(kill_width=p.kill_width_out)


def disk_ensemble(n: int = 48, seed: int = 2024) -> list:
    """Seeded ensemble of planet-disks: Nr uniform over the multiples of 32 in
    [128, 512], Nphi = 3 Nr, q log-uniform in [1e-5, 3e-3], alpha log-uniform in
    [1e-4, 1e-2], h/r uniform in [0.03, 0.08]; otherwise as ``planet_disk`` on
    r in [0.4, 2.5].  Draws come from the SplitMix64 sequence, four per disk."""
    from .initial import splitmix64_uniform

    u = 0.5 * (splitmix64_uniform(seed, 4 * n).reshape(n, 4) + 1.0)  # U(0, 1)
    out = []
    sizes = list(range(128, 513, 32))
    for a, b, c, d in u:
        nr = sizes[min(int(a * len(sizes)), len(sizes) - 1)]
        q = 10.0 ** (math.log10(1.0e-5) + b * (math.log10(3.0e-3) - math.log10(1.0e-5)))
        alpha = 10.0 ** (-4.0 + c * 2.0)
        h = 0.03 + d * 0.05
        out.append(planet_disk(nr, 3 * nr, q=q, alpha=alpha, h=h))
    return out


# --------------------------------------------------------------------- 3D
def validate_3d(p: Params) -> None:
    """What the 3D form covers: the spherical disk of the reference's 3D preset
    (include/para_files/Adiabatic_CPD.h: geometries 2/4/5) or a cartesian box,
    ideal or isothermal gas, periodic azimuth, no viscosity, orbital advection,
    dust, cooling or two-body frame."""
    if (p.geomx, p.geomy, p.geomz) not in ((2, 4, 5), (0, 0, 0)):
        raise ValueError("3D geometries: spherical (2, 4, 5) or cartesian (0, 0, 0)")
    if p.xres < 2 * NPAD or p.yres < 2 * NPAD or p.zres < 2 * NPAD or p.xres % 2:
        raise ValueError("3D resolutions: at least 6 cells per axis, even xres")
    if any(g not in (0, 1, 2, 3, 4) for g in (p.gridx, p.gridy, p.gridz)):
        raise ValueError("grids must be 0 to 4")
    if p.EOS_flag not in (0, 2):
        raise ValueError("EOS_flag must be 0 (isothermal) or 2 (adiabatic)")
    if any(b not in (0, 1, 2) for b in (p.bound_lft, p.bound_rgh)):
        raise ValueError("radial boundaries must be 0, 1 or 2")
    if any(b not in (0, 1, 2, 3) for b in (p.bound_bom, p.bound_top)):
        raise ValueError("polar boundaries must be 0, 1, 2 or 3")
    if p.visc_flag or p.OrbAdv_flag or p.dust_flag or p.cool_flag or p.twobd_flag:
        raise ValueError("3D runs without viscosity, orbital advection, dust, cooling and two-body frame")
    if p.n_planet not in (0, 1):
        raise ValueError("n_planet must be 0 or 1")
    axes_np(p)  # every non-uniform spacing must exist at these resolutions
    analytic = p.kill_flag or 0 in (p.bound_lft, p.bound_rgh, p.bound_bom, p.bound_top)
    if analytic and p.init_flag != 3:
        raise ValueError("analytic ghosts or wave damping need the spherical disk state (init_flag 3)")


def spherical_disk(nr: int = 384, nphi: int = 768, ntheta: int = 216, *, q: float = 3.0e-5, h: float = 0.05,
                   gam: float = 1.4, EOS_flag: int = 2, kill: int = 1) -> Params:
    """The reference's 3D preset (include/para_files/Adiabatic_CPD.h): spherical
    r in [0.7, 1.3] (fine around r = 1), the full azimuth (fine around the
    planet), the upper half of the disk from 4 H above the midplane to the
    midplane (fine towards the midplane), ideal gas with the internal-energy
    equation, Sigma ~ r^-2.5 in vertical hydrostatic balance (init_flag 3), one
    planet of q = 3e-5 ramped over one orbit with smoothing 0.01 R_Hill-like
    length, wave damping 1 H wide at both radial edges, analytic radial ghosts
    and reflecting polar boundaries."""
    return Params(
        ndim=3, xres=nr, yres=nphi, zres=ntheta, geomx=2, geomy=4, geomz=5, gridx=2, gridy=4, gridz=3,
        xmin=0.7, xmax=1.3, ymin=0.0, ymax=TWOPI, zmin=HPI - 4.0 * h, zmax=HPI,
        EOS_flag=EOS_flag, internal_e_flag=1, gam=gam, CFL=0.3,
        bound_lft=0, bound_rgh=0, bound_bom=2, bound_top=2, init_flag=3, frame_omega=1.0,
        p_alpha=1.5 - 0.5 * 1.0 + 1.5, p_beta=1.0, ss_alpha=0.001, sc_h=h, planet_radius=1.0,
        visc_flag=0, OrbAdv_flag=0, kill_flag=kill, kill_width=1.0, kill_width_out=1.0,
        n_planet=1, planet_mass=q, planet_ecc=0.0, rs_fac=0.01, ramp_time=TWOPI,
    )


def cartesian_box(nx: int = 32, ny: int = 32, nz: int = 32, *, gam: float = 1.4, internal_e_flag: int = 0) -> Params:
    """A cartesian unit box, ideal gas: reflecting at x = 0, zero gradient at
    x = 1, periodic in y, reflecting at z = 0 and zero gradient at z = 1; no
    rotating frame and no gravity.  Its state comes from a restart file."""
    return Params(
        ndim=3, xres=nx, yres=ny, zres=nz, geomx=0, geomy=0, geomz=0, gridx=0, gridy=0, gridz=0,
        xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0,
        EOS_flag=2, internal_e_flag=internal_e_flag, gam=gam, CFL=0.4,
        bound_lft=2, bound_rgh=1, bound_bom=2, bound_top=1, init_flag=4, frame_omega=0.0,
        visc_flag=0, OrbAdv_flag=0, kill_flag=0, n_planet=1, planet_mass=0.0,
    )


# ------------------------------------------------------------- host maths
def _stretch(dmax: float, dmin: float, L: float, N: int) -> float:
    """Exponent of the power-law cell growth of the non-uniform spacings
    (src/geom/geom.cu:43,65,84); the reference's grid is NaN where it does not exist."""
    arg = 1.0 - (dmax - dmin) / (L - N * dmin)
    if not arg > 0.0:
        raise ValueError("this non-uniform spacing needs more cells (the reference's grid would be NaN)")
    return math.log(arg) / math.log(1.0 - 1.0 / N)


def _spacing(grid: int, amin: float, amax: float, length: int, p: "Params | None"):
    """Faces a[0 .. length-1] of one axis (src/geom/geom.cu:22-89): 0 linear,
    1 logarithmic, 2 fine in the middle, 3 fine towards amax, 4 fine over the
    radial extent around the middle (2-4 need the radial grid's xres/xmin/xmax
    and sc_h of ``p``)."""
    import numpy as np

    i = np.arange(length, dtype=np.float64)
    if grid == 0:
        return amin + (amax - amin) * i / float(length - 1)
    if grid == 1:
        return amin * np.exp(math.log(amax / amin) * i / float(length - 1))
    a = np.zeros(length)
    if grid == 2:
        N = (length - 1) // 2
        L = (amax - amin) / 2.0
        dmin = (L / N) / 32.0
        dmax = (PI - L) / N
        k = _stretch(dmax, dmin, L, N)
        for m in range(N):
            a[m] = (amax + amin) / 2.0 - (N - m) * dmin - (L - N * dmin) * math.pow((N - m) / N, k)
        for m in range(N + 1):
            a[N + m] = (amax + amin) / 2.0 + m * dmin + (L - N * dmin) * math.pow(m / N, k)
    elif grid == 3:
        N = length - 1
        L = amax - amin
        dmin = ((p.xmax - p.xmin) / p.xres) / 32.0
        dmax = p.sc_h / 16.0
        k = _stretch(dmax, dmin, L, N)
        for m in range(N + 1):
            a[m] = amax - (N - m) * dmin - (L - N * dmin) * math.pow((N - m) / N, k)
    elif grid == 4:
        N = p.xres // 2
        N2 = (length - 1 - 2 * N) // 2
        L = (p.xmax - p.xmin) / 2.0
        L2 = (amax - amin - 2.0 * L) / 2.0
        dmin = (L / N) / 32.0
        dmax = L2 / N2
        k = _stretch(dmax, dmin, L, N)
        for m in range(N2):
            a[m] = amin + m * dmax
        for m in range(N):
            a[m + N2] = (amax + amin) / 2.0 - (N - m) * dmin - (L - N * dmin) * math.pow((N - m) / N, k)
        for m in range(N):
            a[m + N2 + N] = (amax + amin) / 2.0 + m * dmin + (L - N * dmin) * math.pow(m / N, k)
        for m in range(N2 + 1):
            a[m + N2 + 2 * N] = amin + 2.0 * L + L2 + m * dmax
    else:
        raise ValueError(f"grid {grid}")
    return a


def make_grid_np(amin: float, amax: float, res: int, pad: int, geom: int, grid: int, p: "Params | None" = None):
    """Faces and cell 'volumes' with ghosts (src/init/init.cu:472-500, volumes
    src/geom/geom.cu:3-20).  The C library builds the authoritative copy with the
    same formulas; this numpy version is used only to place initial conditions."""
    import numpy as np

    a = np.zeros(res + 2 * pad + 1)
    a[pad:pad + res + 1] = _spacing(grid, amin, amax, res + 1, p)
    for k in range(pad):
        if grid == 1:
            a[k] = amin * math.exp(math.log(amax / amin) * float(k - pad) / float(res))
            a[res + pad + 1 + k] = amin * math.exp(math.log(amax / amin) * float(res + 1 + k) / float(res))
        else:
            a[k] = a[pad] - (a[2 * pad - k] - a[pad])
            a[res + pad + 1 + k] = a[res + pad] + (a[res + pad] - a[res + pad - 1 - k])
    dr = a[1:] - a[:-1]
    if geom == 1:
        v = dr * (a[:-1] + dr / 2.0)
    elif geom == 2:
        v = dr * (a[:-1] * a[:-1] + a[:-1] * dr + dr * dr / 3.0)
    elif geom == 5:
        v = dr * np.where(dr < 1.0e-4, np.sin(a[:-1] + 0.5 * dr), (np.cos(a[:-1]) - np.cos(a[:-1] + dr)) / dr)
    else:
        v = dr.copy()
    return a, v


def axes_np(p: "Params"):
    """(faces, volumes) of x, y and z of a 3D grid, ghosts included."""
    return (make_grid_np(p.xmin, p.xmax, p.xres, NPAD, p.geomx, p.gridx, p),
            make_grid_np(p.ymin, p.ymax, p.yres, NPAD, p.geomy, p.gridy, p),
            make_grid_np(p.zmin, p.zmax, p.zres, NPAD, p.geomz, p.gridz, p))
