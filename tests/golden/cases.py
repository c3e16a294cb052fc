"""Golden cases: configurations on which the unmodified reference was run (on a
B200, built for sm_100a by oracle/ref_build.py) from restart-injected initial
states.  make_golden.py in this folder generates the fixtures; the tests compare
the oracle and the CUDA path against them.
"""
from __future__ import annotations

import math
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from penguin_b200 import params as P  # noqa: E402

T0_DISK = 5.0 * 2.0 * math.pi      # restart at 5 orbits: planet mass halfway up its 10-orbit ramp
SEED = 7


def _disk64():
    return P.reference_disk(64, 192)


def _disk32(**kw):
    return P.reference_disk(32, 96).replace(**kw)


def cases() -> list[dict]:
    """name, params, initial-state kind/seed, restart time, step limit, end time."""
    # tol: relative-L1 bound (density, pressure and momentum) between the oracle and
    # the reference's own output, set from the measured differences with margin.
    # Cases with the planet amplify rounding-level differences near it step by step.
    # cuda_tol: the same bound for the CUDA path against the reference's output,
    # 1e-12 or below wherever the reference itself allows it.  floors.json (beside
    # this file, made by make_golden.py's floor phase) holds how far the reference
    # moves from itself when every input density moves by one ulp; the three bounds
    # above 1e-12 sit at that floor: the Sod tube after 10 steps (CUDA 1.65e-12,
    # floor 2.55e-12) and to t = 0.2 (8.7e-13, floor 1.2e-12), where the limiter
    # and monotonicity branches at the discontinuities amplify rounding, and the
    # total-energy adiabatic disk (5.9e-11, floor 4.1e-11; see adiabatic_cases).
    # The CUDA kernels apply the 4th-order slopes as per-index weights built from
    # the reference's own rounded grid moments (penguin_b200/csrc/pg_engine.cu), so
    # what remains is the rounding of the reference's per-call arithmetic.
    sod = P.sod_tube(1024)
    out = [
        dict(name="sod_n1", params=sod, init="sod", t0=0.0, max_step=1, end_time=0.2, tol=1e-14, cuda_tol=1e-14),
        dict(name="sod_n10", params=sod, init="sod", t0=0.0, max_step=10, end_time=0.2, tol=1e-11, cuda_tol=3e-12),
        dict(name="sod_t02", params=sod, init="sod", t0=0.0, max_step=1000000000, end_time=0.2, tol=5e-12,
             cuda_tol=1e-12),
    ]
    for n, tol, ctol in ((1, 1e-12, 1e-14), (10, 1e-10, 2e-13), (50, 1e-9, 1e-12)):
        out.append(dict(name=f"disk64_n{n}", params=_disk64(), init="disk", t0=T0_DISK, max_step=n, end_time=1.0e30,
                        tol=tol, cuda_tol=ctol))
    variants = {
        "sweeps": dict(visc_flag=0, OrbAdv_flag=0, kill_flag=0, planet_mass=0.0),
        "visc": dict(visc_flag=1, OrbAdv_flag=0, kill_flag=0, planet_mass=0.0),
        "orbadv": dict(visc_flag=0, OrbAdv_flag=1, kill_flag=0, planet_mass=0.0),
        "kill_planet": dict(visc_flag=0, OrbAdv_flag=0, kill_flag=1),
    }
    for k, kw in variants.items():
        out.append(dict(name=f"disk32_{k}_n10", params=_disk32(**kw), init="disk", t0=T0_DISK, max_step=10,
                        end_time=1.0e30, tol=2e-12 if k == "kill_planet" else 1e-14, cuda_tol=3e-14))
    return out + adiabatic_cases() + two_body_cases() + preset_cases()


def preset_default(nr: int = 64, nphi: int = 192):
    """The reference's include/para_files/default.h at a reduced resolution: log
    radii on [0.3, 10], Sigma ~ r^-1.5, flat h/r 0.05, alpha 1e-3, the two-body
    frame with q 1e-3 on an e = 0.05 orbit (smoothing 0.5 H, mass ramp over one
    orbit), cooling with beta 0.01 (cool_flag 1; the EOS is isothermal),
    zero-gradient inner and analytic outer boundaries, orbital advection, no
    wave damping, CFL 0.3."""
    return P.Params(
        ndim=2, xres=nr, yres=nphi, geomx=1, geomy=3, gridx=1, gridy=0, xmin=0.3, xmax=10.0,
        EOS_flag=0, internal_e_flag=1, gam=1.0, CFL=0.3, bound_lft=1, bound_rgh=0, init_flag=2,
        frame_omega=1.0, p_alpha=1.5, p_beta=1.0, ss_alpha=1.0e-3, sc_h=0.05, planet_radius=1.0,
        visc_flag=1, OrbAdv_flag=1, kill_flag=0, kill_width=1.0, kill_width_out=1.0, n_planet=1,
        planet_mass=1.0e-3, planet_ecc=0.05, rs_fac=0.5, ramp_time=2.0 * math.pi,
        cool_flag=1, beta_cool=0.01, twobd_flag=1)


def preset_cases() -> list[dict]:
    """The reference's default configuration (include/para_files/default.h; CI_Tau.h
    differs only in resolution), 64x192, from the seeded disk after 5 orbits."""
    p = preset_default()
    return [dict(name="default64_n10", params=p, init="disk", t0=T0_DISK, max_step=10, end_time=1.0e30,
                 tol=1e-13, cuda_tol=1e-13)]


def two_body_cases() -> list[dict]:
    """The 64x192 planet-disk in the two-body frame (twobd_flag 1): the star and
    the planet orbit their barycentre and both pull as inertial point masses
    (src/planet/planet.cu:135-175, src/solver/force/forces.cu:89-106, 182-327),
    on a circular orbit and on an eccentric one (e = 0.05).

    The disk starts in equilibrium about the origin, not the barycentre, so it
    departs from init_C by ~2e-3 in ten steps instead of the 1e-4 noise.  Wave
    damping pulls that departure back with the __sinf ramp the oracle evaluates
    as sinf (see adiabatic_cases), so the oracle's bound is looser (95 % of its
    difference from the reference lies in the damping zones); the CUDA path,
    with the reference's intrinsic, keeps the tight bound."""
    base = _disk64().replace(twobd_flag=1)
    return [
        dict(name="tb64_n1", params=base, init="disk", t0=T0_DISK, max_step=1, end_time=1.0e30,
             tol=5e-12, cuda_tol=1e-14),
        dict(name="tb64_n10", params=base, init="disk", t0=T0_DISK, max_step=10, end_time=1.0e30,
             tol=1e-9, cuda_tol=3e-13),
        dict(name="tb64_ecc_n10", params=base.replace(planet_ecc=0.05), init="disk", t0=T0_DISK, max_step=10,
             end_time=1.0e30, tol=1e-9, cuda_tol=3e-13),
    ]


def adiabatic_cases() -> list[dict]:
    """Adiabatic planet-disks (EOS_flag 2, gamma 1.4) at 64x192 with the planet,
    viscosity, orbital advection and damping of the disk cases: the internal-energy
    form (internal_e_flag 1, the reference's default), the total-energy form, and
    Newtonian cooling (cool_flag 1 and 2).  The cooled disks start 20 % hotter than
    cs^2 (p = 1.2 cs^2 Sigma, init "disk_hot") so that cooling has a temperature
    excess to relax.

    tol (oracle vs the reference) is set from the measured differences with
    margin.  Two effects set them.  (1) The damping ramp is the FP32 intrinsic
    __sinf (src/killwave/killwave.cu:8-14), which the oracle evaluates as sinf:
    the ramps differ by up to ~4e-7, which is invisible when damping acts on the
    1e-4 noise but shows (~1e-9 per step in the damping zones) when it pulls the
    20 % pressure excess of the hot disks back.  The one-step cooling case
    therefore runs without damping and pins the cooling law at rounding level;
    the CUDA path uses the same intrinsic as the reference and keeps the tight
    bound everywhere.  (2) The total-energy form is ill-conditioned: its pressure
    is the small difference of the total and the orbital kinetic energy, so a
    1e-15 change of the input moves p by ~6e-11 after one step (that form heats
    the disk several-fold in ten steps, in the reference as here)."""
    base = _disk64().replace(EOS_flag=2, gam=1.4)
    e1 = dict(internal_e_flag=1)
    c1 = dict(internal_e_flag=1, cool_flag=1, beta_cool=0.5)
    c2 = dict(internal_e_flag=1, cool_flag=2, beta_cool=0.05)
    et = dict(internal_e_flag=0)
    specs = [  # name, params, init, steps, tol, cuda_tol
        ("adi64_n10", e1, "disk", 10, 1e-10, 2e-13),
        ("adi64_etot_n1", et, "disk", 1, 1e-10, 3e-13),
        ("adi64_etot_n10", et, "disk", 10, 1e-7, 1.2e-10),
        ("adi64_cool1_nokill_n1", dict(c1, kill_flag=0), "disk_hot", 1, 1e-14, 1e-14),
        ("adi64_cool1_n10", c1, "disk_hot", 10, 2e-9, 3e-13),
        ("adi64_cool2_n10", c2, "disk_hot", 10, 2e-10, 3e-13),
    ]
    return [dict(name=n, params=base.replace(**kw), init=init, t0=T0_DISK, max_step=m, end_time=1.0e30,
                 tol=tol, cuda_tol=ctol) for n, kw, init, m, tol, ctol in specs]


def dust_cases() -> list[dict]:
    """Gas + one dust fluid (the gas+dust disk's physics at 64x192): alpha 1e-4, q 3e-4,
    Stokes 0.01 and 0.1, dust-to-gas 0.01.  The dust starts from init_CD (the
    reference's restart loads gas only).  tol: oracle vs the reference's output for
    the gas and dust fields; the reference's dust reconstruction reads a stale
    shared-memory flattening coefficient (see oracle/oracle.c, dust_flux), so these
    fixtures come from its kernels run by oracle/ref_stages.cu with that memory
    zeroed (make_golden.py, _run_dust).  Measured oracle agreement: 1e-15 after one
    step, 2e-11 after ten (the planet amplifies gas rounding as in disk64_n10)."""
    out = []
    for st, tag in ((0.01, "st001"), (0.1, "st01")):
        p = P.reference_disk(64, 192, q=3.0e-4, alpha=1.0e-4).replace(dust_flag=1, Stokes=st, D_G_ratio=0.01)
        out.append(dict(name=f"dust64_{tag}_n10", params=p, init="disk", t0=T0_DISK, max_step=10, end_time=1.0e30,
                        tol=1e-10, cuda_tol=5e-13, dust=True))
    p = P.reference_disk(64, 192, q=3.0e-4, alpha=1.0e-4).replace(dust_flag=1, Stokes=0.1, D_G_ratio=0.01)
    out.append(dict(name="dust64_st01_n1", params=p, init="disk", t0=T0_DISK, max_step=1, end_time=1.0e30,
                    tol=1e-12, cuda_tol=1e-14, dust=True))
    out.append(dict(name="dust64_st01_noplanet_n10", params=p.replace(planet_mass=0.0), init="disk", t0=T0_DISK,
                    max_step=10, end_time=1.0e30, tol=1e-10, cuda_tol=5e-13, dust=True))
    return out


def ave_cases() -> list[dict]:
    """ave_flag: the 64x192 disk case of ``cases`` built with the time average on
    (interval 10, longer than the 10 steps' 0.44, so no dump clips a step): at
    max_step the reference writes the state and the trapezoid average of the
    states over the steps divided by the interval (main.cu:343-351, 411-422;
    src/output/output.cu:250-330) as binary_<label>_ave_00001."""
    return [dict(name="disk64_ave_n10", params=_disk64(), init="disk", t0=T0_DISK, max_step=10, end_time=1.0e30,
                 tol=1e-10, cuda_tol=2e-12, ave_interval=10.0)]


def size_cases() -> list[dict]:
    """The workloads at their own sizes, built from the reference for a direct
    comparison on the GPU (the outputs, 100 MB and more, are made at test time
    and not stored): the 1024x3072 planet-disk from t = 0 (the workload's start,
    planet mass ramping from zero) and from 5 orbits (planet at half mass), and
    the 256x768 gradient disk (no wave damping).  The 1024x3072 disk takes the
    single damping width the reference has (2.4 H on both sides)."""
    d1024 = P.reference_disk(1024, 3072)
    return [
        dict(name="size_disk1024_n5", params=d1024, init="disk", seed=1234, t0=0.0, max_step=5, end_time=1.0e30,
             cuda_tol=1e-12, tools=("slopes",)),
        dict(name="size_disk1024_orb5_n5", params=d1024, init="disk", seed=1234, t0=T0_DISK, max_step=5,
             end_time=1.0e30, cuda_tol=1e-12),
        dict(name="size_adj256_n20", params=P.adjoint_disk(), init="disk", seed=1234, t0=0.0, max_step=20,
             end_time=1.0e30, cuda_tol=1e-12),
    ]


def timing_cases() -> list[dict]:
    """Full-size planet-disk runs of the reference, used only to time it on the B200."""
    c2 = P.reference_disk(1024, 3072)
    return [
        dict(name="ref_disk1024_n20", params=c2, init="disk", t0=T0_DISK, max_step=20, end_time=1.0e30),
        dict(name="ref_disk1024_n220", params=c2, init="disk", t0=T0_DISK, max_step=220, end_time=1.0e30),
    ]


def cases3d() -> list[dict]:
    """3D configurations (ndim 3): the reference's spherical preset
    (include/para_files/Adiabatic_CPD.h) at 32x64x16, adiabatic with wave damping,
    analytic radial ghosts and reflecting polar boundaries, and an isothermal
    variant with zero-gradient / reflecting radial ends and a zero-gradient upper
    polar boundary, both restarted after one orbit (planet at full mass) with
    seeded noise in density and in the radial and polar velocities; and a
    cartesian box (32x32x16) with structure at every scale.  The fixtures hold
    only the output fields (the initial states are regenerated from the seeds).

    The preset's grids put 6e-4 wide cells at r = 1 and phi = pi, and there the
    reference's arithmetic amplifies rounding by x / dx and more (its 4th-order
    moments (x1^4 - x0^4) / (x1^3 - x0^3), src/solver/recon/recon.cu:242-301,
    and x_l + u dt in the characteristic states, src/solver/riemann/states.cu:
    27-60): the same unmodified sources compiled with -fmad=false run 3.4e-10
    from the default build after 10 steps (floors.json "fma_floor", made by
    make_golden.py's fmafloor phase).  The oracle, which evaluates the
    reference's expressions without FMA contraction, sits at that same 3.4e-10
    (tol) and the CUDA path at 3.6e-12 (cuda_tol 5e-12, 1.5 % of that floor;
    one step: 1.7e-13 after the radial sweep, confined to the fine cells).  On
    the cartesian box (uniform grid) the two builds agree to 5e-16 and the CUDA
    path to 5e-16 (6e-15 in momentum).  The reference is deterministic and its one-ulp density
    floor is 5e-15 (floors.json "floor")."""
    sph = P.spherical_disk(32, 64, 16)
    iso = sph.replace(EOS_flag=0, gam=1.0, kill_flag=0, bound_lft=1, bound_rgh=2, bound_top=1)
    return [
        dict(name="sph32_n10", params=sph, init="sph", seed=SEED, t0=2.0 * math.pi, max_step=10,
             end_time=1.0e30, tol=1e-9, cuda_tol=5e-12, z_zdiv=16),
        dict(name="sph32_iso_n10", params=iso, init="sph", seed=SEED, t0=2.0 * math.pi, max_step=10,
             end_time=1.0e30, tol=1e-9, cuda_tol=5e-12, z_zdiv=16),
        dict(name="box32_n10", params=P.cartesian_box(32, 32, 16), init="box", seed=SEED, t0=0.0, max_step=10,
             end_time=1.0e30, tol=3e-14, cuda_tol=1e-14, z_zdiv=16),
    ]


def size_cases3d() -> list[dict]:
    """The reference's 3D preset at its own size (384x768x216, 63.7 M cells),
    restarted after one orbit from the seeded spherical disk, 3 steps: the
    reference (default build and -fmad=false build) runs at test time on the
    GPU and the CUDA path is compared with it there."""
    return [dict(name="size_sph384_n3", params=P.spherical_disk(), init="sph", seed=1234, t0=2.0 * math.pi,
                 max_step=3, end_time=1.0e30, z_zdiv=24)]


def initial_state(case: dict) -> dict:
    from penguin_b200 import initial as I

    p = case["params"]
    if case["init"] == "sph":
        return I.spherical_state(p, seed=case.get("seed", SEED), vnoise=1.0e-3)
    if case["init"] == "box":
        return I.box_state(p, seed=case.get("seed", SEED))
    if case["init"] == "sod":
        return I.sod_state(p)
    st = I.disk_state(p, seed=case.get("seed", SEED))
    if case["init"] == "disk_hot":
        st["p"] = 1.2 * st["p"]
    return st
