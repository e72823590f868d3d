"""The lightsmith problems behind the ``solve_*`` and ``driver_*`` fixtures, shared by the fixture generator
and the tests that pose them to ``ls.solve`` (importing this module needs the lightsmith sources on sys.path,
``refsrc.add_to_path``), and ``flatten_result``, the numeric content of a lightsmith result."""

from __future__ import annotations

import numpy as np

import lightsmith as ls
from device_problems import device_problem  # noqa: F401  (re-exported for the problem table)

DRUDE_LORENTZ = dict(eps_inf=5.9, wp_ev=9.0, gamma_ev=0.07,
                     poles=[{"delta_eps": 1.3, "omega0_ev": 2.6, "gamma_ev": 0.6},
                            {"delta_eps": 1.5, "omega0_ev": 3.7, "gamma_ev": 1.0}])


def c0_problem():
    """The dispersive sphere at full size: r = 40 nm Drude-Lorentz (eps_inf 5.9, wp 9.0 eV, gamma 0.07 eV, poles
    (1.3, 2.6 eV, 0.6 eV) and (1.5, 3.7 eV, 1.0 eV)) in n = 1.33, 81 wavelengths 400-800 nm, 2 nm cells, CPML
    12, courant 0.99, padding and gap 28 nm (129^3 cells), staircase, exactly 4000 steps, dft_stride 100."""
    mat = ls.DrudeLorentz(**DRUDE_LORENTZ)
    return ls.Simulation(particles=[ls.Particle(shape=ls.Sphere(radius_nm=40.0), material=mat)], medium_index=1.33,
                         wavelengths={"start_nm": 400.0, "stop_nm": 800.0, "num": 81},
                         options={"fdtd": dict(spacing_nm=2.0, pml_cells=12, courant=0.99, symmetry="off",
                                               mesh_refinement="staircase", padding_nm=28.0, pml_gap_nm=28.0,
                                               dft_stride=100, run_time_fs=3999.5 * 1.1431535 / 299.792458)})


def sphere_problem(mesh: str, symmetry: str = "off"):
    """A 16 nm Drude-Lorentz sphere (the c0 metal) in n = 1.33, 4 nm cells, CPML 8, 9 wavelengths, 400 steps."""
    mat = ls.DrudeLorentz(**DRUDE_LORENTZ)
    return ls.Simulation(particles=[ls.Particle(shape=ls.Sphere(radius_nm=16.0), material=mat)], medium_index=1.33,
                         wavelengths={"start_nm": 400.0, "stop_nm": 800.0, "num": 9},
                         options={"fdtd": dict(spacing_nm=4.0, pml_cells=8, symmetry=symmetry, mesh_refinement=mesh,
                                               padding_nm=8.0, pml_gap_nm=8.0, dft_stride=10,
                                               run_time_fs=399.5 * 2.2863 / 299.792458)})


def sphere_fields_problem():
    """The 16 nm sphere (staircase) with lightsmith's field outputs: the total E on an xz plane through it and
    the differential scattering cross section at three polar angles in two azimuthal planes."""
    from lightsmith.spec import FarFieldRequest, NearFieldRequest, Outputs
    p = sphere_problem("staircase")
    outputs = Outputs(near_field=NearFieldRequest(plane="xz", half_width_nm=24.0, points=9,
                                                  wavelengths_nm=[500.0, 700.0]),
                      far_field=FarFieldRequest(theta_deg=[0.0, 60.0, 120.0], phi_deg=[0.0, 90.0],
                                                wavelengths_nm=[500.0, 700.0]))
    return p.model_copy(update={"outputs": outputs})


def dielectric_sphere_problem():
    """A non-dispersive sphere (n = 2, radius 16 nm) in n = 1.33 with conformal interfaces (off-diagonal 1/eps)."""
    return ls.Simulation(particles=[ls.Particle(shape=ls.Sphere(radius_nm=16.0), material=ls.ConstantIndex(n_real=2.0))],
                         medium_index=1.33, wavelengths={"start_nm": 400.0, "stop_nm": 800.0, "num": 9},
                         options={"fdtd": dict(spacing_nm=4.0, pml_cells=8, symmetry="off",
                                               mesh_refinement="conformal", padding_nm=8.0, pml_gap_nm=8.0,
                                               dft_stride=10, run_time_fs=399.5 * 2.2863 / 299.792458)})


def periodic_problem(theta: float, phi: float, pol: str):
    """A square lattice (300 nm) of TiO2-like pillars (n = 2, radius 80 nm, 120 nm tall) on glass, 15 nm cells."""
    from lightsmith.problems import Circle, Incidence, PatternedLayer, PeriodicProblem, Structure2D
    CI = ls.ConstantIndex
    return PeriodicProblem(
        lattice_a1_nm=(300, 0), lattice_a2_nm=(0, 300), superstrate=CI(n_real=1.0), substrate=CI(n_real=1.45),
        layers=[PatternedLayer(thickness_nm=120, background=CI(n_real=1.0),
                               shapes=[Structure2D(profile=Circle(radius_nm=80), material=CI(n_real=2.0))])],
        wavelengths=[500.0, 650.0], incidence=Incidence(theta_deg=theta, phi_deg=phi, polarizations=[pol]),
        options={"fdtd": {"spacing_nm": 15.0, "run_time_fs": 6.0}})


def emission_problem():
    """A dipole 15 nm off an n = 2 sphere (radius 30 nm) in vacuum, 4 nm cells."""
    from lightsmith.problems import Dipole, EmissionProblem
    return EmissionProblem(particles=[ls.Particle(shape=ls.Sphere(radius_nm=30), material=ls.ConstantIndex(n_real=2.0))],
                           wavelengths=[500.0, 700.0], dipole=Dipole(position_nm=(0, 0, 45), orientation=(1, 0, 1)),
                           options={"fdtd": {"spacing_nm": 4.0, "run_time_fs": 2.0}})


# every problem of the whole-solve comparisons, by name: the sphere solves of the solve_sphere_* fixtures, the
# conformal dielectric sphere, and the periodic, emission and device problems of the driver_* fixtures
SOLVE_PROBLEMS = {
    "sphere_staircase": lambda: sphere_problem("staircase"),
    "sphere_subpixel": lambda: sphere_problem("subpixel"),
    "sphere_conformal": lambda: sphere_problem("conformal"),
    "sphere_symmetric": lambda: sphere_problem("staircase", "auto"),
    "sphere_defaults": lambda: sphere_problem("conformal", "auto"),
    "sphere_fields": sphere_fields_problem,
    "dielectric_conformal": dielectric_sphere_problem,
    "periodic_normal": lambda: periodic_problem(0.0, 0.0, "s"),
    "periodic_oblique": lambda: periodic_problem(30.0, 10.0, "p"),
    "emission": emission_problem,
    "device_2d": lambda: device_problem(2),
    "device_3d": lambda: device_problem(3),
}


def with_options(problem, **fdtd):
    """``problem`` with its FDTD options updated."""
    opts = dict(problem.options.get("fdtd", {}))
    opts.update(fdtd)
    return problem.model_copy(update={"options": {**problem.options, "fdtd": opts}})


def flatten_result(res) -> dict[str, np.ndarray]:
    """Every numeric leaf of a lightsmith result (``model_dump``), by its path, as float or complex arrays;
    provenance, warnings and strings are left out."""
    out: dict[str, np.ndarray] = {}

    def numeric(v):
        try:
            a = np.asarray(v)
        except (ValueError, TypeError):
            return None
        return a if a.dtype.kind in "fciub" and a.dtype != object else None

    def walk(path, v):
        if isinstance(v, dict):
            for k, x in v.items():
                walk(f"{path}/{k}" if path else str(k), x)
            return
        if isinstance(v, (list, tuple)) and v and all(isinstance(x, dict) for x in v):
            for i, x in enumerate(v):
                walk(f"{path}[{i}]", x)
            return
        a = numeric(v) if v is not None and not isinstance(v, (str, bool)) else None
        if a is not None and a.size:
            out[path] = a.astype(complex if a.dtype.kind == "c" else float)

    dump = res.model_dump()
    for k in ("provenance", "warnings", "method", "backend", "kind"):
        dump.pop(k, None)
    walk("", dump)
    return out
