"""Device problems shared by the fixture generator and the host tests of the differentiable solve (importing
this module needs the lightsmith sources on sys.path, ``refsrc.add_to_path``)."""

import lightsmith as ls


def device_problem(dimension: int):
    """A silicon waveguide width step (500 -> 700 nm) in silica between two x-normal ports: 2D at 25 nm cells
    (TE), or a 220 nm thick wire in 3D at 40 nm cells."""
    from lightsmith.problems import Box, DeviceProblem, Port, Prism, Rectangle, Structure
    si, sio2 = ls.ConstantIndex(n_real=3.48), ls.ConstantIndex(n_real=1.44)
    if dimension == 2:
        def rect(cx, sy):
            return Structure(geometry=Prism(profile=Rectangle(center_nm=(cx, 0), size_nm=(2000, sy)), z_min_nm=-110,
                                            z_max_nm=110), material=si)
        return DeviceProblem(
            dimension=2, background=sio2, structures=[rect(-1000, 500), rect(1000, 700)],
            domain_size_nm=(2000, 2400, 0), wavelengths=[1500.0, 1600.0],
            ports=[Port(name="o1", center_nm=(-800, 0, 0), size_nm=(0, 2000, 1), direction="+"),
                   Port(name="o2", center_nm=(800, 0, 0), size_nm=(0, 2000, 1), direction="-")],
            options={"fdtd": {"spacing_nm": 25.0, "polarization": "te", "precision": "double", "run_time_fs": 30.0}})
    return DeviceProblem(
        structures=[Structure(geometry=Box(center_nm=(-600, 0, 0), size_nm=(1200, 500, 220)), material=si),
                    Structure(geometry=Box(center_nm=(600, 0, 0), size_nm=(1200, 700, 220)), material=si)],
        background=sio2, domain_size_nm=(1200, 1600, 1200), wavelengths=[1500.0, 1600.0],
        ports=[Port(name="o1", center_nm=(-600, 0, 0), size_nm=(0, 1600, 1200), direction="+"),
               Port(name="o2", center_nm=(600, 0, 0), size_nm=(0, 1600, 1200), direction="-")],
        options={"fdtd": {"spacing_nm": 40.0, "run_time_fs": 20.0}})


def diff_device_problem(dimension: int = 3):
    """The width step of ``device_problem`` meshed subpixel in float64: the problem of the differentiable
    solve's fixtures, whose runs and S lightsmith's driver makes alike."""
    p = device_problem(dimension)
    extra = {"mesh_refinement": "subpixel", "precision": "double"}
    if dimension == 2:
        extra["run_time_fs"] = 90.0  # the pulse through the step to the far port
    return p.model_copy(update={"options": {"fdtd": {**p.options["fdtd"], **extra}}})
