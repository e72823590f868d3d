"""The allocation-free DFT sample against the engine's own sample.

``lsfdtd_dft_sample_noalloc`` serves callers that cannot allocate device memory (a host runtime that only
lends the library the buffers it owns, or a process whose device memory all comes from one external pool):
the scratch of its energy reduction is a static device array inside the library. Here it samples the same
monitor as an engine does through ``lsfdtd_engine_sample`` (which reduces into caller-provided scratch), two
samples in a row, and the accumulators and the energy must agree.
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # the same arithmetic in the same order: agreement to the last bits


def _desc(mon, acc_e, acc_h, dev_arrays, E, H):
    from lightsmith_b200 import _abi

    omega, e_idx, h1, h2 = dev_arrays
    d = _abi.MonitorDesc()
    d.n_freq = len(mon["omega"])
    d.omega = omega.data_ptr()
    d.n_e, d.e_idx = len(mon["e_idx"]), e_idx.data_ptr()
    d.n_h, d.h_idx1, d.h_idx2 = len(mon["h_idx1"]), h1.data_ptr(), h2.data_ptr()
    d.acc_e, d.acc_h = acc_e.data_ptr(), acc_h.data_ptr()
    d.energy, d.space = int(mon["energy"]), 0
    d.E_src, d.H_src = E.data_ptr(), H.data_ptr()
    return d


def test_noalloc_sample_matches_engine_sample_twice(golden):
    import torch

    from lightsmith_b200 import _abi
    from lightsmith_b200.engine import Engine

    L = _abi.lib()
    plan = golden("engine_yee_cpml_dipole")["plan"]
    eng = Engine.from_plan(plan, precision="single", fused=False)
    mon = plan["monitors"][0]
    assert mon["energy"] == 1 and mon["h_idx1"] is not None
    dev = eng.dev
    nf = len(mon["omega"])
    acc_e = torch.zeros((nf, len(mon["e_idx"])), dtype=torch.complex128, device=dev)
    acc_h = torch.zeros((nf, len(mon["h_idx1"])), dtype=torch.complex128, device=dev)
    energy = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    arrays = (torch.as_tensor(mon["omega"], dtype=torch.float64, device=dev),
              *(torch.as_tensor(mon[k], dtype=torch.int64, device=dev) for k in ("e_idx", "h_idx1", "h_idx2")))
    for call in range(2):
        eng.step(plan["stride"] * (call + 2))  # advance (the pulse grows), then sample both ways
        eng.sample()
        d = _desc(mon, acc_e, acc_h, arrays, eng.E, eng.H)
        rc = L.lsfdtd_dft_sample_noalloc(C.byref(d), _abi.F32, 0, eng.n.data_ptr(), eng.dt, energy.data_ptr(),
                                         eng.stream.cuda_stream)
        _abi.check(rc, "lsfdtd_dft_sample_noalloc")
        torch.cuda.synchronize(dev)
        ref_e, ref_h = eng.results(0)
        assert np.abs(ref_e).max() > 0
        np.testing.assert_allclose(acc_e.cpu().numpy(), ref_e, rtol=RTOL, atol=0)
        np.testing.assert_allclose(acc_h.cpu().numpy(), ref_h, rtol=RTOL, atol=0)
        np.testing.assert_allclose(energy.cpu().numpy()[0], eng.energy.cpu().numpy()[0], rtol=RTOL, atol=0)

    # after those calls, more calls change neither the device's free memory nor torch's reserved pool
    torch.cuda.synchronize(dev)
    free0, reserved0 = torch.cuda.mem_get_info(dev)[0], torch.cuda.memory_reserved(dev)
    for _ in range(4):
        rc = L.lsfdtd_dft_sample_noalloc(C.byref(d), _abi.F32, 0, eng.n.data_ptr(), eng.dt, energy.data_ptr(),
                                         eng.stream.cuda_stream)
        _abi.check(rc, "lsfdtd_dft_sample_noalloc")
    torch.cuda.synchronize(dev)
    assert torch.cuda.mem_get_info(dev)[0] == free0
    assert torch.cuda.memory_reserved(dev) == reserved0
    eng.close()


def test_noalloc_sample_rejects_monitors_beyond_its_scratch():
    import torch

    from lightsmith_b200 import _abi

    L = _abi.lib()
    dev = torch.device("cuda", 0)
    small = torch.zeros(4, dtype=torch.int64, device=dev)
    acc = torch.zeros(4, dtype=torch.complex128, device=dev)
    field = torch.zeros(8, dtype=torch.float32, device=dev)
    omega = torch.ones(1, dtype=torch.float64, device=dev)
    d = _abi.MonitorDesc()
    d.n_freq, d.omega = 1, omega.data_ptr()
    d.n_e, d.e_idx = 8192 * 256 + 1, small.data_ptr()  # one block past the static scratch; nothing is launched
    d.acc_e, d.E_src = acc.data_ptr(), field.data_ptr()
    d.energy, d.space = 0, 0
    rc = L.lsfdtd_dft_sample_noalloc(C.byref(d), _abi.F32, 0, small.data_ptr(), 1.0, None, None)
    assert rc == _abi.EINVAL
    assert b"exceed the static scratch" in L.lsfdtd_last_error()
