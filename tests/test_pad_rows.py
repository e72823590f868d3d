"""``plan.pad_rows`` on the host: flat indices moved to the wider rows, 1/eps frozen (zero) from the last
plane lightsmith steps on, monitors of a source's own arrays left alone, and plans it must not touch kept."""

import numpy as np

from lightsmith_b200.plan import DipoleSource, PMLSpec, _remap_flat, make_plan, pad_rows


def _plan(shape=(6, 5, 7)):
    rng = np.random.default_rng(0)
    inv = 1.0 / rng.uniform(1, 4, size=shape)
    N = int(np.prod(shape))
    dip = DipoleSource(np.array([N + 2 * 35 + 3, 10]), np.array([0.5, 0.5]), np.zeros(50))

    class M:
        omega = np.array([0.1])
        e_idx = np.array([0, N + 17, 2 * N + N - 1])
        h_idx1 = np.array([1, 2, 3])
        h_idx2 = np.array([4, 5, 6])
        energy = 0
        source = None

    return make_plan(shape=shape, dx=10.0, dt=5.0, single=False, inv_eps=inv, groups=[],
                     pml=PMLSpec(cells=((2, 2),) * 3), sources=[dip], monitors=[M()], dft_stride=5), N


def test_pad_rows_moves_every_flat_index_and_freezes_the_new_planes():
    plan, N = _plan()
    p = pad_rows(plan)
    assert p["shape"] == (6, 5, 8) and p["pad_z"] == 1
    # a flat index (c, x, y, z) -> the same (c, x, y, z) on rows of 8
    for f in (0, 17, N + 36, 2 * N + N - 1):
        c, rest = divmod(f, N)
        x, r = divmod(rest, 5 * 7)
        y, z = divmod(r, 7)
        assert _remap_flat([f], (6, 5, 7), 8)[0] == c * 6 * 5 * 8 + (x * 5 + y) * 8 + z
    assert np.array_equal(p["monitors"][0]["e_idx"], _remap_flat(plan["monitors"][0]["e_idx"], (6, 5, 7), 8))
    assert np.array_equal(p["monitors"][0]["h_idx2"], _remap_flat(plan["monitors"][0]["h_idx2"], (6, 5, 7), 8))
    assert np.array_equal(p["sources"][0].idx, _remap_flat(plan["sources"][0].idx, (6, 5, 7), 8))
    inv0, inv1 = np.asarray(plan["inv_eps"]), np.asarray(p["inv_eps"])
    assert np.array_equal(inv1[..., :6], inv0[..., :6]) and not np.any(inv1[..., 6:])
    assert pad_rows(p) is p  # padded once


def test_pad_rows_keeps_plans_it_must_not_change():
    plan, _ = _plan((6, 5, 8))
    assert pad_rows(plan) is plan  # rows already a multiple of 4
    plan, _ = _plan()
    assert pad_rows({**plan, "periodic": (True, True, False)})["shape"] == plan["shape"]
