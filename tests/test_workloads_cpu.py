"""The dispersive-cluster workload's geometry (lightsmith_b200.workloads.cluster_instance), on the CPU."""

import numpy as np


def test_cluster_instance_geometry():
    from lightsmith_b200.workloads import SILVER, cluster_instance

    for seed in (0, 3):
        plan, info = cluster_instance(seed)
        n = plan["shape"][0]
        assert 96 <= n <= 256 and plan["shape"] == (n, n, n)
        sph = info["spheres"]
        assert 3 <= len(sph) <= 12
        for a in range(len(sph)):
            assert 10 <= sph[a][1] <= 40
            for b in range(a):
                assert np.linalg.norm(sph[a][0] - sph[b][0]) >= sph[a][1] + sph[b][1]
        (g,) = plan["groups"]
        assert g["w"] is None and g["media"][0]["eps_inf"] == SILVER.eps_inf and len(g["media"][0]["poles"]) == 3
        cells = n ** 3
        node = np.unique(g["idx"] % cells)
        assert len(g["idx"]) == 3 * len(node)  # every component of a metal node
        inv = np.asarray(plan["inv_eps"])
        assert np.all(inv.reshape(-1)[node] == 1.0)
        box = info["box"]
        pml = plan["pml"]["cells"][0][0]
        for lo, hi in box:
            assert pml + 2 < lo < hi < n - pml - 2
        bsl = tuple(slice(a, b) for a, b in box)
        metal = np.zeros(cells, bool)
        metal[node] = True
        assert not np.any(info["shell"] & metal.reshape(plan["shape"])[bsl])
        assert info["shell"].sum() > 0
        # the dipole's nodes lie outside the design box and inside the flux box
        (dip,) = plan["sources"]
        ijk = np.stack(np.unravel_index(np.asarray(dip.idx) % cells, plan["shape"]), axis=1)
        assert not np.any(np.all((ijk >= [a for a, _ in box]) & (ijk < [b for _, b in box]), axis=1))
        mon = plan["monitors"][0]
        mk = np.stack(np.unravel_index(np.asarray(mon["e_idx"]) % cells, plan["shape"]), axis=1)
        assert np.all(mk.min(axis=0) < ijk.min(axis=0)) and np.all(mk.max(axis=0) > ijk.max(axis=0))
        assert len(mon["omega"]) == 24
