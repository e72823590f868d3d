"""CPU oracle of lightsmith's FDTD path: TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import this package, and
only as the checker; the product path (``lightsmith_b200``) never calls it. ``engine`` restates the time step,
``post`` the scattering cross sections.
"""
