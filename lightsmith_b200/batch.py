"""Batched Bloch-periodic sweeps: many independent oblique runs advanced by one persistent kernel.

lightsmith solves an oblique-incidence periodic problem one fixed-k_par run at a time
(``backends/_fdtd/periodic.py:503-518``, each ``_run_oblique``, ``periodic.py:426-459``). ``BlochBatch``
takes the engines of such runs, built as usual (``Engine.from_plan`` of each run's plan), and advances all of
them together: one launch of ``k_bloch_batch`` per call (replayed as a CUDA graph), whose CTAs take whole runs,
longest first, and step each through its steps with its monitors sampled every ``dft_stride`` steps. The
engines keep their device state and step counters, so their fields and DFT accumulators (``Engine.results``)
are read as after their own chunks.
"""

from __future__ import annotations

import ctypes as C

from . import _abi


class BlochBatch:
    """The runs of ``engines`` (complex fields, periodic x and y, CPML along z, one Bloch column source),
    each to run until its step count reaches ``last`` (an int for all, or one per engine). ``cluster_ctas``:
    CTAs per run (1 to 16: a thread-block cluster; more: a group meeting at barriers in global memory, in a
    cooperative launch; 0: groups of half the CTAs resident at once); ``max_clusters``: runs in flight (0: as
    many as fit)."""

    def __init__(self, engines, last, cluster_ctas: int = 0, max_clusters: int = 0):
        import torch

        self.engines = list(engines)
        if not self.engines:
            raise ValueError("a batch needs at least one engine")
        n = len(self.engines)
        last = [int(last)] * n if isinstance(last, int) else [int(v) for v in last]
        if len(last) != n:
            raise ValueError("one last step per engine")
        self.dev = self.engines[0].dev
        if any(e.dev != self.dev for e in self.engines):
            raise ValueError("the engines of a batch share one device")
        L = _abi.lib()
        torch.cuda.synchronize(self.dev)  # the engines' set-up (zeroed fields, copied tables) is complete
        h = C.c_void_p()
        arr = (C.c_void_p * n)(*[e._h.value for e in self.engines])
        _abi.check(L.lsfdtd_batch_create_shaped(arr, n, (C.c_int64 * n)(*last), int(cluster_ctas), int(max_clusters),
                                                C.byref(h)), "lsfdtd_batch_create_shaped")
        self._h = h
        nbytes = C.c_size_t()
        _abi.check(L.lsfdtd_batch_scratch_bytes(h, C.byref(nbytes)), "lsfdtd_batch_scratch_bytes")
        self.scratch = torch.empty(max(int(nbytes.value), 256), dtype=torch.uint8, device=self.dev)
        _abi.check(L.lsfdtd_batch_set_scratch(h, self.scratch.data_ptr(), int(nbytes.value)),
                   "lsfdtd_batch_set_scratch")
        self.stream = torch.cuda.Stream(device=self.dev)
        self.last = last

    @property
    def ctas(self) -> int:
        return int(_abi.lib().lsfdtd_batch_ctas(self._h))

    def run(self, steps: int, launches: int = 1, use_graph: bool = True) -> None:
        """``launches`` launches in which every run advances ``steps`` steps (or to its last step)."""
        import torch

        cur = torch.cuda.current_stream(self.dev)
        self.stream.wait_stream(cur)
        _abi.check(_abi.lib().lsfdtd_batch_run(self._h, int(steps), int(launches), int(bool(use_graph)),
                                               self.stream.cuda_stream), "lsfdtd_batch_run")
        cur.wait_stream(self.stream)

    def run_to_end(self, steps_per_launch: int = 256, use_graph: bool = True) -> int:
        """Launches until every run has reached its last step; returns the launch count."""
        todo = max(last - e.n_host for e, last in zip(self.engines, self.last))
        launches = -(-todo // steps_per_launch) if todo > 0 else 0
        if launches:
            self.run(steps_per_launch, launches, use_graph)
        return launches

    def diverged(self) -> list[int]:
        """Indices of the runs whose fields turned non-finite (each retired after that step; its device step
        counter ``Engine.n`` holds the steps it ran). Synchronises."""
        import torch

        torch.cuda.synchronize(self.dev)
        out = []
        for i, e in enumerate(self.engines):
            st = C.c_int32()
            _abi.lib().lsfdtd_engine_status(e._h, e.stream.cuda_stream, C.byref(st))
            if st.value == 2:
                out.append(i)
        return out

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            import torch

            torch.cuda.synchronize(self.dev)
            _abi.lib().lsfdtd_batch_destroy(h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 (interpreter shutdown)
            pass
