"""Failure paths of the CUDA engine that need a GPU, made without faulting it.

The fused pass bounds every wait on its copy ring by a clock budget; a CTA that runs out records the engine's
status word, waits (bounded) for its own copies still in flight and returns, and ``Engine.check_status``
raises. Here a negative budget makes every wait one on a barrier that nothing completes (a flag nothing sets),
for 10^5 cycles, while every copy the pass issued still completes and is drained: the status must be
reported, stay set until cleared, and the GPU must go on answering (a fresh engine on the same plan matches the
oracle afterwards).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_copy_wait_timeout_is_reported_and_the_gpu_still_answers(golden):
    from lightsmith_b200 import _abi
    from lightsmith_b200.engine import Engine
    from oracle.engine import OracleEngine

    plan = golden("engine_yee_cpml_dipole")["plan"]
    eng = Engine.from_plan(plan, precision="single")
    assert eng.fused and eng.uses_tma
    eng.check_status()
    eng.set_wait_budget(-100000)  # every wait runs out after 1e5 cycles (about 50 us)
    eng.chunk(1)
    with pytest.raises(_abi.LsfdtdError, match="gave up waiting"):
        eng.check_status()
    with pytest.raises(_abi.LsfdtdError):  # the word stays set until cleared
        eng.check_status()
    eng.clear_status()
    eng.check_status()
    eng.close()

    # the context is intact: a new engine with the default budget steps the same plan as the oracle does
    eng = Engine.from_plan(plan, precision="double")
    ref = OracleEngine(plan)
    for _ in range(3):
        eng.chunk(1, use_graph=True)
        ref.chunk()
    eng.check_status()
    err = float(np.abs(eng.E.cpu().numpy() - ref.E).max() / np.abs(ref.E).max())
    eng.close()
    assert err < 1e-9
