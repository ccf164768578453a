"""Failure detection as statuses: a box whose forces overflow reports
LIMA_ERR_NUMERIC from the step or the next synchronisation instead of
exiting, and the engine answers afterwards.  Made on the host by the input
(two waters 0.001 nm apart: the physics path's FP32 LJ forces overflow to
inf, the positions to inf and then NaN, which the integrator flags); no GPU
fault is involved, and every index the kernels derive from a position is
clamped.  Reference semantics flags, as the reference does, a critical force
on compound particles only (Engine.cu compoundKernel), so an overflowing
solvent pair is not a status there."""
import numpy as np
import pytest

from quantom_b200 import systems as S

pytestmark = pytest.mark.gpu


def test_overflowing_forces_are_a_numeric_status(gpu):
    E = gpu
    s = S.make_system("tiny_solvent", seed=3)
    s.solvents["pos"][1] = s.solvents["pos"][0] + np.float32(0.001)
    s.solvents["pos_tsub1"][1] = s.solvents["pos"][1]
    p = E.default_params(box_len=s.spec.box_len, cutoff=s.spec.cutoff, dt=s.spec.dt,
                         semantics=E.SEMANTICS_PHYSICS, skin=0.1, switch_on=1.0, nlist_period=10)
    with E.Engine(s, p) as eng:
        with pytest.raises(E.LimaError) as ei:
            eng.step(4)
            eng.synchronize()
        assert ei.value.status == E.ERR_NUMERIC
        # the context still answers: the flags were cleared when reported
        eng.synchronize()
        assert len(eng.solvents()) == s.n_solvents
