"""The 2-D isentropic vortex configuration at full size: 256 x 256 x 1 points, o8 differences, o10
filter every step, RK4 at CFL 0.5, 1000 steps, FP64 -- the GPU against the C + OpenMP restatement of
the oracle (oracle/cruna_cpu.c, itself equal to the numpy oracle to rounding), on the four non-trivial
conservative fields (rho w stays zero).  Tolerance 1e-11 relative L2 per field: the two evaluate the
same sums in different orders, and 1000 steps accumulate the per-step rounding differences."""
import numpy as np
import pytest

from oracle import cpu_twin
from oracle import cruna_oracle as O
from public_b200 import cases
from public_b200.cruna import Cruna, Settings

pytestmark = pytest.mark.gpu


def test_vortex_256_1000_steps_against_the_cpu_restatement():
    s, q0 = cases.isentropic_vortex(n=256)
    assert cpu_twin.supports(s)
    ref = np.asfortranarray(q0.copy())
    cpu_twin.run(s, ref, None, 1000)
    with Cruna(Settings.from_dict(s)) as c:
        got = c.calc_direct(q0, 1000)
    errs = [O.rel_l2(got[..., v], ref[..., v]) for v in (0, 1, 2, 4)]
    assert max(errs) < 1e-11, errs
    assert np.max(np.abs(got[..., 3])) == 0.0
