"""z-slab decomposition on one GPU: a single rank exchanging halos with itself (periodic wrap) runs the
direct and adjoint loops on a slab extended by H = 2R halo planes; its interior must equal the
single-domain periodic run (the same arithmetic per point, so to rounding level or exactly)."""
import numpy as np
import pytest

from public_b200 import cases
from public_b200.cruna import Cruna, CrunaError, Settings
from public_b200.slabs import ZSlabs

pytestmark = pytest.mark.gpu


def _tgv():
    s, q = cases.taylor_green(n=16, seed=2)
    # a longer periodic box in z: (16, 16, 24) points, same dx
    q = np.asfortranarray(np.concatenate([q, q[:, :, :8]], axis=2))
    s = dict(s, n=(16, 16, 24), x1=(s["x1"][0], s["x1"][1], s["x1"][2] * 1.5), mu0=0.02, ai_freq=(1, 1, 1))
    return s, q


@pytest.mark.parametrize("generic", [False, True])
def test_self_exchanging_slab_matches_single_domain(generic):
    s, q = _tgv()
    sl = ZSlabs(s["n"], halo=8)
    with Cruna(Settings.from_dict(s)) as c:
        c.force_generic(generic)
        ref, Q = c.calc_direct(q, 3, store=True)
        qs0 = np.asfortranarray(0.01 * (q - q.mean(axis=(0, 1, 2))))
        aref = c.calc_adjoint(qs0, Q)
    with Cruna(Settings.from_dict(sl.local_settings(s))) as c:
        c.force_generic(generic)
        sl.attach(c)
        got = c.calc_direct(sl.local_state(q), 3)
        adj = c.calc_adjoint(sl.local_state(qs0), [sl.local_state(x) for x in Q])
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(sl.interior(got) - ref)) <= 1e-13 * scale
    assert np.max(np.abs(sl.interior(adj) - aref)) <= 1e-13 * np.max(np.abs(aref))


def test_slab_mode_rejects_gradients():
    s, q = _tgv()
    sl = ZSlabs(s["n"], halo=8)
    with Cruna(Settings.from_dict(sl.local_settings(s))) as c:
        sl.attach(c)
        with pytest.raises(CrunaError) as e:
            c.gradient(sl.local_state(q), 2, 2, c.objective("kinetic_energy"))
        assert e.value.code == -5
