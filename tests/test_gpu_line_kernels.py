"""Line operators on lines long enough for the library's fast kernels (compile-time radius stencils;
the fused explicit-part + dgttrs kernel of compact operators along y and z): every derivative and
filter scheme in every direction against the oracle, and the mixing layer's RHS (compact y
derivatives, open filter, characteristic boundaries, sponge) on a grid where those kernels run.
Tolerances as in the operator parity tests: 1e-13 relative to the field maximum, 1e-12 for compact
cores; 1e-12 relative L2 per variable for the RHS."""
import numpy as np
import pytest

from oracle import cruna_oracle as O
from public_b200 import cases
from public_b200.cruna import Cruna, Settings

pytestmark = pytest.mark.gpu

N = (40, 36, 34)          # longer than 2 * (closure rows + radius) + 1 for every scheme
COMPACT = {"o4_i_c_p_pade", "o4_i_c_o_pade", "o6_i_c_p", "o6_i_c_o"}


def rel_max(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("scheme", [s for s in O.DIFF_SCHEMES if s != "empty"])
def test_diff_long_lines(scheme):
    q = cases.smooth_random_state(N, seed=11)
    x1 = (1.0, 1.3, 0.9)
    cfg = O.Config(n=N, diff=(scheme,) * 3, x1=x1)
    with Cruna(Settings(n=N, diff=(scheme,) * 3, x1=x1)) as c:
        dx = c.dx
        for d in range(3):
            got = getattr(c, f"Dx{d + 1}")(q[..., 1:4], h=dx[d])
            for v in range(3):
                ref = O.Dx(cfg, d, np.asfortranarray(q[..., 1 + v]), dx[d])
                tol = 1e-12 if scheme in COMPACT else 1e-13
                assert rel_max(got[..., v], ref) < tol, (scheme, d, v, rel_max(got[..., v], ref))


@pytest.mark.parametrize("scheme", [s for s in O.FILTER_SCHEMES if s != "empty"])
def test_filter_long_lines(scheme):
    q = cases.smooth_random_state(N, seed=12)
    cfg = O.Config(n=N, filt=(scheme,) * 3, alpha=0.3)
    with Cruna(Settings(n=N, filt=(scheme,) * 3, alpha=0.3)) as c:
        for d in range(3):
            got = getattr(c, f"filter_i{d + 1}")(q)
            ref = O.filter_dir(cfg, d, np.asfortranarray(q))
            assert rel_max(got, ref) < 1e-12, (scheme, d, rel_max(got, ref))


def test_mixing_layer_rhs_long_lines():
    s, q = cases.mixing_layer(n=(40, 36, 24))
    cfg = O.Config(**{k: v for k, v in s.items() if k in {f.name for f in O.dataclasses.fields(O.Config)}})
    S = O.Solver(cfg, qref=q.copy())
    rng = np.random.default_rng(3)
    qp = np.asfortranarray(q * (1.0 + 1e-3 * rng.standard_normal(q.shape)))
    ref = S.rhs_direct(qp)
    qs = np.asfortranarray(rng.standard_normal(q.shape))
    refs = S.rhs_adjoint(qs, qp, np.zeros_like(qp))
    with Cruna(Settings.from_dict(s), qref=q) as c:
        got = c.rhs_direct(qp)
        gots = c.rhs_adjoint(qs, qp)
    for v in range(5):
        for a, b in ((got, ref), (gots, refs)):
            nb = np.linalg.norm(b[..., v])
            if nb > 0:
                assert np.linalg.norm(a[..., v] - b[..., v]) / nb < 1e-12, v
