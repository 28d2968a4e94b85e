"""GPU parity at the configurations' own sizes (the benchmark's workload and the mixing layer's
scheme set), against the oracle's C + OpenMP restatement (oracle/cruna_cpu.c, equal to the numpy
oracle to rounding) or the numpy oracle itself.

* Taylor-Green 256^3 FP64, o8 differences and the o10 explicit filter in both loops -- exactly the
  step pair bench.py times (a direct RK4 step + filters, then a continuous-adjoint RK4 step + filters
  on the new direct state): 3 pairs, 1e-12 relative L2 per conservative variable.
* 2-D isentropic vortex 256^2: 100 steps at 1e-12 (the 1000-step run is in test_gpu_vortex_config).
* Mixing layer 128 x 96 x 64 with the full mixing-layer scheme set (o8 x/z, o6 compact y derivative
  with one-sided boundary rows, o10 open y filter, type-201 characteristic rows at both y ends, a
  20-point sponge): 5 direct and 3 adjoint steps against the numpy oracle at 1e-12.  96 points along
  y make the compact y solve run its long-line code path with several chunks in flight.
"""
import numpy as np
import pytest

from oracle import cpu_twin
from oracle import cruna_oracle as O
from public_b200 import cases
from public_b200.cruna import Cruna, Settings

pytestmark = pytest.mark.gpu

CFG_FIELDS = {f.name for f in O.dataclasses.fields(O.Config)}


def rel_l2_state(a, b):
    """Relative L2 per conservative variable; momentum components are measured against
    max(their own norm, |rho| * c), the sound-speed scale, so a component that is small by symmetry
    is not measured against its own tiny norm."""
    rho, p = b[..., 0], b[..., 4]
    c = float(np.sqrt(1.4 * np.mean(np.abs(p)) / np.mean(np.abs(rho))))
    out = []
    for v in range(5):
        nb = np.linalg.norm(b[..., v].ravel())
        if v in (1, 2, 3):
            nb = max(nb, np.linalg.norm(rho.ravel()) * c)
        out.append(float(np.linalg.norm((a[..., v] - b[..., v]).ravel()) / nb))
    return out


def rel_l2_vars(a, b):
    return [float(np.linalg.norm((a[..., v] - b[..., v]).ravel()) / np.linalg.norm(b[..., v].ravel()))
            for v in range(b.shape[-1])]


def test_taylor_green_256_bench_step_pairs_match_cpu_restatement():
    import torch

    n = 256
    s, q0 = cases.taylor_green(n=n, seed=0)
    s["ai_freq"] = (1, 1, 1)
    assert cpu_twin.supports(s)
    qs0 = cases.smooth_random_state((n, n, n), seed=5, p0=0.0, rho0=0.0, amp=1e-3)
    q_ref = np.array(q0, order="F", copy=True)
    qs_ref = np.array(qs0, order="F", copy=True)
    cpu_twin.run(s, q_ref, qs_ref, 3)
    dev = torch.device("cuda", 0)
    q = torch.from_numpy(np.ascontiguousarray(q0.ravel(order="F"))).to(dev)
    qs = torch.from_numpy(np.ascontiguousarray(qs0.ravel(order="F"))).to(dev)
    torch.cuda.synchronize()
    with Cruna(Settings.from_dict(s)) as c:
        assert c.rhs_path == "fused"
        for nt in range(3):
            c.run_direct_dev(q.data_ptr(), nt, 1)
            c.run_adjoint_dev(qs.data_ptr(), q.data_ptr(), None, nt + 1, 1)
        c.sync()
    got_q = q.cpu().numpy().reshape(q0.shape, order="F")
    got_qs = qs.cpu().numpy().reshape(q0.shape, order="F")
    eq, eqs = rel_l2_state(got_q, q_ref), rel_l2_vars(got_qs, qs_ref)
    assert max(eq) < 1e-12, eq
    assert max(eqs) < 1e-12, eqs


def test_vortex_256_100_steps_at_1e12():
    s, q0 = cases.isentropic_vortex(n=256)
    assert cpu_twin.supports(s)
    ref = np.asfortranarray(q0.copy())
    cpu_twin.run(s, ref, None, 100)
    with Cruna(Settings.from_dict(s)) as c:
        got = c.calc_direct(q0, 100)
    errs = [O.rel_l2(got[..., v], ref[..., v]) for v in (0, 1, 2, 4)]
    assert max(errs) < 1e-12, errs


def test_mixing_layer_128x96x64_direct_and_adjoint_match_oracle():
    n = (128, 96, 64)
    s, q0 = cases.mixing_layer(n=n)
    S = O.Solver(O.Config(**{k: v for k, v in s.items() if k in CFG_FIELDS}), qref=q0.copy())
    q5, Q = S.calc_direct(q0, 5, store=True)
    qs0 = cases.smooth_random_state(n, seed=3, p0=0.0, rho0=0.0, amp=1e-2)
    qs_ref, _ = S.calc_adjoint(qs0, Q[2:])
    with Cruna(Settings.from_dict(s), qref=q0) as c:
        assert c.rhs_path == "generic"
        got = c.calc_direct(q0, 5)
        got_qs = c.calc_adjoint(qs0, Q[2:])
    eq, eqs = rel_l2_state(got, q5), rel_l2_vars(got_qs, qs_ref)
    assert max(eq) < 1e-12, eq
    assert max(eqs) < 1e-12, eqs


def test_mixing_layer_100_step_pairs_match_cpu_restatement():
    """Longer horizon on the mixing layer's scheme set: 100 (direct step + filters, continuous-adjoint
    step + filters) pairs on 64 x 48 x 32 against the C restatement, which covers the compact y
    derivatives, the open y filter, the type-201 rows and the sponge.  The reference's continuous adjoint
    grows here (about 3x per 100 steps at this point of the horizon, 7x later: the adjoint of the
    unstable shear layer, with the sponge off in the adjoint as in the reference), so the adjoint is
    compared at 1e-10 and the direct state at 1e-12."""
    import torch

    n = (64, 48, 32)
    s, q0 = cases.mixing_layer(n=n)
    assert cpu_twin.supports(s)
    qs0 = cases.smooth_random_state(n, seed=3, p0=0.0, rho0=0.0, amp=1e-3)
    q_ref = np.array(q0, order="F", copy=True)
    qs_ref = np.array(qs0, order="F", copy=True)
    cpu_twin.run(s, q_ref, qs_ref, 100, qref=q0)
    dev = torch.device("cuda", 0)
    q = torch.from_numpy(np.ascontiguousarray(q0.ravel(order="F"))).to(dev)
    qs = torch.from_numpy(np.ascontiguousarray(qs0.ravel(order="F"))).to(dev)
    torch.cuda.synchronize()
    with Cruna(Settings.from_dict(s), qref=q0) as c:
        for nt in range(100):
            c.run_direct_dev(q.data_ptr(), nt, 1)
            c.run_adjoint_dev(qs.data_ptr(), q.data_ptr(), None, nt + 1, 1)
        c.sync()
    got_q = q.cpu().numpy().reshape(q0.shape, order="F")
    got_qs = qs.cpu().numpy().reshape(q0.shape, order="F")
    eq, eqs = rel_l2_state(got_q, q_ref), rel_l2_vars(got_qs, qs_ref)
    assert max(eq) < 1e-12, eq
    assert max(eqs) < 1e-10, eqs
