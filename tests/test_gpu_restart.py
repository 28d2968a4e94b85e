"""GPU tests of cruna_run_hpc, the direct main loop with snapshots and restart
(src/main/cruna_hpc.f90:99-299): a run stopped by its step budget in one process and continued from
restartfile.bin in a second process ends bit-identical to the same run done in one go, and every
snapshot written on the way holds the state of its step."""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from public_b200 import cases, cruna
from public_b200.cruna import Cruna, Settings

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = textwrap.dedent("""
    import sys
    import numpy as np
    sys.path.insert(0, {root!r})
    from public_b200 import cases
    from public_b200.cruna import Cruna, Settings
    s, q0 = cases.taylor_green(n=16, seed=2)
    s["mu0"] = 0.02
    s["di_freq"] = (2, 3, 1)
    with Cruna(Settings.from_dict(s)) as c:
        q, stopped, pos = c.run_hpc(q0, {wdir!r}, steps={steps}, subsets={subsets}, dsfreq={dsfreq},
                                    restart={restart}, max_steps={max_steps})
    np.save({out!r}, q)
    print("STOPPED" if stopped else "DONE", pos[0], pos[1])
""")


def run_process(wdir, out, steps, subsets, dsfreq, restart, max_steps):
    code = SCRIPT.format(root=ROOT, wdir=str(wdir), out=str(out), steps=steps, subsets=subsets, dsfreq=dsfreq,
                         restart=restart, max_steps=max_steps)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    return r.stdout.split()


def settings():
    s, q0 = cases.taylor_green(n=16, seed=2)
    s["mu0"] = 0.02
    s["di_freq"] = (2, 3, 1)           # filters on the step index: a restart must keep the phase
    return s, q0


@pytest.mark.parametrize("subsets,steps,stop", [(1, 12, 5), (2, 6, 6), (2, 6, 9)])
def test_run_split_across_two_processes_is_bit_identical(tmp_path, subsets, steps, stop):
    s, q0 = settings()
    (tmp_path / "one").mkdir()
    with Cruna(Settings.from_dict(s)) as c:
        full, stopped, pos = c.run_hpc(q0, str(tmp_path / "one"), steps=steps, subsets=subsets, dsfreq=4)
        assert not stopped and pos == (subsets, steps)
        plain = c.calc_direct(q0, steps) if subsets == 1 else None
    if plain is not None:
        assert np.array_equal(full, plain)
    wdir = tmp_path / "split"
    wdir.mkdir()
    first = run_process(wdir, tmp_path / "a.npy", steps, subsets, 4, False, stop)
    assert first[0] == "STOPPED" and cruna.read_restart(str(wdir)) == (int(first[1]), int(first[2]))
    if subsets == 2 and stop == 9:
        # stopped inside subset 2 at step 3: nt0 = 4 there, and subset 2 is the last one, so the
        # reference's quirk (nt0 applies to every later subset) does not arise
        assert (int(first[1]), int(first[2])) == (2, 3)
    second = run_process(wdir, tmp_path / "b.npy", steps, subsets, 4, True, 0)
    assert second[0] == "DONE"
    got = np.load(tmp_path / "b.npy")
    assert np.array_equal(got.view(np.uint64), full.view(np.uint64))
    # the snapshot of the last step and the one of the stop point hold those states
    last, _ = cruna.read_snapshot(cruna.io_fname(str(wdir), "data_direct_snapshot", ns=subsets, nt=steps))
    assert np.array_equal(last, full)
    stopq, params = cruna.read_snapshot(cruna.io_fname(str(wdir), "data_direct_snapshot", ns=int(first[1]),
                                                       nt=int(first[2])))
    assert np.array_equal(stopq, np.load(tmp_path / "a.npy"))
    assert f"time.nt = {first[2]}" in params


def test_periodic_snapshots_hold_the_states_of_their_steps(tmp_path):
    s, q0 = settings()
    with Cruna(Settings.from_dict(s)) as c:
        c.run_hpc(q0, str(tmp_path), steps=8, subsets=1, dsfreq=4)
        ref = c.calc_direct(q0, 8, store=True)[1]
    for nt in (0, 4, 8):
        q, _ = cruna.read_snapshot(cruna.io_fname(str(tmp_path), "data_direct_snapshot", ns=1, nt=nt))
        assert np.array_equal(q, ref[nt]), nt
    assert cruna.read_restart(str(tmp_path)) == (1, 8)
