"""GPU test of cruna_rhs_direct_noalloc, the allocation-free direct RHS.

That entry point is for callers that cannot allocate device memory where they need an RHS: their
device memory is owned by another allocator (for instance a framework's caching pool) or their time
loop must keep the footprint it planned at start-up, so they cannot create a context (cruna_init
allocates).  It uses a static device array as its scratch.  This test calls it through the C ABI on
device buffers the test itself provides, twice in a row on different grids, and compares each result
with the context-based cruna_rhs_direct_dev on the same input (same kernels, so the FP64 tolerance of
the parity suite, 1e-12, is ample).  The file name makes pytest collect it after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from public_b200 import cases
from public_b200.cruna import Cruna, Settings

pytestmark = pytest.mark.gpu


def _run_both(settings: dict, q: np.ndarray):
    import torch

    st = Settings.from_dict(settings)
    n = int(np.prod(st.n))
    dev = torch.device("cuda", 0)
    qd = torch.from_numpy(np.ascontiguousarray(q.ravel(order="F"))).to(dev)
    r_ref = torch.empty_like(qd)
    r_new = torch.full_like(qd, float("nan"))
    with Cruna(st) as c:
        c.rhs_direct_dev(qd.data_ptr(), r_ref.data_ptr())
        c.sync()
        lib = c.lib
        cfg = st.to_struct(lib)
    err = C.create_string_buffer(256)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = lib.cruna_rhs_direct_noalloc(C.byref(cfg), C.c_void_p(qd.data_ptr()), C.c_void_p(r_new.data_ptr()),
                                      C.c_void_p(stream), err, 256)
    assert rc == 0, err.value.decode()
    torch.cuda.synchronize()
    a = r_new.cpu().numpy().reshape(st.n + (5,), order="F")
    b = r_ref.cpu().numpy().reshape(st.n + (5,), order="F")
    assert a.size == 5 * n
    return a, b


def _check(a, b):
    assert np.all(np.isfinite(a))
    for v in range(5):
        scale = max(float(np.max(np.abs(b[..., v]))), 1e-300)
        assert float(np.max(np.abs(a[..., v] - b[..., v]))) <= 1e-12 * scale, v


def test_noalloc_rhs_matches_context_rhs_twice():
    s1, q1 = cases.taylor_green(n=24, seed=4)
    s1["mu0"] = 0.01
    a1, b1 = _run_both(s1, q1)
    _check(a1, b1)
    # second call in a row: another grid and an open explicit scheme, on the same static scratch
    n2 = (20, 18, 16)
    q2 = cases.smooth_random_state(n2, seed=9, p0=1.0, rho0=1.0, amp=0.05)
    s2 = dict(n=n2, diff=("o4_e_c_p", "o4_e_c_o", "o8_e_c_p"), x1=(1.0, 1.1, 0.9), R=1.0, W=1.0, T0=1.0,
              mu0=0.02)
    a2, b2 = _run_both(s2, q2)
    _check(a2, b2)


def test_noalloc_rejects_grids_beyond_its_scratch():
    from public_b200.cruna import load_library

    lib = load_library()
    st = Settings(n=(64, 64, 33), diff=("o4_e_c_p",) * 3)
    cfg = st.to_struct(lib)
    err = C.create_string_buffer(256)
    rc = lib.cruna_rhs_direct_noalloc(C.byref(cfg), C.c_void_p(16), C.c_void_p(16), None, err, 256)
    assert rc == -1 and b"131072" in err.value


def test_noalloc_orders_its_work_on_the_callers_stream():
    """The work is enqueued on the stream the caller passes: q is written on a side stream just before
    the call, only that stream is synchronised, and the result still matches the context RHS."""
    import torch

    s, q = cases.taylor_green(n=16, seed=6)
    s["mu0"] = 0.01
    st = Settings.from_dict(s)
    dev = torch.device("cuda", 0)
    q_host = torch.from_numpy(np.ascontiguousarray(q.ravel(order="F"))).pin_memory()
    qd = torch.from_numpy(np.ascontiguousarray(q.ravel(order="F"))).to(dev)
    r_ref = torch.empty_like(qd)
    with Cruna(st) as c:
        c.rhs_direct_dev(qd.data_ptr(), r_ref.data_ptr())
        c.sync()
        lib = c.lib
        cfg = st.to_struct(lib)
    side = torch.cuda.Stream(device=dev)
    q_side = torch.zeros_like(qd)
    r_new = torch.full_like(qd, float("nan"))
    torch.cuda.synchronize()
    err = C.create_string_buffer(256)
    with torch.cuda.stream(side):
        q_side.copy_(q_host, non_blocking=True)       # q arrives on the side stream only
        rc = lib.cruna_rhs_direct_noalloc(C.byref(cfg), C.c_void_p(q_side.data_ptr()),
                                          C.c_void_p(r_new.data_ptr()), C.c_void_p(side.cuda_stream), err, 256)
    assert rc == 0, err.value.decode()
    side.synchronize()
    a = r_new.cpu().numpy().reshape(st.n + (5,), order="F")
    b = r_ref.cpu().numpy().reshape(st.n + (5,), order="F")
    _check(a, b)
