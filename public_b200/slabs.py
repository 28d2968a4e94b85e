"""z-slab decomposition of a periodic grid over ranks (one GPU each), replacing the reference's MPI
pencil transposes (src/parallelism/transpose_mpi_cartesian.f90) for runs over several GPUs.

Each rank's context holds its slab of nz = n3 / world planes extended by H halo planes on both sides
(the library's periodic z scheme then runs unchanged on nz + 2H planes); before every pass that
reads z-neighbours the library calls back (``cruna_set_halo_exchange``) and ``ZSlabs.exchange``
refreshes the halos from the neighbouring slabs: the lowest H interior planes go to the rank below
(its upper halo), the highest H to the rank above (its lower halo), periodically.  With H >= 2R (R
the derivative half-width) the interior planes are exactly the single-domain result.  One rank
exchanges with itself (periodic wrap), which is how the path is exercised on one GPU; several ranks
use torch.distributed point-to-point (NCCL on GPUs, gloo on CPU tensors).
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Tuple

import numpy as np

HALO_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p)


class _RawDevice:
    """A device pointer exposed through __cuda_array_interface__ (zero-copy torch.as_tensor)."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


class ZSlabs:
    def __init__(self, n: Tuple[int, int, int], halo: int, rank: int = 0, world: int = 1):
        n1, n2, n3 = n
        if n3 % world:
            raise ValueError("n3 must be divisible by the number of ranks")
        self.n, self.H, self.rank, self.world = (n1, n2, n3), int(halo), int(rank), int(world)
        self.nz = n3 // world
        if self.nz < self.H:
            raise ValueError("slab thinner than its halo")
        self.local_n = (n1, n2, self.nz + 2 * self.H)
        self.plane = n1 * n2
        self._cb = None

    # ---- set-up ----------------------------------------------------------------------------------
    def local_settings(self, s: Dict) -> Dict:
        """Settings of this rank's extended slab from the global periodic settings (same dx)."""
        x0, x1 = list(s.get("x0", (0.0, 0.0, 0.0))), list(s.get("x1", (1.0, 1.0, 1.0)))
        dz = (x1[2] - x0[2]) / self.n[2]
        z0 = x0[2] + (self.rank * self.nz - self.H) * dz
        x0[2], x1[2] = z0, z0 + self.local_n[2] * dz
        return dict(s, n=self.local_n, x0=tuple(x0), x1=tuple(x1))

    def local_state(self, q_global: np.ndarray) -> np.ndarray:
        """This rank's extended slab (halo planes filled periodically) of a global state (n1,n2,n3,nf)."""
        k = (np.arange(self.local_n[2]) + self.rank * self.nz - self.H) % self.n[2]
        return np.asfortranarray(q_global[:, :, k, :])

    def interior(self, q_local: np.ndarray) -> np.ndarray:
        return q_local[:, :, self.H:self.H + self.nz, ...]

    # ---- exchange --------------------------------------------------------------------------------
    def exchange(self, flat, nfields: int):
        """Refresh the halo planes of `nfields` Fortran-ordered fields stored in the 1-D tensor `flat`."""
        import torch
        H, nz = self.H, self.nz
        v = flat[: nfields * self.local_n[2] * self.plane].view(nfields, nz + 2 * H, self.plane)
        if self.world == 1:
            v[:, :H] = v[:, nz:nz + H]
            v[:, nz + H:] = v[:, H:2 * H]
            return
        import torch.distributed as dist
        below = (self.rank - 1) % self.world
        above = (self.rank + 1) % self.world
        send_lo = v[:, H:2 * H].contiguous()           # becomes the upper halo of the rank below
        send_hi = v[:, nz:nz + H].contiguous()         # becomes the lower halo of the rank above
        recv_lo = torch.empty_like(send_lo)            # from the rank below: its highest planes
        recv_hi = torch.empty_like(send_hi)            # from the rank above: its lowest planes
        # messages between one pair of ranks match in posting order (two ranks: below == above), so
        # every rank sends its high planes first and receives its lower halo first
        ops = [dist.P2POp(dist.isend, send_hi, above), dist.P2POp(dist.isend, send_lo, below),
               dist.P2POp(dist.irecv, recv_lo, below), dist.P2POp(dist.irecv, recv_hi, above)]
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        v[:, :H] = recv_lo
        v[:, nz + H:] = recv_hi

    def callback(self):
        """A C function pointer for cruna_set_halo_exchange (kept alive by this object)."""
        import torch
        count_per_field = self.local_n[0] * self.local_n[1] * self.local_n[2]

        def fn(user, ptr, nfields, stream):
            try:
                t = torch.as_tensor(_RawDevice(ptr, nfields * count_per_field), device="cuda")
                with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
                    self.exchange(t, int(nfields))
                return 0
            except Exception:  # the library turns a non-zero status into CRUNA_ERR_CUDA
                return 1

        self._cb = HALO_FN(fn)
        return self._cb

    def attach(self, solver) -> None:
        """Install the exchange on a public_b200.cruna.Cruna context of this rank's slab."""
        solver.set_halo_exchange(self.callback())
