"""Batched form: many independent domains advanced by one graph launch per step.

    b = Batch(device=0)
    for d in domains:            # hicar_b200.Domain objects after adv_init
        b.add(d, dt)
    for _ in range(nsteps):
        b.step()                 # apply_forcing + advect for every member
    b.sync(); d.fetch("qv")

The members keep their own device fields (the C-ABI handles); the batch owns
the member tables, the (member, species, tile) work list and the two CUDA
graphs (one per buffer parity).  See icar_adv_batch_* in include/icar_adv.h.
"""
from __future__ import annotations

import ctypes as C

from . import _lib as L


class BatchError(L.IcarAdvError):
    pass


class Batch:
    def __init__(self, device: int = 0):
        self._lib = L.load()
        h = C.c_void_p()
        self._check(self._lib.icar_adv_batch_create(int(device), C.byref(h)), None)
        self._b = h
        self.device = device
        self.members: list = []

    def _check(self, code: int, b) -> None:
        if code != L.OK:
            msg = self._lib.icar_adv_batch_last_error(b)
            raise BatchError(code, msg.decode() if msg else "")

    def add(self, domain, dt_seconds: float) -> None:
        domain._flush()
        self._check(self._lib.icar_adv_batch_add(self._b, domain.handle, C.c_double(dt_seconds)), self._b)
        self.members.append(domain)

    def remove(self, domain) -> None:
        self._check(self._lib.icar_adv_batch_remove(self._b, domain.handle), self._b)
        self.members.remove(domain)

    def set_dt(self, domain, dt_seconds: float) -> None:
        self._check(self._lib.icar_adv_batch_set_dt(self._b, domain.handle, C.c_double(dt_seconds)), self._b)

    def set_tile_shape(self, shape: int) -> None:
        self._check(self._lib.icar_adv_batch_set_tile_shape(self._b, int(shape)), self._b)

    def set_path(self, path: int) -> None:
        """0: donor-cell kernel + fused correction (default); 2: single-pass
        kernel, bit-exact; 3: single-pass kernel, fast arithmetic."""
        self._check(self._lib.icar_adv_batch_set_path(self._b, int(path)), self._b)

    def set_species_group(self, group: int) -> None:
        self._check(self._lib.icar_adv_batch_set_species_group(self._b, int(group)), self._b)

    def set_stream(self, cuda_stream: int) -> None:
        self._check(self._lib.icar_adv_batch_set_stream(self._b, C.c_void_p(cuda_stream)), self._b)

    def step(self) -> None:
        self._check(self._lib.icar_adv_batch_step(self._b), self._b)

    def sync(self) -> None:
        self._check(self._lib.icar_adv_batch_sync(self._b), self._b)

    def wait(self, timeout_s: float) -> bool:
        """Bounded wait for the queued steps: True when they are done, False
        when timeout_s passed first (the steps stay queued)."""
        code = self._lib.icar_adv_batch_sync_timeout(self._b, C.c_double(timeout_s))
        if code == L.TIMEOUT:
            return False
        self._check(code, self._b)
        return True

    def profile(self, enable: bool = True) -> None:
        self._check(self._lib.icar_adv_batch_profile(self._b, int(enable)), self._b)

    def profile_read(self) -> dict:
        ms, steps, kps, cs = C.c_double(), C.c_int64(), C.c_int64(), C.c_int64()
        self._check(self._lib.icar_adv_batch_profile_read(self._b, C.byref(ms), C.byref(steps), C.byref(kps),
                                                          C.byref(cs)), self._b)
        return {"ms": ms.value, "steps": steps.value, "kernels_per_step": kps.value,
                "cell_species_per_step": cs.value}

    def close(self) -> None:
        if getattr(self, "_b", None) is not None:
            self._lib.icar_adv_batch_destroy(self._b)
            self._b = None
            self.members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
