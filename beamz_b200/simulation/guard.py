"""Divergence guard of the stepping engines.

The reference warns before a run when the Courant number exceeds its limit
(beamz/simulation/fdtd.py:375-383, beamz/helpers.py:21-53) and then steps on; an
unstable run fills the fields with inf/NaN and every monitor and DFT sum with them.
Here the engines scan the E field on the device every ``every`` steps
(``bz_field_check``: a value that is not finite or above ``limit`` in magnitude
records BZ_ERR_DIVERGED and the step in two device words). The words are read when
the run ends (``raise_if_diverged``), so the check costs one pass over one field
array per ``every`` steps and no host synchronisation while stepping.
"""
from __future__ import annotations

import torch

from .. import _native as nat

CHECK_EVERY = 512
FIELD_LIMIT = 1e30


class DivergenceGuard:
    def __init__(self, device, every: int = CHECK_EVERY, limit: float = FIELD_LIMIT):
        self.status = torch.zeros(2, dtype=torch.int64, device=device)
        self.every = max(1, int(every))
        self.limit = float(limit)
        self.next = self.every
        self.launches = 0

    def check(self, field: torch.Tensor, bz_dtype: int, step: int) -> None:
        nat.field_check(field.data_ptr(), bz_dtype, field.numel(), self.limit, step, self.status.data_ptr(),
                        torch.cuda.current_stream().cuda_stream)
        self.launches += 1

    def maybe_check(self, field: torch.Tensor, bz_dtype: int, step: int) -> None:
        if step >= self.next:
            self.check(field, bz_dtype, step)
            self.next = (step // self.every + 1) * self.every

    def reset(self) -> None:
        self.status.zero_()
        self.next = self.every

    def raise_if_diverged(self, what: str = "") -> None:
        code, step = (int(v) for v in self.status.tolist())
        if code != 0:
            raise nat.NativeError(nat.BZ_ERR_DIVERGED,
                                  f"the fields diverged by step {step}: a value is not finite or exceeds "
                                  f"{self.limit:g}{what}")
