"""Step-state checkpoints of the stepping engines (the reference has none for a
simulation; its only persistence is Monitor.save_data, beamz/devices/monitors.py:569-589).

``engine_state(eng)`` folds the monitor samples still in the ring into the float64 DFT
sums, moves the recorded monitor rows to the host, and returns on the host: both copies
of every field array, the DFT sums, the accumulated power, the recorded rows, the step
index and the material/layout it belongs to. ``load_engine_state(eng, state)`` puts that
into an engine built for the same problem (same grid, precision, components, designs,
sources and monitors: checked) so that stepping continues from it.

Continuing a restored run gives the bits of the uninterrupted run when the checkpoint is
taken where the uninterrupted run has folded every pending sample anyway: after a whole
number of graph chunks of ``run_steps`` (``eng.chunk`` steps in 2D, 32 in 3D). Elsewhere
the fields and records are still identical and the DFT sums differ only by the grouping
of their float64 additions.
"""
from __future__ import annotations

import numpy as np
import torch

FORMAT = "beamz_b200.engine_state.v1"


def _field_arrays(eng) -> dict:
    if hasattr(eng, "f"):  # 3D
        return {k: v for k, v in eng.f.items()}
    return {"Ez": eng.ez, "Hx": eng.hx, "Hy": eng.hy}


def _rec_owner(eng):
    return getattr(eng, "mops", None) if hasattr(eng, "mops") else getattr(eng, "gops", None)


def engine_state(eng) -> dict:
    eng._fold()
    if eng.record is not None:
        eng._maybe_drain(force=True)
    fields = {k: [c.detach().cpu().clone() for c in copies] for k, copies in _field_arrays(eng).items()}
    rec = _rec_owner(eng)
    return {
        "format": FORMAT,
        "kind": "3d" if hasattr(eng, "f") else "2d",
        "dtype": str(eng.dtype),
        "n_designs": eng.n_designs,
        "n_comp": eng.n_comp,
        "shape": tuple(fields["Ez"][0].shape),
        "n_steps": eng.n_steps,
        "step_index": int(eng.step_index),
        "folded": int(eng._folded),
        "fields": fields,
        "dft": None if eng.dft is None else eng.dft.detach().cpu().clone(),
        "power": None if eng.power is None else eng.power.detach().cpu().clone(),
        "records": [np.array(r) for r in getattr(eng, "_rec_host", [])],
        "rec_step0": int(rec.rec_step0) if (rec is not None and eng.record is not None) else 0,
        "ce_sum": float(eng.ce.double().sum()),
        "loss_sum": float(eng.loss.double().sum()),
    }


def load_engine_state(eng, st: dict) -> None:
    if st.get("format") != FORMAT:
        raise ValueError("not an engine state written by beamz_b200 (format tag missing or different)")
    kind = "3d" if hasattr(eng, "f") else "2d"
    arrays = _field_arrays(eng)
    checks = [("kind", kind), ("dtype", str(eng.dtype)), ("n_designs", eng.n_designs), ("n_comp", eng.n_comp),
              ("shape", tuple(arrays["Ez"][0].shape)), ("n_steps", eng.n_steps)]
    for key, want in checks:
        if st[key] != want:
            raise ValueError(f"checkpoint {key} {st[key]!r} does not match this simulation's {want!r}")
    if (st["dft"] is None) != (eng.dft is None) or (st["power"] is None) != (eng.power is None):
        raise ValueError("checkpoint monitors / power accumulation do not match this simulation")
    for name, val in (("ce_sum", float(eng.ce.double().sum())), ("loss_sum", float(eng.loss.double().sum()))):
        if not np.isclose(st[name], val, rtol=1e-12, atol=0.0):
            raise ValueError("checkpoint was taken on a different material grid")
    for k, copies in arrays.items():
        for dst, src in zip(copies, st["fields"][k]):
            dst.copy_(src.to(dst.device))
    if eng.dft is not None:
        eng.dft.copy_(st["dft"].to(eng.dft.device))
    if eng.power is not None:
        eng.power.copy_(st["power"].to(eng.power.device))
    eng.step_index = st["step_index"]
    eng._folded = st["folded"]
    if eng.record is not None:
        eng._rec_host = [np.array(r) for r in st["records"]]
        _rec_owner(eng).rec_step0 = st["rec_step0"]
    eng._graphs.clear()
    eng.guard.reset()
    eng.guard.next = (eng.step_index // eng.guard.every + 1) * eng.guard.every
    torch.cuda.current_stream().synchronize()
