"""The B200 backend: CUDA tensors plus the Backend interface's two updates.

Arrays are ``torch`` tensors on the current CUDA device. ``update_h_fields`` and
``update_e_field`` run the unfused kernels of libbeamz_b200 on arrays with the
reference's shapes (returning the updated arrays like the NumPy backend); the
``FDTD`` class itself does not use them and steps with the fused kernel instead.
"""
from __future__ import annotations

import numpy as np
import torch

from ... import _native as nat
from .base import Backend

_NP2TORCH = {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
             np.dtype(np.complex64): torch.complex64, np.dtype(np.complex128): torch.complex128}


class B200Backend(Backend):
    device = "cuda"

    def __init__(self, **kwargs):
        if not torch.cuda.is_available():
            raise RuntimeError("beamz_b200 needs a CUDA GPU (sm_100a); none is visible")
        self.options = dict(kwargs)
        self.dev = torch.device("cuda", torch.cuda.current_device())

    def _dtype(self, dtype):
        if dtype is None:
            return torch.float64
        if isinstance(dtype, torch.dtype):
            return dtype
        return _NP2TORCH[np.dtype(dtype)]

    def zeros(self, shape, dtype=None):
        return torch.zeros(shape, dtype=self._dtype(dtype), device=self.dev)

    def ones(self, shape, dtype=None):
        return torch.ones(shape, dtype=self._dtype(dtype), device=self.dev)

    def copy(self, array):
        return array.clone()

    def to_numpy(self, array):
        if isinstance(array, torch.Tensor):
            return array.detach().cpu().numpy()
        return np.asarray(array)

    def from_numpy(self, array):
        return torch.as_tensor(np.ascontiguousarray(array)).to(self.dev)

    def roll(self, array, shift, axis=None):
        return torch.roll(array, shift, dims=axis)

    @staticmethod
    def _real_layout(t: torch.Tensor):
        if t.is_complex():
            return torch.view_as_real(t), 2, (nat.BZ_F32 if t.dtype == torch.complex64 else nat.BZ_F64)
        return t, 1, (nat.BZ_F32 if t.dtype == torch.float32 else nat.BZ_F64)

    def _prep(self, Hx, Hy, Ez):
        cplx = any(isinstance(a, torch.Tensor) and a.is_complex() for a in (Hx, Hy, Ez))
        wide = any(a.dtype in (torch.float64, torch.complex128) for a in (Hx, Hy, Ez))
        dt = (torch.complex128 if wide else torch.complex64) if cplx else (torch.float64 if wide else torch.float32)
        return [self.from_numpy(a) if not isinstance(a, torch.Tensor) else a.to(self.dev) for a in (Hx, Hy, Ez)], dt

    def update_h_fields(self, Hx, Hy, Ez, sigma, dx, dy, dt, mu_0, eps_0):
        (Hx, Hy, Ez), ft = self._prep(Hx, Hy, Ez)
        Hx, Hy, Ez = (a.to(ft).contiguous() for a in (Hx, Hy, Ez))
        ny, nx = Ez.shape
        rt = torch.float64 if ft in (torch.float64, torch.complex128) else torch.float32
        sg = torch.as_tensor(sigma).to(self.dev, rt).contiguous()
        hx, nc, code = self._real_layout(Hx)
        hy, _, _ = self._real_layout(Hy)
        ez, _, _ = self._real_layout(Ez)
        nat.update_h2d(code, ny, nx, nc, hx.data_ptr(), hy.data_ptr(), ez.data_ptr(), sg.data_ptr(), float(dx),
                       float(dy), float(dt), float(mu_0), float(eps_0), torch.cuda.current_stream().cuda_stream)
        return Hx, Hy

    def update_e_field(self, Ez, Hx, Hy, sigma, epsilon_r, dx, dy, dt, eps_0):
        (Hx, Hy, Ez), ft = self._prep(Hx, Hy, Ez)
        Hx, Hy, Ez = (a.to(ft).contiguous() for a in (Hx, Hy, Ez))
        ny, nx = Ez.shape
        rt = torch.float64 if ft in (torch.float64, torch.complex128) else torch.float32
        sg = torch.as_tensor(sigma).to(self.dev, rt).contiguous()
        er = torch.as_tensor(epsilon_r).to(self.dev, rt).contiguous()
        ez, nc, code = self._real_layout(Ez)
        hx, _, _ = self._real_layout(Hx)
        hy, _, _ = self._real_layout(Hy)
        nat.update_e2d(code, ny, nx, nc, ez.data_ptr(), hx.data_ptr(), hy.data_ptr(), sg.data_ptr(), er.data_ptr(),
                       float(dx), float(dy), float(dt), float(eps_0), torch.cuda.current_stream().cuda_stream)
        return Ez
