"""The adjoint of the step on the GPU (tq_adj_*), behind a forward/backward pair with the
torch.autograd.Function contract — forward(ctx, *inputs) saves what backward needs in ctx,
backward(ctx, grad_output) returns one gradient per input — without torch, as the host the
reference runs on (JavaScript) has none.

    cena = cenarios.cena_adjunto()                 # the scene: walls, particles, faucet, target
    adj = AdjuntoGPU(cena)
    ctx = Contexto()
    perda = PassoDiferenciavel.forward(ctx, adj, v0, theta)
    dv0, dtheta = PassoDiferenciavel.backward(ctx, 1.0)

The differentiated map is the substep with air tracking off, surface tension 0 and the density
correction off, its discrete structure held at the forward run's (include/tanque.h, tq_adj_*).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi


class AdjuntoGPU:
    """A tq_adj handle: the scene on the device, checkpoints of the last forward run."""

    def __init__(self, cena: dict, dispositivo: int = 0):
        self._lig = _abi.carregar()
        self._mantem, sc = _abi.cena_adjunto_c(cena)
        h = C.c_void_p()
        self._lig("adj_create", C.byref(sc), int(dispositivo), C.byref(h))
        self._h = h
        self.n0 = int(sc.n_particles)

    def fechar(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lig("adj_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.fechar()
        except Exception:
            pass

    def frente(self, v0, theta) -> float:
        v = np.ascontiguousarray(v0, dtype=np.float32).ravel()
        if v.size != 2 * self.n0:
            raise ValueError(f"v0 must hold 2 velocities for each of the {self.n0} particles")
        t = (C.c_double * 2)(float(theta[0]), float(theta[1]))
        perda = C.c_double()
        self._lig("adj_forward", self._h, v.ctypes.data if v.size else None, t, C.byref(perda))
        return perda.value

    def tras(self, grad_perda: float = 1.0):
        dv = np.zeros(2 * self.n0, np.float32)
        dt = (C.c_double * 2)()
        self._lig("adj_backward", self._h, float(grad_perda), dv.ctypes.data if dv.size else None, dt)
        return dv.reshape(-1, 2), np.array([dt[0], dt[1]])


class Contexto:
    """What forward saves for backward (torch's ctx)."""

    def save_for_backward(self, *objs):
        self.saved = objs


class PassoDiferenciavel:
    """forward: (adjunto, initial velocities, faucet velocity) -> loss; backward: the incoming
    gradient of the loss -> (None for the handle, dL/dv0, dL/dtheta).  The handle keeps the
    forward run's checkpoints; backward recomputes each segment from them."""

    @staticmethod
    def forward(ctx: Contexto, adjunto: AdjuntoGPU, v0, theta) -> float:
        perda = adjunto.frente(v0, theta)
        ctx.save_for_backward(adjunto)
        return perda

    @staticmethod
    def backward(ctx: Contexto, grad_perda: float):
        (adjunto,) = ctx.saved
        dv0, dtheta = adjunto.tras(grad_perda)
        return None, dv0, dtheta
