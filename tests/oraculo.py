"""Test-side binding of the CPU oracle (oracle/liboracle.so), mirroring the product binding.

Only tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg load the oracle.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from tanque import _abi
from tanque.simulacao import Simulacao

RAIZ = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SO = os.path.join(RAIZ, "oracle", "liboracle.so")

_P, _I, _D = C.c_void_p, C.c_int32, C.c_double

ASSINATURAS_ORACULO = dict(_abi.ASSINATURAS)
ASSINATURAS_ORACULO.update({
    "create_fp64": (C.c_int, [C.POINTER(_abi.TqOptions), C.POINTER(_P)]),
    "solve_pressure": (C.c_int, [_I, _I, _P, _P, _P, _I, _D, C.POINTER(_abi.TqBubbles), _I, C.POINTER(_D), _I,
                                 C.POINTER(_I), C.POINTER(_abi.TqSolveInfo)]),
    "vcycle": (C.c_int, [_I, _I, _P, _P, _P]),
    "scene_new": (_P, [_I, _I, _D]),
    "scene_free": (None, [_P]),
    "scene_trace": (None, [_P, _D, _D, _D, _D, _D, _I]),
    "scene_clear": (None, [_P]),
    "scene_sdf": (C.POINTER(C.c_float), [_P]),
    "scene_distance": (_D, [_P, _D, _D]),
    "scene_normal": (None, [_P, _D, _D, C.POINTER(_D), C.POINTER(_D)]),
    "scene_solid_cell": (_I, [_P, _I, _I]),
    "passo_maximo": (_D, [_D, _D, _D, _I, _D]),
    "semear_retangulo": (_I, [_D, _D, _D, _D, _D, C.POINTER(_D), C.POINTER(C.c_uint32), _P, _I]),
    "splat": (None, [_P, _I, _I, _I, _D, _I, _I, _P]),
    "adj_create": (C.c_int, [C.POINTER(_abi.TqAdjScene), C.POINTER(_P)]),
    "adj_destroy": (C.c_int, [_P]),
    "adj_forward": (C.c_int, [_P, _P, _P, _I, C.POINTER(_D)]),
    "adj_backward": (C.c_int, [_P, _P, _P]),
    "adj_count": (C.c_int, [_P, C.POINTER(_I)]),
})


class _Crua:
    """Calls that return values instead of a status (scene helpers)."""

    def __init__(self, lib):
        self.lib = lib

    def __getattr__(self, nome):
        return getattr(self.lib, "tqo_" + nome)


_CACHE = {}


def carregar_oraculo() -> _abi.Ligacao:
    if "lig" not in _CACHE:
        if not os.path.exists(SO):
            raise RuntimeError(f"oracle not built: make -C {os.path.dirname(SO)}")
        lib = C.CDLL(SO)
        lig = _abi.Ligacao(lib, "tqo_", ASSINATURAS_ORACULO)
        for nome in ["scene_new", "scene_free", "scene_trace", "scene_clear", "scene_sdf", "scene_distance",
                     "scene_normal", "scene_solid_cell", "passo_maximo", "semear_retangulo", "splat"]:
            fn = getattr(lib, "tqo_" + nome)
            fn.restype, fn.argtypes = ASSINATURAS_ORACULO[nome]
        lig.cru = _Crua(lib)
        _CACHE["lig"] = lig
    return _CACHE["lig"]


class CenaOraculo:
    """The oracle's Cena (js/cena.js restated in C++) with the product Cena's interface."""

    def __init__(self, nx, ny, h):
        self.o = carregar_oraculo().cru
        self.nx, self.ny, self.h = nx, ny, h
        self.mw, self.mh = 2 * nx, 2 * ny
        self.largura, self.altura = nx * h, ny * h
        self._c = self.o.scene_new(nx, ny, h)

    def __del__(self):
        try:
            self.o.scene_free(self._c)
        except Exception:
            pass

    def tracar(self, x0, y0, x1, y1, raio, apagar=False):
        self.o.scene_trace(self._c, x0, y0, x1, y1, raio, 1 if apagar else 0)

    def limpar(self):
        self.o.scene_clear(self._c)

    def atualizar(self):
        return True

    @property
    def sdf(self):
        p = self.o.scene_sdf(self._c)
        return np.ctypeslib.as_array(p, shape=(self.mw * self.mh,)).copy()

    @property
    def solido(self):
        return (self.sdf < 0).astype(np.uint8)

    def distancia(self, x, y):
        return self.o.scene_distance(self._c, x, y)

    def normal(self, x, y):
        a, b = C.c_double(), C.c_double()
        self.o.scene_normal(self._c, x, y, C.byref(a), C.byref(b))
        return a.value, b.value

    def celulaSolida(self, i, j):
        return bool(self.o.scene_solid_cell(self._c, i, j))


class SimulacaoOraculo(Simulacao):
    """SimulacaoCPU restated (the oracle), driven through the same surface as SimulacaoGPU."""

    def __init__(self, cena, opcoes=None, fp64=False):
        opcoes = dict(opcoes or {})
        opcoes.setdefault("p2g_mode", _abi.TQ_P2G_FLOAT)
        super().__init__(carregar_oraculo(), cena, opcoes, criar="create_fp64" if fp64 else "create")


def mancha_oraculo(particulas, nx, ny, h, largura, altura):
    """tqo_splat: the oracle's splat of a particle list (rows of 12 floats), (5, altura, largura)."""
    p = np.ascontiguousarray(particulas, dtype=np.float32).ravel()
    out = np.zeros(5 * largura * altura, dtype=np.float32)
    carregar_oraculo().cru.splat(p.ctypes.data, p.size // 12, nx, ny, h, largura, altura, out.ctypes.data)
    return out.reshape(5, altura, largura)


def resolver_pressao_oraculo(tipo, div, q, iteracoes=3, tolerancia=0.0, bolhas=None, precond=0, info=None):
    from tanque.simulacao import resolver_pressao
    return resolver_pressao(tipo, div, q, iteracoes, tolerancia, bolhas, precond=precond, info=info,
                            ligacao=carregar_oraculo())


def ciclo_v_oraculo(tipo, b):
    from tanque.simulacao import ciclo_v
    return ciclo_v(tipo, b, ligacao=carregar_oraculo())


class AdjuntoOraculo:
    """The FP64 CPU adjoint (oracle/adjunto_oracle.cpp) of a tanque.cenarios.cena_adjunto scene."""

    def __init__(self, cena: dict):
        self.lig = carregar_oraculo()
        self._mantem, sc = _abi.cena_adjunto_c(cena)
        h = C.c_void_p()
        self.lig("adj_create", C.byref(sc), C.byref(h))
        self._h = h
        self.n0 = cena["positions"].shape[0]

    def __del__(self):
        try:
            self.lig("adj_destroy", self._h)
        except Exception:
            pass

    def forward(self, v0, theta, gravar=True) -> float:
        v = np.ascontiguousarray(v0, dtype=np.float64).ravel()
        t = np.ascontiguousarray(theta, dtype=np.float64)
        perda = C.c_double()
        self.lig("adj_forward", self._h, v.ctypes.data, t.ctypes.data, 1 if gravar else 0, C.byref(perda))
        return perda.value

    def backward(self):
        gv = np.zeros(2 * self.n0, np.float64)
        gt = np.zeros(2, np.float64)
        self.lig("adj_backward", self._h, gv.ctypes.data, gt.ctypes.data)
        return gv.reshape(-1, 2), gt
