"""ctypes binding of the C-ABI declared in include/tanque.h.

`carregar()` loads the in-tree libtanque.so (built by `make` in tanque-de-agua_b200/) and
fails loudly when it is missing: there is no CPU fallback for the simulation step.
`ligar(lib, prefixo)` attaches the signatures to any library exporting the same entry points
under a prefix (the test suite uses it for the oracle, whose entry points mirror these ones).
"""
from __future__ import annotations

import ctypes as C
import os

RAIZ_PACOTE = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CAMINHO_LIB = os.path.join(RAIZ_PACOTE, "libtanque.so")

TQ_OK = 0
TQ_E_ARG = -1
TQ_E_CUDA = -2
TQ_E_NOMEM = -3
TQ_E_CAPACITY = -4
TQ_E_TIMEOUT = -5
TQ_E_NODEV = -6
TQ_E_STATE = -7

TQ_PREC_FP32, TQ_PREC_FP16, TQ_PREC_BF16 = 0, 1, 2
TQ_ENGINE_PLAIN, TQ_ENGINE_FUSED = 0, 1
TQ_P2G_FLOAT, TQ_P2G_FIXED = 0, 1
TQ_PRECOND_REFERENCE, TQ_PRECOND_BLOCK, TQ_PRECOND_BLOCK_1 = 0, 1, 2

# enum tq_field (include/tanque.h) -> (numpy dtype, size in units of N / nu / nv / 4096 / sdf)
CAMPOS_ENUM = {
    "tipo": 0, "rotulo": 1, "contagemCelula": 2, "solidoCelula": 3, "u": 4, "v": 5, "q": 6,
    "div": 7, "densidade": 8, "fase": 9, "curvatura": 10, "qAr": 11, "pressaoBolha": 12,
    "volumeAlvo": 13, "volumeBolha": 14, "rhsBolha": 15, "yBolha": 16, "vivo": 17,
    "uValida": 18, "vValida": 19, "uPeso": 20, "vPeso": 21, "normalX": 22, "normalY": 23,
    "corCelula": 24, "accU": 25, "accV": 26, "accCel": 27, "accCor": 28, "sdf": 29,
}
TQ_SCALAR_VMAX, TQ_SCALAR_PRIMEIRA, TQ_SCALAR_TIPOS_PRONTOS = 0, 1, 2
TQ_SCALAR_PCG_ITERS, TQ_SCALAR_PCG_RES0, TQ_SCALAR_PCG_RES = 3, 4, 5
TQ_SCALAR_LAUNCHES = 6
TQ_SCALAR_GRAVITY_X, TQ_SCALAR_GRAVITY_Y = 7, 8
TQ_SCALAR_PCG_TRUE_RES, TQ_SCALAR_PCG_CONVERGED = 9, 10
TQ_SCALAR_SOLVES, TQ_SCALAR_SOLVES_CAPPED, TQ_SCALAR_SOLVE_ITERS = 11, 12, 13
TQ_SCALAR_SOLVE_MAX_REL, TQ_SCALAR_SOLVE_REPLACEMENTS = 14, 15
TQ_SCALAR_CLOSED_REGIONS, TQ_SCALAR_GRAPH_FRAME_MS = 16, 17


class TqOptions(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("h", C.c_double), ("gravity", C.c_double * 2),
        ("iterations", C.c_int32), ("air", C.c_int32), ("tau_density", C.c_double),
        ("surface_tension", C.c_double), ("tolerance", C.c_double), ("precision", C.c_int32),
        ("engine", C.c_int32), ("p2g_mode", C.c_int32), ("capacity", C.c_int32),
        ("device", C.c_int32), ("preconditioner", C.c_int32), ("fused_ctas", C.c_int32),
        ("reserved", C.c_int32 * 5),
    ]


class TqTool(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("pad", C.c_int32), ("x", C.c_double), ("y", C.c_double),
        ("radius", C.c_double), ("vx", C.c_double), ("vy", C.c_double), ("absorb", C.c_double * 3),
    ]


class TqBubbles(C.Structure):
    _fields_ = [("rotulo", C.c_void_p), ("rhs", C.c_void_p), ("y", C.c_void_p)]


class TqFaucet(C.Structure):
    _fields_ = [
        ("x", C.c_double), ("y", C.c_double), ("radius", C.c_double), ("vx", C.c_double), ("vy", C.c_double),
        ("dt", C.c_double), ("absorb", C.c_double * 3), ("seed", C.c_uint32), ("pad", C.c_int32),
    ]


class TqAdjScene(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("h", C.c_double), ("dt", C.c_double), ("steps", C.c_int32),
        ("checkpoint_every", C.c_int32), ("gravity", C.c_double * 2), ("sdf", C.c_void_p), ("positions", C.c_void_p),
        ("affine", C.c_void_p), ("faucet_positions", C.c_void_p), ("target", C.c_void_p), ("n_particles", C.c_int32),
        ("faucet_per_step", C.c_int32),
    ]


class TqSolveInfo(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32), ("converged", C.c_int32), ("replacements", C.c_int32),
        ("closed_regions", C.c_int32),
        ("residual0", C.c_double), ("residual", C.c_double), ("true_residual", C.c_double),
    ]


class ErroTanque(RuntimeError):
    """Raised for a non-zero status of the C-ABI."""

    def __init__(self, status: int, onde: str, msg: str = ""):
        super().__init__(f"{onde}: status {status} ({msg})")
        self.status = status


_P = C.c_void_p
_I = C.c_int32
_D = C.c_double
_F = C.POINTER(C.c_float)

# name -> (restype, argtypes); the same list serves libtanque (tq_) and the oracle (tqo_).
ASSINATURAS = {
    "create": (C.c_int, [C.POINTER(TqOptions), C.POINTER(_P)]),
    "destroy": (C.c_int, [_P]),
    "set_walls": (C.c_int, [_P, _P, _I, _I]),
    "add_particles": (C.c_int, [_P, _P, _I, _I, C.POINTER(_I)]),
    "clear_particles": (C.c_int, [_P]),
    "apply_tool": (C.c_int, [_P, C.POINTER(TqTool)]),
    "advance": (C.c_int, [_P, _D, _I]),
    "substep": (C.c_int, [_P, _D]),
    "update_air": (C.c_int, [_P]),
    "reset_air": (C.c_int, [_P]),
    "count": (C.c_int, [_P, C.POINTER(_I)]),
    "get_particles": (C.c_int, [_P, _P, _I, C.POINTER(_I)]),
    "set_particles": (C.c_int, [_P, _P, _I]),
    "get_field": (C.c_int, [_P, _I, _P, C.c_int64]),
    "set_field": (C.c_int, [_P, _I, _P, C.c_int64]),
    "get_scalar": (C.c_int, [_P, _I, C.POINTER(_D)]),
    "set_scalar": (C.c_int, [_P, _I, _D]),
    "last_norms": (C.c_int, [_P, C.POINTER(_D), _I, C.POINTER(_I)]),
    "solve_pressure": (C.c_int, [_I, _I, _P, _P, _P, _I, _D, C.POINTER(TqBubbles), _I, _I, _I,
                                 C.POINTER(_D), _I, C.POINTER(_I), C.POINTER(TqSolveInfo)]),
    "vcycle": (C.c_int, [_I, _I, _P, _P, _P, _I]),
}
SO_PRODUTO = {
    "advance_graph": (C.c_int, [_P, _D, _I]),
    "launch_graph": (C.c_int, [_P, _D, _I]),
    "emit_faucet": (C.c_int, [_P, C.POINTER(TqFaucet), C.POINTER(_I)]),
    "set_tanks": (C.c_int, [_P, _I, _P]),
    "get_tank_residuals": (C.c_int, [_P, C.POINTER(_D), _I, C.POINTER(_I)]),
    "adj_create": (C.c_int, [C.POINTER(TqAdjScene), _I, C.POINTER(_P)]),
    "adj_destroy": (C.c_int, [_P]),
    "adj_forward": (C.c_int, [_P, _P, C.POINTER(_D), C.POINTER(_D)]),
    "adj_backward": (C.c_int, [_P, _D, _P, C.POINTER(_D)]),
    "sync": (C.c_int, [_P]),
    "get_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "set_timing": (C.c_int, [_P, _I]),
    "get_timing": (C.c_int, [_P, C.POINTER(_D), _I, C.POINTER(_I)]),
    "options_default": (None, [C.POINTER(TqOptions), _I, _I, _D]),
    "status_string": (C.c_char_p, [C.c_int]),
    "trace_wall": (C.c_int, [_P, _D, _D, _D, _D, _D, _I]),
    "clear_walls": (C.c_int, [_P]),
    "splat": (C.c_int, [_P, _I, _I, _P]),
    "last_error": (C.c_char_p, []),
}


class Ligacao:
    """The entry points of one library under one prefix, with error checking."""

    def __init__(self, lib: C.CDLL, prefixo: str, assinaturas: dict):
        self.lib = lib
        self.prefixo = prefixo
        self.f = {}
        for nome, (res, args) in assinaturas.items():
            fn = getattr(lib, prefixo + nome, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
            self.f[nome] = fn
        erro = getattr(lib, prefixo + "last_error", None)
        if erro is not None:
            erro.restype = C.c_char_p
            erro.argtypes = []
        self._erro = erro

    def tem(self, nome: str) -> bool:
        return nome in self.f

    def __call__(self, nome: str, *args):
        st = self.f[nome](*args)
        if st != TQ_OK:
            msg = self._erro().decode(errors="replace") if self._erro else ""
            raise ErroTanque(st, self.prefixo + nome, msg)
        return st


_LIGACAO = None


def carregar(caminho: str | None = None) -> Ligacao:
    """Loads libtanque.so (in-tree) once; raises if it has not been built."""
    global _LIGACAO
    if _LIGACAO is not None and caminho is None:
        return _LIGACAO
    alvo = caminho or CAMINHO_LIB
    if not os.path.exists(alvo):
        raise RuntimeError(
            f"libtanque.so not found at {alvo}: build it with `make -C tanque-de-agua_b200` "
            "(there is no CPU fallback for the simulation step)")
    lib = C.CDLL(alvo)
    assin = dict(ASSINATURAS)
    assin.update(SO_PRODUTO)
    lig = Ligacao(lib, "tq_", assin)
    if caminho is None:
        _LIGACAO = lig
    return lig


def opcoes_padrao(nx: int, ny: int, h: float, **kw) -> TqOptions:
    """tq_options_default plus keyword overrides (field names of tq_options)."""
    o = TqOptions()
    o.nx, o.ny, o.h = nx, ny, h
    o.gravity[0], o.gravity[1] = 0.0, -9.81
    o.iterations = 3
    o.air = 1
    o.tau_density = 0.1
    o.surface_tension = 0.0728
    o.tolerance = 0.0
    o.precision = TQ_PREC_FP32
    o.engine = TQ_ENGINE_PLAIN
    o.p2g_mode = TQ_P2G_FIXED
    o.capacity = 0
    o.device = 0
    o.preconditioner = TQ_PRECOND_REFERENCE
    for k, v in kw.items():
        if k == "gravity":
            o.gravity[0], o.gravity[1] = v
        else:
            setattr(o, k, v)
    return o


def cena_adjunto_c(cena: dict):
    """tq_adj_scene of a tanque.cenarios.cena_adjunto dict; returns (arrays to keep alive, struct)."""
    import numpy as np
    arr = {k: np.ascontiguousarray(cena[k], dtype=np.float32) for k in ("sdf", "positions", "faucet_positions", "target")}
    sc = TqAdjScene()
    sc.nx, sc.ny, sc.h, sc.dt = cena["nx"], cena["ny"], cena["h"], cena["dt"]
    sc.steps, sc.checkpoint_every = cena["steps"], cena.get("checkpoint_every", 10)
    sc.gravity[0], sc.gravity[1] = cena.get("gravity", (0.0, -9.81))
    sc.sdf = arr["sdf"].ctypes.data
    sc.positions = arr["positions"].ctypes.data if arr["positions"].size else None
    sc.affine = None
    sc.faucet_positions = arr["faucet_positions"].ctypes.data if arr["faucet_positions"].size else None
    sc.target = arr["target"].ctypes.data
    sc.n_particles = arr["positions"].shape[0]
    sc.faucet_per_step = arr["faucet_positions"].shape[1] if arr["faucet_positions"].ndim == 3 else 0
    return arr, sc
