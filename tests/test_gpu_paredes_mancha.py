"""Wall tracing and the headless splat on the GPU, through the C-ABI, against the oracle.

- tq_trace_wall: capsule segments drawn and erased on the device mask equal, bit for bit, the
  mask the oracle's Cena.tracar restatement makes (and the package's numpy Cena), and so do
  the solid cells; tq_clear_walls gives back the empty tank's frame.
- tq_splat: the splat of the handle's particles (with dye and foam), before and after a
  frame of substeps, equals the oracle's splat of the same particles bit for bit (64-bit fixed-point sums), for
  targets at, above and below the grid's resolution, square or not.
"""
import numpy as np
import pytest

from estado import cena_bolha
from oraculo import CenaOraculo, mancha_oraculo
from tanque import Cena, SimulacaoGPU, _abi
from tanque.constantes import CAMPOS

pytestmark = pytest.mark.gpu

TRACOS = [
    (0.10, 0.10, 0.40, 0.25, 0.012, False),
    (0.35, 0.05, 0.35, 0.45, 0.020, False),
    (0.20, 0.30, 0.20, 0.30, 0.030, False),  # a dot (zero-length segment)
    (0.30, 0.20, 0.38, 0.22, 0.015, True),   # erase across a wall
    (0.00, 0.00, 0.20, 0.00, 0.015, True),   # erase reaching the frame: the frame stays
    (0.55, 0.55, 0.70, 0.30, 0.008, False),  # partly outside the tank
]


def test_tracar_paredes_no_dispositivo(lib_gpu):
    nx, ny, h = 64, 48, 0.01
    g = SimulacaoGPU(Cena(nx, ny, h), {"iterations": 3})
    co = CenaOraculo(nx, ny, h)
    cp = Cena(nx, ny, h)
    for (x0, y0, x1, y1, r, apagar) in TRACOS:
        g.tracarParede(x0, y0, x1, y1, r, apagar)
        co.tracar(x0, y0, x1, y1, r, apagar)
        cp.tracar(x0, y0, x1, y1, r, apagar)
        sdf = g.campo("sdf")
        assert np.array_equal(sdf.view(np.uint32), co.sdf.view(np.uint32))
        assert np.array_equal(sdf.view(np.uint32), np.asarray(cp.sdf, dtype=np.float32).view(np.uint32))
        assert np.array_equal(g.campo("solidoCelula"), _solidos(co, nx, ny))
    g.limparParedes()
    assert np.array_equal(g.campo("sdf").view(np.uint32), Cena(nx, ny, h).sdf.view(np.uint32))
    assert np.array_equal(g.campo("solidoCelula"), _solidos(Cena(nx, ny, h), nx, ny))
    with pytest.raises(_abi.ErroTanque) as e:
        g.tracarParede(float("nan"), 0.0, 0.1, 0.1, 0.01)
    assert e.value.status == _abi.TQ_E_ARG
    g.fechar()


def _solidos(cena, nx, ny):
    """Cena.celulaSolida (js/cena.js:119-127) for every cell, from the mask."""
    m = np.asarray(cena.sdf, dtype=np.float64).reshape(2 * ny, 2 * nx)
    s = m[0::2, 0::2] + m[0::2, 1::2] + m[1::2, 0::2] + m[1::2, 1::2]
    return (s < 0).astype(np.uint8).ravel()


@pytest.mark.parametrize("alvo", [(60, 60), (120, 96), (37, 23)], ids=["celulas", "dobro", "menor"])
def test_mancha_contra_o_oraculo(lib_gpu, alvo):
    cena, agua = cena_bolha(Cena)
    g = SimulacaoGPU(cena, {"tolerance": 1e-6, "iterations": 200, "precision": _abi.TQ_PREC_FP16,
                            "engine": _abi.TQ_ENGINE_FUSED})
    g.adicionar(agua, False)
    w, hp = alvo
    p = g.p.reshape(-1, CAMPOS).copy()
    p[::3, 8] = np.linspace(0.0, 1.0, len(p[::3]), dtype=np.float32)  # foam on a third of them
    g.definirParticulas(p)
    for passo in range(2):
        p = g.p.reshape(-1, CAMPOS)
        img = g.mancha(w, hp)
        ref = mancha_oraculo(p, cena.nx, cena.ny, cena.h, w, hp)
        assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))
        assert img[0].max() > 1.0 and np.any(img[2] > 0) and np.any(img[4] > 0)
        g.avancar(1 / 60, 8)
    g.fechar()
