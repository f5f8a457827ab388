"""Closed regions on the GPU (tolerance mode): water sealed by walls, on which A is singular.

- Solver: the hand-built grids of the oracle's tests (a sealed box of water, with and without
  an air pocket) through tq_solve_pressure on every engine, against the oracle: both converge
  to 1e-6 of the projected system, report one closed region and the same ||r0||, pin the
  region's root at 0, and q agrees to 1e-4.
- Simulation: a tank with a walled box of sealed water under its surface (with and without an
  air pocket inside), three substeps from the same state against the oracle (integers bit for
  bit, u, v and q to 1e-3, positions to 1e-5 m), then 200 substeps with every solve converged.
- Tank 29 of the 256-tank batch (285 x 142 cells, h = 3 mm), whose wall segments seal a
  77-cell cavity: in the batch one of its substeps once ran to the 1000-iteration cap with a
  diverging residual (2e6 ||r0||).  Alone, four frames (64 substeps) with no capped solve.
"""
import math

import numpy as np
import pytest

from estado import comparar_passo, copiar_estado, erro_relativo, regioes_fechadas, sem_constante
from oraculo import SimulacaoOraculo, resolver_pressao_oraculo
from tanque import Cena, SimulacaoGPU, _abi, passo_maximo
from tanque.lote import gerar_tanques, montar_atlas
from tanque.simulacao import resolver_pressao
from test_oracle_regioes import RAIZ, dados

pytestmark = pytest.mark.gpu

MOTORES = [
    pytest.param(_abi.TQ_PREC_FP32, _abi.TQ_ENGINE_PLAIN, _abi.TQ_PRECOND_REFERENCE, id="fp32-plain"),
    pytest.param(_abi.TQ_PREC_FP32, _abi.TQ_ENGINE_FUSED, _abi.TQ_PRECOND_REFERENCE, id="fp32-fused"),
    pytest.param(_abi.TQ_PREC_FP16, _abi.TQ_ENGINE_FUSED, _abi.TQ_PRECOND_BLOCK, id="fp16-fused-block"),
    pytest.param(_abi.TQ_PREC_FP16, _abi.TQ_ENGINE_FUSED, _abi.TQ_PRECOND_BLOCK_1, id="fp16-fused-block1"),
]


@pytest.mark.parametrize("bolha", [False, True], ids=["agua-selada", "selada-com-bolha"])
@pytest.mark.parametrize("precisao,motor,precond", MOTORES)
def test_solve_com_regiao_fechada(lib_gpu, bolha, precisao, motor, precond):
    tipo, div, bol = dados(bolha)
    res = {}
    for lado in ("gpu", "oraculo"):
        q = np.zeros(tipo.size, np.float32)
        b = {k: v.copy() for k, v in bol.items()} if bol else None
        info = {}
        if lado == "gpu":
            resolver_pressao(tipo, div, q, 1000, 1e-6, b, precisao, motor, precond, info=info)
        else:
            resolver_pressao_oraculo(tipo, div, q, 1000, 1e-6, b, precond=precond, info=info)
        res[lado] = (q, b, info)
    (qg, bg, ig), (qo, bo, io) = res["gpu"], res["oraculo"]
    assert ig["converged"] == 1 and ig["closed_regions"] == 1, ig
    assert qg[RAIZ] == 0.0 and qo[RAIZ] == 0.0
    assert 0 <= ig["true_residual"] <= 1e-6 * ig["residual0"]
    assert abs(ig["residual0"] - io["residual0"]) <= 1e-6 * io["residual0"]
    reg = regioes_fechadas(tipo, bol["rotulo"].reshape(tipo.shape) if bol else np.zeros(tipo.shape, np.uint32))
    assert len(reg) == 1
    if bol:  # the bubble pressures enter the comparison as the bubbles' cells
        for q, b in ((qg, bg), (qo, bo)):
            rot = b["rotulo"]
            q[rot == 5] = b["y"][5]
            q[rot == 7] = b["y"][7]
    e = erro_relativo(sem_constante(qg, tipo, reg), sem_constante(qo, tipo, reg))
    assert e <= 1e-4, e


def caixa_selada(bolha: bool):
    """A 64 x 64 tank (h = 1 cm) with water to 60 % of its height and, under the water, a box of
    2-cell walls (columns 12..35, rows 6..23) whose inside is sealed water; with `bolha` a
    5 x 4-cell air pocket inside the box (an enclosed bubble).  Returns (scene, particles)."""
    from tanque.cenarios import semear_retangulo, semente
    from tanque.constantes import CAMPOS, MOLDURA, SDF_MAX
    h, nx, ny = 0.01, 64, 64
    c = Cena(nx, ny, h)
    r = c.r
    m = np.asarray(c.sdf, dtype=np.float32).reshape(ny * r, nx * r).copy()
    for i0, i1, j0, j1 in [(12, 36, 6, 8), (12, 36, 22, 24), (12, 14, 6, 24), (34, 36, 6, 24)]:
        m[j0 * r:j1 * r, i0 * r:i1 * r] = -SDF_MAX
    c.sdf[:] = m.ravel()
    mm = MOLDURA * h
    agua = semear_retangulo(mm, mm, nx * h - mm, 0.6 * ny * h, h, (0, 0, 0), semente(5)).reshape(-1, CAMPOS)
    if bolha:
        x, y = agua[:, 0] / h, agua[:, 1] / h
        agua = agua[~((x >= 20) & (x < 25) & (y >= 15) & (y < 19))]
    return c, agua.ravel().copy()


@pytest.mark.parametrize("bolha", [False, True], ids=["agua-selada", "selada-com-bolha"])
@pytest.mark.parametrize("precisao,motor,precond", MOTORES)
def test_caixa_selada_contra_o_oraculo(lib_gpu, bolha, precisao, motor, precond):
    cena, agua = caixa_selada(bolha)
    opc = {"tolerance": 1e-6, "iterations": 1000, "preconditioner": precond}
    o = SimulacaoOraculo(cena, dict(opc, p2g_mode=_abi.TQ_P2G_FIXED))
    g = SimulacaoGPU(cena, dict(opc, precision=precisao, engine=motor))
    for s in (o, g):
        s.adicionar(agua, False)
        s.avancar(1 / 240, 1)
    for quadro in range(3):
        copiar_estado(o, g)
        o.avancar(1 / 240, 1)
        g.avancar(1 / 240, 1)
        assert o.escalar(_abi.TQ_SCALAR_CLOSED_REGIONS) == 1
        assert g.escalar(_abi.TQ_SCALAR_CLOSED_REGIONS) == 1
        assert g.escalar(_abi.TQ_SCALAR_PCG_CONVERGED) == 1
        comparar_passo(o, g, f"substep {quadro}", fechadas=True)
    # 200 substeps on the GPU: every solve converges
    g.definirEscalar(_abi.TQ_SCALAR_SOLVES, 0)
    for _ in range(50):
        g.avancar(4 / 240, 4)
    assert g.escalar(_abi.TQ_SCALAR_SOLVES) == 200
    assert g.escalar(_abi.TQ_SCALAR_SOLVES_CAPPED) == 0
    assert g.escalar(_abi.TQ_SCALAR_SOLVE_MAX_REL) <= 1e-6


@pytest.mark.parametrize("precisao,motor,precond", MOTORES)
def test_tanque_29_do_lote(lib_gpu, precisao, motor, precond):
    """Tank 29 of the batch, alone: four frames, every solve converged."""
    h = 0.003
    t = gerar_tanques(h=h)[29]
    at = montar_atlas(Cena, [t], h)
    dt = passo_maximo(h, t["ny"] * h)
    sub = math.ceil((1 / 60) / dt - 1e-9)
    opc = {"tolerance": 1e-6, "iterations": 1000, "precision": precisao, "engine": motor, "preconditioner": precond}
    g = SimulacaoGPU(at["cena"], opc)
    g.adicionar(at["particulas"], False)
    g.definirEscalar(_abi.TQ_SCALAR_SOLVES, 0)
    for _ in range(4):
        g.avancar(1 / 60, sub)
    assert g.escalar(_abi.TQ_SCALAR_SOLVES) == 4 * sub
    assert g.escalar(_abi.TQ_SCALAR_SOLVES_CAPPED) == 0
    assert g.escalar(_abi.TQ_SCALAR_SOLVE_MAX_REL) <= 1e-6
