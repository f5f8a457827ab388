"""Parity of the CUDA library with the oracle, stage by stage and for whole substeps.

Integer work is compared bit for bit: the x65536 particle-to-grid sums, cell flags, particle
counts, air labels, bubble ids, target volumes and alive sets.  Floating-point fields are
compared with the tolerances written next to each assertion.  The oracle runs with the same
particle-to-grid semantics as the library (TQ_P2G_FIXED).
"""
import math

import numpy as np
import pytest

from estado import CENAS, copiar_estado, erro_relativo
from oraculo import CenaOraculo, SimulacaoOraculo, ciclo_v_oraculo, resolver_pressao_oraculo
from tanque import Cena, SimulacaoGPU, _abi, ciclo_v, resolver_pressao
from tanque.constantes import AGUA, AR, CAMPOS, MAX_BOLHAS, passo_maximo

pytestmark = pytest.mark.gpu

OPC_FIXO = {"p2g_mode": _abi.TQ_P2G_FIXED}


def par(nome, opcoes=None):
    """The same scene in the oracle and on the GPU (walls built once, by the oracle's Cena)."""
    cena_o, agua = CENAS[nome](CenaOraculo)
    cena_g = Cena(cena_o.nx, cena_o.ny, cena_o.h)
    cena_g.sdf[:] = cena_o.sdf
    o = SimulacaoOraculo(cena_o, dict(OPC_FIXO, **(opcoes or {})))
    g = SimulacaoGPU(cena_g, dict(opcoes or {}))
    o.adicionar(agua, False)
    g.adicionar(agua, False)
    return o, g


def problema_de_pressao(nome, passos=6):
    """A real pressure problem: the state of a scene after a few oracle frames."""
    cena_o, agua = CENAS[nome](CenaOraculo)
    o = SimulacaoOraculo(cena_o, OPC_FIXO)
    o.adicionar(agua, False)
    for _ in range(passos):
        o.avancar(1 / 60, 2)
    nx, ny = o.nx, o.ny
    tipo = o.campo("tipo").reshape(ny, nx)
    div = o.campo("div").reshape(ny, nx)
    rot = o.campo("rotulo")
    return tipo, div, rot, o


# ------------------------------------------------------------------ V-cycle
@pytest.mark.parametrize("nome", ["barragem", "bolha", "copo"])
@pytest.mark.parametrize("prec,tol", [(_abi.TQ_PREC_FP32, 2e-5), (_abi.TQ_PREC_FP16, 2e-3), (_abi.TQ_PREC_BF16, 2e-2)],
                         ids=["fp32", "fp16", "bf16"])
def test_ciclo_v(lib_gpu, nome, prec, tol):
    tipo, div, rot, _ = problema_de_pressao(nome)
    t0 = tipo.copy()
    t0[(tipo == AR) & (rot.reshape(tipo.shape) >= 2)] = AGUA
    b = div.astype(np.float32)
    x_o = ciclo_v_oraculo(t0, b)
    x_g = ciclo_v(t0, b, precisao=prec)
    # FP32 arithmetic on the GPU vs double-then-round in the oracle; half storage adds its
    # own rounding: relative L-infinity tolerance per storage type.
    assert erro_relativo(x_g, x_o) < tol


@pytest.mark.parametrize("nx,ny", [(13, 9), (40, 30), (161, 77), (840, 536)])
def test_ciclo_v_tamanhos(lib_gpu, nx, ny):
    """Grids with odd sizes, a single level, and the 450k-cell grid; random water/air/walls."""
    rng = np.random.default_rng(nx * 1000 + ny)
    tipo = np.full((ny, nx), AGUA, np.uint8)
    tipo[rng.random((ny, nx)) < 0.08] = 0
    tipo[: ny // 6, :] = AR
    tipo[:, 0] = tipo[:, -1] = tipo[0, :] = tipo[-1, :] = 0
    b = rng.standard_normal((ny, nx)).astype(np.float32)
    b[tipo != AGUA] = 0
    x_o = ciclo_v_oraculo(tipo, b)
    x_g = ciclo_v(tipo, b)
    assert erro_relativo(x_g, x_o) < 2e-5


# ------------------------------------------------------------------ PCG
MOTORES = [pytest.param(_abi.TQ_ENGINE_PLAIN, id="plain"), pytest.param(_abi.TQ_ENGINE_FUSED, id="fused")]


@pytest.mark.parametrize("motor", MOTORES)
@pytest.mark.parametrize("nome", ["barragem", "bolha", "copo"])
@pytest.mark.parametrize("com_bolhas", [False, True], ids=["sem-bolhas", "com-bolhas"])
def test_pcg_iteracoes_fixas(lib_gpu, nome, com_bolhas, motor):
    tipo, div, rot, o = problema_de_pressao(nome)
    q0 = np.zeros(tipo.size, np.float32)
    bol_o = bol_g = None
    if com_bolhas:
        rhs = o.campo("rhsBolha")
        y = o.campo("yBolha")
        bol_o = dict(rotulo=rot.copy(), rhs=rhs.copy(), y=y.copy())
        bol_g = dict(rotulo=rot.copy(), rhs=rhs.copy(), y=y.copy())
    q_o, q_g = q0.copy(), q0.copy()
    n_o = resolver_pressao_oraculo(tipo, div, q_o, 3, 0.0, bol_o)
    n_g = resolver_pressao(tipo, div, q_g, 3, 0.0, bol_g, motor=motor)
    assert len(n_o) == len(n_g) == 4
    # FP32 CG with FP64 dots vs the oracle's double-then-round: 1e-4 relative on q and on the
    # residual history (the fixed three iterations amplify rounding differences a little).
    assert erro_relativo(q_g, q_o) < 1e-4
    assert erro_relativo(n_g, n_o) < 1e-3
    if com_bolhas:
        assert erro_relativo(bol_g["y"], bol_o["y"]) < 1e-3


@pytest.mark.parametrize("motor", MOTORES)
@pytest.mark.parametrize("prec", [_abi.TQ_PREC_FP32, _abi.TQ_PREC_FP16, _abi.TQ_PREC_BF16], ids=["fp32", "fp16", "bf16"])
def test_pcg_tolerancia(lib_gpu, prec, motor):
    """With a tolerance the solve runs to ||r|| <= 1e-6 ||r0|| (the oracle agrees on q)."""
    tipo, div, rot, o = problema_de_pressao("copo")
    q_o = np.zeros(tipo.size, np.float32)
    q_g = q_o.copy()
    n_o = resolver_pressao_oraculo(tipo, div, q_o, 200, 1e-6)
    n_g = resolver_pressao(tipo, div, q_g, 200, 1e-6, precisao=prec, motor=motor)
    assert n_g[-1] <= 1e-6 * n_g[0]
    assert n_o[-1] <= 1e-6 * n_o[0]
    assert erro_relativo(q_g, q_o) < 1e-4
    assert len(n_g) <= len(n_o) + 3


# ------------------------------------------------------------------ air tracker
def _bolhas_em_movimento(nx, ny, quadros, seed):
    """A sequence of cell-flag grids: water with drifting, splitting and merging air blobs."""
    rng = np.random.default_rng(seed)
    jj, ii = np.mgrid[0:ny, 0:nx]
    cx = rng.uniform(5, nx - 5, 9)
    cy = rng.uniform(5, ny * 0.7, 9)
    r = rng.uniform(1.2, 5, 9)
    vx = rng.uniform(-0.8, 0.8, 9)
    vy = rng.uniform(0.2, 1.2, 9)
    seq = []
    for f in range(quadros):
        tipo = np.full((ny, nx), AGUA, np.uint8)
        tipo[int(ny * 0.8):, :] = AR
        for k in range(9):
            x, y = cx[k] + vx[k] * f, cy[k] + vy[k] * f
            rr = r[k] * (1 + 0.3 * math.sin(f * 0.7 + k))
            tipo[(ii - x) ** 2 + (jj - y) ** 2 < rr * rr] = AR
        tipo[rng.random((ny, nx)) < 0.01] = AR  # vacuum specks
        tipo[:2, :] = tipo[-2:, :] = 0
        tipo[:, :2] = tipo[:, -2:] = 0
        seq.append(tipo.ravel())
    return seq


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_rastreador_de_ar_bit_exato(lib_gpu, seed):
    nx, ny = 80, 64
    h = 0.01
    o = SimulacaoOraculo(CenaOraculo(nx, ny, h), OPC_FIXO)
    g = SimulacaoGPU(Cena(nx, ny, h))
    pres = np.random.default_rng(seed).uniform(-50, 50, MAX_BOLHAS).astype(np.float32)
    o.definirCampo("pressaoBolha", pres)
    g.definirCampo("pressaoBolha", pres)
    for f, tipo in enumerate(_bolhas_em_movimento(nx, ny, 40, seed)):
        for s in (o, g):
            s.definirCampo("tipo", tipo)
            s.definirEscalar(_abi.TQ_SCALAR_TIPOS_PRONTOS, 1)
            s.atualizarAr()
        for campo in ["rotulo", "vivo"]:
            assert np.array_equal(g.campo(campo), o.campo(campo)), f"quadro {f}: {campo}"
        for campo in ["volumeAlvo", "pressaoBolha"]:
            assert np.array_equal(g.campo(campo).view(np.uint32), o.campo(campo).view(np.uint32)), f"quadro {f}: {campo}"


# ------------------------------------------------------------------ whole substeps
INTEIROS = ["accU", "accV", "accCel", "accCor", "tipo", "contagemCelula", "rotulo", "vivo", "volumeBolha"]
# field -> relative L-infinity tolerance after one substep from identical state
FLUTUANTES = {"u": 1e-4, "v": 1e-4, "q": 1e-4, "div": 1e-5, "fase": 1e-6, "curvatura": 1e-4, "qAr": 1e-4,
              "pressaoBolha": 1e-3, "volumeAlvo": 0.0}


@pytest.mark.parametrize("motor", MOTORES)
@pytest.mark.parametrize("nome", ["barragem", "bolha", "copo"])
def test_subpasso_paridade(lib_gpu, nome, motor):
    o, g = par(nome, {"engine": motor})
    dt = passo_maximo(o.h, o.cena.altura, None)
    for quadro in range(8):
        copiar_estado(o, g)
        o.avancar(1 / 60 / 3, 1)
        g.avancar(1 / 60 / 3, 1)
        for campo in INTEIROS:
            a, b = g.campo(campo), o.campo(campo)
            assert np.array_equal(a, b), f"quadro {quadro}: {campo} differs in {np.count_nonzero(a != b)} entries"
        for campo, tol in FLUTUANTES.items():
            e = erro_relativo(g.campo(campo), o.campo(campo))
            assert e <= tol, f"quadro {quadro}: {campo} relative error {e:.3g} > {tol}"
        pg, po = g.p.reshape(-1, CAMPOS), o.p.reshape(-1, CAMPOS)
        assert pg.shape == po.shape
        # positions: 1e-6 m absolute; velocities and affine terms 1e-4 relative
        assert float(np.max(np.abs(pg[:, :2].astype(np.float64) - po[:, :2]))) < 1e-6
        assert erro_relativo(pg[:, 2:8], po[:, 2:8]) < 1e-4
        assert erro_relativo(pg[:, 8:], po[:, 8:]) < 1e-5
        assert abs(g.vMax - o.vMax) <= 1e-4 * max(o.vMax, 1e-6)
    del dt


@pytest.mark.parametrize("ordem", ["embaralhada", "meio-a-meio"])
def test_particulas_em_qualquer_ordem(lib_gpu, ordem):
    """The particle-to-grid sums are the oracle's bit for bit, and the grid-to-particle
    transfer within the substep tolerances, whatever the particle order.  Shuffled particles
    give every block of 256 a bounding box larger than its shared-memory sums hold, so each
    contribution goes to the grid directly; with only the second half shuffled, the blocks of
    the first half sum in shared memory and the rest directly.  A third of the particles carry
    dye."""
    o, g = par("bolha")
    o.avancar(1 / 60 / 3, 1)
    P = o.p.reshape(-1, CAMPOS).copy()
    n = len(P)
    assert n > 8 * 256
    rng = np.random.default_rng(11)
    perm = rng.permutation(n)
    if ordem == "meio-a-meio":
        perm = np.concatenate([np.arange(n // 2), n // 2 + rng.permutation(n - n // 2)])
    P = P[perm]
    P[::3, 9:12] = rng.random((len(P[::3]), 3)).astype(np.float32)
    o.definirParticulas(P)
    copiar_estado(o, g)
    o.avancar(1 / 60 / 3, 1)
    g.avancar(1 / 60 / 3, 1)
    for campo in ["accU", "accV", "accCel", "accCor"]:
        a, b = g.campo(campo), o.campo(campo)
        assert np.array_equal(a, b), f"{campo} differs in {np.count_nonzero(a != b)} entries"
    assert np.count_nonzero(g.campo("accCor")) > 0
    pg, po = g.p.reshape(-1, CAMPOS), o.p.reshape(-1, CAMPOS)
    assert pg.shape == po.shape
    assert float(np.max(np.abs(pg[:, :2].astype(np.float64) - po[:, :2]))) < 1e-6
    assert erro_relativo(pg[:, 2:8], po[:, 2:8]) < 1e-4
    assert erro_relativo(pg[:, 8:], po[:, 8:]) < 1e-5


@pytest.mark.parametrize("motor", MOTORES)
def test_deterministico(lib_gpu, motor):
    """Two runs of the same scene produce identical bits."""
    def rodar():
        _, g = par("bolha", {"engine": motor})
        for _ in range(6):
            g.avancar(1 / 60, 3)
        return g.p.copy(), g.campo("q")
    p1, q1 = rodar()
    p2, q2 = rodar()
    assert np.array_equal(p1.view(np.uint32), p2.view(np.uint32))
    assert np.array_equal(q1.view(np.uint32), q2.view(np.uint32))


@pytest.mark.parametrize("motor", MOTORES)
def test_solvers_vivos_de_tamanhos_diferentes(lib_gpu, motor):
    """Two live tanks whose coarsest levels need different shared memory: the one created
    first (the larger coarsest level) still launches after the second one is created."""
    from tanque.cenarios import semear_retangulo_rapido

    def tanque(nx, ny, h):
        cena = Cena(nx, ny, h)
        g = SimulacaoGPU(cena, {"engine": motor, "tolerance": 1e-6, "iterations": 50})
        g.adicionar(semear_retangulo_rapido(3 * h, 3 * h, 0.5 * cena.largura, 0.6 * cena.altura, h), False)
        return g

    a = tanque(100, 60, 0.01)   # coarsest level 13x8
    b = tanque(300, 200, 0.004)  # coarsest level 10x7
    for _ in range(2):
        a.avancar(1 / 120, 2)
        b.avancar(1 / 120, 2)
    assert a.n > 0 and b.n > 0
    assert np.all(np.isfinite(a.campo("q"))) and np.all(np.isfinite(b.campo("q")))


def test_gravidade_em_execucao(lib_gpu):
    """sim.gravidade changed between frames (MotorCPU.gravidade, js/motor.js:96): the next
    substeps use it on the GPU exactly as in the oracle."""
    o, g = par("barragem")
    for s in (o, g):
        s.avancar(1 / 60 / 3, 1)
        s.gravidade = (3.5, -4.0)
    assert g.gravidade == (3.5, -4.0) == o.gravidade
    copiar_estado(o, g)
    o.avancar(1 / 60 / 3, 1)
    g.avancar(1 / 60 / 3, 1)
    for campo in ["accU", "accV", "tipo"]:
        assert np.array_equal(g.campo(campo), o.campo(campo)), campo
    assert erro_relativo(g.campo("u"), o.campo("u")) <= 1e-4
    assert erro_relativo(g.campo("v"), o.campo("v")) <= 1e-4
