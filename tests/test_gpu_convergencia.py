"""Tolerance mode, the block preconditioner, solve statistics and CUDA-graph frames on the GPU.

Tolerance mode (tq_solve_pressure, tq_options.tolerance > 0) keeps q in FP64 during the solve
and stops on the true residual; the oracle does the same on the CPU.  Both preconditioners
solve the same system, so to the tolerance they give the same q; the parity tolerances are the
ones of the reference-preconditioner tests (1e-4 relative on q).
"""
import numpy as np
import pytest

from estado import CENAS, erro_relativo
from oraculo import CenaOraculo, SimulacaoOraculo, resolver_pressao_oraculo
from tanque import Cena, SimulacaoGPU, _abi, resolver_pressao
from tanque.constantes import CAMPOS

pytestmark = pytest.mark.gpu

OPC_FIXO = {"p2g_mode": _abi.TQ_P2G_FIXED}
MOTORES = [pytest.param(_abi.TQ_ENGINE_PLAIN, id="plain"), pytest.param(_abi.TQ_ENGINE_FUSED, id="fused")]
PRECS = [pytest.param(_abi.TQ_PREC_FP32, id="fp32"), pytest.param(_abi.TQ_PREC_FP16, id="fp16")]


def problema(nome, passos=6):
    cena_o, agua = CENAS[nome](CenaOraculo)
    o = SimulacaoOraculo(cena_o, OPC_FIXO)
    o.adicionar(agua, False)
    for _ in range(passos):
        o.avancar(1 / 60, 2)
    nx, ny = o.nx, o.ny
    bol = dict(rotulo=o.campo("rotulo"), rhs=o.campo("rhsBolha"), y=o.campo("yBolha"))
    return o.campo("tipo").reshape(ny, nx), o.campo("div").reshape(ny, nx), bol


@pytest.mark.parametrize("motor", MOTORES)
@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("precond", [_abi.TQ_PRECOND_REFERENCE, _abi.TQ_PRECOND_BLOCK, _abi.TQ_PRECOND_BLOCK_1],
                         ids=["referencia", "bloco", "bloco1"])
@pytest.mark.parametrize("nome", ["bolha", "copo"])
def test_tolerancia_verdadeira(lib_gpu, nome, precond, prec, motor):
    """Both engines stop on the true FP64 residual; q, y and the iteration count agree with the
    oracle's run of the same preconditioner."""
    tipo, div, bol = problema(nome)
    q_o = np.zeros(tipo.size, np.float32)
    q_g = q_o.copy()
    b_o = {k: v.copy() for k, v in bol.items()}
    b_g = {k: v.copy() for k, v in bol.items()}
    i_o, i_g = {}, {}
    n_o = resolver_pressao_oraculo(tipo, div, q_o, 400, 1e-6, b_o, precond=precond, info=i_o)
    n_g = resolver_pressao(tipo, div, q_g, 400, 1e-6, b_g, precisao=prec, motor=motor, precond=precond, info=i_g)
    assert i_o["converged"] == 1 and i_g["converged"] == 1
    assert 0 <= i_g["true_residual"] <= 1e-6 * i_g["residual0"]
    assert abs(i_g["residual0"] - i_o["residual0"]) <= 1e-6 * i_o["residual0"]
    assert i_g["iterations"] == len(n_g) - 1
    assert erro_relativo(q_g, q_o) < 1e-4
    ativos = np.nonzero(b_o["y"] != bol["y"])[0]
    if ativos.size:
        assert erro_relativo(b_g["y"][ativos], b_o["y"][ativos]) < 1e-3
    # FP32 arithmetic and 16-bit V-cycle storage change the iterates a little, not the rate
    folga = 3 if prec == _abi.TQ_PREC_FP32 else 0.25 * len(n_o)
    assert len(n_g) <= len(n_o) + folga


def labirinto_sintetico(nx=210, ny=150, seed=7):
    """A pressure problem with walls 2 cells thick (thinner than a cell from the third level
    down, where the block preconditioner's face masks close faces between water cells) and
    enclosed air pockets with labels >= 2."""
    from tanque.constantes import AGUA, AR, SOLIDO
    rng = np.random.default_rng(seed)
    tipo = np.full((ny, nx), AGUA, np.uint8)
    tipo[int(0.8 * ny):, :] = AR
    for x0 in range(12, nx - 6, 14):  # vertical walls with a gap alternating bottom / top
        tipo[2:ny - 2, x0:x0 + 2] = SOLIDO
        g = 4 if (x0 // 14) % 2 else int(0.8 * ny) - 10
        tipo[g:g + 6, x0:x0 + 2] = AGUA if g < int(0.8 * ny) else AR
    tipo[:2, :] = tipo[-2:, :] = SOLIDO
    tipo[:, :2] = tipo[:, -2:] = SOLIDO
    rot = np.zeros((ny, nx), np.uint32)
    rot[tipo == AR] = 1
    jj, ii = np.mgrid[0:ny, 0:nx]
    for k, (cx, cy, r) in enumerate([(30, 40, 5), (75, 60, 7), (130, 30, 4), (180, 80, 6)]):
        bolha = ((ii - cx) ** 2 + (jj - cy) ** 2 < r * r) & (tipo == AGUA)
        tipo[bolha] = AR
        rot[bolha] = 2 + k
    div = rng.standard_normal((ny, nx)).astype(np.float32)
    div[tipo != AGUA] = 0
    rhs = np.zeros(4096, np.float32)
    rhs[2:6] = rng.standard_normal(4).astype(np.float32)
    return tipo, div, dict(rotulo=rot.ravel(), rhs=rhs, y=np.zeros(4096, np.float32))


@pytest.mark.parametrize("motor", MOTORES)
@pytest.mark.parametrize("prec", PRECS)
def test_bloco_paredes_finas(lib_gpu, prec, motor):
    """The block preconditioner's coarse masks on thin walls: the GPU solve matches the oracle's
    (q, y) and needs about as many iterations (a smoother that summed across a closed face
    would diverge or crawl)."""
    tipo, div, bol = labirinto_sintetico()
    q_o = np.zeros(tipo.size, np.float32)
    q_g = q_o.copy()
    b_o = {k: v.copy() for k, v in bol.items()}
    b_g = {k: v.copy() for k, v in bol.items()}
    i_o, i_g = {}, {}
    resolver_pressao_oraculo(tipo, div, q_o, 600, 1e-6, b_o, precond=_abi.TQ_PRECOND_BLOCK, info=i_o)
    resolver_pressao(tipo, div, q_g, 600, 1e-6, b_g, precisao=prec, motor=motor, precond=_abi.TQ_PRECOND_BLOCK,
                     info=i_g)
    assert i_o["converged"] == 1 and i_g["converged"] == 1
    assert erro_relativo(q_g, q_o) < 1e-4
    assert erro_relativo(b_g["y"][2:6], b_o["y"][2:6]) < 1e-3
    folga = 3 if prec == _abi.TQ_PREC_FP32 else 0.25 * i_o["iterations"]
    assert i_g["iterations"] <= i_o["iterations"] + folga


@pytest.mark.parametrize("motor", MOTORES)
def test_bloco_converge_mais_depressa(lib_gpu, motor):
    """On a scene with trapped air the block preconditioner needs fewer iterations."""
    tipo, div, bol = problema("bolha")
    its = {}
    for pc in (_abi.TQ_PRECOND_REFERENCE, _abi.TQ_PRECOND_BLOCK):
        q = np.zeros(tipo.size, np.float32)
        info = {}
        resolver_pressao(tipo, div, q, 400, 1e-6, {k: v.copy() for k, v in bol.items()}, motor=motor, precond=pc,
                         info=info)
        its[pc] = info["iterations"]
    assert its[_abi.TQ_PRECOND_BLOCK] <= its[_abi.TQ_PRECOND_REFERENCE]


@pytest.mark.parametrize("motor", MOTORES)
def test_cap_relatado(lib_gpu, motor):
    tipo, div, bol = problema("copo")
    q = np.zeros(tipo.size, np.float32)
    info = {}
    n = resolver_pressao(tipo, div, q, 4, 1e-12, {k: v.copy() for k, v in bol.items()}, motor=motor, info=info)
    assert len(n) == 5 and info["iterations"] == 4
    assert info["converged"] == 0 and info["true_residual"] > 1e-12 * info["residual0"]


@pytest.mark.parametrize("motor", MOTORES)
def test_estatisticas_de_solves(lib_gpu, motor):
    cena_o, agua = CENAS["bolha"](CenaOraculo)
    cena = Cena(cena_o.nx, cena_o.ny, cena_o.h)
    cena.sdf[:] = cena_o.sdf
    g = SimulacaoGPU(cena, {"engine": motor, "tolerance": 1e-6, "iterations": 300, "precision": _abi.TQ_PREC_FP16,
                            "preconditioner": _abi.TQ_PRECOND_BLOCK})
    g.adicionar(agua, False)
    g.avancar(1 / 60, 3)
    assert g.escalar(_abi.TQ_SCALAR_SOLVES) == 3
    assert g.escalar(_abi.TQ_SCALAR_SOLVES_CAPPED) == 0
    assert 0 < g.escalar(_abi.TQ_SCALAR_SOLVE_MAX_REL) <= 1e-6
    assert g.escalar(_abi.TQ_SCALAR_PCG_CONVERGED) == 1
    assert g.escalar(_abi.TQ_SCALAR_SOLVE_ITERS) >= 3
    assert g.escalar(_abi.TQ_SCALAR_PCG_TRUE_RES) <= 1e-6 * g.escalar(_abi.TQ_SCALAR_PCG_RES0)
    g.definirEscalar(_abi.TQ_SCALAR_SOLVES, 0)
    assert g.escalar(_abi.TQ_SCALAR_SOLVES) == 0 and g.escalar(_abi.TQ_SCALAR_SOLVE_ITERS) == 0


@pytest.mark.parametrize("motor", MOTORES)
def test_substeps_bloco_paridade(lib_gpu, motor):
    """Whole frames with the block preconditioner against the oracle's, from the same state:
    integers bit-exact, q/u/v to the parity tolerances."""
    from estado import INTEIROS, copiar_estado
    opc = {"tolerance": 1e-6, "iterations": 300, "preconditioner": _abi.TQ_PRECOND_BLOCK}
    cena_o, agua = CENAS["bolha"](CenaOraculo)
    cena = Cena(cena_o.nx, cena_o.ny, cena_o.h)
    cena.sdf[:] = cena_o.sdf
    o = SimulacaoOraculo(cena_o, dict(OPC_FIXO, **opc))
    g = SimulacaoGPU(cena, dict(opc, engine=motor))
    o.adicionar(agua, False)
    for quadro in range(4):
        copiar_estado(o, g)
        o.avancar(1 / 60 / 3, 1)
        g.avancar(1 / 60 / 3, 1)
        for campo in INTEIROS:
            assert np.array_equal(g.campo(campo), o.campo(campo)), f"{quadro}: {campo}"
        for campo in ["q", "u", "v"]:
            assert erro_relativo(g.campo(campo), o.campo(campo)) <= 1e-4, f"{quadro}: {campo}"
        pg, po = g.p.reshape(-1, CAMPOS), o.p.reshape(-1, CAMPOS)
        assert float(np.max(np.abs(pg[:, :2].astype(np.float64) - po[:, :2]))) < 1e-6


@pytest.mark.parametrize("prec", PRECS)
def test_grafo_bit_identico(lib_gpu, prec):
    """A frame replayed from a CUDA graph (tq_advance_graph) gives the bits of tq_advance."""
    def rodar(grafo):
        cena_o, agua = CENAS["bolha"](CenaOraculo)
        cena = Cena(cena_o.nx, cena_o.ny, cena_o.h)
        cena.sdf[:] = cena_o.sdf
        g = SimulacaoGPU(cena, {"engine": _abi.TQ_ENGINE_FUSED, "tolerance": 1e-6, "iterations": 300, "precision": prec,
                                "preconditioner": _abi.TQ_PRECOND_BLOCK})
        g.adicionar(agua, False)
        for _ in range(4):
            if grafo:
                g.avancarGrafo(1 / 60, 4)
            else:
                g.avancar(1 / 60, 4)
        return g.p.copy(), g.campo("q"), g.escalar(_abi.TQ_SCALAR_SOLVES)
    p1, q1, s1 = rodar(False)
    p2, q2, s2 = rodar(True)
    assert s1 == s2 == 16
    assert np.array_equal(p1.view(np.uint32), p2.view(np.uint32))
    assert np.array_equal(q1.view(np.uint32), q2.view(np.uint32))


def test_grafo_plano_com_tolerancia_recusado(lib_gpu):
    cena = Cena(40, 30, 0.01)
    g = SimulacaoGPU(cena, {"engine": _abi.TQ_ENGINE_PLAIN, "tolerance": 1e-6, "iterations": 50})
    with pytest.raises(_abi.ErroTanque) as e:
        g.avancarGrafo(1 / 60, 2)
    assert e.value.status == _abi.TQ_E_STATE


@pytest.mark.parametrize("precond", [_abi.TQ_PRECOND_REFERENCE, _abi.TQ_PRECOND_BLOCK], ids=["referencia", "bloco"])
@pytest.mark.parametrize("motor", MOTORES)
@pytest.mark.parametrize("nome", ["bolha", "copo"])
def test_solve_nao_herda_o_anterior(lib_gpu, nome, motor, precond):
    """A handle that has solved before gives the same substep, bit for bit, as a fresh handle
    given the same state: nothing of a solve (its stop flag, its bubble sums) reaches the next.
    A scene with trapped air and the cup scene, every solve to the tolerance."""
    from estado import copiar_estado
    opc = {"tolerance": 1e-6, "iterations": 1000, "precision": _abi.TQ_PREC_FP32, "engine": motor,
           "preconditioner": precond}
    cena, agua = CENAS[nome](Cena)
    usada = SimulacaoGPU(cena, opc)
    usada.adicionar(agua, False)
    for _ in range(3):
        usada.avancar(1 / 120, 2)
    nova = SimulacaoGPU(cena, opc)
    copiar_estado(usada, nova)
    for s in (usada, nova):
        s.subpasso(1 / 240)
        assert s.escalar(_abi.TQ_SCALAR_PCG_CONVERGED) == 1
    if nome == "bolha":  # trapped air: bubble rows in the solve
        assert int(np.count_nonzero(usada.campo("vivo"))) >= 1
    for campo in ["q", "u", "v", "pressaoBolha"]:
        assert np.array_equal(usada.campo(campo), nova.campo(campo)), campo
    assert usada.escalar(_abi.TQ_SCALAR_PCG_ITERS) == nova.escalar(_abi.TQ_SCALAR_PCG_ITERS)
