"""The oracle's tolerance mode and its block preconditioner (CPU, no GPU).

Tolerance mode keeps q in double during the solve and stops on the true residual
||b - A q|| <= tol ||r0||; the block preconditioner (TQ_PRECOND_BLOCK) replaces the reference's
bubble spread/gather with a Jacobi step on the bubble rows and builds coarse neighbour masks
from the fine faces.  Both solve the same system: to the tolerance they give the same q.
"""
import numpy as np
import pytest

from estado import CENAS, erro_relativo
from oraculo import CenaOraculo, SimulacaoOraculo, resolver_pressao_oraculo
from tanque import _abi
from tanque.constantes import AGUA

OPC_FIXO = {"p2g_mode": _abi.TQ_P2G_FIXED}


def problema(nome, passos=6):
    cena_o, agua = CENAS[nome](CenaOraculo)
    o = SimulacaoOraculo(cena_o, OPC_FIXO)
    o.adicionar(agua, False)
    for _ in range(passos):
        o.avancar(1 / 60, 2)
    nx, ny = o.nx, o.ny
    bol = dict(rotulo=o.campo("rotulo"), rhs=o.campo("rhsBolha"), y=o.campo("yBolha"))
    return o.campo("tipo").reshape(ny, nx), o.campo("div").reshape(ny, nx), bol


def resolver(tipo, div, bol, precond, iters=400, tol=1e-6):
    q = np.zeros(tipo.size, np.float32)
    b = {k: v.copy() for k, v in bol.items()}
    info = {}
    n = resolver_pressao_oraculo(tipo, div, q, iters, tol, b, precond=precond, info=info)
    return q, b, n, info


@pytest.mark.parametrize("bloco", [_abi.TQ_PRECOND_BLOCK, _abi.TQ_PRECOND_BLOCK_1], ids=["bloco", "bloco1"])
@pytest.mark.parametrize("nome", ["bolha", "copo"])
def test_bloco_e_referencia_dao_o_mesmo_q(nome, bloco):
    tipo, div, bol = problema(nome)
    q_r, b_r, n_r, i_r = resolver(tipo, div, bol, _abi.TQ_PRECOND_REFERENCE)
    q_b, b_b, n_b, i_b = resolver(tipo, div, bol, bloco)
    for i in (i_r, i_b):
        assert i["converged"] == 1
        assert 0 <= i["true_residual"] <= 1e-6 * i["residual0"]
        assert i["iterations"] == len(n_r if i is i_r else n_b) - 1
    # two solutions of the same system to 1e-6 of ||r0||: q agrees far below the parity
    # tolerances of the GPU tests
    assert erro_relativo(q_b, q_r) < 1e-5
    ativos = np.nonzero(b_r["y"] != bol["y"])[0]
    if ativos.size:
        assert erro_relativo(b_b["y"][ativos], b_r["y"][ativos]) < 1e-5


def test_verdade_igual_ao_residuo_recalculado():
    """The reported true residual is ||b - A q|| of the FP64 iterate: recomputed here in numpy
    from the returned float q it agrees to the float rounding of q (no bubbles)."""
    tipo, div, _ = problema("barragem")
    sem_bolhas = {"rotulo": np.zeros(tipo.size, np.uint32), "rhs": np.zeros(4096, np.float32),
                  "y": np.zeros(4096, np.float32)}
    q, _, n, info = resolver(tipo, div, sem_bolhas, _abi.TQ_PRECOND_REFERENCE)
    ny, nx = tipo.shape
    Q = q.reshape(ny, nx).astype(np.float64)
    agua = tipo == AGUA
    livre = tipo != 0
    r = np.zeros_like(Q)
    for j in range(ny):
        for i in range(nx):
            if not agua[j, i]:
                continue
            k, s = 0, 0.0
            for a, b in ((i - 1, j), (i + 1, j), (i, j - 1), (i, j + 1)):
                if 0 <= a < nx and 0 <= b < ny and livre[b, a]:
                    k += 1
                    s += Q[b, a] if agua[b, a] else 0.0
            r[j, i] = -float(div[j, i]) - (k * Q[j, i] - s)
    rv = float(np.sqrt(np.sum(r[agua] ** 2)))
    assert info["converged"] == 1
    # float rounding of q: about 1e-7 |A| |q| per cell on top of the FP64 iterate's residual
    piso = 1e-7 * 8 * float(np.sqrt(np.sum(Q[agua] ** 2)))
    assert abs(rv - info["true_residual"]) <= piso + 1e-9


def test_cap_sem_convergir():
    tipo, div, bol = problema("copo")
    _, _, n, info = resolver(tipo, div, bol, _abi.TQ_PRECOND_REFERENCE, iters=4, tol=1e-12)
    assert info["iterations"] == 4 and len(n) == 5
    assert info["converged"] == 0
    assert info["true_residual"] > 1e-12 * info["residual0"]


def test_iteracoes_fixas_inalteradas():
    """tolerance = 0 (the reference's fixed count) ignores the new machinery: no true residual."""
    tipo, div, bol = problema("copo")
    _, _, n, info = resolver(tipo, div, bol, _abi.TQ_PRECOND_REFERENCE, iters=3, tol=0.0)
    assert len(n) == 4 and info["true_residual"] == -1.0 and info["converged"] == 0


def test_estatisticas_da_simulacao():
    cena_o, agua = CENAS["bolha"](CenaOraculo)
    o = SimulacaoOraculo(cena_o, dict(OPC_FIXO, tolerance=1e-6, iterations=300, preconditioner=_abi.TQ_PRECOND_BLOCK))
    o.adicionar(agua, False)
    o.avancar(1 / 60, 3)
    assert o.escalar(_abi.TQ_SCALAR_SOLVES) == 3
    assert o.escalar(_abi.TQ_SCALAR_SOLVES_CAPPED) == 0
    assert 0 < o.escalar(_abi.TQ_SCALAR_SOLVE_MAX_REL) <= 1e-6
    assert o.escalar(_abi.TQ_SCALAR_PCG_CONVERGED) == 1
    o.definirEscalar(_abi.TQ_SCALAR_SOLVES, 0)
    assert o.escalar(_abi.TQ_SCALAR_SOLVES) == 0 and o.escalar(_abi.TQ_SCALAR_SOLVE_ITERS) == 0
