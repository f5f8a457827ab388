"""Closed regions in the oracle's tolerance mode (CPU, no GPU).

Water sealed by walls (no air cell at pressure 0 around it) makes A singular on that region, and
the right-hand side's mean over it cannot be removed by any q.  In tolerance mode the solve
first removes each closed region's mean (over its water cells and the active bubbles inside)
and pins the region's smallest water cell at q = 0, so it converges; open regions are
untouched.  The grids here are built by hand:

    a tank with a solid frame, water in the lower part with air above (open), and inside the
    water a walled box of sealed water (closed), optionally holding an air pocket (a bubble).
"""
import numpy as np
import pytest

from oraculo import resolver_pressao_oraculo
from tanque import _abi
from tanque.constantes import AGUA, AR, SOLIDO

NX, NY = 48, 40


def grade(bolha: bool):
    """(tipo, rotulo): water rows 2..27, air above; a box of walls at columns 14..33, rows 6..19
    whose inside (16..31 x 8..17) is sealed water; with `bolha` an air pocket of label 5 at
    columns 20..23, rows 13..15 inside the box, and a second open-water bubble (label 7) in the
    open region."""
    tipo = np.full((NY, NX), AR, np.uint8)
    tipo[2:28, 2:NX - 2] = AGUA
    tipo[:2, :] = SOLIDO
    tipo[NY - 2:, :] = SOLIDO
    tipo[:, :2] = SOLIDO
    tipo[:, NX - 2:] = SOLIDO
    tipo[6:20, 14:34] = SOLIDO
    tipo[8:18, 16:32] = AGUA
    rotulo = np.zeros((NY, NX), np.uint32)
    rotulo[tipo == AR] = 1
    if bolha:
        tipo[13:16, 20:24] = AR
        rotulo[13:16, 20:24] = 5
        tipo[22:24, 6:9] = AR
        rotulo[22:24, 6:9] = 7
    return tipo, rotulo


def dados(bolha: bool, seed=3):
    rng = np.random.default_rng(seed)
    tipo, rotulo = grade(bolha)
    div = np.where(tipo == AGUA, rng.standard_normal(tipo.shape), 0).astype(np.float32)
    bol = None
    if bolha:
        rhs = np.zeros(4096, np.float32)
        rhs[5], rhs[7] = 3.5, -1.25
        bol = dict(rotulo=rotulo.ravel().copy(), rhs=rhs, y=np.zeros(4096, np.float32))
    return tipo, div, bol


RAIZ = 8 * NX + 16  # the box's smallest water cell: its root, pinned at q = 0


def residuo(tipo, div, q, bol, rhs_b, sem=None):
    """b - A q in FP64 over the unknowns (water rows; bubble rows when bol), with the given
    right-hand sides (numpy restatement of the operator, js/pressao-cpu.js:84-93, 318-328);
    `sem`: a water cell whose row is left out."""
    ny, nx = tipo.shape
    Q = q.reshape(ny, nx).astype(np.float64)
    rot = bol["rotulo"].reshape(ny, nx) if bol else None
    y = bol["y"].astype(np.float64) if bol else None
    rw, faces, soma = [], {}, {}
    for j in range(ny):
        for i in range(nx):
            if tipo[j, i] == AGUA:
                if sem == i + j * nx:
                    continue
                k, s = 0, 0.0
                for a, b in ((i - 1, j), (i + 1, j), (i, j - 1), (i, j + 1)):
                    if tipo[b, a] == SOLIDO:
                        continue
                    k += 1
                    if tipo[b, a] == AGUA:
                        s += Q[b, a]
                    elif bol is not None and rot[b, a] >= 2:
                        s += y[rot[b, a]]
                rw.append(-float(div[j, i]) - (k * Q[j, i] - s))
            elif tipo[j, i] == AR and bol is not None and rot[j, i] >= 2:
                r = int(rot[j, i])
                for a, b in ((i - 1, j), (i + 1, j), (i, j - 1), (i, j + 1)):
                    if tipo[b, a] == AGUA:
                        faces[r] = faces.get(r, 0) + 1
                        soma[r] = soma.get(r, 0.0) + Q[b, a]
    rb = [float(rhs_b[r]) - (faces[r] * y[r] - soma[r]) for r in faces]
    return np.array(rw + rb)


def projetado(tipo, div, bol):
    """The projection restated in numpy: the box's water cells and bubble 5 lose their mean."""
    caixa = np.zeros(tipo.shape, bool)
    caixa[8:18, 16:32] = True
    agua = caixa & (tipo == AGUA)
    b = [-div[agua].astype(np.float64)]
    if bol is not None:
        b.append(np.array([float(bol["rhs"][5])]))
    b = np.concatenate(b)
    m = b.mean()
    d2 = div.copy()
    d2[agua] = (div[agua].astype(np.float64) + m).astype(np.float32)
    rhs2 = bol["rhs"].copy() if bol is not None else None
    if bol is not None:
        rhs2[5] = np.float32(float(bol["rhs"][5]) - m)
    return d2, rhs2


@pytest.mark.parametrize("bolha", [False, True], ids=["agua-selada", "selada-com-bolha"])
@pytest.mark.parametrize("precond", [_abi.TQ_PRECOND_REFERENCE, _abi.TQ_PRECOND_BLOCK, _abi.TQ_PRECOND_BLOCK_1],
                         ids=["ref", "bloco", "bloco1"])
def test_regiao_fechada_converge(bolha, precond):
    tipo, div, bol = dados(bolha)
    q = np.zeros(tipo.size, np.float32)
    b = {k: v.copy() for k, v in bol.items()} if bol else None
    info = {}
    resolver_pressao_oraculo(tipo, div, q, 1000, 1e-6, b, precond=precond, info=info)
    assert info["converged"] == 1 and info["closed_regions"] == 1, info
    assert info["iterations"] < 200
    assert 0 <= info["true_residual"] <= 1e-6 * info["residual0"]
    assert q[RAIZ] == 0.0  # the region's root (its smallest water cell) is pinned at 0
    # the solution solves the projected system: its residual, recomputed here from the returned
    # float q, is within the tolerance of the projected r0 plus the float rounding of q (about
    # 1e-7 |A| |q| per cell); the pinned row is not an unknown of the solve, and holds by itself
    d2, rhs2 = projetado(tipo, div, bol)
    r = residuo(tipo, d2, q, b, rhs2)
    r0 = residuo(tipo, d2, np.zeros_like(q), dict(b, y=bol["y"]) if bol else None, rhs2, sem=RAIZ)
    assert abs(np.linalg.norm(r0) - info["residual0"]) <= 1e-6 * info["residual0"]
    piso = 1e-7 * 8 * float(np.linalg.norm(q))
    assert np.linalg.norm(r) <= 1e-6 * np.linalg.norm(r0) + piso


def test_regioes_abertas_intocadas():
    """With the box's water open to the air above (a gap in its lid), nothing is projected and
    the solve is the unprojected one."""
    tipo, div, _ = dados(False)
    tipo[6:8, 24:26] = AR  # the gap: the box's water faces air at pressure 0
    q = np.zeros(tipo.size, np.float32)
    info = {}
    resolver_pressao_oraculo(tipo, div, q, 1000, 1e-6, None, precond=_abi.TQ_PRECOND_REFERENCE, info=info)
    assert info["converged"] == 1 and info["closed_regions"] == 0
    r = residuo(tipo, div, q, None, None)
    r0 = residuo(tipo, div, np.zeros_like(q), None, None)
    assert np.linalg.norm(r) <= 1e-6 * np.linalg.norm(r0) + 1e-7 * 8 * float(np.linalg.norm(q))


def test_sem_projecao_nao_converge_e_contagem_fixa_intocada():
    """Without the projection the sealed system has no solution: the fixed-count mode (the
    reference's) runs its iterations on the unprojected right-hand side, whose residual cannot
    fall below the box's mean component."""
    tipo, div, _ = dados(False)
    q = np.zeros(tipo.size, np.float32)
    info = {}
    resolver_pressao_oraculo(tipo, div, q, 300, 0.0, None, precond=_abi.TQ_PRECOND_REFERENCE, info=info)
    assert info["closed_regions"] == 0
    caixa = np.zeros(tipo.shape, bool)
    caixa[8:18, 16:32] = True
    media = float(-div[caixa & (tipo == AGUA)].astype(np.float64).mean())
    piso = abs(media) * np.sqrt(np.count_nonzero(caixa & (tipo == AGUA)))
    r = residuo(tipo, div, q, None, None)
    assert np.linalg.norm(r) >= 0.99 * piso > 0
