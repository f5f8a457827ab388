"""Batched tanks laid out as tank atlases (tanque.lote), on the CPU with the oracle.

- Layout: the tanks stand side by side, top-aligned, with MARGEM wall columns either side of
  their own frames; the rest of the atlas is wall; the grouping keeps each atlas's coarsest
  multigrid level within its limit and places every tank once.
- Independence: one substep of a 3-tank atlas against each tank cut out of the atlas (its
  columns with their margins, as a scene of its own) run alone, compared on the tank's own
  columns.  With h = 1/128 the
  offsets between the two are exact in float32, so every field computed before the pressure
  solve is equal bit for bit on the tank's columns: particle-to-grid sums, flags, counts,
  density, phase, curvature, air pressure, divergence.  The pressure solve shares its
  scalars across the atlas, so q, u, v agree to the solve's accuracy (1e-3 relative; both
  solves stop at ||r|| <= 1e-6 ||r0||), and the air labels agree up to renumbering.
"""
import numpy as np
import pytest

from oraculo import SimulacaoOraculo
from tanque import Cena, _abi
from tanque.constantes import CAMPOS, MOLDURA, SDF_MAX
from tanque.lote import MARGEM, Lote, agrupar, gerar_tanques, largura_atlas, montar_atlas, niveis, recortar

H = 1 / 128
SOLVE = {"tolerance": 1e-6, "iterations": 200, "p2g_mode": _abi.TQ_P2G_FIXED}


def _tanques(n=3, s=9):
    return gerar_tanques(n=n, s=s, h=H, largura=(30, 60), altura=(24, 40))


def test_gerador_da_carga_de_256_tanques():
    t = gerar_tanques()
    w = np.array([x["nx"] for x in t])
    a = np.array([x["ny"] for x in t])
    assert len(t) == 256
    assert w.min() >= 64 and w.max() <= 512 and a.min() >= 64 and a.max() <= 320
    assert 8.0e6 < int((w * a).sum()) < 9.6e6  # about 8.8 M cells
    for x in t:
        x0, y0, x1, y1 = x["agua"]
        frac = (x1 - x0) * (y1 - y0) / ((x["nx"] - 2 * MOLDURA) * (x["ny"] - 2 * MOLDURA) * 0.003 ** 2)
        assert 0.19 <= frac <= 0.71
    assert t == gerar_tanques()  # seeded


def test_agrupar_respeita_o_nivel_grosso():
    t = gerar_tanques()
    grupos = agrupar(t, 12000)
    assert sorted(k for g in grupos for k in g) == list(range(256))
    for g in grupos:
        ts = [t[k] for k in g]
        gx, gy = niveis(largura_atlas(ts), max(x["ny"] for x in ts))[-1]
        assert gx * gy <= 12000 or len(g) == 1


def test_montar_atlas():
    t = _tanques()
    at = montar_atlas(Cena, t, H)
    c = at["cena"]
    assert c.nx == sum(x["nx"] + 2 * MARGEM for x in t) and c.ny == max(x["ny"] for x in t)
    m = np.asarray(c.sdf).reshape(c.ny * c.r, c.nx * c.r)
    for k, x in enumerate(t):
        x0, y0 = at["x0"][k], at["y0"][k]
        assert y0 == c.ny - x["ny"]
        # the tank's own mask, margins and the rows below it are wall
        assert np.all(m[:, (x0 - MARGEM) * c.r:x0 * c.r] == -SDF_MAX)
        assert np.all(m[:y0 * c.r, x0 * c.r:(x0 + x["nx"]) * c.r] == -SDF_MAX)
        propria = Cena(x["nx"], x["ny"], H)
        for tr in x["tracos"]:
            propria.tracar(tr["x0"], tr["y0"], tr["x1"], tr["y1"], tr["raio"])
        assert np.array_equal(m[y0 * c.r:, x0 * c.r:(x0 + x["nx"]) * c.r],
                              np.asarray(propria.sdf).reshape(x["ny"] * c.r, x["nx"] * c.r))
    p = at["particulas"].reshape(-1, CAMPOS)
    assert len(p) == sum(at["semeadas"])


def _rotulos_equivalentes(a, b):
    """Equal up to a renumbering of the labels >= 2 (0: not air, 1: atmosphere)."""
    assert np.array_equal(a < 2, b < 2) and np.array_equal(a[a < 2], b[a < 2])
    pares = set(zip(a[a >= 2].tolist(), b[a >= 2].tolist()))
    assert len({x for x, _ in pares}) == len(pares) == len({y for _, y in pares})


@pytest.mark.parametrize("k", [0, 1, 2])
def test_tanque_independente_no_atlas(k):
    t = _tanques()
    at = montar_atlas(Cena, t, H)
    nx, ny = at["cena"].nx, at["cena"].ny
    x0 = at["x0"][k]
    a, b = x0 - MARGEM, x0 + t[k]["nx"] + MARGEM
    corte = recortar(Cena, at["cena"], a, b)
    inicio = sum(at["semeadas"][:k])
    p = at["particulas"].reshape(-1, CAMPOS)[inicio:inicio + at["semeadas"][k]].copy()
    p[:, 0] -= np.float32(a * H)  # exact: a * H is a multiple of 2^-7
    so = SimulacaoOraculo(at["cena"], dict(SOLVE))
    sk = SimulacaoOraculo(corte, dict(SOLVE))
    so.adicionar(at["particulas"], False)
    sk.adicionar(p.ravel(), False)
    for s in (so, sk):
        s.avancar(1 / 240, 1)
    nk = b - a
    # compared on the tank's own columns (frame included): in the atlas x0 .. x0 + w, in the cut
    # MARGEM .. MARGEM + w (the cut's outermost columns are a domain edge, the atlas's are not)
    w = t[k]["nx"]
    A0, K0 = x0, MARGEM
    celula = lambda s, nome: np.asarray(s.campo(nome)).reshape(s.ny, s.nx)  # noqa: E731
    for nome in ["tipo", "contagemCelula", "densidade", "fase", "curvatura", "qAr", "div"]:
        A = celula(so, nome)[:, A0:A0 + w]
        B = celula(sk, nome)[:, K0:K0 + w]
        assert np.array_equal(A.view(np.uint32) if A.dtype == np.float32 else A,
                              B.view(np.uint32) if B.dtype == np.float32 else B), nome
    # fixed-point sums, (value, weight) pairs per cell / face
    assert np.array_equal(np.asarray(so.campo("accCel")).reshape(ny, nx, 2)[:, A0:A0 + w],
                          np.asarray(sk.campo("accCel")).reshape(ny, nk, 2)[:, K0:K0 + w])
    assert np.array_equal(np.asarray(so.campo("accU")).reshape(ny, nx + 1, 2)[:, A0:A0 + w + 1],
                          np.asarray(sk.campo("accU")).reshape(ny, nk + 1, 2)[:, K0:K0 + w + 1])
    assert np.array_equal(np.asarray(so.campo("accV")).reshape(ny + 1, nx, 2)[:, A0:A0 + w],
                          np.asarray(sk.campo("accV")).reshape(ny + 1, nk, 2)[:, K0:K0 + w])
    _rotulos_equivalentes(celula(so, "rotulo")[:, A0:A0 + w], celula(sk, "rotulo")[:, K0:K0 + w])
    qa = celula(so, "q")[:, A0:A0 + w].astype(np.float64)
    qb = celula(sk, "q")[:, K0:K0 + w].astype(np.float64)
    assert np.max(np.abs(qa - qb)) <= 1e-3 * max(np.max(np.abs(qb)), 1e-30)
    ua = np.asarray(so.campo("u")).reshape(ny, nx + 1)[:, A0:A0 + w + 1].astype(np.float64)
    ub = np.asarray(sk.campo("u")).reshape(ny, nk + 1)[:, K0:K0 + w + 1].astype(np.float64)
    assert np.max(np.abs(ua - ub)) <= 1e-3 * max(np.max(np.abs(ub)), 1e-30)


def test_lote_avanca_e_separa_os_tanques():
    t = _tanques(n=5, s=3)
    lote = Lote(lambda c, o: SimulacaoOraculo(c, o), Cena, t, H, dict(SOLVE), limite_grosso=200)
    assert len(lote.atlas) >= 2  # a small coarse limit splits the batch
    n0 = [len(lote.particulas(k)) for k in range(5)]
    lote.avancar(1 / 240, 2)
    for k in range(5):
        q = lote.particulas(k)
        assert len(q) == n0[k]  # no particle leaves its tank
        assert np.all(q[:, 0] > 0) and np.all(q[:, 0] < t[k]["nx"] * H)
        assert lote.campo(k, "tipo").shape == (t[k]["ny"], t[k]["nx"])


@pytest.mark.parametrize("partes", [1, 2, 3, 8])
def test_repartir_entre_gpus(partes):
    from tanque.lote import repartir
    t = gerar_tanques()
    grupos = repartir(t, partes)
    assert sorted(k for g in grupos for k in g) == list(range(256))
    cargas = [sum(t[k]["nx"] * t[k]["ny"] for k in g) for g in grupos]
    maior = max(x["nx"] * x["ny"] for x in t)
    assert max(cargas) - min(cargas) <= maior  # LPT: within one tank of balance


def test_autoajuste_escolhe_o_mais_rapido():
    """tanque.lote.autoajustar builds the batch per candidate grouping, times its frames and keeps
    the fastest (here a fake simulation whose frame costs a fixed time per atlas plus a time per
    atlas cell: the candidates trade atlas count against padding)."""
    import time as _t

    from tanque import Cena
    from tanque.lote import Lote, autoajustar, gerar_tanques

    class Falsa:
        def __init__(self, cena, opcoes):
            self.celulas = cena.nx * cena.ny

        def adicionar(self, p, checar):
            return 0

        def avancar(self, dt, sub):
            _t.sleep(0.004 + self.celulas * 2e-8)

        def sincronizar(self):
            pass

    t = gerar_tanques(n=24, s=9, h=1 / 128, largura=(40, 160), altura=(30, 120))
    melhor, tempos = autoajustar(Falsa, Cena, t, 1 / 128, {}, 1 / 60, 2, candidatos=(200, 800, 3200))
    assert set(tempos) == {200, 800, 3200}
    assert melhor == min(tempos, key=tempos.get)
    grupos = {lim: len(Lote(Falsa, Cena, t, 1 / 128, {}, limite_grosso=lim).atlas) for lim in tempos}
    assert grupos[200] >= grupos[800] >= grupos[3200]  # a larger limit makes fewer atlases


@pytest.mark.parametrize("total", [148, 60, 9, 7])
def test_repartir_ctas(total):
    """The SMs split between atlases in proportion to their cells, each at least the minimum
    (or total // atlases when that is smaller), the sum within the SM count; no split with
    more atlases than SMs."""
    from tanque.lote import repartir_ctas
    pesos = [3_000_000, 2_900_000, 740_000, 700_000, 500_000, 170_000, 160_000, 150_000]
    c = repartir_ctas(pesos, total)
    if total < len(pesos):
        assert c is None
        return
    assert len(c) == len(pesos) and sum(c) <= total
    assert min(c) >= max(1, min(4, total // len(pesos)))
    if total >= 60:
        assert c == sorted(c, reverse=True)  # larger atlases, more CTAs
        assert c[0] >= int(total * pesos[0] / sum(pesos)) - len(pesos)
    assert repartir_ctas([], total) == []



def test_pesar_por_iteracoes():
    """tanque.lote.pesar_por_iteracoes: the SM split by cells, then by cells x the solves' mean
    iterations (read from the handles' solve records after a frame), each timed over a frame;
    the faster is kept.  Fake simulations whose solves take more iterations on smaller atlases,
    a frame lasting as long as the slowest atlas (cells x iterations / CTAs), gain from it."""
    import time as _t

    from tanque import Cena, _abi
    from tanque.lote import Lote, pesar_por_iteracoes

    class Falsa:
        def __init__(self, cena, opcoes):
            self.celulas = cena.nx * cena.ny
            self.iters = 2e5 / self.celulas
            self.ctas = opcoes.get("fused_ctas", 148)
            self.ms, self.solves, self.acum = 0.0, 0, 0.0

        def adicionar(self, p, checar):
            return 0

        def lancarGrafo(self, dt, sub):
            self.ms = 1e-3 * self.celulas * self.iters / self.ctas
            self.solves += sub
            self.acum += sub * self.iters

        def sincronizar(self):
            pass

        def definirEscalar(self, qual, v):
            assert qual == _abi.TQ_SCALAR_SOLVES and v == 0
            self.solves, self.acum = 0, 0.0

        def escalar(self, qual):
            return {_abi.TQ_SCALAR_SOLVES: self.solves, _abi.TQ_SCALAR_SOLVE_ITERS: self.acum}[qual]

        def fechar(self):
            pass

    orig = Lote.avancar

    def avancar(self, dt, sub=1, grafo=False):
        orig(self, dt, sub, grafo)
        _t.sleep(max(s.ms for s in self.sims) / 1000)

    t = gerar_tanques(n=16, s=5, h=1 / 128, largura=(40, 120), altura=(30, 60))
    Lote.avancar = avancar
    try:
        pesos, tempos = pesar_por_iteracoes(Falsa, Cena, t, 1 / 128, {"engine": _abi.TQ_ENGINE_FUSED}, 1 / 60, 2,
                                            200, 148)
    finally:
        Lote.avancar = orig
    assert set(tempos) == {"celulas", "trabalho"}
    assert tempos["trabalho"] < tempos["celulas"]
    assert pesos is not None and max(pesos) / min(pesos) < 1.01  # cells x iterations: equal here
