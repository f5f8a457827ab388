"""The reference's behavioural test suite (testes/fisica.test.js, testes/cena.test.js), as
functions of a simulation factory so the same bodies run on the oracle (CPU) and on the CUDA
library (GPU).  Bounds and scenes are the reference's own; `rodar` is the reference's
adaptive frame loop (testes/fisica.test.js:12-19).
"""
from __future__ import annotations

import math

import numpy as np

from tanque.cenarios import MODELOS, semear_agua, semear_retangulo, semente
from tanque.constantes import CAMPOS, MOLDURA, PARTICULAS_POR_CELULA, PINCEL_MIN_CELULAS, passo_maximo

QUADRO = 1 / 60


def rodar(sim, segundos, a_cada=None):
    quadros = round(segundos / QUADRO)
    for f in range(quadros):
        sub = math.ceil(QUADRO / passo_maximo(sim.h, sim.cena.altura, sim.vMax, QUADRO))
        sim.avancar(QUADRO, sub)
        if a_cada:
            a_cada(f * QUADRO)


def particulas(sim) -> np.ndarray:
    return sim.p.reshape(-1, CAMPOS)


def velocidade_maxima(sim) -> float:
    p = particulas(sim)
    return float(np.max(np.hypot(p[:, 2].astype(np.float64), p[:, 3].astype(np.float64)))) if len(p) else 0.0


def distancias(cena, x, y) -> np.ndarray:
    """Cena.distancia (js/cena.js:102-106) for arrays of points."""
    w, hh = cena.mw, cena.mh
    sdf = np.asarray(cena.sdf, dtype=np.float64)
    fx = np.clip((x / cena.h) * 2 - 0.5, 0, w - 1)
    fy = np.clip((y / cena.h) * 2 - 0.5, 0, hh - 1)
    x0 = np.minimum(np.floor(fx), w - 2).astype(np.int64)
    y0 = np.minimum(np.floor(fy), hh - 2).astype(np.int64)
    tx, ty = fx - x0, fy - y0
    k = y0 * w + x0
    return (sdf[k] * (1 - tx) + sdf[k + 1] * tx) * (1 - ty) + (sdf[k + w] * (1 - tx) + sdf[k + w + 1] * tx) * ty


def menor_distancia_a_parede(sim) -> float:
    p = particulas(sim).astype(np.float64)
    return float(np.min(distancias(sim.cena, p[:, 0], p[:, 1]))) if len(p) else math.inf


def montar_modelo(F, nome, nx, ny, h, aleatorio, opcoes=None):
    cena = F.Cena(nx, ny, h)
    m = MODELOS[nome](cena.largura, cena.altura, h)
    for t in m["tracos"]:
        cena.tracar(t["x0"], t["y0"], t["x1"], t["y1"], t["raio"])
    cena.atualizar()
    sim = F.sim(cena, opcoes)
    for a in m["agua"]:
        sim.adicionar(semear_agua(a, h, (0.0, 0.0, 0.0), aleatorio), False)
    return cena, sim, m


# ------------------------------------------------------------------ fisica.test.js
def agua_parada(F, tensao, limite):
    """:31-43 — still water stays still (vmax < limit after 3 s)."""
    h = 0.01
    cena = F.Cena(60, 40, h)
    sim = F.sim(cena, {} if tensao is None else {"tensao": tensao})
    m = MOLDURA * h
    sim.adicionar(semear_retangulo(m, m, 0.6 - m, 0.2, h, (0, 0, 0), semente(3)), False)
    rodar(sim, 3)
    v = velocidade_maxima(sim)
    assert v < limite, f"velocidade máxima {v} m/s"


def gota_quadrada(F):
    """:45-66 — with g = 0 surface tension rounds a square drop."""
    h, n = 0.002, 70
    lado = 32 * h
    centro = (n * h) / 2

    def medir(tensao):
        cena = F.Cena(n, n, h)
        opc = {"gravidade": (0.0, 0.0)}
        if tensao is not None:
            opc["tensao"] = tensao
        sim = F.sim(cena, opc)
        sim.adicionar(semear_retangulo(centro - lado / 2, centro - lado / 2, centro + lado / 2, centro + lado / 2, h,
                                       (0, 0, 0), semente(8)), False)
        rodar(sim, 1.2)
        p = particulas(sim).astype(np.float64)
        cx, cy = p[:, 0].mean(), p[:, 1].mean()
        return float(np.max(np.abs(p[:, 0] - cx) + np.abs(p[:, 1] - cy))) / lado

    com, sem = medir(None), medir(0.0)
    assert sem > 0.93, f"sem tensão a gota não devia mudar de forma ({sem:.2f})"
    assert com < 0.88, f"com tensão a gota devia ficar redonda ({com:.2f}; círculo = 0,80)"


def copo_nao_vaza(F):
    """:68-76 — the cup neither leaks nor loses particles."""
    _, sim, _ = montar_modelo(F, "copo", 90, 60, 0.01, semente(11))
    n0 = sim.n
    assert n0 > 1000
    pior = [math.inf]

    def cada(_t):
        pior[0] = min(pior[0], menor_distancia_a_parede(sim))
    rodar(sim, 4, cada)
    assert sim.n == n0, "partículas sumiram"
    assert pior[0] > -0.05, f"partícula entrou na parede (distância {pior[0]} células)"


def pincel_fino_segura_jato(F):
    """:78-94 — the thinnest brush wall holds a 3.5 m/s jet."""
    h = 0.01
    cena = F.Cena(80, 60, h)
    cena.tracar(0.2, 0, 0.62, 0.6, PINCEL_MIN_CELULAS * h)
    cena.atualizar()
    sim = F.sim(cena, None)
    jato = semear_retangulo(0.03, 0.35, 0.12, 0.55, h, (0, 0, 0), semente(5))
    jato[2::CAMPOS] = 3.5
    jato[3::CAMPOS] = -1
    sim.adicionar(jato, False)
    vazou = [0]

    def cada(_t):
        p = particulas(sim).astype(np.float64)
        vazou[0] += int(np.sum((p[:, 0] - 0.2) * 0.6 - p[:, 1] * 0.42 > 0))
    rodar(sim, 3, cada)
    assert vazou[0] == 0, f"{vazou[0]} partículas passaram para o outro lado"


def barragem_conserva_volume(F):
    """:96-116 — mean surface level after a dam break within 6 % + h/2 of area/width."""
    h, nx, ny = 0.01, 80, 60
    cena = F.Cena(nx, ny, h)
    sim = F.sim(cena, None)
    m = MOLDURA * h
    sim.adicionar(semear_retangulo(m, m, 0.3, 0.42, h, (0, 0, 0), semente(9)), False)
    area = sim.area()
    rodar(sim, 10)
    p = particulas(sim)
    topo = np.zeros(nx, dtype=np.float32)
    i = np.floor(p[:, 0].astype(np.float64) / h).astype(np.int64)
    np.maximum.at(topo, i, p[:, 1])
    sel = topo[MOLDURA + 3: nx - MOLDURA - 3].astype(np.float64)
    nivel = sel.sum() / len(sel) - m
    esperado = area / (nx * h - 2 * m)
    assert abs(nivel - esperado) < 0.06 * esperado + 0.5 * h, f"nível {nivel:.4f} m, esperado {esperado:.4f} m"


def vasos_comunicantes(F):
    """:118-138 — water settles at the same level in the three vessels (within 2h)."""
    h = 0.01
    cena, sim, _ = montar_modelo(F, "vasos", 100, 64, h, semente(21))
    mm = MODELOS["vasos"](cena.largura, cena.altura, h)
    tr = mm["tracos"]
    xs = [tr[0]["x0"], tr[2]["x0"], (tr[3]["x0"] + tr[3]["x1"]) / 2, tr[1]["x0"]]
    niveis = [[], [], []]

    def cada(t):
        if t < 12:
            return
        p = particulas(sim).astype(np.float64)
        for k in range(3):
            sel = (p[:, 0] > xs[k] + 2.5 * h) & (p[:, 0] < xs[k + 1] - 2.5 * h)
            niveis[k].append(float(np.max(p[sel, 1])) if sel.any() else 0.0)
    rodar(sim, 16, cada)
    media = [sum(l) / len(l) for l in niveis]
    dif = max(media) - min(media)
    assert dif < 2 * h, f"níveis {media} m (diferença {dif / h:.1f} células)"


def densidade_de_repouso(F):
    """:140-159 — interior cells hold about 4 particles."""
    _, sim, _ = montar_modelo(F, "copo", 90, 60, 0.01, semente(4))
    rodar(sim, 5)
    nx, ny = sim.nx, sim.ny
    cont = sim.contagemCelula.reshape(ny, nx).astype(np.int64)
    sol = sim.solidoCelula.reshape(ny, nx)
    soma, n = 0, 0
    for j in range(2, ny - 2):
        for i in range(2, nx - 2):
            blk = (cont[j - 1:j + 2, i - 1:i + 2] == 0) | (sol[j - 1:j + 2, i - 1:i + 2] != 0)
            if not blk.any():
                soma += cont[j, i]
                n += 1
    assert n > 50, "quase não sobrou água no miolo"
    media = soma / n
    assert abs(media - PARTICULAS_POR_CELULA) < 0.4, f"média de {media:.2f} partículas por célula"


def tanque_com_bolha(F, ar):
    """:163-177"""
    h = 0.01
    cena = F.Cena(60, 60, h)
    sim = F.sim(cena, {"ar": ar})
    m = MOLDURA * h
    agua = semear_retangulo(m, m, 0.6 - m, 0.45, h, (0, 0, 0), semente(5)).reshape(-1, CAMPOS)
    x, y = agua[:, 0].astype(np.float64), agua[:, 1].astype(np.float64)
    fora = (x - 0.3) ** 2 + (y - 0.12) ** 2 >= 0.05 ** 2
    sim.adicionar(agua[fora].ravel(), False)
    return sim


def medir_bolhas(sim):
    """:179-188"""
    tipo = sim.tipo.reshape(sim.ny, sim.nx)
    rot = sim.rotulo.reshape(sim.ny, sim.nx)
    sel = (tipo == 2) & (rot >= 2)
    n = int(sel.sum())
    if not n:
        return n, None
    j = np.nonzero(sel)[0]
    return n, float(((j + 0.5) * sim.h).sum() / n)


def bolha_sobe(F):
    """:190-200 — an air bubble keeps its volume and rises."""
    sim = tanque_com_bolha(F, True)
    rodar(sim, 0.1)
    n0, a0 = medir_bolhas(sim)
    rodar(sim, 0.5)
    n1, a1 = medir_bolhas(sim)
    v0 = math.pi * 25
    assert n0 > 0.8 * v0, f"bolha encolheu no começo: {n0} de {v0:.0f} células"
    assert n1 > 0.75 * v0, f"bolha perdeu ar subindo: {n1} de {v0:.0f} células"
    assert a1 - a0 > 0.1, f"bolha subiu só {(a1 - a0) * 100:.1f} cm em 0,5 s"


def remontar_nao_perde_bolha(F):
    """:202-222 — rebuilding a scene over existing water keeps the new scene's bubble."""
    sim = tanque_com_bolha(F, True)
    m = MOLDURA * sim.h
    cheio = semear_retangulo(m, m, 0.6 - m, 0.45, sim.h, (0, 0, 0), semente(6))
    sim.n = 0
    sim.reiniciarAr()
    sim.adicionar(cheio, False)
    rodar(sim, 0.1)
    com_bolha = tanque_com_bolha(F, True)
    nova = com_bolha.p.copy()
    sim.n = 0
    sim.reiniciarAr()
    sim.adicionar(nova, False)
    rodar(sim, 0.1)
    v0 = math.pi * 25
    celulas, _ = medir_bolhas(sim)
    assert celulas > 0.8 * v0, f"a bolha do cenário novo virou vácuo: {celulas} de {v0:.0f} células"


def sem_ar_buraco_fecha(F):
    """:224-230"""
    sim = tanque_com_bolha(F, False)
    rodar(sim, 0.3)
    tipo = sim.tipo.reshape(sim.ny, sim.nx)
    vazias = int((tipo[3:25, 20:40] == 2).sum())
    assert vazias < 10, f"{vazias} células vazias onde era o buraco"


def ampulheta(F):
    """:232-250 — the hourglass drains much more slowly with air."""
    def em_cima(ar):
        h = 0.01
        cena = F.Cena(60, 90, h)
        m = MODELOS["ampulheta"](cena.largura, cena.altura, h)
        for t in m["tracos"]:
            cena.tracar(t["x0"], t["y0"], t["x1"], t["y1"], t["raio"])
        cena.atualizar()
        sim = F.sim(cena, {"ar": ar})
        for a in m["agua"]:
            sim.adicionar(semear_agua(a, h, (0, 0, 0), semente(2)), False)
        n0 = sim.n
        rodar(sim, 1)
        p = particulas(sim)
        return float(np.sum(p[:, 1] > cena.altura / 2)) / n0
    com, sem = em_cima(True), em_cima(False)
    assert sem < 0.1, f"sem ar, depois de 1 s ainda sobrava {sem * 100:.0f}% em cima"
    assert com > 0.4, f"com ar, depois de 1 s só sobrava {com * 100:.0f}% em cima"


# ------------------------------------------------------------------ cena.test.js
def cena_moldura(Cena):
    """testes/cena.test.js:9-18"""
    h = 0.01
    c = Cena(40, 30, h)
    assert c.celulaSolida(0, 0)
    assert c.celulaSolida(MOLDURA - 1, 15)
    assert not c.celulaSolida(MOLDURA, 15)
    assert not c.celulaSolida(20, 15)
    assert c.distancia(0.2, 0.15) == 10
    assert abs(c.distancia(MOLDURA * h + 3 * h, 0.15) - 3) < 0.05


def cena_distancia(Cena):
    """testes/cena.test.js:20-32"""
    h = 0.01
    c = Cena(60, 60, h)
    c.tracar(0.3, 0.3, 0.3, 0.3, 0.02)
    for d in [0.03, 0.045, 0.06, 0.08]:
        esperado = (d - 0.02) / h
        assert abs(c.distancia(0.3 + d, 0.3) - esperado) < 0.35
    assert c.distancia(0.3, 0.3) < -1.5
    assert c.celulaSolida(30, 30)
    nx, ny = c.normal(0.35, 0.3)
    assert nx > 0.99 and abs(ny) < 0.05


def cena_apagar(Cena):
    """testes/cena.test.js:34-44"""
    h = 0.01
    c = Cena(40, 30, h)
    c.tracar(0.1, 0.1, 0.3, 0.1, 0.015)
    assert c.celulaSolida(20, 10)
    c.tracar(0, 0.1, 0.4, 0.1, 0.03, True)
    c.tracar(0, 0, 0.4, 0.3, 0.05, True)
    assert not c.celulaSolida(20, 10)
    assert c.celulaSolida(0, 10) and c.celulaSolida(39, 10) and c.celulaSolida(20, 0)


def cena_incremental(Cena):
    """testes/cena.test.js:46-66 — the incremental SDF equals one rebuilt from scratch."""
    h = 0.01
    aleatorio = semente(7)
    a = Cena(70, 50, h)
    tracos = []
    for _ in range(25):
        t = dict(x0=aleatorio() * 0.7, y0=aleatorio() * 0.5, x1=aleatorio() * 0.7, y1=aleatorio() * 0.5,
                 raio=0.013 + aleatorio() * 0.03, apagar=aleatorio() < 0.25)
        tracos.append(t)
        a.tracar(t["x0"], t["y0"], t["x1"], t["y1"], t["raio"], t["apagar"])
    b = Cena(70, 50, h)
    for t in tracos:
        b.tracar(t["x0"], t["y0"], t["x1"], t["y1"], t["raio"], t["apagar"])
    assert float(np.max(np.abs(a.sdf - b.sdf))) < 1e-5
    assert np.array_equal(a.solido, b.solido)
    return a, tracos
