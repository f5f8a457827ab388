"""Batched tanks: many independent tanks advanced together as tank atlases.

A batch of tanks (the 256-tank workload: widths log-uniform in [64, 512] cells, heights
log-uniform in [64, 320], random wall segments, a water rectangle filling 20-70 % of the tank,
4 particles per cell) is laid out in a few atlases.  An atlas is one grid in which the tanks
stand side by side, top-aligned, each with its own 2-cell frame and MARGEM solid columns on
either side; everything else is wall.  One simulation advances an atlas, so every stage of the
substep (particle-to-grid, flags, air labels, surface, divergence, the pressure solve,
gradient, extrapolation, grid-to-particle) runs as one launch for all the tanks in it, instead
of one launch per tank.

Why the tanks stay independent inside an atlas:
- pressure: walls are Neumann boundaries, so the pressure matrix is block diagonal, one block
  per tank; the preconditioner's coarse levels mix tanks, which changes the iterates but not the
  solution;
- air: a component of air cells never crosses a wall, and a tank's air reaches the top row
  (ny - MOLDURA - 1, the atmosphere test of js/ar.js:56-153) exactly as in a tank of its own
  because the tanks are top-aligned;
- the stencils that read across walls (the 3-layer wall extension and the (1 2 1) blurs of
  the surface stage, js/fisica-cpu.js:306-374) reach about 5 cells, less than the
  2 * (MOLDURA + MARGEM) solid columns between two tanks' water.
What the tanks share: the substep dt and the solve's scalars (one alpha and beta per PCG
iteration, and the stopping rule ||r|| <= tol ||r0|| on the whole atlas).  The solution each
tank gets is its own block's, to the atlas's tolerance.

Atlases are grouped so that the coarsest multigrid level of each stays small (the fused
engine solves the coarsest levels inside one CTA's shared memory): tanks are sorted by height,
tallest first, and added to the current atlas while its coarsest level has at most
`limite_grosso` cells.
"""
from __future__ import annotations

import math

import numpy as np

from . import _abi
from .cenarios import raio_de_parede, semear_retangulo_rapido, semente
from .constantes import CAMPOS, MOLDURA, SDF_MAX

MARGEM = 6  # solid columns on each side of a tank's frame in an atlas
LIMITE_GROSSO = 12000  # cells of an atlas's coarsest multigrid level


def gerar_tanques(n: int = 256, s: int = 4, h: float = 0.003, largura=(64, 512), altura=(64, 320)) -> list[dict]:
    """The seeded batch: per tank its size in cells (frame included, log-uniform in the given
    ranges), wall segments (metres, tank coordinates), water rectangle and particle seed.  All
    draws come from semente(s)."""
    al = semente(s)
    r = raio_de_parede(h)
    m = MOLDURA * h
    tanques = []
    for k in range(n):
        nx = int(round(math.exp(math.log(largura[0]) + al() * math.log(largura[1] / largura[0]))))
        ny = int(round(math.exp(math.log(altura[0]) + al() * math.log(altura[1] / altura[0]))))
        W, H = nx * h, ny * h
        tracos = []
        for _ in range(math.floor(al() * 4)):
            cx, cy = m + al() * (W - 2 * m), m + al() * (H - 2 * m)
            ang = al() * math.pi
            comp = (0.1 + 0.3 * al()) * (W - 2 * m)
            dx, dy = 0.5 * comp * math.cos(ang), 0.5 * comp * math.sin(ang)
            tracos.append(dict(x0=cx - dx, y0=cy - dy, x1=cx + dx, y1=cy + dy, raio=r))
        cheio = 0.2 + 0.5 * al()
        fl = 0.4 + 0.6 * al()
        fa = min(0.95, cheio / fl)
        agua = (m, m, m + fl * (W - 2 * m), m + fa * (H - 2 * m))
        tanques.append(dict(nx=nx, ny=ny, tracos=tracos, agua=agua, semente=1000 + k))
    return tanques


def niveis(nx: int, ny: int) -> list[tuple[int, int]]:
    """montarNiveis (js/pressao-cpu.js:24-41): levels halve (ceil) while min(nx, ny) > 12."""
    out = [(nx, ny)]
    while min(nx, ny) > 12:
        nx, ny = (nx + 1) // 2, (ny + 1) // 2
        out.append((nx, ny))
    return out


def largura_atlas(tanques: list[dict], margem: int = MARGEM) -> int:
    return sum(t["nx"] + 2 * margem for t in tanques)


def agrupar(tanques: list[dict], limite_grosso: int = LIMITE_GROSSO, margem: int = MARGEM) -> list[list[int]]:
    """Tank indices per atlas: tallest first, an atlas grows while its coarsest level has at
    most `limite_grosso` cells."""
    ordem = sorted(range(len(tanques)), key=lambda k: (-tanques[k]["ny"], k))
    grupos: list[list[int]] = []
    atual: list[int] = []
    for k in ordem:
        prova = atual + [k]
        ts = [tanques[i] for i in prova]
        gx, gy = niveis(largura_atlas(ts, margem), max(t["ny"] for t in ts))[-1]
        if atual and gx * gy > limite_grosso:
            grupos.append(atual)
            atual = [k]
        else:
            atual = prova
    if atual:
        grupos.append(atual)
    return grupos


def montar_atlas(Cena, tanques: list[dict], h: float, margem: int = MARGEM) -> dict:
    """One atlas: the scene (walls), each tank's column / row offset, and the particles.

    Each tank's walls are drawn on a scene of its own (frame included) and pasted into the
    atlas mask, top-aligned; the rest of the atlas is wall.  Particles are seeded in tank
    coordinates and moved by the tank's offset."""
    ny = max(t["ny"] for t in tanques)
    x0s = []
    x = 0
    for t in tanques:
        x0s.append(x + margem)
        x += t["nx"] + 2 * margem
    cena = Cena(x, ny, h)
    r = cena.r
    mascara = np.full((ny * r, x * r), -SDF_MAX, dtype=np.float32)
    partes, y0s, contagens = [], [], []
    for t, x0 in zip(tanques, x0s):
        c = Cena(t["nx"], t["ny"], h)
        for tr in t["tracos"]:
            c.tracar(tr["x0"], tr["y0"], tr["x1"], tr["y1"], tr["raio"])
        y0 = ny - t["ny"]
        mascara[y0 * r:ny * r, x0 * r:(x0 + t["nx"]) * r] = np.asarray(c.sdf, dtype=np.float32).reshape(t["ny"] * r, t["nx"] * r)
        p = semear_retangulo_rapido(*t["agua"], h, s=t["semente"]).reshape(-1, CAMPOS).copy()
        p[:, 0] = (p[:, 0].astype(np.float64) + x0 * h).astype(np.float32)
        p[:, 1] = (p[:, 1].astype(np.float64) + y0 * h).astype(np.float32)
        partes.append(p)
        y0s.append(y0)
        contagens.append(len(p))
    cena.sdf[:] = mascara.ravel()
    particulas = np.concatenate(partes).ravel() if partes else np.zeros(0, np.float32)
    return dict(cena=cena, x0=x0s, y0=y0s, nx=[t["nx"] for t in tanques], particulas=particulas,
                semeadas=contagens)


def recortar(Cena, cena_atlas, x0: int, x1: int):
    """The columns [x0, x1) of an atlas as a scene of their own (same mask values): a tank
    with its margins, for checking that the atlas leaves it independent."""
    r = cena_atlas.r
    c = Cena(x1 - x0, cena_atlas.ny, cena_atlas.h)
    m = np.asarray(cena_atlas.sdf).reshape(cena_atlas.ny * r, cena_atlas.nx * r)
    c.sdf[:] = m[:, x0 * r:x1 * r].ravel()
    return c


def repartir_ctas(pesos: list[float], total: int, minimo: int = 4) -> list[int] | None:
    """The SMs of one GPU split between atlases whose persistent solves run side by side: each
    atlas gets CTAs in proportion to its weight (its cells), at least `minimo` (or
    total // atlases when smaller), and the counts add up to at most `total` (one CTA per SM, so
    every solve stays co-resident).  None when there are more atlases than SMs."""
    n = len(pesos)
    if n == 0:
        return []
    if n > total:
        return None
    minimo = max(1, min(minimo, total // n))
    W = float(sum(pesos)) or 1.0
    c = [max(minimo, int(total * p / W)) for p in pesos]
    while sum(c) > total:  # take from the largest share above the minimum
        k = max(range(n), key=lambda i: (c[i], -i))
        if c[k] <= minimo:
            break
        c[k] -= 1
    return c


class Lote:
    """A batch of tanks as atlases, each advanced by one simulation made by `fabrica(cena,
    opcoes)` (SimulacaoGPU, or the oracle's class in tests).

    `sms`: the GPU's SM count, to run the atlases' frames side by side: each atlas's fused
    solve gets a share of the SMs (tq_options.fused_ctas, repartir_ctas by cells) and
    avancar(grafo=True) queues every atlas's frame (tq_launch_graph) before waiting for any."""

    def __init__(self, fabrica, Cena, tanques: list[dict], h: float, opcoes: dict | None = None,
                 limite_grosso: int = LIMITE_GROSSO, margem: int = MARGEM, sms: int | None = None,
                 pesos: list[float] | None = None, minimo: int = 4):
        self.tanques = tanques
        self.h = h
        self.margem = margem
        self.grupos = agrupar(tanques, limite_grosso, margem)
        self.atlas, self.sims = [], []
        self.onde = {}  # tank -> (atlas, position in the atlas)
        atlas = [montar_atlas(Cena, [tanques[k] for k in g], h, margem) for g in self.grupos]
        fundido = (opcoes or {}).get("engine", _abi.TQ_ENGINE_PLAIN) == _abi.TQ_ENGINE_FUSED
        if pesos is None:
            pesos = [at["cena"].nx * at["cena"].ny for at in atlas]
        self.ctas = repartir_ctas(pesos, sms, minimo) if sms and fundido and len(atlas) > 1 else None
        for a, g in enumerate(self.grupos):
            at = atlas[a]
            o_at = dict(opcoes or {})
            if self.ctas:
                o_at["fused_ctas"] = self.ctas[a]
            sim = fabrica(at["cena"], o_at)
            sim.adicionar(at["particulas"], False)
            # every tank's own convergence (tq_set_tanks) where the engine offers it: the fused
            # engine in tolerance mode
            o = dict(opcoes or {})
            if (hasattr(sim, "definirTanques") and o.get("tolerance", 0) > 0
                    and o.get("engine", _abi.TQ_ENGINE_PLAIN) == _abi.TQ_ENGINE_FUSED):
                sim.definirTanques([(x0, y0, tanques[k]["nx"], tanques[k]["ny"])
                                    for x0, y0, k in zip(at["x0"], at["y0"], g)])
            self.atlas.append(at)
            self.sims.append(sim)
            for i, k in enumerate(g):
                self.onde[k] = (a, i)

    @property
    def celulas(self) -> int:
        return sum(at["cena"].nx * at["cena"].ny for at in self.atlas)

    @property
    def celulas_tanques(self) -> int:
        return sum(t["nx"] * t["ny"] for t in self.tanques)

    @property
    def n(self) -> int:
        return sum(s.n for s in self.sims)

    def avancar(self, dt: float, subpassos: int = 1, grafo: bool = False):
        """One frame of every atlas (each on its simulation's stream); with `grafo` the
        substeps replay from each atlas's CUDA graph (tq_advance_graph) where available, and
        with the SMs split between the atlases (`sms`) every frame is queued before the first
        is waited for, so the atlases run side by side."""
        if grafo and self.ctas and all(hasattr(s, "lancarGrafo") for s in self.sims):
            for s in self.sims:
                s.lancarGrafo(dt, subpassos)
            for s in self.sims:
                s.sincronizar()
            return
        for s in self.sims:
            if grafo and hasattr(s, "avancarGrafo"):
                s.avancarGrafo(dt, subpassos)
            else:
                s.avancar(dt, subpassos)

    def sincronizar(self):
        for s in self.sims:
            if hasattr(s, "sincronizar"):
                s.sincronizar()

    def ms_atlas(self) -> list[float]:
        """Device time (ms) of each atlas's last frame replayed from its graph
        (TQ_SCALAR_GRAPH_FRAME_MS)."""
        return [s.escalar(_abi.TQ_SCALAR_GRAPH_FRAME_MS) for s in self.sims]

    def colunas(self, k: int) -> tuple[int, int, int]:
        """(atlas, first column, end column) of tank k's cells, frame included."""
        a, i = self.onde[k]
        x0 = self.atlas[a]["x0"][i]
        return a, x0, x0 + self.atlas[a]["nx"][i]

    def campo(self, k: int, nome: str) -> np.ndarray:
        """A cell field of tank k (rows of the tank, frame included), as ny x nx."""
        a, x0, x1 = self.colunas(k)
        at = self.atlas[a]
        ny, nx = at["cena"].ny, at["cena"].nx
        y0 = at["y0"][self.onde[k][1]]
        return np.asarray(self.sims[a].campo(nome)).reshape(ny, nx)[y0:, x0:x1]

    def particulas(self, k: int) -> np.ndarray:
        """Tank k's particles (rows of 12 floats), in tank coordinates."""
        a, x0, x1 = self.colunas(k)
        y0 = self.atlas[a]["y0"][self.onde[k][1]]
        p = np.asarray(self.sims[a].p).reshape(-1, CAMPOS)
        sel = (p[:, 0] >= x0 * self.h) & (p[:, 0] < x1 * self.h)
        q = p[sel].copy()
        q[:, 0] -= np.float32(x0 * self.h)
        q[:, 1] -= np.float32(y0 * self.h)
        return q

    def fechar(self):
        for s in self.sims:
            if hasattr(s, "fechar"):
                s.fechar()


def autoajustar(fabrica, Cena, tanques: list[dict], h: float, opcoes: dict, dt: float, subpassos: int,
                candidatos=(2000, 3000, 4000, 6000, 12000), repeticoes: int = 1,
                sms: int | None = None) -> tuple[int, dict]:
    """The atlas grouping by measurement: for each candidate limit of the coarsest level's cells
    (which sets how many atlases the batch makes, their padding, and each atlas's V-cycle depth
    and coarsest-level size), build the batch, run one warm-up frame, then time `repeticoes`
    frames of every atlas (wall time after the handles' streams drain), and keep the fastest.
    Candidates whose coarsest level exceeds what the fused solver's CTA 0 holds are skipped by
    the grouping itself.  Returns (limit, {limit: seconds per frame})."""
    import time
    tempos = {}
    for lim in candidatos:
        lote = Lote(fabrica, Cena, tanques, h, opcoes, limite_grosso=lim, sms=sms)
        try:
            lote.avancar(dt, subpassos, grafo=True)
            lote.sincronizar()
            t0 = time.perf_counter()
            for _ in range(repeticoes):
                lote.avancar(dt, subpassos, grafo=True)
            lote.sincronizar()
            tempos[lim] = (time.perf_counter() - t0) / repeticoes
        finally:
            lote.fechar()
    melhor = min(tempos, key=lambda k: (tempos[k], k))
    return melhor, tempos


def pesar_por_iteracoes(fabrica, Cena, tanques: list[dict], h: float, opcoes: dict, dt: float, subpassos: int,
                        limite_grosso: int, sms: int) -> tuple[list[float] | None, dict]:
    """Weights of the SM split between side-by-side atlases, by measurement: an atlas's work is
    its cells times its solves' mean iteration count (the per-tank stop makes atlases of equal
    size take different counts).  The split by cells runs a warm-up frame and a timed frame,
    whose solve records give each atlas's mean iterations; the split by cells x iterations
    then runs the same; the faster is kept.  Returns its weights (None: the cells) and the
    seconds per frame of both."""
    import time
    tempos, pesos_trab = {}, None
    for nome in ("celulas", "trabalho"):
        lote = Lote(fabrica, Cena, tanques, h, opcoes, limite_grosso=limite_grosso, sms=sms,
                    pesos=None if nome == "celulas" else pesos_trab)
        try:
            if lote.ctas is None:
                return None, {}
            lote.avancar(dt, subpassos, grafo=True)
            for s in lote.sims:
                s.definirEscalar(_abi.TQ_SCALAR_SOLVES, 0)
            t0 = time.perf_counter()
            lote.avancar(dt, subpassos, grafo=True)
            tempos[nome] = time.perf_counter() - t0
            if nome == "celulas":
                pesos_trab = []
                for at, s in zip(lote.atlas, lote.sims):
                    n = max(s.escalar(_abi.TQ_SCALAR_SOLVES), 1.0)
                    pesos_trab.append(at["cena"].nx * at["cena"].ny * s.escalar(_abi.TQ_SCALAR_SOLVE_ITERS) / n)
        finally:
            lote.fechar()
    melhor = min(tempos, key=lambda k: (tempos[k], k))
    return (pesos_trab if melhor == "trabalho" else None), tempos


def repartir(tanques: list[dict], partes: int) -> list[list[int]]:
    """Tank indices per GPU: largest tank first onto the least-loaded GPU (by cells).  The tanks
    are independent, so the GPUs share no data while they step."""
    carga = [0] * partes
    out: list[list[int]] = [[] for _ in range(partes)]
    for k in sorted(range(len(tanques)), key=lambda k: (-tanques[k]["nx"] * tanques[k]["ny"], k)):
        p = min(range(partes), key=lambda i: (carga[i], i))
        out[p].append(k)
        carga[p] += tanques[k]["nx"] * tanques[k]["ny"]
    return [sorted(o) for o in out]


# Algorithmic HBM bytes of the pressure solve per atlas cell: (per PCG iteration, per solve's
# setup), for FP32 and 16-bit V-cycle storage (the same model as the single-tank benchmark).
BYTES_POR_CELULA_ITER = {"fp32": (156.0, 110.0), "fp16": (120.0, 85.0), "bf16": (120.0, 85.0)}
# the same with TQ_PRECOND_BLOCK_1 (one smoother pass a leg on the levels above 0)
BYTES_POR_CELULA_ITER_BLOCO = {"fp32": (147.3, 101.3), "fp16": (115.3, 80.3), "bf16": (115.3, 80.3)}
