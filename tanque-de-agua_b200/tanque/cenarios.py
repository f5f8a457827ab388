"""Scene builders: seeded particle seeding and the wall/water layouts of the workloads.

`semente` is the seeded LCG of testes/apoio.js:4-9 and `semear_retangulo` the 2x2-jittered
seeding of js/fisica-cpu.js:705-727, both producing the reference's exact floats.  The preset
scenes (copo, vasos, ampulheta, labirinto, ...) follow js/modelos.js; they are the scenes the
reference's tests run and the synthetic benchmark scenes are built from.
"""
from __future__ import annotations

import math

import numpy as np

from .constantes import CAMPOS, MOLDURA, PARTICULAS_POR_CELULA


def semente(s: int = 1):
    """testes/apoio.js:4-9: s = (s*1664525 + 1013904223) mod 2^32, returns s / 2^32."""
    estado = [s & 0xFFFFFFFF]

    def aleatorio() -> float:
        estado[0] = (estado[0] * 1664525 + 1013904223) & 0xFFFFFFFF
        return estado[0] / 4294967296
    return aleatorio


def semear_retangulo(x0, y0, x1, y1, h, absorcao=(0.0, 0.0, 0.0), aleatorio=None) -> np.ndarray:
    """semearRetangulo (js/fisica-cpu.js:705-727): 2x2 jittered particles per cell."""
    if aleatorio is None:
        aleatorio = semente(1)
    lado = round(math.sqrt(PARTICULAS_POR_CELULA))
    passo = h / lado
    xa, xb = min(x0, x1), max(x0, x1)
    ya, yb = min(y0, y1), max(y0, y1)
    ia, ib = math.ceil(xa / passo - 0.5), math.floor(xb / passo - 0.5)
    ja, jb = math.ceil(ya / passo - 0.5), math.floor(yb / passo - 0.5)
    n = max(0, ib - ia + 1) * max(0, jb - ja + 1)
    lista = np.zeros(n * CAMPOS, dtype=np.float32)
    k = 0
    for j in range(ja, jb + 1):
        for i in range(ia, ib + 1):
            o = k * CAMPOS
            lista[o] = (i + 0.5 + (aleatorio() - 0.5) * 0.5) * passo
            lista[o + 1] = (j + 0.5 + (aleatorio() - 0.5) * 0.5) * passo
            lista[o + 9], lista[o + 10], lista[o + 11] = absorcao
            k += 1
    return lista


def semear_retangulo_rapido(x0, y0, x1, y1, h, absorcao=(0.0, 0.0, 0.0), s: int = 1) -> np.ndarray:
    """semear_retangulo vectorised for large blocks (same LCG stream, same floats)."""
    lado = round(math.sqrt(PARTICULAS_POR_CELULA))
    passo = h / lado
    xa, xb = min(x0, x1), max(x0, x1)
    ya, yb = min(y0, y1), max(y0, y1)
    ia, ib = math.ceil(xa / passo - 0.5), math.floor(xb / passo - 0.5)
    ja, jb = math.ceil(ya / passo - 0.5), math.floor(yb / passo - 0.5)
    ni, nj = max(0, ib - ia + 1), max(0, jb - ja + 1)
    n = ni * nj
    # the LCG stream: 2n draws, computed with 64-bit integers
    r = _fluxo_lcg(s, 2 * n)
    jj, ii = np.divmod(np.arange(n, dtype=np.int64), ni) if ni else (np.zeros(0, np.int64), np.zeros(0, np.int64))
    i = ii + ia
    j = jj + ja
    lista = np.zeros((n, CAMPOS), dtype=np.float32)
    lista[:, 0] = ((i + 0.5 + (r[0::2] - 0.5) * 0.5) * passo).astype(np.float32)
    lista[:, 1] = ((j + 0.5 + (r[1::2] - 0.5) * 0.5) * passo).astype(np.float32)
    lista[:, 9:12] = np.asarray(absorcao, dtype=np.float32)
    return lista.ravel()


def _fluxo_lcg(s: int, n: int) -> np.ndarray:
    """n successive draws of semente(s) as float64 (vectorised by blocks of LCG jumps)."""
    out = np.empty(n, dtype=np.float64)
    if n == 0:
        return out
    a, c, m = 1664525, 1013904223, 1 << 32
    bloco = min(n, 4096)
    # coefficients of x_{k} = A_k x_0 + C_k for k = 1..bloco
    A = np.empty(bloco, dtype=np.uint64)
    Cc = np.empty(bloco, dtype=np.uint64)
    ak, ck = 1, 0
    for k in range(bloco):
        ak = (ak * a) % m
        ck = (ck * a + c) % m
        A[k], Cc[k] = ak, ck
    x = s & 0xFFFFFFFF
    feito = 0
    while feito < n:
        t = min(bloco, n - feito)
        v = (A[:t] * np.uint64(x) + Cc[:t]) & np.uint64(0xFFFFFFFF)
        out[feito:feito + t] = v.astype(np.float64) / 4294967296
        x = int(v[t - 1])
        feito += t
    return out


def dentro_do_poligono(x, y, pts) -> bool:
    """dentroDoPoligono (js/modelos.js:216-223), even-odd rule."""
    dentro = False
    j = len(pts) - 1
    for i in range(len(pts)):
        xi, yi = pts[i]
        xj, yj = pts[j]
        if (yi > y) != (yj > y) and x < ((xj - xi) * (y - yi)) / (yj - yi) + xi:
            dentro = not dentro
        j = i
    return dentro


def semear_agua(entrada: dict, h: float, absorcao=(0.0, 0.0, 0.0), aleatorio=None) -> np.ndarray:
    """semearAgua (js/modelos.js:229-242): rectangle, or polygon clipped at limiteY."""
    if "poligono" not in entrada:
        return semear_retangulo(entrada["x0"], entrada["y0"], entrada["x1"], entrada["y1"], h, absorcao, aleatorio)
    pts = entrada["poligono"]
    xs = [q[0] for q in pts]
    ys = [q[1] for q in pts]
    topo = min(max(ys), entrada.get("limiteY", math.inf))
    bruto = semear_retangulo(min(xs), min(ys), max(xs), topo, h, absorcao, aleatorio).reshape(-1, CAMPOS)
    keep = [k for k in range(len(bruto)) if dentro_do_poligono(float(bruto[k, 0]), float(bruto[k, 1]), pts)]
    return bruto[keep].ravel()


# ------------------------------------------------------------------ preset scenes (js/modelos.js)
def raio_de_parede(h: float) -> float:
    return max(1.6 * h, 0.006)


def _linha(pts, raio, fechar=False):
    n = len(pts) if fechar else len(pts) - 1
    return [dict(x0=pts[k][0], y0=pts[k][1], x1=pts[(k + 1) % len(pts)][0], y1=pts[(k + 1) % len(pts)][1], raio=raio)
            for k in range(n)]


def _palco(W, H, h):
    m = MOLDURA * h
    largura = min(W - 2 * m, 1.7 * H)
    return dict(x0=(W - largura) / 2, largura=largura, chao=m, teto=H - m, altura=H - 2 * m,
                X=lambda f: (W - largura) / 2 + f * largura, Y=lambda f: m + f * (H - 2 * m))


def modelo_copo(W, H, h):
    p, r = _palco(W, H, h), raio_de_parede(h)
    cx = W / 2
    meia = min(p["largura"] * 0.14, p["altura"] * 0.2)
    base = p["chao"] + r
    topo = p["Y"](0.46)
    return dict(tracos=_linha([[cx - meia * 1.18, topo], [cx - meia, base], [cx + meia, base], [cx + meia * 1.18, topo]], r),
                agua=[dict(x0=cx - meia * 0.75, y0=p["Y"](0.66), x1=cx + meia * 0.75, y1=p["Y"](0.97))])


def modelo_ampulheta(W, H, h):
    p, r = _palco(W, H, h), raio_de_parede(h)
    cx = W / 2
    meia = min(p["largura"] * 0.2, p["altura"] * 0.3)
    pescoco = r + 1.8 * h
    topo, meio, base = p["Y"](0.94), p["Y"](0.5), p["Y"](0.06)
    contorno = [
        [cx - meia, topo], [cx + meia, topo], [cx + meia, topo - (topo - meio) * 0.25],
        [cx + pescoco, meio],
        [cx + meia, base + (meio - base) * 0.25], [cx + meia, base], [cx - meia, base],
        [cx - meia, base + (meio - base) * 0.25], [cx - pescoco, meio],
        [cx - meia, topo - (topo - meio) * 0.25],
    ]
    folga = r + h
    dentro = [
        [cx - meia + folga, topo - folga], [cx + meia - folga, topo - folga],
        [cx + meia - folga, topo - (topo - meio) * 0.25],
        [cx + pescoco * 0.3, meio + (topo - meio) * 0.12],
        [cx - pescoco * 0.3, meio + (topo - meio) * 0.12],
        [cx - meia + folga, topo - (topo - meio) * 0.25],
    ]
    return dict(tracos=_linha(contorno, r, True), agua=[dict(poligono=dentro, limiteY=meio + (topo - meio) * 0.72)])


def modelo_vasos(W, H, h):
    p, r = _palco(W, H, h), raio_de_parede(h)
    xa, xb = p["X"](0.18), p["X"](0.82)
    topo = p["Y"](0.82)
    vao = p["Y"](0.1)
    d1, d2 = xa + (xb - xa) * 0.3, xa + (xb - xa) * 0.52
    tracos = (_linha([[xa, topo], [xa, p["chao"]]], r) + _linha([[xb, topo], [xb, p["chao"]]], r)
              + _linha([[d1, topo], [d1, vao]], r) + _linha([[d2, topo], [d2 + (xb - d2) * 0.18, vao]], r))
    return dict(tracos=tracos, agua=[dict(x0=xa, y0=p["Y"](0.02), x1=d1, y1=p["Y"](0.62))])


def labirinto(W, H, h, aleatorio, linhas=6, corredor=None, raio=None, x0=None, y0=None, colunas=None):
    """Recursive-backtracker labyrinth of js/modelos.js:133-185.  With `corredor`/`raio` the
    cell pitch and wall radius are given in metres (the benchmark's 8-cell corridors and
    4-cell walls) instead of being fitted to the stage."""
    p = _palco(W, H, h)
    r = raio if raio is not None else raio_de_parede(h)
    if corredor is None:
        altura = p["altura"] * 0.78
        tam = altura / linhas
        colunas = max(3, min(10, math.floor((p["largura"] * 0.9) / tam)))
    else:
        tam = corredor
    largura = colunas * tam
    bx0 = W / 2 - largura / 2 if x0 is None else x0
    by0 = p["chao"] + p["altura"] * 0.03 if y0 is None else y0
    dir_ = [[True] * linhas for _ in range(colunas)]
    baixo = [[True] * linhas for _ in range(colunas)]
    visto = [[False] * linhas for _ in range(colunas)]
    pilha = [(0, linhas - 1)]
    visto[0][linhas - 1] = True
    while pilha:
        c, l = pilha[-1]
        viz = [(a, b) for (a, b) in [(c + 1, l), (c - 1, l), (c, l + 1), (c, l - 1)]
               if 0 <= a < colunas and 0 <= b < linhas and not visto[a][b]]
        if not viz:
            pilha.pop()
            continue
        a, b = viz[math.floor(aleatorio() * len(viz))]
        if a == c + 1:
            dir_[c][l] = False
        elif a == c - 1:
            dir_[a][l] = False
        elif b == l + 1:
            baixo[c][b] = False
        else:
            baixo[c][l] = False
        visto[a][b] = True
        pilha.append((a, b))
    X = lambda c: bx0 + c * tam  # noqa: E731
    Y = lambda l: by0 + l * tam  # noqa: E731
    tracos = []

    def seg(xa, ya, xb, yb):
        tracos.append(dict(x0=xa, y0=ya, x1=xb, y1=yb, raio=r))
    for c in range(colunas):
        for l in range(linhas):
            if dir_[c][l] and c < colunas - 1:
                seg(X(c + 1), Y(l), X(c + 1), Y(l + 1))
            if baixo[c][l] and l > 0:
                seg(X(c), Y(l), X(c + 1), Y(l))
    seg(X(0), Y(0), X(0), Y(linhas))
    seg(X(colunas), Y(0), X(colunas), Y(linhas))
    seg(X(1), Y(linhas), X(colunas), Y(linhas))
    seg(X(0), Y(0), X(colunas - 1), Y(0))
    folga = r + h
    return dict(tracos=tracos, agua=[dict(x0=X(0) + folga, y0=Y(linhas) + p["altura"] * 0.04, x1=X(1) - folga,
                                          y1=p["teto"] - 2 * h)], X=X, Y=Y, tam=tam, colunas=colunas)


MODELOS = {"copo": modelo_copo, "ampulheta": modelo_ampulheta, "vasos": modelo_vasos}


def montar_modelo(nome, nx, ny, h, aleatorio, Cena, fabrica):
    """montarModelo of testes/fisica.test.js:18-26 with a simulation factory."""
    cena = Cena(nx, ny, h)
    m = MODELOS[nome](cena.largura, cena.altura, h)
    for t in m["tracos"]:
        cena.tracar(t["x0"], t["y0"], t["x1"], t["y1"], t["raio"])
    cena.atualizar()
    sim = fabrica(cena)
    for a in m["agua"]:
        sim.adicionar(semear_agua(a, h, (0.0, 0.0, 0.0), aleatorio), False)
    return cena, sim, m


# ------------------------------------------------------------------ the ultra scene
def cena_ultra(Cena, nx: int = 840, ny: int = 536, h: float = 0.0016):
    """The 450k-cell scene of the throughput benchmark: a seeded labyrinth (56 x 22 cells of 12h,
    walls of radius 2h, from 40 % of the height) over water filling the tank to 85 %, and a
    faucet 12 cells wide at 1.2 m/s at the labyrinth's entrance (js/principal.js:301-321).
    Returns (cena, wall traces, particles, faucet)."""
    cena = Cena(nx, ny, h)
    W, Hh = cena.largura, cena.altura
    tam = 12 * h
    colunas, linhas = 56, 22
    x0 = (W - colunas * tam) / 2
    y0 = 0.40 * Hh
    lab = labirinto(W, Hh, h, semente(3), linhas=linhas, corredor=tam, raio=2 * h, x0=x0, y0=y0, colunas=colunas)
    for t in lab["tracos"]:
        cena.tracar(t["x0"], t["y0"], t["x1"], t["y1"], t["raio"])
    m = 2 * h
    agua = semear_retangulo_rapido(m, m, W - m, 0.85 * Hh, h, (0.0, 0.0, 0.0), s=3)
    torneira = dict(x=lab["X"](0) + tam / 2, y=lab["Y"](linhas) + 10 * h, raio=6 * h, vx=0.0, vy=-1.2, h=h)
    return cena, lab["tracos"], agua, torneira


def jato_torneira(torneira: dict, quadro: int, dt: float) -> np.ndarray:
    """emitirTorneira (js/principal.js:301-321) with a seeded LCG in place of Math.random:
    particles in a disk of the jet's radius, at the jet velocity, for frame `quadro`."""
    h = torneira["h"]
    r0 = torneira["raio"]
    vx, vy = torneira["vx"], torneira["vy"]
    vazao = 2 * r0 * max(0.7, math.hypot(vx, vy))
    n = min(40000, math.floor((vazao * dt) / (h * h) * 4 + 0.5))  # Math.round
    al = semente(1000 + quadro)
    lista = np.zeros((n, CAMPOS), dtype=np.float32)
    for k in range(n):
        a = al() * math.pi * 2
        r = math.sqrt(al()) * r0
        lista[k, 0] = torneira["x"] + math.cos(a) * r
        lista[k, 1] = torneira["y"] + math.sin(a) * r
        lista[k, 2] = vx
        lista[k, 3] = vy
    return lista.ravel()


# ------------------------------------------------------------------ benchmark configurations
def cena_barragem_160(Cena):
    """Dam break of the benchmark set: 160 x 100 cells, h = 6.25 mm (1.0 x 0.625 m), the tank's
    wall frame, a water block x in [0, 0.4 m], y in [0, 0.375 m] seeded 2 x 2 per cell with the
    LCG of semente(1), at rest.  Returns (cena, particles)."""
    h = 0.00625
    cena = Cena(160, 100, h)
    m = MOLDURA * h
    return cena, semear_retangulo_rapido(m, m, 0.4, 0.375, h, s=1)


def cena_ar_preso(Cena, nx: int = 480, ny: int = 270, h: float = 0.0022):
    """Trapped air of the benchmark set: a tank 60 % full with an inverted cup of 4-cell walls
    half submerged (an air pocket under its top, the water inside lower than outside) and 8
    circular air voids of radius 6-15 cells near the bottom (positions and radii from the LCG
    of semente(2)); 2 x 2 particles per cell.  Returns (cena, particles)."""
    cena = Cena(nx, ny, h)
    W, H = cena.largura, cena.altura
    raio = 2 * h
    cx0, cx1, cy0, cy1 = 0.35 * W, 0.65 * W, 0.35 * H, 0.75 * H
    cena.tracar(cx0, cy0, cx0, cy1, raio)
    cena.tracar(cx1, cy0, cx1, cy1, raio)
    cena.tracar(cx0, cy1, cx1, cy1, raio)
    m = MOLDURA * h
    agua = semear_retangulo_rapido(m, m, W - m, 0.6 * H, h, s=2).reshape(-1, CAMPOS)
    x, y = agua[:, 0].astype(np.float64), agua[:, 1].astype(np.float64)
    fora = ~((x > cx0) & (x < cx1) & (y > 0.45 * H))  # the pocket under the cup
    al = semente(2)
    for _ in range(8):
        r = (6 + 9 * al()) * h
        bx = m + r + al() * (W - 2 * (m + r))
        by = m + r + al() * (0.25 * H - r)
        fora &= (x - bx) ** 2 + (y - by) ** 2 >= r * r
    return cena, agua[fora].ravel()


def cena_adjunto(nx: int = 256, ny: int = 160, h: float = 0.004, passos: int = 60, dt: float = 1 / 240,
                 jato: int = 6, seed: int = 5) -> dict:
    """The differentiable scene of the adjoint (tq_adj_*): an empty tank (the frame of
    MOLDURA cells), a block of water seeded 2 x 2 per cell (semearRetangulo, js/fisica-cpu.js:705-727)
    with seeded initial velocities, a faucet near the top left that emits at every step a slab of
    `jato` cells by one cell, 4 particles a cell on a jittered 2 x 2 lattice (the jet density of
    js/principal.js:301-321, whose slab per frame is the jet's length over the frame; a jet of
    about 1 m/s moves about a cell a step here), and a seeded target blob of water fraction.
    Returns arrays: sdf (2ny, 2nx), positions (n, 2), v0 (n, 2), faucet_positions
    (passos, 4 jato, 2), target (ny, nx), theta0 (2,)."""
    from .cena import Cena
    cena = Cena(nx, ny, h)
    m = MOLDURA * h
    W, H = nx * h, ny * h
    al = semente(seed)
    bloco = semear_retangulo(m, m, m + 0.3 * W, m + 0.35 * H, h, (0, 0, 0), al).reshape(-1, CAMPOS)
    pos = bloco[:, :2].astype(np.float32)
    v0 = np.stack([[(al() - 0.5) * 0.4, (al() - 0.5) * 0.4] for _ in range(len(pos))]).astype(np.float32)
    x0, y0 = m + 0.10 * W, H - m - 0.18 * H
    fp = np.zeros((passos, 4 * jato, 2), np.float32)
    for s_ in range(passos):
        for k in range(jato):
            for q in range(4):
                fp[s_, 4 * k + q] = (x0 + (k + (q & 1) * 0.5 + 0.25 + (al() - 0.5) * 0.25) * h,
                                     y0 + ((q >> 1) * 0.5 + 0.25 + (al() - 0.5) * 0.25) * h)
    jj, ii = np.mgrid[0:ny, 0:nx]
    tx, ty, tr = (0.35 + 0.3 * al()) * nx, (0.1 + 0.2 * al()) * ny, (0.08 + 0.05 * al()) * nx
    alvo = np.clip(1.2 - np.hypot(ii + 0.5 - tx, jj + 0.5 - ty) / tr, 0, 1).astype(np.float32)
    return {"nx": nx, "ny": ny, "h": h, "dt": dt, "steps": passos, "checkpoint_every": 10,
            "sdf": np.asarray(cena.sdf, np.float32).reshape(2 * ny, 2 * nx), "positions": pos, "v0": v0,
            "faucet_positions": fp, "target": alvo, "theta0": np.array([0.9, -0.4])}
