"""Helpers shared by the GPU parity tests: scenes, state transfer oracle -> CUDA, comparisons."""
from __future__ import annotations

import math

import numpy as np

from oraculo import CenaOraculo, SimulacaoOraculo
from tanque import _abi
from tanque.cenarios import MODELOS, semear_agua, semear_retangulo, semente
from tanque.constantes import CAMPOS, MOLDURA

# Fields that describe the state between substeps (what SimulacaoCPU carries over).
ESTADO = ["q", "rotulo", "pressaoBolha", "volumeAlvo", "vivo", "tipo", "contagemCelula"]
ESCALARES = [_abi.TQ_SCALAR_PRIMEIRA, _abi.TQ_SCALAR_TIPOS_PRONTOS]


def cena_barragem(Cn, nx=60, ny=40, h=0.01):
    cena = Cn(nx, ny, h)
    m = MOLDURA * h
    agua = semear_retangulo(m, m, 0.45 * nx * h, 0.6 * ny * h, h, (0, 0, 0), semente(1))
    return cena, agua


def cena_bolha(Cn, n=60, h=0.01):
    cena = Cn(n, n, h)
    m = MOLDURA * h
    agua = semear_retangulo(m, m, n * h - m, 0.45, h, (0, 0, 0), semente(5)).reshape(-1, CAMPOS)
    x, y = agua[:, 0].astype(np.float64), agua[:, 1].astype(np.float64)
    fora = (x - 0.3) ** 2 + (y - 0.12) ** 2 >= 0.05 ** 2
    # some dye so the dye sums are exercised
    agua[: len(agua) // 3, 9] = 1.5
    agua[: len(agua) // 5, 11] = 0.25
    return cena, agua[fora].ravel()


def cena_copo(Cn, nx=90, ny=60, h=0.01):
    cena = Cn(nx, ny, h)
    m = MODELOS["copo"](cena.largura, cena.altura, h)
    for t in m["tracos"]:
        cena.tracar(t["x0"], t["y0"], t["x1"], t["y1"], t["raio"])
    agua = np.concatenate([semear_agua(a, h, (0, 0, 0), semente(11)) for a in m["agua"]])
    return cena, agua


CENAS = {"barragem": cena_barragem, "bolha": cena_bolha, "copo": cena_copo}


def copiar_estado(de, para):
    """Copies the between-substeps state of `de` into `para` (both Simulacao)."""
    para.definirParticulas(de.p)
    for nome in ESTADO:
        para.definirCampo(nome, de.campo(nome))
    for s in ESCALARES:
        para.definirEscalar(s, de.escalar(s))


def erro_relativo(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    escala = max(float(np.max(np.abs(b))) if b.size else 0.0, 1e-30)
    return float(np.max(np.abs(a - b))) / escala if a.size else 0.0


# Fields compared bit for bit after a substep from the same state: particle-to-grid sums, flags,
# counts, air labels, bubble liveness and volumes.
INTEIROS = ["accU", "accV", "accCel", "accCor", "tipo", "contagemCelula", "rotulo", "vivo", "volumeBolha"]


def comparar_passo(o, g, quadro, tol_campos=1e-3, tol_pos=1e-5, fechadas=False):
    """GPU `g` against the oracle `o` after the same substep: integers bit for bit; pressure
    and velocities to the solve's accuracy (relative L-infinity); positions in metres.  With
    `fechadas` q is compared without each closed region's constant (regioes_fechadas)."""
    for campo in INTEIROS:
        a, b = g.campo(campo), o.campo(campo)
        assert np.array_equal(a, b), f"{quadro}: {campo} differs in {np.count_nonzero(a != b)} entries"
    for campo in ["q", "u", "v"]:
        a, b = g.campo(campo), o.campo(campo)
        if campo == "q" and fechadas:
            tipo = o.campo("tipo").reshape(o.ny, o.nx)
            reg = regioes_fechadas(tipo, o.campo("rotulo").reshape(o.ny, o.nx))
            a, b = sem_constante(a, tipo, reg), sem_constante(b, tipo, reg)
        e = erro_relativo(a, b)
        assert e <= tol_campos, f"{quadro}: {campo} relative error {e:.3g}"
    pg, po = g.p.reshape(-1, CAMPOS), o.p.reshape(-1, CAMPOS)
    assert pg.shape == po.shape, quadro
    assert float(np.max(np.abs(pg[:, :2].astype(np.float64) - po[:, :2]))) < tol_pos, quadro


def regioes_fechadas(tipo, rotulo) -> list[np.ndarray]:
    """Masks (ny x nx) of the closed regions of a solve: water cells joined to their water
    neighbours and to the active bubbles they face (a label >= 2 on an interior air cell facing
    water), in a component no water cell of which faces other air.  Each mask holds the water
    cells and the bubbles' air cells."""
    from scipy import ndimage
    from tanque.constantes import AGUA, AR
    ny, nx = tipo.shape
    agua = tipo == AGUA
    viz = np.zeros_like(agua)
    viz[:, 1:] |= agua[:, :-1]
    viz[:, :-1] |= agua[:, 1:]
    viz[1:, :] |= agua[:-1, :]
    viz[:-1, :] |= agua[1:, :]
    interior = np.zeros_like(agua)
    interior[1:-1, 1:-1] = True
    cand = (tipo == AR) & (rotulo >= 2) & (rotulo < 4096)
    ativas = np.unique(rotulo[cand & viz & interior])
    bolha = cand & np.isin(rotulo, ativas)
    rot, n = ndimage.label(agua | bolha)
    dirichlet = (tipo == AR) & ~bolha
    toca = np.zeros_like(agua)
    toca[:, 1:] |= dirichlet[:, :-1]
    toca[:, :-1] |= dirichlet[:, 1:]
    toca[1:, :] |= dirichlet[:-1, :]
    toca[:-1, :] |= dirichlet[1:, :]
    abertas = set(np.unique(rot[agua & toca]))
    return [rot == k for k in range(1, n + 1) if k not in abertas and np.any(agua & (rot == k))]


def sem_constante(q, tipo, regioes) -> np.ndarray:
    """q with each closed region's mean over its water cells removed (on the whole region): the
    constant a singular region's pressure is only defined up to."""
    from tanque.constantes import AGUA
    q = np.asarray(q, dtype=np.float64).reshape(tipo.shape).copy()
    for m in regioes:
        q[m] -= q[m & (tipo == AGUA)].mean()
    return q.ravel()


def divergencia(sim) -> np.ndarray:
    """Discrete divergence of the MAC velocities on water cells (per unit cell width), 0 elsewhere:
    u[i+1,j] - u[i,j] + v[i,j+1] - v[i,j] (js/fisica-cpu.js:456-470's form without the density
    term)."""
    nx, ny = sim.nx, sim.ny
    u = sim.campo("u").astype(np.float64).reshape(ny, nx + 1)
    v = sim.campo("v").astype(np.float64).reshape(ny + 1, nx)
    d = (u[:, 1:] - u[:, :-1]) + (v[1:, :] - v[:-1, :])
    d[sim.campo("tipo").reshape(ny, nx) != 1] = 0.0
    return d


def volume_na_grade(sim) -> float:
    """Water volume on the grid: the sum over cells of the fraction min(1, rho / 4)
    (js/fisica-cpu.js:309) times h^2."""
    return float(np.sum(np.minimum(1.0, sim.campo("densidade").astype(np.float64) / 4.0))) * sim.h * sim.h


def nivel_medio(sim) -> tuple[float, float]:
    """The reference's volume check (testes/fisica.test.js:96-116): the mean over the columns away
    from the walls of the highest particle's height, above the frame, and the level the water's
    area would fill."""
    from tanque.constantes import MOLDURA
    h, nx = sim.h, sim.nx
    p = sim.p.reshape(-1, CAMPOS)
    topo = np.zeros(nx, np.float32)
    i = np.floor(p[:, 0].astype(np.float64) / h).astype(np.int64)
    ok = (i >= 0) & (i < nx)
    np.maximum.at(topo, i[ok], p[ok, 1])
    m = MOLDURA * h
    cols = topo[MOLDURA + 3: nx - MOLDURA - 3].astype(np.float64)
    return float(cols.mean()) - m, sim.area() / (nx * h - 2 * m)
