"""Physics constants and grid/time-step helpers of the tank (values of js/constantes.js)."""
from __future__ import annotations

import math

GRAVIDADE = 9.81
DENSIDADE_AGUA = 1000.0
TENSAO_SUPERFICIAL = 0.0728
MAX_BOLHAS = 4096
VOLTA_VOLUME_BOLHA = 0.05
PRESSAO_BOLHA_MAX = 20000.0
FATOR_CAPILAR = 0.4
PASSO_MAX = 0.008
PROFUNDIDADE = 0.05
PARTICULAS_POR_CELULA = 4
RES_MASCARA = 2
SDF_MAX = 10.0
MOLDURA = 2
RAIO_PARTICULA = 0.3
CFL = 2.0
MICROPASSO = 0.8
MAX_MICROPASSOS = 4
TAU_DENSIDADE = 0.1
EXCESSO_MIN = -0.5
EXCESSO_MAX = 1.0
ITERACOES_PCG = 3
CAMADAS_EXTRAPOLACAO = 2
PARTICULAS_MAX_POR_CELULA = 4.6
PINCEL_MIN_CELULAS = 1.3
PINCEL_MAX_CELULAS = 8
CAMPOS = 12  # x y vx vy cux cuy cvx cvy espuma absR absG absB (js/fisica-cpu.js:26)
SOLIDO, AGUA, AR = 0, 1, 2

QUALIDADES = {
    "ultra": (450_000, 0.0016),
    "maximo": (220_000, 0.0022),
    "alto": (130_000, 0.0026),
    "medio": (70_000, 0.0032),
    "leve": (32_000, 0.0040),
    "cpu": (9_000, 0.0060),
}


def dimensoes_da_grade(largura_m: float, altura_m: float, qualidade: str = "alto"):
    """dimensoesDaGrade (js/constantes.js:152-160): (nx, ny, h) for a W x H m tank."""
    celulas, h_min = QUALIDADES.get(qualidade, QUALIDADES["alto"])
    h = math.sqrt((largura_m * altura_m) / celulas)
    h = max(h, h_min)
    ny = max(24, _round_js(altura_m / h))
    h = altura_m / ny
    nx = max(24, _round_js(largura_m / h))
    return nx, ny, h


def passo_maximo(h: float, altura_m: float, v_max: float | None = None, dt_quadro: float = 1 / 60) -> float:
    """passoMaximo (js/constantes.js:167-175): the largest safe substep."""
    queda = math.sqrt(2 * GRAVIDADE * altura_m) * 1.15 + 0.5
    v = queda if v_max is None else min(queda, v_max * 1.2 + GRAVIDADE * dt_quadro + 0.25)
    capilar = FATOR_CAPILAR * math.sqrt((DENSIDADE_AGUA * h * h * h) / (2 * math.pi * TENSAO_SUPERFICIAL))
    return min((CFL * h) / max(v, 0.3), capilar, PASSO_MAX)


def _round_js(x: float) -> int:
    """Math.round: halves round up (toward +infinity)."""
    return math.floor(x + 0.5)
