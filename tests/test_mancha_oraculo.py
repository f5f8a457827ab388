"""The oracle's headless splat (WGSL_MANCHA, js/gpu/render.js:11-43) and the new boundary calls'
argument errors, on the CPU.

Known answers pin the restatement:
- one particle on a pixel centre gives 1 there and (1 - r^2)^2 at the neighbours, with
  r = distance / (2.1 h), in every plane scaled by the particle's extra values;
- a particle outside the target or dead (x < 0) adds nothing;
- water seeded at 4 particles per cell gives, away from its edges, the renderer's own
  normalisation phi0 = 4 pi 2.1^2 / 3 (js/gpu/render.js:242), to the seeding's noise.
"""
import ctypes as C
import math

import numpy as np
import pytest

from oraculo import mancha_oraculo
from tanque import _abi
from tanque.cenarios import semear_retangulo_rapido
from tanque.constantes import CAMPOS

H_CEL = 0.01


def _particula(x, y, extra=(0.0, 0.0, 0.0, 0.0)):
    p = np.zeros(CAMPOS, dtype=np.float32)
    p[0], p[1] = x, y
    p[8:12] = extra
    return p


def test_uma_particula_no_centro_de_um_pixel():
    nx = ny = 20
    w = hp = 20  # one pixel per cell
    # pixel (i=7, row 5 from the top) has its centre at x = 7.5 h, y = H - 5.5 h
    x, y = 7.5 * H_CEL, (ny - 5.5) * H_CEL
    img = mancha_oraculo(_particula(x, y, (0.5, 1.0, 2.0, 0.25)), nx, ny, H_CEL, w, hp)
    assert img[0, 5, 7] == 1.0
    assert img[1, 5, 7] == 0.5 and img[2, 5, 7] == 1.0 and img[3, 5, 7] == 2.0 and img[4, 5, 7] == 0.25
    raio = np.float32(2.1 * H_CEL)
    for (di, dj) in [(1, 0), (0, 1), (-1, 0), (1, 1), (2, 0)]:
        u = np.float32(di * H_CEL) / raio
        v = np.float32(dj * H_CEL) / raio
        r2 = float(u) ** 2 + float(v) ** 2
        esperado = (1 - r2) ** 2 if r2 < 1 else 0.0
        assert abs(float(img[0, 5 + dj, 7 + di]) - esperado) < 1e-5, (di, dj)
    assert img[0, 5, 10] == 0.0  # 3 cells away: outside the 2.1-cell disk
    assert np.isclose(img[0].sum(), img[0][img[0] > 0].sum())


def test_particula_morta_ou_fora_nao_conta():
    img = mancha_oraculo(np.concatenate([_particula(-1.0, 0.05), _particula(5.0, 5.0)]), 10, 10, H_CEL, 10, 10)
    assert not img.any()


def test_agua_uniforme_da_phi0():
    nx, ny = 40, 30
    agua = semear_retangulo_rapido(0.0, 0.0, nx * H_CEL, ny * H_CEL, H_CEL, s=7)
    for w, hp in [(nx, ny), (2 * nx, 2 * ny), (nx // 2, ny // 2)]:
        img = mancha_oraculo(agua, nx, ny, H_CEL, w, hp)
        miolo = img[0, hp // 4: 3 * hp // 4, w // 4: 3 * w // 4]
        phi0 = 4 * math.pi * 2.1 ** 2 / 3
        assert abs(float(miolo.mean()) - phi0) < 0.03 * phi0, (w, hp, float(miolo.mean()), phi0)


def test_erros_de_argumento_das_novas_chamadas():
    lig = _abi.carregar()
    for nome, args in [("trace_wall", (None, 0.0, 0.0, 1.0, 1.0, 0.1, 0)), ("clear_walls", (None,)),
                       ("splat", (None, 8, 8, None))]:
        with pytest.raises(_abi.ErroTanque) as e:
            lig(nome, *args)
        assert e.value.status == _abi.TQ_E_ARG, nome
    assert C.CDLL(_abi.CAMINHO_LIB).tq_splat
