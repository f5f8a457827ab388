"""The tank walls: a signed distance field on a 2x2-per-cell grid (js/cena.js:14-165).

Host-side scene state, as in the reference (the browser's Cena is host JavaScript); the
simulation reads the SDF through tq_set_walls.  Arithmetic is IEEE double per element with a
float32 store, the same operations in the same order as js/cena.js, vectorised with numpy.
"""
from __future__ import annotations

import math

import numpy as np

from .constantes import MOLDURA, RES_MASCARA, SDF_MAX


class Cena:
    def __init__(self, nx: int, ny: int, h: float):
        self.nx, self.ny, self.h = nx, ny, h
        self.r = RES_MASCARA
        self.mw, self.mh = nx * self.r, ny * self.r
        self.largura = nx * h
        self.altura = ny * h
        self.sdf = np.zeros(self.mw * self.mh, dtype=np.float32)
        self.tracos = []
        self.mudou = False
        self.revisao = 0
        self._zerar()

    # Cena#moldura (js/cena.js:132-137) on coordinate arrays
    def _moldura(self, x: np.ndarray, y: np.ndarray) -> np.ndarray:
        r = self.r
        m = MOLDURA * r - 0.5
        a = np.minimum(np.minimum(x - m, (self.mw - 1) - m - x), np.minimum(y - m, (self.mh - 1) - m - y)) / r
        return np.clip(a, -SDF_MAX, SDF_MAX)

    def _zerar(self):
        y, x = np.mgrid[0:self.mh, 0:self.mw].astype(np.float64)
        self.sdf[:] = self._moldura(x, y).astype(np.float32).ravel()
        self.mudou = True
        self.revisao += 1

    @property
    def solido(self) -> np.ndarray:
        return (self.sdf < 0).astype(np.uint8)

    def tracar(self, x0, y0, x1, y1, raio, apagar=False, registrar=True):
        """tracar (js/cena.js:43-72): a capsule wall segment (metres), drawn or erased."""
        if registrar:
            self.tracos.append(dict(x0=x0, y0=y0, x1=x1, y1=y1, raio=raio, apagar=apagar))
        r = self.r
        s = r / self.h
        ax, ay, bx, by = x0 * s - 0.5, y0 * s - 0.5, x1 * s - 0.5, y1 * s - 0.5
        rp = raio * s
        alc = rp + SDF_MAX * r + 1
        xmin = max(0, math.floor(min(ax, bx) - alc))
        xmax = min(self.mw - 1, math.ceil(max(ax, bx) + alc))
        ymin = max(0, math.floor(min(ay, by) - alc))
        ymax = min(self.mh - 1, math.ceil(max(ay, by) + alc))
        if xmin > xmax or ymin > ymax:
            return
        dx, dy = bx - ax, by - ay
        len2 = dx * dx + dy * dy
        yy, xx = np.mgrid[ymin:ymax + 1, xmin:xmax + 1].astype(np.float64)
        if len2 > 0:
            t = ((xx - ax) * dx + (yy - ay) * dy) / len2
        else:
            t = np.zeros_like(xx)
        t = np.where(t < 0, 0.0, np.where(t > 1, 1.0, t))
        px = ax + t * dx - xx
        py = ay + t * dy - yy
        d = (np.sqrt(px * px + py * py) - rp) / r
        d = np.where(d > SDF_MAX, SDF_MAX, np.where(d < -SDF_MAX, -SDF_MAX, d))
        vista = self.sdf.reshape(self.mh, self.mw)[ymin:ymax + 1, xmin:xmax + 1]
        atual = vista.astype(np.float64)
        if apagar:
            v = np.maximum(atual, -d)
            v = np.minimum(v, self._moldura(xx, yy))
        else:
            v = np.minimum(atual, d)
        vista[...] = v.astype(np.float32)
        self.mudou = True
        self.revisao += 1

    def limpar(self):
        self.tracos = []
        self._zerar()

    def refazer(self, tracos):
        self.tracos = []
        self._zerar()
        for t in tracos:
            self.tracar(t["x0"], t["y0"], t["x1"], t["y1"], t["raio"], t.get("apagar", False))

    def atualizar(self) -> bool:
        m = self.mudou
        self.mudou = False
        return m

    def _bilinear(self, fx: float, fy: float) -> float:
        w, hh = self.mw, self.mh
        if fx != fx or fy != fy:
            return float("nan")
        fx = 0.0 if fx < 0 else (w - 1.0 if fx > w - 1 else fx)
        fy = 0.0 if fy < 0 else (hh - 1.0 if fy > hh - 1 else fy)
        x0 = int(min(math.floor(fx), w - 2))
        y0 = int(min(math.floor(fy), hh - 2))
        tx, ty = fx - x0, fy - y0
        k = y0 * w + x0
        d = self.sdf
        return ((float(d[k]) * (1 - tx) + float(d[k + 1]) * tx) * (1 - ty)
                + (float(d[k + w]) * (1 - tx) + float(d[k + w + 1]) * tx) * ty)

    def distancia(self, x: float, y: float) -> float:
        """Distance (cells) from a point (metres) to the walls, bilinear (js/cena.js:102-106)."""
        return self._bilinear((x / self.h) * self.r - 0.5, (y / self.h) * self.r - 0.5)

    def normal(self, x: float, y: float):
        fx = (x / self.h) * self.r - 0.5
        fy = (y / self.h) * self.r - 0.5
        gx = self._bilinear(fx + 1, fy) - self._bilinear(fx - 1, fy)
        gy = self._bilinear(fx, fy + 1) - self._bilinear(fx, fy - 1)
        n = math.hypot(gx, gy)
        return (gx / n, gy / n) if n > 1e-9 else (0.0, 1.0)

    def celulaSolida(self, i: int, j: int) -> bool:
        if i < 0 or j < 0 or i >= self.nx or j >= self.ny:
            return True
        w, r = self.mw, self.r
        a, b = i * r, j * r
        s = (float(self.sdf[b * w + a]) + float(self.sdf[b * w + a + 1])
             + float(self.sdf[(b + 1) * w + a]) + float(self.sdf[(b + 1) * w + a + 1]))
        return s < 0
