"""The FP64 CPU adjoint (the checker of the CUDA adjoint) against FP64 central finite differences
of its own forward run with the discrete structure frozen (CPU, no GPU).  A small tank for the
time the CPU suite allows; the GPU tests run the full 256 x 160 scene."""
import numpy as np

from oraculo import AdjuntoOraculo
from tanque.cenarios import cena_adjunto


def test_adjunto_fp64_contra_diferencas_finitas():
    c = cena_adjunto(nx=48, ny=32, h=0.01, passos=12)
    a = AdjuntoOraculo(c)
    v0, th = c["v0"].astype(np.float64), c["theta0"]
    a.forward(v0, th, True)
    gv, gt = a.backward()
    rng = np.random.default_rng(1)
    for k in rng.choice(len(v0), 8, replace=False):
        for comp in range(2):
            vp, vm = v0.copy(), v0.copy()
            vp[k, comp] += 1e-6
            vm[k, comp] -= 1e-6
            fd = (a.forward(vp, th, False) - a.forward(vm, th, False)) / 2e-6
            assert abs(gv[k, comp] - fd) <= 1e-4 * max(abs(fd), 1e-3), (k, comp, gv[k, comp], fd)
    for comp in range(2):
        tp, tm = th.copy(), th.copy()
        tp[comp] += 1e-8
        tm[comp] -= 1e-8
        fd = (a.forward(v0, tp, False) - a.forward(v0, tm, False)) / 2e-8
        assert abs(gt[comp] - fd) <= 1e-4 * abs(fd), (comp, gt[comp], fd)
