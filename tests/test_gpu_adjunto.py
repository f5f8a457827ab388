"""The CUDA adjoint of the step (tq_adj_*, FP64 on the GPU) against the FP64 CPU adjoint of the
oracle (the same frozen-structure map) and against FP64 central finite differences of the oracle's
forward run, on a small tank and on the 256 x 160, 60-step scene; the forward/backward pair's
Function contract; checkpoint intervals that change nothing.

Bounds: the GPU and the CPU adjoints differ by the order of FP64 atomic sums and the solves'
1e-12 residuals: 1e-6 relative (dL/dv0 is returned in FP32).  Against finite differences: 1e-4
relative, the north_star's bound (the faucet direction's map is stiff: its differences use a step
of 1e-8)."""
import numpy as np
import pytest

from oraculo import AdjuntoOraculo
from tanque.adjunto import AdjuntoGPU, Contexto, PassoDiferenciavel
from tanque.cenarios import cena_adjunto

pytestmark = pytest.mark.gpu


def rel_inf(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30))


@pytest.mark.parametrize("tamanho", [dict(nx=48, ny=32, h=0.01, passos=12), dict()], ids=["48x32-12", "256x160-60"])
def test_adjunto_gpu_igual_ao_fp64_da_cpu(lib_gpu, tamanho, capsys):
    c = cena_adjunto(**tamanho)
    o = AdjuntoOraculo(c)
    g = AdjuntoGPU(c)
    v0, th = c["v0"], c["theta0"]
    L_o = o.forward(v0.astype(np.float64), th, True)
    gv_o, gt_o = o.backward()
    L_g = g.frente(v0, th)
    gv_g, gt_g = g.tras(1.0)
    with capsys.disabled():
        print(f"\n{c['nx']}x{c['ny']} {c['steps']} steps: loss {L_g:.10g} vs {L_o:.10g}; dv0 rel {rel_inf(gv_g, gv_o):.2e}, "
              f"dtheta {gt_g} vs {gt_o}")
    assert abs(L_g - L_o) <= 1e-9 * abs(L_o)
    assert rel_inf(gv_g, gv_o) <= 1e-6
    assert rel_inf(gt_g, gt_o) <= 1e-6
    # against central differences of the FP64 forward run (frozen structure)
    rng = np.random.default_rng(3)
    vd = v0.astype(np.float64)
    for k in rng.choice(len(v0), 2, replace=False):
        vp, vm = vd.copy(), vd.copy()
        vp[k, 0] += 1e-6
        vm[k, 0] -= 1e-6
        fd = (o.forward(vp, th, False) - o.forward(vm, th, False)) / 2e-6
        assert abs(gv_g[k, 0] - fd) <= 1e-4 * max(abs(fd), 1e-3), (k, gv_g[k, 0], fd)
    for comp in range(2):
        tp, tm = th.copy(), th.copy()
        tp[comp] += 1e-8
        tm[comp] -= 1e-8
        fd = (o.forward(vd, tp, False) - o.forward(vd, tm, False)) / 2e-8
        assert abs(gt_g[comp] - fd) <= 1e-4 * abs(fd), (comp, gt_g[comp], fd)


def test_contrato_function(lib_gpu):
    """forward saves the handle; backward scales by the incoming gradient and returns one gradient
    per input (None for the handle)."""
    c = cena_adjunto(nx=48, ny=32, h=0.01, passos=12)
    g = AdjuntoGPU(c)
    ctx = Contexto()
    perda = PassoDiferenciavel.forward(ctx, g, c["v0"], c["theta0"])
    nada, dv1, dt1 = PassoDiferenciavel.backward(ctx, 1.0)
    assert nada is None and perda > 0
    ctx2 = Contexto()
    assert PassoDiferenciavel.forward(ctx2, g, c["v0"], c["theta0"]) == pytest.approx(perda, rel=1e-12)
    _, dv2, dt2 = PassoDiferenciavel.backward(ctx2, 2.0)
    assert rel_inf(dv2, 2 * dv1) <= 1e-6 and rel_inf(dt2, 2 * dt1) <= 1e-9


@pytest.mark.parametrize("k", [1, 7, 60])
def test_intervalo_de_checkpoint(lib_gpu, k):
    """Recomputing from checkpoints every k steps gives the gradient of one tape of the whole run."""
    base = cena_adjunto(passos=60)
    c = dict(base, checkpoint_every=k)
    g0, g1 = AdjuntoGPU(base), AdjuntoGPU(c)
    g0.frente(base["v0"], base["theta0"])
    gv0, gt0 = g0.tras(1.0)
    g1.frente(base["v0"], base["theta0"])
    gv1, gt1 = g1.tras(1.0)
    assert rel_inf(gv1, gv0) <= 1e-9 and rel_inf(gt1, gt0) <= 1e-9
