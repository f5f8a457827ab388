"""Batched tanks on the GPU: atlases (tanque.lote) against the oracle on the same atlas, for the
FP32 plain engine and the FP16 fused one (also with its skipping of wall blocks forced on every
level): 8 tanks, and 12 wide flat ones whose coarsest multigrid level is large enough for the
coarsest sweeps to run on a whole CTA.  Skipping wall blocks must not change a bit of the
fused solve.

From the same state, one air relabel and two substeps, every pressure solve to
||r|| <= 1e-6 ||r0||: integers bit for bit (particle-to-grid sums, flags, counts, air labels,
bubble ids and volumes), q, u, v to 1e-3 relative, positions to 1e-5 m.  Then the whole batch
helper advances two atlases of the same tanks on the GPU and keeps every particle in its tank.
"""
import numpy as np
import pytest

from estado import comparar_passo, copiar_estado
from oraculo import SimulacaoOraculo
from tanque import Cena, SimulacaoGPU, _abi
from tanque.lote import Lote, gerar_tanques, montar_atlas

pytestmark = pytest.mark.gpu

H = 1 / 128
SOLVE = {"tolerance": 1e-6, "iterations": 200}
MOTORES = [pytest.param({"precision": _abi.TQ_PREC_FP32, "engine": _abi.TQ_ENGINE_PLAIN}, id="fp32-plain"),
           pytest.param({"precision": _abi.TQ_PREC_FP16, "engine": _abi.TQ_ENGINE_FUSED}, id="fp16-fused"),
           pytest.param({"precision": _abi.TQ_PREC_FP16, "engine": _abi.TQ_ENGINE_FUSED, "fused_ctas": 21},
                        id="fp16-fused-21-ctas"),
           pytest.param({"precision": _abi.TQ_PREC_FP16, "engine": _abi.TQ_ENGINE_FUSED, "paredes": True},
                        id="fp16-fused-pulando-paredes")]
# The fused engine skips blocks of wall alone on levels of at least two rounds of its warps;
# a threshold of 1 block (read when a handle is created) makes every grid level skip them.
LIMIAR = "TQ_WALL_SKIP_MIN_BLOCKS"


def _tanques():
    return gerar_tanques(n=8, s=21, h=H, largura=(40, 120), altura=(30, 90))


def _largos():
    """A wide, flat atlas: its coarsest level (238 x 7) has more than 1024 cells, so CTA 0's
    coarsest sweeps run on every warp."""
    return gerar_tanques(n=12, s=22, h=H, largura=(120, 200), altura=(36, 50))


@pytest.mark.parametrize("tanques", [_tanques, _largos], ids=["8-tanques", "largo"])
@pytest.mark.parametrize("opcoes", MOTORES)
def test_atlas_contra_o_oraculo(lib_gpu, opcoes, tanques, monkeypatch):
    opcoes = dict(opcoes)
    if opcoes.pop("paredes", False):
        monkeypatch.setenv(LIMIAR, "1")
    at = montar_atlas(Cena, tanques(), H)
    o = SimulacaoOraculo(at["cena"], dict(SOLVE, p2g_mode=_abi.TQ_P2G_FIXED))
    g = SimulacaoGPU(at["cena"], dict(SOLVE, **opcoes))
    for s in (o, g):
        s.adicionar(at["particulas"], False)
        s.avancar(1 / 240, 1)  # the water is moving before the compared substeps
    copiar_estado(o, g)
    for s in (o, g):
        s.atualizarAr()
    for campo in ["rotulo", "vivo"]:
        assert np.array_equal(g.campo(campo), o.campo(campo)), campo
    for quadro in range(2):
        copiar_estado(o, g)
        o.avancar(1 / 240, 1)
        g.avancar(1 / 240, 1)
        comparar_passo(o, g, f"substep {quadro}")
    g.fechar()


def test_pular_paredes_nao_muda_nada(lib_gpu, monkeypatch):
    """Skipping wall blocks rewrites no value a pass would have written (their cells stay 0),
    so the fused solve gives the same bits with and without it."""
    at = montar_atlas(Cena, _largos(), H)
    sims = []
    for limiar in ["1", "2147483647"]:
        monkeypatch.setenv(LIMIAR, limiar)
        g = SimulacaoGPU(at["cena"], dict(SOLVE, precision=_abi.TQ_PREC_FP16, engine=_abi.TQ_ENGINE_FUSED))
        g.adicionar(at["particulas"], False)
        sims.append(g)
    for _ in range(2):
        for g in sims:
            g.avancar(1 / 240, 2)
        for campo in ["q", "u", "v", "rotulo"]:
            a, b = sims[0].campo(campo), sims[1].campo(campo)
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), campo
        assert np.array_equal(sims[0].p.view(np.uint32), sims[1].p.view(np.uint32))
    for g in sims:
        g.fechar()


def test_lote_no_gpu(lib_gpu):
    t = _tanques()
    lote = Lote(lambda c, o: SimulacaoGPU(c, o), Cena, t, H,
                dict(SOLVE, precision=_abi.TQ_PREC_FP16, engine=_abi.TQ_ENGINE_FUSED), limite_grosso=300)
    assert len(lote.atlas) >= 2
    n0 = [len(lote.particulas(k)) for k in range(len(t))]
    for _ in range(3):
        lote.avancar(1 / 60, 4)
    lote.sincronizar()
    for k in range(len(t)):
        q = lote.particulas(k)
        assert len(q) == n0[k]
        assert np.all(np.isfinite(q[:, :4]))
        assert np.all(q[:, 0] > 0) and np.all(q[:, 0] < t[k]["nx"] * H)
    lote.fechar()


def test_atlas_lado_a_lado(lib_gpu):
    """The atlases' frames side by side: the SMs split between the atlases' fused solves
    (tq_options.fused_ctas) and every frame queued before any is waited for
    (tq_launch_graph).  Against the same batch stepped one atlas at a time on the whole GPU:
    every solve of both converges for every tank, and the particles agree to the solves'
    accuracy (positions to 1e-4 m after two frames; the reductions' order differs with the CTA
    count, so the bits do)."""
    import torch
    t = _tanques()
    opc = dict(SOLVE, iterations=1000, precision=_abi.TQ_PREC_FP16, engine=_abi.TQ_ENGINE_FUSED,
               preconditioner=_abi.TQ_PRECOND_BLOCK)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    lado = Lote(lambda c, o: SimulacaoGPU(c, o), Cena, t, H, opc, limite_grosso=300, sms=sms)
    seq = Lote(lambda c, o: SimulacaoGPU(c, o), Cena, t, H, opc, limite_grosso=300)
    assert lado.ctas is not None and len(lado.ctas) == len(lado.sims) >= 2 and sum(lado.ctas) <= sms
    assert seq.ctas is None
    for lote in (lado, seq):
        for s in lote.sims:
            s.definirEscalar(_abi.TQ_SCALAR_SOLVES, 0)
        for _ in range(2):
            lote.avancar(1 / 60, 4, grafo=True)
        lote.sincronizar()
        for s in lote.sims:
            assert s.escalar(_abi.TQ_SCALAR_SOLVES) == 8
            assert s.escalar(_abi.TQ_SCALAR_SOLVES_CAPPED) == 0
            r = s.residuosTanques()
            agua = r[:, 0] > 0
            assert np.all(r[agua, 1] <= 1e-6 * r[agua, 0])
    for k in range(len(t)):
        a, b = lado.particulas(k), seq.particulas(k)
        assert a.shape == b.shape
        assert float(np.max(np.abs(a[:, :2].astype(np.float64) - b[:, :2]))) < 1e-4
    lado.fechar()
    seq.fechar()


@pytest.mark.parametrize("precond", [_abi.TQ_PRECOND_REFERENCE, _abi.TQ_PRECOND_BLOCK], ids=["referencia", "bloco"])
def test_cada_tanque_converge_sozinho(lib_gpu, precond):
    """With the atlas's tanks registered (tq_set_tanks, done by Lote for the fused engine in
    tolerance mode) every solve stops only when each tank's true residual is within 1e-6 of
    its own initial residual: checked on every tank after every substep of two frames."""
    t = _tanques()
    opc = dict(SOLVE, iterations=1000, precision=_abi.TQ_PREC_FP16, engine=_abi.TQ_ENGINE_FUSED,
               preconditioner=precond)
    lote = Lote(lambda c, o: SimulacaoGPU(c, o), Cena, t, H, opc, limite_grosso=300)
    for _ in range(2):
        for s in lote.sims:
            s.atualizarAr()
            for _ in range(3):
                s.subpasso(1 / 240)
                r = s.residuosTanques()
                assert len(r) > 0
                agua = r[:, 0] > 0
                assert np.all(r[agua, 1] <= 1e-6 * r[agua, 0]), r[agua]
                assert s.escalar(_abi.TQ_SCALAR_PCG_CONVERGED) == 1
    lote.fechar()
