"""The throughput benchmark's own scene (840x536, 1.25 M particles, labyrinth and faucet) against
the oracle: the GPU runs the scene for two frames with the faucet, its state is copied into the
oracle, and both run one more substep solving to the true residual 1e-6.  Integers bit-exact;
q, u, v to 1e-3 relative; positions to 1e-5 m.  Each oracle substep takes a few seconds.
"""
import numpy as np
import pytest

from estado import INTEIROS, copiar_estado, erro_relativo
from oraculo import CenaOraculo, SimulacaoOraculo
from tanque import Cena, SimulacaoGPU, _abi
from tanque.cenarios import cena_ultra, jato_torneira
from tanque.constantes import CAMPOS

pytestmark = pytest.mark.gpu

SUB = 14


@pytest.mark.parametrize("precond", [_abi.TQ_PRECOND_REFERENCE, _abi.TQ_PRECOND_BLOCK, _abi.TQ_PRECOND_BLOCK_1],
                         ids=["referencia", "bloco", "bloco1"])
def test_subpasso_ultra(lib_gpu, precond):
    opc = {"tolerance": 1e-6, "iterations": 1000, "preconditioner": precond}
    cena_g, _, agua, torneira = cena_ultra(Cena)
    cena_o, _, _, _ = cena_ultra(CenaOraculo)
    assert np.array_equal(np.asarray(cena_g.sdf).view(np.uint32), cena_o.sdf.view(np.uint32))
    g = SimulacaoGPU(cena_g, dict(opc, engine=_abi.TQ_ENGINE_FUSED, precision=_abi.TQ_PREC_FP16))
    g.adicionar(agua, False)
    for q in range(2):
        g.adicionar(jato_torneira(torneira, q, 1 / 60), True)
        g.avancar(1 / 60, SUB)
    o = SimulacaoOraculo(cena_o, dict(opc, p2g_mode=_abi.TQ_P2G_FIXED))
    copiar_estado(g, o)
    o.definirCampo("yBolha", g.campo("yBolha"))
    for s in (o, g):
        s.subpasso(1 / 60 / SUB)
    for campo in INTEIROS:
        a, b = g.campo(campo), o.campo(campo)
        assert np.array_equal(a, b), f"{campo} differs in {np.count_nonzero(a != b)} entries"
    for campo in ["q", "u", "v"]:
        e = erro_relativo(g.campo(campo), o.campo(campo))
        assert e <= 1e-3, f"{campo} relative error {e:.3g}"
    pg, po = g.p.reshape(-1, CAMPOS), o.p.reshape(-1, CAMPOS)
    assert pg.shape == po.shape
    assert float(np.max(np.abs(pg[:, :2].astype(np.float64) - po[:, :2]))) < 1e-5
    for s in (o, g):
        assert s.escalar(_abi.TQ_SCALAR_PCG_CONVERGED) == 1
        assert s.escalar(_abi.TQ_SCALAR_PCG_TRUE_RES) <= 1e-6 * s.escalar(_abi.TQ_SCALAR_PCG_RES0)


def test_erro_ultra_contra_fp64(lib_gpu, capsys):
    """One substep of the bench scene in the mixed configuration against the FP64 oracle (double
    storage everywhere) from the same state: the errors of FP32 arithmetic and FP16 V-cycle
    storage once both solves meet the true 1e-6.  Bound: 1e-3 relative on q, u, v and the
    divergence; bubble volumes exact."""
    from estado import divergencia
    opc = {"tolerance": 1e-6, "iterations": 1000, "preconditioner": _abi.TQ_PRECOND_BLOCK_1}
    cena_g, _, agua, torneira = cena_ultra(Cena)
    cena_o, _, _, _ = cena_ultra(CenaOraculo)
    g = SimulacaoGPU(cena_g, dict(opc, engine=_abi.TQ_ENGINE_FUSED, precision=_abi.TQ_PREC_FP16))
    g.adicionar(agua, False)
    g.adicionar(jato_torneira(torneira, 0, 1 / 60), True)
    g.avancar(1 / 60, SUB)
    o = SimulacaoOraculo(cena_o, dict(opc, p2g_mode=_abi.TQ_P2G_FIXED), fp64=True)
    copiar_estado(g, o)
    o.definirCampo("yBolha", g.campo("yBolha"))
    for s in (o, g):
        s.subpasso(1 / 60 / SUB)
    erros = {c: erro_relativo(g.campo(c), o.campo(c)) for c in ["q", "u", "v"]}
    erros["div"] = erro_relativo(divergencia(g), divergencia(o))
    vb_g, vb_o = g.campo("volumeBolha"), o.campo("volumeBolha")
    ativas = np.nonzero(vb_o)[0]
    with capsys.disabled():
        print("\n840x536 mixed vs FP64 oracle: " + ", ".join(f"{k} {v:.2e}" for k, v in erros.items()))
    assert np.array_equal(vb_g[ativas], vb_o[ativas])
    assert max(erros.values()) <= 1e-3, erros
