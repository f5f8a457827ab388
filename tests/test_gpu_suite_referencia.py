"""The reference's behavioural suite (testes/fisica.test.js) on the CUDA library, with the
reference's own scenes and bounds (tests/suite_referencia.py, the bodies the oracle is pinned
with).  Two configurations: the FP32 plain engine at the reference's fixed 3 PCG iterations,
and the FP16 fused engine with the block preconditioner solving every substep to 1e-6.
"""
import types

import pytest

import suite_referencia as S
from tanque import Cena, SimulacaoGPU, _abi

pytestmark = pytest.mark.gpu

CONFIGS = {
    "plano-fp32-3it": {"engine": _abi.TQ_ENGINE_PLAIN, "precision": _abi.TQ_PREC_FP32},
    "fundido-fp16-1e-6": {"engine": _abi.TQ_ENGINE_FUSED, "precision": _abi.TQ_PREC_FP16, "tolerance": 1e-6,
                          "iterations": 1000, "preconditioner": _abi.TQ_PRECOND_BLOCK},
}


def fabrica(nome):
    return types.SimpleNamespace(Cena=Cena, sim=lambda cena, opc: SimulacaoGPU(cena, dict(opc or {}, **CONFIGS[nome])))


CFG = [pytest.param(k, id=k) for k in CONFIGS]


@pytest.mark.parametrize("cfg", CFG)
@pytest.mark.parametrize("tensao,limite", [(0.0, 0.01), (None, 0.02)], ids=["sem-tensao", "com-tensao"])
def test_agua_parada(lib_gpu, cfg, tensao, limite):
    S.agua_parada(fabrica(cfg), tensao, limite)


@pytest.mark.parametrize("cfg", CFG)
def test_gota_quadrada(lib_gpu, cfg):
    S.gota_quadrada(fabrica(cfg))


@pytest.mark.parametrize("cfg", CFG)
def test_copo_nao_vaza(lib_gpu, cfg):
    S.copo_nao_vaza(fabrica(cfg))


@pytest.mark.parametrize("cfg", CFG)
def test_pincel_fino_segura_jato(lib_gpu, cfg):
    S.pincel_fino_segura_jato(fabrica(cfg))


@pytest.mark.parametrize("cfg", CFG)
def test_barragem_conserva_volume(lib_gpu, cfg):
    S.barragem_conserva_volume(fabrica(cfg))


@pytest.mark.parametrize("cfg", CFG)
def test_vasos_comunicantes(lib_gpu, cfg):
    S.vasos_comunicantes(fabrica(cfg))


@pytest.mark.parametrize("cfg", CFG)
def test_densidade_de_repouso(lib_gpu, cfg):
    S.densidade_de_repouso(fabrica(cfg))


@pytest.mark.parametrize("cfg", CFG)
def test_bolha_sobe(lib_gpu, cfg):
    S.bolha_sobe(fabrica(cfg))


@pytest.mark.parametrize("cfg", CFG)
def test_remontar_nao_perde_bolha(lib_gpu, cfg):
    S.remontar_nao_perde_bolha(fabrica(cfg))


@pytest.mark.parametrize("cfg", CFG)
def test_sem_ar_buraco_fecha(lib_gpu, cfg):
    S.sem_ar_buraco_fecha(fabrica(cfg))


@pytest.mark.parametrize("cfg", CFG)
def test_ampulheta(lib_gpu, cfg):
    S.ampulheta(fabrica(cfg))
