"""Pins the oracle: the reference's own behavioural suite (testes/fisica.test.js,
testes/cena.test.js) run on the CPU restatement, with the reference's bounds.

The reference CPU engine accumulates the particle-to-grid sums in float (TQ_P2G_FLOAT); the
suite runs in that mode and again with the integer sums the CUDA library uses (TQ_P2G_FIXED),
which must meet the same bounds.
"""
import types

import numpy as np
import pytest

import suite_referencia as S
from oraculo import CenaOraculo, SimulacaoOraculo
from tanque import Cena
from tanque import _abi


def fabrica(p2g):
    return types.SimpleNamespace(
        Cena=CenaOraculo,
        sim=lambda cena, opc: SimulacaoOraculo(cena, dict(opc or {}, p2g_mode=p2g)),
    )


MODOS = [pytest.param(_abi.TQ_P2G_FLOAT, id="p2g-float"), pytest.param(_abi.TQ_P2G_FIXED, id="p2g-fixo")]


@pytest.mark.parametrize("p2g", MODOS)
@pytest.mark.parametrize("tensao,limite", [(0.0, 0.01), (None, 0.02)], ids=["sem-tensao", "com-tensao"])
def test_agua_parada(p2g, tensao, limite):
    S.agua_parada(fabrica(p2g), tensao, limite)


@pytest.mark.parametrize("p2g", MODOS)
def test_gota_quadrada(p2g):
    S.gota_quadrada(fabrica(p2g))


@pytest.mark.parametrize("p2g", MODOS)
def test_copo_nao_vaza(p2g):
    S.copo_nao_vaza(fabrica(p2g))


@pytest.mark.parametrize("p2g", MODOS)
def test_pincel_fino_segura_jato(p2g):
    S.pincel_fino_segura_jato(fabrica(p2g))


@pytest.mark.parametrize("p2g", MODOS)
def test_barragem_conserva_volume(p2g):
    S.barragem_conserva_volume(fabrica(p2g))


@pytest.mark.parametrize("p2g", MODOS)
def test_vasos_comunicantes(p2g):
    S.vasos_comunicantes(fabrica(p2g))


@pytest.mark.parametrize("p2g", MODOS)
def test_densidade_de_repouso(p2g):
    S.densidade_de_repouso(fabrica(p2g))


@pytest.mark.parametrize("p2g", MODOS)
def test_bolha_sobe(p2g):
    S.bolha_sobe(fabrica(p2g))


@pytest.mark.parametrize("p2g", MODOS)
def test_remontar_nao_perde_bolha(p2g):
    S.remontar_nao_perde_bolha(fabrica(p2g))


@pytest.mark.parametrize("p2g", MODOS)
def test_sem_ar_buraco_fecha(p2g):
    S.sem_ar_buraco_fecha(fabrica(p2g))


@pytest.mark.parametrize("p2g", MODOS)
def test_ampulheta(p2g):
    S.ampulheta(fabrica(p2g))


# ------------------------------------------------------------------ cena.test.js
@pytest.mark.parametrize("Cn", [CenaOraculo, Cena], ids=["oraculo", "produto"])
def test_cena_moldura(Cn):
    S.cena_moldura(Cn)


@pytest.mark.parametrize("Cn", [CenaOraculo, Cena], ids=["oraculo", "produto"])
def test_cena_distancia(Cn):
    S.cena_distancia(Cn)


@pytest.mark.parametrize("Cn", [CenaOraculo, Cena], ids=["oraculo", "produto"])
def test_cena_apagar(Cn):
    S.cena_apagar(Cn)


@pytest.mark.parametrize("Cn", [CenaOraculo, Cena], ids=["oraculo", "produto"])
def test_cena_incremental(Cn):
    S.cena_incremental(Cn)


def test_cena_produto_igual_ao_oraculo():
    """The host-side scene builder of the package produces the oracle's SDF bit for bit."""
    a, tracos = S.cena_incremental(Cena)
    b = CenaOraculo(70, 50, 0.01)
    for t in tracos:
        b.tracar(t["x0"], t["y0"], t["x1"], t["y1"], t["raio"], t["apagar"])
    assert np.array_equal(a.sdf.view(np.uint32), b.sdf.view(np.uint32))
