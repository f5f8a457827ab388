"""CPU checks of the boundary: libtanque.so loads, exports every entry point include/tanque.h
declares, the ctypes layouts match the header, and argument errors are reported (no GPU needed:
only calls that fail before touching a device are made)."""
import ctypes as C
import os
import re

import pytest

from tanque import _abi

RAIZ = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(RAIZ, "include", "tanque.h")


def _declaradas():
    texto = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(tq_[a-z_]+)\s*\(", texto, re.M)))


def test_biblioteca_exporta_tudo():
    lib = C.CDLL(_abi.CAMINHO_LIB)
    nomes = _declaradas()
    assert len(nomes) >= 25
    faltam = [n for n in nomes if not hasattr(lib, n)]
    assert not faltam, f"not exported: {faltam}"


def test_oraculo_espelha_a_interface():
    """The oracle exports the tq_ simulation entry points under tqo_ (parity tests drive both)."""
    lib = C.CDLL(os.path.join(RAIZ, "oracle", "liboracle.so"))
    for nome in _abi.ASSINATURAS:
        assert hasattr(lib, "tqo_" + nome), nome


def test_layout_das_estruturas():
    assert C.sizeof(_abi.TqOptions) == 112
    assert _abi.TqOptions.h.offset == 8
    assert _abi.TqOptions.gravity.offset == 16
    assert _abi.TqOptions.tolerance.offset == 56
    assert _abi.TqOptions.preconditioner.offset == 84
    assert C.sizeof(_abi.TqSolveInfo) == 40
    assert C.sizeof(_abi.TqFaucet) == 80
    assert C.sizeof(_abi.TqAdjScene) == 96
    assert _abi.TqAdjScene.n_particles.offset == 88
    assert C.sizeof(_abi.TqTool) == 72
    assert C.sizeof(_abi.TqBubbles) == 24


def test_erros_de_argumento_sem_gpu():
    lig = _abi.carregar()
    o = _abi.opcoes_padrao(2, 2, 0.01)  # grid too small: rejected before any CUDA call
    h = C.c_void_p()
    with pytest.raises(_abi.ErroTanque) as e:
        lig("create", C.byref(o), C.byref(h))
    assert e.value.status == _abi.TQ_E_ARG
    with pytest.raises(_abi.ErroTanque) as e:
        lig("advance", None, 1 / 60, 1)
    assert e.value.status == _abi.TQ_E_ARG
    o = _abi.opcoes_padrao(10, 10, 0.01, p2g_mode=_abi.TQ_P2G_FLOAT)
    with pytest.raises(_abi.ErroTanque) as e:
        lig("create", C.byref(o), C.byref(h))
    assert e.value.status == _abi.TQ_E_ARG
    assert lig.lib.tq_status_string(_abi.TQ_E_TIMEOUT)


def test_gravidade_escalar_no_oraculo():
    """TQ_SCALAR_GRAVITY_X/Y read back what was set (oracle side of the mirrored surface)."""
    from oraculo import CenaOraculo, SimulacaoOraculo
    o = SimulacaoOraculo(CenaOraculo(20, 16, 0.01))
    assert o.gravidade == (0.0, -9.81)
    o.gravidade = (1.5, -2.0)
    assert o.gravidade == (1.5, -2.0)
    o.fechar()
