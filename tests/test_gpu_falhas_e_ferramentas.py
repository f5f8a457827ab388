"""The device paths outside the substep: particle insertion with the full-cell check, the tools
(sponge, hand, dye), and the fused solver's bounded grid-barrier wait giving up.

Insertion and tools run from the same state in the oracle and on the GPU; particles are
compared bit for bit (both restate js/fisica-cpu.js:92-152 in the reference's double
arithmetic).  The wait test shortens the barrier's limit and holds one CTA back at the first
barrier of one solve (test hooks read from the environment when a handle is created): the
solve returns TQ_E_TIMEOUT, nothing hangs, and the next solve on the same handle is normal.
"""
import numpy as np
import pytest

from estado import CENAS, INTEIROS, copiar_estado, erro_relativo
from oraculo import CenaOraculo, SimulacaoOraculo
from tanque import Cena, SimulacaoGPU, _abi
from tanque.constantes import CAMPOS

pytestmark = pytest.mark.gpu

OPC_FIXO = {"p2g_mode": _abi.TQ_P2G_FIXED}


def par(nome, opcoes=None):
    cena_o, agua = CENAS[nome](CenaOraculo)
    cena_g = Cena(cena_o.nx, cena_o.ny, cena_o.h)
    cena_g.sdf[:] = cena_o.sdf
    o = SimulacaoOraculo(cena_o, dict(OPC_FIXO, **(opcoes or {})))
    g = SimulacaoGPU(cena_g, dict(opcoes or {}))
    o.adicionar(agua, False)
    return o, g


def mesmo_estado(o, g, quadros=2):
    """The oracle runs a few substeps, then its state is copied into g (contagemCelula included)."""
    for _ in range(quadros):
        o.avancar(1 / 60 / 3, 1)
    copiar_estado(o, g)


def bits(a):
    return np.asarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.parametrize("ferramenta", [
    {"tipo": "esponja", "x": 0.12, "y": 0.08, "raio": 0.05},
    {"tipo": "mao", "x": 0.15, "y": 0.10, "raio": 0.07, "vx": 0.8, "vy": -0.3},
    {"tipo": "corante", "x": 0.10, "y": 0.05, "raio": 0.06, "absorcao": (0.3, 1.5, 2.25)},
], ids=["esponja", "mao", "corante"])
def test_ferramenta_paridade(lib_gpu, ferramenta):
    o, g = par("barragem")
    mesmo_estado(o, g)
    n0 = o.n
    o.aplicarFerramenta(ferramenta)
    g.aplicarFerramenta(ferramenta)
    assert g.n == o.n
    if ferramenta["tipo"] == "esponja":
        assert o.n < n0
    assert np.array_equal(bits(g.p), bits(o.p))


def test_adicionar_com_celula_cheia(lib_gpu):
    """adicionar(lista, checarCheia=true) (js/fisica-cpu.js:92-111): particles in walls, outside
    the grid or in cells already holding 3 or more are skipped; the rest keep their order."""
    o, g = par("barragem")
    mesmo_estado(o, g)
    rng = np.random.default_rng(4)
    k = 3000
    lista = np.zeros((k, CAMPOS), np.float32)
    lista[:, 0] = rng.uniform(-0.05, o.nx * o.h + 0.05, k)   # some outside the grid
    lista[:, 1] = rng.uniform(-0.05, o.ny * o.h + 0.05, k)
    lista[:, 2:4] = rng.normal(0, 0.3, (k, 2))
    lista[:, 9:12] = rng.uniform(0, 2, (k, 3))
    a_o = o.adicionar(lista, True)
    a_g = g.adicionar(lista, True)
    assert a_g == a_o and 0 < a_o < k
    assert np.array_equal(bits(g.p), bits(o.p))
    # and without the check, only the wall / inside-SDF filter applies
    b_o = o.adicionar(lista, False)
    b_g = g.adicionar(lista, False)
    assert b_g == b_o and b_o > a_o
    assert np.array_equal(bits(g.p), bits(o.p))


def test_barreira_desiste_e_o_proximo_solve_e_normal(lib_gpu, monkeypatch):
    opc = {"engine": _abi.TQ_ENGINE_FUSED, "tolerance": 1e-6, "iterations": 300}
    monkeypatch.setenv("TQ_BARRIER_WAIT_CYCLES", "2000000")   # ~1 ms at 1.9 GHz
    monkeypatch.setenv("TQ_BARRIER_HOLD_CTA", "3")
    monkeypatch.setenv("TQ_BARRIER_HOLD_CYCLES", "8000000")   # ~4 ms, then it arrives
    o, g = par("bolha", opc)
    for nome in ("TQ_BARRIER_WAIT_CYCLES", "TQ_BARRIER_HOLD_CTA", "TQ_BARRIER_HOLD_CYCLES"):
        monkeypatch.delenv(nome)
    mesmo_estado(o, g)
    with pytest.raises(_abi.ErroTanque) as e:
        g.avancar(1 / 60 / 3, 1)
    assert e.value.status == _abi.TQ_E_TIMEOUT
    # the handle's state after a failed solve is undefined until restored: restore, then the
    # next substep is a normal one, in parity with the oracle
    copiar_estado(o, g)
    o.avancar(1 / 60 / 3, 1)
    g.avancar(1 / 60 / 3, 1)
    for campo in INTEIROS:
        assert np.array_equal(g.campo(campo), o.campo(campo)), campo
    for campo in ["q", "u", "v"]:
        assert erro_relativo(g.campo(campo), o.campo(campo)) <= 1e-4, campo
    assert g.escalar(_abi.TQ_SCALAR_PCG_CONVERGED) == 1


def test_torneira_no_dispositivo(lib_gpu):
    """tq_emit_faucet (emitirTorneira on the device) against the host generator's list through
    tq_add_particles(check_full=1), from the same state: the same count kept and the same
    particles.  Positions to 1e-6 m (the device's cos/sin may round the last double bit
    differently from the host's before the float store); velocity and dye bit-exact."""
    from tanque.cenarios import jato_torneira
    o, g = par("barragem")
    mesmo_estado(o, g)
    g2 = SimulacaoGPU(g.cena, {})
    copiar_estado(o, g2)
    torneira = dict(x=0.3, y=0.32, raio=0.03, vx=0.4, vy=-1.1, h=g.h)
    for quadro in range(3):
        lista = jato_torneira(torneira, quadro, 1 / 60)
        a_host = g.adicionar(lista, True)
        a_disp = g2.emitirTorneira(torneira, 1 / 60, 1000 + quadro)
        assert a_disp == a_host and a_host > 0
        p1, p2 = g.p.reshape(-1, CAMPOS), g2.p.reshape(-1, CAMPOS)
        assert p1.shape == p2.shape
        assert float(np.max(np.abs(p1[:, :2].astype(np.float64) - p2[:, :2]))) <= 1e-6
        assert np.array_equal(bits(p1[:, 2:]), bits(p2[:, 2:]))
