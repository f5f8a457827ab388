"""SimulacaoGPU: the reference's `SimulacaoCPU` surface (js/fisica-cpu.js:28-671) over the C-ABI.

Method and field names are the JavaScript ones, so code written against SimulacaoCPU (the
reference's tests, MotorCPU) reads the same here.  Fields are copied out of the device on
access; the handle owns the device state.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .constantes import CAMPOS, ITERACOES_PCG, MAX_BOLHAS, PARTICULAS_POR_CELULA, TAU_DENSIDADE, TENSAO_SUPERFICIAL

_FERRAMENTAS = {"nenhuma": 0, "esponja": 1, "mao": 2, "corante": 3}


class Simulacao:
    """Drives any library exporting the tq_* entry points (or a prefixed mirror of them)."""

    _DTYPES = {
        "tipo": np.uint8, "solidoCelula": np.uint8, "vivo": np.uint8, "uValida": np.uint8, "vValida": np.uint8,
        "rotulo": np.uint32, "contagemCelula": np.uint32, "accU": np.int32, "accV": np.int32, "accCel": np.int32,
        "accCor": np.int32,
    }

    def __init__(self, ligacao: _abi.Ligacao, cena, opcoes: dict | None = None, criar: str = "create"):
        opcoes = dict(opcoes or {})
        self._lig = ligacao
        self.cena = cena
        self.nx, self.ny, self.h = cena.nx, cena.ny, cena.h
        self.nu = (self.nx + 1) * self.ny
        self.nv = self.nx * (self.ny + 1)
        g = opcoes.pop("gravidade", None)
        tensao = opcoes.pop("tensao", None)
        o = _abi.opcoes_padrao(
            self.nx, self.ny, self.h,
            iterations=opcoes.pop("iteracoes", ITERACOES_PCG),
            air=1 if opcoes.pop("ar", True) else 0,
            tau_density=opcoes.pop("tauDensidade", TAU_DENSIDADE),
            surface_tension=TENSAO_SUPERFICIAL if tensao is None else tensao,
        )
        if g is not None:
            o.gravity[0], o.gravity[1] = g
        for k, v in opcoes.items():  # tq_options field names (tolerance, precision, engine, ...)
            if k == "gravity":
                o.gravity[0], o.gravity[1] = v
            else:
                setattr(o, k, v)
        self.opcoes = o
        self.arAtivo = bool(o.air)
        h = C.c_void_p()
        self._lig(criar, C.byref(o), C.byref(h))
        self._h = h
        self.atualizarParedes()

    # ---------------------------------------------------------------- lifecycle
    def fechar(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lig("destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.fechar()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.fechar()

    # ---------------------------------------------------------------- SimulacaoCPU surface
    @property
    def gravidade(self):
        return (self.escalar(_abi.TQ_SCALAR_GRAVITY_X), self.escalar(_abi.TQ_SCALAR_GRAVITY_Y))

    @gravidade.setter
    def gravidade(self, g):
        """sim.gravidade = [gx, gy] (MotorCPU.gravidade, js/motor.js:96): used from the next substep."""
        self.definirEscalar(_abi.TQ_SCALAR_GRAVITY_X, float(g[0]))
        self.definirEscalar(_abi.TQ_SCALAR_GRAVITY_Y, float(g[1]))

    def atualizarParedes(self):
        """atualizarParedes (js/fisica-cpu.js:80-85) after Cena edits: upload the SDF."""
        sdf = np.ascontiguousarray(self.cena.sdf, dtype=np.float32)
        self._lig("set_walls", self._h, sdf.ctypes.data, self.cena.mw, self.cena.mh)

    def adicionar(self, lista, checarCheia: bool = True) -> int:
        """adicionar (js/fisica-cpu.js:92-111); returns the number of particles kept."""
        a = np.ascontiguousarray(lista, dtype=np.float32).ravel()
        n = a.size // CAMPOS
        aceitas = C.c_int32(0)
        self._lig("add_particles", self._h, a.ctypes.data, n, 1 if checarCheia else 0, C.byref(aceitas))
        return aceitas.value

    def aplicarFerramenta(self, f: dict | None):
        """aplicarFerramenta (js/fisica-cpu.js:129-152)."""
        if not f or f.get("tipo", "nenhuma") == "nenhuma":
            return
        t = _abi.TqTool()
        t.kind = _FERRAMENTAS[f["tipo"]]
        t.x, t.y, t.radius = f["x"], f["y"], f["raio"]
        t.vx, t.vy = f.get("vx", 0.0), f.get("vy", 0.0)
        ab = f.get("absorcao", (0.0, 0.0, 0.0))
        t.absorb[0], t.absorb[1], t.absorb[2] = ab
        self._lig("apply_tool", self._h, C.byref(t))

    def avancar(self, dt: float, subpassos: int = 1):
        """avancar (js/fisica-cpu.js:155-159)."""
        self._lig("advance", self._h, float(dt), int(subpassos))
        self._andou = True

    def lancarGrafo(self, dt: float, subpassos: int = 1):
        """avancarGrafo without waiting for the frame (tq_launch_graph); sincronizar() waits
        and reports a solve that gave up."""
        self._lig("launch_graph", self._h, float(dt), int(subpassos))
        self._andou = True

    def avancarGrafo(self, dt: float, subpassos: int = 1):
        """avancar with the substeps replayed from a CUDA graph (tq_advance_graph): same bits."""
        self._lig("advance_graph", self._h, float(dt), int(subpassos))
        self._andou = True

    def atualizarAr(self):
        self._lig("update_air", self._h)

    def reiniciarAr(self):
        self._lig("reset_air", self._h)

    def subpasso(self, dt: float):
        self._lig("substep", self._h, float(dt))
        self._andou = True

    def area(self) -> float:
        """area (js/fisica-cpu.js:192-194): water area in m^2 from the particle count."""
        return (self.n / PARTICULAS_POR_CELULA) * self.h * self.h

    def limparAgua(self):
        """MotorCPU.limparAgua (js/motor.js:95)."""
        self._lig("clear_particles", self._h)
        self.reiniciarAr()

    @property
    def n(self) -> int:
        v = C.c_int32(0)
        self._lig("count", self._h, C.byref(v))
        return v.value

    @n.setter
    def n(self, valor: int):
        # The reference's tests empty the tank with `sim.n = 0` (testes/fisica.test.js:235).
        if valor != 0:
            raise ValueError("only sim.n = 0 is supported; use definirParticulas")
        self._lig("clear_particles", self._h)

    @property
    def p(self) -> np.ndarray:
        """sim.p.subarray(0, n*CAMPOS) in the reference's particle order."""
        n = self.n
        out = np.empty(n * CAMPOS, dtype=np.float32)
        m = C.c_int32(0)
        self._lig("get_particles", self._h, out.ctypes.data if n else None, n, C.byref(m))
        return out[: m.value * CAMPOS]

    def definirParticulas(self, lista):
        a = np.ascontiguousarray(lista, dtype=np.float32).ravel()
        self._lig("set_particles", self._h, a.ctypes.data if a.size else None, a.size // CAMPOS)

    def _tamanho(self, nome: str) -> int:
        N = self.nx * self.ny
        tam = {
            "u": self.nu, "v": self.nv, "uValida": self.nu, "vValida": self.nv, "uPeso": self.nu, "vPeso": self.nv,
            "pressaoBolha": MAX_BOLHAS, "volumeAlvo": MAX_BOLHAS, "volumeBolha": MAX_BOLHAS, "rhsBolha": MAX_BOLHAS,
            "yBolha": MAX_BOLHAS, "vivo": MAX_BOLHAS, "corCelula": 3 * N, "accCor": 3 * N, "accU": 2 * self.nu,
            "accV": 2 * self.nv, "accCel": 2 * N, "sdf": 4 * N,
        }
        return tam.get(nome, N)

    def campo(self, nome: str) -> np.ndarray:
        """Copy of a state field (names of include/tanque.h's tq_field, as in the JavaScript)."""
        dt = self._DTYPES.get(nome, np.float32)
        out = np.empty(self._tamanho(nome), dtype=dt)
        self._lig("get_field", self._h, _abi.CAMPOS_ENUM[nome], out.ctypes.data, out.nbytes)
        return out

    def definirCampo(self, nome: str, valores):
        dt = self._DTYPES.get(nome, np.float32)
        a = np.ascontiguousarray(valores, dtype=dt).ravel()
        self._lig("set_field", self._h, _abi.CAMPOS_ENUM[nome], a.ctypes.data, a.nbytes)

    def escalar(self, qual: int) -> float:
        v = C.c_double(0)
        self._lig("get_scalar", self._h, qual, C.byref(v))
        return v.value

    def definirEscalar(self, qual: int, valor: float):
        self._lig("set_scalar", self._h, qual, float(valor))

    def normas(self) -> np.ndarray:
        n = C.c_int32(0)
        buf = (C.c_double * 1024)()
        self._lig("last_norms", self._h, buf, 1024, C.byref(n))
        return np.array(buf[: n.value])

    @property
    def vMax(self):
        """Largest particle speed of the last G2P; None before the first substep (the
        reference's field is undefined until then, js/fisica-cpu.js:637)."""
        if not getattr(self, "_andou", False):
            return None
        return self.escalar(_abi.TQ_SCALAR_VMAX)

    # typed-array fields the reference's tests and facade read (testes/fisica.test.js, js/motor.js)
    tipo = property(lambda self: self.campo("tipo"))
    rotulo = property(lambda self: self.campo("rotulo"))
    contagemCelula = property(lambda self: self.campo("contagemCelula"))
    solidoCelula = property(lambda self: self.campo("solidoCelula"))
    q = property(lambda self: self.campo("q"))
    u = property(lambda self: self.campo("u"))
    v = property(lambda self: self.campo("v"))
    pressaoBolha = property(lambda self: self.campo("pressaoBolha"))


class SimulacaoGPU(Simulacao):
    """`new SimulacaoCPU(cena, opcoes)` on the B200 (libtanque.so)."""

    def __init__(self, cena, opcoes: dict | None = None):
        super().__init__(_abi.carregar(), cena, opcoes)

    def sincronizar(self):
        self._lig("sync", self._h)

    def definirTanques(self, retangulos):
        """The tanks of an atlas (tq_set_tanks): (x0, y0, largura, altura) in cells each, in
        disjoint column ranges.  In tolerance mode every tank's own true residual must then meet
        the tolerance of its own initial residual.  Fused engine only."""
        r = np.ascontiguousarray(np.asarray(retangulos, dtype=np.int32).reshape(-1, 4))
        self._lig("set_tanks", self._h, len(r), r.ctypes.data if len(r) else None)

    def residuosTanques(self) -> np.ndarray:
        """(tanks, 2): ||r0|| and the true ||r|| of each tank at the last solve's end."""
        n = C.c_int32(0)
        self._lig("get_tank_residuals", self._h, None, 0, C.byref(n))
        buf = (C.c_double * (2 * max(n.value, 1)))()
        self._lig("get_tank_residuals", self._h, buf, 2 * n.value, C.byref(n))
        return np.array(buf[: 2 * n.value]).reshape(-1, 2)

    def emitirTorneira(self, torneira: dict, dt: float, semente: int, absorcao=(0.0, 0.0, 0.0)) -> int:
        """emitirTorneira (js/principal.js:301-321) on the device (tq_emit_faucet): the jet of
        `torneira` (x, y, raio, vx, vy) for `dt` seconds, the LCG seeded with `semente` in place
        of Math.random, through adicionar(lista, true).  Returns the particles kept."""
        f = _abi.TqFaucet()
        f.x, f.y, f.radius = torneira["x"], torneira["y"], torneira["raio"]
        f.vx, f.vy, f.dt = torneira["vx"], torneira["vy"], float(dt)
        f.absorb[0], f.absorb[1], f.absorb[2] = absorcao
        f.seed = int(semente) & 0xFFFFFFFF
        aceitas = C.c_int32(0)
        self._lig("emit_faucet", self._h, C.byref(f), C.byref(aceitas))
        return aceitas.value

    def tracarParede(self, x0, y0, x1, y1, raio, apagar: bool = False):
        """Cena.tracar (js/cena.js:43-72) + atualizarParedes on the device mask (tq_trace_wall).
        The handle's mask then differs from self.cena's until the scene draws the same segment."""
        self._lig("trace_wall", self._h, float(x0), float(y0), float(x1), float(y1), float(raio), 1 if apagar else 0)

    def limparParedes(self):
        """Cena.limpar (js/cena.js:74-77) + atualizarParedes on the device (tq_clear_walls)."""
        self._lig("clear_walls", self._h)

    def mancha(self, largura: int, altura: int, saida=None):
        """The renderer's particle splat (WGSL_MANCHA, tq_splat) as a (5, altura, largura) array:
        sum of weights, weight x foam, weight x the three absorptions; row 0 at the top.  With
        `saida` (a CUDA torch tensor of 5 * largura * altura float32) the image stays on the
        device and `saida` is returned."""
        import torch
        buf = saida if saida is not None else torch.empty(5 * largura * altura, dtype=torch.float32, device="cuda")
        if buf.dtype != torch.float32 or not buf.is_cuda or buf.numel() != 5 * largura * altura:
            raise ValueError("saida must be a CUDA float32 tensor of 5 * largura * altura elements")
        self._lig("splat", self._h, largura, altura, buf.data_ptr())
        return buf if saida is not None else buf.cpu().numpy().reshape(5, altura, largura)

    ETAPAS = ["p2g", "tipos_rotulos", "superficie", "divergencia_bolhas", "pressao", "gradiente_extrapolacao", "g2p"]

    def tempos(self, ligar: bool | None = None):
        """Stage timing (CUDA events on the handle's stream).  `ligar=True` starts/resets the
        accumulation; without arguments returns the totals since then (ms per stage, air
        relabel ms, substeps, pressure iterations, relabels)."""
        if ligar is not None:
            self._lig("set_timing", self._h, 1 if ligar else 0)
            return None
        n = C.c_int32(0)
        buf = (C.c_double * 16)()
        self._lig("get_timing", self._h, buf, 16, C.byref(n))
        v = list(buf[: n.value])
        out = {e: v[i] for i, e in enumerate(self.ETAPAS)}
        out.update(ar=v[7], subpassos=int(v[8]), iteracoes=int(v[9]), reetiquetagens=int(v[10]))
        return out

    def stream(self) -> int:
        """The handle's cudaStream_t (as an integer), for torch.cuda.ExternalStream."""
        p = C.c_void_p()
        self._lig("get_stream", self._h, C.byref(p))
        return p.value or 0

    @staticmethod
    def lancamentos() -> int:
        """Kernels launched by this process so far (all handles)."""
        lig = _abi.carregar()
        v = C.c_double(0)
        lig.f["get_scalar"](None, _abi.TQ_SCALAR_LAUNCHES, C.byref(v))
        return int(v.value)


def resolver_pressao(tipo, div, q, iteracoes=ITERACOES_PCG, tolerancia=0.0, bolhas=None, precisao=0, motor=0,
                     precond=0, info: dict | None = None, ligacao: _abi.Ligacao | None = None):
    """resolverPCG (js/pressao-cpu.js:296-402) through tq_solve_pressure; q is updated in place.

    bolhas: optional dict(rotulo=uint32[N], rhs=float32[4096], y=float32[4096]); y is updated.
    precond: TQ_PRECOND_*.  info: optional dict, filled with tq_solve_info's fields.
    Returns the residual-norm history."""
    lig = ligacao or _abi.carregar()
    ny, nx = tipo.shape
    tipo = np.ascontiguousarray(tipo, dtype=np.uint8)
    div = np.ascontiguousarray(div, dtype=np.float32)
    assert q.dtype == np.float32 and q.flags.c_contiguous
    b = None
    if bolhas is not None:
        b = _abi.TqBubbles()
        b.rotulo = bolhas["rotulo"].ctypes.data
        b.rhs = bolhas["rhs"].ctypes.data
        b.y = bolhas["y"].ctypes.data
    normas = (C.c_double * 1024)()
    nn = C.c_int32(0)
    args = [nx, ny, tipo.ctypes.data, div.ctypes.data, q.ctypes.data, iteracoes, tolerancia,
            C.byref(b) if b is not None else None]
    if lig.prefixo == "tq_":
        args += [precisao, motor]
    inf = _abi.TqSolveInfo()
    args += [precond, normas, 1024, C.byref(nn), C.byref(inf)]
    lig("solve_pressure", *args)
    if info is not None:
        info.update({k: getattr(inf, k) for k, _ in _abi.TqSolveInfo._fields_})
    return np.array(normas[: nn.value])


def ciclo_v(tipo, b, precisao=0, ligacao: _abi.Ligacao | None = None) -> np.ndarray:
    """cicloV (js/pressao-cpu.js:241-255) through tq_vcycle: one V-cycle from x = 0."""
    lig = ligacao or _abi.carregar()
    ny, nx = tipo.shape
    tipo = np.ascontiguousarray(tipo, dtype=np.uint8)
    b = np.ascontiguousarray(b, dtype=np.float32)
    x = np.zeros_like(b)
    args = [nx, ny, tipo.ctypes.data, b.ctypes.data, x.ctypes.data]
    if lig.prefixo == "tq_":
        args.append(precisao)
    lig("vcycle", *args)
    return x
