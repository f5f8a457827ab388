#!/usr/bin/env python
"""Throughput of the tank's simulation step on the 450k-cell ultra scene (B200).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: 840x536 MAC grid, h = 1.6 mm, a seeded labyrinth (8-cell corridors, 4-cell walls)
in the upper half of the tank, water up to 85 % of the height, a faucet jet 12 cells wide at
1.2 m/s at the labyrinth's entrance, surface tension 0.0728 N/m, air pockets tracked.  A bench
step is one simulated 1/60 s frame: one air relabel and 14 substeps of 1/840 s (below the
capillary limit of 1.197 ms at this h).  Every pressure solve runs to ||r|| <= 1e-6 ||r0||.
The metric is substeps per second.

Every pressure solve stops on the TRUE residual ||b - A q|| <= 1e-6 ||r0|| (FP64, q accumulated in
FP64), with an iteration cap of 1000; each arm reports the fraction of its solves that converged
and the largest true relative residual.  `value` is the mixed-precision configuration (fused
engine, FP16 V-cycle storage, block preconditioner, frames replayed from a CUDA graph) timed on
the device, the faucet's particles made on the device each frame (tq_emit_faucet); `fp32_fused` is the
same engine with FP32 storage; `fp32_plain` is the one-launch-per-step FP32 engine with the
reference's preconditioner (the reference's algorithm on the GPU); `e2e` is the mixed
configuration through the C-ABI with host buffers (faucet particles in, every particle out, each
frame; the device-timed arms make the same jet on the device, tq_emit_faucet).  --impl reference
times the CPU oracle (the reference engine's algorithm restated in C++,
single-threaded as the reference is) on the same scene.
With --gpus N > 1 each rank (relaunched under torch.distributed.run when WORLD_SIZE is unset)
advances its own replica (a tank does not shard).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

RAIZ = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(RAIZ, "tanque-de-agua_b200"),):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "steps/s @450k cells & MGPCG HBM GB/s: mixed vs FP32 plain at 1e-6 residual"
NX, NY, H = 840, 536, 0.0016
SUB = 14
DT_QUADRO = 1 / 60
TOL = 1e-6
MAX_ITER = 1000
# Algorithmic HBM bytes of one PCG iteration per fine cell (5-point operator, V-cycle with
# 4 smoother passes per level, restriction and prolongation, dots and vector updates) for
# FP32 V-cycle storage and for 16-bit storage, plus the setup of a solve (initial residual,
# first V-cycle).
BYTES_ITER = {"fp32": 156.0, "fp16": 120.0, "bf16": 120.0}
BYTES_SETUP = {"fp32": 110.0, "fp16": 85.0, "bf16": 85.0}
# TQ_PRECOND_BLOCK_1's V-cycle takes one smoother pass a leg on the levels above 0, whose
# cells add up to a third of level 0's: per fine cell its V-cycle moves 71 + (2*13 + 10 + 9) / 3
# = 86 B instead of 71 * 4/3 = 94.7 (FP32), 38 + (2*7 + 5.5 + 4.5) / 3 = 46 B instead of
# 38 * 4/3 = 50.7 (16-bit).
BYTES_ITER_BLOCO = {"fp32": 147.3, "fp16": 115.3, "bf16": 115.3}
BYTES_SETUP_BLOCO = {"fp32": 101.3, "fp16": 80.3, "bf16": 80.3}
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one fused FP16 solve of this
# scene with TQ_PRECOND_BLOCK_1, from one ncu capture of the kernel: the solve's working set
# stays in L2.
TRAFEGO_SOLVE_BYTES = 17_849_856
# Particle bytes a substep's particle kernels move per particle: P2G reads its three float4
# records (position/velocity, affine terms, foam/dye); G2P reads the first and third and
# writes all three.  The grid reads behind them are cached (L1/L2) and not counted.
BYTES_PARTICULA = {"p2g": 48, "g2p": 80}


def picos():
    try:
        with open(os.path.join(RAIZ, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------ scene
def construir_cena(Cena, *_):
    """Walls and water of the ultra scene (tanque.cenarios.cena_ultra): (cena, traces, particles, faucet)."""
    from tanque.cenarios import cena_ultra
    return cena_ultra(Cena, NX, NY, H)


def jato(torneira, quadro, dt=DT_QUADRO):
    """The faucet's particles of frame `quadro` (tanque.cenarios.jato_torneira)."""
    from tanque.cenarios import jato_torneira
    return jato_torneira(torneira, quadro, dt)


# ------------------------------------------------------------------ clocks
class Relogios:
    """nvidia-smi sampling during the timed region (clocks and throttle reasons)."""

    CAMPOS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, indice):
        self.indice = indice
        self.proc = None
        self.saida = None

    def __enter__(self):
        try:
            self.saida = open(os.devnull if False else f"/tmp/tq_clocks_{os.getpid()}.csv", "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.indice}", f"--query-gpu={self.CAMPOS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.saida, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.saida:
            self.saida.close()

    def resumo(self):
        try:
            linhas = [l.split(",") for l in open(self.saida.name).read().strip().splitlines() if l.strip()]
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(l[1]) for l in linhas if len(l) >= 9]
        mx = [float(l[2]) for l in linhas if len(l) >= 9]
        razoes = set()
        nomes = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in linhas:
            if len(l) < 9:
                continue
            for nome, v in zip(nomes, l[5:9]):
                if v.strip().lower() == "active":
                    razoes.add(nome)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sob_carga = [v for v in sm if v > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(sob_carga), "sm_max_mhz": max(mx), "reasons": sorted(razoes),
                "samples": len(sm)}


# ------------------------------------------------------------------ CPU oracle
def medir_oraculo(passos, aquecimento, orcamento_s=None):
    """Substeps/s of the CPU oracle (reference CPU semantics: float P2G sums) on the scene."""
    sys.path.insert(0, os.path.join(RAIZ, "tests"))
    from oraculo import CenaOraculo, SimulacaoOraculo
    from tanque import _abi
    from tanque.cenarios import labirinto, semear_retangulo_rapido, semente
    cena, _, agua, _ = construir_cena(CenaOraculo, semente, labirinto, semear_retangulo_rapido)
    sim = SimulacaoOraculo(cena, {"p2g_mode": _abi.TQ_P2G_FLOAT, "tolerance": TOL, "iterations": MAX_ITER})
    sim.adicionar(agua, False)
    n_part = sim.n
    dt = DT_QUADRO / SUB
    sim.atualizarAr()
    for _ in range(aquecimento):
        sim.subpasso(dt)
    feitos = 0
    t0 = time.perf_counter()
    while feitos < passos:
        sim.subpasso(dt)
        feitos += 1
        if orcamento_s is not None and time.perf_counter() - t0 > orcamento_s:
            break
    t = time.perf_counter() - t0
    return feitos / t, feitos, n_part


def medir_oraculo_lote(orcamento_s=20.0):
    """Tank-substeps/s of the CPU oracle on the 256-tank batch: the tanks in seed order, each a
    scene of its own, one substep each in turn until the time budget is spent."""
    sys.path.insert(0, os.path.join(RAIZ, "tests"))
    from oraculo import SimulacaoOraculo
    from tanque import Cena, _abi, passo_maximo
    from tanque.cenarios import semear_retangulo_rapido
    from tanque.lote import gerar_tanques
    todos = gerar_tanques(h=LOTE_H)
    dt = DT_QUADRO / math.ceil(DT_QUADRO / passo_maximo(LOTE_H, max(t["ny"] for t in todos) * LOTE_H) - 1e-9)
    sims, feitos, t0 = [], 0, time.perf_counter()
    tempo = 0.0
    for t in todos:
        cena = Cena(t["nx"], t["ny"], LOTE_H)
        for tr in t["tracos"]:
            cena.tracar(tr["x0"], tr["y0"], tr["x1"], tr["y1"], tr["raio"])
        sim = SimulacaoOraculo(cena, {"p2g_mode": _abi.TQ_P2G_FLOAT, "tolerance": TOL, "iterations": MAX_ITER})
        sim.adicionar(semear_retangulo_rapido(*t["agua"], LOTE_H, s=t["semente"]), False)
        sim.atualizarAr()
        sim.subpasso(dt)  # warm-up
        a = time.perf_counter()
        sim.subpasso(dt)
        tempo += time.perf_counter() - a
        feitos += 1
        if time.perf_counter() - t0 > orcamento_s:
            break
    return feitos / tempo, feitos


# ------------------------------------------------------------------ replicas
def tempos_max_ranks(tempos, dist, dispositivo):
    """This rank's device times (ms) -> their maximum over the ranks, on every rank: the job's time
    is its slowest replica's."""
    t = np.asarray(tempos, dtype=np.float64)
    if dist is None:
        return t
    import torch
    tt = torch.tensor(t, device=dispositivo)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return tt.cpu().numpy()


def vazao_replicas(mundo, passos, subpassos, ms):
    """Whole-job substeps per second: each of the `mundo` ranks advanced its own tank (a replica;
    a tank does not shard) through `passos` frames of `subpassos` substeps in `ms`."""
    return mundo * passos * subpassos / (ms / 1000.0)


# ------------------------------------------------------------------ GPU arm
def estatisticas_solve(s):
    """Convergence record of the handle's solves since the last reset (device counters)."""
    from tanque import _abi
    n = s.escalar(_abi.TQ_SCALAR_SOLVES)
    cap = s.escalar(_abi.TQ_SCALAR_SOLVES_CAPPED)
    return {"solves": int(n), "converged_frac": round(1.0 - cap / n, 4) if n else None,
            "max_true_rel_residual": s.escalar(_abi.TQ_SCALAR_SOLVE_MAX_REL),
            "mean_iters": round(s.escalar(_abi.TQ_SCALAR_SOLVE_ITERS) / n, 2) if n else None,
            "replacements": int(s.escalar(_abi.TQ_SCALAR_SOLVE_REPLACEMENTS))}


def executar_gpu(args, rank, mundo, dist):
    import torch
    from tanque import Cena, SimulacaoGPU, _abi
    from tanque.cenarios import labirinto, semear_retangulo_rapido, semente

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    cena, _, agua, torneira = construir_cena(Cena, semente, labirinto, semear_retangulo_rapido)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    hbm, origem_pico = picos()
    # the faucet's particles of every frame, in pinned host memory (the jet is the scene's input)
    jatos = []
    for q in range(args.warmup + args.steps):
        j = jato(torneira, q)
        buf = torch.empty(j.size, dtype=torch.float32, pin_memory=True).numpy()
        buf[:] = j
        jatos.append(buf)

    def nova(precisao, motor, precond):
        s = SimulacaoGPU(cena, {"tolerance": TOL, "iterations": MAX_ITER, "precision": precisao, "engine": motor,
                                "preconditioner": precond, "device": dev})
        s.adicionar(agua, False)
        return s

    def barreira():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def medir(precisao, motor, precond, grafo=False, etapas=False, com_relogio=False, e2e=False):
        """Frames of the scene with the faucet: warm-up, then `steps` timed frames with CUDA
        events on the handle's stream (L2 flushed before each, outside the events).  e2e adds
        the read-back of every particle to the host inside the events."""
        import ctypes as C
        s = nova(precisao, motor, precond)
        ext = torch.cuda.ExternalStream(s.stream())
        avancar = s.avancarGrafo if grafo else s.avancar
        lig = _abi.carregar()
        cap = s.opcoes.capacity or math.ceil(NX * NY * 4.6)
        saida = torch.empty(cap * 12, dtype=torch.float32, pin_memory=True).numpy() if e2e else None
        for q in range(args.warmup):
            if e2e:
                s.adicionar(jatos[q], True)
            else:
                s.emitirTorneira(torneira, DT_QUADRO, 1000 + q)
            avancar(DT_QUADRO, SUB)
        s.sincronizar()
        barreira()
        s.definirEscalar(_abi.TQ_SCALAR_SOLVES, 0)
        if etapas:
            s.tempos(True)
        l0 = SimulacaoGPU.lancamentos()
        eventos, h2d, d2h = [], 0, 0
        rel = Relogios(dev) if com_relogio else None
        if rel:
            rel.__enter__()
        for q in range(args.steps):
            with torch.cuda.stream(ext):
                flush.zero_()  # L2 flush between timed steps (outside the events)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            ent = jatos[args.warmup + q]
            if e2e:  # the drop-in path: the host's jet list crosses to the device
                s.adicionar(ent, True)
                h2d += ent.nbytes
            else:  # inputs resident: the same jet made on the device (tq_emit_faucet)
                s.emitirTorneira(torneira, DT_QUADRO, 1000 + args.warmup + q)
            avancar(DT_QUADRO, SUB)
            if e2e:
                n = C.c_int32(0)
                lig("get_particles", s._h, saida.ctypes.data, cap, C.byref(n))
                d2h += n.value * 48
            e1.record(ext)
            eventos.append((e0, e1))
        s.sincronizar()
        torch.cuda.synchronize()
        if rel:
            rel.__exit__()
        res = dict(ms=sum(a.elapsed_time(b) for a, b in eventos), lancamentos=SimulacaoGPU.lancamentos() - l0,
                   particulas=s.n, relogios=rel.resumo() if rel else None, solve=estatisticas_solve(s),
                   etapas=s.tempos() if etapas else None, h2d=h2d / args.steps, d2h=d2h / args.steps)
        s.fechar()
        return res

    FUSED, PLAIN = _abi.TQ_ENGINE_FUSED, _abi.TQ_ENGINE_PLAIN
    # the block preconditioner with one smoother pass a leg above level 0: the faster of the two
    # block cycles on this latency-bound scene (the batch's large atlases take TQ_PRECOND_BLOCK)
    BLOCO, REF = _abi.TQ_PRECOND_BLOCK_1, _abi.TQ_PRECOND_REFERENCE
    misto = medir(_abi.TQ_PREC_FP16, FUSED, BLOCO, grafo=True, com_relogio=True)
    misto_etapas = medir(_abi.TQ_PREC_FP16, FUSED, BLOCO, etapas=True)
    fundido32 = medir(_abi.TQ_PREC_FP32, FUSED, BLOCO, grafo=True)
    plano = medir(_abi.TQ_PREC_FP32, PLAIN, REF, etapas=True)
    e2e = medir(_abi.TQ_PREC_FP16, FUSED, BLOCO, grafo=True, e2e=True)

    tempos = tempos_max_ranks([misto["ms"], fundido32["ms"], plano["ms"], e2e["ms"]], dist, "cuda")
    valor, valor_f32, valor_plano, valor_e2e = (vazao_replicas(mundo, args.steps, SUB, t) for t in tempos)

    def roofline(res, rotulo, bloco=False):
        et = res["etapas"]
        n_sub = max(et["subpassos"], 1)
        iters = et["iteracoes"] / n_sub
        t_solve = et["pressao"] / n_sub / 1000
        bi, bs = (BYTES_ITER_BLOCO, BYTES_SETUP_BLOCO) if bloco else (BYTES_ITER, BYTES_SETUP)
        b = NX * NY * (iters * bi[rotulo] + bs[rotulo])
        gbs = b / t_solve / 1e9 if t_solve > 0 else 0.0
        return dict(iters=iters, ms_solve=t_solve * 1000, gbs=gbs, bytes=b)

    def particulas_gbs(res, n, pico):
        """Particle bytes per second of the P2G and G2P stages (BYTES_PARTICULA x particles over
        the stage's device time per substep); the P2G stage also zeroes the sums and computes
        the face velocities."""
        et = res["etapas"]
        n_sub = max(et["subpassos"], 1)
        out = {"bytes_per_particle": BYTES_PARTICULA, "particles": n}
        for k, b in BYTES_PARTICULA.items():
            t = et[k] / n_sub / 1000
            gbs = n * b / t / 1e9 if t > 0 else 0.0
            out[k + "_gbs"] = round(gbs, 1)
            out[k + "_frac_of_hbm"] = round(gbs / pico, 4)
        return out

    r_m = roofline(misto_etapas, "fp16", bloco=True)
    r_p = roofline(plano, "fp32")
    if rank != 0:
        return None
    linha = {
        "metric": METRIC,
        "value": round(valor, 2),
        "unit": "steps/s",
        "n_gpus": mundo,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(tempos[0] / args.steps, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {
            "workload": "ultra scene 840x536 h=1.6mm, labyrinth 8-cell corridors/4-cell walls, faucet 12 cells at 1.2 m/s "
                        "added every frame, sigma=0.0728; one step = 1 relabel + 14 substeps of 1/840 s",
            "particles": misto["particulas"], "tolerance": TOL, "tolerance_on": "true FP64 residual ||b - A q||",
            "iteration_cap": MAX_ITER, "mixed_precision": "fp16 V-cycle storage",
            "mixed_engine": "fused, block preconditioner with one smoother pass a leg above level 0 "
                            "(TQ_PRECOND_BLOCK_1), frames replayed from a CUDA graph",
            "l2": "flushed (256 MB write) between timed steps", "parallelism": f"replicas x{mundo}",
        },
        "mixed": {"solve": misto["solve"], "mgpcg_gbs": round(r_m["gbs"], 1), "pcg_iters": round(r_m["iters"], 2),
                  "ms_solve": round(r_m["ms_solve"], 4), "speedup_vs_fp32_plain": round(valor / valor_plano, 3),
                  "speedup_vs_fp32_fused": round(valor / valor_f32, 3)},
        "fp32_fused": {"value": round(valor_f32, 2), "unit": "steps/s", "solve": fundido32["solve"],
                       "engine": "fused, TQ_PRECOND_BLOCK_1, CUDA graph"},
        "fp32_plain": {"value": round(valor_plano, 2), "unit": "steps/s", "solve": plano["solve"],
                       "mgpcg_gbs": round(r_p["gbs"], 1), "pcg_iters": round(r_p["iters"], 2),
                       "ms_solve": round(r_p["ms_solve"], 4),
                       "engine": "plain (one launch per reference dispatch), reference preconditioner"},
        "stages_ms_per_substep": {k: round(misto_etapas["etapas"][k] / max(misto_etapas["etapas"]["subpassos"], 1), 4)
                                  for k in SimulacaoGPU.ETAPAS},
        "particle_stages": particulas_gbs(misto_etapas, misto["particulas"], hbm),
        "roofline": {"kernel": "MGPCG pressure solve (k_mgpcg)", "bound": "hbm", "achieved": round(r_m["gbs"], 1),
                     "peak": hbm, "peak_source": origem_pico, "unit": "GB/s",
                     "frac": round(r_m["gbs"] / hbm, 4), "traffic": TRAFEGO_SOLVE_BYTES,
                     "bytes_per_launch": round(r_m["bytes"])},
        "e2e": {"value": round(valor_e2e, 2), "unit": "steps/s", "h2d_bytes_per_step": int(e2e["h2d"]),
                "d2h_bytes_per_step": int(e2e["d2h"]), "solve": e2e["solve"]},
        "gpu_launches": int(misto["lancamentos"]),
        "clocks": misto["relogios"],
    }
    return linha


# ------------------------------------------------------------------ the 256-tank batch
LOTE_H = 0.003
METRIC_LOTE = "tank-substeps/s @256-tank batch (8.8M cells): mixed vs FP32 plain at 1e-6 residual"


def executar_lote(args, rank, mundo, dist):
    """--workload lote: the 256-tank batch (tanque.lote), its tanks split over the GPUs by cells
    and laid out in atlases; a step is one 1/60 s frame of every tank."""
    import ctypes as C

    import torch
    from tanque import Cena, SimulacaoGPU, _abi, passo_maximo
    from tanque.lote import BYTES_POR_CELULA_ITER, BYTES_POR_CELULA_ITER_BLOCO, Lote, gerar_tanques, repartir

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    todos = gerar_tanques(h=LOTE_H)
    meus = [todos[k] for k in repartir(todos, mundo)[rank]]
    dt = passo_maximo(LOTE_H, max(t["ny"] for t in todos) * LOTE_H)
    sub = math.ceil(DT_QUADRO / dt - 1e-9)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    hbm, origem_pico = picos()

    def barreira():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def opcoes(precisao, motor):
        precond = _abi.TQ_PRECOND_BLOCK if motor == _abi.TQ_ENGINE_FUSED else _abi.TQ_PRECOND_REFERENCE
        return {"tolerance": TOL, "iterations": MAX_ITER, "precision": precisao, "engine": motor,
                "preconditioner": precond, "device": dev}

    # the atlas grouping, chosen by measuring candidates (tanque.lote.autoajustar) on the mixed
    # configuration, before any timed or warm-up frame
    from tanque.lote import autoajustar, pesar_por_iteracoes
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    limite, ajuste = autoajustar(lambda c, o: SimulacaoGPU(c, o), Cena, meus, LOTE_H,
                                 opcoes(_abi.TQ_PREC_FP16, _abi.TQ_ENGINE_FUSED), DT_QUADRO, sub, sms=sms)
    # then the SMs' split between the side-by-side atlases: by cells, or by cells x iterations
    pesos, ajuste_ctas = pesar_por_iteracoes(lambda c, o: SimulacaoGPU(c, o), Cena, meus, LOTE_H,
                                             opcoes(_abi.TQ_PREC_FP16, _abi.TQ_ENGINE_FUSED), DT_QUADRO, sub,
                                             limite, sms)

    def medir(precisao, motor, com_relogio=False, e2e=False, grafo=None):
        """Frames of the batch (`grafo`: each atlas's frame from its CUDA graph, the default
        for the fused engine, with the SMs split between the atlases so their frames run side
        by side); stage timing is recorded by eager frames only, each atlas on the whole GPU."""
        grafo = motor == _abi.TQ_ENGINE_FUSED if grafo is None else grafo
        lote = Lote(lambda c, o: SimulacaoGPU(c, o), Cena, meus, LOTE_H, opcoes(precisao, motor), limite_grosso=limite,
                    sms=sms if grafo else None, pesos=pesos if grafo else None)
        fluxos = [torch.cuda.ExternalStream(s.stream()) for s in lote.sims]
        lig = _abi.carregar()
        saidas = []
        if e2e:
            for s in lote.sims:
                cap = s.n + 16
                saidas.append((torch.empty(cap * 12, dtype=torch.float32, pin_memory=True).numpy(), cap))
        for q in range(args.warmup):
            lote.avancar(DT_QUADRO, sub, grafo=grafo)
        lote.sincronizar()
        barreira()
        for s in lote.sims:
            s.tempos(True)
            s.definirEscalar(_abi.TQ_SCALAR_SOLVES, 0)
        l0 = SimulacaoGPU.lancamentos()
        rel = Relogios(dev) if com_relogio else None
        if rel:
            rel.__enter__()
        eventos, d2h = [], 0
        for q in range(args.steps):
            p0 = fluxos[0]
            with torch.cuda.stream(p0):
                flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e0.record(p0)
            for f in fluxos[1:]:
                f.wait_event(e0)
            lote.avancar(DT_QUADRO, sub, grafo=grafo)
            if e2e:
                for s, (buf, cap) in zip(lote.sims, saidas):
                    n = C.c_int32(0)
                    lig("get_particles", s._h, buf.ctypes.data, cap, C.byref(n))
                    d2h += n.value * 48
            for f in fluxos[1:]:
                e = torch.cuda.Event()
                e.record(f)
                p0.wait_event(e)
            e1 = torch.cuda.Event(enable_timing=True)
            e1.record(p0)
            eventos.append((e0, e1))
        lote.sincronizar()
        torch.cuda.synchronize()
        if rel:
            rel.__exit__()
        lanc = SimulacaoGPU.lancamentos() - l0
        ms = sum(a.elapsed_time(b) for a, b in eventos)
        etapas = [s.tempos() for s in lote.sims]
        # each tank's own true residual at the last solve (registered tanks: fused engine), and
        # the atlases' solve records
        piores = []
        for s in lote.sims:
            r = s.residuosTanques()
            if len(r):
                agua = r[:, 0] > 0
                piores.append(float(np.max(r[agua, 1] / r[agua, 0])) if agua.any() else 0.0)
        solves = [estatisticas_solve(s) for s in lote.sims]
        celulas = [at["cena"].nx * at["cena"].ny for at in lote.atlas]
        ms_atlas = [round(x, 2) for x in lote.ms_atlas()] if grafo else None
        res = dict(ms=ms, lancamentos=lanc, particulas=lote.n, etapas=etapas, celulas=celulas, ctas=lote.ctas,
                   ms_atlas=ms_atlas,
                   max_rel_tanque=max(piores) if piores else None, solves=solves,
                   atlas=[[at["cena"].nx, at["cena"].ny] for at in lote.atlas], relogios=rel.resumo() if rel else None,
                   d2h=d2h / max(args.steps, 1))
        lote.fechar()
        return res

    def solve(res, rotulo, bloco=False):
        """Pressure-solve figures of one rank: algorithmic MGPCG bytes over the solves' time."""
        t = sum(e["pressao"] for e in res["etapas"]) / 1000
        mb = BYTES_POR_CELULA_ITER_BLOCO if bloco else BYTES_POR_CELULA_ITER
        b = sum(c * (e["iteracoes"] * mb[rotulo][0] + e["subpassos"] * mb[rotulo][1])
                for c, e in zip(res["celulas"], res["etapas"]))
        iters = sum(e["iteracoes"] for e in res["etapas"]) / max(sum(e["subpassos"] for e in res["etapas"]), 1)
        return dict(gbs=b / t / 1e9 if t > 0 else 0.0, iters=iters, bytes=b, s=t)

    misto = medir(_abi.TQ_PREC_FP16, _abi.TQ_ENGINE_FUSED, com_relogio=True)
    # the same configuration eagerly, for the solve's stage time (a graph records no events)
    misto_etapas = medir(_abi.TQ_PREC_FP16, _abi.TQ_ENGINE_FUSED, grafo=False)
    plano = medir(_abi.TQ_PREC_FP32, _abi.TQ_ENGINE_PLAIN)
    e2e = medir(_abi.TQ_PREC_FP16, _abi.TQ_ENGINE_FUSED, e2e=True)
    tempos = tempos_max_ranks([misto["ms"], plano["ms"], e2e["ms"]], dist, "cuda")
    valor, valor_plano, valor_e2e = (len(todos) * args.steps * sub / (t / 1000) for t in tempos)
    r_m, r_p = solve(misto_etapas, "fp16"), solve(plano, "fp32")
    if rank != 0:
        return None
    return {
        "metric": METRIC_LOTE,
        "value": round(valor, 1),
        "unit": "tank-substeps/s",
        "n_gpus": mundo,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(tempos[0] / args.steps, 3),
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {
            "workload": f"256 tanks (seed 4): widths logU[64,512], heights logU[64,320] cells, h=3mm, random walls, "
                        f"water 20-70 %, 4 ppc; one step = 1 relabel + {sub} substeps of {DT_QUADRO / sub * 1000:.3f} ms "
                        "for every tank",
            "tank_cells": sum(t["nx"] * t["ny"] for t in todos), "atlases_rank0": misto["atlas"],
            "atlas_padding_frac_rank0": round(1 - sum(t["nx"] * t["ny"] for t in meus) / sum(misto["celulas"]), 4),
            "autotuner": {"coarsest_level_limit": limite,
                          "seconds_per_frame_by_limit": {str(k): round(v, 4) for k, v in ajuste.items()}},
            "atlas_cells_rank0": sum(misto["celulas"]), "particles_rank0": misto["particulas"], "tolerance": TOL,
            "mixed_precision": "fp16 V-cycle storage",
            "mixed_engine": "fused, block preconditioner (TQ_PRECOND_BLOCK), each atlas's frame replayed from a CUDA "
                            "graph, the atlases "
                            "side by side on shares of the SMs (fused_ctas)",
            "fused_ctas_rank0": misto["ctas"],
            "sm_split": {"weights": "cells x mean iterations" if pesos is not None else "cells",
                         "min_ctas": 4, "seconds_per_frame": {k: round(v, 4) for k, v in ajuste_ctas.items()}},
            "l2": "flushed (256 MB write) between timed steps", "parallelism": f"tanks split over {mundo} GPU(s) by cells",
        },
        "fp32_plain": {"value": round(valor_plano, 1), "unit": "tank-substeps/s", "mgpcg_gbs": round(r_p["gbs"], 1),
                       "ms_solve_per_substep_all_atlases": round(r_p["s"] * 1000 / max(args.steps * sub, 1), 3),
                       "pcg_iters_per_atlas_substep": round(r_p["iters"], 2),
                       "stop": "the atlas's true residual as a whole (the plain engine has no per-tank test)",
                       "solves_per_atlas": plano["solves"]},
        "mixed": {"mgpcg_gbs": round(r_m["gbs"], 1), "pcg_iters_per_atlas_substep": round(r_m["iters"], 2),
                  "ms_solve_per_substep_all_atlases": round(r_m["s"] * 1000 / max(args.steps * sub, 1), 3),
                  "eager_value": round(len(todos) * args.steps * sub / (misto_etapas["ms"] / 1000), 1),
                  "speedup_vs_fp32_plain": round(valor / valor_plano, 3),
                  "stop": "every tank's own true residual <= 1e-6 of its own r0 (tq_set_tanks)",
                  "max_tank_true_rel_residual_last_solve": misto["max_rel_tanque"],
                  "last_frame_ms_per_atlas": misto["ms_atlas"],
                  "solves_per_atlas": misto["solves"]},
        "roofline": {"kernel": "MGPCG pressure solve", "bound": "hbm", "achieved": round(r_m["gbs"], 1),
                     "peak": hbm, "peak_source": origem_pico, "unit": "GB/s", "frac": round(r_m["gbs"] / hbm, 4),
                     "traffic": None},
        "e2e": {"value": round(valor_e2e, 1), "unit": "tank-substeps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(e2e["d2h"])},
        "gpu_launches": int(misto["lancamentos"]),
        "clocks": misto["relogios"],
    }


# ------------------------------------------------------------------ the adjoint (256 x 160, 60 steps)
METRIC_ADJ = "adjoint gradient evaluations/s @256x160, 60 steps (forward + backward, 32 candidate controls)"


def executar_adjunto(args, rank, mundo, dist):
    """--workload adjunto: the adjoint scene (tanque.cenarios.cena_adjunto: 256 x 160, h = 4 mm,
    60 steps of 1/240 s, a dam-break block and a faucet, loss = L2 distance of the final water
    fraction to a seeded target blob); a step is one gradient evaluation (forward with checkpoints
    every 10 steps, backward with recomputation) of each of 32 candidate controls (initial
    velocities and faucet velocity perturbed from a seed), the 32 handles driven by host threads
    so their solves overlap on the GPU.  value = gradient evaluations per second."""
    import concurrent.futures as cf

    import torch
    from tanque.adjunto import AdjuntoGPU
    from tanque.cenarios import cena_adjunto

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    cena = cena_adjunto()
    K = 32
    rng = np.random.default_rng(7 + rank)
    controles = [(cena["v0"] + rng.normal(0, 0.05, cena["v0"].shape).astype(np.float32),
                  cena["theta0"] + rng.normal(0, 0.1, 2)) for _ in range(K)]
    alcas = [AdjuntoGPU(cena, dev) for _ in range(K)]

    def um(k):
        a = alcas[k]
        v, th = controles[k]
        t0 = time.perf_counter()
        L = a.frente(v, th)
        t1 = time.perf_counter()
        gv, gt = a.tras(1.0)
        t2 = time.perf_counter()
        return L, gt, t1 - t0, t2 - t1

    pool = cf.ThreadPoolExecutor(max_workers=K)
    for _ in range(args.warmup):
        list(pool.map(um, range(K)))
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ini = torch.cuda.Event(enable_timing=True)
    fim = torch.cuda.Event(enable_timing=True)
    l0 = None
    from tanque import SimulacaoGPU
    l0 = SimulacaoGPU.lancamentos()
    ini.record()
    t0 = time.perf_counter()
    res = []
    for _ in range(args.steps):
        res = list(pool.map(um, range(K)))
    t = time.perf_counter() - t0
    fim.record()
    torch.cuda.synchronize()
    lanc = SimulacaoGPU.lancamentos() - l0
    ms = tempos_max_ranks([t * 1000.0], dist, "cuda")[0]
    pool.shutdown()
    for a in alcas:
        a.fechar()
    if rank != 0:
        return None
    valor = mundo * K * args.steps / (ms / 1000.0)
    return {
        "metric": METRIC_ADJ, "value": round(valor, 3), "unit": "gradients/s", "n_gpus": mundo, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 2), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "adjoint: 256x160 h=4mm, 60 steps of 1/240 s, dam-break block + faucet, "
                               "L2 water-fraction loss to a seeded blob; 32 candidate controls per step",
                   "particles": int(cena["positions"].shape[0]), "checkpoint_every": 10,
                   "controls": K, "timing": "host wall clock over the threads (each call waits for its stream)"},
        "per_control_ms": {"forward": round(1000 * float(np.mean([r[2] for r in res])), 2),
                           "backward": round(1000 * float(np.mean([r[3] for r in res])), 2)},
        "gpu_launches": int(lanc),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU-oracle timing")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain", dest="fused", action="store_false", help="mixed config on the plain engine")
    ap.add_argument("--workload", default="ultra", choices=["ultra", "lote", "adjunto"],
                    help="ultra: the 450k-cell scene (default); lote: the 256-tank batch; adjunto: the adjoint")
    args = ap.parse_args()

    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: relaunch this command under torch.distributed.run
        import socket
        with socket.socket() as so:
            so.bind(("127.0.0.1", 0))
            porta = so.getsockname()[1]
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
               "--master-addr=127.0.0.1", f"--master-port={porta}", os.path.abspath(__file__)] + sys.argv[1:]
        sys.exit(subprocess.call(cmd))
    mundo = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "ours" and mundo != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE {mundo}")

    if args.impl == "reference" and args.workload == "lote":
        if rank != 0:
            return
        v, feitos = medir_oraculo_lote(args.cpu_budget)
        linha = {
            "metric": METRIC_LOTE, "impl": "reference", "value": round(v, 3), "unit": "tank-substeps/s",
            "n_gpus": args.gpus, "steps": feitos, "warmup": 1, "ms_per_step": round(1000 / v, 2),
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "256-tank batch (as ours); one step = one substep of one tank", "tolerance": TOL},
            "cpu_baseline": {"value": round(v, 3), "unit": "tank-substeps/s", "cores": 1, "kind": "port",
                             "sample": f"one substep of each of the first {feitos} tanks after one warm-up substep, "
                                       "CPU oracle (reference CPU engine restated in C++, single thread)"},
            "e2e": {"value": round(v, 3), "unit": "tank-substeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(linha))
        return
    if args.impl == "reference" and args.workload == "adjunto":
        if rank != 0:
            return
        # the reference has no adjoint: the CPU arm is the oracle's FP64 adjoint (the checker),
        # one gradient evaluation of the scene's control per step
        sys.path.insert(0, os.path.join(RAIZ, "tests"))
        from oraculo import AdjuntoOraculo
        from tanque.cenarios import cena_adjunto
        cena = cena_adjunto()
        a = AdjuntoOraculo(cena)
        v0 = cena["v0"].astype(np.float64)
        t0 = time.perf_counter()
        feitos = 0
        while feitos < max(1, args.steps):
            a.forward(v0, cena["theta0"], True)
            a.backward()
            feitos += 1
            if time.perf_counter() - t0 > args.cpu_budget:
                break
        v = feitos / (time.perf_counter() - t0)
        print(json.dumps({
            "metric": METRIC_ADJ, "impl": "reference", "value": round(v, 4), "unit": "gradients/s",
            "n_gpus": args.gpus, "steps": feitos, "warmup": 0, "ms_per_step": round(1000 / v, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "adjoint scene as ours; one step = one gradient evaluation of one control"},
            "cpu_baseline": {"value": round(v, 4), "unit": "gradients/s", "cores": 1, "kind": "port",
                             "sample": f"{feitos} forward + backward runs of the FP64 CPU adjoint (the oracle's "
                                       "checker; the reference has no adjoint), single thread"},
            "e2e": {"value": round(v, 4), "unit": "gradients/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return
    if args.impl == "reference":
        if rank != 0:
            return
        # each step: one substep of the scene on the CPU oracle
        v, feitos, n_part = medir_oraculo(args.steps, args.warmup)
        linha = {
            "metric": METRIC, "impl": "reference", "value": round(v, 4), "unit": "steps/s", "n_gpus": args.gpus,
            "steps": feitos, "warmup": args.warmup, "ms_per_step": round(1000 / v, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "ultra scene 840x536 h=1.6mm (as ours); one step = one substep of 1/840 s",
                       "particles": n_part, "tolerance": TOL},
            "cpu_baseline": {"value": round(v, 4), "unit": "steps/s", "cores": 1, "kind": "port",
                             "sample": f"{feitos} substeps after {args.warmup} warm-up substeps, CPU oracle "
                                       "(reference CPU engine restated in C++, single thread)"},
            "e2e": {"value": round(v, 4), "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(linha))
        return

    dist = None
    if mundo > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    corre = {"lote": executar_lote, "adjunto": executar_adjunto}.get(args.workload, executar_gpu)
    linha = corre(args, rank, mundo, dist)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0 and linha is not None:
        if mundo == 1 and not args.no_cpu_baseline and args.workload == "lote":
            v, feitos = medir_oraculo_lote(args.cpu_budget)
            linha["cpu_baseline"] = {"value": round(v, 3), "unit": "tank-substeps/s", "cores": 1, "kind": "port",
                                     "sample": f"one substep of each of the first {feitos} tanks of the batch after "
                                               "one warm-up substep (CPU oracle, single thread)"}
        if mundo == 1 and not args.no_cpu_baseline and args.workload == "ultra":
            v, feitos, n_part = medir_oraculo(10 ** 6, 1, orcamento_s=args.cpu_budget)
            linha["cpu_baseline"] = {"value": round(v, 4), "unit": "steps/s", "cores": 1, "kind": "port",
                                     "sample": f"{feitos} substeps of the same scene after 1 warm-up substep "
                                               "(CPU oracle, single thread)"}
        print(json.dumps(linha))


if __name__ == "__main__":
    main()
