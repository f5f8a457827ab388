"""Runs a benchmark scene on the GPU for a few frames and prints, as JSON, the per-stage device
times of the last frame or, with --phases, the fused solver's per-phase times of one substep.

    python -m tanque.rodar [--scene ultra|atlas] [--frames F] [--substeps S] [--precision 0|1|2]
                           [--engine 0|1] [--precond 0|1|2] [--tolerance T] [--iterations K]
                           [--phases]

`ultra` is the 450k-cell scene of the throughput benchmark; `atlas` is the largest atlas of
the 256-tank batch (tanque.lote).  Frames are 1/60 s split into S substeps (default: 14 for
ultra, the capillary limit for the atlas); every pressure solve runs to the tolerance, or
exactly K iterations with --tolerance 0.

It is the small, self-contained driver for single-kernel profiler captures (a handful of
launches of the pressure solve on the real workload) and for the phase trace: with --phases
the fused kernel stamps the global timer at every grid barrier of one more substep
(tq_get_phase_trace), and the medians over that solve's PCG iterations are printed per phase.
The trace needs --tolerance 0: in tolerance mode the iterations that check the true residual
add phases, so the iterations of a solve do not all have the same phases.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math

import numpy as np

from . import Cena, SimulacaoGPU, _abi, passo_maximo
from .cenarios import cena_ultra
from .lote import agrupar, gerar_tanques, montar_atlas, niveis

SMEM_SECAO = 200 * 1024  # the fused engine's shared-memory budget for its coarse section
SECAO_MAX_CELULAS = 2048


def secao(lv) -> int:
    """First level of the fused engine's coarse section (the rule of criarFundido)."""
    L, Lc, total = len(lv), len(lv), 0
    for l in range(L - 1, 0, -1):
        n = lv[l][0] * lv[l][1]
        b = 3 * ((n * 4 + 15) & ~15) + ((n + 15) & ~15)
        if total + b > SMEM_SECAO or (n > SECAO_MAX_CELULAS and l < L - 1):
            break
        total += b
        Lc = l
    return Lc


def rotulos(Lc: int, bloco: bool = False) -> list[str]:
    """The fused solver's phases of one PCG iteration; with the block preconditioner the levels
    above 0 take one smoother pass a leg."""
    out = ["DA", "B"]
    for l in range(Lc):
        if bloco and l >= 1:
            out += [f"s8 L{l}", f"restr {l}>{l + 1}"]
        else:
            out += [("s0+spread L0" if l == 0 else f"s0 L{l}"), f"s8 L{l}", f"restr {l}>{l + 1}"]
    out += ["coarse section"]
    for l in range(Lc - 1, -1, -1):
        out += [f"prol+s8 L{l}"] if bloco and l >= 1 else [f"prol+s8 L{l}", ("s0+gather L0" if l == 0 else f"s0 L{l} up")]
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--scene", default="ultra", choices=["ultra", "atlas"])
    ap.add_argument("--frames", type=int, default=2)
    ap.add_argument("--substeps", type=int, default=0, help="0: 14 (ultra) or the capillary limit (atlas)")
    ap.add_argument("--precision", type=int, default=1, help="0 FP32, 1 FP16, 2 BF16 V-cycle storage")
    ap.add_argument("--engine", type=int, default=1, help="0 plain, 1 fused")
    ap.add_argument("--precond", type=int, default=1,
                    help="0 reference, 1 block preconditioner, 2 block with one smoother pass a leg above level 0")
    ap.add_argument("--tolerance", type=float, default=1e-6)
    ap.add_argument("--iterations", type=int, default=1000, help="iteration cap (the count with --tolerance 0)")
    ap.add_argument("--phases", action="store_true", help="per-phase times of one more substep (fused engine)")
    args = ap.parse_args(argv)
    if args.phases and args.tolerance > 0:
        ap.error("--phases needs --tolerance 0 (a fixed iteration count, the same phases every iteration)")
    if args.scene == "ultra":
        cena, _, agua, _ = cena_ultra(Cena)
        sub = args.substeps or 14
    else:
        h = 0.003
        t = gerar_tanques(h=h)
        at = montar_atlas(Cena, [t[k] for k in agrupar(t)[0]], h)
        cena, agua = at["cena"], at["particulas"]
        sub = args.substeps or math.ceil((1 / 60) / passo_maximo(h, cena.ny * h) - 1e-9)
    sim = SimulacaoGPU(cena, {"tolerance": args.tolerance, "iterations": args.iterations, "precision": args.precision,
                              "engine": args.engine, "preconditioner": args.precond})
    sim.adicionar(agua, False)
    for q in range(args.frames):
        if q == args.frames - 1:
            sim.tempos(True)
        sim.avancar(1 / 60, sub)
    out = {"scene": args.scene, "grid": [cena.nx, cena.ny], "particles": sim.n, "frames": args.frames,
           "substeps": sub, "last_frame_ms": sim.tempos(),
           "solves": {"n": sim.escalar(_abi.TQ_SCALAR_SOLVES), "capped": sim.escalar(_abi.TQ_SCALAR_SOLVES_CAPPED),
                      "iters": sim.escalar(_abi.TQ_SCALAR_SOLVE_ITERS),
                      "max_true_rel": sim.escalar(_abi.TQ_SCALAR_SOLVE_MAX_REL),
                      "replacements": sim.escalar(_abi.TQ_SCALAR_SOLVE_REPLACEMENTS)}}
    if args.phases:
        lig = _abi.carregar()
        lig.lib.tq_get_phase_trace.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.c_int32, C.POINTER(C.c_int32)]
        sim.tempos(True)
        lig("set_timing", sim._h, 2)
        sim.subpasso(1 / 60 / sub)
        it = sim.tempos()["iteracoes"]
        buf = (C.c_uint64 * 65536)()
        n = C.c_int32()
        lig.lib.tq_get_phase_trace(sim._h, buf, 65536, C.byref(n))
        d = np.diff(np.array(buf[:n.value], dtype=np.int64)) / 1000.0
        Lc = secao(niveis(cena.nx, cena.ny))
        nomes = rotulos(Lc, args.precond == _abi.TQ_PRECOND_BLOCK_1)
        per = len(nomes)
        # the last iteration runs DA and B only, then the closing barrier
        fim = len(d) - 3
        ini = fim - (it - 1) * per
        if it > 1 and ini >= 0:
            med = np.median(d[ini:fim].reshape(it - 1, per), axis=0)
            out["phases_us"] = {r: round(float(v), 2) for r, v in zip(nomes, med)}
            out["iteration_us"] = round(float(med.sum()), 1)
            out["pcg_iterations"] = it
            out["setup_us"] = round(float(d[:ini].sum()), 1)
    print(json.dumps(out))
    sim.fechar()


if __name__ == "__main__":
    main()
