"""Runs the benchmark's 450k-cell ultra scene on the GPU for a few frames and prints the
per-stage device times of the last frame, as one JSON line.

    python -m tanque.rodar [--frames F] [--substeps S] [--precision 0|1|2] [--engine 0|1]
                           [--tolerance T]

It is the small, self-contained driver for single-kernel profiler captures (a handful of
launches of the pressure solve on the real workload) and a quick check of where a frame's time
goes.  Frames are 1/60 s split into S substeps; every pressure solve runs to the tolerance.
"""
from __future__ import annotations

import argparse
import json

from . import Cena, SimulacaoGPU
from .cenarios import cena_ultra


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--frames", type=int, default=2)
    ap.add_argument("--substeps", type=int, default=14)
    ap.add_argument("--precision", type=int, default=1, help="0 FP32, 1 FP16, 2 BF16 V-cycle storage")
    ap.add_argument("--engine", type=int, default=1, help="0 plain, 1 fused")
    ap.add_argument("--tolerance", type=float, default=1e-6)
    args = ap.parse_args(argv)
    cena, _, agua, _ = cena_ultra(Cena)
    sim = SimulacaoGPU(cena, {"tolerance": args.tolerance, "iterations": 200, "precision": args.precision,
                              "engine": args.engine})
    sim.adicionar(agua, False)
    for q in range(args.frames):
        if q == args.frames - 1:
            sim.tempos(True)
        sim.avancar(1 / 60, args.substeps)
    t = sim.tempos()
    print(json.dumps({"particles": sim.n, "frames": args.frames, "last_frame_ms": t}))
    sim.fechar()


if __name__ == "__main__":
    main()
