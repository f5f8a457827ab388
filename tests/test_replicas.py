"""The N-GPU path of bench.py is "replicas only": every rank advances its own tank, the job's time
is the maximum over the ranks and the throughput counts every rank's substeps.  Checked here with
two gloo ranks on the CPU (the reduction and the accounting; the tanks themselves need a GPU)."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

RAIZ = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _porta_livre():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, mundo, porta, fila):
    sys.path.insert(0, RAIZ)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(porta))
    dist.init_process_group("gloo", rank=rank, world_size=mundo)
    try:
        # each replica measured its own three arms; rank 1 is the slower one in two of them
        meus = [100.0 + 50.0 * rank, 200.0 - 20.0 * rank, 300.0 + 10.0 * rank]
        t = bench.tempos_max_ranks(meus, dist, "cpu")
        v = bench.vazao_replicas(mundo, 6, 14, t[0])
        fila.put((rank, list(t), v))
    finally:
        dist.destroy_process_group()


def test_tempo_maximo_e_vazao_de_duas_replicas():
    ctx = mp.get_context("spawn")
    fila = ctx.Queue()
    porta = _porta_livre()
    ps = [ctx.Process(target=_rank, args=(r, 2, porta, fila)) for r in range(2)]
    for p in ps:
        p.start()
    res = [fila.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, v in res:
        assert t == [150.0, 200.0, 310.0]           # every rank holds the maximum
        assert v == pytest.approx(2 * 6 * 14 / 0.150)  # both replicas' substeps over the slowest time


def test_uma_replica_sem_process_group():
    sys.path.insert(0, RAIZ)
    import bench
    assert list(bench.tempos_max_ranks([1.0, 2.0], None, "cpu")) == [1.0, 2.0]
    assert bench.vazao_replicas(1, 6, 14, 1000.0) == pytest.approx(84.0)


def test_bench_lanca_um_rank_por_gpu():
    """`bench.py --gpus 2` outside torchrun relaunches itself under torch.distributed.run with 2
    ranks (127.0.0.1); here the CPU reference arm of the adjoint workload, which rank 0 alone runs
    and prints (the other rank exits 0 without work)."""
    import json
    import subprocess
    env = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    r = subprocess.run([sys.executable, os.path.join(RAIZ, "bench.py"), "--gpus", "2", "--impl", "reference",
                        "--workload", "adjunto", "--steps", "1", "--cpu-budget", "0.1"],
                       capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    linhas = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(linhas) == 1  # one line, from rank 0
    d = json.loads(linhas[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2
