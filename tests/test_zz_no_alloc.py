"""tq_vcycle_noalloc: the V-cycle with its level hierarchy in a static device array.

The GPU test calls it through the C-ABI on device buffers and compares it with tq_vcycle (the
entry point that allocates) on the same inputs, two calls in a row with different right-hand
sides, so state left in the scratch by the first call would show in the second.  The CPU test
checks that a grid beyond the scratch's capacity is refused before any device work.
This file sorts last so that the GPU test also runs after every other test in one process.
"""
import ctypes as C

import numpy as np
import pytest

from estado import erro_relativo
from tanque import _abi, ciclo_v
from tanque.constantes import AGUA, AR

BYTES_SCRATCH = 16 << 20


def _ligar():
    lib = C.CDLL(_abi.CAMINHO_LIB)
    f = lib.tq_vcycle_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
    lib.tq_last_error.restype = C.c_char_p
    lib.tq_last_error.argtypes = []
    return lib, f


def _tipos(nx, ny, semente):
    """Water with scattered walls, an air layer on top and a closed air pocket in the water."""
    rng = np.random.default_rng(semente)
    tipo = np.full((ny, nx), AGUA, np.uint8)
    tipo[rng.random((ny, nx)) < 0.08] = 0
    tipo[: ny // 6, :] = AR
    tipo[ny // 2: ny // 2 + 4, nx // 3: nx // 3 + 6] = AR
    tipo[:, 0] = tipo[:, -1] = tipo[0, :] = tipo[-1, :] = 0
    return tipo


def test_grade_grande_demais_recusada():
    """A grid whose levels exceed the 16 MiB scratch: TQ_E_CAPACITY, the bytes named, no device call."""
    lib, f = _ligar()
    st = f(4000, 3000, 1, 1, 1, _abi.TQ_PREC_FP32, None)  # pointers never dereferenced: refused first
    assert st == _abi.TQ_E_CAPACITY
    msg = lib.tq_last_error().decode()
    assert "bytes" in msg and str(BYTES_SCRATCH) in msg
    # sizes whose level arithmetic would overflow int are refused before it runs
    for nx, ny in [(2**31 - 1, 16), (16, 2**31 - 1), (1 << 21, 4), (1 << 15, 1 << 15)]:
        assert f(nx, ny, 1, 1, 1, _abi.TQ_PREC_FP32, None) == _abi.TQ_E_CAPACITY, (nx, ny)
    assert f(2, 2, 1, 1, 1, _abi.TQ_PREC_FP32, None) == _abi.TQ_E_ARG
    assert f(40, 30, 1, 1, 1, 7, None) == _abi.TQ_E_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny", [(161, 77), (840, 536), (1280, 720)])
@pytest.mark.parametrize("prec", [_abi.TQ_PREC_FP32, _abi.TQ_PREC_FP16, _abi.TQ_PREC_BF16],
                         ids=["fp32", "fp16", "bf16"])
def test_sem_alocar_igual_ao_ciclo_v(lib_gpu, nx, ny, prec):
    import torch

    lib, f = _ligar()
    tipo = _tipos(nx, ny, nx + ny)
    rng = np.random.default_rng(nx * ny)
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    t_d = torch.from_numpy(tipo.reshape(-1)).to(dev)
    x_d = torch.empty(nx * ny, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    for chamada in range(2):  # two calls in a row, different right-hand sides
        b = rng.standard_normal((ny, nx)).astype(np.float32)
        b[tipo != AGUA] = 0
        b_d = torch.from_numpy(b.reshape(-1)).to(dev)
        x_d.fill_(float("nan"))  # every output cell must be written
        torch.cuda.synchronize()
        st = f(nx, ny, t_d.data_ptr(), b_d.data_ptr(), x_d.data_ptr(), prec, C.c_void_p(stream.cuda_stream))
        assert st == _abi.TQ_OK, lib.tq_last_error().decode()
        torch.cuda.synchronize()
        x_sem = x_d.cpu().numpy().reshape(ny, nx)
        x_ref = ciclo_v(tipo, b, precisao=prec)
        assert np.all(np.isfinite(x_sem)), f"call {chamada}: unwritten cells"
        # Same kernels and launch shapes on the same inputs: expected bit-identical; the
        # stated bound is a relative L-infinity error of 1e-6.
        assert erro_relativo(x_sem, x_ref) <= 1e-6, f"call {chamada}"
