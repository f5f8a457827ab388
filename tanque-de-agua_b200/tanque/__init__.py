"""tanque — B200 simulation step of the 2-D FLIP/APIC water tank behind a C-ABI.

The package is the host-side mirror of the reference's CPU engine interface:
  SimulacaoGPU        the `SimulacaoCPU` surface (js/fisica-cpu.js) over libtanque.so
  Cena                the wall SDF builder (js/cena.js)
  resolver_pressao    `resolverPCG` (js/pressao-cpu.js) on the device
  ciclo_v             `cicloV` (js/pressao-cpu.js) on the device
"""
from .cena import Cena
from .constantes import dimensoes_da_grade, passo_maximo
from .simulacao import Simulacao, SimulacaoGPU, ciclo_v, resolver_pressao

__all__ = ["Cena", "Simulacao", "SimulacaoGPU", "ciclo_v", "resolver_pressao", "dimensoes_da_grade", "passo_maximo"]
