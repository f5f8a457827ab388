// pcg_interno.cuh — the pressure-solver object shared by the plain engine (pcg.cu) and the
// fused engine (pcg_fundido.cu).
#pragma once
#include <vector>

#include "common.cuh"

namespace tq {

// Levels with at least this many cells store the V-cycle vectors in 16-bit when a
// half-precision mode is selected (the small coarse levels stay FP32).
constexpr int MEIA_MIN_CELULAS = 16384;

struct Fundido;

struct Pcg {
  int nx, ny, N, precisao, motor;
  int ctasFundido = 0;  // the fused engine's CTA count (0: one per SM)
  int L;
  int nxL[MAX_NIVEIS], nyL[MAX_NIVEIS];
  bool meia[MAX_NIVEIS];  // level stored in half precision
  uint8_t* tipoL[MAX_NIVEIS];
  uint8_t* vizL[MAX_NIVEIS];
  void *bL[MAX_NIVEIS], *xL[MAX_NIVEIS], *tmpL[MAX_NIVEIS];  // 4 bytes per element allocated
  uint8_t* vizOp;
  double* q64 = nullptr;  // the plain engine's FP64 iterate (tolerance mode), allocated on first use
  const int* parar = nullptr;  // the running plain solve's stop flag (NivelDev::parar)
  size_t smemGrosso = 0;
  Fundido* fundido = nullptr;
  Regioes* regioes = nullptr;  // tolerance mode's closed-region projection, allocated on first use
};

// pcg_fundido.cu
Fundido* criarFundido(Pcg* p);
void destruirFundido(Fundido* f);
int resolverPressaoFundido(Pcg* p, const Dev& d, int iteracoes, double tol, bool bolhas, int precond,
                           cudaStream_t s);
int erroFundido(Fundido* f, cudaStream_t s);
void perfilFundido(Fundido* f, bool ligar);
int lerPerfilFundido(Fundido* f, unsigned long long* out, int cap);

}  // namespace tq
