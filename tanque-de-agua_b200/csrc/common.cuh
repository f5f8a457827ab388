// common.cuh — constants, device-state layout and small device helpers shared by every
// translation unit of libtanque.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/tanque.h"

namespace tq {

// ------------------------------------------------------------ physics constants
// Values of js/constantes.js:8-104 (the reference reads every number from there).
constexpr double GRAVIDADE = 9.81;
constexpr double DENSIDADE_AGUA = 1000;
constexpr double TENSAO_SUPERFICIAL = 0.0728;
constexpr int MAX_BOLHAS = 4096;
constexpr int MAX_TANQUES = 4096;  // tanks of one atlas (tq_set_tanks)
constexpr double VOLTA_VOLUME_BOLHA = 0.05;
constexpr double PRESSAO_BOLHA_MAX = 20000;
constexpr double PARTICULAS_POR_CELULA = 4;
constexpr int RES_MASCARA = 2;
constexpr double SDF_MAX = 10;
constexpr int MOLDURA = 2;
constexpr double RAIO_MANCHA = 2.1;  // splat radius in cells (js/constantes.js:120)
constexpr double RAIO_PARTICULA = 0.3;
constexpr double MICROPASSO = 0.8;
constexpr double MAX_MICROPASSOS = 4;
constexpr double TAU_DENSIDADE = 0.1;
constexpr double EXCESSO_MIN = -0.5;
constexpr double EXCESSO_MAX = 1.0;
constexpr int ITERACOES_PCG = 3;
constexpr double ESPUMA_V0 = 1.1, ESPUMA_V1 = 2.8, ESPUMA_TAXA = 5, ESPUMA_VIDA = 1.2;
constexpr double DIFUSAO_CORANTE = 3;
constexpr double PARTICULAS_MAX_POR_CELULA = 4.6;
constexpr int CAMPOS = 12;
constexpr int MIN_BOLHA_CELULAS = 4;
constexpr uint8_t SOLIDO = 0, AGUA = 1, AR = 2;

// Multigrid (js/pressao-cpu.js:17-20)
constexpr int BLOCO = 16;
constexpr int VARREDURAS = 4;
constexpr int VARREDURAS_GROSSO = 64;
constexpr int MAX_NIVEIS = 16;

// Fixed-point scales of the deterministic per-bubble sums (64-bit integer atomics make the
// result independent of the order the cells arrive in).
constexpr double ESCALA_BOLHA = 4294967296.0;  // 2^32

// ------------------------------------------------------------ device scalars
// Scalars the kernels of one substep exchange without a host round trip.
struct Escalares {
  double rz, pap, alpha, beta;
  double norma0, norma;
  double escalaMG;            // 1/||r|| applied before a half-precision V-cycle
  unsigned long long vmaxBits;  // largest particle speed of the last G2P (double bits)
  int n;                      // live particle count (authoritative)
  int mortas;                 // particles marked dead since the last compaction
  int iters;                  // iterations done by the running solve
  int pronto;                 // the running solve met its tolerance
  int erro;                   // device-side error flag (bounded waits, capacity)
  int verificar;              // plain engine, tolerance mode: a true-residual check is due
  int reiniciar;              // plain engine: the true residual is to replace r (k_substituir)
  double proxTroca;           // plain engine: the recursive norm that triggers the next replacement
  int aceitas;                // particles accepted by the last add
  int pendentes;              // label-propagation work list length
  int regioes;                // closed regions the last tolerance-mode solve projected (pcg.cu)
  unsigned int tickets[16];   // last-block-done counters of the reductions
  // convergence of the solves (tolerance mode), written on the device at the end of each solve
  double normaVerd;           // true ||b - A q|| of the last solve's iterate (-1: fixed count)
  int convergiu;              // the last solve met its tolerance on the true residual
  int trocas;                 // residual replacements of the last solve
  long long solves, capados, itersAcum, trocasAcum;  // accumulated since the last reset
  double maxRel;              // largest true ||b - A q|| / ||r0|| since the last reset
  double normas[1024];        // residual history of the running solve
};

// ------------------------------------------------------------ multigrid level
template <class T>
struct NivelDev {
  int nx, ny;
  uint8_t* tipo;  // SOLIDO/AGUA/AR as the preconditioner sees them
  uint8_t* viz;   // bits 0-3: free neighbours (left, right, down, up); bit 4: water
  T *b, *x, *tmp;
  // a solve's stop flag (Escalares::pronto): once set, the V-cycle kernels of the iterations the
  // host queued past convergence return at once; null outside a solve
  const int* parar = nullptr;
};

// ------------------------------------------------------------ device state
// Plain pointers into the handle's device memory; passed by value to the kernels.
struct Dev {
  int nx, ny, N, nu, nv, mw, mh;
  double h;
  float hf;
  int cap;
  // walls
  const float* sdf;
  uint8_t* solido;
  // particles (structure of arrays of float4): p0 = (x, y, vx, vy), p1 = (cux, cuy, cvx, cvy),
  // p2 = (espuma, absR, absG, absB); pid = insertion order
  float4 *p0, *p1, *p2;
  unsigned long long* pid;
  float4 *q0, *q1, *q2;  // compaction targets
  unsigned long long* qid;
  // particle-to-grid sums (fixed point)
  int2 *accU, *accV, *accCel;
  int* accCor;
  // faces
  float *u, *v, *uTmp, *vTmp;
  uint8_t *uVal, *vVal, *uValTmp, *vValTmp;
  // cells
  uint8_t* tipo;
  uint32_t* rotulo;
  uint8_t* pend;
  int* lista;
  float *div, *q, *qAr, *fase, *faseTmp, *nX, *nY, *kap;
  uint8_t *cheio, *cheioTmp;
  // bubbles
  float *pressaoBolha, *volumeAlvo, *volumeBolhaF, *rhsBolhaF, *yBolhaF;
  uint8_t* vivo;
  uint32_t *volB, *facesB, *celsB;
  long long* accB;  // fixed-point per-bubble sums
  double *rhsB, *yB, *rb, *zb, *zvb, *pb, *apb;
  float *ybf, *pbf;  // bubble values as the f32 grid sees them
  // PCG vectors
  float *r, *z, *zOld, *p, *ap;
  // reductions
  double* parciais;
  Escalares* esc;
  // tanks of an atlas (tq_set_tanks): a cell (i, j) belongs to tank colTanque[i] when
  // y0T[t] <= j < y1T[t]; per tank the squared norms of the initial and the true residual
  int nTanques;
  int *colTanque, *y0T, *y1T;
  double *r0T, *rvT;
  int* tanqueBolha;  // per bubble label: its tank (-1: none)
};

// The tank of cell c, or -1 (no tanks, or a cell outside every tank).
__device__ inline int tanqueDe(const Dev& d, int c) {
  if (!d.nTanques) return -1;
  const int i = c % d.nx, j = c / d.nx;
  const int t = d.colTanque[i];
  return (t >= 0 && j >= d.y0T[t] && j < d.y1T[t]) ? t : -1;
}

// ------------------------------------------------------------ helpers
__host__ __device__ inline int clampi(int v, int a, int b) { return v < a ? a : v > b ? b : v; }

// Math.floor of a double used as an int, saturated (the reference clamps right after).
__device__ inline int floori(double v) {
  if (!(v == v)) return 0;
  if (v > 2e9) return 2000000000;
  if (v < -2e9) return -2000000000;
  return (int)floor(v);
}

__device__ inline double suave(double a, double b, double x) {  // js/fisica-cpu.js:692-695
  double t = fmin(1.0, fmax(0.0, (x - a) / (b - a)));
  return t * t * (3 - 2 * t);
}

// Bilinear SDF sample (Cena.#bilinear, js/cena.js:156-165) in double arithmetic.
__device__ inline double sdfBilinear(const float* __restrict__ sdf, int mw, int mh, double fx, double fy) {
  if (fx != fx || fy != fy) return nan("");
  double w = mw, hh = mh;
  if (fx < 0) fx = 0;
  else if (fx > w - 1) fx = w - 1;
  if (fy < 0) fy = 0;
  else if (fy > hh - 1) fy = hh - 1;
  int x0 = (int)fmin(floor(fx), w - 2), y0 = (int)fmin(floor(fy), hh - 2);
  double tx = fx - x0, ty = fy - y0;
  size_t k = (size_t)y0 * mw + x0;
  double a = sdf[k], b = sdf[k + 1], c = sdf[k + mw], d = sdf[k + mw + 1];
  return (a * (1 - tx) + b * tx) * (1 - ty) + (c * (1 - tx) + d * tx) * ty;
}

// Cena.distancia (js/cena.js:102-106)
__device__ inline double distancia(const Dev& d, double x, double y) {
  double fx = (x / d.h) * RES_MASCARA - 0.5, fy = (y / d.h) * RES_MASCARA - 0.5;
  return sdfBilinear(d.sdf, d.mw, d.mh, fx, fy);
}

// Cena.normal (js/cena.js:109-116)
__device__ inline void normalSdf(const Dev& d, double x, double y, double* nx, double* ny) {
  double fx = (x / d.h) * RES_MASCARA - 0.5, fy = (y / d.h) * RES_MASCARA - 0.5;
  double gx = sdfBilinear(d.sdf, d.mw, d.mh, fx + 1, fy) - sdfBilinear(d.sdf, d.mw, d.mh, fx - 1, fy);
  double gy = sdfBilinear(d.sdf, d.mw, d.mh, fx, fy + 1) - sdfBilinear(d.sdf, d.mw, d.mh, fx, fy - 1);
  double n = hypot(gx, gy);
  if (n > 1e-9) { *nx = gx / n; *ny = gy / n; }
  else { *nx = 0; *ny = 1; }
}

// Flat-index neighbour test with the reference's out-of-range semantics (a JS typed-array
// read past either end is `undefined`, equal to nothing).
__device__ inline bool tipoEm(const uint8_t* tipo, long c, long N, uint8_t t) {
  return c >= 0 && c < N && tipo[c] == t;
}

// Storage conversions of the multigrid vectors.
template <class T> __device__ inline float carregar(T v);
template <> __device__ inline float carregar<float>(float v) { return v; }
template <> __device__ inline float carregar<__half>(__half v) { return __half2float(v); }
template <> __device__ inline float carregar<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <class T> __device__ inline T guardar(float v);
template <> __device__ inline float guardar<float>(float v) { return v; }
template <> __device__ inline __half guardar<__half>(float v) { return __float2half_rn(v); }
template <> __device__ inline __nv_bfloat16 guardar<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

// Fixed-point accumulation of a double into a 64-bit integer.
__device__ inline void somaFixa(long long* acc, double v, double escala) {
  long long q = __double2ll_rn(v * escala);
  if (q) atomicAdd((unsigned long long*)acc, (unsigned long long)q);
}

inline int blocos(long n, int t) { return (int)((n + t - 1) / t); }

// Every kernel launch of the library goes through `lanca`, which counts it (the count is
// reported by tq_get_scalar(TQ_SCALAR_LAUNCHES)).
void contarLancamento();
template <class... P, class... A>
inline void lanca(void (*k)(P...), dim3 g, dim3 b, size_t sm, cudaStream_t s, A&&... a) {
  contarLancamento();
  k<<<g, b, sm, s>>>(static_cast<P>(a)...);
}

}  // namespace tq
