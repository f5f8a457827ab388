// sim.cu — the tq_sim handle and the C-ABI entry points of include/tanque.h: device memory,
// the substep orchestration (SimulacaoCPU.subpasso, js/fisica-cpu.js:176-189), state copies
// and error reporting.  Every entry point returns a status and never throws.
#include <array>
#include <atomic>
#include <cstddef>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

using namespace tq;

namespace tq {
static std::atomic<long long> g_lancamentos{0};
void contarLancamento() { g_lancamentos.fetch_add(1, std::memory_order_relaxed); }
}  // namespace tq

namespace {

thread_local char g_erro[512] = "";

int falha(int status, const char* msg) {
  std::snprintf(g_erro, sizeof g_erro, "%s", msg);
  return status;
}
int falhaCuda(cudaError_t e, const char* onde) {
  std::snprintf(g_erro, sizeof g_erro, "%s: %s", onde, cudaGetErrorString(e));
  return TQ_E_CUDA;
}
#define CK(expr)                                       \
  do {                                                 \
    cudaError_t e_ = (expr);                           \
    if (e_ != cudaSuccess) return falhaCuda(e_, #expr); \
  } while (0)

// Cena#moldura (js/cena.js:132-137): the empty tank's SDF.
void molduraSdf(std::vector<float>& sdf, int nx, int ny) {
  const int r = RES_MASCARA, mw = nx * r, mh = ny * r;
  sdf.resize((size_t)mw * mh);
  double m = MOLDURA * r - 0.5;
  for (int y = 0; y < mh; y++)
    for (int x = 0; x < mw; x++) {
      double d = std::fmin(std::fmin(x - m, (double)(mw - 1) - m - x), std::fmin(y - m, (double)(mh - 1) - m - y)) / r;
      d = d > SDF_MAX ? SDF_MAX : d < -SDF_MAX ? -SDF_MAX : d;
      sdf[(size_t)y * mw + x] = (float)d;
    }
}

}  // namespace

struct tq_sim {
  tq_options o;
  int nx, ny, N, nu, nv, mw, mh;
  cudaStream_t s = nullptr;
  Dev d{};
  int nHint = 0;
  unsigned long long proximoId = 0;
  bool tiposProntos = false;
  Pcg* pcg = nullptr;
  Rastreador* ar = nullptr;
  int *cont = nullptr, *offs = nullptr, *estado = nullptr;
  float* staging = nullptr;
  size_t stagingCap = 0;
  unsigned long long* mancha = nullptr;  // tq_splat's fixed-point sums (5 planes), grown on demand
  size_t manchaCap = 0;
  std::vector<void*> alocados;
  // Stage timing (tq_set_timing): a pool of events recorded at the stage boundaries of every
  // substep and relabel, read back once by tq_get_timing.
  bool timing = false;
  std::vector<cudaEvent_t> pool;
  size_t usados = 0;
  std::vector<std::array<int, 8>> regSub;
  std::vector<std::array<int, 2>> regAr;
  std::array<int, 8>* atual = nullptr;
  long long itersBase = 0;  // Escalares::itersAcum when timing started
  // tq_advance_graph: the substeps of a frame captured once and replayed; valid for the same dt
  // and substep count while the live particle count stays within the captured launch bound
  cudaGraph_t grafo = nullptr;
  cudaGraphExec_t grafoExec = nullptr;
  double grafoDt = 0, grafoG[2] = {0, 0};  // gravity is a kernel argument baked into the graph
  int grafoSub = 0, grafoN = -1;
  // device time of the last graph frame: events around its launch on the handle's stream
  cudaEvent_t quadroEv[2] = {nullptr, nullptr};
  bool quadroMedido = false;
};

namespace {

template <class T>
bool aloca(tq_sim* s, T** p, size_t n) {
  void* q = nullptr;
  if (cudaMalloc(&q, n * sizeof(T) + 16) != cudaSuccess) return false;
  cudaMemset(q, 0, n * sizeof(T) + 16);
  s->alocados.push_back(q);
  *p = (T*)q;
  return true;
}

int garantirStaging(tq_sim* s, size_t floats) {
  if (floats <= s->stagingCap) return TQ_OK;
  if (s->staging) cudaFree(s->staging);
  s->staging = nullptr;
  s->stagingCap = 0;
  size_t cap = floats < 4096 ? 4096 : floats;
  CK(cudaMalloc(&s->staging, cap * sizeof(float)));
  s->stagingCap = cap;
  return TQ_OK;
}

// Device count read back (the host only keeps an upper bound between calls).
int lerContagem(tq_sim* s, int* n) {
  CK(cudaMemcpyAsync(n, &s->d.esc->n, sizeof(int), cudaMemcpyDeviceToHost, s->s));
  CK(cudaStreamSynchronize(s->s));
  s->nHint = *n;
  return TQ_OK;
}

void compactar(tq_sim* s) { lancarCompactar(s->d, s->nHint, s->cont, s->offs, s->estado, s->s); }

constexpr size_t MAX_EVENTOS = 1 << 15;

// Records the next pool event on the stream; returns its index, or -1 when timing is off or
// the pool is exhausted.
int evento(tq_sim* s) {
  if (!s->timing) return -1;
  if (s->usados == s->pool.size()) {
    if (s->pool.size() >= MAX_EVENTOS) return -1;
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return -1;
    s->pool.push_back(e);
  }
  int i = (int)s->usados++;
  cudaEventRecord(s->pool[i], s->s);
  return i;
}
// Stage boundary i (0..7) of the running substep.
void marca(tq_sim* s, int i) {
  if (!s->timing) return;
  if (i == 0) {
    s->regSub.push_back({-1, -1, -1, -1, -1, -1, -1, -1});
    s->atual = &s->regSub.back();
  }
  if (s->atual) (*s->atual)[i] = evento(s);
}

// P2G + flags only (the first half of atualizarAr when the flags are stale, js/fisica-cpu.js:164).
void paraGradeETipos(tq_sim* s) {
  const Dev& d = s->d;
  cudaMemsetAsync(d.accU, 0, sizeof(int2) * d.nu, s->s);
  cudaMemsetAsync(d.accV, 0, sizeof(int2) * d.nv, s->s);
  cudaMemsetAsync(d.accCel, 0, sizeof(int2) * d.N, s->s);
  cudaMemsetAsync(d.accCor, 0, sizeof(int) * 3 * d.N, s->s);
  lancarP2G(d, s->nHint, s->s);
  lancarTipos(d, false, s->s);
  s->tiposProntos = true;
}

int subpasso(tq_sim* s, double dt) {
  const Dev& d = s->d;
  const bool ar = s->o.air != 0;
  cudaStream_t st = s->s;
  marca(s, 0);
  cudaMemsetAsync(d.accU, 0, sizeof(int2) * d.nu, st);
  cudaMemsetAsync(d.accV, 0, sizeof(int2) * d.nv, st);
  cudaMemsetAsync(d.accCel, 0, sizeof(int2) * d.N, st);
  cudaMemsetAsync(d.accCor, 0, sizeof(int) * 3 * d.N, st);
  lancarP2G(d, s->nHint, st);                                              // #paraGrade
  lancarFaces(d, (float)(s->o.gravity[0] * dt), (float)(s->o.gravity[1] * dt), st);  // #gravidadeEFronteira
  marca(s, 1);
  lancarTipos(d, ar, st);                                                  // #tipos
  s->tiposProntos = true;
  if (ar) lancarPropagarRotulos(d, st);                                    // #propagarRotulos
  marca(s, 2);
  lancarSuperficie(d, st);                                                 // #superficie
  marca(s, 3);
  lancarPressaoDoAr(d, dt, s->o.surface_tension, st);                      // #pressaoDoAr
  lancarClassificar(d, dt, s->o.tau_density, st);                          // #classificar
  if (ar) lancarLadoDireitoBolhas(d, dt, st);                              // #ladoDireitoDasBolhas
  marca(s, 4);
  int r = resolverPressao(s->pcg, d, s->o.iterations, s->o.tolerance, ar, s->o.preconditioner, st);  // #pressao
  if (r) return r == TQ_E_CUDA ? falha(r, "pressure solve failed") : r;
  lancarPosPressao(d, dt, ar, st);
  marca(s, 5);
  lancarGradiente(d, st);                                                  // #gradiente
  lancarExtrapolar(d, st);                                                 // #extrapolar
  marca(s, 6);
  cudaMemsetAsync(&d.esc->vmaxBits, 0, sizeof(unsigned long long), st);
  lancarG2P(d, s->nHint, dt, st);                                          // #paraParticulas
  marca(s, 7);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return falhaCuda(e, "substep launch");
  return TQ_OK;
}

int tamanhoCampo(tq_sim* s, int f, size_t* elems, size_t* elem) {
  const size_t N = s->N, nu = s->nu, nv = s->nv;
  switch (f) {
    case TQ_FIELD_TIPO: case TQ_FIELD_SOLIDO: *elems = N; *elem = 1; return TQ_OK;
    case TQ_FIELD_ROTULO: case TQ_FIELD_CONTAGEM: *elems = N; *elem = 4; return TQ_OK;
    case TQ_FIELD_U: case TQ_FIELD_U_PESO: *elems = nu; *elem = 4; return TQ_OK;
    case TQ_FIELD_V: case TQ_FIELD_V_PESO: *elems = nv; *elem = 4; return TQ_OK;
    case TQ_FIELD_U_VALIDA: *elems = nu; *elem = 1; return TQ_OK;
    case TQ_FIELD_V_VALIDA: *elems = nv; *elem = 1; return TQ_OK;
    case TQ_FIELD_Q: case TQ_FIELD_DIV: case TQ_FIELD_DENSIDADE: case TQ_FIELD_FASE: case TQ_FIELD_CURVATURA:
    case TQ_FIELD_QAR: case TQ_FIELD_NORMAL_X: case TQ_FIELD_NORMAL_Y: *elems = N; *elem = 4; return TQ_OK;
    case TQ_FIELD_PRESSAO_BOLHA: case TQ_FIELD_VOLUME_ALVO: case TQ_FIELD_VOLUME_BOLHA: case TQ_FIELD_RHS_BOLHA:
    case TQ_FIELD_Y_BOLHA: *elems = MAX_BOLHAS; *elem = 4; return TQ_OK;
    case TQ_FIELD_VIVO: *elems = MAX_BOLHAS; *elem = 1; return TQ_OK;
    case TQ_FIELD_COR_CELULA: case TQ_FIELD_ACC_COR: *elems = 3 * N; *elem = 4; return TQ_OK;
    case TQ_FIELD_ACC_U: *elems = 2 * nu; *elem = 4; return TQ_OK;
    case TQ_FIELD_ACC_V: *elems = 2 * nv; *elem = 4; return TQ_OK;
    case TQ_FIELD_ACC_CEL: *elems = 2 * N; *elem = 4; return TQ_OK;
    case TQ_FIELD_SDF: *elems = (size_t)s->mw * s->mh; *elem = 4; return TQ_OK;
  }
  return falha(TQ_E_ARG, "unknown field");
}

int baixar(tq_sim* s, void* dst, const void* src, size_t bytes) {
  CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s->s));
  CK(cudaStreamSynchronize(s->s));
  return TQ_OK;
}

__global__ void k_zerar_contagem(int2* acc, int n) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n) acc[c].y = 0;
}
__global__ void k_gravar_contagem(int2* acc, const uint32_t* cnt, int n) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n) acc[c].y = (int)cnt[c];
}

int iniciarCuda(int device) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) return falha(TQ_E_NODEV, "no CUDA device");
  if (device < 0 || device >= n) return falha(TQ_E_NODEV, "CUDA device ordinal out of range");
  CK(cudaSetDevice(device));
  return TQ_OK;
}

}  // namespace

// =============================================================== C-ABI
extern "C" {

void tq_options_default(tq_options* o, int32_t nx, int32_t ny, double h) {
  std::memset(o, 0, sizeof *o);
  o->nx = nx;
  o->ny = ny;
  o->h = h;
  o->gravity[0] = 0;
  o->gravity[1] = -GRAVIDADE;
  o->iterations = ITERACOES_PCG;
  o->air = 1;
  o->tau_density = TAU_DENSIDADE;
  o->surface_tension = TENSAO_SUPERFICIAL;
  o->tolerance = 0;
  o->precision = TQ_PREC_FP32;
  o->engine = TQ_ENGINE_PLAIN;
  o->p2g_mode = TQ_P2G_FIXED;
  o->capacity = 0;
  o->device = 0;
}

const char* tq_status_string(int st) {
  switch (st) {
    case TQ_OK: return "ok";
    case TQ_E_ARG: return "bad argument";
    case TQ_E_CUDA: return "CUDA error";
    case TQ_E_NOMEM: return "out of memory";
    case TQ_E_CAPACITY: return "capacity exceeded";
    case TQ_E_TIMEOUT: return "bounded device wait gave up";
    case TQ_E_NODEV: return "no CUDA device";
    case TQ_E_STATE: return "invalid state";
  }
  return "unknown status";
}
const char* tq_last_error(void) { return g_erro; }

int tq_create(const tq_options* o, tq_sim** out) {
  if (!o || !out) return falha(TQ_E_ARG, "null argument");
  *out = nullptr;
  if (o->nx < 3 || o->ny < 3 || !(o->h > 0)) return falha(TQ_E_ARG, "grid must be at least 3x3 with h > 0");
  if ((long long)o->nx * o->ny > (1LL << 28)) return falha(TQ_E_ARG, "grid too large");
  if (o->iterations < 1 || o->iterations > 1000) return falha(TQ_E_ARG, "iterations must be in [1, 1000]");
  if (o->p2g_mode != TQ_P2G_FIXED) return falha(TQ_E_ARG, "the CUDA library implements TQ_P2G_FIXED only");
  if (o->precision < TQ_PREC_FP32 || o->precision > TQ_PREC_BF16) return falha(TQ_E_ARG, "bad precision");
  if (o->engine != TQ_ENGINE_PLAIN && o->engine != TQ_ENGINE_FUSED) return falha(TQ_E_ARG, "bad engine");
  if (o->preconditioner < TQ_PRECOND_REFERENCE || o->preconditioner > TQ_PRECOND_BLOCK_1)
    return falha(TQ_E_ARG, "bad preconditioner");
  if (o->fused_ctas < 0) return falha(TQ_E_ARG, "fused_ctas must be >= 0");
  int st = iniciarCuda(o->device);
  if (st) return st;
  tq_sim* s = new (std::nothrow) tq_sim();
  if (!s) return falha(TQ_E_NOMEM, "host allocation failed");
  s->o = *o;
  s->nx = o->nx;
  s->ny = o->ny;
  s->N = o->nx * o->ny;
  s->nu = (o->nx + 1) * o->ny;
  s->nv = o->nx * (o->ny + 1);
  s->mw = o->nx * RES_MASCARA;
  s->mh = o->ny * RES_MASCARA;
  int cap = o->capacity > 0 ? o->capacity : (int)std::ceil(s->N * PARTICULAS_MAX_POR_CELULA);
  if (cudaStreamCreateWithFlags(&s->s, cudaStreamNonBlocking) != cudaSuccess) {
    delete s;
    return falha(TQ_E_CUDA, "stream creation failed");
  }
  Dev& d = s->d;
  d.nx = s->nx;
  d.ny = s->ny;
  d.N = s->N;
  d.nu = s->nu;
  d.nv = s->nv;
  d.mw = s->mw;
  d.mh = s->mh;
  d.h = o->h;
  d.hf = (float)o->h;
  d.cap = cap;
  const size_t N = s->N, nu = s->nu, nv = s->nv;
  float* sdf = nullptr;
  bool ok = aloca(s, &sdf, (size_t)s->mw * s->mh);
  d.sdf = sdf;
  ok = ok && aloca(s, &d.solido, N) && aloca(s, &d.p0, cap) && aloca(s, &d.p1, cap) && aloca(s, &d.p2, cap) &&
       aloca(s, &d.pid, cap) && aloca(s, &d.q0, cap) && aloca(s, &d.q1, cap) && aloca(s, &d.q2, cap) &&
       aloca(s, &d.qid, cap) && aloca(s, &d.accU, nu) && aloca(s, &d.accV, nv) && aloca(s, &d.accCel, N) &&
       aloca(s, &d.accCor, 3 * N) && aloca(s, &d.u, nu) && aloca(s, &d.v, nv) && aloca(s, &d.uTmp, nu) &&
       aloca(s, &d.vTmp, nv) && aloca(s, &d.uVal, nu) && aloca(s, &d.vVal, nv) && aloca(s, &d.uValTmp, nu) &&
       aloca(s, &d.vValTmp, nv) && aloca(s, &d.tipo, N) && aloca(s, &d.rotulo, N) && aloca(s, &d.pend, N) &&
       aloca(s, &d.lista, N) && aloca(s, &d.div, N) && aloca(s, &d.q, N) && aloca(s, &d.qAr, N) &&
       aloca(s, &d.fase, N) && aloca(s, &d.faseTmp, N) && aloca(s, &d.nX, N) && aloca(s, &d.nY, N) &&
       aloca(s, &d.kap, N) && aloca(s, &d.cheio, N) && aloca(s, &d.cheioTmp, N) &&
       aloca(s, &d.pressaoBolha, MAX_BOLHAS) && aloca(s, &d.volumeAlvo, MAX_BOLHAS) &&
       aloca(s, &d.volumeBolhaF, MAX_BOLHAS) && aloca(s, &d.rhsBolhaF, MAX_BOLHAS) &&
       aloca(s, &d.yBolhaF, MAX_BOLHAS) && aloca(s, &d.vivo, MAX_BOLHAS) && aloca(s, &d.volB, MAX_BOLHAS) &&
       aloca(s, &d.facesB, MAX_BOLHAS) && aloca(s, &d.celsB, MAX_BOLHAS) && aloca(s, &d.accB, MAX_BOLHAS) &&
       aloca(s, &d.rhsB, MAX_BOLHAS) && aloca(s, &d.yB, MAX_BOLHAS) && aloca(s, &d.rb, MAX_BOLHAS) &&
       aloca(s, &d.zb, MAX_BOLHAS) && aloca(s, &d.zvb, MAX_BOLHAS) && aloca(s, &d.pb, MAX_BOLHAS) &&
       aloca(s, &d.apb, MAX_BOLHAS) && aloca(s, &d.ybf, MAX_BOLHAS) && aloca(s, &d.pbf, MAX_BOLHAS) &&
       aloca(s, &d.r, N) && aloca(s, &d.z, N) && aloca(s, &d.zOld, N) && aloca(s, &d.p, N) &&
       aloca(s, &d.ap, N) && aloca(s, &d.parciais, 4096) && aloca(s, &d.esc, 1);
  int nbMax = blocos(cap > (int)N ? cap : (int)N, 1024) + 1;
  ok = ok && aloca(s, &s->cont, nbMax) && aloca(s, &s->offs, nbMax) && aloca(s, &s->estado, 4);
  if (ok) s->pcg = criarPcg(s->nx, s->ny, o->precision, o->engine, o->fused_ctas);
  if (ok && s->pcg) s->ar = criarRastreador(s->nx, s->ny);
  if (!ok || !s->pcg || !s->ar) {
    tq_destroy(s);
    return falha(TQ_E_NOMEM, "device allocation failed");
  }
  std::vector<float> m;
  molduraSdf(m, s->nx, s->ny);
  if (cudaMemcpy(sdf, m.data(), m.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
    tq_destroy(s);
    return falha(TQ_E_CUDA, "upload failed");
  }
  lancarSolidos(d, s->s);
  if (cudaStreamSynchronize(s->s) != cudaSuccess) {
    tq_destroy(s);
    return falha(TQ_E_CUDA, "initialisation failed");
  }
  *out = s;
  return TQ_OK;
}

int tq_destroy(tq_sim* s) {
  if (!s) return TQ_OK;
  if (s->s) cudaStreamSynchronize(s->s);
  if (s->grafoExec) cudaGraphExecDestroy(s->grafoExec);
  if (s->grafo) cudaGraphDestroy(s->grafo);
  for (auto& e : s->quadroEv)
    if (e) cudaEventDestroy(e);
  destruirPcg(s->pcg);
  destruirRastreador(s->ar);
  for (void* p : s->alocados) cudaFree(p);
  if (s->staging) cudaFree(s->staging);
  if (s->mancha) cudaFree(s->mancha);
  for (auto& e : s->pool) cudaEventDestroy(e);
  if (s->s) cudaStreamDestroy(s->s);
  delete s;
  return TQ_OK;
}

int tq_set_walls(tq_sim* s, const float* sdf, int32_t mw, int32_t mh) {
  if (!s || !sdf) return falha(TQ_E_ARG, "null argument");
  if (mw != s->mw || mh != s->mh) return falha(TQ_E_ARG, "sdf must be (2*nx) x (2*ny)");
  CK(cudaMemcpyAsync((void*)s->d.sdf, sdf, (size_t)mw * mh * 4, cudaMemcpyHostToDevice, s->s));
  lancarSolidos(s->d, s->s);
  CK(cudaStreamSynchronize(s->s));
  return TQ_OK;
}

int tq_trace_wall(tq_sim* s, double x0, double y0, double x1, double y1, double radius, int32_t erase) {
  if (!s) return falha(TQ_E_ARG, "null handle");
  if (!std::isfinite(x0) || !std::isfinite(y0) || !std::isfinite(x1) || !std::isfinite(y1) || !std::isfinite(radius))
    return falha(TQ_E_ARG, "non-finite wall segment");
  lancarTracar(s->d, x0, y0, x1, y1, radius, erase != 0, s->s);
  lancarSolidos(s->d, s->s);
  CK(cudaStreamSynchronize(s->s));
  return TQ_OK;
}

int tq_clear_walls(tq_sim* s) {
  if (!s) return falha(TQ_E_ARG, "null handle");
  lancarZerarMascara(s->d, s->s);
  lancarSolidos(s->d, s->s);
  CK(cudaStreamSynchronize(s->s));
  return TQ_OK;
}

int tq_splat(tq_sim* s, int32_t w, int32_t h, float* out) {
  if (!s || !out) return falha(TQ_E_ARG, "null argument");
  if (w < 1 || h < 1 || (long long)w * h > (1LL << 26)) return falha(TQ_E_ARG, "target must be 1..2^26 pixels");
  const size_t total = (size_t)5 * w * h;
  if (total > s->manchaCap) {
    if (s->mancha) cudaFree(s->mancha);
    s->mancha = nullptr;
    s->manchaCap = 0;
    CK(cudaMalloc(&s->mancha, total * sizeof(unsigned long long)));
    s->manchaCap = total;
  }
  int n = 0;
  int st = lerContagem(s, &n);
  if (st) return st;
  lancarMancha(s->d, n, w, h, s->mancha, out, s->s);
  CK(cudaStreamSynchronize(s->s));
  return TQ_OK;
}

int tq_add_particles(tq_sim* s, const float* list, int32_t n, int32_t check, int32_t* accepted) {
  if (!s || (n > 0 && !list) || n < 0) return falha(TQ_E_ARG, "bad particle list");
  if (accepted) *accepted = 0;
  if (n == 0) return TQ_OK;
  int atual = 0;
  int st = lerContagem(s, &atual);
  if (st) return st;
  if ((long long)atual + n > s->d.cap) return falha(TQ_E_CAPACITY, "particle capacity exceeded");
  st = garantirStaging(s, (size_t)n * CAMPOS);
  if (st) return st;
  CK(cudaMemcpyAsync(s->staging, list, (size_t)n * CAMPOS * 4, cudaMemcpyHostToDevice, s->s));
  lancarAdicionar(s->d, s->staging, n, check ? 1 : 0, s->cont, s->offs, s->proximoId, s->s);
  int a = 0;
  CK(cudaMemcpyAsync(&a, &s->d.esc->aceitas, sizeof(int), cudaMemcpyDeviceToHost, s->s));
  CK(cudaStreamSynchronize(s->s));
  s->proximoId += (unsigned long long)a;
  s->nHint = atual + a;
  if (accepted) *accepted = a;
  return TQ_OK;
}

int tq_set_tanks(tq_sim* s, int32_t n, const int32_t* rects) {
  if (!s || n < 0 || (n > 0 && !rects)) return falha(TQ_E_ARG, "bad tank list");
  if (n > MAX_TANQUES) return falha(TQ_E_CAPACITY, "more tanks than an atlas may hold (4096)");
  if (n > 0 && motorPcg(s->pcg) != TQ_ENGINE_FUSED)
    return falha(TQ_E_STATE, "per-tank convergence needs the fused engine");
  std::vector<int> col(s->nx, -1), y0(n > 0 ? n : 1), y1(n > 0 ? n : 1);
  for (int t = 0; t < n; t++) {
    const int x0 = rects[4 * t], yy = rects[4 * t + 1], w = rects[4 * t + 2], hh = rects[4 * t + 3];
    if (x0 < 0 || yy < 0 || w < 1 || hh < 1 || x0 + w > s->nx || yy + hh > s->ny)
      return falha(TQ_E_ARG, "tank rectangle outside the grid");
    for (int i = x0; i < x0 + w; i++) {
      if (col[i] >= 0) return falha(TQ_E_ARG, "tanks must occupy disjoint column ranges");
      col[i] = t;
    }
    y0[t] = yy;
    y1[t] = yy + hh;
  }
  Dev& d = s->d;
  if (!d.colTanque) {
    if (!aloca(s, &d.colTanque, s->nx) || !aloca(s, &d.y0T, MAX_TANQUES) || !aloca(s, &d.y1T, MAX_TANQUES) ||
        !aloca(s, &d.r0T, MAX_TANQUES) || !aloca(s, &d.rvT, MAX_TANQUES) || !aloca(s, &d.tanqueBolha, MAX_BOLHAS))
      return falha(TQ_E_NOMEM, "device allocation failed");
  }
  CK(cudaMemcpyAsync(d.colTanque, col.data(), sizeof(int) * s->nx, cudaMemcpyHostToDevice, s->s));
  if (n > 0) {
    CK(cudaMemcpyAsync(d.y0T, y0.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s->s));
    CK(cudaMemcpyAsync(d.y1T, y1.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s->s));
    CK(cudaMemsetAsync(d.r0T, 0, sizeof(double) * n, s->s));
    CK(cudaMemsetAsync(d.rvT, 0, sizeof(double) * n, s->s));
  }
  CK(cudaStreamSynchronize(s->s));
  d.nTanques = n;
  return TQ_OK;
}

int tq_get_tank_residuals(tq_sim* s, double* out, int32_t cap, int32_t* n) {
  if (!s) return falha(TQ_E_ARG, "null handle");
  const int nt = s->d.nTanques;
  if (n) *n = nt;
  if (!out || nt == 0) return TQ_OK;
  std::vector<double> r0(nt), rv(nt);
  CK(cudaMemcpyAsync(r0.data(), s->d.r0T, sizeof(double) * nt, cudaMemcpyDeviceToHost, s->s));
  CK(cudaMemcpyAsync(rv.data(), s->d.rvT, sizeof(double) * nt, cudaMemcpyDeviceToHost, s->s));
  CK(cudaStreamSynchronize(s->s));
  for (int t = 0; t < nt && 2 * t + 1 < cap; t++) {
    out[2 * t] = std::sqrt(r0[t]);
    out[2 * t + 1] = std::sqrt(rv[t]);
  }
  return TQ_OK;
}

int tq_emit_faucet(tq_sim* s, const tq_faucet* f, int32_t* accepted) {
  if (!s || !f) return falha(TQ_E_ARG, "null argument");
  if (accepted) *accepted = 0;
  if (!std::isfinite(f->x) || !std::isfinite(f->y) || !(f->radius >= 0) || !std::isfinite(f->vx) ||
      !std::isfinite(f->vy) || !(f->dt >= 0) || !std::isfinite(f->radius) || !std::isfinite(f->dt))
    return falha(TQ_E_ARG, "non-finite or negative faucet parameters");
  // n = min(40000, Math.round((vazao * dt) / h^2 * PARTICULAS_POR_CELULA)), vazao = 2 r max(0.7, |v|)
  const double h = s->o.h;
  const double vazao = 2 * f->radius * std::fmax(0.7, std::hypot(f->vx, f->vy));
  const double nr = std::floor((vazao * f->dt) / (h * h) * PARTICULAS_POR_CELULA + 0.5);
  const int n = (int)std::fmin(40000.0, nr);
  if (n <= 0) return TQ_OK;
  int atual = 0;
  int st = lerContagem(s, &atual);
  if (st) return st;
  if ((long long)atual + n > s->d.cap) return falha(TQ_E_CAPACITY, "particle capacity exceeded");
  st = garantirStaging(s, (size_t)n * CAMPOS);
  if (st) return st;
  const float ab[3] = {(float)f->absorb[0], (float)f->absorb[1], (float)f->absorb[2]};
  lancarTorneira(s->staging, n, f->seed, f->x, f->y, f->radius, (float)f->vx, (float)f->vy, ab, s->s);
  lancarAdicionar(s->d, s->staging, n, 1, s->cont, s->offs, s->proximoId, s->s);  // motor.adicionar(lista, true)
  int a = 0;
  CK(cudaMemcpyAsync(&a, &s->d.esc->aceitas, sizeof(int), cudaMemcpyDeviceToHost, s->s));
  CK(cudaStreamSynchronize(s->s));
  s->proximoId += (unsigned long long)a;
  s->nHint = atual + a;
  if (accepted) *accepted = a;
  return TQ_OK;
}

int tq_clear_particles(tq_sim* s) {
  if (!s) return falha(TQ_E_ARG, "null handle");
  CK(cudaMemsetAsync(&s->d.esc->n, 0, sizeof(int), s->s));
  CK(cudaMemsetAsync(&s->d.esc->mortas, 0, sizeof(int), s->s));
  lanca(k_zerar_contagem, blocos(s->N, 256), 256, 0, s->s, s->d.accCel, s->N);
  CK(cudaStreamSynchronize(s->s));
  s->nHint = 0;
  return TQ_OK;
}

int tq_apply_tool(tq_sim* s, const tq_tool* t) {
  if (!s || !t) return falha(TQ_E_ARG, "null argument");
  if (t->kind == 0) return TQ_OK;
  if (t->kind < 0 || t->kind > 3) return falha(TQ_E_ARG, "bad tool kind");
  lancarFerramenta(s->d, s->nHint, *t, s->s);
  compactar(s);
  CK(cudaGetLastError());
  return TQ_OK;
}

int tq_update_air(tq_sim* s) {
  if (!s) return falha(TQ_E_ARG, "null handle");
  if (!s->tiposProntos) paraGradeETipos(s);
  int e0 = evento(s);
  int r = atualizarRastreador(s->ar, s->d, s->s);
  int e1 = evento(s);
  if (e0 >= 0 && e1 >= 0) s->regAr.push_back({e0, e1});
  if (r == TQ_E_TIMEOUT) return falha(r, "air labelling: union-find retry bound reached");
  if (r) return falha(r, "air labelling failed");
  return TQ_OK;
}

int tq_reset_air(tq_sim* s) {
  if (!s) return falha(TQ_E_ARG, "null handle");
  s->tiposProntos = false;
  reiniciarRastreador(s->ar, s->d, s->s);
  CK(cudaMemsetAsync(s->d.pressaoBolha, 0, MAX_BOLHAS * 4, s->s));
  CK(cudaStreamSynchronize(s->s));
  return TQ_OK;
}

// The end of tq_substep / tq_advance: compaction, launch errors, and a fused solve that gave up
// on a bounded wait (waits for the stream once).
static int fimDePasso(tq_sim* s) {
  compactar(s);
  CK(cudaGetLastError());
  int r = erroPcg(s->pcg, s->s);
  if (r == TQ_E_TIMEOUT) return falha(r, "pressure solve: a grid barrier wait gave up");
  if (r) return falhaCuda(cudaGetLastError(), "pressure solve");
  return TQ_OK;
}

int tq_substep(tq_sim* s, double dt) {
  if (!s) return falha(TQ_E_ARG, "null handle");
  if (!(dt > 0)) return falha(TQ_E_ARG, "dt must be > 0");
  int r = subpasso(s, dt);
  if (r) return r;
  return fimDePasso(s);
}

int tq_advance(tq_sim* s, double dt, int32_t sub) {
  if (!s) return falha(TQ_E_ARG, "null handle");
  if (!(dt > 0) || sub < 1) return falha(TQ_E_ARG, "need dt > 0 and substeps >= 1");
  if (s->o.air) {
    int r = tq_update_air(s);
    if (r) return r;
  }
  double d = dt / sub;
  for (int k = 0; k < sub; k++) {
    int r = subpasso(s, d);
    if (r) return r;
  }
  return fimDePasso(s);
}

// tq_advance_graph without the final wait: the frame is queued on the handle's stream and its
// solve errors are reported by tq_sync.
static int lancarGrafo(tq_sim* s, double dt, int32_t sub);

int tq_advance_graph(tq_sim* s, double dt, int32_t sub) {
  int r = lancarGrafo(s, dt, sub);
  return r ? r : fimDePasso(s);
}

int tq_launch_graph(tq_sim* s, double dt, int32_t sub) {
  int r = lancarGrafo(s, dt, sub);
  if (r) return r;
  compactar(s);
  CK(cudaGetLastError());
  return TQ_OK;
}

static int lancarGrafo(tq_sim* s, double dt, int32_t sub) {
  if (!s) return falha(TQ_E_ARG, "null handle");
  if (!(dt > 0) || sub < 1) return falha(TQ_E_ARG, "need dt > 0 and substeps >= 1");
  if (motorPcg(s->pcg) == TQ_ENGINE_PLAIN && s->o.tolerance > 0)
    return falha(TQ_E_STATE, "the plain engine reads its stop flag on the host in tolerance mode: not capturable");
  if (s->o.air) {
    int r = tq_update_air(s);
    if (r) return r;
  }
  const bool timing = s->timing;
  if (!s->grafoExec || s->grafoDt != dt || s->grafoSub != sub || s->nHint > s->grafoN ||
      s->grafoG[0] != s->o.gravity[0] || s->grafoG[1] != s->o.gravity[1]) {
    if (s->grafoExec) cudaGraphExecDestroy(s->grafoExec);
    if (s->grafo) cudaGraphDestroy(s->grafo);
    s->grafoExec = nullptr;
    s->grafo = nullptr;
    s->timing = false;  // stage events are not recorded into the graph
    if (s->o.tolerance > 0 && reservarTolerancia(s->pcg)) {  // no allocation inside the capture
      s->timing = timing;
      return falha(TQ_E_NOMEM, "tolerance-mode buffers");
    }
    CK(cudaStreamBeginCapture(s->s, cudaStreamCaptureModeThreadLocal));
    int r = TQ_OK;
    for (int k = 0; k < sub && !r; k++) r = subpasso(s, dt / sub);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->s, &g);
    s->timing = timing;
    if (r) {
      if (g) cudaGraphDestroy(g);
      return r;
    }
    if (e != cudaSuccess) return falhaCuda(e, "capturing the frame's substeps");
    e = cudaGraphInstantiate(&s->grafoExec, g, 0);
    if (e != cudaSuccess) {
      cudaGraphDestroy(g);
      s->grafoExec = nullptr;
      return falhaCuda(e, "instantiating the frame's graph");
    }
    s->grafo = g;
    s->grafoDt = dt;
    s->grafoSub = sub;
    s->grafoN = s->nHint;
    s->grafoG[0] = s->o.gravity[0];
    s->grafoG[1] = s->o.gravity[1];
  }
  if (!s->quadroEv[0] && (cudaEventCreate(&s->quadroEv[0]) != cudaSuccess ||
                          cudaEventCreate(&s->quadroEv[1]) != cudaSuccess))
    return falhaCuda(cudaGetLastError(), "frame events");
  CK(cudaEventRecord(s->quadroEv[0], s->s));
  contarLancamento();
  CK(cudaGraphLaunch(s->grafoExec, s->s));
  CK(cudaEventRecord(s->quadroEv[1], s->s));
  s->quadroMedido = true;
  return TQ_OK;
}

int tq_count(tq_sim* s, int32_t* n) {
  if (!s || !n) return falha(TQ_E_ARG, "null argument");
  int v = 0;
  int st = lerContagem(s, &v);
  if (st) return st;
  *n = v;
  return TQ_OK;
}

int tq_get_particles(tq_sim* s, float* out, int32_t cap, int32_t* n) {
  if (!s) return falha(TQ_E_ARG, "null handle");
  int v = 0;
  int st = lerContagem(s, &v);
  if (st) return st;
  if (n) *n = v;
  if (!out) return TQ_OK;
  if (cap < v) return falha(TQ_E_ARG, "output buffer too small");
  if (v == 0) return TQ_OK;
  st = garantirStaging(s, (size_t)v * CAMPOS);
  if (st) return st;
  lancarEmpacotar(s->d, s->staging, v, s->s);
  CK(cudaMemcpyAsync(out, s->staging, (size_t)v * CAMPOS * 4, cudaMemcpyDeviceToHost, s->s));
  CK(cudaStreamSynchronize(s->s));
  return TQ_OK;
}

int tq_set_particles(tq_sim* s, const float* list, int32_t n) {
  if (!s || n < 0 || (n > 0 && !list)) return falha(TQ_E_ARG, "bad particle list");
  if (n > s->d.cap) return falha(TQ_E_CAPACITY, "particle capacity exceeded");
  if (n > 0) {
    int st = garantirStaging(s, (size_t)n * CAMPOS);
    if (st) return st;
    CK(cudaMemcpyAsync(s->staging, list, (size_t)n * CAMPOS * 4, cudaMemcpyHostToDevice, s->s));
    lancarDesempacotar(s->d, s->staging, n, s->proximoId, s->s);
  }
  s->proximoId += (unsigned long long)n;
  CK(cudaMemcpyAsync(&s->d.esc->n, &n, sizeof(int), cudaMemcpyHostToDevice, s->s));
  CK(cudaMemsetAsync(&s->d.esc->mortas, 0, sizeof(int), s->s));
  CK(cudaStreamSynchronize(s->s));
  s->nHint = n;
  return TQ_OK;
}

int tq_get_field(tq_sim* s, int32_t f, void* out, int64_t bytes) {
  if (!s || !out) return falha(TQ_E_ARG, "null argument");
  size_t elems, elem;
  int st = tamanhoCampo(s, f, &elems, &elem);
  if (st) return st;
  if ((size_t)bytes != elems * elem) return falha(TQ_E_ARG, "field size mismatch");
  const Dev& d = s->d;
  switch (f) {
    case TQ_FIELD_TIPO: return baixar(s, out, d.tipo, bytes);
    case TQ_FIELD_SOLIDO: return baixar(s, out, d.solido, bytes);
    case TQ_FIELD_ROTULO: return baixar(s, out, d.rotulo, bytes);
    case TQ_FIELD_U: return baixar(s, out, d.u, bytes);
    case TQ_FIELD_V: return baixar(s, out, d.v, bytes);
    case TQ_FIELD_U_VALIDA: return baixar(s, out, d.uVal, bytes);
    case TQ_FIELD_V_VALIDA: return baixar(s, out, d.vVal, bytes);
    case TQ_FIELD_Q: return baixar(s, out, d.q, bytes);
    case TQ_FIELD_DIV: return baixar(s, out, d.div, bytes);
    case TQ_FIELD_FASE: return baixar(s, out, d.fase, bytes);
    case TQ_FIELD_CURVATURA: return baixar(s, out, d.kap, bytes);
    case TQ_FIELD_QAR: return baixar(s, out, d.qAr, bytes);
    case TQ_FIELD_NORMAL_X: return baixar(s, out, d.nX, bytes);
    case TQ_FIELD_NORMAL_Y: return baixar(s, out, d.nY, bytes);
    case TQ_FIELD_PRESSAO_BOLHA: return baixar(s, out, d.pressaoBolha, bytes);
    case TQ_FIELD_VOLUME_ALVO: return baixar(s, out, d.volumeAlvo, bytes);
    case TQ_FIELD_VOLUME_BOLHA: return baixar(s, out, d.volumeBolhaF, bytes);
    case TQ_FIELD_RHS_BOLHA: return baixar(s, out, d.rhsBolhaF, bytes);
    case TQ_FIELD_Y_BOLHA: return baixar(s, out, d.yBolhaF, bytes);
    case TQ_FIELD_VIVO: return baixar(s, out, d.vivo, bytes);
    case TQ_FIELD_ACC_U: return baixar(s, out, d.accU, bytes);
    case TQ_FIELD_ACC_V: return baixar(s, out, d.accV, bytes);
    case TQ_FIELD_ACC_CEL: return baixar(s, out, d.accCel, bytes);
    case TQ_FIELD_ACC_COR: return baixar(s, out, d.accCor, bytes);
    case TQ_FIELD_SDF: return baixar(s, out, d.sdf, bytes);
    case TQ_FIELD_CONTAGEM:
    case TQ_FIELD_DENSIDADE: {
      std::vector<int2> a(s->N);
      st = baixar(s, a.data(), d.accCel, a.size() * sizeof(int2));
      if (st) return st;
      for (int c = 0; c < s->N; c++) {
        if (f == TQ_FIELD_CONTAGEM) ((uint32_t*)out)[c] = (uint32_t)a[c].y;
        else ((float*)out)[c] = (float)a[c].x * (1.0f / 65536.0f);
      }
      return TQ_OK;
    }
    case TQ_FIELD_U_PESO:
    case TQ_FIELD_V_PESO: {
      size_t n = f == TQ_FIELD_U_PESO ? s->nu : s->nv;
      std::vector<int2> a(n);
      st = baixar(s, a.data(), f == TQ_FIELD_U_PESO ? d.accU : d.accV, n * sizeof(int2));
      if (st) return st;
      for (size_t k = 0; k < n; k++) ((float*)out)[k] = (float)a[k].y * (1.0f / 65536.0f);
      return TQ_OK;
    }
    case TQ_FIELD_COR_CELULA: {
      std::vector<int> a(3 * (size_t)s->N);
      st = baixar(s, a.data(), d.accCor, a.size() * 4);
      if (st) return st;
      for (size_t k = 0; k < a.size(); k++) ((float*)out)[k] = (float)a[k] * (1.0f / 256.0f);
      return TQ_OK;
    }
  }
  return falha(TQ_E_ARG, "unknown field");
}

int tq_set_field(tq_sim* s, int32_t f, const void* in, int64_t bytes) {
  if (!s || !in) return falha(TQ_E_ARG, "null argument");
  size_t elems, elem;
  int st = tamanhoCampo(s, f, &elems, &elem);
  if (st) return st;
  if ((size_t)bytes != elems * elem) return falha(TQ_E_ARG, "field size mismatch");
  const Dev& d = s->d;
  void* dst = nullptr;
  switch (f) {
    case TQ_FIELD_TIPO: dst = d.tipo; break;
    case TQ_FIELD_ROTULO: dst = d.rotulo; break;
    case TQ_FIELD_Q: dst = d.q; break;
    case TQ_FIELD_PRESSAO_BOLHA: dst = d.pressaoBolha; break;
    case TQ_FIELD_VOLUME_ALVO: dst = d.volumeAlvo; break;
    case TQ_FIELD_Y_BOLHA: dst = d.yBolhaF; break;
    case TQ_FIELD_VIVO: dst = d.vivo; break;
    case TQ_FIELD_SDF: dst = (void*)d.sdf; break;
    case TQ_FIELD_CONTAGEM: {
      uint32_t* tmp = nullptr;
      CK(cudaMallocAsync((void**)&tmp, bytes, s->s));
      CK(cudaMemcpyAsync(tmp, in, bytes, cudaMemcpyHostToDevice, s->s));
      lanca(k_gravar_contagem, blocos(s->N, 256), 256, 0, s->s, d.accCel, tmp, s->N);
      CK(cudaFreeAsync(tmp, s->s));
      CK(cudaStreamSynchronize(s->s));
      return TQ_OK;
    }
    default: return falha(TQ_E_ARG, "field is not writable");
  }
  CK(cudaMemcpyAsync(dst, in, bytes, cudaMemcpyHostToDevice, s->s));
  if (f == TQ_FIELD_SDF) lancarSolidos(d, s->s);
  CK(cudaStreamSynchronize(s->s));
  return TQ_OK;
}

int tq_get_scalar(tq_sim* s, int32_t w, double* out) {
  if (out && w == TQ_SCALAR_LAUNCHES) {  // process-wide: no handle needed
    *out = (double)g_lancamentos.load();
    return TQ_OK;
  }
  if (!s || !out) return falha(TQ_E_ARG, "null argument");
  switch (w) {
    case TQ_SCALAR_VMAX: {
      unsigned long long b = 0;
      int st = baixar(s, &b, &s->d.esc->vmaxBits, sizeof b);
      if (st) return st;
      double v;
      std::memcpy(&v, &b, 8);
      *out = v;
      return TQ_OK;
    }
    case TQ_SCALAR_LAUNCHES: *out = (double)g_lancamentos.load(); return TQ_OK;
    case TQ_SCALAR_PRIMEIRA: *out = primeiraRastreador(s->ar); return TQ_OK;
    case TQ_SCALAR_TIPOS_PRONTOS: *out = s->tiposProntos ? 1 : 0; return TQ_OK;
    case TQ_SCALAR_PCG_ITERS: {
      int v = 0;
      int st = baixar(s, &v, &s->d.esc->iters, sizeof v);
      if (st) return st;
      *out = v;
      return TQ_OK;
    }
    case TQ_SCALAR_PCG_TRUE_RES: return baixar(s, out, &s->d.esc->normaVerd, sizeof(double));
    case TQ_SCALAR_GRAPH_FRAME_MS: {
      *out = 0.0;
      if (!s->quadroMedido) return TQ_OK;
      CK(cudaEventSynchronize(s->quadroEv[1]));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, s->quadroEv[0], s->quadroEv[1]));
      *out = ms;
      return TQ_OK;
    }
    case TQ_SCALAR_CLOSED_REGIONS: {
      int v = 0;
      int st = baixar(s, &v, &s->d.esc->regioes, sizeof v);
      if (st) return st;
      *out = v;
      return TQ_OK;
    }
    case TQ_SCALAR_PCG_CONVERGED:
    case TQ_SCALAR_SOLVES:
    case TQ_SCALAR_SOLVES_CAPPED:
    case TQ_SCALAR_SOLVE_ITERS:
    case TQ_SCALAR_SOLVE_MAX_REL:
    case TQ_SCALAR_SOLVE_REPLACEMENTS: {
      Escalares e;
      int st = baixar(s, &e, s->d.esc, offsetof(Escalares, normas));
      if (st) return st;
      *out = w == TQ_SCALAR_PCG_CONVERGED  ? (double)e.convergiu
             : w == TQ_SCALAR_SOLVES       ? (double)e.solves
             : w == TQ_SCALAR_SOLVES_CAPPED ? (double)e.capados
             : w == TQ_SCALAR_SOLVE_ITERS  ? (double)e.itersAcum
             : w == TQ_SCALAR_SOLVE_MAX_REL ? e.maxRel
                                            : (double)e.trocasAcum;
      return TQ_OK;
    }
    case TQ_SCALAR_GRAVITY_X: *out = s->o.gravity[0]; return TQ_OK;
    case TQ_SCALAR_GRAVITY_Y: *out = s->o.gravity[1]; return TQ_OK;
    case TQ_SCALAR_PCG_RES0:
    case TQ_SCALAR_PCG_RES: {
      double v[2];
      int st = baixar(s, v, &s->d.esc->norma0, sizeof v);
      if (st) return st;
      *out = w == TQ_SCALAR_PCG_RES0 ? v[0] : v[1];
      return TQ_OK;
    }
  }
  return falha(TQ_E_ARG, "unknown scalar");
}

int tq_set_scalar(tq_sim* s, int32_t w, double v) {
  if (!s) return falha(TQ_E_ARG, "null handle");
  switch (w) {
    case TQ_SCALAR_PRIMEIRA: definirPrimeiraRastreador(s->ar, v != 0); return TQ_OK;
    case TQ_SCALAR_TIPOS_PRONTOS: s->tiposProntos = v != 0; return TQ_OK;
    case TQ_SCALAR_GRAVITY_X: s->o.gravity[0] = v; return TQ_OK;
    case TQ_SCALAR_GRAVITY_Y: s->o.gravity[1] = v; return TQ_OK;
    case TQ_SCALAR_SOLVES: {  // 0 resets the accumulated solve statistics
      if (v != 0) return falha(TQ_E_ARG, "TQ_SCALAR_SOLVES can only be reset to 0");
      Escalares* e = s->d.esc;
      CK(cudaMemsetAsync(&e->solves, 0, sizeof e->solves + sizeof e->capados + sizeof e->itersAcum +
                                            sizeof e->trocasAcum + sizeof e->maxRel, s->s));
      CK(cudaStreamSynchronize(s->s));
      s->itersBase = 0;  // the stage timing counts iterations from the same origin
      return TQ_OK;
    }
    case TQ_SCALAR_VMAX: {
      unsigned long long b;
      std::memcpy(&b, &v, 8);
      CK(cudaMemcpyAsync(&s->d.esc->vmaxBits, &b, 8, cudaMemcpyHostToDevice, s->s));
      CK(cudaStreamSynchronize(s->s));
      return TQ_OK;
    }
  }
  return falha(TQ_E_ARG, "scalar not writable");
}

int tq_last_norms(tq_sim* s, double* out, int32_t cap, int32_t* n) {
  if (!s) return falha(TQ_E_ARG, "null handle");
  std::vector<double> tmp(1024);
  int k = normasPcg(s->pcg, s->d, tmp.data(), 1024, s->s);
  if (k < 0) return falhaCuda(cudaGetLastError(), "reading the residual history");
  if (n) *n = k;
  if (out)
    for (int i = 0; i < k && i < cap; i++) out[i] = tmp[i];
  return TQ_OK;
}

int tq_sync(tq_sim* s) {
  if (!s) return falha(TQ_E_ARG, "null handle");
  CK(cudaStreamSynchronize(s->s));
  int r = erroPcg(s->pcg, s->s);  // a solve queued by tq_launch_graph that gave up
  if (r == TQ_E_TIMEOUT) return falha(r, "pressure solve: a bounded wait gave up");
  if (r) return falhaCuda(cudaGetLastError(), "pressure solve");
  return TQ_OK;
}

int tq_get_stream(tq_sim* s, void** stream) {
  if (!s || !stream) return falha(TQ_E_ARG, "null argument");
  *stream = (void*)s->s;
  return TQ_OK;
}

int tq_set_timing(tq_sim* s, int32_t on) {
  if (!s) return falha(TQ_E_ARG, "null handle");
  CK(cudaStreamSynchronize(s->s));
  s->timing = on != 0;
  perfilPcg(s->pcg, on >= 2);
  s->usados = 0;
  s->regSub.clear();
  s->regAr.clear();
  s->atual = nullptr;
  long long base = 0;
  CK(cudaMemcpy(&base, &s->d.esc->itersAcum, sizeof base, cudaMemcpyDeviceToHost));
  s->itersBase = base;
  return TQ_OK;
}

// Accumulated stage times since tq_set_timing (ms): [0..6] p2g+faces, flags+labels, surface,
// divergence+bubbles, pressure solve, gradient+extrapolation, g2p; [7] air relabels;
// [8] substeps timed; [9] pressure iterations in total; [10] relabels timed.
int tq_get_timing(tq_sim* s, double* ms, int32_t cap, int32_t* n) {
  if (!s) return falha(TQ_E_ARG, "null handle");
  double v[11] = {0};
  if (s->timing) {
    CK(cudaStreamSynchronize(s->s));
    auto dur = [&](int a, int b) -> double {
      float t = 0;
      if (a < 0 || b < 0 || cudaEventElapsedTime(&t, s->pool[a], s->pool[b]) != cudaSuccess) return 0.0;
      return t;
    };
    int completos = 0;
    for (auto& r : s->regSub) {
      if (r[7] < 0) continue;
      for (int i = 0; i < 7; i++) v[i] += dur(r[i], r[i + 1]);
      completos++;
    }
    for (auto& r : s->regAr) v[7] += dur(r[0], r[1]);
    v[8] = completos;
    long long acum = 0;
    CK(cudaMemcpy(&acum, &s->d.esc->itersAcum, sizeof acum, cudaMemcpyDeviceToHost));
    v[9] = (double)(acum - s->itersBase);
    v[10] = (double)s->regAr.size();
    cudaGetLastError();
  }
  if (n) *n = 11;
  if (ms)
    for (int i = 0; i < 11 && i < cap; i++) ms[i] = v[i];
  return TQ_OK;
}

int tq_get_phase_trace(tq_sim* s, uint64_t* out, int32_t cap, int32_t* n) {
  if (!s) return falha(TQ_E_ARG, "null handle");
  CK(cudaStreamSynchronize(s->s));
  std::vector<unsigned long long> tmp(cap > 0 ? cap : -cap);
  int k = cap != 0 ? lerPerfilPcg(s->pcg, tmp.data(), cap) : 0;
  if (n) *n = k;
  if (out)
    for (int i = 0; i < k; i++) out[i] = tmp[i];
  return TQ_OK;
}

// ---------------------------------------------------------------- standalone solver
int tq_solve_pressure(int32_t nx, int32_t ny, const uint8_t* tipo, const float* div, float* q, int32_t iterations,
                      double tolerance, const tq_bubbles* b, int32_t precision, int32_t engine, int32_t precond,
                      double* norms, int32_t norms_cap, int32_t* n_norms, tq_solve_info* info) {
  if (nx < 3 || ny < 3 || !tipo || !div || !q || iterations < 1 || iterations > 1000)
    return falha(TQ_E_ARG, "bad arguments");
  if (b && (!b->rotulo || !b->rhs || !b->y)) return falha(TQ_E_ARG, "bad bubbles");
  tq_options o;
  tq_options_default(&o, nx, ny, 1.0);
  o.precision = precision;
  o.engine = engine;
  o.capacity = 1;
  o.iterations = iterations;
  o.tolerance = tolerance;
  o.preconditioner = precond;
  tq_sim* s = nullptr;
  int st = tq_create(&o, &s);
  if (st) return st;
  const size_t N = (size_t)nx * ny;
  const Dev& d = s->d;
  auto fim = [&](int r) {
    tq_destroy(s);
    return r;
  };
  if (cudaMemcpyAsync(d.tipo, tipo, N, cudaMemcpyHostToDevice, s->s) != cudaSuccess ||
      cudaMemcpyAsync(d.div, div, N * 4, cudaMemcpyHostToDevice, s->s) != cudaSuccess ||
      cudaMemcpyAsync(d.q, q, N * 4, cudaMemcpyHostToDevice, s->s) != cudaSuccess)
    return fim(falha(TQ_E_CUDA, "upload failed"));
  if (b) {
    if (cudaMemcpyAsync(d.rotulo, b->rotulo, N * 4, cudaMemcpyHostToDevice, s->s) != cudaSuccess ||
        cudaMemcpyAsync(d.rhsBolhaF, b->rhs, MAX_BOLHAS * 4, cudaMemcpyHostToDevice, s->s) != cudaSuccess ||
        cudaMemcpyAsync(d.yBolhaF, b->y, MAX_BOLHAS * 4, cudaMemcpyHostToDevice, s->s) != cudaSuccess)
      return fim(falha(TQ_E_CUDA, "upload failed"));
  }
  st = resolverPressao(s->pcg, d, iterations, tolerance, b != nullptr, precond, s->s);
  if (st) return fim(st == TQ_E_CUDA ? falha(st, "pressure solve failed") : st);
  st = erroPcg(s->pcg, s->s);
  if (st) return fim(st == TQ_E_TIMEOUT ? falha(st, "pressure solve: a grid barrier wait gave up") : st);
  if (cudaMemcpyAsync(q, d.q, N * 4, cudaMemcpyDeviceToHost, s->s) != cudaSuccess)
    return fim(falha(TQ_E_CUDA, "download failed"));
  if (b && cudaMemcpyAsync(b->y, d.yBolhaF, MAX_BOLHAS * 4, cudaMemcpyDeviceToHost, s->s) != cudaSuccess)
    return fim(falha(TQ_E_CUDA, "download failed"));
  if (cudaStreamSynchronize(s->s) != cudaSuccess) return fim(falha(TQ_E_CUDA, "solve failed"));
  std::vector<double> tmp(1024);
  int k = normasPcg(s->pcg, s->d, tmp.data(), 1024, s->s);
  if (k < 0) return fim(falha(TQ_E_CUDA, "reading the residual history"));
  if (n_norms) *n_norms = k;
  if (norms)
    for (int i = 0; i < k && i < norms_cap; i++) norms[i] = tmp[i];
  if (info) {
    Escalares e;
    if (cudaMemcpy(&e, s->d.esc, offsetof(Escalares, normas), cudaMemcpyDeviceToHost) != cudaSuccess)
      return fim(falha(TQ_E_CUDA, "reading the solve record"));
    info->iterations = e.iters;
    info->converged = e.convergiu;
    info->replacements = e.trocas;
    info->closed_regions = tolerance > 0 ? e.regioes : 0;
    info->residual0 = e.norma0;
    info->residual = e.norma;
    info->true_residual = e.normaVerd;
  }
  return fim(TQ_OK);
}

int tq_vcycle(int32_t nx, int32_t ny, const uint8_t* tipo, const float* b, float* x, int32_t precision) {
  if (nx < 3 || ny < 3 || !tipo || !b || !x) return falha(TQ_E_ARG, "bad arguments");
  int st = iniciarCuda(0);
  if (st) return st;
  if (precision < TQ_PREC_FP32 || precision > TQ_PREC_BF16) return falha(TQ_E_ARG, "bad precision");
  Pcg* p = criarPcg(nx, ny, precision, TQ_ENGINE_PLAIN);
  if (!p) return falha(TQ_E_NOMEM, "device allocation failed");
  const size_t N = (size_t)nx * ny;
  uint8_t* dt = nullptr;
  float *db = nullptr, *dx = nullptr;
  cudaStream_t s = nullptr;
  int r = TQ_OK;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess || cudaMalloc(&dt, N) != cudaSuccess ||
      cudaMalloc(&db, N * 4) != cudaSuccess || cudaMalloc(&dx, N * 4) != cudaSuccess)
    r = falha(TQ_E_NOMEM, "device allocation failed");
  if (!r && (cudaMemcpyAsync(dt, tipo, N, cudaMemcpyHostToDevice, s) != cudaSuccess ||
             cudaMemcpyAsync(db, b, N * 4, cudaMemcpyHostToDevice, s) != cudaSuccess))
    r = falha(TQ_E_CUDA, "upload failed");
  if (!r) r = cicloVDispositivo(p, dt, db, dx, s);
  if (!r && (cudaMemcpyAsync(x, dx, N * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
             cudaStreamSynchronize(s) != cudaSuccess))
    r = falha(TQ_E_CUDA, "V-cycle failed");
  cudaFree(dt);
  cudaFree(db);
  cudaFree(dx);
  if (s) cudaStreamDestroy(s);
  destruirPcg(p);
  return r;
}

int tq_vcycle_noalloc(int32_t nx, int32_t ny, const uint8_t* tipo, const float* b, float* x, int32_t precision,
                      void* stream) {
  if (nx < 3 || ny < 3 || !tipo || !b || !x) return falha(TQ_E_ARG, "tq_vcycle_noalloc: bad arguments");
  if (precision < TQ_PREC_FP32 || precision > TQ_PREC_BF16) return falha(TQ_E_ARG, "tq_vcycle_noalloc: bad precision");
  // sizes far beyond any scratch are refused before the level arithmetic sees them
  if (nx > (1 << 20) || ny > (1 << 20) || (long long)nx * ny > (1LL << 28))
    return falha(TQ_E_CAPACITY, "tq_vcycle_noalloc: grid larger than 2^20 cells a side or 2^28 cells");
  const size_t preciso = bytesScratchVCiclo(nx, ny);
  if (preciso > BYTES_SCRATCH_VCICLO) {
    std::snprintf(g_erro, sizeof g_erro,
                  "tq_vcycle_noalloc: a %dx%d grid needs %zu bytes of scratch for its levels; the static scratch "
                  "holds %zu bytes",
                  nx, ny, preciso, BYTES_SCRATCH_VCICLO);
    return TQ_E_CAPACITY;
  }
  void* scratch = nullptr;
  int st = enderecoScratchVCiclo(&scratch);
  if (st == TQ_E_NODEV) return falha(st, "tq_vcycle_noalloc: no current CUDA device");
  if (st) return falha(st, "tq_vcycle_noalloc: cudaGetSymbolAddress of the scratch failed");
  // an error left by earlier, unrelated work on this thread is reported as such (and cleared),
  // not as a failure of this call's launches
  cudaError_t antes = cudaGetLastError();
  if (antes != cudaSuccess) {
    std::snprintf(g_erro, sizeof g_erro, "tq_vcycle_noalloc: a CUDA error was pending before the call: %s",
                  cudaGetErrorString(antes));
    return TQ_E_CUDA;
  }
  st = cicloVSemAlocar(scratch, nx, ny, tipo, b, x, precision, (cudaStream_t)stream);
  if (st) return falha(st, "tq_vcycle_noalloc: V-cycle launch failed");
  return TQ_OK;
}

}  // extern "C"
