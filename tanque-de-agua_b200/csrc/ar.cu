// ar.cu — RastreadorDeAr.atualizar (js/ar.js:56-153) on the device: enclosed-air pockets
// (4-connected air components), atmosphere test, bubble ids stable through overlap with the
// previous frame, target volume split/merged by overlap, births with the lowest free id.
//
// The reference is sequential and order-dependent; every order-dependent rule is restated
// with an order-independent construction that yields the same labels bit for bit:
//   component index k   = rank of the component's smallest cell (union-find that always
//                         links the larger root under the smaller makes that cell the root);
//   gas Map order       = pairs (component, old label) sorted by the pair's first cell;
//   ordem (stable sort) = sort by (novoAlvo descending, k ascending);
//   owners              = for each old label, the earliest position in ordem claiming it;
//   births              = j-th unlabelled component of ordem gets the j-th free id.
// Built with -fmad=false: the target-volume sums are the reference's double arithmetic.
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "uniao.cuh"

namespace tq {

constexpr unsigned long long VAZIO = ~0ull;

struct Rastreador {
  int nx, ny, N;
  int primeira = 1;
  int Hc;  // hash capacity (power of two)
  int* pai;
  uint32_t *cnt, *atm;
  uint8_t* topo;
  int* compIdx;
  unsigned long long* hk;
  uint32_t* hcnt;
  int* hfirst;
  // per component (capacity N)
  uint32_t *celK, *atmK, *rotK;
  uint8_t* topoK;
  float* novoAlvo;
  int *dono, *gasCount, *gasOff;
  // pairs and order (capacity N)
  unsigned long long *parKey, *parVal, *ordKey;
  // per label
  int* ganhador;
  uint8_t* vivoNovo;
  int* livres;
  float* pNova;
  uint32_t* sob;
  int* nasceu;
  // counters: 0 K, 1 P, 2 M, 3 nLivres, 4 error
  int* cont;
  int *blocoCont, *blocoOff;
  int nBlocos;
};

// ---------------------------------------------------------------- union-find (uniao.cuh)
__global__ void k_ar_iniciar(Rastreador r, const uint8_t* tipo) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= r.N) return;
  r.pai[c] = tipo[c] == AR ? c : -1;
  r.cnt[c] = 0;
  r.atm[c] = 0;
  r.topo[c] = 0;
}
// js/ar.js:61-69
__global__ void k_ar_unir(Rastreador r, const uint8_t* tipo) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= r.N || tipo[c] != AR) return;
  int i = c % r.nx, j = c / r.nx;
  bool ok = true;
  if (i > 0 && tipo[c - 1] == AR) ok &= unir(r.pai, c, c - 1);
  if (j > 0 && tipo[c - r.nx] == AR) ok &= unir(r.pai, c, c - r.nx);
  if (!ok) atomicExch(&r.cont[4], 1);
}
// Every cell points straight at its root afterwards.  The walk only reads: a path-halving
// write here could replace a root some other thread has just stored with a non-root
// ancestor.  The only writes of this kernel store roots, so concurrent walks stay valid.
__global__ void k_ar_achatar(Rastreador r) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= r.N || r.pai[c] < 0) return;
  r.pai[c] = raizLeitura(r.pai, c);
}

// Per-cell statistics of js/ar.js:75-95, gathered at the component's root: cells, touches the
// top band, cells that were atmosphere, and per old bubble label the cells and the first cell.
__device__ inline unsigned hashChave(unsigned long long k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  return (unsigned)k;
}
__global__ void k_ar_estatisticas(Rastreador r, const uint32_t* rotulo) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= r.N) return;
  int rt = r.pai[c];
  if (rt < 0) return;
  atomicAdd(&r.cnt[rt], 1u);
  int topoLinha = r.ny - MOLDURA - 1;
  if (c / r.nx >= topoLinha) r.topo[rt] = 1;
  uint32_t antigo = rotulo[c];
  if (antigo == 1) atomicAdd(&r.atm[rt], 1u);
  else if (antigo >= 2) {
    unsigned long long chave = ((unsigned long long)(unsigned)rt << 32) | antigo;
    unsigned h = hashChave(chave) & (unsigned)(r.Hc - 1);
    for (int t = 0; t < r.Hc; t++) {
      unsigned long long prev = atomicCAS(&r.hk[h], VAZIO, chave);
      if (prev == VAZIO || prev == chave) {
        atomicAdd(&r.hcnt[h], 1u);
        atomicMin(&r.hfirst[h], c);
        return;
      }
      h = (h + 1) & (unsigned)(r.Hc - 1);
    }
    atomicExch(&r.cont[4], 2);
  }
}

// ---------------------------------------------------------------- scans
__device__ int rankBloco1024(bool keep, int* total) {
  __shared__ int somas[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned m = __ballot_sync(0xffffffffu, keep);
  int rank = __popc(m & ((1u << lane) - 1u));
  __syncthreads();
  if (lane == 0) somas[w] = __popc(m);
  __syncthreads();
  const int nw = (int)(blockDim.x >> 5);
  if (w == 0) {
    int v = lane < nw ? somas[lane] : 0;  // slots of absent warps were never written
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += t;
    }
    somas[lane] = v;
  }
  __syncthreads();
  int base = w ? somas[w - 1] : 0;
  *total = somas[nw - 1];
  return base + rank;
}
__device__ int scanBlocoUnico(const int* cont, int* offs, int n) {
  __shared__ int carry;
  __shared__ int s[1024];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += 1024) {
    int i = base + threadIdx.x;
    int v = i < n ? cont[i] : 0;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
      int t = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0;
      __syncthreads();
      s[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < n) offs[i] = carry + s[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += s[1023];
    __syncthreads();
  }
  return carry;
}

// Component index k = rank of the root among all roots in raster order (js/ar.js:75-85).
__global__ void k_ar_raizes_contar(Rastreador r) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  bool raizc = c < r.N && r.pai[c] == c;
  int t;
  rankBloco1024(raizc, &t);
  if (threadIdx.x == 0) r.blocoCont[blockIdx.x] = t;
}
__global__ void k_ar_raizes_scan(Rastreador r) {
  int total = scanBlocoUnico(r.blocoCont, r.blocoOff, r.nBlocos);
  if (threadIdx.x == 0) r.cont[0] = total;
}
__global__ void k_ar_raizes_gravar(Rastreador r) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  bool raizc = c < r.N && r.pai[c] == c;
  int t;
  int rank = rankBloco1024(raizc, &t);
  if (!raizc) return;
  int k = r.blocoOff[blockIdx.x] + rank;
  r.compIdx[c] = k;
  r.celK[k] = r.cnt[c];
  r.atmK[k] = r.atm[c];
  r.topoK[k] = r.topo[c];
  r.gasCount[k] = 0;
  r.rotK[k] = 0;
  r.dono[k] = -1;
  r.novoAlvo[k] = 0.0f;
}

// Occupied hash slots -> pair list keyed (k, first cell); value (label, cells).
__global__ void k_ar_pares(Rastreador r) {
  int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= r.Hc) return;
  unsigned long long chave = r.hk[h];
  if (chave == VAZIO) return;
  int rt = (int)(chave >> 32);
  uint32_t rotulo = (uint32_t)(chave & 0xffffffffu);
  int k = r.compIdx[rt];
  int slot = atomicAdd(&r.cont[1], 1);
  r.parKey[slot] = ((unsigned long long)(unsigned)k << 32) | (unsigned)r.hfirst[h];
  r.parVal[slot] = ((unsigned long long)rotulo << 32) | r.hcnt[h];
  atomicAdd(&r.gasCount[k], 1);
}

// ---------------------------------------------------------------- sorting
// Ascending sort of (key, value) pairs: one CTA bitonic network in shared memory up to 2048
// elements, the same network over global memory beyond that.
__global__ void k_bitonic_local(unsigned long long* key, unsigned long long* val, int n) {
  __shared__ unsigned long long sk[2048];
  __shared__ unsigned long long sv[2048];
  int m = 1;
  while (m < n) m <<= 1;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    sk[i] = i < n ? key[i] : VAZIO;
    sv[i] = i < n ? (val ? val[i] : 0ull) : 0ull;
  }
  __syncthreads();
  for (int kk = 2; kk <= m; kk <<= 1)
    for (int j = kk >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < m; i += blockDim.x) {
        int l = i ^ j;
        if (l > i) {
          bool asc = (i & kk) == 0;
          unsigned long long a = sk[i], b = sk[l];
          if ((a > b) == asc) {
            sk[i] = b;
            sk[l] = a;
            unsigned long long t = sv[i];
            sv[i] = sv[l];
            sv[l] = t;
          }
        }
      }
      __syncthreads();
    }
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    key[i] = sk[i];
    if (val) val[i] = sv[i];
  }
}
__global__ void k_bitonic_passo(unsigned long long* key, unsigned long long* val, int m, int kk, int j) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  int l = i ^ j;
  if (l <= i) return;
  bool asc = (i & kk) == 0;
  unsigned long long a = key[i], b = key[l];
  if ((a > b) == asc) {
    key[i] = b;
    key[l] = a;
    if (val) {
      unsigned long long t = val[i];
      val[i] = val[l];
      val[l] = t;
    }
  }
}
__global__ void k_preencher(unsigned long long* key, unsigned long long* val, int n, int m) {
  int i = n + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  key[i] = VAZIO;
  if (val) val[i] = 0;
}
// `key`/`val` must hold the next power of two >= n entries for n > 2048.
static void ordenar(unsigned long long* key, unsigned long long* val, int n, cudaStream_t s) {
  if (n <= 1) return;
  if (n <= 2048) {
    lanca(k_bitonic_local, 1, 1024, 0, s, key, val, n);
    return;
  }
  int m = 1;
  while (m < n) m <<= 1;
  lanca(k_preencher, blocos(m - n, 256), 256, 0, s, key, val, n, m);
  for (int kk = 2; kk <= m; kk <<= 1)
    for (int j = kk >> 1; j > 0; j >>= 1) lanca(k_bitonic_passo, blocos(m, 256), 256, 0, s, key, val, m, kk, j);
}

// ---------------------------------------------------------------- canonicalisation
__global__ void k_ar_gas_scan(Rastreador r) {
  int total = scanBlocoUnico(r.gasCount, r.gasOff, r.cont[0]);
  (void)total;
}

__device__ inline bool fica(const Rastreador& r, int k) { return r.topoK[k] || r.celK[k] >= (uint32_t)MIN_BOLHA_CELULAS; }

// sobreposicaoTotal (js/ar.js:102-106): cells of each old label inside components that stay.
__global__ void k_ar_sobreposicao(Rastreador r) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r.cont[1]) return;
  int k = (int)(r.parKey[i] >> 32);
  if (!fica(r, k)) return;
  uint32_t rotulo = (uint32_t)(r.parVal[i] >> 32);
  uint32_t q = (uint32_t)(r.parVal[i] & 0xffffffffu);
  if (rotulo < (uint32_t)MAX_BOLHAS) atomicAdd(&r.sob[rotulo], q);
}

// novoAlvo and dono (js/ar.js:108-125), the gas Map walked in insertion order.
__global__ void k_ar_alvo(Rastreador r, const float* volumeAlvo) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= r.cont[0]) return;
  if (!fica(r, k) || r.topoK[k]) return;
  double v = 0;
  int melhor = 0, dono = -1;
  if (r.primeira) v = r.celK[k];
  else {
    v = r.atmK[k];
    int o = r.gasOff[k], n = r.gasCount[k];
    for (int t = 0; t < n; t++) {
      uint32_t rotulo = (uint32_t)(r.parVal[o + t] >> 32);
      int q = (int)(r.parVal[o + t] & 0xffffffffu);
      double alvo = rotulo < (uint32_t)MAX_BOLHAS ? (double)volumeAlvo[rotulo] : nan("");
      double sob = rotulo < (uint32_t)MAX_BOLHAS ? (double)r.sob[rotulo] : 0.0;
      v += alvo * (q / sob);
      if (q > melhor) { melhor = q; dono = (int)rotulo; }
    }
  }
  r.novoAlvo[k] = (float)v;
  r.dono[k] = dono;
}

// ordem (js/ar.js:129-130): closed components of >= 4 target cells, by target descending,
// ties by component index.  Key: (~bits(novoAlvo)) << 32 | k.
__global__ void k_ar_ordem(Rastreador r) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= r.cont[0]) return;
  if (r.topoK[k] || !(r.novoAlvo[k] >= (float)MIN_BOLHA_CELULAS)) return;
  unsigned bits = __float_as_uint(r.novoAlvo[k]);
  int slot = atomicAdd(&r.cont[2], 1);
  r.ordKey[slot] = ((unsigned long long)(~bits) << 32) | (unsigned)k;
}

// Owners (js/ar.js:131-134): each old label goes to the earliest component in ordem it owns.
__global__ void k_ar_donos_marcar(Rastreador r) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r.cont[2]) return;
  int k = (int)(r.ordKey[i] & 0xffffffffu);
  int d = r.dono[k];
  if (d >= 2 && d < MAX_BOLHAS) atomicMin(&r.ganhador[d], i);
}
__global__ void k_ar_donos_gravar(Rastreador r) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r.cont[2]) return;
  int k = (int)(r.ordKey[i] & 0xffffffffu);
  int d = r.dono[k];
  if (d >= 2 && d < MAX_BOLHAS && r.ganhador[d] == i) {
    r.rotK[k] = (uint32_t)d;
    r.vivoNovo[d] = 1;
  }
}

// Free ids (js/ar.js:137-139): labels >= 2 alive neither now nor in the previous frame, in order.
__global__ void k_ar_livres(Rastreador r, const uint8_t* vivo) {
  int total = 0;
  // one 1024-thread block; ids 2..4095 in 4 chunks
  for (int base = 0; base < MAX_BOLHAS; base += 1024) {
    int id = base + threadIdx.x;
    bool livre = id >= 2 && !r.vivoNovo[id] && !vivo[id];
    int t;
    int rank = rankBloco1024(livre, &t);
    if (livre) r.livres[total + rank] = id;
    total += t;
    __syncthreads();
  }
  if (threadIdx.x == 0) r.cont[3] = total;
}

// Births (js/ar.js:135-144): the j-th component of ordem still without a label gets the j-th
// free id; once the ids run out the rest stay unlabelled (vacuum).  The initial pressure is
// the owner's previous pressure, written after every read (pNova -> pressaoBolha).
__global__ void k_ar_nascer_contar(Rastreador r) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool sem = false;
  if (i < r.cont[2]) {
    int k = (int)(r.ordKey[i] & 0xffffffffu);
    sem = r.rotK[k] == 0;
  }
  int t;
  rankBloco1024(sem, &t);
  if (threadIdx.x == 0) r.blocoCont[blockIdx.x] = t;
}
__global__ void k_ar_nascer_scan(Rastreador r, int nb) { scanBlocoUnico(r.blocoCont, r.blocoOff, nb); }
__global__ void k_ar_nascer(Rastreador r, const float* pressaoBolha) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool sem = false;
  int k = 0;
  if (i < r.cont[2]) {
    k = (int)(r.ordKey[i] & 0xffffffffu);
    sem = r.rotK[k] == 0;
  }
  int t;
  int rank = rankBloco1024(sem, &t);
  if (!sem) return;
  int j = r.blocoOff[blockIdx.x] + rank;
  if (j >= r.cont[3]) return;
  int id = r.livres[j];
  r.rotK[k] = (uint32_t)id;
  r.vivoNovo[id] = 1;
  int d = r.dono[k];
  r.pNova[id] = d >= 2 && d < MAX_BOLHAS ? pressaoBolha[d] : 0.0f;
  r.nasceu[id] = 1;
}
__global__ void k_ar_aplicar_bolhas(Rastreador r, float* pressaoBolha, float* volumeAlvo, uint8_t* vivo) {
  int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= MAX_BOLHAS) return;
  if (r.nasceu[id]) pressaoBolha[id] = r.pNova[id];
  vivo[id] = r.vivoNovo[id];
  volumeAlvo[id] = 0.0f;
}
// Atmosphere label, target volumes, final per-cell labels (js/ar.js:145-150).
__global__ void k_ar_volumes(Rastreador r, float* volumeAlvo) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= r.cont[0]) return;
  if (r.topoK[k]) {
    r.rotK[k] = 1;
    return;
  }
  uint32_t l = r.rotK[k];
  if (l >= 2) volumeAlvo[l] = r.novoAlvo[k];
}
__global__ void k_ar_rotular(Rastreador r, uint32_t* rotulo) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= r.N) return;
  int rt = r.pai[c];
  rotulo[c] = rt >= 0 ? r.rotK[r.compIdx[rt]] : 0u;
}

// ---------------------------------------------------------------- host side
Rastreador* criarRastreador(int nx, int ny) {
  Rastreador* r = new Rastreador();
  r->nx = nx;
  r->ny = ny;
  r->N = nx * ny;
  int hc = 1024;
  while (hc < 2 * r->N) hc <<= 1;
  r->Hc = hc;
  int N = r->N;
  int cap = 1;
  while (cap < N) cap <<= 1;  // power of two for the global sort
  r->nBlocos = blocos(N, 1024);
  bool ok = true;
  ok &= cudaMalloc(&r->pai, N * sizeof(int)) == cudaSuccess;
  ok &= cudaMalloc(&r->cnt, N * sizeof(uint32_t)) == cudaSuccess;
  ok &= cudaMalloc(&r->atm, N * sizeof(uint32_t)) == cudaSuccess;
  ok &= cudaMalloc(&r->topo, N) == cudaSuccess;
  ok &= cudaMalloc(&r->compIdx, N * sizeof(int)) == cudaSuccess;
  ok &= cudaMalloc(&r->hk, (size_t)hc * 8) == cudaSuccess;
  ok &= cudaMalloc(&r->hcnt, (size_t)hc * 4) == cudaSuccess;
  ok &= cudaMalloc(&r->hfirst, (size_t)hc * 4) == cudaSuccess;
  ok &= cudaMalloc(&r->celK, N * 4) == cudaSuccess;
  ok &= cudaMalloc(&r->atmK, N * 4) == cudaSuccess;
  ok &= cudaMalloc(&r->rotK, N * 4) == cudaSuccess;
  ok &= cudaMalloc(&r->topoK, N) == cudaSuccess;
  ok &= cudaMalloc(&r->novoAlvo, N * 4) == cudaSuccess;
  ok &= cudaMalloc(&r->dono, N * 4) == cudaSuccess;
  ok &= cudaMalloc(&r->gasCount, N * 4) == cudaSuccess;
  ok &= cudaMalloc(&r->gasOff, N * 4) == cudaSuccess;
  ok &= cudaMalloc(&r->parKey, (size_t)cap * 8) == cudaSuccess;
  ok &= cudaMalloc(&r->parVal, (size_t)cap * 8) == cudaSuccess;
  ok &= cudaMalloc(&r->ordKey, (size_t)cap * 8) == cudaSuccess;
  ok &= cudaMalloc(&r->ganhador, MAX_BOLHAS * 4) == cudaSuccess;
  ok &= cudaMalloc(&r->vivoNovo, MAX_BOLHAS) == cudaSuccess;
  ok &= cudaMalloc(&r->livres, MAX_BOLHAS * 4) == cudaSuccess;
  ok &= cudaMalloc(&r->pNova, MAX_BOLHAS * 4) == cudaSuccess;
  ok &= cudaMalloc(&r->sob, MAX_BOLHAS * 4) == cudaSuccess;
  ok &= cudaMalloc(&r->nasceu, MAX_BOLHAS * 4) == cudaSuccess;
  ok &= cudaMalloc(&r->cont, 8 * sizeof(int)) == cudaSuccess;
  ok &= cudaMalloc(&r->blocoCont, (r->nBlocos + 1) * sizeof(int)) == cudaSuccess;
  ok &= cudaMalloc(&r->blocoOff, (r->nBlocos + 1) * sizeof(int)) == cudaSuccess;
  if (!ok) {
    destruirRastreador(r);
    return nullptr;
  }
  return r;
}

void destruirRastreador(Rastreador* r) {
  if (!r) return;
  void* ps[] = {r->pai, r->cnt, r->atm, r->topo, r->compIdx, r->hk, r->hcnt, r->hfirst, r->celK, r->atmK,
                r->rotK, r->topoK, r->novoAlvo, r->dono, r->gasCount, r->gasOff, r->parKey, r->parVal,
                r->ordKey, r->ganhador, r->vivoNovo, r->livres, r->pNova, r->sob, r->nasceu, r->cont,
                r->blocoCont, r->blocoOff};
  for (void* p : ps) cudaFree(p);
  delete r;
}

// reiniciar (js/ar.js:37-42)
void reiniciarRastreador(Rastreador* r, const Dev& d, cudaStream_t s) {
  cudaMemsetAsync(d.rotulo, 0, (size_t)d.N * 4, s);
  cudaMemsetAsync(d.volumeAlvo, 0, MAX_BOLHAS * 4, s);
  cudaMemsetAsync(d.vivo, 0, MAX_BOLHAS, s);
  r->primeira = 1;
}
int primeiraRastreador(Rastreador* r) { return r->primeira; }
void definirPrimeiraRastreador(Rastreador* r, int v) { r->primeira = v ? 1 : 0; }

__global__ void k_preencher_int(int* p, int v, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

int atualizarRastreador(Rastreador* r, const Dev& d, cudaStream_t s) {
  const int N = r->N;
  const int nb = blocos(N, 256);
  Rastreador R = *r;
  cudaMemsetAsync(r->cont, 0, 8 * sizeof(int), s);
  cudaMemsetAsync(r->hk, 0xff, (size_t)r->Hc * 8, s);
  cudaMemsetAsync(r->hcnt, 0, (size_t)r->Hc * 4, s);
  lanca(k_preencher_int, blocos(r->Hc, 256), 256, 0, s, r->hfirst, 0x7fffffff, r->Hc);
  cudaMemsetAsync(r->sob, 0, MAX_BOLHAS * 4, s);
  cudaMemsetAsync(r->vivoNovo, 0, MAX_BOLHAS, s);
  cudaMemsetAsync(r->nasceu, 0, MAX_BOLHAS * 4, s);
  lanca(k_preencher_int, blocos(MAX_BOLHAS, 256), 256, 0, s, r->ganhador, 0x7fffffff, MAX_BOLHAS);
  lanca(k_ar_iniciar, nb, 256, 0, s, R, d.tipo);
  lanca(k_ar_unir, nb, 256, 0, s, R, d.tipo);
  lanca(k_ar_achatar, nb, 256, 0, s, R);
  lanca(k_ar_estatisticas, nb, 256, 0, s, R, d.rotulo);
  lanca(k_ar_raizes_contar, r->nBlocos, 1024, 0, s, R);
  lanca(k_ar_raizes_scan, 1, 1024, 0, s, R);
  lanca(k_ar_raizes_gravar, r->nBlocos, 1024, 0, s, R);
  lanca(k_ar_pares, blocos(r->Hc, 256), 256, 0, s, R);
  int h[8];
  if (cudaMemcpyAsync(h, r->cont, sizeof h, cudaMemcpyDeviceToHost, s) != cudaSuccess) return TQ_E_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return TQ_E_CUDA;
  if (h[4]) return TQ_E_TIMEOUT;
  const int K = h[0], P = h[1];
  ordenar(r->parKey, r->parVal, P, s);
  if (K > 0) {
    lanca(k_ar_gas_scan, 1, 1024, 0, s, R);
    lanca(k_ar_sobreposicao, blocos(P > 0 ? P : 1, 256), 256, 0, s, R);
    lanca(k_ar_alvo, blocos(K, 256), 256, 0, s, R, d.volumeAlvo);
    lanca(k_ar_ordem, blocos(K, 256), 256, 0, s, R);
  }
  if (cudaMemcpyAsync(h, r->cont, sizeof h, cudaMemcpyDeviceToHost, s) != cudaSuccess) return TQ_E_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return TQ_E_CUDA;
  const int M = h[2];
  ordenar(r->ordKey, nullptr, M, s);
  int nbM = blocos(M > 0 ? M : 1, 1024);
  if (M > 0) {
    lanca(k_ar_donos_marcar, blocos(M, 256), 256, 0, s, R);
    lanca(k_ar_donos_gravar, blocos(M, 256), 256, 0, s, R);
  }
  lanca(k_ar_livres, 1, 1024, 0, s, R, d.vivo);
  if (M > 0) {
    lanca(k_ar_nascer_contar, nbM, 1024, 0, s, R);
    lanca(k_ar_nascer_scan, 1, 1024, 0, s, R, nbM);
    lanca(k_ar_nascer, nbM, 1024, 0, s, R, d.pressaoBolha);
  }
  lanca(k_ar_aplicar_bolhas, blocos(MAX_BOLHAS, 256), 256, 0, s, R, d.pressaoBolha, d.volumeAlvo, d.vivo);
  if (K > 0) lanca(k_ar_volumes, blocos(K, 256), 256, 0, s, R, d.volumeAlvo);
  lanca(k_ar_rotular, nb, 256, 0, s, R, d.rotulo);
  r->primeira = 0;
  return cudaGetLastError() == cudaSuccess ? TQ_OK : TQ_E_CUDA;
}

}  // namespace tq
