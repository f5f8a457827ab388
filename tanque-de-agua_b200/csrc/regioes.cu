// regioes.cu — the closed regions of a pressure solve and the consistency projection of its
// right-hand side (tolerance mode; no counterpart in the reference).
//
// The unknowns of resolverPCG (js/pressao-cpu.js:296-402) are the water cells and one pressure
// per active bubble.  A 4-connected set of them that touches no Dirichlet cell (air outside an
// active bubble, whose pressure is 0) is a closed region: water sealed by walls, with or
// without enclosed air.  On it A is the Neumann Laplacian, singular, its null vector the
// constant over the region's water cells and bubble pressures; b has a component along that
// vector (the density correction of compressed water, a bubble's volume recovery: neither can
// act in a sealed box), which no iterate can remove.  The reference runs a fixed count of
// iterations and returns what it reaches; a solve that stops on ||b - A q|| <= tol ||r0||
// could never stop, and CG's iterate drifts along the null vector.  So in tolerance mode each
// closed region's right-hand side loses its mean over the region's unknowns,
//   b_R <- b_R - (sum_R b / n_R) 1,   n_R = water cells + active bubbles of R,
// which makes the system consistent without touching any open region.  A consistent singular
// system still leaves the preconditioner singular there (the V-cycle sees the same sealed
// region), and CG's scalars then take the rounding of a huge null-space component; so each
// closed region's root cell is also pinned: the solve sees it as air at pressure 0 (q = 0
// there), which makes the region's block nonsingular and fixes its constant.  With the
// projected right-hand side the pinned row's equation holds by itself (the rows of a closed
// region sum to 0), so the solution is the projected system's with q = 0 at the root.  A root
// carrying a bubble label (only possible with caller-provided labels) is not pinned.  The
// solve reads the projected and pinned copies (Regioes::div, ::rhs, ::tipo); the handle's own
// fields stay as computed.
//
// Labels: union-find over the water cells and one node per bubble (index N + label), water
// joined to its water neighbours and to the bubble node of each active bubble it faces; a
// component's root is its smallest index, always a water cell.
#include "common.cuh"
#include "kernels.cuh"
#include "uniao.cuh"

namespace tq {

constexpr int MAX_REGIOES = 4096;  // closed regions projected per solve (more: the rest as they are)

struct Regioes {
  int N = 0;
  int* pai = nullptr;        // N + MAX_BOLHAS
  int* idR = nullptr;        // N: per root, its closed-region index or -1
  uint8_t* toca = nullptr;   // N: the water cell faces a Dirichlet cell / the root's region is open
  uint8_t* aberto = nullptr; // N
  uint8_t* ativa = nullptr;  // MAX_BOLHAS: the bubble has a water face
  double* soma = nullptr;    // MAX_REGIOES
  int* cont = nullptr;       // MAX_REGIOES + 3: counts, the region count, this solve's and the sticky error flag
  float* div = nullptr;      // N: the projected -b on water
  float* rhs = nullptr;      // MAX_BOLHAS: the projected bubble right-hand sides
  uint8_t* tipo = nullptr;   // N: the solve's cell types, closed regions' roots pinned as air
};

namespace {

__global__ void k_reg_iniciar(Regioes R, const uint8_t* tipo) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < R.N) {
    R.pai[c] = tipo[c] == AGUA ? c : -1;
    R.toca[c] = 0;
    R.aberto[c] = 0;
  }
  if (c < MAX_BOLHAS) {
    R.pai[R.N + c] = R.N + c;
    R.ativa[c] = 0;
  }
  if (c < MAX_REGIOES) {
    R.soma[c] = 0.0;
    R.cont[c] = 0;
  }
  if (c < 2) R.cont[MAX_REGIOES + c] = 0;
}

// Active bubbles as k_bolhas_faces counts them: an interior air cell of the label with a water
// neighbour.
__global__ void k_reg_bolhas(Regioes R, Dev d) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N) return;
  const int nx = d.nx, i = c % nx, j = c / nx;
  if (i < 1 || j < 1 || i >= nx - 1 || j >= d.ny - 1 || d.tipo[c] != AR) return;
  const uint32_t b = d.rotulo[c];
  if (b < 2 || b >= (uint32_t)MAX_BOLHAS) return;
  if (d.tipo[c - 1] == AGUA || d.tipo[c + 1] == AGUA || d.tipo[c - nx] == AGUA || d.tipo[c + nx] == AGUA)
    R.ativa[b] = 1;
}

// Water joins its water neighbours (left and down; the others join it) and the bubble node of
// each active bubble it faces; any other air neighbour is Dirichlet (valorViz's 0).
__global__ void k_reg_unir(Regioes R, Dev d, int bolhas) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N || d.tipo[c] != AGUA) return;
  const int nx = d.nx, i = c % nx, j = c / nx;
  const int nb[4] = {c - 1, c + 1, c - nx, c + nx};
  const bool dentro[4] = {i > 0, i < nx - 1, j > 0, j < d.ny - 1};
  bool ok = true, toca = false;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    if (!dentro[q]) continue;
    const uint8_t t = d.tipo[nb[q]];
    if (t == AGUA) {
      if (q == 0 || q == 2) ok &= unir(R.pai, c, nb[q]);
    } else if (t == AR) {
      const uint32_t b = d.rotulo[nb[q]];
      if (bolhas && b >= 2 && b < (uint32_t)MAX_BOLHAS && R.ativa[b]) ok &= unir(R.pai, c, R.N + (int)b);
      else toca = true;
    }
  }
  if (toca) R.toca[c] = 1;
  if (!ok) R.cont[MAX_REGIOES + 1] = 1;
}

__global__ void k_reg_achatar(Regioes R) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= R.N + MAX_BOLHAS || R.pai[c] < 0) return;
  R.pai[c] = raizLeitura(R.pai, c);
}

__global__ void k_reg_abrir(Regioes R) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= R.N || !R.toca[c]) return;
  R.aberto[R.pai[c]] = 1;
}

__global__ void k_reg_ids(Regioes R) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= R.N || R.pai[c] != c) return;  // roots only (water cells)
  int id = -1;
  if (!R.aberto[c]) {
    id = atomicAdd(&R.cont[MAX_REGIOES], 1);
    if (id >= MAX_REGIOES) id = -1;
  }
  R.idR[c] = id;
}

// The closed-region index of a node (water cell or bubble node), -1 when open or uncounted; a
// bubble node left alone (no water joined it) has no region.
__device__ inline int regiaoDe(const Regioes& R, int no) {
  const int r = R.pai[no];
  return r >= 0 && r < R.N ? R.idR[r] : -1;
}

__global__ void k_reg_somar(Regioes R, Dev d, int bolhas) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < R.N && d.tipo[c] == AGUA) {
    const int id = regiaoDe(R, c);
    if (id >= 0) {
      atomicAdd(&R.soma[id], -(double)d.div[c]);
      atomicAdd(&R.cont[id], 1);
    }
  }
  if (bolhas && c >= 2 && c < MAX_BOLHAS && R.ativa[c]) {
    const int id = regiaoDe(R, R.N + c);
    if (id >= 0) {
      atomicAdd(&R.soma[id], (double)d.rhsBolhaF[c]);
      atomicAdd(&R.cont[id], 1);
    }
  }
}

__global__ void k_reg_projetar(Regioes R, Dev d, int bolhas) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  auto media = [&](int id) { return R.soma[id] / (double)R.cont[id]; };
  if (c < R.N) {
    float v = d.div[c];
    uint8_t t = d.tipo[c];
    if (t == AGUA) {
      const int id = regiaoDe(R, c);
      if (id >= 0) {
        v = (float)((double)v + media(id));
        if (R.pai[c] == c && (!bolhas || d.rotulo[c] < 2)) t = AR;  // the pinned root
      }
    }
    R.div[c] = v;
    R.tipo[c] = t;
  }
  if (c < MAX_BOLHAS) {
    float v = d.rhsBolhaF[c];
    if (bolhas && c >= 2 && R.ativa[c]) {
      const int id = regiaoDe(R, R.N + c);
      if (id >= 0) v = (float)((double)v - media(id));
    }
    R.rhs[c] = v;
  }
  if (c == 0) {
    const int n = R.cont[MAX_REGIOES];
    d.esc->regioes = n < MAX_REGIOES ? n : MAX_REGIOES;
    if (R.cont[MAX_REGIOES + 1]) R.cont[MAX_REGIOES + 2] = 1;  // sticky until erroRegioes reads it
  }
}

}  // namespace

Regioes* criarRegioes(int N) {
  Regioes* R = new Regioes();
  R->N = N;
  const size_t n = (size_t)N;
  bool ok = cudaMalloc(&R->pai, (n + MAX_BOLHAS) * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&R->idR, n * sizeof(int)) == cudaSuccess && cudaMalloc(&R->toca, n) == cudaSuccess &&
            cudaMalloc(&R->aberto, n) == cudaSuccess && cudaMalloc(&R->ativa, MAX_BOLHAS) == cudaSuccess &&
            cudaMalloc(&R->soma, MAX_REGIOES * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&R->cont, (MAX_REGIOES + 3) * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&R->div, n * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&R->rhs, MAX_BOLHAS * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&R->tipo, n) == cudaSuccess;
  if (ok) ok = cudaMemset(R->cont + MAX_REGIOES + 2, 0, sizeof(int)) == cudaSuccess;
  if (!ok) {
    destruirRegioes(R);
    return nullptr;
  }
  return R;
}

// TQ_E_TIMEOUT when a labelling since the last call gave up on its bounded union loop (the
// flag is cleared), else TQ_OK.  Waits for the stream.
int erroRegioes(Regioes* R, cudaStream_t s) {
  if (!R) return TQ_OK;
  int h = 0;
  if (cudaMemcpyAsync(&h, R->cont + MAX_REGIOES + 2, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return TQ_E_CUDA;
  if (!h) return TQ_OK;
  if (cudaMemsetAsync(R->cont + MAX_REGIOES + 2, 0, sizeof(int), s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return TQ_E_CUDA;
  return TQ_E_TIMEOUT;
}

void destruirRegioes(Regioes* R) {
  if (!R) return;
  cudaFree(R->pai);
  cudaFree(R->idR);
  cudaFree(R->toca);
  cudaFree(R->aberto);
  cudaFree(R->ativa);
  cudaFree(R->soma);
  cudaFree(R->cont);
  cudaFree(R->div);
  cudaFree(R->rhs);
  cudaFree(R->tipo);
  delete R;
}

// Queues the labelling and the projection on s; *out gets d with div, rhsBolhaF and tipo
// pointing at the projected and pinned copies.  Nothing waits for the device.
void projetarFechadas(Regioes* R, const Dev& d, bool bolhas, cudaStream_t s, Dev* out) {
  const int N = d.N;
  const int nb = blocos(N, 256), nbMax = blocos(N > MAX_BOLHAS ? N : MAX_BOLHAS, 256);
  lanca(k_reg_iniciar, nbMax, 256, 0, s, *R, (const uint8_t*)d.tipo);
  if (bolhas) lanca(k_reg_bolhas, nb, 256, 0, s, *R, d);
  lanca(k_reg_unir, nb, 256, 0, s, *R, d, bolhas ? 1 : 0);
  lanca(k_reg_achatar, blocos((long)N + MAX_BOLHAS, 256), 256, 0, s, *R);
  lanca(k_reg_abrir, nb, 256, 0, s, *R);
  lanca(k_reg_ids, nb, 256, 0, s, *R);
  lanca(k_reg_somar, nbMax, 256, 0, s, *R, d, bolhas ? 1 : 0);
  lanca(k_reg_projetar, nbMax, 256, 0, s, *R, d, bolhas ? 1 : 0);
  *out = d;
  out->div = R->div;
  out->rhsBolhaF = R->rhs;
  out->tipo = R->tipo;
}

}  // namespace tq
