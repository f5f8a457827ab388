// pcg.cu — MGPCG pressure projection: PCG with a multigrid V-cycle preconditioner, each
// enclosed air pocket one extra unknown ("supercell").  Restates js/pressao-cpu.js
// (resolverPCG :296-402, cicloV :241-255 and its parts) on the device.
//
// This file is the PLAIN engine: one launch per step of the algorithm, the iteration loop on
// the host.  The V-cycle vectors (b, x, tmp of every level) are stored as T = float, __half or
// __nv_bfloat16 (levels below 16k cells stay float); arithmetic is FP32; dot products and
// norms are FP64 with a fixed reduction order (bitwise reproducible); per-bubble sums are
// 64-bit fixed point.
#include <mutex>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "pcg_interno.cuh"
#include <type_traits>

namespace tq {

// ---------------------------------------------------------------- types and neighbours
// The preconditioner's level-0 types: bubble air counts as water (js/pressao-cpu.js:305-308);
// with TQ_PRECOND_BLOCK (bloco) it stays air.
__global__ void k_mg_tipo0(const uint8_t* tipo, const uint32_t* rot, uint8_t* t0, int N, int bolhas, int bloco) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  uint8_t t = tipo[c];
  if (bolhas && !bloco && t == AR && rot[c] >= 2) t = AGUA;
  t0[c] = t;
}

// tiposGrossos (js/pressao-cpu.js:63-81): air if any child is air, else water if any is water.
__global__ void k_mg_tipo_grosso(const uint8_t* tf, int fnx, int fny, uint8_t* tg, int gnx, int gny) {
  int C = blockIdx.x * blockDim.x + threadIdx.x;
  if (C >= gnx * gny) return;
  int I = C % gnx, J = C / gnx;
  bool ar = false, agua = false;
  for (int b = 0; b < 2; b++)
    for (int a = 0; a < 2; a++) {
      int i = 2 * I + a, j = 2 * J + b;
      if (i >= fnx || j >= fny) continue;
      uint8_t t = tf[i + j * fnx];
      if (t == AR) ar = true;
      else if (t == AGUA) agua = true;
    }
  tg[C] = ar ? AR : agua ? AGUA : SOLIDO;
}

// prepararVizinhos (js/pressao-cpu.js:44-60) packed in one byte: bits 0-3 = free (non-wall)
// left/right/down/up neighbours, bit 4 = the cell itself is water.
__global__ void k_viz(const uint8_t* tipo, int nx, int ny, uint8_t* viz) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nx * ny) return;
  int i = c % nx, j = c / nx;
  int m = 0;
  if (i > 0 && tipo[c - 1] != SOLIDO) m |= 1;
  if (i < nx - 1 && tipo[c + 1] != SOLIDO) m |= 2;
  if (j > 0 && tipo[c - nx] != SOLIDO) m |= 4;
  if (j < ny - 1 && tipo[c + nx] != SOLIDO) m |= 8;
  if (tipo[c] == AGUA) m |= 16;
  viz[c] = (uint8_t)m;
}

// TQ_PRECOND_BLOCK's coarse masks: bits 0-3 open where a fine face across the coarse face joins
// two non-wall fine cells (both coarse cells not wall), bit 4 water.
__global__ void k_viz_faces(const uint8_t* tf, int fnx, int fny, const uint8_t* tg, int gnx, int gny, uint8_t* viz) {
  int C = blockIdx.x * blockDim.x + threadIdx.x;
  if (C >= gnx * gny) return;
  const int I = C % gnx, J = C / gnx;
  int m = 0;
  if (tg[C] != SOLIDO) {
    auto livre = [&](int i, int j) { return i >= 0 && j >= 0 && i < fnx && j < fny && tf[i + j * fnx] != SOLIDO; };
    auto horiz = [&](int i0, int i1) {
      return (livre(i0, 2 * J) && livre(i1, 2 * J)) || (livre(i0, 2 * J + 1) && livre(i1, 2 * J + 1));
    };
    auto vert = [&](int j0, int j1) {
      return (livre(2 * I, j0) && livre(2 * I, j1)) || (livre(2 * I + 1, j0) && livre(2 * I + 1, j1));
    };
    if (I > 0 && tg[C - 1] != SOLIDO && horiz(2 * I - 1, 2 * I)) m |= 1;
    if (I < gnx - 1 && tg[C + 1] != SOLIDO && horiz(2 * I + 1, 2 * I + 2)) m |= 2;
    if (J > 0 && tg[C - gnx] != SOLIDO && vert(2 * J - 1, 2 * J)) m |= 4;
    if (J < gny - 1 && tg[C + gnx] != SOLIDO && vert(2 * J + 1, 2 * J + 2)) m |= 8;
    if (tg[C] == AGUA) m |= 16;
  }
  viz[C] = (uint8_t)m;
}

// ---------------------------------------------------------------- V-cycle kernels
// suavizar (js/pressao-cpu.js:99-150): each 16x16 block reads the snapshot `src` (18x18 with
// its one-cell border, zero outside the grid), runs VARREDURAS red-black sweeps inside the
// block, and writes water cells to `dst` (other cells 0).  desl = 0 or 8 shifts the block
// lattice; ordem = 0 sweeps red then black, 1 black then red.
template <class T>
__global__ void __launch_bounds__(256) k_suavizar(NivelDev<T> n, int desl, int ordem, const T* __restrict__ src,
                                                  T* __restrict__ dst, const T* __restrict__ b) {
  __shared__ float qs[18 * 18];
  if (n.parar && *n.parar) return;  // uniform over the CTA
  const int nx = n.nx, ny = n.ny;
  const int ox = (int)blockIdx.x * 16 - desl, oy = (int)blockIdx.y * 16 - desl;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  for (int s = threadIdx.x; s < 324; s += 256) {
    int sx = s % 18 - 1 + ox, sy = s / 18 - 1 + oy;
    qs[s] = (sx >= 0 && sy >= 0 && sx < nx && sy < ny) ? carregar(src[sx + sy * nx]) : 0.0f;
  }
  const int gx = ox + tx, gy = oy + ty;
  const bool dentro = gx >= 0 && gy >= 0 && gx < nx && gy < ny;
  const int c = gx + gy * nx;
  int vz = dentro ? n.viz[c] : 0;
  float bv = dentro ? carregar(b[c]) : 0.0f;
  const int li = (ty + 1) * 18 + tx + 1;
  const int m = vz & 15;
  const int k = __popc(m);
  const bool ativo = (vz & 16) && k > 0;
  const float invk = ativo ? 1.0f / (float)k : 0.0f;
  const int minhaCor = (gx + gy + 1) & 1;
  __syncthreads();
#pragma unroll
  for (int it = 0; it < VARREDURAS; it++) {
#pragma unroll
    for (int o = 0; o < 2; o++) {
      int cor = o ^ ordem;
      if (ativo && minhaCor == cor) {
        float s = 0.0f;
        if (m & 1) s += qs[li - 1];
        if (m & 2) s += qs[li + 1];
        if (m & 4) s += qs[li - 18];
        if (m & 8) s += qs[li + 18];
        float q = qs[li];
        qs[li] = q + ((s + bv) * invk - q);
      }
      __syncthreads();
    }
  }
  if (dentro) dst[c] = guardar<T>((vz & 16) ? qs[li] : 0.0f);
}

// restringir (js/pressao-cpu.js:159-188) as a gather: coarse b = P^T (b - A x) over the 4x4
// fine window (weights 1/4, 3/4, 3/4, 1/4), only on coarse water cells; coarse x = 0.
template <class TF>
__device__ inline float residuoFino(const NivelDev<TF>& f, const TF* __restrict__ x, const TF* __restrict__ b, int i, int j) {
  if (i < 0 || j < 0 || i >= f.nx || j >= f.ny) return 0.0f;
  int c = i + j * f.nx;
  int vz = f.viz[c];
  if (!(vz & 16)) return 0.0f;
  float s = 0.0f;
  if (vz & 1) s += carregar(x[c - 1]);
  if (vz & 2) s += carregar(x[c + 1]);
  if (vz & 4) s += carregar(x[c - f.nx]);
  if (vz & 8) s += carregar(x[c + f.nx]);
  return carregar(b[c]) - ((float)__popc(vz & 15) * carregar(x[c]) - s);
}

template <class TF, class TG>
__global__ void k_restringir(NivelDev<TF> f, const TF* __restrict__ xf, const TF* __restrict__ bf, NivelDev<TG> g) {
  int C = blockIdx.x * blockDim.x + threadIdx.x;
  if (C >= g.nx * g.ny || (f.parar && *f.parar)) return;
  g.x[C] = guardar<TG>(0.0f);
  if (!(g.viz[C] & 16)) {
    g.b[C] = guardar<TG>(0.0f);
    return;
  }
  int I = C % g.nx, J = C / g.nx;
  const float w[4] = {0.25f, 0.75f, 0.75f, 0.25f};
  float s = 0.0f;
  for (int bb = 0; bb < 4; bb++) {
    int j = 2 * J - 1 + bb;
    for (int a = 0; a < 4; a++) {
      int i = 2 * I - 1 + a;
      s += residuoFino(f, xf, bf, i, j) * (w[a] * w[bb]);
    }
  }
  g.b[C] = guardar<TG>(s);
}

// prolongar (js/pressao-cpu.js:191-214): fine x += bilinear interpolation of the coarse
// correction, coarse water cells only.
__device__ inline int grossoBase(int i) { return (i & 1) == 0 ? (i >> 1) - 1 : (i - 1) >> 1; }
__device__ inline float pesoBase(int i) { return (i & 1) == 0 ? 0.25f : 0.75f; }

template <class TG, class TF>
__global__ void k_prolongar(NivelDev<TG> g, NivelDev<TF> f, TF* __restrict__ xf) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= f.nx * f.ny || (f.parar && *f.parar)) return;
  if (!(f.viz[c] & 16)) return;
  int i = c % f.nx, j = c / f.nx;
  int I0 = grossoBase(i), J0 = grossoBase(j);
  float wx0 = pesoBase(i), wy0 = pesoBase(j);
  float e = 0.0f;
  for (int b = 0; b < 2; b++) {
    int J = J0 + b;
    if (J < 0 || J >= g.ny) continue;
    float wy = b ? 1.0f - wy0 : wy0;
    for (int a = 0; a < 2; a++) {
      int I = I0 + a;
      if (I < 0 || I >= g.nx) continue;
      int C = I + J * g.nx;
      if (g.viz[C] & 16) e += carregar(g.x[C]) * ((a ? 1.0f - wx0 : wx0) * wy);
    }
  }
  xf[c] = guardar<TF>(carregar(xf[c]) + e);
}

// resolverGrosso (js/pressao-cpu.js:217-238): VARREDURAS_GROSSO alternating red-black sweeps
// in place on the coarsest level, one CTA; the level lives in shared memory when it fits.
__global__ void __launch_bounds__(1024) k_grosso(NivelDev<float> n, int emShared) {
  extern __shared__ unsigned char dyn[];
  if (n.parar && *n.parar) return;  // uniform over the CTA
  const int N = n.nx * n.ny, nx = n.nx;
  float* x = n.x;
  const float* b = n.b;
  const uint8_t* viz = n.viz;
  if (emShared) {
    float* xs = (float*)dyn;
    float* bs = xs + N;
    uint8_t* vs = (uint8_t*)(bs + N);
    for (int c = threadIdx.x; c < N; c += blockDim.x) {
      xs[c] = x[c];
      bs[c] = b[c];
      vs[c] = viz[c];
    }
    x = xs;
    b = bs;
    viz = vs;
    __syncthreads();
  }
  for (int k = 0; k < VARREDURAS_GROSSO; k++)
    for (int o = 0; o < 2; o++) {
      int cor = (k & 1) ? 1 - o : o;
      for (int c = threadIdx.x; c < N; c += blockDim.x) {
        int i = c % nx, j = c / nx;
        int vz = viz[c];
        if (!(vz & 16) || ((i + j + 1) & 1) != cor) continue;
        int q = __popc(vz & 15);
        if (!q) continue;
        float s = 0.0f;
        if (vz & 1) s += x[c - 1];
        if (vz & 2) s += x[c + 1];
        if (vz & 4) s += x[c - nx];
        if (vz & 8) s += x[c + nx];
        x[c] = (s + b[c]) / (float)q;
      }
      __syncthreads();
    }
  if (emShared)
    for (int c = threadIdx.x; c < N; c += blockDim.x) n.x[c] = x[c];
}

// ---------------------------------------------------------------- PCG kernels
// Value a water cell's neighbour contributes to A*v (js/pressao-cpu.js:84-93 after difundir,
// :318-324): water -> v, air of an active bubble -> that bubble's value (as stored in the
// f32 grid), anything else -> 0.
__device__ inline float valorViz(const Dev& d, const float* v, const float* vbf, int n, bool bolhas) {
  uint8_t t = d.tipo[n];
  if (t == AGUA) return v[n];
  if (bolhas && t == AR) {
    uint32_t r = d.rotulo[n];
    if (r >= 2 && r < (uint32_t)MAX_BOLHAS && d.facesB[r] > 0) return vbf[r];
  }
  return 0.0f;
}
__device__ inline float aplicarA(const Dev& d, const uint8_t* vizOp, const float* v, const float* vbf, int c, bool bolhas) {
  int vz = vizOp[c];
  float s = 0.0f;
  if (vz & 1) s += valorViz(d, v, vbf, c - 1, bolhas);
  if (vz & 2) s += valorViz(d, v, vbf, c + 1, bolhas);
  if (vz & 4) s += valorViz(d, v, vbf, c - d.nx, bolhas);
  if (vz & 8) s += valorViz(d, v, vbf, c + d.nx, bolhas);
  return (float)__popc(vz & 15) * v[c] - s;
}

// r = -div - A q on water cells (js/pressao-cpu.js:331-338); q = 0 elsewhere.
__global__ void k_pcg_inicio(Dev d, const uint8_t* vizOp, int bolhas, double* q64) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N) return;
  if (d.tipo[c] != AGUA) {
    d.q[c] = 0.0f;
    d.r[c] = 0.0f;
    return;
  }
  d.r[c] = -d.div[c] - aplicarA(d, vizOp, d.q, d.ybf, c, bolhas != 0);
  if (q64) q64[c] = (double)d.q[c];  // tolerance mode: the FP64 iterate
}

// Active bubbles (montarBolhas, js/pressao-cpu.js:271-288): faces = number of (interior bubble
// cell, water neighbour) pairs; cels = every air cell carrying an active label (:345-351).
__global__ void k_bolhas_faces(Dev d) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N) return;
  const int nx = d.nx;
  int i = c % nx, j = c / nx;
  if (i < 1 || j < 1 || i >= nx - 1 || j >= d.ny - 1) return;
  uint32_t b = d.rotulo[c];
  if (b < 2 || b >= (uint32_t)MAX_BOLHAS || d.tipo[c] != AR) return;
  unsigned k = (d.tipo[c - 1] == AGUA) + (d.tipo[c + 1] == AGUA) + (d.tipo[c - nx] == AGUA) + (d.tipo[c + nx] == AGUA);
  if (k) atomicAdd(&d.facesB[b], k);
}
__global__ void k_bolhas_celulas(Dev d) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N) return;
  uint32_t b = d.rotulo[c];
  if (b < 2 || b >= (uint32_t)MAX_BOLHAS || d.tipo[c] != AR || d.facesB[b] == 0) return;
  atomicAdd(&d.celsB[b], 1u);
}
// Initial bubble values: y from the caller (f32), zero for inactive labels.
__global__ void k_bolhas_inicio(Dev d) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= MAX_BOLHAS) return;
  bool at = b >= 2 && d.facesB[b] > 0;
  double y = at ? (double)d.yBolhaF[b] : 0.0;
  d.yB[b] = y;
  d.ybf[b] = (float)y;
  d.rb[b] = d.zb[b] = d.zvb[b] = d.pb[b] = d.apb[b] = 0.0;
  d.pbf[b] = 0.0f;
}

// Bubble rows of A*v (aplicarBolhas, js/pressao-cpu.js:325-328): out[b] = faces[b]*vb[b] -
// sum over the bubble's water faces of v[water cell].  The sum is 64-bit fixed point (2^-40).
constexpr double ESCALA_PCG = 1099511627776.0;  // 2^40
__global__ void k_bolhas_somar_v(Dev d, const float* v) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N || d.esc->pronto) return;
  const int nx = d.nx;
  int i = c % nx, j = c / nx;
  if (i < 1 || j < 1 || i >= nx - 1 || j >= d.ny - 1) return;
  uint32_t b = d.rotulo[c];
  if (b < 2 || b >= (uint32_t)MAX_BOLHAS || d.tipo[c] != AR) return;
  double s = 0;
  if (d.tipo[c - 1] == AGUA) s += (double)v[c - 1];
  if (d.tipo[c + 1] == AGUA) s += (double)v[c + 1];
  if (d.tipo[c - nx] == AGUA) s += (double)v[c - nx];
  if (d.tipo[c + nx] == AGUA) s += (double)v[c + nx];
  if (s != 0) somaFixa(&d.accB[b], s, ESCALA_PCG);
}
// modo 0: rb = rhs - (faces*y - sum)  (initial bubble residual, :339-341)
// modo 1: apb = faces*pb - sum
__global__ void k_bolhas_linhas(Dev d, int modo) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= MAX_BOLHAS || d.esc->pronto) return;
  if (b < 2 || d.facesB[b] == 0) return;
  double soma = (double)d.accB[b] / ESCALA_PCG;
  if (modo == 0) d.rb[b] = (double)d.rhsBolhaF[b] - (d.facesB[b] * d.yB[b] - soma);
  else d.apb[b] = d.facesB[b] * d.pb[b] - soma;
}

// precondicionar, js/pressao-cpu.js:352-361 — before the V-cycle: level-0 b = r, each active
// bubble's residual spread evenly over its cells; x = 0.  `escala` normalises the right-hand
// side for half-precision storage (the V-cycle is linear).
template <class T>
__global__ void k_pre_espalhar(Dev d, NivelDev<T> n0, int bolhas) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N || d.esc->pronto) return;
  float e = (float)d.esc->escalaMG;
  float v = d.r[c];
  if (bolhas && d.tipo[c] == AR) {
    uint32_t b = d.rotulo[c];
    if (b >= 2 && b < (uint32_t)MAX_BOLHAS && d.celsB[b] > 0) v = (float)(d.rb[b] / d.celsB[b]);
  }
  n0.b[c] = guardar<T>(v * e);
  n0.x[c] = guardar<T>(0.0f);
}
// After the V-cycle: z = x, except active bubble cells, whose mean correction becomes the
// bubble's z (the transpose of spreading) and whose grid value is zeroed.
template <class T>
__global__ void k_pre_juntar(Dev d, NivelDev<T> n0, int bolhas) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N || d.esc->pronto) return;
  float inv = (float)(1.0 / d.esc->escalaMG);
  float x = carregar(n0.x[c]) * inv;
  if (bolhas && d.tipo[c] == AR) {
    uint32_t b = d.rotulo[c];
    if (b >= 2 && b < (uint32_t)MAX_BOLHAS && d.celsB[b] > 0) {
      somaFixa(&d.accB[b], (double)x / d.celsB[b], ESCALA_PCG);
      d.z[c] = 0.0f;
      return;
    }
  }
  d.z[c] = x;
}
// The bubbles' z: the gathered mean correction, or with TQ_PRECOND_BLOCK (bloco) a Jacobi step on
// the bubble's row, r_b / faces_b.
__global__ void k_pre_bolhas(Dev d, int bloco) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= MAX_BOLHAS || d.esc->pronto) return;
  const bool at = b >= 2 && d.facesB[b] > 0;
  d.zb[b] = !at ? 0.0 : bloco ? d.rb[b] / (double)d.facesB[b] : (double)d.accB[b] / ESCALA_PCG;
}

// ap = A p on water cells (js/pressao-cpu.js:367-373).
__global__ void k_aplicar(Dev d, const uint8_t* vizOp, int bolhas) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N || d.esc->pronto) return;
  d.ap[c] = d.tipo[c] == AGUA ? aplicarA(d, vizOp, d.p, d.pbf, c, bolhas != 0) : 0.0f;
}

// q += alpha p, r -= alpha Ap on water; bubbles likewise (js/pressao-cpu.js:377-385).
__global__ void k_atualizar(Dev d, double* q64) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (d.esc->pronto) return;
  double alfa = d.esc->alpha;
  if (c < MAX_BOLHAS && c >= 2 && d.facesB[c] > 0) {
    d.yB[c] += alfa * d.pb[c];
    d.rb[c] -= alfa * d.apb[c];
    d.ybf[c] = (float)d.yB[c];
  }
  if (c >= d.N || d.tipo[c] != AGUA) return;
  float a = (float)alfa;
  if (q64) q64[c] += alfa * (double)d.p[c];
  else d.q[c] = d.q[c] + a * d.p[c];
  d.r[c] = d.r[c] - a * d.ap[c];
}

__device__ inline double somaBloco(double v, double* sh);  // block sum (valid in thread 0), below

// Tolerance mode replaces the recursive FP32 residual by the true one each time the recursive one
// has fallen by this factor since the last replacement (as the fused engine and the oracle do).
constexpr double FATOR_TROCA = 1e-3;

// Tolerance mode, once the recursive residual met the tolerance (Escalares::verificar): the true
// residual in FP64 from the FP64 iterate and the bubble pressures.  Water cells: rt = -div - A q
// into d.ap (free until the next A p) and rt^2 into per-CTA partials; interior air of active
// bubbles: the sum of q over its water faces into the bubble's fixed-point sum (accB, zeroed
// before).  k_verdade_fim finishes the norm and decides.
__global__ void __launch_bounds__(256) k_verdade(Dev d, const uint8_t* vizOp, const double* q64, int bolhas) {
  __shared__ double sh[32];
  if (!d.esc->verificar || d.esc->pronto) return;  // uniform over the grid
  double s = 0;
  const int nx = d.nx;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.N; c += gridDim.x * blockDim.x) {
    const uint8_t t = d.tipo[c];
    if (t == AGUA) {
      const int vz = vizOp[c];
      double sv = 0;
      const int nb[4] = {c - 1, c + 1, c - nx, c + nx};
#pragma unroll
      for (int q = 0; q < 4; q++) {
        if (!(vz & (1 << q))) continue;
        const uint8_t tn = d.tipo[nb[q]];
        if (tn == AGUA) sv += q64[nb[q]];
        else if (bolhas && tn == AR) {
          const uint32_t r = d.rotulo[nb[q]];
          if (r >= 2 && r < (uint32_t)MAX_BOLHAS && d.facesB[r] > 0) sv += d.yB[r];
        }
      }
      const double rt = -(double)d.div[c] - ((double)__popc(vz & 15) * q64[c] - sv);
      d.ap[c] = (float)rt;
      s += rt * rt;
    } else if (bolhas && t == AR) {
      const int i = c % nx, j = c / nx;
      if (i < 1 || j < 1 || i >= nx - 1 || j >= d.ny - 1) continue;
      const uint32_t b = d.rotulo[c];
      if (b < 2 || b >= (uint32_t)MAX_BOLHAS || d.facesB[b] == 0) continue;
      double t2 = 0;
      if (d.tipo[c - 1] == AGUA) t2 += q64[c - 1];
      if (d.tipo[c + 1] == AGUA) t2 += q64[c + 1];
      if (d.tipo[c - nx] == AGUA) t2 += q64[c - nx];
      if (d.tipo[c + nx] == AGUA) t2 += q64[c + nx];
      if (t2 != 0) somaFixa(&d.accB[b], t2, ESCALA_PCG);
    }
  }
  const double tb = somaBloco(s, sh);
  if (threadIdx.x == 0) d.parciais[2 * blockIdx.x] = tb;
}
// One CTA: the true norm (partials in block order, then the bubble rows rhs - (faces y - sum)),
// and the decision: converged or at the cap -> pronto; else the bubble rows take their true
// residual, reiniciar is set (k_substituir copies the water part into r).
__global__ void __launch_bounds__(256) k_verdade_fim(Dev d, int blocosVerdade, int cap, double tol, int bolhas,
                                                    int meiaPrecisao) {
  __shared__ double sh[32];
  __shared__ int substituir;
  Escalares* e = d.esc;
  if (!e->verificar || e->pronto) return;
  double p1 = 0, q1 = 0;
  for (int k = threadIdx.x; k < blocosVerdade; k += blockDim.x) p1 += d.parciais[2 * k];
  auto rbv = [&](int b) { return (double)d.rhsBolhaF[b] - (d.facesB[b] * d.yB[b] - (double)d.accB[b] / ESCALA_PCG); };
  if (bolhas)
    for (int b = threadIdx.x; b < MAX_BOLHAS; b += blockDim.x)
      if (b >= 2 && d.facesB[b] > 0) {
        const double v = rbv(b);
        q1 += v * v;
      }
  const double T1 = somaBloco(p1, sh), B1 = somaBloco(q1, sh);
  if (threadIdx.x == 0) {
    const double nv = sqrt(T1 + B1);
    const bool ok = nv <= tol * e->norma0;
    e->normaVerd = nv;
    e->verificar = 0;
    substituir = 0;
    if (ok || e->iters >= cap) {
      e->pronto = 1;
      e->convergiu = ok ? 1 : 0;
    } else {
      e->reiniciar = 1;
      e->trocas++;
      e->proxTroca = nv * FATOR_TROCA;
      e->norma = nv;
      e->escalaMG = (meiaPrecisao && nv > 0) ? 1.0 / nv : 1.0;
      substituir = 1;
    }
  }
  __syncthreads();
  if (substituir && bolhas)
    for (int b = threadIdx.x; b < MAX_BOLHAS; b += blockDim.x)
      if (b >= 2 && d.facesB[b] > 0) d.rb[b] = rbv(b);
}
// After a replacement: r = the true residual on water cells.
__global__ void k_substituir(Dev d) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N || !d.esc->reiniciar || d.esc->pronto) return;
  if (d.tipo[c] == AGUA) d.r[c] = d.ap[c];
}

// p = z + beta p on water (0 elsewhere); bubbles likewise (js/pressao-cpu.js:395-396).
__global__ void k_direcao(Dev d) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (d.esc->pronto) return;
  double beta = d.esc->beta;
  if (c < MAX_BOLHAS && c >= 2 && d.facesB[c] > 0) {
    d.pb[c] = d.zb[c] + beta * d.pb[c];
    d.pbf[c] = (float)d.pb[c];
  }
  if (c >= d.N) return;
  d.p[c] = d.tipo[c] == AGUA ? d.z[c] + (float)beta * d.p[c] : 0.0f;
}
// p = z, pb = zb (js/pressao-cpu.js:363-364)
__global__ void k_copiar_pz(Dev d) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < MAX_BOLHAS) {
    d.pb[c] = d.zb[c];
    d.pbf[c] = (float)d.zb[c];
    d.zvb[c] = 0.0;
  }
  if (c < d.N) d.p[c] = d.z[c];
}
// zOld = z, zvb = zb (js/pressao-cpu.js:388-389)
__global__ void k_guardar_z(Dev d) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (d.esc->pronto) return;
  if (c < MAX_BOLHAS) d.zvb[c] = d.zb[c];
  if (c < d.N) d.zOld[c] = d.z[c];
}
// End of the solve: non-water q = 0; bubbles hand back their pressure (js/pressao-cpu.js:399-400).
// Tolerance mode: q = the FP64 iterate rounded; the solve's convergence record (thread 0).
__global__ void k_pcg_fim(Dev d, int bolhas, const double* q64, double tol) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (bolhas && c >= 2 && c < MAX_BOLHAS && d.facesB[c] > 0) d.yBolhaF[c] = (float)d.yB[c];
  if (c < d.N) {
    if (d.tipo[c] != AGUA) d.q[c] = 0.0f;
    else if (q64) d.q[c] = (float)q64[c];
  }
  if (c == 0) {
    Escalares* e = d.esc;
    if (!q64) {
      e->normaVerd = -1.0;
      e->convergiu = 0;
    }
    e->solves++;
    if (q64 && !e->convergiu) e->capados++;
    e->itersAcum += e->iters;
    e->trocasAcum += e->trocas;
    if (q64 && e->norma0 > 0 && e->normaVerd / e->norma0 > e->maxRel) e->maxRel = e->normaVerd / e->norma0;
  }
}

// ---------------------------------------------------------------- dot products
// Two FP64 dot products over water cells (a*b1, a*b2) plus the bubble terms, in a fixed
// reduction order; the last block to finish does the scalar step of the running solve.
enum ModoProduto { NORMA0 = 0, RZ0 = 1, PAP = 2, NORMA = 3, BETA = 4 };

constexpr int DOT_BLOCOS = 296;
constexpr int DOT_T = 256;

__device__ inline double somaBloco(double v, double* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double t = 0;
  if (w == 0) {
    t = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  }
  __syncthreads();
  return t;  // valid in thread 0
}

__global__ void __launch_bounds__(DOT_T) k_produto(Dev d, int modo, const float* a, const float* b1, const float* b2,
                                                 int it, double tol, int bolhas, int meiaPrecisao, int cap) {
  __shared__ double sh[32];
  __shared__ bool ultimo;
  if (modo != NORMA0 && d.esc->pronto) return;  // uniform over the grid
  double s1 = 0, s2 = 0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.N; c += gridDim.x * blockDim.x) {
    if (d.tipo[c] != AGUA) continue;
    double av = a[c];
    s1 += av * (double)b1[c];
    if (b2) s2 += av * (double)b2[c];
  }
  double t1 = somaBloco(s1, sh);
  double t2 = b2 ? somaBloco(s2, sh) : 0.0;
  if (threadIdx.x == 0) {
    d.parciais[2 * blockIdx.x] = t1;
    d.parciais[2 * blockIdx.x + 1] = t2;
    __threadfence();
    unsigned v = atomicAdd(&d.esc->tickets[0], 1u);
    ultimo = v == gridDim.x - 1;
  }
  __syncthreads();
  if (!ultimo) return;
  __threadfence();
  // the last block: partials in block order, then the bubble terms in label order
  double p1 = 0, p2 = 0;
  for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) {
    p1 += __ldcg(&d.parciais[2 * k]);
    p2 += __ldcg(&d.parciais[2 * k + 1]);
  }
  double q1 = 0, q2 = 0;
  if (bolhas) {
    for (int b = threadIdx.x; b < MAX_BOLHAS; b += blockDim.x) {
      if (b < 2 || d.facesB[b] == 0) continue;
      switch (modo) {
        case NORMA0:
        case NORMA: q1 += d.rb[b] * d.rb[b]; break;
        case RZ0: q1 += d.rb[b] * d.zb[b]; break;
        case PAP: q1 += d.pb[b] * d.apb[b]; break;
        case BETA: q1 += d.rb[b] * d.zb[b]; q2 += d.rb[b] * d.zvb[b]; break;
      }
    }
  }
  double T1 = somaBloco(p1, sh), T2 = somaBloco(p2, sh);
  double B1 = somaBloco(q1, sh), B2 = somaBloco(q2, sh);
  if (threadIdx.x == 0) {
    Escalares* e = d.esc;
    e->tickets[0] = 0;
    double x1 = T1 + B1, x2 = T2 + B2;
    switch (modo) {
      case NORMA0: {
        double nr = sqrt(x1);
        e->norma0 = e->norma = nr;
        e->normas[0] = nr;
        e->iters = 0;
        e->pronto = 0;
        e->verificar = 0;
        e->reiniciar = 0;
        e->trocas = 0;
        e->convergiu = 0;
        e->normaVerd = -1.0;
        e->proxTroca = nr * FATOR_TROCA;
        e->escalaMG = (meiaPrecisao && nr > 0) ? 1.0 / nr : 1.0;
        break;
      }
      case RZ0: e->rz = x1; break;
      case PAP: e->pap = x1; e->alpha = fabs(x1) < 1e-30 ? 0.0 : e->rz / x1; break;
      case NORMA: {
        double nr = sqrt(x1);
        e->norma = nr;
        if (it + 1 < 1024) e->normas[it + 1] = nr;
        e->iters = it + 1;
        // tolerance mode: the recursive residual met the tolerance, or fell by FATOR_TROCA since
        // the last replacement, or the cap came: the true residual decides (k_verdade,
        // k_verdade_fim)
        e->verificar = tol > 0 && (nr <= tol * e->norma0 || nr <= e->proxTroca || it + 1 >= cap);
        e->escalaMG = (meiaPrecisao && nr > 0) ? 1.0 / nr : 1.0;
        break;
      }
      case BETA: {
        double rzNovo = x1, cruzado = x2;
        // (after a residual replacement the direction carries on: no restart)
        e->beta = fabs(e->rz) < 1e-30 ? 0.0 : fmax(0.0, (rzNovo - cruzado) / e->rz);
        e->reiniciar = 0;
        e->rz = rzNovo;
        break;
      }
    }
  }
}

// ---------------------------------------------------------------- the solver object


Pcg* criarPcg(int nx, int ny, int precisao, int motor, int ctasFundido) {
  Pcg* p = new Pcg();
  p->ctasFundido = ctasFundido;
  p->nx = nx;
  p->ny = ny;
  p->N = nx * ny;
  p->precisao = precisao;
  p->motor = motor;
  // montarNiveis (js/pressao-cpu.js:24-41): halve (ceil) while min(nx, ny) > 12
  int L = 0;
  int a = nx, b = ny;
  p->nxL[0] = a;
  p->nyL[0] = b;
  L = 1;
  while ((a < b ? a : b) > 12 && L < MAX_NIVEIS) {
    a = (a + 1) / 2;
    b = (b + 1) / 2;
    p->nxL[L] = a;
    p->nyL[L] = b;
    L++;
  }
  p->L = L;
  bool ok = true;
  for (int l = 0; l < L; l++) {
    size_t n = (size_t)p->nxL[l] * p->nyL[l];
    p->meia[l] = precisao != TQ_PREC_FP32 && n >= (size_t)MEIA_MIN_CELULAS;
    const size_t e = 4;  // room for FP32 whatever the engine stores
    ok &= cudaMalloc(&p->tipoL[l], n) == cudaSuccess;
    ok &= cudaMalloc(&p->vizL[l], n) == cudaSuccess;
    ok &= cudaMalloc(&p->bL[l], n * e) == cudaSuccess;
    ok &= cudaMalloc(&p->xL[l], n * e) == cudaSuccess;
    ok &= cudaMalloc(&p->tmpL[l], n * e) == cudaSuccess;
  }
  ok &= cudaMalloc(&p->vizOp, p->N) == cudaSuccess;
  size_t nc = (size_t)p->nxL[L - 1] * p->nyL[L - 1];
  p->smemGrosso = nc * 9 <= 200 * 1024 ? nc * 9 : 0;
  if (p->smemGrosso) {
    // The attribute is per kernel, shared by every solver in the process: it is always raised
    // to the 200 KB cap, never set to this grid's size, which would fail the launches of a
    // solver on a grid with a larger coarsest level.
    if (cudaFuncSetAttribute(k_grosso, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess)
      p->smemGrosso = 0;
  }
  if (ok && motor == TQ_ENGINE_FUSED) {
    // Grids with a single level (min(nx, ny) <= 12) have nothing to hand to the coarse
    // section: they run on the plain engine.
    p->fundido = criarFundido(p);
    if (!p->fundido) {
      cudaGetLastError();
      p->motor = TQ_ENGINE_PLAIN;
    }
  }
  if (!ok) {
    destruirPcg(p);
    return nullptr;
  }
  return p;
}

void destruirPcg(Pcg* p) {
  if (!p) return;
  destruirFundido(p->fundido);
  for (int l = 0; l < p->L; l++) {
    cudaFree(p->tipoL[l]);
    cudaFree(p->vizL[l]);
    cudaFree(p->bL[l]);
    cudaFree(p->xL[l]);
    cudaFree(p->tmpL[l]);
  }
  cudaFree(p->vizOp);
  if (p->q64) cudaFree(p->q64);
  destruirRegioes(p->regioes);
  delete p;
}

// Level descriptor with the storage type chosen at run time.
template <class T>
static NivelDev<T> nivel(Pcg* p, int l) {
  NivelDev<T> n;
  n.nx = p->nxL[l];
  n.ny = p->nyL[l];
  n.tipo = p->tipoL[l];
  n.viz = p->vizL[l];
  n.b = (T*)p->bL[l];
  n.x = (T*)p->xL[l];
  n.tmp = (T*)p->tmpL[l];
  n.parar = p->parar;
  return n;
}

// Dispatch on the storage type of level l.
template <class F>
static void comTipo(Pcg* p, int l, F f) {
  if (!p->meia[l]) f((float*)nullptr);
  else if (p->precisao == TQ_PREC_FP16) f((__half*)nullptr);
  else f((__nv_bfloat16*)nullptr);
}

static void suavizarNivel(Pcg* p, int l, int desl, int ordem, bool paraTmp, cudaStream_t s) {
  comTipo(p, l, [&](auto* tag) {
    using T = std::remove_pointer_t<decltype(tag)>;
    NivelDev<T> n = nivel<T>(p, l);
    dim3 g((n.nx + desl + 15) / 16, (n.ny + desl + 15) / 16);
    if (paraTmp) lanca(k_suavizar<T>, g, 256, 0, s, n, desl, ordem, n.x, n.tmp, n.b);
    else lanca(k_suavizar<T>, g, 256, 0, s, n, desl, ordem, n.tmp, n.x, n.b);
  });
}

static void restringirNivel(Pcg* p, int l, cudaStream_t s) {
  comTipo(p, l, [&](auto* tf) {
    using TF = std::remove_pointer_t<decltype(tf)>;
    comTipo(p, l + 1, [&](auto* tg) {
      using TG = std::remove_pointer_t<decltype(tg)>;
      NivelDev<TF> f = nivel<TF>(p, l);
      NivelDev<TG> g = nivel<TG>(p, l + 1);
      lanca(k_restringir<TF, TG>, blocos((long)g.nx * g.ny, 256), 256, 0, s, f, f.x, f.b, g);
    });
  });
}

static void prolongarNivel(Pcg* p, int l, cudaStream_t s) {
  comTipo(p, l + 1, [&](auto* tg) {
    using TG = std::remove_pointer_t<decltype(tg)>;
    comTipo(p, l, [&](auto* tf) {
      using TF = std::remove_pointer_t<decltype(tf)>;
      NivelDev<TG> g = nivel<TG>(p, l + 1);
      NivelDev<TF> f = nivel<TF>(p, l);
      lanca(k_prolongar<TG, TF>, blocos((long)f.nx * f.ny, 256), 256, 0, s, g, f, f.x);
    });
  });
}

// cicloV (js/pressao-cpu.js:241-255); level-0 b and x = 0 already in place.
// umaPassada (TQ_PRECOND_BLOCK_1): the levels above 0 take one smoother pass a leg (shift 8), whose
// output (in tmp) becomes the level's x by swapping the two buffers; each level swaps twice a
// cycle, so the buffers are back in place at its end (and a captured graph repeats itself).
static void cicloV(Pcg* p, cudaStream_t s, bool umaPassada = false) {
  const int L = p->L;
  auto trocar = [&](int l) { std::swap(p->xL[l], p->tmpL[l]); };
  for (int l = 0; l < L - 1; l++) {
    if (umaPassada && l >= 1) {
      suavizarNivel(p, l, 8, 0, true, s);
      trocar(l);
    } else {
      suavizarNivel(p, l, 0, 0, true, s);
      suavizarNivel(p, l, 8, 0, false, s);
    }
    restringirNivel(p, l, s);
  }
  NivelDev<float> g = nivel<float>(p, L - 1);
  if (L == 1) cudaMemsetAsync(g.x, 0, sizeof(float) * g.nx * g.ny, s);
  lanca(k_grosso, 1, 1024, p->smemGrosso, s, g, p->smemGrosso ? 1 : 0);
  for (int l = L - 2; l >= 0; l--) {
    prolongarNivel(p, l, s);
    if (umaPassada && l >= 1) {
      suavizarNivel(p, l, 8, 1, true, s);
      trocar(l);
    } else {
      suavizarNivel(p, l, 8, 1, true, s);
      suavizarNivel(p, l, 0, 1, false, s);
    }
  }
}

// Types and neighbour masks of every level for this solve (bloco: TQ_PRECOND_BLOCK's coarse
// masks from the fine faces).
static void prepararNiveis(Pcg* p, const uint8_t* tipo0, bool bloco, cudaStream_t s) {
  if (tipo0 != p->tipoL[0]) cudaMemcpyAsync(p->tipoL[0], tipo0, p->N, cudaMemcpyDeviceToDevice, s);
  for (int l = 1; l < p->L; l++)
    lanca(k_mg_tipo_grosso, blocos((long)p->nxL[l] * p->nyL[l], 256), 256, 0, s, p->tipoL[l - 1], p->nxL[l - 1],
          p->nyL[l - 1], p->tipoL[l], p->nxL[l], p->nyL[l]);
  for (int l = 0; l < p->L; l++) {
    const int nb = blocos((long)p->nxL[l] * p->nyL[l], 256);
    if (bloco && l >= 1)
      lanca(k_viz_faces, nb, 256, 0, s, p->tipoL[l - 1], p->nxL[l - 1], p->nyL[l - 1], p->tipoL[l], p->nxL[l],
            p->nyL[l], p->vizL[l]);
    else
      lanca(k_viz, nb, 256, 0, s, p->tipoL[l], p->nxL[l], p->nyL[l], p->vizL[l]);
  }
}

static void precondicionar(Pcg* p, const Dev& d, bool bolhas, bool bloco, bool umaPassada, cudaStream_t s) {
  int nb = blocos(d.N, 256);
  const bool espalhar = bolhas && !bloco;  // with BLOCK the V-cycle does not see the bubbles
  comTipo(p, 0, [&](auto* tag) {
    using T = std::remove_pointer_t<decltype(tag)>;
    lanca(k_pre_espalhar<T>, nb, 256, 0, s, d, nivel<T>(p, 0), espalhar ? 1 : 0);
  });
  cicloV(p, s, umaPassada);
  if (espalhar) cudaMemsetAsync(d.accB, 0, MAX_BOLHAS * sizeof(long long), s);
  comTipo(p, 0, [&](auto* tag) {
    using T = std::remove_pointer_t<decltype(tag)>;
    lanca(k_pre_juntar<T>, nb, 256, 0, s, d, nivel<T>(p, 0), espalhar ? 1 : 0);
  });
  if (bolhas) lanca(k_pre_bolhas, blocos(MAX_BOLHAS, 256), 256, 0, s, d, bloco ? 1 : 0);
}

static void produto(Pcg* p, const Dev& d, int modo, const float* a, const float* b1, const float* b2, int it,
                    double tol, bool bolhas, int cap, cudaStream_t s) {
  lanca(k_produto, DOT_BLOCOS, DOT_T, 0, s, d, modo, a, b1, b2, it, tol, bolhas ? 1 : 0,
        p->precisao != TQ_PREC_FP32 ? 1 : 0, cap);
}

// Iterations the plain engine queues between two reads of the stop flag.  Every kernel of an
// iteration returns at once after the flag is set, so the result is the same as stopping at the
// exact iteration, with one host round trip per LOTE_VERIFICACAO iterations instead of one each.
constexpr int LOTE_VERIFICACAO = 8;

int reservarTolerancia(Pcg* p) {
  if (!p->regioes && !(p->regioes = criarRegioes(p->N))) return TQ_E_NOMEM;
  if (p->motor != TQ_ENGINE_FUSED && !p->q64 && cudaMalloc(&p->q64, (size_t)p->N * sizeof(double)) != cudaSuccess)
    return TQ_E_NOMEM;
  return TQ_OK;
}

int resolverPressao(Pcg* p, const Dev& d0, int iteracoes, double tol, bool bolhas, int precond, cudaStream_t s) {
  Dev d = d0;
  double* q64 = nullptr;
  if (tol > 0) {
    if (reservarTolerancia(p)) return TQ_E_NOMEM;
    projetarFechadas(p->regioes, d0, bolhas, s, &d);  // d reads the projected right-hand sides
    q64 = p->q64;
  }
  if (p->motor == TQ_ENGINE_FUSED) return resolverPressaoFundido(p, d, iteracoes, tol, bolhas, precond, s);
  const bool bloco = precond == TQ_PRECOND_BLOCK || precond == TQ_PRECOND_BLOCK_1;
  const bool umaPassada = precond == TQ_PRECOND_BLOCK_1;
  const int nb = blocos(d.N, 256);
  const int nbx = blocos(d.N > MAX_BOLHAS ? d.N : MAX_BOLHAS, 256);
  // operator (true types) and preconditioner types
  lanca(k_viz, nb, 256, 0, s, d.tipo, d.nx, d.ny, p->vizOp);
  lanca(k_mg_tipo0, nb, 256, 0, s, d.tipo, d.rotulo, p->tipoL[0], d.N, bolhas ? 1 : 0, bloco ? 1 : 0);
  prepararNiveis(p, p->tipoL[0], bloco, s);
  cudaMemsetAsync(d.facesB, 0, MAX_BOLHAS * sizeof(uint32_t), s);
  cudaMemsetAsync(d.celsB, 0, MAX_BOLHAS * sizeof(uint32_t), s);
  // the previous solve left its stop flag set: clear it before the first kernel that tests it
  // (the initial bubble sums and rows below; NORMA0 resets the rest of the record)
  cudaMemsetAsync(&d.esc->pronto, 0, sizeof(int), s);
  if (bolhas) {
    lanca(k_bolhas_faces, nb, 256, 0, s, d);
    lanca(k_bolhas_celulas, nb, 256, 0, s, d);
  }
  lanca(k_bolhas_inicio, blocos(MAX_BOLHAS, 256), 256, 0, s, d);
  lanca(k_pcg_inicio, nb, 256, 0, s, d, p->vizOp, bolhas ? 1 : 0, q64);
  if (bolhas) {
    cudaMemsetAsync(d.accB, 0, MAX_BOLHAS * sizeof(long long), s);
    lanca(k_bolhas_somar_v, nb, 256, 0, s, d, d.q);
    lanca(k_bolhas_linhas, blocos(MAX_BOLHAS, 256), 256, 0, s, d, 0);
  }
  produto(p, d, NORMA0, d.r, d.r, nullptr, 0, tol, bolhas, iteracoes, s);
  p->parar = &d.esc->pronto;  // the V-cycle kernels return once the solve has stopped
  precondicionar(p, d, bolhas, bloco, umaPassada, s);
  lanca(k_copiar_pz, nbx, 256, 0, s, d);
  produto(p, d, RZ0, d.r, d.z, nullptr, 0, tol, bolhas, iteracoes, s);
  int it = 0;
  for (; it < iteracoes; it++) {
    lanca(k_aplicar, nb, 256, 0, s, d, p->vizOp, bolhas ? 1 : 0);
    if (bolhas) {
      cudaMemsetAsync(d.accB, 0, MAX_BOLHAS * sizeof(long long), s);
      lanca(k_bolhas_somar_v, nb, 256, 0, s, d, d.p);
      lanca(k_bolhas_linhas, blocos(MAX_BOLHAS, 256), 256, 0, s, d, 1);
    }
    produto(p, d, PAP, d.p, d.ap, nullptr, it, tol, bolhas, iteracoes, s);
    lanca(k_atualizar, nbx, 256, 0, s, d, q64);
    produto(p, d, NORMA, d.r, d.r, nullptr, it, tol, bolhas, iteracoes, s);
    if (q64) {  // the true residual, when NORMA found the recursive one within the tolerance
      if (bolhas) cudaMemsetAsync(d.accB, 0, MAX_BOLHAS * sizeof(long long), s);
      lanca(k_verdade, DOT_BLOCOS, 256, 0, s, d, p->vizOp, q64, bolhas ? 1 : 0);
      lanca(k_verdade_fim, 1, 256, 0, s, d, DOT_BLOCOS, iteracoes, tol, bolhas ? 1 : 0,
            p->precisao != TQ_PREC_FP32 ? 1 : 0);
      lanca(k_substituir, nb, 256, 0, s, d);
    }
    if (it == iteracoes - 1) break;
    if (tol > 0 && it % LOTE_VERIFICACAO == LOTE_VERIFICACAO - 1) {
      int pronto = 0;
      if (cudaMemcpyAsync(&pronto, &d.esc->pronto, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess) {
        p->parar = nullptr;
        return TQ_E_CUDA;
      }
      if (pronto) break;
    }
    lanca(k_guardar_z, nbx, 256, 0, s, d);
    precondicionar(p, d, bolhas, bloco, umaPassada, s);
    produto(p, d, BETA, d.r, d.z, d.zOld, it, tol, bolhas, iteracoes, s);
    lanca(k_direcao, nbx, 256, 0, s, d);
  }
  p->parar = nullptr;
  lanca(k_pcg_fim, nbx, 256, 0, s, d, bolhas ? 1 : 0, q64, tol);
  return cudaGetLastError() == cudaSuccess ? TQ_OK : TQ_E_CUDA;
}

// The residual history of the last solve (Escalares::normas), read from the device.
int normasPcg(Pcg* p, const Dev& d, double* out, int cap, cudaStream_t s) {
  (void)p;
  int iters = 0;
  if (cudaMemcpyAsync(&iters, &d.esc->iters, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return -1;
  int n = iters + 1 < 1024 ? iters + 1 : 1024;
  int k = n < cap ? n : cap;
  if (k > 0 && (cudaMemcpyAsync(out, d.esc->normas, sizeof(double) * k, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess))
    return -1;
  return n;
}
int erroPcg(Pcg* p, cudaStream_t s) {
  const int e = erroFundido(p->fundido, s);
  return e ? e : erroRegioes(p->regioes, s);
}
int motorPcg(Pcg* p) { return p->motor; }
void perfilPcg(Pcg* p, bool ligar) { perfilFundido(p->fundido, ligar); }
int lerPerfilPcg(Pcg* p, unsigned long long* out, int cap) { return lerPerfilFundido(p->fundido, out, cap); }

// One V-cycle on caller-provided device buffers (tq_vcycle).
template <class T>
__global__ void k_carregar_b(NivelDev<T> n0, const float* b) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n0.nx * n0.ny) return;
  n0.b[c] = guardar<T>(b[c]);
  n0.x[c] = guardar<T>(0.0f);
}
template <class T>
__global__ void k_descarregar_x(NivelDev<T> n0, float* x) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n0.nx * n0.ny) return;
  x[c] = carregar(n0.x[c]);
}
int cicloVDispositivo(Pcg* p, const uint8_t* tipo, const float* b, float* x, cudaStream_t s, bool preparar,
                      const int* parar) {
  if (preparar) prepararNiveis(p, tipo, false, s);
  p->parar = parar;  // the cycle's kernels return at once while *parar != 0
  int nb = blocos(p->N, 256);
  comTipo(p, 0, [&](auto* tag) {
    using T = std::remove_pointer_t<decltype(tag)>;
    lanca(k_carregar_b<T>, nb, 256, 0, s, nivel<T>(p, 0), b);
  });
  cicloV(p, s);
  comTipo(p, 0, [&](auto* tag) {
    using T = std::remove_pointer_t<decltype(tag)>;
    lanca(k_descarregar_x<T>, nb, 256, 0, s, nivel<T>(p, 0), x);
  });
  p->parar = nullptr;
  return cudaGetLastError() == cudaSuccess ? TQ_OK : TQ_E_CUDA;
}

// ---------------------------------------------------------------- V-cycle without allocation
// The level hierarchy of tq_vcycle_noalloc lives in this file-scope device array instead of
// cudaMalloc'd buffers.  Level 0 reads the caller's types in place; every other array is
// carved from the scratch on 256-byte boundaries.  The call writes every scratch byte it
// reads before reading it (types and masks of every level, level-0 b and x = 0, the
// restriction's b and x = 0 on each coarse level), so nothing has to start at zero and
// nothing carries over from one call to the next.
static __device__ __align__(256) unsigned char g_scratchVCiclo[BYTES_SCRATCH_VCICLO];

namespace {
constexpr size_t ALINHA_SCRATCH = 256;
inline size_t alinhar(size_t n) { return (n + ALINHA_SCRATCH - 1) & ~(ALINHA_SCRATCH - 1); }

// The level sizes of montarNiveis (js/pressao-cpu.js:24-41), as criarPcg builds them.
int niveisDe(int nx, int ny, int* nxL, int* nyL) {
  int L = 1, a = nx, b = ny;
  nxL[0] = a;
  nyL[0] = b;
  while ((a < b ? a : b) > 12 && L < MAX_NIVEIS) {
    a = (a + 1) / 2;
    b = (b + 1) / 2;
    nxL[L] = a;
    nyL[L] = b;
    L++;
  }
  return L;
}
}  // namespace

size_t bytesScratchVCiclo(int nx, int ny) {
  int nxL[MAX_NIVEIS], nyL[MAX_NIVEIS];
  const int L = niveisDe(nx, ny, nxL, nyL);
  size_t total = 0;
  for (int l = 0; l < L; l++) {
    const size_t n = (size_t)nxL[l] * nyL[l];
    if (l > 0) total += alinhar(n);  // types (level 0 uses the caller's)
    total += alinhar(n) + 3 * alinhar(n * 4);  // masks, b, x, tmp
  }
  return total;
}

// Device address of the scratch on the current device.  The address is looked up with
// cudaGetSymbolAddress once per device and context: the cache holds, per device ordinal, the
// context the address belongs to, and a different current context (the device was reset, or the
// primary context was released and created again, which loads the module anew) looks it up
// again instead of handing out a stale address.  The current context comes from the driver's
// cuCtxGetCurrent, reached through cudaGetDriverEntryPoint (no link to libcuda).
namespace {
using CtxGetCurrent = int (*)(void**);
CtxGetCurrent ctxGetCurrent() {
  static CtxGetCurrent fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      f = nullptr;
    }
    return (CtxGetCurrent)f;
  }();
  return fn;
}
}  // namespace

int enderecoScratchVCiclo(void** out) {
  static std::mutex mtx;
  static void* base[64] = {};
  static void* ctxDe[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return TQ_E_NODEV;
  std::lock_guard<std::mutex> g(mtx);
  void* ctx = nullptr;
  CtxGetCurrent f = ctxGetCurrent();
  if (!f) return TQ_E_CUDA;
  if (!base[dev] || f(&ctx) != 0 || !ctx || ctx != ctxDe[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_scratchVCiclo) != cudaSuccess || !p) {
      cudaGetLastError();
      base[dev] = nullptr;
      return TQ_E_CUDA;
    }
    // the lookup makes the runtime's primary context current if none was: read it after
    if (f(&ctx) != 0 || !ctx) return TQ_E_CUDA;
    base[dev] = p;
    ctxDe[dev] = ctx;
  }
  *out = base[dev];
  return TQ_OK;
}

int cicloVSemAlocar(void* scratch, int nx, int ny, const uint8_t* tipo, const float* b, float* x, int precisao,
                    cudaStream_t s) {
  Pcg p{};
  p.nx = nx;
  p.ny = ny;
  p.N = nx * ny;
  p.precisao = precisao;
  p.motor = TQ_ENGINE_PLAIN;
  p.L = niveisDe(nx, ny, p.nxL, p.nyL);
  unsigned char* cur = (unsigned char*)scratch;
  for (int l = 0; l < p.L; l++) {
    const size_t n = (size_t)p.nxL[l] * p.nyL[l];
    p.meia[l] = precisao != TQ_PREC_FP32 && n >= (size_t)MEIA_MIN_CELULAS;
    if (l == 0) {
      p.tipoL[0] = const_cast<uint8_t*>(tipo);  // only read (prepararNiveis copies nothing)
    } else {
      p.tipoL[l] = cur;
      cur += alinhar(n);
    }
    p.vizL[l] = cur;
    cur += alinhar(n);
    p.bL[l] = cur;
    cur += alinhar(n * 4);
    p.xL[l] = cur;
    cur += alinhar(n * 4);
    p.tmpL[l] = cur;
    cur += alinhar(n * 4);
  }
  // The coarsest solve stages its level in shared memory only within the default 48 KB, which
  // needs no function attribute.
  const size_t nc = (size_t)p.nxL[p.L - 1] * p.nyL[p.L - 1];
  p.smemGrosso = nc * 9 <= 48 * 1024 ? nc * 9 : 0;
  return cicloVDispositivo(&p, tipo, b, x, s);
}

}  // namespace tq
