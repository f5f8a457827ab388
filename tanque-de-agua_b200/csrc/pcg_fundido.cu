// pcg_fundido.cu — FUSED engine of the MGPCG pressure projection: the whole solve of
// resolverPCG (js/pressao-cpu.js:296-402) in ONE persistent cooperative launch.
//
// One CTA of 384 threads per SM (12 warps: room for ~170 registers a thread); phases are separated by a grid barrier (monotonic arrival
// counter, release-add / acquire-poll) whose waits are bounded: a wait that exceeds ~1 s sets
// an error flag, every CTA returns, and the host reports TQ_E_TIMEOUT.
// Per PCG iteration: [DA] p = z + beta p fused with A p and p.Ap, [B] the q/r/bubble updates
// with r.r, [C] the convergence test fused with spreading the residual into the V-cycle's
// right-hand side, the V-cycle, and the gather of z with r.z and r.zOld.
// The V-cycle is the reference's preconditioner (cicloV, js/pressao-cpu.js:241-255):
//   - grid levels: the snapshot block smoother with one WARP per 16x16 block (8 cells per
//     lane, warp-synchronous red-black sweeps in a per-warp shared tile); the prolongation of
//     the coarse correction is folded into the tile load of the first smoother pass on the way
//     up; the restriction is a per-warp tile (a 32-cell coarse row segment and its fine
//     footprint staged in shared memory);
//   - the coarse levels (the largest suffix of levels fitting in ~200 KB) run inside CTA 0's
//     shared memory, warps mapped to rows, while the other CTAs wait at the barrier.
// Scalars (alpha, beta, norms) are FP64 sums of per-CTA partials in a fixed order, computed
// redundantly by every CTA after the barrier, so all CTAs hold the same bits without another
// barrier; per-bubble sums are 64-bit fixed point as in the plain engine.
#include <cstdio>
#include <cstdlib>
#include <type_traits>

#include "common.cuh"
#include "kernels.cuh"
#include "pcg_interno.cuh"

namespace tq {

constexpr int TF = 384;
constexpr int WARPS = TF / 32;
constexpr long long LIMITE_CICLOS = 2000000000LL;  // ~1 s at 1.9 GHz
constexpr double ESC = 1099511627776.0;            // 2^40, per-bubble fixed point
constexpr size_t SMEM_GROSSO_MAX = 200 * 1024;
// Levels up to this many cells run in CTA 0's coarse section; larger ones as grid phases,
// where their 16x16 blocks spread over the SMs instead of queueing on one SM's warps.
constexpr size_t SECAO_MAX_CELULAS = 2048;
// The coarsest solve as a stored matrix: up to DENSO_MAX changing cells (water with a free
// neighbour) on a coarsest level of at most DENSO_MAPA_MAX cells.  Layout at offDenso: the
// matrix (DENSO_MAX^2 floats), the cells (int), their neighbours' list indices (4 int each),
// 1/k (float), and a header (count, count of colour 0).
constexpr int DENSO_MAX = 128;
constexpr int DENSO_MAPA_MAX = DENSO_MAX * DENSO_MAX;
constexpr size_t DENSO_BYTES = (size_t)DENSO_MAX * DENSO_MAX * 4 + (size_t)DENSO_MAX * 4 * 6 + 16;
constexpr size_t SMEM_CTA_MAX = 227 * 1024 - 2048;  // dynamic shared memory cap (static share aside)
// The whole coarse section (levels Lc..L-1 of the V-cycle, from x = 0) is a linear map of level
// Lc's right side, fixed during a solve.  For a top section level of at most SECAO_DENSA_MAX
// cells, a solve that may run at least SECAO_DENSA_MIN_ITERS iterations builds that map once (a
// column per water cell, every CTA running the section on unit vectors) and applies it as one
// grid-wide matrix-vector product per V-cycle, instead of CTA 0 running the section alone.
constexpr int SECAO_DENSA_MAX = 2048;
constexpr int SECAO_DENSA_MIN_ITERS = 30;
// The coarsest level's sweeps run on one warp up to this many cells, on every warp of CTA 0 above.
constexpr int GROSSO_UM_WARP = 1024;
constexpr int NPARC = 4;                           // partial slots per CTA
// Tolerance mode replaces the recursive FP32 residual by the true one (FP64) each time the
// recursive one has fallen by this factor since the last replacement: the rounding it gathers,
// about 1e-7 of the residual it started from per iteration, then stays far below the tolerance.
constexpr double FATOR_TROCA = 1e-3;
// With tanks (tq_set_tanks) the whole grid's recursive residual below the tolerance only starts
// the per-tank checks of the true residual: one every VERIF_TANQUES iterations.  Measured on the
// 256-tank batch: 4,069 tank-substeps/s every 2 iterations, 3,993 every one (more checks), 3,955
// every 4 (more iterations past the stop).
constexpr int VERIF_TANQUES = 2;
constexpr int PERFIL_MAX = 1 << 16;                // phase-trace capacity
constexpr int PERFIL_SECAO = 1 << 14;              // coarse-section stamps (after the phase trace)
// per-warp shared-memory areas (floats)
constexpr int CT = 121;                            // 11x11 coarse tile for the folded prolongation
constexpr int SUAV_W = CT + 7;                     // the coarse tile of a PROL pass
// restriction staging of up to two coarse rows: x (8 x 68), b / residual (floats) + viz (bytes) (6 x 66)
constexpr int REST_W = 8 * 68 + 3 * 6 * 66;

struct NivelF {
  int nx, ny, meia, pad;
  uint8_t* viz;
  uint8_t* tipo;
  void *b, *x, *tmp;
};

// Blocks of a level for a smoother pass with shift `desl`.
__host__ __device__ __forceinline__ int blocosNivel(int nx, int ny, int desl) {
  return ((nx + desl + 15) >> 4) * ((ny + desl + 15) >> 4);
}

struct Fundido {
  int G = 0, Lc = 0;
  uint8_t* solidos = nullptr;  // wall-block flags (Args::sol) of the levels that use them
  bool comParedes[MAX_NIVEIS] = {};  // level l skips wall blocks (its flags exist)
  uint8_t* sol[MAX_NIVEIS] = {};      // level l's flags in `solidos` (Args::sol)
  size_t smem = 0;
  NivelF* niveis = nullptr;  // level table (device)
  double* parc = nullptr;
  unsigned* bar = nullptr;
  int* erro = nullptr;
  long long* accZ = nullptr;
  double *zb2 = nullptr, *pb2 = nullptr;
  int* ativos = nullptr;
  int* nAtivos = nullptr;
  float *p2 = nullptr, *z2 = nullptr;
  float *xc = nullptr, *bc = nullptr;
  int offDenso = -1;  // byte offset of the coarsest level's matrix in CTA 0's shared memory
  bool secaoDensa = false;  // the section's matrix can be built (buffers below allocated)
  float* mSecao = nullptr;   // nW x nW, row i = water cell i of level Lc
  int *wSecao = nullptr, *wInv = nullptr, *nW = nullptr;  // water cells of level Lc, cell -> row, count
  unsigned* densoG = nullptr;  // the coarsest level's matrix block, copied from CTA 0 to every CTA
  uint16_t* op = nullptr;
  unsigned long long* rotB = nullptr;
  void* kern = nullptr;
  unsigned long long* perfil = nullptr;
  bool perfilar = false;
  double* q64 = nullptr;     // the FP64 iterate of a tolerance-mode solve
  long long* accV = nullptr; // per-bubble fixed-point sums of the true residual
  // Bounded-wait test hooks, read from the environment when the solver is created:
  // TQ_BARRIER_WAIT_CYCLES sets the grid barrier's limit (SM clock cycles); TQ_BARRIER_HOLD_CTA
  // and TQ_BARRIER_HOLD_CYCLES make that CTA wait that many cycles before it arrives at the
  // first barrier of the NEXT solve only (one-shot), so the other CTAs' waits run out.
  long long limite = LIMITE_CICLOS;
  int segurarCta = -1;
  long long segurarCiclos = 0;
  // red-black sweeps per smoother pass with the block preconditioner: measured on the 840x536
  // scene, 2 to 8 sweeps change the solve's time by under 5 % (fewer iterations, costlier
  // passes), so the reference's count stays
  int varredurasBloco = VARREDURAS;
};

struct Args {
  Dev d;
  int L, Lc;
  const NivelF* niv;
  uint8_t* vizOp;
  int iteracoes;
  double tol;
  int bolhas, escalar;
  double* parc;
  unsigned* bar;
  int* erro;
  long long* accZ;
  double *zb2, *pb2;
  int* ativos;
  int* nAtivos;
  float *p2, *z2;
  float *xc, *bc;
  int offDenso;  // coarsest-level matrix in CTA 0's dynamic shared memory (-1: sweeps)
  int secaoDensa;  // 1: the section may be replaced by its matrix
  float* mSecao;
  int *wSecao, *wInv, *nWp;
  unsigned* densoG;
  uint16_t* op;  // per-cell operator descriptor of level 0 (OP_*)
  // per-cell bubble labels of level 0, 12 bits each: bits 0-11 the cell's own (air of an active
  // bubble), 12-23 / 24-35 / 36-47 / 48-59 its left / right / down / up neighbour's (0: none)
  unsigned long long* rotB;
  unsigned long long* perfil;  // [0] count, [1..] %globaltimer at each barrier (null: off)
  // per level: 1 per 16x16 block whose cells are all wall (out-of-grid cells count as wall), the
  // blocks of shift 0 then those of shift 8; null where the level does not skip wall blocks
  uint8_t* sol[MAX_NIVEIS];
  long long limite;          // grid barrier wait limit (cycles)
  int segurarCta;            // test hook: this CTA arrives late at the first barrier (-1: none)
  long long segurarCiclos;   // ... after waiting this many cycles (bounded)
  int bloco;  // TQ_PRECOND_BLOCK: bubble rows Jacobi, V-cycle on water, coarse masks from faces
  int varreduras;  // red-black sweeps per smoother pass (VARREDURAS, the reference's, unless BLOCK)
  int umaPassada;  // BLOCK_1: one smoother pass a leg on the grid levels above 0 (see cicloV)
  // tolerance mode: q accumulates in FP64 (q64) and the solve stops on the true residual
  // ||b - A q64|| (FP64), with residual replacement; null in fixed-count mode
  double* q64;
  long long* accV;
};

// The level table, copied into shared memory at kernel start: every phase reads its level's
// sizes and pointers without an L2 round trip in front of its first data load.
__shared__ NivelF s_niv[MAX_NIVEIS];

// Phase trace of the fused solve (the %globaltimer at every grid barrier of the last solve).
void perfilFundido(Fundido* f, bool ligar) {
  if (!f) return;
  f->perfilar = ligar;
  if (ligar && !f->perfil) {
    if (cudaMalloc(&f->perfil, (PERFIL_MAX + 2 + PERFIL_SECAO) * sizeof(unsigned long long)) != cudaSuccess) {
      f->perfil = nullptr;
      f->perfilar = false;
    }
  }
}
int lerPerfilFundido(Fundido* f, unsigned long long* out, int cap) {
  if (!f || !f->perfil) return 0;
  if (cap < 0) {  // the coarse-section stamps instead of the phase trace
    unsigned long long n = 0;
    if (cudaMemcpy(&n, f->perfil + PERFIL_MAX + 1, sizeof n, cudaMemcpyDeviceToHost) != cudaSuccess) return 0;
    if (n > PERFIL_SECAO) n = PERFIL_SECAO;
    int k = (int)(n < (unsigned long long)(-cap) ? n : (unsigned long long)(-cap));
    if (k > 0 && cudaMemcpy(out, f->perfil + PERFIL_MAX + 2, k * 8, cudaMemcpyDeviceToHost) != cudaSuccess) return 0;
    return k;
  }
  unsigned long long n = 0;
  if (cudaMemcpy(&n, f->perfil, sizeof n, cudaMemcpyDeviceToHost) != cudaSuccess) return 0;
  if (n > PERFIL_MAX) n = PERFIL_MAX;
  int k = (int)(n < (unsigned long long)cap ? n : (unsigned long long)cap);
  if (k > 0 && cudaMemcpy(out, f->perfil + 1, k * sizeof(unsigned long long), cudaMemcpyDeviceToHost) != cudaSuccess)
    return 0;
  return k;
}

// ---------------------------------------------------------------- small helpers
template <class T>
__device__ __forceinline__ T ldcg(const T* p) { return __ldcg(p); }
template <>
__device__ __forceinline__ __half ldcg<__half>(const __half* p) {
  return __ushort_as_half(__ldcg((const unsigned short*)p));
}
template <>
__device__ __forceinline__ __nv_bfloat16 ldcg<__nv_bfloat16>(const __nv_bfloat16* p) {
  return __ushort_as_bfloat16(__ldcg((const unsigned short*)p));
}
__device__ __forceinline__ int ldcg8(const uint8_t* p) { return (int)__ldcg((const unsigned char*)p); }
// Loads of a smoother pass's snapshot, right-hand side and masks: through L1 (ld.ca), where
// the lines a warp shares with the blocks beside it may already be.  These arrays were last
// written before the grid barrier that opens the pass, whose acquire orders the loads after
// those writes (PTX memory model; the cache operator is a hint), and the pass writes other
// arrays.  Measured: 1,085 against 1,099 us per iteration on the 38,370x316 atlas, no change
// on the 840x536 scene.
template <class T>
__device__ __forceinline__ T ldsv(const T* p) { return __ldca(p); }
template <>
__device__ __forceinline__ __half ldsv<__half>(const __half* p) {
  return __ushort_as_half(__ldca((const unsigned short*)p));
}
template <>
__device__ __forceinline__ __nv_bfloat16 ldsv<__nv_bfloat16>(const __nv_bfloat16* p) {
  return __ushort_as_bfloat16(__ldca((const unsigned short*)p));
}
__device__ __forceinline__ int ldsv8(const uint8_t* p) { return (int)__ldca((const unsigned char*)p); }

__device__ __forceinline__ void gravarN(int meia, void* v, int c, float x) {
  if (meia == 0) ((float*)v)[c] = x;
  else if (meia == 1) ((__half*)v)[c] = __float2half_rn(x);
  else ((__nv_bfloat16*)v)[c] = __float2bfloat16_rn(x);
}

__device__ __forceinline__ unsigned lerAdquirir(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void somarLiberar(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid barrier: every CTA adds 1 (release) to a counter that only grows during the solve and
// waits (acquire) until it reaches epoch * gridDim.  The wait is bounded.  Returns false when
// this CTA gave up (its wait ran out, or it saw another CTA's error flag while waiting); a CTA
// that gave up returns, so the others give up at their next barrier.
__device__ bool barreira(const Args& a, unsigned& epoca) {
  __shared__ int falhou;
  __syncthreads();
  if (threadIdx.x == 0) {
    if (epoca == 0 && (int)blockIdx.x == a.segurarCta) {  // test hook: a late arrival, bounded
      const long long t = clock64();
      while (clock64() - t < a.segurarCiclos) __nanosleep(1000);
    }
    epoca++;
    const unsigned alvo = epoca * gridDim.x;
    somarLiberar(a.bar, 1u);
    long long t0 = clock64();
    int f = 0;
    for (unsigned voltas = 0;; voltas++) {
      if (lerAdquirir(a.bar) >= alvo) break;
      if ((voltas & 255u) == 255u) {
        if (*(volatile int*)a.erro) {
          f = 1;
          break;
        }
        if (clock64() - t0 > a.limite) {
          atomicExch(a.erro, 1);
          f = 1;
          break;
        }
      }
    }
    falhou = f;
    if (a.perfil && blockIdx.x == 0) {
      unsigned long long t;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
      unsigned long long k = a.perfil[0]++;
      if (k < PERFIL_MAX) a.perfil[1 + k] = t;
    }
  }
  __syncthreads();
  return falhou == 0;
}

// Block sum of a double (valid in thread 0).
__device__ double somaBloco(double v, double* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double t = 0;
  if (w == 0) {
    t = lane < WARPS ? sh[lane] : 0.0;  // only WARPS slots were written
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  }
  return t;
}

// Sums, in CTA order, of the per-CTA partials of channels 0 and 1, plus up to two sums over
// the active bubbles (ascending labels).  Warp 0 of every CTA does the same work on the same
// data, so every CTA obtains the same bits.
template <class F0, class F1>
__device__ void somasGlobais(const Args& a, int nAt, F0 f0, F1 f1, double* sh, double out[4]) {
  __syncthreads();
  if (threadIdx.x < 32) {
    // Loads go out in batches before the sums (a rolled load-add loop waits one L2 round trip
    // per step); each lane still adds its terms in ascending order.
    double v0 = 0, v1 = 0, b0 = 0, b1 = 0;
    constexpr int UC = 5;  // 5 x 32 slots cover one CTA per SM
    for (int k0 = 0; k0 < (int)gridDim.x; k0 += 32 * UC) {
      double p0[UC], p1[UC];
#pragma unroll
      for (int u = 0; u < UC; u++) {
        const int k = k0 + threadIdx.x + 32 * u;
        p0[u] = k < (int)gridDim.x ? __ldcg(&a.parc[k * NPARC + 0]) : 0.0;
        p1[u] = k < (int)gridDim.x ? __ldcg(&a.parc[k * NPARC + 1]) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < UC; u++) {
        v0 += p0[u];
        v1 += p1[u];
      }
    }
    constexpr int UB = 4;
    for (int k0 = 0; k0 < nAt; k0 += 32 * UB) {
      int bs[UB];
#pragma unroll
      for (int u = 0; u < UB; u++) {
        const int k = k0 + threadIdx.x + 32 * u;
        bs[u] = k < nAt ? __ldcg(&a.ativos[k]) : -1;
      }
      double t0[UB], t1[UB];
#pragma unroll
      for (int u = 0; u < UB; u++) {
        t0[u] = bs[u] >= 0 ? f0(bs[u]) : 0.0;
        t1[u] = bs[u] >= 0 ? f1(bs[u]) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < UB; u++) {
        b0 += t0[u];
        b1 += t1[u];
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      v0 += __shfl_down_sync(0xffffffffu, v0, o);
      v1 += __shfl_down_sync(0xffffffffu, v1, o);
      b0 += __shfl_down_sync(0xffffffffu, b0, o);
      b1 += __shfl_down_sync(0xffffffffu, b1, o);
    }
    if (threadIdx.x == 0) {
      sh[0] = v0;
      sh[1] = v1;
      sh[2] = b0;
      sh[3] = b1;
    }
  }
  __syncthreads();
  out[0] = sh[0];
  out[1] = sh[1];
  out[2] = sh[2];
  out[3] = sh[3];
  __syncthreads();
}

__device__ __forceinline__ bool bolhaAtiva(const Args& a, uint32_t r) {
  return r >= 2 && r < (uint32_t)MAX_BOLHAS && __ldcg(&a.d.facesB[r]) > 0;
}

// The preconditioned residual z_b of active bubble b: REFERENCE, the mean V-cycle correction
// over its cells (the gather's fixed-point sum, precondicionar js/pressao-cpu.js:357-361);
// BLOCK, a Jacobi step on its row, r_b / faces_b (its diagonal).
__device__ __forceinline__ double zbDe(const Args& a, int b) {
  return a.bloco ? __ldcg(&a.d.rb[b]) / (double)__ldcg(&a.d.facesB[b]) : (double)__ldcg(&a.accZ[b]) / ESC;
}

// Free-neighbour bits (0-3: left, right, down, up) of coarse cell (I, J) of level g from the
// faces of its finer level f (TQ_PRECOND_BLOCK): a coarse face is open when both coarse cells
// are not wall and a fine face across it (between fine columns 2I+1 and 2I+2 in rows 2J, 2J+1,
// or the vertical counterpart) joins two non-wall fine cells.  Walls thinner than a coarse cell
// then still separate the water on either side.
__device__ __noinline__ int vizinhosPorFaces(const NivelF& f, const NivelF& g, int I, int J) {
  const int C = I + J * g.nx;
  if (ldcg8(g.tipo + C) == SOLIDO) return 0;
  auto livre = [&](int i, int j) {
    return i >= 0 && j >= 0 && i < f.nx && j < f.ny && ldcg8(f.tipo + i + j * f.nx) != SOLIDO;
  };
  auto horiz = [&](int i0, int i1) {
    return (livre(i0, 2 * J) && livre(i1, 2 * J)) || (livre(i0, 2 * J + 1) && livre(i1, 2 * J + 1));
  };
  auto vert = [&](int j0, int j1) {
    return (livre(2 * I, j0) && livre(2 * I, j1)) || (livre(2 * I + 1, j0) && livre(2 * I + 1, j1));
  };
  int m = 0;
  if (I > 0 && ldcg8(g.tipo + C - 1) != SOLIDO && horiz(2 * I - 1, 2 * I)) m |= 1;
  if (I < g.nx - 1 && ldcg8(g.tipo + C + 1) != SOLIDO && horiz(2 * I + 1, 2 * I + 2)) m |= 2;
  if (J > 0 && ldcg8(g.tipo + C - g.nx) != SOLIDO && vert(2 * J - 1, 2 * J)) m |= 4;
  if (J < g.ny - 1 && ldcg8(g.tipo + C + g.nx) != SOLIDO && vert(2 * J + 1, 2 * J + 2)) m |= 8;
  return m;
}

// Per-cell operator descriptor of level 0 (built once per solve): bits 0-3 the left, right,
// down and up neighbours are water; OP_AGUA the cell is water; OP_FACE interior air of an
// active bubble (its water faces enter the bubble's row); OP_VIZ_BOLHA a free neighbour is
// air of an active bubble; OP_BOLHA air of an active bubble; bits 8-10 the number of free
// (non-wall) neighbours.
constexpr int OP_AGUA = 16, OP_FACE = 32, OP_VIZ_BOLHA = 64, OP_BOLHA = 128;
// Level 0's neighbour masks also carry, above bits 0-4, the cell's OP_BOLHA and OP_AGUA.
constexpr int V0_BOLHA = 32, V0_AGUA = 64;

__device__ __forceinline__ int grossoBaseF(int i) { return (i & 1) == 0 ? (i >> 1) - 1 : (i - 1) >> 1; }
__device__ __forceinline__ float pesoBaseF(int i) { return (i & 1) == 0 ? 0.25f : 0.75f; }

// ---------------------------------------------------------------- block sweeps
// 1/k for k free neighbours (k = 1..4), the correctly rounded float constants.
__device__ __forceinline__ float inversoVizinhos(int k) {
  return k == 1 ? 1.0f : k == 2 ? 0.5f : k == 3 ? (1.0f / 3.0f) : 0.25f;
}

// ---------------------------------------------------------------- grid-level smoother
// Modes of a smoother pass over a grid level:
//   M_NORMAL   snapshot = src, right side = b;
//   M_PROL     snapshot = x + P(x_coarse) (prolongar, js/pressao-cpu.js:191-214), built while
//              loading: the first pass on the way up;
//   M_ZERO     snapshot = 0: the first pass on the way down, whose x the restriction (or the
//              spread) leaves at 0 (js/pressao-cpu.js:186, :354);
//   M_ESPALHAR level 0, first pass: also spreads the residual into b (precondicionar,
//              js/pressao-cpu.js:353-355), b = escala * r, bubble cells their bubble's mean;
//   M_JUNTAR   level 0, last pass: instead of storing x, gathers z = x / escala (:357-361),
//              bubble cells' share into the bubble's fixed-point sum, and the partials of r.z
//              and r.zOld.
enum { M_NORMAL = 0, M_PROL = 1, M_ZERO = 2, M_ESPALHAR = 3, M_JUNTAR = 4 };

// What the spread and the gather need (level 0).
struct Reuniao {
  float escala;          // b = escala * residual; z = x / escala
  float* zNovo;
  const float* zVelho;   // previous z (r.zOld), or null
};

// ---------------------------------------------------------------- register-resident block sweep
// Lane l of the warp that owns a 16x16 block holds, for each colour c and m = 0..3, the cell of
// colour c in row 4g + m (g = l >> 3) among the columns 2k, 2k + 1 (k = l & 7): its column is
// (c + 1 + m) & 1, since a cell's colour is (row + column + 1) & 1 (js/pressao-cpu.js:120).  It
// also holds the block's frame next to its cells: left and right of its rows (k = 0, k = 7),
// below and above its columns (g = 0, g = 3).  In a half-sweep of colour COR every neighbour of
// an updated cell has the other colour: the lane's own other cell in the row, the rows m -/+ 1
// of the lane (same column), the row in lane l -/+ 1, the row below row 0 in lane l - 8 (its
// m = 3), the row above row 3 in lane l + 8 (its m = 0), or the frame: 6 shuffles a half-sweep,
// which keeps the shuffle pipe, shared by the SM's warps, half as busy as rows g + 4m would.
// A half-sweep reads no value that it writes.
// Every snapshot holds x = 0 on cells that are not water (the passes store 0 there, the frame
// outside the grid is 0), so a wall neighbour adds +0 and the sum needs no mask; only 1/k and
// whether the cell changes come from the mask.  The exception is TQ_PRECOND_BLOCK's coarse
// levels, whose masks close faces between two water cells across a thin wall: with `masc` the
// neighbours the mask leaves out are dropped from the sum (masc is uniform over the grid).
struct Moldura {
  float esq[4], dir[4];  // frame left / right of the lane's rows (k = 0 / k = 7)
  float bai[2], cim[2];  // frame below / above the lane's columns (g = 0 / g = 3), by column
};

template <int COR>
__device__ __forceinline__ void meiaReg(float (&x)[2][4], const float (&bq)[2][4], const float (&iq)[2][4],
                                        const float (&at)[2][4], const Moldura& f, const int (&v)[2][4], bool masc) {
  const int lane = threadIdx.x & 31, g = lane >> 3, k = lane & 7;
  float H[4];
#pragma unroll
  for (int m = 0; m < 4; m++)  // row m's neighbour in lane l + 1 (colour COR in the odd column) or l - 1
    H[m] = __shfl_sync(0xffffffffu, x[1 - COR][m], (((COR + 1 + m) & 1) ? lane + 1 : lane - 1) & 31);
  const float D = __shfl_sync(0xffffffffu, x[1 - COR][3], (lane - 8) & 31);
  const float U = __shfl_sync(0xffffffffu, x[1 - COR][0], (lane + 8) & 31);
#pragma unroll
  for (int m = 0; m < 4; m++) {
    const int jc = (COR + 1 + m) & 1;  // the column of colour COR in row m
    const float y = x[1 - COR][m];
    float esq = jc ? y : (k == 0 ? f.esq[m] : H[m]);
    float dir = jc ? (k == 7 ? f.dir[m] : H[m]) : y;
    float baixo = m >= 1 ? x[1 - COR][m >= 1 ? m - 1 : 0] : (g >= 1 ? D : f.bai[jc]);
    float cima = m <= 2 ? x[1 - COR][m <= 2 ? m + 1 : 3] : (g <= 2 ? U : f.cim[jc]);
    if (masc) {
      const int mk = v[COR][m];
      esq = (mk & 1) ? esq : 0.0f;
      dir = (mk & 2) ? dir : 0.0f;
      baixo = (mk & 4) ? baixo : 0.0f;
      cima = (mk & 8) ? cima : 0.0f;
    }
    const float sm = ((esq + dir) + baixo) + cima;
    const float q = x[COR][m];
    const float dlt = (sm + bq[COR][m]) * iq[COR][m] - q;
    x[COR][m] = fmaf(at[COR][m], dlt, q);  // at = 1 (the cell changes) or 0: exact either way
  }
}

// The VARREDURAS red-black sweeps (js/pressao-cpu.js:114-137) of the warp's block in registers;
// v = neighbour mask | 16 water | 128 in grid, bq = right side; ordem 0 sweeps colour 0 first.
__device__ __forceinline__ void varrerReg(float (&x)[2][4], const int (&v)[2][4], const float (&bq)[2][4],
                                         const Moldura& f, int ordem, bool masc, int nVarr) {
  float iq[2][4], at[2][4];
#pragma unroll
  for (int c = 0; c < 2; c++)
#pragma unroll
    for (int m = 0; m < 4; m++) {
      const int mk = v[c][m] & 15;
      iq[c][m] = inversoVizinhos(__popc(mk));
      at[c][m] = ((v[c][m] & 16) && mk) ? 1.0f : 0.0f;
    }
  // rolled loop: the pass code stays small in the instruction cache, which each phase enters cold
#pragma unroll 1
  for (int h = 0; h < 2 * nVarr; h++) {
    if (((h & 1) ^ ordem) == 0) meiaReg<0>(x, bq, iq, at, f, v, masc);
    else meiaReg<1>(x, bq, iq, at, f, v, masc);
  }
}

// Bilinear coarse correction at fine cell (sx, sy) from the 11x11 coarse tile ct whose origin is
// (cx0, cy0) (prolongar, js/pressao-cpu.js:191-214).
__device__ __forceinline__ float correcaoGrossa(const float* ct, int cx0, int cy0, int sx, int sy) {
  const int I0 = grossoBaseF(sx) - cx0, J0 = grossoBaseF(sy) - cy0;
  const float wx0 = pesoBaseF(sx), wy0 = pesoBaseF(sy);
  float e = 0.0f;
#pragma unroll
  for (int b = 0; b < 2; b++) {
    const float wy = b ? 1.0f - wy0 : wy0;
#pragma unroll
    for (int aa = 0; aa < 2; aa++) e += ct[(J0 + b) * 11 + I0 + aa] * ((aa ? 1.0f - wx0 : wx0) * wy);
  }
  return e;
}

// suavizar (js/pressao-cpu.js:99-150) for one 16x16 block, by one warp, in registers (see
// meiaReg).  Every global load of the block (cells, frame, flags, right side; with PROL the
// coarse tile) goes out in one batch.
template <class T, int MODO>
__device__ __forceinline__ void suavizarBloco(const Args& a, const NivelF& n, int blk, int nbx, int desl, int ordem,
                                              const T* src, T* dst, float* area, const NivelF& g,
                                              const float* xcSecao, const Reuniao& ru, double& s0, double& s1) {
  constexpr bool PROL = MODO == M_PROL;
  constexpr bool ZERO = MODO == M_ZERO || MODO == M_ESPALHAR;
  const int lane = threadIdx.x & 31, gl = lane >> 3, k = lane & 7;
  const int bx = blk % nbx, by = blk / nbx;
  const int ox = bx * 16 - desl, oy = by * 16 - desl;
  const int nx = n.nx, ny = n.ny;
  const T* b = (const T*)n.b;
  // PROL: the coarse tile (columns from (ox-2)>>1, rows from (oy-2)>>1, 11x11) is loaded first,
  // so that every load of the block is in flight before any result is used.  Coarse x is 0 off
  // water (a grid level's snapshot, or the section's output, zeroed before the solve off water),
  // so the tile needs no water flags.
  const int cx0 = (ox - 2) >> 1, cy0 = (oy - 2) >> 1;
  float cv[4];
  if (PROL) {
    int C[4];
    bool ok[4];
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
      const int s = lane + 32 * kk;
      const int I = cx0 + s % 11, J = cy0 + s / 11;
      ok[kk] = s < CT && I >= 0 && J >= 0 && I < g.nx && J < g.ny;
      C[kk] = ok[kk] ? I + J * g.nx : 0;
    }
    // the coarse values' storage type is chosen once (warp-uniform), so the four loads are
    // straight-line code in flight together
    if (xcSecao) {
#pragma unroll
      for (int kk = 0; kk < 4; kk++) cv[kk] = ok[kk] ? __ldcg(xcSecao + C[kk]) : 0.0f;
    } else if (g.meia == 1) {
#pragma unroll
      for (int kk = 0; kk < 4; kk++) cv[kk] = ok[kk] ? __half2float(ldcg((const __half*)g.x + C[kk])) : 0.0f;
    } else if (g.meia == 2) {
#pragma unroll
      for (int kk = 0; kk < 4; kk++)
        cv[kk] = ok[kk] ? __bfloat162float(ldcg((const __nv_bfloat16*)g.x + C[kk])) : 0.0f;
    } else {
#pragma unroll
      for (int kk = 0; kk < 4; kk++) cv[kk] = ok[kk] ? __ldcg((const float*)g.x + C[kk]) : 0.0f;
    }
  }
  float x[2][4], bq[2][4];  // [colour][m], see meiaReg
  int v[2][4], cel[2][4];
  int om[2][4];  // M_ESPALHAR: the cells' own bubble labels (0: not bubble air)
  Moldura f;
  unsigned aguaF = 0;  // PROL: water flags of the frame cells (bits 0-3 left, 4-7 right, 8-9 below, 10-11 above)
#pragma unroll
  for (int cr = 0; cr < 2; cr++)
#pragma unroll
    for (int m = 0; m < 4; m++) {
      const int gx = ox + 2 * k + ((cr + 1 + m) & 1), gy = oy + 4 * gl + m;
      const bool dentro = gx >= 0 && gy >= 0 && gx < nx && gy < ny;
      const int c = gx + gy * nx;
      cel[cr][m] = dentro ? c : -1;
      v[cr][m] = dentro ? (ldsv8(n.viz + c) | 128) : 0;
      x[cr][m] = (!ZERO && dentro) ? carregar(ldsv(src + c)) : 0.0f;
      if (MODO == M_ESPALHAR) {
        bq[cr][m] = dentro ? __ldcg(a.d.r + c) : 0.0f;
        om[cr][m] = (v[cr][m] & V0_BOLHA) ? (int)(__ldcg(a.rotB + c) & 0xfff) : 0;  // own bubble label
      } else {
        bq[cr][m] = dentro ? carregar(ldsv(b + c)) : 0.0f;
      }
    }
  // The block's frame: lane i loads the left (i < 16) or right column's row i & 15 and the
  // bottom (i < 16) or top row's column i & 15; the lanes next to the frame (k = 0 / 7 for the
  // columns, g = 0 / 3 for the rows) take their values by shuffle.  With PROL the same two cells'
  // water flags come along (gathered by ballot below).
  int vzLR = 0, vzBT = 0;
  {
    const int fr = lane & 15;
    const int gxA = lane < 16 ? ox - 1 : ox + 16, gyA = oy + fr;
    const int gxB = ox + fr, gyB = lane < 16 ? oy - 1 : oy + 16;
    const bool okA = gxA >= 0 && gxA < nx && gyA >= 0 && gyA < ny;
    const bool okB = gxB >= 0 && gxB < nx && gyB >= 0 && gyB < ny;
    if (PROL) {
      vzLR = okA ? ldsv8(n.viz + gxA + gyA * nx) : 0;
      vzBT = okB ? ldsv8(n.viz + gxB + gyB * nx) : 0;
    }
    if (ZERO) {
#pragma unroll
      for (int m = 0; m < 4; m++) f.esq[m] = f.dir[m] = 0.0f;
#pragma unroll
      for (int j = 0; j < 2; j++) f.bai[j] = f.cim[j] = 0.0f;
    } else {
      const float xA = okA ? carregar(ldsv(src + gxA + gyA * nx)) : 0.0f;
      const float xB = okB ? carregar(ldsv(src + gxB + gyB * nx)) : 0.0f;
#pragma unroll
      for (int m = 0; m < 4; m++) f.esq[m] = f.dir[m] = __shfl_sync(0xffffffffu, xA, (k == 7 ? 16 : 0) + 4 * gl + m);
#pragma unroll
      for (int j = 0; j < 2; j++) f.bai[j] = f.cim[j] = __shfl_sync(0xffffffffu, xB, (gl == 3 ? 16 : 0) + 2 * k + j);
    }
  }
  if (MODO == M_ESPALHAR) {
    // cells of active bubbles take their bubble's mean residual; b is stored in the storage
    // type and the sweep uses the stored value
#pragma unroll
    for (int cr = 0; cr < 2; cr++)
#pragma unroll
      for (int m = 0; m < 4; m++) {
        if (cel[cr][m] < 0) continue;
        float val = bq[cr][m];
        if (om[cr][m]) val = (float)(__ldcg(a.d.rb + om[cr][m]) / __ldcg(a.d.celsB + om[cr][m]));
        const T bt = guardar<T>(val * ru.escala);
        ((T*)n.b)[cel[cr][m]] = bt;
        bq[cr][m] = carregar(bt);
      }
  }
  if (PROL) {
    // the frame's water flags of this lane's frame cells: bits 0-3 left rows 4g..4g+3 (k = 0),
    // 4-7 right (k = 7), 8-9 below columns 2k, 2k+1 (g = 0), 10-11 above (g = 3)
    const unsigned mLR = __ballot_sync(0xffffffffu, (vzLR & 16) != 0);
    const unsigned mBT = __ballot_sync(0xffffffffu, (vzBT & 16) != 0);
    if (k == 0) aguaF |= (mLR >> (4 * gl)) & 0xFu;
    if (k == 7) aguaF |= ((mLR >> (16 + 4 * gl)) & 0xFu) << 4;
    if (gl == 0) aguaF |= ((mBT >> (2 * k)) & 3u) << 8;
    if (gl == 3) aguaF |= ((mBT >> (16 + 2 * k)) & 3u) << 10;
    // coarse tile: columns from (ox-2)>>1, rows from (oy-2)>>1, 11x11 (x, 0 off water and off
    // the grid); the snapshot of every fine water cell, frame included, is x + P(x_coarse)
    float* ct = area;
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
      const int s = lane + 32 * kk;
      if (s < CT) ct[s] = cv[kk];
    }
    __syncwarp();
#pragma unroll
    for (int cr = 0; cr < 2; cr++)
#pragma unroll
      for (int m = 0; m < 4; m++)
        if (v[cr][m] & 16) x[cr][m] += correcaoGrossa(ct, cx0, cy0, ox + 2 * k + ((cr + 1 + m) & 1), oy + 4 * gl + m);
#pragma unroll
    for (int m = 0; m < 4; m++) {
      const int gy = oy + 4 * gl + m;
      if (aguaF >> m & 1) f.esq[m] += correcaoGrossa(ct, cx0, cy0, ox - 1, gy);
      if (aguaF >> (4 + m) & 1) f.dir[m] += correcaoGrossa(ct, cx0, cy0, ox + 16, gy);
    }
#pragma unroll
    for (int j = 0; j < 2; j++) {
      const int gx = ox + 2 * k + j;
      if (aguaF >> (8 + j) & 1) f.bai[j] += correcaoGrossa(ct, cx0, cy0, gx, oy - 1);
      if (aguaF >> (10 + j) & 1) f.cim[j] += correcaoGrossa(ct, cx0, cy0, gx, oy + 16);
    }
    __syncwarp();
  }
  // a block with no cell to update (air, solid, walled-in water) keeps its values: the warp skips
  // the sweeps (fmaf(0, d, q) = q for every cell of the block)
  bool mexe = false;
#pragma unroll
  for (int cr = 0; cr < 2; cr++)
#pragma unroll
    for (int m = 0; m < 4; m++) mexe |= (v[cr][m] & 16) && (v[cr][m] & 15);
  if (__any_sync(0xffffffffu, mexe)) varrerReg(x, v, bq, f, ordem, a.bloco != 0, a.varreduras);
  if (MODO == M_JUNTAR) {
    const float inv = 1.0f / ru.escala;
    float rv[2][4], zv[2][4];
    int lb[2][4];
    // the warp-uniform tests (bubbles, a previous z) outside the loads, so each group of loads
    // is straight-line code in flight together
#pragma unroll
    for (int cr = 0; cr < 2; cr++)
#pragma unroll
      for (int m = 0; m < 4; m++) rv[cr][m] = __ldcg(a.d.r + (cel[cr][m] < 0 ? 0 : cel[cr][m]));
    // a cell's own label is set only on bubble air (V0_BOLHA in its mask): loaded there alone
#pragma unroll
    for (int cr = 0; cr < 2; cr++)
#pragma unroll
      for (int m = 0; m < 4; m++)
        lb[cr][m] = (v[cr][m] & V0_BOLHA) ? (int)(__ldcg(a.rotB + cel[cr][m]) & 0xfff) : 0;
    if (ru.zVelho) {
#pragma unroll
      for (int cr = 0; cr < 2; cr++)
#pragma unroll
        for (int m = 0; m < 4; m++) zv[cr][m] = __ldcg(ru.zVelho + (cel[cr][m] < 0 ? 0 : cel[cr][m]));
    } else {
#pragma unroll
      for (int cr = 0; cr < 2; cr++)
#pragma unroll
        for (int m = 0; m < 4; m++) zv[cr][m] = 0.0f;
    }
    unsigned cels[2][4];
#pragma unroll
    for (int cr = 0; cr < 2; cr++)
#pragma unroll
      for (int m = 0; m < 4; m++) cels[cr][m] = lb[cr][m] ? __ldcg(a.d.celsB + lb[cr][m]) : 1u;
    // a bubble cell's share of z goes to its bubble's fixed-point sum; the lane adds its
    // consecutive cells of one bubble before the atomic (integer sums: same result)
    int labA = 0;
    long long acc = 0;
#pragma unroll
    for (int cr = 0; cr < 2; cr++)
#pragma unroll
      for (int m = 0; m < 4; m++) {
        const int c = cel[cr][m];
        if (c < 0) continue;
        const float xz = carregar(guardar<T>((v[cr][m] & 16) ? x[cr][m] : 0.0f)) * inv;
        if (lb[cr][m]) {
          const long long q = __double2ll_rn((double)xz / cels[cr][m] * ESC);
          if (lb[cr][m] != labA) {
            if (labA && acc) atomicAdd((unsigned long long*)&a.accZ[labA], (unsigned long long)acc);
            labA = lb[cr][m];
            acc = 0;
          }
          acc += q;
          ru.zNovo[c] = 0.0f;
          continue;
        }
        ru.zNovo[c] = xz;
        if (v[cr][m] & V0_AGUA) {
          s0 += (double)rv[cr][m] * (double)xz;
          if (ru.zVelho) s1 += (double)rv[cr][m] * (double)zv[cr][m];
        }
      }
    if (labA && acc) atomicAdd((unsigned long long*)&a.accZ[labA], (unsigned long long)acc);
  } else {
#pragma unroll
    for (int cr = 0; cr < 2; cr++)
#pragma unroll
      for (int m = 0; m < 4; m++)
        if (cel[cr][m] >= 0) dst[cel[cr][m]] = guardar<T>((v[cr][m] & 16) ? x[cr][m] : 0.0f);
  }
}

template <class T, int MODO>
__device__ __noinline__ void faseSuavizarT(const Args& a, int l, int desl, int ordem, bool paraTmp, float* areas,
                                           const Reuniao& ru, double* sh) {
  const NivelF n = s_niv[l];
  const int nbx = (n.nx + desl + 15) >> 4, nby = (n.ny + desl + 15) >> 4;
  const int nb = nbx * nby;
  const int w = threadIdx.x >> 5;
  float* area = areas + w * SUAV_W;
  const T* src = (const T*)(paraTmp ? n.x : n.tmp);
  T* dst = (T*)(paraTmp ? n.tmp : n.x);
  NivelF g{};
  if (MODO == M_PROL) g = s_niv[l + 1];
  const float* xcSecao = (MODO == M_PROL && l + 1 == a.Lc) ? a.xc : nullptr;
  double s0 = 0.0, s1 = 0.0;
  // with more blocks than warps (exc > 0), the warps that take two blocks take the last 2 exc
  // blocks of the row-major order, the top rows: air above the water in a tank, whose blocks
  // skip their sweeps, so the pass lasts about one water block
  const int tot = WARPS * gridDim.x, exc = nb - tot;
  const int tw = w * gridDim.x + blockIdx.x;  // the warp's first block index
  auto blocoDe = [&](int t) { return exc > 0 ? nb - 1 - (t + exc) % nb : t; };
  if (a.sol[l]) {
    // Blocks of wall alone are skipped: their cells hold x = 0 in both snapshots (zeroed before
    // the solve, and a pass writes 0 off water) and b = 0, so a pass would rewrite the same
    // zeros.  The flags of the warp's first 32 blocks come in one load, lane k's for its k-th.
    const uint8_t* fl = a.sol[l] + (desl ? blocosNivel(n.nx, n.ny, 0) : 0);
    const int tk = tw + (threadIdx.x & 31) * tot;
    const unsigned paredes = __ballot_sync(0xffffffffu, tk < nb && ldcg8(fl + blocoDe(tk)) != 0);
    int k = 0;
    for (int t = tw; t < nb; t += tot, k++) {
      const int blk = blocoDe(t);
      if (k < 32 ? (paredes >> k) & 1u : ldcg8(fl + blk) != 0) continue;
      suavizarBloco<T, MODO>(a, n, blk, nbx, desl, ordem, src, dst, area, g, xcSecao, ru, s0, s1);
    }
  } else {
    for (int t = tw; t < nb; t += tot)
      suavizarBloco<T, MODO>(a, n, blocoDe(t), nbx, desl, ordem, src, dst, area, g, xcSecao, ru, s0, s1);
  }
  if (MODO == M_JUNTAR) {
    const double t0 = somaBloco(s0, sh);
    const double t1 = somaBloco(s1, sh);
    if (threadIdx.x == 0) {
      a.parc[blockIdx.x * NPARC + 0] = t0;
      a.parc[blockIdx.x * NPARC + 1] = t1;
    }
  }
}

// Every grid level below the coarse section is stored as T (criarFundido), so a 16-bit kernel
// carries no FP32 copy of the passes: smaller code, which each phase enters cold.
template <class T>
__device__ void faseSuavizar(const Args& a, int l, int desl, int ordem, bool paraTmp, int modo, float* areas, int meia,
                             const Reuniao& ru, double* sh) {
  (void)meia;
  {
    switch (modo) {
      case M_PROL: faseSuavizarT<T, M_PROL>(a, l, desl, ordem, paraTmp, areas, ru, sh); break;
      case M_ZERO: faseSuavizarT<T, M_ZERO>(a, l, desl, ordem, paraTmp, areas, ru, sh); break;
      case M_ESPALHAR: faseSuavizarT<T, M_ESPALHAR>(a, l, desl, ordem, paraTmp, areas, ru, sh); break;
      case M_JUNTAR: faseSuavizarT<T, M_JUNTAR>(a, l, desl, ordem, paraTmp, areas, ru, sh); break;
      default: faseSuavizarT<T, M_NORMAL>(a, l, desl, ordem, paraTmp, areas, ru, sh);
    }
  }
}

// ---------------------------------------------------------------- restriction
// restringir (js/pressao-cpu.js:159-188) as a gather, one warp per region of R coarse rows x 32
// columns: the fine footprint (x on 2R+4 rows x 68 columns; b and flags on 2R+2 x 66) is staged
// in the warp's shared area, residuals computed once, then each lane sums its 4x4 windows.
template <class TFino, int R>
__device__ __forceinline__ void faseRestringirR(const Args& a, int l, float* areas) {
  constexpr int RXn = (2 * R + 4) * 68, RBn = (2 * R + 2) * 66;
  constexpr int KX = (RXn + 31) / 32, KB = (RBn + 31) / 32;
  static_assert(RXn + 3 * RBn <= REST_W, "restriction staging area");
  const NivelF f = s_niv[l];
  const NivelF g = s_niv[l + 1];
  const bool secao = l + 1 == a.Lc;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  float* xs = areas + w * REST_W;
  float* bs = xs + RXn;
  float* rs = bs + RBn;
  uint8_t* vs = (uint8_t*)(rs + RBn);
  const float pes[4] = {0.25f, 0.75f, 0.75f, 0.25f};
  const int nseg = (g.nx + 31) >> 5;
  const int total = nseg * ((g.ny + R - 1) / R);
  // A region whose coarse cells lie in wall blocks of the coarse level (its shift-0 flags; its
  // 32 columns span two blocks, its rows one) is skipped: those cells keep b = 0.  The flags of
  // the warp's first 32 regions come in one load, lane k's for its k-th.
  const uint8_t* flg = a.sol[l + 1];
  const int gbx = (g.nx + 15) >> 4;
  auto paredeReg = [&](int seg) {
    const int by = ((seg / nseg) * R) >> 4, bx = ((seg % nseg) * 32) >> 4;
    return ldcg8(flg + by * gbx + bx) != 0 && (bx + 1 >= gbx || ldcg8(flg + by * gbx + bx + 1) != 0);
  };
  const int t0 = w * gridDim.x + blockIdx.x, tot = WARPS * gridDim.x;
  unsigned paredes = 0;
  if (flg) {
    const int tk = t0 + lane * tot;
    paredes = __ballot_sync(0xffffffffu, tk < total && paredeReg(tk));
  }
  int kr = 0;
  for (int seg = t0; seg < total; seg += tot, kr++) {
    if (flg && (kr < 32 ? (paredes >> kr) & 1u : paredeReg(seg))) continue;
    const int J0 = (seg / nseg) * R, I0 = (seg % nseg) * 32;
    const int fi0 = 2 * I0 - 2, fj0 = 2 * J0 - 2;  // x window origin (fine)
    const int I = I0 + lane;
    int gvz[R];
#pragma unroll
    for (int r = 0; r < R; r++) gvz[r] = (I < g.nx && J0 + r < g.ny) ? ldcg8(g.viz + I + (J0 + r) * g.nx) : 0;
    // staging loads issued as one batch per array (registers, then shared memory)
    {
      float xv[KX];
#pragma unroll
      for (int k = 0; k < KX; k++) {
        const int s = lane + 32 * k;
        const int i = fi0 + s % 68, j = fj0 + s / 68;
        xv[k] = (s < RXn && i >= 0 && j >= 0 && i < f.nx && j < f.ny) ? carregar(ldcg((const TFino*)f.x + i + j * f.nx)) : 0.0f;
      }
      float bv[KB];
      int vv[KB];
#pragma unroll
      for (int k = 0; k < KB; k++) {
        const int s = lane + 32 * k;
        const int i = fi0 + 1 + s % 66, j = fj0 + 1 + s / 66;
        const bool d = s < RBn && i >= 0 && j >= 0 && i < f.nx && j < f.ny;
        const int c = i + j * f.nx;
        vv[k] = d ? ldcg8(f.viz + c) : 0;
        bv[k] = d ? carregar(ldcg((const TFino*)f.b + c)) : 0.0f;
      }
#pragma unroll
      for (int k = 0; k < KX; k++) {
        const int s = lane + 32 * k;
        if (s < RXn) xs[s] = xv[k];
      }
#pragma unroll
      for (int k = 0; k < KB; k++) {
        const int s = lane + 32 * k;
        if (s < RBn) {
          vs[s] = (uint8_t)vv[k];
          bs[s] = bv[k];
        }
      }
    }
    __syncwarp();
    {
      // residuals of the fine cells: every shared load of the lane's cells goes out before the
      // first store.  x is 0 off water and outside the grid, so the neighbour sum needs no
      // mask (but TQ_PRECOND_BLOCK's coarse masks can close a face between two water cells);
      // the residual is 0 off water.
      const bool masc = a.bloco != 0;
      float rv[KB];
#pragma unroll
      for (int k = 0; k < KB; k++) {
        const int s = lane + 32 * k < RBn ? lane + 32 * k : 0;
        const float* xc = xs + (s / 66 + 1) * 68 + s % 66 + 1;
        const int vz = vs[s];
        const float t = masc ? ((((vz & 1) ? xc[-1] : 0.0f) + ((vz & 2) ? xc[1] : 0.0f)) + ((vz & 4) ? xc[-68] : 0.0f)) +
                                   ((vz & 8) ? xc[68] : 0.0f)
                             : ((xc[-1] + xc[1]) + xc[-68]) + xc[68];
        rv[k] = (vz & 16) ? bs[s] - ((float)__popc(vz & 15) * xc[0] - t) : 0.0f;
      }
#pragma unroll
      for (int k = 0; k < KB; k++)
        if (lane + 32 * k < RBn) rs[lane + 32 * k] = rv[k];
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < R; r++)
      if (I < g.nx && J0 + r < g.ny) {
        const int C = I + (J0 + r) * g.nx;
        float soma = 0.0f;
        if (gvz[r] & 16) {
#pragma unroll
          for (int bb = 0; bb < 4; bb++)
#pragma unroll
            for (int aa = 0; aa < 4; aa++) soma += rs[(2 * r + bb) * 66 + 2 * lane + aa] * (pes[aa] * pes[bb]);
        }
        if (secao) a.bc[C] = soma;
        else gravarN(g.meia, g.b, C, soma);  // x of the coarse level: its first pass reads 0
      }
    __syncwarp();
  }
}

// Two coarse rows per warp where one-row segments would take four or more rounds of the
// grid's warps (the finest restriction of a large atlas): half the rounds, each with the 6
// residual rows of 2 coarse rows instead of 2 x 4.
template <class TFino>
__device__ void faseRestringir(const Args& a, int l, float* areas) {
  const NivelF g = s_niv[l + 1];
  if (((g.nx + 31) >> 5) * g.ny > 4 * WARPS * (int)gridDim.x) faseRestringirR<TFino, 2>(a, l, areas);
  else faseRestringirR<TFino, 1>(a, l, areas);
}

// ---------------------------------------------------------------- coarse section (CTA 0)
// Level arrays live in CTA 0's dynamic shared memory and are addressed by offsets from the
// `extern __shared__` array, so every access compiles to a shared-memory access.
struct NivelS {
  int nx, ny;
  int xa, xb, b;  // float offsets
  int v;          // byte offset
};

// One smoother pass over a level held in shared memory: the level's 16x16 blocks are taken in
// turn by the CTA's warps, each sweeping its block in registers (varrerReg) from the snapshot
// `src` and writing `dst`.
__device__ void passoS(float* F, const uint8_t* U, const NivelS n, int desl, int ordem, int src, int dst, bool masc,
                       int nVarr) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, gl = lane >> 3, k = lane & 7;
  const int nx = n.nx, ny = n.ny;
  const int nbx = (nx + desl + 15) >> 4, nby = (ny + desl + 15) >> 4;
  for (int blk = w; blk < nbx * nby; blk += WARPS) {
    const int ox = (blk % nbx) * 16 - desl, oy = (blk / nbx) * 16 - desl;
    float x[2][4], bq[2][4];  // [colour][m], see meiaReg
    int v[2][4], cel[2][4];
    Moldura f;
#pragma unroll
    for (int cr = 0; cr < 2; cr++)
#pragma unroll
      for (int m = 0; m < 4; m++) {
        const int gx = ox + 2 * k + ((cr + 1 + m) & 1), gy = oy + 4 * gl + m;
        const bool dentro = gx >= 0 && gy >= 0 && gx < nx && gy < ny;
        const int c = gx + gy * nx;
        cel[cr][m] = dentro ? c : -1;
        v[cr][m] = dentro ? (U[n.v + c] | 128) : 0;
        x[cr][m] = dentro ? F[src + c] : 0.0f;
        bq[cr][m] = dentro ? F[n.b + c] : 0.0f;
      }
#pragma unroll
    for (int m = 0; m < 4; m++) {
      const int gy = oy + 4 * gl + m;
      const bool okL = k == 0 && ox - 1 >= 0 && gy >= 0 && gy < ny;
      const bool okR = k == 7 && ox + 16 < nx && gy >= 0 && gy < ny;
      f.esq[m] = okL ? F[src + ox - 1 + gy * nx] : 0.0f;
      f.dir[m] = okR ? F[src + ox + 16 + gy * nx] : 0.0f;
    }
#pragma unroll
    for (int j = 0; j < 2; j++) {
      const int gx = ox + 2 * k + j;
      const bool okB = gl == 0 && gx >= 0 && gx < nx && oy - 1 >= 0;
      const bool okT = gl == 3 && gx >= 0 && gx < nx && oy + 16 < ny;
      f.bai[j] = okB ? F[src + gx + (oy - 1) * nx] : 0.0f;
      f.cim[j] = okT ? F[src + gx + (oy + 16) * nx] : 0.0f;
    }
    varrerReg(x, v, bq, f, ordem, masc, nVarr);
#pragma unroll
    for (int cr = 0; cr < 2; cr++)
#pragma unroll
      for (int m = 0; m < 4; m++)
        if (cel[cr][m] >= 0) F[dst + cel[cr][m]] = (v[cr][m] & 16) ? x[cr][m] : 0.0f;
  }
  __syncthreads();
}

// The coarsest solve (resolverGrosso, js/pressao-cpu.js:217-238) is VARREDURAS_GROSSO
// red-black sweeps from x = 0: a linear map of the right side, fixed for the whole PCG solve
// because the cell types are.  CTA 0 builds that map once per solve: column j is the sweeps
// applied to b = e_j, every thread of the first nL sweeping its own column (stored at
// M[i * nL + j], so a warp touches consecutive words).  Each V-cycle then applies it as a
// matrix-vector product.  Leaves the header count > DENSO_MAX when the level has more changing
// cells, and the section keeps the sweeps.
struct Denso {
  float* M;
  int* celula;  // cell | free-neighbour mask << 24, colour 0 first
  int* viz4;    // list index of each free neighbour (left, right, down, up) or -1
  float* inv;   // 1/k
  int* cab;     // [0] count, [1] count of colour 0
};
__device__ __forceinline__ Denso denso(unsigned char* dyn, int off) {
  Denso z;
  z.M = (float*)(dyn + off);
  z.celula = (int*)(z.M + DENSO_MAX * DENSO_MAX);
  z.viz4 = z.celula + DENSO_MAX;
  z.inv = (float*)(z.viz4 + 4 * DENSO_MAX);
  z.cab = (int*)(z.inv + DENSO_MAX);
  return z;
}

__device__ __noinline__ void montarDenso(const Args& a, unsigned char* dyn) {
  const Denso z = denso(dyn, a.offDenso);
  const NivelF n = s_niv[a.L - 1];
  const int nx = n.nx, N = n.nx * n.ny;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int* mapa = (int*)z.M;  // cell -> list index, while the matrix is not written yet
  if (w == 0) {
    int base = 0, n0 = 0;
    for (int cor = 0; cor < 2; cor++) {
      for (int c0 = 0; c0 < N; c0 += 32) {
        const int c = c0 + lane;
        const bool minha = c < N && ((((c % nx) + (c / nx) + 1) & 1) == cor);
        const int vz = minha ? ldcg8(n.viz + c) : 0;
        const bool ok = minha && (vz & 16) && (vz & 15);
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        const int pos = base + __popc(m & ((1u << lane) - 1u));
        if (minha) mapa[c] = ok ? pos : -1;
        if (ok && pos < DENSO_MAX) z.celula[pos] = c | ((vz & 15) << 24);
        base += __popc(m);
      }
      if (cor == 0) n0 = base;
    }
    if (lane == 0) {
      z.cab[0] = base;
      z.cab[1] = n0;
    }
  }
  __syncthreads();
  const int nL = z.cab[0];
  if (nL > DENSO_MAX) return;
  for (int i = threadIdx.x; i < nL; i += TF) {
    const int e = z.celula[i], c = e & 0xffffff, mk = e >> 24;
    z.viz4[4 * i + 0] = (mk & 1) ? mapa[c - 1] : -1;
    z.viz4[4 * i + 1] = (mk & 2) ? mapa[c + 1] : -1;
    z.viz4[4 * i + 2] = (mk & 4) ? mapa[c - nx] : -1;
    z.viz4[4 * i + 3] = (mk & 8) ? mapa[c + nx] : -1;
    z.inv[i] = inversoVizinhos(__popc(mk));
  }
  __syncthreads();
  for (int k = threadIdx.x; k < nL * nL; k += TF) z.M[k] = 0.0f;
  __syncthreads();
  const int j = threadIdx.x;
  if (j < nL) {
    const int n0 = z.cab[1];
    for (int k = 0; k < VARREDURAS_GROSSO; k++)
      for (int o = 0; o < 2; o++) {
        const int cor = (k & 1) ? 1 - o : o;
        const int i0 = cor ? n0 : 0, i1 = cor ? nL : n0;
        for (int i = i0; i < i1; i++) {
          float t = 0.0f;
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const int v = z.viz4[4 * i + q];
            t += v >= 0 ? z.M[v * nL + j] : 0.0f;
          }
          z.M[i * nL + j] = (t + (i == j ? 1.0f : 0.0f)) * z.inv[i];
        }
      }
  }
  __syncthreads();
}

// x = M b on the coarsest level (one warp per row, lanes over the row, fixed-order warp sum).
__device__ void aplicarDenso(const Denso& z, float* F, int xa, int b) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nL = z.cab[0];
  for (int i = w; i < nL; i += WARPS) {
    float s = 0.0f;
    for (int j = lane; j < nL; j += 32) s += z.M[i * nL + j] * F[b + (z.celula[j] & 0xffffff)];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) F[xa + (z.celula[i] & 0xffffff)] = s;
  }
}

// Stamp of the coarse-section trace (CTA 0, thread 0, when tracing).
__device__ __forceinline__ void marcaSecao(const Args& a, bool marcar = true) {
  if (marcar && a.perfil && threadIdx.x == 0) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    unsigned long long* base = a.perfil + PERFIL_MAX + 1;
    unsigned long long k = base[0]++;
    if (k < PERFIL_SECAO) base[1 + k] = t;
  }
}

// Levels Lc..L-1 of the V-cycle inside CTA 0: loads b of level Lc (a.bc), runs the down
// passes and restrictions, the coarsest red-black solve (one warp), the prolongations and up
// passes, and stores x of level Lc (a.xc).
__device__ __noinline__ void secaoGrossa(const Args& a, unsigned char* smem, NivelS* s, int* tileOff, int coluna) {
  const bool marcar = coluna < 0 && blockIdx.x == 0;
  float* F = (float*)smem;
  uint8_t* U = smem;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  marcaSecao(a, marcar);
  if (threadIdx.x == 0) {
    int off = 0;  // bytes
    for (int l = a.Lc; l < a.L; l++) {
      const NivelF n = s_niv[l];
      const int N = n.nx * n.ny;
      NivelS& t = s[l];
      t.nx = n.nx;
      t.ny = n.ny;
      t.xa = off / 4;
      off += (N * 4 + 15) & ~15;
      t.xb = off / 4;
      off += (N * 4 + 15) & ~15;
      t.b = off / 4;
      off += (N * 4 + 15) & ~15;
      t.v = off;
      off += (N + 15) & ~15;
    }
    *tileOff = off;
  }
  __syncthreads();
  const int celJ = coluna >= 0 ? __ldcg(a.wSecao + coluna) : -1;  // column build: b = unit vector
  for (int l = a.Lc; l < a.L; l++) {
    const NivelS t = s[l];
    const uint8_t* viz = s_niv[l].viz;
    const int N = t.nx * t.ny;
    for (int c0 = 0; c0 < N; c0 += 4 * TF) {  // loads in batches of 4 per thread
      int vv[4];
      float bb[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int c = c0 + threadIdx.x + k * TF;
        vv[k] = c < N ? ldcg8(viz + c) : 0;
        bb[k] = (c < N && l == a.Lc) ? (coluna < 0 ? __ldcg(a.bc + c) : (c == celJ ? 1.0f : 0.0f)) : 0.0f;
      }
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int c = c0 + threadIdx.x + k * TF;
        if (c < N) {
          U[t.v + c] = (uint8_t)vv[k];
          F[t.xa + c] = 0.0f;
          if (l == a.Lc) F[t.b + c] = bb[k];
        }
      }
    }
  }
  __syncthreads();
  marcaSecao(a, marcar);
  const float pes[4] = {0.25f, 0.75f, 0.75f, 0.25f};
  // the block preconditioner's single pass (see cicloV) ends in xb: the level's two buffers swap
  // roles in this CTA's table (rebuilt at each call)
  auto trocarS = [&](int l) {
    if (threadIdx.x == 0) {
      const int t = s[l].xa;
      s[l].xa = s[l].xb;
      s[l].xb = t;
    }
    __syncthreads();
  };
  for (int l = a.Lc; l < a.L - 1; l++) {
    NivelS f = s[l];
    const NivelS g = s[l + 1];
    if (a.umaPassada) {
      passoS(F, U, f, 8, 0, f.xa, f.xb, a.bloco != 0, a.varreduras);
      trocarS(l);
      f = s[l];
    } else {
      passoS(F, U, f, 0, 0, f.xa, f.xb, a.bloco != 0, a.varreduras);
      marcaSecao(a, marcar);
      passoS(F, U, f, 8, 0, f.xb, f.xa, a.bloco != 0, a.varreduras);
    }
    marcaSecao(a, marcar);
    // restringir: residuals of the fine level into its free x buffer, then the 4x4 gathers.
    // Out-of-range and dry neighbours enter with weight or value 0, which adds +0 to a sum.
    {
      const int Nf = f.nx * f.ny;
      const float* x = F + f.xa;
      for (int c = threadIdx.x; c < Nf; c += TF) {
        const int vz = U[f.v + c];
        const float a0 = x[(vz & 1) ? c - 1 : c], a1 = x[(vz & 2) ? c + 1 : c];
        const float a2 = x[(vz & 4) ? c - f.nx : c], a3 = x[(vz & 8) ? c + f.nx : c];
        const float xc = x[c], bc = F[f.b + c];
        float t = 0.0f;
        t += (vz & 1) ? a0 : 0.0f;
        t += (vz & 2) ? a1 : 0.0f;
        t += (vz & 4) ? a2 : 0.0f;
        t += (vz & 8) ? a3 : 0.0f;
        F[f.xb + c] = (vz & 16) ? bc - ((float)__popc(vz & 15) * xc - t) : 0.0f;
      }
      __syncthreads();
      const float* r = F + f.xb;
      for (int C = threadIdx.x; C < g.nx * g.ny; C += TF) {
        const int I = C % g.nx, J = C / g.nx;
        float rv[16];
#pragma unroll
        for (int bb = 0; bb < 4; bb++) {
          const int j = min(max(2 * J - 1 + bb, 0), f.ny - 1);
#pragma unroll
          for (int aa = 0; aa < 4; aa++) rv[bb * 4 + aa] = r[min(max(2 * I - 1 + aa, 0), f.nx - 1) + j * f.nx];
        }
        float sum = 0.0f;
#pragma unroll
        for (int bb = 0; bb < 4; bb++) {
          const int j = 2 * J - 1 + bb;
#pragma unroll
          for (int aa = 0; aa < 4; aa++) {
            const int i = 2 * I - 1 + aa;
            const bool dentro = i >= 0 && j >= 0 && i < f.nx && j < f.ny;
            sum += dentro ? rv[bb * 4 + aa] * (pes[aa] * pes[bb]) : 0.0f;
          }
        }
        F[g.b + C] = (U[g.v + C] & 16) ? sum : 0.0f;
        F[g.xa + C] = 0.0f;
      }
    }
    __syncthreads();
    marcaSecao(a, marcar);
  }
  const bool comDenso = a.offDenso >= 0 && denso(smem, a.offDenso).cab[0] <= DENSO_MAX;
  if (comDenso) {
    const NivelS n = s[a.L - 1];
    aplicarDenso(denso(smem, a.offDenso), F, n.xa, n.b);
  } else if (s[a.L - 1].nx * s[a.L - 1].ny > GROSSO_UM_WARP || w == 0) {
    // resolverGrosso (js/pressao-cpu.js:217-238): one warp on a small level, every warp of the
    // CTA on a large one (a wide, flat coarsest level of a tank atlas)
    const bool todos = s[a.L - 1].nx * s[a.L - 1].ny > GROSSO_UM_WARP;
    const int P = todos ? WARPS : 1;
    auto sincronizar = [&]() {
      if (todos) __syncthreads();
      else __syncwarp();
    };
    const NivelS n = s[a.L - 1];
    const int nx = n.nx, N = n.nx * n.ny;
    float* x = F + n.xa;
    // The cells that change (water with a free neighbour), listed per colour in the free x
    // buffer as cell | mask << 24, colour 0 first, in cell order: each warp lists a slice of
    // the cells (a multiple of 32) at the offset of the slices before it.
    int* lista = (int*)(F + n.xb);
    __shared__ int contW[2][WARPS];
    const int fatia = ((N + P * 32 - 1) / (P * 32)) * 32;
    const int lo = min(w * fatia, N), hi = min(lo + fatia, N);
    auto muda = [&](int c, int cor) {
      const int vz = c < hi ? U[n.v + c] : 0;
      const bool ok = c < hi && (vz & 16) && (vz & 15) && ((((c % nx) + (c / nx) + 1) & 1) == cor);
      return ok ? (c | ((vz & 15) << 24)) : -1;
    };
#pragma unroll
    for (int cor = 0; cor < 2; cor++) {
      int k = 0;
      for (int c0 = lo; c0 < hi; c0 += 32) k += __popc(__ballot_sync(0xffffffffu, muda(c0 + lane, cor) >= 0));
      if (lane == 0) contW[cor][w] = k;
    }
    sincronizar();
    int cont[2] = {0, 0}, base[2] = {0, 0};
    for (int q = 0; q < P; q++)
#pragma unroll
      for (int cor = 0; cor < 2; cor++) {
        if (q == w) base[cor] = cont[cor];
        cont[cor] += contW[cor][q];
      }
    base[1] += cont[0];
#pragma unroll
    for (int cor = 0; cor < 2; cor++) {
      int b = base[cor];
      for (int c0 = lo; c0 < hi; c0 += 32) {
        const int e = muda(c0 + lane, cor);
        const unsigned m = __ballot_sync(0xffffffffu, e >= 0);
        if (e >= 0) lista[b + __popc(m & ((1u << lane) - 1u))] = e;
        b += __popc(m);
      }
    }
    sincronizar();
    const int t0 = todos ? threadIdx.x : lane, nt = P * 32;
    for (int k = 0; k < VARREDURAS_GROSSO; k++)
      for (int o = 0; o < 2; o++) {
        const int cor = (k & 1) ? 1 - o : o;
        const int ini = cor ? cont[0] : 0, n_ = cont[cor];
        for (int e0 = t0; e0 < n_; e0 += 2 * nt) {
          const int eA = e0, eB = e0 + nt;
          const int EA = lista[ini + eA], EB = eB < n_ ? lista[ini + eB] : -1;
          float va[5], vb[5];
          {
            const int c = EA & 0xffffff, mk = EA >> 24;
            va[0] = x[(mk & 1) ? c - 1 : c];
            va[1] = x[(mk & 2) ? c + 1 : c];
            va[2] = x[(mk & 4) ? c - nx : c];
            va[3] = x[(mk & 8) ? c + nx : c];
            va[4] = F[n.b + c];
          }
          {  // an idle entry (-1) reads cell 0
            const int c = EB < 0 ? 0 : EB & 0xffffff, mk = EB < 0 ? 0 : EB >> 24;
            vb[0] = x[(mk & 1) ? c - 1 : c];
            vb[1] = x[(mk & 2) ? c + 1 : c];
            vb[2] = x[(mk & 4) ? c - nx : c];
            vb[3] = x[(mk & 8) ? c + nx : c];
            vb[4] = F[n.b + c];
          }
          {
            const int mk = EA >> 24;
            float t = 0.0f;
            t += (mk & 1) ? va[0] : 0.0f;
            t += (mk & 2) ? va[1] : 0.0f;
            t += (mk & 4) ? va[2] : 0.0f;
            t += (mk & 8) ? va[3] : 0.0f;
            x[EA & 0xffffff] = (t + va[4]) * inversoVizinhos(__popc(mk));
          }
          if (EB >= 0) {
            const int mk = EB >> 24;
            float t = 0.0f;
            t += (mk & 1) ? vb[0] : 0.0f;
            t += (mk & 2) ? vb[1] : 0.0f;
            t += (mk & 4) ? vb[2] : 0.0f;
            t += (mk & 8) ? vb[3] : 0.0f;
            x[EB & 0xffffff] = (t + vb[4]) * inversoVizinhos(__popc(mk));
          }
        }
        sincronizar();
      }
  }
  __syncthreads();
  marcaSecao(a, marcar);
  for (int l = a.L - 2; l >= a.Lc; l--) {
    const NivelS g = s[l + 1];
    const NivelS f = s[l];
    // prolongar: coarse x is 0 on every dry coarse cell, out-of-range corners get weight 0
    for (int c = threadIdx.x; c < f.nx * f.ny; c += TF) {
      const int i = c % f.nx, j = c / f.nx;
      const int I0 = grossoBaseF(i), J0 = grossoBaseF(j);
      const float wx0 = pesoBaseF(i), wy0 = pesoBaseF(j);
      float gv[4];
#pragma unroll
      for (int b = 0; b < 2; b++) {
        const int J = min(max(J0 + b, 0), g.ny - 1);
#pragma unroll
        for (int aa = 0; aa < 2; aa++) gv[b * 2 + aa] = F[g.xa + min(max(I0 + aa, 0), g.nx - 1) + J * g.nx];
      }
      const float xf = F[f.xa + c];
      float e = 0.0f;
#pragma unroll
      for (int b = 0; b < 2; b++) {
        const int J = J0 + b;
        const float wy = b ? 1.0f - wy0 : wy0;
#pragma unroll
        for (int aa = 0; aa < 2; aa++) {
          const int I = I0 + aa;
          const bool dentro = I >= 0 && J >= 0 && I < g.nx && J < g.ny;
          e += dentro ? gv[b * 2 + aa] * ((aa ? 1.0f - wx0 : wx0) * wy) : 0.0f;
        }
      }
      if (U[f.v + c] & 16) F[f.xa + c] = xf + e;
    }
    __syncthreads();
    marcaSecao(a, marcar);
    passoS(F, U, f, 8, 1, f.xa, f.xb, a.bloco != 0, a.varreduras);
    if (a.umaPassada) {
      trocarS(l);
    } else {
      marcaSecao(a, marcar);
      passoS(F, U, f, 0, 1, f.xb, f.xa, a.bloco != 0, a.varreduras);
    }
    marcaSecao(a, marcar);
  }
  const NivelS t = s[a.Lc];
  const int Nc = t.nx * t.ny;
  if (coluna < 0) {
    for (int c = threadIdx.x; c < Nc; c += TF) a.xc[c] = F[t.xa + c];
  } else {  // column `coluna` of the section's matrix, rows = water cells of level Lc
    const int nW = __ldcg(a.nWp);
    for (int c = threadIdx.x; c < Nc; c += TF) {
      const int r = __ldcg(a.wInv + c);
      if (r >= 0) a.mSecao[(size_t)r * nW + coluna] = F[t.xa + c];
    }
  }
}

// x of level Lc = M b over its water cells, every CTA staging b in shared memory and each warp
// producing rows (lanes over the row, fixed-order warp sum).  Entries off water stay 0.
__device__ void aplicarSecaoDensa(const Args& a, unsigned char* dyn) {
  const int nW = __ldcg(a.nWp);
  float* bs = (float*)dyn;
  for (int j = threadIdx.x; j < nW; j += TF) bs[j] = __ldcg(a.bc + __ldcg(a.wSecao + j));
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (int i = (threadIdx.x >> 5) * gridDim.x + blockIdx.x; i < nW; i += WARPS * gridDim.x) {
    const float* Mi = a.mSecao + (size_t)i * nW;
    float sm = 0.0f;
#pragma unroll 8
    for (int j = lane; j < nW; j += 32) sm += __ldcg(Mi + j) * bs[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sm += __shfl_xor_sync(0xffffffffu, sm, o);
    if (lane == 0) a.xc[__ldcg(a.wSecao + i)] = sm;
  }
}

// ---------------------------------------------------------------- the V-cycle
// After a single smoother pass (x -> tmp) the pass's output becomes the level's x: every CTA
// swaps the two snapshots in its own copy of the level table, at the same point of the solve.
// The barrier that follows (it opens with __syncthreads) publishes the swap to the CTA.
__device__ __forceinline__ void trocarXTmp(int l) {
  __syncthreads();
  if (threadIdx.x == 0) {
    void* t = s_niv[l].x;
    s_niv[l].x = s_niv[l].tmp;
    s_niv[l].tmp = t;
  }
}

// cicloV (js/pressao-cpu.js:241-255) between the spread of the residual (first pass) and the
// gather of z (last pass): 5 Lc + 1 phases, each ending at a grid barrier.  With
// TQ_PRECOND_BLOCK_1 the grid levels above 0 take one smoother pass a leg (shift 8, red-black
// down and black-red up, so the cycle stays symmetric): 3 Lc + 3 phases.
template <class T>
__device__ bool cicloV(const Args& a, unsigned& ep, float* areas, unsigned char* smem, NivelS* tabS, int* tileOff,
                       const Reuniao& ru, double* sh, bool secaoDensa) {
  for (int l = 0; l < a.Lc; l++) {
    const int meia = s_niv[l].meia;
    if (a.umaPassada && l >= 1) {
      faseSuavizar<T>(a, l, 8, 0, true, M_ZERO, areas, meia, ru, sh);
      trocarXTmp(l);
      if (!barreira(a, ep)) return false;
    } else {
      faseSuavizar<T>(a, l, 0, 0, true, l == 0 ? M_ESPALHAR : M_ZERO, areas, meia, ru, sh);
      if (!barreira(a, ep)) return false;
      faseSuavizar<T>(a, l, 8, 0, false, M_NORMAL, areas, meia, ru, sh);
      if (!barreira(a, ep)) return false;
    }
    faseRestringir<T>(a, l, areas);
    if (!barreira(a, ep)) return false;
  }
  if (secaoDensa) aplicarSecaoDensa(a, smem);
  else if (blockIdx.x == 0) secaoGrossa(a, smem, tabS, tileOff, -1);
  if (!barreira(a, ep)) return false;
  for (int l = a.Lc - 1; l >= 0; l--) {
    const int meia = s_niv[l].meia;
    faseSuavizar<T>(a, l, 8, 1, true, M_PROL, areas, meia, ru, sh);
    if (a.umaPassada && l >= 1) {
      trocarXTmp(l);
      if (!barreira(a, ep)) return false;
      continue;
    }
    if (!barreira(a, ep)) return false;
    faseSuavizar<T>(a, l, 0, 1, false, l == 0 ? M_JUNTAR : M_NORMAL, areas, meia, ru, sh);
    if (!barreira(a, ep)) return false;
  }
  return true;
}

// ---------------------------------------------------------------- PCG pieces
// A*v at water cell c (js/pressao-cpu.js:84-93 after difundir): neighbours that are water give
// val(n), active-bubble air gives valB(label), anything else 0.
template <class FV, class FB>
__device__ __forceinline__ float aplicarF(const Args& a, int c, FV val, FB valB) {
  const Dev& d = a.d;
  const int vz = ldcg8(a.vizOp + c);
  float s = 0.0f;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    if (!(vz & (1 << k))) continue;
    const int n = k == 0 ? c - 1 : k == 1 ? c + 1 : k == 2 ? c - d.nx : c + d.nx;
    const int t = ldcg8(d.tipo + n);
    if (t == AGUA) s += val(n);
    else if (a.bolhas && t == AR) {
      uint32_t r = __ldcg(d.rotulo + n);
      if (bolhaAtiva(a, r)) s += valB(r);
    }
  }
  return (float)__popc(vz & 15) * val(c) - s;
}

constexpr int KDA = 4;  // cells per thread per batch in [DA]

// [DA] of a PCG iteration over this CTA's cells: p = z + beta p (z alone on the first
// iteration), A p (js/pressao-cpu.js:84-93, bubble neighbours through their p), the partial of
// p.Ap (channel 0) and, for air of active bubbles, the sums over their water faces.  Cells go in
// batches of KDA per thread: descriptors first, then every z and p the batch needs.  z and p
// come through L1 (ld.ca): a warp's five loads of each share lines, which the L1 then serves
// instead of five L2 requests.  Both were last written before the grid barrier that opens this
// phase, whose acquire orders these loads after those writes as it does any other load (PTX
// memory model; the cache operator is a hint).  Measured on the 38,370x316 atlas: 109 against
// 170 us for the phase, with the bubble labels loaded only where the descriptor needs them and
// no stores off water.
__device__ __noinline__ void faseDA(const Args& a, const float* zc, const float* pv, float* pn, bool prim, float betaf,
                                    double beta, const double* pbVelho, double* sh) {
  const Dev& d = a.d;
  const int N = d.N, nx = d.nx;
  const int gt0 = blockIdx.x * TF + threadIdx.x, GT = gridDim.x * TF, lim = N;
  auto pbNovoV = [&](int b) {
    const double zb = zbDe(a, b);
    return prim ? zb : zb + beta * __ldcg(&pbVelho[b]);
  };
  double s = 0;
  for (int c0 = gt0; c0 < lim; c0 += KDA * GT) {
    int m[KDA];
#pragma unroll
    for (int k = 0; k < KDA; k++) {
      const int c = c0 + k * GT;
      m[k] = c < lim ? __ldcg(a.op + c) : 0;
    }
    float zv[KDA][5], pw[KDA][5];
    unsigned long long rl[KDA];
#pragma unroll
    for (int k = 0; k < KDA; k++) {
      // neighbour indices from the cell index alone, so these loads go out with the
      // descriptors' (the descriptor then picks the water neighbours, which are inside the
      // grid; an index across a row's end reads a value that no flag selects)
      const int c = c0 + k * GT < lim ? c0 + k * GT : 0;
      const int nb[5] = {c, c > 0 ? c - 1 : c, c < N - 1 ? c + 1 : c, c >= nx ? c - nx : c, c < N - nx ? c + nx : c};
#pragma unroll
      for (int q = 0; q < 5; q++) {
        zv[k][q] = __ldca(zc + nb[q]);
        pw[k][q] = prim ? 0.0f : __ldca(pv + nb[q]);
      }
    }
    // the packed labels of the bubble neighbours, only where the descriptor says a bubble is
    // next to the cell (most cells have none: 8 bytes a cell saved)
#pragma unroll
    for (int k = 0; k < KDA; k++)
      rl[k] = (a.bolhas && (m[k] & (OP_VIZ_BOLHA | OP_FACE))) ? __ldcg(a.rotB + c0 + k * GT) : 0ull;
#pragma unroll
    for (int k = 0; k < KDA; k++) {
      const int c = c0 + k * GT;
      if (c >= lim) continue;
      const int mk = m[k];
      float pq[5];
#pragma unroll
      for (int q = 0; q < 5; q++) pq[q] = prim ? zv[k][q] : zv[k][q] + betaf * pw[k][q];
      if (mk & OP_AGUA) {
        // water neighbours in the order left, right, down, up; air of an active bubble
        // contributes its bubble's p
        float sv = 0.0f;
#pragma unroll
        for (int q = 0; q < 4; q++) {
          if (mk & (1 << q)) sv += pq[q + 1];
          else if (mk & OP_VIZ_BOLHA) {  // neighbour q is air of an active bubble: that bubble's p
            const int r = (int)(rl[k] >> (12 + 12 * q)) & 0xfff;
            if (r) sv += (float)pbNovoV(r);
          }
        }
        const float apc = (float)(mk >> 8) * pq[0] - sv;
        pn[c] = pq[0];
        d.ap[c] = apc;
        s += (double)pq[0] * apc;
      } else {  // p and Ap off water are never read: nothing stored
        if (mk & OP_FACE) {  // the bubble's row: sum of p over its water faces
          double t = 0;
#pragma unroll
          for (int q = 0; q < 4; q++)
            if (mk & (1 << q)) t += (double)pq[q + 1];
          if (t != 0) somaFixa(&d.accB[(int)(rl[k] & 0xfff)], t, ESC);
        }
      }
    }
  }
  const double tb = somaBloco(s, sh);
  if (threadIdx.x == 0) a.parc[blockIdx.x * NPARC + 0] = tb;
}

// Per-tank sums of v^2 over the water cells of each tank of an atlas (tq_set_tanks) into destino:
// a warp-uniform loop over 32-cell segments; a segment inside one tank is reduced by shuffles and
// added with one FP64 atomic, a segment across tanks adds lane by lane.  Summation order varies
// with the schedule (FP64 rounding, far below the tolerance); every CTA later reads the same sums.
__device__ __noinline__ void somarPorTanque(const Args& a, const float* v, double* destino) {
  const Dev& d = a.d;
  const int N = d.N, GT = gridDim.x * TF, lane = threadIdx.x & 31;
  for (int c0 = blockIdx.x * TF + (threadIdx.x & ~31); c0 < N; c0 += GT) {
    const int c = c0 + lane;
    int t = -1;
    double x = 0.0;
    if (c < N && d.tipo[c] == AGUA) {
      t = tanqueDe(d, c);
      if (t >= 0) {
        x = (double)__ldcg(v + c);
        x *= x;
      }
    }
    const int t0 = __shfl_sync(0xffffffffu, t, 0);
    if (__all_sync(0xffffffffu, t == t0)) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane == 0 && t0 >= 0 && x != 0.0) atomicAdd(destino + t0, x);
    } else if (t >= 0 && x != 0.0) {
      atomicAdd(destino + t, x);
    }
  }
}

// Every tank's true residual within the tolerance of its own initial one: ||r_t||^2 = the water
// sums (d.rvT) plus the squared true rows of the tank's bubbles, against tol^2 ||r0_t||^2.  Thread
// t takes tanks t, t + TF, ..., adding its bubbles in the active list's order, so every CTA
// reaches the same answer from the same global values (the barrier before made them visible).
// Nothing is written here: every CTA reads d.rvT in this phase.  With `gravar` (CTA 0 alone,
// after the solve's last barrier) the totals go to d.rvT for tq_get_tank_residuals.
template <class FB>
__device__ bool tanquesConvergiram(const Args& a, int nAt, FB rbVerd, bool gravar = false) {
  const Dev& d = a.d;
  bool ok = true;
  for (int t = threadIdx.x; t < d.nTanques; t += TF) {
    double s = __ldcg(d.rvT + t);
    for (int k = 0; k < nAt; k++) {
      const int b = __ldcg(&a.ativos[k]);
      if (__ldcg(d.tanqueBolha + b) != t) continue;
      const double v = rbVerd(b);
      s += v * v;
    }
    const double r0 = __ldcg(d.r0T + t);
    ok = ok && s <= a.tol * a.tol * r0;
    if (gravar) d.rvT[t] = s;
  }
  return __syncthreads_and(ok) != 0;
}

// The true residual of a tolerance-mode solve, in FP64 from the FP64 iterate q64 and the bubble
// pressures yB: on water cells r = -div - A q (js/pressao-cpu.js:331-338, bubble neighbours
// through their y), written to d.r in FP32 (the replacement, when it comes to that) and summed
// squared into channel 0; on the interior air of active bubbles, the sum of q over the bubble's
// water faces into its fixed-point sum accV (the bubble row, :339-341, is finished after the
// next barrier).
__device__ __noinline__ void faseVerdade(const Args& a, double* sh) {
  const Dev& d = a.d;
  const int N = d.N, nx = d.nx;
  const int gt0 = blockIdx.x * TF + threadIdx.x, GT = gridDim.x * TF;
  double s = 0;
  // batches of KDA cells a thread, as in [DA]: descriptors, then the five q of each cell (through
  // L1, written before this phase's barrier) and its divergence, then the bubble labels where
  // the descriptor needs them
  for (int c0 = gt0; c0 < N; c0 += KDA * GT) {
    int m[KDA];
#pragma unroll
    for (int k = 0; k < KDA; k++) m[k] = c0 + k * GT < N ? __ldcg(a.op + c0 + k * GT) : 0;
    double qv[KDA][5];
    float dv[KDA];
#pragma unroll
    for (int k = 0; k < KDA; k++) {
      const int c = c0 + k * GT < N ? c0 + k * GT : 0;
      const int nb[5] = {c, c > 0 ? c - 1 : c, c < N - 1 ? c + 1 : c, c >= nx ? c - nx : c, c < N - nx ? c + nx : c};
#pragma unroll
      for (int q = 0; q < 5; q++) qv[k][q] = __ldca(a.q64 + nb[q]);
      dv[k] = __ldcg(d.div + c);
    }
    unsigned long long rl[KDA];
#pragma unroll
    for (int k = 0; k < KDA; k++)
      rl[k] = (a.bolhas && (m[k] & (OP_VIZ_BOLHA | OP_FACE))) ? __ldcg(a.rotB + c0 + k * GT) : 0ull;
#pragma unroll
    for (int k = 0; k < KDA; k++) {
      const int mk = m[k], c = c0 + k * GT;
      if (!(mk & (OP_AGUA | OP_FACE))) continue;
      if (mk & OP_AGUA) {
        double sv = 0;
#pragma unroll
        for (int q = 0; q < 4; q++) {
          if (mk & (1 << q)) sv += qv[k][q + 1];
          else if (mk & OP_VIZ_BOLHA) {
            const int r = (int)(rl[k] >> (12 + 12 * q)) & 0xfff;
            if (r) sv += __ldcg(d.yB + r);
          }
        }
        const double rt = -(double)dv[k] - ((double)(mk >> 8) * qv[k][0] - sv);
        d.r[c] = (float)rt;
        s += rt * rt;
      } else {
        double t = 0;
#pragma unroll
        for (int q = 0; q < 4; q++)
          if (mk & (1 << q)) t += qv[k][q + 1];
        if (t != 0) somaFixa(&a.accV[(int)(rl[k] & 0xfff)], t, ESC);
      }
    }
  }
  const double tb = somaBloco(s, sh);
  if (threadIdx.x == 0) {
    a.parc[blockIdx.x * NPARC + 0] = tb;
    a.parc[blockIdx.x * NPARC + 1] = 0.0;
  }
  if (d.nTanques) somarPorTanque(a, d.r, d.rvT);  // d.r holds the true residual now (FP32)
}

// The wall-block flags of the levels that have them (Args::sol), both shifts: one warp per
// block, 8 cells a lane; a block is wall when every cell of it in the grid is.
__device__ __noinline__ void marcarParedes(const Args& a) {
  const int lane = threadIdx.x & 31, wg = (threadIdx.x >> 5) * gridDim.x + blockIdx.x, nw = WARPS * gridDim.x;
  for (int l = 0; l < a.Lc; l++) {
    const NivelF n = s_niv[l];
    if (!a.sol[l]) continue;
    for (int desl = 0; desl <= 8; desl += 8) {
      const int nbx = (n.nx + desl + 15) >> 4, nb = blocosNivel(n.nx, n.ny, desl);
      uint8_t* fl = a.sol[l] + (desl ? blocosNivel(n.nx, n.ny, 0) : 0);
      for (int blk = wg; blk < nb; blk += nw) {
        const int ox = (blk % nbx) * 16 - desl, oy = (blk / nbx) * 16 - desl;
        const int gy = oy + (lane >> 1), gx0 = ox + (lane & 1) * 8;
        bool parede = true;
        for (int k = 0; k < 8; k++) {
          const int gx = gx0 + k;
          if (gx >= 0 && gy >= 0 && gx < n.nx && gy < n.ny) parede &= ldcg8(n.tipo + gx + gy * n.nx) == SOLIDO;
        }
        const bool todos = __all_sync(0xffffffffu, parede);
        if (lane == 0) fl[blk] = todos ? 1 : 0;
      }
    }
  }
}

// ---------------------------------------------------------------- the kernel
template <class T>
__global__ void __launch_bounds__(TF, 1) k_mgpcg(const __grid_constant__ Args a) {
  extern __shared__ __align__(16) unsigned char dyn[];
  __shared__ double sh[32];
  __shared__ NivelS tabS[MAX_NIVEIS];
  __shared__ int tileOff;
  float* areas = (float*)dyn;
  const Dev& d = a.d;
  const int N = d.N, nx = d.nx, ny = d.ny;
  const int gt0 = blockIdx.x * TF + threadIdx.x;
  const int GT = gridDim.x * TF;
  unsigned ep = 0;
  double somas[4];
  if (threadIdx.x < a.L) s_niv[threadIdx.x] = a.niv[threadIdx.x];
  __syncthreads();

  // ---- setup: level-0 preconditioner types, operator masks, bubble faces
  {
    uint8_t* t0 = s_niv[0].tipo;
    for (int c = gt0; c < N; c += GT) {
      const int t = d.tipo[c];
      const uint32_t rot = d.rotulo[c];
      // REFERENCE: enclosed air of a bubble is water to the V-cycle (js/pressao-cpu.js:305-308);
      // BLOCK: it stays air (free surface), the bubble rows take a Jacobi step instead
      t0[c] = (a.bolhas && !a.bloco && t == AR && rot >= 2) ? AGUA : (uint8_t)t;
      const int i = c % nx, j = c / nx;
      int m = 0;
      if (i > 0 && d.tipo[c - 1] != SOLIDO) m |= 1;
      if (i < nx - 1 && d.tipo[c + 1] != SOLIDO) m |= 2;
      if (j > 0 && d.tipo[c - nx] != SOLIDO) m |= 4;
      if (j < ny - 1 && d.tipo[c + nx] != SOLIDO) m |= 8;
      if (t == AGUA) m |= 16;
      a.vizOp[c] = (uint8_t)m;
      if (a.bolhas && t == AR && rot >= 2 && rot < (uint32_t)MAX_BOLHAS && i >= 1 && j >= 1 && i < nx - 1 &&
          j < ny - 1) {
        unsigned k = (d.tipo[c - 1] == AGUA) + (d.tipo[c + 1] == AGUA) + (d.tipo[c - nx] == AGUA) +
                     (d.tipo[c + nx] == AGUA);
        if (k) atomicAdd(&d.facesB[rot], k);
      }
    }
  }
  if (!barreira(a, ep)) return;
  // ---- coarse types (tiposGrossos, js/pressao-cpu.js:63-81), one level per phase
  for (int l = 1; l < a.L; l++) {
    const NivelF f = s_niv[l - 1];
    const NivelF g = s_niv[l];
    for (int C = gt0; C < g.nx * g.ny; C += GT) {
      const int I = C % g.nx, J = C / g.nx;
      bool ar = false, agua = false;
      for (int b = 0; b < 2; b++)
        for (int aa = 0; aa < 2; aa++) {
          int i = 2 * I + aa, j = 2 * J + b;
          if (i >= f.nx || j >= f.ny) continue;
          int t = ldcg8(f.tipo + i + j * f.nx);
          if (t == AR) ar = true;
          else if (t == AGUA) agua = true;
        }
      g.tipo[C] = ar ? AR : agua ? AGUA : SOLIDO;
    }
    if (!barreira(a, ep)) return;
  }
  // ---- neighbour masks of every level, bubble cell counts, active list, initial y
  for (int l = 0; l < a.L; l++) {
    const NivelF n = s_niv[l];
    for (int c = gt0; c < n.nx * n.ny; c += GT) {
      const int i = c % n.nx, j = c / n.nx;
      const uint8_t* tp = n.tipo;
      int m = 0;
      if (l >= 1 && a.bloco) {
        m = vizinhosPorFaces(s_niv[l - 1], n, i, j);
      } else {
        if (i > 0 && ldcg8(tp + c - 1) != SOLIDO) m |= 1;
        if (i < n.nx - 1 && ldcg8(tp + c + 1) != SOLIDO) m |= 2;
        if (j > 0 && ldcg8(tp + c - n.nx) != SOLIDO) m |= 4;
        if (j < n.ny - 1 && ldcg8(tp + c + n.nx) != SOLIDO) m |= 8;
      }
      if (ldcg8(tp + c) == AGUA) m |= 16;
      if (l == 0) {  // the descriptor's water and bubble-air bits (OP_AGUA, OP_BOLHA) for the
                     // spread and the gather; every other reader masks bits 0-4.  With BLOCK
                     // the V-cycle does not see bubbles: no cell spreads or gathers for one.
        const int t = d.tipo[c];
        if (t == AGUA) m |= V0_AGUA;
        else if (a.bolhas && !a.bloco && t == AR && bolhaAtiva(a, d.rotulo[c])) m |= V0_BOLHA;
      }
      n.viz[c] = (uint8_t)m;
    }
  }
  marcarParedes(a);
  for (int c = gt0; c < N; c += GT) {  // the operator descriptor (bubble faces are complete)
    const int i = c % nx, j = c / nx;
    const int t = d.tipo[c];
    int m = 0, livres = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const bool existe = k == 0 ? i > 0 : k == 1 ? i < nx - 1 : k == 2 ? j > 0 : j < ny - 1;
      if (!existe) continue;
      const int nb = k == 0 ? c - 1 : k == 1 ? c + 1 : k == 2 ? c - nx : c + nx;
      const int tn = d.tipo[nb];
      if (tn != SOLIDO) livres++;
      if (tn == AGUA) m |= 1 << k;
      else if (a.bolhas && tn == AR && bolhaAtiva(a, d.rotulo[nb])) m |= OP_VIZ_BOLHA;
    }
    if (t == AGUA) m |= OP_AGUA;
    if (a.bolhas && t == AR && bolhaAtiva(a, d.rotulo[c])) {
      m |= OP_BOLHA;
      if (i >= 1 && j >= 1 && i < nx - 1 && j < ny - 1) m |= OP_FACE;
    }
    a.op[c] = (uint16_t)(m | (livres << 8));
    if (d.nTanques && (m & OP_FACE)) d.tanqueBolha[d.rotulo[c] & 0xfffu] = tanqueDe(d, c);  // same for all its cells
    unsigned long long rl = 0;
    if (a.bolhas && (m & (OP_BOLHA | OP_VIZ_BOLHA))) {
      if (m & OP_BOLHA) rl = d.rotulo[c] & 0xfffu;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const bool existe = k == 0 ? i > 0 : k == 1 ? i < nx - 1 : k == 2 ? j > 0 : j < ny - 1;
        if (!existe) continue;
        const int nb = k == 0 ? c - 1 : k == 1 ? c + 1 : k == 2 ? c - nx : c + nx;
        if (d.tipo[nb] == AR && bolhaAtiva(a, d.rotulo[nb]))
          rl |= (unsigned long long)(d.rotulo[nb] & 0xfffu) << (12 + 12 * k);
      }
    }
    a.rotB[c] = rl;
  }
  if (a.bolhas) {
    for (int c = gt0; c < N; c += GT) {
      uint32_t b = d.rotulo[c];
      if (b >= 2 && b < (uint32_t)MAX_BOLHAS && d.tipo[c] == AR && __ldcg(&d.facesB[b]) > 0)
        atomicAdd(&d.celsB[b], 1u);
    }
    if (blockIdx.x == 0) {
      if (threadIdx.x < 32) {  // active labels in ascending order (one warp, ballot-compacted)
        int base = 0;
        for (int b0 = 0; b0 < MAX_BOLHAS; b0 += 32) {
          int b = b0 + threadIdx.x;
          bool at = b >= 2 && __ldcg(&d.facesB[b]) > 0;
          unsigned m = __ballot_sync(0xffffffffu, at);
          if (at) a.ativos[base + __popc(m & ((1u << threadIdx.x) - 1u))] = b;
          base += __popc(m);
        }
        if (threadIdx.x == 0) *a.nAtivos = base;
      }
      for (int b = threadIdx.x; b < MAX_BOLHAS; b += TF) {
        bool at = b >= 2 && __ldcg(&d.facesB[b]) > 0;
        d.yB[b] = at ? (double)d.yBolhaF[b] : 0.0;
        d.rb[b] = 0.0;
        d.zb[b] = a.zb2[b] = 0.0;
        d.pb[b] = a.pb2[b] = 0.0;
      }
    }
  } else if (blockIdx.x == 0 && threadIdx.x == 0) {
    *a.nAtivos = 0;
  }
  if (!barreira(a, ep)) return;
  const int nAt = a.bolhas ? __ldcg(a.nAtivos) : 0;

  // ---- r = -div - A q (js/pressao-cpu.js:331-338), bubble aq sums
  {
    double s = 0;
    for (int c = gt0; c < N; c += GT) {
      if (d.tipo[c] != AGUA) {
        d.q[c] = 0.0f;
        d.r[c] = 0.0f;
        continue;
      }
      float ar = aplicarF(a, c, [&](int n) { return __ldcg(d.q + n); },
                          [&](uint32_t r) { return (float)__ldcg(d.yB + r); });
      float rv = -d.div[c] - ar;
      d.r[c] = rv;
      if (a.q64) a.q64[c] = (double)d.q[c];
      s += (double)rv * rv;
    }
    if (a.bolhas)
      for (int c = gt0; c < N; c += GT) {
        const int i = c % nx, j = c / nx;
        if (i < 1 || j < 1 || i >= nx - 1 || j >= ny - 1) continue;
        uint32_t b = d.rotulo[c];
        if (d.tipo[c] != AR || !bolhaAtiva(a, b)) continue;
        double t = 0;
        if (d.tipo[c - 1] == AGUA) t += (double)__ldcg(d.q + c - 1);
        if (d.tipo[c + 1] == AGUA) t += (double)__ldcg(d.q + c + 1);
        if (d.tipo[c - nx] == AGUA) t += (double)__ldcg(d.q + c - nx);
        if (d.tipo[c + nx] == AGUA) t += (double)__ldcg(d.q + c + nx);
        if (t != 0) somaFixa(&d.accB[b], t, ESC);
      }
    double tb = somaBloco(s, sh);
    if (threadIdx.x == 0) {
      a.parc[blockIdx.x * NPARC + 0] = tb;
      a.parc[blockIdx.x * NPARC + 1] = 0.0;
    }
  }
  // the coarsest level's matrix (its neighbour masks are complete since the last barrier)
  if (blockIdx.x == 0 && a.offDenso >= 0) {
    montarDenso(a, dyn);
    if (a.secaoDensa) {  // every CTA will need it to build the section's columns
      const unsigned* src = (const unsigned*)(dyn + a.offDenso);
      for (int k = threadIdx.x; k < (int)(DENSO_BYTES / 4); k += TF) a.densoG[k] = src[k];
    }
  }
  if (a.secaoDensa && blockIdx.x == (gridDim.x > 1 ? 1 : 0) && threadIdx.x < 32) {
    // the water cells of level Lc, in cell order (one warp, ballot-compacted)
    const NivelF n = s_niv[a.Lc];
    const int Nc = n.nx * n.ny;
    int base = 0;
    for (int c0 = 0; c0 < Nc; c0 += 32) {
      const int c = c0 + threadIdx.x;
      const bool agua = c < Nc && (ldcg8(n.viz + c) & 16);
      const unsigned m = __ballot_sync(0xffffffffu, agua);
      const int pos = base + __popc(m & ((1u << threadIdx.x) - 1u));
      if (c < Nc) a.wInv[c] = agua ? pos : -1;
      if (agua) a.wSecao[pos] = c;
      base += __popc(m);
    }
    if (threadIdx.x == 0) *a.nWp = base;
  }
  if (!barreira(a, ep)) return;
  // each tank's ||r0||^2, water rows (r is complete since the barrier; read at the checks, many
  // barriers later)
  if (d.nTanques && a.q64) somarPorTanque(a, d.r, d.r0T);
  // rb = rhs - (faces*y - sum) (js/pressao-cpu.js:339-341); norm0
  auto rbInicial = [&](int b) {
    return (double)d.rhsBolhaF[b] - (__ldcg(&d.facesB[b]) * __ldcg(&d.yB[b]) - (double)__ldcg(&d.accB[b]) / ESC);
  };
  somasGlobais(a, nAt, [&](int b) { double v = rbInicial(b); return v * v; }, [](int) { return 0.0; }, sh, somas);
  const double norma0 = sqrt(somas[0] + somas[2]);
  if (blockIdx.x == 0) {
    for (int k = threadIdx.x; k < nAt; k += TF) {
      int b = __ldcg(&a.ativos[k]);
      d.rb[b] = rbInicial(b);
      if (d.nTanques && a.q64) {  // the bubble rows of each tank's ||r0||^2
        const int t = __ldcg(d.tanqueBolha + b);
        if (t >= 0) atomicAdd(d.r0T + t, d.rb[b] * d.rb[b]);
      }
    }
    if (threadIdx.x == 0) {
      d.esc->norma0 = d.esc->norma = norma0;
      d.esc->normas[0] = norma0;
      d.esc->iters = 0;
      d.esc->pronto = 0;
    }
  }
  if (!barreira(a, ep)) return;  // rb visible before spreading
  // ---- the section's matrix: every CTA builds its share of the columns with its own copy of
  // the coarsest level's matrix
  const bool secaoDensa = a.secaoDensa && a.iteracoes >= SECAO_DENSA_MIN_ITERS;
  if (secaoDensa) {
    unsigned* blocoDenso = (unsigned*)(dyn + a.offDenso);
    for (int k = threadIdx.x; k < (int)(DENSO_BYTES / 4); k += TF) blocoDenso[k] = __ldcg(a.densoG + k);
    __syncthreads();
    const int nW = __ldcg(a.nWp);
    for (int col = blockIdx.x; col < nW; col += gridDim.x) secaoGrossa(a, dyn, tabS, &tileOff, col);
    const NivelF nc = s_niv[a.Lc];
    for (int c = gt0; c < nc.nx * nc.ny; c += GT) a.xc[c] = 0.0f;  // off water, x of level Lc stays 0
    if (!barreira(a, ep)) return;
  }
  float escala = (a.escalar && norma0 > 0) ? (float)(1.0 / norma0) : 1.0f;
  if (blockIdx.x == 0)
    for (int b = threadIdx.x; b < MAX_BOLHAS; b += TF) {
      a.accZ[b] = 0;
      d.accB[b] = 0;
    }
  if (!cicloV<T>(a, ep, areas, dyn, tabS, &tileOff, Reuniao{escala, d.z, nullptr}, sh, secaoDensa)) return;
  int cz = 0, cp = 0;  // which of the two z / p buffers holds the latest values
  auto zbAtual = [&](int b) { return zbDe(a, b); };
  somasGlobais(a, nAt, [&](int b) { return __ldcg(&d.rb[b]) * zbAtual(b); }, [](int) { return 0.0; }, sh, somas);
  double rz = somas[0] + somas[2];
  double beta = 0.0;
  bool primeira = true;
  int itersFeitas = 0, trocas = 0;
  bool convergiu = false;
  double normaVerd = -1.0;
  double proxTroca = norma0 * FATOR_TROCA;  // the next residual replacement's threshold
  int proxVerif = 0;                          // with tanks: the next iteration that may check
  auto rbVerd = [&](int b) {  // a bubble's true row, from faseVerdade's sums
    return (double)d.rhsBolhaF[b] - (__ldcg(&d.facesB[b]) * __ldcg(&d.yB[b]) - (double)__ldcg(&a.accV[b]) / ESC);
  };

  for (int it = 0; it < a.iteracoes; it++) {
    float* zc = cz ? a.z2 : d.z;
    float* zo = cz ? d.z : a.z2;
    const float* pv = cp ? a.p2 : d.p;
    float* pn = cp ? d.p : a.p2;
    const double* zbOld = cz ? d.zb : a.zb2;
    double* zbCur = cz ? a.zb2 : d.zb;
    const double* pbVelho = cp ? a.pb2 : d.pb;
    double* pbNovo = cp ? d.pb : a.pb2;
    // ---- [DA] beta, p = z + beta p, A p, p.Ap, bubble rows
    if (!primeira) {
      somasGlobais(a, nAt, [&](int b) { return __ldcg(&d.rb[b]) * zbAtual(b); },
                   [&](int b) { return __ldcg(&d.rb[b]) * __ldcg(&zbOld[b]); }, sh, somas);
      const double rzNovo = somas[0] + somas[2], cruz = somas[1] + somas[3];
      beta = fabs(rz) < 1e-30 ? 0.0 : fmax(0.0, (rzNovo - cruz) / rz);
      rz = rzNovo;
    }
    const float betaf = (float)beta;
    const bool prim = primeira;
    auto pbNovoV = [&](int b) { return prim ? zbAtual(b) : zbAtual(b) + beta * __ldcg(&pbVelho[b]); };
    if (blockIdx.x == 0)
      for (int k = threadIdx.x; k < nAt; k += TF) {
        int b = __ldcg(&a.ativos[k]);
        zbCur[b] = zbAtual(b);
        pbNovo[b] = pbNovoV(b);
      }
    faseDA(a, zc, pv, pn, prim, betaf, beta, pbVelho, sh);
    if (!barreira(a, ep)) return;
    // ---- [B] alpha; q += alpha p, r -= alpha Ap; bubbles; r.r
    auto apbV = [&](int b) {
      return __ldcg(&d.facesB[b]) * __ldcg(&pbNovo[b]) - (double)__ldcg(&d.accB[b]) / ESC;
    };
    somasGlobais(a, nAt, [&](int b) { return __ldcg(&pbNovo[b]) * apbV(b); }, [](int) { return 0.0; }, sh, somas);
    const double pap = somas[0] + somas[2];
    const double alfa = fabs(pap) < 1e-30 ? 0.0 : rz / pap;
    {
      const float af = (float)alfa;
      double s = 0;
      for (int c0 = gt0; c0 < N; c0 += 4 * GT) {  // batches of 4 cells: all loads first
        int m[4];
        float qv[4], pnv[4], rv[4], apv[4];
        double qd[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const int c = c0 + k * GT < N ? c0 + k * GT : 0;
          m[k] = c0 + k * GT < N ? __ldcg(a.op + c) : 0;
          if (a.q64) qd[k] = __ldcg(a.q64 + c);
          else qv[k] = __ldcg(d.q + c);
          pnv[k] = __ldcg(pn + c);
          rv[k] = __ldcg(d.r + c);
          apv[k] = __ldcg(d.ap + c);
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
          if (!(m[k] & OP_AGUA)) continue;
          const int c = c0 + k * GT;
          if (a.q64) a.q64[c] = qd[k] + alfa * (double)pnv[k];
          else d.q[c] = qv[k] + af * pnv[k];
          const float r = rv[k] - af * apv[k];
          d.r[c] = r;
          s += (double)r * r;
        }
      }
      if (blockIdx.x == 0) {
        double sb = 0;
        for (int k = threadIdx.x; k < nAt; k += TF) {
          int b = __ldcg(&a.ativos[k]);
          d.yB[b] += alfa * __ldcg(&pbNovo[b]);
          double rbn = __ldcg(&d.rb[b]) - alfa * apbV(b);
          d.rb[b] = rbn;
          sb += rbn * rbn;
        }
        s += sb;
        for (int b = threadIdx.x; b < MAX_BOLHAS; b += TF) {
          a.accZ[b] = 0;
          if (a.q64) a.accV[b] = 0;
        }
        if (a.q64)
          for (int t = threadIdx.x; t < d.nTanques; t += TF) d.rvT[t] = 0.0;
      }
      double tb = somaBloco(s, sh);
      if (threadIdx.x == 0) a.parc[blockIdx.x * NPARC + 0] = tb;
    }
    if (!barreira(a, ep)) return;
    // ---- [C] norm, convergence, spread the residual
    somasGlobais(a, 0, [](int) { return 0.0; }, [](int) { return 0.0; }, sh, somas);
    double norma = sqrt(somas[0]);
    itersFeitas = it + 1;
    const bool ultima = it == a.iteracoes - 1;
    bool fim = ultima || (a.tol > 0 && norma <= a.tol * norma0);
    if (fim && !ultima && d.nTanques && it < proxVerif && norma > proxTroca) fim = false;
    if (a.q64 && (fim || norma <= proxTroca)) {
      // tolerance mode: the true residual of the FP64 iterate decides, and replaces the
      // recursive one unless the solve ends here
      proxVerif = it + VERIF_TANQUES;
      faseVerdade(a, sh);
      if (!barreira(a, ep)) return;
      somasGlobais(a, nAt, [&](int b) { const double v = rbVerd(b); return v * v; }, [](int) { return 0.0; }, sh, somas);
      normaVerd = sqrt(somas[0] + somas[2]);
      // with tanks, each tank's own residual decides; without, the whole grid's
      convergiu = d.nTanques ? tanquesConvergiram(a, nAt, rbVerd) : normaVerd <= a.tol * norma0;
      fim = convergiu || ultima;
      if (!fim) {
        // replacement: r (water) was rewritten by faseVerdade, the bubble rows follow; the
        // iteration goes on with the same search direction
        trocas++;
        proxTroca = normaVerd * FATOR_TROCA;
        norma = normaVerd;
        if (blockIdx.x == 0)
          for (int k = threadIdx.x; k < nAt; k += TF) {
            const int b = __ldcg(&a.ativos[k]);
            d.rb[b] = rbVerd(b);
          }
        if (!barreira(a, ep)) return;  // rb visible before the spread
      }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      if (it + 1 < 1024) d.esc->normas[it + 1] = norma;
      d.esc->iters = it + 1;
      d.esc->norma = norma;
      d.esc->pronto = fim ? 1 : 0;
    }
    if (fim) break;
    escala = (a.escalar && norma > 0) ? (float)(1.0 / norma) : 1.0f;
    if (blockIdx.x == 0)
      for (int b = threadIdx.x; b < MAX_BOLHAS; b += TF) d.accB[b] = 0;
    if (!cicloV<T>(a, ep, areas, dyn, tabS, &tileOff, Reuniao{escala, zo, zc}, sh, secaoDensa)) return;
    cz ^= 1;
    cp ^= 1;
    primeira = false;
  }
  // ---- end: q = 0 off water (the FP64 iterate rounded on water); bubbles hand back their
  // pressure; the solve's convergence record
  if (!barreira(a, ep)) return;
  for (int c = gt0; c < N; c += GT) {
    if (d.tipo[c] != AGUA) d.q[c] = 0.0f;
    else if (a.q64) d.q[c] = (float)__ldcg(a.q64 + c);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    Escalares* e = d.esc;
    const bool ok = a.q64 && convergiu;
    e->normaVerd = a.q64 ? normaVerd : -1.0;
    e->convergiu = ok ? 1 : 0;
    e->trocas = trocas;
    e->solves++;
    if (a.q64 && !ok) e->capados++;
    e->itersAcum += itersFeitas;
    e->trocasAcum += trocas;
    if (a.q64 && norma0 > 0 && normaVerd / norma0 > e->maxRel) e->maxRel = normaVerd / norma0;
  }
  if (blockIdx.x == 0 && d.nTanques && a.q64) tanquesConvergiram(a, nAt, rbVerd, true);  // each tank's total
  if (blockIdx.x == 0)
    for (int k = threadIdx.x; k < nAt; k += TF) {
      int b = __ldcg(&a.ativos[k]);
      d.yBolhaF[b] = (float)__ldcg(&d.yB[b]);
    }
}

// ---------------------------------------------------------------- host side
template <class T>
static void* kernelDe() { return (void*)k_mgpcg<T>; }

Fundido* criarFundido(Pcg* p) {
  if (p->L < 2) return nullptr;  // no coarse level to hand to the coarse section
  Fundido* f = new Fundido();
  // coarse section: the longest suffix of levels (not level 0) fitting the shared budget
  int Lc = p->L;
  size_t bytes = 0;
  for (int l = p->L - 1; l >= 1; l--) {
    size_t n = (size_t)p->nxL[l] * p->nyL[l];
    size_t b = 3 * ((n * 4 + 15) & ~(size_t)15) + ((n + 15) & ~(size_t)15);
    if (bytes + b > SMEM_GROSSO_MAX || (n > SECAO_MAX_CELULAS && l < p->L - 1)) break;
    bytes += b;
    Lc = l;
  }
  if (Lc >= p->L) {  // even the coarsest level does not fit
    delete f;
    return nullptr;
  }
  f->Lc = Lc;
  // 16-bit storage on every grid level below the coarse section (the smallest included), so the
  // kernel's passes exist in one storage type only (faseSuavizar); the level buffers hold 4 bytes
  // an element whatever they store
  if (p->precisao != TQ_PREC_FP32)
    for (int l = 0; l < Lc; l++) p->meia[l] = true;
  size_t porWarp = (size_t)(SUAV_W > REST_W ? SUAV_W : REST_W) * 4;
  size_t areas = (size_t)WARPS * porWarp;
  f->smem = bytes > areas ? bytes : areas;
  {  // the coarsest level's matrix after everything else, when the level is small enough
    const size_t nGrosso = (size_t)p->nxL[p->L - 1] * p->nyL[p->L - 1];
    const size_t off = (f->smem + 15) & ~(size_t)15;
    if (nGrosso <= (size_t)DENSO_MAPA_MAX && off + DENSO_BYTES <= SMEM_CTA_MAX) {
      f->offDenso = (int)off;
      f->smem = off + DENSO_BYTES;
    }
  }
  const size_t nSecao = (size_t)p->nxL[Lc] * p->nyL[Lc];
  f->secaoDensa = f->offDenso >= 0 && nSecao <= (size_t)SECAO_DENSA_MAX && Lc < p->L - 1;
  f->kern = p->precisao == TQ_PREC_FP16   ? kernelDe<__half>()
            : p->precisao == TQ_PREC_BF16 ? kernelDe<__nv_bfloat16>()
                                          : kernelDe<float>();
  int dev = 0, sms = 0, porSM = 0;
  // The attribute is per kernel and shared by every solver in the process: raise it to the
  // largest size any grid uses (f->smem <= SMEM_CTA_MAX), never lower it to this grid's.
  const size_t smemMax = SMEM_CTA_MAX;
  bool ok = cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
            cudaFuncSetAttribute(f->kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemMax) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&porSM, f->kern, TF, f->smem) == cudaSuccess && porSM >= 1;
  if (ok) {
    // one CTA per SM (co-resident, as the grid barrier needs), or the requested fewer
    f->G = p->ctasFundido > 0 && p->ctasFundido < sms ? p->ctasFundido : sms;
    const size_t N = p->N;
    const size_t nLc = (size_t)p->nxL[Lc] * p->nyL[Lc];
    ok = cudaMalloc(&f->niveis, MAX_NIVEIS * sizeof(NivelF)) == cudaSuccess &&
         cudaMalloc(&f->parc, (size_t)f->G * NPARC * sizeof(double)) == cudaSuccess &&
         cudaMalloc(&f->bar, 2 * sizeof(unsigned)) == cudaSuccess && cudaMalloc(&f->erro, sizeof(int)) == cudaSuccess &&
         cudaMalloc(&f->accZ, MAX_BOLHAS * sizeof(long long)) == cudaSuccess &&
         cudaMalloc(&f->zb2, MAX_BOLHAS * sizeof(double)) == cudaSuccess &&
         cudaMalloc(&f->pb2, MAX_BOLHAS * sizeof(double)) == cudaSuccess &&
         cudaMalloc(&f->ativos, MAX_BOLHAS * sizeof(int)) == cudaSuccess &&
         cudaMalloc(&f->nAtivos, sizeof(int)) == cudaSuccess && cudaMalloc(&f->p2, N * 4) == cudaSuccess &&
         cudaMalloc(&f->z2, N * 4) == cudaSuccess && cudaMalloc(&f->xc, nLc * 4) == cudaSuccess &&
         cudaMalloc(&f->bc, nLc * 4) == cudaSuccess && cudaMalloc(&f->op, N * sizeof(uint16_t)) == cudaSuccess &&
         cudaMalloc(&f->rotB, N * sizeof(unsigned long long)) == cudaSuccess &&
         cudaMalloc(&f->q64, N * sizeof(double)) == cudaSuccess &&
         cudaMalloc(&f->accV, MAX_BOLHAS * sizeof(long long)) == cudaSuccess;
    // Wall blocks are skipped on levels of at least two full rounds of the grid's warps (a
    // tank atlas's finest levels): there the flags' one extra load per warp and pass is paid
    // back; a level of one round (the 450k-cell scene's) keeps no flags.
    // TQ_WALL_SKIP_MIN_BLOCKS in the environment (read when the handle is created) sets the
    // threshold in blocks; the tests use 1 to skip on every grid level and 0x7fffffff for none.
    long long limiar = 2LL * WARPS * f->G;
    if (const char* e = getenv("TQ_WALL_SKIP_MIN_BLOCKS")) limiar = atoll(e);
    if (const char* e = getenv("TQ_BARRIER_WAIT_CYCLES")) {
      const long long v = atoll(e);
      if (v > 0 && v <= LIMITE_CICLOS) f->limite = v;
    }
    if (const char* e = getenv("TQ_BARRIER_HOLD_CTA")) f->segurarCta = atoi(e);
    if (const char* e = getenv("TQ_BARRIER_HOLD_CYCLES")) {
      const long long v = atoll(e);
      f->segurarCiclos = v > 0 && v <= 4 * LIMITE_CICLOS ? v : 0;
    }
    size_t nFlags = 0;
    for (int l = 0; l < Lc; l++) {
      f->comParedes[l] = blocosNivel(p->nxL[l], p->nyL[l], 0) >= limiar;
      if (f->comParedes[l]) nFlags += blocosNivel(p->nxL[l], p->nyL[l], 0) + blocosNivel(p->nxL[l], p->nyL[l], 8);
    }
    ok = ok && (nFlags == 0 || cudaMalloc(&f->solidos, nFlags) == cudaSuccess);
    if (ok && f->secaoDensa)
      ok = cudaMalloc(&f->mSecao, nLc * nLc * 4) == cudaSuccess && cudaMalloc(&f->wSecao, nLc * 4) == cudaSuccess &&
           cudaMalloc(&f->wInv, nLc * 4) == cudaSuccess && cudaMalloc(&f->nW, 4) == cudaSuccess &&
           cudaMalloc(&f->densoG, DENSO_BYTES) == cudaSuccess;
  }
  if (ok) {
    NivelF tab[MAX_NIVEIS] = {};
    for (int l = 0; l < p->L; l++) {
      NivelF& n = tab[l];
      n.nx = p->nxL[l];
      n.ny = p->nyL[l];
      n.meia = (l < Lc && p->meia[l]) ? (p->precisao == TQ_PREC_FP16 ? 1 : 2) : 0;
      n.viz = p->vizL[l];
      n.tipo = p->tipoL[l];
      n.b = p->bL[l];
      n.x = p->xL[l];
      n.tmp = p->tmpL[l];
    }
    size_t off = 0;
    for (int l = 0; l < Lc; l++) {
      if (!f->comParedes[l]) continue;
      f->sol[l] = f->solidos + off;
      off += blocosNivel(p->nxL[l], p->nyL[l], 0) + blocosNivel(p->nxL[l], p->nyL[l], 8);
    }
    ok = cudaMemcpy(f->niveis, tab, sizeof tab, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(f->bar, 0, 2 * sizeof(unsigned)) == cudaSuccess && cudaMemset(f->erro, 0, sizeof(int)) == cudaSuccess;
  }
  if (!ok) {
    cudaGetLastError();
    destruirFundido(f);
    return nullptr;
  }
  return f;
}

void destruirFundido(Fundido* f) {
  if (!f) return;
  void* ps[] = {f->niveis, f->parc, f->bar, f->erro, f->accZ, f->zb2, f->pb2, f->ativos,
                f->nAtivos, f->p2, f->z2, f->xc, f->bc, f->perfil, f->op, f->rotB, f->mSecao, f->wSecao, f->wInv, f->nW,
                f->densoG, f->solidos, f->q64, f->accV};
  for (void* q : ps)
    if (q) cudaFree(q);
  delete f;
}

// Queues the solve on `s` and returns without waiting: the iteration count, the residual history
// and the convergence record stay on the device (Escalares), and a bounded wait that gave up
// leaves f->erro set for erroFundido to report.  Nothing here waits for the device, so a frame
// of substeps can be captured in a CUDA graph.
int resolverPressaoFundido(Pcg* p, const Dev& d, int iteracoes, double tol, bool bolhas, int precond,
                           cudaStream_t s) {
  Fundido* f = p->fundido;
  Args a{};
  a.bloco = precond == TQ_PRECOND_BLOCK || precond == TQ_PRECOND_BLOCK_1 ? 1 : 0;
  a.varreduras = a.bloco ? f->varredurasBloco : VARREDURAS;
  a.umaPassada = precond == TQ_PRECOND_BLOCK_1 ? 1 : 0;
  a.limite = f->limite;
  a.segurarCta = f->segurarCta;
  a.segurarCiclos = f->segurarCiclos;
  f->segurarCta = -1;  // the hold is one-shot
  a.q64 = tol > 0 ? f->q64 : nullptr;
  a.accV = f->accV;
  a.d = d;
  a.L = p->L;
  a.Lc = f->Lc;
  a.niv = f->niveis;
  a.vizOp = p->vizOp;
  a.iteracoes = iteracoes;
  a.tol = tol;
  a.bolhas = bolhas ? 1 : 0;
  a.escalar = p->precisao != TQ_PREC_FP32 ? 1 : 0;
  a.parc = f->parc;
  a.bar = f->bar;
  a.erro = f->erro;
  a.accZ = f->accZ;
  a.zb2 = f->zb2;
  a.pb2 = f->pb2;
  a.ativos = f->ativos;
  a.nAtivos = f->nAtivos;
  a.p2 = f->p2;
  a.z2 = f->z2;
  for (int l = 0; l < MAX_NIVEIS; l++) a.sol[l] = f->sol[l];
  a.xc = f->xc;
  a.bc = f->bc;
  a.offDenso = f->offDenso;
  a.secaoDensa = f->secaoDensa ? 1 : 0;
  a.mSecao = f->mSecao;
  a.wSecao = f->wSecao;
  a.wInv = f->wInv;
  a.nWp = f->nW;
  a.densoG = f->densoG;
  a.op = f->op;
  a.rotB = f->rotB;
  a.perfil = f->perfilar ? f->perfil : nullptr;
  if (a.perfil) {
    cudaMemsetAsync(f->perfil, 0, sizeof(unsigned long long), s);
    cudaMemsetAsync(f->perfil + PERFIL_MAX + 1, 0, sizeof(unsigned long long), s);
  }
  cudaMemsetAsync(d.facesB, 0, MAX_BOLHAS * sizeof(uint32_t), s);
  cudaMemsetAsync(d.celsB, 0, MAX_BOLHAS * sizeof(uint32_t), s);
  cudaMemsetAsync(d.accB, 0, MAX_BOLHAS * sizeof(long long), s);
  if (d.nTanques && tol > 0) cudaMemsetAsync(d.r0T, 0, (size_t)d.nTanques * sizeof(double), s);
  cudaMemsetAsync(f->bar, 0, 2 * sizeof(unsigned), s);
  // f->erro is not cleared here: a solve that gave up keeps it set until erroFundido reads it,
  // and every later solve of the frame then stops at its first barrier instead of waiting.
  // The levels that skip wall blocks start the solve with their snapshots and right side at 0,
  // and with level 0 so do both z vectors (a pass never writes anything else off water).
  for (int l = 0; l < f->Lc; l++) {
    if (!f->comParedes[l]) continue;
    const size_t bytes = (size_t)p->nxL[l] * p->nyL[l] * (p->meia[l] ? 2 : 4);
    cudaMemsetAsync(p->xL[l], 0, bytes, s);
    cudaMemsetAsync(p->tmpL[l], 0, bytes, s);
    cudaMemsetAsync(p->bL[l], 0, bytes, s);
  }
  if (f->comParedes[0]) {
    cudaMemsetAsync(d.z, 0, (size_t)d.N * 4, s);
    cudaMemsetAsync(f->z2, 0, (size_t)d.N * 4, s);
  }
  void* args[] = {&a};
  contarLancamento();
  cudaError_t e = cudaLaunchCooperativeKernel(f->kern, dim3(f->G), dim3(TF), args, f->smem, s);
  if (e != cudaSuccess) return TQ_E_CUDA;
  return TQ_OK;
}

// TQ_E_TIMEOUT when a solve since the last call gave up on a bounded wait (the flag is cleared),
// else TQ_OK.  Waits for the stream.
int erroFundido(Fundido* f, cudaStream_t s) {
  if (!f) return TQ_OK;
  int h = 0;
  if (cudaMemcpyAsync(&h, f->erro, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return TQ_E_CUDA;
  if (!h) return TQ_OK;
  if (cudaMemsetAsync(f->erro, 0, sizeof(int), s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
    return TQ_E_CUDA;
  return TQ_E_TIMEOUT;
}

}  // namespace tq
