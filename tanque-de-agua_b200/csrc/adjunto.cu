// adjunto.cu — the hand-written adjoint of the substep on the GPU (tq_adj_*), in FP64.
//
// The differentiable configuration of SimulacaoCPU.subpasso (js/fisica-cpu.js:176-189): air
// tracking off, surface tension 0, density correction off.  A step is: the faucet's particles
// (velocity theta) through adicionar's wall filter (:100), APIC P2G with float sums (:198-267),
// gravity and wall faces (:271-291), cell flags (:293-299), the divergence (:456-481 without the
// density and air terms), the pressure solve of resolverPCG's system (js/pressao-cpu.js:296-402)
// to a relative 1e-12, the gradient (:519-545), two extrapolation layers (:547-552, 673-690) and
// G2P with micro-steps and wall collisions (:556-661; foam and dye do not enter the loss).  The
// loss is the sum over cells of (min(1, rho/4) - target)^2 with rho the bilinear density at the
// cell centres (:244-254).
//
// Forward: every `checkpoint_every` steps the particle state is kept.  Backward: each segment is
// recomputed from its checkpoint, recording the step's tape (the state at the step's start, the
// P2G sums, flags, valid masks, the grid velocities G2P read, and per particle the micro-step
// count, clamps, collision branches and the positions before each micro-move), then gone back
// through in reverse.  The discrete structure is the forward run's (the checker, the FP64 CPU
// adjoint of the oracle, freezes the same decisions).  Transposes: P2G's reverse is a gather over
// each particle's 2 x 2 stencils; G2P's reverse scatters into the grid's adjoint with FP64
// atomics; the pressure solve is self-adjoint (A symmetric), so the adjoint solve is the same
// solve.  The solve is CG in FP64 preconditioned by the library's FP32 V-cycle (cicloV,
// js/pressao-cpu.js:241-255), with the Polak-Ribiere beta that tolerates the FP32 rounding of
// the preconditioner.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <utility>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace tq {
namespace {

constexpr int MMAX = 4;           // MAX_MICROPASSOS
constexpr int CAMADAS_EXT = 2;    // CAMADAS_EXTRAPOLACAO
constexpr int TB = 256;
constexpr double TOL_SOLVE = 1e-12;

// particle state: 8 doubles a particle, structure of arrays (x, y, vx, vy, cux, cuy, cvx, cvy)
struct Estado {
  double* c[8];
};

struct Dispositivo {
  int nx, ny, N, nu, nv, mw, mh;
  double h, dt, gx, gy, vmax;
  const float* sdf;
  const uint8_t* solido;
};

// ---------------------------------------------------------------- SDF with derivatives
// Cena.#bilinear (js/cena.js:156-165) on the mask and its derivatives in mask pixels.
__device__ double bilD(const Dispositivo& D, double fx, double fy, double* dfx, double* dfy) {
  bool cx = false, cy = false;
  const int w = D.mw, hh = D.mh;
  if (fx < 0) { fx = 0; cx = true; }
  else if (fx > w - 1) { fx = w - 1; cx = true; }
  if (fy < 0) { fy = 0; cy = true; }
  else if (fy > hh - 1) { fy = hh - 1; cy = true; }
  const int x0 = (int)fmin(floor(fx), (double)(w - 2)), y0 = (int)fmin(floor(fy), (double)(hh - 2));
  const double tx = fx - x0, ty = fy - y0;
  const size_t k = (size_t)y0 * w + x0;
  const double a = D.sdf[k], b = D.sdf[k + 1], c = D.sdf[k + w], d = D.sdf[k + w + 1];
  if (dfx) *dfx = cx ? 0.0 : (b - a) * (1 - ty) + (d - c) * ty;
  if (dfy) *dfy = cy ? 0.0 : (c - a) * (1 - tx) + (d - b) * tx;
  return (a * (1 - tx) + b * tx) * (1 - ty) + (c * (1 - tx) + d * tx) * ty;
}
// Cena.distancia (js/cena.js:102-106) with its gradient in metres
__device__ double distD(const Dispositivo& D, double x, double y, double* gx, double* gy) {
  double dfx, dfy;
  const double v = bilD(D, (x / D.h) * RES_MASCARA - 0.5, (y / D.h) * RES_MASCARA - 0.5, &dfx, &dfy);
  if (gx) *gx = dfx * RES_MASCARA / D.h;
  if (gy) *gy = dfy * RES_MASCARA / D.h;
  return v;
}
// Cena.normal (js/cena.js:109-116) with its Jacobian J[i][j] = d n_i / d x_j
__device__ void normalD(const Dispositivo& D, double x, double y, double n[2], double J[2][2]) {
  const double fx = (x / D.h) * RES_MASCARA - 0.5, fy = (y / D.h) * RES_MASCARA - 0.5;
  double a1, a2, b1, b2, c1, c2, d1, d2;
  const double g0 = bilD(D, fx + 1, fy, &a1, &a2) - bilD(D, fx - 1, fy, &b1, &b2);
  const double g1 = bilD(D, fx, fy + 1, &c1, &c2) - bilD(D, fx, fy - 1, &d1, &d2);
  const double s = RES_MASCARA / D.h;
  const double G[2][2] = {{(a1 - b1) * s, (a2 - b2) * s}, {(c1 - d1) * s, (c2 - d2) * s}};
  const double nn = hypot(g0, g1);
  if (nn > 1e-9) {
    n[0] = g0 / nn;
    n[1] = g1 / nn;
    const double P[2][2] = {{(1 - n[0] * n[0]) / nn, -n[0] * n[1] / nn}, {-n[1] * n[0] / nn, (1 - n[1] * n[1]) / nn}};
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 2; j++) J[i][j] = P[i][0] * G[0][j] + P[i][1] * G[1][j];
  } else {
    n[0] = 0;
    n[1] = 1;
    J[0][0] = J[0][1] = J[1][0] = J[1][1] = 0;
  }
}

// ---------------------------------------------------------------- stencils and sampling
struct Est {
  int i0, j0, W;
  double tx, ty;
};
// kind 0: u faces, 1: v faces, 2: cell centres (js/fisica-cpu.js:214-248's clamps)
__device__ __forceinline__ Est est(const Dispositivo& D, int kind, double x, double y) {
  const double inv = 1 / D.h;
  Est e;
  double fx, fy;
  if (kind == 0) {
    fx = x * inv, fy = y * inv - 0.5;
    e.i0 = clampi((int)floor(fx), 0, D.nx - 1), e.j0 = clampi((int)floor(fy), 0, D.ny - 2), e.W = D.nx + 1;
  } else if (kind == 1) {
    fx = x * inv - 0.5, fy = y * inv;
    e.i0 = clampi((int)floor(fx), 0, D.nx - 2), e.j0 = clampi((int)floor(fy), 0, D.ny - 1), e.W = D.nx;
  } else {
    fx = x * inv - 0.5, fy = y * inv - 0.5;
    e.i0 = clampi((int)floor(fx), 0, D.nx - 2), e.j0 = clampi((int)floor(fy), 0, D.ny - 2), e.W = D.nx;
  }
  e.tx = fx - e.i0;
  e.ty = fy - e.j0;
  return e;
}

// Grid velocity and affine terms at (x, y) (js/fisica-cpu.js:566-591) with the cross derivatives
// kux = d cux/dy = d cuy/dx (likewise kvx); d vx/dx = cux, d vx/dy = cuy.
struct Amostra {
  double vx, vy, cux, cuy, cvx, cvy, kux, kvx;
  Est eu, ev;
};
__device__ Amostra amostrar(const Dispositivo& D, const double* ug, const double* vg, double x, double y) {
  const double inv = 1 / D.h;
  Amostra s{};
  s.eu = est(D, 0, x, y);
  s.ev = est(D, 1, x, y);
#pragma unroll
  for (int b = 0; b < 2; b++)
#pragma unroll
    for (int a = 0; a < 2; a++) {
      double wx = a ? s.eu.tx : 1 - s.eu.tx, wy = b ? s.eu.ty : 1 - s.eu.ty;
      double val = ug[s.eu.i0 + a + (s.eu.j0 + b) * s.eu.W];
      s.vx += wx * wy * val;
      s.cux += (a ? 1 : -1) * wy * inv * val;
      s.cuy += wx * (b ? 1 : -1) * inv * val;
      s.kux += (a ? 1 : -1) * (b ? 1 : -1) * inv * inv * val;
      wx = a ? s.ev.tx : 1 - s.ev.tx, wy = b ? s.ev.ty : 1 - s.ev.ty;
      val = vg[s.ev.i0 + a + (s.ev.j0 + b) * s.ev.W];
      s.vy += wx * wy * val;
      s.cvx += (a ? 1 : -1) * wy * inv * val;
      s.cvy += wx * (b ? 1 : -1) * inv * val;
      s.kvx += (a ? 1 : -1) * (b ? 1 : -1) * inv * inv * val;
    }
  return s;
}
// Transpose of amostrar: adjoints bv = (vx, vy, cux, cuy, cvx, cvy) into the grid (atomics) and
// into the position.
__device__ void amostrarT(const Dispositivo& D, const Amostra& s, const double bv[6], double* ugb, double* vgb,
                          double* xb, double* yb) {
  const double inv = 1 / D.h;
#pragma unroll
  for (int b = 0; b < 2; b++)
#pragma unroll
    for (int a = 0; a < 2; a++) {
      double wx = a ? s.eu.tx : 1 - s.eu.tx, wy = b ? s.eu.ty : 1 - s.eu.ty;
      const double gu = bv[0] * wx * wy + bv[2] * (a ? 1 : -1) * wy * inv + bv[3] * wx * (b ? 1 : -1) * inv;
      if (gu != 0) atomicAdd(ugb + s.eu.i0 + a + (s.eu.j0 + b) * s.eu.W, gu);
      wx = a ? s.ev.tx : 1 - s.ev.tx, wy = b ? s.ev.ty : 1 - s.ev.ty;
      const double gv = bv[1] * wx * wy + bv[4] * (a ? 1 : -1) * wy * inv + bv[5] * wx * (b ? 1 : -1) * inv;
      if (gv != 0) atomicAdd(vgb + s.ev.i0 + a + (s.ev.j0 + b) * s.ev.W, gv);
    }
  *xb += bv[0] * s.cux + bv[1] * s.cvx + bv[3] * s.kux + bv[5] * s.kvx;
  *yb += bv[0] * s.cuy + bv[1] * s.cvy + bv[2] * s.kux + bv[4] * s.kvx;
}
// The adjoint of the speed clamp v vmax / |v| (active branch)
__device__ __forceinline__ void limitarT(double vx, double vy, double vmax, double* bx, double* by) {
  const double v = hypot(vx, vy), nx = vx / v, ny = vy / v, f = vmax / v;
  const double dot = *bx * nx + *by * ny;
  *bx = f * (*bx - dot * nx);
  *by = f * (*by - dot * ny);
}

// ---------------------------------------------------------------- the tape of one step
struct Fita {
  int n;                 // particles at the step's start (after the faucet)
  double* P;             // 8 x cap: the state at the step's start
  double *U, *V, *UW, *VW;
  uint8_t* tipo;
  uint8_t* val;          // (CAMADAS_EXT + 1) x (nu + nv): valid masks before each layer, and after
  double *ug, *vg;       // the grid G2P read
  int* micro;            // per particle
  int* bits;             // per particle: bit 0 clampV, bit 1 dead; bits 2+3m col, 3+3m cut, 4+3m clampW
  double* xm;            // per particle (MMAX + 1) x 2: positions before each micro-move, then the end
  int* vivos;            // the particles alive after G2P, in order
  int nVivos;
};

__device__ __forceinline__ double* Pc(const Fita& f, int cap, int c) { return f.P + (size_t)c * cap; }

// ---------------------------------------------------------------- forward kernels
// the faucet's accepted particles of the step, appended after the n current ones
__global__ void k_adj_torneira(Estado E, int n, const double* fpos, const int* aceitos, int nAceitos, double th0,
                               double th1) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nAceitos) return;
  const int q = aceitos[k];
  const int i = n + k;
  E.c[0][i] = fpos[2 * q];
  E.c[1][i] = fpos[2 * q + 1];
  E.c[2][i] = th0;
  E.c[3][i] = th1;
  E.c[4][i] = E.c[5][i] = E.c[6][i] = E.c[7][i] = 0;
}

// P2G float sums in double (js/fisica-cpu.js:198-267) and the particle count per cell
__global__ void k_adj_p2g(Dispositivo D, Estado E, int n, double* U, double* UW, double* V, double* VW, int* cont) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double x = E.c[0][k], y = E.c[1][k], vx = E.c[2][k], vy = E.c[3][k];
  const double cux = E.c[4][k], cuy = E.c[5][k], cvx = E.c[6][k], cvy = E.c[7][k], h = D.h;
  Est e = est(D, 0, x, y);
#pragma unroll
  for (int b = 0; b < 2; b++)
#pragma unroll
    for (int a = 0; a < 2; a++) {
      const double w = (a ? e.tx : 1 - e.tx) * (b ? e.ty : 1 - e.ty);
      const double dx = (e.i0 + a) * h - x, dy = (e.j0 + b + 0.5) * h - y;
      const int idx = e.i0 + a + (e.j0 + b) * e.W;
      atomicAdd(U + idx, w * (vx + cux * dx + cuy * dy));
      atomicAdd(UW + idx, w);
    }
  e = est(D, 1, x, y);
#pragma unroll
  for (int b = 0; b < 2; b++)
#pragma unroll
    for (int a = 0; a < 2; a++) {
      const double w = (a ? e.tx : 1 - e.tx) * (b ? e.ty : 1 - e.ty);
      const double dx = (e.i0 + a + 0.5) * h - x, dy = (e.j0 + b) * h - y;
      const int idx = e.i0 + a + (e.j0 + b) * e.W;
      atomicAdd(V + idx, w * (vy + cvx * dx + cvy * dy));
      atomicAdd(VW + idx, w);
    }
  const int ci = clampi((int)floor(x / h), 0, D.nx - 1), cj = clampi((int)floor(y / h), 0, D.ny - 1);
  atomicAdd(cont + ci + cj * D.nx, 1);
}

// #tipos (:293-299)
__global__ void k_adj_tipos(Dispositivo D, const int* cont, uint8_t* tipo) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= D.N) return;
  tipo[c] = D.solido[c] ? SOLIDO : cont[c] > 0 ? AGUA : AR;
}

// u = U / UW where weighted, gravity there, wall faces 0 (:271-291)
__global__ void k_adj_faces(Dispositivo D, const double* U, const double* UW, const double* V, const double* VW,
                            double* u, double* v) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = D.nx, ny = D.ny;
  if (k < D.nu) {
    const int i = k % (nx + 1), j = k / (nx + 1);
    double x = UW[k] > 0 ? U[k] / UW[k] + D.gx * D.dt : 0.0;
    if (i == 0 || i == nx || D.solido[i - 1 + j * nx] || D.solido[i + j * nx]) x = 0;
    u[k] = x;
  }
  if (k < D.nv) {
    const int i = k % nx, j = k / nx;
    double x = VW[k] > 0 ? V[k] / VW[k] + D.gy * D.dt : 0.0;
    if (j == 0 || j == ny || D.solido[i + (j - 1) * nx] || D.solido[i + j * nx]) x = 0;
    v[k] = x;
  }
}

// b = -div on water cells (#classificar without the density and air terms)
__global__ void k_adj_div(Dispositivo D, const uint8_t* tipo, const double* u, const double* v, double* b) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= D.N) return;
  const int nx = D.nx, i = c % nx, j = c / nx;
  b[c] = tipo[c] == AGUA ? -(u[i + 1 + j * (nx + 1)] - u[i + j * (nx + 1)] + v[i + (j + 1) * nx] - v[i + j * nx]) : 0.0;
}

// #gradiente (:519-545) and the valid masks
__global__ void k_adj_gradiente(Dispositivo D, const uint8_t* tipo, const double* q, double* u, double* v,
                                uint8_t* vu, uint8_t* vv) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = D.nx, ny = D.ny;
  if (k < D.nu) {
    const int i = k % (nx + 1), j = k / (nx + 1);
    const uint8_t tl = i > 0 ? tipo[i - 1 + j * nx] : SOLIDO, tr = i < nx ? tipo[i + j * nx] : SOLIDO;
    if (tl == SOLIDO || tr == SOLIDO) { u[k] = 0; vu[k] = 1; }
    else if (tl == AGUA || tr == AGUA) {
      u[k] -= (tr == AGUA ? q[i + j * nx] : 0.0) - (tl == AGUA ? q[i - 1 + j * nx] : 0.0);
      vu[k] = 1;
    } else vu[k] = 0;
  }
  if (k < D.nv) {
    const int i = k % nx, j = k / nx;
    const uint8_t tb = j > 0 ? tipo[i + (j - 1) * nx] : SOLIDO, tt = j < ny ? tipo[i + j * nx] : SOLIDO;
    if (tb == SOLIDO || tt == SOLIDO) { v[k] = 0; vv[k] = 1; }
    else if (tb == AGUA || tt == AGUA) {
      v[k] -= (tt == AGUA ? q[i + j * nx] : 0.0) - (tb == AGUA ? q[i + (j - 1) * nx] : 0.0);
      vv[k] = 1;
    } else vv[k] = 0;
  }
}

// one extrapolation layer of one component (extrapolarComponente, js/fisica-cpu.js:673-690):
// reads a and the masks before the layer, writes the new values and masks
__global__ void k_adj_extrap(const double* a, const uint8_t* val, double* out, uint8_t* valOut, int w, int hh) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= w * hh) return;
  const int i = k % w, j = k / w;
  out[k] = a[k];
  valOut[k] = val[k];
  if (val[k]) return;
  double s = 0;
  int m = 0;
  if (i > 0 && val[k - 1]) { s += a[k - 1]; m++; }
  if (i < w - 1 && val[k + 1]) { s += a[k + 1]; m++; }
  if (j > 0 && val[k - w]) { s += a[k - w]; m++; }
  if (j < hh - 1 && val[k + w]) { s += a[k + w]; m++; }
  if (m > 0) {
    out[k] = s / m;
    valOut[k] = 1;
  }
}

// G2P (#paraParticulas, :556-661, without foam and dye), recording the tape; alive flag per particle
__global__ void k_adj_g2p(Dispositivo D, Estado E, int n, int cap, const double* ug, const double* vg, Fita f,
                          Estado S, int* vivo) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double vmax = D.vmax, dt = D.dt, h = D.h;
  const double x0 = E.c[0][k], y0 = E.c[1][k];
  const Amostra sm = amostrar(D, ug, vg, x0, y0);
  double vx = sm.vx, vy = sm.vy;
  const double vel = hypot(vx, vy);
  int bits = 0;
  if (vel > vmax) {
    vx *= vmax / vel;
    vy *= vmax / vel;
    bits |= 1;
  }
  const int mi = (int)fmin(MAX_MICROPASSOS, fmax(1.0, ceil((fmin(vel, vmax) * dt) / (MICROPASSO * h))));
  const double dm = dt / mi;
  double x = x0, y = y0;
  bool morta = false;
  for (int m = 0; m < mi; m++) {
    f.xm[((size_t)k * (MMAX + 1) + m) * 2] = x;
    f.xm[((size_t)k * (MMAX + 1) + m) * 2 + 1] = y;
    double wx = vx, wy = vy;
    if (mi > 1) {
      const Amostra w = amostrar(D, ug, vg, x, y);
      wx = w.vx, wy = w.vy;
      const double vw = hypot(wx, wy);
      if (vw > vmax) {
        wx *= vmax / vw;
        wy *= vmax / vw;
        bits |= 1 << (4 + 3 * m);
      }
    }
    x += wx * dm;
    y += wy * dm;
    const double d = distD(D, x, y, nullptr, nullptr);
    if (d < RAIO_PARTICULA) {
      bits |= 1 << (2 + 3 * m);
      if (d < -SDF_MAX + 0.5) {
        morta = true;
        bits |= 2;
        break;
      }
      double nn[2], J[2][2];
      normalD(D, x, y, nn, J);
      const double e = (RAIO_PARTICULA - d) * h;
      x += nn[0] * e;
      y += nn[1] * e;
      const double vn = vx * nn[0] + vy * nn[1];
      if (vn < 0) {
        vx -= vn * nn[0];
        vy -= vn * nn[1];
        bits |= 1 << (3 + 3 * m);
      }
    }
  }
  if (!morta) {
    f.xm[((size_t)k * (MMAX + 1) + mi) * 2] = x;
    f.xm[((size_t)k * (MMAX + 1) + mi) * 2 + 1] = y;
  }
  f.micro[k] = mi;
  f.bits[k] = bits;
  vivo[k] = morta ? 0 : 1;
  S.c[0][k] = x;
  S.c[1][k] = y;
  S.c[2][k] = vx;
  S.c[3][k] = vy;
  S.c[4][k] = sm.cux;
  S.c[5][k] = sm.cuy;
  S.c[6][k] = sm.cvx;
  S.c[7][k] = sm.cvy;
  (void)cap;
}

// stable compaction of the alive particles: exclusive prefix over one CTA of 1024 threads
// (a few tens of thousands of particles), the alive ones to E in order, their indices to vivos
__global__ void __launch_bounds__(1024) k_adj_compactar(Estado S, const int* vivo, int n, Estado E, int* vivos,
                                                        int* nVivos) {
  __shared__ int soma[1024];
  __shared__ int base;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  for (int c0 = 0; c0 < n; c0 += 1024) {
    const int k = c0 + threadIdx.x;
    const int v = k < n ? vivo[k] : 0;
    soma[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {  // inclusive scan (Hillis-Steele)
      const int t = threadIdx.x >= o ? soma[threadIdx.x - o] : 0;
      __syncthreads();
      soma[threadIdx.x] += t;
      __syncthreads();
    }
    if (v) {
      const int dst = base + soma[threadIdx.x] - 1;
      for (int q = 0; q < 8; q++) E.c[q][dst] = S.c[q][k];
      vivos[dst] = k;
    }
    __syncthreads();
    if (threadIdx.x == 1023) base += soma[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) *nVivos = base;
}

// density at cell centres (:244-254)
__global__ void k_adj_densidade(Dispositivo D, Estado E, int n, double* rho) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const Est e = est(D, 2, E.c[0][k], E.c[1][k]);
  const int c = e.i0 + e.j0 * D.nx;
  atomicAdd(rho + c, (1 - e.tx) * (1 - e.ty));
  atomicAdd(rho + c + 1, e.tx * (1 - e.ty));
  atomicAdd(rho + c + D.nx, (1 - e.tx) * e.ty);
  atomicAdd(rho + c + D.nx + 1, e.tx * e.ty);
}

// per-cell loss terms (min(1, rho/4) - target)^2 and their derivative in rho
__global__ void k_adj_perda(Dispositivo D, const double* rho, const double* alvo, double* termo, double* rhob) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= D.N) return;
  const double r4 = rho[c] / 4, f = fmin(1.0, r4), d = f - alvo[c];
  termo[c] = d * d;
  rhob[c] = r4 < 1 ? 2 * d * 0.25 : 0.0;
}

// ---------------------------------------------------------------- deterministic FP64 sums
// a . b over n (b null: sum of a), per-CTA partials in CTA order, then one CTA sums them in
// order: the same bits every run.
constexpr int SOMA_CTAS = 148;
__device__ double somaCta(double v) {
  __shared__ double sh[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double t = 0;
  if (w == 0) {
    t = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  }
  return t;
}
__global__ void k_adj_produto(const double* a, const double* b, int n, double* parc) {
  double s = 0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) s += b ? a[k] * b[k] : a[k];
  const double t = somaCta(s);
  if (threadIdx.x == 0) parc[blockIdx.x] = t;
}
__global__ void k_adj_somar(const double* parc, int m, double* out) {
  double s = 0;
  for (int k = threadIdx.x; k < m; k += blockDim.x) s += parc[k];
  const double t = somaCta(s);
  if (threadIdx.x == 0) *out = t;
}

// ---------------------------------------------------------------- CG kernels
// The CG's scalars live on the device (esc): [0] ||b||^2, [1] alpha, [2] beta, [3] r.z, [4] the
// latest dot, [5] a second dot, [6] the stop flag (as a double: 0 running, else the iteration
// count at the stop, at least 1), [8] the same flag as an int for the V-cycle's kernels, [9] the
// iterations done.  Every kernel of an iteration returns at once after the flag is set, so the
// host reads it only now and then and the result is that of stopping at the exact iteration.
enum { E_B2 = 0, E_AL = 1, E_BE = 2, E_RZ = 3, E_D1 = 4, E_D2 = 5, E_PARA = 6, E_PARA_INT = 8, E_IT = 9, E_N = 10 };
__device__ inline void pararCG(double* esc, int iteracoes) {
  esc[E_PARA] = iteracoes > 0 ? iteracoes : 1;
  *reinterpret_cast<int*>(esc + E_PARA_INT) = 1;
}

// A v on water cells (js/pressao-cpu.js:84-93, true types; air is 0)
__global__ void k_adj_aplicar(Dispositivo D, const uint8_t* tipo, const double* v, double* out, const double* esc) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= D.N || (esc && esc[E_PARA] != 0)) return;
  if (tipo[c] != AGUA) { out[c] = 0; return; }
  const int nx = D.nx, ny = D.ny, i = c % nx, j = c / nx;
  int k = 0;
  double s = 0;
  const int nb[4] = {c - 1, c + 1, c - nx, c + nx};
  const bool ok[4] = {i > 0, i < nx - 1, j > 0, j < ny - 1};
#pragma unroll
  for (int t = 0; t < 4; t++) {
    if (!ok[t] || tipo[nb[t]] == SOLIDO) continue;
    k++;
    if (tipo[nb[t]] == AGUA) s += v[nb[t]];
  }
  out[c] = k * v[c] - s;
}
__global__ void k_adj_axpy2(int n, const uint8_t* tipo, const double* esc, double* q, const double* p, double* r,
                            const double* ap) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n || tipo[c] != AGUA || esc[E_PARA] != 0) return;
  const double a = esc[E_AL];
  q[c] += a * p[c];
  r[c] -= a * ap[c];
}
__global__ void k_adj_direcao(int n, const uint8_t* tipo, const double* esc, const double* z, double* p) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n || esc[E_PARA] != 0) return;
  p[c] = tipo[c] == AGUA ? z[c] + esc[E_BE] * p[c] : 0.0;
}
// z from the FP32 V-cycle: r scaled to unit norm (esc[E_D1] = ||r||^2) before, back after
__global__ void k_adj_para_float(int n, const uint8_t* tipo, const double* r, const double* esc, int qual, float* b) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const double nr = sqrt(esc[qual]);
  b[c] = tipo[c] == AGUA ? (float)(r[c] * (nr > 0 ? 1.0 / nr : 1.0)) : 0.0f;
}
__global__ void k_adj_de_float(int n, const uint8_t* tipo, const float* x, const double* esc, int qual, double* z) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n || esc[E_PARA] != 0) return;
  const double nr = sqrt(esc[qual]);
  z[c] = tipo[c] == AGUA ? (double)x[c] * (nr > 0 ? nr : 1.0) : 0.0;
}
__global__ void k_adj_mascarar(int n, const uint8_t* tipo, const double* b, double* r, double* q) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  r[c] = tipo[c] == AGUA ? b[c] : 0.0;
  q[c] = 0.0;
}
__global__ void k_adj_copiar_se(double* dst, const double* src, size_t n, const double* esc) {
  if (esc[E_PARA] != 0) return;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    dst[k] = src[k];
}
// the scalar steps of one CG iteration (one thread; the iteration count in E_IT): modo 0 start
// (||b||^2 in E_D1 -> E_B2, the flag cleared unless b = 0, no iterations); 1 alpha = rz / p.Ap
// (E_D1); 2 the stop test on r.r (E_D1); 3 Polak-Ribiere beta from r.z (E_D1) and r.zOld (E_D2),
// the iteration counted; 4 rz
__global__ void k_adj_escalares(double* esc, int modo, double tol2) {
  if (modo == 0) {
    esc[E_B2] = esc[E_D1];
    esc[E_PARA] = 0.0;
    esc[E_IT] = 0.0;
    *reinterpret_cast<int*>(esc + E_PARA_INT) = 0;
    if (esc[E_B2] == 0) pararCG(esc, 0);
    return;
  }
  if (esc[E_PARA] != 0) return;
  const int it = (int)esc[E_IT];
  if (modo == 1) {
    const double pap = esc[E_D1];
    if (pap == 0) pararCG(esc, it);
    else esc[E_AL] = esc[E_RZ] / pap;
  } else if (modo == 2) {
    if (esc[E_D1] <= tol2 * esc[E_B2]) pararCG(esc, it + 1);
  } else if (modo == 3) {
    const double rzn = esc[E_D1], cruz = esc[E_D2];
    esc[E_BE] = fmax(0.0, (rzn - cruz) / esc[E_RZ]);
    esc[E_RZ] = rzn;
    esc[E_IT] = it + 1;
  } else if (modo == 4) {
    esc[E_RZ] = esc[E_D1];
  }
}

// ---------------------------------------------------------------- backward kernels
// final positions' adjoint from the loss (the density stencil's derivatives)
__global__ void k_adj_perda_T(Dispositivo D, Estado E, int n, const double* rhob, Estado B) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const Est e = est(D, 2, E.c[0][k], E.c[1][k]);
  const int c = e.i0 + e.j0 * D.nx;
  const double r00 = rhob[c], r10 = rhob[c + 1], r01 = rhob[c + D.nx], r11 = rhob[c + D.nx + 1], inv = 1 / D.h;
  B.c[0][k] = inv * (-(1 - e.ty) * r00 + (1 - e.ty) * r10 - e.ty * r01 + e.ty * r11);
  B.c[1][k] = inv * (-(1 - e.tx) * r00 - e.tx * r10 + (1 - e.tx) * r01 + e.tx * r11);
  for (int q = 2; q < 8; q++) B.c[q][k] = 0;
}

// G2P reverse of output particle o (input particle vivos[o]): position adjoint into Bin, grid
// adjoint into ugb / vgb (atomics)
__global__ void k_adj_g2p_T(Dispositivo D, Fita f, int cap, Estado B, Estado Bin, double* ugb, double* vgb) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= f.nVivos) return;
  const int k = f.vivos[o];
  const double vmax = D.vmax, dt = D.dt, h = D.h;
  const double px = Pc(f, cap, 0)[k], py = Pc(f, cap, 1)[k];
  const Amostra sm = amostrar(D, f.ug, f.vg, px, py);
  const int mi = f.micro[k], bits = f.bits[k];
  const double dm = dt / mi;
  auto pos = [&](int m, int c) { return f.xm[((size_t)k * (MMAX + 1) + m) * 2 + c]; };
  // the particle velocity before each micro-step (collisions cut it)
  double vxm[MMAX + 1], vym[MMAX + 1];
  double vx = sm.vx, vy = sm.vy;
  if (bits & 1) {
    const double vel = hypot(vx, vy);
    vx *= vmax / vel;
    vy *= vmax / vel;
  }
  for (int m = 0; m < mi; m++) {
    vxm[m] = vx, vym[m] = vy;
    if ((bits >> (2 + 3 * m) & 1) && (bits >> (3 + 3 * m) & 1)) {
      const double xa = pos(m, 0), ya = pos(m, 1);
      double wx = vx, wy = vy;
      if (mi > 1) {
        const Amostra w = amostrar(D, f.ug, f.vg, xa, ya);
        wx = w.vx, wy = w.vy;
        if (bits >> (4 + 3 * m) & 1) {
          const double vw = hypot(wx, wy);
          wx *= vmax / vw;
          wy *= vmax / vw;
        }
      }
      double nn[2], J[2][2];
      normalD(D, xa + wx * dm, ya + wy * dm, nn, J);
      const double vn = vx * nn[0] + vy * nn[1];
      vx -= vn * nn[0];
      vy -= vn * nn[1];
    }
  }
  double xb = B.c[0][o], yb = B.c[1][o], vxb = B.c[2][o], vyb = B.c[3][o];
  for (int m = mi - 1; m >= 0; m--) {
    const double xa = pos(m, 0), ya = pos(m, 1);
    double wx = vxm[m], wy = vym[m];
    Amostra w{};
    if (mi > 1) {
      w = amostrar(D, f.ug, f.vg, xa, ya);
      wx = w.vx, wy = w.vy;
      if (bits >> (4 + 3 * m) & 1) {
        const double vw = hypot(wx, wy);
        wx *= vmax / vw;
        wy *= vmax / vw;
      }
    }
    const double xp = xa + wx * dm, yp = ya + wy * dm;
    if (bits >> (2 + 3 * m) & 1) {
      double dgx, dgy, nn[2], J[2][2];
      const double d = distD(D, xp, yp, &dgx, &dgy);
      normalD(D, xp, yp, nn, J);
      const double e = (RAIO_PARTICULA - d) * h;
      double xpb = 0, ypb = 0;
      if (bits >> (3 + 3 * m) & 1) {  // v_after = v - (v.n) n
        const double v0x = vxm[m], v0y = vym[m], vn = v0x * nn[0] + v0y * nn[1];
        const double bn = vxb * nn[0] + vyb * nn[1];
        const double gnx = -(v0x * bn + vn * vxb), gny = -(v0y * bn + vn * vyb);
        xpb += gnx * J[0][0] + gny * J[1][0];
        ypb += gnx * J[0][1] + gny * J[1][1];
        vxb -= bn * nn[0];
        vyb -= bn * nn[1];
      }
      // x_after = xp + n(xp) (R - d(xp)) h
      const double be = xb * nn[0] + yb * nn[1], gnx = xb * e, gny = yb * e;
      xpb += xb + gnx * J[0][0] + gny * J[1][0] - be * h * dgx;
      ypb += yb + gnx * J[0][1] + gny * J[1][1] - be * h * dgy;
      xb = xpb, yb = ypb;
    }
    double wxb = xb * dm, wyb = yb * dm;
    if (mi > 1) {
      if (bits >> (4 + 3 * m) & 1) limitarT(w.vx, w.vy, vmax, &wxb, &wyb);
      const double bv[6] = {wxb, wyb, 0, 0, 0, 0};
      amostrarT(D, w, bv, ugb, vgb, &xb, &yb);
    } else {
      vxb += wxb;
      vyb += wyb;
    }
  }
  if (bits & 1) limitarT(sm.vx, sm.vy, vmax, &vxb, &vyb);
  const double bv[6] = {vxb, vyb, B.c[4][o], B.c[5][o], B.c[6][o], B.c[7][o]};
  amostrarT(D, sm, bv, ugb, vgb, &xb, &yb);
  Bin.c[0][k] = xb;
  Bin.c[1][k] = yb;
}

// reverse of one extrapolation layer: a face filled in the layer hands its adjoint to the valid
// neighbours it averaged; out starts as a copy of xb
__global__ void k_adj_extrap_T(const double* xb, const uint8_t* val, const uint8_t* valDepois, double* out, int w,
                               int hh) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= w * hh) return;
  if (val[k] || !valDepois[k]) return;
  const int i = k % w, j = k / w;
  int m = 0;
  if (i > 0 && val[k - 1]) m++;
  if (i < w - 1 && val[k + 1]) m++;
  if (j > 0 && val[k - w]) m++;
  if (j < hh - 1 && val[k + w]) m++;
  const double g = xb[k] / m;
  atomicAdd(out + k, -xb[k]);
  if (i > 0 && val[k - 1]) atomicAdd(out + k - 1, g);
  if (i < w - 1 && val[k + 1]) atomicAdd(out + k + 1, g);
  if (j > 0 && val[k - w]) atomicAdd(out + k - w, g);
  if (j < hh - 1 && val[k + w]) atomicAdd(out + k + w, g);
}

// the gradient's reverse as a gather per cell: qb = sum over the cell's faces with a water side
// and no wall side of -/+ the face adjoint (the cell is the face's right / left side)
__global__ void k_adj_grad_T(Dispositivo D, const uint8_t* tipo, const double* ugb, const double* vgb, double* qb) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= D.N) return;
  if (tipo[c] != AGUA) { qb[c] = 0; return; }
  const int nx = D.nx, ny = D.ny, i = c % nx, j = c / nx;
  double s = 0;
  // left face (i, j): this cell is its right side
  if (i > 0 && tipo[c - 1] != SOLIDO) s -= ugb[i + j * (nx + 1)];
  // right face (i+1, j): this cell is its left side
  if (i < nx - 1 && tipo[c + 1] != SOLIDO) s += ugb[i + 1 + j * (nx + 1)];
  if (j > 0 && tipo[c - nx] != SOLIDO) s -= vgb[i + j * nx];
  if (j < ny - 1 && tipo[c + nx] != SOLIDO) s += vgb[i + (j + 1) * nx];
  qb[c] = s;
}

// faces: + the divergence's reverse (div adjoint = -lam), then wall faces 0, then the
// normalisation's reverse (u = U / UW) into Ub, UWb
__global__ void k_adj_faces_T(Dispositivo D, const uint8_t* tipo, const double* lam, const double* ugb,
                              const double* vgb, const double* U, const double* UW, const double* V, const double* VW,
                              double* Ub, double* UWb, double* Vb, double* VWb) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = D.nx, ny = D.ny;
  if (k < D.nu) {
    const int i = k % (nx + 1), j = k / (nx + 1);
    double g = ugb[k];
    const bool tr = i < nx && tipo[i + j * nx] == AGUA, tl = i > 0 && tipo[i - 1 + j * nx] == AGUA;
    if (tl) g += -lam[i - 1 + j * nx];  // right face of cell i-1: d div / d u = +1
    if (tr) g -= -lam[i + j * nx];      // left face of cell i: -1
    if (i == 0 || i == nx || D.solido[i - 1 + j * nx] || D.solido[i + j * nx]) g = 0;
    if (UW[k] > 0) {
      Ub[k] = g / UW[k];
      UWb[k] = -g * U[k] / (UW[k] * UW[k]);
    } else Ub[k] = UWb[k] = 0;
  }
  if (k < D.nv) {
    const int i = k % nx, j = k / nx;
    double g = vgb[k];
    const bool tt = j < ny && tipo[i + j * nx] == AGUA, tb = j > 0 && tipo[i + (j - 1) * nx] == AGUA;
    if (tb) g += -lam[i + (j - 1) * nx];
    if (tt) g -= -lam[i + j * nx];
    if (j == 0 || j == ny || D.solido[i + (j - 1) * nx] || D.solido[i + j * nx]) g = 0;
    if (VW[k] > 0) {
      Vb[k] = g / VW[k];
      VWb[k] = -g * V[k] / (VW[k] * VW[k]);
    } else Vb[k] = VWb[k] = 0;
  }
}

// P2G reverse per particle: a gather of its 2 x 2 stencils into its state adjoint (adds to the
// position adjoint G2P's reverse left in Bin)
__global__ void k_adj_p2g_T(Dispositivo D, Fita f, int cap, const double* Ub, const double* UWb, const double* Vb,
                            const double* VWb, Estado Bin) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= f.n) return;
  const double x = Pc(f, cap, 0)[k], y = Pc(f, cap, 1)[k], vx = Pc(f, cap, 2)[k], vy = Pc(f, cap, 3)[k];
  const double cux = Pc(f, cap, 4)[k], cuy = Pc(f, cap, 5)[k], cvx = Pc(f, cap, 6)[k], cvy = Pc(f, cap, 7)[k];
  const double h = D.h, inv = 1 / h;
  double bx = 0, by = 0, bvx = 0, bvy = 0, bcux = 0, bcuy = 0, bcvx = 0, bcvy = 0;
  Est e = est(D, 0, x, y);
#pragma unroll
  for (int b = 0; b < 2; b++)
#pragma unroll
    for (int a = 0; a < 2; a++) {
      const double wx = a ? e.tx : 1 - e.tx, wy = b ? e.ty : 1 - e.ty, w = wx * wy;
      const double dx = (e.i0 + a) * h - x, dy = (e.j0 + b + 0.5) * h - y;
      const int idx = e.i0 + a + (e.j0 + b) * e.W;
      const double g = Ub[idx], t = (vx + cux * dx + cuy * dy) * g + UWb[idx];
      bvx += w * g;
      bcux += w * dx * g;
      bcuy += w * dy * g;
      bx += (a ? 1 : -1) * inv * wy * t - w * cux * g;
      by += wx * (b ? 1 : -1) * inv * t - w * cuy * g;
    }
  e = est(D, 1, x, y);
#pragma unroll
  for (int b = 0; b < 2; b++)
#pragma unroll
    for (int a = 0; a < 2; a++) {
      const double wx = a ? e.tx : 1 - e.tx, wy = b ? e.ty : 1 - e.ty, w = wx * wy;
      const double dx = (e.i0 + a + 0.5) * h - x, dy = (e.j0 + b) * h - y;
      const int idx = e.i0 + a + (e.j0 + b) * e.W;
      const double g = Vb[idx], t = (vy + cvx * dx + cvy * dy) * g + VWb[idx];
      bvy += w * g;
      bcvx += w * dx * g;
      bcvy += w * dy * g;
      bx += (a ? 1 : -1) * inv * wy * t - w * cvx * g;
      by += wx * (b ? 1 : -1) * inv * t - w * cvy * g;
    }
  Bin.c[0][k] += bx;
  Bin.c[1][k] += by;
  Bin.c[2][k] = bvx;
  Bin.c[3][k] = bvy;
  Bin.c[4][k] = bcux;
  Bin.c[5][k] = bcuy;
  Bin.c[6][k] = bcvx;
  Bin.c[7][k] = bcvy;
}

__global__ void k_adj_zerar(double* a, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) a[k] = 0;
}
__global__ void k_adj_saida_v(Estado B, int n, double escala, float* dv) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  dv[2 * k] = (float)(B.c[2][k] * escala);
  dv[2 * k + 1] = (float)(B.c[3][k] * escala);
}
__global__ void k_adj_entrada_v(Estado E, int n, const float* v0, const double* pos0, const double* C0) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  E.c[0][k] = pos0[2 * k];
  E.c[1][k] = pos0[2 * k + 1];
  E.c[2][k] = v0[2 * k];
  E.c[3][k] = v0[2 * k + 1];
  for (int q = 0; q < 4; q++) E.c[4 + q][k] = C0[4 * k + q];
}

}  // namespace
}  // namespace tq

using namespace tq;

struct tq_adj {
  Dispositivo D;
  int passos, K, n0, nf, cap, N, nu, nv;
  cudaStream_t s = nullptr;
  Pcg* pcg = nullptr;
  std::vector<void*> mem;
  // scene
  float* sdf;
  uint8_t* solido;
  double *pos0, *C0, *fpos, *alvo;
  std::vector<int> nAceitos;  // faucet particles accepted per step
  int* aceitos;               // steps x nf: indices of the accepted ones (first nAceitos[s])
  // state
  double* bufE;  // 8 x cap: current state
  double* bufS;  // 8 x cap: G2P output before compaction
  int *vivo, *nVivosD;
  double* ckpt;                // checkpoints: (steps/K + 1) x 8 x cap
  std::vector<int> nCkpt;
  double theta[2] = {0, 0};
  int nFinal = 0;
  bool temFrente = false;
  // grid work
  double *U, *V, *UW, *VW, *u, *v, *u2, *v2, *b, *q, *rho, *termo, *rhob;
  int* cont;
  uint8_t* tipo;
  uint8_t* valT;  // scratch masks
  // tape of a segment: K steps
  std::vector<Fita> fita;
  double *fP, *fU, *fV, *fUW, *fVW, *fug, *fvg, *fxm;
  uint8_t *ftipo, *fval;
  int *fbits, *fmicro, *fvivos;
  // adjoints
  double *bufB, *bufBin;  // 8 x cap
  double *ugb, *vgb, *ugb2, *vgb2, *qb, *lam, *Ub, *UWb, *Vb, *VWb;
  // CG
  double *r, *z, *zv, *p, *ap, *parc, *esc;  // esc: the CG's scalars (E_*) and a host-read slot (7)
  int itFrente = 0, itTras = 0;                // the last forward / adjoint solve's iteration count
  uint8_t* tipoCG = nullptr;                   // the solve's cell types (copied in at each solve)
  double* xCG = nullptr;                       // the solve's iterate (copied out at the end)
  cudaGraphExec_t grafoCG = nullptr;           // one CG iteration (resolver)
  float *bf, *xf;
  double gth[2] = {0, 0};
};

namespace {

thread_local char g_erroAdj[256] = "";

template <class T>
bool alocar(tq_adj* a, T** p, size_t n) {
  void* q = nullptr;
  if (cudaMalloc(&q, (n ? n : 1) * sizeof(T)) != cudaSuccess) return false;
  a->mem.push_back(q);
  *p = (T*)q;
  return true;
}

Estado estado(double* buf, int cap) {
  Estado e;
  for (int q = 0; q < 8; q++) e.c[q] = buf + (size_t)q * cap;
  return e;
}

int gridDe(long n) { return (int)((n + TB - 1) / TB); }

double somaHost(tq_adj* a, const double* x, const double* y, int n) {
  // slot 7 of esc: apart from the CG's scalars
  contarLancamento();
  k_adj_produto<<<SOMA_CTAS, TB, 0, a->s>>>(x, y, n, a->parc);
  contarLancamento();
  k_adj_somar<<<1, TB, 0, a->s>>>(a->parc, SOMA_CTAS, a->esc + 7);
  double v = 0;
  cudaMemcpyAsync(&v, a->esc + 7, sizeof v, cudaMemcpyDeviceToHost, a->s);
  cudaStreamSynchronize(a->s);
  return v;
}

// a . b (b null: sum of a) into esc[slot] on the device (deterministic two-pass sum)
void somaDisp(tq_adj* a, const double* x, const double* y, int n, double* destino) {
  contarLancamento();
  k_adj_produto<<<SOMA_CTAS, TB, 0, a->s>>>(x, y, n, a->parc);
  contarLancamento();
  k_adj_somar<<<1, TB, 0, a->s>>>(a->parc, SOMA_CTAS, destino);
}

// A x = b on the water cells of `tipo` (device): CG in FP64 preconditioned by the FP32 V-cycle,
// Polak-Ribiere beta, to ||r|| <= 1e-12 ||b||.  The scalars stay on the device.  The host reads
// the stop flag every VERIFICAR iterations, and at every iteration from two before the count
// the previous solve of the same kind took (*estimativa, updated here): the solves of a run
// take similar counts, so few iterations run past the stop (each of those returns at once in
// every kernel but still costs its launches).  Returns TQ_OK or an error.
constexpr int VERIFICAR = 8;
int resolver(tq_adj* a, const uint8_t* tipoIn, const double* bdev, double* xOut, int* estimativa) {
  const int N = a->N;
  const int g = gridDe(N);
  cudaStream_t st = a->s;
  double* esc = a->esc;
  const int* pararInt = reinterpret_cast<const int*>(esc + E_PARA_INT);
  // the solve works on the handle's own type and iterate buffers, so one captured iteration
  // serves every solve of the handle (forward and adjoint, every step of the tape)
  const uint8_t* tipo = a->tipoCG;
  double* x = a->xCG;
  if (cudaMemcpyAsync(a->tipoCG, tipoIn, N, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return TQ_E_CUDA;
  auto escalares = [&](int modo) {
    contarLancamento();
    k_adj_escalares<<<1, 1, 0, st>>>(esc, modo, TOL_SOLVE * TOL_SOLVE);
  };
  auto precond = [&](int qual, bool preparar) {  // z = M r (the V-cycle on r scaled to unit norm; ||r||^2 in esc[qual])
    contarLancamento();
    k_adj_para_float<<<g, TB, 0, st>>>(N, tipo, a->r, esc, qual, a->bf);
    int e = cicloVDispositivo(a->pcg, tipo, a->bf, a->xf, st, preparar, pararInt);
    contarLancamento();
    k_adj_de_float<<<g, TB, 0, st>>>(N, tipo, a->xf, esc, qual, a->z);
    return e;
  };
  auto iteracao = [&]() {
    contarLancamento();
    k_adj_aplicar<<<g, TB, 0, st>>>(a->D, tipo, a->p, a->ap, esc);
    somaDisp(a, a->p, a->ap, N, esc + E_D1);
    escalares(1);  // alpha
    contarLancamento();
    k_adj_axpy2<<<g, TB, 0, st>>>(N, tipo, esc, x, a->p, a->r, a->ap);
    somaDisp(a, a->r, a->r, N, esc + E_D1);
    escalares(2);  // stop test
    contarLancamento();
    k_adj_copiar_se<<<g, TB, 0, st>>>(a->zv, a->z, N, esc);
    const int e = precond(E_D1, false);
    somaDisp(a, a->r, a->z, N, esc + E_D1);
    somaDisp(a, a->r, a->zv, N, esc + E_D2);
    escalares(3);  // beta, the iteration counted
    contarLancamento();
    k_adj_direcao<<<g, TB, 0, st>>>(N, tipo, esc, a->z, a->p);
    return e;
  };
  contarLancamento();
  k_adj_mascarar<<<g, TB, 0, st>>>(N, tipo, bdev, a->r, x);
  somaDisp(a, a->r, a->r, N, esc + E_D1);
  escalares(0);  // ||b||^2, flag
  if (precond(E_B2, true)) return TQ_E_CUDA;  // the levels' types and masks, once per solve
  contarLancamento();
  k_adj_copiar_se<<<g, TB, 0, st>>>(a->p, a->z, N, esc);
  somaDisp(a, a->r, a->z, N, esc + E_D1);
  escalares(4);  // rz
  // one CG iteration as a CUDA graph, captured on the handle's first solve: its 50-odd small
  // launches replay as one (every argument is a buffer of the handle; the scalars live in esc)
  if (!a->grafoCG) {
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return TQ_E_CUDA;
    const int e = iteracao();
    cudaGraph_t gr = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(st, &gr);
    if (e || ec != cudaSuccess || cudaGraphInstantiate(&a->grafoCG, gr, 0) != cudaSuccess) {
      if (gr) cudaGraphDestroy(gr);
      a->grafoCG = nullptr;
      std::snprintf(g_erroAdj, sizeof g_erroAdj, "capturing the adjoint solve's CG iteration failed");
      return TQ_E_CUDA;
    }
    cudaGraphDestroy(gr);
  }
  for (int it = 0; it < 2000; it++) {
    contarLancamento();
    if (cudaGraphLaunch(a->grafoCG, st) != cudaSuccess) return TQ_E_CUDA;
    if (it % VERIFICAR == VERIFICAR - 1 || it + 1 >= *estimativa - 2) {
      double para = 0;
      if (cudaMemcpyAsync(&para, esc + E_PARA, sizeof para, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess)
        return TQ_E_CUDA;
      if (para != 0) {
        *estimativa = (int)para;
        return cudaMemcpyAsync(xOut, x, sizeof(double) * N, cudaMemcpyDeviceToDevice, st) == cudaSuccess ? TQ_OK
                                                                                                      : TQ_E_CUDA;
      }
    }
  }
  std::snprintf(g_erroAdj, sizeof g_erroAdj, "adjoint pressure solve did not reach 1e-12 in 2000 iterations");
  return TQ_E_TIMEOUT;
}

// One forward step from a->bufE (n particles): records the tape into f when f is non-null; the
// new state (compacted) back into a->bufE; returns the new count (or a negative status).
int passoFrente(tq_adj* a, int s, int n, Fita* f) {
  const int cap = a->cap, N = a->N, nu = a->nu, nv = a->nv;
  const Dispositivo& D = a->D;
  cudaStream_t st = a->s;
  Estado E = estado(a->bufE, cap);
  const int na = a->nAceitos[s];
  if (na) {
    contarLancamento();
    k_adj_torneira<<<gridDe(na), TB, 0, st>>>(E, n, a->fpos + (size_t)s * a->nf * 2, a->aceitos + (size_t)s * a->nf,
                                              na, a->theta[0], a->theta[1]);
  }
  n += na;
  double *U = f ? f->U : a->U, *V = f ? f->V : a->V, *UW = f ? f->UW : a->UW, *VW = f ? f->VW : a->VW;
  uint8_t* tipo = f ? f->tipo : a->tipo;
  if (f) {
    f->n = n;
    cudaMemcpyAsync(f->P, a->bufE, sizeof(double) * 8 * cap, cudaMemcpyDeviceToDevice, st);
  }
  cudaMemsetAsync(U, 0, sizeof(double) * nu, st);
  cudaMemsetAsync(UW, 0, sizeof(double) * nu, st);
  cudaMemsetAsync(V, 0, sizeof(double) * nv, st);
  cudaMemsetAsync(VW, 0, sizeof(double) * nv, st);
  cudaMemsetAsync(a->cont, 0, sizeof(int) * N, st);
  if (n) {
    contarLancamento();
    k_adj_p2g<<<gridDe(n), TB, 0, st>>>(D, E, n, U, UW, V, VW, a->cont);
  }
  contarLancamento();
  k_adj_tipos<<<gridDe(N), TB, 0, st>>>(D, a->cont, tipo);
  const int nf = nu > nv ? nu : nv;
  contarLancamento();
  k_adj_faces<<<gridDe(nf), TB, 0, st>>>(D, U, UW, V, VW, a->u, a->v);
  contarLancamento();
  k_adj_div<<<gridDe(N), TB, 0, st>>>(D, tipo, a->u, a->v, a->b);
  int r = resolver(a, tipo, a->b, a->q, &a->itFrente);
  if (r) return r;
  uint8_t* val = f ? f->val : a->valT;  // (CAMADAS_EXT + 1) x (nu + nv)
  contarLancamento();
  k_adj_gradiente<<<gridDe(nf), TB, 0, st>>>(D, tipo, a->q, a->u, a->v, val, val + nu);
  double *ua = a->u, *va = a->v, *ub = a->u2, *vb = a->v2;
  for (int l = 0; l < CAMADAS_EXT; l++) {
    uint8_t* m0 = val + (size_t)l * (nu + nv);
    uint8_t* m1 = val + (size_t)(l + 1) * (nu + nv);
    contarLancamento();
    k_adj_extrap<<<gridDe(nu), TB, 0, st>>>(ua, m0, ub, m1, D.nx + 1, D.ny);
    contarLancamento();
    k_adj_extrap<<<gridDe(nv), TB, 0, st>>>(va, m0 + nu, vb, m1 + nu, D.nx, D.ny + 1);
    double* t = ua;
    ua = ub;
    ub = t;
    t = va;
    va = vb;
    vb = t;
  }
  Fita tmp{};
  Fita& F = f ? *f : tmp;
  if (f) {
    cudaMemcpyAsync(f->ug, ua, sizeof(double) * nu, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(f->vg, va, sizeof(double) * nv, cudaMemcpyDeviceToDevice, st);
  } else {
    F.xm = a->fxm;  // scratch (the tape's first step area) when not recording
    F.micro = a->fmicro;
    F.bits = a->fbits;
  }
  Estado S = estado(a->bufS, cap);
  if (n) {
    contarLancamento();
    k_adj_g2p<<<gridDe(n), TB, 0, st>>>(D, E, n, cap, ua, va, F, S, a->vivo);
  }
  int* vivos = f ? f->vivos : a->fvivos;
  contarLancamento();
  k_adj_compactar<<<1, 1024, 0, st>>>(S, a->vivo, n, E, vivos, a->nVivosD);
  int nv2 = 0;
  if (cudaMemcpyAsync(&nv2, a->nVivosD, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return TQ_E_CUDA;
  if (f) f->nVivos = nv2;
  return nv2;
}

}  // namespace

extern "C" {

int tq_adj_create(const tq_adj_scene* d, int32_t device, tq_adj** out) {
  if (!d || !out) return TQ_E_ARG;
  *out = nullptr;
  if (d->nx < 16 || d->ny < 16 || !(d->h > 0) || !(d->dt > 0) || d->steps < 1 || d->n_particles < 0 ||
      d->faucet_per_step < 0 || !d->sdf || !d->target || (d->n_particles > 0 && !d->positions) ||
      (d->faucet_per_step > 0 && !d->faucet_positions) || (long long)d->nx * d->ny > (1LL << 24))
    return TQ_E_ARG;
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess || device < 0 || device >= nd) return TQ_E_NODEV;
  if (cudaSetDevice(device) != cudaSuccess) return TQ_E_CUDA;
  tq_adj* a = new (std::nothrow) tq_adj();
  if (!a) return TQ_E_NOMEM;
  a->passos = d->steps;
  a->K = d->checkpoint_every > 0 ? d->checkpoint_every : 10;
  a->n0 = d->n_particles;
  a->nf = d->faucet_per_step;
  a->cap = a->n0 + a->nf * a->passos + 1;
  a->N = d->nx * d->ny;
  a->nu = (d->nx + 1) * d->ny;
  a->nv = d->nx * (d->ny + 1);
  Dispositivo& D = a->D;
  D.nx = d->nx, D.ny = d->ny, D.N = a->N, D.nu = a->nu, D.nv = a->nv, D.mw = 2 * d->nx, D.mh = 2 * d->ny;
  D.h = d->h, D.dt = d->dt, D.gx = d->gravity[0], D.gy = d->gravity[1];
  D.vmax = (MICROPASSO * MAX_MICROPASSOS * d->h) / d->dt;
  const int cap = a->cap, N = a->N, nu = a->nu, nv = a->nv, K = a->K;
  const int nck = a->passos / K + 1;
  bool ok = cudaStreamCreateWithFlags(&a->s, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && alocar(a, &a->sdf, (size_t)4 * N) && alocar(a, &a->solido, N) && alocar(a, &a->pos0, 2 * (size_t)cap) &&
       alocar(a, &a->C0, 4 * (size_t)cap) && alocar(a, &a->fpos, (size_t)2 * a->nf * a->passos + 2) &&
       alocar(a, &a->alvo, N) && alocar(a, &a->aceitos, (size_t)a->nf * a->passos + 1) &&
       alocar(a, &a->bufE, 8 * (size_t)cap) && alocar(a, &a->bufS, 8 * (size_t)cap) && alocar(a, &a->vivo, cap) &&
       alocar(a, &a->nVivosD, 1) && alocar(a, &a->ckpt, (size_t)nck * 8 * cap) && alocar(a, &a->U, nu) &&
       alocar(a, &a->V, nv) && alocar(a, &a->UW, nu) && alocar(a, &a->VW, nv) && alocar(a, &a->u, nu) &&
       alocar(a, &a->v, nv) && alocar(a, &a->u2, nu) && alocar(a, &a->v2, nv) && alocar(a, &a->b, N) &&
       alocar(a, &a->q, N) && alocar(a, &a->rho, N) && alocar(a, &a->termo, N) && alocar(a, &a->rhob, N) &&
       alocar(a, &a->cont, N) && alocar(a, &a->tipo, N) && alocar(a, &a->valT, (size_t)(CAMADAS_EXT + 1) * (nu + nv)) &&
       alocar(a, &a->fP, (size_t)K * 8 * cap) && alocar(a, &a->fU, (size_t)K * nu) && alocar(a, &a->fV, (size_t)K * nv) &&
       alocar(a, &a->fUW, (size_t)K * nu) && alocar(a, &a->fVW, (size_t)K * nv) && alocar(a, &a->fug, (size_t)K * nu) &&
       alocar(a, &a->fvg, (size_t)K * nv) && alocar(a, &a->fxm, (size_t)K * cap * (MMAX + 1) * 2) &&
       alocar(a, &a->ftipo, (size_t)K * N) && alocar(a, &a->fval, (size_t)K * (CAMADAS_EXT + 1) * (nu + nv)) &&
       alocar(a, &a->fbits, (size_t)K * cap) && alocar(a, &a->fmicro, (size_t)K * cap) &&
       alocar(a, &a->fvivos, (size_t)K * cap) && alocar(a, &a->bufB, 8 * (size_t)cap) &&
       alocar(a, &a->bufBin, 8 * (size_t)cap) && alocar(a, &a->ugb, nu) && alocar(a, &a->vgb, nv) &&
       alocar(a, &a->ugb2, nu) && alocar(a, &a->vgb2, nv) && alocar(a, &a->qb, N) && alocar(a, &a->lam, N) &&
       alocar(a, &a->Ub, nu) && alocar(a, &a->UWb, nu) && alocar(a, &a->Vb, nv) && alocar(a, &a->VWb, nv) &&
       alocar(a, &a->r, N) && alocar(a, &a->z, N) && alocar(a, &a->zv, N) && alocar(a, &a->p, N) &&
       alocar(a, &a->ap, N) && alocar(a, &a->parc, SOMA_CTAS) && alocar(a, &a->esc, E_N) && alocar(a, &a->bf, N) &&
       alocar(a, &a->xf, N) && alocar(a, &a->tipoCG, N) && alocar(a, &a->xCG, N);
  if (ok) a->pcg = criarPcg(d->nx, d->ny, TQ_PREC_FP32, TQ_ENGINE_PLAIN);
  if (!ok || !a->pcg) {
    tq_adj_destroy(a);
    return TQ_E_NOMEM;
  }
  // scene data to the device (doubles from the caller's floats)
  std::vector<double> tmp;
  auto subir = [&](double* dst, const float* src, size_t n) {
    tmp.assign(n, 0.0);
    for (size_t k = 0; k < n && src; k++) tmp[k] = src[k];
    return cudaMemcpy(dst, tmp.data(), n * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess;
  };
  ok = cudaMemcpy(a->sdf, d->sdf, sizeof(float) * 4 * N, cudaMemcpyHostToDevice) == cudaSuccess &&
       subir(a->pos0, d->positions, 2 * (size_t)a->n0) && subir(a->C0, d->affine, 4 * (size_t)a->n0) &&
       subir(a->fpos, d->faucet_positions, (size_t)2 * a->nf * a->passos) && subir(a->alvo, d->target, N);
  // solid cells (Cena.celulaSolida, js/cena.js:119-127) and the faucet's insert filter
  // (adicionar, js/fisica-cpu.js:100: SDF > RAIO_PARTICULA + 0.05), on the host
  std::vector<uint8_t> sol(N);
  const int mw = 2 * d->nx;
  for (int j = 0; j < d->ny; j++)
    for (int i = 0; i < d->nx; i++) {
      const float* m = d->sdf;
      const int x = 2 * i, y = 2 * j;
      const double s = (double)m[(size_t)y * mw + x] + m[(size_t)y * mw + x + 1] + m[(size_t)(y + 1) * mw + x] +
                       m[(size_t)(y + 1) * mw + x + 1];
      sol[i + j * d->nx] = s < 0;
    }
  std::vector<int> acc((size_t)a->nf * a->passos + 1, 0);
  a->nAceitos.assign(a->passos, 0);
  for (int s = 0; s < a->passos; s++) {
    int c = 0;
    for (int k = 0; k < a->nf; k++) {
      const double x = d->faucet_positions[((size_t)s * a->nf + k) * 2], y = d->faucet_positions[((size_t)s * a->nf + k) * 2 + 1];
      // Cena.distancia on the host, in double (js/cena.js:102-106, 156-165)
      double fx = (x / d->h) * 2 - 0.5, fy = (y / d->h) * 2 - 0.5;
      const int w = mw, hh = 2 * d->ny;
      fx = fx < 0 ? 0 : fx > w - 1 ? w - 1 : fx;
      fy = fy < 0 ? 0 : fy > hh - 1 ? hh - 1 : fy;
      const int x0 = (int)std::fmin(std::floor(fx), (double)(w - 2)), y0 = (int)std::fmin(std::floor(fy), (double)(hh - 2));
      const double tx = fx - x0, ty = fy - y0;
      const size_t q = (size_t)y0 * w + x0;
      const double sd = (d->sdf[q] * (1 - tx) + d->sdf[q + 1] * tx) * (1 - ty) +
                        (d->sdf[q + w] * (1 - tx) + d->sdf[q + w + 1] * tx) * ty;
      if (sd > RAIO_PARTICULA + 0.05) acc[(size_t)s * a->nf + c++] = k;
    }
    a->nAceitos[s] = c;
  }
  ok = ok && cudaMemcpy(a->solido, sol.data(), N, cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemcpy(a->aceitos, acc.data(), acc.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
  D.sdf = a->sdf;
  D.solido = a->solido;
  // the segment's tape
  a->fita.resize(K);
  for (int k = 0; k < K; k++) {
    Fita& f = a->fita[k];
    f.P = a->fP + (size_t)k * 8 * cap;
    f.U = a->fU + (size_t)k * nu;
    f.V = a->fV + (size_t)k * nv;
    f.UW = a->fUW + (size_t)k * nu;
    f.VW = a->fVW + (size_t)k * nv;
    f.ug = a->fug + (size_t)k * nu;
    f.vg = a->fvg + (size_t)k * nv;
    f.xm = a->fxm + (size_t)k * cap * (MMAX + 1) * 2;
    f.tipo = a->ftipo + (size_t)k * N;
    f.val = a->fval + (size_t)k * (CAMADAS_EXT + 1) * (nu + nv);
    f.bits = a->fbits + (size_t)k * cap;
    f.micro = a->fmicro + (size_t)k * cap;
    f.vivos = a->fvivos + (size_t)k * cap;
  }
  if (!ok) {
    tq_adj_destroy(a);
    return TQ_E_CUDA;
  }
  *out = a;
  return TQ_OK;
}

int tq_adj_destroy(tq_adj* a) {
  if (!a) return TQ_OK;
  if (a->s) cudaStreamSynchronize(a->s);
  if (a->grafoCG) cudaGraphExecDestroy(a->grafoCG);
  destruirPcg(a->pcg);
  for (void* p : a->mem) cudaFree(p);
  if (a->s) cudaStreamDestroy(a->s);
  delete a;
  return TQ_OK;
}

int tq_adj_forward(tq_adj* a, const float* v0, const double* theta, double* loss) {
  if (!a || !theta || !loss || (a->n0 > 0 && !v0)) return TQ_E_ARG;
  const int cap = a->cap;
  a->theta[0] = theta[0];
  a->theta[1] = theta[1];
  float* dv = nullptr;
  if (a->n0) {
    if (cudaMalloc(&dv, sizeof(float) * 2 * a->n0) != cudaSuccess) return TQ_E_NOMEM;
    cudaMemcpyAsync(dv, v0, sizeof(float) * 2 * a->n0, cudaMemcpyHostToDevice, a->s);
    contarLancamento();
    k_adj_entrada_v<<<gridDe(a->n0), TB, 0, a->s>>>(estado(a->bufE, cap), a->n0, dv, a->pos0, a->C0);
  }
  int n = a->n0;
  a->nCkpt.assign(a->passos / a->K + 1, 0);
  for (int s = 0; s < a->passos; s++) {
    if (s % a->K == 0) {  // checkpoint
      cudaMemcpyAsync(a->ckpt + (size_t)(s / a->K) * 8 * cap, a->bufE, sizeof(double) * 8 * cap,
                      cudaMemcpyDeviceToDevice, a->s);
      a->nCkpt[s / a->K] = n;
    }
    n = passoFrente(a, s, n, nullptr);
    if (n < 0) {
      if (dv) cudaFree(dv);
      return n;
    }
  }
  a->nFinal = n;
  cudaMemsetAsync(a->rho, 0, sizeof(double) * a->N, a->s);
  if (n) {
    contarLancamento();
    k_adj_densidade<<<gridDe(n), TB, 0, a->s>>>(a->D, estado(a->bufE, cap), n, a->rho);
  }
  contarLancamento();
  k_adj_perda<<<gridDe(a->N), TB, 0, a->s>>>(a->D, a->rho, a->alvo, a->termo, a->rhob);
  *loss = somaHost(a, a->termo, nullptr, a->N);
  // the final state's position adjoint (the loss's), kept for backward
  if (n) {
    contarLancamento();
    k_adj_perda_T<<<gridDe(n), TB, 0, a->s>>>(a->D, estado(a->bufE, cap), n, a->rhob, estado(a->bufB, cap));
  }
  cudaError_t e = cudaStreamSynchronize(a->s);
  if (dv) cudaFree(dv);
  if (e != cudaSuccess || cudaGetLastError() != cudaSuccess) return TQ_E_CUDA;
  a->temFrente = true;
  return TQ_OK;
}

int tq_adj_backward(tq_adj* a, double grad_loss, float* dv0, double* dtheta) {
  if (!a || !dtheta || (a->n0 > 0 && !dv0)) return TQ_E_ARG;
  if (!a->temFrente) return TQ_E_STATE;
  const int cap = a->cap, nu = a->nu, nv = a->nv, N = a->N, K = a->K;
  cudaStream_t st = a->s;
  double gth[2] = {0, 0};
  // bufB holds the adjoint of the state after the last step (from the forward run)
  const int nseg = (a->passos + K - 1) / K;
  for (int sg = nseg - 1; sg >= 0; sg--) {
    const int s0 = sg * K, s1 = std::min(a->passos, s0 + K);
    // recompute the segment from its checkpoint, recording the tape (bufB is not touched)
    cudaMemcpyAsync(a->bufE, a->ckpt + (size_t)sg * 8 * cap, sizeof(double) * 8 * cap, cudaMemcpyDeviceToDevice, st);
    int n = a->nCkpt[sg];
    for (int s = s0; s < s1; s++) {
      n = passoFrente(a, s, n, &a->fita[s - s0]);
      if (n < 0) return n;
    }
    // back through the segment
    for (int s = s1 - 1; s >= s0; s--) {
      Fita& f = a->fita[s - s0];
      Estado B = estado(a->bufB, cap), Bin = estado(a->bufBin, cap);
      contarLancamento();
      k_adj_zerar<<<256, TB, 0, st>>>(a->bufBin, (size_t)8 * cap);
      cudaMemsetAsync(a->ugb, 0, sizeof(double) * nu, st);
      cudaMemsetAsync(a->vgb, 0, sizeof(double) * nv, st);
      if (f.nVivos) {
        contarLancamento();
        k_adj_g2p_T<<<gridDe(f.nVivos), TB, 0, st>>>(a->D, f, cap, B, Bin, a->ugb, a->vgb);
      }
      // extrapolation layers in reverse
      for (int l = CAMADAS_EXT - 1; l >= 0; l--) {
        const uint8_t* m0 = f.val + (size_t)l * (nu + nv);
        const uint8_t* m1 = f.val + (size_t)(l + 1) * (nu + nv);
        cudaMemcpyAsync(a->ugb2, a->ugb, sizeof(double) * nu, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(a->vgb2, a->vgb, sizeof(double) * nv, cudaMemcpyDeviceToDevice, st);
        contarLancamento();
        k_adj_extrap_T<<<gridDe(nu), TB, 0, st>>>(a->ugb, m0, m1, a->ugb2, a->D.nx + 1, a->D.ny);
        contarLancamento();
        k_adj_extrap_T<<<gridDe(nv), TB, 0, st>>>(a->vgb, m0 + nu, m1 + nu, a->vgb2, a->D.nx, a->D.ny + 1);
        std::swap(a->ugb, a->ugb2);
        std::swap(a->vgb, a->vgb2);
      }
      // gradient reverse (gather per cell), the adjoint solve, divergence / walls / normalisation
      contarLancamento();
      k_adj_grad_T<<<gridDe(N), TB, 0, st>>>(a->D, f.tipo, a->ugb, a->vgb, a->qb);
      int r = resolver(a, f.tipo, a->qb, a->lam, &a->itTras);
      if (r) return r;
      const int nfc = nu > nv ? nu : nv;
      contarLancamento();
      k_adj_faces_T<<<gridDe(nfc), TB, 0, st>>>(a->D, f.tipo, a->lam, a->ugb, a->vgb, f.U, f.UW, f.V, f.VW, a->Ub,
                                                a->UWb, a->Vb, a->VWb);
      // P2G reverse: the state adjoint at the step's start
      if (f.n) {
        contarLancamento();
        k_adj_p2g_T<<<gridDe(f.n), TB, 0, st>>>(a->D, f, cap, a->Ub, a->UWb, a->Vb, a->VWb, Bin);
      }
      // the faucet's particles of this step: their velocity is theta
      const int na = a->nAceitos[s], nAnt = f.n - na;
      if (na) {
        gth[0] += somaHost(a, Bin.c[2] + nAnt, nullptr, na);
        gth[1] += somaHost(a, Bin.c[3] + nAnt, nullptr, na);
      }
      std::swap(a->bufB, a->bufBin);
    }
  }
  if (a->n0) {
    float* dv = nullptr;
    if (cudaMalloc(&dv, sizeof(float) * 2 * a->n0) != cudaSuccess) return TQ_E_NOMEM;
    contarLancamento();
    k_adj_saida_v<<<gridDe(a->n0), TB, 0, st>>>(estado(a->bufB, cap), a->n0, grad_loss, dv);
    cudaMemcpyAsync(dv0, dv, sizeof(float) * 2 * a->n0, cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    cudaFree(dv);
    if (e != cudaSuccess) return TQ_E_CUDA;
  }
  dtheta[0] = gth[0] * grad_loss;
  dtheta[1] = gth[1] * grad_loss;
  // the final-state adjoint is consumed: a second backward needs a new forward
  a->temFrente = false;
  return cudaGetLastError() == cudaSuccess ? TQ_OK : TQ_E_CUDA;
}

}  // extern "C"
