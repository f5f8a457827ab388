// adjunto_oracle.cpp — TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
//
// The FP64 CPU forward and hand-written adjoint of the differentiable configuration of the
// substep: the checker of the CUDA adjoint (tq_adj_*), and the model its finite-difference tests
// differentiate.  The reference has no adjoint; the forward restates SimulacaoCPU.subpasso
// (js/fisica-cpu.js:176-189) with air tracking off (opcoes.ar = false), surface tension 0 and the
// density correction off (tauDensidade -> infinity), so a substep is: #paraGrade (APIC P2G,
// :198-267), #gravidadeEFronteira (:271-291), #tipos (:293-299), #classificar without the density
// and air terms (:456-481), #pressao (an exact solve of resolverPCG's system, js/pressao-cpu.js:
// 296-402), #gradiente (:519-545), #extrapolar (:547-552, 673-690) and #paraParticulas (G2P with
// micro-steps and wall collisions, :556-661).  Foam and dye do not enter the loss and are left
// out.  Its discrete structure — cell flags, valid masks, the faces with weight, micro-step counts,
// the speed clamps, collision branches, kills and the faucet's insert filter — is recorded by a
// forward run and can be frozen for later runs, so central finite differences differentiate the
// same smooth map the adjoint does.
//
// Loss: sum over cells of (min(1, rho/4) - target)^2, rho the bilinear particle density at cell
// centres (#paraGrade's `densidade`, :244-254; the fraction of #superficie, :309).  Controls: the
// initial particle velocities and the faucet velocity theta (2 scalars) given to the particles the
// faucet emits at the start of every step (js/principal.js:301-321's jet, positions given).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "oracle.h"

// tanque_oracle.cpp: A q = b on the water cells of `tipo` (FP64 MGPCG to a relative 1e-13).
void resolverExatoFP64(int nx, int ny, const uint8_t* tipo, const double* b, double* q);

namespace {

constexpr double RAIO_PARTICULA = 0.3, MICROPASSO = 0.8, MAX_MICROPASSOS = 4, SDF_MAX = 10;
constexpr int RES = 2, CAMADAS = 2;
constexpr uint8_t SOLIDO = 0, AGUA = 1, AR = 2;

inline int clampi(int v, int a, int b) { return v < a ? a : v > b ? b : v; }

// Cena.#bilinear (js/cena.js:156-165) on the mask, with its derivatives in mask pixels.
struct Sdf {
  const float* s;
  int w, hh;
  double h;
  double bil(double fx, double fy, double* dfx, double* dfy) const {
    bool cx = false, cy = false;
    if (fx < 0) { fx = 0; cx = true; }
    else if (fx > w - 1) { fx = w - 1; cx = true; }
    if (fy < 0) { fy = 0; cy = true; }
    else if (fy > hh - 1) { fy = hh - 1; cy = true; }
    int x0 = (int)std::min(std::floor(fx), (double)(w - 2)), y0 = (int)std::min(std::floor(fy), (double)(hh - 2));
    double tx = fx - x0, ty = fy - y0;
    size_t k = (size_t)y0 * w + x0;
    double a = s[k], b = s[k + 1], c = s[k + w], d = s[k + w + 1];
    if (dfx) *dfx = cx ? 0.0 : (b - a) * (1 - ty) + (d - c) * ty;
    if (dfy) *dfy = cy ? 0.0 : (c - a) * (1 - tx) + (d - b) * tx;
    return (a * (1 - tx) + b * tx) * (1 - ty) + (c * (1 - tx) + d * tx) * ty;
  }
  // Cena.distancia (js/cena.js:102-106) and its gradient in metres
  double dist(double x, double y, double* gx, double* gy) const {
    double dfx, dfy;
    double v = bil((x / h) * RES - 0.5, (y / h) * RES - 0.5, &dfx, &dfy);
    if (gx) *gx = dfx * RES / h;
    if (gy) *gy = dfy * RES / h;
    return v;
  }
  // Cena.normal (js/cena.js:109-116) and its Jacobian J[i][j] = d n_i / d x_j
  void normal(double x, double y, double n[2], double J[2][2]) const {
    double fx = (x / h) * RES - 0.5, fy = (y / h) * RES - 0.5;
    double a1, a2, b1, b2, c1, c2, d1, d2;
    double g0 = bil(fx + 1, fy, &a1, &a2) - bil(fx - 1, fy, &b1, &b2);
    double g1 = bil(fx, fy + 1, &c1, &c2) - bil(fx, fy - 1, &d1, &d2);
    double G[2][2] = {{(a1 - b1) * RES / h, (a2 - b2) * RES / h}, {(c1 - d1) * RES / h, (c2 - d2) * RES / h}};
    double nn = std::hypot(g0, g1);
    if (nn > 1e-9) {
      n[0] = g0 / nn;
      n[1] = g1 / nn;
      double P[2][2] = {{(1 - n[0] * n[0]) / nn, -n[0] * n[1] / nn}, {-n[1] * n[0] / nn, (1 - n[1] * n[1]) / nn}};
      for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) J[i][j] = P[i][0] * G[0][j] + P[i][1] * G[1][j];
    } else {
      n[0] = 0;
      n[1] = 1;
      J[0][0] = J[0][1] = J[1][0] = J[1][1] = 0;
    }
  }
};

// Bilinear stencil of a particle on one staggered grid: u faces (kind 0, nodes at (i h, (j+1/2) h),
// (nx+1) x ny) or v faces (kind 1, nodes at ((i+1/2) h, j h), nx x (ny+1)) or cell centres (kind 2,
// the density, nx x ny), with the clamps of js/fisica-cpu.js:214-248.
struct Estencil {
  int i0, j0, W;  // lower-left node and the row width
  double tx, ty;
};
inline Estencil estencil(int kind, double x, double y, int nx, int ny, double h) {
  const double inv = 1 / h;
  Estencil e;
  double fx, fy;
  if (kind == 0) {
    fx = x * inv, fy = y * inv - 0.5;
    e.i0 = clampi((int)std::floor(fx), 0, nx - 1), e.j0 = clampi((int)std::floor(fy), 0, ny - 2), e.W = nx + 1;
  } else if (kind == 1) {
    fx = x * inv - 0.5, fy = y * inv;
    e.i0 = clampi((int)std::floor(fx), 0, nx - 2), e.j0 = clampi((int)std::floor(fy), 0, ny - 1), e.W = nx;
  } else {
    fx = x * inv - 0.5, fy = y * inv - 0.5;
    e.i0 = clampi((int)std::floor(fx), 0, nx - 2), e.j0 = clampi((int)std::floor(fy), 0, ny - 2), e.W = nx;
  }
  e.tx = fx - e.i0;
  e.ty = fy - e.j0;
  return e;
}

struct Particula {
  double x, y, vx, vy, cux, cuy, cvx, cvy;
};

// What the forward records of one step (and the frozen structure for the next runs).
struct Passo {
  std::vector<Particula> P;      // state at the step's start (after the faucet)
  std::vector<double> U, V, UW, VW;  // P2G sums
  std::vector<uint8_t> tipo;
  std::vector<uint8_t> temU, temV;   // faces with weight (UW > 0)
  std::vector<double> ug, vg;        // grid velocities G2P reads (after extrapolation)
  std::vector<uint8_t> valU[CAMADAS + 1], valV[CAMADAS + 1];  // valid masks before each layer
  // G2P, per particle
  std::vector<int> micro;
  std::vector<uint8_t> clampV, morta;
  std::vector<uint8_t> col, corta, clampW;  // per particle x MAX_MICROPASSOS
  std::vector<double> xm;                   // positions before each micro-move (2 per slot)
  std::vector<uint8_t> aceitaTorneira;      // the faucet's insert filter
  std::vector<int> vivos;                   // indices (into P) of the particles alive after G2P
};

struct Adj {
  int nx, ny, N, nu, nv;
  double h, dt, g[2];
  int passos, n0, nf;
  Sdf sdf;
  std::vector<float> mascara;
  std::vector<double> pos0, C0, fpos, alvo;
  std::vector<Passo> fita;
  bool gravado = false;
  double perda = 0;
  std::vector<double> rho;  // final density
  std::vector<Particula> fim;
};

// ---------------------------------------------------------------- pressure: A q = b (water cells)
// resolverPCG's system (js/pressao-cpu.js:84-93 with the true types): k q - sum of water
// neighbours' q, k the free (non-wall) neighbours, air q = 0; solved exactly, not with the
// reference's three iterations, by the oracle's own MGPCG in double storage to a relative 1e-13
// (tanque_oracle.cpp).  A is symmetric, so the adjoint solve is the same call.
void resolver(const Adj& a, const std::vector<uint8_t>& tipo, const std::vector<double>& b, std::vector<double>& q) {
  q.assign(a.N, 0.0);
  resolverExatoFP64(a.nx, a.ny, tipo.data(), b.data(), q.data());
}

// ---------------------------------------------------------------- grid sampling (G2P)
// Velocity and affine terms at (x, y) (js/fisica-cpu.js:566-591), with their derivatives:
// d(vx)/dx = cux, d(vx)/dy = cuy (likewise v), d(cux)/dy = d(cuy)/dx = kxy (the cross term).
struct Amostra {
  double vx, vy, cux, cuy, cvx, cvy, kux, kvx;  // kux = d cux/dy = d cuy/dx; kvx for v
  Estencil eu, ev;
};
Amostra amostrar(const Adj& a, const std::vector<double>& ug, const std::vector<double>& vg, double x, double y) {
  const double inv = 1 / a.h;
  Amostra s{};
  s.eu = estencil(0, x, y, a.nx, a.ny, a.h);
  s.ev = estencil(1, x, y, a.nx, a.ny, a.h);
  for (int b = 0; b < 2; b++)
    for (int aa = 0; aa < 2; aa++) {
      double wx = aa ? s.eu.tx : 1 - s.eu.tx, wy = b ? s.eu.ty : 1 - s.eu.ty;
      double val = ug[s.eu.i0 + aa + (s.eu.j0 + b) * s.eu.W];
      s.vx += wx * wy * val;
      s.cux += (aa ? 1 : -1) * wy * inv * val;
      s.cuy += wx * (b ? 1 : -1) * inv * val;
      s.kux += (aa ? 1 : -1) * (b ? 1 : -1) * inv * inv * val;
      wx = aa ? s.ev.tx : 1 - s.ev.tx, wy = b ? s.ev.ty : 1 - s.ev.ty;
      val = vg[s.ev.i0 + aa + (s.ev.j0 + b) * s.ev.W];
      s.vy += wx * wy * val;
      s.cvx += (aa ? 1 : -1) * wy * inv * val;
      s.cvy += wx * (b ? 1 : -1) * inv * val;
      s.kvx += (aa ? 1 : -1) * (b ? 1 : -1) * inv * inv * val;
    }
  return s;
}
// Transpose of amostrar: adjoints of (vx, vy, cux, cuy, cvx, cvy) into the grid (ugb, vgb) and into
// the position (xb, yb).
void amostrarT(const Adj& a, const Amostra& s, const double bv[6], std::vector<double>& ugb, std::vector<double>& vgb,
               double* xb, double* yb) {
  const double inv = 1 / a.h;
  for (int b = 0; b < 2; b++)
    for (int aa = 0; aa < 2; aa++) {
      double wx = aa ? s.eu.tx : 1 - s.eu.tx, wy = b ? s.eu.ty : 1 - s.eu.ty;
      ugb[s.eu.i0 + aa + (s.eu.j0 + b) * s.eu.W] +=
          bv[0] * wx * wy + bv[2] * (aa ? 1 : -1) * wy * inv + bv[3] * wx * (b ? 1 : -1) * inv;
      wx = aa ? s.ev.tx : 1 - s.ev.tx, wy = b ? s.ev.ty : 1 - s.ev.ty;
      vgb[s.ev.i0 + aa + (s.ev.j0 + b) * s.ev.W] +=
          bv[1] * wx * wy + bv[4] * (aa ? 1 : -1) * wy * inv + bv[5] * wx * (b ? 1 : -1) * inv;
    }
  *xb += bv[0] * s.cux + bv[1] * s.cvx + bv[3] * s.kux + bv[5] * s.kvx;
  *yb += bv[0] * s.cuy + bv[1] * s.cvy + bv[2] * s.kux + bv[4] * s.kvx;
}

// Speed clamp v * vmax / |v| and its adjoint (when active).
inline void limitarT(double vx, double vy, double vmax, double* bx, double* by) {
  double v = std::hypot(vx, vy), nx = vx / v, ny = vy / v, f = vmax / v;
  double dot = *bx * nx + *by * ny;
  *bx = f * (*bx - dot * nx);
  *by = f * (*by - dot * ny);
}

// ---------------------------------------------------------------- one forward step
// `gravar`: record the structure; else the recorded structure of step `s` is applied.
void passo(Adj& a, int s, std::vector<Particula>& P, double th0, double th1, bool gravar) {
  Passo& T = a.fita[s];
  const int nx = a.nx, ny = a.ny, N = a.N, nu = a.nu, nv = a.nv;
  const double h = a.h, dt = a.dt;
  // the faucet: its particles of this step (velocity theta, no affine term), through adicionar's
  // filter (js/fisica-cpu.js:100: SDF > RAIO_PARTICULA + 0.05; no full-cell check)
  if (gravar) T.aceitaTorneira.assign(a.nf, 0);
  for (int k = 0; k < a.nf; k++) {
    double x = a.fpos[((size_t)s * a.nf + k) * 2], y = a.fpos[((size_t)s * a.nf + k) * 2 + 1];
    if (gravar) T.aceitaTorneira[k] = a.sdf.dist(x, y, nullptr, nullptr) > RAIO_PARTICULA + 0.05;
    if (T.aceitaTorneira[k]) P.push_back({x, y, th0, th1, 0, 0, 0, 0});
  }
  T.P = P;
  const int n = (int)P.size();
  // P2G (js/fisica-cpu.js:198-267), float sums in double
  T.U.assign(nu, 0); T.UW.assign(nu, 0); T.V.assign(nv, 0); T.VW.assign(nv, 0);
  std::vector<int> cont(N, 0);
  for (const Particula& p : P) {
    Estencil e = estencil(0, p.x, p.y, nx, ny, h);
    for (int b = 0; b < 2; b++)
      for (int aa = 0; aa < 2; aa++) {
        double w = (aa ? e.tx : 1 - e.tx) * (b ? e.ty : 1 - e.ty);
        double dx = (e.i0 + aa) * h - p.x, dy = (e.j0 + b + 0.5) * h - p.y;
        int idx = e.i0 + aa + (e.j0 + b) * e.W;
        T.U[idx] += w * (p.vx + p.cux * dx + p.cuy * dy);
        T.UW[idx] += w;
      }
    e = estencil(1, p.x, p.y, nx, ny, h);
    for (int b = 0; b < 2; b++)
      for (int aa = 0; aa < 2; aa++) {
        double w = (aa ? e.tx : 1 - e.tx) * (b ? e.ty : 1 - e.ty);
        double dx = (e.i0 + aa + 0.5) * h - p.x, dy = (e.j0 + b) * h - p.y;
        int idx = e.i0 + aa + (e.j0 + b) * e.W;
        T.V[idx] += w * (p.vy + p.cvx * dx + p.cvy * dy);
        T.VW[idx] += w;
      }
    int ci = clampi((int)std::floor(p.x / h), 0, nx - 1), cj = clampi((int)std::floor(p.y / h), 0, ny - 1);
    cont[ci + cj * nx]++;
  }
  std::vector<uint8_t> solido(N);
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      // Cena.celulaSolida (js/cena.js:119-127): the sum of the cell's 4 mask samples < 0
      int x = i * RES, y = j * RES;
      const float* m = a.mascara.data();
      double sm = (double)m[(size_t)y * a.sdf.w + x] + m[(size_t)y * a.sdf.w + x + 1] + m[(size_t)(y + 1) * a.sdf.w + x] +
                  m[(size_t)(y + 1) * a.sdf.w + x + 1];
      solido[i + j * nx] = sm < 0;
    }
  if (gravar) {
    T.temU.resize(nu);
    T.temV.resize(nv);
    for (int k = 0; k < nu; k++) T.temU[k] = T.UW[k] > 0;
    for (int k = 0; k < nv; k++) T.temV[k] = T.VW[k] > 0;
    T.tipo.resize(N);
    for (int c = 0; c < N; c++) T.tipo[c] = solido[c] ? SOLIDO : cont[c] > 0 ? AGUA : AR;  // #tipos
  }
  std::vector<double> u(nu, 0.0), v(nv, 0.0);
  // (a frozen run can meet a weightless face the recorded run weighted: it stays 0, not 0/0)
  for (int k = 0; k < nu; k++) u[k] = T.temU[k] && T.UW[k] > 0 ? T.U[k] / T.UW[k] : 0;
  for (int k = 0; k < nv; k++) v[k] = T.temV[k] && T.VW[k] > 0 ? T.V[k] / T.VW[k] : 0;
  // #gravidadeEFronteira (:271-291)
  for (int j = 0; j < ny; j++)
    for (int i = 0; i <= nx; i++) {
      int k = i + j * (nx + 1);
      if (T.temU[k]) u[k] += a.g[0] * dt;
      if (i == 0 || i == nx || solido[i - 1 + j * nx] || solido[i + j * nx]) u[k] = 0;
    }
  for (int j = 0; j <= ny; j++)
    for (int i = 0; i < nx; i++) {
      int k = i + j * nx;
      if (T.temV[k]) v[k] += a.g[1] * dt;
      if (j == 0 || j == ny || solido[i + (j - 1) * nx] || solido[i + j * nx]) v[k] = 0;
    }
  const std::vector<uint8_t>& tipo = T.tipo;
  // #classificar without the density and air terms, #pressao's solve
  std::vector<double> b(N, 0.0), q;
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      int c = i + j * nx;
      if (tipo[c] != AGUA) continue;
      b[c] = -(u[i + 1 + j * (nx + 1)] - u[i + j * (nx + 1)] + v[i + (j + 1) * nx] - v[i + j * nx]);
    }
  resolver(a, tipo, b, q);
  // #gradiente (:519-545)
  std::vector<uint8_t> vu(nu), vv(nv);
  for (int j = 0; j < ny; j++)
    for (int i = 0; i <= nx; i++) {
      int k = i + j * (nx + 1);
      uint8_t tl = i > 0 ? tipo[i - 1 + j * nx] : SOLIDO, tr = i < nx ? tipo[i + j * nx] : SOLIDO;
      if (tl == SOLIDO || tr == SOLIDO) { u[k] = 0; vu[k] = 1; continue; }
      if (tl == AGUA || tr == AGUA) {
        u[k] -= (tr == AGUA ? q[i + j * nx] : 0) - (tl == AGUA ? q[i - 1 + j * nx] : 0);
        vu[k] = 1;
      } else vu[k] = 0;
    }
  for (int j = 0; j <= ny; j++)
    for (int i = 0; i < nx; i++) {
      int k = i + j * nx;
      uint8_t tb = j > 0 ? tipo[i + (j - 1) * nx] : SOLIDO, tt = j < ny ? tipo[i + j * nx] : SOLIDO;
      if (tb == SOLIDO || tt == SOLIDO) { v[k] = 0; vv[k] = 1; continue; }
      if (tb == AGUA || tt == AGUA) {
        v[k] -= (tt == AGUA ? q[i + j * nx] : 0) - (tb == AGUA ? q[i + (j - 1) * nx] : 0);
        vv[k] = 1;
      } else vv[k] = 0;
    }
  // #extrapolar (:547-552, extrapolarComponente :673-690)
  auto extrap = [](std::vector<double>& x, std::vector<uint8_t>& val, int w, int hh) {
    std::vector<double> tmp(x);
    std::vector<int> novas;
    for (int j = 0; j < hh; j++)
      for (int i = 0; i < w; i++) {
        int k = i + j * w;
        if (val[k]) continue;
        double s = 0;
        int m = 0;
        if (i > 0 && val[k - 1]) { s += x[k - 1]; m++; }
        if (i < w - 1 && val[k + 1]) { s += x[k + 1]; m++; }
        if (j > 0 && val[k - w]) { s += x[k - w]; m++; }
        if (j < hh - 1 && val[k + w]) { s += x[k + w]; m++; }
        if (m > 0) { tmp[k] = s / m; novas.push_back(k); }
      }
    x = tmp;
    for (int k : novas) val[k] = 1;
  };
  for (int l = 0; l < CAMADAS; l++) {
    T.valU[l] = vu;
    T.valV[l] = vv;
    extrap(u, vu, nx + 1, ny);
    extrap(v, vv, nx, ny + 1);
  }
  T.valU[CAMADAS] = vu;
  T.valV[CAMADAS] = vv;
  T.ug = u;
  T.vg = v;
  // #paraParticulas (:556-661) without foam and dye
  const double vmax = (MICROPASSO * MAX_MICROPASSOS * h) / dt;
  const int M = (int)MAX_MICROPASSOS;
  if (gravar) {
    T.micro.assign(n, 1);
    T.clampV.assign(n, 0);
    T.morta.assign(n, 0);
    T.col.assign((size_t)n * M, 0);
    T.corta.assign((size_t)n * M, 0);
    T.clampW.assign((size_t)n * M, 0);
  }
  T.xm.assign((size_t)n * (M + 1) * 2, 0.0);
  std::vector<Particula> saida;
  T.vivos.clear();
  for (int k = 0; k < n; k++) {
    Particula p = P[k];
    Amostra sm = amostrar(a, u, v, p.x, p.y);
    double vx = sm.vx, vy = sm.vy;
    double vel = std::hypot(vx, vy);
    if (gravar) T.clampV[k] = vel > vmax;
    if (T.clampV[k]) { vx *= vmax / vel; vy *= vmax / vel; }
    if (gravar)
      T.micro[k] = (int)std::min(MAX_MICROPASSOS, std::max(1.0, std::ceil((std::min(vel, vmax) * dt) / (MICROPASSO * h))));
    const int mi = T.micro[k];
    const double dm = dt / mi;
    double x = p.x, y = p.y;
    bool morta = false;
    for (int m = 0; m < mi; m++) {
      T.xm[((size_t)k * (M + 1) + m) * 2] = x;
      T.xm[((size_t)k * (M + 1) + m) * 2 + 1] = y;
      double wx = vx, wy = vy;
      if (mi > 1) {
        Amostra w = amostrar(a, u, v, x, y);
        wx = w.vx, wy = w.vy;
        double vw = std::hypot(wx, wy);
        if (gravar) T.clampW[(size_t)k * M + m] = vw > vmax;
        if (T.clampW[(size_t)k * M + m]) { wx *= vmax / vw; wy *= vmax / vw; }
      }
      x += wx * dm;
      y += wy * dm;
      double d = a.sdf.dist(x, y, nullptr, nullptr);
      if (gravar) T.col[(size_t)k * M + m] = d < RAIO_PARTICULA;
      if (T.col[(size_t)k * M + m]) {
        if (gravar && d < -SDF_MAX + 0.5) T.morta[k] = 1;
        if (T.morta[k]) { morta = true; break; }
        double nn[2], J[2][2];
        a.sdf.normal(x, y, nn, J);
        double empurra = (RAIO_PARTICULA - d) * h;
        x += nn[0] * empurra;
        y += nn[1] * empurra;
        double vn = vx * nn[0] + vy * nn[1];
        if (gravar) T.corta[(size_t)k * M + m] = vn < 0;
        if (T.corta[(size_t)k * M + m]) { vx -= vn * nn[0]; vy -= vn * nn[1]; }
      }
    }
    T.xm[((size_t)k * (M + 1) + mi) * 2] = x;
    T.xm[((size_t)k * (M + 1) + mi) * 2 + 1] = y;
    if (morta) continue;
    T.vivos.push_back(k);
    saida.push_back({x, y, vx, vy, sm.cux, sm.cuy, sm.cvx, sm.cvy});
  }
  P = saida;
}

// Density at cell centres (js/fisica-cpu.js:244-254) and the loss.
double perdaDe(Adj& a, const std::vector<Particula>& P) {
  const int nx = a.nx, ny = a.ny;
  a.rho.assign(a.N, 0.0);
  for (const Particula& p : P) {
    Estencil e = estencil(2, p.x, p.y, nx, ny, a.h);
    int c = e.i0 + e.j0 * nx;
    a.rho[c] += (1 - e.tx) * (1 - e.ty);
    a.rho[c + 1] += e.tx * (1 - e.ty);
    a.rho[c + nx] += (1 - e.tx) * e.ty;
    a.rho[c + nx + 1] += e.tx * e.ty;
  }
  double L = 0;
  for (int c = 0; c < a.N; c++) {
    double f = std::min(1.0, a.rho[c] / 4), d = f - a.alvo[c];
    L += d * d;
  }
  return L;
}

double frente(Adj& a, const double* v0, const double* th, bool gravar) {
  if (gravar) a.fita.assign(a.passos, Passo{});
  std::vector<Particula> P(a.n0);
  for (int k = 0; k < a.n0; k++)
    P[k] = {a.pos0[2 * k], a.pos0[2 * k + 1], v0[2 * k], v0[2 * k + 1], a.C0[4 * k], a.C0[4 * k + 1], a.C0[4 * k + 2],
            a.C0[4 * k + 3]};
  for (int s = 0; s < a.passos; s++) passo(a, s, P, th[0], th[1], gravar);
  a.fim = P;
  a.gravado = true;
  a.perda = perdaDe(a, P);
  return a.perda;
}

// ---------------------------------------------------------------- the adjoint
void tras(Adj& a, double* gv0, double* gth) {
  const int nx = a.nx, ny = a.ny, N = a.N, nu = a.nu, nv = a.nv, M = (int)MAX_MICROPASSOS;
  const double h = a.h, dt = a.dt, inv = 1 / h;
  // loss -> final particle positions
  std::vector<double> rb(N);
  for (int c = 0; c < N; c++) rb[c] = a.rho[c] / 4 < 1 ? 2 * (a.rho[c] / 4 - a.alvo[c]) * 0.25 : 0.0;
  std::vector<Particula> B(a.fim.size(), Particula{0, 0, 0, 0, 0, 0, 0, 0});
  for (size_t k = 0; k < a.fim.size(); k++) {
    const Particula& p = a.fim[k];
    Estencil e = estencil(2, p.x, p.y, nx, ny, h);
    int c = e.i0 + e.j0 * nx;
    double r00 = rb[c], r10 = rb[c + 1], r01 = rb[c + nx], r11 = rb[c + nx + 1];
    B[k].x = inv * (-(1 - e.ty) * r00 + (1 - e.ty) * r10 - e.ty * r01 + e.ty * r11);
    B[k].y = inv * (-(1 - e.tx) * r00 - e.tx * r10 + (1 - e.tx) * r01 + e.tx * r11);
  }
  gth[0] = gth[1] = 0;
  const double vmax = (MICROPASSO * MAX_MICROPASSOS * h) / dt;
  for (int s = a.passos - 1; s >= 0; s--) {
    const Passo& T = a.fita[s];
    const int n = (int)T.P.size();
    std::vector<Particula> Bin(n, Particula{0, 0, 0, 0, 0, 0, 0, 0});
    std::vector<double> ugb(nu, 0.0), vgb(nv, 0.0);
    // G2P reverse, particle by particle
    for (size_t o = 0; o < T.vivos.size(); o++) {
      const int k = T.vivos[o];
      const Particula& p = T.P[k];
      const Particula& bo = B[o];
      Amostra sm = amostrar(a, T.ug, T.vg, p.x, p.y);
      // replay the velocity through the micro-steps (collisions change it)
      const int mi = T.micro[k];
      const double dm = dt / mi;
      double vx = sm.vx, vy = sm.vy;
      if (T.clampV[k]) { double vel = std::hypot(vx, vy); vx *= vmax / vel; vy *= vmax / vel; }
      std::vector<double> vxm(mi + 1), vym(mi + 1);  // particle velocity before each micro-step
      for (int m = 0; m < mi; m++) {
        vxm[m] = vx, vym[m] = vy;
        if (T.col[(size_t)k * M + m] && T.corta[(size_t)k * M + m]) {
          // position after the move (before the push): the normal is taken there
          double xa = T.xm[((size_t)k * (M + 1) + m) * 2], ya = T.xm[((size_t)k * (M + 1) + m) * 2 + 1];
          double wx = vx, wy = vy;
          if (mi > 1) {
            Amostra w = amostrar(a, T.ug, T.vg, xa, ya);
            wx = w.vx, wy = w.vy;
            if (T.clampW[(size_t)k * M + m]) { double vw = std::hypot(wx, wy); wx *= vmax / vw; wy *= vmax / vw; }
          }
          double xp = xa + wx * dm, yp = ya + wy * dm, nn[2], J[2][2];
          a.sdf.normal(xp, yp, nn, J);
          double vn = vx * nn[0] + vy * nn[1];
          vx -= vn * nn[0];
          vy -= vn * nn[1];
        }
      }
      double xb = bo.x, yb = bo.y, vxb = bo.vx, vyb = bo.vy;
      for (int m = mi - 1; m >= 0; m--) {
        double xa = T.xm[((size_t)k * (M + 1) + m) * 2], ya = T.xm[((size_t)k * (M + 1) + m) * 2 + 1];
        double wx = vxm[m], wy = vym[m];
        Amostra w{};
        if (mi > 1) {
          w = amostrar(a, T.ug, T.vg, xa, ya);
          wx = w.vx, wy = w.vy;
          if (T.clampW[(size_t)k * M + m]) { double vw = std::hypot(wx, wy); wx *= vmax / vw; wy *= vmax / vw; }
        }
        double xp = xa + wx * dm, yp = ya + wy * dm;  // after the move
        if (T.col[(size_t)k * M + m]) {
          double dgx, dgy, nn[2], J[2][2];
          double d = a.sdf.dist(xp, yp, &dgx, &dgy);
          a.sdf.normal(xp, yp, nn, J);
          double e = (RAIO_PARTICULA - d) * h;
          // velocity cut: v_after = v - (v.n) n, v = vxm[m]
          double xpb = 0, ypb = 0;
          if (T.corta[(size_t)k * M + m]) {
            double v0x = vxm[m], v0y = vym[m], vn = v0x * nn[0] + v0y * nn[1];
            double bn = vxb * nn[0] + vyb * nn[1];
            // d v_after / d n = -(v n^T) - vn I ; through J to the position
            double gnx = -(v0x * bn + vn * vxb), gny = -(v0y * bn + vn * vyb);  // adjoint of n
            xpb += gnx * J[0][0] + gny * J[1][0];
            ypb += gnx * J[0][1] + gny * J[1][1];
            vxb -= bn * nn[0];
            vyb -= bn * nn[1];
          }
          // push: x_after = xp + n(xp) e(xp), e = (R - d) h
          double bxe = xb * nn[0] + yb * nn[1];  // adjoint of e
          double gnx = xb * e, gny = yb * e;     // adjoint of n
          xpb += xb + gnx * J[0][0] + gny * J[1][0] - bxe * h * dgx;
          ypb += yb + gnx * J[0][1] + gny * J[1][1] - bxe * h * dgy;
          xb = xpb, yb = ypb;
        }
        // move: xp = xa + w dm
        double wxb = xb * dm, wyb = yb * dm;
        if (mi > 1) {
          if (T.clampW[(size_t)k * M + m]) limitarT(w.vx, w.vy, vmax, &wxb, &wyb);
          double bv[6] = {wxb, wyb, 0, 0, 0, 0};
          amostrarT(a, w, bv, ugb, vgb, &xb, &yb);
        } else {
          vxb += wxb;
          vyb += wyb;
        }
      }
      // the sampled velocity (through the clamp) and affine terms at the start position
      if (T.clampV[k]) limitarT(sm.vx, sm.vy, vmax, &vxb, &vyb);
      double bv[6] = {vxb, vyb, bo.cux, bo.cuy, bo.cvx, bo.cvy};
      amostrarT(a, sm, bv, ugb, vgb, &xb, &yb);
      Bin[k].x = xb;
      Bin[k].y = yb;
    }
    // extrapolation reverse (layers in reverse)
    auto extrapT = [](std::vector<double>& xb, const std::vector<uint8_t>& val, const std::vector<uint8_t>& valDepois,
                      int w, int hh) {
      std::vector<double> out(xb);
      for (int j = 0; j < hh; j++)
        for (int i = 0; i < w; i++) {
          int k = i + j * w;
          if (val[k] || !valDepois[k]) continue;  // not filled in this layer
          int m = 0;
          if (i > 0 && val[k - 1]) m++;
          if (i < w - 1 && val[k + 1]) m++;
          if (j > 0 && val[k - w]) m++;
          if (j < hh - 1 && val[k + w]) m++;
          double g = xb[k] / m;
          out[k] -= xb[k];
          if (i > 0 && val[k - 1]) out[k - 1] += g;
          if (i < w - 1 && val[k + 1]) out[k + 1] += g;
          if (j > 0 && val[k - w]) out[k - w] += g;
          if (j < hh - 1 && val[k + w]) out[k + w] += g;
        }
      xb = out;
    };
    for (int l = CAMADAS - 1; l >= 0; l--) {
      extrapT(ugb, T.valU[l], T.valU[l + 1], nx + 1, ny);
      extrapT(vgb, T.valV[l], T.valV[l + 1], nx, ny + 1);
    }
    // gradient reverse: q adjoint; wall faces stop the adjoint
    const std::vector<uint8_t>& tipo = T.tipo;
    std::vector<double> qb(N, 0.0);
    for (int j = 0; j < ny; j++)
      for (int i = 0; i <= nx; i++) {
        int k = i + j * (nx + 1);
        uint8_t tl = i > 0 ? tipo[i - 1 + j * nx] : SOLIDO, tr = i < nx ? tipo[i + j * nx] : SOLIDO;
        if (tl == SOLIDO || tr == SOLIDO) { ugb[k] = 0; continue; }
        if (tl == AGUA || tr == AGUA) {
          if (tr == AGUA) qb[i + j * nx] -= ugb[k];
          if (tl == AGUA) qb[i - 1 + j * nx] += ugb[k];
        }
      }
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i < nx; i++) {
        int k = i + j * nx;
        uint8_t tb = j > 0 ? tipo[i + (j - 1) * nx] : SOLIDO, tt = j < ny ? tipo[i + j * nx] : SOLIDO;
        if (tb == SOLIDO || tt == SOLIDO) { vgb[k] = 0; continue; }
        if (tb == AGUA || tt == AGUA) {
          if (tt == AGUA) qb[i + j * nx] -= vgb[k];
          if (tb == AGUA) qb[i + (j - 1) * nx] += vgb[k];
        }
      }
    // pressure reverse: q = A^-1 b, b = -div  ->  div adjoint = -A^-1 qb
    std::vector<double> lam;
    resolver(a, tipo, qb, lam);
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        int c = i + j * nx;
        if (tipo[c] != AGUA) continue;
        double db = -lam[c];  // adjoint of div (b = -div -> bb = lam, divb = -lam)
        ugb[i + 1 + j * (nx + 1)] += db;
        ugb[i + j * (nx + 1)] -= db;
        vgb[i + (j + 1) * nx] += db;
        vgb[i + j * nx] -= db;
      }
    // gravity and walls reverse: wall faces were set to 0
    for (int j = 0; j < ny; j++)
      for (int i = 0; i <= nx; i++) {
        int k = i + j * (nx + 1);
        bool sl = i > 0 && tipo[i - 1 + j * nx] == SOLIDO, sr = i < nx && tipo[i + j * nx] == SOLIDO;
        if (i == 0 || i == nx || sl || sr) ugb[k] = 0;
      }
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i < nx; i++) {
        int k = i + j * nx;
        bool sb = j > 0 && tipo[i + (j - 1) * nx] == SOLIDO, st = j < ny && tipo[i + j * nx] == SOLIDO;
        if (j == 0 || j == ny || sb || st) vgb[k] = 0;
      }
    // normalisation reverse: u = U / UW
    std::vector<double> Ub(nu, 0.0), UWb(nu, 0.0), Vb(nv, 0.0), VWb(nv, 0.0);
    for (int k = 0; k < nu; k++)
      if (T.temU[k]) { Ub[k] = ugb[k] / T.UW[k]; UWb[k] = -ugb[k] * T.U[k] / (T.UW[k] * T.UW[k]); }
    for (int k = 0; k < nv; k++)
      if (T.temV[k]) { Vb[k] = vgb[k] / T.VW[k]; VWb[k] = -vgb[k] * T.V[k] / (T.VW[k] * T.VW[k]); }
    // P2G reverse
    for (int k = 0; k < n; k++) {
      const Particula& p = T.P[k];
      Particula& b = Bin[k];
      Estencil e = estencil(0, p.x, p.y, nx, ny, h);
      for (int bb = 0; bb < 2; bb++)
        for (int aa = 0; aa < 2; aa++) {
          double wx = aa ? e.tx : 1 - e.tx, wy = bb ? e.ty : 1 - e.ty, w = wx * wy;
          double dx = (e.i0 + aa) * h - p.x, dy = (e.j0 + bb + 0.5) * h - p.y;
          int idx = e.i0 + aa + (e.j0 + bb) * e.W;
          double val = p.vx + p.cux * dx + p.cuy * dy, g = Ub[idx];
          b.vx += w * g;
          b.cux += w * dx * g;
          b.cuy += w * dy * g;
          double t = val * g + UWb[idx];
          b.x += (aa ? 1 : -1) * inv * wy * t - w * p.cux * g;
          b.y += wx * (bb ? 1 : -1) * inv * t - w * p.cuy * g;
        }
      e = estencil(1, p.x, p.y, nx, ny, h);
      for (int bb = 0; bb < 2; bb++)
        for (int aa = 0; aa < 2; aa++) {
          double wx = aa ? e.tx : 1 - e.tx, wy = bb ? e.ty : 1 - e.ty, w = wx * wy;
          double dx = (e.i0 + aa + 0.5) * h - p.x, dy = (e.j0 + bb) * h - p.y;
          int idx = e.i0 + aa + (e.j0 + bb) * e.W;
          double val = p.vy + p.cvx * dx + p.cvy * dy, g = Vb[idx];
          b.vy += w * g;
          b.cvx += w * dx * g;
          b.cvy += w * dy * g;
          double t = val * g + VWb[idx];
          b.x += (aa ? 1 : -1) * inv * wy * t - w * p.cvx * g;
          b.y += wx * (bb ? 1 : -1) * inv * t - w * p.cvy * g;
        }
    }
    // the faucet's particles of this step: their velocity is theta
    int nAnt = n;
    for (int k = a.nf - 1; k >= 0; k--)
      if (T.aceitaTorneira[k]) {
        nAnt--;
        gth[0] += Bin[nAnt].vx;
        gth[1] += Bin[nAnt].vy;
      }
    Bin.resize(nAnt);
    B = Bin;
  }
  for (int k = 0; k < a.n0; k++) {
    gv0[2 * k] = B[k].vx;
    gv0[2 * k + 1] = B[k].vy;
  }
}

}  // namespace

struct tqo_adj {
  Adj a;
};

extern "C" {

int tqo_adj_create(const tq_adj_scene* d, tqo_adj** out) {
  if (!d || !out || d->nx < 3 || d->ny < 3 || !(d->h > 0) || !(d->dt > 0) || d->steps < 1 || d->n_particles < 0 ||
      !d->sdf || !d->target || (d->n_particles > 0 && !d->positions) || d->faucet_per_step < 0 ||
      (d->faucet_per_step > 0 && !d->faucet_positions))
    return TQ_E_ARG;
  auto* s = new tqo_adj();
  Adj& a = s->a;
  a.nx = d->nx, a.ny = d->ny, a.N = d->nx * d->ny, a.nu = (d->nx + 1) * d->ny, a.nv = d->nx * (d->ny + 1);
  a.h = d->h, a.dt = d->dt, a.g[0] = d->gravity[0], a.g[1] = d->gravity[1];
  a.passos = d->steps, a.n0 = d->n_particles, a.nf = d->faucet_per_step;
  a.mascara.assign(d->sdf, d->sdf + (size_t)4 * a.N);
  a.sdf = Sdf{a.mascara.data(), 2 * a.nx, 2 * a.ny, a.h};
  a.pos0.assign(d->positions, d->positions + 2 * (size_t)a.n0);
  a.C0.assign(4 * (size_t)a.n0, 0.0);
  if (d->affine)
    for (size_t k = 0; k < 4 * (size_t)a.n0; k++) a.C0[k] = d->affine[k];
  a.fpos.assign((size_t)a.passos * a.nf * 2, 0.0);
  for (size_t k = 0; k < a.fpos.size(); k++) a.fpos[k] = d->faucet_positions[k];
  a.alvo.assign(d->target, d->target + a.N);
  *out = s;
  return TQ_OK;
}

int tqo_adj_destroy(tqo_adj* s) {
  delete s;
  return TQ_OK;
}

// Forward in double.  record != 0 records the discrete structure; record = 0 applies the structure
// of the last recording run (the frozen map of the finite-difference checks).
int tqo_adj_forward(tqo_adj* s, const double* v0, const double* theta, int32_t record, double* loss) {
  if (!s || !theta || !loss || (s->a.n0 > 0 && !v0)) return TQ_E_ARG;
  if (!record && !s->a.gravado) return TQ_E_STATE;
  *loss = frente(s->a, v0, theta, record != 0);
  return TQ_OK;
}

// The adjoint of the last forward run (its tape): dL/dv0 (2 per initial particle), dL/dtheta.
int tqo_adj_backward(tqo_adj* s, double* dv0, double* dtheta) {
  if (!s || !dtheta || (s->a.n0 > 0 && !dv0)) return TQ_E_ARG;
  if (!s->a.gravado) return TQ_E_STATE;
  tras(s->a, dv0, dtheta);
  return TQ_OK;
}

int tqo_adj_count(tqo_adj* s, int32_t* n) {
  if (!s || !n) return TQ_E_ARG;
  *n = (int32_t)s->a.fim.size();
  return TQ_OK;
}

}  // extern "C"
