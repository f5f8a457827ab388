// tanque_oracle.cpp — TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
//
// CPU restatement of the reference's CPU engine for the simulation substep, used as the
// checker by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg only.
//
//   js/fisica-cpu.js   SimulacaoCPU (whole file)         -> struct Sim
//   js/pressao-cpu.js  MGPCG (whole file)                -> struct Niveis, cicloV, resolverPCG
//   js/ar.js           RastreadorDeAr (whole file)       -> struct Rastreador
//   js/cena.js         Cena SDF (lines 14-165)           -> struct Cena
//   js/constantes.js   constants, passoMaximo, dimensoesDaGrade
//   testes/apoio.js    semente (seeded LCG)
//
// Numeric semantics follow the JavaScript the restatement reads: every local is a double,
// every Float32Array store rounds to float (storage type S; S = double gives the FP64
// oracle), Uint8/Uint32 stores wrap, Array.prototype.sort is stable, Map iteration follows
// insertion order.  Build with -ffp-contract=off: JavaScript never fuses a multiply-add.
// Math.hypot and Math.exp map to glibc hypot/exp, which can differ from V8's in the last
// bit; they only feed normals, speed clamps and the foam decay.
//
// Parity pinning: there is no JavaScript engine on this machine or on the GPU box, so the
// restatement cannot be diffed against SimulacaoCPU itself.  It is pinned against the
// reference's own behavioural test suite (testes/fisica.test.js, testes/cena.test.js),
// ported to tests/test_oracle_suite_referencia.py, which it must pass with the reference's
// own bounds.
//
// One option goes beyond the reference: p2g_mode = TQ_P2G_FIXED replaces the float P2G
// sums by the integer (x65536) sums of the reference's GPU engine (js/gpu/fisica.js:77-131,
// the `faces` normalisation at :135-160) so that integer fields can be compared bit for bit
// with the CUDA library.  Its f32 arithmetic is spelled out operation by operation in
// p2g_fixed() below; the CUDA kernel performs the same operations.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <utility>
#include <vector>

#include "oracle.h"

namespace {

// ------------------------------------------------------------- js/constantes.js:8-104
constexpr double GRAVIDADE = 9.81;
constexpr double DENSIDADE_AGUA = 1000;
constexpr double TENSAO_SUPERFICIAL = 0.0728;
constexpr int MAX_BOLHAS = 4096;
constexpr double VOLTA_VOLUME_BOLHA = 0.05;
constexpr double PRESSAO_BOLHA_MAX = 20000;
constexpr double FATOR_CAPILAR = 0.4;
constexpr double PASSO_MAX = 0.008;
constexpr double PARTICULAS_POR_CELULA = 4;
constexpr int RES_MASCARA = 2;
constexpr double SDF_MAX = 10;
constexpr int MOLDURA = 2;
constexpr double RAIO_PARTICULA = 0.3;
constexpr double CFL = 2.0;
constexpr double MICROPASSO = 0.8;
constexpr double MAX_MICROPASSOS = 4;
constexpr double TAU_DENSIDADE = 0.1;
constexpr double EXCESSO_MIN = -0.5;
constexpr double EXCESSO_MAX = 1.0;
constexpr int ITERACOES_PCG = 3;
constexpr int CAMADAS_EXTRAPOLACAO = 2;
constexpr double ESPUMA_V0 = 1.1, ESPUMA_V1 = 2.8, ESPUMA_TAXA = 5, ESPUMA_VIDA = 1.2;
constexpr double DIFUSAO_CORANTE = 3;
constexpr double PARTICULAS_MAX_POR_CELULA = 4.6;
constexpr int CAMPOS = 12;  // js/fisica-cpu.js:26
constexpr uint8_t SOLIDO = 0, AGUA = 1, AR = 2;
constexpr uint32_t ATMOSFERA = 1;           // js/ar.js:18
constexpr int MIN_BOLHA_CELULAS = 4;        // js/ar.js:20
constexpr int BLOCO = 16, VARREDURAS = 4;   // js/pressao-cpu.js:17-18
constexpr int VARREDURAS_GROSSO = 64;       // js/pressao-cpu.js:20

inline int clampi(int v, int a, int b) { return v < a ? a : v > b ? b : v; }  // :697-699
// Math.floor of a double that is then used as an int (the reference clamps right after).
inline int floori(double v) {
  if (!(v == v)) return 0;
  if (v > 2e9) return 2000000000;
  if (v < -2e9) return -2000000000;
  return (int)std::floor(v);
}
inline double suave(double a, double b, double x) {  // js/fisica-cpu.js:692-695
  double t = std::min(1.0, std::max(0.0, (x - a) / (b - a)));
  return t * t * (3 - 2 * t);
}

// ------------------------------------------------------------- js/cena.js:14-165
struct Cena {
  int nx, ny;
  double h;
  int r, mw, mh;
  double largura, altura;
  std::vector<float> sdf;
  Cena(int nx_, int ny_, double h_)
      : nx(nx_), ny(ny_), h(h_), r(RES_MASCARA), mw(nx_ * RES_MASCARA), mh(ny_ * RES_MASCARA),
        largura(nx_ * h_), altura(ny_ * h_), sdf((size_t)nx_ * RES_MASCARA * ny_ * RES_MASCARA) {
    zerar();
  }
  // #moldura, js/cena.js:132-137
  double moldura(int x, int y) const {
    double m = MOLDURA * r - 0.5;
    double d = std::min(std::min(x - m, (double)(mw - 1) - m - x),
                        std::min(y - m, (double)(mh - 1) - m - y)) / r;
    return d > SDF_MAX ? SDF_MAX : d < -SDF_MAX ? -SDF_MAX : d;
  }
  // #zerar, js/cena.js:139-144
  void zerar() {
    for (int y = 0; y < mh; y++)
      for (int x = 0; x < mw; x++) sdf[(size_t)y * mw + x] = (float)moldura(x, y);
  }
  // tracar, js/cena.js:43-72
  void tracar(double x0, double y0, double x1, double y1, double raio, bool apagar) {
    double s = r / h;
    double ax = x0 * s - 0.5, ay = y0 * s - 0.5, bx = x1 * s - 0.5, by = y1 * s - 0.5;
    double rp = raio * s;
    double alc = rp + SDF_MAX * r + 1;
    double fxmin = std::floor(std::min(ax, bx) - alc), fxmax = std::ceil(std::max(ax, bx) + alc);
    double fymin = std::floor(std::min(ay, by) - alc), fymax = std::ceil(std::max(ay, by) + alc);
    double xmin = std::max(0.0, fxmin), xmax = std::min((double)(mw - 1), fxmax);
    double ymin = std::max(0.0, fymin), ymax = std::min((double)(mh - 1), fymax);
    if (xmin > xmax || ymin > ymax) return;
    double dx = bx - ax, dy = by - ay;
    double len2 = dx * dx + dy * dy;
    for (int y = (int)ymin; y <= (int)ymax; y++) {
      for (int x = (int)xmin; x <= (int)xmax; x++) {
        double t = len2 > 0 ? ((x - ax) * dx + (y - ay) * dy) / len2 : 0;
        t = t < 0 ? 0 : t > 1 ? 1 : t;
        double px = ax + t * dx - x, py = ay + t * dy - y;
        double d = (std::sqrt(px * px + py * py) - rp) / r;
        if (d > SDF_MAX) d = SDF_MAX;
        else if (d < -SDF_MAX) d = -SDF_MAX;
        size_t k = (size_t)y * mw + x;
        double v = apagar ? std::max((double)sdf[k], -d) : std::min((double)sdf[k], d);
        if (apagar) v = std::min(v, moldura(x, y));
        sdf[k] = (float)v;
      }
    }
  }
  // #bilinear, js/cena.js:156-165
  double bilinear(double fx, double fy) const {
    if (fx != fx || fy != fy) return NAN;
    double w = mw, hh = mh;
    if (fx < 0) fx = 0;
    else if (fx > w - 1) fx = w - 1;
    if (fy < 0) fy = 0;
    else if (fy > hh - 1) fy = hh - 1;
    int x0 = (int)std::min(std::floor(fx), w - 2), y0 = (int)std::min(std::floor(fy), hh - 2);
    double tx = fx - x0, ty = fy - y0;
    size_t k = (size_t)y0 * mw + x0;
    const float* d = sdf.data();
    return ((double)d[k] * (1 - tx) + (double)d[k + 1] * tx) * (1 - ty) +
           ((double)d[k + mw] * (1 - tx) + (double)d[k + mw + 1] * tx) * ty;
  }
  // distancia, js/cena.js:102-106
  double distancia(double x, double y) const {
    double fx = (x / h) * r - 0.5, fy = (y / h) * r - 0.5;
    return bilinear(fx, fy);
  }
  // normal, js/cena.js:109-116
  void normal(double x, double y, double* onx, double* ony) const {
    double fx = (x / h) * r - 0.5, fy = (y / h) * r - 0.5;
    double gx = bilinear(fx + 1, fy) - bilinear(fx - 1, fy);
    double gy = bilinear(fx, fy + 1) - bilinear(fx, fy - 1);
    double n = std::hypot(gx, gy);
    if (n > 1e-9) { *onx = gx / n; *ony = gy / n; }
    else { *onx = 0; *ony = 1; }
  }
  // celulaSolida, js/cena.js:119-127
  bool celulaSolida(int i, int j) const {
    if (i < 0 || j < 0 || i >= nx || j >= ny) return true;
    int a = i * r, b = j * r;
    double s = (double)sdf[(size_t)b * mw + a] + (double)sdf[(size_t)b * mw + a + 1] +
               (double)sdf[(size_t)(b + 1) * mw + a] + (double)sdf[(size_t)(b + 1) * mw + a + 1];
    return s < 0;
  }
};

// ------------------------------------------------------------- js/pressao-cpu.js
template <class S>
struct Nivel {
  int nx = 0, ny = 0;
  std::vector<uint8_t> tipo, viz, cnt;
  std::vector<S> b, x, tmp, r;
};

template <class S>
struct Niveis {
  std::vector<Nivel<S>> n;
  Nivel<S> op;  // niveis.operador (:302)
  bool cgPronto = false;
  std::vector<S> r, z, zVelho, p, ap;  // n0.cg (:311)
};

// montarNiveis, js/pressao-cpu.js:24-41
template <class S>
void montarNiveis(Niveis<S>& L, int nx, int ny) {
  L.n.clear();
  Nivel<S> a;
  a.nx = nx;
  a.ny = ny;
  L.n.push_back(a);
  while (std::min(L.n.back().nx, L.n.back().ny) > 12) {
    Nivel<S> g;
    g.nx = (L.n.back().nx + 1) / 2;
    g.ny = (L.n.back().ny + 1) / 2;
    L.n.push_back(g);
  }
  for (auto& n : L.n) {
    size_t k = (size_t)n.nx * n.ny;
    n.tipo.assign(k, 0);
    n.b.assign(k, 0);
    n.x.assign(k, 0);
    n.tmp.assign(k, 0);
    n.r.assign(k, 0);
    n.viz.assign(k, 0);
    n.cnt.assign(k, 0);
  }
}

// prepararVizinhos, js/pressao-cpu.js:44-60 (one level)
template <class S>
void prepararVizinhos(Nivel<S>& n) {
  int nx = n.nx, ny = n.ny;
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      int c = i + j * nx;
      int m = 0;
      if (i > 0 && n.tipo[c - 1] != SOLIDO) m |= 1;
      if (i < nx - 1 && n.tipo[c + 1] != SOLIDO) m |= 2;
      if (j > 0 && n.tipo[c - nx] != SOLIDO) m |= 4;
      if (j < ny - 1 && n.tipo[c + nx] != SOLIDO) m |= 8;
      n.viz[c] = (uint8_t)m;
      n.cnt[c] = (uint8_t)((m & 1) + ((m >> 1) & 1) + ((m >> 2) & 1) + ((m >> 3) & 1));
    }
}

// tiposGrossos, js/pressao-cpu.js:63-81
template <class S>
void tiposGrossos(Niveis<S>& L) {
  for (size_t l = 1; l < L.n.size(); l++) {
    Nivel<S>& f = L.n[l - 1];
    Nivel<S>& g = L.n[l];
    for (int J = 0; J < g.ny; J++)
      for (int I = 0; I < g.nx; I++) {
        bool temAr = false, temAgua = false;
        for (int b = 0; b < 2; b++)
          for (int a = 0; a < 2; a++) {
            int i = 2 * I + a, j = 2 * J + b;
            if (i >= f.nx || j >= f.ny) continue;
            uint8_t t = f.tipo[i + j * f.nx];
            if (t == AR) temAr = true;
            else if (t == AGUA) temAgua = true;
          }
        g.tipo[I + J * g.nx] = temAr ? AR : temAgua ? AGUA : SOLIDO;
      }
  }
}

// aplicar, js/pressao-cpu.js:84-93
template <class S>
inline double aplicar(const Nivel<S>& n, const S* v, int i, int j) {
  int c = i + j * n.nx;
  int m = n.viz[c];
  double s = 0;
  if (m & 1) s += (double)v[c - 1];
  if (m & 2) s += (double)v[c + 1];
  if (m & 4) s += (double)v[c - n.nx];
  if (m & 8) s += (double)v[c + n.nx];
  return n.cnt[c] * (double)v[c] - s;
}

// suavizar, js/pressao-cpu.js:99-150
template <class S>
void suavizar(Nivel<S>& n, int desl, const int ordem[2], double omega) {
  int nx = n.nx, ny = n.ny;
  std::vector<S>& src = n.x;
  std::vector<S>& dst = n.tmp;
  dst = src;
  const int L = BLOCO + 2;
  S local[(BLOCO + 2) * (BLOCO + 2)];
  for (int oy = -desl; oy < ny; oy += BLOCO) {
    for (int ox = -desl; ox < nx; ox += BLOCO) {
      for (int ly = 0; ly < L; ly++)
        for (int lx = 0; lx < L; lx++) {
          int i = ox + lx - 1, j = oy + ly - 1;
          local[lx + ly * L] = i >= 0 && j >= 0 && i < nx && j < ny ? src[i + j * nx] : (S)0;
        }
      for (int it = 0; it < VARREDURAS; it++) {
        for (int o = 0; o < 2; o++) {
          int cor = ordem[o];
          for (int ly = 1; ly <= BLOCO; ly++)
            for (int lx = 1; lx <= BLOCO; lx++) {
              int i = ox + lx - 1, j = oy + ly - 1;
              if (i < 0 || j < 0 || i >= nx || j >= ny) continue;
              if (((i + j + 1) & 1) != cor) continue;
              int c = i + j * nx;
              if (n.tipo[c] != AGUA) continue;
              int k = n.cnt[c];
              if (k == 0) continue;
              int m = n.viz[c], e = lx + ly * L;
              double s = 0;
              if (m & 1) s += (double)local[e - 1];
              if (m & 2) s += (double)local[e + 1];
              if (m & 4) s += (double)local[e - L];
              if (m & 8) s += (double)local[e + L];
              double q = local[lx + ly * L];
              local[lx + ly * L] = (S)(q + omega * ((s + (double)n.b[c]) / k - q));
            }
        }
      }
      for (int ly = 1; ly <= BLOCO; ly++)
        for (int lx = 1; lx <= BLOCO; lx++) {
          int i = ox + lx - 1, j = oy + ly - 1;
          if (i < 0 || j < 0 || i >= nx || j >= ny) continue;
          int c = i + j * nx;
          dst[c] = n.tipo[c] == AGUA ? local[lx + ly * L] : (S)0;
        }
    }
  }
  std::swap(n.x, n.tmp);  // n.x = dst; n.tmp = src
}

// grossoBase / pesoBase, js/pressao-cpu.js:155-156
inline int grossoBase(int i) { return (i & 1) == 0 ? (i >> 1) - 1 : (i - 1) >> 1; }
inline double pesoBase(int i) { return (i & 1) == 0 ? 0.25 : 0.75; }

// restringir, js/pressao-cpu.js:159-188
template <class S>
void restringir(Nivel<S>& f, Nivel<S>& g) {
  int fnx = f.nx, fny = f.ny, gnx = g.nx, gny = g.ny;
  for (int j = 0; j < fny; j++)
    for (int i = 0; i < fnx; i++) {
      int c = i + j * fnx;
      f.r[c] = f.tipo[c] == AGUA ? (S)((double)f.b[c] - aplicar(f, f.x.data(), i, j)) : (S)0;
    }
  std::fill(g.b.begin(), g.b.end(), (S)0);
  std::fill(g.x.begin(), g.x.end(), (S)0);
  for (int j = 0; j < fny; j++) {
    int J0 = grossoBase(j);
    double wy0 = pesoBase(j), wy1 = 1 - wy0;
    for (int i = 0; i < fnx; i++) {
      double r = f.r[i + j * fnx];
      if (r == 0) continue;
      int I0 = grossoBase(i);
      double wx0 = pesoBase(i), wx1 = 1 - wx0;
      for (int b = 0; b < 2; b++) {
        int J = J0 + b;
        if (J < 0 || J >= gny) continue;
        double wy = b ? wy1 : wy0;
        for (int a = 0; a < 2; a++) {
          int I = I0 + a;
          if (I < 0 || I >= gnx) continue;
          int C = I + J * gnx;
          if (g.tipo[C] == AGUA) g.b[C] = (S)((double)g.b[C] + r * (a ? wx1 : wx0) * wy);
        }
      }
    }
  }
}

// prolongar, js/pressao-cpu.js:191-214
template <class S>
void prolongar(Nivel<S>& g, Nivel<S>& f) {
  int fnx = f.nx, fny = f.ny, gnx = g.nx, gny = g.ny;
  for (int j = 0; j < fny; j++) {
    int J0 = grossoBase(j);
    double wy0 = pesoBase(j), wy1 = 1 - wy0;
    for (int i = 0; i < fnx; i++) {
      int c = i + j * fnx;
      if (f.tipo[c] != AGUA) continue;
      int I0 = grossoBase(i);
      double wx0 = pesoBase(i), wx1 = 1 - wx0;
      double e = 0;
      for (int b = 0; b < 2; b++) {
        int J = J0 + b;
        if (J < 0 || J >= gny) continue;
        double wy = b ? wy1 : wy0;
        for (int a = 0; a < 2; a++) {
          int I = I0 + a;
          if (I < 0 || I >= gnx) continue;
          int C = I + J * gnx;
          if (g.tipo[C] == AGUA) e += (double)g.x[C] * (a ? wx1 : wx0) * wy;
        }
      }
      f.x[c] = (S)((double)f.x[c] + e);
    }
  }
}

// resolverGrosso, js/pressao-cpu.js:217-238
template <class S>
void resolverGrosso(Nivel<S>& n) {
  int nx = n.nx, ny = n.ny;
  std::vector<S>& x = n.x;
  for (int k = 0; k < VARREDURAS_GROSSO; k++)
    for (int o = 0; o < 2; o++) {
      int cor = (k & 1) ? 1 - o : o;
      for (int c = 0; c < nx * ny; c++) {
        int i = c % nx, j = c / nx;
        if (n.tipo[c] != AGUA || ((i + j + 1) & 1) != cor) continue;
        int q = n.cnt[c];
        if (!q) continue;
        int m = n.viz[c];
        double s = 0;
        if (m & 1) s += (double)x[c - 1];
        if (m & 2) s += (double)x[c + 1];
        if (m & 4) s += (double)x[c - nx];
        if (m & 8) s += (double)x[c + nx];
        x[c] = (S)((s + (double)n.b[c]) / q);
      }
    }
}

// cicloV, js/pressao-cpu.js:241-255.  umaPassada (TQ_PRECOND_BLOCK_1; no counterpart in the
// reference): the levels above 0 take one smoother pass a leg, shift 8, red-black on the way
// down and black-red on the way up (the cycle stays symmetric).  On dumped pressure problems of
// the 840x536 scene it costs 5-10 % more PCG iterations and saves 6 of the fused solver's 23
// phases per iteration.
template <class S>
void cicloV(Niveis<S>& L, double omega = 1, bool umaPassada = false) {
  const int ida[2] = {0, 1}, volta[2] = {1, 0};
  int NL = (int)L.n.size();
  std::fill(L.n[0].x.begin(), L.n[0].x.end(), (S)0);
  for (int l = 0; l < NL - 1; l++) {
    const bool um = umaPassada && l >= 1;
    if (!um) suavizar(L.n[l], 0, ida, omega);
    suavizar(L.n[l], 8, ida, omega);
    restringir(L.n[l], L.n[l + 1]);
  }
  resolverGrosso(L.n[NL - 1]);
  for (int l = NL - 2; l >= 0; l--) {
    const bool um = umaPassada && l >= 1;
    prolongar(L.n[l + 1], L.n[l]);
    suavizar(L.n[l], 8, volta, omega);
    if (!um) suavizar(L.n[l], 0, volta, omega);
  }
}

// produto, js/pressao-cpu.js:257-261
template <class S>
double produto(const std::vector<S>& a, const std::vector<S>& b, const uint8_t* tipo) {
  double s = 0;
  for (size_t k = 0; k < a.size(); k++)
    if (tipo[k] == AGUA) s += (double)a[k] * (double)b[k];
  return s;
}

// The bubble vectors of resolverPCG are JS Maps keyed by label (values are doubles); labels
// are < MAX_BOLHAS, so a dense table plus the insertion-ordered key list restates them.
struct MapaB {
  std::vector<double> v = std::vector<double>(MAX_BOLHAS, 0.0);
  double get(uint32_t b) const { return v[b]; }
  void set(uint32_t b, double x) { v[b] = x; }
};

template <class S>
struct BolhasPCG {           // `bolhas` argument: { rotulo, rhs, y }
  const uint32_t* rotulo;
  const S* rhs;
  S* y;
};

// Coarse neighbour masks from the fine level's faces (TQ_PRECOND_BLOCK; no counterpart in the
// reference): the face between coarse cells C and its right neighbour is open when both are not
// wall and some fine face across the coarse face (between fine columns 2I+1 and 2I+2, rows 2J and
// 2J+1) joins two non-wall fine cells; likewise vertically.
template <class S>
void vizinhosPorFaces(const Nivel<S>& f, Nivel<S>& g) {
  auto livre = [&](int i, int j) { return i >= 0 && j >= 0 && i < f.nx && j < f.ny && f.tipo[i + j * f.nx] != SOLIDO; };
  for (int J = 0; J < g.ny; J++)
    for (int I = 0; I < g.nx; I++) {
      int C = I + J * g.nx, m = 0;
      if (g.tipo[C] != SOLIDO) {
        auto h = [&](int i0, int i1) {  // a fine face between columns i0, i1 in rows 2J, 2J+1
          return (livre(i0, 2 * J) && livre(i1, 2 * J)) || (livre(i0, 2 * J + 1) && livre(i1, 2 * J + 1));
        };
        auto v = [&](int j0, int j1) {
          return (livre(2 * I, j0) && livre(2 * I, j1)) || (livre(2 * I + 1, j0) && livre(2 * I + 1, j1));
        };
        if (I > 0 && g.tipo[C - 1] != SOLIDO && h(2 * I - 1, 2 * I)) m |= 1;
        if (I < g.nx - 1 && g.tipo[C + 1] != SOLIDO && h(2 * I + 1, 2 * I + 2)) m |= 2;
        if (J > 0 && g.tipo[C - g.nx] != SOLIDO && v(2 * J - 1, 2 * J)) m |= 4;
        if (J < g.ny - 1 && g.tipo[C + g.nx] != SOLIDO && v(2 * J + 1, 2 * J + 2)) m |= 8;
      }
      g.viz[C] = (uint8_t)m;
      g.cnt[C] = (uint8_t)((m & 1) + ((m >> 1) & 1) + ((m >> 2) & 1) + ((m >> 3) & 1));
    }
}

// Tolerance mode replaces the recursive residual by the true one each time the recursive one has
// fallen by this factor since the last replacement (or since r0): the FP32 rounding the
// recursive residual gathers (about 1e-7 of the residual it started from, per iteration) is
// then far below the tolerance by the end of the solve.
constexpr double FATOR_TROCA = 1e-3;

// What a solve reports beside q (tq_solve_info), and the closed regions it projected.
struct InfoPCG {
  int iters = 0, convergiu = 0, trocas = 0, regioes = 0;
  double r0 = 0, r = 0, rv = -1;
};

// Closed regions of a tolerance-mode solve (no counterpart in the reference; the library's
// regioes.cu).  The unknowns are the water cells and one pressure per active bubble (a label
// >= 2 with an interior air cell facing water, as montarBolhas finds them).  A 4-connected set
// of them, water joined to water and to the active bubbles it faces, that touches no Dirichlet
// cell (air outside an active bubble) is closed: A is singular on it, its null vector the
// constant, and b's component along it cannot be removed by any q.  Each closed region's
// right-hand side (-div on water, rhs on bubbles) loses its mean over the region's unknowns, in
// double, rounded back to S.  Each projected region's root (its smallest water cell) is then
// pinned: tipoSolve marks it air at pressure 0 for the solve (unless it carries a bubble
// label), which makes the region's block nonsingular; with the projected right-hand side the
// pinned row holds by itself.  Returns the number of closed regions (at most MAX_REGIOES are
// projected, as on the device).
constexpr int MAX_REGIOES = 4096;
template <class S>
int projetarFechadas(int nx, int ny, const uint8_t* tipo, const uint32_t* rot, S* div, S* rhs, uint8_t* tipoSolve) {
  const int N = nx * ny;
  std::vector<char> ativa(MAX_BOLHAS, 0);
  if (rot)
    for (int j = 1; j < ny - 1; j++)
      for (int i = 1; i < nx - 1; i++) {
        const int c = i + j * nx;
        const uint32_t b = rot[c];
        if (tipo[c] != AR || b < 2 || b >= (uint32_t)MAX_BOLHAS) continue;
        if (tipo[c - 1] == AGUA || tipo[c + 1] == AGUA || tipo[c - nx] == AGUA || tipo[c + nx] == AGUA) ativa[b] = 1;
      }
  std::vector<int> pai(N + MAX_BOLHAS);
  for (int c = 0; c < N + MAX_BOLHAS; c++) pai[c] = c;
  auto raiz = [&](int a) {
    while (pai[a] != a) {
      pai[a] = pai[pai[a]];
      a = pai[a];
    }
    return a;
  };
  auto unir = [&](int a, int b) {
    a = raiz(a);
    b = raiz(b);
    if (a != b) pai[a > b ? a : b] = a < b ? a : b;  // the smallest index is the root
  };
  std::vector<char> toca(N, 0);
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      const int c = i + j * nx;
      if (tipo[c] != AGUA) continue;
      const int nb[4] = {c - 1, c + 1, c - nx, c + nx};
      const bool dentro[4] = {i > 0, i < nx - 1, j > 0, j < ny - 1};
      for (int q = 0; q < 4; q++) {
        if (!dentro[q]) continue;
        const uint8_t t = tipo[nb[q]];
        if (t == AGUA) unir(c, nb[q]);
        else if (t == AR) {
          const uint32_t b = rot ? rot[nb[q]] : 0;
          if (rot && b >= 2 && b < (uint32_t)MAX_BOLHAS && ativa[b]) unir(c, N + (int)b);
          else toca[c] = 1;
        }
      }
    }
  std::vector<char> aberto(N, 0);
  for (int c = 0; c < N; c++)
    if (tipo[c] == AGUA && toca[c]) aberto[raiz(c)] = 1;
  std::vector<int> id(N, -1);
  int nReg = 0;
  for (int c = 0; c < N; c++)
    if (tipo[c] == AGUA && raiz(c) == c && !aberto[c]) {
      if (nReg < MAX_REGIOES) id[c] = nReg;
      nReg++;
    }
  std::vector<double> soma(MAX_REGIOES, 0.0);
  std::vector<long> cont(MAX_REGIOES, 0);
  for (int c = 0; c < N; c++) {
    if (tipo[c] != AGUA) continue;
    const int r = id[raiz(c)];
    if (r < 0) continue;
    soma[r] += -(double)div[c];
    cont[r]++;
  }
  if (rot)
    for (int b = 2; b < MAX_BOLHAS; b++) {
      if (!ativa[b]) continue;
      const int r = id[raiz(N + b)];
      if (r < 0) continue;
      soma[r] += (double)rhs[b];
      cont[r]++;
    }
  for (int c = 0; c < N; c++) {
    tipoSolve[c] = tipo[c];
    if (tipo[c] != AGUA) continue;
    const int r = id[raiz(c)];
    if (r < 0) continue;
    div[c] = (S)((double)div[c] + soma[r] / (double)cont[r]);
    if (raiz(c) == c && (!rot || rot[c] < 2)) tipoSolve[c] = AR;
  }
  if (rot)
    for (int b = 2; b < MAX_BOLHAS; b++) {
      if (!ativa[b]) continue;
      const int r = id[raiz(N + b)];
      if (r >= 0) rhs[b] = (S)((double)rhs[b] - soma[r] / (double)cont[r]);
    }
  return nReg < MAX_REGIOES ? nReg : MAX_REGIOES;
}

// resolverPCG, js/pressao-cpu.js:296-402.  tol = 0 is the reference's fixed count.  tol > 0 (no
// counterpart in the reference) keeps q in double during the solve and stops when the TRUE
// residual ||b - A q|| (double, from the double iterate and the bubbles' y) is <= tol*||r0||,
// or at the cap.  The true residual is recomputed when the recursive one meets the tolerance, and
// each time the recursive one has fallen by FATOR_TROCA since the last replacement; unless the
// solve ends there, it replaces the recursive one and the iteration goes on with the same
// search direction (a residual replacement without restart).
// precond = TQ_PRECOND_BLOCK (and BLOCK_1, with one smoother pass a leg above level 0, see
// cicloV) replaces precondicionar (:352-361) by the block-diagonal form:
// bubble rows z_b = r_b / faces_b, the V-cycle on the water alone (enclosed air stays air) with
// coarse neighbour masks from the fine faces (vizinhosPorFaces).
template <class S>
std::vector<double> resolverPCG(Niveis<S>& L, const uint8_t* tipo, const S* div, S* q,
                                int iteracoes, const BolhasPCG<S>* bolhas, double tol,
                                int precond = TQ_PRECOND_REFERENCE, InfoPCG* info = nullptr) {
  const bool bloco = precond == TQ_PRECOND_BLOCK || precond == TQ_PRECOND_BLOCK_1;
  const bool umaPassada = precond == TQ_PRECOND_BLOCK_1;
  Nivel<S>& n0 = L.n[0];
  int nx = n0.nx, ny = n0.ny;
  int k = nx * ny;
  // tolerance mode: the solve reads copies of div and the bubble rhs in which every closed
  // region's right-hand side has lost its mean (projetarFechadas)
  std::vector<S> divP, rhsP;
  std::vector<uint8_t> tipoP;
  BolhasPCG<S> bP{};
  int regioes = 0;
  if (tol > 0) {
    divP.assign(div, div + k);
    tipoP.assign(k, 0);
    if (bolhas) {
      rhsP.assign(bolhas->rhs, bolhas->rhs + MAX_BOLHAS);
      bP = *bolhas;
      bP.rhs = rhsP.data();
      bolhas = &bP;
    }
    regioes = projetarFechadas<S>(nx, ny, tipo, bolhas ? bolhas->rotulo : nullptr, divP.data(),
                                  bolhas ? rhsP.data() : nullptr, tipoP.data());
    div = divP.data();
    tipo = tipoP.data();
  }
  Nivel<S>& op = L.op;
  if (op.nx != nx || op.ny != ny) {
    op.nx = nx;
    op.ny = ny;
    op.tipo.assign(k, 0);
    op.viz.assign(k, 0);
    op.cnt.assign(k, 0);
  }
  std::copy(tipo, tipo + k, op.tipo.begin());
  prepararVizinhos(op);
  std::copy(tipo, tipo + k, n0.tipo.begin());
  if (bolhas && !bloco)
    for (int c = 0; c < k; c++)
      if (tipo[c] == AR && bolhas->rotulo[c] >= 2) n0.tipo[c] = AGUA;
  tiposGrossos(L);
  prepararVizinhos(L.n[0]);
  for (size_t l = 1; l < L.n.size(); l++) {
    if (bloco) vizinhosPorFaces(L.n[l - 1], L.n[l]);
    else prepararVizinhos(L.n[l]);
  }
  if (!L.cgPronto) {
    L.r.assign(k, 0);
    L.z.assign(k, 0);
    L.zVelho.assign(k, 0);
    L.p.assign(k, 0);
    L.ap.assign(k, 0);
    L.cgPronto = true;
  }
  std::vector<S>&r = L.r, &z = L.z, &zVelho = L.zVelho, &p = L.p, &ap = L.ap;
  // montarBolhas, js/pressao-cpu.js:271-288
  std::vector<uint32_t> pares;  // [label, water cell] per face
  std::vector<int> faces(MAX_BOLHAS, 0);
  std::vector<char> temFace(MAX_BOLHAS, 0);
  std::vector<uint32_t> ativos;  // faces.keys() in insertion order
  const uint32_t* rot = bolhas ? bolhas->rotulo : nullptr;
  if (bolhas) {
    for (int j = 1; j < ny - 1; j++)
      for (int i = 1; i < nx - 1; i++) {
        int c = i + j * nx;
        uint32_t b = rot[c];
        if (b < 2 || tipo[c] == AGUA || tipo[c] == SOLIDO) continue;
        if (tipo[c - 1] == AGUA) { pares.push_back(b); pares.push_back(c - 1); }
        if (tipo[c + 1] == AGUA) { pares.push_back(b); pares.push_back(c + 1); }
        if (tipo[c - nx] == AGUA) { pares.push_back(b); pares.push_back(c - nx); }
        if (tipo[c + nx] == AGUA) { pares.push_back(b); pares.push_back(c + nx); }
      }
    for (size_t m = 0; m < pares.size(); m += 2) {
      uint32_t b = pares[m];
      if (!temFace[b]) { temFace[b] = 1; ativos.push_back(b); }
      faces[b]++;
    }
  }
  MapaB yb, rb, zb, zvb, pb, apb, aq;
  for (uint32_t b : ativos) yb.set(b, (double)bolhas->y[b]);
  auto difundir = [&](std::vector<S>& grade, const MapaB& valores) {
    if (!rot) return;
    for (int c = 0; c < k; c++) {
      uint32_t b = rot[c];
      if (b >= 2 && tipo[c] == AR) grade[c] = (S)(b < (uint32_t)MAX_BOLHAS && temFace[b] ? valores.get(b) : 0.0);
    }
  };
  auto aplicarBolhas = [&](const std::vector<S>& grade, const MapaB& valores, MapaB& saida) {
    for (uint32_t b : ativos) saida.set(b, faces[b] * valores.get(b));
    for (size_t m = 0; m < pares.size(); m += 2)
      saida.set(pares[m], saida.get(pares[m]) - (double)grade[pares[m + 1]]);
  };
  auto produtoB = [&](const MapaB& a, const MapaB& b) {
    double s = 0;
    for (uint32_t x : ativos) s += a.get(x) * b.get(x);
    return s;
  };

  for (int c = 0; c < k; c++)
    if (tipo[c] != AGUA) q[c] = 0;
  std::vector<S> qv(q, q + k);
  difundir(qv, yb);
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      int c = i + j * nx;
      r[c] = tipo[c] == AGUA ? (S)(-(double)div[c] - aplicar(op, qv.data(), i, j)) : (S)0;
    }
  aplicarBolhas(qv, yb, aq);
  for (uint32_t b : ativos) rb.set(b, (double)bolhas->rhs[b] - aq.get(b));
  auto norma = [&]() { return std::sqrt(produto(r, r, tipo) + produtoB(rb, rb)); };
  std::vector<double> normas{norma()};
  // tolerance mode: the double iterate (water cells) and the true residual from it
  const bool verdade = tol > 0;
  std::vector<double> qd;
  if (verdade) qd.assign(qv.begin(), qv.end());
  auto residuoVerdadeiro = [&](bool substituir) {
    std::vector<double> g(qd);
    if (rot)
      for (int c = 0; c < k; c++) {
        uint32_t b = rot[c];
        if (b >= 2 && tipo[c] == AR) g[c] = b < (uint32_t)MAX_BOLHAS && temFace[b] ? yb.get(b) : 0.0;
      }
    double s = 0;
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        int c = i + j * nx;
        if (tipo[c] != AGUA) continue;
        int m = op.viz[c];
        double t = 0;
        if (m & 1) t += g[c - 1];
        if (m & 2) t += g[c + 1];
        if (m & 4) t += g[c - nx];
        if (m & 8) t += g[c + nx];
        double rt = -(double)div[c] - (op.cnt[c] * g[c] - t);
        s += rt * rt;
        if (substituir) r[c] = (S)rt;
      }
    MapaB somaB;
    for (size_t m = 0; m < pares.size(); m += 2) somaB.set(pares[m], somaB.get(pares[m]) + qd[pares[m + 1]]);
    for (uint32_t b : ativos) {
      double rt = (double)bolhas->rhs[b] - (faces[b] * yb.get(b) - somaB.get(b));
      s += rt * rt;
      if (substituir) rb.set(b, rt);
    }
    return std::sqrt(s);
  };
  // celulasDe (js/pressao-cpu.js:345-351)
  std::vector<int> celulasDe(MAX_BOLHAS, 0);
  if (rot)
    for (int c = 0; c < k; c++) {
      uint32_t b = rot[c];
      if (b >= 2 && b < (uint32_t)MAX_BOLHAS && tipo[c] == AR && temFace[b]) celulasDe[b]++;
    }
  auto tem = [&](uint32_t b) { return b < (uint32_t)MAX_BOLHAS && celulasDe[b] > 0; };
  auto precondicionar = [&](std::vector<S>& destino, MapaB& destinoB) {
    n0.b = r;
    if (bloco) {  // bubble air is air to the V-cycle (r = 0 there); bubble rows: Jacobi
      cicloV(L, 1.0, umaPassada);
      destino = n0.x;
      for (uint32_t b : ativos) destinoB.set(b, rb.get(b) / faces[b]);
      return;
    }
    if (rot)
      for (int c = 0; c < k; c++) {
        uint32_t b = rot[c];
        if (tem(b) && tipo[c] == AR) n0.b[c] = (S)(rb.get(b) / celulasDe[b]);
      }
    cicloV(L);
    destino = n0.x;
    for (uint32_t b : ativos) destinoB.set(b, 0);
    if (rot)
      for (int c = 0; c < k; c++) {
        uint32_t b = rot[c];
        if (tem(b) && tipo[c] == AR) {
          destinoB.set(b, destinoB.get(b) + (double)n0.x[c] / celulasDe[b]);
          destino[c] = 0;
        }
      }
  };
  InfoPCG inf;
  inf.r0 = normas[0];
  double proxTroca = normas[0] * FATOR_TROCA;  // the next residual replacement's threshold
  precondicionar(z, zb);
  p = z;
  for (uint32_t b : ativos) pb.set(b, zb.get(b));
  double rz = produto(r, z, tipo) + produtoB(rb, zb);
  for (int it = 0; it < iteracoes; it++) {
    difundir(p, pb);
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        int c = i + j * nx;
        ap[c] = tipo[c] == AGUA ? (S)aplicar(op, p.data(), i, j) : (S)0;
      }
    aplicarBolhas(p, pb, apb);
    double pap = produto(p, ap, tipo) + produtoB(pb, apb);
    double alfa = std::fabs(pap) < 1e-30 ? 0 : rz / pap;
    for (int c = 0; c < k; c++) {
      if (tipo[c] != AGUA) continue;
      if (verdade) qd[c] += alfa * (double)p[c];
      else qv[c] = (S)((double)qv[c] + alfa * (double)p[c]);
      r[c] = (S)((double)r[c] - alfa * (double)ap[c]);
    }
    for (uint32_t b : ativos) {
      yb.set(b, yb.get(b) + alfa * pb.get(b));
      rb.set(b, rb.get(b) - alfa * apb.get(b));
    }
    normas.push_back(norma());
    inf.iters = it + 1;
    if (verdade && (normas.back() <= tol * normas[0] || normas.back() <= proxTroca || it == iteracoes - 1)) {
      const bool ultima = it == iteracoes - 1;
      // the true residual: below the tolerance or at the cap the solve ends; otherwise it
      // replaces r and rb and the search direction carries on (no restart)
      const double rv = residuoVerdadeiro(false);
      inf.rv = rv;
      if (rv <= tol * normas[0] || ultima) {
        inf.convergiu = rv <= tol * normas[0] ? 1 : 0;
        break;
      }
      residuoVerdadeiro(true);
      inf.trocas++;
      proxTroca = rv * FATOR_TROCA;
    }
    if (it == iteracoes - 1) break;
    zVelho = z;
    for (uint32_t b : ativos) zvb.set(b, zb.get(b));
    precondicionar(z, zb);
    double rzNovo = produto(r, z, tipo) + produtoB(rb, zb);
    double cruzado = produto(r, zVelho, tipo) + produtoB(rb, zvb);
    double beta = std::fabs(rz) < 1e-30 ? 0 : std::max(0.0, (rzNovo - cruzado) / rz);
    rz = rzNovo;
    for (int c = 0; c < k; c++) p[c] = tipo[c] == AGUA ? (S)((double)z[c] + beta * (double)p[c]) : (S)0;
    for (uint32_t b : ativos) pb.set(b, zb.get(b) + beta * pb.get(b));
  }
  if (verdade)
    for (int c = 0; c < k; c++) qv[c] = (S)qd[c];
  for (int c = 0; c < k; c++) q[c] = tipo[c] != AGUA ? (S)0 : qv[c];
  if (bolhas)
    for (uint32_t b : ativos) bolhas->y[b] = (S)yb.get(b);
  inf.r = normas.back();
  inf.regioes = regioes;
  if (info) *info = inf;
  return normas;
}

}  // namespace

// A q = b on the water cells of `tipo` with resolverPCG's operator, in double storage, to a
// relative residual of 1e-13 (the reference preconditioner, at most 2000 iterations): the exact
// pressure solve of the FP64 adjoint checker (adjunto_oracle.cpp).
void resolverExatoFP64(int nx, int ny, const uint8_t* tipo, const double* b, double* q) {
  Niveis<double> L;
  montarNiveis(L, nx, ny);
  const size_t N = (size_t)nx * ny;
  std::vector<double> div(N);
  for (size_t c = 0; c < N; c++) div[c] = -b[c];  // resolverPCG solves A q = -div
  std::fill(q, q + N, 0.0);
  resolverPCG<double>(L, tipo, div.data(), q, 2000, nullptr, 1e-13);
}

namespace {

// ------------------------------------------------------------- js/ar.js:22-159
template <class S>
struct Rastreador {
  int nx, ny;
  std::vector<uint32_t> rotulo;
  std::vector<int32_t> pai, componente, numero;
  std::vector<S> volumeAlvo;
  std::vector<uint8_t> vivo;
  bool primeira = true;
  Rastreador(int nx_, int ny_)
      : nx(nx_), ny(ny_), rotulo((size_t)nx_ * ny_, 0), pai((size_t)nx_ * ny_),
        componente((size_t)nx_ * ny_), numero((size_t)nx_ * ny_, -1), volumeAlvo(MAX_BOLHAS, 0),
        vivo(MAX_BOLHAS, 0) {}
  void reiniciar() {  // :37-42
    std::fill(rotulo.begin(), rotulo.end(), 0);
    std::fill(volumeAlvo.begin(), volumeAlvo.end(), (S)0);
    std::fill(vivo.begin(), vivo.end(), 0);
    primeira = true;
  }
  int raiz(int a) {  // :44-48
    while (pai[a] != a) { pai[a] = pai[pai[a]]; a = pai[a]; }
    return a;
  }
  void unir(int a, int b) {  // :155-158
    int ra = raiz(a), rb = raiz(b);
    if (ra != rb) pai[std::max(ra, rb)] = std::min(ra, rb);
  }
  struct Info {
    int celulas = 0;
    bool topo = false;
    int atm = 0;
    std::vector<std::pair<uint32_t, int>> gas;  // Map(old label -> cells), insertion order
  };
  // atualizar, js/ar.js:56-153.  Returns the births (label, initial pressure).
  template <class F>
  std::vector<std::pair<uint32_t, double>> atualizar(const uint8_t* tipo, F pressaoAnterior) {
    int n = nx * ny;
    for (int c = 0; c < n; c++) pai[c] = tipo[c] == AR ? c : -1;
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        int c = i + j * nx;
        if (pai[c] < 0) continue;
        if (i > 0 && pai[c - 1] >= 0) unir(c, c - 1);
        if (j > 0 && pai[c - nx] >= 0) unir(c, c - nx);
      }
    int topo = ny - MOLDURA - 1;
    std::vector<int> raizes;
    std::vector<Info> info;
    for (int c = 0; c < n; c++) {
      if (pai[c] < 0) { componente[c] = -1; continue; }
      int r = raiz(c);
      int k = numero[r];
      if (k < 0) {
        k = (int)info.size();
        numero[r] = k;
        raizes.push_back(r);
        info.emplace_back();
      }
      componente[c] = k;
      Info& d = info[k];
      d.celulas++;
      if (c / nx >= topo) d.topo = true;
      uint32_t antigo = rotulo[c];
      if (antigo == ATMOSFERA) d.atm++;
      else if (antigo >= 2) {
        bool achou = false;
        for (auto& g : d.gas)
          if (g.first == antigo) { g.second++; achou = true; break; }
        if (!achou) d.gas.emplace_back(antigo, 1);
      }
    }
    for (int r : raizes) numero[r] = -1;
    auto fica = [](const Info& d) { return d.topo || d.celulas >= MIN_BOLHA_CELULAS; };
    // sobreposicaoTotal, :102-106.  Old labels may exceed MAX_BOLHAS only if a caller wrote
    // them; the Map then still works, so keep a sparse fallback.
    std::vector<double> sob(MAX_BOLHAS, 0.0);
    std::vector<std::pair<uint32_t, double>> sobExtra;
    auto sobAdd = [&](uint32_t r, double q) {
      if (r < (uint32_t)MAX_BOLHAS) { sob[r] += q; return; }
      for (auto& e : sobExtra)
        if (e.first == r) { e.second += q; return; }
      sobExtra.emplace_back(r, q);
    };
    auto sobGet = [&](uint32_t r) {
      if (r < (uint32_t)MAX_BOLHAS) return sob[r];
      for (auto& e : sobExtra)
        if (e.first == r) return e.second;
      return 0.0;
    };
    for (auto& d : info) {
      if (d.gas.empty() || !fica(d)) continue;
      for (auto& g : d.gas) sobAdd(g.first, g.second);
    }
    int K = (int)info.size();
    std::vector<float> novoAlvo(K, 0.0f);  // Float32Array (:108)
    std::vector<int32_t> dono(K, -1);
    for (int k = 0; k < K; k++) {
      Info& d = info[k];
      if (!fica(d) || d.topo) continue;
      double v = 0;
      int melhor = 0;
      if (primeira) v = d.celulas;
      else {
        v = d.atm;
        for (auto& g : d.gas) {
          double alvoOld = g.first < (uint32_t)MAX_BOLHAS ? (double)volumeAlvo[g.first] : NAN;
          v += alvoOld * (g.second / sobGet(g.first));
          if (g.second > melhor) { melhor = g.second; dono[k] = (int32_t)g.first; }
        }
      }
      novoAlvo[k] = (float)v;
    }
    std::vector<uint32_t> rotuloDaComp(K, 0);
    std::vector<uint8_t> vivoNovo(MAX_BOLHAS, 0);
    std::vector<int> ordem;
    for (int k = 0; k < K; k++)
      if (!info[k].topo && novoAlvo[k] >= MIN_BOLHA_CELULAS) ordem.push_back(k);
    std::stable_sort(ordem.begin(), ordem.end(),
                     [&](int a, int b) { return novoAlvo[b] - novoAlvo[a] < 0; });
    for (int k : ordem) {
      int32_t r = dono[k];
      if (r >= 2 && r < MAX_BOLHAS && !vivoNovo[r]) { rotuloDaComp[k] = (uint32_t)r; vivoNovo[r] = 1; }
    }
    std::vector<std::pair<uint32_t, double>> nascidas;
    int livre = 2;
    for (int k : ordem) {
      if (rotuloDaComp[k]) continue;
      while (livre < MAX_BOLHAS && (vivoNovo[livre] || vivo[livre])) livre++;
      if (livre >= MAX_BOLHAS) break;
      rotuloDaComp[k] = (uint32_t)livre;
      vivoNovo[livre] = 1;
      nascidas.emplace_back((uint32_t)livre, dono[k] >= 2 ? pressaoAnterior((uint32_t)dono[k]) : 0.0);
    }
    for (int k = 0; k < K; k++)
      if (info[k].topo) rotuloDaComp[k] = ATMOSFERA;
    std::fill(volumeAlvo.begin(), volumeAlvo.end(), (S)0);
    for (int k = 0; k < K; k++)
      if (rotuloDaComp[k] >= 2) volumeAlvo[rotuloDaComp[k]] = (S)novoAlvo[k];
    for (int c = 0; c < n; c++) rotulo[c] = componente[c] >= 0 ? rotuloDaComp[componente[c]] : 0;
    vivo = vivoNovo;
    primeira = false;
    return nascidas;
  }
};

// ------------------------------------------------------------- js/fisica-cpu.js:28-690
struct SimBase {
  virtual ~SimBase() {}
};

template <class S>
struct Sim : SimBase {
  Cena cena;
  int nx, ny;
  double h;
  double gravidade[2];
  int iteracoes;
  double tauDensidade, tensao, tol;
  bool arAtivo;
  int p2gMode;
  int nu, nv;
  std::vector<S> u, v, uPeso, vPeso, uTmp, vTmp, densidade, corCelula, div, q, fase, faseTmp,
      normalX, normalY, curvatura, qAr, pressaoBolha, volumeBolha, rhsBolha, yBolha;
  std::vector<uint8_t> uValida, vValida, tipo, solidoCelula, preenchido;
  std::vector<uint32_t> contagemCelula;
  std::vector<int32_t> novas;
  std::vector<int32_t> accU, accV, accCel, accCor;  // fixed-point sums (TQ_P2G_FIXED)
  Rastreador<S> rastreador;
  Niveis<S> niveis;
  bool tiposProntos = false;
  int n = 0;
  int capacidade;
  std::vector<float> p;  // Float32Array of CAMPOS per particle
  double vMax = 0;
  std::vector<double> normas;
  int precond;
  InfoPCG info;  // the last solve
  // accumulated since the last reset (TQ_SCALAR_SOLVES = 0)
  long long solves = 0, capados = 0, itersAcum = 0, trocasAcum = 0;
  double maxRel = 0;

  Sim(const tq_options& o)
      : cena(o.nx, o.ny, o.h), nx(o.nx), ny(o.ny), h(o.h), iteracoes(o.iterations),
        tauDensidade(o.tau_density), tensao(o.surface_tension), tol(o.tolerance),
        arAtivo(o.air != 0), p2gMode(o.p2g_mode), rastreador(o.nx, o.ny), precond(o.preconditioner) {
    gravidade[0] = o.gravity[0];
    gravidade[1] = o.gravity[1];
    nu = (nx + 1) * ny;
    nv = nx * (ny + 1);
    int N = nx * ny;
    u.assign(nu, 0); v.assign(nv, 0); uPeso.assign(nu, 0); vPeso.assign(nv, 0);
    uValida.assign(nu, 0); vValida.assign(nv, 0); uTmp.assign(nu, 0); vTmp.assign(nv, 0);
    densidade.assign(N, 0); contagemCelula.assign(N, 0); corCelula.assign(3 * N, 0);
    tipo.assign(N, 0); solidoCelula.assign(N, 0); div.assign(N, 0); q.assign(N, 0);
    fase.assign(N, 0); faseTmp.assign(N, 0); normalX.assign(N, 0); normalY.assign(N, 0);
    curvatura.assign(N, 0); qAr.assign(N, 0);
    pressaoBolha.assign(MAX_BOLHAS, 0); volumeBolha.assign(MAX_BOLHAS, 0);
    rhsBolha.assign(MAX_BOLHAS, 0); yBolha.assign(MAX_BOLHAS, 0);
    accU.assign(2 * nu, 0); accV.assign(2 * nv, 0); accCel.assign(2 * N, 0); accCor.assign(3 * N, 0);
    montarNiveis(niveis, nx, ny);
    capacidade = o.capacity > 0 ? o.capacity : (int)std::ceil(N * PARTICULAS_MAX_POR_CELULA);
    atualizarParedes();
  }

  // atualizarParedes, :80-85
  void atualizarParedes() {
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) solidoCelula[i + j * nx] = cena.celulaSolida(i, j) ? 1 : 0;
  }

  // adicionar, :92-111
  int adicionar(const float* lista, int total, bool checarCheia) {
    int aceitas = 0;
    for (int k = 0; k < total; k++) {
      const float* o = lista + (size_t)k * CAMPOS;
      double x = o[0], y = o[1];
      if (!(cena.distancia(x, y) > RAIO_PARTICULA + 0.05)) continue;
      if (checarCheia) {
        double fi = std::floor(x / h), fj = std::floor(y / h);
        if (fi < 0 || fj < 0 || fi >= nx || fj >= ny) continue;
        int i = (int)fi, j = (int)fj;
        if (contagemCelula[i + j * nx] >= PARTICULAS_POR_CELULA - 1) continue;
      }
      p.insert(p.end(), o, o + CAMPOS);
      n++;
      aceitas++;
    }
    return aceitas;
  }

  // remover, :114-126
  template <class F>
  int remover(F fn) {
    int w = 0;
    for (int k = 0; k < n; k++) {
      float* o = p.data() + (size_t)k * CAMPOS;
      if (fn((double)o[0], (double)o[1], k)) continue;
      if (w != k) std::memmove(p.data() + (size_t)w * CAMPOS, o, CAMPOS * sizeof(float));
      w++;
    }
    int removidas = n - w;
    n = w;
    p.resize((size_t)n * CAMPOS);
    return removidas;
  }

  // aplicarFerramenta, :129-152
  void aplicarFerramenta(const tq_tool& f) {
    if (f.kind == 0) return;
    double r2 = f.radius * f.radius;
    if (f.kind == 1) {
      remover([&](double x, double y, int) { return (x - f.x) * (x - f.x) + (y - f.y) * (y - f.y) < r2; });
      return;
    }
    for (int k = 0; k < n; k++) {
      float* o = p.data() + (size_t)k * CAMPOS;
      double d2 = ((double)o[0] - f.x) * ((double)o[0] - f.x) + ((double)o[1] - f.y) * ((double)o[1] - f.y);
      if (d2 >= r2) continue;
      double peso = 1 - std::sqrt(d2 / r2);
      if (f.kind == 2) {
        double a = std::min(1.0, peso * 0.9);
        o[2] = (float)((double)o[2] + (f.vx - (double)o[2]) * a);
        o[3] = (float)((double)o[3] + (f.vy - (double)o[3]) * a);
      } else if (f.kind == 3) {
        o[9] = (float)f.absorb[0];
        o[10] = (float)f.absorb[1];
        o[11] = (float)f.absorb[2];
      }
    }
  }

  // avancar, :155-159
  void avancar(double dt, int subpassos) {
    if (arAtivo) atualizarAr();
    double d = dt / subpassos;
    for (int s = 0; s < subpassos; s++) subpasso(d);
  }
  // atualizarAr, :162-167
  void atualizarAr() {
    if (!tiposProntos) { paraGrade(); tipos(); }
    auto nascidas = rastreador.atualizar(tipo.data(), [&](uint32_t r) {
      return r < (uint32_t)MAX_BOLHAS ? (double)pressaoBolha[r] : NAN;
    });
    for (auto& nb : nascidas) pressaoBolha[nb.first] = (S)nb.second;
  }
  // reiniciarAr, :170-174
  void reiniciarAr() {
    tiposProntos = false;
    rastreador.reiniciar();
    std::fill(pressaoBolha.begin(), pressaoBolha.end(), (S)0);
  }
  // subpasso, :176-189
  void subpasso(double dt) {
    paraGrade();
    gravidadeEFronteira(dt);
    tipos();
    if (arAtivo) propagarRotulos();
    superficie();
    pressaoDoAr(dt);
    classificar(dt);
    if (arAtivo) ladoDireitoDasBolhas(dt);
    pressao(dt);
    gradiente();
    extrapolar();
    paraParticulas(dt);
  }

  // #paraGrade, :198-267 (TQ_P2G_FLOAT) and the fixed-point variant.
  void paraGrade() {
    if (p2gMode == TQ_P2G_FIXED) { p2g_fixed(); return; }
    std::fill(u.begin(), u.end(), (S)0); std::fill(v.begin(), v.end(), (S)0);
    std::fill(uPeso.begin(), uPeso.end(), (S)0); std::fill(vPeso.begin(), vPeso.end(), (S)0);
    std::fill(densidade.begin(), densidade.end(), (S)0);
    std::fill(contagemCelula.begin(), contagemCelula.end(), 0u);
    std::fill(corCelula.begin(), corCelula.end(), (S)0);
    double inv = 1 / h;
    for (int k = 0; k < n; k++) {
      const float* o = p.data() + (size_t)k * CAMPOS;
      double x = o[0], y = o[1], vx = o[2], vy = o[3];
      double cux = o[4], cuy = o[5], cvx = o[6], cvy = o[7];
      {
        double fx = x * inv, fy = y * inv - 0.5;
        int i0 = clampi(floori(fx), 0, nx - 1), j0 = clampi(floori(fy), 0, ny - 2);
        double tx = fx - i0, ty = fy - j0;
        for (int b = 0; b < 2; b++) {
          double wy = b ? ty : 1 - ty;
          double dy = (j0 + b + 0.5) * h - y;
          for (int a = 0; a < 2; a++) {
            double w = (a ? tx : 1 - tx) * wy;
            double dx = (i0 + a) * h - x;
            int idx = i0 + a + (j0 + b) * (nx + 1);
            u[idx] = (S)((double)u[idx] + w * (vx + cux * dx + cuy * dy));
            uPeso[idx] = (S)((double)uPeso[idx] + w);
          }
        }
      }
      {
        double fx = x * inv - 0.5, fy = y * inv;
        int i0 = clampi(floori(fx), 0, nx - 2), j0 = clampi(floori(fy), 0, ny - 1);
        double tx = fx - i0, ty = fy - j0;
        for (int b = 0; b < 2; b++) {
          double wy = b ? ty : 1 - ty;
          double dy = (j0 + b) * h - y;
          for (int a = 0; a < 2; a++) {
            double w = (a ? tx : 1 - tx) * wy;
            double dx = (i0 + a + 0.5) * h - x;
            int idx = i0 + a + (j0 + b) * nx;
            v[idx] = (S)((double)v[idx] + w * (vy + cvx * dx + cvy * dy));
            vPeso[idx] = (S)((double)vPeso[idx] + w);
          }
        }
      }
      {
        double fx = x * inv - 0.5, fy = y * inv - 0.5;
        int i0 = clampi(floori(fx), 0, nx - 2), j0 = clampi(floori(fy), 0, ny - 2);
        double tx = fx - i0, ty = fy - j0;
        int c = i0 + j0 * nx;
        densidade[c] = (S)((double)densidade[c] + (1 - tx) * (1 - ty));
        densidade[c + 1] = (S)((double)densidade[c + 1] + tx * (1 - ty));
        densidade[c + nx] = (S)((double)densidade[c + nx] + (1 - tx) * ty);
        densidade[c + nx + 1] = (S)((double)densidade[c + nx + 1] + tx * ty);
      }
      int ci = clampi(floori(x * inv), 0, nx - 1), cj = clampi(floori(y * inv), 0, ny - 1);
      int cc = ci + cj * nx;
      contagemCelula[cc]++;
      corCelula[cc * 3] = (S)((double)corCelula[cc * 3] + (double)o[9]);
      corCelula[cc * 3 + 1] = (S)((double)corCelula[cc * 3 + 1] + (double)o[10]);
      corCelula[cc * 3 + 2] = (S)((double)corCelula[cc * 3 + 2] + (double)o[11]);
    }
    for (int k = 0; k < nu; k++)
      if (uPeso[k] > 0) u[k] = (S)((double)u[k] / (double)uPeso[k]);
    for (int k = 0; k < nv; k++)
      if (vPeso[k] > 0) v[k] = (S)((double)v[k] / (double)vPeso[k]);
  }

  // Fixed-point P2G: the integer accumulation of js/gpu/fisica.js:81-131, in f32 arithmetic
  // exactly as the CUDA kernel performs it (no fused multiply-add, round half to even):
  //   hf = (float)h, inv = 1.0f/hf
  //   u faces: fx = x*inv, fy = y*inv - 0.5f; i0 = clamp(floor(fx), 0, nx-1), j0 = clamp(floor(fy), 0, ny-2)
  //            tx = fx - i0, ty = fy - j0; w = (a ? tx : 1-tx) * (b ? ty : 1-ty)
  //            dx = (float)(i0+a)*hf - x, dy = ((float)(j0+b) + 0.5f)*hf - y
  //            val = vx + (cux*dx + cuy*dy); acc += (rint(w*val*65536), rint(w*65536))
  //   v faces likewise with fx = x*inv - 0.5f, fy = y*inv, dx = ((float)(i0+a) + 0.5f)*hf - x.
  //   density: fx = x*inv - 0.5f, fy = y*inv - 0.5f, clamp to [0, n-2], rint(weight*65536).
  //   count: clamp(floor(x*inv)), clamp(floor(y*inv)); dye: rint(abs*256) if any abs != 0.
  // The face velocity is then (float)acc / (float)weight and the cell density
  // (float)acc * 2^-16 (exact), as js/gpu/fisica.js:147,176 do.
  void p2g_fixed() {
    int N = nx * ny;
    std::fill(accU.begin(), accU.end(), 0); std::fill(accV.begin(), accV.end(), 0);
    std::fill(accCel.begin(), accCel.end(), 0); std::fill(accCor.begin(), accCor.end(), 0);
    const float hf = (float)h;
    const float inv = 1.0f / hf;
    auto fl = [](float v, int lo, int hi) {
      float f = std::floor(v);
      f = std::fmin(std::fmax(f, (float)lo), (float)hi);
      return (int)f;
    };
    auto rnd = [](float v) { return (int32_t)std::nearbyint(v); };
    for (int k = 0; k < n; k++) {
      const float* o = p.data() + (size_t)k * CAMPOS;
      const float x = o[0], y = o[1], vx = o[2], vy = o[3], cux = o[4], cuy = o[5], cvx = o[6], cvy = o[7];
      {
        float fx = x * inv, fy = y * inv - 0.5f;
        int i0 = fl(fx, 0, nx - 1), j0 = fl(fy, 0, ny - 2);
        float tx = fx - (float)i0, ty = fy - (float)j0;
        for (int b = 0; b < 2; b++)
          for (int a = 0; a < 2; a++) {
            float wx = a ? tx : 1.0f - tx, wy = b ? ty : 1.0f - ty;
            float w = wx * wy;
            float dx = (float)(i0 + a) * hf - x;
            float dy = ((float)(j0 + b) + 0.5f) * hf - y;
            float t1 = cux * dx, t2 = cuy * dy;
            float val = vx + (t1 + t2);
            float wv = w * val;
            int idx = i0 + a + (j0 + b) * (nx + 1);
            accU[2 * idx] += rnd(wv * 65536.0f);
            accU[2 * idx + 1] += rnd(w * 65536.0f);
          }
      }
      {
        float fx = x * inv - 0.5f, fy = y * inv;
        int i0 = fl(fx, 0, nx - 2), j0 = fl(fy, 0, ny - 1);
        float tx = fx - (float)i0, ty = fy - (float)j0;
        for (int b = 0; b < 2; b++)
          for (int a = 0; a < 2; a++) {
            float wx = a ? tx : 1.0f - tx, wy = b ? ty : 1.0f - ty;
            float w = wx * wy;
            float dx = ((float)(i0 + a) + 0.5f) * hf - x;
            float dy = (float)(j0 + b) * hf - y;
            float t1 = cvx * dx, t2 = cvy * dy;
            float val = vy + (t1 + t2);
            float wv = w * val;
            int idx = i0 + a + (j0 + b) * nx;
            accV[2 * idx] += rnd(wv * 65536.0f);
            accV[2 * idx + 1] += rnd(w * 65536.0f);
          }
      }
      {
        float fx = x * inv - 0.5f, fy = y * inv - 0.5f;
        int i0 = fl(fx, 0, nx - 2), j0 = fl(fy, 0, ny - 2);
        float tx = fx - (float)i0, ty = fy - (float)j0;
        float ox = 1.0f - tx, oy = 1.0f - ty;
        int c = i0 + j0 * nx;
        accCel[2 * c] += rnd((ox * oy) * 65536.0f);
        accCel[2 * (c + 1)] += rnd((tx * oy) * 65536.0f);
        accCel[2 * (c + nx)] += rnd((ox * ty) * 65536.0f);
        accCel[2 * (c + nx + 1)] += rnd((tx * ty) * 65536.0f);
      }
      int ci = fl(x * inv, 0, nx - 1), cj = fl(y * inv, 0, ny - 1);
      int cc = ci + cj * nx;
      accCel[2 * cc + 1] += 1;
      if (o[9] != 0.0f || o[10] != 0.0f || o[11] != 0.0f) {
        accCor[3 * cc] += rnd(o[9] * 256.0f);
        accCor[3 * cc + 1] += rnd(o[10] * 256.0f);
        accCor[3 * cc + 2] += rnd(o[11] * 256.0f);
      }
    }
    for (int k = 0; k < nu; k++) {
      int32_t w = accU[2 * k + 1];
      uPeso[k] = (S)((float)w * (1.0f / 65536.0f));
      u[k] = w > 0 ? (S)((float)accU[2 * k] / (float)w) : (S)0;
    }
    for (int k = 0; k < nv; k++) {
      int32_t w = accV[2 * k + 1];
      vPeso[k] = (S)((float)w * (1.0f / 65536.0f));
      v[k] = w > 0 ? (S)((float)accV[2 * k] / (float)w) : (S)0;
    }
    for (int c = 0; c < N; c++) {
      densidade[c] = (S)((float)accCel[2 * c] * (1.0f / 65536.0f));
      contagemCelula[c] = (uint32_t)accCel[2 * c + 1];
      for (int q3 = 0; q3 < 3; q3++) corCelula[3 * c + q3] = (S)((float)accCor[3 * c + q3] * (1.0f / 256.0f));
    }
  }

  // #gravidadeEFronteira, :271-291.  In TQ_P2G_FIXED mode the gravity impulse is added in
  // f32 as (float)(g*dt), matching js/gpu/fisica.js:147 and the CUDA kernel.
  void gravidadeEFronteira(double dt) {
    double gx = gravidade[0], gy = gravidade[1];
    const uint8_t* sol = solidoCelula.data();
    const bool fixo = p2gMode == TQ_P2G_FIXED;
    const float gdx = (float)(gx * dt), gdy = (float)(gy * dt);
    for (int j = 0; j < ny; j++)
      for (int i = 0; i <= nx; i++) {
        int k = i + j * (nx + 1);
        if (uPeso[k] > 0) u[k] = fixo ? (S)((float)u[k] + gdx) : (S)((double)u[k] + gx * dt);
        bool s = i == 0 || i == nx || sol[i - 1 + j * nx] || sol[i + j * nx];
        if (s) u[k] = 0;
      }
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i < nx; i++) {
        int k = i + j * nx;
        if (vPeso[k] > 0) v[k] = fixo ? (S)((float)v[k] + gdy) : (S)((double)v[k] + gy * dt);
        bool s = j == 0 || j == ny || sol[i + (j - 1) * nx] || sol[i + j * nx];
        if (s) v[k] = 0;
      }
  }

  // #tipos, :293-299
  void tipos() {
    tiposProntos = true;
    int N = nx * ny;
    for (int c = 0; c < N; c++) tipo[c] = solidoCelula[c] ? SOLIDO : contagemCelula[c] > 0 ? AGUA : AR;
  }

  // #superficie, :306-346
  void superficie() {
    int N = nx * ny;
    S* f = fase.data();
    S* t = faseTmp.data();
    for (int c = 0; c < N; c++)
      f[c] = tipo[c] == SOLIDO ? (S)0 : (S)std::min(1.0, (double)densidade[c] / PARTICULAS_POR_CELULA);
    const int passadas = 2;
    for (int passada = 0; passada <= passadas; passada++) {
      estenderNaParede(f);
      if (passada == passadas) break;
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          int c = i + j * nx;
          int im = i > 0 ? c - 1 : c, ip = i < nx - 1 ? c + 1 : c;
          t[c] = (S)(((double)f[im] + 2 * (double)f[c] + (double)f[ip]) * 0.25);
        }
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          int c = i + j * nx;
          int jm = j > 0 ? c - nx : c, jp = j < ny - 1 ? c + nx : c;
          f[c] = (S)(((double)t[jm] + 2 * (double)t[c] + (double)t[jp]) * 0.25);
        }
    }
    S *nX = normalX.data(), *nY = normalY.data(), *kap = curvatura.data();
    for (int j = 1; j < ny - 1; j++)
      for (int i = 1; i < nx - 1; i++) {
        int c = i + j * nx;
        double gx = ((double)f[c + 1] - (double)f[c - 1]) * 0.5, gy = ((double)f[c + nx] - (double)f[c - nx]) * 0.5;
        double g = std::hypot(gx, gy);
        nX[c] = g > 1e-3 ? (S)(gx / g) : (S)0;
        nY[c] = g > 1e-3 ? (S)(gy / g) : (S)0;
      }
    for (int j = 1; j < ny - 1; j++)
      for (int i = 1; i < nx - 1; i++) {
        int c = i + j * nx;
        kap[c] = (S)(-(((double)nX[c + 1] - (double)nX[c - 1]) + ((double)nY[c + nx] - (double)nY[c - nx])) / (2 * h));
      }
  }

  // #estenderNaParede, :353-374
  void estenderNaParede(S* f) {
    int N = nx * ny;
    if ((int)preenchido.size() != N) preenchido.assign(N, 0);
    if ((int)novas.size() != N) novas.assign(N, 0);
    uint8_t* cheio = preenchido.data();
    for (int c = 0; c < N; c++) cheio[c] = tipo[c] == SOLIDO ? 0 : 1;
    for (int camada = 0; camada < 3; camada++) {
      int cn = 0;
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          int c = i + j * nx;
          if (cheio[c]) continue;
          double s = 0;
          int k = 0;
          if (i > 0 && cheio[c - 1]) { s += (double)f[c - 1]; k++; }
          if (i < nx - 1 && cheio[c + 1]) { s += (double)f[c + 1]; k++; }
          if (j > 0 && cheio[c - nx]) { s += (double)f[c - nx]; k++; }
          if (j < ny - 1 && cheio[c + nx]) { s += (double)f[c + nx]; k++; }
          if (k) { faseTmp[c] = (S)(s / k); novas[cn++] = c; }
        }
      for (int qn = 0; qn < cn; qn++) {
        int c = novas[qn];
        f[c] = faseTmp[c];
        cheio[c] = 1;
      }
    }
  }

  // #pressaoDoAr, :381-403
  void pressaoDoAr(double dt) {
    double escala = dt / (DENSIDADE_AGUA * h);
    double kMax = 1 / h;
    std::fill(qAr.begin(), qAr.end(), (S)0);
    for (int j = 1; j < ny - 1; j++)
      for (int i = 1; i < nx - 1; i++) {
        int c = i + j * nx;
        if (tipo[c] != AR) continue;
        double pp = 0;
        if (tensao > 0) {
          double s = curvatura[c];
          int k = 1;
          if (tipo[c - 1] == AGUA) { s += (double)curvatura[c - 1]; k++; }
          if (tipo[c + 1] == AGUA) { s += (double)curvatura[c + 1]; k++; }
          if (tipo[c - nx] == AGUA) { s += (double)curvatura[c - nx]; k++; }
          if (tipo[c + nx] == AGUA) { s += (double)curvatura[c + nx]; k++; }
          if (k > 1) pp += tensao * std::max(-kMax, std::min(kMax, s / k));
        }
        qAr[c] = (S)(pp * escala);
      }
  }

  // #propagarRotulos, :409-422
  void propagarRotulos() {
    int N = nx * ny;
    uint32_t* rot = rastreador.rotulo.data();
    for (int c = 0; c < N; c++)
      if (tipo[c] != AR) rot[c] = 0;
    for (int passada = 0; passada < 2; passada++)
      for (int j = 1; j < ny - 1; j++)
        for (int i = 1; i < nx - 1; i++) {
          int c = i + j * nx;
          if (tipo[c] != AR || rot[c]) continue;
          uint32_t r = rot[c - 1];
          if (!r) r = rot[c + 1];
          if (!r) r = rot[c - nx];
          if (!r) r = rot[c + nx];
          rot[c] = r;
        }
  }

  // #ladoDireitoDasBolhas, :429-454
  void ladoDireitoDasBolhas(double dt) {
    const uint32_t* rot = rastreador.rotulo.data();
    std::fill(rhsBolha.begin(), rhsBolha.end(), (S)0);
    std::fill(volumeBolha.begin(), volumeBolha.end(), (S)0);
    for (int j = 1; j < ny - 1; j++)
      for (int i = 1; i < nx - 1; i++) {
        int c = i + j * nx;
        uint32_t r = rot[c];
        if (tipo[c] != AR || r < 2 || r >= (uint32_t)MAX_BOLHAS) continue;
        volumeBolha[r] = (S)((double)volumeBolha[r] + 1);
        double t = qAr[c];
        if (tipo[c - 1] == AGUA) rhsBolha[r] = (S)((double)rhsBolha[r] + ((double)u[i + j * (nx + 1)] - t));
        if (tipo[c + 1] == AGUA) rhsBolha[r] = (S)((double)rhsBolha[r] + (-(double)u[i + 1 + j * (nx + 1)] - t));
        if (tipo[c - nx] == AGUA) rhsBolha[r] = (S)((double)rhsBolha[r] + ((double)v[i + j * nx] - t));
        if (tipo[c + nx] == AGUA) rhsBolha[r] = (S)((double)rhsBolha[r] + (-(double)v[i + (j + 1) * nx] - t));
      }
    const S* alvo = rastreador.volumeAlvo.data();
    double paraQ = dt / (DENSIDADE_AGUA * h);
    for (int r = 2; r < MAX_BOLHAS; r++) {
      if (volumeBolha[r] == 0) continue;
      rhsBolha[r] = (S)((double)rhsBolha[r] + VOLTA_VOLUME_BOLHA * ((double)alvo[r] - (double)volumeBolha[r]) * h / dt);
      yBolha[r] = (S)((double)pressaoBolha[r] * paraQ);
    }
  }

  // Flat-index neighbour read of a typed array: out-of-range reads are `undefined` in JS.
  inline bool tipoIgual(long c, uint8_t t) const {
    return c >= 0 && c < (long)tipo.size() && tipo[c] == t;
  }

  // #classificar, :456-482
  void classificar(double dt) {
    double alvo = h / std::max(tauDensidade, dt);
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        int c = i + j * nx;
        uint8_t t = tipo[c];
        if (t != AGUA) { div[c] = 0; q[c] = 0; continue; }
        double d = (double)u[i + 1 + j * (nx + 1)] - (double)u[i + j * (nx + 1)] +
                   (double)v[i + (j + 1) * nx] - (double)v[i + j * nx];
        double excesso = (double)densidade[c] / PARTICULAS_POR_CELULA - 1;
        if (excesso < 0 && !miolo(i, j)) excesso = 0;
        excesso = std::min(EXCESSO_MAX, std::max(EXCESSO_MIN, excesso));
        double ar = 0;
        if (tipoIgual((long)c - 1, AR)) ar += (double)qAr[c - 1];
        if (tipoIgual((long)c + 1, AR)) ar += (double)qAr[c + 1];
        if (tipoIgual((long)c - nx, AR)) ar += (double)qAr[c - nx];
        if (tipoIgual((long)c + nx, AR)) ar += (double)qAr[c + nx];
        div[c] = (S)(d - alvo * excesso - ar);
      }
  }
  // #miolo, :484-494
  bool miolo(int i, int j) const {
    if (i < 1 || j < 1 || i >= nx - 1 || j >= ny - 1) return false;
    for (int b = -1; b <= 1; b++)
      for (int a = -1; a <= 1; a++) {
        int c = i + a + (j + b) * nx;
        if (solidoCelula[c] || contagemCelula[c] == 0) return false;
      }
    return true;
  }

  // #pressao, :498-515
  void pressao(double dt) {
    BolhasPCG<S> b{rastreador.rotulo.data(), rhsBolha.data(), yBolha.data()};
    normas = resolverPCG(niveis, tipo.data(), div.data(), q.data(), iteracoes, arAtivo ? &b : nullptr, tol, precond,
                         &info);
    solves++;
    itersAcum += info.iters;
    trocasAcum += info.trocas;
    if (tol > 0) {
      if (!info.convergiu) capados++;
      if (info.r0 > 0 && info.rv / info.r0 > maxRel) maxRel = info.rv / info.r0;
    }
    double paraPa = (DENSIDADE_AGUA * h) / dt;
    const uint32_t* rot = rastreador.rotulo.data();
    int N = nx * ny;
    for (int c = 0; c < N; c++) {
      if (tipo[c] != AR) continue;
      uint32_t r = rot[c];
      bool bolha = arAtivo && r >= 2 && r < (uint32_t)MAX_BOLHAS && volumeBolha[r] != 0;
      q[c] = (S)((double)qAr[c] + (bolha ? (double)yBolha[r] : 0.0));
    }
    if (arAtivo)
      for (int r = 2; r < MAX_BOLHAS; r++)
        if (volumeBolha[r] != 0)
          pressaoBolha[r] = (S)std::max(-PRESSAO_BOLHA_MAX, std::min(PRESSAO_BOLHA_MAX, (double)yBolha[r] * paraPa));
  }

  // #gradiente, :519-545
  void gradiente() {
    for (int j = 0; j < ny; j++)
      for (int i = 0; i <= nx; i++) {
        int k = i + j * (nx + 1);
        uint8_t tl = i > 0 ? tipo[i - 1 + j * nx] : SOLIDO;
        uint8_t tr = i < nx ? tipo[i + j * nx] : SOLIDO;
        if (tl == SOLIDO || tr == SOLIDO) { u[k] = 0; uValida[k] = 1; continue; }
        if (tl == AGUA || tr == AGUA) {
          u[k] = (S)((double)u[k] - ((double)q[i + j * nx] - (double)q[i - 1 + j * nx]));
          uValida[k] = 1;
        } else uValida[k] = 0;
      }
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i < nx; i++) {
        int k = i + j * nx;
        uint8_t tb = j > 0 ? tipo[i + (j - 1) * nx] : SOLIDO;
        uint8_t tt = j < ny ? tipo[i + j * nx] : SOLIDO;
        if (tb == SOLIDO || tt == SOLIDO) { v[k] = 0; vValida[k] = 1; continue; }
        if (tb == AGUA || tt == AGUA) {
          v[k] = (S)((double)v[k] - ((double)q[i + j * nx] - (double)q[i + (j - 1) * nx]));
          vValida[k] = 1;
        } else vValida[k] = 0;
      }
  }

  // extrapolarComponente, :673-690
  static void extrapolarComponente(std::vector<S>& a, std::vector<S>& tmp, std::vector<uint8_t>& valida, int w, int hh) {
    tmp = a;
    std::vector<int> nv;
    for (int j = 0; j < hh; j++)
      for (int i = 0; i < w; i++) {
        int k = i + j * w;
        if (valida[k]) continue;
        double soma = 0;
        int n = 0;
        if (i > 0 && valida[k - 1]) { soma += (double)a[k - 1]; n++; }
        if (i < w - 1 && valida[k + 1]) { soma += (double)a[k + 1]; n++; }
        if (j > 0 && valida[k - w]) { soma += (double)a[k - w]; n++; }
        if (j < hh - 1 && valida[k + w]) { soma += (double)a[k + w]; n++; }
        if (n > 0) { tmp[k] = (S)(soma / n); nv.push_back(k); }
      }
    a = tmp;
    for (int k : nv) valida[k] = 1;
  }
  // #extrapolar, :547-552
  void extrapolar() {
    for (int camada = 0; camada < CAMADAS_EXTRAPOLACAO; camada++) {
      extrapolarComponente(u, uTmp, uValida, nx + 1, ny);
      extrapolarComponente(v, vTmp, vValida, nx, ny + 1);
    }
  }

  // #velocidadeEm, :641-661
  void velocidadeEm(double x, double y, double vmax, double* ox, double* oy) const {
    double inv = 1 / h;
    double vx, vy;
    {
      double fx = x * inv, fy = y * inv - 0.5;
      int i0 = clampi(floori(fx), 0, nx - 1), j0 = clampi(floori(fy), 0, ny - 2);
      double tx = fx - i0, ty = fy - j0;
      int k = i0 + j0 * (nx + 1);
      vx = ((double)u[k] * (1 - tx) + (double)u[k + 1] * tx) * (1 - ty) +
           ((double)u[k + nx + 1] * (1 - tx) + (double)u[k + nx + 2] * tx) * ty;
    }
    {
      double fx = x * inv - 0.5, fy = y * inv;
      int i0 = clampi(floori(fx), 0, nx - 2), j0 = clampi(floori(fy), 0, ny - 1);
      double tx = fx - i0, ty = fy - j0;
      int k = i0 + j0 * nx;
      vy = ((double)v[k] * (1 - tx) + (double)v[k + 1] * tx) * (1 - ty) +
           ((double)v[k + nx] * (1 - tx) + (double)v[k + nx + 1] * tx) * ty;
    }
    double vv = std::hypot(vx, vy);
    if (vv > vmax) { *ox = vx * vmax / vv; *oy = vy * vmax / vv; }
    else { *ox = vx; *oy = vy; }
  }

  // #paraParticulas (G2P), :556-638
  void paraParticulas(double dt) {
    double inv = 1 / h;
    double vmax = (MICROPASSO * MAX_MICROPASSOS * h) / dt;
    double decai = std::exp(-dt / ESPUMA_VIDA);
    double mistura = std::min(1.0, dt / DIFUSAO_CORANTE);
    bool mortas = false;
    double maior = 0;
    for (int k = 0; k < n; k++) {
      float* o = p.data() + (size_t)k * CAMPOS;
      double x = o[0], y = o[1];
      double vx = 0, vy = 0, cux = 0, cuy = 0, cvx = 0, cvy = 0;
      {
        double fx = x * inv, fy = y * inv - 0.5;
        int i0 = clampi(floori(fx), 0, nx - 1), j0 = clampi(floori(fy), 0, ny - 2);
        double tx = fx - i0, ty = fy - j0;
        for (int b = 0; b < 2; b++)
          for (int a = 0; a < 2; a++) {
            double val = u[i0 + a + (j0 + b) * (nx + 1)];
            double wx = a ? tx : 1 - tx, wy = b ? ty : 1 - ty;
            vx += wx * wy * val;
            cux += (a ? 1 : -1) * wy * inv * val;
            cuy += wx * (b ? 1 : -1) * inv * val;
          }
      }
      {
        double fx = x * inv - 0.5, fy = y * inv;
        int i0 = clampi(floori(fx), 0, nx - 2), j0 = clampi(floori(fy), 0, ny - 1);
        double tx = fx - i0, ty = fy - j0;
        for (int b = 0; b < 2; b++)
          for (int a = 0; a < 2; a++) {
            double val = v[i0 + a + (j0 + b) * nx];
            double wx = a ? tx : 1 - tx, wy = b ? ty : 1 - ty;
            vy += wx * wy * val;
            cvx += (a ? 1 : -1) * wy * inv * val;
            cvy += wx * (b ? 1 : -1) * inv * val;
          }
      }
      double vel = std::hypot(vx, vy);
      int ci = clampi(floori(x * inv), 0, nx - 1), cj = clampi(floori(y * inv), 0, ny - 1);
      double rarefeita = suave(0.95, 0.45, (double)densidade[ci + cj * nx] / PARTICULAS_POR_CELULA);
      double fonte = suave(ESPUMA_V0, ESPUMA_V1, vel) * rarefeita;
      double espuma = std::min(1.0, (double)o[8] * decai + fonte * ESPUMA_TAXA * dt);
      uint32_t nCel = contagemCelula[ci + cj * nx];
      if (nCel > 1) {
        int cc = (ci + cj * nx) * 3;
        for (int qq = 0; qq < 3; qq++)
          o[9 + qq] = (float)((double)o[9 + qq] + ((double)corCelula[cc + qq] / nCel - (double)o[9 + qq]) * mistura);
      }
      if (vel > vmax) { vx *= vmax / vel; vy *= vmax / vel; }
      if (vel > maior) maior = vel;
      double micro = std::min(MAX_MICROPASSOS, std::max(1.0, std::ceil((std::min(vel, vmax) * dt) / (MICROPASSO * h))));
      double dm = dt / micro;
      bool morta = false;
      for (int m = 0; m < (int)micro; m++) {
        double wx = vx, wy = vy;
        if (micro > 1) velocidadeEm(x, y, vmax, &wx, &wy);
        x += wx * dm;
        y += wy * dm;
        double d = cena.distancia(x, y);
        if (d < RAIO_PARTICULA) {
          if (d < -SDF_MAX + 0.5) { morta = true; break; }
          double nX, nY;
          cena.normal(x, y, &nX, &nY);
          double empurra = (RAIO_PARTICULA - d) * h;
          x += nX * empurra;
          y += nY * empurra;
          double vn = vx * nX + vy * nY;
          if (vn < 0) { vx -= vn * nX; vy -= vn * nY; }
        }
      }
      if (morta) { o[0] = NAN; mortas = true; continue; }
      o[0] = (float)x; o[1] = (float)y; o[2] = (float)vx; o[3] = (float)vy;
      o[4] = (float)cux; o[5] = (float)cuy; o[6] = (float)cvx; o[7] = (float)cvy;
      o[8] = (float)espuma;
    }
    if (mortas) remover([](double x, double, int) { return x != x; });
    vMax = maior;
  }
};

// ------------------------------------------------------------- C interface helpers
thread_local char g_err[256];
int fail(int code, const char* msg) {
  std::snprintf(g_err, sizeof g_err, "%s", msg);
  return code;
}

}  // namespace

// =============================================================== C interface
struct tqo_scene {
  Cena c;
};

struct tqo_sim {
  bool fp64;
  std::unique_ptr<Sim<float>> f;
  std::unique_ptr<Sim<double>> d;
};

template <class S, class T>
static int copiar(std::vector<T>& v, void* out, const void* in, int64_t bytes) {
  (void)sizeof(S);
  if (bytes != (int64_t)(v.size() * sizeof(T))) return fail(TQ_E_ARG, "field size mismatch");
  if (out) std::memcpy(out, v.data(), bytes);
  else std::memcpy(v.data(), in, bytes);
  return TQ_OK;
}
// Float fields are exchanged as f32 even in the FP64 variant.
template <class S>
static int copiarF(std::vector<S>& v, void* out, const void* in, int64_t bytes) {
  if (bytes != (int64_t)(v.size() * sizeof(float))) return fail(TQ_E_ARG, "field size mismatch");
  if (out) {
    float* o = (float*)out;
    for (size_t k = 0; k < v.size(); k++) o[k] = (float)v[k];
  } else {
    const float* i = (const float*)in;
    for (size_t k = 0; k < v.size(); k++) v[k] = (S)i[k];
  }
  return TQ_OK;
}

template <class S>
static int campo(Sim<S>& S_, int32_t field, void* out, const void* in, int64_t bytes) {
  switch (field) {
    case TQ_FIELD_TIPO: return copiar<S>(S_.tipo, out, in, bytes);
    case TQ_FIELD_ROTULO: return copiar<S>(S_.rastreador.rotulo, out, in, bytes);
    case TQ_FIELD_CONTAGEM: return copiar<S>(S_.contagemCelula, out, in, bytes);
    case TQ_FIELD_SOLIDO: return copiar<S>(S_.solidoCelula, out, in, bytes);
    case TQ_FIELD_U: return copiarF(S_.u, out, in, bytes);
    case TQ_FIELD_V: return copiarF(S_.v, out, in, bytes);
    case TQ_FIELD_Q: return copiarF(S_.q, out, in, bytes);
    case TQ_FIELD_DIV: return copiarF(S_.div, out, in, bytes);
    case TQ_FIELD_DENSIDADE: return copiarF(S_.densidade, out, in, bytes);
    case TQ_FIELD_FASE: return copiarF(S_.fase, out, in, bytes);
    case TQ_FIELD_CURVATURA: return copiarF(S_.curvatura, out, in, bytes);
    case TQ_FIELD_QAR: return copiarF(S_.qAr, out, in, bytes);
    case TQ_FIELD_PRESSAO_BOLHA: return copiarF(S_.pressaoBolha, out, in, bytes);
    case TQ_FIELD_VOLUME_ALVO: return copiarF(S_.rastreador.volumeAlvo, out, in, bytes);
    case TQ_FIELD_VOLUME_BOLHA: return copiarF(S_.volumeBolha, out, in, bytes);
    case TQ_FIELD_RHS_BOLHA: return copiarF(S_.rhsBolha, out, in, bytes);
    case TQ_FIELD_Y_BOLHA: return copiarF(S_.yBolha, out, in, bytes);
    case TQ_FIELD_VIVO: return copiar<S>(S_.rastreador.vivo, out, in, bytes);
    case TQ_FIELD_U_VALIDA: return copiar<S>(S_.uValida, out, in, bytes);
    case TQ_FIELD_V_VALIDA: return copiar<S>(S_.vValida, out, in, bytes);
    case TQ_FIELD_U_PESO: return copiarF(S_.uPeso, out, in, bytes);
    case TQ_FIELD_V_PESO: return copiarF(S_.vPeso, out, in, bytes);
    case TQ_FIELD_NORMAL_X: return copiarF(S_.normalX, out, in, bytes);
    case TQ_FIELD_NORMAL_Y: return copiarF(S_.normalY, out, in, bytes);
    case TQ_FIELD_COR_CELULA: return copiarF(S_.corCelula, out, in, bytes);
    case TQ_FIELD_ACC_U: return copiar<S>(S_.accU, out, in, bytes);
    case TQ_FIELD_ACC_V: return copiar<S>(S_.accV, out, in, bytes);
    case TQ_FIELD_ACC_CEL: return copiar<S>(S_.accCel, out, in, bytes);
    case TQ_FIELD_ACC_COR: return copiar<S>(S_.accCor, out, in, bytes);
    case TQ_FIELD_SDF: {
      int st = copiar<S>(S_.cena.sdf, out, in, bytes);
      if (!out && st == TQ_OK) S_.atualizarParedes();
      return st;
    }
  }
  return fail(TQ_E_ARG, "unknown field");
}

extern "C" {

tqo_scene* tqo_scene_new(int32_t nx, int32_t ny, double h) { return new tqo_scene{Cena(nx, ny, h)}; }
void tqo_scene_free(tqo_scene* c) { delete c; }
void tqo_scene_trace(tqo_scene* c, double x0, double y0, double x1, double y1, double radius, int32_t erase) {
  c->c.tracar(x0, y0, x1, y1, radius, erase != 0);
}
void tqo_scene_clear(tqo_scene* c) { c->c.zerar(); }
const float* tqo_scene_sdf(tqo_scene* c) { return c->c.sdf.data(); }
double tqo_scene_distance(tqo_scene* c, double x, double y) { return c->c.distancia(x, y); }
void tqo_scene_normal(tqo_scene* c, double x, double y, double* nx, double* ny) { c->c.normal(x, y, nx, ny); }
int32_t tqo_scene_solid_cell(tqo_scene* c, int32_t i, int32_t j) { return c->c.celulaSolida(i, j) ? 1 : 0; }

// WGSL_MANCHA (js/gpu/render.js:11-43) restated on the CPU: the w x h target covers the tank
// (W = nx h, H = ny h as f32, row 0 at the top); a live particle (x >= 0) adds at each pixel
// centre within raio = RAIO_MANCHA h (f32) the weight (1 - r^2)^2, r = |centre - position| /
// raio, and that weight times its extra vector (foam, three absorptions), in f32 arithmetic;
// the sums are 64-bit fixed point (2^32) and `out` gets them as floats, 5 planes of w x h.
void tqo_splat(const float* p12, int32_t n, int32_t nx, int32_t ny, double h, int32_t w, int32_t hp, float* out) {
  const size_t plano = (size_t)w * hp;
  std::vector<long long> acc(5 * plano, 0);
  const float W = (float)(nx * h), H = (float)(ny * h), raio = (float)(2.1 * h);
  const float px = W / (float)w, py = H / (float)hp;
  auto fixo = [](float v) { return (long long)std::nearbyint((double)v * 4294967296.0); };
  for (int32_t k = 0; k < n; k++) {
    const float* p = p12 + (size_t)k * CAMPOS;
    const float x = p[0], y = p[1];
    if (!(x == x) || !(y == y) || x < 0.0f) continue;
    const float e[4] = {p[8], p[9], p[10], p[11]};
    const int i0 = std::max(0, (int)std::floor((x - raio) / px - 0.5f) - 1);
    const int i1 = std::min(w - 1, (int)std::ceil((x + raio) / px - 0.5f) + 1);
    const int j0 = std::max(0, (int)std::floor((H - (y + raio)) / py - 0.5f) - 1);
    const int j1 = std::min(hp - 1, (int)std::ceil((H - (y - raio)) / py - 0.5f) + 1);
    for (int j = j0; j <= j1; j++) {
      const float v = ((H - ((float)j + 0.5f) * py) - y) / raio;
      for (int i = i0; i <= i1; i++) {
        const float u = (((float)i + 0.5f) * px - x) / raio;
        const float r2 = u * u + v * v;
        if (r2 >= 1.0f) continue;
        const float wt = (1.0f - r2) * (1.0f - r2);
        const size_t q = (size_t)j * w + i;
        acc[q] += fixo(wt);
        for (int c = 0; c < 4; c++)
          if (e[c] != 0.0f) acc[(c + 1) * plano + q] += fixo(wt * e[c]);
      }
    }
  }
  for (size_t q = 0; q < 5 * plano; q++) out[q] = (float)((double)acc[q] * (1.0 / 4294967296.0));
}

// passoMaximo, js/constantes.js:167-175
double tqo_passo_maximo(double h, double altura, double vmax, int32_t has_vmax, double dt_frame) {
  double queda = std::sqrt(2 * GRAVIDADE * altura) * 1.15 + 0.5;
  double v = !has_vmax ? queda : std::min(queda, vmax * 1.2 + GRAVIDADE * dt_frame + 0.25);
  double capilar = FATOR_CAPILAR * std::sqrt((DENSIDADE_AGUA * h * h * h) / (2 * M_PI * TENSAO_SUPERFICIAL));
  return std::min(std::min((CFL * h) / std::max(v, 0.3), capilar), PASSO_MAX);
}

// dimensoesDaGrade, js/constantes.js:152-160
void tqo_dimensoes(double largura, double altura, int32_t celulas, double h_min, int32_t* nx, int32_t* ny, double* h) {
  double hh = std::sqrt((largura * altura) / celulas);
  hh = std::max(hh, h_min);
  double fy = std::max(24.0, std::round(altura / hh));
  hh = altura / fy;
  double fx = std::max(24.0, std::round(largura / hh));
  *nx = (int32_t)fx;
  *ny = (int32_t)fy;
  *h = hh;
}

// semearRetangulo (js/fisica-cpu.js:705-727) with semente (testes/apoio.js:4-9).
// Note: Math.round rounds half up; std::round rounds half away from zero — identical for the
// non-negative arguments used here (sqrt(4) = 2).
int32_t tqo_semear_retangulo(double x0, double y0, double x1, double y1, double h, const double* absorb,
                             uint32_t* seed, float* out, int32_t cap) {
  double lado = std::round(std::sqrt(PARTICULAS_POR_CELULA));
  double passo = h / lado;
  double xa = std::min(x0, x1), xb = std::max(x0, x1);
  double ya = std::min(y0, y1), yb = std::max(y0, y1);
  double ia = std::ceil(xa / passo - 0.5), ib = std::floor(xb / passo - 0.5);
  double ja = std::ceil(ya / passo - 0.5), jb = std::floor(yb / passo - 0.5);
  double nn = std::max(0.0, ib - ia + 1) * std::max(0.0, jb - ja + 1);
  int32_t n = (int32_t)nn;
  if (!out) return n;
  if (n > cap) return -1;
  uint32_t s = *seed;
  auto aleatorio = [&]() {
    s = s * 1664525u + 1013904223u;
    return s / 4294967296.0;
  };
  int k = 0;
  for (double j = ja; j <= jb; j++)
    for (double i = ia; i <= ib; i++) {
      float* o = out + (size_t)k * CAMPOS;
      std::memset(o, 0, CAMPOS * sizeof(float));
      o[0] = (float)((i + 0.5 + (aleatorio() - 0.5) * 0.5) * passo);
      o[1] = (float)((j + 0.5 + (aleatorio() - 0.5) * 0.5) * passo);
      o[9] = (float)absorb[0];
      o[10] = (float)absorb[1];
      o[11] = (float)absorb[2];
      k++;
    }
  *seed = s;
  return n;
}

static int validar(const tq_options* o) {
  if (!o) return fail(TQ_E_ARG, "null options");
  if (o->nx < 3 || o->ny < 3 || !(o->h > 0)) return fail(TQ_E_ARG, "grid must be at least 3x3 with h > 0");
  if (o->iterations < 1) return fail(TQ_E_ARG, "iterations must be >= 1");
  if (o->p2g_mode != TQ_P2G_FLOAT && o->p2g_mode != TQ_P2G_FIXED) return fail(TQ_E_ARG, "bad p2g_mode");
  if (o->preconditioner < TQ_PRECOND_REFERENCE || o->preconditioner > TQ_PRECOND_BLOCK_1)
    return fail(TQ_E_ARG, "bad preconditioner");
  return TQ_OK;
}

int tqo_create(const tq_options* o, tqo_sim** out) {
  int st = validar(o);
  if (st) return st;
  if (!out) return fail(TQ_E_ARG, "null out");
  auto* s = new tqo_sim{false, std::make_unique<Sim<float>>(*o), nullptr};
  *out = s;
  return TQ_OK;
}
int tqo_create_fp64(const tq_options* o, tqo_sim** out) {
  int st = validar(o);
  if (st) return st;
  if (!out) return fail(TQ_E_ARG, "null out");
  auto* s = new tqo_sim{true, nullptr, std::make_unique<Sim<double>>(*o)};
  *out = s;
  return TQ_OK;
}
int tqo_destroy(tqo_sim* s) {
  delete s;
  return TQ_OK;
}

#define TQO_DISPATCH(s, expr)        \
  do {                               \
    if (!s) return fail(TQ_E_ARG, "null handle"); \
    if (s->fp64) { auto& S_ = *s->d; expr; } \
    else { auto& S_ = *s->f; expr; } \
  } while (0)

int tqo_set_walls(tqo_sim* s, const float* sdf, int32_t mw, int32_t mh) {
  TQO_DISPATCH(s, {
    if (!sdf || mw != S_.cena.mw || mh != S_.cena.mh) return fail(TQ_E_ARG, "sdf size must be 2nx x 2ny");
    std::copy(sdf, sdf + (size_t)mw * mh, S_.cena.sdf.begin());
    S_.atualizarParedes();
  });
  return TQ_OK;
}
int tqo_add_particles(tqo_sim* s, const float* list, int32_t n, int32_t check, int32_t* accepted) {
  TQO_DISPATCH(s, {
    if (n < 0 || (n > 0 && !list)) return fail(TQ_E_ARG, "bad particle list");
    if (S_.n + n > S_.capacidade) return fail(TQ_E_CAPACITY, "particle capacity exceeded");
    int a = S_.adicionar(list, n, check != 0);
    if (accepted) *accepted = a;
  });
  return TQ_OK;
}
int tqo_clear_particles(tqo_sim* s) {
  TQO_DISPATCH(s, {
    S_.n = 0;
    S_.p.clear();
    std::fill(S_.contagemCelula.begin(), S_.contagemCelula.end(), 0u);
  });
  return TQ_OK;
}
int tqo_apply_tool(tqo_sim* s, const tq_tool* t) {
  if (!t) return fail(TQ_E_ARG, "null tool");
  TQO_DISPATCH(s, S_.aplicarFerramenta(*t));
  return TQ_OK;
}
int tqo_advance(tqo_sim* s, double dt, int32_t sub) {
  if (sub < 1 || !(dt > 0)) return fail(TQ_E_ARG, "need dt > 0 and substeps >= 1");
  TQO_DISPATCH(s, S_.avancar(dt, sub));
  return TQ_OK;
}
int tqo_substep(tqo_sim* s, double dt) {
  if (!(dt > 0)) return fail(TQ_E_ARG, "need dt > 0");
  TQO_DISPATCH(s, S_.subpasso(dt));
  return TQ_OK;
}
int tqo_update_air(tqo_sim* s) {
  TQO_DISPATCH(s, S_.atualizarAr());
  return TQ_OK;
}
int tqo_reset_air(tqo_sim* s) {
  TQO_DISPATCH(s, S_.reiniciarAr());
  return TQ_OK;
}
int tqo_count(tqo_sim* s, int32_t* n) {
  TQO_DISPATCH(s, { if (n) *n = S_.n; });
  return TQ_OK;
}
int tqo_get_particles(tqo_sim* s, float* out, int32_t cap, int32_t* n) {
  TQO_DISPATCH(s, {
    if (n) *n = S_.n;
    if (out) {
      if (cap < S_.n) return fail(TQ_E_ARG, "output buffer too small");
      std::copy(S_.p.begin(), S_.p.begin() + (size_t)S_.n * CAMPOS, out);
    }
  });
  return TQ_OK;
}
int tqo_set_particles(tqo_sim* s, const float* list, int32_t n) {
  TQO_DISPATCH(s, {
    if (n < 0 || (n > 0 && !list)) return fail(TQ_E_ARG, "bad particle list");
    if (n > S_.capacidade) return fail(TQ_E_CAPACITY, "particle capacity exceeded");
    S_.p.assign(list, list + (size_t)n * CAMPOS);
    S_.n = n;
  });
  return TQ_OK;
}

int tqo_get_field(tqo_sim* s, int32_t field, void* out, int64_t bytes) {
  if (!out) return fail(TQ_E_ARG, "null out");
  TQO_DISPATCH(s, return campo(S_, field, out, nullptr, bytes));
}
int tqo_set_field(tqo_sim* s, int32_t field, const void* in, int64_t bytes) {
  if (!in) return fail(TQ_E_ARG, "null in");
  TQO_DISPATCH(s, return campo(S_, field, nullptr, in, bytes));
}
int tqo_get_scalar(tqo_sim* s, int32_t which, double* out) {
  if (!out) return fail(TQ_E_ARG, "null out");
  TQO_DISPATCH(s, {
    switch (which) {
      case TQ_SCALAR_VMAX: *out = S_.vMax; break;
      case TQ_SCALAR_PRIMEIRA: *out = S_.rastreador.primeira ? 1 : 0; break;
      case TQ_SCALAR_TIPOS_PRONTOS: *out = S_.tiposProntos ? 1 : 0; break;
      case TQ_SCALAR_PCG_ITERS: *out = S_.normas.empty() ? 0 : (double)(S_.normas.size() - 1); break;
      case TQ_SCALAR_PCG_RES0: *out = S_.normas.empty() ? 0 : S_.normas.front(); break;
      case TQ_SCALAR_PCG_RES: *out = S_.normas.empty() ? 0 : S_.normas.back(); break;
      case TQ_SCALAR_GRAVITY_X: *out = S_.gravidade[0]; break;
      case TQ_SCALAR_GRAVITY_Y: *out = S_.gravidade[1]; break;
      case TQ_SCALAR_PCG_TRUE_RES: *out = S_.info.rv; break;
      case TQ_SCALAR_PCG_CONVERGED: *out = S_.info.convergiu; break;
      case TQ_SCALAR_SOLVES: *out = (double)S_.solves; break;
      case TQ_SCALAR_SOLVES_CAPPED: *out = (double)S_.capados; break;
      case TQ_SCALAR_SOLVE_ITERS: *out = (double)S_.itersAcum; break;
      case TQ_SCALAR_SOLVE_MAX_REL: *out = S_.maxRel; break;
      case TQ_SCALAR_SOLVE_REPLACEMENTS: *out = (double)S_.trocasAcum; break;
      case TQ_SCALAR_CLOSED_REGIONS: *out = S_.info.regioes; break;
      case TQ_SCALAR_GRAPH_FRAME_MS: *out = 0.0; break;  // no graphs on the CPU
      default: return fail(TQ_E_ARG, "unknown scalar");
    }
  });
  return TQ_OK;
}
int tqo_set_scalar(tqo_sim* s, int32_t which, double value) {
  TQO_DISPATCH(s, {
    switch (which) {
      case TQ_SCALAR_VMAX: S_.vMax = value; break;
      case TQ_SCALAR_PRIMEIRA: S_.rastreador.primeira = value != 0; break;
      case TQ_SCALAR_TIPOS_PRONTOS: S_.tiposProntos = value != 0; break;
      case TQ_SCALAR_GRAVITY_X: S_.gravidade[0] = value; break;  // sim.gravidade (js/motor.js:96)
      case TQ_SCALAR_GRAVITY_Y: S_.gravidade[1] = value; break;
      case TQ_SCALAR_SOLVES:  // 0 resets the accumulated solve statistics
        if (value != 0) return fail(TQ_E_ARG, "TQ_SCALAR_SOLVES can only be reset to 0");
        S_.solves = S_.capados = S_.itersAcum = S_.trocasAcum = 0;
        S_.maxRel = 0;
        break;
      default: return fail(TQ_E_ARG, "scalar not writable");
    }
  });
  return TQ_OK;
}
int tqo_last_norms(tqo_sim* s, double* out, int32_t cap, int32_t* n) {
  TQO_DISPATCH(s, {
    if (n) *n = (int32_t)S_.normas.size();
    if (out)
      for (int32_t k = 0; k < cap && k < (int32_t)S_.normas.size(); k++) out[k] = S_.normas[k];
  });
  return TQ_OK;
}

int tqo_solve_pressure(int32_t nx, int32_t ny, const uint8_t* tipo, const float* div, float* q,
                       int32_t iterations, double tolerance, const tq_bubbles* bubbles,
                       int32_t preconditioner, double* norms, int32_t norms_cap, int32_t* n_norms,
                       tq_solve_info* info) {
  if (nx < 3 || ny < 3 || !tipo || !div || !q || iterations < 1) return fail(TQ_E_ARG, "bad arguments");
  if (preconditioner < TQ_PRECOND_REFERENCE || preconditioner > TQ_PRECOND_BLOCK_1)
    return fail(TQ_E_ARG, "bad preconditioner");
  Niveis<float> L;
  montarNiveis(L, nx, ny);
  BolhasPCG<float> b{};
  std::vector<float> rhs, y;
  if (bubbles) {
    if (!bubbles->rotulo || !bubbles->rhs || !bubbles->y) return fail(TQ_E_ARG, "bad bubbles");
    b.rotulo = bubbles->rotulo;
    b.rhs = bubbles->rhs;
    b.y = bubbles->y;
  }
  InfoPCG inf;
  auto normas = resolverPCG<float>(L, tipo, div, q, iterations, bubbles ? &b : nullptr, tolerance, preconditioner, &inf);
  if (info) {
    info->iterations = inf.iters;
    info->converged = inf.convergiu;
    info->replacements = inf.trocas;
    info->closed_regions = inf.regioes;
    info->residual0 = inf.r0;
    info->residual = inf.r;
    info->true_residual = inf.rv;
  }
  if (n_norms) *n_norms = (int32_t)normas.size();
  if (norms)
    for (int32_t k = 0; k < norms_cap && k < (int32_t)normas.size(); k++) norms[k] = normas[k];
  return TQ_OK;
}

int tqo_vcycle(int32_t nx, int32_t ny, const uint8_t* tipo, const float* b, float* x) {
  if (nx < 3 || ny < 3 || !tipo || !b || !x) return fail(TQ_E_ARG, "bad arguments");
  Niveis<float> L;
  montarNiveis(L, nx, ny);
  size_t k = (size_t)nx * ny;
  std::copy(tipo, tipo + k, L.n[0].tipo.begin());
  tiposGrossos(L);
  for (auto& n : L.n) prepararVizinhos(n);
  std::copy(b, b + k, L.n[0].b.begin());
  cicloV(L);
  std::copy(L.n[0].x.begin(), L.n[0].x.end(), x);
  return TQ_OK;
}

const char* tqo_last_error(void) { return g_err; }

}  // extern "C"
