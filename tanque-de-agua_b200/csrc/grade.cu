// grade.cu — per-cell and per-face kernels of the substep between the particle transfers and
// around the pressure solve: wall cells, cell flags, air-label propagation, surface fraction /
// normal / curvature, surface-tension air pressure, divergence with density correction,
// bubble right-hand sides, air pressure after the solve, pressure gradient and velocity
// extrapolation.
//
// Built with -fmad=false and written in double arithmetic with f32 stores, the way the
// reference's JavaScript computes (double locals, Float32Array stores): these stages then
// agree with the oracle bit for bit except where a transcendental (hypot) is involved.
#include "common.cuh"
#include "kernels.cuh"

namespace tq {

// Cena.celulaSolida (js/cena.js:119-127) for every cell: SimulacaoCPU.atualizarParedes.
__global__ void k_solidos(Dev d) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N) return;
  int i = c % d.nx, j = c / d.nx;
  int a = i * RES_MASCARA, b = j * RES_MASCARA;
  const float* s = d.sdf;
  double soma = (double)s[(size_t)b * d.mw + a] + (double)s[(size_t)b * d.mw + a + 1] +
                (double)s[(size_t)(b + 1) * d.mw + a] + (double)s[(size_t)(b + 1) * d.mw + a + 1];
  d.solido[c] = soma < 0 ? 1 : 0;
}

// Cena#moldura (js/cena.js:131-137): distance (cells) from mask point (x, y) to the frame's
// inner edge, positive inside the tank, clamped to +-SDF_MAX.
__device__ double molduraMascara(int x, int y, int mw, int mh) {
  const double m = MOLDURA * RES_MASCARA - 0.5;
  const double d = fmin(fmin(x - m, (double)(mw - 1) - m - x), fmin(y - m, (double)(mh - 1) - m - y)) / RES_MASCARA;
  return d > SDF_MAX ? SDF_MAX : d < -SDF_MAX ? -SDF_MAX : d;
}

// Cena.tracar (js/cena.js:43-72) on the device mask: one thread per mask point of the
// segment's box (x0, y0, nbx x nby), the capsule distance in double precision as the reference
// computes it, min into the mask (draw) or max of its negation capped by the frame (erase).
__global__ void k_tracar(float* sdf, int mw, int mh, int x0, int y0, int nbx, int nby, double ax, double ay, double dx,
                         double dy, double len2, double rp, int apagar) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nbx * nby) return;
  const int x = x0 + idx % nbx, y = y0 + idx / nbx;
  double t = len2 > 0 ? ((x - ax) * dx + (y - ay) * dy) / len2 : 0;
  t = t < 0 ? 0 : t > 1 ? 1 : t;
  const double px = ax + t * dx - x, py = ay + t * dy - y;
  double d = (sqrt(px * px + py * py) - rp) / RES_MASCARA;
  if (d > SDF_MAX) d = SDF_MAX;
  else if (d < -SDF_MAX) d = -SDF_MAX;
  const size_t k = (size_t)y * mw + x;
  double v = apagar ? fmax((double)sdf[k], -d) : fmin((double)sdf[k], d);
  if (apagar) v = fmin(v, molduraMascara(x, y, mw, mh));
  sdf[k] = (float)v;
}

// Cena#zerar (js/cena.js:139-144): the mask of an empty tank, the frame alone.
__global__ void k_zerar_mascara(float* sdf, int mw, int mh) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= mw * mh) return;
  sdf[idx] = (float)molduraMascara(idx % mw, idx / mw, mw, mh);
}

// #tipos (js/fisica-cpu.js:293-299); with `ar`, the first step of #propagarRotulos (:412,
// non-air cells lose their label) and the initial water fraction of #superficie (:309).
__global__ void k_tipos(Dev d, int ar, int fase) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N) return;
  uint8_t t = d.solido[c] ? SOLIDO : d.accCel[c].y > 0 ? AGUA : AR;
  d.tipo[c] = t;
  if (ar && t != AR) d.rotulo[c] = 0;
  if (fase) {
    double dens = (float)d.accCel[c].x * (1.0f / 65536.0f);
    d.fase[c] = t == SOLIDO ? 0.0f : (float)fmin(1.0, dens / PARTICULAS_POR_CELULA);
  }
}

// ---------------------------------------------------------------- label propagation
// #propagarRotulos (js/fisica-cpu.js:409-422): two in-place raster passes over the interior;
// an unlabelled air cell takes the first non-zero of (left, right, down, up).  In raster order
// the left and lower neighbours already hold this pass's value while the right and upper ones
// hold the value from before the pass.  That makes each pass a system whose dependencies
// point only backwards in raster order, so it has exactly one solution, and repeating the
// update until nothing changes reaches it whatever order the cells are visited in.  Only the
// cells that were unlabelled air at the start of the pass ("pending") change; for a pending
// right/upper neighbour the before-the-pass value is 0.
__global__ void k_rotulos_pendentes(Dev d, int passada) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N) return;
  int i = c % d.nx, j = c / d.nx;
  bool interior = i >= 1 && j >= 1 && i < d.nx - 1 && j < d.ny - 1;
  bool p = interior && d.tipo[c] == AR && d.rotulo[c] == 0;
  if (passada > 0) p = p && d.pend[c];
  d.pend[c] = p ? 1 : 0;
  if (p) {
    int slot = atomicAdd(&d.esc->pendentes, 1);
    d.lista[slot] = c;
  }
}

__global__ void k_rotulos_resolver(Dev d) {
  __shared__ int mudou;
  const int n = d.esc->pendentes;
  const int nx = d.nx;
  uint32_t* rot = d.rotulo;
  const uint8_t* pend = d.pend;
  // Each sweep fixes at least one more cell of the longest dependency chain; n + 2 sweeps
  // always suffice.
  for (int volta = 0; volta < n + 2; volta++) {
    if (threadIdx.x == 0) mudou = 0;
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
      int c = d.lista[t];
      uint32_t r = rot[c - 1];
      if (!r) r = pend[c + 1] ? 0u : rot[c + 1];
      if (!r) r = rot[c - nx];
      if (!r) r = pend[c + nx] ? 0u : rot[c + nx];
      if (r != rot[c]) {
        rot[c] = r;
        mudou = 1;
      }
    }
    __syncthreads();
    if (!mudou) break;
    __syncthreads();
  }
  if (threadIdx.x == 0) d.esc->pendentes = 0;
}

// ---------------------------------------------------------------- surface
// #estenderNaParede (js/fisica-cpu.js:353-374): three layers, each a wall cell not yet filled
// takes the mean of its filled 4-neighbours.  `marca` records the layer a wall cell was
// filled in (255: not yet); a neighbour counts as filled in layer L if it is not a wall or was
// filled in an earlier layer, so f can be updated in place.
__global__ void k_estender(Dev d, int camada) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N) return;
  uint8_t* marca = d.cheio;
  if (d.tipo[c] != SOLIDO) return;
  if (camada > 1 && marca[c] < camada) return;
  int i = c % d.nx, j = c / d.nx;
  const int nx = d.nx, ny = d.ny;
  auto cheio = [&](int n) { return d.tipo[n] != SOLIDO || (camada > 1 && marca[n] < camada); };
  double s = 0;
  int k = 0;
  float* f = d.fase;
  if (i > 0 && cheio(c - 1)) { s += (double)f[c - 1]; k++; }
  if (i < nx - 1 && cheio(c + 1)) { s += (double)f[c + 1]; k++; }
  if (j > 0 && cheio(c - nx)) { s += (double)f[c - nx]; k++; }
  if (j < ny - 1 && cheio(c + nx)) { s += (double)f[c + nx]; k++; }
  if (k) {
    d.faseTmp[c] = (float)(s / k);
    marca[c] = (uint8_t)camada;
  } else if (camada == 1) {
    marca[c] = 255;
  }
}
// The new values of a layer land in faseTmp and are committed here, so no cell of the layer
// reads a value written in the same layer.
__global__ void k_estender_gravar(Dev d, int camada) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N) return;
  if (d.tipo[c] == SOLIDO && d.cheio[c] == camada) d.fase[c] = d.faseTmp[c];
}

// The separable (1 2 1)/4 blur of #superficie (js/fisica-cpu.js:314-328).
__global__ void k_borrar_x(Dev d) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N) return;
  int i = c % d.nx;
  int im = i > 0 ? c - 1 : c, ip = i < d.nx - 1 ? c + 1 : c;
  const float* f = d.fase;
  d.faseTmp[c] = (float)(((double)f[im] + 2 * (double)f[c] + (double)f[ip]) * 0.25);
}
__global__ void k_borrar_y(Dev d) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N) return;
  int j = c / d.nx;
  int jm = j > 0 ? c - d.nx : c, jp = j < d.ny - 1 ? c + d.nx : c;
  const float* t = d.faseTmp;
  d.fase[c] = (float)(((double)t[jm] + 2 * (double)t[c] + (double)t[jp]) * 0.25);
}

// Normal = grad f / |grad f| and curvature = -div n / (2h) on the interior
// (js/fisica-cpu.js:330-345).  Border cells are never written (they stay 0).
__global__ void k_normais(Dev d) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N) return;
  int i = c % d.nx, j = c / d.nx;
  if (i < 1 || j < 1 || i >= d.nx - 1 || j >= d.ny - 1) return;
  const float* f = d.fase;
  double gx = ((double)f[c + 1] - (double)f[c - 1]) * 0.5, gy = ((double)f[c + d.nx] - (double)f[c - d.nx]) * 0.5;
  double g = hypot(gx, gy);
  d.nX[c] = g > 1e-3 ? (float)(gx / g) : 0.0f;
  d.nY[c] = g > 1e-3 ? (float)(gy / g) : 0.0f;
}
__global__ void k_curvatura(Dev d) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N) return;
  int i = c % d.nx, j = c / d.nx;
  if (i < 1 || j < 1 || i >= d.nx - 1 || j >= d.ny - 1) return;
  double a = ((double)d.nX[c + 1] - (double)d.nX[c - 1]) + ((double)d.nY[c + d.nx] - (double)d.nY[c - d.nx]);
  d.kap[c] = (float)(-a / (2 * d.h));
}

// #pressaoDoAr (js/fisica-cpu.js:381-403): surface-tension jump on interior air cells, in
// units of q = p*dt/(rho*h).
__global__ void k_pressao_ar(Dev d, double dt, double tensao) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N) return;
  int i = c % d.nx, j = c / d.nx;
  const int nx = d.nx;
  float out = 0.0f;
  if (i >= 1 && j >= 1 && i < nx - 1 && j < d.ny - 1 && d.tipo[c] == AR) {
    double pp = 0;
    if (tensao > 0) {
      const float* kap = d.kap;
      double s = kap[c];
      int k = 1;
      if (d.tipo[c - 1] == AGUA) { s += (double)kap[c - 1]; k++; }
      if (d.tipo[c + 1] == AGUA) { s += (double)kap[c + 1]; k++; }
      if (d.tipo[c - nx] == AGUA) { s += (double)kap[c - nx]; k++; }
      if (d.tipo[c + nx] == AGUA) { s += (double)kap[c + nx]; k++; }
      double kMax = 1 / d.h;
      if (k > 1) pp += tensao * fmax(-kMax, fmin(kMax, s / k));
    }
    out = (float)(pp * (dt / (DENSIDADE_AGUA * d.h)));
  }
  d.qAr[c] = out;
}

// #classificar + #miolo (js/fisica-cpu.js:456-494): the right-hand side of the projection,
// divergence minus the density correction minus the known air pressure of neighbours.
__global__ void k_classificar(Dev d, double dt, double tau) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N) return;
  const int nx = d.nx, ny = d.ny;
  int i = c % nx, j = c / nx;
  if (d.tipo[c] != AGUA) {
    d.div[c] = 0.0f;
    d.q[c] = 0.0f;
    return;
  }
  double alvo = d.h / fmax(tau, dt);
  double dv = (double)d.u[i + 1 + j * (nx + 1)] - (double)d.u[i + j * (nx + 1)] +
              (double)d.v[i + (j + 1) * nx] - (double)d.v[i + j * nx];
  double dens = (float)d.accCel[c].x * (1.0f / 65536.0f);
  double excesso = dens / PARTICULAS_POR_CELULA - 1;
  if (excesso < 0) {
    bool miolo = i >= 1 && j >= 1 && i < nx - 1 && j < ny - 1;
    for (int b = -1; b <= 1 && miolo; b++)
      for (int a = -1; a <= 1; a++) {
        int n = i + a + (j + b) * nx;
        if (d.solido[n] || d.accCel[n].y == 0) { miolo = false; break; }
      }
    if (!miolo) excesso = 0;
  }
  excesso = fmin(EXCESSO_MAX, fmax(EXCESSO_MIN, excesso));
  double ar = 0;
  long N = d.N;
  if (tipoEm(d.tipo, (long)c - 1, N, AR)) ar += (double)d.qAr[c - 1];
  if (tipoEm(d.tipo, (long)c + 1, N, AR)) ar += (double)d.qAr[c + 1];
  if (tipoEm(d.tipo, (long)c - nx, N, AR)) ar += (double)d.qAr[c - nx];
  if (tipoEm(d.tipo, (long)c + nx, N, AR)) ar += (double)d.qAr[c + nx];
  d.div[c] = (float)(dv - alvo * excesso - ar);
}

// #ladoDireitoDasBolhas (js/fisica-cpu.js:429-454): per bubble, the water flowing into it
// now minus the surface-tension term of each water face, its cell count, then the volume
// recovery term and the initial pressure guess.  The per-bubble sums are 64-bit fixed point
// (2^-32) so their value does not depend on the order cells arrive in.
__global__ void k_bolhas_somar(Dev d) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N) return;
  const int nx = d.nx;
  int i = c % nx, j = c / nx;
  if (i < 1 || j < 1 || i >= nx - 1 || j >= d.ny - 1) return;
  uint32_t r = d.rotulo[c];
  if (d.tipo[c] != AR || r < 2 || r >= (uint32_t)MAX_BOLHAS) return;
  atomicAdd(&d.volB[r], 1u);
  double t = d.qAr[c];
  double s = 0;
  if (d.tipo[c - 1] == AGUA) s += (double)d.u[i + j * (nx + 1)] - t;
  if (d.tipo[c + 1] == AGUA) s += -(double)d.u[i + 1 + j * (nx + 1)] - t;
  if (d.tipo[c - nx] == AGUA) s += (double)d.v[i + j * nx] - t;
  if (d.tipo[c + nx] == AGUA) s += -(double)d.v[i + (j + 1) * nx] - t;
  somaFixa(&d.accB[r], s, ESCALA_BOLHA);
}

__global__ void k_bolhas_fechar(Dev d, double dt) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= MAX_BOLHAS) return;
  uint32_t vol = r >= 2 ? d.volB[r] : 0u;
  double soma = (double)d.accB[r] / ESCALA_BOLHA;
  float rhs = (float)soma;
  d.volumeBolhaF[r] = (float)vol;
  if (vol) {
    rhs = (float)((double)rhs + VOLTA_VOLUME_BOLHA * ((double)d.volumeAlvo[r] - (double)vol) * d.h / dt);
    float y = (float)((double)d.pressaoBolha[r] * (dt / (DENSIDADE_AGUA * d.h)));
    d.yBolhaF[r] = y;
  }
  d.rhsBolhaF[r] = rhs;
  d.rhsB[r] = rhs;
  d.yB[r] = d.yBolhaF[r];
}

// #pressao after resolverPCG (js/fisica-cpu.js:503-514): air cells get the surface-tension
// pressure plus their bubble's pressure; bubbles keep their pressure in Pa (clamped).
__global__ void k_pos_pressao(Dev d, int ar) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.N) return;
  if (d.tipo[c] != AR) return;
  uint32_t r = d.rotulo[c];
  bool bolha = ar && r >= 2 && r < (uint32_t)MAX_BOLHAS && d.volumeBolhaF[r] != 0.0f;
  d.q[c] = (float)((double)d.qAr[c] + (bolha ? (double)d.yBolhaF[r] : 0.0));
}
__global__ void k_pos_pressao_bolhas(Dev d, double dt) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < 2 || r >= MAX_BOLHAS) return;
  if (d.volumeBolhaF[r] == 0.0f) return;
  double paraPa = (DENSIDADE_AGUA * d.h) / dt;
  d.pressaoBolha[r] = (float)fmax(-PRESSAO_BOLHA_MAX, fmin(PRESSAO_BOLHA_MAX, (double)d.yBolhaF[r] * paraPa));
}

// #gradiente (js/fisica-cpu.js:519-545)
__global__ void k_gradiente(Dev d) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = d.nx, ny = d.ny;
  const uint8_t* tipo = d.tipo;
  const float* q = d.q;
  if (k < d.nu) {
    int i = k % (nx + 1), j = k / (nx + 1);
    uint8_t tl = i > 0 ? tipo[i - 1 + j * nx] : SOLIDO;
    uint8_t tr = i < nx ? tipo[i + j * nx] : SOLIDO;
    if (tl == SOLIDO || tr == SOLIDO) { d.u[k] = 0.0f; d.uVal[k] = 1; }
    else if (tl == AGUA || tr == AGUA) {
      d.u[k] = (float)((double)d.u[k] - ((double)q[i + j * nx] - (double)q[i - 1 + j * nx]));
      d.uVal[k] = 1;
    } else d.uVal[k] = 0;
  }
  if (k < d.nv) {
    int i = k % nx, j = k / nx;
    uint8_t tb = j > 0 ? tipo[i + (j - 1) * nx] : SOLIDO;
    uint8_t tt = j < ny ? tipo[i + j * nx] : SOLIDO;
    if (tb == SOLIDO || tt == SOLIDO) { d.v[k] = 0.0f; d.vVal[k] = 1; }
    else if (tb == AGUA || tt == AGUA) {
      d.v[k] = (float)((double)d.v[k] - ((double)q[i + j * nx] - (double)q[i + (j - 1) * nx]));
      d.vVal[k] = 1;
    } else d.vVal[k] = 0;
  }
}

// extrapolarComponente (js/fisica-cpu.js:673-690), one layer for u and v: an invalid face takes
// the mean of its valid 4-neighbours; reads (a, valid), writes (aOut, validOut).
__device__ inline void extrapolar1(const float* a, const uint8_t* val, float* ao, uint8_t* vo, int k, int w, int hh) {
  int i = k % w, j = k / w;
  if (val[k]) { ao[k] = a[k]; vo[k] = 1; return; }
  double soma = 0;
  int n = 0;
  if (i > 0 && val[k - 1]) { soma += (double)a[k - 1]; n++; }
  if (i < w - 1 && val[k + 1]) { soma += (double)a[k + 1]; n++; }
  if (j > 0 && val[k - w]) { soma += (double)a[k - w]; n++; }
  if (j < hh - 1 && val[k + w]) { soma += (double)a[k + w]; n++; }
  if (n > 0) { ao[k] = (float)(soma / n); vo[k] = 1; }
  else { ao[k] = a[k]; vo[k] = 0; }
}
__global__ void k_extrapolar(Dev d, int volta) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < d.nu) {
    if (!volta) extrapolar1(d.u, d.uVal, d.uTmp, d.uValTmp, k, d.nx + 1, d.ny);
    else extrapolar1(d.uTmp, d.uValTmp, d.u, d.uVal, k, d.nx + 1, d.ny);
  }
  if (k < d.nv) {
    if (!volta) extrapolar1(d.v, d.vVal, d.vTmp, d.vValTmp, k, d.nx, d.ny + 1);
    else extrapolar1(d.vTmp, d.vValTmp, d.v, d.vVal, k, d.nx, d.ny + 1);
  }
}

// ---------------------------------------------------------------- host launchers
void lancarSolidos(const Dev& d, cudaStream_t s) { lanca(k_solidos, blocos(d.N, 256), 256, 0, s, d); }
void lancarTracar(const Dev& d, double x0m, double y0m, double x1m, double y1m, double raio, bool apagar,
                  cudaStream_t s) {
  // the box and the segment in mask points, on the host in the same double arithmetic
  const double r = RES_MASCARA, esc = r / d.h;
  const double ax = x0m * esc - 0.5, ay = y0m * esc - 0.5, bx = x1m * esc - 0.5, by = y1m * esc - 0.5;
  const double rp = raio * esc;
  const double alc = rp + SDF_MAX * r + 1;
  const double xmin = fmax(0.0, floor(fmin(ax, bx) - alc)), xmax = fmin((double)(d.mw - 1), ceil(fmax(ax, bx) + alc));
  const double ymin = fmax(0.0, floor(fmin(ay, by) - alc)), ymax = fmin((double)(d.mh - 1), ceil(fmax(ay, by) + alc));
  if (!(xmin <= xmax) || !(ymin <= ymax)) return;
  const int nbx = (int)(xmax - xmin) + 1, nby = (int)(ymax - ymin) + 1;
  const double dx = bx - ax, dy = by - ay;
  lanca(k_tracar, blocos(nbx * nby, 256), 256, 0, s, (float*)d.sdf, d.mw, d.mh, (int)xmin, (int)ymin, nbx, nby, ax, ay, dx, dy,
        dx * dx + dy * dy, rp, apagar ? 1 : 0);
}
void lancarZerarMascara(const Dev& d, cudaStream_t s) {
  lanca(k_zerar_mascara, blocos(d.mw * d.mh, 256), 256, 0, s, (float*)d.sdf, d.mw, d.mh);
}
void lancarTipos(const Dev& d, bool ar, cudaStream_t s) {
  lanca(k_tipos, blocos(d.N, 256), 256, 0, s, d, ar ? 1 : 0, 1);
}
void lancarPropagarRotulos(const Dev& d, cudaStream_t s) {
  for (int passada = 0; passada < 2; passada++) {
    lanca(k_rotulos_pendentes, blocos(d.N, 256), 256, 0, s, d, passada);
    lanca(k_rotulos_resolver, 1, 1024, 0, s, d);
  }
}
void lancarSuperficie(const Dev& d, cudaStream_t s) {
  int nb = blocos(d.N, 256);
  for (int passada = 0; passada <= 2; passada++) {
    for (int camada = 1; camada <= 3; camada++) {
      lanca(k_estender, nb, 256, 0, s, d, camada);
      lanca(k_estender_gravar, nb, 256, 0, s, d, camada);
    }
    if (passada == 2) break;
    lanca(k_borrar_x, nb, 256, 0, s, d);
    lanca(k_borrar_y, nb, 256, 0, s, d);
  }
  lanca(k_normais, nb, 256, 0, s, d);
  lanca(k_curvatura, nb, 256, 0, s, d);
}
void lancarPressaoDoAr(const Dev& d, double dt, double tensao, cudaStream_t s) {
  lanca(k_pressao_ar, blocos(d.N, 256), 256, 0, s, d, dt, tensao);
}
void lancarClassificar(const Dev& d, double dt, double tau, cudaStream_t s) {
  lanca(k_classificar, blocos(d.N, 256), 256, 0, s, d, dt, tau);
}
void lancarLadoDireitoBolhas(const Dev& d, double dt, cudaStream_t s) {
  cudaMemsetAsync(d.volB, 0, MAX_BOLHAS * sizeof(uint32_t), s);
  cudaMemsetAsync(d.accB, 0, MAX_BOLHAS * sizeof(long long), s);
  lanca(k_bolhas_somar, blocos(d.N, 256), 256, 0, s, d);
  lanca(k_bolhas_fechar, blocos(MAX_BOLHAS, 256), 256, 0, s, d, dt);
}
void lancarPosPressao(const Dev& d, double dt, bool ar, cudaStream_t s) {
  lanca(k_pos_pressao, blocos(d.N, 256), 256, 0, s, d, ar ? 1 : 0);
  if (ar) lanca(k_pos_pressao_bolhas, blocos(MAX_BOLHAS, 256), 256, 0, s, d, dt);
}
void lancarGradiente(const Dev& d, cudaStream_t s) {
  int m = d.nu > d.nv ? d.nu : d.nv;
  lanca(k_gradiente, blocos(m, 256), 256, 0, s, d);
}
void lancarExtrapolar(const Dev& d, cudaStream_t s) {
  int m = d.nu > d.nv ? d.nu : d.nv;
  lanca(k_extrapolar, blocos(m, 256), 256, 0, s, d, 0);
  lanca(k_extrapolar, blocos(m, 256), 256, 0, s, d, 1);
}

}  // namespace tq
