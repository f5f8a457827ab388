// particulas.cu — particle kernels of the substep: particle-to-grid transfer (fixed point),
// face normalisation + gravity + wall faces, grid-to-particle transfer with APIC, micro-step
// advection and wall collision, and the particle bookkeeping (insert, tools, compaction).
//
// Built with -fmad=false: the f32 operations of the fixed-point transfer must be exactly the
// sequence the oracle restates (no contraction into fused multiply-adds), and the double
// arithmetic of the grid-to-particle transfer then follows the reference's JavaScript
// (double locals, f32 stores) operation for operation.
#include "common.cuh"
#include "kernels.cuh"

namespace tq {

// ---------------------------------------------------------------- P2G
// Integer particle-to-grid sums of js/gpu/fisica.js:77-131 (APIC velocity with affine term,
// weights, bilinear density at cell centres, particle count, dye x256).  The CPU engine's
// float sums (js/fisica-cpu.js:198-267) depend on particle order; integer sums do not, so
// any thread schedule and any grouping of the additions produce the same bits.
__device__ __forceinline__ int chao(float v, int lo, int hi) {
  float f = floorf(v);
  f = fminf(fmaxf(f, (float)lo), (float)hi);
  return (int)f;
}

// The cell of a particle (the count's and the dye's cell): every sum of the particle lands in
// columns ci-1..ci+1 and rows cj-1..cj+1 (u faces at column i, v faces at row j, cell centres).
__device__ __forceinline__ void celulaDe(float x, float y, float inv, int nx, int ny, int& ci, int& cj) {
  ci = chao(x * inv, 0, nx - 1);
  cj = chao(y * inv, 0, ny - 1);
}

// Every integer contribution of one particle, handed to `soma(tipo, i, j, componente, valor)`:
// tipo 0 a u face (componente 0 the weighted velocity, 1 the weight), 1 a v face, 2 a cell
// centre (0 the density weight, 1 the count), 3 the cell's dye (componente 0-2).
template <class F>
__device__ __forceinline__ void contribuicoes(const float4& a, const float4& c, const float4& e, int nx, int ny,
                                              float hf, float inv, int ci, int cj, F soma) {
  const float x = a.x, y = a.y;
  {
    float fx = x * inv, fy = y * inv - 0.5f;
    int i0 = chao(fx, 0, nx - 1), j0 = chao(fy, 0, ny - 2);
    float tx = fx - (float)i0, ty = fy - (float)j0;
#pragma unroll
    for (int b = 0; b < 2; b++)
#pragma unroll
      for (int aa = 0; aa < 2; aa++) {
        float wx = aa ? tx : 1.0f - tx, wy = b ? ty : 1.0f - ty;
        float w = wx * wy;
        float dx = (float)(i0 + aa) * hf - x;
        float dy = ((float)(j0 + b) + 0.5f) * hf - y;
        float t1 = c.x * dx, t2 = c.y * dy;
        float val = a.z + (t1 + t2);
        float wv = w * val;
        soma(0, i0 + aa, j0 + b, 0, __float2int_rn(wv * 65536.0f));
        soma(0, i0 + aa, j0 + b, 1, __float2int_rn(w * 65536.0f));
      }
  }
  {
    float fx = x * inv - 0.5f, fy = y * inv;
    int i0 = chao(fx, 0, nx - 2), j0 = chao(fy, 0, ny - 1);
    float tx = fx - (float)i0, ty = fy - (float)j0;
#pragma unroll
    for (int b = 0; b < 2; b++)
#pragma unroll
      for (int aa = 0; aa < 2; aa++) {
        float wx = aa ? tx : 1.0f - tx, wy = b ? ty : 1.0f - ty;
        float w = wx * wy;
        float dx = ((float)(i0 + aa) + 0.5f) * hf - x;
        float dy = (float)(j0 + b) * hf - y;
        float t1 = c.z * dx, t2 = c.w * dy;
        float val = a.w + (t1 + t2);
        float wv = w * val;
        soma(1, i0 + aa, j0 + b, 0, __float2int_rn(wv * 65536.0f));
        soma(1, i0 + aa, j0 + b, 1, __float2int_rn(w * 65536.0f));
      }
  }
  {
    float fx = x * inv - 0.5f, fy = y * inv - 0.5f;
    int i0 = chao(fx, 0, nx - 2), j0 = chao(fy, 0, ny - 2);
    float tx = fx - (float)i0, ty = fy - (float)j0;
    float ox = 1.0f - tx, oy = 1.0f - ty;
    soma(2, i0, j0, 0, __float2int_rn((ox * oy) * 65536.0f));
    soma(2, i0 + 1, j0, 0, __float2int_rn((tx * oy) * 65536.0f));
    soma(2, i0, j0 + 1, 0, __float2int_rn((ox * ty) * 65536.0f));
    soma(2, i0 + 1, j0 + 1, 0, __float2int_rn((tx * ty) * 65536.0f));
  }
  soma(2, ci, cj, 1, 1);
  if (e.y != 0.0f || e.z != 0.0f || e.w != 0.0f) {
    soma(3, ci, cj, 0, __float2int_rn(e.y * 256.0f));
    soma(3, ci, cj, 1, __float2int_rn(e.z * 256.0f));
    soma(3, ci, cj, 2, __float2int_rn(e.w * 256.0f));
  }
}

// One CTA of P2G_T consecutive particles.  The reference's particle order (kept: it is what
// the host reads back) stays spatially coherent: particles are seeded cell by cell, move at
// most a cell or so per substep, and compaction is stable.  So the CTA first takes the
// bounding box of its particles' cells; when the box with its one-cell halo fits in
// P2G_CAIXA entries, the contributions go to shared-memory sums of the box and each nonzero
// sum then reaches the grid with one global atomic (the particles of a cell share their faces
// and centres: about a third of the global atomics of one per contribution).  A CTA whose box
// is larger (particles scattered) adds every contribution to the grid directly.
constexpr int P2G_T = 256;
constexpr int P2G_CAIXA = 1024;

__global__ void __launch_bounds__(P2G_T) k_p2g(Dev d) {
  __shared__ int2 sU[P2G_CAIXA], sV[P2G_CAIXA], sC[P2G_CAIXA];
  __shared__ int sD[3 * P2G_CAIXA];
  __shared__ int caixa[4];  // min ci, min cj, max ci, max cj of the CTA's live particles
  const int k = blockIdx.x * P2G_T + threadIdx.x;
  const int nx = d.nx, ny = d.ny;
  const float hf = d.hf;
  const float inv = __fdiv_rn(1.0f, hf);
  float4 a = make_float4(0.f, 0.f, 0.f, 0.f), c = a, e = a;
  bool vivo = k < d.esc->n;
  if (vivo) {
    a = d.p0[k];
    vivo = a.x == a.x;  // NaN: marked dead earlier in this frame
  }
  int ci = 0, cj = 0;
  if (vivo) {
    c = d.p1[k];
    e = d.p2[k];
    celulaDe(a.x, a.y, inv, nx, ny, ci, cj);
  }
  if (threadIdx.x == 0) {
    caixa[0] = caixa[1] = 0x7fffffff;
    caixa[2] = caixa[3] = -1;
  }
  __syncthreads();
  {
    const int mi = __reduce_min_sync(0xffffffffu, vivo ? ci : 0x7fffffff);
    const int mj = __reduce_min_sync(0xffffffffu, vivo ? cj : 0x7fffffff);
    const int Mi = __reduce_max_sync(0xffffffffu, vivo ? ci : -1);
    const int Mj = __reduce_max_sync(0xffffffffu, vivo ? cj : -1);
    if ((threadIdx.x & 31) == 0 && Mi >= 0) {
      atomicMin(&caixa[0], mi);
      atomicMin(&caixa[1], mj);
      atomicMax(&caixa[2], Mi);
      atomicMax(&caixa[3], Mj);
    }
  }
  __syncthreads();
  if (caixa[2] < 0) return;  // no live particle in this CTA (uniform)
  const int I0 = caixa[0] - 1, J0 = caixa[1] - 1;
  const int W = caixa[2] - caixa[0] + 3, H = caixa[3] - caixa[1] + 3;
  if (W * H > P2G_CAIXA) {  // scattered particles: one global atomic per contribution (uniform)
    if (vivo)
      contribuicoes(a, c, e, nx, ny, hf, inv, ci, cj, [&](int t, int i, int j, int comp, int v) {
        if (t == 0) atomicAdd(comp ? &d.accU[i + j * (nx + 1)].y : &d.accU[i + j * (nx + 1)].x, v);
        else if (t == 1) atomicAdd(comp ? &d.accV[i + j * nx].y : &d.accV[i + j * nx].x, v);
        else if (t == 2) atomicAdd(comp ? &d.accCel[i + j * nx].y : &d.accCel[i + j * nx].x, v);
        else atomicAdd(&d.accCor[3 * (i + j * nx) + comp], v);
      });
    return;
  }
  const int nb = W * H;
  for (int t = threadIdx.x; t < nb; t += P2G_T) {
    sU[t] = sV[t] = sC[t] = make_int2(0, 0);
    sD[3 * t] = sD[3 * t + 1] = sD[3 * t + 2] = 0;
  }
  __syncthreads();
  if (vivo)
    contribuicoes(a, c, e, nx, ny, hf, inv, ci, cj, [&](int t, int i, int j, int comp, int v) {
      const int b = (i - I0) + (j - J0) * W;
      if (t == 0) atomicAdd(comp ? &sU[b].y : &sU[b].x, v);
      else if (t == 1) atomicAdd(comp ? &sV[b].y : &sV[b].x, v);
      else if (t == 2) atomicAdd(comp ? &sC[b].y : &sC[b].x, v);
      else atomicAdd(&sD[3 * b + comp], v);
    });
  __syncthreads();
  // a box entry that no particle touched holds 0 in every sum (and may lie outside the
  // grid): only nonzero sums are added, each at an index inside its array
  for (int t = threadIdx.x; t < nb; t += P2G_T) {
    const int i = I0 + t % W, j = J0 + t / W;
    const int2 u = sU[t], v = sV[t], cc = sC[t];
    if (u.x) atomicAdd(&d.accU[i + j * (nx + 1)].x, u.x);
    if (u.y) atomicAdd(&d.accU[i + j * (nx + 1)].y, u.y);
    if (v.x) atomicAdd(&d.accV[i + j * nx].x, v.x);
    if (v.y) atomicAdd(&d.accV[i + j * nx].y, v.y);
    if (cc.x) atomicAdd(&d.accCel[i + j * nx].x, cc.x);
    if (cc.y) atomicAdd(&d.accCel[i + j * nx].y, cc.y);
#pragma unroll
    for (int q = 0; q < 3; q++)
      if (sD[3 * t + q]) atomicAdd(&d.accCor[3 * (i + j * nx) + q], sD[3 * t + q]);
  }
}

// Face velocity from the sums, gravity impulse where a particle contributed, zero on wall
// faces: js/fisica-cpu.js:265-266 + :271-291 in the integer form of js/gpu/fisica.js:135-160.
__global__ void k_faces(Dev d, float gdx, float gdy) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = d.nx, ny = d.ny;
  if (k < d.nu) {
    int i = k % (nx + 1), j = k / (nx + 1);
    int2 a = d.accU[k];
    float val = 0.0f;
    if (a.y > 0) val = __fadd_rn(__fdiv_rn((float)a.x, (float)a.y), gdx);
    bool s = i == 0 || i == nx || d.solido[i - 1 + j * nx] || d.solido[i + j * nx];
    d.u[k] = s ? 0.0f : val;
  }
  if (k < d.nv) {
    int i = k % nx, j = k / nx;
    int2 a = d.accV[k];
    float val = 0.0f;
    if (a.y > 0) val = __fadd_rn(__fdiv_rn((float)a.x, (float)a.y), gdy);
    bool s = j == 0 || j == ny || d.solido[i + (j - 1) * nx] || d.solido[i + j * nx];
    d.v[k] = s ? 0.0f : val;
  }
}

// ---------------------------------------------------------------- G2P
// #velocidadeEm, js/fisica-cpu.js:641-661
__device__ inline void velocidadeEm(const Dev& d, double x, double y, double vmax, double* ox, double* oy) {
  const int nx = d.nx, ny = d.ny;
  double inv = 1 / d.h;
  double vx, vy;
  {
    double fx = x * inv, fy = y * inv - 0.5;
    int i0 = clampi(floori(fx), 0, nx - 1), j0 = clampi(floori(fy), 0, ny - 2);
    double tx = fx - i0, ty = fy - j0;
    int k = i0 + j0 * (nx + 1);
    vx = ((double)d.u[k] * (1 - tx) + (double)d.u[k + 1] * tx) * (1 - ty) +
         ((double)d.u[k + nx + 1] * (1 - tx) + (double)d.u[k + nx + 2] * tx) * ty;
  }
  {
    double fx = x * inv - 0.5, fy = y * inv;
    int i0 = clampi(floori(fx), 0, nx - 2), j0 = clampi(floori(fy), 0, ny - 1);
    double tx = fx - i0, ty = fy - j0;
    int k = i0 + j0 * nx;
    vy = ((double)d.v[k] * (1 - tx) + (double)d.v[k + 1] * tx) * (1 - ty) +
         ((double)d.v[k + nx] * (1 - tx) + (double)d.v[k + nx + 1] * tx) * ty;
  }
  double vv = hypot(vx, vy);
  if (vv > vmax) { *ox = vx * vmax / vv; *oy = vy * vmax / vv; }
  else { *ox = vx; *oy = vy; }
}

// #paraParticulas, js/fisica-cpu.js:556-638: APIC gather of v and C, foam and dye, speed
// clamp, micro-steps through the projected grid velocity with SDF push-out, kill when deep
// in a wall.  Dead particles get x = NaN and are removed by the compaction at the end of the
// call (the reference removes them at the end of the same loop, :636).
// The largest speed of the warp's live particles into *alvo (double bits; speeds are >= 0, so
// their bits order as unsigned integers): the high words' maximum, then the low words' among the
// lanes holding it, each by one __reduce_max_sync, and one atomicMax per warp instead of one per
// particle on a single address.
__device__ __forceinline__ void maxVelocidadeWarp(unsigned ativos, double vel, unsigned long long* alvo) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(vel);
  const unsigned hi = (unsigned)(b >> 32), lo = (unsigned)b;
  const unsigned mhi = __reduce_max_sync(ativos, hi);
  const unsigned comMax = __ballot_sync(ativos, hi == mhi);
  if (hi == mhi) {
    const unsigned mlo = __reduce_max_sync(comMax, lo);
    if ((int)(threadIdx.x & 31) == __ffs(comMax) - 1) {
      const unsigned long long m = ((unsigned long long)mhi << 32) | mlo;
      if (m) atomicMax(alvo, m);
    }
  }
}

__global__ void k_g2p(Dev d, double dt) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const bool dentro = k < d.esc->n;
  const float4 a = dentro ? d.p0[k] : make_float4(0.f, 0.f, 0.f, 0.f);
  const bool vivo = dentro && a.x == a.x;  // a particle marked dead earlier is skipped
  const unsigned ativos = __ballot_sync(0xffffffffu, vivo);  // every lane of the warp takes part
  if (!vivo) return;
  const float4 e = d.p2[k];
  const int nx = d.nx, ny = d.ny;
  const double h = d.h;
  double x = a.x, y = a.y;
  const double inv = 1 / h;
  const double vmax = (MICROPASSO * MAX_MICROPASSOS * h) / dt;
  const double decai = exp(-dt / ESPUMA_VIDA);
  const double mistura = fmin(1.0, dt / DIFUSAO_CORANTE);
  double vx = 0, vy = 0, cux = 0, cuy = 0, cvx = 0, cvy = 0;
  {
    double fx = x * inv, fy = y * inv - 0.5;
    int i0 = clampi(floori(fx), 0, nx - 1), j0 = clampi(floori(fy), 0, ny - 2);
    double tx = fx - i0, ty = fy - j0;
    for (int b = 0; b < 2; b++)
      for (int aa = 0; aa < 2; aa++) {
        double val = d.u[i0 + aa + (j0 + b) * (nx + 1)];
        double wx = aa ? tx : 1 - tx, wy = b ? ty : 1 - ty;
        vx += wx * wy * val;
        cux += (aa ? 1 : -1) * wy * inv * val;
        cuy += wx * (b ? 1 : -1) * inv * val;
      }
  }
  {
    double fx = x * inv - 0.5, fy = y * inv;
    int i0 = clampi(floori(fx), 0, nx - 2), j0 = clampi(floori(fy), 0, ny - 1);
    double tx = fx - i0, ty = fy - j0;
    for (int b = 0; b < 2; b++)
      for (int aa = 0; aa < 2; aa++) {
        double val = d.v[i0 + aa + (j0 + b) * nx];
        double wx = aa ? tx : 1 - tx, wy = b ? ty : 1 - ty;
        vy += wx * wy * val;
        cvx += (aa ? 1 : -1) * wy * inv * val;
        cvy += wx * (b ? 1 : -1) * inv * val;
      }
  }
  double vel = hypot(vx, vy);
  int ci = clampi(floori(x * inv), 0, nx - 1), cj = clampi(floori(y * inv), 0, ny - 1);
  int cc = ci + cj * nx;
  int2 cel = d.accCel[cc];
  double dens = (float)cel.x * (1.0f / 65536.0f);
  double rarefeita = suave(0.95, 0.45, dens / PARTICULAS_POR_CELULA);
  double fonte = suave(ESPUMA_V0, ESPUMA_V1, vel) * rarefeita;
  double espuma = fmin(1.0, (double)e.x * decai + fonte * ESPUMA_TAXA * dt);
  float abs0 = e.y, abs1 = e.z, abs2 = e.w;
  if (cel.y > 1) {
    double n = cel.y;
    double c0 = (float)d.accCor[3 * cc] * (1.0f / 256.0f);
    double c1 = (float)d.accCor[3 * cc + 1] * (1.0f / 256.0f);
    double c2 = (float)d.accCor[3 * cc + 2] * (1.0f / 256.0f);
    abs0 = (float)((double)abs0 + (c0 / n - (double)abs0) * mistura);
    abs1 = (float)((double)abs1 + (c1 / n - (double)abs1) * mistura);
    abs2 = (float)((double)abs2 + (c2 / n - (double)abs2) * mistura);
  }
  if (vel > vmax) { vx *= vmax / vel; vy *= vmax / vel; }
  maxVelocidadeWarp(ativos, vel > 0 ? vel : 0.0, &d.esc->vmaxBits);  // (NaN and 0 leave the maximum alone)
  double micro = fmin(MAX_MICROPASSOS, fmax(1.0, ceil((fmin(vel, vmax) * dt) / (MICROPASSO * h))));
  double dm = dt / micro;
  int nm = (int)micro;
  for (int m = 0; m < nm; m++) {
    double wx = vx, wy = vy;
    if (nm > 1) velocidadeEm(d, x, y, vmax, &wx, &wy);
    x += wx * dm;
    y += wy * dm;
    double dist = distancia(d, x, y);
    if (dist < RAIO_PARTICULA) {
      if (dist < -SDF_MAX + 0.5) {
        d.p0[k].x = __int_as_float(0x7fc00000);
        atomicAdd(&d.esc->mortas, 1);
        return;
      }
      double nX, nY;
      normalSdf(d, x, y, &nX, &nY);
      double empurra = (RAIO_PARTICULA - dist) * h;
      x += nX * empurra;
      y += nY * empurra;
      double vn = vx * nX + vy * nY;
      if (vn < 0) { vx -= vn * nX; vy -= vn * nY; }
    }
  }
  d.p0[k] = make_float4((float)x, (float)y, (float)vx, (float)vy);
  d.p1[k] = make_float4((float)cux, (float)cuy, (float)cvx, (float)cvy);
  d.p2[k] = make_float4((float)espuma, abs0, abs1, abs2);
}

// ---------------------------------------------------------------- block scan helper
// Exclusive rank of `keep` among the threads of a 1024-thread block; *total = block count.
__device__ int rankNoBloco(bool keep, int* total) {
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
#pragma unroll
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

// Exclusive scan of `n` block counts by one 1024-thread block; returns the total.
__device__ int scanUmBloco(const int* cont, int* offs, int n) {
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += 1024) {
    int i = base + threadIdx.x;
    int v = i < n ? cont[i] : 0;
    // inclusive scan of v across the block
    __shared__ int s[1024];
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

// ---------------------------------------------------------------- compaction
// Stable removal of particles whose x is NaN (dead in G2P, or removed by the sponge tool):
// the reference's `remover` keeps the survivors' order (js/fisica-cpu.js:114-126).  All four
// kernels return at once when nothing died.
__global__ void k_compactar_contar(Dev d, int* cont) {
  if (d.esc->mortas == 0) return;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  int n = d.esc->n;
  bool viva = k < n && d.p0[k].x == d.p0[k].x;
  int total;
  rankNoBloco(viva, &total);
  if (threadIdx.x == 0) cont[blockIdx.x] = total;
}

__global__ void k_compactar_scan(Dev d, const int* cont, int* offs, int nb, int* estado) {
  if (d.esc->mortas == 0) {
    if (threadIdx.x == 0) estado[0] = 0;
    return;
  }
  int total = scanUmBloco(cont, offs, nb);
  if (threadIdx.x == 0) {
    estado[0] = 1;
    estado[1] = d.esc->n;  // count before
    d.esc->n = total;
    d.esc->mortas = 0;
  }
}

__global__ void k_compactar_mover(Dev d, const int* offs, const int* estado) {
  if (!estado[0]) return;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  int n = estado[1];
  bool viva = k < n && d.p0[k].x == d.p0[k].x;
  int total;
  int r = rankNoBloco(viva, &total);
  if (viva) {
    int o = offs[blockIdx.x] + r;
    d.q0[o] = d.p0[k];
    d.q1[o] = d.p1[k];
    d.q2[o] = d.p2[k];
    d.qid[o] = d.pid[k];
  }
}

__global__ void k_compactar_copiar(Dev d, const int* estado) {
  if (!estado[0]) return;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.esc->n) return;
  d.p0[k] = d.q0[k];
  d.p1[k] = d.q1[k];
  d.p2[k] = d.q2[k];
  d.pid[k] = d.qid[k];
}

// ---------------------------------------------------------------- insert
// SimulacaoCPU.adicionar (js/fisica-cpu.js:92-111): keep a new particle when the SDF at it is
// > RAIO_PARTICULA + 0.05 and, with checarCheia, its cell held < PARTICULAS_POR_CELULA - 1
// particles at the last transfer.  Survivors are appended in list order.
__global__ void k_adicionar_contar(Dev d, const float* lista, int total, int checar, int* cont) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  bool ok = false;
  if (k < total) {
    const float* o = lista + (size_t)k * CAMPOS;
    double x = o[0], y = o[1];
    ok = distancia(d, x, y) > RAIO_PARTICULA + 0.05;
    if (ok && checar) {
      double fi = floor(x / d.h), fj = floor(y / d.h);
      if (fi < 0 || fj < 0 || fi >= d.nx || fj >= d.ny) ok = false;
      else {
        int c = (int)fi + (int)fj * d.nx;
        if (d.accCel[c].y >= PARTICULAS_POR_CELULA - 1) ok = false;
      }
    }
  }
  int t;
  rankNoBloco(ok, &t);
  if (threadIdx.x == 0) cont[blockIdx.x] = t;
}

__global__ void k_adicionar_scan(Dev d, const int* cont, int* offs, int nb) {
  int total = scanUmBloco(cont, offs, nb);
  if (threadIdx.x == 0) d.esc->aceitas = total;
}

__global__ void k_adicionar_mover(Dev d, const float* lista, int total, int checar, const int* offs,
                                  unsigned long long idBase) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  bool ok = false;
  const float* o = lista + (size_t)min(k, max(total - 1, 0)) * CAMPOS;
  if (k < total) {
    double x = o[0], y = o[1];
    ok = distancia(d, x, y) > RAIO_PARTICULA + 0.05;
    if (ok && checar) {
      double fi = floor(x / d.h), fj = floor(y / d.h);
      if (fi < 0 || fj < 0 || fi >= d.nx || fj >= d.ny) ok = false;
      else {
        int c = (int)fi + (int)fj * d.nx;
        if (d.accCel[c].y >= PARTICULAS_POR_CELULA - 1) ok = false;
      }
    }
  }
  int t;
  int r = rankNoBloco(ok, &t);
  if (ok) {
    int pos = offs[blockIdx.x] + r;
    int dst = d.esc->n + pos;  // esc->n grows only in k_adicionar_fim, after this kernel
    d.p0[dst] = make_float4(o[0], o[1], o[2], o[3]);
    d.p1[dst] = make_float4(o[4], o[5], o[6], o[7]);
    d.p2[dst] = make_float4(o[8], o[9], o[10], o[11]);
    d.pid[dst] = idBase + (unsigned long long)pos;
  }
}

__global__ void k_adicionar_fim(Dev d) { d.esc->n += d.esc->aceitas; }

// ---------------------------------------------------------------- state copies
__global__ void k_empacotar(Dev d, float* out, int n) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  float4 a = d.p0[k], b = d.p1[k], c = d.p2[k];
  float* o = out + (size_t)k * CAMPOS;
  o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
  o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
  o[8] = c.x; o[9] = c.y; o[10] = c.z; o[11] = c.w;
}

__global__ void k_desempacotar(Dev d, const float* in, int n, unsigned long long idBase) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float* o = in + (size_t)k * CAMPOS;
  d.p0[k] = make_float4(o[0], o[1], o[2], o[3]);
  d.p1[k] = make_float4(o[4], o[5], o[6], o[7]);
  d.p2[k] = make_float4(o[8], o[9], o[10], o[11]);
  d.pid[k] = idBase + (unsigned long long)k;
}

// ---------------------------------------------------------------- tools
// SimulacaoCPU.aplicarFerramenta (js/fisica-cpu.js:129-152).  The sponge marks particles dead
// (removed by the compaction, order kept); the hand pulls velocities; the dye paints.
__global__ void k_ferramenta(Dev d, tq_tool f) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.esc->n) return;
  float4 a = d.p0[k];
  if (!(a.x == a.x)) return;
  double r2 = f.radius * f.radius;
  double dx = (double)a.x - f.x, dy = (double)a.y - f.y;
  double d2 = dx * dx + dy * dy;
  if (f.kind == 1) {
    if (d2 < r2) {
      d.p0[k].x = __int_as_float(0x7fc00000);
      atomicAdd(&d.esc->mortas, 1);
    }
    return;
  }
  if (d2 >= r2) return;
  double peso = 1 - sqrt(d2 / r2);
  if (f.kind == 2) {
    double al = fmin(1.0, peso * 0.9);
    a.z = (float)((double)a.z + (f.vx - (double)a.z) * al);
    a.w = (float)((double)a.w + (f.vy - (double)a.w) * al);
    d.p0[k] = a;
  } else if (f.kind == 3) {
    float4 e = d.p2[k];
    e.y = (float)f.absorb[0];
    e.z = (float)f.absorb[1];
    e.w = (float)f.absorb[2];
    d.p2[k] = e;
  }
}

// ---------------------------------------------------------------- faucet
// emitirTorneira (js/principal.js:301-321) on the device, with the LCG of testes/apoio.js:4-9 in
// place of Math.random: particle k takes the generator's draws 2k+1 and 2k+2 from the seed, reached
// by jumping the LCG ahead (s -> A s + C composed with itself by squaring), so every thread makes
// its particle independently and the list equals the one a host loop makes.  In a disk of the
// jet's radius around (cx, cy): angle a = u1 * pi * 2, radius sqrt(u2) * raio, in the reference's
// double arithmetic, stored as float; velocity and dye as given, foam and affine terms 0.
__device__ __forceinline__ uint32_t lcgSalto(uint32_t s, uint32_t k) {
  uint32_t A = 1664525u, C = 1013904223u, a = 1u, c = 0u;
  while (k) {
    if (k & 1u) {
      a *= A;
      c = c * A + C;
    }
    C = (A + 1u) * C;
    A *= A;
    k >>= 1;
  }
  return a * s + c;
}
__global__ void k_torneira(float* lista, int n, uint32_t semente, double cx, double cy, double raio, float vx, float vy,
                           float a0, float a1, float a2) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint32_t s1 = lcgSalto(semente, 2u * (uint32_t)k + 1u);
  const uint32_t s2 = s1 * 1664525u + 1013904223u;
  const double u1 = s1 / 4294967296.0, u2 = s2 / 4294967296.0;
  const double a = u1 * 3.141592653589793 * 2, r = sqrt(u2) * raio;
  float* o = lista + (size_t)k * CAMPOS;
  o[0] = (float)(cx + cos(a) * r);
  o[1] = (float)(cy + sin(a) * r);
  o[2] = vx;
  o[3] = vy;
  o[4] = o[5] = o[6] = o[7] = o[8] = 0.0f;
  o[9] = a0;
  o[10] = a1;
  o[11] = a2;
}

// ---------------------------------------------------------------- host launchers
void lancarTorneira(float* lista, int n, uint32_t semente, double cx, double cy, double raio, float vx, float vy,
                    const float absorb[3], cudaStream_t s) {
  if (n > 0) lanca(k_torneira, blocos(n, 256), 256, 0, s, lista, n, semente, cx, cy, raio, vx, vy, absorb[0], absorb[1],
                   absorb[2]);
}
// ---------------------------------------------------------------- headless splat
// WGSL_MANCHA (js/gpu/render.js:11-43) without a graphics pipeline: every live particle adds,
// at each pixel centre of a w x h target covering the tank (row 0 at the top, as the render
// target), the weight (1 - r^2)^2 with r the distance over raio = RAIO_MANCHA h, and that
// weight times its foam and its three absorptions.  The f32 operations are the restatement's
// (no fused multiply-add in this file); the sums are 64-bit fixed point (2^32), so they do
// not depend on the order of the atomics.
__device__ __forceinline__ long long fixoMancha(float v) { return __double2ll_rn((double)v * 4294967296.0); }

__global__ void k_mancha(Dev d, int n, int w, int hp, float W, float H, float raio, unsigned long long* acc) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float4 a = d.p0[k], e = d.p2[k];
  const float x = a.x, y = a.y;
  if (!(x == x) || !(y == y) || x < 0.0f) return;
  const float px = W / (float)w, py = H / (float)hp;
  const int i0 = max(0, (int)floorf((x - raio) / px - 0.5f) - 1), i1 = min(w - 1, (int)ceilf((x + raio) / px - 0.5f) + 1);
  const int j0 = max(0, (int)floorf((H - (y + raio)) / py - 0.5f) - 1);
  const int j1 = min(hp - 1, (int)ceilf((H - (y - raio)) / py - 0.5f) + 1);
  const size_t plano = (size_t)w * hp;
  for (int j = j0; j <= j1; j++) {
    const float v = ((H - ((float)j + 0.5f) * py) - y) / raio;
    for (int i = i0; i <= i1; i++) {
      const float u = (((float)i + 0.5f) * px - x) / raio;
      const float r2 = u * u + v * v;
      if (r2 >= 1.0f) continue;
      const float wt = (1.0f - r2) * (1.0f - r2);
      unsigned long long* q = acc + (size_t)j * w + i;
      atomicAdd(q, (unsigned long long)fixoMancha(wt));
      if (e.x != 0.0f) atomicAdd(q + plano, (unsigned long long)fixoMancha(wt * e.x));
      if (e.y != 0.0f) atomicAdd(q + 2 * plano, (unsigned long long)fixoMancha(wt * e.y));
      if (e.z != 0.0f) atomicAdd(q + 3 * plano, (unsigned long long)fixoMancha(wt * e.z));
      if (e.w != 0.0f) atomicAdd(q + 4 * plano, (unsigned long long)fixoMancha(wt * e.w));
    }
  }
}

__global__ void k_mancha_float(const long long* acc, float* out, size_t total) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < total) out[k] = (float)((double)acc[k] * (1.0 / 4294967296.0));
}

void lancarMancha(const Dev& d, int n, int w, int hp, unsigned long long* acc, float* out, cudaStream_t s) {
  const size_t total = (size_t)5 * w * hp;
  cudaMemsetAsync(acc, 0, total * sizeof(unsigned long long), s);
  const float W = (float)(d.nx * d.h), H = (float)(d.ny * d.h), raio = (float)(RAIO_MANCHA * d.h);
  if (n > 0) lanca(k_mancha, blocos(n, 256), 256, 0, s, d, n, w, hp, W, H, raio, acc);
  lanca(k_mancha_float, (unsigned)((total + 255) / 256), 256, 0, s, (const long long*)acc, out, total);
}

void lancarP2G(const Dev& d, int nHint, cudaStream_t s) {
  if (nHint > 0) lanca(k_p2g, blocos(nHint, P2G_T), P2G_T, 0, s, d);
}
void lancarFaces(const Dev& d, float gdx, float gdy, cudaStream_t s) {
  int m = d.nu > d.nv ? d.nu : d.nv;
  lanca(k_faces, blocos(m, 256), 256, 0, s, d, gdx, gdy);
}
void lancarG2P(const Dev& d, int nHint, double dt, cudaStream_t s) {
  if (nHint > 0) lanca(k_g2p, blocos(nHint, 128), 128, 0, s, d, dt);
}
void lancarCompactar(const Dev& d, int nHint, int* cont, int* offs, int* estado, cudaStream_t s) {
  if (nHint <= 0) return;
  int nb = blocos(nHint, 1024);
  lanca(k_compactar_contar, nb, 1024, 0, s, d, cont);
  lanca(k_compactar_scan, 1, 1024, 0, s, d, cont, offs, nb, estado);
  lanca(k_compactar_mover, nb, 1024, 0, s, d, offs, estado);
  lanca(k_compactar_copiar, nb, 1024, 0, s, d, estado);
}
void lancarAdicionar(const Dev& d, const float* lista, int total, int checar, int* cont, int* offs,
                     unsigned long long idBase, cudaStream_t s) {
  int nb = blocos(total, 1024);
  lanca(k_adicionar_contar, nb, 1024, 0, s, d, lista, total, checar, cont);
  lanca(k_adicionar_scan, 1, 1024, 0, s, d, cont, offs, nb);
  lanca(k_adicionar_mover, nb, 1024, 0, s, d, lista, total, checar, offs, idBase);
  lanca(k_adicionar_fim, 1, 1, 0, s, d);
}
void lancarEmpacotar(const Dev& d, float* out, int n, cudaStream_t s) {
  if (n > 0) lanca(k_empacotar, blocos(n, 256), 256, 0, s, d, out, n);
}
void lancarDesempacotar(const Dev& d, const float* in, int n, unsigned long long idBase, cudaStream_t s) {
  if (n > 0) lanca(k_desempacotar, blocos(n, 256), 256, 0, s, d, in, n, idBase);
}
void lancarFerramenta(const Dev& d, int nHint, const tq_tool& f, cudaStream_t s) {
  if (nHint > 0) lanca(k_ferramenta, blocos(nHint, 256), 256, 0, s, d, f);
}

}  // namespace tq
