// kernels.cuh — host launchers of the substep kernels (one translation unit each).
#pragma once
#include "common.cuh"

namespace tq {

// particulas.cu
void lancarP2G(const Dev& d, int nHint, cudaStream_t s);
void lancarFaces(const Dev& d, float gdx, float gdy, cudaStream_t s);
void lancarG2P(const Dev& d, int nHint, double dt, cudaStream_t s);
void lancarCompactar(const Dev& d, int nHint, int* cont, int* offs, int* estado, cudaStream_t s);
void lancarAdicionar(const Dev& d, const float* lista, int total, int checar, int* cont, int* offs,
                     unsigned long long idBase, cudaStream_t s);
void lancarEmpacotar(const Dev& d, float* out, int n, cudaStream_t s);
void lancarDesempacotar(const Dev& d, const float* in, int n, unsigned long long idBase, cudaStream_t s);
void lancarFerramenta(const Dev& d, int nHint, const tq_tool& f, cudaStream_t s);
// emitirTorneira's particle list (12 floats each) into a device buffer
void lancarTorneira(float* lista, int n, uint32_t semente, double cx, double cy, double raio, float vx, float vy,
                    const float absorb[3], cudaStream_t s);

// grade.cu
void lancarSolidos(const Dev& d, cudaStream_t s);
void lancarTracar(const Dev& d, double x0, double y0, double x1, double y1, double raio, bool apagar, cudaStream_t s);
void lancarZerarMascara(const Dev& d, cudaStream_t s);
void lancarMancha(const Dev& d, int n, int w, int hp, unsigned long long* acc, float* out, cudaStream_t s);
void lancarTipos(const Dev& d, bool ar, cudaStream_t s);
void lancarPropagarRotulos(const Dev& d, cudaStream_t s);
void lancarSuperficie(const Dev& d, cudaStream_t s);
void lancarPressaoDoAr(const Dev& d, double dt, double tensao, cudaStream_t s);
void lancarClassificar(const Dev& d, double dt, double tau, cudaStream_t s);
void lancarLadoDireitoBolhas(const Dev& d, double dt, cudaStream_t s);
void lancarPosPressao(const Dev& d, double dt, bool ar, cudaStream_t s);
void lancarGradiente(const Dev& d, cudaStream_t s);
void lancarExtrapolar(const Dev& d, cudaStream_t s);

// regioes.cu — the closed regions of a solve (water sealed from every Dirichlet cell): their
// right-hand side projected onto A's range and one cell of each pinned at 0 (tolerance mode).
struct Regioes;
Regioes* criarRegioes(int N);
void destruirRegioes(Regioes* R);
// Queues the labelling and projection; *out = d with div / rhsBolhaF / tipo at the solve's copies.
void projetarFechadas(Regioes* R, const Dev& d, bool bolhas, cudaStream_t s, Dev* out);
int erroRegioes(Regioes* R, cudaStream_t s);

// pcg.cu — the pressure solve on the handle's grid.
struct Pcg;
// ctasFundido: the fused engine's CTA count (0: one per SM).
Pcg* criarPcg(int nx, int ny, int precisao, int motor, int ctasFundido = 0);
void destruirPcg(Pcg* p);
// Solves for d.q on the cells d.tipo marks as water; bubbles from d.rotulo / d.rhsB / d.yB when
// `bolhas`; precond is TQ_PRECOND_*.  The FUSED engine queues the solve without waiting; the
// PLAIN engine reads its stop flag every few iterations in tolerance mode.  The iteration count,
// residual history and convergence record stay in d.esc.  Returns TQ_OK or an error status.
// In tolerance mode the right-hand side of each closed region first loses its mean (regioes.cu).
int resolverPressao(Pcg* p, const Dev& d, int iteracoes, double tol, bool bolhas, int precond, cudaStream_t s);
// Allocates what a tolerance-mode solve allocates on first use (before a stream capture).
int reservarTolerancia(Pcg* p);
// The last solve's residual history from the device (waits for the stream); its length, or -1.
int normasPcg(Pcg* p, const Dev& d, double* out, int cap, cudaStream_t s);
// TQ_E_TIMEOUT if a fused solve since the last call gave up on a bounded wait (waits for the stream).
int erroPcg(Pcg* p, cudaStream_t s);
// The engine a solver actually runs (a FUSED request falls back to PLAIN on one-level grids).
int motorPcg(Pcg* p);
// Phase trace of the fused engine (%globaltimer at each grid barrier of the last solve).
void perfilPcg(Pcg* p, bool ligar);
int lerPerfilPcg(Pcg* p, unsigned long long* out, int cap);
// One V-cycle on device buffers (tq_vcycle).  A solver running many on the same types prepares
// the levels once (preparar on its first call only) and may pass a device stop flag.
int cicloVDispositivo(Pcg* p, const uint8_t* tipo, const float* b, float* x, cudaStream_t s, bool preparar = true,
                      const int* parar = nullptr);
// One V-cycle with the level hierarchy in a static device array (tq_vcycle_noalloc): its
// capacity, the bytes a grid needs, the array's address on the current device (looked up once
// per device) and the cycle itself.
constexpr size_t BYTES_SCRATCH_VCICLO = (size_t)16 << 20;
size_t bytesScratchVCiclo(int nx, int ny);
int enderecoScratchVCiclo(void** out);
int cicloVSemAlocar(void* scratch, int nx, int ny, const uint8_t* tipo, const float* b, float* x, int precisao,
                    cudaStream_t s);

// ar.cu — RastreadorDeAr.atualizar on the device.
struct Rastreador;
Rastreador* criarRastreador(int nx, int ny);
void destruirRastreador(Rastreador* r);
void reiniciarRastreador(Rastreador* r, const Dev& d, cudaStream_t s);
int atualizarRastreador(Rastreador* r, const Dev& d, cudaStream_t s);
int primeiraRastreador(Rastreador* r);
void definirPrimeiraRastreador(Rastreador* r, int v);

}  // namespace tq
