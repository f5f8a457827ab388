/*
 * tanque.h — C-ABI of the B200 simulation step of the 2-D FLIP/APIC water tank.
 *
 * This is the drop-in boundary for the reference's CPU engine: one handle replaces one
 * `new SimulacaoCPU(cena, opcoes)` (js/fisica-cpu.js:28-77) and each entry point below
 * names the JavaScript method it stands in for.  Two more entry points stand in for the
 * standalone exports of js/pressao-cpu.js (`resolverPCG`, `cicloV`).
 *
 * Conventions (the reference's JS owns typed arrays; here the caller owns host buffers):
 *   - every function returns TQ_OK (0) or a negative TQ_E_* code and never throws;
 *   - host pointers are plain caller-owned buffers, read or written only during the call;
 *   - the library owns all device memory; one handle = one CUDA stream; a handle is not
 *     thread-safe, separate handles may run on separate host threads;
 *   - every wait on the device is bounded and reports TQ_E_TIMEOUT instead of hanging;
 *   - particles are 12 floats each, the reference's CAMPOS layout
 *     (x y vx vy cux cuy cvx cvy espuma absR absG absB, js/fisica-cpu.js:26);
 *   - cell (i, j) is index i + j*nx; u faces (nx+1)*ny, v faces nx*(ny+1)
 *     (js/fisica-cpu.js:39-40); the wall SDF is (2nx) x (2ny) (js/cena.js:19-24).
 */
#ifndef TANQUE_H
#define TANQUE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status codes */
#define TQ_OK 0
#define TQ_E_ARG (-1)       /* bad argument (null handle, size mismatch, bad enum) */
#define TQ_E_CUDA (-2)      /* a CUDA runtime call failed */
#define TQ_E_NOMEM (-3)     /* device or host allocation failed */
#define TQ_E_CAPACITY (-4)  /* particle capacity or a fixed table size exceeded */
#define TQ_E_TIMEOUT (-5)   /* a bounded device-side wait gave up */
#define TQ_E_NODEV (-6)     /* no CUDA device, or the requested one is missing */
#define TQ_E_STATE (-7)     /* call not valid in the handle's current state */

/* ---------------------------------------------------------------- option enums */
/* Storage type of the multigrid preconditioner's vectors (x, b, tmp on every level).
 * Arithmetic is FP32 in all cases; CG vectors stay FP32, dots/norms FP64. */
#define TQ_PREC_FP32 0
#define TQ_PREC_FP16 1
#define TQ_PREC_BF16 2

/* Execution engine of the pressure solve.
 * PLAIN: one kernel launch per reference dispatch (the decomposition of js/gpu/pcg.js and
 *        js/gpu/multigrid.js), host-driven iteration loop.
 * FUSED: the whole MGPCG solve in one persistent cooperative kernel with bounded grid
 *        barriers; the coarse levels run inside one CTA's shared memory. */
#define TQ_ENGINE_PLAIN 0
#define TQ_ENGINE_FUSED 1

/* Preconditioner of the pressure solve.
 * REFERENCE: cicloV as js/pressao-cpu.js:241-255 and precondicionar (:352-361): enclosed air
 *            of an active bubble counts as water in the V-cycle, the bubble's residual is
 *            spread evenly over its cells and its correction is their mean.
 * BLOCK:     no counterpart in the reference.  A block-diagonal preconditioner: the bubble
 *            rows take a Jacobi step (z_b = r_b / faces_b), and the V-cycle runs on the water
 *            alone with enclosed air as free surface; coarse neighbour masks come from the
 *            fine level's faces (a coarse face is open only where a fine face across it joins
 *            two non-wall cells), so coarse levels do not connect water through thin walls.
 *            Same smoother, transfers and coarse solve as REFERENCE.  With a tolerance the
 *            solve converges to the same q (within the tolerance) in about half the
 *            iterations on scenes with trapped air; with a fixed iteration count the iterates
 *            differ from the reference's.  FUSED engine only. */
#define TQ_PRECOND_REFERENCE 0
#define TQ_PRECOND_BLOCK 1
/* TQ_PRECOND_BLOCK_1: TQ_PRECOND_BLOCK whose V-cycle takes one smoother pass a leg on the
 *            levels above 0 (shift 8, red-black down and black-red up, so it stays symmetric)
 *            instead of two: more iterations, fewer and cheaper ones.  Faster where the solve
 *            is latency-bound (the 840x536 scene: 107 iterations of 122 us against 97 of 152
 *            us); slower on large atlases, whose level-0 passes dominate. */
#define TQ_PRECOND_BLOCK_1 2

/* Particle-to-grid transfer semantics (the oracle implements both; the CUDA library only
 * TQ_P2G_FIXED, the integer accumulation of js/gpu/fisica.js:77-131). */
#define TQ_P2G_FLOAT 0 /* js/fisica-cpu.js:198-267: float sums in particle order */
#define TQ_P2G_FIXED 1 /* i32 sums of round(w*val*65536): order independent, bit-exact */

/* ---------------------------------------------------------------- options */
/* Mirrors `new SimulacaoCPU(cena, opcoes)` (js/fisica-cpu.js:29-37, 64) plus the scene
 * size of `new Cena(nx, ny, h)` (js/cena.js:15-18). */
typedef struct tq_options {
  int32_t nx, ny;            /* grid cells (Cena.nx, Cena.ny) */
  double h;                  /* cell size in metres (Cena.h) */
  double gravity[2];         /* opcoes.gravidade, default {0, -9.81} */
  int32_t iterations;        /* opcoes.iteracoes (ITERACOES_PCG = 3); with tolerance > 0:
                                the iteration cap */
  int32_t air;               /* opcoes.ar (bubble tracking on/off), default 1 */
  double tau_density;        /* opcoes.tauDensidade, default TAU_DENSIDADE = 0.1 s */
  double surface_tension;    /* opcoes.tensao, default TENSAO_SUPERFICIAL = 0.0728 N/m */
  double tolerance;          /* 0: fixed iteration count as in the reference; > 0: stop when
                                the TRUE residual ||b - A q|| <= tolerance * ||r0||, both
                                in FP64 with the norm of js/pressao-cpu.js:342 (see
                                tq_solve_pressure) */
  int32_t precision;         /* TQ_PREC_* */
  int32_t engine;            /* TQ_ENGINE_* */
  int32_t p2g_mode;          /* TQ_P2G_* */
  int32_t capacity;          /* particle capacity; 0: ceil(nx*ny*PARTICULAS_MAX_POR_CELULA) */
  int32_t device;            /* CUDA device ordinal */
  int32_t preconditioner;    /* TQ_PRECOND_*, default TQ_PRECOND_REFERENCE */
  int32_t fused_ctas;        /* FUSED engine: CTAs of the persistent solve (one per SM at
                                most); 0 = one per SM.  Fewer let several handles' solves run
                                side by side (tq_launch_graph) */
  int32_t reserved[5];
} tq_options;

/* Fills defaults for an nx x ny tank of cell size h. */
void tq_options_default(tq_options* o, int32_t nx, int32_t ny, double h);

/* ---------------------------------------------------------------- tools */
/* aplicarFerramenta(f) (js/fisica-cpu.js:129-152). kind: 0 none, 1 esponja (sponge, removes
 * particles in the circle), 2 mao (hand, pulls velocities toward (vx, vy)), 3 corante (dye). */
typedef struct tq_tool {
  int32_t kind;
  int32_t pad;
  double x, y, radius, vx, vy;
  double absorb[3];
} tq_tool;

/* ---------------------------------------------------------------- handle */
typedef struct tq_sim tq_sim;

/* new SimulacaoCPU(cena, opcoes) (js/fisica-cpu.js:29-77).  The walls start as the empty
 * tank of `new Cena(nx, ny, h)` (frame of MOLDURA cells, js/cena.js:132-144). */
int tq_create(const tq_options* opts, tq_sim** out);
int tq_destroy(tq_sim* s);

/* Cena edits + SimulacaoCPU.atualizarParedes() (js/fisica-cpu.js:80-85): uploads the caller's
 * SDF (mw = 2*nx by mh = 2*ny floats, in cells) and recomputes the solid-cell mask
 * (Cena.celulaSolida, js/cena.js:119-127). */
int tq_set_walls(tq_sim* s, const float* sdf, int32_t mw, int32_t mh);

/* Cena.tracar(x0, y0, x1, y1, raio, apagar) (js/cena.js:43-72) + atualizarParedes, on the
 * device: draws (erase = 0) or erases (erase != 0) a capsule wall segment (metres) in the
 * handle's SDF mask, in the reference's double arithmetic, and recomputes the solid cells.
 * The mask equals, bit for bit, the one Cena.tracar makes.  Non-finite arguments: TQ_E_ARG
 * (the JavaScript draws nothing or NaNs). */
int tq_trace_wall(tq_sim* s, double x0, double y0, double x1, double y1, double radius, int32_t erase);

/* Cena.limpar() (js/cena.js:74-77, #zerar :139-144) + atualizarParedes on the device: the mask
 * of an empty tank (the frame alone) and its solid cells. */
int tq_clear_walls(tq_sim* s);

/* The particle splat of the renderer (WGSL_MANCHA, js/gpu/render.js:11-43, drawn in
 * js/gpu/render.js:236-265) without a graphics API: into `out`, a DEVICE buffer of 5 * w * h
 * floats (planes of w x h pixels covering the tank, row 0 at the top), every live particle
 * adds at each pixel centre within RAIO_MANCHA = 2.1 cells the weight (1 - r^2)^2 (plane 0),
 * times its foam (plane 1) and times its three absorptions (planes 2-4); r is the distance
 * over the radius.  Sums are 64-bit fixed point (2^-32), so the image does not depend on the
 * order of the particles; the renderer keeps them in half floats.  Runs on the handle's
 * stream and returns when `out` is written.  w * h above 2^26: TQ_E_ARG. */
int tq_splat(tq_sim* s, int32_t w, int32_t h, float* out);

/* SimulacaoCPU.adicionar(lista, checarCheia) (js/fisica-cpu.js:92-111).  Particles inside
 * walls or (check_full) in a cell already holding >= 3 particles are skipped.  *accepted
 * receives the count kept.  Particles beyond capacity: TQ_E_CAPACITY, nothing added. */
int tq_add_particles(tq_sim* s, const float* list, int32_t n, int32_t check_full,
                     int32_t* accepted);

/* The faucet: emitirTorneira (js/principal.js:301-321) on the device.  Emits, through
 * adicionar(lista, true)'s filter (walls, full cells), min(40000, round(2 r max(0.7, |v|) dt /
 * h^2 * 4)) particles in a disk of radius r around (x, y) at velocity (vx, vy) with the given dye;
 * the LCG of testes/apoio.js:4-9 seeded with `seed` stands in for Math.random (particle k takes
 * draws 2k+1, 2k+2: angle u1 * 2 pi, radius sqrt(u2) r), so the list equals the one the same LCG
 * makes on the host.  The caller computes the jet's velocity (the reference derives it from the
 * pointer). *accepted receives the count kept; beyond capacity: TQ_E_CAPACITY, nothing added. */
typedef struct tq_faucet {
  double x, y;        /* jet centre (m) */
  double radius;      /* jet radius (m) */
  double vx, vy;      /* jet velocity (m/s) */
  double dt;          /* the time the emission covers (s) */
  double absorb[3];   /* dye of the emitted water */
  uint32_t seed;
  int32_t pad;
} tq_faucet;
int tq_emit_faucet(tq_sim* s, const tq_faucet* faucet, int32_t* accepted);

/* Tanks of an atlas (no counterpart in the reference, which steps one tank): n rectangles of
 * cells, 4 int32 each (x0, y0, width, height), side by side in disjoint column ranges, walls
 * between them.  The tanks' systems are independent blocks of the atlas's pressure system; in
 * tolerance mode the solve then stops only when EVERY tank's own true residual is within the
 * tolerance of ITS OWN initial residual (bubble rows counted with the tank holding the bubble),
 * not the atlas's as a whole.  FUSED engine only (TQ_E_STATE otherwise); at most 4096 tanks;
 * n = 0 returns to the whole-grid test. */
int tq_set_tanks(tq_sim* s, int32_t n, const int32_t* rects);
/* After a solve with tanks: 2 doubles per tank, ||r0_t|| and the true ||r_t|| at the solve's end
 * (*n receives the tank count). */
int tq_get_tank_residuals(tq_sim* s, double* out, int32_t cap, int32_t* n);

/* MotorCPU.limparAgua without the air reset: sim.n = 0, contagemCelula.fill(0)
 * (js/motor.js:95). */
int tq_clear_particles(tq_sim* s);

/* SimulacaoCPU.aplicarFerramenta(f) (js/fisica-cpu.js:129-152). */
int tq_apply_tool(tq_sim* s, const tq_tool* tool);

/* SimulacaoCPU.avancar(dt, subpassos) (js/fisica-cpu.js:155-159): relabels the air once,
 * then runs `substeps` substeps of dt/substeps. */
int tq_advance(tq_sim* s, double dt, int32_t substeps);

/* SimulacaoCPU.subpasso(dt) (js/fisica-cpu.js:176-189). */
int tq_substep(tq_sim* s, double dt);

/* avancar(dt, subpassos) (js/fisica-cpu.js:155-159) with the substeps replayed from a CUDA
 * graph: the air relabel runs as in tq_advance, then the `substeps` substeps are captured into
 * a graph on the first call and replayed on later calls with the same dt and substep count
 * (recaptured when they, or the gravity, change, or the particle count grows past the captured
 * launch bound).
 * Results are bit-identical to tq_advance.  Stage timing is not recorded for the replayed
 * substeps.  The PLAIN engine in tolerance mode reads its stop flag on the host and cannot be
 * captured: TQ_E_STATE.  No counterpart in the reference (it has no graph API). */
int tq_advance_graph(tq_sim* s, double dt, int32_t substeps);
/* tq_advance_graph without the wait at its end: the frame is queued on the handle's stream and
 * the call returns (the air relabel before it still waits for the stream).  Handles on
 * different streams then step side by side: with tq_options.fused_ctas splitting the SMs,
 * their persistent solves run at the same time.  A solve that gave up on a bounded wait is
 * reported by the next tq_sync. */
int tq_launch_graph(tq_sim* s, double dt, int32_t substeps);

/* SimulacaoCPU.atualizarAr() (js/fisica-cpu.js:162-167) — RastreadorDeAr.atualizar
 * (js/ar.js:56-153) on the device. */
int tq_update_air(tq_sim* s);

/* SimulacaoCPU.reiniciarAr() (js/fisica-cpu.js:170-174). */
int tq_reset_air(tq_sim* s);

/* sim.n */
int tq_count(tq_sim* s, int32_t* n);

/* sim.p.subarray(0, 12*n) in the reference's order (insertion order, dead particles removed
 * stably).  cap is the capacity of `out` in particles. */
int tq_get_particles(tq_sim* s, float* out, int32_t cap, int32_t* n);

/* Replaces every particle (state restore; no filtering). */
int tq_set_particles(tq_sim* s, const float* list, int32_t n);

/* Copies a field out of / into the handle.  `bytes` must equal the field's size. */
enum tq_field {
  TQ_FIELD_TIPO = 0,            /* u8  N      tipo            (js/fisica-cpu.js:52) */
  TQ_FIELD_ROTULO = 1,          /* u32 N      rotulo          (js/ar.js:27) */
  TQ_FIELD_CONTAGEM = 2,        /* u32 N      contagemCelula  (js/fisica-cpu.js:50) */
  TQ_FIELD_SOLIDO = 3,          /* u8  N      solidoCelula    (js/fisica-cpu.js:53) */
  TQ_FIELD_U = 4,               /* f32 nu     u               (js/fisica-cpu.js:41) */
  TQ_FIELD_V = 5,               /* f32 nv     v */
  TQ_FIELD_Q = 6,               /* f32 N      q (pressure, p*dt/(rho*h)) */
  TQ_FIELD_DIV = 7,             /* f32 N      div */
  TQ_FIELD_DENSIDADE = 8,       /* f32 N      densidade */
  TQ_FIELD_FASE = 9,            /* f32 N      fase (blurred water fraction) */
  TQ_FIELD_CURVATURA = 10,      /* f32 N      curvatura */
  TQ_FIELD_QAR = 11,            /* f32 N      qAr */
  TQ_FIELD_PRESSAO_BOLHA = 12,  /* f32 4096   pressaoBolha (Pa) */
  TQ_FIELD_VOLUME_ALVO = 13,    /* f32 4096   rastreador.volumeAlvo */
  TQ_FIELD_VOLUME_BOLHA = 14,   /* f32 4096   volumeBolha */
  TQ_FIELD_RHS_BOLHA = 15,      /* f32 4096   rhsBolha */
  TQ_FIELD_Y_BOLHA = 16,        /* f32 4096   yBolha */
  TQ_FIELD_VIVO = 17,           /* u8  4096   rastreador.vivo */
  TQ_FIELD_U_VALIDA = 18,       /* u8  nu     uValida */
  TQ_FIELD_V_VALIDA = 19,       /* u8  nv     vValida */
  TQ_FIELD_U_PESO = 20,         /* f32 nu     uPeso */
  TQ_FIELD_V_PESO = 21,         /* f32 nv     vPeso */
  TQ_FIELD_NORMAL_X = 22,       /* f32 N      normalX */
  TQ_FIELD_NORMAL_Y = 23,       /* f32 N      normalY */
  TQ_FIELD_COR_CELULA = 24,     /* f32 3N     corCelula */
  TQ_FIELD_ACC_U = 25,          /* i32 2nu    fixed-point (value, weight) sums, TQ_P2G_FIXED */
  TQ_FIELD_ACC_V = 26,          /* i32 2nv */
  TQ_FIELD_ACC_CEL = 27,        /* i32 2N     (density*65536, particle count) */
  TQ_FIELD_ACC_COR = 28,        /* i32 3N     dye*256 */
  TQ_FIELD_SDF = 29,            /* f32 4N     wall SDF (2nx by 2ny) */
  TQ_FIELD_COUNT_ = 30
};
int tq_get_field(tq_sim* s, int32_t field, void* out, int64_t bytes);
int tq_set_field(tq_sim* s, int32_t field, const void* in, int64_t bytes);

/* Scalars (read; some writable for state restore). */
enum tq_scalar {
  TQ_SCALAR_VMAX = 0,           /* sim.vMax: largest particle speed of the last G2P */
  TQ_SCALAR_PRIMEIRA = 1,       /* rastreador.primeira (1/0) — writable */
  TQ_SCALAR_TIPOS_PRONTOS = 2,  /* sim.tiposProntos (1/0) — writable */
  TQ_SCALAR_PCG_ITERS = 3,      /* iterations run by the last pressure solve */
  TQ_SCALAR_PCG_RES0 = 4,       /* ||r0|| of the last solve */
  TQ_SCALAR_PCG_RES = 5,        /* final ||r|| of the last solve */
  TQ_SCALAR_LAUNCHES = 6,       /* kernels launched by this process so far (all handles) */
  TQ_SCALAR_GRAVITY_X = 7,      /* sim.gravidade[0] (m/s^2) — writable, used from the next */
  TQ_SCALAR_GRAVITY_Y = 8,      /* sim.gravidade[1]   substep (MotorCPU.gravidade, js/motor.js:96) */
  /* Convergence of the pressure solves (tolerance mode; no counterpart in the reference,
   * whose solve runs a fixed count).  The solves record these on the device: reading them
   * waits for the handle's stream, the solves themselves never wait for the host. */
  TQ_SCALAR_PCG_TRUE_RES = 9,   /* ||b - A q|| (FP64) of the last solve's iterate; -1 without
                                   a tolerance */
  TQ_SCALAR_PCG_CONVERGED = 10, /* 1: the last solve met its tolerance on the true residual;
                                   0: it stopped at the iteration cap */
  TQ_SCALAR_SOLVES = 11,        /* solves since the last reset — writing 0 resets 11-15 */
  TQ_SCALAR_SOLVES_CAPPED = 12, /* of them, stopped at the cap without converging */
  TQ_SCALAR_SOLVE_ITERS = 13,   /* their iterations in total */
  TQ_SCALAR_SOLVE_MAX_REL = 14, /* largest true ||b - A q|| / ||r0|| among them */
  TQ_SCALAR_SOLVE_REPLACEMENTS = 15, /* residual replacements among them (see tq_solve_pressure) */
  TQ_SCALAR_CLOSED_REGIONS = 16, /* closed regions (water sealed from every air cell at pressure
                                    0) whose right-hand side the last tolerance-mode solve
                                    projected onto A's range (see tq_solve_pressure) */
  TQ_SCALAR_GRAPH_FRAME_MS = 17, /* device time (ms) of the last frame replayed from the graph
                                    (tq_advance_graph / tq_launch_graph); waits for it; 0 before
                                    the first */
  TQ_SCALAR_COUNT_ = 18
};
int tq_get_scalar(tq_sim* s, int32_t which, double* out);
int tq_set_scalar(tq_sim* s, int32_t which, double value);

/* The residual-norm history `normas` returned by the last resolverPCG call
 * (js/pressao-cpu.js:343, 386, 401). */
int tq_last_norms(tq_sim* s, double* out, int32_t cap, int32_t* n);

/* Waits for the handle's stream; reports a queued solve that gave up on a bounded wait
 * (TQ_E_TIMEOUT). */
int tq_sync(tq_sim* s);

/* The handle's CUDA stream (a cudaStream_t), for callers that order their own device work
 * or timing events with the simulation's. */
int tq_get_stream(tq_sim* s, void** stream);

/* Stage timing with CUDA events on the handle's stream.  tq_set_timing(1) starts (and resets)
 * the accumulation; tq_get_timing returns 11 values accumulated since then:
 * [0..6] ms in p2g+faces, cell flags+labels, surface, divergence+bubbles, pressure solve,
 * gradient+extrapolation, g2p; [7] ms in air relabels; [8] substeps timed; [9] pressure
 * iterations in total; [10] relabels timed. */
int tq_set_timing(tq_sim* s, int32_t enabled);
int tq_get_timing(tq_sim* s, double* ms_out, int32_t cap, int32_t* n);

/* With tq_set_timing(s, 2) the fused engine also records a phase trace of its last pressure
 * solve: the device %globaltimer (ns) as each grid barrier completes.  Consecutive
 * differences are the durations of the solve's phases. */
int tq_get_phase_trace(tq_sim* s, uint64_t* out, int32_t cap, int32_t* n);

/* ---------------------------------------------------------------- standalone solver */
/* Bubble description for the standalone solve: `bolhas = { rotulo, rhs, y }` of
 * resolverPCG (js/pressao-cpu.js:291-296).  y is read as the initial guess and receives
 * the solved bubble pressures of the active bubbles. */
typedef struct tq_bubbles {
  const uint32_t* rotulo; /* N labels (0 none, 1 atmosphere, >=2 bubble) */
  const float* rhs;       /* 4096 */
  float* y;               /* 4096 */
} tq_bubbles;

/* What a solve reports beside q (tq_solve_pressure's `info`, may be NULL). */
typedef struct tq_solve_info {
  int32_t iterations;    /* iterations run */
  int32_t converged;     /* tolerance mode: 1 when ||b - A q|| <= tolerance * ||r0||; else 0 */
  int32_t replacements;  /* residual replacements (tolerance mode) */
  int32_t closed_regions; /* tolerance mode: closed regions whose right-hand side was projected */
  double residual0;      /* ||r0|| (of the projected right-hand side in tolerance mode) */
  double residual;       /* the last recursive ||r|| */
  double true_residual;  /* ||b - A q|| in FP64 of the final iterate (tolerance mode), else -1 */
} tq_solve_info;

/* resolverPCG(niveis, tipo, div, q, iteracoes, bolhas) (js/pressao-cpu.js:296-402) on the
 * device: solves n*q - sum(q_nb) = -div on water cells starting from q.
 * tolerance = 0 runs exactly `iterations`, as the reference does (ITERACOES_PCG = 3).
 * tolerance > 0 (no counterpart in the reference) accumulates q in FP64 during the solve and
 * stops when the TRUE residual ||b - A q||, recomputed in FP64 from the FP64 iterate and the
 * bubble pressures, is <= tolerance * ||r0||, or at `iterations` (the cap).  The true residual
 * is recomputed whenever the recursive FP32 one meets the tolerance, and each time the
 * recursive one has fallen by 1e-3 since the last recomputation; unless the solve ends there,
 * the true residual replaces the recursive one and CG goes on with the same search direction
 * (residual replacement), which keeps the FP32 rounding of the recursive residual far below
 * the tolerance.
 * Closed regions (tolerance mode): a 4-connected set of unknowns (water cells, joined to their
 * water neighbours and to the active bubbles they face) that touches no air cell at pressure 0
 * is water sealed by walls; A is singular on it (its null vector the constant over the
 * region's water cells and bubble pressures) and b's component along that vector cannot be
 * removed, so a solve stopping on the residual could never stop there.  Before the solve each
 * closed region's right-hand side (-div on water, rhs on bubbles) loses its mean over the
 * region's unknowns; open regions are untouched and the caller's div and rhs are not written.
 * The reference, with its fixed count, solves the unprojected system as far as it gets.
 * q is returned rounded to FP32, so b - A q of the returned float q carries their rounding
 * (about 1e-7 of |A| |q| per cell) on top of the reported true residual.
 * norms receives the recursive residual history (initial, then one per iteration).
 * preconditioner: TQ_PRECOND_*; TQ_PRECOND_BLOCK needs engine TQ_ENGINE_FUSED. */
int tq_solve_pressure(int32_t nx, int32_t ny, const uint8_t* tipo, const float* div, float* q,
                      int32_t iterations, double tolerance, const tq_bubbles* bubbles,
                      int32_t precision, int32_t engine, int32_t preconditioner, double* norms,
                      int32_t norms_cap, int32_t* n_norms, tq_solve_info* info);

/* cicloV(niveis) (js/pressao-cpu.js:241-255) on the device: one V-cycle approximately
 * solving A x = b on the level-0 grid described by `tipo` (the types the preconditioner
 * sees), starting from x = 0.  x receives the result. */
int tq_vcycle(int32_t nx, int32_t ny, const uint8_t* tipo, const float* b, float* x,
              int32_t precision);

/* The same V-cycle as tq_vcycle, for callers that must not allocate device memory while
 * they run (no counterpart in the reference).  A host engine whose allocator already holds
 * the device memory it is allowed to use, or that cannot afford cudaFree's device-wide
 * synchronisation or an allocation failing in the middle of a frame, gets the V-cycle's
 * level hierarchy from a static device array instead: nothing is allocated or freed.
 *
 * tipo, b and x are DEVICE pointers on the current device (N = nx*ny bytes, floats, floats;
 * x is written, b and tipo only read); the work is queued on `stream` (a cudaStream_t, NULL
 * for the default stream) and the call returns without waiting for it.
 * Limit: the levels of the grid must fit in 16 MiB of scratch (about 13 bytes per level-0
 * cell plus 14 per coarse cell: roughly 900,000 cells, e.g. 1280x720); a larger grid
 * returns TQ_E_CAPACITY, with the bytes it needs in tq_last_error, before any device work.
 * Nothing in the scratch needs to start at zero: each call writes what it reads.
 * The scratch is shared by every call on a device: calls whose work overlaps in time (two
 * streams, or two host threads) race on it and corrupt each other's results, so keep the
 * calls on one device in one stream, or wait for one before issuing the next.
 * The first call on each device does a one-time set-up (it looks up the scratch's device
 * address); a caller that captures streams makes that first call before capturing.  The
 * address belongs to the device's current context: after cudaDeviceReset (or a primary
 * context released and made again) the next call sees the new context and looks the address
 * up again, which is again a set-up call.  Grids above 2^20 cells a side or 2^28 cells are
 * refused with TQ_E_CAPACITY before any size arithmetic.  A CUDA error left pending by earlier
 * work on the calling thread is reported (and cleared) as TQ_E_CUDA without launching. */
int tq_vcycle_noalloc(int32_t nx, int32_t ny, const uint8_t* tipo, const float* b, float* x,
                      int32_t precision, void* stream);

/* ---------------------------------------------------------------- adjoint of the step */
/* No counterpart in the reference (it has no gradients).  A differentiable simulation: the
 * substep of SimulacaoCPU.subpasso (js/fisica-cpu.js:176-189) with air tracking off, surface
 * tension 0 and the density correction off — P2G (APIC), gravity and wall faces, cell flags, the
 * pressure projection (resolverPCG's system solved to a relative 1e-12), gradient, extrapolation,
 * G2P with micro-steps and wall collisions — run forward and backward in FP64 on the GPU.  The
 * discrete structure (cell flags, valid masks, micro-step counts, speed clamps, collision branches,
 * kills, the faucet's insert filter) is the forward run's, held fixed in the backward run: the
 * gradient is that of the smooth map the forward run sits on.
 *
 * Loss: sum over cells of (min(1, rho/4) - target)^2, rho the bilinear particle density at the
 * cell centres after the last step (#paraGrade's densidade, js/fisica-cpu.js:244-254).
 * Controls: the initial particle velocities (2 per particle) and the faucet velocity theta (2
 * scalars), the velocity of the particles the faucet emits at the start of every step at the
 * given positions (they pass adicionar's wall filter, js/fisica-cpu.js:100).
 * The forward run keeps the state every `checkpoint_every` steps; the backward run recomputes
 * each segment from its checkpoint and goes back through it (the torch.autograd.Function
 * contract: forward saves what backward needs). */
typedef struct tq_adj_scene {
  int32_t nx, ny;
  double h, dt;
  int32_t steps;
  int32_t checkpoint_every;     /* steps between checkpoints; 0: 10 */
  double gravity[2];
  const float* sdf;             /* wall SDF, (2 nx) x (2 ny), as tq_set_walls */
  const float* positions;       /* 2 per initial particle (x, y) in metres */
  const float* affine;          /* 4 per initial particle (cux cuy cvx cvy), or NULL for 0 */
  const float* faucet_positions;/* steps x faucet_per_step x 2 */
  const float* target;          /* nx * ny target water fraction */
  int32_t n_particles;
  int32_t faucet_per_step;
} tq_adj_scene;

typedef struct tq_adj tq_adj;
int tq_adj_create(const tq_adj_scene* scene, int32_t device, tq_adj** out);
int tq_adj_destroy(tq_adj* a);
/* The forward run: v0 = 2 per initial particle, theta = 2; *loss receives the loss. */
int tq_adj_forward(tq_adj* a, const float* v0, const double* theta, double* loss);
/* The backward run of the last forward run: dL/dv0 (2 per initial particle, FP32) and dL/dtheta
 * (2), scaled by `grad_loss` (the incoming gradient of the loss). */
int tq_adj_backward(tq_adj* a, double grad_loss, float* dv0, double* dtheta);

/* ---------------------------------------------------------------- errors */
const char* tq_status_string(int status);
/* Last error message of the calling thread (CUDA error text or argument problem). */
const char* tq_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* TANQUE_H */
