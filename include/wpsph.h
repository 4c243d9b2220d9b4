/* wpsph.h — C ABI of libwpsph.so, the B200 (sm_100a) IISPH time step.
 *
 * The reference (Mo-ZheHan/WarpSPH) has no native layer: its Python class
 * wp_sph.solver.IISPH (wp_sph/solver/IISPH.py:736) drives Warp kernels.  These
 * entry points are what that class binds through ctypes in place of its Warp
 * arrays and launches; each declaration names the reference code it replaces.
 *
 * Conventions
 *   - Every int-returning call returns SPH_OK (0) or a negative SPH_E_* code;
 *     sph_last_error() describes the last failure.  Nothing throws or exits.
 *   - Host buffers are caller-owned and copied; device buffers are owned by the
 *     context.  Arrays are in the caller's ORIGINAL particle order; the cell-
 *     sorted order the kernels use internally is never exposed.
 *   - One context = one CUDA device + one CUDA stream.  A context is not
 *     thread-safe; distinct contexts are independent.
 *   - float3 arrays are packed xyz, 3 floats per particle.
 */
#ifndef WPSPH_H
#define WPSPH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WPSPH_ABI_VERSION 1

#define SPH_OK 0
#define SPH_E_INVALID -1   /* bad argument or call order */
#define SPH_E_CUDA -2      /* CUDA runtime error */
#define SPH_E_CAPACITY -3  /* neighbour capacity exceeded (raise max_ff / max_fb) */
#define SPH_E_NONFINITE -4 /* NaN/Inf in pressure or velocity */
#define SPH_E_TIMEOUT -5   /* a bounded grid-wide wait expired */
#define SPH_E_NOMEM -6     /* device allocation failed */
#define SPH_E_TOO_LARGE -7 /* input larger than a fixed-size limit (sph_boundary_psi_noalloc) */

/* SphStepStats.flags bits */
#define SPH_F_FF_OVERFLOW 0x1
#define SPH_F_FB_OVERFLOW 0x2
#define SPH_F_NONFINITE 0x4
#define SPH_F_TIMEOUT 0x8
#define SPH_F_NOT_CONVERGED 0x10 /* hit the iteration cap (IISPH.py:1202-1207: a print) */

/* Warm-start modes for the pressure solve (IISPH.py:166-174). */
#define SPH_WARM_ZERO 0 /* p <- 0, the reference's behaviour (IISPH.py:173) */
#define SPH_WARM_HALF 1 /* p <- 0.5 p_prev (the variant at IISPH.py:174) */
#define SPH_WARM_MLP 2  /* first iterate <- learned per-particle MLP prediction */

typedef struct SphParams {
  double spacing;    /* DIAMETER (wp_sph/main.py:26) */
  double h;          /* SMOOTHING_LENGTH = 2*DIAMETER (main.py:57) */
  double rho0;       /* RHO_0 (main.py:30) */
  double gravity;    /* GRAVITY (main.py:25); acts along -y */
  double omega;      /* OMEGA, relaxed-Jacobi weight (main.py:27) */
  double eta;        /* ETA, average density error tolerance (main.py:28) */
  double inv_small;  /* INV_SMALL (main.py:29) */
  double vis_mu;     /* VIS_MU (main.py:61) */
  double fluid_mass; /* FLUID_MASS = RHO_0*DIAMETER^3 (main.py:59) */
  double sigma;      /* SIGMA = 8/(pi h^3) (main.py:60) */
  double dt_max;     /* TIME_STEP_MAX = 0.05*DIAMETER (main.py:58) */
  double cfl_len;    /* 0.4*DIAMETER (IISPH.py:1369) */
  double dt0;        /* first step's dt (IISPH.py:747) */
  double domain_min[3], domain_max[3]; /* neighbour-grid extent; zero extent = fit to particles */
  int32_t w_table_size;  /* W_SIZE (sph_funcs.py:43) */
  int32_t g_table_size;  /* GRAD_W_SIZE (sph_funcs.py:44) */
  int32_t min_iter;      /* 2  (IISPH.py:1201) */
  int32_t max_loop;      /* 100 (IISPH.py:1202) */
  int32_t fixed_iters;   /* -1 = converge; >= 1 = exactly this many iterations */
  int32_t warm_start;    /* SPH_WARM_* */
  int32_t max_ff;        /* fluid-fluid neighbour capacity per particle */
  int32_t max_fb;        /* fluid-boundary neighbour capacity per particle */
  int32_t keep_fb_lists; /* unused (fluid-boundary lists are always kept); must be 0 or 1 */
  int32_t use_graph;     /* replay the step as a CUDA graph */
  int32_t device;        /* CUDA device ordinal */
  int32_t block_size;    /* threads per block of the neighbour build (0 = 128) */
  int32_t timeout_ms;    /* bound on every grid-wide wait */
  int32_t jacobi_block;  /* threads per block of the pressure solve: 128 or 256 with any
                            (jacobi_ppt, jacobi_unroll) below, or 512 / 1024 with (1, 4)
                            (0 = 1024) */
  int32_t jacobi_ppt;    /* particles per solve thread: 1 or 2 (0 = 1) */
  int32_t jacobi_unroll; /* neighbour-loop unroll of the solve: 2, 4 or 8 (0 = 4) */
  int32_t move_boundary;  /* 1: boundary particles move with their velocities, x += v dt after
                            every step's drift (update_rigid_x, IISPH.py:651-671, 1356-1365), and
                            the boundary grid is rebuilt every step (IISPH.py:1415-1416); psi
                            keeps the values of sph_set_boundary, as the reference computes it
                            once (IISPH.py:811-821) */
  int32_t warm_continue;  /* 1 (SPH_WARM_MLP only): after a solve that stopped at the iteration
                            cap, the next step of that scene starts from the capped solve's final
                            pressure (or from sph_set_pressure's, if called in between) instead
                            of the network's prediction; sph_set_fluid forgets the cap */
  int32_t plain_loads;    /* 1: every neighbour gather uses plain global loads; 0 (default): the
                            gathers of arrays that a kernel only reads (the solve's second-pass
                            positions, the neighbour build's positions and velocities) go through
                            the texture path, from texture objects over the same arrays, beside
                            the plain loads of the rest; same values, same results */
} SphParams;

typedef struct SphStepStats { /* for a batch: max over scenes, dt and time of scene 0 */
  int32_t iterations; /* Jacobi iterations executed (IISPH.py:1200-1296 `loop`) */
  int32_t flags;      /* SPH_F_* */
  double avg_err;     /* average_rho_error (IISPH.py:1489-1494), FP64 reduction */
  double v_max;       /* max |v| after the kick (IISPH.py:688) */
  double dt;          /* dt used by this step */
  double dt_next;     /* CFL dt for the next step (IISPH.py:1368-1370) */
  double sim_time;    /* sim_time after this step (IISPH.py:1367) */
  int64_t n_ff_pairs; /* sum of fluid-fluid neighbour counts */
  int64_t n_fb_pairs; /* sum of fluid-boundary neighbour counts */
  int32_t max_ff_count, max_fb_count;
  int64_t step_index;
} SphStepStats;

typedef struct SphCtx SphCtx;

/* Reference defaults: the constants of wp_sph/main.py:25-61 and sph_funcs.py:43-44. */
int sph_params_default(SphParams* p);

/* Replaces IISPH.__init__'s array allocation and hash-grid creation (IISPH.py:770-805). */
int sph_create(const SphParams* params, SphCtx** out);
void sph_destroy(SphCtx* ctx);
const char* sph_last_error(const SphCtx* ctx);

/* Kernel tables (sph_funcs.py:47-86).  Optional: without it the library builds
 * the tables itself from params (FP64 then float32, as sph_funcs.py does). */
int sph_set_tables(SphCtx* ctx, const float* w_table, int32_t w_size, const float* g_table, int32_t g_size);

/* The tables sph_create builds when none are set, written to caller buffers of
 * params->w_table_size and params->g_table_size floats.  Host only (no GPU). */
int sph_build_tables(const SphParams* params, float* w_table, float* g_table);

/* Boundary particles (IISPH.py:990-991) and their volume psi, computed once
 * (compute_boundary_density, IISPH.py:23-49, launched at IISPH.py:811-821). */
int sph_set_boundary(SphCtx* ctx, const float* xb3, const float* vb3, int64_t nb);

/* Fluid particles (IISPH.py:993-994) with velocities (NULL = zero). */
int sph_set_fluid(SphCtx* ctx, const float* x3, const float* v3, int64_t n);

/* Replace positions, velocities and pressures (original order) of the current
 * fluid particles, keeping everything else the solver carries from step to
 * step: dt, simulated time, the neighbour grid and the warm_continue cap flags
 * (sph_set_fluid starts a new state and forgets them).  For callers that keep
 * the state in host memory between steps (a checkpoint round trip, a coupled
 * host-side code): stepping on after sph_get_fluid + sph_update_fluid gives
 * the same result as stepping on directly.  n must equal the fluid count.
 * p = NULL keeps the pressures on the device (the reference's state is x and
 * v; the pressure is only the warm start's history), so a round trip of x
 * and v alone also steps on exactly as the device would.
 * No counterpart in the reference, whose state lives in Warp arrays. */
int sph_update_fluid(SphCtx* ctx, const float* x3, const float* v3, const float* p, int64_t n);

/* Append `count` fluid particles (velocities NULL = zero, pressure 0) to the
 * current state, keeping every existing particle's state; the new particles get
 * original ids n .. n + count - 1.  For emitters (an inlet adding a layer of
 * particles every few steps).  No counterpart in the reference, whose particle
 * set is fixed at init_particles (IISPH.py:857-1000).  Single-scene contexts
 * only.  The neighbour grid is not refitted: give params->domain_* to cover the
 * region the emitted fluid will reach (particles outside the grid stay correct,
 * in the clamped edge cells, but make those cells long). */
int sph_add_fluid(SphCtx* ctx, const float* x3, const float* v3, int64_t count);

/* ---- Batches of independent scenes ---------------------------------------
 * No counterpart in the reference (one scene per IISPH object).  All scenes
 * share the physical parameters and advance together: one sort, one build and
 * one persistent solve per step, in which each scene keeps its own grid, dt,
 * CFL, residual, convergence decision and iteration count; a converged scene
 * drops out of the remaining Jacobi passes.  Fluid and boundary arrays of the
 * batch are the scenes' arrays concatenated in scene order (sph_set_fluid,
 * sph_get_fluid, ... then take and return those concatenations). */
typedef struct SphSceneDesc {
  const float* x3;  /* n x 3 fluid positions */
  const float* v3;  /* n x 3 fluid velocities, NULL = zero */
  int64_t n;
  const float* xb3; /* nb x 3 boundary positions */
  const float* vb3; /* NULL = static */
  int64_t nb;
  double domain_min[3], domain_max[3]; /* grid extent; zero extent = fit to the particles */
} SphSceneDesc;

int sph_create_batch(const SphParams* params, const SphSceneDesc* scenes, int32_t nscenes, SphCtx** out);
int32_t sph_num_scenes(const SphCtx* ctx);
/* fluid_off / boundary_off: nscenes + 1 prefix offsets into the concatenated arrays. */
int sph_get_scene_ranges(SphCtx* ctx, int64_t* fluid_off, int64_t* boundary_off);
/* Per-scene results of the last step (arrays of nscenes; any may be NULL):
 * Jacobi iterations, average density error, max |v|, next dt, simulated time. */
int sph_get_scene_stats(SphCtx* ctx, int32_t* iterations, double* avg_err, double* v_max, double* dt,
                        double* sim_time);

/* Pressure carried into the next step's warm start (SPH_WARM_HALF / SPH_WARM_MLP). */
int sph_set_pressure(SphCtx* ctx, const float* p, int64_t n);

/* One time step: IISPH.step() (IISPH.py:1002-1371).  Blocks until the step's
 * statistics are on the host when out != NULL. */
int sph_step(SphCtx* ctx, SphStepStats* out);

/* nsteps time steps back to back with one host synchronisation; per-step stats
 * (up to 4096 most recent) are then available from sph_get_stats_history. */
int sph_steps(SphCtx* ctx, int32_t nsteps, SphStepStats* last);
int sph_get_stats_history(SphCtx* ctx, SphStepStats* out, int32_t count);

/* Asynchronous form for callers that time with CUDA events on sph_stream():
 * enqueue nsteps steps with no host synchronisation.  Flags surface at the
 * next sph_get_stats/sph_step. */
int sph_launch_steps(SphCtx* ctx, int32_t nsteps);
/* Capture the step's CUDA graph now (it is otherwise captured by the first
 * step), so that a caller's first timed step excludes the capture. */
int sph_prepare(SphCtx* ctx);
/* Enqueue one part of a step without the graph (for per-kernel timing on
 * sph_stream): 0 = cell sort + neighbour build, 1 = pressure solve (2 then 3),
 * 2 = warm-start inference only (a no-op unless SPH_WARM_MLP),
 * 3 = persistent Jacobi solve with the fused kick/drift/CFL only.
 * Phases 0, 1 (or 0, 2, 3) in order make one step. */
int sph_launch_phase(SphCtx* ctx, int32_t phase);

/* Test hook for the solve's failure path (no reference counterpart): from the
 * next step on, block `block` of the persistent solve skips its first
 * grid-barrier arrival, so every block's bounded wait (timeout_ms) runs out;
 * the step then returns SPH_E_TIMEOUT with the state, time and dt as they were
 * before it.  -1 turns the hook off. */
int sph_test_stall_barrier(SphCtx* ctx, int32_t block);
/* Test hook for the warm-start inference's failure path (no reference
 * counterpart): with on = 1 the tensor-core inference issues no MMA, so its
 * first bounded mbarrier wait runs out; the kernel frees its tensor memory and
 * sets SPH_F_TIMEOUT, the solve then stops at its first barrier, and the step
 * returns SPH_E_TIMEOUT with the state as it was.  0 turns the hook off. */
int sph_test_withhold_mma(SphCtx* ctx, int32_t on);

/* IISPH.neighbor_search() (IISPH.py:1408-1482): cell sort + neighbour build +
 * density for the current state, without advancing time. */
int sph_neighbor_search(SphCtx* ctx);

/* Read back state in original order; any pointer may be NULL.
 * x/v/p/rho/rho_adv mirror the IISPH attributes of the same names (IISPH.py:783-788). */
int sph_get_fluid(SphCtx* ctx, float* x3, float* v3, float* p, float* rho, float* rho_adv);
/* Intermediate terms of the last step: term_d_ii, term_a_ii, sum_d_ij_p_j, v_adv
 * (IISPH.py:784, 792-797), and term_Ap_i of the last pass. */
int sph_get_terms(SphCtx* ctx, float* d_ii3, float* a_ii, float* s3, float* v_adv3, float* Ap);
/* boundary_x and boundary_phi (IISPH.py:789, 990) in original boundary order. */
int sph_get_boundary(SphCtx* ctx, float* xb3, float* psi);
/* Neighbour sets of the last build in original ids, CSR per fluid particle,
 * ids ascending (ff_neighbor_* / fs_neighbor_*, IISPH.py:798-805). */
int sph_get_neighbors(SphCtx* ctx, int64_t* ff_off, int32_t* ff_idx, int64_t ff_cap,
                      int64_t* fb_off, int32_t* fb_idx, int64_t fb_cap);

int sph_get_stats(SphCtx* ctx, SphStepStats* out);
/* Override dt / 1/dt for the next step (the reference's self.dt, self.inv_dt). */
int sph_set_dt(SphCtx* ctx, double dt, double inv_dt);
/* Solid sampling of a closed triangle mesh (scene generation): replaces the
 * reference's model sampler (wp_sph/solver/model.py:14-60, `_sample_points` +
 * `load_model`), used by init_particles for mesh scenes (IISPH.py:952-989).
 * The caller passes the mesh (nv vertices, FP64 xyz; nt triangles, vertex
 * indices) and the lattice axes xs, ys, zs (strictly ascending; the reference
 * takes np.arange(lo, hi, spacing) over the mesh bounds); the library writes,
 * in lattice order (x slowest, z fastest), every lattice point inside the
 * mesh, transformed as p @ rot + pos (rot9 row-major 3 x 3, as numpy's
 * `points @ rot`), as float32 xyz into out3 (cap points) and the number of
 * such points into *count.  Inside means an odd number of crossings of the
 * ray from the point along +x strictly beyond it (each crossing of a closed
 * mesh counted once, also through shared edges and vertices).  A point on a
 * face normal to x is inside on a face where +x enters the solid and outside
 * on one where it leaves; elsewhere on the surface rounding decides.
 * Returns SPH_E_TOO_LARGE (with *count set) if cap is too small,
 * SPH_E_CAPACITY if one lattice line crosses the mesh more than 1024 times. */
int sph_sample_solid(const double* verts3, int64_t nv, const int32_t* tris3, int64_t nt, const double* xs,
                     int32_t nx, const double* ys, int32_t ny, const double* zs, int32_t nz, const double* rot9,
                     const double* pos3, float* out3, int64_t cap, int64_t* count, int32_t device);

/* Boundary volumes psi for callers that must not allocate device memory.
 * No counterpart in the reference: the reference always runs inside Warp,
 * which allocates freely.  This is for callers that cannot call cudaMalloc —
 * e.g. a host framework whose memory pool owns the device and forbids
 * allocations behind its back, or real-time code that must not allocate after
 * start-up because an allocation can block or fail at any time.  The caller
 * passes device pointers:
 * d_xb3 (nb x 3 floats, boundary positions), d_w_table (params->w_table_size
 * floats, the W table) and d_psi (nb floats, output in input order); it gets
 * the same psi as sph_set_boundary computes.  The library allocates nothing:
 * its scratch is one static device array of at most 24 MiB that every device
 * loading the library keeps until process exit.  Limits: nb <=
 * SPH_NOALLOC_MAX_BOUNDARY (else SPH_E_TOO_LARGE, before any GPU work) and at
 * most SPH_NOALLOC_MAX_CELLS grid cells (a coarser grid is chosen beyond that).
 * Runs on the calling thread's current device, on `stream` (a cudaStream_t,
 * NULL = default stream).  The first call on each device looks up the
 * scratch's device address (cudaGetSymbolAddress) and keeps it: do not use
 * this entry point on a device after cudaDeviceReset.  When params->domain_*
 * is empty the call reads the points' bounding box back to the host and so
 * synchronises `stream`; with a domain it only enqueues work (domain bounds
 * must be finite, else SPH_E_INVALID).  The psi output is complete when
 * `stream` is next synchronised.  All calls share the scratch, which keeps
 * the last call's contents: calls whose GPU work overlaps (other streams or
 * threads) race. */
#define SPH_NOALLOC_MAX_BOUNDARY 262144
#define SPH_NOALLOC_MAX_CELLS 1048576
int sph_boundary_psi_noalloc(const SphParams* params, const float* d_xb3, int64_t nb, const float* d_w_table,
                             float* d_psi, void* stream);

/* ---- Learned pressure warm start (SPH_WARM_MLP) -------------------------
 * No counterpart in the reference, whose solve starts from p = 0
 * (IISPH.py:166-174).  A per-particle MLP 10 -> 64 -> 64 -> 1 (ReLU, BF16
 * tensor-core products, FP32 accumulate) predicts the solve's starting
 * pressure from SPH_MLP_FEATURES dimensionless inputs the neighbour build
 * computes and uses it as the solve's first iterate; the unchanged Jacobi
 * loop (at least 2 iterations, average density error <= eta) still decides
 * convergence.
 * The network is residual on a base taken in FP32 (no BF16 rounding on the
 * skip path): u = max(input 3, input 10), the larger of the previous step's
 * pressure, asinh(p_prev / (rho0 g h)), and the hydrostatic pressure of the
 * fluid column above the particle, asinh(depth / h) (depth = highest fluid
 * particle of the particle's neighbour-grid column (x, z) minus its own y).
 * The prediction is
 *   p = sinh(max(u + min(y * t_scale, SPH_MLP_MAX_RISE), 0)) * rho0 * g * h;
 * the bounded rise keeps one over-predicted particle (which the solve's test,
 * counting only compressed particles, would not see) from being kicked out.
 * Weights travel as one FP32 blob of SPH_MLP_BLOB floats:
 *   mu[11], sd[11]   input standardisation (x - mu) / sd
 *   t_scale          output unit of y
 *   W1[11][64] b1[64] W2[64][64] b2[64] w3[64] b3   (SPH_MLP_PARAMS, W[in][out])
 * sph_get_features gives t = asinh(p / (rho0 g h)) of the converged pressure
 * (pressures span orders of magnitude; asinh keeps them on one scale); the
 * network is trained on the residual t - u.  sph_mlp_train and sph_mlp_eval
 * regress y * t_scale on whatever target array they are given. */
#define SPH_MLP_FEATURES 11
#define SPH_MLP_PARAMS 4993
#define SPH_MLP_BLOB 5016
#define SPH_MLP_MAX_RISE 0.5f

typedef struct SphMlpTrainConfig {
  int32_t epochs;
  int32_t batch;
  float lr, beta1, beta2, eps; /* Adam */
  uint32_t seed;               /* minibatch shuffling */
  int32_t device;
} SphMlpTrainConfig;

/* Install the network used by SPH_WARM_MLP. */
int sph_set_mlp(SphCtx* ctx, const float* blob, int32_t n);
/* Compute the network inputs at every step (needed to collect training data). */
int sph_set_record_features(SphCtx* ctx, int32_t on);
/* After a step: per fluid particle (original order) its SPH_MLP_FEATURES inputs
 * and the training target asinh(p / (rho0 g h)) of its converged pressure. */
int sph_get_features(SphCtx* ctx, float* feat, float* target);
/* After a step with sph_set_record_features(ctx, 1): per fluid particle
 * (original order) the pressure the step's Jacobi solve started from — the
 * iterate that replaces init_pressure (IISPH.py:166-174): the first update_p
 * from p = 0 with SPH_WARM_ZERO, 0.5 p_prev with SPH_WARM_HALF (before the
 * extra Ap_0 pass), and with SPH_WARM_MLP the network's prediction or, after
 * a capped solve with warm_continue, that solve's final pressure. */
int sph_get_solve_start(SphCtx* ctx, float* p);
/* The neighbour grid of scene `scene` (0 for a single scene), for tools that
 * restate per-cell quantities: out[0..2] origin xyz, out[3] 1 / cell size
 * (y, z), out[4] 1 / cell size along x (half cells), out[5..7] cells along
 * x, y, z, out[8] the scene's first global cell id.  Float fields hold the
 * float32 values the kernels use. */
int sph_get_grid(SphCtx* ctx, int32_t scene, double* out9);
/* Train in place: Adam on mean squared error over shuffled minibatches, on the
 * GPU with the library's own forward/backward kernels.  blob supplies mu, sd,
 * t_scale and the initial weights; epoch_loss (epochs floats) may be NULL. */
int sph_mlp_train(const SphMlpTrainConfig* cfg, const float* feat, const float* target, int64_t n, float* blob,
                  float* epoch_loss);
/* Network outputs (units of t_scale) and, with target, the gradient of the mean
 * squared error: grad[SPH_MLP_PARAMS] in blob parameter order, then the loss. */
int sph_mlp_eval(const float* blob, const float* feat, const float* target, int64_t n, int32_t device,
                 float* pred, float* grad);

/* ABI self-description, needs no GPU: out[0] = WPSPH_ABI_VERSION,
 * out[1] = sizeof(SphParams), out[2] = sizeof(SphStepStats). */
int sph_abi_info(int32_t* out, int32_t count);
int64_t sph_num_fluid(const SphCtx* ctx);
int64_t sph_num_boundary(const SphCtx* ctx);
/* The context's cudaStream_t, for event timing by the caller. */
void* sph_stream(SphCtx* ctx);
int sph_synchronize(SphCtx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* WPSPH_H */
