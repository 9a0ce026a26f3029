/*
 * amk.h -- C ABI of the B200-native antimatter-kernel particle path.
 *
 * One shared library (libamk.so, sm_100a) replaces the reference's per-step
 * hot path: the three Coulomb solvers, the Boris push in the Penning-trap
 * field with cyclotron cooling, the annihilation contact search and the
 * energy diagnostics. Particle state lives in HBM as structure-of-arrays
 * (positions and velocities FP64, trap-centred) for the life of a context.
 *
 * Conventions (all functions):
 *   - return AMK_OK (0) or a negative AMK_ERR_* code; nothing throws across
 *     the ABI; amk_last_error() gives a message for the calling thread;
 *   - host buffers are caller-owned and only read/written during the call;
 *   - device buffers are owned by the context; one CUDA stream per context;
 *     a context is not re-entrant (one host thread at a time);
 *   - SI units throughout (m, m/s, kg, C, N, J, s).
 *
 * Reference interfaces replaced (paths inside the antimatter-kernel tree):
 *   ComputeStandardCoulombForces      src/interaction/coulomb_interaction.h:10
 *   ComputeBarnesHutCoulombForces     src/interaction/barnes-hut.h:76
 *   BarnesHutTree                     src/interaction/barnes-hut.h:28-74
 *   ComputeFastMultipoleCoulombForces src/interaction/fast-multipole.h:73
 *   FastMultipoleSolver               src/interaction/fast-multipole.h:46-71
 *   LorentzForce::Run                 src/forces/lorentz.h:15-35
 *   CyclotronCooling::Run             src/forces/cooling.h:16-40
 *   AnnihilationInteraction::Run      src/interaction/annihilation.h:11-20
 *   ComputeTotalEnergy                src/analysis/energy_analysis.h:35
 *   PhysicsParams/InteractionParams/StochasticParams::LoadParams
 *                                     src/params/{physics,interaction,stochastic}_params.h
 */
#ifndef AMK_H_
#define AMK_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define AMK_OK 0
#define AMK_ERR_INVALID (-1)     /* bad argument or configuration            */
#define AMK_ERR_CUDA (-2)        /* CUDA runtime error                       */
#define AMK_ERR_NOMEM (-3)       /* device allocation failed                 */
#define AMK_ERR_STATE (-4)       /* call made in the wrong state             */
#define AMK_ERR_TIMEOUT (-5)     /* a bounded device-side wait gave up       */
#define AMK_ERR_UNSUPPORTED (-6) /* option not built                         */
#define AMK_ERR_LIMIT (-7)       /* size beyond a documented maximum         */
#define AMK_ERR_IO (-8)          /* file could not be read                   */

/* ------------------------------------------------------------ enumerations */
/* Coulomb / energy methods: interaction_params.cc:14-28 ("standard",
 * "barnes-hut", "fast-multipole") plus the tiled all-pairs direct sum. */
#define AMK_METHOD_STANDARD 0
#define AMK_METHOD_BARNES_HUT 1
#define AMK_METHOD_FAST_MULTIPOLE 2
#define AMK_METHOD_ALLPAIRS 3

/* ParticleSpecies, src/agents/particle_species.h:9-17 (same values). */
#define AMK_ANTIPROTON 0
#define AMK_POSITRON 1
#define AMK_ANTIHYDROGEN 2
#define AMK_ELECTRON 3
#define AMK_PROTON 4
#define AMK_ANTIHELIUM 5
#define AMK_MAX_SPECIES 6

/* ------------------------------------------------------------ parameters */
/* Mirrors the params.json keys read by physics_params.cc:42-100,
 * interaction_params.cc:30-47 and stochastic_params.cc:13-24. */
typedef struct amk_params {
  int seed;                     /* "seed"                                  */
  double b0;                    /* "b0" [T]                                */
  double trap_voltage;          /* "trap_voltage" [V]                      */
  double z0;                    /* "z0" [m]                                */
  double rho0;                  /* "rho0" [m]                              */
  double dt;                    /* derived, physics_params.cc:60-74 [s]    */
  long num_steps;               /* "num_steps"                             */
  double bath_temperature;      /* "bath_temperature" [K]                  */
  double cooling_scale;         /* "cooling_scale"                         */
  int cooling_enabled;          /* cooling behaviour attached (default 1)  */
  int coulomb_forces_enabled;   /* "coulomb_forces_enabled"                */
  int coulomb_method;           /* "coulomb_computation_method"            */
  int energy_method;            /* "energy_computation_method"             */
  double cutoff_radius;         /* "cutoff_radius" [m]                     */
  double barnes_hut_theta;      /* "barnes_hut_theta"                      */
  double fast_multipole_order;  /* "fast_multipole_order" (real, truncated) */
  double fast_multipole_theta;  /* "fast_multipole_theta"                  */
  int fmm_learned;              /* learned p=2 correction (no reference key) */
  int annihilation_enabled;     /* "annihilation_enabled"                  */
  double contact_radius;        /* "contact_radius" [m]                    */
  double annihilation_probability; /* "annihilation_probability"          */
  int n_species;                /* entries of "particle_populations"       */
  int species[AMK_MAX_SPECIES];
  long populations[AMK_MAX_SPECIES];
  double temperatures[AMK_MAX_SPECIES]; /* "particle_temperatures" [K]    */
  double cloud_radii[3];        /* "initial_cloud_radii" radius_x/y/z [m] */
  /* learned p=2 FMM correction (no reference keys) */
  long learned_audit_interval;  /* steps between direct-sum audits (0 = never) */
  double learned_error_budget;  /* RMS relative force error allowed by the audit */
  int learned_fallback_order;   /* plain FMM order used after a failed audit */
  long learned_audit_samples;   /* particles checked per audit */
} amk_params;

/* Defaults of the reference's ParamGroups (physics_params.h:21-46,
 * interaction_params.h:28-55, stochastic_params.h:11-29). */
int amk_params_default(amk_params* out);

/* Reads a params.json file with the reference's keys. Missing keys keep the
 * values already in *inout; dt is re-derived as physics_params.cc:60-74 does.
 * Method strings accept "standard", "barnes-hut", "fast-multipole" (and the
 * README spellings "barnes_hut", "fast_multipole", plus "allpairs"). */
int amk_params_load_json(const char* path, amk_params* inout);

/* Validation of physics_params.cc:126-160, interaction_params.cc:71-115 and
 * stochastic_params.cc:35-46. `strict` = 1 keeps the reference's
 * cooling_scale <= 1 rule (physics_params.cc:139). */
int amk_params_validate(const amk_params* p, int strict);

/* dt rule of physics_params.cc:60-74 for a species list. */
double amk_dt_for_species(int n_species, const int* species, double b0);

/* Default mass [kg] and charge [C], particle_species.h:27-46. */
int amk_species_properties(int species, double* mass, double* charge);

/* Characteristic dimension d = sqrt(z0^2/2 + rho0^2/4), penning_trap.cc:15-20. */
double amk_trap_dimension(double z0, double rho0);

/* Perpendicular-energy e-folding time, cooling.cc:16-22. */
double amk_cooling_time(double charge, double mass, double b_mag);

/* ------------------------------------------------------------ context */
typedef struct amk_ctx amk_ctx;

/* Creates a context on CUDA device `device` with its own stream. */
int amk_create(const amk_params* params, int device, amk_ctx** out);
int amk_destroy(amk_ctx* ctx);

/* Last error message of the calling thread (never NULL). */
const char* amk_last_error(void);

/* Replaces the context's stream (a cudaStream_t; NULL = the context's own). */
int amk_set_stream(amk_ctx* ctx, void* cuda_stream);
int amk_get_stream(amk_ctx* ctx, void** cuda_stream);
int amk_synchronize(amk_ctx* ctx);

/* Updates the physics/interaction/stochastic parameters of a live context. */
int amk_set_params(amk_ctx* ctx, const amk_params* params);
int amk_get_params(const amk_ctx* ctx, amk_params* out);

/* ------------------------------------------------------------ particles */
/* Loads n particles from host arrays (positions trap-centred). Mass and
 * charge come from the species defaults; all particles start alive; the
 * first push back-staggers v by dt/2 (lorentz.cc:56-60). */
int amk_set_particles(amk_ctx* ctx, long n, const double* x, const double* y,
                      const double* z, const double* vx, const double* vy,
                      const double* vz, const uint8_t* species);

/* Same, from device pointers already resident on the context's device. */
int amk_set_particles_device(amk_ctx* ctx, long n, const double* x, const double* y,
                             const double* z, const double* vx, const double* vy,
                             const double* vz, const uint8_t* species);

/* Overwrites positions and velocities of the current particle set from host
 * arrays (same n; species, alive flags, step counter and the half-step
 * stagger are kept). For callers that keep the state on the host and hand
 * it to the GPU each step. */
int amk_update_state(amk_ctx* ctx, const double* x, const double* y, const double* z,
                     const double* vx, const double* vy, const double* vz);

/* Overrides per-particle charge and mass (ChargedAntiparticle::SetCharge /
 * SetMass). Either pointer may be NULL. */
int amk_set_charge_mass(amk_ctx* ctx, const double* charge, const double* mass);

/* Host arrays overwrite per-particle state of the context (n entries each):
 * the Coulomb-force slots (ChargedAntiparticle::SetCoulombForce), the stable
 * ids that key the cooling and annihilation random streams (creation order
 * by default; an adapter passes its agents' uids), the alive flags
 * (MarkAnnihilated). amk_set_step_state sets the completed-step counter
 * (the next push and annihilation draw with step + 1) and whether the
 * velocities are already staggered back by dt/2 (LorentzForce's per-agent
 * flag, lorentz.h:34). */
int amk_set_forces(amk_ctx* ctx, const double* fx, const double* fy, const double* fz);
int amk_set_ids(amk_ctx* ctx, const uint32_t* ids);
int amk_set_alive(amk_ctx* ctx, const uint8_t* alive);
int amk_set_step_state(amk_ctx* ctx, long step, int staggered);

/* Builds the reference's initial cloud from the context's parameters
 * (penning_trap.cc:51-160: uniform ellipsoid by rejection sampling with
 * std::default_random_engine(seed), Maxwellian velocities with a fresh
 * std::mt19937(seed) per species) and loads it. */
int amk_init_particles(amk_ctx* ctx);

/* The reference's cloud generators restated on the GPU for large clouds and
 * sweeps (penning_trap.cc:51-160): species in the reference's order,
 * positions uniform in the ellipsoid of radii cloud_radii
 * (AMK_CLOUD_UNIFORM_ELLIPSOID, the reference's shape) or Gaussian with
 * those standard deviations (AMK_CLOUD_GAUSSIAN), Maxwellian velocities per
 * species with the reference's drift removal and sqrt(n/(n-1)) rescale.
 * Draws come from Philox keyed by (seed, particle index), not from the
 * reference's std:: engines (amk_init_particles reproduces those), so the
 * cloud is deterministic and independent of the GPU's scheduling.
 * amk_batch_init_particles generates every instance of a sweep (instance
 * i from params[i], each identical to the same instance generated alone)
 * and sets the batch (amk_batch_set with the implied offsets). */
#define AMK_CLOUD_UNIFORM_ELLIPSOID 0
#define AMK_CLOUD_GAUSSIAN 1
int amk_init_particles_gpu(amk_ctx* ctx, int distribution);
int amk_batch_init_particles(amk_ctx* ctx, int n_inst, const amk_params* params, int distribution);

/* Copies the state back. Any pointer may be NULL. alive[i] = 0 once
 * annihilated. */
int amk_get_particles(amk_ctx* ctx, double* x, double* y, double* z, double* vx,
                      double* vy, double* vz, uint8_t* alive);
int amk_get_particles_device(amk_ctx* ctx, double* x, double* y, double* z, double* vx,
                             double* vy, double* vz, uint8_t* alive);
long amk_num_particles(const amk_ctx* ctx);
long amk_num_alive(amk_ctx* ctx);

/* ------------------------------------------------------------ forces */
/* Each solver writes the Coulomb force on every alive particle into the
 * context's force slot (the agent's coulomb_force_), which the next push
 * consumes and zeroes (lorentz.cc:53,70). Dead or neutral particles get 0. */

/* Cutoff direct sum, coulomb_interaction.cc:23-80 (rc <= 0: zero forces). */
int amk_coulomb_standard(amk_ctx* ctx, double cutoff_radius);
/* Exact all-pairs direct sum (no cutoff), tiled on the GPU. */
int amk_coulomb_allpairs(amk_ctx* ctx);
/* Barnes-Hut, barnes-hut.cc:271-299 (leaf capacity 8). */
int amk_coulomb_barnes_hut(amk_ctx* ctx, double theta);
/* Cartesian FMM, fast-multipole.cc:684-713 (order clamped to [1,8], leaf
 * capacity 32). learned != 0 selects the p=2 far field plus the learned
 * correction (order is then ignored). */
int amk_coulomb_fmm(amk_ctx* ctx, int order, double theta, int learned);
/* Dispatches on the context's coulomb_method (antimatter-kernel.cc:155-160). */
int amk_coulomb(amk_ctx* ctx);
/* Copies the force slot back to the host. */
int amk_get_forces(amk_ctx* ctx, double* fx, double* fy, double* fz);

/* ------------------------------------------------------------ behaviours */
/* LorentzForce::Run then CyclotronCooling::Run for every alive particle
 * (lorentz.cc:37-71, cooling.cc:24-66), fused in one kernel. Cooling noise
 * is Philox4x32-10 keyed by (seed, step, particle id). The push ends a step:
 * it advances the step counter (steps are numbered from 1). */
int amk_push(amk_ctx* ctx);
/* AnnihilationInteraction::Run for every alive particle, deterministic:
 * greedy matching in ascending (owner id, partner id) order over contacts
 * r^2 < contact_radius^2 whose Philox draw u(owner->partner) < p, with the
 * draws keyed by the step of the last push (1 before any push). Returns
 * the number of particles annihilated this call in *marked (may be NULL). */
int amk_annihilate(amk_ctx* ctx, long* marked);
/* One or more full steps: Coulomb (context method) -> push+cooling ->
 * annihilation, as antimatter-kernel.cc:153-162. */
int amk_step(amk_ctx* ctx, int nsteps);
long amk_step_count(const amk_ctx* ctx);

/* ------------------------------------------------------------ energy */
typedef struct amk_energy_out {
  double kinetic;          /* sum 1/2 m v^2 over alive particles        */
  double trap_potential;   /* sum q phi_trap(x)                          */
  double coulomb_potential;/* per the energy method                      */
  double total;
  long num_active;
} amk_energy_out;

/* ComputeTotalEnergy, energy_analysis.cc:84-145. time_centre != 0 averages
 * the potentials with the previous call's (EnergyHistory, :126-142). The
 * Coulomb term uses the context's energy_method: standard = shifted-cutoff
 * pair sum (:16-43), barnes-hut = BH potential walk (:45-69),
 * fast-multipole = FMM energy (:71-81), allpairs = exact pair sum. All
 * reductions are FP64. */
int amk_energy(amk_ctx* ctx, int time_centre, amk_energy_out* out);

/* ------------------------------------------------------------ solver mirrors */
/* Stateless counterparts of the reference's solver classes, on caller
 * buffers (host memory). They use the context only for its device, stream
 * and scratch; the context's particle state is untouched.
 *   BarnesHutTree(theta, leaf_capacity).Build + ComputeForce per source
 *   (self excluded) / ComputePotential: barnes-hut.h:40-44.
 *   FastMultipoleSolver(order, theta, leaf_capacity).Compute: fast-multipole.h:55-64
 * phi / energy outputs may be NULL. phi_i = sum_j q_j / r_ij (no k). */
int amk_solve_allpairs(amk_ctx* ctx, long n, const double* x, const double* y,
                       const double* z, const double* q, double* fx, double* fy,
                       double* fz, double* phi);
int amk_solve_cutoff(amk_ctx* ctx, long n, const double* x, const double* y,
                     const double* z, const double* q, double cutoff_radius, double* fx,
                     double* fy, double* fz);
int amk_solve_barnes_hut(amk_ctx* ctx, long n, const double* x, const double* y,
                         const double* z, const double* q, double theta, long leaf_capacity,
                         double* fx, double* fy, double* fz, double* phi);
int amk_solve_fmm(amk_ctx* ctx, long n, const double* x, const double* y, const double* z,
                  const double* q, int order, double theta, long leaf_capacity,
                  double* fx, double* fy, double* fz, double* energy);

/* Builds the Barnes-Hut octree of the given sources (BarnesHutTree::Build,
 * barnes-hut.cc:38-164) and copies its nodes out in the reference's order
 * and layout: node_f64 holds 12 doubles per node (centre xyz, half size,
 * positive charge, |negative| charge, positive centre xyz, negative centre
 * xyz), node_i64 holds 11 per node (children[8] with -1 for none, begin, end,
 * is_leaf). Returns the node count (BarnesHutTree::NumNodes) or an error. */
long amk_bh_tree_dump(amk_ctx* ctx, long n, const double* x, const double* y, const double* z,
                      const double* q, long leaf_capacity, long max_nodes, double* node_f64,
                      long* node_i64);

/* Arithmetic of the FMM's M2L class products on this context.
 * AMK_FMM_FP64 (default): FP64 tensor cores (mma.m8n8k4) and FP64 per-pair
 * products -- the reference's arithmetic, results within 1e-9 of the
 * reference's FastMultipoleSolver. AMK_FMM_TENSOR: for orders 5 to 7 the
 * products run on the 5th-generation tensor cores with split-BF16 operands
 * (three BF16 terms per operand, six products, FP32 accumulation in tensor
 * memory) and FP32 per-pair products summed in FP64; relative error of an
 * M2L term about 2^-22, below the truncation error of those orders; classes
 * of fewer than 4 pairs are folded by reflection into the class of |v|. The
 * near field (P2P) then runs in FP32 on double-float positions (pair
 * differences exact to FP32 rounding for touching leaves, FP32 offsets from
 * the centre of separated ones, FP64 sums per source leaf). Tree,
 * expansions, L2L and L2P stay FP64. The mode also selects FP32 leaf sums
 * (same double-float differences) in the Barnes-Hut walk, whose opening test
 * and node monopoles stay FP64. */
#define AMK_FMM_FP64 0
#define AMK_FMM_TENSOR 1
int amk_set_fmm_precision(amk_ctx* ctx, int mode);
int amk_get_fmm_precision(const amk_ctx* ctx);

/* Interaction counts of the context's last FMM evaluation: out[0] cells,
 * [1] leaves, [2] M2L pairs, [3] P2P leaf pairs, [4] P2P particle pairs,
 * [5] tree depth, [6] sources, [7] order (the quantities the reference's
 * phases scale with, fast-multipole.cc:484-661); [8] M2L pairs evaluated as
 * class products, [9] displacement classes (summed over pair chunks),
 * [10] pair chunks. n <= 11. */
int amk_fmm_stats(amk_ctx* ctx, long* out, int n);

/* ------------------------------------------------------------ learned correction */
/* No counterpart in the reference. A 35 -> 128 -> 128 -> 128 -> 3 MLP (GELU,
 * BF16 weights, FP32 accumulation) that corrects the p=2 FMM far field.
 * Parameters are FP32 masters, flat: W1[128][35] b1[128] W2[128][128] b2
 * W3[128][128] b3 W4[3][128] b4[3] (row = output unit). Inference runs on
 * the tensor cores (tcgen05.mma, accumulators in tensor memory); training
 * (forward, backward, Adam with beta = 0.9, 0.999) in FP32 on the CUDA cores
 * with the same BF16-rounded weights. Loss: mean squared error. */
int amk_mlp_num_params(void);
int amk_mlp_set_params(amk_ctx* ctx, const float* params, long n);
int amk_mlp_get_params(amk_ctx* ctx, float* params, long n);
/* y[n][3] = MLP(x[n][35]) on the tensor cores (host buffers). */
int amk_mlp_forward(amk_ctx* ctx, const float* x, long n, float* y);
/* Loss and dLoss/dparams of one batch (FP32 path); grad, loss, yhat may be NULL. */
int amk_mlp_gradients(amk_ctx* ctx, const float* x, const float* target, long n, float* grad,
                      float* loss, float* yhat);
/* `steps` Adam steps on consecutive windows of `batch` samples. */
int amk_mlp_train(amk_ctx* ctx, const float* x, const float* target, long n, int steps, long batch,
                  float lr, float* final_loss);

/* Trains the correction on the context's particles: p=2 FMM at theta, the
 * particles of about `sample_leaves` leaves, exact FP64 fields for them, and
 * `steps` Adam steps (batch, lr) on the residual (E_exact - E_p2)/|E_far|.
 * Marks the correction usable and clears a previous fallback. */
int amk_fmm_train_correction(amk_ctx* ctx, double theta, int sample_leaves, int steps, long batch,
                             float lr, float* final_loss, long* samples);
/* RMS relative force error against the exact FP64 sum over `samples` evenly
 * spaced particles, for plain FMM of `order` (learned = 0) or the learned
 * p=2 correction (learned = 1). */
int amk_fmm_audit(amk_ctx* ctx, int order, double theta, int learned, long samples, double* rms);
/* trained: the correction is usable; fallback: an audit failed and the
 * context now runs plain FMM at learned_fallback_order; last_error: the
 * last audit's RMS relative error. */
int amk_fmm_learned_state(amk_ctx* ctx, int* trained, int* fallback, double* last_error);

/* ------------------------------------------------------------ audit and tuning */
/* No counterpart in the reference. RMS and maximum relative error of the
 * context's current forces (as left by the last amk_coulomb* call) against
 * an FP64 exact Coulomb sum (the reference's theta = 0 force) for `samples`
 * evenly spaced alive, charged particles. max_rel may be NULL. */
int amk_force_error(amk_ctx* ctx, long samples, double* rms, double* max_rel);

/* Leaf capacities used by amk_coulomb_fmm / amk_coulomb_barnes_hut and
 * amk_step (defaults 32 and 8, the reference's fast-multipole.h:50 and
 * barnes-hut.h:30). Other values build other trees than the reference's. */
int amk_set_leaf_sizes(amk_ctx* ctx, int fmm_leaf, int bh_leaf);
int amk_get_leaf_sizes(const amk_ctx* ctx, int* fmm_leaf, int* bh_leaf);

typedef struct amk_tune_candidate {
  int method;    /* AMK_METHOD_*                                 */
  int order;     /* FMM order (0 otherwise)                      */
  double theta;  /* FMM / Barnes-Hut opening angle               */
  int leaf;      /* leaf capacity (0 for all-pairs)              */
  double ms;     /* median device time of one force evaluation; -1 = skipped */
  double rms;    /* RMS relative force error vs FP64 exact; -1 = skipped     */
  int meets;     /* rms <= the error budget                      */
} amk_tune_candidate;
#define AMK_TUNE_NO_ALLPAIRS 1
#define AMK_TUNE_NO_FMM 2
#define AMK_TUNE_NO_BARNES_HUT 4
/* Autotuner: on the context's own particles, times (CUDA events, median of
 * 3 after a warm call) and audits (amk_force_error with `samples`) the
 * all-pairs solver, the FMM for orders 4..8 x theta 0.6/0.55/0.5375/0.525/
 * 0.5/0.475/0.45/0.4 x leaf 16/32/64/128/256 (higher orders skipped once a
 * lower one meets the budget; up to 204 candidates with the others) and
 * Barnes-Hut for theta 0.5/0.3/0.2, then sets the context's Coulomb method,
 * order, theta and leaf size to the fastest candidate whose RMS error is
 * <= error_budget. out (max_out entries, may be NULL) receives every
 * candidate; chosen = its index (-1 and AMK_ERR_LIMIT when none meets). */
int amk_autotune(amk_ctx* ctx, double error_budget, long samples, int flags, amk_tune_candidate* out,
                 int max_out, int* n_out, int* chosen);

/* ------------------------------------------------------------ batched sweep */
/* No counterpart in the reference, which runs one instance per process
 * (antimatter-kernel.cc:153-162); a parameter sweep is many such runs. A
 * batch splits the context's particle set into up to AMK_BATCH_MAX_INSTANCES
 * independent instances: instance i owns particles [offsets[i],
 * offsets[i+1]) (offsets[0] = 0, offsets[n_inst] = particle count) and
 * steps with params[i] (trap, dt, cooling, annihilation, Coulomb method;
 * seed per instance). Each instance gives the results it gives alone in a
 * context of its own (random streams use the index within the instance).
 * Setting a batch renumbers the particle ids within each instance; after it
 * the single-instance amk_push / amk_annihilate / amk_step refuse the context
 * (AMK_ERR_STATE) until amk_set_particles or amk_init_particles loads a new
 * set. Per-instance learned FMM is not available (AMK_ERR_UNSUPPORTED). */
#define AMK_BATCH_MAX_INSTANCES 512
int amk_batch_set(amk_ctx* ctx, int n_inst, const amk_params* params, const long* offsets);
/* nsteps steps of every instance. All-pairs instances share one persistent
 * launch; cutoff, Barnes-Hut and FMM instances run their solver on their
 * own slice. graph_chunk > 0 captures chunks of that many steps in a CUDA
 * graph and replays them when no instance uses Barnes-Hut or the FMM (whose
 * tree builds synchronise with the host). serial != 0 steps the instances
 * one at a time with the single-instance kernels instead (the same results
 * up to FP32 rounding of the all-pairs sums; the comparison baseline). */
int amk_batch_step(amk_ctx* ctx, int nsteps, int graph_chunk, int serial);
/* The Coulomb forces of every instance for the current positions (the first
 * phase of a batched step), readable with amk_get_forces; the next step
 * recomputes them. */
int amk_batch_coulomb(amk_ctx* ctx);
/* overflow: 1 if a step inside a CUDA graph chunk found more annihilation
 * contacts than the contact buffer held (those beyond were dropped; that
 * amk_batch_step call returned AMK_ERR_LIMIT). Steps outside graphs read the
 * contact count back and enlarge the buffer instead; a graph is captured with
 * twice the largest count seen so far. alive_counts (n_inst entries, may be
 * NULL): live particles per instance. */
int amk_batch_status(amk_ctx* ctx, int* overflow, long* alive_counts);
/* Batch autotuner: chooses each instance's Coulomb method by measurement
 * under an RMS force-error budget (audited against the FP64 exact sum with
 * `samples` particles): the batched all-pairs launch is timed and its cost
 * split over instances by N_i^2; FMM configurations (order 4/6/8, theta
 * 0.5/0.35, leaf 32/64) are timed and audited on the largest instance, and
 * the fastest that meets the budget replaces all-pairs on each instance,
 * largest first, where it is faster there. Rebuilds the batch; methods_out
 * (n_inst entries, may be NULL) receives the chosen AMK_METHOD_* (-1 for
 * instances without Coulomb forces). */
int amk_batch_autotune(amk_ctx* ctx, double error_budget, long samples, int* methods_out);
/* amk_energy for every instance of the batch: out[i] (n_inst entries) with
 * instance i's kinetic, trap and Coulomb energies under its own parameters
 * and energy method, and its own time-centring history. */
int amk_batch_energy(amk_ctx* ctx, int time_centre, amk_energy_out* out);
/* n_instances, all-pairs work units (instance, 256-target block) and
 * whether the batch can run as CUDA graphs. */
int amk_batch_info(const amk_ctx* ctx, long* n_instances, long* work_units, int* graphable);

/* ------------------------------------------------------------ checkpoint / export */
/* Checkpoint/resume, in place of BioDynaMo's backup and restore of the
 * simulation (the reference runs inside BioDynaMo, which provides them;
 * bdm.toml:1-4). amk_checkpoint_save writes the context's parameters,
 * step counter, Boris back-stagger flag, energy time-centring history,
 * learned-correction state and network, the all-pairs Morton order and the
 * full particle state (x, v, force slots, q, m, species, alive, ids) to
 * `path` (written to path.tmp, then renamed), with an FNV-1a checksum;
 * amk_checkpoint_load replaces the context's parameters and state with the
 * file's, so the restored context continues bit for bit like the saved one.
 * A context holding a batch is refused (AMK_ERR_STATE). Corrupt, truncated
 * or foreign files: AMK_ERR_INVALID. amk_checkpoint_info reads a file's
 * header (particles, step, parameters) without a GPU. */
int amk_checkpoint_save(amk_ctx* ctx, const char* path);
int amk_checkpoint_load(amk_ctx* ctx, const char* path);
int amk_checkpoint_info(const char* path, long* n, long* step, amk_params* params);
/* Headless particle export in place of BioDynaMo's ParaView export
 * (bdm.toml:6-13: ChargedAntiparticle agents, additional data member
 * species_id): a VTK XML UnstructuredGrid (.vtu) of the live particles as
 * vertex cells, point data species_id (Int32), velocity (Float64 x 3) and
 * id (UInt32), the simulated time (step * dt) as field data TimeValue;
 * binary != 0 appends the arrays as raw little-endian data, 0 writes ASCII.
 * amk_write_vtu does the same from host arrays (alive and ids may be NULL)
 * without a GPU; amk_write_pvd writes a ParaView collection of n files. */
int amk_export_vtk(amk_ctx* ctx, const char* path, int binary);
int amk_write_vtu(const char* path, long n, const double* x, const double* y, const double* z,
                  const double* vx, const double* vy, const double* vz, const uint8_t* species,
                  const uint8_t* alive, const uint32_t* ids, double time, int binary);
int amk_write_pvd(const char* path, long n, const char* const* files, const double* times);

/* ------------------------------------------------------------ allocation-free */
/* No counterpart in the reference. The cutoff Coulomb solver (same results
 * as amk_coulomb_standard / amk_solve_cutoff) for callers that cannot let a
 * library allocate device memory -- a host code whose device memory is
 * owned by its own pool allocator, or a per-step loop that cannot take the
 * device-wide synchronisation of cudaMalloc/cudaFree. It allocates nothing:
 * its scratch is one static device array (about 2.4 MB) that every GPU
 * loading the library holds until exit. All pointers are device arrays on
 * the current device; alive may be NULL (all alive); the work is queued on
 * `stream` (a cudaStream_t, NULL = legacy default stream).
 * n <= AMK_NOALLOC_MAX_PARTICLES, else AMK_ERR_LIMIT. The first call on a
 * device looks up the array's address; make it during set-up, before any
 * stream capture. Calls share the array: calls that overlap on the GPU
 * race. Every one of the n force entries is written: particles that are
 * dead (alive[i] == 0), neutral, or at a non-finite position get a zero
 * force (the reference's drivers leave an annihilated agent's slot
 * untouched instead). cutoff_radius <= 0 writes zero forces for all. */
#define AMK_NOALLOC_MAX_PARTICLES 65536
int amk_coulomb_standard_noalloc(const double* x, const double* y, const double* z,
                                 const double* q, const uint8_t* alive, long n,
                                 double cutoff_radius, double* fx, double* fy, double* fz,
                                 void* stream);

/* ------------------------------------------------------------ profiling */
/* Per-phase device time (CUDA events on the context stream) accumulated
 * since the last reset, in ms. Phases: see AMK_PHASE_*. */
#define AMK_PHASE_STAGE 0
#define AMK_PHASE_ALLPAIRS 1
#define AMK_PHASE_CUTOFF 2
#define AMK_PHASE_SORT 3
#define AMK_PHASE_TREE 4
#define AMK_PHASE_BH_WALK 5
#define AMK_PHASE_FMM_UP 6
#define AMK_PHASE_FMM_LISTS 7
#define AMK_PHASE_FMM_M2L 8
#define AMK_PHASE_FMM_DOWN 9
#define AMK_PHASE_FMM_P2P 10
#define AMK_PHASE_MLP 11
#define AMK_PHASE_PUSH 12
#define AMK_PHASE_ANNIHILATION 13
#define AMK_PHASE_ENERGY 14
#define AMK_PHASE_FMM_M2L_PRODUCTS 15 /* the class-product kernels inside FMM_M2L */
#define AMK_PHASE_FMM_NEAR 16         /* FP32 near-field pair kernel (tensor mode, its own stream) */
#define AMK_NUM_PHASES 17
int amk_set_profiling(amk_ctx* ctx, int enabled);
int amk_phase_times(amk_ctx* ctx, double* ms_out, long* launches_out, int n);
int amk_reset_phase_times(amk_ctx* ctx);
/* Number of kernels this library launched on the context since creation. */
long amk_kernel_launches(const amk_ctx* ctx);
/* FP32 FMA-pipe throughput of the context's device in TFLOP/s (2 flops per
 * FFMA), measured by a short probe kernel on the context stream: the
 * roofline denominator of the FP32-bound pair kernels. */
int amk_measure_fp32_peak(amk_ctx* ctx, double* tflops, double* ms);
/* FP64 tensor-pipe throughput (mma.m8n8k4 with FP64 operands, 512 flops
 * per warp instruction) in TFLOP/s: the roofline denominator of the FMM's
 * M2L class products. */
int amk_measure_fp64_peak(amk_ctx* ctx, double* tflops, double* ms);

#ifdef __cplusplus
}
#endif
#endif /* AMK_H_ */
