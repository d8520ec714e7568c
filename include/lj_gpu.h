/*
 * lj_gpu.h -- C ABI of the B200 engine for lennard-jonesium's NVE hot path.
 *
 * Every entry point is plain C: opaque context pointer, plain pointers and
 * sizes, int status codes.  All host arrays are borrowed for the duration of
 * the call only.  A context owns its device buffers and one CUDA stream; use
 * one context per host thread (the reference runs one simulation per thread,
 * src/cpp/lennardjonesium/api/simulation_pool.cpp:35-42).  No entry point keeps
 * global mutable state except where a comment says otherwise.
 *
 * Per-atom host arrays use the reference's SystemState layout when stride is 4:
 * Eigen::Matrix4Xd column-major, (x0, y0, z0, w0, x1, ...), with w ignored on
 * input and written as 0 on output (physics/system_state.hpp:85-95).  stride 3
 * packs (x, y, z) per atom.
 *
 * Reference interfaces replaced (paths relative to the reference checkout):
 *   engine::Integrator / VelocityVerletIntegrator::operator()
 *       src/cpp/lennardjonesium/engine/integrator.hpp:34-102, integrator.cpp:62-88
 *   engine::ShortRangeForceCalculation::operator()
 *       src/cpp/lennardjonesium/engine/force_calculation.hpp:63-79, force_calculation.cpp:46-71
 *   engine::CellListParticlePairFilter::pairs
 *       src/cpp/lennardjonesium/engine/particle_pair_filter.cpp:132-192
 *   engine::PeriodicBoundaryCondition::operator()
 *       src/cpp/lennardjonesium/engine/boundary_condition.cpp:37-50
 *   physics::LennardJonesForce::compute
 *       src/cpp/lennardjonesium/physics/lennard_jones_force.cpp:76-128
 *   physics::ThermodynamicMeasurement::operator()
 *       src/cpp/lennardjonesium/physics/measurements.hpp:59-70
 *   physics::set_temperature
 *       src/cpp/lennardjonesium/physics/transformations.cpp:94-116
 */
#ifndef LJ_GPU_H
#define LJ_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference reports misuse through assert() only
 * (e.g. force_calculation.cpp:43, particle_pair_filter.cpp:61-64,
 * lennard_jones_force.cpp:45); here each of those conditions returns LJ_ERR_ARG. */
#define LJ_OK 0
#define LJ_ERR_ARG 1        /* invalid argument (bad size, box below cutoff, null pointer) */
#define LJ_ERR_CUDA 2       /* a CUDA call failed; lj_gpu_last_error() has the message */
#define LJ_ERR_NONFINITE 3  /* a non-finite energy or virial appeared during a step */
#define LJ_ERR_TIMEOUT 4    /* a bounded device-side loop reached its bound (lj_batch_step) */
#define LJ_ERR_CAPACITY 5   /* a neighbour list overflowed its capacity; results are invalid */

/* Arithmetic of the pair kernel. */
#define LJ_PRECISION_FP64 0   /* the drop-in: FP64 throughout */
#define LJ_PRECISION_MIXED 1  /* FP32 pair arithmetic; FP64 accumulation, integration, sums */

/* Pair force.  LJ is physics::LennardJonesForce (quadratic-spline truncation,
 * eps = sigma = 1).  CONSTANT is the reference's test mock
 * tests/cpp/mock/constant_short_range_force.cpp:31-59 (used for its known
 * answers).  NONE means the integrator carries no force calculation, as an
 * Integrator built without a ShortRangeForce (integrator.cpp:78-79). */
#define LJ_FORCE_NONE 0
#define LJ_FORCE_LJ 1
#define LJ_FORCE_CONSTANT 2

typedef struct lj_params {
    int particle_count;      /* N >= 1 */
    double box[3];           /* periodic box edge lengths (tools::BoundingBox) */
    double cutoff_distance;  /* rc; each box edge must be >= rc (particle_pair_filter.cpp:61-64) */
    double time_delta;       /* dt */
    int precision;           /* LJ_PRECISION_* */
    int force_kind;          /* LJ_FORCE_* */
    double force_strength;   /* LJ_FORCE_CONSTANT only */
    int periodic;            /* 1: PeriodicBoundaryCondition each step; 0: none (LJ_FORCE_NONE only) */
    int device;              /* CUDA device ordinal */
    double skin;             /* Verlet-list skin; < 0 selects the default (0.3) */
    int neighbor_capacity;   /* list entries per atom; 0 selects a density-based default */
    int force_block;         /* atoms per block of the pair kernel: 64, 128 or 256; 0 selects 128 */
    /* Mixed path: 0 adds FP32 sums of 8 consecutive pair forces (and V, W)
     * into the FP64 per-atom accumulators; 1 adds every pair's FP32 force, V
     * and W in FP64 (no FP32 summation; slower). */
    int mixed_per_pair;
} lj_params;

/* One ThermodynamicMeasurement::Result (physics/measurements.hpp:42-56). */
typedef struct lj_thermo {
    double time;
    double kinetic_energy;
    double potential_energy;
    double total_energy;
    double virial;
    double temperature;
    double mean_square_displacement;
} lj_thermo;

/* One physics::ThermodynamicAnalyzer result (physics/analyzers.cpp:44-159):
 * window means of T and TE, pressure rho (<T> + <W> / 3N), the
 * microcanonical specific heat from the variance of T, and the diffusion
 * coefficient from the MSD-vs-time slope. */
typedef struct lj_observation {
    double temperature;
    double density;
    double total_energy;
    double pressure;
    double specific_heat;
    double diffusion_coefficient;
} lj_observation;

/* Counters describing the work done so far (for tests and tuning). */
typedef struct lj_stats {
    long long steps;           /* velocity-Verlet steps taken */
    long long list_builds;     /* neighbour-list rebuilds (cell binning + list) */
    int neighbor_capacity;     /* list entries per atom */
    int list_cells[3];         /* cell grid used for list builds */
    int max_neighbors;         /* largest list seen at the last build */
    int small_box;             /* 1: explicit lattice images, rebuilt every step */
    double skin;               /* skin in use (0 in small-box mode) */
    long long kernel_launches; /* kernels this context has launched */
} lj_stats;

typedef struct lj_ctx lj_ctx;

/* Fill *p with the defaults of the reference's Configuration
 * (api/configuration.hpp: rc 2.5, dt 0.005) plus FP64, LJ, periodic, device 0. */
void lj_gpu_default_params(lj_params* p);

/* Create a context with zeroed state (SystemState(N), system_state.cpp:29-37). */
int lj_gpu_create(const lj_params* params, lj_ctx** out);
int lj_gpu_destroy(lj_ctx* ctx);

/* Last error message of this context (static storage owned by the context). */
const char* lj_gpu_last_error(const lj_ctx* ctx);
const char* lj_gpu_status_string(int status);

/* Replace the whole state.  x, v, disp, F: N atoms each at `stride` doubles
 * (3 or 4); any of v, disp, F may be NULL for zeros.  time, pe, virial are the
 * SystemState scalars. */
int lj_gpu_upload_state(lj_ctx* ctx, const double* x, const double* v, const double* disp,
                        const double* F, int stride, double time, double pe, double virial);

/* Copy the state out in atom-id order; NULL outputs are skipped. */
int lj_gpu_download_state(lj_ctx* ctx, double* x, double* v, double* disp, double* F, int stride,
                          double* time, double* pe, double* virial);

/* ShortRangeForceCalculation::operator(): clear F, PE, W and recompute them
 * from the current positions.  pe, virial may be NULL. */
int lj_gpu_compute_forces(lj_ctx* ctx, double* pe, double* virial);

/* Integrator::operator()(nsteps) followed, after every step, by a
 * ThermodynamicMeasurement: out (may be NULL) receives nsteps records. */
int lj_gpu_step(lj_ctx* ctx, int nsteps, lj_thermo* out);

/* Instantaneous ThermodynamicMeasurement of the current state. */
int lj_gpu_measure(lj_ctx* ctx, lj_thermo* out);

/* Multiply every velocity by factor. */
int lj_gpu_scale_velocities(lj_ctx* ctx, double factor);

/* physics::set_temperature(target): v *= sqrt(target / T) with T measured from
 * the current velocities; *measured (may be NULL) receives that T. */
int lj_gpu_set_temperature(lj_ctx* ctx, double target, double* measured);

/* The reference's cell binning of the current positions, for bit-exact checks
 * (particle_pair_filter.cpp:141-154, cell_list_array.cpp:34-52):
 *   shape[3]        floor(L / rc) per axis
 *   cell_of[N]      flat cell index (x-major) of each atom id
 *   offsets[nc+1]   exclusive prefix of the per-cell counts
 *   members[N]      atom ids, cell-major, ascending within each cell
 * Any output may be NULL; offsets needs shape[0]*shape[1]*shape[2]+1 ints
 * (call once with offsets NULL to learn the shape). */
int lj_gpu_debug_cells(lj_ctx* ctx, int* shape, int* cell_of, int* offsets, int* members);

/* The pair set the force kernel used for the current positions: every
 * unordered pair within the cutoff once, as (i < j by atom id, image code,
 * r^2) with image code 9*(ix+1)+3*(iy+1)+(iz+1) and separation
 * (x_i - x_j) - image * L.  Writes at most cap entries (in no particular
 * order) and returns the total count, or a negative status. */
long long lj_gpu_debug_pairs(lj_ctx* ctx, long long cap, int* i, int* j, int* image, double* r2);

/* Radial distribution histogram of the current positions: ordered pairs
 * (i != j) at minimum-image distance r < rmax in bin floor(r * nbins / rmax).
 * rmax must be <= min(L) / 2.  hist receives nbins counts.  (New: the reference
 * has no RDF.) */
int lj_gpu_rdf(lj_ctx* ctx, int nbins, double rmax, unsigned long long* hist);

/* The RDF sampled along a run without host round trips (new, like lj_gpu_rdf):
 * lj_gpu_rdf_accumulate enqueues one sample of the current positions on the
 * context's stream, adding its counts to a device-resident histogram, and
 * returns without waiting; the cell-list scratch is allocated on the first
 * sample and kept, so later samples allocate nothing.  Every sample of one
 * accumulation must use the same nbins and rmax (LJ_ERR_ARG otherwise).
 * lj_gpu_rdf_read waits for the stream and copies the summed counts (nbins of
 * the accumulation; hist may be NULL) and the number of samples (may be NULL).
 * lj_gpu_rdf_reset starts a new accumulation. */
int lj_gpu_rdf_accumulate(lj_ctx* ctx, int nbins, double rmax);
int lj_gpu_rdf_read(lj_ctx* ctx, unsigned long long* hist, long long* samples);
int lj_gpu_rdf_reset(lj_ctx* ctx);

int lj_gpu_get_stats(const lj_ctx* ctx, lj_stats* out);

/* ThermodynamicAnalyzer over the last sample_size step records, computed on
 * the device from the context's record ring without copying the records:
 * 2 <= sample_size <= 1024 (the ring) and <= the steps taken.  density is the
 * system's rho (the analyzer's SystemParameters). */
int lj_gpu_window_stats(lj_ctx* ctx, int sample_size, double density, lj_observation* out);

/* The same analysis on the host over n records (oldest first), in the
 * reference's summation order: the restatement the control protocol uses. */
int lj_window_stats_host(const lj_thermo* records, int n, int particle_count, double density, lj_observation* out);

/* Trajectory stream: the trajectory output the reference leaves as a TODO
 * (control/simulation_controller.hpp:47-50), in the format of its snapshot
 * file (output/sinks.cpp:162-204: two header rows, then one row
 * "TimeStep,ParticleID,x,y,z,vx,vy,vz,fx,fy,fz" per atom in id order).
 * After lj_gpu_trajectory_open, whenever lj_gpu_step or lj_gpu_step_async
 * completes a step whose count (steps this context has taken) is a multiple
 * of `every`, that state's frame is copied to pinned host memory on the
 * context's stream and written by a background thread while the GPU runs on
 * (two frames in flight at most; frames above 32 768 atoms are formatted in
 * blocks on up to 16 short-lived threads and written in row order).  lj_gpu_trajectory_close waits for every
 * frame, closes the file and reports how many frames it holds (may be NULL).
 * lj_gpu_destroy closes an open trajectory. */
int lj_gpu_trajectory_open(lj_ctx* ctx, const char* path, int every);
int lj_gpu_trajectory_close(lj_ctx* ctx, long long* frames);

/* The context's CUDA stream (a cudaStream_t), for callers that time or order
 * work against it (e.g. torch.cuda.ExternalStream). */
void* lj_gpu_stream(lj_ctx* ctx);

/* Enqueue nsteps steps without waiting and without copying records back (the
 * per-step records stay in the device ring).  lj_gpu_synchronize() waits and
 * reports any capacity or non-finite error raised meanwhile. */
int lj_gpu_step_async(lj_ctx* ctx, int nsteps);
int lj_gpu_synchronize(lj_ctx* ctx);

/* Device time of each phase of the step, accumulated over nsteps real steps
 * with CUDA events recorded between the phases on the context's stream.  The
 * host reads the rebuild criterion after each kick/drift (one synchronisation
 * per step; that wait is part of no phase) and launches the rebuild chain
 * only when it holds, as one graph launch (its kernels back to back, as
 * inside the step graphs). */
typedef struct lj_phase_times {
    double kick_drift_ms;  /* first half kick, drift, wrap, displacement check */
    double rebuild_ms;     /* cell binning + neighbour list, launched only on the steps whose
                              rebuild criterion holds (as in the step graphs) */
    double force_ms;       /* pair force + second kick + partial sums */
    double finalize_ms;    /* fixed-order reduction and record */
    long long steps;
    long long rebuilds;
} lj_phase_times;
int lj_gpu_step_timed(lj_ctx* ctx, int nsteps, lj_phase_times* out);

/* Project autotuner: times `steps` steps of the system described by base and
 * the state (x, v; N x stride doubles) for each candidate skin (0.15 to 0.7;
 * it sets the list-cell edge rc + skin and the rebuild frequency) and
 * pair-kernel block size (atoms
 * per block: 64, 128, 256), each in a fresh context from the same
 * state, and writes the fastest parameters to *best (and its ms per step). */
int lj_gpu_autotune(const lj_params* base, const double* x, const double* v, int stride, int steps,
                    lj_params* best, double* best_ms_per_step);

/* Measured FMA throughput of the CUDA-core FP64 and FP32 pipes of a device
 * (TFLOP/s, 2 flops per FMA): the roofline denominators of the pair kernels. */
int lj_gpu_fma_peaks(int device, double* fp64_tflops, double* fp32_tflops);

/* Allocation-free radial distribution histogram.  No counterpart in the
 * reference (it has no RDF, and it never runs on a GPU).
 *
 * For callers that may not call cudaMalloc -- an application whose GPU memory
 * belongs to its own pool allocator, or a per-step analysis hook in a loop
 * that cannot afford cudaMalloc's latency and implicit synchronisation.  The
 * caller passes device buffers it already owns:
 *   pos   device, N x 4 doubles (SystemState layout), 16-byte aligned
 *   hist  device, nbins unsigned 64-bit counts (overwritten)
 *   box   host, 3 edge lengths; rmax <= min(box) / 2
 *   stream  cudaStream_t to run on (NULL: the legacy default stream)
 *   pos must be 16-byte aligned and hist 8-byte aligned (LJ_ERR_ARG otherwise).
 * The work is enqueued on the stream and the call returns without waiting.
 * Counts are those of lj_gpu_rdf.  Limits: N <= 131072 and nbins <= 12288;
 * larger inputs return LJ_ERR_ARG.  The cell list has at most 32768 cells:
 * a box that holds more cells of edge rmax gets coarser cells (same counts,
 * more candidate pairs).
 *
 * Scratch is one fixed device array inside this library (about 5.3 MB, held on
 * every GPU that loads the library until the process exits).  The first call
 * on a device looks up that array's device address (cudaGetSymbolAddress) and
 * caches it, so make the first call on each device before any stream capture;
 * a device reset (cudaDeviceReset) may move the array and invalidates the
 * cached address, so do not call this after resetting a device.  Calls share
 * the array: calls whose GPU work overlaps (other streams, other threads) race
 * and must be serialised by the caller. */
int lj_gpu_rdf_noalloc(const double* pos, int N, const double* box, int nbins, double rmax,
                       unsigned long long* hist, void* stream);

/* engine::InitialCondition (engine/initial_condition.cpp:49-104,
 * tools/cubic_lattice.cpp:38-86): FCC positions and libstdc++-seeded
 * Maxwell-Boltzmann velocities with zero momentum and angular momentum,
 * rescaled to T.  Host only (no GPU needed).  x, v: N x 4 doubles;
 * *side receives the cubic box edge. */
int lj_initial_condition(int N, double temperature, double density, unsigned seed, double* x, double* v,
                         double* side);

/* ------------------------------------------------------------------------
 * Whole simulations: api::Simulation::run (api/simulation.cpp:72-117) with the
 * control protocol of control::SimulationController
 * (control/simulation_controller.cpp:39-146), the equilibration and
 * observation phases (control/simulation_phase.cpp:40-135), the analyzers
 * (physics/analyzers.cpp:44-159) and the four output files in the formats of
 * output/sinks.cpp:40-204.  Fields mirror api::Configuration
 * (api/configuration.hpp:35-102).
 * ------------------------------------------------------------------------ */
typedef struct lj_sim_config {
    double temperature, density;
    int particle_count;
    unsigned random_seed;
    double cutoff_distance, time_delta;
    const char* eq_name;
    double eq_tolerance;
    int eq_sample_size, eq_adjustment_interval, eq_steady_state_time, eq_timeout;
    const char* ob_name;
    double ob_tolerance;
    int ob_sample_size, ob_observation_interval, ob_observation_count;
    const char* event_log;
    const char* thermodynamic_log;
    const char* observation_log;
    const char* snapshot_log;
    int precision;  /* LJ_PRECISION_* */
    int device;
} lj_sim_config;

typedef struct lj_sim_result {
    long long time_steps;
    int outcome;       /* 0 completed, 1 aborted in equilibration, 2 aborted in observation */
    int observations;
    double seconds;
} lj_sim_result;

/* Run one simulation to completion, writing the four files; echo != 0 also
 * prints each event line to stdout as it happens (SimulationBuffer,
 * api/simulation_buffer.cpp:35-58).  Thread-safe across distinct calls (each
 * owns its context), as the reference's SimulationPool runs one per thread. */
int lj_sim_run(const lj_sim_config* cfg, int echo, lj_sim_result* result);

/* A whole sweep on one batched engine (lj_batch_*): n configurations sharing
 * cutoff and time step, each with its own control protocol and four files,
 * all systems stepping together in chunks that end at the earliest step at
 * which any running simulation can act.  results (may be NULL) receives n
 * entries.  The batched form of run_sweep. */
int lj_sim_run_batch(const lj_sim_config* cfgs, int n, int echo, lj_sim_result* results);

/* The number format of the CSV files (fmt's "{}" for a double, as used by
 * output/sinks.cpp:116-204): shortest round-trip digits, fixed notation for
 * decimal exponents in [-4, 16), otherwise d.ddde+XX.  Writes a NUL-terminated
 * string of at most cap bytes. */
int lj_format_double(double v, char* out, int cap);

/* ShortRangeForce::potential / virial / force along z (physics/forces.hpp:80-84)
 * of physics::LennardJonesForce: out = {V, W, F_z} at separation r (host only). */
int lj_pair_along_z(double cutoff, double r, double* out);

/* ------------------------------------------------------------------------
 * Batched systems: many independent systems of uneven size advanced together,
 * one kernel launch (and one CUDA graph per chunk of steps) for all of them,
 * over a packed system table.  Replaces, for a sweep, the reference's
 * SimulationPool of one-simulation-per-thread workers
 * (api/simulation_pool.cpp:35-101) driven by run_sweep
 * (src/python/lennardjonesium/orchestration/run_sweep.py:37-139).  Each system
 * evolves exactly as it would alone through lj_gpu_* (FP64, LJ force,
 * periodic); every box edge must be at least 3 * cutoff.
 * ------------------------------------------------------------------------ */
typedef struct lj_batch_system {
    int particle_count;
    double box[3];
    double time_delta;
    double skin;  /* < 0: the default rule of lj_gpu_create */
} lj_batch_system;

typedef struct lj_batch lj_batch;

int lj_batch_create(const lj_batch_system* systems, int nsys, double cutoff, int device, lj_batch** out);
int lj_batch_destroy(lj_batch* batch);
const char* lj_batch_last_error(const lj_batch* batch);
/* Replace one system's state: positions and velocities (N x stride doubles,
 * v may be NULL); displacements, forces, time and energies restart at zero. */
int lj_batch_upload_system(lj_batch* batch, int sys, const double* x, const double* v, int stride);
int lj_batch_download_system(lj_batch* batch, int sys, double* x, double* v, double* F, int stride);
/* An inactive system is frozen: its atoms are not integrated and it takes no steps. */
int lj_batch_set_active(lj_batch* batch, int sys, int active);
/* nsteps steps of every active system; out (may be NULL) receives nsteps x nsys
 * records, step-major (inactive systems' entries are not written).  The steps
 * run as one CUDA-graph launch per chunk of up to 256 steps: a device-side
 * loop over 8-step bodies (each step's rebuild chain behind a conditional
 * node), plus single launches for the last nsteps mod 8 steps.  The loop is
 * bounded: a launch that reaches its iteration bound before its step count
 * stops there and the call returns LJ_ERR_TIMEOUT (the systems are then short
 * of the requested steps). */
int lj_batch_step(lj_batch* batch, int nsteps, lj_thermo* out);
/* Atoms per block of the batch's pair kernel: 64, 128 (the default) or 256.
 * With the same block size (lj_params.force_block) and skin, a batched system
 * evolves bit for bit as it does alone. */
int lj_batch_set_force_block(lj_batch* batch, int force_block);

/* List cells per block of the batch's list build (one warp per cell): 2, 4
 * (the default) or 8.  The lists do not depend on it. */
int lj_batch_set_list_tile(lj_batch* batch, int cells);

/* Batch autotuner (the batched counterpart of lj_gpu_autotune): times `steps`
 * steps of the whole batch for every candidate Verlet skin (0.2, 0.3, 0.4, 0.5,
 * each clipped by the box as in lj_gpu_create), pair-kernel block size (64,
 * 128, 256) and list-build tile (2, 4, 8 cells per block), each in a fresh
 * batch from the state x, v (every system's atoms in table order, stride
 * doubles per atom; v may be NULL), and writes the fastest to *best.  The
 * pair kernel runs one atom per thread in every candidate. */
typedef struct lj_batch_tuning {
    double skin;
    int force_block;
    int list_cells_per_block;
    double ms_per_step;
} lj_batch_tuning;
int lj_batch_autotune(const lj_batch_system* systems, int nsys, double cutoff, int device, const double* x,
                      const double* v, int stride, int steps, lj_batch_tuning* best);

/* The iteration bound of a chunk launch: 0 (the default) bounds it at the
 * iterations the chunk needs; a positive limit overrides that, and a limit
 * below a chunk's iterations makes its launch stop with LJ_ERR_TIMEOUT (the
 * way the bound is tested). */
int lj_batch_set_iteration_limit(lj_batch* batch, int limit);
/* Instantaneous measurement of every system: out receives nsys records. */
int lj_batch_measure(lj_batch* batch, lj_thermo* out);
/* physics::set_temperature for one system (transformations.cpp:94-116). */
int lj_batch_set_temperature(lj_batch* batch, int sys, double target, double* measured);
/* ThermodynamicAnalyzer of every system over the last sample_size batch steps
 * (2 <= sample_size <= 256, the batch's record ring), on the device, one block
 * per system: density[nsys] in, out[nsys] receives each system's result.  A
 * system inactive during part of the window keeps its older records there. */
int lj_batch_window_stats(lj_batch* batch, int sample_size, const double* density, lj_observation* out);
/* Totals for tests and tuning: atoms, neighbour-list builds per system, direct kernel launches. */
int lj_batch_info(const lj_batch* batch, int* total_atoms, long long* builds_per_system, long long* kernel_launches);

/* ------------------------------------------------------------------------
 * Differentiable NVE: velocity Verlet (integrator.cpp:62-88) over the LJ
 * spline generalised to an energy scale epsilon and a length scale sigma
 * (lennard_jones_force.cpp:68-121 is the case epsilon = sigma = 1; the cutoff
 * is cutoff_sigma * sigma), FP64, with a hand-written discrete adjoint.
 * The outputs are the time averages over steps 1..M of the total potential
 * energy and of the virial pressure rho (T + W / 3N) (physics/analyzers.cpp:73-75).
 * The backward pass runs the reverse velocity-Verlet sweep with one force
 * Hessian-vector product per step, recomputing each segment of
 * checkpoint_every steps from a stored checkpoint, and returns the exact
 * gradient of w_pe * PE_avg + w_p * P_avg with respect to the initial
 * positions and velocities, epsilon and sigma.  There is no reference
 * counterpart: the reference has no derivatives.  Every box edge must hold
 * at least 3 cells of edge cutoff_sigma * sigma.
 * ------------------------------------------------------------------------ */
typedef struct lj_adj_params {
    int particle_count;
    double box[3];
    double time_delta;
    int steps;            /* M >= 1 */
    int checkpoint_every; /* k >= 1: states kept every k steps, segments recomputed */
    double epsilon;
    double sigma;
    double cutoff_sigma;  /* cutoff in units of sigma (2.5 in the reference's runs) */
    int device;
} lj_adj_params;

typedef struct lj_adj_ctx lj_adj_ctx;

int lj_adj_create(const lj_adj_params* params, lj_adj_ctx** out);
int lj_adj_destroy(lj_adj_ctx* ctx);
const char* lj_adj_last_error(const lj_adj_ctx* ctx);
/* New epsilon and sigma for the next forward pass (the cutoff stays cutoff_sigma * sigma). */
int lj_adj_set_potential(lj_adj_ctx* ctx, double epsilon, double sigma);
/* Run M steps from (x0, v0) (N x stride doubles): out2 = {PE_avg, P_avg};
 * series (may be NULL) receives M x 4 doubles {PE, W, KE, P} of states 1..M. */
int lj_adj_forward(lj_adj_ctx* ctx, const double* x0, const double* v0, int stride, double* out2, double* series);
/* Gradient of w_pe * PE_avg + w_p * P_avg at the last forward pass.  Any
 * output pointer may be NULL. */
int lj_adj_backward(lj_adj_ctx* ctx, double w_pe, double w_p, double* dx0, double* dv0, int stride,
                    double* depsilon, double* dsigma);

#ifdef __cplusplus
}
#endif

#endif /* LJ_GPU_H */
