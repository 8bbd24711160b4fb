/*
 * gbght.h — C ABI of the B200-native IF-RK time step of GBGHomogeneousTurbulence.jl.
 *
 * One opaque handle holds a run: the domain, the flow conditions, the spectral state, the step's
 * registers, the observables deposited at the end of an iteration, and (optionally) the tracers.
 * The library owns all device memory. Every call returns a status code. gbght_last_error() returns
 * the message of the last failing call on a handle, and gbght_global_error() that of a failed
 * create. Calls on one handle are not thread-safe. They run on the handle's own CUDA stream, and
 * every call that returns data to the host synchronises that stream.
 *
 * Arrays cross the boundary in the reference's own layouts:
 *  - spectral fields: complex128 interleaved (re, im), row-major [comp][kz][ky][kx], kx in
 *    [0, N/2]. This is the column-major (kx, ky, kz, comp) rfft array of the reference.
 *    The forward transform is unnormalised, as in the reference (docs/src/validation.md:72-74).
 *  - physical fields: float64 row-major [comp][z][y][x], node i at x = i·L/N.
 *  - tracer positions and point values: float64 [3][M], the (M, 3) column-major array of the
 *    reference's PointSet / VectorPointValues.
 *
 * Every entry point cites the reference interface it replaces (file:line within the reference
 * project). Status codes map onto the reference's exception types: GBGHT_ERR_ARGUMENT is an
 * ArgumentError, and GBGHT_ERR_SCHEDULE is an ErrorException (a schedule refusal or a blow-up).
 */
#ifndef GBGHT_H
#define GBGHT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gbght_run gbght_run;

enum gbght_status {
  GBGHT_OK = 0,
  GBGHT_ERR_ARGUMENT = 1,   /* ArgumentError: a bad argument or an unsupported configuration */
  GBGHT_ERR_SCHEDULE = 2,   /* ErrorException: refused schedule (stale/missing deposit), blow-up */
  GBGHT_ERR_CUDA = 3,       /* a CUDA runtime error; the message names the call */
  GBGHT_ERR_DEVICE = 4      /* a device-side status bit was raised (see gbght_status_word) */
};

enum gbght_precision { GBGHT_FP64 = 0, GBGHT_FP32_MIXED = 1 };
/* The field integration schemes (src/Propagator.jl): IFLowStorageRK4 (:304-320), IFLowStorageRK3
 * (:267-274), IFHeun (:456-544), IFSSPRK3 (:599-691). */
enum gbght_scheme { GBGHT_IFRK4 = 0, GBGHT_IFRK3 = 1, GBGHT_IFHEUN = 2, GBGHT_IFSSPRK3 = 3 };
/* The forcing strategies (src/Forcing.jl), for either field:
 *  NONE                 NoForcing.
 *  CONSTANT_POWER       ConstantPower (:1069-1117): A = ε/(2 k_band) re-solved at every stage, a
 *                       per-stage source A·𝟙_band·f.
 *  LINEAR               Linear (:636-653): a steady rate A on the band, folded into the
 *                       integrating factor exp((A(κ) − D|κ|²)·δt) (src/Generator.jl:565-581).
 *  VARIANCE_CONTROLLER  VarianceController (:1041-1067): A = (ε − G(k − k∞)/tℓ)/(2 k_band) at
 *                       every stage, with k and ε the field's whole variance and dissipation.
 *  VARIANCE_RESCALING   VarianceRescaling (:575-596): after the step, the band is rescaled by one
 *                       factor so the band's (`over` = 0) or the whole field's (`over` = 1)
 *                       variance equals `target`. First order in time, as in the reference.
 *  STOCHASTIC_OU        StochasticOU (:1224-1415): an additive force, the same at every stage of a
 *                       step, held on a companion grid of Nc = 2·(highest_shell + 1) points and
 *                       advanced once per step on the host (an Ornstein–Uhlenbeck process with
 *                       stationary mean square `target` = σ² and correlation time `turnover_time`
 *                       = T_L). The caller hands each step's force in by gbght_forcing_source_set
 *                       before the step; highest_shell must be finite and its band inside the
 *                       retained 2/3 ball.
 * The variance is ½⟨|u|²⟩ for the velocity and ⟨φ²⟩ for the scalar (src/Forcing.jl:456). */
enum gbght_forcing {
  GBGHT_FORCING_NONE = 0,
  GBGHT_FORCING_CONSTANT_POWER = 1,
  GBGHT_FORCING_LINEAR = 2,
  GBGHT_FORCING_VARIANCE_CONTROLLER = 3,
  GBGHT_FORCING_VARIANCE_RESCALING = 4,
  GBGHT_FORCING_STOCHASTIC_OU = 5
};
enum gbght_rescaling_over { GBGHT_OVER_BAND = 0, GBGHT_OVER_TOTAL = 1 };

/* One field's forcing: the kind and the parameters that kind reads. The band is the shells
 * lowest..highest, shell h covering [h − ½, h + ½)·2π/L; highest is an integer shell or INFINITY
 * (every mode but the mean). */
typedef struct gbght_forcing_params {
  int kind;               /* gbght_forcing */
  double rate;            /* ConstantPower injection_rate ε, or Linear rate A */
  double target;          /* VarianceController k∞ (> 0), or VarianceRescaling target (≥ 0) */
  double gain;            /* VarianceController gain G ≥ 0 */
  double turnover_time;   /* VarianceController tℓ > 0, given explicitly */
  int over;               /* VarianceRescaling: gbght_rescaling_over */
  int lowest_shell;       /* ≥ 1 */
  double highest_shell;   /* ≥ lowest_shell */
} gbght_forcing_params;

/* The particle integration schemes (src/ParticlePropagator.jl:48-256): Heun = ABM(1); ABM(k),
 * k = 1..7, the k-step Adams–Bashforth–Moulton predictor–corrector of order k + 1; AB(k), k = 1..8,
 * the k-step Adams–Bashforth of order k. The weights are re-solved every step from the samples'
 * times; while the trail holds fewer than k samples the step is ABM(samples held). */
enum gbght_tracer_scheme { GBGHT_HEUN = 0, GBGHT_ABM = 1, GBGHT_AB = 2 };

/* Device status bits (gbght_status_word). */
#define GBGHT_STATUS_NONFINITE_SPEED 0x1u
#define GBGHT_STATUS_EMPTY_BAND      0x2u
#define GBGHT_STATUS_COPY_TIMEOUT    0x4u  /* a bulk copy missed its bounded wait */

typedef struct gbght_config {
  int grid_points_per_axis;  /* N; supported: 8 12 16 24 32 48 64 96 128 192 256 384 512 */
  double side_length;        /* L */
  int precision;             /* gbght_precision */
  int scheme;                /* gbght_scheme (field integration) */
  double viscosity;          /* ν > 0 */
  double schmidt;            /* Sc > 0; scalar diffusivity ν/Sc */
  int scalar;                /* 1: carry the passive scalar */
  gbght_forcing_params velocity_forcing;   /* any kind */
  gbght_forcing_params scalar_forcing;     /* any kind; needs scalar = 1 unless NONE */
  double mean_gradient[3];   /* uniform mean scalar gradient G (extension; 0 = none) */
  int64_t tracers;           /* M ≥ 0 tracers */
  double cfl;                /* C of the advective CFL rule */
  double max_dt;             /* caller's ceiling on Δt (INFINITY = none) */
  int device;                /* CUDA device ordinal */
  int tracer_scheme;         /* gbght_tracer_scheme */
  int tracer_steps;          /* k of ABM(k) / AB(k); 1 for Heun. The trail keeps k samples */
  int shortened_first_steps; /* 1: shorten the first steps while a k > 1 scheme's trail fills
                                (src/SimulationRun.jl:1099-1132); a fixed dt is then refused */
  int interpolation;          /* gbght_interpolation: the tracers' grid→point scheme */
  int interpolation_points;   /* stencil width per axis, 4, 6 or 8 (Lalescu, Lagrange) */
  int interpolation_smoothness; /* LalescuSpline's order of continuity, 1..min(3, points − 2) */
  int dealiasing;             /* gbght_dealiasing */
  int houli_order;            /* HouLi's filter order (default 36) */
  double houli_strength;      /* HouLi's damping at the Nyquist mode; ≤ 0: −log(eps) of the precision */
  int tracer_gather;          /* Catmull–Rom gathers: 0 automatic (the default: warp-cooperative in
                                 FP64 with fewer tracers than one per 50 grid points, else per
                                 tracer, the faster measured in each case), 1 one thread per tracer,
                                 2 warp-cooperative (16 lanes per tracer); all agree bit for bit */
} gbght_config;

/* The dealiasing strategies (src/SimulationDomain.jl:73-177). TWO_THIRDS: the closed 2/3 ball, the
 * state stored on it. HOULI (Hou & Li 2007): no cutoff; the nonlinear terms are multiplied by
 * exp(−strength·(|κ|/κ_Ny)^order) (src/SimulationDomain.jl:365-376), and the state is stored on
 * every mode but the Nyquist planes, where the filter is ≈ eps: the reference's retained band is the
 * whole grid, and what it keeps on those planes is at round-off. PHASE_SHIFT (Patterson & Orszag
 * 1971, Rogallo 1981): each stage's nonlinear terms are the average of the grid's and those of the
 * grid displaced by half a cell along every axis, shifted back, on the closed ball of radius
 * (2√2/3)·κ_Ny (src/SimulationDomain.jl:177-184, src/Generator.jl:502-519,668-704); twice the
 * transforms of TWO_THIRDS per stage. The adjoint is built for TWO_THIRDS only. */
enum gbght_dealiasing { GBGHT_TWO_THIRDS = 0, GBGHT_HOULI = 1, GBGHT_PHASE_SHIFT = 2 };

/* The tracers' interpolation schemes (src/Particles.jl:61-70, schemes of GBGPeriodicFields):
 * CatmullRom = LalescuSpline(4) (the default); LalescuSpline(n; smoothness m), the degree 2m + 1
 * Hermite polynomial per cell with the derivatives from centred (n − 1)-point differences
 * (Lalescu, Teaca & Carati 2010); LagrangeSpline(n), the degree n − 1 Lagrange polynomial through
 * the n taps. The adjoint of the tracers is built for CatmullRom. */
enum gbght_interpolation { GBGHT_CATMULL_ROM = 0, GBGHT_LALESCU = 1, GBGHT_LAGRANGE = 2 };

/* Fill `cfg` with the defaults: N=64, L=2π, FP64, IF-RK4, ν=0.01, Sc=1, scalar on, no forcing
 * of either field (each forcing block: rate 0, target 0, gain 1, turnover time 0, over = band,
 * shells 1–2), G=0, no tracers, Heun, no shortened start, CFL 0.5, max_dt=∞, device 0,
 * Catmull–Rom interpolation (4 points, smoothness 1), TwoThirds dealiasing (HouLi: order 36, default
 * strength). */
void gbght_config_default(gbght_config* cfg);

/* Build a run on a FixedDomain with TwoThirds, HouLi or PhaseShift dealiasing, with its generator and
 * registers.
 * Replaces FixedDomain(...) (src/SimulationDomain.jl:295-328), FlowConditions
 * (src/Generator.jl:81-140), the forcings of either field (ConstantPower src/Forcing.jl:1069-1075,
 * Linear :636-643, VarianceController :828-875, VarianceRescaling :558-572), allocate_buffers
 * (src/Propagator.jl:717-723) and ObservablesCache (src/Cache.jl:150-173). The state starts at
 * zero. */
int gbght_create(gbght_run** out, const gbght_config* cfg);
void gbght_destroy(gbght_run* run);
const char* gbght_last_error(const gbght_run* run);
const char* gbght_global_error(void);
const char* gbght_version(void);

/* Retained-band geometry: K (largest retained |m| per axis) and the dealias cutoff (the Nyquist
 * wavenumber under HouLi).
 * Replaces max_retained_wavenumber (src/SimulationDomain.jl:413-419). */
int gbght_geometry(const gbght_run* run, int* K, double* cutoff);

/* Spectral state import/export in the reference layout, from and into host memory or device memory
 * of the run's device (a CUDA.jl CuArray or a torch tensor; unified addressing tells them apart):
 * a device array is converted by a kernel in place, with no staging through the host. Memory of
 * another device is refused with ARGUMENT. phi_hat may be NULL when the run carries no scalar. Import refuses (ARGUMENT) a state with content outside the retained
 * 2/3 ball: the library stores only the retained modes. Every state the reference's seeders
 * and steps produce is band-limited. Import invalidates the deposit.
 * Replaces ResolvedFields(û, φ̂) (src/State.jl:119-137) and the state read/write of
 * ext/GBGHomogeneousTurbulenceHDF5Ext.jl. */
int gbght_state_import(gbght_run* run, const double* u_hat, const double* phi_hat);
int gbght_state_export(gbght_run* run, double* u_hat, double* phi_hat);

/* The force of a StochasticOU field (field 0 velocity, 1 scalar) for the next step: its physical
 * amplitudes a_k (the coefficients of e^{iκ·x}) on the companion grid, complex128 in the companion's
 * reference layout [comp][kz][ky][kx] (kx ≤ Nc/2, 3 components for the velocity, 1 for the scalar),
 * host or device memory. Every stage of the next step adds N³·a_k to the field's right-hand side on
 * the forcing's band, where the run's modes and the companion's coincide. Each step consumes the
 * force: a step of a StochasticOU field without a force set since the last step is refused with
 * SCHEDULE, as the reference advances the process once per step (prepare_forcing!,
 * src/Forcing.jl:1401-1411). Replaces _advance_process! / add_forcing_source!(::StochasticOU)
 * (:1362-1415); the host draws and transforms, as the reference's draws are made on the host. */
int gbght_forcing_source_set(gbght_run* run, int field, const double* amplitudes, int companion_points);

/* One field step of the configured scheme with step dt > 0, in place. Requires a current field
 * deposit, i.e. gbght_deposit after the last state change; otherwise SCHEDULE. The step advances
 * velocity and scalar together, then applies the forcings' post-step projections and the Leray
 * and reality projections. Replaces step!(::IFLowStorageRK4 / ::IFLowStorageRK3 / ::IFHeun /
 * ::IFSSPRK3, state, generator, domain, buffers, cache, dt) (src/Propagator.jl:267-274,304-419,
 * 456-544,599-691). */
int gbght_step(gbght_run* run, double dt);

/* An ensemble of runs stepped together: members of any supported sizes and configurations, on one
 * device, each a distinct run. gbght_ensemble_step is gbght_step then gbght_deposit for every
 * member with the same dt. On the GPU the members' launches are captured once per dt as one CUDA
 * graph whose branches run on the members' own streams (so small grids run side by side), and the
 * graph is replayed on later calls; the max-speed readbacks follow the replay. A member whose
 * deposit is not current, or whose deposit slots were reused by another call since, is deposited
 * first. Tracers are not moved (as with gbght_step). The ensemble holds the member handles, which
 * must outlive it. The batching form of the configs: ensembles of uneven grids (32³, 48³, 64³). */
typedef struct gbght_ensemble gbght_ensemble;
int gbght_ensemble_create(gbght_ensemble** out, gbght_run* const* members, int n);
void gbght_ensemble_destroy(gbght_ensemble* ensemble);
int gbght_ensemble_step(gbght_ensemble* ensemble, double dt);
const char* gbght_ensemble_last_error(const gbght_ensemble* ensemble);
/* Member batching. Members whose step launches the same kernels (precision, N, dealiasing,
 * scheme, scalar, velocity forcing kind; NoForcing, ConstantPower or Linear, and no PhaseShift or
 * StochasticOU) may form groups of at most `max_group` members, and the graph then holds one
 * launch per pass for each group instead of one per member. The group's kernels are a separate
 * compilation of the same CTA code, so a member's results equal those of stepping it alone to
 * round-off (not bit for bit: relative differences near 1e-16 in FP64 and 5e-8 in FP32-mixed after
 * a step); members with equal inputs stay bitwise equal to each other. `max_group` ≤ 1 (the
 * default) captures one launch per member and pass, bit for bit the lone steps.
 * gbght_ensemble_autotune makes the following steps try group sizes 1, 2, 4, … up to the largest
 * set of batchable members, two steps each (a capture, then a replay timed by CUDA events), and then
 * keep the fastest; gbght_ensemble_tuning reports the current size, whether the tuning is done and
 * the replay times so far (ms[i] for the i-th candidate). gbght_ensemble_units reports the
 * launching units (groups and lone members) of the last captured graph, 0 before the first step.
 * No reference counterpart: the reference steps one simulation per call. */
int gbght_ensemble_set_batching(gbght_ensemble* ensemble, int max_group);
int gbght_ensemble_autotune(gbght_ensemble* ensemble);
int gbght_ensemble_tuning(const gbght_ensemble* ensemble, int* max_group, int* done, float* ms, int capacity);
int gbght_ensemble_units(const gbght_ensemble* ensemble, int* units);

/* A scheme's advective-CFL ceiling under the 2/3 rule: 0.96 (RK4), 0.5 (RK3, SSPRK3), 0.25 (Heun).
 * Replaces recommended_cfl(scheme, domain) (src/Propagator.jl:906-919) for TwoThirds. */
int gbght_recommended_cfl(int scheme, double* cfl);
/* The same ceiling for a dealiasing strategy (gbght_dealiasing): × (2/3)/f, f the fraction of the
 * Nyquist wavenumber the strategy retains (2/3, 1 for HouLi, 2√2/3 for PhaseShift).
 * Replaces recommended_cfl(scheme, domain) (src/Propagator.jl:915-916). */
int gbght_recommended_cfl_dealiased(int scheme, int dealiasing, double* cfl);

/* The closing field deposit: the velocity in physical representation and max|u|.
 * Replaces deposit!(cache, state, domain, buffers) (src/Propagator.jl:808-842). */
int gbght_deposit(gbght_run* run);

/* The deposited max|u| (sqrt of the maximum of |u|²). Replaces max_speed(cache)
 * (src/Cache.jl:416-421, src/Observables.jl:304-305). */
int gbght_max_speed(gbght_run* run, double* speed);

/* The advective CFL step for the deposited velocity. Replaces cfl_timestep(sim)
 * (src/SimulationRun.jl:1051-1096). */
int gbght_cfl_timestep(gbght_run* run, double* dt);

/* Export the deposited physical velocity, [3][N][N][N] float64. Replaces velocity_physical(cache)
 * (src/Cache.jl:291-299). */
int gbght_velocity_physical_export(gbght_run* run, double* u);

/* Write a prescribed physical velocity into the deposit slot, as the reference's test fake does
 * (test/prescribed_flow.jl:16-21). The spectral state is untouched. The tracers are then advected
 * in this field. */
int gbght_velocity_physical_import(gbght_run* run, const double* u);

/* Observables of the current state: k, ε, ⟨φ²⟩, ε_φ (FP64 reductions).
 * Replaces kinetic_energy_and_dissipation (src/Observables.jl:170-173) and
 * scalar_variance_and_dissipation (src/Observables.jl:345-380). */
int gbght_observables(gbght_run* run, double out[4]);

/* Shell spectrum of the velocity (which = 0, E(κ) = radial_spectrum/(2Δκ)) or of the scalar
 * (which = 1, radial_spectrum/Δκ). Shell n covers [n − ½, n + ½)·Δκ. `n` is the capacity of
 * `out`; gbght_spectrum_length gives the shell count. Replaces energy_spectrum
 * (src/Observables.jl:502-514). */
int gbght_spectrum_length(const gbght_run* run, int* n);
int gbght_spectrum(gbght_run* run, int which, double* out, int n);

/* The derivative skewness of the state, C·3⟨det S⟩/⟨S:S⟩^{3/2} with S the strain rate in physical
 * space, ⟨S:S⟩ = ½Σ|κ|²|û|² and C = (4/7)√(15/2); 0 for a strain-free state. It allocates a
 * transient buffer of six physical fields and leaves the state and the deposit unchanged.
 * Replaces derivative_skewness(û, domain) (src/Observables.jl:466-478). */
int gbght_derivative_skewness(gbght_run* run, double* skewness);

/* The kinetic energy and dissipation below scale: for every box side l = nL/N (n = 1..N),
 * k(l) = ½Σ(1 − W_l²)|û|² and ε(l) = νΣ|κ|²(1 − W_l²)|û|², W_l(κ) = ∏_a sinc(κ_a l/2) the
 * transfer function of the box mean (normalised sums, FP64). `n` is the capacity of each output
 * (at least N); `scales` may be NULL. Replaces kinetic_energy_and_dissipation_below_scale(û, domain,
 * viscosity) (src/Observables.jl:253-263). An occasional diagnostic: its cost grows as N⁴. */
int gbght_energy_below_scale(gbght_run* run, double* scales, double* k, double* eps, int n);

/* Tracer positions [3][M], copied as given (the push wraps them into [0, L)), from and into host
 * memory or device memory of the run's device. Import clears the trail. Replaces
 * Tracers(domain; positions) (src/Particles.jl:145-176). */
int gbght_tracers_import(gbght_run* run, const double* X);
int gbght_tracers_export(gbght_run* run, double* X);

/* The newest velocity sample at the tracers [3][M] and its time. Replaces
 * velocity_at_particles_trail (src/Cache.jl). */
int gbght_tracer_sample_export(gbght_run* run, double* values, double* t);

/* The j-th newest sample of the trail (j = 0 the newest, j < the samples held) [3][M] and its time,
 * as held: a checkpoint stores them all, oldest to newest, to restore a multistep scheme's trail.
 * Replaces the trail's read in write_simulation (ext/GBGHomogeneousTurbulenceHDF5Ext.jl:426-561). */
int gbght_tracer_trail_export(gbght_run* run, int j, double* values, double* t);

/* Empty the trail, and push an earlier sample [3][M] at time t (later than the newest held) without
 * moving the tracers or pairing the epochs: a checkpoint's restore of the samples a multistep
 * scheme integrates over, before the ordinary particle deposit adds the newest. Replaces
 * reset_velocity_at_particles! and restore_velocity_at_particles! (src/Cache.jl:380-389). */
int gbght_tracer_trail_reset(gbght_run* run);
int gbght_tracer_sample_restore(gbght_run* run, const double* values, double t);

/* Advance the tracers one step of size dt of the configured particle scheme (Heun, ABM(k), AB(k))
 * through the deposited velocity and the trail's samples. The step requires the newest trail sample
 * to be at the current positions, and the fields to be exactly one step ahead of it; otherwise
 * SCHEDULE. Replaces advect!(scheme, tracers, domain, cache, dt; traversal)
 * (src/ParticlePropagator.jl:282-352). */
int gbght_advect(gbght_run* run, double dt);

/* The particle deposit: sample the deposited velocity at the tracers, labelled with time t.
 * Replaces deposit!(cache, tracers, t; traversal) (src/ParticlePropagator.jl:378-386). */
int gbght_deposit_tracers(gbght_run* run, double t);

/* Catmull–Rom gather of the deposited velocity at arbitrary positions X [3][M] → out [3][M].
 * Replaces interpolate_at_particles!(out, u, tracers) (src/Particles.jl:290-293). */
int gbght_interpolate_velocity(gbght_run* run, const double* X, int64_t M, double* out);

/* One iteration of the run layer: Δt (dt > 0 fixed, dt <= 0 the CFL rule with the start-up bound
 * under shortened_first_steps, where a fixed dt is refused), step, deposit, the particle scheme's
 * push and the particle deposit, blow-up guards, clock. The Δt taken is returned in *dt_taken (may
 * be NULL). Replaces advance!(sim; dt) (src/SimulationRun.jl:1155-1229). */
int gbght_advance(gbght_run* run, double dt, double* dt_taken);

/* The run's clock. Replaces current_time / current_step (src/SimulationRun.jl). */
int gbght_clock(const gbght_run* run, double* time, int64_t* step);
int gbght_set_clock(gbght_run* run, double time, int64_t step);

/* Device status bits raised since the last call (GBGHT_STATUS_*); reading clears them. */
int gbght_status_word(gbght_run* run, uint32_t* word);

/* No counterpart in the reference: the failure path of the device's bounded waits, exercised on
 * purpose. A kernel on the run's stream arms a barrier for a copy that is never issued and waits at
 * most `cycles` clock cycles (1 ≤ cycles ≤ 1e9); the wait expires, raises
 * GBGHT_STATUS_COPY_TIMEOUT, and returns, exactly as a wait on a lost copy does in the step's
 * kernels. The call then returns GBGHT_ERR_DEVICE, as a deposit does after such an expiry; the bit
 * stays raised until gbght_status_word reads it. Nothing faults, and the run stays usable. */
int gbght_selftest_wait_timeout(gbght_run* run, int64_t cycles);

/* CUDA-event timing on the run's own stream (no counterpart in the reference, which has no
 * profiling; used by the benchmark to time kernels where they are launched).
 * gbght_profile(run, 1) clears the counters and brackets every later kernel launch with events;
 * gbght_profile(run, 0) stops. gbght_profile_read returns, for kernel kind `kind`
 * (GBGHT_KERNEL_*), the number of launches and their summed duration in milliseconds.
 * gbght_timer(run, 0, NULL) records a start event; gbght_timer(run, 1, &ms) records a stop
 * event, waits for it and returns the elapsed milliseconds. */
enum gbght_kernel {
  GBGHT_KERNEL_Y_INVERSE = 0,   /* inverse y-transform pass */
  GBGHT_KERNEL_X_PRODUCTS = 1,  /* x pass: c2r, u×ω and uφ, r2c */
  GBGHT_KERNEL_Y_FORWARD = 2,   /* forward y-transform pass */
  GBGHT_KERNEL_Z_EPILOGUE = 3,  /* z-forward, IF-RK stage update, z-inverse */
  GBGHT_KERNEL_X_VELOCITY = 4,  /* deposit: physical velocity and max|u| */
  GBGHT_KERNEL_FORCE_AMP = 5,   /* band-forcing amplitudes, VarianceRescaling's rescale */
  GBGHT_KERNEL_REALITY = 6,     /* end-of-step reality projection */
  GBGHT_KERNEL_TRACERS = 7,     /* tracer gather / Adams push */
  GBGHT_KERNEL_OBSERVABLES = 8, /* k, ε, ⟨φ²⟩, ε_φ reductions, their row sums for the band forcings,
                                   the diagnostics' reductions */
  GBGHT_KERNEL_TRAVERSAL = 9,   /* tracer traversal order: tile keys, scan, scatter */
  GBGHT_KERNEL_X_ADJOINT = 10,  /* the adjoint x pass: c2r of fields and sources, their products, r2c */
  GBGHT_KERNEL_Z_ADJOINT = 11,  /* the adjoint z pass: z-forward, the λ update, the next stage's sources */
  GBGHT_KERNEL_Z_SHIFT = 12     /* PhaseShift: the displaced grid's z-inverse, and the shift back of its
                                   products averaged into the grid's */
};
int gbght_profile(gbght_run* run, int enable);
int gbght_profile_read(gbght_run* run, int kind, int64_t* launches, double* total_ms);
int gbght_timer(gbght_run* run, int op, double* ms);

/* No counterpart in the reference: an allocation-free form of the deposit's velocity recovery,
 * for callers that cannot allocate device memory. A caller whose device memory is owned by another
 * allocator (for example a framework's caching pool that has reserved the GPU) cannot call
 * cudaMalloc, and neither can a loop that keeps the reference's rule of no field-scale allocation
 * inside a step. This call takes no run handle and allocates nothing. It reads the spectral
 * velocity u_hat (device memory, complex128 [3][N][N][N/2+1], the reference layout), writes the
 * physical velocity u (device memory, float64 [3][N][N][N]) and, if max_speed is not NULL,
 * returns max|u| on the host. The values are those gbght_deposit + gbght_velocity_physical_export
 * give for the same spectrum (FP64).
 * Every intermediate lives in one file-scope device array of 12 MiB, held by each GPU that loads the
 * library until the process exits; on the host the call uses static storage only. N is limited to
 * 8, 12, 16, 24, 32, 48 or 64; a larger N is refused with GBGHT_ERR_ARGUMENT before any work. A
 * spectrum with content outside the retained 2/3 ball is also refused with GBGHT_ERR_ARGUMENT, but
 * only after the kernels have run: `u` then holds the velocity of the truncated spectrum.
 * The first call on a device looks up the array's address; a call whose grid differs from the
 * previous call's on that device re-encodes its tensor maps and re-uploads its twiddles into the
 * array. Calls share the array, so two calls whose work overlaps on the GPU (other streams, other
 * host threads) race: serialise them. `stream` is a cudaStream_t (NULL: the default stream). Every
 * call synchronises that stream once, to read back max|u| and the status word, so no call may be
 * made inside a stream capture. Errors are reported through gbght_global_error(). */
int gbght_velocity_physical_noalloc(int grid_points_per_axis, double side_length, const double* u_hat,
                                    double* u, double* max_speed, void* stream);

/* The discrete adjoint of the field step (no counterpart in the reference, which has no AD; the
 * step it differentiates is _low_storage_2n_step!, src/Propagator.jl:326-419, with velocity_rhs! /
 * scalar_rhs!, src/Generator.jl:484-534,648-730, and ConstantPower's source,
 * src/Forcing.jl:1091-1117). It is the exact transpose of the discrete map gbght_step computes for
 * IFLowStorageRK4 / IFLowStorageRK3 with NoForcing, ConstantPower or Linear forcing on either field
 * and the mean scalar gradient, for the inner products Σ_x a·b (physical) and Σ w·Re(conj(x)·y)
 * (spectral, w = 1 on the kx = 0 plane and 2 elsewhere), restricted to the retained 2/3 ball.
 *
 * gbght_adjoint_create allocates the adjoint registers (λ, the stage states) and `snapshots`
 * device slots for the state (0..64), for a checkpointing schedule that stores states on the
 * device. λ crosses in the reference layout, host or device memory (as gbght_state_import);
 * content outside the retained ball is refused and clears λ. gbght_adjoint_step replaces λ by
 * J(q)ᵀλ, J the Jacobian of one step of size dt at the run's current state q; it runs the step's
 * stages again to keep their states, leaves q (and the deposit) as they were, and adds to the
 * forcing gradient the derivative of the loss with respect to each ConstantPower injection rate
 * ε (velocity, scalar) through that step. gbght_adjoint_add_observable adds `weight` times the
 * gradient of an observable of the current state to λ: the kinetic energy k (which = 0, gradient
 * û/N⁶) or the scalar variance ⟨φ²⟩ (which = 1, gradient 2φ̂/N⁶). gbght_adjoint_forcing_gradient
 * returns the accumulated dL/dε of the two fields (and clears it when `reset`);
 * gbght_adjoint_clear sets λ and the gradient to zero. gbght_snapshot_save / _load copy the state
 * into / out of a slot (load makes the deposit stale, as an import does). */
enum gbght_observable { GBGHT_OBSERVABLE_KINETIC_ENERGY = 0, GBGHT_OBSERVABLE_SCALAR_VARIANCE = 1 };
int gbght_adjoint_create(gbght_run* run, int snapshots);
int gbght_adjoint_import(gbght_run* run, const double* lam_u, const double* lam_phi);
int gbght_adjoint_export(gbght_run* run, double* lam_u, double* lam_phi);
int gbght_adjoint_step(gbght_run* run, double dt);
int gbght_adjoint_add_observable(gbght_run* run, int which, double weight);
int gbght_adjoint_forcing_gradient(gbght_run* run, double out[2], int reset);
int gbght_adjoint_clear(gbght_run* run);
int gbght_snapshot_save(gbght_run* run, int slot);
int gbght_snapshot_load(gbght_run* run, int slot);

/* The tracers in the adjoint (Heun tracers with Catmull–Rom gathers; the reference's
 * src/ParticlePropagator.jl:288-315,378-386 differentiated). A snapshot of a run with tracers also
 * holds the positions and the trail's newest sample with its time, and the clock.
 * gbght_adjoint_advance is the reverse of one whole advance! iteration at the run's current state
 * (q, X, f): λ holds the cotangent of the state after the iteration and the tracer register that
 * of (X', f'); the tracers' push and closing deposit are reversed first (their gathers add to λ),
 * then the field step; the run is left at (q, X, f) with its deposit current.
 * gbght_adjoint_deposit_tracers reverses the particle deposit f = u(X) alone at the current state
 * (the sample a Simulation takes at construction): λ += its gathers' part, λ_X += …, λ_f = 0.
 * gbght_adjoint_tracers_import / _export move the tracer cotangents (λ_X, λ_f), [3][M] each, host
 * or device memory. The gathers' adjoint adds with atomics, so results agree with any other order
 * to round-off, not bit for bit. */
int gbght_adjoint_advance(gbght_run* run, double dt);
int gbght_adjoint_deposit_tracers(gbght_run* run);
int gbght_adjoint_tracers_import(gbght_run* run, const double* lam_X, const double* lam_f);
int gbght_adjoint_tracers_export(gbght_run* run, double* lam_X, double* lam_f);

/* Wait for all work queued on the run's stream. */
int gbght_synchronize(gbght_run* run);

#ifdef __cplusplus
}
#endif

#endif /* GBGHT_H */
