// The engine: device buffers and the launch sequence of the IF-RK step for one (precision, N).
//
// The same source builds two ways. With nvcc it is the CUDA library: kernels launched on the
// run's stream. With -DGBGHT_EMU and a host C++ compiler, every "device" buffer is host memory
// and every launch runs the same CTA bodies block by block with one thread (NT = 1). That build
// exists only to check the kernels' index arithmetic on a CPU against the oracle; the product
// library is the CUDA build and has no host path.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "passes.cuh"
#include "tracers.cuh"

#ifndef GBGHT_EMU
#include <cuda_runtime.h>
#endif

namespace gbght {

// One field's forcing (a copy of gbght_forcing_params, validated). kind: 0 none,
// 1 ConstantPower, 2 Linear, 3 VarianceController, 4 VarianceRescaling.
struct ForcingParams {
  int kind;
  double rate;            // ConstantPower ε, or Linear A
  double target;          // VarianceController k∞, or VarianceRescaling target
  double gain;            // VarianceController G
  double turnover_time;   // VarianceController tℓ
  int over;               // VarianceRescaling: 0 band, 1 total
  int lowest_shell;
  double highest_shell;
};
enum ForcingKind {
  kForceNone = 0, kForceConstantPower = 1, kForceLinear = 2, kForceController = 3, kForceRescaling = 4,
  kForceStochastic = 5
};

// The parameters of a run that the engine needs (a copy of the public config, validated).
struct RunParams {
  int N;
  double L;
  int precision;
  int scheme;
  double viscosity, schmidt;
  int scalar;
  ForcingParams vf;          // velocity forcing
  ForcingParams sf;          // scalar forcing (kind 0 when the run carries no scalar)
  double G[3];
  int64_t tracers;
  int trail_capacity;        // sample slots of the tracers' trail (the Adams scheme's k)
  Stencil stencil;           // the tracers' interpolation weights (n = 0: Catmull–Rom)
  int dealias;               // 0 TwoThirds, 1 HouLi, 2 PhaseShift
  int houli_order;           // HouLi's filter order (36 by default)
  double houli_strength;     // HouLi's strength; ≤ 0 for the default −log(eps(T))
  int tracer_gather;         // Catmull–Rom gathers: 0 automatic, 1 one thread per tracer, 2 warp-cooperative
  int device;
};

// Host-visible results of the reductions.
struct Observables {
  double k, eps, var, chi;
};

// The message an engine call returns when a bounded device wait expired (device status 0x4); the
// C ABI reports it as GBGHT_ERR_DEVICE rather than as a CUDA runtime error.
inline const char* const kDeviceTimeoutMessage =
    "a bulk copy did not complete within its bounded wait (device status 0x4)";

class Engine {
 public:
  virtual ~Engine() {}
  // All methods return nullptr on success, else a static or engine-owned error message.
  virtual const char* init(const RunParams& p) = 0;
  // The state crosses in the reference layout, from and into host memory or device memory of the
  // run's device (told apart by the pointer's attributes).
  virtual const char* import_state(const double* uh, const double* ph, bool* outside) = 0;
  virtual const char* export_state(double* uh, double* ph) = 0;
  virtual const char* step(double dt, const double* a, const double* b, const double* d, int S) = 0;
  virtual const char* deposit(double* max_speed2) = 0;
  // The deposit split in two: its launches alone (no host synchronisation, so a CUDA graph can
  // hold them), and the readback of max|u|² and of the device status once they have run.
  virtual const char* deposit_launch() = 0;
  virtual const char* deposit_read(double* max_speed2) = 0;
  // The run's CUDA stream (nullptr in the host-check build); whether B slots 0..2 hold the
  // deposit's y-inverse (the next step's first stage reuses them); whether per-launch profiling
  // is on (its events cannot sit in a captured graph).
  virtual void* cuda_stream() const = 0;
  virtual bool deposit_fresh() const = 0;
  virtual bool profiling() const = 0;
  // Member-batched stepping of an ensemble. group_key() is equal for runs whose step and deposit
  // launch the same kernels with the same grids, and 0 for a run that steps alone (PhaseShift, a
  // StochasticOU source, a forcing with per-stage row sums or a post-step rescale).
  // group_prepare() builds the members' launch records in this (the first) member's device memory,
  // synchronously, before a capture; group_launch() then issues the group's step and deposit, one
  // launch per pass over all members, on this member's stream.
  virtual uint64_t group_key() const = 0;
  virtual const char* group_prepare(Engine* const* members, int n, double dt, const double* a, const double* b,
                                    const double* d, int S) = 0;
  virtual const char* group_launch() = 0;
  // a StochasticOU field's force for the next step: companion amplitudes [comp][nc][nc][nc/2+1]
  virtual const char* forcing_source(int field, const double* amplitudes, int nc) = 0;
  virtual const char* velocity_export(double* u) = 0;
  virtual const char* velocity_import(const double* u) = 0;
  virtual const char* observables(Observables* o) = 0;
  // the scalar variance alone (the blow-up guard of advance!), reading φ̂ only
  virtual const char* scalar_variance(double* var) = 0;
  virtual const char* spectrum(int which, double* out, int nshell) = 0;
  // k(l) and ε(l) for every side l = nL/N, n = 1..N (src/Observables.jl:253-263)
  virtual const char* below_scale(double nu, double* k, double* eps) = 0;
  // derivative_skewness of the state (src/Observables.jl:466-478)
  virtual const char* skewness(double* out) = 0;
  virtual const char* tracers_set(const double* X) = 0;
  virtual const char* tracers_get(double* X) = 0;
  virtual const char* tracer_sample_get(double* F, int slot) = 0;
  virtual const char* tracer_sample_set(const double* F, int slot) = 0;
  // One Adams step of every tracer (J = 0: none) and, when w.out_slot ≥ 0, the sample at the new
  // positions into that trail slot
  virtual const char* tracers_run(const AdamsStep& w) = 0;
  virtual const char* gather(const double* X, int64_t M, double* out) = 0;
  virtual const char* sync() = 0;
  // CUDA-event timing on the run's stream: per-kernel launch counts and total milliseconds while
  // profiling is on, and a start/stop pair around any region.
  virtual const char* profile(int enable) = 0;
  virtual const char* profile_read(int kind, int64_t* launches, double* total_ms) = 0;
  virtual const char* timer(int op, double* ms) = 0;
  virtual const char* status(uint32_t* word) = 0;
  // A bounded device wait made to expire after `cycles` clock cycles on the run's stream (a copy
  // that is never issued); returns kDeviceTimeoutMessage once the expiry is seen, as any call that
  // reads the status word does. The run stays usable.
  virtual const char* expire_wait(long long cycles) = 0;
  // The discrete adjoint of the low-storage schemes' step (adjoint.cuh). adjoint_init allocates
  // the adjoint registers and `snapshots` device state slots. λ crosses in the reference layout
  // (host or device memory). adjoint_step replaces λ by J(q)ᵀλ for the step of size dt at the
  // current state q, accumulating the ConstantPower rates' gradients, and leaves q as it was.
  virtual const char* adjoint_init(int snapshots) = 0;
  virtual const char* adjoint_import(const double* lu, const double* lp, bool* outside) = 0;
  virtual const char* adjoint_export(double* lu, double* lp) = 0;
  // `push` (nullptr: the fields alone): the tracers' Heun push and closing deposit of the same
  // iteration, with the forward's weights and the trail slot of the sample before the push; its
  // adjoint updates the tracer cotangents and adds the gathers' part to λ before the field stages.
  virtual const char* adjoint_step(double dt, const double* a, const double* b, const double* d, int S,
                                   const AdamsStep* push = nullptr, int f_slot = 0) = 0;
  // the tracer cotangents (positions, newest sample), [3][M] each, host or device memory
  virtual const char* adjoint_tracers_import(const double* lX, const double* lf) = 0;
  virtual const char* adjoint_tracers_export(double* lX, double* lf) = 0;
  // the particle deposit's adjoint at the current positions and deposit: λ_u += Wᵀλ_f, λ_X += …, λ_f = 0
  virtual const char* adjoint_deposit_tracers() = 0;
  virtual const char* adjoint_add(double wu, double wp) = 0;
  virtual const char* adjoint_gradient(double* g, int reset) = 0;
  virtual const char* adjoint_clear() = 0;
  // a snapshot holds the state and, with tracers, the positions and the trail sample in `f_slot`
  virtual const char* snapshot_save(int slot, int f_slot) = 0;
  virtual const char* snapshot_load(int slot, int f_slot) = 0;
  virtual int K() const = 0;
  virtual double cutoff() const = 0;
};

// Kernel kinds reported by Engine::profile_read (and gbght_profile_read).
enum ProfileKind {
  PROF_Y_INVERSE = 0,
  PROF_X_PRODUCTS = 1,
  PROF_Y_FORWARD = 2,
  PROF_Z_EPILOGUE = 3,
  PROF_X_VELOCITY = 4,
  PROF_FORCE_AMP = 5,
  PROF_REALITY = 6,
  PROF_TRACERS = 7,
  PROF_OBSERVABLES = 8,
  PROF_TRAVERSAL = 9,
  PROF_X_ADJOINT = 10,
  PROF_Z_ADJOINT = 11,
  PROF_Z_SHIFT = 12,
  PROF_KINDS = 13
};

Engine* make_engine(int N, int precision, int dealias, std::string* err);
bool supported_N(int N);

}  // namespace gbght
