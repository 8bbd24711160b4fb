// The C ABI (include/gbght.h): argument checks, the run layer's schedule checks and clock, and
// the calls into the engine. The checks and their messages follow the reference's own refusals;
// each function's comment in gbght.h cites the interface it replaces.
#include "../../include/gbght.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "gbght_engine.cuh"

using gbght::Engine;

struct gbght_run {
  gbght_config cfg{};
  std::unique_ptr<Engine> eng;
  std::string err;
  // the field side of the schedule (src/Cache.jl epochs)
  int64_t fields_epoch = 0;
  int64_t deposit_epoch = -1;
  double max_speed = 0.0;
  // the tracer side: the trail of the velocity at the particles (src/Particles.jl:440-520), a ring
  // of `capacity` device slots, and the epoch pairing of src/Cache.jl:340-390
  int trail_capacity = 1;
  int trail_count = 0;          // samples held
  int trail_newest = -1;        // ring slot of the newest
  double trail_time[gbght::kTrailMax] = {};
  bool sampled = false;         // a particle deposit has paired the tracer and field epochs
  bool sample_at_positions = false;
  int64_t sample_epoch = 0;
  // StochasticOU: whether each field's force was set for the next step
  bool source_fresh[2] = {false, false};
  // the clock
  double time = 0.0;
  int64_t step = 0;
  // the snapshot slots' clocks and newest-sample times (the device holds their states)
  std::vector<double> snap_time, snap_sample_time;
  std::vector<int64_t> snap_step;
};

namespace {

thread_local std::string g_global_error;

int fail(gbght_run* r, int code, const std::string& msg) {
  if (r) r->err = msg;
  return code;
}

int engine_call(gbght_run* r, const char* e) {
  if (!e) return GBGHT_OK;
  return fail(r, e == gbght::kDeviceTimeoutMessage ? GBGHT_ERR_DEVICE : GBGHT_ERR_CUDA, e);
}

// Carpenter & Kennedy (1994) five-stage 2N tableau and Williamson's three-stage one, as rounded
// from their exact rationals (src/Propagator.jl:267-274,304-320); d = differences of the rounded
// abscissae.
struct Tableau {
  int S;
  double a[5], b[5], d[5];
};

// IFHeun and IFSSPRK3 are not low-storage schemes: the engine builds their stages itself (S = 0).
Tableau tableau(int scheme) {
  Tableau t{};
  if (scheme == GBGHT_IFHEUN || scheme == GBGHT_IFSSPRK3) return t;
  if (scheme == GBGHT_IFRK3) {
    t.S = 3;
    const double a[3] = {0.0, -5.0 / 9.0, -153.0 / 128.0};
    const double b[3] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};
    const double d[3] = {1.0 / 3.0, 5.0 / 12.0, 1.0 / 4.0};
    for (int i = 0; i < 3; ++i) { t.a[i] = a[i]; t.b[i] = b[i]; t.d[i] = d[i]; }
    return t;
  }
  t.S = 5;
  t.a[0] = 0.0;
  t.a[1] = -567301805773.0 / 1357537059087.0;
  t.a[2] = -2404267990393.0 / 2016746695238.0;
  t.a[3] = -3550918686646.0 / 2091501179385.0;
  t.a[4] = -1275806237668.0 / 842570457699.0;
  t.b[0] = 1432997174477.0 / 9575080441755.0;
  t.b[1] = 5161836677717.0 / 13612068292357.0;
  t.b[2] = 1720146321549.0 / 2090206949498.0;
  t.b[3] = 3134564353537.0 / 4481467310338.0;
  t.b[4] = 2277821191437.0 / 14882151754819.0;
  const double c2 = 1432997174477.0 / 9575080441755.0;
  const double c3 = 2526269341429.0 / 6820363962896.0;
  const double c4 = 2006345519317.0 / 3224310063776.0;
  const double c5 = 2802321613138.0 / 2924317926251.0;
  t.d[0] = c2;
  t.d[1] = c3 - c2;
  t.d[2] = c4 - c3;
  t.d[3] = c5 - c4;
  t.d[4] = 1.0 - c5;
  return t;
}

bool finite_positive(double v) { return std::isfinite(v) && v > 0.0; }

// The band's shell bounds, as `_check_shells` (src/Forcing.jl:387-403) refuses them: the lowest
// at least 1, the highest an integer shell or infinity, and not below the lowest.
std::string shell_error(int lowest, double highest) {
  if (lowest < 1)
    return "`lowest_shell` must be at least 1, got " + std::to_string(lowest) +
           ": shell 0 is the mean (κ = 0) mode, which a band forcing cannot legitimately drive";
  if (!(highest == INFINITY || (std::isfinite(highest) && highest == std::floor(highest))))
    return "`highest_shell` must be an integer shell or `Inf` (every retained mode but the mean), got " +
           std::to_string(highest);
  if (!(highest >= lowest))
    return "`highest_shell` must be at least `lowest_shell`, got " + std::to_string(highest) + " < " +
           std::to_string(lowest) + ": the band would be empty and the forcing would silently do nothing";
  return std::string();
}

// A field's forcing block, refused as the reference's constructors refuse it
// (src/Forcing.jl:558-572, 636-643, 828-875, 1069-1075). `who` names the field.
std::string forcing_error(const gbght_forcing_params& f, const char* who) {
  const std::string w = std::string(who) + " ";
  switch (f.kind) {
    case GBGHT_FORCING_NONE:
      return std::string();
    case GBGHT_FORCING_CONSTANT_POWER:
      if (!std::isfinite(f.rate)) return w + "ConstantPower `injection_rate` must be finite";
      break;
    case GBGHT_FORCING_LINEAR:
      if (!std::isfinite(f.rate)) return w + "Linear `rate` must be finite";
      break;
    case GBGHT_FORCING_VARIANCE_CONTROLLER:
      if (!(std::isfinite(f.target) && f.target > 0))
        return w + "VarianceController `target` must be finite and positive, got " + std::to_string(f.target) +
               ": it is the variance the controller holds, and the rate divides by the band's own variance";
      if (!(std::isfinite(f.gain) && f.gain >= 0))
        return w + "VarianceController `gain` must be finite and non-negative, got " + std::to_string(f.gain) +
               ": a negative gain makes the restoring term push the variance AWAY from the target";
      if (!finite_positive(f.turnover_time))
        return w + "VarianceController `turnover_time` must be finite and positive, got " +
               std::to_string(f.turnover_time);
      break;
    case GBGHT_FORCING_STOCHASTIC_OU:
      if (!(std::isfinite(f.target) && f.target >= 0))
        return w + "StochasticOU `forcing_variance` must be finite and non-negative, got " + std::to_string(f.target) +
               ": it is the stationary mean square of the term the forcing adds, and its square root sets the "
               "amplitude of every draw";
      if (!finite_positive(f.turnover_time))
        return w + "StochasticOU `correlation_time` must be finite and positive, got " +
               std::to_string(f.turnover_time) + ": it is the Ornstein–Uhlenbeck relaxation time T_L";
      if (!std::isfinite(f.highest_shell))
        return w + "StochasticOU needs a finite `highest_shell`, got Inf: it adds its process rather than "
                   "multiplying the field, so its band must stay below the dealias cutoff";
      break;
    case GBGHT_FORCING_VARIANCE_RESCALING:
      if (f.over != GBGHT_OVER_BAND && f.over != GBGHT_OVER_TOTAL)
        return w + "VarianceRescaling `over` must be :band or :total";
      if (!(std::isfinite(f.target) && f.target >= 0))
        return w + "VarianceRescaling `target` must be finite and non-negative, got " + std::to_string(f.target) +
               ": it is the kinetic energy or scalar variance the forcing holds, and the rescale takes its "
               "square root";
      break;
    default:
      return w + "forcing: unknown kind " + std::to_string(f.kind);
  }
  const std::string m = shell_error(f.lowest_shell, f.highest_shell);
  return m.empty() ? m : w + "forcing: " + m;
}

gbght::ForcingParams to_forcing(const gbght_forcing_params& f) {
  gbght::ForcingParams p{};
  p.kind = f.kind;
  p.rate = f.rate;
  p.target = f.target;
  p.gain = f.gain;
  p.turnover_time = f.turnover_time;
  p.over = f.over;
  p.lowest_shell = f.lowest_shell;
  p.highest_shell = f.highest_shell;
  return p;
}

void forcing_default(gbght_forcing_params* f) {
  f->kind = GBGHT_FORCING_NONE;
  f->rate = 0.0;
  f->target = 0.0;
  f->gain = 1.0;
  f->turnover_time = 0.0;
  f->over = GBGHT_OVER_BAND;
  f->lowest_shell = 1;
  f->highest_shell = 2.0;
}

int check_run(gbght_run* r) { return r ? GBGHT_OK : GBGHT_ERR_ARGUMENT; }

int require_deposit(gbght_run* r, const char* what) {
  if (r->deposit_epoch != r->fields_epoch)
    return fail(r, GBGHT_ERR_SCHEDULE,
                std::string(what) + ": the deposited velocity is stale (the fields moved since the last "
                "deposit); close each step with gbght_deposit");
  return GBGHT_OK;
}

int do_deposit(gbght_run* r) {
  double m2 = 0.0;
  int rc = engine_call(r, r->eng->deposit(&m2));
  if (rc) return rc;
  r->max_speed = std::sqrt(m2);
  r->deposit_epoch = r->fields_epoch;
  return GBGHT_OK;
}

// The trail's j-th newest sample's slot.
int trail_slot(const gbght_run* r, int j) {
  return ((r->trail_newest - j) % r->trail_capacity + r->trail_capacity) % r->trail_capacity;
}
// The slot the next sample goes to (the oldest once the ring is full).
int trail_next(const gbght_run* r) { return (r->trail_newest + 1) % r->trail_capacity; }
void trail_push(gbght_run* r, double t) {
  r->trail_newest = trail_next(r);
  r->trail_time[r->trail_newest] = t;
  if (r->trail_count < r->trail_capacity) r->trail_count += 1;
}
double trail_newest_time(const gbght_run* r) { return r->trail_time[r->trail_newest]; }

// The particle scheme's step over h from the trail (`advect!`, src/ParticlePropagator.jl:339-352):
// its own k samples once the trail holds them, else the corrected ABM of the samples present.
gbght::AdamsStep adams_step(const gbght_run* r, double h) {
  const int k = r->cfg.tracer_steps;
  const bool full = r->trail_count >= k;
  const int J = full ? k : r->trail_count;
  const bool corrected = full ? r->cfg.tracer_scheme != GBGHT_AB : true;
  double times[gbght::kTrailMax];
  gbght::AdamsStep w{};
  for (int j = 0; j < J; ++j) {
    w.slot[j] = trail_slot(r, j);
    times[j] = r->trail_time[w.slot[j]];
  }
  gbght::adams_step_weights(times, J, h, corrected, &w);
  w.out_slot = -1;
  return w;
}

int tracer_order(const gbght_config& c) { return c.tracer_scheme == GBGHT_AB ? c.tracer_steps : c.tracer_steps + 1; }

// The start-up bound under shortened_first_steps (`_startup_bound`, src/SimulationRun.jl:1117-1132):
// growth(order)·(t₀ − t₋₁) once the trail holds two samples, else τ(Δt/τ)^(order/3) with τ = √(ν/ε),
// ε the state's dissipation; infinite otherwise.
int startup_bound(gbght_run* r, double dt, double* bound) {
  const gbght_config& c = r->cfg;
  *bound = INFINITY;
  if (!(c.shortened_first_steps && c.tracers > 0 && c.tracer_steps > 1)) return GBGHT_OK;
  const int order = tracer_order(c);
  if (r->trail_count > 1) {
    const double growth = order <= 5 ? 2.0 : order <= 7 ? 1.5 : 1.25;
    *bound = growth * (r->trail_time[trail_slot(r, 0)] - r->trail_time[trail_slot(r, 1)]);
    return GBGHT_OK;
  }
  gbght::Observables o{};
  int rc = engine_call(r, r->eng->observables(&o));
  if (rc) return rc;
  const double tau = std::sqrt(c.viscosity / o.eps);
  if (std::isfinite(tau) && tau > 0) *bound = tau * std::pow(dt / tau, order / 3.0);
  return GBGHT_OK;
}

// cfl_timestep (src/SimulationRun.jl:1051-1096): the advective, resolution and caller's bounds, and
// the start-up bound.
int cfl_dt(gbght_run* r, double* out) {
  const gbght_config& c = r->cfg;
  const double dx = c.side_length / c.grid_points_per_axis;
  const double advective = r->max_speed > 0 ? c.cfl * dx / r->max_speed : c.cfl * dx;
  const double nu = c.viscosity, kap = c.viscosity / c.schmidt;
  const double D = c.scalar ? std::max(nu, kap) : nu;
  const double kmin = 2.0 * M_PI / c.side_length;
  const double resolution = 1.0 / (D * kmin * kmin);
  const double base = std::min(std::min(advective, resolution), c.max_dt);
  double bound;
  if (int rc = startup_bound(r, base, &bound)) return rc;
  *out = std::min(bound, base);
  return GBGHT_OK;
}

}  // namespace

namespace gbght {
// The message gbght_global_error() returns, set by entry points that have no run handle.
void set_global_error(const std::string& msg) { g_global_error = msg; }
}  // namespace gbght

extern "C" {

void gbght_config_default(gbght_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof *c);
  c->grid_points_per_axis = 64;
  c->side_length = 2.0 * M_PI;
  c->precision = GBGHT_FP64;
  c->scheme = GBGHT_IFRK4;
  c->viscosity = 0.01;
  c->schmidt = 1.0;
  c->scalar = 1;
  forcing_default(&c->velocity_forcing);
  forcing_default(&c->scalar_forcing);
  c->tracers = 0;
  c->tracer_scheme = GBGHT_HEUN;
  c->tracer_steps = 1;
  c->shortened_first_steps = 0;
  c->cfl = 0.5;
  c->max_dt = INFINITY;
  c->device = 0;
  c->interpolation = GBGHT_CATMULL_ROM;
  c->interpolation_points = 4;
  c->interpolation_smoothness = 1;
  c->dealiasing = GBGHT_TWO_THIRDS;
  c->houli_order = 36;
  c->houli_strength = 0.0;
  c->tracer_gather = 0;
}

int gbght_recommended_cfl_dealiased(int scheme, int dealiasing, double* cfl) {
  // `recommended_cfl(scheme, domain)` (src/Propagator.jl:915-916): the base ceiling × (2/3)/f, f the
  // retained fraction of the Nyquist wavenumber (src/SimulationDomain.jl:182-184): × 1 for TwoThirds,
  // × 2/3 for HouLi (f = 1), × 1/√2 for PhaseShift (f = 2√2/3)
  if (dealiasing != GBGHT_TWO_THIRDS && dealiasing != GBGHT_HOULI && dealiasing != GBGHT_PHASE_SHIFT)
    return GBGHT_ERR_ARGUMENT;
  const int rc = gbght_recommended_cfl(scheme, cfl);
  if (rc != GBGHT_OK) return rc;
  if (dealiasing == GBGHT_HOULI) *cfl = *cfl * 2.0 / 3.0;
  if (dealiasing == GBGHT_PHASE_SHIFT) *cfl = *cfl / std::sqrt(2.0);
  return rc;
}

int gbght_recommended_cfl(int scheme, double* cfl) {
  // `_base_cfl` (src/Propagator.jl:906-913); the 2/3 rule's factor (2/3)/(2/3) leaves it unchanged
  if (!cfl) return GBGHT_ERR_ARGUMENT;
  switch (scheme) {
    case GBGHT_IFRK4: *cfl = 0.96; return GBGHT_OK;
    case GBGHT_IFRK3: *cfl = 0.5; return GBGHT_OK;
    case GBGHT_IFSSPRK3: *cfl = 0.5; return GBGHT_OK;
    case GBGHT_IFHEUN: *cfl = 0.25; return GBGHT_OK;
    default: return GBGHT_ERR_ARGUMENT;
  }
}

const char* gbght_version(void) { return "gbght-b200 0.1.0"; }
const char* gbght_global_error(void) { return g_global_error.c_str(); }
const char* gbght_last_error(const gbght_run* r) { return r ? r->err.c_str() : "null run"; }

int gbght_create(gbght_run** out, const gbght_config* cfg) {
  if (!out || !cfg) {
    g_global_error = "null argument";
    return GBGHT_ERR_ARGUMENT;
  }
  *out = nullptr;
  auto bad = [&](const std::string& m) {
    g_global_error = m;
    return GBGHT_ERR_ARGUMENT;
  };
  if (!gbght::supported_N(cfg->grid_points_per_axis))
    return bad("grid_points_per_axis must be one of 8 12 16 24 32 48 64 96 128 192 256 384 512, got " +
               std::to_string(cfg->grid_points_per_axis));
  if (!finite_positive(cfg->side_length)) return bad("side_length must be positive and finite");
  if (!(cfg->viscosity > 0))
    return bad("`viscosity` must be positive, got " + std::to_string(cfg->viscosity) +
               ": it sets the Reynolds number through Re = 1/ν, and a non-positive value has no dissipation scale");
  if (!(cfg->schmidt > 0))
    return bad("`schmidt` must be positive, got " + std::to_string(cfg->schmidt) +
               ": the scalar diffusivity is ν/Sc, so a non-positive Schmidt number makes it infinite or negative");
  if (cfg->precision != GBGHT_FP64 && cfg->precision != GBGHT_FP32_MIXED) return bad("unknown precision");
  if (cfg->scheme != GBGHT_IFRK4 && cfg->scheme != GBGHT_IFRK3 && cfg->scheme != GBGHT_IFHEUN &&
      cfg->scheme != GBGHT_IFSSPRK3)
    return bad("unknown field integration scheme");
  {
    std::string m = forcing_error(cfg->velocity_forcing, "velocity");
    if (!m.empty()) return bad(m);
    m = forcing_error(cfg->scalar_forcing, "scalar");
    if (!m.empty()) return bad(m);
  }
  if (cfg->scalar_forcing.kind != GBGHT_FORCING_NONE && !cfg->scalar)
    return bad("a scalar forcing was given, but the run carries no scalar: set `scalar = 1`, or leave "
               "`scalar_forcing` at NoForcing");
  for (int i = 0; i < 3; ++i)
    if (!std::isfinite(cfg->mean_gradient[i])) return bad("mean_gradient must be finite");
  if (!cfg->scalar && (cfg->mean_gradient[0] != 0 || cfg->mean_gradient[1] != 0 || cfg->mean_gradient[2] != 0))
    return bad("a mean scalar gradient was given, but the run carries no scalar");
  if (cfg->tracers < 0) return bad("tracers must be non-negative");
  if (cfg->tracer_scheme == GBGHT_HEUN) {
    if (cfg->tracer_steps != 1) return bad("Heun is ABM(1): `tracer_steps` must be 1");
  } else if (cfg->tracer_scheme == GBGHT_ABM) {
    if (cfg->tracer_steps < 1 || cfg->tracer_steps > 7)
      return bad("`ABM(k)` takes a number of steps `k` from 1 to 7, got " + std::to_string(cfg->tracer_steps) +
                 ": the four-point Gauss–Legendre rule that integrates the weights is exact only through the "
                 "degree `k = 7` needs");
  } else if (cfg->tracer_scheme == GBGHT_AB) {
    if (cfg->tracer_steps < 1 || cfg->tracer_steps > 8)
      return bad("`AB(k)` takes a number of steps `k` from 1 to 8, got " + std::to_string(cfg->tracer_steps) +
                 ": the four-point Gauss–Legendre rule that integrates the weights is exact only through "
                 "degree 7");
  } else {
    return bad("unknown particle integration scheme");
  }
  gbght::Stencil stencil{};
  if (cfg->interpolation != GBGHT_CATMULL_ROM) {
    if (cfg->interpolation != GBGHT_LALESCU && cfg->interpolation != GBGHT_LAGRANGE)
      return bad("unknown interpolation scheme");
    if (const char* e = gbght::make_stencil(cfg->interpolation, cfg->interpolation_points,
                                            cfg->interpolation_smoothness, &stencil))
      return bad(e);
    if (cfg->interpolation_points > cfg->grid_points_per_axis)
      return bad("the interpolation stencil is wider than the grid");
  }
  if (cfg->dealiasing != GBGHT_TWO_THIRDS && cfg->dealiasing != GBGHT_HOULI && cfg->dealiasing != GBGHT_PHASE_SHIFT)
    return bad("unknown dealiasing strategy (TwoThirds, HouLi and PhaseShift are built)");
  if (cfg->dealiasing == GBGHT_HOULI && (cfg->houli_order < 2 || cfg->houli_order % 2 || !std::isfinite(cfg->houli_strength)))
    return bad("HouLi's `order` must be an even integer ≥ 2 and its `strength` finite");
  if (cfg->tracer_gather < 0 || cfg->tracer_gather > 2)
    return bad("tracer_gather must be 0 (automatic), 1 (per tracer) or 2 (warp-cooperative)");
  if (!finite_positive(cfg->cfl)) return bad("cfl must be positive and finite");
  if (!(cfg->max_dt > 0)) return bad("max_dt must be positive");

  auto r = std::make_unique<gbght_run>();
  r->cfg = *cfg;
  r->trail_capacity = cfg->tracer_steps;
  std::string err;
  r->eng.reset(gbght::make_engine(cfg->grid_points_per_axis, cfg->precision, cfg->dealiasing, &err));
  if (!r->eng) return bad(err);
  gbght::RunParams p{};
  p.N = cfg->grid_points_per_axis;
  p.L = cfg->side_length;
  p.precision = cfg->precision;
  p.scheme = cfg->scheme;
  p.viscosity = cfg->viscosity;
  p.schmidt = cfg->schmidt;
  p.scalar = cfg->scalar ? 1 : 0;
  p.vf = to_forcing(cfg->velocity_forcing);
  p.sf = cfg->scalar ? to_forcing(cfg->scalar_forcing) : gbght::ForcingParams{};
  for (int i = 0; i < 3; ++i) p.G[i] = cfg->mean_gradient[i];
  p.tracers = cfg->tracers;
  p.trail_capacity = cfg->tracer_steps;
  p.stencil = stencil;
  p.dealias = cfg->dealiasing;
  p.houli_order = cfg->houli_order;
  p.houli_strength = cfg->houli_strength;
  p.tracer_gather = cfg->tracer_gather;
  p.device = cfg->device;
  if (const char* e = r->eng->init(p)) {
    g_global_error = e;
    return GBGHT_ERR_CUDA;
  }
  for (int f = 0; f < 2; ++f) {   // StochasticOU's band below the dealias cutoff (src/Forcing.jl:1327-1333)
    const gbght_forcing_params& fp = f == 0 ? cfg->velocity_forcing : cfg->scalar_forcing;
    if (fp.kind != GBGHT_FORCING_STOCHASTIC_OU) continue;
    const double high = (fp.highest_shell + 0.5) * (2.0 * M_PI / cfg->side_length);
    if (!(high <= r->eng->cutoff()))
      return bad("the forcing band (shells " + std::to_string(fp.lowest_shell) + "-" +
                 std::to_string(int(fp.highest_shell)) + ") reaches |κ| = " + std::to_string(high) +
                 ", past the dealias cutoff " + std::to_string(r->eng->cutoff()) +
                 "; an additive force would fill modes the dealiasing holds empty. Lower the shells, or "
                 "enlarge the grid.");
  }
  *out = r.release();
  return GBGHT_OK;
}

void gbght_destroy(gbght_run* r) { delete r; }

int gbght_geometry(const gbght_run* r, int* K, double* cutoff) {
  if (!r) return GBGHT_ERR_ARGUMENT;
  if (K) *K = r->eng->K();
  if (cutoff) *cutoff = r->eng->cutoff();
  return GBGHT_OK;
}

int gbght_state_import(gbght_run* r, const double* u_hat, const double* phi_hat) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (!u_hat) return fail(r, GBGHT_ERR_ARGUMENT, "u_hat is null");
  if (r->cfg.scalar && !phi_hat)
    return fail(r, GBGHT_ERR_ARGUMENT, "this run carries a passive scalar, so phi_hat must be given");
  bool outside = false;
  int rc = engine_call(r, r->eng->import_state(u_hat, phi_hat, &outside));
  if (rc) return rc;
  if (outside)
    return fail(r, GBGHT_ERR_ARGUMENT,
                "the state has content outside the retained 2/3 ball; this backend stores only the "
                "retained modes (every state the seeders and steps produce is band-limited)");
  r->fields_epoch += 1;   // a new state: the deposit is stale
  return GBGHT_OK;
}

int gbght_state_export(gbght_run* r, double* u_hat, double* phi_hat) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (!u_hat) return fail(r, GBGHT_ERR_ARGUMENT, "u_hat is null");
  return engine_call(r, r->eng->export_state(u_hat, r->cfg.scalar ? phi_hat : nullptr));
}

namespace {
bool stochastic(const gbght_run* r, int f) {
  return (f == 0 ? r->cfg.velocity_forcing.kind : r->cfg.scalar_forcing.kind) == GBGHT_FORCING_STOCHASTIC_OU;
}
// A StochasticOU field's force is set once per step (prepare_forcing!, src/Forcing.jl:1401-1411).
int require_sources(gbght_run* r) {
  for (int f = 0; f < 2; ++f)
    if (stochastic(r, f) && !r->source_fresh[f])
      return fail(r, GBGHT_ERR_SCHEDULE, std::string("the ") + (f == 0 ? "velocity" : "scalar") +
                                             "'s StochasticOU force was not set for this step: advance its process "
                                             "and hand it in with gbght_forcing_source_set");
  return GBGHT_OK;
}
void consume_sources(gbght_run* r) { r->source_fresh[0] = r->source_fresh[1] = false; }
}  // namespace

int gbght_forcing_source_set(gbght_run* r, int field, const double* amplitudes, int companion_points) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (field != 0 && field != 1) return fail(r, GBGHT_ERR_ARGUMENT, "field must be 0 (velocity) or 1 (scalar)");
  if (!stochastic(r, field)) return fail(r, GBGHT_ERR_ARGUMENT, "the field carries no StochasticOU forcing");
  if (!amplitudes) return fail(r, GBGHT_ERR_ARGUMENT, "amplitudes is null");
  const char* e = r->eng->forcing_source(field, amplitudes, companion_points);
  if (e && std::strstr(e, "companion")) return fail(r, GBGHT_ERR_ARGUMENT, e);
  if (int rc = engine_call(r, e)) return rc;
  r->source_fresh[field] = true;
  return GBGHT_OK;
}

int gbght_step(gbght_run* r, double dt) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (!finite_positive(dt))
    return fail(r, GBGHT_ERR_ARGUMENT, "the timestep must be positive and finite, got " + std::to_string(dt));
  if (int rc = require_deposit(r, "step")) return rc;
  if (int rc = require_sources(r)) return rc;
  const Tableau t = tableau(r->cfg.scheme);
  int rc = engine_call(r, r->eng->step(dt, t.a, t.b, t.d, t.S));
  if (rc) return rc;
  consume_sources(r);
  r->fields_epoch += 1;
  return GBGHT_OK;
}

int gbght_deposit(gbght_run* r) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  return do_deposit(r);
}

struct gbght_ensemble {
  std::vector<gbght_run*> members;
  std::string err;
  int batching = 1;   // the most members of equal group keys that share one launch per pass (≤ 1: none)
#ifndef GBGHT_EMU
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t exec = nullptr;
  double exec_dt = 0.0;
  int units = 0;   // launching units of the captured graph (groups and lone members)
  // the batching autotuner: candidate group sizes, the one being tried, its step (0: capture and
  // run untimed, 1: timed replay), the replay times, the events that time them
  std::vector<int> tune_cands;
  size_t tune_i = 0;
  int tune_phase = 0;
  std::vector<float> tune_ms;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
#endif
};

namespace {
int ens_fail(gbght_ensemble* e, int code, const std::string& m) {
  e->err = m;
  return code;
}
#ifndef GBGHT_EMU
void ens_release_graph(gbght_ensemble* e) {
  if (e->exec) cudaGraphExecDestroy(e->exec);
  e->exec = nullptr;
}
// Capture every member's step and deposit launches as one graph. With batching on, members with
// equal group keys form a group whose first member launches each pass once for all of them (its
// launch records are built before the capture); every other member launches its own. Member 0's
// stream forks to the other launching streams through an event and joins them back at the end.
int ens_capture(gbght_ensemble* e, double dt) {
  ens_release_graph(e);
  std::vector<std::vector<gbght_run*>> units;   // a group (first member launches) or a lone member
  for (gbght_run* m : e->members) {
    const uint64_t key = e->batching >= 2 ? m->eng->group_key() : 0;
    bool placed = false;
    for (auto& u : units)
      if (key != 0 && int(u.size()) < e->batching && u[0]->eng->group_key() == key) {
        u.push_back(m);
        placed = true;
        break;
      }
    if (!placed) units.push_back({m});
  }
  for (auto& u : units) {
    if (u.size() < 2) continue;
    std::vector<gbght::Engine*> engines;
    for (gbght_run* m : u) engines.push_back(m->eng.get());
    const Tableau t = tableau(u[0]->cfg.scheme);
    if (const char* err = u[0]->eng->group_prepare(engines.data(), int(engines.size()), dt, t.a, t.b, t.d, t.S))
      return ens_fail(e, GBGHT_ERR_CUDA, err);
  }
  e->units = int(units.size());
  cudaStream_t s0 = static_cast<cudaStream_t>(e->members[0]->eng->cuda_stream());
  cudaError_t ce = cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal);
  if (ce != cudaSuccess) return ens_fail(e, GBGHT_ERR_CUDA, std::string("cudaStreamBeginCapture: ") + cudaGetErrorString(ce));
  const char* err = nullptr;
  std::string where;   // the first failing call, for the message
  auto api = [&](cudaError_t r, const char* what, size_t unit) {
    if (r != cudaSuccess && where.empty())
      where = std::string(what) + " (unit " + std::to_string(unit) + "): " + cudaGetErrorString(r);
  };
  api(cudaEventRecord(e->fork, s0), "cudaEventRecord(fork)", 0);
  for (size_t i = 1; i < units.size(); ++i)
    api(cudaStreamWaitEvent(static_cast<cudaStream_t>(units[i][0]->eng->cuda_stream()), e->fork, 0),
        "cudaStreamWaitEvent(fork)", i);
  for (size_t i = 0; i < units.size(); ++i) {
    auto& u = units[i];
    if (u.size() >= 2) {
      if (!err) err = u[0]->eng->group_launch();
    } else {
      const Tableau t = tableau(u[0]->cfg.scheme);
      if (!err) err = u[0]->eng->step(dt, t.a, t.b, t.d, t.S);
      if (!err) err = u[0]->eng->deposit_launch();
    }
    if (err && where.empty()) where = std::string(err) + " (unit " + std::to_string(i) + ")";
  }
  for (size_t i = 1; i < units.size(); ++i) {
    api(cudaEventRecord(e->join[i], static_cast<cudaStream_t>(units[i][0]->eng->cuda_stream())),
        "cudaEventRecord(join)", i);
    api(cudaStreamWaitEvent(s0, e->join[i], 0), "cudaStreamWaitEvent(join)", i);
  }
  if (!where.empty() && !err) err = "capture";
  cudaGraph_t graph = nullptr;
  ce = cudaStreamEndCapture(s0, &graph);
  if (err || ce != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return ens_fail(e, GBGHT_ERR_CUDA, !where.empty() ? where : std::string("cudaStreamEndCapture: ") + cudaGetErrorString(ce));
  }
  ce = cudaGraphInstantiate(&e->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ce != cudaSuccess) {
    e->exec = nullptr;
    return ens_fail(e, GBGHT_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ce));
  }
  e->exec_dt = dt;
  return GBGHT_OK;
}
#endif
}  // namespace

int gbght_ensemble_create(gbght_ensemble** out, gbght_run* const* members, int n) {
  if (!out || !members || n < 1) {
    g_global_error = "an ensemble needs at least one member";
    return GBGHT_ERR_ARGUMENT;
  }
  *out = nullptr;
  auto e = std::make_unique<gbght_ensemble>();
  for (int i = 0; i < n; ++i) {
    if (!members[i]) {
      g_global_error = "a member is null";
      return GBGHT_ERR_ARGUMENT;
    }
    for (gbght_run* m : e->members)
      if (m == members[i]) {
        g_global_error = "a run appears twice in the ensemble";
        return GBGHT_ERR_ARGUMENT;
      }
    if (stochastic(members[i], 0) || stochastic(members[i], 1)) {
      g_global_error = "a StochasticOU member takes its force per step; step it alone";
      return GBGHT_ERR_ARGUMENT;
    }
    if (members[i]->cfg.device != members[0]->cfg.device) {
      g_global_error = "the members must share one device";
      return GBGHT_ERR_ARGUMENT;
    }
    e->members.push_back(members[i]);
  }
#ifndef GBGHT_EMU
  cudaError_t ce = cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming);
  e->join.assign(size_t(n), nullptr);
  for (int i = 1; i < n && ce == cudaSuccess; ++i) ce = cudaEventCreateWithFlags(&e->join[i], cudaEventDisableTiming);
  if (ce != cudaSuccess) {
    g_global_error = std::string("cudaEventCreate: ") + cudaGetErrorString(ce);
    return GBGHT_ERR_CUDA;
  }
#endif
  *out = e.release();
  return GBGHT_OK;
}

void gbght_ensemble_destroy(gbght_ensemble* e) {
  if (!e) return;
#ifndef GBGHT_EMU
  ens_release_graph(e);
  if (e->t0) cudaEventDestroy(e->t0);
  if (e->t1) cudaEventDestroy(e->t1);
  if (e->fork) cudaEventDestroy(e->fork);
  for (cudaEvent_t ev : e->join)
    if (ev) cudaEventDestroy(ev);
#endif
  delete e;
}

const char* gbght_ensemble_last_error(const gbght_ensemble* e) { return e ? e->err.c_str() : "null ensemble"; }

int gbght_ensemble_set_batching(gbght_ensemble* e, int max_group) {
  if (!e || max_group < 0) return GBGHT_ERR_ARGUMENT;
  if (max_group < 1) max_group = 1;
  if (e->batching != max_group) {
    e->batching = max_group;
#ifndef GBGHT_EMU
    ens_release_graph(e);   // recaptured at the next step
#endif
  }
  return GBGHT_OK;
}

int gbght_ensemble_autotune(gbght_ensemble* e) {
  if (!e) return GBGHT_ERR_ARGUMENT;
#ifndef GBGHT_EMU
  // candidates: 1 (no batching), then 2, 4, … up to the largest set of members with one group key
  std::map<uint64_t, int> count;
  int largest = 1;
  for (gbght_run* m : e->members) {
    const uint64_t k = m->eng->group_key();
    if (k) largest = std::max(largest, ++count[k]);
  }
  e->tune_cands.clear();
  e->tune_ms.clear();
  for (int c = 1; c < largest; c *= 2) e->tune_cands.push_back(c);
  if (largest > 1) e->tune_cands.push_back(largest);
  e->tune_i = e->tune_cands.size() > 1 ? 0 : e->tune_cands.size();
  e->tune_phase = 0;
  if (!e->t0 && cudaEventCreate(&e->t0) != cudaSuccess) return ens_fail(e, GBGHT_ERR_CUDA, "cudaEventCreate");
  if (!e->t1 && cudaEventCreate(&e->t1) != cudaSuccess) return ens_fail(e, GBGHT_ERR_CUDA, "cudaEventCreate");
#endif
  return GBGHT_OK;
}

int gbght_ensemble_tuning(const gbght_ensemble* e, int* batching, int* done, float* ms, int capacity) {
  if (!e || !batching || !done) return GBGHT_ERR_ARGUMENT;
  *batching = e->batching;
#ifdef GBGHT_EMU
  *done = 1;
  (void)ms;
  (void)capacity;
#else
  *done = e->tune_i >= e->tune_cands.size();
  for (int i = 0; ms && i < capacity && size_t(i) < e->tune_ms.size(); ++i) ms[i] = e->tune_ms[i];
#endif
  return GBGHT_OK;
}

int gbght_ensemble_units(const gbght_ensemble* e, int* units) {
  if (!e || !units) return GBGHT_ERR_ARGUMENT;
#ifdef GBGHT_EMU
  *units = 0;
#else
  *units = e->exec ? e->units : 0;
#endif
  return GBGHT_OK;
}

int gbght_ensemble_step(gbght_ensemble* e, double dt) {
  if (!e) return GBGHT_ERR_ARGUMENT;
  if (!finite_positive(dt))
    return ens_fail(e, GBGHT_ERR_ARGUMENT, "the timestep must be positive and finite, got " + std::to_string(dt));
  // every member starts from a current deposit whose slots the first stage may reuse
  for (gbght_run* m : e->members) {
    if (m->deposit_epoch != m->fields_epoch || !m->eng->deposit_fresh()) {
      if (int rc = do_deposit(m)) return ens_fail(e, rc, m->err);
    }
    if (m->eng->profiling()) return ens_fail(e, GBGHT_ERR_ARGUMENT, "a member has per-launch profiling on");
  }
#ifdef GBGHT_EMU
  for (gbght_run* m : e->members) {
    const Tableau t = tableau(m->cfg.scheme);
    if (int rc = engine_call(m, m->eng->step(dt, t.a, t.b, t.d, t.S))) return ens_fail(e, rc, m->err);
    m->fields_epoch += 1;
    if (int rc = do_deposit(m)) return ens_fail(e, rc, m->err);
  }
  return GBGHT_OK;
#else
  const bool tuning = e->tune_i < e->tune_cands.size();
  if (tuning && e->tune_phase == 0 && e->batching != e->tune_cands[e->tune_i]) {
    e->batching = e->tune_cands[e->tune_i];
    ens_release_graph(e);
  }
  if (!e->exec || e->exec_dt != dt) {
    if (int rc = ens_capture(e, dt)) return rc;
    if (tuning) e->tune_phase = 0;   // a capture step is not timed
  }
  cudaStream_t s0 = static_cast<cudaStream_t>(e->members[0]->eng->cuda_stream());
  const bool timed = tuning && e->tune_phase == 1;
  cudaError_t ce = timed ? cudaEventRecord(e->t0, s0) : cudaSuccess;
  if (ce == cudaSuccess) ce = cudaGraphLaunch(e->exec, s0);
  if (ce == cudaSuccess && timed) ce = cudaEventRecord(e->t1, s0);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(s0);
  if (ce != cudaSuccess) return ens_fail(e, GBGHT_ERR_CUDA, std::string("ensemble graph: ") + cudaGetErrorString(ce));
  if (tuning) {
    if (timed) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e->t0, e->t1);
      e->tune_ms.push_back(ms);
      e->tune_i += 1;
      e->tune_phase = 0;
      if (e->tune_i == e->tune_cands.size()) {   // keep the fastest
        size_t best = 0;
        for (size_t i = 1; i < e->tune_ms.size(); ++i)
          if (e->tune_ms[i] < e->tune_ms[best]) best = i;
        if (e->batching != e->tune_cands[best]) {
          e->batching = e->tune_cands[best];
          ens_release_graph(e);
        }
      }
    } else {
      e->tune_phase = 1;
    }
  }
  for (gbght_run* m : e->members) {
    m->fields_epoch += 1;
    double m2 = 0.0;
    if (int rc = engine_call(m, m->eng->deposit_read(&m2))) return ens_fail(e, rc, m->err);
    m->max_speed = std::sqrt(m2);
    m->deposit_epoch = m->fields_epoch;
  }
  return GBGHT_OK;
#endif
}

int gbght_max_speed(gbght_run* r, double* speed) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (r->deposit_epoch < 0) return fail(r, GBGHT_ERR_SCHEDULE, "max_speed: nothing has been deposited");
  if (speed) *speed = r->max_speed;
  return GBGHT_OK;
}

int gbght_cfl_timestep(gbght_run* r, double* dt) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (r->deposit_epoch < 0) return fail(r, GBGHT_ERR_SCHEDULE, "cfl_timestep: nothing has been deposited");
  if (!std::isfinite(r->max_speed))
    return fail(r, GBGHT_ERR_SCHEDULE,
                "non-finite velocity at step " + std::to_string(r->step) + ": the run appears to have blown up");
  double D = 0.0;
  if (int rc = cfl_dt(r, &D)) return rc;
  if (dt) *dt = D;
  return GBGHT_OK;
}

int gbght_velocity_physical_export(gbght_run* r, double* u) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (!u) return fail(r, GBGHT_ERR_ARGUMENT, "u is null");
  if (r->deposit_epoch < 0) return fail(r, GBGHT_ERR_SCHEDULE, "velocity_physical: nothing has been deposited");
  return engine_call(r, r->eng->velocity_export(u));
}

int gbght_velocity_physical_import(gbght_run* r, const double* u) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (!u) return fail(r, GBGHT_ERR_ARGUMENT, "u is null");
  int rc = engine_call(r, r->eng->velocity_import(u));
  if (rc) return rc;
  r->fields_epoch += 1;
  r->deposit_epoch = r->fields_epoch;
  return GBGHT_OK;
}

int gbght_observables(gbght_run* r, double out[4]) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (!out) return fail(r, GBGHT_ERR_ARGUMENT, "out is null");
  gbght::Observables o{};
  int rc = engine_call(r, r->eng->observables(&o));
  if (rc) return rc;
  out[0] = o.k;
  out[1] = o.eps;
  out[2] = r->cfg.scalar ? o.var : NAN;
  out[3] = r->cfg.scalar ? o.chi : NAN;
  return GBGHT_OK;
}

int gbght_spectrum_length(const gbght_run* r, int* n) {
  if (!r || !n) return GBGHT_ERR_ARGUMENT;
  *n = int(std::floor(std::sqrt(3.0) * r->cfg.grid_points_per_axis / 2.0 + 0.5)) + 1;
  return GBGHT_OK;
}

int gbght_spectrum(gbght_run* r, int which, double* out, int n) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (!out || n <= 0) return fail(r, GBGHT_ERR_ARGUMENT, "out is null or empty");
  if (which != 0 && which != 1) return fail(r, GBGHT_ERR_ARGUMENT, "which must be 0 (velocity) or 1 (scalar)");
  if (which == 1 && !r->cfg.scalar) return fail(r, GBGHT_ERR_ARGUMENT, "the run carries no scalar");
  return engine_call(r, r->eng->spectrum(which, out, n));
}

int gbght_derivative_skewness(gbght_run* r, double* skewness) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (!skewness) return fail(r, GBGHT_ERR_ARGUMENT, "skewness is null");
  return engine_call(r, r->eng->skewness(skewness));
}

int gbght_energy_below_scale(gbght_run* r, double* scales, double* k, double* eps, int n) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  const int N = r->cfg.grid_points_per_axis;
  if (n < N || !k || !eps) return fail(r, GBGHT_ERR_ARGUMENT, "the outputs must hold grid_points_per_axis values");
  int rc = engine_call(r, r->eng->below_scale(r->cfg.viscosity, k, eps));
  if (rc) return rc;
  if (scales)
    for (int i = 0; i < N; ++i) scales[i] = (i + 1) * r->cfg.side_length / N;
  return GBGHT_OK;
}

int gbght_tracers_import(gbght_run* r, const double* X) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (r->cfg.tracers <= 0) return fail(r, GBGHT_ERR_ARGUMENT, "the run was built without tracers");
  if (!X) return fail(r, GBGHT_ERR_ARGUMENT, "X is null");
  int rc = engine_call(r, r->eng->tracers_set(X));
  if (rc) return rc;
  r->trail_count = 0;   // new positions: the trail starts again
  r->trail_newest = -1;
  r->sampled = false;
  r->sample_at_positions = false;
  return GBGHT_OK;
}

int gbght_tracer_trail_reset(gbght_run* r) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (r->cfg.tracers <= 0) return fail(r, GBGHT_ERR_ARGUMENT, "the run was built without tracers");
  r->trail_count = 0;
  r->trail_newest = -1;
  r->sampled = false;
  r->sample_at_positions = false;
  return GBGHT_OK;
}

int gbght_tracer_sample_restore(gbght_run* r, const double* values, double t) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (r->cfg.tracers <= 0) return fail(r, GBGHT_ERR_ARGUMENT, "the run was built without tracers");
  if (!values) return fail(r, GBGHT_ERR_ARGUMENT, "values is null");
  if (!std::isfinite(t)) return fail(r, GBGHT_ERR_ARGUMENT, "the sample time must be finite");
  if (r->trail_count > 0 && !(t > trail_newest_time(r)))
    return fail(r, GBGHT_ERR_ARGUMENT, "the sample time must be later than the previous sample's");
  int rc = engine_call(r, r->eng->tracer_sample_set(values, trail_next(r)));
  if (rc) return rc;
  trail_push(r, t);
  return GBGHT_OK;
}

int gbght_tracers_export(gbght_run* r, double* X) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (r->cfg.tracers <= 0) return fail(r, GBGHT_ERR_ARGUMENT, "the run was built without tracers");
  if (!X) return fail(r, GBGHT_ERR_ARGUMENT, "X is null");
  return engine_call(r, r->eng->tracers_get(X));
}

int gbght_tracer_sample_export(gbght_run* r, double* values, double* t) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (r->cfg.tracers <= 0) return fail(r, GBGHT_ERR_ARGUMENT, "the run was built without tracers");
  if (r->trail_count == 0) return fail(r, GBGHT_ERR_SCHEDULE, "the trail holds no sample yet");
  if (!r->sample_at_positions)
    return fail(r, GBGHT_ERR_SCHEDULE, "the trail is stale: the positions moved since its newest sample");
  if (t) *t = trail_newest_time(r);
  return values ? engine_call(r, r->eng->tracer_sample_get(values, r->trail_newest)) : GBGHT_OK;
}

int gbght_tracer_trail_export(gbght_run* r, int j, double* values, double* t) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (r->cfg.tracers <= 0) return fail(r, GBGHT_ERR_ARGUMENT, "the run was built without tracers");
  if (j < 0 || j >= r->trail_count)
    return fail(r, GBGHT_ERR_ARGUMENT, "the trail holds " + std::to_string(r->trail_count) + " sample(s); sample " +
                                           std::to_string(j) + " was asked for");
  const int slot = trail_slot(r, j);
  if (t) *t = r->trail_time[slot];
  return values ? engine_call(r, r->eng->tracer_sample_get(values, slot)) : GBGHT_OK;
}

int gbght_selftest_wait_timeout(gbght_run* r, int64_t cycles) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (cycles < 1 || cycles > 1000000000LL)
    return fail(r, GBGHT_ERR_ARGUMENT, "cycles must lie in [1, 1e9]");
  return engine_call(r, r->eng->expire_wait(static_cast<long long>(cycles)));
}

static int advect_checks(gbght_run* r, double dt) {
  if (r->cfg.tracers <= 0) return fail(r, GBGHT_ERR_ARGUMENT, "the run was built without tracers");
  if (!finite_positive(dt))
    return fail(r, GBGHT_ERR_ARGUMENT,
                "`dt` must be positive and finite, got " + std::to_string(dt) +
                    ": the samples a particle scheme integrates over must lie at increasing times");
  if (r->trail_count == 0 || !r->sample_at_positions)
    return fail(r, GBGHT_ERR_SCHEDULE, "the trail's newest sample was not taken at the current positions");
  if (int rc = require_deposit(r, "advect")) return rc;
  if (r->fields_epoch != r->sample_epoch + 1)
    return fail(r, GBGHT_ERR_SCHEDULE,
                "the fields must be exactly one step ahead of the tracer positions to advance them");
  return GBGHT_OK;
}

int gbght_advect(gbght_run* r, double dt) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (int rc = advect_checks(r, dt)) return rc;
  int rc = engine_call(r, r->eng->tracers_run(adams_step(r, dt)));
  if (rc) return rc;
  rc = engine_call(r, r->eng->sync());
  if (rc) return rc;
  r->sample_at_positions = false;
  return GBGHT_OK;
}

int gbght_deposit_tracers(gbght_run* r, double t) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (r->cfg.tracers <= 0) return fail(r, GBGHT_ERR_ARGUMENT, "the cache was built without tracers");
  if (!std::isfinite(t)) return fail(r, GBGHT_ERR_ARGUMENT, "the sample time must be finite");
  if (int rc = require_deposit(r, "deposit (particles)")) return rc;
  if (r->trail_count > 0 && !(t > trail_newest_time(r)))
    return fail(r, GBGHT_ERR_ARGUMENT, "the sample time must be later than the previous sample's");
  if (r->sampled) {
    if (r->sample_at_positions)
      return fail(r, GBGHT_ERR_SCHEDULE, "a second sample at the same positions: advance the tracers first");
    if (r->fields_epoch != r->sample_epoch + 1)
      return fail(r, GBGHT_ERR_SCHEDULE, "the fields and the tracer positions belong to different times");
  }
  gbght::AdamsStep w{};   // the gather alone, into the trail's next slot
  w.out_slot = trail_next(r);
  int rc = engine_call(r, r->eng->tracers_run(w));
  if (rc) return rc;
  rc = engine_call(r, r->eng->sync());
  if (rc) return rc;
  trail_push(r, t);
  r->sampled = true;
  r->sample_at_positions = true;
  r->sample_epoch = r->fields_epoch;
  return GBGHT_OK;
}

int gbght_interpolate_velocity(gbght_run* r, const double* X, int64_t M, double* out) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (M < 0 || (M > 0 && (!X || !out))) return fail(r, GBGHT_ERR_ARGUMENT, "bad positions or output");
  if (r->deposit_epoch < 0) return fail(r, GBGHT_ERR_SCHEDULE, "nothing has been deposited");
  return engine_call(r, r->eng->gather(X, M, out));
}

int gbght_advance(gbght_run* r, double dt, double* dt_taken) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (int rc = require_deposit(r, "advance")) return rc;
  if (dt > 0 && r->cfg.shortened_first_steps && r->cfg.tracers > 0 && r->cfg.tracer_steps > 1)
    return fail(r, GBGHT_ERR_ARGUMENT,
                "this run was built with `shortened_first_steps`, which chooses the timestep itself while the "
                "particle scheme starts, and a fixed `dt` was given: drop `dt`, or build the run without "
                "`shortened_first_steps`");
  double D = dt;
  if (!(dt > 0)) {
    if (!std::isfinite(r->max_speed))
      return fail(r, GBGHT_ERR_SCHEDULE, "non-finite velocity at step " + std::to_string(r->step) +
                                             ": the run appears to have blown up");
    if (int rc = cfl_dt(r, &D)) return rc;
  }
  if (!finite_positive(D))
    return fail(r, GBGHT_ERR_ARGUMENT, "the timestep must be positive and finite, got " + std::to_string(D));
  const double t_new = r->time + D;
  if (!(t_new > r->time))
    return fail(r, GBGHT_ERR_ARGUMENT, "the timestep is too small to advance the clock");
  const bool tracers = r->cfg.tracers > 0;
  if (tracers && (r->trail_count == 0 || !r->sample_at_positions))
    return fail(r, GBGHT_ERR_SCHEDULE, "the tracers' last push was never closed by a particle deposit");
  if (tracers && r->sample_epoch != r->fields_epoch)
    return fail(r, GBGHT_ERR_SCHEDULE, "the fields were stepped alone since the tracers' last sample");
  if (int rc = require_sources(r)) return rc;
  const Tableau t = tableau(r->cfg.scheme);
  int rc = engine_call(r, r->eng->step(D, t.a, t.b, t.d, t.S));
  if (rc) return rc;
  consume_sources(r);
  r->fields_epoch += 1;
  if ((rc = do_deposit(r))) return rc;
  if (tracers) {
    // push and closing particle deposit in one launch; the same functions as advect + deposit
    gbght::AdamsStep w = adams_step(r, D);
    w.out_slot = trail_next(r);
    rc = engine_call(r, r->eng->tracers_run(w));
    if (rc) return rc;
    trail_push(r, t_new);
    r->sample_epoch = r->fields_epoch;
    r->sample_at_positions = true;
  }
  if (!std::isfinite(r->max_speed))
    return fail(r, GBGHT_ERR_SCHEDULE, "non-finite velocity at step " + std::to_string(r->step + 1) +
                                           ": the run appears to have blown up");
  if (r->cfg.scalar) {
    double var = 0.0;
    if ((rc = engine_call(r, r->eng->scalar_variance(&var)))) return rc;
    if (!std::isfinite(var))
      return fail(r, GBGHT_ERR_SCHEDULE, "non-finite scalar at step " + std::to_string(r->step + 1) +
                                             ": the run appears to have blown up");
  }
  r->time = t_new;
  r->step += 1;
  if (dt_taken) *dt_taken = D;
  return GBGHT_OK;
}

int gbght_clock(const gbght_run* r, double* time, int64_t* step) {
  if (!r) return GBGHT_ERR_ARGUMENT;
  if (time) *time = r->time;
  if (step) *step = r->step;
  return GBGHT_OK;
}

int gbght_set_clock(gbght_run* r, double time, int64_t step) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (!std::isfinite(time) || step < 0) return fail(r, GBGHT_ERR_ARGUMENT, "bad clock");
  r->time = time;
  r->step = step;
  return GBGHT_OK;
}

int gbght_status_word(gbght_run* r, uint32_t* word) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  uint32_t w = 0;
  int rc = engine_call(r, r->eng->status(&w));
  if (rc) return rc;
  if (!std::isfinite(r->max_speed)) w |= GBGHT_STATUS_NONFINITE_SPEED;
  if (word) *word = w;
  return GBGHT_OK;
}

// ---- the discrete adjoint of the step ----------------------------------------------------------------
int gbght_adjoint_create(gbght_run* r, int snapshots) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  const gbght_config& c = r->cfg;
  if (c.scheme != GBGHT_IFRK4 && c.scheme != GBGHT_IFRK3)
    return fail(r, GBGHT_ERR_ARGUMENT, "the adjoint is built for the low-storage schemes IFLowStorageRK4 and "
                                       "IFLowStorageRK3");
  auto ok_forcing = [](int k) {
    return k == GBGHT_FORCING_NONE || k == GBGHT_FORCING_CONSTANT_POWER || k == GBGHT_FORCING_LINEAR;
  };
  if (!ok_forcing(c.velocity_forcing.kind) || (c.scalar && !ok_forcing(c.scalar_forcing.kind)))
    return fail(r, GBGHT_ERR_ARGUMENT, "the adjoint is built for NoForcing, ConstantPower and Linear forcing");
  if (c.dealiasing != GBGHT_TWO_THIRDS) return fail(r, GBGHT_ERR_ARGUMENT, "the adjoint is built for TwoThirds dealiasing");
  if (snapshots < 0 || snapshots > 64) return fail(r, GBGHT_ERR_ARGUMENT, "snapshots must lie in [0, 64]");
  return engine_call(r, r->eng->adjoint_init(snapshots));
}

int gbght_adjoint_import(gbght_run* r, const double* lam_u, const double* lam_phi) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (!lam_u) return fail(r, GBGHT_ERR_ARGUMENT, "lam_u is null");
  if (r->cfg.scalar && !lam_phi)
    return fail(r, GBGHT_ERR_ARGUMENT, "this run carries a passive scalar, so lam_phi must be given");
  bool outside = false;
  int rc = engine_call(r, r->eng->adjoint_import(lam_u, lam_phi, &outside));
  if (rc) return rc;
  if (outside)
    return fail(r, GBGHT_ERR_ARGUMENT, "the cotangent has content outside the retained 2/3 ball, where the state "
                                       "has none; the adjoint register was cleared");
  return GBGHT_OK;
}

int gbght_adjoint_export(gbght_run* r, double* lam_u, double* lam_phi) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (!lam_u) return fail(r, GBGHT_ERR_ARGUMENT, "lam_u is null");
  return engine_call(r, r->eng->adjoint_export(lam_u, r->cfg.scalar ? lam_phi : nullptr));
}

int gbght_adjoint_step(gbght_run* r, double dt) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (!finite_positive(dt))
    return fail(r, GBGHT_ERR_ARGUMENT, "the timestep must be positive and finite, got " + std::to_string(dt));
  const Tableau t = tableau(r->cfg.scheme);
  return engine_call(r, r->eng->adjoint_step(dt, t.a, t.b, t.d, t.S));
}

int gbght_adjoint_add_observable(gbght_run* r, int which, double weight) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (!std::isfinite(weight)) return fail(r, GBGHT_ERR_ARGUMENT, "the weight must be finite");
  const double n = r->cfg.grid_points_per_axis, n6 = n * n * n * n * n * n;
  if (which == GBGHT_OBSERVABLE_KINETIC_ENERGY) return engine_call(r, r->eng->adjoint_add(weight / n6, 0.0));
  if (which == GBGHT_OBSERVABLE_SCALAR_VARIANCE) {
    if (!r->cfg.scalar) return fail(r, GBGHT_ERR_ARGUMENT, "the run carries no scalar");
    return engine_call(r, r->eng->adjoint_add(0.0, 2.0 * weight / n6));
  }
  return fail(r, GBGHT_ERR_ARGUMENT, "unknown observable");
}

int gbght_adjoint_forcing_gradient(gbght_run* r, double out[2], int reset) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  double g[2] = {0.0, 0.0};
  int rc = engine_call(r, r->eng->adjoint_gradient(g, reset));
  if (rc) return rc;
  if (out) {
    out[0] = g[0];
    out[1] = g[1];
  }
  return GBGHT_OK;
}

int gbght_adjoint_clear(gbght_run* r) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  return engine_call(r, r->eng->adjoint_clear());
}

int gbght_snapshot_save(gbght_run* r, int slot) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  const bool tr = r->cfg.tracers > 0;
  if (tr && (r->trail_count == 0 || !r->sample_at_positions))
    return fail(r, GBGHT_ERR_SCHEDULE, "a snapshot of a run with tracers needs the newest sample at the positions");
  const char* e = r->eng->snapshot_save(slot, tr ? r->trail_newest : 0);
  if (e && std::strstr(e, "snapshot")) return fail(r, GBGHT_ERR_ARGUMENT, e);
  if (int rc = engine_call(r, e)) return rc;
  if (size_t(slot) >= r->snap_time.size()) {
    r->snap_time.resize(slot + 1);
    r->snap_step.resize(slot + 1);
    r->snap_sample_time.resize(slot + 1);
  }
  r->snap_time[slot] = r->time;
  r->snap_step[slot] = r->step;
  r->snap_sample_time[slot] = tr ? trail_newest_time(r) : 0.0;
  return GBGHT_OK;
}

int gbght_snapshot_load(gbght_run* r, int slot) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (slot < 0 || size_t(slot) >= r->snap_time.size()) return fail(r, GBGHT_ERR_ARGUMENT, "no such snapshot slot");
  const bool tr = r->cfg.tracers > 0;
  if (tr && r->trail_newest < 0) return fail(r, GBGHT_ERR_SCHEDULE, "the tracers' trail is empty");
  const char* e = r->eng->snapshot_load(slot, tr ? r->trail_newest : 0);
  if (e && std::strstr(e, "snapshot")) return fail(r, GBGHT_ERR_ARGUMENT, e);
  int rc = engine_call(r, e);
  if (rc) return rc;
  r->fields_epoch += 1;   // a new state: the deposit is stale
  r->time = r->snap_time[slot];
  r->step = r->snap_step[slot];
  if (tr) {   // the trail holds the snapshot's newest sample, at the restored positions
    r->trail_count = 1;
    r->trail_time[r->trail_newest] = r->snap_sample_time[slot];
    r->sampled = true;
    r->sample_at_positions = true;
    r->sample_epoch = r->fields_epoch;
  }
  return GBGHT_OK;
}

int gbght_adjoint_advance(gbght_run* r, double dt) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (r->cfg.tracers <= 0 || r->cfg.tracer_scheme != GBGHT_HEUN || r->cfg.interpolation != GBGHT_CATMULL_ROM)
    return fail(r, GBGHT_ERR_ARGUMENT, "the adjoint of an iteration's tracer push is built for Heun tracers with "
                                       "CatmullRom interpolation");
  if (!finite_positive(dt))
    return fail(r, GBGHT_ERR_ARGUMENT, "the timestep must be positive and finite, got " + std::to_string(dt));
  if (r->trail_count == 0 || !r->sample_at_positions)
    return fail(r, GBGHT_ERR_SCHEDULE, "the trail's newest sample was not taken at the current positions");
  const Tableau t = tableau(r->cfg.scheme);
  gbght::AdamsStep w = adams_step(r, dt);
  int rc = engine_call(r, r->eng->adjoint_step(dt, t.a, t.b, t.d, t.S, &w, r->trail_newest));
  if (rc) return rc;
  r->deposit_epoch = r->fields_epoch;   // the deposit of the state was rebuilt
  return GBGHT_OK;
}

int gbght_adjoint_tracers_import(gbght_run* r, const double* lam_X, const double* lam_f) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (!lam_X || !lam_f) return fail(r, GBGHT_ERR_ARGUMENT, "lam_X and lam_f must be given");
  return engine_call(r, r->eng->adjoint_tracers_import(lam_X, lam_f));
}

int gbght_adjoint_tracers_export(gbght_run* r, double* lam_X, double* lam_f) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (!lam_X || !lam_f) return fail(r, GBGHT_ERR_ARGUMENT, "lam_X and lam_f must be given");
  return engine_call(r, r->eng->adjoint_tracers_export(lam_X, lam_f));
}

int gbght_adjoint_deposit_tracers(gbght_run* r) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (r->cfg.interpolation != GBGHT_CATMULL_ROM)
    return fail(r, GBGHT_ERR_ARGUMENT, "the adjoint of the particle deposit is built for CatmullRom interpolation");
  if (int rc = require_deposit(r, "adjoint of the particle deposit")) return rc;
  return engine_call(r, r->eng->adjoint_deposit_tracers());
}

int gbght_profile(gbght_run* r, int enable) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  return engine_call(r, r->eng->profile(enable));
}

int gbght_profile_read(gbght_run* r, int kind, int64_t* launches, double* total_ms) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  int64_t n = 0;
  double ms = 0.0;
  const char* e = r->eng->profile_read(kind, &n, &ms);
  if (e) return fail(r, GBGHT_ERR_ARGUMENT, e);
  if (launches) *launches = n;
  if (total_ms) *total_ms = ms;
  return GBGHT_OK;
}

int gbght_timer(gbght_run* r, int op, double* ms) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  if (op != 0 && op != 1) return fail(r, GBGHT_ERR_ARGUMENT, "op must be 0 (start) or 1 (stop)");
  return engine_call(r, r->eng->timer(op, ms));
}

int gbght_synchronize(gbght_run* r) {
  if (check_run(r)) return GBGHT_ERR_ARGUMENT;
  return engine_call(r, r->eng->sync());
}

}  // extern "C"
