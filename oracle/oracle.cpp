// CPU oracle for the brian2cuda hot path — TEST INFRASTRUCTURE ONLY.
//
// This file restates, as plain sequential C++ (OpenMP only on independent per-neuron
// loops), the algorithm brian2cuda generates for the hot path.  It is the checker the
// GPU library is compared against; it is never linked into or called by the product.
// Only tests/, __graft_entry__.smoke() and bench.py (CPU baseline arm) load it.
//
// It follows the reference's structure, not the GPU design:
//   * Brian2's schedule per step: all state updates, all thresholds, every synaptic
//     pathway (on_pre pathways, then on_post pathways; each one advance + push + deliver),
//     all resets, then the clock tick (templates/network.cu:65-115, clocks.h:33-37).
//   * Spike queues: `CudaSpikeQueue` with one post block (brianlib/spikequeue.h):
//     advance() clears slot current_offset and moves to the next slot (504-511);
//     push_bundles() appends each bundle id of a spiking neuron to slot
//     (current_offset + delay) % num_queues (432-502); the effect code then walks the
//     bundles of slot current_offset (peek, 513-516; templates/synapses.cu:117-162).
//     num_queues = max_delay + 1 (templates/synapses_push_spikes.cu:392-393); bundles are
//     the synapses of one presynaptic neuron with one delay, in synapse order
//     (synapses_push_spikes.cu:460-544).
//   * Spikespace: thresholder appends spiking indices (templates/threshold.cu:19-45); here
//     in ascending order, the canonical form.
//   * Refractoriness: not_refractory = timestep(t - lastspike) >= timestep(refractory)
//     with timestep(t, dt) = (int64)((t + 1e-3 dt)/dt) (cuda_generator.py:997-1006);
//     threshold `cond and not_refractory`; on a spike not_refractory = false and
//     lastspike = t (threshold.cu:37-42).  lastspike starts at -1e4 s.
//   * Integrators: the exact propagator of the linear LIF (examples/cuba.py:125-132) and
//     Brian2's exponential Euler for COBAHH (examples/cobahh.py:159-180); rate functions of
//     the form c*x/(exp(x/a) - 1) through Brian2's exprel (z_over_expm1 below), which keeps
//     their removable singularity finite (the literal form is 0/0 there).
//   * Event-driven STDP (examples/stdp.py:125-186) with float32 elapsed time in float32
//     mode (brian2cuda/device.py:1034-1039); clip as cuda_generator.py:902-914.
//   * Hines solver: the domain-decomposition method of brian2cuda/templates/
//     spatialstateupdate.cu (matrix 36-77, per-section solves 128-192, branch-point system
//     202-307, combination 316-351, currents 359-387), restated from the cable equation
//     (see the Hines section below).
//   * Philox-4x32-10 connectivity generation restated from Salmon et al., SC 2011.
//   * Inputs: TimedArray values held over each interval of the array's dt, clamped to the
//     last row (brian2cuda/timedarray.py:10-58), as a LIF drive, an HH current or a
//     PoissonGroup rate; PoissonInput as weight * Binomial(N, rate dt) per neuron and step
//     in the synapses slot (the BinomialFunction of brian2cuda/binomial.py:12-121), drawn
//     by sequential-search inversion from one Philox word; SpikeGeneratorGroup periods
//     (templates/spikegenerator.cu:42-49: step t emits the entries of step t mod period).
//   * Monitors: StateMonitor at the start of a step, PopulationRateMonitor at its end
//     (templates/statemonitor.cu, templates/ratemonitor.cu).
//
// Arithmetic: R = double (reference mode) or float (same-precision mode).
#include <stdint.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace {

enum { LIF = 1, HH = 2, POISSON = 3, SPIKEGEN = 4, MODEL = 5 };

// A group whose arithmetic a caller supplies (generated models): phase 0 advances the state
// vars[nv][n] by one step (mask = not_refractory in, normals = the step's normal numbers
// [nn][n]), phase 1 writes the threshold condition into mask, phase 2 resets the n_idx
// neurons idx.  Returns 0 on success.
typedef int (*ModelFn)(void* user, int phase, int64_t ts, double t, double dt, int64_t n,
                       double* vars, uint8_t* mask, const int32_t* idx, int64_t n_idx,
                       const double* normals);
enum { V = 0, GE = 1, GI = 2, M = 3, H = 4, N = 5, LASTSPIKE = 6, NOT_REF = 7 };
enum { ADD = 1, STDP = 2 };
enum { SYN_I = 0, SYN_J = 1, SYN_DELAY = 2, SYN_W = 3, SYN_APRE = 4, SYN_APOST = 5, SYN_LU = 6 };

int64_t timestep(double t, double dt) { return (int64_t)((t + 1e-3 * dt) / dt); }

inline float xexp(float x) { return std::exp(x); }
inline double xexp(double x) { return std::exp(x); }
inline float xfma(float a, float b, float c) { return std::fma(a, b, c); }
inline float xexpm1(float x) { return std::expm1(x); }
inline double xexpm1(double x) { return std::expm1(x); }
// x/(exp(x) - 1) = 1/exprel(x), Brian2's exprel (brian2cuda/cuda_generator.py:858-867): the
// removable singularity at 0 takes its limit.  The COBAHH and HH-1952 rate functions written
// as c*x/(exp(x/a) - 1) are evaluated as c*a*z_over_expm1(x/a).
template <typename R>
R z_over_expm1(R z) {
  return std::fabs(z) < (R)1e-16 ? (R)1 : z / xexpm1(z);
}
inline double xfma(double a, double b, double c) { return std::fma(a, b, c); }

template <typename R>
R clip(R v, R lo, R hi) {
  if (v < lo) return lo;
  if (v > hi) return hi;
  return v;
}

// ---- Philox-4x32-10 ----------------------------------------------------------------------
struct Ctr { uint32_t v[4]; };
Ctr philox(Ctr c, uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c.v[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.v[2];
    Ctr n;
    n.v[0] = (uint32_t)(p1 >> 32) ^ c.v[1] ^ k0;
    n.v[1] = (uint32_t)p1;
    n.v[2] = (uint32_t)(p0 >> 32) ^ c.v[3] ^ k1;
    n.v[3] = (uint32_t)p0;
    c = n;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// ---- groups --------------------------------------------------------------------------------
template <typename R>
struct Group {
  int kind = 0;
  int64_t n = 0;
  // LIF: El taum taue taui ke ki Vt Vr refractory has_threshold has_reset unless_refractory
  // HH : Cm gl El EK ENa gNa gK VT Ee Ei taue taui Vthr refractory
  std::vector<double> p;
  double rate = 0;
  std::vector<R> var[7];
  std::vector<uint8_t> not_ref;
  std::vector<int32_t> spikes;  // spikespace of the current step, ascending
  std::vector<std::pair<int64_t, int32_t>> sg;  // spike generator (step, idx), sorted
  int64_t sg_period = 0;                        // > 0: the entries repeat every period steps
  std::vector<std::vector<R>> uniforms;         // Poisson: queued rows, one per step
  size_t uni_next = 0;
  std::vector<std::pair<int64_t, int32_t>> recorded;  // (step, idx)
  // TimedArray input (brian2cuda/timedarray.py:10-58): values [rows][cols] held over each
  // interval of the array's dt; step ts reads row min(ts * mul / div, rows - 1), the
  // interval holding t = ts dt on aligned time grids; one column or one per neuron.
  std::vector<R> ta;
  int64_t ta_rows = 0, ta_cols = 0, ta_mul = 1, ta_div = 1;
  // PoissonInputs: (target variable, N, rate*dt, weight, stream id)
  struct PIn {
    int var;
    int64_t n;
    double p, w;
    uint32_t id;
  };
  std::vector<PIn> pins;
  // MODEL: the caller's arithmetic, its variable count, normal draws per step, refractory
  // period, reset flag and the queued normal numbers (one row of nn*n per step)
  ModelFn model_fn = nullptr;
  void* model_user = nullptr;
  int model_nv = 0, model_nn = 0, model_reset = 0, model_thr = 0;
  double model_ref = 0;
  std::vector<std::vector<double>> normals;
  size_t nrm_next = 0;
  R input(int64_t ts, int64_t i) const {
    if (ta.empty()) return (R)0;
    const int64_t row = std::min(ts * ta_mul / ta_div, ta_rows - 1);
    return ta[row * ta_cols + (ta_cols == 1 ? 0 : i)];
  }
  double refractory() const {
    if (kind == LIF) return p[8];
    if (kind == HH) return p[13];
    if (kind == MODEL) return model_ref;
    return 0;
  }
};

// ---- pathways ------------------------------------------------------------------------------
template <typename R>
struct Syn {
  int pre = -1, post = -1, target = 0, effect = 0;
  int64_t n = 0;
  std::vector<int32_t> i, j, delay;
  std::vector<R> w, apre, apost, lu;
  R w_scalar = 0;
  bool has_w = false;
  double stdp[7] = {0};  // taupre taupost dApre dApost wmin wmax pre_adds_weight
  // bundles: (pre, delay) -> synapse ids in synapse order
  int max_delay = 0;
  std::vector<int64_t> bundle_off;       // [n_pre * (max_delay+1) + 1]
  std::vector<int64_t> bundle_syn;
  // queue
  int num_queues = 1;
  int current_offset = 0;
  std::vector<std::vector<int64_t>> queue;  // slot -> bundle ids (key = pre*(D+1)+delay)
  // on_post (delay 0): synapses by post
  std::vector<int64_t> post_off, post_syn;
  // deliveries still due from before a change of delays: (step, synapse)
  std::vector<std::pair<int64_t, int64_t>> legacy;
};

// StateMonitor (brian2cuda/templates/statemonitor.cu: one value per recorded index per tick
// of the monitor's clock) recording at the start of a step, before the groups update
// (Brian2's default when='start'), at every step divisible by `every`.
struct StateMon {
  int gid = -1, var = 0, every = 1;
  std::vector<int64_t> idx;
  std::vector<int64_t> steps;
  std::vector<double> vals;   // [records][idx]
};
// PopulationRateMonitor (templates/ratemonitor.cu): the group's spike count of every step,
// after the synaptic effects and resets (when='end'); rate = count / (N dt).
struct RateMon {
  int gid = -1;
  std::vector<int64_t> steps;
  std::vector<int64_t> counts;
};

// Dynamic state of a net (Network.store()/restore()): group variables and spikespaces,
// Poisson read positions, delay queues and STDP synapse variables.  Monitors keep their
// records across a restore, as the GPU library's do.
template <typename R>
struct NetSnap {
  bool valid = false;
  int64_t ts = 0;
  std::vector<std::array<std::vector<R>, 7>> var;
  std::vector<std::vector<uint8_t>> not_ref;
  std::vector<std::vector<int32_t>> spikes;
  std::vector<size_t> uni_next;
  std::vector<std::vector<std::vector<int64_t>>> queue;
  std::vector<int> current_offset;
  std::vector<std::vector<R>> w, apre, apost, lu;
};

template <typename R>
struct Net {
  double dt;
  int64_t ts = 0;
  std::vector<Group<R>> groups;
  std::vector<Syn<R>> syns;
  std::vector<StateMon> smons;
  std::vector<RateMon> rmons;
  bool built = false;
  bool reset_first = false;   // schedule: thresholds, resets, synapses
  uint64_t seed = 0;          // the net's seed (PoissonInput streams)
  int32_t n_pins = 0;
  NetSnap<R> snap;
  std::string err;
};

template <typename R>
void build_syn(Net<R>& net, Syn<R>& s) {
  const int64_t npre = net.groups[s.pre].n;
  const int D = s.max_delay + 1;
  s.bundle_off.assign(npre * D + 1, 0);
  for (int64_t k = 0; k < s.n; ++k) s.bundle_off[(int64_t)s.i[k] * D + s.delay[k] + 1]++;
  for (size_t q = 1; q < s.bundle_off.size(); ++q) s.bundle_off[q] += s.bundle_off[q - 1];
  s.bundle_syn.assign(s.n, 0);
  std::vector<int64_t> fill(s.bundle_off.begin(), s.bundle_off.end() - 1);
  for (int64_t k = 0; k < s.n; ++k) s.bundle_syn[fill[(int64_t)s.i[k] * D + s.delay[k]]++] = k;
  s.num_queues = D;
  s.current_offset = 0;
  s.queue.assign(D, {});
  if (s.effect == STDP) {
    const int64_t npost = net.groups[s.post].n;
    s.post_off.assign(npost + 1, 0);
    for (int64_t k = 0; k < s.n; ++k) s.post_off[s.j[k] + 1]++;
    for (int64_t q = 1; q <= npost; ++q) s.post_off[q] += s.post_off[q - 1];
    s.post_syn.assign(s.n, 0);
    std::vector<int64_t> f(s.post_off.begin(), s.post_off.end() - 1);
    for (int64_t k = 0; k < s.n; ++k) s.post_syn[f[s.j[k]]++] = k;
    s.apre.assign(s.n, 0);
    s.apost.assign(s.n, 0);
    s.lu.assign(s.n, 0);
  }
}

// ---- one step -------------------------------------------------------------------------------
// dv/dt = (El + u - v + ke ge + ki gi)/taum with u the TimedArray input, constant over the
// step: the exact propagator with El + u in place of El.
template <typename R>
void update_lif(Group<R>& g, int64_t ts, double t, double dt) {
  const double El = g.p[0], taum = g.p[1], taue = g.p[2], taui = g.p[3], ke = g.p[4], ki = g.p[5];
  const bool leak = std::isfinite(taum) && taum > 0;
  const double A = leak ? std::exp(-dt / taum) : 1.0;
  const double De = taue > 0 ? std::exp(-dt / taue) : 0.0;
  const double Di = taui > 0 ? std::exp(-dt / taui) : 0.0;
  auto coupling = [&](double k, double tau, double D) {
    if (k == 0.0 || !leak) return 0.0;
    if (tau == taum) return k * (dt / taum) * A;
    return k * tau / (tau - taum) * (D - A);
  };
  const double Be = coupling(ke, taue, De), Bi = coupling(ki, taui, Di);
  const R rA = (R)A, rBe = (R)Be, rBi = (R)Bi, rDe = (R)De, rDi = (R)Di, rEl = (R)El;
  const double refr = g.p[8];
  const int64_t ref_steps = refr > 0 ? timestep(refr, dt) : -1;
  const bool unless = g.p[11] != 0;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < g.n; ++i) {
    bool nr = true;
    if (ref_steps >= 0) nr = timestep(t - (double)g.var[LASTSPIKE][i], dt) >= ref_steps;
    const R v = g.var[V][i], ge = g.var[GE][i], gi = g.var[GI][i];
    const R El_u = rEl + g.input(ts, i);
    R vn = xfma(rBi, gi, xfma(rBe, ge, xfma(rA, (R)(v - El_u), El_u)));
    if (unless && !nr) vn = v;
    g.var[V][i] = vn;
    g.var[GE][i] = rDe * ge;
    g.var[GI][i] = rDi * gi;
    g.not_ref[i] = nr ? 1 : 0;
  }
}

template <typename R>
R expeuler(R x, R A, R B, R dt) {
  const R BA = B / A;
  return -BA + (BA + x) * xexp(A * dt);
}

// The TimedArray input enters as an external current: Cm dv/dt = ... + I.
template <typename R>
void update_hh(Group<R>& g, int64_t ts, double t, double dt) {
  const R Cm = (R)g.p[0], gl = (R)g.p[1], El = (R)g.p[2], EK = (R)g.p[3], ENa = (R)g.p[4];
  const R gNa = (R)g.p[5], gK = (R)g.p[6], VT = (R)g.p[7], Ee = (R)g.p[8], Ei = (R)g.p[9];
  const R De = (R)std::exp(-dt / g.p[10]), Di = (R)std::exp(-dt / g.p[11]);
  const R dtR = (R)dt;
  const double refr = g.p[13];
  const int64_t ref_steps = refr > 0 ? timestep(refr, dt) : -1;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < g.n; ++i) {
    bool nr = true;
    if (ref_steps >= 0) nr = timestep(t - (double)g.var[LASTSPIKE][i], dt) >= ref_steps;
    const R v = g.var[V][i], m = g.var[M][i], h = g.var[H][i], n = g.var[N][i];
    const R ge = g.var[GE][i], gi = g.var[GI][i];
    // examples/cobahh.py:169-180 in SI units
    const R am = (R)1280 * z_over_expm1(((R)13e-3 - v + VT) / (R)4e-3);
    const R bm = (R)1400 * z_over_expm1((v - VT - (R)40e-3) / (R)5e-3);
    const R ah = (R)128 * xexp(((R)17e-3 - v + VT) / (R)18e-3);
    const R bh = (R)4000 / ((R)1 + xexp(((R)40e-3 - v + VT) / (R)5e-3));
    const R an = (R)160 * z_over_expm1(((R)15e-3 - v + VT) / (R)5e-3);
    const R bn = (R)500 * xexp(((R)10e-3 - v + VT) / (R)40e-3);
    const R gna = gNa * (m * m * m) * h;
    const R gk = gK * (n * n * n * n);
    const R Av = -(gl + ge + gi + gna + gk) / Cm;
    const R Bv = (gl * El + ge * Ee + gi * Ei + gna * ENa + gk * EK + g.input(ts, i)) / Cm;
    g.var[V][i] = expeuler(v, Av, Bv, dtR);
    g.var[M][i] = expeuler(m, -(am + bm), am, dtR);
    g.var[H][i] = expeuler(h, -(ah + bh), ah, dtR);
    g.var[N][i] = expeuler(n, -(an + bn), an, dtR);
    g.var[GE][i] = De * ge;
    g.var[GI][i] = Di * gi;
    g.not_ref[i] = nr ? 1 : 0;
  }
}

// Runs a phase of a MODEL group's callback on a double copy of its variables.
template <typename R>
bool model_phase(Net<R>& net, Group<R>& g, int phase, double t, uint8_t* mask,
                 const std::vector<int32_t>* idx) {
  const int64_t n = g.n;
  std::vector<double> x((size_t)g.model_nv * n);
  for (int v = 0; v < g.model_nv; ++v)
    for (int64_t i = 0; i < n; ++i) x[(size_t)v * n + i] = (double)g.var[v][i];
  const double* nrm = nullptr;
  if (phase == 0 && g.model_nn > 0) {
    if (g.nrm_next >= g.normals.size()) {
      net.err = "model group ran out of normal numbers";
      return false;
    }
    nrm = g.normals[g.nrm_next++].data();
  }
  const int rc = g.model_fn(g.model_user, phase, net.ts, t, net.dt, n, x.data(), mask,
                            idx ? idx->data() : nullptr, idx ? (int64_t)idx->size() : 0, nrm);
  if (rc != 0) {
    net.err = "model callback failed";
    return false;
  }
  if (phase != 1)
    for (int v = 0; v < g.model_nv; ++v)
      for (int64_t i = 0; i < n; ++i) g.var[v][i] = (R)x[(size_t)v * n + i];
  return true;
}

template <typename R>
bool update_model(Net<R>& net, Group<R>& g, double t) {
  const double refr = g.refractory();
  const int64_t ref_steps = refr > 0 ? timestep(refr, net.dt) : -1;
  for (int64_t i = 0; i < g.n; ++i) {
    bool nr = true;
    if (ref_steps >= 0) nr = timestep(t - (double)g.var[LASTSPIKE][i], net.dt) >= ref_steps;
    g.not_ref[i] = nr ? 1 : 0;
  }
  return model_phase(net, g, 0, t, g.not_ref.data(), nullptr);
}

template <typename R>
bool threshold(Net<R>& net, Group<R>& g, double t) {
  g.spikes.clear();
  if (g.kind == MODEL) {
    if (g.model_thr) {
      std::vector<uint8_t> cond(g.n, 0);
      if (!model_phase(net, g, 1, t, cond.data(), nullptr)) return false;
      const bool refr = g.refractory() > 0;
      for (int64_t i = 0; i < g.n; ++i) {
        if (cond[i] && (!refr || g.not_ref[i])) {
          g.spikes.push_back((int32_t)i);
          if (refr) {
            g.not_ref[i] = 0;
            g.var[LASTSPIKE][i] = (R)t;
          }
        }
      }
    }
  } else if (g.kind == LIF || g.kind == HH) {
    const bool has_thr = g.kind == HH || g.p[9] != 0;
    if (!has_thr) return true;
    const R thr = (R)(g.kind == LIF ? g.p[6] : g.p[12]);
    const bool refr = g.refractory() > 0;
    for (int64_t i = 0; i < g.n; ++i) {
      const bool cond = g.var[V][i] > thr && (!refr || g.not_ref[i]);
      if (cond) {
        g.spikes.push_back((int32_t)i);
        if (refr) {
          g.not_ref[i] = 0;
          g.var[LASTSPIKE][i] = (R)t;
        }
      }
    }
  } else if (g.kind == POISSON) {
    if (g.uni_next >= g.uniforms.size()) {
      net.err = "Poisson group ran out of uniforms";
      return false;
    }
    const std::vector<R>& u = g.uniforms[g.uni_next++];
    const R thr = (R)(g.rate * net.dt);
    for (int64_t i = 0; i < g.n; ++i) {
      // a TimedArray gives the rate in Hz: u < rate(t) dt
      const R th = g.ta.empty() ? thr : (R)((double)g.input(net.ts, i) * net.dt);
      if (u[i] < th) g.spikes.push_back((int32_t)i);
    }
  } else if (g.kind == SPIKEGEN) {
    // with a period, step ts emits the entries of step ts mod period
    const int64_t bin = g.sg_period > 0 ? net.ts % g.sg_period : net.ts;
    auto lo = std::lower_bound(g.sg.begin(), g.sg.end(), std::make_pair(bin, (int32_t)-1));
    for (auto it = lo; it != g.sg.end() && it->first == bin; ++it) g.spikes.push_back(it->second);
  }
  for (int32_t i : g.spikes) g.recorded.emplace_back(net.ts, i);
  return true;
}

template <typename R>
void pathway_pre(Net<R>& net, Syn<R>& s, double t) {
  // advance
  s.queue[s.current_offset].clear();
  s.current_offset = (s.current_offset + 1) % s.num_queues;
  // push
  const int D = s.max_delay + 1;
  for (int32_t pre : net.groups[s.pre].spikes) {
    for (int d = 0; d < D; ++d) {
      const int64_t key = (int64_t)pre * D + d;
      if (s.bundle_off[key + 1] > s.bundle_off[key])
        s.queue[(s.current_offset + d) % s.num_queues].push_back(key);
    }
  }
  // deliver
  Group<R>& tgt = net.groups[s.post];
  std::vector<R>& T = tgt.var[s.target];
  const R taupre = (R)s.stdp[0], taupost = (R)s.stdp[1], dApre = (R)s.stdp[2];
  const R wmin = (R)s.stdp[4], wmax = (R)s.stdp[5];
  const bool adds = s.stdp[6] != 0;
  if (!s.legacy.empty()) {
    // spikes sent before a change of delays arrive with the delay they were sent with
    for (const auto& e : s.legacy)
      if (e.first == net.ts) T[s.j[e.second]] += s.has_w ? s.w[e.second] : s.w_scalar;
    s.legacy.erase(std::remove_if(s.legacy.begin(), s.legacy.end(),
                                  [&](const auto& e) { return e.first <= net.ts; }),
                   s.legacy.end());
  }
  for (int64_t key : s.queue[s.current_offset]) {
    for (int64_t q = s.bundle_off[key]; q < s.bundle_off[key + 1]; ++q) {
      const int64_t k = s.bundle_syn[q];
      if (s.effect == ADD) {
        T[s.j[k]] += s.has_w ? s.w[k] : s.w_scalar;
      } else {
        const R tau = (R)(t - (double)s.lu[k]);
        R apre = s.apre[k] * xexp(-tau / taupre);
        R apost = s.apost[k] * xexp(-tau / taupost);
        const R w = s.w[k];
        if (adds) T[s.j[k]] += w;
        apre = apre + dApre;
        s.w[k] = clip(w + apost, wmin, wmax);
        s.apre[k] = apre;
        s.apost[k] = apost;
        s.lu[k] = (R)t;
      }
    }
  }
}

template <typename R>
void pathway_post(Net<R>& net, Syn<R>& s, double t) {
  const R taupre = (R)s.stdp[0], taupost = (R)s.stdp[1], dApost = (R)s.stdp[3];
  const R wmin = (R)s.stdp[4], wmax = (R)s.stdp[5];
  // Each synapse has one postsynaptic neuron, so the spiking neurons' synapse sets are
  // disjoint and the per-synapse updates are the same in any order of the neurons.
  const std::vector<int32_t>& spk = net.groups[s.post].spikes;
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t x = 0; x < (int64_t)spk.size(); ++x) {
    const int32_t j = spk[x];
    for (int64_t q = s.post_off[j]; q < s.post_off[j + 1]; ++q) {
      const int64_t k = s.post_syn[q];
      const R tau = (R)(t - (double)s.lu[k]);
      R apre = s.apre[k] * xexp(-tau / taupre);
      R apost = s.apost[k] * xexp(-tau / taupost);
      apost = apost + dApost;
      s.w[k] = clip(s.w[k] + apre, wmin, wmax);
      s.apre[k] = apre;
      s.apost[k] = apost;
      s.lu[k] = (R)t;
    }
  }
}

// Binomial(n, p) by sequential-search inversion (Devroye 1986, ch. X.4): u uniform in (0, 1)
// from word 0 of Philox(counter = (neuron, step low, step high, id), key = (seed low,
// seed high ^ 0xB1A0)); P(X = 0) = q^n, P(X = x) = P(X = x - 1) ((n + 1) s / x - s) with
// s = p / q; p above 1/2 is drawn as n minus a Binomial(n, 1 - p).  Plain double
// arithmetic in the order written (the build does not contract it into fused operations).
int64_t binomial_draw(int64_t n, double p, uint64_t seed, uint32_t id, int64_t ts, int64_t i) {
  const bool rev = p > 0.5;
  const double pp = rev ? 1.0 - p : p;
  const double q = 1.0 - pp;
  const double qn = std::pow(q, (double)n);
  const double s = q > 0 ? pp / q : 0.0;
  const double a = (double)(n + 1) * s;
  const Ctr w = philox(Ctr{{(uint32_t)i, (uint32_t)ts, (uint32_t)((uint64_t)ts >> 32), id}},
                       (uint32_t)seed, (uint32_t)(seed >> 32) ^ 0xB1A0u);
  double u = ((double)w.v[0] + 0.5) * 0x1p-32;
  double r = qn;
  int64_t x = 0;
  while (u > r && x < n) {
    u = u - r;
    ++x;
    r = r * (a / (double)x - s);
  }
  return rev ? n - x : x;
}

// Brian2's PoissonInput: every neuron of the group adds w * Binomial(N, rate dt) to its
// target variable, at the start of the synapses slot.
template <typename R>
void poisson_inputs(Net<R>& net, Group<R>& g) {
  for (const auto& in : g.pins)
    for (int64_t i = 0; i < g.n; ++i) {
      const int64_t x = binomial_draw(in.n, in.p, net.seed, in.id, net.ts, i);
      g.var[in.var][i] += (R)x * (R)in.w;
    }
}

template <typename R>
bool step(Net<R>& net) {
  const double t = (double)net.ts * net.dt;
  for (StateMon& m : net.smons) {
    if (net.ts % m.every != 0) continue;
    const Group<R>& g = net.groups[m.gid];
    m.steps.push_back(net.ts);
    for (int64_t i : m.idx)
      m.vals.push_back(m.var == NOT_REF ? (double)g.not_ref[i] : (double)g.var[m.var][i]);
  }
  for (Group<R>& g : net.groups) {
    if (g.kind == LIF) update_lif(g, net.ts, t, net.dt);
    else if (g.kind == HH) update_hh(g, net.ts, t, net.dt);
    else if (g.kind == MODEL && !update_model(net, g, t)) return false;
  }
  for (Group<R>& g : net.groups)
    if (!threshold(net, g, t)) return false;
  bool reset_ok = true;
  auto resets = [&]() {
    for (Group<R>& g : net.groups) {
      if (g.kind == LIF && g.p[10] != 0)
        for (int32_t i : g.spikes) g.var[V][i] = (R)g.p[7];
      if (g.kind == MODEL && g.model_reset && !g.spikes.empty())
        reset_ok = model_phase(net, g, 2, t, nullptr, &g.spikes) && reset_ok;
    }
  };
  if (net.reset_first) resets();
  for (Group<R>& g : net.groups) poisson_inputs(net, g);
  for (Syn<R>& s : net.syns) pathway_pre(net, s, t);
  for (Syn<R>& s : net.syns)
    if (s.effect == STDP) pathway_post(net, s, t);
  if (!net.reset_first) resets();
  if (!reset_ok) return false;
  for (RateMon& m : net.rmons) {
    m.steps.push_back(net.ts);
    m.counts.push_back((int64_t)net.groups[m.gid].spikes.size());
  }
  ++net.ts;
  return true;
}

template <typename R>
int add_group(Net<R>& net, Group<R>&& g) {
  if (net.built || g.n <= 0) return -1;
  for (auto& v : g.var) v.assign(g.n, (R)0);
  g.not_ref.assign(g.n, 1);
  if (g.refractory() > 0) g.var[LASTSPIKE].assign(g.n, (R)-1e4);
  net.groups.push_back(std::move(g));
  return (int)net.groups.size() - 1;
}

template <typename R>
void ensure_built(Net<R>& net) {
  if (net.built) return;
  for (Syn<R>& s : net.syns) build_syn(net, s);
  net.built = true;
}

// ---- Hines (SpatialNeuron) --------------------------------------------------------------------
// Backward-Euler step of the cable equation of a branched neuron, solved by domain
// decomposition: the method of brian2cuda/templates/spatialstateupdate.cu (matrix 18-93,
// per-section solves 128-192, branch-point system 202-307, combination 316-351), restated
// here from the mathematics.
//  - Compartment j of a neuron couples to compartment j-1 of the same section through the
//    axial conductance g[j] = 1 / (Ri (1/r_end[j-1] + 1/r_start[j])) (r: cross section over
//    half length); g is 0 at the first compartment of every section.  A section's first
//    compartment couples to the section's start node through g0 = r_start/Ri, its last one
//    to its end node through gn = r_end/Ri.
//  - Per section: three tridiagonal solves with the same matrix, x* for the membrane
//    equation with both node voltages 0, u_start and u_end with a unit voltage at one node.
//    Any solution of the section is v = x* + V_start u_start + V_end u_end.
//  - Node 0 is the start of the root section (sealed: its voltage is that of the first
//    compartment); node k+1 is the end of section k, where its child sections start.
//    Kirchhoff's current law at every node gives one equation per node in the node voltages;
//    the system is a tree (a node couples to its parent node and to its children's end
//    nodes), eliminated from the leaves to the root and then substituted back.  Sections are
//    numbered so that a parent precedes its children.
template <typename RC>
struct Hines {
  int nn = 0;
  std::vector<int64_t> comp_off;
  std::vector<int32_t> sec_off, starts, ends, parent;   // starts/ends neuron-local
  std::vector<double> area, r_start, r_end;             // per compartment
  double Cm, Ri, El, EK, ENa, gl, gNa, gK, Vthr, dt;
  // per compartment: matrix row without the membrane conductance (low couples j to j-1,
  // up couples j to j+1), and the right-hand sides of the two unit-node solves
  std::vector<double> low, diag, up, rhs_start, rhs_end;
  std::vector<double> g0, gn;                           // per section: node couplings
  std::vector<double> v, Ic, soma_I;
  std::vector<RC> m, h, n;
  std::vector<int32_t> spikes, above;
};

template <typename RC>
void hines_prepare(Hines<RC>& H) {
  const int64_t NC = H.comp_off[H.nn];
  H.low.assign(NC, 0); H.diag.assign(NC, 0); H.up.assign(NC, 0);
  H.rhs_start.assign(NC, 0); H.rhs_end.assign(NC, 0);
  H.g0.assign(H.sec_off[H.nn], 0); H.gn.assign(H.sec_off[H.nn], 0);
  std::vector<double> g(NC + 1, 0.0);   // axial conductance into compartment j from j-1
  for (int b = 0; b < H.nn; ++b) {
    const int64_t c0 = H.comp_off[b], c1 = H.comp_off[b + 1];
    std::vector<char> first(c1 - c0, 0);
    for (int k = H.sec_off[b]; k < H.sec_off[b + 1]; ++k) first[H.starts[k]] = 1;
    for (int64_t j = c0; j < c1; ++j)
      g[j] = first[j - c0] ? 0.0 : 1.0 / (H.Ri * (1.0 / H.r_end[j - 1] + 1.0 / H.r_start[j]));
    g[c1] = 0.0;
    for (int64_t j = c0; j < c1; ++j) {
      H.low[j] = g[j] / H.area[j];
      H.up[j] = g[j + 1] / H.area[j];
      H.diag[j] = -(H.Cm / H.dt) - (g[j] + g[j + 1]) / H.area[j];
    }
    for (int k = H.sec_off[b]; k < H.sec_off[b + 1]; ++k) {
      const int64_t f = c0 + H.starts[k], l = c0 + H.ends[k] - 1;
      H.g0[k] = H.r_start[f] / H.Ri;
      H.gn[k] = H.r_end[l] / H.Ri;
      H.diag[f] -= H.g0[k] / H.area[f];
      H.diag[l] -= H.gn[k] / H.area[l];
      H.rhs_start[f] = -H.g0[k] / H.area[f];
      H.rhs_end[l] = -H.gn[k] / H.area[l];
    }
  }
}

template <typename RC>
RC hh_ee(RC x, RC a, RC b, RC dt) {
  const RC A = -(a + b);
  const RC BA = a / A;
  return -BA + (BA + x) * xexp(A * dt);
}

template <typename RC>
void hines_step(Hines<RC>& H, bool write_currents) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int b = 0; b < H.nn; ++b) {
    const int64_t c0 = H.comp_off[b];
    const int nc = (int)(H.comp_off[b + 1] - c0);
    const int s0 = H.sec_off[b], ns = H.sec_off[b + 1] - s0;
    std::vector<double> gtot(nc), I0(nc), vprev(nc), xs(nc), us(nc), ue(nc), c(nc);
    double* v = &H.v[c0];
    // membrane conductance and current from the state at the start of the step, then gates
    for (int j = 0; j < nc; ++j) {
      const double md = (double)H.m[c0 + j], hd = (double)H.h[c0 + j], nd = (double)H.n[c0 + j];
      const double gna = H.gNa * (md * md * md * hd);
      const double gk = H.gK * (nd * nd * nd * nd);
      gtot[j] = H.gl + gna + gk;
      I0[j] = H.gl * H.El + gna * H.ENa + gk * H.EK;
      if (j == 0) I0[j] += H.soma_I[b];
      vprev[j] = v[j];
      const RC vr = (RC)v[j], dtR = (RC)H.dt;
      const RC am = (RC)1000 * z_over_expm1(((RC)25e-3 - vr) / (RC)10e-3);
      const RC bm = (RC)4000 * xexp(-vr / (RC)18e-3);
      const RC ah = (RC)70 * xexp(-vr / (RC)20e-3);
      const RC bh = (RC)1000 / (xexp(((RC)30e-3 - vr) / (RC)10e-3) + (RC)1);
      const RC an = (RC)100 * z_over_expm1(((RC)10e-3 - vr) / (RC)10e-3);
      const RC bn = (RC)125 * xexp(-vr / (RC)80e-3);
      H.m[c0 + j] = hh_ee(H.m[c0 + j], am, bm, dtR);
      H.h[c0 + j] = hh_ee(H.h[c0 + j], ah, bh, dtR);
      H.n[c0 + j] = hh_ee(H.n[c0 + j], an, bn, dtR);
    }
    // per section: one Thomas pass (forward elimination with the reciprocal pivot, then
    // back substitution) for the three right-hand sides x*, u_start, u_end
    for (int k = 0; k < ns; ++k) {
      const int lo = H.starts[s0 + k], hi = H.ends[s0 + k];
      double cprev = 0.0;
      for (int j = lo; j < hi; ++j) {
        const int64_t q = c0 + j;
        const double lw = j > lo ? H.low[q] : 0.0;
        const double piv = 1.0 / (H.diag[q] - gtot[j] - lw * cprev);
        c[j] = H.up[q] * piv;
        xs[j] = (-(H.Cm / H.dt) * v[j] - I0[j] - (j > lo ? lw * xs[j - 1] : 0.0)) * piv;
        us[j] = (H.rhs_start[q] - (j > lo ? lw * us[j - 1] : 0.0)) * piv;
        ue[j] = (H.rhs_end[q] - (j > lo ? lw * ue[j - 1] : 0.0)) * piv;
        cprev = c[j];
      }
      for (int j = hi - 2; j >= lo; --j) {
        xs[j] -= c[j] * xs[j + 1];
        us[j] -= c[j] * us[j + 1];
        ue[j] -= c[j] * ue[j + 1];
      }
    }
    // node system: node n's equation D[n] V_n + toward_parent[n] V_parent(n)
    // + sum over child nodes c of into_parent[c] V_c = rhs[n]
    const int nodes = ns + 1;
    std::vector<int> parent_node(nodes, -1);
    std::vector<double> D(nodes, 0.0), rhs(nodes, 0.0), toward_parent(nodes, 0.0),
        into_parent(nodes, 0.0), V(nodes, 0.0);
    auto start_node = [&](int k) { return k == 0 ? 0 : H.parent[s0 + k] + 1; };
    for (int k = 0; k < ns; ++k) {
      const int f = H.starts[s0 + k], l = H.ends[s0 + k] - 1;
      const int sn = start_node(k), en = k + 1;
      const double g0 = H.g0[s0 + k], gn = H.gn[s0 + k];
      parent_node[en] = sn;
      // end node: current from the section's last compartment
      D[en] += gn * (1.0 - ue[l]);
      toward_parent[en] = -gn * us[l];
      rhs[en] += gn * xs[l];
      if (k == 0) {
        // node 0 takes the voltage of the root's first compartment
        D[0] = us[f] - 1.0;
        into_parent[en] = ue[f];
        rhs[0] = -xs[f];
      } else {
        // start node: current into the section's first compartment
        D[sn] += g0 * (1.0 - us[f]);
        into_parent[en] = -g0 * ue[f];
        rhs[sn] += g0 * xs[f];
      }
    }
    // elimination from the leaves: a node's children have larger numbers, so going down
    // from the last node every child is complete when its parent takes it in
    std::vector<std::vector<int>> child_nodes(nodes);
    for (int nd = 1; nd < nodes; ++nd) child_nodes[parent_node[nd]].push_back(nd);
    for (int p = nodes - 1; p >= 0; --p)
      for (int nd : child_nodes[p]) {
        const double f = into_parent[nd] / D[nd];
        D[p] -= f * toward_parent[nd];
        rhs[p] -= f * rhs[nd];
      }
    V[0] = rhs[0] / D[0];
    for (int nd = 1; nd < nodes; ++nd)
      V[nd] = (rhs[nd] - toward_parent[nd] * V[parent_node[nd]]) / D[nd];
    for (int k = 0; k < ns; ++k)
      for (int j = H.starts[s0 + k]; j < H.ends[s0 + k]; ++j)
        v[j] = xs[j] + V[start_node(k)] * us[j] + V[k + 1] * ue[j];
    if (write_currents)
      for (int j = 0; j < nc; ++j) H.Ic[c0 + j] = H.Cm * (v[j] - vprev[j]) / H.dt;
    const int ab = v[0] > H.Vthr ? 1 : 0;
    if (ab && !H.above[b]) H.spikes[b]++;
    H.above[b] = ab;
  }
}

// ---- C API ------------------------------------------------------------------------------------
struct Handle {
  bool f32;
  Net<float> nf;
  Net<double> nd;
};

#define DISPATCH(h, fn, ...) ((h)->f32 ? fn<float>((h)->nf, __VA_ARGS__) : fn<double>((h)->nd, __VA_ARGS__))

template <typename R>
int api_group(Net<R>& net, int kind, int64_t n, const double* p, int np, double rate) {
  Group<R> g;
  g.kind = kind;
  g.n = n;
  if (p) g.p.assign(p, p + np);
  g.rate = rate;
  return add_group(net, std::move(g));
}

template <typename R>
int api_spikegen(Net<R>& net, int64_t n, int64_t ns, const int32_t* idx, const int64_t* st) {
  Group<R> g;
  g.kind = SPIKEGEN;
  g.n = n;
  for (int64_t k = 0; k < ns; ++k) g.sg.emplace_back(st[k], idx[k]);
  std::sort(g.sg.begin(), g.sg.end());
  return add_group(net, std::move(g));
}

template <typename R>
int api_poisson_input(Net<R>& net, int gid, int var, int64_t n, double rate, double w) {
  if (gid < 0 || gid >= (int)net.groups.size()) return -1;
  Group<R>& g = net.groups[gid];
  if ((g.kind != LIF && g.kind != HH) || (var != V && var != GE && var != GI) || n < 0 ||
      g.pins.size() >= 2)
    return -1;
  g.pins.push_back({var, n, rate * net.dt, w, (uint32_t)net.n_pins});
  return net.n_pins++;
}

template <typename R>
int api_timedarray(Net<R>& net, int gid, const double* vals, int64_t rows, int64_t cols,
                   int64_t mul, int64_t div) {
  if (gid < 0 || gid >= (int)net.groups.size()) return -1;
  Group<R>& g = net.groups[gid];
  if ((g.kind != LIF && g.kind != HH && g.kind != POISSON) || rows < 1 ||
      (cols != 1 && cols != g.n) || mul < 1 ||
      div < 1)
    return -1;
  g.ta.assign(vals, vals + rows * cols);   // rounded to R once, as the device copy is
  g.ta_rows = rows;
  g.ta_cols = cols;
  g.ta_mul = mul;
  g.ta_div = div;
  return 0;
}

template <typename R>
int api_spikegen_period(Net<R>& net, int gid, int64_t period) {
  if (gid < 0 || gid >= (int)net.groups.size() || net.groups[gid].kind != SPIKEGEN ||
      period < 0)
    return -1;
  Group<R>& g = net.groups[gid];
  for (const auto& e : g.sg)
    if (period > 0 && e.first >= period) return -1;
  g.sg_period = period;
  return 0;
}

template <typename R>
int api_state(Net<R>& net, int gid, int var, double* vals, int64_t n, int set) {
  if (gid < 0 || gid >= (int)net.groups.size()) return -1;
  Group<R>& g = net.groups[gid];
  if (n != g.n || var < 0 || var > NOT_REF) return -1;
  for (int64_t i = 0; i < n; ++i) {
    if (var == NOT_REF) {
      if (set) g.not_ref[i] = vals[i] != 0; else vals[i] = g.not_ref[i];
    } else {
      if (set) g.var[var][i] = (R)vals[i]; else vals[i] = (double)g.var[var][i];
    }
  }
  return 0;
}

template <typename R>
int api_synapses(Net<R>& net, int pre, int post, int target, int effect, int64_t n,
                 const int32_t* i, const int32_t* j, const double* w, double w_scalar,
                 const int32_t* delay, int32_t delay_scalar, const double* stdp) {
  if (net.built) return -1;
  if (pre < 0 || post < 0 || pre >= (int)net.groups.size() || post >= (int)net.groups.size())
    return -1;
  Syn<R> s;
  s.pre = pre; s.post = post; s.target = target; s.effect = effect; s.n = n;
  s.i.assign(i, i + n);
  s.j.assign(j, j + n);
  s.delay.assign(n, delay_scalar);
  if (delay) s.delay.assign(delay, delay + n);
  s.max_delay = 0;
  for (int32_t d : s.delay) s.max_delay = std::max(s.max_delay, d);
  s.has_w = w != nullptr || effect == STDP;
  s.w_scalar = (R)w_scalar;
  if (s.has_w) {
    s.w.assign(n, (R)w_scalar);
    if (w) for (int64_t k = 0; k < n; ++k) s.w[k] = (R)w[k];
  }
  if (stdp) std::copy(stdp, stdp + 7, s.stdp);
  net.syns.push_back(std::move(s));
  return (int)net.syns.size() - 1;
}

// connect(p) restated from the paper's Philox: pair (i, j) connects when word (j mod 4) of
// Philox(counter = (j/4, i, 0x5EED, 0), key = seed) is below floor(p * 2^32); its delay is
// dmin + floor(word0 * nd / 2^32) of Philox(counter = (j, i, 0xDE1A, 1), key = seed).
// Synapses are numbered in (i, delay, j) order.
template <typename R>
int api_random(Net<R>& net, int pre, int lo, int hi, int post, int target, double p,
               int32_t dmin, int32_t dmax, double w, uint64_t seed) {
  if (pre < 0 || post < 0 || pre >= (int)net.groups.size() || post >= (int)net.groups.size())
    return -1;
  if (lo < 0 || hi > net.groups[pre].n || lo >= hi) return -1;
  const int64_t npost = net.groups[post].n;
  const uint64_t thr = p >= 1.0 ? ((uint64_t)1 << 32) : (p <= 0 ? 0 : (uint64_t)(p * 4294967296.0));
  const int32_t nd = dmax - dmin + 1;
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  // Rows are independent: each row's synapses are drawn in (j) order and stably sorted by
  // delay; a first pass counts the synapses of every row so that the rows can be written in
  // parallel straight into the synapse arrays (the 2e8-synapse network needs this).
  const int64_t rows = hi - lo;
  std::vector<int64_t> row_off(rows + 1, 0);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t r = 0; r < rows; ++r) {
    const uint32_t i = (uint32_t)(lo + r);
    int64_t c = 0;
    for (int64_t jq = 0; 4 * jq < npost; ++jq) {
      const Ctr x = philox(Ctr{{(uint32_t)jq, i, 0x5EEDu, 0u}}, k0, k1);
      for (int e = 0; e < 4 && 4 * jq + e < npost; ++e) c += (uint64_t)x.v[e] < thr;
    }
    row_off[r + 1] = c;
  }
  for (int64_t r = 0; r < rows; ++r) row_off[r + 1] += row_off[r];
  const int64_t n = row_off[rows];
  if (net.built) return -1;
  Syn<R> s;
  s.pre = pre; s.post = post; s.target = target; s.effect = ADD; s.n = n;
  s.i.resize(n);
  s.j.resize(n);
  s.delay.resize(n);
  int32_t max_d = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(max : max_d)
  for (int64_t r = 0; r < rows; ++r) {
    const uint32_t i = (uint32_t)(lo + r);
    std::vector<std::pair<int32_t, int32_t>> row;  // (delay, j)
    for (int64_t jq = 0; 4 * jq < npost; ++jq) {
      const Ctr x = philox(Ctr{{(uint32_t)jq, i, 0x5EEDu, 0u}}, k0, k1);
      for (int e = 0; e < 4 && 4 * jq + e < npost; ++e) {
        if ((uint64_t)x.v[e] < thr) {
          const uint32_t j = (uint32_t)(4 * jq + e);
          const Ctr rd = philox(Ctr{{j, i, 0xDE1Au, 1u}}, k0, k1);
          const int32_t d = dmin + (int32_t)(((uint64_t)rd.v[0] * (uint64_t)(uint32_t)nd) >> 32);
          row.emplace_back(d, (int32_t)j);
        }
      }
    }
    std::stable_sort(row.begin(), row.end(),
                     [](const auto& a, const auto& b) { return a.first < b.first; });
    int64_t k = row_off[r];
    for (auto& y : row) {
      s.i[k] = (int32_t)i; s.j[k] = y.second; s.delay[k] = y.first;
      max_d = std::max(max_d, y.first);
      ++k;
    }
  }
  s.max_delay = max_d;
  s.has_w = false;
  s.w_scalar = (R)w;
  net.syns.push_back(std::move(s));
  return (int)net.syns.size() - 1;
}

template <typename R>
int64_t api_syn_count(Net<R>& net, int sid) {
  if (sid < 0 || sid >= (int)net.syns.size()) return -1;
  return net.syns[sid].n;
}

template <typename R>
int api_syn_get(Net<R>& net, int sid, int var, double* out, int64_t n) {
  if (sid < 0 || sid >= (int)net.syns.size()) return -1;
  ensure_built(net);
  Syn<R>& s = net.syns[sid];
  if (n != s.n) return -1;
  for (int64_t k = 0; k < n; ++k) {
    switch (var) {
      case SYN_I: out[k] = s.i[k]; break;
      case SYN_J: out[k] = s.j[k]; break;
      case SYN_DELAY: out[k] = s.delay[k]; break;
      case SYN_W: out[k] = s.has_w ? (double)s.w[k] : (double)s.w_scalar; break;
      case SYN_APRE: out[k] = s.effect == STDP ? (double)s.apre[k] : 0; break;
      case SYN_APOST: out[k] = s.effect == STDP ? (double)s.apost[k] : 0; break;
      case SYN_LU: out[k] = s.effect == STDP ? (double)s.lu[k] : 0; break;
      default: return -1;
    }
  }
  return 0;
}

template <typename R>
int api_group_model(Net<R>& net, int64_t n, int nv, int nn, int has_thr, int has_reset,
                    double refractory, ModelFn fn, void* user) {
  if (nv < 1 || nv > 6 || nn < 0 || !fn) return -1;
  Group<R> g;
  g.kind = MODEL;
  g.n = n;
  g.model_fn = fn;
  g.model_user = user;
  g.model_nv = nv;
  g.model_nn = nn;
  g.model_thr = has_thr;
  g.model_reset = has_reset;
  g.model_ref = refractory;
  return add_group(net, std::move(g));
}

template <typename R>
int api_normals(Net<R>& net, int gid, const double* u, int64_t steps, int64_t n) {
  if (gid < 0 || gid >= (int)net.groups.size()) return -1;
  Group<R>& g = net.groups[gid];
  if (g.kind != MODEL || n != (int64_t)g.model_nn * g.n) return -1;
  for (int64_t k = 0; k < steps; ++k) g.normals.emplace_back(u + k * n, u + (k + 1) * n);
  return 0;
}

// New delays of an additive Synapses object between runs: the bundles still in its queue
// become explicit (step, synapse) deliveries with their old delays, and the bundle tables
// and the queue are rebuilt for the new delays (the reference's queue keeps what it holds
// and pushes later spikes with the new delays, brian2cuda/brianlib/spikequeue.h:98-201).
template <typename R>
int api_syn_set_delays(Net<R>& net, int sid, const int32_t* d, int64_t n) {
  if (sid < 0 || sid >= (int)net.syns.size()) return -1;
  ensure_built(net);
  Syn<R>& s = net.syns[sid];
  if (n != s.n || s.effect != ADD) return -1;
  const int nq = s.num_queues;
  for (int o = 1; o < nq; ++o) {
    // slot current_offset + o holds the bundles due o steps after the last simulated step
    for (int64_t key : s.queue[(s.current_offset + o) % nq])
      for (int64_t q = s.bundle_off[key]; q < s.bundle_off[key + 1]; ++q)
        s.legacy.emplace_back(net.ts - 1 + o, s.bundle_syn[q]);
  }
  s.delay.assign(d, d + n);
  s.max_delay = 0;
  for (int64_t k = 0; k < n; ++k) {
    if (d[k] < 0) return -1;
    s.max_delay = std::max(s.max_delay, d[k]);
  }
  build_syn(net, s);
  return 0;
}

template <typename R>
int api_uniforms(Net<R>& net, int gid, const double* u, int64_t steps, int64_t n) {
  if (gid < 0 || gid >= (int)net.groups.size()) return -1;
  Group<R>& g = net.groups[gid];
  if (g.kind != POISSON || n != g.n) return -1;
  for (int64_t k = 0; k < steps; ++k) g.uniforms.emplace_back(u + k * n, u + (k + 1) * n);
  return 0;
}

template <typename R>
int api_store(Net<R>& net) {
  ensure_built(net);
  NetSnap<R>& S = net.snap;
  S.ts = net.ts;
  S.var.clear(); S.not_ref.clear(); S.spikes.clear(); S.uni_next.clear();
  for (const Group<R>& g : net.groups) {
    std::array<std::vector<R>, 7> v;
    for (int k = 0; k < 7; ++k) v[k] = g.var[k];
    S.var.push_back(std::move(v));
    S.not_ref.push_back(g.not_ref);
    S.spikes.push_back(g.spikes);
    S.uni_next.push_back(g.uni_next);
  }
  S.queue.clear(); S.current_offset.clear(); S.w.clear(); S.apre.clear(); S.apost.clear();
  S.lu.clear();
  for (const Syn<R>& sy : net.syns) {
    S.queue.push_back(sy.queue);
    S.current_offset.push_back(sy.current_offset);
    S.w.push_back(sy.effect == STDP ? sy.w : std::vector<R>());
    S.apre.push_back(sy.apre);
    S.apost.push_back(sy.apost);
    S.lu.push_back(sy.lu);
  }
  S.valid = true;
  return 0;
}

template <typename R>
int api_restore(Net<R>& net) {
  const NetSnap<R>& S = net.snap;
  if (!S.valid) return -1;
  net.ts = S.ts;
  for (size_t g = 0; g < net.groups.size(); ++g) {
    for (int k = 0; k < 7; ++k) net.groups[g].var[k] = S.var[g][k];
    net.groups[g].not_ref = S.not_ref[g];
    net.groups[g].spikes = S.spikes[g];
    net.groups[g].uni_next = S.uni_next[g];
  }
  for (size_t q = 0; q < net.syns.size(); ++q) {
    Syn<R>& sy = net.syns[q];
    sy.queue = S.queue[q];
    sy.current_offset = S.current_offset[q];
    if (sy.effect == STDP) sy.w = S.w[q];
    sy.apre = S.apre[q];
    sy.apost = S.apost[q];
    sy.lu = S.lu[q];
  }
  return 0;
}

template <typename R>
int api_run(Net<R>& net, int64_t steps, int64_t) {
  ensure_built(net);
  for (int64_t k = 0; k < steps; ++k)
    if (!step(net)) return -1;
  return 0;
}

template <typename R>
int64_t api_spikes(Net<R>& net, int gid, int32_t* idx, int64_t* st, int64_t cap) {
  if (gid < 0 || gid >= (int)net.groups.size()) return -1;
  auto rec = net.groups[gid].recorded;
  std::sort(rec.begin(), rec.end());
  for (int64_t k = 0; k < (int64_t)rec.size() && k < cap; ++k) {
    if (st) st[k] = rec[k].first;
    if (idx) idx[k] = rec[k].second;
  }
  return (int64_t)rec.size();
}

template <typename R>
int api_statemon(Net<R>& net, int gid, int var, const int64_t* idx, int64_t n, int every) {
  if (gid < 0 || gid >= (int)net.groups.size() || var < 0 || var > NOT_REF || every < 1)
    return -1;
  StateMon m;
  m.gid = gid; m.var = var; m.every = every;
  for (int64_t k = 0; k < n; ++k) {
    if (idx[k] < 0 || idx[k] >= net.groups[gid].n) return -1;
    m.idx.push_back(idx[k]);
  }
  net.smons.push_back(std::move(m));
  return (int)net.smons.size() - 1;
}

template <typename R>
int64_t api_statemon_get(Net<R>& net, int mid, int64_t* steps, double* vals, int64_t cap) {
  if (mid < 0 || mid >= (int)net.smons.size()) return -1;
  const StateMon& m = net.smons[mid];
  const int64_t n = (int64_t)m.steps.size(), ni = (int64_t)m.idx.size();
  for (int64_t r = 0; r < n && r < cap; ++r) {
    if (steps) steps[r] = m.steps[r];
    if (vals) std::copy(m.vals.begin() + r * ni, m.vals.begin() + (r + 1) * ni, vals + r * ni);
  }
  return n;
}

template <typename R>
int api_ratemon(Net<R>& net, int gid) {
  if (gid < 0 || gid >= (int)net.groups.size()) return -1;
  RateMon m;
  m.gid = gid;
  net.rmons.push_back(std::move(m));
  return (int)net.rmons.size() - 1;
}

template <typename R>
int64_t api_ratemon_get(Net<R>& net, int mid, int64_t* steps, int64_t* counts, int64_t cap) {
  if (mid < 0 || mid >= (int)net.rmons.size()) return -1;
  const RateMon& m = net.rmons[mid];
  const int64_t n = (int64_t)m.steps.size();
  for (int64_t r = 0; r < n && r < cap; ++r) {
    if (steps) steps[r] = m.steps[r];
    if (counts) counts[r] = m.counts[r];
  }
  return n;
}

// Bundles still queued after the last step: (offset a >= 1 at which it is delivered, pre,
// delay), sorted.  Slot (current_offset + a) % num_queues is delivered a steps from now.
template <typename R>
int64_t api_queue(Net<R>& net, int sid, int32_t* off, int32_t* pre, int32_t* dl, int64_t cap) {
  if (sid < 0 || sid >= (int)net.syns.size()) return -1;
  ensure_built(net);
  Syn<R>& s = net.syns[sid];
  const int D = s.max_delay + 1;
  std::vector<std::array<int32_t, 3>> out;
  for (int a = 1; a < s.num_queues; ++a) {
    for (int64_t key : s.queue[(s.current_offset + a) % s.num_queues])
      out.push_back({a, (int32_t)(key / D), (int32_t)(key % D)});
  }
  std::sort(out.begin(), out.end());
  for (int64_t k = 0; k < (int64_t)out.size() && k < cap; ++k) {
    if (off) off[k] = out[k][0];
    if (pre) pre[k] = out[k][1];
    if (dl) dl[k] = out[k][2];
  }
  return (int64_t)out.size();
}

struct HinesHandle {
  bool f32;
  Hines<float> hf;
  Hines<double> hd;
};

template <typename RC>
void hines_init(Hines<RC>& H, int nn, const int64_t* comp_off, const int32_t* sec_off,
                const int32_t* st, const int32_t* en, const int32_t* par, const double* d,
                const double* L, const double* p, double dt) {
  H.nn = nn;
  H.comp_off.assign(comp_off, comp_off + nn + 1);
  H.sec_off.assign(sec_off, sec_off + nn + 1);
  const int32_t S = sec_off[nn];
  const int64_t C = comp_off[nn];
  H.starts.assign(st, st + S);
  H.ends.assign(en, en + S);
  H.parent.assign(par, par + S);
  H.area.resize(C); H.r_start.resize(C); H.r_end.resize(C);
  for (int64_t c = 0; c < C; ++c) {
    H.area[c] = M_PI * d[c] * L[c];
    // cross section over half the length, towards either end of a cylinder
    H.r_start[c] = H.r_end[c] = M_PI * d[c] * d[c] / (2.0 * L[c]);
  }
  H.Cm = p[0]; H.Ri = p[1]; H.El = p[2]; H.EK = p[3]; H.ENa = p[4]; H.gl = p[5]; H.gNa = p[6];
  H.gK = p[7]; H.Vthr = p[8]; H.dt = dt;
  H.v.assign(C, 0); H.Ic.assign(C, 0); H.soma_I.assign(nn, 0);
  H.m.assign(C, 0); H.h.assign(C, 0); H.n.assign(C, 0);
  H.spikes.assign(nn, 0); H.above.assign(nn, 0);
  hines_prepare(H);
}

}  // namespace

extern "C" {

// flags: bit 0 = float32 arithmetic, bit 1 = resets before synapses
void* orc_create(double dt, int flags) {
  Handle* h = new Handle();
  h->f32 = (flags & 1) != 0;
  h->nf.dt = dt;
  h->nd.dt = dt;
  h->nf.reset_first = h->nd.reset_first = (flags & 2) != 0;
  return h;
}
void orc_set_seed(void* hp, uint64_t seed) {
  Handle* h = static_cast<Handle*>(hp);
  h->nf.seed = h->nd.seed = seed;
}
void orc_destroy(void* h) { delete static_cast<Handle*>(h); }
const char* orc_error(void* hp) {
  Handle* h = static_cast<Handle*>(hp);
  return h->f32 ? h->nf.err.c_str() : h->nd.err.c_str();
}
// LIF params (12): El taum taue taui ke ki Vt Vr refractory has_threshold has_reset unless
int orc_group_lif(void* hp, int64_t n, const double* p) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_group, LIF, n, p, 12, 0.0);
}
// HH params (14): Cm gl El EK ENa gNa gK VT Ee Ei taue taui Vthr refractory
int orc_group_hh(void* hp, int64_t n, const double* p) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_group, HH, n, p, 14, 0.0);
}
int orc_group_model(void* hp, int64_t n, int nv, int nn, int has_thr, int has_reset,
                    double refractory, ModelFn fn, void* user) {
  Handle* h = static_cast<Handle*>(hp);
  return h->f32 ? api_group_model(h->nf, n, nv, nn, has_thr, has_reset, refractory, fn, user)
                : api_group_model(h->nd, n, nv, nn, has_thr, has_reset, refractory, fn, user);
}
int orc_set_normals(void* hp, int gid, const double* u, int64_t steps, int64_t n) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_normals, gid, u, steps, n);
}
int orc_group_poisson(void* hp, int64_t n, double rate) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_group, POISSON, n, nullptr, 0, rate);
}
int orc_group_spikegen(void* hp, int64_t n, int64_t ns, const int32_t* idx, const int64_t* st) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_spikegen, n, ns, idx, st);
}
// PoissonInput of group gid onto var: N inputs at rate Hz, weight w; returns its stream id
int orc_poisson_input(void* hp, int gid, int var, int64_t n, double rate, double w) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_poisson_input, gid, var, n, rate, w);
}
// TimedArray: values [rows][cols], step ts reads row min(ts * mul / div, rows - 1)
int orc_timedarray(void* hp, int gid, const double* v, int64_t rows, int64_t cols, int64_t mul,
                   int64_t div) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_timedarray, gid, v, rows, cols, mul, div);
}
// SpikeGeneratorGroup period in steps (0: none); every entry must lie inside it
int orc_spikegen_period(void* hp, int gid, int64_t period) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_spikegen_period, gid, period);
}
int orc_state_set(void* hp, int gid, int var, const double* v, int64_t n) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_state, gid, var, const_cast<double*>(v), n, 1);
}
int orc_state_get(void* hp, int gid, int var, double* v, int64_t n) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_state, gid, var, v, n, 0);
}
// stdp (7): taupre taupost dApre dApost wmin wmax pre_adds_weight
int orc_synapses(void* hp, int pre, int post, int target, int effect, int64_t n,
                 const int32_t* i, const int32_t* j, const double* w, double w_scalar,
                 const int32_t* delay, int32_t delay_scalar, const double* stdp) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_synapses, pre, post, target, effect, n, i, j, w, w_scalar, delay,
                  delay_scalar, stdp);
}
int orc_synapses_random(void* hp, int pre, int lo, int hi, int post, int target, double p,
                        int32_t dmin, int32_t dmax, double w, uint64_t seed) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_random, pre, lo, hi, post, target, p, dmin, dmax, w, seed);
}
int64_t orc_syn_count(void* hp, int sid) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_syn_count, sid);
}
int orc_syn_get(void* hp, int sid, int var, double* out, int64_t n) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_syn_get, sid, var, out, n);
}
int orc_set_uniforms(void* hp, int gid, const double* u, int64_t steps, int64_t n) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_uniforms, gid, u, steps, n);
}
int orc_run(void* hp, int64_t steps) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_run, steps, 0);
}
void orc_clear_spikes(void* hp) {
  Handle* h = static_cast<Handle*>(hp);
  if (h->f32) { for (auto& g : h->nf.groups) g.recorded.clear(); }
  else { for (auto& g : h->nd.groups) g.recorded.clear(); }
}
int orc_syn_set_delays(void* hp, int sid, const int32_t* d, int64_t n) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_syn_set_delays, sid, d, n);
}
int orc_store(void* hp) {
  Handle* h = static_cast<Handle*>(hp);
  return h->f32 ? api_store(h->nf) : api_store(h->nd);
}
int orc_restore(void* hp) {
  Handle* h = static_cast<Handle*>(hp);
  return h->f32 ? api_restore(h->nf) : api_restore(h->nd);
}
int64_t orc_timestep(void* hp) {
  Handle* h = static_cast<Handle*>(hp);
  return h->f32 ? h->nf.ts : h->nd.ts;
}
int64_t orc_spikes(void* hp, int gid, int32_t* idx, int64_t* st, int64_t cap) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_spikes, gid, idx, st, cap);
}
int orc_statemon(void* hp, int gid, int var, const int64_t* idx, int64_t n, int every) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_statemon, gid, var, idx, n, every);
}
int64_t orc_statemon_get(void* hp, int mid, int64_t* steps, double* vals, int64_t cap) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_statemon_get, mid, steps, vals, cap);
}
int orc_ratemon(void* hp, int gid) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_ratemon, gid);
}
int64_t orc_ratemon_get(void* hp, int mid, int64_t* steps, int64_t* counts, int64_t cap) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_ratemon_get, mid, steps, counts, cap);
}
int64_t orc_queue(void* hp, int sid, int32_t* off, int32_t* pre, int32_t* dl, int64_t cap) {
  Handle* h = static_cast<Handle*>(hp);
  return DISPATCH(h, api_queue, sid, off, pre, dl, cap);
}

// Hines. p (9): Cm Ri El EK ENa gl gNa gK Vthr
void* orc_hines_create(int nn, const int64_t* comp_off, const int32_t* sec_off,
                       const int32_t* st, const int32_t* en, const int32_t* par,
                       const double* d, const double* L, const double* p, double dt, int f32) {
  HinesHandle* h = new HinesHandle();
  h->f32 = f32 != 0;
  if (h->f32) hines_init(h->hf, nn, comp_off, sec_off, st, en, par, d, L, p, dt);
  else hines_init(h->hd, nn, comp_off, sec_off, st, en, par, d, L, p, dt);
  return h;
}
void orc_hines_destroy(void* h) { delete static_cast<HinesHandle*>(h); }
int orc_hines_set_current(void* hp, const double* I) {
  HinesHandle* h = static_cast<HinesHandle*>(hp);
  auto set = [&](auto& H) {
    for (int b = 0; b < H.nn; ++b) H.soma_I[b] = I ? I[b] / H.area[H.comp_off[b]] : 0.0;
  };
  if (h->f32) set(h->hf); else set(h->hd);
  return 0;
}
// vars: 0 v, 1 m, 2 h, 3 n, 4 Ic (values as doubles)
int orc_hines_state(void* hp, int var, double* vals, int64_t n, int set) {
  HinesHandle* h = static_cast<HinesHandle*>(hp);
  auto go = [&](auto& H) {
    if (n != H.comp_off[H.nn]) return -1;
    for (int64_t c = 0; c < n; ++c) {
      switch (var) {
        case 0: if (set) H.v[c] = vals[c]; else vals[c] = H.v[c]; break;
        case 1: if (set) H.m[c] = vals[c]; else vals[c] = H.m[c]; break;
        case 2: if (set) H.h[c] = vals[c]; else vals[c] = H.h[c]; break;
        case 3: if (set) H.n[c] = vals[c]; else vals[c] = H.n[c]; break;
        case 4: if (set) H.Ic[c] = vals[c]; else vals[c] = H.Ic[c]; break;
        default: return -1;
      }
    }
    return 0;
  };
  return h->f32 ? go(h->hf) : go(h->hd);
}
int orc_hines_run(void* hp, int64_t steps) {
  HinesHandle* h = static_cast<HinesHandle*>(hp);
  for (int64_t k = 0; k < steps; ++k) {
    if (h->f32) hines_step(h->hf, k == steps - 1);
    else hines_step(h->hd, k == steps - 1);
  }
  return 0;
}
int orc_hines_spikes(void* hp, int32_t* out, int n) {
  HinesHandle* h = static_cast<HinesHandle*>(hp);
  auto& sp = h->f32 ? h->hf.spikes : h->hd.spikes;
  if (n != (int)sp.size()) return -1;
  std::copy(sp.begin(), sp.end(), out);
  return 0;
}

}  // extern "C"
