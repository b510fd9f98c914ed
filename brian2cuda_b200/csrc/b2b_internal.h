// Internal types of libb2b shared by the host runtime (api.cu) and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <curand.h>
#include <stdint.h>

#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/b2b.h"

namespace b2b {

constexpr int kMaxVars = 8;          // v, ge, gi, m, h, n, lastspike, not_refractory
constexpr int kPad = 128;            // population and group offsets are padded to this
constexpr int kBlock = 256;          // threads per CTA for the per-neuron kernels
constexpr int kChunk = 128;          // synapses one warp takes from a bundle per work item
constexpr int kMaxProjBatch = 8;     // additive projections delivered by one launch
constexpr int kNumSMs = 148;         // B200

enum Kind { KIND_LIF = 1, KIND_HH = 2, KIND_POISSON = 3, KIND_SPIKEGEN = 4, KIND_MODEL = 5 };

// Launcher exported by a generated model's shared object (b2b_group_model): phase 0 steps
// every neuron of the population `pop` (a PopDev), phase 1 applies the deferred reset.
typedef int32_t (*ModelLaunchFn)(const void* pop, const int64_t* clock, int32_t k, double dt,
                                 int32_t* status, void* stream, int32_t dtype, int32_t phase);
typedef int32_t (*ModelInfoFn)(b2b_model_info* info);

// Parameters of a generated-model group as its kernel reads them.
struct ModelGroupDev {
  int64_t offset, n;
  int64_t ref_steps;                      // timestep(refractory, dt); -1 = no refractoriness
};

// Per-group parameters as the kernels read them (doubles; cast to the state type in-kernel).
// TimedArray input of a group (b2b_timedarray): values[rows][cols] in the population's
// dtype, one column for the whole group or one per neuron; step ts reads row
// min(ts * mul / div, rows - 1).  val == NULL: no input.
struct TimedInput {
  const void* val;
  int64_t rows, cols, mul, div;
};
// PoissonInput of a group (b2b_poisson_input): every step each neuron adds weight * X to
// variable `var`, X ~ Binomial(n, p) drawn by inversion (neuron_math.cuh) from one Philox
// word of counter (group-local index, step low, step high, id), key (k0, k1).  qn = q^n,
// s = p/q, a = (n + 1) s with p = min(rate dt, 1 - rate dt) (reverse: X = n - draw).
constexpr int kMaxPoissonInputs = 2;
struct PoissonIn {
  int64_t n;
  double qn, s, a, weight;
  int32_t var, reverse;
  uint32_t id, k0, k1, pad;
};
struct PoissonInputs {
  int32_t count;
  int32_t after_reset;                    // the schedule resets before the synapses slot
  PoissonIn in[kMaxPoissonInputs];
};
// Inputs of one group, in an array beside the groups' parameters (PopDev::inputs) so that
// the parameters keep their size and populations without inputs never read it.
struct GroupInputs {
  TimedInput ta;                          // LIF: volts added to El; HH: amperes
  PoissonInputs pin;
};
struct LifDev {
  double A, Be, Bi, De, Di, El, Vt, Vr;   // exact propagator coefficients + threshold/reset
  int64_t ref_steps;                      // timestep(refractory, dt); -1 = no refractoriness
  int64_t offset, n;                      // group range inside the population
  int32_t has_threshold, has_reset, unless_refractory, pad;
};
// float32 copies of the HH constants (rounded on the host as the device would round them),
// so a float32 update loads 4-byte values and converts nothing.
struct HhFloat {
  float Cm, gl, El, EK, ENa, gNa, gK, VT, Ee, Ei, De, Di, Vthr, inv_Cm;
};
struct HhDev {
  double Cm, gl, El, EK, ENa, gNa, gK, VT, Ee, Ei, De, Di, Vthr;
  int64_t ref_steps;
  int64_t offset, n;
  double inv_Cm;                          // 1/Cm (the float32 update multiplies by it)
  HhFloat f;
};
struct PoissonDev {
  double p_spike;                         // rate * dt
  int64_t offset, n;
};

// Device view of a population (all groups of one kind and dtype laid out back to back).
struct PopDev {
  void* var[kMaxVars];            // SoA state, NOT_REFRACTORY as uint8
  const void* params;             // LifDev/HhDev/PoissonDev[n_groups]
  const int32_t* vec_group;       // group id per 4-neuron vector (NULL when one group)
  const GroupInputs* inputs;      // [n_groups] TimedArray / PoissonInput inputs, or NULL
  int64_t n;                      // padded neuron count (multiple of kPad)
  int32_t n_groups;
  int32_t ring_len;               // spike history slots (>= max delay + 2)
  int32_t* ring_idx;              // [ring_len][n] spike indices per step
  int32_t* ring_cnt;              // [ring_len] spike counts per step
  int32_t* mon_idx;               // spike monitor (or NULL)
  int64_t* mon_step;
  unsigned long long* mon_cnt;
  int64_t mon_cap;
  const void* rng;                // uniform buffer [steps][n] (Poisson); generated models:
                                  // [steps][n_uniform][n]
  const void* rng_normal;         // generated models: normal buffer [steps][n_normal][n]
  const int32_t* sg_idx;          // spike generator entries sorted by step
  const int64_t* sg_step;
  int64_t sg_n;
  int64_t sg_period;              // > 0: the entries repeat every sg_period steps
  int32_t late_reset;             // reset must run after synaptic delivery
  int32_t pad;
  // The step as two concurrent launches (pending.cu): per variable (v, ge, gi), [2][n] input
  // delivered during the previous step, which the update adds in and clears (NULL: none).
  void* fold[3];
};

// Device view of a projection (merged Synapses objects with one source population, one
// target variable and one effect).
struct ProjDev {
  const int32_t* src_ring_idx;
  const int32_t* src_ring_cnt;
  int64_t src_n;                  // ring row stride (padded source population size)
  int32_t src_ring_len;
  int32_t dmin, nd;               // delays dmin .. dmin+nd-1
  // source steps whose spikes this projection delivers: [src_lo, src_hi).  After a change
  // of delays between runs, the projection as built before delivers the spikes sent before
  // the change (src_hi = the first step after it) and the rebuilt one the later spikes.
  int64_t src_lo = 0;
  int64_t src_hi = INT64_MAX;
  int32_t chunks;                 // work items per bundle = ceil(max bundle / kChunk)
  const int64_t* off;             // [n_src*nd + 1] bundle offsets, key = pre*nd + (d-dmin)
  const int32_t* post;            // [n_syn] target index in the target population
  const void* w;                  // [n_syn] weights or NULL
  double w_scalar;
  void* target;                   // target variable array (all members share it: n_mem == 1)
  // Members with different target variables (additive projections): member m covers
  // presynaptic indices below mem_hi[m] and adds into targets[mem_var[m]].
  int32_t n_mem;
  int32_t pad_mem;
  const int64_t* mem_hi;
  const int8_t* mem_var;
  const double* mem_w;            // per-member scalar weight (members differ), or NULL
  void* targets[3];               // per variable v, ge, gi
  // STDP
  void* syn4;                     // per synapse {w, Apre, Apost, lastupdate}, interleaved so
                                  // that a strided (on_post) visit touches one sector
  double taupre, taupost, dApre, dApost, wmin, wmax;
  int32_t pre_adds_weight;
  int32_t aggregate;              // warp-aggregate atomics (few targets)
  // on_post pathway (transposed index)
  const int32_t* post_ring_idx;
  const int32_t* post_ring_cnt;
  int64_t post_src_n;
  int32_t post_ring_len;
  int32_t post_chunks;
  const int64_t* post_off;        // [n_post + 1]
  const int32_t* post_syn;        // synapse positions grouped by post
  // Order of the STDP records: NULL, record s belongs to synapse position s; otherwise the
  // records follow the post-grouped index (record r is synapse post_syn[r], so on_post walks
  // contiguous records) and rec_of[s] is the record of synapse position s.
  const int32_t* rec_of;
};

// Device view of a state monitor (monitor.cu): variable src (es-byte elements) of the
// population rows idx[0..n_idx), one record [n_idx] per step divisible by `every`.
struct StateMonDev {
  const uint8_t* src;
  const int64_t* idx;             // population-level rows
  uint8_t* buf;                   // [cap][n_idx]
  int64_t* steps;                 // [cap] step of each record
  unsigned long long* cnt;        // records written
  unsigned int* ticket;           // CTAs done with the current record
  int64_t n_idx, cap;
  int32_t every, es;
};

// Device view of a population-rate monitor: spike count per step of the population rows
// [lo, hi) (the whole population when `whole`), from the spike-history ring.
struct RateMonDev {
  const int32_t* ring_idx;
  const int32_t* ring_cnt;
  int64_t ring_n;                 // ring row stride (padded population size)
  int32_t ring_len, whole;
  int64_t lo, hi;
  int32_t* buf;                   // [cap] spike counts
  int64_t* steps;                 // [cap]
  unsigned long long* cnt;
  int64_t cap;
};

// Device view of the delivery of the two-launch step (pending.cu): one population and its
// additive projections, whose targets are redirected to double-buffered input accumulators.
struct PendingDev {
  PopDev pop;
  ProjDev proj[kMaxProjBatch];
  int32_t n_proj, nd_max;
  void* acc[3];                   // per target variable (v, ge, gi): [2][pop.n] or NULL
  int32_t group;                  // delivery: lanes per work item (4, 8 or 16)
  int32_t pad_group;
};

// Device view of the one-CTA path for small networks (small.cu): one LIF/HH population of at
// most 4096 neurons and its additive projections onto itself.
struct SmallDev {
  PopDev pop;
  ProjDev proj[kMaxProjBatch];
  int32_t proj_target[kMaxProjBatch];   // target variable of each projection's first member
  int32_t n_proj, nd_max;
  int32_t warp_prefix;                  // every projection has <= 64 delays
  int32_t ring_in_smem;                 // the spike-history ring is mirrored in shared memory
  int32_t cluster;                      // CTAs of the one thread-block cluster (1: one CTA)
  int32_t pull;                         // cluster form with the effects gathered per slice
  int64_t slice;                        // neurons per CTA of the cluster (multiple of 4)
  // pull form (synapses without delays or weights of their own): for projection p and rank
  // r of the cluster, the synapses into r's slice grouped by presynaptic neuron: n + 1
  // offsets at pull_off + (p C + r)(n + 1) and slice-local targets at
  // pull_tgt + pull_base[p (C + 1) + r]
  const int32_t* pull_off;
  const uint16_t* pull_tgt;
  const int64_t* pull_base;
  int32_t pull_max_tgt;                 // most synapses (of all projections) into one slice
  int32_t pull_pad;
};

struct Group {
  int kind = 0, dtype = 0, pop = -1;
  int64_t n = 0, offset = 0;
  b2b_lif_params lif{};
  b2b_hh_params hh{};
  double rate = 0;
  std::vector<int32_t> sg_idx;
  std::vector<int64_t> sg_step;
  int64_t sg_period = 0;                      // steps; 0: no repetition
  std::vector<std::vector<uint8_t>> staged;   // per var host bytes staged before finalize
  int64_t mon_cap = 0;
  b2b_mlp* surr = nullptr;                    // gating surrogate (HH float32), or none
  double surr_tol = 0;
  int32_t surr_judge = 1;
  // TimedArray input (b2b_timedarray): values row-major [ta_rows][ta_cols], row of step ts
  // = min(ts * ta_mul / ta_div, ta_rows - 1)
  std::vector<double> ta;
  int64_t ta_rows = 0, ta_cols = 0, ta_mul = 1, ta_div = 1;
  std::vector<PoissonIn> pins;                // PoissonInputs (b2b_poisson_input)
  // generated model (b2b_group_model): its shared object, launcher and requirements
  void* model_dl = nullptr;
  ModelLaunchFn model_launch = nullptr;
  b2b_model_info minfo{};
  double model_refractory = 0;
};

struct Pop {
  int kind = 0, dtype = 0;
  int64_t n = 0;
  std::vector<int> groups;
  PopDev dev{};
  void* params_dev = nullptr;
  int32_t* vec_group_dev = nullptr;
  std::vector<void*> allocs;
  int64_t rng_steps = 0;          // rows held by the uniform buffer
  void* rng_buf = nullptr;
  void* rng_normal_buf = nullptr; // generated models: normal numbers [steps][n_normal][n]
  ModelLaunchFn model_launch = nullptr;   // generated model (one group per population)
  b2b_model_info minfo{};
  bool late_reset = false;
  bool inputs = false;            // some group has a TimedArray or PoissonInput input
  int max_delay = 0;
  // gating surrogate of a float32 HH population (surrogate.cu), or none
  const void* surr_img = nullptr;
  unsigned long long* surr_cnt = nullptr;     // [0] neuron-updates, [1] exact fallbacks
  float surr_tol = 0.f;
  int32_t surr_judge = 1;
  // launch shape chosen by b2b_autotune (0: the built-in heuristic)
  int32_t tune_e = 0;             // neurons per thread, 1 or 4
  int32_t tune_block = 0;         // threads per CTA, 128 or 256
  int32_t tune_ctas = 0;          // surrogate kernel: CTAs per SM
};

// Launch shape of one additive delivery launch (b2b_autotune; 0: built-in heuristic).
struct AddTune {
  int32_t grid = 0;               // CTAs per projection
  int32_t group = 0;              // lanes per work item: 8, 16 or 32
  int32_t cluster = 0;            // 1: accumulate in the distributed shared memory of
                                  // thread-block clusters, then flush (propagate.cu)
};

struct StateMon {  // one StateMonitor (b2b_statemon)
  int gid = -1, var = 0, every = 1;
  std::vector<int64_t> idx;       // group-local
  int64_t cap = 0;
  StateMonDev dev{};
};

struct RateMon {  // one PopulationRateMonitor (b2b_ratemon)
  int gid = -1;
  int64_t cap = 0;
  RateMonDev dev{};
};

struct Syn {  // one user-level Synapses object
  int pre_gid = -1, post_gid = -1, target_var = 0, effect = 0;
  int64_t n = 0;
  std::vector<int32_t> i, j, delay;          // host input (empty for generated)
  std::vector<uint8_t> w;                    // host weights (dtype of target) or empty
  double w_scalar = 0;
  int32_t delay_scalar = 0;
  b2b_stdp_params stdp{};
  bool generated = false;
  double p = 0; int32_t gdmin = 0, gdmax = 0; uint64_t gseed = 0;
  int proj = -1;
  int64_t base = 0;                          // first position inside the projection
  int32_t dmin = 0, dmax = 0;
  int64_t* inv = nullptr;                    // input index -> position (host-given synapses)
  int32_t pre_lo = 0, pre_hi = 0;            // presynaptic subgroup (group-local)
};

struct Proj {
  int src_pop = -1, dst_pop = -1, target_var = 0, effect = 0, dtype = 0;
  bool multi_target = false;                 // members add into different variables
  std::vector<int> members;                  // Syn ids, sorted by source range
  int32_t dmin = 0, dmax = 0;
  int64_t n_syn = 0;
  int64_t max_bundle = 0, max_post_bundle = 0;
  ProjDev dev{};
  int64_t* off = nullptr;
  int32_t* post = nullptr;
  void* w = nullptr;
  std::vector<void*> allocs;
  int32_t* rec_buf = nullptr;                // STDP: record of each synapse, post-grouped order
  // A projection retired by b2b_syn_set_delays: it only delivers the spikes sent before the
  // change (dev.src_hi) and is dropped once the last of them has arrived (after this step).
  // Retired projections follow the live ones in b2b_net::projs and belong to no Synapses.
  int64_t retire_after = -1;
  uint8_t var_mask = 0;                      // bit v: some member adds into variable v
  int64_t dst_n = 0;                         // padded size of the target population
};

}  // namespace b2b

namespace b2b {
struct Snapshot {
  bool valid = false;
  int64_t ts = 0;
  unsigned long long rng_offset = 0;
  std::vector<void*> buffers;      // device copies, one per entry of the state list
};
}  // namespace b2b

struct b2b_net {
  b2b_config cfg{};
  std::vector<b2b::Snapshot> snapshots;
  unsigned long long rng_offset = 0;       // uniforms drawn so far from the cuRAND stream
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bool finalized = false;
  int64_t ts = 0;                          // next step to simulate
  int64_t* d_clock = nullptr;              // device copy of ts at chunk start
  int32_t* d_status = nullptr;
  curandGenerator_t gen = nullptr;
  std::vector<b2b::Group> groups;
  std::vector<b2b::Pop> pops;
  std::vector<b2b::Syn> syns;
  std::vector<b2b::Proj> projs;
  std::vector<std::vector<const b2b::Proj*>> add_batches;  // additive projections per launch
  int32_t n_pins = 0;                      // PoissonInputs added (their Philox stream ids)
  std::vector<b2b::AddTune> add_tune;      // launch shape per add batch (b2b_autotune)
  std::vector<b2b::StateMon> smons;        // state monitors, recorded at the start of a step
  std::vector<b2b::RateMon> rmons;         // rate monitors, recorded at the end of a step
  b2b::StateMonDev* d_smons = nullptr;     // device copies of smons[].dev / rmons[].dev
  b2b::RateMonDev* d_rmons = nullptr;
  int64_t smon_max_idx = 0;                // largest recorded index count
  std::vector<void*> mon_allocs;
  bool small = false;                      // the small-network path runs every step (small.cu)
  bool small_ok = false;                   // the net allows that path (sdev is built)
  // the pull form's connectivity on the host (offsets by presynaptic neuron, targets), and
  // its per-slice device copy for the current cluster size
  bool pull_ok = false;
  std::vector<std::vector<int64_t>> pull_host_off;   // per projection
  std::vector<std::vector<int32_t>> pull_host_post;
  void* pull_buf = nullptr;
  // pinned host staging of spike-monitor reads (b2b_spikemon_fetch)
  void* fetch_pinned = nullptr;
  size_t fetch_pinned_bytes = 0;
  b2b::SmallDev sdev{};
  bool two_launch = false;                 // the step as two concurrent launches (pending.cu)
  bool two_launch_ok = false;              // the net allows them (their buffers exist)
  // the step as two concurrent launches: the delivery into pdev's accumulators (on a second
  // stream, pending_grid CTAs) and the update through fold_dev, ordered by events
  b2b::PendingDev pdev{};
  b2b::PopDev fold_dev{};                  // the population's view whose update folds acc in
  int pending_grid = 0;
  // the same two halves as one grid per step on the net's stream (neuron.cu), the delivery
  // with one_launch_grid CTAs after the update's; only where two_launch_ok
  bool one_launch = false;
  bool one_launch_ok = false;
  int one_launch_grid = 0;
  bool one_launch_chained = false;         // programmatic dependent launch between steps
  cudaStream_t stream2 = nullptr;
  // per-step form with several populations: populations 1.. update on streams of their own,
  // forked from and joined to the net's stream every step (the updates are independent)
  std::vector<cudaStream_t> pop_streams;
  cudaEvent_t ev_pop_fork = nullptr;
  std::vector<cudaEvent_t> ev_pop_join;
  cudaEvent_t ev_n = nullptr, ev_d[2] = {nullptr, nullptr};
  std::vector<void*> pending_allocs;
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  // b2b_profile_graph: while set, enqueue_steps records prof_ev[(k * prof_sites + site) * 2]
  // before and [.. + 1] after every launch site of step k (event-record nodes when captured)
  cudaEvent_t* prof_ev = nullptr;
  int prof_sites = 0;
  int64_t launches = 0;
  int64_t graph_nodes = 0;
  int64_t last_chunk_steps = 0;
  std::string err;
  std::vector<b2b_hines*> hines;
};

// Kernel launch entry points (implemented in the .cu files, called by api.cu).
namespace b2b {
cudaError_t launch_pop_step(const Pop& pop, const int64_t* clock, int k, double dt,
                            int32_t* status, cudaStream_t s);
// The same with another device view of the population (its fold buffers set).
cudaError_t launch_pop_step_dev(const Pop& pop, const PopDev& dev, const int64_t* clock, int k,
                                double dt, int32_t* status, cudaStream_t s);
cudaError_t launch_pop_late_reset(const Pop& pop, const int64_t* clock, int k,
                                  cudaStream_t s);
cudaError_t launch_proj_pre(const Proj& pr, const int64_t* clock, int k, double dt,
                            int32_t* status, cudaStream_t s);
cudaError_t launch_proj_post(const Proj& pr, const int64_t* clock, int k, double dt,
                             int32_t* status, cudaStream_t s);
// One launch for n (<= kMaxProjBatch) additive projections of equal dtype / weight mode.
cudaError_t launch_proj_add_batch(const Proj* const* prs, int n, const int64_t* clock, int k,
                                  cudaStream_t s, const AddTune* tune = nullptr);
// Whether such a launch can accumulate in thread-block clusters (AddTune::cluster).
bool add_batch_cluster_capable(const Proj* const* prs, int n);
cudaError_t launch_tick(int64_t* clock, int steps, cudaStream_t s);
// All state monitors (start of step k of the chunk) / all rate monitors (end of the step).
cudaError_t launch_statemon(const StateMonDev* d_mons, int n_mons, int64_t max_idx,
                            const int64_t* clock, int k, int32_t* status, cudaStream_t s);
cudaError_t launch_ratemon(const RateMonDev* d_mons, int n_mons, const int64_t* clock, int k,
                           int32_t* status, cudaStream_t s);
// COBAHH step of a population with a gating surrogate attached (surrogate.cu).
cudaError_t launch_hh_surrogate(const Pop& pop, const int64_t* clock, int k, double dt,
                                int32_t* status, cudaStream_t s);
// (v, m, h, n) rows of neurons [off, off + n) of a float32 HH population.
cudaError_t launch_hh_sample(const Pop& pop, int64_t off, int64_t n, float* dev_x,
                             cudaStream_t s);
// Packed device image and device ordinal of a surrogate network.
const void* mlp_image(const b2b_mlp* m);
int mlp_device(const b2b_mlp* m);
// Small networks (small.cu): `steps` steps of the net in one one-CTA launch.
size_t small_smem(const SmallDev& D, int kind, int dtype);
// Shared memory of one CTA of the small path's cluster forms.
size_t small_cluster_smem(const SmallDev& D, int kind, int dtype);
// Whether the cluster form of the small-network path (D.cluster CTAs of D.slice neurons) can
// be launched on the current device.
bool small_cluster_possible(const SmallDev& D, int kind, int dtype);
cudaError_t launch_small(const SmallDev& D, int kind, int dtype, const int64_t* clock,
                         int steps, double dt, int32_t* status, cudaStream_t s);
// The two-launch step (pending.cu): the delivery into the pending input of the step, and the
// fold of the pending input at the end of a chunk.
cudaError_t launch_pending_delivery(const PendingDev& F, int dtype, int grid,
                                    const int64_t* clock, int k, cudaStream_t s);
// The step as one launch (neuron.cu): the update's CTAs, then deliver_ctas delivering CTAs
// (counted in CTAs of kBlock threads); chained: with programmatic dependent launch on the
// previous launch of the stream.
bool one_launch_supported(const Pop& pop, const PendingDev& F);
cudaError_t launch_one_launch_step(const Pop& pop, const PopDev& U, const PendingDev& F,
                                   int deliver_ctas, bool chained, const int64_t* clock, int k,
                                   double dt, int32_t* status, cudaStream_t s);
cudaError_t launch_fold_pending(const PendingDev& F, int dtype, const int64_t* clock, int k_last,
                                cudaStream_t s);
}  // namespace b2b
