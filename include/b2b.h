/*
 * b2b.h — C ABI of libb2b, the B200 (sm_100a) simulation backend that replaces the
 * per-code-object CUDA kernels which brian2cuda generates for a Brian2 network.
 *
 * brian2cuda renders one kernel plus one host launcher `_run_<codeobject>()` per Brian2
 * code object and calls them from `Network::run` (brian2cuda/templates/network.cu:40-137).
 * libb2b replaces that generated hot path with a handful of fused, hand-written kernels
 * that own the state of the whole network.  The generated host code (or ctypes) builds a
 * network once through this header and then advances it with b2b_run().
 *
 * Conventions
 *   - Every entry point returns b2b_status.  Nothing calls exit(); the message of the last
 *     failure is kept per network (b2b_last_error).  The reference prints and exits
 *     instead (brian2cuda/brianlib/cuda_utils.h:77-132).
 *   - Plain C types only: pointers, sizes, int32/int64/double.  Arrays passed in are host
 *     pointers unless the name says `dev`.
 *   - One b2b_net per host thread; nets are independent of each other.
 *   - All device work of a net runs on one CUDA stream (the caller's, or one the net owns).
 *     b2b_run() is asynchronous; b2b_sync() waits and reports device-side status.
 *   - Time: t = timestep * dt, timestep an int64 (brian2cuda/brianlib/clocks.h:33-37).
 *     Delays are integer numbers of steps; Brian2 rounds a delay in seconds to steps as
 *     (int)(delay/dt + 0.5) (brian2cuda/templates/synapses_push_spikes.cu:375).
 */
#ifndef B2B_H
#define B2B_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define B2B_ABI_VERSION 1

/* ---- status codes ---------------------------------------------------------------- */
typedef int32_t b2b_status;
enum {
  B2B_OK = 0,
  B2B_ERR_INVALID_ARG = 1,    /* bad argument (NULL, size, unknown enum, index range)  */
  B2B_ERR_OOM = 2,            /* device or host allocation failed                      */
  B2B_ERR_QUEUE_OVERFLOW = 3, /* a fixed-capacity device buffer (monitor) overflowed   */
  B2B_ERR_TIMEOUT = 4,        /* a bounded device-side wait gave up                    */
  B2B_ERR_CUDA = 5,           /* a CUDA runtime / cuRAND call failed                   */
  B2B_ERR_STATE = 6,          /* call not valid now (e.g. adding groups after finalize)*/
  B2B_ERR_UNSUPPORTED = 7,    /* combination not implemented                           */
  B2B_ERR_INDEX = 8           /* out-of-range index found in input or by a checked kernel */
};

typedef struct b2b_net b2b_net;

/* Numeric type of a group's state (Brian2's core.default_float_dtype). */
enum { B2B_F32 = 1, B2B_F64 = 2 };

/* Network flags (b2b_config.flags). */
enum {
  B2B_NET_NO_GRAPH = 1,   /* launch every step eagerly instead of replaying CUDA graphs */
  B2B_NET_CHECKED = 2,    /* every launch site a kernel of its own (no small-network path,
                             no two-launch form unless B2B_NET_TWO_LAUNCH is also set), so a
                             fault or a device status names one launch; input indices are
                             checked on the host in every mode (B2B_ERR_INDEX)           */
  B2B_NET_RESET_BEFORE_SYNAPSES = 4, /* schedule start, groups, thresholds, resets, synapses,
                                        end (Brian2 prefs core.network.default_schedule);
                                        default: resets after synapses                   */
  B2B_NET_TWO_LAUNCH = 8,      /* run every step as two concurrent launches (neuron update, and
                             the delivery of spikes of earlier steps into a double-buffered
                             input) whenever the net allows it: one LIF/HH population, additive
                             synapses onto ge/gi only, all delays >= 1 step, no state or rate
                             monitor.  Without this flag or B2B_NET_PER_STEP such a net uses
                             the two launches when its population has at most 2^18 neurons,
                             and b2b_autotune picks the faster of the two forms             */
  B2B_NET_SMALL = 16,     /* run a small network (one LIF/HH population of <= 4096 neurons
                             with additive synapses onto itself) on the small-network path:
                             every step of a chunk in one launch, the state in shared
                             memory, as one CTA or as one thread-block cluster of 8 or 16
                             CTAs (b2b_autotune site kind 14), the cluster either pushing
                             the effects or, for synapses without delays or weights of their
                             own, gathering them at the targets.  Without this flag such a
                             net runs the per-step kernels until b2b_autotune measures the
                             path faster (CUBA 4000: 4.3 against 5.4 us per step)         */
  B2B_NET_PER_STEP = 32,  /* always the per-step kernels (one launch per population, then
                             the delivery), never the two concurrent launches             */
  B2B_NET_ONE_LAUNCH = 64 /* where the net allows the two concurrent launches (see
                             B2B_NET_TWO_LAUNCH) and every projection has at most 64
                             delays, no TimedArray or PoissonInput drives the population and
                             no gating surrogate is attached: run both halves of a step as
                             one launch (the update's CTAs, then the delivery's), one launch
                             boundary per step on the net's stream; b2b_autotune otherwise
                             picks among the three forms                                  */
};

typedef struct {
  double dt;                /* time step in seconds                                      */
  int32_t device;           /* CUDA device ordinal                                       */
  int32_t steps_per_graph;  /* steps captured per CUDA graph; 0 selects 50               */
  uint64_t seed;            /* seed of the cuRAND Philox generator and of b2b_connect    */
  void* stream;             /* cudaStream_t to run on, or NULL: the net creates its own  */
  int32_t flags;            /* B2B_NET_* bits                                            */
  int32_t reserved;
} b2b_config;

/* Replaces the generated `brian_start()` / `_init_arrays()` pair
 * (brian2cuda/templates/run.cu:15-32, objects.cu:340-489). */
b2b_status b2b_create(const b2b_config* cfg, b2b_net** out);
/* Replaces `brian_end()` / `_dealloc_arrays()` (run.cu:34-38, objects.cu:654-726). */
b2b_status b2b_destroy(b2b_net* net);
/* Copies the message of the net's last failure into buf (always NUL-terminated). */
b2b_status b2b_last_error(const b2b_net* net, char* buf, size_t len);
const char* b2b_status_string(b2b_status s);
int32_t b2b_abi_version(void);

/* ---- neuron groups ---------------------------------------------------------------- */
/* Linear leaky integrate-and-fire, integrated with the exact (closed-form) propagator
 * Brian2's `method='exact'` emits for
 *     dv/dt  = (El - v + ke*ge + ki*gi)/taum   [(unless refractory)]
 *     dge/dt = -ge/taue,  dgi/dt = -gi/taui
 * CUBA (examples/cuba.py:125-132): ke = ki = 1.  The STDP benchmark neuron
 * (brian2cuda/tests/features/speed.py:629-640): ke = Ee - vr, ki = 0.
 * taum = +inf gives a non-leaky `v : 1` group.  Threshold `v > Vt` (and not_refractory
 * when refractory > 0), reset `v = Vr` (brian2cuda/templates/threshold.cu:19-45,
 * reset.cu:3-27).  Replaces the stateupdater/thresholder/resetter code objects. */
typedef struct {
  double El, taum, taue, taui, ke, ki;   /* volts, seconds, dimensionless factors */
  double Vt, Vr, refractory;             /* refractory in seconds; 0 = none         */
  int32_t has_threshold, has_reset, unless_refractory, reserved;
} b2b_lif_params;

/* Conductance-based Hodgkin-Huxley (examples/cobahh.py:159-180), integrated with the
 * exponential-Euler scheme of Brian2's `method='exponential_euler'`.  Threshold
 * `v > Vthr` and not_refractory; no reset.  All SI units. */
typedef struct {
  double Cm, gl, El, EK, ENa, gNa, gK, VT, Ee, Ei, taue, taui, Vthr, refractory;
} b2b_hh_params;

b2b_status b2b_group_lif(b2b_net* net, int64_t n, int32_t dtype, const b2b_lif_params* p,
                         int32_t* gid);
b2b_status b2b_group_hh(b2b_net* net, int64_t n, int32_t dtype, const b2b_hh_params* p,
                        int32_t* gid);
/* PoissonGroup: neuron i spikes in a step when u_i < rate*dt, u_i one uniform from the
 * net's cuRAND buffer (brian2cuda/templates/rand.cu:340-463 fills the same kind of
 * per-step bulk buffer; `_rand` reads it in place, cuda_generator.py:938-943). */
b2b_status b2b_group_poisson(b2b_net* net, int64_t n, int32_t dtype, double rate_hz,
                             int32_t* gid);
/* SpikeGeneratorGroup: neuron idx[k] spikes at step[k]
 * (brian2cuda/templates/spikegenerator.cu:41-148). */
b2b_status b2b_group_spikegen(b2b_net* net, int64_t n, int64_t n_spikes, const int32_t* idx,
                              const int64_t* step, int32_t* gid);
/* SpikeGeneratorGroup(..., period=P): the entries repeat every period_steps steps (step ts
 * emits the entries of step ts mod period_steps; every entry must lie inside the period),
 * brian2cuda/templates/spikegenerator.cu:42-49, 88-96.  0 = no repetition.  Before
 * b2b_finalize; the SpikeGeneratorGroups of one net share one period. */
b2b_status b2b_spikegen_period(b2b_net* net, int32_t gid, int64_t period_steps);

/* TimedArray input of a LIF, HH or Poisson group (replaces the function brian2cuda/timedarray.py:
 * 10-58 generates for `ta(t)` / `ta(t, i)` in the group's equations).  values[rows][cols]
 * (row-major float64, converted to the group's dtype) are sampled every dt_array seconds and
 * held over each interval: step ts reads row floor(ts * dt / dt_array), clamped to rows - 1.
 * cols = 1: one value for the whole group; cols = n: one per neuron.  The value I enters
 *     LIF: dv/dt = (El + I - v + ke*ge + ki*gi)/taum     (I in volts)
 *     HH:  Cm dv/dt = ... + I                           (I in amperes)
 *     PoissonGroup: the rate in Hz, replacing the group's constant rate
 *                   (PoissonGroup(N, rates='ta(t)')): spike when u < I dt
 * dt_array must be an integer multiple or an integer fraction of the net's dt (aligned time
 * grids).  Before b2b_finalize; a later call for the same group replaces the array.  Not
 * combinable with the gating surrogate. */
b2b_status b2b_timedarray(b2b_net* net, int32_t gid, const double* values, int64_t rows,
                          int64_t cols, double dt_array);

/* PoissonInput of a LIF or HH group (Brian2's PoissonInput, whose per-step draw
 * brian2cuda implements as a BinomialFunction, brian2cuda/binomial.py:12-121): every step,
 * in the synapses slot (after the threshold, before the reset of the default schedule), each
 * neuron of the group adds weight * X to variable var (B2B_VAR_V, _GE or _GI), X ~
 * Binomial(n_inputs, rate_hz * dt) drawn independently per neuron and step from the net's
 * seed.  The draw is exact inversion for every n * p (the reference switches to a normal
 * approximation above n p = 5).  At most two per group; before b2b_finalize.  *pid receives
 * the input's index (its random stream).  Not combinable with the gating surrogate; a net
 * with one runs the per-step or two-launch form, not the small-network path. */
b2b_status b2b_poisson_input(b2b_net* net, int32_t gid, int32_t var, int64_t n_inputs,
                             double rate_hz, double weight, int32_t* pid);

/* ---- generated neuron models -------------------------------------------------------------
 * A neuron model that no hand-written kernel integrates: the device plugin generates its
 * state update, threshold and reset from the Brian2 equations as CUDA device code around this
 * library's kernel template (brian2cuda_b200/csrc/model_kernel.cuh), compiles it with nvcc
 * into a shared object (the role of the code objects brian2cuda generates and compiles,
 * brian2cuda/cuda_generator.py:281-461, templates/common_group.cu:108-160), and the net loads
 * it and launches it every step like its own kernels.  The object exports
 *   int32_t b2b_model_info_v1(b2b_model_info* info);
 *   int32_t b2b_model_launch_v1(const void* pop, const int64_t* clock, int32_t k, double dt,
 *                               int32_t* status, void* stream, int32_t dtype, int32_t phase);
 * (phase 0: update, threshold and, unless deferred, reset of every neuron; phase 1: the
 * deferred reset of the step's spiking neurons).  State variable k of the model is variable
 * index k of this API (B2B_VAR_V = 0 ... B2B_VAR_N = 5); LASTSPIKE and NOT_REFRACTORY as for the
 * other groups.  Synapses may add into variables 0, 1 and 2. */
#define B2B_MODEL_ABI 1
#define B2B_MODEL_MAX_VARS 6
typedef struct {
  int32_t abi;           /* B2B_MODEL_ABI                                                    */
  int32_t n_vars;        /* state variables, 1 .. B2B_MODEL_MAX_VARS                         */
  int32_t n_normal;      /* standard normal numbers per neuron and step (noise xi, randn())  */
  int32_t n_uniform;     /* uniform numbers per neuron and step (rand())                     */
  int32_t reset_mask;    /* bit k set: the reset writes variable k                           */
  int32_t has_threshold;
} b2b_model_info;

/* Adds a group of n neurons integrated by the generated model in the shared object at
 * module_path (its variables in dtype; refractory in seconds, 0 = none: while refractory the
 * threshold is off and the model's `(unless refractory)` variables are held).  The numbers the
 * model draws come from the net's cuRAND generator, one bulk buffer per chunk of steps
 * (templates/rand.cu:340-463 fills the same kind of buffer), readable with
 * b2b_rng_normals_get / b2b_rng_uniforms_get.  Before b2b_finalize. */
b2b_status b2b_group_model(b2b_net* net, int64_t n, int32_t dtype, const char* module_path,
                           double refractory, int32_t* gid);
/* Normal numbers the last b2b_run chunk drew for generated-model group gid: `steps` rows of
 * n_normal x (group size) values, row k = step k of the chunk, draw d of neuron i at
 * [k][d * size + i]. */
b2b_status b2b_rng_normals_get(b2b_net* net, int32_t gid, void* host, int64_t steps,
                               int64_t n);

/* State variables of a group.  Values are in the group's dtype; NOT_REFRACTORY is uint8. */
enum {
  B2B_VAR_V = 0, B2B_VAR_GE = 1, B2B_VAR_GI = 2, B2B_VAR_M = 3, B2B_VAR_H = 4, B2B_VAR_N = 5,
  B2B_VAR_LASTSPIKE = 6, B2B_VAR_NOT_REFRACTORY = 7
};
/* Host <-> device copies of one variable (replaces the generated H2D/D2H copies of
 * `_array_<group>_<var>`, brian2cuda/device.py:558-658, objects.cu:522-641).
 * Before b2b_finalize the values are staged on the host. */
b2b_status b2b_state_set(b2b_net* net, int32_t gid, int32_t var, const void* host, int64_t n);
b2b_status b2b_state_get(b2b_net* net, int32_t gid, int32_t var, void* host, int64_t n);
/* Device pointer to a group's variable (after b2b_finalize); the net owns the memory. */
b2b_status b2b_state_ptr(b2b_net* net, int32_t gid, int32_t var, void** dev, int64_t* n);

/* ---- synapses ---------------------------------------------------------------------- */
/* Effect of a presynaptic spike (the on_pre code of a Synapses object). */
enum {
  B2B_EFFECT_ADD = 1,   /* target_var[post] += w                                         */
  B2B_EFFECT_STDP = 2   /* event-driven additive STDP with on_pre and on_post pathways   */
};

/* examples/stdp.py:125-186, brian2cuda/tests/features/speed.py:627-663:
 *   on_pre : Apre, Apost decayed to t; target += w (if pre_adds_weight);
 *            Apre += dApre; w = clip(w + Apost, wmin, wmax); lastupdate = t
 *   on_post: Apre, Apost decayed to t; Apost += dApost; w = clip(w + Apre, wmin, wmax);
 *            lastupdate = t                                                          */
typedef struct {
  double taupre, taupost, dApre, dApost, wmin, wmax;
  int32_t pre_adds_weight, reserved;
} b2b_stdp_params;

/* Adds a Synapses object with explicit connectivity (i -> j, group-local indices).
 * w: per-synapse weights in the target group's dtype, or NULL to use w_scalar.
 * delay_steps: per-synapse delays in steps, or NULL to use delay_scalar.
 * stdp: required for B2B_EFFECT_STDP (w then is the initial weight), else NULL.
 * Replaces connectivity preprocessing `_before_run_<pathway>_push_spikes`
 * (brian2cuda/templates/synapses_push_spikes.cu:171-993). */
b2b_status b2b_synapses(b2b_net* net, int32_t pre_gid, int32_t post_gid, int32_t target_var,
                        int32_t effect, int64_t n_syn, const int32_t* i, const int32_t* j,
                        const void* w, double w_scalar, const int32_t* delay_steps,
                        int32_t delay_scalar, const b2b_stdp_params* stdp, int32_t* sid);

/* Adds a Synapses object whose connectivity is generated on the GPU: every pair (i, j),
 * i in the presynaptic subgroup [pre_lo, pre_hi) of pre_gid (Brian2's `P[lo:hi]`), j in
 * post_gid, is connected with probability p (Brian2 `connect(p=...)`); each synapse gets a
 * delay drawn uniformly from the integers [dmin, dmax] and weight w.  Generation is
 * counter-based (Philox-4x32-10 keyed by seed and the group-local (i, j)), so it is
 * reproducible and independent of launch shape.  Replaces host-serial synapse creation
 * (brian2cuda/templates/synapses_create_generator.cu:164-271).  Synapses are numbered in
 * (i, delay, j) order; i and j are group-local. */
b2b_status b2b_synapses_random(b2b_net* net, int32_t pre_gid, int32_t pre_lo, int32_t pre_hi,
                               int32_t post_gid, int32_t target_var, double p, int32_t dmin,
                               int32_t dmax, double w, uint64_t seed, int32_t* sid);

/* The same generator as b2b_synapses_random, writing into caller-provided device arrays and
 * allocating nothing (no counterpart in the reference).  For callers that cannot allocate
 * device memory: applications whose device memory belongs to a pooling allocator (PyTorch's
 * caching allocator, RMM) that a library cudaMalloc would bypass, and host loops that cannot
 * afford the implicit device synchronisation of cudaMalloc/cudaFree.
 * Rows i in [pre_lo, pre_hi) (at most B2B_STATIC_MAX_ROWS of them, else B2B_ERR_INVALID_ARG)
 * against posts j in [0, n_post); synapses are written in (i, j) order as int32 i, j and delay
 * (steps, uniform on [dmin, dmax]) up to `capacity` entries; *n_syn receives the number
 * generated, and B2B_ERR_QUEUE_OVERFLOW is returned when it exceeds capacity.  Runs on
 * `stream` of `device` and waits for it.  Scratch: a file-scope device array of
 * B2B_STATIC_MAX_ROWS + 1 int64 (8 MiB) that every GPU loading the library holds until exit;
 * its device address is looked up (cudaGetSymbolAddress) on the first call on each device, and
 * again on the first call after the device's context changed (cudaDeviceReset), so make that
 * first call before any stream capture.  A CUDA error already pending on entry is returned as
 * B2B_ERR_CUDA without being cleared.  All calls share the array: calls that overlap on the
 * GPU race. */
#define B2B_STATIC_MAX_ROWS (1 << 20)
b2b_status b2b_connect_random_static(int32_t device, void* stream, int32_t pre_lo,
                                     int32_t pre_hi, int32_t n_post, double p, int32_t dmin,
                                     int32_t dmax, uint64_t seed, int32_t* dev_i, int32_t* dev_j,
                                     int32_t* dev_delay, int64_t capacity, int64_t* n_syn);

/* Measures the ceiling of the additive delivery on `device`: the rate of scattered float32
 * atomic additions (one per synaptic event, as brian2cuda's effect kernels do with atomicAdd,
 * brian2cuda/templates/synapses.cu:117-162; no counterpart as a measurement) into an array of
 * n_targets floats, at indices uniform over the array.  *loaded_per_s: every event's index
 * loaded from an n_events-entry int32 array in device memory first (the delivery's form);
 * *hashed_per_s: the index computed in registers (the atomics alone); *dsmem_per_s: the
 * same additions into the distributed shared memory of 8-CTA thread-block clusters (the
 * array split into one slice per CTA; 0 when a slice exceeds 200 KB).  Best of `reps` timed
 * launches after one warm-up each.  Allocates and frees its own buffers; runs on `stream`. */
b2b_status b2b_atomic_rate(int32_t device, void* stream, int64_t n_targets, int64_t n_events,
                           int32_t reps, double* loaded_per_s, double* hashed_per_s,
                           double* dsmem_per_s);

/* Self-tests of two device-side building blocks (no counterpart in the reference):
 * b2b_wait_selftest runs one CTA that waits with the kernels' bounded mbarrier wait (`polls`
 * polls, at most 2^20) on a barrier that nothing arrives on (arrive = 0: the wait gives up,
 * the CTA records B2B_ERR_TIMEOUT in the status word and returns) or that thread 0 arrives on
 * first (arrive = 1: B2B_OK); *device_status receives the status word.
 * b2b_recip_selftest evaluates the multicompartment solver's reciprocal (the reciprocal
 * unit's approximation refined by two Newton-Raphson steps) at x[0..n) into y. */
b2b_status b2b_wait_selftest(int32_t device, void* stream, uint32_t polls, int32_t arrive,
                             int32_t* device_status);
b2b_status b2b_recip_selftest(int32_t device, const double* x, double* y, int64_t n);

/* Synapse variables. I, J, DELAY are int32; the others use the target group's dtype. */
enum {
  B2B_SYN_I = 0, B2B_SYN_J = 1, B2B_SYN_DELAY = 2, B2B_SYN_W = 3, B2B_SYN_APRE = 4,
  B2B_SYN_APOST = 5, B2B_SYN_LASTUPDATE = 6
};
b2b_status b2b_syn_count(b2b_net* net, int32_t sid, int64_t* n);
/* New per-synapse delays (steps, in the order the synapses were given) of additive Synapses
 * object sid between runs (Brian2's `S.delay = ...` before another run()).  As in Brian2,
 * spikes already sent keep the delay they were sent with and spikes from the next step on
 * use the new ones (brian2cuda/tests/test_network_multiple_runs.py:110-156): the projection
 * as built stays, delivering only spikes of earlier steps, until its last one has arrived;
 * the rebuilt one delivers the later spikes.  A population's spike-history ring grows when
 * the new delays need it (snapshots taken before become unusable).  Not for connectivity
 * generated on the GPU, STDP synapses or a net made to run the small-network path with
 * B2B_NET_SMALL (B2B_ERR_UNSUPPORTED); a net on that path by the autotuner's choice goes
 * back to the per-step kernels. */
b2b_status b2b_syn_set_delays(b2b_net* net, int32_t sid, const int32_t* delay_steps,
                              int64_t n);
/* Reads a synapse variable in the order the synapses were given (after b2b_finalize). */
b2b_status b2b_syn_get(b2b_net* net, int32_t sid, int32_t var, void* host, int64_t n);

/* Number of outgoing synapses of every neuron of group gid over all Synapses objects that
 * leave it (Brian2's Synapses.N_outgoing summed over pathways; brian2cuda computes it on the
 * host in synapses_create templates); host receives n = group size int32 counts. */
b2b_status b2b_out_degree(b2b_net* net, int32_t gid, int32_t* host, int64_t n);

/* ---- lifecycle ---------------------------------------------------------------------- */
/* Lays out state, builds the delay-sorted connectivity on the GPU and captures the step
 * graphs (the role of the generated before_run code). */
b2b_status b2b_finalize(b2b_net* net);
/* Advances the network by n_steps time steps; asynchronous (replaces the per-step loop
 * of Network::run, brian2cuda/templates/network.cu:40-137, with no host sync per step). */
b2b_status b2b_run(b2b_net* net, int64_t n_steps);
/* Waits for the net's stream; *device_status receives the device status word
 * (B2B_OK, B2B_ERR_QUEUE_OVERFLOW, B2B_ERR_INDEX, ...). */
b2b_status b2b_sync(b2b_net* net, int32_t* device_status);
/* Device-side checkpoint of the net's dynamic state in `slot` (>= 0): state variables and
 * spike-history rings of every population, synaptic variables of STDP projections, the
 * clock and the cuRAND offset (spike monitors keep recording).  b2b_restore copies the
 * checkpoint back.  Brian2's Network.store()/restore(); the reference's device raises
 * NotImplementedError for both (brian2cuda/device.py:1783-1789). */
b2b_status b2b_store(b2b_net* net, int32_t slot);
b2b_status b2b_restore(b2b_net* net, int32_t slot);
/* Current time step (the next step to simulate) and time in seconds. */
b2b_status b2b_time(b2b_net* net, int64_t* timestep, double* t);
/* Number of kernels launched so far by b2b_run (eager launches plus graph kernel nodes). */
b2b_status b2b_kernel_launches(b2b_net* net, int64_t* n);
/* How b2b_run advances the net (after b2b_finalize): *mode = 1 for every step as two
 * concurrent launches (B2B_NET_TWO_LAUNCH, or chosen automatically), 3 for both halves of
 * every step as one launch (B2B_NET_ONE_LAUNCH or the autotuner), 2 for a small network run by
 * one CTA or one thread-block cluster per chunk of steps, 0 for per-step kernels replayed from
 * CUDA graphs. */
b2b_status b2b_run_mode(b2b_net* net, int32_t* mode);
/* Profiling run (the role of run(..., profile=True): per-code-object device timing,
 * brian2cuda/templates/common_group.cu:170-174, 328-337, objects.cu:603-629).  Advances the
 * network by n_steps with eager launches, timing every launch with a CUDA event pair on the
 * net's stream, and returns per launch site the mean device time of one launch in ms.
 * Sites, in order: the state monitors (kind 9, one launch for all, when there are any), one
 * per population (kind 1), one per launch of additive on_pre delivery (kind 6: the additive
 * projections that share a kernel variant are delivered by one launch, with its tuned
 * shape), one per STDP projection's on_pre delivery (kind 2), one per STDP projection's
 * on_post delivery (kind 3), one per population with a deferred reset (kind 4), the rate
 * monitors (kind 10, one launch for all); or, when the net runs every step as two
 * concurrent launches (b2b_run_mode 1), the delivery into the pending input (kind 5) and the
 * neuron update folding it in (kind 1), launched one after the other; or, in the one-launch
 * form (b2b_run_mode 3), the one kernel of the step (kind 13); or, for a small network
 * run by one CTA or cluster (b2b_run_mode 2), that kernel advancing one step (kind 7).  *n_sites receives the number
 * of sites (<= cap filled). */
b2b_status b2b_profile(b2b_net* net, int64_t n_steps, double* mean_ms, int32_t* site_kind,
                       int32_t cap, int32_t* n_sites);
/* The same sites timed where b2b_run runs them: the step graph of steps_per_graph steps is
 * captured with a CUDA event-record node before and after every launch site of every step,
 * and replayed to advance the net by n_steps (a multiple of steps_per_graph).  mean_ms[k]
 * receives site k's mean device time per simulated step inside the replayed graphs (in the
 * two-launch form the two sites overlap in time; the one-CTA path's one launch covers a whole
 * graph of steps), *step_ms the mean time of one whole step (replays timed by an event pair on
 * the net's stream; the added event nodes are part of it).  Same site order and kinds as
 * b2b_profile.  The profiling variant of the per-code-object timers of run(profile=True)
 * (brian2cuda/templates/common_group.cu:170-174), which synchronise after every launch. */
b2b_status b2b_profile_graph(b2b_net* net, int64_t n_steps, double* mean_ms, int32_t* site_kind,
                             int32_t cap, int32_t* n_sites, double* step_ms);

/* Autotuner (no counterpart in the reference, which picks launch shapes from fixed rules,
 * brian2cuda/device.py:383-394): launch site by launch site it times candidate launch shapes
 * on the net's own current state and keeps the fastest.  A trial restores the same
 * checkpoint, captures the step graph with the candidate shape and times `trial_steps` whole
 * steps run as b2b_run runs them (graph replays), so a shape is judged by the step time it
 * gives.  Populations: neurons per thread (1, 2 or 4) x threads per CTA (128 or 256), or, with a
 * gating surrogate, CTAs per SM (2..6); additive delivery launches: lanes per work item
 * (2, 4, 8, 16, 32) x CTAs (1/2, 1, 2, 4, 8 per SM); STDP projections: the order of the synapse
 * records (0 synapse order, 1 grouped by postsynaptic neuron, where on_post reads contiguous
 * records; the live records and every snapshot are permuted together, and b2b_syn_get reads
 * through the order); a net that can run every step as two concurrent launches: the pending
 * delivery's lanes per item x CTAs (kind 5), then the form itself (kind 11: choice_a 2 one
 * launch per step holding both halves, with choice_b delivering CTAs (of 256 threads; 0: the
 * built-in 1.5 per SM) after the update's, 3 the
 * same with each step's launch chained to the previous one by programmatic dependent launch;
 * 1 two launches; 0 the per-step kernels).  Afterwards the state, clock and monitor counts are as before the call,
 * and the next b2b_run captures its graph with the chosen shapes.  A candidate must be 2 % faster than the best so far (starting from the built-in
 * rule) to be chosen.  A choice of 0 means the built-in rule won.  The trials should cover a
 * representative stretch of the run (bursts included). */
typedef struct {
  int32_t site_kind;     /* 1 population, 6 additive delivery launch, 8 STDP records,
                            5 pending delivery of the two-launch step, 11 step form
                            (0 per-step kernels, 1 two launches, 2 one launch,
                            3 one launch chained),
                            12 additive delivery launch accumulated in the distributed
                            shared memory of 8-CTA thread-block clusters (choice_a 1) or
                            with one global atomic per event (0); float32 launches onto
                            one population of at most ~400k padded elements;
                            14 the small-network path: choice_a 0 not used, 1 one CTA,
                            8 or 16 a cluster of that many CTAs, choice_b 1 gathering the
                            effects at the targets                                        */
  int32_t site_index;    /* population / delivery launch / projection index              */
  int32_t choice_a;      /* neurons per thread (surrogate: CTAs per SM) / lanes per item /
                            record order / step form                                      */
  int32_t choice_b;      /* threads per CTA / CTAs                                       */
  double best_ms;        /* mean device time of one whole step with the chosen shape     */
  double default_ms;     /* the same with the built-in rule                              */
} b2b_tune_result;
b2b_status b2b_autotune(b2b_net* net, int32_t trial_steps, b2b_tune_result* out, int32_t cap,
                        int32_t* n_out);
/* Applies launch shapes an earlier b2b_autotune chose (of a net built the same way), so that
 * a run can reuse a tuning without repeating its trials. */
b2b_status b2b_tune_apply(b2b_net* net, const b2b_tune_result* r, int32_t n);

/* ---- monitors and inspection ---------------------------------------------------------- */
/* Records every spike of group gid as (step, index) into a device buffer of `capacity`
 * entries (replaces brian2cuda/templates/spikemonitor.cu without per-step resizes).
 * Must be called before b2b_finalize. */
b2b_status b2b_spikemon(b2b_net* net, int32_t gid, int64_t capacity);
/* Copies recorded spikes sorted by (step, index); *n receives the total recorded. */
b2b_status b2b_spikemon_get(b2b_net* net, int32_t gid, int64_t* n, int32_t* idx,
                            int64_t* step, int64_t cap);
/* The same for the subgroup G[lo:hi] (SpikeMonitor(G[lo:hi]), indices relative to lo, as
 * brian2cuda/tests/test_monitor.py:23-45 expects), read from the group's monitor. */
b2b_status b2b_spikemon_get_range(b2b_net* net, int32_t gid, int64_t lo, int64_t hi,
                                  int64_t* n, int32_t* idx, int64_t* step, int64_t cap);
/* Incremental readout: *total receives the number of entries the monitor of gid's
 * population has recorded; entries [start, min(total, start + cap)) are copied in recording
 * order, keeping those of group gid (group-local index), and *n receives how many were kept.
 * Lets a caller drain new spikes after every run chunk (the role of the per-run result
 * files, brian2cuda/templates/objects.cu:522-641).  The copy goes through a page-locked host
 * buffer kept by the net (grown to the largest read, freed by b2b_destroy). */
b2b_status b2b_spikemon_fetch(b2b_net* net, int32_t gid, int64_t start, int64_t* total,
                              int64_t* n, int32_t* idx, int64_t* step, int64_t cap);
/* b2b_spikemon_fetch without the group filter: entries of every monitored group of gid's
 * population, with population indices (group k's neuron i is b2b_group_offset(k) + i). */
b2b_status b2b_spikemon_fetch_population(b2b_net* net, int32_t gid, int64_t start,
                                         int64_t* total, int64_t* n, int32_t* idx,
                                         int64_t* step, int64_t cap);
/* Index of group gid's first neuron in its population (after b2b_finalize). */
b2b_status b2b_group_offset(b2b_net* net, int32_t gid, int64_t* offset);
/* StateMonitor (brian2cuda/templates/statemonitor.cu; Brian2's StateMonitor(G, var,
 * record=idx, dt=every*dt), when='start'): at the start of every step divisible by `every`,
 * before any group updates, copies variable `var` of neurons idx[0..n) of group gid into a
 * device buffer of `capacity` records.  A record is one value per recorded neuron, in the
 * variable's type (the group's dtype; uint8 for NOT_REFRACTORY).  Records beyond the
 * capacity are dropped and b2b_sync reports B2B_ERR_QUEUE_OVERFLOW.  Recording appends
 * across b2b_run calls and b2b_restore, as the spike monitor does.  Before b2b_finalize;
 * *mid receives the monitor's index. */
b2b_status b2b_statemon(b2b_net* net, int32_t gid, int32_t var, const int64_t* idx, int64_t n,
                        int32_t every, int64_t capacity, int32_t* mid);
/* *n_records receives the number of records so far; the first min(*n_records, cap) are
 * copied: their steps (int64, may be NULL) and values (cap x n elements, may be NULL). */
b2b_status b2b_statemon_get(b2b_net* net, int32_t mid, int64_t* n_records, int64_t* steps,
                            void* values, int64_t cap);
/* PopulationRateMonitor (templates/ratemonitor.cu): the number of spikes of group gid in
 * every step, recorded at the end of the step (after synaptic effects and resets, Brian2's
 * when='end'); the rate is count / (group size * dt).  Capacity and overflow as for
 * b2b_statemon.  Before b2b_finalize. */
b2b_status b2b_ratemon(b2b_net* net, int32_t gid, int64_t capacity, int32_t* mid);
b2b_status b2b_ratemon_get(b2b_net* net, int32_t mid, int64_t* n_records, int64_t* steps,
                           int32_t* counts, int64_t cap);
/* Spikes of group gid in the last completed step, sorted ascending (the canonical form of
 * the spikespace, brian2cuda/templates/objects.cu:458-479). */
b2b_status b2b_spikes_last(b2b_net* net, int32_t gid, int64_t* n, int32_t* idx, int64_t cap);
/* Delay-queue contents of Synapses object sid: every (pre, delay) bundle still due after
 * the last completed step, with the step offset (1..max_delay) at which it is due, sorted
 * by (offset, pre, delay).  Matches the content of the CudaSpikeQueue slots
 * (brian2cuda/brianlib/spikequeue.h:432-516) with one post block. */
b2b_status b2b_queue_get(b2b_net* net, int32_t sid, int64_t* n, int32_t* offset,
                         int32_t* pre, int32_t* delay, int64_t cap);
/* Uniform numbers the last b2b_run chunk consumed for Poisson group gid: `steps` rows of
 * n values each (row k = step k of the chunk); for a generated-model group, rows of
 * n_uniform x (group size) values laid out as for b2b_rng_normals_get. */
b2b_status b2b_rng_uniforms_get(b2b_net* net, int32_t gid, void* host, int64_t steps,
                                int64_t n);

/* ---- multicompartment (SpatialNeuron) batch ------------------------------------------------ */
/* A batch of independent multicompartment HH neurons, each a tree of sections (branches) of
 * cylindrical compartments.  One b2b_hines_step advances all neurons by one dt with the
 * Hines scheme brian2cuda runs in five kernels (brian2cuda/templates/spatialstateupdate.cu:
 * 18-93 host matrix preparation, 108-113 channels, 128-192 per-section Thomas solves with
 * three right-hand sides, 202-307 coupling solve, 316-351 combine, 359-387 currents).
 *
 * Layout per neuron b: compartments [comp_off[b], comp_off[b+1]) of the flat arrays;
 * sections [sec_off[b], sec_off[b+1]); section s covers neuron-local compartments
 * [sec_start[s], sec_end[s]) and hangs off section sec_parent[s] (-1 for the root section,
 * which must be the first one of its neuron and start at compartment 0).
 * Geometry: diameter and length (m) per compartment.  Ri in ohm*m, Cm in F/m^2. */
typedef struct {
  double Cm, Ri, El, EK, ENa, gl, gNa, gK;   /* F/m^2, ohm*m, V, S/m^2 */
  double Vthr;                                /* soma spike threshold (V), upward crossing */
  int32_t channel_dtype;                      /* B2B_F32 or B2B_F64 gating variables;
                                                 the cable solve is always float64      */
  int32_t reserved;
} b2b_hines_params;

typedef struct b2b_hines b2b_hines;
b2b_status b2b_hines_create(b2b_net* net, int32_t n_neurons, const int64_t* comp_off,
                            const int32_t* sec_off, const int32_t* sec_start,
                            const int32_t* sec_end, const int32_t* sec_parent,
                            const double* diameter, const double* length,
                            const b2b_hines_params* p, b2b_hines** out);
/* Per-neuron current injected into compartment 0 (A); NULL clears it. */
b2b_status b2b_hines_set_current(b2b_hines* h, const double* soma_current);
/* vars: 0 = v (f64), 1 = m, 2 = h, 3 = n (channel_dtype), 4 = Ic (f64, capacitive current
 * density of the last step, A/m^2).  Channels follow the Hodgkin-Huxley 1952 rate functions
 * of examples/compartmental/hh_with_spikes_cuda.py:31-50 (v measured from rest). */
b2b_status b2b_hines_state_set(b2b_hines* h, int32_t var, const void* host, int64_t n);
b2b_status b2b_hines_state_get(b2b_hines* h, int32_t var, void* host, int64_t n);
/* Advances all neurons by n_steps; soma spike counts accumulate per neuron. */
b2b_status b2b_hines_run(b2b_hines* h, int64_t n_steps);
b2b_status b2b_hines_spike_counts(b2b_hines* h, int32_t* host, int32_t n);
b2b_status b2b_hines_destroy(b2b_hines* h);

/* ---- gating surrogate (no counterpart in the reference) ------------------------------------
 * A 4 -> 64 -> 64 -> 3 perceptron (tanh hidden units, BF16 weights and activations, FP32
 * accumulation on the sm_100a tensor cores) that predicts the exponential-Euler step of the
 * COBAHH gating variables (m, h, n) over one dt from (v, m, h, n).  brian2cuda integrates the
 * gates only with the code Brian2 generates for method='exponential_euler'
 * (examples/cobahh.py:159-180); that integrator stays here as the fallback and the judge.
 * Samples are float32 rows (v, m, h, n) in SI units; targets and predictions are rows
 * (m', h', n').  The network computes y = W3 tanh(W2 tanh(W1 xh + b1) + b2) + b3 with
 * xh = ((v, m, h, n) - in_shift) * in_scale and predicts clip(x + out_scale * y, 0, 1). */
typedef struct b2b_mlp b2b_mlp;
#define B2B_MLP_NPARAMS 4675  /* W1[64][4], b1[64], W2[64][64], b2[64], W3[3][64], b3[3] */

/* Creates a network with seeded Xavier-uniform weights and zero biases on `device`; all its
 * work runs on `stream` (a cudaStream_t, or NULL for one it owns). */
b2b_status b2b_mlp_create(int32_t device, void* stream, uint64_t seed, b2b_mlp** out);
b2b_status b2b_mlp_destroy(b2b_mlp* m);
/* fp32 master parameters, B2B_MLP_NPARAMS values in the order above. */
b2b_status b2b_mlp_params_get(b2b_mlp* m, float* host, int64_t n);
b2b_status b2b_mlp_params_set(b2b_mlp* m, const float* host, int64_t n);
/* Input/output scaling: 11 floats in_shift[4], in_scale[4], out_scale[3]. */
b2b_status b2b_mlp_scaling_get(b2b_mlp* m, float* host11);
b2b_status b2b_mlp_scaling_set(b2b_mlp* m, const float* host11);
/* Sets the scaling from a dataset: v's range maps to [-1, 1], m/h/n's [0, 1] to [-1, 1],
 * out_scale = the largest |target - input| per gate. */
b2b_status b2b_mlp_fit_scaling(b2b_mlp* m, const float* dev_x, const float* dev_t, int64_t n);
/* n predictions (raw = 0: clip(x + out_scale * y, 0, 1); raw = 1: the outputs y). */
b2b_status b2b_mlp_forward(b2b_mlp* m, const float* dev_x, float* dev_out, int64_t n,
                           int32_t raw);
/* Gradient of the mean loss mean_s sum_o (y_o - (t_o - x_o)/out_scale_o)^2 over the n
 * samples, in parameter order, and the loss itself. */
b2b_status b2b_mlp_grad(b2b_mlp* m, const float* dev_x, const float* dev_t, int64_t n,
                        float* host_grad, int64_t n_grad, double* loss);
/* Adam (beta 0.9/0.999) with a cosine-decayed learning rate over `epochs` passes of
 * minibatches of `batch` samples (a multiple of 128) in a fresh pseudo-random order per
 * epoch; loss_per_epoch (epochs values, or NULL) receives each epoch's mean loss. */
b2b_status b2b_mlp_train(b2b_mlp* m, const float* dev_x, const float* dev_t, int64_t n,
                         int32_t epochs, int32_t batch, double lr, double* loss_per_epoch);
/* Training targets: the exact exponential-Euler gating step (the kernel's own integrator) of
 * n samples for the COBAHH parameters p and time step dt, on `stream` of `device`. */
b2b_status b2b_hh_gating_exact(const b2b_hh_params* p, double dt, const float* dev_x,
                               float* dev_t, int64_t n, int32_t device, void* stream);
/* Copies (v, m, h, n) of the first n neurons of float32 HH group gid into dev_x (device rows
 * of 4 floats), on the net's stream: trajectory samples for training. */
b2b_status b2b_hh_gating_sample(b2b_net* net, int32_t gid, float* dev_x, int64_t n);
/* Steps every HH group of gid's (float32) population with the surrogate's gating update
 * (before b2b_finalize; m must outlive the net).  A neuron is re-stepped exactly when its v
 * lies outside the range the scaling maps to [-1, 1], or, with judge = 1, when a predicted
 * gate differs from the exact update by more than tol. */
b2b_status b2b_group_hh_surrogate(b2b_net* net, int32_t gid, b2b_mlp* m, double tol,
                                  int32_t judge);
/* Neuron-updates made with the surrogate attached and how many of them fell back. */
b2b_status b2b_surrogate_stats(b2b_net* net, int32_t gid, int64_t* updates, int64_t* fallbacks);

#ifdef __cplusplus
}
#endif
#endif /* B2B_H */
